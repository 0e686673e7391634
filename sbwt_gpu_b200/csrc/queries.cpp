// queries.cpp -- query files in and answer text out (host side of the CLI),
// plus the thread-local error buffer of the C ABI.
#include <charconv>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "sbwt_gpu.h"
#include "common.h"

namespace sbwt {

namespace {
thread_local char g_error[1024] = "";
}

int set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error, sizeof g_error, fmt, ap);
    va_end(ap);
    return 1;
}

void clear_error() { g_error[0] = '\0'; }

const char *last_error() { return g_error; }

}  // namespace sbwt

extern "C" const char *sbwt_last_error(void) { return sbwt::last_error(); }

// ----------------------------------------------------------- query reader
//
// KmerSearch::read_file (include/epicseq/kmer_search.hpp:319-342): every line
// that does not start with '>' is one read and all its bytes but the '\n' are
// letters (non-ACGT bytes pack as A); empty lines give no read.  The
// reference's getline arithmetic drops the last letter of a final line that
// has no '\n' (letters_in_row = gcount - 1, :328); here that letter is kept.
// FASTQ (no reference counterpart: the reference reads FASTA only): a file
// whose first byte is '@' is read as four-line records (@header, sequence,
// '+' line, qualities), the sequence line being the read.
//
// The reader streams: the file is read in blocks of kReadBlock bytes and
// handed out in batches of whole reads, so a caller can search one batch
// while the next is being read (the reference reads the whole file with
// getline before anything else runs).

namespace sbwt {
namespace {

constexpr size_t kReadBlock = 16u << 20;

// Growable malloc'd array (the batches hand their buffers to the caller,
// who frees them with sbwt_queries_free).
template <class T>
bool reserve(T *&p, uint64_t &cap, uint64_t need) {
    if (need <= cap) return true;
    uint64_t c = cap ? cap : 1024;
    while (c < need) c *= 2;
    T *q = (T *)std::realloc(p, c * sizeof(T));
    if (!q) return false;
    p = q;
    cap = c;
    return true;
}

}  // namespace
}  // namespace sbwt

struct sbwt_reader {
    FILE *f = nullptr;
    std::string path;
    uint32_t k = 31;
    int fastq = -1;                // -1 not known yet (first byte), 0 FASTA / plain lines, 1 FASTQ
    std::vector<uint8_t> buf;      // file bytes not parsed yet: [pos, end)
    size_t pos = 0, end = 0;
    bool eof = false;
    uint64_t line = 0;             // lines consumed (a FASTQ record is lines 4r .. 4r+3)
    uint64_t size_hint = 0;        // file size (letters capacity of a whole-file batch)
};

namespace sbwt {
namespace {

// Refills the buffer; false at the end of the file with nothing left.
int refill(sbwt_reader *rd) {
    if (rd->eof) return 0;
    if (rd->pos > 0) {  // keep the unparsed tail at the front
        std::memmove(rd->buf.data(), rd->buf.data() + rd->pos, rd->end - rd->pos);
        rd->end -= rd->pos;
        rd->pos = 0;
    }
    if (rd->buf.size() - rd->end < kReadBlock) rd->buf.resize(rd->end + kReadBlock);
    const size_t got = std::fread(rd->buf.data() + rd->end, 1, rd->buf.size() - rd->end, rd->f);
    if (got == 0) {
        if (std::ferror(rd->f)) return set_error("The file %s can not be read.", rd->path.c_str());
        rd->eof = true;
    }
    rd->end += got;
    return 0;
}

}  // namespace
}  // namespace sbwt

extern "C" int sbwt_reader_open(const char *path, uint32_t k, sbwt_reader **out) {
    sbwt::clear_error();
    if (!out || !path) return sbwt::set_error("NULL argument");
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) return sbwt::set_error("The file %s can not be opened.", path);
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size <= 0) {
        std::fclose(f);
        return sbwt::set_error("The size of the file %s is too small to contain any data.", path);  // :421-426
    }
    sbwt_reader *rd = new (std::nothrow) sbwt_reader();
    if (!rd) {
        std::fclose(f);
        return sbwt::set_error("out of host memory");
    }
    rd->f = f;
    rd->path = path;
    rd->k = k;
    rd->size_hint = (uint64_t)size;
    *out = rd;
    return 0;
}

extern "C" void sbwt_reader_close(sbwt_reader *rd) {
    if (!rd) return;
    if (rd->f) std::fclose(rd->f);
    delete rd;
}

extern "C" int sbwt_reader_next(sbwt_reader *rd, uint64_t max_letters, sbwt_queries *out) {
    sbwt::clear_error();
    if (!rd || !out) return sbwt::set_error("NULL argument");
    std::memset(out, 0, sizeof(*out));
    uint8_t *letters = nullptr;
    uint64_t *starts = nullptr;
    uint64_t cap_l = 0, cap_r = 0, nl = 0, nr = 0, nk = 0;
    if (max_letters == 0) max_letters = ~0ull;
    if (!sbwt::reserve(letters, cap_l, std::min<uint64_t>(rd->size_hint, max_letters) + 64) ||
        !sbwt::reserve(starts, cap_r, 1024)) {
        std::free(letters);
        std::free(starts);
        return sbwt::set_error("out of host memory");
    }
    int rc = 0;
    for (;;) {
        uint8_t *b = rd->buf.data();
        const uint8_t *nlp = rd->pos < rd->end ? (const uint8_t *)std::memchr(b + rd->pos, '\n', rd->end - rd->pos)
                                               : nullptr;
        if (!nlp && !rd->eof) {
            if ((rc = sbwt::refill(rd)) != 0) break;
            continue;
        }
        if (!nlp && rd->pos >= rd->end) break;  // end of file
        const size_t lend = nlp ? (size_t)(nlp - b) : rd->end;
        const uint8_t *ln = b + rd->pos;
        const size_t len = lend - rd->pos;
        if (rd->fastq < 0) rd->fastq = (len > 0 && ln[0] == '@') ? 1 : 0;
        bool is_read = false;
        if (rd->fastq == 1) {
            const uint64_t role = rd->line & 3u;
            if (role == 0 && len == 0 && !nlp) {  // a final empty line
                rd->pos = lend;
                continue;
            }
            if ((role == 0 && (len == 0 || ln[0] != '@')) || (role == 2 && (len == 0 || ln[0] != '+'))) {
                rc = sbwt::set_error("The file %s is not FASTQ: line %llu should start with '%c'.", rd->path.c_str(),
                                     (unsigned long long)rd->line + 1, role == 0 ? '@' : '+');
                break;
            }
            is_read = role == 1;
        } else {
            is_read = len > 0 && ln[0] != '>';
        }
        if (is_read && nr > 0 && nl + len > max_letters) break;  // the batch is full: this read starts the next
        if (is_read) {
            if (!sbwt::reserve(letters, cap_l, nl + len + 64) || !sbwt::reserve(starts, cap_r, nr + 2)) {
                rc = sbwt::set_error("out of host memory");
                break;
            }
            starts[nr++] = nl;
            std::memcpy(letters + nl, ln, len);
            nl += len;
            if (len >= rd->k) nk += len - rd->k + 1;
        }
        rd->line++;
        rd->pos = nlp ? lend + 1 : lend;
    }
    if (rc == 0 && rd->fastq == 1 && rd->eof && rd->pos >= rd->end && (rd->line & 3u) != 0)
        rc = sbwt::set_error("The file %s ends inside a FASTQ record.", rd->path.c_str());
    if (rc) {
        std::free(letters);
        std::free(starts);
        return rc;
    }
    std::memset(letters + nl, 0, 32);  // add_paddings, kmer_search.hpp:292-301
    starts[nr] = nl;
    out->letters = letters;
    out->n_letters = nl;
    out->row_starts = starts;
    out->n_rows = nr;
    out->n_kmers = nk;
    return 0;
}

extern "C" int sbwt_queries_read(const char *path, uint32_t k, sbwt_queries *out) {
    sbwt::clear_error();
    if (!out) return sbwt::set_error("out is NULL");
    std::memset(out, 0, sizeof(*out));
    sbwt_reader *rd = nullptr;
    if (sbwt_reader_open(path, k, &rd)) return 1;
    const int rc = sbwt_reader_next(rd, 0, out);
    sbwt_reader_close(rd);
    return rc;
}

extern "C" void sbwt_queries_free(sbwt_queries *q) {
    if (!q) return;
    std::free(q->letters);
    std::free(q->row_starts);
    std::memset(q, 0, sizeof(*q));
}

// ResultsPersister::save_results_to_file (include/epicseq/results_persister.hpp:
// 82-95): per read, each answer as a signed int64 and one space, then '\n'.
// A read shorter than k gives an empty line (the reference's row length
// underflows there, :85).
extern "C" int64_t sbwt_format_answers(const uint64_t *row_starts, uint64_t n_rows, uint32_t k,
                                       const uint64_t *answers, char *out, uint64_t cap) {
    sbwt::clear_error();
    uint64_t o = 0, j = 0;
    char tmp[24];
    for (uint64_t r = 0; r < n_rows; r++) {
        const uint64_t len = row_starts[r + 1] - row_starts[r];
        const uint64_t cnt = len >= k ? len - k + 1 : 0;
        for (uint64_t i = 0; i < cnt; i++) {
            const auto res = std::to_chars(tmp, tmp + sizeof tmp, (long long)(int64_t)answers[j++]);
            const uint64_t m = (uint64_t)(res.ptr - tmp);
            if (out) {
                if (o + m + 1 > cap) return -1;
                std::memcpy(out + o, tmp, m);
                out[o + m] = ' ';
            }
            o += m + 1;
        }
        if (out) {
            if (o + 1 > cap) return -1;
            out[o] = '\n';
        }
        o += 1;
    }
    return (int64_t)o;
}

extern "C" int sbwt_queries_read_many(const char *const *paths, int n_files, uint32_t k, sbwt_queries *out,
                                      uint64_t *file_rows) {
    sbwt::clear_error();
    if (!out || !paths || n_files <= 0) return sbwt::set_error("sbwt_queries_read_many: bad arguments");
    std::memset(out, 0, sizeof(*out));
    std::vector<sbwt_queries> parts((size_t)n_files);
    std::vector<int> rc((size_t)n_files, 0);
    std::vector<std::string> err((size_t)n_files);
#pragma omp parallel for schedule(dynamic, 1)
    for (int f = 0; f < n_files; f++) {
        rc[f] = sbwt_queries_read(paths[f], k, &parts[f]);
        if (rc[f]) err[f] = sbwt::last_error();
    }
    int bad = -1;
    for (int f = 0; f < n_files; f++)
        if (rc[f] && bad < 0) bad = f;
    uint64_t nl = 0, nr = 0, nk = 0;
    for (int f = 0; f < n_files && bad < 0; f++) {
        nl += parts[f].n_letters;
        nr += parts[f].n_rows;
        nk += parts[f].n_kmers;
    }
    uint8_t *letters = bad < 0 ? (uint8_t *)std::malloc(nl + 64) : nullptr;
    uint64_t *rows = bad < 0 ? (uint64_t *)std::malloc((nr + 1) * sizeof(uint64_t)) : nullptr;
    if (bad < 0 && (!letters || !rows)) bad = n_files;
    if (bad >= 0) {
        for (auto &q : parts) sbwt_queries_free(&q);
        std::free(letters);
        std::free(rows);
        if (bad == n_files) return sbwt::set_error("out of host memory");
        return sbwt::set_error("%s", err[(size_t)bad].c_str());
    }
    uint64_t lo = 0, ro = 0;
    for (int f = 0; f < n_files; f++) {
        const sbwt_queries &q = parts[f];
        if (file_rows) file_rows[f] = ro;
        if (q.n_letters) std::memcpy(letters + lo, q.letters, q.n_letters);
        for (uint64_t r = 0; r < q.n_rows; r++) rows[ro + r] = q.row_starts[r] + lo;
        lo += q.n_letters;
        ro += q.n_rows;
        sbwt_queries_free(&parts[f]);
    }
    if (file_rows) file_rows[n_files] = ro;
    rows[nr] = nl;
    std::memset(letters + nl, 0, 32);
    out->letters = letters;
    out->n_letters = nl;
    out->row_starts = rows;
    out->n_rows = nr;
    out->n_kmers = nk;
    return 0;
}
