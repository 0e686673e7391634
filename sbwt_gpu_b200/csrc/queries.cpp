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

// KmerSearch::read_file (include/epicseq/kmer_search.hpp:319-342): every line
// that does not start with '>' is one read and all its bytes but the '\n' are
// letters (non-ACGT bytes pack as A); empty lines give no read.  The
// reference's getline arithmetic drops the last letter of a final line that
// has no '\n' (letters_in_row = gcount - 1, :328); here that letter is kept.
extern "C" int sbwt_queries_read(const char *path, uint32_t k, sbwt_queries *out) {
    sbwt::clear_error();
    if (!out) return sbwt::set_error("out is NULL");
    std::memset(out, 0, sizeof(*out));
    FILE *f = std::fopen(path, "rb");
    if (!f) return sbwt::set_error("The file %s can not be opened.", path);
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size <= 0) {
        std::fclose(f);
        return sbwt::set_error("The size of the file %s is too small to contain any data.", path);  // :421-426
    }
    uint8_t *raw = (uint8_t *)std::malloc((size_t)size + 64);
    if (!raw) {
        std::fclose(f);
        return sbwt::set_error("Allocating memory for the query file fails.");
    }
    const size_t got = std::fread(raw, 1, (size_t)size, f);
    std::fclose(f);
    if (got != (size_t)size) {
        std::free(raw);
        return sbwt::set_error("The file %s can not be read.", path);
    }
    // compact in place: letters never move right of their source bytes
    std::vector<uint64_t> starts;
    starts.reserve((size_t)size / 100 + 16);
    uint64_t nl = 0, nk = 0;
    size_t pos = 0;
    const size_t n = (size_t)size;
    while (pos < n) {
        const uint8_t *nlp = (const uint8_t *)std::memchr(raw + pos, '\n', n - pos);
        const size_t end = nlp ? (size_t)(nlp - raw) : n;
        const size_t len = end - pos;
        if (len > 0 && raw[pos] != '>') {
            starts.push_back(nl);
            std::memmove(raw + nl, raw + pos, len);
            nl += len;
            if (len >= k) nk += len - k + 1;
        }
        pos = end + 1;
    }
    std::memset(raw + nl, 0, 32);  // add_paddings, kmer_search.hpp:292-301
    const uint64_t rows = starts.size();
    uint64_t *rs = (uint64_t *)std::malloc((rows + 1) * sizeof(uint64_t));
    if (!rs) {
        std::free(raw);
        return sbwt::set_error("out of host memory");
    }
    if (rows) std::memcpy(rs, starts.data(), rows * sizeof(uint64_t));
    rs[rows] = nl;
    out->letters = raw;
    out->n_letters = nl;
    out->row_starts = rs;
    out->n_rows = rows;
    out->n_kmers = nk;
    return 0;
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
