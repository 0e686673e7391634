// cli.cpp -- `sbwt_search`, the command-line drop-in for the reference's
// build/search program (src/search.cpp:9-26).  Flags keep the reference's
// names and ranges (include/parameters.hpp:13-37, 79-297); answers go to
// stdout in the reference's format (include/epicseq/results_persister.hpp:
// 82-95), timings to stderr.
//
//   sbwt_search --file-a=A --file-c=C --file-g=G --file-t=T --file-queries=Q
//               [--k=30] [--k-presearch=12] [--without-presearch]
//               [--bits-in-superblock=1024] [--rank-structure=poppy|cum-poppy]
//               [--with-shuffles] [--threads-per-block=N]
//               [--device-set-limit-presearch=64] [--device-set-limit-search=64]
//               [--do-not-store-results] [--layout=lines|poppy]
//               [--kmers-per-thread=N] [--threads-per-kmer=1|2|4]
//               [--search-mode=every|skip|stream]
//
// The query file (FASTA, or FASTQ when its first byte is '@') is read by a
// thread of its own in batches of whole reads (sbwt_reader_next) while the
// previous batch is searched, formatted and written, so file reading
// overlaps the search instead of preceding it (the reference reads the whole
// file first, include/epicseq/kmer_search.hpp:319-342).
//
// Differences from the reference: errors return a non-zero exit status
// (the reference always returns 0, src/search.cpp:14-25); --rank-structure=
// flat-poppy, which the reference parses but never implements
// (parameters.hpp:196-200), is rejected; --unified-searches and
// --rank-word-size (unused on the reference's live path) are accepted and
// ignored.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <regex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "sbwt_gpu.h"

namespace {

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void print_help() {
    std::fprintf(stderr,
                 "usage: sbwt_search --file-a=A --file-c=C --file-g=G --file-t=T --file-queries=Q [--k=30]\n"
                 "       [--k-presearch=12 | --without-presearch] [--bits-in-superblock=1024]\n"
                 "       [--rank-structure=poppy|cum-poppy] [--with-shuffles] [--threads-per-block=N]\n"
                 "       [--device-set-limit-presearch=32|64|128] [--device-set-limit-search=32|64|128]\n"
                 "       [--do-not-store-results] [--layout=lines|poppy] [--kmers-per-thread=N]\n"
                 "       [--threads-per-kmer=1|2|4] [--search-mode=every|skip|stream]\n");
}

struct Options {
    std::string a, c, g, t, queries;
    bool with_presearch = true, store = true;
    int limit_presearch = 64, limit_search = 64;
    sbwt_params p;
};

int parse(int argc, char **argv, Options &o) {
    sbwt_params_default(&o.p);
    if (argc == 1 || std::string(argv[1]) == "help") {
        print_help();
        return 2;
    }
    const std::regex sb_re{"^--bits-in-superblock=(256|512|1024|2048|4096)$"};
    const std::regex lp_re{"^--device-set-limit-presearch=(32|64|128)$"};
    const std::regex ls_re{"^--device-set-limit-search=(32|64|128)$"};
    const std::regex k_re{"^--k=([3-9]|([1-2][0-9])|3[0-2])$"};
    const std::regex kp_re{"^--k-presearch=([1-9]|(1[0-5]))$"};
    const std::regex tpb_re{"^--threads-per-block=([0-9][0-9][0-9]?[0-9]?)$"};
    const std::regex kpt_re{"^--kmers-per-thread=([0-8])$"};
    const std::regex tpk_re{"^--threads-per-kmer=(1|2|4)$"};
    std::smatch m;
    for (int i = 1; i < argc; i++) {
        const std::string s = argv[i];
        auto val = [&](const char *prefix) { return s.substr(std::strlen(prefix)); };
        if (s == "--without-presearch") o.with_presearch = false;
        else if (s == "--do-not-store-results") o.store = false;
        else if (s == "--with-shuffles") o.p.with_shuffles = 1;
        else if (s == "--rank-structure=poppy") o.p.rank_structure = SBWT_POPPY;
        else if (s == "--rank-structure=cum-poppy") o.p.rank_structure = SBWT_CUM_POPPY;
        else if (s == "--rank-structure=flat-poppy") {
            std::fprintf(stderr, "The rank structure flat-poppy has no implementation.\n");
            return 1;
        } else if (s == "--unified-searches" || s.rfind("--rank-word-size=", 0) == 0) {
            std::fprintf(stderr, "Ignoring %s.\n", s.c_str());
        } else if (s == "--layout=lines") o.p.layout = SBWT_LAYOUT_LINES;
        else if (s == "--layout=poppy") o.p.layout = SBWT_LAYOUT_POPPY;
        else if (s == "--search-mode=every") o.p.search_mode = SBWT_SEARCH_EVERY_KMER;
        else if (s == "--search-mode=skip") o.p.search_mode = SBWT_SEARCH_SKIP_ABSENT;
        else if (s == "--search-mode=stream") o.p.search_mode = SBWT_SEARCH_STREAM;
        else if (std::regex_match(s, m, sb_re)) o.p.bits_in_superblock = (uint32_t)std::stoul(m[1]);
        else if (std::regex_match(s, m, lp_re)) o.limit_presearch = std::stoi(m[1]);
        else if (std::regex_match(s, m, ls_re)) o.limit_search = std::stoi(m[1]);
        else if (std::regex_match(s, m, k_re)) o.p.k = (uint32_t)std::stoul(m[1]);
        else if (std::regex_match(s, m, kp_re)) o.p.k_presearch = (uint32_t)std::stoul(m[1]);
        else if (std::regex_match(s, m, kpt_re)) o.p.kmers_per_thread = (uint32_t)std::stoul(m[1]);
        else if (std::regex_match(s, m, tpk_re)) o.p.threads_per_kmer = (uint32_t)std::stoul(m[1]);
        else if (std::regex_match(s, m, tpb_re)) {
            const unsigned v = (unsigned)std::stoul(m[1]);
            if (v < 32 || v > 256 || v % 32)  // parameters.hpp:202-212 (our kernels take at most 256)
                std::fprintf(stderr, "Number of threads per block should have been at least 32 and at most 256. "
                                     "We use now the default.\n");
            else
                o.p.threads_per_block = v;
        } else if (s.rfind("--file-a=", 0) == 0) o.a = val("--file-a=");
        else if (s.rfind("--file-c=", 0) == 0) o.c = val("--file-c=");
        else if (s.rfind("--file-g=", 0) == 0) o.g = val("--file-g=");
        else if (s.rfind("--file-t=", 0) == 0) o.t = val("--file-t=");
        else if (s.rfind("--file-queries=", 0) == 0) o.queries = val("--file-queries=");
        else if (s.rfind("--file-answers=", 0) == 0) { /* the reference's legacy checker only */ }
        else std::fprintf(stderr, "Unknown argument %s ignored.\n", s.c_str());
    }
    if (o.with_presearch) {
        if (o.p.k_presearch < 5 || o.p.k_presearch > 13) {  // parameters.hpp:253-265
            std::fprintf(stderr, "The value of the prefix of k-mers to be presearched must be at least 5 and at most 13.\n");
            o.p.k_presearch = 12;
        }
        if (o.p.k_presearch > o.p.k) o.p.k_presearch = o.p.k;
    } else {
        o.p.k_presearch = 0;
    }
    if (o.p.bits_in_superblock == 4096 && o.p.rank_structure != SBWT_POPPY) {  // parameters.hpp:273-277
        std::fprintf(stderr, "Superblock size 4096 bits is supported only in the rank structure version poppy. "
                             "Please choose some other parameters.\n");
        return 1;
    }
    if (o.a.empty() || o.c.empty() || o.g.empty() || o.t.empty() || o.queries.empty()) {
        std::fprintf(stderr, "The four bit vector files and the query file are required.\n");
        print_help();
        return 1;
    }
    return 0;
}

// Searches the reads of q in batches of at most kBatchLetters letters and
// writes the reference's text for them to `out`.  The device buffers persist
// across calls.  The environment variable SBWT_CLI_BATCH_LETTERS sets
// another batch size (also the size of the reader's batches).
uint64_t kBatchLetters = 1ull << 28;

struct Writer {
    uint8_t *d_letters = nullptr;
    uint64_t *d_rows = nullptr, *d_ans = nullptr;
    char *d_text = nullptr, *h_text = nullptr;
    uint64_t cap_l = 0, cap_r = 0, cap_a = 0, cap_t = 0, cap_h = 0;
    std::vector<uint64_t> rows;

    template <class T>
    static bool grow(T *&p, uint64_t &cap, uint64_t need) {
        if (need <= cap) return true;
        cudaFree(p);
        p = nullptr;
        cap = 0;
        if (cudaMalloc((void **)&p, need * sizeof(*p)) != cudaSuccess) return false;
        cap = need;
        return true;
    }

    ~Writer() {
        cudaFree(d_letters);
        cudaFree(d_rows);
        cudaFree(d_ans);
        cudaFree(d_text);
        cudaFreeHost(h_text);
    }

    int run(sbwt_index *ix, const sbwt_queries &q, uint32_t k, FILE *out) {
        uint64_t r0 = 0;
        while (r0 < q.n_rows) {
            // rows [r0, r1): at least one, at most kBatchLetters letters unless one read is longer
            uint64_t r1 = r0 + 1;
            while (r1 < q.n_rows && q.row_starts[r1 + 1] - q.row_starts[r0] <= kBatchLetters) r1++;
            const uint64_t base = q.row_starts[r0], nl = q.row_starts[r1] - base, nr = r1 - r0;
            rows.resize(nr + 1);
            uint64_t nk = 0;
            for (uint64_t r = 0; r <= nr; r++) {
                rows[r] = q.row_starts[r0 + r] - base;
                if (r < nr) {
                    const uint64_t len = q.row_starts[r0 + r + 1] - q.row_starts[r0 + r];
                    nk += len >= k ? len - k + 1 : 0;
                }
            }
            uint64_t bytes = 0;
            if (!grow(d_letters, cap_l, nl + 1) || !grow(d_rows, cap_r, nr + 1) || !grow(d_ans, cap_a, nk + 1))
                return 1;
            if (cudaMemcpy(d_letters, q.letters + base, nl, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(d_rows, rows.data(), (nr + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice) != cudaSuccess)
                return 1;
            if (nk && sbwt_search_reads(ix, d_letters, nl, d_rows, nr, d_ans, nullptr, nk, nullptr)) return 1;
            if (sbwt_format_answers_device(d_rows, nr, k, d_ans, nk, nullptr, 0, &bytes, nullptr) ||
                !grow(d_text, cap_t, bytes + 1))
                return 1;
            if (sbwt_format_answers_device(d_rows, nr, k, d_ans, nk, d_text, cap_t, &bytes, nullptr)) return 1;
            if (bytes + 1 > cap_h) {
                cudaFreeHost(h_text);
                h_text = nullptr;
                cap_h = 0;
                if (cudaMallocHost((void **)&h_text, bytes + 1) != cudaSuccess) return 1;
                cap_h = bytes + 1;
            }
            if (cudaMemcpy(h_text, d_text, bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
                std::fwrite(h_text, 1, bytes, out) != bytes)
                return 1;
            r0 = r1;
        }
        return 0;
    }
};

// Reads the query file's batches on a thread of its own, at most two ahead
// of the consumer.
struct Prefetch {
    sbwt_reader *rd = nullptr;
    uint32_t k = 31;
    std::mutex m;
    std::condition_variable cv;
    std::deque<sbwt_queries> ready;
    bool done = false;
    std::string error;
    double read_ms = 0;  // time the reader thread spent reading
    std::thread th;

    void start() {
        th = std::thread([this] {
            for (;;) {
                {
                    std::unique_lock<std::mutex> lk(m);
                    cv.wait(lk, [this] { return ready.size() < 2 || done; });
                    if (done) return;
                }
                const auto t = std::chrono::steady_clock::now();
                sbwt_queries q;
                const int rc = sbwt_reader_next(rd, kBatchLetters, &q);
                const double ms = ms_since(t);
                std::lock_guard<std::mutex> lk(m);
                read_ms += ms;
                if (rc) error = sbwt_last_error();
                if (rc || q.n_rows == 0) {
                    if (!rc) sbwt_queries_free(&q);
                    done = true;
                    cv.notify_all();
                    return;
                }
                ready.push_back(q);
                cv.notify_all();
            }
        });
    }
    // The next batch, or false at the end (or on an error: see `error`).
    bool next(sbwt_queries &q) {
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [this] { return !ready.empty() || done; });
        if (ready.empty()) return false;
        q = ready.front();
        ready.pop_front();
        cv.notify_all();
        return true;
    }
    void stop() {
        {
            std::lock_guard<std::mutex> lk(m);
            done = true;
            cv.notify_all();
        }
        if (th.joinable()) th.join();
        for (auto &q : ready) sbwt_queries_free(&q);
        ready.clear();
    }
};

}  // namespace

int main(int argc, char **argv) {
    Options o;
    const int prc = parse(argc, argv, o);
    if (prc == 2) return 0;
    if (prc) return 1;
    const auto t_main = std::chrono::steady_clock::now();
    cudaSetDevice(o.p.device);
    cudaFree(nullptr);  // creates the CUDA context here, so that its cost is reported on its own
    std::fprintf(stderr, "%f ms for creating the CUDA context.\n", ms_since(t_main));
    cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, o.limit_presearch);  // presearch.hpp:34-37
    auto t0 = std::chrono::steady_clock::now();
    sbwt_index *ix = nullptr;
    if (sbwt_index_load(o.a.c_str(), o.c.c_str(), o.g.c_str(), o.t.c_str(), &o.p, &ix)) {
        std::fprintf(stderr, "%s\n", sbwt_last_error());
        return 1;
    }
    uint64_t n = 0, C[5];
    sbwt_index_info(ix, &n, C, nullptr, nullptr);
    std::fprintf(stderr, "%f ms for reading the bit vector files, constructing the rank data structures, "
                         "presearching and sending to the device (%llu columns).\n",
                 ms_since(t0), (unsigned long long)n);
    if (o.p.layout == SBWT_LAYOUT_POPPY &&
        sbwt_configure(ix, SBWT_LAYOUT_POPPY, o.p.bits_in_superblock, o.p.rank_structure, o.p.with_shuffles,
                       o.p.kmers_per_thread, o.p.threads_per_kmer, o.p.threads_per_block)) {
        std::fprintf(stderr, "%s\n", sbwt_last_error());
        sbwt_index_free(ix);
        return 1;
    }
    cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, o.limit_search);  // search_caller.hpp:91-96
    if (const char *e = std::getenv("SBWT_CLI_BATCH_LETTERS")) {
        const unsigned long long v = std::strtoull(e, nullptr, 10);
        if (v) kBatchLetters = v;
    }
    auto t1 = std::chrono::steady_clock::now();
    Prefetch pf;
    pf.k = o.p.k;
    if (sbwt_reader_open(o.queries.c_str(), o.p.k, &pf.rd)) {
        std::fprintf(stderr, "%s\n", sbwt_last_error());
        sbwt_index_free(ix);
        return 1;
    }
    pf.start();
    int rc = 0;
    uint64_t n_kmers = 0;
    double wait_ms = 0;
    {
        Writer wr;
        std::vector<uint64_t> answers;
        for (;;) {
            const auto tw = std::chrono::steady_clock::now();
            sbwt_queries q;
            const bool more = pf.next(q);
            wait_ms += ms_since(tw);
            if (!more) break;
            n_kmers += q.n_kmers;
            if (o.store) {
                // letters + offsets to the device, search, text formatted on the device
                // (sbwt_format_answers_device), text back and written in read order
                if (wr.run(ix, q, o.p.k, stdout)) {
                    const char *msg = sbwt_last_error();
                    std::fprintf(stderr, "%s\n", msg && *msg ? msg : cudaGetErrorString(cudaGetLastError()));
                    rc = 1;
                }
            } else {
                answers.resize(q.n_kmers ? q.n_kmers : 1);
                if (sbwt_search_reads_host(ix, q.letters, q.n_letters, q.row_starts, q.n_rows, answers.data(),
                                           q.n_kmers)) {
                    std::fprintf(stderr, "%s\n", sbwt_last_error());
                    rc = 1;
                }
            }
            sbwt_queries_free(&q);
            if (rc) break;
        }
        std::fflush(stdout);
    }
    pf.stop();
    sbwt_reader_close(pf.rd);
    if (!rc && !pf.error.empty()) {
        std::fprintf(stderr, "%s\n", pf.error.c_str());
        rc = 1;
    }
    const double ms_total = ms_since(t1);
    std::fprintf(stderr, "Reading the query file: %f ms (on its own thread, overlapped with the search; %f ms "
                         "waiting for it).\n", pf.read_ms, wait_ms);
    std::fprintf(stderr, "Search (host to device, pack, search%s, device to host): %f ms.\n",
                 o.store ? ", answer text, writing" : "", ms_total - wait_ms);
    std::fprintf(stderr, "Number of k-mers queried: %llu\n", (unsigned long long)n_kmers);
    if (n_kmers) std::fprintf(stderr, "Total per query: %f ns.\n", ms_total * 1e6 / (double)n_kmers);
    if (!o.store) std::fprintf(stderr, "The results are not stored to the file.\n");
    sbwt_index_free(ix);
    std::fprintf(stderr, "%f ms in total, from the start of main.\n", ms_since(t_main));
    return rc;
}
