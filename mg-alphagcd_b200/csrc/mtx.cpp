// mtx.cpp -- Matrix Market loader with the reference's rules
// (init_data_from_mtx, src/mmio/mmio_wrapper.cu:76-295):
//   * banner containing "general" -> general path, "symmetric" -> symmetric
//     path (:97-102); '%' lines are skipped (:104-106); the size line is
//     "rows cols nnz" (:114);
//   * every entry line is "<row> <col>[ <value>]" with 1-based ids; the
//     fields are found the way the reference does it (atoi at the line start,
//     then at one past the first ' ', the value one past the next ' ');
//   * symmetric: weight forced to 1.0 (:141-142), off-diagonal entries
//     mirrored (:163-170), rows hold their file-order entries followed by the
//     mirrored ones (stable sort by row, :181);
//   * general: entries with col >= row skipped (:239), weight = atof of the
//     third field or 1.0 (:243-250), each kept entry stored in both rows in
//     file order (the reference fills rows with 80 OpenMP threads, :271-288,
//     so its in-row order is unspecified).
// Malformed input returns MG_ERR_FORMAT (the reference asserts or crashes);
// blank lines are skipped.
//
// Throughput: the file is memory-mapped and split at line boundaries into one
// chunk per thread; each thread parses its chunk into (row, col[, w]) arrays.
// The CSR is then built by a parallel stable counting sort: rows are grouped
// into buckets of 2^k consecutive rows, every (chunk, direct/mirrored) segment
// counts its records per bucket, the records are scattered bucket by bucket
// (segments in file order, so the order stays stable), and each bucket is
// finished into its rows by one thread.  The result equals a serial
// file-order fill.
//
// Binary CSR cache ("<path>.mgcsr", little-endian):
//   64-byte header {magic "MGCSR1\n\0", u32 header bytes, u32 weighted,
//   u64 n, u64 nnz, u64 source size, i64 source mtime s, i64 source mtime ns,
//   u64 0}, then offsets u64[n+1], cols u32[nnz], padding to 8 bytes, and
//   weights f64[nnz] when weighted.  It is used only when the .mtx file's
//   size and modification time match the header; it is mapped read-only and
//   handed out without a copy.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <thread>
#include <vector>

#include "host_csr.h"

mg_host_csr::~mg_host_csr() {
    if (map) munmap(map, map_len);
}

namespace mg {

namespace {

constexpr char kMagic[8] = {'M', 'G', 'C', 'S', 'R', '1', '\n', '\0'};

struct CacheHeader {
    char magic[8];
    uint32_t header_bytes;
    uint32_t weighted;
    uint64_t n;
    uint64_t nnz;
    uint64_t src_size;
    int64_t src_mtime_s;
    int64_t src_mtime_ns;
    uint64_t reserved;
};
static_assert(sizeof(CacheHeader) == 64, "cache header is 64 bytes");

unsigned thread_count() {
    unsigned t = std::thread::hardware_concurrency();
    return std::max(1u, std::min(64u, t ? t : 1u));
}

// Run fn(i) for i in [0, count) on up to `threads` threads (dynamic schedule).
void parallel_for(size_t count, unsigned threads, const std::function<void(size_t)> &fn) {
    threads = (unsigned)std::min<size_t>(threads, count);
    if (threads <= 1) {
        for (size_t i = 0; i < count; i++) fn(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> th;
    for (unsigned t = 0; t < threads; t++)
        th.emplace_back([&] {
            for (size_t i; (i = next.fetch_add(1)) < count;) fn(i);
        });
    for (auto &x : th) x.join();
}

// atoi of a field that ends at the line end: leading blanks, a sign, digits
inline long field_int(const char *p, const char *end) {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) p++;
    bool neg = false;
    if (p < end && (*p == '+' || *p == '-')) neg = *p++ == '-';
    long v = 0;
    for (; p < end && *p >= '0' && *p <= '9'; p++)
        if (v < (1L << 40)) v = v * 10 + (*p - '0');  // saturates far above any row count
    return neg ? -v : v;
}
// atof of a field that ends at the line end (bounded copy, then strtod)
inline double field_real(const char *p, const char *end) {
    char buf[128];
    size_t n = std::min<size_t>((size_t)(end - p), sizeof(buf) - 1);
    memcpy(buf, p, n);
    buf[n] = 0;
    return strtod(buf, nullptr);
}

struct Part {
    std::vector<uint32_t> r, c;
    std::vector<double> w;  // general files only
    size_t diag = 0;        // entries with r == c (symmetric files)
    bool ok = true;
};

// Parse the entry lines of [p, end).
void parse_chunk(const char *p, const char *end, bool symmetric, uint32_t nrow, Part &out) {
    const size_t guess = (size_t)(end - p) / 12 + 16;
    out.r.reserve(guess);
    out.c.reserve(guess);
    if (!symmetric) out.w.reserve(guess);
    while (p < end) {
        const char *eol = (const char *)memchr(p, '\n', (size_t)(end - p));
        const char *le = eol ? eol : end;
        if (le > p) {
            const long r = field_int(p, le) - 1;
            const char *ch = (const char *)memchr(p, ' ', (size_t)(le - p));
            if (!ch) {
                out.ok = false;
                return;
            }
            ch++;
            const long c = field_int(ch, le) - 1;
            const char *ch2 = (const char *)memchr(ch, ' ', (size_t)(le - ch));
            if (r < 0 || c < 0 || (unsigned long)r >= nrow || (unsigned long)c >= nrow) {
                out.ok = false;
                return;
            }
            if (symmetric) {
                out.r.push_back((uint32_t)r);
                out.c.push_back((uint32_t)c);
                out.diag += r == c;
            } else if (c < r) {
                out.r.push_back((uint32_t)r);
                out.c.push_back((uint32_t)c);
                out.w.push_back(ch2 ? field_real(ch2 + 1, le) : 1.0);
            }
        }
        p = le + 1;
    }
}

// One run of records in file order: kind 0 = (r -> c), 1 = mirrored (c -> r,
// diagonal skipped), 2 = general (r -> c then c -> r per entry).
struct Segment {
    const Part *part;
    int kind;
};

inline size_t segment_records(const Segment &s) {
    const size_t m = s.part->r.size();
    return s.kind == 0 ? m : s.kind == 1 ? m - s.part->diag : 2 * m;
}

// Visit the records of a segment in order: fn(row, col, entry index).
template <class F>
inline void for_records(const Segment &s, F &&fn) {
    const Part &P = *s.part;
    const size_t m = P.r.size();
    if (s.kind == 0) {
        for (size_t i = 0; i < m; i++) fn(P.r[i], P.c[i], i);
    } else if (s.kind == 1) {
        for (size_t i = 0; i < m; i++)
            if (P.r[i] != P.c[i]) fn(P.c[i], P.r[i], i);
    } else {
        for (size_t i = 0; i < m; i++) {
            fn(P.r[i], P.c[i], i);
            fn(P.c[i], P.r[i], i);
        }
    }
}

mg_status build_csr(uint32_t nrow, bool symmetric, const std::vector<Part> &parts, unsigned threads,
                    mg_host_csr &out, std::string &err) {
    std::vector<Segment> segs;
    for (auto &p : parts) segs.push_back({&p, symmetric ? 0 : 2});
    if (symmetric)
        for (auto &p : parts) segs.push_back({&p, 1});
    uint64_t total = 0;
    for (auto &s : segs) total += segment_records(s);
    if (total >= 0xFFFFFFFFull) {
        err = "more than 2^32-1 directed entries";
        return MG_ERR_UNSUPPORTED;
    }
    // buckets of 2^bs rows, about 16K of them
    int bs = 6;
    while (((uint64_t)nrow >> bs) > 16384) bs++;
    const size_t NB = ((size_t)nrow >> bs) + 1, NS = segs.size();
    std::vector<uint64_t> pos(NS * NB, 0), bstart(NB + 1, 0);
    parallel_for(NS, threads, [&](size_t s) {
        uint64_t *h = &pos[s * NB];
        for_records(segs[s], [&](uint32_t row, uint32_t, size_t) { h[row >> bs]++; });
    });
    uint64_t run = 0;
    for (size_t b = 0; b < NB; b++) {
        bstart[b] = run;
        for (size_t s = 0; s < NS; s++) {
            const uint64_t c = pos[s * NB + b];
            pos[s * NB + b] = run;
            run += c;
        }
    }
    bstart[NB] = run;
    // records grouped by bucket, file order inside each bucket
    std::unique_ptr<uint32_t[]> tr(new uint32_t[total ? total : 1]), tc(new uint32_t[total ? total : 1]);
    std::unique_ptr<double[]> tw(symmetric ? nullptr : new double[total ? total : 1]);
    parallel_for(NS, threads, [&](size_t s) {
        uint64_t *p = &pos[s * NB];
        const Part &P = *segs[s].part;
        for_records(segs[s], [&](uint32_t row, uint32_t col, size_t i) {
            const uint64_t q = p[row >> bs]++;
            tr[q] = row;
            tc[q] = col;
            if (!symmetric) tw[q] = P.w[i];
        });
    });
    out.n = nrow;
    out.nnz = total;
    out.weighted = symmetric ? 0 : 1;
    out.off_buf.reset(new uint64_t[(size_t)nrow + 1]);
    out.cols_buf.reset(new uint32_t[total ? total : 1]);
    if (!symmetric) out.w_buf.reset(new double[total ? total : 1]);
    uint64_t *off = out.off_buf.get();
    uint32_t *cols = out.cols_buf.get();
    double *w = out.w_buf.get();
    const size_t rows_per = (size_t)1 << bs;
    parallel_for(NB, threads, [&](size_t b) {
        const uint64_t lo = (uint64_t)b << bs;
        if (lo >= nrow) return;
        const uint64_t hi = std::min<uint64_t>(nrow, lo + rows_per);
        std::vector<uint64_t> cur(hi - lo + 1, 0);
        for (uint64_t q = bstart[b]; q < bstart[b + 1]; q++) cur[tr[q] - lo + 1]++;
        cur[0] = bstart[b];
        for (uint64_t r = 1; r <= hi - lo; r++) cur[r] += cur[r - 1];
        for (uint64_t r = lo; r < hi; r++) off[r] = cur[r - lo];
        for (uint64_t q = bstart[b]; q < bstart[b + 1]; q++) {
            const uint64_t d = cur[tr[q] - lo]++;
            cols[d] = tc[q];
            if (w) w[d] = tw[q];
        }
    });
    off[nrow] = total;
    out.off = off;
    out.cols = cols;
    out.w = w;
    return MG_OK;
}

std::string cache_path(const char *path) { return std::string(path) + ".mgcsr"; }

size_t cache_bytes(uint64_t n, uint64_t nnz, bool weighted) {
    size_t b = sizeof(CacheHeader) + 8 * (n + 1) + 4 * nnz;
    b = (b + 7) & ~(size_t)7;
    if (weighted) b += 8 * nnz;
    return b;
}

// Map the cache of `path` if it matches `st`; false if absent or stale.
bool read_cache(const char *path, const struct stat &st, mg_host_csr &out) {
    const std::string cp = cache_path(path);
    int fd = open(cp.c_str(), O_RDONLY);
    if (fd < 0) return false;
    struct stat cs;
    if (fstat(fd, &cs) != 0 || (size_t)cs.st_size < sizeof(CacheHeader)) {
        close(fd);
        return false;
    }
    void *m = mmap(nullptr, (size_t)cs.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (m == MAP_FAILED) return false;
    const CacheHeader *h = (const CacheHeader *)m;
    bool ok = memcmp(h->magic, kMagic, 8) == 0 && h->header_bytes == sizeof(CacheHeader) && h->weighted <= 1 &&
              h->n < 0xFFFFFFFFull && h->nnz < 0xFFFFFFFFull && h->src_size == (uint64_t)st.st_size &&
              h->src_mtime_s == (int64_t)st.st_mtim.tv_sec && h->src_mtime_ns == (int64_t)st.st_mtim.tv_nsec &&
              cache_bytes(h->n, h->nnz, h->weighted) == (size_t)cs.st_size;
    if (ok) {
        const char *base = (const char *)m;
        const uint64_t *off = (const uint64_t *)(base + sizeof(CacheHeader));
        ok = off[0] == 0 && off[h->n] == h->nnz;
        for (uint64_t i = 0; ok && i < h->n; i++) ok = off[i] <= off[i + 1];
        if (ok) {
            madvise(m, (size_t)cs.st_size, MADV_WILLNEED);
            out.n = (uint32_t)h->n;
            out.nnz = h->nnz;
            out.weighted = (int)h->weighted;
            out.off = off;
            out.cols = (const uint32_t *)(base + sizeof(CacheHeader) + 8 * (h->n + 1));
            const size_t woff = (sizeof(CacheHeader) + 8 * (h->n + 1) + 4 * h->nnz + 7) & ~(size_t)7;
            out.w = h->weighted ? (const double *)(base + woff) : nullptr;
            out.map = m;
            out.map_len = (size_t)cs.st_size;
            out.from_cache = 1;
            return true;
        }
    }
    munmap(m, (size_t)cs.st_size);
    return false;
}

bool write_all(FILE *f, const void *p, size_t bytes) { return bytes == 0 || fwrite(p, 1, bytes, f) == bytes; }

// Write the cache through a temporary file and a rename; false on failure.
bool write_cache(const char *path, const struct stat &st, const mg_host_csr &c) {
    const std::string cp = cache_path(path);
    const std::string tmp = cp + ".tmp." + std::to_string((long)getpid());
    FILE *f = fopen(tmp.c_str(), "wb");
    if (!f) return false;
    CacheHeader h;
    memset(&h, 0, sizeof h);
    memcpy(h.magic, kMagic, 8);
    h.header_bytes = sizeof(CacheHeader);
    h.weighted = (uint32_t)c.weighted;
    h.n = c.n;
    h.nnz = c.nnz;
    h.src_size = (uint64_t)st.st_size;
    h.src_mtime_s = (int64_t)st.st_mtim.tv_sec;
    h.src_mtime_ns = (int64_t)st.st_mtim.tv_nsec;
    const uint64_t zero = 0;
    const size_t pad = (8 - (sizeof(CacheHeader) + 8 * ((size_t)c.n + 1) + 4 * c.nnz) % 8) % 8;
    bool ok = write_all(f, &h, sizeof h) && write_all(f, c.off, 8 * ((size_t)c.n + 1)) &&
              write_all(f, c.cols, 4 * c.nnz) && write_all(f, &zero, pad) &&
              (!c.weighted || write_all(f, c.w, 8 * c.nnz));
    ok = fclose(f) == 0 && ok;
    if (ok) ok = rename(tmp.c_str(), cp.c_str()) == 0;
    if (!ok) unlink(tmp.c_str());
    return ok;
}

}  // namespace

mg_status load_mtx_csr(const char *path, int flags, mg_host_csr &out, std::string &err) {
    int fd = open(path, O_RDONLY);
    if (fd < 0) {
        err = std::string("cannot open ") + path;
        return MG_ERR_IO;
    }
    struct stat st;
    if (fstat(fd, &st) != 0) {
        close(fd);
        err = std::string("cannot stat ") + path;
        return MG_ERR_IO;
    }
    if ((flags & MG_LOAD_CACHE_READ) && read_cache(path, st, out)) {
        close(fd);
        return MG_OK;
    }
    const size_t size = (size_t)st.st_size;
    if (size == 0) {
        close(fd);
        err = "empty file";
        return MG_ERR_FORMAT;
    }
    void *m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (m == MAP_FAILED) {
        err = std::string("cannot map ") + path;
        return MG_ERR_IO;
    }
    madvise(m, size, MADV_SEQUENTIAL);
    struct Unmap {
        void *m;
        size_t n;
        ~Unmap() { munmap(m, n); }
    } unmap{m, size};
    const char *p = (const char *)m, *end = p + size;
    auto next_line = [&](const char *&q) -> std::string {
        const char *e = (const char *)memchr(q, '\n', (size_t)(end - q));
        const char *le = e ? e : end;
        std::string l(q, le);
        q = e ? e + 1 : end;
        return l;
    };
    std::string banner = next_line(p);
    bool symmetric = false;
    if (banner.find("general") != std::string::npos) symmetric = false;
    else if (banner.find("symmetric") != std::string::npos) symmetric = true;
    std::string line;
    do {
        if (p >= end) {
            err = "missing size line";
            return MG_ERR_FORMAT;
        }
        line = next_line(p);
    } while (!line.empty() && line[0] == '%');
    unsigned nrow = 0, ncol = 0, nnz = 0;
    if (sscanf(line.c_str(), "%u %u %u", &nrow, &ncol, &nnz) != 3) {
        err = "bad size line";
        return MG_ERR_FORMAT;
    }
    // one chunk per thread, cut at line boundaries
    unsigned nt = thread_count();
    const size_t body = (size_t)(end - p);
    if (body < (1u << 20)) nt = 1;
    std::vector<const char *> cut(nt + 1);
    cut[0] = p;
    cut[nt] = end;
    for (unsigned t = 1; t < nt; t++) {
        const char *q = p + body * t / nt;
        if (q < cut[t - 1]) q = cut[t - 1];
        const char *e = (const char *)memchr(q, '\n', (size_t)(end - q));
        cut[t] = e ? e + 1 : end;
    }
    std::vector<Part> parts(nt);
    parallel_for(nt, nt, [&](size_t t) { parse_chunk(cut[t], cut[t + 1], symmetric, nrow, parts[t]); });
    for (auto &pt : parts)
        if (!pt.ok) {
            err = "malformed entry line";
            return MG_ERR_FORMAT;
        }
    uint64_t num = 0;
    for (auto &pt : parts) num += pt.r.size();
    if (num > nnz || (symmetric && num != nnz)) {
        err = "entry count does not match the size line";
        return MG_ERR_FORMAT;
    }
    mg_status s = build_csr(nrow, symmetric, parts, thread_count(), out, err);
    if (s != MG_OK) return s;
    if (flags & MG_LOAD_CACHE_WRITE) out.cache_written = write_cache(path, st, out) ? 1 : 0;
    return MG_OK;
}

}  // namespace mg
