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
// The file is read in one block and parsed by several threads; results are
// concatenated in file order.  Malformed input returns MG_ERR_FORMAT (the
// reference asserts or crashes).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mgagcd.h"

namespace mg {

namespace {

struct Entry {
    uint32_t r, c;
    double w;
};

// strchr restricted to [p, end)
inline const char *find_space(const char *p, const char *end) {
    const void *q = memchr(p, ' ', (size_t)(end - p));
    return (const char *)q;
}

// atoi / atof on a field that ends at the line end (copy to a small buffer)
inline long field_atoi(const char *p, const char *end) {
    char buf[64];
    size_t n = std::min<size_t>((size_t)(end - p), sizeof(buf) - 1);
    memcpy(buf, p, n);
    buf[n] = 0;
    return atol(buf);
}
inline double field_atof(const char *p, const char *end) {
    char buf[128];
    size_t n = std::min<size_t>((size_t)(end - p), sizeof(buf) - 1);
    memcpy(buf, p, n);
    buf[n] = 0;
    return atof(buf);
}

// Parse entry lines in [p, end).  Returns false on a malformed line.
bool parse_chunk(const char *p, const char *end, bool symmetric, uint32_t nrow, std::vector<Entry> &out) {
    while (p < end) {
        const char *eol = (const char *)memchr(p, '\n', (size_t)(end - p));
        const char *le = eol ? eol : end;
        if (le > p) {
            long r = field_atoi(p, le) - 1;
            const char *ch = find_space(p, le);
            if (!ch) return false;
            ch++;
            long c = field_atoi(ch, le) - 1;
            const char *ch2 = find_space(ch, le);
            if (r < 0 || c < 0 || (unsigned long)r >= nrow || (unsigned long)c >= nrow) return false;
            if (symmetric || c < r) {
                double w = 1.0;
                if (!symmetric && ch2) w = field_atof(ch2 + 1, le);
                out.push_back(Entry{(uint32_t)r, (uint32_t)c, w});
            }
        }
        p = le + 1;
    }
    return true;
}

}  // namespace

mg_status load_mtx_host(const char *path, uint32_t &n, std::vector<uint64_t> &off, std::vector<uint32_t> &cols,
                        std::vector<double> &w, std::string &err) {
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        err = std::string("cannot open ") + path;
        return MG_ERR_IO;
    }
    fseek(fp, 0, SEEK_END);
    long size = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    std::string buf((size_t)std::max<long>(size, 0), '\0');
    if (size > 0 && fread(&buf[0], 1, (size_t)size, fp) != (size_t)size) {
        fclose(fp);
        err = "short read";
        return MG_ERR_IO;
    }
    fclose(fp);
    const char *p = buf.data(), *end = p + buf.size();
    auto next_line = [&](const char *&q) -> std::string {
        const char *e = (const char *)memchr(q, '\n', (size_t)(end - q));
        const char *le = e ? e : end;
        std::string l(q, le);
        q = e ? e + 1 : end;
        return l;
    };
    if (p >= end) {
        err = "empty file";
        return MG_ERR_FORMAT;
    }
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
    // split the entry section into per-thread chunks at line boundaries
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    size_t body = (size_t)(end - p);
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
    std::vector<std::vector<Entry>> parts(nt);
    std::vector<char> ok(nt, 1);
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++)
        th.emplace_back([&, t] { ok[t] = parse_chunk(cut[t], cut[t + 1], symmetric, nrow, parts[t]); });
    for (auto &x : th) x.join();
    for (unsigned t = 0; t < nt; t++)
        if (!ok[t]) {
            err = "malformed entry line";
            return MG_ERR_FORMAT;
        }
    uint64_t num = 0;
    for (auto &v : parts) num += v.size();
    if (num > nnz || (symmetric && num != nnz)) {
        err = "entry count does not match the size line";
        return MG_ERR_FORMAT;
    }
    n = nrow;
    off.assign((size_t)nrow + 1, 0);
    for (auto &v : parts)
        for (auto &x : v) {
            off[x.r + 1]++;
            if (!symmetric || x.r != x.c) off[x.c + 1]++;
        }
    for (uint32_t i = 0; i < nrow; i++) off[i + 1] += off[i];
    uint64_t total = off[nrow];
    if (total >= 0xFFFFFFFFull) {
        err = "more than 2^32-1 directed entries";
        return MG_ERR_UNSUPPORTED;
    }
    cols.resize(total);
    w.resize(total);
    std::vector<uint64_t> cur(off.begin(), off.end() - 1);
    if (symmetric) {
        for (auto &v : parts)
            for (auto &x : v) {
                uint64_t q = cur[x.r]++;
                cols[q] = x.c;
                w[q] = 1.0;
            }
        for (auto &v : parts)
            for (auto &x : v)
                if (x.r != x.c) {
                    uint64_t q = cur[x.c]++;
                    cols[q] = x.r;
                    w[q] = 1.0;
                }
    } else {
        for (auto &v : parts)
            for (auto &x : v) {
                uint64_t q = cur[x.r]++;
                cols[q] = x.c;
                w[q] = x.w;
                q = cur[x.c]++;
                cols[q] = x.r;
                w[q] = x.w;
            }
    }
    return MG_OK;
}

}  // namespace mg
