// host_csr.h -- a symmetric CSR in host memory, as the Matrix Market loader
// produces it: either heap arrays built by the parser or a read-only mapping
// of a binary CSR cache file.  Host-only code (no CUDA).
#pragma once

#include <cstdint>
#include <memory>
#include <string>

#include "../../include/mgagcd.h"

struct mg_host_csr {
    uint32_t n = 0;
    uint64_t nnz = 0;
    int weighted = 0;    // 0: every weight is 1 (symmetric files), 1: f64 weights
    int from_cache = 0;  // 1: the arrays come from the binary cache
    int cache_written = 0;
    const uint64_t *off = nullptr;
    const uint32_t *cols = nullptr;
    const double *w = nullptr;  // NULL when !weighted
    // storage behind the pointers
    std::unique_ptr<uint64_t[]> off_buf;
    std::unique_ptr<uint32_t[]> cols_buf;
    std::unique_ptr<double[]> w_buf;
    void *map = nullptr;
    size_t map_len = 0;
    ~mg_host_csr();
};

namespace mg {
// Load `path` with the reference's .mtx rules.  flags: MG_LOAD_CACHE_READ
// (use "<path>.mgcsr" when it matches the file's size and modification time),
// MG_LOAD_CACHE_WRITE (write that cache after parsing; failures to write are
// not errors).
mg_status load_mtx_csr(const char *path, int flags, mg_host_csr &out, std::string &err);
}  // namespace mg
