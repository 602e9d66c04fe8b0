/*
 * oracle.c -- CPU restatement of the MG-alphaGCD Louvain hot path (C11 + OpenMP).
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, by __graft_entry__.smoke() as
 * the checker and by bench.py's CPU baseline.  The product library never
 * links or calls it.  Built with -ffp-contract=off so that every floating
 * point expression is evaluated exactly as written (no fused multiply-add),
 * which is what makes the local-move gains bit-identical to the reference's
 * double-precision kernels.
 *
 * Reference files are cited relative to the MG-alphaGCD source tree.
 */
#include "oracle.h"

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OR_EMPTY 0xFFFFFFFFu

void or_free(void *p) { free(p); }

void or_graph_free(or_graph *g) {
    if (!g) return;
    free(g->offsets);
    free(g->cols);
    free(g->weights);
    g->offsets = NULL;
    g->cols = NULL;
    g->weights = NULL;
    g->n = 0;
    g->nnz = 0;
}

int or_set_threads(int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    return omp_get_max_threads();
}
int or_get_threads(void) { return omp_get_max_threads(); }

static inline double wt(const or_graph *g, uint64_t e) { return g->weights ? g->weights[e] : 1.0; }

/* ======================================================================== */
/* Loader -- follows src/mmio/mmio_wrapper.cu:76-295.                        */
/*  * banner line: "general" -> general path, "symmetric" -> symmetric path   */
/*    (mmio_wrapper.cu:97-102); comment lines start with '%' (:104-106);     */
/*  * symmetric: every entry gets weight 1.0 (:141-142), off-diagonal entries */
/*    are mirrored (:163-170), then a stable sort by row (:181), so a row    */
/*    holds its file-order entries followed by its mirrored entries;         */
/*  * general: entries with col >= row are skipped (:239), the optional      */
/*    third token is the weight, else 1.0 (:243-250); each kept entry is      */
/*    stored in both rows (:277-288).  The reference fills rows with 80      */
/*    OpenMP threads (row order unspecified); this restatement uses the      */
/*    order a single thread produces: file order.                            */
/* Malformed input (which makes the reference assert or crash) returns -2.  */
/* ======================================================================== */
int or_load_mtx(const char *path, or_graph *out) {
    memset(out, 0, sizeof(*out));
    FILE *fp = fopen(path, "r");
    if (!fp) return -1;
    char line[1000];
    if (!fgets(line, sizeof line, fp)) { fclose(fp); return -2; }
    int symmetric = 0;
    if (strstr(line, "general")) symmetric = 0;
    else if (strstr(line, "symmetric")) symmetric = 1;
    do {
        if (!fgets(line, sizeof line, fp)) { fclose(fp); return -2; }
    } while (line[0] == '%');
    unsigned nrow = 0, ncol = 0, nnz = 0;
    if (sscanf(line, "%u %u %u", &nrow, &ncol, &nnz) != 3) { fclose(fp); return -2; }

    uint32_t *row = (uint32_t *)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    uint32_t *col = (uint32_t *)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    double *val = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
    uint64_t num = 0;
    int rc = 0;
    while (fgets(line, sizeof line, fp)) {
        char *ch = line;
        long r = atoi(ch) - 1;
        ch = strchr(ch, ' ');
        if (!ch) { rc = -2; break; }
        ch++;
        long c = atoi(ch) - 1;
        ch = strchr(ch, ' ');
        if (r < 0 || c < 0 || (unsigned long)r >= nrow || (unsigned long)c >= nrow) { rc = -2; break; }
        if (!symmetric && c >= r) continue;
        if (num >= nnz) { rc = -2; break; }
        double w = 1.0;
        if (!symmetric && ch != NULL) { ch++; w = atof(ch); }
        row[num] = (uint32_t)r;
        col[num] = (uint32_t)c;
        val[num] = w;
        num++;
    }
    fclose(fp);
    if (rc == 0 && symmetric && num != nnz) rc = -2;
    if (rc != 0) { free(row); free(col); free(val); return rc; }

    uint64_t *off = (uint64_t *)calloc((size_t)nrow + 1, sizeof(uint64_t));
    uint64_t total;
    if (symmetric) {
        uint64_t extra = 0;
        for (uint64_t i = 0; i < num; i++) extra += (row[i] != col[i]);
        total = num + extra;
        for (uint64_t i = 0; i < num; i++) {
            off[row[i] + 1]++;
            if (row[i] != col[i]) off[col[i] + 1]++;
        }
    } else {
        total = 2 * num;
        for (uint64_t i = 0; i < num; i++) { off[row[i] + 1]++; off[col[i] + 1]++; }
    }
    for (uint32_t i = 0; i < nrow; i++) off[i + 1] += off[i];
    uint32_t *cols = (uint32_t *)malloc(sizeof(uint32_t) * (total ? total : 1));
    double *w = (double *)malloc(sizeof(double) * (total ? total : 1));
    uint64_t *cur = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)nrow + 1));
    memcpy(cur, off, sizeof(uint64_t) * ((size_t)nrow + 1));
    if (symmetric) {
        /* stable sort by row of [originals..., mirrored...] */
        for (uint64_t i = 0; i < num; i++) { uint64_t p = cur[row[i]]++; cols[p] = col[i]; w[p] = 1.0; }
        for (uint64_t i = 0; i < num; i++)
            if (row[i] != col[i]) { uint64_t p = cur[col[i]]++; cols[p] = row[i]; w[p] = 1.0; }
    } else {
        for (uint64_t i = 0; i < num; i++) {
            uint64_t p = cur[row[i]]++; cols[p] = col[i]; w[p] = val[i];
            p = cur[col[i]]++; cols[p] = row[i]; w[p] = val[i];
        }
    }
    free(cur); free(row); free(col); free(val);
    out->n = nrow;
    out->nnz = total;
    out->offsets = off;
    out->cols = cols;
    out->weights = w;
    return 0;
}

/* ======================================================================== */
/* Generators.  Integer-only counter-based RNG (splitmix64 finaliser) so   */
/* that the CUDA generators produce the identical graph.                    */
/* ======================================================================== */
uint64_t or_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline uint64_t rng_key(uint64_t seed, uint64_t stream) {
    return or_mix64(seed * 0x2545F4914F6CDD1Dull + stream);
}
static inline uint64_t rng_at(uint64_t key, uint64_t ctr) {
    return or_mix64(key + ctr * 0x9E3779B97F4A7C15ull);
}
static inline uint32_t uni32(uint32_t x, uint32_t range) {
    return (uint32_t)(((uint64_t)x * range) >> 32);
}

static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}
typedef struct { uint32_t c; double w; } cw_t;
static int cmp_cw(const void *a, const void *b) {
    const cw_t *x = (const cw_t *)a, *y = (const cw_t *)b;
    if (x->c != y->c) return (x->c > y->c) - (x->c < y->c);
    return (x->w > y->w) - (x->w < y->w);
}

int or_csr_from_pairs(uint32_t n, uint64_t m, const uint32_t *u, const uint32_t *v,
                      const double *w, or_graph *out) {
    memset(out, 0, sizeof(*out));
    uint64_t *deg = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    for (uint64_t i = 0; i < m; i++) {
        if (u[i] >= n || v[i] >= n) { free(deg); return -2; }
    }
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < m; i++) {
        if (u[i] == v[i]) continue;
#pragma omp atomic
        deg[u[i] + 1]++;
#pragma omp atomic
        deg[v[i] + 1]++;
    }
    for (uint32_t i = 0; i < n; i++) deg[i + 1] += deg[i];
    uint64_t tot = deg[n];
    uint64_t *cur = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)n + 1));
    memcpy(cur, deg, sizeof(uint64_t) * ((size_t)n + 1));
    uint32_t *cols = (uint32_t *)malloc(sizeof(uint32_t) * (tot ? tot : 1));
    double *ws = w ? (double *)malloc(sizeof(double) * (tot ? tot : 1)) : NULL;
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < m; i++) {
        if (u[i] == v[i]) continue;
        uint64_t p, q;
#pragma omp atomic capture
        p = cur[u[i]]++;
#pragma omp atomic capture
        q = cur[v[i]]++;
        cols[p] = v[i];
        cols[q] = u[i];
        if (ws) { ws[p] = w[i]; ws[q] = w[i]; }
    }
    free(cur);
    /* sort + dedup each row */
    uint64_t *newdeg = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 1024)
    for (uint32_t r = 0; r < n; r++) {
        uint64_t lo = deg[r], hi = deg[r + 1];
        if (hi == lo) continue;
        if (!ws) {
            qsort(cols + lo, hi - lo, sizeof(uint32_t), cmp_u32);
            uint64_t k = lo;
            for (uint64_t e = lo; e < hi; e++)
                if (e == lo || cols[e] != cols[k - 1]) cols[k++] = cols[e];
            newdeg[r + 1] = k - lo;
        } else {
            cw_t *tmp = (cw_t *)malloc(sizeof(cw_t) * (hi - lo));
            for (uint64_t e = lo; e < hi; e++) { tmp[e - lo].c = cols[e]; tmp[e - lo].w = ws[e]; }
            qsort(tmp, hi - lo, sizeof(cw_t), cmp_cw);
            uint64_t k = lo;
            for (uint64_t e = 0; e < hi - lo; e++)
                if (e == 0 || tmp[e].c != tmp[e - 1].c) { cols[k] = tmp[e].c; ws[k] = tmp[e].w; k++; }
            newdeg[r + 1] = k - lo;
            free(tmp);
        }
    }
    for (uint32_t i = 0; i < n; i++) newdeg[i + 1] += newdeg[i];
    uint64_t nt = newdeg[n];
    uint32_t *c2 = (uint32_t *)malloc(sizeof(uint32_t) * (nt ? nt : 1));
    double *w2 = ws ? (double *)malloc(sizeof(double) * (nt ? nt : 1)) : NULL;
#pragma omp parallel for schedule(dynamic, 1024)
    for (uint32_t r = 0; r < n; r++) {
        uint64_t len = newdeg[r + 1] - newdeg[r];
        memcpy(c2 + newdeg[r], cols + deg[r], len * sizeof(uint32_t));
        if (ws) memcpy(w2 + newdeg[r], ws + deg[r], len * sizeof(double));
    }
    free(cols); free(ws); free(deg);
    out->n = n;
    out->nnz = nt;
    out->offsets = newdeg;
    out->cols = c2;
    out->weights = w2;
    return 0;
}

/* R-MAT edge k: level l (0 = most significant bit) draws a 32-bit value x
 * from word l/2 (low half for even l, high half for odd l) and picks the
 * quadrant with thresholds t1 < t2 < t3 on [0, 2^32). */
int or_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                uint64_t seed, or_graph *out) {
    if (scale < 1 || scale > 31 || edge_factor < 1) return -2;
    uint32_t n = 1u << scale;
    uint64_t m = (uint64_t)edge_factor << scale;
    uint64_t t1 = (uint64_t)(a * 4294967296.0);
    uint64_t t2 = (uint64_t)((a + b) * 4294967296.0);
    uint64_t t3 = (uint64_t)((a + b + c) * 4294967296.0);
    uint64_t key = rng_key(seed, 0x524d4154ull /* "RMAT" */);
    uint32_t *u = (uint32_t *)malloc(sizeof(uint32_t) * m);
    uint32_t *v = (uint32_t *)malloc(sizeof(uint32_t) * m);
    int words = (scale + 1) / 2;
#pragma omp parallel for schedule(static)
    for (uint64_t k = 0; k < m; k++) {
        uint32_t uu = 0, vv = 0;
        for (int wi = 0; wi < words; wi++) {
            uint64_t r = rng_at(key, k * (uint64_t)words + (uint64_t)wi);
            for (int h = 0; h < 2; h++) {
                int l = 2 * wi + h;
                if (l >= scale) break;
                uint64_t x = h ? (r >> 32) : (r & 0xFFFFFFFFull);
                uint32_t bu, bv;
                if (x < t1) { bu = 0; bv = 0; }
                else if (x < t2) { bu = 0; bv = 1; }
                else if (x < t3) { bu = 1; bv = 0; }
                else { bu = 1; bv = 1; }
                uu |= bu << (scale - 1 - l);
                vv |= bv << (scale - 1 - l);
            }
        }
        u[k] = uu;
        v[k] = vv;
    }
    int rc = or_csr_from_pairs(n, m, u, v, NULL, out);
    free(u); free(v);
    return rc;
}

/* Planted partition: blocks [b*n/B, (b+1)*n/B).  round(n*d_in/2) intra pairs
 * (block, two members) and round(n*d_out/2) inter pairs (two distinct
 * blocks, one member each); self-loops and duplicates removed. */
int or_gen_sbm(uint32_t n, uint32_t blocks, double mean_degree, double intra_frac,
               uint64_t seed, or_graph *out) {
    if (blocks < 1 || n < blocks) return -2;
    double din = mean_degree * intra_frac;
    double dout = mean_degree - din;
    uint64_t min_ = (uint64_t)llround((double)n * din / 2.0);
    uint64_t mout = blocks > 1 ? (uint64_t)llround((double)n * dout / 2.0) : 0;
    uint64_t m = min_ + mout;
    uint32_t *u = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    uint32_t *v = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    uint64_t kin = rng_key(seed, 0x53424d31ull), kout = rng_key(seed, 0x53424d32ull);
#pragma omp parallel for schedule(static)
    for (uint64_t k = 0; k < m; k++) {
        if (k < min_) {
            uint64_t r0 = rng_at(kin, 2 * k), r1 = rng_at(kin, 2 * k + 1);
            uint32_t bb = uni32((uint32_t)r0, blocks);
            uint32_t lo = (uint32_t)((uint64_t)bb * n / blocks), hi = (uint32_t)((uint64_t)(bb + 1) * n / blocks);
            u[k] = lo + uni32((uint32_t)(r0 >> 32), hi - lo);
            v[k] = lo + uni32((uint32_t)r1, hi - lo);
        } else {
            uint64_t j = k - min_;
            uint64_t r0 = rng_at(kout, 2 * j), r1 = rng_at(kout, 2 * j + 1);
            uint32_t b1 = uni32((uint32_t)r0, blocks);
            uint32_t b2 = uni32((uint32_t)(r0 >> 32), blocks - 1);
            if (b2 >= b1) b2++;
            uint32_t lo1 = (uint32_t)((uint64_t)b1 * n / blocks), hi1 = (uint32_t)((uint64_t)(b1 + 1) * n / blocks);
            uint32_t lo2 = (uint32_t)((uint64_t)b2 * n / blocks), hi2 = (uint32_t)((uint64_t)(b2 + 1) * n / blocks);
            u[k] = lo1 + uni32((uint32_t)r1, hi1 - lo1);
            v[k] = lo2 + uni32((uint32_t)(r1 >> 32), hi2 - lo2);
        }
    }
    int rc = or_csr_from_pairs(n, m, u, v, NULL, out);
    free(u); free(v);
    return rc;
}

/* Chung-Lu: expected degrees w_i = c*(i+i0)^(-1/(gamma-1)), i0 chosen so
 * that w_0 = max_degree, c so that the mean is mean_degree (then capped at
 * max_degree).  round(n*mean/2) pairs, endpoints drawn from the CDF of w
 * held as 63-bit fixed point.  Optional weights: float32(lognormal(0,1)),
 * a function of the unordered pair only (Box-Muller on two hashed uniforms). */
int or_gen_chunglu(uint32_t n, double exponent, double mean_degree, double max_degree,
                   int lognormal_weights, uint64_t seed, or_graph *out) {
    if (n < 2 || exponent <= 1.0) return -2;
    double alpha = 1.0 / (exponent - 1.0);
    double *wd = (double *)malloc(sizeof(double) * n);
    /* choose i0 so that w_0/mean(w) = max/mean using the integral approximation */
    double lo = 1e-6, hi = (double)n;
    for (int it = 0; it < 200; it++) {
        double i0 = 0.5 * (lo + hi);
        double integ = (alpha == 1.0) ? log((n + i0) / i0)
                                      : (pow(n + i0, 1.0 - alpha) - pow(i0, 1.0 - alpha)) / (1.0 - alpha);
        double ratio = pow(i0, -alpha) / (integ / n);
        if (ratio > max_degree / mean_degree) lo = i0; else hi = i0;
    }
    double i0 = 0.5 * (lo + hi);
    double s = 0;
    for (uint32_t i = 0; i < n; i++) { wd[i] = pow((double)i + i0, -alpha); s += wd[i]; }
    double cst = mean_degree * n / s;
    double tot = 0;
    for (uint32_t i = 0; i < n; i++) {
        wd[i] *= cst;
        if (wd[i] > max_degree) wd[i] = max_degree;
        tot += wd[i];
    }
    uint64_t *cdf = (uint64_t *)malloc(sizeof(uint64_t) * n);
    double acc = 0;
    for (uint32_t i = 0; i < n; i++) {
        acc += wd[i];
        double f = acc / tot;
        if (f > 1.0) f = 1.0;
        cdf[i] = (uint64_t)(f * 9223372036854775808.0);
    }
    cdf[n - 1] = 0x8000000000000000ull;
    free(wd);
    uint64_t m = (uint64_t)llround((double)n * mean_degree / 2.0);
    uint32_t *u = (uint32_t *)malloc(sizeof(uint32_t) * m);
    uint32_t *v = (uint32_t *)malloc(sizeof(uint32_t) * m);
    uint64_t key = rng_key(seed, 0x434c5547ull);
#pragma omp parallel for schedule(static)
    for (uint64_t k = 0; k < m; k++) {
        for (int side = 0; side < 2; side++) {
            uint64_t x = rng_at(key, 2 * k + side) >> 1; /* 63 bits */
            /* first index with cdf > x */
            uint32_t a = 0, b = n - 1;
            while (a < b) {
                uint32_t mid = a + (b - a) / 2;
                if (cdf[mid] > x) b = mid; else a = mid + 1;
            }
            if (side == 0) u[k] = a; else v[k] = a;
        }
    }
    free(cdf);
    double *w = NULL;
    if (lognormal_weights) {
        w = (double *)malloc(sizeof(double) * m);
        uint64_t kw = rng_key(seed, 0x4c4f474eull);
#pragma omp parallel for schedule(static)
        for (uint64_t k = 0; k < m; k++) {
            uint32_t a = u[k] < v[k] ? u[k] : v[k], b = u[k] < v[k] ? v[k] : u[k];
            uint64_t h1 = or_mix64(kw ^ (((uint64_t)a << 32) | b));
            uint64_t h2 = or_mix64(h1);
            double u1 = ((double)(h1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);
            double u2 = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
            double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
            w[k] = (double)(float)exp(z);
        }
    }
    int rc = or_csr_from_pairs(n, m, u, v, w, out);
    free(u); free(v); free(w);
    return rc;
}

/* ======================================================================== */
/* Degree binning -- src/bin/BIN.cu.                                        */
/* ======================================================================== */
static int bin_of(int scheme, uint64_t d) {
    if (scheme == 0) { /* BIN.cu:72-92 */
        if (d <= 2) return 0;
        if (d <= 4) return 1;
        if (d <= 8) return 2;
        if (d <= 16) return 3;
        if (d <= 32) return 4;
        if (d <= 128) return 5;
        if (d <= 512) return 6;
        if (d <= 2048) return 7;
        if (d <= 4094) return 8;
        return 9;
    } else if (scheme == 1) { /* BIN.cu:159-181 */
        if (d <= 32) return 0;
        if (d <= 64) return 1;
        if (d <= 128) return 2;
        if (d <= 256) return 3;
        if (d <= 512) return 4;
        if (d <= 1024) return 5;
        if (d <= 2048) return 6;
        if (d <= 4096) return 7;
        if (d <= 8192) return 8;
        if (d <= 12288) return 9;
        return 10;
    } else { /* BIN.cu:248-266 */
        if (d <= 32) return 0;
        if (d <= 64) return 1;
        if (d <= 128) return 2;
        if (d <= 256) return 3;
        if (d <= 512) return 4;
        if (d <= 1024) return 5;
        if (d <= 2048) return 6;
        if (d <= 4095) return 7;
        return 8;
    }
}
static int bin_count(int scheme) { return scheme == 0 ? 10 : scheme == 1 ? 11 : 9; }

int or_bins(int scheme, uint32_t n, const uint64_t *offsets, uint32_t *sizes,
            uint32_t *bin_offsets, uint32_t *perm, uint32_t *max_degree) {
    if (scheme < 0 || scheme > 2) return -2;
    int nb = bin_count(scheme);
    uint32_t cnt[11] = {0};
    uint64_t md = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint64_t d = offsets[i + 1] - offsets[i];
        if (d > md) md = d;
        cnt[bin_of(scheme, d)]++;
    }
    uint32_t off[11] = {0};
    for (int b = 1; b < nb; b++) off[b] = off[b - 1] + cnt[b - 1];
    for (int b = 0; b < 11; b++) {
        sizes[b] = b < nb ? cnt[b] : 0;
        bin_offsets[b] = b < nb ? off[b] : 0;
    }
    if (perm) {
        uint32_t cur[11];
        memcpy(cur, off, sizeof cur);
        for (uint32_t i = 0; i < n; i++) perm[cur[bin_of(scheme, offsets[i + 1] - offsets[i])]++] = i;
    }
    *max_degree = (uint32_t)md;
    return 0;
}

/* ======================================================================== */
/* Vertex weights, mass, modularity.                                        */
/* ======================================================================== */
int or_vertex_weights(const or_graph *g, double *k) { /* louvain.cu:30-74 */
#pragma omp parallel for schedule(dynamic, 4096)
    for (uint32_t i = 0; i < g->n; i++) {
        double s = 0;
        for (uint64_t e = g->offsets[i]; e < g->offsets[i + 1]; e++) s += wt(g, e);
        k[i] = s;
    }
    return 0;
}

double or_mass(const or_graph *g) { /* host_graph.cpp:112-115 */
    double s = 0;
    for (uint64_t e = 0; e < g->nnz; e++) s += wt(g, e);
    return s;
}

int or_is_integral(const or_graph *g) {
    if (!g->weights) return g->nnz < 4294967296ull;
    double tot = 0;
    for (uint64_t e = 0; e < g->nnz; e++) {
        double w = g->weights[e];
        if (w < 0 || w != floor(w)) return 0;
        tot += w;
    }
    return tot < 4294967296.0;
}

/* Exact conversion used by both this oracle and the CUDA engine when the
 * graph is integral: Q = S_in/mass - S2/(mass*mass) with S_in and S2 exact
 * 64-bit integer sums (louvain.cu:233-235 gives the formula; the reference
 * sums in double, here the sums are exact). */
double or_modularity_sigma(const or_graph *g, const uint32_t *C, const double *sigma,
                           double mass, int integral) {
    uint32_t n = g->n;
    if (integral) {
        uint64_t sin = 0, s2 = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : sin)
        for (uint32_t i = 0; i < n; i++)
            for (uint64_t e = g->offsets[i]; e < g->offsets[i + 1]; e++)
                if (C[g->cols[e]] == C[i]) sin += (uint64_t)wt(g, e);
#pragma omp parallel for schedule(static) reduction(+ : s2)
        for (uint32_t c = 0; c < n; c++) {
            uint64_t s = (uint64_t)sigma[c];
            s2 += s * s;
        }
        return (double)sin / mass - (double)s2 / (mass * mass);
    }
    double sin = 0, s2 = 0;
    for (uint32_t i = 0; i < n; i++)
        for (uint64_t e = g->offsets[i]; e < g->offsets[i + 1]; e++)
            if (C[g->cols[e]] == C[i]) sin += wt(g, e);
    for (uint32_t c = 0; c < n; c++) s2 += sigma[c] * sigma[c];
    return sin / mass - s2 / (mass * mass);
}

double or_modularity(const or_graph *g, const uint32_t *C) {
    double *k = (double *)malloc(sizeof(double) * (g->n ? g->n : 1));
    double *sig = (double *)calloc(g->n ? g->n : 1, sizeof(double));
    or_vertex_weights(g, k);
    for (uint32_t i = 0; i < g->n; i++) {
        if (C[i] >= g->n) { free(k); free(sig); return NAN; }
        sig[C[i]] += k[i];
    }
    double mass = or_mass(g);
    double q = or_modularity_sigma(g, C, sig, mass, or_is_integral(g));
    free(k); free(sig);
    return q;
}

/* ======================================================================== */
/* One local-move sweep.  Per vertex i (louvain.cu:404-589 / 591-807 /      */
/* 810-1030, identical arithmetic in all three kernel shapes):              */
/*   src = C[i], a = sigma[src] - k_i                      (:481-495)        */
/*   edge (i,j,w), c = C[j]: c != src -> k_ic += w, else j != i -> e += w   */
/*                                                         (:506-518)        */
/*   gain_c = (k_ic - (e - k_i*(a - sigma[c])/(2m))) / m,  m = mass/2        */
/*                                                         (:454, :541-543)  */
/*   argmax starting from (0, src); ties -> smaller id when up, larger when */
/*   down (:544-575); version 2 clamps to min/max(dst, src) (:579-585).      */
/* Version 1 inserts only c < src (up) / c > src (down) and does not clamp */
/* (louvain_gl.cu:504, :578).                                               */
/* ======================================================================== */
static inline double lm_gain(double kic, double e, double ki, double a, double sc, double m) {
    double t = ki * (a - sc);
    t = t / (2.0 * m);
    t = e - t;
    double g = kic - t;
    return g / m;
}

static uint32_t max_row(const or_graph *g) {
    uint64_t md = 0;
    for (uint32_t i = 0; i < g->n; i++) {
        uint64_t d = g->offsets[i + 1] - g->offsets[i];
        if (d > md) md = d;
    }
    return (uint32_t)md;
}

static uint32_t pow2_at_least(uint64_t x) {
    uint32_t p = 16;
    while (p < x) p <<= 1;
    return p;
}

int or_local_move(const or_graph *g, int version, int up, const uint32_t *C,
                  const double *sigma_tot, const double *k, double mass,
                  uint32_t *C_new, uint64_t *distinct_pairs) {
    const double m = mass / 2.0;
    uint32_t cap = pow2_at_least(2ull * max_row(g) + 2);
    uint64_t dsum = 0;
#pragma omp parallel reduction(+ : dsum)
    {
        uint32_t *key = (uint32_t *)malloc(sizeof(uint32_t) * cap);
        double *val = (double *)malloc(sizeof(double) * cap);
        uint32_t *used = (uint32_t *)malloc(sizeof(uint32_t) * cap);
        for (uint32_t s = 0; s < cap; s++) key[s] = OR_EMPTY;
#pragma omp for schedule(dynamic, 512)
        for (uint32_t i = 0; i < g->n; i++) {
            uint32_t src = C[i];
            double ki = k[i];
            double a = sigma_tot[src] - ki;
            double e_src = 0;
            uint32_t nused = 0;
            uint64_t deg = g->offsets[i + 1] - g->offsets[i];
            uint32_t tcap = pow2_at_least(2 * deg + 2);
            uint32_t mask = tcap - 1;
            for (uint64_t e = g->offsets[i]; e < g->offsets[i + 1]; e++) {
                uint32_t j = g->cols[e];
                uint32_t c = C[j];
                double w = wt(g, e);
                int cand = version == 1 ? (up ? c < src : c > src) : c != src;
                if (cand) {
                    uint32_t h = (c * 2654435761u) & mask;
                    while (key[h] != OR_EMPTY && key[h] != c) h = (h + 1) & mask;
                    if (key[h] == OR_EMPTY) { key[h] = c; val[h] = 0; used[nused++] = h; }
                    val[h] += w;
                } else if (c == src && j != i) {
                    e_src += w;
                }
            }
            double best = 0.0;
            uint32_t dst = src;
            for (uint32_t u = 0; u < nused; u++) {
                uint32_t h = used[u];
                uint32_t c = key[h];
                double gn = lm_gain(val[h], e_src, ki, a, sigma_tot[c], m);
                if (gn > best || (gn == best && (up ? c < dst : c > dst))) { best = gn; dst = c; }
                key[h] = OR_EMPTY;
            }
            dsum += nused;
            if (version == 1) C_new[i] = dst;
            else C_new[i] = up ? (dst < src ? dst : src) : (dst > src ? dst : src);
        }
        free(key); free(val); free(used);
    }
    if (distinct_pairs) *distinct_pairs = dsum;
    return 0;
}

/* Sigma update from C -> C_new (louvain.cu:1299-1396): delta per community
 * accumulated over moved vertices in ascending order, then added. */
static void sigma_update(uint32_t n, const uint32_t *C, const uint32_t *Cn, const double *k,
                         double *sigma, double *delta) {
    memset(delta, 0, sizeof(double) * n);
    for (uint32_t v = 0; v < n; v++)
        if (C[v] != Cn[v]) { delta[C[v]] -= k[v]; delta[Cn[v]] += k[v]; }
    for (uint32_t c = 0; c < n; c++) sigma[c] += delta[c];
}

/* ======================================================================== */
/* Coarsening -- src/coarsen_graph/coarsen_graph_mg.cu:2054-2240.           */
/* relabel: flag used ids, inclusive scan, C' = scan[C]-1 (:211-226,        */
/* :267-286, :1330-1363).  Row r of the next level holds, for every        */
/* neighbour community c of the members of r (r itself included), the sum */
/* of the edge weights (:816-1125); the reference emits a row in hash-slot */
/* order, here rows are sorted by c.  Sums run over members in ascending   */
/* vertex id and edges in CSR order.                                        */
/* ======================================================================== */
int or_coarsen(const or_graph *g, const uint32_t *C, uint32_t *C_dense, or_graph *out,
               uint64_t *upper_degree) {
    uint32_t n = g->n;
    memset(out, 0, sizeof(*out));
    uint32_t *newid = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
    for (uint32_t v = 0; v < n; v++) {
        if (C[v] >= n) { free(newid); return -2; }
        newid[C[v]] = 1;
    }
    uint32_t nn = 0;
    for (uint32_t c = 0; c < n; c++) { uint32_t f = newid[c]; newid[c] = nn; nn += f; }
    uint32_t *cd = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t v = 0; v < n; v++) cd[v] = newid[C[v]];
    free(newid);
    /* members by community, ascending vertex id */
    uint64_t *moff = (uint64_t *)calloc((size_t)nn + 1, sizeof(uint64_t));
    for (uint32_t v = 0; v < n; v++) moff[cd[v] + 1]++;
    for (uint32_t r = 0; r < nn; r++) moff[r + 1] += moff[r];
    uint32_t *mem = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    {
        uint64_t *cur = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)nn + 1));
        memcpy(cur, moff, sizeof(uint64_t) * ((size_t)nn + 1));
        for (uint32_t v = 0; v < n; v++) mem[cur[cd[v]]++] = v;
        free(cur);
    }
    if (upper_degree) {
        upper_degree[0] = 0;
        for (uint32_t r = 0; r < nn; r++) {
            uint64_t s = 0;
            for (uint64_t p = moff[r]; p < moff[r + 1]; p++) s += g->offsets[mem[p] + 1] - g->offsets[mem[p]];
            upper_degree[r + 1] = upper_degree[r] + s;
        }
    }
    uint64_t *roff = (uint64_t *)calloc((size_t)nn + 1, sizeof(uint64_t));
    /* pass 1: distinct neighbour communities per row */
#pragma omp parallel
    {
        uint32_t cap = 16;
        uint32_t *key = (uint32_t *)malloc(sizeof(uint32_t) * cap);
        for (uint32_t s = 0; s < cap; s++) key[s] = OR_EMPTY;
#pragma omp for schedule(dynamic, 64)
        for (uint32_t r = 0; r < nn; r++) {
            uint64_t tot = 0;
            for (uint64_t p = moff[r]; p < moff[r + 1]; p++) tot += g->offsets[mem[p] + 1] - g->offsets[mem[p]];
            uint32_t need = pow2_at_least(2 * tot + 2);
            if (need > cap) {
                free(key); cap = need;
                key = (uint32_t *)malloc(sizeof(uint32_t) * cap);
                for (uint32_t s = 0; s < cap; s++) key[s] = OR_EMPTY;
            }
            uint32_t mask = need - 1, cnt = 0;
            for (uint64_t p = moff[r]; p < moff[r + 1]; p++) {
                uint32_t u = mem[p];
                for (uint64_t e = g->offsets[u]; e < g->offsets[u + 1]; e++) {
                    uint32_t c = cd[g->cols[e]];
                    uint32_t h = (c * 2654435761u) & mask;
                    while (key[h] != OR_EMPTY && key[h] != c) h = (h + 1) & mask;
                    if (key[h] == OR_EMPTY) { key[h] = c; cnt++; }
                }
            }
            roff[r + 1] = cnt;
            for (uint32_t s = 0; s < need; s++) key[s] = OR_EMPTY;
        }
        free(key);
    }
    for (uint32_t r = 0; r < nn; r++) roff[r + 1] += roff[r];
    uint64_t nnz = roff[nn];
    uint32_t *cols = (uint32_t *)malloc(sizeof(uint32_t) * (nnz ? nnz : 1));
    double *ws = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
    /* pass 2: sums, then sort the row by neighbour community */
#pragma omp parallel
    {
        uint32_t cap = 16;
        uint32_t *key = (uint32_t *)malloc(sizeof(uint32_t) * cap);
        double *val = (double *)malloc(sizeof(double) * cap);
        for (uint32_t s = 0; s < cap; s++) key[s] = OR_EMPTY;
#pragma omp for schedule(dynamic, 64)
        for (uint32_t r = 0; r < nn; r++) {
            uint64_t len = roff[r + 1] - roff[r];
            uint32_t need = pow2_at_least(2 * len + 2);
            if (need > cap) {
                free(key); free(val); cap = need;
                key = (uint32_t *)malloc(sizeof(uint32_t) * cap);
                val = (double *)malloc(sizeof(double) * cap);
                for (uint32_t s = 0; s < cap; s++) key[s] = OR_EMPTY;
            }
            uint32_t mask = need - 1;
            for (uint64_t p = moff[r]; p < moff[r + 1]; p++) {
                uint32_t u = mem[p];
                for (uint64_t e = g->offsets[u]; e < g->offsets[u + 1]; e++) {
                    uint32_t c = cd[g->cols[e]];
                    uint32_t h = (c * 2654435761u) & mask;
                    while (key[h] != OR_EMPTY && key[h] != c) h = (h + 1) & mask;
                    if (key[h] == OR_EMPTY) { key[h] = c; val[h] = 0; }
                    val[h] += wt(g, e);
                }
            }
            uint32_t *rc = cols + roff[r];
            uint64_t q = 0;
            for (uint32_t s = 0; s < need; s++)
                if (key[s] != OR_EMPTY) rc[q++] = key[s];
            qsort(rc, q, sizeof(uint32_t), cmp_u32);
            for (uint64_t t = 0; t < q; t++) {
                uint32_t c = rc[t];
                uint32_t h = (c * 2654435761u) & mask;
                while (key[h] != c) h = (h + 1) & mask;
                ws[roff[r] + t] = val[h];
            }
            for (uint32_t s = 0; s < need; s++) key[s] = OR_EMPTY;
        }
        free(key); free(val);
    }
    free(moff); free(mem);
    if (C_dense) memcpy(C_dense, cd, sizeof(uint32_t) * n);
    free(cd);
    out->n = nn;
    out->nnz = nnz;
    out->offsets = roff;
    out->cols = cols;
    out->weights = ws;
    return 0;
}

/* ======================================================================== */
/* Full Louvain -- src/louvain/louvain.cu:1401-1715.                        */
/* ======================================================================== */
static void trace_row(double *trace, int max_trace, int *rows, int phase, int loop, double q, double dq) {
    if (trace && *rows < max_trace) {
        double *t = trace + 4 * (*rows);
        t[0] = phase; t[1] = loop; t[2] = q; t[3] = dq;
    }
    (*rows)++;
}

static void compose_dense(uint32_t n0, uint32_t *assignment, const uint32_t *C, uint32_t n) {
    uint32_t *id = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
    for (uint32_t v = 0; v < n; v++) id[C[v]] = 1;
    uint32_t k = 0;
    for (uint32_t c = 0; c < n; c++) { uint32_t f = id[c]; id[c] = k; k += f; }
    for (uint32_t v = 0; v < n0; v++) assignment[v] = id[C[assignment[v]]];
    free(id);
}

int or_louvain(const or_graph *g0, int version, double threshold, int max_phases,
               uint32_t *assignment, double *trace, int max_trace,
               uint32_t *level_sizes, int max_levels, or_result *res) {
    memset(res, 0, sizeof(*res));
    double mass = or_mass(g0);
    int integral = or_is_integral(g0);
    uint32_t n0 = g0->n;
    for (uint32_t v = 0; v < n0; v++) assignment[v] = v;
    or_graph cur = *g0; /* borrowed at level 0 */
    int owned = 0;
    double Qh = 0, Qold = -1;
    int phase = 0, rows = 0, iters = 0, levels = 0;
    uint32_t *C = NULL, *Cn = NULL;
    while (phase < max_phases && (Qh - Qold) > threshold) {
        Qold = Qh;
        uint32_t n = cur.n;
        if (levels < max_levels && level_sizes) level_sizes[levels] = n;
        levels++;
        C = (uint32_t *)realloc(C, sizeof(uint32_t) * (n ? n : 1));
        Cn = (uint32_t *)realloc(Cn, sizeof(uint32_t) * (n ? n : 1));
        double *k = (double *)malloc(sizeof(double) * (n ? n : 1));
        double *sig = (double *)malloc(sizeof(double) * (n ? n : 1));
        double *delta = (double *)malloc(sizeof(double) * (n ? n : 1));
        for (uint32_t v = 0; v < n; v++) C[v] = v;
        or_vertex_weights(&cur, k);
        memcpy(sig, k, sizeof(double) * n);
        double newQ = or_modularity_sigma(&cur, C, sig, mass, integral);
        double curQ = newQ - 1;
        trace_row(trace, max_trace, &rows, phase, 0, newQ, 0.0);
        int up = 1, loop = 0;
        while ((newQ - curQ) > threshold) {
            curQ = newQ;
            or_local_move(&cur, version, up, C, sig, k, mass, Cn, NULL);
            up = !up;
            sigma_update(n, C, Cn, k, sig, delta);
            newQ = or_modularity_sigma(&cur, Cn, sig, mass, integral);
            if ((newQ - curQ) > threshold) memcpy(C, Cn, sizeof(uint32_t) * n);
            else newQ = curQ;
            loop++;
            iters++;
            trace_row(trace, max_trace, &rows, phase, loop, newQ, newQ - curQ);
        }
        free(k); free(sig); free(delta);
        Qh = newQ;
        if ((Qh - Qold) <= threshold) {
            compose_dense(n0, assignment, C, n);
            break;
        }
        or_graph nxt;
        uint32_t *cd = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
        or_coarsen(&cur, C, cd, &nxt, NULL);
        for (uint32_t v = 0; v < n0; v++) assignment[v] = cd[assignment[v]];
        free(cd);
        if (owned) or_graph_free(&cur);
        cur = nxt;
        owned = 1;
        phase++;
    }
    uint32_t ncom = 0;
    for (uint32_t v = 0; v < n0; v++) if (assignment[v] + 1 > ncom) ncom = assignment[v] + 1;
    if (owned) or_graph_free(&cur);
    free(C); free(Cn);
    res->modularity = Qh;
    res->phases = phase;
    res->levels = levels;
    res->iterations = iters;
    res->trace_rows = rows;
    res->communities = ncom;
    return 0;
}

double or_time_phase0(const or_graph *g, int version, int iters, uint64_t *edges_done) {
    uint32_t n = g->n;
    double mass = or_mass(g);
    int integral = or_is_integral(g);
    uint32_t *C = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint32_t *Cn = (uint32_t *)malloc(sizeof(uint32_t) * n);
    double *k = (double *)malloc(sizeof(double) * n);
    double *sig = (double *)malloc(sizeof(double) * n);
    double *delta = (double *)malloc(sizeof(double) * n);
    for (uint32_t v = 0; v < n; v++) C[v] = v;
    or_vertex_weights(g, k);
    memcpy(sig, k, sizeof(double) * n);
    double t0 = omp_get_wtime();
    int up = 1;
    volatile double sink = 0;
    for (int it = 0; it < iters; it++) {
        or_local_move(g, version, up, C, sig, k, mass, Cn, NULL);
        up = !up;
        sigma_update(n, C, Cn, k, sig, delta);
        sink += or_modularity_sigma(g, Cn, sig, mass, integral);
        memcpy(C, Cn, sizeof(uint32_t) * n);
    }
    double t1 = omp_get_wtime();
    (void)sink;
    free(C); free(Cn); free(k); free(sig); free(delta);
    if (edges_done) *edges_done = (uint64_t)iters * g->nnz;
    return t1 - t0;
}

/* ======================================================================== */
/* Check of the engine's division by a run constant: for divisor d with      */
/* r = RN(1/d), q0 = RN(x*r), rem = fma(-q0, d, x), q = fma(rem, r, q0)      */
/* equals RN(x/d) (Markstein's theorem).  Counts mismatches over n inputs   */
/* x drawn from the gain's value range for each divisor.                    */
/* ======================================================================== */
uint64_t or_check_const_division(uint64_t n, uint64_t seed, const double *divisors, int nd) {
    uint64_t bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (uint64_t i = 0; i < n; i++) {
        uint64_t h = or_mix64(seed + i);
        double d = divisors[i % (uint64_t)nd];
        double r = 1.0 / d;
        /* x: random mantissa, exponent spread over +-2^60 around d, both signs */
        int ex = (int)((h >> 52) % 121) - 60;
        double m = 1.0 + (double)(h & 0xFFFFFFFFFFFFFull) / 4503599627370496.0;
        double x = ldexp(m, ex) * d * ((h >> 63) ? -1.0 : 1.0);
        if (i % 7 == 0) x = (double)(int64_t)(h % 4000000000ull) - 2000000000.0; /* integers */
        double q0 = x * r;
        double rem = fma(-q0, d, x);
        double q = fma(rem, r, q0);
        if (q != x / d) bad++;
    }
    return bad;
}
