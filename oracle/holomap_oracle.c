/*
 * holomap_oracle.c -- CPU restatement of holomap's exact kNN + smooth-kNN path
 * and of the fuzzy simplicial set that consumes it.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product is
 * compared against; it is never linked into libholomap_cuda.so and the product
 * never calls it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline / reference arm load it (through oracle/holomap_oracle.py).
 *
 * Every function restates one piece of the reference (mnmal-ai/holomap, Rust)
 * in the same binary32 / binary64 operation order, so that, compiled with
 * -ffp-contract=off and without -ffast-math, it reproduces the reference's
 * rounding step by step:
 *
 *   oracle_euclidean     src/metric.rs:42-53
 *   oracle_cosine        src/metric.rs:58-70
 *   oracle_manhattan     extension (no reference metric; same conventions)
 *   oracle_exact_knn     src/knn.rs:22-55   (self override :35-43, order :46-52)
 *   oracle_smooth_knn    src/smooth_knn.rs:23-80, mean :82-84
 *   oracle_expf          libm crate 0.2.16 `expf`, reached from
 *                        src/smooth_knn.rs:46 via src/fmath.rs:119-122
 *   oracle_fuzzy_graph   src/fuzzy.rs:25-91 (t-conorm :67-75)
 *   oracle_laplacian     src/sparse.rs:21-35, 56-71 (CSR, degrees, S)
 *   oracle_laplacian_matvec  src/sparse.rs:78-84
 *   oracle_lanczos       src/eigen.rs:95-238 (tridiagonal by Jacobi rotations:
 *                        nalgebra's SymmetricEigen is not available here)
 *
 * Parity pins: kNN indices and distances are checked against the reference's
 * own known-answer tests (src/knn.rs:64-105, src/metric.rs:92-102) and the
 * umap-learn golden fixtures tests/fixtures/stage2_*.json (indices exact,
 * values 1e-5).  rho/sigma are pinned to 1e-5 by src/smooth_knn.rs:104-124 and
 * the same fixtures.  The fuzzy graph is pinned by src/fuzzy.rs:97-155 and
 * the fixtures' graph_rows / graph_cols (exact) and graph_vals (1e-5,
 * src/fixture_parity.rs:101-117).  The Laplacian is pinned by
 * src/sparse.rs:116-160; the eigenpairs to the reference's tolerances by
 * src/eigen.rs:300-335 and the scipy eigenpairs of
 * tests/fixtures/spectral_cloud_connected.json (src/fixture_parity.rs:125-185).
 * The libm crate's source is not available here, so
 * oracle_expf restates its published algorithm (see the comment there); the
 * bit-level identity of sigma with the Rust binary is therefore unpinned
 * beyond those 1e-5 checks.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { ORACLE_EUCLIDEAN = 0, ORACLE_COSINE = 1, ORACLE_MANHATTAN = 2 };

/* ------------------------------------------------------------------ metrics */

/* src/metric.rs:42-53: per dimension d = f64(x) - f64(y); sq += d*d in
 * sequence; result = f32(sqrt(sq)). */
float oracle_euclidean(const float *a, const float *b, size_t d)
{
    double sq = 0.0;
    for (size_t t = 0; t < d; ++t) {
        double diff = (double)a[t] - (double)b[t];
        double p = diff * diff;
        sq = sq + p;
    }
    return (float)sqrt(sq);
}

/* Rust's f64::max(r, 0.0): returns the non-NaN operand when one is NaN. */
static double rust_max0(double r)
{
    if (isnan(r)) return 0.0;
    return r > 0.0 ? r : 0.0;
}

/* src/metric.rs:58-70: three sequential binary64 accumulators, then
 * (1 - dot / (sqrt(na) * sqrt(nb))).max(0.0) cast to f32. */
float oracle_cosine(const float *a, const float *b, size_t d)
{
    double dot = 0.0, na = 0.0, nb = 0.0;
    for (size_t t = 0; t < d; ++t) {
        double x = (double)a[t], y = (double)b[t];
        double xy = x * y, xx = x * x, yy = y * y;
        dot = dot + xy;
        na = na + xx;
        nb = nb + yy;
    }
    double den = sqrt(na) * sqrt(nb);
    double q = dot / den;
    double r = 1.0 - q;
    return (float)rust_max0(r);
}

/* Extension metric (the reference has none): sequential binary64 sum of
 * |f64(x) - f64(y)|, cast to f32 -- the same conventions as euclidean. */
float oracle_manhattan(const float *a, const float *b, size_t d)
{
    double s = 0.0;
    for (size_t t = 0; t < d; ++t) {
        double diff = (double)a[t] - (double)b[t];
        s = s + fabs(diff);
    }
    return (float)s;
}

typedef float (*metric_fn)(const float *, const float *, size_t);

static metric_fn pick_metric(int metric)
{
    switch (metric) {
    case ORACLE_EUCLIDEAN: return oracle_euclidean;
    case ORACLE_COSINE: return oracle_cosine;
    case ORACLE_MANHATTAN: return oracle_manhattan;
    default: return NULL;
    }
}

/* --------------------------------------------------------------- exact kNN */

/* f32::total_cmp as an unsigned key: negative values have all bits flipped,
 * non-negative values get the sign bit set.  (src/knn.rs:48) */
static uint32_t total_order_bits(float f)
{
    uint32_t b;
    memcpy(&b, &f, sizeof b);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

static float key_dist(uint64_t key)
{
    uint32_t t = (uint32_t)(key >> 32);
    uint32_t b = (t & 0x80000000u) ? (t & 0x7fffffffu) : ~t;
    float f;
    memcpy(&f, &b, sizeof f);
    return f;
}

static int cmp_u64(const void *x, const void *y)
{
    uint64_t a = *(const uint64_t *)x, b = *(const uint64_t *)y;
    return (a > b) - (a < b);
}

/* One row of src/knn.rs:31-53: all n distances (self forced to 0.0), a full
 * sort by (total_cmp(dist), index), then the first k.  `keys` is n-long
 * scratch. */
static void knn_row(const float *data, size_t n, size_t d, size_t k,
                    metric_fn dist, size_t i, uint64_t *keys,
                    uint32_t *idx_out, float *dist_out)
{
    const float *a = data + i * d;
    for (size_t j = 0; j < n; ++j) {
        float v = (j == i) ? 0.0f : dist(a, data + j * d, d);
        keys[j] = ((uint64_t)total_order_bits(v) << 32) | (uint64_t)(uint32_t)j;
    }
    qsort(keys, n, sizeof(uint64_t), cmp_u64);
    for (size_t t = 0; t < k; ++t) {
        idx_out[t] = (uint32_t)(keys[t] & 0xffffffffu);
        dist_out[t] = key_dist(keys[t]);
    }
}

/* src/knn.rs:22-55 for rows [row_begin, row_end); outputs are written at
 * (i - row_begin) * k.  Returns 0, or -1 on bad arguments / allocation. */
int oracle_exact_knn_rows(const float *data, size_t n, size_t d, size_t k,
                          int metric, size_t row_begin, size_t row_end,
                          uint32_t *idx_out, float *dist_out)
{
    metric_fn dist = pick_metric(metric);
    if (!dist || d == 0 || k == 0 || k > n || row_end > n || row_begin > row_end)
        return -1;
    uint64_t *keys = (uint64_t *)malloc(n * sizeof(uint64_t));
    if (!keys) return -1;
    for (size_t i = row_begin; i < row_end; ++i)
        knn_row(data, n, d, k, dist, i, keys, idx_out + (i - row_begin) * k,
                dist_out + (i - row_begin) * k);
    free(keys);
    return 0;
}

int oracle_exact_knn(const float *data, size_t n, size_t d, size_t k,
                     int metric, uint32_t *idx_out, float *dist_out)
{
    return oracle_exact_knn_rows(data, n, d, k, metric, 0, n, idx_out, dist_out);
}

/* Row-parallel variant used only as a timed CPU baseline: rows are split in
 * contiguous blocks over `threads` POSIX threads.  Each row's arithmetic is
 * identical to the serial path, so the outputs are the same bytes. */
struct mt_job {
    const float *data;
    size_t n, d, k, r0, r1, row_begin;
    int metric;
    uint32_t *idx;
    float *dist;
    int rc;
};

static void *mt_worker(void *p)
{
    struct mt_job *j = (struct mt_job *)p;
    j->rc = oracle_exact_knn_rows(j->data, j->n, j->d, j->k, j->metric, j->r0,
                                  j->r1, j->idx + (j->r0 - j->row_begin) * j->k,
                                  j->dist + (j->r0 - j->row_begin) * j->k);
    return NULL;
}

int oracle_exact_knn_rows_mt(const float *data, size_t n, size_t d, size_t k,
                             int metric, size_t row_begin, size_t row_end,
                             uint32_t *idx_out, float *dist_out, int threads)
{
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    size_t rows = row_end > row_begin ? row_end - row_begin : 0;
    if ((size_t)threads > rows) threads = rows ? (int)rows : 1;
    pthread_t tid[256];
    struct mt_job jobs[256];
    size_t per = rows / (size_t)threads, extra = rows % (size_t)threads, r = row_begin;
    for (int t = 0; t < threads; ++t) {
        size_t cnt = per + ((size_t)t < extra ? 1 : 0);
        jobs[t] = (struct mt_job){data, n, d, k, r, r + cnt, row_begin, metric,
                                  idx_out, dist_out, 0};
        r += cnt;
    }
    int started = 0;
    for (int t = 0; t < threads; ++t) {
        if (pthread_create(&tid[t], NULL, mt_worker, &jobs[t]) != 0) {
            mt_worker(&jobs[t]);
            tid[t] = 0;
        } else {
            ++started;
        }
    }
    int rc = 0;
    for (int t = 0; t < threads; ++t) {
        if (tid[t]) pthread_join(tid[t], NULL);
        if (jobs[t].rc) rc = jobs[t].rc;
    }
    (void)started;
    return rc;
}

/* ------------------------------------------------------------------- expf */

/*
 * oracle_expf: the libm crate (0.2.16, rust-lang) implements expf after
 * FreeBSD msun's e_expf.c, the Sun/FreeBSD single-precision method:
 *
 *   - |x| >= 88.7228 (positive) overflows to +inf (x * 2^127), x <= -103.972
 *     returns +0, NaN is returned unchanged;
 *   - x is reduced to r = x - k*ln2 with ln2 split in a 24-bit-exact head
 *     (0x3f317200) and a tail (0x35bfbe8e); k = 0 below |x| = ln2/2, k = +-1
 *     up to 1.5*ln2, otherwise the truncation of x/ln2 +- 1/2 (1/ln2 rounded
 *     to binary32, 0x3fb8aa3b);
 *   - |x| <= 2^-14 returns 1 + x directly;
 *   - exp(r) = 1 + (r*c/(2-c) - lo + hi) with c = r - r^2 (P1 + r^2 P2), the
 *     degree-2 minimax fit of r(e^r+1)/(e^r-1) on [-0.34568, 0.34568]
 *     (P1 = 0x3e2aaa8f, P2 = 0xbb355215);
 *   - the result is scaled by 2^k with a single final rounding (scalbnf).
 *
 * Every operation below is one binary32 operation with round-to-nearest, in
 * the order the method evaluates them; the CUDA port (smooth_knn.cu) performs
 * the same sequence with __f*_rn intrinsics.
 */
static float f32_from_bits(uint32_t b)
{
    float f;
    memcpy(&f, &b, sizeof f);
    return f;
}

static uint32_t f32_bits(float f)
{
    uint32_t b;
    memcpy(&b, &f, sizeof b);
    return b;
}

/* y * 2^n with a single rounding: scale toward the target by exact powers of
 * two while the intermediate stays normal, then one last multiply. */
static float oracle_scalbnf(float y, int n)
{
    if (n > 127) {
        y = y * f32_from_bits(0x7f000000u); /* 2^127 */
        n -= 127;
        if (n > 127) {
            y = y * f32_from_bits(0x7f000000u);
            n -= 127;
            if (n > 127) n = 127;
        }
    } else if (n < -126) {
        y = y * f32_from_bits(0x0c800000u); /* 2^-102 */
        n += 102;
        if (n < -126) {
            y = y * f32_from_bits(0x0c800000u);
            n += 102;
            if (n < -126) n = -126;
        }
    }
    return y * f32_from_bits((uint32_t)(0x7f + n) << 23);
}

float oracle_expf(float x)
{
    const float ln2_hi = f32_from_bits(0x3f317200u);
    const float ln2_lo = f32_from_bits(0x35bfbe8eu);
    const float inv_ln2 = f32_from_bits(0x3fb8aa3bu);
    const float p1 = f32_from_bits(0x3e2aaa8fu);
    const float p2 = f32_from_bits(0xbb355215u);

    uint32_t bits = f32_bits(x);
    int neg = (int)(bits >> 31);
    uint32_t mag = bits & 0x7fffffffu;

    if (mag >= 0x42aeac50u) {              /* |x| >= 87.33655 or NaN */
        if (mag > 0x7f800000u) return x;   /* NaN */
        if (!neg && mag >= 0x42b17218u)    /* x >= 88.72284: overflow */
            return x * f32_from_bits(0x7f000000u);
        if (neg && mag >= 0x42cff1b5u)     /* x <= -103.97208: underflow */
            return 0.0f;
    }

    float hi, lo, r;
    int k;
    if (mag > 0x3eb17218u) {               /* |x| > ln2/2 */
        if (mag > 0x3f851592u) {           /* |x| > 1.5 ln2 */
            float t = inv_ln2 * x;
            t = t + (neg ? -0.5f : 0.5f);
            k = (int)t;                    /* truncation toward zero */
        } else {
            k = neg ? -1 : 1;
        }
        float kf = (float)k;
        float khi = kf * ln2_hi;
        hi = x - khi;
        lo = kf * ln2_lo;
        r = hi - lo;
    } else if (mag > 0x39000000u) {        /* |x| > 2^-14 */
        k = 0;
        hi = x;
        lo = 0.0f;
        r = x;
    } else {
        return 1.0f + x;
    }

    float rr = r * r;
    float poly = rr * p2;
    poly = p1 + poly;
    poly = rr * poly;
    float c = r - poly;
    float num = r * c;
    float den = 2.0f - c;
    float q = num / den;
    q = q - lo;
    q = q + hi;
    float y = 1.0f + q;
    return k == 0 ? y : oracle_scalbnf(y, k);
}

/* ------------------------------------------------------------- smooth kNN */

/* src/smooth_knn.rs:82-84: f32(sequential f64 sum / f64(len)). */
float oracle_mean(const float *v, size_t len)
{
    double s = 0.0;
    for (size_t t = 0; t < len; ++t) s = s + (double)v[t];
    return (float)(s / (double)len);
}

/* One row of src/smooth_knn.rs:31-78.  `mean_all_floor` is
 * 1e-3f * mean_all (only read when the row has no positive distance). */
static void smooth_row(const float *row, size_t k, double target,
                       float mean_all, float *sigma_out, float *rho_out)
{
    const float min_k_dist_scale = 1e-3f;
    float rho = 0.0f;
    for (size_t t = 0; t < k; ++t) {
        if (row[t] > 0.0f) { rho = row[t]; break; }
    }
    float lo = 0.0f, hi = 3.40282347e38f /* f32::MAX */, mid = 1.0f;
    for (int it = 0; it < 64; ++it) {
        float psum = 0.0f;
        for (size_t t = 1; t < k; ++t) {
            float dd = row[t] - rho;
            if (dd > 0.0f) {
                float q = dd / mid;
                psum = psum + oracle_expf(-q);
            } else {
                psum = psum + 1.0f;
            }
        }
        double ps = (double)psum;
        if (fabs(ps - target) < 1e-5) break;
        if (ps > target) {
            hi = mid;
            mid = (lo + hi) / 2.0f;
        } else {
            lo = mid;
            if (hi >= 3.40282347e38f)
                mid = mid * 2.0f;
            else
                mid = (lo + hi) / 2.0f;
        }
    }
    float sigma = mid;
    float floor_v = rho > 0.0f ? min_k_dist_scale * oracle_mean(row, k)
                               : min_k_dist_scale * mean_all;
    if (sigma < floor_v) sigma = floor_v;
    *sigma_out = sigma;
    *rho_out = rho;
}

/* src/smooth_knn.rs:23-80.  target = log2(k) through the platform log2, as
 * Rust's f64::log2 does (src/smooth_knn.rs:25). */
int oracle_smooth_knn(const float *dists, size_t n, size_t k, float *sigma_out,
                      float *rho_out)
{
    if (k == 0 || n == 0) return -1;
    double target = log2((double)k);
    float mean_all = oracle_mean(dists, n * k);
    for (size_t i = 0; i < n; ++i)
        smooth_row(dists + i * k, k, target, mean_all, sigma_out + i, rho_out + i);
    return 0;
}

/* The same per-row arithmetic with an explicit mean_all, for checking rows of
 * a larger graph without re-reading all of it. */
int oracle_smooth_knn_rows(const float *dists, size_t rows, size_t k,
                           float mean_all, float *sigma_out, float *rho_out)
{
    if (k == 0) return -1;
    double target = log2((double)k);
    for (size_t i = 0; i < rows; ++i)
        smooth_row(dists + i * k, k, target, mean_all, sigma_out + i, rho_out + i);
    return 0;
}

double oracle_log2(double x) { return log2(x); }

void oracle_expf_array(const float *x, float *y, size_t n)
{
    for (size_t t = 0; t < n; ++t) y[t] = oracle_expf(x[t]);
}

/* -------------------------------------------------------------- fuzzy graph */

typedef struct {
    uint32_t r, c;
    float v;
} coo_t;

static int cmp_coo(const void *x, const void *y)
{
    const coo_t *a = (const coo_t *)x, *b = (const coo_t *)y;
    if (a->r != b->r) return a->r < b->r ? -1 : 1;
    if (a->c != b->c) return a->c < b->c ? -1 : 1;
    return 0;
}

/* Value of directed entry (r, c), 0 when absent (src/fuzzy.rs:52-57: a binary
 * search over the (row, col)-sorted directed list). */
static float lookup(const coo_t *dir, size_t m, uint32_t r, uint32_t c)
{
    size_t lo = 0, hi = m;
    while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if (dir[mid].r < r || (dir[mid].r == r && dir[mid].c < c)) lo = mid + 1;
        else hi = mid;
    }
    return (lo < m && dir[lo].r == r && dir[lo].c == c) ? dir[lo].v : 0.0f;
}

/* src/fuzzy.rs:25-91.  Directed strengths (self edges skipped,
 * w = 1 when d - rho <= 0 or sigma == 0, else expf(-(d / sigma)), zeros
 * dropped), sorted by (row, col); the support is the union of (r, c) and
 * (c, r) over them, deduplicated and sorted; each support entry gets the
 * binary32 t-conorm (v + vt) - v * vt and is kept when nonzero.  Outputs hold
 * up to 2 n k entries; returns the entry count, or -1 on allocation failure. */
long long oracle_fuzzy_graph(const uint32_t *idx, const float *dist, const float *sigma,
                             const float *rho, size_t n, size_t k, uint32_t *rows_out,
                             uint32_t *cols_out, float *vals_out)
{
    coo_t *dir = (coo_t *)malloc(sizeof(coo_t) * (n * k + 1));
    coo_t *sup = (coo_t *)malloc(sizeof(coo_t) * (2 * n * k + 1));
    if (!dir || !sup) {
        free(dir);
        free(sup);
        return -1;
    }
    size_t m = 0;
    for (size_t i = 0; i < n; ++i) {
        for (size_t j = 0; j < k; ++j) {
            uint32_t col = idx[i * k + j];
            if ((size_t)col == i) continue;
            volatile float d = dist[i * k + j] - rho[i];
            float val;
            if (d <= 0.0f || sigma[i] == 0.0f) {
                val = 1.0f;
            } else {
                volatile float q = d / sigma[i];
                val = oracle_expf(-q);
            }
            if (val != 0.0f) {
                dir[m].r = (uint32_t)i;
                dir[m].c = col;
                dir[m].v = val;
                ++m;
            }
        }
    }
    qsort(dir, m, sizeof(coo_t), cmp_coo);
    size_t s = 0;
    for (size_t e = 0; e < m; ++e) {
        sup[s].r = dir[e].r;
        sup[s].c = dir[e].c;
        ++s;
        sup[s].r = dir[e].c;
        sup[s].c = dir[e].r;
        ++s;
    }
    qsort(sup, s, sizeof(coo_t), cmp_coo);
    long long out = 0;
    for (size_t e = 0; e < s; ++e) {
        if (e > 0 && sup[e].r == sup[e - 1].r && sup[e].c == sup[e - 1].c) continue;  /* dedup */
        float v = lookup(dir, m, sup[e].r, sup[e].c);
        float vt = lookup(dir, m, sup[e].c, sup[e].r);
        volatile float sum = v + vt;
        volatile float prod = v * vt;
        float w = sum - prod;
        if (w != 0.0f) {
            rows_out[out] = sup[e].r;
            cols_out[out] = sup[e].c;
            vals_out[out] = w;
            ++out;
        }
    }
    free(dir);
    free(sup);
    return out;
}

/* ---------------------------------------------------- spectral stage */

/* Csr::from_fuzzy + Laplacian::new (src/sparse.rs:21-35, 56-71): indptr
 * (n + 1) by counting rows, degrees as sequential binary64 sums of the
 * widened weights, s[p] = w[p] * (inv_sqrt[i] * inv_sqrt[j]).  Sums start
 * from -0.0, the neutral element of the binary64 Sum of Rust >= 1.93. */
int oracle_laplacian(const uint32_t *rows, const uint32_t *cols, const float *vals, size_t n, size_t nnz,
                     uint64_t *indptr, double *svals, double *degrees) {
    double *inv = (double *)malloc((n ? n : 1) * sizeof(double));
    if (!inv) return -1;
    memset(indptr, 0, (n + 1) * sizeof(uint64_t));
    for (size_t p = 0; p < nnz; ++p) indptr[rows[p] + 1] += 1;
    for (size_t i = 0; i < n; ++i) indptr[i + 1] += indptr[i];
    for (size_t i = 0; i < n; ++i) {
        double s = -0.0;
        for (uint64_t p = indptr[i]; p < indptr[i + 1]; ++p) s += (double)vals[p];
        degrees[i] = s;
        inv[i] = 1.0 / sqrt(s);
    }
    for (size_t i = 0; i < n; ++i)
        for (uint64_t p = indptr[i]; p < indptr[i + 1]; ++p)
            svals[p] = (double)vals[p] * (inv[i] * inv[cols[p]]);
    free(inv);
    return 0;
}

/* Laplacian::matvec (src/sparse.rs:78-84): y = x - S x, row sums in order */
void oracle_laplacian_matvec(const uint64_t *indptr, const uint32_t *cols, const double *svals, size_t n,
                             const double *x, double *y) {
    for (size_t i = 0; i < n; ++i) {
        double s = -0.0;
        for (uint64_t p = indptr[i]; p < indptr[i + 1]; ++p) s += svals[p] * x[cols[p]];
        y[i] = x[i] - s;
    }
}

/* src/eigen.rs:225-227 */
static double sp_dot(const double *a, const double *b, size_t n) {
    double s = -0.0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* src/eigen.rs:66-72 */
static double sp_hash01(size_t i, uint32_t salt) {
    uint32_t h = ((uint32_t)i + salt) * 2654435761u;
    return (double)(h >> 8) / (double)(1u << 24);
}

/* Eigenpairs of a small symmetric matrix a (m x m, row-major, destroyed) by
 * cyclic Jacobi rotations; vals[m], vecs (m x m, row-major, eigenvectors as
 * columns).  Stands in for nalgebra's SymmetricEigen, whose source is not
 * available here: the eigenpairs agree to rounding, not bit for bit. */
static void sp_jacobi(int m, double *a, double *vals, double *vecs) {
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) vecs[i * m + j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        int rotated = 0;
        for (int p = 0; p < m; ++p)
            for (int q = p + 1; q < m; ++q) {
                double apq = a[p * m + q];
                if (fabs(apq) <= 1e-300 || fabs(apq) <= 1e-18 * (fabs(a[p * m + p]) + fabs(a[q * m + q]))) {
                    a[p * m + q] = a[q * m + p] = 0.0;
                    continue;
                }
                rotated = 1;
                double theta = (a[q * m + q] - a[p * m + p]) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int r = 0; r < m; ++r) {
                    double arp = a[r * m + p], arq = a[r * m + q];
                    a[r * m + p] = c * arp - s * arq;
                    a[r * m + q] = s * arp + c * arq;
                }
                for (int r = 0; r < m; ++r) {
                    double apr = a[p * m + r], aqr = a[q * m + r];
                    a[p * m + r] = c * apr - s * aqr;
                    a[q * m + r] = s * apr + c * aqr;
                }
                for (int r = 0; r < m; ++r) {
                    double vrp = vecs[r * m + p], vrq = vecs[r * m + q];
                    vecs[r * m + p] = c * vrp - s * vrq;
                    vecs[r * m + q] = s * vrp + c * vrq;
                }
            }
        if (!rotated) break;
    }
    for (int i = 0; i < m; ++i) vals[i] = a[i * m + i];
}

/* lanczos_eigenpairs (src/eigen.rs:95-223) with canonical_sign (:74-90):
 * modified Gram-Schmidt twice against the basis then the locked vectors,
 * sequential dot products, the same start vector, restarts, lock test and
 * cycle bound (max_cycles; the reference's is 200).  values[k] ascending,
 * vectors column-major n x k.  Returns
 * the number of pairs found, -1 on allocation failure; *cycles_out gets the
 * cycle count. */
long long oracle_lanczos(const uint64_t *indptr, const uint32_t *cols, const double *svals, size_t n, size_t k,
                         size_t max_cycles, double *values, double *vectors, size_t *cycles_out) {
    size_t m = 8 * k > 60 ? 8 * k : 60;
    if (m > n) m = n;
    const double LOCK_TOL = 1e-10;
    const size_t MAX_CYCLES = max_cycles; /* 200 in the reference; smaller for timing samples */
    double *locked = (double *)malloc(k * n * sizeof(double));
    double *lvals = (double *)malloc(k * sizeof(double));
    double *basis = (double *)malloc((m + 1) * n * sizeof(double));
    double *tmp = (double *)malloc(n * sizeof(double));
    double *w = (double *)malloc(n * sizeof(double));
    double *r = (double *)malloc(n * sizeof(double));
    double *x = (double *)malloc(n * sizeof(double));
    double *alphas = (double *)malloc(m * sizeof(double));
    double *betas = (double *)malloc(m * sizeof(double));
    double *T = (double *)malloc(m * m * sizeof(double));
    double *ev = (double *)malloc(m * sizeof(double));
    double *Z = (double *)malloc(m * m * sizeof(double));
    size_t *order = (size_t *)malloc(m * sizeof(size_t));
    if (!locked || !lvals || !basis || !tmp || !w || !r || !x || !alphas || !betas || !T || !ev || !Z || !order)
        return -1;
    size_t nl = 0, cycle = 0;
    for (size_t i = 0; i < n; ++i) r[i] = 1.0 + 0.01 * (sp_hash01(i, 0) - 0.5);
    int have_r = 1;
    while (nl < k && cycle < MAX_CYCLES) {
        ++cycle;
        if (!have_r)
            for (size_t i = 0; i < n; ++i) r[i] = sp_hash01(i, (uint32_t)(cycle - 1)) - 0.5;
        have_r = 1;
        for (int pass = 0; pass < 2; ++pass)
            for (size_t u = 0; u < nl; ++u) {
                double c = sp_dot(r, locked + u * n, n);
                for (size_t i = 0; i < n; ++i) r[i] -= c * locked[u * n + i];
            }
        double rnorm = sqrt(sp_dot(r, r, n));
        if (rnorm < 1e-12) {
            for (size_t i = 0; i < n; ++i) r[i] = sp_hash01(i, (uint32_t)cycle) - 0.5;
            continue;
        }
        for (size_t i = 0; i < n; ++i) basis[i] = r[i] / rnorm;
        size_t steps = m < n - nl ? m : n - nl;
        size_t na = 0, nb = 0;
        for (;;) {
            size_t j = na;
            const double *vj = basis + j * n;
            oracle_laplacian_matvec(indptr, cols, svals, n, vj, tmp);
            for (size_t i = 0; i < n; ++i) w[i] = 2.0 * vj[i] - tmp[i];
            alphas[na++] = sp_dot(w, vj, n);
            for (int pass = 0; pass < 2; ++pass) {
                for (size_t u = 0; u <= j; ++u) {
                    double c = sp_dot(w, basis + u * n, n);
                    for (size_t i = 0; i < n; ++i) w[i] -= c * basis[u * n + i];
                }
                for (size_t u = 0; u < nl; ++u) {
                    double c = sp_dot(w, locked + u * n, n);
                    for (size_t i = 0; i < n; ++i) w[i] -= c * locked[u * n + i];
                }
            }
            if (na == steps) break;
            double beta = sqrt(sp_dot(w, w, n));
            if (beta < 1e-12) break;
            for (size_t i = 0; i < n; ++i) basis[(j + 1) * n + i] = w[i] / beta;
            betas[nb++] = beta;
        }
        size_t t = na;
        for (size_t i = 0; i < t * t; ++i) T[i] = 0.0;
        for (size_t i = 0; i < t; ++i) T[i * t + i] = alphas[i];
        for (size_t i = 0; i < nb; ++i) T[i * t + i + 1] = T[(i + 1) * t + i] = betas[i];
        sp_jacobi((int)t, T, ev, Z);
        for (size_t i = 0; i < t; ++i) order[i] = i;
        for (size_t i = 1; i < t; ++i) { /* stable insertion sort, descending */
            size_t v = order[i], j = i;
            while (j > 0 && ev[order[j - 1]] < ev[v]) { order[j] = order[j - 1]; --j; }
            order[j] = v;
        }
        size_t take = k - nl + 1;
        if (take > t) take = t;
        int next = 0;
        for (size_t c = 0; c < take; ++c) {
            size_t col = order[c];
            double theta = ev[col];
            for (size_t i = 0; i < n; ++i) x[i] = 0.0;
            for (size_t s = 0; s < t; ++s) {
                double cf = Z[s * t + col];
                for (size_t i = 0; i < n; ++i) x[i] += cf * basis[s * n + i];
            }
            double nx = sqrt(sp_dot(x, x, n));
            for (size_t i = 0; i < n; ++i) x[i] /= nx;
            oracle_laplacian_matvec(indptr, cols, svals, n, x, tmp);
            double res = -0.0;
            for (size_t i = 0; i < n; ++i) {
                double e = 2.0 * x[i] - tmp[i] - theta * x[i];
                res += e * e;
            }
            res = sqrt(res);
            if (res < LOCK_TOL && nl < k) {
                memcpy(locked + nl * n, x, n * sizeof(double));
                lvals[nl++] = 2.0 - theta;
            } else if (!next) {
                memcpy(r, x, n * sizeof(double));
                next = 1;
            }
        }
        if (!next) have_r = 0;
    }
    /* ascending lambda (stable), canonical sign */
    size_t *idx = order; /* m >= k */
    size_t found = nl < k ? nl : k;
    size_t *ord2 = (size_t *)malloc((nl ? nl : 1) * sizeof(size_t));
    for (size_t i = 0; i < nl; ++i) ord2[i] = i;
    for (size_t i = 1; i < nl; ++i) {
        size_t v = ord2[i], j = i;
        while (j > 0 && lvals[ord2[j - 1]] > lvals[v]) { ord2[j] = ord2[j - 1]; --j; }
        ord2[j] = v;
    }
    (void)idx;
    for (size_t j = 0; j < found; ++j) {
        values[j] = lvals[ord2[j]];
        double *out = vectors + j * n;
        memcpy(out, locked + ord2[j] * n, n * sizeof(double));
        size_t pivot = 0;
        for (size_t i = 0; i < n; ++i)
            if (fabs(out[i]) > fabs(out[pivot]) + 1e-15) pivot = i;
        if (out[pivot] < 0.0)
            for (size_t i = 0; i < n; ++i) out[i] = -out[i];
    }
    free(ord2);
    free(locked); free(lvals); free(basis); free(tmp); free(w); free(r); free(x);
    free(alphas); free(betas); free(T); free(ev); free(Z); free(order);
    if (cycles_out) *cycles_out = cycle;
    return (long long)found;
}
