// spectral.cu -- the normalized graph Laplacian of the fuzzy graph and its
// smallest eigenpairs, the spectral stage that follows the fuzzy graph
// (src/sparse.rs:19-85, src/eigen.rs:31-238, called from spectral_layout_single
// at src/spectral.rs:70-83).
//
// Laplacian (bit-exact with the reference).  From the (row, col)-sorted COO:
//   indptr[r]  = first entry whose row is >= r (src/sparse.rs:21-35 counts rows;
//                on sorted rows both give the same offsets),
//   degree[i]  = sequential binary64 sum of the row's widened weights
//                (src/sparse.rs:57-61),
//   s[p]       = f64(w[p]) * ((1 / sqrt(degree[i])) * (1 / sqrt(degree[j])))
//                (src/sparse.rs:62-69),
// and L x = x - S x with each row's products summed in column order
// (src/sparse.rs:78-84).  Sums start from -0.0, the neutral element of the
// binary64 `Sum` of the reference's toolchain (Rust >= 1.93); it changes
// nothing but the sign of an exactly-zero sum.
//
// Eigenpairs.  Lanczos with locking and warm restarts on B = 2I - L
// following src/eigen.rs:95-223 step for step: the fixed hashed start vector,
// per-cycle Krylov dimension max(8k, 60) (at most n), alpha before the
// re-orthogonalisation, two orthogonalisation passes against the basis and
// the locked vectors, the 1e-12 breakdown test, Ritz pairs of the tridiagonal
// largest first, explicit residual ||B x - theta x|| < 1e-10 to lock, restart
// from the best unconverged Ritz vector, 200 cycles at most, and the
// canonical sign of each vector.  Where the device differs in operation order
// (dot products as fixed two-stage tree reductions; classical Gram-Schmidt,
// applied twice, in place of the modified form; the implicit QL method for
// the tridiagonal in place of nalgebra's SymmetricEigen) the eigenpairs agree
// with the reference to its own tolerances rather than bit for bit.  Every
// reduction has a fixed order, so a graph gives the same bits on every run
// (src/eigen.rs:337-344 asks that of the reference).  The reference uses a
// dense eigensolver when n <= 2000 (src/eigen.rs:31-37); this build runs the
// Lanczos path at every n, as the reference's own spectral parity test does
// for both paths (src/fixture_parity.rs:158-185).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "hm_internal.cuh"

namespace hm {

constexpr unsigned SP_FULL = 0xffffffffu;

// ------------------------------------------------------------- Laplacian

__global__ void csr_indptr_kernel(const uint32_t *__restrict__ rows, uint64_t nnz, uint64_t n,
                                  uint64_t *__restrict__ indptr) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r > n) return;
    uint64_t lo = 0, hi = nnz;
    while (lo < hi) {
        const uint64_t mid = lo + ((hi - lo) >> 1);
        if ((uint64_t)rows[mid] < r) lo = mid + 1;
        else hi = mid;
    }
    indptr[r] = lo;
}

__global__ void degree_kernel(const uint64_t *__restrict__ indptr, const float *__restrict__ vals, uint64_t n,
                              double *__restrict__ deg) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = -0.0;
    for (uint64_t p = indptr[i], e = indptr[i + 1]; p < e; ++p) s = __dadd_rn(s, (double)vals[p]);
    deg[i] = s;
}

__device__ __forceinline__ double inv_sqrt_rn(double d) { return __ddiv_rn(1.0, __dsqrt_rn(d)); }

__global__ void normalize_kernel(const uint32_t *__restrict__ rows, const uint32_t *__restrict__ cols,
                                 const float *__restrict__ vals, uint64_t nnz, const double *__restrict__ deg,
                                 double *__restrict__ svals) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    const double a = inv_sqrt_rn(deg[rows[p]]), b = inv_sqrt_rn(deg[cols[p]]);
    svals[p] = __dmul_rn((double)vals[p], __dmul_rn(a, b));
}

// One warp per row: the products of a 32-entry chunk are formed in parallel,
// then added into the row sum one after another in column order.  Writes
// y = L x; with `bop`, also w = 2 x - L x (the operator B of src/eigen.rs:129-131).
__global__ void __launch_bounds__(256) lap_matvec_kernel(const uint64_t *__restrict__ indptr,
                                                         const uint32_t *__restrict__ cols,
                                                         const double *__restrict__ svals, uint64_t n,
                                                         const double *__restrict__ x, double *__restrict__ y,
                                                         double *__restrict__ w) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;  // whole warps
    const uint64_t lo = indptr[i], hi = indptr[i + 1];
    double acc = -0.0;
    for (uint64_t c0 = lo; c0 < hi; c0 += 32) {
        const uint64_t p = c0 + lane;
        const double prod = p < hi ? __dmul_rn(svals[p], x[cols[p]]) : 0.0;
        const uint32_t cnt = hi - c0 < 32 ? (uint32_t)(hi - c0) : 32u;
        for (uint32_t s = 0; s < cnt; ++s) acc = __dadd_rn(acc, __shfl_sync(SP_FULL, prod, s));
    }
    if (lane == 0) {
        const double xi = x[i];
        const double lx = __dsub_rn(xi, acc);
        if (y) y[i] = lx;
        if (w) w[i] = __dsub_rn(__dmul_rn(2.0, xi), lx);
    }
}

// ---------------------------------------------------- Lanczos building blocks
// Dot products of the w vector with `nu` vectors U[u] (stride n), as fixed
// two-stage reductions: block b of the grid's x dimension sums a 2048-element
// chunk (8 strided elements per thread, then a fixed tree), and one warp per
// vector sums the chunk partials in a fixed order.

constexpr int SP_THREADS = 256, SP_PER_THREAD = 8, SP_CHUNK = SP_THREADS * SP_PER_THREAD;

__device__ __forceinline__ double warp_sum_fixed(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(SP_FULL, v, o));
    return v;
}

__global__ void __launch_bounds__(SP_THREADS) dots_partial_kernel(const double *__restrict__ U, uint32_t nu,
                                                                  const double *__restrict__ w, uint64_t n,
                                                                  double *__restrict__ partial) {
    __shared__ double red[SP_THREADS / 32];
    const uint32_t u = blockIdx.y;
    const uint64_t c0 = (uint64_t)blockIdx.x * SP_CHUNK;
    const double *uv = U + (uint64_t)u * n;
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < SP_PER_THREAD; ++q) {
        const uint64_t i = c0 + threadIdx.x + (uint64_t)q * SP_THREADS;
        if (i < n) s = __dadd_rn(s, __dmul_rn(uv[i], w[i]));
    }
    s = warp_sum_fixed(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < SP_THREADS / 32 ? red[threadIdx.x] : 0.0;
        t = warp_sum_fixed(t);
        if (threadIdx.x == 0) partial[(uint64_t)u * gridDim.x + blockIdx.x] = t;
    }
}

__global__ void dots_finish_kernel(const double *__restrict__ partial, uint32_t nchunk, uint32_t nu,
                                   double *__restrict__ out) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (u >= nu) return;
    double s = 0.0;
    for (uint32_t c = lane; c < nchunk; c += 32) s = __dadd_rn(s, partial[(uint64_t)u * nchunk + c]);
    s = warp_sum_fixed(s);
    if (lane == 0) out[u] = s;
}

// w[i] -= sum over u of c[u] * U[u][i], subtracted in order of u
__global__ void project_out_kernel(const double *__restrict__ U, uint32_t nu, const double *__restrict__ c,
                                   double *__restrict__ w, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = w[i];
    for (uint32_t u = 0; u < nu; ++u) a = __dsub_rn(a, __dmul_rn(c[u], U[(uint64_t)u * n + i]));
    w[i] = a;
}

// dst[i] = src[i] / s
__global__ void divide_kernel(const double *__restrict__ src, double s, double *__restrict__ dst, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __ddiv_rn(src[i], s);
}

// x[i] = sum over s of y[s] * V[s][i], added in order of s from 0
__global__ void combine_kernel(const double *__restrict__ V, uint32_t nb, const double *__restrict__ y,
                               double *__restrict__ x, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = 0.0;
    for (uint32_t s = 0; s < nb; ++s) a = __dadd_rn(a, __dmul_rn(y[s], V[(uint64_t)s * n + i]));
    x[i] = a;
}

// z[i] = 2 x[i] - (L x)[i] - theta x[i], the Ritz residual (src/eigen.rs:196-203)
__global__ void residual_kernel(const double *__restrict__ x, const double *__restrict__ lx, double theta,
                                double *__restrict__ z, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xi = x[i];
    z[i] = __dsub_rn(__dsub_rn(__dmul_rn(2.0, xi), lx[i]), __dmul_rn(theta, xi));
}

// ------------------------------------------------------ tridiagonal eigen (host)
// Eigenvalues and eigenvectors of the symmetric tridiagonal matrix with
// diagonal d[0..m) and off-diagonal e[0..m-1): the implicit QL method with
// Wilkinson shifts and plane rotations (Bowdler, Martin, Reinsch and
// Wilkinson, "The QR and QL algorithms for symmetric matrices", 1968; the
// tql2 procedure).  z (m x m, row-major) receives the eigenvectors as
// columns.  Returns false if an eigenvalue needs more than 60 sweeps.
static bool tridiag_eigen(std::vector<double> &d, std::vector<double> e, std::vector<double> &z) {
    const int m = (int)d.size();
    e.resize(m, 0.0);
    e[m - 1] = 0.0;
    z.assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; ++i) z[(size_t)i * m + i] = 1.0;
    for (int l = 0; l < m; ++l) {
        int iter = 0;
        for (;;) {
            int mm = l;
            for (; mm < m - 1; ++mm) {
                const double dd = std::fabs(d[mm]) + std::fabs(d[mm + 1]);
                if (std::fabs(e[mm]) <= DBL_EPSILON * dd) break;
            }
            if (mm == l) break;
            if (++iter > 60) return false;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[mm] - d[l] + e[l] / (g + std::copysign(r, g));
            double s = 1.0, c = 1.0, p = 0.0;
            bool deflated = false;
            for (int i = mm - 1; i >= l; --i) {
                double f = s * e[i];
                const double b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[mm] = 0.0;
                    deflated = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                for (int q = 0; q < m; ++q) {
                    f = z[(size_t)q * m + i + 1];
                    z[(size_t)q * m + i + 1] = s * z[(size_t)q * m + i] + c * f;
                    z[(size_t)q * m + i] = c * z[(size_t)q * m + i] - s * f;
                }
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[mm] = 0.0;
        }
    }
    return true;
}

// Knuth multiplicative hash in [0, 1) (src/eigen.rs:66-72)
static double hash01(uint64_t i, uint32_t salt) {
    const uint32_t h = ((uint32_t)i + salt) * 2654435761u;
    return (double)(h >> 8) / (double)(1u << 24);
}

// canonical sign (src/eigen.rs:74-90): the first component of largest
// magnitude (by more than 1e-15) is made positive
static void canonical_sign(double *v, uint64_t n) {
    uint64_t pivot = 0;
    for (uint64_t i = 0; i < n; ++i)
        if (std::fabs(v[i]) > std::fabs(v[pivot]) + 1e-15) pivot = i;
    if (v[pivot] < 0.0)
        for (uint64_t i = 0; i < n; ++i) v[i] = -v[i];
}

// Device state of one Lanczos run.
struct Lanczos {
    uint64_t n = 0;
    uint32_t k = 0, m = 0, rows_cap = 0, nchunk = 0;
    const uint64_t *indptr = nullptr;
    const uint32_t *cols = nullptr;
    const double *svals = nullptr;
    double *U = nullptr;     // locked vectors, then the cycle's basis (rows_cap x n)
    double *X = nullptr;     // Ritz vector candidates ((k + 1) x n)
    double *w = nullptr, *t = nullptr, *r = nullptr;
    double *partial = nullptr, *coef = nullptr, *scal = nullptr, *alphas = nullptr;
    cudaStream_t s = nullptr;

    int matvec_b(const double *x, double *lx, double *bx) {
        const unsigned blocks = (unsigned)((n * 32 + 255) / 256);
        lap_matvec_kernel<<<blocks, 256, 0, s>>>(indptr, cols, svals, n, x, lx, bx);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch();
        return HM_OK;
    }
    // out[0..nu) = U[0..nu) . v, on the device
    int dots(const double *Ub, uint32_t nu, const double *v, double *out) {
        if (nu == 0) return HM_OK;
        dots_partial_kernel<<<dim3(nchunk, nu), SP_THREADS, 0, s>>>(Ub, nu, v, n, partial);
        HM_CUDA_TRY(cudaGetLastError());
        dots_finish_kernel<<<(nu * 32 + 255) / 256, 256, 0, s>>>(partial, nchunk, nu, out);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch(2);
        return HM_OK;
    }
    int dot_host(const double *a, const double *b, double *out) {
        HM_TRY(dots(a, 1, b, scal));
        HM_CUDA_TRY(cudaMemcpyAsync(out, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        HM_CUDA_TRY(cudaStreamSynchronize(s));
        return HM_OK;
    }
    // v -= U[0..nu) (U . v), twice
    int orthogonalize(double *v, uint32_t nu) {
        if (nu == 0) return HM_OK;
        for (int pass = 0; pass < 2; ++pass) {
            HM_TRY(dots(U, nu, v, coef));
            project_out_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(U, nu, coef, v, n);
            HM_CUDA_TRY(cudaGetLastError());
            count_launch();
        }
        return HM_OK;
    }
    int divide(const double *src, double by, double *dst) {
        divide_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, by, dst, n);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch();
        return HM_OK;
    }
    int upload_hashed(double *dst, uint32_t salt, bool start) {
        std::vector<double> h(n);
        for (uint64_t i = 0; i < n; ++i) h[i] = start ? 1.0 + 0.01 * (hash01(i, 0) - 0.5) : hash01(i, salt) - 0.5;
        HM_CUDA_TRY(cudaMemcpyAsync(dst, h.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
        HM_CUDA_TRY(cudaStreamSynchronize(s));
        return HM_OK;
    }

    // src/eigen.rs:95-223; values_out / vectors_out (column-major n x found)
    int run(double *values_out, double *vectors_out, uint32_t *found_out, uint32_t *cycles_out) {
        const double LOCK_TOL = 1e-10;
        const uint32_t MAX_CYCLES = 200;
        std::vector<double> locked_vals;
        uint32_t L = 0;
        HM_TRY(upload_hashed(r, 0, true));
        uint32_t cycle = 0;
        std::vector<double> alpha_h, beta_h, z;
        while (L < k && cycle < MAX_CYCLES) {
            ++cycle;
            HM_TRY(orthogonalize(r, L));
            double rr = 0.0;
            HM_TRY(dot_host(r, r, &rr));
            const double rnorm = std::sqrt(rr);
            if (rnorm < 1e-12) {
                HM_TRY(upload_hashed(r, cycle, false));
                continue;
            }
            double *basis = U + (uint64_t)L * n;
            HM_TRY(divide(r, rnorm, basis));
            const uint32_t steps = (uint32_t)std::min<uint64_t>(m, n - L);
            beta_h.clear();
            uint32_t nsteps = 0;
            for (;;) {
                const uint32_t j = nsteps;
                const double *vj = basis + (uint64_t)j * n;
                HM_TRY(matvec_b(vj, t, w));
                HM_TRY(dots(vj, 1, w, alphas + j));
                ++nsteps;
                HM_TRY(orthogonalize(w, L + j + 1));
                if (nsteps == steps) break;
                double ww = 0.0;
                HM_TRY(dot_host(w, w, &ww));
                const double beta = std::sqrt(ww);
                if (beta < 1e-12) break;  // invariant subspace
                HM_TRY(divide(w, beta, basis + (uint64_t)(j + 1) * n));
                beta_h.push_back(beta);
            }
            // Ritz pairs of the tridiagonal, largest theta first
            alpha_h.assign(nsteps, 0.0);
            HM_CUDA_TRY(cudaMemcpyAsync(alpha_h.data(), alphas, nsteps * sizeof(double), cudaMemcpyDeviceToHost, s));
            HM_CUDA_TRY(cudaStreamSynchronize(s));
            std::vector<double> theta = alpha_h;
            if (!tridiag_eigen(theta, beta_h, z))
                return set_error(HM_ERR_UNSUPPORTED, "tridiagonal eigensolver did not converge");
            std::vector<uint32_t> order(nsteps);
            for (uint32_t q = 0; q < nsteps; ++q) order[q] = q;
            std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return theta[a] > theta[b]; });
            const uint32_t take = std::min<uint32_t>(nsteps, k - L + 1);
            std::vector<double> ycol(nsteps);
            std::vector<double> resid(take);
            for (uint32_t c = 0; c < take; ++c) {
                const uint32_t col = order[c];
                for (uint32_t q = 0; q < nsteps; ++q) ycol[q] = z[(size_t)q * nsteps + col];
                HM_CUDA_TRY(cudaMemcpyAsync(coef, ycol.data(), nsteps * sizeof(double), cudaMemcpyHostToDevice, s));
                double *xc = X + (uint64_t)c * n;
                combine_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(basis, nsteps, coef, xc, n);
                HM_CUDA_TRY(cudaGetLastError());
                count_launch();
                double xx = 0.0;
                HM_TRY(dot_host(xc, xc, &xx));
                HM_TRY(divide(xc, std::sqrt(xx), xc));
                HM_TRY(matvec_b(xc, t, nullptr));
                residual_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(xc, t, theta[col], w, n);
                HM_CUDA_TRY(cudaGetLastError());
                count_launch();
                double zz = 0.0;
                HM_TRY(dot_host(w, w, &zz));
                resid[c] = std::sqrt(zz);
            }
            // lock converged pairs; warm-restart from the best unconverged one
            bool have_next = false;
            for (uint32_t c = 0; c < take; ++c) {
                const double *xc = X + (uint64_t)c * n;
                if (resid[c] < LOCK_TOL && L < k) {
                    HM_CUDA_TRY(cudaMemcpyAsync(U + (uint64_t)L * n, xc, n * sizeof(double), cudaMemcpyDeviceToDevice,
                                                s));
                    locked_vals.push_back(2.0 - theta[order[c]]);
                    ++L;
                } else if (!have_next) {
                    HM_CUDA_TRY(cudaMemcpyAsync(r, xc, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
                    have_next = true;
                }
            }
            if (!have_next) HM_TRY(upload_hashed(r, cycle, false));
        }
        // ascending lambda, canonical orientation
        std::vector<uint32_t> idx(L);
        for (uint32_t q = 0; q < L; ++q) idx[q] = q;
        std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return locked_vals[a] < locked_vals[b]; });
        const uint32_t found = std::min(k, L);
        for (uint32_t j = 0; j < found; ++j) {
            values_out[j] = locked_vals[idx[j]];
            double *out = vectors_out + (uint64_t)j * n;
            HM_CUDA_TRY(cudaMemcpyAsync(out, U + (uint64_t)idx[j] * n, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        HM_CUDA_TRY(cudaStreamSynchronize(s));
        for (uint32_t j = 0; j < found; ++j) canonical_sign(vectors_out + (uint64_t)j * n, n);
        *found_out = found;
        if (cycles_out) *cycles_out = cycle;
        return HM_OK;
    }
};

static int laplacian_launch(const uint32_t *d_rows, const uint32_t *d_cols, const float *d_vals, uint64_t n,
                            uint64_t nnz, uint64_t *d_indptr, double *d_svals, double *d_degrees, cudaStream_t s) {
    csr_indptr_kernel<<<(unsigned)((n + 1 + 255) / 256), 256, 0, s>>>(d_rows, nnz, n, d_indptr);
    HM_CUDA_TRY(cudaGetLastError());
    degree_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_indptr, d_vals, n, d_degrees);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch(2);
    if (nnz) {
        normalize_kernel<<<(unsigned)((nnz + 255) / 256), 256, 0, s>>>(d_rows, d_cols, d_vals, nnz, d_degrees,
                                                                      d_svals);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch();
    }
    return HM_OK;
}

// Device bytes of an eigenpair run (beyond the Laplacian itself).
static size_t lanczos_bytes(uint64_t n, uint32_t k, uint32_t *m_out, uint32_t *rows_out, uint32_t *nchunk_out) {
    const uint32_t m = (uint32_t)std::min<uint64_t>(n, std::max<uint32_t>(8 * k, 60));
    const uint32_t rows = k + m + 1;
    const uint32_t nchunk = (uint32_t)((n + SP_CHUNK - 1) / SP_CHUNK);
    if (m_out) *m_out = m;
    if (rows_out) *rows_out = rows;
    if (nchunk_out) *nchunk_out = nchunk;
    return ((size_t)rows + k + 1 + 3) * n * 8 + (size_t)rows * nchunk * 8 + (size_t)rows * 8 * 3 + 4096;
}

}  // namespace hm

using namespace hm;

extern "C" {

int hm_laplacian_device(const uint32_t *d_rows, const uint32_t *d_cols, const float *d_vals, uint64_t n,
                        uint64_t nnz, uint64_t *d_indptr, double *d_svals, double *d_degrees, void *stream) {
    clear_error();
    if (!d_rows || !d_cols || !d_vals || !d_indptr || !d_svals || !d_degrees)
        return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0) return set_error(HM_ERR_INVALID, "empty graph");
    return laplacian_launch(d_rows, d_cols, d_vals, n, nnz, d_indptr, d_svals, d_degrees,
                            static_cast<cudaStream_t>(stream));
}

int hm_laplacian_matvec_device(const uint64_t *d_indptr, const uint32_t *d_cols, const double *d_svals,
                               uint64_t n, const double *d_x, double *d_y, void *stream) {
    clear_error();
    if (!d_indptr || !d_cols || !d_svals || !d_x || !d_y) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0) return set_error(HM_ERR_INVALID, "empty graph");
    const unsigned blocks = (unsigned)((n * 32 + 255) / 256);
    lap_matvec_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_indptr, d_cols, d_svals, n, d_x, d_y,
                                                                            nullptr);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

size_t hm_eigenpairs_workspace_bytes(uint64_t n, uint32_t k) {
    clear_error();
    if (n == 0 || k == 0 || k > n) {
        set_error(HM_ERR_INVALID, "need 1 <= k <= n");
        return 0;
    }
    if (k > 1024) {
        set_error(HM_ERR_UNSUPPORTED, "k above 1024");
        return 0;
    }
    return lanczos_bytes(n, k, nullptr, nullptr, nullptr);
}

int hm_eigenpairs_device(const uint64_t *d_indptr, const uint32_t *d_cols, const double *d_svals, uint64_t n,
                         uint32_t k, void *d_workspace, size_t workspace_bytes, void *stream, double *values_out,
                         double *vectors_out, uint32_t *found_out, uint32_t *cycles_out) {
    clear_error();
    if (!d_indptr || !d_cols || !d_svals || !d_workspace || !values_out || !vectors_out || !found_out)
        return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0 || k == 0 || k > n) return set_error(HM_ERR_INVALID, "need 1 <= k <= n");
    if (k > 1024) return set_error(HM_ERR_UNSUPPORTED, "k above 1024");
    if (n > 0xffffffffull) return set_error(HM_ERR_UNSUPPORTED, "n above 2^32 - 1");
    Lanczos lz;
    lz.n = n;
    lz.k = k;
    const size_t need = lanczos_bytes(n, k, &lz.m, &lz.rows_cap, &lz.nchunk);
    if (workspace_bytes < need)
        return set_error(HM_ERR_INVALID, "workspace of %zu bytes is below the %zu needed", workspace_bytes, need);
    if (reinterpret_cast<uintptr_t>(d_workspace) % 256) return set_error(HM_ERR_INVALID, "workspace must be 256-byte aligned");
    char *p = static_cast<char *>(d_workspace);
    auto take = [&](size_t bytes) {
        char *here = p;
        p += round_up(bytes, 256);
        return reinterpret_cast<double *>(here);
    };
    lz.U = take((size_t)lz.rows_cap * n * 8);
    lz.X = take((size_t)(k + 1) * n * 8);
    lz.w = take(n * 8);
    lz.t = take(n * 8);
    lz.r = take(n * 8);
    lz.partial = take((size_t)lz.rows_cap * lz.nchunk * 8);
    lz.coef = take((size_t)lz.rows_cap * 8);
    lz.alphas = take((size_t)lz.rows_cap * 8);
    lz.scal = take(64);
    lz.indptr = d_indptr;
    lz.cols = d_cols;
    lz.svals = d_svals;
    lz.s = static_cast<cudaStream_t>(stream);
    return lz.run(values_out, vectors_out, found_out, cycles_out);
}

int hm_spectral_eigenpairs(const uint32_t *rows, const uint32_t *cols, const float *vals, uint64_t n, uint64_t nnz,
                           uint32_t k, double *values_out, double *vectors_out, uint32_t *found_out,
                           uint32_t *cycles_out) {
    clear_error();
    if (!rows || !cols || !vals || !values_out || !vectors_out || !found_out)
        return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0 || k == 0 || k > n) return set_error(HM_ERR_INVALID, "need 1 <= k <= n");
    for (uint64_t p = 0; p < nnz; ++p) {
        if (rows[p] >= n || cols[p] >= n)
            return set_error(HM_ERR_INVALID, "entry %llu is outside the n x n graph", (unsigned long long)p);
        if (p && rows[p] < rows[p - 1])
            return set_error(HM_ERR_INVALID, "rows are not sorted at entry %llu", (unsigned long long)p);
    }
    const size_t ws = hm_eigenpairs_workspace_bytes(n, k);
    if (ws == 0) return HM_ERR_UNSUPPORTED;
    const size_t o_rows = 0, o_cols = round_up(nnz * 4 + 1, 256), o_vals = o_cols + round_up(nnz * 4 + 1, 256);
    const size_t o_ind = o_vals + round_up(nnz * 4 + 1, 256), o_sv = o_ind + round_up((n + 1) * 8, 256);
    const size_t o_deg = o_sv + round_up(nnz * 8 + 1, 256), o_ws = o_deg + round_up(n * 8, 256);
    char *d = nullptr;
    HM_CUDA_TRY(cudaMalloc(&d, o_ws + ws));
    int rc = HM_OK;
    do {
        cudaError_t err = cudaMemcpy(d + o_rows, rows, nnz * 4, cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemcpy(d + o_cols, cols, nnz * 4, cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemcpy(d + o_vals, vals, nnz * 4, cudaMemcpyHostToDevice);
        if (err != cudaSuccess) {
            rc = set_error(HM_ERR_CUDA, "copy in: %s", cudaGetErrorString(err));
            break;
        }
        auto *ind = reinterpret_cast<uint64_t *>(d + o_ind);
        auto *sv = reinterpret_cast<double *>(d + o_sv);
        rc = laplacian_launch(reinterpret_cast<uint32_t *>(d + o_rows), reinterpret_cast<uint32_t *>(d + o_cols),
                              reinterpret_cast<float *>(d + o_vals), n, nnz, ind, sv,
                              reinterpret_cast<double *>(d + o_deg), nullptr);
        if (rc != HM_OK) break;
        rc = hm_eigenpairs_device(ind, reinterpret_cast<uint32_t *>(d + o_cols), sv, n, k, d + o_ws, ws, nullptr,
                                  values_out, vectors_out, found_out, cycles_out);
    } while (false);
    cudaFree(d);
    return rc;
}

int hm_debug_tridiag_eigen(const double *d, const double *e, uint32_t m, double *vals_out, double *vecs_out) {
    clear_error();
    if (!d || !vals_out || !vecs_out || (m > 1 && !e) || m == 0) return set_error(HM_ERR_INVALID, "bad arguments");
    std::vector<double> dd(d, d + m), ee(e ? e : d, e ? e + (m - 1) : d), z;
    if (!tridiag_eigen(dd, ee, z)) return set_error(HM_ERR_UNSUPPORTED, "tridiagonal eigensolver did not converge");
    std::memcpy(vals_out, dd.data(), m * sizeof(double));
    std::memcpy(vecs_out, z.data(), (size_t)m * m * sizeof(double));
    return HM_OK;
}

}  // extern "C"
