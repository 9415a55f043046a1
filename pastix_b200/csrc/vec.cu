// Vector kernels for the solve glue and the refinement (sm_100a).
//
//   k_spmv        y = alpha*A*x + beta*y on the permuted matrix in CSR, FP64
//                 (bcsc_zspmv, bcsc/bcsc_zspmv.c:629; the bcsc stores A by
//                 columns, its NoTrans product on the transposed values is
//                 the row product computed here)
//   k_dot_part    deterministic two-pass reductions for dot and nrm2
//                 (bvec_zdotc / bvec_znrm2, bcsc/bvec_zcompute.c:71,561)
//   k_axpy/scal   bvec_zaxpy / bvec_zscal (bcsc/bvec_zcompute.c:398,259)
//   k_gemv        x += W y with a small dense y (bvec_zgemv, :1112)
//   k_permute     b_perm[perm[i]] = b[i] and back (bvec_zlapmr, bcsc/bvec_zlapmr.c:668)
//   k_cast        FP64 <-> FP32 copies (pastixRhsDoubletoSingle, sopalin/pastix_rhs.c:162)
//   k_sampled     G[e] = alpha * l[row(e)] * x[col(e)] over the matrix pattern
//                 (adjoint of the values, no counterpart in the reference)
#include <cuda_runtime.h>
#include <cstdint>

#include <algorithm>
#include <vector>

namespace pgpu {

// SpMV with a group of G lanes per row.
template <int G>
__global__ void k_spmv(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                       const double *__restrict__ val, double alpha, const double *__restrict__ x, double beta,
                       double *__restrict__ y) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int lane = threadIdx.x % G;
    double acc = 0.0;
    if (gid < n) {
        const int b = rowptr[gid], e = rowptr[gid + 1];
        for (int p = b + lane; p < e; p += G) acc += val[p] * x[col[p]];
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, G);
    if (lane == 0 && gid < n) y[gid] = alpha * acc + (beta == 0.0 ? 0.0 : beta * y[gid]);
}

// SpMV by row blocks of at most SPMV_ROWS rows and SPMV_CAP stored entries
// (partition `part`, built once on the host by spmv_partition): the block's
// products val[p] * x[col[p]] are formed with fully coalesced loads of val and
// col into shared memory, then each thread sums one row of them.  A row longer
// than SPMV_CAP gets a block of its own, reduced by the whole block.
constexpr int SPMV_ROWS = 256, SPMV_CAP = 2304;
__global__ void __launch_bounds__(256) k_spmv_stream(const int *__restrict__ part, const int *__restrict__ rowptr,
                                                     const int *__restrict__ col, const double *__restrict__ val,
                                                     double alpha, const double *__restrict__ x, double beta,
                                                     double *__restrict__ y) {
    __shared__ double prod[SPMV_CAP];
    __shared__ double red[8];
    const int r0 = part[blockIdx.x], r1 = part[blockIdx.x + 1];
    const int p0 = rowptr[r0], p1 = rowptr[r1];
    const int tid = threadIdx.x;
    if (p1 - p0 <= SPMV_CAP) {
#pragma unroll 3
        for (int p = p0 + tid; p < p1; p += 256) prod[p - p0] = val[p] * x[col[p]];
        __syncthreads();
        const int r = r0 + tid;
        if (r < r1) {
            const int b = rowptr[r] - p0, e = rowptr[r + 1] - p0;
            double acc = 0.0;
            for (int q = b; q < e; q++) acc += prod[q];
            y[r] = alpha * acc + (beta == 0.0 ? 0.0 : beta * y[r]);
        }
    } else {  // one long row
        double acc = 0.0;
        for (int p = p0 + tid; p < p1; p += 256) acc += val[p] * x[col[p]];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if ((tid & 31) == 0) red[tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < 8; w++) t += red[w];
            y[r0] = alpha * t + (beta == 0.0 ? 0.0 : beta * y[r0]);
        }
    }
}

constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 296;  // 2 x 148 SMs

// per-block partial sums of a[i]*b[i] (b == a gives a squared norm)
__global__ void k_dot_part(int64_t n, const double *__restrict__ a, const double *__restrict__ b,
                           double *__restrict__ part) {
    __shared__ double sh[RED_THREADS / 32];
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += a[i] * b[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < RED_THREADS / 32) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) part[blockIdx.x] = v;
    }
}

// final reduction of the partials in a fixed order; out = sum (or sqrt(sum))
__global__ void k_dot_final(const double *__restrict__ part, int np, int do_sqrt, double *out) {
    __shared__ double sh[RED_THREADS / 32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += part[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < RED_THREADS / 32) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) *out = do_sqrt ? sqrt(v) : v;
    }
}

__global__ void k_axpy(int64_t n, double alpha, const double *__restrict__ x, double *__restrict__ y) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += alpha * x[i];
}
// y = x + beta * y
__global__ void k_xpby(int64_t n, const double *__restrict__ x, double beta, double *__restrict__ y) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = x[i] + beta * y[i];
}
__global__ void k_scal(int64_t n, double alpha, double *__restrict__ x) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] *= alpha;
}
// x += W[:, 0:m] * yv  (W column major, ld = n, yv in device memory)
__global__ void k_gemv(int64_t n, int m, const double *__restrict__ W, const double *__restrict__ yv,
                       double *__restrict__ x) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < m; j++) acc += W[i + (int64_t)j * n] * yv[j];
        x[i] += acc;
    }
}

// dst[perm[i] + j*ldd] = src[i + j*lds] (forward) or dst[i] = src[perm[i]] (backward)
template <typename TS, typename TD>
__global__ void k_permute(int n, int nrhs, const int64_t *__restrict__ perm, int forward, const TS *__restrict__ src,
                          int64_t lds, TD *__restrict__ dst, int64_t ldd) {
    int64_t tot = (int64_t)n * nrhs;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(e % n);
        int64_t j = e / n;
        if (forward) dst[perm[i] + j * ldd] = (TD)src[i + j * lds];
        else dst[i + j * ldd] = (TD)src[perm[i] + j * lds];
    }
}

template <typename TS, typename TD>
__global__ void k_cast(int64_t n, const TS *__restrict__ src, TD *__restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (TD)src[i];
}

// G[e] = alpha * l[row[e]] * x[col[e]] for the stored entries e of the matrix;
// with symmetric storage an off-diagonal entry stands for a_ij and a_ji and
// collects both terms.
__global__ void k_sampled(int64_t nnz, const int *__restrict__ erow, const int *__restrict__ ecol, double alpha,
                          const double *__restrict__ l, const double *__restrict__ x, double *__restrict__ G,
                          int sym) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = erow[e], j = ecol[e];
        double v = l[i] * x[j];
        if (sym && i != j) v += l[j] * x[i];
        G[e] = alpha * v;
    }
}

// ------------------------------ launchers ---------------------------------
static inline int nblk(int64_t n, int t = 256) {
    int64_t b = (n + t - 1) / t;
    return (int)(b < 148 * 32 ? (b < 1 ? 1 : b) : 148 * 32);
}

// ---------------------------------------------------------------------------
// Column-batched vector kernels of the batched GMRES (one Krylov process per
// right-hand side, all columns advanced together; refinement/z_refine_gmres.c
// applied to a block of columns).  A block of nb columns has leading
// dimension ld; per-column scalars live in device memory, so a Gram-Schmidt
// step needs no host round trip.
// ---------------------------------------------------------------------------
constexpr int SPMM_CB = 8;  // columns per CTA row of k_spmm (A read once per 8 columns)

// Y[:, c] = alpha A X[:, c] + beta Y[:, c] for the CTA's SPMM_CB columns.
template <int G>
__global__ void k_spmm(int n, int nb, const int *__restrict__ rowptr, const int *__restrict__ col,
                       const double *__restrict__ val, double alpha, const double *__restrict__ X, int64_t ldx,
                       double beta, double *__restrict__ Y, int64_t ldy) {
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int lane = threadIdx.x % G;
    const int c0 = blockIdx.y * SPMM_CB;
    double acc[SPMM_CB];
#pragma unroll
    for (int c = 0; c < SPMM_CB; c++) acc[c] = 0.0;
    if (gid < n) {
        const int b = rowptr[gid], e = rowptr[gid + 1];
        for (int p = b + lane; p < e; p += G) {
            const double a = val[p];
            const int64_t j = col[p];
#pragma unroll
            for (int c = 0; c < SPMM_CB; c++)
                if (c0 + c < nb) acc[c] += a * X[j + (int64_t)(c0 + c) * ldx];
        }
    }
#pragma unroll
    for (int c = 0; c < SPMM_CB; c++)
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o, G);
    if (lane == 0 && gid < n) {
#pragma unroll
        for (int c = 0; c < SPMM_CB; c++) {
            if (c0 + c >= nb) break;
            double *y = Y + gid + (int64_t)(c0 + c) * ldy;
            *y = alpha * acc[c] + (beta == 0.0 ? 0.0 : beta * *y);
        }
    }
}

// out[j * nb + c] = sum_i A_j[i, c] B[i, c] for the J blocks A_j = A + j * sA
// (sqrt of it when do_sqrt); one CTA per (column, block), fixed-order
// reductions (deterministic).
__global__ void k_dots_cols(int64_t n, int nb, const double *__restrict__ A, int64_t sA, int64_t lda,
                            const double *__restrict__ B, int64_t ldb, int do_sqrt, double *__restrict__ out) {
    __shared__ double sh[32];
    const int c = blockIdx.x, j = blockIdx.y;
    const double *a = A + (int64_t)j * sA + (int64_t)c * lda;
    const double *b = B + (int64_t)c * ldb;
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += a[i] * b[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < blockDim.x / 32) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) out[(int64_t)j * nb + c] = do_sqrt ? sqrt(v) : v;
    }
}

// Y[:, c] -= s[c] X[:, c]
__global__ void k_axpy_cols(int64_t n, int nb, const double *__restrict__ s, const double *__restrict__ X,
                            int64_t ldx, double *__restrict__ Y, int64_t ldy) {
    const int c = blockIdx.y;
    const double f = s[c];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        Y[i + c * ldy] -= f * X[i + c * ldx];
}

// X[:, c] *= f[c] (inverse = 0), or X[:, c] /= f[c] where f[c] > 1e-50 (inverse = 1)
__global__ void k_scal_cols(int64_t n, int nb, const double *__restrict__ f, int inverse, double *__restrict__ X,
                            int64_t ldx) {
    const int c = blockIdx.y;
    double g = f[c];
    if (inverse) {
        if (!(g > 1e-50)) return;
        g = 1.0 / g;
    }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        X[i + c * ldx] *= g;
}

// X[:, c] += sum_{j < m} W_j[:, c] y[j * nb + c], W_j = W + j * sW (ld n)
__global__ void k_gemv_cols(int64_t n, int nb, int m, const double *__restrict__ W, int64_t sW,
                            const double *__restrict__ y, double *__restrict__ X, int64_t ldx) {
    const int c = blockIdx.y;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < m; j++) acc += W[(int64_t)j * sW + (int64_t)c * n + i] * y[(int64_t)j * nb + c];
        X[i + c * ldx] += acc;
    }
}

// P[:, c] = Z[:, c] + beta[c] P[:, c]
__global__ void k_xpby_cols(int64_t n, int nb, const double *__restrict__ Z, const double *__restrict__ beta,
                            double *__restrict__ P) {
    const int c = blockIdx.y;
    const double b = beta[c];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        P[i + c * n] = Z[i + c * n] + b * P[i + c * n];
}

void launch_spmm(int n, int nb, const int *rowptr, const int *col, const double *val, double alpha, const double *X,
                 int64_t ldx, double beta, double *Y, int64_t ldy, cudaStream_t st) {
    if (n <= 0 || nb <= 0) return;
    const int G = 4;
    dim3 grid((unsigned)(((int64_t)n * G + 255) / 256), (unsigned)((nb + SPMM_CB - 1) / SPMM_CB));
    k_spmm<G><<<grid, 256, 0, st>>>(n, nb, rowptr, col, val, alpha, X, ldx, beta, Y, ldy);
}
void launch_dots_cols(int64_t n, int nb, int nblk, const double *A, int64_t sA, int64_t lda, const double *B,
                      int64_t ldb, int do_sqrt, double *out, cudaStream_t st) {
    if (nb <= 0 || nblk <= 0) return;
    k_dots_cols<<<dim3(nb, nblk), 1024, 0, st>>>(n, nb, A, sA, lda, B, ldb, do_sqrt, out);
}
static dim3 cols_grid(int64_t n, int nb) {
    const int64_t bx = std::min<int64_t>((n + 255) / 256, std::max<int64_t>(1, 148 * 8 / std::max(1, nb)));
    return dim3((unsigned)std::max<int64_t>(1, bx), (unsigned)nb);
}
void launch_axpy_cols(int64_t n, int nb, const double *s, const double *X, int64_t ldx, double *Y, int64_t ldy,
                      cudaStream_t st) {
    if (nb > 0) k_axpy_cols<<<cols_grid(n, nb), 256, 0, st>>>(n, nb, s, X, ldx, Y, ldy);
}
void launch_scal_cols(int64_t n, int nb, const double *f, int inverse, double *X, int64_t ldx, cudaStream_t st) {
    if (nb > 0) k_scal_cols<<<cols_grid(n, nb), 256, 0, st>>>(n, nb, f, inverse, X, ldx);
}
void launch_xpby_cols(int64_t n, int nb, const double *Z, const double *beta, double *P, cudaStream_t st) {
    if (nb > 0) k_xpby_cols<<<cols_grid(n, nb), 256, 0, st>>>(n, nb, Z, beta, P);
}
void launch_gemv_cols(int64_t n, int nb, int m, const double *W, int64_t sW, const double *y, double *X, int64_t ldx,
                      cudaStream_t st) {
    if (nb > 0 && m > 0) k_gemv_cols<<<cols_grid(n, nb), 256, 0, st>>>(n, nb, m, W, sW, y, X, ldx);
}

// Row blocks of k_spmv_stream: consecutive rows, at most SPMV_ROWS of them and
// SPMV_CAP entries, a longer row alone.  part[0] = 0, part[nblocks] = n.
void spmv_partition(int n, const int *rowptr, std::vector<int> &part) {
    part.assign(1, 0);
    int r = 0;
    while (r < n) {
        int e = r + 1;
        while (e < n && e - r < SPMV_ROWS && rowptr[e + 1] - rowptr[r] <= SPMV_CAP) e++;
        part.push_back(e);
        r = e;
    }
}
void launch_spmv_stream(int nblocks, const int *part, const int *rowptr, const int *col, const double *val,
                        double alpha, const double *x, double beta, double *y, cudaStream_t st) {
    if (nblocks > 0) k_spmv_stream<<<nblocks, 256, 0, st>>>(part, rowptr, col, val, alpha, x, beta, y);
}

void launch_spmv(int n, int64_t nnz, const int *rowptr, const int *col, const double *val, double alpha,
                 const double *x, double beta, double *y, cudaStream_t st) {
    if (n <= 0) return;
    double avg = n ? (double)nnz / n : 0;
    if (avg <= 12) {
        constexpr int G = 4;
        int64_t thr = (int64_t)n * G;
        k_spmv<G><<<(unsigned)((thr + 255) / 256), 256, 0, st>>>(n, rowptr, col, val, alpha, x, beta, y);
    } else {
        constexpr int G = 16;
        int64_t thr = (int64_t)n * G;
        k_spmv<G><<<(unsigned)((thr + 255) / 256), 256, 0, st>>>(n, rowptr, col, val, alpha, x, beta, y);
    }
}
int reduce_partials() { return RED_BLOCKS; }
void launch_dot(int64_t n, const double *a, const double *b, double *part, int do_sqrt, double *out,
                cudaStream_t st) {
    k_dot_part<<<RED_BLOCKS, RED_THREADS, 0, st>>>(n, a, b, part);
    k_dot_final<<<1, RED_THREADS, 0, st>>>(part, RED_BLOCKS, do_sqrt, out);
}
void launch_axpy(int64_t n, double alpha, const double *x, double *y, cudaStream_t st) {
    k_axpy<<<nblk(n), 256, 0, st>>>(n, alpha, x, y);
}
void launch_xpby(int64_t n, const double *x, double beta, double *y, cudaStream_t st) {
    k_xpby<<<nblk(n), 256, 0, st>>>(n, x, beta, y);
}
void launch_scal(int64_t n, double alpha, double *x, cudaStream_t st) { k_scal<<<nblk(n), 256, 0, st>>>(n, alpha, x); }
void launch_gemv(int64_t n, int m, const double *W, const double *yv, double *x, cudaStream_t st) {
    k_gemv<<<nblk(n), 256, 0, st>>>(n, m, W, yv, x);
}
template <typename TS, typename TD>
void launch_permute(int n, int nrhs, const int64_t *perm, int forward, const TS *src, int64_t lds, TD *dst,
                    int64_t ldd, cudaStream_t st) {
    k_permute<TS, TD><<<nblk((int64_t)n * nrhs), 256, 0, st>>>(n, nrhs, perm, forward, src, lds, dst, ldd);
}
template <typename TS, typename TD>
void launch_cast(int64_t n, const TS *src, TD *dst, cudaStream_t st) {
    k_cast<TS, TD><<<nblk(n), 256, 0, st>>>(n, src, dst);
}
void launch_sampled(int64_t nnz, const int *erow, const int *ecol, double alpha, const double *l, const double *x,
                    double *G, int sym, cudaStream_t st) {
    if (nnz <= 0) return;
    k_sampled<<<nblk(nnz), 256, 0, st>>>(nnz, erow, ecol, alpha, l, x, G, sym);
}

template void launch_permute<double, double>(int, int, const int64_t *, int, const double *, int64_t, double *,
                                             int64_t, cudaStream_t);
template void launch_permute<double, float>(int, int, const int64_t *, int, const double *, int64_t, float *, int64_t,
                                            cudaStream_t);
template void launch_permute<float, double>(int, int, const int64_t *, int, const float *, int64_t, double *, int64_t,
                                            cudaStream_t);
template void launch_cast<double, float>(int64_t, const double *, float *, cudaStream_t);
template void launch_cast<float, double>(int64_t, const float *, double *, cudaStream_t);

}  // namespace pgpu
