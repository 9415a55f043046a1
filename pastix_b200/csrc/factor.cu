// Factorization kernels of the B200 numerical phase (sm_100a).
//
// Per elimination level the host launches:
//   k_panel_small  one CTA per narrow cblk: the whole panel is factored in
//                  shared memory (diagonal factor + off-diagonal TRSM);
//   k_diag_large   one CTA per wide cblk: blocked diagonal factorization;
//   k_trsm         one CTA per row tile of a wide cblk's off-diagonal panel;
//   k_update       one CTA per output tile of the supernode-to-supernode
//                  updates, with the scatter-add into the facing cblk fused
//                  into the epilogue.
//
// Numerics follow the reference kernels:
//   POTRF  core_zpotf2sp / core_zpotrfsp   kernels/core_zpotrfsp.c:68-190
//   GETRF  core_zgetf2sp / core_zgetrfsp   kernels/core_zgetrfsp.c:65-200,
//          cpucblk_zgetrfsp1d_getrf :217-275 (geadd U^T into L, getmo back)
//   SYTRF  core_zsytf2sp / core_zsytrfsp   kernels/core_zsytrfsp.c:66-220
//   TRSM   cpucblk_ztrsmsp                 kernels/core_ztrsmsp.c:356
//   GEMM   core_zgemmsp_2d2d               kernels/core_zgemmsp.c:404-474
// including the static-pivot rule: a diagonal entry whose modulus is below
// the criterion is replaced by the criterion (POTRF) or by +/- criterion
// keeping its sign (GETRF, SYTRF), and counted.
#include "device.cuh"

#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include <algorithm>

namespace pgpu {

template <typename T> __device__ __forceinline__ T dev_abs(T x) { return x < T(0) ? -x : x; }
__device__ __forceinline__ double dev_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dev_sqrt(float x) { return sqrtf(x); }

// Static pivoting of one diagonal entry (reference :80-89 of each kernel).
template <typename T, int FACT>
__device__ __forceinline__ T static_pivot(T d, double crit, int &npiv) {
    if ((double)dev_abs(d) < crit) {
        if (FACT == FACT_POTRF) d = (T)crit;
        else d = (d < T(0)) ? (T)(-crit) : (T)crit;
        npiv++;
    }
    if (FACT == FACT_POTRF) d = dev_sqrt(d);
    return d;
}

// ---------------------------------------------------------------------------
// Coefficient initialisation: scatter the (permuted) matrix entries into the
// zeroed panels (cpucblk_zfillin_fr, kernels/cpucblk_zinit.c:395-487).  The maps
// are built once on the host from the matrix pattern.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_fill_coef(int64_t nnz, const double *__restrict__ vals, const int64_t *__restrict__ lmap,
                            const int64_t *__restrict__ umap, T *__restrict__ L, T *__restrict__ U) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) {
        double v = vals[e];
        int64_t p = lmap[e];
        if (p >= 0) L[p] = (T)v;
        if (umap) {
            int64_t q = umap[e];
            if (q >= 0) U[q] = (T)v;
        }
    }
}

// ---------------------------------------------------------------------------
// Narrow cblks: whole panel (and U^T panel for LU) in shared memory,
// right-looking column sweep over the width.  Column c: pivot, scale the
// column below the diagonal, rank-1 update of the remaining columns on all
// panel rows.  This is potf2/getf2/sytf2 on the diagonal block fused with the
// off-diagonal TRSM.
// ---------------------------------------------------------------------------
constexpr int PS_FB_CACHE = 512;  // facing bloks whose first rows k_panel_small keeps in shared memory
// Shared memory of k_panel_small: the panel (twice for GETRF) and its int tables.
__host__ __device__ inline long long panel_small_smem_bytes(long long panel_elems, int tsize, int maxst) {
    return panel_elems * tsize + 4LL * (2 * maxst + 2 * PS_FB_CACHE);
}

template <typename T, int FACT>
__global__ void __launch_bounds__(256) k_panel_small(DevStruct s, const int *__restrict__ list, T *L, T *U,
                                                      FactParams fp) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *P = reinterpret_cast<T *>(smem_raw);
    const int k = list[blockIdx.x];
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int tot = st * nc;
    const int tid = threadIdx.x, nt = blockDim.x;
    T *gL = L + s.cb_coef[k];
    T *gU = (FACT == FACT_GETRF) ? U + s.cb_coef[k] : nullptr;
    T *Q = P + tot;
    batched_copy<8, T>(tot, [&](int i) { return gL[i]; }, [&](int i, T v) { P[i] = v; });
    if (FACT == FACT_GETRF) batched_copy<8, T>(tot, [&](int i) { return gU[i]; }, [&](int i, T v) { Q[i] = v; });
    __shared__ int npiv;
    if (tid == 0) npiv = 0;
    __syncthreads();
    if (FACT == FACT_GETRF) {  // L_kk += (U^T)_kk^T : the full diagonal block
        for (int e = tid; e < nc * nc; e += nt) {
            int i = e % nc, j = e / nc;
            P[i + j * st] += Q[j + i * st];
        }
        __syncthreads();
    }
    for (int c = 0; c < nc; c++) {
        if (tid == 0) {
            int np = npiv;
            P[c + c * st] = static_pivot<T, FACT>(P[c + c * st], __ldg(fp.criterion), np);
            npiv = np;
        }
        __syncthreads();
        const T inv = T(1) / P[c + c * st];
        for (int i = c + 1 + tid; i < st; i += nt) {
            if (FACT == FACT_SYTRF && i < nc) P[c + i * st] = P[i + c * st];  // D*L^T into the upper part
            P[i + c * st] *= inv;
        }
        __syncthreads();
        const int w = nc - c - 1;
        if (w > 0) {
            const int h = st - c - 1;
            for (int e = tid; e < h * w; e += nt) {
                int i = c + 1 + e % h, j = c + 1 + e / h;
                if (FACT == FACT_POTRF) {
                    if (i >= j) P[i + j * st] -= P[i + c * st] * P[j + c * st];
                } else if (FACT == FACT_SYTRF) {
                    if (i >= j) P[i + j * st] -= P[i + c * st] * P[c + j * st];
                } else {
                    P[i + j * st] -= P[i + c * st] * P[c + j * st];
                }
            }
            if (FACT == FACT_GETRF) {  // U^T rows below the diagonal block: A[j, r] -= L[j,c] U[c,r]
                const int h2 = st - nc;
                for (int e = tid; e < h2 * w; e += nt) {
                    int r = nc + e % h2, j = c + 1 + e / h2;
                    Q[r + j * st] -= P[j + c * st] * Q[r + c * st];
                }
            }
        }
        __syncthreads();
    }
    if (FACT == FACT_GETRF) {  // (U^T)_kk = (L\U)_kk^T
        for (int e = tid; e < nc * nc; e += nt) {
            int i = e % nc, j = e / nc;
            Q[j + i * st] = P[i + j * st];
        }
        __syncthreads();
        for (int i = tid; i < tot; i += nt) gU[i] = Q[i];
    }
    for (int i = tid; i < tot; i += nt) gL[i] = P[i];
    if (tid == 0 && npiv) atomicAdd(fp.nbpivots, npiv);
    // the updates of every task of this cblk (core_zgemmsp_2d2d), from the
    // factored panel still in shared memory, scattered into the facing panels
    // with reductions; rtab / ctab: target rows and columns of one task
    __syncthreads();
    int *rtab = reinterpret_cast<int *>(P + (FACT == FACT_GETRF ? 2 : 1) * tot);
    int *ctab = rtab + st;
    int *fbr = ctab + st;           // first rows of the facing cblk's bloks (when they fit)
    int *fbo = fbr + PS_FB_CACHE;   // and their row offsets
    const int *ridx = s.rowidx + s.cb_rowidx[k];
    for (int b = s.cb_fblok[k] + 1; b < s.cb_fblok[k + 1]; b++) {
        const int f = s.bk_fcblk[b];
        const int row0 = s.bk_rowoff[b];
        const int n = s.bk_lrow[b] - s.bk_frow[b] + 1;
        const int M = st - row0;
        const int fb0 = s.cb_fblok[f], nbf = s.cb_fblok[f + 1] - fb0;
        const bool cached = nbf <= PS_FB_CACHE;
        if (cached)
            for (int e = tid; e < nbf; e += nt) {
                fbr[e] = s.bk_frow[fb0 + e];
                fbo[e] = s.bk_rowoff[fb0 + e];
            }
        __syncthreads();
        for (int i = tid; i < M; i += nt) {
            const int g = ridx[row0 + i];
            int lo = 0, hi = nbf - 1;
            while (lo < hi) {  // last blok of f whose first row is <= g
                const int mid = (lo + hi + 1) >> 1;
                if ((cached ? fbr[mid] : s.bk_frow[fb0 + mid]) <= g) lo = mid;
                else hi = mid - 1;
            }
            rtab[i] = (cached ? fbo[lo] : s.bk_rowoff[fb0 + lo]) + (g - (cached ? fbr[lo] : s.bk_frow[fb0 + lo]));
        }
        for (int j = tid; j < n; j += nt) ctab[j] = ridx[row0 + j] - s.cb_fcol[f];
        __syncthreads();
        T *Cl = L + s.cb_coef[f];
        const int stf = s.cb_stride[f];
        for (int e = tid; e < M * n; e += nt) {
            const int i = e % M, j = e / M;
            T v = T(0);
            for (int c = 0; c < nc; c++) {
                T bj = (FACT == FACT_GETRF) ? Q[(row0 + j) + c * st] : P[(row0 + j) + c * st];
                if (FACT == FACT_SYTRF) bj *= P[c + c * st];
                v += P[(row0 + i) + c * st] * bj;
            }
            atomicAdd(&Cl[rtab[i] + (size_t)ctab[j] * stf], -v);
        }
        if (FACT == FACT_GETRF) {  // U side: rows strictly below the blok, into the U panel of f
            T *Cu = U + s.cb_coef[f];
            const int M1 = M - n;
            for (int e = tid; e < M1 * n; e += nt) {
                const int i = n + e % M1, j = e / M1;
                T v = T(0);
                for (int c = 0; c < nc; c++) v += Q[(row0 + i) + c * st] * P[(row0 + j) + c * st];
                atomicAdd(&Cu[rtab[i] + (size_t)ctab[j] * stf], -v);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Wide cblks.  The diagonal block is factored by column panels of DNB = 32;
// for every 32 x 32 diagonal sub-block jj the inverse Z_jj of its upper
// triangular factor T_jj is formed and kept (device scratch `dinv`, one or two
// 32 x 32 blocks per sub-block), so that the off-diagonal TRSM X T = A becomes
// a blocked sequence of GEMMs: X_j = A_j Z_jj, A_{>j} -= X_j T_{j,>j} (the
// inverted-diagonal-block TRSM used by GPU BLAS libraries).  T per kind:
//   POTRF  T = L_kk^T           SYTRF  T = D_kk L_kk^T
//   GETRF  side 0: T = U_kk      side 1: T = L_kk^T (unit)
// ---------------------------------------------------------------------------
constexpr int DNB = 32;
constexpr int DLDW = DNB + 1;

// T_jj(i, k) of the 32 x 32 sub-block whose factored rows are in Wb (row major, ld DLDW)
template <typename T, int FACT>
__device__ __forceinline__ T tblk(const T *Wb, int i, int k, int side) {
    if (k < i) return T(0);
    if (FACT == FACT_POTRF) return Wb[k * DLDW + i];
    if (FACT == FACT_SYTRF) return (k == i) ? Wb[i * DLDW + i] : Wb[i * DLDW + i] * Wb[k * DLDW + i];
    if (side == 0) return Wb[i * DLDW + k];
    return (k == i) ? T(1) : Wb[k * DLDW + i];
}

// Warp: Z = T^{-1} (upper, 32 x 32), lane j forms column j by back substitution.
// rinv (smem, 32) receives 1 / T(i, i).  nb <= 32 valid rows/cols; the rest is identity.
template <typename T, int FACT>
__device__ __forceinline__ void warp_upper_inverse(const T *Wb, int nb, int side, T *rinv, T *Z, int ldz, T *gZ) {
    const int lane = threadIdx.x & 31;
    rinv[lane] = (lane < nb) ? T(1) / tblk<T, FACT>(Wb, lane, lane, side) : T(1);
    __syncwarp();
    T z[32];
#pragma unroll
    for (int i = 31; i >= 0; i--) {
        T acc = T(0);
#pragma unroll
        for (int k = i + 1; k < 32; k++)
            if (k < nb && i < nb) acc += tblk<T, FACT>(Wb, i, k, side) * z[k];
        z[i] = (i > lane) ? T(0) : ((i == lane) ? rinv[i] : -acc * rinv[i]);
    }
#pragma unroll
    for (int i = 0; i < 32; i++) {
        Z[i * ldz + lane] = z[i];
        if (gZ) gZ[i * 32 + lane] = z[i];
    }
}

template <typename T, int FACT>
__global__ void __launch_bounds__(256) k_diag_large(DevStruct s, const int *__restrict__ list, T *L, T *U, T *dinv,
                                                     FactParams fp) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int k = list[blockIdx.x];
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    T *W = reinterpret_cast<T *>(smem_raw);  // m x DNB panel, row major, ld DLDW
    T *R = W + (size_t)nc * DLDW;            // GETRF: DNB x t strip of U, row major, ld nc + 1
    const int ldr = nc + 1;
    __shared__ T Z0[DNB * DLDW], Z1[DNB * DLDW];
    __shared__ T rinv[DNB];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    T *A = L + s.cb_coef[k];
    T *gZ = dinv + s.cb_dinv[k];
    const int nzb = (nc + DNB - 1) / DNB;
    __shared__ int npiv;
    __shared__ T dsh[DNB];
    if (tid == 0) npiv = 0;
    if (FACT == FACT_GETRF) {  // L_kk += (U^T)_kk^T : the full diagonal block
        const T *Ut = U + s.cb_coef[k];
        batched_copy<8, T>(
            nc * nc, [&](int e) { int i = e % nc, j = e / nc; return A[i + (size_t)j * st] + Ut[j + (size_t)i * st]; },
            [&](int e, T v) { int i = e % nc, j = e / nc; A[i + (size_t)j * st] = v; });
    }
    __syncthreads();
    for (int jb = 0; jb < nc; jb += DNB) {
        const int nb = min(DNB, nc - jb);
        const int m = nc - jb;       // panel rows
        const int t = m - nb;        // trailing size
        batched_copy<8, T>(
            m * nb, [&](int e) { int i = e % m, c = e / m; return A[(jb + i) + (size_t)(jb + c) * st]; },
            [&](int e, T v) { int i = e % m, c = e / m; W[i * DLDW + c] = v; });
        if (FACT == FACT_GETRF)
            batched_copy<8, T>(
                nb * t, [&](int e) { int c = e % nb, q = e / nb; return A[(jb + c) + (size_t)(jb + nb + q) * st]; },
                [&](int e, T v) { int c = e % nb, q = e / nb; R[c * ldr + q] = v; });
        __syncthreads();
        if (warp == 0) {
            // 1. factor the nb x nb top block in registers, one row per lane
            T r[32];
#pragma unroll
            for (int j = 0; j < 32; j++)
                r[j] = (lane < nb && j < nb) ? W[lane * DLDW + j] : (lane == j ? T(1) : T(0));
            int np = 0;
#pragma unroll
            for (int c = 0; c < 32; c++) {
                if (c < nb) {
                    const T d = static_pivot<T, FACT>(__shfl_sync(0xffffffffu, r[c], c), __ldg(fp.criterion), np);
                    const T inv = T(1) / d;
                    const T u = r[c];
                    if (lane == c) r[c] = d;
                    else if (lane > c) r[c] *= inv;
#pragma unroll
                    for (int j = c + 1; j < 32; j++) {
                        if (j < nb) {
                            if (FACT == FACT_POTRF) {
                                const T ljc = __shfl_sync(0xffffffffu, r[c], j);
                                if (lane >= j) r[j] -= r[c] * ljc;
                            } else if (FACT == FACT_SYTRF) {
                                const T ujc = __shfl_sync(0xffffffffu, u, j);
                                if (lane >= j) r[j] -= r[c] * ujc;
                            } else {
                                const T ucj = __shfl_sync(0xffffffffu, r[j], c);
                                if (lane > c) r[j] -= r[c] * ucj;
                            }
                        }
                    }
                }
            }
            if (lane < nb)
#pragma unroll
                for (int j = 0; j < 32; j++)
                    if (j < nb) W[lane * DLDW + j] = r[j];
            if (lane == 0 && np) npiv += np;
            __syncwarp();
            // 2. inverse of the triangular factor of the block (and of L^T for GETRF's U side)
            warp_upper_inverse<T, FACT>(W, nb, 0, rinv, Z0, DLDW, gZ + (size_t)(jb / DNB) * 1024);
            if (FACT == FACT_GETRF) {
                __syncwarp();
                warp_upper_inverse<T, FACT>(W, nb, 1, rinv, Z1, DLDW, gZ + (size_t)(nzb + jb / DNB) * 1024);
            }
        }
        __syncthreads();
        if (FACT == FACT_SYTRF && tid < nb) dsh[tid] = W[tid * DLDW + tid];
        // 3. panel rows below the block, X T_jj = A by substitution: one row per
        //    thread held in registers, T_jj (staged in Z1 unless GETRF) and the
        //    reciprocals of its diagonal in shared memory
        if (FACT != FACT_GETRF) {
            for (int e = tid; e < 1024; e += nt) {
                int i = e >> 5, j = e & 31;
                Z1[i * DLDW + j] = (i < nb && j < nb) ? tblk<T, FACT>(W, i, j, 0) : T(0);
            }
        }
        if (tid < 32) rinv[tid] = (tid < nb) ? T(1) / tblk<T, FACT>(W, tid, tid, 0) : T(1);
        __syncthreads();
        for (int r = nb + tid; r < m; r += nt) {
            T x[32];
#pragma unroll
            for (int c = 0; c < 32; c++) x[c] = (c < nb) ? W[r * DLDW + c] : T(0);
#pragma unroll
            for (int c = 0; c < 32; c++) {
                x[c] *= rinv[c];
#pragma unroll
                for (int j = c + 1; j < 32; j++) {
                    T tcj;
                    if (FACT == FACT_GETRF) tcj = (c < nb && j < nb) ? W[c * DLDW + j] : T(0);
                    else tcj = Z1[c * DLDW + j];
                    x[j] -= x[c] * tcj;
                }
            }
#pragma unroll
            for (int c = 0; c < 32; c++)
                if (c < nb) W[r * DLDW + c] = x[c];
        }
        if (FACT == FACT_GETRF)  // U12 <- L11^{-1} U12 (unit lower), one column per thread
            for (int q = tid; q < t; q += nt) {
                T col[32];
#pragma unroll
                for (int i = 0; i < 32; i++) col[i] = (i < nb) ? R[i * ldr + q] : T(0);
#pragma unroll
                for (int c = 0; c < 32; c++)
#pragma unroll
                    for (int i = c + 1; i < 32; i++)
                        if (i < nb && c < nb) col[i] -= W[i * DLDW + c] * col[c];
#pragma unroll
                for (int i = 0; i < 32; i++)
                    if (i < nb) R[i * ldr + q] = col[i];
            }
        __syncthreads();
        for (int e = tid; e < m * nb; e += nt) {
            int i = e % m, c = e / m;
            A[(jb + i) + (size_t)(jb + c) * st] = W[i * DLDW + c];
        }
        if (FACT == FACT_GETRF)
            for (int e = tid; e < nb * t; e += nt) {
                int c = e % nb, q = e / nb;
                A[(jb + c) + (size_t)(jb + nb + q) * st] = R[c * ldr + q];
            }
        // 4. trailing update A22 -= L21 * B^T (4x4 blocks; lower triangle for the symmetric kinds)
        if (t > 0) {
            const int nbt = (t + 3) / 4;
            const int nblk = (FACT == FACT_GETRF) ? nbt * nbt : nbt * (nbt + 1) / 2;
            for (int id = tid; id < nblk; id += nt) {
                int bi, bj;
                if (FACT == FACT_GETRF) {
                    bi = id % nbt;
                    bj = id / nbt;
                } else {
                    bi = (int)((sqrt(8.0 * id + 1.0) - 1.0) * 0.5);
                    while (bi * (bi + 1) / 2 > id) bi--;
                    while ((bi + 1) * (bi + 2) / 2 <= id) bi++;
                    bj = id - bi * (bi + 1) / 2;
                }
                T acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) acc[i][j] = T(0);
                for (int c = 0; c < nb; c++) {
                    T a[4], b[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        int r = bi * 4 + i;
                        a[i] = (r < t) ? W[(nb + r) * DLDW + c] : T(0);
                    }
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        int q = bj * 4 + j;
                        if (FACT == FACT_GETRF) b[j] = (q < t) ? R[c * ldr + q] : T(0);
                        else if (FACT == FACT_SYTRF) b[j] = (q < t) ? dsh[c] * W[(nb + q) * DLDW + c] : T(0);
                        else b[j] = (q < t) ? W[(nb + q) * DLDW + c] : T(0);
                    }
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int j = 0; j < 4; j++) acc[i][j] += a[i] * b[j];
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    int q = bj * 4 + j;
                    if (q >= t) continue;
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        int r = bi * 4 + i;
                        if (r >= t || (FACT != FACT_GETRF && r < q)) continue;
                        A[(jb + nb + r) + (size_t)(jb + nb + q) * st] -= acc[i][j];
                    }
                }
            }
        }
        __syncthreads();
    }
    if (FACT == FACT_SYTRF) {  // upper part of the diagonal block holds D L^T
        batched_copy<8, T>(
            nc * nc,
            [&](int e) {
                int i = e % nc, j = e / nc;
                return (i < j) ? A[i + (size_t)i * st] * A[j + (size_t)i * st] : T(0);
            },
            [&](int e, T v) { int i = e % nc, j = e / nc; if (i < j) A[i + (size_t)j * st] = v; });
    }
    if (FACT == FACT_GETRF) {  // (U^T)_kk = (L\U)_kk^T
        __syncthreads();
        T *Ut = U + s.cb_coef[k];
        batched_copy<8, T>(
            nc * nc, [&](int e) { int i = e % nc, j = e / nc; return A[i + (size_t)j * st]; },
            [&](int e, T v) { int i = e % nc, j = e / nc; Ut[j + (size_t)i * st] = v; });
    }
    if (tid == 0 && npiv) atomicAdd(fp.nbpivots, npiv);
}

// Off-diagonal TRSM of a wide cblk on a tile of TRSM_ROWS panel rows held
// row-major in shared memory, blocked by 32 columns with the inverted
// diagonal sub-blocks from k_diag_large.  blockIdx.y = GETRF side.
constexpr int TRSM_ROWS = 32;
constexpr int TRSM_MAXT = 10;  // column chunks of 32 per GEMM pass

template <typename T, int FACT>
__global__ void __launch_bounds__(256) k_trsm(DevStruct s, const RowTile *__restrict__ tiles, T *L, T *U,
                                               const T *__restrict__ dinv) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const RowTile tl = tiles[blockIdx.x];
    const int side = blockIdx.y;
    const int k = tl.cblk;
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int rows = min(TRSM_ROWS, st - tl.r0);
    const int ld = nc + 1;
    T *X = reinterpret_cast<T *>(smem_raw);  // TRSM_ROWS x nc, row major, ld
    T *Ts = X + TRSM_ROWS * ld;              // 32 x (nc - jb) strip of T from column jb, row major, ld
    __shared__ T Zs[DNB * DLDW], Rs[TRSM_ROWS * DLDW];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const T *D = L + s.cb_coef[k];  // diagonal block (ld = st) of the L panel
    T *A = ((FACT == FACT_GETRF && side == 1) ? U : L) + s.cb_coef[k] + tl.r0;
    const bool unit = (FACT == FACT_GETRF && side == 1);
    const int nzb = (nc + DNB - 1) / DNB;
    const T *gZ = dinv + s.cb_dinv[k] + (size_t)(side ? nzb : 0) * 1024;
    batched_copy<8, T>(
        TRSM_ROWS * nc,
        [&](int e) { int i = e % TRSM_ROWS, j = e / TRSM_ROWS; return (i < rows) ? A[i + (size_t)j * st] : T(0); },
        [&](int e, T v) { int i = e % TRSM_ROWS, j = e / TRSM_ROWS; X[i * ld + j] = v; });
    for (int jb = 0; jb < nc; jb += 32) {
        const int nb = min(32, nc - jb);
        const int wdt = nc - jb;
        __syncthreads();
        batched_copy<8, T>(
            nb * wdt,
            [&](int e) {  // T(jb + a, jb + q)
                int q = e % wdt, a = e / wdt;
                int ga = jb + a, gb = jb + q;
                T t;
                if (gb < ga) t = T(0);
                else if (FACT == FACT_POTRF) t = D[gb + (size_t)ga * st];
                else if (FACT == FACT_SYTRF) t = (gb == ga) ? D[ga + (size_t)ga * st]
                                                              : D[ga + (size_t)ga * st] * D[gb + (size_t)ga * st];
                else if (side == 0) t = D[ga + (size_t)gb * st];
                else t = D[gb + (size_t)ga * st];
                return t;
            },
            [&](int e, T v) { int q = e % wdt, a = e / wdt; Ts[a * ld + q] = v; });
        batched_copy<4, T>(
            1024, [&](int e) { return gZ[(size_t)(jb / DNB) * 1024 + e]; },
            [&](int e, T v) { Zs[(e >> 5) * DLDW + (e & 31)] = v; });
        __syncthreads();
        // X_j <- A_j T_jj^{-1}: product with the inverted block Z, then one residual
        // correction X_j += (A_j - X_j T_jj) Z; warp w owns rows 4w..4w+3, lane = column
        {
            const int r0 = warp * 4;
            T a[4], x0[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                a[i] = (lane < nb) ? X[(r0 + i) * ld + jb + lane] : T(0);
                x0[i] = T(0);
            }
            for (int c = 0; c < nb; c++) {
                const T z = Zs[c * DLDW + lane];
#pragma unroll
                for (int i = 0; i < 4; i++) x0[i] += X[(r0 + i) * ld + jb + c] * z;
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (lane < nb) X[(r0 + i) * ld + jb + lane] = x0[i];
            __syncwarp();
            T rr[4];
#pragma unroll
            for (int i = 0; i < 4; i++) rr[i] = a[i];
            for (int c = 0; c < nb; c++) {
                const T t = (c <= lane && lane < nb) ? ((c == lane && unit) ? T(1) : Ts[c * ld + lane]) : T(0);
#pragma unroll
                for (int i = 0; i < 4; i++) rr[i] -= X[(r0 + i) * ld + jb + c] * t;
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 4; i++) Rs[(r0 + i) * DLDW + lane] = (lane < nb) ? rr[i] : T(0);
            __syncwarp();
            for (int c = 0; c < nb; c++) {
                const T z = Zs[c * DLDW + lane];
#pragma unroll
                for (int i = 0; i < 4; i++) x0[i] += Rs[(r0 + i) * DLDW + c] * z;
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (lane < nb) X[(r0 + i) * ld + jb + lane] = x0[i];
        }
        __syncthreads();
        // X[:, jb+nb:] -= X[:, jb:jb+nb] * Ts[:, nb:]
        const int rest = wdt - nb;
        for (int cb = 0; cb < rest; cb += 32 * TRSM_MAXT) {
            T acc[4][TRSM_MAXT];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int t = 0; t < TRSM_MAXT; t++) acc[i][t] = T(0);
            const int r0 = warp * 4;
            for (int kk = 0; kk < nb; kk++) {
                T a[4];
#pragma unroll
                for (int i = 0; i < 4; i++) a[i] = X[(r0 + i) * ld + jb + kk];
#pragma unroll
                for (int t = 0; t < TRSM_MAXT; t++) {
                    const int q = cb + lane + 32 * t;
                    if (q < rest) {
                        const T bq = Ts[kk * ld + nb + q];
#pragma unroll
                        for (int i = 0; i < 4; i++) acc[i][t] += a[i] * bq;
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < TRSM_MAXT; t++) {
                const int q = cb + lane + 32 * t;
                if (q < rest) {
#pragma unroll
                    for (int i = 0; i < 4; i++) X[(r0 + i) * ld + jb + nb + q] -= acc[i][t];
                }
            }
        }
    }
    __syncthreads();
    for (int e = tid; e < rows * nc; e += blockDim.x) {
        int i = e % rows, j = e / rows;
        A[i + (size_t)j * st] = X[i * ld + j];
    }
}

// ---------------------------------------------------------------------------
// Update GEMM with fused scatter-add (core_zgemmsp_2d2d semantics).  For task
// (src k, blok b facing f): C_f[rows(i) -> f, cols(b) -> f] -= A_i * B_b^T for
// every blok i >= b of k (i > b on the U side of LU).  The M rows of the task
// are contiguous in the src panel, so one tile covers consecutive panel rows;
// each row's place in f is found by binary search over f's bloks.
// SIMT FP64/FP32 register-tiled GEMM: BM x BN tile, BK deep, TM x TN per thread.
// ---------------------------------------------------------------------------
template <int BM, int BN, int BK, int TM, int TN>
struct UpdCfg {
    static constexpr int THREADS = (BM / TM) * (BN / TN);
};

template <typename T, int FACT, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    k_update(DevStruct s, const UpdTile *__restrict__ tiles, T *L, T *U) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int TX = BM / TM;  // threads along rows
    __shared__ T As[BK][BM + 1];
    __shared__ T Bs[BK][BN + 1];
    __shared__ int rt[BM];
    __shared__ int ct[BN];
    __shared__ T dsc[BK];

    const UpdTile tl = tiles[blockIdx.x];
    const TaskDev tk = s.tasks[tl.task];
    const int k = tk.src, f = tk.dst;
    const int K = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int shift = tl.side ? tk.n : 0;
    const int M = tk.m - shift;
    const int arow = tk.row0 + shift + tl.mt * BM;  // first src panel row of the A tile
    const int brow = tk.row0 + tl.nt * BN;          // first src panel row of the B tile
    const int mrows = min(BM, M - tl.mt * BM);
    const int ncols = min(BN, tk.n - tl.nt * BN);
    const int tid = threadIdx.x;
    const T *Ap = ((FACT == FACT_GETRF && tl.side == 1) ? U : L) + s.cb_coef[k];
    const T *Bp = ((FACT == FACT_GETRF && tl.side == 0) ? U : L) + s.cb_coef[k];
    const T *Dk = L + s.cb_coef[k];
    T *Cp = ((FACT == FACT_GETRF && tl.side == 1) ? U : L) + s.cb_coef[f];
    const int stf = s.cb_stride[f];

    // target rows / columns in the facing panel
    const int *ridx = s.rowidx + s.cb_rowidx[k];
    if (tid < BM) {
        int r = -1;
        if (tid < mrows) {
            int g = ridx[arow + tid];
            int lo = s.cb_fblok[f], hi = s.cb_fblok[f + 1] - 1;
            while (lo < hi) {  // last blok of f with frow <= g
                int mid = (lo + hi + 1) >> 1;
                if (s.bk_frow[mid] <= g) lo = mid; else hi = mid - 1;
            }
            r = s.bk_rowoff[lo] + (g - s.bk_frow[lo]);
        }
        rt[tid] = r;
    }
    if (tid < BN) ct[tid] = (tid < ncols) ? (ridx[brow + tid] - s.cb_fcol[f]) : -1;

    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] = T(0);

    const int tx = tid % TX, ty = tid / TX;
    for (int k0 = 0; k0 < K; k0 += BK) {
        batched_copy<(BK * BM + NT - 1) / NT, T>(
            BK * BM,
            [&](int e) {
                int kk = e / BM, r = e % BM;
                return (r < mrows && k0 + kk < K) ? Ap[(arow + r) + (size_t)(k0 + kk) * st] : T(0);
            },
            [&](int e, T v) { As[e / BM][e % BM] = v; });
        batched_copy<(BK * BN + NT - 1) / NT, T>(
            BK * BN,
            [&](int e) {
                int kk = e / BN, c = e % BN;
                return (c < ncols && k0 + kk < K) ? Bp[(brow + c) + (size_t)(k0 + kk) * st] : T(0);
            },
            [&](int e, T v) { Bs[e / BN][e % BN] = v; });
        if (FACT == FACT_SYTRF && tid < BK)
            dsc[tid] = (k0 + tid < K) ? Dk[(k0 + tid) + (size_t)(k0 + tid) * st] : T(0);
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            T a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; i++) a[i] = As[kk][tx + i * TX];
#pragma unroll
            for (int j = 0; j < TN; j++) b[j] = Bs[kk][ty + j * (BN / TN)];
            if (FACT == FACT_SYTRF) {
#pragma unroll
                for (int j = 0; j < TN; j++) b[j] *= dsc[kk];
            }
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[i][j] += a[i] * b[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < TN; j++) {
        int c = ty + j * (BN / TN);
        int cc = ct[c];
        if (cc < 0) continue;
        T *dst[TM];
#pragma unroll
        for (int i = 0; i < TM; i++) {
            int rr = rt[tx + i * TX];
            dst[i] = (rr < 0) ? nullptr : Cp + rr + (size_t)cc * stf;
        }
        if (tk.excl && sizeof(T) == 8) {  // FP32 updates of different levels may overlap: reductions only
            T old[TM];
#pragma unroll
            for (int i = 0; i < TM; i++) old[i] = dst[i] ? *dst[i] : T(0);
#pragma unroll
            for (int i = 0; i < TM; i++)
                if (dst[i]) *dst[i] = old[i] - acc[i][j];
        } else {
#pragma unroll
            for (int i = 0; i < TM; i++)
                if (dst[i]) atomicAdd(dst[i], -acc[i][j]);
        }
    }
}

// ---------------------------------------------------------------------------
// FP64 update on the tensor cores: the same task/tile semantics as k_update
// with a 128 x 64 output tile, 16-deep k steps double-buffered in shared
// memory by cp.async, and DMMA (mma.sync m8n8k4 f64) on 8 warps arranged
// 4 x 2, each warp owning a 32 x 32 block of 4 x 4 DMMA tiles.  The scatter
// into the facing panel is the epilogue, as in k_update.
// ---------------------------------------------------------------------------
constexpr int DM_BM = 128, DM_BN = 64, DM_BK = 16;
constexpr int DM_LDA = DM_BM + 8, DM_LDB = DM_BN + 8;  // row strides = 8 mod 16 doubles: 2 wavefronts per fragment load
constexpr size_t DM_SMEM = sizeof(double) * 2 * DM_BK * (DM_LDA + DM_LDB);

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    int sz = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <int FACT>
__global__ void __launch_bounds__(256) k_update_dmma(DevStruct s, const UpdTile *__restrict__ tiles, double *L,
                                                      double *U) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *As = reinterpret_cast<double *>(smem_raw);  // [2][DM_BK][DM_LDA]
    double *Bs = As + 2 * DM_BK * DM_LDA;               // [2][DM_BK][DM_LDB]
    __shared__ int rt[DM_BM];
    __shared__ int ct[DM_BN];
    __shared__ double dsc[2][DM_BK];

    const UpdTile tl = tiles[blockIdx.x];
    const TaskDev tk = s.tasks[tl.task];
    const int k = tk.src, f = tk.dst;
    const int K = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int shift = tl.side ? tk.n : 0;
    const int M = tk.m - shift;
    const int arow = tk.row0 + shift + tl.mt * DM_BM;
    const int brow = tk.row0 + tl.nt * DM_BN;
    const int mrows = min(DM_BM, M - tl.mt * DM_BM);
    const int ncols = min(DM_BN, tk.n - tl.nt * DM_BN);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double *Ap = ((FACT == FACT_GETRF && tl.side == 1) ? U : L) + s.cb_coef[k];
    const double *Bp = ((FACT == FACT_GETRF && tl.side == 0) ? U : L) + s.cb_coef[k];
    const double *Dk = L + s.cb_coef[k];
    double *Cp = ((FACT == FACT_GETRF && tl.side == 1) ? U : L) + s.cb_coef[f];
    const int stf = s.cb_stride[f];

    const int *ridx = s.rowidx + s.cb_rowidx[k];
    if (tid < DM_BM) {
        int r = -1;
        if (tid < mrows) {
            int g = ridx[arow + tid];
            int lo = s.cb_fblok[f], hi = s.cb_fblok[f + 1] - 1;
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if (s.bk_frow[mid] <= g) lo = mid; else hi = mid - 1;
            }
            r = s.bk_rowoff[lo] + (g - s.bk_frow[lo]);
        }
        rt[tid] = r;
    }
    if (tid < DM_BN) ct[tid] = (tid < ncols) ? (ridx[brow + tid] - s.cb_fcol[f]) : -1;

    auto load_stage = [&](int buf, int k0) {
        double *as = As + buf * DM_BK * DM_LDA;
        double *bs = Bs + buf * DM_BK * DM_LDB;
#pragma unroll
        for (int q = 0; q < (DM_BK * DM_BM) / 256; q++) {
            int e = tid + q * 256;
            int kk = e / DM_BM, r = e % DM_BM;
            bool v = (r < mrows) && (k0 + kk < K);
            const double *src = v ? Ap + (arow + r) + (size_t)(k0 + kk) * st : Ap;
            cp_async8(as + kk * DM_LDA + r, src, v);
        }
#pragma unroll
        for (int q = 0; q < (DM_BK * DM_BN) / 256; q++) {
            int e = tid + q * 256;
            int kk = e / DM_BN, c = e % DM_BN;
            bool v = (c < ncols) && (k0 + kk < K);
            const double *src = v ? Bp + (brow + c) + (size_t)(k0 + kk) * st : Bp;
            cp_async8(bs + kk * DM_LDB + c, src, v);
        }
        if (FACT == FACT_SYTRF && tid < DM_BK)
            dsc[buf][tid] = (k0 + tid < K) ? Dk[(k0 + tid) + (size_t)(k0 + tid) * st] : 0.0;
        cp_async_commit();
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
    const int g = lane >> 2, q4 = lane & 3;
    const int nk = (K + DM_BK - 1) / DM_BK;
    load_stage(0, 0);
    for (int kt = 0; kt < nk; kt++) {
        if (kt + 1 < nk) {
            load_stage((kt + 1) & 1, (kt + 1) * DM_BK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double *as = As + (kt & 1) * DM_BK * DM_LDA;
        const double *bs = Bs + (kt & 1) * DM_BK * DM_LDB;
#pragma unroll
        for (int kk = 0; kk < DM_BK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = as[(kk + q4) * DM_LDA + wm + i * 8 + g];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                b[j] = bs[(kk + q4) * DM_LDB + wn + j * 8 + g];
                if (FACT == FACT_SYTRF) b[j] *= dsc[kt & 1][kk + q4];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        __syncthreads();
    }
    // epilogue: scatter into the facing panel; exclusive targets are updated by
    // plain read-modify-write with the 8 reads of a row issued together
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = wm + i * 8 + g;
        const int rr = rt[r];
        if (rr < 0) continue;
        double *dst[8];
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int cc = ct[wn + j * 8 + q4 * 2 + h];
                dst[j * 2 + h] = (cc < 0) ? nullptr : Cp + rr + (size_t)cc * stf;
            }
        if (tk.excl) {
            double old[8];
#pragma unroll
            for (int q = 0; q < 8; q++) old[q] = dst[q] ? *dst[q] : 0.0;
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (dst[q]) *dst[q] = old[q] - acc[i][q >> 1][q & 1];
        } else {
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (dst[q]) atomicAdd(dst[q], -acc[i][q >> 1][q & 1]);
        }
    }
}

// ---------------------------------------------------------------------------
// Off-diagonal TRSM on FP64 tensor cores (DMMA m8n8k4), X T = A for a tile of
// 32 panel rows of a wide cblk, T the upper triangular factor of the diagonal
// block (L^T for POTRF, D L^T for SYTRF, U and L^T for the two GETRF sides),
// as cpucblk_ztrsmsp (kernels/core_ztrsmsp.c:356).  The whole 32 x nc tile
// stays in registers as 8 x 8 accumulator fragments: warp w owns the column
// fragments w, w + 8, w + 16, ... (nc <= TD_MAXNC).  Column block j (32
// columns) is solved with the inverted diagonal sub-block Z = T_jj^{-1} from
// k_diag_large plus one residual correction, X_j = X0 + (A_j - X0 T_jj) Z
// with X0 = A_j Z, then subtracted from the fragments to its right with T's
// rows of block j read straight from the (L2-resident) diagonal block.
// Storage may be FP32 (mixed precision); the arithmetic is FP64 throughout.
// ---------------------------------------------------------------------------
constexpr int TD_Q = 6;                 // column fragments per warp
constexpr int TD_MAXNC = 8 * TD_Q * 8;  // 384 columns
constexpr int TD_LDS = 36;              // shared row stride (doubles): 2 wavefronts per fragment load

// T(a, b) of the upper triangular factor, a <= b < nc (callers guarantee it).
template <typename T, int FACT>
__device__ __forceinline__ double trsm_tval(const T *D, int st, int a, int b, int side) {
    if (FACT == FACT_POTRF) return (double)D[b + (size_t)a * st];
    if (FACT == FACT_SYTRF) {
        const double da = (double)D[a + (size_t)a * st];
        return (a == b) ? da : da * (double)D[b + (size_t)a * st];
    }
    if (side == 0) return (double)D[a + (size_t)b * st];
    return (a == b) ? 1.0 : (double)D[b + (size_t)a * st];
}

template <typename T, int FACT>
__global__ void __launch_bounds__(256, 2) k_trsm_dmma(DevStruct s, const RowTile *__restrict__ tiles, T *L, T *U,
                                                       const T *__restrict__ dinv) {
    __shared__ double As[32 * TD_LDS], Xs[32 * TD_LDS], Rs[32 * TD_LDS];
    const RowTile tl = tiles[blockIdx.x];
    const int side = blockIdx.y;
    const int k = tl.cblk;
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int rows = min(32, st - tl.r0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const T *D = L + s.cb_coef[k];
    T *A = ((FACT == FACT_GETRF && side == 1) ? U : L) + s.cb_coef[k] + tl.r0;
    const int nzb = (nc + 31) / 32;
    const int ncf = (nc + 7) / 8;
    const T *gZ = dinv + s.cb_dinv[k] + (size_t)(side ? nzb : 0) * 1024;

    double acc[4][TD_Q][2];
#pragma unroll
    for (int q = 0; q < TD_Q; q++) {
        const int c0 = 8 * (warp + 8 * q) + 2 * t4;
#pragma unroll
        for (int rf = 0; rf < 4; rf++) {
            const int r = 8 * rf + g;
#pragma unroll
            for (int e = 0; e < 2; e++)
                acc[rf][q][e] = (r < rows && c0 + e < nc) ? (double)A[r + (size_t)(c0 + e) * st] : 0.0;
        }
    }
    const int orf = warp >> 1, ocf = 2 * (warp & 1);  // this warp's fragments of the 32 x 32 block solve
    for (int j = 0; j < nzb; j++) {
        const int jb = 32 * j;
        // i. the owners of block j hand their fragments over to shared memory
#pragma unroll
        for (int q = 0; q < TD_Q; q++) {
            const int cf = warp + 8 * q;
            if ((cf >> 2) == j) {
                const int cc = 8 * (cf & 3) + 2 * t4;
#pragma unroll
                for (int rf = 0; rf < 4; rf++) {
                    As[(8 * rf + g) * TD_LDS + cc] = acc[rf][q][0];
                    As[(8 * rf + g) * TD_LDS + cc + 1] = acc[rf][q][1];
                }
            }
        }
        __syncthreads();
        const T *Zj = gZ + (size_t)j * 1024;
        double x0[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        // ii-a. X0 = A_j Z
#pragma unroll
        for (int ks = 0; ks < 8; ks++) {
            const double a = As[(8 * orf + g) * TD_LDS + 4 * ks + t4];
#pragma unroll
            for (int c = 0; c < 2; c++)
                dmma884(x0[c][0], x0[c][1], a, (double)Zj[(4 * ks + t4) * 32 + 8 * (ocf + c) + g]);
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
            Xs[(8 * orf + g) * TD_LDS + 8 * (ocf + c) + 2 * t4] = x0[c][0];
            Xs[(8 * orf + g) * TD_LDS + 8 * (ocf + c) + 2 * t4 + 1] = x0[c][1];
        }
        __syncthreads();
        // ii-b. R = A_j - X0 T_jj
        double rr[2][2];
#pragma unroll
        for (int c = 0; c < 2; c++) {
            rr[c][0] = As[(8 * orf + g) * TD_LDS + 8 * (ocf + c) + 2 * t4];
            rr[c][1] = As[(8 * orf + g) * TD_LDS + 8 * (ocf + c) + 2 * t4 + 1];
        }
#pragma unroll
        for (int ks = 0; ks < 8; ks++) {
            const double a = -Xs[(8 * orf + g) * TD_LDS + 4 * ks + t4];
            const int ta = jb + 4 * ks + t4;
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const int tb = jb + 8 * (ocf + c) + g;
                const double b = (ta <= tb && tb < nc) ? trsm_tval<T, FACT>(D, st, ta, tb, side) : 0.0;
                dmma884(rr[c][0], rr[c][1], a, b);
            }
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
            Rs[(8 * orf + g) * TD_LDS + 8 * (ocf + c) + 2 * t4] = rr[c][0];
            Rs[(8 * orf + g) * TD_LDS + 8 * (ocf + c) + 2 * t4 + 1] = rr[c][1];
        }
        __syncthreads();
        // ii-c. X_j = X0 + R Z, to shared memory and to the panel
#pragma unroll
        for (int ks = 0; ks < 8; ks++) {
            const double a = Rs[(8 * orf + g) * TD_LDS + 4 * ks + t4];
#pragma unroll
            for (int c = 0; c < 2; c++)
                dmma884(x0[c][0], x0[c][1], a, (double)Zj[(4 * ks + t4) * 32 + 8 * (ocf + c) + g]);
        }
        {
            const int r = 8 * orf + g;
#pragma unroll
            for (int c = 0; c < 2; c++) {
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int cc = 8 * (ocf + c) + 2 * t4 + e;
                    Xs[r * TD_LDS + cc] = x0[c][e];
                    if (r < rows && jb + cc < nc) A[r + (size_t)(jb + cc) * st] = (T)x0[c][e];
                }
            }
        }
        __syncthreads();
        // iii. fragments right of block j: acc -= X_j T(block j rows, their columns)
        if (4 * j + 4 < ncf) {
#pragma unroll 2
            for (int ks = 0; ks < 8; ks++) {
                const int ta = jb + 4 * ks + t4;
                double a[4];
#pragma unroll
                for (int rf = 0; rf < 4; rf++) a[rf] = -Xs[(8 * rf + g) * TD_LDS + 4 * ks + t4];
                double b[TD_Q];
#pragma unroll
                for (int q = 0; q < TD_Q; q++) {
                    const int cf = warp + 8 * q;
                    const int tb = 8 * cf + g;
                    b[q] = (cf >= 4 * j + 4 && ta < nc && tb < nc) ? trsm_tval<T, FACT>(D, st, ta, tb, side) : 0.0;
                }
#pragma unroll
                for (int q = 0; q < TD_Q; q++) {
                    const int cf = warp + 8 * q;
                    if (cf >= 4 * j + 4 && cf < ncf) {
#pragma unroll
                        for (int rf = 0; rf < 4; rf++) dmma884(acc[rf][q][0], acc[rf][q][1], a[rf], b[q]);
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Diagonal block of a wide cblk on FP64 tensor cores (nc <= DG_MAXNC).  Right
// looking by 32-column panels, as core_zpotrfsp / core_zgetrfsp /
// core_zsytrfsp block their diagonal factorization:
//   1. the (nc - jb) x 32 panel is staged in shared memory (FP64, row major);
//   2. one warp factors its 32 x 32 top block in registers with static
//      pivoting; one or two warps invert the triangular factor(s) (kept in
//      `dinv` for the TRSM and the solve);
//   3. the rows below (and GETRF's U strip) are solved 8 rows per warp with
//      X = X0 + (A - X0 T) Z, X0 = A Z, on DMMA m8n8k4;
//   4. the trailing block is updated from global memory in 16 x 16 blocks, the
//      lower triangle for the symmetric kinds.
// Storage may be FP32 (mixed precision); the arithmetic is FP64.
// ---------------------------------------------------------------------------
constexpr int DG_LD = 36;      // shared row stride (doubles): 2 wavefronts per fragment access
constexpr int DG_MAXNC = 384;
constexpr int DG_NBLK = 2;     // trailing-update blocks in flight per warp

__host__ __device__ inline long long diag_dmma_smem_bytes(int nc) { return (long long)nc * DG_LD * 8; }

// T_jj(a, b), a <= b, of the factored top block W (row major, ld DG_LD).
template <int FACT>
__device__ __forceinline__ double dg_t(const double *W, int a, int b, int side) {
    if (FACT == FACT_POTRF) return W[b * DG_LD + a];
    if (FACT == FACT_SYTRF) return (a == b) ? W[a * DG_LD + a] : W[a * DG_LD + a] * W[b * DG_LD + a];
    if (side == 0) return W[a * DG_LD + b];
    return (a == b) ? 1.0 : W[b * DG_LD + a];
}

// Pivot of a factorization step: the (warp-uniform) diagonal value a after
// static pivoting, and the reciprocal that scales its column.  POTRF takes one
// reciprocal square root: d = a rsqrt(a), 1 / d = rsqrt(a).
template <int FACT>
__device__ __forceinline__ void dg_pivot(double a, double crit, int &np, double &d, double &inv) {
    const bool rep = fabs(a) < crit;  // selects rather than a branch: this sits on the step's critical path
    np += rep ? 1 : 0;
    a = rep ? ((FACT == FACT_POTRF || a >= 0.0) ? crit : -crit) : a;
    if (FACT == FACT_POTRF) {
        const double rs = rsqrt(a);
        d = a * rs;
        inv = rs;
    } else {
        d = a;
        inv = 1.0 / a;
    }
}

constexpr int DG_BLD = 34;        // row stride (doubles) of the published factor steps
constexpr int DG_SPIN = 1 << 22;  // bound on a warp's wait for the factorization's progress
constexpr int PGPU_STATUS_TIMEOUT = 3;

// One warp: factor the nb x nb top block held row major in W (ld DG_LD) in
// place, one row per lane in registers, with static pivoting; returns the
// number of replaced pivots.  POTRF leaves L (lower), SYTRF L (unit, strictly
// lower) and D on the diagonal, GETRF L (unit, strictly lower) and U.
//
// Step c publishes, in row c of Pub (ld DG_BLD, 16-byte aligned), what the
// other lanes need for their update and what the inverse warps need, then
// bumps *prog to c + 1:
//   POTRF  Pub[c][i] = L(i, c)           (i > c), d_c at i = c;
//   SYTRF  Pub[c][i] = D(c) L(i, c)      (i > c), d_c at i = c;
//   GETRF  Pub[c][j] = row c of L \ U    (L(c, j) for j < c, d_c, U(c, j) for j > c);
// and Pub[c][32] = 1 / d_c.  The row is read back as 16-byte pairs; each step
// updates and pivots the next column before the rest of the row, so the
// reciprocal (square root) of the next pivot overlaps the remaining updates.
template <int FACT, bool FULL>
__device__ __forceinline__ int dg_factor32_impl(double *W, int nbr, double crit, double *Pub, volatile int *prog) {
    const int nb = FULL ? 32 : nbr;  // a full block compiles without any bound test
    const int lane = threadIdx.x & 31;
    double r[32];
#pragma unroll
    for (int j = 0; j < 32; j++) r[j] = (lane < nb && j < nb) ? W[lane * DG_LD + j] : (lane == j ? 1.0 : 0.0);
    int np = 0;
    double d, inv;
    dg_pivot<FACT>(__shfl_sync(0xffffffffu, r[0], 0), crit, np, d, inv);
#pragma unroll
    for (int c = 0; c < 32; c++) {
        if (c < nb) {
            double *Pc = Pub + c * DG_BLD;
            const double u = r[c];
            if (lane == c) r[c] = d;
            else if (lane > c) r[c] *= inv;
            if (FACT == FACT_GETRF) {
                if (lane == c) {
#pragma unroll
                    for (int j = 0; j < 32; j += 2) *reinterpret_cast<double2 *>(Pc + j) = make_double2(r[j], r[j + 1]);
                    Pc[32] = inv;
                }
            } else {
                Pc[lane] = (FACT == FACT_SYTRF && lane != c) ? u : r[c];
                if (lane == c) Pc[32] = inv;
            }
            __syncwarp();
            if (lane == 0) {
                __threadfence_block();
                *prog = c + 1;
            }
            double v[32];
#pragma unroll
            for (int j = (c + 1) & ~1; j < 32; j += 2) {
                const double2 t = *reinterpret_cast<const double2 *>(Pc + j);
                v[j] = t.x;
                v[j + 1] = t.y;
            }
            auto upd = [&](int j) {
                if (FACT == FACT_GETRF) {
                    if (lane > c) r[j] -= r[c] * v[j];
                } else if (lane >= j) {
                    r[j] -= r[c] * v[j];
                }
            };
            if (c + 1 < 32) {
                upd(c + 1);
                if (c + 1 < nb) dg_pivot<FACT>(__shfl_sync(0xffffffffu, r[c + 1], c + 1), crit, np, d, inv);
            }
#pragma unroll
            for (int j = c + 2; j < 32; j++) upd(j);
        }
    }
    if (lane < nb)
#pragma unroll
        for (int j = 0; j < 32; j++)
            if (j < nb) W[lane * DG_LD + j] = r[j];
    return np;
}
// POTRF / SYTRF: the same factorization and publication by blocks of 8
// columns, so that the lanes exchange data once per block instead of once per
// column.  Step b: the 8 rows of the diagonal block write their entries to
// Blk; every lane factors that 8 x 8 block itself (the same arithmetic in every
// lane), solves its own row against it, writes and publishes the 8 values
// (Pub as above; Blk + 64 keeps row r's 8 values contiguous for the update)
// and updates the rest of its row; the row then moves 8 places left, so the
// loop over the blocks runs rolled with static register indices.  `Blk`: 320
// doubles, 16-byte aligned.  Block b is announced by an arrival at named
// barrier 1 + b (bar_n threads: this warp, the inverse warp and the warps that
// solve the rows below the block in step (dg_follow_rows), which wait there)
// instead of through *prog.
template <int FACT>
__device__ __noinline__ int dg_factor32_sym(double *W, int nb, double crit, double *Pub, volatile int *prog,
                                            double *Blk, int bar_n, double *gX, int ldx) {
    const int lane = threadIdx.x & 31;
    double *D8 = Blk, *Xr = Blk + 64;
    double r[32];
#pragma unroll
    for (int j = 0; j < 32; j++) r[j] = (lane < nb && j < nb) ? W[lane * DG_LD + j] : (lane == j ? 1.0 : 0.0);
    int np = 0;
#pragma unroll 1
    for (int jb = 0; jb < nb; jb += 8) {
        const int q = lane - jb;
        if (q >= 0 && q < 8) {
#pragma unroll
            for (int c = 0; c < 8; c += 2) *reinterpret_cast<double2 *>(D8 + q * 8 + c) = make_double2(r[c], r[c + 1]);
        }
        __syncwarp();
        double a[8][8];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int c = 0; c <= i; c += 2) {
                const double2 t = *reinterpret_cast<const double2 *>(D8 + i * 8 + c);
                a[i][c] = t.x;
                a[i][c + 1] = t.y;
            }
        // the 8 x 8 diagonal block, right looking (every lane alike)
        double dd[8], iv[8];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            int npc = 0;
            dg_pivot<FACT>((jb + c < nb) ? a[c][c] : 1.0, crit, npc, dd[c], iv[c]);  // identity beyond nb
            np += (jb + c < nb) ? npc : 0;
            double uc[8], lc[8];
#pragma unroll
            for (int i = c + 1; i < 8; i++) {
                uc[i] = a[i][c];
                lc[i] = uc[i] * iv[c];
                a[i][c] = lc[i];
            }
#pragma unroll
            for (int j = c + 1; j < 8; j++)
#pragma unroll
                for (int i = j; i < 8; i++) a[i][j] -= lc[i] * ((FACT == FACT_SYTRF) ? uc[j] : lc[j]);
        }
        // this lane's 8 values: L below the block's diagonal, the pivot on it, the
        // untouched upper part above it
        double x[8];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            // every term but the last is ready before x[c - 1]: one FMA and one product per column
            double sc = r[c];
#pragma unroll
            for (int k = 0; k < c; k++) sc -= x[k] * ((FACT == FACT_SYTRF) ? a[c][k] * dd[k] : a[c][k]);
            const double xc = sc * iv[c];
            x[c] = (lane > jb + c) ? xc : ((lane == jb + c) ? dd[c] : r[c]);
        }
        double pv[8];  // published: POTRF L(i, c); SYTRF D(c) L(i, c); the pivot on the diagonal
#pragma unroll
        for (int c = 0; c < 8; c++) pv[c] = (FACT == FACT_SYTRF && lane != jb + c) ? x[c] * dd[c] : x[c];
#pragma unroll
        for (int c = 0; c < 8; c++) {  // rows jb + c <= 31 of Pub exist even beyond nb (never read there)
            if (lane < nb && jb + c < nb) {
                W[lane * DG_LD + jb + c] = x[c];
                if (gX) gX[lane + (size_t)(jb + c) * ldx] = x[c];
            }
            Pub[(jb + c) * DG_BLD + lane] = pv[c];
            if (lane == c) Pub[(jb + c) * DG_BLD + 32] = iv[c];
        }
#pragma unroll
        for (int c = 0; c < 8; c += 2) *reinterpret_cast<double2 *>(Xr + lane * 8 + c) = make_double2(pv[c], pv[c + 1]);
        __syncwarp();
        // block published: release the inverse warp(s) waiting at named barrier 1 + jb / 8
        asm volatile("bar.arrive %0, %1;" ::"r"(1 + jb / 8), "r"(bar_n) : "memory");
        // rank-8 update of the rest of the row (lower part: columns jb + j <= lane), by
        // groups of 8 columns that exist; no branch inside a group, so its columns overlap
#pragma unroll
        for (int g = 8; g < 32; g += 8) {
            if (jb + g < 32) {
#pragma unroll
                for (int j = g; j < g + 8; j++) {
                    const double *xr = Xr + (jb + j) * 8;
                    double s0 = 0.0, s1 = 0.0;
#pragma unroll
                    for (int c = 0; c < 8; c += 2) {
                        const double2 t = *reinterpret_cast<const double2 *>(xr + c);
                        s0 += x[c] * t.x;
                        s1 += x[c + 1] * t.y;
                    }
                    const double nv = r[j] - (s0 + s1);
                    r[j] = (lane >= jb + j) ? nv : r[j];
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 24; j++) r[j] = r[j + 8];
#pragma unroll
        for (int j = 24; j < 32; j++) r[j] = 0.0;
        __syncwarp();  // D8 and Xr are rewritten by the next block
    }
    return np;
}

// One warp beside dg_factor32_sym: rows lane < nrows of W (row major, ld
// DG_LD: rows below the top block being factored, every earlier update
// applied) solved against the block's factor as it is published -- the
// off-diagonal TRSM of kernels/core_ztrsmsp.c by substitution, in step with the
// factorization instead of after it.  After named barrier 1 + jb / 8 (bar_n
// threads), with P(c, j) = Pub[jb + c][jb + j] (POTRF L(jb + j, jb + c), SYTRF
// D(jb + c) L(jb + j, jb + c)) and Pub[jb + c][32] = 1 / d:
//   x_c = (w_c - sum_{k<c} x_k P(k, c)) / d_c      (L(i, jb + c), written in place
//                                                   and to gX, column-major, ld ldx)
//   w_j -= sum_c x_c P(c, j)                        (the row's later columns)
// bar_n = 0: the factorization has published every block already (no waits).
template <int FACT>
__device__ __noinline__ void dg_follow_rows(double *W, int nrows, int nb, const double *Pub, int bar_n, double *gX,
                                            int ldx) {
    const int lane = threadIdx.x & 31;
    const bool own = lane < nrows;
    double r[32];
#pragma unroll
    for (int j = 0; j < 32; j++) r[j] = (own && j < nb) ? W[lane * DG_LD + j] : 0.0;
#pragma unroll 1
    for (int jb = 0; jb < nb; jb += 8) {
        if (bar_n) asm volatile("bar.sync %0, %1;" ::"r"(1 + jb / 8), "r"(bar_n) : "memory");
        const double *P = Pub + jb * DG_BLD + jb;
        double x[8];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            double sc = r[c];
#pragma unroll
            for (int k = 0; k < c; k++) sc -= x[k] * P[k * DG_BLD + c];
            x[c] = sc * Pub[(jb + c) * DG_BLD + 32];
        }
#pragma unroll
        for (int c = 0; c < 8; c++)
            if (own && jb + c < nb) {
                W[lane * DG_LD + jb + c] = x[c];
                gX[lane + (size_t)(jb + c) * ldx] = x[c];
            }
        // rank-8 update of the later columns, by groups of 8 that exist
#pragma unroll
        for (int g = 8; g < 32; g += 8) {
            if (jb + g < 32) {
#pragma unroll
                for (int j = g; j < g + 8; j++) {
                    double s0 = 0.0, s1 = 0.0;
#pragma unroll
                    for (int c = 0; c < 8; c += 2) {
                        s0 += x[c] * P[c * DG_BLD + j];
                        s1 += x[c + 1] * P[(c + 1) * DG_BLD + j];
                    }
                    r[j] -= s0 + s1;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 24; j++) r[j] = r[j + 8];
#pragma unroll
        for (int j = 24; j < 32; j++) r[j] = 0.0;
    }
}

// One warp: rows r < nrows of Wr (row major, ld DG_LD, 32 columns) lose the
// update of one finished panel, C -= A B: A(r, k) = Xa[r + k ldx] (the panel's
// rows, global memory), B (32 x 32, ld DG_LD, zero outside the blocks) staged
// in shared memory.  All 32 A loads of a lane are issued at once; DMMA 8 x 8 x 4.
__device__ __noinline__ void dg_rows_update(double *Wr, int nrows, const double *Xa, int ldx, const double *Bs) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    double av[4][8], c[4][4][2];
#pragma unroll
    for (int f = 0; f < 4; f++) {
        const int r = 8 * f + g;
        const bool ok = r < nrows;
#pragma unroll
        for (int ks = 0; ks < 8; ks++) av[f][ks] = ok ? -__ldcg(Xa + r + (size_t)(4 * ks + t4) * ldx) : 0.0;
#pragma unroll
        for (int cf = 0; cf < 4; cf++)
#pragma unroll
            for (int e = 0; e < 2; e++) c[f][cf][e] = ok ? Wr[r * DG_LD + 8 * cf + 2 * t4 + e] : 0.0;
    }
#pragma unroll
    for (int ks = 0; ks < 8; ks++)
#pragma unroll
        for (int cf = 0; cf < 4; cf++) {
            const double bb = Bs[(4 * ks + t4) * DG_LD + 8 * cf + g];
#pragma unroll
            for (int f = 0; f < 4; f++) dmma884(c[f][cf][0], c[f][cf][1], av[f][ks], bb);
        }
#pragma unroll
    for (int f = 0; f < 4; f++) {
        const int r = 8 * f + g;
        if (r < nrows)
#pragma unroll
            for (int cf = 0; cf < 4; cf++)
#pragma unroll
                for (int e = 0; e < 2; e++) Wr[r * DG_LD + 8 * cf + 2 * t4 + e] = c[f][cf][e];
    }
    __syncwarp();
}

template <int FACT>
__device__ __forceinline__ int dg_factor32(double *W, int nb, double crit, double *Pub, volatile int *prog,
                                           int bar_n = 64, double *gX = nullptr, int ldx = 0) {
    if (FACT != FACT_GETRF)
        return dg_factor32_sym<FACT>(W, nb, crit, Pub, prog, Pub + 32 * DG_BLD, bar_n, gX, ldx);
    return (nb == 32) ? dg_factor32_impl<FACT, true>(W, 32, crit, Pub, prog)
                      : dg_factor32_impl<FACT, false>(W, nb, crit, Pub, prog);
}

// One warp, next to the factorization of the top block: Z = T_jj^{-1} (side 0;
// side 1: GETRF's L^T) to shared memory (row major, ld DG_LD) and to `gZ`
// (32 x 32 row major), identity beyond nb.  With M = T^T lower triangular
// (POTRF L, SYTRF L D, GETRF U^T, or L for side 1), Z = (M^{-1})^T: lane j
// forms column j of M^{-1} by forward substitution, row i as soon as the
// factorization has published step i (M(i, k) = Pub[k][i], side 1 Pub[i][k]),
// so the inverse ends one step after the factorization.  POTRF / SYTRF wait at
// the named barrier of each 8-row block (bar_n threads); GETRF polls *prog, and a
// wait that runs past its bound records PGPU_STATUS_TIMEOUT in `status` and
// stops waiting.
template <typename T, int FACT>
__device__ __forceinline__ void dg_inverse_pipe(const double *Pub, int nb, int side, const volatile int *prog,
                                                double *Z, T *gZ, int *status, int bar_n = 64) {
    const int lane = threadIdx.x & 31;
    const bool lower_l = FACT == FACT_GETRF && side == 1;
    double y[32];
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 32; i++) {
        if (i < nb) {
            if (FACT != FACT_GETRF) {  // POTRF / SYTRF: block i / 8 announced at a named barrier
                if ((i & 7) == 0) asm volatile("bar.sync %0, %1;" ::"r"(1 + i / 8), "r"(bar_n) : "memory");
            } else {
                for (int spins = 0; ok && *prog <= i;)
                    if (++spins > DG_SPIN) ok = false;
                __threadfence_block();
            }
            const double rinv = lower_l ? 1.0 : Pub[i * DG_BLD + 32];
            double a0 = (i == lane) ? 1.0 : 0.0, a1 = 0.0;
#pragma unroll
            for (int k = 0; k < i; k++) {
                const double m = lower_l ? Pub[i * DG_BLD + k] : Pub[k * DG_BLD + i];
                if (k & 1) a1 -= m * y[k];
                else a0 -= m * y[k];
            }
            y[i] = (a0 + a1) * rinv;
        } else {
            y[i] = (i == lane) ? 1.0 : 0.0;
        }
    }
    if (!ok && lane == 0) atomicExch(status, PGPU_STATUS_TIMEOUT);
#pragma unroll
    for (int i = 0; i < 32; i++) Z[lane * DG_LD + i] = y[i];
    __syncwarp();
#pragma unroll 4
    for (int i = 0; i < 32; i++) gZ[i * 32 + lane] = (T)Z[i * DG_LD + lane];
}

// CTA-wide transfer of a rows x cols region in 8 x 4 sub-tiles: lane (g, t4)
// moves element (8 rb + g, 4 cb + t4), UNR sub-tiles in flight per warp, so
// both a column-major global side and a row-major (ld DG_LD) shared side are
// accessed without waste.
template <int UNR, typename LoadF, typename StoreF>
__device__ __forceinline__ void dg_copy(int rows, int cols, LoadF ld, StoreF stf) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int nrb = (rows + 7) >> 3, tot = nrb * ((cols + 3) >> 2);
    for (int i0 = warp; i0 < tot; i0 += nw * UNR) {
        double v[UNR];
#pragma unroll
        for (int u = 0; u < UNR; u++) {
            const int i = i0 + u * nw;
            const int r = 8 * (i % nrb) + g, c = 4 * (i / nrb) + t4;
            v[u] = (i < tot && r < rows && c < cols) ? ld(r, c) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < UNR; u++) {
            const int i = i0 + u * nw;
            const int r = 8 * (i % nrb) + g, c = 4 * (i / nrb) + t4;
            if (i < tot && r < rows && c < cols) stf(r, c, v[u]);
        }
    }
}

// One warp: X T = A for an 8 x 32 row fragment.  a_at(row, col) reads A,
// t_at(a, b) reads T (zero outside its upper nb x nb part), Z = T^{-1} in
// shared memory, Sw an 8 x DG_LD scratch of this warp; store(row, col, x).
template <typename AF, typename TF, typename SF>
__device__ __forceinline__ void dg_solve8(AF a_at, TF t_at, const double *Z, double *Sw, SF store) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    double x[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
    for (int ks = 0; ks < 8; ks++) {
        const double a = a_at(g, 4 * ks + t4);
#pragma unroll
        for (int cf = 0; cf < 4; cf++) dmma884(x[cf][0], x[cf][1], a, Z[(4 * ks + t4) * DG_LD + 8 * cf + g]);
    }
#pragma unroll
    for (int cf = 0; cf < 4; cf++) {
        Sw[g * DG_LD + 8 * cf + 2 * t4] = x[cf][0];
        Sw[g * DG_LD + 8 * cf + 2 * t4 + 1] = x[cf][1];
    }
    __syncwarp();
    double r[4][2];
#pragma unroll
    for (int cf = 0; cf < 4; cf++) {
        r[cf][0] = a_at(g, 8 * cf + 2 * t4);
        r[cf][1] = a_at(g, 8 * cf + 2 * t4 + 1);
    }
#pragma unroll
    for (int ks = 0; ks < 8; ks++) {
        const double a = -Sw[g * DG_LD + 4 * ks + t4];
#pragma unroll
        for (int cf = 0; cf < 4; cf++) dmma884(r[cf][0], r[cf][1], a, t_at(4 * ks + t4, 8 * cf + g));
    }
    __syncwarp();
#pragma unroll
    for (int cf = 0; cf < 4; cf++) {
        Sw[g * DG_LD + 8 * cf + 2 * t4] = r[cf][0];
        Sw[g * DG_LD + 8 * cf + 2 * t4 + 1] = r[cf][1];
    }
    __syncwarp();
#pragma unroll
    for (int ks = 0; ks < 8; ks++) {
        const double a = Sw[g * DG_LD + 4 * ks + t4];
#pragma unroll
        for (int cf = 0; cf < 4; cf++) dmma884(x[cf][0], x[cf][1], a, Z[(4 * ks + t4) * DG_LD + 8 * cf + g]);
    }
#pragma unroll
    for (int cf = 0; cf < 4; cf++) {
        store(g, 8 * cf + 2 * t4, x[cf][0]);
        store(g, 8 * cf + 2 * t4 + 1, x[cf][1]);
    }
    __syncwarp();
}

template <typename T, int FACT>
__global__ void __launch_bounds__(256, 1) k_diag_dmma(DevStruct s, const int *__restrict__ list, T *L, T *U, T *dinv,
                                                       FactParams fp) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *W = reinterpret_cast<double *>(smem_raw);  // (nc - jb) x 32 panel, row major, ld DG_LD
    __shared__ double Z0[32 * DG_LD], Z1[32 * DG_LD];
    __shared__ __align__(16) double Sx[8][8 * DG_LD];  // also the published steps of the top block's factorization
    __shared__ double dsh[32];
    __shared__ int npiv, prog;
    const int k = list[blockIdx.x];
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t4 = lane & 3;
    T *A = L + s.cb_coef[k];
    T *gZ = dinv + s.cb_dinv[k];
    const int nzb = (nc + 31) / 32;
    if (tid == 0) npiv = 0;
    if (FACT == FACT_GETRF) {  // L_kk += (U^T)_kk^T : the full diagonal block
        const T *Ut = U + s.cb_coef[k];
        batched_copy<8, T>(
            nc * nc, [&](int e) { int i = e % nc, j = e / nc; return A[i + (size_t)j * st] + Ut[j + (size_t)i * st]; },
            [&](int e, T v) { int i = e % nc, j = e / nc; A[i + (size_t)j * st] = v; });
    }
    __syncthreads();
    for (int jb = 0; jb < nc; jb += 32) {
        const int nb = min(32, nc - jb), m = nc - jb, t = m - nb;
        T *Ap = A + jb + (size_t)jb * st;  // top-left corner of the panel
        dg_copy<4>(
            m, 32, [&](int r, int c) { return (c < nb) ? (double)Ap[r + (size_t)c * st] : 0.0; },
            [&](int r, int c, double v) { W[r * DG_LD + c] = v; });
        if (tid == 0) prog = 0;
        __syncthreads();
        // 2. factor the top block (warp 0), one row per lane in registers; its inverse(s)
        //    one step behind (warps 1 and 2)
        if (warp == 0) {
            const int np = dg_factor32<FACT>(W, nb, __ldg(fp.criterion), &Sx[0][0], &prog);
            if (lane == 0 && np) npiv += np;
        } else if (warp == 1) {
            dg_inverse_pipe<T, FACT>(&Sx[0][0], nb, 0, &prog, Z0, gZ + (size_t)(jb / 32) * 1024, fp.status);
        } else if (FACT == FACT_GETRF && warp == 2) {
            dg_inverse_pipe<T, FACT>(&Sx[0][0], nb, 1, &prog, Z1, gZ + (size_t)(nzb + jb / 32) * 1024, fp.status);
        }
        __syncthreads();
        if (FACT == FACT_SYTRF && tid < 32) dsh[tid] = (tid < nb) ? W[tid * DG_LD + tid] : 0.0;
        __syncthreads();
        // 3. rows below the block (and the U strip of GETRF), 8 rows per warp
        const int nrf = (t + 7) / 8;
        for (int i = warp; i < nrf; i += 8) {
            const int r0 = 32 + 8 * i;
            dg_solve8(
                [&](int row, int col) { return (r0 + row < m) ? W[(r0 + row) * DG_LD + col] : 0.0; },
                [&](int a, int b) { return (a <= b && b < nb) ? dg_t<FACT>(W, a, b, 0) : 0.0; }, Z0, Sx[warp],
                [&](int row, int col, double v) {
                    if (r0 + row < m) W[(r0 + row) * DG_LD + col] = v;
                });
        }
        if (FACT == FACT_GETRF) {  // U12^T (t x 32, columns of the panel's upper part) X L11^T = U12^T
            for (int i = warp; i < nrf; i += 8) {
                const int q0 = 32 + 8 * i;
                dg_solve8(
                    [&](int row, int col) {
                        return (q0 + row < m) ? (double)Ap[col + (size_t)(q0 + row) * st] : 0.0;
                    },
                    [&](int a, int b) { return (a <= b && b < nb) ? dg_t<FACT>(W, a, b, 1) : 0.0; }, Z1, Sx[warp],
                    [&](int row, int col, double v) {
                        if (q0 + row < m) Ap[col + (size_t)(q0 + row) * st] = (T)v;
                    });
            }
        }
        __syncthreads();
        dg_copy<4>(
            m, nb, [&](int r, int c) { return W[r * DG_LD + c]; },
            [&](int r, int c, double v) { Ap[r + (size_t)c * st] = (T)v; });
        // 4. trailing update A22 -= L21 B^T in 16 x 16 blocks (B = L21, L21 D or U12^T)
        if (t > 0) {
            T *C = Ap + 32 + (size_t)32 * st;
            const int nbk = (t + 15) / 16;
            const int tot = (FACT == FACT_GETRF) ? nbk * nbk : nbk * (nbk + 1) / 2;
            // each warp keeps DG_NBLK blocks in flight: their C loads are issued together
            constexpr int NB = DG_NBLK;
            for (int id0 = warp; id0 < tot; id0 += 8 * NB) {
                int bi[NB], bj[NB];
                double c[NB][2][2][2];
#pragma unroll
                for (int u = 0; u < NB; u++) {
                    const int id = id0 + 8 * u;
                    if (FACT == FACT_GETRF) {
                        bi[u] = id % nbk;
                        bj[u] = id / nbk;
                    } else {
                        int x = (int)((sqrt(8.0 * id + 1.0) - 1.0) * 0.5);
                        while (x * (x + 1) / 2 > id) x--;
                        while ((x + 1) * (x + 2) / 2 <= id) x++;
                        bi[u] = x;
                        bj[u] = id - x * (x + 1) / 2;
                    }
                    if (id >= tot) bi[u] = bj[u] = nbk;  // no block: every row and column masked
#pragma unroll
                    for (int rf = 0; rf < 2; rf++)
#pragma unroll
                        for (int cf = 0; cf < 2; cf++)
#pragma unroll
                            for (int e = 0; e < 2; e++) {
                                const int r = 16 * bi[u] + 8 * rf + g, q = 16 * bj[u] + 8 * cf + 2 * t4 + e;
                                const bool ok = r < t && q < t && (FACT == FACT_GETRF || r >= q);
                                c[u][rf][cf][e] = ok ? (double)C[r + (size_t)q * st] : 0.0;
                            }
                }
#pragma unroll
                for (int ks = 0; ks < 8; ks++) {
                    const int kk = 4 * ks + t4;
#pragma unroll
                    for (int u = 0; u < NB; u++) {
                        double a[2], b[2];
#pragma unroll
                        for (int rf = 0; rf < 2; rf++) {
                            const int r = 16 * bi[u] + 8 * rf + g;
                            a[rf] = (r < t) ? -W[(32 + r) * DG_LD + kk] : 0.0;
                        }
#pragma unroll
                        for (int cf = 0; cf < 2; cf++) {
                            const int q = 16 * bj[u] + 8 * cf + g;
                            if (FACT == FACT_GETRF) b[cf] = (q < t) ? (double)Ap[kk + (size_t)(32 + q) * st] : 0.0;
                            else if (FACT == FACT_SYTRF) b[cf] = (q < t) ? W[(32 + q) * DG_LD + kk] * dsh[kk] : 0.0;
                            else b[cf] = (q < t) ? W[(32 + q) * DG_LD + kk] : 0.0;
                        }
#pragma unroll
                        for (int rf = 0; rf < 2; rf++)
#pragma unroll
                            for (int cf = 0; cf < 2; cf++)
                                dmma884(c[u][rf][cf][0], c[u][rf][cf][1], a[rf], b[cf]);
                    }
                }
#pragma unroll
                for (int u = 0; u < NB; u++)
#pragma unroll
                    for (int rf = 0; rf < 2; rf++)
#pragma unroll
                        for (int cf = 0; cf < 2; cf++)
#pragma unroll
                            for (int e = 0; e < 2; e++) {
                                const int r = 16 * bi[u] + 8 * rf + g, q = 16 * bj[u] + 8 * cf + 2 * t4 + e;
                                if (r < t && q < t && (FACT == FACT_GETRF || r >= q))
                                    C[r + (size_t)q * st] = (T)c[u][rf][cf][e];
                            }
            }
        }
        __syncthreads();
    }
    if (FACT == FACT_SYTRF) {  // upper part of the diagonal block holds D L^T
        batched_copy<8, T>(
            nc * nc,
            [&](int e) {
                int i = e % nc, j = e / nc;
                return (i < j) ? A[i + (size_t)i * st] * A[j + (size_t)i * st] : T(0);
            },
            [&](int e, T v) { int i = e % nc, j = e / nc; if (i < j) A[i + (size_t)j * st] = v; });
    }
    if (FACT == FACT_GETRF) {  // (U^T)_kk = (L\U)_kk^T
        T *Ut = U + s.cb_coef[k];
        batched_copy<8, T>(
            nc * nc, [&](int e) { int i = e % nc, j = e / nc; return A[i + (size_t)j * st]; },
            [&](int e, T v) { int i = e % nc, j = e / nc; Ut[j + (size_t)i * st] = v; });
    }
    if (tid == 0 && npiv) atomicAdd(fp.nbpivots, npiv);
}

// ---------------------------------------------------------------------------
// Diagonal block of a wide cblk factored by a cluster of DC CTAs (one per SM)
// that keeps the whole block in shared memory: 32-column panel p lives in the
// shared memory of CTA p % DC (rows 32 p .. nc - 1, all rows for GETRF, FP64,
// row major, ld DG_LD).  Step p: the owner factors panel p (top block in
// registers, inverse, rows below by X = X0 + (A - X0 T) Z on DMMA) and writes
// it out; after a cluster barrier every CTA updates its own panels q > p,
// reading panel p from the owner's shared memory (distributed shared memory)
// -- for GETRF first the U block U_pq = L_pp^{-1} A_pq, as in the right
// looking core_zgetrfsp.  Nothing of the trailing matrix goes through global
// memory, so the step is bound by the owner's factorization and the cluster
// barrier rather than by L2 round trips.
// ---------------------------------------------------------------------------
constexpr int DC = 8;                      // CTAs per cluster
constexpr int DC_MIN_NC = 96;              // narrower blocks stay on one CTA
// dynamic shared memory next to the static ~37 KB
__host__ __device__ constexpr long long dc_max_smem(int) { return 180 * 1024LL; }
constexpr int DC_SLOTS = (DG_MAXNC / 32 + DC - 1) / DC;  // panels one CTA can own (nc <= DG_MAXNC)
// POTRF / SYTRF: every finished panel is also written (FP64, column-major nc x nc,
// from its top row down) to a per-cblk area of global memory, from which the
// other CTAs read it for their updates: eight CTAs reading one CTA's shared
// memory at once through the cluster are bound by that one SM, while L2 serves
// them in parallel.
constexpr size_t DC_SCR_DOUBLES = (size_t)DG_MAXNC * DG_MAXNC;
constexpr int DC_MAX_CLUSTERS = 160 / DC;  // cblks of one launch: count * DC <= SM count

__host__ __device__ inline int dc_lo(int p, int fact) { return fact == FACT_GETRF ? 0 : 32 * p; }
// Shared memory (doubles) of the panels CTA `rank` owns for a block of width nc.
__host__ __device__ inline long long dc_panel_doubles(int nc, int fact, int rank) {
    const int np = (nc + 31) / 32;
    long long n = 0;
    for (int p = rank; p < np; p += DC) n += (long long)(nc - dc_lo(p, fact)) * DG_LD;
    return n;
}
// GETRF: the inverted (L_pp)^T of each panel a CTA factors, read by the other
// CTAs, one slot per panel it owns, ahead of the panels
__host__ __device__ inline long long dc_zs1_doubles(int fact) {
    return fact == FACT_GETRF ? (long long)DC_SLOTS * 32 * DG_LD : 0;
}
__host__ __device__ inline long long diag_cluster_smem_bytes(int nc, int fact) {
    return 8 * (dc_zs1_doubles(fact) + dc_panel_doubles(nc, fact, 0));  // CTA 0 holds the most
}

// Cluster-scope flag of one CTA, read from another CTA of the cluster.
__device__ __forceinline__ uint32_t dsmem_map(const void *local, int rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(r)
                 : "r"((uint32_t)__cvta_generic_to_shared(local)), "r"(rank));
    return r;
}
__device__ __forceinline__ int dsmem_ld_acquire(uint32_t addr) {
    int v;
    asm volatile("ld.acquire.cluster.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ void dsmem_st_release(uint32_t addr, int v) {
    asm volatile("st.release.cluster.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
// Wait until the cluster-shared flag at `addr` reaches `target`, with back-off;
// false once DG_SPIN polls have gone by without it.
__device__ __forceinline__ bool dc_wait(uint32_t addr, int target) {
    for (int spins = 0; dsmem_ld_acquire(addr) < target;) {
        if (++spins > DG_SPIN) return false;
        __nanosleep(20);
    }
    return true;
}

template <typename T, int FACT>
__global__ void __cluster_dims__(DC, 1, 1) __launch_bounds__(256, 1)
    k_diag_cluster(DevStruct s, const int *__restrict__ list, T *L, T *U, T *dinv, FactParams fp) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // GETRF: inverted (L_pp)^T of each panel factored here (read by the other CTAs
    // for U_pq), one slot per panel; then this CTA's panels, one after the other
    double *Zs1 = reinterpret_cast<double *>(smem_raw);
    double *Wl = Zs1 + dc_zs1_doubles(FACT);
    __shared__ double Zs0[32 * DG_LD];                   // inverted top block of the panel being factored here
    __shared__ __align__(16) double Sx[8][8 * DG_LD];  // also the published steps of the top block's factorization
    __shared__ double Tb[32 * DG_LD];                    // the top block being factored
    __shared__ double Bs[32 * DG_LD];                    // an update's B block
    __shared__ int npiv, prog, fpart, fdone;             // announcements of this CTA's panels (below)
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int k = list[blockIdx.x / DC];
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int np = (nc + 31) / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t4 = lane & 3;
    T *A = L + s.cb_coef[k];
    T *gZ = dinv + s.cb_dinv[k];
    double *X = fp.dscr + (size_t)(blockIdx.x / DC) * DC_SCR_DOUBLES;  // this cblk's finished panels (POTRF / SYTRF)
    const double crit = __ldg(fp.criterion);  // read once, off the panel steps' chain
    if (tid == 0) {
        npiv = 0;
        fpart = 0;
        fdone = 0;
    }
    // panel p of CTA p % DC: its offset inside that CTA's shared memory
    auto poff = [&](int p) {
        long long off = 0;
        for (int q = p % DC; q < p; q += DC) off += (long long)(nc - dc_lo(q, FACT)) * DG_LD;
        return off;
    };
    auto panel = [&](int p) -> double * {  // generic pointer, local or in another CTA of the cluster
        double *base = cluster.map_shared_rank(Wl, p % DC);
        return base + poff(p);
    };
    // load this CTA's panels (GETRF: L_kk += (U^T)_kk^T on the way)
    for (int p = rank; p < np; p += DC) {
        const int lo = dc_lo(p, FACT), rows = nc - lo, nb = min(32, nc - 32 * p);
        double *W = Wl + poff(p);
        const T *Ut = U + s.cb_coef[k];
        dg_copy<12>(
            rows, 32,
            [&](int r, int c) {
                if (c >= nb) return 0.0;
                const int i = lo + r, j = 32 * p + c;
                double v = (double)A[i + (size_t)j * st];
                if (FACT == FACT_GETRF) v += (double)Ut[j + (size_t)i * st];
                return v;
            },
            [&](int r, int c, double v) { W[r * DG_LD + c] = v; });
    }
    cluster.sync();  // panels loaded and flags cleared in every CTA before any flag is read

    // Panels are announced through this CTA's flags: fdone = p + 1 once all rows
    // of panel p are final.  GETRF announces in two stages: fpart = p + 1 once
    // its factored top block and the rows that form the top block of panel p + 1
    // are final; the owner of panel p + 1 starts on its top block at fpart, so
    // the rest of panel p's TRSM and every other update run beside the chain
    //   rows of p for p + 1's top -> p + 1's top updated -> factored -> ...
    auto publish = [&](int *flag, int p) {
        __syncthreads();
        if (tid == 0) {
            asm volatile("fence.acq_rel.cluster;" ::: "memory");
            dsmem_st_release(dsmem_map(flag, rank), p + 1);
        }
    };
    // Wait until the owner of panel p has raised `flag` to p + 1 (bounded; on
    // expiry the status word records PGPU_STATUS_TIMEOUT and the CTA carries on,
    // so that the kernel ends).
    auto wait_flag = [&](int *flag, int p) {
        if (p % DC != rank && tid == 0 && !dc_wait(dsmem_map(flag, p % DC), p + 1))
            atomicExch(fp.status, PGPU_STATUS_TIMEOUT);
        __syncthreads();
    };
    // Top block of this CTA's panel p (every update from panels < p applied to
    // it): factored by warp 0 with static pivoting, inverted beside it.
    auto factor_top = [&](int p) {
        const int nb = min(32, nc - 32 * p);
        const int lop = dc_lo(p, FACT);
        double *Wt = Wl + poff(p) + (32 * p - lop) * DG_LD;  // top block
        double *Z1 = (FACT == FACT_GETRF) ? Zs1 + (p / DC) * 32 * DG_LD : Zs1;
        for (int e = tid; e < nb * DG_LD; e += blockDim.x) Tb[e] = Wt[e];  // the panel has nb rows left at its top
        if (tid == 0) prog = 0;
        __syncthreads();
        if (warp == 0) {
            const int n = dg_factor32<FACT>(Tb, nb, crit, &Sx[0][0], &prog);
            if (lane == 0 && n) npiv += n;
        } else if (warp == 1) {
            dg_inverse_pipe<T, FACT>(&Sx[0][0], nb, 0, &prog, Zs0, gZ + (size_t)p * 1024, fp.status);
        } else if (FACT == FACT_GETRF && warp == 2) {
            dg_inverse_pipe<T, FACT>(&Sx[0][0], nb, 1, &prog, Z1, gZ + (size_t)(np + p) * 1024, fp.status);
        }
        __syncthreads();
        for (int e = tid; e < nb * DG_LD; e += blockDim.x) Wt[e] = Tb[e];
        __syncthreads();
    };
    // Rows [ra, rb) (below the top block) of this CTA's panel p against its
    // factored top block (still in Tb, inverse in Zs0): X T = A.
    auto trsm_rows = [&](int p, int ra, int rb) {
        const int nb = min(32, nc - 32 * p);
        const int lop = dc_lo(p, FACT);
        double *W = Wl + poff(p);
        const double *Wt = W + (32 * p - lop) * DG_LD;  // the factored top block
        rb = min(rb, nc);
        const int nrf = (rb - ra + 7) / 8;
        for (int i = warp; i < nrf; i += 8) {
            const int r8 = ra + 8 * i;
            dg_solve8(
                [&](int row, int col) { return (r8 + row < rb) ? W[(r8 + row - lop) * DG_LD + col] : 0.0; },
                [&](int a, int b) { return (a <= b && b < nb) ? dg_t<FACT>(Wt, a, b, 0) : 0.0; }, Zs0, Sx[warp],
                [&](int row, int col, double v) {
                    if (r8 + row < rb) {
                        W[(r8 + row - lop) * DG_LD + col] = v;
                        if (FACT != FACT_GETRF && col < nb) X[(r8 + row) + (size_t)(32 * p + col) * nc] = v;
                    }
                });
        }
    };
    // Rows [ra, rb) of this CTA's panel q updated by the factored panel p (read
    // remotely).  GETRF: the call that starts at the first row also forms the
    // U block U_pq = L_pp^{-1} A_pq that every row's update reads.
    auto update_rows = [&](int p, int q, int ra, int rb) {
        const int nb = min(32, nc - 32 * p);
        const int lop = dc_lo(p, FACT);
        const double *Wp = panel(p);
        const double *Wpt = Wp + (32 * p - lop) * DG_LD;
        const int nbq = min(32, nc - 32 * q);
        const int loq = dc_lo(q, FACT);
        double *Wq = Wl + poff(q);
        if (q >= np) return;  // (uniform) no such panel
        const int rs = (FACT == FACT_GETRF) ? 32 * p + 32 : 32 * q;
        if (FACT == FACT_GETRF && ra <= rs) {  // (U_pq)^T L_pp^T = (A_pq)^T, 8 columns per warp
            const double *Zr = cluster.map_shared_rank(Zs1 + (p / DC) * 32 * DG_LD, p % DC);
            double *Ab = Wq + (32 * p - loq) * DG_LD;  // rows 32 p .. 32 p + 31 of panel q
            if (warp < 4) {
                const int c0 = 8 * warp;
                dg_solve8(
                    [&](int row, int col) { return (c0 + row < nbq) ? Ab[col * DG_LD + c0 + row] : 0.0; },
                    [&](int a, int b) { return (a <= b && b < nb) ? dg_t<FACT>(Wpt, a, b, 1) : 0.0; }, Zr,
                    Sx[warp], [&](int row, int col, double v) {
                        if (c0 + row < nbq) Ab[col * DG_LD + c0 + row] = v;
                    });
            }
            __syncthreads();
        }
        ra = max(ra, rs);
        rb = min(rb, nc);
        if (ra >= rb) return;
        // B block of this update (32 x 32: k by the columns of panel q) staged
        // locally, every remote load of a thread issued before its stores
        double bv[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = tid + 256 * u, kk = e >> 5, cc = e & 31;
            double b = 0.0;
            if (cc < nbq && kk < nb) {
                if (FACT == FACT_GETRF) b = Wq[(32 * p + kk - loq) * DG_LD + cc];
                else {
                    const double *Xp = X + (size_t)(32 * p + kk) * nc;  // column 32 p + kk
                    b = __ldcg(Xp + 32 * q + cc);
                    if (FACT == FACT_SYTRF) b *= __ldcg(Xp + 32 * p + kk);
                }
            }
            bv[u] = b;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = tid + 256 * u;
            Bs[(e >> 5) * DG_LD + (e & 31)] = bv[u];
        }
        __syncthreads();
        // two 8-row fragments per warp at a time: their 16 remote A values are
        // requested together and their DMMA chains interleave
        const int nrf = (rb - ra + 7) / 8;
        for (int i = warp; i < nrf; i += 16) {
            double av[2][8], c[2][4][2];
            bool rowok[2];
#pragma unroll
            for (int f = 0; f < 2; f++) {
                const int r = ra + 8 * (i + 8 * f) + g;
                rowok[f] = (i + 8 * f < nrf) && r < rb;
#pragma unroll
                for (int ks = 0; ks < 8; ks++) {
                    if (FACT == FACT_GETRF) av[f][ks] = rowok[f] ? -Wp[(r - lop) * DG_LD + 4 * ks + t4] : 0.0;
                    else av[f][ks] = rowok[f] ? -__ldcg(X + r + (size_t)(32 * p + 4 * ks + t4) * nc) : 0.0;
                }
#pragma unroll
                for (int cf = 0; cf < 4; cf++)
#pragma unroll
                    for (int e = 0; e < 2; e++)
                        c[f][cf][e] = rowok[f] ? Wq[(r - loq) * DG_LD + 8 * cf + 2 * t4 + e] : 0.0;
            }
#pragma unroll
            for (int ks = 0; ks < 8; ks++)
#pragma unroll
                for (int cf = 0; cf < 4; cf++) {
                    const double bb = Bs[(4 * ks + t4) * DG_LD + 8 * cf + g];
#pragma unroll
                    for (int f = 0; f < 2; f++) dmma884(c[f][cf][0], c[f][cf][1], av[f][ks], bb);
                }
#pragma unroll
            for (int f = 0; f < 2; f++) {
                const int r = ra + 8 * (i + 8 * f) + g;
#pragma unroll
                for (int cf = 0; cf < 4; cf++)
#pragma unroll
                    for (int e = 0; e < 2; e++)
                        if (rowok[f]) Wq[(r - loq) * DG_LD + 8 * cf + 2 * t4 + e] = c[f][cf][e];
            }
        }
        __syncthreads();
    };
    // Rows of panel p after its top block: first those that form the top block
    // of panel p + 1, announced at once, then the others.
    auto finish_panel = [&](int p) {
        const int r0 = 32 * p + 32;
        trsm_rows(p, r0, r0 + 32);
        publish(&fpart, p);
        trsm_rows(p, r0 + 32, nc);
        publish(&fdone, p);
    };

    // POTRF / SYTRF: panel q, every update but that of panel pu (-1: none)
    // applied, and that one applied to its top block (B block of the update
    // still staged in Bs).  Warp 0 factors the top block in place, warp 1
    // inverts it one step behind, and up to six more warps each take 32 rows
    // below it: they apply panel pu's update to their rows (dg_rows_update)
    // while the factorization starts, then solve the rows in step with it
    // (dg_follow_rows), so the panel is final one block step after its top
    // block and is announced then (fdone = q + 1), while the inverse (kept for
    // the later TRSM kernels and the solve) is still being written.  Rows beyond
    // the followers' 192 (blocks wider than 224 columns, first panels) are
    // taken 32 at a time by the same warps once their first rows are done,
    // against the then complete factorization.
    // panel p (final) from shared memory to the factor in global memory
    auto write_panel = [&](int p) {
        const int lop = dc_lo(p, FACT), nb = min(32, nc - 32 * p);
        const double *W = Wl + poff(p);
        dg_copy<8>(
            nc - lop, nb, [&](int r, int c) { return W[r * DG_LD + c]; },
            [&](int r, int c, double v) { A[(lop + r) + (size_t)(32 * p + c) * st] = (T)v; });
    };
    constexpr int DC_FOLLOW = 6;
    auto factor_panel = [&](int q, int pu) {
        const int nb = min(32, nc - 32 * q);
        double *W = Wl + poff(q);  // lo = 32 q: the top block is the panel's first nb rows
        const int nr = nc - 32 * q - nb;
        const int nch = (nr + 31) / 32;  // 32-row chunks below the top block
        const int F = min(DC_FOLLOW, nch);
        const int bar_n = 64 + 32 * F;
        __syncthreads();
        double *Xq = X + 32 * q + (size_t)(32 * q) * nc;  // the panel's mirror from its top row
        if (warp == 0) {
            const int n = dg_factor32<FACT>(W, nb, crit, &Sx[0][0], &prog, bar_n, Xq, nc);
            if (lane == 0 && n) npiv += n;
        } else if (warp == 1) {
            dg_inverse_pipe<T, FACT>(&Sx[0][0], nb, 0, &prog, Zs0, gZ + (size_t)q * 1024, fp.status, bar_n);
        } else if (warp - 2 < F) {
            for (int f = warp - 2; f < nch; f += DC_FOLLOW) {
                double *Wf = W + (nb + 32 * f) * DG_LD;
                const int nrows = min(32, nr - 32 * f);
                if (pu >= 0) dg_rows_update(Wf, nrows, X + 32 * q + nb + 32 * f + (size_t)(32 * pu) * nc, nc, Bs);
                dg_follow_rows<FACT>(Wf, nrows, nb, &Sx[0][0], f < DC_FOLLOW ? bar_n : 0, Xq + nb + 32 * f, nc);
            }
        }
        if (warp != 1 && warp < 2 + F) {
            asm volatile("bar.sync 5, %0;" ::"r"(32 * (1 + F)) : "memory");
            if (tid == 0) {
                asm volatile("fence.acq_rel.cluster;" ::: "memory");
                dsmem_st_release(dsmem_map(&fdone, rank), q + 1);
            }
        }
        __syncthreads();
    };

    if (FACT != FACT_GETRF) {
        // a panel goes out to the factor as soon as it is final and the CTA's
        // updates of the step are issued: the CTA waits for the next panels anyway
        int wq = -1;  // the panel this CTA finished last, not yet written
        if (rank == 0) {
            factor_panel(0, -1);
            wq = 0;
        }
        for (int p = 0; p + 1 < np; p++) {
            const int q1 = p + 1;
            int q0 = q1 + ((rank - q1) % DC + DC) % DC;  // this CTA's first panel after p
            wait_flag(&fdone, p);
            if (q0 == q1) {  // the critical chain: panel p + 1 as soon as panel p is final
                update_rows(p, q1, 0, 32 * q1 + 32);  // its top block; the rows below in factor_panel
                factor_panel(q1, p);
                q0 += DC;
                wq = q1;
            }
            for (int q = q0; q < np; q += DC) update_rows(p, q, 0, nc);
            if (wq >= 0) {
                write_panel(wq);
                wq = -1;
            }
        }
        if (wq >= 0) write_panel(wq);
    } else {
        if (rank == 0) {
            factor_top(0);
            finish_panel(0);
        }
        for (int p = 0; p + 1 < np; p++) {
            const int q1 = p + 1;
            int q0 = q1 + ((rank - q1) % DC + DC) % DC;  // this CTA's first panel after p
            if (q0 == q1) {
                // the critical chain: p + 1's top block as soon as the rows it needs are final
                wait_flag(&fpart, p);
                update_rows(p, q1, 0, 32 * q1 + 32);
                factor_top(q1);
                wait_flag(&fdone, p);
                update_rows(p, q1, 32 * q1 + 32, 32 * q1 + 64);  // the rows of p + 2's top block
                const int r0 = 32 * q1 + 32;
                trsm_rows(q1, r0, r0 + 32);
                publish(&fpart, q1);
                update_rows(p, q1, 32 * q1 + 64, nc);
                trsm_rows(q1, r0 + 32, nc);
                publish(&fdone, q1);
                q0 += DC;
            } else {
                wait_flag(&fdone, p);
            }
            for (int q = q0; q < np; q += DC) update_rows(p, q, 0, nc);
        }
    }
    wait_flag(&fdone, np - 1);  // every panel is final before the write-out and the tail below
    // GETRF: this CTA's panels are final: write them out
    if (FACT == FACT_GETRF)
        for (int p = rank; p < np; p += DC) write_panel(p);
    __threadfence();
    cluster.sync();  // all panels written; no CTA leaves while its shared memory may still be read
    if (rank == 0) {
        if (FACT == FACT_SYTRF) {  // upper part of the diagonal block holds D L^T
            batched_copy<8, T>(
                nc * nc,
                [&](int e) {
                    int i = e % nc, j = e / nc;
                    return (i < j) ? A[i + (size_t)i * st] * A[j + (size_t)i * st] : T(0);
                },
                [&](int e, T v) { int i = e % nc, j = e / nc; if (i < j) A[i + (size_t)j * st] = v; });
        }
        if (FACT == FACT_GETRF) {  // (U^T)_kk = (L\U)_kk^T
            T *Ut = U + s.cb_coef[k];
            batched_copy<8, T>(
                nc * nc, [&](int e) { int i = e % nc, j = e / nc; return A[i + (size_t)j * st]; },
                [&](int e, T v) { int i = e % nc, j = e / nc; Ut[j + (size_t)i * st] = v; });
        }
    }
    __syncthreads();
    if (tid == 0 && npiv) atomicAdd(fp.nbpivots, npiv);
}

// ---------------------------------------------------------------------------
// FP32 update GEMM with fused scatter-add on the 5th-generation tensor cores
// (tcgen05.mma kind::f16, FP32 accumulator in tensor memory).
//
// Operands.  Each FP32 panel value is split once into three BF16 terms
// a = a0 + a1 + a2 (24 significant bits) by k_split, right after its level's
// TRSM, into an image laid out exactly as the tensor cores read shared memory
// (K-major, no swizzle, core matrices of 8 rows x 16 bytes).  The product of a
// tile is accumulated from the six terms a_i b_j with i + j <= 2; the dropped
// terms are below 2^-24 of the product.
//
// Image of cblk k (bytes from sp_off[k]): term p, K block kb of TC_BK
// columns, row group g of 8 panel rows at ((p * nkb + kb) * ng + g) * TC_GROUP;
// inside a group, column chunk c (8 columns) at 128 c, row r at 16 r, column j
// at 2 j.  ng = ceil(stride / 8) + 16 so that a window of 16 row groups from
// any row group of the panel stays inside the (zero padded) image.
//
// Tiles.  A task's A rows and B rows are covered by 128-row windows aligned to
// row groups; rows and columns outside the task are masked in the epilogue.
// The tile loop itself (bulk copies through mbarrier stages, MMAs, tensor
// memory epilogue) is the persistent engine tc_persistent below.  Every wait
// is bounded; on expiry the kernel records PGPU_STATUS_TIMEOUT and returns.
// ---------------------------------------------------------------------------
constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 32;
constexpr int TC_CH = TC_BK / 8;                    // 8-column chunks per K block
constexpr int TC_GROUP = 128 * TC_CH;               // bytes of 8 rows x TC_BK columns of one term
constexpr int TC_PIECE = (TC_BM / 8) * TC_GROUP;    // one term of a 128-row operand block
constexpr int TC_STAGE = 6 * TC_PIECE;              // A0 A1 A2 B0 B1 B2
constexpr int TC_SPIN = 1 << 20;                    // try_wait rounds before giving up

__host__ __device__ inline int split_nkb(int nc) { return (nc + TC_BK - 1) / TC_BK; }
__host__ __device__ inline int split_ng(int st) { return (st + 7) / 8 + 16; }
__host__ __device__ inline long long split_bytes(int nc, int st) {
    return 3LL * split_nkb(nc) * split_ng(st) * TC_GROUP;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared memory matrix descriptor: K-major, no swizzle; the next 8 K elements
// 128 bytes on (LBO), the next 8 rows TC_GROUP bytes on (SBO); version 1.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
           ((uint64_t)(TC_GROUP >> 4) << 32) | (1ull << 46);
}
// Instruction descriptor: BF16 x BF16 -> FP32, both operands K-major, M = 128, N = n.
__device__ __forceinline__ uint32_t tc_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
// Bounded wait for the completion of the phase of `bar` with parity `parity`.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (int it = 0; it < TC_SPIN; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bulk copy global -> shared (this GPU's memory, no multicast), completion on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}
// a = t0 + t1 + t2 in BF16 (round to nearest at each step), as 16-bit patterns.
__device__ __forceinline__ void split_bf16x3(float a, uint32_t &t0, uint32_t &t1, uint32_t &t2) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(a);
    float r = a - __bfloat162float(h0);
    const __nv_bfloat16 h1 = __float2bfloat16_rn(r);
    r -= __bfloat162float(h1);
    const __nv_bfloat16 h2 = __float2bfloat16_rn(r);
    t0 = __bfloat16_as_ushort(h0);
    t1 = __bfloat16_as_ushort(h1);
    t2 = __bfloat16_as_ushort(h2);
}

// Split 128-row slabs of FP32 panels into their BF16 image.  `scale` multiplies
// column c by the diagonal entry D[c][c] of the panel (the L D operand of LDL^T).
// CTAs per 128-row slab in k_split / k_split_dense: the slab's 8-column chunks
// are spread over them, so that the few tall panels of the upper levels are
// converted by many SMs instead of one CTA walking ~40 chunks in sequence.
constexpr int SPLIT_CTAS = 8;

__global__ void __launch_bounds__(256) k_split(DevStruct s, const SplitSlab *__restrict__ slabs, const float *P,
                                               const float *Dp, const int64_t *__restrict__ sp_off,
                                               unsigned char *img, int scale) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    const SplitSlab sl = slabs[blockIdx.x];
    const int k = sl.cblk;
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int nkb = split_nkb(nc), ng = split_ng(st);
    const float *A = P + s.cb_coef[k];
    const float *D = Dp + s.cb_coef[k];
    unsigned char *out = img + sp_off[k];
    const int rows = min(128, 8 * ((st + 7) / 8) - sl.r0);  // whole row groups of the panel
    const int nch = TC_CH * nkb;                             // 8-column chunks
    // the slab's chunks go round robin to the gridDim.y CTAs of the slab
    const int G = gridDim.y, nq = (nch - (int)blockIdx.y + G - 1) / G;
    const int items = 128 * max(nq, 0);
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int r = it & 127, ch = (int)blockIdx.y + (it >> 7) * G;
        if (r >= rows) continue;
        const int pr = sl.r0 + r;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int c = 8 * ch + j;
            v[j] = (pr < st && c < nc) ? A[pr + (size_t)c * st] : 0.f;
            if (scale && pr < st && c < nc) v[j] *= D[c + (size_t)c * st];
        }
        uint32_t w[3][4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            uint32_t a0, a1, a2, b0, b1, b2;
            split_bf16x3(v[2 * j], a0, a1, a2);
            split_bf16x3(v[2 * j + 1], b0, b1, b2);
            w[0][j] = a0 | (b0 << 16);
            w[1][j] = a1 | (b1 << 16);
            w[2][j] = a2 | (b2 << 16);
        }
        const size_t base = (size_t)(ch / TC_CH) * ng * TC_GROUP + (size_t)(pr >> 3) * TC_GROUP +
                            (ch % TC_CH) * 128 + (pr & 7) * 16;
#pragma unroll
        for (int p = 0; p < 3; p++)
            *reinterpret_cast<uint4 *>(out + base + (size_t)p * nkb * ng * TC_GROUP) =
                make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
    }
}

// Operands of one 128 x nmma tile: A rows from row group ga of a BF16 image
// with ngA row groups, B rows from group gb of one with ngB groups; nkb K
// blocks; `term*` bytes between the three terms of an image.
struct TcOperands {
    const unsigned char *iA, *iB;
    size_t termA, termB;
    int ngA, ngB, nkb, ga, gb, nmma;
};

// ---------------------------------------------------------------------------
// Inverse of the upper triangular factor T of a wide cblk's diagonal block
// (T as in the off-diagonal TRSM: L^T for POTRF, D L^T for SYTRF, U and L^T
// for the two GETRF sides), so that the FP32 TRSM X T = A becomes the GEMM
// X = A T^{-1} on the tensor cores.  CTA (cblk, block column j, side) forms
// block column j of T^{-1} from the inverted 32 x 32 diagonal blocks Z_i:
//   Y_j = Z_j,   Y_i = -Z_i sum_{k = i+1..j} T_ik Y_k   (i = j-1 .. 0)
// on DMMA in FP64, and stores it transposed (row c of the output = column c
// of T^{-1}) in FP32, ready to be split into the BF16 operand image.
// ---------------------------------------------------------------------------
// Dynamic shared memory of k_trinv for blocks of up to maxnzb 32-column blocks:
// the block column of T^{-1} (FP64) and two buffers, each with one block row
// of T and one inverted diagonal block Z_i (FP32).
constexpr int TI_ZLD = 36;  // row stride of Z_i (floats): conflict-free fragment loads
__host__ __device__ inline int ti_ts_ld(int maxnzb) { return 32 * maxnzb + 4; }
__host__ __device__ inline long long trinv_smem_bytes(int maxnzb) {
    return 32LL * maxnzb * DG_LD * 8 + 2 * 32LL * (ti_ts_ld(maxnzb) + TI_ZLD) * 4;
}

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool valid) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    int sz = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}

// T^{-1} of the diagonal block of a cblk, one 32-column block column j per
// CTA, by the backward recurrence Y_j = Z_j, Y_i = -Z_i (T_{i, i+1..j}
// Y_{i+1..j}) over the inverted 32 x 32 diagonal blocks Z_i.  The copies of
// block row i - 1 of T and of Z_{i-1} (cp.async, two buffers) are in flight
// while block row i is computed: the recurrence is latency-bound and the
// loads, not the DMMA, would otherwise set its pace.  Off the diagonal T is a
// plain copy of the factor (T(a, b) = L(b, a); the LU's U(a, b) on the L
// side), scaled by d_a for LDL^T -- a factor of the row, applied to the
// accumulated row of T Y.
template <typename T, int FACT>
__global__ void __launch_bounds__(256, 1) k_trinv(DevStruct s, const int *__restrict__ list, const T *L, const T *U,
                                                   const T *__restrict__ dinv, const int64_t *__restrict__ ti_off,
                                                   float *tinv, int maxnzb) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    static_assert(sizeof(T) == 4, "k_trinv stages FP32 factors");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *Yb = reinterpret_cast<double *>(smem_raw);       // rows 0 .. 32 j + 31 of the block column, ld DG_LD
    const int tld = ti_ts_ld(maxnzb);
    float *Ts = reinterpret_cast<float *>(Yb + 32 * maxnzb * DG_LD);  // 2 x block row i of T, ld tld
    float *Zf = Ts + 2 * 32 * tld;                                     // 2 x Z_i, ld TI_ZLD
    __shared__ double Ss[32 * DG_LD];
    const int k = list[blockIdx.x];
    const int j = blockIdx.y;
    const int side = blockIdx.z;
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int nzb = (nc + 31) / 32;
    if (j >= nzb || ti_off[k] < 0) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
    const T *D = L + s.cb_coef[k];
    const T *gZ = dinv + s.cb_dinv[k] + (size_t)(side ? nzb : 0) * 1024;
    float *out = tinv + ti_off[k] + (size_t)side * nc * nc;
    const int orf = warp >> 1, ocf = 2 * (warp & 1);  // this warp's two 8 x 8 fragments of a 32 x 32 block
    const bool trans = (FACT == FACT_GETRF && side == 0);  // T = U, stored by columns in the L panel
    // issue the copies of block row i of T (columns 32 (i + 1) .. 32 j + 31) and Z_i into buffer b
    auto stage = [&](int i, int b) {
        const int k0 = 32 * (i + 1), K = 32 * (j - i);
        float *ts = Ts + b * 32 * tld;
        if (trans) {
            for (int e = tid; e < 32 * K; e += 256) {
                const int r = e & 31, c = e >> 5, col = k0 + c;
                const bool v = col < nc;
                cp_async4(ts + r * tld + c, v ? D + 32 * i + r + (size_t)col * st : D, v);
            }
        } else {
            for (int e = tid; e < 32 * K; e += 256) {
                const int r = e / K, c = e - r * K, col = k0 + c;
                const bool v = col < nc;
                cp_async4(ts + r * tld + c, v ? D + col + (size_t)(32 * i + r) * st : D, v);
            }
        }
        float *zs = Zf + b * 32 * TI_ZLD;
        for (int e = tid; e < 1024; e += 256) cp_async4(zs + (e >> 5) * TI_ZLD + (e & 31), gZ + (size_t)i * 1024 + e, true);
        cp_async_commit();
    };
    if (j > 0) stage(j - 1, 0);
    // Y_j = Z_j
    for (int e = tid; e < 1024; e += blockDim.x) Yb[(32 * j + (e >> 5)) * DG_LD + (e & 31)] = (double)gZ[(size_t)j * 1024 + e];
    for (int i = j - 1, b = 0; i >= 0; i--, b ^= 1) {
        if (i > 0) {
            stage(i - 1, b ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const float *ts = Ts + b * 32 * tld;
        const float *zs = Zf + b * 32 * TI_ZLD;
        const int k0 = 32 * (i + 1), K = 32 * (j - i);
        // S = T_{i, i+1..j} Y_{i+1..j}, K (a multiple of 32) split over four
        // accumulator chains: with the loads staged ahead, the DMMA latency of
        // one long chain set the pace
        double acc4[4][2][2] = {};
        for (int ks = 0; ks < K / 4; ks += 4) {
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const double a = (double)ts[(8 * orf + g) * tld + 4 * (ks + h) + t4];
#pragma unroll
                for (int c = 0; c < 2; c++)
                    dmma884(acc4[h][c][0], acc4[h][c][1], a, Yb[(k0 + 4 * (ks + h) + t4) * DG_LD + 8 * (ocf + c) + g]);
            }
        }
        double acc[2][2];
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int e = 0; e < 2; e++) acc[c][e] = (acc4[0][c][e] + acc4[1][c][e]) + (acc4[2][c][e] + acc4[3][c][e]);
        double scale = 1.0;
        if (FACT == FACT_SYTRF) {
            const int a = 32 * i + 8 * orf + g;
            scale = (double)D[a + (size_t)a * st];
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
            Ss[(8 * orf + g) * DG_LD + 8 * (ocf + c) + 2 * t4] = scale * acc[c][0];
            Ss[(8 * orf + g) * DG_LD + 8 * (ocf + c) + 2 * t4 + 1] = scale * acc[c][1];
        }
        __syncthreads();
        // Y_i = -Z_i S
        double y[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
        for (int ks = 0; ks < 8; ks++) {
            const double a = -(double)zs[(8 * orf + g) * TI_ZLD + 4 * ks + t4];
#pragma unroll
            for (int c = 0; c < 2; c++) dmma884(y[c][0], y[c][1], a, Ss[(4 * ks + t4) * DG_LD + 8 * (ocf + c) + g]);
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
            Yb[(32 * i + 8 * orf + g) * DG_LD + 8 * (ocf + c) + 2 * t4] = y[c][0];
            Yb[(32 * i + 8 * orf + g) * DG_LD + 8 * (ocf + c) + 2 * t4 + 1] = y[c][1];
        }
        __syncthreads();
    }
    __syncthreads();
    // out[c + kk * nc] = T^{-1}[kk][c] for the block column's columns c and rows kk <= 32 j + 31
    const int ncol = min(32, nc - 32 * j);
    for (int e = tid; e < 32 * (j + 1) * 32; e += blockDim.x) {
        const int kk = e >> 5, c = e & 31;
        if (c < ncol && kk < nc) out[(32 * j + c) + (size_t)kk * nc] = (float)Yb[kk * DG_LD + c];
    }
}

// Split slabs of dense column-major FP32 matrices into their BF16 images.
__global__ void __launch_bounds__(256) k_split_dense(const DenseSlab *__restrict__ slabs, const float *src,
                                                     unsigned char *img) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    const DenseSlab sl = slabs[blockIdx.x];
    const int nkb = split_nkb(sl.cols), ng = split_ng(sl.rows);
    const float *A = src + sl.src;
    unsigned char *out = img + sl.img;
    const int rows = min(128, 8 * ((sl.rows + 7) / 8) - sl.r0);
    const int nch = TC_CH * nkb;
    const int G = gridDim.y, nq = (nch - (int)blockIdx.y + G - 1) / G;  // chunks round robin over the slab's CTAs
    for (int it = threadIdx.x; it < 128 * max(nq, 0); it += blockDim.x) {
        const int r = it & 127, ch = (int)blockIdx.y + (it >> 7) * G;
        if (r >= rows) continue;
        const int pr = sl.r0 + r;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int c = 8 * ch + j;
            v[j] = (pr < sl.rows && c < sl.cols) ? A[pr + (size_t)c * sl.ld] : 0.f;
        }
        uint32_t w[3][4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            uint32_t a0, a1, a2, b0, b1, b2;
            split_bf16x3(v[2 * j], a0, a1, a2);
            split_bf16x3(v[2 * j + 1], b0, b1, b2);
            w[0][j] = a0 | (b0 << 16);
            w[1][j] = a1 | (b1 << 16);
            w[2][j] = a2 | (b2 << 16);
        }
        const size_t base = (size_t)(ch / TC_CH) * ng * TC_GROUP + (size_t)(pr >> 3) * TC_GROUP +
                            (ch % TC_CH) * 128 + (pr & 7) * 16;
#pragma unroll
        for (int p = 0; p < 3; p++)
            *reinterpret_cast<uint4 *>(out + base + (size_t)p * nkb * ng * TC_GROUP) =
                make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
    }
}

// FP32 off-diagonal TRSM as the GEMM X = A T^{-1} on tcgen05 (k_trsm_tcp
// below): A from the BF16 image of the panel taken before the TRSM, T^{-1}
// from the image of its transpose (k_trinv, k_split_dense); the 128 x 128 tile
// of X overwrites the panel rows below the diagonal block.  Tile: cblk, mt
// (128-row window from the first off-diagonal row group), nt (128 columns),
// side (GETRF U panel).

// ---------------------------------------------------------------------------
// Persistent, warp-specialized form of the tcgen05 tile loop.  A CTA walks the
// tiles blockIdx.x, blockIdx.x + gridDim.x, ...: warp 4 (one thread) issues the
// bulk copies of every K block through TP_STAGES shared-memory stages, warp 5
// (one thread) issues the MMAs into one of two 128-column accumulators in
// tensor memory, and warps 0-3 drain the other accumulator (tcgen05.ld, one
// tile row per thread) while the next tile is multiplied.  Hand-offs:
// full/empty mbarriers per stage (bulk-copy bytes / tcgen05.commit), tfull per
// accumulator (tcgen05.commit), tempty per accumulator (128 epilogue arrivals).
// Two CTAs per SM hold all 512 tensor-memory columns.  Every wait is bounded;
// a role that gives up makes the others give up too and the kernel records
// PGPU_STATUS_TIMEOUT.
//   setup(t, op)            operands of tile t
//   rowinfo(t, op, row)     per-row value kept in a register by the epilogue thread
//   colinfo(t, op, col)     per-column value shared through shared memory
//   epi(t, op, rinfo, ct, row, c0, v)  accumulator columns c0 .. c0 + 15 of a row
// ---------------------------------------------------------------------------
constexpr int TP_STAGES = 2;
constexpr size_t TP_SMEM = (size_t)TP_STAGES * TC_STAGE;
constexpr int TP_THREADS = 192;

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// OR of `pred` over the 128 epilogue threads (named barrier 1, which also orders them)
__device__ __forceinline__ int epi_bar_or(int pred) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\tbarrier.red.or.pred q, 1, 128, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"(pred)
        : "memory");
    return r;
}

constexpr int TQ = 4;  // tile-index ring between the producer and the other roles

// The persistent tile engine.  Tiles come from a device work queue: the
// producer claims the next tile index with an atomic on *queue (zeroed before
// the launch) and hands it to the MMA issuer and the epilogue warps through a
// ring of TQ slots guarded by mbarriers; an index past `count` ends every
// role.  CTAs that draw cheap tiles simply draw more, so uneven tile costs
// (source widths, masked rows) do not leave SMs idle at the end of a launch.
template <typename Setup, typename RowInfo, typename ColInfo, typename Epi>
__device__ __forceinline__ void tc_persistent(int count, int *queue, int *status, Setup setup, RowInfo rowinfo,
                                              ColInfo colinfo, Epi epi) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[TP_STAGES], empty[TP_STAGES], tfull[2], tempty[2], tq_full[TQ], tq_empty[TQ];
    __shared__ uint32_t tmem_sh;
    __shared__ int ctab[2][TC_BN];
    __shared__ int tq[TQ];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                     "r"(2 * TC_BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int i = 0; i < TP_STAGES; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(&tfull[i], 1);
            mbar_init(&tempty[i], 4 * 32);
        }
        for (int i = 0; i < TQ; i++) {
            mbar_init(&tq_full[i], 1);
            mbar_init(&tq_empty[i], 1 + 4 * 32);  // the MMA issuer and the 128 epilogue threads
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_sh;
    int late = 0;
    if (warp == 4) {
        if (lane == 0) {  // producer: claims tiles, loads their operands
            uint32_t g = 0;
            // the claim of the next tile is issued one tile ahead, so that its
            // round trip to L2 overlaps this tile's copies
            int next = atomicAdd(queue, 1);
            for (int j = 0; !late; j++) {
                const int slot = j % TQ;
                if (j >= TQ && !mbar_wait(&tq_empty[slot], ((j / TQ) - 1) & 1)) {
                    late = 1;
                    break;
                }
                int t = next;
                if (t >= count) t = -1;
                else next = atomicAdd(queue, 1);
                tq[slot] = t;
                mbar_arrive(&tq_full[slot]);
                if (t < 0) break;
                TcOperands op;
                setup(t, op);
                const uint32_t bbytes = (uint32_t)(op.nmma / 8) * TC_GROUP;
                for (int kb = 0; kb < op.nkb; kb++, g++) {
                    const int sidx = g % TP_STAGES;
                    if (g >= TP_STAGES && !mbar_wait(&empty[sidx], ((g / TP_STAGES) - 1) & 1)) {
                        late = 1;
                        break;
                    }
                    unsigned char *sp = smem_raw + (size_t)sidx * TC_STAGE;
                    mbar_expect_tx(&full[sidx], 3u * TC_PIECE + 3u * bbytes);
#pragma unroll
                    for (int p = 0; p < 3; p++) {
                        bulk_g2s(sp + p * TC_PIECE, op.iA + p * op.termA + ((size_t)kb * op.ngA + op.ga) * TC_GROUP,
                                 TC_PIECE, &full[sidx]);
                        bulk_g2s(sp + (3 + p) * TC_PIECE,
                                 op.iB + p * op.termB + ((size_t)kb * op.ngB + op.gb) * TC_GROUP, bbytes, &full[sidx]);
                    }
                }
            }
        }
    } else if (warp == 5) {
        if (lane == 0) {  // MMA issuer
            const uint32_t sbase = smem_u32(smem_raw);
            uint32_t g = 0;
            for (int i = 0; !late; i++) {
                const int slot = i % TQ;
                if (!mbar_wait(&tq_full[slot], (i / TQ) & 1)) {
                    late = 1;
                    break;
                }
                const int t = tq[slot];
                mbar_arrive(&tq_empty[slot]);
                if (t < 0) break;
                TcOperands op;
                setup(t, op);
                const int b = i & 1;
                if (i >= 2 && !mbar_wait(&tempty[b], ((i >> 1) - 1) & 1)) {
                    late = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t idesc = tc_idesc(op.nmma);
                const uint32_t acc = tmem + (uint32_t)(TC_BN * b);
                for (int kb = 0; kb < op.nkb; kb++, g++) {
                    const int sidx = g % TP_STAGES;
                    if (!mbar_wait(&full[sidx], (g / TP_STAGES) & 1)) {
                        late = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st0 = sbase + sidx * TC_STAGE;
#pragma unroll
                    for (int ks = 0; ks < TC_BK / 16; ks++) {
#pragma unroll
                        for (int p = 0; p < 6; p++) {
                            const int pa = (p == 2 || p == 4) ? 1 : (p == 5 ? 2 : 0);
                            const int pb = (p == 1 || p == 4) ? 1 : (p == 3 ? 2 : 0);
                            tc_mma(acc, tc_desc(st0 + pa * TC_PIECE + ks * 256),
                                   tc_desc(st0 + (3 + pb) * TC_PIECE + ks * 256), idesc, (kb | ks | p) != 0);
                        }
                    }
                    tc_commit(&empty[sidx]);
                }
                if (late) break;
                tc_commit(&tfull[b]);
            }
        }
    } else {  // epilogue warps 0-3: tile row = tid, tensor-memory lanes 32 warp .. 32 warp + 31
        for (int i = 0;; i++) {
            const int slot = i % TQ;
            const int qfail = epi_bar_or(!mbar_wait(&tq_full[slot], (i / TQ) & 1));
            if (qfail) {
                late = 1;
                break;
            }
            const int t = tq[slot];
            mbar_arrive(&tq_empty[slot]);
            if (t < 0) break;
            TcOperands op;
            setup(t, op);
            const int b = i & 1;
            const int rinfo = rowinfo(t, op, tid);
            ctab[b][tid] = colinfo(t, op, tid);
            const int fail = epi_bar_or(!mbar_wait(&tfull[b], (i >> 1) & 1));
            if (fail) {
                late = 1;
                break;
            }
            tc_fence_after();
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(TC_BN * b);
#pragma unroll 1
            for (int c0 = 0; c0 < op.nmma; c0 += 16) {
                float v[16];
                tmem_ld16(taddr + c0, v);
                epi(t, op, rinfo, ctab[b], tid, c0, v);
            }
            tc_fence_before();
            mbar_arrive(&tempty[b]);
        }
    }
    __syncwarp();
    const int aborted = __syncthreads_or(late);
    if (aborted && tid == 0) atomicExch(status, PGPU_STATUS_TIMEOUT);
    tc_fence_after();
    if (warp == 5) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC_BN));
}

template <int FACT>
__global__ void __launch_bounds__(TP_THREADS, 2) k_update_tcp(DevStruct s, const UpdTile *__restrict__ tiles,
                                                               int count, float *L, float *U,
                                                               const unsigned char *img0, const unsigned char *img1,
                                                               const int64_t *__restrict__ sp_off, int *queue,
                                                               int *status) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    if (*(volatile int *)status != 0) return;
    auto setup = [&](int t, TcOperands &op) {
        const UpdTile tl = tiles[t];
        const TaskDev tk = s.tasks[tl.task];
        const int k = tk.src;
        const int K = s.cb_lcol[k] - s.cb_fcol[k] + 1;
        const int st = s.cb_stride[k];
        const int ra = tk.row0 + (tl.side ? tk.n : 0);
        const int rbe = tk.row0 + tk.n;
        const bool swap = (FACT == FACT_GETRF && tl.side == 1);
        op.nkb = split_nkb(K);
        op.ngA = op.ngB = split_ng(st);
        op.termA = op.termB = (size_t)op.nkb * op.ngA * TC_GROUP;
        op.ga = (ra >> 3) + 16 * tl.mt;
        op.gb = (tk.row0 >> 3) + 16 * tl.nt;
        op.nmma = (min(TC_BN, rbe - 8 * op.gb) + 15) & ~15;
        op.iA = (swap ? img1 : img0) + sp_off[k];
        op.iB = ((FACT == FACT_POTRF) ? img0 : (swap ? img0 : img1)) + sp_off[k];
    };
    auto rowinfo = [&](int t, const TcOperands &op, int row) {  // offset of the target row in the facing panel
        const UpdTile tl = tiles[t];
        const TaskDev tk = s.tasks[tl.task];
        const int k = tk.src, f = tk.dst;
        const int ra = tk.row0 + (tl.side ? tk.n : 0), rend = tk.row0 + tk.m;
        const int pr = 8 * op.ga + row;
        if (pr < ra || pr >= rend) return -1;
        const int g = s.rowidx[s.cb_rowidx[k] + pr];
        int lo = s.cb_fblok[f], hi = s.cb_fblok[f + 1] - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s.bk_frow[mid] <= g) lo = mid;
            else hi = mid - 1;
        }
        return s.bk_rowoff[lo] + (g - s.bk_frow[lo]);
    };
    auto colinfo = [&](int t, const TcOperands &op, int col) {  // target column in the facing panel
        const UpdTile tl = tiles[t];
        const TaskDev tk = s.tasks[tl.task];
        const int pc = 8 * op.gb + col;
        if (pc < tk.row0 || pc >= tk.row0 + tk.n) return -1;
        return s.rowidx[s.cb_rowidx[tk.src] + pc] - s.cb_fcol[tk.dst];
    };
    auto epi = [&](int t, const TcOperands &op, int rr, const int *ct, int row, int c0, const float *v) {
        if (rr < 0) return;
        const UpdTile tl = tiles[t];
        const TaskDev tk = s.tasks[tl.task];
        const bool swap = (FACT == FACT_GETRF && tl.side == 1);
        float *Cp = (swap ? U : L) + s.cb_coef[tk.dst] + rr;
        const int stf = s.cb_stride[tk.dst];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int cc = ct[c0 + j];
            if (cc >= 0) atomicAdd(Cp + (size_t)cc * stf, -v[j]);  // reduction without return
        }
    };
    tc_persistent(count, queue, status, setup, rowinfo, colinfo, epi);
}

template <int FACT>
__global__ void __launch_bounds__(TP_THREADS, 2) k_trsm_tcp(DevStruct s, const UpdTile *__restrict__ tiles, int count,
                                                             float *L, float *U, const unsigned char *img0,
                                                             const unsigned char *img1,
                                                             const int64_t *__restrict__ sp_off,
                                                             const unsigned char *timg,
                                                             const int64_t *__restrict__ ti_img, int *queue,
                                                             int *status) {
    pdl_wait();  // the kernel ahead in the stream has ended (programmatic dependent launch)
    if (*(volatile int *)status != 0) return;
    auto setup = [&](int t, TcOperands &op) {
        const UpdTile tl = tiles[t];
        const int k = tl.task;
        const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
        const int st = s.cb_stride[k];
        const bool uside = (FACT == FACT_GETRF && tl.side == 1);
        op.nkb = split_nkb(nc);
        op.ngA = split_ng(st);
        op.ngB = split_ng(nc);
        op.termA = (size_t)op.nkb * op.ngA * TC_GROUP;
        op.termB = (size_t)op.nkb * op.ngB * TC_GROUP;
        op.ga = (nc >> 3) + 16 * tl.mt;
        op.gb = 16 * tl.nt;
        op.nmma = (min(TC_BN, nc - 128 * tl.nt) + 15) & ~15;
        op.iA = (uside ? img1 : img0) + sp_off[k];
        op.iB = timg + ti_img[k] + (uside ? (size_t)3 * op.termB : 0);
    };
    auto rowinfo = [&](int t, const TcOperands &op, int row) {  // panel row, -1 outside the rows below
        const int k = tiles[t].task;
        const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
        const int pr = 8 * op.ga + row;
        return (pr >= nc && pr < s.cb_stride[k]) ? pr : -1;
    };
    auto colinfo = [&](int t, const TcOperands &op, int col) {
        const int k = tiles[t].task;
        const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
        const int c = 128 * tiles[t].nt + col;
        return (c < nc) ? c : -1;
    };
    auto epi = [&](int t, const TcOperands &op, int pr, const int *ct, int row, int c0, const float *v) {
        if (pr < 0) return;
        const UpdTile tl = tiles[t];
        const int k = tl.task;
        const int st = s.cb_stride[k];
        float *P = ((FACT == FACT_GETRF && tl.side == 1) ? U : L) + s.cb_coef[k] + pr;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int c = ct[c0 + j];
            if (c >= 0) P[(size_t)c * st] = v[j];
        }
    };
    tc_persistent(count, queue, status, setup, rowinfo, colinfo, epi);
}

// ---------------------------------------------------------------------------
// Host launch wrappers (called from the driver with level lists in device memory)
// ---------------------------------------------------------------------------
static int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            n = 1;
    }
    return n;
}
template <typename T>
void launch_fill_coef(int64_t nnz, const double *vals, const int64_t *lmap, const int64_t *umap, T *L, T *U,
                      cudaStream_t st) {
    if (nnz <= 0) return;
    int blocks = (int)std::min<int64_t>((nnz + 255) / 256, 148 * 16);
    k_fill_coef<T><<<blocks, 256, 0, st>>>(nnz, vals, lmap, umap, L, U);
}

static thread_local bool t_pdl = false;
void set_pdl(bool on) { t_pdl = on; }
bool pdl_enabled() { return t_pdl; }

template <typename T, int FACT>
void launch_panel_small(const DevStruct &s, const int *list, int count, size_t smem, T *L, T *U,
                        const FactParams &fp, cudaStream_t st) {
    if (count <= 0) return;
    launch_k(k_panel_small<T, FACT>, count, 128, smem, st, s, list, L, U, fp);
}

template <typename T, int FACT>
void launch_diag_large(const DevStruct &s, const int *list, int count, int maxnc, size_t smem, T *L, T *U, T *dinv,
                       const FactParams &fp, cudaStream_t st) {
    if (count <= 0) return;
    static int nsm = 0;
    if (nsm == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            nsm = 1;
    }
    const long long csm = diag_cluster_smem_bytes(maxnc, FACT);
    if (maxnc <= DG_MAXNC && maxnc >= DC_MIN_NC && (long long)count * DC <= nsm && count <= DC_MAX_CLUSTERS &&
        csm <= dc_max_smem(FACT))
        launch_k(k_diag_cluster<T, FACT>, count * DC, 256, (size_t)csm, st, s, list, L, U, dinv, fp);
    else if (maxnc <= DG_MAXNC)
        launch_k(k_diag_dmma<T, FACT>, count, 256, (size_t)diag_dmma_smem_bytes(maxnc), st, s, list, L, U, dinv, fp);
    else
        launch_k(k_diag_large<T, FACT>, count, 256, smem, st, s, list, L, U, dinv, fp);
}

template <typename T, int FACT>
void launch_trsm(const DevStruct &s, const RowTile *tiles, int count, int maxnc, size_t smem, T *L, T *U,
                 const T *dinv, cudaStream_t st) {
    if (count <= 0) return;
    dim3 grid(count, FACT == FACT_GETRF ? 2 : 1);
    if (maxnc <= TD_MAXNC)
        k_trsm_dmma<T, FACT><<<grid, 256, 0, st>>>(s, tiles, L, U, dinv);
    else
        launch_k(k_trsm<T, FACT>, grid, 256, smem, st, s, tiles, L, U, dinv);
}

template <typename T, int FACT>
void launch_update(const DevStruct &s, const UpdTile *tiles, int count, T *L, T *U, cudaStream_t st) {
    if (count <= 0) return;
    launch_k(k_update<T, FACT, 64, 64, 16, 4, 4>, count, 256, 0, st, s, tiles, L, U);
}

// big tiles (128 x 64): DMMA for FP64, SIMT 8 x 4 per thread for FP32
template <typename T, int FACT>
void launch_update_big(const DevStruct &s, const UpdTile *tiles, int count, T *L, T *U, cudaStream_t st) {
    if (count <= 0) return;
    if constexpr (sizeof(T) == 8)
        k_update_dmma<FACT><<<count, 256, DM_SMEM, st>>>(s, tiles, L, U);
    else
        k_update<T, FACT, 128, 64, 16, 8, 4><<<count, 256, 0, st>>>(s, tiles, L, U);
}

// FP32 updates of 128 x 128 tiles on tcgen05 from the split BF16 images
template <int FACT>
void launch_update_tc(const DevStruct &s, const UpdTile *tiles, int count, float *L, float *U,
                      const unsigned char *img0, const unsigned char *img1, const int64_t *sp_off, int *queue,
                      int *status, cudaStream_t st) {
    if (count <= 0) return;
    const int grid = std::min(count, 2 * sm_count());
    launch_k(k_update_tcp<FACT>, grid, TP_THREADS, TP_SMEM, st, s, tiles, count, L, U, img0, img1, sp_off, queue, status);
}

template <int FACT>
void launch_trinv(const DevStruct &s, const int *list, int count, int maxnzb, const float *L, const float *U,
                  const float *dinv, const int64_t *ti_off, float *tinv, cudaStream_t st) {
    if (count <= 0 || maxnzb <= 0) return;
    dim3 grid(count, maxnzb, FACT == FACT_GETRF ? 2 : 1);
    launch_k(k_trinv<float, FACT>, grid, 256, (size_t)trinv_smem_bytes(maxnzb), st, s, list, L, U, dinv, ti_off, tinv,
             maxnzb);
}

void launch_split_dense(const DenseSlab *slabs, int count, const float *src, unsigned char *img, cudaStream_t st) {
    if (count <= 0) return;
    launch_k(k_split_dense, dim3(count, SPLIT_CTAS), 256, 0, st, slabs, src, img);
}

template <int FACT>
void launch_trsm_tc(const DevStruct &s, const UpdTile *tiles, int count, float *L, float *U,
                    const unsigned char *img0, const unsigned char *img1, const int64_t *sp_off,
                    const unsigned char *timg, const int64_t *ti_img, int *queue, int *status, cudaStream_t st) {
    if (count <= 0) return;
    const int grid = std::min(count, 2 * sm_count());
    launch_k(k_trsm_tcp<FACT>, grid, TP_THREADS, TP_SMEM, st, s, tiles, count, L, U, img0, img1, sp_off, timg, ti_img,
             queue, status);
}

void launch_split(const DevStruct &s, const SplitSlab *slabs, int count, const float *P, const float *D,
                  const int64_t *sp_off, unsigned char *img, int scale, cudaStream_t st) {
    if (count <= 0) return;
    launch_k(k_split, dim3(count, SPLIT_CTAS), 256, 0, st, s, slabs, P, D, sp_off, img, scale);
}

long long split_image_bytes(int nc, int st) { return split_bytes(nc, st); }
long long panel_small_bytes(long long panel_elems, int tsize, int maxst) {
    return panel_small_smem_bytes(panel_elems, tsize, maxst);
}
int trinv_max_blocks() { return DG_MAXNC / 32; }

// Self-test of the bounded waits, on a two-CTA cluster: CTA 1 waits, as
// k_diag_cluster does, on a flag of CTA 0 that nothing raises, while CTA 0
// waits, as the tcgen05 engine does, on an mbarrier phase that nothing
// completes.  Both waits give up; timed_out[r] counts CTA r's, and the kernel
// ends with the context usable.
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(32) k_wait_selftest(int *timed_out) {
    namespace cg = cooperative_groups;
    __shared__ int flag;
    __shared__ __align__(8) uint64_t bar;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    if (threadIdx.x == 0) {
        flag = 0;
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    cluster.sync();
    if (threadIdx.x == 0) {
        const bool ok = (rank == 1) ? dc_wait(dsmem_map(&flag, 0), 1) : mbar_wait(&bar, 0);
        if (!ok) atomicAdd(timed_out + rank, 1);
    }
    cluster.sync();  // CTA 0's shared memory outlives CTA 1's reads
}
cudaError_t wait_selftest(int *timed_out_host) {
    int *d = nullptr;
    cudaError_t e = cudaMalloc(&d, 2 * sizeof(int));
    if (e != cudaSuccess) return e;
    if ((e = cudaMemset(d, 0, 2 * sizeof(int))) == cudaSuccess) {
        k_wait_selftest<<<2, 32>>>(d);
        if ((e = cudaGetLastError()) == cudaSuccess && (e = cudaDeviceSynchronize()) == cudaSuccess)
            e = cudaMemcpy(timed_out_host, d, 2 * sizeof(int), cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    return e;
}
size_t diag_cluster_scratch_doubles() { return DC_MAX_CLUSTERS * DC_SCR_DOUBLES; }

// Opt every kernel with dynamic shared memory into the largest size the
// device allows next to its static shared memory.
template <typename K>
static cudaError_t opt_in_smem(K kernel) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

template <typename T, int FACT>
cudaError_t set_smem_attrs(size_t, size_t, size_t) {
    cudaError_t e;
    if ((e = opt_in_smem(k_panel_small<T, FACT>)) != cudaSuccess) return e;
    if ((e = opt_in_smem(k_diag_large<T, FACT>)) != cudaSuccess) return e;
    if ((e = opt_in_smem(k_trsm<T, FACT>)) != cudaSuccess) return e;
    if ((e = opt_in_smem(k_diag_dmma<T, FACT>)) != cudaSuccess) return e;
    if ((e = opt_in_smem(k_diag_cluster<T, FACT>)) != cudaSuccess) return e;
    if constexpr (sizeof(T) == 8) {
        if ((e = opt_in_smem(k_update_dmma<FACT>)) != cudaSuccess) return e;
    } else {
        if ((e = opt_in_smem(k_update_tcp<FACT>)) != cudaSuccess) return e;
        if ((e = opt_in_smem(k_trsm_tcp<FACT>)) != cudaSuccess) return e;
        if ((e = opt_in_smem(k_trinv<float, FACT>)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

#define PGPU_INST_FACT(T, F)                                                                                     \
    template void launch_panel_small<T, F>(const DevStruct &, const int *, int, size_t, T *, T *,                \
                                           const FactParams &, cudaStream_t);                                    \
    template void launch_diag_large<T, F>(const DevStruct &, const int *, int, int, size_t, T *, T *, T *,       \
                                          const FactParams &, cudaStream_t);                                     \
    template void launch_trsm<T, F>(const DevStruct &, const RowTile *, int, int, size_t, T *, T *, const T *,   \
                                    cudaStream_t);                                                               \
    template void launch_update<T, F>(const DevStruct &, const UpdTile *, int, T *, T *, cudaStream_t);          \
    template void launch_update_big<T, F>(const DevStruct &, const UpdTile *, int, T *, T *, cudaStream_t);      \
    template cudaError_t set_smem_attrs<T, F>(size_t, size_t, size_t);

PGPU_INST_FACT(double, FACT_POTRF)
PGPU_INST_FACT(double, FACT_SYTRF)
PGPU_INST_FACT(double, FACT_GETRF)
PGPU_INST_FACT(float, FACT_POTRF)
PGPU_INST_FACT(float, FACT_SYTRF)
PGPU_INST_FACT(float, FACT_GETRF)
template void launch_trinv<FACT_POTRF>(const DevStruct &, const int *, int, int, const float *, const float *,
                                      const float *, const int64_t *, float *, cudaStream_t);
template void launch_trsm_tc<FACT_POTRF>(const DevStruct &, const UpdTile *, int, float *, float *, const unsigned char *,
                                        const unsigned char *, const int64_t *, const unsigned char *,
                                        const int64_t *, int *, int *, cudaStream_t);
template void launch_update_tc<FACT_POTRF>(const DevStruct &, const UpdTile *, int, float *, float *,
                                           const unsigned char *, const unsigned char *, const int64_t *, int *,
                                           int *, cudaStream_t);
template void launch_trinv<FACT_SYTRF>(const DevStruct &, const int *, int, int, const float *, const float *,
                                      const float *, const int64_t *, float *, cudaStream_t);
template void launch_trsm_tc<FACT_SYTRF>(const DevStruct &, const UpdTile *, int, float *, float *, const unsigned char *,
                                        const unsigned char *, const int64_t *, const unsigned char *,
                                        const int64_t *, int *, int *, cudaStream_t);
template void launch_update_tc<FACT_SYTRF>(const DevStruct &, const UpdTile *, int, float *, float *,
                                           const unsigned char *, const unsigned char *, const int64_t *, int *,
                                           int *, cudaStream_t);
template void launch_trinv<FACT_GETRF>(const DevStruct &, const int *, int, int, const float *, const float *,
                                      const float *, const int64_t *, float *, cudaStream_t);
template void launch_trsm_tc<FACT_GETRF>(const DevStruct &, const UpdTile *, int, float *, float *, const unsigned char *,
                                        const unsigned char *, const int64_t *, const unsigned char *,
                                        const int64_t *, int *, int *, cudaStream_t);
template void launch_update_tc<FACT_GETRF>(const DevStruct &, const UpdTile *, int, float *, float *,
                                           const unsigned char *, const unsigned char *, const int64_t *, int *,
                                           int *, cudaStream_t);
template void launch_fill_coef<double>(int64_t, const double *, const int64_t *, const int64_t *, double *,
                                       double *, cudaStream_t);
template void launch_fill_coef<float>(int64_t, const double *, const int64_t *, const int64_t *, float *,
                                      float *, cudaStream_t);

}  // namespace pgpu
