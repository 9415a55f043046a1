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
template <typename T, int FACT>
__global__ void __launch_bounds__(256) k_panel_small(DevStruct s, const int *__restrict__ list, T *L, T *U,
                                                      FactParams fp) {
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
    for (int i = tid; i < tot; i += nt) P[i] = gL[i];
    if (FACT == FACT_GETRF)
        for (int i = tid; i < tot; i += nt) Q[i] = gU[i];
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
            P[c + c * st] = static_pivot<T, FACT>(P[c + c * st], fp.criterion, np);
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
}

// ---------------------------------------------------------------------------
// Wide cblks, diagonal block: blocked right-looking factorization by column
// panels of DNB = 32 columns held row-major in shared memory.  Per panel:
//   1. warp 0 factors the 32 x 32 top block column by column (pivot, scale,
//      rank-1 update), as potf2 / getf2 / sytf2;
//   2. the panel rows below are solved against that block, one warp per row,
//      block columns on the lanes (the TRSM of the blocked algorithm);
//   3. the trailing part of the diagonal block is updated from shared memory
//      with 4 x 4 register tiles (SYRK / GEMM of the blocked algorithm).
// GETRF keeps the 32-row strip of U to the right of the panel in shared
// memory as well (its rows are solved with the unit lower factor).
// ---------------------------------------------------------------------------
constexpr int DNB = 32;
constexpr int DLDW = DNB + 1;

template <typename T, int FACT>
__global__ void __launch_bounds__(256) k_diag_large(DevStruct s, const int *__restrict__ list, T *L, T *U,
                                                     FactParams fp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int k = list[blockIdx.x];
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    T *W = reinterpret_cast<T *>(smem_raw);  // m x DNB panel, row major, ld DLDW
    T *R = W + (size_t)nc * DLDW;            // GETRF: DNB x t strip of U, row major, ld nc + 1
    const int ldr = nc + 1;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    T *A = L + s.cb_coef[k];
    __shared__ int npiv;
    __shared__ T dsh[DNB];
    if (tid == 0) npiv = 0;
    if (FACT == FACT_GETRF) {  // L_kk += (U^T)_kk^T : the full diagonal block
        const T *Ut = U + s.cb_coef[k];
        for (int e = tid; e < nc * nc; e += nt) {
            int i = e % nc, j = e / nc;
            A[i + (size_t)j * st] += Ut[j + (size_t)i * st];
        }
    }
    __syncthreads();
    for (int jb = 0; jb < nc; jb += DNB) {
        const int nb = min(DNB, nc - jb);
        const int m = nc - jb;       // panel rows
        const int t = m - nb;        // trailing size
        for (int e = tid; e < m * nb; e += nt) {
            int i = e % m, c = e / m;
            W[i * DLDW + c] = A[(jb + i) + (size_t)(jb + c) * st];
        }
        if (FACT == FACT_GETRF)
            for (int e = tid; e < nb * t; e += nt) {
                int c = e % nb, q = e / nb;
                R[c * ldr + q] = A[(jb + c) + (size_t)(jb + nb + q) * st];
            }
        __syncthreads();
        // 1. the nb x nb top block, by warp 0
        if (warp == 0) {
            int np = 0;
            for (int c = 0; c < nb; c++) {
                T d = static_pivot<T, FACT>(W[c * DLDW + c], fp.criterion, np);
                __syncwarp();
                if (lane == c) W[c * DLDW + c] = d;
                const T inv = T(1) / d;
                if (lane > c && lane < nb) {
                    if (FACT == FACT_SYTRF) W[c * DLDW + lane] = W[lane * DLDW + c];  // D L^T copy
                    W[lane * DLDW + c] *= inv;
                }
                __syncwarp();
                if (lane > c && lane < nb) {
                    const T lic = W[lane * DLDW + c];
                    for (int j = c + 1; j < nb; j++) {
                        if (FACT == FACT_POTRF) {
                            if (lane >= j) W[lane * DLDW + j] -= lic * W[j * DLDW + c];
                        } else if (FACT == FACT_SYTRF) {
                            if (lane >= j) W[lane * DLDW + j] -= lic * W[c * DLDW + j];
                        } else {
                            W[lane * DLDW + j] -= lic * W[c * DLDW + j];
                        }
                    }
                }
                __syncwarp();
            }
            if (lane == 0 && np) npiv += np;
        }
        __syncthreads();
        if (FACT == FACT_SYTRF && tid < nb) dsh[tid] = W[tid * DLDW + tid];
        // 2. panel rows below the block: x T = a, lanes = block columns
        for (int r = nb + warp; r < m; r += nt / 32) {
            T x = (lane < nb) ? W[r * DLDW + lane] : T(0);
            for (int c = 0; c < nb; c++) {
                if (lane == c) x /= W[c * DLDW + c];
                T xc = __shfl_sync(0xffffffffu, x, c);
                if (lane > c && lane < nb) {
                    T tcl = (FACT == FACT_POTRF) ? W[lane * DLDW + c] : W[c * DLDW + lane];
                    x -= xc * tcl;
                }
            }
            if (lane < nb) W[r * DLDW + lane] = x;
        }
        if (FACT == FACT_GETRF)  // U12 <- L11^{-1} U12 (unit lower), one column per thread
            for (int q = tid; q < t; q += nt)
                for (int c = 0; c < nb; c++) {
                    const T u = R[c * ldr + q];
                    for (int j = c + 1; j < nb; j++) R[j * ldr + q] -= W[j * DLDW + c] * u;
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
        // 3. trailing update A22 -= L21 * B^T (4x4 blocks; lower triangle for the symmetric kinds)
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
        for (int e = tid; e < nc * nc; e += nt) {
            int i = e % nc, j = e / nc;
            if (i < j) A[i + (size_t)j * st] = A[i + (size_t)i * st] * A[j + (size_t)i * st];
        }
    }
    if (FACT == FACT_GETRF) {  // (U^T)_kk = (L\U)_kk^T
        __syncthreads();
        T *Ut = U + s.cb_coef[k];
        for (int e = tid; e < nc * nc; e += nt) {
            int i = e % nc, j = e / nc;
            Ut[j + (size_t)i * st] = A[i + (size_t)j * st];
        }
    }
    if (tid == 0 && npiv) atomicAdd(fp.nbpivots, npiv);
}

// ---------------------------------------------------------------------------
// Wide cblks, off-diagonal TRSM: X T = A for a tile of TRSM_ROWS panel rows,
// T the upper triangular factor of the diagonal block:
//   POTRF       T = L_kk^T            (Right, Lower, Trans, NonUnit)
//   SYTRF       T = D_kk L_kk^T        (Right, Upper, NoTrans, NonUnit on DL^T)
//   GETRF side0 T = U_kk  (upper of L) (Right, Upper, NoTrans, NonUnit)
//   GETRF side1 T = L_kk^T (unit)      (Right, Upper, NoTrans, Unit on U panel)
// blockIdx.y selects the GETRF side.  Blocked by 32 columns (the blocked
// algorithm of a BLAS TRSM): a 32-wide block is solved by substitution, one
// warp per 4 rows with the block's columns on the lanes, then the columns to
// its right are updated by a register-tiled GEMM from shared memory.  The tile
// of X (row major) and the current 32-row strip of T live in shared memory.
// ---------------------------------------------------------------------------
constexpr int TRSM_ROWS = 32;
constexpr int TRSM_MAXT = 10;  // column chunks of 32 per GEMM pass

template <typename T, int FACT>
__global__ void __launch_bounds__(256) k_trsm(DevStruct s, const RowTile *__restrict__ tiles, T *L, T *U) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const RowTile tl = tiles[blockIdx.x];
    const int side = blockIdx.y;
    const int k = tl.cblk;
    const int nc = s.cb_lcol[k] - s.cb_fcol[k] + 1;
    const int st = s.cb_stride[k];
    const int rows = min(TRSM_ROWS, st - tl.r0);
    const int ld = nc + 1;
    T *X = reinterpret_cast<T *>(smem_raw);  // TRSM_ROWS x nc, row major, ld
    T *Ts = X + TRSM_ROWS * ld;              // 32 x (nc - jb) strip of T, row major, ld
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const T *D = L + s.cb_coef[k];  // diagonal block (ld = st) of the L panel
    T *A = ((FACT == FACT_GETRF && side == 1) ? U : L) + s.cb_coef[k] + tl.r0;
    const bool unit = (FACT == FACT_GETRF && side == 1);
    for (int e = tid; e < TRSM_ROWS * nc; e += blockDim.x) {
        int i = e % TRSM_ROWS, j = e / TRSM_ROWS;
        X[i * ld + j] = (i < rows) ? A[i + (size_t)j * st] : T(0);
    }
    for (int jb = 0; jb < nc; jb += 32) {
        const int nb = min(32, nc - jb);
        const int wdt = nc - jb;
        __syncthreads();
        for (int e = tid; e < nb * wdt; e += blockDim.x) {  // Ts[a][q] = T(jb + a, jb + q)
            int q = e % wdt, a = e / wdt;
            int ga = jb + a, gb = jb + q;
            T t;
            if (gb < ga) t = T(0);
            else if (FACT == FACT_POTRF) t = D[gb + (size_t)ga * st];
            else if (FACT == FACT_SYTRF) t = (gb == ga) ? D[ga + (size_t)ga * st]
                                                          : D[ga + (size_t)ga * st] * D[gb + (size_t)ga * st];
            else if (side == 0) t = D[ga + (size_t)gb * st];
            else t = D[gb + (size_t)ga * st];
            Ts[a * ld + q] = t;
        }
        __syncthreads();
        // substitution on the 32-wide block: warp w owns rows 4w .. 4w+3
#pragma unroll
        for (int rr = 0; rr < 4; rr++) {
            const int r = warp * 4 + rr;
            T x = (lane < nb) ? X[r * ld + jb + lane] : T(0);
            for (int c = 0; c < nb; c++) {
                if (!unit && lane == c) x /= Ts[c * ld + c];
                T xc = __shfl_sync(0xffffffffu, x, c);
                if (lane > c && lane < nb) x -= xc * Ts[c * ld + lane];
            }
            if (lane < nb) X[r * ld + jb + lane] = x;
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
        for (int e = tid; e < BK * BM; e += NT) {
            int kk = e / BM, r = e % BM;
            T v = T(0);
            if (r < mrows && k0 + kk < K) v = Ap[(arow + r) + (size_t)(k0 + kk) * st];
            As[kk][r] = v;
        }
        for (int e = tid; e < BK * BN; e += NT) {
            int kk = e / BN, c = e % BN;
            T v = T(0);
            if (c < ncols && k0 + kk < K) v = Bp[(brow + c) + (size_t)(k0 + kk) * st];
            Bs[kk][c] = v;
        }
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
#pragma unroll
        for (int i = 0; i < TM; i++) {
            int r = tx + i * TX;
            int rr = rt[r];
            if (rr < 0) continue;
            T *dst = Cp + rr + (size_t)cc * stf;
            if (tk.excl) *dst -= acc[i][j];
            else atomicAdd(dst, -acc[i][j]);
        }
    }
}

// ---------------------------------------------------------------------------
// Host launch wrappers (called from the driver with level lists in device memory)
// ---------------------------------------------------------------------------
template <typename T>
void launch_fill_coef(int64_t nnz, const double *vals, const int64_t *lmap, const int64_t *umap, T *L, T *U,
                      cudaStream_t st) {
    if (nnz <= 0) return;
    int blocks = (int)std::min<int64_t>((nnz + 255) / 256, 148 * 16);
    k_fill_coef<T><<<blocks, 256, 0, st>>>(nnz, vals, lmap, umap, L, U);
}

template <typename T, int FACT>
void launch_panel_small(const DevStruct &s, const int *list, int count, size_t smem, T *L, T *U,
                        const FactParams &fp, cudaStream_t st) {
    if (count <= 0) return;
    k_panel_small<T, FACT><<<count, 128, smem, st>>>(s, list, L, U, fp);
}

template <typename T, int FACT>
void launch_diag_large(const DevStruct &s, const int *list, int count, size_t smem, T *L, T *U,
                       const FactParams &fp, cudaStream_t st) {
    if (count <= 0) return;
    k_diag_large<T, FACT><<<count, 256, smem, st>>>(s, list, L, U, fp);
}

template <typename T, int FACT>
void launch_trsm(const DevStruct &s, const RowTile *tiles, int count, size_t smem, T *L, T *U, cudaStream_t st) {
    if (count <= 0) return;
    dim3 grid(count, FACT == FACT_GETRF ? 2 : 1);
    k_trsm<T, FACT><<<grid, 256, smem, st>>>(s, tiles, L, U);
}

template <typename T, int FACT>
void launch_update(const DevStruct &s, const UpdTile *tiles, int count, T *L, T *U, cudaStream_t st) {
    if (count <= 0) return;
    k_update<T, FACT, 64, 64, 16, 4, 4><<<count, 256, 0, st>>>(s, tiles, L, U);
}

template <typename T, int FACT>
cudaError_t set_smem_attrs(size_t small_max, size_t diag_max, size_t trsm_max) {
    cudaError_t e;
    e = cudaFuncSetAttribute(k_panel_small<T, FACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)small_max);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_diag_large<T, FACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_max);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_trsm<T, FACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_max);
}

#define PGPU_INST_FACT(T, F)                                                                                     \
    template void launch_panel_small<T, F>(const DevStruct &, const int *, int, size_t, T *, T *,                \
                                           const FactParams &, cudaStream_t);                                    \
    template void launch_diag_large<T, F>(const DevStruct &, const int *, int, size_t, T *, T *,                 \
                                          const FactParams &, cudaStream_t);                                     \
    template void launch_trsm<T, F>(const DevStruct &, const RowTile *, int, size_t, T *, T *, cudaStream_t);     \
    template void launch_update<T, F>(const DevStruct &, const UpdTile *, int, T *, T *, cudaStream_t);          \
    template cudaError_t set_smem_attrs<T, F>(size_t, size_t, size_t);

PGPU_INST_FACT(double, FACT_POTRF)
PGPU_INST_FACT(double, FACT_SYTRF)
PGPU_INST_FACT(double, FACT_GETRF)
PGPU_INST_FACT(float, FACT_POTRF)
PGPU_INST_FACT(float, FACT_SYTRF)
PGPU_INST_FACT(float, FACT_GETRF)
template void launch_fill_coef<double>(int64_t, const double *, const int64_t *, const int64_t *, double *,
                                       double *, cudaStream_t);
template void launch_fill_coef<float>(int64_t, const double *, const int64_t *, const int64_t *, float *,
                                      float *, cudaStream_t);

}  // namespace pgpu
