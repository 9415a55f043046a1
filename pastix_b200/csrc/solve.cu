// Supernodal triangular solve kernels (sm_100a).
//
// The right-hand sides live on the device in the permuted numbering, column
// major with leading dimension ldy.  A solve with a block-lower panel P (the L
// panel, or the U^T panel of an LU factor) is, level by level:
//   forward   y_k <- P_kk^{-1} y_k;  y[rows(k)] -= P_off(k) y_k       (diag kernels, k_fwd_update)
//   backward  x_k <- P_kk^{-T} (x_k - P_off(k)^T x[rows(k)])            (k_bwd_update, diag kernels)
// which restates solve_cblk_ztrsmsp_forward / _backward
// (kernels/solve_ztrsmsp.c:302, :468) and solve_blok_ztrsm / _zgemm (:76, :160)
// with the step table of pastix_subtask_solve_adv (sopalin/pastix_task_solve.c:543-649):
//   POTRF  L (non-unit) then L^T;  SYTRF  L (unit), D, L^T (unit);
//   GETRF  L (unit) then U through the stored U^T panel (non-unit).
// Independent cblks of one level run in one launch.  The off-diagonal
// products use 64 x 64 tiles of the panel (rows x columns) so that a level's
// wide cblks spread over many CTAs; partial sums go to the right-hand sides by
// atomics.  Diagonal blocks of wide cblks are applied with the inverted 32 x 32
// sub-blocks kept by the factorization (a blocked triangular solve whose
// diagonal steps are small matrix-vector products); narrow cblks use
// substitution by one warp per right-hand side.
#include "device.cuh"

#include <cooperative_groups.h>

namespace pgpu {

constexpr int ST_R = 64, ST_C = 64;  // solve update tile: panel rows x panel columns

// ---------------------------------------------------------------------------
// Narrow cblks: substitution, blocks of 32 rows on the lanes of a warp, one
// warp per right-hand side.
// ---------------------------------------------------------------------------
template <typename T, int RC>
__global__ void __launch_bounds__(256) k_fwd_diag(DevStruct s, const int *__restrict__ list, const T *P, int unit,
                                                   T *Y, int ldy, int nrhs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *y = reinterpret_cast<T *>(smem_raw);  // nc x RC
    const int k = list[blockIdx.x];
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC;
    const int nr = min(RC, nrhs - j0);
    const T *D = P + s.cb_coef[k];
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < nc * nr; e += nt) {
        int i = e % nc, j = e / nc;
        y[i + j * nc] = Y[(fc + i) + (size_t)(j0 + j) * ldy];
    }
    __syncthreads();
    for (int jb = 0; jb < nc; jb += 32) {
        const int nb = min(32, nc - jb);
        {
            const int lane = tid & 31, warp = tid >> 5;
            const T rd = (!unit && lane < nb) ? T(1) / D[(jb + lane) + (size_t)(jb + lane) * st] : T(1);
            T drow[32];  // row jb + lane of the block, loaded before the dependent sweep
#pragma unroll
            for (int c = 0; c < 32; c++)
                drow[c] = (c < lane && lane < nb) ? D[(jb + lane) + (size_t)(jb + c) * st] : T(0);
            for (int j = warp; j < nr; j += nt / 32) {
                T v = (lane < nb) ? y[jb + lane + j * nc] : T(0);
#pragma unroll
                for (int c = 0; c < 32; c++) {
                    if (c < nb) {
                        if (lane == c) v *= rd;
                        const T vc = __shfl_sync(0xffffffffu, v, c);
                        v -= drow[c] * vc;
                    }
                }
                if (lane < nb) y[jb + lane + j * nc] = v;
            }
        }
        __syncthreads();
        for (int e = tid; e < (nc - jb - nb) * nr; e += nt) {
            int i = jb + nb + e % (nc - jb - nb), j = e / (nc - jb - nb);
            T acc = T(0);
            for (int c = 0; c < nb; c++) acc += D[i + (size_t)(jb + c) * st] * y[jb + c + j * nc];
            y[i + j * nc] -= acc;
        }
        __syncthreads();
    }
    for (int e = tid; e < nc * nr; e += nt) {
        int i = e % nc, j = e / nc;
        Y[(fc + i) + (size_t)(j0 + j) * ldy] = y[i + j * nc];
    }
}

template <typename T, int RC>
__global__ void __launch_bounds__(256) k_bwd_diag(DevStruct s, const int *__restrict__ list, const T *P, int unit,
                                                   T *Y, int ldy, int nrhs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *y = reinterpret_cast<T *>(smem_raw);
    const int k = list[blockIdx.x];
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC;
    const int nr = min(RC, nrhs - j0);
    const T *D = P + s.cb_coef[k];
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < nc * nr; e += nt) {
        int i = e % nc, j = e / nc;
        y[i + j * nc] = Y[(fc + i) + (size_t)(j0 + j) * ldy];
    }
    __syncthreads();
    for (int je = nc; je > 0; je -= 32) {
        const int jb = max(0, je - 32);
        const int nb = je - jb;
        {
            const int lane = tid & 31, warp = tid >> 5;
            const T rd = (!unit && lane < nb) ? T(1) / D[(jb + lane) + (size_t)(jb + lane) * st] : T(1);
            T dcol[32];  // column jb + lane of the block, loaded before the dependent sweep
#pragma unroll
            for (int c = 0; c < 32; c++)
                dcol[c] = (lane < c && c < nb) ? D[(jb + c) + (size_t)(jb + lane) * st] : T(0);
            for (int j = warp; j < nr; j += nt / 32) {
                T v = (lane < nb) ? y[jb + lane + j * nc] : T(0);
#pragma unroll
                for (int c = 31; c >= 0; c--) {
                    if (c < nb) {
                        if (lane == c) v *= rd;
                        const T vc = __shfl_sync(0xffffffffu, v, c);
                        v -= dcol[c] * vc;
                    }
                }
                if (lane < nb) y[jb + lane + j * nc] = v;
            }
        }
        __syncthreads();
        for (int e = tid; e < jb * nr; e += nt) {
            int i = e % jb, j = e / jb;
            T acc = T(0);
            for (int c = 0; c < nb; c++) acc += D[(jb + c) + (size_t)i * st] * y[jb + c + j * nc];
            y[i + j * nc] -= acc;
        }
        __syncthreads();
    }
    for (int e = tid; e < nc * nr; e += nt) {
        int i = e % nc, j = e / nc;
        Y[(fc + i) + (size_t)(j0 + j) * ldy] = y[i + j * nc];
    }
}

// One right-hand side: one warp per narrow cblk (width <= 64, since
// stride * width <= 4096), eight cblks per CTA -- the leaves of the tree are
// tens of thousands of such cblks, and a CTA each left seven of its warps
// idle.  y_k lives in two registers per lane (columns lane, 32 + lane); the
// substitution steps are those of k_fwd_diag / k_bwd_diag.
template <typename T>
__device__ __forceinline__ T warp_fwd_block(const T *D, int st, int jb, int nb, int unit, int lane, T v) {
    const T rd = (!unit && lane < nb) ? T(1) / D[(jb + lane) + (size_t)(jb + lane) * st] : T(1);
    T drow[32];
#pragma unroll
    for (int c = 0; c < 32; c++) drow[c] = (c < lane && lane < nb) ? D[(jb + lane) + (size_t)(jb + c) * st] : T(0);
#pragma unroll
    for (int c = 0; c < 32; c++) {
        if (c < nb) {
            if (lane == c) v *= rd;
            const T vc = __shfl_sync(0xffffffffu, v, c);
            v -= drow[c] * vc;
        }
    }
    return v;
}
template <typename T>
__device__ __forceinline__ T warp_bwd_block(const T *D, int st, int jb, int nb, int unit, int lane, T v) {
    const T rd = (!unit && lane < nb) ? T(1) / D[(jb + lane) + (size_t)(jb + lane) * st] : T(1);
    T dcol[32];
#pragma unroll
    for (int c = 0; c < 32; c++) dcol[c] = (lane < c && c < nb) ? D[(jb + c) + (size_t)(jb + lane) * st] : T(0);
#pragma unroll
    for (int c = 31; c >= 0; c--) {
        if (c < nb) {
            if (lane == c) v *= rd;
            const T vc = __shfl_sync(0xffffffffu, v, c);
            v -= dcol[c] * vc;
        }
    }
    return v;
}

template <typename T>
__global__ void __launch_bounds__(256) k_fwd_diag_w(DevStruct s, const int *__restrict__ list, int count, const T *P,
                                                     int unit, T *Y) {
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (w >= count) return;  // whole warps
    const int k = list[w];
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const T *D = P + s.cb_coef[k];
    T y0 = lane < nc ? Y[fc + lane] : T(0);
    T y1 = 32 + lane < nc ? Y[fc + 32 + lane] : T(0);
    y0 = warp_fwd_block<T>(D, st, 0, min(32, nc), unit, lane, y0);
    if (nc > 32) {  // rows 32 .. nc - 1 of the diagonal block: y1 -= D[32 + lane, 0..31] y0
        const int r = 32 + lane;
        T acc = T(0);
#pragma unroll
        for (int c = 0; c < 32; c++) {
            const T yc = __shfl_sync(0xffffffffu, y0, c);
            if (r < nc) acc += D[r + (size_t)c * st] * yc;
        }
        y1 = warp_fwd_block<T>(D, st, 32, nc - 32, unit, lane, y1 - acc);
    }
    if (lane < nc) Y[fc + lane] = y0;
    if (32 + lane < nc) Y[fc + 32 + lane] = y1;
}

template <typename T>
__global__ void __launch_bounds__(256) k_bwd_diag_w(DevStruct s, const int *__restrict__ list, int count, const T *P,
                                                     int unit, T *Y) {
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (w >= count) return;
    const int k = list[w];
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const T *D = P + s.cb_coef[k];
    T y0 = lane < nc ? Y[fc + lane] : T(0);
    T y1 = 32 + lane < nc ? Y[fc + 32 + lane] : T(0);
    if (nc > 32) {  // the last block first, then its contribution to rows 0..31: y0 -= D[32 + c, lane] y1[c]
        y1 = warp_bwd_block<T>(D, st, 32, nc - 32, unit, lane, y1);
        T acc = T(0);
#pragma unroll
        for (int c = 0; c < 32; c++) {
            const T yc = __shfl_sync(0xffffffffu, y1, c);
            if (32 + c < nc) acc += D[(32 + c) + (size_t)lane * st] * yc;
        }
        y0 -= acc;
    }
    y0 = warp_bwd_block<T>(D, st, 0, min(32, nc), unit, lane, y0);
    if (lane < nc) Y[fc + lane] = y0;
    if (32 + lane < nc) Y[fc + 32 + lane] = y1;
}

// ---------------------------------------------------------------------------
// Wide cblks: blocked diagonal solves with the inverted 32 x 32 sub-blocks Z
// (Z = T^{-1}, T the upper factor of the sub-block, see factor.cu):
//   forward   y_j <- S Z^T y_j,  then  y[below] -= P[below, j] y_j
//   backward  x_j -= P[below, j]^T x[below],  then  x_j <- Z S x_j
// with S = D (LDL^T, scaled) or I.  zside picks the Z set (GETRF: 0 = U, 1 = L^T).
// ---------------------------------------------------------------------------
// Diagonal steps with the full inverse of the block's triangular factor, kept
// (transposed, FP32) by the FP32 factorization for its TRSM: Pt = T^{-T},
// column major nc x nc, lower triangular.  Forward: y <- S Pt y; backward:
// x <- Pt^T S x (S = D for LDL^T, else I) -- the blocked steps of
// solve_cblk_ztrsmsp_forward / _backward as one dense product, for RC
// right-hand sides.  A cluster of TC CTAs shares one cblk: every CTA copies
// y_k to its shared memory, and the lower triangle of Pt is cut into 32 x 32
// tiles spread over the cluster's 8 * TC warps (at most two each, 32
// independent coalesced loads per lane), so that no warp walks a long row or
// column alone.  Partial sums go by distributed-shared-memory atomics to the
// CTA that owns the 32 outputs (block b -> CTA b % TC); a second cluster
// barrier orders every partial before the owners overwrite y_k in place.
constexpr int TC = 8;

// Tile t of the lower triangle of an nch x nch block grid, row by row:
// (i, jc) with jc <= i and t = i (i + 1) / 2 + jc.
__device__ __forceinline__ void tri_tile(int t, int &i, int &jc) {
    i = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
    while ((i + 1) * (i + 2) / 2 <= t) i++;
    while (i * (i + 1) / 2 > t) i--;
    jc = t - i * (i + 1) / 2;
}

template <typename T, int RC>
__global__ void __cluster_dims__(TC, 1, 1) __launch_bounds__(256)
    k_fwd_diag_tinv(DevStruct s, const int *__restrict__ list, int zside, int scaled, const T *Ldiag, T *Y, int ldy,
                    int nrhs, const float *__restrict__ tinv, const int64_t *__restrict__ ti_off) {
    __shared__ float ys[RC][384];
    __shared__ float acc[RC][384];
    const int k = list[blockIdx.x / TC];
    const int64_t off = ti_off[k];
    if (off < 0) return;  // the whole cluster leaves: k_fwd_diag_inv takes this cblk
    cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC, nr = min(RC, nrhs - j0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int npad = 32 * ((nc + 31) / 32);  // whole 32-blocks: the tiles read ys up to npad
    for (int e = tid; e < npad * RC; e += blockDim.x) {
        const int i = e % npad, j = e / npad;
        ys[j][i] = (j < nr && i < nc) ? (float)Y[fc + i + (size_t)(j0 + j) * ldy] : 0.f;
        acc[j][i] = 0.f;
    }
    cluster.sync();  // every copy of y_k made, every accumulator cleared
    const float *Pt = tinv + off + (size_t)zside * nc * nc;
    const int nch = (nc + 31) / 32, ntile = nch * (nch + 1) / 2;
    for (int t = rank * 8 + warp; t < ntile; t += TC * 8) {
        int i, jc;
        tri_tile(t, i, jc);
        const int r = 32 * i + lane, c0 = 32 * jc;
        float a[RC];
#pragma unroll
        for (int j = 0; j < RC; j++) a[j] = 0.f;
        if (r < nc) {
            float p[32];
#pragma unroll
            for (int u = 0; u < 32; u++) p[u] = (c0 + u < nc) ? Pt[r + (size_t)(c0 + u) * nc] : 0.f;
#pragma unroll
            for (int u = 0; u < 32; u++)
#pragma unroll
                for (int j = 0; j < RC; j++) a[j] += p[u] * ys[j][c0 + u];
            float *dst = cluster.map_shared_rank(&acc[0][0], i % TC);
#pragma unroll
            for (int j = 0; j < RC; j++)
                if (j < nr) atomicAdd(dst + j * 384 + r, a[j]);
        }
    }
    cluster.sync();  // every partial sum in place
    for (int cb = rank * 32; cb < nc; cb += TC * 32)
        for (int e = tid; e < 32 * RC; e += blockDim.x) {
            const int l = e & 31, j = e >> 5, c = cb + l;
            if (c < nc && j < nr) {
                float v = acc[j][c];
                if (scaled) v *= (float)Ldiag[s.cb_coef[k] + c + (size_t)c * st];
                Y[fc + c + (size_t)(j0 + j) * ldy] = (T)v;
            }
        }
}

// Groups of 8 right-hand sides: 8 products per loaded element make the work
// compute-heavy enough that 32-row (forward) or 32-column (backward) blocks
// round robin over the cluster's CTAs, with no cross-CTA partial sums, beat the
// tiled kernels (whose remote atomics grow with the number of right-hand
// sides); a single right-hand side uses the tiled kernels.
template <typename T, int RC>
__global__ void __cluster_dims__(TC, 1, 1) __launch_bounds__(256)
    k_fwd_diag_tinv_rr(DevStruct s, const int *__restrict__ list, int zside, int scaled, const T *Ldiag, T *Y, int ldy,
                    int nrhs, const float *__restrict__ tinv, const int64_t *__restrict__ ti_off) {
    __shared__ float ys[RC][384];
    __shared__ float part[8][RC][33];
    const int k = list[blockIdx.x / TC];
    const int64_t off = ti_off[k];
    if (off < 0) return;  // the whole cluster leaves: k_fwd_diag_inv takes this cblk
    cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC, nr = min(RC, nrhs - j0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < nc * RC; e += blockDim.x) {
        const int i = e % nc, j = e / nc;
        ys[j][i] = j < nr ? (float)Y[fc + i + (size_t)(j0 + j) * ldy] : 0.f;
    }
    cluster.sync();
    const float *Pt = tinv + off + (size_t)zside * nc * nc;
    for (int cb = rank * 32; cb < nc; cb += TC * 32) {
        const int c = cb + lane;
        const int kend = min(nc, cb + 32);  // Pt is lower triangular: columns past the block are zero
        float acc[RC];
#pragma unroll
        for (int j = 0; j < RC; j++) acc[j] = 0.f;
        if (c < nc) {
#pragma unroll 8
            for (int kk = warp; kk < kend; kk += 8) {
                const float pv = Pt[c + (size_t)kk * nc];
#pragma unroll
                for (int j = 0; j < RC; j++) acc[j] += pv * ys[j][kk];
            }
        }
#pragma unroll
        for (int j = 0; j < RC; j++) part[warp][j][lane] = acc[j];
        __syncthreads();
        for (int o = tid; o < 32 * RC; o += blockDim.x) {
            const int l = o & 31, j = o >> 5, cc = cb + l;
            if (cc < nc && j < nr) {
                float v = 0.f;
#pragma unroll
                for (int w = 0; w < 8; w++) v += part[w][j][l];
                if (scaled) v *= (float)Ldiag[s.cb_coef[k] + cc + (size_t)cc * st];
                Y[fc + cc + (size_t)(j0 + j) * ldy] = (T)v;
            }
        }
        __syncthreads();
    }
}

template <typename T, int RC>
__global__ void __cluster_dims__(TC, 1, 1) __launch_bounds__(256)
    k_bwd_diag_tinv_rr(DevStruct s, const int *__restrict__ list, int zside, int scaled, const T *Ldiag, T *Y, int ldy,
                    int nrhs, const float *__restrict__ tinv, const int64_t *__restrict__ ti_off) {
    __shared__ float xs[RC][384];
    const int k = list[blockIdx.x / TC];
    const int64_t off = ti_off[k];
    if (off < 0) return;  // the whole cluster leaves: k_bwd_diag_inv takes this cblk
    cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC, nr = min(RC, nrhs - j0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < nc * RC; e += blockDim.x) {
        const int i = e % nc, j = e / nc;
        float v = j < nr ? (float)Y[fc + i + (size_t)(j0 + j) * ldy] : 0.f;
        if (scaled) v *= (float)Ldiag[s.cb_coef[k] + i + (size_t)i * st];
        xs[j][i] = v;
    }
    cluster.sync();
    const float *Pt = tinv + off + (size_t)zside * nc * nc;
    // x_c = sum_{r >= c} Pt[r, c] xs[r]: four columns per warp, lanes over the rows (coalesced)
    for (int cb = rank * 32; cb < nc; cb += TC * 32) {
        const int c0 = cb + 4 * warp;
        float acc[4][RC];
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int j = 0; j < RC; j++) acc[u][j] = 0.f;
        for (int r = c0 + lane; r < nc; r += 32) {
            float pv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) pv[u] = (c0 + u < nc && r >= c0 + u) ? Pt[r + (size_t)(c0 + u) * nc] : 0.f;
#pragma unroll
            for (int j = 0; j < RC; j++) {
                const float xr = xs[j][r];
#pragma unroll
                for (int u = 0; u < 4; u++) acc[u][j] += pv[u] * xr;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int j = 0; j < RC; j++) {
                float v = acc[u][j];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0 && c0 + u < nc && j < nr) Y[fc + c0 + u + (size_t)(j0 + j) * ldy] = (T)v;
            }
    }
}

// Sum over the 32 lanes of v[u] for every u at once (butterfly transpose
// reduction, 31 shuffles): on return lane l holds in v[0] the sum of v[l].
__device__ __forceinline__ void lane_sums32(float (&v)[32], int lane) {
#pragma unroll
    for (int sft = 16; sft >= 1; sft >>= 1) {
        const bool upper = (lane & sft) != 0;
#pragma unroll
        for (int u = 0; u < sft; u++) {
            const float send = upper ? v[u] : v[u + sft];
            const float keep = upper ? v[u + sft] : v[u];
            v[u] = keep + __shfl_xor_sync(0xffffffffu, send, sft);
        }
    }
}

template <typename T, int RC>
__global__ void __cluster_dims__(TC, 1, 1) __launch_bounds__(256)
    k_bwd_diag_tinv(DevStruct s, const int *__restrict__ list, int zside, int scaled, const T *Ldiag, T *Y, int ldy,
                    int nrhs, const float *__restrict__ tinv, const int64_t *__restrict__ ti_off) {
    __shared__ float xs[RC][384];
    __shared__ float acc[RC][384];
    const int k = list[blockIdx.x / TC];
    const int64_t off = ti_off[k];
    if (off < 0) return;  // the whole cluster leaves: k_bwd_diag_inv takes this cblk
    cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC, nr = min(RC, nrhs - j0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int npad = 32 * ((nc + 31) / 32);
    for (int e = tid; e < npad * RC; e += blockDim.x) {
        const int i = e % npad, j = e / npad;
        float v = (j < nr && i < nc) ? (float)Y[fc + i + (size_t)(j0 + j) * ldy] : 0.f;
        if (scaled && i < nc) v *= (float)Ldiag[s.cb_coef[k] + i + (size_t)i * st];
        xs[j][i] = v;
        acc[j][i] = 0.f;
    }
    cluster.sync();
    const float *Pt = tinv + off + (size_t)zside * nc * nc;
    // x_c = sum_{r >= c} Pt[r, c] xs[r]: tile (row block i, column block jc <= i), lanes over the rows
    const int nch = (nc + 31) / 32, ntile = nch * (nch + 1) / 2;
    for (int t = rank * 8 + warp; t < ntile; t += TC * 8) {
        int i, jc;
        tri_tile(t, i, jc);
        const int r = 32 * i + lane, c0 = 32 * jc;
        float p[32];
#pragma unroll
        for (int u = 0; u < 32; u++)
            p[u] = (r < nc && c0 + u < nc && r >= c0 + u) ? Pt[r + (size_t)(c0 + u) * nc] : 0.f;
        float *dst = cluster.map_shared_rank(&acc[0][0], jc % TC);
#pragma unroll
        for (int j = 0; j < RC; j++) {
            if (j >= nr) break;
            const float xr = r < nc ? xs[j][r] : 0.f;
            float v[32];
#pragma unroll
            for (int u = 0; u < 32; u++) v[u] = p[u] * xr;
            lane_sums32(v, lane);
            if (c0 + lane < nc) atomicAdd(dst + j * 384 + c0 + lane, v[0]);
        }
    }
    cluster.sync();  // every partial sum in place
    for (int cb = rank * 32; cb < nc; cb += TC * 32)
        for (int e = tid; e < 32 * RC; e += blockDim.x) {
            const int l = e & 31, j = e >> 5, c = cb + l;
            if (c < nc && j < nr) Y[fc + c + (size_t)(j0 + j) * ldy] = (T)acc[j][c];
        }
}

template <typename T, int RC>
__global__ void __launch_bounds__(256) k_fwd_diag_inv(DevStruct s, const int *__restrict__ list, const T *P,
                                                       const T *__restrict__ dinv, int zside, int scaled,
                                                       const T *Ldiag, T *Y, int ldy, int nrhs,
                                                       const float *__restrict__ tinv,
                                                       const int64_t *__restrict__ ti_off) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *y = reinterpret_cast<T *>(smem_raw);  // nc x RC
    __shared__ T Z[32 * 33];
    __shared__ T yb[32 * RC];
    const int k = list[blockIdx.x];
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC;
    const int nr = min(RC, nrhs - j0);
    const T *D = P + s.cb_coef[k];
    const T *Dl = Ldiag + s.cb_coef[k];
    const int nzb = (nc + 31) / 32;
    const T *gZ = dinv + s.cb_dinv[k] + (size_t)(zside ? nzb : 0) * 1024;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tinv != nullptr && ti_off[k] >= 0) return;  // k_fwd_diag_tinv applies the kept full inverse
    for (int e = tid; e < nc * nr; e += nt) {
        int i = e % nc, j = e / nc;
        y[i + j * nc] = Y[(fc + i) + (size_t)(j0 + j) * ldy];
    }
    for (int jb = 0; jb < nc; jb += 32) {
        const int nb = min(32, nc - jb);
        for (int e = tid; e < 1024; e += nt) Z[(e >> 5) * 33 + (e & 31)] = gZ[(size_t)(jb / 32) * 1024 + e];
        __syncthreads();
        for (int e = tid; e < 32 * RC; e += nt) {  // yb = S Z^T y_j
            int i = e & 31, j = e >> 5;
            T acc = T(0);
            if (i < nb && j < nr) {
                for (int c = 0; c <= i; c++) acc += Z[c * 33 + i] * y[jb + c + j * nc];
                if (scaled) acc *= Dl[(jb + i) + (size_t)(jb + i) * st];
            }
            yb[e] = acc;
        }
        __syncthreads();
        for (int e = tid; e < 32 * RC; e += nt) {
            int i = e & 31, j = e >> 5;
            if (i < nb && j < nr) y[jb + i + j * nc] = yb[e];
        }
        __syncthreads();
        // rows below inside the diagonal block (the block is full when rows remain):
        // one row per thread, its 32 panel entries loaded together
        for (int r = jb + 32 + tid; r < nc; r += nt) {
            T p[32];
#pragma unroll
            for (int c = 0; c < 32; c++) p[c] = D[r + (size_t)(jb + c) * st];
            T acc[RC];
#pragma unroll
            for (int j = 0; j < RC; j++) acc[j] = T(0);
#pragma unroll
            for (int c = 0; c < 32; c++) {
                const T pc = p[c];
#pragma unroll
                for (int j = 0; j < RC; j++) acc[j] += pc * yb[c + j * 32];
                asm volatile("" ::: "memory");  // keeps the compiler from hoisting all shared loads ahead
            }
#pragma unroll
            for (int j = 0; j < RC; j++)
                if (j < nr) y[r + j * nc] -= acc[j];
        }
        __syncthreads();
    }
    for (int e = tid; e < nc * nr; e += nt) {
        int i = e % nc, j = e / nc;
        Y[(fc + i) + (size_t)(j0 + j) * ldy] = y[i + j * nc];
    }
}

// Backward, right looking inside the diagonal block: once x_j is final its
// contribution P[block j, c]^T x_j is removed from every earlier column c, one
// warp per column (coalesced 32-row reads, shuffle reductions).
template <typename T, int RC>
__global__ void __launch_bounds__(256) k_bwd_diag_inv(DevStruct s, const int *__restrict__ list, const T *P,
                                                       const T *__restrict__ dinv, int zside, int scaled,
                                                       const T *Ldiag, T *Y, int ldy, int nrhs,
                                                       const float *__restrict__ tinv,
                                                       const int64_t *__restrict__ ti_off) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *y = reinterpret_cast<T *>(smem_raw);  // nc x RC
    __shared__ T Z[32 * 33];
    __shared__ T yb[32 * RC];
    const int k = list[blockIdx.x];
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC;
    const int nr = min(RC, nrhs - j0);
    const T *D = P + s.cb_coef[k];
    const T *Dl = Ldiag + s.cb_coef[k];
    const int nzb = (nc + 31) / 32;
    const T *gZ = dinv + s.cb_dinv[k] + (size_t)(zside ? nzb : 0) * 1024;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    if (tinv != nullptr && ti_off[k] >= 0) return;  // k_bwd_diag_tinv applies the kept full inverse
    for (int e = tid; e < nc * nr; e += nt) {
        int i = e % nc, j = e / nc;
        y[i + j * nc] = Y[(fc + i) + (size_t)(j0 + j) * ldy];
    }
    __syncthreads();
    for (int b = nzb - 1; b >= 0; b--) {
        const int jb = b * 32;
        const int nb = min(32, nc - jb);
        for (int e = tid; e < 1024; e += nt) Z[(e >> 5) * 33 + (e & 31)] = gZ[(size_t)b * 1024 + e];
        for (int e = tid; e < 32 * RC; e += nt) {  // yb = S x_j (contributions of later blocks already removed)
            int i = e & 31, j = e >> 5;
            T v = T(0);
            if (i < nb && j < nr) {
                v = y[jb + i + j * nc];
                if (scaled) v *= Dl[(jb + i) + (size_t)(jb + i) * st];
            }
            yb[e] = v;
        }
        __syncthreads();
        for (int e = tid; e < 32 * RC; e += nt) {  // x_j = Z yb
            int i = e & 31, j = e >> 5;
            if (i < nb && j < nr) {
                T acc = T(0);
                for (int c = i; c < nb; c++) acc += Z[i * 33 + c] * yb[c + j * 32];
                y[jb + i + j * nc] = acc;
            }
        }
        __syncthreads();
        for (int c0 = 8 * warp; c0 < jb; c0 += nt / 4) {  // x_c -= P[block j, c]^T x_j, 8 columns per warp
            T p[8];
#pragma unroll
            for (int u = 0; u < 8; u++)
                p[u] = (lane < nb && c0 + u < jb) ? D[(jb + lane) + (size_t)(c0 + u) * st] : T(0);
#pragma unroll
            for (int j = 0; j < RC; j++) {
                if (j >= nr) break;
                const T xv = (lane < nb) ? y[jb + lane + j * nc] : T(0);
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    T v = p[u] * xv;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    if (lane == 0 && c0 + u < jb) y[c0 + u + j * nc] -= v;
                }
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < nc * nr; e += nt) {
        int i = e % nc, j = e / nc;
        Y[(fc + i) + (size_t)(j0 + j) * ldy] = y[i + j * nc];
    }
}

// ---------------------------------------------------------------------------
// Off-diagonal products on 64 x 64 panel tiles (RowTile.r0 = first row, the
// tile's column block is blockIdx.z).  Forward: y[row(r)] -= P[r, cols] y_k[cols];
// backward: x_k[c] -= sum_r P[r, c] x[row(r)].
// ---------------------------------------------------------------------------
template <typename T, int RC>
__global__ void __launch_bounds__(256) k_fwd_update(DevStruct s, const RowTile *__restrict__ tiles, const T *P,
                                                     T *Y, int ldy, int nrhs) {
    __shared__ T yk[ST_C * RC];
    __shared__ T part[4][ST_R * RC];
    const RowTile tl = tiles[blockIdx.x];
    const int k = tl.cblk;
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int c0 = blockIdx.z * ST_C;
    if (c0 >= nc) return;
    const int ncol = min(ST_C, nc - c0);
    const int st = s.cb_stride[k];
    const int rows = min(ST_R, st - tl.r0);
    const int j0 = blockIdx.y * RC;
    const int nr = min(RC, nrhs - j0);
    const int tid = threadIdx.x;
    const int r = tid % ST_R, g = tid / ST_R, cb = 16 * g;  // 4 column groups of 16
    // the panel tile and the target rows do not depend on y_k: their loads are issued first and
    // overlap the staging of y_k (one memory round trip per tile instead of three)
    T p[16];
    {
        const T *Pr = P + s.cb_coef[k] + tl.r0 + r + (size_t)c0 * st;
#pragma unroll
        for (int u = 0; u < 16; u++) p[u] = (r < rows && cb + u < ncol) ? Pr[(size_t)(cb + u) * st] : T(0);
    }
    const int gr = (tid < ST_R && tid < rows) ? s.rowidx[s.cb_rowidx[k] + tl.r0 + tid] : 0;
    for (int e = tid; e < ST_C * RC; e += 256) {
        int c = e % ST_C, j = e / ST_C;
        yk[e] = (c < ncol && j < nr) ? Y[(fc + c0 + c) + (size_t)(j0 + j) * ldy] : T(0);
    }
    __syncthreads();
    T acc[RC];
#pragma unroll
    for (int j = 0; j < RC; j++) acc[j] = T(0);
#pragma unroll
    for (int u = 0; u < 16; u++)
#pragma unroll
        for (int j = 0; j < RC; j++) acc[j] += p[u] * yk[cb + u + j * ST_C];
#pragma unroll
    for (int j = 0; j < RC; j++) part[g][r + j * ST_R] = acc[j];
    __syncthreads();
    if (tid < ST_R && tid < rows) {
#pragma unroll
        for (int j = 0; j < RC; j++) {
            if (j >= nr) break;
            T v = part[0][tid + j * ST_R] + part[1][tid + j * ST_R] + part[2][tid + j * ST_R] + part[3][tid + j * ST_R];
            atomicAdd(&Y[gr + (size_t)(j0 + j) * ldy], -v);
        }
    }
}

template <typename T, int RC>
__global__ void __launch_bounds__(256) k_bwd_update(DevStruct s, const RowTile *__restrict__ tiles, const T *P,
                                                     T *Y, int ldy, int nrhs) {
    __shared__ T xr[ST_R * RC];
    const RowTile tl = tiles[blockIdx.x];
    const int k = tl.cblk;
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int c0 = blockIdx.z * ST_C;
    if (c0 >= nc) return;
    const int ncol = min(ST_C, nc - c0);
    const int st = s.cb_stride[k];
    const int rows = min(ST_R, st - tl.r0);
    const int j0 = blockIdx.y * RC;
    const int nr = min(RC, nrhs - j0);
    const int tid = threadIdx.x;
    const int *ridx = s.rowidx + s.cb_rowidx[k] + tl.r0;
    // thread (row r, 16-column group g): 16 independent coalesced loads of the
    // panel tile, issued before the gather of x (which needs the row indices
    // first), so that the two overlap
    const T *Pk = P + s.cb_coef[k] + tl.r0 + (size_t)c0 * st;
    const int r = tid % ST_R, g = tid / ST_R, cb = 16 * g;
    T p[16];
#pragma unroll
    for (int u = 0; u < 16; u++) p[u] = (r < rows && cb + u < ncol) ? Pk[r + (size_t)(cb + u) * st] : T(0);
    for (int e = tid; e < ST_R * RC; e += 256) {
        int i = e % ST_R, j = e / ST_R;
        xr[e] = (i < rows && j < nr) ? Y[ridx[i] + (size_t)(j0 + j) * ldy] : T(0);
    }
    __syncthreads();
    if constexpr (RC == 1) {
        // the products P[r, c] x[r] staged in shared memory (row stride 65: no
        // bank conflicts on either side), then one thread per column sums its 64 rows
        __shared__ T prod[ST_C * (ST_R + 1)];
        const T xv = xr[r];
#pragma unroll
        for (int u = 0; u < 16; u++) prod[(cb + u) * (ST_R + 1) + r] = p[u] * xv;
        __syncthreads();
        if (tid < ncol) {
            T v = T(0);
#pragma unroll 16
            for (int i = 0; i < ST_R; i++) v += prod[tid * (ST_R + 1) + i];
            atomicAdd(&Y[(fc + c0 + tid) + (size_t)j0 * ldy], -v);
        }
        return;
    } else {
        // out[c, j] = sum_r P[r, c] x[r, j]: the tile staged transposed in shared memory,
        // then 64 columns x RC dot products
        __shared__ T pt[ST_C * (ST_R + 1)];
#pragma unroll
        for (int u = 0; u < 16; u++) pt[(cb + u) * (ST_R + 1) + r] = p[u];
        __syncthreads();
        for (int o = tid; o < ST_C * RC; o += 256) {
            const int c = o % ST_C, j = o / ST_C;
            if (c < ncol && j < nr) {
                T v = T(0);
#pragma unroll 16
                for (int i = 0; i < ST_R; i++) v += pt[c * (ST_R + 1) + i] * xr[i + j * ST_R];
                atomicAdd(&Y[(fc + c0 + c) + (size_t)(j0 + j) * ldy], -v);
            }
        }
    }
}

// Diagonal step of LDL^T: x_i /= D_i (solve_cblk_zdiag, kernels/solve_ztrsmsp.c:664).
template <typename T>
__global__ void k_diag_scale(DevStruct s, const T *L, T *Y, int ldy, int nrhs) {
    const int k = blockIdx.x;
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const T *D = L + s.cb_coef[k];
    for (int e = threadIdx.x; e < nc * nrhs; e += blockDim.x) {
        int i = e % nc, j = e / nc;
        Y[(fc + i) + (size_t)j * ldy] /= D[i + (size_t)i * st];
    }
}

// ------------------------------ launchers ---------------------------------
#define PGPU_RC_DISPATCH(nrhs, KERNEL, GRIDX, SMEM_PER_RC, ...)                                      \
    do {                                                                                            \
        if ((nrhs) == 1) {                                                                          \
            KERNEL<T, 1><<<dim3(GRIDX, 1, ZDIM), 256, (SMEM_PER_RC) * 1, st>>>(__VA_ARGS__);       \
        } else {                                                                                    \
            KERNEL<T, 8><<<dim3(GRIDX, ((nrhs) + 7) / 8, ZDIM), 256, (SMEM_PER_RC) * 8, st>>>(__VA_ARGS__); \
        }                                                                                           \
    } while (0)

template <typename T>
void launch_fwd_diag(const DevStruct &s, const int *list, int count, int maxnc, const T *P, int unit, T *Y, int ldy,
                     int nrhs, cudaStream_t st) {
    if (count <= 0) return;
    if (nrhs == 1) {  // narrow cblks (width <= 64): one warp each
        k_fwd_diag_w<T><<<(count + 7) / 8, 256, 0, st>>>(s, list, count, P, unit, Y);
        return;
    }
    const int ZDIM = 1;
    PGPU_RC_DISPATCH(nrhs, k_fwd_diag, count, (size_t)maxnc * sizeof(T), s, list, P, unit, Y, ldy, nrhs);
}
template <typename T>
void launch_bwd_diag(const DevStruct &s, const int *list, int count, int maxnc, const T *P, int unit, T *Y, int ldy,
                     int nrhs, cudaStream_t st) {
    if (count <= 0) return;
    if (nrhs == 1) {
        k_bwd_diag_w<T><<<(count + 7) / 8, 256, 0, st>>>(s, list, count, P, unit, Y);
        return;
    }
    const int ZDIM = 1;
    PGPU_RC_DISPATCH(nrhs, k_bwd_diag, count, (size_t)maxnc * sizeof(T), s, list, P, unit, Y, ldy, nrhs);
}
// ntinv: how many cblks of the list have a kept full inverse (FP32 factors);
// those go to the 8-CTA cluster kernels, the rest to the blocked kernels, and
// a kernel with no cblk of its own is not launched.
template <typename T>
void launch_fwd_diag_inv(const DevStruct &s, const int *list, int count, int maxnc, const T *P, const T *dinv,
                         int zside, int scaled, const T *Ld, T *Y, int ldy, int nrhs, const float *tinv,
                         const int64_t *ti_off, int ntinv, cudaStream_t st) {
    if (count <= 0) return;
    if (tinv == nullptr) ntinv = 0;
    const int ZDIM = 1;
    if (ntinv > 0) {
        if (nrhs == 1) k_fwd_diag_tinv<T, 1><<<count * TC, 256, 0, st>>>(s, list, zside, scaled, Ld, Y, ldy, nrhs, tinv, ti_off);
        else k_fwd_diag_tinv_rr<T, 8><<<dim3(count * TC, (nrhs + 7) / 8), 256, 0, st>>>(s, list, zside, scaled, Ld, Y, ldy, nrhs, tinv, ti_off);
    }
    if (ntinv < count)
        PGPU_RC_DISPATCH(nrhs, k_fwd_diag_inv, count, (size_t)maxnc * sizeof(T), s, list, P, dinv, zside, scaled, Ld,
                         Y, ldy, nrhs, tinv, ti_off);
}
template <typename T>
void launch_bwd_diag_inv(const DevStruct &s, const int *list, int count, int maxnc, const T *P, const T *dinv,
                         int zside, int scaled, const T *Ld, T *Y, int ldy, int nrhs, const float *tinv,
                         const int64_t *ti_off, int ntinv, cudaStream_t st) {
    if (count <= 0) return;
    if (tinv == nullptr) ntinv = 0;
    const int ZDIM = 1;
    if (ntinv > 0) {
        if (nrhs == 1) k_bwd_diag_tinv<T, 1><<<count * TC, 256, 0, st>>>(s, list, zside, scaled, Ld, Y, ldy, nrhs, tinv, ti_off);
        else k_bwd_diag_tinv_rr<T, 8><<<dim3(count * TC, (nrhs + 7) / 8), 256, 0, st>>>(s, list, zside, scaled, Ld, Y, ldy, nrhs, tinv, ti_off);
    }
    if (ntinv < count)
        PGPU_RC_DISPATCH(nrhs, k_bwd_diag_inv, count, (size_t)maxnc * sizeof(T), s, list, P, dinv, zside, scaled, Ld,
                         Y, ldy, nrhs, tinv, ti_off);
}
template <typename T>
void launch_fwd_update(const DevStruct &s, const RowTile *tiles, int count, int maxnc, const T *P, T *Y, int ldy,
                       int nrhs, cudaStream_t st) {
    if (count <= 0) return;
    const int ZDIM = (maxnc + ST_C - 1) / ST_C;
    PGPU_RC_DISPATCH(nrhs, k_fwd_update, count, 0, s, tiles, P, Y, ldy, nrhs);
}
template <typename T>
void launch_bwd_update(const DevStruct &s, const RowTile *tiles, int count, int maxnc, const T *P, T *Y, int ldy,
                       int nrhs, cudaStream_t st) {
    if (count <= 0) return;
    const int ZDIM = (maxnc + ST_C - 1) / ST_C;
    PGPU_RC_DISPATCH(nrhs, k_bwd_update, count, 0, s, tiles, P, Y, ldy, nrhs);
}
template <typename T>
void launch_diag_scale(const DevStruct &s, int cblknbr, const T *L, T *Y, int ldy, int nrhs, cudaStream_t st) {
    if (cblknbr <= 0) return;
    k_diag_scale<T><<<cblknbr, 128, 0, st>>>(s, L, Y, ldy, nrhs);
}
int solve_rows_per_tile() { return ST_R; }

#define PGPU_INST_SOLVE(T)                                                                                       \
    template void launch_fwd_diag<T>(const DevStruct &, const int *, int, int, const T *, int, T *, int, int,     \
                                     cudaStream_t);                                                              \
    template void launch_bwd_diag<T>(const DevStruct &, const int *, int, int, const T *, int, T *, int, int,     \
                                     cudaStream_t);                                                              \
    template void launch_fwd_diag_inv<T>(const DevStruct &, const int *, int, int, const T *, const T *, int,     \
                                         int, const T *, T *, int, int, const float *, const int64_t *, int,     \
                                         cudaStream_t);                                                          \
    template void launch_bwd_diag_inv<T>(const DevStruct &, const int *, int, int, const T *, const T *, int,     \
                                         int, const T *, T *, int, int, const float *, const int64_t *, int,     \
                                         cudaStream_t);                                                          \
    template void launch_fwd_update<T>(const DevStruct &, const RowTile *, int, int, const T *, T *, int, int,    \
                                       cudaStream_t);                                                            \
    template void launch_bwd_update<T>(const DevStruct &, const RowTile *, int, int, const T *, T *, int, int,    \
                                       cudaStream_t);                                                            \
    template void launch_diag_scale<T>(const DevStruct &, int, const T *, T *, int, int, cudaStream_t);

PGPU_INST_SOLVE(double)
PGPU_INST_SOLVE(float)

}  // namespace pgpu
