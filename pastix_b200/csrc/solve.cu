// Supernodal triangular solve kernels (sm_100a).
//
// The right-hand sides live on the device in the permuted numbering, column
// major with leading dimension n.  A solve with a block-lower panel P (the L
// panel, or the U^T panel of an LU factor) is, level by level:
//   forward   y_k <- P_kk^{-1} y_k;  y[rows(k)] -= P_off(k) y_k       (k_fwd_diag, k_fwd_update)
//   backward  x_k <- P_kk^{-T} (x_k - P_off(k)^T x[rows(k)])            (k_bwd_update, k_bwd_diag)
// which restates solve_cblk_ztrsmsp_forward / _backward
// (kernels/solve_ztrsmsp.c:302, :468) and solve_blok_ztrsm / _zgemm (:76, :160)
// with the step table of pastix_subtask_solve_adv (sopalin/pastix_task_solve.c:543-649):
//   POTRF  L (non-unit) then L^T;  SYTRF  L (unit), D, L^T (unit);
//   GETRF  L (unit) then U through the stored U^T panel (non-unit).
// Independent cblks of one level run in one launch; the scatter of the
// forward update uses atomics because several cblks of a level can face the
// same rows.
#include "device.cuh"

namespace pgpu {

constexpr int RC = 8;      // right-hand sides per CTA (gridDim.y covers nrhs)
constexpr int SROWS = 128; // panel rows per update tile (one per thread)

// Forward diagonal solve: y_k <- P_kk^{-1} y_k (lower, unit or not).  One CTA
// per cblk; blocks of 32 columns are solved by warp 0 with shuffles, the rest
// of the block column is updated by all threads.
template <typename T>
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
        if (tid < 32) {
            const int lane = tid;
            for (int j = 0; j < nr; j++) {
                T v = (lane < nb) ? y[jb + lane + j * nc] : T(0);
                for (int c = 0; c < nb; c++) {
                    if (lane == c && !unit) v /= D[(jb + c) + (size_t)(jb + c) * st];
                    T vc = __shfl_sync(0xffffffffu, v, c);
                    if (lane > c && lane < nb) v -= D[(jb + lane) + (size_t)(jb + c) * st] * vc;
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

// Forward update: y[row(r)] -= sum_c P[r, c] y_k[c] for the off-diagonal rows
// of a row tile (one thread per row).
template <typename T>
__global__ void __launch_bounds__(SROWS) k_fwd_update(DevStruct s, const RowTile *__restrict__ tiles, const T *P,
                                                       T *Y, int ldy, int nrhs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *yk = reinterpret_cast<T *>(smem_raw);  // nc x RC
    const RowTile tl = tiles[blockIdx.x];
    const int k = tl.cblk;
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC;
    const int nr = min(RC, nrhs - j0);
    const int tid = threadIdx.x;
    for (int e = tid; e < nc * nr; e += blockDim.x) {
        int i = e % nc, j = e / nc;
        yk[i + j * nc] = Y[(fc + i) + (size_t)(j0 + j) * ldy];
    }
    __syncthreads();
    const int r = tl.r0 + tid;
    if (r >= st || tid >= SROWS) return;
    const T *Pr = P + s.cb_coef[k] + r;
    T acc[RC];
#pragma unroll
    for (int j = 0; j < RC; j++) acc[j] = T(0);
    for (int c = 0; c < nc; c++) {
        T p = Pr[(size_t)c * st];
#pragma unroll
        for (int j = 0; j < RC; j++) acc[j] += p * yk[c + j * nc];
    }
    const int g = s.rowidx[s.cb_rowidx[k] + r];
#pragma unroll
    for (int j = 0; j < RC; j++)
        if (j < nr) atomicAdd(&Y[g + (size_t)(j0 + j) * ldy], -acc[j]);
}

// Backward update: x_k[c] -= sum_r P[r, c] x[row(r)] over a row tile; warps
// reduce over rows, one shared accumulator per (column, rhs).
template <typename T>
__global__ void __launch_bounds__(SROWS) k_bwd_update(DevStruct s, const RowTile *__restrict__ tiles, const T *P,
                                                       T *Y, int ldy, int nrhs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *xr = reinterpret_cast<T *>(smem_raw);  // SROWS x RC gathered x[row(r)]
    const RowTile tl = tiles[blockIdx.x];
    const int k = tl.cblk;
    const int fc = s.cb_fcol[k];
    const int nc = s.cb_lcol[k] - fc + 1;
    const int st = s.cb_stride[k];
    const int j0 = blockIdx.y * RC;
    const int nr = min(RC, nrhs - j0);
    const int tid = threadIdx.x;
    const int rows = min(SROWS, st - tl.r0);
    const int *ridx = s.rowidx + s.cb_rowidx[k] + tl.r0;
    for (int e = tid; e < SROWS * RC; e += blockDim.x) {
        int i = e % SROWS, j = e / SROWS;
        xr[e] = (i < rows && j < nr) ? Y[ridx[i] + (size_t)(j0 + j) * ldy] : T(0);
    }
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const T *Pk = P + s.cb_coef[k] + tl.r0;
    // each warp owns columns c = warp, warp+nw, ...; lanes stride over rows
    for (int c = warp; c < nc; c += nw) {
        T acc[RC];
#pragma unroll
        for (int j = 0; j < RC; j++) acc[j] = T(0);
        for (int i = lane; i < rows; i += 32) {
            T p = Pk[i + (size_t)c * st];
#pragma unroll
            for (int j = 0; j < RC; j++) acc[j] += p * xr[i + j * SROWS];
        }
#pragma unroll
        for (int j = 0; j < RC; j++) {
            T v = acc[j];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0 && j < nr) atomicAdd(&Y[(fc + c) + (size_t)(j0 + j) * ldy], -v);
        }
    }
}

// Backward diagonal solve: x_k <- P_kk^{-T} x_k (P_kk lower; unit or not).
template <typename T>
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
    // blocks of 32 from the bottom: solve the block with warp 0, then update
    // the rows above it (x_i -= sum_c P[c, i] x_c for c in the block).
    for (int je = nc; je > 0; je -= 32) {
        const int jb = max(0, je - 32);
        const int nb = je - jb;
        if (tid < 32) {
            const int lane = tid;
            for (int j = 0; j < nr; j++) {
                T v = (lane < nb) ? y[jb + lane + j * nc] : T(0);
                for (int c = nb - 1; c >= 0; c--) {
                    if (lane == c && !unit) v /= D[(jb + c) + (size_t)(jb + c) * st];
                    T vc = __shfl_sync(0xffffffffu, v, c);
                    if (lane < c) v -= D[(jb + c) + (size_t)(jb + lane) * st] * vc;
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

template <typename T>
static inline dim3 rgrid(int count, int nrhs) { return dim3(count, (nrhs + RC - 1) / RC); }

template <typename T>
void launch_fwd_diag(const DevStruct &s, const int *list, int count, int maxnc, const T *P, int unit, T *Y, int ldy,
                     int nrhs, cudaStream_t st) {
    if (count <= 0) return;
    k_fwd_diag<T><<<rgrid<T>(count, nrhs), 256, (size_t)maxnc * RC * sizeof(T), st>>>(s, list, P, unit, Y, ldy, nrhs);
}
template <typename T>
void launch_fwd_update(const DevStruct &s, const RowTile *tiles, int count, int maxnc, const T *P, T *Y, int ldy,
                       int nrhs, cudaStream_t st) {
    if (count <= 0) return;
    k_fwd_update<T><<<rgrid<T>(count, nrhs), SROWS, (size_t)maxnc * RC * sizeof(T), st>>>(s, tiles, P, Y, ldy, nrhs);
}
template <typename T>
void launch_bwd_update(const DevStruct &s, const RowTile *tiles, int count, const T *P, T *Y, int ldy, int nrhs,
                       cudaStream_t st) {
    if (count <= 0) return;
    k_bwd_update<T><<<rgrid<T>(count, nrhs), SROWS, (size_t)SROWS * RC * sizeof(T), st>>>(s, tiles, P, Y, ldy, nrhs);
}
template <typename T>
void launch_bwd_diag(const DevStruct &s, const int *list, int count, int maxnc, const T *P, int unit, T *Y, int ldy,
                     int nrhs, cudaStream_t st) {
    if (count <= 0) return;
    k_bwd_diag<T><<<rgrid<T>(count, nrhs), 256, (size_t)maxnc * RC * sizeof(T), st>>>(s, list, P, unit, Y, ldy, nrhs);
}
template <typename T>
void launch_diag_scale(const DevStruct &s, int cblknbr, const T *L, T *Y, int ldy, int nrhs, cudaStream_t st) {
    if (cblknbr <= 0) return;
    k_diag_scale<T><<<cblknbr, 128, 0, st>>>(s, L, Y, ldy, nrhs);
}
int solve_rows_per_tile() { return SROWS; }

#define PGPU_INST_SOLVE(T)                                                                                       \
    template void launch_fwd_diag<T>(const DevStruct &, const int *, int, int, const T *, int, T *, int, int,     \
                                     cudaStream_t);                                                              \
    template void launch_fwd_update<T>(const DevStruct &, const RowTile *, int, int, const T *, T *, int, int,    \
                                       cudaStream_t);                                                            \
    template void launch_bwd_update<T>(const DevStruct &, const RowTile *, int, const T *, T *, int, int,         \
                                       cudaStream_t);                                                            \
    template void launch_bwd_diag<T>(const DevStruct &, const int *, int, int, const T *, int, T *, int, int,     \
                                     cudaStream_t);                                                              \
    template void launch_diag_scale<T>(const DevStruct &, int, const T *, T *, int, int, cudaStream_t);

PGPU_INST_SOLVE(double)
PGPU_INST_SOLVE(float)

}  // namespace pgpu
