// Device-side view of the solver structure and the launch lists of the B200
// numerical phase.  Everything here is plain device pointers; the host driver
// (api.cu) owns the allocations.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace pgpu {

// Factorization kinds (pastix_factotype_t of include/pastix/api.h).
enum FactKind : int { FACT_POTRF = 0, FACT_SYTRF = 1, FACT_GETRF = 2 };

// One update task: C_dst -= A(rows [row0 + a_shift, stride_src)) * B(rows [row0, row0+n))^T,
// scattered into the panel of dst.  a_shift is 0 for the L side and n for the
// U side of an LU update (core_zgemmsp_2d2d shift, kernels/core_zgemmsp.c:433).
struct TaskDev {
    int src, dst;
    int row0, n;      // the blok facing dst: panel row offset and height
    int m;            // rows of src from row0 to the end of its panel
    int excl;         // 1: no other source of the same level writes dst
};

// One output tile of an update task.
struct UpdTile {
    int task;
    int mt, nt;       // tile coordinates inside the task's (m x n) product
    int side;         // 0: L side, 1: U side (LU only)
};

// Rows of one off-diagonal TRSM tile (k_trsm); its shared memory holds the
// tile and a 32-row strip of the triangular factor, 2 x 32 x (nc + 1) elements.
__host__ __device__ inline int trsm_tile_rows(int) { return 32; }
__host__ __device__ inline long long trsm_smem_elems(int nc) { return 2LL * 32 * (nc + 1); }
// Elements of the inverted diagonal sub-blocks kept for a wide cblk of width nc.
__host__ __device__ inline long long dinv_elems(int nc, int fact) {
    return (long long)((nc + 31) / 32) * 1024 * (fact == FACT_GETRF ? 2 : 1);
}

// Shared memory of k_diag_large for a cblk of width nc: the nc x 32 column
// panel (ld 33) and, for GETRF, the 32 x nc strip of U (ld nc + 1).
__host__ __device__ inline long long diag_smem_elems(int nc, int fact) {
    return (long long)nc * 33 + (fact == FACT_GETRF ? 32LL * (nc + 1) : 0);
}

// One row tile of a cblk's off-diagonal panel (TRSM and solve updates).
struct RowTile {
    int cblk;
    int r0;           // first panel row of the tile (>= width: below the diagonal block)
};

// A slab of 128 panel rows of one cblk, split into BF16 terms by k_split.
struct SplitSlab {
    int cblk;
    int r0;
};

// A slab of 128 rows of a dense column-major FP32 matrix split into its BF16
// image by k_split_dense (the transposed triangular inverses of k_trinv).
struct DenseSlab {
    int64_t src;  // element offset of the matrix
    int64_t img;  // byte offset of its image
    int ld, rows, cols, r0;
};

struct DevStruct {
    int n;
    int cblknbr;
    const int *cb_fcol, *cb_lcol, *cb_stride, *cb_fblok;
    const int64_t *cb_coef;     // panel offset (elements) of each cblk
    const int64_t *cb_rowidx;   // offset of each cblk in rowidx
    const int64_t *cb_dinv;     // offset of each wide cblk's inverted 32x32 diagonal sub-blocks (-1: none)
    const int *bk_frow, *bk_lrow, *bk_rowoff, *bk_fcblk;
    const int *rowidx;          // global row of every panel row
    const TaskDev *tasks;
};

// Per-call scalars for the factorization kernels.
// Programmatic dependent launch: a kernel launched with
// cudaLaunchAttributeProgrammaticStreamSerialization may be scheduled before the
// kernel ahead of it in the stream has ended; it waits here, before its first
// memory access, until that kernel has ended and its writes are visible.
// Without such a launch it returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Launches of the FP32 factorization's level chains may overlap the launch of
// each kernel with the end of the one ahead of it in its stream (every kernel
// launched this way waits in pdl_wait first); switched on per host thread by
// set_pdl.
void set_pdl(bool on);
bool pdl_enabled();
template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args) {
    if (!pdl_enabled()) {
        kernel<<<grid, block, smem, st>>>(args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

struct FactParams {
    const double *criterion;    // static pivoting threshold (eps * ||A||_F), in device memory so that
                                // a captured launch sequence stays valid when the values change
    int *nbpivots;              // device counter
    int *status;                // device status word (0 = fine)
    double *dscr;               // k_diag_cluster: the finished panels of each cblk of a launch, DC_SCR_DOUBLES per cblk
};

// Element-wise transfer by a whole CTA with UNR independent loads in flight per
// thread: st(e, ld(e)) for e in [0, total).  All loads of a batch are issued
// before its stores, so a staging loop costs one memory round trip per UNR
// elements instead of one per element.
template <int UNR, typename V, typename LoadF, typename StoreF>
__device__ __forceinline__ void batched_copy(int total, LoadF ld, StoreF stf) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e0 = tid; e0 < total; e0 += nt * UNR) {
        V v[UNR];
#pragma unroll
        for (int u = 0; u < UNR; u++) {
            const int e = e0 + u * nt;
            if (e < total) v[u] = ld(e);
        }
#pragma unroll
        for (int u = 0; u < UNR; u++) {
            const int e = e0 + u * nt;
            if (e < total) stf(e, v[u]);
        }
    }
}

}  // namespace pgpu
