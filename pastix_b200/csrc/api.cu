// Host driver of the B200 numerical phase: pastix_data_t, the pastix_task_* /
// pastix_subtask_* entry points, device residency of the factor, and the
// level-by-level launch sequence of the factorization and of the solve.
//
// Entry points follow the reference's control flow and argument checks:
//   pastixInitParam / pastixInit / pastixFinalize   common/api.c:420,905,928
//   pastix_task_analyze                             blend/pastix_task_analyze.c:53
//   pastix_subtask_spm2bcsc/bcsc2ctab/sopalin       sopalin/pastix_task_sopalin.c:93,213,412
//   pastix_task_numfact                             sopalin/pastix_task_sopalin.c:654
//   pastix_subtask_applyorder/trsm/diag/solve(_adv) sopalin/pastix_task_solve.c:169,296,422,512,713
//   pastix_task_solve                               sopalin/pastix_task_solve.c:758
//   pastix_subtask_refine / pastix_task_refine      refinement/pastix_task_refine.c:106,236
//   pastix()                                        sopalin/pastix.c:103
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include <unistd.h>

#include "../../include/pastix_b200.h"
#include "device.cuh"
#include "symbol.hpp"

namespace pgpu {
// factor.cu
template <typename T>
void launch_fill_coef(int64_t, const double *, const int64_t *, const int64_t *, T *, T *, cudaStream_t);
template <typename T, int F>
void launch_panel_small(const DevStruct &, const int *, int, size_t, T *, T *, const FactParams &, cudaStream_t);
template <typename T, int F>
void launch_diag_large(const DevStruct &, const int *, int, int, size_t, T *, T *, T *, const FactParams &,
                       cudaStream_t);
template <typename T, int F>
void launch_trsm(const DevStruct &, const RowTile *, int, int, size_t, T *, T *, const T *, cudaStream_t);
template <typename T, int F>
void launch_update(const DevStruct &, const UpdTile *, int, T *, T *, cudaStream_t);
template <typename T, int F>
void launch_update_big(const DevStruct &, const UpdTile *, int, T *, T *, cudaStream_t);
template <int F>
void launch_update_tc(const DevStruct &, const UpdTile *, int, float *, float *, const unsigned char *,
                      const unsigned char *, const int64_t *, int *, int *, cudaStream_t);
void launch_split(const DevStruct &, const SplitSlab *, int, const float *, const float *, const int64_t *,
                  unsigned char *, int, cudaStream_t);
long long split_image_bytes(int nc, int st);
long long panel_small_bytes(long long panel_elems, int tsize, int maxst);
int trinv_max_blocks();
size_t diag_cluster_scratch_doubles();
cudaError_t wait_selftest(int *timed_out_host);
void set_pdl(bool on);
template <int F>
void launch_trinv(const DevStruct &, const int *, int, int, const float *, const float *, const float *,
                  const int64_t *, float *, cudaStream_t);
void launch_split_dense(const DenseSlab *, int, const float *, unsigned char *, cudaStream_t);
template <int F>
void launch_trsm_tc(const DevStruct &, const UpdTile *, int, float *, float *, const unsigned char *,
                    const unsigned char *, const int64_t *, const unsigned char *, const int64_t *, int *, int *,
                    cudaStream_t);
template <typename T, int F>
cudaError_t set_smem_attrs(size_t, size_t, size_t);
// solve.cu
template <typename T>
void launch_fwd_diag(const DevStruct &, const int *, int, int, const T *, int, T *, int, int, cudaStream_t);
template <typename T>
void launch_fwd_update(const DevStruct &, const RowTile *, int, int, const T *, T *, int, int, cudaStream_t);
template <typename T>
void launch_bwd_update(const DevStruct &, const RowTile *, int, int, const T *, T *, int, int, cudaStream_t);
template <typename T>
void launch_fwd_diag_inv(const DevStruct &, const int *, int, int, const T *, const T *, int, int, const T *, T *,
                         int, int, const float *, const int64_t *, int, cudaStream_t);
template <typename T>
void launch_bwd_diag_inv(const DevStruct &, const int *, int, int, const T *, const T *, int, int, const T *, T *,
                         int, int, const float *, const int64_t *, int, cudaStream_t);
template <typename T>
void launch_bwd_diag(const DevStruct &, const int *, int, int, const T *, int, T *, int, int, cudaStream_t);
template <typename T>
void launch_diag_scale(const DevStruct &, int, const T *, T *, int, int, cudaStream_t);
int solve_rows_per_tile();
// vec.cu
void spmv_partition(int n, const int *rowptr, std::vector<int> &part);
void launch_spmv_stream(int nblocks, const int *part, const int *rowptr, const int *col, const double *val,
                        double alpha, const double *x, double beta, double *y, cudaStream_t st);
void launch_spmv(int, int64_t, const int *, const int *, const double *, double, const double *, double, double *,
                 cudaStream_t);
int reduce_partials();
void launch_dot(int64_t, const double *, const double *, double *, int, double *, cudaStream_t);
void launch_axpy(int64_t, double, const double *, double *, cudaStream_t);
void launch_xpby(int64_t, const double *, double, double *, cudaStream_t);
void launch_scal(int64_t, double, double *, cudaStream_t);
void launch_gemv(int64_t, int, const double *, const double *, double *, cudaStream_t);
void launch_spmm(int, int, const int *, const int *, const double *, double, const double *, int64_t, double, double *,
                 int64_t, cudaStream_t);
void launch_dots_cols(int64_t, int, int, const double *, int64_t, int64_t, const double *, int64_t, int, double *,
                      cudaStream_t);
void launch_axpy_cols(int64_t, int, const double *, const double *, int64_t, double *, int64_t, cudaStream_t);
void launch_scal_cols(int64_t, int, const double *, int, double *, int64_t, cudaStream_t);
void launch_gemv_cols(int64_t, int, int, const double *, int64_t, const double *, double *, int64_t, cudaStream_t);
void launch_xpby_cols(int64_t, int, const double *, const double *, double *, cudaStream_t);
template <typename TS, typename TD>
void launch_permute(int, int, const int64_t *, int, const TS *, int64_t, TD *, int64_t, cudaStream_t);
template <typename TS, typename TD>
void launch_cast(int64_t, const TS *, TD *, cudaStream_t);
void launch_sampled(int64_t, const int *, const int *, double, const double *, const double *, double *, int,
                    cudaStream_t);
}  // namespace pgpu

using pgpu::idx_t;

// kernel classes for launch accounting (pgpu_profile_get)
enum : int {
    PC_FILL = 0, PC_PANEL_SMALL, PC_DIAG_LARGE, PC_TRSM, PC_UPDATE, PC_FWD_DIAG, PC_FWD_UPDATE, PC_BWD_UPDATE,
    PC_BWD_DIAG, PC_SPMV, PC_VEC, PC_UPDATE_BIG, PC_SPLIT, PGPU_NCLASS
};

// ---------------------------------------------------------------------------
// internal state
// ---------------------------------------------------------------------------
enum : int {
    STEP_INIT = 1 << 0, STEP_ORDERING = 1 << 1, STEP_SYMBFACT = 1 << 2, STEP_ANALYSE = 1 << 3,
    STEP_CSC2BCSC = 1 << 4, STEP_BCSC2CTAB = 1 << 5, STEP_NUMFACT = 1 << 6, STEP_SOLVE = 1 << 7,
    STEP_REFINE = 1 << 8
};

namespace {

constexpr idx_t SMALL_PANEL_ELEMS = 4096;  // st*nc below which a cblk is factored in one CTA's smem

template <typename X>
struct DBuf {  // owning device buffer
    X *p = nullptr;
    size_t n = 0;
    ~DBuf() { reset(); }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t cnt) {
        if (cnt == n && p) return cudaSuccess;
        reset();
        if (cnt == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, cnt * sizeof(X));
        if (e == cudaSuccess) n = cnt;
        return e;
    }
    cudaError_t upload(const std::vector<X> &v, cudaStream_t st) {
        cudaError_t e = alloc(v.size());
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpyAsync(p, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice, st);
    }
};

// Launch lists of one level, as offsets into the flat device arrays.
struct LevelLists {
    int small0, small1;     // k_panel_small cblks
    int large0, large1;     // k_diag_large cblks
    int trsm0, trsm1;       // k_trsm row tiles
    int upd0, upd1;         // k_update tiles (64 x 64), FP64 factors
    int upds0, upds1;       // k_update tiles (64 x 64), FP32 factors (tasks the tcgen05 kernel does not take)
    int updb0, updb1;       // big update tiles (128 x 64): DMMA for FP64
    int updt0, updt1;       // the same tasks in 128-row aligned windows: tcgen05 for FP32
    int updtn, updsn;       // FP32 lists: tiles before these target the next level's cblks
    int spl0, spl1;         // 128-row slabs of the level's cblks split into BF16 terms (FP32)
    int tt0, tt1;           // FP32 TRSM as GEMM tiles (tcgen05), task = cblk
    int ds0, ds1;           // 128-row slabs of the transposed triangular inverses
    int tr32_0, tr32_1;     // FP32: DMMA TRSM tiles of the wide cblks the GEMM form does not take
    int ti_maxnzb;          // 32-column blocks of the widest cblk with a triangular inverse
    int cb0, cb1;           // all cblks of the level (solve diag)
    int st0, st1;           // solve row tiles
    int maxnc;
    int trsm_maxnc;         // widest cblk with TRSM tiles
    int diag_maxnc;         // widest cblk of the large list
    size_t small_smem_elems, diag_smem_elems, trsm_smem_elems;
    int small_maxst;        // tallest narrow cblk (tables of the fused updates)
    int ntinv;              // wide cblks with a kept full triangular inverse (FP32 factors)
};

struct Device {
    bool ready = false;
    int dev = -1;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;                      // FP32 factorization: updates of later levels
    std::vector<cudaEvent_t> ev_chain, ev_rest;       // per level: panels final / far updates done
    // structure
    DBuf<int> cb_fcol, cb_lcol, cb_stride, cb_fblok, bk_frow, bk_lrow, bk_rowoff, bk_fcblk, rowidx;
    DBuf<int64_t> cb_coef, cb_rowidx, cb_dinv, sp_off;
    DBuf<pgpu::SplitSlab> split_slabs;
    DBuf<int64_t> ti_off, ti_img;
    DBuf<pgpu::DenseSlab> dense_slabs;
    DBuf<pgpu::UpdTile> trsm_tc_tiles;
    DBuf<pgpu::RowTile> trsm_tiles32;
    DBuf<float> tinv;                // transposed triangular inverses (FP32 factors)
    DBuf<unsigned char> timg;        // their BF16 images
    DBuf<unsigned char> img0, img1;  // BF16 images of the FP32 panels (tcgen05 operands)
    DBuf<pgpu::TaskDev> tasks;
    DBuf<int> small_list, large_list, level_cblks;
    DBuf<pgpu::RowTile> trsm_tiles, solve_tiles;
    DBuf<pgpu::UpdTile> upd_tiles, upd_big_tiles, upd_tc_tiles, upd_tiles32;
    // matrix
    DBuf<double> vals, csr_val;
    DBuf<int64_t> lmap, umap, csr_src, perm;
    DBuf<int> csr_rowptr, csr_col, e_row, e_col;
    DBuf<int> spmv_part;     // row blocks of the streamed SpMV
    int spmv_nblocks = 0;
    // factor
    DBuf<unsigned char> Lc, Uc, dinv;  // panels; inverted 32x32 diagonal sub-blocks of wide cblks
    int fltsize = 0;
    // work
    DBuf<int> counters;      // [0] nbpivots, [1] status
    DBuf<int> queues;        // tile work-queue heads of the tcgen05 launches, 3 per level, zeroed per factorization
    DBuf<double> dcscr;      // finished panels of the cluster diagonal kernel (read by the cluster's other CTAs)
    DBuf<double> crit;       // static pivoting threshold of the current factorization
    DBuf<double> part, scal; // reduction partials, scalars
    DBuf<double> w1, w2;     // permuted double work vectors
    DBuf<float> wf;          // float work for mixed precision
    DBuf<double> ws[16];     // grow-only work areas (no allocation in the steady state)
    pgpu::DevStruct ds{};
};

}  // namespace

// One captured launch sequence: the key names the sequence and every device
// address baked into its launches; `launches` is its per-class launch count.
struct GraphEntry {
    std::vector<uintptr_t> key;
    cudaGraphExec_t exec = nullptr;
    int64_t launches[PGPU_NCLASS] = {0};
    uint64_t used = 0;
};
struct GraphCache {
    static constexpr size_t kMax = 16;  // least recently used entries beyond this are dropped
    std::vector<GraphEntry> e;
    uint64_t tick = 0;
    ~GraphCache() { clear(); }
    void clear() {
        for (auto &g : e)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        e.clear();
    }
};

struct pastix_rhs_s {
    int8_t allocated;
    int flttype;           // SpmDouble or SpmFloat
    pastix_int_t m, n, ld;
    void *b;               // device memory, permuted numbering
};

struct pastix_data_s {
    pastix_int_t *iparm = nullptr;
    double *dparm = nullptr;
    int steps = 0;
    // analysed pattern
    idx_t n = 0, nnz = 0;
    int mtxtype = SpmGeneral;
    std::vector<idx_t> colptr, rowind;  // 0-based copy of the pattern
    pgpu::Graph graph;
    pgpu::Order order;
    bool user_order = false;
    idx_t dof = 1;              // unknowns per node of a node ordering
    pgpu::Graph node_graph;     // dof > 1: the node graph
    pgpu::Order node_order;     // dof > 1: the ordering of the nodes
    pgpu::Symbol symbol;
    pgpu::Solver solver;
    // value maps (host, structure only)
    std::vector<int64_t> lmap, umap, csr_src;
    std::vector<int> csr_rowptr, csr_col, e_row, e_col;
    idx_t csr_nnz = 0;
    std::vector<LevelLists> levels;
    // host copies of the launch lists
    std::vector<int> small_list, large_list, level_cblks;
    std::vector<pgpu::RowTile> trsm_tiles, solve_tiles;
    std::vector<pgpu::UpdTile> upd_tiles, upd_big_tiles, upd_tc_tiles, upd_tiles32;
    std::vector<pgpu::TaskDev> tasks;
    std::vector<int64_t> cb_dinv;
    std::vector<int64_t> sp_off;             // byte offset of each cblk's BF16 image (-1: none)
    int64_t split_total = 0;
    std::vector<pgpu::SplitSlab> split_slabs;
    std::vector<int64_t> ti_off, ti_img;     // per cblk: FP32 TRSM by GEMM (-1: DMMA TRSM)
    int64_t tinv_total = 0, timg_total = 0;
    std::vector<pgpu::DenseSlab> dense_slabs;
    std::vector<pgpu::UpdTile> trsm_tc_tiles;
    std::vector<pgpu::RowTile> trsm_tiles32;
    int64_t dinv_total = 0;
    int factotype = PastixFactPOTRF;
    int mixed = 0;
    double anorm = 0.0;
    double crit_host = 0.0;  // source of the threshold's copy to the device
    // bucket boundaries of the update tiles (pgpu_set_tuning / pgpu_autotune):
    // FP64 tasks with blok height >= tune_dmma_n and source width >= tune_dmma_k take
    // 128 x 64 DMMA tiles, the others 64 x 64 SIMT tiles; FP32 tasks whose source is
    // at least tune_tc_k wide take tcgen05 tiles (split BF16 terms), the others SIMT
    int tune_dmma_n = 32, tune_dmma_k = 32, tune_tc_k = 32;
    Device dev;
    // launch accounting: per kernel class, launches always counted, device time when profiling
    bool prof_on = false;
    int64_t launches[PGPU_NCLASS] = {0};
    double prof_ms[PGPU_NCLASS] = {0};
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_ev;
    // executable CUDA graphs of the fixed launch sequences (declared after `dev`, so destroyed first)
    bool use_graphs = true;
    GraphCache graphs;
    // GMRES refinement of several right-hand sides as one block (pgpu_refine_block)
    bool refine_block = true;
    std::string dir_global;  // per-instance output directory of PastixIOSave (created on first save)
};

// Run one launch of kernel class `cls` with `count` blocks through `fn`, on
// stream `st` (the library stream by default).
template <typename Fn>
static inline void launch_cls(pastix_data_t *pd, int cls, long long count, Fn &&fn, cudaStream_t st = nullptr) {
    if (count <= 0) return;
    pd->launches[cls]++;
    if (!pd->prof_on) { fn(); return; }
    if (!st) st = pd->dev.stream;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
    fn();
    cudaEventRecord(b, st);
    pd->prof_ev.push_back({cls, {a, b}});
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
enum : int { WS_SOLVE = 0, WS_ORDER, WS_GMV, WS_GMW, WS_GMG, WS_VEC, WS_BP, WS_XP, WS_RB, WS_RX, WS_BGV, WS_BGS,
             WS_SPSV, WS_GMH };

// Persistent device work area `slot` of at least `count` doubles (grown, never shrunk).
static double *work(Device &d, int slot, size_t count) {
    DBuf<double> &b = d.ws[slot];
    if (b.n < count) {
        if (b.alloc(count) != cudaSuccess) return nullptr;
    }
    return b.p;
}
static void perr(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    fprintf(stderr, "pastix_b200: ");
    vfprintf(stderr, fmt, ap);
    fprintf(stderr, "\n");
    va_end(ap);
}

#define CUDA_TRY(call)                                                                    \
    do {                                                                                  \
        cudaError_t _e = (call);                                                          \
        if (_e != cudaSuccess) {                                                          \
            perr("%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
            return PASTIX_ERR_INTERNAL;                                                   \
        }                                                                                 \
    } while (0)

// Run the launch sequence `fn` (which enqueues on the library stream, returns a
// PASTIX code and does not synchronize) as a CUDA graph: captured and
// instantiated on the first call with `key`, replayed by one cudaGraphLaunch
// afterwards.  Runs `fn` directly while per-launch profiling is on or graphs
// are switched off (pgpu_graphs).  The capture is thread-local, so other
// threads' CUDA calls are unaffected; work joined from another stream through
// events (the FP32 side stream) becomes part of the graph.
template <typename Fn>
static int run_graphed(pastix_data_t *pd, const std::vector<uintptr_t> &key, Fn &&fn) {
    if (pd->prof_on || !pd->use_graphs) return fn();
    Device &d = pd->dev;
    GraphCache &gc = pd->graphs;
    for (auto &g : gc.e) {
        if (g.key != key) continue;
        CUDA_TRY(cudaGraphLaunch(g.exec, d.stream));
        for (int c = 0; c < PGPU_NCLASS; c++) pd->launches[c] += g.launches[c];
        g.used = ++gc.tick;
        return PASTIX_SUCCESS;
    }
    int64_t before[PGPU_NCLASS];
    std::memcpy(before, pd->launches, sizeof(before));
    CUDA_TRY(cudaStreamBeginCapture(d.stream, cudaStreamCaptureModeThreadLocal));
    const int rc = fn();
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(d.stream, &graph);
    if (rc != PASTIX_SUCCESS || ce != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        if (rc == PASTIX_SUCCESS) perr("stream capture failed: %s", cudaGetErrorString(ce));
        (void)cudaGetLastError();
        return rc != PASTIX_SUCCESS ? rc : PASTIX_ERR_INTERNAL;
    }
    GraphEntry ent;
    const cudaError_t ie = cudaGraphInstantiate(&ent.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        perr("graph instantiation failed: %s", cudaGetErrorString(ie));
        return PASTIX_ERR_INTERNAL;
    }
    ent.key = key;
    for (int c = 0; c < PGPU_NCLASS; c++) ent.launches[c] = pd->launches[c] - before[c];
    ent.used = ++gc.tick;
    if (gc.e.size() >= GraphCache::kMax) {  // drop the least recently used entry
        size_t lru = 0;
        for (size_t i = 1; i < gc.e.size(); i++)
            if (gc.e[i].used < gc.e[lru].used) lru = i;
        CUDA_TRY(cudaStreamSynchronize(d.stream));
        cudaGraphExecDestroy(gc.e[lru].exec);
        gc.e.erase(gc.e.begin() + (long)lru);
    }
    gc.e.push_back(std::move(ent));
    CUDA_TRY(cudaGraphLaunch(gc.e.back().exec, d.stream));
    return PASTIX_SUCCESS;
}

static double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static int fact_kind(const pastix_data_t *pd) {
    int f = pd->factotype;
    if (f == PastixFactLLT || f == PastixFactPOTRF) return pgpu::FACT_POTRF;
    if (f == PastixFactLDLT || f == PastixFactHETRF) return pgpu::FACT_SYTRF;
    return pgpu::FACT_GETRF;
}

// ---------------------------------------------------------------------------
// parameters (common/api.c:420-571)
// ---------------------------------------------------------------------------
extern "C" void pastixInitParam(pastix_int_t *iparm, double *dparm) {
    if (!iparm || !dparm) return;
    for (int i = 0; i < IPARM_SIZE; i++) iparm[i] = 0;
    for (int i = 0; i < DPARM_SIZE; i++) dparm[i] = 0.0;
    iparm[IPARM_VERBOSE] = PastixVerboseNo;
    iparm[IPARM_ORDERING] = PastixOrderScotch;
    iparm[IPARM_ORDERING_DEFAULT] = 1;
    iparm[IPARM_SCOTCH_MT] = 1;
    iparm[IPARM_SCOTCH_SWITCH_LEVEL] = 120;
    iparm[IPARM_SCOTCH_CMAX] = 100000;
    iparm[IPARM_SCOTCH_FRAT] = 8;
    iparm[IPARM_METIS_CTYPE] = -1;
    iparm[IPARM_METIS_RTYPE] = -1;
    iparm[IPARM_METIS_NSEPS] = 1;
    iparm[IPARM_METIS_NITER] = 10;
    iparm[IPARM_METIS_UFACTOR] = 200;
    iparm[IPARM_METIS_COMPRESS] = 1;
    iparm[IPARM_METIS_SEED] = 3452;
    iparm[IPARM_AMALGAMATION_LVLCBLK] = 5;
    iparm[IPARM_AMALGAMATION_LVLBLAS] = 5;
    iparm[IPARM_REORDERING_STOP] = INT64_MAX;
    iparm[IPARM_SPLITTING_STRATEGY] = 1;  // PastixSplitKway
    iparm[IPARM_SPLITTING_LEVELS_KWAY] = INT64_MAX;
    iparm[IPARM_SPLITTING_PROJECTIONS_DEPTH] = 3;
    iparm[IPARM_SPLITTING_PROJECTIONS_DISTANCE] = 3;
    iparm[IPARM_SPLITTING_PROJECTIONS_WIDTH] = 1;
    iparm[IPARM_MIN_BLOCKSIZE] = 160;
    iparm[IPARM_MAX_BLOCKSIZE] = 320;
    iparm[IPARM_TASKS2D_LEVEL] = -1;
    iparm[IPARM_TASKS2D_WIDTH] = 160;
    iparm[IPARM_FACTORIZATION] = PastixFactLU;
    iparm[IPARM_FACTO_LOOK_SIDE] = 1;  // PastixFactRightLooking
    iparm[IPARM_TRANSPOSE_SOLVE] = PastixNoTrans;
    iparm[IPARM_APPLYPERM_WS] = 1;
    iparm[IPARM_REFINEMENT] = PastixRefineGMRES;
    iparm[IPARM_ITERMAX] = 250;
    iparm[IPARM_GMRES_IM] = 25;
    iparm[IPARM_SCHEDULER] = PastixSchedDynamic;
    iparm[IPARM_THREAD_NBR] = -1;
    iparm[IPARM_SOCKET_NBR] = -1;
    iparm[IPARM_GPU_NBR] = 1;
    iparm[IPARM_GPU_MEMORY_PERCENTAGE] = 95;
    iparm[IPARM_GPU_MEMORY_BLOCK_SIZE] = 32 * 1024;
    iparm[IPARM_COMPRESS_MIN_WIDTH] = 128;
    iparm[IPARM_COMPRESS_MIN_HEIGHT] = 20;
    iparm[IPARM_COMPRESS_METHOD] = 1;  // PQRCP
    iparm[IPARM_COMPRESS_PRESELECT] = 1;
    iparm[IPARM_COMPRESS_ILUK] = -2;
    iparm[IPARM_MODIFY_PARAMETER] = 1;
    iparm[IPARM_START_TASK] = PastixTaskOrdering;
    iparm[IPARM_END_TASK] = PastixTaskClean;
    iparm[IPARM_FLOAT] = -1;
    iparm[IPARM_MTX_TYPE] = -1;
    iparm[IPARM_DOF_NBR] = 1;
    dparm[DPARM_EPSILON_REFINEMENT] = -1.;
    dparm[DPARM_RELATIVE_ERROR] = -1.;
    dparm[DPARM_EPSILON_MAGN_CTRL] = 0.;
    dparm[DPARM_COMPRESS_TOLERANCE] = 0.01;
    dparm[DPARM_COMPRESS_MIN_RATIO] = 1.0;
}

extern "C" void pastixInit(pastix_data_t **pd, PASTIX_Comm, pastix_int_t *iparm, double *dparm) {
    if (!pd) return;
    *pd = nullptr;
    if (!iparm || !dparm) {
        perr("pastixInit: iparm and dparm must be given (call pastixInitParam first)");
        return;
    }
    pastix_data_t *p = new pastix_data_t();
    p->iparm = iparm;
    p->dparm = dparm;
    p->steps = STEP_INIT;
    *pd = p;
}

extern "C" void pastixInitWithAffinity(pastix_data_t **pd, PASTIX_Comm c, pastix_int_t *iparm, double *dparm,
                                       const int *) {
    pastixInit(pd, c, iparm, dparm);
}

extern "C" void pastixFinalize(pastix_data_t **pd) {
    if (!pd || !*pd) return;
    pastix_data_t *p = *pd;
    if (p->dev.ready) {
        cudaSetDevice(p->dev.dev);
        cudaStreamSynchronize(p->dev.stream);
    }
    cudaStream_t st = p->dev.stream;
    if (p->dev.ready) {
        if (p->dev.side) cudaStreamSynchronize(p->dev.side);
        for (auto *v : {&p->dev.ev_chain, &p->dev.ev_rest})
            for (cudaEvent_t e : *v) cudaEventDestroy(e);
        if (p->dev.side) cudaStreamDestroy(p->dev.side);
    }
    delete p;  // DBuf destructors free device memory
    if (st) cudaStreamDestroy(st);
    *pd = nullptr;
}

// ---------------------------------------------------------------------------
// Analysis files (IPARM_IO_STRATEGY).  The ordering and the block symbolic
// matrix in the reference's plain-text formats, so that a file written by
// either library loads in the other:
//   ordering (order/order_io.c:44-120, 199-258): "1", cblknbr, vertnbr, then
//     rangtab (cblknbr + 1), permtab (vertnbr), treetab (cblknbr; absent in
//     version 0), whitespace separated, base = rangtab[0];
//   symbol (symbol/symbol_io.c:51-180): "1", cblknbr, bloknbr, nodenbr,
//     baseval, then fcolnum lcolnum bloknum per cblk and frownum lrownum
//     fcblknm per blok.
// Loads: the ordering from $PASTIX_FILE_ORDER or "ordername", the symbol from
// "symbname" (pastix_subtask_order with a personal ordering,
// pastix_subtask_symbfact); saves: "ordergen" (or $PASTIX_FILE_ORDER) and
// "symbgen" in a directory "<$PASTIX_OUTPUT_DIR or pastix>-XXXXXX" created
// once per instance (common/api.c:85-140).
// ---------------------------------------------------------------------------
static bool read_ints(FILE *f, idx_t *v, size_t count) {
    for (size_t i = 0; i < count; i++) {
        long long x;
        if (fscanf(f, "%lld", &x) != 1) return false;
        v[i] = (idx_t)x;
    }
    return true;
}

static int order_read(FILE *f, pgpu::Order &o) {
    idx_t hdr[3];
    if (!read_ints(f, hdr, 3) || (hdr[0] != 0 && hdr[0] != 1) || hdr[1] < 0 || hdr[2] < 1 || hdr[1] > hdr[2]) {
        perr("pastixOrderLoad: bad header");
        return PASTIX_ERR_FILE;
    }
    const idx_t cb = hdr[1], n = hdr[2];
    o = pgpu::Order{};
    o.n = n;
    o.cblknbr = cb;
    o.rangtab.resize(cb + 1);
    o.permtab.resize(n);
    if (!read_ints(f, o.rangtab.data(), cb + 1) || !read_ints(f, o.permtab.data(), n)) {
        perr("pastixOrderLoad: truncated file");
        return PASTIX_ERR_FILE;
    }
    if (hdr[0] == 1) {
        o.treetab.resize(cb);
        if (!read_ints(f, o.treetab.data(), cb)) {
            perr("pastixOrderLoad: truncated file");
            return PASTIX_ERR_FILE;
        }
    }
    const idx_t base = o.rangtab[0];
    for (auto &v : o.rangtab) v -= base;
    for (auto &v : o.permtab) v -= base;
    for (auto &v : o.treetab) v = v < 0 ? -1 : v - base;
    if (o.rangtab[cb] != n) {
        perr("pastixOrderLoad: rangtab does not cover the %lld vertices", (long long)n);
        return PASTIX_ERR_FILE;
    }
    o.peritab.assign(n, -1);
    for (idx_t i = 0; i < n; i++) {
        if (o.permtab[i] < 0 || o.permtab[i] >= n || o.peritab[o.permtab[i]] >= 0) {
            perr("pastixOrderLoad: permtab is not a permutation");
            return PASTIX_ERR_FILE;
        }
        o.peritab[o.permtab[i]] = i;
    }
    // version 0 keeps rangtab without treetab (order/order_io.c:80-85); the
    // ordering step finds the supernodes again when it needs a tree
    return PASTIX_SUCCESS;
}

// Integers 8 to a line, tab separated (intSave / putc of order/order_io.c).
static void write_ints(FILE *f, const idx_t *v, size_t count) {
    for (size_t i = 0; i < count; i++) fprintf(f, "%lld%c", (long long)v[i], (i % 8 == 7 || i + 1 == count) ? '\n' : '\t');
}

static int order_write(FILE *f, const pgpu::Order &o) {
    if (o.rangtab.empty() || o.treetab.empty() || (idx_t)o.permtab.size() != o.n) {
        perr("pastixOrderSave: the ordering needs permtab, rangtab and treetab");
        return PASTIX_ERR_BADPARAMETER;
    }
    fprintf(f, "1\n%lld\t%lld\n", (long long)o.cblknbr, (long long)o.n);
    write_ints(f, o.rangtab.data(), o.cblknbr + 1);
    write_ints(f, o.permtab.data(), o.n);
    write_ints(f, o.treetab.data(), o.cblknbr);
    return ferror(f) ? PASTIX_ERR_FILE : PASTIX_SUCCESS;
}

static int symbol_read(FILE *f, pgpu::Symbol &sy) {
    idx_t hdr[5];
    if (!read_ints(f, hdr, 5) || hdr[0] < 0 || hdr[0] > 1 || hdr[1] < 1 || hdr[2] < hdr[1] || hdr[3] < hdr[1]) {
        perr("symbol file: bad header");
        return PASTIX_ERR_FILE;
    }
    const idx_t cb = hdr[1], bk = hdr[2], b = hdr[4];
    sy = pgpu::Symbol{};
    sy.nodenbr = hdr[3];
    sy.cblktab.resize(cb + 1);
    sy.bloktab.resize(bk);
    for (idx_t k = 0; k < cb; k++) {
        idx_t v[3];
        if (!read_ints(f, v, 3) || v[0] > v[1]) { perr("symbol file: bad cblk %lld", (long long)k); return PASTIX_ERR_FILE; }
        sy.cblktab[k] = pgpu::SymCblk{v[0] - b, v[1] - b, v[2] - b};
    }
    sy.cblktab[cb] = pgpu::SymCblk{sy.nodenbr, sy.nodenbr, bk};
    for (idx_t k = 0; k < cb; k++)
        if (sy.cblktab[k].bloknum < 0 || sy.cblktab[k].bloknum >= sy.cblktab[k + 1].bloknum) {
            perr("symbol file: bloknum of cblk %lld out of order", (long long)k);
            return PASTIX_ERR_FILE;
        }
    for (idx_t i = 0; i < bk; i++) {
        idx_t v[3];
        if (!read_ints(f, v, 3) || v[0] > v[1] || v[2] - b < 0 || v[2] - b >= cb) {
            perr("symbol file: bad blok %lld", (long long)i);
            return PASTIX_ERR_FILE;
        }
        sy.bloktab[i] = pgpu::SymBlok{v[0] - b, v[1] - b, 0, v[2] - b};
    }
    for (idx_t k = 0; k < cb; k++)  // owning cblk of every blok
        for (idx_t i = sy.cblktab[k].bloknum; i < sy.cblktab[k + 1].bloknum; i++) sy.bloktab[i].lcblknm = k;
    return PASTIX_SUCCESS;
}

static int symbol_write(FILE *f, const pgpu::Symbol &sy) {
    fprintf(f, "1\n%lld\t%lld\t%lld\t%lld\n", (long long)sy.cblknbr(), (long long)sy.bloknbr(), (long long)sy.nodenbr,
            0LL);
    for (idx_t k = 0; k < sy.cblknbr(); k++)
        fprintf(f, "%lld\t%lld\t%lld\n", (long long)sy.cblktab[k].fcolnum, (long long)sy.cblktab[k].lcolnum,
                (long long)sy.cblktab[k].bloknum);
    for (const auto &bl : sy.bloktab)
        fprintf(f, "%lld\t%lld\t%lld\n", (long long)bl.frownum, (long long)bl.lrownum, (long long)bl.fcblknm);
    return ferror(f) ? PASTIX_ERR_FILE : PASTIX_SUCCESS;
}

// "<$PASTIX_OUTPUT_DIR or pastix>-XXXXXX", created on first use (pastix_gendirectories).
static const char *output_dir(pastix_data_t *pd) {
    if (pd->dir_global.empty()) {
        const char *pre = getenv("PASTIX_OUTPUT_DIR");
        std::string tmpl = std::string(pre && *pre ? pre : "pastix") + "-XXXXXX";
        std::vector<char> buf(tmpl.begin(), tmpl.end());
        buf.push_back('\0');
        if (!mkdtemp(buf.data())) {
            perr("cannot create the output directory %s", tmpl.c_str());
            return nullptr;
        }
        pd->dir_global = buf.data();
    }
    return pd->dir_global.c_str();
}

static int order_save_file(pastix_data_t *pd, const pgpu::Order &o) {
    const char *dir = output_dir(pd);
    if (!dir) return PASTIX_ERR_FILE;
    const char *env = getenv("PASTIX_FILE_ORDER");
    const std::string path = std::string(dir) + "/" + (env && *env ? env : "ordergen");
    FILE *f = fopen(path.c_str(), "w");
    if (!f) { perr("cannot write %s", path.c_str()); return PASTIX_ERR_FILE; }
    int rc = order_write(f, o);
    if (fclose(f) != 0 && rc == PASTIX_SUCCESS) rc = PASTIX_ERR_FILE;
    return rc;
}

static int order_load_file(pgpu::Order &o) {
    const char *env = getenv("PASTIX_FILE_ORDER");
    const char *path = env && *env ? env : "ordername";
    FILE *f = fopen(path, "r");
    if (!f) { perr("pastixOrderLoad: cannot open %s", path); return PASTIX_ERR_FILE; }
    int rc = order_read(f, o);
    fclose(f);
    return rc;
}

// pastixOrderLoad (order/order_io.c:132): the ordering file of $PASTIX_FILE_ORDER
// or "ordername" into *ordemesh (arrays allocated here, freed by pastixOrderExit).
extern "C" int pastixOrderLoad(const pastix_data_t *, pastix_order_t *ordemesh) {
    if (!ordemesh) return PASTIX_ERR_BADPARAMETER;
    pgpu::Order o;
    int rc = order_load_file(o);
    if (rc) return rc;
    memset(ordemesh, 0, sizeof(*ordemesh));
    auto dup = [](const std::vector<idx_t> &v) {
        pastix_int_t *p = (pastix_int_t *)malloc(std::max<size_t>(1, v.size()) * sizeof(pastix_int_t));
        if (!v.empty()) memcpy(p, v.data(), v.size() * sizeof(pastix_int_t));
        return p;
    };
    ordemesh->baseval = 0;
    ordemesh->vertnbr = o.n;
    ordemesh->cblknbr = o.cblknbr;
    ordemesh->permtab = dup(o.permtab);
    ordemesh->peritab = dup(o.peritab);
    ordemesh->rangtab = o.rangtab.empty() ? nullptr : dup(o.rangtab);
    ordemesh->treetab = o.treetab.empty() ? nullptr : dup(o.treetab);
    return PASTIX_SUCCESS;
}

// pastixOrderSave (order/order_io.c:296): *ordemesh to "<output dir>/ordergen"
// (or $PASTIX_FILE_ORDER).
extern "C" int pastixOrderSave(pastix_data_t *pd, const pastix_order_t *ordemesh) {
    if (!pd || !ordemesh || !ordemesh->permtab || !ordemesh->rangtab || !ordemesh->treetab || ordemesh->vertnbr < 1)
        return PASTIX_ERR_BADPARAMETER;
    pgpu::Order o;
    const idx_t b = ordemesh->baseval;
    o.n = ordemesh->vertnbr;
    o.cblknbr = ordemesh->cblknbr;
    for (idx_t i = 0; i < o.n; i++) o.permtab.push_back(ordemesh->permtab[i] - b);
    for (idx_t k = 0; k <= o.cblknbr; k++) o.rangtab.push_back(ordemesh->rangtab[k] - b);
    for (idx_t k = 0; k < o.cblknbr; k++) o.treetab.push_back(ordemesh->treetab[k] < 0 ? -1 : ordemesh->treetab[k] - b);
    return order_save_file(pd, o);
}

// ---------------------------------------------------------------------------
// ordering
// ---------------------------------------------------------------------------
extern "C" int pastixOrderGrid(pastix_order_t **myorder, pastix_int_t nx, pastix_int_t ny, pastix_int_t nz) {
    if (!myorder || !*myorder || nx < 1 || ny < 1 || nz < 1) return PASTIX_ERR_BADPARAMETER;
    pgpu::Order o;
    try {
        pgpu::order_grid(o, nx, ny, nz);
    } catch (const std::exception &e) {
        perr("pastixOrderGrid: %s", e.what());
        return PASTIX_ERR_BADPARAMETER;
    }
    pastix_order_t *ord = *myorder;
    memset(ord, 0, sizeof(*ord));
    ord->baseval = 0;
    ord->vertnbr = o.n;
    ord->cblknbr = o.cblknbr;
    auto dup = [](const std::vector<idx_t> &v) {
        pastix_int_t *p = (pastix_int_t *)malloc(std::max<size_t>(1, v.size()) * sizeof(pastix_int_t));
        if (!v.empty()) memcpy(p, v.data(), v.size() * sizeof(pastix_int_t));
        return p;
    };
    ord->permtab = dup(o.permtab);
    ord->peritab = dup(o.peritab);
    ord->rangtab = dup(o.rangtab);
    ord->treetab = dup(o.treetab);
    return PASTIX_SUCCESS;
}

extern "C" void pastixOrderExit(pastix_order_t *o) {
    if (!o) return;
    free(o->permtab);
    free(o->peritab);
    free(o->rangtab);
    free(o->treetab);
    free(o->selevtx);
    free(o->sndetab);
    free(o->peritab_exp);
    memset(o, 0, sizeof(*o));
}

static int check_spm(const spmatrix_t *spm) {
    if (!spm) { perr("spm is NULL"); return PASTIX_ERR_BADPARAMETER; }
    if (spm->fmttype != SpmCSC) { perr("only CSC input is supported"); return PASTIX_ERR_BADPARAMETER; }
    if (spm->mtxtype != SpmGeneral && spm->mtxtype != SpmSymmetric) {
        perr("mtxtype must be SpmGeneral or SpmSymmetric (real arithmetic)");
        return PASTIX_ERR_BADPARAMETER;
    }
    if (spm->dof != 1 && spm->dof != 0) { perr("give dof>1 matrices expanded (dof = 1)"); return PASTIX_ERR_BADPARAMETER; }
    if (spm->n <= 0 || !spm->colptr || (spm->nnz > 0 && !spm->rowptr)) return PASTIX_ERR_BADPARAMETER;
    if (spm->baseval != 0 && spm->baseval != 1) return PASTIX_ERR_BADPARAMETER;
    return PASTIX_SUCCESS;
}

// pastix_subtask_order (order/pastix_subtask_order.c:100): build the graph and
// the ordering.  PastixOrderPersonal uses the given order (grid or user
// permutation); any other value uses the built-in nested dissection of the
// graph, since Scotch and Metis are not part of this library.
extern "C" int pastix_subtask_order(pastix_data_t *pd, const spmatrix_t *spm, pastix_order_t *myorder) {
    if (!pd) return PASTIX_ERR_BADPARAMETER;
    int rc = check_spm(spm);
    if (rc) return rc;
    const idx_t n = spm->n, b = spm->baseval, nnz = spm->colptr[n] - b;
    pd->n = n;
    pd->nnz = nnz;
    pd->mtxtype = spm->mtxtype;
    pd->colptr.assign(n + 1, 0);
    pd->rowind.assign(nnz, 0);
    for (idx_t j = 0; j <= n; j++) pd->colptr[j] = spm->colptr[j] - b;
    for (idx_t e = 0; e < nnz; e++) {
        idx_t r = spm->rowptr[e] - b;
        if (r < 0 || r >= n) { perr("row index out of range"); return PASTIX_ERR_BADPARAMETER; }
        pd->rowind[e] = r;
    }
    for (idx_t j = 0; j < n; j++)
        if (pd->colptr[j + 1] < pd->colptr[j]) return PASTIX_ERR_BADPARAMETER;
    // symmetric graph without the diagonal
    {
        std::vector<idx_t> deg(n + 1, 0);
        for (idx_t j = 0; j < n; j++)
            for (idx_t e = pd->colptr[j]; e < pd->colptr[j + 1]; e++) {
                idx_t i = pd->rowind[e];
                if (i != j) { deg[i + 1]++; deg[j + 1]++; }
            }
        for (idx_t i = 0; i < n; i++) deg[i + 1] += deg[i];
        std::vector<idx_t> adj(deg[n]);
        std::vector<idx_t> pos(deg.begin(), deg.end() - 1);
        for (idx_t j = 0; j < n; j++)
            for (idx_t e = pd->colptr[j]; e < pd->colptr[j + 1]; e++) {
                idx_t i = pd->rowind[e];
                if (i != j) { adj[pos[i]++] = j; adj[pos[j]++] = i; }
            }
        pd->graph.n = n;
        pd->graph.colptr.assign(n + 1, 0);
        pd->graph.rowind.clear();
        pd->graph.rowind.reserve(adj.size());
        for (idx_t i = 0; i < n; i++) {
            auto b0 = adj.begin() + deg[i], b1 = adj.begin() + deg[i + 1];
            std::sort(b0, b1);
            auto e1 = std::unique(b0, b1);
            pd->graph.rowind.insert(pd->graph.rowind.end(), b0, e1);
            pd->graph.colptr[i + 1] = (idx_t)pd->graph.rowind.size();
        }
    }
    pgpu::Order &o = pd->order;
    o = pgpu::Order{};
    idx_t dof = 1;  // > 1: the ordering numbers nodes of dof unknowns each
    const bool personal = pd->iparm[IPARM_ORDERING] == PastixOrderPersonal;
    if (personal && (pd->iparm[IPARM_IO_STRATEGY] & PastixIOLoad)) {
        // the ordering file replaces the personal ordering (order/order_compute_personal.c:71-77)
        rc = order_load_file(o);
        if (rc) return rc;
        if (o.n != n) {
            if (n % o.n != 0) { perr("loaded ordering size mismatch"); return PASTIX_ERR_BADPARAMETER; }
            dof = n / o.n;
        }
        pd->user_order = true;
    } else if (personal && myorder && myorder->permtab) {
        idx_t vn = myorder->vertnbr, ob = myorder->baseval;
        if (vn <= 0 || n % vn != 0) { perr("personal order size mismatch"); return PASTIX_ERR_BADPARAMETER; }
        o.n = vn;
        o.permtab.resize(vn);
        o.peritab.resize(vn);
        for (idx_t i = 0; i < vn; i++) o.permtab[i] = myorder->permtab[i] - ob;
        if (myorder->peritab)
            for (idx_t i = 0; i < vn; i++) o.peritab[i] = myorder->peritab[i] - ob;
        else
            for (idx_t i = 0; i < vn; i++) o.peritab[o.permtab[i]] = i;
        if (myorder->rangtab && myorder->treetab && myorder->cblknbr > 0) {
            o.cblknbr = myorder->cblknbr;
            o.rangtab.resize(o.cblknbr + 1);
            o.treetab.resize(o.cblknbr);
            for (idx_t k = 0; k <= o.cblknbr; k++) o.rangtab[k] = myorder->rangtab[k] - ob;
            for (idx_t k = 0; k < o.cblknbr; k++) o.treetab[k] = myorder->treetab[k] < 0 ? -1 : myorder->treetab[k] - ob;
        }
        dof = n / vn;
        pd->user_order = true;
    } else {
        // identity start; nested dissection of the graph is applied below
        o.n = n;
        o.permtab.resize(n);
        o.peritab.resize(n);
        pgpu::order_nd_graph(o, pd->graph);
        pd->user_order = false;
    }
    // A node ordering of a matrix with dof unknowns per node is analysed on the
    // node graph, as the reference analyses spm->dof > 1 matrices, and expanded
    // to unknowns afterwards.
    pd->dof = dof;
    pd->node_graph = pgpu::Graph{};
    if (dof > 1) pgpu::graph_collapse(pd->graph, dof, pd->node_graph);
    const pgpu::Graph &g = dof > 1 ? pd->node_graph : pd->graph;
    if (o.rangtab.empty() || o.treetab.empty()) {  // order/pastix_subtask_order.c:360-364
        o.rangtab.clear();
        o.treetab.clear();
        o.cblknbr = 0;
        pgpu::order_find_supernodes(o, g);
    }
    // supernodes renumbered by tree level (order/pastix_subtask_order.c:399-401)
    pgpu::order_apply_level_order(o, pd->iparm[IPARM_TASKS2D_LEVEL], pd->iparm[IPARM_TASKS2D_WIDTH]);
    std::string err = pgpu::order_check(o);
    if (!err.empty()) { perr("ordering check failed: %s", err.c_str()); return PASTIX_ERR_BADPARAMETER; }
    if (pd->iparm[IPARM_IO_STRATEGY] & PastixIOSave) {  // order/pastix_subtask_order.c:485
        rc = order_save_file(pd, o);
        if (rc) return rc;
    }
    pd->node_order = pgpu::Order{};
    if (dof > 1) {
        pd->node_order = o;
        pgpu::order_expand_dof(o, dof);
    }
    pd->steps = STEP_INIT | STEP_ORDERING;
    return PASTIX_SUCCESS;
}

static int symbol_save_file(pastix_data_t *pd) {
    const char *dir = output_dir(pd);
    if (!dir) return PASTIX_ERR_FILE;
    const std::string path = std::string(dir) + "/symbgen";
    FILE *f = fopen(path.c_str(), "w");
    if (!f) { perr("cannot write %s", path.c_str()); return PASTIX_ERR_FILE; }
    int rc = symbol_write(f, pd->symbol);
    if (fclose(f) != 0 && rc == PASTIX_SUCCESS) rc = PASTIX_ERR_FILE;
    return rc;
}

extern "C" int pastix_subtask_symbfact(pastix_data_t *pd) {
    if (!pd || !(pd->steps & STEP_ORDERING)) {
        perr("pastix_subtask_symbfact: pastix_subtask_order() has to be called first");
        return PASTIX_ERR_BADPARAMETER;
    }
    double t0 = now_s();
    if (pd->iparm[IPARM_IO_STRATEGY] & PastixIOLoad) {  // symbol/pastix_subtask_symbfact.c:156-163
        FILE *f = fopen("symbname", "r");
        if (!f) { perr("pastix_subtask_symbfact: cannot open symbname"); return PASTIX_ERR_FILE; }
        int rc = symbol_read(f, pd->symbol);
        fclose(f);
        if (rc) return rc;
        // structural checks before anything walks the loaded structure
        std::string err = pgpu::symbol_check(pd->symbol);
        if (!err.empty()) {
            perr("pastix_subtask_symbfact: symbol file fails its checks: %s", err.c_str());
            return PASTIX_ERR_FILE;
        }
        if (pd->symbol.nodenbr != pd->order.n) {
            perr("pastix_subtask_symbfact: the symbol file has %lld columns, the matrix %lld",
                 (long long)pd->symbol.nodenbr, (long long)pd->order.n);
            return PASTIX_ERR_BADPARAMETER;
        }
    } else {
        pgpu::symbol_fax(pd->symbol, pd->graph, pd->order);
    }
    if (pd->iparm[IPARM_IO_STRATEGY] & PastixIOSave) {  // symbol/pastix_subtask_symbfact.c:275-285
        int rc = symbol_save_file(pd);
        if (rc) return rc;
    }
    pd->dparm[DPARM_SYMBFACT_TIME] = now_s() - t0;
    pd->steps |= STEP_SYMBFACT;
    return PASTIX_SUCCESS;
}

// pastix_subtask_reordering (symbol/pastix_subtask_reordering.c:60): the rows
// of every supernode reordered to group the bloks that face it, then the block
// symbolic factorization again with the new ordering.
extern "C" int pastix_subtask_reordering(pastix_data_t *pd) {
    if (!pd || !(pd->steps & STEP_SYMBFACT)) return PASTIX_ERR_BADPARAMETER;
    double t0 = now_s();
    // a loaded analysis (PastixIOLoad) was saved after its reordering
    if (!(pd->iparm[IPARM_IO_STRATEGY] & PastixIOLoad) && (idx_t)pd->order.treetab.size() == pd->symbol.cblknbr() &&
        pd->graph.n == pd->order.n && (pd->dof == 1 || pd->node_order.n * pd->dof == pd->order.n)) {
        const idx_t split = pd->iparm[IPARM_REORDERING_SPLIT], stop = pd->iparm[IPARM_REORDERING_STOP];
        if (pd->dof > 1) {  // rows of nodes, on the node structure
            pgpu::Symbol nsym;
            pgpu::symbol_fax(nsym, pd->node_graph, pd->node_order);
            pgpu::symbol_reorder_rows(nsym, pd->node_order, split, stop);
            pd->order = pd->node_order;
            pgpu::order_expand_dof(pd->order, pd->dof);
        } else {
            pgpu::symbol_reorder_rows(pd->symbol, pd->order, split, stop);
        }
        if (pd->iparm[IPARM_IO_STRATEGY] & PastixIOSave) {
            int rc = order_save_file(pd, pd->dof > 1 ? pd->node_order : pd->order);
            if (rc) return rc;
        }
        pgpu::symbol_fax(pd->symbol, pd->graph, pd->order);
        if (pd->iparm[IPARM_IO_STRATEGY] & PastixIOSave) {  // the symbolic step runs again and saves
            int rc = symbol_save_file(pd);
            if (rc) return rc;
        }
    }
    pd->dparm[DPARM_REORDER_TIME] = now_s() - t0;
    return PASTIX_SUCCESS;
}

// Host-side construction of the value maps and of the launch lists.
static int build_maps_and_lists(pastix_data_t *pd) {
    const pgpu::Solver &sv = pd->solver;
    const idx_t n = pd->n, nnz = pd->nnz;
    const auto &perm = pd->order.permtab;
    const int fk = fact_kind(pd);
    const bool sym = pd->mtxtype == SpmSymmetric;
    // column -> cblk
    std::vector<int> col2cb(n);
    for (idx_t k = 0; k < sv.cblknbr; k++)
        for (idx_t c = sv.cb_fcol[k]; c <= sv.cb_lcol[k]; c++) col2cb[c] = (int)k;
    auto rowpos = [&](idx_t k, idx_t r) -> idx_t {
        idx_t lo = sv.cb_fblok[k], hi = sv.cb_fblok[k + 1] - 1;
        while (lo < hi) {
            idx_t mid = (lo + hi + 1) / 2;
            if (sv.bk_frow[mid] <= r) lo = mid; else hi = mid - 1;
        }
        if (r < sv.bk_frow[lo] || r > sv.bk_lrow[lo]) return -1;
        return sv.bk_rowoff[lo] + (r - sv.bk_frow[lo]);
    };
    auto coefpos = [&](idx_t r, idx_t c) -> int64_t {  // lower position (r >= c) in the L-shaped panel
        idx_t k = col2cb[c];
        idx_t rp = rowpos(k, r);
        if (rp < 0) return -2;
        return sv.cb_coef[k] + rp + (c - sv.cb_fcol[k]) * sv.cb_stride[k];
    };
    pd->lmap.assign(nnz, -1);
    pd->umap.clear();
    if (fk == pgpu::FACT_GETRF) pd->umap.assign(nnz, -1);
    pd->e_row.resize(nnz);
    pd->e_col.resize(nnz);
    std::vector<std::pair<idx_t, idx_t>> ent;  // (permuted row, permuted col) of the full matrix, with source
    std::vector<int64_t> src;
    ent.reserve(sym ? 2 * nnz : nnz);
    src.reserve(sym ? 2 * nnz : nnz);
    for (idx_t j = 0; j < n; j++) {
        for (idx_t e = pd->colptr[j]; e < pd->colptr[j + 1]; e++) {
            idx_t i = pd->rowind[e];
            pd->e_row[e] = (int)i;
            pd->e_col[e] = (int)j;
            idx_t pi = perm[i], pj = perm[j];
            ent.emplace_back(pi, pj);
            src.push_back(e);
            if (sym && pi != pj) { ent.emplace_back(pj, pi); src.push_back(e); }
            idx_t r = std::max(pi, pj), c = std::min(pi, pj);
            if (sym) {
                int64_t p = coefpos(r, c);
                if (p == -2) { perr("entry outside the symbolic structure"); return PASTIX_ERR_INTERNAL; }
                pd->lmap[e] = p;
                if (fk == pgpu::FACT_GETRF && pi != pj) pd->umap[e] = p;
            } else if (pi >= pj) {
                int64_t p = coefpos(pi, pj);
                if (p == -2) { perr("entry outside the symbolic structure"); return PASTIX_ERR_INTERNAL; }
                pd->lmap[e] = p;
            } else if (fk == pgpu::FACT_GETRF) {
                int64_t p = coefpos(pj, pi);
                if (p == -2) { perr("entry outside the symbolic structure"); return PASTIX_ERR_INTERNAL; }
                pd->umap[e] = p;
            }
        }
    }
    // CSR of the permuted full matrix (counting sort by row, then by column)
    idx_t fn = (idx_t)ent.size();
    pd->csr_nnz = fn;
    if (fn >= (idx_t)INT32_MAX) { perr("matrix too large for 32-bit CSR"); return PASTIX_ERR_INTEGER_TYPE; }
    std::vector<idx_t> order(fn);
    {
        std::vector<idx_t> cnt(n + 1, 0), tmp(fn);
        for (idx_t p = 0; p < fn; p++) cnt[ent[p].second + 1]++;
        for (idx_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
        for (idx_t p = 0; p < fn; p++) tmp[cnt[ent[p].second]++] = p;
        std::fill(cnt.begin(), cnt.end(), 0);
        for (idx_t p = 0; p < fn; p++) cnt[ent[p].first + 1]++;
        for (idx_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
        pd->csr_rowptr.assign(n + 1, 0);
        for (idx_t i = 0; i <= n; i++) pd->csr_rowptr[i] = (int)cnt[i];
        for (idx_t q = 0; q < fn; q++) {
            idx_t p = tmp[q];
            order[cnt[ent[p].first]++] = p;
        }
    }
    pd->csr_col.resize(fn);
    pd->csr_src.resize(fn);
    for (idx_t q = 0; q < fn; q++) {
        pd->csr_col[q] = (int)ent[order[q]].second;
        pd->csr_src[q] = src[order[q]];
        if (q > 0 && pd->csr_col[q] == pd->csr_col[q - 1]) {
            idx_t row = std::upper_bound(pd->csr_rowptr.begin(), pd->csr_rowptr.end(), (int)q) - pd->csr_rowptr.begin() - 1;
            if (pd->csr_rowptr[row] != (int)q) {
                perr("duplicate entry in the matrix (symmetric matrices store one triangle)");
                return PASTIX_ERR_BADPARAMETER;
            }
        }
    }

    // ---- launch lists per level ----
    pd->levels.assign(sv.nlevels, LevelLists{});
    pd->small_list.clear(); pd->large_list.clear(); pd->level_cblks.clear();
    pd->trsm_tiles.clear(); pd->solve_tiles.clear(); pd->upd_tiles.clear(); pd->upd_big_tiles.clear();
    pd->upd_tc_tiles.clear();
    pd->upd_tiles32.clear();
    // exclusive tasks: dst targeted by a single source in the level
    pd->tasks.resize(sv.tasks.size());
    {
        // number of distinct sources writing each dst within a level
        std::vector<int> last_src(sv.cblknbr, -1), nsrc(sv.cblknbr, 0);
        for (idx_t l = 0; l < sv.nlevels; l++) {
            for (idx_t t = sv.lvl_task_ptr[l]; t < sv.lvl_task_ptr[l + 1]; t++) {
                const auto &tk = sv.tasks[t];
                if (last_src[tk.dst] != (int)tk.src) {
                    nsrc[tk.dst]++;
                    last_src[tk.dst] = (int)tk.src;
                }
            }
            for (idx_t t = sv.lvl_task_ptr[l]; t < sv.lvl_task_ptr[l + 1]; t++) {
                const auto &tk = sv.tasks[t];
                pgpu::TaskDev d;
                d.src = (int)tk.src; d.dst = (int)tk.dst; d.row0 = (int)tk.row0; d.n = (int)tk.n; d.m = (int)tk.m;
                d.excl = nsrc[tk.dst] == 1 ? 1 : 0;
                pd->tasks[t] = d;
            }
            for (idx_t t = sv.lvl_task_ptr[l]; t < sv.lvl_task_ptr[l + 1]; t++) {
                last_src[sv.tasks[t].dst] = -1;
                nsrc[sv.tasks[t].dst] = 0;
            }
        }
    }
    const int SR = pgpu::solve_rows_per_tile();
    pd->cb_dinv.assign(sv.cblknbr, -1);
    pd->dinv_total = 0;
    // BF16 images for the tcgen05 updates (FP32 factors): sources of big tasks
    pd->sp_off.assign(sv.cblknbr, -1);
    pd->split_total = 0;
    pd->split_slabs.clear();
    for (const auto &tk : sv.tasks) {
        const idx_t K = sv.cb_lcol[tk.src] - sv.cb_fcol[tk.src] + 1;
        if (K >= pd->tune_tc_k && K * sv.cb_stride[tk.src] > SMALL_PANEL_ELEMS && pd->sp_off[tk.src] < 0)
            pd->sp_off[tk.src] = 0;
    }
    for (idx_t k = 0; k < sv.cblknbr; k++) {
        if (pd->sp_off[k] < 0) continue;
        pd->sp_off[k] = pd->split_total;
        pd->split_total += pgpu::split_image_bytes((int)(sv.cb_lcol[k] - sv.cb_fcol[k] + 1), (int)sv.cb_stride[k]);
    }
    // FP32 TRSM by GEMM with the triangular inverse: wide cblks with rows below and a BF16 image
    pd->ti_off.assign(sv.cblknbr, -1);
    pd->ti_img.assign(sv.cblknbr, -1);
    pd->tinv_total = pd->timg_total = 0;
    pd->dense_slabs.clear();
    pd->trsm_tc_tiles.clear();
    pd->trsm_tiles32.clear();
    const int nsides = (fk == pgpu::FACT_GETRF) ? 2 : 1;
    for (idx_t k = 0; k < sv.cblknbr; k++) {
        const idx_t nc = sv.cb_lcol[k] - sv.cb_fcol[k] + 1, st = sv.cb_stride[k];
        if (pd->sp_off[k] < 0 || st <= nc || st * nc <= SMALL_PANEL_ELEMS || nc > 32 * pgpu::trinv_max_blocks())
            continue;
        pd->ti_off[k] = pd->tinv_total;
        pd->ti_img[k] = pd->timg_total;
        pd->tinv_total += (int64_t)nsides * nc * nc;
        pd->timg_total += (int64_t)nsides * pgpu::split_image_bytes((int)nc, (int)nc);
    }
    for (idx_t l = 0; l < sv.nlevels; l++) {
        LevelLists &L = pd->levels[l];
        L.small0 = (int)pd->small_list.size();
        L.large0 = (int)pd->large_list.size();
        L.trsm0 = (int)pd->trsm_tiles.size();
        L.cb0 = (int)pd->level_cblks.size();
        L.st0 = (int)pd->solve_tiles.size();
        L.maxnc = 1;
        L.trsm_maxnc = 0;
        L.diag_maxnc = 0;
        L.small_smem_elems = L.diag_smem_elems = L.trsm_smem_elems = 0;
        L.small_maxst = 0;
        for (idx_t p = sv.lvl_ptr[l]; p < sv.lvl_ptr[l + 1]; p++) {
            idx_t k = sv.lvl_cblk[p];
            idx_t nc = sv.cb_lcol[k] - sv.cb_fcol[k] + 1, st = sv.cb_stride[k];
            L.maxnc = std::max<int>(L.maxnc, (int)nc);
            pd->level_cblks.push_back((int)k);
            if (st * nc <= SMALL_PANEL_ELEMS) {
                pd->small_list.push_back((int)k);
                L.small_smem_elems = std::max<size_t>(L.small_smem_elems, (size_t)(st * nc) * (fk == pgpu::FACT_GETRF ? 2 : 1));
                L.small_maxst = std::max<int>(L.small_maxst, (int)st);
            } else {
                pd->large_list.push_back((int)k);
                pd->cb_dinv[k] = pd->dinv_total;
                L.diag_maxnc = std::max<int>(L.diag_maxnc, (int)nc);
                pd->dinv_total += pgpu::dinv_elems((int)nc, fk);
                L.diag_smem_elems = std::max<size_t>(L.diag_smem_elems, (size_t)pgpu::diag_smem_elems((int)nc, fk));
                int bm = pgpu::trsm_tile_rows((int)nc);
                for (idx_t r = nc; r < st; r += bm) pd->trsm_tiles.push_back(pgpu::RowTile{(int)k, (int)r});
                if (st > nc) L.trsm_smem_elems = std::max<size_t>(L.trsm_smem_elems, (size_t)pgpu::trsm_smem_elems((int)nc));
                if (st > nc) L.trsm_maxnc = std::max<int>(L.trsm_maxnc, (int)nc);
            }
            for (idx_t r = nc; r < st; r += SR) pd->solve_tiles.push_back(pgpu::RowTile{(int)k, (int)r});
        }
        L.spl0 = (int)pd->split_slabs.size();
        for (idx_t p = sv.lvl_ptr[l]; p < sv.lvl_ptr[l + 1]; p++) {
            idx_t k = sv.lvl_cblk[p];
            if (pd->sp_off[k] < 0) continue;
            for (idx_t r = 0; r < sv.cb_stride[k]; r += 128) pd->split_slabs.push_back(pgpu::SplitSlab{(int)k, (int)r});
        }
        L.spl1 = (int)pd->split_slabs.size();
        L.tt0 = (int)pd->trsm_tc_tiles.size();
        L.ds0 = (int)pd->dense_slabs.size();
        L.tr32_0 = (int)pd->trsm_tiles32.size();
        L.ti_maxnzb = 0;
        for (idx_t p = sv.lvl_ptr[l]; p < sv.lvl_ptr[l + 1]; p++) {
            idx_t k = sv.lvl_cblk[p];
            const idx_t nc = sv.cb_lcol[k] - sv.cb_fcol[k] + 1, st = sv.cb_stride[k];
            if (st * nc <= SMALL_PANEL_ELEMS || st <= nc) continue;
            if (pd->ti_off[k] < 0) {
                for (idx_t r = nc; r < st; r += pgpu::trsm_tile_rows((int)nc))
                    pd->trsm_tiles32.push_back(pgpu::RowTile{(int)k, (int)r});
                continue;
            }
            L.ti_maxnzb = std::max<int>(L.ti_maxnzb, (int)((nc + 31) / 32));
            const idx_t mt = (nc % 8 + (st - nc) + 127) / 128, nt = (nc + 127) / 128;
            for (int side = 0; side < nsides; side++) {
                for (idx_t a = 0; a < mt; a++)
                    for (idx_t c = 0; c < nt; c++) pd->trsm_tc_tiles.push_back(pgpu::UpdTile{(int)k, (int)a, (int)c, side});
                const int64_t src = pd->ti_off[k] + (int64_t)side * nc * nc;
                const int64_t img = pd->ti_img[k] + (int64_t)side * pgpu::split_image_bytes((int)nc, (int)nc);
                for (idx_t r = 0; r < nc; r += 128)
                    pd->dense_slabs.push_back(pgpu::DenseSlab{src, img, (int)nc, (int)nc, (int)nc, (int)r});
            }
        }
        L.ntinv = 0;
        for (int i = L.large0; i < (int)pd->large_list.size(); i++) L.ntinv += pd->ti_off[pd->large_list[i]] >= 0;
        L.tt1 = (int)pd->trsm_tc_tiles.size();
        L.ds1 = (int)pd->dense_slabs.size();
        L.tr32_1 = (int)pd->trsm_tiles32.size();
        L.small1 = (int)pd->small_list.size();
        L.large1 = (int)pd->large_list.size();
        L.trsm1 = (int)pd->trsm_tiles.size();
        L.cb1 = (int)pd->level_cblks.size();
        L.st1 = (int)pd->solve_tiles.size();
        L.upd0 = (int)pd->upd_tiles.size();
        L.updb0 = (int)pd->upd_big_tiles.size();
        L.updt0 = (int)pd->upd_tc_tiles.size();
        L.upds0 = (int)pd->upd_tiles32.size();
        std::vector<pgpu::UpdTile> tc_far, s32_far;  // tiles whose target is two or more levels up
        for (idx_t t = sv.lvl_task_ptr[l]; t < sv.lvl_task_ptr[l + 1]; t++) {
            const auto &tk = sv.tasks[t];
            const idx_t K = sv.cb_lcol[tk.src] - sv.cb_fcol[tk.src] + 1;
            if (K * sv.cb_stride[tk.src] <= SMALL_PANEL_ELEMS) continue;  // done by k_panel_small
            const bool big = tk.n >= pd->tune_dmma_n && K >= pd->tune_dmma_k;  // FP64: DMMA tiles
            const bool tc = K >= pd->tune_tc_k;                                // FP32: tcgen05 tiles
            const idx_t BM = big ? 128 : 64, BN = 64;
            auto &list = big ? pd->upd_big_tiles : pd->upd_tiles;
            for (int side = 0; side < (fk == pgpu::FACT_GETRF ? 2 : 1); side++) {
                idx_t M = tk.m - (side ? tk.n : 0);
                if (M <= 0) continue;
                idx_t mt = (M + BM - 1) / BM, ntl = (tk.n + BN - 1) / BN;
                for (idx_t a = 0; a < mt; a++)
                    for (idx_t c = 0; c < ntl; c++) {
                        // symmetric kinds: skip tiles strictly above the diagonal of the square part
                        if (fk != pgpu::FACT_GETRF && (a + 1) * BM <= c * BN) continue;
                        list.push_back(pgpu::UpdTile{(int)t, (int)a, (int)c, side});
                    }
                const bool near = sv.cb_level[tk.dst] == (idx_t)l + 1;
                if (!tc) {  // FP32 tasks with a narrow source: SIMT 64 x 64 tiles
                    const idx_t mt3 = (M + 63) / 64, nt3 = (tk.n + 63) / 64;
                    for (idx_t a = 0; a < mt3; a++)
                        for (idx_t c = 0; c < nt3; c++) {
                            if (fk != pgpu::FACT_GETRF && (a + 1) * 64 <= c * 64) continue;
                            (near ? pd->upd_tiles32 : s32_far).push_back(pgpu::UpdTile{(int)t, (int)a, (int)c, side});
                        }
                }
                if (tc) {  // tcgen05 tiles (FP32 factors): 128-row windows aligned to groups of 8 rows
                    const idx_t TB = 128;
                    const idx_t ra = tk.row0 + (side ? tk.n : 0);
                    const idx_t mt2 = (ra % 8 + M + TB - 1) / TB, nt2 = (tk.row0 % 8 + tk.n + TB - 1) / TB;
                    for (idx_t a = 0; a < mt2; a++)
                        for (idx_t c = 0; c < nt2; c++) {
                            if (fk != pgpu::FACT_GETRF && (a + 1) * TB <= c * TB) continue;
                            (near ? pd->upd_tc_tiles : tc_far).push_back(pgpu::UpdTile{(int)t, (int)a, (int)c, side});
                        }
                }
            }
        }
        L.upd1 = (int)pd->upd_tiles.size();
        L.updb1 = (int)pd->upd_big_tiles.size();
        L.updtn = (int)pd->upd_tc_tiles.size();
        L.updsn = (int)pd->upd_tiles32.size();
        pd->upd_tc_tiles.insert(pd->upd_tc_tiles.end(), tc_far.begin(), tc_far.end());
        pd->upd_tiles32.insert(pd->upd_tiles32.end(), s32_far.begin(), s32_far.end());
        L.updt1 = (int)pd->upd_tc_tiles.size();
        L.upds1 = (int)pd->upd_tiles32.size();
    }
    return PASTIX_SUCCESS;
}

// pastix_subtask_blend (blend/pastix_subtask_blend.c:121): split, solver
// structure, schedule.
extern "C" int pastix_subtask_blend(pastix_data_t *pd) {
    if (!pd || !(pd->steps & STEP_SYMBFACT)) {
        perr("pastix_subtask_blend: pastix_subtask_symbfact() has to be called first");
        return PASTIX_ERR_BADPARAMETER;
    }
    double t0 = now_s();
    idx_t bmin = pd->iparm[IPARM_MIN_BLOCKSIZE], bmax = pd->iparm[IPARM_MAX_BLOCKSIZE];
    if (bmin > bmax || bmin < 1) { perr("IPARM_MIN_BLOCKSIZE > IPARM_MAX_BLOCKSIZE"); return PASTIX_ERR_BADPARAMETER; }
    // the wide-cblk kernels keep a (32 x width) strip per operand in shared memory
    if (bmax > 384) { perr("IPARM_MAX_BLOCKSIZE above 384 is not supported by the GPU kernels"); return PASTIX_ERR_BADPARAMETER; }
    // The reference splits the supernodes of a dof > 1 matrix on its node
    // symbol, widths counted in nodes (blend/splitsymbol.c:78-102 on the symbol
    // before the expansion of blend/solver_matrix_gen.c).  That is done here
    // whenever the expanded widths fit the kernels (IPARM_MAX_BLOCKSIZE * dof
    // <= 384); otherwise the split counts unknowns, so that no cblk is wider
    // than IPARM_MAX_BLOCKSIZE unknowns.
    if (pd->dof > 1 && bmax * pd->dof <= 384 && pd->node_order.n * pd->dof == pd->order.n &&
        !(pd->iparm[IPARM_IO_STRATEGY] & PastixIOLoad)) {
        pgpu::Symbol nsym;
        pgpu::symbol_fax(nsym, pd->node_graph, pd->node_order);
        pgpu::symbol_split(nsym, bmin, bmax);
        pgpu::symbol_expand(nsym, pd->dof, pd->symbol);
    } else {
        pgpu::symbol_split(pd->symbol, bmin, bmax);
    }
    std::string err = pgpu::symbol_check(pd->symbol);
    if (!err.empty()) { perr("symbol check failed: %s", err.c_str()); return PASTIX_ERR_INTERNAL; }
    pd->factotype = (int)pd->iparm[IPARM_FACTORIZATION];
    int fk = fact_kind(pd);
    pgpu::solver_build(pd->solver, pd->symbol, fk);
    int rc = build_maps_and_lists(pd);
    if (rc) return rc;
    pd->dparm[DPARM_FACT_THFLOPS] = pd->solver.thflops;
    pd->iparm[IPARM_NNZEROS] = pd->solver.nnzl * (fk == pgpu::FACT_GETRF ? 2 : 1);
    pd->dparm[DPARM_BLEND_TIME] = now_s() - t0;
    pd->steps |= STEP_ANALYSE;
    pd->dev.ready = false;  // structure changed: device copy must be rebuilt
    return PASTIX_SUCCESS;
}

extern "C" int pastix_task_analyze(pastix_data_t *pd, const spmatrix_t *spm) {
    if (!pd) return PASTIX_ERR_BADPARAMETER;
    double t0 = now_s();
    int rc = pastix_subtask_order(pd, spm, nullptr);
    if (rc) return rc;
    rc = pastix_subtask_symbfact(pd);
    if (rc) return rc;
    rc = pastix_subtask_reordering(pd);
    if (rc) return rc;
    rc = pastix_subtask_blend(pd);
    pd->dparm[DPARM_ANALYZE_TIME] = now_s() - t0;
    return rc;
}

extern "C" int pgpu_solver_info(const pastix_data_t *pd, pgpu_solver_info_t *info) {
    if (!pd || !info || !(pd->steps & STEP_ANALYSE)) return PASTIX_ERR_BADPARAMETER;
    const pgpu::Solver &sv = pd->solver;
    info->n = sv.n;
    info->cblknbr = sv.cblknbr;
    info->bloknbr = sv.bloknbr;
    info->coefnbr = sv.coefnbr;
    info->nlevels = sv.nlevels;
    info->ntasks = (pastix_int_t)sv.tasks.size();
    info->cb_fcol = sv.cb_fcol.data();
    info->cb_lcol = sv.cb_lcol.data();
    info->cb_fblok = sv.cb_fblok.data();
    info->cb_stride = sv.cb_stride.data();
    info->cb_coef = sv.cb_coef.data();
    info->cb_level = sv.cb_level.data();
    info->bk_frow = sv.bk_frow.data();
    info->bk_lrow = sv.bk_lrow.data();
    info->bk_fcblk = sv.bk_fcblk.data();
    info->bk_lcblk = sv.bk_lcblk.data();
    info->bk_rowoff = sv.bk_rowoff.data();
    info->permtab = pd->order.permtab.data();
    info->peritab = pd->order.peritab.data();
    info->thflops = sv.thflops;
    return PASTIX_SUCCESS;
}

// ---------------------------------------------------------------------------
// device residency
// ---------------------------------------------------------------------------
template <typename X>
static std::vector<int> to_i32(const std::vector<X> &v) {
    std::vector<int> r(v.size());
    for (size_t i = 0; i < v.size(); i++) r[i] = (int)v[i];
    return r;
}

static int device_setup(pastix_data_t *pd) {
    Device &d = pd->dev;
    if (d.ready) { CUDA_TRY(cudaSetDevice(d.dev)); return PASTIX_SUCCESS; }
    if (d.stream) CUDA_TRY(cudaStreamSynchronize(d.stream));
    pd->graphs.clear();  // captured launches name the old structure
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        perr("no CUDA device available: the numerical phase runs on the GPU only");
        return PASTIX_ERR_INTERNAL;
    }
    if (d.dev < 0) CUDA_TRY(cudaGetDevice(&d.dev));
    CUDA_TRY(cudaSetDevice(d.dev));
    if (!d.stream) CUDA_TRY(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
    if (!d.side) CUDA_TRY(cudaStreamCreateWithFlags(&d.side, cudaStreamNonBlocking));
    while (d.ev_chain.size() < pd->levels.size()) {
        cudaEvent_t a, b;
        CUDA_TRY(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
        d.ev_chain.push_back(a);
        d.ev_rest.push_back(b);
    }
    cudaStream_t st = d.stream;
    const pgpu::Solver &sv = pd->solver;
    if (sv.n >= INT32_MAX || (idx_t)sv.rowidx.size() >= INT32_MAX) { perr("problem too large"); return PASTIX_ERR_INTEGER_TYPE; }
    CUDA_TRY(d.cb_fcol.upload(to_i32(sv.cb_fcol), st));
    CUDA_TRY(d.cb_lcol.upload(to_i32(sv.cb_lcol), st));
    CUDA_TRY(d.cb_stride.upload(to_i32(sv.cb_stride), st));
    CUDA_TRY(d.cb_fblok.upload(to_i32(sv.cb_fblok), st));
    CUDA_TRY(d.bk_frow.upload(to_i32(sv.bk_frow), st));
    CUDA_TRY(d.bk_lrow.upload(to_i32(sv.bk_lrow), st));
    CUDA_TRY(d.bk_rowoff.upload(to_i32(sv.bk_rowoff), st));
    CUDA_TRY(d.bk_fcblk.upload(to_i32(sv.bk_fcblk), st));
    CUDA_TRY(d.rowidx.upload(to_i32(sv.rowidx), st));
    std::vector<int64_t> coef(sv.cb_coef.begin(), sv.cb_coef.end()), ridx(sv.cb_rowidx.begin(), sv.cb_rowidx.end());
    CUDA_TRY(d.cb_coef.upload(coef, st));
    CUDA_TRY(d.cb_rowidx.upload(ridx, st));
    CUDA_TRY(d.cb_dinv.upload(pd->cb_dinv, st));
    CUDA_TRY(d.tasks.upload(pd->tasks, st));
    CUDA_TRY(d.small_list.upload(pd->small_list, st));
    CUDA_TRY(d.large_list.upload(pd->large_list, st));
    CUDA_TRY(d.level_cblks.upload(pd->level_cblks, st));
    CUDA_TRY(d.trsm_tiles.upload(pd->trsm_tiles, st));
    CUDA_TRY(d.solve_tiles.upload(pd->solve_tiles, st));
    CUDA_TRY(d.upd_tiles.upload(pd->upd_tiles, st));
    CUDA_TRY(d.upd_big_tiles.upload(pd->upd_big_tiles, st));
    CUDA_TRY(d.upd_tc_tiles.upload(pd->upd_tc_tiles, st));
    CUDA_TRY(d.upd_tiles32.upload(pd->upd_tiles32, st));
    CUDA_TRY(d.sp_off.upload(pd->sp_off, st));
    CUDA_TRY(d.ti_off.upload(pd->ti_off, st));
    CUDA_TRY(d.ti_img.upload(pd->ti_img, st));
    if (!pd->dense_slabs.empty()) CUDA_TRY(d.dense_slabs.upload(pd->dense_slabs, st));
    if (!pd->trsm_tc_tiles.empty()) CUDA_TRY(d.trsm_tc_tiles.upload(pd->trsm_tc_tiles, st));
    if (!pd->trsm_tiles32.empty()) CUDA_TRY(d.trsm_tiles32.upload(pd->trsm_tiles32, st));
    if (!pd->split_slabs.empty()) CUDA_TRY(d.split_slabs.upload(pd->split_slabs, st));
    CUDA_TRY(d.lmap.upload(pd->lmap, st));
    if (!pd->umap.empty()) CUDA_TRY(d.umap.upload(pd->umap, st));
    else d.umap.reset();
    CUDA_TRY(d.csr_src.upload(pd->csr_src, st));
    CUDA_TRY(d.csr_rowptr.upload(pd->csr_rowptr, st));
    {
        std::vector<int> part;
        pgpu::spmv_partition((int)pd->n, pd->csr_rowptr.data(), part);
        d.spmv_nblocks = (int)part.size() - 1;
        CUDA_TRY(d.spmv_part.upload(part, st));
    }
    CUDA_TRY(d.csr_col.upload(pd->csr_col, st));
    CUDA_TRY(d.e_row.upload(pd->e_row, st));
    CUDA_TRY(d.e_col.upload(pd->e_col, st));
    std::vector<int64_t> perm(pd->order.permtab.begin(), pd->order.permtab.end());
    CUDA_TRY(d.perm.upload(perm, st));
    CUDA_TRY(d.vals.alloc(std::max<idx_t>(1, pd->nnz)));
    CUDA_TRY(d.csr_val.alloc(std::max<idx_t>(1, pd->csr_nnz)));
    CUDA_TRY(d.counters.alloc(4));
    CUDA_TRY(d.queues.alloc(std::max<size_t>(1, 3 * pd->levels.size())));
    CUDA_TRY(d.dcscr.alloc(pgpu::diag_cluster_scratch_doubles()));
    CUDA_TRY(d.crit.alloc(1));
    CUDA_TRY(cudaMemsetAsync(d.counters.p, 0, 4 * sizeof(int), st));
    CUDA_TRY(d.part.alloc(pgpu::reduce_partials()));
    CUDA_TRY(d.scal.alloc(64));
    pgpu::DevStruct &s = d.ds;
    s.n = (int)sv.n;
    s.cblknbr = (int)sv.cblknbr;
    s.cb_fcol = d.cb_fcol.p; s.cb_lcol = d.cb_lcol.p; s.cb_stride = d.cb_stride.p; s.cb_fblok = d.cb_fblok.p;
    s.cb_coef = d.cb_coef.p; s.cb_rowidx = d.cb_rowidx.p; s.cb_dinv = d.cb_dinv.p;
    s.bk_frow = d.bk_frow.p; s.bk_lrow = d.bk_lrow.p; s.bk_rowoff = d.bk_rowoff.p; s.bk_fcblk = d.bk_fcblk.p;
    s.rowidx = d.rowidx.p;
    s.tasks = d.tasks.p;
    static bool attrs = false;
    if (!attrs) {
        const size_t mx = 220 * 1024;
        CUDA_TRY((pgpu::set_smem_attrs<double, pgpu::FACT_POTRF>(mx, mx, mx)));
        CUDA_TRY((pgpu::set_smem_attrs<double, pgpu::FACT_SYTRF>(mx, mx, mx)));
        CUDA_TRY((pgpu::set_smem_attrs<double, pgpu::FACT_GETRF>(mx, mx, mx)));
        CUDA_TRY((pgpu::set_smem_attrs<float, pgpu::FACT_POTRF>(mx, mx, mx)));
        CUDA_TRY((pgpu::set_smem_attrs<float, pgpu::FACT_SYTRF>(mx, mx, mx)));
        CUDA_TRY((pgpu::set_smem_attrs<float, pgpu::FACT_GETRF>(mx, mx, mx)));
        attrs = true;
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    d.ready = true;
    return PASTIX_SUCCESS;
}

// ---------------------------------------------------------------------------
// numerical factorization
// ---------------------------------------------------------------------------
template <typename T, int F>
static int run_factor(pastix_data_t *pd, double criterion) {
    Device &d = pd->dev;
    cudaStream_t st = d.stream;
    T *L = reinterpret_cast<T *>(d.Lc.p);
    T *U = reinterpret_cast<T *>(d.Uc.p);
    T *Dinv = reinterpret_cast<T *>(d.dinv.p);
    (void)criterion;  // copied to d.crit by the caller
    pgpu::FactParams fp{d.crit.p, d.counters.p, d.counters.p + 1, d.dcscr.p};
    // FP32: the updates of level l whose targets sit two or more levels up run on a
    // second stream and overlap level l + 1 (all FP32 update writes are reductions)
    // (the profiled pass keeps one stream so that each class's events time it alone)
    const bool two = sizeof(T) == 4 && !pd->prof_on;
    const cudaStream_t sd = two ? d.side : st;
    // FP32 (launched kernel by kernel, not as a graph): each launch of the level
    // chain overlaps the end of the kernel ahead of it (programmatic dependent launch)
    struct PdlScope {
        explicit PdlScope(bool on) { pgpu::set_pdl(on); }
        ~PdlScope() { pgpu::set_pdl(false); }
    } pdl_scope(two);
    if constexpr (sizeof(T) == 4)
        CUDA_TRY(cudaMemsetAsync(d.queues.p, 0, 3 * pd->levels.size() * sizeof(int), st));
    if (two) {
        CUDA_TRY(cudaEventRecord(d.ev_chain[0], st));
        CUDA_TRY(cudaStreamWaitEvent(d.side, d.ev_chain[0], 0));
    }
    for (size_t l = 0; l < pd->levels.size(); l++) {
        const LevelLists &lv = pd->levels[l];
        if (two && l >= 2) CUDA_TRY(cudaStreamWaitEvent(st, d.ev_rest[l - 2], 0));
        launch_cls(pd, PC_PANEL_SMALL, lv.small1 - lv.small0, [&] {
            pgpu::launch_panel_small<T, F>(d.ds, d.small_list.p + lv.small0, lv.small1 - lv.small0,
                                           (size_t)pgpu::panel_small_bytes((long long)lv.small_smem_elems,
                                                                           (int)sizeof(T), lv.small_maxst),
                                           L, U, fp, st);
        });
        launch_cls(pd, PC_DIAG_LARGE, lv.large1 - lv.large0, [&] {
            pgpu::launch_diag_large<T, F>(d.ds, d.large_list.p + lv.large0, lv.large1 - lv.large0, lv.diag_maxnc,
                                          lv.diag_smem_elems * sizeof(T), L, U, Dinv, fp, st);
        });
        if constexpr (sizeof(T) == 8) {
            launch_cls(pd, PC_TRSM, lv.trsm1 - lv.trsm0, [&] {
                pgpu::launch_trsm<T, F>(d.ds, d.trsm_tiles.p + lv.trsm0, lv.trsm1 - lv.trsm0, lv.trsm_maxnc,
                                        lv.trsm_smem_elems * sizeof(T), L, U, Dinv, st);
            });
        } else {
            // FP32: X = A T^{-1} on tcgen05 -- inverses, their images, the panels' images before the TRSM
            launch_cls(pd, PC_TRSM, lv.tt1 - lv.tt0, [&] {
                pgpu::launch_trinv<F>(d.ds, d.large_list.p + lv.large0, lv.large1 - lv.large0, lv.ti_maxnzb, L, U,
                                      Dinv, d.ti_off.p, d.tinv.p, st);
                pgpu::launch_split_dense(d.dense_slabs.p + lv.ds0, lv.ds1 - lv.ds0, d.tinv.p, d.timg.p, st);
                const pgpu::SplitSlab *sl = d.split_slabs.p + lv.spl0;
                const int cnt = lv.spl1 - lv.spl0;
                pgpu::launch_split(d.ds, sl, cnt, L, L, d.sp_off.p, d.img0.p, 0, st);
                if (F == pgpu::FACT_GETRF) pgpu::launch_split(d.ds, sl, cnt, U, L, d.sp_off.p, d.img1.p, 0, st);
                pgpu::launch_trsm_tc<F>(d.ds, d.trsm_tc_tiles.p + lv.tt0, lv.tt1 - lv.tt0, L, U, d.img0.p, d.img1.p,
                                        d.sp_off.p, d.timg.p, d.ti_img.p, d.queues.p + 3 * l, d.counters.p + 1, st);
            });
            launch_cls(pd, PC_TRSM, lv.tr32_1 - lv.tr32_0, [&] {
                pgpu::launch_trsm<T, F>(d.ds, d.trsm_tiles32.p + lv.tr32_0, lv.tr32_1 - lv.tr32_0, lv.trsm_maxnc,
                                        lv.trsm_smem_elems * sizeof(T), L, U, Dinv, st);
            });
        }
        if constexpr (sizeof(T) == 8) {
            launch_cls(pd, PC_UPDATE, lv.upd1 - lv.upd0, [&] {
                pgpu::launch_update<T, F>(d.ds, d.upd_tiles.p + lv.upd0, lv.upd1 - lv.upd0, L, U, st);
            });
        } else {
            launch_cls(pd, PC_UPDATE, lv.updsn - lv.upds0, [&] {
                pgpu::launch_update<T, F>(d.ds, d.upd_tiles32.p + lv.upds0, lv.updsn - lv.upds0, L, U, st);
            });
        }
        if constexpr (sizeof(T) == 4) {
            launch_cls(pd, PC_SPLIT, lv.spl1 - lv.spl0, [&] {
                const pgpu::SplitSlab *sl = d.split_slabs.p + lv.spl0;
                const int cnt = lv.spl1 - lv.spl0;
                pgpu::launch_split(d.ds, sl, cnt, L, L, d.sp_off.p, d.img0.p, 0, st);
                if (F == pgpu::FACT_SYTRF) pgpu::launch_split(d.ds, sl, cnt, L, L, d.sp_off.p, d.img1.p, 1, st);
                if (F == pgpu::FACT_GETRF) pgpu::launch_split(d.ds, sl, cnt, U, L, d.sp_off.p, d.img1.p, 0, st);
            });
            launch_cls(pd, PC_UPDATE_BIG, lv.updtn - lv.updt0, [&] {
                pgpu::launch_update_tc<F>(d.ds, d.upd_tc_tiles.p + lv.updt0, lv.updtn - lv.updt0, L, U, d.img0.p,
                                          d.img1.p, d.sp_off.p, d.queues.p + 3 * l + 1, d.counters.p + 1, st);
            });
            // far targets on the side stream, once this level's panels and images are final
            if (two) {
                CUDA_TRY(cudaEventRecord(d.ev_chain[l], st));
                CUDA_TRY(cudaStreamWaitEvent(d.side, d.ev_chain[l], 0));
            }
            launch_cls(
                pd, PC_UPDATE, lv.upds1 - lv.updsn,
                [&] {
                    pgpu::launch_update<T, F>(d.ds, d.upd_tiles32.p + lv.updsn, lv.upds1 - lv.updsn, L, U, sd);
                },
                sd);
            launch_cls(
                pd, PC_UPDATE_BIG, lv.updt1 - lv.updtn,
                [&] {
                    pgpu::launch_update_tc<F>(d.ds, d.upd_tc_tiles.p + lv.updtn, lv.updt1 - lv.updtn, L, U,
                                              d.img0.p, d.img1.p, d.sp_off.p, d.queues.p + 3 * l + 2,
                                              d.counters.p + 1, sd);
                },
                sd);
            if (two) CUDA_TRY(cudaEventRecord(d.ev_rest[l], d.side));
        } else {
            launch_cls(pd, PC_UPDATE_BIG, lv.updb1 - lv.updb0, [&] {
                pgpu::launch_update_big<T, F>(d.ds, d.upd_big_tiles.p + lv.updb0, lv.updb1 - lv.updb0, L, U, st);
            });
        }
    }
    if (two) {  // the library stream resumes once every far update is in
        CUDA_TRY(cudaEventRecord(d.ev_chain[0], d.side));
        CUDA_TRY(cudaStreamWaitEvent(st, d.ev_chain[0], 0));
    }
    CUDA_TRY(cudaGetLastError());
    return PASTIX_SUCCESS;
}

// spm values (host or device) -> device values
static int upload_values(pastix_data_t *pd, const void *values, bool on_device, int flttype) {
    Device &d = pd->dev;
    if (flttype == SpmDouble) {
        CUDA_TRY(cudaMemcpyAsync(d.vals.p, values, pd->nnz * sizeof(double),
                                 on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, d.stream));
    } else if (flttype == SpmFloat && !on_device) {
        std::vector<double> tmp(pd->nnz);
        const float *f = (const float *)values;
        for (idx_t i = 0; i < pd->nnz; i++) tmp[i] = f[i];
        CUDA_TRY(cudaMemcpyAsync(d.vals.p, tmp.data(), pd->nnz * sizeof(double), cudaMemcpyHostToDevice, d.stream));
        CUDA_TRY(cudaStreamSynchronize(d.stream));
    } else {
        perr("unsupported value type");
        return PASTIX_ERR_BADPARAMETER;
    }
    return PASTIX_SUCCESS;
}

__global__ void k_gather_csr(int64_t nnz, const int64_t *__restrict__ src, const double *__restrict__ vals,
                             double *__restrict__ out) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x)
        out[q] = vals[src[q]];
}

// bcsc analogue: permuted CSR values + ||A||_F (sopalin/pastix_task_sopalin.c:93-160)
static int values_to_csr(pastix_data_t *pd) {
    Device &d = pd->dev;
    int blocks = (int)std::min<int64_t>((pd->csr_nnz + 255) / 256, 148 * 16);
    k_gather_csr<<<std::max(blocks, 1), 256, 0, d.stream>>>(pd->csr_nnz, d.csr_src.p, d.vals.p, d.csr_val.p);
    pgpu::launch_dot(pd->csr_nnz, d.csr_val.p, d.csr_val.p, d.part.p, 1, d.scal.p, d.stream);
    double nrm = 0;
    CUDA_TRY(cudaMemcpyAsync(&nrm, d.scal.p, sizeof(double), cudaMemcpyDeviceToHost, d.stream));
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    pd->anorm = nrm;
    pd->dparm[DPARM_A_NORM] = nrm;
    return PASTIX_SUCCESS;
}

static int spm2bcsc_common(pastix_data_t *pd, const void *values, bool on_device, int flttype) {
    if (!(pd->steps & STEP_ANALYSE)) {
        perr("pastix_subtask_spm2bcsc: pastix_task_analyze() has to be called first");
        return PASTIX_ERR_BADPARAMETER;
    }
    int rc = device_setup(pd);
    if (rc) return rc;
    rc = upload_values(pd, values, on_device, flttype);
    if (rc) return rc;
    rc = values_to_csr(pd);
    if (rc) return rc;
    pd->steps |= STEP_CSC2BCSC;
    pd->steps &= ~(STEP_BCSC2CTAB | STEP_NUMFACT);
    return PASTIX_SUCCESS;
}

extern "C" int pastix_subtask_spm2bcsc(pastix_data_t *pd, spmatrix_t *spm) {
    if (!pd) return PASTIX_ERR_BADPARAMETER;
    int rc = check_spm(spm);
    if (rc) return rc;
    if (spm->n != pd->n || spm->colptr[spm->n] - spm->baseval != pd->nnz) {
        perr("pastix_subtask_spm2bcsc: the matrix does not match the analysed pattern");
        return PASTIX_ERR_BADPARAMETER;
    }
    if (!spm->values) return PASTIX_ERR_BADPARAMETER;
    return spm2bcsc_common(pd, spm->values, false, spm->flttype);
}

// coeftabInit (sopalin/coeftab.c:205): allocate and fill the panels
extern "C" int pastix_subtask_bcsc2ctab(pastix_data_t *pd) {
    if (!pd || !(pd->steps & STEP_CSC2BCSC)) {
        perr("pastix_subtask_bcsc2ctab: pastix_subtask_spm2bcsc() has to be called first");
        return PASTIX_ERR_BADPARAMETER;
    }
    Device &d = pd->dev;
    CUDA_TRY(cudaSetDevice(d.dev));
    pd->mixed = pd->iparm[IPARM_MIXED] ? 1 : 0;
    const int fs = pd->mixed ? 4 : 8;
    const int fk = fact_kind(pd);
    const size_t bytes = (size_t)std::max<idx_t>(1, pd->solver.coefnbr) * fs;
    if (d.Lc.n != bytes) CUDA_TRY(d.Lc.alloc(bytes));
    if (fk == pgpu::FACT_GETRF) { if (d.Uc.n != bytes) CUDA_TRY(d.Uc.alloc(bytes)); }
    else d.Uc.reset();
    const size_t dbytes = (size_t)std::max<int64_t>(1, pd->dinv_total) * fs;
    if (d.dinv.n != dbytes) CUDA_TRY(d.dinv.alloc(dbytes));
    d.fltsize = fs;
    if (pd->mixed && pd->split_total > 0) {  // BF16 images: padding must read as zero, so clear on (re)allocation
        const size_t sb = (size_t)pd->split_total;
        const int nimg = (fk == pgpu::FACT_POTRF) ? 1 : 2;
        if (d.img0.n != sb) {
            CUDA_TRY(d.img0.alloc(sb));
            CUDA_TRY(cudaMemsetAsync(d.img0.p, 0, sb, d.stream));
        }
        if (nimg == 2 && d.img1.n != sb) {
            CUDA_TRY(d.img1.alloc(sb));
            CUDA_TRY(cudaMemsetAsync(d.img1.p, 0, sb, d.stream));
        }
        if (nimg == 1) d.img1.reset();
        // triangular inverses: entries below their blocks are never written, so clear on (re)allocation
        if (pd->tinv_total > 0 && d.tinv.n != (size_t)pd->tinv_total) {
            CUDA_TRY(d.tinv.alloc((size_t)pd->tinv_total));
            CUDA_TRY(cudaMemsetAsync(d.tinv.p, 0, (size_t)pd->tinv_total * sizeof(float), d.stream));
        }
        if (pd->timg_total > 0 && d.timg.n != (size_t)pd->timg_total) {
            CUDA_TRY(d.timg.alloc((size_t)pd->timg_total));
            CUDA_TRY(cudaMemsetAsync(d.timg.p, 0, (size_t)pd->timg_total, d.stream));
        }
    } else {
        d.img0.reset();
        d.img1.reset();
        d.tinv.reset();
        d.timg.reset();
    }
    CUDA_TRY(cudaMemsetAsync(d.Lc.p, 0, bytes, d.stream));
    if (d.Uc.p) CUDA_TRY(cudaMemsetAsync(d.Uc.p, 0, bytes, d.stream));
    const int64_t *um = d.Uc.p ? d.umap.p : nullptr;
    launch_cls(pd, PC_FILL, pd->nnz, [&] {
        if (pd->mixed)
            pgpu::launch_fill_coef<float>(pd->nnz, d.vals.p, d.lmap.p, um, (float *)d.Lc.p, (float *)d.Uc.p, d.stream);
        else
            pgpu::launch_fill_coef<double>(pd->nnz, d.vals.p, d.lmap.p, um, (double *)d.Lc.p, (double *)d.Uc.p,
                                           d.stream);
    });
    CUDA_TRY(cudaGetLastError());
    pd->dparm[DPARM_MEM_FR] = (double)bytes * (d.Uc.p ? 2 : 1);
    pd->steps |= STEP_BCSC2CTAB;
    return PASTIX_SUCCESS;
}

// pastix_subtask_sopalin (sopalin/pastix_task_sopalin.c:412-560)
extern "C" int pastix_subtask_sopalin(pastix_data_t *pd) {
    if (!pd || !(pd->steps & STEP_BCSC2CTAB)) {
        perr("pastix_subtask_sopalin: pastix_subtask_bcsc2ctab() has to be called first");
        return PASTIX_ERR_BADPARAMETER;
    }
    Device &d = pd->dev;
    CUDA_TRY(cudaSetDevice(d.dev));
    double *dparm = pd->dparm;
    double threshold;
    if (dparm[DPARM_EPSILON_MAGN_CTRL] < 0.) threshold = -dparm[DPARM_EPSILON_MAGN_CTRL];
    else if (dparm[DPARM_EPSILON_MAGN_CTRL] == 0.) threshold = ldexp(1.0, -53) * pd->anorm;  // dlamch('e') * ||A||
    else threshold = dparm[DPARM_EPSILON_MAGN_CTRL] * pd->anorm;
    CUDA_TRY(cudaMemsetAsync(d.counters.p, 0, 2 * sizeof(int), d.stream));
    pd->crit_host = threshold;
    CUDA_TRY(cudaMemcpyAsync(d.crit.p, &pd->crit_host, sizeof(double), cudaMemcpyHostToDevice, d.stream));
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    double t0 = now_s();
    int fk = fact_kind(pd), rc;
    if (pd->mixed) {
        // FP32 factors: launched kernel by kernel.  Replayed as a graph, the same launches ran
        // 12% slower on a B200 (100^3 Laplacian: 83 ms against 74 ms, with or without the side
        // stream in the graph), so only the solves of this precision are graphed.
        if (fk == pgpu::FACT_POTRF) rc = run_factor<float, pgpu::FACT_POTRF>(pd, threshold);
        else if (fk == pgpu::FACT_SYTRF) rc = run_factor<float, pgpu::FACT_SYTRF>(pd, threshold);
        else rc = run_factor<float, pgpu::FACT_GETRF>(pd, threshold);
    } else {
        // FP64: the whole level sequence is one CUDA graph per (kind, buffers)
        const std::vector<uintptr_t> key{1, (uintptr_t)fk, (uintptr_t)d.Lc.p, (uintptr_t)d.Uc.p, (uintptr_t)d.dinv.p};
        rc = run_graphed(pd, key, [&]() -> int {
            if (fk == pgpu::FACT_POTRF) return run_factor<double, pgpu::FACT_POTRF>(pd, threshold);
            if (fk == pgpu::FACT_SYTRF) return run_factor<double, pgpu::FACT_SYTRF>(pd, threshold);
            return run_factor<double, pgpu::FACT_GETRF>(pd, threshold);
        });
    }
    if (rc) return rc;
    int cnt[2] = {0, 0};
    CUDA_TRY(cudaMemcpyAsync(cnt, d.counters.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, d.stream));
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    double t = now_s() - t0;
    if (cnt[1] != 0) { perr("device status %d after factorization", cnt[1]); return PASTIX_ERR_INTERNAL; }
    dparm[DPARM_FACT_TIME] = t;
    dparm[DPARM_FACT_FLOPS] = t > 0 ? dparm[DPARM_FACT_THFLOPS] / t : 0.0;
    dparm[DPARM_FACT_RLFLOPS] = dparm[DPARM_FACT_THFLOPS];
    pd->iparm[IPARM_STATIC_PIVOTING] = cnt[0];
    pd->steps |= STEP_NUMFACT;
    return PASTIX_SUCCESS;
}

extern "C" int pastix_task_numfact(pastix_data_t *pd, spmatrix_t *spm) {
    if (!pd) return PASTIX_ERR_BADPARAMETER;
    int rc = pastix_subtask_spm2bcsc(pd, spm);
    if (rc) return rc;
    rc = pastix_subtask_bcsc2ctab(pd);
    if (rc) return rc;
    return pastix_subtask_sopalin(pd);
}

extern "C" int pgpu_numfact_device(pastix_data_t *pd, const double *values_dev) {
    if (!pd || !values_dev) return PASTIX_ERR_BADPARAMETER;
    int rc = spm2bcsc_common(pd, values_dev, true, SpmDouble);
    if (rc) return rc;
    rc = pastix_subtask_bcsc2ctab(pd);
    if (rc) return rc;
    return pastix_subtask_sopalin(pd);
}

extern "C" int pgpu_get_coeftab(const pastix_data_t *pd, void *L, void *U) {
    if (!pd || !(pd->steps & STEP_NUMFACT) || !L) return PASTIX_ERR_BADPARAMETER;
    const Device &d = pd->dev;
    CUDA_TRY(cudaSetDevice(d.dev));
    size_t bytes = (size_t)pd->solver.coefnbr * d.fltsize;
    CUDA_TRY(cudaMemcpyAsync(L, d.Lc.p, bytes, cudaMemcpyDeviceToHost, d.stream));
    if (U && d.Uc.p) CUDA_TRY(cudaMemcpyAsync(U, d.Uc.p, bytes, cudaMemcpyDeviceToHost, d.stream));
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    return PASTIX_SUCCESS;
}

extern "C" int pgpu_wait_selftest(int *timed_out) {
    if (!timed_out) return PASTIX_ERR_BADPARAMETER;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PASTIX_ERR_INTERNAL;
    return pgpu::wait_selftest(timed_out) == cudaSuccess ? PASTIX_SUCCESS : PASTIX_ERR_INTERNAL;
}

extern "C" int pgpu_device_status(const pastix_data_t *pd) {
    if (!pd || !pd->dev.ready) return 0;
    int cnt[2] = {0, 0};
    if (cudaMemcpy(cnt, pd->dev.counters.p, 2 * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return cnt[1];
}

// ---------------------------------------------------------------------------
// solve on permuted device vectors
// ---------------------------------------------------------------------------
// Full inverses of the wide cblks' diagonal factors: kept by the FP32 factorization only.
template <typename T>
static const float *tinv_of(const Device &d) {
    return (sizeof(T) == 4 && d.tinv.n > 0) ? d.tinv.p : nullptr;
}

// Forward sweep with the block-lower panel P (unit diagonal or not).  Wide
// cblks apply their diagonal blocks with the inverted sub-blocks (set zside,
// D scaling for LDL^T), narrow ones by substitution.
template <typename T>
static void sweep_forward(pastix_data_t *pd, const T *P, int unit, int zside, int scaled, T *Y, int ldy, int nrhs) {
    Device &d = pd->dev;
    const T *Ld = reinterpret_cast<const T *>(d.Lc.p);
    const T *Dinv = reinterpret_cast<const T *>(d.dinv.p);
    for (size_t l = 0; l < pd->levels.size(); l++) {
        const LevelLists &lv = pd->levels[l];
        launch_cls(pd, PC_FWD_DIAG, lv.small1 - lv.small0, [&] {
            pgpu::launch_fwd_diag<T>(d.ds, d.small_list.p + lv.small0, lv.small1 - lv.small0, lv.maxnc, P, unit, Y,
                                     ldy, nrhs, d.stream);
        });
        launch_cls(pd, PC_FWD_DIAG, lv.large1 - lv.large0, [&] {
            pgpu::launch_fwd_diag_inv<T>(d.ds, d.large_list.p + lv.large0, lv.large1 - lv.large0, lv.maxnc, P, Dinv,
                                         zside, scaled, Ld, Y, ldy, nrhs, tinv_of<T>(d), d.ti_off.p, lv.ntinv,
                                         d.stream);
        });
        launch_cls(pd, PC_FWD_UPDATE, lv.st1 - lv.st0, [&] {
            pgpu::launch_fwd_update<T>(d.ds, d.solve_tiles.p + lv.st0, lv.st1 - lv.st0, lv.maxnc, P, Y, ldy, nrhs,
                                       d.stream);
        });
    }
}
// Backward sweep: solve P^T x = y with P block lower.
template <typename T>
static void sweep_backward(pastix_data_t *pd, const T *P, int unit, int zside, int scaled, T *Y, int ldy, int nrhs) {
    Device &d = pd->dev;
    const T *Ld = reinterpret_cast<const T *>(d.Lc.p);
    const T *Dinv = reinterpret_cast<const T *>(d.dinv.p);
    for (size_t l = pd->levels.size(); l-- > 0;) {
        const LevelLists &lv = pd->levels[l];
        launch_cls(pd, PC_BWD_UPDATE, lv.st1 - lv.st0, [&] {
            pgpu::launch_bwd_update<T>(d.ds, d.solve_tiles.p + lv.st0, lv.st1 - lv.st0, lv.maxnc, P, Y, ldy, nrhs,
                                       d.stream);
        });
        launch_cls(pd, PC_BWD_DIAG, lv.small1 - lv.small0, [&] {
            pgpu::launch_bwd_diag<T>(d.ds, d.small_list.p + lv.small0, lv.small1 - lv.small0, lv.maxnc, P, unit, Y,
                                     ldy, nrhs, d.stream);
        });
        launch_cls(pd, PC_BWD_DIAG, lv.large1 - lv.large0, [&] {
            pgpu::launch_bwd_diag_inv<T>(d.ds, d.large_list.p + lv.large0, lv.large1 - lv.large0, lv.maxnc, P, Dinv,
                                         zside, scaled, Ld, Y, ldy, nrhs, tinv_of<T>(d), d.ti_off.p, lv.ntinv,
                                         d.stream);
        });
    }
}

// Solve A X = B (trans = 0) or A^T X = B (trans = 1) in place on permuted
// device vectors of type T (the factor's arithmetic).
template <typename T>
static void solve_perm(pastix_data_t *pd, int trans, T *Y, int ldy, int nrhs) {
    Device &d = pd->dev;
    const T *L = reinterpret_cast<const T *>(d.Lc.p);
    const T *U = reinterpret_cast<const T *>(d.Uc.p);
    int fk = fact_kind(pd);
    if (fk == pgpu::FACT_POTRF) {
        sweep_forward<T>(pd, L, 0, 0, 0, Y, ldy, nrhs);
        sweep_backward<T>(pd, L, 0, 0, 0, Y, ldy, nrhs);
    } else if (fk == pgpu::FACT_SYTRF) {
        sweep_forward<T>(pd, L, 1, 0, 1, Y, ldy, nrhs);
        launch_cls(pd, PC_VEC, 1, [&] {
            pgpu::launch_diag_scale<T>(d.ds, (int)pd->solver.cblknbr, L, Y, ldy, nrhs, d.stream);
        });
        sweep_backward<T>(pd, L, 1, 0, 1, Y, ldy, nrhs);
    } else if (!trans) {  // L (unit) then U through U^T
        sweep_forward<T>(pd, L, 1, 1, 0, Y, ldy, nrhs);
        sweep_backward<T>(pd, U, 0, 0, 0, Y, ldy, nrhs);
    } else {  // A^T = U^T L^T
        sweep_forward<T>(pd, U, 0, 0, 0, Y, ldy, nrhs);
        sweep_backward<T>(pd, L, 1, 1, 0, Y, ldy, nrhs);
    }
}

// FP64 permuted vectors in, FP64 out; FP32 factors go through a float copy.
static int solve_perm_d(pastix_data_t *pd, int trans, double *Y, int ldy, int nrhs) {
    Device &d = pd->dev;
    if (!pd->mixed) {
        const std::vector<uintptr_t> key{2, 0, (uintptr_t)trans, (uintptr_t)fact_kind(pd), (uintptr_t)Y,
                                         (uintptr_t)ldy, (uintptr_t)nrhs, (uintptr_t)d.Lc.p, (uintptr_t)d.Uc.p,
                                         (uintptr_t)d.dinv.p};
        return run_graphed(pd, key, [&]() -> int {
            solve_perm<double>(pd, trans, Y, ldy, nrhs);
            CUDA_TRY(cudaGetLastError());
            return PASTIX_SUCCESS;
        });
    }
    size_t need = (size_t)pd->n * nrhs;
    if (d.wf.n < need) CUDA_TRY(d.wf.alloc(need));
    const std::vector<uintptr_t> key{2, 1, (uintptr_t)trans, (uintptr_t)fact_kind(pd), (uintptr_t)Y, (uintptr_t)ldy,
                                     (uintptr_t)nrhs, (uintptr_t)d.Lc.p, (uintptr_t)d.Uc.p, (uintptr_t)d.dinv.p,
                                     (uintptr_t)d.tinv.p, (uintptr_t)d.wf.p};
    return run_graphed(pd, key, [&]() -> int {
        for (int j = 0; j < nrhs; j++)
            pgpu::launch_cast<double, float>(pd->n, Y + (size_t)j * ldy, d.wf.p + (size_t)j * pd->n, d.stream);
        solve_perm<float>(pd, trans, d.wf.p, (int)pd->n, nrhs);
        for (int j = 0; j < nrhs; j++)
            pgpu::launch_cast<float, double>(pd->n, d.wf.p + (size_t)j * pd->n, Y + (size_t)j * ldy, d.stream);
        CUDA_TRY(cudaGetLastError());
        return PASTIX_SUCCESS;
    });
}

static int check_numfact(const pastix_data_t *pd, const char *who) {
    if (!pd || !(pd->steps & STEP_NUMFACT)) {
        perr("%s: pastix_task_numfact() has to be called first", who);
        return PASTIX_ERR_BADPARAMETER;
    }
    return PASTIX_SUCCESS;
}

// Device solve in the original numbering: B (n x nrhs, ld ldb) overwritten.
static int solve_device_orig(pastix_data_t *pd, int trans, int nrhs, double *B, idx_t ldb, cudaStream_t user) {
    Device &d = pd->dev;
    CUDA_TRY(cudaSetDevice(d.dev));
    const idx_t n = pd->n;
    size_t need = (size_t)n * nrhs;
    if (d.w1.n < need) CUDA_TRY(d.w1.alloc(need));
    cudaEvent_t ev = nullptr;
    if (user != d.stream) {  // order the library stream after the caller's (NULL = legacy default) stream
        CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CUDA_TRY(cudaEventRecord(ev, user));
        CUDA_TRY(cudaStreamWaitEvent(d.stream, ev, 0));
    }
    pgpu::launch_permute<double, double>((int)n, nrhs, d.perm.p, 1, B, ldb, d.w1.p, n, d.stream);
    int rc = solve_perm_d(pd, trans, d.w1.p, (int)n, nrhs);
    if (rc) return rc;
    pgpu::launch_permute<double, double>((int)n, nrhs, d.perm.p, 0, d.w1.p, n, B, ldb, d.stream);
    if (ev) {
        CUDA_TRY(cudaEventRecord(ev, d.stream));
        CUDA_TRY(cudaStreamWaitEvent(user, ev, 0));
        cudaEventDestroy(ev);
    }
    CUDA_TRY(cudaGetLastError());
    return PASTIX_SUCCESS;
}

extern "C" int pgpu_solve_device(pastix_data_t *pd, pastix_int_t nrhs, double *B, pastix_int_t ldb, void *stream) {
    int rc = check_numfact(pd, "pgpu_solve_device");
    if (rc) return rc;
    if (nrhs < 1 || ldb < pd->n || !B) return PASTIX_ERR_BADPARAMETER;
    return solve_device_orig(pd, 0, (int)nrhs, B, ldb, (cudaStream_t)stream);
}

extern "C" int pgpu_solve_transposed_device(pastix_data_t *pd, pastix_int_t nrhs, double *B, pastix_int_t ldb,
                                            void *stream) {
    int rc = check_numfact(pd, "pgpu_solve_transposed_device");
    if (rc) return rc;
    if (nrhs < 1 || ldb < pd->n || !B) return PASTIX_ERR_BADPARAMETER;
    return solve_device_orig(pd, 1, (int)nrhs, B, ldb, (cudaStream_t)stream);
}

extern "C" int pastix_task_solve(pastix_data_t *pd, pastix_int_t m, pastix_int_t nrhs, void *B, pastix_int_t ldb) {
    int rc = check_numfact(pd, "pastix_task_solve");
    if (rc) return rc;
    if (m != pd->n || nrhs < 1 || ldb < m || !B) return PASTIX_ERR_BADPARAMETER;
    Device &d = pd->dev;
    CUDA_TRY(cudaSetDevice(d.dev));
    double t0 = now_s();
    double *buf = work(d, WS_SOLVE, (size_t)m * nrhs);
    if (!buf) return PASTIX_ERR_OUTOFMEMORY;
    CUDA_TRY(cudaMemcpy2DAsync(buf, m * sizeof(double), B, ldb * sizeof(double), m * sizeof(double), nrhs,
                               cudaMemcpyHostToDevice, d.stream));
    int trans = pd->iparm[IPARM_TRANSPOSE_SOLVE] == PastixTrans ? 1 : 0;
    rc = solve_device_orig(pd, trans, (int)nrhs, buf, m, d.stream);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy2DAsync(B, ldb * sizeof(double), buf, m * sizeof(double), m * sizeof(double), nrhs,
                               cudaMemcpyDeviceToHost, d.stream));
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    pd->dparm[DPARM_SOLV_TIME] = now_s() - t0;
    pd->steps |= STEP_SOLVE;
    return PASTIX_SUCCESS;
}

// ---------------------------------------------------------------------------
// subtask-level solve API on pastix_rhs_t (sopalin/pastix_task_solve.c)
// ---------------------------------------------------------------------------
extern "C" int pastixRhsInit(pastix_rhs_t *rhs) {
    if (!rhs) return PASTIX_ERR_BADPARAMETER;
    *rhs = (pastix_rhs_t)calloc(1, sizeof(struct pastix_rhs_s));
    (*rhs)->flttype = SpmDouble;
    return PASTIX_SUCCESS;
}
extern "C" int pastixRhsFinalize(pastix_rhs_t rhs) {
    if (!rhs) return PASTIX_ERR_BADPARAMETER;
    if (rhs->allocated && rhs->b) cudaFree(rhs->b);
    free(rhs);
    return PASTIX_SUCCESS;
}
static int rhs_alloc(pastix_rhs_t r, int flt, pastix_int_t m, pastix_int_t n) {
    size_t es = flt == SpmFloat ? 4 : 8;
    if (r->allocated && r->b) cudaFree(r->b);
    r->b = nullptr;
    CUDA_TRY(cudaMalloc(&r->b, std::max<size_t>(1, (size_t)m * n) * es));
    r->allocated = 1;
    r->flttype = flt;
    r->m = m;
    r->n = n;
    r->ld = m;
    return PASTIX_SUCCESS;
}
extern "C" int pastixRhsDoubletoSingle(const pastix_rhs_t dB, pastix_rhs_t sB) {
    if (!dB || !sB || dB->flttype != SpmDouble) return PASTIX_ERR_BADPARAMETER;
    int rc = rhs_alloc(sB, SpmFloat, dB->m, dB->n);
    if (rc) return rc;
    for (pastix_int_t j = 0; j < dB->n; j++)
        pgpu::launch_cast<double, float>(dB->m, (const double *)dB->b + j * dB->ld, (float *)sB->b + j * sB->ld, 0);
    CUDA_TRY(cudaDeviceSynchronize());
    return PASTIX_SUCCESS;
}
extern "C" int pastixRhsSingleToDouble(const pastix_rhs_t sB, pastix_rhs_t dB) {
    if (!dB || !sB || sB->flttype != SpmFloat || dB->flttype != SpmDouble || !dB->b) return PASTIX_ERR_BADPARAMETER;
    for (pastix_int_t j = 0; j < sB->n; j++)
        pgpu::launch_cast<float, double>(sB->m, (const float *)sB->b + j * sB->ld, (double *)dB->b + j * dB->ld, 0);
    CUDA_TRY(cudaDeviceSynchronize());
    return PASTIX_SUCCESS;
}

// Forward: B (host, original numbering) -> Bp (device, permuted, FP64).
// Backward: Bp -> B.
extern "C" int pastix_subtask_applyorder(pastix_data_t *pd, pastix_dir_t dir, pastix_int_t m, pastix_int_t n, void *B,
                                         pastix_int_t ldb, pastix_rhs_t Bp) {
    if (!pd || !(pd->steps & STEP_ANALYSE) || !Bp || m != pd->n || n < 1 || ldb < m || !B) return PASTIX_ERR_BADPARAMETER;
    int rc = device_setup(pd);
    if (rc) return rc;
    Device &d = pd->dev;
    double *tmp = work(d, WS_ORDER, (size_t)m * n);
    if (!tmp) return PASTIX_ERR_OUTOFMEMORY;
    if (dir == PastixDirForward) {
        if (!(Bp->b && Bp->m == m && Bp->n == n && Bp->flttype == SpmDouble)) {
            rc = rhs_alloc(Bp, SpmDouble, m, n);
            if (rc) return rc;
        }
        CUDA_TRY(cudaMemcpy2DAsync(tmp, m * 8, B, ldb * 8, m * 8, n, cudaMemcpyHostToDevice, d.stream));
        pgpu::launch_permute<double, double>((int)m, (int)n, d.perm.p, 1, tmp, m, (double *)Bp->b, Bp->ld, d.stream);
    } else {
        if (!Bp->b || Bp->flttype != SpmDouble) return PASTIX_ERR_BADPARAMETER;
        pgpu::launch_permute<double, double>((int)m, (int)n, d.perm.p, 0, (const double *)Bp->b, Bp->ld, tmp, m, d.stream);
        CUDA_TRY(cudaMemcpy2DAsync(B, ldb * 8, tmp, m * 8, m * 8, n, cudaMemcpyDeviceToHost, d.stream));
    }
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    return PASTIX_SUCCESS;
}

// pastix_subtask_trsm: one triangular sweep on a permuted device rhs
// (side = Left only; uplo/trans/diag select the sweep as in the reference's
// step table, sopalin/pastix_task_solve.c:543-649).
extern "C" int pastix_subtask_trsm(pastix_data_t *pd, pastix_side_t side, pastix_uplo_t uplo, pastix_trans_t trans,
                                   pastix_diag_t diag, pastix_rhs_t b) {
    int rc = check_numfact(pd, "pastix_subtask_trsm");
    if (rc) return rc;
    if (side != PastixLeft || !b || !b->b) return PASTIX_ERR_BADPARAMETER;
    Device &d = pd->dev;
    int fk = fact_kind(pd);
    int unit = diag == PastixUnit;
    int isd = b->flttype == SpmDouble;
    if ((pd->mixed && isd) || (!pd->mixed && !isd)) {
        perr("pastix_subtask_trsm: rhs precision must match the factor's");
        return PASTIX_ERR_BADPARAMETER;
    }
    // which panel: lower sweeps (uplo Lower, NoTrans) use L; upper sweeps use L^T,
    // or U through the U^T panel for GETRF.
    auto run = [&](auto *Y) {
        using T = std::remove_pointer_t<decltype(Y)>;
        const T *L = reinterpret_cast<const T *>(d.Lc.p);
        const T *U = reinterpret_cast<const T *>(d.Uc.p);
        // inverted diagonal sub-blocks: LU keeps U^{-1} (set 0) and L^{-T} (set 1);
        // LL^T / LDL^T keep one set (LDL^T folds D into it)
        const int sy = fk == pgpu::FACT_SYTRF;
        if (uplo == PastixLower && trans == PastixNoTrans)
            sweep_forward<T>(pd, L, unit, fk == pgpu::FACT_GETRF ? 1 : 0, sy, Y, (int)b->ld, (int)b->n);
        else if (uplo == PastixLower)
            sweep_backward<T>(pd, L, unit, fk == pgpu::FACT_GETRF ? 1 : 0, sy, Y, (int)b->ld, (int)b->n);
        else if (uplo == PastixUpper && trans == PastixNoTrans)
            sweep_backward<T>(pd, fk == pgpu::FACT_GETRF ? U : L, unit, 0, sy, Y, (int)b->ld, (int)b->n);
        else sweep_forward<T>(pd, fk == pgpu::FACT_GETRF ? U : L, unit, 0, sy, Y, (int)b->ld, (int)b->n);
    };
    if (isd) run((double *)b->b);
    else run((float *)b->b);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    return PASTIX_SUCCESS;
}

extern "C" int pastix_subtask_diag(pastix_data_t *pd, pastix_rhs_t b) {
    int rc = check_numfact(pd, "pastix_subtask_diag");
    if (rc) return rc;
    if (!b || !b->b || fact_kind(pd) != pgpu::FACT_SYTRF) return PASTIX_ERR_BADPARAMETER;
    Device &d = pd->dev;
    if (b->flttype == SpmDouble && !pd->mixed)
        pgpu::launch_diag_scale<double>(d.ds, (int)pd->solver.cblknbr, (const double *)d.Lc.p, (double *)b->b, (int)b->ld,
                                        (int)b->n, d.stream);
    else if (b->flttype == SpmFloat && pd->mixed)
        pgpu::launch_diag_scale<float>(d.ds, (int)pd->solver.cblknbr, (const float *)d.Lc.p, (float *)b->b, (int)b->ld,
                                       (int)b->n, d.stream);
    else return PASTIX_ERR_BADPARAMETER;
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    return PASTIX_SUCCESS;
}

extern "C" int pastix_subtask_solve_adv(pastix_data_t *pd, pastix_trans_t transA, pastix_rhs_t b) {
    int rc = check_numfact(pd, "pastix_subtask_solve");
    if (rc) return rc;
    if (!b || !b->b || b->flttype != SpmDouble) return PASTIX_ERR_BADPARAMETER;
    rc = solve_perm_d(pd, transA == PastixNoTrans ? 0 : 1, (double *)b->b, (int)b->ld, (int)b->n);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(pd->dev.stream));
    return PASTIX_SUCCESS;
}

extern "C" int pastix_subtask_solve(pastix_data_t *pd, pastix_rhs_t b) {
    return pastix_subtask_solve_adv(pd, PastixNoTrans, b);
}

// ---------------------------------------------------------------------------
// refinement on the device (refinement/z_refine_*.c), one rhs at a time
// ---------------------------------------------------------------------------
namespace {
struct Refiner {
    pastix_data_t *pd;
    Device &d;
    int64_t n;
    bool precond;
    explicit Refiner(pastix_data_t *p) : pd(p), d(p->dev), n(p->n), precond((p->steps & STEP_NUMFACT) != 0) {}
    double dot(const double *a, const double *b) {
        pgpu::launch_dot(n, a, b, d.part.p, 0, d.scal.p, d.stream);
        double v = 0;
        cudaMemcpyAsync(&v, d.scal.p, sizeof(double), cudaMemcpyDeviceToHost, d.stream);
        cudaStreamSynchronize(d.stream);
        return v;
    }
    double norm(const double *a) {
        pgpu::launch_dot(n, a, a, d.part.p, 1, d.scal.p, d.stream);
        double v = 0;
        cudaMemcpyAsync(&v, d.scal.p, sizeof(double), cudaMemcpyDeviceToHost, d.stream);
        cudaStreamSynchronize(d.stream);
        return v;
    }
    void spmv(double alpha, const double *x, double beta, double *y) {
        launch_cls(pd, PC_SPMV, 1, [&] {
            pgpu::launch_spmv_stream(d.spmv_nblocks, d.spmv_part.p, d.csr_rowptr.p, d.csr_col.p, d.csr_val.p, alpha,
                                     x, beta, y, d.stream);
        });
    }
    void copy(const double *a, double *b) { cudaMemcpyAsync(b, a, n * 8, cudaMemcpyDeviceToDevice, d.stream); }
    void axpy(double a, const double *x, double *y) { pgpu::launch_axpy(n, a, x, y, d.stream); }
    void scal(double a, double *x) { pgpu::launch_scal(n, a, x, d.stream); }
    // M^{-1} x in place, solved in one fixed work vector so that the captured
    // solve graph is the same for every Krylov vector
    int spsv(double *x) {
        if (!precond) return 0;
        double *s = work(d, WS_SPSV, (size_t)n);
        if (!s) return PASTIX_ERR_OUTOFMEMORY;
        cudaMemcpyAsync(s, x, n * 8, cudaMemcpyDeviceToDevice, d.stream);
        int rc = solve_perm_d(pd, 0, s, (int)n, 1);
        cudaMemcpyAsync(x, s, n * 8, cudaMemcpyDeviceToDevice, d.stream);
        return rc;
    }
};

// GMRES(im), right preconditioned (refinement/z_refine_gmres.c:49-371)
static int refine_gmres(Refiner &R, double *x, const double *b, double eps, int itermax, int im, int &iters_out) {
    const int64_t n = R.n;
    const int im1 = im + 1;
    struct { double *p; } V{work(R.d, WS_GMV, (size_t)n * im1)}, W{work(R.d, WS_GMW, (size_t)n * im)},
        gdev{work(R.d, WS_GMG, im1)}, hdev{work(R.d, WS_GMH, im1)};
    if (!V.p || !W.p || !gdev.p || !hdev.p) return PASTIX_ERR_OUTOFMEMORY;
    std::vector<double> H((size_t)im * im1, 0.0), gcos(im), gsin(im), G(im1);
    double normb = R.norm(b);
    if (normb == 0.) normb = 1;
    double normx = R.norm(x);
    int iters = 0;
    double resid_b = 0;
    bool outflag = true;
    while (outflag) {
        double *v0 = V.p;
        R.copy(b, v0);
        if (normx > 0.) R.spmv(-1., x, 1., v0);
        double resid = R.norm(v0);
        resid_b = resid / normb;
        if (resid_b <= eps) break;
        R.scal(1.0 / resid, v0);
        G[0] = resid;
        int i = -1;
        bool inflag = true;
        while (inflag) {
            i++;
            double *Hi = H.data() + (size_t)i * im1;
            double *Vi = V.p + (size_t)i * n;
            double *Wi = W.p + (size_t)i * n;
            R.copy(Vi, Wi);
            if (R.spsv(Wi)) return PASTIX_ERR_INTERNAL;
            double *Vn = Vi + n;
            R.spmv(1.0, Wi, 0., Vn);
            // modified Gram-Schmidt with the coefficients kept on the device (the
            // same operations in the same order as host scalars would take), read
            // back once per Arnoldi step
            for (int j = 0; j <= i; j++) {
                pgpu::launch_dot(n, Vn, V.p + (size_t)j * n, R.d.part.p, 0, hdev.p + j, R.d.stream);
                pgpu::launch_axpy_cols(n, 1, hdev.p + j, V.p + (size_t)j * n, n, Vn, n, R.d.stream);
            }
            pgpu::launch_dot(n, Vn, Vn, R.d.part.p, 1, hdev.p + i + 1, R.d.stream);
            pgpu::launch_scal_cols(n, 1, hdev.p + i + 1, 1, Vn, n, R.d.stream);  // when the norm is > 1e-50
            if (cudaMemcpyAsync(Hi, hdev.p, (size_t)(i + 2) * sizeof(double), cudaMemcpyDeviceToHost, R.d.stream) !=
                    cudaSuccess ||
                cudaStreamSynchronize(R.d.stream) != cudaSuccess)
                return PASTIX_ERR_INTERNAL;
            for (int j = 0; j < i; j++) {
                double t = Hi[j];
                Hi[j] = gcos[j] * t + gsin[j] * Hi[j + 1];
                Hi[j + 1] = gcos[j] * Hi[j + 1] - gsin[j] * t;
            }
            double t = std::sqrt(Hi[i] * Hi[i] + Hi[i + 1] * Hi[i + 1]);
            if (std::fabs(t) <= eps) t = eps;
            gcos[i] = Hi[i] / t;
            gsin[i] = Hi[i + 1] / t;
            G[i + 1] = -gsin[i] * G[i];
            G[i] = gcos[i] * G[i];
            Hi[i] = gcos[i] * Hi[i] + gsin[i] * Hi[i + 1];
            resid = std::fabs(G[i + 1]);
            resid_b = resid / normb;
            iters++;
            if (i + 1 >= im || resid_b <= eps || iters >= itermax) inflag = false;
        }
        // y = H^{-1} G (upper triangular, i+1 columns)
        int m = i + 1;
        std::vector<double> y(G.begin(), G.begin() + m);
        for (int r = m - 1; r >= 0; r--) {
            double s = y[r];
            for (int c = r + 1; c < m; c++) s -= H[(size_t)c * im1 + r] * y[c];
            y[r] = s / H[(size_t)r * im1 + r];
        }
        cudaMemcpyAsync(gdev.p, y.data(), m * 8, cudaMemcpyHostToDevice, R.d.stream);
        pgpu::launch_gemv(n, m, R.precond ? W.p : V.p, gdev.p, x, R.d.stream);
        cudaStreamSynchronize(R.d.stream);
        normx = 1.0;
        if (iters >= itermax) outflag = false;
    }
    iters_out = iters;
    return PASTIX_SUCCESS;
}

// preconditioned CG (refinement/z_refine_grad.c:49-175)
static int refine_cg(Refiner &R, double *x, const double *b, double eps, int itermax, int &iters_out) {
    const int64_t n = R.n;
    double *wv = work(R.d, WS_VEC, (size_t)n * 4);
    if (!wv) return PASTIX_ERR_OUTOFMEMORY;
    struct { double *p; } r{wv}, p{wv + n}, z{wv + 2 * n}, q{wv + 3 * n};
    double normb = R.norm(b);
    if (normb == 0.) normb = 1;
    double normx = R.norm(x);
    R.copy(b, r.p);
    if (normx > 0.) R.spmv(-1., x, 1., r.p);
    double resid_b = R.norm(r.p) / normb;
    // z = M^{-1} r is only needed when the loop runs; the residual test is
    // taken before the preconditioner solve (same iterates as the reference)
    if (resid_b > eps && itermax > 0) {
        R.copy(r.p, z.p);
        if (R.spsv(z.p)) return PASTIX_ERR_INTERNAL;
        R.copy(z.p, p.p);
    }
    int it = 0;
    while (resid_b > eps && it < itermax) {
        it++;
        R.spmv(1.0, p.p, 0., q.p);
        double beta = R.dot(r.p, z.p);
        double alpha = beta / R.dot(q.p, p.p);
        R.axpy(alpha, p.p, x);
        R.axpy(-alpha, q.p, r.p);
        resid_b = R.norm(r.p) / normb;
        if (resid_b <= eps || it >= itermax) break;
        R.copy(r.p, z.p);
        if (R.spsv(z.p)) return PASTIX_ERR_INTERNAL;
        double rz = R.dot(r.p, z.p);
        beta = rz / beta;
        pgpu::launch_xpby(n, z.p, beta, p.p, R.d.stream);  // p = z + beta p
    }
    iters_out = it;
    return PASTIX_SUCCESS;
}

// preconditioned BiCGStab (refinement/z_refine_bicgstab.c:49-228)
static int refine_bicgstab(Refiner &R, double *x, const double *b, double eps, int itermax, int &iters_out) {
    const int64_t n = R.n;
    double *wv = work(R.d, WS_VEC, (size_t)n * 9);
    if (!wv) return PASTIX_ERR_OUTOFMEMORY;
    struct { double *p; } r{wv}, r2{wv + n}, p{wv + 2 * n}, y{wv + 3 * n}, v{wv + 4 * n}, s{wv + 5 * n},
        z{wv + 6 * n}, t{wv + 7 * n}, t2{wv + 8 * n};
    double normb = R.norm(b);
    if (normb == 0.) normb = 1;
    double normx = R.norm(x);
    R.copy(b, r.p);
    if (normx > 0.) R.spmv(-1., x, 1., r.p);
    double resid_b = R.norm(r.p) / normb;
    R.copy(r.p, r2.p);
    R.copy(r.p, p.p);
    int it = 0;
    while (resid_b > eps && it < itermax) {
        it++;
        R.copy(p.p, y.p);
        if (R.spsv(y.p)) return PASTIX_ERR_INTERNAL;
        R.spmv(1.0, y.p, 0., v.p);
        double alpha = R.dot(v.p, r2.p);
        double beta = R.dot(r.p, r2.p);
        alpha = beta / alpha;
        R.copy(r.p, s.p);
        R.axpy(-alpha, v.p, s.p);
        R.copy(s.p, z.p);
        if (R.spsv(z.p)) return PASTIX_ERR_INTERNAL;
        R.spmv(1.0, z.p, 0., t.p);
        R.copy(t.p, t2.p);
        if (R.spsv(t2.p)) return PASTIX_ERR_INTERNAL;
        double w = R.dot(t2.p, z.p) / R.dot(t2.p, t2.p);
        R.axpy(alpha, y.p, x);
        R.axpy(w, z.p, x);
        R.copy(s.p, r.p);
        R.axpy(-w, t.p, r.p);
        double v1 = R.dot(r.p, r2.p);
        double bb = (v1 / beta) * (alpha / w);
        R.axpy(-w, v.p, p.p);
        R.scal(bb, p.p);
        R.axpy(1., r.p, p.p);
        resid_b = R.norm(r.p) / normb;
    }
    iters_out = it;
    return PASTIX_SUCCESS;
}

// simple iterative refinement (refinement/z_refine_pivot.c:48-157)
static int refine_sr(Refiner &R, double *x, const double *b, double eps, int itermax, int &iters_out) {
    const int64_t n = R.n;
    if (!R.precond) return PASTIX_ERR_BADPARAMETER;
    double *wv = work(R.d, WS_VEC, (size_t)n * 2);
    if (!wv) return PASTIX_ERR_OUTOFMEMORY;
    struct { double *p; } r{wv}, dx{wv + n};
    double normb = R.norm(b);
    if (normb == 0.) normb = 1;
    int it = 0;
    double last = 0;
    while (true) {
        R.copy(b, r.p);
        R.spmv(-1., x, 1., r.p);
        double berr = R.norm(r.p) / normb;
        if (it == 0) last = 3 * berr;
        if (it < itermax && berr > eps && berr <= last / 2.) {
            R.copy(r.p, dx.p);
            if (R.spsv(dx.p)) return PASTIX_ERR_INTERNAL;
            R.axpy(1.0, dx.p, x);
            last = berr;
            it++;
        } else break;
    }
    iters_out = it;
    return PASTIX_SUCCESS;
}
}  // namespace

// Refinement of permuted device vectors x (in/out) for rhs b (one column each).
// GMRES(im) on a block of nb columns at once (permuted numbering): one Krylov
// process per column, exactly the steps of refine_gmres (right
// preconditioning, modified Gram-Schmidt, Givens rotations, per-column
// convergence test and iteration count), with every vector operation applied
// to the whole block -- one multi-column preconditioner solve, one SpMV pass
// per 8 columns, column-wise dots kept on the device -- and one host
// synchronization per iteration for the Givens step.  Columns that have
// converged keep their iterate; their Krylov vectors are carried along unused.
static int refine_gmres_block(pastix_data_t *pd, double *X, int64_t ldx, const double *B, int64_t ldb, int nb,
                              double eps, int itermax, int im, std::vector<int> &iters) {
    Device &d = pd->dev;
    const int64_t n = pd->n;
    const int im1 = im + 1;
    const int64_t blk = n * nb;  // one Krylov index for all columns
    double *V = work(d, WS_BGV, (size_t)blk * (2 * im + 2));
    double *sc = work(d, WS_BGS, (size_t)(im + 2) * nb * 2);
    if (!V || !sc) return PASTIX_ERR_OUTOFMEMORY;
    double *W = V + (size_t)blk * im1;     // preconditioned directions W_0 .. W_{im-1}
    double *Sb = W + (size_t)blk * im;     // the block solved by the preconditioner (one captured graph)
    double *hdev = sc;                     // (im + 2) x nb: Gram-Schmidt coefficients, norms
    double *fdev = sc + (size_t)(im + 2) * nb;
    auto spmm = [&](double alpha, const double *x, int64_t lx, double beta, double *y, int64_t ly) {
        launch_cls(pd, PC_SPMV, 1, [&] {
            pgpu::launch_spmm((int)n, nb, d.csr_rowptr.p, d.csr_col.p, d.csr_val.p, alpha, x, lx, beta, y, ly,
                              d.stream);
        });
    };
    auto col_norms = [&](const double *A, int64_t lda, std::vector<double> &out) -> int {
        pgpu::launch_dots_cols(n, nb, 1, A, 0, lda, A, lda, 1, hdev, d.stream);
        out.resize(nb);
        CUDA_TRY(cudaMemcpyAsync(out.data(), hdev, nb * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
        CUDA_TRY(cudaStreamSynchronize(d.stream));
        return PASTIX_SUCCESS;
    };
    std::vector<double> normb, normx, resid, hh((size_t)(im + 2) * nb), fac(nb), ycoef((size_t)im * nb);
    int rc = col_norms(B, ldb, normb);
    if (rc) return rc;
    for (auto &v : normb)
        if (v == 0.) v = 1;
    std::vector<std::vector<double>> H(nb, std::vector<double>((size_t)im * im1)), G(nb, std::vector<double>(im1)),
        gc(nb, std::vector<double>(im)), gs(nb, std::vector<double>(im));
    std::vector<char> done(nb, 0), act(nb, 0);
    std::vector<int> m(nb, 0);
    iters.assign(nb, 0);
    for (;;) {
        // V_0 = B - A X, the residual of every column
        for (int c = 0; c < nb; c++)
            CUDA_TRY(cudaMemcpyAsync(V + c * n, B + c * ldb, n * sizeof(double), cudaMemcpyDeviceToDevice, d.stream));
        spmm(-1.0, X, ldx, 1.0, V, n);
        rc = col_norms(V, n, resid);
        if (rc) return rc;
        bool any = false;
        for (int c = 0; c < nb; c++) {
            if (!done[c] && (resid[c] / normb[c] <= eps || iters[c] >= itermax)) done[c] = 1;
            act[c] = !done[c];
            any |= act[c];
            fac[c] = act[c] ? 1.0 / resid[c] : 0.0;
            G[c][0] = resid[c];
            m[c] = 0;
        }
        if (!any) break;
        CUDA_TRY(cudaMemcpyAsync(fdev, fac.data(), nb * sizeof(double), cudaMemcpyHostToDevice, d.stream));
        pgpu::launch_scal_cols(n, nb, fdev, 0, V, n, d.stream);
        for (int i = 0; i < im; i++) {
            double *Vi = V + (size_t)i * blk, *Wi = W + (size_t)i * blk, *Vn = Vi + blk;
            CUDA_TRY(cudaMemcpyAsync(Sb, Vi, (size_t)blk * sizeof(double), cudaMemcpyDeviceToDevice, d.stream));
            rc = solve_perm_d(pd, 0, Sb, (int)n, nb);
            if (rc) return rc;
            CUDA_TRY(cudaMemcpyAsync(Wi, Sb, (size_t)blk * sizeof(double), cudaMemcpyDeviceToDevice, d.stream));
            spmm(1.0, Wi, n, 0.0, Vn, n);
            for (int j = 0; j <= i; j++) {  // modified Gram-Schmidt, coefficients kept on the device
                double *hj = hdev + (size_t)j * nb;
                pgpu::launch_dots_cols(n, nb, 1, V + (size_t)j * blk, 0, n, Vn, n, 0, hj, d.stream);
                pgpu::launch_axpy_cols(n, nb, hj, V + (size_t)j * blk, n, Vn, n, d.stream);
            }
            double *hn = hdev + (size_t)(i + 1) * nb;
            pgpu::launch_dots_cols(n, nb, 1, Vn, 0, n, Vn, n, 1, hn, d.stream);
            pgpu::launch_scal_cols(n, nb, hn, 1, Vn, n, d.stream);
            CUDA_TRY(cudaMemcpyAsync(hh.data(), hdev, (size_t)(i + 2) * nb * sizeof(double), cudaMemcpyDeviceToHost,
                                     d.stream));
            CUDA_TRY(cudaStreamSynchronize(d.stream));
            bool more = false;
            for (int c = 0; c < nb; c++) {
                if (!act[c]) continue;
                double *Hi = H[c].data() + (size_t)i * im1;
                for (int j = 0; j <= i + 1; j++) Hi[j] = hh[(size_t)j * nb + c];
                for (int j = 0; j < i; j++) {
                    double t = Hi[j];
                    Hi[j] = gc[c][j] * t + gs[c][j] * Hi[j + 1];
                    Hi[j + 1] = gc[c][j] * Hi[j + 1] - gs[c][j] * t;
                }
                double t = std::sqrt(Hi[i] * Hi[i] + Hi[i + 1] * Hi[i + 1]);
                if (std::fabs(t) <= eps) t = eps;
                gc[c][i] = Hi[i] / t;
                gs[c][i] = Hi[i + 1] / t;
                G[c][i + 1] = -gs[c][i] * G[c][i];
                G[c][i] = gc[c][i] * G[c][i];
                Hi[i] = gc[c][i] * Hi[i] + gs[c][i] * Hi[i + 1];
                iters[c]++;
                m[c] = i + 1;
                if (i + 1 >= im || std::fabs(G[c][i + 1]) / normb[c] <= eps || iters[c] >= itermax) act[c] = 0;
                more |= act[c];
            }
            if (!more) break;
        }
        // X += W y with y = H^{-1} G per column (upper triangular, m[c] columns)
        std::fill(ycoef.begin(), ycoef.end(), 0.0);
        int mmax = 0;
        for (int c = 0; c < nb; c++) {
            const int mc = m[c];
            mmax = std::max(mmax, mc);
            std::vector<double> y(G[c].begin(), G[c].begin() + mc);
            for (int r = mc - 1; r >= 0; r--) {
                double t = y[r];
                for (int q = r + 1; q < mc; q++) t -= H[c][(size_t)q * im1 + r] * y[q];
                y[r] = t / H[c][(size_t)r * im1 + r];
            }
            for (int r = 0; r < mc; r++) ycoef[(size_t)r * nb + c] = y[r];
        }
        if (mmax > 0) {
            CUDA_TRY(cudaMemcpyAsync(hdev, ycoef.data(), (size_t)mmax * nb * sizeof(double), cudaMemcpyHostToDevice,
                                     d.stream));
            pgpu::launch_gemv_cols(n, nb, mmax, W, blk, hdev, X, ldx, d.stream);
        }
        for (int c = 0; c < nb; c++)
            if (iters[c] >= itermax) done[c] = 1;  // as refine_gmres: no residual test after the last cycle
    }
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    return PASTIX_SUCCESS;
}

// Preconditioned CG on a block of nb columns (permuted numbering): the steps
// of refine_cg for every column at once -- one multi-column preconditioner
// solve and one SpMV pass per 8 columns per iteration; per-column alpha and
// beta from column-wise dots (one host round trip each); a column that has
// converged gets alpha = beta = 0, so its iterate stays where it stopped.
static int refine_cg_block(pastix_data_t *pd, double *X, int64_t ldx, const double *B, int64_t ldb, int nb, double eps,
                           int itermax, std::vector<int> &iters) {
    Device &d = pd->dev;
    const int64_t n = pd->n;
    const int64_t blk = n * nb;
    double *Rb = work(d, WS_BGV, (size_t)blk * 5);
    double *sc = work(d, WS_BGS, (size_t)nb * 4);
    if (!Rb || !sc) return PASTIX_ERR_OUTOFMEMORY;
    double *Pb = Rb + blk, *Zb = Pb + blk, *Qb = Zb + blk, *Sb = Qb + blk;
    double *d0 = sc, *d1 = sc + nb, *fa = sc + 2 * nb, *fb = sc + 3 * nb;
    auto spmm = [&](double alpha, const double *x, int64_t lx, double beta, double *y) {
        launch_cls(pd, PC_SPMV, 1, [&] {
            pgpu::launch_spmm((int)n, nb, d.csr_rowptr.p, d.csr_col.p, d.csr_val.p, alpha, x, lx, beta, y, n,
                              d.stream);
        });
    };
    auto fetch = [&](const double *src, std::vector<double> &out) -> int {
        out.resize(nb);
        CUDA_TRY(cudaMemcpyAsync(out.data(), src, nb * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
        CUDA_TRY(cudaStreamSynchronize(d.stream));
        return PASTIX_SUCCESS;
    };
    auto precond = [&]() -> int {  // Z = M^{-1} R, solved in one fixed block
        CUDA_TRY(cudaMemcpyAsync(Sb, Rb, (size_t)blk * sizeof(double), cudaMemcpyDeviceToDevice, d.stream));
        int rc = solve_perm_d(pd, 0, Sb, (int)n, nb);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(Zb, Sb, (size_t)blk * sizeof(double), cudaMemcpyDeviceToDevice, d.stream));
        return PASTIX_SUCCESS;
    };
    std::vector<double> normb, resid, rz, pq, rzn, a(nb), bcoef(nb);
    pgpu::launch_dots_cols(n, nb, 1, B, 0, ldb, B, ldb, 1, d0, d.stream);
    int rc = fetch(d0, normb);
    if (rc) return rc;
    for (auto &v : normb)
        if (v == 0.) v = 1;
    for (int c = 0; c < nb; c++)
        CUDA_TRY(cudaMemcpyAsync(Rb + c * n, B + c * ldb, n * sizeof(double), cudaMemcpyDeviceToDevice, d.stream));
    spmm(-1.0, X, ldx, 1.0, Rb);
    pgpu::launch_dots_cols(n, nb, 1, Rb, 0, n, Rb, n, 1, d0, d.stream);
    if ((rc = fetch(d0, resid))) return rc;
    std::vector<char> act(nb);
    bool any = false;
    iters.assign(nb, 0);
    for (int c = 0; c < nb; c++) {
        act[c] = resid[c] / normb[c] > eps && itermax > 0;
        any |= act[c];
    }
    if (!any) return PASTIX_SUCCESS;
    if ((rc = precond())) return rc;
    CUDA_TRY(cudaMemcpyAsync(Pb, Zb, (size_t)blk * sizeof(double), cudaMemcpyDeviceToDevice, d.stream));
    pgpu::launch_dots_cols(n, nb, 1, Rb, 0, n, Zb, n, 0, d0, d.stream);
    if ((rc = fetch(d0, rz))) return rc;
    for (int it = 1; any; it++) {
        spmm(1.0, Pb, n, 0.0, Qb);
        pgpu::launch_dots_cols(n, nb, 1, Qb, 0, n, Pb, n, 0, d1, d.stream);
        if ((rc = fetch(d1, pq))) return rc;
        for (int c = 0; c < nb; c++) a[c] = act[c] ? rz[c] / pq[c] : 0.0;
        std::vector<double> na(nb);
        for (int c = 0; c < nb; c++) na[c] = -a[c];
        CUDA_TRY(cudaMemcpyAsync(fa, na.data(), nb * sizeof(double), cudaMemcpyHostToDevice, d.stream));
        CUDA_TRY(cudaMemcpyAsync(fb, a.data(), nb * sizeof(double), cudaMemcpyHostToDevice, d.stream));
        pgpu::launch_axpy_cols(n, nb, fa, Pb, n, X, ldx, d.stream);  // X += alpha P
        pgpu::launch_axpy_cols(n, nb, fb, Qb, n, Rb, n, d.stream);   // R -= alpha Q
        pgpu::launch_dots_cols(n, nb, 1, Rb, 0, n, Rb, n, 1, d0, d.stream);
        if ((rc = fetch(d0, resid))) return rc;
        any = false;
        for (int c = 0; c < nb; c++) {
            if (!act[c]) continue;
            iters[c] = it;
            if (resid[c] / normb[c] <= eps || it >= itermax) act[c] = 0;
            any |= act[c];
        }
        if (!any) break;
        if ((rc = precond())) return rc;
        pgpu::launch_dots_cols(n, nb, 1, Rb, 0, n, Zb, n, 0, d0, d.stream);
        if ((rc = fetch(d0, rzn))) return rc;
        for (int c = 0; c < nb; c++) {
            bcoef[c] = act[c] ? rzn[c] / rz[c] : 0.0;
            if (act[c]) rz[c] = rzn[c];
        }
        CUDA_TRY(cudaMemcpyAsync(fa, bcoef.data(), nb * sizeof(double), cudaMemcpyHostToDevice, d.stream));
        pgpu::launch_xpby_cols(n, nb, Zb, fa, Pb, d.stream);  // P = Z + beta P
    }
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    return PASTIX_SUCCESS;
}

static int refine_perm(pastix_data_t *pd, double *x, const double *b, int &iters);

// Refinement of nrhs permuted columns: GMRES or CG in blocks of columns (as
// many as a quarter of the free device memory holds, at most 256) when several
// right-hand sides are refined, one column at a time otherwise (the
// reference's loop, refinement/pastix_task_refine.c:121-164).
static int refine_columns(pastix_data_t *pd, double *X, int64_t ldx, const double *B, int64_t ldb, int nrhs,
                          pastix_int_t &maxit) {
    maxit = 0;
    const int method = (int)pd->iparm[IPARM_REFINEMENT];
    const bool gm = method != PastixRefineCG && method != PastixRefineSR && method != PastixRefineBiCGSTAB;
    if (nrhs > 1 && method == PastixRefineCG && pd->refine_block) {
        size_t fr = 0, tot = 0;
        CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        const size_t per_col = (size_t)pd->n * 5 * sizeof(double) + (size_t)pd->n * 12;
        const int cap = (int)std::max<size_t>(1, std::min<size_t>(256, fr / 4 / std::max<size_t>(1, per_col)));
        for (int c0 = 0; c0 < nrhs; c0 += cap) {
            const int nb = std::min(cap, nrhs - c0);
            std::vector<int> it;
            int rc = refine_cg_block(pd, X + (size_t)c0 * ldx, ldx, B + (size_t)c0 * ldb, ldb, nb,
                                     pd->dparm[DPARM_EPSILON_REFINEMENT], (int)pd->iparm[IPARM_ITERMAX], it);
            if (rc) return rc;
            for (int v : it) maxit = std::max<pastix_int_t>(maxit, v);
        }
        return PASTIX_SUCCESS;
    }
    if (nrhs > 1 && gm && pd->refine_block) {
        const int im = (int)std::max<pastix_int_t>(1, pd->iparm[IPARM_GMRES_IM]);
        size_t fr = 0, tot = 0;
        CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        const size_t per_col = (size_t)pd->n * (2 * im + 2) * sizeof(double) + (size_t)pd->n * 12;
        const int cap = (int)std::max<size_t>(1, std::min<size_t>(256, fr / 4 / std::max<size_t>(1, per_col)));
        for (int c0 = 0; c0 < nrhs; c0 += cap) {
            const int nb = std::min(cap, nrhs - c0);
            std::vector<int> it;
            int rc = refine_gmres_block(pd, X + (size_t)c0 * ldx, ldx, B + (size_t)c0 * ldb, ldb, nb,
                                        pd->dparm[DPARM_EPSILON_REFINEMENT], (int)pd->iparm[IPARM_ITERMAX], im, it);
            if (rc) return rc;
            for (int v : it) maxit = std::max<pastix_int_t>(maxit, v);
        }
        return PASTIX_SUCCESS;
    }
    for (int j = 0; j < nrhs; j++) {
        int it = 0;
        int rc = refine_perm(pd, X + (size_t)j * ldx, B + (size_t)j * ldb, it);
        if (rc) return rc;
        maxit = std::max<pastix_int_t>(maxit, it);
    }
    return PASTIX_SUCCESS;
}

static int refine_perm(pastix_data_t *pd, double *x, const double *b, int &iters) {
    Refiner R(pd);
    double eps = pd->dparm[DPARM_EPSILON_REFINEMENT];
    int itermax = (int)pd->iparm[IPARM_ITERMAX];
    switch (pd->iparm[IPARM_REFINEMENT]) {
        case PastixRefineCG: return refine_cg(R, x, b, eps, itermax, iters);
        case PastixRefineSR: return refine_sr(R, x, b, eps, itermax, iters);
        case PastixRefineBiCGSTAB: return refine_bicgstab(R, x, b, eps, itermax, iters);
        default: return refine_gmres(R, x, b, eps, itermax, (int)std::max<pastix_int_t>(1, pd->iparm[IPARM_GMRES_IM]), iters);
    }
}

extern "C" int pastix_subtask_refine(pastix_data_t *pd, pastix_rhs_t Bp, pastix_rhs_t Xp) {
    if (!pd || !(pd->steps & STEP_CSC2BCSC) || !Bp || !Xp || !Bp->b || !Xp->b) return PASTIX_ERR_BADPARAMETER;
    if (Bp->flttype != SpmDouble || Xp->flttype != SpmDouble) return PASTIX_ERR_BADPARAMETER;
    if (pd->dparm[DPARM_EPSILON_REFINEMENT] < 0.) pd->dparm[DPARM_EPSILON_REFINEMENT] = 1e-12;  // FP64 input
    CUDA_TRY(cudaSetDevice(pd->dev.dev));
    double t0 = now_s();
    pd->iparm[IPARM_NBITER] = 0;
    pastix_int_t maxit = 0;
    int rc = refine_columns(pd, (double *)Xp->b, Xp->ld, (const double *)Bp->b, Bp->ld, (int)Bp->n, maxit);
    if (rc) return rc;
    pd->iparm[IPARM_NBITER] = maxit;
    CUDA_TRY(cudaStreamSynchronize(pd->dev.stream));
    pd->dparm[DPARM_REFINE_TIME] = now_s() - t0;
    return PASTIX_SUCCESS;
}

extern "C" int pastix_task_refine(pastix_data_t *pd, pastix_int_t n, pastix_int_t nrhs, void *B, pastix_int_t ldb,
                                  void *X, pastix_int_t ldx) {
    if (!pd || !(pd->steps & STEP_CSC2BCSC)) {
        perr("pastix_task_refine: the matrix values must be given first (pastix_task_numfact)");
        return PASTIX_ERR_BADPARAMETER;
    }
    if (n != pd->n || nrhs < 1 || ldb < n || ldx < n || !B || !X) return PASTIX_ERR_BADPARAMETER;
    int rc = device_setup(pd);
    if (rc) return rc;
    struct pastix_rhs_s Bs{}, Xs{};  // permuted copies in the library's work areas
    Bs.flttype = Xs.flttype = SpmDouble;
    Bs.m = Xs.m = n;
    Bs.n = Xs.n = nrhs;
    Bs.ld = Xs.ld = n;
    Bs.b = work(pd->dev, WS_RB, (size_t)n * nrhs);
    Xs.b = work(pd->dev, WS_RX, (size_t)n * nrhs);
    if (!Bs.b || !Xs.b) return PASTIX_ERR_OUTOFMEMORY;
    rc = pastix_subtask_applyorder(pd, PastixDirForward, n, nrhs, B, ldb, &Bs);
    if (!rc) rc = pastix_subtask_applyorder(pd, PastixDirForward, n, nrhs, X, ldx, &Xs);
    if (!rc) rc = pastix_subtask_refine(pd, &Bs, &Xs);
    if (!rc) rc = pastix_subtask_applyorder(pd, PastixDirBackward, n, nrhs, X, ldx, &Xs);
    return rc;
}

extern "C" int pastix_task_solve_and_refine(pastix_data_t *pd, pastix_int_t n, pastix_int_t nrhs, void *B,
                                            pastix_int_t ldb, void *X, pastix_int_t ldx) {
    if (!pd || !B || !X || ldx < n || ldb < n) return PASTIX_ERR_BADPARAMETER;
    for (pastix_int_t j = 0; j < nrhs; j++)
        memcpy((double *)X + j * ldx, (const double *)B + j * ldb, n * sizeof(double));
    int rc = pastix_task_solve(pd, n, nrhs, X, ldx);
    if (rc) return rc;
    return pastix_task_refine(pd, n, nrhs, B, ldb, X, ldx);
}

// ---------------------------------------------------------------------------
// adjoint helpers and device SpMV in the original numbering
// ---------------------------------------------------------------------------
extern "C" int pgpu_sampled_outer(pastix_data_t *pd, double alpha, const double *lambda, const double *x, double *G,
                                  void *stream) {
    if (!pd || !pd->dev.ready || !lambda || !x || !G) return PASTIX_ERR_BADPARAMETER;
    CUDA_TRY(cudaSetDevice(pd->dev.dev));
    cudaStream_t st = (cudaStream_t)stream;  // the caller's stream; NULL = legacy default stream
    launch_cls(pd, PC_VEC, 1, [&] {
        pgpu::launch_sampled(pd->nnz, pd->dev.e_row.p, pd->dev.e_col.p, alpha, lambda, x, G,
                             pd->mtxtype == SpmSymmetric ? 1 : 0, st);
    });
    CUDA_TRY(cudaGetLastError());
    return PASTIX_SUCCESS;
}

extern "C" int pgpu_spmv_device(pastix_data_t *pd, double alpha, const double *x, double beta, double *y,
                                void *stream) {
    if (!pd || !(pd->steps & STEP_CSC2BCSC) || !x || !y) return PASTIX_ERR_BADPARAMETER;
    Device &d = pd->dev;
    CUDA_TRY(cudaSetDevice(d.dev));
    if (d.w1.n < (size_t)pd->n) CUDA_TRY(d.w1.alloc(pd->n));
    if (d.w2.n < (size_t)pd->n) CUDA_TRY(d.w2.alloc(pd->n));
    CUDA_TRY(cudaStreamSynchronize(d.stream));  // the work vectors are shared with the library stream
    cudaStream_t st = (cudaStream_t)stream;     // the caller's stream; NULL = legacy default stream
    pgpu::launch_permute<double, double>((int)pd->n, 1, d.perm.p, 1, x, pd->n, d.w1.p, pd->n, st);
    pgpu::launch_permute<double, double>((int)pd->n, 1, d.perm.p, 1, y, pd->n, d.w2.p, pd->n, st);
    launch_cls(pd, PC_SPMV, 1, [&] {
        pgpu::launch_spmv_stream(d.spmv_nblocks, d.spmv_part.p, d.csr_rowptr.p, d.csr_col.p, d.csr_val.p, alpha,
                                 d.w1.p, beta, d.w2.p, st);
    }, st ? st : cudaStreamLegacy);
    pgpu::launch_permute<double, double>((int)pd->n, 1, d.perm.p, 0, d.w2.p, pd->n, y, pd->n, st);
    CUDA_TRY(cudaGetLastError());
    return PASTIX_SUCCESS;
}

// ---------------------------------------------------------------------------
// legacy one-call interface (sopalin/pastix.c:103-541), tasks START..END
// ---------------------------------------------------------------------------
extern "C" int pastix(pastix_data_t **pdp, PASTIX_Comm comm, pastix_int_t n, pastix_int_t *colptr, pastix_int_t *rowptr,
                      void *values, pastix_int_t *perm, pastix_int_t *invp, void *B, pastix_int_t nrhs,
                      pastix_int_t *iparm, double *dparm) {
    if (!pdp || !iparm || !dparm) return PASTIX_ERR_BADPARAMETER;
    if (iparm[IPARM_MODIFY_PARAMETER] == 0) {
        pastixInitParam(iparm, dparm);
        iparm[IPARM_MODIFY_PARAMETER] = 1;
        return PASTIX_SUCCESS;
    }
    if (!*pdp) {
        pastixInit(pdp, comm, iparm, dparm);
        if (!*pdp) return PASTIX_ERR_ALLOC;
    }
    pastix_data_t *pd = *pdp;
    spmatrix_t spm;
    memset(&spm, 0, sizeof(spm));
    spm.mtxtype = (iparm[IPARM_MTX_TYPE] == SpmSymmetric ||
                   (iparm[IPARM_MTX_TYPE] == -1 && iparm[IPARM_FACTORIZATION] != PastixFactLU))
                      ? SpmSymmetric : SpmGeneral;
    spm.flttype = SpmDouble;
    spm.fmttype = SpmCSC;
    spm.baseval = colptr ? colptr[0] : 0;
    spm.n = spm.gN = n;
    spm.nnz = spm.gnnz = colptr ? colptr[n] - spm.baseval : 0;
    spm.dof = 1;
    spm.colptr = colptr;
    spm.rowptr = rowptr;
    spm.values = values;
    int start = (int)iparm[IPARM_START_TASK], end = (int)iparm[IPARM_END_TASK];
    int rc = PASTIX_SUCCESS;
    if (start <= PastixTaskOrdering && end >= PastixTaskOrdering) {
        pastix_order_t ord;
        memset(&ord, 0, sizeof(ord));
        pastix_order_t *po = nullptr;
        if (iparm[IPARM_ORDERING] == PastixOrderPersonal && perm) {
            ord.vertnbr = n;
            ord.baseval = 0;
            ord.permtab = perm;
            ord.peritab = invp;
            po = &ord;
        }
        rc = pastix_subtask_order(pd, &spm, po);
        if (!rc && perm && iparm[IPARM_ORDERING] != PastixOrderPersonal)
            for (pastix_int_t i = 0; i < n; i++) {
                perm[i] = pd->order.permtab[i];
                if (invp) invp[i] = pd->order.peritab[i];
            }
    }
    if (!rc && start <= PastixTaskSymbfact && end >= PastixTaskSymbfact) rc = pastix_subtask_symbfact(pd);
    if (!rc && start <= PastixTaskAnalyze && end >= PastixTaskAnalyze) rc = pastix_subtask_blend(pd);
    if (!rc && start <= PastixTaskNumfact && end >= PastixTaskNumfact) rc = pastix_task_numfact(pd, &spm);
    if (!rc && start <= PastixTaskSolve && end >= PastixTaskSolve && B && nrhs > 0) {
        std::vector<double> b0((size_t)n * nrhs);
        memcpy(b0.data(), B, b0.size() * sizeof(double));
        rc = pastix_task_solve(pd, n, nrhs, B, n);
        if (!rc && start <= PastixTaskRefine && end >= PastixTaskRefine)
            rc = pastix_task_refine(pd, n, nrhs, b0.data(), n, B, n);
    }
    if (!rc && end >= PastixTaskClean) pastixFinalize(pdp);
    return rc;
}

// ---------------------------------------------------------------------------
// B200 extensions: stream, refinement on device, launch accounting
// ---------------------------------------------------------------------------
extern "C" void *pgpu_stream(pastix_data_t *pd) {
    if (!pd || !(pd->steps & STEP_ANALYSE)) return nullptr;
    if (device_setup(pd) != PASTIX_SUCCESS) return nullptr;
    return (void *)pd->dev.stream;
}

extern "C" int pgpu_solve_refine_device(pastix_data_t *pd, pastix_int_t nrhs, const double *B, pastix_int_t ldb,
                                        double *X, pastix_int_t ldx) {
    int rc = check_numfact(pd, "pgpu_solve_refine_device");
    if (rc) return rc;
    if (nrhs < 1 || ldb < pd->n || ldx < pd->n || !B || !X) return PASTIX_ERR_BADPARAMETER;
    Device &d = pd->dev;
    CUDA_TRY(cudaSetDevice(d.dev));
    const idx_t n = pd->n;
    struct { double *p; } bp{work(d, WS_BP, (size_t)n * nrhs)}, xp{work(d, WS_XP, (size_t)n * nrhs)};
    if (!bp.p || !xp.p) return PASTIX_ERR_OUTOFMEMORY;
    launch_cls(pd, PC_VEC, 1, [&] { pgpu::launch_permute<double, double>((int)n, (int)nrhs, d.perm.p, 1, B, ldb, bp.p, n, d.stream); });
    CUDA_TRY(cudaMemcpyAsync(xp.p, bp.p, (size_t)n * nrhs * 8, cudaMemcpyDeviceToDevice, d.stream));
    rc = solve_perm_d(pd, 0, xp.p, (int)n, (int)nrhs);
    if (rc) return rc;
    if (pd->dparm[DPARM_EPSILON_REFINEMENT] < 0.) pd->dparm[DPARM_EPSILON_REFINEMENT] = 1e-12;
    double t0 = now_s();
    pd->iparm[IPARM_NBITER] = 0;
    pastix_int_t maxit = 0;
    rc = refine_columns(pd, xp.p, n, bp.p, n, (int)nrhs, maxit);
    if (rc) return rc;
    pd->iparm[IPARM_NBITER] = maxit;
    launch_cls(pd, PC_VEC, 1, [&] { pgpu::launch_permute<double, double>((int)n, (int)nrhs, d.perm.p, 0, xp.p, n, X, ldx, d.stream); });
    CUDA_TRY(cudaStreamSynchronize(d.stream));
    pd->dparm[DPARM_REFINE_TIME] = now_s() - t0;
    return PASTIX_SUCCESS;
}

// Rebuild the launch lists after a change of the tile buckets; the device
// copy and every captured graph are rebuilt on the next numerical step.
static int retune(pastix_data_t *pd, int dmma_n, int dmma_k, int tc_k) {
    if (pd->dev.ready) CUDA_TRY(cudaStreamSynchronize(pd->dev.stream));
    pd->tune_dmma_n = dmma_n;
    pd->tune_dmma_k = dmma_k;
    pd->tune_tc_k = tc_k;
    int rc = build_maps_and_lists(pd);
    if (rc) return rc;
    pd->dev.ready = false;
    pd->steps &= ~(STEP_CSC2BCSC | STEP_BCSC2CTAB | STEP_NUMFACT);
    return PASTIX_SUCCESS;
}

extern "C" int pgpu_set_tuning(pastix_data_t *pd, pastix_int_t dmma_n, pastix_int_t dmma_k, pastix_int_t tc_k) {
    if (!pd || !(pd->steps & STEP_ANALYSE)) return PASTIX_ERR_BADPARAMETER;
    if (dmma_n < 1 || dmma_k < 1 || tc_k < 32) return PASTIX_ERR_BADPARAMETER;  // tcgen05 tiles need K >= 32
    return retune(pd, (int)dmma_n, (int)dmma_k, (int)tc_k);
}

extern "C" int pgpu_get_tuning(const pastix_data_t *pd, pastix_int_t *vals) {
    if (!pd || !vals) return PASTIX_ERR_BADPARAMETER;
    vals[0] = pd->tune_dmma_n;
    vals[1] = pd->tune_dmma_k;
    vals[2] = pd->tune_tc_k;
    return PASTIX_SUCCESS;
}

// Autotuner of the update tile buckets: for the factor precision in use, every
// candidate bucket boundary is applied (launch lists rebuilt), the matrix is
// factorized from the device values twice and the faster run's device time
// kept; the fastest candidate stays in effect, with the factorization done.
extern "C" int pgpu_autotune(pastix_data_t *pd, const double *values_dev, pastix_int_t *chosen) {
    if (!pd || !values_dev || !(pd->steps & STEP_ANALYSE)) return PASTIX_ERR_BADPARAMETER;
    if (pd->prof_on) {
        perr("pgpu_autotune: not available while pgpu_profile timing is enabled");
        return PASTIX_ERR_BADPARAMETER;
    }
    pd->mixed = pd->iparm[IPARM_MIXED] ? 1 : 0;
    std::vector<std::array<int, 3>> cands;
    if (pd->mixed) {
        for (int tk : {32, 48, 64, 96}) cands.push_back({pd->tune_dmma_n, pd->tune_dmma_k, tk});
    } else {
        for (int n : {8, 16, 32, 64})
            for (int k : {16, 32}) cands.push_back({n, k, pd->tune_tc_k});
    }
    // the buckets in effect are timed first; another candidate replaces them only when it is
    // at least 2 % faster (run-to-run noise of a factorization is about that)
    const std::array<int, 3> cur{pd->tune_dmma_n, pd->tune_dmma_k, pd->tune_tc_k};
    cands.erase(std::remove(cands.begin(), cands.end(), cur), cands.end());
    cands.insert(cands.begin(), cur);
    double best = 1e300;
    std::array<int, 3> arg = cur;
    for (const auto &c : cands) {
        int rc = retune(pd, c[0], c[1], c[2]);
        if (rc) return rc;
        double t = 1e300;
        for (int rep = 0; rep < 3; rep++) {  // the first run also allocates and captures
            rc = pgpu_numfact_device(pd, values_dev);
            if (rc) return rc;
            if (rep) t = std::min(t, pd->dparm[DPARM_FACT_TIME]);
        }
        if (c == cur) {
            best = t;
        } else if (t < 0.98 * best) {
            best = t;
            arg = c;
        }
    }
    int rc = retune(pd, arg[0], arg[1], arg[2]);
    if (rc) return rc;
    rc = pgpu_numfact_device(pd, values_dev);
    if (rc) return rc;
    if (chosen) {
        chosen[0] = arg[0];
        chosen[1] = arg[1];
        chosen[2] = arg[2];
    }
    return PASTIX_SUCCESS;
}

extern "C" int pgpu_refine_block(pastix_data_t *pd, int enable) {
    if (!pd) return PASTIX_ERR_BADPARAMETER;
    pd->refine_block = enable != 0;
    return PASTIX_SUCCESS;
}

extern "C" int pgpu_graphs(pastix_data_t *pd, int enable) {
    if (!pd) return PASTIX_ERR_BADPARAMETER;
    if (pd->dev.ready) CUDA_TRY(cudaStreamSynchronize(pd->dev.stream));
    pd->graphs.clear();
    pd->use_graphs = enable != 0;
    return PASTIX_SUCCESS;
}

extern "C" int pgpu_profile(pastix_data_t *pd, int enable) {
    if (!pd) return PASTIX_ERR_BADPARAMETER;
    for (auto &e : pd->prof_ev) {
        cudaEventDestroy(e.second.first);
        cudaEventDestroy(e.second.second);
    }
    pd->prof_ev.clear();
    for (int i = 0; i < PGPU_NCLASS; i++) { pd->prof_ms[i] = 0; pd->launches[i] = 0; }
    pd->prof_on = enable != 0;
    return PASTIX_SUCCESS;
}

extern "C" int pgpu_profile_get(pastix_data_t *pd, double *ms, long long *launches, int nclass) {
    if (!pd || nclass < 1) return PASTIX_ERR_BADPARAMETER;
    if (pd->dev.ready) CUDA_TRY(cudaStreamSynchronize(pd->dev.stream));
    for (auto &e : pd->prof_ev) {
        float t = 0;
        CUDA_TRY(cudaEventElapsedTime(&t, e.second.first, e.second.second));
        pd->prof_ms[e.first] += t;
        cudaEventDestroy(e.second.first);
        cudaEventDestroy(e.second.second);
    }
    pd->prof_ev.clear();
    for (int i = 0; i < nclass && i < PGPU_NCLASS; i++) {
        if (ms) ms[i] = pd->prof_ms[i];
        if (launches) launches[i] = pd->launches[i];
    }
    return PASTIX_SUCCESS;
}

// ---------------------------------------------------------------------------
// Import of an analysis computed elsewhere (the reference's own
// pastix_task_analyze): the ordering and the block symbolic structure of its
// SolverMatrix, taken as plain arrays.  Replaces pastix_subtask_order /
// symbfact / reordering / blend for the given spm pattern.
// ---------------------------------------------------------------------------
extern "C" int pgpu_set_symbol(pastix_data_t *pd, const spmatrix_t *spm, const pastix_int_t *permtab,
                               pastix_int_t cblknbr, const pastix_int_t *cb_fcol, const pastix_int_t *cb_lcol,
                               const pastix_int_t *cb_fblok, pastix_int_t bloknbr, const pastix_int_t *bk_frow,
                               const pastix_int_t *bk_lrow, const pastix_int_t *bk_fcblk) {
    if (!pd || !spm || !permtab || cblknbr < 1 || bloknbr < cblknbr || !cb_fcol || !cb_lcol || !cb_fblok || !bk_frow ||
        !bk_lrow || !bk_fcblk)
        return PASTIX_ERR_BADPARAMETER;
    // pattern (and graph) as in pastix_subtask_order, with the given permutation
    pastix_order_t ord;
    memset(&ord, 0, sizeof(ord));
    ord.vertnbr = spm->n;
    ord.permtab = const_cast<pastix_int_t *>(permtab);
    std::vector<pastix_int_t> rang{0, spm->n}, tree{-1};
    ord.cblknbr = 1;
    ord.rangtab = rang.data();
    ord.treetab = tree.data();
    pastix_int_t saved = pd->iparm[IPARM_ORDERING];
    pd->iparm[IPARM_ORDERING] = PastixOrderPersonal;
    int rc = pastix_subtask_order(pd, spm, &ord);
    pd->iparm[IPARM_ORDERING] = saved;
    if (rc) return rc;
    pgpu::Symbol &sy = pd->symbol;
    sy = pgpu::Symbol{};
    sy.nodenbr = spm->n;
    sy.cblktab.resize(cblknbr + 1);
    for (pastix_int_t k = 0; k < cblknbr; k++) sy.cblktab[k] = pgpu::SymCblk{cb_fcol[k], cb_lcol[k], cb_fblok[k]};
    sy.cblktab[cblknbr] = pgpu::SymCblk{spm->n, spm->n - 1, bloknbr};
    sy.bloktab.resize(bloknbr);
    for (pastix_int_t k = 0; k < cblknbr; k++) {
        pastix_int_t be = (k + 1 < cblknbr) ? cb_fblok[k + 1] : bloknbr;
        if (cb_fblok[k] < 0 || be > bloknbr || be <= cb_fblok[k]) return PASTIX_ERR_BADPARAMETER;
        for (pastix_int_t b = cb_fblok[k]; b < be; b++)
            sy.bloktab[b] = pgpu::SymBlok{bk_frow[b], bk_lrow[b], k, bk_fcblk[b]};
    }
    std::string err = pgpu::symbol_check(sy);
    if (!err.empty()) { perr("pgpu_set_symbol: structure check failed: %s", err.c_str()); return PASTIX_ERR_BADPARAMETER; }
    pd->factotype = (int)pd->iparm[IPARM_FACTORIZATION];
    int fk = fact_kind(pd);
    pgpu::solver_build(pd->solver, sy, fk);
    rc = build_maps_and_lists(pd);
    if (rc) return rc;
    pd->dparm[DPARM_FACT_THFLOPS] = pd->solver.thflops;
    pd->iparm[IPARM_NNZEROS] = pd->solver.nnzl * (fk == pgpu::FACT_GETRF ? 2 : 1);
    pd->steps = STEP_INIT | STEP_ORDERING | STEP_SYMBFACT | STEP_ANALYSE;
    pd->dev.ready = false;
    return PASTIX_SUCCESS;
}

// ---------------------------------------------------------------------------
// Device solve with no allocation.  Some callers cannot allocate device
// memory at call time: code running inside a region that must not
// synchronize (cudaMalloc / cudaFree serialize against every stream of the
// device), or an application that reserves the whole heap up front.  This
// variant of pgpu_solve_device takes its permuted work vector (and the float
// copy of the mixed-precision path) from a fixed array in the module's global
// memory instead of the grow-only work areas of pgpu_solve_device.  The first
// call on a device looks the array's address up and creates the ordering
// event; later calls on that device only launch kernels.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kStaticElems = PGPU_STATIC_SOLVE_ELEMS;
// kStaticElems FP64 elements followed by kStaticElems FP32 elements.  Nothing
// in it has to start at zero: every element a call reads is written earlier in
// the same call (the permute fills the FP64 part, the cast the FP32 part).
static __device__ __align__(256) unsigned char g_static_solve[kStaticElems * (sizeof(double) + sizeof(float))];

constexpr int kMaxDevices = 64;
struct StaticSolveSlot {
    bool ready = false;
    unsigned char *base = nullptr;  // address of g_static_solve in this device's context
    cudaEvent_t ev = nullptr;       // orders the library stream with the caller's stream
};
static StaticSolveSlot g_static_slots[kMaxDevices];
static std::mutex g_static_mutex;

// Set-up of the device current on this thread.
static int static_solve_setup(int dev, StaticSolveSlot **out) {
    if (dev < 0 || dev >= kMaxDevices) return PASTIX_ERR_BADPARAMETER;
    std::lock_guard<std::mutex> lock(g_static_mutex);
    StaticSolveSlot &s = g_static_slots[dev];
    if (!s.ready) {
        void *p = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&p, g_static_solve));
        CUDA_TRY(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
        s.base = static_cast<unsigned char *>(p);
        s.ready = true;
    }
    *out = &s;
    return PASTIX_SUCCESS;
}
}  // namespace

extern "C" int pgpu_solve_device_static(pastix_data_t *pd, pastix_int_t nrhs, double *B, pastix_int_t ldb,
                                        void *stream) {
    int rc = check_numfact(pd, "pgpu_solve_device_static");
    if (rc) return rc;
    if (nrhs < 1 || ldb < pd->n || !B) return PASTIX_ERR_BADPARAMETER;
    const size_t need = (size_t)pd->n * (size_t)nrhs;
    if (need > kStaticElems) {
        perr("pgpu_solve_device_static: n * nrhs = %zu exceeds the fixed work array of %zu elements "
             "(use pgpu_solve_device)", need, kStaticElems);
        return PASTIX_ERR_BADPARAMETER;
    }
    if (pd->prof_on) {  // timed launch accounting creates events and grows a host list
        perr("pgpu_solve_device_static: not available while pgpu_profile timing is enabled");
        return PASTIX_ERR_BADPARAMETER;
    }
    Device &d = pd->dev;
    CUDA_TRY(cudaSetDevice(d.dev));
    StaticSolveSlot *slot = nullptr;
    rc = static_solve_setup(d.dev, &slot);
    if (rc) return rc;
    double *Y = reinterpret_cast<double *>(slot->base);
    float *Yf = reinterpret_cast<float *>(slot->base + kStaticElems * sizeof(double));
    const idx_t n = pd->n;
    cudaStream_t user = (cudaStream_t)stream;
    if (user != d.stream) {
        if (cudaEventRecord(slot->ev, user) != cudaSuccess) {
            // the cached event (and symbol address) belong to a context that is
            // gone, e.g. after a device reset: redo the set-up on the next call
            std::lock_guard<std::mutex> lock(g_static_mutex);
            slot->ready = false;
            perr("pgpu_solve_device_static: ordering event unusable (device reset?)");
            return PASTIX_ERR_INTERNAL;
        }
        CUDA_TRY(cudaStreamWaitEvent(d.stream, slot->ev, 0));
    }
    pgpu::launch_permute<double, double>((int)n, (int)nrhs, d.perm.p, 1, B, ldb, Y, n, d.stream);
    if (!pd->mixed) {
        solve_perm<double>(pd, 0, Y, (int)n, (int)nrhs);
    } else {
        for (int j = 0; j < nrhs; j++)
            pgpu::launch_cast<double, float>(n, Y + (size_t)j * n, Yf + (size_t)j * n, d.stream);
        solve_perm<float>(pd, 0, Yf, (int)n, (int)nrhs);
        for (int j = 0; j < nrhs; j++)
            pgpu::launch_cast<float, double>(n, Yf + (size_t)j * n, Y + (size_t)j * n, d.stream);
    }
    pgpu::launch_permute<double, double>((int)n, (int)nrhs, d.perm.p, 0, Y, n, B, ldb, d.stream);
    if (user != d.stream) {
        CUDA_TRY(cudaEventRecord(slot->ev, d.stream));
        CUDA_TRY(cudaStreamWaitEvent(user, slot->ev, 0));
    }
    CUDA_TRY(cudaGetLastError());
    return PASTIX_SUCCESS;
}
