/*
 * pastix_b200.h -- C ABI of the B200 numerical phase for PaStiX.
 *
 * The library is a drop-in for the numerical half of PaStiX 6.4: it keeps the
 * public entry points of include/pastix.h (pastixInit, pastix_task_numfact,
 * pastix_task_solve, pastix_task_refine, pastix(), the numeric subtasks) with
 * the same argument meaning, the same iparm/dparm indices and the same error
 * codes, and runs the factorization, the triangular solves, the residual SpMV
 * and the refinement as CUDA kernels for sm_100a on one GPU.  There is no CPU
 * fallback: every numerical entry point returns PASTIX_ERR_INTERNAL when no
 * CUDA device can be used.
 *
 * Enumerations, parameter indices and the order structure below restate the
 * reference's interface (include/pastix/api.h, include/pastix/order.h,
 * include/pastix/datatypes.h); their names and numeric values must stay
 * identical for binary compatibility of iparm/dparm arrays.  spmatrix_t
 * restates the fields of the SpM library's matrix descriptor that PaStiX reads
 * (the spm submodule itself is not part of the reference checkout).
 */
#ifndef PASTIX_B200_H
#define PASTIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int64_t pastix_int_t;   /* PASTIX_INT64 build (include/pastix/datatypes.h:30) */
typedef int     PASTIX_Comm;    /* single process: the communicator is a placeholder  */

/* ---- SpM descriptor (restated; fields used by pastix_task_* of the reference) ---- */
typedef enum spm_coeftype_e {
    SpmPattern = 0, SpmFloat = 2, SpmDouble = 3, SpmComplex32 = 4, SpmComplex64 = 5
} spm_coeftype_t;
typedef enum spm_mtxtype_e {
    SpmGeneral = 111, SpmSymmetric = 112, SpmHermitian = 113
} spm_mtxtype_t;
typedef enum spm_fmttype_e { SpmCSC = 0, SpmCSR = 1, SpmIJV = 2 } spm_fmttype_t;

typedef struct spmatrix_s {
    spm_mtxtype_t  mtxtype;   /* SpmGeneral or SpmSymmetric                               */
    spm_coeftype_t flttype;   /* SpmDouble (SpmFloat input is promoted)                   */
    spm_fmttype_t  fmttype;   /* SpmCSC                                                   */
    pastix_int_t   baseval;   /* 0 or 1                                                   */
    pastix_int_t   gN;        /* global size                                              */
    pastix_int_t   n;         /* local size (= gN, one process)                           */
    pastix_int_t   gnnz;
    pastix_int_t   nnz;       /* stored entries; symmetric: one triangle                  */
    pastix_int_t   gNexp, nexp, gnnzexp, nnzexp;
    pastix_int_t   dof;       /* 1: scalar entries (expanded matrices are given scalar)   */
    pastix_int_t  *dofs;
    int            layout;
    pastix_int_t  *colptr;    /* n+1                                                      */
    pastix_int_t  *rowptr;    /* nnz                                                      */
    pastix_int_t  *loc2glob;
    void          *values;    /* nnz                                                      */
    pastix_int_t  *glob2loc;
    int            clustnum, clustnbr;
    PASTIX_Comm    comm;
    int            replicated;
} spmatrix_t;

/* ---- parameters (include/pastix/api.h:35-187, same order and values) ---- */
typedef enum pastix_iparm_e {
    IPARM_VERBOSE, IPARM_IO_STRATEGY,
    IPARM_NNZEROS, IPARM_NNZEROS_BLOCK_LOCAL, IPARM_ALLOCATED_TERMS, IPARM_PRODUCE_STATS, IPARM_TRACE,
    IPARM_MC64,
    IPARM_ORDERING, IPARM_ORDERING_DEFAULT,
    IPARM_SCOTCH_MT, IPARM_SCOTCH_SWITCH_LEVEL, IPARM_SCOTCH_CMIN, IPARM_SCOTCH_CMAX, IPARM_SCOTCH_FRAT,
    IPARM_METIS_CTYPE, IPARM_METIS_RTYPE, IPARM_METIS_NO2HOP, IPARM_METIS_NSEPS, IPARM_METIS_NITER,
    IPARM_METIS_UFACTOR, IPARM_METIS_COMPRESS, IPARM_METIS_CCORDER, IPARM_METIS_PFACTOR,
    IPARM_METIS_SEED, IPARM_METIS_DBGLVL,
    IPARM_AMALGAMATION_LVLBLAS, IPARM_AMALGAMATION_LVLCBLK,
    IPARM_REORDERING_SPLIT, IPARM_REORDERING_STOP, IPARM_SPLITTING_STRATEGY,
    IPARM_SPLITTING_LEVELS_PROJECTIONS, IPARM_SPLITTING_LEVELS_KWAY,
    IPARM_SPLITTING_PROJECTIONS_DEPTH, IPARM_SPLITTING_PROJECTIONS_DISTANCE,
    IPARM_SPLITTING_PROJECTIONS_WIDTH,
    IPARM_MIN_BLOCKSIZE, IPARM_MAX_BLOCKSIZE, IPARM_TASKS2D_LEVEL, IPARM_TASKS2D_WIDTH, IPARM_ALLCAND,
    IPARM_INCOMPLETE, IPARM_LEVEL_OF_FILL,
    IPARM_FACTORIZATION, IPARM_FACTO_LOOK_SIDE, IPARM_STATIC_PIVOTING, IPARM_FREE_CSCUSER,
    IPARM_SCHUR_FACT_MODE,
    IPARM_TRANSPOSE_SOLVE, IPARM_SCHUR_SOLV_MODE, IPARM_APPLYPERM_WS,
    IPARM_REFINEMENT, IPARM_NBITER, IPARM_ITERMAX, IPARM_GMRES_IM,
    IPARM_SCHEDULER, IPARM_THREAD_NBR, IPARM_SOCKET_NBR, IPARM_AUTOSPLIT_COMM,
    IPARM_GPU_NBR, IPARM_GPU_MEMORY_PERCENTAGE, IPARM_GPU_MEMORY_BLOCK_SIZE, IPARM_GLOBAL_ALLOCATION,
    IPARM_COMPRESS_MIN_WIDTH, IPARM_COMPRESS_MIN_HEIGHT, IPARM_COMPRESS_WHEN, IPARM_COMPRESS_METHOD,
    IPARM_COMPRESS_ORTHO, IPARM_COMPRESS_RELTOL, IPARM_COMPRESS_PRESELECT, IPARM_COMPRESS_ILUK,
    IPARM_MIXED, IPARM_FTZ,
    IPARM_MPI_THREAD_LEVEL,
    IPARM_MODIFY_PARAMETER, IPARM_START_TASK, IPARM_END_TASK, IPARM_FLOAT, IPARM_MTX_TYPE, IPARM_DOF_NBR,
    IPARM_SIZE
} pastix_iparm_t;

typedef enum pastix_dparm_e {
    DPARM_FILL_IN, DPARM_EPSILON_REFINEMENT, DPARM_RELATIVE_ERROR, DPARM_EPSILON_MAGN_CTRL,
    DPARM_ORDER_TIME, DPARM_SYMBFACT_TIME, DPARM_REORDER_TIME, DPARM_BLEND_TIME, DPARM_ANALYZE_TIME,
    DPARM_PRED_FACT_TIME, DPARM_FACT_TIME, DPARM_FACT_FLOPS, DPARM_FACT_THFLOPS, DPARM_FACT_RLFLOPS,
    DPARM_FACT_ENERGY, DPARM_MEM_FR, DPARM_MEM_LR, DPARM_SOLV_TIME, DPARM_SOLV_FLOPS,
    DPARM_SOLV_THFLOPS, DPARM_SOLV_RLFLOPS, DPARM_SOLV_ENERGY, DPARM_REFINE_TIME, DPARM_A_NORM,
    DPARM_COMPRESS_TOLERANCE, DPARM_COMPRESS_MIN_RATIO,
    DPARM_SIZE
} pastix_dparm_t;

typedef enum pastix_task_e {
    PastixTaskInit = 0, PastixTaskOrdering = 1, PastixTaskSymbfact = 2, PastixTaskAnalyze = 3,
    PastixTaskNumfact = 4, PastixTaskSolve = 5, PastixTaskRefine = 6, PastixTaskClean = 7
} pastix_task_t;

typedef enum pastix_verbose_e { PastixVerboseNot = 0, PastixVerboseNo = 1, PastixVerboseYes = 2 } pastix_verbose_t;

typedef enum pastix_refine_e {
    PastixRefineGMRES, PastixRefineCG, PastixRefineSR, PastixRefineBiCGSTAB
} pastix_refine_t;

typedef enum pastix_factotype_e {
    PastixFactPOTRF = 0, PastixFactSYTRF = 1, PastixFactGETRF = 2, PastixFactPXTRF = 3,
    PastixFactHETRF = 4,
    PastixFactLLH = 0, PastixFactLDLT = 1, PastixFactLU = 2, PastixFactLLT = 3, PastixFactLDLH = 4
} pastix_factotype_t;

typedef enum pastix_scheduler_e {
    PastixSchedSequential = 0, PastixSchedStatic = 1, PastixSchedParsec = 2,
    PastixSchedStarPU = 3, PastixSchedDynamic = 4
} pastix_scheduler_t;

typedef enum pastix_ordering_e {
    PastixOrderScotch, PastixOrderMetis, PastixOrderPersonal, PastixOrderPtScotch, PastixOrderParMetis
} pastix_ordering_t;

typedef enum pastix_error_e {
    PASTIX_SUCCESS = 0, PASTIX_ERR_UNKNOWN = 1, PASTIX_ERR_ALLOC = 2, PASTIX_ERR_NOTIMPLEMENTED = 3,
    PASTIX_ERR_OUTOFMEMORY = 4, PASTIX_ERR_THREAD = 5, PASTIX_ERR_INTERNAL = 6,
    PASTIX_ERR_BADPARAMETER = 7, PASTIX_ERR_FILE = 8, PASTIX_ERR_INTEGER_TYPE = 9,
    PASTIX_ERR_IO = 10, PASTIX_ERR_MPI = 11
} pastix_error_t;

typedef enum pastix_trans_e { PastixNoTrans = 111, PastixTrans = 112, PastixConjTrans = 113 } pastix_trans_t;
typedef enum pastix_uplo_e { PastixUpper = 121, PastixLower = 122, PastixUpperLower = 123 } pastix_uplo_t;
typedef enum pastix_diag_e { PastixNonUnit = 131, PastixUnit = 132 } pastix_diag_t;
typedef enum pastix_side_e { PastixLeft = 141, PastixRight = 142 } pastix_side_t;
typedef enum pastix_dir_e { PastixDirForward = 391, PastixDirBackward = 392 } pastix_dir_t;
typedef enum pastix_coefside_e { PastixLCoef = 0, PastixUCoef = 1, PastixLUCoef = 2 } pastix_coefside_t;

/* ---- ordering (include/pastix/order.h:40-52) ---- */
typedef struct pastix_order_s {
    pastix_int_t  baseval;
    pastix_int_t  vertnbr;
    pastix_int_t  cblknbr;
    pastix_int_t *permtab;
    pastix_int_t *peritab;
    pastix_int_t *rangtab;
    pastix_int_t *treetab;
    int8_t       *selevtx;
    pastix_int_t  sndenbr;
    pastix_int_t *sndetab;
    pastix_int_t *peritab_exp;
} pastix_order_t;

typedef struct pastix_data_s pastix_data_t;
typedef struct pastix_rhs_s *pastix_rhs_t;

/* IPARM_IO_STRATEGY values (include/pastix/api.h:228-236).  PastixIOLoad: a
 * personal ordering is read from the ordering file and the block symbol from
 * "symbname"; PastixIOSave: both are written ("ordergen", "symbgen") after
 * ordering and symbolic factorization.  The graph and CSC variants are not
 * implemented (ignored). */
typedef enum pastix_io_e {
    PastixIONo = 0, PastixIOLoad = 1, PastixIOSave = 2, PastixIOLoadGraph = 4, PastixIOSaveGraph = 8,
    PastixIOLoadCSC = 16, PastixIOSaveCSC = 32
} pastix_io_t;

/* ---- main API (include/pastix.h:56-125) ---- */
/* replaces include/pastix.h:89 (pastixInitParam, common/api.c:420) */
void pastixInitParam(pastix_int_t *iparm, double *dparm);
/* replaces include/pastix.h:92 (pastixInit, common/api.c:905) */
void pastixInit(pastix_data_t **pastix_data, PASTIX_Comm pastix_comm, pastix_int_t *iparm, double *dparm);
/* replaces include/pastix.h:97 (pastixInitWithAffinity); bindtab is ignored */
void pastixInitWithAffinity(pastix_data_t **pastix_data, PASTIX_Comm pastix_comm, pastix_int_t *iparm,
                            double *dparm, const int *bindtab);
/* replaces include/pastix.h:103 (pastixFinalize, common/api.c:928) */
void pastixFinalize(pastix_data_t **pastix_data);

/* replaces include/pastix.h:109 (pastix_task_analyze, blend/pastix_task_analyze.c:53) */
int pastix_task_analyze(pastix_data_t *pastix_data, const spmatrix_t *spm);
/* replaces include/pastix.h:111 (pastix_task_numfact, sopalin/pastix_task_sopalin.c:654) */
int pastix_task_numfact(pastix_data_t *pastix_data, spmatrix_t *spm);
/* replaces include/pastix.h:113 (pastix_task_solve, sopalin/pastix_task_solve.c:758);
 * B (m x nrhs, leading dimension ldb, host memory) is overwritten by X */
int pastix_task_solve(pastix_data_t *pastix_data, pastix_int_t m, pastix_int_t nrhs, void *B,
                      pastix_int_t ldb);
/* replaces include/pastix.h:118 (pastix_task_refine, refinement/pastix_task_refine.c:236) */
int pastix_task_refine(pastix_data_t *pastix_data, pastix_int_t n, pastix_int_t nrhs, void *B,
                       pastix_int_t ldb, void *X, pastix_int_t ldx);
/* replaces include/pastix.h:125 (pastix_task_solve_and_refine, refinement/pastix_task_refine.c:359) */
int pastix_task_solve_and_refine(pastix_data_t *pastix_data, pastix_int_t n, pastix_int_t nrhs,
                                 void *B, pastix_int_t ldb, void *X, pastix_int_t ldx);
/* replaces include/pastix.h:63 (legacy one-call pastix(), sopalin/pastix.c:103) */
int pastix(pastix_data_t **pastix_data, PASTIX_Comm pastix_comm, pastix_int_t n, pastix_int_t *colptr,
           pastix_int_t *rowptr, void *values, pastix_int_t *perm, pastix_int_t *invp, void *B,
           pastix_int_t nrhs, pastix_int_t *iparm, double *dparm);

/* ---- analysis subtasks (include/pastix.h:136-141) ---- */
/* replaces order/pastix_subtask_order.c:100; myorder: PastixOrderPersonal input (may be NULL) */
int pastix_subtask_order(pastix_data_t *pastix_data, const spmatrix_t *spm, pastix_order_t *myorder);
/* replaces symbol/pastix_subtask_symbfact.c:86 */
int pastix_subtask_symbfact(pastix_data_t *pastix_data);
/* replaces symbol/pastix_subtask_reordering.c:60 (kept as a no-op step, see DESIGN) */
int pastix_subtask_reordering(pastix_data_t *pastix_data);
/* replaces blend/pastix_subtask_blend.c:121 */
int pastix_subtask_blend(pastix_data_t *pastix_data);

/* ---- numerical subtasks (include/pastix.h:146-177) ---- */
/* replaces sopalin/pastix_task_sopalin.c:93 */
int pastix_subtask_spm2bcsc(pastix_data_t *pastix_data, spmatrix_t *spm);
/* replaces sopalin/pastix_task_sopalin.c:213 */
int pastix_subtask_bcsc2ctab(pastix_data_t *pastix_data);
/* replaces sopalin/pastix_task_sopalin.c:412 */
int pastix_subtask_sopalin(pastix_data_t *pastix_data);
/* replaces sopalin/pastix_task_solve.c:169; Bp receives a device-resident permuted copy */
int pastix_subtask_applyorder(pastix_data_t *pastix_data, pastix_dir_t dir, pastix_int_t m,
                              pastix_int_t n, void *B, pastix_int_t ldb, pastix_rhs_t Bp);
/* replaces sopalin/pastix_task_solve.c:296 */
int pastix_subtask_trsm(pastix_data_t *pastix_data, pastix_side_t side, pastix_uplo_t uplo,
                        pastix_trans_t trans, pastix_diag_t diag, pastix_rhs_t b);
/* replaces sopalin/pastix_task_solve.c:422 */
int pastix_subtask_diag(pastix_data_t *pastix_data, pastix_rhs_t b);
/* replaces sopalin/pastix_task_solve.c:713 */
int pastix_subtask_solve(pastix_data_t *pastix_data, pastix_rhs_t b);
/* replaces sopalin/pastix_task_solve.c:512 */
int pastix_subtask_solve_adv(pastix_data_t *pastix_data, pastix_trans_t transA, pastix_rhs_t b);
/* replaces refinement/pastix_task_refine.c:106 */
int pastix_subtask_refine(pastix_data_t *pastix_data, pastix_rhs_t b, pastix_rhs_t x);

/* ---- right-hand sides (include/pastix.h:196-201, sopalin/pastix_rhs.c:44-242) ---- */
int pastixRhsInit(pastix_rhs_t *rhs);
int pastixRhsFinalize(pastix_rhs_t rhs);
int pastixRhsDoubletoSingle(const pastix_rhs_t dB, pastix_rhs_t sB);
int pastixRhsSingleToDouble(const pastix_rhs_t sB, pastix_rhs_t dB);

/* ---- ordering helpers (include/pastix/order.h) ---- */
/* replaces order/order_grids.c:307 (pastixOrderGrid); *myorder must point to a struct */
int pastixOrderGrid(pastix_order_t **myorder, pastix_int_t nx, pastix_int_t ny, pastix_int_t nz);
/* replaces order/order_io.c:132 (pastixOrderLoad): reads the reference's ordering
 * text format from $PASTIX_FILE_ORDER or "ordername" into *ordemesh (0-based;
 * rangtab / treetab NULL for a version-0 file without the elimination tree) */
int pastixOrderLoad(const pastix_data_t *pastix_data, pastix_order_t *ordemesh);
/* replaces order/order_io.c:296 (pastixOrderSave): writes *ordemesh in the same
 * format to "ordergen" (or $PASTIX_FILE_ORDER) in the instance's output
 * directory "<$PASTIX_OUTPUT_DIR or pastix>-XXXXXX" */
int pastixOrderSave(pastix_data_t *pastix_data, const pastix_order_t *ordemesh);
/* replaces order/order.c (pastixOrderExit): frees the arrays of an order filled by this library */
void pastixOrderExit(pastix_order_t *ordeptr);

/* ---- B200 extensions: device-resident entry points, all on the library's stream ---- */

/* Structure of the solver, host arrays owned by pastix_data (valid until the next analysis). */
typedef struct pgpu_solver_info_s {
    pastix_int_t n, cblknbr, bloknbr, coefnbr, nlevels, ntasks;
    const pastix_int_t *cb_fcol, *cb_lcol, *cb_fblok, *cb_stride, *cb_coef, *cb_level;
    const pastix_int_t *bk_frow, *bk_lrow, *bk_fcblk, *bk_lcblk, *bk_rowoff;
    const pastix_int_t *permtab, *peritab;
    double thflops;
} pgpu_solver_info_t;
/* Fills *info after pastix_task_analyze; returns PASTIX_ERR_BADPARAMETER before it. */
int pgpu_solver_info(const pastix_data_t *pastix_data, pgpu_solver_info_t *info);

/* Imports an analysis made elsewhere -- the SolverMatrix of the reference's own
 * pastix_task_analyze -- for the pattern of `spm`: the permutation (permtab[v]
 * = new index of vertex v) and the block symbolic structure as plain arrays
 * (cblk k: columns cb_fcol[k]..cb_lcol[k], bloks cb_fblok[k]..cb_fblok[k+1]-1
 * (bloknbr ends the last cblk), diagonal blok first; blok b: rows
 * bk_frow[b]..bk_lrow[b] facing cblk bk_fcblk[b]).  Stands for
 * pastix_subtask_order + symbfact + reordering + blend (blend/solver.h:141-279
 * gives the fields).  IPARM_FACTORIZATION must be set before the call. */
int pgpu_set_symbol(pastix_data_t *pastix_data, const spmatrix_t *spm, const pastix_int_t *permtab,
                    pastix_int_t cblknbr, const pastix_int_t *cb_fcol, const pastix_int_t *cb_lcol,
                    const pastix_int_t *cb_fblok, pastix_int_t bloknbr, const pastix_int_t *bk_frow,
                    const pastix_int_t *bk_lrow, const pastix_int_t *bk_fcblk);

/* Copies the factor panels to host memory in the library's layout (per cblk a
 * column-major stride x width panel at cb_coef[k]).  L and U are coefnbr
 * elements each, of the factorization's arithmetic (double, or float under
 * IPARM_MIXED); U may be NULL (only GETRF has a U panel). */
int pgpu_get_coeftab(const pastix_data_t *pastix_data, void *L, void *U);

/* Solve on device memory: B is an n x nrhs column-major FP64 array in the
 * ORIGINAL numbering, on the current CUDA device, overwritten by X.  `stream`
 * is the caller's cudaStream_t (NULL = the legacy default stream): the solve
 * starts after the work already queued on it, and work queued on it after the
 * call sees X.  The call returns without waiting for the result. */
int pgpu_solve_device(pastix_data_t *pastix_data, pastix_int_t nrhs, double *B, pastix_int_t ldb,
                      void *stream);
/* Transposed solve A^T X = B on device memory (adjoint), same conventions. */
int pgpu_solve_transposed_device(pastix_data_t *pastix_data, pastix_int_t nrhs, double *B,
                                 pastix_int_t ldb, void *stream);
/* Numerical factorization from device-resident values (nnz FP64 entries in the
 * order of the spm given to pastix_task_analyze). */
int pgpu_numfact_device(pastix_data_t *pastix_data, const double *values_dev);
/* Sampled outer product for the adjoint: G[e] = alpha * lambda[row(e)] * x[col(e)]
 * for every stored entry e of the analysed spm (original numbering, device
 * memory); with SpmSymmetric storage an off-diagonal entry e = (i, j) stands for
 * a_ij and a_ji and receives alpha * (lambda[i] x[j] + lambda[j] x[i]).  With
 * lambda = A^{-T} g and alpha = -1 this is the gradient of <g, A^{-1} b> with
 * respect to the stored values.  No counterpart in the reference. */
int pgpu_sampled_outer(pastix_data_t *pastix_data, double alpha, const double *lambda,
                       const double *x, double *G, void *stream);
/* Residual SpMV on device memory: y = alpha*A*x + beta*y (original numbering),
 * on the caller's stream (NULL = legacy default stream). */
int pgpu_spmv_device(pastix_data_t *pastix_data, double alpha, const double *x, double beta,
                     double *y, void *stream);
/* Last device status word (0 = fine); non-zero after a bounded wait expired. */
int pgpu_device_status(const pastix_data_t *pastix_data);
/* Self-test of the kernels' bounded waits on the current device: one wait on
 * a cluster flag that nothing raises and one on an mbarrier that nothing
 * completes; both must give up.  timed_out[0..1] receive how many did (1, 1
 * expected).  Takes a few seconds.  No counterpart in the reference. */
int pgpu_wait_selftest(int *timed_out);

/* The library's CUDA stream (cudaStream_t) after the analysis; every entry
 * point above orders its work on it.  NULL before pastix_task_analyze. */
void *pgpu_stream(pastix_data_t *pastix_data);

/* Solve then refine on device memory (pastix_task_solve_and_refine on the GPU):
 * B, X are n x nrhs FP64 arrays in the original numbering, X receives the
 * refined solution; IPARM_REFINEMENT selects GMRES / CG / SR / BiCGStab. */
int pgpu_solve_refine_device(pastix_data_t *pastix_data, pastix_int_t nrhs, const double *B, pastix_int_t ldb,
                             double *X, pastix_int_t ldx);

/* pgpu_solve_device without any allocation, for callers that cannot allocate
 * device memory when they solve.  No counterpart in the reference.  Its work
 * vectors live in one fixed array in the library's module memory: n * nrhs may
 * not exceed PGPU_STATIC_SOLVE_ELEMS (12 bytes per element, 12 MiB in all);
 * larger calls return PASTIX_ERR_BADPARAMETER and touch nothing.  The first
 * call on a device sets up that device (looks the array up, creates one
 * event): make it before any stream capture.  The array is shared by every
 * pastix_data_t of the process on that device, so calls that overlap in time
 * (two host threads, or two streams without ordering between them) race on
 * it.  Not available while pgpu_profile timing is on.  The set-up is cached
 * per device for the life of the process; after a device reset a call fails
 * once with PASTIX_ERR_INTERNAL and the next one redoes the set-up.  Same
 * arguments and stream semantics as pgpu_solve_device (A X = B). */
#define PGPU_STATIC_SOLVE_ELEMS 1048576
int pgpu_solve_device_static(pastix_data_t *pastix_data, pastix_int_t nrhs, double *B, pastix_int_t ldb,
                             void *stream);

/* Launch accounting.  pgpu_profile(pd, 1) resets the counters and times every
 * launch with CUDA events on the library stream; pgpu_profile(pd, 0) resets
 * and only counts.  pgpu_profile_get returns, per kernel class (fill, panel,
 * diag, trsm, update, fwd diag, fwd update, bwd update, bwd diag, spmv, vec,
 * big update tiles, BF16 split of FP32 panels),
 * the summed device milliseconds and the launch counts. */
int pgpu_profile(pastix_data_t *pastix_data, int enable);

/* CUDA graphs of the fixed launch sequences (no counterpart in the reference,
 * whose numerical phase is scheduled by threads, sopalin/pastix_task_sopalin.c:51-58).
 * With graphs on (the default) the FP64 factorization's per-level launches
 * (pastix_subtask_sopalin) and the two sweeps of each solve (both precisions)
 * are captured into one CUDA graph on first use and replayed by a single
 * cudaGraphLaunch afterwards (FP32 factorizations launch kernel by kernel:
 * measured faster than their graph); a graph is keyed by the precision, the factorization kind and
 * every device buffer its launches name, and is dropped when the analysis
 * changes.  The static-pivot threshold is read from device memory, so a
 * replay with new matrix values is exact.  pgpu_graphs(pd, 0) drops the
 * graphs and launches kernel by kernel; per-launch profiling (pgpu_profile
 * with enable = 1) also launches kernel by kernel. */
int pgpu_graphs(pastix_data_t *pastix_data, int enable);

/* GMRES and CG refinement of several right-hand sides as one block (default
 * on): the per-column GMRES of refinement/z_refine_gmres.c, or the per-column
 * CG of refinement/z_refine_grad.c (same steps, iterates and stopping test per
 * column), advanced for all columns together, so that each
 * preconditioner application is one multi-column solve instead of one solve
 * per column (the reference refines the columns one after the other,
 * refinement/pastix_task_refine.c:121-164).  enable = 0 restores the column
 * loop.  Blocks hold as many columns as a quarter of the free device memory
 * allows (GMRES: 2 im + 2 vectors each, CG: 5), at most 256; BiCGStab and
 * simple refinement keep the column loop. */
int pgpu_refine_block(pastix_data_t *pastix_data, int enable);

/* Bucket boundaries of the supernode update tiles (no counterpart in the
 * reference, whose update GEMM is one BLAS call per blok,
 * kernels/core_zgemmsp.c:404-474).  FP64 factors: an update task whose facing
 * blok has at least dmma_n rows and whose source cblk is at least dmma_k wide
 * runs as 128 x 64 DMMA tiles, any other as 64 x 64 FMA tiles (defaults 32,
 * 32).  FP32 factors: a task whose source is at least tc_k (>= 32) wide runs on
 * tcgen05 with split BF16 operands, narrower ones as FMA tiles (default 32).
 * Setting them rebuilds the launch lists: the next pastix_task_numfact /
 * pgpu_numfact_device refactorizes.  pgpu_get_tuning returns the three values. */
int pgpu_set_tuning(pastix_data_t *pastix_data, pastix_int_t dmma_n, pastix_int_t dmma_k, pastix_int_t tc_k);
int pgpu_get_tuning(const pastix_data_t *pastix_data, pastix_int_t *vals);

/* Autotuner of those bucket boundaries for the analysed matrix: each candidate
 * (FP64: dmma_n in {8, 16, 32, 64} x dmma_k in {16, 32}; FP32: tc_k in
 * {32, 48, 64, 96}) is applied and timed on a factorization of the given
 * device values (spm value order, as pgpu_numfact_device); the buckets in
 * effect are kept unless a candidate is at least 2 % faster, and the matrix is
 * left factorized with the buckets chosen.  chosen (if not NULL)
 * receives {dmma_n, dmma_k, tc_k}. */
int pgpu_autotune(pastix_data_t *pastix_data, const double *values_dev, pastix_int_t *chosen);
int pgpu_profile_get(pastix_data_t *pastix_data, double *ms, long long *launches, int nclass);

#ifdef __cplusplus
}
#endif
#endif /* PASTIX_B200_H */
