// Host-side analysis structures of the B200 numerical phase.
//
// The numerical phase consumes the same objects that PaStiX's analysis step
// (pastix_task_analyze, blend/pastix_task_analyze.c:53) hands to the numerical
// factorization: an ordering (include/pastix/order.h:40-52), a block symbolic
// matrix (symbol/symbol.h) and the solver structure built from it
// (blend/solver.h:141-279).  These C++ types hold the fields the numerical
// phase reads, in plain arrays, with 64-bit indices as in PaStiX's default
// PASTIX_INT64 build.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace pgpu {

using idx_t = int64_t;

// Ordering: permtab[v] = new index of vertex v, peritab = inverse,
// rangtab[k]..rangtab[k+1]-1 = columns of supernode k, treetab[k] = father
// (-1 for the root).  Same meaning as pastix_order_t.
struct Order {
    idx_t n = 0;
    idx_t cblknbr = 0;
    std::vector<idx_t> permtab, peritab, rangtab, treetab;
};

// One column block of the symbolic matrix (symbol_cblk_t).
struct SymCblk {
    idx_t fcolnum, lcolnum;  // inclusive column range
    idx_t bloknum;           // first blok (the diagonal one)
};

// One block (symbol_blok_t): rows [frownum, lrownum] facing cblk fcblknm.
struct SymBlok {
    idx_t frownum, lrownum;
    idx_t lcblknm, fcblknm;
};

struct Symbol {
    idx_t nodenbr = 0;
    std::vector<SymCblk> cblktab;  // size cblknbr + 1 (sentinel bloknum)
    std::vector<SymBlok> bloktab;
    idx_t cblknbr() const { return (idx_t)cblktab.size() - 1; }
    idx_t bloknbr() const { return (idx_t)bloktab.size(); }
};

// Undirected adjacency graph (CSC without the diagonal, both triangles).
struct Graph {
    idx_t n = 0;
    std::vector<idx_t> colptr, rowind;
};

// Update task: source cblk k sends C_f -= A(rows >= row0) * B(rows [row0, row0+N))^T
// into the facing cblk f.  One task per off-diagonal blok (the granularity of
// core_zgemmsp_2d2d, kernels/core_zgemmsp.c:404-474).
struct Task {
    idx_t src;      // source cblk
    idx_t dst;      // facing cblk
    idx_t blok;     // the off-diagonal blok b of src facing dst
    idx_t row0;     // row offset of b inside the src panel
    idx_t n;        // rows of b
    idx_t m;        // rows of src from b (inclusive) to the end of the panel
};

// Solver structure: symbol + numeric layout + schedule, all host side.
struct Solver {
    idx_t n = 0;            // matrix size (expanded by dof)
    idx_t cblknbr = 0, bloknbr = 0;
    int factotype = 0;      // 0 POTRF, 1 SYTRF, 2 GETRF (pastix_factotype_t)

    // cblk arrays (size cblknbr + 1 where a sentinel is needed)
    std::vector<idx_t> cb_fcol, cb_lcol, cb_fblok, cb_stride, cb_coef, cb_level;
    std::vector<idx_t> cb_brow;         // browtab start, size cblknbr+1
    // blok arrays
    std::vector<idx_t> bk_frow, bk_lrow, bk_fcblk, bk_lcblk, bk_rowoff;
    std::vector<idx_t> browtab;         // bloks facing each cblk (grouped per cblk)
    std::vector<idx_t> rowidx;          // global row index of every panel row (size Σ stride)
    std::vector<idx_t> cb_rowidx;       // start of each cblk in rowidx (size cblknbr+1)
    idx_t coefnbr = 0;                  // Σ stride*width

    // levels: cblks of level l are lvl_cblk[lvl_ptr[l] .. lvl_ptr[l+1])
    idx_t nlevels = 0;
    std::vector<idx_t> lvl_ptr, lvl_cblk;
    // update tasks grouped by level of their source cblk
    std::vector<Task> tasks;
    std::vector<idx_t> lvl_task_ptr;

    double thflops = 0.0;     // pastixSymbolGetFlops (theoretical)
    idx_t nnzl = 0;           // Σ stride*width, lower factor entries incl. diag blocks
};

// ---- analysis steps ----
void order_grid(Order &o, idx_t nx, idx_t ny, idx_t nz);
void order_expand_dof(Order &o, idx_t dof);
void graph_collapse(const Graph &g, idx_t dof, Graph &out);
void order_find_supernodes(Order &o, const Graph &g);
void order_apply_level_order(Order &o, idx_t level2d, idx_t width2d);
void symbol_reorder_rows(const Symbol &s, Order &o, idx_t split_level, idx_t stop);
void order_nd_graph(Order &o, const Graph &g, idx_t leaf = 64);
std::string order_check(const Order &o);
void symbol_fax(Symbol &s, const Graph &g, const Order &o);
void symbol_split(Symbol &s, idx_t blcolmin, idx_t blcolmax);
void symbol_expand(const Symbol &node, idx_t dof, Symbol &out);
std::string symbol_check(const Symbol &s);
double symbol_flops(const Symbol &s, int factotype);
void solver_build(Solver &sv, const Symbol &s, int factotype);

}  // namespace pgpu
