// Host-side analysis for the B200 numerical phase: grid nested dissection,
// supernode detection, block symbolic factorization, supernode splitting and
// the solver layout / level schedule consumed by the CUDA kernels.
//
// Each routine restates the algorithm of the PaStiX analysis step it replaces
// (file:line given per function); the data structures and code are this
// project's own.
#include "symbol.hpp"

#include <algorithm>
#include <cstdio>
#include <numeric>
#include <sstream>
#include <stdexcept>

namespace pgpu {

static inline idx_t iceil(idx_t a, idx_t b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// Grid nested dissection (order/order_grids.c:139-276, pastixOrderGrid :307).
// A box is cut by a plane orthogonal to its longest direction (ties prefer x,
// then y); the plane gets the highest numbers still free, then the lower
// half, then the upper half are ordered recursively.  Boxes with fewer than
// 15 vertices are leaves, numbered x-slowest inside the box.  Vertex index is
// x + nx*y + nx*ny*z.
// ---------------------------------------------------------------------------
namespace {
struct GridND {
    idx_t nx, ny, nz;
    idx_t next;                      // highest number not yet given
    std::vector<idx_t> *perm;
    std::vector<idx_t> top, depth;   // per supernode, in creation order

    idx_t vid(idx_t x, idx_t y, idx_t z) const { return x + nx * (y + ny * z); }

    void plane(int dir, idx_t c, idx_t x0, idx_t xn, idx_t y0, idx_t yn, idx_t z0, idx_t zn) {
        // the separator plane is numbered with its two remaining directions in
        // (outer, inner) order = (y,z) for an x cut, (x,z) for y, (x,y) for z
        if (dir == 0) {
            for (idx_t y = y0; y < yn; y++)
                for (idx_t z = z0; z < zn; z++) (*perm)[vid(c, y, z)] = next--;
        } else if (dir == 1) {
            for (idx_t x = x0; x < xn; x++)
                for (idx_t z = z0; z < zn; z++) (*perm)[vid(x, c, z)] = next--;
        } else {
            for (idx_t x = x0; x < xn; x++)
                for (idx_t y = y0; y < yn; y++) (*perm)[vid(x, y, c)] = next--;
        }
    }

    void rec(idx_t x0, idx_t xn, idx_t y0, idx_t yn, idx_t z0, idx_t zn, idx_t d) {
        idx_t lx = xn - x0, ly = yn - y0, lz = zn - z0;
        top.push_back(next);
        depth.push_back(d);
        if (lx * ly * lz < 15) {
            idx_t k = 0;
            for (idx_t x = x0; x < xn; x++)
                for (idx_t y = y0; y < yn; y++)
                    for (idx_t z = z0; z < zn; z++) (*perm)[vid(x, y, z)] = next - (k++);
            next -= k;
            return;
        }
        int dir = 0;
        if (ly > lx) dir = 1;
        if (lz > lx && lz > ly) dir = 2;
        if (dir == 0) {
            idx_t c = x0 + lx / 2;
            plane(0, c, x0, xn, y0, yn, z0, zn);
            rec(x0, c, y0, yn, z0, zn, d + 1);
            rec(c + 1, xn, y0, yn, z0, zn, d + 1);
        } else if (dir == 1) {
            idx_t c = y0 + ly / 2;
            plane(1, c, x0, xn, y0, yn, z0, zn);
            rec(x0, xn, y0, c, z0, zn, d + 1);
            rec(x0, xn, c + 1, yn, z0, zn, d + 1);
        } else {
            idx_t c = z0 + lz / 2;
            plane(2, c, x0, xn, y0, yn, z0, zn);
            rec(x0, xn, y0, yn, z0, c, d + 1);
            rec(x0, xn, y0, yn, c + 1, zn, d + 1);
        }
    }
};
}  // namespace

void order_grid(Order &o, idx_t nx, idx_t ny, idx_t nz) {
    if (nx < 1 || ny < 1 || nz < 1) throw std::invalid_argument("order_grid: bad grid size");
    idx_t n = nx * ny * nz;
    o.n = n;
    o.permtab.assign(n, -1);
    GridND g{nx, ny, nz, n - 1, &o.permtab, {}, {}};
    g.rec(0, nx, 0, ny, 0, nz, 1);
    o.peritab.assign(n, 0);
    for (idx_t i = 0; i < n; i++) o.peritab[o.permtab[i]] = i;
    // supernodes were created top-down with decreasing numbers: reverse them
    idx_t cb = (idx_t)g.top.size();
    o.cblknbr = cb;
    o.rangtab.assign(cb + 1, 0);
    std::vector<idx_t> dep(cb);
    for (idx_t i = 0; i < cb; i++) {
        o.rangtab[i + 1] = g.top[cb - 1 - i] + 1;
        dep[i] = g.depth[cb - 1 - i];
    }
    // father = first later supernode that is shallower (order_grids.c:371-380)
    o.treetab.assign(cb, -1);
    for (idx_t i = 0; i + 1 < cb; i++) {
        for (idx_t j = i + 1; j < cb; j++)
            if (dep[j] < dep[i]) { o.treetab[i] = j; break; }
    }
}

// Node graph of a matrix with dof unknowns per node (unknown v*dof+d belongs
// to node v): two nodes are adjacent when any of their unknowns are.
void graph_collapse(const Graph &g, idx_t dof, Graph &out) {
    const idx_t nn = g.n / dof;
    out.n = nn;
    out.colptr.assign(nn + 1, 0);
    out.rowind.clear();
    std::vector<idx_t> mark(nn, -1), adj;
    for (idx_t v = 0; v < nn; v++) {
        adj.clear();
        for (idx_t d = 0; d < dof; d++) {
            idx_t i = v * dof + d;
            for (idx_t e = g.colptr[i]; e < g.colptr[i + 1]; e++) {
                idx_t w = g.rowind[e] / dof;
                if (w != v && mark[w] != v) { mark[w] = v; adj.push_back(w); }
            }
        }
        std::sort(adj.begin(), adj.end());
        out.rowind.insert(out.rowind.end(), adj.begin(), adj.end());
        out.colptr[v + 1] = (idx_t)out.rowind.size();
    }
}

// Expand a node ordering to dof unknowns per node (pastixOrderExpand,
// order/order.c): unknown v*dof+d of node v keeps node order, dof-major.
void order_expand_dof(Order &o, idx_t dof) {
    if (dof <= 1) return;
    idx_t n = o.n;
    std::vector<idx_t> perm(n * dof), peri(n * dof);
    for (idx_t v = 0; v < n; v++)
        for (idx_t d = 0; d < dof; d++) perm[v * dof + d] = o.permtab[v] * dof + d;
    for (idx_t i = 0; i < n * dof; i++) peri[perm[i]] = i;
    o.permtab.swap(perm);
    o.peritab.swap(peri);
    for (auto &r : o.rangtab) r *= dof;
    o.n = n * dof;
}

// ---------------------------------------------------------------------------
// Supernodes renumbered level by level of the elimination tree
// (orderApplyLevelOrder, order/order_apply_level_order.c:95-338).  The tree is
// walked breadth first from the roots; the sons of a supernode are queued in
// reverse index order, and the final numbering is the reverse of the queue,
// so that the roots come last and every son precedes its father.  With
// level2d < 0 (automatic 2D tasks), supernodes of at least width2d columns
// whose father is a root or a 2D supernode with exactly two sons are "2D"
// and are queued ahead of all the others, level by level as well.  Columns
// keep their order inside each supernode.
// ---------------------------------------------------------------------------
void order_apply_level_order(Order &o, idx_t level2d, idx_t width2d) {
    const idx_t cb = o.cblknbr;
    if (cb <= 1) return;
    // sons of every node in increasing index order; roots are the sons of -1
    std::vector<idx_t> nsons(cb + 1, 0), first(cb + 2, 0), sons(cb);
    for (idx_t k = 0; k < cb; k++) nsons[o.treetab[k] + 1]++;
    for (idx_t f = 0; f <= cb; f++) first[f + 1] = first[f] + nsons[f];
    {
        std::vector<idx_t> pos(first.begin(), first.end() - 1);
        for (idx_t k = 0; k < cb; k++) sons[pos[o.treetab[k] + 1]++] = k;
    }
    auto sons_of = [&](idx_t f) { return std::make_pair(first[f + 1], first[f + 2]); };  // f = -1 for roots
    std::vector<idx_t> queue(cb), father(o.treetab);  // father becomes the new number of the father
    if (level2d < 0) {
        std::vector<char> is2d(cb, 0);
        idx_t n2d = 0;
        for (idx_t k = cb - 1; k >= 0; k--) {
            idx_t f = o.treetab[k], size = o.rangtab[k + 1] - o.rangtab[k];
            if (size >= width2d && (f == -1 || (is2d[f] && nsons[f + 1] == 2))) { is2d[k] = 1; n2d++; }
        }
        idx_t p2 = 0, p1 = n2d;
        auto roots = sons_of(-1);
        for (idx_t r = roots.first; r < roots.second; r++) {
            idx_t k = sons[r];
            if (is2d[k]) queue[p2++] = k; else queue[p1++] = k;
        }
        for (idx_t i = 0; i < cb; i++) {
            idx_t node = queue[i];
            auto sr = sons_of(node);
            idx_t s2 = 0;
            for (idx_t r = sr.first; r < sr.second; r++) s2 += is2d[sons[r]];
            idx_t s1 = (sr.second - sr.first) - s2, c2 = 0, c1 = 0;
            for (idx_t r = sr.first; r < sr.second; r++) {
                idx_t son = sons[r];
                if (is2d[son]) queue[p2 + s2 - 1 - c2++] = son;
                else queue[p1 + s1 - 1 - c1++] = son;
                father[son] = cb - 1 - i;
            }
            p2 += s2;
            p1 += s1;
        }
    } else {
        auto roots = sons_of(-1);
        idx_t pos = roots.second - roots.first;
        std::copy(sons.begin() + roots.first, sons.begin() + roots.second, queue.begin());
        for (idx_t i = 0; i < cb; i++) {
            idx_t node = queue[i];
            auto sr = sons_of(node);
            idx_t ns = sr.second - sr.first;
            for (idx_t j = 0; j < ns; j++) {
                idx_t son = sons[sr.first + j];
                queue[pos + ns - 1 - j] = son;
                father[son] = cb - 1 - i;
            }
            pos += ns;
        }
    }
    std::vector<idx_t> rang(cb + 1, 0), tree(cb), peri(o.n);
    for (idx_t i = 0; i < cb; i++) {
        idx_t node = queue[cb - 1 - i];
        idx_t size = o.rangtab[node + 1] - o.rangtab[node];
        rang[i + 1] = rang[i] + size;
        tree[i] = father[node];
        std::copy(o.peritab.begin() + o.rangtab[node], o.peritab.begin() + o.rangtab[node + 1], peri.begin() + rang[i]);
    }
    o.rangtab.swap(rang);
    o.treetab.swap(tree);
    o.peritab.swap(peri);
    for (idx_t i = 0; i < o.n; i++) o.permtab[o.peritab[i]] = i;
}

// ---------------------------------------------------------------------------
// Reordering of the unknowns inside each supernode (pastixSymbolReordering,
// symbol/symbol_reordering.c:619-660, per supernode :455-610, tour :107-370).
// Row i of supernode k is described by the sorted list of the supernodes whose
// off-diagonal bloks cover it; rows with close lists should be adjacent so that
// the bloks they form are few.  The rows are inserted one by one into a cyclic
// tour that starts with a ghost row (empty list), at the position that adds the
// least Hamming distance between neighbours (ties broken by the smaller cut),
// and the tour is read from the row after the ghost.  split_level separates
// the lists into contributors of the upper levels of the tree (their distance
// only gates the candidate positions) and of the lower levels; stop caps every
// distance.  Each supernode is independent of the others.
// ---------------------------------------------------------------------------
namespace {
struct RowSets {
    std::vector<idx_t> ptr, val;  // row r: val[ptr[r] .. ptr[r+1])
    idx_t size(idx_t r) const { return r < 0 ? 0 : ptr[r + 1] - ptr[r]; }
};

// |A xor B| of two sorted lists, capped at stop; the ghost row (-1) is empty
idx_t hamming(const RowSets &v, idx_t a, idx_t b, idx_t stop) {
    if (a == -1) return v.size(b);
    if (b == -1) return v.size(a);
    idx_t na = v.size(a), nb = v.size(b);
    if (na - nb >= stop || nb - na >= stop) return stop;
    const idx_t *x = v.val.data() + v.ptr[a], *xe = x + na;
    const idx_t *y = v.val.data() + v.ptr[b], *ye = y + nb;
    idx_t sum = 0;
    while (x < xe && y < ye) {
        if (*x == *y) { x++; y++; }
        else if (*x < *y) { while (x < xe && *x < *y) { sum++; x++; } }
        else { while (y < ye && *x > *y) { sum++; y++; } }
        if (sum >= stop) return stop;
    }
    sum += (xe - x) + (ye - y);
    return sum >= stop ? stop : sum;
}

// Tour of `size` rows; returns the new order of the local row indices.
std::vector<idx_t> row_tour(idx_t size, const RowSets &lw, const RowSets &up, idx_t stop) {
    std::vector<idx_t> tour(size + 1), len(size + 1, 0);
    tour[0] = -1;
    tour[1] = 0;
    len[0] = len[1] = hamming(lw, 0, -1, stop);
    for (idx_t i = 1; i < size; i++) {
        idx_t before = hamming(lw, i, tour[0], stop);
        idx_t after = hamming(lw, i, tour[1], stop);
        idx_t up_after = hamming(up, i, tour[1], 1);
        idx_t best = before + after - len[0], bpos = 1, cut = -1;
        for (idx_t j = 1; j < i; j++) {
            idx_t up_before = up_after;
            up_after = hamming(up, i, tour[j + 1], 1);
            if (up_before < 1 || up_after < 1) {
                before = (after == -1) ? hamming(lw, i, tour[j], stop) : after;
                after = hamming(lw, i, tour[j + 1], stop);
                idx_t l = before + after - len[j];
                if (l == best) {
                    if (before < cut) { cut = before; best = l; bpos = j + 1; }
                    if (after < cut) { cut = after; best = l; bpos = j + 1; }
                }
                if (l < best) {
                    cut = before;
                    best = l;
                    bpos = j + 1;
                    if (after < cut) cut = after;
                }
                if (after == 0) {  // an identical row: go right after it
                    best = l;
                    bpos = j + 1;
                    break;
                }
            } else {
                after = -1;
            }
        }
        idx_t to_first = hamming(lw, i, tour[0], stop);
        idx_t to_last = hamming(lw, i, tour[i], stop);
        before = hamming(lw, i, tour[bpos - 1], stop);
        after = hamming(lw, i, tour[bpos], stop);
        if (to_first + to_last - len[i] < best) bpos = i + 1;
        if (bpos > 0) len[bpos - 1] = before;
        if (bpos < i + 1) {  // shift the tail right and insert
            idx_t k = i, l = after;
            for (idx_t j = bpos; j < i + 2; j++) {
                std::swap(tour[j], k);
                std::swap(len[j], l);
            }
        } else {
            tour[i + 1] = i;
            len[i + 1] = to_first;
        }
    }
    idx_t ghost = 0;
    for (idx_t i = 0; i < size; i++)
        if (tour[i] == -1) ghost = i;
    std::vector<idx_t> out(size);
    for (idx_t i = 0; i < size; i++) out[i] = tour[(i + 1 + ghost) % (size + 1)];
    return out;
}
}  // namespace

void symbol_reorder_rows(const Symbol &s, Order &o, idx_t split_level, idx_t stop) {
    const idx_t cb = s.cblknbr();
    // depth of every supernode in the ordering's tree (root = 1)
    std::vector<idx_t> level(cb, 0);
    idx_t maxdepth = 0;
    for (idx_t k = cb - 1; k >= 0; k--) {  // fathers have larger numbers
        idx_t f = o.treetab[k];
        level[k] = (f < 0) ? 1 : level[f] + 1;
        maxdepth = std::max(maxdepth, level[k]);
    }
    // bloks facing each supernode, in increasing blok number (pastixSymbolBuildRowtab)
    std::vector<idx_t> bptr(cb + 1, 0), brow;
    for (idx_t b = 0; b < s.bloknbr(); b++)
        if (s.bloktab[b].fcblknm != s.bloktab[b].lcblknm) bptr[s.bloktab[b].fcblknm + 1]++;
    for (idx_t k = 0; k < cb; k++) bptr[k + 1] += bptr[k];
    brow.resize(bptr[cb]);
    {
        std::vector<idx_t> pos(bptr.begin(), bptr.end() - 1);
        for (idx_t b = 0; b < s.bloknbr(); b++)
            if (s.bloktab[b].fcblknm != s.bloktab[b].lcblknm) brow[pos[s.bloktab[b].fcblknm]++] = b;
    }
    std::vector<idx_t> weight(maxdepth);
    for (idx_t k = 0; k < cb; k++) {
        const SymCblk &c = s.cblktab[k];
        const idx_t size = c.lcolnum - c.fcolnum + 1;
        // move the split level until neither side dominates (symbol_reordering.c:487-530)
        std::fill(weight.begin(), weight.end(), 0);
        for (idx_t e = bptr[k]; e < bptr[k + 1]; e++) {
            const SymBlok &b = s.bloktab[brow[e]];
            weight[level[b.lcblknm] - 1] += b.lrownum - b.frownum + 1;
        }
        idx_t split = split_level;
        for (int sign = 0;;) {
            idx_t upw = 0, lww = 0, i = 0;
            for (; i < split && i < maxdepth; i++) upw += weight[i];
            for (; i < maxdepth; i++) lww += weight[i];
            if (lww < 5 * upw && lww > 10 && upw > 10 && sign <= 0) { split--; sign--; continue; }
            if (lww > 3 * upw && lww > 10 && upw > 10 && sign >= 0) { split++; sign++; continue; }
            break;
        }
        if (size < 3) continue;
        RowSets lw, up;
        lw.ptr.assign(size + 1, 0);
        up.ptr.assign(size + 1, 0);
        for (idx_t e = bptr[k]; e < bptr[k + 1]; e++) {
            const SymBlok &b = s.bloktab[brow[e]];
            RowSets &v = (level[b.lcblknm] <= split) ? up : lw;
            for (idx_t r = b.frownum; r <= b.lrownum; r++) v.ptr[r - c.fcolnum + 1]++;
        }
        for (idx_t r = 0; r < size; r++) { lw.ptr[r + 1] += lw.ptr[r]; up.ptr[r + 1] += up.ptr[r]; }
        lw.val.resize(lw.ptr[size]);
        up.val.resize(up.ptr[size]);
        {
            std::vector<idx_t> pl(lw.ptr.begin(), lw.ptr.end() - 1), pu(up.ptr.begin(), up.ptr.end() - 1);
            for (idx_t e = bptr[k]; e < bptr[k + 1]; e++) {
                const SymBlok &b = s.bloktab[brow[e]];
                bool isup = level[b.lcblknm] <= split;
                for (idx_t r = b.frownum; r <= b.lrownum; r++) {
                    idx_t lr = r - c.fcolnum;
                    if (isup) up.val[pu[lr]++] = b.lcblknm; else lw.val[pl[lr]++] = b.lcblknm;
                }
            }
        }
        std::vector<idx_t> t = row_tour(size, lw, up, stop);
        std::vector<idx_t> seg(size);
        for (idx_t i = 0; i < size; i++) seg[i] = o.peritab[c.fcolnum + t[i]];
        std::copy(seg.begin(), seg.end(), o.peritab.begin() + c.fcolnum);
    }
    for (idx_t i = 0; i < o.n; i++) o.permtab[o.peritab[i]] = i;
}

// ---------------------------------------------------------------------------
// Built-in ordering for matrices without a grid or user ordering: nested
// dissection of the adjacency graph with breadth-first level-set separators.
// It stands in for the Scotch / Metis orderings of
// order/pastix_subtask_order.c:272-316, which are external libraries.  A part
// is cut at the middle BFS level from a pseudo-peripheral vertex; the level
// is the separator and takes the highest numbers of the part's range.
// Disconnected parts are split into components first; parts of at most
// `leaf` vertices are numbered in BFS order.
// ---------------------------------------------------------------------------
void order_nd_graph(Order &o, const Graph &g, idx_t leaf) {
    const idx_t n = g.n;
    o.n = n;
    o.permtab.assign(n, -1);
    o.peritab.assign(n, -1);
    o.rangtab.clear();
    o.treetab.clear();
    o.cblknbr = 0;
    std::vector<idx_t> part(n, 0), level(n, -1), stamp(n, -1);
    idx_t nextpart = 1;
    struct Item { std::vector<idx_t> v; idx_t lo; idx_t id; };
    std::vector<Item> stack;
    {
        Item it;
        it.v.resize(n);
        std::iota(it.v.begin(), it.v.end(), 0);
        it.lo = 0;
        it.id = 0;
        stack.push_back(std::move(it));
    }
    idx_t bfs_id = 0;
    // BFS restricted to vertices of part id; fills order and levels, returns last vertex
    std::vector<idx_t> q;
    auto bfs = [&](idx_t src, idx_t id, idx_t &depth) {
        bfs_id++;
        q.clear();
        q.push_back(src);
        stamp[src] = bfs_id;
        level[src] = 0;
        for (size_t h = 0; h < q.size(); h++) {
            idx_t v = q[h];
            for (idx_t e = g.colptr[v]; e < g.colptr[v + 1]; e++) {
                idx_t u = g.rowind[e];
                if (part[u] == id && stamp[u] != bfs_id) {
                    stamp[u] = bfs_id;
                    level[u] = level[v] + 1;
                    q.push_back(u);
                }
            }
        }
        depth = level[q.back()];
        return q.back();
    };
    while (!stack.empty()) {
        Item it = std::move(stack.back());
        stack.pop_back();
        const idx_t m = (idx_t)it.v.size();
        if (m == 0) continue;
        for (idx_t v : it.v) part[v] = it.id;
        idx_t depth = 0;
        idx_t a = bfs(it.v[0], it.id, depth);
        if ((idx_t)q.size() < m) {  // disconnected: this component, then the rest
            Item c1, c2;
            c1.v = q;
            c2.v.reserve(m - q.size());
            for (idx_t v : it.v)
                if (stamp[v] != bfs_id) c2.v.push_back(v);
            c1.lo = it.lo;
            c2.lo = it.lo + (idx_t)c1.v.size();
            c1.id = nextpart++;
            c2.id = nextpart++;
            stack.push_back(std::move(c2));
            stack.push_back(std::move(c1));
            continue;
        }
        if (m <= leaf) {
            for (idx_t i = 0; i < m; i++) o.permtab[q[i]] = it.lo + i;
            continue;
        }
        for (int sweep = 0; sweep < 2; sweep++) {  // pseudo-peripheral vertex
            idx_t d2 = 0;
            idx_t b = bfs(a, it.id, d2);
            if (d2 <= depth) break;
            depth = d2;
            a = b;
        }
        bfs(a, it.id, depth);
        std::vector<idx_t> cnt(depth + 2, 0);
        for (idx_t v : q) cnt[level[v]]++;
        idx_t half = m / 2, acc = 0, sep = 0;
        for (idx_t l = 0; l <= depth; l++) {
            acc += cnt[l];
            if (acc > half) { sep = l; break; }
        }
        if (depth == 0) {  // a clique-like part: number as a leaf
            for (idx_t i = 0; i < m; i++) o.permtab[q[i]] = it.lo + i;
            continue;
        }
        Item A, B;
        std::vector<idx_t> S;
        for (idx_t v : q) {
            if (level[v] < sep) A.v.push_back(v);
            else if (level[v] > sep) B.v.push_back(v);
            else S.push_back(v);
        }
        idx_t hi = it.lo + m;
        for (idx_t i = 0; i < (idx_t)S.size(); i++) o.permtab[S[i]] = hi - (idx_t)S.size() + i;
        A.lo = it.lo;
        B.lo = it.lo + (idx_t)A.v.size();
        A.id = nextpart++;
        B.id = nextpart++;
        stack.push_back(std::move(B));
        stack.push_back(std::move(A));
    }
    for (idx_t i = 0; i < n; i++) o.peritab[o.permtab[i]] = i;
}

// ---------------------------------------------------------------------------
// Supernodes of a user ordering (orderFindSupernodes, order/order_find_supernodes.c):
// elimination tree by Liu's algorithm on the permuted graph, column structures
// by merging children, then column j+1 joins j's supernode when it is j's
// father and struct(j) = {j+1} U struct(j+1).
// ---------------------------------------------------------------------------
void order_find_supernodes(Order &o, const Graph &g) {
    idx_t n = g.n;
    if ((idx_t)o.permtab.size() != n) throw std::invalid_argument("order_find_supernodes: size mismatch");
    const auto &perm = o.permtab, &peri = o.peritab;
    std::vector<idx_t> parent(n, -1), anc(n, -1);
    for (idx_t j = 0; j < n; j++) {
        idx_t v = peri[j];
        for (idx_t e = g.colptr[v]; e < g.colptr[v + 1]; e++) {
            idx_t i = perm[g.rowind[e]];
            while (i != -1 && i < j) {
                idx_t nxt = anc[i];
                anc[i] = j;
                if (nxt == -1) parent[i] = j;
                i = nxt;
            }
        }
    }
    std::vector<idx_t> head(n, -1), next(n, -1);  // children lists
    for (idx_t j = n - 1; j >= 0; j--)
        if (parent[j] >= 0) { next[j] = head[parent[j]]; head[parent[j]] = j; }
    std::vector<std::vector<idx_t>> st(n);
    std::vector<idx_t> mark(n, -1), cnt(n, 0);
    for (idx_t j = 0; j < n; j++) {
        std::vector<idx_t> s;
        idx_t v = peri[j];
        for (idx_t e = g.colptr[v]; e < g.colptr[v + 1]; e++) {
            idx_t i = perm[g.rowind[e]];
            if (i > j && mark[i] != j) { mark[i] = j; s.push_back(i); }
        }
        for (idx_t c = head[j]; c != -1; c = next[c]) {
            for (idx_t i : st[c])
                if (i > j && mark[i] != j) { mark[i] = j; s.push_back(i); }
            std::vector<idx_t>().swap(st[c]);
        }
        cnt[j] = (idx_t)s.size();
        st[j].swap(s);
    }
    std::vector<idx_t> rang{0};
    for (idx_t j = 0; j + 1 < n; j++) {
        bool same = (parent[j] == j + 1) && (cnt[j] == cnt[j + 1] + 1);
        if (!same) rang.push_back(j + 1);
    }
    if (n > 0) rang.push_back(n);
    o.cblknbr = (idx_t)rang.size() - 1;
    o.rangtab = rang;
    std::vector<idx_t> sn(n);
    for (idx_t k = 0; k < o.cblknbr; k++)
        for (idx_t c = rang[k]; c < rang[k + 1]; c++) sn[c] = k;
    o.treetab.assign(o.cblknbr, -1);
    for (idx_t k = 0; k < o.cblknbr; k++) {
        idx_t p = parent[rang[k + 1] - 1];
        o.treetab[k] = (p < 0) ? -1 : sn[p];
    }
}

std::string order_check(const Order &o) {
    std::ostringstream err;
    idx_t n = o.n;
    if ((idx_t)o.permtab.size() != n || (idx_t)o.peritab.size() != n) return "size";
    std::vector<char> seen(n, 0);
    for (idx_t i = 0; i < n; i++) {
        idx_t p = o.permtab[i];
        if (p < 0 || p >= n || seen[p]) { err << "permtab not a permutation at " << i; return err.str(); }
        seen[p] = 1;
        if (o.peritab[p] != i) { err << "peritab not inverse at " << p; return err.str(); }
    }
    if (o.rangtab.empty() || o.rangtab.front() != 0 || o.rangtab.back() != n) return "rangtab bounds";
    for (idx_t k = 0; k < o.cblknbr; k++) {
        if (o.rangtab[k + 1] <= o.rangtab[k]) { err << "empty supernode " << k; return err.str(); }
        idx_t f = o.treetab[k];
        if (f != -1 && f <= k) { err << "treetab not increasing at " << k; return err.str(); }
    }
    return "";
}

// ---------------------------------------------------------------------------
// Block symbolic factorization (pastixSymbolFaxDirect symbol/symbol_fax_direct.c:66,
// body symbol/symbol_fax.c:152-519).  The rows of cblk k below its diagonal
// block are the union of (a) the permuted graph neighbours of its columns that
// lie after the cblk and (b) the rows of every contributing cblk c (a cblk
// whose first off-diagonal blok faces k) that lie after k.  The union is cut
// into maximal runs of consecutive rows that face a single cblk; each run is
// one blok.  The diagonal blok comes first.
// ---------------------------------------------------------------------------
void symbol_fax(Symbol &s, const Graph &g, const Order &o) {
    idx_t cbn = o.cblknbr;
    const auto &rang = o.rangtab;
    s.nodenbr = o.n;
    s.cblktab.assign(cbn + 1, SymCblk{0, 0, 0});
    s.bloktab.clear();
    s.bloktab.reserve(cbn * 4);
    std::vector<idx_t> chead(cbn, -1), cnext(cbn, -1);  // contribution chains
    std::vector<idx_t> col2cblk(o.n);
    for (idx_t k = 0; k < cbn; k++)
        for (idx_t c = rang[k]; c < rang[k + 1]; c++) col2cblk[c] = k;

    std::vector<std::pair<idx_t, idx_t>> iv;
    for (idx_t k = 0; k < cbn; k++) {
        idx_t fcol = rang[k], lcol = rang[k + 1] - 1;
        s.cblktab[k] = SymCblk{fcol, lcol, (idx_t)s.bloktab.size()};
        iv.clear();
        for (idx_t c = fcol; c <= lcol; c++) {
            idx_t v = o.peritab[c];
            for (idx_t e = g.colptr[v]; e < g.colptr[v + 1]; e++) {
                idx_t r = o.permtab[g.rowind[e]];
                if (r > lcol) iv.emplace_back(r, r);
            }
        }
        for (idx_t c = chead[k]; c != -1; c = cnext[c]) {
            for (idx_t b = s.cblktab[c].bloknum + 1; b < s.cblktab[c + 1].bloknum; b++) {
                const SymBlok &bk = s.bloktab[b];
                if (bk.frownum > lcol) iv.emplace_back(bk.frownum, bk.lrownum);
            }
        }
        std::sort(iv.begin(), iv.end());
        s.bloktab.push_back(SymBlok{fcol, lcol, k, k});
        idx_t i = 0, m = (idx_t)iv.size();
        while (i < m) {
            idx_t a = iv[i].first, b = iv[i].second;
            i++;
            while (i < m && iv[i].first <= b + 1) { b = std::max(b, iv[i].second); i++; }
            while (a <= b) {  // split the run at cblk boundaries
                idx_t f = col2cblk[a];
                idx_t e = std::min(b, rang[f + 1] - 1);
                s.bloktab.push_back(SymBlok{a, e, k, f});
                a = e + 1;
            }
        }
        idx_t fb = s.cblktab[k].bloknum;
        if ((idx_t)s.bloktab.size() > fb + 1) {
            idx_t f = s.bloktab[fb + 1].fcblknm;
            cnext[k] = chead[f];
            chead[f] = k;
        }
    }
    s.cblktab[cbn] = SymCblk{o.n, o.n - 1, (idx_t)s.bloktab.size()};
}

// ---------------------------------------------------------------------------
// Supernode splitting (splitSymbol blend/splitsymbol.c:522, splitSmart :378-499,
// computeNbSplit :78-102, computeSmallestSplit :168-210, extraCblkMerge
// blend/extracblk.c:222).  A cblk wider than blcolmax is cut into pieces of
// about width/ceil(width/blcolmax) columns; each cut point may move by up to
// 10% of the step to where it cuts the fewest existing bloks.  Piece j keeps a
// dense blok facing every later piece of the same cblk plus the original
// off-diagonal bloks; every blok facing a split cblk is cut at the pieces.
// ---------------------------------------------------------------------------
static idx_t nb_split(idx_t width, idx_t bmin, idx_t bmax) {
    if (width <= bmax) return 1;
    idx_t nseq = iceil(width, bmax);
    if (nseq > 1 && (width / nseq) < bmin) nseq--;
    return nseq;
}

static idx_t smallest_split(const idx_t *nbl, idx_t step, idx_t mn, idx_t mx, idx_t pct) {
    idx_t limit = iceil(step * pct, 100);
    if (step >= mx) return mx - 1;
    idx_t lavg = step - 1;
    idx_t lmin = std::max(lavg - limit - 1, mn);
    idx_t lmax = std::min(lavg + limit + 1, mx);
    idx_t best = lavg, nb = nbl[lavg];
    for (idx_t i = lavg + 1; i < lmax; i++)
        if (nbl[i] < nb) { best = i; nb = nbl[i]; }
    for (idx_t i = lavg - 1; i > lmin; i--)
        if (nbl[i] < nb) { best = i; nb = nbl[i]; }
    return best;
}

void symbol_split(Symbol &s, idx_t bmin, idx_t bmax) {
    idx_t cbn = s.cblknbr();
    std::vector<std::vector<std::pair<idx_t, idx_t>>> pieces(cbn);
    std::vector<idx_t> nbl;  // blocks cut between line i and i+1, from line fsplit
    idx_t fsplit = -1;
    bool any = false;
    for (idx_t k = 0; k < cbn; k++) {
        idx_t fcol = s.cblktab[k].fcolnum, lcol = s.cblktab[k].lcolnum;
        idx_t width = lcol - fcol + 1;
        if (nb_split(width, bmin, bmax) <= 1) { pieces[k].emplace_back(fcol, lcol); continue; }
        any = true;
        if (fsplit < 0) {
            fsplit = fcol;
            nbl.assign(s.nodenbr - fsplit + 1, 0);
            for (const auto &b : s.bloktab) {
                if (b.lrownum < fsplit) continue;
                for (idx_t l = std::max(b.frownum, fsplit); l < b.lrownum; l++) nbl[l - fsplit]++;
            }
        }
        idx_t fc = fcol;
        while (fc <= lcol) {
            idx_t nseq = nb_split(width, bmin, bmax);
            if (nseq == 1) { pieces[k].emplace_back(fc, lcol); fc = lcol + 1; continue; }
            idx_t step = iceil(width, nseq);
            idx_t lwidth = width - bmin;
            idx_t lc = fc + smallest_split(nbl.data() + (fc - fsplit), step, bmin, lwidth, 10);
            pieces[k].emplace_back(fc, lc);
            width -= lc - fc + 1;
            fc = lc + 1;
        }
        idx_t add = (idx_t)pieces[k].size() - 1;
        for (idx_t b = s.cblktab[k].bloknum + 1; b < s.cblktab[k + 1].bloknum; b++)
            for (idx_t l = s.bloktab[b].frownum; l < s.bloktab[b].lrownum; l++) nbl[l - fsplit] += add;
    }
    if (!any) return;

    std::vector<idx_t> first(cbn + 1, 0);
    for (idx_t k = 0; k < cbn; k++) first[k + 1] = first[k] + (idx_t)pieces[k].size();
    Symbol ns;
    ns.nodenbr = s.nodenbr;
    ns.cblktab.reserve(first[cbn] + 1);
    ns.bloktab.reserve(s.bloktab.size() * 2);
    for (idx_t k = 0; k < cbn; k++) {
        const auto &pk = pieces[k];
        idx_t np = (idx_t)pk.size();
        for (idx_t j = 0; j < np; j++) {
            idx_t me = first[k] + j;
            ns.cblktab.push_back(SymCblk{pk[j].first, pk[j].second, (idx_t)ns.bloktab.size()});
            for (idx_t jj = j; jj < np; jj++)  // dense triangle of the split diagonal block
                ns.bloktab.push_back(SymBlok{pk[jj].first, pk[jj].second, me, first[k] + jj});
            for (idx_t b = s.cblktab[k].bloknum + 1; b < s.cblktab[k + 1].bloknum; b++) {
                const SymBlok &ob = s.bloktab[b];
                const auto &pf = pieces[ob.fcblknm];
                idx_t fr = ob.frownum;
                for (idx_t q = 0; q < (idx_t)pf.size() && fr <= ob.lrownum; q++) {
                    if (fr > pf[q].second) continue;
                    idx_t lr = std::min(ob.lrownum, pf[q].second);
                    ns.bloktab.push_back(SymBlok{fr, lr, me, first[ob.fcblknm] + q});
                    fr = lr + 1;
                }
            }
        }
    }
    ns.cblktab.push_back(SymCblk{s.nodenbr, s.nodenbr - 1, (idx_t)ns.bloktab.size()});
    s = std::move(ns);
}

// Symbol of nodes -> symbol of unknowns, dof per node (the expansion
// blend/solver_matrix_gen.c applies when it builds the solver of a dof > 1
// matrix): every column or row range [f, l] becomes [f*dof, l*dof + dof-1].
void symbol_expand(const Symbol &node, idx_t dof, Symbol &out) {
    out.nodenbr = node.nodenbr * dof;
    out.cblktab = node.cblktab;
    for (auto &c : out.cblktab) {
        c.fcolnum *= dof;
        c.lcolnum = c.lcolnum * dof + dof - 1;
    }
    out.cblktab.back().fcolnum = out.nodenbr;
    out.cblktab.back().lcolnum = out.nodenbr - 1;
    out.bloktab = node.bloktab;
    for (auto &b : out.bloktab) {
        b.frownum *= dof;
        b.lrownum = b.lrownum * dof + dof - 1;
    }
}

std::string symbol_check(const Symbol &s) {
    std::ostringstream err;
    idx_t cbn = s.cblknbr();
    idx_t prev = -1;
    for (idx_t k = 0; k < cbn; k++) {
        const SymCblk &c = s.cblktab[k];
        if (c.fcolnum != prev + 1 || c.lcolnum < c.fcolnum) { err << "cblk range " << k; return err.str(); }
        prev = c.lcolnum;
        idx_t fb = c.bloknum, lb = s.cblktab[k + 1].bloknum;
        if (lb <= fb) { err << "no diagonal blok " << k; return err.str(); }
        const SymBlok &d = s.bloktab[fb];
        if (d.frownum != c.fcolnum || d.lrownum != c.lcolnum || d.fcblknm != k) { err << "diag " << k; return err.str(); }
        idx_t last = c.lcolnum;
        for (idx_t b = fb + 1; b < lb; b++) {
            const SymBlok &bk = s.bloktab[b];
            if (bk.lcblknm != k) { err << "lcblknm " << b; return err.str(); }
            if (bk.frownum <= last || bk.lrownum < bk.frownum) { err << "blok order " << b; return err.str(); }
            const SymCblk &f = s.cblktab[bk.fcblknm];
            if (bk.fcblknm <= k || bk.frownum < f.fcolnum || bk.lrownum > f.lcolnum) { err << "facing " << b; return err.str(); }
            last = bk.lrownum;
        }
    }
    if (prev != s.nodenbr - 1) return "columns do not cover the matrix";
    return "";
}

// ---------------------------------------------------------------------------
// Theoretical factorization flops (pastixSymbolGetFlops symbol/symbol_cost.c:422,
// sum1d :53-88, real tables symbol/symbol_cost_flops.c:291-306, macros
// common/flops.h:49-104).  factotype: 0 POTRF, 1 SYTRF, 2 GETRF, 3 PXTRF, 4 HETRF.
// ---------------------------------------------------------------------------
static double fl_gemm(double m, double n, double k) { return 2.0 * m * n * k; }
static double fl_syrk(double k, double n) { return k * n * (n + 1.0); }
static double fl_trsm_right(double m, double n) {  // FLOPS_DTRSM(Right, m, n): TRMM_2(n, m) mults twice
    return 2.0 * (0.5 * m * n * (n + 1.0));
}
static double fl_potrf(double n) {
    return n * (((1. / 6.) * n + 0.5) * n + (1. / 3.)) + n * (((1. / 6.) * n) * n - (1. / 6.));
}
static double fl_sytrf(double n) {
    return n * (((1. / 6.) * n + 0.5) * n + (10. / 3.)) + n * (((1. / 6.) * n) * n - (1. / 6.));
}
static double fl_getrf(double m, double n) {
    double mu, ad;
    if (m < n) {
        mu = 0.5 * m * (m * (n - (1. / 3.) * m - 1.) + n) + (2. / 3.) * m;
        ad = 0.5 * m * (m * (n - (1. / 3.) * m) - n) + (1. / 6.) * m;
    } else {
        mu = 0.5 * n * (n * (m - (1. / 3.) * n - 1.) + m) + (2. / 3.) * n;
        ad = 0.5 * n * (n * (m - (1. / 3.) * n) - m) + (1. / 6.) * n;
    }
    return mu + ad;
}

double symbol_flops(const Symbol &s, int factotype) {
    double tot = 0.0;
    for (idx_t k = 0; k < s.cblknbr(); k++) {
        double N = (double)(s.cblktab[k].lcolnum - s.cblktab[k].fcolnum + 1);
        double M = 0;
        for (idx_t b = s.cblktab[k].bloknum + 1; b < s.cblktab[k + 1].bloknum; b++)
            M += (double)(s.bloktab[b].lrownum - s.bloktab[b].frownum + 1);
        double f;
        switch (factotype) {
            case 1: case 4:  // SYTRF
                f = fl_sytrf(N);
                if (M > 0) f += fl_trsm_right(M, N) + N * M + fl_syrk(N, M) + M * M;
                break;
            case 2:  // GETRF
                f = fl_getrf(N, N);
                if (M > 0) f += 2.0 * fl_trsm_right(M, N) + fl_gemm(M, M, N);
                break;
            default:  // POTRF / PXTRF
                f = fl_potrf(N);
                if (M > 0) f += fl_trsm_right(M, N) + fl_syrk(N, M);
        }
        tot += f;
    }
    return tot;
}

// ---------------------------------------------------------------------------
// Solver layout and schedule.
//
// Layout (this project's own, replacing the 2D per-blok layout of
// blend/solver_matrix_gen_utils.h:69-176): every cblk is one column-major
// panel of stride rows x width columns, ld = stride, diagonal block on top,
// off-diagonal bloks below in blok order.  LU keeps a second panel of the same
// shape for U^T (the ucoeftab of the reference).
//
// Levels: level(k) = 1 + max level of the cblks that have a blok facing k
// (0 when none).  All cblks of a level are independent, so one level is one
// batch of kernels; this replaces the contribution counters of
// kernels/cpucblk_zmpi_coeftab.c:543-614.
// ---------------------------------------------------------------------------
void solver_build(Solver &sv, const Symbol &s, int factotype) {
    idx_t cbn = s.cblknbr(), bkn = s.bloknbr();
    sv = Solver{};
    sv.n = s.nodenbr;
    sv.cblknbr = cbn;
    sv.bloknbr = bkn;
    sv.factotype = factotype;
    sv.cb_fcol.resize(cbn); sv.cb_lcol.resize(cbn); sv.cb_fblok.resize(cbn + 1);
    sv.cb_stride.resize(cbn); sv.cb_coef.resize(cbn + 1); sv.cb_level.resize(cbn);
    sv.cb_rowidx.resize(cbn + 1);
    sv.bk_frow.resize(bkn); sv.bk_lrow.resize(bkn); sv.bk_fcblk.resize(bkn);
    sv.bk_lcblk.resize(bkn); sv.bk_rowoff.resize(bkn);
    idx_t coef = 0, rows = 0;
    for (idx_t k = 0; k < cbn; k++) {
        const SymCblk &c = s.cblktab[k];
        sv.cb_fcol[k] = c.fcolnum;
        sv.cb_lcol[k] = c.lcolnum;
        sv.cb_fblok[k] = c.bloknum;
        idx_t off = 0;
        for (idx_t b = c.bloknum; b < s.cblktab[k + 1].bloknum; b++) {
            const SymBlok &bk = s.bloktab[b];
            sv.bk_frow[b] = bk.frownum;
            sv.bk_lrow[b] = bk.lrownum;
            sv.bk_fcblk[b] = bk.fcblknm;
            sv.bk_lcblk[b] = bk.lcblknm;
            sv.bk_rowoff[b] = off;
            off += bk.lrownum - bk.frownum + 1;
        }
        sv.cb_stride[k] = off;
        sv.cb_coef[k] = coef;
        sv.cb_rowidx[k] = rows;
        coef += off * (c.lcolnum - c.fcolnum + 1);
        rows += off;
    }
    sv.cb_fblok[cbn] = bkn;
    sv.cb_coef[cbn] = coef;
    sv.cb_rowidx[cbn] = rows;
    sv.coefnbr = coef;
    sv.nnzl = coef;
    sv.rowidx.resize(rows);
    for (idx_t k = 0; k < cbn; k++) {
        idx_t r = sv.cb_rowidx[k];
        for (idx_t b = sv.cb_fblok[k]; b < sv.cb_fblok[k + 1]; b++)
            for (idx_t g = sv.bk_frow[b]; g <= sv.bk_lrow[b]; g++) sv.rowidx[r++] = g;
    }
    // browtab: off-diagonal bloks facing each cblk, by increasing source cblk
    sv.cb_brow.assign(cbn + 1, 0);
    for (idx_t b = 0; b < bkn; b++)
        if (sv.bk_fcblk[b] != sv.bk_lcblk[b]) sv.cb_brow[sv.bk_fcblk[b] + 1]++;
    for (idx_t k = 0; k < cbn; k++) sv.cb_brow[k + 1] += sv.cb_brow[k];
    sv.browtab.resize(sv.cb_brow[cbn]);
    {
        std::vector<idx_t> pos(sv.cb_brow.begin(), sv.cb_brow.end() - 1);
        for (idx_t b = 0; b < bkn; b++)
            if (sv.bk_fcblk[b] != sv.bk_lcblk[b]) sv.browtab[pos[sv.bk_fcblk[b]]++] = b;
    }
    // levels
    idx_t maxl = 0;
    for (idx_t k = 0; k < cbn; k++) {
        idx_t l = 0;
        for (idx_t p = sv.cb_brow[k]; p < sv.cb_brow[k + 1]; p++)
            l = std::max(l, sv.cb_level[sv.bk_lcblk[sv.browtab[p]]] + 1);
        sv.cb_level[k] = l;
        maxl = std::max(maxl, l);
    }
    sv.nlevels = cbn ? maxl + 1 : 0;
    sv.lvl_ptr.assign(sv.nlevels + 1, 0);
    for (idx_t k = 0; k < cbn; k++) sv.lvl_ptr[sv.cb_level[k] + 1]++;
    for (idx_t l = 0; l < sv.nlevels; l++) sv.lvl_ptr[l + 1] += sv.lvl_ptr[l];
    sv.lvl_cblk.resize(cbn);
    {
        std::vector<idx_t> pos(sv.lvl_ptr.begin(), sv.lvl_ptr.end() - 1);
        for (idx_t k = 0; k < cbn; k++) sv.lvl_cblk[pos[sv.cb_level[k]]++] = k;
    }
    // update tasks, grouped by the level of their source
    sv.lvl_task_ptr.assign(sv.nlevels + 1, 0);
    sv.tasks.clear();
    for (idx_t l = 0; l < sv.nlevels; l++) {
        for (idx_t p = sv.lvl_ptr[l]; p < sv.lvl_ptr[l + 1]; p++) {
            idx_t k = sv.lvl_cblk[p];
            for (idx_t b = sv.cb_fblok[k] + 1; b < sv.cb_fblok[k + 1]; b++) {
                Task t;
                t.src = k;
                t.dst = sv.bk_fcblk[b];
                t.blok = b;
                t.row0 = sv.bk_rowoff[b];
                t.n = sv.bk_lrow[b] - sv.bk_frow[b] + 1;
                t.m = sv.cb_stride[k] - t.row0;
                sv.tasks.push_back(t);
            }
        }
        sv.lvl_task_ptr[l + 1] = (idx_t)sv.tasks.size();
    }
    sv.thflops = symbol_flops(s, factotype);
}

}  // namespace pgpu
