// forest.cpp -- host quadtree forest on a brick of trees.
//
// Stands in for the p4est forest that the reference's AMR driver owns
// (src/amr/src/amr_initialize.c:213-314, amr_regrid.c:101-125,
// amr_external.c:211-508), which is not available here. It produces the
// same flat arrays the reference hands to hpc_amr_evolve_solver:
//   cell_info  3 ints per quad  {type, level, soln offset = 4 n^2 * id}
//              (amr_external.c:358-360)
//   face_info 11 ints per face  {ftype 1 boundary / 2 full / 3 hanging,
//              side of the full (or only) quad, its id, 4 neighbour ids,
//              4 neighbour sides}                (amr_external.c:389-507)
//   geom      12 doubles per quad, corners n1(-,-) n2(+,-) n3(-,+) n4(+,+)
//              (amr_p4est_utilities.c:15-81)
//
// Semantics kept from p4est: trees of a brick are numbered along the
// Morton curve of their (tx,ty) position; leaves are ordered by tree, then
// Morton index; refine replaces a leaf by its four z-ordered children;
// coarsen replaces a complete family by its parent; balance enforces the
// 2:1 condition across faces and corners (P4EST_CONNECT_FULL).
//
// Deliberate, documented choices where p4est's behaviour is not part of the
// solver arithmetic: faces are listed in order of the first leaf (in Morton
// order) that touches them, sides 0..3; for a full face side[0] follows
// p4est's rule (lower quadrant inside a tree, lower tree / lower face
// across trees); a refined child inherits its parent's tag.
#include "amrgpu_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace amrgpu {

namespace {

// Host threads for the forest's per-leaf loops: AMRGPU_HOST_THREADS, else
// the hardware's count, at most 16.
int host_threads()
{
    static const int n = [] {
        if (const char *e = std::getenv("AMRGPU_HOST_THREADS")) {
            const int v = std::atoi(e);
            if (v >= 1) return std::min(v, 64);
        }
        const unsigned hw = std::thread::hardware_concurrency();
        return int(std::max(1u, std::min(hw, 16u)));
    }();
    return n;
}

// fn(begin, end, chunk) over [0, n) in contiguous chunks, one thread each;
// one chunk (no thread) below `grain` items per thread.
template <typename Fn>
int parallel_chunks(size_t n, size_t grain, Fn fn)
{
    int nt = int(std::min<size_t>(size_t(host_threads()), std::max<size_t>(1, n / std::max<size_t>(grain, 1))));
    if (nt <= 1) {
        fn(size_t(0), n, 0);
        return 1;
    }
    std::vector<std::thread> th;
    th.reserve(size_t(nt));
    for (int c = 0; c < nt; ++c)
        th.emplace_back(fn, n * size_t(c) / size_t(nt), n * size_t(c + 1) / size_t(nt), c);
    for (auto &t : th) t.join();
    return nt;
}

constexpr int kMaxLevel = 30;
constexpr int64_t kRootLen = int64_t(1) << kMaxLevel;

inline int64_t qlen(int level) { return int64_t(1) << (kMaxLevel - level); }

inline uint64_t spread_bits(uint64_t v)
{
    v &= 0x3fffffffULL;
    v = (v | (v << 16)) & 0x0000ffff0000ffffULL;
    v = (v | (v << 8)) & 0x00ff00ff00ff00ffULL;
    v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0fULL;
    v = (v | (v << 2)) & 0x3333333333333333ULL;
    v = (v | (v << 1)) & 0x5555555555555555ULL;
    return v;
}

inline uint64_t morton(int64_t x, int64_t y) { return spread_bits(uint64_t(x)) | (spread_bits(uint64_t(y)) << 1); }

struct Key {
    int tree, level;
    int64_t x, y;
};

}  // namespace

struct Forest {
    int nx = 1, ny = 1;
    int periodic[2] = {0, 0};
    double xlo[3] = {0, 0, 0};
    double scale = 1.0;
    // tree id -> brick position and back
    std::vector<int> tree_tx, tree_ty;
    std::vector<int> tree_at;  // [ty*nx+tx] -> tree id
    std::vector<Leaf> leaves;
    // output buffer of forest_adapt's single pass, swapped with `leaves`
    // afterwards; its capacity is kept from regrid to regrid
    std::vector<Leaf> spare;
    // advanced by every call that may change the leaves, so that a copy of
    // them elsewhere (a session's device leaves) can tell it is current
    uint64_t version = 0;

    int tree_of(int tx, int ty) const { return tree_at[size_t(ty) * nx + tx]; }

    // Morton index of each leaf's lower corner and the first leaf of each
    // tree: leaves stay sorted by (tree, Morton) through refine, coarsen and
    // balance, so point location is a binary search within the tree.
    mutable std::vector<uint64_t> keys;
    mutable std::vector<int> tree_begin;

    void sort_leaves()
    {
        std::sort(leaves.begin(), leaves.end(), [](const Leaf &a, const Leaf &b) {
            if (a.tree != b.tree) return a.tree < b.tree;
            return morton(a.x, a.y) < morton(b.x, b.y);
        });
    }

    void rebuild_keys() const
    {
        const size_t nl = leaves.size();
        keys.resize(nl);
        tree_begin.assign(size_t(nx) * ny + 1, int(nl));
        for (size_t i = nl; i-- > 0;) {
            keys[i] = morton(leaves[i].x, leaves[i].y);
            tree_begin[size_t(leaves[i].tree)] = int(i);
        }
        for (size_t t = tree_begin.size() - 1; t-- > 0;)
            tree_begin[t] = std::min(tree_begin[t], tree_begin[t + 1]);
    }

    // Leaf containing the point (x,y) of a tree: the last leaf of the tree
    // whose corner precedes the point on the Morton curve.
    int locate(int tree, int64_t x, int64_t y) const
    {
        const uint64_t m = morton(x, y);
        const uint64_t *b = keys.data() + tree_begin[size_t(tree)];
        const uint64_t *e = keys.data() + tree_begin[size_t(tree) + 1];
        return int(std::upper_bound(b, e, m) - keys.data()) - 1;
    }

    // Same-level neighbour region of (tree,level,x,y) across offset (dx,dy)
    // in units of the quadrant length; false when it leaves the domain.
    // At level kMaxLevel this moves a point by one finest unit.
    bool shifted(int tree, int level, int64_t x, int64_t y, int dx, int dy, Key &out) const
    {
        int64_t L = qlen(level);
        int64_t nxq = x + dx * L, nyq = y + dy * L;
        int tx = tree_tx[tree], ty = tree_ty[tree];
        if (nxq < 0) { nxq += kRootLen; tx -= 1; }
        if (nxq >= kRootLen) { nxq -= kRootLen; tx += 1; }
        if (nyq < 0) { nyq += kRootLen; ty -= 1; }
        if (nyq >= kRootLen) { nyq -= kRootLen; ty += 1; }
        if (tx < 0 || tx >= nx) {
            if (!periodic[0]) return false;
            tx = (tx + nx) % nx;
        }
        if (ty < 0 || ty >= ny) {
            if (!periodic[1]) return false;
            ty = (ty + ny) % ny;
        }
        out = Key{tree_of(tx, ty), level, nxq, nyq};
        return true;
    }

    // Leaf two or more levels coarser than q holding q's neighbour region
    // across (dx,dy) (q is the fine side of a 2:1 violation), else -1.
    int too_coarse_neighbour(const Leaf &q, int dx, int dy) const
    {
        Key k;
        if (!shifted(q.tree, q.level, q.x, q.y, dx, dy, k)) return -1;
        int c = locate(k.tree, k.x, k.y);
        return leaves[size_t(c)].level < q.level - 1 ? c : -1;
    }

    // True when a leaf touching q across a face or a corner is two or more
    // levels finer (q is the coarse side of a 2:1 violation). Faces are
    // walked leaf by leaf along the edge; corners take the diagonal point.
    bool has_too_fine_neighbour(const Leaf &q) const
    {
        const int64_t L = qlen(q.level);
        const int lim = q.level + 2;
        for (int s = 0; s < 4; ++s) {
            for (int64_t t = 0; t < L;) {
                int64_t px = q.x, py = q.y;
                int dx = 0, dy = 0;
                if (s == 0) { py += t; dx = -1; }
                if (s == 1) { px += L - 1; py += t; dx = 1; }
                if (s == 2) { px += t; dy = -1; }
                if (s == 3) { px += t; py += L - 1; dy = 1; }
                Key k;
                if (!shifted(q.tree, kMaxLevel, px, py, dx, dy, k)) break;
                const Leaf &c = leaves[size_t(locate(k.tree, k.x, k.y))];
                if (c.level >= lim) return true;
                const int64_t len = qlen(c.level);
                t += (s < 2) ? (c.y + len - k.y) : (c.x + len - k.x);
            }
        }
        for (int dy = -1; dy <= 1; dy += 2)
            for (int dx = -1; dx <= 1; dx += 2) {
                Key k;
                int64_t px = dx < 0 ? q.x : q.x + L - 1, py = dy < 0 ? q.y : q.y + L - 1;
                if (!shifted(q.tree, kMaxLevel, px, py, dx, dy, k)) continue;
                if (leaves[size_t(locate(k.tree, k.x, k.y))].level >= lim) return true;
            }
        return false;
    }
};

namespace {

void side_offset(int side, int &dx, int &dy)
{
    dx = 0; dy = 0;
    switch (side) {
    case 0: dx = -1; break;
    case 1: dx = 1; break;
    case 2: dy = -1; break;
    case 3: dy = 1; break;
    }
}

}  // namespace

Forest *forest_new_brick(int nx, int ny, int px, int py, double xlo, double ylo, double zlo,
                         double scale, int level)
{
    if (nx < 1 || ny < 1 || level < 0 || level > kMaxLevel) return nullptr;
    Forest *f = new Forest;
    f->nx = nx; f->ny = ny;
    f->periodic[0] = px ? 1 : 0; f->periodic[1] = py ? 1 : 0;
    f->xlo[0] = xlo; f->xlo[1] = ylo; f->xlo[2] = zlo;
    f->scale = scale;
    std::vector<std::pair<uint64_t, int>> order;
    for (int ty = 0; ty < ny; ++ty)
        for (int tx = 0; tx < nx; ++tx) order.push_back({morton(tx, ty), ty * nx + tx});
    std::sort(order.begin(), order.end());
    f->tree_tx.resize(order.size());
    f->tree_ty.resize(order.size());
    f->tree_at.resize(order.size());
    for (size_t t = 0; t < order.size(); ++t) {
        int lin = order[t].second;
        f->tree_tx[t] = lin % nx;
        f->tree_ty[t] = lin / nx;
        f->tree_at[size_t(lin)] = int(t);
    }
    int64_t per = int64_t(1) << level;
    int64_t L = qlen(level);
    f->leaves.reserve(size_t(nx) * ny * per * per);
    for (int t = 0; t < nx * ny; ++t)
        for (int64_t j = 0; j < per; ++j)
            for (int64_t i = 0; i < per; ++i) {
                Leaf q;
                q.tree = t; q.level = level; q.x = i * L; q.y = j * L;
                q.tag = 0; q.type = 0;
                f->leaves.push_back(q);
            }
    f->sort_leaves();
    forest_begin_regrid(f);
    return f;
}

void forest_destroy(Forest *f) { delete f; }

int forest_num_quads(const Forest *f) { return int(f->leaves.size()); }

const std::vector<Leaf> &forest_leaves(const Forest *f) { return f->leaves; }
std::vector<Leaf> &forest_leaves_mut(Forest *f)
{
    ++f->version;
    return f->leaves;
}

uint64_t forest_version(const Forest *f) { return f->version; }

void forest_grow_leaves(Forest *f, size_t n)
{
    ++f->version;
    std::vector<Leaf> &L = f->leaves;
    if (L.capacity() < n) L.reserve(n + n / 4);
    L.resize(n);
}

namespace {

// Replaces every leaf i with refine(i) true by its four z-ordered children,
// in place: the output index of a leaf is never below its input index, so
// the leaves are rewritten from the end backwards, down to the first
// refined leaf `first` (nout leaves in all); the prefix before it is not
// touched. Children take the parent's fields with child_tag (or the
// parent's tag when child_tag < 0) and dirty = 1; other leaves keep
// theirs, with dirty = keep_dirty (or as they are when keep_dirty < 0).
// Leaves are written field by field or whole, never copied whole right
// after some of their fields were overwritten (that stalls on store
// forwarding).
template <class Pred>
void refine_rewrite(Forest *f, size_t first, size_t nout, Pred refine, int child_tag, int keep_dirty)
{
    std::vector<Leaf> &L = f->leaves;
    const size_t n = L.size();
    if (nout == n) return;
    forest_grow_leaves(f, nout);
    size_t k = nout;
    for (size_t i = n; i-- > first;) {
        const bool r = refine(i);  // reads leaf i before anything at or below k-1 >= i is written
        const Leaf p = L[i];
        if (r) {
            const int64_t h = qlen(p.level + 1);
            for (int c = 3; c >= 0; --c) {
                Leaf &ch = L[--k];
                ch = p;
                ch.level = p.level + 1;
                ch.x = p.x + (c & 1) * h;
                ch.y = p.y + ((c >> 1) & 1) * h;
                if (child_tag >= 0) ch.tag = child_tag;
                ch.dirty = 1;
            }
        } else {
            Leaf &d = L[--k];
            d = p;
            if (keep_dirty >= 0) d.dirty = keep_dirty;
        }
    }
}

template <class Pred>
void refine_in_place(Forest *f, Pred refine, int child_tag, int keep_dirty)
{
    std::vector<Leaf> &L = f->leaves;
    const size_t n = L.size();
    size_t nout = n, first = n;
    for (size_t i = 0; i < n; ++i)
        if (refine(i)) {
            nout += 3;
            if (first == n) first = i;
        }
    if (keep_dirty >= 0)
        for (size_t i = 0; i < first; ++i) L[i].dirty = keep_dirty;
    refine_rewrite(f, first, nout, refine, child_tag, keep_dirty);
}

// Coarsening of complete families, in place and forwards: a leaf's output
// index never exceeds its input index, and each family (flag(i) per input
// index i, read before anything at it is written) is read before its parent
// is written.
template <class Flag>
void coarsen_in_place(Forest *f, Flag flag, int min_level)
{
    std::vector<Leaf> &L = f->leaves;
    size_t i = 0, w = 0, n = L.size();
    while (i < n) {
        const Leaf &a = L[i];
        bool family = false;
        if (a.level > 0 && a.level > min_level && i + 3 < n) {
            int64_t P = qlen(a.level - 1);
            int64_t px = (a.x / P) * P, py = (a.y / P) * P;
            if (a.x == px && a.y == py) {
                family = true;
                for (int c = 0; c < 4 && family; ++c) {
                    const Leaf &b = L[i + c];
                    int64_t h = qlen(a.level);
                    if (b.tree != a.tree || b.level != a.level || b.x != px + (c & 1) * h ||
                        b.y != py + ((c >> 1) & 1) * h || !flag(i + c) ||
                        b.src_kind != kRemapCopy || b.src != L[i].src + c)
                        family = false;
                }
            }
        }
        if (family) {
            Leaf p = a;
            p.level = a.level - 1;
            int64_t P = qlen(p.level);
            p.x = (a.x / P) * P;
            p.y = (a.y / P) * P;
            p.type = L[i + 3].type;  // the reference keeps the last child's type
            p.tag = 0;
            p.src = a.src;
            p.src_kind = kRemapAverage;
            p.dirty = 1;
            L[w++] = p;
            i += 4;
        } else {
            if (w != i) L[w] = L[i];
            ++w;
            ++i;
        }
    }
    L.resize(w);
}

}  // namespace

void forest_begin_regrid(Forest *f)
{
    ++f->version;
    for (size_t i = 0; i < f->leaves.size(); ++i) {
        f->leaves[i].src = int(i);
        f->leaves[i].src_kind = kRemapCopy;
    }
}

int forest_refine(Forest *f, const int *flags, int max_level)
{
    ++f->version;
    const std::vector<Leaf> &L = f->leaves;
    // children inherit the refine tag
    refine_in_place(f, [&](size_t i) { return flags[i] && L[i].level < max_level && L[i].level < kMaxLevel; }, 1,
                    -1);
    return int(f->leaves.size());
}

int forest_coarsen(Forest *f, const int *flags, int min_level)
{
    ++f->version;
    coarsen_in_place(f, [&](size_t i) { return flags[i] != 0; }, min_level);
    return int(f->leaves.size());
}

int forest_adapt(Forest *f, const int *tags, int refine_value, int coarsen_value, int min_level, int max_level)
{
    ++f->version;
    // One pass over the leaves into the spare buffer, equal to begin_regrid,
    // storing the tags, forest_refine and then forest_coarsen: the children
    // of a refined leaf all carry their parent's source index, so they never
    // form a coarsenable family, and a family is four consecutive unrefined
    // leaves (siblings, all tagged coarsen_value above min_level).
    std::vector<Leaf> &L = f->leaves;
    std::vector<Leaf> &out = f->spare;
    const size_t n = L.size();
    auto refines = [&](size_t i) {
        return tags[i] == refine_value && L[i].level < max_level && L[i].level < kMaxLevel;
    };
    auto coarsens = [&](size_t i) { return tags[i] == coarsen_value && L[i].level > min_level; };
    size_t nref = 0;
    for (size_t i = 0; i < n; ++i) nref += refines(i) ? 1 : 0;
    if (out.capacity() < n + 3 * nref) out.reserve(std::max(n + 3 * nref + (n + 3 * nref) / 4, L.capacity()));
    out.resize(n + 3 * nref);
    size_t w = 0, i = 0;
    while (i < n) {
        const Leaf &a = L[i];
        if (refines(i)) {
            const int64_t h = qlen(a.level + 1);
            for (int c = 0; c < 4; ++c) {
                Leaf &ch = out[w++];
                ch = a;
                ch.level = a.level + 1;
                ch.x = a.x + (c & 1) * h;
                ch.y = a.y + ((c >> 1) & 1) * h;
                ch.tag = 1;  // children carry the refine tag
                ch.src = int(i);
                ch.src_kind = kRemapCopy;
                ch.dirty = 1;
            }
            ++i;
            continue;
        }
        bool family = false;
        int64_t px = 0, py = 0;
        if (a.level > 0 && a.level > min_level && i + 3 < n) {
            const int64_t P = qlen(a.level - 1), h = qlen(a.level);
            px = (a.x / P) * P;
            py = (a.y / P) * P;
            if (a.x == px && a.y == py) {
                family = true;
                for (int c = 0; c < 4 && family; ++c) {
                    const Leaf &b = L[i + c];
                    if (b.tree != a.tree || b.level != a.level || b.x != px + (c & 1) * h ||
                        b.y != py + ((c >> 1) & 1) * h || refines(i + c) || !coarsens(i + c))
                        family = false;
                }
            }
        }
        Leaf &d = out[w++];
        d = a;
        d.src = int(i);
        if (family) {
            d.level = a.level - 1;
            d.x = px;
            d.y = py;
            d.type = L[i + 3].type;  // the reference keeps the last child's type
            d.tag = 0;
            d.src_kind = kRemapAverage;
            d.dirty = 1;
            i += 4;
        } else {
            d.tag = tags[i];
            d.src_kind = kRemapCopy;
            ++i;
        }
    }
    out.resize(w);
    L.swap(out);
    return int(L.size());
}

int forest_balance(Forest *f)
{
    ++f->version;
    // Refine until every leaf's face and corner neighbours are at most one
    // level coarser (2:1 across faces and corners). Leaves untouched since
    // the last balance are pairwise balanced, so every violation has a
    // dirty leaf on one side: each pass checks only dirty leaves, as the
    // fine side (flag the too-coarse neighbour) and as the coarse side
    // (flag itself); the children it creates are the next pass's dirty set.
    // The result is the same minimal balanced refinement as checking every
    // leaf on every pass.
    // The checks of one pass only read the forest: they run on host threads
    // over the dirty leaves, each thread listing the leaves it flags.
    for (int iter = 0; iter < 64; ++iter) {
        f->rebuild_keys();
        const size_t nl = f->leaves.size();
        std::vector<int> dirty;
        for (size_t i = 0; i < nl; ++i)
            if (f->leaves[i].dirty) dirty.push_back(int(i));
        std::vector<std::vector<int>> hits((size_t)host_threads());
        parallel_chunks(dirty.size(), 512, [&](size_t b, size_t e, int t) {
            std::vector<int> &h = hits[size_t(t)];
            for (size_t k = b; k < e; ++k) {
                const int i = dirty[k];
                const Leaf &q = f->leaves[size_t(i)];
                if (q.level >= 2)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            if (!dx && !dy) continue;
                            const int c = f->too_coarse_neighbour(q, dx, dy);
                            if (c >= 0) h.push_back(c);
                        }
                if (q.level + 2 <= kMaxLevel && f->has_too_fine_neighbour(q)) h.push_back(i);
            }
        });
        std::vector<unsigned char> flags(nl, 0);
        bool any = false;
        for (const auto &h : hits)
            for (int c : h) {
                flags[size_t(c)] = 1;
                any = true;
            }
        if (!any) {
            for (Leaf &q : f->leaves) q.dirty = 0;
            return int(f->leaves.size());
        }
        // balance refinement keeps the refined quad's own tag on its children
        refine_in_place(f, [&](size_t i) { return flags[i] != 0; }, -1, 0);
    }
    return -1;
}

bool forest_is_balanced(const Forest *f)
{
    f->rebuild_keys();
    for (const Leaf &q : f->leaves) {
        if (q.level < 2) continue;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
                if ((dx || dy) && f->too_coarse_neighbour(q, dx, dy) >= 0) return false;
    }
    return true;
}

// amr_p4est_utilities.c:15-81, 2D branch: corners of a quadrant through the
// brick tree's vertices (vertex = integer brick position * scale + lo).
void forest_brick(const Forest *f, BrickView *out)
{
    out->nx = f->nx;
    out->ny = f->ny;
    out->periodic[0] = f->periodic[0];
    out->periodic[1] = f->periodic[1];
    for (int k = 0; k < 3; ++k) out->xlo[k] = f->xlo[k];
    out->scale = f->scale;
    out->tree_tx = f->tree_tx.data();
    out->tree_ty = f->tree_ty.data();
    out->tree_at = f->tree_at.data();
}

void forest_quad_corners(const Forest *f, const Leaf &q, double xyz[12])
{
    const double intsize = 1.0 / double(kRootLen);
    double h2 = 0.5 * intsize * double(qlen(q.level));
    int tx = f->tree_tx[size_t(q.tree)], ty = f->tree_ty[size_t(q.tree)];
    double v[4][3];
    for (int k = 0; k < 4; ++k) {
        int vx = tx + (k & 1), vy = ty + ((k >> 1) & 1);
        v[k][0] = double(vx) * f->scale + f->xlo[0];
        v[k][1] = double(vy) * f->scale + f->xlo[1];
        v[k][2] = 0.0 * f->scale + f->xlo[2];
    }
    const double eta_z = 0.0;
    int k = 0;
    for (int yi = 0; yi < 2; ++yi) {
        double eta_y = intsize * double(q.y) + h2 * (1.0 + (2 * yi - 1));
        for (int xi = 0; xi < 2; ++xi) {
            double eta_x = intsize * double(q.x) + h2 * (1.0 + (2 * xi - 1));
            for (int j = 0; j < 3; ++j)
                xyz[3 * k + j] = ((1. - eta_z) * ((1. - eta_y) * ((1. - eta_x) * v[0][j] + eta_x * v[1][j]) +
                                                  eta_y * ((1. - eta_x) * v[2][j] + eta_x * v[3][j])));
            ++k;
        }
    }
}

// amr_initialize.c:326 -- quadrant edge length used by the per-quad callbacks
double forest_quad_h(const Forest *f, const Leaf &q)
{
    return f->scale * double(qlen(q.level)) / double(kRootLen);
}

namespace {

constexpr uint64_t kForestMagic = 0x31464741524d4147ULL;  // "GAMRAGF1"

template <typename T>
void put(std::vector<unsigned char> &o, const T &v)
{
    const unsigned char *p = reinterpret_cast<const unsigned char *>(&v);
    o.insert(o.end(), p, p + sizeof(T));
}

template <typename T>
bool get(const unsigned char *&p, const unsigned char *end, T &v)
{
    if (size_t(end - p) < sizeof(T)) return false;
    std::memcpy(&v, p, sizeof(T));
    p += sizeof(T);
    return true;
}

}  // namespace

std::vector<unsigned char> forest_save(const Forest *f)
{
    std::vector<unsigned char> o;
    put(o, kForestMagic);
    put(o, int32_t(f->nx));
    put(o, int32_t(f->ny));
    put(o, int32_t(f->periodic[0]));
    put(o, int32_t(f->periodic[1]));
    for (double v : f->xlo) put(o, v);
    put(o, f->scale);
    put(o, int64_t(f->leaves.size()));
    for (const Leaf &q : f->leaves) {
        put(o, int32_t(q.tree));
        put(o, int32_t(q.level));
        put(o, int64_t(q.x));
        put(o, int64_t(q.y));
        put(o, int32_t(q.tag));
        put(o, int32_t(q.type));
    }
    return o;
}

Forest *forest_load(const unsigned char *data, size_t size)
{
    const unsigned char *p = data, *end = data + size;
    uint64_t magic = 0;
    int32_t nx, ny, px, py;
    double xlo[3], scale;
    int64_t nl;
    if (!get(p, end, magic) || magic != kForestMagic || !get(p, end, nx) || !get(p, end, ny) || !get(p, end, px) ||
        !get(p, end, py) || !get(p, end, xlo[0]) || !get(p, end, xlo[1]) || !get(p, end, xlo[2]) ||
        !get(p, end, scale) || !get(p, end, nl))
        return nullptr;
    if (nx < 1 || ny < 1 || nl < 1 || int64_t(size_t(end - p)) < nl * 32) return nullptr;
    Forest *f = forest_new_brick(nx, ny, px, py, xlo[0], xlo[1], xlo[2], scale, 0);
    if (!f) return nullptr;
    f->leaves.clear();
    f->leaves.reserve(size_t(nl));
    for (int64_t k = 0; k < nl; ++k) {
        int32_t tree, level, tag, type;
        int64_t x, y;
        get(p, end, tree);
        get(p, end, level);
        get(p, end, x);
        get(p, end, y);
        get(p, end, tag);
        get(p, end, type);
        const bool ok = tree >= 0 && tree < nx * ny && level >= 0 && level <= kMaxLevel && x >= 0 && y >= 0 &&
                        x < kRootLen && y < kRootLen && x % qlen(level) == 0 && y % qlen(level) == 0;
        if (!ok) {
            delete f;
            return nullptr;
        }
        Leaf q;
        q.tree = tree;
        q.level = level;
        q.x = x;
        q.y = y;
        q.tag = tag;
        q.type = type;
        q.src = int(k);
        q.src_kind = kRemapCopy;
        f->leaves.push_back(q);
    }
    // the leaves must tile every tree in (tree, Morton) order
    unsigned __int128 covered = 0;  // in units of a level-30 quadrant
    for (size_t k = 0; k < f->leaves.size(); ++k) {
        const Leaf &q = f->leaves[k];
        if (k > 0) {
            const Leaf &a = f->leaves[k - 1];
            if (a.tree > q.tree || (a.tree == q.tree && morton(a.x, a.y) >= morton(q.x, q.y))) {
                delete f;
                return nullptr;
            }
        }
        covered += (unsigned __int128)1 << (2 * (kMaxLevel - q.level));
    }
    if (covered != (unsigned __int128)(nx * ny) << (2 * kMaxLevel)) {
        delete f;
        return nullptr;
    }
    return f;
}

int forest_external(const Forest *f, int nelem_subgrid, int nfields, int *cell_info,
                    int *face_info, double *geom, int *nface_out, int *dof_out)
{
    const int nq = int(f->leaves.size());
    const int nftm = nfields * nelem_subgrid * nelem_subgrid;
    f->rebuild_keys();
    // leaf exactly at (tree, level, x, y), else -1
    auto find = [&](int tree, int level, int64_t x, int64_t y) {
        int c = f->locate(tree, x, y);
        const Leaf &l = f->leaves[size_t(c)];
        return (l.level == level && l.x == x && l.y == y) ? c : -1;
    };
    for (int i = 0; i < nq; ++i) {
        const Leaf &q = f->leaves[size_t(i)];
        cell_info[3 * i + 0] = q.type;
        cell_info[3 * i + 1] = q.level;
        cell_info[3 * i + 2] = nftm * i;
        forest_quad_corners(f, q, &geom[12 * i]);
    }
    // Faces are listed in order of the first leaf (by index) that takes part
    // in them, sides 0..3 at that leaf: leaf i emits the face on its side s
    // when no participant of that face has a smaller index (a leaf that is
    // its own periodic neighbour emits from its even side). Every (leaf,
    // side) is decided independently, so leaves are split among host
    // threads and the per-chunk face lists are concatenated in leaf order.
    struct Part {
        std::vector<int> rec;
        int err = 0;
    };
    std::vector<Part> parts((size_t)host_threads());
    parallel_chunks(size_t(nq), 2048, [&](size_t b, size_t e, int t) {
        Part &P = parts[size_t(t)];
        P.rec.reserve((e - b) * 2 * 11);
        for (size_t ii = b; ii < e && !P.err; ++ii) {
            const int i = int(ii);
            const Leaf &q = f->leaves[ii];
            for (int s = 0; s < 4; ++s) {
                int dx, dy;
                side_offset(s, dx, dy);
                const int opp = s ^ 1;
                int v[11];
                for (int k = 0; k < 11; ++k) v[k] = -1;
                bool emit = true;
                Key k;
                if (!f->shifted(q.tree, q.level, q.x, q.y, dx, dy, k)) {
                    v[0] = 1; v[1] = s; v[2] = i;
                } else {
                    const int c0 = f->locate(k.tree, k.x, k.y);
                    const int lvl0 = f->leaves[size_t(c0)].level;
                    if (lvl0 == q.level) {
                        const int j = c0;
                        // side[0]: lower quadrant inside a tree; across trees
                        // the lower tree id, then the lower face number.
                        bool this_first;
                        const int tq = q.tree, tj = f->leaves[size_t(j)].tree;
                        if (tq == tj) this_first = (s & 1) == 1;
                        else this_first = (tq < tj) || (tq == tj && s < opp);
                        if (i == j) this_first = (s & 1) == 0;
                        const int a = this_first ? i : j, sa = this_first ? s : opp;
                        const int bq = this_first ? j : i, sb = this_first ? opp : s;
                        v[0] = 2; v[1] = sa; v[2] = a; v[3] = bq; v[7] = sb;
                        emit = (i < j) || (i == j && (s & 1) == 0);
                    } else if (lvl0 < q.level - 1) {
                        P.err = -2;  // not 2:1 balanced
                        break;
                    } else if (lvl0 == q.level - 1) {
                        // coarser neighbour: this quad is one of two hanging quads
                        const int c = c0;
                        const int64_t Lp = qlen(q.level - 1), L = qlen(q.level);
                        const int64_t base_x = (q.x / Lp) * Lp, base_y = (q.y / Lp) * Lp;
                        int fine[2];
                        for (int h = 0; h < 2; ++h) {
                            if (s < 2) fine[h] = find(q.tree, q.level, q.x, base_y + h * L);
                            else fine[h] = find(q.tree, q.level, base_x + h * L, q.y);
                        }
                        if (fine[0] < 0 || fine[1] < 0) {
                            P.err = -2;
                            break;
                        }
                        v[0] = 3; v[1] = opp; v[2] = c;
                        v[3] = fine[0]; v[4] = fine[1]; v[7] = s; v[8] = s;
                        emit = i == std::min(c, std::min(fine[0], fine[1]));
                    } else {
                        // finer neighbours: this quad is the full side of a hanging face
                        const int64_t Lc = qlen(q.level + 1);
                        int fine[2];
                        for (int h = 0; h < 2; ++h) {
                            if (s < 2)
                                fine[h] = find(k.tree, q.level + 1, (s == 0) ? k.x + Lc : k.x, k.y + h * Lc);
                            else
                                fine[h] = find(k.tree, q.level + 1, k.x + h * Lc, (s == 2) ? k.y + Lc : k.y);
                        }
                        if (fine[0] < 0 || fine[1] < 0) {
                            P.err = -3;  // not 2:1 balanced
                            break;
                        }
                        v[0] = 3; v[1] = s; v[2] = i;
                        v[3] = fine[0]; v[4] = fine[1]; v[7] = opp; v[8] = opp;
                        emit = i < std::min(fine[0], fine[1]);
                    }
                }
                if (emit) P.rec.insert(P.rec.end(), v, v + 11);
            }
        }
    });
    int nface = 0;
    for (const Part &P : parts) {
        if (P.err) return P.err;
        std::memcpy(face_info + 11 * size_t(nface), P.rec.data(), sizeof(int) * P.rec.size());
        nface += int(P.rec.size() / 11);
    }
    *nface_out = nface;
    *dof_out = nftm * nq;
    return 0;
}

}  // namespace amrgpu
