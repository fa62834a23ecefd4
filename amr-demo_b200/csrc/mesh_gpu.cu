// mesh_gpu.cu -- a forest's 2:1 balance and its mesh's quad descriptors on
// the GPU.
//
// Balance (forest_balance's passes, forest.cpp): every pass checks the
// leaves created since the last pass (dirty), as the fine side of a
// violation (a face or corner neighbour region held by a leaf two or more
// levels coarser: that leaf is flagged) and as the coarse side (a leaf two
// or more levels finer along an edge or at a corner: the leaf itself is
// flagged); flagged leaves are replaced by their four z-ordered children,
// which are the next pass's dirty set. One thread per leaf checks; the
// refinement is a scan of 4-or-1 counts and a scatter, so Morton order is
// kept. Same passes, same result as the host's.
//
// After a regrid the host forest has its new leaves (tree, level, x, y in
// Morton order). The reference's driver then lists the mesh's faces
// (amr_external.c:389-507) and the solver decodes them per quad
// (physics_rhs_structured.c:73-262); the host path of this library does the
// same (forest_external, then decode_mesh). Here the device does both in
// one pass per (leaf, side), with the forest's rules of forest_external:
//
//   * the side's same-level neighbour region (across tree faces of the
//     brick, periodic where the brick is) and the leaf holding it, found by
//     binary search over the leaves' Morton keys within the tree;
//   * the face type: boundary, full (same level), hanging with this leaf
//     fine (coarser neighbour) or coarse (two finer neighbours);
//   * the face's emitter, the participant with the smallest index, from
//     its side (a leaf that is its own periodic neighbour emits from its
//     even side): faces are numbered in emission order, leaf by leaf, sides
//     0..3, so an exclusive scan of the per-(leaf, side) "emits" flags
//     gives every face its index in the host's face list;
//   * the side descriptor the host decode writes (kind, neighbours, the
//     level that sizes the face, the boundary condition) and the face
//     index as accumulation rank; the corners with the host's arithmetic
//     (forest_quad_corners), each operation explicitly rounded.
//
// A 2:1 violation is reported through status[0]; status[1] gets the face
// count. The result is byte-identical to decode_mesh(forest_external(...)).
#include <cuda_runtime.h>

#include <algorithm>

#include <cub/device/device_scan.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include "device_common.cuh"
#include "mesh_gpu.h"

namespace amrgpu {

namespace {

constexpr int kMaxLevelG = 30;
constexpr long long kRootLenG = 1ll << kMaxLevelG;

__device__ __forceinline__ long long qlen_d(int level) { return 1ll << (kMaxLevelG - level); }

__device__ __forceinline__ unsigned long long spread_bits_d(unsigned long long v)
{
    v &= 0xffffffffULL;
    v = (v | (v << 16)) & 0x0000ffff0000ffffULL;
    v = (v | (v << 8)) & 0x00ff00ff00ff00ffULL;
    v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0fULL;
    v = (v | (v << 2)) & 0x3333333333333333ULL;
    v = (v | (v << 1)) & 0x5555555555555555ULL;
    return v;
}

__device__ __forceinline__ unsigned long long morton_d(long long x, long long y)
{
    return spread_bits_d((unsigned long long)x) | (spread_bits_d((unsigned long long)y) << 1);
}

struct KeyD {
    int tree;
    long long x, y;
};

__device__ bool shifted_d(const ForestDev &F, int tree, int level, long long x, long long y, int dx, int dy,
                          KeyD &out)
{
    const long long L = qlen_d(level);
    long long nxq = x + dx * L, nyq = y + dy * L;
    int tx = F.tree_tx[tree], ty = F.tree_ty[tree];
    if (nxq < 0) { nxq += kRootLenG; tx -= 1; }
    if (nxq >= kRootLenG) { nxq -= kRootLenG; tx += 1; }
    if (nyq < 0) { nyq += kRootLenG; ty -= 1; }
    if (nyq >= kRootLenG) { nyq -= kRootLenG; ty += 1; }
    if (tx < 0 || tx >= F.nx) {
        if (!F.px) return false;
        tx = (tx + F.nx) % F.nx;
    }
    if (ty < 0 || ty >= F.ny) {
        if (!F.py) return false;
        ty = (ty + F.ny) % F.ny;
    }
    out.tree = F.tree_at[ty * F.nx + tx];
    out.x = nxq;
    out.y = nyq;
    return true;
}

// last leaf of the tree whose corner precedes (x,y) on the Morton curve.
// With the cell table: the leaves of a level-kCellTabLevel cell are
// contiguous, so the search covers only the cell's leaves, and a leaf that
// covers the whole cell is the answer at once.
__device__ int locate_d(const ForestDev &F, int tree, long long x, long long y)
{
    const unsigned long long m = morton_d(x, y);
    int lo = F.tree_begin[tree], hi = F.tree_begin[tree + 1];  // upper_bound in [lo, hi)
    if (F.cell_tab) {
        constexpr int sh = kMaxLevelG - kCellTabLevel;
        const int c = int(morton_d(x >> sh, y >> sh));
        const int *tab = F.cell_tab + size_t(tree) * kCellTabCells;
        const int first = tab[c];
        if (F.leaves[first].y <= kCellTabLevel) return first;
        lo = first;
        hi = c + 1 < kCellTabCells ? tab[c + 1] : hi;
    }
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (F.keys[mid] <= m) lo = mid + 1;
        else hi = mid;
    }
    return lo - 1;
}

__device__ int find_d(const ForestDev &F, int tree, int level, long long x, long long y)
{
    const int c = locate_d(F, tree, x, y);
    if (c < 0) return -1;
    const int4 l = F.leaves[c];
    return (l.y == level && l.z == x && l.w == y) ? c : -1;
}

__global__ void keys_kernel(ForestDev F);

// One thread per (dirty leaf, check): checks 0-7 look at the eight face
// and corner neighbour regions for a leaf two or more levels coarser (that
// leaf is flagged), checks 8-11 walk the four edges leaf by leaf and 12-15
// look at the four corners for a leaf two or more levels finer (the dirty
// leaf itself is flagged). Splitting a leaf's checks over threads shortens
// each thread's chain of dependent binary searches; the flags are the same.
__device__ __forceinline__ void balance_check_leaf(const ForestDev &F, unsigned char *flags, int i, int item)
{
    {
        const int4 q = F.leaves[i];
        if (item < 8) {
            // fine side: the neighbour region across a face or a corner
            if (q.y < 2) return;
            const int d = item < 4 ? item : item + 1;  // 0..8 without the centre 4
            const int dx = d % 3 - 1, dy = d / 3 - 1;
            KeyD k;
            if (!shifted_d(F, q.x, q.y, q.z, q.w, dx, dy, k)) return;
            const int c = locate_d(F, k.tree, k.x, k.y);
            if (c >= 0 && F.leaves[c].y < q.y - 1) flags[c] = 1;
            return;
        }
        // coarse side
        if (q.y + 2 > kMaxLevelG) return;
        const long long L = qlen_d(q.y);
        const int lim = q.y + 2;
        bool fine = false;
        if (item < 12) {
            const int s = item - 8;
            // a leaf of level < lim spans at least L/2 of the edge: the walk
            // takes a few steps; the guard only bounds a malformed forest
            int guard = 0;
            for (long long tt = 0; tt < L && guard < 64; ++guard) {
                long long px = q.z, py = q.w;
                int dx = 0, dy = 0;
                if (s == 0) { py += tt; dx = -1; }
                if (s == 1) { px += L - 1; py += tt; dx = 1; }
                if (s == 2) { px += tt; dy = -1; }
                if (s == 3) { px += tt; py += L - 1; dy = 1; }
                KeyD k;
                if (!shifted_d(F, q.x, kMaxLevelG, px, py, dx, dy, k)) break;
                const int c = locate_d(F, k.tree, k.x, k.y);
                if (c < 0) break;
                const int4 cl = F.leaves[c];
                if (cl.y >= lim) {
                    fine = true;
                    break;
                }
                const long long len = qlen_d(cl.y);
                const long long adv = (s < 2) ? ((long long)cl.w + len - k.y) : ((long long)cl.z + len - k.x);
                if (adv <= 0) break;
                tt += adv;
            }
        } else {
            const int cidx = item - 12;
            const int dx = (cidx & 1) ? 1 : -1, dy = (cidx & 2) ? 1 : -1;
            KeyD k;
            const long long px = dx < 0 ? q.z : q.z + L - 1, py = dy < 0 ? q.w : q.w + L - 1;
            if (shifted_d(F, q.x, kMaxLevelG, px, py, dx, dy, k)) {
                const int c = locate_d(F, k.tree, k.x, k.y);
                if (c >= 0 && F.leaves[c].y >= lim) fine = true;
            }
        }
        if (fine) flags[i] = 1;
    }
}

__device__ __forceinline__ void balance_check_item(const ForestDev &F, const unsigned char *dirty,
                                                   unsigned char *flags, long long t)
{
    const int i = int(t >> 4);
    if (dirty[i]) balance_check_leaf(F, flags, i, int(t & 15));
}

__global__ void balance_check_kernel(ForestDev F, const unsigned char *dirty, unsigned char *flags)
{
    const long long total = 16ll * F.nq;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x)
        balance_check_item(F, dirty, flags, t);
}

// Leaves after a balance pass per leaf: 4 if flagged for refinement, else
// 1, and 0 past the last leaf (the scan's extra entry holds the total).
struct BalanceCount {
    const unsigned char *flags;
    int nq;
    __host__ __device__ int operator()(int i) const { return i < nq ? (flags[i] ? 4 : 1) : 0; }
};
using BalanceCountIt = thrust::transform_iterator<BalanceCount, thrust::counting_iterator<int>, int>;

// flagged leaves -> four z-ordered children at pos[i]..pos[i]+3 (dirty),
// others copied (clean); origin: the leaf of the pass's input it came from
__device__ __forceinline__ void balance_refine_item(int i, const int4 *in, const int *orig_in,
                                                    const unsigned char *flags, const int *pos, int4 *out,
                                                    int *orig_out, unsigned char *dirty_out)
{
    const int4 p = in[i];
    const int o = orig_in[i];
    const int at = pos[i];
    if (flags[i]) {
        const int h = int(qlen_d(p.y + 1));
        for (int c = 0; c < 4; ++c) {
            out[at + c] = make_int4(p.x, p.y + 1, p.z + (c & 1) * h, p.w + ((c >> 1) & 1) * h);
            orig_out[at + c] = o;
            dirty_out[at + c] = 1;
        }
    } else {
        out[at] = p;
        orig_out[at] = o;
        dirty_out[at] = 0;
    }
}

__global__ void balance_refine_kernel(int nq, const int4 *in, const int *orig_in, const unsigned char *flags,
                                      const int *pos, int4 *out, int *orig_out, unsigned char *dirty_out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x)
        balance_refine_item(i, in, orig_in, flags, pos, out, orig_out, dirty_out);
}

// Remap table of the balanced leaves: leaf k descends from pre-balance leaf
// orig[k] and inherits its kind / source.
__global__ void remap_gather_kernel(int n, const int *orig, const int *kind0, const int *src0, int *kind, int *src)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int o = orig[k];
        kind[k] = kind0[o];
        src[k] = src0[o];
    }
}

__global__ void keys_kernel(ForestDev F)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F.nq; i += gridDim.x * blockDim.x) {
        const int4 l = F.leaves[i];
        F.keys[i] = morton_d(l.z, l.w);
    }
}

// Start of a balance pass in one launch: each leaf's Morton key, a cleared
// refine flag and the first leaf of each tree (tb[t] = first leaf of tree t
// or of a later tree when t has none; tb[ntrees] = nq).
__device__ __forceinline__ void pass_prep_item(const ForestDev &F, int ntrees, int *tb, unsigned char *flags, int i)
{
    const int nq = F.nq;
    if (i == nq) {
        const int last = nq == 0 ? -1 : F.leaves[nq - 1].x;
        for (int u = last + 1; u <= ntrees; ++u) tb[u] = nq;
    } else {
        const int4 l = F.leaves[i];
        F.keys[i] = morton_d(l.z, l.w);
        flags[i] = 0;
        const int prev = i == 0 ? -1 : F.leaves[i - 1].x;
        for (int u = prev + 1; u <= l.x; ++u) tb[u] = i;  // trees without leaves start here too
        if (F.cell_tab) {
            // a leaf at or above the table's level is the first leaf of every
            // cell it covers (a Morton-contiguous run); a finer one is the
            // first of its cell when it holds the cell's lower corner
            constexpr int sh = kMaxLevelG - kCellTabLevel;
            int *tab = F.cell_tab + size_t(l.x) * kCellTabCells;
            const int c0 = int(morton_d(l.z >> sh, l.w >> sh));
            if (l.y <= kCellTabLevel) {
                const int run = 1 << (2 * (kCellTabLevel - l.y));
                for (int k = 0; k < run; ++k) tab[c0 + k] = i;
            } else if (((l.z | l.w) & ((1 << sh) - 1)) == 0) {
                tab[c0] = i;
            }
        }
    }
}

__global__ void pass_prep_kernel(ForestDev F, int ntrees, int *tb, unsigned char *flags)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= F.nq; i += gridDim.x * blockDim.x)
        pass_prep_item(F, ntrees, tb, flags, i);
}

// One thread per (leaf, side): the side descriptor (rank filled later), the
// emits flag and the emitter slot; the leaf's corners from side 0's thread.
__device__ __forceinline__ void sides_item(const ForestDev &F, QuadDesc *out, int *emits, int *emitter, int *status,
                                           int t)
{
    {
        const int i = t >> 2, s = t & 3;
        const int4 q = F.leaves[i];  // tree, level, x, y
        const int dx = s == 0 ? -1 : (s == 1 ? 1 : 0);
        const int dy = s == 2 ? -1 : (s == 3 ? 1 : 0);
        const int opp = s ^ 1;
        SideDesc d;
        d.kind = kSideNone;
        d.nbr0 = -1;
        d.nbr1 = -1;
        d.rank = -1;
        d.level = q.y;
        d.bc = 0;
        int emit = 0, em = t;
        KeyD k;
        if (!shifted_d(F, q.x, q.y, q.z, q.w, dx, dy, k)) {
            d.kind = kSideBoundary;
            d.bc = F.bc[s];
            emit = 1;
        } else {
            const int c0 = locate_d(F, k.tree, k.x, k.y);
            const int lvl0 = c0 >= 0 ? F.leaves[c0].y : -1;
            if (c0 < 0 || lvl0 < q.y - 1) {
                atomicOr(status, 1);  // neighbour two or more levels coarser
            } else if (lvl0 == q.y) {
                const int j = c0;
                d.kind = kSideFull;
                d.nbr0 = j;
                emit = (i < j) || (i == j && (s & 1) == 0);
                em = (i < j) ? t : (i > j ? 4 * j + opp : 4 * i + (s & ~1));
            } else if (lvl0 == q.y - 1) {
                // this leaf is one of the two fine leaves of a hanging face
                const int c = c0;
                const long long Lp = qlen_d(q.y - 1), L = qlen_d(q.y);
                const long long bx = ((long long)q.z / Lp) * Lp, by = ((long long)q.w / Lp) * Lp;
                int fine[2];
                for (int h = 0; h < 2; ++h)
                    fine[h] = (s < 2) ? find_d(F, q.x, q.y, q.z, by + h * L) : find_d(F, q.x, q.y, bx + h * L, q.w);
                if (fine[0] < 0 || fine[1] < 0) {
                    atomicOr(status, 2);
                } else {
                    d.kind = kSideFineHang;
                    d.nbr0 = c;
                    const int mf = min(fine[0], fine[1]);
                    const int mn = min(c, mf);
                    emit = (i == mn);
                    em = (mn == c) ? 4 * c + opp : 4 * mn + s;
                }
            } else {
                // this leaf is the coarse side: two finer neighbours
                const long long Lc = qlen_d(q.y + 1);
                int fine[2];
                for (int h = 0; h < 2; ++h) {
                    if (s < 2) fine[h] = find_d(F, k.tree, q.y + 1, (s == 0) ? k.x + Lc : k.x, k.y + h * Lc);
                    else fine[h] = find_d(F, k.tree, q.y + 1, k.x + h * Lc, (s == 2) ? k.y + Lc : k.y);
                }
                if (fine[0] < 0 || fine[1] < 0) {
                    atomicOr(status, 2);
                } else {
                    d.kind = kSideCoarseHang;
                    d.nbr0 = fine[0];
                    d.nbr1 = fine[1];
                    d.level = q.y + 1;
                    const int mf = min(fine[0], fine[1]);
                    emit = i < mf;
                    em = emit ? t : 4 * mf + opp;
                }
            }
        }
        out[i].side[s] = d;
        emits[t] = emit;
        emitter[t] = em;
        if (s == 0) {
            // forest_quad_corners: bilinear map of the tree's brick square
            const double intsize = 1.0 / double(kRootLenG);
            const double h2 = __dmul_rn(__dmul_rn(0.5, intsize), double(qlen_d(q.y)));
            const int tx = F.tree_tx[q.x], ty = F.tree_ty[q.x];
            double v[4][2];
            for (int c = 0; c < 4; ++c) {
                const int vx = tx + (c & 1), vy = ty + ((c >> 1) & 1);
                v[c][0] = __dadd_rn(__dmul_rn(double(vx), F.scale), F.xlo[0]);
                v[c][1] = __dadd_rn(__dmul_rn(double(vy), F.scale), F.xlo[1]);
            }
            const double one_z = __dsub_rn(1.0, 0.0);  // (1 - eta_z), eta_z = 0
            int kk = 0;
            for (int yi = 0; yi < 2; ++yi) {
                const double ey = __dadd_rn(__dmul_rn(intsize, double(q.w)), __dmul_rn(h2, 1.0 + (2 * yi - 1)));
                for (int xi = 0; xi < 2; ++xi) {
                    const double ex = __dadd_rn(__dmul_rn(intsize, double(q.z)), __dmul_rn(h2, 1.0 + (2 * xi - 1)));
                    for (int j = 0; j < 2; ++j) {
                        const double lo_ = __dadd_rn(__dmul_rn(__dsub_rn(1.0, ex), v[0][j]), __dmul_rn(ex, v[1][j]));
                        const double hi_ = __dadd_rn(__dmul_rn(__dsub_rn(1.0, ex), v[2][j]), __dmul_rn(ex, v[3][j]));
                        out[i].corner[2 * kk + j] =
                            __dmul_rn(one_z, __dadd_rn(__dmul_rn(__dsub_rn(1.0, ey), lo_), __dmul_rn(ey, hi_)));
                    }
                    ++kk;
                }
            }
        }
    }
}

__global__ void sides_kernel(ForestDev F, QuadDesc *out, int *emits, int *emitter, int *status)
{
    const int total = 4 * F.nq;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x)
        sides_item(F, out, emits, emitter, status, t);
}

__global__ void rank_kernel(int nq, QuadDesc *out, const int *emits, const int *scan, const int *emitter,
                            int *status)
{
    const int total = 4 * nq;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        out[t >> 2].side[t & 3].rank = scan[emitter[t]];
        if (t == total - 1) status[1] = scan[t] + emits[t];
    }
}

// ---------------------------------------------------------------- the
// balance loop and the descriptor build in one cooperative launch.
//
// Every phase of every pass runs as a grid-stride loop over all blocks,
// separated by device-wide barriers, so a whole 2:1 balance (until a pass
// finds nothing to refine), the quad descriptors of the balanced leaves and
// their remap table cost one launch and one read-back instead of a few
// launches and a read-back per pass. The phases are the kernels above, item
// for item, so the leaves, descriptors and tables are the same.

// Device-wide barrier of a cooperative launch: the last block to arrive
// resets the count and advances the generation; the others wait for the
// generation to move, at most kBarrierSpins polls. A wait that runs out
// sets `abort` and every block leaves at its next barrier, so a fault in the
// loop's logic ends the kernel with an error instead of hanging it.
constexpr long long kBarrierSpins = 1ll << 22;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ bool grid_barrier(BalanceCtl *ctl)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned gen = ld_acquire_u32(&ctl->bar_gen);
        __threadfence();
        const unsigned arrived = atomicAdd(&ctl->bar_count, 1u) + 1u;
        int ok = 1;
        if (arrived == gridDim.x) {
            atomicExch(&ctl->bar_count, 0u);
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            long long spins = 0;
            while (ld_acquire_u32(&ctl->bar_gen) == gen) {
                if (++spins > kBarrierSpins) {
                    ok = 0;
                    atomicExch(&ctl->abort, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok && *(volatile int *)&ctl->abort == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

// Exclusive scan of cnt(0..n-1) into pos[0..n-1] and the total into pos[n],
// over all blocks: each block takes a contiguous chunk, each thread a
// contiguous run of it; block sums go through bsum and a barrier. Returns
// false when a barrier gave up.
template <typename Cnt>
__device__ bool grid_scan(int n, Cnt cnt, int *pos, int *bsum, BalanceCtl *ctl)
{
    __shared__ int s_warp[32];
    __shared__ int s_off, s_tot;
    const int T = blockDim.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = T >> 5;
    const int chunk = (n + gridDim.x - 1) / gridDim.x;
    const int lo = min(n, (int)blockIdx.x * chunk), hi = min(n, lo + chunk);
    const int per = (chunk + T - 1) / T;
    const int tlo = min(hi, lo + (int)threadIdx.x * per), thi = min(hi, tlo + per);
    int sum = 0;
    for (int i = tlo; i < thi; ++i) sum += cnt(i);
    int incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    if (w == 0) {
        int v = lane < nw ? s_warp[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d) v += u;
        }
        if (lane < nw) s_warp[lane] = v;  // inclusive warp prefixes
    }
    __syncthreads();
    const int texcl = incl - sum + (w > 0 ? s_warp[w - 1] : 0);
    if (threadIdx.x == 0) bsum[blockIdx.x] = s_warp[nw - 1];
    if (!grid_barrier(ctl)) return false;
    // this block's offset and the total, from every block's sum
    int off = 0, tot = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += T) {
        const int v = __ldcg(bsum + b);
        tot += v;
        if (b < (int)blockIdx.x) off += v;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        off += __shfl_xor_sync(0xffffffffu, off, d);
        tot += __shfl_xor_sync(0xffffffffu, tot, d);
    }
    if (threadIdx.x == 0) s_off = s_tot = 0;
    __syncthreads();
    if (lane == 0) {
        atomicAdd(&s_off, off);
        atomicAdd(&s_tot, tot);
    }
    __syncthreads();
    int run = s_off + texcl;
    for (int i = tlo; i < thi; ++i) {
        pos[i] = run;
        run += cnt(i);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) pos[n] = s_tot;
    return grid_barrier(ctl);
}

// The adapt phase's decisions for one leaf, those of forest_adapt
// (forest.cpp): a leaf refines when tagged refine_value below max_level; a
// complete family of four siblings (consecutive in Morton order, same tree
// and level, none refining, all tagged coarsen_value above min_level)
// becomes its parent, written where its first child was. Family starts
// never overlap (the second to fourth children are not aligned to a parent
// of their level), so each leaf decides on its own.
__device__ __forceinline__ bool adapt_refines(const AdaptArgs &ad, const int4 q, int tag)
{
    return tag == ad.refine_value && q.y < ad.max_level && q.y < kMaxLevelG;
}

__device__ __forceinline__ bool adapt_coarsens(const AdaptArgs &ad, const int4 q, int tag)
{
    return tag == ad.coarsen_value && q.y > ad.min_level;
}

__device__ bool adapt_family_start(const AdaptArgs &ad, const int4 *in, int n, int i)
{
    const int4 p = in[i];
    if (!(p.y > 0 && p.y > ad.min_level && i + 3 < n)) return false;
    const long long P = qlen_d(p.y - 1), h = qlen_d(p.y);
    const long long px = (p.z / P) * P, py = (p.w / P) * P;
    if (p.z != px || p.w != py) return false;
    for (int c = 0; c < 4; ++c) {
        const int4 b = in[i + c];
        const int t = ad.tags[i + c];
        if (b.x != p.x || b.y != p.y || b.z != px + (c & 1) * h || b.w != py + ((c >> 1) & 1) * h ||
            adapt_refines(ad, b, t) || !adapt_coarsens(ad, b, t))
            return false;
    }
    return true;
}

// Leaves leaf i of the adapt becomes: 4 (refined), 0 (second to fourth
// child of a coarsened family), else 1. fs: family-start marks.
__device__ __forceinline__ int adapt_count(const AdaptArgs &ad, const int4 *in, const unsigned char *fs, int i)
{
    if (adapt_refines(ad, in[i], ad.tags[i])) return 4;
    const bool member = (i >= 1 && __ldcg(fs + i - 1)) || (i >= 2 && __ldcg(fs + i - 2)) ||
                        (i >= 3 && __ldcg(fs + i - 3));
    return member ? 0 : 1;
}

// Writes leaf i's output leaves at pos[i] (the exclusive scan of the
// counts): children of a refined leaf (new, source = the leaf), a family's
// parent (new, the mean of the family), or the leaf itself (source = the
// leaf). Origins are the identity: the balance then refers back to these.
__device__ __forceinline__ void adapt_write_item(const AdaptArgs &ad, const int4 *in, const unsigned char *fs,
                                                 const int *pos, int4 *out, int *orig_out,
                                                 unsigned char *dirty_out, int i)
{
    const int4 q = in[i];
    const int at = __ldcg(pos + i);
    if (adapt_refines(ad, q, ad.tags[i])) {
        const int h = int(qlen_d(q.y + 1));
        for (int c = 0; c < 4; ++c) {
            out[at + c] = make_int4(q.x, q.y + 1, q.z + (c & 1) * h, q.w + ((c >> 1) & 1) * h);
            orig_out[at + c] = at + c;
            dirty_out[at + c] = 1;
            ad.kind[at + c] = 0;  // injection from the parent
            ad.src[at + c] = i;
        }
        return;
    }
    if (__ldcg(pos + i + 1) == at) return;  // absorbed into a family's parent
    if (__ldcg(fs + i)) {
        out[at] = make_int4(q.x, q.y - 1, q.z, q.w);  // the first child's corner is the parent's
        dirty_out[at] = 1;
        ad.kind[at] = 1;  // mean of the four children
    } else {
        out[at] = q;
        dirty_out[at] = 0;
        ad.kind[at] = 0;
    }
    orig_out[at] = at;
    ad.src[at] = i;
}

__global__ void __launch_bounds__(256) balance_loop_kernel(const BalanceLoopArgs a)
{
    BalanceCtl *ctl = a.ctl;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    int nl = a.nl, live = a.live, passes = 0;
    bool ok = true, done = false, overflow = false, refined = false;
    ForestDev F = a.F;
    int adapted = 0, adapt_total = 0;
    if (a.adapt) {
        // refine / coarsen by tags from buffer `live` into the other buffer
        const int4 *in = a.leaves[live];
        unsigned char *fs = a.flags;
        for (int i = gtid; i < nl; i += gstride) fs[i] = adapt_family_start(a.ad, in, nl, i) ? 1 : 0;
        ok = grid_barrier(ctl);
        if (ok) ok = grid_scan(nl, [&](int i) { return adapt_count(a.ad, in, fs, i); }, a.pos, a.bsum, ctl);
        if (ok) {
            adapt_total = __ldcg(a.pos + nl);
            if (adapt_total > a.cap) {
                overflow = true;
            } else {
                for (int i = gtid; i < nl; i += gstride)
                    adapt_write_item(a.ad, in, fs, a.pos, a.leaves[1 - live], a.orig[1 - live], a.dirty[1 - live],
                                     i);
                ok = grid_barrier(ctl);
                live = 1 - live;
                nl = adapt_total;
                adapted = adapt_total;
            }
        }
    }
    int ndirty = -1;  // -1: check every leaf marked dirty (the first pass)
    for (int pass = 0; pass < 64 && ok && !overflow; ++pass) {
        ++passes;
        F.leaves = a.leaves[live];
        F.nq = nl;
        unsigned char *flags = a.flags;
        for (int i = gtid; i <= nl; i += gstride) pass_prep_item(F, a.ntrees, a.tree_begin, flags, i);
        if (!(ok = grid_barrier(ctl))) break;
        if (ndirty >= 0) {
            // the leaves the previous pass created, listed by its refinement
            for (int t = gtid; t < 16 * ndirty; t += gstride)
                balance_check_leaf(F, flags, __ldcg(a.dirty_list + (t >> 4)), t & 15);
        } else {
            for (long long t = gtid; t < 16ll * nl; t += gstride) balance_check_item(F, a.dirty[live], flags, t);
        }
        if (!(ok = grid_barrier(ctl))) break;
        if (!(ok = grid_scan(nl, [&](int i) { return __ldcg(flags + i) ? 4 : 1; }, a.pos, a.bsum, ctl))) break;
        const int total = __ldcg(a.pos + nl);
        if (total == nl) {
            done = true;
            break;
        }
        if (total > a.cap) {
            overflow = true;
            break;
        }
        for (int i = gtid; i < nl; i += gstride) {
            balance_refine_item(i, a.leaves[live], a.orig[live], flags, a.pos, a.leaves[1 - live], a.orig[1 - live],
                                a.dirty[1 - live]);
            if (__ldcg(flags + i)) {
                // leaves flagged before i: (pos[i] - i) / 3; their children
                // come first in the list
                const int at = __ldcg(a.pos + i), k = 4 * ((at - i) / 3);
                for (int c = 0; c < 4; ++c) a.dirty_list[k + c] = at + c;
            }
        }
        if (!(ok = grid_barrier(ctl))) break;
        ndirty = 4 * ((total - nl) / 3);
        live = 1 - live;
        nl = total;
        refined = true;
    }
    // the balanced leaves' remap table and descriptors (keys and tree starts
    // are the last pass's, which refined nothing)
    if (ok && done && a.build) {
        if (a.ad.kind) {
            for (int k = gtid; k < nl; k += gstride) {
                const int o = __ldcg(a.orig[live] + k);
                a.kind[k] = __ldcg(a.ad.kind + o);
                a.src[k] = __ldcg(a.ad.src + o);
            }
        } else if (a.kind0) {
            for (int k = gtid; k < nl; k += gstride) {
                const int o = a.orig[live][k];
                a.kind[k] = a.kind0[o];
                a.src[k] = a.src0[o];
            }
        }
        for (int t = gtid; t < 4 * nl; t += gstride) sides_item(F, a.out, a.emits, a.emitter, a.status, t);
        ok = grid_barrier(ctl);
        if (ok) ok = grid_scan(4 * nl, [&](int t) { return __ldcg(a.emits + t); }, a.scan, a.bsum, ctl);
        if (ok) {
            for (int t = gtid; t < 4 * nl; t += gstride) a.out[t >> 2].side[t & 3].rank = __ldcg(a.scan + a.emitter[t]);
            if (gtid == 0) a.status[1] = nl > 0 ? __ldcg(a.scan + 4 * nl) : 0;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->nl = nl;
        ctl->live = live;
        ctl->passes = passes;
        ctl->result = !ok ? kBalanceTimeout : overflow ? kBalanceOverflow : done ? kBalanceDone : kBalanceNoConverge;
        ctl->refined = refined ? 1 : 0;
        ctl->adapted = adapted;
        ctl->adapt_total = adapt_total;
    }
}

int grid_for(long long n, int sms)
{
    long long g = (n + 255) / 256;
    const long long cap = (long long)sms * 16;
    return int(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

size_t balance_scan_bytes(int nq)
{
    size_t bytes = 0;
    const BalanceCountIt it(thrust::counting_iterator<int>(0), BalanceCount{nullptr, 0});
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, it, (int *)nullptr, (nq > 0 ? nq : 1) + 1);
    return bytes;
}

cudaError_t launch_balance_pass(const ForestDev &F, int ntrees, int *tree_begin, const unsigned char *dirty,
                                unsigned char *flags, int *pos, void *scan_tmp, size_t scan_bytes, int sms,
                                cudaStream_t st)
{
    if (F.nq <= 0) return cudaSuccess;
    pass_prep_kernel<<<grid_for(F.nq + 1ll, sms), 256, 0, st>>>(F, ntrees, tree_begin, flags);
    balance_check_kernel<<<grid_for(16ll * F.nq, sms), 256, 0, st>>>(F, dirty, flags);
    size_t bytes = scan_bytes;
    const BalanceCountIt it(thrust::counting_iterator<int>(0), BalanceCount{flags, F.nq});
    cudaError_t e = cub::DeviceScan::ExclusiveSum(scan_tmp, bytes, it, pos, F.nq + 1, st);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_remap_gather(int n, const int *orig, const int *kind0, const int *src0, int *kind, int *src,
                                int sms, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    remap_gather_kernel<<<grid_for(n, sms), 256, 0, st>>>(n, orig, kind0, src0, kind, src);
    return cudaGetLastError();
}

cudaError_t launch_balance_refine(int nq, const int4 *in, const int *orig_in, const unsigned char *flags,
                                  const int *pos, int4 *out, int *orig_out, unsigned char *dirty_out, int sms,
                                  cudaStream_t st)
{
    if (nq <= 0) return cudaSuccess;
    balance_refine_kernel<<<grid_for(nq, sms), 256, 0, st>>>(nq, in, orig_in, flags, pos, out, orig_out, dirty_out);
    return cudaGetLastError();
}

size_t build_quads_scan_bytes(int nq)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int *)nullptr, (int *)nullptr, 4 * (nq > 0 ? nq : 1));
    return bytes;
}

cudaError_t launch_build_quads(const ForestDev &F, QuadDesc *out, int *emits, int *scan, int *emitter,
                               void *scan_tmp, size_t scan_bytes, int *status, int sms, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(status, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess || F.nq <= 0) return e;
    keys_kernel<<<grid_for(F.nq, sms), 256, 0, st>>>(F);
    sides_kernel<<<grid_for(4ll * F.nq, sms), 256, 0, st>>>(F, out, emits, emitter, status);
    size_t bytes = scan_bytes;
    e = cub::DeviceScan::ExclusiveSum(scan_tmp, bytes, emits, scan, 4 * F.nq, st);
    if (e != cudaSuccess) return e;
    rank_kernel<<<grid_for(4ll * F.nq, sms), 256, 0, st>>>(F.nq, out, emits, scan, emitter, status);
    return cudaGetLastError();
}


cudaError_t launch_balance_loop(const BalanceLoopArgs &a, int sms, cudaStream_t st)
{
    // one block per SM at most (a cooperative launch needs every block
    // resident), fewer for small forests: about 8 of the 16 checks per leaf
    // per thread, since every block takes part in every barrier
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, balance_loop_kernel, 256, 0);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorLaunchOutOfResources;
    const long long want = (16ll * std::max(a.nl, 1) + 8 * 256 - 1) / (8 * 256);
    const int grid = int(std::max(1ll, std::min<long long>(want, (long long)sms)));
    BalanceLoopArgs args = a;
    void *p[] = {&args};
    e = cudaMemsetAsync(a.ctl, 0, sizeof(BalanceCtl), st);
    if (e == cudaSuccess && a.stall_test) e = cudaMemsetAsync(&a.ctl->bar_count, 0x40, sizeof(unsigned), st);
    if (e == cudaSuccess && a.build) e = cudaMemsetAsync(a.status, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel((const void *)balance_loop_kernel, dim3(grid), dim3(256), p, 0, st);
}

size_t balance_loop_bsum_ints(int sms) { return size_t(std::max(sms, 1)); }

}  // namespace amrgpu
