// mesh_gpu.h -- host launcher of mesh_gpu.cu (quad descriptors of a forest
// built on the GPU).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace amrgpu {

struct QuadDesc;

// Device view of a forest's leaves and brick.
// Point location over a tree's leaves starts in a table of the tree's
// level-kCellTabLevel cells (Morton order): the first leaf in each cell.
constexpr int kCellTabLevel = 7;
constexpr int kCellTabCells = 1 << (2 * kCellTabLevel);
constexpr int kCellTabMaxTrees = 256;  // larger bricks search whole trees

struct ForestDev {
    const int4 *leaves;        // (tree, level, x, y) per leaf, Morton order within trees
    unsigned long long *keys;  // Morton key per leaf (written by the build)
    const int *tree_begin;     // first leaf of each tree, ntrees + 1 entries
    const int *tree_tx, *tree_ty, *tree_at;
    int nx, ny, px, py;
    double xlo[3];
    double scale;
    int bc[4];
    int nq;
    // null, or kCellTabCells entries per tree: the first leaf of each
    // level-kCellTabLevel cell (the one-launch balance fills it every pass)
    int *cell_tab = nullptr;
};

// One 2:1 balance pass over F's leaves in three launches (F.keys written,
// F.tree_begin rebuilt into tree_begin, flags cleared; the checks; the
// scan): flags[i] = 1 for leaves to refine, pos (nq + 1 entries) the
// exclusive scan of the 4-or-1 counts, so pos[nq] is the new leaf count.
size_t balance_scan_bytes(int nq);
cudaError_t launch_balance_pass(const ForestDev &F, int ntrees, int *tree_begin, const unsigned char *dirty,
                                unsigned char *flags, int *pos, void *scan_tmp, size_t scan_bytes, int sms,
                                cudaStream_t st);
// kind[k] = kind0[orig[k]], src[k] = src0[orig[k]] for k < n: the remap
// table of balanced leaves from that of the leaves they descend from.
cudaError_t launch_remap_gather(int n, const int *orig, const int *kind0, const int *src0, int *kind, int *src,
                                int sms, cudaStream_t st);
// The pass's refinement: out / orig_out / dirty_out at the scanned positions.
cudaError_t launch_balance_refine(int nq, const int4 *in, const int *orig_in, const unsigned char *flags,
                                  const int *pos, int4 *out, int *orig_out, unsigned char *dirty_out, int sms,
                                  cudaStream_t st);

// The whole 2:1 balance (passes until one refines nothing), then the quad
// descriptors of the balanced leaves and their remap table, in one
// cooperative launch (device-wide barriers between the phases, each wait
// bounded). Leaf buffers are double-buffered: the loop starts from
// buffer `live` with nl leaves and ends with ctl->live / ctl->nl.
enum { kBalanceDone = 1, kBalanceOverflow = 2, kBalanceNoConverge = 3, kBalanceTimeout = 4 };
struct BalanceCtl {
    unsigned bar_count, bar_gen;  // the barrier
    int abort;                    // set by a barrier wait that ran out
    int nl, live, passes, refined;
    int result;                   // kBalance*
    int adapted;                  // leaves after the adapt phase (0: no adapt ran or it overflowed)
    int adapt_total;              // leaves the adapt phase needs (also on overflow)
};
// Refine / coarsen of the loop's starting leaves by per-leaf tags, before
// the balance: the host forest's forest_adapt, leaf for leaf (forest.cpp).
struct AdaptArgs {
    const int *tags;              // one per starting leaf
    int refine_value, coarsen_value, min_level, max_level;
    int *kind, *src;              // remap table of the adapted leaves
};
struct BalanceLoopArgs {
    ForestDev F;                  // brick and tree tables; leaves / nq set per pass, keys written
    int ntrees;
    int *tree_begin;              // ntrees + 1 entries, rebuilt every pass
    int4 *leaves[2];
    int *orig[2];
    unsigned char *dirty[2];
    int nl, live, cap;            // leaves at the start, their buffer, each buffer's capacity
    unsigned char *flags;         // cap
    int *pos;                     // cap + 1
    int *dirty_list;              // cap: the leaves a pass created, for the next pass's checks
    int *bsum;                    // one per block (balance_loop_bsum_ints)
    BalanceCtl *ctl;
    int build;                    // then the descriptors of the balanced leaves:
    QuadDesc *out;                //   cap descriptors
    int *emits, *scan, *emitter;  //   4 cap (+1 for scan) ints each
    int *status;                  //   [0] 2:1 violation bits, [1] face count
    const int *kind0, *src0;      //   remap table of the leaves the loop started from (or null)
    int *kind, *src;              //   ... gathered for the balanced leaves
    int stall_test;               // nonzero: the barrier's arrival count starts out of reach, so
                                  // every wait runs out (tests of the bounded wait)
    int adapt;                    // nonzero: adapt the starting leaves first (ad)
    AdaptArgs ad;                 // ad.kind non-null: the balanced leaves' remap table comes from
                                  //   ad.kind / ad.src (an adapt of this or an earlier launch)
};
cudaError_t launch_balance_loop(const BalanceLoopArgs &a, int sms, cudaStream_t st);
size_t balance_loop_bsum_ints(int sms);

// Scratch of the face-numbering scan for nq leaves.
size_t build_quads_scan_bytes(int nq);

// out[0..nq): descriptors; emits / scan / emitter: 4*nq ints each;
// status (device, 2 ints): [0] 2:1 violation bits, [1] face count.
cudaError_t launch_build_quads(const ForestDev &F, QuadDesc *out, int *emits, int *scan, int *emitter,
                               void *scan_tmp, size_t scan_bytes, int *status, int sms, cudaStream_t st);

}  // namespace amrgpu
