// mesh_gpu.h -- host launcher of mesh_gpu.cu (quad descriptors of a forest
// built on the GPU).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace amrgpu {

struct QuadDesc;

// Device view of a forest's leaves and brick.
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

// Scratch of the face-numbering scan for nq leaves.
size_t build_quads_scan_bytes(int nq);

// out[0..nq): descriptors; emits / scan / emitter: 4*nq ints each;
// status (device, 2 ints): [0] 2:1 violation bits, [1] face count.
cudaError_t launch_build_quads(const ForestDev &F, QuadDesc *out, int *emits, int *scan, int *emitter,
                               void *scan_tmp, size_t scan_bytes, int *status, int sms, cudaStream_t st);

}  // namespace amrgpu
