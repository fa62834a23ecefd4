// device_common.cuh -- device-side data layout shared by all kernels.
//
// State in HBM is structure-of-arrays: field f of cell c of quad q lives at
// Q[f][q*n*n + j*n + i] (i fastest), so a quad's patch is four contiguous
// n*n slabs of doubles. Per quad the kernels read a 128-byte QuadDesc with
// its four sides' neighbour descriptions and its corner coordinates.
#pragma once

#include <cstdint>

namespace amrgpu {

enum SideKind : int {
    kSideNone = 0,
    kSideBoundary = 1,   // physical boundary: bc flux on this quad only
    kSideFull = 2,       // conforming neighbour nbr0
    kSideCoarseHang = 3, // this quad is coarse; fine neighbours nbr0, nbr1
    kSideFineHang = 4    // this quad is one of two fine quads; coarse nbr0
};

struct SideDesc {
    int kind;
    int nbr0;
    int nbr1;
    int rank;   // position of the face in face_info: order of accumulation
    int level;  // level whose cell_h sizes the face normal
    int bc;     // boundary condition type for kSideBoundary
};

struct QuadDesc {
    SideDesc side[4];   // 96 bytes
    double corner[8];   // x,y of n1(-,-) n2(+,-) n3(-,+) n4(+,+): 64 bytes
};
static_assert(sizeof(QuadDesc) == 160, "QuadDesc layout");

// Mixed patch sizes (8x8 and 16x16 quads in one mesh; extension): per quad
// its patch size n, the offset of its first cell in the state arrays
// (cells, not doubles: cell_info[2] / 4) and its level, and per side the
// neighbour's patch size, the cell offsets of nbr0 / nbr1, and for a
// kSideFineHang side which half of the coarse edge this quad covers (0: the
// half at the coarse edge's lower coordinate). Read only by the mixed-size
// kernels; uniform meshes keep QuadDesc alone.
struct MixSide {
    int n;
    int base0;
    int base1;
    int half;
};

struct MixDesc {
    int n;
    int base;
    int level;
    int pad;
    MixSide side[4];
};
static_assert(sizeof(MixDesc) == 80, "MixDesc layout");

// Per-step scalars kept on the device, cycled over three slots so that a
// step reads slot s%3, writes its successor's dt candidates into (s+1)%3 and
// re-arms (s+2)%3 without racing concurrently running blocks.
struct StepSlot {
    unsigned long long dt_bits;  // min over cells of the CFL step, as uint64 image
    double time;                 // simulated time at the start of the step
};

struct DeviceScalars {
    StepSlot slot[3];
    double norm_sq;           // sum of k^2 of the last stage of the last step
    double dt_used;           // step size of the last step
    unsigned int done_blocks; // last-block-done counter (norm reduction, work counter reset)
    int flags;                // bit 0: non-finite residual, bit 1: rho<=0 or p<=0
    int steps;                // steps taken with a positive step size
    unsigned int work_next;   // dynamic quad counter of the row-sweep kernel (reset by its last block)
};

enum { kFlagNonFinite = 1, kFlagNegative = 2, kFlagTimeout = 4 };

// Programmatic dependent launch between the stage kernels of a stream. A
// stage kernel is launched with programmatic stream serialisation, so the
// hardware may schedule its blocks into the SM slots that the previous
// stage's finished blocks free, before that grid has ended. Every stage
// kernel therefore begins with stage_launch_gate(): it lets the next stage
// be scheduled (launch_dependents: that kernel waits in turn), then waits
// until the previous grid has completed and its writes are visible (wait)
// before any load or store. Launched without the attribute, or after work
// that is not a stage kernel, both instructions return at once.
__device__ __forceinline__ void stage_launch_gate()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

}  // namespace amrgpu
