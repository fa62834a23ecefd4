// session.cu -- host driver of the GPU time-step path.
//
// A session owns the device copy of one mesh epoch (quad descriptors built
// from cell_info / face_info / geom), the SoA state buffers, the per-step
// device scalars, the chosen stage-kernel variant and the CUDA graphs of
// whole steps. hpc_amr_evolve_solver / physics_go_gpu keep one session
// alive across calls and rebuild it when the mesh changes.
//
// The step loop replaces physics_runge_kutta_interface.c:23-357: the number
// of steps of a segment is known on the host from istep and the interval
// flags, dt never leaves the device (each step's last stage folds the next
// step's CFL minimum), and the host synchronises once per segment to read
// the residual norm and the error flags.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "amrgpu_internal.h"
#include "device_common.cuh"
#include "launch_table.h"
#include "halo_kernels.h"
#include "mesh_gpu.h"
#include "misc_kernels.h"
#include "stage_kernel.cuh"

using namespace amrgpu;

namespace {

enum { RX = 0, RY = 1, RZ = 2, RK = 3 };

struct StagePlan {
    int in, a0, a1, out0, out1;
};

// Buffer roles of each stage, per scheme, over three state buffers X, Y, Z
// and one auxiliary K. A stage reads halos only from `in`; a0/a1 are read and
// out0/out1 written for the thread's own cells only, so in-place roles are
// race-free.
const std::vector<StagePlan> &plan_of(int scheme, bool &swap_xy)
{
    static const std::vector<StagePlan> rk1 = {{RX, -1, -1, RY, -1}};
    static const std::vector<StagePlan> rk2 = {{RX, -1, -1, RY, RK}, {RY, RK, -1, RX, -1}};
    static const std::vector<StagePlan> rk3 = {{RX, -1, -1, RY, RK}, {RY, RX, RK, RX, RK}, {RX, RK, -1, RY, -1}};
    static const std::vector<StagePlan> rk4 = {
        {RX, -1, -1, RY, RK}, {RY, RX, RK, RZ, RK}, {RZ, RX, RK, RY, RK}, {RY, RX, RK, RX, -1}};
    static const std::vector<StagePlan> ls = {
        {RX, -1, -1, RY, RK}, {RY, RK, -1, RX, RK}, {RX, RK, -1, RY, RK}, {RY, RK, -1, RX, RK}, {RX, RK, -1, RY, RK}};
    static const std::vector<StagePlan> so = {{RX, -1, -1, RY, -1}, {RY, RX, -1, RZ, -1}, {RZ, RX, -1, RX, -1}};
    switch (scheme) {
    case kSchemeRK1: swap_xy = true; return rk1;
    case kSchemeRK2: swap_xy = false; return rk2;
    case kSchemeRK3: swap_xy = true; return rk3;
    case kSchemeRK4: swap_xy = false; return rk4;
    case kSchemeLSERK45: swap_xy = true; return ls;
    default: swap_xy = false; return so;
    }
}

bool cuda_ok(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return true;
    set_error(AMRGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// The device's name (cudaDeviceProp::name), looked up once per device.
std::string device_name(int dev)
{
    static std::mutex mu;
    static std::map<int, std::string> names;
    std::lock_guard<std::mutex> lk(mu);
    auto it = names.find(dev);
    if (it != names.end()) return it->second;
    cudaDeviceProp prop;
    std::string name = cudaGetDeviceProperties(&prop, dev) == cudaSuccess ? std::string(prop.name) : "unknown";
    for (char &c : name)
        if (c == '"' || c == '\\') c = '_';
    names[dev] = name;
    return name;
}

uint64_t fnv1a(const void *p, size_t bytes, uint64_t h = 1469598103934665603ULL)
{
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < bytes; ++i) {
        h ^= b[i];
        h *= 1099511628211ULL;
    }
    return h;
}

}  // namespace

struct amrgpu_session {
    PhysicsConfig cfg;
    int n = 0, nquad = 0, nghost = 0, nface = 0, dof = 0;
    long long ncells_total = 0, stride = 0;
    std::vector<QuadDesc> h_quads;
    QuadDesc *d_quads = nullptr;
    double *buf[4] = {nullptr, nullptr, nullptr, nullptr};
    int role[4] = {0, 1, 2, 3};
    double *d_aos = nullptr;
    DeviceScalars *d_scal = nullptr;
    DeviceScalars h_scal{};
    double *d_partials = nullptr;
    int partial_cap = 0;
    double *d_tot = nullptr;
    long long cap_stride = 0;  // cells per field the state buffers hold
    int cap_quads = 0;         // quads the tag and remap arrays hold
    int cap_desc = 0;          // quads d_quads holds
    QuadDesc *d_quads_alt = nullptr;  // build target of amrgpu_session_regrid_forest
    int cap_desc_alt = 0;
    PinnedRing ring;                  // pinned chunks for pageable state transfers
    void *h_stage = nullptr;          // pinned staging of a forest's leaves
    size_t h_stage_bytes = 0;
    void *d_mesh_scratch = nullptr;   // device scratch of the descriptor build
    size_t mesh_scratch_bytes = 0;
    void *d_fstage = nullptr;         // device copy of a staged forest and its keys
    size_t fstage_bytes = 0;
    void *d_bal[2] = {nullptr, nullptr};  // balance: leaves / origin / dirty, double-buffered
    void *d_bal_work = nullptr;           // balance: flags, counts, positions, keys, trees, scan temp
    void *d_remap0 = nullptr;             // balance + regrid: remap kind / source of the pre-balance leaves
    size_t remap0_bytes = 0;
    int bal_cap = 0;                      // leaves the balance buffers hold
    int bal_trees = 0;                    // trees the balance work area holds tables for
    // the forest whose leaves the balance buffers still hold (buffer
    // dev_live, nquad leaves, the session's mesh), at version
    // dev_forest_version: a regrid of that unchanged forest adapts them on
    // the device instead of staging the host's leaves
    const Forest *dev_forest = nullptr;
    uint64_t dev_forest_version = 0;
    int dev_live = 0;
    cudaEvent_t ev_tags = nullptr;        // the tags' copy to the host has landed
    bool rect = true;                 // every quad an axis-aligned rectangle
    bool launch_pinned = false;       // the stage launch was chosen by the caller
    bool tune_pending = false;        // the autotuner runs before the next step
    std::string gpu_name;             // key of the autotuner's choices
    int *d_tags = nullptr;
    int *d_kind = nullptr;
    int *d_src = nullptr;
    void *d_scratch = nullptr;  // scratch of kernels outside this file (session_scratch)
    int *d_send = nullptr;      // halo send list: local quads whose records go to other ranks
    int nsend = 0;
    size_t scratch_bytes = 0;
    const void *occ_kernel = nullptr;  // launch whose occupancy occ_per_sm is
    int occ_per_sm = 0;
    cudaStream_t stream = nullptr;
    int form = AMRGPU_FORM_FP64_EXACT;
    const StageLaunch *launch = nullptr;
    int grid = 0;
    long long step_index = 0;
    int stage_pos = 0;  // stages of the current step enqueued by step_stage (0: at a step boundary)
    int64_t launches = 0;
    // counters saved by amrgpu_session_capture_mark
    long long mark_step = -1;
    int mark_roles[4] = {0, 1, 2, 3};
    int64_t mark_launches = 0;
    std::map<int, cudaGraphExec_t> graphs;
    bool primed = false;
    double t0 = 0.0;
    int sms = 148;
    // mixed patch sizes (8x8 and 16x16 quads in one mesh; extension)
    bool mixed = false;
    std::vector<int> qn;              // patch size of each quad
    std::vector<MixDesc> h_mix;
    MixDesc *d_mix = nullptr;         // per-quad sizes and offsets of the current mesh
    int cap_mix = 0;
    MixDesc *d_mix_old = nullptr;     // ... of the mesh before a regrid (remap source)
    int cap_mix_old = 0;
    int *d_work = nullptr;            // work list: the 16x16 quads, then the 8x8 quads
    int *d_work_old = nullptr;        // ... of the mesh before a regrid (kept until it is applied)
    int cap_work_old = 0;
    std::vector<int> h_work;
    bool has_rule = false;            // patch size by level for regrids built on the device
    SizeRule rule{};
    void *d_mix_scratch = nullptr;    // sizes / offsets / scans of the device build
    size_t mix_scratch_bytes = 0;
    int cap_work = 0;
    int nwork16 = 0, nwork8 = 0;
};

namespace {

double *rolebuf(amrgpu_session *s, int r) { return r < 0 ? nullptr : s->buf[s->role[r]]; }

int scheme_of(const amrgpu_session *s)
{
    int sc = s->cfg.time_scheme;
    if (s->form == AMRGPU_FORM_FP32_FLUX && sc == 3) return kSchemeRK3ShuOsher;
    return sc;
}

// Patch sizes of a mesh from the reference's own layout: quad q's state
// starts at cell_info[3q+2] and holds 4 n^2 doubles (the reference's
// sizes[] array, physics_go.c:78-86, gives the same numbers). A mesh whose
// offsets are 4 n^2 q for the configured n is uniform; otherwise every quad
// must hold an 8x8 or a 16x16 patch (mixed sizes, an extension), with no
// ghost quads. On success cells = the local quads' cells.
int mesh_sizes(const amrgpu_mesh_t *m, int n, bool &mixed, std::vector<int> &qn, long long &cells)
{
    const int nq = m->ncell, ntot = m->ncell + m->nghost;
    const long long nftm = 4LL * n * n;
    bool uniform = (long long)m->dof == nftm * nq;
    for (int q = 0; q < ntot && uniform; ++q)
        if ((long long)m->cell_info[3 * q + 2] != nftm * q) uniform = false;
    mixed = !uniform;
    qn.assign(size_t(nq), n);
    cells = (long long)nq * n * n;
    if (uniform) return AMRGPU_OK;
    if (m->nghost != 0) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: ghost quads are not supported");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (nq > 0 && m->cell_info[2] != 0) {
        set_error(AMRGPU_ERR_MESH, "cell_info[2] of quad 0 is not 0");
        return AMRGPU_ERR_MESH;
    }
    for (int q = 0; q < nq; ++q) {
        const long long a = m->cell_info[3 * q + 2];
        const long long b = (q + 1 < nq) ? (long long)m->cell_info[3 * (q + 1) + 2] : (long long)m->dof;
        const long long sz = b - a;
        if (sz != 4 * 64 && sz != 4 * 256) {
            set_error(AMRGPU_ERR_MESH, "quad " + std::to_string(q) + " holds " + std::to_string(sz) +
                                           " doubles: patches must be uniform or 8x8 / 16x16 (4*64 / 4*256)");
            return AMRGPU_ERR_MESH;
        }
        qn[size_t(q)] = sz == 4 * 64 ? 8 : 16;
    }
    cells = (long long)m->dof / 4;
    return AMRGPU_OK;
}

// face_info -> per-quad side descriptors, following the decode of
// physics_rhs_structured.c:73-262 (side parity picks left/right, side_plus,
// level_l / level_r for cell_h, ind < dof guards real quads).
int decode_mesh(amrgpu_session *s, const amrgpu_mesh_t *m)
{
    const int nq = m->ncell, ntot = m->ncell + m->nghost;
    const int n = s->n;
    const int nftm = 4 * n * n;
    s->h_quads.assign(size_t(nq), QuadDesc{});
    for (int q = 0; q < ntot && !s->mixed; ++q) {
        int off = m->cell_info[3 * q + 2];
        if (off != nftm * q) {
            set_error(AMRGPU_ERR_MESH, "cell_info[2] is not 4*n*n*id (quads must be contiguous)");
            return AMRGPU_ERR_MESH;
        }
    }
    for (int q = 0; q < nq; ++q) {
        for (int k = 0; k < 4; ++k) {
            s->h_quads[size_t(q)].side[k].kind = kSideNone;
            s->h_quads[size_t(q)].corner[2 * k] = m->geom[12 * q + 3 * k];
            s->h_quads[size_t(q)].corner[2 * k + 1] = m->geom[12 * q + 3 * k + 1];
        }
    }
    auto level = [&](int c) { return m->cell_info[3 * c + 1]; };
    auto set_side = [&](int q, int side, int kind, int n0, int n1, int rank, int lvl, int bc) -> bool {
        if (q < 0 || q >= ntot) return false;
        if (q >= nq) return true;  // ghost: no residual
        SideDesc &d = s->h_quads[size_t(q)].side[side];
        if (d.kind != kSideNone) return false;
        d.kind = kind;
        d.nbr0 = n0;
        d.nbr1 = n1;
        d.rank = rank;
        d.level = lvl;
        d.bc = bc;
        return true;
    };
    for (int f = 0; f < m->nface; ++f) {
        const int *fi = m->face_info + 11 * f;
        int ftype = fi[0], side = fi[1], cell = fi[2];
        bool ok = side >= 0 && side < 4 && cell >= 0 && cell < ntot;
        if (ok && ftype == 1) {
            ok = set_side(cell, side, kSideBoundary, -1, -1, f, level(cell), s->cfg.bc[side]);
        } else if (ok && ftype == 2) {
            int left = (side % 2 == 0) ? fi[3] : cell;
            int right = (side % 2 == 0) ? cell : fi[3];
            int hs = (side % 2 == 0) ? side + 1 : side;
            ok = left >= 0 && left < ntot && right >= 0 && right < ntot;
            if (ok) {
                int lvl = level(left);
                ok = set_side(left, hs, kSideFull, right, -1, f, lvl, 0) &&
                     set_side(right, hs - 1, kSideFull, left, -1, f, lvl, 0);
            }
        } else if (ok && ftype == 3) {
            int f0 = fi[3], f1 = fi[4];
            ok = f0 >= 0 && f0 < ntot && f1 >= 0 && f1 < ntot;
            if (ok) {
                int lvl = level(f0);
                int fine_side = (side % 2 == 0) ? side + 1 : side - 1;
                ok = set_side(cell, side, kSideCoarseHang, f0, f1, f, lvl, 0) &&
                     set_side(f0, fine_side, kSideFineHang, cell, -1, f, lvl, 0) &&
                     set_side(f1, fine_side, kSideFineHang, cell, -1, f, lvl, 0);
            }
        } else {
            ok = false;
        }
        if (!ok) {
            set_error(ftype == 5 ? AMRGPU_ERR_UNSUPPORTED : AMRGPU_ERR_MESH,
                      "face " + std::to_string(f) + " cannot be decoded (type " + std::to_string(ftype) + ")");
            return ftype == 5 ? AMRGPU_ERR_UNSUPPORTED : AMRGPU_ERR_MESH;
        }
    }
    for (int q = 0; q < nq; ++q)
        for (int k = 0; k < 4; ++k)
            if (s->h_quads[size_t(q)].side[k].kind == kSideNone) {
                set_error(AMRGPU_ERR_MESH, "quad " + std::to_string(q) + " side " + std::to_string(k) +
                                               " belongs to no face");
                return AMRGPU_ERR_MESH;
            }
    return AMRGPU_OK;
}

// Mixed-size descriptors and work list of a decoded mesh (s->h_quads,
// s->qn): per quad its size, first cell and level; per side the
// neighbour's size and first cells, and the geometric order of a hanging
// edge's two fine quads (half: for a coarse side 1 when nbr1 lies at the
// edge's lower coordinate, for a fine side 1 when this quad covers the
// upper half). The work list holds the 16x16 quads in mesh order, then the
// 8x8 quads.
int build_mix(amrgpu_session *s, const amrgpu_mesh_t *m)
{
    const int nq = s->nquad;
    s->h_mix.assign(size_t(nq), MixDesc{});
    auto base = [&](int q) { return m->cell_info[3 * q + 2] / 4; };
    // lower coordinate of quad q along the edge of side k (y for the x
    // sides 0 / 1, x for the y sides 2 / 3)
    auto along = [&](int q, int k) { return s->h_quads[size_t(q)].corner[k < 2 ? 1 : 0]; };
    auto edge_len = [&](int q, int k) {
        const double *g = s->h_quads[size_t(q)].corner;
        return k < 2 ? std::fabs(g[5] - g[1]) : std::fabs(g[2] - g[0]);
    };
    for (int q = 0; q < nq; ++q) {
        MixDesc &md = s->h_mix[size_t(q)];
        md.n = s->qn[size_t(q)];
        md.base = base(q);
        md.level = m->cell_info[3 * q + 1];
        for (int k = 0; k < 4; ++k) {
            const SideDesc &d = s->h_quads[size_t(q)].side[k];
            MixSide &ms = md.side[k];
            ms.n = md.n;
            ms.base0 = ms.base1 = 0;
            ms.half = 0;
            if (d.kind == kSideFull || d.kind == kSideCoarseHang || d.kind == kSideFineHang) {
                ms.n = s->qn[size_t(d.nbr0)];
                ms.base0 = base(d.nbr0);
            }
            if (d.kind == kSideCoarseHang) {
                if (s->qn[size_t(d.nbr1)] != s->qn[size_t(d.nbr0)]) {
                    set_error(AMRGPU_ERR_MESH, "mixed patch sizes: the two fine quads on quad " + std::to_string(q) +
                                                   "'s hanging side " + std::to_string(k) +
                                                   " differ in size (siblings must share one patch size)");
                    return AMRGPU_ERR_MESH;
                }
                ms.base1 = base(d.nbr1);
                ms.half = along(d.nbr1, k) < along(d.nbr0, k) ? 1 : 0;
            } else if (d.kind == kSideFineHang) {
                ms.half = along(q, k) - along(d.nbr0, k) > 0.25 * edge_len(q, k) ? 1 : 0;
            }
        }
    }
    std::vector<int> work;
    work.reserve(size_t(nq));
    for (int q = 0; q < nq; ++q)
        if (s->qn[size_t(q)] == 16) work.push_back(q);
    s->nwork16 = int(work.size());
    for (int q = 0; q < nq; ++q)
        if (s->qn[size_t(q)] == 8) work.push_back(q);
    s->nwork8 = int(work.size()) - s->nwork16;
    s->h_work = std::move(work);
    return AMRGPU_OK;
}

// Descriptors and work list of a mixed mesh to the device (grown buffers).
// keep_old: the current descriptors move to d_mix_old first (the remap of
// a regrid reads the old mesh's offsets).
int mix_buffers(amrgpu_session *s, int nq, bool keep_old)
{
    if (keep_old) {
        std::swap(s->d_mix, s->d_mix_old);
        std::swap(s->cap_mix, s->cap_mix_old);
        std::swap(s->d_work, s->d_work_old);
        std::swap(s->cap_work, s->cap_work_old);
    }
    if (nq > s->cap_mix || !s->d_mix) {
        cudaStreamSynchronize(s->stream);
        cudaFree(s->d_mix);
        s->d_mix = nullptr;
        s->cap_mix = 0;
        const int c = std::max(2 * nq, 1);
        if (!cuda_ok(cudaMalloc(&s->d_mix, sizeof(MixDesc) * size_t(c)), "cudaMalloc mixed descriptors"))
            return AMRGPU_ERR_CUDA;
        s->cap_mix = c;
    }
    if (nq > s->cap_work || !s->d_work) {
        cudaStreamSynchronize(s->stream);
        cudaFree(s->d_work);
        s->d_work = nullptr;
        s->cap_work = 0;
        const int c = std::max(2 * nq, 1);
        if (!cuda_ok(cudaMalloc(&s->d_work, sizeof(int) * size_t(c)), "cudaMalloc work list")) return AMRGPU_ERR_CUDA;
        s->cap_work = c;
    }
    return AMRGPU_OK;
}

int upload_mix(amrgpu_session *s, bool keep_old)
{
    const int nq = s->nquad;
    if (int rc = mix_buffers(s, nq, keep_old)) return rc;
    if (nq > 0 &&
        (!cuda_ok(cudaMemcpyAsync(s->d_mix, s->h_mix.data(), sizeof(MixDesc) * size_t(nq), cudaMemcpyHostToDevice,
                                  s->stream),
                  "upload mixed descriptors") ||
         !cuda_ok(cudaMemcpyAsync(s->d_work, s->h_work.data(), sizeof(int) * size_t(nq), cudaMemcpyHostToDevice,
                                  s->stream),
                  "upload work list")))
        return AMRGPU_ERR_CUDA;
    // the host vectors stay alive until the next build (the copies above
    // read them asynchronously)
    return AMRGPU_OK;
}

// Undoes mix_buffers(..., true) after a regrid that failed before it was
// applied: the session's descriptors and work list are the old mesh's again.
void mix_restore(amrgpu_session *s)
{
    std::swap(s->d_mix, s->d_mix_old);
    std::swap(s->cap_mix, s->cap_mix_old);
    std::swap(s->d_work, s->d_work_old);
    std::swap(s->cap_work, s->cap_work_old);
}

// Sizes and offsets of a uniform session's current mesh into d_mix (the
// remap source of a regrid that turns it into a mixed one).
int upload_uniform_mix(amrgpu_session *s)
{
    s->qn.assign(size_t(s->nquad), s->n);
    s->h_mix.assign(size_t(s->nquad), MixDesc{});
    for (int q = 0; q < s->nquad; ++q) {
        s->h_mix[size_t(q)].n = s->n;
        s->h_mix[size_t(q)].base = q * s->n * s->n;
    }
    s->h_work.assign(size_t(s->nquad), 0);
    return upload_mix(s, false);
}

// Cells of the local quads.
long long local_cells(const amrgpu_session *s)
{
    return s->mixed ? s->ncells_total : (long long)s->nquad * s->n * s->n;
}

// The FP32-flux form takes face normals and volumes from each quad's
// spacing, which needs axis-aligned rectangular quads (every brick mesh).
bool quads_are_rectangles(const amrgpu_session *s)
{
    for (const QuadDesc &q : s->h_quads) {
        const double *g = q.corner;
        double sx = std::fabs(g[2] - g[0]) + std::fabs(g[5] - g[1]);
        double tol = 1e-12 * sx;
        if (std::fabs(g[0] - g[4]) > tol || std::fabs(g[2] - g[6]) > tol || std::fabs(g[1] - g[3]) > tol ||
            std::fabs(g[5] - g[7]) > tol || !(g[2] > g[0]) || !(g[5] > g[1]))
            return false;
    }
    return true;
}

// The launch a session uses unless one was chosen: the first compiled entry
// for its patch size, except that a row sweep (one warp per quad or quad
// pair, each running a serial sweep) gives way to the first block kernel
// when the mesh has too few quads to occupy the GPU with sweep warps
// (fewer than 1024 warps: measured slower on 256-1024 quads, faster from
// 2048 warps on).
const StageLaunch *default_launch(int form, int n, int nquad)
{
    const StageLaunch *tab;
    const int cnt = (form == AMRGPU_FORM_FP32_FLUX) ? stage_table_fp32(&tab) : stage_table_fp64(&tab);
    const StageLaunch *first = nullptr, *block = nullptr;
    for (int i = 0; i < cnt; ++i) {
        if (tab[i].n != n) continue;
        if (!first) first = &tab[i];
        if (!block && !tab[i].sweep) block = &tab[i];
    }
    if (first && first->sweep && block) {
        const int qpw = first->qpb / (first->threads / 32);
        const long long warps = (nquad + qpw - 1) / qpw;
        if (warps < 1024) return block;
    }
    return first;
}

// The launch a session uses: the mixed-size sweep for a mixed mesh, else
// default_launch.
const StageLaunch *session_default_launch(const amrgpu_session *s)
{
    return s->mixed ? stage_launch_mixed() : default_launch(s->form, s->n, s->nquad);
}

const StageLaunch *find_launch(int form, int n, int qpb, int threads)
{
    const StageLaunch *tab;
    int cnt = (form == AMRGPU_FORM_FP32_FLUX) ? stage_table_fp32(&tab) : stage_table_fp64(&tab);
    for (int i = 0; i < cnt; ++i)
        if (tab[i].n == n && (qpb <= 0 || tab[i].qpb == qpb) && (threads <= 0 || tab[i].threads == threads))
            return &tab[i];
    return nullptr;
}

int configure_launch(amrgpu_session *s, const StageLaunch *L)
{
    if (!L) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "no stage kernel for this patch size");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (s->form == AMRGPU_FORM_FP32_FLUX && !s->rect) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "the FP32-flux form needs axis-aligned rectangular quads");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (s->mixed && (s->form != AMRGPU_FORM_FP32_FLUX || L->n != 0)) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: the FP32-flux form's mixed-size sweep only");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (s->occ_kernel != L->kernel) {
        if (!cuda_ok(cudaFuncSetAttribute(L->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L->smem)),
                     "cudaFuncSetAttribute"))
            return AMRGPU_ERR_CUDA;
        for (const void *k : L->kernel_so)
            if (k && !cuda_ok(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L->smem)),
                              "cudaFuncSetAttribute"))
                return AMRGPU_ERR_CUDA;
        int occ = 0;
        if (!cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, L->kernel, L->threads, L->smem),
                     "occupancy"))
            return AMRGPU_ERR_CUDA;
        s->occ_kernel = L->kernel;
        s->occ_per_sm = occ;
    }
    int per_sm = s->occ_per_sm;
    if (per_sm < 1) per_sm = 1;
    int groups = (s->nquad + L->qpb - 1) / L->qpb;
    if (s->mixed) {
        // work items (a 16x16 quad or a pair of 8x8 quads) per block = warps
        const int items = s->nwork16 + (s->nwork8 + 1) / 2;
        const int warps = L->threads / 32;
        groups = (items + warps - 1) / warps;
    }
    int g = std::min(groups, per_sm * s->sms);
    if (g < 1) g = 1;
    if (g > s->partial_cap) {
        cudaFree(s->d_partials);
        s->d_partials = nullptr;
        if (!cuda_ok(cudaMalloc(&s->d_partials, sizeof(double) * size_t(g)), "cudaMalloc partials"))
            return AMRGPU_ERR_CUDA;
        s->partial_cap = g;
    }
    s->launch = L;
    s->grid = g;
    for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
    return AMRGPU_OK;
}

// Arms the step slots (slot step_index % 3 holds the step about to run, the
// others the dt cap) and folds the first step's CFL minimum. keep_time
// re-arms on the device from the time already there (in-place regrid);
// otherwise the slots start at t0 from the host.
int prime(amrgpu_session *s, bool keep_time = false)
{
    int p = int(s->step_index % 3);
    double cap = s->cfg.dt;
    if (keep_time) {
        if (!cuda_ok(launch_rearm(s->d_scal, p, cap, s->stream), "rearm scalars")) return AMRGPU_ERR_CUDA;
        s->launches++;
    } else {
        std::memset(&s->h_scal, 0, sizeof(s->h_scal));
        for (int k = 0; k < 3; ++k) {
            std::memcpy(&s->h_scal.slot[k].dt_bits, &cap, sizeof(double));
            s->h_scal.slot[k].time = s->t0;
        }
        if (!cuda_ok(cudaMemcpyAsync(s->d_scal, &s->h_scal, sizeof(DeviceScalars), cudaMemcpyHostToDevice,
                                     s->stream),
                     "prime scalars"))
            return AMRGPU_ERR_CUDA;
    }
    bool cfl_on = s->cfg.time_scheme != 2;
    if (cfl_on && s->nquad > 0) {
        CflArgs a;
        std::memset(&a, 0, sizeof(a));
        a.quads = s->d_quads;
        a.mix = s->d_mix;
        a.qin = rolebuf(s, RX);
        a.scal = s->d_scal;
        a.stride = s->stride;
        a.nquad = s->nquad;
        a.slot = p;
        a.cfl = s->cfg.cfl;
        const void *k = s->mixed ? cfl_kernel_mixed()
                                 : (s->form == AMRGPU_FORM_FP32_FLUX ? cfl_kernel_fp32(s->n) : cfl_kernel_fp64(s->n));
        long long cells = local_cells(s);
        int g = int(std::min<long long>((cells + 255) / 256, (long long)s->sms * 8));
        if (s->mixed) g = int(std::min<long long>(((long long)s->nquad * 32 + 255) / 256, (long long)s->sms * 8));
        if (g < 1) g = 1;
        void *args[] = {&a};
        if (!cuda_ok(cudaLaunchKernel(k, dim3(g), dim3(256), args, 0, s->stream), "cfl kernel"))
            return AMRGPU_ERR_CUDA;
        s->launches++;
    }
    s->primed = true;
    return AMRGPU_OK;
}

// Launch of a stage kernel (every one begins with stage_launch_gate) with
// programmatic stream serialisation: its blocks may be scheduled while the
// previous stage kernel's last blocks are still running, and wait on the
// device for that grid to complete, so the launch gap between stages is
// hidden. AMRGPU_PDL=0 launches with plain stream order instead.
cudaError_t launch_stage_kernel(const amrgpu_session *s, StageArgs &a, const void *kernel)
{
    static const bool pdl = [] {
        const char *e = std::getenv("AMRGPU_PDL");
        return !(e && std::atoi(e) == 0);
    }();
    void *args[] = {&a};
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(s->grid);
    lc.blockDim = dim3(s->launch->threads);
    lc.dynamicSmemBytes = s->launch->smem;
    lc.stream = s->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelExC(&lc, kernel, args);
}

// Stage st (0-based) of the current step: its kernel arguments and launch.
int enqueue_stage(amrgpu_session *s, size_t st)
{
    int scheme = scheme_of(s);
    bool swap_xy = false;
    const auto &plan = plan_of(scheme, swap_xy);
    int p = int(s->step_index % 3);
    StageArgs a;
    std::memset(&a, 0, sizeof(a));
    a.quads = s->d_quads;
    a.partials = s->d_partials;
    a.scal = s->d_scal;
    a.stride = s->stride;
    a.nquad = s->nquad;
    a.scheme = scheme;
    a.cfl_on = s->cfg.time_scheme != 2;
    a.slot_read = p;
    a.slot_write = (p + 1) % 3;
    a.slot_reset = (p + 2) % 3;
    a.h_base = s->cfg.coarse_grid_h;
    a.cfl = s->cfg.cfl;
    a.dt_cap = s->cfg.dt;
    a.final_time = s->cfg.final_time;
    for (int k = 0; k < 4; ++k) a.qinflow[k] = 0.0;
    if (s->cfg.initial_condition == 5) {
        double ms = s->cfg.ic_params[0] != 0.0 ? s->cfg.ic_params[0] : 2.0;
        shock_state(s->cfg.gamma, ms, 1.0, 1.0, a.qinflow);
    }
    a.stage = int(st) + 1;
    a.last_stage = (st + 1 == plan.size()) ? 1 : 0;
    a.qin = rolebuf(s, plan[st].in);
    a.a0 = rolebuf(s, plan[st].a0);
    a.a1 = rolebuf(s, plan[st].a1);
    a.out0 = rolebuf(s, plan[st].out0);
    a.out1 = rolebuf(s, plan[st].out1);
    a.mix = s->d_mix;
    a.work = s->d_work;
    a.nwork16 = s->nwork16;
    a.nwork8 = s->nwork8;
    // the stages of a three-stage scheme run the variant specialised for
    // them when the launch has one for this scheme
    const void *k = s->launch->kernel;
    if (scheme == s->launch->so_scheme && st < 3 && s->launch->kernel_so[st]) k = s->launch->kernel_so[st];
    if (!cuda_ok(launch_stage_kernel(s, a, k), "stage kernel")) return AMRGPU_ERR_CUDA;
    s->launches++;
    return AMRGPU_OK;
}

// After the last stage of a step: buffer roles and the step counter.
void finish_step(amrgpu_session *s)
{
    bool swap_xy = false;
    plan_of(scheme_of(s), swap_xy);
    if (swap_xy) std::swap(s->role[RX], s->role[RY]);
    s->step_index++;
}

int enqueue_step(amrgpu_session *s)
{
    bool swap_xy = false;
    const auto &plan = plan_of(scheme_of(s), swap_xy);
    for (size_t st = 0; st < plan.size(); ++st) {
        int rc = enqueue_stage(s, st);
        if (rc) return rc;
    }
    finish_step(s);
    return AMRGPU_OK;
}

}  // namespace

namespace {

// A residual-only stage of the current launch: reads the state (role X)
// and writes the residual into role Z, which no scheme carries across a
// step boundary. Used by amrgpu_session_rhs and by the autotuner.
bool launch_rhs_stage(amrgpu_session *s)
{
    StageArgs a;
    std::memset(&a, 0, sizeof(a));
    a.quads = s->d_quads;
    a.qin = rolebuf(s, RX);
    a.out0 = rolebuf(s, RZ);
    a.partials = s->d_partials;
    a.scal = s->d_scal;
    a.stride = s->stride;
    a.nquad = s->nquad;
    a.scheme = kSchemeRhsOnly;
    a.stage = 1;
    a.last_stage = 0;
    a.cfl_on = 0;
    a.slot_read = int(s->step_index % 3);
    a.slot_write = (a.slot_read + 1) % 3;
    a.slot_reset = (a.slot_read + 2) % 3;
    a.h_base = s->cfg.coarse_grid_h;
    a.cfl = s->cfg.cfl;
    a.dt_cap = s->cfg.dt;
    if (s->cfg.initial_condition == 5) {
        double ms = s->cfg.ic_params[0] != 0.0 ? s->cfg.ic_params[0] : 2.0;
        amrgpu::shock_state(s->cfg.gamma, ms, 1.0, 1.0, a.qinflow);
    }
    a.mix = s->d_mix;
    a.work = s->d_work;
    a.nwork16 = s->nwork16;
    a.nwork8 = s->nwork8;
    if (!cuda_ok(launch_stage_kernel(s, a, s->launch->kernel), "rhs kernel")) return false;
    s->launches++;
    return true;
}

constexpr int kTuneMinQuads = 256;

int quad_bucket(int nquad)
{
    int b = 0;
    while ((2LL << b) <= (long long)nquad) ++b;
    return b;
}

// Launches that may replace the default: all of the patch size for the FP64
// form (every shape gives the same bits); for the FP32-flux form only the
// shapes of the default's family (row sweep or block kernel), which agree
// bit for bit among themselves.
bool tune_candidate(const amrgpu_session *s, const StageLaunch &L, const StageLaunch *def)
{
    if (s->mixed) return L.n == 0;
    if (L.n != s->n) return false;
    if (s->form == AMRGPU_FORM_FP32_FLUX && def && L.sweep != def->sweep) return false;
    return true;
}

// Chooses the session's stage launch: the stored choice for its key when
// there is one (and retime is false), else the fastest candidate, timed
// with residual-only stages on the session's current state.
int autotune_session(amrgpu_session *s, bool retime)
{
    s->tune_pending = false;
    if (s->nquad == 0) return AMRGPU_OK;
    const StageLaunch *tab;
    const int cnt = s->mixed ? stage_table_mixed(&tab)
                             : (s->form == AMRGPU_FORM_FP32_FLUX) ? stage_table_fp32(&tab) : stage_table_fp64(&tab);
    const StageLaunch *def = session_default_launch(s);
    TuneEntry key;
    key.gpu = s->gpu_name;
    key.sms = s->sms;
    key.form = s->form;
    key.n = s->mixed ? 0 : s->n;  // 0: the mixed-size sweep
    key.bucket = quad_bucket(s->nquad);
    TuneEntry hit;
    if (!retime && tune_lookup(key, &hit)) {
        for (int i = 0; i < cnt; ++i)
            if (tune_candidate(s, tab[i], def) && tab[i].qpb == hit.qpb && tab[i].threads == hit.threads &&
                tab[i].min_blocks == hit.min_blocks)
                return configure_launch(s, &tab[i]);
    }
    cudaEvent_t e0, e1;
    if (!cuda_ok(cudaEventCreate(&e0), "tune event")) return AMRGPU_ERR_CUDA;
    if (!cuda_ok(cudaEventCreate(&e1), "tune event")) {
        cudaEventDestroy(e0);
        return AMRGPU_ERR_CUDA;
    }
    const StageLaunch *best = nullptr;
    float best_ms = 0.f;
    constexpr int kReps = 3;
    for (int i = 0; i < cnt; ++i) {
        if (!tune_candidate(s, tab[i], def)) continue;
        if (configure_launch(s, &tab[i]) != AMRGPU_OK) {
            set_error(AMRGPU_OK, "");
            continue;
        }
        bool ok = launch_rhs_stage(s);  // warm-up (first launch of a kernel)
        ok = ok && cuda_ok(cudaEventRecord(e0, s->stream), "tune record");
        for (int r = 0; r < kReps && ok; ++r) ok = launch_rhs_stage(s);
        ok = ok && cuda_ok(cudaEventRecord(e1, s->stream), "tune record");
        ok = ok && cuda_ok(cudaEventSynchronize(e1), "tune sync");
        float ms = 0.f;
        if (ok) ok = cuda_ok(cudaEventElapsedTime(&ms, e0, e1), "tune elapsed");
        if (!ok) break;
        ms /= kReps;
        if (!best || ms < best_ms) {
            best = &tab[i];
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!best) return configure_launch(s, def);
    int rc = configure_launch(s, best);
    if (rc == AMRGPU_OK) {
        TuneEntry e = key;
        e.qpb = best->qpb;
        e.threads = best->threads;
        e.min_blocks = best->min_blocks;
        e.ms = best_ms;
        tune_store(e);
    }
    return rc;
}

// The autotuner, when a step is about to run on a default launch: sessions
// of at least kTuneMinQuads quads, unless AMRGPU_AUTOTUNE=0.
int maybe_autotune(amrgpu_session *s)
{
    if (!s->tune_pending) return AMRGPU_OK;
    s->tune_pending = false;
    if (s->launch_pinned || s->nquad < kTuneMinQuads) return AMRGPU_OK;
    if (const char *e = std::getenv("AMRGPU_AUTOTUNE"); e && std::atoi(e) == 0) return AMRGPU_OK;
    return autotune_session(s, false);
}

}  // namespace

int session_create_cfg(amrgpu_session_t **out, const amrgpu_mesh_t *m, const PhysicsConfig &c);

extern "C" {

int amrgpu_session_create(amrgpu_session_t **out, const amrgpu_mesh_t *m, const amrgpu_config_t *cfg)
{
    if (cfg) amrgpu_config_set(cfg);  // keeps global and session in step
    return session_create_cfg(out, m, global_config());
}

}  // extern "C"

// A session on mesh m with configuration c (the public create passes the
// library's global configuration; the evolve entry points pass the one
// they resolved).
int session_create_cfg(amrgpu_session_t **out, const amrgpu_mesh_t *m, const PhysicsConfig &c)
{
    if (!out || !m || !m->cell_info || !m->geom || (m->nface > 0 && !m->face_info) || m->ncell < 0 ||
        m->nghost < 0) {
        set_error(AMRGPU_ERR_ARG, "session_create: null or negative arguments");
        return AMRGPU_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error(AMRGPU_ERR_NO_DEVICE, "no CUDA device visible");
        return AMRGPU_ERR_NO_DEVICE;
    }
    amrgpu_session *s = new amrgpu_session;
    s->cfg = c;
    s->n = s->cfg.nelem_subgrid;
    s->form = s->cfg.form;
    if (s->cfg.dim != 2 || s->cfg.nfields != 4) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "only dim 2 with 4 fields");
        delete s;
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (s->cfg.time_scheme < 1 || s->cfg.time_scheme > 5) {
        set_error(AMRGPU_ERR_CONFIG, "time_scheme must be 1..5");
        delete s;
        return AMRGPU_ERR_CONFIG;
    }
    s->nquad = m->ncell;
    s->nghost = m->nghost;
    s->nface = m->nface;
    s->dof = m->dof;
    long long mesh_cells = 0;
    int rc = mesh_sizes(m, s->n, s->mixed, s->qn, mesh_cells);
    if (rc != AMRGPU_OK) {
        delete s;
        return rc;
    }
    if (s->mixed && s->form != AMRGPU_FORM_FP32_FLUX) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: the FP32-flux form only (gpu_form: 1)");
        delete s;
        return AMRGPU_ERR_UNSUPPORTED;
    }
    rc = decode_mesh(s, m);
    if (rc != AMRGPU_OK) {
        delete s;
        return rc;
    }
    if (s->mixed) {
        rc = build_mix(s, m);
        if (rc != AMRGPU_OK) {
            delete s;
            return rc;
        }
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, dev);
    s->ncells_total = s->mixed ? mesh_cells : (long long)(m->ncell + m->nghost) * s->n * s->n;
    s->stride = ((s->ncells_total + 31) / 32) * 32;
    if (s->stride == 0) s->stride = 32;
    // state buffers hold a quarter more cells than the mesh, so that a regrid
    // that grows the mesh a little reuses them; the AoS staging and the
    // totals partials are sized for the same capacity
    s->cap_stride = ((s->stride + s->stride / 4 + 31) / 32) * 32;
    bool ok = cuda_ok(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
    for (int k = 0; k < 4 && ok; ++k) {
        ok = cuda_ok(cudaMalloc(&s->buf[k], sizeof(double) * 4 * size_t(s->cap_stride)), "cudaMalloc state");
        if (ok)
            ok = cuda_ok(cudaMemsetAsync(s->buf[k], 0, sizeof(double) * 4 * size_t(s->cap_stride), s->stream), "memset");
    }
    if (ok) ok = cuda_ok(cudaMalloc(&s->d_aos, sizeof(double) * 4 * size_t(s->cap_stride)), "cudaMalloc aos");
    if (ok) ok = cuda_ok(cudaMalloc(&s->d_scal, sizeof(DeviceScalars)), "cudaMalloc scalars");
    if (ok && s->nquad > 0) {
        ok = cuda_ok(cudaMalloc(&s->d_quads, sizeof(QuadDesc) * size_t(s->nquad)), "cudaMalloc quads");
        if (ok)
            ok = cuda_ok(cudaMemcpy(s->d_quads, s->h_quads.data(), sizeof(QuadDesc) * size_t(s->nquad),
                                    cudaMemcpyHostToDevice),
                         "upload quads");
    }
    if (ok) ok = cuda_ok(cudaMalloc(&s->d_tot, sizeof(double) * 4 * size_t(totals_grid(s->cap_stride))), "cudaMalloc totals");
    if (ok && s->mixed) ok = upload_mix(s, false) == AMRGPU_OK;
    s->cap_quads = std::max(s->nquad, 1);
    s->cap_desc = s->nquad;
    s->rect = quads_are_rectangles(s);
    for (int **p : {&s->d_tags, &s->d_kind, &s->d_src})
        if (ok) ok = cuda_ok(cudaMalloc(p, sizeof(int) * size_t(s->cap_quads)), "cudaMalloc quad arrays");
    if (!ok) {
        amrgpu_session_destroy(s);
        return AMRGPU_ERR_CUDA;
    }
    const StageLaunch *L = session_default_launch(s);
    const char *env_q = std::getenv("AMRGPU_QPB");
    const char *env_t = std::getenv("AMRGPU_THREADS");
    if ((env_q || env_t) && !s->mixed) {
        const StageLaunch *L2 = find_launch(s->form, s->n, env_q ? std::atoi(env_q) : 0, env_t ? std::atoi(env_t) : 0);
        if (L2) {
            L = L2;
            s->launch_pinned = true;
        }
    }
    rc = configure_launch(s, L);
    if (rc != AMRGPU_OK) {
        amrgpu_session_destroy(s);
        return rc;
    }
    s->gpu_name = device_name(dev);
    s->tune_pending = !s->launch_pinned;
    *out = s;
    return AMRGPU_OK;
}

extern "C" {

void amrgpu_session_destroy(amrgpu_session_t *s)
{
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
    for (int k = 0; k < 4; ++k) cudaFree(s->buf[k]);
    cudaFree(s->d_aos);
    cudaFree(s->d_scal);
    cudaFree(s->d_partials);
    cudaFree(s->d_quads);
    cudaFree(s->d_tot);
    cudaFree(s->d_tags);
    cudaFree(s->d_kind);
    cudaFree(s->d_src);
    cudaFree(s->d_scratch);
    cudaFree(s->d_send);
    cudaFree(s->d_quads_alt);
    cudaFree(s->d_mesh_scratch);
    cudaFree(s->d_fstage);
    cudaFree(s->d_bal[0]);
    cudaFree(s->d_bal[1]);
    cudaFree(s->d_remap0);
    cudaFree(s->d_bal_work);
    cudaFreeHost(s->h_stage);
    if (s->ev_tags) cudaEventDestroy(s->ev_tags);
    cudaFree(s->d_mix);
    cudaFree(s->d_mix_old);
    cudaFree(s->d_work);
    cudaFree(s->d_work_old);
    cudaFree(s->d_mix_scratch);
    s->ring.release();
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int amrgpu_session_set_form(amrgpu_session_t *s, int form)
{
    if (!s || (form != AMRGPU_FORM_FP64_EXACT && form != AMRGPU_FORM_FP32_FLUX)) return AMRGPU_ERR_ARG;
    if (form == s->form) return AMRGPU_OK;
    if (s->mixed) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: the FP32-flux form only");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    // keep the current state where the canonical X role points
    s->form = form;
    s->cfg.form = form;
    s->launch_pinned = false;
    s->tune_pending = true;
    return configure_launch(s, default_launch(form, s->n, s->nquad));
}

int amrgpu_session_set_launch(amrgpu_session_t *s, int qpb, int threads)
{
    if (!s) return AMRGPU_ERR_ARG;
    const StageLaunch *L = find_launch(s->form, s->n, qpb, threads);
    if (!L) {
        set_error(AMRGPU_ERR_ARG, "no compiled variant with that shape");
        return AMRGPU_ERR_ARG;
    }
    s->launch_pinned = true;
    return configure_launch(s, L);
}

int amrgpu_session_set_launch_variant(amrgpu_session_t *s, int index)
{
    if (!s) return AMRGPU_ERR_ARG;
    const StageLaunch *tab;
    const int cnt = (s->form == AMRGPU_FORM_FP32_FLUX) ? stage_table_fp32(&tab) : stage_table_fp64(&tab);
    int k = 0;
    for (int i = 0; i < cnt; ++i) {
        if (tab[i].n != s->n) continue;
        if (k++ == index) {
            s->launch_pinned = true;
            return configure_launch(s, &tab[i]);
        }
    }
    set_error(AMRGPU_ERR_ARG, "no compiled variant with that index");
    return AMRGPU_ERR_ARG;
}

int amrgpu_session_launch_variant(const amrgpu_session_t *s)
{
    if (!s || !s->launch) return -1;
    const StageLaunch *tab;
    const int cnt = (s->form == AMRGPU_FORM_FP32_FLUX) ? stage_table_fp32(&tab) : stage_table_fp64(&tab);
    int k = 0;
    for (int i = 0; i < cnt; ++i) {
        if (tab[i].n != s->n) continue;
        if (&tab[i] == s->launch) return k;
        ++k;
    }
    return -1;
}

int amrgpu_session_launch_variants(const amrgpu_session_t *s, int *qpb, int *threads, int cap)
{
    if (!s || cap < 0) return -AMRGPU_ERR_ARG;
    const StageLaunch *tab;
    const int cnt = (s->form == AMRGPU_FORM_FP32_FLUX) ? stage_table_fp32(&tab) : stage_table_fp64(&tab);
    int k = 0;
    for (int i = 0; i < cnt; ++i) {
        if (tab[i].n != s->n) continue;
        if (k < cap && qpb && threads) {
            qpb[k] = tab[i].qpb;
            threads[k] = tab[i].threads;
        }
        ++k;
    }
    return k;
}

int amrgpu_session_launch_variant_info(const amrgpu_session_t *s, int index, int *qpb, int *threads,
                                       int *min_blocks, int *sweep)
{
    if (!s) return AMRGPU_ERR_ARG;
    const StageLaunch *tab;
    const int cnt = (s->form == AMRGPU_FORM_FP32_FLUX) ? stage_table_fp32(&tab) : stage_table_fp64(&tab);
    int k = 0;
    for (int i = 0; i < cnt; ++i) {
        if (tab[i].n != s->n) continue;
        if (k++ != index) continue;
        if (qpb) *qpb = tab[i].qpb;
        if (threads) *threads = tab[i].threads;
        if (min_blocks) *min_blocks = tab[i].min_blocks;
        if (sweep) *sweep = tab[i].sweep;
        return AMRGPU_OK;
    }
    set_error(AMRGPU_ERR_ARG, "no compiled variant with that index");
    return AMRGPU_ERR_ARG;
}

int amrgpu_session_upload(amrgpu_session_t *s, const double *soln)
{
    if (!s || !soln) return AMRGPU_ERR_ARG;
    size_t bytes = sizeof(double) * 4 * size_t(s->ncells_total);
    if (bytes) {
        // pinned caller arrays go straight to the device; pageable ones
        // through the session's pinned chunks (staging.cu)
        if (!ring_h2d(s->ring, s->d_aos, soln, bytes, s->stream)) return AMRGPU_ERR_CUDA;
        if (!cuda_ok(launch_aos_to_soa(s->d_aos, rolebuf(s, RX), s->ncells_total, s->stride, s->stream), "aos_to_soa"))
            return AMRGPU_ERR_CUDA;
        s->launches++;
    }
    return prime(s);
}

int amrgpu_session_download(amrgpu_session_t *s, double *soln)
{
    if (!s || !soln) return AMRGPU_ERR_ARG;
    long long cells = local_cells(s);
    if (cells) {
        if (!cuda_ok(launch_soa_to_aos(rolebuf(s, RX), s->d_aos, cells, s->stride, s->stream), "soa_to_aos"))
            return AMRGPU_ERR_CUDA;
        s->launches++;
        if (!ring_d2h(s->ring, soln, s->d_aos, sizeof(double) * 4 * size_t(cells), s->stream))
            return AMRGPU_ERR_CUDA;
    }
    return cuda_ok(cudaStreamSynchronize(s->stream), "sync") ? AMRGPU_OK : AMRGPU_ERR_CUDA;
}

int amrgpu_session_step_stage(amrgpu_session_t *s, int *stage, int *stages_per_step)
{
    if (!s) return AMRGPU_ERR_ARG;
    if (!s->primed) {
        int rc = prime(s);
        if (rc) return rc;
    }
    if (s->stage_pos == 0 && s->nquad > 0) {
        if (int rc = maybe_autotune(s)) return rc;
    }
    bool swap_xy = false;
    const auto &plan = plan_of(scheme_of(s), swap_xy);
    if (stage) *stage = s->stage_pos + 1;
    if (stages_per_step) *stages_per_step = int(plan.size());
    if (s->nquad > 0) {
        int rc = enqueue_stage(s, size_t(s->stage_pos));
        if (rc) return rc;
    }
    if (++s->stage_pos == int(plan.size())) {
        s->stage_pos = 0;
        finish_step(s);
    }
    return AMRGPU_OK;
}

double *amrgpu_session_stage_input(amrgpu_session_t *s, long long *field_stride)
{
    if (!s) return nullptr;
    bool swap_xy = false;
    const auto &plan = plan_of(scheme_of(s), swap_xy);
    if (field_stride) *field_stride = s->stride;
    return rolebuf(s, plan[size_t(s->stage_pos)].in);
}

int amrgpu_session_capture_mark(amrgpu_session_t *s)
{
    if (!s) return AMRGPU_ERR_ARG;
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_capture_mark: a step begun with step_stage is not finished");
        return AMRGPU_ERR_ARG;
    }
    if (!s->primed) {
        if (int rc = prime(s)) return rc;
    }
    if (s->nquad > 0) {
        if (int rc = maybe_autotune(s)) return rc;
    }
    if (!cuda_ok(cudaStreamSynchronize(s->stream), "sync")) return AMRGPU_ERR_CUDA;
    s->mark_step = s->step_index;
    std::memcpy(s->mark_roles, s->role, sizeof(s->role));
    s->mark_launches = s->launches;
    return AMRGPU_OK;
}

int amrgpu_session_capture_rewind(amrgpu_session_t *s)
{
    if (!s || s->mark_step < 0) return AMRGPU_ERR_ARG;
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_capture_rewind: the captured work ends inside a step");
        return AMRGPU_ERR_ARG;
    }
    s->step_index = s->mark_step;
    std::memcpy(s->role, s->mark_roles, sizeof(s->role));
    s->launches = s->mark_launches;
    s->mark_step = -1;
    return AMRGPU_OK;
}

int amrgpu_session_advance(amrgpu_session_t *s, int nsteps)
{
    if (!s || nsteps < 0 || s->stage_pos != 0) return AMRGPU_ERR_ARG;
    bool swap_xy = false;
    const auto &plan = plan_of(scheme_of(s), swap_xy);
    // the step's own launches: stage kernels, and the halo kernels of a
    // session with a send list (pack and unpack before every stage)
    const int per_stage = 1 + (s->nsend > 0 ? 1 : 0) + (s->nghost > 0 ? 1 : 0);
    s->launches += (int64_t)nsteps * (int64_t)plan.size() * per_stage;
    if (swap_xy && (nsteps % 2)) std::swap(s->role[RX], s->role[RY]);
    s->step_index += nsteps;
    return AMRGPU_OK;
}

long long amrgpu_session_step_index(const amrgpu_session_t *s) { return s ? s->step_index : -1; }

unsigned long long *amrgpu_session_dt_slot(amrgpu_session_t *s)
{
    if (!s) return nullptr;
    return &s->d_scal->slot[s->step_index % 3].dt_bits;
}

int amrgpu_session_set_halo(amrgpu_session_t *s, const int *send_quads, int nsend)
{
    if (!s || nsend < 0 || (nsend > 0 && !send_quads)) return AMRGPU_ERR_ARG;
    if (s->mixed && nsend > 0) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: no ghost exchange");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    for (int k = 0; k < nsend; ++k)
        if (send_quads[k] < 0 || send_quads[k] >= s->nquad) {
            set_error(AMRGPU_ERR_ARG, "set_halo: send entry " + std::to_string(k) + " is not a local quad");
            return AMRGPU_ERR_ARG;
        }
    if (nsend > s->nsend || !s->d_send) {
        cudaFree(s->d_send);
        s->d_send = nullptr;
        s->nsend = 0;
        if (!cuda_ok(cudaMalloc(&s->d_send, sizeof(int) * size_t(nsend > 0 ? nsend : 1)), "halo list"))
            return AMRGPU_ERR_CUDA;
    }
    if (nsend > 0 &&
        !cuda_ok(cudaMemcpyAsync(s->d_send, send_quads, sizeof(int) * size_t(nsend), cudaMemcpyHostToDevice,
                                 s->stream),
                 "H2D halo list"))
        return AMRGPU_ERR_CUDA;
    if (!cuda_ok(cudaStreamSynchronize(s->stream), "sync")) return AMRGPU_ERR_CUDA;
    s->nsend = nsend;
    return AMRGPU_OK;
}

int amrgpu_session_halo_pack(amrgpu_session_t *s, int first, int count, double *d_out)
{
    if (!s || first < 0 || count < 0 || first + count > s->nsend || (count > 0 && !d_out)) return AMRGPU_ERR_ARG;
    bool swap_xy = false;
    const auto &plan = plan_of(scheme_of(s), swap_xy);
    const double *q = rolebuf(s, plan[size_t(s->stage_pos)].in);
    if (!cuda_ok(launch_halo_pack(q, s->stride, s->n, s->d_send + first, count, d_out, s->sms, s->stream),
                 "halo pack"))
        return AMRGPU_ERR_CUDA;
    if (count > 0) s->launches++;
    return AMRGPU_OK;
}

int amrgpu_session_halo_unpack(amrgpu_session_t *s, int first_ghost, int count, const double *d_in)
{
    if (!s || first_ghost < 0 || count < 0 || first_ghost + count > s->nghost || (count > 0 && !d_in))
        return AMRGPU_ERR_ARG;
    bool swap_xy = false;
    const auto &plan = plan_of(scheme_of(s), swap_xy);
    double *q = rolebuf(s, plan[size_t(s->stage_pos)].in);
    if (!cuda_ok(launch_halo_unpack(q, s->stride, s->n, s->nquad + first_ghost, count, d_in, s->sms, s->stream),
                 "halo unpack"))
        return AMRGPU_ERR_CUDA;
    if (count > 0) s->launches++;
    return AMRGPU_OK;
}

int amrgpu_session_halo_pack_edges(amrgpu_session_t *s, int first, int count, double *d_out)
{
    if (!s || first < 0 || count < 0 || first + count > s->nsend || (count > 0 && !d_out)) return AMRGPU_ERR_ARG;
    bool swap_xy = false;
    const auto &plan = plan_of(scheme_of(s), swap_xy);
    const double *q = rolebuf(s, plan[size_t(s->stage_pos)].in);
    if (!cuda_ok(launch_halo_pack_edges(q, s->stride, s->n, s->d_send + first, count, d_out, s->sms, s->stream),
                 "halo pack"))
        return AMRGPU_ERR_CUDA;
    if (count > 0) s->launches++;
    return AMRGPU_OK;
}

int amrgpu_session_halo_unpack_edges(amrgpu_session_t *s, int first_ghost, int count, const double *d_in)
{
    if (!s || first_ghost < 0 || count < 0 || first_ghost + count > s->nghost || (count > 0 && !d_in))
        return AMRGPU_ERR_ARG;
    bool swap_xy = false;
    const auto &plan = plan_of(scheme_of(s), swap_xy);
    double *q = rolebuf(s, plan[size_t(s->stage_pos)].in);
    if (!cuda_ok(launch_halo_unpack_edges(q, s->stride, s->n, s->nquad + first_ghost, count, d_in, s->sms,
                                          s->stream),
                 "halo unpack"))
        return AMRGPU_ERR_CUDA;
    if (count > 0) s->launches++;
    return AMRGPU_OK;
}

int amrgpu_session_local_scalars(amrgpu_session_t *s, double *norm_sq, int *flags)
{
    if (!s) return AMRGPU_ERR_ARG;
    if (norm_sq) *norm_sq = s->h_scal.norm_sq;
    if (flags) *flags = s->h_scal.flags;
    return AMRGPU_OK;
}

int amrgpu_session_step(amrgpu_session_t *s, int nsteps)
{
    if (!s || nsteps < 0) return AMRGPU_ERR_ARG;
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_step: a step begun with step_stage is not finished");
        return AMRGPU_ERR_ARG;
    }
    if (!s->primed) {
        int rc = prime(s);
        if (rc) return rc;
    }
    if (s->nquad == 0) return AMRGPU_OK;
    if (int rc = maybe_autotune(s)) return rc;
    for (int k = 0; k < nsteps; ++k) {
        int rc = enqueue_step(s);
        if (rc) return rc;
    }
    return AMRGPU_OK;
}

int amrgpu_session_step_graph(amrgpu_session_t *s, int nsteps, int graph_steps)
{
    if (!s || nsteps < 0) return AMRGPU_ERR_ARG;
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_step_graph: a step begun with step_stage is not finished");
        return AMRGPU_ERR_ARG;
    }
    if (graph_steps < 6) graph_steps = 6;
    graph_steps -= graph_steps % 6;
    if (!s->primed) {
        int rc = prime(s);
        if (rc) return rc;
    }
    if (s->nquad == 0) return AMRGPU_OK;
    if (int rc = maybe_autotune(s)) return rc;
    int done = 0;
    // align to a 6-step boundary: slot phase (3) and buffer-role parity (2)
    while (done < nsteps && (s->step_index % 6) != 0) {
        int rc = enqueue_step(s);
        if (rc) return rc;
        ++done;
    }
    while (nsteps - done >= graph_steps) {
        auto it = s->graphs.find(graph_steps);
        if (it == s->graphs.end()) {
            cudaGraph_t g;
            long long si = s->step_index;
            int roles[4];
            std::memcpy(roles, s->role, sizeof(roles));
            int64_t l0 = s->launches;
            if (!cuda_ok(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture"))
                return AMRGPU_ERR_CUDA;
            for (int k = 0; k < graph_steps; ++k) enqueue_step(s);
            if (!cuda_ok(cudaStreamEndCapture(s->stream, &g), "end capture")) return AMRGPU_ERR_CUDA;
            cudaGraphExec_t ge;
            if (!cuda_ok(cudaGraphInstantiate(&ge, g, 0), "graph instantiate")) return AMRGPU_ERR_CUDA;
            cudaGraphDestroy(g);
            s->graphs[graph_steps] = ge;
            s->step_index = si;
            std::memcpy(s->role, roles, sizeof(roles));
            s->launches = l0;
            it = s->graphs.find(graph_steps);
        }
        if (!cuda_ok(cudaGraphLaunch(it->second, s->stream), "graph launch")) return AMRGPU_ERR_CUDA;
        // advance host-side bookkeeping exactly as the captured steps did
        bool swap_xy = false;
        const auto &plan = plan_of(scheme_of(s), swap_xy);
        s->launches += (int64_t)graph_steps * (int64_t)plan.size();
        if (swap_xy && (graph_steps % 2)) std::swap(s->role[RX], s->role[RY]);
        s->step_index += graph_steps;
        done += graph_steps;
    }
    while (done < nsteps) {
        int rc = enqueue_step(s);
        if (rc) return rc;
        ++done;
    }
    return AMRGPU_OK;
}

int amrgpu_session_sync(amrgpu_session_t *s, amrgpu_report_t *rep)
{
    if (!s) return AMRGPU_ERR_ARG;
    if (!cuda_ok(cudaMemcpyAsync(&s->h_scal, s->d_scal, sizeof(DeviceScalars), cudaMemcpyDeviceToHost, s->stream),
                 "D2H scalars"))
        return AMRGPU_ERR_CUDA;
    if (!cuda_ok(cudaStreamSynchronize(s->stream), "sync")) return AMRGPU_ERR_CUDA;
    int p = int(s->step_index % 3);
    if (rep) {
        rep->steps_done = s->h_scal.steps;
        rep->time = s->h_scal.slot[p].time;
        rep->dt_last = s->h_scal.dt_used;
        rep->residual_norm = std::sqrt(s->h_scal.norm_sq);
        rep->nan_detected = (s->h_scal.flags & kFlagNonFinite) ? 1 : 0;
        rep->error = rep->nan_detected ? AMRGPU_ERR_NONFINITE
                                       : ((s->h_scal.flags & kFlagNegative) ? AMRGPU_ERR_NEGATIVE : AMRGPU_OK);
    }
    return AMRGPU_OK;
}

int amrgpu_session_rhs(amrgpu_session_t *s, double *rhs)
{
    if (!s || !rhs) return AMRGPU_ERR_ARG;
    if (s->nquad == 0) return AMRGPU_OK;
    if (!launch_rhs_stage(s)) return AMRGPU_ERR_CUDA;
    s->launches++;
    long long cells = local_cells(s);
    if (!cuda_ok(launch_soa_to_aos(rolebuf(s, RZ), s->d_aos, cells, s->stride, s->stream), "soa_to_aos"))
        return AMRGPU_ERR_CUDA;
    s->launches++;
    if (!cuda_ok(cudaMemcpyAsync(rhs, s->d_aos, sizeof(double) * 4 * size_t(cells), cudaMemcpyDeviceToHost, s->stream),
                 "D2H rhs"))
        return AMRGPU_ERR_CUDA;
    return cuda_ok(cudaStreamSynchronize(s->stream), "sync") ? AMRGPU_OK : AMRGPU_ERR_CUDA;
}

int amrgpu_session_cfl_dt(amrgpu_session_t *s, double *dt)
{
    if (!s || !dt) return AMRGPU_ERR_ARG;
    long long keep = s->step_index;
    int rc = prime(s);
    if (rc) return rc;
    s->step_index = keep;
    rc = amrgpu_session_sync(s, nullptr);
    if (rc) return rc;
    std::memcpy(dt, &s->h_scal.slot[s->step_index % 3].dt_bits, sizeof(double));
    if (s->cfg.time_scheme == 2) *dt = s->cfg.dt;
    return AMRGPU_OK;
}

const double *amrgpu_session_state_device(amrgpu_session_t *s, int field)
{
    if (!s || field < 0 || field > 3) return nullptr;
    return rolebuf(s, RX) + size_t(field) * size_t(s->stride);
}

int amrgpu_session_cells(const amrgpu_session_t *s) { return s ? int(local_cells(s)) : 0; }

void *amrgpu_session_stream(amrgpu_session_t *s) { return s ? (void *)s->stream : nullptr; }

int64_t amrgpu_session_launch_count(const amrgpu_session_t *s) { return s ? s->launches : 0; }

int amrgpu_session_autotune(amrgpu_session_t *s, int retime)
{
    if (!s) return AMRGPU_ERR_ARG;
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_autotune: a step begun with step_stage is not finished");
        return AMRGPU_ERR_ARG;
    }
    if (!s->primed) {
        set_error(AMRGPU_ERR_ARG, "session_autotune: no state uploaded");
        return AMRGPU_ERR_ARG;
    }
    s->launch_pinned = false;
    return autotune_session(s, retime != 0);
}

int amrgpu_tune_cache_get(const char *gpu, int sms, int form, int n, int nquad, int *qpb, int *threads,
                          int *min_blocks, double *ms)
{
    if (!gpu) return 0;
    TuneEntry key, hit;
    key.gpu = gpu;
    key.sms = sms;
    key.form = form;
    key.n = n;
    key.bucket = quad_bucket(nquad);
    if (!tune_lookup(key, &hit)) return 0;
    if (qpb) *qpb = hit.qpb;
    if (threads) *threads = hit.threads;
    if (min_blocks) *min_blocks = hit.min_blocks;
    if (ms) *ms = hit.ms;
    return 1;
}

int amrgpu_tune_cache_put(const char *gpu, int sms, int form, int n, int nquad, int qpb, int threads,
                          int min_blocks, double ms)
{
    if (!gpu || nquad < 1) return AMRGPU_ERR_ARG;
    TuneEntry e;
    e.gpu = gpu;
    for (char &c : e.gpu)
        if (c == '"' || c == '\\') c = '_';
    e.sms = sms;
    e.form = form;
    e.n = n;
    e.bucket = quad_bucket(nquad);
    e.qpb = qpb;
    e.threads = threads;
    e.min_blocks = min_blocks;
    e.ms = ms;
    tune_store(e);
    return AMRGPU_OK;
}

void amrgpu_tune_cache_reload(void) { tune_forget(); }

}  // extern "C"

namespace amrgpu {

bool session_view(amrgpu_session_t *s, SessionView *v)
{
    if (!s || !v) return false;
    if (s->mixed) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: not supported by this call (uniform meshes only)");
        return false;
    }
    v->n = s->n;
    v->nquad = s->nquad;
    v->stride = s->stride;
    v->q = rolebuf(s, RX);
    v->quads = s->d_quads;
    v->stream = s->stream;
    return true;
}

void *session_scratch(amrgpu_session_t *s, size_t bytes)
{
    if (!s) return nullptr;
    if (bytes > s->scratch_bytes) {
        cudaStreamSynchronize(s->stream);
        cudaFree(s->d_scratch);
        s->d_scratch = nullptr;
        s->scratch_bytes = 0;
        const size_t want = bytes + bytes / 4;
        if (cudaMalloc(&s->d_scratch, want) != cudaSuccess) return nullptr;
        s->scratch_bytes = want;
    }
    return s->d_scratch;
}

void session_count_launches(amrgpu_session_t *s, int k)
{
    if (s) s->launches += k;
}

}  // namespace amrgpu

extern "C" {

int amrgpu_session_totals(amrgpu_session_t *s, double totals[4])
{
    if (!s || !totals) return AMRGPU_ERR_ARG;
    long long cells = local_cells(s);
    int g = totals_grid(std::max<long long>(cells, 1));
    if (s->mixed) {
        g = std::min(g, totals_mixed_grid(std::max(s->nquad, 1)));
        if (!cuda_ok(launch_totals_mixed(s->d_quads, s->d_mix, rolebuf(s, RX), s->stride, s->nquad, s->d_tot, g,
                                         s->stream),
                     "totals"))
            return AMRGPU_ERR_CUDA;
    } else if (!cuda_ok(launch_totals(s->n, s->d_quads, rolebuf(s, RX), s->stride, s->nquad, s->d_tot, g, s->stream),
                        "totals")) {
        return AMRGPU_ERR_CUDA;
    }
    s->launches++;
    std::vector<double> h(size_t(4 * g));
    if (!cuda_ok(cudaMemcpyAsync(h.data(), s->d_tot, sizeof(double) * 4 * size_t(g), cudaMemcpyDeviceToHost, s->stream),
                 "D2H totals"))
        return AMRGPU_ERR_CUDA;
    if (!cuda_ok(cudaStreamSynchronize(s->stream), "sync")) return AMRGPU_ERR_CUDA;
    for (int f = 0; f < 4; ++f) {
        double t = 0.0;
        for (int b = 0; b < g; ++b) t += h[size_t(4 * b + f)];
        totals[f] = t;
    }
    return AMRGPU_OK;
}

}  // extern "C"

namespace {

// The session's refinement tags of the current state into d_tags.
bool launch_tags(amrgpu_session *s)
{
    TagMethods m;
    int nm = std::min(s->cfg.amr_ntag_methods, 5);
    for (int k = 0; k < 5; ++k) {
        m.method[k] = k < nm ? s->cfg.amr_tag_methods[size_t(k)] : 0;
        m.tol[k] = k < nm ? s->cfg.amr_tag_tolerances[size_t(k)] : 0.0;
    }
    const bool ok = cuda_ok(s->mixed ? launch_tag_mixed(rolebuf(s, RX), s->d_quads, s->d_mix, s->nquad, nm, m,
                                                        s->d_tags, s->stream)
                                     : launch_tag(s->n, rolebuf(s, RX), s->d_quads, s->nquad, nm, m, s->d_tags,
                                                  s->stream),
                            "tag kernel");
    s->launches++;
    return ok;
}

}  // namespace

extern "C" {

int amrgpu_session_tag(amrgpu_session_t *s, int *tags)
{
    if (!s || !tags) return AMRGPU_ERR_ARG;
    if (s->nquad == 0) return AMRGPU_OK;
    bool ok = launch_tags(s);
    if (ok)
        ok = cuda_ok(cudaMemcpyAsync(tags, s->d_tags, sizeof(int) * size_t(s->nquad), cudaMemcpyDeviceToHost,
                                     s->stream),
                     "D2H tags");
    if (ok) ok = cuda_ok(cudaStreamSynchronize(s->stream), "sync");
    return ok ? AMRGPU_OK : AMRGPU_ERR_CUDA;
}

int amrgpu_session_remap(amrgpu_session_t *dst, amrgpu_session_t *src, const int *kind, const int *src_index)
{
    if (!dst || !src || !kind || !src_index || dst->n != src->n) return AMRGPU_ERR_ARG;
    if (dst->mixed || src->mixed) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: use amrgpu_session_regrid (in place)");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    for (int q = 0; q < dst->nquad; ++q) {
        int lim = kind[q] == 0 ? src->nquad - 1 : src->nquad - 4;
        if (src_index[q] < 0 || src_index[q] > lim) {
            set_error(AMRGPU_ERR_ARG, "remap source index out of range");
            return AMRGPU_ERR_ARG;
        }
    }
    cudaStreamSynchronize(src->stream);
    bool ok = cuda_ok(cudaMemcpyAsync(dst->d_kind, kind, sizeof(int) * size_t(dst->nquad), cudaMemcpyHostToDevice,
                                      dst->stream),
                      "H2D remap") &&
              cuda_ok(cudaMemcpyAsync(dst->d_src, src_index, sizeof(int) * size_t(dst->nquad),
                                      cudaMemcpyHostToDevice, dst->stream),
                      "H2D remap");
    if (ok && dst->nquad > 0) {
        ok = cuda_ok(launch_remap(dst->n, rolebuf(src, RX), src->stride, rolebuf(dst, RX), dst->stride, dst->d_kind,
                                  dst->d_src, dst->nquad, dst->stream),
                     "remap kernel");
        dst->launches++;
    }
    if (!ok) return AMRGPU_ERR_CUDA;
    dst->t0 = src->h_scal.slot[src->step_index % 3].time;
    return prime(dst);
}

}  // extern "C"

namespace {

// Per-quad tag and remap arrays for nq quads (grown by a quarter beyond the
// need so that a slowly growing mesh reallocates rarely; cudaFree
// synchronises the device).
int ensure_quad_arrays(amrgpu_session *s, int nq)
{
    if (nq <= s->cap_quads) return AMRGPU_OK;
    const int cap = 2 * nq;
    int *arr[3] = {nullptr, nullptr, nullptr};
    bool ok = true;
    for (int k = 0; k < 3 && ok; ++k) ok = cuda_ok(cudaMalloc(&arr[k], sizeof(int) * size_t(cap)), "cudaMalloc quad arrays");
    if (!ok) {
        for (int *p : arr) cudaFree(p);
        return AMRGPU_ERR_CUDA;
    }
    // the tags are kept (a device adapt that grows its buffers reads them
    // again); kind and source are outputs
    if (s->d_tags && s->cap_quads > 0)
        ok = cuda_ok(cudaMemcpyAsync(arr[0], s->d_tags, sizeof(int) * size_t(s->cap_quads), cudaMemcpyDeviceToDevice,
                                     s->stream),
                     "tags copy");
    cudaStreamSynchronize(s->stream);
    if (!ok) {
        for (int *p : arr) cudaFree(p);
        return AMRGPU_ERR_CUDA;
    }
    cudaFree(s->d_tags);
    cudaFree(s->d_kind);
    cudaFree(s->d_src);
    s->d_tags = arr[0];
    s->d_kind = arr[1];
    s->d_src = arr[2];
    s->cap_quads = cap;
    return AMRGPU_OK;
}

// A descriptor buffer for at least nq quads (contents not kept).
int ensure_desc(amrgpu_session *s, QuadDesc **buf, int *cap, int nq)
{
    if (nq <= *cap && *buf) return AMRGPU_OK;
    const int c = std::max(2 * nq, 1);
    QuadDesc *d = nullptr;
    if (!cuda_ok(cudaMalloc(&d, sizeof(QuadDesc) * size_t(c)), "cudaMalloc quads")) return AMRGPU_ERR_CUDA;
    cudaStreamSynchronize(s->stream);
    cudaFree(*buf);
    *buf = d;
    *cap = c;
    return AMRGPU_OK;
}

// The state moves to the new mesh of nq quads (descriptors already in
// d_quads, remap kind / source in d_kind / d_src): into the spare buffer Y
// of the same capacity, or a fresh set when the mesh outgrew the capacity.
// fuse_cfl: the remap also folds the next segment's first CFL minimum
// (remap_cfl_kernel; s->d_quads must hold the new mesh's descriptors), so
// no separate CFL pass follows.
int apply_regrid(amrgpu_session *s, int nq, int nface, long long mixed_cells = -1, bool fuse_cfl = false)
{
    s->dev_forest = nullptr;  // the new mesh's leaves are the caller's to record
    const long long cells = mixed_cells >= 0 ? mixed_cells : (long long)nq * s->n * s->n;
    const long long stride = std::max<long long>(((cells + 31) / 32) * 32, 32);
    double *qold = rolebuf(s, RX);
    const long long old_stride = s->stride;
    double *fresh[4] = {nullptr, nullptr, nullptr, nullptr};
    long long cap = s->cap_stride;
    bool ok = true;
    if (stride > s->cap_stride) {
        // twice the need: large device allocations and frees cost
        // milliseconds each (tens on some hosts), so an adaptive run that
        // keeps growing should meet them rarely
        cap = ((2 * stride + 31) / 32) * 32;
        for (int k = 0; k < 4 && ok; ++k)
            ok = cuda_ok(cudaMalloc(&fresh[k], sizeof(double) * 4 * size_t(cap)), "cudaMalloc state");
        double *aos = nullptr;
        double *tot = nullptr;
        if (ok) ok = cuda_ok(cudaMalloc(&aos, sizeof(double) * 4 * size_t(cap)), "cudaMalloc aos");
        if (ok) ok = cuda_ok(cudaMalloc(&tot, sizeof(double) * 4 * size_t(totals_grid(cap))), "cudaMalloc totals");
        if (!ok) {
            for (double *p : fresh) cudaFree(p);
            cudaFree(aos);
            cudaFree(tot);
            return AMRGPU_ERR_CUDA;
        }
        cudaStreamSynchronize(s->stream);
        cudaFree(s->d_aos);
        cudaFree(s->d_tot);
        s->d_aos = aos;
        s->d_tot = tot;
    }
    double *qnew = fresh[0] ? fresh[0] : rolebuf(s, RY);
    const void *rcfl = nullptr;
    if (fuse_cfl && mixed_cells < 0 && nq > 0 && s->primed && s->cfg.time_scheme != 2)
        rcfl = s->form == AMRGPU_FORM_FP32_FLUX ? remap_cfl_kernel_fp32(s->n) : remap_cfl_kernel_fp64(s->n);
    if (rcfl) {
        // the slots re-armed (dt cap) first, as prime() does
        const int p = int(s->step_index % 3);
        ok = cuda_ok(launch_rearm(s->d_scal, p, s->cfg.dt, s->stream), "rearm scalars");
        s->launches++;
        RemapCflArgs ra;
        std::memset(&ra, 0, sizeof(ra));
        ra.qold = qold;
        ra.stride_old = old_stride;
        ra.qnew = qnew;
        ra.kind = s->d_kind;
        ra.src = s->d_src;
        ra.cfl.quads = s->d_quads;
        ra.cfl.scal = s->d_scal;
        ra.cfl.stride = stride;
        ra.cfl.nquad = nq;
        ra.cfl.slot = p;
        ra.cfl.cfl = s->cfg.cfl;
        const long long cells_new = (long long)nq * s->n * s->n;
        const int g = int(std::max(1ll, std::min<long long>((cells_new + 255) / 256, (long long)s->sms * 16)));
        void *args[] = {&ra};
        if (ok) ok = cuda_ok(cudaLaunchKernel(rcfl, dim3(g), dim3(256), args, 0, s->stream), "remap + CFL kernel");
        s->launches++;
    } else if (nq > 0) {
        if (mixed_cells >= 0)
            ok = cuda_ok(launch_remap_mixed(qold, old_stride, s->d_mix_old, qnew, stride, s->d_mix, s->d_kind, s->d_src,
                                            nq, s->stream),
                         "remap kernel");
        else
            ok = cuda_ok(launch_remap(s->n, qold, old_stride, qnew, stride, s->d_kind, s->d_src, nq, s->stream),
                         "remap kernel");
        s->launches++;
    }
    if (!ok) {
        for (double *p : fresh) cudaFree(p);
        return AMRGPU_ERR_CUDA;
    }
    if (fresh[0]) {
        cudaStreamSynchronize(s->stream);
        for (int k = 0; k < 4; ++k) {
            cudaFree(s->buf[k]);
            s->buf[k] = fresh[k];
            s->role[k] = k;
        }
        s->cap_stride = cap;
    } else {
        std::swap(s->role[RX], s->role[RY]);
    }
    s->nquad = nq;
    s->nghost = 0;
    s->nface = nface;
    s->dof = int(4 * cells);
    s->ncells_total = cells;
    s->stride = stride;
    // a launch chosen by the caller stays; the default follows the mesh size
    const bool keep = s->launch_pinned && s->launch && (s->launch->n == 0) == s->mixed;
    int rc = configure_launch(s, keep ? s->launch : session_default_launch(s));
    if (!s->launch_pinned) s->tune_pending = true;
    if (rc != AMRGPU_OK) return rc;
    if (rcfl) return AMRGPU_OK;  // re-armed and the CFL minimum folded already
    return prime(s, s->primed);
}

// A device buffer of at least `need` bytes (contents not kept; grown to twice
// the need, at least 1 MB, so that a fluctuating mesh reallocates rarely).
int ensure_dev(amrgpu_session *s, void **buf, size_t *bytes, size_t need)
{
    if (need <= *bytes && *buf) return AMRGPU_OK;
    cudaStreamSynchronize(s->stream);
    cudaFree(*buf);
    *buf = nullptr;
    *bytes = 0;
    const size_t want = std::max<size_t>(2 * need, size_t(1) << 20);
    if (!cuda_ok(cudaMalloc(buf, want), "cudaMalloc scratch")) return AMRGPU_ERR_CUDA;
    *bytes = want;
    return AMRGPU_OK;
}

// Pinned host staging of at least `bytes`; when the buffer is kept, waits
// for the copies still reading or writing it.
int ensure_stage(amrgpu_session *s, size_t bytes)
{
    if (bytes <= s->h_stage_bytes) return cuda_ok(cudaStreamSynchronize(s->stream), "sync") ? AMRGPU_OK : AMRGPU_ERR_CUDA;
    cudaStreamSynchronize(s->stream);
    cudaFreeHost(s->h_stage);
    s->h_stage = nullptr;
    s->h_stage_bytes = 0;
    // pinning host pages is slow: grow by 2x, at least 1 MB
    const size_t want = std::max<size_t>(2 * bytes, size_t(1) << 20);
    if (!cuda_ok(cudaHostAlloc(&s->h_stage, want, cudaHostAllocDefault), "cudaHostAlloc staging")) return AMRGPU_ERR_CUDA;
    s->h_stage_bytes = want;
    return AMRGPU_OK;
}

void set_brick(ForestDev &F, const BrickView &B, const int *bc)
{
    F.nx = B.nx;
    F.ny = B.ny;
    F.px = B.periodic[0];
    F.py = B.periodic[1];
    for (int k = 0; k < 3; ++k) F.xlo[k] = B.xlo[k];
    F.scale = B.scale;
    for (int k = 0; k < 4; ++k) F.bc[k] = bc ? bc[k] : 0;
}

// Descriptors of the device forest F (leaves, tree tables and key buffer on
// the device; remap table already queued into d_kind / d_src) into the spare
// descriptor buffer; on success it becomes the live one and the state is
// remapped. A 2:1 violation leaves the session as it was.
int build_and_apply(amrgpu_session *s, const ForestDev &F)
{
    const int nq = F.nq;
    int rc = ensure_desc(s, &s->d_quads_alt, &s->cap_desc_alt, nq);
    if (rc) return rc;
    const size_t scan_bytes = build_quads_scan_bytes(nq);
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t q4 = al(sizeof(int) * 4 * size_t(std::max(nq, 1)));
    const size_t o_emit = 0, o_scan = q4, o_emtr = 2 * q4, o_tmp = 3 * q4;
    const size_t o_stat = o_tmp + al(scan_bytes);
    rc = ensure_dev(s, &s->d_mesh_scratch, &s->mesh_scratch_bytes, o_stat + 256);  // status: 2 + 2 pad + 3 ints
    if (rc) return rc;
    char *base = static_cast<char *>(s->d_mesh_scratch);
    int *d_status = reinterpret_cast<int *>(base + o_stat);
    if (!cuda_ok(launch_build_quads(F, s->d_quads_alt, reinterpret_cast<int *>(base + o_emit),
                                    reinterpret_cast<int *>(base + o_scan), reinterpret_cast<int *>(base + o_emtr),
                                    base + o_tmp, scan_bytes, d_status, s->sms, s->stream),
                 "build quads"))
        return AMRGPU_ERR_CUDA;
    s->launches += nq > 0 ? 4 : 0;
    // mixed patch sizes by the session's level rule: sizes, offsets,
    // neighbour descriptors and the work list from the new descriptors
    int *d_mstat = d_status + 4;
    // once the mixed descriptor buffers are swapped, a failure puts the old
    // mesh's back: the session stays on the old mesh until apply_regrid
    bool swapped = false;
    auto fail = [&](int code) {
        if (swapped) mix_restore(s);
        return code;
    };
    if (s->has_rule) {
        if (!s->mixed && (rc = upload_uniform_mix(s))) return rc;
        rc = mix_buffers(s, nq, true);
        swapped = true;
        if (rc) return fail(rc);
        const size_t n1 = al(sizeof(int) * (size_t(nq) + 1));
        const size_t sb = build_mix_scan_bytes(nq);
        if ((rc = ensure_dev(s, &s->d_mix_scratch, &s->mix_scratch_bytes, 4 * n1 + al(sb)))) return fail(rc);
        char *mb = static_cast<char *>(s->d_mix_scratch);
        if (!cuda_ok(launch_build_mix(F.leaves, s->d_quads_alt, nq, s->rule, s->d_mix, s->d_work,
                                      reinterpret_cast<int *>(mb), reinterpret_cast<int *>(mb + n1),
                                      reinterpret_cast<int *>(mb + 2 * n1), reinterpret_cast<int *>(mb + 3 * n1),
                                      mb + 4 * n1, sb, d_mstat, s->stream),
                     "build mixed descriptors"))
            return fail(AMRGPU_ERR_CUDA);
        s->launches += 4;
    }
    int *status = reinterpret_cast<int *>(s->h_stage);  // staging is at least 64 bytes
    if (!cuda_ok(cudaMemcpyAsync(status, d_status, (s->has_rule ? 7 : 2) * sizeof(int), cudaMemcpyDeviceToHost,
                                 s->stream),
                 "D2H status") ||
        !cuda_ok(cudaStreamSynchronize(s->stream), "sync"))
        return fail(AMRGPU_ERR_CUDA);
    if (status[0]) {
        set_error(AMRGPU_ERR_MESH, "session regrid from a forest: the forest is not 2:1 balanced");
        return fail(AMRGPU_ERR_MESH);
    }
    if (s->has_rule && status[4]) {
        set_error(AMRGPU_ERR_MESH, "mixed patch sizes: the two fine quads of a hanging edge differ in size");
        return fail(AMRGPU_ERR_MESH);
    }
    const int nface = nq > 0 ? status[1] : 0;
    std::swap(s->d_quads, s->d_quads_alt);
    std::swap(s->cap_desc, s->cap_desc_alt);
    s->h_quads.clear();  // the live descriptors exist on the device only
    s->rect = true;      // brick quads are axis-aligned rectangles
    if (s->has_rule) {
        s->mixed = true;
        s->h_mix.clear();  // (device only, like the quad descriptors)
        s->h_work.clear();
        s->qn.clear();
        s->nwork16 = status[6];
        s->nwork8 = nq - status[6];
        return apply_regrid(s, nq, nface, (long long)status[5]);
    }
    return apply_regrid(s, nq, nface);
}

bool check_remap(const amrgpu_session *s, int nq, const int *kind, const int *src_index)
{
    for (int q = 0; q < nq; ++q) {
        const int lim = kind[q] == 0 ? s->nquad - 1 : s->nquad - 4;
        if ((kind[q] != 0 && kind[q] != 1) || src_index[q] < 0 || src_index[q] > lim) {
            set_error(AMRGPU_ERR_ARG, "remap kind or source index out of range");
            return false;
        }
    }
    return true;
}

}  // namespace

extern "C" {

int amrgpu_session_regrid(amrgpu_session_t *s, const amrgpu_mesh_t *m, const int *kind, const int *src_index)
{
    if (!s || !m || !kind || !src_index || !m->cell_info || !m->geom || (m->nface > 0 && !m->face_info) ||
        m->ncell < 0 || m->nghost < 0) {
        set_error(AMRGPU_ERR_ARG, "session_regrid: null or negative arguments");
        return AMRGPU_ERR_ARG;
    }
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_regrid: a step begun with step_stage is not finished");
        return AMRGPU_ERR_ARG;
    }
    if (m->nghost != 0) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "session_regrid: ghost quads need a ghost exchange after the remap");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    bool mixed_new = false;
    std::vector<int> qn_new;
    long long cells_new = 0;
    if (int e = mesh_sizes(m, s->n, mixed_new, qn_new, cells_new)) return e;
    // a mixed regrid (either mesh mixed) runs the mixed-size path from here
    // on; it needs the FP32-flux form and a launch the session chose
    const bool mixed_path = mixed_new || s->mixed;
    if (mixed_path && (s->form != AMRGPU_FORM_FP32_FLUX || (s->launch_pinned && !s->mixed))) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: the FP32-flux form with the library's launch only");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (!check_remap(s, m->ncell, kind, src_index)) return AMRGPU_ERR_ARG;
    if (mixed_path && !s->mixed) {
        if (int e = upload_uniform_mix(s)) return e;
    }
    std::vector<QuadDesc> old = std::move(s->h_quads);
    const bool was_mixed = s->mixed;
    s->mixed = mixed_path;
    int rc = decode_mesh(s, m);
    if (rc == AMRGPU_OK && s->form == AMRGPU_FORM_FP32_FLUX && !quads_are_rectangles(s)) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "the FP32-flux form needs axis-aligned rectangular quads");
        rc = AMRGPU_ERR_UNSUPPORTED;
    }
    if (rc != AMRGPU_OK) {
        s->h_quads = std::move(old);
        s->mixed = was_mixed;
        return rc;
    }
    const int nq = m->ncell;
    // buffers first (they only grow), so that nothing below fails after the
    // mixed descriptors are swapped except the copies
    rc = ensure_quad_arrays(s, nq);
    if (rc == AMRGPU_OK) rc = ensure_desc(s, &s->d_quads, &s->cap_desc, nq);
    if (rc != AMRGPU_OK) {
        s->h_quads = std::move(old);
        s->mixed = was_mixed;
        return rc;
    }
    if (mixed_path) {
        const int nq_old = s->nquad;
        s->nquad = nq;
        std::vector<int> qn_keep = std::move(s->qn);
        std::vector<MixDesc> mix_keep = std::move(s->h_mix);
        std::vector<int> work_keep = std::move(s->h_work);
        const int n16_keep = s->nwork16, n8_keep = s->nwork8;
        s->qn = std::move(qn_new);
        rc = build_mix(s, m);
        if (rc != AMRGPU_OK) {
            // the session stays on the old mesh
            s->qn = std::move(qn_keep);
            s->h_mix = std::move(mix_keep);
            s->h_work = std::move(work_keep);
            s->nwork16 = n16_keep;
            s->nwork8 = n8_keep;
            s->h_quads = std::move(old);
            s->mixed = was_mixed;
            s->nquad = nq_old;
            return rc;
        }
        rc = upload_mix(s, true);
        s->nquad = nq_old;  // apply_regrid moves the session to the new mesh
        if (rc != AMRGPU_OK) {
            mix_restore(s);
            s->qn = std::move(qn_keep);
            s->h_mix = std::move(mix_keep);
            s->h_work = std::move(work_keep);
            s->nwork16 = n16_keep;
            s->nwork8 = n8_keep;
            s->h_quads = std::move(old);
            s->mixed = was_mixed;
            return rc;
        }
    }
    bool ok = cuda_ok(cudaMemcpyAsync(s->d_kind, kind, sizeof(int) * size_t(nq), cudaMemcpyHostToDevice, s->stream),
                      "H2D remap") &&
              cuda_ok(cudaMemcpyAsync(s->d_src, src_index, sizeof(int) * size_t(nq), cudaMemcpyHostToDevice,
                                      s->stream),
                      "H2D remap");
    if (ok && nq > 0)
        ok = cuda_ok(cudaMemcpyAsync(s->d_quads, s->h_quads.data(), sizeof(QuadDesc) * size_t(nq),
                                     cudaMemcpyHostToDevice, s->stream),
                     "upload quads");
    if (!ok) return AMRGPU_ERR_CUDA;
    s->rect = (s->form != AMRGPU_FORM_FP32_FLUX) ? quads_are_rectangles(s) : true;
    return apply_regrid(s, nq, m->nface, mixed_path ? cells_new : -1);
}

int amrgpu_session_regrid_forest(amrgpu_session_t *s, const amrgpu_forest_t *f)
{
    if (!s || !f || !f->f) return AMRGPU_ERR_ARG;
    if (s->mixed && !s->has_rule) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: set a patch-size rule (amrgpu_session_set_patch_rule) "
                                          "or regrid through amrgpu_session_regrid");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_regrid_forest: a step begun with step_stage is not finished");
        return AMRGPU_ERR_ARG;
    }
    if (s->nghost != 0) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "session_regrid_forest: ghost quads need a ghost exchange after the remap");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    const std::vector<Leaf> &L = forest_leaves(f->f);
    BrickView B;
    forest_brick(f->f, &B);
    const int nq = int(L.size());
    const int ntrees = B.nx * B.ny;
    // pinned staging: leaves (int4), kind, src, tree_begin, tree_tx, tree_ty, tree_at
    const size_t n_int = 4 * size_t(nq) + 2 * size_t(nq) + size_t(ntrees + 1) + 3 * size_t(ntrees);
    const size_t stage_bytes = sizeof(int) * n_int;
    int rc = ensure_stage(s, stage_bytes);
    if (rc) return rc;
    int *hs = static_cast<int *>(s->h_stage);
    int *h_leaves = hs, *h_kind = hs + 4 * size_t(nq), *h_src = h_kind + nq, *h_tb = h_src + nq;
    int *h_tx = h_tb + ntrees + 1, *h_ty = h_tx + ntrees, *h_at = h_ty + ntrees;
    for (int t = 0; t <= ntrees; ++t) h_tb[t] = nq;
    for (int i = nq - 1; i >= 0; --i) {
        const Leaf &q = L[size_t(i)];
        h_leaves[4 * i + 0] = q.tree;
        h_leaves[4 * i + 1] = q.level;
        h_leaves[4 * i + 2] = int(q.x);
        h_leaves[4 * i + 3] = int(q.y);
        h_kind[i] = q.src_kind;
        h_src[i] = q.src;
        h_tb[q.tree] = i;
    }
    for (int t = ntrees - 1; t >= 0; --t) h_tb[t] = std::min(h_tb[t], h_tb[t + 1]);
    for (int t = 0; t < ntrees; ++t) {
        h_tx[t] = B.tree_tx[t];
        h_ty[t] = B.tree_ty[t];
        h_at[t] = B.tree_at[t];
    }
    if (!check_remap(s, nq, h_kind, h_src)) return AMRGPU_ERR_ARG;
    rc = ensure_quad_arrays(s, nq);
    if (rc) return rc;
    // device copy of the staged ints, then the leaves' Morton keys
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t o_keys = al(stage_bytes);
    rc = ensure_dev(s, &s->d_fstage, &s->fstage_bytes, o_keys + sizeof(unsigned long long) * size_t(std::max(nq, 1)));
    if (rc) return rc;
    char *base = static_cast<char *>(s->d_fstage);
    int *d_stage = reinterpret_cast<int *>(base);
    bool ok = cuda_ok(cudaMemcpyAsync(d_stage, hs, stage_bytes, cudaMemcpyHostToDevice, s->stream), "H2D forest") &&
              cuda_ok(cudaMemcpyAsync(s->d_kind, h_kind, sizeof(int) * size_t(nq), cudaMemcpyHostToDevice,
                                      s->stream),
                      "H2D remap") &&
              cuda_ok(cudaMemcpyAsync(s->d_src, h_src, sizeof(int) * size_t(nq), cudaMemcpyHostToDevice, s->stream),
                      "H2D remap");
    if (!ok) return AMRGPU_ERR_CUDA;
    ForestDev F;
    F.leaves = reinterpret_cast<const int4 *>(d_stage);
    F.keys = reinterpret_cast<unsigned long long *>(base + o_keys);
    F.tree_begin = d_stage + (h_tb - hs);
    F.tree_tx = d_stage + (h_tx - hs);
    F.tree_ty = d_stage + (h_ty - hs);
    F.tree_at = d_stage + (h_at - hs);
    set_brick(F, B, s->cfg.bc);
    F.nq = nq;
    return build_and_apply(s, F);
}

}  // extern "C"

namespace {

// Balance buffers for cap leaves: per buffer int4 leaves, int origin,
// uint8 dirty; work: flags (uint8), positions (cap + 1: the last is the
// total), keys, tree begin, brick tables, scan temp.
struct BalLayout {
    size_t o_orig, o_dirty, buf;
    size_t o_flags, o_pos, o_keys, o_tb, o_tx, o_ty, o_at, o_cell, o_tmp, o_dlist, work;
    size_t scan_bytes;
};

BalLayout bal_layout(int cap, int ntrees)
{
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    BalLayout L;
    const size_t c = size_t(std::max(cap, 1));
    L.o_orig = al(16 * c);
    L.o_dirty = L.o_orig + al(4 * c);
    L.buf = L.o_dirty + al(c);
    L.scan_bytes = balance_scan_bytes(int(c));
    L.o_flags = 0;
    L.o_pos = al(c);
    L.o_keys = L.o_pos + al(4 * (c + 1));
    L.o_tb = L.o_keys + al(8 * c);
    L.o_tx = L.o_tb + al(4 * size_t(ntrees + 1));
    L.o_ty = L.o_tx + al(4 * size_t(ntrees));
    L.o_at = L.o_ty + al(4 * size_t(ntrees));
    L.o_cell = L.o_at + al(4 * size_t(ntrees));
    // the one-launch balance's cell table, used for bricks of up to
    // kCellTabMaxTrees trees (sized monotonically in ntrees: a work area
    // allocated for more trees serves a forest with fewer)
    const size_t cell = 4 * size_t(std::min(ntrees, kCellTabMaxTrees)) * kCellTabCells;
    L.o_tmp = L.o_cell + al(cell);
    L.o_dlist = L.o_tmp + al(L.scan_bytes);
    L.work = L.o_dlist + al(4 * c);
    return L;
}

// Grows the balance buffers to cap leaves, keeping the first keep leaves of
// buffer `live` (leaves, origin, dirty). The buffers are laid out by the
// forest's tree count ntrees (bal_layout(cap, ntrees)); they are allocated
// for max(ntrees, bal_trees) trees, so that a reservation for more trees
// also serves a forest with fewer.
int bal_grow(amrgpu_session *s, int cap, int ntrees, int live, int keep)
{
    s->dev_forest = nullptr;
    const int alloc_trees = std::max(ntrees, s->bal_trees);
    const BalLayout A = bal_layout(cap, alloc_trees);
    const BalLayout L = bal_layout(cap, ntrees);
    const BalLayout O = bal_layout(s->bal_cap, ntrees);
    void *nb[2] = {nullptr, nullptr};
    void *nw = nullptr;
    bool ok = cuda_ok(cudaMalloc(&nb[0], A.buf), "cudaMalloc balance") &&
              cuda_ok(cudaMalloc(&nb[1], A.buf), "cudaMalloc balance") &&
              cuda_ok(cudaMalloc(&nw, A.work), "cudaMalloc balance");
    if (ok && keep > 0 && s->d_bal[live]) {
        char *src = static_cast<char *>(s->d_bal[live]);
        char *dst = static_cast<char *>(nb[0]);
        ok = cuda_ok(cudaMemcpyAsync(dst, src, 16 * size_t(keep), cudaMemcpyDeviceToDevice, s->stream), "balance copy") &&
             cuda_ok(cudaMemcpyAsync(dst + L.o_orig, src + O.o_orig, 4 * size_t(keep), cudaMemcpyDeviceToDevice,
                                     s->stream),
                     "balance copy") &&
             cuda_ok(cudaMemcpyAsync(dst + L.o_dirty, src + O.o_dirty, size_t(keep), cudaMemcpyDeviceToDevice,
                                     s->stream),
                     "balance copy");
        // brick tables live in the work area (same forest: same tree count)
        if (ok && s->d_bal_work && s->bal_trees >= ntrees)
            ok = cuda_ok(cudaMemcpyAsync(static_cast<char *>(nw) + L.o_tx, static_cast<char *>(s->d_bal_work) + O.o_tx,
                                         L.o_tmp - L.o_tx, cudaMemcpyDeviceToDevice, s->stream),
                         "balance copy");
    }
    if (ok) ok = cuda_ok(cudaStreamSynchronize(s->stream), "sync");
    if (!ok) {
        cudaFree(nb[0]);
        cudaFree(nb[1]);
        cudaFree(nw);
        return AMRGPU_ERR_CUDA;
    }
    cudaFree(s->d_bal[0]);
    cudaFree(s->d_bal[1]);
    cudaFree(s->d_bal_work);
    s->d_bal[0] = nb[0];
    s->d_bal[1] = nb[1];
    s->d_bal_work = nw;
    s->bal_cap = cap;
    s->bal_trees = alloc_trees;
    return AMRGPU_OK;
}

// Stages a forest's leaves for the device balance: leaves (int4), origin
// (identity), dirty marks, brick tables and, with remap, the pre-balance
// remap kind / source (range-checked against the session's quads) into
// d_remap0; grows the balance buffers to 1.5 times the leaves.
int stage_leaves(amrgpu_session *s, std::vector<Leaf> &leaves, const BrickView &B, int ntrees, bool remap)
{
    s->dev_forest = nullptr;
    const int nl = int(leaves.size());
    // staging: leaves (int4), origin, remap kind / source (with remap),
    // dirty bytes, brick tables
    const size_t nrm = remap ? 2 * size_t(nl) : 0;
    size_t sb = 16 * size_t(nl) + 4 * size_t(nl) + 4 * nrm + size_t(nl) + 12 * size_t(ntrees) + 64;
    int rc = ensure_stage(s, sb);
    if (rc) return rc;
    if (remap) {
        rc = ensure_dev(s, &s->d_remap0, &s->remap0_bytes, 4 * nrm + 16);
        if (rc) return rc;
    }
    {
        int *h = static_cast<int *>(s->h_stage);
        int *h_orig = h + 4 * size_t(nl);
        int *h_rm = h_orig + nl;  // kind[nl], source[nl]
        unsigned char *h_dirty = reinterpret_cast<unsigned char *>(h_rm + nrm);
        bool bad = false;
        for (int i = 0; i < nl; ++i) {
            const Leaf &q = leaves[size_t(i)];
            h[4 * i + 0] = q.tree;
            h[4 * i + 1] = q.level;
            h[4 * i + 2] = int(q.x);
            h[4 * i + 3] = int(q.y);
            h_orig[i] = i;
            h_dirty[i] = q.dirty ? 1 : 0;
            if (remap) {
                // balance children inherit these, so the pre-balance range
                // check covers the balanced table
                const int lim = q.src_kind == 0 ? s->nquad - 1 : s->nquad - 4;
                bad |= (q.src_kind != 0 && q.src_kind != 1) || q.src < 0 || q.src > lim;
                h_rm[i] = q.src_kind;
                h_rm[nl + i] = q.src;
            }
        }
        if (bad) {
            set_error(AMRGPU_ERR_ARG, "remap kind or source index out of range");
            return AMRGPU_ERR_ARG;
        }
        int *h_tab = reinterpret_cast<int *>(h_dirty + ((size_t(nl) + 15) & ~size_t(15)));
        for (int t = 0; t < ntrees; ++t) {
            h_tab[t] = B.tree_tx[t];
            h_tab[ntrees + t] = B.tree_ty[t];
            h_tab[2 * ntrees + t] = B.tree_at[t];
        }
        const int cap = std::max(nl + nl / 2, 64);  // passes that outgrow it grow it (2x)
        if (cap > s->bal_cap || ntrees > s->bal_trees) {
            rc = bal_grow(s, std::max(cap, s->bal_cap), ntrees, 0, 0);
            if (rc) return rc;
        }
        const BalLayout L = bal_layout(s->bal_cap, ntrees);
        char *b0 = static_cast<char *>(s->d_bal[0]);
        char *w = static_cast<char *>(s->d_bal_work);
        bool ok = cuda_ok(cudaMemcpyAsync(b0, h, 16 * size_t(nl), cudaMemcpyHostToDevice, s->stream), "H2D balance") &&
                  cuda_ok(cudaMemcpyAsync(b0 + L.o_orig, h_orig, 4 * size_t(nl), cudaMemcpyHostToDevice, s->stream),
                          "H2D balance") &&
                  cuda_ok(cudaMemcpyAsync(b0 + L.o_dirty, h_dirty, size_t(nl), cudaMemcpyHostToDevice, s->stream),
                          "H2D balance") &&
                  cuda_ok(cudaMemcpyAsync(w + L.o_tx, h_tab, 4 * size_t(ntrees), cudaMemcpyHostToDevice, s->stream),
                          "H2D balance") &&
                  cuda_ok(cudaMemcpyAsync(w + L.o_ty, h_tab + ntrees, 4 * size_t(ntrees), cudaMemcpyHostToDevice,
                                          s->stream),
                          "H2D balance") &&
                  cuda_ok(cudaMemcpyAsync(w + L.o_at, h_tab + 2 * ntrees, 4 * size_t(ntrees), cudaMemcpyHostToDevice,
                                          s->stream),
                          "H2D balance");
        if (ok && remap && nl > 0)
            ok = cuda_ok(cudaMemcpyAsync(s->d_remap0, h_rm, 4 * nrm, cudaMemcpyHostToDevice, s->stream), "H2D remap");
        if (!ok) return AMRGPU_ERR_CUDA;
    }
    return AMRGPU_OK;
}

// The balanced leaves (buffer `live`, nl of them) back into the host
// forest: coordinates and origin read back (leaves_back_enqueue, which
// records ev_tags when they have landed), then rewritten in place
// (leaves_back_finish, after waiting for that event). The device may go on
// with other work in between.
int leaves_back_enqueue(amrgpu_session *s, int nl, int live, int ntrees)
{
    int rc = ensure_stage(s, 20 * size_t(nl) + 64);
    if (rc) return rc;
    if (!s->ev_tags && !cuda_ok(cudaEventCreateWithFlags(&s->ev_tags, cudaEventDisableTiming), "event"))
        return AMRGPU_ERR_CUDA;
    const BalLayout L = bal_layout(s->bal_cap, ntrees);
    char *in = static_cast<char *>(s->d_bal[live]);
    int *h = static_cast<int *>(s->h_stage);
    int *h_orig = h + 4 * size_t(nl);
    if (nl > 0 &&
        (!cuda_ok(cudaMemcpyAsync(h, in, 16 * size_t(nl), cudaMemcpyDeviceToHost, s->stream), "D2H balance") ||
         !cuda_ok(cudaMemcpyAsync(h_orig, in + L.o_orig, 4 * size_t(nl), cudaMemcpyDeviceToHost, s->stream),
                  "D2H balance")))
        return AMRGPU_ERR_CUDA;
    return cuda_ok(cudaEventRecord(s->ev_tags, s->stream), "event") ? AMRGPU_OK : AMRGPU_ERR_CUDA;
}

int leaves_back_finish(amrgpu_session *s, Forest *fo, int nl)
{
    std::vector<Leaf> &leaves = forest_leaves_mut(fo);
    if (!cuda_ok(cudaEventSynchronize(s->ev_tags), "sync")) return AMRGPU_ERR_CUDA;
    const int *h = static_cast<const int *>(s->h_stage);
    const int *h_orig = h + 4 * size_t(nl);
    if (nl != int(leaves.size())) {
        // in place, from the end backwards: balance only refines, so leaf k
        // comes from input leaf h_orig[k] <= k (non-decreasing in k), which
        // is read before anything at or below it is overwritten; the prefix
        // of leaves the balance left alone is not touched. Field by field:
        // copying a whole leaf right after overwriting some of its fields
        // stalls on store forwarding.
        const int n0 = int(leaves.size());
        int first = 0;
        while (first < n0 && h_orig[first] == first && h[4 * first + 1] == leaves[size_t(first)].level)
            leaves[size_t(first++)].dirty = 0;
        forest_grow_leaves(fo, size_t(nl));
        for (int k = nl - 1; k >= first; --k) {
            const Leaf &p = leaves[size_t(h_orig[k])];
            Leaf &d = leaves[size_t(k)];
            d.tree = p.tree;
            d.tag = p.tag;
            d.type = p.type;
            d.src = p.src;
            d.src_kind = p.src_kind;
            d.level = h[4 * k + 1];
            d.x = h[4 * k + 2];
            d.y = h[4 * k + 3];
            d.dirty = 0;
        }
    } else {
        for (Leaf &q : leaves) q.dirty = 0;
    }
    return AMRGPU_OK;
}

int leaves_back_to_host(amrgpu_session *s, Forest *fo, int nl, int live, int ntrees)
{
    const int rc = leaves_back_enqueue(s, nl, live, ntrees);
    return rc ? rc : leaves_back_finish(s, fo, nl);
}

// 2:1 balance of forest fo with every pass on the session's GPU; the
// balanced leaves stay in d_bal[*live_out] (with the last pass's keys and
// tree starts in the work area) and are copied back into the host forest.
// With remap, the remap table of the balanced leaves (kind / source of the
// pre-balance leaf each one descends from, validated against the session's
// current quad count) is gathered into d_kind / d_src on the device.
// Returns the leaf count or -error.
int balance_impl(amrgpu_session *s, Forest *fo, int *live_out, bool remap)
{
    std::vector<Leaf> &leaves = forest_leaves_mut(fo);
    BrickView B;
    forest_brick(fo, &B);
    const int ntrees = B.nx * B.ny;
    int nl = int(leaves.size());
    int rc = stage_leaves(s, leaves, B, ntrees, remap);
    if (rc) return -rc;
    int live = 0;
    bool done = false, refined = false;
    for (int pass = 0; pass < 64 && !done; ++pass) {
        const BalLayout L = bal_layout(s->bal_cap, ntrees);
        char *in = static_cast<char *>(s->d_bal[live]);
        char *w = static_cast<char *>(s->d_bal_work);
        ForestDev F;
        F.leaves = reinterpret_cast<const int4 *>(in);
        F.keys = reinterpret_cast<unsigned long long *>(w + L.o_keys);
        F.tree_begin = reinterpret_cast<const int *>(w + L.o_tb);
        F.tree_tx = reinterpret_cast<const int *>(w + L.o_tx);
        F.tree_ty = reinterpret_cast<const int *>(w + L.o_ty);
        F.tree_at = reinterpret_cast<const int *>(w + L.o_at);
        F.nx = B.nx;
        F.ny = B.ny;
        F.px = B.periodic[0];
        F.py = B.periodic[1];
        for (int k = 0; k < 3; ++k) F.xlo[k] = B.xlo[k];
        F.scale = B.scale;
        for (int k = 0; k < 4; ++k) F.bc[k] = 0;
        F.nq = nl;
        unsigned char *flags = reinterpret_cast<unsigned char *>(w + L.o_flags);
        int *pos = reinterpret_cast<int *>(w + L.o_pos);
        if (!cuda_ok(launch_balance_pass(F, ntrees, reinterpret_cast<int *>(w + L.o_tb),
                                         reinterpret_cast<const unsigned char *>(in + L.o_dirty), flags, pos,
                                         w + L.o_tmp, L.scan_bytes, s->sms, s->stream),
                     "balance pass"))
            return -AMRGPU_ERR_CUDA;
        s->launches += 4;
        int total = 0;
        int *ht = static_cast<int *>(s->h_stage);  // staging is free: the uploads above have completed by now
        if (nl > 0) {
            if (!cuda_ok(cudaMemcpyAsync(ht, pos + nl, sizeof(int), cudaMemcpyDeviceToHost, s->stream), "D2H") ||
                !cuda_ok(cudaStreamSynchronize(s->stream), "sync"))
                return -AMRGPU_ERR_CUDA;
            total = ht[0];
        }
        if (total == nl) {
            done = true;
            break;
        }
        if (total > s->bal_cap) {
            rc = bal_grow(s, 2 * total, ntrees, live, nl);
            if (rc) return -rc;
            live = 0;
            // flags and positions were in the old work area: redo the pass
            continue;
        }
        const BalLayout L2 = bal_layout(s->bal_cap, ntrees);
        char *out = static_cast<char *>(s->d_bal[1 - live]);
        if (!cuda_ok(launch_balance_refine(nl, reinterpret_cast<const int4 *>(in),
                                           reinterpret_cast<const int *>(in + L2.o_orig), flags, pos,
                                           reinterpret_cast<int4 *>(out), reinterpret_cast<int *>(out + L2.o_orig),
                                           reinterpret_cast<unsigned char *>(out + L2.o_dirty), s->sms, s->stream),
                     "balance refine"))
            return -AMRGPU_ERR_CUDA;
        s->launches++;
        live = 1 - live;
        nl = total;
        refined = true;
    }
    if (!done) {
        set_error(AMRGPU_ERR_MESH, "forest_balance_device: no balance after 64 passes");
        return -AMRGPU_ERR_MESH;
    }
    *live_out = live;
    if (remap && nl > 0) {
        rc = ensure_quad_arrays(s, nl);
        if (rc) return -rc;
        const BalLayout L = bal_layout(s->bal_cap, ntrees);
        const int *rm = static_cast<const int *>(s->d_remap0);
        const int n0 = int(leaves.size());
        if (!cuda_ok(launch_remap_gather(nl, reinterpret_cast<const int *>(static_cast<char *>(s->d_bal[live]) + L.o_orig),
                                         rm, rm + n0, s->d_kind, s->d_src, s->sms, s->stream),
                     "remap gather"))
            return -AMRGPU_ERR_CUDA;
        s->launches++;
    }
    if (!refined) {
        for (Leaf &q : leaves) q.dirty = 0;
        return nl;
    }
    rc = leaves_back_to_host(s, fo, nl, live, ntrees);
    return rc ? -rc : nl;
}

// The whole regrid of an adapted forest with the balance passes, the quad
// descriptors of the balanced leaves and their remap table in one
// cooperative launch (launch_balance_loop) and one read-back; the balanced
// leaves go back to the host forest, then the state is remapped as by
// build_and_apply. Sessions with a patch-size rule take balance_impl and
// build_and_apply instead (the mixed build needs the leaf count first).
// The balance, descriptors and remap table in one cooperative launch (plus
// read-backs), then the remap. Staged: the host forest's leaves go to the
// device first. With ad (device adapt): the loop starts from the leaves the
// balance buffers still hold for this forest (dev_live), refines / coarsens
// them by ad's tags on the device, and host_work (the host forest's own
// adapt, which must reach the same leaves) runs while the launch does.
int balance_regrid_fused(amrgpu_session *s, Forest *fo, bool stall_test = false, AdaptArgs *ad = nullptr,
                         const std::function<int()> &host_work = {})
{
    BrickView B;
    forest_brick(fo, &B);
    const int ntrees = B.nx * B.ny;
    int rc;
    int n0 = s->nquad, live = 0;
    if (ad) {
        live = s->dev_live;
        // the adapted leaves' remap table, kind then source, at a split
        // fixed for this regrid (a later growth of the leaf buffers keeps
        // d_remap0)
        if ((rc = ensure_dev(s, &s->d_remap0, &s->remap0_bytes, 8 * size_t(s->bal_cap) + 16))) return rc;
        ad->kind = static_cast<int *>(s->d_remap0);
        ad->src = ad->kind + s->bal_cap;
    } else {
        std::vector<Leaf> &leaves = forest_leaves_mut(fo);
        n0 = int(leaves.size());
        if ((rc = stage_leaves(s, leaves, B, ntrees, true))) return rc;
    }
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    int nl = n0;
    bool adapt_pending = ad != nullptr, host_done = !host_work;
    int adapted = -1;
    BalanceCtl ctl{};
    int status[2] = {0, 0};
    for (int attempt = 0;; ++attempt) {
        const int cap = s->bal_cap;
        if ((rc = ensure_desc(s, &s->d_quads_alt, &s->cap_desc_alt, cap))) return rc;
        if ((rc = ensure_quad_arrays(s, cap))) return rc;
        if (ad) ad->tags = s->d_tags;  // kept by a growth of the quad arrays
        const size_t n4 = al(sizeof(int) * (4 * size_t(cap) + 1));
        const size_t o_emits = 0, o_scan = n4, o_emitter = 2 * n4, o_status = 3 * n4;
        const size_t o_bsum = o_status + 256, o_ctl = o_bsum + al(sizeof(int) * balance_loop_bsum_ints(s->sms));
        if ((rc = ensure_dev(s, &s->d_mesh_scratch, &s->mesh_scratch_bytes, o_ctl + al(sizeof(BalanceCtl)))))
            return rc;
        char *base = static_cast<char *>(s->d_mesh_scratch);
        const BalLayout L = bal_layout(cap, ntrees);
        char *w = static_cast<char *>(s->d_bal_work);
        BalanceLoopArgs a{};
        set_brick(a.F, B, s->cfg.bc);
        a.F.keys = reinterpret_cast<unsigned long long *>(w + L.o_keys);
        a.F.tree_begin = reinterpret_cast<const int *>(w + L.o_tb);
        a.F.tree_tx = reinterpret_cast<const int *>(w + L.o_tx);
        a.F.tree_ty = reinterpret_cast<const int *>(w + L.o_ty);
        a.F.tree_at = reinterpret_cast<const int *>(w + L.o_at);
        if (ntrees <= kCellTabMaxTrees) a.F.cell_tab = reinterpret_cast<int *>(w + L.o_cell);
        a.ntrees = ntrees;
        a.tree_begin = reinterpret_cast<int *>(w + L.o_tb);
        for (int k = 0; k < 2; ++k) {
            char *b = static_cast<char *>(s->d_bal[k]);
            a.leaves[k] = reinterpret_cast<int4 *>(b);
            a.orig[k] = reinterpret_cast<int *>(b + L.o_orig);
            a.dirty[k] = reinterpret_cast<unsigned char *>(b + L.o_dirty);
        }
        a.nl = nl;
        a.live = live;
        a.cap = cap;
        a.flags = reinterpret_cast<unsigned char *>(w + L.o_flags);
        a.pos = reinterpret_cast<int *>(w + L.o_pos);
        a.dirty_list = reinterpret_cast<int *>(w + L.o_dlist);
        a.bsum = reinterpret_cast<int *>(base + o_bsum);
        a.ctl = reinterpret_cast<BalanceCtl *>(base + o_ctl);
        a.build = 1;
        a.out = s->d_quads_alt;
        a.emits = reinterpret_cast<int *>(base + o_emits);
        a.scan = reinterpret_cast<int *>(base + o_scan);
        a.emitter = reinterpret_cast<int *>(base + o_emitter);
        a.status = reinterpret_cast<int *>(base + o_status);
        if (ad) {
            a.adapt = adapt_pending ? 1 : 0;
            a.ad = *ad;
        } else {
            const int *rm = static_cast<const int *>(s->d_remap0);
            a.kind0 = rm;
            a.src0 = rm + n0;
        }
        a.kind = s->d_kind;
        a.src = s->d_src;
        a.stall_test = stall_test ? 1 : 0;
        if (!cuda_ok(launch_balance_loop(a, s->sms, s->stream), "balance loop")) return AMRGPU_ERR_CUDA;
        s->launches++;
        // the staged leaves were read by the uploads before the launch: the
        // staging takes the results
        char *h = static_cast<char *>(s->h_stage);
        if (!cuda_ok(cudaMemcpyAsync(h, a.ctl, sizeof(BalanceCtl), cudaMemcpyDeviceToHost, s->stream), "D2H") ||
            !cuda_ok(cudaMemcpyAsync(h + 256, a.status, sizeof(status), cudaMemcpyDeviceToHost, s->stream), "D2H"))
            return AMRGPU_ERR_CUDA;
        if (!host_done) {
            host_done = true;
            if ((rc = host_work())) {
                cudaStreamSynchronize(s->stream);
                return rc;
            }
        }
        if (!cuda_ok(cudaStreamSynchronize(s->stream), "sync")) return AMRGPU_ERR_CUDA;
        std::memcpy(&ctl, h, sizeof(ctl));
        std::memcpy(status, h + 256, sizeof(status));
        if (adapt_pending && ctl.adapted > 0) {
            adapt_pending = false;
            adapted = ctl.adapted;
        }
        if (ctl.result == kBalanceOverflow && attempt < 16) {
            // more leaves than the buffers hold: grow (keeping the live
            // leaves, their origin and dirty marks) and go on from there;
            // an adapt that did not fit runs again from its own leaves
            const int need = adapt_pending ? ctl.adapt_total + ctl.adapt_total / 2 : 0;
            if ((rc = bal_grow(s, std::max(2 * s->bal_cap, need), ntrees, ctl.live, ctl.nl))) return rc;
            if (adapt_pending) {
                if ((rc = ensure_dev(s, &s->d_remap0, &s->remap0_bytes, 8 * size_t(s->bal_cap) + 16))) return rc;
                ad->kind = static_cast<int *>(s->d_remap0);
                ad->src = ad->kind + s->bal_cap;
            }
            nl = ctl.nl;
            live = 0;
            continue;
        }
        break;
    }
    if (ctl.result == kBalanceTimeout) {
        set_error(AMRGPU_ERR_CUDA, "balance loop: a device-wide barrier wait ran out");
        return AMRGPU_ERR_CUDA;
    }
    if (ctl.result != kBalanceDone) {
        set_error(AMRGPU_ERR_MESH, "forest_balance_device: no balance after 64 passes");
        return AMRGPU_ERR_MESH;
    }
    nl = ctl.nl;
    if (status[0]) {
        set_error(AMRGPU_ERR_MESH, "session regrid from a forest: the forest is not 2:1 balanced");
        return AMRGPU_ERR_MESH;
    }
    std::vector<Leaf> &leaves = forest_leaves_mut(fo);
    if (ad && adapted != int(leaves.size())) {
        set_error(AMRGPU_ERR_MESH, "device adapt: the leaves differ from the host forest's adapt");
        return AMRGPU_ERR_MESH;
    }
    // the balanced leaves' copy back is queued before the remap and the
    // next step's CFL minimum; the host forest is rebuilt while they run
    if (ctl.refined && (rc = leaves_back_enqueue(s, nl, ctl.live, ntrees))) return rc;
    std::swap(s->d_quads, s->d_quads_alt);
    std::swap(s->cap_desc, s->cap_desc_alt);
    s->h_quads.clear();  // the live descriptors exist on the device only
    s->rect = true;      // brick quads are axis-aligned rectangles
    if ((rc = apply_regrid(s, nl, nl > 0 ? status[1] : 0, -1, true))) return rc;
    if (ctl.refined) {
        if ((rc = leaves_back_finish(s, fo, nl))) return rc;
    } else {
        for (Leaf &q : leaves) q.dirty = 0;
    }
    // the balance buffers hold this forest's leaves: the next regrid of it
    // can adapt them on the device
    s->dev_forest = fo;
    s->dev_forest_version = forest_version(fo);
    s->dev_live = ctl.live;
    return AMRGPU_OK;
}

}  // namespace

extern "C" {

int amrgpu_forest_balance_device(amrgpu_forest_t *f, amrgpu_session_t *s)
{
    if (!f || !f->f || !s) return -AMRGPU_ERR_ARG;

    int live = 0;
    return balance_impl(s, f->f, &live, false);
}

int amrgpu_session_balance_regrid(amrgpu_session_t *s, amrgpu_forest_t *f)
{
    if (!s || !f || !f->f) return AMRGPU_ERR_ARG;
    if (s->mixed && !s->has_rule) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: set a patch-size rule (amrgpu_session_set_patch_rule) "
                                          "or regrid through amrgpu_session_regrid");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_balance_regrid: a step begun with step_stage is not finished");
        return AMRGPU_ERR_ARG;
    }
    if (s->nghost != 0) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "session_balance_regrid: ghost quads need a ghost exchange after the remap");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    // one cooperative launch for the balance, the descriptors and the remap
    // table, unless a patch-size rule needs the mixed build on the way
    static const bool fused = [] {
        const char *e = std::getenv("AMRGPU_FUSED_BALANCE");
        return !(e && std::atoi(e) == 0);
    }();
    if (fused && !s->has_rule) return balance_regrid_fused(s, f->f);
    int live = 0;
    const int nq = balance_impl(s, f->f, &live, true);  // remap table into d_kind / d_src
    if (nq < 0) return -nq;
    BrickView B;
    forest_brick(f->f, &B);
    const int ntrees = B.nx * B.ny;
    // the descriptors straight from the balanced leaves on the device
    const BalLayout BL = bal_layout(s->bal_cap, ntrees);
    char *in = static_cast<char *>(s->d_bal[live]);
    char *w = static_cast<char *>(s->d_bal_work);
    ForestDev F;
    F.leaves = reinterpret_cast<const int4 *>(in);
    F.keys = reinterpret_cast<unsigned long long *>(w + BL.o_keys);
    F.tree_begin = reinterpret_cast<const int *>(w + BL.o_tb);
    F.tree_tx = reinterpret_cast<const int *>(w + BL.o_tx);
    F.tree_ty = reinterpret_cast<const int *>(w + BL.o_ty);
    F.tree_at = reinterpret_cast<const int *>(w + BL.o_at);
    set_brick(F, B, s->cfg.bc);
    F.nq = nq;
    return build_and_apply(s, F);
}

int amrgpu_session_adapt_regrid(amrgpu_session_t *s, amrgpu_forest_t *f, const int *tags, int *tags_out,
                                int refine_value, int coarsen_value, int min_level, int max_level)
{
    if (!s || !f || !f->f) return AMRGPU_ERR_ARG;
    Forest *fo = f->f;
    const int nq = s->nquad;
    if (forest_num_quads(fo) != nq) {
        set_error(AMRGPU_ERR_ARG, "session_adapt_regrid: the forest's quads are not the session's mesh");
        return AMRGPU_ERR_ARG;
    }
    if (s->mixed && !s->has_rule) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: set a patch-size rule (amrgpu_session_set_patch_rule) "
                                          "or regrid through amrgpu_session_regrid");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_adapt_regrid: a step begun with step_stage is not finished");
        return AMRGPU_ERR_ARG;
    }
    if (s->nghost != 0) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "session_adapt_regrid: ghost quads need a ghost exchange after the remap");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    static const bool fused = [] {
        const char *e = std::getenv("AMRGPU_FUSED_BALANCE");
        return !(e && std::atoi(e) == 0);
    }();
    const bool device = fused && !s->has_rule && nq > 0 && s->dev_forest == fo &&
                        s->dev_forest_version == forest_version(fo);
    // the tags on the device (the tag kernel, or the caller's) and on the
    // host (copied back while the device goes on), in the staging after
    // the balance's read-back slots
    int rc = ensure_quad_arrays(s, std::max(nq, s->bal_cap));
    if (!rc) rc = ensure_stage(s, 512 + sizeof(int) * size_t(nq));
    if (rc) return rc;
    if (!s->ev_tags && !cuda_ok(cudaEventCreateWithFlags(&s->ev_tags, cudaEventDisableTiming), "event"))
        return AMRGPU_ERR_CUDA;
    int *h_tags = reinterpret_cast<int *>(static_cast<char *>(s->h_stage) + 512);
    if (nq > 0) {
        bool ok;
        if (tags) {
            std::memcpy(h_tags, tags, sizeof(int) * size_t(nq));
            ok = cuda_ok(cudaMemcpyAsync(s->d_tags, h_tags, sizeof(int) * size_t(nq), cudaMemcpyHostToDevice,
                                         s->stream),
                         "H2D tags");
        } else {
            ok = launch_tags(s) && cuda_ok(cudaMemcpyAsync(h_tags, s->d_tags, sizeof(int) * size_t(nq),
                                                           cudaMemcpyDeviceToHost, s->stream),
                                           "D2H tags");
        }
        if (!ok || !cuda_ok(cudaEventRecord(s->ev_tags, s->stream), "event")) return AMRGPU_ERR_CUDA;
    }
    // the host forest's own adapt, with the tags as they arrive
    auto host_adapt = [&]() -> int {
        if (nq > 0 && !tags && !cuda_ok(cudaEventSynchronize(s->ev_tags), "sync")) return AMRGPU_ERR_CUDA;
        if (tags_out && nq > 0) std::memcpy(tags_out, h_tags, sizeof(int) * size_t(nq));
        forest_adapt(fo, h_tags, refine_value, coarsen_value, min_level, max_level);
        return AMRGPU_OK;
    };
    if (!device) {
        if ((rc = host_adapt())) return rc;
        return amrgpu_session_balance_regrid(s, f);
    }
    AdaptArgs ad{};
    ad.tags = s->d_tags;
    ad.refine_value = refine_value;
    ad.coarsen_value = coarsen_value;
    ad.min_level = min_level;
    ad.max_level = max_level;
    return balance_regrid_fused(s, fo, false, &ad, host_adapt);
}

int amrgpu_session_holds_forest(const amrgpu_session_t *s, const amrgpu_forest_t *f)
{
    if (!s || !f || !f->f) return 0;
    return s->dev_forest == f->f && s->dev_forest_version == forest_version(f->f) ? 1 : 0;
}

int amrgpu_session_reserve(amrgpu_session_t *s, long long cells, int quads)
{
    if (!s || cells < 0 || quads < 0) {
        set_error(AMRGPU_ERR_ARG, "session_reserve: null session or negative size");
        return AMRGPU_ERR_ARG;
    }
    if (s->stage_pos != 0) {
        set_error(AMRGPU_ERR_ARG, "session_reserve: a step begun with step_stage is not finished");
        return AMRGPU_ERR_ARG;
    }
    // buffers may move: captured step graphs hold their addresses
    if (!cuda_ok(cudaStreamSynchronize(s->stream), "sync")) return AMRGPU_ERR_CUDA;
    for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    // a device buffer grown to want elements, its first keep elements kept
    auto grow_keep = [&](void **p, int *cap, size_t elem, int keep, int want) -> bool {
        if (want <= *cap && *p) return true;
        void *d = nullptr;
        if (!cuda_ok(cudaMalloc(&d, elem * size_t(std::max(want, 1))), "cudaMalloc reserve")) return false;
        if (keep > 0 && *p &&
            !cuda_ok(cudaMemcpyAsync(d, *p, elem * size_t(keep), cudaMemcpyDeviceToDevice, s->stream), "reserve copy")) {
            cudaFree(d);
            return false;
        }
        if (!cuda_ok(cudaStreamSynchronize(s->stream), "sync")) {
            cudaFree(d);
            return false;
        }
        cudaFree(*p);
        *p = d;
        *cap = std::max(want, 1);
        return true;
    };
    // the state: four role buffers (their contents kept, field f of cell c
    // stays at [f * stride + c]), the AoS staging and the totals partials
    const long long need = ((std::max<long long>(cells, 1) + 31) / 32) * 32;
    if (need > s->cap_stride) {
        double *fresh[4] = {nullptr, nullptr, nullptr, nullptr};
        double *aos = nullptr, *tot = nullptr;
        const size_t bytes = sizeof(double) * 4 * size_t(need);
        bool ok = true;
        for (int k = 0; k < 4 && ok; ++k) ok = cuda_ok(cudaMalloc(&fresh[k], bytes), "cudaMalloc reserve state");
        if (ok) ok = cuda_ok(cudaMalloc(&aos, bytes), "cudaMalloc reserve aos");
        if (ok) ok = cuda_ok(cudaMalloc(&tot, sizeof(double) * 4 * size_t(totals_grid(need))), "cudaMalloc reserve totals");
        for (int k = 0; k < 4 && ok; ++k)
            ok = cuda_ok(cudaMemcpyAsync(fresh[k], s->buf[k], sizeof(double) * 4 * size_t(s->stride),
                                         cudaMemcpyDeviceToDevice, s->stream),
                         "reserve copy");
        if (ok) ok = cuda_ok(cudaStreamSynchronize(s->stream), "sync");
        if (!ok) {
            for (double *p : fresh) cudaFree(p);
            cudaFree(aos);
            cudaFree(tot);
            return AMRGPU_ERR_CUDA;
        }
        for (int k = 0; k < 4; ++k) {
            cudaFree(s->buf[k]);
            s->buf[k] = fresh[k];
        }
        cudaFree(s->d_aos);
        cudaFree(s->d_tot);
        s->d_aos = aos;
        s->d_tot = tot;
        s->cap_stride = need;
    }
    if (quads == 0) return AMRGPU_OK;
    // per-quad tables: tags / remap, the live descriptors (kept) and the
    // build target of the next regrid
    int rc = ensure_quad_arrays(s, quads);
    if (rc) return rc;
    if (!grow_keep(reinterpret_cast<void **>(&s->d_quads), &s->cap_desc, sizeof(QuadDesc), s->nquad, quads))
        return AMRGPU_ERR_CUDA;
    if (!grow_keep(reinterpret_cast<void **>(&s->d_quads_alt), &s->cap_desc_alt, sizeof(QuadDesc), 0, quads))
        return AMRGPU_ERR_CUDA;
    // mixed patch sizes: the live sizes / work list (kept) and the spare pair
    if (s->mixed || s->has_rule) {
        const int keep = s->mixed ? s->nquad : 0;
        if (!grow_keep(reinterpret_cast<void **>(&s->d_mix), &s->cap_mix, sizeof(MixDesc), keep, quads) ||
            !grow_keep(reinterpret_cast<void **>(&s->d_work), &s->cap_work, sizeof(int), keep, quads) ||
            !grow_keep(reinterpret_cast<void **>(&s->d_mix_old), &s->cap_mix_old, sizeof(MixDesc), 0, quads) ||
            !grow_keep(reinterpret_cast<void **>(&s->d_work_old), &s->cap_work_old, sizeof(int), 0, quads))
            return AMRGPU_ERR_CUDA;
        const size_t n1 = al(sizeof(int) * (size_t(quads) + 1));
        if ((rc = ensure_dev(s, &s->d_mix_scratch, &s->mix_scratch_bytes, 4 * n1 + al(build_mix_scan_bytes(quads)))))
            return rc;
    }
    // descriptor build scratch (as build_and_apply lays it out)
    const size_t q4 = al(sizeof(int) * 4 * size_t(quads));
    if ((rc = ensure_dev(s, &s->d_mesh_scratch, &s->mesh_scratch_bytes,
                         3 * q4 + al(build_quads_scan_bytes(quads)) + 256)))
        return rc;
    // balance: pre-balance remap table, leaf buffers for the passes (the
    // balance sizes them at 1.5 times the leaves), tables for up to 64
    // trees, pinned staging of the leaves
    if ((rc = ensure_dev(s, &s->d_remap0, &s->remap0_bytes, 8 * size_t(quads) + 16))) return rc;
    const int bcap = std::max(quads + quads / 2, 64);
    const int btrees = std::max(s->bal_trees, 64);
    if (bcap > s->bal_cap || btrees > s->bal_trees) {
        if ((rc = bal_grow(s, std::max(bcap, s->bal_cap), btrees, 0, 0))) return rc;
    }
    return ensure_stage(s, 32 * size_t(bcap) + 12 * size_t(btrees) + 4096);
}

int amrgpu_session_balance_stall_test(amrgpu_session_t *s, amrgpu_forest_t *f)
{
    if (!s || !f || !f->f || s->has_rule || s->stage_pos != 0 || s->nghost != 0) return AMRGPU_ERR_ARG;
    return balance_regrid_fused(s, f->f, true);
}

int amrgpu_session_quad_descriptors(amrgpu_session_t *s, void *out, int cap)
{
    if (!s || (cap > 0 && !out) || cap < 0) return -AMRGPU_ERR_ARG;
    const int n = std::min(cap, s->nquad);
    if (n > 0 && (!cuda_ok(cudaMemcpyAsync(out, s->d_quads, sizeof(QuadDesc) * size_t(n), cudaMemcpyDeviceToHost,
                                           s->stream),
                           "D2H quads") ||
                  !cuda_ok(cudaStreamSynchronize(s->stream), "sync")))
        return -AMRGPU_ERR_CUDA;
    return s->nquad;
}

int amrgpu_session_face_count(const amrgpu_session_t *s) { return s ? s->nface : -1; }

}  // extern "C"

// ======================================================================
// The reference's evolve entry points
// ======================================================================
// The reference's configuration globals (physics_var_interface.h:20-39,
// physics_var_physics.h:21-49, physics_var_simulation.h:20-37), declared
// weak: when the reference's physics layer is built with -D_GPU_ and linked
// against this library, they resolve to its definitions (filled by its own
// hpc_amr_initialize_solver -> physics_initialize); otherwise they stay
// unresolved (null address). Layouts are the reference's, field for field.
extern "C" {
struct RefPhysicsInterface {
    int dim, nfringe, nfields, nelem_subgrid;
    int extern_cell_size, extern_face_size, extern_edge_size, extern_node_size, extern_mpi_comm_size;
    int nlevels;
    double coarse_grid_h;
};
struct RefPhysicsFluid {
    int initial_condition;
    int bc[6];
    int amr_ntag_methods;
    int *amr_tag_methods;
    double *amr_tag_tolerances;
    double cfl, mach, alpha, beta, gamma, density, pressure;
};
struct RefPhysicsSimulation {
    int checkpoint_interval, visualization_interval, regrid_interval;
    int time_scheme, time_steps;
    double dt;
};
extern RefPhysicsInterface d_physics_interface __attribute__((weak));
extern RefPhysicsFluid d_physics_fluid __attribute__((weak));
extern RefPhysicsSimulation d_physics_simulation __attribute__((weak));
}
static_assert(sizeof(RefPhysicsInterface) == 48, "physics_interface_t layout");
static_assert(sizeof(RefPhysicsFluid) == 104, "physics_fluid_t layout");
static_assert(sizeof(RefPhysicsSimulation) == 32, "physics_simulation_t layout");

namespace {

// The reference's physics layer is in this process and its
// physics_initialize has run (it stores nfields from the driver, > 0).
bool reference_config_present()
{
    return &d_physics_interface != nullptr && &d_physics_fluid != nullptr && &d_physics_simulation != nullptr &&
           d_physics_interface.nfields > 0;
}

// PhysicsConfig from the reference's globals; the extensions this library
// adds (form, final time, NaN abort, IC parameters) come from its own
// configuration.
PhysicsConfig config_from_reference()
{
    PhysicsConfig c = global_config();
    const RefPhysicsInterface &I = d_physics_interface;
    const RefPhysicsFluid &F = d_physics_fluid;
    const RefPhysicsSimulation &S = d_physics_simulation;
    c.dim = I.dim;
    c.nfringe = I.nfringe;
    c.nfields = I.nfields;
    c.nelem_subgrid = I.nelem_subgrid;
    c.extern_cell_size = I.extern_cell_size;
    c.extern_face_size = I.extern_face_size;
    c.extern_mpi_comm_size = I.extern_mpi_comm_size;
    c.nlevels = I.nlevels;
    c.coarse_grid_h = I.coarse_grid_h;
    c.initial_condition = F.initial_condition;
    for (int k = 0; k < 6; ++k) c.bc[k] = F.bc[k];
    c.amr_ntag_methods = F.amr_ntag_methods;
    c.amr_tag_methods.clear();
    c.amr_tag_tolerances.clear();
    for (int k = 0; k < F.amr_ntag_methods && F.amr_tag_methods && F.amr_tag_tolerances; ++k) {
        c.amr_tag_methods.push_back(F.amr_tag_methods[k]);
        c.amr_tag_tolerances.push_back(F.amr_tag_tolerances[k]);
    }
    c.cfl = F.cfl;  // already 0.25*cfl*time_scheme (physics_initialize.c)
    c.mach = F.mach;
    c.alpha = F.alpha;
    c.beta = F.beta;
    c.gamma = F.gamma;
    c.density = F.density;
    c.pressure = F.pressure;
    auto interval = [](int v) { return v > 0 ? v : 2147483647; };
    c.checkpoint_interval = interval(S.checkpoint_interval);
    c.visualization_interval = interval(S.visualization_interval);
    c.regrid_interval = interval(S.regrid_interval);
    c.time_scheme = S.time_scheme;
    c.time_steps = S.time_steps;
    c.dt = S.dt;
    return c;
}

// The configuration an evolve call runs with. physics_go_gpu is called by
// the reference's physics layer (physics_evolve_interface.c:42-46), so the
// reference's globals come first there; hpc_amr_evolve_solver replaces that
// layer, so this library's own configuration comes first. Either falls back
// to the other; with neither initialised the call is refused.
bool resolve_config(bool from_reference_layer, PhysicsConfig &out)
{
    const bool ref = reference_config_present();
    const bool own = config_initialized();
    if (from_reference_layer ? ref : (ref && !own)) {
        out = config_from_reference();
        return true;
    }
    if (own) {
        out = global_config();
        return true;
    }
    set_error(AMRGPU_ERR_CONFIG,
              "no configuration: neither this library's hpc_amr_initialize_solver / amrgpu_config_set nor the "
              "reference's physics_initialize has run");
    return false;
}

// The caller's MPI operations (amrgpu_set_comm_ops), process-wide.
std::mutex g_comm_mu;
amrgpu_comm_ops_t g_comm_ops{};
bool g_comm_set = false;

bool comm_ops(amrgpu_comm_ops_t &out)
{
    std::lock_guard<std::mutex> lk(g_comm_mu);
    if (g_comm_set) out = g_comm_ops;
    return g_comm_set;
}

// Ghost-exchange buffers of a multi-rank evolve session: the send-list
// records and the ghost records on the device and in pinned host memory,
// plus a pinned word for the CFL step's cross-rank MIN.
struct HaloBuffers {
    double *d_send = nullptr, *d_recv = nullptr, *h_send = nullptr, *h_recv = nullptr;
    unsigned long long *h_dt = nullptr;
    size_t send_cap = 0, recv_cap = 0;

    void release()
    {
        cudaFree(d_send);
        cudaFree(d_recv);
        cudaFreeHost(h_send);
        cudaFreeHost(h_recv);
        cudaFreeHost(h_dt);
        *this = HaloBuffers{};
    }
    bool reserve(size_t nsend_doubles, size_t nrecv_doubles)
    {
        if (!h_dt && !cuda_ok(cudaMallocHost(&h_dt, sizeof(unsigned long long)), "pinned dt word")) return false;
        if (nsend_doubles > send_cap) {
            cudaFree(d_send);
            cudaFreeHost(h_send);
            d_send = h_send = nullptr;
            send_cap = 0;
            if (!cuda_ok(cudaMalloc(&d_send, sizeof(double) * nsend_doubles), "halo send buffer") ||
                !cuda_ok(cudaMallocHost(&h_send, sizeof(double) * nsend_doubles), "pinned halo send buffer"))
                return false;
            send_cap = nsend_doubles;
        }
        if (nrecv_doubles > recv_cap) {
            cudaFree(d_recv);
            cudaFreeHost(h_recv);
            d_recv = h_recv = nullptr;
            recv_cap = 0;
            if (!cuda_ok(cudaMalloc(&d_recv, sizeof(double) * nrecv_doubles), "halo receive buffer") ||
                !cuda_ok(cudaMallocHost(&h_recv, sizeof(double) * nrecv_doubles), "pinned halo receive buffer"))
                return false;
            recv_cap = nrecv_doubles;
        }
        return true;
    }
};

struct EvolveCache {
    amrgpu_session *s = nullptr;
    // the mesh the session was built from, kept to compare byte for byte
    std::vector<int> cell_info, face_info;
    std::vector<double> geom;
    std::vector<int> send, recv;  // the rank's (quad, peer) lists
    int ncell = -1, nghost = -1, nface = -1, dof = -1;
    uint64_t cfg_hash = 0;
    double sim_time = 0.0;
    int end_istep = -1;  // *istep at the end of the last call
    HaloBuffers halo;

    ~EvolveCache()
    {
        // at thread exit (ranks run as threads) or process exit; CUDA
        // calls during the runtime's own teardown return an error and
        // free nothing, which is harmless here
        if (s) amrgpu_session_destroy(s);
        halo.release();
    }
};

// One cache per calling thread: ranks that run as threads of one process
// each keep their own session.
EvolveCache &cache()
{
    static thread_local EvolveCache c;
    return c;
}

uint64_t cfg_hash(const PhysicsConfig &c)
{
    uint64_t h = fnv1a(&c.time_scheme, sizeof(int));
    h = fnv1a(&c.dt, sizeof(double), h);
    h = fnv1a(&c.cfl, sizeof(double), h);
    h = fnv1a(c.bc, sizeof(c.bc), h);
    h = fnv1a(&c.form, sizeof(int), h);
    h = fnv1a(&c.final_time, sizeof(double), h);
    h = fnv1a(&c.coarse_grid_h, sizeof(double), h);
    h = fnv1a(&c.nelem_subgrid, sizeof(int), h);
    h = fnv1a(&c.initial_condition, sizeof(int), h);
    h = fnv1a(c.ic_params, sizeof(c.ic_params), h);
    return h;
}

// True when (cell_info, face_info, geom) and the counts equal the cached
// mesh's, compared byte for byte (a hash alone could collide and reuse the
// wrong quad descriptors).
bool same_mesh(const EvolveCache &ec, int ncell, int nghost, int nface, int dof, const int *cell_info,
               const int *face_info, const double *geom)
{
    if (!ec.s || ec.ncell != ncell || ec.nghost != nghost || ec.nface != nface || ec.dof != dof) return false;
    const size_t nc = size_t(ncell + nghost);
    return std::memcmp(ec.cell_info.data(), cell_info, sizeof(int) * 3 * nc) == 0 &&
           std::memcmp(ec.face_info.data(), face_info, sizeof(int) * 11 * size_t(nface)) == 0 &&
           std::memcmp(ec.geom.data(), geom, sizeof(double) * 12 * nc) == 0;
}

// The send / receive lists of a multi-rank call against what the GPU path
// needs: send entries name local quads, ghost k is receive entry k (the
// reference's driver stacks ghosts by owner rank after the local quads,
// physics_mpi.c:54 relies on it), every record is 4 n^2 doubles.
bool check_rank_lists(int ncell, int nghost, int nsend, int nrecv, const int *send, const int *recv,
                      const int *sizes, int stride, int n)
{
    auto fail = [](const std::string &m) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "multi-rank evolve: " + m);
        return false;
    };
    if (stride < 2) return fail("extern_mpi_comm_size < 2");
    if (nsend < 0 || nrecv < 0 || nghost < 0) return fail("negative list size");
    if (nrecv != nghost) return fail("nrecv != nghost");
    if ((nsend > 0 && !send) || (nrecv > 0 && !recv) || !sizes) return fail("missing send / recv / sizes");
    for (int k = 0; k < nsend; ++k)
        if (send[stride * k] < 0 || send[stride * k] >= ncell)
            return fail("send entry " + std::to_string(k) + " is not a local quad");
    for (int k = 0; k < nrecv; ++k)
        if (recv[stride * k] != ncell + k)
            return fail("receive entry " + std::to_string(k) + " is not ghost quad " + std::to_string(ncell + k));
    for (int q = 0; q < ncell + nghost; ++q)
        if (sizes[q] != 4 * n * n) return fail("sizes[" + std::to_string(q) + "] != 4 n^2");
    return true;
}

// A multi-rank segment of `steps` steps on an uploaded session: before
// every stage the send-list records go to the peers and the ghost records
// come back (pack on the device, one pinned copy each way, the caller's
// exchange); after the upload and after every step the CFL step is the
// MIN over ranks. Stops early once final_time is reached (every rank sees
// the same time). Returns the steps taken, or -1 on error.
int run_multirank(amrgpu_session *s, EvolveCache &ec, const amrgpu_comm_ops_t &ops, amrgpu_comm_t comm,
                  int stride, int steps, double final_time, amrgpu_report_t &rep)
{
    const int nsend = int(ec.send.size()) / stride, nrecv = int(ec.recv.size()) / stride;
    // ghost records in the edge-strip format: the stage kernels read only a
    // ghost's cells that face this rank's quads
    const size_t rec = size_t(16) * size_t(s->n);
    HaloBuffers &hb = ec.halo;
    auto reduce_dt = [&]() -> bool {
        unsigned long long *slot = amrgpu_session_dt_slot(s);
        if (!cuda_ok(cudaMemcpyAsync(hb.h_dt, slot, sizeof(*slot), cudaMemcpyDeviceToHost, s->stream), "D2H dt") ||
            !cuda_ok(cudaStreamSynchronize(s->stream), "sync"))
            return false;
        double v;
        std::memcpy(&v, hb.h_dt, sizeof(v));
        if (ops.allreduce(comm, &v, 0) != 0) {
            set_error(AMRGPU_ERR_CUDA, "multi-rank evolve: the caller's MIN all-reduce failed");
            return false;
        }
        std::memcpy(hb.h_dt, &v, sizeof(v));
        return cuda_ok(cudaMemcpyAsync(slot, hb.h_dt, sizeof(*slot), cudaMemcpyHostToDevice, s->stream), "H2D dt") &&
               cuda_ok(cudaStreamSynchronize(s->stream), "sync");
    };
    auto exchange = [&]() -> bool {
        if (nsend > 0) {
            if (amrgpu_session_halo_pack_edges(s, 0, nsend, hb.d_send) != AMRGPU_OK ||
                !cuda_ok(cudaMemcpyAsync(hb.h_send, hb.d_send, sizeof(double) * rec * size_t(nsend),
                                         cudaMemcpyDeviceToHost, s->stream),
                         "D2H halo"))
                return false;
        }
        if (!cuda_ok(cudaStreamSynchronize(s->stream), "sync")) return false;
        if (ops.exchange(comm, nsend, ec.send.data(), nrecv, ec.recv.data(), stride, int(rec), hb.h_send,
                         hb.h_recv) != 0) {
            set_error(AMRGPU_ERR_CUDA, "multi-rank evolve: the caller's ghost exchange failed");
            return false;
        }
        if (nrecv > 0) {
            if (!cuda_ok(cudaMemcpyAsync(hb.d_recv, hb.h_recv, sizeof(double) * rec * size_t(nrecv),
                                         cudaMemcpyHostToDevice, s->stream),
                         "H2D halo") ||
                amrgpu_session_halo_unpack_edges(s, 0, nrecv, hb.d_recv) != AMRGPU_OK)
                return false;
        }
        return true;
    };
    if (!reduce_dt()) return -1;
    int taken = 0;
    for (int k = 0; k < steps; ++k) {
        int st = 0, per = 0;
        do {
            if (!exchange() || amrgpu_session_step_stage(s, &st, &per) != AMRGPU_OK) return -1;
        } while (st != per);
        if (!reduce_dt()) return -1;
        ++taken;
        if (final_time > 0.0) {
            if (amrgpu_session_sync(s, &rep) != AMRGPU_OK) return -1;
            if (rep.time >= final_time) break;
        }
    }
    if (amrgpu_session_sync(s, &rep) != AMRGPU_OK) return -1;
    double nsq = s->h_scal.norm_sq;
    if (ops.allreduce(comm, &nsq, 1) != 0) {
        set_error(AMRGPU_ERR_CUDA, "multi-rank evolve: the caller's SUM all-reduce failed");
        return -1;
    }
    rep.residual_norm = std::sqrt(nsq);
    if (std::isnan(nsq)) rep.nan_detected = 1;
    return taken;
}

void evolve(bool from_reference_layer, int *dim, int *unstructured, int *nfields, int *nelem_subgrid, int *ncell,
            int *nghost, int *nface, int *dof, int *cell_info, int *face_info, int *nsend, int *nrecv, int *send,
            int *recv, int *sizes, double *geom, double *soln, int *istep, int *regrid, int *visualize,
            int *checkpoint, int *evolve_solution, amrgpu_comm_t comm, double *total_time, double *compute_time,
            double *residual_time)
{
    set_error(AMRGPU_OK, "");  // amrgpu_last_error() reports this call
    PhysicsConfig c;
    if (!resolve_config(from_reference_layer, c)) {
        *evolve_solution = 0;
        return;
    }
    // physics_go.c:66-69
    if (*istep >= c.time_steps) {
        *evolve_solution = 0;
        return;
    }
    if (*dim != 2 || *unstructured != 0 || *nfields != 4) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "GPU path: 2D structured with 4 fields only");
        *evolve_solution = 0;
        return;
    }
    const bool multirank = *nsend != 0 || *nrecv != 0 || *nghost != 0;
    amrgpu_comm_ops_t ops{};
    const int stride = c.extern_mpi_comm_size;
    if (multirank) {
        if (!comm_ops(ops)) {
            set_error(AMRGPU_ERR_UNSUPPORTED,
                      "multi-rank evolve (ghost quads) needs the caller's MPI operations: include "
                      "physics_go_gpu.h in the MPI program or call amrgpu_set_comm_ops");
            *evolve_solution = 0;
            return;
        }
        if (!check_rank_lists(*ncell, *nghost, *nsend, *nrecv, send, recv, sizes, stride, *nelem_subgrid)) {
            *evolve_solution = 0;
            return;
        }
    }
    c.dim = *dim;
    c.nfields = *nfields;
    c.nelem_subgrid = *nelem_subgrid;
    if (const char *f = std::getenv("AMRGPU_FORM")) c.form = std::atoi(f);

    auto wall0 = std::chrono::steady_clock::now();
    EvolveCache &ec = cache();
    const uint64_t ch = cfg_hash(c);
    // simulated time (for the final-time stop) continues only when this call
    // picks up where the last one ended: same configuration, *istep equal
    // to the istep the last call returned, and not a fresh start at 0
    const bool continuing = ec.s && ec.cfg_hash == ch && *istep > 0 && *istep == ec.end_istep;
    if (!continuing) ec.sim_time = 0.0;
    const size_t nsend_ints = multirank ? size_t(stride) * size_t(*nsend) : 0;
    const size_t nrecv_ints = multirank ? size_t(stride) * size_t(*nrecv) : 0;
    const bool same_lists = ec.send.size() == nsend_ints && ec.recv.size() == nrecv_ints &&
                            (nsend_ints == 0 || std::memcmp(ec.send.data(), send, sizeof(int) * nsend_ints) == 0) &&
                            (nrecv_ints == 0 || std::memcmp(ec.recv.data(), recv, sizeof(int) * nrecv_ints) == 0);
    if (ec.cfg_hash != ch || !same_lists ||
        !same_mesh(ec, *ncell, *nghost, *nface, *dof, cell_info, face_info, geom)) {
        if (ec.s) amrgpu_session_destroy(ec.s);
        ec.s = nullptr;
        amrgpu_mesh_t m{*ncell, *nghost, *nface, *dof, cell_info, face_info, geom};
        amrgpu_session *s = nullptr;
        const int rc = session_create_cfg(&s, &m, c);
        if (rc != AMRGPU_OK) {
            *evolve_solution = 0;
            return;
        }
        ec.send.assign(send, send + nsend_ints);
        ec.recv.assign(recv, recv + nrecv_ints);
        if (multirank) {
            std::vector<int> quads(static_cast<size_t>(*nsend));
            for (int k = 0; k < *nsend; ++k) quads[size_t(k)] = send[stride * k];
            const size_t rec = size_t(16) * size_t(*nelem_subgrid);  // edge-strip records
            if (amrgpu_session_set_halo(s, quads.data(), *nsend) != AMRGPU_OK ||
                !ec.halo.reserve(rec * size_t(std::max(*nsend, 1)), rec * size_t(std::max(*nrecv, 1)))) {
                amrgpu_session_destroy(s);
                *evolve_solution = 0;
                return;
            }
        }
        const size_t nc = size_t(*ncell + *nghost);
        ec.s = s;
        ec.cell_info.assign(cell_info, cell_info + 3 * nc);
        ec.face_info.assign(face_info, face_info + 11 * size_t(*nface));
        ec.geom.assign(geom, geom + 12 * nc);
        ec.ncell = *ncell;
        ec.nghost = *nghost;
        ec.nface = *nface;
        ec.dof = *dof;
        ec.cfg_hash = ch;
    }
    amrgpu_session *s = ec.s;
    s->cfg = c;
    s->t0 = ec.sim_time;
    s->step_index = 0;
    s->role[0] = 0; s->role[1] = 1; s->role[2] = 2; s->role[3] = 3;
    if (amrgpu_session_upload(s, soln) != AMRGPU_OK) {
        *evolve_solution = 0;
        ec.end_istep = -1;
        return;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s->stream);
    // number of steps of this segment (physics_runge_kutta_interface.c:213-229)
    int steps = 0;
    int is = *istep;
    for (;;) {
        ++steps;
        ++is;
        if (is >= c.time_steps || is % c.regrid_interval == 0 || is % c.checkpoint_interval == 0 ||
            is % c.visualization_interval == 0)
            break;
    }
    amrgpu_report_t rep{};
    int taken = 0;
    if (multirank) {
        taken = run_multirank(s, ec, ops, comm, stride, steps, c.final_time, rep);
        if (taken < 0) {
            *evolve_solution = 0;
            ec.end_istep = -1;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return;
        }
        if (c.final_time > 0.0 && rep.time >= c.final_time) *evolve_solution = 0;
        steps = taken;
    } else if (c.final_time > 0.0) {
        // the device clips dt at final_time; run in chunks and stop once reached
        int left = steps;
        while (left > 0) {
            int chunk = std::min(left, 240);
            if (amrgpu_session_step_graph(s, chunk, 60) != AMRGPU_OK) break;
            left -= chunk;
            amrgpu_session_sync(s, &rep);
            taken = rep.steps_done;
            if (rep.time >= c.final_time || rep.error) break;
        }
        if (rep.time >= c.final_time) *evolve_solution = 0;
        steps = taken;
    } else {
        int rc = (steps >= 12) ? amrgpu_session_step_graph(s, steps, std::min(steps - steps % 6, 600))
                               : amrgpu_session_step(s, steps);
        if (rc == AMRGPU_OK) amrgpu_session_sync(s, &rep);
    }
    cudaEventRecord(e1, s->stream);
    if (amrgpu_session_download(s, soln) != AMRGPU_OK) {
        *evolve_solution = 0;
        return;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ec.sim_time = rep.time;
    *istep += steps;
    ec.end_istep = *istep;
    if (*istep % c.regrid_interval == 0) *regrid = 1;
    if (*istep % c.checkpoint_interval == 0) *checkpoint = 1;
    if (*istep % c.visualization_interval == 0) *visualize = 1;
    double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    *total_time += wall;
    *compute_time += ms * 1e-3;
    *residual_time += ms * 1e-3;
    // physics_go.c:105-118 and physics_runtime_statistics.c:82-86
    int cells = *dof / *nfields;
    double cmin = cells, cmax = cells, ctot = cells;
    int rank = 0, nranks = 1;
    if (multirank) {
        // the same collectives on every rank, in the same order
        ops.allreduce(comm, &cmin, 0);
        ops.allreduce(comm, &cmax, 2);
        ops.allreduce(comm, &ctot, 1);
        double one = 1.0;
        ops.allreduce(comm, &one, 1);
        nranks = int(one);
        ops.rank(comm, &rank);
    }
    double resid = rep.residual_norm / std::pow(ctot, 1.0 / double(*dim));
    if (!std::getenv("AMRGPU_QUIET") && rank == 0) {
        std::printf("[ amr ] istep: %d\n", *istep);
        std::printf("[ amr ] processor dofs (min,max,avg,total): %d, %d, %d, %d \n", int(cmin), int(cmax),
                    int(ctot / double(nranks)), int(ctot));
        std::printf("[physics] iterations: %d, gpu time: %e, residual: %1.15e\n", steps, ms * 1e-3, resid);
        int nres = c.time_scheme;
        if (steps > 0 && cells > 0)
            std::printf("[physics] time/dof (gpu): %e\n", (ms * 1e-3) / double(cells) / double(steps) / double(nres));
    }
    if (rep.nan_detected || std::isnan(rep.residual_norm)) {
        std::printf("[solve] nan detected in residual aborting\n");
        set_error(AMRGPU_ERR_NONFINITE, "non-finite residual norm");
        *evolve_solution = 0;
        const char *ab = std::getenv("AMRGPU_ABORT_ON_NAN");
        if (ab && std::atoi(ab) == 1) std::exit(3);
    }
}

}  // namespace

extern "C" {

int amrgpu_evolve_config(int from_reference_layer, amrgpu_config_t *out)
{
    if (!out) return AMRGPU_ERR_ARG;
    PhysicsConfig c;
    if (!resolve_config(from_reference_layer != 0, c)) return AMRGPU_ERR_CONFIG;
    config_to_public(c, out);
    return AMRGPU_OK;
}

void hpc_amr_evolve_solver(int *dim, int *unstructured, int *nfields, int *nsub_elem, int *ncell, int *nghost,
                           int *nface, int *dof, int *cell_info, int *face_info, int *nsend, int *nrecv, int *send,
                           int *recv, int *sizes, double *geom, double *soln, int *istep, int *regrid,
                           int *visualize, int *checkpoint, int *evolve_solution, amrgpu_comm_t mpicomm_ext,
                           double *total_time, double *compute_time, double *residual_time)
{
    evolve(false, dim, unstructured, nfields, nsub_elem, ncell, nghost, nface, dof, cell_info, face_info, nsend, nrecv,
           send, recv, sizes, geom, soln, istep, regrid, visualize, checkpoint, evolve_solution, mpicomm_ext,
           total_time, compute_time, residual_time);
}

void physics_go_gpu(int *dim, int *unstructured, int *nfields, int *nelem_subgrid, int *ncell, int *nghost,
                    int *nface, int *dof, int *cell_info, int *face_info, int *nsend, int *nrecv, int *send,
                    int *recv, int *sizes, double *geom, double *soln, int *istep, int *regrid, int *visualize,
                    int *checkpoint, int *evolve_solution, amrgpu_comm_t mpicomm_ext, double *total_time,
                    double *compute_time, double *residual_time)
{
    evolve(true, dim, unstructured, nfields, nelem_subgrid, ncell, nghost, nface, dof, cell_info, face_info, nsend, nrecv,
           send, recv, sizes, geom, soln, istep, regrid, visualize, checkpoint, evolve_solution, mpicomm_ext,
           total_time, compute_time, residual_time);
}

int amrgpu_session_set_patch_rule(amrgpu_session_t *s, const int *size_of_level, int nlevels)
{
    if (!s || nlevels < 0 || nlevels > 32 || (nlevels > 0 && !size_of_level)) return AMRGPU_ERR_ARG;
    if (nlevels == 0) {
        s->has_rule = false;
        return AMRGPU_OK;
    }
    if (s->form != AMRGPU_FORM_FP32_FLUX || (s->launch_pinned && !s->mixed) || s->nghost != 0) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "mixed patch sizes: the FP32-flux form with the library's launch, no ghosts");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    SizeRule r{};
    for (int l = 0; l < 32; ++l) {
        const int v = size_of_level[std::min(l, nlevels - 1)];
        if (v != 8 && v != 16) {
            set_error(AMRGPU_ERR_ARG, "patch-size rule: sizes must be 8 or 16");
            return AMRGPU_ERR_ARG;
        }
        r.size[l] = v;
    }
    s->rule = r;
    s->has_rule = true;
    return AMRGPU_OK;
}

int amrgpu_set_comm_ops(const amrgpu_comm_ops_t *ops)
{
    if (ops && (!ops->rank || !ops->exchange || !ops->allreduce)) return AMRGPU_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_comm_mu);
    if (ops) g_comm_ops = *ops;
    g_comm_set = ops != nullptr;
    return AMRGPU_OK;
}

int amrgpu_has_comm_ops(void)
{
    amrgpu_comm_ops_t o;
    return comm_ops(o) ? 1 : 0;
}

}  // extern "C"
