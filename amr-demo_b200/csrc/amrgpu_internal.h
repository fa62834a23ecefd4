// amrgpu_internal.h -- declarations shared by the host C++ and CUDA sources
// of libamrgpu. Nothing here is part of the public C ABI (include/amrgpu.h).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "amrgpu.h"

namespace amrgpu {

// ---------------------------------------------------------------- forest
enum { kRemapCopy = 0, kRemapAverage = 1 };

struct Leaf {
    int tree;
    int level;
    int64_t x, y;   // lower corner in units of 2^-30 of the tree
    int tag;        // refinement tag carried through a regrid
    int type;       // cell type (cell_info[0])
    int src;        // provenance within the current regrid (see forest_begin_regrid)
    int src_kind;   // kRemapCopy: data of old leaf src; kRemapAverage: mean of old src..src+3
    int dirty = 0;  // created by refine / coarsen / balance since the last completed balance
};

struct Forest;
Forest *forest_new_brick(int nx, int ny, int px, int py, double xlo, double ylo, double zlo,
                         double scale, int level);
void forest_destroy(Forest *f);
int forest_num_quads(const Forest *f);
const std::vector<Leaf> &forest_leaves(const Forest *f);
std::vector<Leaf> &forest_leaves_mut(Forest *f);
// Advanced by every call that may change the leaves (forest_leaves_mut
// included): equal values mean unchanged leaves.
uint64_t forest_version(const Forest *f);
// Resizes the forest's leaves to n, reserving a quarter more when the
// capacity runs out (a regrid then rarely touches freshly allocated pages).
void forest_grow_leaves(Forest *f, size_t n);
void forest_begin_regrid(Forest *f);
int forest_refine(Forest *f, const int *flags, int max_level);
int forest_coarsen(Forest *f, const int *flags, int min_level);
// begin_regrid, the tags, refinement of the quads tagged refine_value below
// max_level (children tagged 1), coarsening of complete families tagged
// coarsen_value above min_level: forest_begin_regrid + forest_refine +
// forest_coarsen in three passes over the leaves; returns the leaf count.
int forest_adapt(Forest *f, const int *tags, int refine_value, int coarsen_value, int min_level, int max_level);
int forest_balance(Forest *f);
bool forest_is_balanced(const Forest *f);
void forest_quad_corners(const Forest *f, const Leaf &q, double xyz[12]);
// Checkpoint image of a forest: brick, periodicity, origin, scale and the
// leaves (tree, level, x, y, tag, type); forest_load returns null on a
// malformed image.
std::vector<unsigned char> forest_save(const Forest *f);
Forest *forest_load(const unsigned char *data, size_t size);
double forest_quad_h(const Forest *f, const Leaf &q);
// The brick a forest lives on: size, periodicity, origin and scale, tree id
// -> brick position (tree_tx, tree_ty) and back (tree_at[ty*nx+tx]).
struct BrickView {
    int nx, ny, periodic[2];
    double xlo[3], scale;
    const int *tree_tx, *tree_ty, *tree_at;
};
void forest_brick(const Forest *f, BrickView *out);
int forest_external(const Forest *f, int nelem_subgrid, int nfields, int *cell_info,
                    int *face_info, double *geom, int *nface_out, int *dof_out);

// ---------------------------------------------------------------- config
// The reference's physics configuration (physics_var_physics.h,
// physics_var_simulation.h, physics_var_interface.h), parsed with the same
// keyword rules as physics_initialize.c:61-197.
struct PhysicsConfig {
    int dim = 2;
    int nfields = 4;
    int nfringe = 2;
    int nelem_subgrid = 2;
    int extern_cell_size = 3;
    int extern_face_size = 11;
    int extern_mpi_comm_size = 2;
    int nlevels = 0;
    double coarse_grid_h = 1.0;

    int initial_condition = 1;
    int bc[6] = {1, 1, 1, 1, 1, 1};
    int amr_ntag_methods = 0;
    std::vector<int> amr_tag_methods;
    std::vector<double> amr_tag_tolerances;
    double cfl = 1.0;  // already scaled by 0.25*time_scheme when read from a file
    double mach = 0.1, alpha = 0.0, beta = 0.0, gamma = 1.4, density = 1.0, pressure = 1.0 / 1.4;

    int checkpoint_interval = 2147483647;
    int visualization_interval = 2147483647;
    int regrid_interval = 2147483647;
    int time_scheme = 1;
    int time_steps = 1;
    double dt = 0.001;

    // extensions (no reference counterpart)
    int form = AMRGPU_FORM_FP64_EXACT;
    double final_time = 0.0;  // > 0: stop at this simulated time, last step clipped
    int abort_on_nan = 0;
    double ic_params[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t ic_seed = 0;
    double noise_amplitude = 0.0;
};

PhysicsConfig &global_config();
// True once hpc_amr_initialize_solver read input.physics or
// amrgpu_config_set was called; evolve refuses to run on bare defaults.
bool config_initialized();
void set_config_initialized(bool v);
int parse_physics_file(const char *path, PhysicsConfig &cfg);
void config_to_public(const PhysicsConfig &c, amrgpu_config_t *o);

// ---------------------------------------------------------------- autotuner
// One tuned choice: the key (GPU name, SM count, form, patch size,
// floor(log2(quads))) and the launch shape picked, with its residual-stage
// time in ms. tune_cache.cpp keeps them in memory and in a JSON file.
struct TuneEntry {
    std::string gpu;
    int sms = 0, form = 0, n = 0, bucket = 0;
    int qpb = 0, threads = 0, min_blocks = 0;
    double ms = 0.0;
};
std::string tune_cache_path();
bool tune_lookup(const TuneEntry &key, TuneEntry *out);
void tune_store(const TuneEntry &e);
void tune_forget();  // drops the in-memory table; the file is read again on next use

// ---------------------------------------------------------------- staging
// Two pinned chunks and their events (staging.cu): pageable host arrays move
// to and from the device through them, host copies overlapping the DMA.
struct PinnedRing {
    static constexpr size_t kChunk = size_t(8) << 20;
    void *buf[2] = {nullptr, nullptr};
    void *ev[2] = {nullptr, nullptr};  // cudaEvent_t
    bool ensure();
    void release();
};
bool host_is_pinned(const void *p);
// dst/src device arrays, stream a cudaStream_t. ring_h2d returns once the
// last chunk is queued (the caller's array may be reused after that);
// ring_d2h returns after the data has landed in dst.
bool ring_h2d(PinnedRing &r, void *dst, const void *src, size_t bytes, void *stream);
bool ring_d2h(PinnedRing &r, void *dst, const void *src, size_t bytes, void *stream);

// ---------------------------------------------------------------- errors
void set_error(int code, const std::string &msg);

// Device-side view of a session's current state for kernels outside
// session.cu (the learned indicator): patch size, quads, SoA state (field
// stride in doubles), quad descriptors and the session's stream.
struct QuadDesc;
struct SessionView {
    int n;
    int nquad;
    long long stride;
    const double *q;
    const QuadDesc *quads;
    void *stream;  // cudaStream_t
};
bool session_view(amrgpu_session_t *s, SessionView *v);
void session_count_launches(amrgpu_session_t *s, int k);
// Device scratch owned by the session, grown (never shrunk) to `bytes`;
// contents are not kept across calls. Null when the allocation fails.
void *session_scratch(amrgpu_session_t *s, size_t bytes);
int last_error();

// ---------------------------------------------------------------- host ICs
void initialize_quadrant_host(const PhysicsConfig &cfg, int nfields, int n, int *cell_type,
                              double h, const double *geom, double *soln, int64_t first_cell_id);
void shock_state(double gamma, double ms, double rho1, double p1, double out[4]);
void tag_feature_host(const PhysicsConfig &cfg, int nfields, int n, const double *soln, int *tag);

}  // namespace amrgpu

// The C ABI's forest handle (amrgpu_forest_t of include/amrgpu.h).
struct amrgpu_forest {
    amrgpu::Forest *f;
};
