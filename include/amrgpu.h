/*
 * amrgpu.h -- C ABI of libamrgpu, the B200 (sm_100a) implementation of the
 * residual / Runge-Kutta / CFL time-step path of amr-demo.
 *
 * Part 1 is the reference's own solver-facing call surface (same names,
 * same argument lists, same in/out meaning), so the reference's AMR driver
 * links against libamrgpu.so in place of libhpc_phys.so + libhpc_solver.so.
 * Part 2 is this library's extended API: device-resident sessions, forms,
 * batched regrid kernels, the host forest and error reporting.
 *
 * All pointers are plain host pointers unless a name says "_device".
 * Nothing here uses torch or C++ types.
 */
#ifndef AMRGPU_H
#define AMRGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The communicator argument of the reference ABI. A caller built with MPI
 * passes its MPI_Comm (see physics_go_gpu.h); the library links no MPI and
 * only hands it to the caller's MPI operations (amrgpu_comm_ops_t) in a
 * multi-rank call. */
#ifndef AMRGPU_COMM_T
#define AMRGPU_COMM_T intptr_t
#endif
typedef AMRGPU_COMM_T amrgpu_comm_t;

/* ======================================================================
 * Part 1 -- the reference's ABI
 * ====================================================================== */

/* Replaces hpc_amr_initialize_solver (src/amr/src/amr_external.h:50,
 * src/physics/src/hpc_amr_initialize_solver.c:16-28): stores the mesh
 * constants and reads "input.physics" from the working directory with the
 * reference's keyword rules (physics_initialize.c:61-197), including
 * cfl <- 0.25*cfl*time_scheme and intervals <= 0 -> INT_MAX. Unlike the
 * reference it does not exit() when the file is missing: it keeps the
 * defaults and reports AMRGPU_ERR_CONFIG through amrgpu_last_error(). */
void hpc_amr_initialize_solver(int *rank, int *dim, double *mesh_scale, int *nlevels,
                               int *nfields, int *nfringe, int *nsub_elem,
                               int *extern_cell_size, int *extern_face_size,
                               int *extern_edge_size, int *extern_node_size,
                               int *extern_mpi_comm_size);

/* Replaces hpc_amr_initialize_quadrant (amr_external.h:67,
 * hpc_amr_initialize_quadrant.c:15-21 -> initial_condition_2d_module.F90:12-131):
 * fills one quadrant's AoS patch with the configured initial condition. */
void hpc_amr_initialize_quadrant(int *dim, int *unstructured, int *nfields, int *nsub_elem,
                                 int *cell_type, double *elem_h, double *elem_xyz,
                                 double *soln);

/* Replaces hpc_amr_regrid_points (amr_external.h:77,
 * physics_regrid_points.c:28-36): no external points. */
void hpc_amr_regrid_points(int *construct_grid, int *nregrid_pts, double *regrid_width,
                           double *regrid_xyzh);

/* Replaces hpc_amr_tag_feature (amr_external.h:92, hpc_amr_tag_feature.c:17-26
 * -> solver_tag_feature.F90:9-52): density-threshold tagging of one quad. */
void hpc_amr_tag_feature(int *dim, int *unstructured, int *nfields, int *nsub_elem,
                         int *cell_type, double *elem_h, double *elem_xyz, double *soln,
                         int *tag);

/* Replaces hpc_amr_coarsen_operator_2d (amr_external.h:146,
 * solver_coarsen_operator_2d.F90:29-53): same-index average of 4 children. */
void hpc_amr_coarsen_operator_2d(int *unstructured, int *nfields, int *nsub_elem,
                                 int *cell_type, double *elem_h, double *elem_xyz,
                                 double *uc1, double *uc2, double *uc3, double *uc4,
                                 double *soln);

/* Replaces hpc_amr_refine_operator_2d (amr_external.h:189,
 * solver_refine_operator_2d.F90:28-55): every child receives the parent patch. */
void hpc_amr_refine_operator_2d(int *unstructured, int *nfields, int *nsub_elem,
                                int *cell_type, double *elem_h, double *elem_xyz,
                                double *soln, double *uc1, double *uc2, double *uc3,
                                double *uc4);

/* Replaces hpc_amr_evolve_solver (amr_external.h:124,
 * hpc_amr_evolve_solver.c:16-49) and, behind it, physics_go
 * (physics_go.c:16-132) with the whole time-step loop of
 * physics_runge_kutta_interface.c:23-357 run on the GPU:
 *   - returns with *evolve_solution = 0 when *istep >= time_steps;
 *   - otherwise copies soln[0:dof) to the device, runs steps until
 *     time_steps or a regrid / checkpoint / visualisation interval is hit,
 *     sets those flags, advances *istep, copies soln back;
 *   - accumulates *total_time, *compute_time, *residual_time (seconds).
 * Device buffers persist across calls and are rebuilt when the mesh
 * (cell_info / face_info / geom) changes. Each call first clears the
 * calling thread's error; errors are reported through
 * amrgpu_last_error(); a non-finite residual sets AMRGPU_ERR_NONFINITE (and
 * exits with code 3 when AMRGPU_ABORT_ON_NAN=1, as the reference's
 * MPI_Abort(comm,3) does). Only 2D structured meshes are accepted. A rank
 * with ghost quads (nghost, nsend, nrecv > 0) needs the caller's MPI
 * operations (amrgpu_comm_ops_t below) and exchanges ghost records before
 * every stage; without them the call is refused (AMRGPU_ERR_UNSUPPORTED).
 * Device state is kept per calling thread (ranks run as threads each get
 * their own). */
void hpc_amr_evolve_solver(int *dim, int *unstructured, int *nfields, int *nsub_elem,
                           int *ncell, int *nghost, int *nface, int *dof, int *cell_info,
                           int *face_info, int *nsend, int *nrecv, int *send, int *recv,
                           int *sizes, double *geom, double *soln, int *istep, int *regrid,
                           int *visualize, int *checkpoint, int *evolve_solution,
                           amrgpu_comm_t mpicomm_ext, double *total_time,
                           double *compute_time, double *residual_time);

/* The reference's reserved GPU plug-point (physics_evolve_interface.c:42-46,
 * declared by the missing physics_go_gpu.h, physics_evolve_interface.h:16-17);
 * same signature as physics_go (physics_go.h:59). Same behaviour as
 * hpc_amr_evolve_solver above. */
void physics_go_gpu(int *dim, int *unstructured, int *nfields, int *nelem_subgrid,
                    int *ncell, int *nghost, int *nface, int *dof, int *cell_info,
                    int *face_info, int *nsend, int *nrecv, int *send, int *recv,
                    int *sizes, double *geom, double *soln, int *istep, int *regrid,
                    int *visualize, int *checkpoint, int *evolve_solution,
                    amrgpu_comm_t mpicomm_ext, double *total_time, double *compute_time,
                    double *residual_time);

/* ======================================================================
 * Part 2 -- extended API (no reference counterpart unless stated)
 * ====================================================================== */

enum {
    AMRGPU_OK = 0,
    AMRGPU_ERR_ARG = 1,          /* invalid argument */
    AMRGPU_ERR_CUDA = 2,         /* CUDA runtime error */
    AMRGPU_ERR_MESH = 3,         /* inconsistent cell_info / face_info */
    AMRGPU_ERR_NONFINITE = 4,    /* NaN/Inf residual or state */
    AMRGPU_ERR_UNSUPPORTED = 5,  /* 3D, unstructured, multi-rank, patch size */
    AMRGPU_ERR_NO_DEVICE = 6,    /* no CUDA device */
    AMRGPU_ERR_CONFIG = 7,       /* input.physics missing or invalid */
    AMRGPU_ERR_TOO_LARGE = 8,    /* request above a stated maximum */
    AMRGPU_ERR_NEGATIVE = 9,     /* non-positive density or pressure */
    AMRGPU_ERR_IO = 10           /* file cannot be written / read, or is malformed */
};

enum {
    AMRGPU_FORM_FP64_EXACT = 0, /* reference arithmetic in FP64, bit-exact order */
    AMRGPU_FORM_FP32_FLUX = 1   /* FP32 flux, FP64 state / sums / RK (Shu-Osher RK3) */
};

int amrgpu_last_error(void);
const char *amrgpu_error_string(int code);
const char *amrgpu_last_error_message(void);
void amrgpu_clear_error(void);

/* Physics configuration, the fields of the reference's d_physics_fluid /
 * d_physics_simulation / d_physics_interface globals plus extensions. */
typedef struct {
    int dim, nfields, nelem_subgrid;
    double coarse_grid_h;        /* h of a level-0 quadrant (mesh_scale) */
    int initial_condition;       /* 0 free stream, 1 Shu vortex; 2..5 extensions */
    int bc[6];                   /* per side: 0 extrapolate, 1 slip, 2 no-slip, 3 inflow */
    int time_scheme;             /* 1 RK1, 2 SSP-RK2, 3 SSP-RK3, 4 RK4, 5 LSERK45 */
    int time_steps;
    double dt;                   /* cap on the CFL step */
    double cfl;                  /* effective (already scaled) CFL */
    double mach, alpha, beta, gamma, density, pressure;
    int checkpoint_interval, visualization_interval, regrid_interval;
    int amr_ntag_methods;
    int amr_tag_methods[5];
    double amr_tag_tolerances[5];
    int form;                    /* AMRGPU_FORM_* */
    double final_time;           /* > 0: stop at this time, last step clipped */
    double ic_params[8];         /* parameters of extension ICs */
    uint64_t ic_seed;            /* seed of extension ICs and density noise */
    double noise_amplitude;      /* uniform density noise amplitude */
} amrgpu_config_t;

void amrgpu_config_defaults(amrgpu_config_t *cfg);
int amrgpu_config_read(const char *path, amrgpu_config_t *cfg);
int amrgpu_config_get(amrgpu_config_t *cfg);
int amrgpu_config_set(const amrgpu_config_t *cfg);

/* The configuration the next evolve call runs with: from_reference_layer = 1
 * for physics_go_gpu, 0 for hpc_amr_evolve_solver. physics_go_gpu is called by
 * the reference's own physics layer built with -D_GPU_
 * (physics_evolve_interface.c:42-46), so it takes the reference's globals
 * d_physics_interface / d_physics_fluid / d_physics_simulation
 * (physics_var_*.h) when that layer is loaded and its physics_initialize has
 * run, else this library's configuration; hpc_amr_evolve_solver takes this
 * library's configuration (hpc_amr_initialize_solver above, or
 * amrgpu_config_set) first and the reference's second. With neither the
 * evolve entry points refuse to run (AMRGPU_ERR_CONFIG, *evolve_solution = 0)
 * and so does this call. The library's extensions (form, final_time, IC
 * parameters) always come from its own configuration. */
int amrgpu_evolve_config(int from_reference_layer, amrgpu_config_t *out);

/* ---------------- the caller's MPI, for multi-rank evolve calls ----------
 * hpc_amr_evolve_solver / physics_go_gpu with ghost quads (nghost, nsend,
 * nrecv > 0) run the reference's multi-rank step on the GPU: before every
 * stage the records of the send-list quads are packed on the device and
 * moved to the ranks that hold them as ghosts (physics_mpi_real_to_ghost,
 * physics_mpi.c:47-122, called by every stage of rk_time_integrators.c), the
 * CFL step is the MIN over ranks (MPI_Allreduce,
 * physics_runge_kutta_interface.c:96,149,205,262,316) and the squared
 * residual norm the SUM (rk_time_integrators.c:74,162,274). This library
 * links no MPI, so the caller supplies these three operations once.
 * physics_go_gpu.h does that automatically in the reference's -D_GPU_
 * build (a load-time constructor compiled against the caller's <mpi.h>);
 * other callers call amrgpu_set_comm_ops themselves. Every rank of a call
 * must make the same calls (they are collectives). Ghost quads must follow
 * the local quads in receive-list order (recv[k*stride] == ncell + k, as
 * the reference's AMR driver numbers them, amr_external.c). */
typedef struct {
    /* *rank = the caller's rank in comm; 0 on success. */
    int (*rank)(amrgpu_comm_t comm, int *rank);
    /* Moves whole-quad records: sendbuf holds record_doubles doubles per
     * send-list entry, in list order; recvbuf receives one record per
     * receive-list entry, in list order. Entries are (quad, peer rank)
     * pairs `stride` ints apart, grouped by peer. 0 on success. */
    int (*exchange)(amrgpu_comm_t comm, int nsend, const int *send, int nrecv, const int *recv, int stride,
                    int record_doubles, const double *sendbuf, double *recvbuf);
    /* In-place all-reduce of one double over comm: op 0 MIN, 1 SUM, 2 MAX.
     * 0 on success. */
    int (*allreduce)(amrgpu_comm_t comm, double *value, int op);
} amrgpu_comm_ops_t;

/* Installs (copies) the operations; NULL removes them. Process-wide. */
int amrgpu_set_comm_ops(const amrgpu_comm_ops_t *ops);
/* 1 when operations are installed. */
int amrgpu_has_comm_ops(void);

/* ---------------- device-resident sessions ---------------- */
typedef struct amrgpu_session amrgpu_session_t;

typedef struct {
    int ncell, nghost, nface, dof;
    const int *cell_info;   /* 3*(ncell+nghost) */
    const int *face_info;   /* 11*nface */
    const double *geom;     /* 12*(ncell+nghost) */
} amrgpu_mesh_t;

typedef struct {
    int steps_done;
    double time;            /* simulated time advanced by this session */
    double dt_last;         /* dt of the last step */
    double residual_norm;   /* sqrt(sum k^2) of the last stage, as rk_*() reports */
    int error;              /* AMRGPU_OK or an error code */
    int nan_detected;
} amrgpu_report_t;

/* Builds device tables for a mesh and a configuration (config NULL: the
 * global configuration). */
int amrgpu_session_create(amrgpu_session_t **out, const amrgpu_mesh_t *mesh,
                          const amrgpu_config_t *cfg);
void amrgpu_session_destroy(amrgpu_session_t *s);
int amrgpu_session_set_form(amrgpu_session_t *s, int form);
int amrgpu_session_set_launch(amrgpu_session_t *s, int quads_per_block, int threads);
/* Stage-launch autotuner (SURVEY build plan step 5; no reference
 * counterpart: the reference has one CPU code path). A session whose launch
 * was not set by the caller tunes on its first step after an upload or a
 * regrid, when it has at least 256 quads and AMRGPU_AUTOTUNE is not 0: each
 * compiled launch shape of its patch size runs a residual-only stage on the
 * session's own state (into a scratch buffer; the solution is untouched) and
 * the fastest is kept. Only shapes that give bits identical to the default
 * launch compete (every FP64 shape; for the FP32-flux form, the row sweeps
 * among themselves and the block kernels among themselves). The choice is
 * stored per (GPU name, SM count, form, patch size, floor(log2(quads))) in
 * memory and in a JSON file -- AMRGPU_TUNE_CACHE (empty: memory only), else
 * $XDG_CACHE_HOME/amrgpu/tune.json or $HOME/.cache/amrgpu/tune.json -- and
 * later sessions with the same key use it without timing. hpc_amr_evolve_solver,
 * physics_go_gpu and every regrid go through the same path.
 * amrgpu_session_autotune tunes now (retime = 1: ignore the stored choice
 * and time again); the chosen shape is then amrgpu_session_launch_variant. */
int amrgpu_session_autotune(amrgpu_session_t *s, int retime);
/* The stored choice for a key (nquad picks the bucket): 1 and the shape
 * when present, 0 when not. */
int amrgpu_tune_cache_get(const char *gpu, int sms, int form, int n, int nquad, int *quads_per_block,
                          int *threads, int *min_blocks, double *ms);
/* Stores a choice (replacing the key's previous one) and rewrites the file. */
int amrgpu_tune_cache_put(const char *gpu, int sms, int form, int n, int nquad, int quads_per_block,
                          int threads, int min_blocks, double ms);
/* Forgets the in-memory choices (the file is read again on next use). */
void amrgpu_tune_cache_reload(void);

/* The compiled stage-kernel launch shapes for the session's form and patch
 * size (the autotuner's candidates): fills up to cap pairs, returns the count. */
int amrgpu_session_launch_variants(const amrgpu_session_t *s, int *quads_per_block, int *threads,
                                   int cap);
/* Selects variant `index` of that list (variants that share a shape are
 * addressed this way); amrgpu_session_launch_variant returns the current
 * index. */
int amrgpu_session_set_launch_variant(amrgpu_session_t *s, int index);
int amrgpu_session_launch_variant(const amrgpu_session_t *s);
/* Shape of variant `index`: quads per CTA, threads, the minimum resident CTAs
 * per SM it was compiled for, and 1 for a row sweep / 0 for a block kernel. */
int amrgpu_session_launch_variant_info(const amrgpu_session_t *s, int index, int *quads_per_block,
                                       int *threads, int *min_blocks, int *sweep);
/* Host AoS soln (reference layout, dof + ghost tail) <-> device SoA state. */
int amrgpu_session_upload(amrgpu_session_t *s, const double *soln_aos);
int amrgpu_session_download(amrgpu_session_t *s, double *soln_aos);
/* Advance nsteps on the device (async on the session stream). */
int amrgpu_session_step(amrgpu_session_t *s, int nsteps);
/* Same, recording the steps as a CUDA graph of graph_steps steps. */
int amrgpu_session_step_graph(amrgpu_session_t *s, int nsteps, int graph_steps);
int amrgpu_session_sync(amrgpu_session_t *s, amrgpu_report_t *rep);
/* One residual evaluation rhs = -R(Q) of the current state (AoS, dof). */
int amrgpu_session_rhs(amrgpu_session_t *s, double *rhs_aos);
/* CFL time step of the current state, capped by the configured dt. */
int amrgpu_session_cfl_dt(amrgpu_session_t *s, double *dt);
/* Device pointer of field f of the SoA state; cells of quad q are
 * [q*n*n, (q+1)*n*n), row-major (i fastest). */
const double *amrgpu_session_state_device(amrgpu_session_t *s, int field);
int amrgpu_session_cells(const amrgpu_session_t *s);
void *amrgpu_session_stream(amrgpu_session_t *s);
/* Kernel launches issued by this session so far. */
int64_t amrgpu_session_launch_count(const amrgpu_session_t *s);
/* Conservation totals sum(vol*Q_f) for the 4 fields, in FP64. */
int amrgpu_session_totals(amrgpu_session_t *s, double totals[4]);

/* ---------------- sharded meshes (one session per rank) ----------------
 * A rank's mesh holds its ncell local quads followed by nghost ghost quads,
 * grouped by owning rank in ascending order (physics_mpi.c:54). The host
 * driver refreshes the ghosts of every stage's input before the stage
 * (physics_mpi_real_to_ghost, rk_time_integrators.c:227-262) and takes the
 * cross-rank MIN of the CFL step before every step
 * (physics_runge_kutta_interface.c:96,149,205,262,316) and the SUM of the
 * squared residual norm (rk_time_integrators.c:74,162,274). One quad's
 * halo record is 4 fields x n*n doubles (whole patch) or 16*n (edge
 * strips, below). */
/* Enqueues the next stage of the current step; reports its 1-based index
 * and the stages of a step. A step begun here is finished here before
 * amrgpu_session_step / step_graph / regrid. */
int amrgpu_session_step_stage(amrgpu_session_t *s, int *stage, int *stages_per_step);
/* Device buffer the next stage reads its own and its neighbours' cells
 * from (SoA, field stride in cells), ghost quads included. */
double *amrgpu_session_stage_input(amrgpu_session_t *s, long long *field_stride);
/* Device address of the CFL step the next step uses, as the uint64 image
 * of a positive double (MIN over ranks = MIN of the doubles). Written by
 * the last stage of a step and by upload. */
unsigned long long *amrgpu_session_dt_slot(amrgpu_session_t *s);
/* Extension: a caller's CUDA graph of whole steps made of step_stage and
 * halo calls (with its own collectives between them). The calls only
 * enqueue work, but they move the session's step counter, stage position
 * and buffer roles as if it had run: capture_mark (at a step boundary;
 * it also runs a pending launch tuning first, which must not be captured)
 * saves them before the capture, capture_rewind restores them after it,
 * and advance(nsteps) moves them by the nsteps whole steps a replay runs.
 * step_index is the session's step counter: the device addresses a step
 * uses repeat with period 6 (three CFL slots, two buffer-role parities),
 * so a graph of step k replays correctly at every step = k mod 6. */
int amrgpu_session_capture_mark(amrgpu_session_t *s);
int amrgpu_session_capture_rewind(amrgpu_session_t *s);
int amrgpu_session_advance(amrgpu_session_t *s, int nsteps);
long long amrgpu_session_step_index(const amrgpu_session_t *s);
/* Local quads (host array, each < ncell) whose records other ranks need,
 * grouped by destination rank (the reference's send list). */
int amrgpu_session_set_halo(amrgpu_session_t *s, const int *send_quads, int nsend);
/* Records of send entries [first, first+count) of the next stage's input
 * -> d_out (device, count * 4*n*n doubles), on the session stream. */
int amrgpu_session_halo_pack(amrgpu_session_t *s, int first, int count, double *d_out);
/* Records d_in (device) -> ghost quads first_ghost .. first_ghost+count-1
 * of the next stage's input, on the session stream. */
int amrgpu_session_halo_unpack(amrgpu_session_t *s, int first_ghost, int count, const double *d_in);
/* The same two calls with edge-strip records: per quad and field the n
 * cells of its side 0 (column 0), 1 (column n-1), 2 (row 0) and 3 (row n-1),
 * 16*n doubles (4x fewer than a whole record at n = 16). The stage kernels
 * read a ghost quad only at cells facing local quads, i.e. on these strips;
 * unpack leaves a ghost's interior cells as they were. The reference-named
 * evolve entry points exchange ghosts in this format. */
int amrgpu_session_halo_pack_edges(amrgpu_session_t *s, int first, int count, double *d_out);
int amrgpu_session_halo_unpack_edges(amrgpu_session_t *s, int first_ghost, int count, const double *d_in);
/* This rank's squared residual norm and flag bits (1 non-finite, 2
 * negative density or pressure) as of the last amrgpu_session_sync. */
int amrgpu_session_local_scalars(amrgpu_session_t *s, double *norm_sq, int *flags);

/* ---------------- host forest (stands in for p4est) ---------------- */
typedef struct amrgpu_forest amrgpu_forest_t;
amrgpu_forest_t *amrgpu_forest_new_brick(int nx, int ny, int periodic_x, int periodic_y,
                                         double xlo, double ylo, double zlo, double scale,
                                         int level);
void amrgpu_forest_destroy(amrgpu_forest_t *f);
int amrgpu_forest_num_quads(const amrgpu_forest_t *f);
/* Per quad: tree, level, x, y (units of 2^-30 of a tree), tag, type. */
int amrgpu_forest_quads(const amrgpu_forest_t *f, int *tree, int *level, int64_t *x, int64_t *y);
int amrgpu_forest_set_tags(amrgpu_forest_t *f, const int *tags);
int amrgpu_forest_get_tags(const amrgpu_forest_t *f, int *tags);
void amrgpu_forest_begin_regrid(amrgpu_forest_t *f);
int amrgpu_forest_refine(amrgpu_forest_t *f, const int *flags, int max_level);
int amrgpu_forest_coarsen(amrgpu_forest_t *f, const int *flags, int min_level);
int amrgpu_forest_balance(amrgpu_forest_t *f);
/* One regrid's refine and coarsen from per-quad tags in a single call (the
 * reference's amr_regrid.c:15-81 steps without the balance): begin_regrid,
 * tags stored on the quads, every quad tagged refine_value below
 * max_level refined (children keep tag 1), then every complete family of
 * quads tagged coarsen_value above min_level coarsened. Returns the quad
 * count, or -error. */
int amrgpu_forest_adapt(amrgpu_forest_t *f, const int *tags, int refine_value, int coarsen_value, int min_level,
                        int max_level);
int amrgpu_forest_is_balanced(const amrgpu_forest_t *f);
/* For every quad after the last begin_regrid: kind 0 = copy (injection)
 * from old quad src, kind 1 = average of old quads src..src+3. */
int amrgpu_forest_remap(const amrgpu_forest_t *f, int *kind, int *src);
/* Upper bound of nface for amrgpu_forest_external (4 per quad). */
int amrgpu_forest_max_faces(const amrgpu_forest_t *f);
int amrgpu_forest_external(const amrgpu_forest_t *f, int nelem_subgrid, int nfields,
                           int *cell_info, int *face_info, double *geom, int *nface,
                           int *dof);
double amrgpu_forest_quad_h(const amrgpu_forest_t *f, int quad);
/* Initial condition of every quad through hpc_amr_initialize_quadrant
 * semantics and the global configuration; soln is AoS (dof). */
int amrgpu_forest_initialize(const amrgpu_forest_t *f, int nelem_subgrid, double *soln);

/* ---------------- batched regrid kernels (GPU) ---------------- */
/* Plain indicator of solver_tag_feature.F90:9-52 for every quad of the
 * session's state, plus the density-jump extension (method 5). */
int amrgpu_session_tag(amrgpu_session_t *s, int *tags);
/* New SoA state for a remapped mesh: kind/src from amrgpu_forest_remap. */
int amrgpu_session_remap(amrgpu_session_t *dst, amrgpu_session_t *src, const int *kind,
                         const int *src_index);
/* In-place regrid: the session takes the new mesh m (no ghost quads) and
 * its state is remapped by kind/src (amrgpu_forest_remap) into the spare
 * state buffer; device arrays are reused while they are large enough and
 * grow to twice the need otherwise. Simulated time and the step
 * counter carry over on the device; the first step's CFL minimum is folded
 * for the new mesh. Replaces the per-regrid rebuild of the reference's
 * amr_regrid.c:82-125 (new ghost layer, new face lists, new soln array). */
int amrgpu_session_regrid(amrgpu_session_t *s, const amrgpu_mesh_t *m, const int *kind,
                          const int *src_index);
/* The same regrid straight from the forest after refine / coarsen / balance:
 * the leaves and the remap table go to the device in one pinned copy and
 * the quad descriptors (face types, neighbours, face order, corners) are
 * built there -- byte-identical to decoding amrgpu_forest_external's
 * arrays, without building them on the host. AMRGPU_ERR_MESH if the forest
 * is not 2:1 balanced (the session keeps its mesh). */
int amrgpu_session_regrid_forest(amrgpu_session_t *s, const amrgpu_forest_t *f);
/* amrgpu_forest_balance with the checks and the refinement of every pass
 * on the session's GPU (same passes, same leaves, tags and remap table);
 * returns the leaf count, or -error. */
int amrgpu_forest_balance_device(amrgpu_forest_t *f, amrgpu_session_t *s);
/* amrgpu_forest_balance_device then amrgpu_session_regrid_forest, with the
 * descriptors built from the balanced leaves already on the device (one
 * upload of the forest per regrid instead of two) and the remap table of
 * the balanced leaves gathered there from the pre-balance leaves they
 * descend from (no remap table built or uploaded by the host after the
 * balance). */
int amrgpu_session_balance_regrid(amrgpu_session_t *s, amrgpu_forest_t *f);
/* One whole regrid of the session and its forest f (whose leaves are the
 * session's mesh): the refinement tags (the session's tag kernel on its
 * current state when tags is NULL, else the caller's, one per quad), then
 * amrgpu_forest_adapt(f, tags, refine_value, coarsen_value, min_level,
 * max_level) and amrgpu_session_balance_regrid(s, f) -- the same forest,
 * mesh and state. When the session's last regrid came from f and f has not
 * changed since, the refine / coarsen also runs on the device, at the head
 * of the balance's single launch, from the leaves the session still holds
 * (no upload of the forest), while the host adapts f from the tags copied
 * back; the two must agree (AMRGPU_ERR_MESH otherwise). tags_out (NULL or
 * one int per quad) receives the tags used. Replaces the tagging, refine /
 * coarsen and balance of the reference's amr_regrid.c:82-125 in one call. */
int amrgpu_session_adapt_regrid(amrgpu_session_t *s, amrgpu_forest_t *f, const int *tags, int *tags_out,
                                int refine_value, int coarsen_value, int min_level, int max_level);
/* 1 when the session still holds f's current leaves on the device (its
 * last regrid came from f and f has not changed since), so that the next
 * amrgpu_session_adapt_regrid of f adapts them there; else 0. */
int amrgpu_session_holds_forest(const amrgpu_session_t *s, const amrgpu_forest_t *f);
/* Test support for the bounded waits of amrgpu_session_balance_regrid's
 * one-launch balance (device-wide barriers between its phases, each wait
 * at most 2^22 polls): runs it with the barrier's arrival count started out
 * of reach, so that every wait runs out (about half a second), the kernel
 * ends and the call returns AMRGPU_ERR_CUDA; the session keeps its mesh
 * and state and the forest its leaves. Sessions without a patch-size rule,
 * at a step boundary, without ghost quads. */
int amrgpu_session_balance_stall_test(amrgpu_session_t *s, amrgpu_forest_t *f);
/* Mixed patch sizes (extension; the reference fixes one size per build):
 * the patch size (8 or 16) of a quad at each level, size_of_level[l] for
 * l < nlevels (the last entry for deeper levels); nlevels = 0 clears it.
 * With a rule set, amrgpu_session_balance_regrid / _regrid_forest build a
 * mesh of mixed sizes on the device (sizes, cell offsets as the running
 * sum of n^2, neighbour sizes, the work list of the mixed-size sweep) and
 * remap the state, resampling by position where a quad's size changes.
 * A mesh passed to amrgpu_session_create / _regrid with per-quad sizes in
 * cell_info[2] (the running sum of 4 n^2) is mixed without a rule. Mixed
 * meshes: FP32-flux form only, no ghost quads, the two fine quads of a
 * hanging edge share one size; an edge between two sizes pairs the cells
 * that cover each piece of the finer side's length, one flux per piece for
 * both quads (conservative). */
int amrgpu_session_set_patch_rule(amrgpu_session_t *s, const int *size_of_level, int nlevels);
/* Extension (the reference allocates per regrid through p4est): grows every
 * device and pinned buffer that a regrid of this session may need -- the
 * state (its contents kept), quad descriptors, remap and tag tables, mixed
 * patch tables, balance buffers (forests of up to 64 trees) and the staging
 * of the forest's leaves -- to hold a mesh of up to `cells` cells and
 * `quads` quads, so that later regrids within those bounds allocate and
 * free nothing (large device allocations and frees cost milliseconds each
 * and synchronise the device). Beyond the bounds the buffers grow as
 * before. Captured step graphs are released. */
int amrgpu_session_reserve(amrgpu_session_t *s, long long cells, int quads);
/* Copies up to cap quad descriptors (160 bytes each: 4 sides x {kind, nbr0,
 * nbr1, face rank, level, bc} ints, then 8 corner doubles) to host memory;
 * returns the session's quad count. */
int amrgpu_session_quad_descriptors(amrgpu_session_t *s, void *out, int cap);
/* Faces of the session's mesh. */
int amrgpu_session_face_count(const amrgpu_session_t *s);

/* ---------------- output: visualisation and checkpoint ---------------- */
/* Unstructured VTK (.vtu, ASCII) of a forest and its AoS state (soln[f +
 * 4*(c + n*n*q)]): as the reference's vtk_write_solution
 * (src/amr/src/amr_vtk.c:23-106) one quad per quadrant, corners shrunk by
 * 0.99999, cell data treeid / level / mpirank and point data rho, rhou,
 * rhov, rhoe = the patch average at every corner (interpolate_solution,
 * amr_vtk.c:109-217); subgrid != 0 writes every subgrid cell as a quad
 * with its own values as cell data instead. */
int amrgpu_write_vtk(const char *path, const amrgpu_forest_t *forest, int n, const double *soln,
                     int subgrid);
/* Checkpoint of the forest, the AoS state, the step and the time (the
 * reference saves the forest and quadrant data with p4est_save,
 * amr_evolve.c:61-64, and has no reader). read_header gives the sizes;
 * read restores a new forest (destroy it with amrgpu_forest_destroy) and
 * fills soln (capacity in doubles, at least 4*n*n*nquad). */
int amrgpu_checkpoint_write(const char *path, const amrgpu_forest_t *forest, int n,
                            const double *soln, int istep, double time);
int amrgpu_checkpoint_read_header(const char *path, int *nquad, int *n, int *istep, double *time);
int amrgpu_checkpoint_read(const char *path, amrgpu_forest_t **forest, double *soln,
                           long long soln_capacity);

/* ---------------- learned refinement indicator ---------------- */
/* No counterpart in the reference: a 400-128-64-3 MLP (GELU) over a patch's
 * normalised conserved variables (8x8 patch, n = 16 patches box-averaged,
 * plus a one-cell neighbour ring) that classifies a quad as 0 = coarsen
 * candidate, 1 = refine, 2 = keep, in place of the plain tagger
 * (solver_tag_feature.F90:9-52 behind hpc_amr_tag_feature,
 * amr_external.h:92). BF16 weights, FP32 accumulation on the tensor cores
 * (tcgen05), AdamW on FP32 master weights; trained on (patch, plain-label)
 * pairs on the GPU. Plain label: J = largest relative density jump of the
 * quad (tag method 5's quantity); refine if J >= tol, coarsen if
 * J < lo_frac*tol, keep otherwise. */
typedef struct amrgpu_mlp amrgpu_mlp_t;
#define AMRGPU_MLP_INPUTS 400
#define AMRGPU_MLP_PARAMS 59779
typedef struct {
    int judged;       /* quads the plain indicator re-scored */
    int disagree;     /* of those, where the learned class differs */
    double rate;      /* disagree / judged (0 when none judged) */
    int coarser;      /* of those, where the learned class leaves the quad
                         coarser than the plain one: plain refine and learned
                         not, or learned coarsen and plain not */
} amrgpu_judge_t;
int amrgpu_mlp_create(amrgpu_mlp_t **out, unsigned long long seed);
void amrgpu_mlp_destroy(amrgpu_mlp_t *m);
/* FP32 parameters, flat: W1[128x400], b1[128], W2[64x128], b2[64], W3[3x64], b3[3]
 * (row-major, W[out][in]); set_params also resets the optimiser state. */
int amrgpu_mlp_get_params(amrgpu_mlp_t *m, float *params);
int amrgpu_mlp_set_params(amrgpu_mlp_t *m, const float *params);
/* Features of every quad of a session's state: nquad x 400 BF16 bit patterns. */
int amrgpu_session_features(amrgpu_session_t *s, uint16_t *features);
/* Largest relative density jump J of every quad. */
int amrgpu_session_jumps(amrgpu_session_t *s, double *jumps);
/* Appends the features and plain labels of every quad of the session to
 * the model's device dataset; returns the dataset size or a negative error. */
long long amrgpu_mlp_dataset_append(amrgpu_mlp_t *m, amrgpu_session_t *s, double tol, double lo_frac);
/* Recomputes the labels of rows [first, first + nquad) from the session's
 * current state (the session must hold the mesh those rows came from):
 * labels that look ahead to a later state of the same mesh. */
int amrgpu_mlp_dataset_relabel(amrgpu_mlp_t *m, amrgpu_session_t *s, long long first, double tol,
                               double lo_frac);
/* As amrgpu_mlp_dataset_relabel, but each row's label is merged with the
 * plain class of the current state instead of replaced, keeping the finer
 * demand: refine if either asks for it, coarsen only if both do, keep
 * otherwise. Called at several later states of one mesh, it labels each
 * quad with what the plain indicator asks for at any of them. */
int amrgpu_mlp_dataset_cover(amrgpu_mlp_t *m, amrgpu_session_t *s, long long first, double tol,
                             double lo_frac);
long long amrgpu_mlp_dataset_size(const amrgpu_mlp_t *m);
int amrgpu_mlp_dataset_clear(amrgpu_mlp_t *m);
/* Labels of the dataset rows [0, n). */
int amrgpu_mlp_dataset_labels(amrgpu_mlp_t *m, int *labels, long long n);
/* One pass of AdamW (beta 0.9/0.999, eps 1e-8, decay on weights only) over
 * the dataset rows in the order perm[0..n), batches of `batch` rows (a
 * multiple of 128; a final partial batch is dropped); mean loss and
 * accuracy of the pass. */
int amrgpu_mlp_train_epoch(amrgpu_mlp_t *m, const int *perm, long long n, int batch, float lr,
                           float weight_decay, double *mean_loss, double *accuracy);
/* Forward and backward of one batch (a multiple of 8 rows) given on the
 * host, no update: logits
 * [B x 3], the flat gradient of the mean cross-entropy (AMRGPU_MLP_PARAMS
 * floats) and the mean loss. */
int amrgpu_mlp_grad(amrgpu_mlp_t *m, const uint16_t *features, const int *labels, int batch,
                    float *logits, float *grad, double *mean_loss);
/* Logits [B x 3] of features given on the host. */
int amrgpu_mlp_predict(amrgpu_mlp_t *m, const uint16_t *features, int batch, float *logits);
/* Learned classes of every quad of the session (tags = class index). The
 * plain indicator re-scores the quads selected by a hash of (seed, quad)
 * below judge_fraction and the agreement is returned in judge. */
int amrgpu_session_learned_tags(amrgpu_session_t *s, amrgpu_mlp_t *m, double judge_fraction,
                                unsigned long long seed, double tol, double lo_frac, int *tags,
                                amrgpu_judge_t *judge);

/* ---------------- allocation-free entry point ---------------- */
/* No counterpart in the reference. Conservation totals sum(vol*Q_f), f =
 * 0..3, of a device-resident SoA state, like amrgpu_session_totals, for
 * callers that cannot let a library allocate: a driver that gives all
 * device memory to its own pool at start-up, or one that checks
 * conservation inside its time-step loop on a busy device, where the
 * device-wide synchronisation of cudaMalloc/cudaFree would stall other
 * streams. The function calls no cudaMalloc, cudaFree or other allocating
 * routine: its scratch is a fixed array in the library's device image (one
 * partial sum per quad, so at most AMRGPU_NOALLOC_MAX_QUADS quads; larger
 * requests return AMRGPU_ERR_TOO_LARGE), held by every GPU that loads the
 * library until the process exits.
 *   q_device        field f of cell c at q_device[f*field_stride + c],
 *                   cells of quad q at [q*n*n, (q+1)*n*n), row-major
 *   corners_device  8 doubles per quad: x,y of n1(-,-) n2(+,-) n3(-,+) n4(+,+)
 *   totals          host array of 4 doubles (written before return)
 *   stream          cudaStream_t to run on (NULL: the legacy default stream)
 * The first call on each device looks up the scratch array's device address
 * (cudaGetSymbolAddress) and must not be made during stream capture. All
 * calls share the scratch array; calls that overlap on the GPU race. The
 * call synchronises `stream` before returning. */
#define AMRGPU_NOALLOC_MAX_QUADS 65536
int amrgpu_totals_noalloc(const double *q_device, long long field_stride,
                          const double *corners_device, int nquad, int n,
                          double totals[4], void *stream);

#ifdef __cplusplus
}
#endif

#endif /* AMRGPU_H */
