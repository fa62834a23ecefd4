"""amrgpu -- Python host mirror of libamrgpu's C ABI.

The reference (amr-demo) drives its physics through per-rank C entry points:
``hpc_amr_initialize_solver``, ``hpc_amr_initialize_quadrant``,
``hpc_amr_tag_feature``, ``hpc_amr_refine_operator_2d``,
``hpc_amr_coarsen_operator_2d`` and ``hpc_amr_evolve_solver``
(src/amr/src/amr_external.h:50-192). This package calls the same entry
points of the B200 library with numpy arrays laid out exactly as
``src/amr/src/amr_external.c`` lays them out, plus the library's extended
API (device-resident sessions, the host forest, batched regrid kernels).
"""
import ctypes as C

import numpy as np

from ._lib import (AmrGpuError, ConfigStruct, MeshStruct, ReportStruct, check, lib, LIB_PATH,
                   PROTOTYPES)

QUAD_DESC = np.dtype([("side", np.int32, (4, 6)), ("corner", np.float64, (8,))])
assert QUAD_DESC.itemsize == 160

FORM_FP64_EXACT = 0
FORM_FP32_FLUX = 1

NFIELDS = 4


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def ip(a):
    return _p(a, C.c_int)


def dp(a):
    return _p(a, C.c_double)


def _iref(v):
    return C.byref(C.c_int(int(v)))


# --------------------------------------------------------------------- config
class Config:
    """The reference's physics configuration (physics_var_*.h) + extensions.

    ``cfl`` is the *effective* CFL: reading an input.physics file applies
    the reference's ``cfl = 0.25*cfl*time_scheme`` (physics_initialize.c:193);
    :meth:`from_input` does the same for keyword arguments.
    """

    def __init__(self, **kw):
        s = ConfigStruct()
        lib().amrgpu_config_defaults(C.byref(s))
        self._s = s
        for k, v in kw.items():
            self[k] = v

    @classmethod
    def from_input(cls, cfl=1.0, time_scheme=1, **kw):
        """Build as physics_initialize.c does from input.physics values."""
        c = cls(time_scheme=time_scheme, **kw)
        c["cfl"] = 0.25 * cfl * time_scheme
        return c

    @classmethod
    def read(cls, path):
        c = cls()
        check(lib().amrgpu_config_read(str(path).encode(), C.byref(c._s)), "config_read")
        return c

    @classmethod
    def current(cls):
        c = cls()
        check(lib().amrgpu_config_get(C.byref(c._s)), "config_get")
        return c

    def apply(self):
        """Make this the library's global configuration."""
        check(lib().amrgpu_config_set(C.byref(self._s)), "config_set")
        return self

    def __setitem__(self, k, v):
        if k in ("bc", "amr_tag_methods", "amr_tag_tolerances", "ic_params"):
            arr = getattr(self._s, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(self._s, k, v)

    def __getitem__(self, k):
        v = getattr(self._s, k)
        if k in ("bc", "amr_tag_methods", "amr_tag_tolerances", "ic_params"):
            return list(v)
        return v

    def as_dict(self):
        return {f: self[f] for f, _ in ConfigStruct._fields_}


# --------------------------------------------------------------------- mesh
class Mesh:
    """Flat arrays of one mesh epoch, as src/amr/src/amr_external.c builds them.

    ``sizes`` (optional): the patch size of every quad for a mesh that mixes
    8x8 and 16x16 patches; cell_info[3q+2] is then the running sum of
    4 n^2 (the reference's own offset layout) and ``n`` the largest size."""

    def __init__(self, n, cell_info, face_info, geom, nface, dof, nghost=0, sizes=None):
        self.n = int(n)
        self.cell_info = np.ascontiguousarray(cell_info, dtype=np.int32)
        self.face_info = np.ascontiguousarray(face_info, dtype=np.int32)
        self.geom = np.ascontiguousarray(geom, dtype=np.float64)
        self.nface = int(nface)
        self.dof = int(dof)
        self.nghost = int(nghost)
        self.ncell = len(self.cell_info) // 3 - self.nghost
        self.sizes = None if sizes is None else np.ascontiguousarray(sizes, dtype=np.int32)

    @property
    def ncells(self):
        if self.sizes is not None:
            return int((self.sizes.astype(np.int64) ** 2).sum())
        return self.ncell * self.n * self.n

    def offsets(self):
        """First cell of every quad (cell_info[2] / 4)."""
        return (self.cell_info[2::3][: self.ncell] // NFIELDS).astype(np.int64)

    def struct(self):
        return MeshStruct(self.ncell, self.nghost, self.nface, self.dof, ip(self.cell_info),
                          ip(self.face_info), dp(self.geom))

    def levels(self):
        return self.cell_info[1::3][: self.ncell].copy()


class ForestMesh:
    """The mesh of a forest as a session built it on the device
    (Session.regrid_forest): sizes at once, the host arrays (cell_info,
    face_info, geom) from amrgpu_forest_external on first use -- valid while
    the forest is unchanged."""

    def __init__(self, forest, n, nface, rule=None):
        self.forest = forest
        self.n = int(n)
        self.ncell = forest.num_quads
        self.nghost = 0
        self.nface = int(nface)
        # mixed patch sizes by the session's level rule
        self.sizes = None if rule is None else forest.patch_sizes(rule)
        self.dof = NFIELDS * (self.ncells if self.sizes is not None else self.n * self.n * self.ncell)
        self._version = forest.version
        self._full = None

    @property
    def ncells(self):
        if self.sizes is not None:
            return int((self.sizes.astype(np.int64) ** 2).sum())
        return self.ncell * self.n * self.n

    def full(self):
        if self._full is None:
            if self.forest.version != self._version:
                raise RuntimeError("the forest changed since this mesh was built")
            self._full = self.forest.mesh(self.n) if self.sizes is None else self.forest.mesh_mixed(self.sizes)
        return self._full

    def __getattr__(self, name):
        if name in ("cell_info", "face_info", "geom", "struct", "levels", "offsets"):
            return getattr(self.full(), name)
        raise AttributeError(name)


class Forest:
    """Host quadtree forest on a brick of trees (stands in for p4est)."""

    def __init__(self, nx=1, ny=1, periodic=(0, 0), lo=(0.0, 0.0, 0.0), scale=1.0, level=0):
        L = lib()
        self._f = L.amrgpu_forest_new_brick(int(nx), int(ny), int(periodic[0]), int(periodic[1]),
                                            float(lo[0]), float(lo[1]), float(lo[2]), float(scale),
                                            int(level))
        if not self._f:
            raise AmrGpuError(L.amrgpu_last_error(), "forest_new_brick")
        self.scale = float(scale)
        self.version = 0  # bumped by every change of the leaves

    def __del__(self):
        f = getattr(self, "_f", None)
        if f and lib is not None:
            try:
                lib().amrgpu_forest_destroy(f)
            except Exception:
                pass
            self._f = None

    @property
    def num_quads(self):
        return lib().amrgpu_forest_num_quads(self._f)

    def write_vtk(self, path, n, soln, subgrid=False):
        """Unstructured VTK (.vtu) of the forest and an AoS state (amrgpu_write_vtk)."""
        a = np.ascontiguousarray(soln, np.float64)
        check(lib().amrgpu_write_vtk(str(path).encode(), self._f, int(n), dp(a), int(bool(subgrid))), "write_vtk")

    def save_checkpoint(self, path, n, soln, istep=0, time=0.0):
        a = np.ascontiguousarray(soln, np.float64)
        check(lib().amrgpu_checkpoint_write(str(path).encode(), self._f, int(n), dp(a), int(istep), float(time)),
              "checkpoint_write")

    @classmethod
    def load_checkpoint(cls, path):
        """(forest, n, soln, istep, time) from amrgpu_checkpoint_write's file."""
        nq, n, ist = C.c_int(0), C.c_int(0), C.c_int(0)
        t = C.c_double(0.0)
        check(lib().amrgpu_checkpoint_read_header(str(path).encode(), C.byref(nq), C.byref(n), C.byref(ist),
                                                  C.byref(t)), "checkpoint_read_header")
        soln = np.zeros(4 * n.value * n.value * nq.value, np.float64)
        h = C.c_void_p()
        check(lib().amrgpu_checkpoint_read(str(path).encode(), C.byref(h), dp(soln), soln.size), "checkpoint_read")
        f = cls.__new__(cls)
        f._f = h.value
        f.scale = None
        f.version = 0
        return f, n.value, soln, ist.value, t.value

    def quads(self):
        n = self.num_quads
        tree = np.zeros(n, np.int32)
        level = np.zeros(n, np.int32)
        x = np.zeros(n, np.int64)
        y = np.zeros(n, np.int64)
        check(lib().amrgpu_forest_quads(self._f, ip(tree), ip(level), _p(x, C.c_int64), _p(y, C.c_int64)))
        return tree, level, x, y

    def begin_regrid(self):
        lib().amrgpu_forest_begin_regrid(self._f)

    def refine(self, flags, max_level=30):
        fl = np.ascontiguousarray(flags, dtype=np.int32)
        assert len(fl) == self.num_quads
        self.version += 1
        return lib().amrgpu_forest_refine(self._f, ip(fl), int(max_level))

    def coarsen(self, flags, min_level=0):
        fl = np.ascontiguousarray(flags, dtype=np.int32)
        assert len(fl) == self.num_quads
        self.version += 1
        return lib().amrgpu_forest_coarsen(self._f, ip(fl), int(min_level))

    def adapt(self, tags, refine_value, coarsen_value, min_level, max_level):
        """begin_regrid, store the tags, refine the quads tagged refine_value
        below max_level (children keep tag 1), coarsen the complete families
        tagged coarsen_value above min_level -- in one call
        (amrgpu_forest_adapt)."""
        t = np.ascontiguousarray(tags, dtype=np.int32)
        assert len(t) == self.num_quads
        self.version += 1
        r = lib().amrgpu_forest_adapt(self._f, ip(t), int(refine_value), int(coarsen_value), int(min_level),
                                      int(max_level))
        if r < 0:
            raise AmrGpuError(-r, "forest_adapt")
        return r

    def balance(self, session=None):
        """2:1 balance; with a session, each pass runs on its GPU
        (amrgpu_forest_balance_device, same result)."""
        self.version += 1
        if session is not None:
            r = lib().amrgpu_forest_balance_device(self._f, session._s)
            if r < 0:
                raise AmrGpuError(-r, "forest_balance_device")
            return r
        r = lib().amrgpu_forest_balance(self._f)
        if r < 0:
            raise AmrGpuError(3, "forest_balance")
        return r

    def is_balanced(self):
        return bool(lib().amrgpu_forest_is_balanced(self._f))

    def set_tags(self, tags):
        t = np.ascontiguousarray(tags, dtype=np.int32)
        check(lib().amrgpu_forest_set_tags(self._f, ip(t)))

    def get_tags(self):
        t = np.zeros(self.num_quads, np.int32)
        check(lib().amrgpu_forest_get_tags(self._f, ip(t)))
        return t

    def remap(self):
        n = self.num_quads
        kind = np.zeros(n, np.int32)
        src = np.zeros(n, np.int32)
        check(lib().amrgpu_forest_remap(self._f, ip(kind), ip(src)))
        return kind, src

    def mesh(self, n):
        L = lib()
        nq = self.num_quads
        cell_info = np.zeros(3 * nq, np.int32)
        face_info = np.full(11 * max(L.amrgpu_forest_max_faces(self._f), 1), -1, np.int32)
        geom = np.zeros(12 * nq, np.float64)
        nface = C.c_int(0)
        dof = C.c_int(0)
        check(L.amrgpu_forest_external(self._f, int(n), NFIELDS, ip(cell_info), ip(face_info), dp(geom),
                                       C.byref(nface), C.byref(dof)), "forest_external")
        return Mesh(n, cell_info, face_info[: 11 * nface.value].copy(), geom, nface.value, dof.value)

    def initialize(self, n):
        """Initial condition of every quad from the global configuration (AoS).
        ``n`` may be a per-quad array of patch sizes (a mixed mesh): every
        quad then gets its own size's initial patch, in mesh order."""
        if np.ndim(n) == 0:
            soln = np.zeros(NFIELDS * int(n) * int(n) * self.num_quads, np.float64)
            check(lib().amrgpu_forest_initialize(self._f, int(n), dp(soln)), "forest_initialize")
            return soln
        sizes = np.asarray(n, np.int64)
        per = {int(k): self.initialize(int(k)).reshape(self.num_quads, -1) for k in np.unique(sizes)}
        return np.concatenate([per[int(k)][q] for q, k in enumerate(sizes)]) if len(sizes) else np.zeros(0)

    def patch_sizes(self, size_of_level):
        """Per-quad patch sizes from a level -> size rule (a callable, or a
        sequence indexed by level)."""
        _, level, _, _ = self.quads()
        if callable(size_of_level):
            table = np.array([int(size_of_level(lv)) for lv in range(32)], np.int32)
        else:
            t = np.asarray(size_of_level, np.int32)
            table = t[np.minimum(np.arange(32), len(t) - 1)]
        return table[level]

    def mesh_mixed(self, sizes):
        """The mesh with per-quad patch sizes (8 or 16): the forest's arrays
        with cell_info[3q+2] = 4 * (cells of the quads before q) and dof the
        sum of 4 n^2."""
        sizes = np.asarray(sizes, np.int32)
        m = self.mesh(int(sizes.max()) if len(sizes) else 16)
        cells = sizes.astype(np.int64) ** 2
        off = np.concatenate([[0], np.cumsum(cells)[:-1]]) if len(cells) else np.zeros(0, np.int64)
        ci = m.cell_info.copy()
        ci[2::3] = (NFIELDS * off).astype(np.int32)
        return Mesh(m.n, ci, m.face_info, m.geom, m.nface, int(NFIELDS * cells.sum()), sizes=sizes)


# --------------------------------------------------------------------- session
class Session:
    """Device-resident state of one mesh epoch (see amrgpu_session_* in amrgpu.h)."""

    def __init__(self, mesh, config=None, form=None):
        L = lib()
        if config is not None:
            if form is not None:
                config["form"] = form
            config.apply()
        elif form is not None:
            c = Config.current()
            c["form"] = form
            c.apply()
        self.mesh = mesh
        h = C.c_void_p()
        ms = mesh.struct()
        check(L.amrgpu_session_create(C.byref(h), C.byref(ms), None), "session_create")
        self._s = h

    def close(self):
        if getattr(self, "_s", None) and lib is not None:
            try:
                lib().amrgpu_session_destroy(self._s)
            except Exception:
                pass
            self._s = None

    def __del__(self):
        self.close()

    def set_form(self, form):
        check(lib().amrgpu_session_set_form(self._s, int(form)), "set_form")

    def launch_variants(self):
        """The compiled (quads per block, threads) launch shapes for this session."""
        q = np.zeros(64, np.int32)
        t = np.zeros(64, np.int32)
        k = lib().amrgpu_session_launch_variants(self._s, ip(q), ip(t), 64)
        return list(zip(q[:k].tolist(), t[:k].tolist()))

    def set_launch_variant(self, index):
        check(lib().amrgpu_session_set_launch_variant(self._s, int(index)), "set_launch_variant")

    def launch_variant(self):
        return lib().amrgpu_session_launch_variant(self._s)

    def launch_variant_info(self, index):
        """(quads per block, threads, min blocks per SM, is_sweep) of a variant."""
        v = [C.c_int() for _ in range(4)]
        check(lib().amrgpu_session_launch_variant_info(self._s, int(index), *[C.byref(x) for x in v]),
              "launch_variant_info")
        return tuple(x.value for x in v)

    def autotune(self, retime=False):
        """Runs the library's stage-launch autotuner now (see
        amrgpu_session_autotune); returns the chosen variant index and shape."""
        check(lib().amrgpu_session_autotune(self._s, int(bool(retime))), "autotune")
        k = self.launch_variant()
        qpb, thr = self.launch_variants()[k]
        return {"variant": k, "quads_per_block": qpb, "threads": thr}

    def set_launch(self, qpb, threads):
        check(lib().amrgpu_session_set_launch(self._s, int(qpb), int(threads)), "set_launch")

    def upload(self, soln):
        a = np.ascontiguousarray(soln, dtype=np.float64)
        check(lib().amrgpu_session_upload(self._s, dp(a)), "upload")

    def download(self, out=None):
        """AoS state of the local quads; into ``out`` (e.g. pinned host
        memory, dof doubles) when given."""
        if out is None:
            out = np.empty(self.mesh.dof, np.float64)
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size < self.mesh.dof:
            raise ValueError("download: out must be a contiguous float64 array of at least dof values")
        check(lib().amrgpu_session_download(self._s, dp(out)), "download")
        return out

    def step(self, nsteps, graph_steps=0):
        if graph_steps:
            check(lib().amrgpu_session_step_graph(self._s, int(nsteps), int(graph_steps)), "step_graph")
        else:
            check(lib().amrgpu_session_step(self._s, int(nsteps)), "step")

    def sync(self):
        r = ReportStruct()
        check(lib().amrgpu_session_sync(self._s, C.byref(r)), "sync")
        return {"steps": r.steps_done, "time": r.time, "dt_last": r.dt_last,
                "residual_norm": r.residual_norm, "error": r.error, "nan": r.nan_detected}

    def rhs(self):
        out = np.empty(self.mesh.dof, np.float64)
        check(lib().amrgpu_session_rhs(self._s, dp(out)), "rhs")
        return out

    def cfl_dt(self):
        v = C.c_double(0.0)
        check(lib().amrgpu_session_cfl_dt(self._s, C.byref(v)), "cfl_dt")
        return v.value

    def totals(self):
        t = np.zeros(4, np.float64)
        check(lib().amrgpu_session_totals(self._s, dp(t)), "totals")
        return t

    def tag(self):
        t = np.zeros(self.mesh.ncell, np.int32)
        check(lib().amrgpu_session_tag(self._s, ip(t)), "tag")
        return t

    def remap_from(self, other, kind, src):
        k = np.ascontiguousarray(kind, np.int32)
        s = np.ascontiguousarray(src, np.int32)
        check(lib().amrgpu_session_remap(self._s, other._s, ip(k), ip(s)), "remap")

    def regrid(self, mesh, kind, src):
        """In place: take the new mesh and remap the state by kind/src."""
        k = np.ascontiguousarray(kind, np.int32)
        s = np.ascontiguousarray(src, np.int32)
        ms = mesh.struct()
        check(lib().amrgpu_session_regrid(self._s, C.byref(ms), ip(k), ip(s)), "regrid")
        self.mesh = mesh

    def set_patch_rule(self, size_of_level):
        """Mixed 8x8 / 16x16 patches by level for the regrids built on the
        device (a callable level -> size, a sequence indexed by level, or
        None to clear); see amrgpu_session_set_patch_rule."""
        if size_of_level is None:
            check(lib().amrgpu_session_set_patch_rule(self._s, None, 0), "set_patch_rule")
            self._rule = None
            return
        f = size_of_level if callable(size_of_level) else (lambda lv: size_of_level[min(lv, len(size_of_level) - 1)])
        table = np.array([int(f(lv)) for lv in range(32)], np.int32)
        check(lib().amrgpu_session_set_patch_rule(self._s, ip(table), 32), "set_patch_rule")
        self._rule = [int(v) for v in table]

    def regrid_forest(self, forest):
        """In place, from the forest after refine / coarsen / balance: quad
        descriptors built on the device, state remapped by the forest's
        remap table (amrgpu_session_regrid_forest)."""
        check(lib().amrgpu_session_regrid_forest(self._s, C.c_void_p(forest._f)), "regrid_forest")
        self.mesh = ForestMesh(forest, self.mesh.n, lib().amrgpu_session_face_count(self._s),
                               getattr(self, "_rule", None))

    def balance_regrid(self, forest):
        """forest.balance(session=self) and self.regrid_forest(forest) in one
        call: the descriptors are built from the balanced leaves on the
        device (amrgpu_session_balance_regrid)."""
        forest.version += 1
        check(lib().amrgpu_session_balance_regrid(self._s, C.c_void_p(forest._f)), "balance_regrid")
        self.mesh = ForestMesh(forest, self.mesh.n, lib().amrgpu_session_face_count(self._s),
                               getattr(self, "_rule", None))

    def adapt_regrid(self, forest, min_level, max_level, tags=None, refine_value=1, coarsen_value=0,
                     return_tags=False):
        """The whole regrid in one call (amrgpu_session_adapt_regrid): the
        session's tags (or `tags`, one per quad), forest.adapt(tags,
        refine_value, coarsen_value, min_level, max_level) and
        self.balance_regrid(forest). The refine / coarsen also runs on the
        device when the session's last regrid came from this unchanged
        forest. return_tags: also return the tags used."""
        n = self.mesh.ncell
        assert forest.num_quads == n
        tin = None if tags is None else np.ascontiguousarray(tags, dtype=np.int32)
        if tin is not None:
            assert len(tin) == n
        tout = np.zeros(n, np.int32) if return_tags else None
        forest.version += 1
        check(lib().amrgpu_session_adapt_regrid(self._s, C.c_void_p(forest._f), None if tin is None else ip(tin),
                                                 None if tout is None else ip(tout), int(refine_value),
                                                 int(coarsen_value), int(min_level), int(max_level)),
              "adapt_regrid")
        self.mesh = ForestMesh(forest, self.mesh.n, lib().amrgpu_session_face_count(self._s),
                               getattr(self, "_rule", None))
        return tout

    def holds_forest(self, forest):
        """True when the next adapt_regrid of `forest` adapts on the device
        (amrgpu_session_holds_forest)."""
        return bool(lib().amrgpu_session_holds_forest(self._s, C.c_void_p(forest._f)))

    def reserve(self, cells, quads):
        """Grows the session's buffers now for meshes of up to `cells` cells
        and `quads` quads, so that regrids within those bounds allocate
        nothing (amrgpu_session_reserve)."""
        check(lib().amrgpu_session_reserve(self._s, int(cells), int(quads)), "reserve")

    def quad_descriptors(self):
        """The device quad descriptors as a structured array (kind, nbr0,
        nbr1, rank, level, bc per side; 8 corner doubles)."""
        n = self.mesh.ncell
        out = np.zeros(n, dtype=QUAD_DESC)
        k = lib().amrgpu_session_quad_descriptors(self._s, out.ctypes.data_as(C.c_void_p), n)
        if k < 0:
            raise AmrGpuError(-k, "quad_descriptors")
        return out

    def state_ptr(self, field):
        return lib().amrgpu_session_state_device(self._s, int(field))

    def stream(self):
        return lib().amrgpu_session_stream(self._s)

    def launch_count(self):
        return lib().amrgpu_session_launch_count(self._s)


# --------------------------------------------------------------------- reference ABI
def initialize_solver(mesh_scale, nelem_subgrid, nlevels=0, rank=0):
    """hpc_amr_initialize_solver: reads input.physics from the working directory."""
    L = lib()
    L.hpc_amr_initialize_solver(_iref(rank), _iref(2), C.byref(C.c_double(mesh_scale)), _iref(nlevels),
                                _iref(NFIELDS), _iref(2), _iref(nelem_subgrid), _iref(3), _iref(11),
                                _iref(0), _iref(0), _iref(2))
    return L.amrgpu_last_error()


def evolve_solver(mesh, soln, istep, entry="hpc_amr_evolve_solver"):
    """One call of the reference's evolve entry point on host arrays.

    ``soln`` (AoS, dof doubles) is updated in place. Returns a dict with
    istep, the regrid/visualize/checkpoint/evolve_solution flags and the
    three accumulated timers, as src/amr/src/amr_external.c:85-106 sees them.
    """
    L = lib()
    fn = getattr(L, entry)
    dim, uns, nf, n = C.c_int(2), C.c_int(0), C.c_int(NFIELDS), C.c_int(mesh.n)
    ncell, nghost, nface, dof = C.c_int(mesh.ncell), C.c_int(0), C.c_int(mesh.nface), C.c_int(mesh.dof)
    nsend, nrecv = C.c_int(0), C.c_int(0)
    send = np.zeros(2, np.int32)
    recv = np.zeros(2, np.int32)
    sizes = np.full(max(mesh.ncell, 1), NFIELDS * mesh.n * mesh.n, np.int32)
    ist = C.c_int(int(istep))
    regrid, vis, chk, evo = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(1)
    tt, ct, rt = C.c_double(0), C.c_double(0), C.c_double(0)
    assert soln.dtype == np.float64 and soln.flags.c_contiguous
    fn(C.byref(dim), C.byref(uns), C.byref(nf), C.byref(n), C.byref(ncell), C.byref(nghost), C.byref(nface),
       C.byref(dof), ip(mesh.cell_info), ip(mesh.face_info), C.byref(nsend), C.byref(nrecv), ip(send), ip(recv),
       ip(sizes), dp(mesh.geom), dp(soln), C.byref(ist), C.byref(regrid), C.byref(vis), C.byref(chk),
       C.byref(evo), 0, C.byref(tt), C.byref(ct), C.byref(rt))
    return {"istep": ist.value, "regrid": regrid.value, "visualize": vis.value, "checkpoint": chk.value,
            "evolve_solution": evo.value, "total_time": tt.value, "compute_time": ct.value,
            "residual_time": rt.value, "error": L.amrgpu_last_error()}


def last_error():
    L = lib()
    return L.amrgpu_last_error(), L.amrgpu_last_error_message().decode(errors="replace")


def clear_error():
    lib().amrgpu_clear_error()
