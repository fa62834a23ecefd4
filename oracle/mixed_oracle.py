"""Residual of a mesh that mixes 8x8 and 16x16 patches, in FP64 -- TEST
INFRASTRUCTURE (only tests/ use it, to check the GPU's mixed-size sweep).

The reference fixes one patch size per build (src/amr/src/var_defines.h:29-32),
so mixed sizes have no reference counterpart; this module restates the
library's face rule for them with the reference's own face physics
(flux_roe_2d, flux_2d_module.F90:63-182, through oracle.flux) and plain
loops, for small periodic meshes of axis-aligned rectangles:

* interior faces of a patch and every edge whose two quads have the same
  patch size follow the reference (physics_rhs_structured.c:73-276,
  solver_residual_subgrid_2d_module.F90:82-126): a full edge pairs the cells
  at the same position, a coarse hanging edge pairs its cell m with cell m of
  each fine quad (two fluxes), with the normal length cell_h of the fine
  level, physics_residual_face_full_hang_structured.c;
* an edge whose quads have different patch sizes is cut into pieces of the
  finer side's cell length; each piece pairs the two cells that cover it,
  its flux (normal length = that cell length) is added to both.

A cell's residual is -(sum of +F at its high faces - F at its low faces) /
volume, edge contributions summed in edge order.
"""
import numpy as np

from . import oracle as O


def _cell_h(h_base, level, n):
    return h_base * (1.0 / 2.0 ** level) / n


def _facing(s, p, n):
    if s == 0:
        return p * n + (n - 1)
    if s == 1:
        return p * n
    if s == 2:
        return (n - 1) * n + p
    return p


def _own(s, m, n):
    if s == 0:
        return m * n
    if s == 1:
        return m * n + n - 1
    if s == 2:
        return m
    return (n - 1) * n + m


def sides(mesh):
    """Per quad and side: (kind, nbr0, nbr1, level) with kind 'full',
    'coarse' (this quad coarse, two fine neighbours), 'fine'; level is the
    level whose cell_h sizes the face (the left quad's for a full face, the
    fine level for a hanging face), as physics_rhs_structured.c decodes
    face_info."""
    nq = mesh.ncell
    level = mesh.cell_info[1::3]
    out = [[None] * 4 for _ in range(nq)]
    fi = mesh.face_info.reshape(-1, 11)
    for f in range(mesh.nface):
        ftype, side, cell = int(fi[f, 0]), int(fi[f, 1]), int(fi[f, 2])
        if ftype == 2:
            left = int(fi[f, 3]) if side % 2 == 0 else cell
            right = cell if side % 2 == 0 else int(fi[f, 3])
            hs = side + 1 if side % 2 == 0 else side
            lv = int(level[left])
            out[left][hs] = ("full", right, -1, lv)
            out[right][hs - 1] = ("full", left, -1, lv)
        elif ftype == 3:
            f0, f1 = int(fi[f, 3]), int(fi[f, 4])
            lv = int(level[f0])
            fine_side = side + 1 if side % 2 == 0 else side - 1
            if mesh.sizes is not None and mesh.sizes[f0] != mesh.sizes[f1]:
                raise ValueError("the two fine quads of a hanging edge must share one patch size")
            out[cell][side] = ("coarse", f0, f1, lv)
            out[f0][fine_side] = ("fine", cell, -1, lv)
            out[f1][fine_side] = ("fine", cell, -1, lv)
        else:
            raise ValueError("face type %d: this restatement handles periodic meshes only" % ftype)
    return out


def rhs(mesh, soln, h_base):
    """Residual (AoS, like soln) of the mixed-size mesh ``mesh`` (with
    ``mesh.sizes``) for the state ``soln``."""
    nq = mesh.ncell
    n_of = np.asarray(mesh.sizes, np.int64)
    base = (mesh.cell_info[2::3][:nq] // 4).astype(np.int64)
    g = mesh.geom.reshape(nq, 4, 3)
    Q = np.asarray(soln, np.float64).reshape(-1, 4)
    S = sides(mesh)
    out = np.zeros_like(Q)

    def q(quad, cell):
        return Q[base[quad] + cell]

    def along(quad, s):
        return g[quad, 0, 1] if s < 2 else g[quad, 0, 0]

    def edge_len(quad, s):
        return abs(g[quad, 2, 1] - g[quad, 0, 1]) if s < 2 else abs(g[quad, 1, 0] - g[quad, 0, 0])

    def face(low, high, s, h):
        nrm = (h, 0.0) if s < 2 else (0.0, h)
        return O.flux(low, high, nrm)

    for quad in range(nq):
        N = int(n_of[quad])
        hx = (g[quad, 1, 0] - g[quad, 0, 0]) / N
        hy = (g[quad, 2, 1] - g[quad, 0, 1]) / N
        vol = hx * hy
        acc = np.zeros((N * N, 4))
        # interior faces
        for j in range(N):
            for i in range(1, N):
                F = face(q(quad, j * N + i - 1), q(quad, j * N + i), 0, hy)
                acc[j * N + i - 1] += F
                acc[j * N + i] -= F
        for j in range(1, N):
            for i in range(N):
                F = face(q(quad, (j - 1) * N + i), q(quad, j * N + i), 2, hx)
                acc[(j - 1) * N + i] += F
                acc[j * N + i] -= F
        # edges, each own edge cell's pieces summed in edge order
        for s in range(4):
            kind, nb0, nb1, lv = S[quad][s]
            nn = int(n_of[nb0])
            for m in range(N):
                own = _own(s, m, N)
                E = np.zeros(4)
                if nn == N:
                    hc = _cell_h(h_base, lv, N)
                    pairs = [(nb0, _facing(s, m, N))]
                    if kind == "coarse":
                        pairs.append((nb1, _facing(s, m, N)))
                    for nb, fc in pairs:
                        lo, hi = (q(quad, own), q(nb, fc)) if s & 1 else (q(nb, fc), q(quad, own))
                        E = E + face(lo, hi, s, hc)
                else:
                    if kind == "full":
                        hp = min(_cell_h(h_base, lv, N), _cell_h(h_base, lv, nn))
                        if nn > N:
                            pieces = [(nb0, m * (nn // N) + k) for k in range(nn // N)]
                        else:
                            pieces = [(nb0, m * nn // N)]
                    elif kind == "coarse":
                        hp = min(_cell_h(h_base, lv - 1, N), _cell_h(h_base, lv, nn))
                        lower, upper = (nb1, nb0) if along(nb1, s) < along(nb0, s) else (nb0, nb1)
                        r = 2 * nn // N if 2 * nn >= N else 1
                        gs = [m * r + k for k in range(r)] if 2 * nn >= N else [m * 2 * nn // N]
                        pieces = [((lower, upper)[gg // nn], gg % nn) for gg in gs]
                    else:
                        hp = min(_cell_h(h_base, lv, N), _cell_h(h_base, lv - 1, nn))
                        half = 1 if along(quad, s) - along(nb0, s) > 0.25 * edge_len(quad, s) else 0
                        pieces = [(nb0, (half * N + m) * nn // (2 * N))]
                    for nb, p in pieces:
                        fc = _facing(s, p, nn)
                        lo, hi = (q(quad, own), q(nb, fc)) if s & 1 else (q(nb, fc), q(quad, own))
                        E = E + face(lo, hi, s, hp)
                # +F at a high face (sides 1, 3), -F at a low face (0, 2)
                acc[own] += E if s & 1 else -E
        out[base[quad]:base[quad] + N * N] = -acc / vol
    return out.reshape(-1)
