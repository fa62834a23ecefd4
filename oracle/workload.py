"""The benchmark's vortex workload built in NumPy -- TEST INFRASTRUCTURE.

Used by bench.py's CPU-baseline legs so that the reference's CPU path is
fed and timed without loading the product library. It produces what the
reference's AMR driver would hand hpc_amr_evolve_solver for a single
periodic tree at a uniform level (external_t, amr_external.c:211-508):

  * quadrants in Morton order (x in the even bits);
  * cell_info = (type 0, level, 4 n^2 * id);
  * geom = the 4 corners of each quadrant by the transfinite map of
    amr_p4est_utilities.c:39-76 (in the same operation order as the
    library's forest, so the arrays are equal bit for bit -- tested);
  * face_info: one full face per (quadrant, side) pair, listed at the first
    of its two quadrants (by index), sides 0..3; side[0] is the odd side's
    quadrant, as p4est orders the two sides of a face inside one tree;
  * the isentropic-vortex initial state of the library's IC 4 (the
    reference's vortex form, initial_condition_2d_module.F90:83-129,
    centred at (xc, yc) with strength beta), evaluated at the sub-cell
    centres; equal to the library's to the rounding of exp / pow.
"""
import math

import numpy as np

NFIELDS = 4
ROOT_LEN = 1 << 30


def _compact(v):
    """Every other bit of v (the inverse of spreading bits for a Morton key)."""
    v = v & 0x5555555555555555
    v = (v | (v >> 1)) & 0x3333333333333333
    v = (v | (v >> 2)) & 0x0F0F0F0F0F0F0F0F
    v = (v | (v >> 4)) & 0x00FF00FF00FF00FF
    v = (v | (v >> 8)) & 0x0000FFFF0000FFFF
    v = (v | (v >> 16)) & 0x00000000FFFFFFFF
    return v


class Mesh:
    """external_t arrays of one rank (the layout the reference's driver and
    the product's Mesh use: cell_info 3 ints, face_info 11 ints, geom 12
    doubles per quadrant)."""

    def __init__(self, n, cell_info, face_info, geom, nface, dof, nghost=0):
        self.n = n
        self.cell_info = np.ascontiguousarray(cell_info, np.int32)
        self.face_info = np.ascontiguousarray(face_info, np.int32)
        self.geom = np.ascontiguousarray(geom, np.float64)
        self.nface = int(nface)
        self.dof = int(dof)
        self.nghost = int(nghost)
        self.ncell = len(self.cell_info) // 3 - self.nghost
        self.ncells = self.ncell * n * n


def uniform_periodic_mesh(level, n, scale=10.0, lo=(0.0, 0.0, 0.0)):
    N = 1 << level
    nq = N * N
    k = np.arange(nq, dtype=np.int64)
    x = _compact(k)
    y = _compact(k >> 1)
    ql = ROOT_LEN >> level
    cell_info = np.zeros((nq, 3), np.int32)
    cell_info[:, 1] = level
    cell_info[:, 2] = NFIELDS * n * n * k
    # corners: the tree's vertices, then the transfinite map of the quadrant
    # (the same expressions as the forest's corner computation)
    v = np.array([[vx * scale + lo[0], vy * scale + lo[1], 0.0 * scale + lo[2]]
                  for vy in (0, 1) for vx in (0, 1)], np.float64)
    intsize = 1.0 / float(ROOT_LEN)
    h2 = 0.5 * intsize * float(ql)
    geom = np.zeros((nq, 4, 3), np.float64)
    X = (x * ql).astype(np.float64)
    Y = (y * ql).astype(np.float64)
    eta_z = 0.0
    c = 0
    for yi in (0, 1):
        eta_y = intsize * Y + h2 * (1.0 + (2 * yi - 1))
        for xi in (0, 1):
            eta_x = intsize * X + h2 * (1.0 + (2 * xi - 1))
            for j in range(3):
                geom[:, c, j] = ((1. - eta_z) * ((1. - eta_y) * ((1. - eta_x) * v[0, j] + eta_x * v[1, j]) +
                                                 eta_y * ((1. - eta_x) * v[2, j] + eta_x * v[3, j])))
            c += 1
    # faces: leaf i, side s (0 -x, 1 +x, 2 -y, 3 +y), neighbour j across
    # the periodic wrap; listed by the first participant, sides in order
    index = np.empty(nq, np.int64)
    index[(y * N + x)] = k
    recs = []
    for s, (dx, dy) in enumerate(((-1, 0), (1, 0), (0, -1), (0, 1))):
        j = index[((y + dy) % N) * N + (x + dx) % N]
        opp = s ^ 1
        same = j == k
        this_first = np.where(same, (s & 1) == 0, (s & 1) == 1)
        emit = (k < j) | (same & ((s & 1) == 0))
        rec = np.full((nq, 11), -1, np.int64)
        rec[:, 0] = 2
        rec[:, 1] = np.where(this_first, s, opp)
        rec[:, 2] = np.where(this_first, k, j)
        rec[:, 3] = np.where(this_first, j, k)
        rec[:, 7] = np.where(this_first, opp, s)
        recs.append((rec, emit))
    order = []
    for s in range(4):
        rec, emit = recs[s]
        order.append(np.stack([k, np.full(nq, s)], axis=1)[emit])
    order = np.concatenate(order)
    order = order[np.lexsort((order[:, 1], order[:, 0]))]
    face_info = np.stack([recs[s][0][i] for i, s in order]) if len(order) else np.zeros((0, 11), np.int64)
    return Mesh(n, cell_info.reshape(-1), face_info.reshape(-1).astype(np.int32), geom.reshape(-1),
                len(face_info), NFIELDS * n * n * nq)


def vortex_state(mesh, xc=5.0, yc=5.0, beta=5.0, a=0.5, gamma=1.4, density=1.0, pressure=1.0,
                 mach=math.sqrt(2.0) / math.sqrt(1.4), alpha=45.0, beta_yaw=0.0):
    """AoS state (soln[f + 4 c]) of the isentropic vortex on every quadrant."""
    n = mesh.n
    g = mesh.geom.reshape(-1, 12)[: mesh.ncell]
    gm1 = gamma - 1.0
    one_o_gm1 = 1.0 / gm1
    pi = 3.141592653589793238462643383279502884197
    two_pi = 6.283185307179586476925286766559005768394
    c0 = math.sqrt(gamma * (pressure / density))
    v0 = mach * c0
    u_in = v0 * math.cos(alpha * pi / 180.0) * math.cos(beta_yaw * pi / 180.0)
    v_in = v0 * math.sin(alpha * pi / 180.0) * math.cos(beta_yaw * pi / 180.0)
    s = 2.0 / float(n)
    idx = np.arange(1, n + 1, dtype=np.float64)
    xi = 0.5 * ((s * (idx - 1.0) - 1.0) + (s * idx - 1.0))  # sub-cell centres in natural coordinates
    om_x, op_x = 0.5 * (1.0 - xi), 0.5 * (1.0 + xi)
    om_e, op_e = om_x, op_x
    # centre (i, j) of quad q: sum over the four corners, left to right
    X = (g[:, None, None, 0] * om_x[None, None, :] * om_e[None, :, None] +
         g[:, None, None, 3] * op_x[None, None, :] * om_e[None, :, None] +
         g[:, None, None, 6] * om_x[None, None, :] * op_e[None, :, None] +
         g[:, None, None, 9] * op_x[None, None, :] * op_e[None, :, None])
    Y = (g[:, None, None, 1] * om_x[None, None, :] * om_e[None, :, None] +
         g[:, None, None, 4] * op_x[None, None, :] * om_e[None, :, None] +
         g[:, None, None, 7] * om_x[None, None, :] * op_e[None, :, None] +
         g[:, None, None, 10] * op_x[None, None, :] * op_e[None, :, None])
    two_a = 2.0 * a
    dT1 = -(gm1 * beta * beta) / (16.0 * a * gamma * pi * pi)
    r2 = (X - xc) * (X - xc) + (Y - yc) * (Y - yc)
    dT = dT1 * np.exp(two_a * (1.0 - r2))
    rho = np.power(1.0 + dT, one_o_gm1)
    ff = beta / two_pi * np.exp(a * (1.0 - r2))
    u = u_in - (Y - yc) * ff
    v = v_in + (X - xc) * ff
    p = pressure + np.power(rho, gamma) - 1.0
    out = np.empty(X.shape + (4,), np.float64)  # [q][j][i][f]
    out[..., 0] = rho
    out[..., 1] = rho * u
    out[..., 2] = rho * v
    out[..., 3] = p * one_o_gm1 + 0.5 * rho * (u * u + v * v)
    return out.reshape(-1)


def vortex_config(n=16, steps=10):
    """The configuration values of the vortex workload as the reference's
    globals take them (cfl already scaled by 0.25 * time_scheme)."""
    return {"time_scheme": 3, "time_steps": steps, "dt": 1.0, "cfl": 0.25 * 0.5 * 3, "coarse_grid_h": 10.0,
            "initial_condition": 4, "gamma": 1.4, "density": 1.0, "pressure": 1.0,
            "mach": math.sqrt(2.0) / math.sqrt(1.4), "alpha": 45.0, "beta": 0.0,
            "checkpoint_interval": 0, "visualization_interval": 0, "regrid_interval": 0,
            "bc": [1] * 6, "final_time": 0.0, "ic_params": [5.0, 5.0, 5.0, 0.5]}
