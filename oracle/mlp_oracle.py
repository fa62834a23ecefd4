"""CPU restatement of the learned refinement indicator -- TEST INFRASTRUCTURE.

Only tests/ use this module, to verify the GPU indicator
(amr-demo_b200/csrc/mlp.cu); the product path never calls it. The indicator
has no reference counterpart; what it stands in for is the reference's
plain tagger (solver_tag_feature.F90:9-52), and its labels come from the
plain indicator's density-jump quantity (the tag kernel's method 5).

Everything is NumPy in FP64. With ``bf16=True`` the values the GPU stores
in BF16 (features, weights, hidden activations, dL, dZ) are rounded to BF16
at the same points, so the GPU's remaining differences are FP32
accumulation and FP32 GELU: a few ulp before a BF16 rounding, i.e. rare
one-ulp BF16 flips. With ``bf16=False`` the network is plain FP64, which
the finite-difference test uses to check this module's own backward pass.
"""
import math

import numpy as np

NIN, NH1, NH2, NOUT = 400, 128, 64, 3
NPARAMS = NH1 * NIN + NH1 + NH2 * NH1 + NH2 + NOUT * NH2 + NOUT
FEAT_SCALE = 10.0


# ------------------------------------------------------------------ BF16
def f32_to_bf16_bits(x):
    """Round FP32 to BF16 (round to nearest even); bit patterns."""
    b = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    b = b + 0x7FFF + ((b >> 16) & 1)
    return (b >> 16).astype(np.uint16)


def bf16_bits_to_f64(bits):
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def bf16(x):
    """FP64 -> FP32 -> BF16 -> FP64 (the GPU's __float2bfloat16_rn of a float)."""
    return bf16_bits_to_f64(f32_to_bf16_bits(np.asarray(x, np.float64).astype(np.float32)))


# ------------------------------------------------------------------ mesh decode
def sides(mesh):
    """Per quad and side: kind (0 boundary / none, 1 one neighbour -- a
    conforming face or the fine side of a hanging face --, 2 the coarse side
    of a hanging face) and the neighbour ids, decoded from the reference's
    face_info (stride 11: ftype, side, cell, 4 neighbour ids, 4 sides;
    physics_rhs_structured.c:73-262 reads it the same way)."""
    nq = mesh.ncell
    kind = np.zeros((nq, 4), np.int64)
    nbr = np.zeros((nq, 4, 2), np.int64)
    fi = np.asarray(mesh.face_info).reshape(-1, 11)[: mesh.nface]
    for f in fi:
        ftype, side, cell = int(f[0]), int(f[1]), int(f[2])
        if ftype == 2:
            left, right = (int(f[3]), cell) if side % 2 == 0 else (cell, int(f[3]))
            hs = side + 1 if side % 2 == 0 else side
            if left < nq:
                kind[left, hs], nbr[left, hs] = 1, (right, right)
            if right < nq:
                kind[right, hs - 1], nbr[right, hs - 1] = 1, (left, left)
        elif ftype == 3:
            fs = side + 1 if side % 2 == 0 else side - 1
            kind[cell, side], nbr[cell, side] = 2, (int(f[3]), int(f[4]))
            for k in (3, 4):
                if int(f[k]) < nq:
                    kind[int(f[k]), fs], nbr[int(f[k]), fs] = 1, (cell, cell)
    return kind, nbr


def _facing(q, s, m):
    """Cell of patch q (array [j][i][f]) that faces side s of its neighbour
    at position m: the neighbour's opposite edge."""
    n = q.shape[0]
    return (q[m, n - 1], q[m, 0], q[n - 1, m], q[0, m])[s]


def _own_edge(q, s, m):
    n = q.shape[0]
    return (q[m, 0], q[m, n - 1], q[0, m], q[n - 1, m])[s]


# ------------------------------------------------------------------ features / labels
def features(soln, mesh, n):
    """BF16 bit patterns [nquad x 400] of the patch features (see
    features_kernel in csrc/mlp.cu): the patch box-averaged to 8x8, a
    one-cell ring from the flux-paired neighbour cells, each field
    normalised by the patch mean state."""
    nq = mesh.ncell
    Q = np.asarray(soln, np.float64).reshape(-1, n, n, 4)
    kind, nbr = sides(mesh)
    R = n // 8
    out = np.zeros((nq, NIN), np.uint16)
    for q in range(nq):
        P = np.zeros((4, 10, 10))
        for J in range(8):
            for I in range(8):
                s = np.zeros(4)
                for dj in range(R):
                    for di in range(R):
                        s = s + Q[q, R * J + dj, R * I + di]
                P[:, J + 1, I + 1] = s * (1.0 / (R * R))
        for sd in range(4):
            for M in range(8):
                s = np.zeros(4)
                for dm in range(R):
                    m = R * M + dm
                    if kind[q, sd] == 1:
                        s = s + _facing(Q[nbr[q, sd, 0]], sd, m)
                    elif kind[q, sd] == 2:
                        s = s + 0.5 * (_facing(Q[nbr[q, sd, 0]], sd, m) + _facing(Q[nbr[q, sd, 1]], sd, m))
                    else:
                        s = s + _own_edge(Q[q], sd, m)
                v = s * (1.0 / R)
                if sd == 0:
                    P[:, M + 1, 0] = v
                elif sd == 1:
                    P[:, M + 1, 9] = v
                elif sd == 2:
                    P[:, 0, M + 1] = v
                else:
                    P[:, 9, M + 1] = v
        for cj, ci, pj, pi in ((0, 0, 1, 1), (0, 9, 1, 8), (9, 0, 8, 1), (9, 9, 8, 8)):
            P[:, cj, ci] = P[:, pj, pi]
        mr, mu, mv, me = (P[f, 1:9, 1:9].sum() / 64.0 for f in range(4))
        pbar = 0.4 * (me - 0.5 * (mu * mu + mv * mv) / mr)
        c2 = 1.4 * pbar / mr
        abar = math.sqrt(max(c2, 1e-24))
        sc = (FEAT_SCALE / mr, FEAT_SCALE / (mr * abar), FEAT_SCALE / (mr * abar), FEAT_SCALE / me)
        mm = (mr, mu, mv, me)
        x = np.concatenate([((P[f] - mm[f]) * sc[f]).ravel() for f in range(4)])
        out[q] = f32_to_bf16_bits(x.astype(np.float32))
    return out


def jumps(soln, mesh, n):
    """Largest relative density jump per quad (the plain indicator's method 5
    quantity): |a - b| / min(a, b) over adjacent cells of the patch and over
    each edge cell and the neighbour cell(s) its face flux pairs it with."""
    Q = np.asarray(soln, np.float64).reshape(-1, n, n, 4)[..., 0]
    kind, nbr = sides(mesh)
    nq = mesh.ncell
    out = np.zeros(nq)
    for q in range(nq):
        p = Q[q]
        J = 0.0
        if n > 1:
            J = max(J, (np.abs(p[:, 1:] - p[:, :-1]) / np.minimum(p[:, 1:], p[:, :-1])).max())
            J = max(J, (np.abs(p[1:, :] - p[:-1, :]) / np.minimum(p[1:, :], p[:-1, :])).max())
        for s in range(4):
            if kind[q, s] == 0:
                continue
            for k in range(2 if kind[q, s] == 2 else 1):
                other = Q[nbr[q, s, k]]
                for m in range(n):
                    a, b = _own_edge(p, s, m), _facing(other, s, m)
                    J = max(J, abs(a - b) / min(a, b))
        out[q] = J
    return out


def labels(J, tol, lo_frac=0.25):
    """0 coarsen (J < lo_frac*tol), 1 refine (J >= tol), 2 keep."""
    J = np.asarray(J)
    return np.where(J >= tol, 1, np.where(J < lo_frac * tol, 0, 2)).astype(np.int32)


# ------------------------------------------------------------------ the network
def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((NH1, NIN), (NH1,), (NH2, NH1), (NH2,), (NOUT, NH2), (NOUT,)):
        k = int(np.prod(shape))
        out.append(p[o:o + k].reshape(shape))
        o += k
    return out


def pack(parts):
    return np.concatenate([np.asarray(a, np.float64).ravel() for a in parts])


_erf = np.vectorize(math.erf)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def forward_backward(params, x, y, bf16_mode=True):
    """Logits [B x 3], mean cross-entropy and the flat gradient of it for
    features x ([B x 400] FP64 values) and labels y."""
    r = bf16 if bf16_mode else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(params)
    W1b, W2b, W3b = r(W1), r(W2), r(W3)
    b1, b2, b3 = (np.asarray(a, np.float32).astype(np.float64) if bf16_mode else a for a in (b1, b2, b3))
    X = np.asarray(x, np.float64)
    B = X.shape[0]
    Z1 = X @ W1b.T + b1
    H1 = r(gelu(Z1))
    Z2 = H1 @ W2b.T + b2
    H2 = r(gelu(Z2))
    L = H2 @ W3b.T + b3
    mx = L.max(axis=1, keepdims=True)
    e = np.exp(L - mx)
    P = e / e.sum(axis=1, keepdims=True)
    Y = np.zeros_like(P)
    Y[np.arange(B), y] = 1.0
    loss = float(np.mean(-np.log(P[np.arange(B), y])))
    dL = r(P - Y)
    dZ2 = r((dL @ W3b) * gelu_grad(Z2))
    dZ1 = r((dZ2 @ W2b) * gelu_grad(Z1))
    g = pack([dZ1.T @ X / B, dZ1.sum(0) / B, dZ2.T @ H1 / B, dZ2.sum(0) / B, dL.T @ H2 / B, dL.sum(0) / B])
    return L, loss, g


def loss_only(params, x, y):
    return forward_backward(params, x, y, bf16_mode=False)[1]


def init_params(seed):
    """The library's deterministic initialisation (MlpState::init):
    U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from splitmix64 of seed and index."""
    M = (1 << 64) - 1
    out = np.zeros(NPARAMS, np.float64)
    fans = [NIN] * 2 + [NH1] * 2 + [NH2] * 2
    sizes = [NH1 * NIN, NH1, NH2 * NH1, NH2, NOUT * NH2, NOUT]
    k = 0
    for fan, sz in zip(fans, sizes):
        for _ in range(sz):
            z = (seed * 0x9E3779B97F4A7C15 + k + 0x632BE59BD9B4E019) & M
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
            z ^= z >> 31
            u = (z >> 11) * (1.0 / 9007199254740992.0)
            out[k] = np.float32((2.0 * u - 1.0) / math.sqrt(fan))
            k += 1
    return out.astype(np.float32)
