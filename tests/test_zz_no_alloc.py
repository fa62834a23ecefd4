"""The allocation-free entry point, amrgpu_totals_noalloc.

Some callers of this library cannot let it allocate device memory: an AMR
driver that gives all device memory to its own pool at start-up, or one that
checks conservation inside its time-step loop on a busy device, where the
device-wide synchronisation of cudaMalloc/cudaFree would stall its other
streams. amrgpu_totals_noalloc computes the conservation totals sum(vol*Q_f)
with its scratch in a fixed array of the library's device image instead.

These tests call it through the C ABI, twice in a row (the second call finds
the first call's contents in the shared scratch array), and compare it with
the session-based entry point amrgpu_session_totals, which allocates its own
scratch, within the 1e-12 relative tolerance of the conservation tests. The
file sorts last so that a run stopping at the first failure has run every
other test before it.
"""
import os

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.gpu

os.environ.setdefault("AMRGPU_QUIET", "1")

AMRGPU_ERR_TOO_LARGE = 8


def corners_on_device(mesh):
    """x,y of each quad's four corners (8 doubles per quad) on the GPU."""
    import torch
    g = np.ascontiguousarray(mesh.geom.reshape(-1, 4, 3)[:, :, :2].reshape(-1))
    t = torch.from_numpy(g).cuda()
    torch.cuda.synchronize()
    return t


@pytest.mark.parametrize("n", [8, 16])
def test_noalloc_totals_equal_session_totals_on_two_calls(ag, n):
    from amrgpu._lib import lib
    f = meshes.two_level_ring(n, periodic=(1, 1))
    cfg = meshes.make_config(n, time_scheme=3, dt=0.01)
    cfg.apply()
    m = f.mesh(n)
    s = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    s.upload(meshes.perturbed(f.initialize(n), 5, amp=1e-2))
    s.step(3)
    ref = s.totals()
    corners = corners_on_device(m)
    q0 = s.state_ptr(0)
    stride = (s.state_ptr(1) - q0) // 8
    for call in range(2):
        out = np.full(4, np.nan)
        rc = lib().amrgpu_totals_noalloc(q0, stride, corners.data_ptr(), m.ncell, n, ag.dp(out), s.stream())
        assert rc == 0, ag.last_error()
        assert np.all(np.abs(out - ref) <= 1e-12 * np.abs(ref) + 1e-13), (call, out, ref)


def test_noalloc_rejects_more_quads_than_its_scratch(ag):
    """Sizes above the stated maximum are refused before any GPU work."""
    from amrgpu._lib import lib
    out = np.zeros(4)
    rc = lib().amrgpu_totals_noalloc(16, 1 << 40, 16, 65537, 16, ag.dp(out), None)
    assert rc == AMRGPU_ERR_TOO_LARGE
    ag.clear_error()
