"""Allocation-free hydro step (wx3d_hydro_step_noalloc) against the
context-based step (wx3d_step).

The entry point serves callers that cannot call cudaMalloc -- hosts whose
device memory belongs to their own pool or framework allocator, or that must
not grow their footprint after start-up.  Here the test plays that caller:
it owns the device buffers (allocated with torch before the call) and checks
two consecutive calls against a context with the same mesh, within the
parity tolerance of the other GPU tests.  The file is named to be collected
last; it passes alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel_l1(a, b):
    """Relative L1 per equation (absolute where the reference is all zero)."""
    out = []
    for e in range(a.shape[1]):
        num, den = np.abs(a[:, e] - b[:, e]).sum(), np.abs(b[:, e]).sum()
        out.append(num / den if den > 0 else num)
    return np.array(out)


def _call(lib, cfg, lb, u_in, u_out, st, stream=0):
    return lib.wx3d_hydro_step_noalloc(
        ctypes.byref(cfg), len(lb), lb.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
        ctypes.c_void_p(u_in.data_ptr()), ctypes.c_void_p(u_out.data_ptr()), ctypes.byref(st),
        ctypes.c_void_p(stream))


@pytest.mark.parametrize("name", ["sedov", "brio-wu", "hll1"])
def test_noalloc_step_matches_context_step(name):
    import torch

    from walicxe3d_b200 import _lib, problems
    from walicxe3d_b200 import config as C
    from walicxe3d_b200.config import WxState
    from walicxe3d_b200.solver import from_problem

    if name == "sedov":
        prob = problems.sedov(2)
    elif name == "brio-wu":
        prob = problems.brio_wu(8)
    else:
        prob = problems.smooth_pulse(2, solver=C.SOLVER_HLL1)
    lib = _lib.load()

    g = from_problem(prob)
    ref = []
    for _ in range(2):
        g.step()
        ref.append((g.download(), g.state))
    g.close()

    dev = torch.device("cuda:0")
    u_in = torch.from_numpy(prob.U.copy()).to(dev)
    u_out = torch.empty_like(u_in)
    cfg = prob.cfg.to_c()
    lb = np.ascontiguousarray(prob.local_blocks, dtype=np.int32)
    st = WxState(0.0, 0.0, 0, 1, 0, 0)
    torch.cuda.synchronize()
    for call in range(2):
        assert _call(lib, cfg, lb, u_in, u_out, st) == 0
        Uref, sref = ref[call]
        got = u_out.cpu().numpy()
        err = rel_l1(got, Uref)
        assert err.max() <= TOL, f"call {call + 1}: relative L1 per eq {err}"
        assert st.it == sref.it
        assert st.time == pytest.approx(sref.time, rel=1e-12)
        assert st.dt == pytest.approx(sref.dt, rel=1e-12)
        u_in, u_out = u_out, u_in  # the next call continues from this result


def test_noalloc_rejects_meshes_beyond_its_fixed_scratch():
    import torch

    from walicxe3d_b200 import _lib, problems
    from walicxe3d_b200.config import WxState

    lib = _lib.load()
    prob = problems.sedov(4)  # 64 blocks x 5 equations = 320: the limit itself
    lb = np.concatenate([prob.local_blocks, [-1]]).astype(np.int32)  # one slot more
    cfg = prob.cfg.to_c()
    u = torch.zeros((len(lb),) + prob.U.shape[1:], dtype=torch.float64, device="cuda:0")
    st = WxState(0.0, 0.0, 0, 1, 0, 0)
    assert _call(lib, cfg, lb, u, torch.empty_like(u), st) == 7  # WX_ERR_INSUFICIENT_NBMAXPROC
    assert st.it == 0
