"""Allocation-free hydro step (wx3d_hydro_step_noalloc) against the
context-based step (wx3d_step).

The entry point serves callers that cannot call cudaMalloc -- hosts whose
device memory belongs to their own pool or framework allocator, or that must
not grow their footprint after start-up.  Here the test plays that caller:
it owns the device buffers (allocated with torch before the call) and checks
consecutive calls against a context with the same mesh, within the parity
tolerance of the other GPU tests.  The cases cover a two-level mesh (coarse
and fine faces), both size limits of the fixed scratch (64 blocks at five
equations, 40 blocks of MHD at eight), a run that crosses an output time,
an empty registry, and the argument checks.  The file is named to be
collected last; it passes alone in a fresh process and after the other
tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10
WX_ERR_INSUFICIENT_NBMAXPROC = 7
WX_ERR_INVALID_ARG = 103


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


def _problem(name):
    from walicxe3d_b200 import config as C
    from walicxe3d_b200 import problems

    if name == "sedov":
        return problems.sedov(2)
    if name == "brio-wu":
        return problems.brio_wu(8)
    if name == "hll1":
        return problems.smooth_pulse(2, solver=C.SOLVER_HLL1)
    if name == "lax":
        return problems.smooth_pulse(2, solver=C.SOLVER_LAX)
    if name == "two-level":
        # 3^3 roots with the centre root (bID 14) refined: 26 + 8 = 34 blocks,
        # six coarse/fine faces, the pulse on the fine blocks
        return problems.amr_pulse(nroot=3, maxlev=2, centre=(0.5, 0.5, 0.5), width=0.08, refine_roots=[14])
    if name == "limit-hd":
        return problems.sedov(4)           # 64 blocks x 5 equations = 320, the limit
    if name == "limit-mhd":
        return problems.brio_wu(40)        # 40 blocks x 8 equations = 320, the limit
    raise ValueError(name)


def _compare(prob, ncalls, tol=TOL):
    """ncalls consecutive allocation-free steps against wx3d_step: state and
    the returned time, dt, it, nextout and output flag after each call."""
    import torch

    from walicxe3d_b200 import _lib
    from walicxe3d_b200.config import WxState
    from walicxe3d_b200.solver import from_problem

    lib = _lib.load()
    g = from_problem(prob)
    ref = []
    for _ in range(ncalls):
        s = g.step()
        ref.append((g.download(), (s.time, s.dt, s.it, s.nextout, s.dumpout)))
    g.close()

    dev = torch.device("cuda:0")
    u_in = torch.from_numpy(prob.U.copy()).to(dev)
    u_out = torch.empty_like(u_in)
    cfg = prob.cfg.to_c()
    lb = np.ascontiguousarray(prob.local_blocks, dtype=np.int32)
    st = WxState(0.0, 0.0, 0, 1, 0, 0)
    torch.cuda.synchronize()
    for call in range(ncalls):
        assert _call(lib, cfg, lb, u_in, u_out, st) == 0
        Uref, (t, dt, it, nextout, dumpout) = ref[call]
        got = u_out.cpu().numpy()
        err = rel_l1(got, Uref)
        assert err.max() <= tol, f"call {call + 1}: relative L1 per eq {err}"
        assert st.it == it
        assert st.time == pytest.approx(t, rel=1e-12)
        assert st.dt == pytest.approx(dt, rel=1e-12)
        assert (st.nextout, bool(st.dumpout)) == (nextout, bool(dumpout)), f"call {call + 1}"
        u_in, u_out = u_out, u_in  # the next call continues from this result
    return [r[1] for r in ref]


@pytest.mark.parametrize("name", ["sedov", "brio-wu", "hll1", "lax", "two-level"])
def test_noalloc_step_matches_context_step(name):
    _compare(_problem(name), 2)


@pytest.mark.parametrize("name", ["limit-hd", "limit-mhd"])
def test_noalloc_step_at_the_scratch_limit(name):
    """Exactly WX3D_NOALLOC_MAX_BLOCK_EQS block-equations: the highest
    offsets of the predictor state, table, work list and control block."""
    prob = _problem(name)
    assert prob.nblocks * prob.cfg.neqtot == 320
    _compare(prob, 2)


def test_noalloc_output_crossing_matches_context_step():
    """An output time falls inside the run: the call that crosses it clips dt,
    reports the crossing and advances nextout; the calls after it, given the
    returned state back, step on with the unclipped dt as wx3d_step does."""
    from walicxe3d_b200.solver import from_problem

    prob = _problem("sedov")
    g = from_problem(prob)
    times = [g.step().time for _ in range(3)]
    g.close()
    # sedov's scalings are 1, so dtout is in code units
    assert prob.cfg.l_sc == 1.0 and prob.cfg.v_sc == 1.0
    prob.cfg.dtout = 0.5 * (times[1] + times[2])
    states = _compare(prob, 5)
    flags = [int(s[4]) for s in states]
    assert flags[:3] == [0, 0, 1]
    assert states[2][0] == pytest.approx(prob.cfg.dtout, rel=1e-14)
    assert [s[3] for s in states] == list(1 + np.cumsum(flags))


def test_noalloc_empty_registry_steps_like_an_empty_mesh():
    """All slots -1: no block is updated and time advances by 1e30*CFL
    clamped to the output time, as wx3d_step does on an empty mesh."""
    import torch

    from walicxe3d_b200 import _lib
    from walicxe3d_b200.config import WxState
    from walicxe3d_b200.solver import Walicxe3D

    prob = _problem("brio-wu")
    prob.cfg.dtout = 0.05
    empty = np.full(4, -1, np.int32)
    w = Walicxe3D(prob.cfg, 4)
    w.set_mesh(empty)
    w.set_state(time=0.0, dt=0.0, it=3, nextout=1)
    ref = [w.step() for _ in range(2)]
    ref = [(s.time, s.dt, s.it, s.nextout, s.dumpout) for s in ref]
    w.close()

    lib = _lib.load()
    u_in = torch.zeros((4,) + prob.U.shape[1:], dtype=torch.float64, device="cuda:0")
    u_out = torch.zeros_like(u_in)
    cfg = prob.cfg.to_c()
    st = WxState(0.0, 0.0, 3, 1, 0, 0)
    for call in range(2):
        assert _call(lib, cfg, empty, u_in, u_out, st) == 0
        assert (st.time, st.dt, st.it, st.nextout, st.dumpout) == ref[call]
        u_in, u_out = u_out, u_in
    assert float(u_out.abs().sum()) == 0.0


def test_noalloc_rejects_meshes_beyond_its_fixed_scratch():
    import torch

    from walicxe3d_b200 import _lib
    from walicxe3d_b200.config import WxState

    lib = _lib.load()
    prob = _problem("limit-hd")
    lb = np.concatenate([prob.local_blocks, [-1]]).astype(np.int32)  # one slot more
    cfg = prob.cfg.to_c()
    u = torch.zeros((len(lb),) + prob.U.shape[1:], dtype=torch.float64, device="cuda:0")
    st = WxState(0.0, 0.0, 0, 1, 0, 0)
    assert _call(lib, cfg, lb, u, torch.empty_like(u), st) == WX_ERR_INSUFICIENT_NBMAXPROC
    assert st.it == 0


def test_noalloc_rejects_overlapping_state_buffers():
    """u_out overlapping u_in (even by one block) is refused before any work."""
    import torch

    from walicxe3d_b200 import _lib
    from walicxe3d_b200.config import WxState

    lib = _lib.load()
    prob = _problem("sedov")
    n = prob.nblocks
    buf = torch.zeros((n + 1,) + prob.U.shape[1:], dtype=torch.float64, device="cuda:0")
    cfg = prob.cfg.to_c()
    lb = np.ascontiguousarray(prob.local_blocks, dtype=np.int32)
    st = WxState(0.0, 0.0, 0, 1, 0, 0)
    assert _call(lib, cfg, lb, buf[:n], buf[1:], st) == WX_ERR_INVALID_ARG
    assert _call(lib, cfg, lb, buf[:n], buf[:n], st) == WX_ERR_INVALID_ARG
    assert st.it == 0
