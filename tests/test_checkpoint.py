"""Checkpoints in the reference's formats: writeBin / writeState written
from device memory (output.f90:156-263) and read back by warmstart
(init.f90:527-623)."""
import numpy as np
import pytest

from walicxe3d_b200 import problems

pytestmark = pytest.mark.gpu


def _amr():
    return problems.blast_amr(nroot=3, maxlev=3, shell_radius=0.1, shell_width=0.02)


def test_write_bin_is_the_reference_stream_layout(tmp_path):
    """int32 nbLocal, then per block int32 bID and U(nb,:,1:16,1:16,1:16):
    FP64, the equation index fastest (an independent NumPy encoding of the
    Fortran stream write must match byte for byte)."""
    from walicxe3d_b200.solver import from_problem
    prob = _amr()
    g = from_problem(prob)
    g.run(3)
    f = tmp_path / "Blocks000.0001.bin"
    g.write_bin(f)
    U = g.download()
    neq = prob.cfg.neqtot
    expect = [np.int32(prob.nblocks).tobytes()]
    for s in range(prob.nblocks):
        expect.append(np.int32(prob.local_blocks[s]).tobytes())
        # U(nb, eq, i, j, k) with nb fixed, column major: eq fastest, then i, j, k
        expect.append(np.ascontiguousarray(np.transpose(U[s], (1, 2, 3, 0))).astype("<f8").tobytes())
    assert f.read_bytes() == b"".join(expect)
    assert f.stat().st_size == 4 + prob.nblocks * (4 + neq * 4096 * 8)


def test_state_file_is_the_reference_format(tmp_path):
    from walicxe3d_b200.solver import from_problem
    prob = problems.sedov(2)
    g = from_problem(prob)
    g.set_state(time=1.2345678901234567e-3, dt=0.0, it=42, nextout=7)
    f = tmp_path / "State.0007.dat"
    g.write_state(f, 7, "./data/")
    t = 1.2345678901234567e-3 * prob.cfg.t_sc
    line1 = f"{t:.15E}".rjust(22) + f"{42:8d}{7:5d}"
    assert f.read_text() == line1 + "\n./data/\n"


def test_warm_start_continues_bit_for_bit(tmp_path):
    """A run written at step 5 and warm-started in a fresh context continues
    exactly like the original run."""
    from walicxe3d_b200.solver import Walicxe3D, from_problem
    prob = _amr()
    a = from_problem(prob)
    for _ in range(5):
        a.step()
    a.write_bin(tmp_path / "b.bin")
    a.write_state(tmp_path / "s.dat", 3, str(tmp_path))
    b = Walicxe3D(prob.cfg, prob.nblocks)
    nout, ddir = b.read_state(tmp_path / "s.dat")
    lb = b.read_bin(tmp_path / "b.bin")
    assert nout == 3 and ddir == str(tmp_path)
    assert np.array_equal(lb[: prob.nblocks], prob.local_blocks)
    sa, sb = a.state, b.state
    assert sb.it == sa.it and sb.nextout == 4
    assert sb.time == pytest.approx(sa.time, rel=1e-15)
    assert np.array_equal(a.download(), b.download())
    for _ in range(5):
        a.step()
        b.step()
    assert np.array_equal(a.download(), b.download())


def test_read_bin_errors(tmp_path):
    from walicxe3d_b200._lib import WxError
    from walicxe3d_b200.solver import Walicxe3D
    prob = problems.sedov(2)
    b = Walicxe3D(prob.cfg, prob.nblocks)
    with pytest.raises(WxError) as e:
        b.read_bin(tmp_path / "missing.bin")
    assert e.value.code == 20
    short = tmp_path / "short.bin"
    short.write_bytes(np.int32(2).tobytes() + np.int32(1).tobytes() + b"\0" * 100)
    with pytest.raises(WxError) as e:
        b.read_bin(short)
    assert e.value.code == 21
