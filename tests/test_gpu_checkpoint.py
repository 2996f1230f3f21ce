"""Checkpoint / restart: a lattice created with the same parameters and loaded
from a checkpoint continues bit for bit as the saved one (populations,
squirmer state, trajectory rows, fields), in every storage form; loading
into another lattice is rejected."""
import numpy as np
import pytest

from lbm_solver_3d_b200.params import Params

pytestmark = pytest.mark.gpu

SLIT = dict(nx=40, ny=26, nz=22, tau=1.0, walls_y=1, walls_z=0, squirmer=1, radius=4.5, b1=0.015, beta=-2.0,
            angle=20, planar=1, traj_every=10, mass_correction_every=7)


def params(**kw):
    p = Params().update(**{**SLIT, **kw})
    p.validate()
    return p


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16"])
def test_restart_continues_bit_for_bit(precision, tmp_path):
    from lbm_solver_3d_b200.solver import Solver
    p = params(precision=precision)
    a = Solver(p)
    a.run(137)            # odd step count: the checkpoint holds the swapped AA parity
    path = tmp_path / "ck.bin"
    a.save(path)
    a.run(113)
    b = Solver(p)
    b.load(path)
    assert b.t == 137
    b.run(113)
    assert a.t == b.t == 250
    sa, sb = a.squirmer(), b.squirmer()
    for k in ("X", "e", "U", "W", "Fh", "Th", "Fc", "Tc"):
        assert np.array_equal(sa[k], sb[k]), k
    assert np.array_equal(a.traj_rows(), b.traj_rows())
    assert np.array_equal(a.get_f(), b.get_f())
    fa, ra, ua = a.fields()
    fb, rb, ub = b.fields()
    assert np.array_equal(fa, fb) and np.array_equal(ra, rb) and np.array_equal(ua, ub)
    a.close(); b.close()


def test_load_rejects_another_lattice():
    from lbm_solver_3d_b200._lib import LbmgpuError
    from lbm_solver_3d_b200.solver import Solver
    a = Solver(params())
    a.run(5)
    data = a.checkpoint()
    for other in (params(nx=41), params(precision="fp32")):
        with pytest.raises(LbmgpuError, match="another lattice"):
            Solver(other).restore(data)
    with pytest.raises(LbmgpuError, match="not a checkpoint"):
        Solver(params()).restore(b"x" * 200)
    with pytest.raises(LbmgpuError, match="truncated"):
        Solver(params()).restore(data[: len(data) // 2])
    a.close()


# Byte layout of the checkpoint header (CkptHeader in csrc/lbmgpu.cu).
HDR_BYTES = 192
OFF_N_LINKS, OFF_F_BYTES, OFF_SQ_BYTES, OFF_WALLS_Y, OFF_TAU = 52, 56, 64, 72, 96


def _links_offset(data: bytes, n_cells: int) -> tuple:
    n_links = int(np.frombuffer(data, np.int32, 1, OFF_N_LINKS)[0])
    f_bytes = int(np.frombuffer(data, np.uint64, 1, OFF_F_BYTES)[0])
    sq_bytes = int(np.frombuffer(data, np.uint64, 1, OFF_SQ_BYTES)[0])
    return HDR_BYTES + f_bytes + n_cells + 32 * n_cells + sq_bytes, n_links


def _patched(data: bytes, off: int, value: np.ndarray) -> bytes:
    b = bytearray(data)
    raw = value.tobytes()
    b[off:off + len(raw)] = raw
    return bytes(b)


def test_load_rejects_corrupt_link_index_and_another_deck():
    """A link node index >= N, a header whose walls flag or tau differ from the
    lattice's, and a checkpoint of another deck are all rejected on the host
    (LBMGPU_ERR_INVALID) before anything reaches the device; the lattice then
    still runs from its own state."""
    from lbm_solver_3d_b200._lib import LBMGPU_ERR_INVALID, LbmgpuError
    from lbm_solver_3d_b200.solver import Solver
    p = params()
    a = Solver(p)
    a.run(9)
    data = a.checkpoint()
    off, n_links = _links_offset(data, p.ncells)
    assert n_links > 0
    bad_link = _patched(data, off + 4 * (n_links - 1), np.array([p.ncells], np.int32))
    bad_neg = _patched(data, off, np.array([-5], np.int32))
    bad_walls = _patched(data, OFF_WALLS_Y, np.array([0], np.int32))
    bad_tau = _patched(data, OFF_TAU, np.array([0.9], np.float64))
    b = Solver(p)
    b.run(3)
    before = b.get_f()
    for blob, msg in ((bad_link, "link node index"), (bad_neg, "link node index"),
                      (bad_walls, "another deck"), (bad_tau, "another deck")):
        with pytest.raises(LbmgpuError, match=msg) as ei:
            b.restore(blob)
        assert ei.value.code == LBMGPU_ERR_INVALID
        assert Solver.check_checkpoint(p, blob) is not None
    # another deck: the same sizes with walls in z, or another tau
    for other in (params(walls_z=1), params(tau=0.9)):
        with pytest.raises(LbmgpuError, match="another deck"):
            Solver(other).restore(data)
    assert np.array_equal(b.get_f(), before)
    b.run(2)
    assert b.t == 5
    assert Solver.check_checkpoint(p, data) is None
    a.close(); b.close()


def test_snapshot_equals_fields_while_the_loop_runs_on():
    """lbmgpu_snapshot_begin captures the fields of the step it follows; steps
    queued after it do not change what lbmgpu_snapshot_read returns, and the
    read may run on another thread while the lattice advances. Pinned host
    buffers give the same values as pageable ones."""
    import threading
    from lbm_solver_3d_b200._lib import LbmgpuError
    from lbm_solver_3d_b200.solver import HostFields, Solver
    s = Solver(params())
    s.run(30)
    ref = [a.copy() for a in s.fields()]
    s.snapshot_begin()
    with pytest.raises(LbmgpuError, match="not been read"):
        s.snapshot_begin()
    got = {}
    out = HostFields(s.N, pinned=True)
    th = threading.Thread(target=lambda: got.update(v=s.snapshot_read(out)))
    th.start()
    s.run(25)          # the loop goes on while the snapshot is read
    th.join()
    for a, b in zip(got["v"], ref):
        assert np.array_equal(a, b)
    later = s.fields_into(HostFields(s.N, pinned=True))
    assert not np.array_equal(later[2], ref[2])     # the lattice did move on
    with pytest.raises(LbmgpuError, match="no snapshot"):
        s.snapshot_read()
    out.close()
    s.close()
