"""Checkpoint and resume on the GPU: a run resumed from a snapshot of old_
and tmp (zsph_snapshot_save / zsph_snapshot_load) continues bit for bit as
the saved run does, and the file holds exactly the device arrays."""
import numpy as np
import pytest

import zsph_b200 as z
from zsph_b200 import cases

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def _assert_same(sa, ta, sb, tb):
    for k in ("pos", "vel", "rhop", "type", "table"):
        assert np.array_equal(_bits(getattr(sa, k)), _bits(getattr(sb, k))), k
    for k in ("hash", "index", "grid_start", "grid_end", "acc_drhodt"):
        assert np.array_equal(_bits(ta[k]), _bits(tb[k])), k


@pytest.mark.parametrize("mk,equations", [(lambda: cases.small(0.04), z.EQ_DELTA), (cases.config0, z.EQ_DELTA),
                                          (lambda: cases.small(0.04), z.EQ_SIMPLE)])
def test_resume_from_a_snapshot_is_bit_exact(tmp_path, mk, equations):
    c = mk()
    path = str(tmp_path / "run.zsnap")
    a = z.Solver.from_case(c)
    a.set_equations(equations)
    a.run(5)
    a.save_snapshot(path, step=5)
    a.run(5)
    want, want_tmp = a.download("old"), a.download_tmp()
    a.close()
    b = z.Solver.from_case(c)  # the case's initial state, replaced by the load
    b.set_equations(equations)
    assert b.load_snapshot(path) == 5
    b.run(5)
    got, got_tmp = b.download("old"), b.download_tmp()
    b.close()
    _assert_same(want, want_tmp, got, got_tmp)


def test_device_snapshot_holds_the_device_arrays(tmp_path):
    c = cases.small(0.04)
    s = z.Solver.from_case(c)
    s.run(3)
    path = str(tmp_path / "s.zsnap")
    s.save_snapshot(path, step=3)
    st, tmp = s.download("old"), s.download_tmp()
    arrays, step = z.snapshot_load_host(path, s.n, s.G, names=["pos", "vel", "rhop", "type", "table", "hash",
                                                                 "index", "grid_start", "grid_end", "acc_drhodt"])
    assert step == 3
    for k in ("pos", "vel", "rhop", "type", "table"):
        assert np.array_equal(_bits(arrays[k]), _bits(getattr(st, k))), k
    for k in ("hash", "index", "grid_start", "grid_end", "acc_drhodt"):
        assert np.array_equal(_bits(arrays[k]), _bits(tmp[k])), k
    # a snapshot of another size is refused without touching the buffers
    other = z.Solver.from_case(cases.small(0.05))
    before = other.download("old")
    with pytest.raises(z.ZsphError) as e:
        other.load_snapshot(path)
    assert e.value.code == z.ZSPH_EINVAL
    after = other.download("old")
    assert np.array_equal(_bits(before.pos), _bits(after.pos))
    other.close()
    s.close()
