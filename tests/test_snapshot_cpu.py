"""Checkpoint snapshots on the CPU, through the host forms of the C ABI
(zsph_snapshot_save_host / zsph_snapshot_load_host): a bit-exact round trip
of every array, NULL arrays left out and skipped, and every damaged or
foreign file refused before anything is written into the destination."""
import os
import struct

import numpy as np
import pytest

import zsph_b200 as z

N, G = 1000, 357


def _arrays(seed=0, n=N, g=G):
    rng = np.random.default_rng(seed)
    out = {}
    for k, (w, dt) in {**z.SNAPSHOT_PTC, **z.SNAPSHOT_TMP}.items():
        rows = g if k in ("grid_start", "grid_end") else n
        shape = (rows, w) if w > 1 else rows
        if dt == np.int32:
            out[k] = rng.integers(-2**31, 2**31 - 1, size=shape, dtype=np.int64).astype(np.int32)
        else:  # any bit pattern, NaNs and denormals included
            out[k] = rng.integers(0, 2**32, size=shape, dtype=np.uint64).astype(np.uint32).view(np.float32)
    return out


def _same_bits(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_round_trip_is_bit_exact(tmp_path):
    a = _arrays(1)
    p = str(tmp_path / "s.zsnap")
    z.snapshot_save_host(p, a, N, G, step=1234)
    b, step = z.snapshot_load_host(p, N, G)
    assert step == 1234
    for k in a:
        assert _same_bits(a[k], b[k]), k
    # file size: 32-byte header, then a 32-byte header and the data per array
    data = sum(v.nbytes for v in a.values())
    assert os.path.getsize(p) == 32 + 32 * len(a) + data


def test_null_arrays_are_left_out_and_skipped(tmp_path):
    a = _arrays(2)
    for k in ("tmp_pos", "tmp_vel", "tmp_rhop", "dofv", "index", "hash", "acc_drhodt"):
        a.pop(k)
    p = str(tmp_path / "s.zsnap")
    z.snapshot_save_host(p, a, N, G, step=7)
    # a destination that the file lacks is an error
    with pytest.raises(z.ZsphError) as e:
        z.snapshot_load_host(p, N, G)
    assert e.value.code == z.ZSPH_EIO and "lacks array" in str(e.value)
    # loading only what was saved, or less, works
    b, step = z.snapshot_load_host(p, N, G, names=list(a))
    assert step == 7 and all(_same_bits(a[k], b[k]) for k in a)
    c, _ = z.snapshot_load_host(p, N, G, names=["pos", "grid_end"])
    assert _same_bits(a["pos"], c["pos"]) and _same_bits(a["grid_end"], c["grid_end"])


@pytest.mark.parametrize("missing", ["pos", "type", "table", "grid_start", "grid_end"])
def test_save_needs_the_state_and_the_cell_bounds(tmp_path, missing):
    a = _arrays(3)
    a.pop(missing)
    with pytest.raises(z.ZsphError) as e:
        z.snapshot_save_host(str(tmp_path / "s.zsnap"), a, N, G)
    assert e.value.code == z.ZSPH_EINVAL and missing in str(e.value)


def test_size_mismatch_is_einval(tmp_path):
    p = str(tmp_path / "s.zsnap")
    z.snapshot_save_host(p, _arrays(4), N, G)
    for n, g in ((N + 1, G), (N, G - 1)):
        with pytest.raises(z.ZsphError) as e:
            z.snapshot_load_host(p, n, g)
        assert e.value.code == z.ZSPH_EINVAL


def _damaged(tmp_path, how):
    a = _arrays(5)
    p = str(tmp_path / f"{how}.zsnap")
    z.snapshot_save_host(p, a, N, G, step=3)
    raw = bytearray(open(p, "rb").read())
    if how == "flipped_bit":
        raw[len(raw) // 2] ^= 0x10
    elif how == "truncated":
        raw = raw[:-100]
    elif how == "trailing":
        raw += b"\0" * 8
    elif how == "magic":
        raw[0:8] = b"NOTASNAP"
    elif how == "byte_order":
        raw[12:16] = struct.pack(">I", 0x01020304) if struct.pack("=I", 1) == b"\1\0\0\0" else \
            struct.pack("<I", 0x01020304)
    elif how == "version":
        raw[8:12] = struct.pack("=I", 99)
    elif how == "array_size":
        raw[32 + 16:32 + 24] = struct.pack("=Q", 12)
    elif how == "array_name":
        raw[32:48] = b"velocity\0\0\0\0\0\0\0\0"
    elif how == "array_count":
        raw[28:32] = struct.pack("=I", 99)
    open(p, "wb").write(bytes(raw))
    return p


@pytest.mark.parametrize("how", ["flipped_bit", "truncated", "trailing", "magic", "byte_order", "version",
                                 "array_size", "array_name", "array_count"])
def test_damaged_files_are_refused_before_any_write(tmp_path, how):
    p = _damaged(tmp_path, how)
    dest = {k: v.copy() for k, v in _arrays(6).items()}
    before = {k: v.copy() for k, v in dest.items()}
    ptc, tmp = z._host_structs(dest)
    import ctypes
    step = ctypes.c_int(-1)
    rc = z.lib.zsph_snapshot_load_host(p.encode(), ctypes.byref(ptc), ctypes.byref(tmp), N, G, ctypes.byref(step))
    assert rc == z.ZSPH_EIO, z.last_error()
    assert step.value == -1
    for k in dest:
        assert _same_bits(dest[k], before[k]), k  # nothing was written


def test_missing_file_and_bad_arguments(tmp_path):
    with pytest.raises(z.ZsphError) as e:
        z.snapshot_load_host(str(tmp_path / "none.zsnap"), N, G)
    assert e.value.code == z.ZSPH_EIO
    with pytest.raises(z.ZsphError) as e:
        z.snapshot_save_host(str(tmp_path / "no_dir" / "s.zsnap"), _arrays(7), N, G)
    assert e.value.code == z.ZSPH_EIO
    with pytest.raises(z.ZsphError) as e:
        z.snapshot_save_host(str(tmp_path / "s.zsnap"), _arrays(7), N, 0)
    assert e.value.code == z.ZSPH_EINVAL


def test_empty_particle_set(tmp_path):
    a = _arrays(8, n=0, g=5)
    p = str(tmp_path / "s.zsnap")
    z.snapshot_save_host(p, a, 0, 5, step=1)
    b, step = z.snapshot_load_host(p, 0, 5)
    assert step == 1 and all(_same_bits(a[k], b[k]) for k in a)


def test_a_failed_save_leaves_the_earlier_snapshot(tmp_path):
    a = _arrays(9)
    p = str(tmp_path / "s.zsnap")
    z.snapshot_save_host(p, a, N, G, step=10)
    os.mkdir(p + ".part")  # the temporary file of the next save cannot be created
    with pytest.raises(z.ZsphError) as e:
        z.snapshot_save_host(p, _arrays(10), N, G, step=20)
    assert e.value.code == z.ZSPH_EIO
    b, step = z.snapshot_load_host(p, N, G)
    assert step == 10 and all(_same_bits(a[k], b[k]) for k in a)
    os.rmdir(p + ".part")
    z.snapshot_save_host(p, _arrays(10), N, G, step=20)  # and a later save replaces it whole
    assert z.snapshot_load_host(p, N, G)[1] == 20
    assert not os.path.exists(p + ".part")


def test_resume_on_the_oracle_is_bit_exact(tmp_path):
    # the reference's step semantics (the FP32 oracle): the state a step
    # carries over is old_ plus the cell bounds, so 3 steps, a snapshot
    # through the file and 3 more steps from a fresh run equal 6 steps
    from oracle import pyoracle as po
    from zsph_b200 import cases
    c = cases.small(0.04)
    a = po.Oracle(c.json, c.state, np.float32)
    a.step(3)
    p = str(tmp_path / "oracle.zsnap")
    n, G = a.p.ptc_num, a.p.grid_num
    z.snapshot_save_host(p, {**a.old, **a.tmp}, n, G, step=3)
    a.step(3)
    b = po.Oracle(c.json, c.state, np.float32)
    loaded, step = z.snapshot_load_host(p, n, G, names=list(b.old) + list(b.tmp))
    assert step == 3
    for d in (b.old, b.tmp):
        for k in d:
            d[k][...] = loaded[k]  # in place: the oracle holds pointers to these arrays
    b.step(3)
    for k in ("pos", "vel", "rhop", "type", "table"):
        assert _same_bits(a.old[k], b.old[k]), k
    for k in ("hash", "index", "grid_start", "grid_end", "acc_drhodt"):
        assert _same_bits(a.tmp[k], b.tmp[k]), k
