"""Legacy VTK particle IO without libVTK (io/write_vtk.cu, io/read_vkt.cu):
format checked by an independent parser, round trips, and the reference
reader's rules (double-only physical arrays, required "type", defaults)."""
import struct

import numpy as np
import pytest

import zsph_b200 as z
from zsph_b200 import cases


def _state(n=257, seed=0):
    rng = np.random.default_rng(seed)
    st = z.State(pos=rng.normal(size=(n, 3)).astype(np.float32), vel=rng.normal(size=(n, 3)).astype(np.float32),
                 rhop=np.stack([1000 + rng.uniform(0, 10, n), rng.uniform(0, 9e3, n)], 1).astype(np.float32),
                 type=rng.integers(0, 2, n).astype(np.int32), table=rng.integers(-5, 5, n).astype(np.int32))
    acc = rng.normal(size=(n, 4)).astype(np.float32)
    return st, acc


def _parse(path):
    """Independent reader of the binary legacy layout the reference writes."""
    data = open(path, "rb").read()
    lines = data.split(b"\n", 5)
    assert lines[0] == b"# vtk DataFile Version 3.0"
    assert lines[2] == b"BINARY" and lines[3] == b"DATASET UNSTRUCTURED_GRID"
    n = int(lines[4].split()[1])
    off = sum(len(l) + 1 for l in lines[:5])
    pos = np.array(struct.unpack(f">{3 * n}f", data[off:off + 12 * n]), np.float32).reshape(n, 3)
    arrays = {}
    rest = data[off + 12 * n:]
    i = 0
    while True:
        j = rest.find(b"SCALARS ", i)
        k = rest.find(b"VECTORS ", i)
        cands = [x for x in (j, k) if x >= 0]
        if not cands:
            break
        s = min(cands)
        hdr_end = rest.find(b"\n", s)
        words = rest[s:hdr_end].split()
        name, typ = words[1].decode(), words[2].decode()
        start = hdr_end + 1
        if words[0] == b"SCALARS":
            start = rest.find(b"\n", start) + 1  # LOOKUP_TABLE line
            comps = 1
        else:
            comps = 3
        code = {"float": "f", "int": "i"}[typ]
        vals = struct.unpack(f">{comps * n}{code}", rest[start:start + 4 * comps * n])
        arrays[name] = np.array(vals).reshape(n, comps) if comps > 1 else np.array(vals)
        i = start + 4 * comps * n
    return pos, arrays


def test_writer_format_is_big_endian_legacy_binary(tmp_path):
    st, acc = _state()
    p = str(tmp_path / "a.vtk")
    z.write_vtk(p, st, acc=acc, flags=z.OUT_REFERENCE)
    pos, arr = _parse(p)
    assert np.array_equal(pos, st.pos)
    assert set(arr) == {"p", "type", "vel", "acc"}  # what the deltasph build writes
    assert np.array_equal(arr["p"].astype(np.float32), st.rhop[:, 1])
    assert np.array_equal(arr["type"], st.type)
    assert np.array_equal(arr["vel"].astype(np.float32), st.vel)
    assert np.array_equal(arr["acc"].astype(np.float32), acc[:, :3])


def test_round_trip_with_float_arrays(tmp_path):
    st, acc = _state(1000, 3)
    p = str(tmp_path / "b.vtk")
    z.write_vtk(p, st, acc=acc, flags=z.OUT_REFERENCE | z.OUT_RHO | z.OUT_TABLE)
    got, gacc = z.read_vtk(p, st.n, rho0=1000.0, accept_float=True)
    for k in ("pos", "vel", "rhop", "type", "table"):
        assert np.array_equal(getattr(got, k), getattr(st, k)), k
    assert np.array_equal(gacc[:, :3], acc[:, :3]) and np.all(gacc[:, 3] == 0)


def test_reference_reader_ignores_float_physical_arrays(tmp_path):
    # read_vkt.cu:61-83 downcasts p/vel/acc/rho to vtkDoubleArray only: the
    # float arrays the writer produces fall back to the defaults
    st, acc = _state(64, 4)
    p = str(tmp_path / "c.vtk")
    z.write_vtk(p, st, acc=acc, flags=z.OUT_REFERENCE | z.OUT_RHO | z.OUT_TABLE)
    got, gacc = z.read_vtk(p, st.n, rho0=999.0, accept_float=False)
    assert np.array_equal(got.pos, st.pos) and np.array_equal(got.type, st.type)
    assert np.array_equal(got.table, st.table)
    assert np.all(got.vel == 0) and np.all(gacc == 0)
    assert np.all(got.rhop[:, 0] == np.float32(999.0)) and np.all(got.rhop[:, 1] == 0)


def test_ascii_double_file_is_read(tmp_path):
    n = 5
    pos = np.arange(15, dtype=np.float64).reshape(n, 3) / 7
    lines = ["# vtk DataFile Version 3.0", "case", "ASCII", "DATASET UNSTRUCTURED_GRID",
             f"POINTS {n} double", " ".join(f"{v:.17g}" for v in pos.ravel()),
             f"CELLS 0 0", "CELL_TYPES 0", f"POINT_DATA {n}",
             "SCALARS p double 1", "LOOKUP_TABLE default", " ".join(str(1.5 * i) for i in range(n)),
             "SCALARS type int 1", "LOOKUP_TABLE default", " ".join(str(i % 2) for i in range(n)),
             "VECTORS vel double", " ".join(str(0.25 * i) for i in range(3 * n))]
    p = tmp_path / "d.vtk"
    p.write_text("\n".join(lines) + "\n")
    got, _ = z.read_vtk(str(p), n, rho0=1000.0)
    assert np.allclose(got.pos, pos.astype(np.float32))
    assert np.allclose(got.rhop[:, 1], [1.5 * i for i in range(n)]) and np.all(got.rhop[:, 0] == 1000)
    assert np.array_equal(got.type, [i % 2 for i in range(n)])
    assert np.allclose(got.vel.ravel(), [0.25 * i for i in range(3 * n)])


def test_reader_errors(tmp_path):
    st, acc = _state(10, 5)
    p = str(tmp_path / "e.vtk")
    z.write_vtk(p, st, acc=acc, flags=z.OUT_P)  # no "type"
    with pytest.raises(z.ZsphError) as e:
        z.read_vtk(p, st.n)
    assert "type" in str(e.value)
    z.write_vtk(p, st, acc=acc, flags=z.OUT_REFERENCE)
    with pytest.raises(z.ZsphError) as e:
        z.read_vtk(p, st.n + 1)
    assert e.value.code == z.ZSPH_EINVAL
    with pytest.raises(z.ZsphError):
        z.read_vtk(str(tmp_path / "missing.vtk"), 3)


def _ascii_case(n, *sections):
    head = ["# vtk DataFile Version 3.0", "case", "ASCII", "DATASET UNSTRUCTURED_GRID",
            f"POINTS {n} double", " ".join("0.125" for _ in range(3 * n))]
    return "\n".join(head + list(sections)) + "\n"


MALFORMED = {
    # a component count of zero or a negative one
    "zero_components": ["POINT_DATA 5", "SCALARS type int 0", "LOOKUP_TABLE default"],
    "negative_components": ["POINT_DATA 5", "SCALARS type int -2", "LOOKUP_TABLE default", "1 1 1 1 1"],
    # a field array with fewer tuples than points, and one of the wrong width
    "short_field": ["POINT_DATA 5", "FIELD FieldData 1", "type 1 2 int", "1 1"],
    "wide_field": ["POINT_DATA 5", "FIELD FieldData 1", "type 2 5 int", " ".join(["1"] * 10)],
    # sizes far beyond the file, and negative ones
    "huge_cells": ["CELLS 1 4000000000000", "POINT_DATA 5"],
    "negative_cells": ["CELLS 1 -5", "POINT_DATA 5"],
    "huge_field": ["POINT_DATA 5", "FIELD FieldData 1", "type 1 999999999999999999 int"],
    "truncated_values": ["POINT_DATA 5", "SCALARS type int 1", "LOOKUP_TABLE default", "1 1"],
}


@pytest.mark.parametrize("name", sorted(MALFORMED))
def test_malformed_files_are_errors_not_crashes(tmp_path, name):
    # sizes and component counts come from the file: each is checked before it
    # is used to allocate or to index, and the reader returns ZSPH_EIO
    p = tmp_path / f"{name}.vtk"
    p.write_text(_ascii_case(5, *MALFORMED[name]))
    with pytest.raises(z.ZsphError) as e:
        z.read_vtk(str(p), 5)
    assert e.value.code == z.ZSPH_EIO


def test_binary_block_checks(tmp_path):
    st, acc = _state(20, 6)
    p = str(tmp_path / "f.vtk")
    z.write_vtk(p, st, acc=acc, flags=z.OUT_REFERENCE)
    data = open(p, "rb").read()
    # cut inside the last binary block
    open(p, "wb").write(data[:-40])
    with pytest.raises(z.ZsphError) as e:
        z.read_vtk(p, st.n)
    assert e.value.code == z.ZSPH_EIO
    # a binary block of a type whose width the reader does not take
    open(p, "wb").write(data.replace(b"SCALARS type int", b"SCALARS type unsigned_char", 1))
    with pytest.raises(z.ZsphError) as e:
        z.read_vtk(p, st.n)
    assert e.value.code == z.ZSPH_EIO and "unsigned_char" in str(e.value)
    # the untouched file still reads
    open(p, "wb").write(data)
    got, _ = z.read_vtk(p, st.n)
    assert np.array_equal(got.type, st.type)


def test_field_arrays_with_metadata_blocks(tmp_path):
    # point arrays as FIELD data, each followed by the METADATA block that
    # VTK's own legacy writer emits (component names, information keys),
    # which ends at an empty line
    n = 4
    lines = ["# vtk DataFile Version 5.1", "vtk output", "ASCII", "DATASET UNSTRUCTURED_GRID",
             f"POINTS {n} double", " ".join(str(0.5 * i) for i in range(3 * n)),
             f"POINT_DATA {n}", "FIELD FieldData 3",
             f"type 1 {n} int", " ".join(str(i % 2) for i in range(n)),
             "METADATA", "INFORMATION 0", "",
             f"vel 3 {n} double", " ".join(str(0.25 * i) for i in range(3 * n)),
             "METADATA", "COMPONENT_NAMES", "X", "Y", "Z", "INFORMATION 1",
             "NAME L2_NORM_RANGE LOCATION vtkDataArray", "DATA 2 0 2.75", "",
             f"p 1 {n} double", " ".join(str(10.0 * i) for i in range(n))]
    p = tmp_path / "g.vtk"
    p.write_text("\n".join(lines) + "\n")
    got, _ = z.read_vtk(str(p), n, rho0=1000.0)
    assert np.array_equal(got.type, [i % 2 for i in range(n)])
    assert np.allclose(got.vel.ravel(), [0.25 * i for i in range(3 * n)])
    assert np.allclose(got.rhop[:, 1], [10.0 * i for i in range(n)])
    assert np.allclose(got.pos.ravel(), [0.5 * i for i in range(3 * n)])


@pytest.mark.parametrize("binary", [False, True])
def test_version_5_1_cells_are_read_past(tmp_path, binary):
    # version 5.1 files (VTK 9's legacy writer) give CELLS as OFFSETS and
    # CONNECTIVITY blocks with their own data types; here one vertex cell per
    # point, offsets in 64-bit and connectivity in 32-bit ints
    n = 3
    pos = (np.arange(3 * n) / 4).astype(">f4")
    types = np.array([1, 0, 1], ">i4")
    offsets = np.arange(n + 1, dtype=">i8")
    conn = np.arange(n, dtype=">i4")
    ctypes_ = np.full(n, 1, ">i4")
    if binary:
        blob = (b"# vtk DataFile Version 5.1\nvtk output\nBINARY\nDATASET UNSTRUCTURED_GRID\n"
                + f"POINTS {n} float\n".encode() + pos.tobytes()
                + f"\nCELLS {n + 1} {n}\nOFFSETS vtktypeint64\n".encode() + offsets.tobytes()
                + b"\nCONNECTIVITY vtktypeint32\n" + conn.tobytes()
                + f"\nCELL_TYPES {n}\n".encode() + ctypes_.tobytes()
                + f"\nPOINT_DATA {n}\nSCALARS type int 1\nLOOKUP_TABLE default\n".encode() + types.tobytes() + b"\n")
    else:
        lines = ["# vtk DataFile Version 5.1", "vtk output", "ASCII", "DATASET UNSTRUCTURED_GRID",
                 f"POINTS {n} float", " ".join(repr(float(v)) for v in pos),
                 f"CELLS {n + 1} {n}", "OFFSETS vtktypeint64", " ".join(map(str, offsets)),
                 "CONNECTIVITY vtktypeint64", " ".join(map(str, conn)),
                 f"CELL_TYPES {n}", " ".join(map(str, ctypes_)),
                 f"POINT_DATA {n}", "SCALARS type int 1", "LOOKUP_TABLE default", " ".join(map(str, types))]
        blob = ("\n".join(lines) + "\n").encode()
    p = tmp_path / "h.vtk"
    p.write_bytes(blob)
    got, _ = z.read_vtk(str(p), n)
    assert np.array_equal(got.pos.ravel(), pos.astype(np.float32))
    assert np.array_equal(got.type, types)


def test_dam_break_case_round_trips_through_vtk(tmp_path):
    c = cases.small(0.04)
    p = str(tmp_path / "input.vtk")
    z.write_vtk(p, c.state, flags=z.OUT_REFERENCE | z.OUT_RHO | z.OUT_TABLE)
    got, _ = z.read_vtk(p, c.n, rho0=float(c.json.rho0), accept_float=True)
    assert np.array_equal(got.pos, c.state.pos) and np.array_equal(got.rhop, c.state.rhop)
