"""PLY ingest (phgpu_ply_info / phgpu_ply_read, host only) against the values
written into generated files.

The reference reads x, y, z, intensity (required) and reflectivity, "noise"
(ambient) and range (optional) of element "vertex" through tinyply as
doubles (ply-helper.cc:26-64); the cloud narrows them to float
(point-cloud.cc:329-348).  Expected values here are therefore
float32(float64(written value)), compared bit for bit.  The files mimic an
Ouster OS-1 export (x, y, z, intensity float; t uint; reflectivity ushort;
ring uchar; noise ushort; range uint) plus ascii / big-endian variants,
elements around the vertices and list properties."""
import struct

import numpy as np
import pytest

FMT = {"char": "b", "uchar": "B", "short": "h", "ushort": "H", "int": "i", "uint": "I", "float": "f",
       "double": "d", "int8": "b", "uint8": "B", "int16": "h", "uint16": "H", "int32": "i", "uint32": "I",
       "float32": "f", "float64": "d"}


def write_ply(path, fmt, elements):
    """elements: list of (name, props, rows); props: list of (name, type) or
    (name, ('list', count_type, item_type)); rows: list of tuples (a list
    property's value is a Python list)."""
    head = ["ply", f"format {fmt} 1.0", "comment generated"]
    for name, props, rows in elements:
        head.append(f"element {name} {len(rows)}")
        for pn, pt in props:
            if isinstance(pt, tuple):
                head.append(f"property list {pt[1]} {pt[2]} {pn}")
            else:
                head.append(f"property {pt} {pn}")
    head.append("end_header")
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n").encode())
        end = "<" if fmt == "binary_little_endian" else ">"
        for name, props, rows in elements:
            for row in rows:
                if fmt == "ascii":
                    parts = []
                    for (pn, pt), v in zip(props, row):
                        if isinstance(pt, tuple):
                            parts += [str(len(v))] + [repr(x) for x in v]
                        else:
                            parts.append(repr(v))
                    f.write((" ".join(parts) + "\n").encode())
                else:
                    for (pn, pt), v in zip(props, row):
                        if isinstance(pt, tuple):
                            f.write(struct.pack(end + FMT[pt[1]], len(v)))
                            for x in v:
                                f.write(struct.pack(end + FMT[pt[2]], x))
                        else:
                            f.write(struct.pack(end + FMT[pt], v))


OUSTER = [("x", "float"), ("y", "float"), ("z", "float"), ("intensity", "float"), ("t", "uint"),
          ("reflectivity", "ushort"), ("ring", "uchar"), ("noise", "ushort"), ("range", "uint")]


def ouster_rows(n, seed):
    rng = np.random.default_rng(seed)
    xyz = rng.normal(0, 20, (n, 3)).astype(np.float32)
    inten = rng.uniform(0, 4000, n).astype(np.float32)
    rows = []
    for k in range(n):
        rows.append((float(xyz[k, 0]), float(xyz[k, 1]), float(xyz[k, 2]), float(inten[k]), int(k * 97),
                     int(rng.integers(0, 65535)), int(k % 64), int(rng.integers(0, 65535)),
                     int(rng.integers(0, 120000))))
    return rows


@pytest.fixture(scope="module")
def nat():
    from phaser_b200 import native
    native.load()
    return native


def col(rows, props, name):
    i = [p[0] for p in props].index(name)
    return np.array([np.float32(np.float64(r[i])) for r in rows], np.float32)


@pytest.mark.parametrize("fmt", ["binary_little_endian", "binary_big_endian", "ascii"])
def test_ouster_layout(nat, tmp_path, fmt):
    rows = ouster_rows(777, 3)
    p = tmp_path / "cloud.ply"
    write_ply(p, fmt, [("vertex", OUSTER, rows)])
    n, present = nat.ply_info(p)
    assert n == 777
    assert present == nat.PHGPU_PLY_REFLECTIVITY | nat.PHGPU_PLY_AMBIENT | nat.PHGPU_PLY_RANGE
    d = nat.ply_read(p)
    for c, name in enumerate(["x", "y", "z", "intensity"]):
        assert np.array_equal(d["xyzi"][:, c], col(rows, OUSTER, name))
    assert np.array_equal(d["reflectivity"], col(rows, OUSTER, "reflectivity"))
    assert np.array_equal(d["ambient"], col(rows, OUSTER, "noise"))
    assert np.array_equal(d["range"], col(rows, OUSTER, "range"))


def test_double_fields_elements_and_lists(nat, tmp_path):
    # a scalar element and a list-carrying element before the vertices, a
    # face list after them, double coordinates narrowed to float
    rng = np.random.default_rng(5)
    props = [("intensity", "uchar"), ("z", "double"), ("x", "double"), ("y", "double")]
    rows = [(int(rng.integers(0, 255)), float(rng.normal()), float(rng.normal() * 1e3), float(rng.normal() * 1e-3))
            for _ in range(300)]
    meta = ("camera", [("fx", "float"), ("id", "int")], [(1.5, 3), (2.5, -4)])
    tags = ("tag", [("ids", ("list", "uchar", "int")), ("w", "short")], [([1, 2, 3], 7), ([], -2), ([9], 1)])
    faces = ("face", [("vertex_indices", ("list", "uchar", "int"))], [([0, 1, 2],), ([2, 3, 4],)])
    for fmt in ["binary_little_endian", "binary_big_endian", "ascii"]:
        p = tmp_path / f"d_{fmt}.ply"
        write_ply(p, fmt, [meta, tags, ("vertex", props, rows), faces])
        n, present = nat.ply_info(p)
        assert (n, present) == (300, 0)
        d = nat.ply_read(p)
        for c, name in enumerate(["x", "y", "z", "intensity"]):
            assert np.array_equal(d["xyzi"][:, c], col(rows, props, name)), (fmt, name)
        assert d["reflectivity"] is None and d["ambient"] is None and d["range"] is None


def test_list_property_inside_vertex(nat, tmp_path):
    props = [("x", "float"), ("nbrs", ("list", "uchar", "ushort")), ("y", "float"), ("z", "float"),
             ("intensity", "float"), ("noise", "int")]
    rows = [(float(k), list(range(k % 4)), float(-k), float(k) / 8, float(k * 3), k - 50) for k in range(100)]
    for fmt in ["binary_little_endian", "ascii"]:
        p = tmp_path / f"l_{fmt}.ply"
        write_ply(p, fmt, [("vertex", props, rows)])
        d = nat.ply_read(p)
        assert np.array_equal(d["xyzi"][:, 0], col(rows, props, "x"))
        assert np.array_equal(d["xyzi"][:, 2], col(rows, props, "z"))
        assert np.array_equal(d["ambient"], col(rows, props, "noise"))
        assert d["reflectivity"] is None


def test_field_names_override(nat, tmp_path):
    # the reference's --phaser_ply_*_str flags rename the requested fields
    props = [("x", "float"), ("y", "float"), ("z", "float"), ("signal", "float"), ("refl", "float"),
             ("ambient", "float"), ("intensity", "float")]
    rows = [tuple(float(v) for v in np.random.default_rng(k).normal(size=7)) for k in range(50)]
    p = tmp_path / "names.ply"
    write_ply(p, "binary_little_endian", [("vertex", props, rows)])
    d = nat.ply_read(p, ["signal", "refl", "ambient", None])
    assert np.array_equal(d["xyzi"][:, 3], col(rows, props, "signal"))
    assert np.array_equal(d["reflectivity"], col(rows, props, "refl"))
    assert np.array_equal(d["ambient"], col(rows, props, "ambient"))
    assert d["range"] is None
    d = nat.ply_read(p)  # defaults: intensity field, no reflectivity / noise / range
    assert np.array_equal(d["xyzi"][:, 3], col(rows, props, "intensity"))
    assert d["reflectivity"] is None


def test_python_mirror(nat, tmp_path):
    from phaser_b200.core import PlyHelper
    rows = ouster_rows(64, 9)
    p = tmp_path / "m.ply"
    write_ply(p, "binary_little_endian", [("vertex", OUSTER, rows)])
    pc = PlyHelper().readPlyFromFile(str(p))
    assert pc.getXYZPoints().shape == (64, 3)
    assert np.array_equal(pc.getIntentsities(), col(rows, OUSTER, "intensity"))
    xyzi, refl, amb = pc.cloud()
    assert np.array_equal(refl, col(rows, OUSTER, "reflectivity"))


def test_errors(nat, tmp_path):
    # missing intensity: the reference aborts (CHECK_GT), here an error status
    p = tmp_path / "noint.ply"
    write_ply(p, "ascii", [("vertex", [("x", "float"), ("y", "float"), ("z", "float")], [(1.0, 2.0, 3.0)])])
    with pytest.raises(nat.PhgpuError, match="intensity"):
        nat.ply_read(p)
    q = tmp_path / "nov.ply"
    write_ply(q, "ascii", [("face", [("a", "int")], [(1,)])])
    with pytest.raises(nat.PhgpuError, match="vertex"):
        nat.ply_info(q)
    r = tmp_path / "notply.ply"
    r.write_bytes(b"hello\n")
    with pytest.raises(nat.PhgpuError):
        nat.ply_info(r)
    with pytest.raises(nat.PhgpuError):
        nat.ply_info(tmp_path / "missing.ply")
    # truncated binary body
    t = tmp_path / "trunc.ply"
    write_ply(t, "binary_little_endian", [("vertex", OUSTER, ouster_rows(10, 1))])
    t.write_bytes(t.read_bytes()[:-7])
    with pytest.raises(nat.PhgpuError, match="truncated"):
        nat.ply_read(t)
    # capacity below the vertex count
    import ctypes as C
    buf = np.zeros((4, 4), np.float32)
    got = C.c_uint32()
    w = tmp_path / "cap.ply"
    write_ply(w, "binary_little_endian", [("vertex", OUSTER, ouster_rows(10, 2))])
    rc = nat.load().phgpu_ply_read(str(w).encode(), None, buf.ctypes.data, None, None, None, 4, C.byref(got))
    assert rc == -5


def test_error_messages_are_printable(nat, tmp_path):
    """A damaged header line is quoted in the error as printable ASCII, so the
    message decodes and the call raises PhgpuError (not a decode error)."""
    p = tmp_path / "bin.ply"
    p.write_bytes(b"ply\nformat ascii 1.0\nelement vert\xfa\xff\x01x\nend_header\n")
    with pytest.raises(nat.PhgpuError) as e:
        nat.ply_info(p)
    msg = str(e.value)
    assert "bad element line" in msg and all(32 <= ord(ch) < 127 for ch in msg)


def test_damaged_files_fail_cleanly(nat, tmp_path):
    """Seeded byte flips, truncations and header edits of valid files: every
    call either reads the file or raises PhgpuError."""
    import random
    src = []
    for fmt in ("binary_little_endian", "ascii", "binary_big_endian"):
        q = tmp_path / f"src_{fmt}.ply"
        write_ply(q, fmt, [("vertex", OUSTER, ouster_rows(12, 7)), ("face", [("vi", ("list", "uchar", "int"))],
                                                                     [([1, 2, 3],)])])
        src.append(q.read_bytes())
    rng = random.Random(1)
    read = failed = 0
    for k in range(150):
        b = bytearray(rng.choice(src))
        hdr_end = bytes(b).find(b"end_header")
        mode = k % 3
        if mode == 0:
            for _ in range(rng.randrange(1, 12)):
                b[rng.randrange(len(b))] = rng.randrange(256)
        elif mode == 1:
            b = b[:rng.randrange(len(b))]
        else:
            for _ in range(rng.randrange(1, 4)):
                b[rng.randrange(max(1, hdr_end))] = rng.choice(b"0123456789 \n\x00abcxyz-\xfa")
        f = tmp_path / f"d{k}.ply"
        f.write_bytes(bytes(b))
        try:
            n, _ = nat.ply_info(f)
            if n <= 1000:
                nat.ply_read(f)
            read += 1
        except nat.PhgpuError:
            failed += 1
    assert read + failed == 150 and failed > 0
