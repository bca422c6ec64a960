"""The HDF5 reader (croma_b200_h5_*) on files written by tests/h5write.py,
an independent writer of the same format subset: every element type
(float32/64, int16/32/64, uint16/32/64) in both byte orders, scalars and
rank 2, compact and contiguous storage, object headers continued in a second
block, nested groups, and groups large enough for their B-tree to split into
several symbol table nodes and two levels.  Each dataset read back equals
what was written; slices equal the whole dataset's elements; a missing path
element, a non-integer dataset read as integers and a read past the end are
refused."""
import numpy as np
import pytest

from conftest import load_package
import h5write

load_package()
from croma_fp_b200 import native  # noqa: E402


def test_round_trip_of_types_layouts_and_groups(tmp_path):
    rng = np.random.default_rng(5)
    data = {
        "f64": rng.normal(size=1000),
        "f32_be": rng.normal(size=33).astype(">f4"),
        "f64_be": rng.normal(size=17).astype(">f8"),
        "i64": rng.integers(-2**62, 2**62, size=50, dtype=np.int64),
        "i32_be": rng.integers(-2**31, 2**31, size=20, dtype=np.int64).astype(">i4"),
        "i16": rng.integers(-2**15, 2**15, size=7, dtype=np.int64).astype("<i2"),
        "u16": rng.integers(0, 2**16, size=9, dtype=np.int64).astype("<u2"),
        "u32_be": rng.integers(0, 2**32, size=9, dtype=np.int64).astype(">u4"),
        "u64": rng.integers(0, 2**62, size=9, dtype=np.int64).astype("<u8"),
        "scalar": np.array(0.85),
        "matrix": rng.normal(size=(6, 5)),
        "small": np.arange(5, dtype=np.float64),
        "group": {"inner": rng.normal(size=64), "deeper": {"leaf": np.arange(12, dtype=np.int64)}},
    }
    for k in range(40):   # forces several symbol table nodes and a two-level B-tree (leaf K = 4)
        data[f"many_{k:02d}"] = np.full(3, float(k))
    path = str(tmp_path / "t.h5")
    h5write.write(path, data, leaf_k=4, compact={"small", "scalar"}, split={"f64", "group/inner", "matrix"})

    def check(name, arr):
        dims, cls, size = native.h5_shape(path, name)
        assert dims == arr.shape and size == arr.dtype.itemsize, name
        assert cls == ("float" if arr.dtype.kind == "f" else "int"), name
        got = native.h5_read(path, name, integer=arr.dtype.kind in "iu")
        assert np.array_equal(got, arr.reshape(-1).astype(got.dtype)), name

    for name, arr in data.items():
        if isinstance(arr, dict):
            continue
        check(name, arr)
    check("group/inner", data["group"]["inner"])
    check("/group/deeper/leaf", data["group"]["deeper"]["leaf"])
    assert np.array_equal(native.h5_read(path, "f64", 100, 37), data["f64"][100:137])
    with pytest.raises(native.CromaError, match="no dataset or group 'nope'"):
        native.h5_read(path, "group/nope")
    with pytest.raises(native.CromaError, match="not an integer dataset"):
        native.h5_read(path, "f64", integer=True)
    with pytest.raises(native.CromaError, match="past the dataset's end"):
        native.h5_read(path, "i16", 5, 3, integer=True)
    with pytest.raises(native.CromaError, match="not a dataset"):
        native.h5_read(path, "group")


def test_corrupted_metadata_gives_errors_not_crashes(tmp_path):
    """Single bytes of the metadata (superblock, object headers, B-tree, symbol
    table nodes, local heap) replaced at random: every read either returns
    the dataset's elements or raises CromaError -- the reader bounds every
    offset, length, count and recursion depth it takes from the file."""
    rng = np.random.default_rng(11)
    data = {f"d{k}": rng.normal(size=64) for k in range(12)}
    data["grp"] = {"x": np.arange(16, dtype=np.int64)}
    path = str(tmp_path / "base.h5")
    h5write.write(path, data, leaf_k=2, split={"d3"})
    raw = open(path, "rb").read()
    # metadata lies before the first dataset's elements and in the tail
    meta = [i for i in range(len(raw)) if i < 96 or raw[i:i + 4] in (b"TREE", b"SNOD", b"HEAP")]
    positions = sorted(set(rng.integers(0, len(raw), 400).tolist()) | set(meta))
    ok = errors = 0
    for n, pos in enumerate(positions[:600]):
        bad = bytearray(raw)
        bad[pos] = (bad[pos] + 1 + int(rng.integers(0, 255))) % 256
        p = tmp_path / f"f{n % 8}.h5"
        p.write_bytes(bytes(bad))
        for name in ("d7", "grp/x"):
            try:
                native.h5_read(str(p), name, integer=(name == "grp/x"))
                ok += 1
            except native.CromaError:
                errors += 1
    assert ok > 0 and errors > 0


def test_cyclic_btree_and_oversized_dataspace_are_refused(tmp_path, monkeypatch):
    """A B-tree whose internal node names itself as a child, and a dataspace
    whose element count overflows, are refused with an error (the walk checks
    that each child sits one level below its parent and bounds the nodes it
    visits; extents are checked against 2^62 elements and bytes)."""
    data = {f"d{k:02d}": np.full(4, float(k)) for k in range(24)}
    path = tmp_path / "tree.h5"
    h5write.write(str(path), data, leaf_k=2)
    raw = bytearray(path.read_bytes())
    pos, roots = 0, []
    while (pos := raw.find(b"TREE", pos)) >= 0:
        if raw[pos + 5] == 1:
            roots.append(pos)
        pos += 4
    assert roots, "the writer made no two-level B-tree"
    root = roots[0]
    raw[root + 32:root + 40] = root.to_bytes(8, "little")   # first child := the node itself
    bad = tmp_path / "cycle.h5"
    bad.write_bytes(bytes(raw))
    with pytest.raises(native.CromaError, match="wrong level"):
        native.h5_read(str(bad), "d23")

    monkeypatch.setattr(h5write, "_space_msg", lambda shape, *a: h5write.struct.pack("<BBBB4x", 1, 3, 0, 0) +
                        h5write.struct.pack("<QQQ", 2**31, 2**31, 2**31))
    big = tmp_path / "big.h5"
    h5write.write(str(big), {"x": np.zeros(4)})
    with pytest.raises(native.CromaError, match="dataspace too large"):
        native.h5_shape(str(big), "x")
    with pytest.raises(native.CromaError, match="dataspace too large"):
        native.h5_read(str(big), "x", 2**62 - 1, 1)


@pytest.mark.parametrize("sb_version,userblock", [(1, 0), (0, 512), (1, 2048)])
def test_superblock_version_1_and_user_blocks(tmp_path, sb_version, userblock):
    """A version-1 superblock (four more bytes before the addresses) and a
    user block before the superblock (signature searched at 512 * 2^k, every
    address relative to the superblock) read the same as the plain layout."""
    rng = np.random.default_rng(sb_version + userblock)
    data = {"a": rng.normal(size=40), "g": {"b": np.arange(9, dtype=np.int64)}, "s": np.array(2.5)}
    path = str(tmp_path / "v.h5")
    h5write.write(path, data, sb_version=sb_version, userblock=userblock, compact={"s"})
    assert np.array_equal(native.h5_read(path, "a"), data["a"])
    assert np.array_equal(native.h5_read(path, "g/b", integer=True), data["g"]["b"])
    assert native.h5_shape(path, "s") == ((), "float", 8) and native.h5_read(path, "s")[0] == 2.5


def test_version_2_dataspaces_scalar_simple_and_null(tmp_path):
    """Version-2 dataspace messages (an explicit scalar / simple / null type
    and no reserved bytes): a scalar reads as one element, rank 1 and 2 as
    their elements, and a null dataspace as no elements."""
    data = {"x": np.linspace(0.0, 1.0, 11), "m": np.arange(12, dtype=np.int64).reshape(3, 4),
            "s": np.array(-7.25), "none": np.zeros(3)}
    path = str(tmp_path / "s2.h5")
    h5write.write(path, data, space_version=2, null={"none"}, compact={"s"})
    assert np.array_equal(native.h5_read(path, "x"), data["x"])
    assert native.h5_shape(path, "m") == ((3, 4), "int", 8)
    assert np.array_equal(native.h5_read(path, "m", integer=True), data["m"].reshape(-1))
    assert native.h5_shape(path, "s") == ((), "float", 8) and native.h5_read(path, "s")[0] == -7.25
    assert native.h5_shape(path, "none")[0] == (0,) and native.h5_read(path, "none").size == 0


def test_c_host_reads_through_the_c_abi(tmp_path):
    """Every public header compiles as C99 (-Wall -Wextra -pedantic, no
    warnings), and a C program linked against the library reads a snapshot
    file through croma_b200_h5_*: the values equal the written ones, and a
    missing dataset comes back as an error message."""
    import os
    import shutil
    import subprocess
    from conftest import ROOT
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    inc = os.path.join(ROOT, "include")
    for h in sorted(os.listdir(inc)):
        src = tmp_path / "h.c"
        src.write_text(f'#include "{h}"\nint main(void) {{ return 0; }}\n')
        r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-Dnp=128", "-Dnpe=128",
                            f"-I{inc}", "-c", str(src), "-o", str(tmp_path / "h.o")], capture_output=True, text=True)
        assert r.returncode == 0, (h, r.stderr)
    libdir = os.path.dirname(native.library_path(128))
    exe = tmp_path / "c_host"
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", f"-I{inc}", os.path.join(ROOT, "tests", "c_host_h5.c"),
                        f"-L{libdir}", "-lcroma_b200_np128", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    dens = np.linspace(1.0e-28, 2.0e-27, 10)
    path = str(tmp_path / "snap.h5")
    h5write.write(path, {"density": dens, "particle_ID": np.arange(7, 17, dtype=np.int64)})
    r = subprocess.run([str(exe), path], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    first, msg = r.stdout.strip().splitlines()
    f = first.split()
    assert f[:4] == ["1", "10", "1", "8"]
    assert [float(x) for x in f[4:7]] == list(dens[2:5]) and f[7:] == ["7", "8"]
    assert "no_such_field" in msg
