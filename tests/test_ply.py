"""The 3DGS PLY reader (ath_ply_read, after readSplatPly in
modules/io/src/SplatReaders.cpp:50-200) on the reference's own splat files
(tests/data/splats/tiny.ply and sh3.ply, kept as their records in
tests/golden/splats_tiny_sh3.npz), on files written here with other property
types and layouts, and on the errors the reference returns."""
import os
import struct

import numpy as np
import pytest

import athenea_b200 as A
from tests.golden.make_golden import REFERENCE_SPLATS

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "splats_tiny_sh3.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _write_ply(path, names, records, types=None, fmt="binary_little_endian", before=None, extra_header=""):
    """A PLY of one vertex element (and optionally an element before it)."""
    types = types or ["float"] * len(names)
    codes = {"float": "f", "double": "d", "uchar": "B", "char": "b", "short": "h", "ushort": "H", "int": "i",
             "uint": "I"}
    header = ["ply", f"format {fmt} 1.0"]
    if before is not None:
        header += [f"element face {before}", "property uchar a", "property uchar b"]
    header += [f"element vertex {records.shape[0]}"]
    header += [f"property {t} {n}" for t, n in zip(types, names)]
    header += [extra_header] if extra_header else []
    header += ["end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(header) + "\n").encode())
        if before is not None:
            f.write(bytes(2 * before))
        if fmt == "ascii":
            for r in records:
                f.write((" ".join(str(float(v)) for v in r) + "\n").encode())
        else:
            for r in records:
                f.write(b"".join(struct.pack("<" + codes[t], (float(v) if codes[t] in "fd" else int(v)))
                                 for t, v in zip(types, r)))


def _expect_encoding(enc, names):
    idx = {n: k for k, n in enumerate(names)}
    assert enc["stride"] == len(names)
    for field, prop in (("x", "x"), ("y", "y"), ("z", "z"), ("opacity", "opacity"), ("scale0", "scale_0"),
                        ("scale1", "scale_1"), ("scale2", "scale_2"), ("rot_w", "rot_0"), ("rot_x", "rot_1"),
                        ("rot_y", "rot_2"), ("rot_z", "rot_3"), ("dc0", "f_dc_0"), ("dc1", "f_dc_1"),
                        ("dc2", "f_dc_2")):
        assert enc[field] == idx[prop], field
    rest = sum(n.startswith("f_rest_") for n in names)
    assert enc["keep_per_colour"] == enc["file_per_colour"] == rest // 3
    if rest:
        assert enc["rest_base"] == idx["f_rest_0"]


@pytest.mark.parametrize("name", ["tiny", "sh3"])
def test_fixture_files_read_back_exactly(native, golden, tmp_path, name):
    records, names = golden[name + "_records"], [str(n) for n in golden[name + "_names"]]
    path = str(tmp_path / f"{name}.ply")
    _write_ply(path, names, records)
    got, enc = A.read_splat_ply(path)
    np.testing.assert_array_equal(got, records)
    _expect_encoding(enc, names)


@pytest.mark.skipif(not os.path.isdir(REFERENCE_SPLATS), reason="the reference's splat files are not here")
@pytest.mark.parametrize("name", ["tiny", "sh3"])
def test_the_reference_files_themselves(native, golden, name):
    import hashlib
    path = os.path.join(REFERENCE_SPLATS, name + ".ply")
    with open(path, "rb") as f:
        assert hashlib.sha256(f.read()).hexdigest() == str(golden[name + "_sha256"])
    got, enc = A.read_splat_ply(path)
    np.testing.assert_array_equal(got, golden[name + "_records"])
    _expect_encoding(enc, [str(n) for n in golden[name + "_names"]])


def test_other_types_are_widened_and_elements_before_vertex_skipped(native, tmp_path):
    names = ["x", "y", "z", "nx", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
             "rot_0", "rot_1", "rot_2", "rot_3", "red"]
    types = ["double", "float", "float", "short", "float", "float", "float", "float", "float", "float", "float",
             "float", "float", "float", "float", "uchar"]
    rng = np.random.default_rng(3)
    records = rng.normal(size=(7, len(names))).astype(np.float32)
    records[:, 3] = rng.integers(-300, 300, size=7)
    records[:, 15] = rng.integers(0, 255, size=7)
    path = str(tmp_path / "mixed.ply")
    _write_ply(path, names, records, types, before=5)
    got, enc = A.read_splat_ply(path)
    np.testing.assert_array_equal(got, records)
    _expect_encoding(enc, names)


def _status(fn):
    with pytest.raises(A.AtheneaError) as e:
        fn()
    return e.value.code


BASE = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1",
        "rot_2", "rot_3"]


def test_errors_are_the_references(native, tmp_path):
    rec = np.zeros((3, len(BASE)), np.float32)
    p = str(tmp_path / "a.ply")
    _write_ply(p, BASE, rec, fmt="ascii")
    assert _status(lambda: A.read_splat_ply(p)) == 4                  # Unsupported: not binary little-endian
    p = str(tmp_path / "b.ply")
    names = [n for n in BASE if n != "opacity"]
    _write_ply(p, names, rec[:, :len(names)])
    assert _status(lambda: A.read_splat_ply(p)) == 3                  # InvalidArgument: not a trained cloud
    p = str(tmp_path / "c.ply")
    _write_ply(p, BASE, rec)
    with open(p, "rb") as f:
        data = f.read()
    with open(p, "wb") as f:
        f.write(data[:-10])
    assert _status(lambda: A.read_splat_ply(p)) == 5                  # IoFailure: ends before its vertices
    p = str(tmp_path / "d.ply")
    names = BASE + [f"f_rest_{k}" for k in range(30)]
    _write_ply(p, names, np.zeros((2, len(names)), np.float32))
    assert _status(lambda: A.read_splat_ply(p)) == 4                  # Unsupported: not a whole degree
    p = str(tmp_path / "e.ply")
    _write_ply(p, BASE, np.zeros((0, len(BASE)), np.float32))
    assert _status(lambda: A.read_splat_ply(p)) == 3                  # InvalidArgument: no vertices
    p = str(tmp_path / "f.ply")
    _write_ply(p, BASE, rec, extra_header="property list uchar int vertex_indices")
    assert _status(lambda: A.read_splat_ply(p)) == 4                  # Unsupported: a list in the vertex element
    assert _status(lambda: A.read_splat_ply(str(tmp_path / "missing.ply"))) == 2   # NotFound


@pytest.mark.gpu
def test_sh3_decodes_and_draws_as_the_restatement(oracle, golden, tmp_path):
    """sh3.ply through the reader, the GPU decode and a frame, against the oracle's decode and frame."""
    import torch
    from tests import gpu_helpers as G
    path = str(tmp_path / "sh3.ply")
    _write_ply(path, [str(n) for n in golden["sh3_names"]], golden["sh3_records"])
    records, enc = A.read_splat_ply(path)
    splats = A.CloudLoader.upload(torch.from_numpy(records).cuda(), enc)
    e = {("rotW" if k == "rot_w" else "rotX" if k == "rot_x" else "rotY" if k == "rot_y" else "rotZ" if k == "rot_z"
          else "restBase" if k == "rest_base" else "filePerColour" if k == "file_per_colour" else k): v
         for k, v in enc.items() if k != "keep_per_colour"}
    pos, shape, sh, _, shw = oracle.decode(records.reshape(-1), e, 15)
    assert splats.count == pos.shape[0]
    np.testing.assert_array_equal(splats.positions[:splats.count].cpu().numpy(), pos)
    np.testing.assert_array_equal(splats.shape[:splats.count].cpu().numpy().view(np.uint32), shape)
    np.testing.assert_array_equal(splats.sh[:splats.count].cpu().numpy().view(np.uint32), sh)
    W, H = 200, 150
    cam = A.Camera.looking_at((0.0, 0.0, 3.0), (0, 0, 0))
    proj = cam.projection_for(W, H)
    raster = A.TileRasterizer.create()
    t = A.RenderTargets.make(W, H)
    raster.render(proj, [A.SplatInstance(splats)], A.RenderSettings(width=W, height=H), t)
    torch.cuda.synchronize()
    want = oracle.render([(pos, shape, sh, 15, shw, np.eye(4), 0)], G.oracle_projection(oracle, proj), W, H)
    assert np.abs(t.colour.cpu().numpy() - want["colour"]).max() <= 1e-5
