"""Writes the golden fixtures of tests/golden/ with the CPU restatement (oracle/).

The reference ships no golden images or key vectors for this path (its tests
compare two GPU renderers at run time), so these fixtures pin the restatement
itself: the reference's own comparison scene (randomCloud(3000, 7) at 250x190,
tests/render/test_splat_render.cpp:77-128, perspective section, with the
partial last tile row and column), its depth keys, cull reasons, pairs and
tile ranges in full, and the image and depth as SHA-256 of their FP32 bytes
plus every 23rd pixel; and the reference's two splat files
(tests/data/splats/tiny.ply and sh3.ply, read where the reference is checked
out) as their vertex records and property names. The scene's 3DGS records come from tests/fixtures.py
(SplatFixtures.h restated); their SHA-256 is kept to catch a drift there.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

W, H = 250, 190
STRIDE = 23


def scene():
    """The fixture's inputs: 3DGS records, the decoded packed cloud, the projection."""
    import athenea_b200 as A
    from oracle import oracle as O
    from tests.fixtures import ENC_BUILDER, random_cloud
    b = random_cloud(3000, 7)
    records = b.records().reshape(-1).astype(np.float32)
    pos, shape, sh, _, shw = O.decode(records, ENC_BUILDER, 3)
    cam = A.Camera.looking_at((1.5, 1.0, 6.0), (0, 0, 0))
    cam.lens.focal = 30.0
    rest_per_colour = {1: 0, 5: 3, 12: 8, 23: 15}[shw]
    return records, (pos, shape, sh, rest_per_colour, shw), cam.projection_for(W, H)


def render(O, packed, proj):
    from tests import gpu_helpers as G
    pos, shape, sh, rpc, shw = packed
    return O.render([(pos, shape, sh, rpc, shw, np.eye(4), 0)], G.oracle_projection(O, proj), W, H)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def reference_splats(root: str | None = None) -> str:
    """The reference checkout's tests/data/splats: `root` (or ATHENEA_REFERENCE, the
    checkout's top directory) joined with that path; "" when neither is given."""
    root = root if root is not None else os.environ.get("ATHENEA_REFERENCE", "")
    return os.path.join(root, "tests", "data", "splats") if root else ""


REFERENCE_SPLATS = reference_splats()


def read_ply_numpy(path):
    """An independent reader for the fixture files (binary little-endian, float
    properties only): (records (N, properties) float32, property names)."""
    with open(path, "rb") as f:
        raw = f.read()
    end = raw.index(b"end_header\n") + len(b"end_header\n")
    names, count = [], 0
    for line in raw[:end].decode().splitlines():
        w = line.split()
        if w[:2] == ["element", "vertex"]:
            count = int(w[2])
        elif w and w[0] == "property":
            assert w[1] == "float", line
            names.append(w[2])
    records = np.frombuffer(raw, np.float32, count * len(names), end).reshape(count, len(names)).copy()
    return records, names, hashlib.sha256(raw).hexdigest()


def ply_fixtures(splats_dir: str):
    """tiny.ply (64 splats, degree 0) and sh3.ply (64 splats, degree 3) of the
    reference's tests/data/splats, as their records and property names."""
    out = {}
    for name in ("tiny", "sh3"):
        records, names, sha = read_ply_numpy(os.path.join(splats_dir, name + ".ply"))
        out[name + "_records"] = records
        out[name + "_names"] = np.array(names)
        out[name + "_sha256"] = sha
    np.savez_compressed(os.path.join(HERE, "splats_tiny_sh3.npz"), **out)
    print("wrote splats_tiny_sh3.npz:", {k: v.shape for k, v in out.items() if hasattr(v, "shape")})


def main():
    """python tests/golden/make_golden.py [reference checkout]: the checkout (or
    ATHENEA_REFERENCE) is read only for its two splat fixture files."""
    from oracle import oracle as O
    O.build()
    records, packed, proj = scene()
    out = render(O, packed, proj)
    b = out["binned"]
    np.savez_compressed(
        os.path.join(HERE, "raster_random3000_250x190.npz"),
        records_sha256=digest(records), keys=out["proj"]["keys"], visible=out["proj"]["visible"],
        touched=out["proj"]["touched"], pair_tiles=b["pair_tiles"], pair_splats=b["pair_splats"],
        ranges=b["ranges"], colour_sha256=digest(out["colour"]), depth_sha256=digest(out["depth"]),
        colour_sample=out["colour"][::STRIDE], depth_sample=out["depth"][::STRIDE])
    print("wrote raster_random3000_250x190.npz:", b["pairs"], "pairs,", int(out["proj"]["visible"].sum()), "visible")
    splats = reference_splats(sys.argv[1] if len(sys.argv) > 1 else None)
    if splats and os.path.isdir(splats):
        ply_fixtures(splats)


if __name__ == "__main__":
    main()
