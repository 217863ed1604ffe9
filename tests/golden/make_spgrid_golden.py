"""Generates tests/golden/spgrid_golden.npz from the reference's own SPGrid code.

The reference's SPGrid sources are compiled in place into oracle/_ref/ref_spgrid
(`make -C oracle ref`, needs the reference tree) and evaluated on seeded inputs:

* the x/y/z bit masks of SPGrid_Mask<7,7,3> (GridState<double,3>) and
  SPGrid_Mask<6,6,3> (GridState<float,3>),
* Linear_Offset and LinearToCoord of coordinates,
* Packed_Add of offset pairs (stencil and page-neighbour steps),
* particle keys, sort order, groups and the first-touch page map of
  sortParticlesAndPolluteGrid on seeded particle clouds, for both layouts.

    python tests/golden/make_spgrid_golden.py
"""
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_spgrid")


def run(mode, payload):
    with tempfile.TemporaryDirectory() as d:
        fin = os.path.join(d, "in.bin")
        fout = os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(payload)
        subprocess.run([DRIVER, mode, fin, fout], check=True)
        with open(fout, "rb") as f:
            return f.read()


def scenes():
    """Seeded particle clouds; coordinates are float32-representable."""
    out = []
    rng = np.random.default_rng(2019)
    # a jittered cube at dx = 1/64, 8 particles per cell (config-0 shape, 8^3 cells)
    dx = 1.0 / 64
    cells = np.stack(np.meshgrid(*[np.arange(8)] * 3, indexing="ij"), -1).reshape(-1, 3)
    x = (np.repeat(cells, 8, 0) + rng.random((cells.shape[0] * 8, 3))) * dx + np.array([0.375, 0.125, 0.375])
    out.append(("cube", dx, x))
    # scattered clusters at dx = 1/256 (config-1 resolution)
    dx = 1.0 / 256
    centers = rng.uniform(0.1, 0.9, size=(6, 3))
    x = np.concatenate([c + rng.normal(scale=0.01, size=(500, 3)) for c in centers])
    out.append(("clusters", dx, x))
    # particles on exact cell faces and half cells (rounding edge cases)
    dx = 1.0 / 32
    g = np.arange(4, 20)
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)[::7].astype(np.float64)
    x = np.concatenate([pts * dx, (pts + 0.5) * dx, (pts + 0.25) * dx])
    out.append(("faces", dx, x))
    return [(n, dx, x.astype(np.float32).astype(np.float64)) for n, dx, x in out]


def main():
    if not os.path.exists(DRIVER):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    res = {}
    raw = run("masks", b"")
    m = np.frombuffer(raw, dtype=np.uint8)
    for k, name in enumerate(["l7", "l6"]):
        chunk = m[k * 40:(k + 1) * 40]
        res[f"masks_{name}"] = np.frombuffer(chunk[:24].tobytes(), dtype=np.uint64)
        res[f"bits_{name}"] = np.frombuffer(chunk[24:].tobytes(), dtype=np.int32)

    rng = np.random.default_rng(7)
    coords = np.concatenate([
        rng.integers(0, 4096, size=(500, 3)),
        np.array([[0, 0, 0], [4095, 4095, 4095], [1, 2, 3], [2047, 2048, 2049], [4, 4, 4], [3, 7, 15]]),
    ]).astype(np.int32)
    res["coords"] = coords
    raw = np.frombuffer(run("offsets", coords.tobytes()), dtype=np.uint8)
    n = coords.shape[0]
    rec = np.dtype([("off", "<u8"), ("c", "<i4", 3)])
    both = np.frombuffer(raw.tobytes(), dtype=rec)
    res["offsets_l7"] = both["off"][:n].copy()
    res["roundtrip_l7"] = both["c"][:n].copy()
    res["offsets_l6"] = both["off"][n:].copy()
    res["roundtrip_l6"] = both["c"][n:].copy()

    # Packed_Add: base offsets plus stencil steps and page-neighbour steps, per layout
    pairs = {}
    for name, xb, yb, zb, off in (("l7", 2, 4, 4, res["offsets_l7"]), ("l6", 4, 4, 4, res["offsets_l6"])):
        steps = [(i, j, k) for i in range(3) for j in range(3) for k in range(3)]
        steps += [(xb * a, yb * b, zb * c) for a in range(2) for b in range(2) for c in range(2)]
        step_idx = np.array(steps, dtype=np.int32)
        pairs[name] = (off, step_idx)
    res["steps_l7"] = pairs["l7"][1]
    res["steps_l6"] = pairs["l6"][1]
    lo7 = np.frombuffer(run("offsets", pairs["l7"][1].tobytes()), dtype=rec)
    lo6 = np.frombuffer(run("offsets", pairs["l6"][1].tobytes()), dtype=rec)
    ns = pairs["l7"][1].shape[0]
    step_off_l7 = lo7["off"][:ns]
    step_off_l6 = lo6["off"][ns:]
    for name, off, soff in (("l7", res["offsets_l7"][:60], step_off_l7), ("l6", res["offsets_l6"][:60], step_off_l6)):
        a = np.repeat(off, len(soff))
        b = np.tile(soff, len(off))
        ab = np.stack([a, b], 1).astype(np.uint64)
        out = np.frombuffer(run("packed_add", ab.tobytes()), dtype=np.uint64)
        half = len(out) // 2
        res[f"padd_a_{name}"] = a
        res[f"padd_b_{name}"] = b
        res[f"padd_{name}"] = (out[:half] if name == "l7" else out[half:]).copy()

    for sname, dx, x in scenes():
        res[f"scene_{sname}_dx"] = np.array(dx)
        res[f"scene_{sname}_x"] = x
        for l2s in (7, 6):
            hdr = np.array([l2s, x.shape[0]], dtype=np.int32).tobytes() + np.array([dx], dtype=np.float64).tobytes()
            raw = run("bin", hdr + np.ascontiguousarray(x, dtype=np.float64).tobytes())
            P = x.shape[0]
            o = 0
            sorter = np.frombuffer(raw, dtype=np.uint64, count=P, offset=o); o += 8 * P
            order = np.frombuffer(raw, dtype=np.int32, count=P, offset=o); o += 4 * P
            base = np.frombuffer(raw, dtype=np.uint64, count=P, offset=o); o += 8 * P
            G = int(np.frombuffer(raw, dtype=np.int64, count=1, offset=o)[0]); o += 8
            groups = np.frombuffer(raw, dtype=np.int32, count=2 * G, offset=o).reshape(G, 2); o += 8 * G
            boff = np.frombuffer(raw, dtype=np.uint64, count=G, offset=o); o += 8 * G
            B = int(np.frombuffer(raw, dtype=np.int64, count=1, offset=o)[0]); o += 8
            blocks = np.frombuffer(raw, dtype=np.uint64, count=B, offset=o); o += 8 * B
            assert o == len(raw)
            key = f"bin_{sname}_l{l2s}"
            res[key + "_sorter"] = sorter.copy()
            res[key + "_order"] = order.copy()
            res[key + "_base"] = base.copy()
            res[key + "_groups"] = groups.copy()
            res[key + "_block_offset"] = boff.copy()
            res[key + "_blocks"] = blocks.copy()
    np.savez_compressed(os.path.join(HERE, "spgrid_golden.npz"), **res)
    print("wrote", os.path.join(HERE, "spgrid_golden.npz"), {k: v.shape for k, v in res.items() if v.ndim})


if __name__ == "__main__":
    main()
