"""Generates the committed golden fixtures under tests/golden/.  Run from the
repository root in a container that has the reference tree:

    python tests/golden/make_golden.py

Inputs: the reference's shipped encoder/CSVEncoder/compressed_dataset.csbd
(a 512-brick MICrONS cut-out, decode-only golden) and seeded synthetic volumes.
Expected outputs come from the reference sources compiled by
``make -C oracle ref`` (full-resolution decode, encoded bytes); coarse LODs,
which the reference's C++ decoder cannot produce (its decodeBrick is valid at
full resolution only), come from the oracle's restatement of decode.wgsl,
which tests/test_oracle.py pins against the pyramid.
"""
import hashlib
import json
import os
import struct
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "fast-compressed-segmentation_b200"))
from oracle import REF_SHIPPED, Oracle, Reference, build  # noqa: E402
from csvb200 import synth  # noqa: E402

SHIPPED = REF_SHIPPED
OUT = os.path.dirname(os.path.abspath(__file__))


def records(img):
    nb = struct.unpack_from("<I", img, 8)[0]
    o = 152
    recs = []
    for _ in range(nb):
        start = o
        ID, P = struct.unpack_from("<2I", img, o)
        o += 8 + 8 * P
        E = struct.unpack_from("<I", img, o)[0]
        o += 4 + E
        ns = struct.unpack_from("<I", img, o)[0]
        o += 4
        recs.append((start, o, ID, P, E, ns))
    return recs


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    build(ref=True)
    O, R = Oracle(), Reference()
    golden = {}

    # 1. subset of the shipped file: smallest, median and largest streams plus
    #    a few spread over the file, same shared model.
    ship = open(SHIPPED, "rb").read()
    recs = records(ship)
    by_e = sorted(range(len(recs)), key=lambda i: recs[i][4])
    pick = sorted(set([by_e[0], by_e[len(by_e) // 2], by_e[-1], 0, 1, 137, 300, 511]))
    sub = bytearray(ship[:152])
    struct.pack_into("<I", sub, 8, len(pick))
    for i in pick:
        sub += ship[recs[i][0]:recs[i][1]]
    sub = bytes(sub)
    open(os.path.join(OUT, "shipped_subset.csbd"), "wb").write(sub)
    full, st, _ = R.decode_all_full(sub, 64)
    assert st.max() == 0
    entry = {"source_bricks": pick, "brick_size": 64, "lod": {}}
    entry["lod"]["6"] = [sha(full[k]) for k in range(len(pick))]
    for t in range(6):
        d, s = O.decode_image(sub, t)
        assert s.max() == 0
        entry["lod"][str(t)] = [sha(d[k]) for k in range(len(pick))]
    golden["shipped_subset"] = entry

    # 2. reference-encoded synthetic volumes (encode goldens); the volume is
    #    recovered from the fixture by a full-resolution decode and cropping.
    cases = [
        ("voronoi_96x80x72_b64", (72, 80, 96), 64, lambda s: synth.voronoi(s, 150, seed=11)),
        ("tubes_64_b32", (64, 64, 64), 32, lambda s: synth.tubes_over_voronoi(s, 60, 12, 2, 6, seed=12)),
        ("tubes_64_b16", (64, 64, 64), 16, lambda s: synth.tubes_over_voronoi(s, 60, 12, 1, 4, seed=13)),
        ("uniform_64_b64", (64, 64, 64), 64, lambda s: np.full(s, 0x1234567890ABCDEF, np.uint64)),
        ("mixed_uniform_128x64x64_b64", (64, 64, 128), 64,
         lambda s: np.concatenate([np.full((64, 64, 64), 7, np.uint64), synth.voronoi((64, 64, 64), 40, seed=14)],
                                  axis=2)),
    ]
    for name, shape, b, gen in cases:
        vol = gen(shape)
        img = R.encode(vol, b)
        assert img == O.encode(vol, b), name
        open(os.path.join(OUT, name + ".csbd"), "wb").write(img)
        levels = b.bit_length()
        e = {"shape_dhw": list(shape), "brick_size": b, "bytes_sha256": hashlib.sha256(img).hexdigest(),
             "volume_sha256": sha(vol), "lod": {}}
        for t in range(levels):
            d, s = O.decode_image(img, t)
            e["lod"][str(t)] = [sha(d[k]) for k in range(d.shape[0])]
        golden[name] = e
    json.dump(golden, open(os.path.join(OUT, "golden.json"), "w"), indent=1)
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
