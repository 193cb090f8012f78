"""CPU: properties of the restated frame loop (oracle/csv_oracle_serve.c) that the device server is checked against.

- resident blocks never overlap and stay inside the cache;
- with a cache large enough and the screen-wide cone, no ray ever enters a brick without data;
- every slot a ray reads holds that brick's labels at the slot's LOD (decoded here independently);
- the reference cone (half-angle fov/2) misses bricks at the sides of a wide screen, the screen cone does not;
- a camera that did not move does not re-plan.
"""
import math

import numpy as np
import pytest

from oracle import OracleServer

W, H = 80, 48
FOV = math.pi / 3


@pytest.fixture(scope="module")
def image(oracle):
    from csvb200.synth import tubes_over_voronoi
    vol = tubes_over_voronoi((64, 64, 64), 80, 20, 1.5, 5.0, 11, zero_frac=0.3)
    return oracle.encode(vol, 16)


def _views(n, r0=110.0, r1=50.0):
    from csvb200.camera import orbit
    return [orbit((32.0, 32.0, 32.0), r0 + (r1 - r0) * f / (n - 1), 0.4 * f, 0.3) for f in range(n)]


def _blocks_disjoint(slots, table):
    res = slots[(slots["flags"] == 0) & (slots["offset"] >= table)]
    spans = sorted((int(s["offset"]), int(s["offset"]) + 8 ** int(s["lod"])) for s in res)
    return all(a[1] <= b[0] for a, b in zip(spans, spans[1:])), spans


@pytest.mark.parametrize("cache", [64 << 20, 96 << 10])
def test_blocks_disjoint_and_inside(oracle, image, cache):
    srv = OracleServer(oracle, image, W, H, FOV, 1, cache)
    nb = int(np.frombuffer(image[8:12], np.uint32)[0])
    table = (nb + 31) // 32 * 32
    rebuilt = 0
    for v in _views(10):
        _, _, st = srv.step([0], [v])
        ok, spans = _blocks_disjoint(srv.slots(), table)
        assert ok
        assert not spans or spans[-1][1] <= cache // 8
        rebuilt += st["rebuilt"]
    if cache < (1 << 20):
        assert rebuilt > 0
    srv.close()


def test_screen_cone_never_misses_with_room(oracle, image):
    srv = OracleServer(oracle, image, W, H, FOV, 1, 64 << 20)
    for v in _views(10):
        _, _, st = srv.step([0], [v])
        assert st["missing"] == [0] and st["entered"][0] > 0
    srv.close()


def test_reference_cone_misses_screen_sides(oracle, image):
    """culling.js:132 uses the vertical half-angle: at 16:9 bricks near the left and right edges are culled."""
    from csvb200.camera import orbit
    from csvb200.synth import voronoi
    img = oracle.encode(voronoi((128, 128, 128), 300, 5, zero_slab=0.0), 8)
    ref = OracleServer(oracle, img, 160, 60, FOV, 0, 64 << 20)
    scr = OracleServer(oracle, img, 160, 60, FOV, 1, 64 << 20)
    v = orbit((64.0, 64.0, 64.0), 90.0, 0.3, 0.05)
    _, _, a = ref.step([0], [v])
    _, _, b = scr.step([0], [v])
    assert a["visible"] <= b["visible"] and b["missing"] == [0]
    assert a["missing"][0] > 0
    ref.close()
    scr.close()


def test_slots_hold_their_bricks_labels(oracle, image):
    srv = OracleServer(oracle, image, W, H, FOV, 1, 64 << 20)
    for v in _views(4):
        srv.step([0], [v])
    slots = srv.slots()
    nb = int(np.frombuffer(image[8:12], np.uint32)[0])
    table = (nb + 31) // 32 * 32
    cache = srv.cache((64 << 20) // 8)
    ids = _ids(image)
    per_lod = {}
    for i, m in enumerate(ids):
        sl = slots[m]
        if sl["flags"]:
            continue
        lod = int(sl["lod"])
        if lod not in per_lod:
            per_lod[lod] = oracle.decode_image(image, lod)[0].reshape(nb, -1)
        want = per_lod[lod][i]
        got = cache[int(sl["offset"]): int(sl["offset"]) + len(want)]
        if sl["offset"] < table:  # palette-0 table: LOD 0 or a uniform brick
            assert np.all(want == cache[int(sl["offset"])])
        else:
            assert np.array_equal(got, want)
    srv.close()


def test_still_camera_does_not_replan(oracle, image):
    srv = OracleServer(oracle, image, W, H, FOV, 1, 64 << 20)
    v = _views(3)
    _, _, a = srv.step([0], [v[0]])
    (p, d) = v[0]
    l2, d2, b = srv.step([0], [((p[0] + 0.1, p[1], p[2]), d)])  # 0.1 units: below the 0.5 threshold
    assert a["planned"] == 1 and b["planned"] == 0 and b["decoded"] == 0
    _, _, c = srv.step([0], [v[1]])
    assert c["planned"] == 1
    srv.close()


def _mixed_schedule(n=8):
    """Session 0 every step; session 1 joins at step 2, skips frames, leaves after step 5."""
    from csvb200.camera import orbit
    a = [orbit((32.0, 32.0, 32.0), 110.0 - 7.0 * f, 0.4 * f, 0.3) for f in range(n)]
    b = [orbit((32.0, 32.0, 32.0), 45.0 + 9.0 * f, 2.0 - 0.3 * f, -0.4) for f in range(n)]
    steps = []
    for f in range(n):
        st = [(0, a[f], True)]
        if 2 <= f <= 5:  # open at step 4 without a new frame: its latest camera is step 3's
            st.append((1, b[3] if f == 4 else b[f], f != 4))
        steps.append(st)
    return steps


def test_each_session_same_alone_and_in_the_mix(oracle, image):
    """A session's images do not depend on the other open sessions (the cache has room for both)."""
    steps = _mixed_schedule()
    mix = OracleServer(oracle, image, W, H, FOV, 1, 64 << 20)
    alone = {0: OracleServer(oracle, image, W, H, FOV, 1, 64 << 20),
             1: OracleServer(oracle, image, W, H, FOV, 1, 64 << 20)}
    for st in steps:
        ml, md, ms = mix.step([s for s, _, _ in st], [v for _, v, _ in st], [r for _, _, r in st])
        j = 0
        for s, v, r in st:
            if not r:
                continue
            al, ad, _ = alone[s].step([0], [v])
            assert np.array_equal(ml[j], al[0]) and np.array_equal(md[j].view(np.uint32), ad[0].view(np.uint32))
            j += 1
    for s in alone.values():
        s.close()
    mix.close()


def _ids(image):
    import struct
    nb = struct.unpack_from("<I", image, 8)[0]
    o, ids = 152, []
    for _ in range(nb):
        ids.append(struct.unpack_from("<I", image, o)[0])
        P = struct.unpack_from("<I", image, o + 4)[0]
        o += 8 + 8 * P
        E = struct.unpack_from("<I", image, o)[0]
        o += 4 + E + 4
    return ids


def test_admission_by_rays_properties(oracle, image):
    """Admission by rays (the reference's useGPUCulling path): the first frame is the cone plan; later frames keep
    a subset of it; every slot still holds its brick's labels; a still camera re-plans on the new requests."""
    from csvb200.camera import orbit
    cone = OracleServer(oracle, image, W, H, FOV, 1, 64 << 20)
    rays = OracleServer(oracle, image, W, H, FOV, 1, 64 << 20, admit=1)
    views = [orbit((32.0, 32.0, 32.0), 70.0, 0.4 + 0.05 * f, 0.3) for f in range(5)]
    views.insert(2, views[1])
    fewer = 0
    for k, v in enumerate(views):
        _, _, a = cone.step([0], [v])
        _, _, b = rays.step([0], [v])
        if k == 0:
            assert a["resident"] == b["resident"]
        else:
            assert b["planned"] == 1 and b["resident"] <= a["resident"]
            fewer += b["resident"] < a["resident"]
        sc, sr = cone.slots(), rays.slots()
        held = (sr["flags"] == 0) & (sr["offset"] >= (64 + 31) // 32 * 32)
        # a block resident for the rays is resident for the cone at the same LOD
        assert np.all(sr["lod"][held] == sc["lod"][held])
    assert fewer > 0
    cone.close()
    rays.close()


def test_compaction_packs_resident_blocks(oracle, image):
    """or_serve_compact: blocks contiguous from the start of the block space, coarse LODs first, the same
    labels where each slot points, and the next steps allocate after them."""
    srv = OracleServer(oracle, image, W, H, FOV, 1, 1 << 20)
    nb = int(np.frombuffer(image[8:12], np.uint32)[0])
    table = (nb + 31) // 32 * 32
    for v in _views(6):
        srv.step([0], [v])
    before = srv.slots()
    held = (before["flags"] == 0) & (before["offset"] >= table)
    n_total = srv.cache(0).size  # noqa: F841  (keeps the call path exercised)
    lab_before = {}
    cache = srv.cache((1 << 20) // 8)
    for m in np.nonzero(held)[0]:
        o, n = int(before["offset"][m]), 8 ** int(before["lod"][m])
        lab_before[m] = cache[o:o + n].copy()
    srv.compact()
    after = srv.slots()
    assert np.array_equal(after["lod"], before["lod"]) and np.array_equal(after["flags"], before["flags"])
    spans = sorted((int(after["lod"][m]), int(after["offset"][m])) for m in np.nonzero(held)[0])
    pos = table
    for lod, off in sorted(spans, key=lambda t: t[1]):
        assert off == pos  # no gaps
        pos += 8 ** lod
    lods_in_order = [lod for lod, off in sorted(spans, key=lambda t: t[1])]
    assert lods_in_order == sorted(lods_in_order)  # coarse LODs first
    cache = srv.cache((1 << 20) // 8)
    for m, lab in lab_before.items():
        o = int(after["offset"][m])
        assert np.array_equal(cache[o:o + len(lab)], lab)
    _, _, st = srv.step([0], [_views(8)[7]])
    ok, _ = _blocks_disjoint(srv.slots(), table)
    assert ok
    srv.close()
