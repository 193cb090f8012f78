"""CPU: the oracle (oracle/csv_oracle.c) against the compiled reference and the golden fixtures."""
import hashlib

import numpy as np
import pytest

from conftest import read_golden
from csvb200 import synth


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_morton_identities(oracle):
    # utils.cpp:45-68: the children of parent m are 8m + c with c = dx + 2dy + 4dz
    for m in [0, 1, 7, 100, 4095, 32767]:
        x, y, z = [], [], []
        import ctypes as C
        xx, yy, zz = C.c_uint32(), C.c_uint32(), C.c_uint32()
        oracle.lib.or_demorton3.argtypes = [C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                            C.POINTER(C.c_uint32)]
        oracle.lib.or_demorton3(m, C.byref(xx), C.byref(yy), C.byref(zz))
        for c in range(8):
            dx, dy, dz = c & 1, (c >> 1) & 1, (c >> 2) & 1
            assert oracle.morton3(2 * xx.value + dx, 2 * yy.value + dy, 2 * zz.value + dz) == 8 * m + c


def test_majority_tie_rule_vs_reference(oracle, reference):
    rng = np.random.default_rng(0)
    for hi in (3, 9, 14, 27, 40, 1 << 62):
        vals = rng.integers(0, hi, size=(20000, 8), dtype=np.uint64)
        for v in vals:
            assert oracle.majority8(v) == reference.majority8(v), v


def test_build_model_vs_reference(oracle, reference):
    rng = np.random.default_rng(1)
    for k in range(3000):
        kind = k % 4
        if kind == 0:
            raw = rng.integers(0, 10, 16)
        elif kind == 1:
            raw = rng.integers(0, 100000, 16)
        elif kind == 2:
            raw = np.zeros(16, np.int64)
            raw[rng.integers(0, 16)] = rng.integers(1, 10 ** 6)
        else:
            raw = (rng.pareto(0.7, 16) * 50).astype(np.int64)
        f1, c1 = oracle.build_model(raw)
        f2, c2 = reference.build_model(raw)
        assert np.array_equal(f1, f2) and np.array_equal(c1, c2), raw
        assert c1[16] == 4096


@pytest.mark.parametrize("b", [64, 32, 16, 8])
def test_encode_bytes_vs_reference(oracle, reference, b):
    vol = synth.tubes_over_voronoi((40, 72, 88), 70, 10, 1.5, 7, seed=100 + b)
    assert oracle.encode(vol, b) == reference.encode(vol, b)


def test_encode_voronoi_slab_vs_reference(oracle, reference):
    vol = synth.voronoi((64, 128, 96), 200, seed=5)
    assert oracle.encode(vol, 64) == reference.encode(vol, 64)


def test_full_decode_vs_reference_and_source(oracle, reference):
    vol = synth.tubes_over_voronoi((64, 64, 128), 80, 16, 2, 9, seed=9)
    img = oracle.encode(vol, 64)
    dec, st = oracle.decode_image(img, 6)
    ref, rst, _ = reference.decode_all_full(img, 64)
    assert st.max() == 0 and rst.max() == 0
    assert np.array_equal(dec, ref)
    for i in range(dec.shape[0]):
        pyr = oracle.pyramid(vol, 64, i)
        assert np.array_equal(dec[i], pyr[6][0])


def test_coarse_lods_equal_pyramid(oracle, reference):
    vol = synth.tubes_over_voronoi((64, 64, 64), 50, 10, 1, 6, seed=21)
    img = oracle.encode(vol, 64)
    ref_pyr = reference.pyramid64(vol, 0)
    or_pyr = oracle.pyramid(vol, 64, 0)
    for t in range(7):
        assert np.array_equal(ref_pyr[t][0], or_pyr[t][0])
        assert np.array_equal(ref_pyr[t][1], or_pyr[t][1])
        d, st = oracle.decode_image(img, t)
        assert st.max() == 0
        assert np.array_equal(d[0], or_pyr[t][0]), t


def test_golden_shipped_subset(oracle, reference, golden):
    img = read_golden("shipped_subset")
    g = golden["shipped_subset"]
    full, st, _ = reference.decode_all_full(img, 64)
    assert st.max() == 0
    assert [sha(full[k]) for k in range(full.shape[0])] == g["lod"]["6"]
    for t in range(7):
        d, s = oracle.decode_image(img, t)
        assert s.max() == 0
        assert [sha(d[k]) for k in range(d.shape[0])] == g["lod"][str(t)], t


def crop_volume(dec, shape_dhw, b, ids):
    """Reassemble bricks (Morton order inside, file order = split order) into a (D, H, W) volume."""
    D, H, W = shape_dhw
    nbx, nby, nbz = -(-W // b), -(-H // b), -(-D // b)
    full = np.zeros((nbz * b, nby * b, nbx * b), np.uint64)
    from oracle import Oracle
    O = Oracle()
    mort = np.array([O.morton3(x, y, z) for z in range(b) for y in range(b) for x in range(b)]).reshape(b, b, b)
    i = 0
    for bx in range(nbx):
        for by in range(nby):
            for bz in range(nbz):
                full[bz * b:(bz + 1) * b, by * b:(by + 1) * b, bx * b:(bx + 1) * b] = dec[i][mort]
                i += 1
    return full[:D, :H, :W]


@pytest.mark.parametrize("name", ["voronoi_96x80x72_b64", "tubes_64_b32", "tubes_64_b16", "uniform_64_b64",
                                  "mixed_uniform_128x64x64_b64"])
def test_golden_encode_roundtrip(oracle, golden, name):
    g = golden[name]
    img = read_golden(name)
    assert hashlib.sha256(img).hexdigest() == g["bytes_sha256"]
    b = g["brick_size"]
    full, st = oracle.decode_image(img, b.bit_length() - 1)
    assert st.max() == 0
    vol = crop_volume(full, g["shape_dhw"], b, None)
    assert sha(vol) == g["volume_sha256"]
    assert oracle.encode(vol, b) == img
    for t in range(b.bit_length()):
        d, s = oracle.decode_image(img, t)
        assert [sha(d[k]) for k in range(d.shape[0])] == g["lod"][str(t)]


def _shipped_bricks():
    """(freq, cum, [(E, enc, nsym)]) of the shipped 8-brick subset (v1 layout: fileIO.cpp:25-96)."""
    import struct
    img = read_golden("shipped_subset")
    freq = np.frombuffer(img[24:88], np.uint32)
    cum = np.frombuffer(img[88:152], np.uint32)
    nb = struct.unpack_from("<I", img, 8)[0]
    o, out = 152, []
    for _ in range(nb):
        ID, P = struct.unpack_from("<2I", img, o)
        o += 8 + 8 * P
        E = struct.unpack_from("<I", img, o)[0]
        enc = img[o + 4:o + 4 + E]
        o += 4 + E
        ns = struct.unpack_from("<I", img, o)[0]
        o += 4
        out.append((E, enc, ns))
    return img, freq, cum, out


def test_rans_states_resume_the_reference_chain(oracle, reference):
    """or_rans_states, the content of a seek-index sidecar, on the shipped bricks: the state before symbol 0 is
    the stream header; after the last nibble of the packed bytes (nSymbols rounded up to even: the encoder
    codes the pad nibble too) the state is the encoder's initial one, 2^23, with every byte read; and 64 symbols decoded from every state sampled each 512 symbols equal the compiled reference decoder's
    nibbles there."""
    img, freq, cum, bricks = _shipped_bricks()
    lut = []
    for x in range(4096):
        s = 0
        while s + 1 < 16 and x >= cum[s + 1]:
            s += 1
        lut.append(s)
    for i, (E, enc, ns) in enumerate(bricks):
        n_all = ns + (ns & 1)  # nibbles of the packed bytes
        st = oracle.rans_states(freq, cum, enc, n_all + 1, 1)  # + 1: the state after the last one too
        assert st.shape == (n_all + 1, 2)
        assert tuple(st[0]) == (int.from_bytes(enc[E - 4:E], "little"), E - 4)
        assert tuple(st[-1]) == (1 << 23, 0)
        sampled = oracle.rans_states(freq, cum, enc, ns, 512)
        assert np.array_equal(sampled, st[:ns:512])
        ref = reference.rans_decode(img, i, ns)
        ref_sym = [(ref[j // 2] >> (4 * (1 - j % 2))) & 15 for j in range(ns)]
        for k, (x, pos) in enumerate(sampled):
            x, pos = int(x), int(pos)
            for j in range(512 * k, min(512 * k + 64, ns)):
                v = x & 4095
                sym = lut[v]
                assert sym == ref_sym[j], (i, k, j)
                x = int(freq[sym]) * (x >> 12) + v - int(cum[sym])
                while x < (1 << 23) and pos > 0:
                    pos -= 1
                    x = (x << 8) | enc[pos]


def test_seek_index_checkpoints_resume_decode(oracle):
    """Each checkpoint (state, byte position, nibble index, palette index) lets the rANS decoder resume."""
    import struct
    img = read_golden("shipped_subset")
    freq = np.frombuffer(img[24:88], np.uint32)
    cum = np.frombuffer(img[88:152], np.uint32)
    o = 152
    for _ in range(3):
        ID, P = struct.unpack_from("<2I", img, o)
        o += 8 + 8 * P
        E = struct.unpack_from("<I", img, o)[0]
        enc = img[o + 4:o + 4 + E]
        o += 4 + E
        ns = struct.unpack_from("<I", img, o)[0]
        o += 4
        nib = oracle.rans_decode(freq, cum, enc, ns)
        nibs = [(nib[i // 2] >> (4 * (1 - i % 2))) & 15 for i in range(ns)]
        n_ops, ls, ck, st = oracle.seek_index(freq, cum, enc, ns, P, 64, 256)
        assert st == 0 and ls[6] == n_ops and ck.shape[0] == -(-n_ops // 256)
        # parse ops serially and check every checkpoint's nibble index and palette index
        sym, ip, op = 1, 0, 0
        starts = {}
        while op < n_ops:
            if op % 256 == 0:
                starts[op] = (sym, ip)
            code = nibs[sym] >> 1
            sym += 2 if code == 6 else 1
            ip += code == 4
            op += 1
        lut = []
        for x in range(4096):
            s = 0
            while s + 1 < 16 and x >= cum[s + 1]:
                s += 1
            lut.append(s)
        for k, (state, pos, csym, cip) in enumerate(ck):
            assert (int(csym), int(cip)) == starts[k * 256]
            x, p = int(state), int(pos)
            for j in range(int(csym), min(ns, int(csym) + 40)):
                v = x & 4095
                s = lut[v]
                x = int(freq[s]) * (x >> 12) + v - int(cum[s])
                while x < (1 << 23) and p > 0:
                    p -= 1
                    x = ((x << 8) | enc[p]) & 0xFFFFFFFF
                assert s == nibs[j]


def test_brick_lod_rule(oracle):
    """camera.js:103-137 restated: finest LOD whose voxels still cover >= 1 pixel."""
    import math
    from csvb200.camera import focal_length
    f = focal_length(1080, math.pi / 3)
    for d in [0.05, 10.0, 100.0, 1000.0, 5000.0, 1e5]:
        lod = oracle.brick_lod((d, 0.0, 0.0), 64.0, (0.0, 0.0, 0.0), f, 6)
        expect = 0
        for k in range(7):
            if f * (64.0 / 2 ** k) / max(d, 0.1) >= 1.0:
                expect = k
            else:
                break
        assert lod == expect


def test_scalar_dda_sees_the_volume(oracle):
    """Scalar DDA smoke on the CPU: a full-resolution cache of a two-label volume, camera outside."""
    import math
    from csvb200.camera import SLOT_DTYPE, camera_uniform, orbit
    vol = np.zeros((32, 32, 32), np.uint64)
    vol[8:24, 8:24, 8:24] = 7
    img = oracle.encode(vol, 16)
    dec, st = oracle.decode_image(img, 4)
    slots = np.zeros(8, SLOT_DTYPE)
    for i in range(8):
        slots[i] = (i * 4096, 4, 0)
    # split order is bx, by, bz (bz fastest); slots are indexed by Morton ID
    ids = [oracle.morton3(bx, by, bz) for bx in range(2) for by in range(2) for bz in range(2)]
    lab = np.zeros(8 * 4096, np.uint64)
    for i, m in enumerate(ids):
        lab[m * 4096:(m + 1) * 4096] = dec[i]
        slots[m] = (m * 4096, 4, 0)
    pos, d = orbit((16.0, 16.0, 16.0), 80.0, 0.3, 0.2)
    l, dep, miss = oracle.render(camera_uniform(pos, d, math.pi / 3), 32, 32, 32.0, 16, 2, slots, lab)
    assert (l == 7).sum() > 20 and set(np.unique(l)) <= {0, 7}
    assert np.isfinite(dep[l == 7]).all() and np.isinf(dep[l == 0]).all()


@pytest.mark.parametrize("shape,b", [((32, 32, 96), 4), ((40, 70, 130), 16), ((72, 80, 96), 64)])
def test_threaded_encode_equals_encode(oracle, shape, b):
    """or_encode_threads (the bench reference arm's input builder) writes or_encode's bytes; with 4^3 bricks the
    every-512th model sample spans several threads' ranges."""
    from csvb200.synth import tubes_over_voronoi
    vol = tubes_over_voronoi(shape, 40, 8, 1.0, 3.0, 5 + b, zero_frac=0.1)
    one = oracle.encode(vol, b)
    for threads in (1, 3, 7):
        assert oracle.encode_threads(vol, b, threads) == one, threads


def test_threaded_encode_equals_reference(oracle, reference):
    vol = oracle.synth_volume((96, 80, 72), 2, 60, 30, 1.0, 4.0, 0.0, 4, threads=2)
    assert oracle.encode_threads(vol, 32, 4) == reference.encode(vol, 32)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_cpu_generator_is_deterministic(oracle, kind):
    """or_synth_volume is a pure function of its arguments: any thread count gives the same volume."""
    a = oracle.synth_volume((48, 40, 64), kind, 80, 12, 1.0, 5.0, 0.1, 9, threads=1)
    b = oracle.synth_volume((48, 40, 64), kind, 80, 12, 1.0, 5.0, 0.1, 9, threads=5)
    assert np.array_equal(a, b)
    assert len(np.unique(a)) > 10
    if kind == 0:
        assert 0.05 < float((a == 0).mean()) < 0.15


def _full_res_cache(oracle, vol, b):
    """Slots and labels of a volume decoded at full resolution, every brick resident (Morton-indexed slots)."""
    from csvb200.camera import SLOT_DTYPE
    D, H, W = vol.shape
    nbx, nby, nbz = W // b, H // b, D // b
    img = oracle.encode(vol, b)
    dec, st = oracle.decode_image(img, b.bit_length() - 1)
    n = b ** 3
    ids = [oracle.morton3(bx, by, bz) for bx in range(nbx) for by in range(nby) for bz in range(nbz)]
    n_slots = 1 << (3 * max(nbx, nby, nbz).bit_length())
    slots = np.zeros(n_slots, SLOT_DTYPE)
    slots["flags"] = 1
    lab = np.zeros(n_slots * n, np.uint64)
    for i, m in enumerate(ids):
        lab[m * n:(m + 1) * n] = dec[i]
        slots[m] = (m * n, b.bit_length() - 1, 0)
    return slots, lab


def _one_ray(oracle, vol, b, pos, direction, hidden=None):
    """The label and depth of the single pixel of a 1x1 image (its ray is the camera's forward axis)."""
    import math
    from csvb200.camera import camera_uniform
    slots, lab = _full_res_cache(oracle, vol, b)
    bpa = vol.shape[0] // b
    l, dep, _ = oracle.render(camera_uniform(pos, direction, math.pi / 3), 1, 1, float(bpa * b), b, bpa, slots, lab,
                              hidden=hidden)
    return int(l[0, 0]), float(dep[0, 0])


def test_scalar_dda_known_answers(oracle):
    """Rays whose first hit and entry distance follow by hand (rayTrace.wgsl:473-563, 647-892 restated): the
    first non-zero, not hidden voxel along the ray, and the ray parameter t where the ray enters that cell
    (the forward axis is a unit vector, so t is a distance in voxels).  The rays are tilted by 1e-3 off the
    axes: the shader sets a zero direction component's inverse to sign(0) / 1e-6 = 0 (rayTrace.wgsl:613-617),
    so a ray parallel to an axis plane never enters the volume -- also a known answer (case 0)."""
    import math
    e = 1e-3
    vol = np.zeros((64, 64, 64), np.uint64)  # vol[z, y, x]
    vol[30:, :, :] = 5
    # 0. exactly along +z into a wall that fills the far half: no hit, infinite depth
    lab, t = _one_ray(oracle, vol, 16, (8.5, 8.5, -10.0), (0.0, 0.0, 1.0))
    assert lab == 0 and math.isinf(t)
    # ... and the same ray tilted enters the wall at z = 30: t = 40 (x and y drift by 0.04)
    lab, t = _one_ray(oracle, vol, 16, (8.5, 8.5, -10.0), (e, e, 1.0))
    assert lab == 5 and t == pytest.approx(40.0, abs=1e-3)
    # 1. along +z from (8.5, 8.5, -10): the voxel x = 8, y = 8, z = 20 is first; its z = 20 face is 30 away
    vol = np.zeros((64, 64, 64), np.uint64)
    vol[20, 8, 8] = 7
    assert _one_ray(oracle, vol, 16, (8.5, 8.5, -10.0), (e, e, 1.0)) == (7, pytest.approx(30.0, abs=1e-3))
    # 2. the same label hidden: the ray goes on to the voxel at z = 40 (t = 50)
    vol[40, 8, 8] = 9
    lab, t = _one_ray(oracle, vol, 16, (8.5, 8.5, -10.0), (e, e, 1.0), hidden=np.array([7], np.uint64))
    assert lab == 9 and t == pytest.approx(50.0, abs=1e-3)
    # 3. along +x from (-5, 8.5, 8.5): the voxel x = 30, y = 8, z = 8 is 35 away
    vol2 = np.zeros((64, 64, 64), np.uint64)
    vol2[8, 8, 30] = 3
    assert _one_ray(oracle, vol2, 16, (-5.0, 8.5, 8.5), (1.0, e, e)) == (3, pytest.approx(35.0, abs=1e-3))
    # 4. at 45 degrees in the x-z plane from (2.5, 8.5, -10) into a slab z >= 32 of label 5: the ray meets
    #    z = 32 after 42 units of z, i.e. t = 42 * sqrt(2) = 59.397, at x = 2.5 + 42 = 44.5 (voxel x = 44)
    vol3 = np.zeros((64, 64, 64), np.uint64)
    vol3[32:, :, :] = 5
    lab, t = _one_ray(oracle, vol3, 16, (2.5, 8.5, -10.0), (1.0, e, 1.0))
    assert lab == 5 and t == pytest.approx(42.0 * math.sqrt(2.0), abs=2e-3)
    # 5. looking away from the volume: nothing is hit, depth is infinite
    lab, t = _one_ray(oracle, vol3, 16, (2.5, 8.5, -10.0), (e, e, -1.0))
    assert lab == 0 and math.isinf(t)


def test_brick_lod_known_answers(oracle):
    """calculateBrickLOD (camera.js:103-137) worked out by hand for a 1920x1080 viewport at fov 60 degrees:
    the screen size is min(W, H) = 1080, so focal = 540 / tan(30 deg) = 935.307; a 64^3 brick at LOD k has
    voxels of 64 / 2^k, and the LOD is the finest k <= 6 with 935.307 * 64 / 2^k / max(d, 0.1) >= 1, i.e.
    d <= 59859.7 / 2^k: thresholds 935.3 (k 6), 1870.6 (5), 3741.2 (4), 7482.5 (3), 14964.9 (2), 29929.8 (1);
    beyond the last, LOD 0.  A 32^3 brick at its finest LOD (5) also has unit voxels, so its thresholds
    are the same numbers one LOD lower: 935.3 (k 5), 1870.6 (4), ..., 14964.9 (1)."""
    import math
    from csvb200.camera import focal_length
    f = focal_length(1080, math.pi / 3)
    assert f == pytest.approx(935.307, abs=1e-3)
    cases64 = [(0.05, 6), (935.0, 6), (936.0, 5), (1870.0, 5), (1871.0, 4), (3741.0, 4), (3742.0, 3), (7482.0, 3),
               (7483.0, 2), (14964.0, 2), (14966.0, 1), (29929.0, 1), (29931.0, 0), (1e5, 0)]
    for d, expect in cases64:
        assert oracle.brick_lod((0.0, d, 0.0), 64.0, (0.0, 0.0, 0.0), f, 6) == expect, (d, expect)
    cases32 = [(935.0, 5), (936.0, 4), (1870.0, 4), (1871.0, 3), (14964.0, 1), (14966.0, 0)]
    for d, expect in cases32:
        # the distance is measured between the brick centre and the camera, in any direction
        assert oracle.brick_lod((d / math.sqrt(3), d / math.sqrt(3), d / math.sqrt(3)), 32.0, (0.0, 0.0, 0.0),
                                f, 5) == expect, (d, expect)
