"""CPU: the selector's restatement (oracle/csv_oracle_select.c, the modes of oracle/csv_oracle.c) pinned
on its own before the device is compared with it.

- every mode and table choice decodes (version-2 image) to the source labels at every LOD;
- mode 0 with no tables is the plain image, which is the compiled reference encoder's, byte for byte;
- the per-mode statistics are the nibble histograms of the images those modes produce;
- the exhaustive choice is the argmin of the estimated bits;
- the network's backward pass agrees with finite differences of its loss;
- the host's table normalisation is buildRansModel.
"""
import struct

import numpy as np
import pytest


@pytest.fixture(scope="module")
def vol():
    from csvb200.synth import tubes_over_voronoi
    return tubes_over_voronoi((40, 48, 64), 40, 10, 1.5, 4.0, 5, zero_frac=0.2)


def test_every_mode_and_table_decodes_to_source(oracle, vol):
    rng = np.random.default_rng(3)
    nb = 3 * 3 * 4
    tables = np.stack([np.full(16, 256, np.uint32), np.array([1000] + [206] * 15, np.uint32)])
    tables[1][-1] += 4096 - int(tables[1].sum())
    plain = oracle.encode(vol, 16)
    for trial in range(3):
        sel = (rng.integers(0, 12, nb) | (rng.integers(0, 2, nb) << 4)).astype(np.uint8)
        img = oracle.encode_sel(vol, 16, sel, tables)
        assert int.from_bytes(img[4:8], "little") == 2
        for lod in range(5):
            a, sa = oracle.decode_image(img, lod)
            b, _ = oracle.decode_image(plain, lod)
            assert np.array_equal(a, b) and int(np.max(sa)) == 0, (trial, lod)


def test_mode0_without_tables_is_the_plain_image(oracle, vol):
    assert oracle.encode_sel(vol, 16, np.zeros(36, np.uint8), None) == oracle.encode(vol, 16)


def test_plain_image_is_the_reference_image(oracle, reference, vol):
    assert oracle.encode(vol, 16) == reference.encode(vol, 16)


def test_stats_are_the_images_nibble_histograms(oracle, vol):
    hist = oracle.encode_stats(vol, 16)
    for mode in (0, 5, 9):
        img = oracle.encode_sel(vol, 16, np.full(36, mode, np.uint8), None)
        freq = np.frombuffer(img[24:88], np.uint32)
        cum = np.frombuffer(img[88:152], np.uint32)
        o = 152
        for i in range(36):
            P = struct.unpack_from("<I", img, o + 4)[0]
            o += 8 + 8 * P
            E = struct.unpack_from("<I", img, o)[0]
            enc = img[o + 4:o + 4 + E]
            ns = struct.unpack_from("<I", img, o + 4 + E)[0]
            o += 8 + E
            nib = np.frombuffer(oracle.rans_decode(freq, cum, enc, ns), np.uint8)
            vals = np.stack([nib >> 4, nib & 15], 1).ravel()[:ns]
            h = np.bincount(vals, minlength=16)
            if ns & 1:
                h[0] += 1
            assert np.array_equal(h, hist[i, mode]), (mode, i)


def test_exhaustive_choice_is_the_argmin(oracle, vol):
    hist = oracle.encode_stats(vol, 16)
    tables = np.stack([np.full(16, 256, np.uint32), np.array([1536, 1024] + [110] * 13 + [106], np.uint32)])
    assert tables.sum(1).tolist() == [4096, 4096]
    sel, cost = oracle.select_exhaustive(hist, tables)
    flat = cost.reshape(len(cost), -1)
    assert np.array_equal(sel & 15, flat.argmin(1) // 2)
    assert np.array_equal(sel >> 4, flat.argmin(1) % 2)
    bits = -np.log2(tables / 4096.0)
    est = np.einsum("bms,ts->bmt", hist.astype(np.float64), bits)
    assert np.allclose(cost / 65536.0, est, rtol=1e-6, atol=1e-3)


def test_network_gradient_matches_finite_differences(oracle):
    """The restated backward pass against central differences of the restated loss (with bf16 rounding off
    the perturbed parameters: the checked entries are biases, added in fp32)."""
    from csvb200 import SelectorNet
    rng = np.random.default_rng(0)
    p = SelectorNet.init_params(1)
    feat = rng.random((40, 32)).astype(np.float32)
    lab = (rng.integers(0, 12, 40) | (rng.integers(0, 16, 40) << 4)).astype(np.uint8)
    loss, g = oracle.mlp_grad(p, feat, lab)
    b3 = 256 * 64 + 256 + 256 * 256 + 256 + 32 * 256
    for k in [b3 + 0, b3 + 5, b3 + 13, b3 + 27]:
        h = 1e-2
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (oracle.mlp_grad(pp, feat, lab)[0] - oracle.mlp_grad(pm, feat, lab)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 2e-2 * max(abs(fd), 1e-2), (k, fd, g[k])
    z = oracle.mlp_forward(p, feat)
    assert z.shape == (40, 32) and np.all(z[:, 28:] == 0)


def test_build_model_matches_reference_rule(oracle):
    from csvb200.selector import build_model
    rng = np.random.default_rng(7)
    for _ in range(200):
        raw = rng.integers(0, 5000, 16) * (rng.random(16) < 0.8)
        f, _ = oracle.build_model(raw.astype(np.uint64))
        assert np.array_equal(build_model(raw), f)
