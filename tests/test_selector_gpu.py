"""GPU: the mode / table selector against its CPU restatement, and what the learned choice buys.

* encoding modes and version-2 images: byte-identical to the oracle's encoder, and every LOD decodes to
  the same labels as the plain (version-1) image;
* per-mode statistics, exhaustive choice and brick features: equal to the oracle's, exactly;
* the network's logits and gradients (tensor-core forward / backward): equal to the oracle's fp32
  restatement with the same bf16 rounding points, within 2 % relative error per tensor (accumulation
  order differs) -- cosine similarity above 0.999;
* training on the exhaustive labels lowers the loss, and the learned choice gives a smaller image than
  the plain encoder on held-out volumes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _vol(codec, shape, seed, kind=1, cells=120, tubes=30):
    import torch
    v = torch.empty(shape, dtype=torch.int64, device="cuda")
    codec.synth_volume(v, kind, cells, tubes if kind == 1 else 0, 1.5, 5.0, 0.2, seed)
    torch.cuda.synchronize()
    return v


def _tables(hist):
    from csvb200.selector import fit_tables
    return fit_tables(hist.cpu().numpy().astype(np.uint64), 6, iters=4)


def _img(codec):
    return bytes(codec.encoded_image_tensor().cpu().numpy())


def test_plain_encode_unchanged(codec, oracle):
    v = _vol(codec, (64, 80, 96), 3)
    codec.encode_device_sel(v, 16)
    assert _img(codec) == oracle.encode(v.cpu().numpy().view(np.uint64), 16)


@pytest.mark.parametrize("brick", [16, 32])
def test_stats_select_and_v2_bytes_match_oracle(codec, oracle, brick):
    import torch
    from csvb200.selector import exhaustive_choice
    v = _vol(codec, (64, 96, 128), 11 + brick)
    vh = v.cpu().numpy().view(np.uint64)
    nb = (64 // brick) * (96 // brick) * (128 // brick)
    hist = torch.empty((nb, 12, 16), dtype=torch.int32, device="cuda")
    codec.encode_stats(v, brick, hist)
    ref_hist = oracle.encode_stats(vh, brick)
    assert np.array_equal(hist.cpu().numpy().view(np.uint32), ref_hist)
    tables = _tables(hist)
    sel, _ = exhaustive_choice(codec, v, brick, tables)
    cost = torch.empty((nb, 12, len(tables)), dtype=torch.int64, device="cuda")
    codec.select_exhaustive(hist, tables, sel, cost)
    ref_sel, ref_cost = oracle.select_exhaustive(ref_hist, tables)
    assert np.array_equal(sel.cpu().numpy(), ref_sel)
    assert np.array_equal(cost.cpu().numpy().view(np.uint64), ref_cost)
    # random choices exercise every mode and table, the exhaustive ones the realistic mix
    rnd = torch.from_numpy(np.random.default_rng(brick).integers(0, 12, nb) |
                           (np.random.default_rng(brick + 1).integers(0, len(tables), nb) << 4)).to(torch.uint8)
    plain = oracle.encode(vh, brick)
    for choice in (sel, rnd.cuda()):
        codec.encode_device_sel(v, brick, tables, choice)
        img = _img(codec)
        assert img == oracle.encode_sel(vh, brick, choice.cpu().numpy(), tables)
        ds = codec.open(img)
        for lod in range(brick.bit_length()):
            got, st = codec.decode_image(img, lod)
            assert int(st.max()) == 0
            assert np.array_equal(got.view(np.uint64), oracle.decode_image(plain, lod)[0].reshape(got.shape)), lod
        ds.close()
        # the encoder's own dataset (seek index from the encoder, one LUT per table)
        from csvb200 import requests, requests_tensor
        dse = codec.open_encoded()
        full = brick.bit_length() - 1
        out = torch.zeros(nb * brick ** 3, dtype=torch.int64, device="cuda")
        st = torch.zeros(nb, dtype=torch.int32, device="cuda")
        codec.decode_batch(dse, requests_tensor(requests(np.arange(nb), np.full(nb, full),
                                                         np.arange(nb, dtype=np.uint64) * brick ** 3)), out, st)
        torch.cuda.synchronize()
        assert int(st.abs().max()) == 0
        assert np.array_equal(out.cpu().numpy().view(np.uint64), oracle.decode_image(plain, full)[0].ravel())
        dse.close()


@pytest.mark.parametrize("shape,brick", [((64, 64, 96), 16), ((70, 50, 64), 32), ((64, 64, 64), 64)])
def test_features_match_oracle(codec, oracle, shape, brick):
    from csvb200.selector import features
    v = _vol(codec, shape, 5 + brick, kind=1 if brick != 32 else 0)
    f = features(codec, v, brick).cpu().numpy()
    ref = oracle.brick_features(v.cpu().numpy().view(np.uint64), brick)
    assert np.array_equal(f.view(np.uint32), ref.view(np.uint32))
    assert (f >= 0).all() and (f <= 1).all()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12))


def test_network_forward_and_gradients_match_oracle(codec, oracle):
    import torch
    from csvb200 import SelectorNet
    from csvb200.selector import exhaustive_choice, features
    v = _vol(codec, (64, 128, 128), 21)
    f = features(codec, v, 16)
    hist = torch.empty((f.shape[0], 12, 16), dtype=torch.int32, device="cuda")
    codec.encode_stats(v, 16, hist)
    tables = _tables(hist)
    lab, _ = exhaustive_choice(codec, v, 16, tables)
    n = 300  # not a multiple of 128: exercises the padded rows
    f, lab = f[:n].contiguous(), lab[:n].contiguous()
    p0 = SelectorNet.init_params(3)
    net = SelectorNet(codec, p0)
    logits = torch.empty((n, 32), device="cuda")
    net.forward(f, d_logits=logits)
    torch.cuda.synchronize()
    ref = oracle.mlp_forward(p0, f.cpu().numpy())
    assert _rel(logits.cpu().numpy(), ref) < 2e-3
    loss = net.grad(f, lab)
    _, g = net.params(grads=True)
    ref_loss, ref_g = oracle.mlp_grad(p0, f.cpu().numpy(), lab.cpu().numpy())
    assert abs(loss - ref_loss) <= 1e-3 * abs(ref_loss)
    o = 0
    for name, size in [("W1", 256 * 64), ("b1", 256), ("W2", 256 * 256), ("b2", 256), ("W3", 32 * 256), ("b3", 32)]:
        a, b = g[o:o + size], ref_g[o:o + size]
        assert _rel(a, b) < 2e-2, (name, _rel(a, b))
        assert float(a @ b) / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30) > 0.999, name
        o += size
    assert net.status() == 0
    net.close()


def test_learned_choice_beats_plain_encoder(codec, oracle):
    """Trained on the exhaustive choices of two volumes, the network's choice on a held-out volume gives a
    smaller image than the plain encoder (mode 0, one model) and stays near the exhaustive choice."""
    import torch
    from csvb200.selector import exhaustive_choice, features, fit_tables, learned_choice, train
    vols = [_vol(codec, (128, 128, 128), s, kind=1, cells=300, tubes=60) for s in (31, 32, 33)]
    feats, hists = [], []
    for v in vols:
        feats.append(features(codec, v, 16))
        h = torch.empty((512, 12, 16), dtype=torch.int32, device="cuda")
        codec.encode_stats(v, 16, h)
        hists.append(h)
    tables = fit_tables(torch.cat(hists[:2]).cpu().numpy().astype(np.uint64), 16, iters=8)
    labels = [exhaustive_choice(codec, v, 16, tables)[0] for v in vols]
    net, losses = train(codec, torch.cat(feats[:2]), torch.cat(labels[:2]), steps=400, batch=512)
    assert np.mean(losses[-20:]) < 0.6 * np.mean(losses[:20])
    held = vols[2]
    codec.encode_device_sel(held, 16)
    plain = codec.encoded_image()[1]
    codec.encode_device_sel(held, 16, tables, labels[2])
    exhaustive = codec.encoded_image()[1]
    sel = learned_choice(net, feats[2])
    codec.encode_device_sel(held, 16, tables, sel)
    learned = codec.encoded_image()[1]
    img = _img(codec)
    lab, st = codec.decode_image(img, 4)
    assert int(st.max()) == 0
    assert np.array_equal(lab.view(np.uint64), oracle.decode_image(oracle.encode(held.cpu().numpy().view(np.uint64),
                                                                                   16), 4)[0].reshape(lab.shape))
    assert exhaustive < plain
    assert learned < plain, (learned, exhaustive, plain)
    assert learned <= exhaustive * 1.05, (learned, exhaustive, plain)
    net.close()
