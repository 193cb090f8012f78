"""GPU: the mode / table selector against its CPU restatement, and what the learned choice buys.

* encoding modes and version-2 images: byte-identical to the oracle's encoder, and every LOD decodes to
  the same labels as the plain (version-1) image;
* per-mode statistics, exhaustive choice and brick features: equal to the oracle's, exactly;
* the network's logits and gradients (tensor-core forward / backward): equal to the oracle's fp32
  restatement with the same bf16 rounding points, within 2 % relative error per tensor (accumulation
  order differs) -- cosine similarity above 0.999;
* training on the exhaustive labels lowers the loss, and on a held-out volume the learned choice codes
  within 1 % of the exhaustive choice at a fraction of the search's cost.
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
    n = 200  # of the 256 bricks; not a multiple of 128: exercises the padded rows
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


def _stream_bytes(img: bytes) -> int:
    """Sum of the bricks' rANS stream lengths of a version-1 or version-2 image."""
    import struct
    ver, nb = struct.unpack_from("<II", img, 4)
    o = 152 if ver == 1 else 28 + 128 * struct.unpack_from("<I", img, 24)[0]
    tot = 0
    for _ in range(nb):
        o += 8 if ver == 2 else 4
        P = struct.unpack_from("<I", img, o)[0]
        o += 4 + 8 * P
        E = struct.unpack_from("<I", img, o)[0]
        tot += E
        o += 8 + E
    return tot


def test_learned_choice_near_exhaustive_and_faster(codec, oracle):
    """What the network gains over the search it replaces, on neurite-like volumes of 64^3 bricks: trained on
    the exhaustive choices of six volumes, its choice on a held-out volume codes within 1 % of the exhaustive
    choice's stream bytes, and choosing costs a fraction of the search (brick statistics and one small
    forward pass instead of every mode's op stream).  Decoding the learned image gives the source labels."""
    import torch
    from csvb200.selector import exhaustive_choice, features, fit_tables, learned_choice, train

    def neurite(seed):
        v = torch.empty((256, 256, 256), dtype=torch.int64, device="cuda")
        codec.synth_volume(v, 1, 375, 50, 2.0, 12.0, 0.15, seed)
        return v

    vols = [neurite(s) for s in range(40, 47)]
    feats, hists = [], []
    for v in vols:
        feats.append(features(codec, v, 64))
        h = torch.empty((64, 12, 16), dtype=torch.int32, device="cuda")
        codec.encode_stats(v, 64, h)
        hists.append(h)
    tables = fit_tables(torch.cat(hists[:6]).cpu().numpy().astype(np.uint64), 16, iters=8)
    labels = [exhaustive_choice(codec, v, 64, tables)[0] for v in vols]
    net, losses = train(codec, torch.cat(feats[:6]), torch.cat(labels[:6]), steps=500, batch=384)
    assert np.mean(losses[-20:]) < 0.5 * losses[0]
    held = vols[6]
    codec.encode_device_sel(held, 64, tables, labels[6])
    exhaustive = _stream_bytes(_img(codec))
    s = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    for _ in range(2):  # warm, then timed
        ev[0].record(s)
        sel = learned_choice(net, features(codec, held, 64))
        ev[1].record(s)
        exhaustive_choice(codec, held, 64, tables)
        ev[2].record(s)
    torch.cuda.synchronize()
    t_learned, t_search = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    codec.encode_device_sel(held, 64, tables, sel)
    img = _img(codec)
    learned = _stream_bytes(img)
    assert learned <= exhaustive * 1.01, (learned, exhaustive)
    assert t_search > 2.0 * t_learned, (t_search, t_learned)
    lab, st = codec.decode_image(img, 6)
    assert int(st.max()) == 0
    assert np.array_equal(lab.reshape(-1).view(np.uint64),
                          oracle.decode_image(oracle.encode(held.cpu().numpy().view(np.uint64), 64), 6)[0].ravel())
    assert net.status() == 0
    net.close()


def test_selector_file_drives_a_learned_encode(codec, oracle, tmp_path):
    """A trained selector saved to a file and loaded again (csv_selector_write / csv_selector_read) gives the
    same network and tables, and csv_encode_learned with it writes the image that the step-by-step path
    (features, the network's choice, csv_encode_device_sel) writes with the original network.  That image
    decodes to the source."""
    import torch
    from csvb200 import SelectorNet
    from csvb200.selector import exhaustive_choice, features, learned_choice, train
    v = _vol(codec, (128, 128, 256), 71)
    h = torch.empty((32, 12, 16), dtype=torch.int32, device="cuda")
    codec.encode_stats(v, 64, h)
    tables = _tables(h)
    net, _ = train(codec, features(codec, v, 64), exhaustive_choice(codec, v, 64, tables)[0], steps=40, batch=32)
    path = str(tmp_path / "selector.csvs")
    net.save(path, tables)
    net2, tables2 = SelectorNet.load(codec, path)
    assert np.array_equal(tables2, tables)
    assert np.array_equal(net2.params().view(np.uint32), net.params().view(np.uint32))
    sel = learned_choice(net, features(codec, v, 64))
    codec.encode_device_sel(v, 64, tables, sel)
    step_by_step = _img(codec)
    n = codec.encode_learned(v, 64, net2, tables2)
    one_call = _img(codec)
    assert len(one_call) == n and one_call == step_by_step
    lab, st = codec.decode_image(one_call, 6)
    assert int(st.max()) == 0
    ref = oracle.decode_image(oracle.encode(v.cpu().numpy().view(np.uint64), 64), 6)[0]
    assert np.array_equal(lab, ref)
    net.close()
    net2.close()
