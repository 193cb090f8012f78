"""GPU: mixed brick sizes in one launch (csv_dataset_concat), the captured decode (CUDA graph) and the autotuner.

Every output is compared label for label with the oracle's decode of each part's
own .csbd image.
"""
import numpy as np
import pytest

from conftest import read_golden

pytestmark = pytest.mark.gpu


def _parts(codec, oracle):
    """A 32^3-brick dataset and a 64^3-brick dataset with different rANS models."""
    import torch
    imgs = []
    for shape, kind, b, seed in [((64, 96, 128), 0, 32, 31), ((64, 128, 128), 1, 64, 32)]:
        vol = torch.empty(shape, dtype=torch.int64, device="cuda")
        codec.synth_volume(vol, kind, 120 if kind == 0 else 300, 0 if kind == 0 else 30, 1.0, 4.0, 0.1, seed)
        codec.encode_device(vol, b)
        imgs.append(bytes(codec.encoded_image_tensor().cpu().numpy()))
    imgs.append(read_golden("shipped_subset"))  # a third model: the reference's own file
    return imgs


def _mixed_requests(sizes_b, rng, n_extra=40):
    """All bricks at full resolution, plus random (brick, lod) repeats; returns requests and expected keys."""
    from csvb200 import requests
    total = sum(n for n, b in sizes_b)
    bricks, lods = [], []
    base = 0
    for n, b in sizes_b:
        full = b.bit_length() - 1
        bricks += list(range(base, base + n))
        lods += [full] * n
        base += n
    brick_b = np.concatenate([[b] * n for n, b in sizes_b])
    for _ in range(n_extra):
        k = int(rng.integers(0, total))
        bricks.append(k)
        lods.append(int(rng.integers(0, int(brick_b[k]).bit_length())))
    bricks, lods = np.array(bricks), np.array(lods)
    sizes = 8 ** lods.astype(np.uint64)
    dst = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    return requests(bricks, lods, dst), bricks, lods, dst, int(sizes.sum())


def _check(out, bricks, lods, dst, parts_ref, offsets):
    for k in range(len(bricks)):
        g = int(bricks[k])
        part = max(i for i, o in enumerate(offsets) if o <= g)
        ref = parts_ref[(part, int(lods[k]))][g - offsets[part]]
        got = out[int(dst[k]):int(dst[k]) + len(ref)]
        assert np.array_equal(got, ref), (k, g, int(lods[k]))


@pytest.fixture(scope="module")
def mixed(codec, oracle):
    imgs = _parts(codec, oracle)
    dss = [codec.open(im) for im in imgs]
    cat = codec.concat(dss)
    sizes_b = [(d.num_bricks, d.brick_size) for d in dss]
    offsets = list(np.cumsum([0] + [n for n, _ in sizes_b])[:-1])
    parts_ref = {}
    for i, im in enumerate(imgs):
        for t in range(sizes_b[i][1].bit_length()):
            parts_ref[(i, t)] = oracle.decode_image(im, t)[0]
    yield cat, dss, sizes_b, offsets, parts_ref
    cat.close()
    for d in dss:
        d.close()


def test_concat_mixed_brick_sizes_one_launch(codec, mixed):
    import torch
    from csvb200 import requests_tensor
    cat, dss, sizes_b, offsets, parts_ref = mixed
    assert cat.num_bricks == sum(n for n, _ in sizes_b)
    reqs, bricks, lods, dst, total = _mixed_requests(sizes_b, np.random.default_rng(4))
    out = torch.full((total,), -3, dtype=torch.int64, device="cuda")
    st = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
    codec.decode_batch(cat, requests_tensor(reqs), out, st)
    torch.cuda.synchronize()
    assert int(st.abs().max()) == 0
    _check(out.cpu().numpy().view(np.uint64), bricks, lods, dst, parts_ref, offsets)


def test_concat_rejects_lod_beyond_its_brick(codec, mixed):
    import torch
    from csvb200 import CSV_BRICK_BADREQ, requests, requests_tensor
    cat, dss, sizes_b, offsets, parts_ref = mixed
    reqs = requests([0, offsets[1]], [6, 6], [0, 0])  # brick 0 is 32^3 (levels 0..5): lod 6 is invalid
    out = torch.zeros(64 ** 3, dtype=torch.int64, device="cuda")
    st = torch.zeros(2, dtype=torch.int32, device="cuda")
    codec.decode_batch(cat, requests_tensor(reqs), out, st)
    assert st.cpu().numpy().tolist() == [CSV_BRICK_BADREQ, 0]


@pytest.mark.parametrize("cfg", [(0, 1, 1, 0), (1, 0, 0, 0), (2, 1, 0, 0), (1, 1, 1, 0), (0, 1, 1, 1), (2, 0, 0, 1),
                                 (0, 1, 1, 2), (1, 0, 0, 2)])
def test_graph_replay_matches(codec, mixed, cfg):
    import torch
    from csvb200 import DecodeConfig, requests_tensor
    cat, dss, sizes_b, offsets, parts_ref = mixed
    reqs, bricks, lods, dst, total = _mixed_requests(sizes_b, np.random.default_rng(5))
    out = torch.zeros(total, dtype=torch.int64, device="cuda")
    st = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
    g = codec.decode_graph(cat, requests_tensor(reqs), out, st, DecodeConfig(*cfg))
    for _ in range(3):
        out.zero_()
        g.launch()
        torch.cuda.synchronize()
        assert int(st.abs().max()) == 0
        _check(out.cpu().numpy().view(np.uint64), bricks, lods, dst, parts_ref, offsets)
    g.close()


def test_split_graph_finishes_before_later_stream_work(codec, mixed):
    """In a split graph each launch (the 64^3 outputs by palette class, then the small outputs) may start
    while the one before still has CTAs running, and the replay ends only after all have: work queued after
    the graph on the same stream, with no synchronisation between, reads every label of every launch."""
    import torch
    from csvb200 import DecodeConfig, requests_tensor
    cat, dss, sizes_b, offsets, parts_ref = mixed
    reqs, bricks, lods, dst, total = _mixed_requests(sizes_b, np.random.default_rng(9))
    assert (lods > 5).any() and (lods <= 5).any()  # both launches have work
    out = torch.zeros(total, dtype=torch.int64, device="cuda")
    st = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
    g = codec.decode_graph(cat, requests_tensor(reqs), out, st, DecodeConfig(0, 1, 0, 0))
    assert g.kernels in (2, 3)  # 3 when the 64^3 outputs span both palette classes
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            out.fill_(-3)
            g.launch(s)
            got, got_st = out.clone(), st.clone()  # same stream, straight after the replay
            s.synchronize()
            assert int(got_st.abs().max()) == 0
            _check(got.cpu().numpy().view(np.uint64), bricks, lods, dst, parts_ref, offsets)
    g.close()


def test_autotune_returns_a_working_config(codec, mixed):
    import torch
    from csvb200 import requests_tensor
    cat, dss, sizes_b, offsets, parts_ref = mixed
    reqs, bricks, lods, dst, total = _mixed_requests(sizes_b, np.random.default_rng(6))
    d_reqs = requests_tensor(reqs)
    out = torch.zeros(total, dtype=torch.int64, device="cuda")
    st = torch.zeros(len(reqs), dtype=torch.int32, device="cuda")
    best, ms = codec.autotune(cat, d_reqs, out, st, reps=3)
    assert ms > 0 and best.ctas_per_sm in (0, 1, 2) and best.stage in (0, 1) and best.lpt in (0, 1)
    assert best.layout in (0, 1, 2)
    out.zero_()
    g = codec.decode_graph(cat, d_reqs, out, st, best)
    g.launch()
    torch.cuda.synchronize()
    _check(out.cpu().numpy().view(np.uint64), bricks, lods, dst, parts_ref, offsets)
    g.close()


def _graph_run(codec, cat, reqs, total, layout=0):
    import torch
    from csvb200 import DecodeConfig, requests_tensor
    out = torch.full((max(total, 1),), -3, dtype=torch.int64, device="cuda")
    st = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
    g = codec.decode_graph(cat, requests_tensor(reqs), out, st, DecodeConfig(0, 1, 0, layout))
    g.launch()
    torch.cuda.synchronize()
    g.close()
    return out.cpu().numpy().view(np.uint64), st.cpu().numpy()


@pytest.mark.parametrize("layout", [0, 1, 2])
@pytest.mark.parametrize("part", ["coarse_only", "full64_only", "mix_with_bad"])
def test_graph_split_by_output_size(codec, mixed, part, layout):
    """A dataset with 64^3 bricks is decoded by two launches (outputs above 32^3, then the rest at three times
    the occupancy, overlapping the first launch's tail; layout 0) or by the small kernel alone (layout 1);
    either part may be empty, and a refused request in either part leaves the others intact."""
    from csvb200 import CSV_BRICK_BADREQ, requests
    cat, dss, sizes_b, offsets, parts_ref = mixed
    rng = np.random.default_rng(8)
    brick_b = np.concatenate([[b] * n for n, b in sizes_b])
    if part == "coarse_only":
        bricks = np.arange(len(brick_b))
        lods = np.array([int(rng.integers(0, min(6, int(b).bit_length()))) for b in brick_b])
    elif part == "full64_only":
        bricks = np.nonzero(brick_b == 64)[0]
        lods = np.full(len(bricks), 6)
    else:
        bricks = np.concatenate([np.arange(len(brick_b)), [0, len(brick_b) + 5, offsets[1]]])
        lods = np.concatenate([[int(b).bit_length() - 1 for b in brick_b], [6, 2, 5]])
    sizes = 8 ** lods.astype(np.uint64)
    dst = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    out, st = _graph_run(codec, cat, requests(bricks, lods, dst), int(sizes.sum()), layout)
    bad = np.zeros(len(bricks), bool)
    if part == "mix_with_bad":
        bad[-3:-1] = True  # a 32^3 brick at LOD 6, a brick past the end
        assert st[bad].tolist() == [CSV_BRICK_BADREQ, CSV_BRICK_BADREQ]
    assert int(np.abs(st[~bad]).max()) == 0
    keep = np.nonzero(~bad)[0]
    _check(out, bricks[keep], lods[keep], dst[keep], parts_ref, offsets)


def test_wide_palettes_in_both_kernel_variants(codec, oracle):
    """Bricks with more than 65535 palette entries (32-bit node values in shared memory), decoded at 64^3 by
    the large variant and at 32^3 and coarser by the small one, in one graph and in one batch."""
    import torch
    from csvb200 import requests, requests_tensor
    g = torch.Generator(device="cuda")
    g.manual_seed(12)
    vol = torch.randint(1, 1 << 40, (64, 64, 128), dtype=torch.int64, device="cuda", generator=g)
    vol[:, :, :16] = 7  # a coarse region so that not every node is a new label
    codec.encode_device(vol, 64)
    img = bytes(codec.encoded_image_tensor().cpu().numpy())
    ds = codec.open(img)
    ref = {t: oracle.decode_image(img, t)[0] for t in range(7)}
    bricks = np.array([0, 1, 0, 1, 1, 0])
    lods = np.array([6, 5, 4, 6, 0, 5])
    sizes = 8 ** lods.astype(np.uint64)
    dst = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    reqs = requests(bricks, lods, dst)
    out, st = _graph_run(codec, ds, reqs, int(sizes.sum()))
    out1, st1 = _graph_run(codec, ds, reqs, int(sizes.sum()), layout=1)  # 32-bit level 5 in scratch
    out2 = torch.zeros(int(sizes.sum()), dtype=torch.int64, device="cuda")
    st2 = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
    codec.decode_batch(ds, requests_tensor(reqs), out2, st2)
    torch.cuda.synchronize()
    for o, s in ((out, st), (out1, st1), (out2.cpu().numpy().view(np.uint64), st2.cpu().numpy())):
        assert int(np.abs(s).max()) == 0
        for k in range(len(bricks)):
            r = ref[int(lods[k])][int(bricks[k])]
            assert np.array_equal(o[int(dst[k]):int(dst[k]) + len(r)], r), k
    ds.close()


def test_graph_reports_its_kernels(codec, mixed):
    """csv_graph_kernels: two or three decode kernels per replay when a dataset with 64^3 bricks is split by
    output size and palette size (layout 0; three when its 64^3 outputs have palettes both below and above
    255 entries), two when split by output size alone (layout 2), one with layout 1, none for an empty
    batch."""
    import torch
    from csvb200 import DecodeConfig, requests_tensor
    cat, dss, sizes_b, offsets, parts_ref = mixed
    reqs, bricks, lods, dst, total = _mixed_requests(sizes_b, np.random.default_rng(5))
    out = torch.zeros(total, dtype=torch.int64, device="cuda")
    st = torch.zeros(len(reqs), dtype=torch.int32, device="cuda")
    for layout, want in ((0, (2, 3)), (1, (1,)), (2, (2,))):
        g = codec.decode_graph(cat, requests_tensor(reqs), out, st, DecodeConfig(0, 1, 0, layout))
        assert g.kernels in want
        g.close()
    g = codec.decode_graph(cat, requests_tensor(reqs), out, st, n=0)
    assert g.kernels == 0
    g.close()


def test_graph_three_parts_by_palette_size(codec, oracle):
    """64^3 outputs of bricks with fewer than 255 palette entries go to the 8-bit variant (three CTAs per SM),
    the other 64^3 outputs to the 16-bit one, and 32^3 and coarser outputs to the small kernel (8-bit values,
    seven CTAs per SM, when all of them have small palettes; else 16-bit, six): three launches (layout 0),
    two without the 8-bit part (layout 2), one with layout 1; every output equals the oracle's, and so does
    one csv_decode_batch of the same requests."""
    import torch
    from csvb200 import requests, requests_tensor
    imgs = []
    for cells, seed in ((24, 41), (9000, 42)):  # palettes of a few entries, and of thousands
        vol = torch.empty((64, 64, 192), dtype=torch.int64, device="cuda")
        codec.synth_volume(vol, 0, cells, 0, 1.0, 1.0, 0.1, seed)
        codec.encode_device(vol, 64)
        imgs.append(bytes(codec.encoded_image_tensor().cpu().numpy()))
    dss = [codec.open(im) for im in imgs]
    cat = codec.concat(dss)
    pal = []
    for im in imgs:
        n = int(np.frombuffer(im[8:12], np.uint32)[0])
        o = 152
        for _ in range(n):
            P = int(np.frombuffer(im[o + 4:o + 8], np.uint32)[0])
            pal.append(P)
            o += 8 + 8 * P
            E = int(np.frombuffer(im[o:o + 4], np.uint32)[0])
            o += 4 + E + 4
    pal = np.array(pal)
    assert (pal[:3] < 255).all() and (pal[3:] >= 255).all() and (pal[3:] < 65535).all()
    ref = {}
    for k, im in enumerate(imgs):
        for t in range(7):
            ref[(k, t)] = oracle.decode_image(im, t)[0]
    rng = np.random.default_rng(3)
    bricks = np.concatenate([np.arange(6), rng.integers(0, 6, 30)])
    lods = np.concatenate([np.full(6, 6), rng.integers(0, 7, 30)])
    sizes = 8 ** lods.astype(np.uint64)
    dst = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    reqs = requests(bricks, lods, dst)
    total = int(sizes.sum())

    def check(out, st):
        assert int(np.abs(st).max()) == 0
        for k in range(len(bricks)):
            g = int(bricks[k])
            r = ref[(g // 3, int(lods[k]))][g % 3]
            assert np.array_equal(out[int(dst[k]):int(dst[k]) + len(r)], r), (k, g, int(lods[k]))

    from csvb200 import DecodeConfig
    for layout, want in ((0, 3), (2, 2), (1, 1)):
        out = torch.full((total,), -3, dtype=torch.int64, device="cuda")
        st = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
        g = codec.decode_graph(cat, requests_tensor(reqs), out, st, DecodeConfig(0, 1, 1, layout))
        assert g.kernels == want, layout
        for _ in range(2):
            out.fill_(-3)
            g.launch()
            torch.cuda.synchronize()
            check(out.cpu().numpy().view(np.uint64), st.cpu().numpy())
        g.close()
    out = torch.full((total,), -3, dtype=torch.int64, device="cuda")
    st = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
    codec.decode_batch(cat, requests_tensor(reqs), out, st)
    torch.cuda.synchronize()
    check(out.cpu().numpy().view(np.uint64), st.cpu().numpy())
    # requests of the small-palette bricks only: both launches (64^3 outputs, then 32^3 and coarser) take
    # 8-bit node values
    bricks = np.concatenate([np.arange(3), rng.integers(0, 3, 30)])
    lods = np.concatenate([np.full(3, 6), rng.integers(0, 6, 30)])
    sizes = 8 ** lods.astype(np.uint64)
    dst = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    reqs = requests(bricks, lods, dst)
    total = int(sizes.sum())
    out = torch.full((total,), -3, dtype=torch.int64, device="cuda")
    st = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
    g = codec.decode_graph(cat, requests_tensor(reqs), out, st, DecodeConfig(0, 1, 0, 0))
    assert g.kernels == 2
    g.launch()
    torch.cuda.synchronize()
    check(out.cpu().numpy().view(np.uint64), st.cpu().numpy())
    g.close()
    cat.close()
    for d in dss:
        d.close()


def test_palette_size_boundary_254_255(codec, oracle):
    """The 8-bit node values stop at palettes of 254 entries (0xFF is kept for label 0): a brick with 254
    distinct labels and one with 255, decoded at every LOD by csv_decode_batch (the dataset as a whole takes
    16 bits), by a split graph (the first brick's 64^3 output in the 8-bit kernel, the second's in the
    16-bit one), and alone (the 254-label image takes 8 bits in both variants), all equal to the oracle."""
    import torch
    from csvb200 import DecodeConfig, requests, requests_tensor
    # one label per x-row of 4^3 blocks (the rows past n - 1 keep the last one); n = 158 and 159 give the
    # encoder's palettes of exactly 254 and 255 entries (its coarse levels add entries of their own)
    def brick(n):
        labels = np.random.default_rng(5).integers(1, 1 << 62, n, dtype=np.uint64)
        sub = np.zeros((16, 16, 16), np.uint64)
        for bz in range(16):
            for by in range(16):
                sub[bz, by, :] = labels[min(16 * bz + by, n - 1)]
        return np.repeat(np.repeat(np.repeat(sub, 4, 0), 4, 1), 4, 2)
    vol = np.zeros((64, 64, 128), np.uint64)
    vol[:, :, :64] = brick(158)
    vol[:, :, 64:] = brick(159)
    img_both = codec.encode(vol, 64)
    img_254 = codec.encode(np.ascontiguousarray(vol[:, :, :64]), 64)
    for img, pals in ((img_both, (254, 255)), (img_254, (254,))):
        o, got = 152, []
        for _ in pals:
            P = int(np.frombuffer(img[o + 4:o + 8], np.uint32)[0])
            got.append(P)
            o += 8 + 8 * P
            E = int(np.frombuffer(img[o:o + 4], np.uint32)[0])
            o += 4 + E + 4
        assert tuple(got) == pals
        ref = {t: oracle.decode_image(img, t)[0] for t in range(7)}
        ds = codec.open(img)
        nb = len(pals)
        bricks = np.concatenate([np.arange(nb)] * 7)
        lods = np.repeat(np.arange(7), nb)
        sizes = 8 ** lods.astype(np.uint64)
        dst = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
        reqs = requests(bricks, lods, dst)
        total = int(sizes.sum())
        outs = []
        out = torch.full((total,), -3, dtype=torch.int64, device="cuda")
        st = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
        codec.decode_batch(ds, requests_tensor(reqs), out, st)
        torch.cuda.synchronize()
        outs.append((out.cpu().numpy().view(np.uint64), st.cpu().numpy()))
        for layout in (0, 1, 2):
            out = torch.full((total,), -3, dtype=torch.int64, device="cuda")
            st = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
            g = codec.decode_graph(ds, requests_tensor(reqs), out, st, DecodeConfig(0, 1, 0, layout))
            g.launch()
            torch.cuda.synchronize()
            g.close()
            outs.append((out.cpu().numpy().view(np.uint64), st.cpu().numpy()))
        for o_, s_ in outs:
            assert int(np.abs(s_).max()) == 0
            for k in range(len(bricks)):
                r = ref[int(lods[k])][int(bricks[k])]
                assert np.array_equal(o_[int(dst[k]):int(dst[k]) + len(r)], r), (pals, k)
        ds.close()
