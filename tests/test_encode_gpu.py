"""GPU: the encoder (csv_encode / csv_encode_device) is byte-identical to the reference encoder.

Expected bytes come from the golden fixtures (made by the reference sources
compiled here) and from the oracle restatement, which tests/test_oracle.py pins
against the reference.  The seek index the encoder emits is checked by decoding
its image at every LOD (csv_open_encoded) against the oracle.
"""
import hashlib

import numpy as np
import pytest

from conftest import read_golden
from test_oracle import crop_volume

pytestmark = pytest.mark.gpu

GOLDEN_CASES = ["voronoi_96x80x72_b64", "tubes_64_b32", "tubes_64_b16", "uniform_64_b64",
                "mixed_uniform_128x64x64_b64"]


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_bytes(codec, oracle, golden, name):
    g = golden[name]
    img = read_golden(name)
    b = g["brick_size"]
    full, st = oracle.decode_image(img, b.bit_length() - 1)
    vol = crop_volume(full, g["shape_dhw"], b, None)
    out = codec.encode(vol, b)
    assert hashlib.sha256(out).hexdigest() == g["bytes_sha256"]


def _device_volume(codec, shape, kind, **kw):
    import torch
    d = torch.empty(shape, dtype=torch.int64, device="cuda")
    codec.synth_volume(d, kind, **kw)
    torch.cuda.synchronize()
    return d


@pytest.mark.parametrize("b", [64, 32, 16, 8, 4, 2])
def test_device_volume_bytes_vs_oracle(codec, oracle, b):
    d = _device_volume(codec, (80, 72, 136), 1, n_cells=250, n_tubes=30, r_min=1.0, r_max=7.0, zero_frac=0.2,
                       seed=40 + b)
    vol = d.cpu().numpy().view(np.uint64)
    n = codec.encode_device(d, b)
    img = bytes(codec.encoded_image_tensor().cpu().numpy())
    assert len(img) == n
    assert img == oracle.encode(vol, b)


def test_bytes_vs_compiled_reference(codec, reference):
    d = _device_volume(codec, (64, 128, 128), 1, n_cells=400, n_tubes=40, r_min=2.0, r_max=10.0, zero_frac=0.15,
                       seed=77)
    vol = d.cpu().numpy().view(np.uint64)
    assert codec.encode(vol, 64) == reference.encode(vol, 64)


def test_frequency_sample_spans_bricks_0_and_512(codec, oracle):
    """Only bricks with file index % 512 == 0 feed the shared model (brickEncoding.hpp:481-482)."""
    d = _device_volume(codec, (72, 64, 64), 0, n_cells=500, zero_frac=0.1, seed=5)  # 8x8x9 = 576 bricks of 8^3
    vol = d.cpu().numpy().view(np.uint64)
    codec.encode_device(d, 8)
    img = bytes(codec.encoded_image_tensor().cpu().numpy())
    assert int(np.frombuffer(img[8:12], np.uint32)[0]) == 576
    assert img == oracle.encode(vol, 8)


def test_tie_heavy_volume(codec, oracle):
    """Few labels with many 4/4 and 2/2/2/2 ties at every pyramid level (majorityVote8 tie rule)."""
    rng = np.random.default_rng(3)
    labels = np.array([13, 26, 39, 1, 14, 2, 3, 0xFFFFFFFFFFFFFFF0], np.uint64)
    vol = labels[rng.integers(0, 8, (64, 64, 64))]
    vol[::2] = labels[rng.integers(0, 3, (32, 64, 64))]
    assert codec.encode(vol, 64) == oracle.encode(vol, 64)
    assert codec.encode(vol, 16) == oracle.encode(vol, 16)


def test_empty_and_tiny_volumes(codec, oracle):
    for shape in [(1, 1, 1), (3, 5, 7), (64, 64, 65)]:
        vol = (np.arange(np.prod(shape), dtype=np.uint64) % 5 + 1).reshape(shape)
        assert codec.encode(vol, 64) == oracle.encode(vol, 64), shape


def test_encoder_seek_index_decodes_every_lod(codec, oracle):
    import torch
    from csvb200 import requests, requests_tensor
    d = _device_volume(codec, (128, 64, 128), 1, n_cells=300, n_tubes=50, r_min=1.0, r_max=8.0, zero_frac=0.15,
                       seed=91)
    codec.encode_device(d, 64)
    img = bytes(codec.encoded_image_tensor().cpu().numpy())
    ds = codec.open_encoded()
    nb = ds.num_bricks
    for t in range(7):
        per = 8 ** t
        reqs = requests(np.arange(nb), np.full(nb, t), np.arange(nb, dtype=np.uint64) * per)
        out = torch.empty(nb * per, dtype=torch.int64, device="cuda")
        st = torch.zeros(nb, dtype=torch.int32, device="cuda")
        codec.decode_batch(ds, requests_tensor(reqs), out, st)
        ref, rst = oracle.decode_image(img, t)
        assert (st.cpu().numpy() == 0).all()
        assert np.array_equal(out.cpu().numpy().view(np.uint64).reshape(nb, per), ref), t
    ds.close()


@pytest.mark.parametrize("shards", [2, 3])
def test_sharded_encode_on_the_device_equals_whole(codec, shards):
    """csv_encode_shard_bricks / csv_encode_shard_finish, one context per x-slab (as one rank each would run
    them): the slabs' records behind one header with the summed sample histogram's model are the whole-volume
    image byte for byte (1536 bricks, so that the every-512th sample falls on several slabs)."""
    from csvb200 import Codec
    from csvb200.dist import DeviceShardEncoder, assemble, slab_of, slab_ranges
    b = 8
    vol = _device_volume(codec, (64, 64, 192), 1, n_cells=200, n_tubes=40, r_min=1.0, r_max=5.0, zero_frac=0.1,
                         seed=91)
    codec.encode_device(vol, b)
    whole = bytes(codec.encoded_image_tensor().cpu().numpy())
    D, H, W = vol.shape
    nyz = -(-H // b) * -(-D // b)
    encs = [DeviceShardEncoder(Codec(0)) for _ in range(shards)]
    ranges = slab_ranges(W, b, shards)
    hists = [e.bricks(slab_of(vol, b, bx0, bx1), b, bx0, bx0 * nyz) for e, (bx0, bx1) in zip(encs, ranges)]
    total = np.sum(hists, axis=0).astype(np.uint64)
    assert assemble([e.finish(total) for e in encs]) == whole


def test_real_bricks_encode_like_the_oracle(codec, oracle):
    """Real segmentation: the MICrONS bricks of the shipped-file subset (tests/golden/shipped_subset.csbd,
    the smallest, median and largest streams and a few spread over the file), decoded and laid side by side
    along x as one volume, encode on the device to the oracle's bytes (the oracle matches the compiled
    reference encoder on the whole 512^3 shipped volume, tests/test_npy_real_data.py)."""
    import torch
    from conftest import read_golden
    img = read_golden("shipped_subset")
    full, st = oracle.decode_image(img, 6)
    assert int(st.max()) == 0
    m = np.arange(64)
    sp = np.zeros(64, np.int64)
    for k in range(10):
        sp |= ((m >> k) & 1) << (3 * k)
    morton = sp[None, None, :] | (sp[None, :, None] << 1) | (sp[:, None, None] << 2)  # [z, y, x]
    vol = np.concatenate([full[i][morton] for i in range(len(full))], axis=2)  # (64, 64, 64 n)
    d = torch.from_numpy(vol.view(np.int64)).cuda()
    codec.encode_device(d, 64)
    assert bytes(codec.encoded_image_tensor().cpu().numpy()) == oracle.encode(vol, 64)
