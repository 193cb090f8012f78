"""GPU: csv_decode_batch_static, the decode entry point that allocates nothing.

It is for callers that cannot call cudaMalloc while they decode (a render loop
that must not stall the device, a host whose device memory all comes from its
own arena).  Its scratch is one fixed device array inside the library, so this
test calls it through the C ABI twice in a row -- the second call runs on the
scratch the first left behind -- and checks both results against
csv_decode_batch, label for label.  This file sorts last so that a run which
stops at the first failure has run every other test already; it also passes
alone in a fresh process.
"""
import numpy as np
import pytest

from conftest import read_golden

pytestmark = pytest.mark.gpu


def _requests(nb, lods, seed):
    from csvb200 import requests
    rng = np.random.default_rng(seed)
    bricks = rng.permutation(np.concatenate([np.arange(nb), rng.integers(0, nb, nb)]))
    lod = rng.choice(lods, len(bricks))
    sizes = 8 ** lod.astype(np.uint64)
    dst = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    return requests(bricks, lod, dst), int(sizes.sum())


@pytest.mark.parametrize("name", ["shipped_subset", "tubes_64_b32"])
def test_static_decode_matches_allocating_decode_twice(codec, name):
    import torch
    from csvb200 import requests_tensor
    img = read_golden(name)
    ds = codec.open(img)
    b = ds.brick_size
    lods = np.arange(b.bit_length())
    for call in range(2):
        reqs, total = _requests(ds.num_bricks, lods, seed=11 + call)
        d_reqs = requests_tensor(reqs)
        ref = torch.full((total,), -1, dtype=torch.int64, device="cuda")
        got = torch.full((total,), -2, dtype=torch.int64, device="cuda")
        st_ref = torch.full((len(reqs),), -1, dtype=torch.int32, device="cuda")
        st_got = torch.full((len(reqs),), -2, dtype=torch.int32, device="cuda")
        codec.decode_batch(ds, d_reqs, ref, st_ref)
        codec.decode_batch_static(ds, d_reqs, got, st_got)
        torch.cuda.synchronize()
        assert torch.equal(st_got, st_ref) and int(st_got.abs().max()) == 0, call
        assert torch.equal(got, ref), call
    ds.close()


def test_static_decode_shipped_subset_golden_hashes(codec, golden):
    """Every LOD of the shipped MICrONS bricks, decoded by the allocation-free entry point (twice, so that the
    second call starts from the first call's scratch), hashed against the golden fixture: the reference
    decoder's output at full resolution, the decode.wgsl restatement at coarser LODs."""
    import hashlib

    import torch
    from csvb200 import requests, requests_tensor
    img = read_golden("shipped_subset")
    ds = codec.open(img)
    nb = ds.num_bricks
    for call in range(2):
        for lod in range(ds.brick_size.bit_length()):
            per = 8 ** lod
            reqs = requests_tensor(requests(np.arange(nb), np.full(nb, lod), np.arange(nb, dtype=np.uint64) * per))
            out = torch.full((nb * per,), -1, dtype=torch.int64, device="cuda")
            st = torch.full((nb,), -1, dtype=torch.int32, device="cuda")
            codec.decode_batch_static(ds, reqs, out, st)
            torch.cuda.synchronize()
            assert int(st.abs().max()) == 0, (call, lod)
            h = out.cpu().numpy().view(np.uint64).reshape(nb, per)
            got = [hashlib.sha256(np.ascontiguousarray(h[k]).tobytes()).hexdigest() for k in range(nb)]
            assert got == golden["shipped_subset"]["lod"][str(lod)], (call, lod)
    ds.close()


def test_static_decode_encoder_dataset_full_resolution(codec):
    """A 64^3-brick dataset from the encoder: 256 bricks through the 47 concurrent slots of the array."""
    import torch
    from csvb200 import requests, requests_tensor
    vol = torch.empty((128, 256, 512), dtype=torch.int64, device="cuda")
    codec.synth_volume(vol, 1, 800, 80, 2.0, 10.0, 0.15, 23)
    codec.encode_device(vol, 64)
    ds = codec.open_encoded()
    nb = ds.num_bricks
    per = 64 ** 3
    reqs = requests_tensor(requests(np.arange(nb), np.full(nb, 6), np.arange(nb, dtype=np.uint64) * per))
    ref = torch.empty(nb * per, dtype=torch.int64, device="cuda")
    st = torch.zeros(nb, dtype=torch.int32, device="cuda")
    codec.decode_batch(ds, reqs, ref, st)
    for _ in range(2):
        got = torch.zeros(nb * per, dtype=torch.int64, device="cuda")
        st2 = torch.full((nb,), -1, dtype=torch.int32, device="cuda")
        codec.decode_batch_static(ds, reqs, got, st2)
        torch.cuda.synchronize()
        assert int(st2.abs().max()) == 0
        assert torch.equal(got, ref)
    ds.close()
