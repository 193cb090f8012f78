"""GPU: the batched brick decoder (csv_decode_batch / csv_decode_image) against the oracle and golden fixtures.

Bit-exact: decoded labels are integers and must equal the oracle's (the
reference C++ decoder at full resolution, the decode.wgsl restatement at
coarser LODs) label for label.
"""
import hashlib
import struct

import numpy as np
import pytest

from conftest import read_golden

pytestmark = pytest.mark.gpu

SYNTH_CASES = ["voronoi_96x80x72_b64", "tubes_64_b32", "tubes_64_b16", "uniform_64_b64",
               "mixed_uniform_128x64x64_b64"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("lod", range(7))
def test_shipped_subset_every_lod(codec, golden, lod):
    img = read_golden("shipped_subset")
    out, st = codec.decode_image(img, lod)
    assert st.max() == 0
    assert [sha(out[k]) for k in range(out.shape[0])] == golden["shipped_subset"]["lod"][str(lod)]


@pytest.mark.parametrize("name", SYNTH_CASES)
def test_golden_synthetic_every_lod(codec, golden, name):
    img = read_golden(name)
    g = golden[name]
    for t in range(g["brick_size"].bit_length()):
        out, st = codec.decode_image(img, t)
        assert st.max() == 0
        assert [sha(out[k]) for k in range(out.shape[0])] == g["lod"][str(t)], (name, t)


def test_uniform_brick_is_palette0(codec):
    img = read_golden("uniform_64_b64")
    out, st = codec.decode_image(img, 6)
    assert st.max() == 0 and np.all(out == np.uint64(0x1234567890ABCDEF))


def _device_volume(codec, shape, kind, **kw):
    import torch
    d = torch.empty(shape, dtype=torch.int64, device="cuda")
    codec.synth_volume(d, kind, **kw)
    torch.cuda.synchronize()
    return d


@pytest.mark.parametrize("b", [64, 32, 16, 8])
def test_device_synth_volume_roundtrip_vs_oracle(codec, oracle, b):
    d = _device_volume(codec, (96, 64, 128), 1, n_cells=300, n_tubes=40, r_min=1.0, r_max=6.0, zero_frac=0.15,
                       seed=3 + b)
    vol = d.cpu().numpy().view(np.uint64)
    img = oracle.encode(vol, b)
    for t in range(b.bit_length()):
        ref, rst = oracle.decode_image(img, t)
        out, st = codec.decode_image(img, t)
        assert rst.max() == 0 and st.max() == 0
        assert np.array_equal(out, ref), (b, t)


def test_batch_mixed_lods_offsets_and_repeats(codec, oracle):
    import torch
    from csvb200 import requests, requests_tensor
    img = read_golden("shipped_subset")
    ds = codec.open(img)
    nb = ds.num_bricks
    rng = np.random.default_rng(7)
    bricks = rng.integers(0, nb, 40)
    lods = rng.integers(0, 7, 40)
    sizes = 8 ** lods
    dst = np.zeros(40, np.uint64)
    off = 3  # odd offsets exercise the unaligned store path
    for k in range(40):
        dst[k] = off
        off += int(sizes[k]) + int(rng.integers(0, 3))
    reqs = requests(bricks, lods, dst)
    d_out = torch.full((off + 5,), -7, dtype=torch.int64, device="cuda")
    d_st = torch.full((40,), -1, dtype=torch.int32, device="cuda")
    codec.decode_batch(ds, requests_tensor(reqs), d_out, d_st)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().view(np.uint64)
    assert (d_st.cpu().numpy() == 0).all()
    ref = {t: oracle.decode_image(img, t)[0] for t in range(7)}
    for k in range(40):
        got = out[int(dst[k]):int(dst[k]) + int(sizes[k])]
        assert np.array_equal(got, ref[int(lods[k])][int(bricks[k])]), k
    # bytes between requests are untouched
    mask = np.ones(len(out), bool)
    for k in range(40):
        mask[int(dst[k]):int(dst[k]) + int(sizes[k])] = False
    assert (out[mask] == np.uint64(2 ** 64 - 7)).all()
    ds.close()


def test_bad_requests_report_status(codec):
    import torch
    from csvb200 import CSV_BRICK_BADREQ, requests, requests_tensor
    ds = codec.open(read_golden("shipped_subset"))
    reqs = requests([0, ds.num_bricks, 1], [7, 3, 2], [0, 0, 0])
    d_out = torch.zeros(1024, dtype=torch.int64, device="cuda")
    d_st = torch.zeros(3, dtype=torch.int32, device="cuda")
    codec.decode_batch(ds, requests_tensor(reqs), d_out, d_st)
    st = d_st.cpu().numpy()
    assert st[0] == CSV_BRICK_BADREQ and st[1] == CSV_BRICK_BADREQ and st[2] == 0
    ds.close()


def test_empty_batch_is_ok(codec):
    import torch
    ds = codec.open(read_golden("tubes_64_b32"))
    e = torch.zeros(0, dtype=torch.uint8, device="cuda")
    codec.decode_batch(ds, e, torch.zeros(1, dtype=torch.int64, device="cuda"),
                       torch.zeros(1, dtype=torch.int32, device="cuda"), n=0)
    ds.close()


def _patch_brick(img: bytes, index: int, P=None, nsym=None) -> bytes:
    b = bytearray(img)
    o = 152
    for i in range(index + 1):
        ID, Pk = struct.unpack_from("<2I", b, o)
        po = o + 4
        o += 8 + 8 * Pk
        E = struct.unpack_from("<I", b, o)[0]
        o += 4 + E
        no = o
        o += 4
    if nsym is not None:
        struct.pack_into("<I", b, no, nsym)
    if P is not None:
        # shrink the palette in place: keep the record layout valid by removing entries
        Pk = struct.unpack_from("<I", b, po)[0]
        cut = (Pk - P) * 8
        start = po + 4 + 8 * P
        del b[start:start + cut]
        struct.pack_into("<I", b, po, P)
    return bytes(b)


def test_forged_palette_overrun_is_clamped_like_wgsl(codec, oracle):
    from csvb200 import CSV_BRICK_PALETTE
    img = _patch_brick(read_golden("shipped_subset"), 3, P=9)  # brick 3 has a 67-entry palette
    for t in (3, 5, 6):
        out, st = codec.decode_image(img, t, check=False)
        ref, rst = oracle.decode_image(img, t)
        # the flag appears once the decoded levels reach a palette index past the cut
        assert bool(st[3] & CSV_BRICK_PALETTE) == bool(rst[3] & 2), t
        assert np.array_equal(out, ref), t
    assert st[3] & CSV_BRICK_PALETTE


def test_truncated_stream_reports_truncation(codec):
    from csvb200 import CSV_BRICK_TRUNCATED
    img = read_golden("shipped_subset")
    ns = 2000
    bad = _patch_brick(img, 1, nsym=ns)
    out, st = codec.decode_image(bad, 6, check=False)
    assert st[1] & CSV_BRICK_TRUNCATED
    assert st[0] == 0 and st[2] == 0


@pytest.mark.parametrize("b", [32, 64])
def test_decode_image_spans_several_chunks(codec, b):
    """csv_decode_image decodes in chunks of at most 256 MiB of labels through two device buffers (one chunk
    decodes while the previous one drains to the host).  A 384^3 volume (432 MiB of labels: two chunks, the
    second partial) comes back equal, brick for brick, to one device-side batch decode of the same image, on
    a first call and on a second one that reuses the buffers."""
    import torch
    from csvb200 import requests, requests_tensor
    vol = torch.empty((384, 384, 384), dtype=torch.int64, device="cuda")
    codec.synth_volume(vol, 1, 300, 40, 1.0, 5.0, 0.1, 77)
    codec.encode_device(vol, b)
    img = bytes(codec.encoded_image_tensor().cpu().numpy())
    del vol
    full = b.bit_length() - 1
    ds = codec.open(img)
    nb = ds.num_bricks
    dev = torch.empty(nb * b ** 3, dtype=torch.int64, device="cuda")
    st = torch.full((nb,), -1, dtype=torch.int32, device="cuda")
    codec.decode_batch(ds, requests_tensor(requests(np.arange(nb), np.full(nb, full),
                                                    np.arange(nb, dtype=np.uint64) * b ** 3)), dev, st)
    torch.cuda.synchronize()
    assert int(st.abs().max()) == 0
    ref = dev.cpu().numpy().view(np.uint64).reshape(nb, -1)
    del dev
    ds.close()
    for _ in range(2):
        out, hst = codec.decode_image(img, full)
        assert int(hst.max()) == 0
        assert np.array_equal(out, ref)
