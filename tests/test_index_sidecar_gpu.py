"""GPU: the seek-index sidecar (csv_index_save / csv_open_indexed) and the index pass's timing query.

A sidecar holds the rANS state before every 512th symbol of each brick.  Its
states must equal the oracle's serial chain (or_rans_states), a dataset opened
with it must decode bit for bit like one opened from the stream headers (and
like the golden fixtures), and a sidecar that does not belong to the image must
be refused with CSV_EFORMAT, whatever part of it is wrong.
"""
import hashlib
import struct

import numpy as np
import pytest

from conftest import read_golden

pytestmark = pytest.mark.gpu

SEED = 512
HEAD = 24


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def parse_sidecar(sc: bytes):
    magic, ver, nb, every, total = struct.unpack_from("<4IQ", sc, 0)
    assert (magic, ver, every) == (0x58565343, 1, SEED)
    rows = np.frombuffer(sc, np.uint32, 3 * nb, HEAD).reshape(nb, 3)
    states = np.frombuffer(sc, np.uint32, 2 * total, HEAD + 12 * nb).reshape(total, 2)
    assert len(sc) == HEAD + 12 * nb + 8 * total
    return rows, states


def build_sidecar(rows, states) -> bytes:
    rows = np.ascontiguousarray(rows, np.uint32)
    states = np.ascontiguousarray(states, np.uint32).reshape(-1, 2)
    return (struct.pack("<4IQ", 0x58565343, 1, rows.shape[0], SEED, states.shape[0]) + rows.tobytes()
            + states.tobytes())


def image_bricks(img: bytes):
    """(freq, cum, [(E, enc, nsym)]) of a .csbd v1 image (fileIO.cpp:25-96)."""
    freq = np.frombuffer(img[24:88], np.uint32)
    cum = np.frombuffer(img[88:152], np.uint32)
    nb = struct.unpack_from("<I", img, 8)[0]
    o, out = 152, []
    for _ in range(nb):
        _, P = struct.unpack_from("<2I", img, o)
        o += 8 + 8 * P
        E = struct.unpack_from("<I", img, o)[0]
        enc = img[o + 4:o + 4 + E]
        o += 4 + E
        out.append((E, enc, struct.unpack_from("<I", img, o)[0]))
        o += 4
    return freq, cum, out


def patch_nsym(img: bytes, index: int, nsym: int) -> bytes:
    b = bytearray(img)
    o = 152
    for i in range(index + 1):
        _, P = struct.unpack_from("<2I", b, o)
        o += 8 + 8 * P
        E = struct.unpack_from("<I", b, o)[0]
        o += 4 + E
        if i == index:
            struct.pack_into("<I", b, o, nsym)
        o += 4
    return bytes(b)


def decode_all(codec, ds, lod: int):
    import torch
    from csvb200 import requests, requests_tensor
    nb, per = ds.num_bricks, 1 << (3 * lod)
    out = torch.zeros(nb * per, dtype=torch.int64, device="cuda")
    st = torch.full((nb,), -1, dtype=torch.int32, device="cuda")
    codec.decode_batch(ds, requests_tensor(requests(np.arange(nb), np.full(nb, lod),
                                                    np.arange(nb, dtype=np.uint64) * per)), out, st)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint64).reshape(nb, per), st.cpu().numpy()


def test_sidecar_states_equal_the_oracle_chain_and_decode_every_lod(codec, oracle, golden):
    img = read_golden("shipped_subset")
    ds = codec.open(img)
    assert ds.index_ms > 0
    sc = ds.index_sidecar()
    rows, states = parse_sidecar(sc)
    freq, cum, bricks = image_bricks(img)
    at = 0
    for i, (E, enc, ns) in enumerate(bricks):
        assert tuple(rows[i]) == (E, ns, -(-ns // SEED))
        want = oracle.rans_states(freq, cum, enc, ns, SEED)
        assert np.array_equal(states[at:at + rows[i, 2]], want), i
        at += rows[i, 2]
    ds2 = codec.open(img, sidecar=sc)
    assert ds2.index_ms > 0
    for t in range(7):
        out, st = decode_all(codec, ds2, t)
        assert st.max() == 0
        assert [sha(out[k]) for k in range(out.shape[0])] == golden["shipped_subset"]["lod"][str(t)], t
    # the same sidecar again, from the dataset the sidecar opened
    assert ds2.index_sidecar() == sc
    ds.close()
    ds2.close()


@pytest.mark.parametrize("name", ["uniform_64_b64", "mixed_uniform_128x64x64_b64", "tubes_64_b16"])
def test_sidecar_golden_images(codec, golden, name):
    """Uniform bricks (root stop bit: no chain, no states) and small bricks (fewer than 512 symbols)."""
    img = read_golden(name)
    g = golden[name]
    sc = codec.open(img).index_sidecar()
    rows, _ = parse_sidecar(sc)
    ds = codec.open(img, sidecar=sc)
    for t in range(g["brick_size"].bit_length()):
        out, st = decode_all(codec, ds, t)
        assert st.max() == 0
        assert [sha(out[k]) for k in range(out.shape[0])] == g["lod"][str(t)], (name, t)
    if name == "uniform_64_b64":
        assert rows[:, 2].max() == 0
    ds.close()


@pytest.mark.parametrize("b", [64, 32])
def test_sidecar_of_an_encoder_dataset_equals_the_opened_one(codec, b):
    """csv_index_save on the encoder's own dataset (its index from the encoder) writes the same sidecar as on
    the image opened from its bytes, and opening with it decodes like csv_open."""
    import torch
    vol = torch.empty((96, 128, 160), dtype=torch.int64, device="cuda")
    codec.synth_volume(vol, 1, 300, 60, 1.0, 6.0, 0.15, 11 + b)
    codec.encode_device(vol, b)
    img = bytes(codec.encoded_image_tensor().cpu().numpy())
    del vol
    dse = codec.open_encoded()
    ds = codec.open(img)
    sc = ds.index_sidecar()
    assert dse.index_sidecar() == sc
    assert dse.index_ms == 0.0
    ds2 = codec.open(img, sidecar=sc)
    full = b.bit_length() - 1
    for t in (full, full - 2):
        a, sa = decode_all(codec, ds, t)
        c, sc2 = decode_all(codec, ds2, t)
        assert sa.max() == 0 and np.array_equal(sa, sc2) and np.array_equal(a, c), t
    for d in (dse, ds, ds2):
        d.close()


def test_sidecar_of_malformed_bricks(codec):
    """A brick whose nSymbols ends inside the level structure (truncated), and one whose nSymbols runs past its
    stream's bytes (the chain continues with no bytes to read): the sidecar's pieces reproduce the serial
    chain, flags included."""
    img = read_golden("shipped_subset")
    _, _, bricks = image_bricks(img)
    bad = patch_nsym(patch_nsym(img, 1, 2000), 2, bricks[2][2] * 2 + 7)
    ds = codec.open(bad)
    sc = ds.index_sidecar()
    ds2 = codec.open(bad, sidecar=sc)
    for t in (3, 6):
        a, sa = decode_all(codec, ds, t)
        c, sc2 = decode_all(codec, ds2, t)
        assert np.array_equal(sa, sc2) and np.array_equal(a, c), t
    assert sa[1] != 0
    ds.close()
    ds2.close()


def test_sidecar_mismatch_is_refused(codec, golden):
    from csvb200 import CsvError
    img = read_golden("shipped_subset")
    sc = codec.open(img).index_sidecar()
    rows, states = parse_sidecar(sc)
    starts = np.concatenate([[0], np.cumsum(rows[:, 2].astype(np.int64))]).astype(np.int64)

    def refused(bad: bytes):
        with pytest.raises(CsvError) as e:
            codec.open(img, sidecar=bad)
        assert e.value.code == -2  # CSV_EFORMAT

    # a stored state of a later piece (the piece before it ends elsewhere)
    s = states.copy()
    s[starts[6] + 3, 0] ^= 0x40
    refused(build_sidecar(rows, s))
    # its byte position only
    s = states.copy()
    s[starts[6] + 3, 1] -= 1
    refused(build_sidecar(rows, s))
    # a position past the stream's end (refused before any step reads there)
    s = states.copy()
    s[starts[4] + 2, 1] = rows[4, 0] + 100
    refused(build_sidecar(rows, s))
    # the first state, which must be the stream header
    s = states.copy()
    s[starts[2], 0] += 1
    refused(build_sidecar(rows, s))
    # header-level mismatches, found before the image is staged
    refused(sc[:-8])
    r = rows.copy()
    r[5, 1] += 1
    refused(build_sidecar(r, states))
    refused(codec.open(read_golden("tubes_64_b32")).index_sidecar())
    # a brick the sidecar gives no states for is indexed from its header: accepted, same decode
    r = rows.copy()
    r[3, 2] = 0
    keep = np.ones(states.shape[0], bool)
    keep[starts[3]:starts[4]] = False
    ds = codec.open(img, sidecar=build_sidecar(r, states[keep]))
    out, st = decode_all(codec, ds, 6)
    assert st.max() == 0
    assert [sha(out[k]) for k in range(out.shape[0])] == golden["shipped_subset"]["lod"]["6"]
    ds.close()


def test_repeated_opens_hold_steady_memory(codec):
    """The temporaries of csv_open (the image copy, the seek index's nibbles and snapshots) come from the
    context's pool, which keeps freed memory for the next open: after the first opens, more opens of the same
    image (with and without its sidecar) take no further device memory, and the index is the same each time."""
    import torch
    vol = torch.empty((128, 128, 192), dtype=torch.int64, device="cuda")
    codec.synth_volume(vol, 1, 400, 80, 1.0, 5.0, 0.1, 21)
    codec.encode_device(vol, 64)
    img = bytes(codec.encoded_image_tensor().cpu().numpy())
    del vol
    torch.cuda.synchronize()
    first = codec.open(img)
    sc = first.index_sidecar()
    ref, _ = decode_all(codec, first, 6)
    first.close()
    for s in (None, sc):  # warm the pool for both paths
        codec.open(img, sidecar=s).close()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k in range(12):
        ds = codec.open(img, sidecar=sc if k % 2 else None)
        if k in (5, 10):
            out, st = decode_all(codec, ds, 6)
            assert st.max() == 0 and np.array_equal(out, ref)
        ds.close()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < (64 << 20), (free0, free1)


@pytest.mark.parametrize("b", [32, 64])
def test_sidecar_of_a_version2_image(codec, b):
    """A version-2 image (each brick names its mode and one of several shared rANS tables): the seeded pieces
    of the bricks on tables other than the first read those tables from global memory.  The sidecar of the
    image opened from its bytes equals the encoder's dataset's, and opening with it decodes every LOD like
    csv_open."""
    import torch
    from csvb200.selector import fit_tables
    v = torch.empty((64, 128, 128), dtype=torch.int64, device="cuda")
    codec.synth_volume(v, 1, 120, 30, 1.5, 5.0, 0.2, 31 + b)
    nb = (64 // b) * (128 // b) * (128 // b)
    hist = torch.empty((nb, 12, 16), dtype=torch.int32, device="cuda")
    codec.encode_stats(v, b, hist)
    tables = fit_tables(hist.cpu().numpy().astype(np.uint64), 6, iters=4)
    rng = np.random.default_rng(b)
    choice = torch.from_numpy(rng.integers(0, 12, nb) | (rng.integers(0, len(tables), nb) << 4)).to(torch.uint8)
    codec.encode_device_sel(v, b, tables, choice.cuda())
    img = bytes(codec.encoded_image_tensor().cpu().numpy())
    del v
    assert struct.unpack_from("<I", img, 4)[0] == 2
    dse = codec.open_encoded()
    ds = codec.open(img)
    sc = ds.index_sidecar()
    assert dse.index_sidecar() == sc
    ds2 = codec.open(img, sidecar=sc)
    for t in range(b.bit_length()):
        a, sa = decode_all(codec, ds, t)
        c, sc2 = decode_all(codec, ds2, t)
        assert sa.max() == 0 and np.array_equal(sa, sc2) and np.array_equal(a, c), t
    for d in (dse, ds, ds2):
        d.close()
