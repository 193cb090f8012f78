"""CPU: .npy ingest as the reference reads it, and a real-data round trip.

* csvb200.npy.load_npy follows loadNpy (fileIO.cpp:186-214) + splitGridIntoBricks (brick.hpp:133-195): the raw
  element buffer in file order, 4-byte elements widened, 8-byte ones copied, other sizes refused, the
  fortran_order flag and byte order ignored, shape[0] the x extent (fastest);
* real data: the shipped MICrONS .csbd (encoder/CSVEncoder/compressed_dataset.csbd, 512 bricks of 64^3)
  decodes to a 512^3 label volume; its re-encode by the oracle is the compiled reference encoder's image of
  that volume byte for byte and decodes back to it (runs where the reference tree is present).  The shipped
  file itself was written by an MSVC build: majority-vote ties follow its unordered_map, so no libstdc++
  build of the same source reproduces its bytes (the reference's own encoder compiled here does not either).
"""
import io
import os
import struct

import numpy as np
import pytest

from oracle import REF_SHIPPED as SHIPPED  # noqa: E402  (the reference tree; absent on GPU machines)


def _npy(arr, fortran=False):
    buf = io.BytesIO()
    np.save(buf, np.asfortranarray(arr) if fortran else arr)
    return buf.getvalue()


def _raw(buf, dtype, n):
    from csvb200.npy import read_npy_header
    _, off = read_npy_header(buf)
    return np.frombuffer(buf, dtype, n, off).astype(np.uint64)


@pytest.mark.parametrize("dtype,fortran", [(np.uint32, False), (np.uint64, False), (np.int32, False),
                                           (np.uint32, True), (np.dtype(">u4"), False), (np.int64, True)])
def test_load_npy_reads_the_buffer_as_the_reference(dtype, fortran):
    from csvb200.npy import load_npy_bytes
    rng = np.random.default_rng(1)
    shape = (6, 4, 5)  # shape[0] is x for the reference
    arr = rng.integers(0, 2 ** 31, shape).astype(dtype)
    buf = _npy(arr, fortran)
    vol = load_npy_bytes(buf)
    W, H, D = shape
    assert vol.shape == (D, H, W) and vol.dtype == np.uint64
    word = np.dtype(dtype).itemsize
    raw = _raw(buf, np.uint32 if word == 4 else np.uint64, W * H * D)  # file order, bits as stored
    for z, y, x in [(0, 0, 0), (1, 2, 3), (4, 3, 5), (2, 0, 1)]:
        assert vol[z, y, x] == raw[x + W * (y + H * z)]


def test_load_npy_refuses_what_the_reference_refuses():
    from csvb200.npy import load_npy_bytes
    with pytest.raises(ValueError, match="element size"):
        load_npy_bytes(_npy(np.zeros((2, 2, 2), np.uint16)))
    with pytest.raises(ValueError, match="3D"):
        load_npy_bytes(_npy(np.zeros((4, 4), np.uint64)))


def test_npy_to_image_equals_compiled_reference(oracle, reference, tmp_path):
    """A .npy on disk through load_npy and the oracle encoder, and through the compiled reference encoder fed
    the same interpretation: the same image."""
    from csvb200.npy import load_npy
    from csvb200.synth import tubes_over_voronoi
    vol = tubes_over_voronoi((40, 36, 48), 25, 8, 1.0, 3.0, 7, zero_frac=0.1) & np.uint64(0xFFFFFFFF)  # 4-byte labels
    p = tmp_path / "v.npy"
    W, H, D = vol.shape[2], vol.shape[1], vol.shape[0]
    # the reference reads shape (W, H, D) over the raw buffer with x fastest: save the volume's buffer
    # (x fastest) under that shape
    np.save(p, np.frombuffer(vol.astype(np.uint32).tobytes(), np.uint32).reshape(W, H, D))
    got = load_npy(str(p))
    assert np.array_equal(got, vol.astype(np.uint64))
    assert oracle.encode(got, 16) == reference.encode(got, 16)


def shipped_volume(oracle, img):
    """The label volume of a version-1 image whose bricks tile a box (brick IDs are the Morton codes of the
    brick coordinates, brick.hpp:160-164; decoded voxels are in Morton order, brickDecoding.hpp:174-242)."""
    nb, b = struct.unpack_from("<II", img, 8)
    labels, st = oracle.decode_image(img, b.bit_length() - 1)
    assert int(st.max()) == 0
    # brick IDs are Morton codes of the brick coordinates (brick.hpp:160-164)
    ids, o = [], 152
    for _ in range(nb):
        ID, P = struct.unpack_from("<II", img, o)
        ids.append(ID)
        o += 8 + 8 * P
        E = struct.unpack_from("<I", img, o)[0]
        o += 8 + E

    def unspread(v):
        r = 0
        for k in range(10):
            r |= ((v >> (3 * k)) & 1) << k
        return r

    coords = np.array([(unspread(i), unspread(i >> 1), unspread(i >> 2)) for i in ids])
    n = coords.max(0) + 1
    vol = np.zeros((n[2] * b, n[1] * b, n[0] * b), np.uint64)
    # decoded bricks are in Morton order of their voxels (brickDecoding.hpp:174-242)
    m = np.arange(b)
    sp = np.zeros(b, np.int64)
    for k in range(10):
        sp |= ((m >> k) & 1) << (3 * k)
    morton = (sp[None, None, :] | (sp[None, :, None] << 1) | (sp[:, None, None] << 2))  # [z, y, x]
    for i, (bx, by, bz) in enumerate(coords):
        vol[bz * b:(bz + 1) * b, by * b:(by + 1) * b, bx * b:(bx + 1) * b] = labels[i][morton]
    return vol, b


@pytest.mark.skipif(not os.path.exists(SHIPPED), reason="the reference tree is not on this machine")
def test_shipped_real_data_encode_equals_compiled_reference(oracle, reference):
    img = open(SHIPPED, "rb").read()
    vol, b = shipped_volume(oracle, img)
    assert vol.shape == (512, 512, 512)
    ours = oracle.encode(vol, b)
    assert ours == reference.encode(vol, b)
    back, st = oracle.decode_image(ours, b.bit_length() - 1)
    assert int(st.max()) == 0
    again, _ = shipped_volume(oracle, ours)
    assert np.array_equal(again, vol)
    # the same labels through two builds of one source: sizes within a few per cent
    assert abs(len(ours) - len(img)) < 0.05 * len(img)
