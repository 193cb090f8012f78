""".npy ingest as the reference encoder reads it (loadNpy, encoder/CSVEncoder/src/fileIO.cpp:186-214, and
splitGridIntoBricks, brick.hpp:133-195).

The reference takes the file's raw element buffer in file order and
  * widens 4-byte elements to uint64 (zero extension) and copies 8-byte ones; any other element size is an
    error (fileIO.cpp:195-212) -- the dtype's kind and byte order are not looked at;
  * ignores the header's fortran_order flag;
  * reads shape[0] as the width (x, fastest), shape[1] as the height, shape[2] as the depth (brick.hpp:139-141),
    i.e. element i is voxel (i % W, (i / W) % H, i / (W * H)).
`load_npy` returns that volume as this package's (D, H, W) uint64 array (x fastest, the layout every encoder
entry point takes), so that csv_encode of it is the reference's encode of the file.
"""
from __future__ import annotations

import ast
import struct

import numpy as np


def read_npy_header(buf: bytes):
    """(header dict, offset of the data) of a .npy file (format versions 1.0, 2.0 and 3.0)."""
    if buf[:6] != b"\x93NUMPY":
        raise ValueError("not a .npy file")
    major = buf[6]
    if major == 1:
        hlen, off = struct.unpack_from("<H", buf, 8)[0], 10
    elif major in (2, 3):
        hlen, off = struct.unpack_from("<I", buf, 8)[0], 12
    else:
        raise ValueError(f"unsupported .npy version {major}")
    header = ast.literal_eval(buf[off:off + hlen].decode("latin1"))
    return header, off + hlen


def load_npy_bytes(buf: bytes) -> np.ndarray:
    header, off = read_npy_header(buf)
    shape = tuple(int(s) for s in header["shape"])
    if len(shape) != 3:
        raise ValueError("Expected a 3D array")  # brick.hpp:136-137
    word = np.dtype(header["descr"]).itemsize
    total = shape[0] * shape[1] * shape[2]
    if word == 4:
        data = np.frombuffer(buf, np.uint32, total, off).astype(np.uint64)
    elif word == 8:
        data = np.frombuffer(buf, np.uint64, total, off).copy()
    else:
        raise ValueError(f"Unsupported .npy element size: {word}")
    W, H, D = shape
    return data.reshape(D, H, W)


def load_npy(path: str) -> np.ndarray:
    """The volume of a .npy file as the reference encoder sees it, shape (D, H, W), uint64."""
    with open(path, "rb") as f:
        return load_npy_bytes(f.read())
