"""Several GPUs, one process each: the volume split into x-slabs of whole bricks.

The reference is single-process (main.cpp:67-84, a single-threaded encoder;
the viewer decodes one file).  Bricks are independent, so decode needs no
exchange at all: each rank opens its own range of a file's bricks
(`sub_image`) and decodes them.  The encoder has exactly one exchange step:
the rANS model is built from the nibble histogram of the bricks whose file
index is a multiple of 512 (brickEncoding.hpp:481-482), which live on
whichever ranks own them.  `encode_sharded` runs that protocol over a
torch.distributed process group (NCCL on GPUs, gloo on the host):

  1. every rank encodes the bricks of its slab (K1) and returns the sample
     histogram of those it owns (csv_encode_shard_bricks);
  2. all-reduce (sum) of the 16 counts;
  3. every rank builds the same model and finishes its records
     (csv_encode_shard_finish);
  4. the record bytes are gathered to rank 0 in rank order, behind one header
     whose numBricks is the total.

The split order puts the x-brick outermost (brick.hpp:152-154), so a slab of
whole x-bricks is a contiguous range of file indices and the concatenation in
rank order is the file order: the result is byte-identical to encoding the
whole volume on one GPU.
"""
from __future__ import annotations

import struct

import numpy as np

HEADER_V1 = 152  # fileIO.cpp:25-49


def slab_ranges(W: int, brick: int, world: int):
    """x-brick ranges [bx0, bx1) per rank, as even as whole bricks allow (the last ranks may be empty)."""
    nbx = -(-W // brick)
    per, extra = divmod(nbx, world)
    out, b0 = [], 0
    for r in range(world):
        n = per + (1 if r < extra else 0)
        out.append((b0, b0 + n))
        b0 += n
    return out


def slab_of(volume, brick: int, bx0: int, bx1: int):
    """The x-slab [bx0*brick, min(bx1*brick, W)) of a (D, H, W) volume, contiguous (numpy or torch)."""
    W = volume.shape[2]
    x0, x1 = bx0 * brick, min(bx1 * brick, W)
    s = volume[:, :, x0:x1]
    return s.contiguous() if hasattr(s, "contiguous") else np.ascontiguousarray(s)


class DeviceShardEncoder:
    """The device encoder as the protocol's backend (csv_encode_shard_bricks / csv_encode_shard_finish)."""

    def __init__(self, codec):
        self.codec = codec

    def bricks(self, slab, brick: int, bx0: int, index_base: int) -> np.ndarray:
        return self.codec.encode_shard_bricks(slab, brick, bx0, index_base)

    def finish(self, hist) -> bytes:
        self.codec.encode_shard_finish(hist)
        return bytes(self.codec.encoded_image_tensor().cpu().numpy())


def _all_gather_bytes(pg, data: bytes, device):
    """Every rank's bytes on every rank (two collectives: lengths, then the padded payloads)."""
    import torch
    world = pg.get_world_size()
    n = torch.tensor([len(data)], dtype=torch.int64, device=device)
    sizes = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    pg.all_gather(sizes, n)
    sizes = [int(s.item()) for s in sizes]
    cap = max(max(sizes), 1)
    buf = torch.zeros(cap, dtype=torch.uint8, device=device)
    if data:
        buf[:len(data)] = torch.frombuffer(bytearray(data), dtype=torch.uint8).to(device)
    parts = [torch.zeros(cap, dtype=torch.uint8, device=device) for _ in range(world)]
    pg.all_gather(parts, buf)
    return [bytes(p[:s].cpu().numpy()) for p, s in zip(parts, sizes)]


def encode_sharded(encoder, slab, brick: int, bx0: int, n_yz_bricks: int, pg, device="cpu"):
    """One rank's part of a sharded encode (see the module docstring).  slab: this rank's (D, H, w) x-slab
    starting at x-brick bx0; n_yz_bricks: bricks per x-brick column of the whole volume (nby * nbz).
    Returns the whole .csbd image on rank 0 and None on the others.  Every rank takes the same collective
    steps in the same order, an empty slab included."""
    import torch
    index_base = bx0 * n_yz_bricks
    empty = slab.shape[2] == 0
    hist = np.zeros(16, np.uint64) if empty else encoder.bricks(slab, brick, bx0, index_base)
    h = torch.from_numpy(hist.astype(np.int64)).to(device)
    pg.all_reduce(h, op=pg.ReduceOp.SUM)
    total = h.cpu().numpy().astype(np.uint64)
    image = b"" if empty else encoder.finish(total)
    parts = _all_gather_bytes(pg, image, device)
    return assemble(parts) if pg.get_rank() == 0 else None


def assemble(parts):
    """The whole image from the slabs' images in rank order (empty ones skipped): one header with the total
    numBricks, then every slab's records."""
    parts = [p for p in parts if p]
    headers = [p[:HEADER_V1] for p in parts]
    if any(hd[12:] != headers[0][12:] for hd in headers):
        raise ValueError("the slabs were encoded with different models")
    head = bytearray(headers[0])
    struct.pack_into("<I", head, 8, sum(struct.unpack_from("<I", p, 8)[0] for p in parts))
    return bytes(head) + b"".join(p[HEADER_V1:] for p in parts)


def brick_ranges(nb: int, world: int):
    """Contiguous file-index ranges [lo, hi) per rank for decoding (independent bricks, no exchange)."""
    per, extra = divmod(nb, world)
    out, lo = [], 0
    for r in range(world):
        n = per + (1 if r < extra else 0)
        out.append((lo, lo + n))
        lo += n
    return out


def voxel_ranges(sizes, world: int):
    """Contiguous request ranges [lo, hi) per rank with about equal output voxels (sizes: voxels per request,
    in order).  Bricks are independent, so each rank decodes its range with no exchange."""
    import numpy as np
    c = np.concatenate([[0], np.cumsum(np.asarray(sizes, np.float64))])
    cuts = [0] + [int(np.searchsorted(c, c[-1] * r / world)) for r in range(1, world)] + [len(c) - 1]
    return [(cuts[r], max(cuts[r], cuts[r + 1])) for r in range(world)]


def sub_image(image: bytes, lo: int, hi: int) -> bytes:
    """A version-1 .csbd image holding bricks [lo, hi) of `image` (same header and model; numBricks = hi - lo).
    Record layout: ID, P, palette[P], E, stream[E], nSymbols (fileIO.cpp:57-96)."""
    magic, ver, nb = struct.unpack_from("<III", image, 0)
    if ver != 1:
        raise ValueError("sub_image reads version-1 images")
    if not 0 <= lo <= hi <= nb:
        raise ValueError("brick range outside the image")
    o, start, end = HEADER_V1, None, None
    for i in range(nb + 1):
        if i == lo:
            start = o
        if i == hi:
            end = o
            break
        P = struct.unpack_from("<I", image, o + 4)[0]
        o += 8 + 8 * P
        E = struct.unpack_from("<I", image, o)[0]
        o += 8 + E
    head = bytearray(image[:HEADER_V1])
    struct.pack_into("<I", head, 8, hi - lo)
    return bytes(head) + image[start:end]
