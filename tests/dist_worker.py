"""One rank of the multi-process tests (tests/test_dist.py starts WORLD_SIZE of these with the rendezvous in the
environment).  The codec work runs on the oracle (CPU) behind the same two-step shard interface the device encoder
has, so that the host protocol of csvb200.dist -- the collectives, their order, the file assembly, the decode
split -- runs on gloo ranks without a GPU.  Exits 0 when every check holds."""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "fast-compressed-segmentation_b200"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402


class OracleShardEncoder:
    """or_encode_shard behind the interface of csvb200.dist.DeviceShardEncoder (the oracle is stateless: the
    second step encodes the slab again with the summed histogram)."""

    def __init__(self, oracle):
        self.o = oracle

    def bricks(self, slab, brick, bx0, index_base):
        self.args = (slab, brick, bx0, index_base)
        return self.o.encode_shard(slab, brick, bx0, index_base)[1]

    def finish(self, hist):
        return self.o.encode_shard(*self.args, hist_in=hist)[0]


def main():
    from oracle import Oracle
    from csvb200.dist import brick_ranges, encode_sharded, slab_ranges, slab_of, sub_image
    from csvb200.synth import tubes_over_voronoi
    import bench

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rank, world = dist.get_rank(), dist.get_world_size()
    o = Oracle()
    bad = 0
    # more than 1024 bricks, so that the every-512th model sample falls on several ranks
    for shape, b in [((32, 32, 96), 4), ((16, 24, 72), 2), ((20, 30, 44), 4)]:
        vol = tubes_over_voronoi(shape, 30, 6, 1.0, 3.0, 11 + b, zero_frac=0.1)
        D, H, W = vol.shape
        nby, nbz = -(-H // b), -(-D // b)
        bx0, bx1 = slab_ranges(W, b, world)[rank]
        slab = slab_of(vol, b, bx0, bx1)
        image = encode_sharded(OracleShardEncoder(o), slab, b, bx0, nby * nbz, dist, device="cpu")
        whole = o.encode(vol, b)
        if rank == 0 and image != whole:
            bad += 1
            print(f"rank 0: sharded image of {shape} b{b} differs from the whole-volume encode", flush=True)
        # decode: each rank its own contiguous range of bricks, no exchange
        nb = int(np.frombuffer(whole[8:12], np.uint32)[0])
        lo, hi = brick_ranges(nb, world)[rank]
        for lod in (0, b.bit_length() - 1):
            ref = o.decode_image(whole, lod)[0]
            if hi > lo:
                got, st = o.decode_image(sub_image(whole, lo, hi), lod)
                if not np.array_equal(got, ref[lo:hi]) or int(st.max()) != 0:
                    bad += 1
                    print(f"rank {rank}: bricks [{lo}, {hi}) at LOD {lod} differ", flush=True)
    # the bench's timing helpers: barrier, then the maximum over ranks
    bench.barrier(dist)
    if bench.max_over_ranks(float(rank + 1), dist, "cpu") != float(world):
        bad += 1
    t = torch.tensor([bad], dtype=torch.int64)
    dist.all_reduce(t)
    dist.destroy_process_group()
    sys.exit(0 if int(t.item()) == 0 else 1)


if __name__ == "__main__":
    main()
