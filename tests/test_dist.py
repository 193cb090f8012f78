"""CPU, several processes: the multi-rank host logic on gloo (tests/dist_worker.py), world sizes 2 and 3.

* sharded encode: x-slabs of whole bricks per rank, one all-reduce of the model's sample histogram, records
  gathered in rank order behind one header -> byte-identical to the whole-volume encode (volumes with more than
  1024 bricks, so that the every-512th sample falls on several ranks; 3 ranks leave an uneven split);
* sharded decode: each rank decodes its contiguous range of bricks from a sub-image, equal to its slice of the
  whole decode, with no exchange;
* the bench's barrier and max-over-ranks timing helpers.
"""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_encode_and_decode_on_gloo_ranks(world):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                   WORLD_SIZE=str(world), LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "tests", "dist_worker.py")], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            p.kill()
            out, _ = p.communicate()
        outs.append(out)
    for rank, (p, out) in enumerate(zip(procs, outs)):
        assert p.returncode == 0, f"rank {rank} exited {p.returncode}:\n{out[-3000:]}"


def test_voxel_ranges_cover_and_balance():
    """The bench's multi-GPU split: contiguous request ranges that cover every request once, each rank's
    voxels within one request of an equal share."""
    import numpy as np
    from csvb200.dist import voxel_ranges
    rng = np.random.default_rng(5)
    for world in (1, 2, 3, 8):
        sizes = np.concatenate([np.full(1000, 32 ** 3), np.full(130, 64 ** 3)])[rng.permutation(1130)]
        r = voxel_ranges(sizes, world)
        assert r[0][0] == 0 and r[-1][1] == len(sizes)
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        share = sizes.sum() / world
        for lo, hi in r:
            assert abs(sizes[lo:hi].sum() - share) <= sizes.max()
