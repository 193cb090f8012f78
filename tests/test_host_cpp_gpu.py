"""GPU: the C++ host API (host/csv_codec.hpp) over the C ABI, run as a real program.

host/example_encode_decode follows the reference's main.cpp flow (encode ->
save -> load -> decode all -> compare with the source) and exits non-zero on any
mismatch; its file must equal the oracle's encoding of the same volume.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu


def pattern(W, H, D):
    z, y, x = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    v = (1 + ((x // 7) ^ (y // 11) ^ (z // 5)) % 9).astype(np.uint64)
    v[((x // 16 + y // 16 + z // 16) % 5) == 0] = 0
    return v * np.uint64(0x9E3779B97F4A7C15)


@pytest.mark.parametrize("dims", [(100, 70, 90, 64), (64, 64, 64, 32), (40, 33, 17, 16)])
def test_example_program_roundtrip(tmp_path, oracle, dims, codec):
    exe = os.path.join(PKG, "host", "example_encode_decode")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", PKG, "host/example_encode_decode"], check=True)
    W, H, D, b = dims
    out = tmp_path / "x.csbd"
    r = subprocess.run([exe, str(W), str(H), str(D), str(b), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches=0" in r.stdout
    assert out.read_bytes() == oracle.encode(pattern(W, H, D), b)
