import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fast-compressed-segmentation_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU and the built native library")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference sources compiled in this container (absent on machines without the reference tree)."""
    from oracle import REF_SO, Reference
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libcsvref.so not built (needs the reference tree)")
    return Reference()


@pytest.fixture(scope="session")
def golden():
    import json
    return json.load(open(os.path.join(GOLDEN, "golden.json")))


def read_golden(name: str) -> bytes:
    return open(os.path.join(GOLDEN, name + ".csbd"), "rb").read()


@pytest.fixture(scope="session")
def codec():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from csvb200 import Codec
    return Codec(0)
