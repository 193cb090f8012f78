"""CPU: the native library builds for sm_100a, loads, and exports every entry point include/csv.h declares."""
import ctypes
import os
import re

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "csv.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(csv_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for f in ["csv_create", "csv_destroy", "csv_last_error", "csv_encode", "csv_encode_device", "csv_open",
              "csv_decode_batch", "csv_decode_image", "csv_close"]:
        assert f in names


def test_library_exports_every_declared_symbol():
    from csvb200 import load_library
    lib = load_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.csv_abi_version() == 1


def test_build_targets_sm100a():
    mk = open(os.path.join(ROOT, "fast-compressed-segmentation_b200", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_no_cpu_fallback_without_gpu():
    """Without a usable device the context cannot be created; nothing falls back to the CPU."""
    import torch
    if torch.cuda.is_available():
        return
    from csvb200 import Codec, CsvError
    try:
        Codec(0)
    except CsvError as e:
        assert e.code == -3
    else:
        raise AssertionError("context created without a GPU")
