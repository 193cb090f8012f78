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


def test_selector_file_round_trip_and_refusals(tmp_path):
    """Selector files (csv_selector_write / csv_selector_read) are host-only: tables and parameters come back
    bit for bit; a flipped byte, a truncated file, tables that do not sum to 4096 and a missing file are
    refused with their codes."""
    import numpy as np
    from csvb200 import MLP_PARAMS, CsvError, load_library, read_selector, write_selector
    lib = load_library()
    rng = np.random.default_rng(3)
    params = rng.standard_normal(MLP_PARAMS).astype(np.float32)
    tables = np.full((5, 16), 256, np.uint32)
    tables[:, 0] += np.arange(5, dtype=np.uint32)
    tables[:, 1] -= np.arange(5, dtype=np.uint32)
    path = str(tmp_path / "sel.csvs")
    write_selector(lib, path, params, tables)
    p2, t2 = read_selector(lib, path)
    assert np.array_equal(p2.view(np.uint32), params.view(np.uint32)) and np.array_equal(t2, tables)
    raw = bytearray(open(path, "rb").read())
    assert len(raw) == 16 + 64 * 5 + 4 * MLP_PARAMS + 4
    for bad, code in [(raw[:-7], -2), (raw[:100] + bytes([raw[100] ^ 1]) + raw[101:], -2)]:
        open(path, "wb").write(bytes(bad))
        try:
            read_selector(lib, path)
        except CsvError as e:
            assert e.code == code
        else:
            raise AssertionError("a damaged selector file was read")
    bad_tables = tables.copy()
    bad_tables[2, 3] += 1
    for args, code in [((str(tmp_path / "x"), params, bad_tables), -1)]:
        try:
            write_selector(lib, *args)
        except CsvError as e:
            assert e.code == code
        else:
            raise AssertionError("tables that do not sum to 4096 were written")
    try:
        read_selector(lib, str(tmp_path / "absent.csvs"))
    except CsvError as e:
        assert e.code == -7
    else:
        raise AssertionError("a missing file was read")
