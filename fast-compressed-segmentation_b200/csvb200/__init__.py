"""Python host binding of the B200 compressed-segmentation-volume codec.

A ctypes layer over the C ABI in include/csv.h (libcsvb200.so, built for
sm_100a).  It mirrors the reference's entry points for this path:

  reference (paths relative to the reference root)      here
  ---------------------------------------------------   ------------------------------
  splitGridIntoBricks + compressDataset +                Codec.encode / encode_device
    saveDatasetToFile (brick.hpp:134,
    brickEncoding.hpp:467, fileIO.cpp:15)
  loadDatasetFromFile (fileIO.cpp:101),                  Codec.open
    loadDatasetFromArrayBuffer (datasetLoader.js:39)
  decodeRansStream + decodeBrick<b>                      Codec.decode_batch / decode_image
    (brickDecoding.cpp:153, brickDecoding.hpp:175),
    decode.wgsl:decodeBrick (:344)

Errors raise ``CsvError`` where the reference throws std::runtime_error.
Device buffers are torch tensors (torch is used only for device memory and
streams).  There is no CPU fallback: a missing library or GPU raises.
"""
from __future__ import annotations

import ctypes as C
import ctypes as C_MOD
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcsvb200.so")

CSV_BRICK_TRUNCATED = 0x1
CSV_BRICK_PALETTE = 0x2
CSV_BRICK_BADOP = 0x4
CSV_BRICK_BADREQ = 0x8
CSV_BRICK_TIMEOUT = 0x10

ERRORS = {-1: "EINVAL", -2: "EFORMAT", -3: "ECUDA", -4: "ENOMEM", -5: "ERANGE", -6: "EBRICK"}

# csv_request: {uint32 brick, uint32 lod, uint64 dst}
REQUEST_DTYPE = np.dtype([("brick", "<u4"), ("lod", "<u4"), ("dst", "<u8")])


class CsvError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Info(C.Structure):
    _fields_ = [("num_bricks", C.c_uint32), ("brick_size", C.c_uint32), ("levels", C.c_uint32),
                ("ops_per_checkpoint", C.c_uint32), ("stream_bytes", C.c_uint64),
                ("palette_entries", C.c_uint64), ("freq", C.c_uint32 * 16), ("cum", C.c_uint32 * 16)]


class DecodeConfig(C.Structure):
    """csv_decode_config: grid CTAs per SM (0 = all that fit), stream staging, largest-first order, and for
    datasets with 64^3 bricks the kernel layout (0: split by output size over two kernels, 1: one kernel)."""
    _fields_ = [("ctas_per_sm", C.c_uint32), ("stage", C.c_uint32), ("lpt", C.c_uint32), ("layout", C.c_uint32)]

    def as_dict(self):
        return {"ctas_per_sm": self.ctas_per_sm, "stage": self.stage, "lpt": self.lpt, "layout": self.layout}


CONE_REFERENCE = 0
CONE_SCREEN = 1
ADMIT_CONE = 0  # csv_serve_config.admit: the cone and LOD plan (the reference as it runs)
ADMIT_RAYS = 1  # only the bricks the session's last render entered (the reference's useGPUCulling path)


class ServeConfig(C.Structure):
    """csv_serve_config."""
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("max_sessions", C.c_uint32), ("cone", C.c_uint32),
                ("fov", C.c_double), ("cache_bytes", C.c_uint64), ("admit", C.c_uint32), ("reserved", C.c_uint32)]


class View(C.Structure):
    """csv_view: camera position and view direction (double)."""
    _fields_ = [("position", C.c_double * 3), ("direction", C.c_double * 3)]


class FrameStats(C.Structure):
    """csv_frame_stats."""
    _fields_ = [("step", C.c_uint64), ("session", C.c_uint32), ("planned", C.c_uint32), ("visible", C.c_uint32),
                ("decoded", C.c_uint32), ("freed", C.c_uint32), ("resident", C.c_uint32), ("rebuilt", C.c_uint32),
                ("entered", C.c_uint32), ("missing", C.c_uint32), ("reserved", C.c_uint32),
                ("decoded_voxels", C.c_uint64), ("ms", C.c_float), ("reserved2", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class ServeInfo(C.Structure):
    """csv_serve_info."""
    _fields_ = [("slots", C.c_void_p), ("n_slots", C.c_uint64), ("cache", C.c_void_p), ("cache_labels", C.c_uint64),
                ("palette_table", C.c_uint64), ("bricks_per_axis", C.c_uint32), ("brick_size", C.c_uint32),
                ("grid_size", C.c_float), ("pad", C.c_uint32), ("focal", C.c_double), ("cos_half", C.c_double),
                ("decode_status", C.c_void_p)]


_lib = None


def library_path() -> str:
    return LIB_PATH


def load_library() -> C.CDLL:
    """Load libcsvb200.so; raises if it was not built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} missing: build it with `make -C fast-compressed-segmentation_b200`")
    L = C.CDLL(LIB_PATH)
    vp, u8p, u32p, u64p = C.c_void_p, C.POINTER(C.c_uint8), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
    L.csv_abi_version.restype = C.c_int
    L.csv_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.csv_destroy.argtypes = [vp]
    L.csv_last_error.restype = C.c_char_p
    L.csv_last_error.argtypes = [vp]
    L.csv_free.argtypes = [vp]
    L.csv_encode.argtypes = [vp, u64p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(u8p),
                             C.POINTER(C.c_size_t)]
    L.csv_encode_device.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp,
                                    C.POINTER(C.c_size_t)]
    L.csv_encoded_image.argtypes = [vp, C.POINTER(vp), C.POINTER(C.c_size_t)]
    L.csv_encode_shard_bricks.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.c_uint32, u64p, vp]
    L.csv_encode_shard_finish.argtypes = [vp, u64p, vp, C.POINTER(C.c_size_t)]
    L.csv_open.argtypes = [vp, u8p, C.c_size_t, C.POINTER(vp)]
    L.csv_open_encoded.argtypes = [vp, C.POINTER(vp)]
    L.csv_dataset_info_get.argtypes = [vp, C.POINTER(_Info)]
    L.csv_dataset_ids.argtypes = [vp, u32p, C.c_uint32]
    L.csv_dataset_index_ms.argtypes = [vp, C.POINTER(C.c_float)]
    L.csv_index_save.argtypes = [vp, vp, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t)]
    L.csv_open_indexed.argtypes = [vp, u8p, C.c_size_t, u8p, C.c_size_t, C.POINTER(vp)]
    L.csv_close.argtypes = [vp]
    L.csv_decode_batch.argtypes = [vp, vp, vp, C.c_uint32, vp, vp, vp]
    L.csv_decode_image.argtypes = [vp, u8p, C.c_size_t, C.c_uint32, u64p, u32p]
    L.csv_decode_batch_static.argtypes = [vp, vp, vp, C.c_uint32, vp, vp, vp]
    L.csv_dataset_concat.argtypes = [vp, C.POINTER(vp), C.c_uint32, C.POINTER(vp)]
    L.csv_decode_graph_create.argtypes = [vp, vp, vp, C.c_uint32, vp, vp, C.POINTER(DecodeConfig), C.POINTER(vp)]
    L.csv_graph_launch.argtypes = [vp, vp]
    L.csv_graph_kernels.argtypes = [vp, C.POINTER(C.c_uint32)]
    L.csv_graph_destroy.argtypes = [vp]
    L.csv_decode_autotune.argtypes = [vp, vp, vp, C.c_uint32, vp, vp, C.c_uint32, C.POINTER(DecodeConfig),
                                      C.POINTER(C.c_float)]
    L.csv_render.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, C.c_uint32, vp, C.c_uint64, vp,
                             vp, C.c_uint32, vp, vp, vp, vp]
    L.csv_lighting_default.argtypes = [C.c_double, C.POINTER(Lighting)]
    L.csv_transfer_function.argtypes = [vp, u64p, C.c_uint32, u64p, u32p, C.c_uint32, C.POINTER(C.c_uint32)]
    L.csv_render_rgba.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, C.c_uint32, vp, C.c_uint64,
                                  vp, vp, vp, C.c_uint32, C.POINTER(Lighting), vp, vp, vp]
    L.csv_synth_volume.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_uint32, C.c_uint32,
                                   C.c_float, C.c_float, C.c_float, C.c_uint64, vp]
    L.csv_serve_create.argtypes = [vp, vp, C.POINTER(ServeConfig), u64p, C.c_uint32, C.POINTER(vp)]
    L.csv_serve_submit.argtypes = [vp, C.c_uint32, C.POINTER(View), vp, vp]
    L.csv_serve_submit_rgba.argtypes = [vp, C.c_uint32, C.POINTER(View), vp]
    L.csv_serve_set_lighting.argtypes = [vp, C.POINTER(Lighting)]
    L.csv_serve_step.argtypes = [vp, vp, C.POINTER(C.c_uint64)]
    L.csv_serve_poll.argtypes = [vp, C.POINTER(FrameStats), C.c_uint32, C.POINTER(C.c_uint32), C.c_int]
    L.csv_serve_camera.argtypes = [vp, C.POINTER(View), vp]
    L.csv_serve_state.argtypes = [vp, C.c_uint32, C.POINTER(ServeInfo)]
    L.csv_serve_close.argtypes = [vp, C.c_uint32]
    L.csv_serve_compact.argtypes = [vp, vp]
    L.csv_serve_destroy.argtypes = [vp]
    L.csv_gemm_bf16.argtypes = [vp, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, C.c_uint32, vp, vp, vp, vp,
                                vp, vp]
    L.csv_encode_stats.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp]
    L.csv_select_exhaustive.argtypes = [vp, vp, C.c_uint32, u32p, C.c_uint32, vp, vp, vp]
    L.csv_encode_device_sel.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.c_uint32,
                                        vp, vp, C.POINTER(C.c_size_t)]
    L.csv_brick_features.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp]
    L.csv_mlp_create.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(vp)]
    L.csv_selector_write.argtypes = [C.c_char_p, C.POINTER(C.c_float), u32p, C.c_uint32]
    L.csv_selector_read.argtypes = [C.c_char_p, C.POINTER(C.c_float), u32p, u32p]
    L.csv_encode_learned.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp, u32p, C.c_uint32,
                                     vp, C.POINTER(C.c_size_t)]
    L.csv_mlp_destroy.argtypes = [vp]
    L.csv_mlp_destroy.restype = None
    L.csv_mlp_params.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.csv_mlp_forward.argtypes = [vp, vp, C.c_uint32, vp, vp, vp]
    L.csv_mlp_grad.argtypes = [vp, vp, vp, C.c_uint32, C.POINTER(C.c_float), vp]
    L.csv_mlp_adam.argtypes = [vp, C.c_float, C.c_float, C.c_float, C.c_float, vp]
    L.csv_mlp_status.argtypes = [vp]
    _lib = L
    return L


def _vp(t):
    """Device pointer of a tensor (or NULL for None) as a ctypes void pointer."""
    return C.c_void_p(t.data_ptr() if t is not None else None)


def _stream_handle(stream) -> int | None:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


class Lighting(C.Structure):
    """csv_lighting: direction towards the light (unnormalised), ambient and diffuse strengths."""
    _fields_ = [("light_dir", C.c_float * 3), ("ambient", C.c_float), ("diffuse", C.c_float), ("pad", C.c_float * 3)]

    def as_array(self):
        return np.array(list(self.light_dir) + [self.ambient, self.diffuse], np.float32)


@dataclass
class DatasetInfo:
    num_bricks: int
    brick_size: int
    levels: int
    ops_per_checkpoint: int
    stream_bytes: int
    palette_entries: int
    freq: tuple
    cum: tuple


class Dataset:
    """A .csbd image staged in HBM with its seek index (csv_open)."""

    def __init__(self, codec: "Codec", handle: int):
        self.codec = codec
        self.handle = C.c_void_p(handle)
        info = _Info()
        codec.lib.csv_dataset_info_get(self.handle, C.byref(info))
        self.info = DatasetInfo(info.num_bricks, info.brick_size, info.levels, info.ops_per_checkpoint,
                                info.stream_bytes, info.palette_entries, tuple(info.freq), tuple(info.cum))

    @property
    def num_bricks(self) -> int:
        return self.info.num_bricks

    @property
    def brick_size(self) -> int:
        return self.info.brick_size

    @property
    def index_ms(self) -> float:
        """Device time of the seek-index passes csv_open ran (0.0 when none ran)."""
        ms = C.c_float()
        self.codec._check(self.codec.lib.csv_dataset_index_ms(self.handle, C.byref(ms)))
        return ms.value

    def index_sidecar(self) -> bytes:
        """csv_index_save: the seek-index sidecar of this dataset's image (give it to Codec.open)."""
        out = C.POINTER(C.c_uint8)()
        n = C.c_size_t()
        self.codec._check(self.codec.lib.csv_index_save(self.codec.handle, self.handle, C.byref(out), C.byref(n)))
        data = C.string_at(out, n.value)
        self.codec.lib.csv_free(out)
        return data

    def ids(self) -> np.ndarray:
        out = np.zeros(max(1, self.num_bricks), np.uint32)
        self.codec._check(self.codec.lib.csv_dataset_ids(self.handle, out.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                          len(out)))
        return out[: self.num_bricks]

    def close(self):
        if self.handle:
            self.codec.lib.csv_close(self.handle)
            self.handle = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DecodeGraph:
    """A captured decode (csv_decode_graph_create); keeps its buffers alive."""

    def __init__(self, codec: "Codec", handle: int, keep):
        self.codec, self.handle, self._keep = codec, C.c_void_p(handle), keep

    def launch(self, stream=None):
        self.codec._check(self.codec.lib.csv_graph_launch(self.handle, C.c_void_p(_stream_handle(stream))))

    @property
    def kernels(self) -> int:
        """Decode kernels one replay launches (csv_graph_kernels)."""
        n = C.c_uint32()
        self.codec._check(self.codec.lib.csv_graph_kernels(self.handle, C.byref(n)))
        return n.value

    def close(self):
        if self.handle:
            self.codec.lib.csv_graph_destroy(self.handle)
            self.handle = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Codec:
    """One context on one CUDA device (csv_create)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.csv_create(device, C.byref(h))
        if rc:
            raise CsvError(rc, f"csv_create(device={device}) failed (no usable CUDA device?)")
        self.handle = h
        self.device = device

    def _check(self, rc: int):
        if rc:
            raise CsvError(rc, self.lib.csv_last_error(self.handle).decode())

    def close(self):
        if getattr(self, "handle", None):
            self.lib.csv_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- encoder -------------------------------------------------------
    def encode(self, volume: np.ndarray, brick_size: int = 64) -> bytes:
        """Host volume (D, H, W) uint64, x fastest -> .csbd v1 bytes."""
        v = np.ascontiguousarray(volume, dtype=np.uint64)
        D, H, W = v.shape
        out = C.POINTER(C.c_uint8)()
        n = C.c_size_t()
        self._check(self.lib.csv_encode(self.handle, v.ctypes.data_as(C.POINTER(C.c_uint64)), W, H, D, brick_size,
                                        C.byref(out), C.byref(n)))
        data = C.string_at(out, n.value)
        self.lib.csv_free(out)
        return data

    def encode_device(self, d_volume, brick_size: int = 64, stream=None) -> int:
        """Device volume (torch uint64/int64 tensor, shape (D, H, W)) -> image length; the image stays on the
        device (see encoded_image)."""
        D, H, W = d_volume.shape
        n = C.c_size_t()
        self._check(self.lib.csv_encode_device(self.handle, C.c_void_p(d_volume.data_ptr()), W, H, D, brick_size,
                                               C.c_void_p(_stream_handle(stream)), C.byref(n)))
        return n.value

    def encode_shard_bricks(self, d_slab, brick_size: int, bx0: int, index_base: int, stream=None) -> np.ndarray:
        """First step of a sharded encode (csv_encode_shard_bricks): the slab's bricks; returns the 16-bin histogram
        (uint64) of its bricks whose file index is a multiple of 512."""
        D, H, W = d_slab.shape
        hist = np.zeros(16, np.uint64)
        self._check(self.lib.csv_encode_shard_bricks(self.handle, C.c_void_p(d_slab.data_ptr()), W, H, D, brick_size,
                                                     bx0, index_base, hist.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                     C.c_void_p(_stream_handle(stream))))
        return hist

    def encode_shard_finish(self, hist, stream=None) -> int:
        """Second step (csv_encode_shard_finish): the model from the histogram summed over all shards, then this
        shard's image (header + its records); returns the image length."""
        h = np.ascontiguousarray(hist, np.uint64)
        n = C.c_size_t()
        self._check(self.lib.csv_encode_shard_finish(self.handle, h.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                     C.c_void_p(_stream_handle(stream)), C.byref(n)))
        return n.value

    def encoded_image(self):
        ptr = C.c_void_p()
        n = C.c_size_t()
        self._check(self.lib.csv_encoded_image(self.handle, C.byref(ptr), C.byref(n)))
        return ptr.value, n.value

    def encoded_image_tensor(self):
        """Zero-copy torch view (uint8, on the device) of the image the last encode_device produced; valid
        until the next encode on this context."""
        import torch
        ptr, n = self.encoded_image()

        class _View:
            __cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 2}

        return torch.as_tensor(_View(), device=f"cuda:{self.device}")

    # ---- datasets ------------------------------------------------------
    def open(self, image: bytes, sidecar: bytes | None = None) -> Dataset:
        """csv_open, or csv_open_indexed with a seek-index sidecar (Dataset.index_sidecar of the same image)."""
        a = np.frombuffer(image, np.uint8)
        h = C.c_void_p()
        if sidecar is None:
            self._check(self.lib.csv_open(self.handle, a.ctypes.data_as(C.POINTER(C.c_uint8)), len(image),
                                          C.byref(h)))
        else:
            sc = np.frombuffer(sidecar, np.uint8)
            self._check(self.lib.csv_open_indexed(self.handle, a.ctypes.data_as(C.POINTER(C.c_uint8)), len(image),
                                                  sc.ctypes.data_as(C.POINTER(C.c_uint8)), len(sidecar),
                                                  C.byref(h)))
        return Dataset(self, h.value)

    def concat(self, parts) -> Dataset:
        """csv_dataset_concat: one dataset with the bricks of every part (each keeps its brick size and model)."""
        arr = (C.c_void_p * len(parts))(*[p.handle.value for p in parts])
        h = C.c_void_p()
        self._check(self.lib.csv_dataset_concat(self.handle, arr, len(parts), C.byref(h)))
        return Dataset(self, h.value)

    def decode_graph(self, ds: Dataset, d_reqs, d_out, d_status, cfg: DecodeConfig | None = None,
                     n: int | None = None) -> "DecodeGraph":
        if n is None:
            n = d_reqs.numel() * d_reqs.element_size() // 16
        g = C.c_void_p()
        self._check(self.lib.csv_decode_graph_create(self.handle, ds.handle, C.c_void_p(d_reqs.data_ptr()), n,
                                                      C.c_void_p(d_out.data_ptr()), C.c_void_p(d_status.data_ptr()),
                                                      C.byref(cfg) if cfg is not None else None, C.byref(g)))
        return DecodeGraph(self, g.value, (ds, d_reqs, d_out, d_status))

    def autotune(self, ds: Dataset, d_reqs, d_out, d_status, reps: int = 5, n: int | None = None):
        """csv_decode_autotune -> (DecodeConfig, median ms)."""
        if n is None:
            n = d_reqs.numel() * d_reqs.element_size() // 16
        best = DecodeConfig()
        ms = C.c_float()
        self._check(self.lib.csv_decode_autotune(self.handle, ds.handle, C.c_void_p(d_reqs.data_ptr()), n,
                                                  C.c_void_p(d_out.data_ptr()), C.c_void_p(d_status.data_ptr()), reps,
                                                  C.byref(best), C.byref(ms)))
        return best, ms.value

    def open_encoded(self) -> Dataset:
        h = C.c_void_p()
        self._check(self.lib.csv_open_encoded(self.handle, C.byref(h)))
        return Dataset(self, h.value)

    # ---- decoder -------------------------------------------------------
    def decode_batch(self, ds: Dataset, d_reqs, d_out, d_status, stream=None, n: int | None = None):
        """d_reqs: device tensor holding csv_request records (16 bytes each, e.g. a uint8 tensor from
        ``requests_tensor``); d_out: uint64/int64 device tensor; d_status: int32 device tensor."""
        if n is None:
            n = d_reqs.numel() * d_reqs.element_size() // 16
        self._check(self.lib.csv_decode_batch(self.handle, ds.handle, C.c_void_p(d_reqs.data_ptr()), n,
                                              C.c_void_p(d_out.data_ptr()), C.c_void_p(d_status.data_ptr()),
                                              C.c_void_p(_stream_handle(stream))))

    def decode_batch_static(self, ds: Dataset, d_reqs, d_out, d_status, stream=None, n: int | None = None):
        """csv_decode_batch_static: the same decode with no allocation; its scratch is the library's fixed
        device array (see include/csv.h), so calls that overlap on the GPU race."""
        if n is None:
            n = d_reqs.numel() * d_reqs.element_size() // 16
        self._check(self.lib.csv_decode_batch_static(self.handle, ds.handle, C.c_void_p(d_reqs.data_ptr()), n,
                                                     C.c_void_p(d_out.data_ptr()), C.c_void_p(d_status.data_ptr()),
                                                     C.c_void_p(_stream_handle(stream))))

    def decode_image(self, image: bytes, lod: int, check: bool = True):
        """Host .csbd bytes -> (labels (numBricks, 8^lod) uint64, status (numBricks,) uint32)."""
        a = np.frombuffer(image, np.uint8)
        nb = int(np.frombuffer(image[8:12], np.uint32)[0])
        out = np.zeros((max(1, nb), 1 << (3 * lod)), np.uint64)
        st = np.zeros(max(1, nb), np.uint32)
        rc = self.lib.csv_decode_image(self.handle, a.ctypes.data_as(C.POINTER(C.c_uint8)), len(image), lod,
                                       out.ctypes.data_as(C.POINTER(C.c_uint64)),
                                       st.ctypes.data_as(C.POINTER(C.c_uint32)))
        if rc and (check or rc != -6):
            self._check(rc)
        return out[:nb], st[:nb]

    # ---- ray marcher ----------------------------------------------------
    def render(self, cam16, width: int, height: int, grid_size: float, brick_size: int, bricks_per_axis: int,
               d_slots, d_labels, d_label_out, d_depth_out, d_requests=None, d_hidden=None, stream=None):
        """Label/depth image (csv_render).  cam16: float32[16] from csvb200.camera.camera_uniform; d_slots: device
        tensor of csv_brick_slot records (16 bytes each)."""
        from .camera import camera_struct
        cam = camera_struct(cam16)
        n_slots = d_slots.numel() * d_slots.element_size() // 16
        self._check(self.lib.csv_render(
            self.handle, C.byref(cam), width, height, grid_size, brick_size, bricks_per_axis,
            C.c_void_p(d_slots.data_ptr()), n_slots, C.c_void_p(d_labels.data_ptr()),
            C.c_void_p(d_hidden.data_ptr() if d_hidden is not None else None),
            0 if d_hidden is None else d_hidden.numel(), C.c_void_p(d_label_out.data_ptr()),
            C.c_void_p(d_depth_out.data_ptr()),
            C.c_void_p(d_requests.data_ptr() if d_requests is not None else None),
            C.c_void_p(_stream_handle(stream))))

    def lighting(self, light_angle_deg: float = 25.0) -> Lighting:
        """The viewer's default lighting for a light at this angle on its west-east arc (csv_lighting_default)."""
        li = Lighting()
        self._check(self.lib.csv_lighting_default(light_angle_deg, C.byref(li)))
        return li

    def transfer_function(self, ds, hidden=None):
        """(keys uint64, rgba uint32) of the dataset's labels (csv_transfer_function); hidden labels transparent."""
        hid = np.ascontiguousarray(hidden if hidden is not None else np.zeros(1, np.uint64), np.uint64)
        nh = 0 if hidden is None else len(hidden)
        n = C.c_uint32()
        self.lib.csv_transfer_function(ds.handle, hid.ctypes.data_as(C.POINTER(C.c_uint64)), nh, None, None, 0,
                                       C.byref(n))
        keys = np.zeros(max(n.value, 1), np.uint64)
        cols = np.zeros(max(n.value, 1), np.uint32)
        self._check(self.lib.csv_transfer_function(ds.handle, hid.ctypes.data_as(C.POINTER(C.c_uint64)), nh,
                                                   keys.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                   cols.ctypes.data_as(C.POINTER(C.c_uint32)), n.value, C.byref(n)))
        return keys[:n.value], cols[:n.value]

    def render_rgba(self, cam16, width: int, height: int, grid_size: float, brick_size: int, bricks_per_axis: int,
                    d_slots, d_labels, d_tf_keys, d_tf_rgba, lighting: Lighting, d_rgba_out, d_requests=None,
                    stream=None):
        """RGBA8 image (csv_render_rgba) through the transfer function (device tensors d_tf_keys uint64 /
        d_tf_rgba int32 or uint32) with the given lighting."""
        from .camera import camera_struct
        cam = camera_struct(cam16)
        n_slots = d_slots.numel() * d_slots.element_size() // 16
        n_tf = d_tf_keys.numel() if d_tf_keys is not None else 0
        self._check(self.lib.csv_render_rgba(
            self.handle, C.byref(cam), width, height, grid_size, brick_size, bricks_per_axis,
            C.c_void_p(d_slots.data_ptr()), n_slots, C.c_void_p(d_labels.data_ptr()),
            C.c_void_p(d_tf_keys.data_ptr() if n_tf else None), C.c_void_p(d_tf_rgba.data_ptr() if n_tf else None),
            n_tf, C.byref(lighting), C.c_void_p(d_rgba_out.data_ptr()),
            C.c_void_p(d_requests.data_ptr() if d_requests is not None else None),
            C.c_void_p(_stream_handle(stream))))

    # ---- tensor-core dense layer ------------------------------------------
    def gemm_bf16(self, A, B, bias=None, mask=None, relu=False, C=None, Cb=None, CbT=None, CT=None, err=None,
                  stream=None):
        """C = epilogue(A . B^T) on the tensor cores (csv_gemm_bf16); A [M][K], B [N][K] bf16 device tensors."""
        M, K = A.shape
        N = B.shape[0]
        self._check(self.lib.csv_gemm_bf16(self.handle, _vp(A), _vp(B), M, N, K, _vp(bias), _vp(mask),
                                           1 if relu else 0, _vp(C), _vp(Cb), _vp(CbT), _vp(CT), _vp(err),
                                           C_MOD.c_void_p(_stream_handle(stream))))

    # ---- mode / table selector -----------------------------------------------
    def encode_stats(self, d_volume, brick_size: int, d_hist, stream=None):
        """Per brick and encoding mode, the 16-bin nibble histogram (d_hist: int32 tensor nb x 12 x 16)."""
        D, H, W = d_volume.shape
        self._check(self.lib.csv_encode_stats(self.handle, _vp(d_volume), W, H, D, brick_size, _vp(d_hist),
                                              C.c_void_p(_stream_handle(stream))))

    def select_exhaustive(self, d_hist, tables, d_sel, d_cost=None, stream=None):
        """Per brick the (mode, table) with the fewest estimated bits -> d_sel (uint8: mode | table << 4)."""
        t = np.ascontiguousarray(tables, np.uint32).reshape(-1, 16)
        self._check(self.lib.csv_select_exhaustive(self.handle, _vp(d_hist), d_hist.shape[0],
                                                   t.ctypes.data_as(C.POINTER(C.c_uint32)), len(t), _vp(d_sel),
                                                   _vp(d_cost), C.c_void_p(_stream_handle(stream))))

    def encode_device_sel(self, d_volume, brick_size: int, tables=None, d_sel=None, stream=None) -> int:
        """Encode with per-brick modes and shared tables (version 2 when tables are given); returns the length."""
        D, H, W = d_volume.shape
        t = None if tables is None else np.ascontiguousarray(tables, np.uint32).reshape(-1, 16)
        n = C.c_size_t()
        self._check(self.lib.csv_encode_device_sel(
            self.handle, _vp(d_volume), W, H, D, brick_size,
            None if t is None else t.ctypes.data_as(C.POINTER(C.c_uint32)), 0 if t is None else len(t),
            _vp(d_sel), C.c_void_p(_stream_handle(stream)), C.byref(n)))
        return n.value

    def encode_learned(self, d_volume, brick_size: int, net: "SelectorNet", tables, stream=None) -> int:
        """csv_encode_learned: features, the network's choices and the encode in one call; the image length."""
        D, H, W = d_volume.shape
        t = np.ascontiguousarray(tables, np.uint32)
        n = C.c_size_t()
        self._check(self.lib.csv_encode_learned(self.handle, C.c_void_p(d_volume.data_ptr()), W, H, D, brick_size,
                                                net.handle, t.ctypes.data_as(C.POINTER(C.c_uint32)), t.shape[0],
                                                C.c_void_p(_stream_handle(stream)), C.byref(n)))
        return n.value

    def brick_features(self, d_volume, brick_size: int, d_features, stream=None):
        """32 statistics per brick (d_features: float32 tensor nb x 32)."""
        D, H, W = d_volume.shape
        self._check(self.lib.csv_brick_features(self.handle, _vp(d_volume), W, H, D, brick_size, _vp(d_features),
                                                C.c_void_p(_stream_handle(stream))))

    # ---- workload generator ---------------------------------------------
    def synth_volume(self, d_volume, kind: int, n_cells: int, n_tubes: int = 0, r_min: float = 0.0,
                     r_max: float = 0.0, zero_frac: float = 0.0, seed: int = 0, stream=None):
        D, H, W = d_volume.shape
        self._check(self.lib.csv_synth_volume(self.handle, C.c_void_p(d_volume.data_ptr()), W, H, D, kind, n_cells,
                                              n_tubes, r_min, r_max, zero_frac, seed,
                                              C.c_void_p(_stream_handle(stream))))


class Server:
    """The viewer's frame loop on the device (csv_serve_*): sessions submit cameras, steps plan, cache, decode and
    render on one stream; poll returns per-frame counters and step times."""

    def __init__(self, codec: Codec, dataset: Dataset, width: int, height: int, fov: float, cache_bytes: int = 0,
                 max_sessions: int = 1, cone: int = CONE_SCREEN, hidden=None, admit: int = ADMIT_CONE):
        self.codec, self.dataset, self.lib = codec, dataset, codec.lib
        cfg = ServeConfig(width, height, max_sessions, cone, fov, cache_bytes, admit, 0)
        hid = np.ascontiguousarray(hidden if hidden is not None else np.zeros(1, np.uint64), np.uint64)
        h = C.c_void_p()
        codec._check(self.lib.csv_serve_create(codec.handle, dataset.handle, C.byref(cfg),
                                               hid.ctypes.data_as(C.POINTER(C.c_uint64)),
                                               0 if hidden is None else len(hidden), C.byref(h)))
        self.handle = h
        self.width, self.height, self.fov = width, height, fov
        self._keep = {}

    @staticmethod
    def view(position, direction) -> View:
        v = View()
        for a in range(3):
            v.position[a] = float(position[a])
            v.direction[a] = float(direction[a])
        return v

    def submit(self, session: int, position, direction, d_label, d_depth):
        v = self.view(position, direction)
        self._keep[session] = (d_label, d_depth)
        self.codec._check(self.lib.csv_serve_submit(self.handle, session, C.byref(v), C.c_void_p(d_label.data_ptr()),
                                                    C.c_void_p(d_depth.data_ptr())))

    def submit_rgba(self, session: int, position, direction, d_rgba):
        """A frame as the viewer shows it: an RGBA8 image (W*H int32/uint32 device tensor) through the dataset's
        transfer function and the server's lighting (csv_serve_submit_rgba)."""
        v = self.view(position, direction)
        self._keep[session] = (d_rgba,)
        self.codec._check(self.lib.csv_serve_submit_rgba(self.handle, session, C.byref(v),
                                                         C.c_void_p(d_rgba.data_ptr())))

    def set_lighting(self, lighting: "Lighting"):
        self.codec._check(self.lib.csv_serve_set_lighting(self.handle, C.byref(lighting)))

    def step(self, stream=None) -> int:
        sid = C.c_uint64()
        self.codec._check(self.lib.csv_serve_step(self.handle, C.c_void_p(_stream_handle(stream)), C.byref(sid)))
        return sid.value

    def poll(self, wait: bool = True, max_frames: int = 4096):
        out = (FrameStats * max_frames)()
        n = C.c_uint32()
        self.codec._check(self.lib.csv_serve_poll(self.handle, out, max_frames, C.byref(n), 1 if wait else 0))
        return [out[i].as_dict() for i in range(n.value)]

    def camera(self, position, direction) -> np.ndarray:
        """The float32[16] camera the server renders this view with."""
        v = self.view(position, direction)
        cam = (C.c_float * 16)()
        self.codec._check(self.lib.csv_serve_camera(self.handle, C.byref(v), cam))
        return np.array(cam[:], np.float32)

    def compact(self, stream=None):
        """CacheState.compact(): resident blocks packed from the start of the block space (csv_serve_compact)."""
        self.codec._check(self.lib.csv_serve_compact(self.handle, C.c_void_p(_stream_handle(stream))))

    def leave(self, session: int):
        """The session closes; its cache blocks are released by the next step."""
        self.codec._check(self.lib.csv_serve_close(self.handle, session))

    def info(self, session: int = 0) -> ServeInfo:
        i = ServeInfo()
        self.codec._check(self.lib.csv_serve_state(self.handle, session, C.byref(i)))
        return i

    def slots_tensor(self, session: int = 0):
        """Device view (uint8, n_slots * 16 bytes) of a session's brick slot table."""
        i = self.info(session)
        return _device_view(i.slots, int(i.n_slots) * 16, "|u1", self.codec.device)

    def cache_tensor(self):
        """Device view (int64) of the label cache: palette-0 table, then blocks."""
        i = self.info()
        return _device_view(i.cache, int(i.cache_labels), "<i8", self.codec.device)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.csv_serve_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _device_view(ptr: int, n: int, typestr: str, device: int):
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 2}

    return torch.as_tensor(_View(), device=f"cuda:{device}")


MLP_PARAMS = 256 * 64 + 256 + 256 * 256 + 256 + 32 * 256 + 32


def write_selector(lib, path: str, params: np.ndarray, tables: np.ndarray):
    p = np.ascontiguousarray(params, np.float32)
    t = np.ascontiguousarray(tables, np.uint32)
    rc = lib.csv_selector_write(os.fsencode(path), p.ctypes.data_as(C.POINTER(C.c_float)),
                                t.ctypes.data_as(C.POINTER(C.c_uint32)), t.shape[0])
    if rc:
        raise CsvError(rc, f"csv_selector_write({path}) failed")


def read_selector(lib, path: str):
    """(params, tables) of a selector file; host only (no device needed)."""
    p = np.zeros(MLP_PARAMS, np.float32)
    t = np.zeros((16, 16), np.uint32)
    n = C.c_uint32()
    rc = lib.csv_selector_read(os.fsencode(path), p.ctypes.data_as(C.POINTER(C.c_float)),
                               t.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(n))
    if rc:
        raise CsvError(rc, f"csv_selector_read({path}) failed")
    return p, t[: n.value].copy()


class SelectorNet:
    """The mode / table selector network on the device (csv_mlp_*)."""

    def __init__(self, codec: Codec, params: np.ndarray):
        self.codec, self.lib = codec, codec.lib
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == MLP_PARAMS
        h = C.c_void_p()
        codec._check(self.lib.csv_mlp_create(codec.handle, p.ctypes.data_as(C.POINTER(C.c_float)), C.byref(h)))
        self.handle = h

    @staticmethod
    def init_params(seed: int = 0) -> np.ndarray:
        """He-uniform weights (unused input columns and output rows zero), zero biases."""
        rng = np.random.default_rng(seed)
        p = np.zeros(MLP_PARAMS, np.float32)
        o = 0
        for rows, cols, fan in [(256, 64, 32), (256, 256, 256), (32, 256, 256)]:
            w = rng.uniform(-1, 1, (rows, cols)) * np.sqrt(6.0 / fan)
            if cols == 64:
                w[:, 32:] = 0
            if rows == 32:
                w[28:, :] = 0
            p[o:o + rows * cols] = w.ravel()
            o += rows * cols + rows
        return p

    def params(self, grads: bool = False):
        p = np.zeros(MLP_PARAMS, np.float32)
        g = np.zeros(MLP_PARAMS, np.float32) if grads else None
        fp = C.POINTER(C.c_float)
        self.codec._check(self.lib.csv_mlp_params(self.handle, p.ctypes.data_as(fp),
                                                  g.ctypes.data_as(fp) if grads else None))
        return (p, g) if grads else p

    def forward(self, d_features, d_logits=None, d_sel=None, stream=None):
        self.codec._check(self.lib.csv_mlp_forward(self.handle, _vp(d_features), d_features.shape[0], _vp(d_logits),
                                                   _vp(d_sel), C.c_void_p(_stream_handle(stream))))

    def grad(self, d_features, d_label, stream=None) -> float:
        loss = C.c_float()
        self.codec._check(self.lib.csv_mlp_grad(self.handle, _vp(d_features), _vp(d_label), d_features.shape[0],
                                                C.byref(loss), C.c_void_p(_stream_handle(stream))))
        return float(loss.value)

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8, stream=None):
        self.codec._check(self.lib.csv_mlp_adam(self.handle, lr, beta1, beta2, eps,
                                                C.c_void_p(_stream_handle(stream))))

    def status(self) -> int:
        return self.lib.csv_mlp_status(self.handle)

    def save(self, path: str, tables: np.ndarray):
        """A selector file with these tables and this network's parameters (csv_selector_write)."""
        write_selector(self.lib, path, self.params(), tables)

    @classmethod
    def load(cls, codec: Codec, path: str):
        """(network, tables) from a selector file (csv_selector_read + csv_mlp_create)."""
        params, tables = read_selector(codec.lib, path)
        return cls(codec, params), tables

    def close(self):
        if getattr(self, "handle", None):
            self.lib.csv_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def requests(bricks, lods, dsts) -> np.ndarray:
    r = np.zeros(len(bricks), REQUEST_DTYPE)
    r["brick"] = bricks
    r["lod"] = lods
    r["dst"] = dsts
    return r


def requests_tensor(reqs: np.ndarray, device="cuda"):
    import torch
    return torch.from_numpy(reqs.view(np.uint8).copy()).to(device)
