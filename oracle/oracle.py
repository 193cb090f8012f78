"""ctypes loader for the CPU checkers.  TEST INFRASTRUCTURE ONLY.

``Oracle``     -> oracle/libcsvoracle.so, this project's C restatement of the
                  reference codec (oracle/csv_oracle.c).
``Reference``  -> oracle/_ref/libcsvref.so, the unmodified reference encoder /
                  decoder sources compiled by ``make -C oracle ref``.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
import this module, and only to check or to time the CPU reference.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libcsvoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcsvref.so")
# The reference project's root: CSV_REFERENCE_ROOT, else where this machine keeps it.  Only the build recipe
# (build(), oracle/Makefile) and fixture generation read it; nothing that runs on a GPU machine needs it.
REF_ROOT = os.environ.get("CSV_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "encoder", "CSVEncoder", "src")
REF_SHIPPED = os.path.join(REF_ROOT, "encoder", "CSVEncoder", "compressed_dataset.csbd")

_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def build(ref: bool | None = None) -> None:
    """Compile the restatement, and the reference library when its sources exist."""
    subprocess.run(["make", "-s", "-C", HERE, "libcsvoracle.so"], check=True)
    if ref is None:
        ref = os.path.isdir(REF_SRC)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_SRC={REF_SRC}"], check=True)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        L.or_morton3.restype = C.c_uint32
        L.or_morton3.argtypes = [C.c_uint32] * 3
        L.or_majority8.restype = C.c_uint64
        L.or_majority8.argtypes = [_u64p]
        L.or_build_model.argtypes = [_u64p, _u32p, _u32p]
        L.or_encode.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_uint32,
                                C.POINTER(_u8p), C.POINTER(C.c_size_t)]
        L.or_transfer_function.argtypes = [_u64p, C.c_uint32, _u64p, C.c_uint32, _u32p]
        L.or_label_rgba.restype = C.c_uint32
        L.or_label_rgba.argtypes = [C.c_uint64, _u64p, _u32p, C.c_uint32]
        L.or_render_rgba_rows.argtypes = [C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.c_float, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64, _u64p, _u64p,
                                          _u32p, C.c_uint32, C.POINTER(C.c_float), _u32p]
        L.or_encode_threads.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_uint32, C.c_uint32,
                                        C.POINTER(_u8p), C.POINTER(C.c_size_t)]
        L.or_synth_volume.argtypes = [_u64p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_uint32, C.c_uint32,
                                      C.c_float, C.c_float, C.c_float, C.c_uint64, C.c_uint32]
        L.or_encode_shard.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_uint32, C.c_uint32, C.c_uint32,
                                      _u64p, _u64p, C.POINTER(_u8p), C.POINTER(C.c_size_t)]
        L.or_pyramid.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_uint32, C.c_uint32,
                                 _u64p, _u8p]
        L.or_rans_decode.argtypes = [_u32p, _u32p, C.c_uint32, _u8p, C.c_uint32, C.c_uint32, _u8p]
        L.or_decode_brick.argtypes = [_u64p, C.c_uint32, _u8p, C.c_uint32, C.c_uint32, C.c_uint32, _u64p]
        L.or_decode_image.argtypes = [_u8p, C.c_size_t, C.c_uint32, _u64p, _u32p]
        L.or_rans_states.argtypes = [_u32p, _u32p, _u8p, C.c_uint32, C.c_uint32, C.c_uint32, _u32p]
        L.or_seek_index.argtypes = [_u32p, _u32p, _u8p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_uint32, _u32p, _u32p, _u32p, C.c_uint32, _u32p]
        L.or_free.argtypes = [C.c_void_p]
        L.or_brick_lod.restype = C.c_uint32
        L.or_brick_lod.argtypes = [C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double), C.c_double, C.c_uint32]
        L.or_render.argtypes = [C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, C.c_uint32,
                                C.c_void_p, C.c_uint64, _u64p, _u64p, C.c_uint32, _u64p, C.POINTER(C.c_float), _u32p]
        fp = C.POINTER(C.c_float)
        L.or_encode_sel.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_uint32, _u8p, _u32p, C.c_uint32,
                                    C.POINTER(_u8p), C.POINTER(C.c_size_t)]
        L.or_encode_stats.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_uint32, _u32p]
        L.or_select_exhaustive.argtypes = [_u32p, C.c_uint32, _u32p, C.c_uint32, _u8p, _u64p]
        L.or_brick_features.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_uint32, fp]
        L.or_mlp_forward.argtypes = [fp, fp, C.c_uint32, fp]
        L.or_mlp_grad.restype = C.c_float
        L.or_mlp_grad.argtypes = [fp, fp, _u8p, C.c_uint32, fp]
        L.or_camera_uniform.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                        C.POINTER(C.c_float)]
        L.or_serve_constants.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.or_serve_new.restype = C.c_void_p
        L.or_serve_new.argtypes = [_u8p, C.c_size_t, C.c_uint32, C.c_uint32, C.c_double, C.c_uint32, C.c_uint64,
                                   _u64p, C.c_uint32]
        L.or_serve_step.argtypes = [C.c_void_p, _u32p, C.POINTER(C.c_double), _u8p, C.c_uint32, _u64p,
                                    C.POINTER(C.c_float), _u32p]
        L.or_serve_set_admit.argtypes = [C.c_void_p, C.c_uint32]
        L.or_serve_compact.restype = C.c_int
        L.or_serve_compact.argtypes = [C.c_void_p]
        L.or_serve_n_slots.restype = C.c_uint64
        L.or_serve_n_slots.argtypes = [C.c_void_p]
        L.or_serve_bricks_per_axis.restype = C.c_uint32
        L.or_serve_bricks_per_axis.argtypes = [C.c_void_p]
        L.or_serve_slots.restype = C.c_void_p
        L.or_serve_slots.argtypes = [C.c_void_p, C.c_uint32]
        L.or_serve_cache.restype = C.c_void_p
        L.or_serve_cache.argtypes = [C.c_void_p]
        L.or_serve_free.argtypes = [C.c_void_p]
        L.or_render_rows.argtypes = [C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                     C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64, _u64p, _u64p, C.c_uint32, _u64p,
                                     C.POINTER(C.c_float), _u32p, _u32p]
        self.lib = L

    def brick_lod(self, center, brick_size, cam, focal, max_lod) -> int:
        c = (C.c_double * 3)(*center)
        p = (C.c_double * 3)(*cam)
        return int(self.lib.or_brick_lod(c, brick_size, p, focal, max_lod))

    def render(self, cam16: np.ndarray, W: int, H: int, grid: float, brick: int, bpa: int, slots: np.ndarray,
               labels: np.ndarray, hidden: np.ndarray | None = None, rows=None, with_requests: bool = False):
        """cam16: float32[16] (camera.js getUniformData layout); slots: structured (offset u8, lod u4, flags u4).

        rows=(y0, ystep) renders only those rows; with_requests adds the per-slot request words."""
        cam = np.ascontiguousarray(cam16, np.float32)
        lab = np.ascontiguousarray(labels, np.uint64)
        hid = np.ascontiguousarray(hidden if hidden is not None else np.zeros(1, np.uint64), np.uint64)
        nh = 0 if hidden is None else len(hidden)
        out = np.zeros(W * H, np.uint64)
        dep = np.zeros(W * H, np.float32)
        miss = np.zeros(W * H, np.uint32)
        sl = np.ascontiguousarray(slots)
        y0, ystep = rows if rows is not None else (0, 1)
        req = np.zeros(len(sl), np.uint32)
        self.lib.or_render_rows(cam.ctypes.data_as(C.POINTER(C.c_float)), W, H, y0, ystep, grid, brick, bpa,
                                sl.ctypes.data, len(sl), _ptr(lab, _u64p), _ptr(hid, _u64p), nh, _ptr(out, _u64p),
                                dep.ctypes.data_as(C.POINTER(C.c_float)), _ptr(miss, _u32p), _ptr(req, _u32p))
        if with_requests:
            return out.reshape(H, W), dep.reshape(H, W), miss.reshape(H, W), req
        return out.reshape(H, W), dep.reshape(H, W), miss.reshape(H, W)

    def transfer_function(self, labels: np.ndarray, hidden=None) -> np.ndarray:
        """RGBA8 of distinct labels given ascending (buildTransferFunctionBuffers + hslToRgb)."""
        lab = np.ascontiguousarray(labels, np.uint64)
        hid = np.ascontiguousarray(hidden if hidden is not None else np.zeros(1, np.uint64), np.uint64)
        out = np.zeros(max(len(lab), 1), np.uint32)
        self.lib.or_transfer_function(_ptr(lab, _u64p), len(lab), _ptr(hid, _u64p),
                                      0 if hidden is None else len(hidden), _ptr(out, _u32p))
        return out[:len(lab)]

    def label_rgba(self, v: int, keys: np.ndarray, cols: np.ndarray) -> int:
        k = np.ascontiguousarray(keys, np.uint64)
        c = np.ascontiguousarray(cols, np.uint32)
        return int(self.lib.or_label_rgba(C.c_uint64(v), _ptr(k, _u64p), _ptr(c, _u32p), len(k)))

    def render_rgba(self, cam16, W: int, H: int, grid: float, brick: int, bpa: int, slots, labels, keys, cols,
                    lighting, rows=None) -> np.ndarray:
        """The RGBA ray march (or_render_rgba_rows); lighting: light_dir[3], ambient, diffuse."""
        cam = np.ascontiguousarray(cam16, np.float32)
        lab = np.ascontiguousarray(labels, np.uint64)
        k = np.ascontiguousarray(keys if len(keys) else np.zeros(1, np.uint64), np.uint64)
        c = np.ascontiguousarray(cols if len(cols) else np.zeros(1, np.uint32), np.uint32)
        li = np.ascontiguousarray(lighting, np.float32)
        sl = np.ascontiguousarray(slots)
        out = np.zeros(W * H, np.uint32)
        y0, ystep = rows if rows is not None else (0, 1)
        self.lib.or_render_rgba_rows(cam.ctypes.data_as(C.POINTER(C.c_float)), W, H, y0, ystep, grid, brick, bpa,
                                     sl.ctypes.data, len(sl), _ptr(lab, _u64p), _ptr(k, _u64p), _ptr(c, _u32p), len(keys),
                                     li.ctypes.data_as(C.POINTER(C.c_float)), _ptr(out, _u32p))
        return out.reshape(H, W)

    def morton3(self, x, y, z) -> int:
        return self.lib.or_morton3(x, y, z)

    # ---- mode / table selector
    def encode_sel(self, vol: np.ndarray, brick: int, sel=None, tables=None) -> bytes:
        """Per-brick mode | table << 4 (sel) and shared tables (n x 16 frequencies) -> version-2 image
        (version 1 when tables is None)."""
        v = np.ascontiguousarray(vol, dtype=np.uint64)
        D, H, W = v.shape
        s = None if sel is None else np.ascontiguousarray(sel, np.uint8)
        t = None if tables is None else np.ascontiguousarray(tables, np.uint32).reshape(-1, 16)
        out = _u8p()
        n = C.c_size_t()
        rc = self.lib.or_encode_sel(_ptr(v, _u64p), W, H, D, brick, None if s is None else _ptr(s, _u8p),
                                    None if t is None else _ptr(t, _u32p), 0 if t is None else len(t),
                                    C.byref(out), C.byref(n))
        if rc:
            raise RuntimeError("oracle encode_sel failed")
        data = C.string_at(out, n.value)
        self.lib.or_free(out)
        return data

    def encode_stats(self, vol: np.ndarray, brick: int) -> np.ndarray:
        v = np.ascontiguousarray(vol, dtype=np.uint64)
        D, H, W = v.shape
        nb = -(-W // brick) * -(-H // brick) * -(-D // brick)
        h = np.zeros((nb, 12, 16), np.uint32)
        if self.lib.or_encode_stats(_ptr(v, _u64p), W, H, D, brick, _ptr(h, _u32p)):
            raise RuntimeError("oracle encode_stats failed")
        return h

    def select_exhaustive(self, hist: np.ndarray, tables):
        h = np.ascontiguousarray(hist, np.uint32)
        t = np.ascontiguousarray(tables, np.uint32).reshape(-1, 16)
        nb = h.shape[0]
        sel = np.zeros(nb, np.uint8)
        cost = np.zeros((nb, 12, len(t)), np.uint64)
        self.lib.or_select_exhaustive(_ptr(h, _u32p), nb, _ptr(t, _u32p), len(t), _ptr(sel, _u8p), _ptr(cost, _u64p))
        return sel, cost

    def brick_features(self, vol: np.ndarray, brick: int) -> np.ndarray:
        v = np.ascontiguousarray(vol, dtype=np.uint64)
        D, H, W = v.shape
        nb = -(-W // brick) * -(-H // brick) * -(-D // brick)
        f = np.zeros((nb, 32), np.float32)
        if self.lib.or_brick_features(_ptr(v, _u64p), W, H, D, brick, f.ctypes.data_as(C.POINTER(C.c_float))):
            raise RuntimeError("oracle features failed")
        return f

    def mlp_forward(self, params: np.ndarray, feat: np.ndarray) -> np.ndarray:
        p = np.ascontiguousarray(params, np.float32)
        f = np.ascontiguousarray(feat, np.float32)
        z = np.zeros((len(f), 32), np.float32)
        fp = C.POINTER(C.c_float)
        self.lib.or_mlp_forward(p.ctypes.data_as(fp), f.ctypes.data_as(fp), len(f), z.ctypes.data_as(fp))
        return z

    def mlp_grad(self, params: np.ndarray, feat: np.ndarray, label: np.ndarray):
        p = np.ascontiguousarray(params, np.float32)
        f = np.ascontiguousarray(feat, np.float32)
        lab = np.ascontiguousarray(label, np.uint8)
        g = np.zeros_like(p)
        fp = C.POINTER(C.c_float)
        loss = self.lib.or_mlp_grad(p.ctypes.data_as(fp), f.ctypes.data_as(fp), _ptr(lab, _u8p), len(f),
                                    g.ctypes.data_as(fp))
        return float(loss), g

    def majority8(self, labels) -> int:
        a = np.ascontiguousarray(labels, dtype=np.uint64)
        return int(self.lib.or_majority8(_ptr(a, _u64p)))

    def build_model(self, raw16):
        raw = np.ascontiguousarray(raw16, dtype=np.uint64)
        f = np.zeros(16, np.uint32)
        c = np.zeros(17, np.uint32)
        self.lib.or_build_model(_ptr(raw, _u64p), _ptr(f, _u32p), _ptr(c, _u32p))
        return f, c

    def encode_shard(self, slab: np.ndarray, brick: int, bx0: int, index_base: int, hist_in=None):
        """One x-slab of a larger volume (or_encode_shard): (image of its bricks, sample histogram)."""
        v = np.ascontiguousarray(slab, dtype=np.uint64)
        D, H, W = v.shape
        out = _u8p()
        n = C.c_size_t()
        h_out = np.zeros(16, np.uint64)
        h_in = None if hist_in is None else np.ascontiguousarray(hist_in, np.uint64)
        rc = self.lib.or_encode_shard(_ptr(v, _u64p), W, H, D, brick, bx0, index_base,
                                      None if h_in is None else _ptr(h_in, _u64p), _ptr(h_out, _u64p),
                                      C.byref(out), C.byref(n))
        if rc:
            raise RuntimeError("oracle shard encode failed")
        data = C.string_at(out, n.value)
        self.lib.or_free(out)
        return data, h_out

    def encode(self, vol: np.ndarray, brick: int) -> bytes:
        """vol has shape (D, H, W) in C order, i.e. x fastest."""
        v = np.ascontiguousarray(vol, dtype=np.uint64)
        D, H, W = v.shape
        out = _u8p()
        n = C.c_size_t()
        rc = self.lib.or_encode(_ptr(v, _u64p), W, H, D, brick, C.byref(out), C.byref(n))
        if rc:
            raise RuntimeError("oracle encode failed")
        data = C.string_at(out, n.value)
        self.lib.or_free(out)
        return data

    def encode_threads(self, vol: np.ndarray, brick: int, threads: int = 0) -> bytes:
        """encode() with the bricks spread over host threads (0: every core); the same bytes."""
        v = np.ascontiguousarray(vol, dtype=np.uint64)
        D, H, W = v.shape
        out = _u8p()
        n = C.c_size_t()
        rc = self.lib.or_encode_threads(_ptr(v, _u64p), W, H, D, brick, threads or (os.cpu_count() or 1),
                                        C.byref(out), C.byref(n))
        if rc:
            raise RuntimeError("oracle encode failed")
        data = C.string_at(out, n.value)
        self.lib.or_free(out)
        return data

    def synth_volume(self, shape, kind: int, n_cells: int, n_tubes: int, r_min: float, r_max: float,
                     zero_frac: float, seed: int, threads: int = 0) -> np.ndarray:
        """The native library's csv_synth_volume restated on the CPU: a (D, H, W) uint64 volume, x fastest."""
        D, H, W = shape
        vol = np.empty((D, H, W), np.uint64)
        rc = self.lib.or_synth_volume(_ptr(vol, _u64p), W, H, D, kind, n_cells, n_tubes, r_min, r_max, zero_frac,
                                      seed, threads or (os.cpu_count() or 1))
        if rc:
            raise RuntimeError("oracle synth failed")
        return vol

    def pyramid(self, vol: np.ndarray, brick: int, index: int):
        v = np.ascontiguousarray(vol, dtype=np.uint64)
        D, H, W = v.shape
        levels = brick.bit_length()
        tot = ((1 << (3 * levels)) - 1) // 7
        lab = np.zeros(tot, np.uint64)
        cst = np.zeros(tot, np.uint8)
        rc = self.lib.or_pyramid(_ptr(v, _u64p), W, H, D, brick, index, _ptr(lab, _u64p), _ptr(cst, _u8p))
        if rc:
            raise RuntimeError("oracle pyramid failed")
        out = []
        for l in range(levels):
            o = ((1 << (3 * l)) - 1) // 7
            out.append((lab[o:o + (1 << (3 * l))], cst[o:o + (1 << (3 * l))]))
        return out

    def decode_image(self, img: bytes, lod: int):
        a = np.frombuffer(img, np.uint8)
        nb = int(np.frombuffer(img[8:12], np.uint32)[0])
        out = np.zeros(nb * (1 << (3 * lod)), np.uint64)
        st = np.zeros(nb, np.uint32)
        rc = self.lib.or_decode_image(_ptr(a, _u8p), len(img), lod, _ptr(out, _u64p), _ptr(st, _u32p))
        if rc < 0:
            raise RuntimeError("oracle decode failed")
        return out.reshape(nb, -1), st

    def rans_decode(self, freq, cum16, enc: bytes, nsym: int) -> bytes:
        f = np.ascontiguousarray(freq, np.uint32)
        c = np.ascontiguousarray(cum16, np.uint32)
        e = np.frombuffer(enc, np.uint8)
        out = np.zeros((nsym + 1) // 2, np.uint8)
        rc = self.lib.or_rans_decode(_ptr(f, _u32p), _ptr(c, _u32p), 4096, _ptr(e, _u8p), len(enc), nsym,
                                     _ptr(out, _u8p))
        if rc:
            raise RuntimeError("oracle rans failed")
        return out.tobytes()

    def decode_brick(self, palette, nib: bytes, brick: int, lod: int):
        p = np.ascontiguousarray(palette, np.uint64)
        n = np.frombuffer(nib, np.uint8) if len(nib) else np.zeros(1, np.uint8)
        out = np.zeros(1 << (3 * lod), np.uint64)
        st = self.lib.or_decode_brick(_ptr(p, _u64p), len(p), _ptr(n, _u8p), len(nib), brick, lod,
                                      _ptr(out, _u64p))
        return out, st

    def rans_states(self, freq, cum16, enc: bytes, nsym: int, every: int) -> np.ndarray:
        """(n, 2) uint32: the chain's state {x, pos} before symbols 0, every, 2 every, ... (or_rans_states)."""
        f = np.ascontiguousarray(freq, np.uint32)
        c = np.ascontiguousarray(cum16, np.uint32)
        e = np.frombuffer(enc, np.uint8) if len(enc) else np.zeros(1, np.uint8)
        out = np.zeros(2 * (nsym // every + 1), np.uint32)
        n = self.lib.or_rans_states(_ptr(f, _u32p), _ptr(c, _u32p), _ptr(e, _u8p), len(enc), nsym, every,
                                    _ptr(out, _u32p))
        if n < 0:
            raise ValueError("stream shorter than its header")
        return out[: 2 * n].reshape(-1, 2)

    def seek_index(self, freq, cum16, enc: bytes, nsym: int, P: int, brick: int, S: int):
        f = np.ascontiguousarray(freq, np.uint32)
        c = np.ascontiguousarray(cum16, np.uint32)
        e = np.frombuffer(enc, np.uint8)
        nops = np.zeros(1, np.uint32)
        ls = np.zeros(8, np.uint32)
        maxc = nsym // S + 2
        ck = np.zeros(4 * maxc, np.uint32)
        nck = np.zeros(1, np.uint32)
        st = self.lib.or_seek_index(_ptr(f, _u32p), _ptr(c, _u32p), _ptr(e, _u8p), len(enc), nsym, P, brick, S,
                                    _ptr(nops, _u32p), _ptr(ls, _u32p), _ptr(ck, _u32p), maxc, _ptr(nck, _u32p))
        return int(nops[0]), ls, ck[:4 * int(nck[0])].reshape(-1, 4), st


SERVE_STATS = ["planned", "visible", "decoded", "freed", "resident", "rebuilt"]
SERVE_NSTATS = 8 + 2 * 8
SLOT_DTYPE = np.dtype([("offset", "<u8"), ("lod", "<u4"), ("flags", "<u4")])


def camera_uniform(oracle: "Oracle", position, direction, fov: float) -> np.ndarray:
    p = (C.c_double * 3)(*position)
    d = (C.c_double * 3)(*direction)
    out = (C.c_float * 16)()
    oracle.lib.or_camera_uniform(p, d, fov, out)
    return np.array(out[:], np.float32)


class OracleServer:
    """The viewer's frame loop restated on the CPU (csv_oracle_serve.c)."""

    def __init__(self, oracle: "Oracle", image: bytes, W: int, H: int, fov: float, cone: int, cache_bytes: int,
                 hidden=None, admit: int = 0):
        self.lib, self.W, self.H = oracle.lib, W, H
        self._img = np.frombuffer(image, np.uint8).copy()
        hid = np.ascontiguousarray(np.sort(hidden) if hidden is not None else np.zeros(1, np.uint64), np.uint64)
        self.h = self.lib.or_serve_new(_ptr(self._img, _u8p), len(self._img), W, H, fov, cone, cache_bytes,
                                       _ptr(hid, _u64p), 0 if hidden is None else len(hidden))
        if not self.h:
            raise ValueError("or_serve_new failed")
        self.lib.or_serve_set_admit(self.h, admit)
        self.n_slots = int(self.lib.or_serve_n_slots(self.h))
        self.bpa = int(self.lib.or_serve_bricks_per_axis(self.h))

    def step(self, sessions, views, render=None):
        """sessions: the open sessions (ascending ids); views: their latest (position[3], direction[3]);
        render: per session, whether it submitted a frame (default all).  Returns labels (r, H, W) and
        depth (r, H, W) of the r rendered sessions, and the stats dict (entered/missing: lists per rendered
        session)."""
        n = len(sessions)
        render = [1] * n if render is None else [1 if r else 0 for r in render]
        r = sum(render)
        ss = np.ascontiguousarray(sessions, np.uint32)
        vv = np.ascontiguousarray([list(p) + list(d) for p, d in views] or [[0.0] * 6], np.float64)
        rr = np.ascontiguousarray(render or [0], np.uint8)
        lab = np.zeros(max(1, r) * self.W * self.H, np.uint64)
        dep = np.zeros(max(1, r) * self.W * self.H, np.float32)
        st = np.zeros(SERVE_NSTATS, np.uint32)
        rc = self.lib.or_serve_step(self.h, _ptr(ss, _u32p), vv.ctypes.data_as(C.POINTER(C.c_double)),
                                    _ptr(rr, _u8p), n, _ptr(lab, _u64p), dep.ctypes.data_as(C.POINTER(C.c_float)),
                                    _ptr(st, _u32p))
        if rc:
            raise ValueError("or_serve_step failed")
        stats = {k: int(st[i]) for i, k in enumerate(SERVE_STATS)}
        stats["decoded_voxels"] = int(st[6]) | (int(st[7]) << 32)
        stats["entered"] = [int(st[8 + 2 * j]) for j in range(r)]
        stats["missing"] = [int(st[9 + 2 * j]) for j in range(r)]
        return lab[: r * self.W * self.H].reshape(r, self.H, self.W), \
            dep[: r * self.W * self.H].reshape(r, self.H, self.W), stats

    def compact(self):
        if self.lib.or_serve_compact(self.h):
            raise ValueError("or_serve_compact failed")

    def slots(self, session: int = 0) -> np.ndarray:
        buf = (C.c_uint8 * (16 * self.n_slots)).from_address(self.lib.or_serve_slots(self.h, session))
        return np.frombuffer(bytes(buf), SLOT_DTYPE)

    def cache(self, n: int) -> np.ndarray:
        buf = (C.c_uint64 * n).from_address(self.lib.or_serve_cache(self.h))
        return np.frombuffer(bytes(buf), np.uint64)

    def close(self):
        if self.h:
            self.lib.or_serve_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Reference:
    """The reference sources compiled here (oracle/_ref/libcsvref.so)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_encode.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_int, C.POINTER(_u8p),
                                 C.POINTER(C.c_size_t), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]
        L.ref_decode_brick_full.argtypes = [_u8p, C.c_size_t, C.c_uint32, _u64p]
        L.ref_decode_all_full.argtypes = [_u8p, C.c_size_t, _u64p, _u32p, C.c_uint32, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]
        L.ref_rans_decode.argtypes = [_u8p, C.c_size_t, C.c_uint32, _u8p, C.POINTER(C.c_size_t)]
        L.ref_majority8.restype = C.c_uint64
        L.ref_majority8.argtypes = [_u64p]
        L.ref_build_model.argtypes = [_u64p, _u32p, _u32p]
        L.ref_load.restype = C.c_void_p
        L.ref_load.argtypes = [_u8p, C.c_size_t]
        L.ref_unload.argtypes = [C.c_void_p]
        L.ref_decode_range.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, _u64p]
        L.ref_decode_strided.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, _u64p]
        L.ref_build_pyramid64.argtypes = [_u64p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_uint32, _u64p, _u8p]
        self.lib = L

    def error(self) -> str:
        return self.lib.ref_last_error().decode()

    def encode(self, vol: np.ndarray, brick: int, timings: bool = False):
        v = np.ascontiguousarray(vol, dtype=np.uint64)
        D, H, W = v.shape
        out = _u8p()
        n = C.c_size_t()
        t = [C.c_double(), C.c_double(), C.c_double()]
        rc = self.lib.ref_encode(_ptr(v, _u64p), W, H, D, brick, C.byref(out), C.byref(n),
                                 C.byref(t[0]), C.byref(t[1]), C.byref(t[2]))
        if rc:
            raise RuntimeError("reference encode failed: " + self.error())
        data = C.string_at(out, n.value)
        self.lib.ref_free(out)
        if timings:
            return data, {"split_ms": t[0].value, "compress_ms": t[1].value, "save_ms": t[2].value}
        return data

    def decode_brick_full(self, img: bytes, index: int, brick: int):
        a = np.frombuffer(img, np.uint8)
        out = np.zeros(brick ** 3, np.uint64)
        rc = self.lib.ref_decode_brick_full(_ptr(a, _u8p), len(img), index, _ptr(out, _u64p))
        if rc:
            raise RuntimeError(self.error())
        return out

    def decode_all_full(self, img: bytes, brick: int, max_bricks: int = 0, keep: bool = True):
        a = np.frombuffer(img, np.uint8)
        nb = int(np.frombuffer(img[8:12], np.uint32)[0])
        if max_bricks:
            nb = min(nb, max_bricks)
        out = np.zeros(nb * brick ** 3, np.uint64) if keep else None
        st = np.zeros(nb, np.uint32)
        tr, tp = C.c_double(), C.c_double()
        n = self.lib.ref_decode_all_full(_ptr(a, _u8p), len(img), _ptr(out, _u64p) if keep else None,
                                         _ptr(st, _u32p), max_bricks, C.byref(tr), C.byref(tp))
        if n < 0:
            raise RuntimeError(self.error())
        return (out.reshape(nb, -1) if keep else None), st, {"rans_ms": tr.value, "replay_ms": tp.value}

    def decode_parallel(self, img: bytes, threads: int, out: np.ndarray | None = None, stride: int = 1) -> int:
        """Full-resolution decode of bricks 0, stride, 2*stride, ... (every brick by default), split over
        `threads` host threads (ctypes releases the GIL).  out (or None) receives the decoded bricks in that
        order.  Returns the number of bricks where the reference threw."""
        from concurrent.futures import ThreadPoolExecutor
        a = np.frombuffer(img, np.uint8)
        h = self.lib.ref_load(_ptr(a, _u8p), len(img))
        if not h:
            raise RuntimeError(self.error())
        nb = int(np.frombuffer(img[8:12], np.uint32)[0])
        b = int(np.frombuffer(img[12:16], np.uint32)[0])
        stride = max(1, int(stride))
        m = len(range(0, nb, stride))
        chunk = -(-m // max(1, threads))

        def run(k):
            s = k * chunk
            c = max(0, min(chunk, m - s))
            p = None if out is None else out.reshape(-1)[s * b ** 3:].ctypes.data_as(_u64p)
            return self.lib.ref_decode_strided(h, s * stride, c, stride, p) if c else 0

        with ThreadPoolExecutor(max_workers=threads) as ex:
            bad = sum(ex.map(run, range(threads)))
        self.lib.ref_unload(h)
        return bad

    def rans_decode(self, img: bytes, index: int, nsym: int) -> bytes:
        a = np.frombuffer(img, np.uint8)
        out = np.zeros((nsym + 1) // 2 + 1, np.uint8)
        n = C.c_size_t()
        rc = self.lib.ref_rans_decode(_ptr(a, _u8p), len(img), index, _ptr(out, _u8p), C.byref(n))
        if rc:
            raise RuntimeError(self.error())
        return out[:n.value].tobytes()

    def majority8(self, labels) -> int:
        a = np.ascontiguousarray(labels, dtype=np.uint64)
        return int(self.lib.ref_majority8(_ptr(a, _u64p)))

    def build_model(self, raw16):
        raw = np.ascontiguousarray(raw16, dtype=np.uint64)
        f = np.zeros(16, np.uint32)
        c = np.zeros(17, np.uint32)
        self.lib.ref_build_model(_ptr(raw, _u64p), _ptr(f, _u32p), _ptr(c, _u32p))
        return f, c

    def pyramid64(self, vol: np.ndarray, index: int):
        v = np.ascontiguousarray(vol, dtype=np.uint64)
        D, H, W = v.shape
        tot = sum(8 ** l for l in range(7))
        lab = np.zeros(tot, np.uint64)
        cst = np.zeros(tot, np.uint8)
        n = self.lib.ref_build_pyramid64(_ptr(v, _u64p), W, H, D, index, _ptr(lab, _u64p), _ptr(cst, _u8p))
        if n < 0:
            raise RuntimeError("pyramid failed")
        # finest-first in the reference; return coarse-first like Oracle.pyramid
        out = []
        o = 0
        for l in range(6, -1, -1):
            cnt = 8 ** l
            out.append((lab[o:o + cnt], cst[o:o + cnt]))
            o += cnt
        return out[::-1]
