"""Benchmark of the B200 compressed-segmentation-volume codec.

Headline (value): bit-exact batched brick decode throughput in Gvox/s and its
%HBM roofline on the uneven-batch workload `mixed1024`: a 1024^3 uint64
volume whose x < 512 half is smooth Voronoi (2000 cells) stored in 32^3 bricks
and whose x >= 512 half is dense tubes (5000 splines, radius 1-4) over it,
stored in 64^3 bricks -- two .csbd images (one brick size per file), 16384 +
2048 bricks, decoded at full resolution in ONE launch (csv_dataset_concat),
captured in a CUDA graph with the configuration the autotuner picks.  One step
= one graph replay (8 GiB of labels written).

The same JSON line carries, on the neurite-like workload `neurite512` (512^3,
400 tubes of radius 2-12 over 3000 Voronoi cells, 64^3 bricks): GPU encode
Mvox/s against the reference encoder compiled from its sources and run on the
host (bytes compared), and that workload's decode throughput.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU: one process per GPU (torchrun); every rank decodes its own
contiguous range of the requests, about 1/N of the voxels (bricks are
independent: no collective on the data path), so scaling is strong and value =
the whole volume's voxels / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fast-compressed-segmentation_b200"))

METRIC = "bit-exact decode Gvox/s & %HBM peak; encode Mvox/s vs CPU; p99 frame ms"
MIXED = dict(name="mixed1024", shape=(1024, 1024, 1024), kind=2, n_cells=2000, n_tubes=5000, r_min=1.0, r_max=4.0,
             zero_frac=0.0, seed=3, split_x=512, brick_left=32, brick_right=64)
# The same generator at 1/8 of the volume (cells and tubes scaled with it): the small case for profiler captures.
MIXED512 = dict(MIXED, name="mixed512", shape=(512, 512, 512), n_cells=250, n_tubes=625, split_x=256)
# The same shape with the dense half pushed toward the size span configs[2] describes: 80,000 tubes of radius
# 0.5-1.5 in the 64^3 half (encoded streams from ~100 B to ~100 KB; palettes far above 300, which the op grammar
# makes unavoidable at these stream sizes).  Reported beside the headline, not instead of it.
MIXED_DENSE = dict(MIXED, name="mixed1024dense", n_tubes=80000, r_min=0.5, r_max=1.5)
WORKLOADS = {w["name"]: w for w in (MIXED, MIXED512, MIXED_DENSE)}
SERVE = dict(name="serve2048", shape=(2048, 2048, 2048), brick=64, kind=1, n_cells=20000, n_tubes=8000, r_min=2.0,
             r_max=12.0, zero_frac=0.15, seed=5, width=1920, height=1080, frames=600, cache_gib=24,
             fov=1.0471975511965976)  # pi/3 (camera.js:19)
SELECTOR = dict(train_volumes=40, steps=1200, seed=700)  # 40 x 512 bricks of 64^3 = 20,480 training bricks
NEURITE = dict(name="neurite512", shape=(512, 512, 512), brick=64, kind=1, n_cells=3000, n_tubes=400, r_min=2.0,
               r_max=12.0, zero_frac=0.15, seed=2)
FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """SM clock and clock-event reasons sampled through NVML every 10 ms during the timed region (read only)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4,
               "hw_power_brake_slowdown": 0x80}

    def __init__(self, device: int):
        import threading
        self.samples, self.reasons, self.max_mhz = [], 0, None
        self.stop_evt = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # noqa: BLE001
            self.nv, self.err = None, str(e)
            return
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        while not self.stop_evt.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                self.reasons |= self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:  # noqa: BLE001
                pass
            self.stop_evt.wait(0.01)

    def stop(self):
        if self.nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [f"nvml unavailable: {self.err}"]}
        self.stop_evt.set()
        self.t.join(timeout=2)
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(n for n, bit in self.REASONS.items() if self.reasons & bit),
                "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x: float, pg, device) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def morton_table(b, device):
    import torch
    idx = torch.arange(b, device=device)
    m = torch.zeros((b, b, b), dtype=torch.int64, device=device)
    for bit in range(10):
        m |= ((idx[None, None, :] >> bit) & 1) << (3 * bit)
        m |= ((idx[None, :, None] >> bit) & 1) << (3 * bit + 1)
        m |= ((idx[:, None, None] >> bit) & 1) << (3 * bit + 2)
    return m


def check_against_volume(out, off, vol, b):
    """Full-resolution bricks at out[off...] (split order, Morton inside) equal the source volume."""
    import torch
    D, H, W = vol.shape
    nbx, nby, nbz = -(-W // b), -(-H // b), -(-D // b)
    m = morton_table(b, vol.device)
    col =nby * nbz * b ** 3  # one column of bricks at fixed bx (by outer, bz inner)
    for bx in range(nbx):
        bricks = out[off + bx * col: off + (bx + 1) * col].view(nby, nbz, b ** 3)[:, :, m]  # (by, bz, z, y, x)
        grid = bricks.permute(1, 2, 0, 3, 4).reshape(nbz * b, nby * b, b)
        src = vol[:, :, bx * b:(bx + 1) * b]
        if not torch.equal(grid[:D, :H, :src.shape[2]], src):
            return False
    return True


def image_bricks(img: bytes):
    """(nSymbols, E) per brick of a .csbd image."""
    import struct
    nb = struct.unpack_from("<I", img, 8)[0]
    o, ns = 152, []
    for _ in range(nb):
        P = struct.unpack_from("<I", img, o + 4)[0]
        o += 8 + 8 * P
        E = struct.unpack_from("<I", img, o)[0]
        o += 4 + E
        ns.append(struct.unpack_from("<I", img, o)[0])
        o += 4
    return nb, ns


def encode_to_host(codec, vol, b):
    import torch
    codec.encode_device(vol, b)
    torch.cuda.synchronize()
    return bytes(codec.encoded_image_tensor().cpu().numpy())


def time_encode(codec, vol, b, reps=3):
    import torch
    s = torch.cuda.current_stream()
    codec.encode_device(vol, b)
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        codec.encode_device(vol, b)
        e1.record(s)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return min(ts)


def run_b200(args):
    import ctypes as C

    import torch
    from csvb200 import Codec, requests, requests_tensor

    world, rank, local, pg = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    codec = Codec(local)
    W = WORKLOADS[args.workload]
    D, H, Wd = W["shape"]
    nvox = D * H * Wd
    sx = W["split_x"]
    bl, br = W["brick_left"], W["brick_right"]

    # ---- workload: generate, encode both halves on the GPU, open, concatenate
    vol = torch.empty(W["shape"], dtype=torch.int64, device=dev)
    codec.synth_volume(vol, W["kind"], W["n_cells"], W["n_tubes"], W["r_min"], W["r_max"], W["zero_frac"], W["seed"])
    left = vol[:, :, :sx].contiguous()
    right = vol[:, :, sx:].contiguous()
    enc_ms_left = time_encode(codec, left, bl)
    img_left = encode_to_host(codec, left, bl)
    ds_left = codec.open_encoded()
    enc_ms_right = time_encode(codec, right, br)
    img_right = encode_to_host(codec, right, br)
    ds_right = codec.open_encoded()
    cat = codec.concat([ds_left, ds_right])
    nl, nr = ds_left.num_bricks, ds_right.num_bricks
    n = nl + nr
    lods = np.array([bl.bit_length() - 1] * nl + [br.bit_length() - 1] * nr)
    sizes = 8 ** lods.astype(np.uint64)
    dst = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    d_reqs = requests_tensor(requests(np.arange(n), lods, dst), dev)
    out = torch.empty(int(sizes.sum()), dtype=torch.int64, device=dev)
    status = torch.zeros(n, dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    # ---- autotune (grid, staging, order), capture the winner, check it
    if args.config:
        from csvb200 import DecodeConfig
        best, tune_ms = DecodeConfig(*[int(v) for v in args.config.split(",")]), 0.0
    else:
        best, tune_ms = codec.autotune(cat, d_reqs, out, status, reps=3)
    graph = codec.decode_graph(cat, d_reqs, out, status, best)
    kernels_per_step = graph.kernels  # decode kernels in one replay
    graph.launch()
    torch.cuda.synchronize()
    assert int(status.abs().max()) == 0, "decode status"
    check = (check_against_volume(out, 0, left, bl) and check_against_volume(out, nl * bl ** 3, right, br))
    del left, right
    # several GPUs: each rank decodes its own contiguous range of the requests, about 1/N of the voxels
    # (strong scaling: the whole workload is fixed; bricks are independent, so no collective)
    lo, hi = 0, n
    if world > 1:
        from csvb200.dist import voxel_ranges
        lo, hi = voxel_ranges(sizes, world)[rank]
        graph.close()
        d_reqs_r = d_reqs.view(n, 16)[lo:hi].reshape(-1).contiguous()
        status_r = status[lo:max(hi, lo + 1)]
        if args.config:
            best_r = best
        else:
            best_r, tune_ms = codec.autotune(cat, d_reqs_r, out, status_r, reps=3)
        graph = codec.decode_graph(cat, d_reqs_r, out, status_r, best_r)
        kernels_per_step = graph.kernels
        best = best_r

    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        flush.add_(1)
        graph.launch()
    torch.cuda.synchronize()
    clk = Clocks(local)
    barrier(pg)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush.add_(1)  # 256 MiB: the L2 holds nothing of the previous step
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        graph.launch(stream)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    barrier(pg)
    clocks = clk.stop()
    ms = statistics.mean(times)
    ms_max = max_over_ranks(ms, pg, dev)
    value = nvox / (ms_max * 1e-3) / 1e9  # the whole volume, decoded by all ranks together
    info = cat.info
    alg_bytes = info.stream_bytes + 8 * info.palette_entries + 16 * n + 8 * int(sizes.sum())
    if world > 1:  # this rank's share of the algorithmic bytes (its streams and palettes, its outputs)
        E_all = np.concatenate([image_stats(img_left)[0], image_stats(img_right)[0]])
        P_all = np.concatenate([image_stats(img_left)[1], image_stats(img_right)[1]])
        alg_bytes = int(E_all[lo:hi].sum() + 8 * P_all[lo:hi].sum()) + 16 * (hi - lo) + 8 * int(sizes[lo:hi].sum())
    hbm, hbm_kind = peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9

    # ---- end to end through the C ABI with host buffers: both images, open + seek index + decode + D2H
    per_img = [(img_left, bl, nl), (img_right, br, nr)]
    first = [0, nl]  # global request index of each image's first brick here
    if world > 1:  # this rank's bricks of each image (sub_image keeps header and model)
        from csvb200.dist import sub_image
        parts = [(sub_image(img_left, min(lo, nl), min(hi, nl)), bl, min(hi, nl) - min(lo, nl), min(lo, nl)),
                 (sub_image(img_right, max(lo, nl) - nl, max(hi, nl) - nl), br, max(hi, nl) - max(lo, nl),
                  max(lo, nl))]
        parts = [p for p in parts if p[2] > 0]
        per_img = [p[:3] for p in parts]
        first = [p[3] for p in parts]
    h_outs = [torch.empty((nb_, b_ ** 3), dtype=torch.int64, pin_memory=True) for _, b_, nb_ in per_img]
    h_st = [np.zeros(nb_, np.uint32) for _, _, nb_ in per_img]
    host_imgs = [np.frombuffer(im, np.uint8) for im, _, _ in per_img]
    # one host thread and one context per file (ctypes releases the GIL): one file's open and seek-index
    # pass overlaps the other's copy to the host, as a viewer loading both halves would run them
    from concurrent.futures import ThreadPoolExecutor
    ctxs = [codec, Codec(local)]

    def decode_file(j):
        im, b_, nb_ = per_img[j]
        c = ctxs[j]
        rc = c.lib.csv_decode_image(c.handle, host_imgs[j].ctypes.data_as(C.POINTER(C.c_uint8)), len(im),
                                    b_.bit_length() - 1, C.cast(h_outs[j].data_ptr(), C.POINTER(C.c_uint64)),
                                    h_st[j].ctypes.data_as(C.POINTER(C.c_uint32)))
        assert rc == 0, c.lib.csv_last_error(c.handle)

    e2e_ms = []
    with ThreadPoolExecutor(max_workers=len(per_img)) as ex:
        for k in range(16):  # one warm-up, fifteen timed: the median (host copies share the machine's PCIe and memory)
            barrier(pg)
            t0 = time.perf_counter()
            list(ex.map(decode_file, range(len(per_img))))
            t1 = time.perf_counter()
            if k > 0:
                e2e_ms.append((t1 - t0) * 1e3)
    e2e_t = max_over_ranks(statistics.median(e2e_ms), pg, dev)
    e2e_ok = all(bool(torch.equal(h_outs[j].view(-1).to(dev),
                                  out[int(dst[first[j]]): int(dst[first[j]]) + per_img[j][2] * per_img[j][1] ** 3]))
                 for j in range(len(per_img)))
    e2e = {"value": round(nvox / (e2e_t * 1e-3) / 1e9, 3), "unit": "Gvox/s",
           "h2d_bytes_per_step": len(img_left) + len(img_right), "d2h_bytes_per_step": 8 * nvox + 4 * n,
           "ms_per_step": round(e2e_t, 2), "ms_samples": [round(t, 1) for t in e2e_ms],
           "path": "csv_decode_image per image, the two images on two host threads and contexts: host .csbd -> "
                   "open (H2D, seek index) -> decode -> D2H labels"}
    del h_outs, ctxs

    # ---- cold open: csv_open of each image from host bytes (H2D of the image + the seek-index pass, which a
    # file the reference encoder wrote needs; an image from the GPU encoder carries its index)
    # index_ms: the device time of the seek-index passes inside that open (CUDA events around them); the
    # sidecar figures open the same bytes with the image's index sidecar (csv_open_indexed)
    cold_open = {"index_ms": {}, "sidecar_ms": {}, "sidecar_index_ms": {}, "sidecar_bytes": {}}
    for name_, im_ in (("32^3", img_left), ("64^3", img_right)):
        ts_, ix_ = [], []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d_ = codec.open(im_)
            torch.cuda.synchronize()
            ts_.append((time.perf_counter() - t0) * 1e3)
            ix_.append(d_.index_ms)
            if _ == 0:
                sc_ = d_.index_sidecar()
            d_.close()
        cold_open[name_] = round(min(ts_), 2)
        cold_open["index_ms"][name_] = round(min(ix_), 3)
        ts_, ix_ = [], []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d_ = codec.open(im_, sidecar=sc_)
            torch.cuda.synchronize()
            ts_.append((time.perf_counter() - t0) * 1e3)
            ix_.append(d_.index_ms)
            d_.close()
        cold_open["sidecar_ms"][name_] = round(min(ts_), 2)
        cold_open["sidecar_index_ms"][name_] = round(min(ix_), 3)
        cold_open["sidecar_bytes"][name_] = len(sc_)

    # ---- neurite512: encode vs the reference encoder on this host, and its decode
    neur = neurite512(codec, dev, args, rank == 0 and world == 1 and not args.no_cpu)

    # ---- serve2048: the frame loop (plan, cache, decode, render) over a 600-frame orbit
    graph.close()
    del out, vol, flush
    torch.cuda.empty_cache()
    dense = None if (args.no_dense or W["name"] != "mixed1024") else dense_leg(codec, dev, args)
    torch.cuda.empty_cache()
    serve = None if args.no_serve else serve2048(codec, dev, args)
    torch.cuda.empty_cache()
    selector = None if args.no_selector else selector1024(codec, dev, args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_decode_sample(img_left, img_right, bl, br)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Gvox/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": workload_config(W, nl, nr, [img_left, img_right]),
            "decode": {"launch": "one CUDA graph (csv_decode_graph)", "decode_config": best.as_dict(),
                       "ranks": world, "requests_rank0": [lo, hi],
                       "autotuned": not args.config, "autotune_ms": round(tune_ms, 4),
                       "device_stream_bytes": info.stream_bytes},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4),
                         "traffic": load_traffic("decode_kernel", W["name"]) if world == 1 else None,
                         "algorithmic_bytes": alg_bytes, "peak_kind": hbm_kind},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps * kernels_per_step,
            "clocks": clocks,
            "encode": {"value": round(nvox / ((enc_ms_left + enc_ms_right) * 1e-3) / 1e6, 1), "unit": "Mvox/s",
                       "ms": round(enc_ms_left + enc_ms_right, 3), "workload": W["name"]},
            "cold_open_ms": cold_open,
            "dense": dense,
            "neurite512": neur,
            "serve2048": serve,
            "selector1024": selector,
            "checks": {"decode_equals_source": check, "e2e_equals_device": e2e_ok},
        }
        print(json.dumps(line))
    cat.close()
    ds_left.close()
    ds_right.close()
    if pg is not None:
        pg.destroy_process_group()


def dense_leg(codec, dev, args):
    """The uneven batch with the dense half at the stream sizes configs[2] describes (mixed1024dense): the same
    one-graph decode with the autotuner's configuration, its throughput, HBM fraction and stream histogram."""
    import torch
    from csvb200 import requests, requests_tensor
    W = MIXED_DENSE
    sx, bl, br = W["split_x"], W["brick_left"], W["brick_right"]
    vol = torch.empty(W["shape"], dtype=torch.int64, device=dev)
    codec.synth_volume(vol, W["kind"], W["n_cells"], W["n_tubes"], W["r_min"], W["r_max"], W["zero_frac"], W["seed"])
    left, right = vol[:, :, :sx].contiguous(), vol[:, :, sx:].contiguous()
    del vol
    img_l = encode_to_host(codec, left, bl)
    dl = codec.open_encoded()
    img_r = encode_to_host(codec, right, br)
    dr = codec.open_encoded()
    cat = codec.concat([dl, dr])
    nl, nr = dl.num_bricks, dr.num_bricks
    n = nl + nr
    lods = np.array([bl.bit_length() - 1] * nl + [br.bit_length() - 1] * nr)
    sizes = 8 ** lods.astype(np.uint64)
    dst = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    d_reqs = requests_tensor(requests(np.arange(n), lods, dst), dev)
    out = torch.empty(int(sizes.sum()), dtype=torch.int64, device=dev)
    status = torch.zeros(n, dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    best, _ = codec.autotune(cat, d_reqs, out, status, reps=3)
    g = codec.decode_graph(cat, d_reqs, out, status, best)
    g.launch()
    torch.cuda.synchronize()
    ok = int(status.abs().max()) == 0 and check_against_volume(out, 0, left, bl) and \
        check_against_volume(out, nl * bl ** 3, right, br)
    del left, right
    st = torch.cuda.current_stream()
    for _ in range(args.warmup):
        flush.add_(1)
        g.launch()
    ts = []
    for _ in range(args.steps):
        flush.add_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        g.launch(st)
        e1.record(st)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = statistics.mean(ts)
    info = cat.info
    alg = info.stream_bytes + 8 * info.palette_entries + 16 * n + 8 * int(sizes.sum())
    hbm, kind = peaks()
    nvox = int(sizes.sum())
    res = {"workload": W["name"], "tubes": W["n_tubes"], "radius": [W["r_min"], W["r_max"]],
           "value": round(nvox / (ms * 1e-3) / 1e9, 3), "unit": "Gvox/s", "ms_per_step": round(ms, 4),
           "roofline": {"achieved": round(alg / (ms * 1e-3) / 1e9, 1), "peak": hbm, "frac": round(alg / (ms * 1e-3) / 1e9 / hbm, 4),
                        "peak_kind": kind, "algorithmic_bytes": alg},
           "streams": stream_histogram([img_l, img_r]), "decode_config": best.as_dict(), "decode_equals_source": ok,
           "note": "headline is mixed1024: its tube half uses the stated 5000 splines of radius 1-4; this leg raises "
                   "the tube count until the 64^3 streams span what configs[2] describes"}
    g.close()
    cat.close()
    dl.close()
    dr.close()
    return res


def selector_leg(codec, dev, args, train_vol, held_vol, train_desc, held_desc):
    """Learned mode / table selector: trained on the 64^3 bricks of SELECTOR["train_volumes"] seeded volumes
    (train_vol(k) fills and returns the k-th), evaluated on a held-out volume (held_vol()) against the
    exhaustive search (every mode's statistics) and the plain encoder.  The trained tables and network go
    through a selector file (csv_selector_write / csv_selector_read) and the learned encode runs as the one
    call csv_encode_learned; its features / network / encode split is timed apart."""
    import tempfile

    import torch
    from csvb200 import SelectorNet
    from csvb200.selector import exhaustive_choice, features, fit_tables, learned_choice, train
    st = torch.cuda.current_stream()

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(st)
        return e

    t0 = time.perf_counter()
    feats, hists = [], []
    for k in range(SELECTOR["train_volumes"]):
        vol = train_vol(k)
        feats.append(features(codec, vol, 64))
        h = torch.empty((feats[-1].shape[0], 12, 16), dtype=torch.int32, device=dev)
        codec.encode_stats(vol, 64, h)
        hists.append(h)
        del vol
    tables = fit_tables(torch.cat(hists).cpu().numpy().astype(np.uint64), 16, iters=8)
    labels = []
    for h in hists:
        sel = torch.empty(h.shape[0], dtype=torch.uint8, device=dev)
        codec.select_exhaustive(h, tables, sel)
        labels.append(sel)
    data_s = time.perf_counter() - t0
    e0 = ev()
    net0, losses = train(codec, torch.cat(feats), torch.cat(labels), steps=SELECTOR["steps"], batch=2048)
    e1 = ev()
    torch.cuda.synchronize()
    train_ms = e0.elapsed_time(e1)
    # the trained selector through a file: what a learned encode outside this process loads
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "selector.csvs")
        net0.save(path, tables)
        file_bytes = os.path.getsize(path)
        net, tables_f = SelectorNet.load(codec, path)
    net0.close()
    assert np.array_equal(tables_f, tables)
    held = held_vol()
    nvox = held.numel()
    res, split = {}, {}
    for rep in range(2):  # warm, then timed
        a = ev()
        codec.encode_device_sel(held, 64)
        b = ev()
        plain = codec.encoded_image()[1]
        c = ev()
        sel_x, _ = exhaustive_choice(codec, held, 64, tables)
        codec.encode_device_sel(held, 64, tables, sel_x)
        d = ev()
        exh = codec.encoded_image()[1]
        e = ev()
        codec.encode_learned(held, 64, net, tables)  # csv_encode_learned: the one call
        f = ev()
        learned = codec.encoded_image()[1]
        # the same three steps apart: features, the network's choice, the version-2 encode
        g = ev()
        fe = features(codec, held, 64)
        h_ = ev()
        sel_l = learned_choice(net, fe)
        i_ = ev()
        codec.encode_device_sel(held, 64, tables, sel_l)
        j_ = ev()
        torch.cuda.synchronize()
        res = {"plain_ms": a.elapsed_time(b), "exhaustive_ms": c.elapsed_time(d), "learned_ms": e.elapsed_time(f)}
        split = {"features_ms": round(g.elapsed_time(h_), 3), "network_ms": round(h_.elapsed_time(i_), 3),
                 "encode_v2_ms": round(i_.elapsed_time(j_), 3)}
    agree = float((sel_x == sel_l).float().mean())
    # the network alone on the tensor cores: one forward pass over 1 Mi feature rows
    rows = 1 << 20
    big = torch.rand((rows, 32), device=dev)
    logits = torch.empty((rows, 32), device=dev)
    net.forward(big, d_logits=logits)
    g0 = ev()
    for _ in range(5):
        net.forward(big, d_logits=logits)
    g1 = ev()
    torch.cuda.synchronize()
    fwd_ms = g0.elapsed_time(g1) / 5
    flops = 2.0 * rows * (64 * 256 + 256 * 256 + 256 * 32)
    peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("bf16_tflops") if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else 1590.0
    out = {
        "train": {"volumes": SELECTOR["train_volumes"], "bricks": int(sum(f.shape[0] for f in feats)),
                  "generator": train_desc, "tables": 16, "modes": 12, "steps": SELECTOR["steps"], "batch": 2048,
                  "train_ms": round(train_ms, 1), "loss_first": round(losses[0], 4),
                  "loss_last": round(float(np.mean(losses[-20:])), 4), "data_s": round(data_s, 2),
                  "selector_file_bytes": file_bytes},
        "held_out": {"volume": list(held.shape[::-1]), "bricks": int(sel_x.numel()), "generator": held_desc},
        "bytes": {"plain": int(plain), "exhaustive": int(exh), "learned": int(learned)},
        "size_loss_vs_exhaustive": round(learned / exh - 1.0, 5),
        "size_vs_plain": round(learned / plain - 1.0, 5),
        "exhaustive_vs_plain": round(exh / plain - 1.0, 5),
        "choice_agreement": round(agree, 4),
        "encode_ms": {k: round(v, 2) for k, v in res.items()},
        "learned_split": split,
        "learned_vs_plain_time": round(res["learned_ms"] / res["plain_ms"], 3),
        "encode_mvox_s": {k[:-3]: round(nvox / (v * 1e-3) / 1e6, 1) for k, v in res.items()},
        "speedup_vs_exhaustive": round(res["exhaustive_ms"] / res["learned_ms"], 2),
        "mlp_forward": {"rows": rows, "ms": round(fwd_ms, 3), "tflops": round(flops / (fwd_ms * 1e-3) / 1e12, 1),
                        "frac_of_bf16_peak": round(flops / (fwd_ms * 1e-3) / 1e12 / peak, 4)},
        "decode": "version-2 image decodes to the same labels as the plain image (tests)",
    }
    net.close()
    del held
    torch.cuda.empty_cache()
    return out


def selector1024(codec, dev, args):
    """The selector on two generators: the neurite-like volumes (trained on 40 x 512^3, held out 1024^3) and the
    uneven batch's dense half (64^3 tube bricks: trained on the x >= 256 halves of 40 mixed512 volumes, held out
    the x >= 512 half of the mixed1024 volume the decode headline uses)."""
    import torch
    N, M, M5 = NEURITE, MIXED, MIXED512

    def neur_train(k):
        v = torch.empty(N["shape"], dtype=torch.int64, device=dev)
        codec.synth_volume(v, N["kind"], N["n_cells"], N["n_tubes"], N["r_min"], N["r_max"], N["zero_frac"],
                           SELECTOR["seed"] + k)
        return v

    def neur_held():
        v = torch.empty((1024, 1024, 1024), dtype=torch.int64, device=dev)
        codec.synth_volume(v, N["kind"], N["n_cells"] * 8, N["n_tubes"] * 8, N["r_min"], N["r_max"], N["zero_frac"],
                           SELECTOR["seed"] + 1000)
        return v

    def mixed_train(k):
        v = torch.empty(M5["shape"], dtype=torch.int64, device=dev)
        codec.synth_volume(v, M5["kind"], M5["n_cells"], M5["n_tubes"], M5["r_min"], M5["r_max"], M5["zero_frac"],
                           SELECTOR["seed"] + 2000 + k)
        return v[:, :, M5["split_x"]:].contiguous()

    def mixed_held():
        v = torch.empty(M["shape"], dtype=torch.int64, device=dev)
        codec.synth_volume(v, M["kind"], M["n_cells"], M["n_tubes"], M["r_min"], M["r_max"], M["zero_frac"], M["seed"])
        return v[:, :, M["split_x"]:].contiguous()

    out = selector_leg(codec, dev, args, neur_train, neur_held,
                       "neurite512 (400 tubes r 2-12, 3000 cells, 15 % 0), 40 seeds",
                       "neurite512 scaled x8 (3200 tubes, 24000 cells), 1024^3")
    out["mixed1024_tubes"] = selector_leg(codec, dev, args, mixed_train, mixed_held,
                                          "mixed512 x >= 256 halves (625 tubes r 1-4 over 250 cells), 40 seeds",
                                          "mixed1024 x >= 512 half (the decode headline's 64^3 image)")
    return out


def orbit_path(n, center, seed, scale=1.0):
    """Seeded orbit with zoom (orbitController.js:100-123 camera placement): two turns, pitch swinging
    +-0.35 rad, radius 1600..3600 voxels (times scale, for smaller volumes), small seeded jitter on every
    frame."""
    import math
    from csvb200.camera import orbit
    rng = np.random.default_rng(seed)
    jit = rng.normal(0.0, 1.0, (n, 3))
    views = []
    for f in range(n):
        t = f / n
        yaw = 2 * math.pi * 2 * t + 0.01 * jit[f, 0]
        pitch = 0.35 * math.sin(2 * math.pi * 3 * t) + 0.01 * jit[f, 1]
        radius = scale * (2600.0 + 1000.0 * math.cos(2 * math.pi * 1.5 * t) + 10.0 * jit[f, 2])
        views.append(orbit(center, radius, yaw, pitch))
    return views


def serve_mix(codec, ds, dev, S, views, admit=0):
    """Continuous batching on the serving workload: four sessions share one server and one cache; they join
    and leave mid-orbit (session 0 the whole orbit, session 1 frames 100-399, session 2 frames 200-499 on a
    second orbit, session 3 from frame 300 on a third), every open session submits a frame each step.  Each
    step is submitted, stepped and polled synchronously, so that the host wall time from the first submit to
    the poll that returns the step's frames is the latency a viewer sees; per session: p50/p99 of the device
    time of the steps it rendered in, and of that submit-to-poll latency."""
    import math

    import torch
    from csvb200 import CONE_SCREEN, Server
    Wp, Hp = S["width"], S["height"]
    n = len(views)
    c = [v / 2.0 for v in S["shape"][::-1]]
    others = [orbit_path(n, c, S["seed"] + 11 * k, scale=0.8 + 0.2 * k) for k in (1, 2, 3)]
    spans = [(0, n), (n // 6, 2 * n // 3), (n // 3, 5 * n // 6), (n // 2, n)]
    paths = [views] + others
    srv = Server(codec, ds, Wp, Hp, S["fov"], cache_bytes=S["cache_gib"] << 30, max_sessions=4, cone=CONE_SCREEN,
                 admit=admit)
    bufs = [(torch.empty(Wp * Hp, dtype=torch.int64, device=dev), torch.empty(Wp * Hp, dtype=torch.float32,
                                                                              device=dev)) for _ in range(4)]
    st = torch.cuda.current_stream()
    dev_ms = {k: [] for k in range(4)}
    lat_ms = {k: [] for k in range(4)}
    joined, left, rebuilds, open_max = 0, 0, 0, 0
    was_open = [False] * 4
    torch.cuda.synchronize()
    for f in range(n):
        t0 = time.perf_counter()
        now_open = [lo <= f < hi for lo, hi in spans]
        for k in range(4):
            if was_open[k] and not now_open[k]:
                srv.leave(k)
                left += 1
            if now_open[k]:
                joined += not was_open[k]
                pos, d = paths[k][f]
                srv.submit(k, pos, d, *bufs[k])
        was_open = now_open
        open_max = max(open_max, sum(now_open))
        srv.step(st)
        frames = srv.poll(wait=True)
        t1 = time.perf_counter()
        for fr in frames:
            dev_ms[fr["session"]].append(fr["ms"])
            lat_ms[fr["session"]].append((t1 - t0) * 1e3)
        rebuilds += frames[0]["rebuilt"] if frames else 0
    srv.close()

    def pct(a, q):
        return round(float(np.percentile(np.array(a), q)), 3) if a else None

    per = {str(k): {"frames": len(dev_ms[k]), "span": list(spans[k]), "p50_ms": pct(dev_ms[k], 50),
                    "p99_ms": pct(dev_ms[k], 99), "submit_to_poll_p50_ms": pct(lat_ms[k], 50),
                    "submit_to_poll_p99_ms": pct(lat_ms[k], 99)} for k in range(4)}
    every = [x for k in range(4) for x in dev_ms[k]]
    lat = [x for k in range(4) for x in lat_ms[k]]
    return {"sessions": per, "joins": joined, "leaves": left, "open_max": open_max, "rebuilds": rebuilds,
            "admit": "rays" if admit else "cone",
            "p99_ms_all": pct(every, 99), "submit_to_poll_p99_ms_all": pct(lat, 99),
            "timing": "device time per step (CUDA events) and host wall time submit -> poll(wait), one step in "
                      "flight"}


def serve2048(codec, dev, args):
    """On-demand decode + render at 1920x1080 over a 2048^3 volume with a 24 GiB decoded-brick cache."""
    import math

    import torch
    from csvb200 import CONE_SCREEN, Server
    S = SERVE
    vol = torch.empty(S["shape"], dtype=torch.int64, device=dev)
    codec.synth_volume(vol, S["kind"], S["n_cells"], S["n_tubes"], S["r_min"], S["r_max"], S["zero_frac"], S["seed"])
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    img_len = codec.encode_device(vol, S["brick"])
    e1.record(st)
    torch.cuda.synchronize()
    enc_ms = e0.elapsed_time(e1)
    ds = codec.open_encoded()
    del vol
    torch.cuda.empty_cache()
    Wp, Hp = S["width"], S["height"]
    srv = Server(codec, ds, Wp, Hp, S["fov"], cache_bytes=S["cache_gib"] << 30, cone=CONE_SCREEN)
    lab = torch.empty(Wp * Hp, dtype=torch.int64, device=dev)
    dep = torch.empty(Wp * Hp, dtype=torch.float32, device=dev)
    c = [v / 2.0 for v in S["shape"][::-1]]
    views = orbit_path(S["frames"], c, S["seed"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record(st)
    for pos, d in views:
        srv.submit(0, pos, d, lab, dep)
        srv.step(st)
    b1.record(st)
    frames = srv.poll(wait=True, max_frames=len(views) + 8)
    wall = time.perf_counter() - t0
    total_ms = b0.elapsed_time(b1)
    ms = np.array([f["ms"] for f in frames])
    dec = np.array([f["decoded"] for f in frames])
    vox = np.array([f["decoded_voxels"] for f in frames])
    out = {
        "workload": S["name"], "volume": list(S["shape"][::-1]), "brick": S["brick"],
        "bricks": ds.num_bricks, "tubes": S["n_tubes"], "voronoi_cells": S["n_cells"],
        "radius": [S["r_min"], S["r_max"]], "zero_frac": S["zero_frac"], "seed": S["seed"],
        "image_bytes": int(img_len), "encode_ms": round(enc_ms, 2),
        "resolution": [Wp, Hp], "frames": len(frames), "cache_gib": S["cache_gib"], "cone": "screen",
        "path": "seeded orbit with zoom, radius 1600-3600, 2 turns",
        "p50_ms": round(float(np.percentile(ms, 50)), 3), "p99_ms": round(float(np.percentile(ms, 99)), 3),
        "max_ms": round(float(ms.max()), 3), "first_frame_ms": round(float(ms[0]), 3),
        "mean_ms": round(float(ms.mean()), 3), "loop_ms": round(total_ms, 2),
        "host_wall_s": round(wall, 3),
        "decoded_bricks": int(dec.sum()), "decoded_bricks_per_s": round(float(dec.sum()) / (ms.sum() * 1e-3), 1),
        "decoded_gvox": round(float(vox.sum()) / 1e9, 3),
        "missing_entered": int(sum(f["missing"] for f in frames)),
        "rebuilds": int(sum(f["rebuilt"] for f in frames)),
        "resident_blocks_last": int(frames[-1]["resident"]),
        "entered_bricks_mean": round(float(np.mean([f["entered"] for f in frames])), 1),
        "hit_pixels_last_frame": round(float((lab != 0).float().mean()), 4),
        "timing": "device time per step (CUDA events around plan, cache, decode, render, census)",
    }
    srv.close()
    # the same orbit with the viewer's RGBA frames (transfer function, shading, shadow rays), fresh cache
    del lab, dep
    torch.cuda.empty_cache()
    srv = Server(codec, ds, Wp, Hp, S["fov"], cache_bytes=S["cache_gib"] << 30, cone=CONE_SCREEN)
    rgba = torch.empty(Wp * Hp, dtype=torch.int32, device=dev)
    for pos, d in views:
        srv.submit_rgba(0, pos, d, rgba)
        srv.step(st)
    fr = srv.poll(wait=True, max_frames=len(views) + 8)
    ms2 = np.array([f["ms"] for f in fr])
    srv.close()
    # continuous batching: four sessions joining and leaving mid-orbit, cone admission and admission by rays
    torch.cuda.empty_cache()
    out["mix"] = serve_mix(codec, ds, dev, S, views, admit=0)
    out["mix_rays"] = serve_mix(codec, ds, dev, S, views, admit=1)
    out["rgba"] = {"p50_ms": round(float(np.percentile(ms2, 50)), 3), "p99_ms": round(float(np.percentile(ms2, 99)), 3),
                   "max_ms": round(float(ms2.max()), 3), "mean_ms": round(float(ms2.mean()), 3),
                   "entered_bricks_mean": round(float(np.mean([f["entered"] for f in fr])), 1),
                   "visible_pixels_last_frame": round(float(((rgba >> 24) != 0).float().mean()), 4),
                   "lighting": "csv_lighting_default(25): ambient 0.5, diffuse 0.8",
                   "timing": "device time per step, frames RGBA8 through csv_render_rgba's colour path"}
    srv.close()
    ds.close()
    torch.cuda.empty_cache()
    return out


def neurite512(codec, dev, args, with_cpu):
    """GPU encode (timed), bytes vs the reference encoder, full-resolution decode throughput."""
    import torch
    from csvb200 import requests, requests_tensor
    W = NEURITE
    b = W["brick"]
    vol = torch.empty(W["shape"], dtype=torch.int64, device=dev)
    codec.synth_volume(vol, W["kind"], W["n_cells"], W["n_tubes"], W["r_min"], W["r_max"], W["zero_frac"], W["seed"])
    nvox = vol.numel()
    enc_ms = time_encode(codec, vol, b)
    image = encode_to_host(codec, vol, b)
    ds = codec.open_encoded()
    nb = ds.num_bricks
    per = b ** 3
    d_reqs = requests_tensor(requests(np.arange(nb), np.full(nb, 6), np.arange(nb, dtype=np.uint64) * per), dev)
    out = torch.empty(nb * per, dtype=torch.int64, device=dev)
    st = torch.zeros(nb, dtype=torch.int32, device=dev)
    graph = codec.decode_graph(ds, d_reqs, out, st)
    graph.launch()
    torch.cuda.synchronize()
    ok = check_against_volume(out, 0, vol, b)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    ts = []
    s = torch.cuda.current_stream()
    for k in range(args.warmup + 20):
        flush.add_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        graph.launch(s)
        e1.record(s)
        e1.synchronize()
        if k >= args.warmup:
            ts.append(e0.elapsed_time(e1))
    dec_ms = statistics.mean(ts)
    res = {"volume": list(W["shape"][::-1]), "bricks": nb, "brick": b, "tubes": W["n_tubes"],
           "radius": [W["r_min"], W["r_max"]], "voronoi_cells": W["n_cells"], "zero_frac": W["zero_frac"],
           "decode_gvox_s": round(nvox / (dec_ms * 1e-3) / 1e9, 2), "decode_ms": round(dec_ms, 4),
           "decode_equals_source": ok, "encode_mvox_s": round(nvox / (enc_ms * 1e-3) / 1e6, 1),
           "encode_ms": round(enc_ms, 3), "image_bytes": len(image)}
    graph.close()
    ds.close()
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import REF_SO, Oracle, Reference
        vol_np = vol.cpu().numpy().view(np.uint64)
        del vol
        if os.path.exists(REF_SO):
            t0 = time.perf_counter()
            ref_img = Reference().encode(vol_np, b)
            kind = "reference"
        else:
            t0 = time.perf_counter()
            ref_img = Oracle().encode(vol_np, b)
            kind = "port"
        cpu_s = time.perf_counter() - t0
        res["cpu_encode"] = {"kind": kind, "cores": 1, "seconds": round(cpu_s, 3),
                             "mvox_s": round(nvox / cpu_s / 1e6, 2),
                             "sample": "whole neurite512 volume: splitGridIntoBricks + compressDataset + "
                                       "saveDatasetToFile, 1 thread"}
        res["encode_speedup_vs_cpu"] = round(res["encode_mvox_s"] / res["cpu_encode"]["mvox_s"], 1)
        res["bytes_identical_to_reference"] = ref_img == image
    return res


def cpu_decode_sample(img_left, img_right, bl, br, n_left=2048, n_right=256):
    """The reference decoder (decodeRansStream + decodeBrick<b>, 1 thread) on the first bricks of each image."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import REF_SO, Oracle, Reference
    if os.path.exists(REF_SO):
        R = Reference()
        t0 = time.perf_counter()
        _, st1, _ = R.decode_all_full(img_left, bl, max_bricks=n_left, keep=False)
        _, st2, _ = R.decode_all_full(img_right, br, max_bricks=n_right, keep=False)
        s = time.perf_counter() - t0
        kind = "reference"
    else:
        O = Oracle()
        t0 = time.perf_counter()
        O.decode_image(img_left, bl.bit_length() - 1)
        O.decode_image(img_right, br.bit_length() - 1)
        s = time.perf_counter() - t0
        kind, n_left, n_right = "port", image_bricks(img_left)[0], image_bricks(img_right)[0]
    vox = n_left * bl ** 3 + n_right * br ** 3
    return {"value": round(vox / s / 1e9, 5), "unit": "Gvox/s", "cores": 1, "kind": kind,
            "sample": f"{n_left} 32^3 bricks + {n_right} 64^3 bricks of the mixed1024 images at full resolution "
                      f"({vox} voxels), decodeRansStream + decodeBrick<b>, 1 thread",
            "seconds": round(s, 3)}


def load_traffic(kernel: str, workload: str):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(kernel, {}).get(workload)


def image_stats(img: bytes):
    """Per brick of a .csbd v1 image: encoded stream bytes E and palette entries P."""
    import struct
    nb = struct.unpack_from("<I", img, 8)[0]
    o, E, P = 152, [], []
    for _ in range(nb):
        p = struct.unpack_from("<I", img, o + 4)[0]
        o += 8 + 8 * p
        e = struct.unpack_from("<I", img, o)[0]
        o += 8 + e
        E.append(e)
        P.append(p)
    return np.array(E, np.int64), np.array(P, np.int64)


def stream_histogram(images):
    """Encoded stream sizes and palette sizes over the bricks of the given images: power-of-two bins of E."""
    E = np.concatenate([image_stats(im)[0] for im in images])
    P = np.concatenate([image_stats(im)[1] for im in images])
    edges = [0, 64, 256, 1024, 4096, 16384, 65536, 131072, 262144, 1 << 40]
    names = ["<64B", "64-256B", "256B-1K", "1-4K", "4-16K", "16-64K", "64-128K", "128-256K", ">=256K"]
    cnt = np.histogram(E, bins=edges)[0]
    return {"bricks_by_stream_bytes": {k: int(c) for k, c in zip(names, cnt)},
            "stream_bytes_min": int(E.min()), "stream_bytes_median": int(np.median(E)), "stream_bytes_max": int(E.max()),
            "palette_max": int(P.max()), "palette_median": int(np.median(P))}


def workload_config(W, nl, nr, images):
    """The config object both arms print: the workload, its sizes and the measured stream-size distribution."""
    D, H, Wd = W["shape"]
    return {"workload": W["name"], "volume": [Wd, H, D],
            "bricks": {"32^3": nl, "64^3": nr, "split_x": W["split_x"]},
            "left": f"Voronoi {W['n_cells']} cells, {W['brick_left']}^3 bricks",
            "right": f"{W['n_tubes']} tubes r {W['r_min']}-{W['r_max']} over it, {W['brick_right']}^3 bricks",
            "lod": "full resolution", "seed": W["seed"],
            "stream_bytes": int(sum(int(image_stats(im)[0].sum()) for im in images)),
            "image_bytes": [len(im) for im in images],
            "streams": stream_histogram(images),
            "l2": "flushed between timed steps (256 MiB buffer); inputs and outputs larger than L2",
            "parallelism": "bricks independent, no collective"}


def run_reference(args):
    """The reference's own CPU decoder (oracle/_ref: decodeRansStream + decodeBrick<b>) on every host thread.

    The input images are built without the product library: the workload generator restated on the CPU
    (oracle or_synth_volume, the same volume as csv_synth_volume) and encoded by the oracle's threaded
    encoder (the same bytes as the reference encoder and the GPU encoder).  Only oracle/ libraries load."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import REF_SO, Oracle, Reference
    W = WORKLOADS[args.workload]
    D, H, Wd = W["shape"]
    sx = W["split_x"]
    bl, br = W["brick_left"], W["brick_right"]
    O = Oracle()
    t0 = time.perf_counter()
    vol = O.synth_volume(W["shape"], W["kind"], W["n_cells"], W["n_tubes"], W["r_min"], W["r_max"], W["zero_frac"],
                         W["seed"])
    img_left = O.encode_threads(np.ascontiguousarray(vol[:, :, :sx]), bl)
    img_right = O.encode_threads(np.ascontiguousarray(vol[:, :, sx:]), br)
    del vol
    prep_s = time.perf_counter() - t0
    nl, nr = image_bricks(img_left)[0], image_bricks(img_right)[0]
    threads = os.cpu_count() or 1
    if os.path.exists(REF_SO):
        R = Reference()
        kind = "reference"

        def step(stride):
            # decodeBrick throws on a brick whose root stop bit is set (the whole brick one label): the
            # reference decodes nothing there; such bricks are counted, not fatal
            return R.decode_parallel(img_left, threads, stride=stride) + \
                R.decode_parallel(img_right, threads, stride=stride)
    else:
        kind, threads = "port", 1

        def step(stride):
            O.decode_image(img_left, bl.bit_length() - 1)
            O.decode_image(img_right, br.bit_length() - 1)
            return 0
    # the first warm-up step sizes the sample: every stride-th brick, so that the remaining warm-up and
    # timed steps take about a minute in all
    t1 = time.perf_counter()
    step(1)
    full_s = time.perf_counter() - t1
    budget_s = 60.0
    stride = max(1, int(np.ceil(full_s * (args.steps + args.warmup - 1) / budget_s)))
    for _ in range(args.warmup - 1):
        step(stride)
    times = []
    thrown = 0
    for _ in range(args.steps):
        t1 = time.perf_counter()
        thrown = step(stride)
        times.append(time.perf_counter() - t1)
    s = statistics.mean(times)
    nvox = len(range(0, nl, stride)) * bl ** 3 + len(range(0, nr, stride)) * br ** 3
    v = nvox / s / 1e9
    sample = (f"every step decodes {'all' if stride == 1 else f'every {stride}th of the'} {nl + nr} bricks of both "
              f"images at full resolution ({nvox} voxels; decodeRansStream + decodeBrick<b>), bricks split over "
              f"{threads} host threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "Gvox/s", "n_gpus": world,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": round(s * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": workload_config(W, nl, nr, [img_left, img_right]),
        "reference": {"bricks_thrown_per_step": int(thrown), "stride": stride, "input_build_s": round(prep_s, 1),
                      "inputs": "oracle CPU generator (= csv_synth_volume) + oracle threaded encoder (= the "
                                "reference encoder's bytes); no product library in this process",
                      "note": "the reference C++ decoder throws on bricks that are one label (root stop bit); "
                              "they are counted, and the GPU decoder fills them with palette[0]"},
        "cpu_baseline": {"value": round(v, 4), "unit": "Gvox/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": round(v, 4), "unit": "Gvox/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline legs")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop leg")
    ap.add_argument("--no-selector", action="store_true", help="skip the learned-selector leg")
    ap.add_argument("--no-dense", action="store_true", help="skip the dense uneven-batch leg")
    ap.add_argument("--config", default=None,
                    help="ctas_per_sm,stage,lpt,layout: use this decode configuration instead of the autotuner's "
                         "(a fixed launch sequence, for profiler captures)")
    ap.add_argument("--workload", default="mixed1024", choices=sorted(WORKLOADS),
                    help="mixed1024: the headline; mixed512: the same generator at 1/8 size (profiler captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
