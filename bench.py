"""Benchmark of the B200 compressed-segmentation-volume codec.

Headline (value): bit-exact batched brick decode throughput in Gvox/s, with
its %HBM roofline, on the neurite-like workload: a 512^3 uint64 volume of 400
cubic-spline tubes (radius 2-12 voxels) over a 3000-cell Voronoi background
with ~15% label 0, 64^3 bricks (512 bricks), every brick decoded at full
resolution.  One step = one csv_decode_batch launch over all 512 bricks from
the HBM-resident compressed dataset.  The same line carries the GPU encode
throughput (Mvox/s) next to the reference CPU encoder, and the end-to-end
number through the C ABI with host buffers.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU: one process per GPU (torchrun); every rank decodes its own copy of
the workload (bricks are independent; no collective on the data path), so
scaling is weak and value = all ranks' voxels / max-over-ranks time.
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
WORKLOAD = dict(name="neurite512_b64", shape=(512, 512, 512), brick=64, kind=1, n_cells=3000, n_tubes=400,
                r_min=2.0, r_max=12.0, zero_frac=0.15, seed=2)
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


def flush_l2(buf):
    buf.add_(1)  # 256 MiB read+write, larger than the 126 MB L2


def dist_setup(args):
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


def cpu_reference(vol_np: np.ndarray, brick: int, gpu_image: bytes):
    """The reference encoder and decoder on the host cores (1 thread: the reference is single-threaded)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import REF_SO, Oracle, Reference
    nvox = int(np.prod(vol_np.shape))
    if os.path.exists(REF_SO):
        R = Reference()
        t0 = time.perf_counter()
        img, tm = R.encode(vol_np, brick, timings=True)
        enc_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        _, st, dtm = R.decode_all_full(img, brick, keep=False)
        dec_s = time.perf_counter() - t0
        kind = "reference"
    else:
        O = Oracle()
        t0 = time.perf_counter()
        img = O.encode(vol_np, brick)
        enc_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.decode_image(img, brick.bit_length() - 1)
        dec_s = time.perf_counter() - t0
        kind = "port"
    return {"kind": kind, "encode_s": enc_s, "decode_s": dec_s, "encode_mvox_s": nvox / enc_s / 1e6,
            "decode_gvox_s": nvox / dec_s / 1e9, "bytes_identical": img == gpu_image}


def run_b200(args):
    import torch
    from csvb200 import Codec, requests, requests_tensor

    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    codec = Codec(local)
    W = WORKLOAD
    D, H, Wd = W["shape"]
    b = W["brick"]
    nvox = D * H * Wd
    vol = torch.empty(W["shape"], dtype=torch.int64, device=dev)
    codec.synth_volume(vol, W["kind"], W["n_cells"], W["n_tubes"], W["r_min"], W["r_max"], W["zero_frac"],
                       W["seed"])
    torch.cuda.synchronize()

    # ---- GPU encode (csv_encode_device), timed on its own
    stream = torch.cuda.current_stream()
    for _ in range(max(1, min(2, args.warmup))):
        img_len = codec.encode_device(vol, b)
    enc_ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        img_len = codec.encode_device(vol, b)
        e1.record(stream)
        torch.cuda.synchronize()
        enc_ms.append(e0.elapsed_time(e1))
    enc_ms_best = min(enc_ms)
    img_dev = codec.encoded_image_tensor()
    n = img_dev.numel()
    image = bytes(img_dev.cpu().numpy())
    ds = codec.open_encoded()
    nb = ds.num_bricks
    lod = b.bit_length() - 1
    per = 1 << (3 * lod)
    reqs = requests_tensor(requests(np.arange(nb), np.full(nb, lod), np.arange(nb, dtype=np.uint64) * per), dev)
    out = torch.empty(nb * per, dtype=torch.int64, device=dev)
    status = torch.zeros(nb, dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    # ---- correctness gate on the bench workload: full-resolution decode == source volume
    codec.decode_batch(ds, reqs, out, status)
    torch.cuda.synchronize()
    assert int(status.abs().max()) == 0, "decode status"
    check = check_against_volume(out, vol, nb, b, W["shape"])

    for _ in range(args.warmup):
        flush_l2(flush)
        codec.decode_batch(ds, reqs, out, status)
    torch.cuda.synchronize()
    clk = Clocks(local)
    barrier(pg)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        codec.decode_batch(ds, reqs, out, status)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    barrier(pg)
    clocks = clk.stop()
    ms = statistics.mean(times)
    ms_max = max_over_ranks(ms, pg, dev)
    value = world * nvox / (ms_max * 1e-3) / 1e9

    info = ds.info
    alg_bytes = info.stream_bytes + 8 * info.palette_entries + 16 * nb + 8 * nb * per
    hbm, hbm_kind = peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    traffic = load_traffic("decode_kernel", W["name"])

    # ---- end to end through the C ABI with host buffers (csv_decode_image: open + seek index + decode + D2H)
    host_img = np.frombuffer(image, np.uint8)
    e2e_ms = []
    h_out = torch.empty((nb, per), dtype=torch.int64, pin_memory=True)
    h_st = np.zeros(nb, np.uint32)
    lib = codec.lib
    import ctypes as C
    for k in range(max(2, min(args.steps, 5)) + 1):
        barrier(pg)
        t0 = time.perf_counter()
        rc = lib.csv_decode_image(codec.handle, host_img.ctypes.data_as(C.POINTER(C.c_uint8)), len(image), lod,
                                  C.cast(h_out.data_ptr(), C.POINTER(C.c_uint64)),
                                  h_st.ctypes.data_as(C.POINTER(C.c_uint32)))
        t1 = time.perf_counter()
        assert rc == 0, codec.lib.csv_last_error(codec.handle)
        if k > 0:
            e2e_ms.append((t1 - t0) * 1e3)
    e2e_best = max_over_ranks(statistics.mean(e2e_ms), pg, dev)
    e2e = {"value": world * nvox / (e2e_best * 1e-3) / 1e9, "unit": "Gvox/s", "h2d_bytes_per_step": len(image),
           "d2h_bytes_per_step": 8 * nb * per + 4 * nb, "ms_per_step": e2e_best,
           "path": "csv_decode_image: host .csbd -> open (H2D, seek index) -> decode -> D2H labels"}
    e2e_ok = bool(np.array_equal(h_out.numpy().view(np.uint64).reshape(-1),
                                 out.cpu().numpy().view(np.uint64)))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        vol_np = vol.cpu().numpy().view(np.uint64)
        ref = cpu_reference(vol_np, b, image)
        cpu = {"value": ref["decode_gvox_s"], "unit": "Gvox/s", "cores": 1, "kind": ref["kind"],
               "sample": f"whole workload ({nb} bricks, {nvox} voxels): splitGridIntoBricks+compressDataset+"
                         f"saveDatasetToFile then decodeRansStream+decodeBrick<64> for every brick, 1 thread",
               "encode_mvox_s": ref["encode_mvox_s"], "encode_s": ref["encode_s"], "decode_s": ref["decode_s"],
               "encode_bytes_identical": ref["bytes_identical"]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Gvox/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": W["name"], "volume": list(W["shape"][::-1]), "brick": b, "bricks": nb,
                       "lod": lod, "tubes": W["n_tubes"], "radius": [W["r_min"], W["r_max"]],
                       "voronoi_cells": W["n_cells"], "zero_frac": W["zero_frac"], "seed": W["seed"],
                       "l2": "flushed between timed steps (256 MiB buffer)",
                       "parallelism": f"weak x{world}, bricks independent, no collective"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4), "traffic": traffic,
                         "algorithmic_bytes": alg_bytes, "peak_kind": hbm_kind},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps,
            "clocks": clocks,
            "encode": {"value": round(nvox / (enc_ms_best * 1e-3) / 1e6, 1), "unit": "Mvox/s",
                       "ms": round(enc_ms_best, 3), "image_bytes": n,
                       "speedup_vs_cpu": (round(nvox / (enc_ms_best * 1e-3) / 1e6 / cpu["encode_mvox_s"], 1)
                                          if cpu else None),
                       "bytes_identical_to_reference": cpu["encode_bytes_identical"] if cpu else None},
            "checks": {"decode_equals_source": check, "e2e_equals_device": e2e_ok},
        }
        print(json.dumps(line))
    ds.close()
    if pg is not None:
        pg.destroy_process_group()


def check_against_volume(out, vol, nb, b, shape):
    """Full-resolution decode equals the source volume (bricks in split order, Morton order inside)."""
    import torch
    D, H, W = shape
    nbx, nby, nbz = -(-W // b), -(-H // b), -(-D // b)
    idx = torch.arange(b, device=out.device)
    m = torch.zeros((b, b, b), dtype=torch.int64, device=out.device)
    for bit in range(10):
        m |= ((idx[None, None, :] >> bit) & 1) << (3 * bit)
        m |= ((idx[None, :, None] >> bit) & 1) << (3 * bit + 1)
        m |= ((idx[:, None, None] >> bit) & 1) << (3 * bit + 2)
    bricks = out.view(nb, b ** 3)
    i = 0
    for bx in range(nbx):
        for by in range(nby):
            for bz in range(nbz):
                src = vol[bz * b:(bz + 1) * b, by * b:(by + 1) * b, bx * b:(bx + 1) * b]
                if not torch.equal(bricks[i][m], src):
                    return False
                i += 1
    return True


def load_traffic(kernel: str, workload: str):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(kernel, {}).get(workload)


def run_reference(args):
    """The reference's own CPU decoder (oracle/_ref: decodeRansStream + decodeBrick<64>), all host threads."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import REF_SO, Oracle, Reference
    W = WORKLOAD
    D, H, Wd = W["shape"]
    b = W["brick"]
    nvox = D * H * Wd
    from csvb200 import Codec
    codec = Codec(0)
    vol = torch.empty(W["shape"], dtype=torch.int64, device="cuda")
    codec.synth_volume(vol, W["kind"], W["n_cells"], W["n_tubes"], W["r_min"], W["r_max"], W["zero_frac"],
                       W["seed"])
    vol_np = vol.cpu().numpy().view(np.uint64)
    del vol
    threads = os.cpu_count() or 1
    if os.path.exists(REF_SO):
        R = Reference()
        image = R.encode(vol_np, b)
        kind = "reference"

        def step():
            bad = R.decode_parallel(image, threads)
            assert bad == 0
    else:
        O = Oracle()
        image = O.encode(vol_np, b)
        kind = "port"
        threads = 1

        def step():
            O.decode_image(image, b.bit_length() - 1)
    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    s = statistics.mean(times)
    v = nvox / s / 1e9
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "Gvox/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(s * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": W["name"], "volume": list(W["shape"][::-1]), "brick": b, "lod": b.bit_length() - 1},
        "cpu_baseline": {"value": round(v, 4), "unit": "Gvox/s", "cores": threads, "kind": kind,
                         "sample": f"every step decodes all {nvox // b ** 3} bricks at full resolution "
                                   f"(decodeRansStream + decodeBrick<64>), bricks split over {threads} host threads"},
        "e2e": {"value": round(v, 4), "unit": "Gvox/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
