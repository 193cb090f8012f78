"""GPU: each workload's own check at its own generator and size.

* the synthetic volumes: the CPU restatement of the generator (oracle or_synth_volume, which the bench's
  reference arm builds its inputs with) equals csv_synth_volume, on small odd shapes and on the full 1024^3
  uneven-batch volume;
* 256^3 Voronoi (1500 cells, a 10 % slab of label 0), 64 bricks of 64^3: the device encoder's bytes equal
  the reference encoder's (compressDataset<64>, brickEncoding.hpp:466-531, compiled from its sources), the
  reference decoder and the device decoder both give back the source at full resolution, and every coarser
  LOD equals the oracle's (decode.wgsl:344-509 restated);
* 512^3 neurite-like volume (400 tubes of radius 2-12 over 3000 cells, 15 % label 0), 512 bricks: bytes equal
  to the reference encoder's, and LOD 0 ... 6 of the device decode equal the oracle's, with LOD 6 equal to the
  source and to the reference decoder's output;
* the serving loop at 1920x1080 over a 512^3 volume of the 2048^3 serving generator (tubes of radius 2-12 over
  Voronoi cells, 15 % label 0; counts scaled to keep its density): three frames of the seeded orbit, every
  frame's label and depth image bit-equal to the scalar DDA of the oracle's frame loop (rayTrace.wgsl:565-906
  restated), with the same slot tables.
"""
import math
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_volume(codec, shape, kind, cells, tubes, r0, r1, zero, seed):
    import torch
    vol = torch.empty(shape, dtype=torch.int64, device="cuda")
    codec.synth_volume(vol, kind, cells, tubes, r0, r1, zero, seed)
    return vol


def _encode(codec, vol, b):
    import torch
    n = codec.encode_device(vol, b)
    torch.cuda.synchronize()
    img = bytes(codec.encoded_image_tensor().cpu().numpy())
    assert len(img) == n
    return img


@pytest.mark.parametrize("shape,kind,args", [
    ((72, 80, 96), 0, (150, 0, 0.0, 0.0, 0.1)),
    ((64, 96, 130), 1, (200, 30, 1.5, 6.0, 0.2)),
    ((96, 64, 128), 2, (120, 60, 1.0, 4.0, 0.0)),
    ((128, 128, 128), 1, (312, 60, 2.0, 12.0, 0.15)),
])
def test_cpu_generator_equals_device(codec, oracle, shape, kind, args):
    import torch
    cells, tubes, r0, r1, zero = args
    dev = _device_volume(codec, shape, kind, cells, tubes, r0, r1, zero, 17 + kind)
    cpu = oracle.synth_volume(shape, kind, cells, tubes, r0, r1, zero, 17 + kind)
    assert torch.equal(dev, torch.from_numpy(cpu.view(np.int64)).cuda())


def test_cpu_generator_equals_device_mixed1024(codec, oracle):
    """The bench's reference arm builds the 1024^3 uneven-batch images from the CPU generator: it must be the
    volume the device arm decodes (2000 cells, 5000 tubes of radius 1-4 in the x >= 512 half, seed 3)."""
    import torch
    shape = (1024, 1024, 1024)
    dev = _device_volume(codec, shape, 2, 2000, 5000, 1.0, 4.0, 0.0, 3)
    cpu = oracle.synth_volume(shape, 2, 2000, 5000, 1.0, 4.0, 0.0, 3)
    same = True
    for z in range(0, 1024, 128):  # slab by slab: 1 GiB per copy
        same &= torch.equal(dev[z:z + 128], torch.from_numpy(cpu[z:z + 128].view(np.int64)).cuda())
    assert same


def test_config1_voronoi256_bytes_and_decode(codec, oracle, reference):
    import bench
    vol = _device_volume(codec, (256, 256, 256), 0, 1500, 0, 0.0, 0.0, 0.10, 1)
    host = vol.cpu().numpy().view(np.uint64)
    zero = float((host == 0).mean())
    assert 0.07 < zero < 0.13  # the slab covers about 10 %
    gpu = _encode(codec, vol, 64)
    t0 = time.perf_counter()
    ref, tm = reference.encode(host, 64, timings=True)
    ref_s = time.perf_counter() - t0
    assert int(np.frombuffer(gpu[8:12], np.uint32)[0]) == 64
    assert gpu == ref, "device bytes differ from the reference encoder's"
    print(f"\nconfig 1: reference encoder {ref_s:.2f} s on 1 core ({16.777216 / ref_s:.1f} Mvox/s; {tm})")
    # the reference decoder gives back the source (bricks that are one label throw there and are skipped)
    rdec, rst, _ = reference.decode_all_full(ref, 64)
    ddev, dst = codec.decode_image(gpu, 6)
    assert int(dst.max()) == 0
    import torch
    assert bench.check_against_volume(torch.from_numpy(ddev.reshape(-1).view(np.int64)).cuda(), 0, vol, 64)
    ok = rst == 0
    assert ok.sum() > 0 and np.array_equal(rdec[ok], ddev[ok])
    for lod in range(0, 6):
        got, st = codec.decode_image(gpu, lod)
        exp, est = oracle.decode_image(gpu, lod)
        assert int(st.max()) == 0 and np.array_equal(got, exp), lod


def test_config2_neurite512_every_lod(codec, oracle, reference):
    import torch

    import bench
    N = bench.NEURITE
    vol = _device_volume(codec, N["shape"], N["kind"], N["n_cells"], N["n_tubes"], N["r_min"], N["r_max"],
                         N["zero_frac"], N["seed"])
    gpu = _encode(codec, vol, 64)
    host = vol.cpu().numpy().view(np.uint64)
    assert gpu == reference.encode(host, 64), "device bytes differ from the reference encoder's"
    del host
    rdec, rst, _ = reference.decode_all_full(gpu, 64)
    for lod in range(6, -1, -1):
        got, st = codec.decode_image(gpu, lod)
        exp, est = oracle.decode_image(gpu, lod)
        assert int(st.max()) == 0 and int(est.max()) == 0
        assert np.array_equal(got, exp), f"LOD {lod} differs from the oracle"
        if lod == 6:
            assert bench.check_against_volume(torch.from_numpy(got.reshape(-1).view(np.int64)).cuda(), 0, vol, 64)
            ok = rst == 0
            assert ok.sum() > 0 and np.array_equal(rdec[ok], got[ok])


def test_config5_serve_1080p_frames_vs_scalar_dda(codec, oracle):
    """Three frames of the seeded orbit at 1920x1080, label and depth bit-equal to the oracle's frame loop."""
    import torch

    import bench
    from csvb200 import CONE_SCREEN, Server
    from oracle import SLOT_DTYPE, OracleServer
    S = bench.SERVE
    shape = (512, 512, 512)
    # the serving generator at 1/64 of its volume: cells scale with the volume, tubes with volume / length
    vol = _device_volume(codec, shape, S["kind"], S["n_cells"] // 64, S["n_tubes"] // 16, S["r_min"], S["r_max"],
                         S["zero_frac"], S["seed"])
    img = _encode(codec, vol, S["brick"])
    del vol
    Wp, Hp, fov = S["width"], S["height"], S["fov"]
    cache = 4 << 30
    ds = codec.open(img)
    srv = Server(codec, ds, Wp, Hp, fov, cache_bytes=cache, cone=CONE_SCREEN)
    ref = OracleServer(oracle, img, Wp, Hp, fov, CONE_SCREEN, cache)
    lab = torch.zeros(Wp * Hp, dtype=torch.int64, device="cuda")
    dep = torch.zeros(Wp * Hp, dtype=torch.float32, device="cuda")
    views = bench.orbit_path(S["frames"], (256.0, 256.0, 256.0), S["seed"], scale=0.25)
    hit = []
    for k in (0, 150, 300):
        pos, d = views[k]
        srv.submit(0, pos, d, lab, dep)
        srv.step()
        fr = srv.poll(wait=True)
        assert len(fr) == 1
        rl, rd, rst = ref.step([0], [(pos, d)], [True])
        for key in ["planned", "decoded", "resident", "decoded_voxels"]:
            assert fr[0][key] == rst[key], (k, key)
        assert np.array_equal(srv.slots_tensor(0).cpu().numpy().view(SLOT_DTYPE), ref.slots(0)), k
        gl = lab.cpu().numpy().view(np.uint64).reshape(Hp, Wp)
        gd = dep.cpu().numpy().reshape(Hp, Wp)
        assert np.array_equal(gl, rl[0]), (k, int((gl != rl[0]).sum()))
        assert np.array_equal(gd.view(np.uint32), rd[0].view(np.uint32)), k
        hit.append(float((gl != 0).mean()))
    assert min(hit) > 0.05, hit  # the frames see the volume
    srv.close()
    ref.close()
    ds.close()
