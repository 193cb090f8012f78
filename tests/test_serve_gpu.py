"""GPU: the serving loop (csv_serve_*) step by step against the CPU restatement of the viewer's frame loop.

Every step is compared with the oracle server fed the same cameras: the brick
slot table (which bricks are resident, at which LOD and at which cache
offset), the per-step counters, and every session's label and depth image,
bit for bit.  Small caches force evictions, free-stack reuse and rebuilds.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H = 96, 64
FOV = math.pi / 3


def _image(codec, shape, b, seed, kind=1):
    import torch
    vol = torch.empty(shape, dtype=torch.int64, device="cuda")
    codec.synth_volume(vol, kind, 200, 40 if kind == 1 else 0, 1.5, 6.0, 0.3, seed)
    codec.encode_device(vol, b)
    return bytes(codec.encoded_image_tensor().cpu().numpy())


@pytest.fixture(scope="module")
def cube16(codec):
    return _image(codec, (128, 128, 128), 16, 41)


@pytest.fixture(scope="module")
def slab32(codec):
    return _image(codec, (96, 128, 256), 32, 42)  # 8 x 4 x 3 bricks: the slot grid holds absent bricks


def _orbit_views(center, n, r0, r1, yaw0=0.2, pitch=0.25):
    from csvb200.camera import orbit
    out = []
    for f in range(n):
        r = r0 + (r1 - r0) * f / max(1, n - 1)
        out.append(orbit(center, r, yaw0 + 0.35 * f, pitch - 0.04 * f))
    return out


def _compare_cache(srv, ref, info, sessions):
    """Every resident block a session's slot table points at holds the oracle's labels."""
    cache = srv.cache_tensor().cpu().numpy().view(np.uint64)
    rc = ref.cache(len(cache))
    for s in sessions:
        slots = ref.slots(s)
        for sl in slots[(slots["flags"] == 0)]:
            n = 8 ** int(sl["lod"]) if sl["offset"] >= info.palette_table else 1
            o = int(sl["offset"])
            assert np.array_equal(cache[o:o + n], rc[o:o + n])


def _run_pair(codec, oracle, img, steps, cache_bytes, cone, sessions=1, hidden=None, leave=None, keep=None,
              admit=0, compact_before=()):
    """steps: per step, the list of (session, (pos, dir)) that submit a frame; leave: {step: [sessions]} closed
    before that step; compact_before: steps before which both caches are compacted (and compared).  Compares GPU
    and oracle after every step; keep collects each session's images."""
    import torch
    from csvb200 import Server
    from oracle import SLOT_DTYPE, OracleServer, camera_uniform
    leave = leave or {}
    ds = codec.open(img)
    srv = Server(codec, ds, W, H, FOV, cache_bytes=cache_bytes, max_sessions=sessions, cone=cone, hidden=hidden,
                 admit=admit)
    ref = OracleServer(oracle, img, W, H, FOV, cone, cache_bytes, hidden=hidden, admit=admit)
    labs = [torch.zeros(W * H, dtype=torch.int64, device="cuda") for _ in range(sessions)]
    deps = [torch.zeros(W * H, dtype=torch.float32, device="cuda") for _ in range(sessions)]
    info = srv.info()
    assert info.n_slots == ref.n_slots and info.bricks_per_axis == ref.bpa
    seen = {"rebuilt": 0, "freed": 0, "planned0": 0, "resident": [], "decoded": []}
    latest = {}
    for k, step in enumerate(steps):
        if k in compact_before:
            srv.compact()
            ref.compact()
            torch.cuda.synchronize()
            assert srv.poll(wait=True) == []  # a compaction reports no frame
            for s in sorted(latest):
                slots = srv.slots_tensor(s).cpu().numpy().view(SLOT_DTYPE)
                assert np.array_equal(slots, ref.slots(s)), ("compact", k, s)
            _compare_cache(srv, ref, info, sorted(latest))
        for s in leave.get(k, []):
            srv.leave(s)
            latest.pop(s, None)
        for s, (pos, d) in step:
            srv.submit(s, pos, d, labs[s], deps[s])
            latest[s] = (pos, d)
            assert np.array_equal(srv.camera(pos, d), camera_uniform(oracle, pos, d, FOV))
        sid = srv.step()
        frames = srv.poll(wait=True)
        subm = sorted(s for s, _ in step)
        assert [f["step"] for f in frames] == [sid] * len(step)
        assert [f["session"] for f in frames] == subm
        open_ = sorted(latest)
        rl, rd, rst = ref.step(open_, [latest[s] for s in open_], [s in subm for s in open_])
        for key in ["planned", "visible", "decoded", "freed", "resident", "rebuilt", "decoded_voxels"]:
            assert all(f[key] == rst[key] for f in frames), (k, key, frames[0][key], rst[key])
        assert [f["entered"] for f in frames] == rst["entered"], k
        assert [f["missing"] for f in frames] == rst["missing"], k
        for s in open_:
            slots = srv.slots_tensor(s).cpu().numpy().view(SLOT_DTYPE)
            assert np.array_equal(slots, ref.slots(s)), (k, s)
        if frames and frames[0]["planned"] and frames[0]["decoded"]:
            assert int(_status(srv, frames[0]["decoded"]).max()) == 0
        for j, s in enumerate(subm):
            gl = labs[s].cpu().numpy().view(np.uint64).reshape(H, W)
            gd = deps[s].cpu().numpy().reshape(H, W)
            assert np.array_equal(gl, rl[j]), (k, s, int((gl != rl[j]).sum()))
            assert np.array_equal(gd.view(np.uint32), rd[j].view(np.uint32)), (k, s)
            if keep is not None:
                keep.setdefault(s, []).append((gl.copy(), gd.copy()))
        if frames:
            seen["rebuilt"] += frames[0]["rebuilt"]
            seen["freed"] += frames[0]["freed"]
            seen["planned0"] += frames[0]["planned"] == 0
            seen["resident"].append(frames[0]["resident"])
            seen["decoded"].append(frames[0]["decoded"])
    # the resident labels equal the oracle's cache wherever a slot points
    _compare_cache(srv, ref, info, sorted(latest))
    srv.close()
    ref.close()
    ds.close()
    return seen


def _status(srv, n):
    from csvb200 import _device_view
    return _device_view(srv.info().decode_status, n, "<u4", srv.codec.device).cpu().numpy()


@pytest.mark.parametrize("cone", [0, 1])
def test_serve_orbit_large_cache(codec, oracle, cube16, cone):
    views = _orbit_views((64.0, 64.0, 64.0), 8, 170.0, 90.0)
    steps = [[(0, v)] for v in views]
    steps.insert(3, [(0, views[2])])  # camera did not move: render only
    seen = _run_pair(codec, oracle, cube16, steps, 64 << 20, cone)
    assert seen["planned0"] == 1 and seen["rebuilt"] == 0 and seen["freed"] > 0


def test_serve_small_cache_rebuilds(codec, oracle, cube16):
    views = _orbit_views((64.0, 64.0, 64.0), 8, 150.0, 60.0)
    seen = _run_pair(codec, oracle, cube16, [[(0, v)] for v in views], 512 << 10, 1)
    assert seen["rebuilt"] > 0


def test_serve_medium_cache_reuses_free_blocks(codec, oracle, slab32):
    views = _orbit_views((128.0, 64.0, 48.0), 10, 260.0, 120.0, yaw0=1.0, pitch=0.4)
    _run_pair(codec, oracle, slab32, [[(0, v)] for v in views], 6 << 20, 1)


def test_serve_two_sessions_one_step(codec, oracle, cube16):
    a = _orbit_views((64.0, 64.0, 64.0), 5, 160.0, 100.0)
    b = _orbit_views((64.0, 64.0, 64.0), 5, 120.0, 200.0, yaw0=2.5, pitch=-0.3)
    steps = [[(0, a[k]), (1, b[k])] for k in range(5)]
    steps.insert(2, [(1, b[1])])  # session 0 open without a new frame
    _run_pair(codec, oracle, cube16, steps, 8 << 20, 1, sessions=2)


def test_serve_each_session_same_alone_and_in_the_mix(codec, oracle, cube16):
    """Continuous batching: session 1 joins while session 0 is served, skips a frame, leaves; session 2 joins
    later.  Every session's images equal the ones it gets served alone, bit for bit."""
    a = _orbit_views((64.0, 64.0, 64.0), 9, 170.0, 70.0)
    b = _orbit_views((64.0, 64.0, 64.0), 9, 60.0, 190.0, yaw0=2.0, pitch=-0.4)
    c = _orbit_views((64.0, 64.0, 64.0), 9, 110.0, 110.0, yaw0=4.0, pitch=0.6)
    steps = []
    for f in range(9):
        st = [(0, a[f])]
        if 2 <= f <= 6 and f != 4:
            st.append((1, b[f]))
        if f >= 5:
            st.append((2, c[f]))
        steps.append(st)
    mix = {}
    _run_pair(codec, oracle, cube16, steps, 64 << 20, 1, sessions=3, leave={7: [1]}, keep=mix)
    for s in range(3):
        alone = {}
        solo = [[(0, v)] for st in steps for (q, v) in st if q == s]
        _run_pair(codec, oracle, cube16, solo, 64 << 20, 1, sessions=1, keep=alone)
        assert len(alone[0]) == len(mix[s])
        for (l1, d1), (l2, d2) in zip(alone[0], mix[s]):
            assert np.array_equal(l1, l2) and np.array_equal(d1.view(np.uint32), d2.view(np.uint32))


def test_serve_hidden_labels(codec, oracle, cube16):
    lab = oracle.decode_image(cube16, 4)[0]
    vals, counts = np.unique(lab[lab != 0], return_counts=True)
    hidden = vals[np.argsort(-counts)[:6]].astype(np.uint64)
    views = _orbit_views((64.0, 64.0, 64.0), 4, 160.0, 110.0)
    _run_pair(codec, oracle, cube16, [[(0, v)] for v in views], 64 << 20, 1, hidden=hidden)


def test_serve_admission_by_rays(codec, oracle, cube16):
    """CSV_ADMIT_RAYS (the reference's useGPUCulling path): the first frame plans by the cone, later frames keep
    only the bricks the rays entered; bricks hidden behind others are released.  Step by step equal to the
    oracle's frame loop in the same mode, and the plan differs from the cone plan's."""
    views = _orbit_views((64.0, 64.0, 64.0), 6, 90.0, 60.0)
    steps = [[(0, v)] for v in views]
    steps.insert(2, [(0, views[1])])  # still camera: the new requests re-plan
    rays = _run_pair(codec, oracle, cube16, steps, 64 << 20, 1, admit=1)
    cone = _run_pair(codec, oracle, cube16, steps, 64 << 20, 1, admit=0)
    assert rays["resident"][0] == cone["resident"][0]  # first frame: the cone plan
    assert all(r <= c for r, c in zip(rays["resident"], cone["resident"]))
    assert any(r < c for r, c in zip(rays["resident"], cone["resident"]))
    assert rays["planned0"] == 0 and cone["planned0"] == 1


def test_serve_admission_by_rays_two_sessions(codec, oracle, cube16):
    a = _orbit_views((64.0, 64.0, 64.0), 5, 150.0, 80.0)
    b = _orbit_views((64.0, 64.0, 64.0), 5, 80.0, 160.0, yaw0=2.5, pitch=-0.3)
    steps = [[(0, a[k]), (1, b[k])] for k in range(5)]
    steps.insert(2, [(1, b[1])])  # session 0 open without a new frame: it keeps its plan's inputs
    _run_pair(codec, oracle, cube16, steps, 8 << 20, 1, sessions=2, admit=1, leave={4: [1]})


@pytest.mark.parametrize("cache", [6 << 20, 64 << 20])
def test_serve_compaction(codec, oracle, slab32, cache):
    """csv_serve_compact (CacheState.compact()): after frees scattered over the stacks, the resident blocks are
    packed from offset 0, coarse LODs first; slot tables, cache contents and the following steps equal the
    oracle's."""
    views = _orbit_views((128.0, 64.0, 48.0), 9, 260.0, 120.0, yaw0=1.0, pitch=0.4)
    seen = _run_pair(codec, oracle, slab32, [[(0, v)] for v in views], cache, 1, compact_before=(4, 7))
    assert seen["freed"] > 0


def test_serve_newest_frame_wins_and_errors(codec, cube16):
    import torch
    from csvb200 import CsvError, Server
    ds = codec.open(cube16)
    srv = Server(codec, ds, W, H, FOV, cache_bytes=16 << 20)
    l1 = torch.zeros(W * H, dtype=torch.int64, device="cuda")
    d1 = torch.zeros(W * H, dtype=torch.float32, device="cuda")
    l2 = torch.zeros_like(l1)
    d2 = torch.zeros_like(d1)
    v = _orbit_views((64.0, 64.0, 64.0), 2, 160.0, 150.0)
    srv.submit(0, *v[0], l1, d1)
    srv.submit(0, *v[1], l2, d2)  # replaces the first
    srv.step()
    frames = srv.poll(wait=True)
    assert len(frames) == 1
    torch.cuda.synchronize()
    assert int((l1 != 0).sum()) == 0 and int((l2 != 0).sum()) > 0
    with pytest.raises(CsvError) as e:
        srv.step()  # nothing submitted
    assert e.value.code == -1
    with pytest.raises(CsvError) as e:
        srv.submit(1, *v[0], l1, d1)  # one session only
    assert e.value.code == -5
    srv.close()
    ds.close()


def test_serve_many_steps_without_polling(codec, cube16):
    """More steps in flight than the ring holds: the server harvests the oldest itself; poll returns all."""
    import torch
    from csvb200 import Server
    ds = codec.open(cube16)
    srv = Server(codec, ds, W, H, FOV, cache_bytes=16 << 20)
    lab = torch.zeros(W * H, dtype=torch.int64, device="cuda")
    dep = torch.zeros(W * H, dtype=torch.float32, device="cuda")
    views = _orbit_views((64.0, 64.0, 64.0), 150, 170.0, 80.0)
    for v in views:
        srv.submit(0, *v, lab, dep)
        srv.step()
    frames = srv.poll(wait=True, max_frames=1000)
    assert [f["step"] for f in frames] == list(range(150))
    assert all(f["ms"] > 0 for f in frames)
    srv.close()
    ds.close()


def test_serve_rgba_frames_are_the_colour_path(codec, cube16):
    """A session that submits RGBA frames, beside one that submits label/depth frames, in the same steps: each
    RGBA frame is csv_render_rgba of that step's cache and slot table through the dataset's transfer function
    (hidden labels transparent) and the server's lighting, word for word; the label session's frames are its
    label render.  RGBA rays run on past the first visible voxel (to alpha 0.95), so they enter at least the
    bricks the label rays enter."""
    import torch
    from csvb200 import Server
    ds = codec.open(cube16)
    keys, cols = codec.transfer_function(ds)
    hidden = keys[::3].copy()
    keys, cols = codec.transfer_function(ds, hidden=hidden)
    d_keys = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    d_cols = torch.from_numpy(cols.view(np.int32).copy()).cuda()
    srv = Server(codec, ds, W, H, FOV, max_sessions=2, hidden=hidden)
    light = codec.lighting(40.0)
    srv.set_lighting(light)
    rgba = torch.zeros(W * H, dtype=torch.int32, device="cuda")
    lab = torch.zeros(W * H, dtype=torch.int64, device="cuda")
    dep = torch.zeros(W * H, dtype=torch.float32, device="cuda")
    info = srv.info()
    for f, (pos, d) in enumerate(_orbit_views((64.0, 64.0, 64.0), 4, 260.0, 150.0)):
        srv.submit_rgba(0, pos, d, rgba)
        srv.submit(1, pos, d, lab, dep)
        srv.step()
        frames = srv.poll(wait=True)
        assert sorted(fr["session"] for fr in frames) == [0, 1]
        cam = srv.camera(pos, d)
        want = torch.empty(W * H, dtype=torch.int32, device="cuda")
        codec.render_rgba(cam, W, H, float(info.bricks_per_axis * 16), 16, info.bricks_per_axis, srv.slots_tensor(0),
                          srv.cache_tensor(), d_keys, d_cols, light, want)
        l2 = torch.empty(W * H, dtype=torch.int64, device="cuda")
        d2 = torch.empty(W * H, dtype=torch.float32, device="cuda")
        d_hid = torch.from_numpy(np.sort(hidden).view(np.int64).copy()).cuda()
        codec.render(cam, W, H, float(info.bricks_per_axis * 16), 16, info.bricks_per_axis, srv.slots_tensor(1),
                     srv.cache_tensor(), l2, d2, d_hidden=d_hid)
        torch.cuda.synchronize()
        assert torch.equal(rgba, want), f
        assert torch.equal(lab, l2) and torch.equal(dep.view(torch.int32), d2.view(torch.int32)), f
        assert (rgba >> 24).any()
        by = {fr["session"]: fr for fr in frames}
        assert by[0]["entered"] >= by[1]["entered"]
    srv.close()
    ds.close()
