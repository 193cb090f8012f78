"""CPU: the colour path's restatement (oracle/csv_oracle_rgba.c) pinned against the reference's own formulas.

* the transfer function: buildTransferFunctionBuffers + hslToRgb (web/scripts/webgpuSetup.js:389-465,
  490-515) written out again here with Python floats (JavaScript numbers are IEEE doubles, Math.round is
  floor(x + 0.5));
* hashLabel (web/shaders/decode.wgsl:135-172) with u32 wrap-around arithmetic;
* the RGBA march on a one-brick scene whose answer is known in closed form.
"""
import math

import numpy as np


def js_tf(i):
    h = (i * 137.5) % 360
    s = 0.55 + (i % 3) * 0.08
    l = 0.35 + (i % 4) * 0.05
    op = 0.25 + (i % 5) * 0.08
    c = (1 - abs(2 * l - 1)) * s
    x = c * (1 - abs((h / 60) % 2 - 1))
    m = l - c / 2
    if h < 60:
        r, g, b = c, x, 0
    elif h < 120:
        r, g, b = x, c, 0
    elif h < 180:
        r, g, b = 0, c, x
    elif h < 240:
        r, g, b = 0, x, c
    elif h < 300:
        r, g, b = x, 0, c
    else:
        r, g, b = c, 0, x
    rr, gg, bb = (math.floor(v + 0.5) for v in ((r + m) * 255, (g + m) * 255, (b + m) * 255))
    R, G, B = (min(math.floor(v * 0.92), 255) for v in (rr, gg, bb))
    return R | (G << 8) | (B << 16) | (math.floor(op * 255) << 24)


def js_hash(v):
    M = 0xFFFFFFFF
    lo, hi = v & M, v >> 32
    lo ^= hi
    lo ^= lo >> 16
    lo = (lo * 0x7feb352d) & M
    lo ^= lo >> 15
    hi ^= lo
    hi ^= hi >> 16
    hi = (hi * 0x85ebca6b) & M
    hi ^= hi >> 13
    return (lo & 0xFF) | (((lo >> 8) & 0xFF) << 8) | (((hi >> 8) & 0xFF) << 16) | (0x40 << 24)


def test_transfer_function_is_the_viewers(oracle):
    rng = np.random.default_rng(2)
    labels = np.unique(rng.integers(1, 2 ** 63, 700, dtype=np.uint64))
    got = oracle.transfer_function(labels)
    assert [int(v) for v in got] == [js_tf(i) for i in range(len(labels))]
    hidden = labels[::7]
    got_h = oracle.transfer_function(labels, hidden)
    assert np.all(got_h[::7] == 0) and np.array_equal(np.delete(got_h, np.s_[::7]), np.delete(got, np.s_[::7]))


def test_hash_label_and_lookup(oracle):
    rng = np.random.default_rng(4)
    keys = np.unique(rng.integers(1, 2 ** 64 - 1, 50, dtype=np.uint64))
    cols = oracle.transfer_function(keys)
    for v in list(keys[:10]) + list(rng.integers(1, 2 ** 64 - 1, 200, dtype=np.uint64)) + [1, 2 ** 32, 2 ** 64 - 2]:
        v = int(v)
        want = int(cols[np.searchsorted(keys, v)]) if v in set(int(k) for k in keys) else js_hash(v)
        assert oracle.label_rgba(v, keys, cols) == want, v
    assert oracle.label_rgba(0, keys, cols) == 0


def test_rgba_march_one_uniform_brick(oracle):
    """One 16^3 brick at LOD 0 filled with one label seen nearly along the z axis (exactly axis-parallel rays
    miss the volume in the shader's slab test: their reciprocal direction component is 0): an unshaded sample
    (alpha 0.25 < 0.35) at stride 16, so the pixel is the label's colour times 1 - (1 - a)^16 alpha,
    composited once."""
    from csvb200.camera import SLOT_DTYPE, camera_uniform
    label = 12345
    keys = np.array([label], np.uint64)
    cols = oracle.transfer_function(keys)  # entry 0: opacity 0.25 -> alpha 63
    a = ((int(cols[0]) >> 24) & 255) / 255.0
    assert a < 0.35
    slots = np.zeros(1, SLOT_DTYPE)
    slots[0] = (0, 0, 0)
    labels = np.array([label], np.uint64)
    cam = camera_uniform((8.0, 8.0, -40.0), (0.01, 0.02, 1.0), math.pi / 3)
    img = oracle.render_rgba(cam, 9, 9, 16.0, 16, 1, slots, labels, keys, cols, [0.4, 0.6, -0.9, 0.5, 0.8])
    px = int(img[4, 4])
    ca = np.float32(1.0) - np.float32(np.power(np.float32(1.0) - np.float32(a), np.float32(16.0)))
    for k in range(3):
        c = np.float32(((int(cols[0]) >> (8 * k)) & 255) / np.float32(255.0))
        assert abs(((px >> (8 * k)) & 255) - int(np.float32(c * ca) * np.float32(255.0))) <= 1
    assert abs((px >> 24) - int(ca * np.float32(255.0))) <= 1
