"""Learned mode / shared-table selector: fitting the shared tables, training the network, choosing per brick.

The reference encodes every brick with one op preference order and one rANS
model per dataset (brickEncoding.hpp:198-282, 481-482).  Here a brick may use
one of 12 decoder-transparent encoding modes and one of up to 16 shared rANS
tables, stored per brick in a version-2 image (include/csv.h).  Three ways to
choose them:

  * plain        mode 0, the dataset's own model: the reference encoder (version 1);
  * exhaustive   csv_encode_stats (every mode's nibble histogram per brick) and
                 csv_select_exhaustive (fewest estimated bits over all pairs);
  * learned      csv_brick_features (32 cheap statistics) and the selector network
                 (csv_mlp_forward), trained here on the exhaustive choices with the
                 library's own tensor-core forward/backward kernels (csv_mlp_grad)
                 and Adam (csv_mlp_adam).

Only the table fitting (a few thousand 16-bin histograms) runs on the host.
"""
from __future__ import annotations

import numpy as np

from . import Codec, SelectorNet

MODES = 12
TABLES = 16
FEATURES = 32


def build_model(raw: np.ndarray) -> np.ndarray:
    """buildRansModel (brickEncoding.cpp:146-200) on a 16-bin histogram: frequencies summing to 4096."""
    f = np.maximum(np.asarray(raw, np.uint64).astype(np.uint32).astype(np.uint64), 1)
    s = np.maximum(f * 4096 // f.sum(), 1)
    while s.sum() < 4096:
        s[0] += 1
    while s.sum() > 4096:
        k = int(np.argmax(s))
        if s[k] <= 1:
            break
        s[k] -= 1
    return s.astype(np.uint32)


def table_bits(tables: np.ndarray) -> np.ndarray:
    """Bits per symbol of each table (n x 16), -log2(f / 4096)."""
    return -np.log2(np.asarray(tables, np.float64) / 4096.0)


def choose(hist: np.ndarray, tables: np.ndarray):
    """Per brick the (mode, table) with the fewest estimated bits (float estimate, for fitting only)."""
    cost = np.einsum("bms,ts->bmt", hist.astype(np.float64), table_bits(tables))
    flat = cost.reshape(len(hist), -1).argmin(1)
    return flat // len(tables), flat % len(tables), cost


def fit_tables(hist: np.ndarray, n_tables: int = TABLES, iters: int = 10, seed: int = 0) -> np.ndarray:
    """Shared tables by alternating assignment (each brick to its cheapest (mode, table)) and refit
    (each table from the histograms of its bricks), started from k-means++ seeds on the mode-0
    histograms."""
    rng = np.random.default_rng(seed)
    h0 = hist[:, 0].astype(np.float64)
    p0 = (h0 + 0.5) / (h0 + 0.5).sum(1, keepdims=True)
    centers = [p0[rng.integers(len(p0))]]
    for _ in range(1, n_tables):
        d = np.min([np.sum(p0 * np.log(p0 / c), 1) for c in centers], 0)  # KL to the nearest centre
        centers.append(p0[rng.choice(len(p0), p=d / d.sum()) if d.sum() > 0 else rng.integers(len(p0))])
    tables = np.stack([build_model(c * 1e6) for c in centers])
    for _ in range(iters):
        m, t, _ = choose(hist, tables)
        new = tables.copy()
        for k in range(n_tables):
            sel = t == k
            if sel.any():
                new[k] = build_model(hist[np.nonzero(sel)[0], m[sel]].sum(0))
        if np.array_equal(new, tables):
            break
        tables = new
    return tables


def train(codec: Codec, d_features, d_labels, steps: int = 600, batch: int = 1024, lr: float = 2e-3, seed: int = 0,
          net: SelectorNet | None = None):
    """Adam on the mean cross-entropy of both heads against the exhaustive labels; minibatches drawn on the
    device.  Returns the network and the loss per step."""
    import torch
    net = net or SelectorNet(codec, SelectorNet.init_params(seed))
    g = torch.Generator(device=d_features.device)
    g.manual_seed(seed)
    n = d_features.shape[0]
    losses = []
    for step in range(steps):
        idx = torch.randint(0, n, (min(batch, n),), device=d_features.device, generator=g)
        f = d_features[idx].contiguous()
        y = d_labels[idx].contiguous()
        losses.append(net.grad(f, y))
        net.adam(lr * (0.5 * (1 + np.cos(np.pi * step / steps))) + 1e-5)
    return net, losses


def learned_choice(net: SelectorNet, d_features):
    """Per brick mode | table << 4 from the network's argmax (uint8 device tensor)."""
    import torch
    sel = torch.empty(d_features.shape[0], dtype=torch.uint8, device=d_features.device)
    net.forward(d_features, d_sel=sel)
    return sel


def exhaustive_choice(codec: Codec, d_volume, brick: int, tables: np.ndarray):
    """Per brick mode | table << 4 from the exhaustive search, and the per-mode histograms."""
    import torch
    D, H, W = d_volume.shape
    nb = -(-W // brick) * -(-H // brick) * -(-D // brick)
    hist = torch.empty((nb, MODES, 16), dtype=torch.int32, device=d_volume.device)
    codec.encode_stats(d_volume, brick, hist)
    sel = torch.empty(nb, dtype=torch.uint8, device=d_volume.device)
    codec.select_exhaustive(hist, tables, sel)
    return sel, hist


def features(codec: Codec, d_volume, brick: int):
    import torch
    D, H, W = d_volume.shape
    nb = -(-W // brick) * -(-H // brick) * -(-D // brick)
    f = torch.empty((nb, FEATURES), dtype=torch.float32, device=d_volume.device)
    codec.brick_features(d_volume, brick, f)
    return f
