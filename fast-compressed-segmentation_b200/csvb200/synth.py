"""Seeded synthetic label volumes (CPU, numpy) for small test cases.

The reference's real input is a MICrONS segmentation cut-out downloaded over
the network (dataset/dataset_downloader.py); it is not available here, so the
codec is exercised on synthetic volumes with the same dtype, layout and
structure: uint64 labels, x fastest (``vol[z, y, x]``, i.e.
``data[x + W*(y + H*z)]`` as brick.hpp:183 reads it), IDs in [1, 2^64-2]
(UINT64_MAX is the decoder's empty sentinel, types.hpp:19).

Large volumes (512^3 and up) are generated on the GPU by ``csv_synth_volume``
in the native library; these numpy versions serve the CPU tests.
"""
from __future__ import annotations

import numpy as np

MAX_ID = np.uint64(0xFFFFFFFFFFFFFFFE)


def random_ids(rng: np.random.Generator, n: int) -> np.ndarray:
    ids = rng.integers(1, 2 ** 63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n, dtype=np.uint64)
    ids = np.minimum(np.maximum(ids, np.uint64(1)), MAX_ID)
    return ids


def voronoi(shape, n_cells: int, seed: int, zero_slab: float = 0.10) -> np.ndarray:
    """Voronoi partition of ``n_cells`` uniform seed points (nearest seed to
    the voxel centre, Euclidean; ties go to the lower seed index), each cell a
    random 64-bit ID, then a random half-space slab of label 0 covering about
    ``zero_slab`` of the volume."""
    from scipy.spatial import cKDTree

    D, H, W = shape
    rng = np.random.default_rng(seed)
    pts = rng.random((n_cells, 3)) * np.array([W, H, D])
    ids = random_ids(rng, n_cells)
    tree = cKDTree(pts)
    zz, yy, xx = np.meshgrid(np.arange(D) + 0.5, np.arange(H) + 0.5, np.arange(W) + 0.5, indexing="ij")
    q = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    _, idx = tree.query(q, k=1)
    vol = ids[idx].reshape(D, H, W)
    if zero_slab > 0:
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        d = q @ n
        thr = np.quantile(d, 1.0 - zero_slab)
        vol.reshape(-1)[d >= thr] = 0
    return vol


def tubes_over_voronoi(shape, n_cells: int, n_tubes: int, r_min: float, r_max: float, seed: int,
                       zero_frac: float = 0.15) -> np.ndarray:
    """Neurite-like volume: random cubic (Catmull-Rom) tubes with radius in
    [r_min, r_max] and random IDs laid over a Voronoi background whose cells
    are set to label 0 until about ``zero_frac`` of the background is 0."""
    D, H, W = shape
    rng = np.random.default_rng(seed + 7919)
    vol = voronoi(shape, n_cells, seed, zero_slab=0.0)
    cells = np.unique(vol)
    rng.shuffle(cells)
    zero_cells = cells[: max(1, int(len(cells) * zero_frac))]
    vol[np.isin(vol, zero_cells)] = 0
    from scipy.spatial import cKDTree

    ids = random_ids(rng, n_tubes)
    ext = np.array([W, H, D], dtype=np.float64)
    for t in range(n_tubes):
        ctrl = rng.random((4, 3)) * ext
        r = rng.uniform(r_min, r_max)
        # the Catmull-Rom segment between ctrl[1] and ctrl[2], sampled densely
        p0, p1, p2, p3 = ctrl
        n_s = int(max(8, 4 * np.linalg.norm(p2 - p1)))
        ts = np.linspace(0, 1, n_s)[:, None]
        pts = 0.5 * ((2 * p1)[None] + (-p0 + p2)[None] * ts + (2 * p0 - 5 * p1 + 4 * p2 - p3)[None] * ts ** 2
                     + (-p0 + 3 * p1 - 3 * p2 + p3)[None] * ts ** 3)
        lo = np.maximum(np.floor(pts.min(0) - r).astype(int), 0)
        hi = np.minimum(np.ceil(pts.max(0) + r).astype(int) + 1, [W, H, D])
        if np.any(hi <= lo):
            continue
        zz, yy, xx = np.meshgrid(np.arange(lo[2], hi[2]) + 0.5, np.arange(lo[1], hi[1]) + 0.5,
                                 np.arange(lo[0], hi[0]) + 0.5, indexing="ij")
        q = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
        d, _ = cKDTree(pts).query(q, k=1, distance_upper_bound=r)
        sub = vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        sub[(d < r).reshape(sub.shape)] = ids[t]
    return vol
