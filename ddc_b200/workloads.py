"""Seeded synthetic inputs of the five benchmark configurations (shared by tests and bench.py).

Random numbers: splitmix64 streams turned into 53-bit uniforms; the seed of configuration c is
0xDDC0 + c and every quantity draws from its own stream (stream id in the high bits).
Arrays use the (row, line) layout with the batch contiguous: DDC's (x, batch) layout_right.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix_uniform(seed: int, stream: int, n: int) -> np.ndarray:
    """n uniforms in [0, 1) from the splitmix64 sequence of (seed, stream)."""
    return splitmix_at(seed, stream, np.arange(n, dtype=np.uint64))


def splitmix_at(seed: int, stream: int, idx) -> np.ndarray:
    """Uniforms number idx (0-based, any shape) of the splitmix64 sequence of (seed, stream): a shard
    of a batch draws exactly the numbers the whole batch would give its lines."""
    idx = np.asarray(idx, dtype=np.uint64)
    with np.errstate(over="ignore"):
        base = np.uint64((seed + (stream << 40)) & 0xFFFFFFFFFFFFFFFF)
        x = base + ((idx + np.uint64(1)) * _GOLDEN)
        z = x
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def cos_family(x, k, ph, order=0):
    """d^order/dx^order cos(2 pi k x + ph) (the reference's CosineEvaluator, cosine_evaluator.hpp:78-81)."""
    return (2 * np.pi * k) ** order * np.cos(np.pi / 2 * order + 2 * np.pi * k * x + ph)


def config1(B: int = 1000, ncells: int = 1000, m: int = 1000):
    """Periodic uniform cubic on [0,1): samples at the Greville points x_i = i/ncells, eval near grid points."""
    seed = 0xDDC0 + 1
    h = 1.0 / ncells
    x = np.arange(ncells) * h
    k = np.floor(splitmix_uniform(seed, 1, B) * 8).astype(np.int64) + 1
    ph = splitmix_uniform(seed, 2, B) * 2 * np.pi
    vals = cos_family(x[:, None], k[None, :], ph[None, :])
    pts_idx = np.arange(m) % ncells
    coords = (pts_idx * h)[:, None] + (splitmix_uniform(seed, 3, m * B).reshape(m, B) - 0.5) * h
    coords = np.mod(coords, 1.0)
    return dict(degree=3, ncells=ncells, x=x, k=k, ph=ph, vals=np.ascontiguousarray(vals),
                coords=np.ascontiguousarray(coords))


def config2_breaks(ncells: int = 1024):
    seed = 0xDDC0 + 2
    h = 1.0 / ncells
    br = np.arange(ncells + 1) * h
    br[1:-1] += (splitmix_uniform(seed, 1, ncells - 1) - 0.5) * 0.6 * h
    br.sort()
    br[0], br[-1] = 0.0, 1.0
    return br


def config2(B: int = 1 << 16, ncells: int = 1024, m: int = 1024, points=None, line0: int = 0, total=None):
    """Non-uniform quintic, Hermite closures (derivative orders 1 and 2 per side), d/dx evaluation.
    Lines [line0, line0 + B) of a batch of `total` lines (default B): a rank's shard of a larger
    batch holds the same inputs as those lines of the whole batch."""
    seed = 0xDDC0 + 2
    total = B if total is None else total
    if not 0 <= line0 and line0 + B <= total:
        raise ValueError("the lines must lie inside the batch")
    br = config2_breaks(ncells)
    lines = np.arange(line0, line0 + B, dtype=np.uint64)
    k = np.floor(splitmix_at(seed, 2, lines) * 8).astype(np.int64) + 1
    ph = splitmix_at(seed, 3, lines) * 2 * np.pi
    out = dict(degree=5, ncells=ncells, breaks=br, k=k, ph=ph)
    if points is not None:
        out["vals"] = np.ascontiguousarray(cos_family(points[:, None], k[None, :], ph[None, :]))
        out["dlo"] = np.ascontiguousarray(np.stack([cos_family(0.0, k, ph, o) for o in (1, 2)]))
        out["dhi"] = np.ascontiguousarray(np.stack([cos_family(1.0, k, ph, o) for o in (1, 2)]))
    idx = np.arange(m, dtype=np.uint64)[:, None] * np.uint64(total) + lines[None, :]
    out["coords"] = np.ascontiguousarray(splitmix_at(seed, 4, idx))
    return out


def config3(nfields: int = 64, ncells: int = 512):
    """2D: x periodic cubic uniform (ncells) x y Hermite cubic uniform (ncells) on [0,1)x[0,1];
    f = sin(2 pi x) cos(pi y) a_b + 0.01 N(0,1), evaluation at the semi-Lagrangian feet
    (x - v dt, y), v ~ U[-1,1] per y row, dt = h/2. Arrays in (x, y, field) layout."""
    seed = 0xDDC0 + 3
    h = 1.0 / ncells
    x = np.arange(ncells) * h                 # periodic cubic Greville points
    y = np.arange(ncells + 1) * h             # Hermite cubic points (break points)
    a = 0.5 + 1.5 * splitmix_uniform(seed, 1, nfields)
    u1 = splitmix_uniform(seed, 2, ncells * (ncells + 1) * nfields)
    u2 = splitmix_uniform(seed, 3, ncells * (ncells + 1) * nfields)
    noise = (np.sqrt(-2.0 * np.log(np.maximum(u1, 1e-300))) * np.cos(2 * np.pi * u2)).reshape(ncells, ncells + 1, nfields)
    base = np.sin(2 * np.pi * x)[:, None, None] * np.cos(np.pi * y)[None, :, None]
    vals = base * a[None, None, :] + 0.01 * noise
    # d/dy at y=0 and y=1 of the smooth part (the noise has no derivative): -pi sin(pi y) = 0 at both ends
    dmin2 = np.zeros((ncells, 1, nfields))
    dmax2 = np.zeros((ncells, 1, nfields))
    v = 2.0 * splitmix_uniform(seed, 4, ncells + 1) - 1.0
    dt = 0.5 * h
    feet_x = x[:, None, None] - v[None, :, None] * dt + np.zeros((1, 1, nfields))
    feet_y = y[None, :, None] + np.zeros((ncells, 1, nfields))
    coords = np.ascontiguousarray(np.stack([feet_x, feet_y], axis=-1))
    return dict(x=x, y=y, vals=np.ascontiguousarray(vals), dmin2=dmin2, dmax2=dmax2, coords=coords, ncells=ncells,
                nfields=nfields, v=v, dt=dt)


def config4(count: int = 4096, nmin: int = 32, nmax: int = 4096, seed: int = 0xDDC0 + 4):
    """Uneven batch: `count` one-line problems, ncells log-uniform in [nmin, nmax], degree uniform in
    1..5, closure uniform in {periodic, Hermite, Greville} (both ends), uniform or perturbed
    (+-0.3 h) mesh on [0, 1], cos(2 pi k x + phi) samples (k in 1..8) with analytic Hermite
    derivatives, evaluation at ncells uniform points per problem."""
    u = splitmix_uniform(seed, 1, count)
    nc = np.floor(np.exp(np.log(nmin) + u * (np.log(nmax + 1) - np.log(nmin)))).astype(np.int64)
    nc = np.clip(nc, nmin, nmax)
    deg = np.floor(splitmix_uniform(seed, 2, count) * 5).astype(np.int64) + 1
    bc = np.floor(splitmix_uniform(seed, 3, count) * 3).astype(np.int64)  # 0 periodic, 1 Hermite, 2 Greville
    uni = splitmix_uniform(seed, 4, count) < 0.5
    k = np.floor(splitmix_uniform(seed, 5, count) * 8).astype(np.int64) + 1
    ph = splitmix_uniform(seed, 6, count) * 2 * np.pi
    probs = []
    for i in range(count):
        n = int(nc[i])
        p = dict(ncells=n, degree=int(deg[i]), closure=("periodic", "hermite", "greville")[int(bc[i])],
                 uniform=bool(uni[i]), k=int(k[i]), ph=float(ph[i]))
        if not p["uniform"]:
            h = 1.0 / n
            br = np.arange(n + 1) * h
            br[1:-1] += (splitmix_uniform(seed + i + 1, 7, n - 1) - 0.5) * 0.6 * h
            br.sort()
            br[0], br[-1] = 0.0, 1.0
            p["breaks"] = br
        p["coords"] = splitmix_uniform(seed + i + 1, 8, n)
        probs.append(p)
    return probs


def config4_samples(p, points, nbv_lo, nbv_hi):
    """Samples at the interpolation points and the Hermite derivatives (orders 1.. at each end)."""
    vals = cos_family(points, p["k"], p["ph"])
    lo = np.array([cos_family(0.0, p["k"], p["ph"], o) for o in range(1, nbv_lo + 1)])
    hi = np.array([cos_family(1.0, p["k"], p["ph"], o) for o in range(1, nbv_hi + 1)])
    return vals, lo, hi


def config4_batch(D, probs, precision="fp64", refine_rounds=2):
    """Builders, evaluators and packed host inputs (flat arrays in problem order) of config4
    problems; `D` is the ddc_b200 package. Each builder solves one line, cut into whole warps of
    chunks: ceil(rows / 512) warps of 32 chunks (at most 16 rows per chunk; problems under 512
    rows take one warp, with chunks as short as the band allows), so no thread of a problem's
    block idles and the chunk sweeps are as short as the warp count permits. precision
    "fp32_refine" builds every problem in FP32 with FP64 refinement."""
    closure = {"periodic": 0, "hermite": 1, "greville": 3}
    builders, evaluators, nevals = [], [], []
    vals, dlo, dhi, coords = [], [], [], []
    for p in probs:
        n, d = p["ncells"], p["degree"]
        per = p["closure"] == "periodic"
        bs = D.UniformBSplines(d, per, 0.0, 1.0, n) if p["uniform"] else D.NonUniformBSplines(d, per, p["breaks"])
        c = closure[p["closure"]]
        chunks = 32 * max(1, -(-bs.size // 512))
        b = D.SplineBuilder(bs, None, c, c, tile_lines=2, chunks=int(min(chunks, 512)), precision=precision,
                            refine_rounds=refine_rounds)
        e = D.SplineEvaluator(bs)
        nlo = b.s_nbv_xmin if c == 1 else 0
        nhi = b.s_nbv_xmax if c == 1 else 0
        v, lo, hi = config4_samples(p, b.interpolation_points, nlo, nhi)
        builders.append(b)
        evaluators.append(e)
        nevals.append(len(p["coords"]))
        vals.append(v)
        dlo.append(lo)
        dhi.append(hi)
        coords.append(p["coords"])
    cat = lambda xs: np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in xs]))
    return dict(builders=builders, evaluators=evaluators, nevals=np.array(nevals, dtype=np.int64), vals=cat(vals),
                dlo=cat(dlo), dhi=cat(dhi), coords=cat(coords))
