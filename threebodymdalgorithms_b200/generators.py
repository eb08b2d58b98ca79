"""Particle inputs identical to the reference's particlegenerator (src/tools), without running it.

UniformGenerator::Generate (src/tools/UniformGenerator.cpp:12-28) draws, per particle and axis,
std::uniform_real_distribution<double>(0, 1) from std::mt19937(seed0); libstdc++ forms each
double from two 32-bit outputs as (x1 + x2 * 2^32) / 2^64 (generate_canonical<double, 53>).
ClusteredGaussGenerator::Generate (src/tools/ClusteredGaussGenerator.cpp:15-47) places
numClusters centres uniformly with std::mt19937(seed1), then numParticles/numClusters particles
per centre offset by three std::normal_distribution<double> objects (one per axis, each caching
its second Marsaglia-polar value) driven by one std::default_random_engine(seed0), which is
minstd_rand0 in libstdc++.  The reference builds each particle with std::make_tuple(...), whose
arguments GCC evaluates right to left, so every particle (and cluster centre) draws z, then y, then
x.  The reference writes these values to CSV with 6 significant digits
and reads them back, so `as_csv_values` applies that same rounding.
"""
from __future__ import annotations

import math

import numpy as np

SEED0, SEED1 = 926762934, 89347587


def _mt19937_raw(seed: int, count: int) -> np.ndarray:
    bg = np.random.MT19937()
    bg._legacy_seeding(seed & 0xFFFFFFFF)  # init_genrand, the same seeding as std::mt19937(seed)
    return bg.random_raw(count).astype(np.uint64)


def _canonical_from_pairs(raw: np.ndarray) -> np.ndarray:
    lo = raw[0::2].astype(np.float64)
    hi = raw[1::2].astype(np.float64)
    v = (lo + hi * 4294967296.0) / 18446744073709551616.0
    return np.where(v >= 1.0, np.nextafter(1.0, 0.0), v)


def uniform(n: int, box=(10.0, 10.0, 10.0), mass: float = 1.0, seed0: int = SEED0, corner=(0.0, 0.0, 0.0),
            velocity=(0.0, 0.0, 0.0)) -> dict:
    u = _canonical_from_pairs(_mt19937_raw(seed0, 6 * n)).reshape(n, 3)[:, ::-1]  # draws z, y, x
    st = {"id": np.arange(n, dtype=np.int32)}
    for d, k in enumerate("xyz"):
        st[k] = corner[d] + u[:, d] * box[d]
    for d, k in enumerate(("vx", "vy", "vz")):
        st[k] = np.full(n, float(velocity[d]))
    for k in ("ax", "ay", "az"):
        st[k] = np.zeros(n)
    st["m"] = np.full(n, float(mass))
    return st


class _MinstdRand0:
    M = 2147483647

    def __init__(self, seed: int):
        s = seed % self.M
        self.x = 1 if s == 0 else s

    def __call__(self) -> int:
        self.x = (self.x * 16807) % self.M
        return self.x

    def canonical(self) -> float:
        r = 2147483646.0  # max - min + 1 with min = 1, max = 2^31 - 2
        a = float(self() - 1)
        b = float(self() - 1)
        v = (a + b * r) / (r * r)
        return math.nextafter(1.0, 0.0) if v >= 1.0 else v


class _Normal:
    """libstdc++ std::normal_distribution<double> (Marsaglia polar method with a cached value)."""

    def __init__(self, mean: float, stddev: float):
        self.mean, self.stddev = mean, stddev
        self.saved = None

    def __call__(self, eng: _MinstdRand0) -> float:
        if self.saved is not None:
            ret, self.saved = self.saved, None
        else:
            while True:
                x = 2.0 * eng.canonical() - 1.0
                y = 2.0 * eng.canonical() - 1.0
                r2 = x * x + y * y
                if not (r2 > 1.0 or r2 == 0.0):
                    break
            mult = math.sqrt(-2.0 * math.log(r2) / r2)
            self.saved = x * mult
            ret = y * mult
        return ret * self.stddev + self.mean


def clustered_gauss(n: int, n_clusters: int, box=(64.0, 64.0, 64.0), mean: float = 0.0, stddev: float = 1.0,
                    mass: float = 1.0, seed0: int = SEED0, seed1: int = SEED1, corner=(0.0, 0.0, 0.0)) -> dict:
    cu = _canonical_from_pairs(_mt19937_raw(seed1, 6 * n_clusters)).reshape(n_clusters, 3)[:, ::-1]
    centres = [tuple(corner[d] + cu[c, d] * box[d] for d in range(3)) for c in range(n_clusters)]
    eng = _MinstdRand0(seed0)
    dist = [_Normal(mean, stddev) for _ in range(3)]
    per = n // n_clusters
    pos = np.empty((per * n_clusters, 3))
    q = 0
    for cx, cy, cz in centres:
        for _ in range(per):
            pos[q, 2] = cz + dist[2](eng)
            pos[q, 1] = cy + dist[1](eng)
            pos[q, 0] = cx + dist[0](eng)
            q += 1
    m = len(pos)
    st = {"id": np.arange(m, dtype=np.int32), "x": pos[:, 0].copy(), "y": pos[:, 1].copy(), "z": pos[:, 2].copy()}
    for k in ("vx", "vy", "vz", "ax", "ay", "az"):
        st[k] = np.zeros(m)
    st["m"] = np.full(m, float(mass))
    return st


def as_csv_values(st: dict) -> dict:
    """Round every value to 6 significant digits, as the reference's CSV write + read does."""
    out = dict(st)
    fmt = np.vectorize(lambda v: float("%g" % v), otypes=[np.float64])
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m"):
        a = np.asarray(st[k], dtype=np.float64)
        out[k] = a.copy() if not a.any() else fmt(a)
    return out


def box_for_density(n: int, density: float = 2.048) -> float:
    """Cube side with n / side^3 = density (131072 at 2.048 gives 40.0)."""
    return (n / density) ** (1.0 / 3.0)


def batch_of_systems(count: int = 64, nmin: int = 512, nmax: int = 4096, density: float = 2.048,
                     seed: int = SEED0) -> list:
    """Independent systems for the batched path: system i has N_i drawn uniformly from nmin..nmax
    (numpy's default generator seeded with `seed`) and is uniform in a cube scaled to `density`,
    drawn like UniformGenerator with seed0 = seed + i.  With the defaults this is the 64-system
    workload of the batched benchmark."""
    rng = np.random.default_rng(seed)
    systems = []
    for i in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        side = box_for_density(n, density)
        systems.append(uniform(n, (side,) * 3, seed0=seed + i))
    return systems


def pack_systems(systems: list):
    """Concatenate systems back to back: (offsets[count + 1], {'x','y','z'} arrays)."""
    offsets = np.cumsum([0] + [len(s["x"]) for s in systems]).astype(np.int64)
    cat = {k: np.concatenate([s[k] for s in systems]) for k in ("x", "y", "z")}
    return offsets, cat
