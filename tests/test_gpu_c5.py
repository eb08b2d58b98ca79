"""The batched differentiation workload at full size: 64 independent systems with N uniform in
512..4096, each uniform at density 2.048 (143,846 particles), in one batched call.

- Forward, mixed precision, against the oracle system by system: P3BCA (cutoff 2) counts bit-exact
  and forces within 1e-5 relative L2 on all 64 systems; AUTA (no cutoff, C(N,3) triplets per
  system) counts exact on all 64 and forces on a sample of particles of 8 systems (the oracle's
  O(N^2) per-particle sum, since the full O(N^3) oracle is too slow at N = 4096).
- The batched adjoint of the force-matching loss
      L = sum_s sum_i |f_i(x; nu) - T_i|^2,   T = FP64 forces at 1.1 nu (held fixed),
  in mixed precision and in FP64 (cotangent 2 (f - T) on the forces, none on the energy), against
  FP64 central finite differences with h = 1e-6 on 8 of the systems: the position gradient on 24
  coordinates per system (the 4 particles with the largest gradient and 4 seeded random ones; a
  coordinate whose perturbation moves a triplet across the cutoff, where the truncated potential
  jumps, is skipped, at most 4 per system) and dL/dnu.  The loss of the finite differences is
  evaluated by the FP64 forward on that system alone with its domain held fixed.
  Tolerances, relative over the sampled coordinates of a system: FP64 1e-6.  Mixed: 1e-5 plus the
  relative difference between the mixed and the FP64 cotangent 2 (f - T) of that system.  The mixed
  pipeline differentiates its own loss, whose cotangent carries the mixed forward's rounding: since
  T is the force at 1.1 nu, f - T is a tenth of f, so a force error of 1e-6 is 1e-5 of the cotangent,
  and it passes into the gradient unchanged (measured: 1.3e-5 on system 13, 1e-6 HVP error aside).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from threebodymdalgorithms_b200 import Context, generators

pytestmark = pytest.mark.gpu

H = 1e-6
NU = 1.0
FD_SYSTEMS = (0, 6, 13, 21, 30, 38, 47, 63)  # 8 of the 64 (system 6 is the smallest, N = 537)


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.fixture(scope="module")
def c5():
    systems = generators.batch_of_systems(64, 512, 4096, 2.048)
    offsets, cat = generators.pack_systems(systems)
    assert int(offsets[-1]) == 143846
    return systems, offsets, cat


def test_c5_batched_p3bca_forward_vs_oracle(c5):
    systems, offsets, cat = c5
    ctx = Context("p3bca", "mixed", 2.0)
    fx, fy, fz, energy, counts = ctx.batch_forces(offsets, cat["x"], cat["y"], cat["z"])
    ctx.close()
    for s, st in enumerate(systems):
        sl = slice(offsets[s], offsets[s + 1])
        L, lo = O.domain(st["x"], st["y"], st["z"])
        rx, ry, rz, rc = O.forces(st["x"], st["y"], st["z"], NU, 2.0, L, lo, nthreads=0)
        assert int(counts[s]) == rc, (s, counts[s], rc)
        got = np.stack([fx[sl], fy[sl], fz[sl]], 1)
        assert rel_l2(got, np.stack([rx, ry, rz], 1)) <= 1e-5, s


def test_c5_batched_auta_forward_vs_oracle(c5):
    systems, offsets, cat = c5
    ctx = Context("auta", "mixed")
    fx, fy, fz, energy, counts = ctx.batch_forces(offsets, cat["x"], cat["y"], cat["z"])
    ctx.close()
    for s, st in enumerate(systems):
        n = len(st["x"])
        assert int(counts[s]) == math.comb(n, 3), s
    rng = np.random.default_rng(5)
    for s in FD_SYSTEMS:
        st = systems[s]
        idx = np.sort(rng.choice(len(st["x"]), 8, replace=False))
        ref = np.stack(O.forces_selected(st["x"], st["y"], st["z"], idx, NU, nthreads=0), 1)
        o = offsets[s]
        got = np.stack([fx[o + idx], fy[o + idx], fz[o + idx]], 1)
        assert rel_l2(got, ref) <= 1e-5, (s, rel_l2(got, ref))


def _one_system_loss(ctx, st, target, L, lo):
    """Force-matching loss of one system with FP64 forces at nu = NU, its domain held fixed."""
    n = len(st["x"])
    fx, fy, fz, e, c = ctx.batch_forces(np.array([0, n], dtype=np.int64), st["x"], st["y"], st["z"],
                                        box=L, lo=lo)
    f = np.stack([fx, fy, fz], 1)
    return float(((f - target) ** 2).sum()), int(c[0])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("mixed", 1e-5)])
def test_c5_force_matching_gradients_vs_finite_differences(c5, precision, tol):
    systems, offsets, cat = c5
    nsys = len(systems)
    # per-system domains, fixed for the finite differences
    doms = [O.domain(st["x"], st["y"], st["z"]) for st in systems]
    box = np.stack([d[0] for d in doms])
    lo = np.stack([d[1] for d in doms])
    tgt = Context("p3bca", "fp64", 2.0, nu=1.1 * NU)
    T = tgt.batch_forces(offsets, cat["x"], cat["y"], cat["z"], box=box, lo=lo)
    tgt.close()
    target = np.stack(T[:3], 1)
    ctx = Context("p3bca", precision, 2.0, nu=NU)
    f = ctx.batch_forces(offsets, cat["x"], cat["y"], cat["z"], box=box, lo=lo)
    gf = 2.0 * (np.stack(f[:3], 1) - target)
    ref = Context("p3bca", "fp64", 2.0, nu=NU)
    gf64 = 2.0 * (np.stack(ref.batch_forces(offsets, cat["x"], cat["y"], cat["z"], box=box, lo=lo)[:3], 1) - target)
    ref.close()
    gx, gy, gz, gnu = ctx.batch_adjoint(offsets, cat["x"], cat["y"], cat["z"], gf[:, 0], gf[:, 1], gf[:, 2],
                                        np.zeros(nsys), box=box, lo=lo)
    ctx.close()
    g = np.stack([gx, gy, gz], 1)
    fd_ctx = Context("p3bca", "fp64", 2.0, nu=NU)
    fd_nu_p = Context("p3bca", "fp64", 2.0, nu=NU + H)
    fd_nu_m = Context("p3bca", "fp64", 2.0, nu=NU - H)
    rng = np.random.default_rng(17)
    for s in FD_SYSTEMS:
        st = {k: systems[s][k].copy() for k in ("x", "y", "z")}
        n = len(st["x"])
        o = offsets[s]
        Ts = target[o:o + n]
        gs = g[o:o + n]
        _, c0 = _one_system_loss(fd_ctx, st, Ts, box[s], lo[s])
        big = np.argsort(-np.linalg.norm(gs, axis=1))[:4]
        rnd = rng.choice(np.setdiff1d(np.arange(n), big), 4, replace=False)
        got, fd = [], []
        for i in np.concatenate([big, rnd]):
            for d, k in enumerate("xyz"):
                st[k][i] += H
                lp, cp = _one_system_loss(fd_ctx, st, Ts, box[s], lo[s])
                st[k][i] -= 2 * H
                lm, cm = _one_system_loss(fd_ctx, st, Ts, box[s], lo[s])
                st[k][i] += H
                # the truncated potential jumps where a triplet crosses the cutoff: a coordinate
                # whose perturbation moves a triplet across it has no finite difference
                if cp != c0 or cm != c0:
                    continue
                got.append(gs[i, d])
                fd.append((lp - lm) / (2 * H))
        assert len(got) >= 20, (s, len(got))
        got, fd = np.array(got), np.array(fd)
        # the cotangent's own rounding (zero for FP64, where gf is gf64)
        tol_s = tol + rel_l2(gf[o:o + n], gf64[o:o + n])
        assert rel_l2(got, fd) <= tol_s, (precision, s, rel_l2(got, fd), tol_s)
        # dL/dnu (forces are linear in nu: the loss is a quadratic in nu)
        lp, _ = _one_system_loss(fd_nu_p, st, Ts, box[s], lo[s])
        lm, _ = _one_system_loss(fd_nu_m, st, Ts, box[s], lo[s])
        fd_nu = (lp - lm) / (2 * H)
        assert abs(gnu[s] - fd_nu) <= tol_s * abs(fd_nu), (precision, s, gnu[s], fd_nu)
    for c in (fd_ctx, fd_nu_p, fd_nu_m):
        c.close()
