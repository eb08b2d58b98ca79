"""Batched systems (one launch over many independent systems of uneven N) and the torch.autograd
harness, against per-system evaluations and the oracle."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from threebodymdalgorithms_b200 import Context, generators

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def make_systems(count, nmin, nmax, seed=11):
    rng = np.random.default_rng(seed)
    systems = []
    for s in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        side = generators.box_for_density(n, 2.048)
        systems.append(generators.uniform(n, (side,) * 3, seed0=926762934 + s))
    return systems


def pack(systems):
    offsets = np.cumsum([0] + [len(s["x"]) for s in systems]).astype(np.int64)
    cat = {k: np.concatenate([s[k] for s in systems]) for k in ("x", "y", "z")}
    return offsets, cat


@pytest.mark.parametrize("algo,cutoff", [("auta", 0.0), ("p3bca", 2.0)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_batch_forces_match_single_systems(algo, cutoff, precision, tol):
    systems = make_systems(9, 3, 700)
    offsets, cat = pack(systems)
    ctx = Context(algo, precision, cutoff)
    fx, fy, fz, energy, counts = ctx.batch_forces(offsets, cat["x"], cat["y"], cat["z"])
    for s, st in enumerate(systems):
        sl = slice(offsets[s], offsets[s + 1])
        L, lo = O.domain(st["x"], st["y"], st["z"])
        rf = O.forces(st["x"], st["y"], st["z"], 1.0, cutoff if cutoff > 0 else -1.0, L, lo, nthreads=0)
        assert int(counts[s]) == rf[3], (s, counts[s], rf[3])
        ref = np.stack(rf[:3], 1)
        got = np.stack([fx[sl], fy[sl], fz[sl]], 1)
        assert rel_l2(got, ref) <= tol, (s, rel_l2(got, ref))
        e_ref = O.energy(st["x"], st["y"], st["z"], 1.0, cutoff if cutoff > 0 else -1.0, L, lo)
        # relative to the magnitude scale of the terms, which have both signs (see test_gpu_parity):
        # the FP64 sum's order follows the device's atomics, so its rounding is bounded by that scale
        e_abs = O.energy_abs(st["x"], st["y"], st["z"], 1.0, cutoff if cutoff > 0 else -1.0, L, lo)
        etol = 1e-12 if precision == "fp64" else 2e-6
        assert abs(energy[s] - e_ref) <= etol * max(e_abs, 1e-30), (s, energy[s], e_ref, e_abs)
    ctx.close()


@pytest.mark.parametrize("algo,cutoff", [("auta", 0.0), ("p3bca", 2.0)])
def test_batch_adjoint_matches_single_systems(algo, cutoff):
    systems = make_systems(5, 20, 300, seed=3)
    offsets, cat = pack(systems)
    rng = np.random.default_rng(1)
    gf = rng.normal(size=(len(cat["x"]), 3))
    ge = rng.normal(size=len(systems))
    ctx = Context(algo, "fp64", cutoff, nu=1.1)
    gx, gy, gz, gnu = ctx.batch_adjoint(offsets, cat["x"], cat["y"], cat["z"], gf[:, 0], gf[:, 1], gf[:, 2], ge)
    for s, st in enumerate(systems):
        sl = slice(offsets[s], offsets[s + 1])
        one = Context(algo, "fp64", cutoff, nu=1.1)
        one.set_state(st)
        rx, ry, rz, rnu = one.adjoint(gf[sl, 0], gf[sl, 1], gf[sl, 2], ge[s])
        one.close()
        assert rel_l2(np.stack([gx[sl], gy[sl], gz[sl]], 1), np.stack([rx, ry, rz], 1)) <= 1e-12
        assert abs(gnu[s] - rnu) <= 1e-12 * abs(rnu)
    ctx.close()


def test_c5_shape_batch():
    """C5's shape: 64 systems with N uniform in 512..4096 at density 2.048, P3BCA c=2, mixed; counts
    against the FP64 batch and forces within the mixed tolerance."""
    systems = make_systems(64, 512, 4096, seed=926762934)
    offsets, cat = pack(systems)
    a = Context("p3bca", "fp64", 2.0)
    b = Context("p3bca", "mixed", 2.0)
    fa = a.batch_forces(offsets, cat["x"], cat["y"], cat["z"])
    fb = b.batch_forces(offsets, cat["x"], cat["y"], cat["z"])
    assert np.array_equal(fa[4], fb[4]) and int(fa[4].sum()) > 0
    assert rel_l2(np.stack(fb[:3], 1), np.stack(fa[:3], 1)) <= 1e-5
    a.close()
    b.close()


def torch_at_energy(x, nu):
    import torch
    i, j, k = torch.combinations(torch.arange(x.shape[0], device=x.device), 3).T
    u, v, w = x[j] - x[i], x[k] - x[i], x[k] - x[j]
    uu, vv, ww = (u * u).sum(1), (v * v).sum(1), (w * w).sum(1)
    cosprod = -((u * v).sum(1) * (u * w).sum(1) * (v * w).sum(1)) / (uu * vv * ww)
    return (nu * (1 + 3 * cosprod) / (uu * vv * ww) ** 1.5).sum()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_autograd_harness(precision, tol):
    torch = pytest.importorskip("torch")
    from threebodymdalgorithms_b200.autograd import AxilrodTeller
    st = generators.uniform(16, (2.5, 2.5, 2.5))
    x0 = np.stack([st["x"], st["y"], st["z"]], 1)
    rng = np.random.default_rng(2)
    gf = torch.tensor(rng.normal(size=(16, 3)), dtype=torch.float64, device="cuda")
    # reference: torch FP64 AT energy, forces = +grad E by autograd
    xr = torch.tensor(x0, dtype=torch.float64, device="cuda", requires_grad=True)
    nur = torch.tensor(1.25, dtype=torch.float64, device="cuda", requires_grad=True)
    er = torch_at_energy(xr, nur)
    (fr,) = torch.autograd.grad(er, xr, create_graph=True)
    lr = (gf * fr).sum() + 0.3 * er
    gx_ref, gnu_ref = torch.autograd.grad(lr, (xr, nur))
    # the CUDA harness
    at = AxilrodTeller("auta", precision)
    x = torch.tensor(x0, dtype=torch.float64, device="cuda", requires_grad=True)
    nu = torch.tensor(1.25, dtype=torch.float64, device="cuda", requires_grad=True)
    f, e = at(x, nu)
    assert rel_l2(f.detach().cpu().numpy(), fr.detach().cpu().numpy()) <= tol
    loss = (gf * f).sum() + 0.3 * e
    loss.backward()
    assert rel_l2(x.grad.cpu().numpy(), gx_ref.cpu().numpy()) <= tol
    assert abs(nu.grad.item() - gnu_ref.item()) <= tol * abs(gnu_ref.item())


def test_autograd_force_matching_step():
    """A force-matching fit of nu: loss = |f(nu) - f_FP64(1.1)|^2 over positions; d loss / d nu from
    the harness equals the analytic 2 (nu - 1.1) |f_1|^2 (forces are linear in nu)."""
    torch = pytest.importorskip("torch")
    from threebodymdalgorithms_b200.autograd import AxilrodTeller
    n = 600
    side = generators.box_for_density(n)
    st = generators.uniform(n, (side,) * 3)
    x = torch.tensor(np.stack([st["x"], st["y"], st["z"]], 1), dtype=torch.float64, device="cuda")
    at = AxilrodTeller("p3bca", "mixed", 2.0)
    target, _ = AxilrodTeller("p3bca", "fp64", 2.0)(x, 1.1)
    nu = torch.tensor(0.8, dtype=torch.float64, device="cuda", requires_grad=True)
    f, _ = at(x, nu)
    loss = ((f - target.detach()) ** 2).sum()
    loss.backward()
    f1, _ = at(x, 1.0)
    expect = 2 * (0.8 - 1.1) * (f1.detach() ** 2).sum().item()
    assert abs(nu.grad.item() - expect) <= 1e-4 * abs(expect)


@pytest.mark.parametrize("algo,cutoff", [("auta", 0.0), ("p3bca", 2.0)])
def test_batch_rejects_non_finite_positions(algo, cutoff):
    from threebodymdalgorithms_b200 import TbmdError
    systems = make_systems(3, 50, 120, seed=5)
    offsets, cat = pack(systems)
    cat["y"][offsets[1] + 7] = np.nan
    ctx = Context(algo, "mixed", cutoff)
    with pytest.raises(TbmdError) as e:
        ctx.batch_forces(offsets, cat["x"], cat["y"], cat["z"])
    assert e.value.status == 2
    ctx.close()
