"""Adjoint (HVP + d/dnu) against FP64 central finite differences (h = 1e-6) of the GPU forward
and against autograd of a small FP64 PyTorch AT reference."""
import numpy as np
import pytest

from threebodymdalgorithms_b200 import Context, generators

pytestmark = pytest.mark.gpu
H = 1e-6


def loss_and_parts(ctx, st, gf, ge):
    ctx.set_state(st)
    fx, fy, fz, e, c = ctx.forces()
    f = np.stack([fx, fy, fz], 1)
    return float((gf * f).sum() + ge * e)


@pytest.mark.parametrize("algo,cutoff", [("auta", 0.0), ("p3bca", 1.6)])
def test_adjoint_vs_finite_differences(algo, cutoff):
    rng = np.random.default_rng(11)
    n = 24
    st = generators.uniform(n, (2.6, 2.6, 2.6))
    gf = rng.normal(size=(n, 3))
    ge = 0.7
    nu = 1.3
    ctx = Context(algo, "fp64", cutoff, nu=nu)
    ctx.set_state(st)
    if algo == "p3bca":  # fix the domain so perturbations do not move it
        L, lo = ctx.cells(False)[2:]
        ctx.set_domain(L, lo)
    gx, gy, gz, gnu = ctx.adjoint(gf[:, 0], gf[:, 1], gf[:, 2], ge)
    g = np.stack([gx, gy, gz], 1)
    fd = np.zeros_like(g)
    for i in range(n):
        for d, k in enumerate("xyz"):
            p = {kk: v.copy() for kk, v in st.items()}
            p[k][i] += H
            lp = loss_and_parts(ctx, p, gf, ge)
            p[k][i] -= 2 * H
            lm = loss_and_parts(ctx, p, gf, ge)
            fd[i, d] = (lp - lm) / (2 * H)
    assert np.linalg.norm(g - fd) <= 1e-6 * np.linalg.norm(fd)
    ctx.close()
    # d/dnu
    lp = loss_and_parts(Context(algo, "fp64", cutoff, nu=nu + H), st, gf, ge)
    lm = loss_and_parts(Context(algo, "fp64", cutoff, nu=nu - H), st, gf, ge)
    assert abs(gnu - (lp - lm) / (2 * H)) <= 1e-6 * abs(gnu)


def torch_at_energy(x, nu):
    import torch
    n = x.shape[0]
    i, j, k = torch.combinations(torch.arange(n), 3).T
    u = x[j] - x[i]
    v = x[k] - x[i]
    w = x[k] - x[j]
    uu, vv, ww = (u * u).sum(1), (v * v).sum(1), (w * w).sum(1)
    cosprod = -((u * v).sum(1) * (u * w).sum(1) * (v * w).sum(1)) / (uu * vv * ww)
    return (nu * (1 + 3 * cosprod) / (uu * vv * ww) ** 1.5).sum()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_adjoint_vs_torch_autograd(precision, tol):
    torch = pytest.importorskip("torch")
    n = 14
    st = generators.uniform(n, (2.4, 2.4, 2.4))
    rng = np.random.default_rng(5)
    gf = rng.normal(size=(n, 3))
    ge = -0.4
    nu = 0.9
    x = torch.tensor(np.stack([st["x"], st["y"], st["z"]], 1), dtype=torch.float64, requires_grad=True)
    nu_t = torch.tensor(nu, dtype=torch.float64, requires_grad=True)
    E = torch_at_energy(x, nu_t)
    (f,) = torch.autograd.grad(E, x, create_graph=True)  # stored forces = +grad E
    L = (torch.tensor(gf) * f).sum() + ge * E
    gx_ref, gnu_ref = torch.autograd.grad(L, (x, nu_t))
    ctx = Context("auta", precision, nu=nu)
    ctx.set_state(st)
    gx, gy, gz, gnu = ctx.adjoint(gf[:, 0], gf[:, 1], gf[:, 2], ge)
    g = np.stack([gx, gy, gz], 1)
    ref = gx_ref.numpy()
    assert np.linalg.norm(g - ref) <= tol * np.linalg.norm(ref)
    assert abs(gnu - gnu_ref.item()) <= tol * abs(gnu_ref.item())
    ctx.close()
