"""torch.autograd harness over the CUDA forces and their adjoint (no reference counterpart).

AxilrodTeller(algorithm, precision, cutoff).forward(x, nu) returns (f, E): the stored forces
f = +grad E of the Axilrod-Teller energy (the reference's sign, AxilrodTeller.cpp:119-129) as an
(n, 3) float64 CUDA tensor and the energy as a 0-d tensor.  Both are differentiable with respect
to the positions x and the strength nu: the backward pass calls the adjoint kernel, which
recomputes the triplet geometry and returns the Hessian-vector product H g_f (plus g_E f) and the
nu gradient; nothing per triplet is stored.  f and E are linear in nu, so the library runs at
nu = 1 and the harness scales by nu.  All kernels run on torch's current stream.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import Context


def _soa(t: torch.Tensor) -> torch.Tensor:
    """(n, 3) -> contiguous (3, n) float64 on the same device."""
    return t.detach().to(torch.float64).t().contiguous()


def _ptrs(t3: torch.Tensor):
    return [C.c_void_p(t3[k].data_ptr()) for k in range(3)]


def _stream(device) -> C.c_void_p:
    """torch's current stream as a cudaStream_t.  torch reports the legacy default stream as 0,
    which the C ABI reads as "the context's own stream"; pass cudaStreamLegacy (1) instead so the
    kernels are ordered with torch's work."""
    h = torch.cuda.current_stream(device).cuda_stream
    return C.c_void_p(h if h else 1)


class _ATFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, nu, engine):
        xs = _soa(x)
        n = xs.shape[1]
        stream = _stream(x.device)
        f1 = torch.empty_like(xs)
        e1 = torch.zeros(1, dtype=torch.float64, device=x.device)
        engine.forces_device(n, *_ptrs(xs), *_ptrs(f1), C.c_void_p(e1.data_ptr()), None, stream=stream)
        ctx.save_for_backward(x, nu)
        ctx.engine = engine
        return (nu * f1).t().contiguous(), nu * e1[0]

    @staticmethod
    def backward(ctx, g_f, g_e):
        x, nu = ctx.saved_tensors
        engine = ctx.engine
        xs = _soa(x)
        n = xs.shape[1]
        stream = _stream(x.device)
        gfs = _soa(g_f) if g_f is not None else torch.zeros_like(xs)
        ge = g_e.to(torch.float64) if g_e is not None else torch.zeros((), dtype=torch.float64, device=x.device)
        f1 = torch.empty_like(xs)
        h1 = torch.empty_like(xs)
        e1 = torch.zeros(1, dtype=torch.float64, device=x.device)
        engine.adjoint_device(n, [*_ptrs(xs), *_ptrs(gfs), C.c_void_p(0), *_ptrs(f1), C.c_void_p(e1.data_ptr()),
                                  *_ptrs(h1)], stream=stream)
        grad_x = (nu * (h1 + ge * f1)).t().contiguous() if ctx.needs_input_grad[0] else None
        grad_nu = ((gfs * f1).sum() + ge * e1[0]) if ctx.needs_input_grad[1] else None
        return grad_x, grad_nu, None


class AxilrodTeller:
    """Differentiable AT forces and energy on one GPU (see module docstring).

    For P3BCA (cutoff > 0) the periodic domain is fixed by `box`/`lo`, or on the first call from
    the positions with the reference's rule (bounding box widened by 1e-4 per side)."""

    def __init__(self, algorithm: str = "auta", precision: str = "fp64", cutoff: float = 0.0, device: int = 0,
                 box=None, lo=None):
        self.engine = Context(algorithm, precision, cutoff, nu=1.0, device=device)
        self.cutoff = float(cutoff)
        self.algorithm = algorithm
        self._domain = None
        if box is not None:
            self.set_domain(box, lo if lo is not None else (0.0, 0.0, 0.0))

    def set_domain(self, box, lo):
        import numpy as np
        self.engine.set_domain(np.asarray(box, dtype=np.float64), np.asarray(lo, dtype=np.float64))
        self._domain = (tuple(box), tuple(lo))

    def __call__(self, x: torch.Tensor, nu) -> tuple[torch.Tensor, torch.Tensor]:
        if not x.is_cuda or x.dim() != 2 or x.shape[1] != 3:
            raise ValueError("x must be an (n, 3) CUDA tensor")
        if not torch.is_tensor(nu):
            nu = torch.tensor(float(nu), dtype=torch.float64, device=x.device)
        if self.algorithm.lower() == "p3bca" and self.cutoff > 0 and self._domain is None:
            xd = x.detach().double()
            mn = xd.min(0).values - 1e-4
            mx = xd.max(0).values + 1e-4
            self.set_domain((mx - mn).abs().tolist(), mn.tolist())
        return _ATFunction.apply(x, nu.to(torch.float64), self.engine)
