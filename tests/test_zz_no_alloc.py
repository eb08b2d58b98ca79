"""The allocation-free NATA entry point (tbmd_nata_forces_noalloc), called through the C ABI.

It serves callers that cannot allocate device memory when they need forces, so it takes caller
device buffers and uses only the library's fixed static scratch.  Its forces must equal those of
the ordinary NATA entry point (tbmd_forces on a NATA context) within the tolerances the other
parity tests use, on two calls in a row (the second call runs on scratch that still holds the
first call's data).  This file is collected last so that a failure here comes after every other
test; it also passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from threebodymdalgorithms_b200 import Context, _lib, generators

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "mixed": 1e-5}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_nata_on_two_calls(precision):
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    code = _lib.PRECISIONS[precision]
    stream = torch.cuda.current_stream(dev)
    for n, box in ((3000, 13.0), (1500, 9.0)):
        st = generators.uniform(n, (box, box, box))
        ctx = Context("nata", precision, nu=1.2)
        ctx.set_state(st)
        fx, fy, fz, _, _ = ctx.forces()
        ctx.close()
        ref = np.stack([fx, fy, fz], 1)
        pos = [torch.tensor(st[k], dtype=torch.float64, device=dev) for k in ("x", "y", "z")]
        out = [torch.full((n,), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
        for call in range(2):
            for o in out:
                o.fill_(float("nan") if call == 0 else 12345.0)  # every entry must be overwritten
            status = lib.tbmd_nata_forces_noalloc(n, *[C.c_void_p(p.data_ptr()) for p in pos], 1.2, code,
                                                  *[C.c_void_p(o.data_ptr()) for o in out],
                                                  C.c_void_p(stream.cuda_stream))
            assert status == 0, _lib.STATUS.get(status)
            torch.cuda.synchronize(dev)
            got = np.stack([o.cpu().numpy() for o in out], 1)
            assert np.isfinite(got).all()
            assert rel_l2(got, ref) <= TOL[precision], (precision, n, call, rel_l2(got, ref))


def test_noalloc_limits():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    n = _lib.NOALLOC_MAX_N + 1
    buf = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(6)]
    ptrs = [C.c_void_p(b.data_ptr()) for b in buf]
    assert lib.tbmd_nata_forces_noalloc(n, *ptrs[:3], 1.0, 0, *ptrs[3:], None) == 8  # TBMD_TOO_LARGE
    assert lib.tbmd_nata_forces_noalloc(0, *ptrs[:3], 1.0, 0, *ptrs[3:], None) == 1
    buf[3].fill_(7.0)
    assert lib.tbmd_nata_forces_noalloc(2, *ptrs[:3], 1.0, 0, *ptrs[3:], None) == 0  # fewer than 3: zeros
    torch.cuda.synchronize(dev)
    assert float(buf[3][:2].abs().sum()) == 0.0
