"""The allocation-free NATA entry point (tbmd_nata_forces_noalloc), called through the C ABI.

It serves callers that cannot allocate device memory when they need forces, so it takes caller
device buffers and uses only the library's fixed static scratch.  Its forces must equal those of
the ordinary NATA entry point (tbmd_forces on a NATA context) within the tolerances the other
parity tests use, on two calls in a row (the second call runs on scratch that still holds the
first call's data).  This file is collected last so that a failure here comes after every other
test; it also passes when run alone in a fresh process.
"""
import ctypes as C
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from threebodymdalgorithms_b200 import Context, _lib, generators

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
TOL = {"fp64": 1e-12, "mixed": 1e-5}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _noalloc(lib, torch, n, pos, out, nu, code, stream):
    return lib.tbmd_nata_forces_noalloc(n, *[C.c_void_p(p.data_ptr()) for p in pos], nu, code,
                                        *[C.c_void_p(o.data_ptr()) for o in out], C.c_void_p(stream.cuda_stream))


# n = 4096 fills the whole static array (32 j-blocks of partial sums, then the counter); n = 3 and 4
# are the smallest sizes that launch the kernels.
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_nata_on_two_calls(precision):
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    code = _lib.PRECISIONS[precision]
    stream = torch.cuda.current_stream(dev)
    for n, box in ((3000, 13.0), (1500, 9.0), (_lib.NOALLOC_MAX_N, 14.0), (3, 2.0), (4, 2.0)):
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
            status = _noalloc(lib, torch, n, pos, out, 1.2, code, stream)
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
    for bad_nu in (float("nan"), float("inf"), float("-inf")):
        assert lib.tbmd_nata_forces_noalloc(8, *ptrs[:3], bad_nu, 0, *ptrs[3:], None) == 1  # TBMD_INVALID_ARG
    buf[3].fill_(7.0)
    assert lib.tbmd_nata_forces_noalloc(2, *ptrs[:3], 1.0, 0, *ptrs[3:], None) == 0  # fewer than 3: zeros
    torch.cuda.synchronize(dev)
    assert float(buf[3][:2].abs().sum()) == 0.0


# Runs in a child process with the driver API only: the call in the device's primary context, then
# the same call with a second context current (its own buffers).  The scratch address looked up in
# the first context is not valid in the second; the entry point must look it up again there.
_TWO_CONTEXTS = r"""
import ctypes as C, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from threebodymdalgorithms_b200 import _lib, generators
lib = _lib.load()
cu = C.CDLL("libcuda.so.1")
def ok(r):
    assert r == 0, r
ok(cu.cuInit(0))
dev = C.c_int()
ok(cu.cuDeviceGet(C.byref(dev), 0))
n = 700
st = generators.uniform(n, (8.0, 8.0, 8.0))
def run_in_current_context():
    ptrs = []
    for _ in range(6):
        p = C.c_uint64()
        ok(cu.cuMemAlloc_v2(C.byref(p), C.c_size_t(8 * n)))
        ptrs.append(p)
    for k, p in zip(("x", "y", "z"), ptrs[:3]):
        a = np.ascontiguousarray(st[k])
        ok(cu.cuMemcpyHtoD_v2(p, a.ctypes.data_as(C.c_void_p), C.c_size_t(8 * n)))
    status = lib.tbmd_nata_forces_noalloc(n, *[C.c_void_p(p.value) for p in ptrs[:3]], 1.0, 0,
                                          *[C.c_void_p(p.value) for p in ptrs[3:]], None)
    assert status == 0, status
    ok(cu.cuCtxSynchronize())
    out = []
    for p in ptrs[3:]:
        a = np.zeros(n)
        ok(cu.cuMemcpyDtoH_v2(a.ctypes.data_as(C.c_void_p), p, C.c_size_t(8 * n)))
        out.append(a)
    for p in ptrs:
        ok(cu.cuMemFree_v2(p))
    return np.stack(out, 1)
primary = C.c_void_p()
ok(cu.cuDevicePrimaryCtxRetain(C.byref(primary), dev))
ok(cu.cuCtxSetCurrent(primary))
a = run_in_current_context()
other = C.c_void_p()
ok(cu.cuCtxCreate_v2(C.byref(other), 0, dev))  # current from here on
b = run_in_current_context()
ok(cu.cuCtxDestroy_v2(other))
ok(cu.cuCtxSetCurrent(primary))
c = run_in_current_context()
print(json.dumps({"finite": bool(np.isfinite(a).all() and np.isfinite(b).all()),
                  "norm": float(np.linalg.norm(a)), "same_b": bool(np.array_equal(a, b)),
                  "same_c": bool(np.array_equal(a, c))}))
"""


def test_noalloc_after_the_context_changes():
    r = subprocess.run([sys.executable, "-c", _TWO_CONTEXTS, str(ROOT)], capture_output=True, text=True,
                       timeout=300, env=dict(os.environ))
    assert r.returncode == 0, r.stdout + r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["finite"] and d["norm"] > 0 and d["same_b"] and d["same_c"], d
