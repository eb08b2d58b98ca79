"""tbmd_step_host against the three calls it combines.

One call that loads host arrays, steps and writes the state back must leave what
tbmd_set_particles + tbmd_step + tbmd_get_particles leave.  IDs, masses, the first step's count
and the positions after one step (the predictor is deterministic) must match exactly.  The rest
matches within what two runs of the same calls give.  The order of particles inside a cell comes
from the cell scatter's atomics, so the summation order of the forces varies between runs: at FP64
rounding in the FP64 form, at FP32 rounding in the mixed form.  After several steps that difference
is amplified by the close pairs' dynamics.  The bars are those of the parity tests."""
import numpy as np
import pytest

from threebodymdalgorithms_b200 import Context, generators

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m", "fx", "fy", "fz")
G = (0.0, -9.81, 0.0)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - b) / (nb if nb > 0 else 1.0)


def separate(algo, prec, cutoff, st, iters):
    ctx = Context(algo, prec, cutoff, 0.001, G)
    ctx.set_state(st)
    counts = ctx.step(iters) if iters else np.zeros(0, dtype=np.uint64)
    out = ctx.get_state()
    ctx.close()
    return out, counts


def tolerance(prec, iters, key):
    if prec == "fp64":
        return 1e-12 if iters <= 1 else 1e-10
    if iters <= 1:
        return 1e-5
    return 1e-4 if key in ("x", "y", "z") else 1e-2


def check_same(a, ca, b, cb, iters, prec):
    assert len(ca) == len(cb) == iters
    if iters:
        assert ca[0] == cb[0]
        assert np.all(np.abs(ca.astype(np.int64) - cb.astype(np.int64)) <= 1e-3 * ca.astype(np.int64) + 2)
    assert np.array_equal(a["id"], b["id"])
    assert np.array_equal(a["m"], b["m"])
    for k in KEYS:
        if iters <= 1 and k in ("x", "y", "z"):
            assert np.array_equal(a[k], b[k]), k
        else:
            assert rel(b[k], a[k]) <= tolerance(prec, iters, k), (k, rel(b[k], a[k]))


def uniform_input(algo):
    n = 4096 if algo == "p3bca" else 512
    side = generators.box_for_density(n) if algo == "p3bca" else 10.0
    st = generators.as_csv_values(generators.uniform(n, (side, side, side)))
    st["id"] = np.arange(n, dtype=np.int32)[::-1].copy()  # non-trivial IDs travel through unchanged
    return st


@pytest.mark.parametrize("algo,prec,cutoff", [("p3bca", "mixed", 2.0), ("p3bca", "fp64", 2.0),
                                              ("auta", "fp64", 0.0), ("nata", "mixed", 0.0)])
def test_step_host_matches_the_separate_calls(algo, prec, cutoff):
    st = uniform_input(algo)
    ctx = Context(algo, prec, cutoff, 0.001, G)
    for iters in (1, 3, 0, 1):  # the context is reused: two calls in a row, and a call without steps
        ref, cref = separate(algo, prec, cutoff, st, iters)
        got, cgot = ctx.step_host(st, iters)
        check_same(ref, cref, got, cgot, iters, prec)
    ctx.close()


def test_step_host_in_place_and_partial_outputs():
    """Outputs may be the input arrays themselves, and any output may be left out."""
    st = uniform_input("p3bca")
    ref, cref = separate("p3bca", "mixed", 2.0, st, 2)
    work = {k: np.array(v, copy=True) for k, v in st.items()}
    ctx = Context("p3bca", "mixed", 2.0, 0.001, G)
    out = {k: work[k] for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")}
    out["fx"] = np.zeros(len(st["x"]))
    got, c = ctx.step_host(work, 2, out=out)
    assert c[0] == cref[0]
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m", "fx"):
        assert got[k] is out[k]
        assert rel(out[k], ref[k]) <= tolerance("mixed", 2, k), k
    assert "fy" not in got and "fz" not in got
    ctx.close()


def test_step_host_after_a_capacity_retry():
    """Clustered particles overflow the first neighbour-list capacity; the step is redone, and the
    copies of the redone attempt are the ones that reach the host."""
    st = generators.clustered_gauss(8192, 16, (32, 32, 32))
    ref, cref = separate("p3bca", "fp64", 2.0, st, 2)
    ctx = Context("p3bca", "fp64", 2.0, 0.001, G)
    got, c = ctx.step_host(st, 2)
    check_same(ref, cref, got, c, 2, "fp64")
    ctx.close()


def test_contiguous_field_blocks():
    """Fields given as the rows of one block (x, y, z, vx, ... back to back in memory) move in one
    transfer per contiguous run; the results are those of separate arrays, through tbmd_step_host
    and through tbmd_set_particles / tbmd_get_particles alike."""
    st = uniform_input("p3bca")
    n = len(st["x"])
    ins = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")
    block_in = np.empty((len(ins), n))
    for r, k in enumerate(ins):
        block_in[r] = st[k] if k in st else (np.ones(n) if k == "m" else np.zeros(n))
    rows_in = {k: block_in[r] for r, k in enumerate(ins)}
    rows_in["id"] = st["id"]
    ref, cref = separate("p3bca", "fp64", 2.0, st, 1)
    block_out = np.zeros((len(KEYS), n))
    out = {k: block_out[r] for r, k in enumerate(KEYS)}
    ctx = Context("p3bca", "fp64", 2.0, 0.001, G)
    got, c = ctx.step_host(rows_in, 1, out=out)
    check_same(ref, cref, got, c, 1, "fp64")
    # the same block through the separate calls
    ctx.set_state(rows_in)
    assert ctx.step(1)[0] == cref[0]
    back = ctx.get_state()
    for k in KEYS:
        assert rel(back[k], ref[k]) <= 1e-12, k
    ctx.close()


def test_step_host_leaves_the_unused_accelerations_out():
    """A step reads ax alone (the predictor applies it on all three axes) and the update overwrites
    ay and az, so tbmd_step_host does not copy them to the device.  The results are still those of
    the three calls, and non-finite values there are still rejected, as tbmd_set_particles rejects
    them."""
    from threebodymdalgorithms_b200 import TbmdError
    st = uniform_input("p3bca")
    rng = np.random.default_rng(5)
    st["ay"] = rng.normal(size=len(st["x"]))
    st["az"] = rng.normal(size=len(st["x"]))
    ref, cref = separate("p3bca", "fp64", 2.0, st, 1)
    ctx = Context("p3bca", "fp64", 2.0, 0.001, G)
    got, c = ctx.step_host(st, 1)
    check_same(ref, cref, got, c, 1, "fp64")
    for k, arr, bad in (("ay", 7, np.nan), ("az", 8, np.inf)):
        b = {kk: np.array(v, copy=True) for kk, v in st.items()}
        b[k][17] = bad
        for call in (lambda: ctx.step_host(b, 1), lambda: ctx.set_state(b)):
            with pytest.raises(TbmdError) as e:
                call()
            assert e.value.status == 2 and f"array {arr}" in str(e.value), str(e.value)
    # the failed calls left the state of the good one
    after = ctx.get_state()
    for key in ("x", "vx", "ay", "fx"):
        assert np.array_equal(after[key], got[key]), key
    ctx.close()
