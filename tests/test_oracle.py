"""The CPU oracle against the reference's own outputs (golden fixtures) and basic identities.

These pin the oracle: single-threaded it must reproduce the reference built from its sources
bit for bit, so that every later comparison of the CUDA path against the oracle is a comparison
against the reference.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_io as G

STATE = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "fx", "fy", "fz")


def run_oracle(inp, meta, nthreads):
    if meta["mode"] == "forces":
        cut = meta["cutoff"] if meta["algo"] == "p3bca" else -1.0
        fx, fy, fz, c = O.forces(inp["x"], inp["y"], inp["z"], meta["nu"], cut, nthreads=nthreads)
        st = {k: inp[k] for k in inp}
        st.update(fx=fx, fy=fy, fz=fz)
        return st, np.array([c], dtype=np.uint64)
    return O.simulate(meta["algo"], meta["iters"], inp, meta["dt"], meta["g"], meta["cutoff"], meta["nu"],
                      nthreads=nthreads)


@pytest.mark.parametrize("name", G.names())
def test_oracle_matches_reference_bitwise(name):
    inp, out, counts, meta = G.load(name)
    st, c = run_oracle(inp, meta, nthreads=1)
    assert np.array_equal(c, counts), (c, counts)
    for k in STATE:
        assert np.array_equal(st[k], out[k]), (k, np.max(np.abs(st[k] - out[k])))


@pytest.mark.parametrize("name", ["p3bca_n1000_c1.5_2steps", "nata_n256_3steps", "p3bca_clustered_n512_c2"])
def test_oracle_threads_close(name):
    inp, out, counts, meta = G.load(name)
    st, c = run_oracle(inp, meta, nthreads=4)
    assert np.array_equal(c, counts)
    for k in ("fx", "fy", "fz", "vx", "vy", "vz"):
        assert np.linalg.norm(st[k] - out[k]) <= 1e-12 * np.linalg.norm(out[k])


def test_reference_count_pin():
    """src/tests/tests.cpp:530-568 pins the N=1000 triplet count to C(1000,3)."""
    inp, out, counts, meta = G.load("tests_fixture_n1000_auta")
    assert int(counts[0]) == math.comb(1000, 3) == 166167000


def test_cells_equal_bruteforce():
    rng = np.random.default_rng(7)
    n = 400
    x, y, z = (rng.uniform(0, 7, n) for _ in range(3))
    for cut in (1.0, 1.7, 2.5):
        a = O.forces(x, y, z, 1.0, cut, nthreads=1, method="brute")
        b = O.forces(x, y, z, 1.0, cut, nthreads=1, method="cells")
        assert a[3] == b[3]
        for u, v in zip(a[:3], b[:3]):
            assert np.array_equal(u, v)


def test_forces_are_plus_energy_gradient():
    rng = np.random.default_rng(3)
    x, y, z = (rng.uniform(0, 2.5, 7) for _ in range(3))
    f = np.stack(O.forces(x, y, z, 1.3, nthreads=1)[:3], 1)
    h = 1e-6
    g = np.zeros_like(f)
    for i in range(7):
        for d in range(3):
            p = [x.copy(), y.copy(), z.copy()]
            p[d][i] += h
            ep = O.energy(*p, nu=1.3, nthreads=1)
            p[d][i] -= 2 * h
            em = O.energy(*p, nu=1.3, nthreads=1)
            g[i, d] = (ep - em) / (2 * h)
    assert np.linalg.norm(f - g) <= 1e-7 * np.linalg.norm(g)


def test_cell_assignment_wraps_periodically():
    L = np.array([10.0, 10.0, 10.0])
    lo = np.zeros(3)
    x = np.array([0.1, 9.9, -0.3, 10.2, 5.0])
    cell, dims = O.cell_assign(x, np.full(5, 1.0), np.full(5, 1.0), 2.0, L, lo)
    assert dims == (4, 4, 4)
    cx = cell % dims[0]
    assert cx.tolist() == [0, 3, 3, 0, 2]


def test_selected_forces_equal_the_reference_run():
    """forces_selected (one particle's triplets, O(n^2)) against the reference's own forces on the
    N=1000 fixture: the same per-triplet arithmetic, summed in another order."""
    inp, out, _, _ = G.load("tests_fixture_n1000_auta")
    idx = np.array([0, 1, 499, 998, 999, 321])
    got = np.stack(O.forces_selected(inp["x"], inp["y"], inp["z"], idx, 1.0, nthreads=4), 1)
    ref = np.stack([out["fx"][idx], out["fy"][idx], out["fz"][idx]], 1)
    assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref)
