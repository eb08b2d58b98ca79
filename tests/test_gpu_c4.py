"""The clustered P3BCA workload at full size: N = 262144 particles in 256 isotropic Gaussian clusters
(sigma 1, 1024 particles each) with centres uniform in a 64^3 box, cutoff 2, drawn like the
reference's ClusteredGaussGenerator (src/tools/ClusteredGaussGenerator.cpp:15-47) and rounded to
its 6-digit CSV values.  Step 0 holds 7,282,646,752 triplets inside the cutoff (the oracle's count);
dense cluster cores give half lists of up to about 1200 entries.

- Forces at the initial positions in both precisions against the oracle's cell list: counts bit
  exact (the cutoff test of Algorithm.cpp:94-100), FP64 within 1e-12 relative L2, mixed within 1e-5.
- Ten FP64 Simulation steps through tbmd_step (one call, the captured step graph replayed) against
  the oracle's step loop (Simulation.cpp:28-49): the count of every step, and positions and
  velocities within the multi-step FP64 tolerance.  The clusters fly apart at once (the count
  falls to about 4.9e6 by step 9), so the later steps are far cheaper than the first.
"""
import numpy as np
import pytest

from oracle import oracle as O
from threebodymdalgorithms_b200 import Context, generators

pytestmark = pytest.mark.gpu

CUTOFF = 2.0
DT = 0.001
G = (0.0, -9.81, 0.0)


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.fixture(scope="module")
def c4():
    st = generators.as_csv_values(generators.clustered_gauss(262144, 256, (64.0, 64.0, 64.0)))
    assert len(st["x"]) == 262144
    return st


def test_c4_forces_vs_oracle(c4):
    st = c4
    L, lo = O.domain(st["x"], st["y"], st["z"])
    fx, fy, fz, c_ref = O.forces(st["x"], st["y"], st["z"], 1.0, CUTOFF, L, lo, nthreads=0)
    assert c_ref == 7282646752
    ref = np.stack([fx, fy, fz], 1)
    for prec, tol in (("fp64", 1e-12), ("mixed", 1e-5)):
        ctx = Context("p3bca", prec, CUTOFF, DT, G)
        ctx.set_state(st)
        gfx, gfy, gfz, e, c = ctx.forces()
        ctx.close()
        assert c == c_ref, (prec, c, c_ref)
        assert rel_l2(np.stack([gfx, gfy, gfz], 1), ref) <= tol, (prec, rel_l2(np.stack([gfx, gfy, gfz], 1), ref))


def test_c4_ten_steps_vs_oracle(c4):
    st = c4
    ref, counts = O.simulate("p3bca", 10, st, DT, G, cutoff=CUTOFF, nthreads=0)
    ctx = Context("p3bca", "fp64", CUTOFF, DT, G, use_graph=True)
    ctx.set_state(st)
    got_counts = ctx.step(10)
    got = ctx.get_state()
    ctx.close()
    assert [int(c) for c in got_counts] == [int(c) for c in counts], (got_counts, counts)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert rel_l2(got[k], ref[k]) <= 1e-10, (k, rel_l2(got[k], ref[k]))
