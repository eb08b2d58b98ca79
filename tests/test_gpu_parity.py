"""Parity of the CUDA path (through the C ABI) with the reference and its oracle.

Bars: triplet counts and cell assignments bit-exact at the same positions; FP64 forces within
rel-L2 1e-12 of the reference for one evaluation (a different but, in exact arithmetic, equal
formulation and summation order); mixed precision within rel-L2 1e-5 on forces (the target
tolerance).  After a multi-step run the dynamics amplify any difference (forces scale like r^-10,
and the close pairs of these random configurations reach accelerations of 1e4-1e6, moving by a
good fraction of their distance within a few steps), so FP64 runs are held to 1e-10 on positions
and velocities and 1e-6 on forces, and mixed runs, whose trajectories diverge from FP64 ones in
the same way, to 1e-4 on positions and 1e-2 on velocities and forces, with per-step counts after
the first step within 0.1% (triplets that sit within the trajectory difference of the cutoff).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_io as GIO
from threebodymdalgorithms_b200 import Context, generators

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP64_MULTISTEP_TOL = 1e-10
FP64_MULTISTEP_FORCE_TOL = 1e-6
MIXED_FORCE_TOL = 1e-5
MIXED_STATE_TOL = 1e-6
MIXED_MULTISTEP_POS_TOL = 1e-4
MIXED_MULTISTEP_TOL = 1e-2
# Mixed energies: |E - E_ref| <= MIXED_ENERGY_TOL * S with S = sum over triplets of
# |nu| (1 + 3 |cos cos cos|) / (r1 r2 r3)^3 (oracle energy_abs).  The triplet terms have both signs
# and a term can cancel inside (1 + 3 cos cos cos), so |E| can be far smaller than S (by 37x in the
# batched test systems); FP32 geometry rounds each part of a term to about 1e-6 of its size.
MIXED_ENERGY_TOL = 2e-6
STATE = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "fx", "fy", "fz")


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def gpu_run(inp, meta, precision, use_graph=True):
    ctx = Context(meta["algo"], precision, meta["cutoff"], meta["dt"], meta["g"], meta["nu"], use_graph=use_graph)
    ctx.set_state(inp)
    if meta["mode"] == "forces":
        fx, fy, fz, e, c = ctx.forces()
        st = ctx.get_state()
        counts = np.array([c], dtype=np.uint64)
    else:
        counts = ctx.step(meta["iters"])
        st = ctx.get_state()
    ctx.close()
    return st, counts


def check_state(st, out, force_tol, state_tol, pos_tol=None):
    for k in STATE:
        tol = force_tol if k.startswith("f") or k.startswith("a") else state_tol
        if pos_tol is not None and k in ("x", "y", "z"):
            tol = pos_tol
        err = rel_l2(st[k], out[k])
        assert err <= tol, (k, err)


def counts_close(c, ref, rel):
    """First step exact; later steps within `rel` (mixed-precision trajectories diverge)."""
    c, ref = c.astype(np.int64), ref.astype(np.int64)
    return c[0] == ref[0] and np.all(np.abs(c - ref) <= rel * ref + 2)


@pytest.mark.parametrize("name", GIO.names())
def test_golden_fp64(name):
    inp, out, counts, meta = GIO.load(name)
    st, c = gpu_run(inp, meta, "fp64")
    assert np.array_equal(c, counts), (c, counts)
    if meta["mode"] == "forces" or meta["iters"] == 1:
        check_state(st, out, FP64_TOL, FP64_TOL)
    else:
        check_state(st, out, FP64_MULTISTEP_FORCE_TOL, FP64_MULTISTEP_TOL)


@pytest.mark.parametrize("name", GIO.names())
def test_golden_mixed(name):
    inp, out, counts, meta = GIO.load(name)
    st, c = gpu_run(inp, meta, "mixed")
    assert counts_close(c, counts, 1e-3), (c, counts)
    if meta["mode"] == "forces" or meta["iters"] == 1:
        check_state(st, out, MIXED_FORCE_TOL, MIXED_STATE_TOL)
    else:
        check_state(st, out, MIXED_MULTISTEP_TOL, MIXED_MULTISTEP_TOL, MIXED_MULTISTEP_POS_TOL)


@pytest.mark.parametrize("name", ["p3bca_n512_c2_3steps", "nata_n256_3steps", "auta_n300_light_3steps"])
def test_graph_and_eager_agree(name):
    inp, out, counts, meta = GIO.load(name)
    a, ca = gpu_run(inp, meta, "fp64", use_graph=True)
    b, cb = gpu_run(inp, meta, "fp64", use_graph=False)
    assert np.array_equal(ca, cb)
    for k in STATE:
        assert rel_l2(a[k], b[k]) <= 1e-13, k


def test_nata_is_deterministic():
    inp, out, counts, meta = GIO.load("nata_n256_3steps")
    a, _ = gpu_run(inp, meta, "fp64")
    b, _ = gpu_run(inp, meta, "fp64")
    for k in STATE:
        assert np.array_equal(a[k], b[k]), k


def forces_of(algo, precision, st, cutoff=0.0):
    ctx = Context(algo, precision, cutoff)
    ctx.set_state(st)
    fx, fy, fz, e, c = ctx.forces()
    ctx.close()
    return np.stack([fx, fy, fz], 1), e, c


def test_auta_vs_oracle_n1024():
    st = generators.as_csv_values(generators.uniform(1024, (12, 12, 12)))
    fx, fy, fz, c = O.forces(st["x"], st["y"], st["z"], 1.0, -1.0, nthreads=0)
    ref = np.stack([fx, fy, fz], 1)
    e_ref = O.energy(st["x"], st["y"], st["z"], 1.0, -1.0)
    e_abs = O.energy_abs(st["x"], st["y"], st["z"], 1.0, -1.0)
    for algo in ("auta", "nata"):
        f64, e64, c64 = forces_of(algo, "fp64", st)
        fmx, emx, cmx = forces_of(algo, "mixed", st)
        assert c64 == cmx == c == math.comb(1024, 3)
        assert rel_l2(f64, ref) <= FP64_TOL
        assert rel_l2(fmx, ref) <= MIXED_FORCE_TOL
        assert abs(e64 - e_ref) <= 1e-12 * abs(e_ref)
        assert abs(emx - e_ref) <= MIXED_ENERGY_TOL * e_abs


def test_c2_n8192_nata_auta_fp64_mixed():
    """C2 (N=8192 uniform in 20^3): the two GPU algorithms and both precisions agree; momentum
    is conserved (sum of forces ~ 0) and the count is C(N,3)."""
    st = generators.as_csv_values(generators.uniform(8192, (20, 20, 20)))
    fa, ea, ca = forces_of("auta", "fp64", st)
    fn, en, cn = forces_of("nata", "fp64", st)
    fm, em, cm = forces_of("auta", "mixed", st)
    fnm, enm, cnm = forces_of("nata", "mixed", st)
    assert ca == cn == cm == cnm == math.comb(8192, 3) == 91592417280
    assert rel_l2(fn, fa) <= FP64_TOL
    assert rel_l2(fm, fa) <= MIXED_FORCE_TOL
    assert rel_l2(fnm, fa) <= MIXED_FORCE_TOL
    assert np.abs(fa.sum(0)).max() <= 1e-9 * np.abs(fa).max() * 8192
    # sum |E_t| over 9.2e10 triplets is too costly for the oracle here; for a uniform system it is
    # within a few percent of |E|, so the bound is taken against |E| with a 5x margin
    assert abs(ea - en) <= 1e-12 * abs(ea) and abs(em - ea) <= 5 * MIXED_ENERGY_TOL * abs(ea)
    # against the oracle: 64 seeded random particles, each with the force of all C(8191, 2) triplets
    # it belongs to, in the reference's per-triplet arithmetic (NATA's view of one particle)
    idx = np.sort(np.random.default_rng(8192).choice(8192, 64, replace=False))
    ref = np.stack(O.forces_selected(st["x"], st["y"], st["z"], idx, 1.0, nthreads=0), 1)
    for f, tol, what in ((fa, FP64_TOL, "auta fp64"), (fn, FP64_TOL, "nata fp64"), (fm, MIXED_FORCE_TOL, "auta mixed"),
                         (fnm, MIXED_FORCE_TOL, "nata mixed")):
        assert rel_l2(f[idx], ref) <= tol, (what, rel_l2(f[idx], ref))
        # and particle by particle, against the largest force of the sample
        assert np.abs(f[idx] - ref).max() <= 10 * tol * np.abs(ref).max(), what


@pytest.mark.parametrize("cutoff", [2.0, 1.5])
def test_c3_p3bca_full_size_vs_oracle(cutoff):
    """C3: N=131072 uniform at density 2.048 (box 40^3), counts bit-exact against the oracle's
    cell list, forces within tolerance, cell assignment bit-exact."""
    n = 131072
    side = generators.box_for_density(n)
    st = generators.as_csv_values(generators.uniform(n, (side, side, side)))
    L, lo = O.domain(st["x"], st["y"], st["z"])
    fx, fy, fz, c_ref = O.forces(st["x"], st["y"], st["z"], 1.0, cutoff, L, lo, nthreads=0)
    ref = np.stack([fx, fy, fz], 1)
    for prec, tol in (("fp64", FP64_TOL), ("mixed", MIXED_FORCE_TOL)):
        ctx = Context("p3bca", prec, cutoff)
        ctx.set_state(st)
        gfx, gfy, gfz, e, c = ctx.forces()
        assert c == c_ref, (prec, c, c_ref)
        assert rel_l2(np.stack([gfx, gfy, gfz], 1), ref) <= tol, prec
        cell, dims, gL, glo = ctx.cells()
        ocell, odims = O.cell_assign(st["x"], st["y"], st["z"], cutoff, L, lo)
        assert dims == odims and np.array_equal(gL, L) and np.array_equal(glo, lo)
        assert np.array_equal(cell, ocell)
        ctx.close()


def test_p3bca_one_million_particles_vs_oracle():
    """N = 1,048,576 uniform at density 2.048 (box 80^3, 8x the C3 volume), cutoff 2: triplet
    counts bit-exact against the oracle's cell list and forces within tolerance, in both
    precisions; a step from zero velocity keeps the positions, so its count is the same."""
    n = 1 << 20
    side = generators.box_for_density(n)
    gen = Context("auta")
    gen.generate(kind="uniform", n=n, box=(side, side, side))
    st = gen.get_state()
    gen.close()
    L, lo = O.domain(st["x"], st["y"], st["z"])
    fx, fy, fz, c_ref = O.forces(st["x"], st["y"], st["z"], 1.0, 2.0, L, lo, nthreads=0)
    ref = np.stack([fx, fy, fz], 1)
    for prec, tol in (("fp64", FP64_TOL), ("mixed", MIXED_FORCE_TOL)):
        ctx = Context("p3bca", prec, 2.0, 0.001, (0.0, -9.81, 0.0))
        ctx.set_state(st)
        gfx, gfy, gfz, e, c = ctx.forces()
        assert c == c_ref, (prec, c, c_ref)
        assert rel_l2(np.stack([gfx, gfy, gfz], 1), ref) <= tol, prec
        assert int(ctx.step(1)[0]) == c_ref
        ctx.close()


def test_p3bca_particles_outside_the_domain():
    """Positions are not wrapped into the box: particles moved one or more box lengths outside an
    explicit domain are binned by wrapping, some into interior cells, and the cutoff test must
    stay the reference's periodic formula on the raw coordinates."""
    rng = np.random.default_rng(3)
    n = 20000
    side = generators.box_for_density(n)
    st = generators.as_csv_values(generators.uniform(n, (side, side, side)))
    L, lo = np.array([side] * 3), np.zeros(3)
    moved = rng.choice(n, 300, replace=False)
    shift = rng.integers(-3, 4, size=(300, 3)) * side + rng.uniform(-0.3, 0.3, size=(300, 3))
    for d, k in enumerate("xyz"):
        st[k][moved] += shift[:, d]
    fx, fy, fz, c_ref = O.forces(st["x"], st["y"], st["z"], 1.0, 2.0, L, lo, nthreads=0)
    ref = np.stack([fx, fy, fz], 1)
    for prec, tol in (("fp64", FP64_TOL), ("mixed", MIXED_FORCE_TOL)):
        ctx = Context("p3bca", prec, 2.0)
        ctx.set_state(st)
        ctx.set_domain(L, lo)
        gfx, gfy, gfz, e, c = ctx.forces()
        assert c == c_ref, (prec, c, c_ref)
        assert rel_l2(np.stack([gfx, gfy, gfz], 1), ref) <= tol, prec
        ctx.close()


def cutoff_triangles(c, L, seed):
    """Isolated triangles: apex s, base j-k of length c (1 + r)^(1/2) in a random direction of the
    x-y plane, so that the base's squared length sits r (relatively) inside or outside cutoff^2,
    with r cycling through 1e-12 .. 1e-4 and a random sign.  The random direction makes the FP32
    rounding of the edges generic (an axis-aligned base of a short binary length would round to
    exactly cutoff^2).  The apex lies one cell layer below its base, so it comes first in the cell
    order and the triplet kernel's third-edge test decides the base; the list test sees only the
    two sides of 0.9.  In every other row the last triangle straddles the periodic boundary in x,
    and the first row's bases cross it in y (the wrapped form of the test).  Triangles are at
    least 2.25 apart (> c) from one another, also across the periodic boundaries of the L^3 box
    with cells of c = L / 20."""
    rng = np.random.default_rng(seed)
    rel = np.array([1e-12, 1e-9, 1e-7, 1e-6, 3e-6, 1e-5, 3e-5, 1e-4])
    nx, ny, nz = 7, 8, 10
    pts, r_of = [], []
    for iz in range(nz):
        for iy in range(ny):
            straddle = iy % 2 == 0
            for ix in range(nx):
                if straddle and ix == 0:
                    continue
                r = rel[len(r_of) % len(rel)] * rng.choice([-1.0, 1.0])
                half = c * math.sqrt(1.0 + r) / 2
                last = straddle and ix == nx - 1
                th = rng.uniform(-1.0, 1.0) if last else rng.uniform(0.0, 2 * math.pi)  # cos >= 0.54
                hx, hy = half * math.cos(th), half * math.sin(th)
                px = L - 0.3 if last else ix * L / nx + 1.0
                py, pz = iy * L / ny + 0.5, iz * 3.0 + 1.4
                pts += [(px, py, pz), ((px - hx) % L, (py - hy) % L, pz + 0.5),
                        ((px + hx) % L, (py + hy) % L, pz + 0.5)]
                r_of.append(r)
    return np.array(pts), np.array(r_of)


def cutoff_sides(c, L, seed):
    """Isolated triangles whose side s-j from the apex is c (1 + r)^(1/2) long (r as in
    cutoff_triangles), in a random direction rising 0.2 c to 0.93 c in z, with k 0.9 from both:
    the apex is alone in the first cell layer of its triangle, so the list kernel's pair test
    decides s-j and the triplet is counted exactly when s-j is inside.  A lattice of 8^3 triangles
    4.5 apart in the L = 36 box (cells of c = 1.5); its first column's sides cross the periodic
    boundary in x when they point to -x."""
    rng = np.random.default_rng(seed)
    rel = np.array([1e-12, 1e-9, 1e-7, 1e-6, 3e-6, 1e-5, 3e-5, 1e-4])
    pts, r_of = [], []
    for iz in range(8):
        for iy in range(8):
            for ix in range(8):
                r = rel[len(r_of) % len(rel)] * rng.choice([-1.0, 1.0])
                cp = c * math.sqrt(1.0 + r)
                th, cz = rng.uniform(0.0, 2 * math.pi), rng.uniform(0.2, 0.93)
                sz = math.sqrt(1.0 - cz * cz)
                d = np.array([sz * math.cos(th), sz * math.sin(th), cz])
                nrm = np.array([-math.sin(th), math.cos(th), 0.0])
                s0 = np.array([ix * 4.5 + 1.0, iy * 4.5 + 1.0, iz * 4.5 + 1.4])
                pts += [s0, (s0 + cp * d) % L, (s0 + 0.5 * cp * d + 0.5 * nrm) % L]
                r_of.append(r)
    return np.array(pts), np.array(r_of)


@pytest.mark.parametrize("family,L", [("third edge", 30.0), ("side", 36.0)])
def test_p3bca_edges_at_the_cutoff(family, L):
    """Forces, counts and the adjoint (FP64 and mixed) include exactly the triangles the
    reference's FP64 test includes, d^2 <= cutoff^2 on the FP64 positions, with one edge 1e-12 to
    1e-4 (relative) from the cutoff: inside the FP32 uncertainty of the mixed forms, whose guard
    bands then defer to the exact test, and just outside the narrow bands, where the FP32 value
    decides.  The near edge is the third edge (the triplet kernel's test) or
    a side from the apex (the list kernel's).  A triangle left out has exactly zero forces and
    adjoint.  The mixed adjoint is within 1e-5 of the FP64 one."""
    c = 1.5
    P, r = cutoff_triangles(c, L, 17) if family == "third edge" else cutoff_sides(c, L, 19)
    st = {"x": P[:, 0].copy(), "y": P[:, 1].copy(), "z": P[:, 2].copy()}
    box, lo = np.full(3, L), np.zeros(3)
    fx, fy, fz, c_ref = O.forces(st["x"], st["y"], st["z"], 1.0, c, box, lo, nthreads=0)
    ref = np.stack([fx, fy, fz], 1)
    inside = r < 0
    assert c_ref == inside.sum()  # every near edge on its intended side of the cutoff
    per_triangle = lambda a: np.abs(a.reshape(-1, 3, 3)).sum((1, 2)) > 0
    assert np.array_equal(per_triangle(ref), inside)
    gf = np.random.default_rng(3).normal(size=P.shape)
    adj = {}
    for prec, tol in (("fp64", FP64_TOL), ("mixed", MIXED_FORCE_TOL)):
        ctx = Context("p3bca", prec, c)
        ctx.set_state(st)
        ctx.set_domain(box, lo)
        gfx, gfy, gfz, e, cnt = ctx.forces()
        f = np.stack([gfx, gfy, gfz], 1)
        assert cnt == c_ref, (prec, cnt, c_ref)
        assert np.array_equal(per_triangle(f), inside), prec
        assert rel_l2(f, ref) <= tol, prec
        gx, gy, gz, _ = ctx.adjoint(gf[:, 0], gf[:, 1], gf[:, 2], 0.0)
        adj[prec] = np.stack([gx, gy, gz], 1)
        assert np.array_equal(per_triangle(adj[prec]), inside), prec
        ctx.close()
    assert rel_l2(adj["mixed"], adj["fp64"]) <= MIXED_FORCE_TOL


@pytest.mark.parametrize("algo", ["p3bca", "auta", "nata"])
def test_mixed_forces_near_coincident_pairs(algo):
    """Pairs 1e-3 apart, planted beside random particles, carry the largest forces of the system.
    A triplet gradient written in a basis whose two terms nearly cancel for them (e.g. grad_j as
    alpha u + gamma v when j, k are close and i is far) loses FP32 digits in proportion to the
    side ratio, about 1e3 here, and shows directly in the relative L2 error.  Mixed forces stay
    within tolerance overall and on every pair member; NATA, which computes each particle's
    gradient on its own, stays within it on every particle."""
    n, npairs = (4096, 8) if algo == "p3bca" else (256, 4)
    side = generators.box_for_density(n)
    rng = np.random.default_rng(5)
    st = generators.uniform(n, (side, side, side))
    host = rng.choice(n - npairs, npairs, replace=False)
    d = rng.normal(size=(npairs, 3))
    d *= 1e-3 / np.linalg.norm(d, axis=1, keepdims=True)
    for a, k in enumerate("xyz"):
        st[k][n - npairs:] = st[k][host] + d[:, a]
    st = generators.as_csv_values(st)
    members = np.concatenate([host, np.arange(n - npairs, n)])
    if algo == "p3bca":
        cutoff = 2.0
        L, lo = O.domain(st["x"], st["y"], st["z"])
        fx, fy, fz, c_ref = O.forces(st["x"], st["y"], st["z"], 1.0, cutoff, L, lo, nthreads=0)
    else:
        cutoff = 0.0
        fx, fy, fz, c_ref = O.forces(st["x"], st["y"], st["z"], 1.0, -1.0, nthreads=0)
    ref = np.stack([fx, fy, fz], 1)
    # The oracle follows the reference's radial expression (AxilrodTeller.cpp:68-81), whose terms
    # in 1/r^6 cancel for a side of 1e-3: for the P3BCA system it is 3.3e-12 (relative L2) from an
    # 80-bit evaluation of the same triplets, while the FP64 side form is 8.7e-16 from it.
    for prec, tol in (("fp64", 1e-10), ("mixed", MIXED_FORCE_TOL)):
        f, e, c = forces_of(algo, prec, st, cutoff)
        assert c == c_ref, (prec, c, c_ref)
        assert rel_l2(f, ref) <= tol, prec
        if prec == "mixed":
            per = np.linalg.norm(f - ref, axis=1) / np.linalg.norm(ref, axis=1)
            assert per[members].max() <= tol, per[members].max()
            if algo == "nata":
                assert per.max() <= tol, per.max()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_p3bca_ten_steps_vs_oracle(prec):
    """Ten Simulation steps at N=16384 (density 2.048, c=2).  FP64 follows the reference's
    trajectory; the mixed run's trajectory diverges chaotically, so its forces are checked by
    re-evaluating FP64 at the mixed run's own final positions."""
    n = 16384
    side = generators.box_for_density(n)
    st = generators.as_csv_values(generators.uniform(n, (side, side, side)))
    ref, counts = O.simulate("p3bca", 10, st, 0.001, (0.0, -9.81, 0.0), cutoff=2.0, nthreads=0)
    ctx = Context("p3bca", prec, 2.0, 0.001, (0.0, -9.81, 0.0))
    ctx.set_state(st)
    c = ctx.step(10)
    got = ctx.get_state()
    ctx.close()
    if prec == "fp64":
        assert np.array_equal(c, counts)
        check_state(got, ref, FP64_MULTISTEP_FORCE_TOL, FP64_MULTISTEP_TOL)
        return
    assert counts_close(c, counts, 1e-3), (c, counts)
    for k in ("x", "y", "z"):
        assert rel_l2(got[k], ref[k]) <= MIXED_MULTISTEP_POS_TOL, k
    L, lo = O.domain(st["x"], st["y"], st["z"])
    f64 = Context("p3bca", "fp64", 2.0)
    f64.set_state({k: got[k] for k in ("x", "y", "z", "m")})
    f64.set_domain(L, lo)
    fx, fy, fz, _, _ = f64.forces()
    f64.close()
    assert rel_l2(np.stack([got["fx"], got["fy"], got["fz"]], 1), np.stack([fx, fy, fz], 1)) <= MIXED_FORCE_TOL


def test_energy_p3bca_vs_oracle():
    n = 4096
    side = generators.box_for_density(n)
    st = generators.uniform(n, (side, side, side))
    L, lo = O.domain(st["x"], st["y"], st["z"])
    e_ref = O.energy(st["x"], st["y"], st["z"], 1.0, 2.0, L, lo)
    e_abs = O.energy_abs(st["x"], st["y"], st["z"], 1.0, 2.0, L, lo)
    _, e64, _ = forces_of("p3bca", "fp64", st, 2.0)
    _, emx, _ = forces_of("p3bca", "mixed", st, 2.0)
    assert abs(e64 - e_ref) <= 1e-12 * abs(e_ref)
    assert abs(emx - e_ref) <= MIXED_ENERGY_TOL * e_abs


def test_clustered_capacity_retry():
    """Clustered input: the mean-density capacity estimate is far too small in the clusters, the
    overflow is detected on the device and the evaluation is redone with a larger capacity."""
    st = generators.clustered_gauss(8192, 16, (32, 32, 32))
    L, lo = O.domain(st["x"], st["y"], st["z"])
    fx, fy, fz, c_ref = O.forces(st["x"], st["y"], st["z"], 1.0, 2.0, L, lo, nthreads=0)
    f, e, c = forces_of("p3bca", "fp64", st, 2.0)
    assert c == c_ref
    assert rel_l2(f, np.stack([fx, fy, fz], 1)) <= FP64_TOL
    ctx = Context("p3bca", "mixed", 2.0, 0.001, (0, -9.81, 0))
    ctx.set_state(st)
    ref, counts = O.simulate("p3bca", 3, st, 0.001, (0.0, -9.81, 0.0), cutoff=2.0, nthreads=0)
    assert counts_close(ctx.step(3), counts, 1e-3)
    # the same particles again: the grown capacity is kept for this particle count, so the step
    # runs once, where a fresh context's first step overflows and runs a second time
    fresh = Context("p3bca", "mixed", 2.0, 0.001, (0, -9.81, 0))
    fresh.set_state(st)
    k0 = fresh.kernel_launches()
    assert fresh.step(1)[0] == counts[0]
    overflowed = fresh.kernel_launches() - k0
    fresh.close()
    for _ in range(2):
        ctx.set_state(st)
        k0 = ctx.kernel_launches()
        assert ctx.step(1)[0] == counts[0]
        assert ctx.kernel_launches() - k0 < overflowed
    ctx.close()


def converging_lattice(m=13, k=40.0, seed=7):
    """m^3 particles on a jittered cubic lattice at density 2.048 (no close pairs), moving towards the
    centre with velocity -k (x - centre)."""
    rng = np.random.default_rng(seed)
    a = (1 / 2.048) ** (1 / 3)
    idx = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    x = (idx + 0.5) * a + rng.uniform(-0.1, 0.1, idx.shape)
    n = len(x)
    st = {"x": x[:, 0].copy(), "y": x[:, 1].copy(), "z": x[:, 2].copy(), "m": np.ones(n),
          "id": np.arange(n, dtype=np.int32)}
    for i, v in enumerate(("vx", "vy", "vz")):
        st[v] = -k * (x[:, i] - x[:, i].mean())
    for f in ("ax", "ay", "az"):
        st[f] = np.zeros(n)
    return st


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_overflow_inside_a_multi_step_call(prec):
    """A converging lattice: its half lists fit the mean-density capacity (160) at the first steps and
    outgrow it at about the eighth of a 10-step call.  The call is re-run from its snapshot with
    larger lists (the triplet kernel skips its work for the rest of the attempt that overflowed),
    and the result is the oracle's.  The grown capacity is kept, so the same call again runs once."""
    st = converging_lattice()
    ref, counts = O.simulate("p3bca", 10, st, 0.001, (0.0, -9.81, 0.0), cutoff=2.0, nthreads=0)
    assert counts[-1] > 1.5 * counts[0]  # the lattice compresses
    ctx = Context("p3bca", prec, 2.0, 0.001, (0.0, -9.81, 0.0))
    runs = []
    for _ in range(2):
        ctx.set_state(st)
        k0 = ctx.kernel_launches()
        c = ctx.step(10)
        runs.append((c, ctx.get_state(), ctx.kernel_launches() - k0))
    ctx.close()
    assert runs[0][2] > runs[1][2]  # the first call ran its steps twice
    for c, got, _ in runs:
        if prec == "fp64":
            assert np.array_equal(c, counts)
            check_state(got, ref, FP64_MULTISTEP_FORCE_TOL, FP64_MULTISTEP_TOL)
        else:
            assert counts_close(c, counts, 1e-3), (c, counts)
            for k in ("x", "y", "z"):
                assert rel_l2(got[k], ref[k]) <= MIXED_MULTISTEP_POS_TOL, k


@pytest.mark.parametrize("n", [1, 2])
def test_fewer_than_three_particles(n):
    st = generators.uniform(n, (3, 3, 3))
    for algo, cut in (("auta", 0.0), ("nata", 0.0), ("p3bca", 2.0)):
        f, e, c = forces_of(algo, "fp64", st, cut)
        assert c == 0 and not f.any() and e == 0.0


def test_bad_inputs_are_rejected():
    from threebodymdalgorithms_b200 import TbmdError
    ctx = Context("auta")
    st = generators.uniform(8, (3, 3, 3))
    st["x"][3] = np.nan
    with pytest.raises(TbmdError) as e:
        ctx.set_state(st)
    assert e.value.status == 2
    st = generators.uniform(8, (3, 3, 3))
    st["m"][0] = 0.0
    with pytest.raises(TbmdError) as e:
        ctx.set_state(st)
    assert e.value.status == 2
    with pytest.raises(TbmdError) as e:
        ctx.step(1)
    assert e.value.status == 3
    ctx.close()


def test_input_check_over_many_blocks():
    """The input check reduces per warp, then per block, then across blocks: with 100,000 particles
    the lowest bad array, the lowest non-positive mass and the domain extremes (as
    RegularGridDecomposition::getDomainMinMax gives them, padded by 1e-4) must still come out exact."""
    from threebodymdalgorithms_b200 import TbmdError
    n = 100_000
    st = generators.uniform(n, (40, 40, 40))
    ctx = Context("p3bca", "fp64", 2.0)
    ctx.set_state(st)
    _, _, L, lo = ctx.cells(with_particles=False)
    for d, k in enumerate(("x", "y", "z")):
        a, b = st[k].min() - 0.0001, st[k].max() + 0.0001
        assert lo[d] == a and L[d] == abs(b - a), k
    bad = {k: np.array(v, copy=True) for k, v in st.items()}
    bad["vz"][77_777] = np.inf  # array 5, in a late block
    bad["y"][99_999] = np.nan   # array 1, in the last block
    with pytest.raises(TbmdError) as e:
        ctx.set_state(bad)
    assert e.value.status == 2 and "array 1" in str(e.value), str(e.value)
    bad = {k: np.array(v, copy=True) for k, v in st.items()}
    bad["m"][93_000] = -1.0
    bad["m"][1_234] = 0.0
    bad["m"][50_001] = 0.0
    with pytest.raises(TbmdError) as e:
        ctx.set_state(bad)
    assert e.value.status == 2 and "particle 1234 " in str(e.value), str(e.value)
    ctx.close()


def test_autotune_keeps_results(tmp_path):
    st = generators.uniform(2048, (12, 12, 12))
    ref, _, _ = forces_of("auta", "mixed", st)
    ctx = Context("auta", "mixed")
    ctx.set_state(st)
    cache = tmp_path / "tune.jsonl"
    t1 = ctx.autotune(str(cache))
    t2 = ctx.autotune(str(cache))  # second call is served from the cache
    assert t1 == t2 and cache.exists()
    fx, fy, fz, e, c = ctx.forces()
    assert rel_l2(np.stack([fx, fy, fz], 1), ref) <= MIXED_FORCE_TOL
    ctx.close()
