"""Layout of the reference's run on P MPI ranks (tbmd_rank_layout_of, tbmd_main -np P) against
the reference's own set-up code.

tests/golden/rank_layouts.json was recorded by tests/golden/make_rank_layouts.py, which runs the
reference's Simulation::Init for rank r of P (oracle/refstub/ref_layout.cpp under the stub MPI's
layout mode) and its Utility::getDecomposition tables.  Host code only: no GPU."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import pytest

from oracle import oracle as O
from threebodymdalgorithms_b200 import TbmdError, rank_layout

ROOT = Path(__file__).resolve().parents[1]
GOLD = json.loads((ROOT / "tests" / "golden" / "rank_layouts.json").read_text())
MAIN = ROOT / "threebodymdalgorithms_b200" / "tbmd_main"
CSV = ROOT / "tests" / "golden" / "p3bca_n512_c2_3steps.csv"
TBMD_RANK_LAYOUT = 9


@pytest.mark.parametrize("decomposition", ["optimal", "naive"])
def test_process_grids_match_the_reference_tables(decomposition):
    """Every P = 1..1030: the grid the reference's table gives (empty past 1024, where its run
    fails) and the one tbmd_rank_layout_of builds."""
    table = GOLD["tables"][decomposition]
    for P in range(1, 1031):
        grid = table[str(P)]
        if not grid:
            with pytest.raises(TbmdError) as e:
                rank_layout("p3bca", P, 1000, 1e-6, [1000.0] * 3, decomposition)
            assert e.value.status == TBMD_RANK_LAYOUT
            continue
        # a cutoff far below the cell width passes the cutoff-window check for every grid
        lay = rank_layout("p3bca", P, 1000, 1e-6, [1000.0] * 3, decomposition)
        assert lay["num_dims"] == len(grid), P
        assert lay["dims"][: len(grid)] == grid and all(d == 1 for d in lay["dims"][len(grid):]), (P, grid)


def test_p3bca_layout_and_exit_match_the_reference_setup():
    """1032 runs of the reference's P3BCA set-up over two inputs, P up to 1024, both grids and cutoffs
    from 0 to 5: where it exits (status 1) the same status and stderr line, elsewhere the same grid and
    cutoff boxes."""
    for case in GOLD["p3bca"]:
        inp = GOLD["inputs"][case["input"]]
        args = ("p3bca", case["P"], inp["n"], case["cutoff"], inp["L"], case["decomp"])
        if case["rc"] != 0:
            assert case["rc"] == 1, case
            with pytest.raises(TbmdError) as e:
                rank_layout(*args)
            assert e.value.status == TBMD_RANK_LAYOUT
            assert str(e.value) == "TBMD_RANK_LAYOUT: " + case["stderr"], case
        else:
            lay = rank_layout(*args)
            assert lay["dims"] == case["dims"], case
            assert lay["cutoff_boxes"] == case["cutoff_boxes"], case
            assert lay["num_dims"] == len(case["grid"]), case


def test_p3bca_shift_steps():
    """Rounds per Simulation step (P3BCA::calcSteps, P3BCA.cpp:79-92) for each grid dimension."""
    one = rank_layout("p3bca", 7, 1000, 2.0, [40.0] * 3)  # 1-D, nCbX = ceil(2 / (40 / 7)) = 1
    assert one["cutoff_boxes"] == [1, 0, 0] and one["shift_steps"] == 2
    two = rank_layout("p3bca", 49, 1000, 3.0, [70.0] * 3, "optimal")  # 7 x 7, cell 10: 1 box each
    assert two["dims"] == [7, 7, 1] and two["shift_steps"] == 2 * 1 * 1 + 1 + 1 + 1
    three = rank_layout("p3bca", 343, 1000, 12.0, [70.0] * 3, "optimal")  # 7^3, cell 10: 2 boxes each
    assert three["dims"] == [7, 7, 7] and three["cutoff_boxes"] == [2, 2, 2]
    assert three["shift_steps"] == 1 + 2 + 2 * (2 * 2 + 1) + 2 * (5 * 5)
    assert rank_layout("p3bca", 1, 1000, 2.0, [40.0] * 3)["shift_steps"] == 1


def test_atom_decomposition_padding_matches_the_reference_setup():
    """NATA / AUTA: every rank holds ceil(N / P) particles, dummies included, and the dummies over
    all ranks are P - N mod P (none when P divides N), as the reference's AtomDecomposition::Init
    gives them rank by rank."""
    for case in GOLD["atom"]:
        n, P = GOLD["inputs"][case["input"]]["n"], case["P"]
        lay = rank_layout(case["algo"], P, n)
        assert all(k == lay["particles_per_rank"] for k in case["my_particles"]), case
        if len(case["ranks"]) == P:
            assert sum(case["my_dummies"]) == lay["dummies"], case
        for r, d in zip(case["ranks"], case["my_dummies"]):
            assert d == (1 if n % P and r < P - n % P else 0), (case, r)


def test_rank_layout_rejects_bad_arguments():
    for bad in (("p3bca", 0, 10, 1.0, [1.0] * 3), ("p3bca", 4, -1, 1.0, [1.0] * 3),
                ("p3bca", 4, 10, 1.0, [0.0, 1.0, 1.0]), ("p3bca", 4, 10, float("nan"), [1.0] * 3)):
        with pytest.raises(TbmdError) as e:
            rank_layout(*bad)
        assert e.value.status == 1


def _main(*args):
    return subprocess.run([str(MAIN), *args], capture_output=True, text=True, timeout=60)


def test_dropin_np_stops_where_the_reference_stops():
    """tbmd_main -np P: the layout is checked on the host before any device work; an invalid
    cutoff window ends the run with the reference's stderr line and status 1, -layoutonly prints the
    layout.  Neither needs a GPU."""
    assert MAIN.exists(), "build the drop-in first (python -m threebodymdalgorithms_b200.build)"
    st = O.read_csv(str(CSV))
    L, _ = O.domain(st["x"], st["y"], st["z"])
    for P, c, dec in ((4, 3.0, "naive"), (3, 0.0, "naive"), (27, 5.0, "optimal"), (9, 5.0, "naive")):
        with pytest.raises(TbmdError) as e:
            rank_layout("p3bca", P, len(st["x"]), c, L, dec)
        r = _main("-a", "p3bca", "-np", str(P), "-decomp", dec, "-c", repr(c), "-csv", str(CSV), "-i", "1")
        assert r.returncode == 1
        assert r.stderr.strip() == str(e.value).split(": ", 1)[1]
    r = _main("-a", "p3bca", "-np", "27", "-decomp", "optimal", "-c", "1", "-csv", str(CSV), "-layoutonly")
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    lay = rank_layout("p3bca", 27, len(st["x"]), 1.0, L, "optimal")
    assert out["dims"] == lay["dims"] and out["cutoff_boxes"] == lay["cutoff_boxes"]
    assert out["shift_steps"] == lay["shift_steps"]
    r = _main("-a", "auta", "-np", "7", "-csv", str(CSV), "-layoutonly")
    assert r.returncode == 0 and json.loads(r.stdout)["dummies"] == 7 - 512 % 7
    r = _main("-a", "p3bca", "-np", "2000", "-c", "1", "-csv", str(CSV))
    assert r.returncode == 1 and "1024" in r.stderr


@pytest.mark.skipif(not (O.REF_DIR / "ref_layout").exists(), reason="reference build (oracle/_ref) not present")
def test_dropin_np_against_the_reference_live():
    """Where the reference's build is present: its own set-up on the committed 512-particle input
    and tbmd_main -np on the same file stop, or not, alike."""
    for P, c, dec in ((2, 0.0, "naive"), (4, 3.0, "naive"), (5, 2.0, "naive"), (9, 2.0, "optimal"),
                      (27, 1.0, "optimal"), (64, 1.5, "optimal"), (12, 4.0, "optimal")):
        rc, err, out = O.reference_layout(str(CSV), "p3bca", P, 0, c, dec)
        r = _main("-a", "p3bca", "-np", str(P), "-decomp", dec, "-c", repr(c), "-csv", str(CSV), "-layoutonly")
        assert r.returncode == rc, (P, c, dec, err, r.stderr)
        if rc:
            assert r.stderr.strip() == err
        else:
            got = json.loads(r.stdout)
            assert got["dims"] == out["dims"] and got["cutoff_boxes"] == out["cutoff_boxes"]
