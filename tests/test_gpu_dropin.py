"""The drop-in executable against the reference executable's own CSV output (golden files)."""
import json
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

from threebodymdalgorithms_b200 import csvio

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
MAIN = ROOT / "threebodymdalgorithms_b200" / "tbmd_main"
GOLDEN = ROOT / "tests" / "golden"


def run_main(args, cwd):
    r = subprocess.run([str(MAIN), *args], capture_output=True, text=True, cwd=cwd)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


@pytest.mark.parametrize("name,args,last", [
    ("c1_auta_n512", ["-a", "auta", "-i", "1"], 0),
    ("p3bca_n512_c2_3steps", ["-a", "p3bca", "-i", "3", "-c", "2.0"], 2),
])
def test_cli_output_matches_reference(name, args, last, tmp_path):
    run_main(args + ["-d", "0.001", "-gx", "0", "-gy", "-9.81", "-gz", "0", "-csv", str(GOLDEN / f"{name}.csv"),
                     "-o", str(tmp_path / "out.csv")], tmp_path)
    mine = (tmp_path / f"out_{last}.csv").read_text().splitlines()
    ref = (GOLDEN / f"{name}_cli_out_{last}.csv").read_text().splitlines()
    assert mine[0] == ref[0] and len(mine) == len(ref)
    # 6-digit text: identical except where an FP64 rounding difference crosses a print boundary
    differing = [i for i in range(len(ref)) if mine[i] != ref[i]]
    assert len(differing) <= 2, differing[:5]
    a = csvio.read_particles(str(tmp_path / f"out_{last}.csv"))
    b = csvio.read_particles(str(GOLDEN / f"{name}_cli_out_{last}.csv"))
    for k in ("x", "vx", "ax"):
        assert np.allclose(a[k], b[k], rtol=2e-6, atol=1e-12)


def test_cli_mixed_and_dump(tmp_path):
    run_main(["-a", "P3BCA", "-i", "2", "-c", "2", "-d", "0.001", "-gy", "-9.81", "-prec", "mixed",
              "-csv", str(GOLDEN / "p3bca_n512_c2_3steps.csv"), "-dumpfull", str(tmp_path / "d.txt"),
              "-op", str(tmp_path / "prof.json"), "-opsteps", str(tmp_path / "steps.json")], tmp_path)
    lines = (tmp_path / "d.txt").read_text().splitlines()
    assert lines[0].startswith("step 0 buffer 1 triplets 12982")
    steps = [json.loads(line) for line in (tmp_path / "steps.json").read_text().splitlines()]
    assert len(steps) == 2 and steps[0]["triplets"] == 12982 and steps[0]["max"] > 0
    prof = json.loads((tmp_path / "prof.json").read_text())
    # the reference's PROFILE_3BMDA document shape (main.cpp:127-451)
    assert set(prof) == {"times", "hitrate", "hitrate per proc", "stvr"}
    forces = prof["times"]["calculateForces"]
    assert forces["time unit"] == "nanosecond" and len(forces["times per proc"]["0"]) == 2
    assert all(t > 0 for t in forces["times per proc"]["0"])
    assert prof["hitrate"]["avg hitrate per sim step"][0] == pytest.approx(12982 / math.comb(512, 3))


def test_cli_np_gives_the_same_results(tmp_path):
    """-np P reproduces the reference's P-rank set-up but computes the same triplets on the GPU: the
    NATA run (a deterministic sweep) writes the same bytes for P = 1 and P = 3, and so does a P3BCA
    run whose cutoff window is valid at P = 3 (the counts are exact; the files agree to 6 digits)."""
    inp = GOLDEN / "p3bca_n512_c2_3steps.csv"
    for P in ("1", "3"):
        d = tmp_path / f"np{P}"
        d.mkdir()
        run_main(["-a", "nata", "-i", "2", "-d", "0.001", "-gy", "-9.81", "-np", P, "-csv", str(inp),
                  "-o", str(d / "o.csv")], d)
        run_main(["-a", "p3bca", "-i", "2", "-c", "1.0", "-d", "0.001", "-gy", "-9.81", "-np", P,
                  "-dumpfull", str(d / "p3.txt"), "-csv", str(inp)], d)
    assert (tmp_path / "np1" / "o_1.csv").read_bytes() == (tmp_path / "np3" / "o_1.csv").read_bytes()
    counts = [[l for l in (tmp_path / f"np{P}" / "p3.txt").read_text().splitlines() if l.startswith("step")]
              for P in ("1", "3")]
    assert counts[0] == counts[1] and len(counts[0]) == 2


def test_checkpoint_resumes_exactly(tmp_path):
    """-checkpoint writes the state as an input CSV at 17 digits: resuming from it with -csv gives the
    same state as running straight through.  NATA's sweep is deterministic, so three steps in one run
    and two steps, a checkpoint and one more step agree bit for bit."""
    inp = str(GOLDEN / "c1_auta_n512.csv")
    common = ["-a", "nata", "-d", "0.001", "-gy", "-9.81"]
    run_main(common + ["-i", "3", "-csv", inp, "-checkpoint", str(tmp_path / "straight.csv")], tmp_path)
    run_main(common + ["-i", "2", "-csv", inp, "-checkpoint", str(tmp_path / "half.csv")], tmp_path)
    run_main(common + ["-i", "1", "-csv", str(tmp_path / "half.csv"), "-checkpoint", str(tmp_path / "resumed.csv")],
             tmp_path)
    a = (tmp_path / "straight.csv").read_text()
    b = (tmp_path / "resumed.csv").read_text()
    assert a.splitlines()[0] == "ID, pX, pY, pZ, vX, vY, vZ, aX, aY, aZ, m, fX, fY, fZ"
    assert a == b
