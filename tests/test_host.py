"""Host-side logic without a GPU: input generators, the reference CSV format, the drop-in CLI."""
import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_io as GIO
from threebodymdalgorithms_b200 import csvio, generators

ROOT = Path(__file__).resolve().parents[1]
MAIN = ROOT / "threebodymdalgorithms_b200" / "tbmd_main"
GOLDEN = ROOT / "tests" / "golden"


def test_uniform_generator_matches_reference_input():
    """c1_auta_n512.csv was written by the reference's particlegenerator."""
    ref = csvio.read_particles(str(GOLDEN / "c1_auta_n512.csv"))
    mine = generators.as_csv_values(generators.uniform(512, (10, 10, 10), 1.0))
    for k in ("x", "y", "z", "vx", "m"):
        assert np.array_equal(ref[k], mine[k]), k


def test_generators_match_reference_fixtures():
    inp, _, _, _ = GIO.load("tests_fixture_n1000_auta")
    mine = generators.as_csv_values(generators.uniform(1000, (10, 10, 10), 1e-4))
    for k in ("x", "y", "z", "m"):
        assert np.array_equal(inp[k], mine[k]), k
    inp, _, _, _ = GIO.load("p3bca_clustered_n512_c2")
    mine = generators.as_csv_values(generators.clustered_gauss(512, 16, (16, 16, 16)))
    for k in ("x", "y", "z"):
        assert np.array_equal(inp[k], mine[k]), k


def test_density_box():
    assert generators.box_for_density(131072, 2.048) == pytest.approx(40.0, abs=1e-12)


@pytest.mark.parametrize("name,step", [("c1_auta_n512", 0), ("p3bca_n512_c2_3steps", 2)])
def test_csv_writer_matches_reference_cli_output(name, step, tmp_path):
    """Writing the reference's full-precision final state reproduces its own CLI file byte for byte."""
    _, out, _, _ = GIO.load(name)
    path = tmp_path / "o.csv"
    csvio.write_step(str(path), out)
    assert path.read_text() == (GOLDEN / f"{name}_cli_out_{step}.csv").read_text()


def test_csv_roundtrip_ignores_force_columns(tmp_path):
    _, out, _, _ = GIO.load("c1_auta_n512")
    path = tmp_path / "o.csv"
    csvio.write_step(str(path), out)
    back = csvio.read_particles(str(path))
    assert np.array_equal(back["id"], np.sort(out["id"]))
    assert np.allclose(back["x"], out["x"][np.argsort(out["id"])], rtol=1e-5)


def test_step_path_like_reference():
    assert csvio.step_path("out.csv", 3) == "out_3.csv"
    assert csvio.step_path("a.b/out.csv", 0) == "a.b/out_0.csv"


def _parse(*args):
    r = subprocess.run([str(MAIN), *args, "-parseonly"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1]), r.stdout


@pytest.mark.skipif(not MAIN.exists(), reason="tbmd_main not built")
def test_cli_defaults_and_flags():
    a, _ = _parse()
    assert a["algorithm"] == "nata" and a["iterations"] == 0 and a["cutoff"] == 0 and a["delta"] == 0
    a, _ = _parse("-a", "p3bca", "-i", "10", "-d", "0.001", "-gx", "0", "-gy", "-9.81", "-gz", "0", "-c", "2",
                  "-csv", "in.csv", "-o", "out.csv")
    assert (a["algorithm"], a["iterations"], a["delta"], a["cutoff"]) == ("p3bca", 10, 0.001, 2.0)
    assert a["g"] == [0.0, -9.81, 0.0] and a["csv"] == "in.csv" and a["out"] == "out.csv"
    a, _ = _parse("--algorithm", "AUTA", "--iterations", "3", "--cutoff", "1.5", "-prec", "mixed")
    assert (a["algorithm"], a["iterations"], a["cutoff"], a["precision"]) == ("auta", 3, 1.5, "mixed")


@pytest.mark.skipif(not MAIN.exists(), reason="tbmd_main not built")
def test_cli_errors_like_reference():
    _, out = _parse("-bogus", "stray")
    assert "CLI parser: unrecognized option: bogus" in out and "unrecognized option: stray" in out
    for bad in (["-i"], ["-a", "fast"], ["-c", "abc"], ["-decomp", "best"]):
        r = subprocess.run([str(MAIN), *bad], capture_output=True, text=True)
        assert r.returncode == 1 and "Help:" in r.stdout, bad


REF_MAIN = ROOT / "oracle" / "_ref" / "ref_main"


@pytest.mark.skipif(not (MAIN.exists() and REF_MAIN.exists()), reason="tbmd_main or the reference build absent")
def test_cli_help_is_the_references():
    """A flag without its value prints the help and exits 1 in both programs (cli.hpp:54-58).  The
    reference's 15 help lines (cli.hpp:27-45, its "-gx,--gravityZ" label included) come out byte for
    byte; this build's own options follow them."""
    ref = subprocess.run([str(REF_MAIN), "-c"], capture_output=True)
    mine = subprocess.run([str(MAIN), "-c"], capture_output=True)
    assert ref.returncode == 1 and mine.returncode == 1
    ref_lines = ref.stdout.split(b"\n")
    assert len(ref_lines) == 16 and ref_lines[-1] == b""
    assert mine.stdout.split(b"\n")[:15] == ref_lines[:15]
    assert b"GPU options:" in mine.stdout


@pytest.mark.skipif(not MAIN.exists(), reason="tbmd_main not built")
def test_cli_missing_input_fails():
    r = subprocess.run([str(MAIN), "-csv", "/nonexistent.csv", "-i", "1"], capture_output=True, text=True)
    assert r.returncode == 1


def _summary(path):
    r = subprocess.run([str(MAIN), "-csv", str(path), "-inputsummary"], capture_output=True, text=True)
    return r.returncode, r.stdout, r.stderr


@pytest.mark.parametrize("name", ["c1_auta_n512.csv", "p3bca_n512_c2_3steps.csv"])
def test_dropin_reads_csv_like_the_reference(name, tmp_path):
    """The drop-in's parallel CSV reader gives exactly what a correctly rounded parse gives (the
    reference reads with strtod semantics), also with blank lines, CRLF line ends and extra columns."""
    src = GOLDEN / name
    lines = src.read_text().splitlines()
    messy = tmp_path / "messy.csv"
    body = [lines[0]] + [l + ", 7, 8" if i % 3 == 0 else l for i, l in enumerate(lines[1:])]
    body.insert(5, "   ")
    body.insert(9, "")
    messy.write_bytes(("\r\n".join(body) + "\r\n").encode())
    ref = csvio.read_particles(str(src))
    for path in (src, messy):
        rc, out, err = _summary(path)
        assert rc == 0, err
        d = json.loads(out)
        assert d["n"] == len(ref["x"]) and d["id_sum"] == int(np.sum(ref["id"]))
        for k, key in enumerate(("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")):
            col = ref[key]
            assert d["columns"][k] == [col[0], col[-1], col.min(), col.max()], key


def test_dropin_csv_errors(tmp_path):
    head = "ID, pX, pY, pZ, vX, vY, vZ, aX, aY, aZ, m\n"
    good = "0, 1, 2, 3, 0, 0, 0, 0, 0, 0, 1\n"
    for body, msg in ((good + "1, 2, 3\n", "row 1 has fewer than 11 columns"),
                      (good + good + "x, 1, 2, 3, 0, 0, 0, 0, 0, 0, 1\n", "row 2: bad ID"),
                      (good + "1, 1, oops, 3, 0, 0, 0, 0, 0, 0, 1\n", "row 1: bad number ' oops'")):
        f = tmp_path / "bad.csv"
        f.write_text(head + body)
        rc, out, err = _summary(f)
        assert rc == 1 and msg in err, (rc, err)
