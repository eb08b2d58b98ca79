"""Generate the golden fixtures in tests/golden/ from the reference itself.

Every fixture is produced by the reference's own code built from its sources by
oracle/Makefile.ref: inputs by its particlegenerator (src/tools, 6-significant-digit CSV, parsed
back exactly as its CSV reader does) or by a hand-written CSV for edge cases, outputs by
oracle/_ref/ref_dump, which drives its Simulation/Algorithm/AxilrodTeller classes at one rank.

Each <name>.npz holds in_<field> (the parsed input), out_<field> (the reference's state after the
run, in its decomposition order, %.17g round-tripped exactly), counts (triplets per step) and meta
(JSON: algorithm, mode, iterations, dt, g, cutoff, nu).

Run in a container that has the reference sources:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent
SEED0, SEED1 = 926762934, 89347587
G = (0.0, -9.81, 0.0)


def write_csv(path, rows):
    with open(path, "w") as f:
        f.write("ID, pX, pY, pZ, vX, vY, vZ, aX, aY, aZ, m\n")
        for r in rows:
            f.write(", ".join(repr(v) if isinstance(v, float) else str(v) for v in r) + "\n")


CASES = []


def case(name, algo, mode="sim", iters=1, dt=0.001, g=G, cutoff=0.0, nu=1.0, gen=None, rows=None, keep_csv=False):
    CASES.append(dict(name=name, algo=algo, mode=mode, iters=iters, dt=dt, g=g, cutoff=cutoff, nu=nu, gen=gen,
                      rows=rows, keep_csv=keep_csv))


# The reference's own test fixture (src/tests/tests.cpp:21-74): 1000 uniform in 10^3, mass 1e-4;
# its count test pins C(1000,3) = 166,167,000 (tests.cpp:530-568).
case("tests_fixture_n1000_auta", "auta", mode="forces", gen=("uniform", 1000, (10, 10, 10), 1e-4))
# C1: plain AUTA, N=512 uniform in 10^3, mass 1, one step, dt 0.001, g (0,-9.81,0).
case("c1_auta_n512", "auta", iters=1, gen=("uniform", 512, (10, 10, 10), 1.0), keep_csv=True)
case("nata_n256_3steps", "nata", iters=3, gen=("uniform", 256, (6, 6, 6), 1.0))
case("auta_n300_light_3steps", "auta", iters=3, gen=("uniform", 300, (5, 5, 5), 1e-3))
case("p3bca_n512_c2_3steps", "p3bca", iters=3, cutoff=2.0, gen=("uniform", 512, (10, 10, 10), 1.0), keep_csv=True)
case("p3bca_n1000_c1.5_2steps", "p3bca", iters=2, cutoff=1.5, gen=("uniform", 1000, (8, 8, 8), 1.0))
case("p3bca_clustered_n512_c2", "p3bca", iters=2, cutoff=2.0,
     gen=("clusteredgauss", 512, (16, 16, 16), 1.0, ["--numclusters", "16", "--distmean", "0", "--diststddev", "1"]))
case("p3bca_light_drift_n400_c2_4steps", "p3bca", iters=4, cutoff=2.0, gen=("uniform", 400, (8, 8, 8), 1e-3))
case("p3bca_n512_c0_nocutoff", "p3bca", iters=1, cutoff=0.0, gen=("uniform", 128, (5, 5, 5), 1.0))
# Edge cases (hand-written inputs).
case("edge_n3_auta", "auta", mode="forces", rows=[(0, 0.0, 0.0, 0.0, 0, 0, 0, 0, 0, 0, 1.0),
                                                   (1, 1.0, 0.2, 0.0, 0, 0, 0, 0, 0, 0, 1.0),
                                                   (2, 0.3, 0.9, 0.4, 0, 0, 0, 0, 0, 0, 1.0)])
case("edge_n4_nata_2steps", "nata", iters=2,
     rows=[(7, 0.0, 0.0, 0.0, 0.5, 0, 0, 1.5, 0, 0, 2.0), (3, 1.1, 0.0, 0.1, 0, -0.2, 0, 0, 0, 0, 1.0),
           (3, 0.2, 1.0, 0.0, 0, 0, 0.3, 0, 0.7, 0, 1.0), (1, 0.5, 0.4, 1.2, 0, 0, 0, -2.0, 0, 0, 0.5)])
# Pairs at exactly the cutoff: a line with spacing 0.75 and c = 1.5 (all values exact in binary),
# so (i, i+1, i+2) has a pair at d == c (inside) and (i, i+1, i+3) is outside.
case("edge_line_exact_cutoff", "p3bca", mode="forces", cutoff=1.5,
     rows=[(i, 0.75 * i, 0.0, 0.0, 0, 0, 0, 0, 0, 0, 1.0) for i in range(12)] +
          [(12 + i, 0.75 * i, 4.0, 0.0, 0, 0, 0, 0, 0, 0, 1.0) for i in range(12)])
# Periodic wrap: two clumps at opposite faces of the box form triplets only through the
# min-image test, while their forces use the raw (unwrapped) displacements.
case("edge_periodic_wrap", "p3bca", mode="forces", cutoff=1.2,
     rows=[(0, 0.05, 5.0, 5.0, 0, 0, 0, 0, 0, 0, 1.0), (1, 0.4, 5.3, 5.1, 0, 0, 0, 0, 0, 0, 1.0),
           (2, 9.95, 5.1, 4.9, 0, 0, 0, 0, 0, 0, 1.0), (3, 9.6, 4.8, 5.2, 0, 0, 0, 0, 0, 0, 1.0),
           (4, 5.0, 0.02, 5.0, 0, 0, 0, 0, 0, 0, 1.0), (5, 5.1, 9.97, 5.3, 0, 0, 0, 0, 0, 0, 1.0),
           (6, 4.8, 9.7, 4.7, 0, 0, 0, 0, 0, 0, 1.0), (7, 5.0, 5.0, 0.0, 0, 0, 0, 0, 0, 0, 1.0),
           (8, 5.2, 5.3, 10.0, 0, 0, 0, 0, 0, 0, 1.0), (9, 2.0, 2.0, 2.0, 0, 0, 0, 0, 0, 0, 1.0)])
# Particles on cell faces: a cubic lattice with spacing equal to the cell width.
case("edge_lattice_faces", "p3bca", mode="forces", cutoff=1.0,
     rows=[(i + 4 * j + 16 * k, 1.0 * i, 1.0 * j, 1.0 * k, 0, 0, 0, 0, 0, 0, 1.0)
           for k in range(4) for j in range(4) for i in range(4)] +
          [(64, 0.5, 0.5, 0.5, 0, 0, 0, 0, 0, 0, 1.0), (65, 1.5, 0.5, 0.5, 0, 0, 0, 0, 0, 0, 1.0)])


def main():
    O.build_reference()
    assert O.reference_available(), "oracle/_ref was not built"
    with tempfile.TemporaryDirectory() as tmp:
        for c in CASES:
            csv = str(Path(tmp) / f"{c['name']}.csv")
            if c["gen"]:
                gen, n, box, mass, *extra = c["gen"]
                O.reference_generate(csv, gen, n, box, mass, SEED0, SEED1, extra[0] if extra else None)
            else:
                write_csv(csv, c["rows"])
            inp = O.read_csv(csv)
            out, counts, secs = O.reference_dump(csv, c["algo"], c["mode"], c["iters"], c["dt"], c["g"], c["cutoff"],
                                                 c["nu"])
            meta = {k: c[k] for k in ("algo", "mode", "iters", "dt", "g", "cutoff", "nu")}
            arrays = {f"in_{k}": v for k, v in inp.items()}
            arrays.update({f"out_{k}": v for k, v in out.items()})
            np.savez_compressed(OUT / f"{c['name']}.npz", counts=counts, meta=np.array(json.dumps(meta)), **arrays)
            if c["keep_csv"]:
                Path(OUT / f"{c['name']}.csv").write_text(Path(csv).read_text())
                # the reference's own executable on the same input: its per-step CSV output files
                base = str(Path(tmp) / f"{c['name']}_cli.csv")
                cmd = [str(O.REF_DIR / "ref_main"), "-a", c["algo"], "-i", str(c["iters"]), "-d", repr(c["dt"]),
                       "-gx", repr(c["g"][0]), "-gy", repr(c["g"][1]), "-gz", repr(c["g"][2]), "-csv", csv,
                       "-o", base]
                if c["algo"] == "p3bca":
                    cmd += ["-c", repr(c["cutoff"])]
                subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
                last = c["iters"] - 1
                Path(OUT / f"{c['name']}_cli_out_{last}.csv").write_text(
                    Path(tmp, f"{c['name']}_cli_{last}.csv").read_text())
            print(f"{c['name']:36s} n={len(inp['x']):5d} counts={counts.tolist()} ({secs:.2f}s)")


if __name__ == "__main__":
    main()
