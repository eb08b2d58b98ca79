"""Generate tests/golden/rank_layouts.json: what the reference's own set-up code decides for a run
on P MPI ranks, recorded by running it here.

oracle/_ref/ref_layout (built by oracle/Makefile.ref) wires the reference's Simulation as its main
does and calls Simulation::Init for one rank of P under the stub MPI's layout mode; the process-grid
tables come from its Utility::getDecomposition.  Recorded:
  tables  both grid tables (optimal, naive) for P = 1..1030;
  inputs  the two input CSVs (reference particlegenerator) and their physical domain sizes;
  p3bca   per (input, P, decomposition, cutoff): exit status, stderr line, grid, dims and cutoff boxes
          of rank 0 (P3BCA.cpp:29-70 decides the same on every rank);
  atom    per (algorithm, input, P): particles and dummies of every rank (AtomDecomposition.cpp:15-41).

Run in a container that has the reference sources:  python tests/golden/make_rank_layouts.py
"""
from __future__ import annotations

import json
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "rank_layouts.json"
INPUTS = {"u1000_cube10": ("uniform", 1000, (10.0, 10.0, 10.0)), "u997_box20x10x30": ("uniform", 997, (20.0, 10.0, 30.0))}
P_P3BCA = list(range(1, 31)) + [32, 36, 48, 64, 100, 125, 216, 343, 360, 512, 1000, 1008, 1024]
CUTOFFS = [0.0, 0.5, 1.0, 2.0, 3.0, 5.0]
P_ATOM = list(range(1, 17)) + [31, 100, 997, 1000, 1001]


def main():
    if not O.reference_available() or not (O.REF_DIR / "ref_layout").exists():
        O.build_reference()
    doc = {"tables": O.reference_grid_tables(), "inputs": {}, "p3bca": [], "atom": []}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (gen, n, box) in INPUTS.items():
            path = f"{tmp}/{name}.csv"
            O.reference_generate(path, gen, n, box)
            st = O.read_csv(path)
            L, lo = O.domain(st["x"], st["y"], st["z"])
            doc["inputs"][name] = {"n": n, "L": [float(v) for v in L]}
            for P in P_P3BCA:
                for dec in ("naive", "optimal"):
                    for c in CUTOFFS:
                        rc, err, out = O.reference_layout(path, "p3bca", P, 0, c, dec)
                        doc["p3bca"].append({"input": name, "P": P, "decomp": dec, "cutoff": c, "rc": rc,
                                             "stderr": err, "grid": out["grid"] if out else None,
                                             "dims": out["dims"] if out else None,
                                             "cutoff_boxes": out["cutoff_boxes"] if out else None})
            for algo in ("nata", "auta"):
                for P in P_ATOM:
                    ranks = range(P) if P <= 16 else sorted({0, 1, P // 2, P - 2, P - 1})
                    mine, dums = [], []
                    for r in ranks:
                        rc, err, out = O.reference_layout(path, algo, P, r)
                        assert rc == 0, (algo, P, r, err)
                        mine.append(out["my_particles"])
                        dums.append(out["my_dummies"])
                    doc["atom"].append({"algo": algo, "input": name, "P": P, "ranks": list(ranks),
                                        "my_particles": mine, "my_dummies": dums})
    OUT.write_text(json.dumps(doc, separators=(",", ":")) + "\n")
    print(OUT, OUT.stat().st_size, "bytes;", len(doc["p3bca"]), "p3bca cases,", len(doc["atom"]), "atom cases")


if __name__ == "__main__":
    main()
