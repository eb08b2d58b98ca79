"""Particle CSV files in the reference's format.

Input (src/utility/utility.cpp:14-24): a header row, then ID, pX, pY, pZ, vX, vY, vZ, aX, aY, aZ, m;
columns after m are ignored, so an output file can be read back as input (restart).
Output (utility.cpp:54-68, Simulation.cpp:74-79, 99-133): one file per step named
<base>_<step>.csv, where <base> is the -o path up to its last '.', rows sorted by ID, every value
written with the default ostream format (6 significant digits, the same as printf "%g").
"""
from __future__ import annotations

import numpy as np

IN_KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")
OUT_HEADER = "ID, pX, pY, pZ, vX, vY, vZ, aX, aY, aZ, m, fX, fY, fZ\n"
OUT_KEYS = IN_KEYS + ("fx", "fy", "fz")


def read_particles(path: str) -> dict:
    rows = []
    ids = []
    with open(path) as f:
        next(f, None)  # header
        for line in f:
            line = line.strip()
            if not line:
                continue
            cells = line.split(",")
            vals = [float(c) for c in cells]
            ids.append(int(cells[0]))
            rows.append(vals[1:11])
    a = np.array(rows, dtype=np.float64).reshape(-1, 10)
    st = {k: np.ascontiguousarray(a[:, i]) for i, k in enumerate(IN_KEYS)}
    st["id"] = np.array(ids, dtype=np.int32)
    return st


def step_path(base: str, step: int) -> str:
    dot = base.rfind(".")
    stem = base if dot < 0 else base[:dot]
    return f"{stem}_{step}.csv"


def write_step(path: str, st: dict) -> None:
    order = np.argsort(st["id"], kind="stable")
    with open(path, "w") as f:
        f.write(OUT_HEADER)
        cols = [st[k] for k in OUT_KEYS]
        for i in order:
            f.write(str(int(st["id"][i])) + ", " + ", ".join("%g" % c[i] for c in cols) + "\n")


def write_input(path: str, st: dict) -> None:
    with open(path, "w") as f:
        f.write("ID, pX, pY, pZ, vX, vY, vZ, aX, aY, aZ, m\n")
        cols = [st[k] for k in IN_KEYS]
        for i in range(len(st["x"])):
            f.write(str(int(st["id"][i])) + ", " + ", ".join("%g" % c[i] for c in cols) + "\n")
