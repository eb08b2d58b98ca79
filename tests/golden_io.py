"""Loading helpers for the golden fixtures in tests/golden (made by tests/golden/make_golden.py)."""
import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")


def names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(z["meta"]))
    inp = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    out = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return inp, out, z["counts"].astype(np.uint64), meta
