"""ctypes wrapper around the CPU oracle (oracle/at_oracle.c) and the reference build (oracle/_ref).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by bench.py's CPU-baseline
leg, never by the product package.  See at_oracle.c for what each function restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
# Where the reference's sources are read when present (the build machine only): the directory named
# by TBMD_REFERENCE_ROOT, else a checkout named "reference" beside this repository.
REFERENCE_ROOT = Path(os.environ.get("TBMD_REFERENCE_ROOT", str(HERE.parent.parent / "reference")))
STUB_INCLUDE = HERE / "refstub" / "inc"  # stand-in mpi.h and Eigen/Dense for the reference's headers

ALGORITHMS = {"nata": 0, "p3bca": 1, "auta": 2}

_lib = None


def build(force: bool = False) -> Path:
    """Compile at_oracle.c into oracle/liboracle.so (gcc, OpenMP, no FMA contraction)."""
    src = HERE / "at_oracle.c"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-shared", "-fPIC", str(src),
                        "-o", str(LIB_PATH), "-lm"], check=True)
    return LIB_PATH


def build_reference(ref_root: str = str(REFERENCE_ROOT), jobs: int = 8) -> bool:
    """Build oracle/_ref from the reference sources with oracle/Makefile.ref; False if absent."""
    if not Path(ref_root, "src").is_dir():
        return (REF_DIR / "ref_dump").exists()
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile.ref"), f"REF={ref_root}", f"-j{jobs}"],
                   check=True)
    return True


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        d = C.POINTER(C.c_double)
        i64 = C.c_int64
        _lib.tbo_domain.argtypes = [i64, d, d, d, d, d]
        _lib.tbo_forces_bruteforce.argtypes = [i64, d, d, d, C.c_double, C.c_double, d, d, d, d, C.c_int]
        _lib.tbo_forces_bruteforce.restype = C.c_uint64
        _lib.tbo_forces_cells.argtypes = [i64, d, d, d, C.c_double, C.c_double, d, d, d, d, d, C.c_int]
        _lib.tbo_forces_cells.restype = C.c_uint64
        _lib.tbo_forces_selected.argtypes = [i64, d, d, d, C.c_double, C.POINTER(C.c_int64), i64, d, d, d,
                                             C.c_int]
        _lib.tbo_forces_selected.restype = None
        _lib.tbo_cell_dims.argtypes = [d, C.c_double, C.POINTER(C.c_int), d]
        _lib.tbo_cell_assign.argtypes = [i64, d, d, d, C.c_double, d, d, C.POINTER(C.c_int),
                                         C.POINTER(C.c_int32)]
        _lib.tbo_energy.argtypes = [i64, d, d, d, C.c_double, C.c_double, d, d, C.c_int]
        _lib.tbo_energy.restype = C.c_double
        _lib.tbo_energy_abs.argtypes = [i64, d, d, d, C.c_double, C.c_double, d, d, C.c_int]
        _lib.tbo_energy_abs.restype = C.c_double
        _lib.tbo_predictor.argtypes = [i64, d, d, d, d, d, d, d, C.c_double]
        _lib.tbo_update.argtypes = [i64, d, d, d, d, d, d, d, d, d, d, C.c_double, d]
        _lib.tbo_simulate.argtypes = [C.c_int, C.c_int, i64] + [d] * 13 + [C.c_double, d, C.c_double,
                                                                            C.c_double, C.POINTER(C.c_uint64),
                                                                            C.c_int]
        _lib.tbo_simulate.restype = C.c_int
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def domain(x, y, z):
    """Fixed P3BCA domain: (L[3], lo[3]) from initial positions with the 1e-4 margin."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    L = np.zeros(3)
    lo = np.zeros(3)
    lib().tbo_domain(len(x), _p(x), _p(y), _p(z), _p(L), _p(lo))
    return L, lo


def forces(x, y, z, nu: float = 1.0, cutoff: float = -1.0, L=None, lo=None, nthreads: int = 0,
           method: str = "auto"):
    """Stored forces (+grad E) and the triplet count at the given positions.

    cutoff <= 0 means no cutoff (NATA/AUTA).  With a cutoff, L/lo default to the domain of these
    positions.  method: "brute" (the reference's O(N^3) loop), "cells", or "auto".
    """
    x, y, z = _f64(x), _f64(y), _f64(z)
    n = len(x)
    if L is None or lo is None:
        L, lo = domain(x, y, z)
    L, lo = _f64(L), _f64(lo)
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    if cutoff > 0 and method in ("auto", "cells"):
        c = lib().tbo_forces_cells(n, _p(x), _p(y), _p(z), nu, cutoff, _p(L), _p(lo), _p(fx), _p(fy), _p(fz),
                                   nthreads)
    else:
        c = lib().tbo_forces_bruteforce(n, _p(x), _p(y), _p(z), nu, cutoff, _p(L), _p(fx), _p(fy), _p(fz),
                                        nthreads)
    if c == 2**64 - 1:
        raise MemoryError("oracle allocation failed")
    return fx, fy, fz, int(c)


def forces_selected(x, y, z, idx, nu: float = 1.0, nthreads: int = 0):
    """Stored forces (+grad E, no cutoff) on the particles idx only, from every triplet containing
    each (O(n^2) per particle, the reference's per-triplet arithmetic).  Returns (fx, fy, fz) of
    len(idx)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    sel = np.ascontiguousarray(idx, dtype=np.int64)
    out = [np.zeros(len(sel)) for _ in range(3)]
    lib().tbo_forces_selected(len(x), _p(x), _p(y), _p(z), nu, sel.ctypes.data_as(C.POINTER(C.c_int64)), len(sel),
                              *[_p(o) for o in out], nthreads)
    return tuple(out)


def cell_dims(L, cutoff):
    L = _f64(L)
    dims = (C.c_int * 3)()
    w = np.zeros(3)
    lib().tbo_cell_dims(_p(L), cutoff, dims, _p(w))
    return tuple(dims), w


def cell_assign(x, y, z, cutoff, L, lo):
    x, y, z, L, lo = _f64(x), _f64(y), _f64(z), _f64(L), _f64(lo)
    cell = np.zeros(len(x), dtype=np.int32)
    dims = (C.c_int * 3)()
    lib().tbo_cell_assign(len(x), _p(x), _p(y), _p(z), cutoff, _p(L), _p(lo), dims,
                          cell.ctypes.data_as(C.POINTER(C.c_int32)))
    return cell, tuple(dims)


def energy(x, y, z, nu=1.0, cutoff=-1.0, L=None, lo=None, nthreads=0):
    x, y, z = _f64(x), _f64(y), _f64(z)
    if L is None or lo is None:
        L, lo = domain(x, y, z)
    L, lo = _f64(L), _f64(lo)
    return float(lib().tbo_energy(len(x), _p(x), _p(y), _p(z), nu, cutoff, _p(L), _p(lo), nthreads))


def energy_abs(x, y, z, nu=1.0, cutoff=-1.0, L=None, lo=None, nthreads=0):
    """Sum over the same triplet set of |nu| (1 + 3 |cos cos cos|) / (r1 r2 r3)^3, the magnitude of
    both parts of each term: the scale of the energy's rounding error (the terms have both signs,
    and one term can cancel inside, so the energy itself can be much smaller)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    if L is None or lo is None:
        L, lo = domain(x, y, z)
    L, lo = _f64(L), _f64(lo)
    return float(lib().tbo_energy_abs(len(x), _p(x), _p(y), _p(z), nu, cutoff, _p(L), _p(lo), nthreads))


FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "fx", "fy", "fz")


def simulate(algorithm: str, iterations: int, state: dict, dt: float, g, cutoff: float = 0.0, nu: float = 1.0,
             nthreads: int = 0):
    """Run the reference step loop on a copy of `state` (dict of float64 arrays incl. 'm').

    Returns (new_state, counts[iterations])."""
    st = {k: _f64(state[k]).copy() for k in FIELDS if k in state}
    n = len(st["x"])
    for k in FIELDS:
        st.setdefault(k, np.zeros(n))
    m = _f64(state["m"])
    g = _f64(g)
    counts = np.zeros(max(iterations, 1), dtype=np.uint64)
    rc = lib().tbo_simulate(ALGORITHMS[algorithm.lower()], iterations, n, *[_p(st[k]) for k in FIELDS], _p(m), dt,
                            _p(g), cutoff, nu, counts.ctypes.data_as(C.POINTER(C.c_uint64)), nthreads)
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    st["m"] = m.copy()
    return st, counts[:iterations]


# ---------------------------------------------------------------------------------------------
# The reference itself (oracle/_ref, built by oracle/Makefile.ref)


def reference_available() -> bool:
    return (REF_DIR / "ref_dump").exists() and (REF_DIR / "particlegenerator").exists()


def reference_generate(path: str, generator: str, n: int, box, mass: float = 1.0, seed0: int = 926762934,
                       seed1: int = 89347587, extra: list | None = None) -> None:
    """Write an input CSV with the reference's particlegenerator (6 significant digits)."""
    cmd = [str(REF_DIR / "particlegenerator"), "--generator", generator, "--numparticles", str(n),
           "--blx", repr(float(box[0])), "--bly", repr(float(box[1])), "--blz", repr(float(box[2])),
           "--mass", repr(float(mass)), "--seed0", str(seed0), "--seed1", str(seed1),
           "--vx", "0", "--vy", "0", "--vz", "0", "--output", path] + (extra or [])
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)


def reference_dump(csv: str, algo: str, mode: str = "sim", iters: int = 1, dt: float = 0.001, g=(0.0, 0.0, 0.0),
                   cutoff: float = 0.0, nu: float = 1.0, timeout: float | None = None):
    """Run the reference's own classes on a CSV; returns (state dict in output order, counts, seconds)."""
    cmd = [str(REF_DIR / "ref_dump"), "--algo", algo, "--csv", csv, "--mode", mode, "--iters", str(iters),
           "--dt", repr(dt), "--g", *[repr(float(v)) for v in g], "--cutoff", repr(cutoff), "--nu", repr(nu)]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout,
                         env=dict(os.environ, OMP_NUM_THREADS="1")).stdout
    counts, rows, t = [], [], 0.0
    for line in out.splitlines():
        f = line.split()
        if f[0] == "step":
            counts.append(int(f[5]))
        elif f[0] == "particle":
            rows.append([float(v) for v in f[1:]])
        elif f[0] == "time_ns":
            t = int(f[1]) * 1e-9
    a = np.array(rows, dtype=np.float64).reshape(-1, 14)
    keys = ("id", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m", "fx", "fy", "fz")
    st = {k: a[:, i].copy() for i, k in enumerate(keys)}
    st["id"] = st["id"].astype(np.int32)
    return st, np.array(counts, dtype=np.uint64), t


def reference_layout(csv: str, algo: str, world_size: int, rank: int = 0, cutoff: float = 0.0,
                     decomposition: str = "naive", timeout: float = 60.0):
    """Run the reference's own set-up (Simulation::Init) for rank `rank` of `world_size` under the
    stub MPI's layout mode (oracle/refstub/ref_layout.cpp).  Returns (exit status, stderr text,
    the JSON it printed or None)."""
    import json
    cmd = [str(REF_DIR / "ref_layout"), "--algo", algo, "--csv", csv, "--cutoff", repr(float(cutoff)),
           "--decomp", decomposition]
    env = dict(os.environ, TBMD_STUB_WORLD_SIZE=str(world_size), TBMD_STUB_RANK=str(rank))
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)
    out = json.loads(r.stdout) if r.returncode == 0 and r.stdout.strip() else None
    return r.returncode, r.stderr.strip(), out


def reference_grid_tables() -> dict:
    """The reference's process-grid tables (Utility::getDecomposition over utility/decompositions.hpp)
    for P = 1..1030, as {"optimal": {P: grid}, "naive": {P: grid}} (an empty grid past the tables)."""
    import json
    r = subprocess.run([str(REF_DIR / "ref_layout"), "--tables"], capture_output=True, text=True, check=True)
    return json.loads(r.stdout)


def read_csv(path: str) -> dict:
    """Read a reference particle CSV (header row; ID, pX..pZ, vX..vZ, aX..aZ, m; extra columns ignored)."""
    a = np.loadtxt(path, delimiter=",", skiprows=1, ndmin=2)
    keys = ("id", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")
    st = {k: np.ascontiguousarray(a[:, i]) for i, k in enumerate(keys)}
    st["id"] = st["id"].astype(np.int32)
    return st
