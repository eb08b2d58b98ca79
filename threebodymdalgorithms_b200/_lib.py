"""ctypes binding of libtbmd.so (include/tbmd.h).  The product path: every call goes to the CUDA
library; there is no CPU fallback.  Loading fails loudly if the library is missing."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

# TBMD_LIBRARY selects another build of the library, e.g. the bounds-checked libtbmd_checked.so
LIB_PATH = Path(os.environ.get("TBMD_LIBRARY") or Path(__file__).resolve().parent / "libtbmd.so")

NATA, P3BCA, AUTA = 0, 1, 2
FP64, MIXED = 0, 1
ALGORITHMS = {"nata": NATA, "p3bca": P3BCA, "auta": AUTA}
PRECISIONS = {"fp64": FP64, "mixed": MIXED}

STATUS = {0: "TBMD_OK", 1: "TBMD_INVALID_ARG", 2: "TBMD_BAD_INPUT", 3: "TBMD_NOT_READY", 4: "TBMD_CAPACITY_RETRY",
          5: "TBMD_CUDA_ERROR", 6: "TBMD_TIMEOUT", 7: "TBMD_NO_DEVICE", 8: "TBMD_TOO_LARGE", 9: "TBMD_RANK_LAYOUT"}
NOALLOC_MAX_N = 4096

# every symbol declared in include/tbmd.h
EXPORTS = ("tbmd_config_init", "tbmd_create", "tbmd_destroy", "tbmd_last_error", "tbmd_status_string",
           "tbmd_abi_version", "tbmd_set_particles", "tbmd_get_particles", "tbmd_num_particles", "tbmd_step",
           "tbmd_forces", "tbmd_adjoint", "tbmd_forces_device", "tbmd_adjoint_device", "tbmd_set_domain",
           "tbmd_cells", "tbmd_batch_forces", "tbmd_batch_adjoint", "tbmd_autotune", "tbmd_tuning", "tbmd_sync",
           "tbmd_kernel_launches", "tbmd_set_profiling", "tbmd_phase_times", "tbmd_nata_forces_noalloc",
           "tbmd_bounds_report",
           "tbmd_generator_init", "tbmd_generate_particles", "tbmd_rank_layout_of", "tbmd_step_host")
PHASES = ("predictor", "cells", "neighbors", "triplets", "update")


class TbmdError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Config(C.Structure):
    _fields_ = [("algorithm", C.c_int32), ("precision", C.c_int32), ("cutoff", C.c_double), ("dt", C.c_double),
                ("g", C.c_double * 3), ("nu", C.c_double), ("device", C.c_int32), ("use_graph", C.c_int32),
                ("stream", C.c_void_p), ("reserved", C.c_int32 * 8)]


class Generator(C.Structure):
    """tbmd_generator: the reference particlegenerator's parameters."""
    _fields_ = [("kind", C.c_int32), ("n", C.c_int64), ("box", C.c_double * 3), ("corner", C.c_double * 3),
                ("velocity", C.c_double * 3), ("mass", C.c_double), ("seed0", C.c_uint32), ("seed1", C.c_uint32),
                ("n_clusters", C.c_int32), ("mean", C.c_double), ("stddev", C.c_double), ("csv_digits", C.c_int32),
                ("reserved", C.c_int32 * 7)]


GENERATORS = {"uniform": 0, "clusteredgauss": 1}


class RankLayout(C.Structure):
    """tbmd_rank_layout: the reference's layout of a run on P MPI ranks."""
    _fields_ = [("world_size", C.c_int32), ("num_dims", C.c_int32), ("dims", C.c_int32 * 3),
                ("cutoff_boxes", C.c_int32 * 3), ("shift_steps", C.c_int32), ("reserved", C.c_int32),
                ("cell_size", C.c_double * 3), ("particles_per_rank", C.c_int64), ("dummies", C.c_int64)]

_lib = None


def bounds_report():
    """Index checks of a bounds-checked build (libtbmd_checked.so): (checked, violations, site, index,
    size) of the first index found outside its array since the last report; checked is False for the
    normal build, which records nothing.  Waits for the device."""
    lib = load()
    v, site, idx, size = C.c_int64(), C.c_int32(), C.c_int64(), C.c_int64()
    checked = lib.tbmd_bounds_report(C.byref(v), C.byref(site), C.byref(idx), C.byref(size))
    return bool(checked), v.value, site.value, idx.value, size.value


def load():
    """Load libtbmd.so and declare the C signatures (raises if the library was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m threebodymdalgorithms_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    d, vp, i32, i64 = C.POINTER(C.c_double), C.c_void_p, C.c_int32, C.c_int64
    pi32, pu64, pi64 = C.POINTER(C.c_int32), C.POINTER(C.c_uint64), C.POINTER(C.c_int64)
    sig = {
        "tbmd_config_init": (None, [C.POINTER(Config)]),
        "tbmd_create": (C.c_int, [C.POINTER(Config), C.POINTER(vp)]),
        "tbmd_destroy": (None, [vp]),
        "tbmd_last_error": (C.c_char_p, [vp]),
        "tbmd_status_string": (C.c_char_p, [C.c_int]),
        "tbmd_abi_version": (i32, []),
        "tbmd_set_particles": (C.c_int, [vp, i64, pi32] + [d] * 10),
        "tbmd_get_particles": (C.c_int, [vp, pi32] + [d] * 13),
        "tbmd_num_particles": (i64, [vp]),
        "tbmd_step": (C.c_int, [vp, i32, pu64]),
        "tbmd_forces": (C.c_int, [vp, d, d, d, d, pu64]),
        "tbmd_adjoint": (C.c_int, [vp, d, d, d, C.c_double, d, d, d, d]),
        "tbmd_forces_device": (C.c_int, [vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "tbmd_adjoint_device": (C.c_int, [vp, i64] + [vp] * 14),
        "tbmd_set_domain": (C.c_int, [vp, d, d]),
        "tbmd_cells": (C.c_int, [vp, pi32, pi32, d, d]),
        "tbmd_batch_forces": (C.c_int, [vp, i32, pi64, d, d, d, d, d, d, d, d, d, pu64]),
        "tbmd_batch_adjoint": (C.c_int, [vp, i32, pi64, d, d, d, d, d, d, d, d, d, d, d, d, d]),
        "tbmd_autotune": (C.c_int, [vp, C.c_char_p]),
        "tbmd_tuning": (C.c_char_p, [vp]),
        "tbmd_sync": (C.c_int, [vp]),
        "tbmd_kernel_launches": (C.c_uint64, [vp]),
        "tbmd_set_profiling": (C.c_int, [vp, i32]),
        "tbmd_phase_times": (i32, [vp, d, pu64, pu64, i32]),
        "tbmd_nata_forces_noalloc": (C.c_int, [i64, vp, vp, vp, C.c_double, i32, vp, vp, vp, vp]),
        "tbmd_generator_init": (None, [C.POINTER(Generator)]),
        "tbmd_generate_particles": (C.c_int, [vp, C.POINTER(Generator)]),
        "tbmd_rank_layout_of": (C.c_int, [i32, i32, i32, C.c_double, d, i64, C.POINTER(RankLayout), C.c_char_p,
                                          i32]),
        "tbmd_step_host": (C.c_int, [vp, i64, pi32] + [d] * 10 + [i32, pu64, pi32] + [d] * 13),
        "tbmd_bounds_report": (i32, [pi64, pi32, pi64, pi64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, "float64 C-contiguous array expected"
    return a.ctypes.data_as(C.POINTER(C.c_double))


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One tbmd_ctx: the GPU-resident Simulation (one device, one stream)."""

    def __init__(self, algorithm="auta", precision="fp64", cutoff=0.0, dt=0.0, g=(0.0, 0.0, 0.0), nu=1.0, device=0,
                 use_graph=True, stream=None):
        lib = load()
        cfg = Config()
        lib.tbmd_config_init(C.byref(cfg))
        cfg.algorithm = ALGORITHMS[algorithm.lower()] if isinstance(algorithm, str) else int(algorithm)
        cfg.precision = PRECISIONS[precision.lower()] if isinstance(precision, str) else int(precision)
        cfg.cutoff = float(cutoff)
        cfg.dt = float(dt)
        for k in range(3):
            cfg.g[k] = float(g[k])
        cfg.nu = float(nu)
        cfg.device = int(device)
        cfg.use_graph = 1 if use_graph else 0
        cfg.stream = stream
        self.cfg = cfg
        h = C.c_void_p()
        st = lib.tbmd_create(C.byref(cfg), C.byref(h))
        if st != 0:
            raise TbmdError(st, "tbmd_create failed")
        self._h = h
        self._lib = lib
        self.n = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.tbmd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise TbmdError(st, self._lib.tbmd_last_error(self._h).decode())

    @property
    def handle(self):
        return self._h

    def set_particles(self, x, y, z, vx=None, vy=None, vz=None, ax=None, ay=None, az=None, m=None, ids=None):
        x, y, z = f64(x), f64(y), f64(z)
        n = len(x)
        zero = np.zeros(n)
        arrs = [x, y, z] + [f64(a) if a is not None else zero for a in (vx, vy, vz, ax, ay, az)]
        arrs.append(f64(m) if m is not None else np.ones(n))
        idp = None
        if ids is not None:
            ids = np.ascontiguousarray(ids, dtype=np.int32)
            idp = ids.ctypes.data_as(C.POINTER(C.c_int32))
        self._check(self._lib.tbmd_set_particles(self._h, n, idp, *[dptr(a) for a in arrs]))
        self.n = n

    def generate(self, kind="uniform", n=0, box=(10.0, 10.0, 10.0), corner=(0.0, 0.0, 0.0), velocity=(0.0, 0.0, 0.0),
                 mass=1.0, seed0=926762934, seed1=89347587, n_clusters=1, mean=0.0, stddev=1.0, csv_digits=6):
        """Generate the reference particlegenerator's particles on the device and load them
        (tbmd_generate_particles).  Returns the number of particles."""
        g = Generator()
        self._lib.tbmd_generator_init(C.byref(g))
        g.kind = GENERATORS[kind] if isinstance(kind, str) else int(kind)
        g.n = int(n)
        for k in range(3):
            g.box[k], g.corner[k], g.velocity[k] = float(box[k]), float(corner[k]), float(velocity[k])
        g.mass, g.seed0, g.seed1 = float(mass), int(seed0) & 0xFFFFFFFF, int(seed1) & 0xFFFFFFFF
        g.n_clusters, g.mean, g.stddev, g.csv_digits = int(n_clusters), float(mean), float(stddev), int(csv_digits)
        self._check(self._lib.tbmd_generate_particles(self._h, C.byref(g)))
        self.n = int(self._lib.tbmd_num_particles(self._h))
        return self.n

    def set_state(self, st: dict):
        self.set_particles(st["x"], st["y"], st["z"], st.get("vx"), st.get("vy"), st.get("vz"), st.get("ax"),
                           st.get("ay"), st.get("az"), st.get("m"), st.get("id"))

    def get_state(self) -> dict:
        n = self.n
        keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m", "fx", "fy", "fz")
        out = {k: np.zeros(n) for k in keys}
        ids = np.zeros(n, dtype=np.int32)
        self._check(self._lib.tbmd_get_particles(self._h, ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 *[dptr(out[k]) for k in keys]))
        out["id"] = ids
        return out

    def step(self, iterations: int = 1) -> np.ndarray:
        counts = np.zeros(max(iterations, 1), dtype=np.uint64)
        self._check(self._lib.tbmd_step(self._h, int(iterations), counts.ctypes.data_as(C.POINTER(C.c_uint64))))
        return counts[:iterations]

    def step_host(self, st: dict, iterations: int = 1, out: dict | None = None):
        """Load the particles of `st`, step, and read the state back, in one call (tbmd_step_host):
        the same results as set_state + step + get_state, with the copies overlapping the step.
        `out` may give preallocated float64 arrays (any subset of x..fz, and id) to write into.
        Returns (state dict, per-step triplet counts)."""
        n = len(st["x"])
        ins = [f64(st[k]) if st.get(k) is not None else (np.ones(n) if k == "m" else np.zeros(n))
               for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")]
        ids_in = None if st.get("id") is None else np.ascontiguousarray(st["id"], dtype=np.int32)
        keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m", "fx", "fy", "fz")
        res = dict(out) if out is not None else {k: np.zeros(n) for k in keys}
        if "id" not in res:
            res["id"] = np.zeros(n, dtype=np.int32)
        counts = np.zeros(max(iterations, 1), dtype=np.uint64)
        ip = C.POINTER(C.c_int32)
        self._check(self._lib.tbmd_step_host(
            self._h, n, None if ids_in is None else ids_in.ctypes.data_as(ip), *[dptr(a) for a in ins],
            int(iterations), counts.ctypes.data_as(C.POINTER(C.c_uint64)), res["id"].ctypes.data_as(ip),
            *[dptr(res.get(k)) for k in keys]))
        self.n = n
        return res, counts[:iterations]

    def forces(self):
        n = self.n
        fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
        e = C.c_double()
        c = C.c_uint64()
        self._check(self._lib.tbmd_forces(self._h, dptr(fx), dptr(fy), dptr(fz), C.byref(e), C.byref(c)))
        return fx, fy, fz, e.value, c.value

    def adjoint(self, gfx, gfy, gfz, g_energy=0.0):
        n = self.n
        gfx, gfy, gfz = f64(gfx), f64(gfy), f64(gfz)
        gx, gy, gz = np.zeros(n), np.zeros(n), np.zeros(n)
        gnu = C.c_double()
        self._check(self._lib.tbmd_adjoint(self._h, dptr(gfx), dptr(gfy), dptr(gfz), float(g_energy), dptr(gx),
                                           dptr(gy), dptr(gz), C.byref(gnu)))
        return gx, gy, gz, gnu.value

    def set_domain(self, L, lo):
        L, lo = f64(L), f64(lo)
        self._check(self._lib.tbmd_set_domain(self._h, dptr(L), dptr(lo)))

    def cells(self, with_particles=True):
        dims = (C.c_int32 * 3)()
        L, lo = np.zeros(3), np.zeros(3)
        cell = np.zeros(self.n, dtype=np.int32) if with_particles else None
        cp = cell.ctypes.data_as(C.POINTER(C.c_int32)) if cell is not None else None
        self._check(self._lib.tbmd_cells(self._h, cp, dims, dptr(L), dptr(lo)))
        return cell, tuple(dims), L, lo

    def batch_forces(self, offsets, x, y, z, box=None, lo=None):
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        nsys = len(offsets) - 1
        x, y, z = f64(x), f64(y), f64(z)
        n = len(x)
        fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
        e = np.zeros(nsys)
        cnt = np.zeros(nsys, dtype=np.uint64)
        box = f64(box) if box is not None else None
        lo = f64(lo) if lo is not None else None
        self._check(self._lib.tbmd_batch_forces(self._h, nsys, offsets.ctypes.data_as(C.POINTER(C.c_int64)),
                                                dptr(box), dptr(lo), dptr(x), dptr(y), dptr(z), dptr(fx), dptr(fy),
                                                dptr(fz), dptr(e), cnt.ctypes.data_as(C.POINTER(C.c_uint64))))
        return fx, fy, fz, e, cnt

    def batch_adjoint(self, offsets, x, y, z, gfx, gfy, gfz, g_energy, box=None, lo=None):
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        nsys = len(offsets) - 1
        x, y, z, gfx, gfy, gfz = (f64(a) for a in (x, y, z, gfx, gfy, gfz))
        ge = f64(g_energy)
        n = len(x)
        gx, gy, gz = np.zeros(n), np.zeros(n), np.zeros(n)
        gnu = np.zeros(nsys)
        box = f64(box) if box is not None else None
        lo = f64(lo) if lo is not None else None
        self._check(self._lib.tbmd_batch_adjoint(self._h, nsys, offsets.ctypes.data_as(C.POINTER(C.c_int64)),
                                                 dptr(box), dptr(lo), dptr(x), dptr(y), dptr(z), dptr(gfx), dptr(gfy),
                                                 dptr(gfz), dptr(ge), dptr(gx), dptr(gy), dptr(gz), dptr(gnu)))
        return gx, gy, gz, gnu

    def forces_device(self, n, x_ptr, y_ptr, z_ptr, fx_ptr, fy_ptr, fz_ptr, e_ptr=None, c_ptr=None, stream=None):
        self._check(self._lib.tbmd_forces_device(self._h, n, x_ptr, y_ptr, z_ptr, fx_ptr, fy_ptr, fz_ptr, e_ptr, c_ptr,
                                                 stream))

    def adjoint_device(self, n, ptrs, stream=None):
        self._check(self._lib.tbmd_adjoint_device(self._h, n, *ptrs, stream))

    def autotune(self, cache_path=None):
        self._check(self._lib.tbmd_autotune(self._h, cache_path.encode() if cache_path else None))
        return self.tuning()

    def tuning(self) -> str:
        return self._lib.tbmd_tuning(self._h).decode()

    def sync(self):
        self._check(self._lib.tbmd_sync(self._h))

    def kernel_launches(self) -> int:
        return int(self._lib.tbmd_kernel_launches(self._h))

    def set_profiling(self, on: bool):
        self._check(self._lib.tbmd_set_profiling(self._h, 1 if on else 0))

    def phase_times(self) -> dict:
        k = len(PHASES)
        ms = np.zeros(k)
        calls = np.zeros(k, dtype=np.uint64)
        launches = np.zeros(k, dtype=np.uint64)
        m = self._lib.tbmd_phase_times(self._h, dptr(ms), calls.ctypes.data_as(C.POINTER(C.c_uint64)),
                                       launches.ctypes.data_as(C.POINTER(C.c_uint64)), k)
        return {PHASES[i]: {"ms": float(ms[i]), "calls": int(calls[i]), "launches": int(launches[i])}
                for i in range(m)}


def rank_layout(algorithm: str, world_size: int, n: int, cutoff: float = 0.0, L=None, decomposition: str = "naive"):
    """Layout of the reference's run of `algorithm` on `world_size` MPI ranks (host only, no GPU):
    process grid, P3BCA cutoff boxes and shift steps, NATA / AUTA dummy padding, as a dict.  Raises
    TbmdError(TBMD_RANK_LAYOUT) with the reference's stderr message where that run would stop
    (tbmd_rank_layout_of, include/tbmd.h)."""
    if decomposition not in ("naive", "optimal"):
        raise ValueError("decomposition must be 'naive' or 'optimal'")
    lib = load()
    out = RankLayout()
    msg = C.create_string_buffer(256)
    Lv = None if L is None else f64(L)
    st = lib.tbmd_rank_layout_of(ALGORITHMS[algorithm.lower()], int(world_size), int(decomposition == "optimal"),
                                 float(cutoff), dptr(Lv), int(n), C.byref(out), msg, len(msg))
    if st != 0:
        raise TbmdError(st, msg.value.decode() or lib.tbmd_status_string(st).decode())
    return {"world_size": out.world_size, "num_dims": out.num_dims, "dims": list(out.dims),
            "cutoff_boxes": list(out.cutoff_boxes), "shift_steps": out.shift_steps,
            "cell_size": list(out.cell_size), "particles_per_rank": out.particles_per_rank,
            "dummies": out.dummies}
