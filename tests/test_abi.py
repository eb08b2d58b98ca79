"""The C ABI library: it is built, loads, exports every entry point include/tbmd.h declares, and
fails loudly (TBMD_NO_DEVICE) instead of falling back when no sm_100 GPU is present."""
import ctypes as C
import re
from pathlib import Path

import pytest

from threebodymdalgorithms_b200 import _lib

INCLUDE = Path(__file__).resolve().parents[1] / "include"
HEADER = INCLUDE / "tbmd.h"


def declared_functions(header=HEADER):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tbmd_[a-z_0-9]+)\s*\(", text)))


def all_declared():
    names = set()
    for h in INCLUDE.glob("*.h"):
        names.update(declared_functions(h))
    return sorted(names)


def test_header_declarations_match_binding():
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(_lib.LIB_PATH))
    names = all_declared()
    assert "tbmd_probe_fma_tflops" in names
    for name in names:
        assert hasattr(lib, name), name


def test_abi_version_and_status_strings():
    lib = _lib.load()
    assert lib.tbmd_abi_version() == 1
    assert lib.tbmd_status_string(0) == b"ok"
    assert lib.tbmd_status_string(7) == b"no sm_100 CUDA device"


def test_config_defaults_match_reference():
    lib = _lib.load()
    cfg = _lib.Config()
    lib.tbmd_config_init(C.byref(cfg))
    # the reference's zero-initialised CLI values, AxilrodTeller(1.0)
    assert (cfg.cutoff, cfg.dt, tuple(cfg.g), cfg.nu) == (0.0, 0.0, (0.0, 0.0, 0.0), 1.0)


def test_create_rejects_bad_config():
    lib = _lib.load()
    cfg = _lib.Config()
    lib.tbmd_config_init(C.byref(cfg))
    cfg.algorithm = 5
    h = C.c_void_p()
    assert lib.tbmd_create(C.byref(cfg), C.byref(h)) == 1
    lib.tbmd_config_init(C.byref(cfg))
    cfg.dt = float("nan")
    assert lib.tbmd_create(C.byref(cfg), C.byref(h)) == 1


def test_no_device_is_a_loud_error():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_lib.TbmdError) as e:
        _lib.Context("auta")
    assert e.value.status == 7


CHECKED = Path(_lib.__file__).resolve().parent / "libtbmd_checked.so"


def test_bounds_report_of_the_normal_build_records_nothing():
    """The normal build has no index checks: tbmd_bounds_report returns 0 (no device needed to ask)."""
    lib = _lib.load()
    v, site = C.c_int64(), C.c_int32()
    if _lib.LIB_PATH.name == "libtbmd.so":
        assert lib.tbmd_bounds_report(C.byref(v), C.byref(site), None, None) == 0


@pytest.mark.skipif(not CHECKED.exists(), reason="bounds-checked build not made (build --bounds-check)")
def test_checked_build_exports_the_same_symbols():
    lib = C.CDLL(str(CHECKED))
    for name in all_declared():
        assert hasattr(lib, name), name
    v = C.c_int64()
    assert lib.tbmd_bounds_report(C.byref(v), None, None, None) == 1
