"""CPU-side checks of the C ABI library: it loads, exports every symbol the
public header declares, and rejects unsupported classes before touching a
device (no compute calls here)."""

import ctypes
import importlib
import pathlib
import re

import numpy as np
import pytest

REPO = pathlib.Path(__file__).resolve().parent.parent
lib_mod = importlib.import_module("electron-integral-playground_b200._lib")


def declared_symbols():
    text = (REPO / "include" / "eip_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    ret = r"(?:int|void|size_t|float|double\s*\*|long long|void\s*\*|const char\s*\*|unsigned long long|eip_\w+\s*\*)"
    return sorted(set(re.findall(r"\b" + ret + r"\s*(\w+)\s*\(", text)))


def test_header_declares_reference_abi():
    syms = declared_symbols()
    for s in ("three_center", "two_center", "nuclear_attraction", "overlap"):
        assert s in syms


def test_library_exports_declared_symbols():
    if not lib_mod.LIB_PATH.exists():
        pytest.skip("library not built")
    L = ctypes.CDLL(str(lib_mod.LIB_PATH))
    for s in declared_symbols():
        assert hasattr(L, s), s


def test_unsupported_class_rejected_without_device():
    if not lib_mod.LIB_PATH.exists():
        pytest.skip("library not built")
    L = lib_mod.lib()
    z = np.zeros(4)
    zi = np.zeros(1, np.int32)
    out = np.zeros(1)
    dp, ip = lib_mod.dp, lib_mod.ip
    assert L.three_center(7, 7, 0, dp(z), dp(z), dp(z), dp(z), ip(zi), ip(zi), 1, dp(z), dp(z), ip(zi), 1,
                          dp(out), 1, 1, True, 0.0) == 1
    assert L.three_center(2, 1, 0, dp(z), dp(z), dp(z), dp(z), ip(zi), ip(zi), 1, dp(z), dp(z), ip(zi), 1,
                          dp(out), 1, 1, True, 0.0) == 1
    assert L.three_center(0, 0, 10, dp(z), dp(z), dp(z), dp(z), ip(zi), ip(zi), 1, dp(z), dp(z), ip(zi), 1,
                          dp(out), 1, 1, True, 0.0) == 1
    assert L.two_center(3, 10, dp(z), dp(z), ip(zi), 1, dp(z), dp(z), ip(zi), 1, dp(out), 1, True, 0.0) == 1
    assert L.nuclear_attraction(0, 7, dp(z), dp(z), dp(z), dp(z), ip(zi), ip(zi), 1, dp(z), 1, dp(out), 1, True,
                                0.0) == 1
    assert L.overlap(1, 0, dp(z), dp(z), dp(z), ip(zi), ip(zi), 1, dp(out), 1, True) == 1
    assert out[0] == 0.0


def test_empty_inputs_are_noops():
    if not lib_mod.LIB_PATH.exists():
        pytest.skip("library not built")
    L = lib_mod.lib()
    z = np.zeros(4)
    zi = np.zeros(1, np.int32)
    out = np.zeros(1)
    dp, ip = lib_mod.dp, lib_mod.ip
    assert L.three_center(0, 0, 0, dp(z), dp(z), dp(z), dp(z), ip(zi), ip(zi), 0, dp(z), dp(z), ip(zi), 1,
                          dp(out), 1, 1, True, 0.0) == 0
    assert L.overlap(0, 0, dp(z), dp(z), dp(z), ip(zi), ip(zi), 0, dp(out), 1, True) == 0


def test_committed_tuning_table_is_valid():
    """The autotuner's table for B200 names every fast class of the bench's
    batch (orbital s-d pairs, auxiliary s-g) with a compiled variant, and the
    library accepts each entry (the setters are host-side; no device)."""
    if not lib_mod.LIB_PATH.exists():
        pytest.skip("library not built")
    at = importlib.import_module("electron-integral-playground_b200.autotune")
    import json

    data = json.loads(at.DEFAULT_CACHE.read_text())
    classes = {f"{li},{lj},{lk}" for li in range(3) for lj in range(li, 3) for lk in range(5)}
    assert set(data["variants"]) == classes
    assert set(data["variants_fp32"]) == classes
    assert all(v in range(at.N_VARIANTS) for v in data["variants"].values())
    assert all(v in at.FP32_VARIANTS for v in data["variants_fp32"].values())
    L = lib_mod.lib()
    saved = {k: (L.eip_tune_get(*map(int, k.split(","))), L.eip_tune_get_fp32(*map(int, k.split(","))))
             for k in classes}
    try:
        at.load()
        for k in classes:
            li, lj, lk = map(int, k.split(","))
            assert L.eip_tune_get(li, lj, lk) == data["variants"][k]
            assert L.eip_tune_get_fp32(li, lj, lk) == data["variants_fp32"][k]
        assert L.eip_tune_set(0, 0, 0, at.N_VARIANTS) == 1  # out of range
    finally:
        for k, (v, v32) in saved.items():
            li, lj, lk = map(int, k.split(","))
            L.eip_tune_set(li, lj, lk, v)
            L.eip_tune_set_fp32(li, lj, lk, v32)


def _noalloc_check(L, li, lj, lk, n_pair, n_aux, spherical=True):
    f = L.eip_three_center_noalloc_check
    f.argtypes = [ctypes.c_int] * 5 + [ctypes.c_bool, ctypes.POINTER(ctypes.c_size_t)]
    f.restype = ctypes.c_int
    need = ctypes.c_size_t(123)
    rc = f(li, lj, lk, n_pair, n_aux, spherical, ctypes.byref(need))
    return rc, need.value


def test_noalloc_admission_check_on_host():
    """The allocation-free entry point's size check runs on the host alone: it
    accepts what fits its fixed working array and rejects the rest."""
    if not lib_mod.LIB_PATH.exists():
        pytest.skip("library not built")
    L = ctypes.CDLL(str(lib_mod.LIB_PATH))
    L.eip_noalloc_scratch_bytes.restype = ctypes.c_size_t
    limit = L.eip_noalloc_scratch_bytes()
    assert limit == 16 << 20
    rc, need = _noalloc_check(L, 1, 2, 3, 20, 30)
    assert rc == 0 and 0 < need <= limit
    # need grows with the primitive triplets: the class's spherical output
    # block per triplet dominates
    per = 8 * 3 * 5 * 7
    assert need >= 20 * 30 * per
    rc, need = _noalloc_check(L, 1, 2, 4, 2000, 3000)
    assert rc == 4 and need > limit
    rc, need = _noalloc_check(L, 0, 0, 0, 10, 70000)  # small, but beyond the auxiliary-primitive limit
    assert rc == 4
    assert _noalloc_check(L, 2, 1, 0, 1, 1)[0] == 1
    assert _noalloc_check(L, 0, 7, 0, 1, 1)[0] == 1
    assert _noalloc_check(L, 0, 0, 10, 1, 1)[0] == 1
    assert _noalloc_check(L, 0, 0, 0, 0, 5) == (0, 0)
