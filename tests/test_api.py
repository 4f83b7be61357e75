"""C-ABI tests that need no GPU: symbols, defaults, setters, validation order.

Mirrors reference test/plfft_interface_test.cpp (defaults :278-299, setter
round trip :301-330, null/invalid rejection :468-643, status strings
:645-660).  Validation happens before any device call, so every rejection
path runs on CPU.
"""
import ctypes
import os
import re
import subprocess

import pytest

import plfft

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("plfft.h", "plfft_cuda.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(plfft_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = plfft.lib()
    missing = [s for s in sorted(declared_symbols()) if not hasattr(L, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", plfft.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (plfft_\w+)", out))
    assert declared_symbols() <= exported


def test_binding_covers_declared_symbols():
    assert declared_symbols() <= set(plfft.exported_symbols())


def test_config_defaults():
    c = plfft.Config.c2c(16, plfft.FORWARD)
    assert c.data_type == plfft.DataType.FP32
    assert c.io_alias == plfft.IoAlias.NO_ALIAS
    assert c.sme_mode == plfft.SmeMode.DISABLED
    assert c.howmany == 1 and c.istride == 1 and c.idist == 16 and c.ostride == 1 and c.odist == 16
    assert c.rigor == plfft.Rigor.MEASURE
    assert c.scale == 1.0


def test_config_setters_round_trip():
    c = plfft.Config.r2c(16)
    c.data_type = plfft.DataType.FP64
    c.io_alias = plfft.IoAlias.MAY_ALIAS
    c.sme_mode = plfft.SmeMode.ENABLED
    c.set_batch(3, 2, 32, 4, 64)
    c.rigor = plfft.Rigor.EXHAUSTIVE
    assert (c.data_type, c.io_alias, c.sme_mode, c.rigor) == (1, 1, 1, 3)
    assert (c.howmany, c.istride, c.idist, c.ostride, c.odist) == (3, 2, 32, 4, 64)


def _create_status(fn, *args):
    L = plfft.lib()
    h = ctypes.c_void_p(0x1234)
    st = getattr(L, fn)(ctypes.byref(h), *args)
    return st, h.value


def test_create_nulls_out_param_on_error():
    st, h = _create_status("plfft_config_create", 8, 0)
    assert st == plfft.Status.INVALID_TRANSFORM_KIND and h is None
    st, h = _create_status("plfft_config_create_r2r", 8, 11)
    assert st == plfft.Status.INVALID_TRANSFORM_KIND and h is None
    L = plfft.lib()
    assert L.plfft_config_create(None, 8, -1) == plfft.Status.NULL_ARGUMENT
    assert L.plfft_config_create_r2c(None, 8) == plfft.Status.NULL_ARGUMENT


def _plan_status(cfg):
    L = plfft.lib()
    h = ctypes.c_void_p(0x1234)
    st = L.plfft_plan_create_from_config(ctypes.byref(h), cfg.handle if cfg else None)
    return st, h.value


def test_plan_rejects_in_reference_order():
    L = plfft.lib()
    assert L.plfft_plan_create_from_config(None, None) == plfft.Status.NULL_ARGUMENT
    st, h = _plan_status(None)
    assert st == plfft.Status.NULL_ARGUMENT and h is None
    # size before batch
    c = plfft.Config.c2c(0)
    c.set_batch(0, 0, 0, 0, 0)
    assert _plan_status(c) == (plfft.Status.INVALID_SIZE, None)
    # batch
    for b in [(0, 1, 1, 1, 1), (2, 1, 0, 1, 1), (2, 0, 1, 1, 1), (1, 1, 0, 0, 0), (2, 1, 1, 1, 0)]:
        c = plfft.Config.c2c(8)
        c.set_batch(*b)
        assert _plan_status(c)[0] == plfft.Status.UNSUPPORTED_BATCH, b
    # howmany == 1 ignores distances
    c = plfft.Config.c2c(8)
    c.set_batch(1, 1, 0, 1, -5)
    c.io_alias = 7
    assert _plan_status(c)[0] == plfft.Status.INVALID_IO_ALIAS
    # alias before sme
    c = plfft.Config.c2c(8)
    c.io_alias = 2
    c.sme_mode = 5
    assert _plan_status(c)[0] == plfft.Status.INVALID_IO_ALIAS
    c.io_alias = 0
    assert _plan_status(c)[0] == plfft.Status.INVALID_SME_MODE
    # sme + r2r, sme + fixed point, sme not built
    c = plfft.Config.r2r(8, plfft.R2RKind.DCT_2)
    c.sme_mode = 1
    assert _plan_status(c)[0] == plfft.Status.SME_UNSUPPORTED_R2R
    c = plfft.Config.c2c(8)
    c.sme_mode = 1
    c.data_type = plfft.DataType.Q15
    assert _plan_status(c)[0] == plfft.Status.SME_UNSUPPORTED_FIXED_POINT
    c.data_type = plfft.DataType.FP32
    assert _plan_status(c)[0] == plfft.Status.SME_NOT_ENABLED
    # rigor before data type
    c = plfft.Config.c2c(8)
    c.rigor = 9
    c.data_type = 42
    assert _plan_status(c)[0] == plfft.Status.INVALID_PLANNER_RIGOR
    c.rigor = 0
    assert _plan_status(c)[0] == plfft.Status.INVALID_DATA_TYPE


def test_status_strings():
    assert plfft.status_to_string(0) == "success"
    assert plfft.status_to_string(1) == "null argument"
    assert plfft.status_to_string(14) == "invalid planning rigor level"
    assert plfft.status_to_string(999) == "unknown status"
    for s in range(15):
        assert plfft.status_to_string(s) != "unknown status"


def test_destroy_accepts_null():
    L = plfft.lib()
    L.plfft_config_destroy(None)
    L.plfft_plan_destroy(None)


@pytest.mark.gpu
def test_plan_snapshots_configuration():
    import numpy as np

    c = plfft.Config.c2c(4)
    p = plfft.Plan(c)
    c.data_type = plfft.DataType.FP64
    c.set_batch(2, 2, 1, 2, 1)
    c.destroy()
    x = np.array([1, 2, 3, 4], np.complex64)
    y = np.zeros(4, np.complex64)
    p.execute(x.ctypes.data, y.ctypes.data)
    assert y[0] == 10.0


@pytest.mark.gpu
def test_interleaved_batch_layout():
    import numpy as np

    c = plfft.Config.c2c(4)
    c.set_batch(2, 2, 1, 2, 1)
    p = plfft.Plan(c)
    x = np.array([1, 10, 2, 20, 3, 30, 4, 40], np.complex64)
    y = np.zeros(8, np.complex64)
    p.execute(x.ctypes.data, y.ctypes.data)
    assert y[0] == 10.0 and y[1] == 100.0
