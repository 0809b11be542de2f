"""The C-ABI library loads and exports every entry point include/*.h
declares; argument validation that needs no GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import zeus_b200 as zb

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(zeus_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "zeus_bfgs_device" in names and "zeus_optimize" in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(zb.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_functions()) <= set(zb.SIGNATURES)


def test_version_and_support_table():
    assert b"sm_100a" in zb.lib().zeus_version()
    assert zb.supported(zb.OBJ_ROSENBROCK, 2, "exact", "dual")
    assert zb.supported(zb.OBJ_ROSENBROCK, 2, "fast", "adjoint")
    assert not zb.supported(zb.OBJ_ROSENBROCK, 3, "exact", "dual")
    assert not zb.supported(zb.OBJ_ROSENBROCK, 2, "exact", "adjoint")


def test_invalid_arguments_fail_loudly_without_gpu():
    L = zb.lib()
    cfg = zb.make_config(100, 10, 1e-8, "fast", "adjoint")
    prob = zb.Problem(zb.OBJ_ROSENBROCK, 3, None, None, 0, 0)  # dim 3 not built
    rc = L.zeus_bfgs_device(C.byref(prob), C.byref(cfg), None, 10, C.byref(zb.RunOutputs()),
                            None, None, 0, None)
    assert rc == zb.E_UNSUPPORTED and "not built" in zb.last_error()
    prob = zb.Problem(zb.OBJ_GAUSSIAN, 8, None, None, 0, 0)  # no matrix
    rc = L.zeus_bfgs_device(C.byref(prob), C.byref(cfg), None, 10, C.byref(zb.RunOutputs()),
                            None, None, 0, None)
    assert rc == zb.E_INVALID
    bad = zb.make_config(-1, 10, 1e-8)
    prob = zb.Problem(zb.OBJ_ROSENBROCK, 2, None, None, 0, 0)
    assert L.zeus_bfgs_device(C.byref(prob), C.byref(bad), None, 10,
                              C.byref(zb.RunOutputs()), None, None, 0, None) == zb.E_INVALID
    exact_adj = zb.make_config(10, 10, 1e-8, "exact", "adjoint")
    assert L.zeus_bfgs_device(C.byref(prob), C.byref(exact_adj), None, 10,
                              C.byref(zb.RunOutputs()), None, None, 0, None) == zb.E_INVALID


def test_nll_sensitivity_rejects_bad_input_without_gpu():
    L = zb.lib()
    ros = zb.Problem(zb.OBJ_ROSENBROCK, 2, None, None, 0, 0)
    assert L.zeus_nll_sensitivity_device(C.byref(ros), 1, 4, None, None, None, None,
                                         None) == zb.E_INVALID
    assert "Poisson NLL" in zb.last_error()
    data = (C.c_double * 4)()
    idata = (C.c_int32 * 4)()
    nll = zb.Problem(zb.OBJ_POISSON_NLL, 4, C.cast(data, C.c_void_p),
                     C.cast(idata, C.c_void_p), 4, 0)
    # runs_per_instance must be positive; buffers are required for n > 0
    assert L.zeus_nll_sensitivity_device(C.byref(nll), 1, 0, None, None, None, None,
                                         None) == zb.E_INVALID
    assert L.zeus_nll_sensitivity_device(C.byref(nll), 1, 4, None, None, None, None,
                                         None) == zb.E_INVALID
    # no toys: nothing to do, no device call
    assert L.zeus_nll_sensitivity_device(C.byref(nll), 0, 4, None, None, None, None,
                                         None) == zb.OK


def test_workspace_sizes():
    L = zb.lib()
    prob = zb.Problem(zb.OBJ_ROSENBROCK, 2, None, None, 0, 0)
    fast = zb.make_config(100, 10, 1e-8, "fast", "adjoint")
    assert L.zeus_bfgs_workspace_size(C.byref(prob), C.byref(fast), 1000) == 0
    # the CTA layout (dim > 32): its blocks' run queue
    prob64 = zb.Problem(zb.OBJ_ROSENBROCK, 64, None, None, 0, 0)
    assert L.zeus_bfgs_workspace_size(C.byref(prob64), C.byref(fast), 1000) == 256
    assert L.zeus_pso_workspace_size(1000, 2) >= 2 * 1000 * 2 * 8
    assert L.zeus_pso_workspace_size(0, 2) == 0


def test_zero_runs_returns_default_result():
    """zeus.cuh:58-60: N == 0 returns Result{} (status -1, fval 37)."""
    r = zb.Zeus(zb.Rosenbrock(2), -5, 5, 0, 100, 10, 10, "rosenbrock", 1e-8, 42, 0)
    assert r.status == -1 and r.fval == 37.0 and r.idx == -1


def test_missing_library_is_an_error(monkeypatch, tmp_path):
    monkeypatch.setattr(zb, "LIB_PATH", tmp_path / "nope.so")
    monkeypatch.setattr(zb, "_lib", None)
    with pytest.raises(RuntimeError, match="missing"):
        zb.lib()
