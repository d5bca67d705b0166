"""The C-ABI library on a host without a GPU: it loads, exports every entry point
the header declares, runs its host-only logic, and fails cleanly (status code,
not a crash) where a device is needed."""
from __future__ import annotations

import ctypes as C
import json
import math
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def header_functions() -> list[str]:
    text = (ROOT / "include" / "aperi_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(am_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(capi_lib):
    from aperi_mech_b200 import capi

    declared = header_functions()
    assert len(declared) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", str(capi.library_path())], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (am_[a-z0-9_]+)$", out, flags=re.M))
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    assert set(capi.EXPORTED) <= set(declared)


def test_complete_properties_host(capi_lib):
    from aperi_mech_b200.model import complete_properties

    g = json.loads((ROOT / "tests" / "golden" / "linear_elastic_properties.json").read_text())
    for a, b in g["valid_pairs"]:
        out = complete_properties(**{a: g["values"][a], b: g["values"][b]})
        for k, v in g["values"].items():
            assert abs(out[k] - v) < g["tol"]
    for bad in g["invalid"]:
        with pytest.raises(ValueError):
            complete_properties(**bad)


def test_status_strings(capi_lib):
    assert capi_lib.am_status_string(0) == b"ok"
    assert capi_lib.am_status_string(4) == b"non-positive Jacobian determinant"


def test_create_without_device_reports_error(capi_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    X = np.zeros((4, 3))
    h = C.c_void_p()
    rc = capi_lib.am_create(4, X.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
    assert rc != 0 and not h.value
    assert len(capi_lib.am_last_error(None)) > 0


def test_create_rejects_bad_input(capi_lib):
    h = C.c_void_p()
    assert capi_lib.am_create(0, None, C.byref(h)) == 1
    X = np.array([[0.0, math.nan, 0.0]])
    assert capi_lib.am_create(1, X.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h)) == 1


def test_noalloc_limit_mirrors_header():
    """The Python constant the no-alloc tests size against is the header's #define."""
    from aperi_mech_b200 import capi

    text = (ROOT / "include" / "aperi_b200.h").read_text()
    m = re.search(r"#define\s+AM_NOALLOC_MAX_TETS\s+(\d+)", text)
    assert m is not None
    assert int(m.group(1)) == capi.AM_NOALLOC_MAX_TETS
