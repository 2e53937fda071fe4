"""The C-ABI library loads and exports every entry point ``include/dgb200.h`` declares.

No compute calls (no GPU needed): only symbol lookup and the error channel.
"""

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "dgb200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(dgb_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_symbols()
    for required in ("dgb_plan_create", "dgb_rhs", "dgb_stable_dt", "dgb_ssprk3_step", "dgb_positivity",
                     "dgb_troubled"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from jax_fluid_sim_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(str(lib_path))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_invalid_arguments_report_errors_without_a_gpu():
    from jax_fluid_sim_b200 import _native as N
    L = N.lib()
    prm = N.Params()
    prm.degree = 4          # the reference raises ValueError for P4 (elements.py:670-672)
    prm.nvars, prm.num_blocks = 5, 1
    handle = ctypes.c_void_p()
    rc = L.dgb_plan_create(ctypes.byref(prm), ctypes.byref(handle))
    assert rc == -1
    assert b"P1, P2, and P3" in L.dgb_last_error()
    with pytest.raises(ValueError):
        N.check(rc)
