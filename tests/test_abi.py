"""The C ABI library: it loads, exports every entry point include/bmc_b200.h declares, and rejects bad
arguments with a status and a message before touching the GPU. CPU only (no compute call)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from bmc_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "bmc_b200.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(bmc_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_entry_points():
    names = declared()
    assert {"bmc_simulate", "bmc_simulate_jvp", "bmc_lm_fit", "bmc_normal_blocks", "bmc_last_error",
            "bmc_version", "bmc_abi_version", "bmc_release", "bmc_simulate_trajectory"} <= set(names)


def test_library_exports_every_declared_symbol():
    L = C.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert set(_lib.EXPORTS) <= set(declared())


def test_abi_version_matches_the_header():
    v = int(re.search(r"#define BMC_ABI_VERSION (\d+)", HEADER.read_text()).group(1))
    assert _lib.lib().bmc_abi_version() == v
    assert b"sm_100a" in _lib.lib().bmc_version()


def test_bad_arguments_return_a_status_and_a_message():
    L = _lib.lib()
    st = L.bmc_simulate(None, None, None, None, None, None, None)
    assert st == 1
    with pytest.raises(RuntimeError, match="null problem"):
        _lib.check(st)
    pr = _lib.Problem(4, 3, 2, 9, 4, 1, 0, 0)          # nine CEST pools: above the compiled maximum
    ev = _lib.Events()
    dummy = C.c_void_p(16)
    st = L.bmc_simulate(pr, dummy, ev, dummy, None, dummy, None)
    assert st == 3
    with pytest.raises(RuntimeError, match="n_cest 9"):
        _lib.check(st)
    pr = _lib.Problem(4, 3, 2, 1, 99, 1, 0, 0)         # mz_loc outside the state
    with pytest.raises(RuntimeError, match="mz_loc 99"):
        _lib.check(L.bmc_simulate(pr, dummy, ev, dummy, None, dummy, None))
    pr = _lib.Problem(0, 3, 2, 1, 4, 1, 0, 0)
    with pytest.raises(RuntimeError, match="sizes must be positive"):
        _lib.check(L.bmc_simulate(pr, dummy, ev, dummy, None, dummy, None))


def test_fit_spec_is_validated():
    L = _lib.lib()
    pr = _lib.Problem(4, 3, 2, 1, 4, 1, 0, 0)
    dummy = C.c_void_p(16)
    ev = _lib.Events(16, 16, 16, 16, 16, 16)
    spec = _lib.FitSpecC()
    spec.n_params = 0
    with pytest.raises(RuntimeError, match="fit spec"):
        _lib.check(L.bmc_lm_fit(pr, dummy, ev, dummy, None, spec, dummy, dummy, dummy, None, None, None))
    spec.n_params, spec.n_iter = 1, 3
    spec.field_row[0] = 99
    with pytest.raises(RuntimeError, match="field row 99"):
        _lib.check(L.bmc_lm_fit(pr, dummy, ev, dummy, None, spec, dummy, dummy, dummy, None, None, None))
    spec.field_row[0] = _lib.SLOT_SPREAD_SIGMA
    with pytest.raises(RuntimeError, match="needs a spread"):
        _lib.check(L.bmc_lm_fit(pr, dummy, ev, dummy, None, spec, dummy, dummy, dummy, None, None, None))


def test_tangent_mode_switch_is_checked():
    """bmc_set_tangent_mode takes BMC_TANGENTS_AUTO or BMC_TANGENTS_FORWARD and refuses anything else."""
    from bmc_b200 import settings
    L = _lib.lib()
    assert L.bmc_set_tangent_mode(7) != 0
    assert L.bmc_set_tangent_mode(_lib.TANGENTS_FORWARD) == 0
    assert L.bmc_set_tangent_mode(_lib.TANGENTS_AUTO) == 0
    with pytest.raises(ValueError):
        settings.use_tangents("reverse")
    assert settings.use_tangents("forward") == "forward" and settings.tangent_mode() == "forward"
    assert settings.use_tangents("auto") == "auto"


def test_design_jvp_arguments_are_checked():
    """bmc_simulate_design_jvp refuses what it does not compute (start-state tangents, a spread-width
    tangent, float32, a whole-state output) and null outputs, with a status, before touching the GPU."""
    L = _lib.lib()
    dummy = C.c_void_p(16)
    ev = _lib.Events(16, 16, 16, 16, 16, 16)
    pr = _lib.Problem(2, 3, 2, 1, 4, 1, 0, 0)
    tg = _lib.Tangents()
    tg.n_tangents = 1
    tg.field_row[0] = 3
    tg.d_seed = 16
    call = lambda p, t, z=dummy, jz=dummy, dz=dummy, djz=dummy: L.bmc_simulate_design_jvp(
        p, dummy, ev, dummy, None, None, None, t, z, jz, dz, djz, None)
    with pytest.raises(RuntimeError, match="null design-derivative output"):
        _lib.check(call(pr, tg, dz=None))
    tg.d_dm0 = 16
    with pytest.raises(RuntimeError, match="start-state tangents"):
        _lib.check(call(pr, tg))
    tg.d_dm0 = None
    tg.field_row[0] = _lib.SEED_SPREAD_SIGMA
    with pytest.raises(RuntimeError, match="seeds the spread"):
        _lib.check(call(pr, tg))
    tg.field_row[0] = 3
    with pytest.raises(RuntimeError, match="float64 only"):
        _lib.check(call(_lib.Problem(2, 3, 2, 1, 4, 1, 1, 0), tg))
    with pytest.raises(RuntimeError, match="mz_loc >= 0"):
        _lib.check(call(_lib.Problem(2, 3, 2, 1, -1, 1, 0, 0), tg))
    tg.n_tangents = 0
    with pytest.raises(RuntimeError, match="tangents: 1"):
        _lib.check(call(pr, tg))
