"""C-ABI checks that need no GPU: the library loads, exports every symbol the header declares,
and refuses bad input with the reference's return codes."""

import ctypes as C

import numpy as np
import pytest

import fereg_b200 as fb


def test_library_exports_every_declared_symbol():
    lib = fb.lib()
    syms = fb.declared_symbols()
    assert "fereg_absorber_residualize" in syms and "fereg_absorber_create" in syms
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_create_rejects_bad_codes_with_rc_198():
    codes = [np.array([0, 1, 5], dtype=np.uint32)]
    with pytest.raises(fb.FeregError) as e:
        fb.Absorber(codes, [2])
    assert e.value.rc == 198


def test_create_rejects_too_few_rows_with_rc_2001():
    with pytest.raises(fb.FeregError) as e:
        fb.Absorber([np.array([0], dtype=np.uint32)], [1])
    assert e.value.rc == 2001


def test_null_handle_is_an_error_not_a_crash():
    lib = fb.lib()
    rc = lib.fereg_absorber_set_weights(None, None)
    assert rc == 198
    assert b"NULL" in lib.fereg_last_error()
