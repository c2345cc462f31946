"""C-ABI checks that need no GPU: the library loads, exports every declared
entry point, and rejects bad parameters before touching the device."""
import ctypes
import subprocess

import pytest


def test_library_exports_every_declared_symbol(native):
    from fhetoothpaste_b200 import _native
    declared = _native.header_symbols()
    assert "tp_br_blind_rotate" in declared and len(declared) >= 12
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, f"declared but not exported: {missing}"


@pytest.mark.parametrize("field,value", [("modulus", 36028797018972161), ("ring_dim", 1000), ("ring_dim", 131072),
                                         ("ring_dim", 64), ("lwe_dim", 0), ("basis", 3), ("basis", 1 << 31),
                                         ("digits", 0), ("digits", 9), ("variant", 7)])
def test_bad_parameters_are_rejected(native, field, value):
    from fhetoothpaste_b200 import _native
    prm = _native.BrParams(1, _native.GOLDILOCKS, 1024, 500, 1 << 16, 4)
    setattr(prm, field, value)
    h = ctypes.c_void_p()
    st = native.tp_br_create(ctypes.byref(prm), 0, ctypes.byref(h))
    assert st == _native.TP_ERR_PARAM
    assert native.tp_last_error().decode()
    assert not h.value


def test_bmmp_requires_even_dimension(native):
    from fhetoothpaste_b200 import _native
    prm = _native.BrParams(2, _native.GOLDILOCKS, 1024, 501, 1 << 16, 4)
    h = ctypes.c_void_p()
    assert native.tp_br_create(ctypes.byref(prm), 0, ctypes.byref(h)) == _native.TP_ERR_PARAM


def test_digits_beyond_gadget_are_rejected(native):
    from fhetoothpaste_b200 import _native
    prm = _native.BrParams(1, _native.GOLDILOCKS, 1024, 500, 1 << 16, 5)  # ceil(64/16) = 4
    h = ctypes.c_void_p()
    assert native.tp_br_create(ctypes.byref(prm), 0, ctypes.byref(h)) == _native.TP_ERR_PARAM


def test_null_context_calls_fail_cleanly(native):
    from fhetoothpaste_b200 import _native
    assert native.tp_br_upload_key(None, None, 0) == _native.TP_ERR_PARAM
    assert native.tp_br_blind_rotate(None, None, None, None, 0) == _native.TP_ERR_PARAM
    assert native.tp_br_check(None, None) == _native.TP_ERR_PARAM
    assert native.tp_br_key_words(None) == 0
    assert native.tp_br_set_split(None, 2) == _native.TP_ERR_PARAM
    assert native.tp_br_get_split(None) == 0
    assert native.tp_br_set_tile(None, 4) == _native.TP_ERR_PARAM
    assert native.tp_ntt_forward(1000, 1, None, None, None) == _native.TP_ERR_PARAM
    assert native.tp_ss_create(None, 1 << 16, 4, 1 << 16, 4, 4, 1 << 16, 0, None) == _native.TP_ERR_PARAM
    assert native.tp_ss_upload_keys(None, None, 0, None, 0, None, 0) == _native.TP_ERR_PARAM
    assert native.tp_ss_accumulator(None, None) == _native.TP_ERR_PARAM
    assert native.tp_lwe_to_rgsw_batch(None, 1, None, None, None) == _native.TP_ERR_PARAM
    assert native.tp_ss_key_words(None, 0) == 0
    assert native.tp_ss_destroy(None) == _native.TP_OK


def test_scheme_switch_rejects_bad_output_gadget(native):
    """Parameter checks run before any device call, so they answer on a machine without a GPU."""
    from fhetoothpaste_b200 import _native
    prm = _native.BrParams(0, _native.GOLDILOCKS, 256, 16, 1 << 16, 4)
    h = ctypes.c_void_p()
    for digits, basis in ((3, 1 << 16), (2, 1 << 16), (4, 3 << 10)):
        assert native.tp_ss_create(ctypes.byref(prm), 1 << 16, 4, 1 << 16, 4, digits, basis, 0,
                                   ctypes.byref(h)) == _native.TP_ERR_PARAM
        assert not h.value


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """No fallback: without the built CUDA library the package refuses to run."""
    from fhetoothpaste_b200 import _native
    monkeypatch.setattr(_native, "LIB_PATH", tmp_path / "libtoothpaste_gpu.so")
    monkeypatch.setattr(_native, "_lib", None)
    with pytest.raises(ImportError):
        _native.lib()


def test_launch_counter_starts_without_launches(native):
    """No kernel has run in a process without a GPU; the counter is exported and readable."""
    assert native.tp_kernel_launches() == 0


def test_short_names_check_their_arguments(native):
    from fhetoothpaste_b200 import _native
    assert native.tp_ctx_create(None, None) == _native.TP_ERR_PARAM
    assert native.tp_brk_upload(None, None, 0, 1) == _native.TP_ERR_LAYOUT
    assert native.tp_brk_upload(None, None, 0, 0) == _native.TP_ERR_PARAM
    assert native.tp_blind_rotate_batch(None, 1, None, None, None, 0, 0, None) == _native.TP_ERR_PARAM
    assert native.tp_ctx_destroy(None) == _native.TP_OK
    assert native.tp_last_error_string() == native.tp_last_error()
