"""ctypes binding of the C ABI in include/toothpaste_gpu.h.

The shared library is built in-tree by fhetoothpaste_b200/build.py. There is no
fallback: if the library is missing or a CUDA call fails, the call raises.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libtoothpaste_gpu.so"
HEADER = PKG.parent / "include" / "toothpaste_gpu.h"

U64 = ctypes.c_uint64
U64P = ctypes.POINTER(ctypes.c_uint64)
VP = ctypes.c_void_p

TP_OK, TP_ERR_PARAM, TP_ERR_OOM, TP_ERR_CUDA, TP_ERR_TIMEOUT, TP_ERR_LAYOUT, TP_ERR_STATE = range(7)
STATUS_NAMES = {0: "TP_OK", 1: "TP_ERR_PARAM", 2: "TP_ERR_OOM", 3: "TP_ERR_CUDA", 4: "TP_ERR_TIMEOUT",
                5: "TP_ERR_LAYOUT", 6: "TP_ERR_STATE"}

TP_BR_CGGI_BINARY, TP_BR_CGGI_TERNARY, TP_BR_BMMP_BINARY = 0, 1, 2
TP_MS_ROUND, TP_MS_FLOOR, TP_MS_CEIL = 0, 1, 2
GOLDILOCKS = 0xFFFFFFFF00000001


class TpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class BrParams(ctypes.Structure):
    _fields_ = [("variant", ctypes.c_int32), ("modulus", U64), ("ring_dim", ctypes.c_uint32),
                ("lwe_dim", ctypes.c_uint32), ("basis", U64), ("digits", ctypes.c_uint32)]


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libtoothpaste_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing; run `python -m fhetoothpaste_b200.build` (needs nvcc)")
    L = ctypes.CDLL(str(LIB_PATH))
    sig = {
        "tp_br_create": (ctypes.c_int, [ctypes.POINTER(BrParams), ctypes.c_int, ctypes.POINTER(VP)]),
        "tp_br_destroy": (ctypes.c_int, [VP]),
        "tp_br_key_words": (U64, [VP]),
        "tp_br_upload_key": (ctypes.c_int, [VP, U64P, U64]),
        "tp_br_blind_rotate": (ctypes.c_int, [VP, U64P, U64P, U64P, ctypes.c_int]),
        "tp_br_blind_rotate_batch": (ctypes.c_int, [VP, U64, VP, VP, U64, VP, U64, ctypes.c_int, VP]),
        "tp_br_blind_rotate_batch_host": (ctypes.c_int, [VP, U64, U64P, U64P, U64, U64P, U64, ctypes.c_int, VP]),
        "tp_br_check": (ctypes.c_int, [VP, VP]),
        "tp_br_set_tile": (ctypes.c_int, [VP, ctypes.c_uint32]),
        "tp_br_get_tile": (ctypes.c_uint32, [VP]),
        "tp_br_set_split": (ctypes.c_int, [VP, ctypes.c_uint32]),
        "tp_br_get_split": (ctypes.c_uint32, [VP]),
        "tp_br_set_mac_form": (ctypes.c_int, [VP, ctypes.c_uint32]),
        "tp_br_get_mac_form": (ctypes.c_uint32, [VP]),
        "tp_br_set_radix": (ctypes.c_int, [VP, ctypes.c_uint32]),
        "tp_br_get_radix": (ctypes.c_uint32, [VP]),
        "tp_br_autotune": (ctypes.c_int, [VP, U64, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_double)]),
        "tp_sample_extract_batch": (ctypes.c_int, [ctypes.c_uint32, U64, VP, VP, VP]),
        "tp_br_batch_graph_create": (ctypes.c_int, [VP, U64, VP, VP, U64, VP, U64, ctypes.c_int, VP,
                                                    ctypes.POINTER(VP)]),
        "tp_graph_launch": (ctypes.c_int, [VP, VP]),
        "tp_graph_destroy": (ctypes.c_int, [VP]),
        "tp_ntt_forward": (ctypes.c_int, [ctypes.c_uint32, U64, VP, VP, VP]),
        "tp_ntt_backward": (ctypes.c_int, [ctypes.c_uint32, U64, VP, VP, VP]),
        "tp_rlwe_ks_create": (ctypes.c_int, [ctypes.c_uint32, U64, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(VP)]),
        "tp_auto_create": (ctypes.c_int, [ctypes.c_uint32, U64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                          ctypes.POINTER(VP)]),
        "tp_pack_create": (ctypes.c_int, [ctypes.c_uint32, U64, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(VP)]),
        "tp_ks_destroy": (ctypes.c_int, [VP]),
        "tp_ks_key_words": (U64, [VP]),
        "tp_ks_upload_key": (ctypes.c_int, [VP, U64P, U64]),
        "tp_ks_set_tile": (ctypes.c_int, [VP, ctypes.c_uint32]),
        "tp_ks_get_tile": (ctypes.c_uint32, [VP]),
        "tp_rlwe_ks_batch": (ctypes.c_int, [VP, U64, VP, VP, VP]),
        "tp_auto_eval_batch": (ctypes.c_int, [VP, U64, VP, VP, VP]),
        "tp_pack_batch": (ctypes.c_int, [VP, U64, U64, VP, VP, VP]),
        "tp_pack_batch_noalloc": (ctypes.c_int, [VP, U64, U64, VP, VP, VP]),
        "tp_pack_subtree_batch": (ctypes.c_int, [VP, U64, U64, VP, VP, VP]),
        "tp_pack_merge_batch": (ctypes.c_int, [VP, U64, U64, ctypes.c_uint32, ctypes.c_int, VP, VP, VP]),
        "tp_pack_consecutive_batch": (ctypes.c_int, [VP, U64, U64, VP, VP, VP]),
        "tp_trace_eval_batch": (ctypes.c_int, [VP, U64, VP, VP, VP]),
        "tp_trace_eval_auto_batch": (ctypes.c_int, [VP, U64, VP, VP, ctypes.c_uint32, VP]),
        "tp_lwe_ks_create": (ctypes.c_int, [U64, ctypes.c_uint32, ctypes.c_uint32, U64, ctypes.c_uint32, ctypes.c_int,
                                            ctypes.POINTER(VP)]),
        "tp_lwe_ks_destroy": (ctypes.c_int, [VP]),
        "tp_lwe_ks_key_words": (U64, [VP]),
        "tp_lwe_ks_upload_key": (ctypes.c_int, [VP, U64P, U64]),
        "tp_lwe_ks_batch": (ctypes.c_int, [VP, U64, VP, VP, VP]),
        "tp_key_file_write": (ctypes.c_int, [ctypes.c_char_p, VP, U64P]),
        "tp_key_file_info": (ctypes.c_int, [ctypes.c_char_p, VP]),
        "tp_key_file_read": (ctypes.c_int, [ctypes.c_char_p, VP, U64P, U64]),
        "tp_br_upload_key_file": (ctypes.c_int, [VP, ctypes.c_char_p]),
        "tp_ks_upload_key_file": (ctypes.c_int, [VP, ctypes.c_char_p]),
        "tp_lwe_ks_upload_key_file": (ctypes.c_int, [VP, ctypes.c_char_p]),
        "tp_modulus_switch_batch": (ctypes.c_int, [U64, VP, U64, U64, ctypes.c_int, VP]),
        "tp_pbs_epilogue_batch": (ctypes.c_int, [VP, U64, VP, VP, U64, VP]),
        "tp_pbs_graph_create": (ctypes.c_int, [VP, VP, U64, VP, VP, VP, U64, VP, ctypes.POINTER(VP)]),
        "tp_ss_create": (ctypes.c_int, [ctypes.POINTER(BrParams), U64, ctypes.c_uint32, U64, ctypes.c_uint32,
                                        ctypes.c_uint32, U64, ctypes.c_int, ctypes.POINTER(VP)]),
        "tp_ss_destroy": (ctypes.c_int, [VP]),
        "tp_ss_key_words": (U64, [VP, ctypes.c_int]),
        "tp_ss_upload_keys": (ctypes.c_int, [VP, U64P, U64, U64P, U64, U64P, U64]),
        "tp_ss_accumulator": (ctypes.c_int, [VP, U64P]),
        "tp_lwe_to_rgsw_batch": (ctypes.c_int, [VP, U64, VP, VP, VP]),
        "tp_sap_create": (ctypes.c_int, [ctypes.POINTER(BrParams), U64, ctypes.c_uint32, U64, ctypes.c_uint32,
                                         ctypes.c_int, ctypes.POINTER(VP)]),
        "tp_sap_destroy": (ctypes.c_int, [VP]),
        "tp_sap_key_words": (U64, [VP, ctypes.c_int]),
        "tp_sap_upload_keys": (ctypes.c_int, [VP, U64P, U64, U64P, U64, U64P, U64]),
        "tp_sap_decompose_batch": (ctypes.c_int, [VP, U64, VP, U64, VP, U64, U64, U64,
                                                  ctypes.POINTER(ctypes.c_uint32), VP]),
        "tp_sap_homtrunc_batch": (ctypes.c_int, [VP, U64, VP, VP, U64, VP]),
        "tp_sap_reset_batch": (ctypes.c_int, [VP, U64, VP, U64, VP]),
        "tp_server_create": (ctypes.c_int, [ctypes.c_int, U64, ctypes.POINTER(VP)]),
        "tp_server_add_set": (ctypes.c_int, [VP, VP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(ctypes.c_uint32)]),
        "tp_server_start": (ctypes.c_int, [VP]),
        "tp_server_set_memory_budget": (ctypes.c_int, [VP, U64]),
        "tp_server_memory": (ctypes.c_int, [VP, ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.POINTER(U64)]),
        "tp_server_submit": (ctypes.c_int, [VP, ctypes.c_uint32, U64P, U64P, U64P, ctypes.POINTER(U64)]),
        "tp_server_wait": (ctypes.c_int, [VP, U64, ctypes.c_uint32]),
        "tp_server_drain": (ctypes.c_int, [VP, ctypes.c_uint32]),
        "tp_server_stats": (ctypes.c_int, [VP, ctypes.POINTER(ctypes.c_double)]),
        "tp_server_reset_stats": (ctypes.c_int, [VP]),
        "tp_server_destroy": (ctypes.c_int, [VP]),
        "tp_server_last_error": (ctypes.c_char_p, []),
        "tp_server_run_poisson": (ctypes.c_int, [VP, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                                 ctypes.c_uint32, ctypes.POINTER(U64P), ctypes.POINTER(U64P), U64P,
                                                 U64]),
        "tp_debug_arith": (ctypes.c_int, [ctypes.c_int, U64, VP, VP, VP, VP, VP]),
        "tp_measure_int_peak": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                                ctypes.POINTER(ctypes.c_double)]),
        "tp_last_error": (ctypes.c_char_p, []),
        "tp_kernel_launches": (U64, []),
        "tp_ctx_create": (ctypes.c_int, [ctypes.POINTER(BrParams), ctypes.POINTER(VP)]),
        "tp_ctx_destroy": (ctypes.c_int, [VP]),
        "tp_brk_upload": (ctypes.c_int, [VP, U64P, U64, ctypes.c_int]),
        "tp_blind_rotate": (ctypes.c_int, [VP, U64P, U64P, U64P, ctypes.c_int]),
        "tp_blind_rotate_batch": (ctypes.c_int, [VP, U64, VP, VP, VP, U64, ctypes.c_int, VP]),
        "tp_auto_ks_batch": (ctypes.c_int, [VP, U64, VP, VP, VP]),
        "tp_last_error_string": (ctypes.c_char_p, []),
        "tp_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != TP_OK:
        raise TpError(status, lib().tp_last_error().decode())


def header_symbols() -> list[str]:
    """Entry points declared in include/toothpaste_gpu.h."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(tp_\w+)\s*\(", text, re.M)))


def ptr(a) -> U64P:
    """uint64 pointer of a contiguous numpy array."""
    return a.ctypes.data_as(U64P)
