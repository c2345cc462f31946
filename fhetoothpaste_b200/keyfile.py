"""Key files: one key in the reference's layout behind a checked header (format in
include/toothpaste_gpu.h and csrc/keyfile.cu), and batches of LWE / RLWE ciphertexts in
the same container. Host-only; no device needed."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat

KINDS = {"blind_rotation": 1, "rlwe_switch": 2, "automorphism": 3, "packing": 4, "lwe_switch": 5,
         "lwe_batch": 16, "rlwe_batch": 17}


class KeyInfo(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("variant", ctypes.c_uint32), ("ring_dim", ctypes.c_uint32),
                ("lwe_dim", ctypes.c_uint32), ("digits", ctypes.c_uint32), ("index", ctypes.c_uint32),
                ("modulus", ctypes.c_uint64), ("basis", ctypes.c_uint64), ("words", ctypes.c_uint64)]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


def write_key_file(path, kind: str, words: np.ndarray, *, ring_dim: int, digits: int, basis: int,
                   variant: int = 0, lwe_dim: int = 0, index: int = 0, modulus: int = nat.GOLDILOCKS) -> None:
    words = np.ascontiguousarray(words, dtype=np.uint64)
    info = KeyInfo(KINDS[kind], variant, ring_dim, lwe_dim, digits, index, modulus, basis, words.size)
    nat.check(nat.lib().tp_key_file_write(str(path).encode(), ctypes.byref(info), nat.ptr(words)))


def key_file_info(path) -> dict:
    info = KeyInfo()
    nat.check(nat.lib().tp_key_file_info(str(path).encode(), ctypes.byref(info)))
    return info.as_dict()


def read_key_file(path) -> tuple[dict, np.ndarray]:
    """(header fields, payload words); raises TpError if the file or its hash does not check."""
    words = np.empty(key_file_info(path)["words"], dtype=np.uint64)
    info = KeyInfo()
    nat.check(nat.lib().tp_key_file_read(str(path).encode(), ctypes.byref(info), nat.ptr(words), words.size))
    return info.as_dict(), words


def write_lwe_batch(path, lwes: np.ndarray, modulus: int) -> None:
    """count x (n+1) LWE words mod `modulus` (2N for rotation inputs, p after a key switch)."""
    lwes = np.ascontiguousarray(lwes, dtype=np.uint64)
    count, row = lwes.shape
    write_key_file(path, "lwe_batch", lwes, ring_dim=0, digits=0, basis=0, lwe_dim=row - 1, index=count,
                   modulus=modulus)


def write_rlwe_batch(path, rlwes: np.ndarray, ntt_domain: bool) -> None:
    """count x 2N RLWE words [A | B] mod p, coefficients or NTT domain."""
    rlwes = np.ascontiguousarray(rlwes, dtype=np.uint64)
    count, row = rlwes.shape
    write_key_file(path, "rlwe_batch", rlwes, ring_dim=row // 2, digits=0, basis=0, variant=int(ntt_domain),
                   index=count)


def read_ciphertext_batch(path) -> tuple[dict, np.ndarray]:
    """(header fields, count x row words) of an LWE or RLWE batch file."""
    info, words = read_key_file(path)
    if info["kind"] not in (KINDS["lwe_batch"], KINDS["rlwe_batch"]):
        raise ValueError(f"{path}: not a ciphertext batch (kind {info['kind']})")
    return info, words.reshape(info["index"], -1)
