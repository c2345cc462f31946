"""Key files: one key in the reference's layout behind a checked header (format in
include/toothpaste_gpu.h and csrc/keyfile.cu). Host-only; no device needed."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat

KINDS = {"blind_rotation": 1, "rlwe_switch": 2, "automorphism": 3, "packing": 4, "lwe_switch": 5}


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
