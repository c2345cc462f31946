"""Key files (host-only): round trip, header fields, the payload's SHA-256 against hashlib, and the
refusals (bad magic, corrupted or truncated payload, too small a buffer)."""
import hashlib

import numpy as np
import pytest

from oracle.oracle import sm64


def test_round_trip_and_hash(native, tmp_path):
    from fhetoothpaste_b200.keyfile import read_key_file, write_key_file
    words = sm64(5, 100_003)
    path = tmp_path / "k.tpkey"
    write_key_file(path, "blind_rotation", words, ring_dim=2048, lwe_dim=630, digits=3, basis=1 << 12, variant=1)
    info, back = read_key_file(path)
    np.testing.assert_array_equal(back, words)
    assert info == {"kind": 1, "variant": 1, "ring_dim": 2048, "lwe_dim": 630, "digits": 3, "index": 0,
                    "modulus": 0xFFFFFFFF00000001, "basis": 1 << 12, "words": words.size}
    raw = path.read_bytes()
    assert raw[:8] == b"TPKEYv1\0" and len(raw) == 128 + 8 * words.size
    assert raw[64:96] == hashlib.sha256(words.astype("<u8").tobytes()).digest()
    assert raw[96:128] == bytes(32)


def test_refusals(native, tmp_path):
    from fhetoothpaste_b200 import TpError
    from fhetoothpaste_b200 import _native as nat
    from fhetoothpaste_b200.keyfile import read_key_file, write_key_file
    words = sm64(6, 4096)
    good = tmp_path / "good.tpkey"
    write_key_file(good, "lwe_switch", words, ring_dim=1024, lwe_dim=0, digits=4, basis=1 << 16)
    raw = bytearray(good.read_bytes())
    cases = {}
    flipped = bytearray(raw)
    flipped[128 + 777] ^= 1
    cases["corrupt"] = bytes(flipped)
    cases["truncated"] = bytes(raw[:-8])
    bad_magic = bytearray(raw)
    bad_magic[0] = ord("X")
    cases["magic"] = bytes(bad_magic)
    cases["short"] = bytes(raw[:100])
    for name, data in cases.items():
        p = tmp_path / f"{name}.tpkey"
        p.write_bytes(data)
        with pytest.raises(TpError) as ei:
            read_key_file(p)
        assert ei.value.status == nat.TP_ERR_LAYOUT, name
    import ctypes
    from fhetoothpaste_b200.keyfile import KeyInfo
    small = np.empty(10, np.uint64)
    assert nat.lib().tp_key_file_read(str(good).encode(), ctypes.byref(KeyInfo()), nat.ptr(small), 10) == \
        nat.TP_ERR_PARAM
    assert nat.lib().tp_key_file_info(b"/nonexistent/x.tpkey", ctypes.byref(KeyInfo())) == nat.TP_ERR_PARAM
