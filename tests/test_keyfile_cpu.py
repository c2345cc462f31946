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


def test_ciphertext_batches(native, tmp_path):
    """LWE and RLWE batches in the same container: round trip, header fields, shape checks."""
    from fhetoothpaste_b200 import TpError
    from fhetoothpaste_b200.keyfile import (read_ciphertext_batch, write_key_file, write_lwe_batch,
                                            write_rlwe_batch)
    from oracle.oracle import P, lwe_inputs, random_acc
    lwes = lwe_inputs(2048, 630, 17, 3)
    write_lwe_batch(tmp_path / "l.tpct", lwes, modulus=4096)
    info, back = read_ciphertext_batch(tmp_path / "l.tpct")
    np.testing.assert_array_equal(back, lwes)
    assert (info["kind"], info["lwe_dim"], info["index"], info["modulus"]) == (16, 630, 17, 4096)
    rl = random_acc(256, 5, 4)
    write_rlwe_batch(tmp_path / "r.tpct", rl, ntt_domain=True)
    info, back = read_ciphertext_batch(tmp_path / "r.tpct")
    np.testing.assert_array_equal(back, rl)
    assert (info["kind"], info["ring_dim"], info["variant"], info["index"], info["modulus"]) == (17, 256, 1, 5, P)
    with pytest.raises(TpError):   # 5 rows of 2N words claimed, 4 given
        write_key_file(tmp_path / "x.tpct", "rlwe_batch", rl[:4], ring_dim=256, digits=0, basis=0, index=5)
    with pytest.raises(TpError):   # domain tag other than coefficients / NTT
        write_key_file(tmp_path / "x.tpct", "rlwe_batch", rl, ring_dim=256, digits=0, basis=0, index=5, variant=2)
    with pytest.raises(ValueError):
        write_key_file(tmp_path / "k.tpkey", "packing", rl, ring_dim=256, digits=4, basis=1 << 16)
        read_ciphertext_batch(tmp_path / "k.tpkey")
