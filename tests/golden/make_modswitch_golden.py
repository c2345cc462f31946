"""Golden vectors for ModulusSwitch (lib/src/static/modulus_switching.cpp:36-93) from the
reference library built in oracle/_ref: source modulus p, targets 2N for N = 128..4096, types
ROUND / FLOOR / CEIL. Inputs include the values next to every boundary m p / 2N, where the
reference's 80-bit long double quotient rounds across the integer. Run in the container
that has the reference build:

    python tests/golden/make_modswitch_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.oracle import P, Reference, ptr, sha256, uniform_mod  # noqa: E402

OUT = Path(__file__).resolve().parent
TARGETS = [256, 2048, 4096, 8192]
KINDS = {"round": 0, "floor": 1, "ceil": 2}


def inputs(target: int) -> np.ndarray:
    """Boundary neighbours of m p / target for m spread over [0, target), extremes, random words."""
    ms = np.unique(np.linspace(0, target - 1, 257).astype(np.int64))
    vals = set()
    for m in ms.tolist():
        base = (m * P) // target
        for d in range(-2, 3):
            if 0 <= base + d < P:
                vals.add(base + d)
    vals.update([0, 1, 2, P - 1, P - 2, P // 2, P // 2 + 1])
    rand = uniform_mod(77 + target, 1024, P).tolist()
    return np.array(sorted(vals) + [int(r) for r in rand], dtype=np.uint64)


def main() -> None:
    ref = Reference()
    manifest, arrays = {}, {}
    for T in TARGETS:
        x = inputs(T)
        arrays[f"in_{T}"] = x
        manifest[str(T)] = {"count": int(x.size), "input_sha256": sha256(x)}
        for kind, code in KINDS.items():
            y = x.copy()
            ref.L.ref_modulus_switch(ptr(y), y.size, P, T, code)
            arrays[f"{kind}_{T}"] = y
    np.savez(OUT / "modswitch.npz", **arrays)
    (OUT / "modswitch.json").write_text(json.dumps(manifest, indent=1) + "\n")
    print("wrote", OUT / "modswitch.npz")


if __name__ == "__main__":
    main()
