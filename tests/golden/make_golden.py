"""Generates the golden fixtures under tests/golden/.

1. rng_vectors.json -- SplitMix64 / xoshiro256++ outputs computed by an
   independent pure-Python restatement of the published algorithms
   (Vigna's SplitMix64 and xoshiro256++ as used by src/rng.zig:10-88).  These
   pin the C oracle's and the device's RNG bit for bit; neither is used to
   produce them.
2. images.json -- SHA-256 digests of f64 HDR images rendered by the C oracle
   for small fixed scenes and seeds (the reference itself cannot run here:
   no Zig toolchain).  They freeze the oracle's output so that any later
   change to it, or to the device path, is caught.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import math
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
MASK = (1 << 64) - 1
GOLDEN_RATIO = 0x9E3779B97F4A7C15


def splitmix64(state: int):
    state = (state + GOLDEN_RATIO) & MASK
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return state, z ^ (z >> 31)


def rotl(x: int, k: int) -> int:
    return ((x << k) | (x >> (64 - k))) & MASK


class PyRng:
    """Pure-Python xoshiro256++ seeded through SplitMix64."""

    def __init__(self, seed: int):
        sm = seed & MASK
        self.s = []
        for _ in range(4):
            sm, v = splitmix64(sm)
            self.s.append(v)

    @staticmethod
    def for_stream(seed: int, stream: int) -> "PyRng":
        sm = (seed ^ ((stream * GOLDEN_RATIO) & MASK)) & MASK
        _, v = splitmix64(sm)
        return PyRng(v)

    def next(self) -> int:
        s = self.s
        result = (rotl((s[0] + s[3]) & MASK, 23) + s[0]) & MASK
        t = (s[1] << 17) & MASK
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = rotl(s[3], 45)
        return result

    def float(self) -> float:
        return (self.next() >> 11) * 2.0 ** -53


def rng_vectors() -> dict:
    out = {"splitmix64_seed0": [], "init": {}, "for_stream": {}, "floats": {}}
    sm = 0
    for _ in range(8):
        sm, v = splitmix64(sm)
        out["splitmix64_seed0"].append(v)
    for seed in (0, 1, 42, 2026, MASK):
        r = PyRng(seed)
        out["init"][str(seed)] = {"state": list(r.s), "next": [r.next() for _ in range(16)]}
    for seed, stream in ((0, 0), (0, 1), (7, 0), (7, 1), (0, 65535), (99, 123456789), (MASK, 2 ** 40 + 3)):
        r = PyRng.for_stream(seed, stream)
        out["for_stream"][f"{seed}:{stream}"] = {"state": list(r.s), "next": [r.next() for _ in range(16)]}
    r = PyRng.for_stream(0, 0)
    out["floats"]["0:0"] = [r.float().hex() for _ in range(16)]
    return out


def image_digest(img) -> str:
    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(img, np.float64).tobytes()).hexdigest()


def image_goldens() -> dict:
    sys.path.insert(0, str(HERE.parent.parent))
    sys.path.insert(0, str(HERE.parent))
    import oracle as O
    import kat_scenes as K
    out = {}
    for name, (scene, opts) in K.golden_cases().items():
        os_ = O.OracleScene.from_scene(scene)
        img = os_.render(**opts, threads=4)
        out[name] = {"options": opts, "sha256": image_digest(img), "mean": [float(x) for x in img.mean(axis=0)]}
    return out


def main() -> None:
    (HERE / "rng_vectors.json").write_text(json.dumps(rng_vectors(), indent=1) + "\n")
    (HERE / "images.json").write_text(json.dumps(image_goldens(), indent=1, sort_keys=True) + "\n")
    print("wrote", HERE / "rng_vectors.json", HERE / "images.json")


if __name__ == "__main__":
    main()
