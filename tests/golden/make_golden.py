"""Generates the committed golden fixtures in tests/golden/.

* rng_kat.json    -- PCG64 streams (src/core/math/rng.hpp:126-207) computed by a
                     pure-Python restatement, independent of the C++ oracle.
* karras_kat.json -- Karras-2012 parent arrays (build_lbvh.cu:164-245) of small
                     key sets, including duplicate keys, computed by a pure-Python
                     restatement.
* cornell_64.npz  -- CPU-oracle output for the 64x64 Cornell box (seed 0): 1-spp
                     first-hit ids and 4-spp radiance. Regenerating it requires the
                     oracle library (oracle/Makefile).

Run:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

M64 = (1 << 64) - 1


def scramble(x):
    z = (x + 0x9e3779b97f4a7c15) & M64
    z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & M64
    z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & M64
    return z ^ (z >> 31)


def pcg_next(state):
    x = state
    count = state >> 59
    state = (state * 6364136223846793005 + 1442695040888963407) & M64
    x ^= x >> (5 + count)
    x = (x * 12605985483714917081) & M64
    return x ^ (x >> 43), state


def pcg_stream(seed, n):
    s = scramble(seed)
    _, s = pcg_next(s)
    s = (s + seed) & M64
    _, s = pcg_next(s)
    out = []
    for _ in range(n):
        v, s = pcg_next(s)
        out.append(v)
    return out


def clz64(v):
    return 64 if v == 0 else 64 - v.bit_length()


def clz32(v):
    return 32 if v == 0 else 32 - v.bit_length()


def karras_parents(keys):
    """Pure-Python Karras hierarchy (build_lbvh.cu:180-245)."""
    n = len(keys)

    def lcp(i, j):
        if j < 0 or j >= n:
            return -1
        if keys[i] == keys[j]:
            return 64 + clz32((i ^ j) & 0xFFFFFFFF)
        return clz64(keys[i] ^ keys[j])

    parents = [0] * (2 * n - 1)
    for i in range(n - 1):
        d = -1 if lcp(i, i + 1) - lcp(i, i - 1) < 0 else 1
        dmin = lcp(i, i - d)
        lmax = 2
        while lcp(i, i + lmax * d) > dmin:
            lmax *= 2
        l = 0
        t = lmax
        while t > 1:
            t //= 2
            if lcp(i, i + (l + t) * d) > dmin:
                l += t
        j = i + l * d
        dnode = lcp(i, j)
        s = 0
        div = 2
        maxdiv = 1 << (32 - clz32(l))
        while div <= maxdiv:
            t = (l + div - 1) // div
            if lcp(i, i + (s + t) * d) > dnode:
                s += t
            div *= 2
        split = i + s * d + min(d, 0)
        left = split + n - 1 if min(i, j) == split else split
        right = split + n if max(i, j) == split + 1 else split + 1
        parents[left] = ~i
        parents[right] = i
        if i == 0:
            parents[0] = 0x10000000
    return parents


def main():
    kat = {"pcg64": {str(s): pcg_stream(s, 8) for s in [0, 1, 7, 1000, 65537, 4294967295]}}
    json.dump(kat, open(os.path.join(HERE, "rng_kat.json"), "w"), indent=1)
    sets = {
        "sorted8": [1, 2, 4, 5, 19, 24, 25, 30],
        "duplicates": [3, 3, 3, 7, 7, 9, 12, 12, 12, 12],
        "two": [0, 5],
        "wide": [0, 1 << 62, (1 << 62) + 1, (1 << 63) - 1],
        "random32": sorted(int(x) for x in np.random.default_rng(7).integers(0, 1 << 62, 32)),
    }
    out = {k: {"keys": v, "parents": karras_parents(v)} for k, v in sets.items()}
    json.dump(out, open(os.path.join(HERE, "karras_kat.json"), "w"), indent=1)
    try:
        from mufflon_b200 import scenes
        from oracle import pyoracle
        spec = scenes.cornell_box(0, 64, 64)
        sc = pyoracle.OracleScene(spec)
        pt = pyoracle.OraclePathTracer(sc, seed=0, max_path=8)
        pt.iterate(1)
        hit = pt.target("Hit ID").astype(np.int16)
        for _ in range(3):
            pt.iterate(1)
        rad = pt.target("Radiance")
        np.savez_compressed(os.path.join(HERE, "cornell_64.npz"), hit_id=hit, radiance=rad)
    except Exception as e:  # the oracle library is optional for the JSON fixtures
        print("skipping cornell_64.npz:", e)


if __name__ == "__main__":
    main()
