"""Writes tests/golden/ref_rng_sfcurves_kat.json from the reference's own code.

`make -C oracle ref` compiles oracle/refpin/refpin.cpp against the reference's
src/core/math/rng.hpp and src/core/math/sfcurves.hpp (behind the stand-in
headers of oracle/refpin/stub) into oracle/_ref/refpin; this script runs it
and stores its known answers: SplitMix64 seeds, PCG64 streams (also for the
per-pixel seeds of a 1080p frame), GoldenRatio2D sequences, and the Morton,
Hilbert and gray-code helpers. tests/test_oracle_refpin.py checks the
oracle's restatements against them.

Run (where the reference sources are present):  python tests/golden/make_ref_kat.py
"""
import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"])
    out = subprocess.check_output([os.path.join(ROOT, "oracle", "_ref", "refpin")], text=True)
    kat = json.loads(out)
    kat = {k: [int(x) for x in v] for k, v in kat.items()}
    kat["_source"] = ("reference src/core/math/rng.hpp and src/core/math/sfcurves.hpp compiled by "
                      "oracle/refpin/refpin.cpp (make -C oracle ref)")
    with open(os.path.join(HERE, "ref_rng_sfcurves_kat.json"), "w") as f:
        json.dump(kat, f, indent=0)
        f.write("\n")


if __name__ == "__main__":
    main()
