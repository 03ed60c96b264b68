"""Regenerates tests/golden/reference_positions.json from the reference updater.

Needs a GPU and oracle/_ref/libpscbfm_ref.so (`make -C oracle ref`, which compiles the reference
sources with two shim headers). For every case in cases.py it drives the reference through its
setter API (oracle/ref_harness.cu) with the engine's counter draw stream for the system's seed,
in the listed runSimulationOnGPU chunks, and records the SHA-256 of the final positions.

    python tests/golden/make_golden.py [--out PATH]
"""
import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from cases import CASES, GOLDEN_JSON, ROOT, positions_digest  # noqa: E402

sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=GOLDEN_JSON)
    args = ap.parse_args()
    out = {}
    for name, (build, chunks) in CASES.items():
        s = build()
        n_colors = int(O.color(s).max()) + 1
        draws = O.counter_draws(s.seed, 0, 2 * n_colors * sum(chunks))
        xyz, used = O.ref_run(s, draws, chunks)
        assert used == len(draws), (name, used, len(draws))
        out[name] = {"n": s.n, "seed": s.seed, "chunks": chunks, "n_colors": n_colors,
                     "sha256": positions_digest(xyz), "head": xyz[:4].tolist()}
        print(name, out[name]["sha256"][:16], flush=True)
    with open(args.out, "w") as f:
        json.dump({"generator": "reference updater (src/pscbfm) on sm_100a via oracle/ref_harness.cu",
                   "draw_stream": "counter (SplitMix64), seed per case", "cases": out}, f, indent=1)


if __name__ == "__main__":
    main()
