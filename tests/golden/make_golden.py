"""Regenerates the reference goldens from the reference updater.

Needs a GPU and oracle/_ref/libpscbfm_ref*.so (`make -C oracle ref`, which compiles the reference
sources with two shim headers). For every case it drives the reference through its setter API
(oracle/ref_harness.cu) with the engine's counter draw stream for the system's seed, in the listed
runSimulationOnGPU chunks, and records the SHA-256 of the final positions.

    python tests/golden/make_golden.py [--out PATH]            # cases.py CASES -> reference_positions.json
    python tests/golden/make_golden.py --long [--out PATH]     # the configs at their stated MCS
                                                               # -> reference_long.json
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from cases import CASES, GOLDEN_JSON, LONG_CASES, LONG_JSON, ROOT, ensemble_cases, positions_digest  # noqa: E402

sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--long", action="store_true", help="the configs at their stated run lengths")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    cases = dict(LONG_CASES, **ensemble_cases()) if args.long else CASES
    out_path = args.out or (LONG_JSON if args.long else GOLDEN_JSON)
    out = {}
    t_all = time.time()
    for name, (build, chunks) in cases.items():
        t0 = time.time()
        s = build()
        n_colors = int(O.color(s).max()) + 1
        draws = O.counter_draws(s.seed, 0, 2 * n_colors * sum(chunks))
        xyz, used = O.ref_run(s, draws, chunks)
        assert used == len(draws), (name, used, len(draws))
        out[name] = {"n": s.n, "seed": s.seed, "chunks": chunks, "n_colors": n_colors, "box": list(s.box),
                     "sha256": positions_digest(xyz), "head": xyz[:4].tolist()}
        print(name, s.n, n_colors, out[name]["sha256"][:16], f"{time.time() - t0:.2f}s", flush=True)
    with open(out_path, "w") as f:
        json.dump({"generator": "reference updater (src/pscbfm) on sm_100a via oracle/ref_harness.cu",
                   "draw_stream": "counter (SplitMix64), seed per case", "cases": out}, f, indent=1)
    print(f"{len(out)} cases in {time.time() - t_all:.1f}s -> {out_path}", flush=True)


if __name__ == "__main__":
    main()
