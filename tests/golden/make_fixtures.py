"""Converts the reference's input fixtures (tests/*.bfm of pscbfm) into tests/golden/ref_fixtures.npz
with pscbfm_b200.bfm_io.read_bfm, so that the tests need neither the reference tree nor the .bfm
files. Positions are stored as int16 (the reference's coordinate type), neighbour lists as the
directed (owner, target) pairs in list order, plus the box, periodicity and forbidden-bond table.

    python tests/golden/make_fixtures.py [/path/to/pscbfm/tests]   (default: $PSCBFM_REFERENCE/tests)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from pscbfm_b200 import bfm_io  # noqa: E402

FILES = {
    "ring": "Ring_N6_n6.bfm",
    "hydrogel": "coloring-test-Hydrogel_HEP_3__PEG_3_NStar_117__NoPerXYZ64_Connected.bfm",
    "linear_chains": "LinearChain_l1024_n64.bfm",
}


def main(src):
    out = {}
    for key, fname in FILES.items():
        s, info = bfm_io.read_bfm(os.path.join(src, fname))
        rows, cols = s.bonds()
        out[f"{key}_xyz"] = s.xyz.astype(np.int16)
        out[f"{key}_pairs"] = np.stack([rows, cols], axis=1).astype(np.uint32)
        out[f"{key}_box"] = np.array(s.box, dtype=np.uint32)
        out[f"{key}_periodic"] = np.array(info["periodic"], dtype=np.uint8)
        out[f"{key}_forbidden"] = s.forbidden.astype(np.uint8)
        out[f"{key}_attributes"] = s.attributes.astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "ref_fixtures.npz"), **out)


if __name__ == "__main__":
    tree = os.environ.get("PSCBFM_REFERENCE", "/root/reference")
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(tree, "tests"))
