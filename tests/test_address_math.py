"""The lattice-address arithmetic of the bond-code kernels (a monomer's corner stored as its
occupancy-lattice address; moves and the front plane as adds confined to one axis's address bits),
checked on the host against plain coordinates for several box shapes: every position, every
direction, the step, the nine front-plane cells and the walls; and the read-back of bond-code
systems, whose x/y/z hold image offsets: the coordinate extracted from an address, the offset plus
it giving the unfolded coordinate back, and the wrap test behind the offset update
(tests/address_check.cu)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_address_arithmetic_matches_coordinates(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    exe = str(tmp_path / "address_check")
    r = subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", os.path.join(ROOT, "pscbfm_b200", "csrc"), os.path.join(ROOT, "tests", "address_check.cu"),
                        "-o", exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    run = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stdout + run.stderr
