"""The C-ABI library: it loads, exports every symbol include/bfm.h declares, the Python binding
declares a signature for each, and without a GPU it fails loudly (no CPU fallback)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from pscbfm_b200 import _lib
from pscbfm_b200 import systems as S
from pscbfm_b200.updater import color_graph, counter_draw


def test_exports_every_declared_symbol():
    L = _lib.load()
    declared = _lib.declared_symbols()
    assert len(declared) >= 35
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared) <= exported


def test_binding_covers_header():
    declared = set(_lib.declared_symbols())
    bound = set(_lib._SIGS) | set(_lib._RET)
    assert declared == bound, (declared ^ bound)


def test_null_handle_and_null_buffers():
    L = _lib.load()
    assert L.bfm_run(None, 1) == _lib.BFM_ERR_NULL_HANDLE
    assert L.bfm_destroy(None) == _lib.BFM_OK
    assert L.bfm_create(None, 0) == _lib.BFM_ERR_INVALID_ARGUMENT


def test_no_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib.load()
    h = C.c_void_p()
    st = L.bfm_create(C.byref(h), 0)
    assert st == _lib.BFM_ERR_CUDA
    assert b"cuda" in L.bfm_last_error(None).lower()


def test_host_colouring_matches_oracle():
    from oracle import oracle as O
    for s in [S.small_chains(), S.rings_and_free(), S.square_network(), S.crosslinked_network(),
              S.serpentine_chains(64, 128, 0.4)]:
        assert np.array_equal(color_graph(s), O.color(s)), s.name


def test_counter_stream_matches_oracle():
    from oracle import oracle as O
    ref = O.counter_draws(42, 0, 64)
    assert [counter_draw(42, k) for k in range(64)] == ref.tolist()
    assert counter_draw(7, 0) != counter_draw(8, 0)


def test_colour_errors():
    L = _lib.load()
    cnt = np.array([1], np.uint32)
    ids = np.array([5], np.uint32)
    out = np.zeros(1, np.uint8)
    nc = C.c_uint32()
    assert L.bfm_color_graph(1, cnt, ids, 1, out, C.byref(nc)) == _lib.BFM_ERR_OUT_OF_RANGE
    assert L.bfm_color_graph(0, cnt, ids, 1, out, C.byref(nc)) == _lib.BFM_ERR_INVALID_ARGUMENT


def test_lemonade_adapter_compiles(tmp_path):
    """include/bfm_lemonade.hpp instantiated with an ingredients type that has the LeMonADE calls the
    reference adapter makes (src/pscbfm/GPUScBFM_AB_Type.h:78-176) compiles and links (the updater
    base class and VectorInt3 come from minimal stand-ins in tests/lemonade_stub)."""
    import os
    src = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lemonade_stub", "caller.cpp")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = tmp_path / "lemonade_caller"
    r = subprocess.run(["g++", "-std=c++14", "-I", os.path.join(root, "include"),
                        "-I", os.path.join(root, "tests", "lemonade_stub"), src, "-o", str(out),
                        "-L", os.path.join(root, "pscbfm_b200"), "-lbfm",
                        "-Wl,-rpath," + os.path.join(root, "pscbfm_b200")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_wrapper_compiles_for_reference_style_callers(tmp_path):
    """A caller written like GPUScBFM_AB_Type::initialize/execute compiles and links against
    include/bfm_updater.hpp + libbfm.so."""
    import os
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include "bfm_updater.hpp"
#include <cstdio>
int main() {
    try {
        UpdaterGPUScBFM_AB_Type u;
        u.setGpu(0);
        u.setPeriodicity(true, true, true);
        u.setNrOfAllMonomers(2);
        u.setMonomerCoordinates(0, 0, 0, 0);
        u.setMonomerCoordinates(1, 2, 0, 0);
        u.setAttribute(0, 1);
        u.setConnectivity(0, 1);
        u.setConnectivity(1, 0);
        u.setLatticeSize(8, 8, 8);
        u.populateLattice();
        for (int dx = -4; dx < 4; ++dx) for (int dy = -4; dy < 4; ++dy) for (int dz = -4; dz < 4; ++dz)
            u.copyBondSet(dx, dy, dz, true);
        u.initialize();
        u.runSimulationOnGPU(10);
        std::printf("%d\n", u.getMonomerPositionInX(1));
        u.cleanup();
    } catch (std::exception const& e) { std::printf("error: %s\n", e.what()); return 1; }
    return 0;
}
''')
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = tmp_path / "caller"
    r = subprocess.run(["g++", "-std=c++14", "-I", os.path.join(root, "include"), str(src), "-o", str(out),
                        "-L", os.path.join(root, "pscbfm_b200"), "-lbfm",
                        "-Wl,-rpath," + os.path.join(root, "pscbfm_b200")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_reference_adapter_compiles_unchanged():
    """The reference's LeMonADE adapter (src/pscbfm/GPUScBFM_AB_Type.h) and its logger header,
    copied unchanged, compile and link over include/bfm_updater.hpp (oracle/Makefile target
    `adapter`); the GPU suite runs the result against the oracle. Needs the reference tree
    ($PSCBFM_REFERENCE, by default where this build's reference lies)."""
    tree = os.environ.get("PSCBFM_REFERENCE", "/root/reference")
    if not os.path.exists(os.path.join(tree, "src", "pscbfm", "GPUScBFM_AB_Type.h")):
        pytest.skip("reference tree not present")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run(["make", "-s", "-B", "-C", os.path.join(root, "oracle"), "adapter", f"REF={tree}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert os.path.exists(os.path.join(root, "oracle", "_ref", "ref_adapter"))
