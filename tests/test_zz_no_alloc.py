"""bfm_sweep_noalloc: the sweep for callers that cannot let the library allocate device memory
(a host program whose own pool already holds the GPU's memory, or a latency-sensitive loop that a
cudaMalloc/cudaFree would stall). The test owns every device buffer (allocated here with torch),
calls the entry point through the C-ABI twice in a row, and checks each result against the
existing allocating entry point (bfm_run) on the same system and draw stream: integer positions,
so the tolerance is zero. This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import pscbfm_b200 as P
from pscbfm_b200 import _lib
from pscbfm_b200 import systems as S
from pscbfm_b200.updater import color_graph

pytestmark = pytest.mark.gpu

PAD = np.iinfo(np.int32).min


def sorted_layout(s):
    """Colour groups in stable original order, each starting at a multiple of 32 slots."""
    col = color_graph(s)
    nC = int(col.max()) + 1
    sizes = np.bincount(col, minlength=nC).astype(np.uint32)
    offs = np.zeros(nC, dtype=np.uint32)
    acc = 0
    for c in range(nC):
        offs[c] = acc
        acc += (int(sizes[c]) + 31) // 32 * 32
    npad = max(acc, 32)
    slot = np.zeros(s.n, dtype=np.int64)
    nxt = offs.astype(np.int64).copy()
    for i in range(s.n):
        slot[i] = nxt[col[i]]
        nxt[col[i]] += 1
    xyz = np.full((3, npad), 0, dtype=np.int32)
    xyz[0, :] = PAD
    xyz[:, slot] = s.xyz.T
    maxc = s.maxc
    nbr = np.zeros((maxc, npad), dtype=np.uint32)
    nnb = np.zeros(npad, dtype=np.uint8)
    nnb[slot] = s.nbr_count
    for k in range(maxc):
        has = s.nbr_count > k
        nbr[k, slot[has]] = slot[s.nbr_ids[has, k]]
    return nC, sizes, offs, npad, slot, xyz, nbr, nnb


def _two_calls_match_bfm_run(s, mcs):
    """Two bfm_sweep_noalloc calls of `mcs` MCS each on caller-owned buffers, each compared with
    bfm_run after the same number of MCS."""
    torch = pytest.importorskip("torch")
    L = _lib.load()
    nC, sizes, offs, npad, slot, xyz, nbr, nnb = sorted_layout(s)
    # existing entry point
    u = P.UpdaterGPUScBFM_AB_Type(0)
    u.load_system(s, mode=P.MODE_LAUNCH)
    u.runSimulationOnGPU(mcs)
    want1 = u.get_coords().copy()
    u.runSimulationOnGPU(mcs)
    want2 = u.get_coords().copy()
    u.close()
    # caller-owned device buffers
    dx, dy, dz = (torch.from_numpy(xyz[a].copy()).cuda() for a in range(3))
    dnbr = torch.from_numpy(nbr.reshape(-1).view(np.int32).copy()).cuda()
    dnnb = torch.from_numpy(nnb.copy()).cuda()
    forb = np.ascontiguousarray(s.forbidden, dtype=np.uint8)
    sysd = _lib.NoallocSystem()
    sysd.x, sysd.y, sysd.z = dx.data_ptr(), dy.data_ptr(), dz.data_ptr()
    sysd.nbr, sysd.nnb = dnbr.data_ptr(), dnnb.data_ptr()
    sysd.npad, sysd.maxc, sysd.n_colors = npad, s.maxc, nC
    sysd.box = (C.c_uint32 * 3)(*s.box)
    sysd.group_offset = offs.ctypes.data
    sysd.group_size = sizes.ctypes.data
    sysd.forbidden = forb.ctypes.data
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    for call, want in enumerate((want1, want2)):
        st = L.bfm_sweep_noalloc(C.byref(sysd), mcs, s.seed, call * mcs * nC, stream, err, 256)
        assert st == _lib.BFM_OK, err.value.decode()
        torch.cuda.synchronize()
        got = np.stack([dx.cpu().numpy(), dy.cpu().numpy(), dz.cpu().numpy()], axis=1)[slot]
        assert np.array_equal(got, want), (s.name, call)


def test_noalloc_matches_bfm_run_on_two_calls():
    for s in (S.small_chains(), S.rings_and_free()):
        _two_calls_match_bfm_run(s, 40)


def test_noalloc_long_calls_reuse_the_step_ring():
    """3 colours x 2000 MCS = 6000 sub-steps per call, more than the 4096 entries of the staged
    sub-step ring, which is then reused from its start in stream order (no host wait)."""
    _two_calls_match_bfm_run(S.rings_and_free(), 2000)


def test_noalloc_rejects_oversized_system():
    L = _lib.load()
    sysd = _lib.NoallocSystem()
    dummy = np.zeros(8, dtype=np.int64)
    sysd.x = sysd.y = sysd.z = sysd.nbr = sysd.nnb = dummy.ctypes.data
    sysd.npad, sysd.maxc, sysd.n_colors = 8_000_000, 2, 2
    sysd.box = (C.c_uint32 * 3)(256, 256, 256)
    offs = np.array([0, 4_000_000], dtype=np.uint32)
    sizes = np.array([4_000_000, 4_000_000], dtype=np.uint32)
    forb = np.ones(512, dtype=np.uint8)
    sysd.group_offset, sysd.group_size, sysd.forbidden = offs.ctypes.data, sizes.ctypes.data, forb.ctypes.data
    err = C.create_string_buffer(256)
    st = L.bfm_sweep_noalloc(C.byref(sysd), 1, 1, 0, None, err, 256)
    assert st == _lib.BFM_ERR_INVALID_ARGUMENT
    assert b"32 MiB" in err.value
