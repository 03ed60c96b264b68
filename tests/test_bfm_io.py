"""The .bfm reader and writer (LeMonADE's file format): write -> read keeps the box, positions, bond
sets, bond table and attributes; the checkpoint header resumes the counter draw stream so that a
run split at a checkpoint equals the run straight through (oracle, on the CPU)."""
import numpy as np
import pytest

from cases import fixture
from oracle import oracle as O
from pscbfm_b200 import bfm_io
from pscbfm_b200 import systems as S


def _pairs(s):
    rows, cols = s.bonds()
    return {(int(min(a, b)), int(max(a, b))) for a, b in zip(rows, cols)}


def _nbr_sets(s):
    return [set(int(v) for v in s.nbr_ids[i, :s.nbr_count[i]]) for i in range(s.n)]


SYSTEMS = {
    "ring": lambda: fixture("ring"),
    "hydrogel": lambda: fixture("hydrogel"),
    "linear_chains": lambda: fixture("linear_chains"),
    "network": S.crosslinked_network,
    "rings_and_free": S.rings_and_free,
    "serpentine": lambda: S.serpentine_chains(32, 64, 0.4, seed=5),
    # walled axes of sides that are not powers of two
    "walled_48x40x24": lambda: S.walled(S.serpentine_chains((48, 40, 24), 16, 0.3, seed=7), walls=7),
}


@pytest.mark.parametrize("key", list(SYSTEMS))
def test_round_trip(key, tmp_path):
    s = SYSTEMS[key]()
    p = str(tmp_path / f"{key}.bfm")
    bfm_io.write_bfm(p, s, mcs=123)
    r, info = bfm_io.read_bfm(p)
    assert info["mcs"] == 123
    assert tuple(r.box) == tuple(s.box)
    assert tuple(r.periodic) == tuple(s.periodic)
    assert np.array_equal(r.xyz, s.xyz)
    assert _pairs(r) == _pairs(s)
    assert _nbr_sets(r) == _nbr_sets(s)
    assert np.array_equal(r.forbidden, s.forbidden)
    assert np.array_equal(r.attributes, s.attributes)


def test_several_frames_last_wins(tmp_path):
    s = S.small_chains()
    moved, _ = O.run(s, 5)
    a, b = str(tmp_path / "a.bfm"), str(tmp_path / "b.bfm")
    bfm_io.write_bfm(a, s, mcs=0)
    bfm_io.write_bfm(b, s, mcs=5, xyz=moved)
    # a second !mcs frame appended to the first file, as LeMonADE's writers do
    frame = open(b).read().split("!mcs=5", 1)[1]
    with open(a, "a") as f:
        f.write("!mcs=5" + frame)
    r, info = bfm_io.read_bfm(a)
    assert info["mcs"] == 5 and np.array_equal(r.xyz, moved)


def test_malformed_files_rejected(tmp_path):
    s = S.rings_and_free()
    p = str(tmp_path / "x.bfm")
    bfm_io.write_bfm(p, s)
    txt = open(p).read()
    bad = tmp_path / "bad.bfm"
    bad.write_text(txt.replace(f"!number_of_monomers={s.n}", f"!number_of_monomers={s.n + 1}"))
    with pytest.raises(ValueError, match="monomers"):
        bfm_io.read_bfm(str(bad))
    bad.write_text(txt.replace("!mcs=0", "!nothing=0"))
    with pytest.raises(ValueError, match="frame"):
        bfm_io.read_bfm(str(bad))


@pytest.mark.parametrize("key", ["linear_chains", "network", "rings_and_free"])
def test_checkpoint_resume_is_bit_continuous(key, tmp_path):
    import dataclasses
    s = SYSTEMS[key]()
    nc = int(O.color(s).max()) + 1
    straight, _ = O.run(s, 50)
    first, _ = O.run(s, 30)
    p = str(tmp_path / "ck.bfm")
    bfm_io.write_bfm(p, s, mcs=30, xyz=first, substep=30 * nc, seed=s.seed)
    r, info = bfm_io.read_bfm(p)
    assert info["substep"] == 30 * nc and info["seed"] == s.seed and info["mcs"] == 30
    # positions from the file, neighbour-list order from the original system
    resumed, _ = O.run(dataclasses.replace(s, xyz=r.xyz.astype(np.int32)), 20, seed=info["seed"],
                       substep0=info["substep"])
    assert np.array_equal(resumed, straight)


def test_file_neighbour_order_is_stable(tmp_path):
    """A system read from a file, written and read again, has the same neighbour lists in the same
    order, so checkpoints of file-loaded systems resume bit-exactly from the file alone."""
    s = SYSTEMS["rings_and_free"]()
    a, b = str(tmp_path / "a.bfm"), str(tmp_path / "b.bfm")
    bfm_io.write_bfm(a, s)
    r1, _ = bfm_io.read_bfm(a)
    bfm_io.write_bfm(b, r1)
    r2, _ = bfm_io.read_bfm(b)
    assert np.array_equal(r1.nbr_count, r2.nbr_count) and np.array_equal(r1.nbr_ids, r2.nbr_ids)
    assert np.array_equal(O.color(r1), O.color(r2))
