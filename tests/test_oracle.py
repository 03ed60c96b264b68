"""The CPU oracle (oracle/bfm_oracle.cpp) checked against the reference itself and against an
independent restatement of its colouring.

Pin: tests/golden/reference_positions.json holds the final positions (SHA-256) that the reference
updater produced on a B200 for each case (make_golden.py); the oracle must reproduce every one.
"""
import json
import os

import numpy as np
import pytest

from cases import CASES, FAST, GOLDEN_JSON, fixture, positions_digest
from oracle import oracle as O
from pscbfm_b200 import systems as S


def _golden():
    with open(GOLDEN_JSON) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("name", FAST)
def test_oracle_reproduces_reference_updater(name):
    g = _golden()[name]
    build, chunks = CASES[name]
    s = build()
    assert s.n == g["n"] and s.seed == g["seed"] and chunks == g["chunks"]
    assert int(O.color(s).max()) + 1 == g["n_colors"]
    xyz, _ = O.run(s, sum(chunks))
    assert positions_digest(xyz) == g["sha256"]
    assert xyz[:4].tolist() == g["head"]


# ---------------------------------------------------------------- colouring, independent restatement

def _colour_reference_style(n, nbrs):
    """graphColoring.tpp:77-293 restated in Python with a dict standing in for std::map."""
    NONE = 255
    colors = [NONE] * n
    used_count = []
    cmap = {}
    for start in range(n):
        if colors[start] != NONE:
            continue
        todo = []
        node = start
        while True:
            for k in cmap:
                cmap[k] = False
            n_uncol, first = 0, -1
            for nb in nbrs[node]:
                c = colors[nb]
                if c != NONE:
                    cmap[c] = True
                else:
                    n_uncol += 1
                    if first == -1:
                        first = nb
            col = 0
            while col < len(cmap) and cmap.setdefault(col, False) and col < 255:
                col += 1
            assert col < 255
            colors[node] = col
            if col >= len(used_count):
                used_count += [0] * (col + 1 - len(used_count))
            used_count[col] += 1
            if n_uncol == 0 and not todo:
                break
            if n_uncol > 1:
                todo.append(node)
            node = first
            if n_uncol == 0:
                while todo:
                    node = todo[-1]
                    n2, f2 = 0, -1
                    for nb in nbrs[node]:
                        if colors[nb] == NONE:
                            n2 += 1
                            if f2 == -1:
                                f2 = nb
                    if n2 < 2:
                        todo.pop()
                    if f2 != -1:
                        node = f2
                        break
                    node = -1
                if not todo and node == -1:
                    break
    # uniform pass; the initial std::sort is an insertion sort (stable) for <= 16 colours
    assert len(used_count) <= 16
    rarest = sorted([(c, k) for c, k in enumerate(used_count)], key=lambda e: e[1])
    target = (n + len(used_count) - 1) // len(used_count)
    for node in range(n):
        if used_count[colors[node]] <= target:
            continue
        i = 0
        while i < len(rarest) and rarest[i][1] < target:
            new = rarest[i][0]
            if all(colors[nb] != new for nb in nbrs[node]):
                old = colors[node]
                used_count[old] -= 1
                used_count[new] += 1
                rarest = [(c, k - (c == old) + (c == new)) for c, k in rarest]
                rarest = sorted(rarest, key=lambda e: e[1])   # stable, like the bubble sort
                colors[node] = new
            i += 1
    return np.array(colors, dtype=np.uint8)


def _lists(s):
    return [s.nbr_ids[i, :s.nbr_count[i]].tolist() for i in range(s.n)]


@pytest.mark.parametrize("key", ["ring", "hydrogel"])
def test_colouring_reference_fixtures(key):
    s = fixture(key)
    assert np.array_equal(O.color(s), _colour_reference_style(s.n, _lists(s)))


@pytest.mark.parametrize("build", [S.rings_and_free, S.square_network, lambda: S.serpentine_chains(32, 16, 0.3),
                                   S.small_chains])
def test_colouring_generated(build):
    s = build()
    assert np.array_equal(O.color(s), _colour_reference_style(s.n, _lists(s)))


def test_colouring_branchy_random_graph():
    rng = np.random.default_rng(3)
    n = 300
    nbrs = [[] for _ in range(n)]
    for _ in range(420):
        a, b = rng.integers(0, n, 2)
        if a != b and b not in nbrs[a] and len(nbrs[a]) < 6 and len(nbrs[b]) < 6:
            nbrs[a].append(int(b))
            nbrs[b].append(int(a))
    cnt = np.array([len(x) for x in nbrs], np.uint32)
    ids = np.zeros((n, 6), np.uint32)
    for i, x in enumerate(nbrs):
        ids[i, :len(x)] = x
    s = S.BfmSystem((32, 32, 32), np.zeros((n, 3), np.int32), cnt, ids, np.ones(n, np.int32))
    col = O.color(s)
    assert np.array_equal(col, _colour_reference_style(n, nbrs))
    for i in range(n):
        assert all(col[i] != col[j] for j in nbrs[i])


# ---------------------------------------------------------------- sweep properties

def _ev_ok(xyz, box):
    L = np.array(box)
    cells = []
    for c in range(8):
        off = np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1])
        q = (xyz + off) % L
        cells.append(q[:, 0] + L[0] * (q[:, 1] + L[1] * q[:, 2]))
    allc = np.concatenate(cells)
    return np.unique(allc).size == allc.size


def _bonds_ok(s, xyz):
    r, c = s.bonds()
    return bool((s.forbidden[S.bond_index(xyz[c] - xyz[r])] == 0).all())


@pytest.mark.parametrize("build", [S.small_chains, S.rings_and_free, S.square_network, S.crosslinked_network])
def test_sweep_keeps_invariants(build):
    s = build()
    xyz, (att, tent, acc) = O.run(s, 200)
    assert _ev_ok(xyz, s.box) and _bonds_ok(s, xyz)
    # attempted = sum of the sizes of the colour groups drawn (with replacement) per sub-step
    col = O.color(s)
    sizes = np.bincount(col)
    draws = O.counter_draws(s.seed, 0, 2 * len(sizes) * 200)
    assert att == int(sizes[draws[0::2] % len(sizes)].sum())
    assert 0 < acc <= tent <= att
    assert not np.array_equal(xyz, s.xyz)


@pytest.mark.parametrize("walls", [1, 2, 4, 7])
def test_walls_keep_monomers_inside(walls):
    s = S.walled(S.serpentine_chains(32, 16, 0.3, seed=5), walls=walls)
    xyz, (att, tent, acc) = O.run(s, 300)
    assert _ev_ok(xyz, s.box) and _bonds_ok(s, xyz)
    for a in range(3):
        if (walls >> a) & 1:
            assert xyz[:, a].min() >= 0 and xyz[:, a].max() <= s.box[a] - 2
            # the walls are reached: without them the chains would spread past them
            assert xyz[:, a].min() == 0 or xyz[:, a].max() == s.box[a] - 2
    assert 0 < acc <= tent <= att
    # a periodic run of the same system differs once monomers meet the walls
    free, _ = O.run(S.walled(s, walls=0), 300)
    assert not np.array_equal(free, xyz)


@pytest.mark.parametrize("box,walls", [((48, 40, 24), 7), ((36, 64, 32), 1), ((32, 44, 64), 2), ((64, 32, 20), 4)])
def test_walled_axes_of_any_side(box, walls):
    """Walled axes take any side >= 4 (the box sits in the lowest cells of a power-of-two lattice
    side; nothing wraps there): excluded volume, the bond set and the walls hold, and the walls are
    reached."""
    s = S.walled(S.serpentine_chains(box, 16, 0.3, seed=9), walls=walls)
    xyz, (att, tent, acc) = O.run(s, 300)
    assert _ev_ok(xyz, s.box) and _bonds_ok(s, xyz)
    for a in range(3):
        if (walls >> a) & 1:
            assert xyz[:, a].min() >= 0 and xyz[:, a].max() <= s.box[a] - 2
            assert xyz[:, a].min() == 0 or xyz[:, a].max() == s.box[a] - 2
    assert 0 < acc <= tent <= att


def test_periodic_axis_needs_a_power_of_two():
    s = S.walled(S.serpentine_chains((48, 32, 32), 16, 0.3, seed=9), walls=2)   # x periodic, 48
    with pytest.raises(RuntimeError, match="powers of two"):
        O.run(s, 1)


def test_monomer_outside_walls_rejected():
    s = S.walled(S.serpentine_chains(32, 16, 0.3, seed=5), walls=1)
    s.xyz = s.xyz.copy()
    s.xyz[3, 0] = 31          # corner at L-1: the cube would stick out
    with pytest.raises(RuntimeError, match="outside the walls"):
        O.run(s, 1)


def test_chunked_run_equals_single_run():
    s = S.rings_and_free()
    nc = int(O.color(s).max()) + 1
    full, _ = O.run(s, 50)
    part, _ = O.run(s, 20)
    s2 = S.BfmSystem(s.box, part.astype(np.int32), s.nbr_count, s.nbr_ids, s.attributes, s.forbidden, seed=s.seed)
    rest, _ = O.run(s2, 30, substep0=20 * nc)
    assert np.array_equal(rest, full)


def test_explicit_draws_equal_counter_stream():
    s = S.small_chains()
    a, sa = O.run(s, 40)
    d = O.counter_draws(s.seed, 0, 2 * 2 * 40)
    b, sb = O.run(s, 40, draws=d)
    assert np.array_equal(a, b) and sa == sb
    with pytest.raises(RuntimeError):
        O.run(s, 41, draws=d)


def test_hash_restatement():
    def h(a):
        M = 0xFFFFFFFF
        a = ((a + 0x7ed55d16) + (a << 12)) & M
        a = ((a ^ 0xc761c23c) ^ (a >> 19)) & M
        a = ((a + 0x165667b1) + (a << 5)) & M
        a = ((a + 0xd3a2646c) ^ (a << 9)) & M
        a = ((a + 0xfd7046c5) + (a << 3)) & M
        a = ((a ^ 0xb55a4f09) ^ (a >> 16)) & M
        return a
    for v in [0, 1, 2, 12345, 0xFFFFFFFF, 0x80000000]:
        assert O.move_hash(v) == h(v)


def test_wrong_bond_set_rejected():
    s = S.small_chains()
    s.forbidden = s.forbidden.copy()
    s.forbidden[S.bond_index(np.array([3, 1, 0]))] = 1
    with pytest.raises(RuntimeError, match="Expected 108 allowed bonds"):
        O.run(s, 1)


def test_sequential_baseline_invariants():
    s = S.small_chains()
    xyz, (att, acc) = O.seq_run(s, 50, seed=1)
    assert att == 50 * s.n and 0 < acc < att
    assert _ev_ok(xyz, s.box) and _bonds_ok(s, xyz)


def test_oracle_observables_basics():
    s = S.small_chains()
    raw = O.observables(s, s.xyz, s.xyz)
    m = 256
    assert raw.size == 5 * m + 513
    assert raw[5 * m + 512] == 0                       # no displacement
    assert raw[5 * m:5 * m + 512].sum() == s.nbr_count.sum()
    # straight chains of 32 with bond (2,0,0): Ree^2 = 62^2
    assert (raw[4 * m:5 * m] == 62 ** 2).all()


def _chain_statistics(s, run, n_blocks=40, block=100, skip=10):
    """Block means of <Ree^2>, <Rg^2> and <b^2> over the chains of s (consecutive ids) after the
    first `skip` blocks."""
    import dataclasses
    mol = O.molecules(s)
    m = int(mol.max()) + 1
    cur, ree, rg, b2 = s, [], [], []
    for b in range(n_blocks):
        xyz = run(cur, block, b)
        cur = dataclasses.replace(cur, xyz=xyz.astype(np.int32))
        c = xyz.astype(np.float64).reshape(m, s.n // m, 3)
        ree.append(((c[:, -1] - c[:, 0]) ** 2).sum(1).mean())
        rg.append(((c - c.mean(1, keepdims=True)) ** 2).sum(2).mean())
        b2.append((np.diff(c, axis=1) ** 2).sum(2).mean())
    return [float(np.mean(v[skip:])) for v in (ree, rg, b2)]


def test_parallel_sweep_samples_like_the_serial_updater():
    """The colour-by-colour parallel sweep and the random-sequential serial updater (the CPU
    baseline) are different Markov chains with the same equilibrium: their chain statistics agree
    within statistical error (not bit for bit)."""
    s = S.serpentine_chains(32, 16, 0.3, seed=5)
    par = _chain_statistics(s, lambda cur, k, b: O.run(cur, k, seed=1000 + b)[0])
    seq = _chain_statistics(s, lambda cur, k, b: O.seq_run(cur, k, seed=2000 + b)[0])
    for name, p, q, tol in zip(("Ree2", "Rg2", "b2"), par, seq, (0.08, 0.08, 0.01)):
        assert abs(p - q) <= tol * q, (name, p, q)
    # and far from the straight initial chains (Ree^2 = (2 (16-1))^2 = 900)
    assert par[0] < 400


def test_oracle_reproduces_reference_at_full_ensemble_length():
    """The smallest ensemble systems after their full 10^4 MCS: the oracle ends where the reference
    updater does (tests/golden/reference_long.json, make_golden.py --long)."""
    from cases import LONG_JSON, ENSEMBLE_MCS, ensemble_case, ensemble_cases
    if not os.path.exists(LONG_JSON):
        pytest.fail("tests/golden/reference_long.json is missing (make_golden.py --long)")
    gold = json.load(open(LONG_JSON))["cases"]
    names = list(ensemble_cases())
    sizes = sorted(range(len(names)), key=lambda i: gold[names[i]]["n"])
    for i in sizes[:4]:
        s = ensemble_case(i)
        g = gold[names[i]]
        assert s.n == g["n"] and s.seed == g["seed"]
        xyz, _ = O.run(s, ENSEMBLE_MCS)
        assert positions_digest(xyz) == g["sha256"], names[i]
