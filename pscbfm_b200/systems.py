"""Synthetic BFM systems: the standard bond set and the straight-chain, network and ensemble
layouts the sweep is measured on.

A system is a box (periodic axes of power-of-two side, or walls along chosen axes of any side),
int32 monomer corner positions (unfolded), directed neighbour lists in the order a
LeMonADE-style caller would pass them to ``setConnectivity`` (for every bond (a, b) in creation
order: b is appended to a's list and a to b's list), integer attributes and the 512-entry forbidden-bond table indexed like
``linearizeBondVectorIndex`` (src/pscbfm/CRITICAL.cu:243-261).

No public dataset is involved: every layout is generated deterministically from its sizes.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from itertools import permutations, product

import numpy as np

__all__ = [
    "BfmSystem", "standard_bond_vectors", "forbidden_table", "bond_index",
    "small_chains", "dense_melt", "crosslinked_network", "serpentine_chains",
    "ensemble_params", "ensemble", "from_bonds",
]


def standard_bond_vectors() -> np.ndarray:
    """The 108 allowed bond vectors: every sign/permutation of (2,0,0), (2,1,0), (2,1,1),
    (2,2,1), (3,0,0), (3,1,0) (the set src/pscbfm/UpdaterGPUScBFM_AB_Type.cu:521 demands)."""
    out = set()
    for base in [(2, 0, 0), (2, 1, 0), (2, 1, 1), (2, 2, 1), (3, 0, 0), (3, 1, 0)]:
        for p in permutations(base):
            for s in product((1, -1), repeat=3):
                out.add((p[0] * s[0], p[1] * s[1], p[2] * s[2]))
    v = np.array(sorted(out), dtype=np.int32)
    assert v.shape == (108, 3)
    return v


def bond_index(d: np.ndarray) -> np.ndarray:
    d = np.asarray(d, dtype=np.int64)
    return ((d[..., 0] & 7) | ((d[..., 1] & 7) << 3) | ((d[..., 2] & 7) << 6)).astype(np.int64)


def forbidden_table(allowed: np.ndarray | None = None) -> np.ndarray:
    """512-entry table, 1 = forbidden, filled for (dx,dy,dz) in [-4,3]^3 as the LeMonADE adapter
    does (src/pscbfm/GPUScBFM_AB_Type.h:120-127)."""
    if allowed is None:
        allowed = standard_bond_vectors()
    t = np.ones(512, dtype=np.uint8)
    t[bond_index(allowed)] = 0
    return t


@dataclass
class BfmSystem:
    box: tuple
    xyz: np.ndarray            # (n, 3) int32
    nbr_count: np.ndarray      # (n,) uint32
    nbr_ids: np.ndarray        # (n, maxc) uint32
    attributes: np.ndarray     # (n,) int32
    forbidden: np.ndarray = field(default_factory=forbidden_table)
    name: str = ""
    seed: int = 0
    periodic: tuple = (True, True, True)   # an axis that is not periodic has walls at 0 and L-1

    @property
    def n(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def walls(self) -> int:
        """Bit a set: axis a is not periodic."""
        return sum(1 << a for a in range(3) if not self.periodic[a])

    @property
    def maxc(self) -> int:
        return int(self.nbr_ids.shape[1])

    def volume_fraction(self) -> float:
        return 8.0 * self.n / float(np.prod(self.box))

    def bonds(self):
        """(i, j) pairs of directed neighbour entries, list order."""
        rows = np.repeat(np.arange(self.n), self.nbr_count)
        mask = np.arange(self.maxc)[None, :] < self.nbr_count[:, None]
        return rows, self.nbr_ids[mask]


def from_bonds(box, xyz, bonds, attributes=None, maxc=None, name="", seed=0) -> BfmSystem:
    """Build neighbour lists from an ordered bond list (a, b): b is appended to a's list and a to b's."""
    xyz = np.ascontiguousarray(xyz, dtype=np.int32)
    n = xyz.shape[0]
    bonds = np.asarray(bonds, dtype=np.int64).reshape(-1, 2)
    # interleave (a->b, b->a) in creation order, then stable-sort by owner
    owners = np.empty(2 * len(bonds), dtype=np.int64)
    targets = np.empty(2 * len(bonds), dtype=np.int64)
    owners[0::2], targets[0::2] = bonds[:, 0], bonds[:, 1]
    owners[1::2], targets[1::2] = bonds[:, 1], bonds[:, 0]
    order = np.argsort(owners, kind="stable")
    owners, targets = owners[order], targets[order]
    count = np.bincount(owners, minlength=n).astype(np.uint32)
    if maxc is None:
        maxc = max(int(count.max()) if n else 0, 1)
    if n and int(count.max()) > maxc:
        raise ValueError("connectivity exceeds maxc")
    start = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(count, out=start[1:])
    slot = np.arange(len(owners)) - start[owners]
    ids = np.zeros((n, maxc), dtype=np.uint32)
    ids[owners, slot] = targets
    if attributes is None:
        attributes = np.ones(n, dtype=np.int32)
    return BfmSystem(tuple(int(b) for b in box), xyz, count, ids,
                     np.asarray(attributes, dtype=np.int32), forbidden_table(), name, seed)


def _straight_chains(L, n_chains, chain_len, spacing, offset_rule):
    """Chains along +x with bond (2,0,0); chain k starts at grid point (a, b) = divmod(k, G) in
    (y, z) with the given spacing; its x offset comes from offset_rule(a)."""
    G = L // spacing
    k = np.arange(n_chains)
    a, b = k // G, k % G
    x0 = offset_rule(a)
    j = np.arange(chain_len)
    x = (x0[:, None] + 2 * j[None, :]).reshape(-1)
    y = np.repeat(spacing * a, chain_len)
    z = np.repeat(spacing * b, chain_len)
    xyz = np.stack([x, y, z], axis=1).astype(np.int32)
    ids = (k[:, None] * chain_len + j[None, :-1]).reshape(-1)
    bonds = np.stack([ids, ids + 1], axis=1)
    return xyz, bonds


def small_chains() -> BfmSystem:
    """Periodic 64^3, 256 chains x 32 monomers (N = 8192, phi = 0.25). Starts on a 16x16 (y, z)
    grid with spacing 4; chains in odd y rows start at x = 32, the others at x = 0."""
    L = 64
    xyz, bonds = _straight_chains(L, 256, 32, 4, lambda a: np.where(a % 2 == 1, 32, 0))
    return from_bonds((L, L, L), xyz, bonds, name="chains64_256x32", seed=42)


def dense_melt() -> BfmSystem:
    """Periodic 256^3, 16384 chains x 64 monomers (N = 1,048,576, phi = 0.5). Starts on a
    128x128 (y, z) grid with spacing 2; chains in odd y rows start at x = 128."""
    L = 256
    xyz, bonds = _straight_chains(L, 16384, 64, 2, lambda a: np.where(a % 2 == 1, 128, 0))
    return from_bonds((L, L, L), xyz, bonds, name="melt256_16384x64", seed=7)


def crosslinked_network() -> BfmSystem:
    """Periodic 128^3 network: 512 six-functional nodes (attribute 1) on an 8^3 grid with
    spacing 16; each node is linked to its +x, +y, +z neighbour (periodic) by a strand of 7
    monomers (attribute 2) with axis bonds of length 2. N = 11,264.

    Node (i, j, k) has id 64 i + 8 j + k. The strand from node n along axis a has ids
    512 + 7 (3 n + a) + m, m = 0..6. Bonds are created strand by strand, node to node."""
    L, G, S = 128, 8, 16
    nodes = np.array([(i, j, k) for i in range(G) for j in range(G) for k in range(G)], dtype=np.int64)
    xyz = [nodes * S]
    bonds = []
    nid = lambda i, j, k: 64 * (i % G) + 8 * (j % G) + (k % G)
    strand_xyz = np.zeros((G ** 3 * 3 * 7, 3), dtype=np.int64)
    for n_, (i, j, k) in enumerate(nodes):
        for a in range(3):
            base = 512 + 7 * (3 * n_ + a)
            step = np.zeros(3, dtype=np.int64)
            step[a] = 2
            for m in range(7):
                strand_xyz[base - 512 + m] = nodes[n_] * S + step * (m + 1)
            nxt = [i, j, k]
            nxt[a] += 1
            chain = [n_] + list(range(base, base + 7)) + [nid(*nxt)]
            bonds.extend(zip(chain[:-1], chain[1:]))
    xyz = np.concatenate([xyz[0], strand_xyz]) % L
    attrs = np.concatenate([np.ones(512, np.int32), np.full(len(strand_xyz), 2, np.int32)])
    return from_bonds((L, L, L), xyz, bonds, attributes=attrs, maxc=8, name="network128_512x6", seed=3)


def serpentine_chains(L, chain_len: int, phi: float, name: str = "", seed: int = 0) -> BfmSystem:
    """Periodic box (L^3 for an int L, Lx x Ly x Lz for a 3-tuple) with floor(phi V / (8 chain_len))
    linear chains (at least one), V the box volume.

    Monomer slots are the points of the lattice 2Z^3 inside the box, visited by a boustrophedon
    path (x fastest, rows reversing, layers reversing) whose consecutive slots are one axis bond
    of length 2 apart. Chain c occupies chain_len consecutive slots starting at slot
    floor(c P / n_chains), P the number of slots, so chains longer than the box fold instead of
    overlapping themselves."""
    box = (L, L, L) if np.isscalar(L) else tuple(int(v) for v in L)
    hx, hy, hz = (v // 2 for v in box)
    P = hx * hy * hz
    n_chains = max(1, int(np.floor(phi * box[0] * box[1] * box[2] / (8 * chain_len))))
    if n_chains * chain_len > P:
        raise ValueError("system does not fit")
    s = np.arange(P, dtype=np.int64)
    zc, rem = s // (hx * hy), s % (hx * hy)
    yr = rem // hx
    yc = np.where(zc % 2 == 0, yr, hy - 1 - yr)
    xr = rem % hx
    row = zc * hy + yr                     # running row count keeps the x direction alternating
    xc = np.where(row % 2 == 0, xr, hx - 1 - xr)
    path = np.stack([2 * xc, 2 * yc, 2 * zc], axis=1)
    starts = (np.arange(n_chains, dtype=np.int64) * P) // n_chains
    slots = (starts[:, None] + np.arange(chain_len)[None, :]).reshape(-1)
    xyz = path[slots].astype(np.int32)
    ids = (np.arange(n_chains)[:, None] * chain_len + np.arange(chain_len - 1)[None, :]).reshape(-1)
    bonds = np.stack([ids, ids + 1], axis=1)
    tag = f"{box[0]}" if box[0] == box[1] == box[2] else "x".join(str(v) for v in box)
    return from_bonds(box, xyz, bonds, name=name or f"serp{tag}_{n_chains}x{chain_len}", seed=seed)


def walled(s: BfmSystem, walls: int = 7, name: str = "") -> BfmSystem:
    """A copy of s with walls along the axes of the bit mask `walls` (bit a: axis a not periodic).
    Every corner must already lie in [0, L-2] along those axes."""
    import dataclasses
    periodic = tuple(not (walls >> a) & 1 for a in range(3))
    for a in range(3):
        if (walls >> a) & 1 and (s.xyz[:, a].min() < 0 or s.xyz[:, a].max() > s.box[a] - 2):
            raise ValueError(f"monomers outside the walls along axis {a}")
    return dataclasses.replace(s, periodic=periodic, name=name or s.name + f"_walls{walls}")


_RING3 = [(0, 0, 0), (2, 0, 0), (1, 2, 0)]
_RING5 = [(0, 0, 0), (2, 0, 0), (3, 2, 0), (1, 3, 0), (-1, 2, 0)]


def rings_and_free(L: int = 32, spacing: int = 8, free_per_cell: int = 1, seed: int = 11) -> BfmSystem:
    """Odd rings (3 and 5 monomers, which need three colours) on a grid of cells with the given
    spacing, alternating per cell, plus `free_per_cell` unbonded monomers per cell (these let the
    uniform colour pass move monomers between colours)."""
    xyz, bonds, attrs = [], [], []
    g = L // spacing
    cell = 0
    for i in range(g):
        for j in range(g):
            for k in range(g):
                base = np.array([i, j, k]) * spacing + 1
                ring = _RING3 if cell % 2 == 0 else _RING5
                start = len(xyz)
                for p in ring:
                    xyz.append(base + np.array(p) + np.array([1, 0, 0]))
                    attrs.append(1)
                for m in range(len(ring)):
                    bonds.append((start + m, start + (m + 1) % len(ring)))
                for f in range(free_per_cell):
                    xyz.append(base + np.array([0, 5, 2 + 2 * f]))
                    attrs.append(2)
                cell += 1
    return from_bonds((L, L, L), np.array(xyz), bonds, attributes=np.array(attrs), name=f"rings{L}", seed=seed)


def square_network(L: int = 64, spacing: int = 16, strand: int = 7, seed: int = 5) -> BfmSystem:
    """Four-functional network: nodes on a (L/spacing)^3 grid linked along +x and +y (periodic) by
    strands of `strand` monomers with axis bonds of length 2 (spacing = 2 (strand + 1))."""
    assert spacing == 2 * (strand + 1)
    G = L // spacing
    nodes = [(i, j, k) for i in range(G) for j in range(G) for k in range(G)]
    nid = {n: t for t, n in enumerate(nodes)}
    xyz = [np.array(n) * spacing for n in nodes]
    bonds = []
    for n in nodes:
        for a in range(2):
            step = np.zeros(3, dtype=np.int64)
            step[a] = 2
            start = len(xyz)
            for m in range(strand):
                xyz.append(np.array(n) * spacing + step * (m + 1))
            nxt = list(n)
            nxt[a] = (nxt[a] + 1) % G
            chain = [nid[n]] + list(range(start, start + strand)) + [nid[tuple(nxt)]]
            bonds.extend(zip(chain[:-1], chain[1:]))
    return from_bonds((L, L, L), np.array(xyz) % L, bonds, name=f"sqnet{L}", seed=seed)


def ensemble_params(n_systems: int = 256, gen_seed: int = 20240611):
    """Per-system (L, chain_len, phi) draws of the batched ensemble: L uniform on {32, 64, 128},
    chain length uniform on {16, 32, 64, 128, 256}, phi uniform on [0.1, 0.5]."""
    rng = np.random.Generator(np.random.PCG64(gen_seed))
    Ls = rng.choice([32, 64, 128], size=n_systems)
    lcs = rng.choice([16, 32, 64, 128, 256], size=n_systems)
    phis = rng.uniform(0.1, 0.5, size=n_systems)
    return [(int(a), int(b), float(c)) for a, b, c in zip(Ls, lcs, phis)]


def ensemble(n_systems: int = 256, base_seed: int = 1000, gen_seed: int = 20240611):
    """The batched ensemble: system i has seed base_seed + i and the layout of serpentine_chains."""
    out = []
    for i, (L, lc, phi) in enumerate(ensemble_params(n_systems, gen_seed)):
        out.append(serpentine_chains(L, lc, phi, name=f"ens{i}_L{L}_lc{lc}", seed=base_seed + i))
    return out
