"""LeMonADE-style .bfm reader and writer (the format of the reference's tests/*.bfm files).

Layout, as the reference fixtures show it:
  - '#' lines are comments; commands start with '!'.
  - !number_of_monomers=N, !box_x= / !box_y= / !box_z=, !periodic_x= / _y= / _z= (0 or 1)
  - !bonds, then lines "a b" (1-based) of bonds not implied by the chain lines, up to a blank line
  - !set_of_bondvectors, then lines "dx dy dz:code" (code = ASCII value of a one-character bond
    code), up to a blank line
  - !attributes, then lines "a-b:v" (1-based ranges), up to a blank line
  - !mcs=K, then one line per chain: "x y z" of its first monomer, one space, then one character
    per further monomer giving the bond vector to it (a code may itself be a space). Monomers
    are numbered in order of appearance. A file may hold several !mcs frames; the last is read.

Neighbour-list order on reading: the explicit !bonds links first (file order), then the chain
links in reading order; each link (a, b) appends b to a's list and a to b's.

The engine adds one comment to the header it writes, "#!bfm_b200 substep=T seed=S", the position
of the counter draw stream, so that a run resumed from the file is bit-continuous.
"""
from __future__ import annotations

import re

import numpy as np

from .systems import BfmSystem, forbidden_table, from_bonds, standard_bond_vectors

_CHAIN = re.compile(r"^(-?\d+) (-?\d+) (-?\d+)(?: (.*))?$")


def _sections(lines):
    """Yields (command, value, body_lines) for every '!' command."""
    i = 0
    n = len(lines)
    while i < n:
        ln = lines[i]
        if ln.startswith("!"):
            cmd, _, val = ln[1:].partition("=")
            body = []
            j = i + 1
            while j < n and lines[j].strip() != "" and not lines[j].startswith("!"):
                if not lines[j].startswith("#"):
                    body.append(lines[j])
                j += 1
            yield cmd.strip(), val.strip(), body
            i = j
        else:
            i += 1


def read_bfm(path: str, seed: int = 0):
    """Returns (system, info) for the last conformation in the file. info holds the periodicity,
    the MCS of the frame and the engine's draw-stream position if the file has one."""
    with open(path, "r", encoding="latin-1") as f:
        lines = [ln.rstrip("\n").rstrip("\r") for ln in f]
    info = {"periodic": [True, True, True], "mcs": 0, "substep": 0, "seed": seed}
    for ln in lines:
        m = re.match(r"^#!bfm_b200 substep=(\d+) seed=(\d+)", ln)
        if m:
            info["substep"], info["seed"] = int(m.group(1)), int(m.group(2))
    n = None
    box = [0, 0, 0]
    extra = []
    codes = {}
    attrs = None
    frame = None
    for cmd, val, body in _sections(lines):
        if cmd == "number_of_monomers":
            n = int(val)
            attrs = np.zeros(n, dtype=np.int32)
        elif cmd in ("box_x", "box_y", "box_z"):
            box["xyz".index(cmd[-1])] = int(val)
        elif cmd in ("periodic_x", "periodic_y", "periodic_z"):
            info["periodic"]["xyz".index(cmd[-1])] = bool(int(val))
        elif cmd == "bonds":
            for b in body:
                a, c = b.split()[:2]
                extra.append((int(a) - 1, int(c) - 1))
        elif cmd == "set_of_bondvectors":
            for b in body:
                vec, code = b.rsplit(":", 1)
                codes[chr(int(code))] = tuple(int(v) for v in vec.split())
        elif cmd == "attributes":
            for b in body:
                rng, v = b.split(":")
                lo, hi = rng.split("-")
                attrs[int(lo) - 1:int(hi)] = int(v)
        elif cmd == "mcs":
            frame = (int(val), body)
    if n is None or frame is None:
        raise ValueError(f"{path}: no !number_of_monomers or no !mcs frame")
    info["mcs"] = frame[0]
    xyz = np.zeros((n, 3), dtype=np.int64)
    chain_bonds = []
    k = 0
    for ln in frame[1]:
        m = _CHAIN.match(ln)
        if not m:
            raise ValueError(f"{path}: bad conformation line {ln!r}")
        p = np.array([int(m.group(1)), int(m.group(2)), int(m.group(3))])
        if k >= n:
            raise ValueError(f"{path}: more monomers than declared")
        xyz[k] = p
        k += 1
        for ch in (m.group(4) or ""):
            if ch not in codes:
                raise ValueError(f"{path}: unknown bond code {ch!r}")
            p = p + np.array(codes[ch])
            xyz[k] = p
            chain_bonds.append((k - 1, k))
            k += 1
    if k != n:
        raise ValueError(f"{path}: frame has {k} monomers, header says {n}")
    allowed = np.array(sorted(set(codes.values())), dtype=np.int32) if codes else standard_bond_vectors()
    s = from_bonds(tuple(box), xyz, extra + chain_bonds, attributes=attrs, name=path.rsplit("/", 1)[-1],
                   seed=info["seed"])
    s.forbidden = forbidden_table(allowed)
    s.periodic = tuple(bool(p) for p in info["periodic"])
    info["bond_vectors"] = codes
    return s, info


def _default_codes():
    vecs = standard_bond_vectors()
    return {tuple(int(c) for c in v): chr(17 + i) for i, v in enumerate(vecs)}


def write_bfm(path: str, system: BfmSystem, mcs: int = 0, xyz=None, substep: int | None = None,
              seed: int | None = None, periodic=None):
    """Writes one frame. Chain lines follow bonds between consecutive ids whose vector has a code;
    every other bond goes to !bonds. The periodicity is the system's unless given."""
    xyz = np.asarray(system.xyz if xyz is None else xyz, dtype=np.int64)
    if periodic is None:
        periodic = system.periodic
    n = system.n
    allowed = [tuple(int(c) for c in v) for v in standard_bond_vectors()]
    forb = system.forbidden
    vecs = [v for v in allowed if not forb[(v[0] & 7) | ((v[1] & 7) << 3) | ((v[2] & 7) << 6)]]
    code_of = {v: chr(17 + i) for i, v in enumerate(vecs)}
    rows, cols = system.bonds()
    pairs = {(int(min(a, b)), int(max(a, b))) for a, b in zip(rows, cols)}
    chain_link = np.zeros(n, dtype=bool)       # chain_link[i]: i continues the line of i-1
    for i in range(1, n):
        if (i - 1, i) in pairs and tuple(int(v) for v in (xyz[i] - xyz[i - 1])) in code_of:
            chain_link[i] = True
    extra = sorted(p for p in pairs if not (p[1] == p[0] + 1 and chain_link[p[1]]))
    out = ["#!version=2.0", "#Bond Fluctuation Model - simulation data file", "#monomer numbering starts at 1"]
    if substep is not None:
        out.append(f"#!bfm_b200 substep={int(substep)} seed={int(system.seed if seed is None else seed)}")
    out += ["", f"!number_of_monomers={n}", "", "!bonds"]
    out += [f"{a + 1} {b + 1}" for a, b in extra]
    out += ["", f"!box_x={system.box[0]}", "", f"!box_y={system.box[1]}", "", f"!box_z={system.box[2]}", ""]
    for ax, p in zip("xyz", periodic):
        out += [f"!periodic_{ax}={int(bool(p))}", ""]
    out.append("!set_of_bondvectors")
    out += [f"{v[0]} {v[1]} {v[2]}:{ord(c)}" for v, c in code_of.items()]
    out += ["", "!attributes"]
    a = system.attributes
    start = 0
    for i in range(1, n + 1):
        if i == n or a[i] != a[start]:
            out.append(f"{start + 1}-{i}:{int(a[start])}")
            start = i
    out += ["", f"!mcs={int(mcs)}"]
    i = 0
    while i < n:
        line = f"{xyz[i][0]} {xyz[i][1]} {xyz[i][2]}"
        codes = []
        j = i + 1
        while j < n and chain_link[j]:
            codes.append(code_of[tuple(int(v) for v in (xyz[j] - xyz[j - 1]))])
            j += 1
        out.append(line + (" " + "".join(codes) if codes else ""))
        i = j
    out.append("")
    with open(path, "w", encoding="latin-1") as f:
        f.write("\n".join(out) + "\n")
