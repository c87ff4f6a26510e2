"""LeMonADE .bfm conformation files and .seeds files (Python side).

Same format as the C++ reader/writer of the pscbfm command-line simulator
(pscbfm_b200/csrc/bfm_io.hpp): header keys !number_of_monomers, !box_*,
!periodic_*, !set_of_bondvectors ("dx dy dz:id"), !attributes ("a-b:c"),
!bonds ("a b", 1-based) and !mcs=AGE frames where each line holds "x y z",
one space and one byte (a bond vector id) per further monomer of the chain.
The reader returns the last frame.
"""
from __future__ import annotations

import numpy as np

from .systems import BONDS_108, System, allowed_table


def standard_bond_ids():
    """The 108 vectors with ids 17..124, in the order the C++ writer uses."""
    out = {}
    i = 17
    for dx in range(-3, 4):
        for dy in range(-3, 4):
            for dz in range(-3, 4):
                a = sorted((abs(dx), abs(dy), abs(dz)))
                if tuple(a) in ((0, 0, 2), (0, 1, 2), (1, 1, 2), (0, 0, 3), (0, 1, 3), (1, 2, 2)):
                    out[i] = (dx, dy, dz)
                    i += 1
    return out


def read_bfm(path):
    """(System, age) of the last !mcs frame of a .bfm file."""
    raw = open(path, "rb").read().split(b"\n")
    lines = [l[:-1] if l.endswith(b"\r") else l for l in raw]
    n = 0
    box = [0, 0, 0]
    periodic = [True, True, True]
    last = None
    for k, l in enumerate(lines):
        s = l.decode("latin-1")
        for key, setter in (("!number_of_monomers=", None), ("!box_x=", 0), ("!box_y=", 1), ("!box_z=", 2)):
            if s.startswith(key):
                v = int(s[len(key):])
                if setter is None:
                    n = v
                else:
                    box[setter] = v
        for a, key in enumerate(("!periodic_x=", "!periodic_y=", "!periodic_z=")):
            if s.startswith(key):
                periodic[a] = int(s[len(key):]) != 0
        if s.startswith("!mcs"):
            last = k
    if n == 0 or last is None:
        raise ValueError(f"{path}: missing !number_of_monomers or !mcs")
    ids, attrs, bonds = {}, np.zeros(n, np.int32), []
    k = 0
    while k < len(lines):
        s = lines[k].decode("latin-1")
        if s in ("!set_of_bondvectors", "!attributes", "!bonds"):
            k += 1
            while k < len(lines) and lines[k] and not lines[k].startswith(b"!"):
                t = lines[k].decode("latin-1")
                if s == "!set_of_bondvectors":
                    vec, i = t.split(":")
                    ids[int(i)] = tuple(int(v) for v in vec.split())
                elif s == "!attributes":
                    rng, v = t.split(":")
                    a, b = (int(x) for x in rng.split("-"))
                    attrs[a - 1:b] = int(v)
                else:
                    a, b = (int(x) for x in t.split())
                    bonds.append((a - 1, b - 1))
                k += 1
            continue
        k += 1
    age_s = lines[last].decode("latin-1")
    age = int(age_s.split("=", 1)[1]) if "=" in age_s else 0
    pos = np.zeros((n, 3), np.int64)
    m = 0
    pairs = []
    for l in lines[last + 1:]:
        if not l or l.startswith(b"!"):
            break
        parts = l.split(b" ", 3)
        x, y, z = int(parts[0]), int(parts[1]), int(parts[2])
        pos[m] = (x, y, z)
        m += 1
        if len(parts) > 3:
            for byte in parts[3]:
                d = ids[byte]
                x, y, z = x + d[0], y + d[1], z + d[2]
                pos[m] = (x, y, z)
                pairs.append((m - 1, m))
                m += 1
    if m != n:
        raise ValueError(f"{path}: frame holds {m} monomers, expected {n}")
    deg = np.zeros(n, np.uint8)
    nbr = np.zeros((n, 8), np.uint32)
    for a, b in pairs + bonds:
        nbr[a, deg[a]] = b
        deg[a] += 1
        nbr[b, deg[b]] = a
        deg[b] += 1
    allowed = allowed_table(np.array(list(ids.values()), dtype=np.int32)) if ids else allowed_table(BONDS_108)
    sys_ = System(tuple(box), pos.astype(np.int32), deg, nbr, allowed, attributes=attrs)
    sys_.periodic = tuple(periodic)
    return sys_, age


def write_bfm(path, system, frames, ids=None):
    """Header plus one !mcs frame per (age, positions) in `frames`."""
    ids = ids or standard_bond_ids()
    inv = {v: k for k, v in ids.items()}
    n = system.n
    attrs = system.attributes if system.attributes is not None else np.zeros(n, np.int32)
    out = bytearray()
    out += b"#!version=2.0\n"
    out += f"!number_of_monomers={n}\n".encode()
    out += "".join(f"!box_{a}={b}\n" for a, b in zip("xyz", system.box)).encode()
    per = getattr(system, "periodic", (True, True, True))
    out += "".join(f"!periodic_{a}={int(bool(p))}\n" for a, p in zip("xyz", per)).encode()
    out += b"!set_of_bondvectors\n"
    for i, v in ids.items():
        out += f"{v[0]} {v[1]} {v[2]}:{i}\n".encode()
    out += b"\n!attributes\n"
    i = 0
    while i < n:
        j = i
        while j + 1 < n and attrs[j + 1] == attrs[i]:
            j += 1
        out += f"{i + 1}-{j + 1}:{attrs[i]}\n".encode()
        i = j + 1
    out += b"\n!bonds\n"
    for i in range(n):
        for k in system.nbr[i, : system.deg[i]]:
            k = int(k)
            if k > i and k != i + 1:
                out += f"{i + 1} {k + 1}\n".encode()
    out += b"\n"
    nb = [set(int(v) for v in system.nbr[i, : system.deg[i]]) for i in range(n)]
    for age, pos in frames:
        pos = np.asarray(pos, dtype=np.int64)
        out += f"!mcs={age}\n".encode()
        i = 0
        while i < n:
            out += f"{pos[i, 0]} {pos[i, 1]} {pos[i, 2]}".encode()
            j = i
            chain = bytearray()
            while j + 1 < n and (j + 1) in nb[j]:
                v = tuple(int(c) for c in pos[j + 1] - pos[j])
                if v not in inv:
                    break
                chain.append(inv[v])
                j += 1
            if chain:
                out += b" " + bytes(chain)
            out += b"\n"
            i = j + 1
        out += b"\n"
    open(path, "wb").write(bytes(out))


def write_seeds(path, words):
    with open(path, "w") as f:
        f.write("\n".join(str(int(w) & 0xFFFFFFFF) for w in words) + "\n")


def read_seeds(path):
    w = np.array([int(v) for v in open(path).read().split()], dtype=np.uint64).astype(np.uint32)
    if w.size < 250:
        raise ValueError(".seeds file needs at least 250 values")
    return w
