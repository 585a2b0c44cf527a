"""Tree topology in GARLI's node layout.

GARLI stores an unrooted tree with a trifurcating root (tree.cpp, treenode.h):
node 0 is the root with children ``left``, ``left->next`` (middle) and
``right``; nodes 1..ntax are the tips (taxon numbers); the other internal nodes
are numbered ntax+1 .. 2*ntax-3 and have exactly two children.  Every node but
the root owns the branch to its ancestor (``dlen``).

The engine and the oracle both take the topology as ``child3`` (an
(nnodes, 3) int32 array of left / middle / right, -1 where absent) plus
``dlen`` (nnodes,) float64.
"""
from __future__ import annotations

import re

import numpy as np


class Node:
    __slots__ = ("children", "label", "blen")

    def __init__(self, label=None, blen=0.0):
        self.children: list[Node] = []
        self.label = label
        self.blen = blen


def parse_newick(s: str) -> Node:
    """Parse a Newick string (comments in square brackets are skipped)."""
    s = re.sub(r"\[[^\]]*\]", "", s).strip()
    if s.endswith(";"):
        s = s[:-1]
    pos = 0

    def parse() -> Node:
        nonlocal pos
        node = Node()
        if s[pos] == "(":
            pos += 1
            while True:
                node.children.append(parse())
                if s[pos] == ",":
                    pos += 1
                    continue
                if s[pos] == ")":
                    pos += 1
                    break
                raise ValueError(f"bad newick at {pos}")
        m = re.match(r"[^:,()]*", s[pos:])
        lab = m.group(0).strip()
        pos += len(m.group(0))
        if lab:
            node.label = lab
        if pos < len(s) and s[pos] == ":":
            pos += 1
            m = re.match(r"[-+0-9.eE]+", s[pos:])
            node.blen = float(m.group(0))
            pos += len(m.group(0))
        return node

    root = parse()
    return root


def to_garli(root: Node, taxon_number: dict[str, int] | None = None):
    """Number a trifurcating-root tree the GARLI way; returns (child3, dlen)."""
    if len(root.children) == 2:
        # rooted input: make the internal child the trifurcating root
        a, b = root.children
        if not a.children:
            a, b = b, a
        b.blen += a.blen
        a.children.append(b)
        a.blen = 0.0
        root = a
    if len(root.children) != 3:
        raise ValueError("root must have three children")
    tips = []

    def collect(n):
        if not n.children:
            tips.append(n)
        for c in n.children:
            collect(c)

    collect(root)
    ntax = len(tips)
    nnodes = 2 * ntax - 2
    child3 = -np.ones((nnodes, 3), dtype=np.int32)
    dlen = np.zeros(nnodes, dtype=np.float64)
    next_internal = [ntax + 1]

    def number(n, is_root=False) -> int:
        if not n.children:
            lab = n.label
            if taxon_number is not None:
                idx = taxon_number[lab]
            else:
                idx = int(lab)
            dlen[idx] = n.blen
            return idx
        if is_root:
            idx = 0
        else:
            idx = next_internal[0]
            next_internal[0] += 1
            dlen[idx] = n.blen
            if len(n.children) != 2:
                raise ValueError("internal nodes must be bifurcating")
        kids = [number(c) for c in n.children]
        if is_root:
            child3[idx] = kids
        else:
            child3[idx] = [kids[0], -1, kids[1]]
        return idx

    number(root, is_root=True)
    return child3, dlen


def postorder_internal(child3: np.ndarray) -> list[int]:
    out = []

    def rec(n):
        for c in child3[n]:
            if c > 0 and child3[c][0] >= 0:
                rec(int(c))
        out.append(n)

    rec(0)
    return out
