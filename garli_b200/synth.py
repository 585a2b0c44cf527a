"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: every alignment is simulated down a random
Yule tree under the configuration's model and compressed into GARLI-ordered
site patterns (patterns.py).

  dna_small   32 taxa, 2,000 sites, GTR+G4 (alpha 0.5), blen ~ Exp(0.1)
  dna_large  128 taxa, 100,000 sites, GTR+I+G4, pinv ~ U(0.05, 0.3)
  aa          64 taxa, 20,000 sites, 20 states +G4 (alpha 0.8), blen ~ Exp(0.15)
  codon       32 taxa, 5,000 codons, GY94 (61 states), one rate, blen ~ Exp(0.2)
  batch       64-taxon base tree, 50,000 sites, GTR+G4, plus NNI/SPR candidates
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import engine
from .patterns import PatternData, compress

STD_CODE = "KNKNTTTTRSRSIIMIQHQHPPPPRRRRLLLLEDEDAAAAGGGGVVVV*Y*YSSSS*CWCLFLF"
SENSE_CODONS = [c for c in range(64) if STD_CODE[c] != "*"]


def yule_tree(ntax: int, rng: np.random.Generator, mean_blen: float):
    """Random rooted Yule topology, unrooted into GARLI's layout (see treeio).

    Returns child3 (nnodes, 3) and dlen (nnodes,); tips are numbered 1..ntax in
    random order, branch lengths are iid Exponential(mean_blen)."""
    # rooted binary tree as parent links; node ids: 0 = root, grow by splitting leaves
    children = {0: []}
    leaves = [0]
    nid = 1
    while len(leaves) < ntax:
        k = int(rng.integers(len(leaves)))
        leaf = leaves.pop(k)
        a, b = nid, nid + 1
        nid += 2
        children[leaf] = [a, b]
        children[a] = []
        children[b] = []
        leaves += [a, b]
    blen = {n: float(rng.exponential(mean_blen)) for n in children}
    # unroot: the internal child of the root becomes the trifurcating root
    a, b = children[0]
    if not children[a]:
        a, b = b, a
    blen[b] += blen[a]
    root = a
    kids = {n: list(c) for n, c in children.items()}
    kids[root] = kids[root] + [b]
    del kids[0]
    # number: tips get a random permutation of 1..ntax; internals in preorder
    tip_nodes = [n for n, c in kids.items() if not c]
    perm = rng.permutation(ntax) + 1
    num = {n: int(perm[i]) for i, n in enumerate(tip_nodes)}
    nnodes = 2 * ntax - 2
    child3 = -np.ones((nnodes, 3), dtype=np.int32)
    dlen = np.zeros(nnodes)
    nxt = [ntax + 1]

    def visit(n, is_root=False):
        if not kids[n]:
            idx = num[n]
            dlen[idx] = blen[n]
            return idx
        if is_root:
            idx = 0
        else:
            idx = nxt[0]
            nxt[0] += 1
            dlen[idx] = blen[n]
        ks = [visit(c) for c in kids[n]]
        child3[idx] = ks if is_root else [ks[0], -1, ks[1]]
        return idx

    visit(root, True)
    return child3, dlen


def preorder(child3: np.ndarray) -> list[int]:
    out, stack = [], [0]
    while stack:
        n = stack.pop()
        out.append(n)
        for c in child3[n][::-1]:
            if c >= 0:
                stack.append(int(c))
    return out


def simulate(child3, dlen, model: engine.Model, nsites: int, rng: np.random.Generator) -> np.ndarray:
    """States (ntax, nsites) simulated down the tree; +I sites are invariant."""
    S, R = model.nstates, model.ncat
    ntax = (child3.shape[0] + 2) // 2
    cat = rng.integers(R, size=nsites)
    inv = rng.random(nsites) < model.pinv if model.has_pinv else np.zeros(nsites, dtype=bool)
    cum_pi = np.cumsum(model.pi)
    states = {0: np.minimum(np.searchsorted(cum_pi, rng.random(nsites) * cum_pi[-1], side="right"), S - 1)}
    for n in preorder(child3):
        if n == 0:
            pass
        par = states[n]
        for c in child3[n]:
            if c < 0:
                continue
            P = model.pmats(dlen[c])  # [R, S, S]
            cum = np.cumsum(P, axis=2)
            rows = cum[cat, par]  # (nsites, S)
            u = rng.random(nsites) * rows[:, -1]
            child = (u[:, None] > rows).sum(axis=1)
            child = np.minimum(child, S - 1)
            child = np.where(inv, par, child)
            states[int(c)] = child
    out = np.zeros((ntax, nsites), dtype=np.uint8)
    for t in range(1, ntax + 1):
        out[t - 1] = states[t]
    return out


@dataclass
class Workload:
    name: str
    child3: np.ndarray
    dlen: np.ndarray
    model: engine.Model
    data: PatternData


def gtr_model(rng, alpha=0.5, ncat=4, pinv=None) -> engine.Model:
    pi = rng.dirichlet([10.0] * 4)
    rel = rng.gamma(2.0, 1.0, size=6)
    rel = rel / rel[5]
    Q, bm = engine.gtr_qmat(rel[:5].tolist() + [1.0], pi)
    rates = engine.discrete_gamma(alpha, ncat) if ncat > 1 else np.ones(1)
    has_pinv = pinv is not None
    return engine.make_model(4, Q, bm, pi, rates, pinv if has_pinv else 0.0, has_pinv)


def aa_model(rng, alpha=0.8, ncat=4) -> engine.Model:
    exch = rng.gamma(1.0, 1.0, size=190)
    pi = rng.dirichlet([5.0] * 20)
    Q, bm = engine.aa_qmat(exch, pi)
    return engine.make_model(20, Q, bm, pi, engine.discrete_gamma(alpha, ncat))


def codon_model(rng) -> engine.Model:
    kappa = rng.uniform(1.5, 4.0)
    omega = rng.uniform(0.1, 1.0)
    pos = [rng.dirichlet([10.0] * 4) for _ in range(3)]
    f = np.array([pos[0][c >> 4] * pos[1][(c >> 2) & 3] * pos[2][c & 3] for c in SENSE_CODONS])
    f = f / f.sum()
    Q, bm = engine.codon_qmat(kappa, omega, f)
    return engine.make_model(61, Q, bm, f, np.ones(1))


def dna_to_masks(states: np.ndarray) -> np.ndarray:
    return (1 << states.astype(np.uint8)).astype(np.uint8)


def make_dna(ntax, nsites, seed, mean_blen=0.1, alpha=0.5, ncat=4, pinv_range=None, name="dna") -> Workload:
    rng = np.random.default_rng(seed)
    child3, dlen = yule_tree(ntax, rng, mean_blen)
    pinv = float(rng.uniform(*pinv_range)) if pinv_range else None
    m = gtr_model(rng, alpha, ncat, pinv)
    st = simulate(child3, dlen, m, nsites, rng)
    pd = compress(dna_to_masks(st), 4)
    return Workload(name, child3, dlen, m, pd)


def dna_small(seed=0) -> Workload:
    return make_dna(32, 2000, seed, name="dna_gtr_g4_32x2000")


def dna_large(seed=1, nsites=100_000, ntax=128) -> Workload:
    return make_dna(ntax, nsites, seed, pinv_range=(0.05, 0.3), name=f"dna_gtr_i_g4_{ntax}x{nsites}")


def aa(seed=2, ntax=64, nsites=20_000) -> Workload:
    rng = np.random.default_rng(seed)
    child3, dlen = yule_tree(ntax, rng, 0.15)
    m = aa_model(rng)
    st = simulate(child3, dlen, m, nsites, rng)
    return Workload(f"aa_g4_{ntax}x{nsites}", child3, dlen, m, compress(st, 20))


def codon(seed=3, ntax=32, ncodons=5_000) -> Workload:
    rng = np.random.default_rng(seed)
    child3, dlen = yule_tree(ntax, rng, 0.2)
    m = codon_model(rng)
    st = simulate(child3, dlen, m, ncodons, rng)
    return Workload(f"codon_gy94_{ntax}x{ncodons}", child3, dlen, m, compress(st, 61))
