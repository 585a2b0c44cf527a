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
class ModelSpec:
    """The parameters a synthetic model is drawn with; ``build_model`` turns
    them into a Model with a chosen library's Q, discrete-gamma and eigen
    functions (the engine's, or any module with the same five functions), so
    that each side of a comparison can build the model with its own math."""

    kind: str  # "gtr", "aa" or "codon"
    pi: np.ndarray
    exch: np.ndarray | None = None  # GTR: 6 relative rates (last = 1); AA: 190 exchangeabilities
    alpha: float = 0.5
    ncat: int = 1
    pinv: float | None = None
    kappa: float = 0.0
    omega: float = 0.0


def build_model(spec: ModelSpec, mathlib=None) -> engine.Model:
    """Model of ``spec`` from ``mathlib``'s gtr_qmat / aa_qmat / codon_qmat,
    discrete_gamma and eigen (default: the engine's host model math)."""
    ml = engine if mathlib is None else mathlib
    if spec.kind == "gtr":
        Q, bm = ml.gtr_qmat(list(spec.exch), spec.pi)
    elif spec.kind == "aa":
        Q, bm = ml.aa_qmat(spec.exch, spec.pi)
    elif spec.kind == "codon":
        Q, bm = ml.codon_qmat(spec.kappa, spec.omega, spec.pi)
    else:
        raise ValueError(spec.kind)
    rates = np.asarray(ml.discrete_gamma(spec.alpha, spec.ncat), dtype=np.float64) if spec.ncat > 1 else np.ones(1)
    ev, U, Ui = ml.eigen(Q, spec.pi)
    has_pinv = spec.pinv is not None
    pinv = float(spec.pinv) if has_pinv else 0.0
    probs = np.full(len(rates), (1.0 - pinv) / len(rates))
    return engine.Model(spec.pi.shape[0], np.ascontiguousarray(spec.pi, dtype=np.float64), Q, bm, ev, U, Ui,
                        rates, probs, pinv, has_pinv)


@dataclass
class Workload:
    name: str
    child3: np.ndarray
    dlen: np.ndarray
    model: engine.Model
    data: PatternData
    spec: ModelSpec | None = None

    def model_with(self, mathlib) -> engine.Model:
        """The same model built with another library's model math."""
        return build_model(self.spec, mathlib)


def gtr_spec(rng, alpha=0.5, ncat=4, pinv=None) -> ModelSpec:
    pi = rng.dirichlet([10.0] * 4)
    rel = rng.gamma(2.0, 1.0, size=6)
    rel = rel / rel[5]
    return ModelSpec("gtr", pi, np.array(rel[:5].tolist() + [1.0]), alpha, ncat if ncat > 1 else 1, pinv)


def aa_spec(rng, alpha=0.8, ncat=4) -> ModelSpec:
    exch = rng.gamma(1.0, 1.0, size=190)
    pi = rng.dirichlet([5.0] * 20)
    return ModelSpec("aa", pi, exch, alpha, ncat)


def codon_spec(rng) -> ModelSpec:
    kappa = rng.uniform(1.5, 4.0)
    omega = rng.uniform(0.1, 1.0)
    pos = [rng.dirichlet([10.0] * 4) for _ in range(3)]
    f = np.array([pos[0][c >> 4] * pos[1][(c >> 2) & 3] * pos[2][c & 3] for c in SENSE_CODONS])
    f = f / f.sum()
    return ModelSpec("codon", f, None, 0.0, 1, None, kappa, omega)


def gtr_model(rng, alpha=0.5, ncat=4, pinv=None, mathlib=None) -> engine.Model:
    return build_model(gtr_spec(rng, alpha, ncat, pinv), mathlib)


def aa_model(rng, alpha=0.8, ncat=4, mathlib=None) -> engine.Model:
    return build_model(aa_spec(rng, alpha, ncat), mathlib)


def codon_model(rng, mathlib=None) -> engine.Model:
    return build_model(codon_spec(rng), mathlib)


def dna_to_masks(states: np.ndarray) -> np.ndarray:
    return (1 << states.astype(np.uint8)).astype(np.uint8)


def make_dna(ntax, nsites, seed, mean_blen=0.1, alpha=0.5, ncat=4, pinv_range=None, name="dna",
             mathlib=None) -> Workload:
    rng = np.random.default_rng(seed)
    child3, dlen = yule_tree(ntax, rng, mean_blen)
    pinv = float(rng.uniform(*pinv_range)) if pinv_range else None
    spec = gtr_spec(rng, alpha, ncat, pinv)
    m = build_model(spec, mathlib)
    st = simulate(child3, dlen, m, nsites, rng)
    pd = compress(dna_to_masks(st), 4)
    return Workload(name, child3, dlen, m, pd, spec)


def dna_small(seed=0, mathlib=None) -> Workload:
    return make_dna(32, 2000, seed, name="dna_gtr_g4_32x2000", mathlib=mathlib)


def dna_large(seed=1, nsites=100_000, ntax=128, mathlib=None) -> Workload:
    return make_dna(ntax, nsites, seed, pinv_range=(0.05, 0.3), name=f"dna_gtr_i_g4_{ntax}x{nsites}",
                    mathlib=mathlib)


def aa(seed=2, ntax=64, nsites=20_000, mathlib=None) -> Workload:
    rng = np.random.default_rng(seed)
    child3, dlen = yule_tree(ntax, rng, 0.15)
    spec = aa_spec(rng)
    m = build_model(spec, mathlib)
    st = simulate(child3, dlen, m, nsites, rng)
    return Workload(f"aa_g4_{ntax}x{nsites}", child3, dlen, m, compress(st, 20), spec)


def codon(seed=3, ntax=32, ncodons=5_000, mathlib=None) -> Workload:
    rng = np.random.default_rng(seed)
    child3, dlen = yule_tree(ntax, rng, 0.2)
    spec = codon_spec(rng)
    m = build_model(spec, mathlib)
    st = simulate(child3, dlen, m, ncodons, rng)
    return Workload(f"codon_gy94_{ntax}x{ncodons}", child3, dlen, m, compress(st, 61), spec)


# ---------------------------------------------------------------- GA candidates
MIN_BRLEN = 1e-8  # defs.h:106


def _adjacency(child3, dlen):
    nb = {}
    ln = {}
    for v in range(child3.shape[0]):
        for c in child3[v]:
            if c >= 0:
                c = int(c)
                nb.setdefault(v, []).append(c)
                nb.setdefault(c, []).append(v)
                ln[(min(v, c), max(v, c))] = float(dlen[c])
    return nb, ln


def _layout(nb, ln, nnodes, root=0):
    """GARLI layout of an unrooted tree rooted at ``root`` (keeps node numbers;
    neighbour order is kept as stored in ``nb``)."""
    child3 = -np.ones((nnodes, 3), dtype=np.int32)
    dlen = np.zeros(nnodes)
    stack = [(root, -1)]
    while stack:
        v, par = stack.pop()
        kids = [c for c in nb[v] if c != par]
        if par >= 0:
            dlen[v] = ln[(min(v, par), max(v, par))]
        if v == root:
            child3[v] = kids
        elif kids:
            child3[v] = [kids[0], -1, kids[1]]
        for c in kids:
            stack.append((c, v))
    return child3, dlen


def spr_move(child3, dlen, rng, radius):
    """One SPR move of Tree::SPRMutate (tree.cpp:3148-3248) on a GARLI-layout tree.

    A random non-root internal node P (the connector) and one of its children
    ``cut`` are chosen; P is pruned (its two other neighbours a, b joined, the
    joined branch keeping the sum of both lengths) and regrafted into a branch
    at edge distance ``radius`` from the joined one (radius 1 = an NNI), both
    halves of that branch getting max(len / 2, min_brlen).  Returns the new
    (child3, dlen) on the same node numbers (root 0 stays the trifurcating
    root) and the connector P, whose left child is ``cut`` and right child the
    lower node of the broken branch, as in GARLI."""
    nnodes = child3.shape[0]
    ntax = (nnodes + 2) // 2
    nb, ln = _adjacency(child3, dlen)
    anc = {int(c): v for v in range(nnodes) for c in child3[v] if c >= 0}
    for _ in range(1000):
        P = int(rng.integers(ntax + 1, nnodes))
        cut = int(child3[P][0] if rng.random() < 0.5 else child3[P][2])
        a, b = [c for c in nb[P] if c != cut]
        # nodes of the cut subtree (on cut's side of P)
        sub, st = set(), [cut]
        while st:
            v = st.pop()
            sub.add(v)
            st += [c for c in nb[v] if c != P and c not in sub]
        # edges of the remaining tree with the joined edge (a, b), by BFS over edges
        nb2 = {v: [c for c in nb[v] if c != P] for v in nb if v != P and v not in sub}
        nb2[a].append(b)
        nb2[b].append(a)
        dist = {(min(a, b), max(a, b)): 0}
        frontier = [(a, b)]
        while frontier:
            nxt = []
            for (x, y) in frontier:
                d = dist[(min(x, y), max(x, y))]
                for end in (x, y):
                    for z in nb2[end]:
                        e = (min(end, z), max(end, z))
                        if e not in dist:
                            dist[e] = d + 1
                            nxt.append(e)
            frontier = nxt
        cands = [e for e, d in dist.items() if d == radius]
        if not cands:
            continue
        u, w = cands[int(rng.integers(len(cands)))]
        break
    else:
        raise RuntimeError("no SPR move of that radius")
    # prune P
    lab = ln.pop((min(a, P), max(a, P)))
    lbp = ln.pop((min(b, P), max(b, P)))
    nb[a] = [b if c == P else c for c in nb[a]]
    nb[b] = [a if c == P else c for c in nb[b]]
    ln[(min(a, b), max(a, b))] = lab + lbp
    # regraft on (u, w): P between them
    t = ln.pop((min(u, w), max(u, w)))
    half = max(t * 0.5, MIN_BRLEN)
    nb[u] = [P if c == w else c for c in nb[u]]
    nb[w] = [P if c == u else c for c in nb[w]]
    ln[(min(u, P), max(u, P))] = half
    ln[(min(w, P), max(w, P))] = half
    # P's neighbours: its future parent (the one of u, w nearer the root) first, then cut, broken
    new_nb = dict(nb)
    new_nb[P] = [u, w, cut]
    c3, dl = _layout(new_nb, ln, nnodes)
    par = next(v for v in range(nnodes) if P in c3[v])
    broken = w if par == u else u
    c3[P] = [cut, -1, broken]
    return c3, dl, P


def ga_candidates(child3, dlen, count, seed, radius_range=(1, 8)):
    """``count`` candidates of one generation, each the base tree after one SPR
    move with radius ~ Uniform{radius_range} (NNI = radius 1)."""
    rng = np.random.default_rng(seed)
    nnodes = child3.shape[0]
    c3s = np.zeros((count, nnodes, 3), dtype=np.int32)
    dls = np.zeros((count, nnodes))
    conn = np.zeros(count, dtype=np.int32)
    for i in range(count):
        r = int(rng.integers(radius_range[0], radius_range[1] + 1))
        c3s[i], dls[i], conn[i] = spr_move(child3, dlen, rng, r)
    return c3s, dls, conn


def batch_workload(seed=4, ntax=64, nsites=50_000, ncand=256, mathlib=None):
    """The GA-population workload: a Yule base tree, GTR+G4, its alignment, and
    ``ncand`` SPR/NNI candidates of it (radius ~ U{1..8})."""
    w = make_dna(ntax, nsites, seed, name=f"ga_batch_dna_gtr_g4_{ntax}x{nsites}_{ncand}cand", mathlib=mathlib)
    c3s, dls, conn = ga_candidates(w.child3, w.dlen, ncand, seed + 1000)
    return w, c3s, dls, conn
