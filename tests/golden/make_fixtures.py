"""Generate the golden fixtures in tests/golden/ from the reference's own test data.

Reads, from the reference tree (never at test time):
  garli/trunk/tests/data/z.11x2178.nex     11 taxa x 2,178 sites (DNA)
  garli/trunk/tests/data/n.G4.start        GTR+I+G4 start tree + [!GarliScore] + [!GarliModel]
  garli/trunk/tests/data/n.G5.start        GTR+I+G5
  garli/trunk/tests/data/c.start           codon (6 nucleotide rates, one omega class)

and writes JSON fixtures holding the compressed site patterns (GARLI's
PatternManager order, garli_b200/patterns.py), the tree in GARLI's node layout,
the model parameters printed by GARLI and GARLI's own score for that tree.
The GarliScore comments are the pins: GARLI computed them with its CPU path
before printing the parameters to 5 decimals, so a rescore agrees to about 1e-3.

    python tests/golden/make_fixtures.py /path/to/garli/trunk
    GARLI_REFERENCE=/path/containing/garli python tests/golden/make_fixtures.py
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from garli_b200 import patterns, treeio  # noqa: E402

if len(sys.argv) > 1:
    REF = sys.argv[1]
elif os.environ.get("GARLI_REFERENCE"):
    REF = os.path.join(os.environ["GARLI_REFERENCE"], "garli", "trunk")
else:
    sys.exit("usage: make_fixtures.py /path/to/garli/trunk (or set GARLI_REFERENCE)")
DATA = os.path.join(REF, "tests", "data")


def read_nexus_matrix(path):
    txt = open(path).read()
    txt = re.sub(r"\[[^\]]*\]", "", txt)
    m = re.search(r"matrix(.*?);", txt, re.S | re.I)
    rows = {}
    order = []
    for line in m.group(1).strip().splitlines():
        parts = line.split()
        if len(parts) < 2:
            continue
        name, seq = parts[0], "".join(parts[1:])
        if name not in rows:
            order.append(name)
            rows[name] = ""
        rows[name] += seq
    return order, rows


def read_start(path):
    txt = open(path).read()
    block = re.search(r"translate(.*?);", txt, re.S | re.I).group(1)
    trans = dict((num, name) for num, name in re.findall(r"(\d+)\s+([^\s,;]+)", block))
    score = float(re.search(r"GarliScore\s+([-0-9.]+)", txt).group(1))
    model = re.search(r"GarliModel([^\]]*)\]", txt).group(1).split()
    newick = re.search(r"tree\s+\S+\s*=\s*(.*?;)", txt, re.S).group(1)
    params = {}
    key = None
    for tok in model:
        if re.fullmatch(r"[a-z]", tok):
            key = tok
            params[key] = []
        else:
            params[key].append(float(tok))
    return trans, score, params, newick


def parse_set(spec, nchar):
    """1-based character numbers of a NEXUS set list ("1-749 751-1008 1930-.")."""
    out = []
    for tok in spec.split():
        if "-" in tok:
            a, b = tok.split("-")
            out.extend(range(int(a), (nchar if b == "." else int(b)) + 1))
        else:
            out.append(int(tok))
    return out


def wtset_sitelike_extra(pd, plain_masks):
    """The scoring tests of n.G4 / n.G5 read z.11x2178.wtset.nex: 2,180 columns
    with an exset and a compensating integer wtset (assumptions block).  Their
    check (tests/runtests.sh) halves the sum of column 2 of the sitelikes file:
    the tree's -lnL plus one -lnL per non-excluded column, written once whatever
    its weight (Tree::OutputSiteLikelihoods, tree.cpp:5500-5560).  With weights
    w_c the number compared is therefore -lnL + 1/2 sum_c (w_c - 1) lnL_c.
    Returns [(pattern index in pd, w_c - 1)] for the columns with w_c != 1,
    after checking that the weighted columns are the plain matrix's columns
    plus all-missing ones (so the tree's lnL is the plain data's)."""
    order, rows = read_nexus_matrix(os.path.join(DATA, "z.11x2178.wtset.nex"))
    txt = open(os.path.join(DATA, "z.11x2178.wtset.nex")).read()
    txt = re.sub(r"\[[^\]]*\]", "", txt)
    nchar = len(rows[order[0]])
    ex = set(parse_set(re.search(r"exset\s*\*\s*\S+\s*=\s*([^;]*);", txt, re.I).group(1), nchar))
    w = {}
    for part in re.search(r"wtset\s*\*\s*\S+\s*=\s*([^;]*);", txt, re.I).group(1).split(","):
        wt, lst = part.split(":")
        for c in parse_set(lst, nchar):
            w[c] = int(wt)
    porder, prows = read_nexus_matrix(os.path.join(DATA, "z.11x2178.nex"))
    assert order == porder
    col = lambda r, o, c: "".join(r[t][c - 1].upper() for t in o)
    missing = lambda s: all(ch in "N?-" for ch in s)
    from collections import Counter
    weighted, plain = Counter(), Counter()
    for c in range(1, nchar + 1):
        if c not in ex and not missing(col(rows, order, c)):
            weighted[col(rows, order, c)] += w.get(c, 1)
    for c in range(1, len(prows[porder[0]]) + 1):
        plain[col(prows, porder, c)] += 1
    assert weighted == plain, "the weighted matrix is not the plain one"
    # pattern of each plain column, by its tip masks
    key = {bytes(pd.tips[:, j].tolist()): j for j in range(pd.npat)}
    extra = []
    for c in sorted(w):
        if c in ex or w[c] == 1 or missing(col(rows, order, c)):
            continue
        j = next(j for j in range(plain_masks.shape[1]) if col(prows, porder, j + 1) == col(rows, order, c))
        extra.append([key[bytes(plain_masks[:, j].tolist())], w[c] - 1])
    return extra


def expected_scr(conf):
    for line in open(os.path.join(DATA, "expected.scr")):
        parts = line.split()
        if parts and parts[0] == conf:
            return float(parts[1])
    raise KeyError(conf)


def dna_fixture(start_name, ncat):
    order, rows = read_nexus_matrix(os.path.join(DATA, "z.11x2178.nex"))
    trans, score, params, newick = read_start(os.path.join(DATA, start_name))
    num_of = {name: int(num) for num, name in trans.items()}
    ntax = len(order)
    masks = np.zeros((ntax, len(rows[order[0]])), dtype=np.uint8)
    for name in order:
        masks[num_of[name] - 1] = [patterns.DNA_CODES[c.upper()] for c in rows[name]]
    pd = patterns.compress(masks, 4)
    tree = treeio.parse_newick(newick)
    child3, dlen = treeio.to_garli(tree)
    return {
        "source": f"garli/trunk/tests/data/z.11x2178.nex + {start_name}",
        "nstates": 4,
        "ntax": ntax,
        "nsites": int(pd.nsites),
        "npat": int(pd.npat),
        "tips_hex": [bytes(r.tolist()).hex() for r in pd.tips],
        "counts": pd.counts.tolist(),
        "last_const": int(pd.last_const),
        "const_states": pd.const_states.tolist(),
        "child3": child3.tolist(),
        "dlen": dlen.tolist(),
        "model": {"r": params["r"], "e": params["e"], "a": params.get("a", [None])[0],
                  "p": params.get("p", [0.0])[0], "ncat": ncat},
        "garli_score": score,
        # the reference's scoring test of this start tree (tests/scoring/<conf>,
        # tests/data/expected.scr, allowed error from tests/runtests.sh)
        "scoring_test": {"conf": start_name.replace(".start", ".conf"),
                         "expected_scr": expected_scr(start_name.replace(".start", ".conf")),
                         "allowed": 0.01, "sitelike_extra": wtset_sitelike_extra(pd, masks)},
    }


STD_CODE = "KNKNTTTTRSRSIIMIQHQHPPPPRRRRLLLLEDEDAAAAGGGGVVVV*Y*YSSSS*CWCLFLF"


def codon_fixture(start_name):
    """CodonData::FillCodonMatrixFromDNA (sequencedata.cpp:364-440): ACGT base-4
    codon numbering, stop codons removed, any gap or ambiguity -> missing (61)."""
    order, rows = read_nexus_matrix(os.path.join(DATA, "z.11x2178.nex"))
    trans, score, params, newick = read_start(os.path.join(DATA, start_name))
    num_of = {name: int(num) for num, name in trans.items()}
    ntax = len(order)
    sense = [c for c in range(64) if STD_CODE[c] != "*"]
    index_of = {c: i for i, c in enumerate(sense)}
    idx = {"A": 0, "C": 1, "G": 2, "T": 3, "U": 3}
    ncod = len(rows[order[0]]) // 3
    states = np.zeros((ntax, ncod), dtype=np.uint8)
    for name in order:
        s = rows[name].upper()
        out = []
        for k in range(ncod):
            trip = s[3 * k: 3 * k + 3]
            if all(ch in idx for ch in trip):
                c = idx[trip[0]] * 16 + idx[trip[1]] * 4 + idx[trip[2]]
                out.append(index_of[c])
            else:
                out.append(61)
        states[num_of[name] - 1] = out
    pd = patterns.compress(states, 61)
    # CodonData::CalcEmpiricalFreqs, CODON_TABLE (sequencedata.cpp:228-276): observed
    # codon counts over all taxa and patterns, one pseudo-count each if any is zero
    emp = np.zeros(61)
    for t in range(ntax):
        for j in range(pd.npat):
            if pd.tips[t, j] != 61:
                emp[pd.tips[t, j]] += pd.counts[j]
    if (emp == 0).any():
        emp += 1.0
    emp = emp / emp.sum()
    tree = treeio.parse_newick(newick)
    child3, dlen = treeio.to_garli(tree)
    return {
        "source": f"garli/trunk/tests/data/z.11x2178.nex (as codons) + {start_name}",
        "nstates": 61,
        "ntax": ntax,
        "nsites": int(pd.nsites),
        "npat": int(pd.npat),
        "tips_hex": [bytes(r.tolist()).hex() for r in pd.tips],
        "counts": pd.counts.tolist(),
        "last_const": int(pd.last_const),
        "const_states": pd.const_states.tolist(),
        "child3": child3.tolist(),
        "dlen": dlen.tolist(),
        "model": {"r": params["r"], "e": params["e"], "e_empirical": emp.tolist(), "o": params["o"], "ncat": 1},
        "garli_score": score,
        # tests/scoring/c.conf: the plain matrix, omega fixed (nonsynonymousfixed),
        # empirical frequencies, six relative rates estimated
        "scoring_test": {"conf": "c.conf", "expected_scr": expected_scr("c.conf"), "allowed": 0.01,
                         "sitelike_extra": []},
    }


def main():
    out = {
        "z11x2178_nG4.json": dna_fixture("n.G4.start", 4),
        "z11x2178_nG5.json": dna_fixture("n.G5.start", 5),
        "z11x2178_codon.json": codon_fixture("c.start"),
    }
    for name, obj in out.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(obj, f, separators=(",", ":"))
        print(name, obj["npat"], "patterns, GarliScore", obj["garli_score"])


if __name__ == "__main__":
    main()
