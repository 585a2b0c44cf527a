"""Site-pattern compression and tip encoding for the likelihood engine.

Follows GARLI's PatternManager (garli/trunk/src/datamatr.cpp):
  * SitePattern::CalcPatternTypeAndNumStates (datamatr.cpp:82-208) gives each
    column a "number of states" used as the primary sort key: 0 = all missing,
    1 = constant (the AND of the DNA masks is non-empty), otherwise max(2, n);
  * PatternManager::NewSort / NewCollapse / NewPack (datamatr.cpp:243-283):
    stable sort by (numStates, state vector), merge identical columns adding
    their counts, drop all-missing columns;
  * NewDetermineConstantSites (datamatr.cpp:334-376): constant patterns come
    first; ``lastConstant`` is the index of the last one and ``constStates`` is
    the AND of the masks (DNA) or the single observed state (AA / codon).

Encoding of tip states (the device form of NucleotideData::CharToDatum,
sequencedata.cpp:672, and MakeAmbigStrings, :278): DNA uses the 4-bit mask
A=1, C=2, G=4, T=8 (15 = missing), NState data uses the state index with
``nstates`` meaning missing.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

DNA_CODES = {
    "A": 1, "C": 2, "G": 4, "T": 8, "U": 8, "M": 3, "R": 5, "S": 6, "V": 7,
    "W": 9, "Y": 10, "H": 11, "K": 12, "D": 13, "B": 14, "N": 15, "-": 15, "?": 15,
}


@dataclass
class PatternData:
    """Compressed alignment: ``tips[t, p]`` is the code of taxon t+1 at pattern p."""

    nstates: int
    tips: np.ndarray  # (ntax, npat) uint8
    counts: np.ndarray  # (npat,) int32
    last_const: int
    const_states: np.ndarray  # (npat,) int32; meaningful for p <= last_const
    nsites: int

    @property
    def ntax(self) -> int:
        return self.tips.shape[0]

    @property
    def npat(self) -> int:
        return self.tips.shape[1]


def dna_chars_to_masks(rows: list[str]) -> np.ndarray:
    out = np.empty((len(rows), len(rows[0])), dtype=np.uint8)
    for i, r in enumerate(rows):
        out[i] = [DNA_CODES[c.upper()] for c in r]
    return out


def _num_states_dna(cols: np.ndarray) -> np.ndarray:
    """numStates per column (columns given as rows of ``cols``: (ncol, ntax))."""
    anded = np.bitwise_and.reduce(cols, axis=1)
    full = cols == 15
    partial_amb = (~full) & ((cols & (cols - 1)) != 0)
    ambig_col = partial_amb.any(axis=1)
    present = np.zeros((cols.shape[0], 4), dtype=bool)
    for k in range(4):
        present[:, k] = ((cols == (1 << k))).any(axis=1)
    nuniq = present.sum(axis=1)
    ns = np.where(nuniq >= 2, nuniq, 2)
    ns = np.where(ambig_col, 2, ns)
    constant = np.where(ambig_col, anded != 0, nuniq == 1)
    ns = np.where(constant, 1, ns)
    missing = anded == 15
    ns = np.where(missing, 0, ns)
    return ns.astype(np.int64)


def _num_states_nstate(cols: np.ndarray, nstates: int) -> np.ndarray:
    ns = np.zeros(cols.shape[0], dtype=np.int64)
    for s in range(nstates):
        ns += (cols == s).any(axis=1)
    ns = np.where(ns >= 2, ns, np.where(ns == 1, 1, 0))
    return ns


def compress(matrix: np.ndarray, nstates: int, weights: np.ndarray | None = None) -> PatternData:
    """Compress an (ntax, nsites) code matrix into GARLI-ordered unique patterns."""
    matrix = np.ascontiguousarray(matrix, dtype=np.uint8)
    ntax, nsites = matrix.shape
    if weights is None:
        weights = np.ones(nsites, dtype=np.int64)
    cols = matrix.T  # (nsites, ntax)
    uniq, inv = np.unique(cols, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    counts = np.bincount(inv, weights=weights, minlength=uniq.shape[0]).astype(np.int64)
    if nstates == 4:
        ns = _num_states_dna(uniq)
    else:
        ns = _num_states_nstate(uniq, nstates)
    keep = (ns > 0) & (counts > 0)
    uniq, counts, ns = uniq[keep], counts[keep], ns[keep]
    # np.unique already orders the columns lexicographically; a stable sort on
    # numStates reproduces SitePattern::operator< (datamatr.cpp:52-72).
    order = np.argsort(ns, kind="stable")
    uniq, counts, ns = uniq[order], counts[order], ns[order]
    last_const = int(np.sum(ns == 1)) - 1
    const_states = np.zeros(uniq.shape[0], dtype=np.int32)
    if last_const >= 0:
        cc = uniq[: last_const + 1]
        if nstates == 4:
            const_states[: last_const + 1] = np.bitwise_and.reduce(cc, axis=1)
        else:
            for p in range(last_const + 1):
                obs = cc[p][cc[p] != nstates]
                const_states[p] = obs[0] if obs.size else nstates
    return PatternData(
        nstates=nstates,
        tips=np.ascontiguousarray(uniq.T, dtype=np.uint8),
        counts=counts.astype(np.int32),
        last_const=last_const,
        const_states=const_states,
        nsites=int(weights.sum()),
    )
