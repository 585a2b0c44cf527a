"""Host-side encoding (datamatr.cpp PatternManager) and the C-ABI surface (no GPU)."""
import ctypes as C
import os
import re

import numpy as np

from garli_b200 import engine, patterns, synth, treeio

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_compress_orders_constant_patterns_first():
    m = patterns.dna_chars_to_masks(["AACGT?", "AACGTA", "AATGTN", "AAC-TA"])
    pd = patterns.compress(m, 4)
    assert pd.counts.sum() == 6
    # constant: A (x2), G with a gap, T, and "?A?A" (missing entries do not break constancy)
    assert pd.last_const == 3
    assert list(pd.const_states[: pd.last_const + 1]) == [1, 4, 8, 1]
    # the constant A pattern absorbed both A columns
    assert pd.counts[0] == 2
    # every compressed pattern is a column of the input
    cols = {bytes(c) for c in m.T}
    assert all(bytes(pd.tips[:, p]) in cols for p in range(pd.npat))


def test_compress_partial_ambiguity_constant():
    # R = A|G with A everywhere else -> constant (AND non-empty), state A
    m = patterns.dna_chars_to_masks(["A", "R", "A"])
    pd = patterns.compress(m, 4)
    assert pd.last_const == 0 and pd.const_states[0] == 1


def test_all_missing_columns_dropped():
    m = patterns.dna_chars_to_masks(["A?", "C?", "G-"])
    pd = patterns.compress(m, 4)
    assert pd.npat == 1 and pd.counts.sum() == 1


def test_newick_to_garli_layout():
    c3, dl = treeio.to_garli(treeio.parse_newick("(1:0.1,(2:0.2,3:0.3):0.05,4:0.4);"))
    assert c3.shape == (6, 3)
    assert list(c3[0]) == [1, 5, 4]
    assert list(c3[5]) == [2, -1, 3]
    assert dl[5] == 0.05 and dl[4] == 0.4


def test_yule_tree_is_valid():
    rng = np.random.default_rng(0)
    c3, dl = synth.yule_tree(50, rng, 0.1)
    seen = []
    for n in range(c3.shape[0]):
        seen += [int(c) for c in c3[n] if c >= 0]
    assert sorted(seen) == list(range(1, 98))
    assert (c3[1:51] == -1).all() and (dl[1:] > 0).all()


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "garli_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gb[mt]?_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = engine.lib()
    names = _header_functions()
    assert len(names) > 40
    for n in names:
        assert hasattr(L, n), n
        assert n in engine.SIGNATURES, n


def test_argument_checks_without_device():
    L = engine.lib()
    det = engine.InstanceDetails()
    # rejected before any device is touched
    assert L.gb_create_instance(11, 27, 5, 100, 1, 20, 4, 0, 1, C.byref(det)) == -7
    assert L.gb_create_instance(1, 27, 4, 100, 1, 20, 4, 0, 1, C.byref(det)) == -5
    assert L.gb_create_instance(11, 27, 4, 100, 1, 20, 9, 0, 1, C.byref(det)) == -5
    assert L.gb_finalize_instance(12345) == -4
    assert L.gbt_score(999, 0, (C.c_double * 3)()) == -4


def test_new_entry_points_reject_bad_handles_and_sizes_without_device():
    """Batched pass, population layer, device eigensolver, tensor-core and FP64
    buffer switches, and the allocation-free edge: invalid handles and sizes are
    rejected before any device work."""
    L = engine.lib()
    d3 = (C.c_double * 12)()
    i4 = (C.c_int * 4)()
    assert L.gb_batch_newton(4321, None, 0, None, 0, None, 1, 3, 16, 0.01, 1e-8, 100.0, d3) == -4
    assert L.gb_set_batch_tuning(4321, 1, 1) == -4
    assert L.gb_get_batch_tuning(4321, i4) == -4
    assert L.gb_set_tensor_cores(4321, 1) == -4
    assert L.gb_set_buffer_precision(4321, 10, 1) == -4
    assert L.gb_set_eigen_from_rate_matrices(4321, 1, i4, d3, d3, d3, None) == -4
    assert L.gbp_score_candidates(4321, 1, i4, d3, i4, 0.01, 0, d3, d3) == -4
    assert L.gbp_get_counters(4321, (C.c_longlong * 6)()) == -4
    assert L.gbp_destroy(4321) == -4
    assert L.gbp_create(4321, 8, i4, d3, 10) == -4
    # the allocation-free edge checks its pattern limit first
    assert L.gb_edge_loglik_static(0, 4, (1 << 22) + 1, None, None, None, None, None, None, None, None, None, None,
                                   0.0, 0, 1, None, None) == -5
    assert L.gb_edge_loglik_static(0, 9, 100, None, None, None, None, None, None, None, None, None, None, 0.0, 0, 1,
                                   None, None) == -5
