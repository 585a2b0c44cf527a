"""garli_b200 -- a B200-native likelihood engine for GARLI's scoring path.

Felsenstein pruning of conditional likelihood arrays with per-site rescaling,
the root log-likelihood reduction and branch-length derivatives for the
Newton-Raphson optimiser, as hand-written sm_100a kernels behind a C ABI
(include/garli_b200.h) that mirrors GARLI's CalculationManager operation lists.
"""
__all__ = ["engine", "patterns", "synth", "treeio", "build"]
