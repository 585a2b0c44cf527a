/*
 * garli_oracle.h -- CPU restatement of GARLI's likelihood hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle for the
 * garli_b200 engine: tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg of bench.py may load it; the engine itself never does.
 *
 * It restates, in plain C, the FP64 (non SINGLE_PRECISION_FLOATS) CPU path
 * of GARLI 2.2 (garli/trunk/src):
 *   model.cpp   UpdateQMat :233, UpdateQMatCodon :442, UpdateQMatAminoAcid :735,
 *               CalcEigenStuff :827, CalcDerivatives :1271, AltCalcPmat :1469,
 *               DiscreteGamma :2170 (+ PointNormal/IncompleteGamma/LnGamma/PointChi2)
 *   tree.cpp    rescale constants :149-172, RescaleRateHet :3370,
 *               RescaleRateHetNState :3492, ConditionalLikelihoodRateHet :3600,
 *               GetTotalScore :3815, UpdateCLAs :3905, Score :4003,
 *               SweepDirtynessOverTree :4247, GetScorePartial* :5597/:6040/:6172/:6273,
 *               CalcFullCLA* :7668/:7843/:7912/:8082/:8291/:8537
 *   optimization.cpp  OptimizeAllBranches :97, OptimizeBranchLength :777,
 *               RecursivelyOptimizeBranches :1042, CalcDerivativesRateHet :1099,
 *               NewtonRaphsonOptimizeBranchLength :1359, GetDerivsPartial* :2412/:3063 (+NState)
 *   sequencedata.cpp  MakeAmbigStrings :278 (tip ambiguity strings)
 *
 * Node numbering follows GARLI: node 0 is the (trifurcating) root, nodes
 * 1..ntax are the tips, ntax+1 .. 2*ntax-3 the other internal nodes.
 */
#ifndef GARLI_ORACLE_H
#define GARLI_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* ---- model (model.cpp) ---- */
void or_gtr_qmat(const double rel[6], const double pi[4], double *Q, double *blen_mult);
void or_aa_qmat(const double *exch190, const double *pi20, double *Q, double *blen_mult);
int  or_codon_qmat(double kappa, double omega, const double *pi61, double *Q, double *blen_mult);
int  or_codon_qmat6(const double *rel6, double omega, const double *pi61, double *Q, double *blen_mult);
/* Eigen system of a time-reversible Q (Q_ij = s_ij pi_j).  eval unscaled. */
int  or_eigen(int S, const double *Q, const double *pi, double *eval, double *U, double *Uinv);
/* GARLI DiscreteGamma (mean-of-category rates, median=false). */
void or_discrete_gamma(double alpha, int ncat, double *rates);
/* P(t), dP/dt, d2P/dt2 for all rate categories, laid out [r][i][j]. */
void or_pmats(int S, int R, const double *eval_scaled, const double *U, const double *Uinv,
              const double *rateMults, double pinv, int has_pinv, double t,
              double *P, double *D1, double *D2);

/* ---- tree engine ---- */
typedef struct OrTree OrTree;

/* child3[n*3+{0,1,2}] = left, middle (root only, else -1), right; -1 for tips.
 * tips[t*npat + p] for tip t=1..ntax stored at row t-1: DNA = 4-bit mask (A=1,C=2,G=4,T=8),
 * NState = state index 0..S-1, S = missing.  constStates: DNA mask / NState state index. */
OrTree *or_tree_new(int ntax, int S, int R, int npat, const int *child3, const double *dlen,
                    const unsigned char *tips, const int *counts, int lastConst,
                    const int *constStates);
void   or_tree_free(OrTree *t);
void   or_tree_set_model(OrTree *t, const double *eval_scaled, const double *U, const double *Uinv,
                         const double *pi, const double *rateMults, const double *rateProbs,
                         double pinv, int has_pinv);
void   or_tree_set_rescale_every(OrTree *t, int every);
int    or_tree_get_rescale_every(const OrTree *t);
double or_tree_score(OrTree *t, int rootNode);
int    or_tree_derivs(OrTree *t, int nd, double *lnl_d1_d2);
double or_tree_nr_optimize(OrTree *t, double precision, int nd);
double or_tree_optimize_all(OrTree *t, double precision);
void   or_tree_set_blen(OrTree *t, int nd, double v);
double or_tree_get_blen(const OrTree *t, int nd);
void   or_tree_dirty_all(OrTree *t);
double or_tree_lnl(const OrTree *t);
/* which: 0 = Down, 1 = UpLeft, 2 = UpRight.  Returns -1 if that CLA is dirty/unallocated. */
int    or_tree_get_cla(const OrTree *t, int nd, int which, double *arr, int *mult);
int    or_tree_cla_rank(const OrTree *t, int nd, int which);
int    or_tree_cla_dirty(const OrTree *t, int nd, int which);
/* per-pattern unscaled log-likelihoods of the last root score (NULL before any score) */
int    or_tree_site_lnl(const OrTree *t, double *out);
long   or_tree_cla_count(const OrTree *t);
long   or_tree_deriv_count(const OrTree *t);
void   or_set_threads(int n);
int    or_get_threads(void);

/* rescale constants (tree.cpp:163-172), exposed for tests */
void   or_rescale_tables(int *incr, double *thresh, double *mult);

#ifdef __cplusplus
}
#endif
#endif
