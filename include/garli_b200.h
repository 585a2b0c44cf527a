/*
 * garli_b200.h -- C ABI of the B200 likelihood engine for GARLI.
 *
 * The engine replaces the compute backend under GARLI's CalculationManager
 * (garli/trunk/src/calculationmanager.h, subsetcalculationmanager.cpp), i.e.
 * the beagle-lib calls GARLI issues today, with hand-written sm_100a kernels.
 * Every entry point takes plain pointers and sizes, returns an int status
 * (GB_SUCCESS or a negative GB_ERROR_* code) and is synchronous from the
 * caller's point of view unless documented otherwise, exactly like the
 * beagle calls it replaces (calculationmanager.cpp:84-125 maps those codes).
 *
 * Index spaces (calculationmanager.h:1147-1215):
 *   buffer index b in [0, tipCount) ............ tip b (GARLI taxon number b+1)
 *   buffer index b in [tipCount, tipCount+partialsBufferCount) .. a CLA buffer;
 *                                                 its scaler array shares the index
 *   matrix index m in [0, matrixBufferCount) .... a P(t) matrix set (P, dP/dt, d2P/dt2)
 *   eigen index e in [0, eigenBufferCount) ...... an eigensystem of Q
 */
#ifndef GARLI_B200_H
#define GARLI_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (beagle-compatible meaning, BEAGLE_ERROR_*) ---- */
#define GB_SUCCESS 0
#define GB_ERROR_GENERAL (-1)
#define GB_ERROR_OUT_OF_MEMORY (-2)
#define GB_ERROR_UNIDENTIFIED_EXCEPTION (-3)
#define GB_ERROR_UNINITIALIZED_INSTANCE (-4)
#define GB_ERROR_OUT_OF_RANGE (-5)
#define GB_ERROR_NO_RESOURCE (-6)
#define GB_ERROR_NO_IMPLEMENTATION (-7)
#define GB_ERROR_FLOATING_POINT (-8)
/* GARLI's throw(1) from RescaleRateHet (tree.cpp:3442,3448): a site fell below
 * 1e-190 between rescalings; the caller lowers rescaleEvery by 2, dirties all
 * CLAs and rescores (tree.cpp:4077-4090). */
#define GB_ERROR_RESCALE_RETRY (-9)
#define GB_ERROR_NO_DEVICE (-10)

/* ---- instance flags ---- */
/* plain form: FP64 CLAs with GARLI's rank-gated, e-based integer rescaling
 * (tree.cpp:149-172, :3370); reproduces GARLI's CPU lnL and scaler counts */
#define GB_FLAG_PLAIN_FP64 (1L << 0)
/* precision form: FP32 CLA storage, per-site power-of-two rescaling after
 * every CLA update (int32 exponent counts), FP64 P(t), sums and Newton step */
#define GB_FLAG_MIXED_FP32 (1L << 1)

typedef struct {
    int resourceNumber; /* CUDA device ordinal */
    long flags;         /* the GB_FLAG_* form in use */
    int paddedPatterns; /* patterns rounded up to the kernel tile */
    long long deviceBytes;
    char deviceName[64];
} gb_instance_details;

/* ClaOperation, calculationmanager.h:39-52.  Child indices are buffer indices
 * (tips or CLA buffers); the matrix indices select the P(t) of each child's
 * branch.  opDepLevel orders the operations: every op of level k only reads
 * buffers written at levels < k (or clean buffers). */
typedef struct {
    int destClaIndex;
    int childClaIndex1;
    int childClaIndex2;
    int transMatIndex1;
    int transMatIndex2;
    int opDepLevel;
} gb_cla_operation;

/* TransMatOperation, calculationmanager.h:54-67 */
typedef struct {
    int destTransMatIndex;
    double edgeLength;
    int eigenIndex; /* modelIndex in GARLI: selects the eigensystem */
    int calcDerivs; /* also fill dP/dt and d2P/dt2 (model.cpp:1271) */
} gb_transmat_operation;

/* ScoringOperation, calculationmanager.h:91-105: the partial CLA on one side
 * of a branch, the child buffer on the other side, and that branch's matrix. */
typedef struct {
    int destClaIndex;   /* unused by the engine (GARLI passes the final scaler slot) */
    int childClaIndex1; /* "partial": always a CLA buffer */
    int childClaIndex2; /* child: tip or CLA buffer */
    int transMatIndex;
    int derivatives;    /* also return d1 and d2 (optimization.cpp:1099) */
} gb_scoring_operation;

/* ---- instance management (beagleCreateInstance / beagleFinalizeInstance) ---- */
int gb_get_device_count(void);
/* subsetcalculationmanager.cpp:105 beagleCreateInstance; stateCount 4, 20 or 61,
 * categoryCount 1..8.  Returns an instance handle (>= 0) or an error code. */
int gb_create_instance(int tipCount, int partialsBufferCount, int stateCount, int patternCount,
                       int eigenBufferCount, int matrixBufferCount, int categoryCount,
                       int resourceNumber, long flags, gb_instance_details *details);
int gb_finalize_instance(int instance);

/* ---- data (subsetcalculationmanager.cpp:177-230) ---- */
/* beagleSetTipStates: DNA codes are 4-bit masks (A=1,C=2,G=4,T=8, 15 = missing,
 * sequencedata.cpp:672); NState codes are state indices, stateCount = missing. */
int gb_set_tip_states(int instance, int tipIndex, const unsigned char *codes);
/* beagleSetPatternWeights: integer pattern counts (datamatr.cpp PatternManager) */
int gb_set_pattern_weights(int instance, const int *counts);
/* constant patterns 0..lastConst and their states (datamatr.cpp:334-376);
 * needed for the +I term of GetScorePartial* (tree.cpp:6118-6130) */
int gb_set_constant_patterns(int instance, int lastConst, const int *constStates);

/* ---- model (subsetcalculationmanager.cpp:232-300, :765-800) ---- */
int gb_set_state_frequencies(int instance, const double *freqs);
/* beagleSetCategoryRates: GARLI's rateMults (model.cpp:2170) */
int gb_set_category_rates(int instance, const double *rates);
/* beagleSetCategoryWeights: GARLI's rateProbs = (1-pinv)/ncat (model.cpp:2199) */
int gb_set_category_weights(int instance, const double *weights);
/* proportion of invariant sites; hasPinv=0 reproduces NoPinvInModel() */
int gb_set_invariant_sites(int instance, double pinv, int hasPinv);
/* beagleSetEigenDecomposition: U (row-major S*S), U^-1, eigenvalues already
 * multiplied by GARLI's blen_multiplier (model.cpp:845) */
int gb_set_eigen_decomposition(int instance, int eigenIndex, const double *eigenVectors,
                               const double *inverseEigenVectors, const double *eigenValues);
/* Model slots: eigen index e also selects the state frequencies, category
 * rates, category weights and invariant-sites term that P(t) (transition
 * matrix operations with eigenIndex e) and edge evaluations under slot e use.
 * The four instance-wide setters above write every slot; this one writes
 * slot eigenIndex only (slot 0 is also the instance-wide model).  One tree
 * scored under several models at once (optimization.cpp:244-268, a Model per
 * candidate parameter value) keeps each model in its own slot. */
int gb_set_model_slot(int instance, int eigenIndex, const double *freqs, const double *rates,
                      const double *weights, double pinv, int hasPinv);

/* ---- operations ---- */
/* Model::CalcEigenStuff (model.cpp:827-856) on the device, FP64, one CTA per
 * model: for each c, the eigensystem of the reversible rate matrix
 * Q[c*S*S ...] (row-major) with stationary frequencies pi[c*S ...] (all > 0)
 * into eigen slot eigenIndices[c], eigenvalues multiplied by blenMults[c]
 * (model.cpp:845).  Symmetrised by diag(pi)^1/2 and diagonalised by cyclic
 * Jacobi; sweepsOut[c] (optional) = Jacobi sweeps used.  For the many models
 * of a model-parameter optimisation at once (optimization.cpp:332-776). */
int gb_set_eigen_from_rate_matrices(int instance, int count, const int *eigenIndices, const double *Q,
                                    const double *pi, const double *blenMults, int *sweepsOut);
/* beagleUpdateTransitionMatrices (subsetcalculationmanager.cpp:232): P(t) and,
 * if requested, dP/dt and d2P/dt2 in FP64 on the device (model.cpp:1271,:1469) */
int gb_update_transition_matrices(int instance, const gb_transmat_operation *ops, int count);
/* beagleSetTransitionMatrix: host-supplied FP64 P (row-major [cat][from][to]) */
int gb_set_transition_matrix(int instance, int matrixIndex, const double *P, const double *D1,
                             const double *D2);
/* beagleUpdatePartials + beagleAccumulateScaleFactors
 * (subsetcalculationmanager.cpp:595-640).  Operations are executed level by
 * level (opDepLevel, ascending); ops of one level run in one batched launch.
 * In the plain form the engine applies GARLI's rescale rule per destination
 * buffer: rank = 2 (tip-tip), child+2 (internal-tip), 2+L+R (internal-internal),
 * rescale when rank >= rescaleEvery (tree.cpp:3991, :7665-8598).  Asynchronous:
 * a GB_ERROR_RESCALE_RETRY condition is reported by the next call that
 * returns results. */
int gb_update_partials(int instance, const gb_cla_operation *ops, int count, int rescaleEvery);
/* CLA launch shapes, chosen by timing on the first op list of >= 2 levels and
 * >= 2^17 pattern-updates (per-tree precision 4-state: the blocks per SM a level
 * launch aims at, of 4, 8, 16, 32; n-state CUDA-core kernel: patterns per
 * tile, a power of two from the warp task -- 16 patterns for 20 states, 8
 * for 61 -- up to 64 and to 8 tasks of one rate category each; a set value is
 * rounded up to the next such tile and capped).  Each pattern's arithmetic does not depend on the
 * shape.  0 re-arms the tuning for the next call, -1 keeps the value, > 0
 * sets it; a call without a 0 turns the tuning off.  out3 = current level
 * target, n-state tile, tuning pending. */
int gb_set_cla_tuning(int instance, int levelBlocksPerSm, int nstateTilePatterns);
int gb_get_cla_tuning(int instance, int *out3);
/* beagleCalculateEdgeLogLikelihoods (subsetcalculationmanager.cpp:765-901):
 * returns lnL and, when op->derivatives, d1 and d2 in outLnL[0..2]. */
int gb_calculate_edge(int instance, const gb_scoring_operation *op, double *out);
/* count edge evaluations with one synchronisation: edge k under model slot
 * modelSlots[k] (NULL: slot 0 for all); out[3k], out[3k+1], out[3k+2] = lnL,
 * d1, d2 of edge k.  A rescale-retry or range condition of any edge is
 * reported for the whole call. */
int gb_calculate_edges(int instance, const gb_scoring_operation *ops, const int *modelSlots, int count,
                       double *out);
/* beagleGetSiteLogLikelihoods of the last gb_calculate_edge (unscaled per pattern) */
int gb_get_site_log_likelihoods(int instance, double *out);
/* beagleGetSiteDerivatives (subsetcalculationmanager.cpp:440): per pattern
 * d lnL_p / dt and d2 lnL_p / dt2 of the last edge evaluation, if it was a
 * derivative one (GB_ERROR_GENERAL otherwise); the pattern-count-weighted sums
 * are that evaluation's d1 and d2 */
int gb_get_site_derivatives(int instance, double *outFirst, double *outSecond);
/* debug read-back (beagleGetPartials / beagleGetScaleFactors); CLA layout
 * [pattern][category][state], converted to FP64 */
int gb_get_partials(int instance, int bufferIndex, double *out);
int gb_get_scale_factors(int instance, int bufferIndex, int *out);
int gb_get_transition_matrix(int instance, int matrixIndex, int which, double *out);
/* rescale rank the engine tracks for a CLA buffer (condlike.h rescaleRank) */
int gb_get_rescale_rank(int instance, int bufferIndex);
/* raw device pointer and size of the CLA pool (for peer copies / profiling) */
int gb_get_partials_pool(int instance, void **devicePtr, long long *bytes);
/* out[0..2] = partialsBufferCount, matrixBufferCount, eigenBufferCount */
int gb_get_instance_capacity(int instance, int *out);
/* out[0..4] = tipCount, partialsBufferCount, stateCount, categoryCount, patternCount */
int gb_get_instance_shape(int instance, int *out);
/* number of engine kernels launched since the instance was created */
long long gb_get_launch_count(int instance);
int gb_synchronize(int instance);
/* message of the last failing call on this thread */
const char *gb_last_error(void);
/* instrumentation: the instance's CUDA stream (cudaStream_t) and optional
 * CUDA-event timing of the CLA and edge kernels on that stream;
 * timing out[0..6] = CLA ms, CLA launches, pattern-updates, edge ms, edge evaluations,
 * algorithmic bytes of the timed CLA launches, FP64 instructions of the timed
 * CLA launches (n-state CUDA-core kernel; 0 for 4 states) */
int gb_get_stream(int instance, void **stream);
int gb_set_kernel_timing(int instance, int on);
int gb_get_kernel_timing(int instance, double *out);

/* ---- graph-resident branch optimisation ----
 * One entry per branch of an OptimizeAllBranches pass (optimization.cpp:97,
 * :1042), in traversal order: the CLA updates that branch's derivatives need
 * (ops[firstOp .. firstOp+opCount), a ClaOperation list as for
 * gb_update_partials), then the Newton-Raphson loop on the branch between
 * partialIndex (the CLA on the ancestor's side) and childIndex, whose length
 * is the device copy for transMatIndex. */
typedef struct {
    int partialIndex;
    int childIndex;
    int transMatIndex;
    int firstOp;
    int opCount;
} gb_nr_branch;
/* device copy of the branch length behind each matrix index */
int gb_set_branch_lengths(int instance, const double *lengths, int count);
int gb_get_branch_lengths(int instance, double *lengths, int count);
/* Runs the whole pass as one CUDA graph (cached while the plan, the model and
 * the rank state are unchanged): no host round trip between Newton iterations
 * or branches.  Every step of the loop is NewtonRaphsonOptimizeBranchLength
 * (optimization.cpp:1359-1971) in FP64 on the device; the P(t) of each matrix
 * always matches its device length on return.  out[0] = summed estimated
 * improvement, out[1] = lnL of the last derivative evaluation, out[2] = number
 * of derivative evaluations.  Returns GB_ERROR_RESCALE_RETRY if a CLA of the
 * pass crossed GARLI's rescale bail-out (the caller restores the lengths,
 * lowers rescaleEvery and reruns). */
int gb_newton_pass(int instance, const gb_nr_branch *branches, int branchCount, const gb_cla_operation *ops,
                   int opCount, int rescaleEvery, double precision, double minLength, double maxLength,
                   double *out);
/* 1 (default): 4-state passes run as one cooperative persistent kernel over a
 * device command queue; 0: as a CUDA graph with a conditional WHILE node per branch */
int gb_set_pass_mode(int instance, int persistent);
/* instrumentation: phase timestamps of the persistent pass kernel, each
 * (phase code << 56) | %globaltimer ns, and of the batched pass kernel, each
 * (phase code << 56) | (active candidates << 40) | low 40 bits of %globaltimer;
 * capacity 0 switches recording off */
int gb_set_pass_trace(int instance, int capacity);
int gb_get_pass_trace(int instance, unsigned long long *out, int count);
/* Newton state of one matrix after a pass: length, improvement, lnL, d1, d2, evaluations */
int gb_get_newton_state(int instance, int matrixIndex, double *out6);

/* precision form, 20 states (up to 4 categories) and 61 states (one
 * category): 1 (default for 61 states) = CLA updates of the FP32 segment on the tensor cores
 * (tcgen05.mma kind::i8: the CLA as 4 and P(t) as 5 base-256 digits over
 * per-row power-of-two scales, exact 32-bit integer accumulation, each P.CLA
 * product within 2.5e-10 of the CLA row's largest entry); 0 (default for 20
 * states, where it is the faster) = the CUDA-core FP64-arithmetic kernel.  A pattern whose product maximum falls below 2^-64
 * switches the instance to the CUDA-core kernel (the score that saw it returns
 * GB_ERROR_RESCALE_RETRY, and the tree drivers redo it). */
int gb_set_tensor_cores(int instance, int on);

/* ---- batched candidate scoring and branch optimisation (4 states) ----
 * A GA generation's candidates (population.cpp:4532-4589: each mutated
 * individual is rescored, tree.cpp:4003, and the branches around its move are
 * optimised, optimization.cpp:882-884 -> NewtonRaphsonOptimizeBranchLength,
 * :1359-1971) run from a device command queue as one CUDA graph: the
 * precision form's CLA levels and per-step coefficient passes as launches of
 * their own, its lockstep Newton runs (and the plain form's whole queue) in a
 * persistent kernel.
 * ops[0..opCount): every candidate's dirty CLA updates, levelled by opDepLevel
 * (uneven counts per candidate are fine; buffers may be shared read-only).
 * steps[c * stepsPerCandidate + k]: step k of candidate c -- optionally the CLA
 * update stepOps[claOp] (the partial of this step, which may read lengths
 * optimised at earlier steps), then Newton-Raphson on the branch between
 * partialIndex and childIndex whose length is the device copy for
 * transMatIndex (gb_set_branch_lengths).  All candidates take step k in
 * lockstep; the matrices hold the optimised P(t) on return.
 * out[4c .. 4c+3] = lnL at the starting lengths (the candidate's rescore),
 * lnL at the optimised lengths, summed estimated improvement, derivative
 * evaluations.  Work-item sizes are autotuned on the first call with
 * candidates.  candidateCount = 0 runs the CLA updates only (e.g. a parent
 * tree's CLAs into FP64 buffers, gb_set_buffer_precision). */
typedef struct {
    int claOp;
    int partialIndex;
    int childIndex;
    int transMatIndex;
} gb_batch_step;
int gb_batch_newton(int instance, const gb_cla_operation *ops, int opCount, const gb_cla_operation *stepOps,
                    int stepOpCount, const gb_batch_step *steps, int candidateCount, int stepsPerCandidate,
                    int rescaleEvery, double precision, double minLength, double maxLength, double *out);
/* precision form: store CLA buffer bufferIndex in FP64 for every pattern (1) or
 * in the instance's FP64/FP32 segments (0).  An FP64 buffer occupies its own
 * slot and the next one (bufferIndex + 1 must be left unused); it is read and
 * written by gb_batch_newton only (and read back by gb_get_partials).  For CLAs
 * many candidates share, such as a GA generation's parent tree. */
int gb_set_buffer_precision(int instance, int bufferIndex, int fp64);
/* work-item sizes: CLA tiles (64 patterns at 4 categories) and edge chunks
 * (256 patterns) per CTA work item; 0, 0 = autotune on the next call */
int gb_set_batch_tuning(int instance, int tilesPerItem, int chunksPerItem);
/* out[0..2] = tiles per item, chunks per item, 1 if the pass replays a CUDA graph */
int gb_get_batch_tuning(int instance, int *out3);
/* instrumentation (while gb_set_kernel_timing is on): out[0] = CUDA-event ms of
 * the batched pass launches on the instance stream, out[1] = launches timed */
int gb_get_batch_timing(int instance, double *out2);
/* instrumentation: with phase timing on, every launch of a batched pass is
 * bracketed by its own CUDA events and launched directly (no graph);
 * out[2k] = accumulated ms, out[2k+1] = launches of phase k: 0 = CLA levels,
 * 1 = coefficient passes, 2 = Newton / score runs.  No counterpart in the
 * reference (GARLI has no device timing). */
int gb_set_batch_phase_timing(int instance, int on);
int gb_get_batch_phase_timing(int instance, double *out6);

/* ---- population layer: a GA generation's candidates on one instance ----
 * A C++ restatement of how GARLI scores the candidates of a generation: each
 * is the base tree after one SPR/NNI move (Tree::SPRMutate, tree.cpp:3148-3248)
 * and shares every unchanged CLA with it (copy-on-write holders,
 * clamanager.h); it is rescored and the three branches at the move's
 * connector nd are optimised in GARLI's order nd->left, nd, nd->right
 * (optimization.cpp:882-884).  CLAs are identified by content (subtree,
 * tips and branch lengths), so only changed ones are recomputed.
 * gbp_create: base tree in GARLI layout; matrixCount <= the instance's
 * matrixBufferCount matrix slots are used.  The instance must hold the model
 * (gb_set_eigen_decomposition etc.) and the tips. */
int gbp_create(int instance, int ntax, const int *child3, const double *dlen, int matrixCount);
int gbp_destroy(int pop);
/* the instance's model changed: recompute the base tree's CLAs on the next call */
int gbp_invalidate(int pop);
/* candidate c: child3s[c*nnodes*3 ...], dlens[c*nnodes ...] (GARLI layout, the
 * base tree's node numbers), connectors[c] = the move's connector node nd.
 * sequential = 0: all candidates in one gb_batch_newton pass; 1: GARLI's
 * per-tree path, one candidate after another with a host Newton loop.
 * out[4c .. 4c+3] as gb_batch_newton; lengthsOut[3c .. 3c+2] = optimised
 * lengths of nd->left, nd, nd->right. */
int gbp_score_candidates(int pop, int candidateCount, const int *child3s, const double *dlens,
                         const int *connectors, double precision, int sequential, double *out,
                         double *lengthsOut);
/* last call: [0] CLA updates (the per-step partials included), [1] pattern-updates,
 * [2] derivative evaluations, [4] edge evaluations (derivative evaluations + the
 * final scores), [5] algorithmic device-memory bytes of the precision form's
 * batched pass, per pattern at R rate categories: a CLA read 16R + 4 B (FP32
 * + scale exponent), 32R + 4 B for an FP64 parent-tree CLA, 1 B for a tip;
 * 16R + 4 B per CLA update written; 8(1 + 3R) + 4 B per coefficient pattern
 * written; 8(1 + 3R) + 12 B per edge-evaluation pattern (at R = 4: 68, 132,
 * 108, 116); [3] base-tree CLA updates since creation */
int gbp_get_counters(int pop, long long *out6);
/* the last call's algorithmic device-memory bytes (out6[5]) split by phase:
 * out[0] CLA levels, out[1] coefficient passes (step partials), out[2] Newton
 * and score sweeps */
int gbp_get_byte_counters(int pop, double *out3);

/* ---- edge evaluation without device allocation ----
 * No counterpart in the reference: GARLI's beagle build lets beagle allocate.
 * For callers that cannot call cudaMalloc -- a plugin inside a host
 * application that owns every device allocation through its own pool, where an
 * allocation would bypass the host's accounting or fail once the pool has
 * reserved the memory, or code on a latency-critical thread that must not take
 * cudaMalloc's implicit device synchronisation -- this evaluates lnL (and d1, d2) across one branch
 * of 4-state data held entirely in the caller's device arrays, with the plain
 * FP64 form's per-site arithmetic (GARLI's e-based integer scalers).  It
 * allocates nothing: its per-block partial sums live in a fixed 96 KiB array
 * that the library keeps on every GPU that loads it, until the process exits.
 *   partial, child ........ FP64 CLAs, layout [pattern][category][4]
 *   childTipCodes ......... instead of child (pass child = NULL): 4-bit masks per pattern
 *   partialScalers, childScalers: int per pattern (childScalers only with a CLA child)
 *   matrices .............. [P | dP | d2P], each [category][from][to] (dP, d2P only
 *                           read when derivatives != 0)
 *   stateFrequencies[4], categoryWeights[categoryCount], patternCounts[patternCount],
 *   constantStates ........ 4-bit mask of a constant pattern, -1 otherwise (read when hasPinv)
 *   out ................... device array of 3 doubles: lnL, d1, d2 (d1 = d2 = 0 without derivatives)
 * All pointers are device pointers on device resourceNumber.  The call is
 * asynchronous on `stream` (a cudaStream_t; NULL = the default stream).
 * patternCount above GB_STATIC_EDGE_MAX_PATTERNS is rejected with
 * GB_ERROR_OUT_OF_RANGE.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress): make that first call before any
 * stream capture.  The address is kept until the process exits: a
 * cudaDeviceReset on that device invalidates it, and the entry point must not
 * be called after one.  Every call shares the one array, so calls that overlap on
 * the GPU (unordered streams) race; calls ordered on one stream do not. */
#define GB_STATIC_EDGE_MAX_PATTERNS 4194304
int gb_edge_loglik_static(int resourceNumber, int categoryCount, int patternCount, const double *partial,
                          const int *partialScalers, const double *child, const int *childScalers,
                          const unsigned char *childTipCodes, const double *matrices,
                          const double *stateFrequencies, const double *categoryWeights,
                          const int *patternCounts, const int *constantStates, double pinv, int hasPinv,
                          int derivatives, void *stream, double *out);

/* ---- host model math (model.cpp), used by the tree layer and by callers ---- */
/* Model::UpdateQMat GTR branch (model.cpp:256-293) */
int gbm_gtr_qmat(const double *rel6, const double *pi4, double *Q, double *blenMult);
/* Model::UpdateQMatAminoAcid, estimated exchangeabilities (model.cpp:735-779) */
int gbm_aa_qmat(const double *exch190, const double *pi20, double *Q, double *blenMult);
/* Model::FillQMatLookup + UpdateQMatCodon, GY94 (model.cpp:296-687) */
int gbm_codon_qmat(double kappa, double omega, const double *pi61, double *Q, double *blenMult);
/* the same with six nucleotide-pair rates (AC, AG, AT, CG, CT, GT; nst = 6) */
int gbm_codon_qmat6(const double *rel6, double omega, const double *pi61, double *Q, double *blenMult);
/* Model::CalcEigenStuff (model.cpp:827-856) for a reversible Q */
int gbm_eigen(int stateCount, const double *Q, const double *pi, double *eigenValues,
              double *eigenVectors, double *inverseEigenVectors);
/* Model::DiscreteGamma (model.cpp:2170-2201), mean-of-category rates */
int gbm_discrete_gamma(double alpha, int categoryCount, double *rates);

/* ---- tree layer: CalculationManager + Tree::Score / branch optimisation ----
 * A C++ restatement of GARLI's holder bookkeeping (clamanager.h, treenode
 * claIndexDown/UL/UR), dependency-levelled operation assembly
 * (CalculationManager::DetermineRequiredOperations, calculationmanager.cpp:522-670)
 * and the Newton-Raphson branch optimiser (optimization.cpp:1359-1971) on top
 * of the instance API above.  Node numbering is GARLI's: 0 = trifurcating
 * root, 1..ntax tips, ntax+1..2*ntax-3 internal; child3 = (left, middle|-1,
 * right) per node. */
int gbt_create(int instance, int ntax, const int *child3, const double *dlen);
int gbt_destroy(int tree);
/* model of the tree: eigen system (unscaled eigenvalues), blen multiplier,
 * frequencies, category rates/weights and pinv */
int gbt_set_model(int tree, const double *eigenValues, const double *eigenVectors,
                  const double *inverseEigenVectors, double blenMult, const double *pi,
                  const double *rates, const double *weights, double pinv, int hasPinv);
/* Tree::Score (tree.cpp:4003) with the rescale retry loop; out[0] = lnL */
int gbt_score(int tree, int rootNode, double *out);
/* Tree::CalcDerivativesRateHet(nd->anc, nd) (optimization.cpp:1099): out = lnL, d1, d2 */
int gbt_derivatives(int tree, int node, double *out);
/* Tree::SetBranchLength + SweepDirtynessOverTree (tree.cpp:4247) */
int gbt_set_branch_length(int tree, int node, double length);
int gbt_get_branch_lengths(int tree, double *dlen);
/* Tree::MakeAllNodesDirty */
int gbt_make_all_dirty(int tree);
/* NewtonRaphsonOptimizeBranchLength (optimization.cpp:1359); out[0] = estimated improvement */
int gbt_optimize_branch(int tree, double precision, int node, double *out);
/* OptimizeAllBranches (optimization.cpp:97); out[0] = improvement, out[1] = final lnL */
int gbt_optimize_all_branches(int tree, double precision, double *out);
/* 1 (default): OptimizeAllBranches runs as one device graph (gb_newton_pass);
 * 0: the host drives each Newton iteration through gbt_derivatives */
int gbt_set_device_newton(int tree, int on);
int gbt_get_rescale_every(int tree);
int gbt_set_rescale_every(int tree, int every);
/* counters: [0] CLA ops issued, [1] pattern-updates (ops x patterns),
 * [2] edge evaluations, [3] scores, [4] rescale retries */
int gbt_get_counters(int tree, long long *out5);
/* CLA buffer index currently holding (node, which) with which 0=Down 1=UL 2=UR; -1 if dirty */
int gbt_cla_buffer(int tree, int node, int which);
/* Tree::Score at root 0 after MakeAllNodesDirty under count models at once
 * (one SetAndEvaluateParameter each, optimization.cpp:244-268): model k uses
 * eigen / model slot eigenIndices[k], matrices (k+1)*nnodes + node and CLA
 * buffers 3*(ntax-2) + k*(ntax-2) + j past the tip buffers; the tree's own
 * CLAs and P(t) stay as they are.  Needs partialsBufferCount >=
 * (3 + count)*(ntax-2) and matrixBufferCount >= (count+1)*nnodes.  lnl[k] =
 * the score under model k; a rescale retry redoes all (tree.cpp:4077-4090). */
int gbt_score_models(int tree, int count, const int *eigenIndices, double *lnl);
/* engine instance the tree runs on */
int gbt_get_instance(int tree);

/* ---- model-parameter optimisation (optimization.cpp:244-776, tree.cpp:7160-7410,
 * population.cpp:2566-2790) ----
 * GARLI's Model parameters of one tree, their setters and
 * Tree::OptimizeBoundedParameter.  Every candidate parameter value is a whole
 * model (Q, eigen system, discrete-gamma rates, pinv weights) scored by a full
 * rescore; evaluation points whose values are fixed before their scores are
 * needed (the bump, the first pair of points, the next pass's pair beside each
 * proposed value) are scored together through gbt_score_models, eigen systems
 * through gb_set_eigen_from_rate_matrices, and the decisions are GARLI's own in
 * GARLI's order. */
enum { GB_MODEL_NUCLEOTIDE = 0, GB_MODEL_AMINO_ACID = 1, GB_MODEL_CODON = 2 };
enum { GB_PARAM_ALPHA = 0, GB_PARAM_PINV = 1, GB_PARAM_STATE_FREQ = 2, GB_PARAM_REL_RATE = 3, GB_PARAM_OMEGA = 4 };
enum { GB_OPT_ALPHA = 1, GB_OPT_PINV = 2, GB_OPT_FREQS = 4, GB_OPT_RATES = 8, GB_OPT_OMEGA = 16 };
typedef struct {
    int kind;          /* GB_MODEL_* */
    int stateCount;    /* 4, 20 or 61 */
    int categoryCount; /* discrete-gamma categories (1: no rate heterogeneity) */
    int nst;           /* nucleotide / codon rate classes: 1, 2 (transition / transversion) or 6 */
    int hasPinv;
    double alpha, pinv;
    double maxPinv;    /* Model::maxPropInvar (model.cpp:1649): constant / all sites */
    double omega;      /* codon dN/dS */
    double rel[6];     /* AC AG AT CG CT GT, GT = 1 (model.h:1518-1531) */
    double pi[64];     /* state frequencies, stateCount used */
} gb_model_params;
/* optimiser for the model of tree; aaExchangeabilities (190, amino acids
 * only) stay fixed.  Installs the model as the tree's model (slot 0). */
int gbo_create(int tree, const gb_model_params *model, const double *aaExchangeabilities);
int gbo_destroy(int opt);
int gbo_get_model(int opt, gb_model_params *out);
int gbo_set_model(int opt, const gb_model_params *model);
/* Tree::OptimizeBoundedParameter(which, lowBound, highBound, setter,
 * targetScoreDigits) for parameter GB_PARAM_*; out[0] = lnL - initial lnL,
 * out[1] = final lnL */
int gbo_optimize_parameter(int opt, int param, int which, double precision, double lowBound, double highBound,
                           double targetScoreDigits, double *out);
/* one pass of Population::BetterFinalOptimization's model part for the
 * parameters in mask (GB_OPT_*), with GARLI's bounds: alpha
 * (population.cpp:2702), pinv (:2727), OptimizeEquilibriumFreqs
 * (tree.cpp:7288), OptimizeRelativeNucRates (tree.cpp:7307), single-class
 * omega (tree.cpp:7186); out[0..4] = improvement per GB_PARAM_* kind */
int gbo_optimize_model(int opt, int mask, double precision, double *out5);
/* Population::BetterFinalOptimization (population.cpp:2566-2790): passes of
 * OptimizeAllBranches + the parameters in mask until GARLI's exit rule;
 * out[0] = final lnL, out[1] = passes, out[2] = model evaluations */
int gbo_final_optimization(int opt, double branchOptPrecision, int mask, int maxPasses, double *out3);
/* depth 0: one model per gbt_score_models call, in GARLI's order; 1: the
 * evaluation points known in advance are scored together; d >= 2: also the
 * higher / lower points of the next d - 1 adaptive widenings of pass 0,
 * speculatively.  Default 4 when patterns x (taxa - 2) <= 2^20, else 1. */
int gbo_set_batching(int opt, int depth);
/* the evaluations of the last OptimizeBoundedParameter call in GARLI's order
 * (SetAndEvaluateParameter values and scores, up to capacity) and the score it
 * started from; returns their number */
int gbo_get_trace(int opt, double *values, double *scores, int capacity, double *initialScore);
/* counters: [0] model evaluations GARLI makes, [1] models scored (speculative
 * ones included), [2] gbt_score_models calls */
int gbo_get_counters(int opt, long long *out3);

#ifdef __cplusplus
}
#endif
#endif /* GARLI_B200_H */
