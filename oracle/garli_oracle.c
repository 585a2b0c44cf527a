/*
 * garli_oracle.c -- CPU restatement of GARLI's FP64 likelihood path.
 *
 * TEST INFRASTRUCTURE ONLY (parity oracle + timed CPU baseline).  The
 * garli_b200 engine never links or calls this file.  See garli_oracle.h for
 * the list of reference functions restated here; each function below cites
 * the GARLI file:line it follows (paths relative to garli/trunk/src).
 *
 * Arithmetic order inside each per-site expression follows the reference
 * source exactly (pairwise sums in the unrolled 4-rate DNA kernels, sequential
 * sums elsewhere), and the parity build uses -ffp-contract=off so that no
 * multiply-add is fused.  OpenMP parallelises the per-pattern loops the way
 * GARLI's --enable-openmp build does (defs.h:30-44).
 */
#include "garli_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXS 64
#define RESCALE_ARRAY_LENGTH 90 /* tree.h:48 */

/* ------------------------------------------------------------------ */
/* rescale constants: tree.cpp:163-172 (FP64 build)                    */
/* ------------------------------------------------------------------ */
static int g_incr[RESCALE_ARRAY_LENGTH];
static double g_thresh[RESCALE_ARRAY_LENGTH];
static double g_mult[RESCALE_ARRAY_LENGTH];
static const double g_reduceRescaleBelow = 1.0e-190;
static const double g_bailOutBelow = 1.0e-250;
static double g_rescaleBelow;
static int g_tables_ready = 0;

static void init_tables(void) {
    if (g_tables_ready) return;
    g_rescaleBelow = exp(-24.0);
    double maxMult = 1.0 / g_bailOutBelow;
    for (int i = 0; i < RESCALE_ARRAY_LENGTH; i++) {
        g_incr[i] = i * 7 - (int)log(g_rescaleBelow);
        g_thresh[i] = exp((double)(-g_incr[i]));
        double m = exp((double)g_incr[i]);
        g_mult[i] = m < maxMult ? m : maxMult;
    }
    g_tables_ready = 1;
}

void or_rescale_tables(int *incr, double *thresh, double *mult) {
    init_tables();
    for (int i = 0; i < RESCALE_ARRAY_LENGTH; i++) {
        if (incr) incr[i] = g_incr[i];
        if (thresh) thresh[i] = g_thresh[i];
        if (mult) mult[i] = g_mult[i];
    }
}

void or_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}
int or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* model                                                               */
/* ------------------------------------------------------------------ */

/* Model::UpdateQMat nucleotide branch, model.cpp:256-293 */
void or_gtr_qmat(const double rel[6], const double pi[4], double *Q, double *blen_mult) {
    double q[4][4];
    memset(q, 0, sizeof(q));
    q[0][1] = rel[0] * pi[1];
    q[0][2] = rel[1] * pi[2];
    q[0][3] = rel[2] * pi[3];
    q[1][2] = rel[3] * pi[2];
    q[1][3] = rel[4] * pi[3];
    q[2][3] = pi[3];
    q[1][0] = rel[0] * pi[0];
    q[2][0] = rel[1] * pi[0];
    q[2][1] = rel[3] * pi[1];
    q[3][0] = rel[2] * pi[0];
    q[3][1] = rel[4] * pi[1];
    q[3][2] = pi[2];
    for (int x = 0; x < 4; x++) {
        double sum = 0.0;
        for (int y = 0; y < 4; y++)
            if (x != y) sum += q[x][y];
        q[x][x] = -sum;
    }
    *blen_mult = (0.5 / ((q[0][1] * pi[0]) + (q[0][2] * pi[0]) + (q[0][3] * pi[0]) + (q[1][2] * pi[1]) +
                         (q[1][3] * pi[1]) + (q[2][3] * pi[2])));
    memcpy(Q, q, sizeof(q));
}

/* Model::UpdateQMatAminoAcid estimated-matrix branch, model.cpp:735-779.
 * exch190 is the upper triangle in row order (from<to). */
void or_aa_qmat(const double *exch190, const double *pi, double *Q, double *blen_mult) {
    const int n = 20;
    for (int f = 0; f < n; f++)
        for (int to = 0; to < n; to++) Q[f * n + to] = pi[to];
    int r = 0;
    for (int f = 0; f < n - 1; f++)
        for (int to = f + 1; to < n; to++) Q[f * n + to] *= exch190[r++];
    r = 0;
    for (int to = 0; to < n - 1; to++)
        for (int f = to + 1; f < n; f++) Q[f * n + to] *= exch190[r++];
    double wsum = 0.0;
    for (int f = 0; f < n; f++) {
        double sum = 0.0;
        for (int to = 0; to < n; to++)
            if (f != to) sum += Q[f * n + to];
        Q[f * n + f] = -sum;
        wsum += sum * pi[f];
    }
    *blen_mult = 1.0 / wsum;
}

/* Standard genetic code, codons in ACGT base-4 order (AAA, AAC, ..., TTT); '*' = stop.
 * Plays the role of GeneticCode::SetStandardCode (sequencedata.h:217). */
static const char *k_std_code = "KNKNTTTTRSRSIIMIQHQHPPPPRRRRLLLLEDEDAAAAGGGGVVVV*Y*YSSSS*CWCLFLF";

/* Model::FillQMatLookup (model.cpp:296-441) + UpdateQMatCodon (model.cpp:442-687)
 * with one omega category: Q_ij = pi_j * r(nucleotide pair) * (omega if
 * nonsynonymous) for codons one nucleotide apart, rel6 in the order
 * AC, AG, AT, CG, CT, GT (qmatLookup bits 8..256, nst = 6). */
int or_codon_qmat6(const double *rel6, double omega, const double *pi61, double *Q, double *blen_mult) {
    int sense[64], ns = 0;
    for (int c = 0; c < 64; c++)
        if (k_std_code[c] != '*') sense[ns++] = c;
    if (ns != 61) return -1;
    const int n = 61;
    static const int pair_index[4][4] = {{-1, 0, 1, 2}, {0, -1, 3, 4}, {1, 3, -1, 5}, {2, 4, 5, -1}};
    for (int a = 0; a < n; a++) {
        for (int b = 0; b < n; b++) {
            int ca = sense[a], cb = sense[b];
            int ndiff = 0, na = 0, nb = 0;
            for (int pos = 0; pos < 3; pos++) {
                int sh = 2 * (2 - pos);
                int x = (ca >> sh) & 3, y = (cb >> sh) & 3;
                if (x != y) { ndiff++; na = x; nb = y; }
            }
            double q = 0.0;
            if (a != b && ndiff == 1) {
                q = pi61[b];
                q *= rel6[pair_index[na][nb]];
                if (k_std_code[ca] != k_std_code[cb]) q *= omega;
            }
            Q[a * n + b] = q;
        }
    }
    double wsum = 0.0;
    for (int x = 0; x < n; x++) {
        double sum = 0.0;
        for (int y = 0; y < n; y++)
            if (x != y) sum += Q[x * n + y];
        Q[x * n + x] = -sum;
        wsum += sum * pi61[x];
    }
    *blen_mult = 1.0 / (wsum * 1.0);
    return 0;
}

/* GY94 (nst = 2): kappa on transitions (qmatLookup bit 2, model.cpp:457-461) */
int or_codon_qmat(double kappa, double omega, const double *pi61, double *Q, double *blen_mult) {
    const double rel6[6] = {1.0, kappa, 1.0, 1.0, kappa, 1.0};
    return or_codon_qmat6(rel6, omega, pi61, Q, blen_mult);
}

/* Eigen system of a reversible rate matrix (the role of CalcEigenStuff ->
 * EigenRealGeneral/InvertMatrix, model.cpp:827-856, linalg.cpp:249/:95).
 * GARLI uses a general real (EISPACK-style) solver; for a reversible Q the
 * symmetric matrix A = D^1/2 Q D^-1/2 (D = diag(pi)) has the same spectrum, so
 * a cyclic Jacobi solve of A gives U = D^-1/2 V and U^-1 = V^T D^1/2.  The
 * product U diag(exp(l t)) U^-1 agrees with the reference's to rounding
 * (checked against linalg.cpp itself by oracle/build_ref.sh + tests). */
int or_eigen(int S, const double *Q, const double *pi, double *eval, double *U, double *Uinv) {
    double *A = (double *)malloc(sizeof(double) * S * S);
    double *V = (double *)malloc(sizeof(double) * S * S);
    double sq[MAXS], isq[MAXS];
    for (int i = 0; i < S; i++) {
        sq[i] = sqrt(pi[i]);
        isq[i] = 1.0 / sq[i];
    }
    for (int i = 0; i < S; i++)
        for (int j = 0; j < S; j++) {
            A[i * S + j] = sq[i] * Q[i * S + j] * isq[j];
            V[i * S + j] = (i == j) ? 1.0 : 0.0;
        }
    /* symmetrise exactly */
    for (int i = 0; i < S; i++)
        for (int j = i + 1; j < S; j++) {
            double m = 0.5 * (A[i * S + j] + A[j * S + i]);
            A[i * S + j] = A[j * S + i] = m;
        }
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < S; i++)
            for (int j = 0; j < S; j++) {
                if (i != j) off += A[i * S + j] * A[i * S + j];
                else diag += A[i * S + i] * A[i * S + i];
            }
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int p = 0; p < S - 1; p++) {
            for (int q = p + 1; q < S; q++) {
                double apq = A[p * S + q];
                if (apq == 0.0) continue;
                double app = A[p * S + p], aqq = A[q * S + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < S; k++) {
                    double akp = A[k * S + p], akq = A[k * S + q];
                    A[k * S + p] = c * akp - s * akq;
                    A[k * S + q] = s * akp + c * akq;
                }
                for (int k = 0; k < S; k++) {
                    double apk = A[p * S + k], aqk = A[q * S + k];
                    A[p * S + k] = c * apk - s * aqk;
                    A[q * S + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < S; k++) {
                    double vkp = V[k * S + p], vkq = V[k * S + q];
                    V[k * S + p] = c * vkp - s * vkq;
                    V[k * S + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    for (int k = 0; k < S; k++) eval[k] = A[k * S + k];
    for (int i = 0; i < S; i++)
        for (int k = 0; k < S; k++) {
            U[i * S + k] = isq[i] * V[i * S + k];
            Uinv[k * S + i] = V[i * S + k] * sq[i];
        }
    free(A);
    free(V);
    return 0;
}

/* ---- discrete gamma (Model::DiscreteGamma, model.cpp:2170-2201) ----
 * GARLI evaluates the chi-square percentage point with AS 91 and the
 * incomplete gamma ratio with AS 32.  The oracle computes the same
 * mathematical quantities to full double precision: log-gamma by the Stirling
 * series with upward recurrence, the regularised lower incomplete gamma by its
 * power series (x < a+1) or Lentz continued fraction, and the gamma quantile by
 * safeguarded Newton iteration on that function. */
static double ln_gamma(double x) {
    double f = 0.0;
    if (x < 7.0) {
        double prod = 1.0;
        while (x < 7.0) { prod *= x; x += 1.0; }
        f = -log(prod);
    }
    double z = 1.0 / (x * x);
    return f + (x - 0.5) * log(x) - x + 0.918938533204672741780329736406 +
           (((-1.0 / 1680.0 * z + 1.0 / 1260.0) * z - 1.0 / 360.0) * z + 1.0 / 12.0) / x;
}

/* regularised lower incomplete gamma P(a, x) */
static double inc_gamma(double x, double a, double lga) {
    if (x <= 0.0) return 0.0;
    double lfac = a * log(x) - x - lga;
    if (x < a + 1.0) {
        double ap = a, sum = 1.0 / a, del = sum;
        for (int n = 0; n < 100000; n++) {
            ap += 1.0;
            del *= x / ap;
            sum += del;
            if (fabs(del) < fabs(sum) * 1e-17) break;
        }
        return sum * exp(lfac);
    } else {
        const double tiny = 1e-300;
        double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
        for (int i = 1; i < 100000; i++) {
            double an = -i * (i - a);
            b += 2.0;
            d = an * d + b;
            if (fabs(d) < tiny) d = tiny;
            c = b + an / c;
            if (fabs(c) < tiny) c = tiny;
            d = 1.0 / d;
            double del = d * c;
            h *= del;
            if (fabs(del - 1.0) < 1e-17) break;
        }
        return 1.0 - exp(lfac) * h;
    }
}

/* quantile of Gamma(shape a, rate 1) at probability p */
static double gamma_quantile(double p, double a) {
    double lga = ln_gamma(a);
    double lo = 0.0, hi = 1.0;
    while (inc_gamma(hi, a, lga) < p) hi *= 2.0;
    double x = 0.5 * (lo + hi);
    for (int it = 0; it < 500; it++) {
        double f = inc_gamma(x, a, lga) - p;
        if (f < 0) lo = x; else hi = x;
        double dens = exp((a - 1.0) * log(x) - x - lga);
        double xn = (dens > 0) ? x - f / dens : 0.5 * (lo + hi);
        if (!(xn > lo && xn < hi)) xn = 0.5 * (lo + hi);
        if (fabs(xn - x) <= 1e-16 * x) { x = xn; break; }
        x = xn;
        if (hi - lo <= 1e-16 * hi) break;
    }
    return x;
}

void or_discrete_gamma(double alpha, int ncat, double *rates) {
    if (ncat <= 1) { rates[0] = 1.0; return; }
    double props[MAXS];
    double factor = alpha / alpha * ncat;
    double lga1 = ln_gamma(alpha + 1.0);
    for (int i = 0; i < ncat - 1; i++)
        props[i] = gamma_quantile((i + 1.0) / ncat, alpha) / alpha; /* POINTGAMMA(p, a, a) */
    for (int i = 0; i < ncat - 1; i++) props[i] = inc_gamma(props[i] * alpha, alpha + 1.0, lga1);
    rates[0] = props[0] * factor;
    rates[ncat - 1] = (1.0 - props[ncat - 2]) * factor;
    for (int i = 1; i < ncat - 1; i++) rates[i] = (props[i] - props[i - 1]) * factor;
}

/* AltCalcPmat (model.cpp:1469-1597) + CalcDerivatives (model.cpp:1271-1358).
 * eval_scaled = eigenvalues already multiplied by blen_multiplier (model.cpp:845). */
void or_pmats(int S, int R, const double *eval_scaled, const double *U, const double *Uinv,
              const double *rateMults, double pinv, int has_pinv, double t, double *P, double *D1,
              double *D2) {
    double ex[MAXS], d1e[MAXS], d2e[MAXS];
    for (int r = 0; r < R; r++) {
        for (int k = 0; k < S; k++) {
            double sev;
            if (!has_pinv) sev = eval_scaled[k] * rateMults[r];
            else sev = eval_scaled[k] * rateMults[r] / (1.0 - pinv);
            ex[k] = exp(sev * t);
            d1e[k] = sev * ex[k];
            d2e[k] = sev * d1e[k];
        }
        for (int i = 0; i < S; i++)
            for (int j = 0; j < S; j++) {
                double sp = 0.0, s1 = 0.0, s2 = 0.0;
                for (int k = 0; k < S; k++) {
                    double x = U[i * S + k] * Uinv[k * S + j];
                    sp += x * ex[k];
                    s1 += x * d1e[k];
                    s2 += x * d2e[k];
                }
                int o = r * S * S + i * S + j;
                if (P) P[o] = (sp > 0.0 ? sp : 0.0);
                if (D1) D1[o] = s1;
                if (D2) D2[o] = s2;
            }
    }
}

/* ------------------------------------------------------------------ */
/* tree engine                                                         */
/* ------------------------------------------------------------------ */

typedef struct {
    double *arr;
    int *mult;
    int rank;
    int dirty;
} OrCla;

struct OrTree {
    int ntax, nnodes, S, R, npat;
    int *left, *right, *next, *anc;
    double *dlen;
    int *counts;
    int lastConst;
    int *constStates;
    /* tips: DNA -> GARLI ambiguity strings (MakeAmbigStrings); NState -> raw states */
    signed char **tipdata;
    int **amap; /* per-site offsets into the DNA ambiguity strings (OPEN_MP ambigMap) */
    /* model */
    double eval[MAXS], *U, *Uinv, pi[MAXS], rateMults[MAXS], rateProbs[MAXS], pinv;
    int has_pinv;
    OrCla *cla; /* 3 per node: [nd*3 + {0 Down,1 UL,2 UR}] */
    int rescaleEvery;
    int threw;
    double lnL;
    double *siteLnL;
    int siteValid;
    long claCount, derivCount;
    double minBrlen, maxBrlen;
    char *optimized;
};

#define DOWN 0
#define UPLEFT 1
#define UPRIGHT 2

static int is_internal(const OrTree *t, int nd) { return nd == 0 || nd > t->ntax; }

/* NucleotideData::MakeAmbigStrings (sequencedata.cpp:278-363) */
static signed char *make_ambig_string(const unsigned char *row, int npat, int *amap) {
    int total = 0;
    for (int j = 0; j < npat; j++) {
        int b = row[j] & 15, ns = 0;
        for (int k = 0; k < 4; k++)
            if (b & (1 << k)) ns++;
        if (ns != 4) total += ns;
        if (ns > 1 || ns == 0 || ns == 4) total++;
    }
    signed char *s = (signed char *)malloc(total > 0 ? total : 1);
    int idx = 0;
    for (int j = 0; j < npat; j++) {
        amap[j] = idx;
        int b = row[j] & 15, ns = 0, code = 0;
        for (int k = 0; k < 4; k++)
            if (b & (1 << k)) { ns++; code = k; }
        if (ns == 1) s[idx++] = (signed char)code;
        else if (ns == 4 || ns == 0) s[idx++] = -4;
        else {
            s[idx++] = (signed char)-ns;
            for (int k = 0; k < 4; k++)
                if (b & (1 << k)) s[idx++] = (signed char)k;
        }
    }
    return s;
}

OrTree *or_tree_new(int ntax, int S, int R, int npat, const int *child3, const double *dlen,
                    const unsigned char *tips, const int *counts, int lastConst,
                    const int *constStates) {
    init_tables();
    OrTree *t = (OrTree *)calloc(1, sizeof(OrTree));
    t->ntax = ntax;
    t->nnodes = 2 * ntax - 2;
    t->S = S;
    t->R = R;
    t->npat = npat;
    int N = t->nnodes;
    t->left = (int *)malloc(sizeof(int) * N);
    t->right = (int *)malloc(sizeof(int) * N);
    t->next = (int *)malloc(sizeof(int) * N);
    t->anc = (int *)malloc(sizeof(int) * N);
    t->dlen = (double *)malloc(sizeof(double) * N);
    t->optimized = (char *)calloc(N, 1);
    for (int i = 0; i < N; i++) {
        t->left[i] = t->right[i] = t->next[i] = t->anc[i] = -1;
        t->dlen[i] = dlen[i];
    }
    for (int i = 0; i < N; i++) {
        int l = child3[i * 3 + 0], m = child3[i * 3 + 1], r = child3[i * 3 + 2];
        if (l < 0) continue;
        t->left[i] = l;
        t->right[i] = r;
        t->anc[l] = i;
        t->anc[r] = i;
        if (m >= 0) {
            t->anc[m] = i;
            t->next[l] = m;
            t->next[m] = r;
        } else {
            t->next[l] = r;
        }
    }
    t->counts = (int *)malloc(sizeof(int) * npat);
    memcpy(t->counts, counts, sizeof(int) * npat);
    t->constStates = (int *)malloc(sizeof(int) * (npat > 0 ? npat : 1));
    for (int i = 0; i < npat; i++) t->constStates[i] = (constStates && i <= lastConst) ? constStates[i] : 0;
    t->lastConst = lastConst;
    t->tipdata = (signed char **)calloc(ntax + 1, sizeof(signed char *));
    t->amap = (int **)calloc(ntax + 1, sizeof(int *));
    for (int tip = 1; tip <= ntax; tip++) {
        const unsigned char *row = tips + (size_t)(tip - 1) * npat;
        t->amap[tip] = (int *)malloc(sizeof(int) * (npat > 0 ? npat : 1));
        if (S == 4) t->tipdata[tip] = make_ambig_string(row, npat, t->amap[tip]);
        else {
            t->tipdata[tip] = (signed char *)malloc(npat);
            for (int j = 0; j < npat; j++) t->tipdata[tip][j] = (signed char)row[j];
        }
    }
    t->U = (double *)calloc(S * S, sizeof(double));
    t->Uinv = (double *)calloc(S * S, sizeof(double));
    t->cla = (OrCla *)calloc(3 * N, sizeof(OrCla));
    for (int i = 0; i < 3 * N; i++) t->cla[i].dirty = 1;
    t->rescaleEvery = 16; /* tree.cpp:163 */
    t->lnL = -1.0;
    t->siteLnL = (double *)malloc(sizeof(double) * (npat > 0 ? npat : 1));
    t->minBrlen = 1e-8; /* defs.h:106 DEF_MIN_BRLEN */
    t->maxBrlen = 100.0; /* defs.h:107 DEF_MAX_BRLEN */
    return t;
}

void or_tree_free(OrTree *t) {
    if (!t) return;
    for (int i = 0; i < 3 * t->nnodes; i++) {
        free(t->cla[i].arr);
        free(t->cla[i].mult);
    }
    free(t->cla);
    for (int tip = 1; tip <= t->ntax; tip++) {
        free(t->tipdata[tip]);
        free(t->amap[tip]);
    }
    free(t->tipdata);
    free(t->amap);
    free(t->left); free(t->right); free(t->next); free(t->anc); free(t->dlen);
    free(t->counts); free(t->constStates); free(t->U); free(t->Uinv); free(t->siteLnL);
    free(t->optimized);
    free(t);
}

void or_tree_set_model(OrTree *t, const double *eval_scaled, const double *U, const double *Uinv,
                       const double *pi, const double *rateMults, const double *rateProbs, double pinv,
                       int has_pinv) {
    int S = t->S;
    memcpy(t->eval, eval_scaled, sizeof(double) * S);
    memcpy(t->U, U, sizeof(double) * S * S);
    memcpy(t->Uinv, Uinv, sizeof(double) * S * S);
    memcpy(t->pi, pi, sizeof(double) * S);
    memcpy(t->rateMults, rateMults, sizeof(double) * t->R);
    memcpy(t->rateProbs, rateProbs, sizeof(double) * t->R);
    t->pinv = pinv;
    t->has_pinv = has_pinv;
    or_tree_dirty_all(t);
}

void or_tree_set_rescale_every(OrTree *t, int every) { t->rescaleEvery = every; }
int or_tree_get_rescale_every(const OrTree *t) { return t->rescaleEvery; }
double or_tree_lnl(const OrTree *t) { return t->lnL; }
long or_tree_cla_count(const OrTree *t) { return t->claCount; }
long or_tree_deriv_count(const OrTree *t) { return t->derivCount; }
double or_tree_get_blen(const OrTree *t, int nd) { return t->dlen[nd]; }

/* Tree::MakeAllNodesDirty */
void or_tree_dirty_all(OrTree *t) {
    for (int i = 0; i < 3 * t->nnodes; i++) t->cla[i].dirty = 1;
    t->lnL = -1.0;
}

static OrCla *cla_of(OrTree *t, int nd, int which) { return &t->cla[nd * 3 + which]; }

static void cla_alloc(OrTree *t, OrCla *c) {
    if (!c->arr) {
        size_t n = (size_t)t->npat * t->R * t->S;
        c->arr = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
        c->mult = (int *)malloc(sizeof(int) * (t->npat > 0 ? t->npat : 1));
    }
}

static void calc_pmat(const OrTree *t, double blen, double *P) {
    or_pmats(t->S, t->R, t->eval, t->U, t->Uinv, t->rateMults, t->pinv, t->has_pinv, blen, P, NULL, NULL);
}

/* ---- DNA CLA kernels ---- */

/* Tree::CalcFullCLAInternalInternal, tree.cpp:7668-7841 */
static void cla_int_int(OrTree *t, OrCla *dest, const OrCla *L, const OrCla *R, const double *Lpr,
                        const double *Rpr) {
    const int nchar = t->npat, nR = t->R;
    if (nR == 4) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nchar; i++) {
            double *d = dest->arr + (size_t)16 * i;
            const double *LCL = L->arr + (size_t)16 * i, *RCL = R->arr + (size_t)16 * i;
            for (int r = 0; r < 4; r++) {
                const double *lp = Lpr + 16 * r, *rp = Rpr + 16 * r;
                const double *lc = LCL + 4 * r, *rc = RCL + 4 * r;
                double L1 = ((lp[0] * lc[0]) + (lp[1] * lc[1])) + ((lp[2] * lc[2]) + (lp[3] * lc[3]));
                double L2 = ((lp[4] * lc[0]) + (lp[5] * lc[1])) + ((lp[6] * lc[2]) + (lp[7] * lc[3]));
                double L3 = ((lp[8] * lc[0]) + (lp[9] * lc[1])) + ((lp[10] * lc[2]) + (lp[11] * lc[3]));
                double L4 = ((lp[12] * lc[0]) + (lp[13] * lc[1])) + ((lp[14] * lc[2]) + (lp[15] * lc[3]));
                double R1 = ((rp[0] * rc[0]) + (rp[1] * rc[1])) + ((rp[2] * rc[2]) + (rp[3] * rc[3]));
                double R2 = ((rp[4] * rc[0]) + (rp[5] * rc[1])) + ((rp[6] * rc[2]) + (rp[7] * rc[3]));
                double R3 = ((rp[8] * rc[0]) + (rp[9] * rc[1])) + ((rp[10] * rc[2]) + (rp[11] * rc[3]));
                double R4 = ((rp[12] * rc[0]) + (rp[13] * rc[1])) + ((rp[14] * rc[2]) + (rp[15] * rc[3]));
                d[4 * r + 0] = L1 * R1;
                d[4 * r + 1] = L2 * R2;
                d[4 * r + 2] = L3 * R3;
                d[4 * r + 3] = L4 * R4;
            }
        }
    } else {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nchar; i++) {
            double *d = dest->arr + (size_t)4 * nR * i;
            const double *LCL = L->arr + (size_t)4 * nR * i, *RCL = R->arr + (size_t)4 * nR * i;
            for (int r = 0; r < nR; r++) {
                const double *lp = Lpr + 16 * r, *rp = Rpr + 16 * r;
                const double *lc = LCL + 4 * r, *rc = RCL + 4 * r;
                double L1 = (lp[0] * lc[0] + lp[1] * lc[1] + lp[2] * lc[2] + lp[3] * lc[3]);
                double L2 = (lp[4] * lc[0] + lp[5] * lc[1] + lp[6] * lc[2] + lp[7] * lc[3]);
                double L3 = (lp[8] * lc[0] + lp[9] * lc[1] + lp[10] * lc[2] + lp[11] * lc[3]);
                double L4 = (lp[12] * lc[0] + lp[13] * lc[1] + lp[14] * lc[2] + lp[15] * lc[3]);
                double R1 = (rp[0] * rc[0] + rp[1] * rc[1] + rp[2] * rc[2] + rp[3] * rc[3]);
                double R2 = (rp[4] * rc[0] + rp[5] * rc[1] + rp[6] * rc[2] + rp[7] * rc[3]);
                double R3 = (rp[8] * rc[0] + rp[9] * rc[1] + rp[10] * rc[2] + rp[11] * rc[3]);
                double R4 = (rp[12] * rc[0] + rp[13] * rc[1] + rp[14] * rc[2] + rp[15] * rc[3]);
                d[4 * r + 0] = L1 * R1;
                d[4 * r + 1] = L2 * R2;
                d[4 * r + 2] = L3 * R3;
                d[4 * r + 3] = L4 * R4;
            }
        }
    }
    for (int i = 0; i < nchar; i++) dest->mult[i] = L->mult[i] + R->mult[i];
    dest->rank = 2 + L->rank + R->rank;
}

/* Tree::CalcFullCLATerminalTerminal, tree.cpp:7912-8080 */
static void cla_tip_tip(OrTree *t, OrCla *dest, const double *Lpr, const double *Rpr,
                        const signed char *Ldata, const signed char *Rdata) {
    const int nchar = t->npat, nR = t->R;
    double *dest_p = dest->arr;
    double tempcla[4 * MAXS];
    for (int i = 0; i < nchar; i++) {
        double *d = dest_p;
        if (*Ldata > -1 && *Rdata > -1) {
            for (int r = 0; r < nR; r++) {
                *(d++) = Lpr[(*Ldata) + 16 * r] * Rpr[(*Rdata) + 16 * r];
                *(d++) = Lpr[(*Ldata + 4) + 16 * r] * Rpr[(*Rdata + 4) + 16 * r];
                *(d++) = Lpr[(*Ldata + 8) + 16 * r] * Rpr[(*Rdata + 8) + 16 * r];
                *(d++) = Lpr[(*Ldata + 12) + 16 * r] * Rpr[(*Rdata + 12) + 16 * r];
            }
            Ldata++;
            Rdata++;
        } else if ((*Ldata == -4 && *Rdata == -4) || (*Ldata == -4 && *Rdata > -1) ||
                   (*Rdata == -4 && *Ldata > -1)) {
            if (*Ldata == -4 && *Rdata == -4) {
                for (int q = 0; q < 4 * nR; q++) *(d++) = 1.0;
            } else if (*Ldata == -4) {
                for (int r = 0; r < nR; r++) {
                    *(d++) = Rpr[(*Rdata) + 16 * r];
                    *(d++) = Rpr[(*Rdata + 4) + 16 * r];
                    *(d++) = Rpr[(*Rdata + 8) + 16 * r];
                    *(d++) = Rpr[(*Rdata + 12) + 16 * r];
                }
            } else {
                for (int r = 0; r < nR; r++) {
                    *(d++) = Lpr[(*Ldata) + 16 * r];
                    *(d++) = Lpr[(*Ldata + 4) + 16 * r];
                    *(d++) = Lpr[(*Ldata + 8) + 16 * r];
                    *(d++) = Lpr[(*Ldata + 12) + 16 * r];
                }
            }
            Ldata++;
            Rdata++;
        } else {
            if (*Ldata > -1) {
                for (int r = 0; r < nR; r++) {
                    d[r * 4] = Lpr[(*Ldata) + 16 * r];
                    d[r * 4 + 1] = Lpr[(*Ldata + 4) + 16 * r];
                    d[r * 4 + 2] = Lpr[(*Ldata + 8) + 16 * r];
                    d[r * 4 + 3] = Lpr[(*Ldata + 12) + 16 * r];
                }
                Ldata++;
            } else if (*Ldata == -4) {
                for (int q = 0; q < 4 * nR; q++) d[q] = 1.0;
                Ldata++;
            } else {
                int ns = -*(Ldata++);
                for (int q = 0; q < 4 * nR; q++) d[q] = 0;
                for (int s = 0; s < ns; s++) {
                    for (int r = 0; r < nR; r++) {
                        d[r * 4] += Lpr[(*Ldata) + 16 * r];
                        d[r * 4 + 1] += Lpr[(*Ldata + 4) + 16 * r];
                        d[r * 4 + 2] += Lpr[(*Ldata + 8) + 16 * r];
                        d[r * 4 + 3] += Lpr[(*Ldata + 12) + 16 * r];
                    }
                    Ldata++;
                }
            }
            if (*Rdata > -1) {
                for (int r = 0; r < nR; r++) {
                    *(d++) *= Rpr[(*Rdata) + 16 * r];
                    *(d++) *= Rpr[(*Rdata + 4) + 16 * r];
                    *(d++) *= Rpr[(*Rdata + 8) + 16 * r];
                    *(d++) *= Rpr[(*Rdata + 12) + 16 * r];
                }
                Rdata++;
            } else if (*Rdata != -4) {
                int ns = -*(Rdata++);
                for (int q = 0; q < 4 * nR; q++) tempcla[q] = 0.0;
                for (int s = 0; s < ns; s++) {
                    for (int r = 0; r < nR; r++) {
                        tempcla[r * 4] += Rpr[(*Rdata) + 16 * r];
                        tempcla[r * 4 + 1] += Rpr[(*Rdata + 4) + 16 * r];
                        tempcla[r * 4 + 2] += Rpr[(*Rdata + 8) + 16 * r];
                        tempcla[r * 4 + 3] += Rpr[(*Rdata + 12) + 16 * r];
                    }
                    Rdata++;
                }
                for (int r = 0; r < nR; r++) {
                    *(d++) *= tempcla[r * 4];
                    *(d++) *= tempcla[r * 4 + 1];
                    *(d++) *= tempcla[r * 4 + 2];
                    *(d++) *= tempcla[r * 4 + 3];
                }
            } else {
                Rdata++;
            }
        }
        dest_p += 4 * nR;
    }
    for (int i = 0; i < nchar; i++) dest->mult[i] = 0;
    dest->rank = 2;
}

/* Tree::CalcFullCLAInternalTerminal, tree.cpp:8291-8535.  pr1 goes with the
 * internal child CL, pr2 with the terminal dat2. */
static void cla_int_tip(OrTree *t, OrCla *dest, const OrCla *LCLA, const double *pr1,
                        const double *pr2, const signed char *dat2, const int *amap) {
    const int nchar = t->npat, nR = t->R;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nchar; i++) {
        const signed char *data2 = dat2 + amap[i];
        double *d = dest->arr + (size_t)4 * nR * i;
        const double *CL1 = LCLA->arr + (size_t)4 * nR * i;
        if (nR == 4) {
            if (*data2 > -1) {
                for (int r = 0; r < 4; r++) {
                    const double *p = pr1 + 16 * r, *c = CL1 + 4 * r;
                    double L1 = ((p[0] * c[0] + p[1] * c[1]) + (p[2] * c[2] + p[3] * c[3]));
                    double L2 = ((p[4] * c[0] + p[5] * c[1]) + (p[6] * c[2] + p[7] * c[3]));
                    double L3 = ((p[8] * c[0] + p[9] * c[1]) + (p[10] * c[2] + p[11] * c[3]));
                    double L4 = ((p[12] * c[0] + p[13] * c[1]) + (p[14] * c[2] + p[15] * c[3]));
                    d[4 * r + 0] = L1 * pr2[*data2 + 16 * r];
                    d[4 * r + 1] = L2 * pr2[*data2 + 4 + 16 * r];
                    d[4 * r + 2] = L3 * pr2[*data2 + 8 + 16 * r];
                    d[4 * r + 3] = L4 * pr2[*data2 + 12 + 16 * r];
                }
                data2++;
            } else if (*data2 == -4) {
                for (int r = 0; r < 4; r++) {
                    const double *p = pr1 + 16 * r, *c = CL1 + 4 * r;
                    d[4 * r + 0] = (p[0] * c[0] + p[1] * c[1] + p[2] * c[2] + p[3] * c[3]);
                    d[4 * r + 1] = (p[4] * c[0] + p[5] * c[1] + p[6] * c[2] + p[7] * c[3]);
                    d[4 * r + 2] = (p[8] * c[0] + p[9] * c[1] + p[10] * c[2] + p[11] * c[3]);
                    d[4 * r + 3] = (p[12] * c[0] + p[13] * c[1] + p[14] * c[2] + p[15] * c[3]);
                }
                data2++;
            } else {
                int ns = -1 * *(data2++);
                for (int j = 0; j < 16; j++) d[j] = 0.0;
                for (int s = 0; s < ns; s++) {
                    for (int r = 0; r < 4; r++) {
                        d[r * 4] += pr2[(*data2) + 16 * r];
                        d[r * 4 + 1] += pr2[(*data2 + 4) + 16 * r];
                        d[r * 4 + 2] += pr2[(*data2 + 8) + 16 * r];
                        d[r * 4 + 3] += pr2[(*data2 + 12) + 16 * r];
                    }
                    data2++;
                }
                for (int r = 0; r < 4; r++) {
                    const double *p = pr1 + 16 * r, *c = CL1 + 4 * r;
                    d[4 * r + 0] *= (p[0] * c[0] + p[1] * c[1] + p[2] * c[2] + p[3] * c[3]);
                    d[4 * r + 1] *= (p[4] * c[0] + p[5] * c[1] + p[6] * c[2] + p[7] * c[3]);
                    d[4 * r + 2] *= (p[8] * c[0] + p[9] * c[1] + p[10] * c[2] + p[11] * c[3]);
                    d[4 * r + 3] *= (p[12] * c[0] + p[13] * c[1] + p[14] * c[2] + p[15] * c[3]);
                }
            }
        } else {
            if (*data2 > -1) {
                for (int r = 0; r < nR; r++) {
                    const double *p = pr1 + 16 * r, *c = CL1 + 4 * r;
                    double L1 = (p[0] * c[0] + p[1] * c[1] + p[2] * c[2] + p[3] * c[3]);
                    double L2 = (p[4] * c[0] + p[5] * c[1] + p[6] * c[2] + p[7] * c[3]);
                    double L3 = (p[8] * c[0] + p[9] * c[1] + p[10] * c[2] + p[11] * c[3]);
                    double L4 = (p[12] * c[0] + p[13] * c[1] + p[14] * c[2] + p[15] * c[3]);
                    d[4 * r + 0] = L1 * pr2[(*data2) + 16 * r];
                    d[4 * r + 1] = L2 * pr2[(*data2 + 4) + 16 * r];
                    d[4 * r + 2] = L3 * pr2[(*data2 + 8) + 16 * r];
                    d[4 * r + 3] = L4 * pr2[(*data2 + 12) + 16 * r];
                }
                data2++;
            } else if (*data2 == -4) {
                for (int r = 0; r < nR; r++) {
                    const double *p = pr1 + 16 * r, *c = CL1 + 4 * r;
                    d[4 * r + 0] = (p[0] * c[0] + p[1] * c[1] + p[2] * c[2] + p[3] * c[3]);
                    d[4 * r + 1] = (p[4] * c[0] + p[5] * c[1] + p[6] * c[2] + p[7] * c[3]);
                    d[4 * r + 2] = (p[8] * c[0] + p[9] * c[1] + p[10] * c[2] + p[11] * c[3]);
                    d[4 * r + 3] = (p[12] * c[0] + p[13] * c[1] + p[14] * c[2] + p[15] * c[3]);
                }
                data2++;
            } else {
                int ns = -1 * *(data2++);
                for (int q = 0; q < 4 * nR; q++) d[q] = 0;
                for (int s = 0; s < ns; s++) {
                    for (int r = 0; r < nR; r++) {
                        d[r * 4] += pr2[(*data2) + 16 * r];
                        d[r * 4 + 1] += pr2[(*data2 + 4) + 16 * r];
                        d[r * 4 + 2] += pr2[(*data2 + 8) + 16 * r];
                        d[r * 4 + 3] += pr2[(*data2 + 12) + 16 * r];
                    }
                    data2++;
                }
                for (int r = 0; r < nR; r++) {
                    const double *p = pr1 + 16 * r, *c = CL1 + 4 * r;
                    d[4 * r + 0] *= (p[0] * c[0] + p[1] * c[1] + p[2] * c[2] + p[3] * c[3]);
                    d[4 * r + 1] *= (p[4] * c[0] + p[5] * c[1] + p[6] * c[2] + p[7] * c[3]);
                    d[4 * r + 2] *= (p[8] * c[0] + p[9] * c[1] + p[10] * c[2] + p[11] * c[3]);
                    d[4 * r + 3] *= (p[12] * c[0] + p[13] * c[1] + p[14] * c[2] + p[15] * c[3]);
                }
            }
        }
    }
    for (int i = 0; i < nchar; i++) dest->mult[i] = LCLA->mult[i];
    dest->rank = LCLA->rank + 2;
}

/* ---- NState CLA kernels ---- */

/* Tree::CalcFullCLAInternalInternalNState, tree.cpp:7843-7910 */
static void cla_int_int_ns(OrTree *t, OrCla *dest, const OrCla *L, const OrCla *R, const double *Lpr,
                           const double *Rpr) {
    const int nchar = t->npat, nR = t->R, ns = t->S;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nchar; i++) {
        double *d = dest->arr + (size_t)ns * nR * i;
        const double *LCL = L->arr + (size_t)ns * nR * i, *RCL = R->arr + (size_t)ns * nR * i;
        for (int rate = 0; rate < nR; rate++) {
            for (int from = 0; from < ns; from++) {
                double L1 = 0.0, R1 = 0.0;
                for (int to = 0; to < ns; to++) {
                    L1 += Lpr[rate * ns * ns + from * ns + to] * LCL[to];
                    R1 += Rpr[rate * ns * ns + from * ns + to] * RCL[to];
                }
                d[from] = L1 * R1;
            }
            LCL += ns;
            RCL += ns;
            d += ns;
        }
    }
    for (int i = 0; i < nchar; i++) dest->mult[i] = L->mult[i] + R->mult[i];
    dest->rank = 2 + L->rank + R->rank;
}

/* Tree::CalcFullCLATerminalTerminalNState, tree.cpp:8082-8160 */
static void cla_tip_tip_ns(OrTree *t, OrCla *dest, const double *Lpr, const double *Rpr,
                           const signed char *Ldata, const signed char *Rdata) {
    const int nchar = t->npat, nR = t->R, ns = t->S;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nchar; i++) {
        double *d = dest->arr + (size_t)ns * nR * i;
        int l = (unsigned char)Ldata[i], r = (unsigned char)Rdata[i];
        if (l < ns && r < ns) {
            for (int rate = 0; rate < nR; rate++)
                for (int from = 0; from < ns; from++)
                    d[rate * ns + from] = Lpr[l + from * ns + rate * ns * ns] * Rpr[r + from * ns + rate * ns * ns];
        } else if (l == ns && r == ns) {
            for (int q = 0; q < nR * ns; q++) d[q] = 1.0;
        } else if (l == ns) {
            for (int rate = 0; rate < nR; rate++)
                for (int from = 0; from < ns; from++) d[rate * ns + from] = Rpr[r + from * ns + rate * ns * ns];
        } else {
            for (int rate = 0; rate < nR; rate++)
                for (int from = 0; from < ns; from++) d[rate * ns + from] = Lpr[l + from * ns + rate * ns * ns];
        }
    }
    for (int i = 0; i < nchar; i++) dest->mult[i] = 0;
    dest->rank = 2;
}

/* Tree::CalcFullCLAInternalTerminalNState, tree.cpp:8537-8600 */
static void cla_int_tip_ns(OrTree *t, OrCla *dest, const OrCla *LCLA, const double *pr1,
                           const double *pr2, const signed char *dat2) {
    const int nchar = t->npat, nR = t->R, ns = t->S;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nchar; i++) {
        double *d = dest->arr + (size_t)ns * nR * i;
        const double *CL1 = LCLA->arr + (size_t)ns * nR * i;
        int s2 = (unsigned char)dat2[i];
        for (int rate = 0; rate < nR; rate++) {
            for (int from = 0; from < ns; from++) {
                double acc = 0.0;
                for (int to = 0; to < ns; to++) acc += pr1[rate * ns * ns + from * ns + to] * CL1[to];
                d[from] = (s2 < ns ? acc * pr2[rate * ns * ns + s2 + from * ns] : acc);
            }
            d += ns;
            CL1 += ns;
        }
    }
    for (int i = 0; i < nchar; i++) dest->mult[i] = LCLA->mult[i];
    dest->rank = LCLA->rank + 2;
}

/* Tree::RescaleRateHet / RescaleRateHetNState, tree.cpp:3370-3598.
 * Returns 1 when GARLI would throw(1) to force a retry with a smaller rescaleEvery. */
static int rescale(OrTree *t, OrCla *c) {
    const int nchar = t->npat, w = t->R * t->S;
    double *dest = c->arr;
    for (int i = 0; i < nchar; i++) {
        double large1;
        if (t->S == 4) {
            large1 = (dest[0] > dest[2] ? dest[0] : dest[2]);
            double large2 = (dest[1] > dest[3] ? dest[1] : dest[3]);
            large1 = (large1 > large2 ? large1 : large2);
            for (int r = 1; r < t->R; r++) {
                large2 = (dest[0 + r * 4] > dest[2 + r * 4] ? dest[0 + r * 4] : dest[2 + r * 4]);
                large1 = (large1 > large2 ? large1 : large2);
                large2 = (dest[1 + r * 4] > dest[3 + r * 4] ? dest[1 + r * 4] : dest[3 + r * 4]);
                large1 = (large1 > large2 ? large1 : large2);
            }
        } else {
            large1 = (dest[0] > dest[1]) ? dest[0] : dest[1];
            for (int s = 2; s < w; s++) large1 = (dest[s] > large1) ? dest[s] : large1;
        }
        if (large1 < g_rescaleBelow) {
            if (large1 < g_reduceRescaleBelow) {
                if (t->rescaleEvery > 2) return 1;
                else if (large1 < g_bailOutBelow) return 1;
            }
            int index = 0;
            while (((index + 1) < RESCALE_ARRAY_LENGTH) && (g_thresh[index + 1] > large1)) index++;
            c->mult[i] += g_incr[index];
            double mult = g_mult[index];
            for (int q = 0; q < w; q++) dest[q] *= mult;
        }
        dest += w;
    }
    c->rank = 0;
    return 0;
}

/* ---- recursion: ConditionalLikelihoodRateHet (tree.cpp:3600-3811) ---- */

static OrCla *get_cla(OrTree *t, int nd, int which, int calc);

/* Tree::UpdateCLAs, tree.cpp:3905-4001 */
static void update_clas(OrTree *t, OrCla *dest, OrCla *first, OrCla *sec, int firstChild, int secChild,
                        double blen1, double blen2) {
    size_t pm = (size_t)t->R * t->S * t->S;
    double *Lpr = (double *)malloc(sizeof(double) * pm);
    double *Rpr = (double *)malloc(sizeof(double) * pm);
    calc_pmat(t, blen1, Lpr);
    calc_pmat(t, blen2, Rpr);
    cla_alloc(t, dest);
    int dna = (t->S == 4);
    if (first && sec) {
        if (dna) cla_int_int(t, dest, first, sec, Lpr, Rpr);
        else cla_int_int_ns(t, dest, first, sec, Lpr, Rpr);
    } else if (!first && !sec) {
        if (dna) cla_tip_tip(t, dest, Lpr, Rpr, t->tipdata[firstChild], t->tipdata[secChild]);
        else cla_tip_tip_ns(t, dest, Lpr, Rpr, t->tipdata[firstChild], t->tipdata[secChild]);
    } else {
        if (!first) {
            if (dna) cla_int_tip(t, dest, sec, Rpr, Lpr, t->tipdata[firstChild], t->amap[firstChild]);
            else cla_int_tip_ns(t, dest, sec, Rpr, Lpr, t->tipdata[firstChild]);
        } else {
            if (dna) cla_int_tip(t, dest, first, Lpr, Rpr, t->tipdata[secChild], t->amap[secChild]);
            else cla_int_tip_ns(t, dest, first, Lpr, Rpr, t->tipdata[secChild]);
        }
    }
    free(Lpr);
    free(Rpr);
    t->claCount++;
    if (dest->rank >= t->rescaleEvery) {
        if (rescale(t, dest)) t->threw = 1;
    }
}

static void compute_cla(OrTree *t, int dir, int nd) {
    int Lchild, Rchild;
    OrCla *LCLA = NULL, *RCLA = NULL;
    double blen1, blen2;
    if (dir == DOWN) {
        Lchild = t->left[nd];
        Rchild = t->right[nd];
        if (is_internal(t, Lchild)) LCLA = get_cla(t, Lchild, DOWN, 1);
        if (t->threw) return;
        if (is_internal(t, Rchild)) RCLA = get_cla(t, Rchild, DOWN, 1);
        if (t->threw) return;
        blen1 = t->dlen[Lchild];
        blen2 = t->dlen[Rchild];
    } else {
        int a = t->anc[nd];
        if (a >= 0) {
            Lchild = a;
            if (t->left[a] == nd) LCLA = get_cla(t, a, UPLEFT, 1);
            else if (t->right[a] == nd) LCLA = get_cla(t, a, UPRIGHT, 1);
            else LCLA = get_cla(t, a, DOWN, 1);
            if (t->threw) return;
            blen1 = t->dlen[nd];
            Rchild = (dir == UPRIGHT) ? t->left[nd] : t->right[nd];
        } else {
            if (dir == UPRIGHT) {
                Lchild = t->left[nd];
                Rchild = t->next[t->left[nd]];
            } else {
                Lchild = t->next[t->left[nd]];
                Rchild = t->right[nd];
            }
            if (is_internal(t, Lchild)) LCLA = get_cla(t, Lchild, DOWN, 1);
            if (t->threw) return;
            blen1 = t->dlen[Lchild];
        }
        if (is_internal(t, Rchild)) RCLA = get_cla(t, Rchild, DOWN, 1);
        if (t->threw) return;
        blen2 = t->dlen[Rchild];
    }
    OrCla *dest = cla_of(t, nd, dir);
    update_clas(t, dest, LCLA, RCLA, Lchild, Rchild, blen1, blen2);
    if (!t->threw) dest->dirty = 0;
}

/* Tree::GetClaSetDown / UpLeft / UpRight, tree.cpp:9378-9410 */
static OrCla *get_cla(OrTree *t, int nd, int which, int calc) {
    OrCla *c = cla_of(t, nd, which);
    if (c->dirty && calc) compute_cla(t, which, nd);
    return c;
}

/* ---- root scoring: GetScorePartial* ---- */

/* Tree::GetScorePartialTerminalRateHet, tree.cpp:6040-6170 */
static double score_tip_dna(OrTree *t, const OrCla *pc, const double *prmat, const signed char *Ldata) {
    const double *partial = pc->arr;
    const int *um = pc->mult;
    const int nR = t->R;
    const double *rp = t->rateProbs, *f = t->pi;
    double tot = 0.0;
    for (int i = 0; i < t->npat; i++) {
        double La = 0.0, Lc = 0.0, Lg = 0.0, Lt = 0.0;
        if (*Ldata > -1) {
            for (int r = 0; r < nR; r++) {
                La += prmat[(*Ldata) + 16 * r] * partial[0] * rp[r];
                Lc += prmat[(*Ldata + 4) + 16 * r] * partial[1] * rp[r];
                Lg += prmat[(*Ldata + 8) + 16 * r] * partial[2] * rp[r];
                Lt += prmat[(*Ldata + 12) + 16 * r] * partial[3] * rp[r];
                partial += 4;
            }
            Ldata++;
        } else if (*Ldata == -4) {
            for (int r = 0; r < nR; r++) {
                La += partial[0] * rp[r];
                Lc += partial[1] * rp[r];
                Lg += partial[2] * rp[r];
                Lt += partial[3] * rp[r];
                partial += 4;
            }
            Ldata++;
        } else {
            int ns = -1 * *(Ldata++);
            for (int s = 0; s < ns; s++) {
                for (int r = 0; r < nR; r++) {
                    La += prmat[(*Ldata) + 16 * r] * partial[4 * r] * rp[r];
                    Lc += prmat[(*Ldata + 4) + 16 * r] * partial[1 + 4 * r] * rp[r];
                    Lg += prmat[(*Ldata + 8) + 16 * r] * partial[2 + 4 * r] * rp[r];
                    Lt += prmat[(*Ldata + 12) + 16 * r] * partial[3 + 4 * r] * rp[r];
                }
                Ldata++;
            }
            partial += 4 * nR;
        }
        double siteL;
        if (t->has_pinv && i <= t->lastConst) {
            double btot = 0.0;
            int cb = t->constStates[i];
            if (cb & 1) btot += f[0];
            if (cb & 2) btot += f[1];
            if (cb & 4) btot += f[2];
            if (cb & 8) btot += f[3];
            if (um[i] == 0) siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]) + t->pinv * btot);
            else siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]) + (t->pinv * btot * exp((double)um[i])));
        } else
            siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]));
        double u = (log(siteL) - um[i]);
        t->siteLnL[i] = u;
        tot += (t->counts[i] * u);
    }
    return tot;
}

/* Tree::GetScorePartialInternalRateHet, tree.cpp:6172-6271 */
static double score_int_dna(OrTree *t, const OrCla *pc, const OrCla *cc, const double *prmat) {
    const int nR = t->R;
    const double *rp = t->rateProbs, *f = t->pi;
    double tot = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : tot)
    for (int i = 0; i < t->npat; i++) {
        const double *partial = pc->arr + (size_t)4 * nR * i;
        const double *CL1 = cc->arr + (size_t)4 * nR * i;
        double La = 0.0, Lc = 0.0, Lg = 0.0, Lt = 0.0;
        for (int r = 0; r < nR; r++) {
            int o = r * 16;
            La += (prmat[o] * CL1[0] + prmat[o + 1] * CL1[1] + prmat[o + 2] * CL1[2] + prmat[o + 3] * CL1[3]) * partial[0] * rp[r];
            Lc += (prmat[o + 4] * CL1[0] + prmat[o + 5] * CL1[1] + prmat[o + 6] * CL1[2] + prmat[o + 7] * CL1[3]) * partial[1] * rp[r];
            Lg += (prmat[o + 8] * CL1[0] + prmat[o + 9] * CL1[1] + prmat[o + 10] * CL1[2] + prmat[o + 11] * CL1[3]) * partial[2] * rp[r];
            Lt += (prmat[o + 12] * CL1[0] + prmat[o + 13] * CL1[1] + prmat[o + 14] * CL1[2] + prmat[o + 15] * CL1[3]) * partial[3] * rp[r];
            partial += 4;
            CL1 += 4;
        }
        double siteL;
        int m1 = pc->mult[i], m2 = cc->mult[i];
        if (t->has_pinv && i <= t->lastConst) {
            double btot = 0.0;
            int cb = t->constStates[i];
            if (cb & 1) btot += f[0];
            if (cb & 2) btot += f[1];
            if (cb & 4) btot += f[2];
            if (cb & 8) btot += f[3];
            if (m1 + m2 == 0) siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]) + t->pinv * btot);
            else siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]) + (t->pinv * btot * exp((double)m1 + m2)));
        } else
            siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]));
        double u = (log(siteL) - m1 - m2);
        t->siteLnL[i] = u;
        tot += (t->counts[i] * u);
    }
    return tot;
}

/* Tree::GetScorePartialInternalNState, tree.cpp:6273-6460 */
static double score_int_ns(OrTree *t, const OrCla *pc, const OrCla *cc, const double *prmat) {
    const int nR = t->R, ns = t->S;
    const double *rp = t->rateProbs, *f = t->pi;
    double tot = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : tot)
    for (int i = 0; i < t->npat; i++) {
        const double *partial = pc->arr + (size_t)ns * nR * i;
        const double *CL1 = cc->arr + (size_t)ns * nR * i;
        double siteL = 0.0;
        if (nR == 1) {
            for (int from = 0; from < ns; from++) {
                double temp = 0.0;
                for (int to = 0; to < ns; to++) temp += prmat[from * ns + to] * CL1[to];
                siteL += temp * partial[from] * f[from];
            }
            siteL *= rp[0];
        } else {
            for (int rate = 0; rate < nR; rate++) {
                double rateL = 0.0;
                int ro = rate * ns * ns;
                for (int from = 0; from < ns; from++) {
                    double tempL = 0.0;
                    int off = from * ns;
                    for (int to = 0; to < ns; to++) tempL += prmat[ro + off + to] * CL1[to];
                    rateL += tempL * partial[from] * f[from];
                }
                siteL += rateL * rp[rate];
                partial += ns;
                CL1 += ns;
            }
        }
        int m1 = pc->mult[i], m2 = cc->mult[i];
        if (t->has_pinv && i <= t->lastConst) {
            if (m1 + m2 == 0) siteL += t->pinv * f[t->constStates[i]];
            else siteL += t->pinv * f[t->constStates[i]] * exp((double)m1 + (double)m2);
        }
        double u = (log(siteL) - m1 - m2);
        t->siteLnL[i] = u;
        if (u < 0.0) tot += (t->counts[i] * u);
    }
    return tot;
}

/* Tree::GetScorePartialTerminalNState, tree.cpp:5597-5800 */
static double score_tip_ns(OrTree *t, const OrCla *pc, const double *prmat, const signed char *Ldat) {
    const int nR = t->R, ns = t->S;
    const double *rp = t->rateProbs, *f = t->pi;
    double tot = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : tot)
    for (int i = 0; i < t->npat; i++) {
        const double *partial = pc->arr + (size_t)ns * nR * i;
        int s = (unsigned char)Ldat[i];
        double siteL = 0.0;
        if (nR == 1) {
            if (s < ns) {
                for (int from = 0; from < ns; from++) siteL += prmat[s + ns * from] * partial[from] * f[from];
            } else {
                for (int from = 0; from < ns; from++) siteL += partial[from] * f[from];
            }
            siteL *= rp[0];
        } else {
            for (int rate = 0; rate < nR; rate++) {
                double rateL = 0.0;
                if (s < ns) {
                    int ro = rate * ns * ns;
                    for (int from = 0; from < ns; from++) rateL += prmat[ro + from * ns + s] * partial[from] * f[from];
                } else {
                    for (int from = 0; from < ns; from++) rateL += partial[from] * f[from];
                }
                siteL += rateL * rp[rate];
                partial += ns;
            }
        }
        int m = pc->mult[i];
        if (t->has_pinv && i <= t->lastConst) {
            if (m == 0) siteL += t->pinv * f[t->constStates[i]];
            else siteL += t->pinv * f[t->constStates[i]] * exp((double)m);
        }
        double u = (log(siteL) - m);
        t->siteLnL[i] = u;
        if (u < 0.0) tot += (t->counts[i] * u);
    }
    return tot;
}

/* Tree::GetTotalScore, tree.cpp:3815-3870 (single model/data subset) */
static void get_total_score(OrTree *t, OrCla *partial, OrCla *child, int childNode, double blen1) {
    double *P = (double *)malloc(sizeof(double) * t->R * t->S * t->S);
    calc_pmat(t, blen1, P);
    if (t->S == 4) {
        if (child) t->lnL = score_int_dna(t, partial, child, P);
        else t->lnL = score_tip_dna(t, partial, P, t->tipdata[childNode]);
    } else {
        if (child) t->lnL = score_int_ns(t, partial, child, P);
        else t->lnL = score_tip_ns(t, partial, P, t->tipdata[childNode]);
    }
    t->siteValid = 1;
    free(P);
}

/* ConditionalLikelihoodRateHet(ROOT, nd), tree.cpp:3686-3811 (no dummy root) */
static void root_score(OrTree *t, int nd) {
    OrCla *partial = NULL, *childCLA = NULL;
    int child;
    double blen1;
    if (!cla_of(t, nd, UPLEFT)->dirty) {
        partial = cla_of(t, nd, UPLEFT);
        child = t->left[nd];
        if (is_internal(t, child)) childCLA = get_cla(t, child, DOWN, 1);
        blen1 = t->dlen[child];
    } else if (!cla_of(t, nd, UPRIGHT)->dirty) {
        partial = cla_of(t, nd, UPRIGHT);
        child = t->right[nd];
        if (is_internal(t, child)) childCLA = get_cla(t, child, DOWN, 1);
        blen1 = t->dlen[child];
    } else {
        partial = get_cla(t, nd, DOWN, 1);
        if (t->threw) return;
        int a = t->anc[nd];
        if (a >= 0) {
            child = a;
            if (t->left[a] == nd) childCLA = get_cla(t, a, UPLEFT, 1);
            else if (t->right[a] == nd) childCLA = get_cla(t, a, UPRIGHT, 1);
            else childCLA = get_cla(t, a, DOWN, 1);
            blen1 = t->dlen[nd];
        } else {
            child = t->next[t->left[nd]];
            if (is_internal(t, child)) childCLA = get_cla(t, child, DOWN, 1);
            blen1 = t->dlen[child];
        }
    }
    if (t->threw) return;
    get_total_score(t, partial, childCLA, child, blen1);
}

/* Tree::Score, tree.cpp:4003-4100: retry with rescaleEvery -= 2 on throw(1) */
double or_tree_score(OrTree *t, int rootNode) {
    for (;;) {
        t->threw = 0;
        root_score(t, rootNode);
        if (!t->threw) break;
        or_tree_dirty_all(t);
        t->rescaleEvery -= 2;
        if (t->rescaleEvery < 2) return NAN;
    }
    return t->lnL;
}

/* ---- branch derivatives ---- */

/* Tree::GetDerivsPartialTerminal, optimization.cpp:2412-2590 */
static void derivs_tip_dna(OrTree *t, const OrCla *pc, const double *prmat, const double *d1mat,
                           const double *d2mat, const signed char *Ldat, const int *amap, double *out) {
    const int nR = t->R;
    const double *rp = t->rateProbs, *f = t->pi;
    double tot1 = 0.0, tot2 = 0.0, totL = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : tot1, tot2, totL)
    for (int i = 0; i < t->npat; i++) {
        const signed char *Ldata = Ldat + amap[i];
        const double *partial = pc->arr + (size_t)4 * nR * i;
        double La = 0, Lc = 0, Lg = 0, Lt = 0, D1a = 0, D1c = 0, D1g = 0, D1t = 0, D2a = 0, D2c = 0, D2g = 0, D2t = 0;
        if (*Ldata > -1) {
            for (int r = 0; r < nR; r++) {
                La += prmat[(*Ldata) + 16 * r] * partial[0] * rp[r];
                D1a += d1mat[(*Ldata) + 16 * r] * partial[0] * rp[r];
                D2a += d2mat[(*Ldata) + 16 * r] * partial[0] * rp[r];
                Lc += prmat[(*Ldata + 4) + 16 * r] * partial[1] * rp[r];
                D1c += d1mat[(*Ldata + 4) + 16 * r] * partial[1] * rp[r];
                D2c += d2mat[(*Ldata + 4) + 16 * r] * partial[1] * rp[r];
                Lg += prmat[(*Ldata + 8) + 16 * r] * partial[2] * rp[r];
                D1g += d1mat[(*Ldata + 8) + 16 * r] * partial[2] * rp[r];
                D2g += d2mat[(*Ldata + 8) + 16 * r] * partial[2] * rp[r];
                Lt += prmat[(*Ldata + 12) + 16 * r] * partial[3] * rp[r];
                D1t += d1mat[(*Ldata + 12) + 16 * r] * partial[3] * rp[r];
                D2t += d2mat[(*Ldata + 12) + 16 * r] * partial[3] * rp[r];
                partial += 4;
            }
            Ldata++;
        } else if (*Ldata == -4) {
            for (int r = 0; r < nR; r++) {
                La += partial[0] * rp[r];
                Lc += partial[1] * rp[r];
                Lg += partial[2] * rp[r];
                Lt += partial[3] * rp[r];
                partial += 4;
            }
            Ldata++;
        } else {
            int ns = -1 * *(Ldata++);
            for (int s = 0; s < ns; s++) {
                for (int r = 0; r < nR; r++) {
                    La += prmat[(*Ldata) + 16 * r] * partial[4 * r] * rp[r];
                    D1a += d1mat[(*Ldata) + 16 * r] * partial[4 * r] * rp[r];
                    D2a += d2mat[(*Ldata) + 16 * r] * partial[4 * r] * rp[r];
                    Lc += prmat[(*Ldata + 4) + 16 * r] * partial[1 + 4 * r] * rp[r];
                    D1c += d1mat[(*Ldata + 4) + 16 * r] * partial[1 + 4 * r] * rp[r];
                    D2c += d2mat[(*Ldata + 4) + 16 * r] * partial[1 + 4 * r] * rp[r];
                    Lg += prmat[(*Ldata + 8) + 16 * r] * partial[2 + 4 * r] * rp[r];
                    D1g += d1mat[(*Ldata + 8) + 16 * r] * partial[2 + 4 * r] * rp[r];
                    D2g += d2mat[(*Ldata + 8) + 16 * r] * partial[2 + 4 * r] * rp[r];
                    Lt += prmat[(*Ldata + 12) + 16 * r] * partial[3 + 4 * r] * rp[r];
                    D1t += d1mat[(*Ldata + 12) + 16 * r] * partial[3 + 4 * r] * rp[r];
                    D2t += d2mat[(*Ldata + 12) + 16 * r] * partial[3 + 4 * r] * rp[r];
                }
                Ldata++;
            }
            partial += 4 * nR;
        }
        double siteL;
        if (t->has_pinv && i <= t->lastConst) {
            double btot = 0.0;
            int cb = t->constStates[i];
            if (cb & 1) btot += f[0];
            if (cb & 2) btot += f[1];
            if (cb & 4) btot += f[2];
            if (cb & 8) btot += f[3];
            siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]) + (t->pinv * btot) * exp((double)pc->mult[i]));
        } else
            siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]));
        double u = log(siteL) - pc->mult[i];
        t->siteLnL[i] = u;
        totL += u * t->counts[i];
        double sd1 = (((D1a * f[0] + D1c * f[1] + D1g * f[2] + D1t * f[3])) / siteL);
        tot1 += sd1 * t->counts[i];
        double sd2 = ((D2a * f[0] + D2c * f[1] + D2g * f[2] + D2t * f[3]) / siteL) - (sd1 * sd1);
        tot2 += sd2 * t->counts[i];
    }
    out[0] = totL;
    out[1] = tot1;
    out[2] = tot2;
}

/* Tree::GetDerivsPartialInternal, optimization.cpp:3063-3228 */
static void derivs_int_dna(OrTree *t, const OrCla *pc, const OrCla *cc, const double *prmat,
                           const double *d1mat, const double *d2mat, double *out) {
    const int nR = t->R;
    const double *rp = t->rateProbs, *f = t->pi;
    double tot1 = 0.0, tot2 = 0.0, totL = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : tot1, tot2, totL)
    for (int i = 0; i < t->npat; i++) {
        const double *partial = pc->arr + (size_t)4 * nR * i;
        const double *CL1 = cc->arr + (size_t)4 * nR * i;
        double La = 0, Lc = 0, Lg = 0, Lt = 0, D1a = 0, D1c = 0, D1g = 0, D1t = 0, D2a = 0, D2c = 0, D2g = 0, D2t = 0;
        for (int r = 0; r < nR; r++) {
            int o = r * 16;
            const double *p = prmat + o, *a = d1mat + o, *b = d2mat + o;
            La += (p[0] * CL1[0] + p[1] * CL1[1] + p[2] * CL1[2] + p[3] * CL1[3]) * partial[0] * rp[r];
            Lc += (p[4] * CL1[0] + p[5] * CL1[1] + p[6] * CL1[2] + p[7] * CL1[3]) * partial[1] * rp[r];
            Lg += (p[8] * CL1[0] + p[9] * CL1[1] + p[10] * CL1[2] + p[11] * CL1[3]) * partial[2] * rp[r];
            Lt += (p[12] * CL1[0] + p[13] * CL1[1] + p[14] * CL1[2] + p[15] * CL1[3]) * partial[3] * rp[r];
            D1a += (a[0] * CL1[0] + a[1] * CL1[1] + a[2] * CL1[2] + a[3] * CL1[3]) * partial[0] * rp[r];
            D1c += (a[4] * CL1[0] + a[5] * CL1[1] + a[6] * CL1[2] + a[7] * CL1[3]) * partial[1] * rp[r];
            D1g += (a[8] * CL1[0] + a[9] * CL1[1] + a[10] * CL1[2] + a[11] * CL1[3]) * partial[2] * rp[r];
            D1t += (a[12] * CL1[0] + a[13] * CL1[1] + a[14] * CL1[2] + a[15] * CL1[3]) * partial[3] * rp[r];
            D2a += (b[0] * CL1[0] + b[1] * CL1[1] + b[2] * CL1[2] + b[3] * CL1[3]) * partial[0] * rp[r];
            D2c += (b[4] * CL1[0] + b[5] * CL1[1] + b[6] * CL1[2] + b[7] * CL1[3]) * partial[1] * rp[r];
            D2g += (b[8] * CL1[0] + b[9] * CL1[1] + b[10] * CL1[2] + b[11] * CL1[3]) * partial[2] * rp[r];
            D2t += (b[12] * CL1[0] + b[13] * CL1[1] + b[14] * CL1[2] + b[15] * CL1[3]) * partial[3] * rp[r];
            partial += 4;
            CL1 += 4;
        }
        double siteL;
        if (t->has_pinv && i <= t->lastConst) {
            double btot = 0.0;
            int cb = t->constStates[i];
            if (cb & 1) btot += f[0];
            if (cb & 2) btot += f[1];
            if (cb & 4) btot += f[2];
            if (cb & 8) btot += f[3];
            siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]) +
                     (t->pinv * btot) * exp((double)cc->mult[i] + pc->mult[i]));
        } else
            siteL = ((La * f[0] + Lc * f[1] + Lg * f[2] + Lt * f[3]));
        double sd1 = (((D1a * f[0] + D1c * f[1] + D1g * f[2] + D1t * f[3])) / siteL);
        double u = log(siteL) - cc->mult[i] - pc->mult[i];
        t->siteLnL[i] = u;
        totL += u * t->counts[i];
        tot1 += t->counts[i] * sd1;
        double sd2 = ((D2a * f[0] + D2c * f[1] + D2g * f[2] + D2t * f[3]) / siteL) - (sd1 * sd1);
        tot2 += t->counts[i] * sd2;
    }
    out[0] = totL;
    out[1] = tot1;
    out[2] = tot2;
}

/* Tree::GetDerivsPartialInternalNState (optimization.cpp:3425, R = 1),
 * GetDerivsPartialInternalNStateRateHet (:3230, R > 1),
 * GetDerivsPartialTerminalNState (:2592, R = 1) and
 * GetDerivsPartialTerminalNStateRateHet (:2860, R > 1). */
static void derivs_ns(OrTree *t, const OrCla *pc, const OrCla *cc, const signed char *tip,
                      const double *prmat, const double *d1mat, const double *d2mat, double *out) {
    const int nR = t->R, ns = t->S;
    const double *rp = t->rateProbs, *f = t->pi;
    double tot1 = 0.0, tot2 = 0.0, totL = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : tot1, tot2, totL)
    for (int i = 0; i < t->npat; i++) {
        const double *partial = pc->arr + (size_t)ns * nR * i;
        const double *CL1 = cc ? cc->arr + (size_t)ns * nR * i : NULL;
        int s = tip ? (unsigned char)tip[i] : 0;
        double siteL = 0.0, siteD1 = 0.0, siteD2 = 0.0;
        if (nR == 1) {
            if (CL1) {
                for (int from = 0; from < ns; from++) {
                    double tL = 0.0, t1 = 0.0, t2 = 0.0;
                    for (int to = 0; to < ns; to++) {
                        tL += prmat[from * ns + to] * CL1[to];
                        t1 += d1mat[from * ns + to] * CL1[to];
                        t2 += d2mat[from * ns + to] * CL1[to];
                    }
                    siteL += tL * partial[from] * f[from];
                    siteD1 += t1 * partial[from] * f[from];
                    siteD2 += t2 * partial[from] * f[from];
                }
            } else if (s != ns) {
                for (int from = 0; from < ns; from++) {
                    siteL += prmat[s + ns * from] * partial[from] * f[from];
                    siteD1 += d1mat[s + ns * from] * partial[from] * f[from];
                    siteD2 += d2mat[s + ns * from] * partial[from] * f[from];
                }
            } else {
                for (int from = 0; from < ns; from++) siteL += partial[from] * f[from];
            }
            siteL *= rp[0];
            siteD1 *= rp[0];
            siteD2 *= rp[0];
        } else {
            for (int rate = 0; rate < nR; rate++) {
                double rL = 0.0, r1 = 0.0, r2 = 0.0;
                int ro = rate * ns * ns;
                if (CL1) {
                    for (int from = 0; from < ns; from++) {
                        double tL = 0.0, t1 = 0.0, t2 = 0.0;
                        int off = from * ns;
                        for (int to = 0; to < ns; to++) {
                            tL += prmat[ro + off + to] * CL1[to];
                            t1 += d1mat[ro + off + to] * CL1[to];
                            t2 += d2mat[ro + off + to] * CL1[to];
                        }
                        rL += tL * partial[from] * f[from];
                        r1 += t1 * partial[from] * f[from];
                        r2 += t2 * partial[from] * f[from];
                    }
                    CL1 += ns;
                } else if (s < ns) {
                    for (int from = 0; from < ns; from++) {
                        int off = from * ns;
                        rL += prmat[ro + off + s] * partial[from] * f[from];
                        r1 += d1mat[ro + off + s] * partial[from] * f[from];
                        r2 += d2mat[ro + off + s] * partial[from] * f[from];
                    }
                } else {
                    for (int from = 0; from < ns; from++) rL += partial[from] * f[from];
                }
                siteL += rL * rp[rate];
                siteD1 += r1 * rp[rate];
                siteD2 += r2 * rp[rate];
                partial += ns;
            }
        }
        int m1 = pc->mult[i], m2 = cc ? cc->mult[i] : 0;
        if (t->has_pinv && i <= t->lastConst) {
            if (cc) siteL += (t->pinv * f[t->constStates[i]] * exp((double)m1) * exp((double)m2));
            else siteL += (t->pinv * f[t->constStates[i]] * exp((double)m1));
        }
        double u = log(siteL) - m1 - m2;
        t->siteLnL[i] = u;
        if (u < 0.0) {
            totL += u * t->counts[i];
            siteD1 /= siteL;
            tot1 += t->counts[i] * siteD1;
            siteD2 = ((siteD2 / siteL) - siteD1 * siteD1);
            tot2 += t->counts[i] * siteD2;
        }
    }
    out[0] = totL;
    out[1] = tot1;
    out[2] = tot2;
}

/* Tree::CalcDerivativesRateHet, optimization.cpp:1099-1194 (single subset) */
static void calc_derivs(OrTree *t, int nd1, int nd2, double *out) {
    OrCla *one, *two = NULL;
    if (t->left[nd1] == nd2) one = get_cla(t, nd1, UPLEFT, 1);
    else if (t->right[nd1] == nd2) one = get_cla(t, nd1, UPRIGHT, 1);
    else one = get_cla(t, nd1, DOWN, 1);
    if (t->threw) return;
    if (is_internal(t, nd2)) two = get_cla(t, nd2, DOWN, 1);
    if (t->threw) return;
    size_t pm = (size_t)t->R * t->S * t->S;
    double *P = (double *)malloc(sizeof(double) * pm * 3);
    or_pmats(t->S, t->R, t->eval, t->U, t->Uinv, t->rateMults, t->pinv, t->has_pinv, t->dlen[nd2], P, P + pm,
             P + 2 * pm);
    if (t->S == 4) {
        if (!two) derivs_tip_dna(t, one, P, P + pm, P + 2 * pm, t->tipdata[nd2], t->amap[nd2], out);
        else derivs_int_dna(t, one, two, P, P + pm, P + 2 * pm, out);
    } else {
        derivs_ns(t, one, two, two ? NULL : t->tipdata[nd2], P, P + pm, P + 2 * pm, out);
    }
    free(P);
    t->lnL = out[0];
    t->siteValid = 1;
    t->derivCount++;
}

int or_tree_derivs(OrTree *t, int nd, double *out) {
    for (;;) {
        t->threw = 0;
        calc_derivs(t, t->anc[nd], nd, out);
        if (!t->threw) return 0;
        or_tree_dirty_all(t);
        t->rescaleEvery -= 2;
        if (t->rescaleEvery < 2) return -1;
    }
}

/* ---- SweepDirtynessOverTree (tree.cpp:4247-4295) and SetBranchLength ---- */
static void sweep(OrTree *t, int nd, int from) {
    t->lnL = -1;
    if (from < 0) {
        if (is_internal(t, nd)) {
            cla_of(t, nd, UPLEFT)->dirty = 1;
            cla_of(t, nd, UPRIGHT)->dirty = 1;
            if (is_internal(t, t->left[nd])) sweep(t, t->left[nd], nd);
            if (is_internal(t, t->right[nd])) sweep(t, t->right[nd], nd);
        }
        if (t->anc[nd] >= 0) sweep(t, t->anc[nd], nd);
    } else {
        if (from == t->anc[nd] || (nd == 0 && from == t->next[t->left[nd]])) {
            cla_of(t, nd, UPLEFT)->dirty = 1;
            cla_of(t, nd, UPRIGHT)->dirty = 1;
            if (is_internal(t, t->left[nd])) sweep(t, t->left[nd], nd);
            if (is_internal(t, t->right[nd])) sweep(t, t->right[nd], nd);
        } else if (from == t->left[nd]) {
            cla_of(t, nd, UPRIGHT)->dirty = 1;
            cla_of(t, nd, DOWN)->dirty = 1;
            if (is_internal(t, t->right[nd])) sweep(t, t->right[nd], nd);
            if (t->anc[nd] >= 0) sweep(t, t->anc[nd], nd);
            else if (is_internal(t, t->next[t->left[nd]])) sweep(t, t->next[t->left[nd]], nd);
        } else if (from == t->right[nd]) {
            cla_of(t, nd, UPLEFT)->dirty = 1;
            cla_of(t, nd, DOWN)->dirty = 1;
            if (is_internal(t, t->left[nd])) sweep(t, t->left[nd], nd);
            if (t->anc[nd] >= 0) sweep(t, t->anc[nd], nd);
            else if (is_internal(t, t->next[t->left[nd]])) sweep(t, t->next[t->left[nd]], nd);
        }
    }
}

/* Tree::SetBranchLength (tree.h:425) */
void or_tree_set_blen(OrTree *t, int nd, double v) {
    t->dlen[nd] = v;
    sweep(t, nd, -1);
}

static int fp_equals(double a, double b, double eps) { return fabs(a - b) < eps; }

/* Tree::NewtonRaphsonOptimizeBranchLength, optimization.cpp:1359-1971
 * (FP64 build, default NR exit rule, OPT_DEBUG off). */
double or_tree_nr_optimize(OrTree *t, double precision1, int nd) {
    const double min_brlen = t->minBrlen, max_brlen = t->maxBrlen;
    double totalEstImprove = 0.0;
    int iter = 0;
    double abs_d1_prev = FLT_MAX;
    const double v_onEntry = t->dlen[nd];
    double v = t->dlen[nd];
    double v_prev = t->dlen[nd];
    double curScore = t->lnL;
    int negProposalNum = 0;
    double knownMin = min_brlen, knownMax = max_brlen;
    double d1, d2, estScoreDelta, estDeltaNR;
    double initialL = 0.0;
    double out[3];
    for (;;) {
        if (or_tree_derivs(t, nd, out) != 0) return NAN;
        if (iter == 0) initialL = t->lnL;
        d1 = out[1];
        d2 = out[2];
        double dlen = t->dlen[nd];
        estDeltaNR = -d1 / d2;
        estScoreDelta = d1 * estDeltaNR + (d2 * estDeltaNR * estDeltaNR * 0.5);
        if (d1 <= 0.0 && dlen < knownMax) knownMax = dlen;
        else if (d1 > 0.0 && dlen > knownMin) knownMin = dlen;
        double abs_d1 = fabs(d1);
        if (d2 >= 0.0) {
            if (d1 <= 0.0) {
                double proposed;
                if (fp_equals(dlen, min_brlen, 1.0e-8)) {
                    if (t->lnL < initialL - pow(10.0, -6.0 + ceil(log10(-t->lnL)))) {
                        or_tree_set_blen(t, nd, v_onEntry);
                        totalEstImprove = 0.0;
                        or_tree_score(t, 0);
                    }
                    return totalEstImprove;
                }
                if (knownMin == min_brlen) {
                    if (dlen <= 1.0e-4) proposed = min_brlen;
                    else if (dlen <= 0.005) proposed = 1.0e-4;
                    else if (dlen <= 0.05) proposed = dlen * 0.1;
                    else proposed = dlen * 0.25;
                } else
                    proposed = (knownMin + dlen) * 0.5;
                if (iter > 0 || proposed == min_brlen) {
                    double estImp = d1 * (proposed - dlen) + (d2 * (proposed - dlen) * (proposed - dlen) * 0.5);
                    if (estImp < precision1) {
                        if (t->lnL >= initialL - 1.0e-4) return totalEstImprove;
                    }
                }
                v = proposed;
                totalEstImprove += precision1;
            } else {
                double proposed;
                if (knownMax == max_brlen) {
                    if (dlen < 0.1) proposed = dlen * 10.0;
                    else proposed = fmin(dlen * 2.0, max_brlen);
                } else
                    proposed = (knownMax + dlen) * 0.5;
                if (iter > 0) {
                    double estImp = d1 * (proposed - dlen) + (d2 * (proposed - dlen) * (proposed - dlen) * 0.5);
                    if (estImp < precision1) {
                        if (t->lnL >= initialL - 1.0e-4) return totalEstImprove;
                    }
                }
                v = proposed;
                totalEstImprove += precision1;
            }
        } else {
            if (d1 < 0.0 && fp_equals(dlen, min_brlen, 1.0e-8)) return totalEstImprove;
            if (d1 > 0.0 && fp_equals(dlen, max_brlen, 1.0e-8)) return totalEstImprove;
            double tol = (iter < 10 ? 1 : iter) * fmax(1.0e-7, DBL_EPSILON * 10.0);
            if (estScoreDelta < precision1 && (iter == 0 || t->lnL + tol >= initialL)) {
                return totalEstImprove;
            } else {
                int noNR = 0;
                if (iter > 10) {
                    if (d1 > 0.0) {
                        if (fp_equals(knownMax, max_brlen, 1e-8)) {
                            if ((iter > 20) && (dlen > (max_brlen / 2.0))) v = max_brlen;
                            else {
                                if (v < 0.2) v = fmin((v + max_brlen) * 0.5, v * 5.0);
                                else v = fmin((v + max_brlen) * 0.5, v * 2.0);
                            }
                            noNR = 1;
                        } else if (((iter - 20) > 0) && ((iter - 20) % 10 == 0)) {
                            v = fmin((v + knownMax) * 0.5, v * 100.0);
                        }
                    } else {
                        if (fp_equals(knownMin, min_brlen, 1e-8)) {
                            if (iter > 20) v = min_brlen;
                            else v = (v + min_brlen) * 0.5;
                            noNR = 1;
                        }
                    }
                }
                if (!noNR) v += estDeltaNR;
            }
            if (v <= knownMin) {
                negProposalNum++;
                if (knownMin == min_brlen) {
                    double deltaToMin = min_brlen - dlen;
                    double scoreDeltaToMin = (deltaToMin * d1 + (deltaToMin * deltaToMin * d2 * 0.5));
                    if (scoreDeltaToMin < precision1) return totalEstImprove;
                    else if (negProposalNum == 1 && dlen > 1e-4 && v_prev != 1e-4) {
                        if (dlen < .005) v = 1e-4;
                        else if (dlen < 0.05) v = dlen * 0.1;
                        else v = dlen * 0.25;
                        double delta = v - dlen;
                        totalEstImprove += (delta * d1 + (delta * delta * d2 * 0.5));
                    } else {
                        v = min_brlen;
                        totalEstImprove += scoreDeltaToMin;
                    }
                } else {
                    double proposed = (knownMin + dlen) * 0.5;
                    double deltaToMin = proposed - dlen;
                    double scoreDeltaToMin = (deltaToMin * d1 + (deltaToMin * deltaToMin * d2 * 0.5));
                    if (scoreDeltaToMin < precision1) return totalEstImprove;
                    v = proposed;
                    totalEstImprove += scoreDeltaToMin;
                }
            } else if (v >= knownMax) {
                if (knownMax == max_brlen) {
                    double deltaToMax = max_brlen - dlen;
                    double scoreDeltaToMax = (deltaToMax * d1 + (deltaToMax * deltaToMax * d2 * 0.5));
                    if (scoreDeltaToMax < precision1) return totalEstImprove;
                    else {
                        v = max_brlen;
                        totalEstImprove += scoreDeltaToMax;
                    }
                } else {
                    double proposed = (knownMax + dlen) * 0.5;
                    double deltaToMax = proposed - dlen;
                    double scoreDeltaToMax = (deltaToMax * d1 + (deltaToMax * deltaToMax * d2 * 0.5));
                    if (scoreDeltaToMax < precision1) return totalEstImprove;
                    v = proposed;
                    totalEstImprove += scoreDeltaToMax;
                }
            } else
                totalEstImprove += estScoreDelta;
            abs_d1_prev = abs_d1;
        }
        (void)abs_d1_prev;
        or_tree_set_blen(t, nd, v);
        /* curScore bookkeeping (optimization.cpp:1849-1872): SetBranchLength leaves lnL = -1,
         * so the "score got worse" branch never triggers; curScore becomes -1. */
        curScore = t->lnL;
        (void)curScore;
        v_prev = v;
        iter++;
        if (iter > 100) {
            or_tree_score(t, t->anc[nd]);
            if (t->lnL > initialL) return totalEstImprove;
            or_tree_set_blen(t, nd, v_onEntry);
            or_tree_score(t, 0);
            return 0.0;
        }
    }
}

/* Tree::OptimizeBranchLength (optimization.cpp:777) + RecursivelyOptimizeBranches
 * (optimization.cpp:1042-1062) as driven by OptimizeAllBranches (optimization.cpp:97). */
static double rec_opt(OrTree *t, int nd, double prec, int radius, int dontGoNext, double scoreIncrease,
                      int ignoreDelta) {
    double delta = 0.0;
    if (!t->optimized[nd]) {
        t->optimized[nd] = 1;
        delta = or_tree_nr_optimize(t, prec, nd);
    }
    scoreIncrease += delta;
    if (t->left[nd] >= 0 && radius > 1 && (!(delta < prec) || ignoreDelta))
        scoreIncrease += rec_opt(t, t->left[nd], prec, radius - 1, 0, 0, ignoreDelta);
    if (t->next[nd] >= 0 && !dontGoNext) {
        if (!t->optimized[t->next[nd]]) scoreIncrease += rec_opt(t, t->next[nd], prec, radius, 0, 0, ignoreDelta);
    }
    return scoreIncrease;
}

double or_tree_optimize_all(OrTree *t, double prec) {
    double improve = 0.0;
    memset(t->optimized, 0, t->nnodes);
    int l = t->left[0], m = t->next[l], r = t->right[0];
    improve = rec_opt(t, l, prec, t->nnodes, 1, improve, 1);
    improve = rec_opt(t, m, prec, t->nnodes, 1, improve, 1);
    improve = rec_opt(t, r, prec, t->nnodes, 1, improve, 1);
    return improve;
}

int or_tree_get_cla(const OrTree *t, int nd, int which, double *arr, int *mult) {
    const OrCla *c = &t->cla[nd * 3 + which];
    if (c->dirty || !c->arr) return -1;
    if (arr) memcpy(arr, c->arr, sizeof(double) * (size_t)t->npat * t->R * t->S);
    if (mult) memcpy(mult, c->mult, sizeof(int) * t->npat);
    return 0;
}
int or_tree_cla_rank(const OrTree *t, int nd, int which) { return t->cla[nd * 3 + which].rank; }
int or_tree_cla_dirty(const OrTree *t, int nd, int which) { return t->cla[nd * 3 + which].dirty; }
int or_tree_site_lnl(const OrTree *t, double *out) {
    if (!t->siteValid) return -1;
    memcpy(out, t->siteLnL, sizeof(double) * t->npat);
    return 0;
}
