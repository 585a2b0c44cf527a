// gb_model.cpp -- host-side model math of the engine (GARLI's Model class,
// garli/trunk/src/model.cpp): rate matrices, their eigensystems and the
// discrete-gamma rates.  These run once per model change; the per-branch
// exponentiation P(t) = U exp(Lambda t) U^-1 runs on the device (gb_pmat.cuh).
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/garli_b200.h"

namespace {

// Standard genetic code in ACGT base-4 codon order (AAA, AAC, ..., TTT); '*' = stop.
// Role of GeneticCode::SetStandardCode (sequencedata.h:217).
const char *kStdCode = "KNKNTTTTRSRSIIMIQHQHPPPPRRRRLLLLEDEDAAAAGGGGVVVV*Y*YSSSS*CWCLFLF";

// Householder reduction of a symmetric matrix to tridiagonal form, accumulating
// the orthogonal transform in z (row-major n x n); d = diagonal, e = sub-diagonal.
void householder_tridiag(int n, std::vector<double> &z, std::vector<double> &d, std::vector<double> &e) {
    auto Z = [&](int i, int j) -> double & { return z[(size_t)i * n + j]; };
    for (int i = n - 1; i > 0; i--) {
        const int l = i - 1;
        double h = 0.0, scale = 0.0;
        if (l > 0) {
            for (int k = 0; k <= l; k++) scale += std::fabs(Z(i, k));
            if (scale == 0.0) {
                e[i] = Z(i, l);
            } else {
                for (int k = 0; k <= l; k++) {
                    Z(i, k) /= scale;
                    h += Z(i, k) * Z(i, k);
                }
                double f = Z(i, l);
                double g = f >= 0.0 ? -std::sqrt(h) : std::sqrt(h);
                e[i] = scale * g;
                h -= f * g;
                Z(i, l) = f - g;
                f = 0.0;
                for (int j = 0; j <= l; j++) {
                    Z(j, i) = Z(i, j) / h;
                    g = 0.0;
                    for (int k = 0; k <= j; k++) g += Z(j, k) * Z(i, k);
                    for (int k = j + 1; k <= l; k++) g += Z(k, j) * Z(i, k);
                    e[j] = g / h;
                    f += e[j] * Z(i, j);
                }
                const double hh = f / (h + h);
                for (int j = 0; j <= l; j++) {
                    f = Z(i, j);
                    e[j] = g = e[j] - hh * f;
                    for (int k = 0; k <= j; k++) Z(j, k) -= (f * e[k] + g * Z(i, k));
                }
            }
        } else {
            e[i] = Z(i, l);
        }
        d[i] = h;
    }
    d[0] = 0.0;
    e[0] = 0.0;
    for (int i = 0; i < n; i++) {
        const int l = i - 1;
        if (d[i] != 0.0) {
            for (int j = 0; j <= l; j++) {
                double g = 0.0;
                for (int k = 0; k <= l; k++) g += Z(i, k) * Z(k, j);
                for (int k = 0; k <= l; k++) Z(k, j) -= g * Z(k, i);
            }
        }
        d[i] = Z(i, i);
        Z(i, i) = 1.0;
        for (int j = 0; j <= l; j++) Z(j, i) = Z(i, j) = 0.0;
    }
}

// QL iteration with implicit shifts on the tridiagonal (d, e); eigenvectors
// accumulate into the columns of z.
bool tridiag_ql(int n, std::vector<double> &d, std::vector<double> &e, std::vector<double> &z) {
    auto Z = [&](int i, int j) -> double & { return z[(size_t)i * n + j]; };
    for (int i = 1; i < n; i++) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    for (int l = 0; l < n; l++) {
        int iter = 0, m;
        do {
            for (m = l; m < n - 1; m++) {
                const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= 1e-300 + 1e-17 * dd) break;
            }
            if (m != l) {
                if (iter++ == 200) return false;
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = std::hypot(g, 1.0);
                g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? std::fabs(r) : -std::fabs(r)));
                double s = 1.0, c = 1.0, p = 0.0;
                int i;
                for (i = m - 1; i >= l; i--) {
                    double f = s * e[i], b = c * e[i];
                    e[i + 1] = (r = std::hypot(f, g));
                    if (r == 0.0) {
                        d[i + 1] -= p;
                        e[m] = 0.0;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    d[i + 1] = g + (p = s * r);
                    g = c * r - b;
                    for (int k = 0; k < n; k++) {
                        f = Z(k, i + 1);
                        Z(k, i + 1) = s * Z(k, i) + c * f;
                        Z(k, i) = c * Z(k, i) - s * f;
                    }
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }
    return true;
}

// ---- discrete gamma: Model::DiscreteGamma (model.cpp:2170-2201) ----
// The chi-square percentage point follows AS 91 (Best & Roberts 1975): a
// starting approximation, then a seven-term Taylor correction iterated until
// the relative change is below 0.5e-6; the incomplete gamma ratio is the
// series / continued-fraction pair used by AS 239.
double ln_gamma(double x) {
    double f = 0.0;
    if (x < 7.0) {
        double prod = 1.0;
        for (; x < 7.0; x += 1.0) prod *= x;
        f = -std::log(prod);
    }
    const double z = 1.0 / (x * x);
    return f + (x - 0.5) * std::log(x) - x + 0.918938533204672742 +
           (((-0.000595238095238 * z + 0.000793650793651) * z - 0.002777777777778) * z + 0.083333333333333) / x;
}

double incomplete_gamma(double x, double alpha, double ln_gamma_alpha) {
    if (x <= 0.0) return 0.0;
    const double factor = std::exp(alpha * std::log(x) - x - ln_gamma_alpha);
    if (x <= 1.0 || x < alpha) {
        double gin = 1.0, term = 1.0, rn = alpha;
        for (int i = 0; i < 100000; i++) {
            rn += 1.0;
            term *= x / rn;
            gin += term;
            if (term <= 1e-16 * gin) break;
        }
        return gin * factor / alpha;
    }
    const double tiny = 1e-300;
    double b = x + 1.0 - alpha, c = 1.0 / tiny, d = 1.0 / b, h = d;
    for (int i = 1; i < 100000; i++) {
        const double an = -i * (i - alpha);
        b += 2.0;
        d = an * d + b;
        if (std::fabs(d) < tiny) d = tiny;
        c = b + an / c;
        if (std::fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        const double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) < 1e-16) break;
    }
    return 1.0 - factor * h;
}

// inverse standard normal (Odeh & Evans 1974, AS 70 rational approximation)
double point_normal(double prob) {
    const double a0 = -0.322232431088, a1 = -1.0, a2 = -0.342242088547, a3 = -0.0204231210245;
    const double a4 = -0.453642210148e-4, b0 = 0.0993484626060, b1 = 0.588581570495;
    const double b2 = 0.531103462366, b3 = 0.103537752850, b4 = 0.38560700634e-2;
    const double p = prob, p1 = (p < 0.5 ? p : 1.0 - p);
    if (p1 < 1e-20) return -9999.0;
    const double y = std::sqrt(std::log(1.0 / (p1 * p1)));
    const double z = y + ((((y * a4 + a3) * y + a2) * y + a1) * y + a0) / ((((y * b4 + b3) * y + b2) * y + b1) * y + b0);
    return p < 0.5 ? -z : z;
}

double point_chi2(double prob, double v) {
    const double e = 0.5e-6, aa = 0.6931471805;
    const double p = prob;
    if (p < 0.000002 || p > 0.999998 || v <= 0.0) return -1.0;
    const double g = ln_gamma(v / 2.0);
    const double xx = v / 2.0, c = xx - 1.0;
    double ch;
    if (v < -1.24 * std::log(p)) {
        ch = std::pow(p * xx * std::exp(g + xx * aa), 1.0 / xx);
        if (ch - e < 0) return ch;
    } else if (v > 0.32) {
        const double x = point_normal(p);
        const double p1 = 0.222222 / v;
        ch = v * std::pow(x * std::sqrt(p1) + 1.0 - p1, 3.0);
        if (ch > 2.2 * v + 6.0) ch = -2.0 * (std::log(1.0 - p) - c * std::log(0.5 * ch) + g);
    } else {
        ch = 0.4;
        const double a = std::log(1.0 - p);
        double q;
        do {
            q = ch;
            const double p1 = 1.0 + ch * (4.67 + ch);
            const double p2 = ch * (6.73 + ch * (6.66 + ch));
            const double t = -0.5 + (4.67 + 2.0 * ch) / p1 - (6.73 + ch * (13.32 + 3.0 * ch)) / p2;
            ch -= (1.0 - std::exp(a + g + 0.5 * ch + c * aa) * p2 / p1) / t;
        } while (std::fabs(q / ch - 1.0) - 0.01 > 0.0);
    }
    for (int it = 0; it < 1000; it++) {
        const double q = ch;
        const double p1 = 0.5 * ch;
        const double t0 = incomplete_gamma(p1, xx, g);
        const double p2 = p - t0;
        const double t = p2 * std::exp(xx * aa + g + p1 - c * std::log(ch));
        const double b = t / ch, a = 0.5 * t - b * c;
        const double s1 = (210.0 + a * (140.0 + a * (105.0 + a * (84.0 + a * (70.0 + 60.0 * a))))) / 420.0;
        const double s2 = (420.0 + a * (735.0 + a * (966.0 + a * (1141.0 + 1278.0 * a)))) / 2520.0;
        const double s3 = (210.0 + a * (462.0 + a * (707.0 + 932.0 * a))) / 2520.0;
        const double s4 = (252.0 + a * (672.0 + 1182.0 * a) + c * (294.0 + a * (889.0 + 1740.0 * a))) / 5040.0;
        const double s5 = (84.0 + 264.0 * a + c * (175.0 + 606.0 * a)) / 2520.0;
        const double s6 = (120.0 + c * (346.0 + 127.0 * c)) / 5040.0;
        ch += t * (1.0 + 0.5 * t * s1 - b * c * (s1 - b * (s2 - b * (s3 - b * (s4 - b * (s5 - b * s6))))));
        if (std::fabs(q / ch - 1.0) <= e) break;
    }
    return ch;
}

}  // namespace

extern "C" {

int gbm_gtr_qmat(const double *rel, const double *pi, double *Q, double *blenMult) {
    double q[4][4] = {{0}};
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
    *blenMult = 0.5 / ((q[0][1] * pi[0]) + (q[0][2] * pi[0]) + (q[0][3] * pi[0]) + (q[1][2] * pi[1]) +
                       (q[1][3] * pi[1]) + (q[2][3] * pi[2]));
    std::memcpy(Q, q, sizeof(q));
    return GB_SUCCESS;
}

int gbm_aa_qmat(const double *exch, const double *pi, double *Q, double *blenMult) {
    const int n = 20;
    for (int f = 0; f < n; f++)
        for (int t = 0; t < n; t++) Q[f * n + t] = pi[t];
    int r = 0;
    for (int f = 0; f < n - 1; f++)
        for (int t = f + 1; t < n; t++) Q[f * n + t] *= exch[r++];
    r = 0;
    for (int t = 0; t < n - 1; t++)
        for (int f = t + 1; f < n; f++) Q[f * n + t] *= exch[r++];
    double w = 0.0;
    for (int f = 0; f < n; f++) {
        double sum = 0.0;
        for (int t = 0; t < n; t++)
            if (f != t) sum += Q[f * n + t];
        Q[f * n + f] = -sum;
        w += sum * pi[f];
    }
    *blenMult = 1.0 / w;
    return GB_SUCCESS;
}

int gbm_codon_qmat6(const double *rel6, double omega, const double *pi, double *Q, double *blenMult) {
    int sense[64], ns = 0;
    for (int c = 0; c < 64; c++)
        if (kStdCode[c] != '*') sense[ns++] = c;
    const int n = 61;
    // nucleotide-pair rate index, AC AG AT CG CT GT (qmatLookup bits 8..256, model.cpp:296-441)
    static const int kPair[4][4] = {{-1, 0, 1, 2}, {0, -1, 3, 4}, {1, 3, -1, 5}, {2, 4, 5, -1}};
    for (int a = 0; a < n; a++)
        for (int b = 0; b < n; b++) {
            const int ca = sense[a], cb = sense[b];
            int ndiff = 0, x0 = 0, y0 = 0;
            for (int pos = 0; pos < 3; pos++) {
                const int sh = 2 * (2 - pos);
                const int x = (ca >> sh) & 3, y = (cb >> sh) & 3;
                if (x != y) {
                    ndiff++;
                    x0 = x;
                    y0 = y;
                }
            }
            double q = 0.0;
            if (a != b && ndiff == 1) {
                q = pi[b];
                q *= rel6[kPair[x0][y0]];
                if (kStdCode[ca] != kStdCode[cb]) q *= omega;  // nonsynonymous (bit 4)
            }
            Q[a * n + b] = q;
        }
    double w = 0.0;
    for (int x = 0; x < n; x++) {
        double sum = 0.0;
        for (int y = 0; y < n; y++)
            if (x != y) sum += Q[x * n + y];
        Q[x * n + x] = -sum;
        w += sum * pi[x];
    }
    *blenMult = 1.0 / w;
    return GB_SUCCESS;
}

int gbm_codon_qmat(double kappa, double omega, const double *pi, double *Q, double *blenMult) {
    const double rel6[6] = {1.0, kappa, 1.0, 1.0, kappa, 1.0};  // GY94: kappa on transitions
    return gbm_codon_qmat6(rel6, omega, pi, Q, blenMult);
}

// Eigensystem of a reversible Q through its symmetric similar matrix
// A = D^1/2 Q D^-1/2, D = diag(pi): Householder tridiagonalisation + implicit QL;
// U = D^-1/2 V, U^-1 = V^T D^1/2.
int gbm_eigen(int n, const double *Q, const double *pi, double *eval, double *U, double *Uinv) {
    if (n < 2 || n > 64) return GB_ERROR_OUT_OF_RANGE;
    std::vector<double> sq(n), isq(n), z((size_t)n * n), d(n), e(n);
    for (int i = 0; i < n; i++) {
        if (!(pi[i] > 0.0)) return GB_ERROR_OUT_OF_RANGE;
        sq[i] = std::sqrt(pi[i]);
        isq[i] = 1.0 / sq[i];
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) z[(size_t)i * n + j] = sq[i] * Q[i * n + j] * isq[j];
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            const double m = 0.5 * (z[(size_t)i * n + j] + z[(size_t)j * n + i]);
            z[(size_t)i * n + j] = z[(size_t)j * n + i] = m;
        }
    householder_tridiag(n, z, d, e);
    if (!tridiag_ql(n, d, e, z)) return GB_ERROR_FLOATING_POINT;
    for (int k = 0; k < n; k++) eval[k] = d[k];
    for (int i = 0; i < n; i++)
        for (int k = 0; k < n; k++) {
            U[i * n + k] = isq[i] * z[(size_t)i * n + k];
            Uinv[k * n + i] = z[(size_t)i * n + k] * sq[i];
        }
    return GB_SUCCESS;
}

int gbm_discrete_gamma(double alpha, int ncat, double *rates) {
    if (ncat < 1 || ncat > 64 || !(alpha > 0.0)) return GB_ERROR_OUT_OF_RANGE;
    if (ncat == 1) {
        rates[0] = 1.0;
        return GB_SUCCESS;
    }
    std::vector<double> props(ncat);
    const double factor = alpha / alpha * ncat;
    const double lnga1 = ln_gamma(alpha + 1.0);
    for (int i = 0; i < ncat - 1; i++) props[i] = point_chi2((i + 1.0) / ncat, 2.0 * alpha) / (2.0 * alpha);
    for (int i = 0; i < ncat - 1; i++) props[i] = incomplete_gamma(props[i] * alpha, alpha + 1.0, lnga1);
    rates[0] = props[0] * factor;
    rates[ncat - 1] = (1.0 - props[ncat - 2]) * factor;
    for (int i = 1; i < ncat - 1; i++) rates[i] = (props[i] - props[i - 1]) * factor;
    return GB_SUCCESS;
}

}  // extern "C"
