// pq_setup.cpp -- host-side model set-up: stratification, the
// non-dimensionalisation and forcing of the double-gyre driver, and the
// seeded synthetic initial condition.
#include <cmath>
#include <cstring>
#include <vector>

#include "pequod_b200.h"

namespace {

const double kPi = 3.14159265358979323846;

// Symmetric eigen-decomposition of a small dense matrix by cyclic Jacobi
// rotations (Golub & Van Loan, Matrix Computations, sec. 8.5).  a: n x n
// row-major, destroyed.  vec: eigenvectors as columns, row-major.
void jacobi_eig(int n, std::vector<double>& a, std::vector<double>& val, std::vector<double>& vec) {
    vec.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) vec[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0;
        for (int r = 0; r < n; ++r)
            for (int c = r + 1; c < n; ++c) off += a[(size_t)r * n + c] * a[(size_t)r * n + c];
        if (off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = a[(size_t)p * n + q];
                if (apq == 0.0) continue;
                const double tau = (a[(size_t)q * n + q] - a[(size_t)p * n + p]) / (2.0 * apq);
                const double t = std::copysign(1.0, tau) / (std::fabs(tau) + std::hypot(1.0, tau));
                const double c = 1.0 / std::hypot(1.0, t), s = t * c;
                for (int k = 0; k < n; ++k) {  // columns p, q
                    const double x = a[(size_t)k * n + p], y = a[(size_t)k * n + q];
                    a[(size_t)k * n + p] = c * x - s * y;
                    a[(size_t)k * n + q] = s * x + c * y;
                }
                for (int k = 0; k < n; ++k) {  // rows p, q
                    const double x = a[(size_t)p * n + k], y = a[(size_t)q * n + k];
                    a[(size_t)p * n + k] = c * x - s * y;
                    a[(size_t)q * n + k] = s * x + c * y;
                }
                for (int k = 0; k < n; ++k) {
                    const double x = vec[(size_t)k * n + p], y = vec[(size_t)k * n + q];
                    vec[(size_t)k * n + p] = c * x - s * y;
                    vec[(size_t)k * n + q] = s * x + c * y;
                }
            }
    }
    val.resize(n);
    for (int i = 0; i < n; ++i) val[i] = a[(size_t)i * n + i];
}

// Gauss-Jordan inverse with partial pivoting, row-major.
bool invert(int n, std::vector<double> a, std::vector<double>& inv) {
    inv.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(a[(size_t)r * n + c]) > std::fabs(a[(size_t)p * n + c])) p = r;
        if (a[(size_t)p * n + c] == 0.0) return false;
        for (int k = 0; k < n; ++k) {
            std::swap(a[(size_t)c * n + k], a[(size_t)p * n + k]);
            std::swap(inv[(size_t)c * n + k], inv[(size_t)p * n + k]);
        }
        const double d = a[(size_t)c * n + c];
        for (int k = 0; k < n; ++k) {
            a[(size_t)c * n + k] /= d;
            inv[(size_t)c * n + k] /= d;
        }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = a[(size_t)r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                a[(size_t)r * n + k] -= f * a[(size_t)c * n + k];
                inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
            }
        }
    }
    return true;
}

uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" {

// Stratification matrix S (s_matrix, qg3p_diagnostics.F90:342-366) is
// tridiagonal with S(k,k+1) S(k+1,k) = s2(k) s1(k+1) > 0, so it is similar to
// a symmetric matrix through a diagonal scaling; its eigenvalues are -ss and
// its eigenvectors the columns of modes_to_z.  As in sort_barotropic (:389-
// 420) the barotropic mode (eigenvalue 0) goes first with all components 1
// and ss(1) = 0; the baroclinic modes follow in order of increasing ss.
int pq_stratification(pq_model_desc* d, int L, const double* H, const double* s1_in, const double* s2_in,
                      double l_scale) {
    if (!d || L < 1 || L > PQ_MAX_LAYERS || !H || l_scale <= 0.0) return PQ_ERR_ARG;
    const double ls2 = l_scale * l_scale;
    for (int k = 0; k < PQ_MAX_LAYERS; ++k) d->h[k] = d->s1[k] = d->s2[k] = d->ss[k] = 0.0;
    for (int k = 0; k < L; ++k) d->h[k] = H[k] / l_scale;
    for (int k = 0; k + 1 < L; ++k) {
        d->s1[k + 1] = ls2 * s1_in[k];
        d->s2[k] = ls2 * s2_in[k];
    }
    std::vector<double> S((size_t)L * L, 0.0);  // row-major
    for (int k = 0; k < L; ++k) {
        if (k > 0) S[(size_t)k * L + k - 1] = d->s1[k];
        if (k + 1 < L) S[(size_t)k * L + k + 1] = d->s2[k];
        double diag = 0.0;
        if (k > 0) diag -= d->s1[k];
        if (k + 1 < L) diag -= d->s2[k];
        S[(size_t)k * L + k] = diag;
    }
    // D S D^-1 symmetric with D = diag(w), w(k+1)/w(k) = sqrt(S(k,k+1)/S(k+1,k)).
    std::vector<double> w(L, 1.0);
    for (int k = 0; k + 1 < L; ++k) {
        const double up = S[(size_t)k * L + k + 1], lo = S[(size_t)(k + 1) * L + k];
        if (!(up > 0.0 && lo > 0.0)) return PQ_ERR_ARG;
        w[k + 1] = w[k] * std::sqrt(up / lo);
    }
    std::vector<double> T((size_t)L * L);
    for (int r = 0; r < L; ++r)
        for (int c = 0; c < L; ++c) T[(size_t)r * L + c] = w[r] * S[(size_t)r * L + c] / w[c];
    std::vector<double> val, vec;
    jacobi_eig(L, T, val, vec);
    // Eigenvalue k of S: val[k]; eigenvector D^-1 q_k.  Barotropic: largest
    // eigenvalue (= 0 up to rounding).
    std::vector<int> ord(L);
    for (int k = 0; k < L; ++k) ord[k] = k;
    for (int a = 1; a < L; ++a)
        for (int b = a; b > 0 && val[ord[b]] > val[ord[b - 1]]; --b) std::swap(ord[b], ord[b - 1]);
    std::vector<double> m2z((size_t)L * L);  // row-major [layer][mode]
    for (int m = 0; m < L; ++m) {
        const int e = ord[m];
        if (m == 0) {
            for (int l = 0; l < L; ++l) m2z[(size_t)l * L] = 1.0;
            d->ss[0] = 0.0;
        } else {
            // Normalise the eigenvector so that its first component is 1.
            const double v0 = vec[(size_t)0 * L + e] / w[0];
            for (int l = 0; l < L; ++l) m2z[(size_t)l * L + m] = (vec[(size_t)l * L + e] / w[l]) / v0;
            d->ss[m] = -val[e];
        }
    }
    std::vector<double> z2m;
    if (!invert(L, m2z, z2m)) return PQ_ERR_ARG;
    for (int k = 0; k < PQ_MAX_LAYERS * PQ_MAX_LAYERS; ++k) d->m2z[k] = d->z2m[k] = 0.0;
    for (int r = 0; r < L; ++r)
        for (int c = 0; c < L; ++c) {
            d->m2z[r + L * c] = m2z[(size_t)r * L + c];  // column-major, leading dimension L
            d->z2m[r + L * c] = z2m[(size_t)r * L + c];
        }
    d->layers = L;
    return PQ_OK;
}

int pq_setup_double_gyre(const pq_physical* p, pq_model_desc* d, double* wind_out, double* t_scale_out) {
    if (!p || !d || p->layers < 1 || p->layers > PQ_MAX_LAYERS || p->ii < 5 || p->jj < 5) return PQ_ERR_ARG;
    std::memset(d, 0, sizeof(*d));
    const int L = p->layers, ii = p->ii, jj = p->jj;
    d->ii = ii;
    d->jj = jj;
    d->scheme = p->scheme;
    d->limiter = p->limiter;
    d->precision = p->precision;
    d->adapt_dt = p->adapt_dt;
    const double u_scale = p->u_scale > 0.0 ? p->u_scale : 1.0;
    const int g_ii_int = ii - 1;
    // qg3.F90:152-168
    const double l_scale = p->basinscale / (double)g_ii_int;
    const double t_scale = l_scale / u_scale;
    d->dt = p->dt / t_scale;
    d->max_dt = p->max_dt > 0.0 ? p->max_dt / t_scale : 1.0e300;
    d->target_cfl = p->target_cfl;
    d->max_dt_increase = p->max_dt_increase;
    d->alpha = l_scale / p->alpha;
    for (int k = 0; k < L; ++k) d->beta[k] = p->beta * l_scale * l_scale / u_scale;
    d->viscosity = p->visc / (l_scale * u_scale);
    d->visc_bot = p->visc_bot * l_scale / u_scale;
    d->ra_nu = 0.02;
    d->ra_alpha = 0.5;
    // Stratification input (qg3p_io.F90:56-102): s2(k) = f0^2/(g'_k H_k),
    // s1(k+1) = f0^2/(g'_k H_(k+1)).
    double s1[PQ_MAX_LAYERS] = {0}, s2[PQ_MAX_LAYERS] = {0};
    for (int k = 0; k + 1 < L; ++k) {
        const double f2g = p->f0 * p->f0 / p->gprime[k];
        s2[k] = f2g / p->H[k];
        s1[k] = f2g / p->H[k + 1];
    }
    int rc = pq_stratification(d, L, p->H, s1, s2, l_scale);
    if (rc != PQ_OK) return rc;
    // Boundary condition (qg3.F90:248-257).
    if (p->partial_slip) {
        d->bc_type = (p->alpha >= 1.0e100) ? PQ_BC_FREE_SLIP : PQ_BC_PARTIAL_SLIP;
        if (d->bc_type == PQ_BC_FREE_SLIP) d->alpha = 0.0;
    } else {
        d->bc_type = PQ_BC_NO_SLIP;
    }
    // Wind forcing, qg3.F90:253-271, with tau scaled by h(1) (:235).
    if (wind_out) {
        const double tau = p->tau / (u_scale * u_scale * (double)g_ii_int) / d->h[0];
        const double a_wind = -1.0 * p->wind_asym, b_wind = 1.0 / p->wind_asym;
        for (int j = 1; j <= jj; ++j)
            for (int i = 1; i <= ii; ++i) {
                const double x = (double)(j - 1) / (double)(jj - 1) - 0.5;
                const double y = -(double)(i - 1) / (double)(ii - 1) + 0.5;
                const double y_mid = p->wind_shift + p->wind_tilt * x;
                double f;
                if (y < y_mid)
                    f = a_wind * std::sin(kPi * (0.5 + y) / (0.5 + y_mid));
                else
                    f = b_wind * std::sin(kPi * (y - y_mid) / (0.5 - y_mid));
                wind_out[(size_t)(i - 1) + (size_t)ii * (j - 1)] = tau * 2.0 * kPi * f;
            }
        d->force_wind = wind_out;
    }
    if (t_scale_out) *t_scale_out = t_scale;
    return PQ_OK;
}

int pq_make_ic(int ii, int jj, int L, uint64_t seed, double amplitude, double sigma, double* out) {
    if (ii < 1 || jj < 1 || L < 1 || !out) return PQ_ERR_ARG;
    const size_t plane = (size_t)ii * jj;
    uint64_t s = seed * 0x2545F4914F6CDD1Dull + 0x1234567ull;
    std::vector<double> noise(plane * L);
    for (size_t k = 0; k < noise.size(); k += 2) {
        // Box-Muller on two uniform (0, 1] variates.
        const double u1 = ((splitmix64(s) >> 11) + 1.0) * (1.0 / 9007199254740992.0);
        const double u2 = ((splitmix64(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        const double r = std::sqrt(-2.0 * std::log(u1));
        noise[k] = r * std::cos(2.0 * kPi * u2);
        if (k + 1 < noise.size()) noise[k + 1] = r * std::sin(2.0 * kPi * u2);
    }
    std::vector<double> ker;
    int R = 0;
    if (sigma > 0.0) {
        R = (int)std::ceil(3.0 * sigma);
        ker.resize(2 * R + 1);
        double t = 0.0;
        for (int q = -R; q <= R; ++q) t += (ker[q + R] = std::exp(-0.5 * (q * q) / (sigma * sigma)));
        for (double& v : ker) v /= t;
    }
    std::vector<double> tmp(plane);
    for (int l = 0; l < L; ++l) {
        double* f = noise.data() + plane * l;
        if (R > 0) {
            for (int j = 0; j < jj; ++j)
                for (int i = 0; i < ii; ++i) {
                    double a = 0.0;
                    for (int q = -R; q <= R; ++q) {
                        const int ik = i + q;
                        if (ik >= 0 && ik < ii) a += ker[q + R] * f[(size_t)ik + (size_t)ii * j];
                    }
                    tmp[(size_t)i + (size_t)ii * j] = a;
                }
            for (int j = 0; j < jj; ++j)
                for (int i = 0; i < ii; ++i) {
                    double a = 0.0;
                    for (int q = -R; q <= R; ++q) {
                        const int jk = j + q;
                        if (jk >= 0 && jk < jj) a += ker[q + R] * tmp[(size_t)i + (size_t)ii * jk];
                    }
                    f[(size_t)i + (size_t)ii * j] = a;
                }
        }
        for (size_t k = 0; k < plane; ++k) out[plane * l + k] = amplitude * f[k];
    }
    return PQ_OK;
}

}  // extern "C"
