// pq_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see pq_oracle.h).
//
// CPU FP64 restatement of PEQUOD's serial QG time-step hot path.  Each routine
// cites the reference file:line it follows (paths relative to the PEQUOD
// source tree).  The serial path is restated for one MPI rank: every halo
// update and flush in the reference is a no-op there (qg3p_base.F90:1895,
// update_pdata returns when n == 1 and not periodic), so none appear here.
//
// Build: see oracle/Makefile.  Compiled without -ffast-math and without FMA
// contraction so that results are deterministic and follow the reference's
// operation order.
#include "pq_oracle.h"

#include <cmath>
#include <cstdint>
#include <limits>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

// Constants exactly as qg3p_params.F90:110-117 declares them.  two_pi, sqrt3
// and hsqt2 are deliberately the reference's truncated literals.
const double PI = 3.14159265358979323846;
const double TWO_PI = 6.28318530717959;
const double SQRT3 = 1.73205080756888;
const double HSQT2 = 0.7071067811865475;

// ---------------------------------------------------------------------------
// Fortran-style views (1-based, column-major).
struct V2 {
    double* p;
    int n1, n2;
    double& operator()(int i, int j) const { return p[(size_t)(i - 1) + (size_t)n1 * (size_t)(j - 1)]; }
};
struct V3 {
    double* p;
    int n1, n2, n3;
    double& operator()(int i, int j, int k) const {
        return p[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (size_t)(k - 1))];
    }
};

// ---------------------------------------------------------------------------
// Index ranges for one rank, allocate_decomp (qg3p_base.F90:775-941).
struct Decomp {
    int ii, jj, layers;
    bool periodic_j;
    int p_a, p_b, p_c, p_d;
    int ii2, jj2, g_ii, g_jj, g_ii2, g_jj2, g_ii_int, g_jj_int;
    int f_i_min, f_i_max, f_j_min, f_j_max;
    int l_i_min, l_i_max, l_j_min, l_j_max;
    int fa_i_min, fa_i_max, fa_j_min, fa_j_max;
    int fb_i_min, fb_i_max, fb_j_min, fb_j_max;
};

Decomp make_decomp(int ii, int jj, int layers, bool periodic_j) {
    Decomp d;
    d.ii = ii;
    d.jj = jj;
    d.layers = layers;
    d.periodic_j = periodic_j;
    d.g_ii = ii;
    d.g_jj = jj;
    d.g_ii2 = ii - 2;
    d.g_ii_int = ii - 1;
    if (periodic_j) {
        d.g_jj2 = jj;
        d.g_jj_int = jj;
    } else {
        d.g_jj2 = jj - 2;
        d.g_jj_int = jj - 1;
    }
    // One process: no neighbours in i; in j the periodic rank is its own
    // neighbour (mpi_cart_rank on a periodic dimension of size one).
    d.p_b = -1;
    d.p_d = -1;
    d.p_a = periodic_j ? 0 : -1;
    d.p_c = periodic_j ? 0 : -1;
    d.ii2 = ii;
    d.jj2 = jj;
    if (d.p_b == -1) d.ii2 -= 1;
    if (d.p_d == -1) d.ii2 -= 1;
    if (d.p_c == -1) d.jj2 -= 1;
    if (d.p_a == -1) d.jj2 -= 1;
    d.f_i_min = d.p_b >= 0 ? 2 : 3;
    d.f_i_max = d.p_d >= 0 ? ii + 1 : ii;
    d.f_j_min = d.p_c >= 0 ? 2 : 3;
    d.f_j_max = d.p_a >= 0 ? jj + 1 : jj;
    d.l_i_min = d.f_i_min - 1;
    d.l_i_max = d.l_i_min + d.ii2 - 1;
    d.l_j_min = d.f_j_min - 1;
    d.l_j_max = d.l_j_min + d.jj2 - 1;
    d.fa_i_min = d.f_i_min - 1;
    d.fa_i_max = d.f_i_max + 1;
    d.fa_j_min = d.f_j_min - 1;
    d.fa_j_max = d.f_j_max + 1;
    d.fb_i_min = d.p_b >= 0 ? d.f_i_min : d.f_i_min - 1;
    d.fb_i_max = d.p_d >= 0 ? d.f_i_max : d.f_i_max + 1;
    d.fb_j_min = d.p_c >= 0 ? d.f_j_min : d.f_j_min - 1;
    d.fb_j_max = d.p_a >= 0 ? d.f_j_max : d.f_j_max + 1;
    return d;
}

// ---------------------------------------------------------------------------
// FFTPACK-derived sine transform, qg3p_helmholtz.F90:168-289, 1370-1591.
struct Rfft {
    int n = 0;
    int nf = 0;
    int ifac[64];
    std::vector<double> wa;  // wa(1:n)
};

struct Sint {
    int n = 0;
    std::vector<double> cc;   // cc(1:n+1)
    std::vector<double> was;  // was(1:n/2)
    Rfft rfft;
};

// rffti1, qg3p_helmholtz.F90:202-289.
void rffti1(Rfft& r, int n) {
    static const int ntryh[9] = {4, 2, 3, 5, 7, 11, 13, 17, 19};
    r.n = n;
    r.wa.assign((size_t)n + 1, 0.0);  // 1-based
    int nl = n, nf = 0, j = 1, ntry = ntryh[0];
    while (nl != 1) {
        while (nl % ntry != 0) {
            j += 1;
            if (j <= 9)
                ntry = ntryh[j - 1];
            else
                ntry += 2;
        }
        nf += 1;
        r.ifac[nf] = ntry;
        nl /= ntry;
        if (ntry == 2 && nf > 1) {
            for (int i = nf; i >= 2; --i) r.ifac[i] = r.ifac[i - 1];
            r.ifac[1] = 2;
        }
    }
    r.nf = nf;
    if (nf == 0) return;
    double argh = TWO_PI / (double)n;
    int is = 0, l1 = 1;
    for (int k1 = 1; k1 <= nf - 1; ++k1) {
        int ip = r.ifac[k1];
        int l2 = l1 * ip;
        int ido = n / l2;
        int ld = 0;
        for (int jj = 1; jj <= ip - 1; ++jj) {
            ld += l1;
            double argld = (double)ld * argh;
            double fi = 0.0;
            for (int ii = 2; ii <= ido - 1; ii += 2) {
                int i = is + ii;
                fi += 1.0;
                double arg = fi * argld;
                r.wa[i - 1] = std::cos(arg);
                r.wa[i] = std::sin(arg);
            }
            is += ido;
        }
        l1 = l2;
    }
}

// sinti, qg3p_helmholtz.F90:168-186.
void sinti(Sint& s, int n) {
    s.n = n;
    s.cc.assign((size_t)n + 2, 0.0);
    int ns2 = n / 2, np1 = n + 1;
    s.was.assign((size_t)ns2 + 1, 0.0);
    double dt = PI / (double)np1;
    for (int i = 1; i <= ns2; ++i) s.was[i] = 2.0 * std::sin((double)i * dt);
    rffti1(s.rfft, np1);
}

// radf2, qg3p_helmholtz.F90:1477-1519.  cc(ido,l1,2) -> ch(ido,2,l1).
// wa1 is a 1-based view (wa1[1] is the first element).
void radf2(int ido, int l1, const double* cc_, double* ch_, const double* wa1) {
    auto cc = [&](int i, int k, int m) -> double { return cc_[(i - 1) + ido * ((k - 1) + l1 * (m - 1))]; };
    auto ch = [&](int i, int m, int k) -> double& { return ch_[(i - 1) + ido * ((m - 1) + 2 * (k - 1))]; };
    for (int k = 1; k <= l1; ++k) {
        ch(1, 1, k) = cc(1, k, 1) + cc(1, k, 2);
        ch(ido, 2, k) = cc(1, k, 1) - cc(1, k, 2);
    }
    if (ido > 2) {
        int idp2 = ido + 2;
        for (int k = 1; k <= l1; ++k) {
            for (int i = 3; i <= ido; i += 2) {
                int ic = idp2 - i;
                double tr2 = wa1[i - 2] * cc(i - 1, k, 2) + wa1[i - 1] * cc(i, k, 2);
                double ti2 = wa1[i - 2] * cc(i, k, 2) - wa1[i - 1] * cc(i - 1, k, 2);
                ch(i, 1, k) = cc(i, k, 1) + ti2;
                ch(ic, 2, k) = ti2 - cc(i, k, 1);
                ch(i - 1, 1, k) = cc(i - 1, k, 1) + tr2;
                ch(ic - 1, 2, k) = cc(i - 1, k, 1) - tr2;
            }
        }
    }
    if (ido % 2 == 0) {
        for (int k = 1; k <= l1; ++k) {
            ch(1, 2, k) = -cc(ido, k, 2);
            ch(ido, 1, k) = cc(ido, k, 1);
        }
    }
}

// radf4, qg3p_helmholtz.F90:1521-1591.  cc(ido,l1,4) -> ch(ido,4,l1).
// wa1/wa2/wa3 are 1-based views (wa[1] is the first element).
void radf4(int ido, int l1, const double* cc_, double* ch_, const double* wa1, const double* wa2,
           const double* wa3) {
    auto cc = [&](int i, int k, int m) -> double { return cc_[(i - 1) + ido * ((k - 1) + l1 * (m - 1))]; };
    auto ch = [&](int i, int m, int k) -> double& { return ch_[(i - 1) + ido * ((m - 1) + 4 * (k - 1))]; };
    for (int k = 1; k <= l1; ++k) {
        double tr1 = cc(1, k, 2) + cc(1, k, 4);
        double tr2 = cc(1, k, 1) + cc(1, k, 3);
        ch(1, 1, k) = tr1 + tr2;
        ch(ido, 4, k) = tr2 - tr1;
        ch(ido, 2, k) = cc(1, k, 1) - cc(1, k, 3);
        ch(1, 3, k) = cc(1, k, 4) - cc(1, k, 2);
    }
    if (ido > 2) {
        int idp2 = ido + 2;
        for (int k = 1; k <= l1; ++k) {
            for (int i = 3; i <= ido; i += 2) {
                int ic = idp2 - i;
                double cr2 = wa1[i - 2] * cc(i - 1, k, 2) + wa1[i - 1] * cc(i, k, 2);
                double ci2 = wa1[i - 2] * cc(i, k, 2) - wa1[i - 1] * cc(i - 1, k, 2);
                double cr3 = wa2[i - 2] * cc(i - 1, k, 3) + wa2[i - 1] * cc(i, k, 3);
                double ci3 = wa2[i - 2] * cc(i, k, 3) - wa2[i - 1] * cc(i - 1, k, 3);
                double cr4 = wa3[i - 2] * cc(i - 1, k, 4) + wa3[i - 1] * cc(i, k, 4);
                double ci4 = wa3[i - 2] * cc(i, k, 4) - wa3[i - 1] * cc(i - 1, k, 4);
                double tr1 = cr2 + cr4;
                double tr4 = cr4 - cr2;
                double ti1 = ci2 + ci4;
                double ti4 = ci2 - ci4;
                double ti2 = cc(i, k, 1) + ci3;
                double ti3 = cc(i, k, 1) - ci3;
                double tr2 = cc(i - 1, k, 1) + cr3;
                double tr3 = cc(i - 1, k, 1) - cr3;
                ch(i - 1, 1, k) = tr1 + tr2;
                ch(ic - 1, 4, k) = tr2 - tr1;
                ch(i, 1, k) = ti1 + ti2;
                ch(ic, 4, k) = ti1 - ti2;
                ch(i - 1, 3, k) = ti4 + tr3;
                ch(ic - 1, 2, k) = tr3 - ti4;
                ch(i, 3, k) = tr4 + ti3;
                ch(ic, 2, k) = tr4 - ti3;
            }
        }
    }
    if (ido % 2 == 0) {
        for (int k = 1; k <= l1; ++k) {
            double ti1 = -HSQT2 * (cc(ido, k, 2) + cc(ido, k, 4));
            double tr1 = HSQT2 * (cc(ido, k, 2) - cc(ido, k, 4));
            ch(ido, 1, k) = tr1 + cc(ido, k, 1);
            ch(ido, 3, k) = cc(ido, k, 1) - tr1;
            ch(1, 2, k) = ti1 - cc(ido, k, 3);
            ch(1, 4, k) = ti1 + cc(ido, k, 3);
        }
    }
}

// rfftf1, qg3p_helmholtz.F90:1428-1475.  cc(1:n), ch(1:n) 0-based pointers.
// Returns 0 on success, -1 for an unsupported factor (the reference aborts).
int rfftf1(const Rfft& r, double* cc, double* ch) {
    int n = r.n, nf = r.nf;
    int l2 = n, iw = n;
    for (int i = 1; i <= nf; ++i) {
        int kh = nf - i;
        int ip = r.ifac[kh + 1];
        int l1 = l2 / ip;
        int ido = n / l2;
        iw = iw - (ip - 1) * ido;
        // wa is stored 1-based; v(k) below is a 1-based view starting at wa(k).
        const double* w = r.wa.data();
        auto v = [&](int k) { return w + k - 1; };
        if (ip == 4) {
            int ix2 = iw + ido;
            int ix3 = ix2 + ido;
            if (i % 2 == 1)
                radf4(ido, l1, cc, ch, v(iw), v(ix2), v(ix3));
            else
                radf4(ido, l1, ch, cc, v(iw), v(ix2), v(ix3));
        } else if (ip == 2) {
            if (i % 2 == 1)
                radf2(ido, l1, cc, ch, v(iw));
            else
                radf2(ido, l1, ch, cc, v(iw));
        } else {
            return -1;  // labort('Missing "radf"... subroutines')
        }
        l2 = l1;
    }
    if (nf % 2 == 0) return 0;
    for (int i = 0; i < n; ++i) cc[i] = ch[i];
    return 0;
}

// sint1, qg3p_helmholtz.F90:1380-1426.  x is 1-based x(1:n+1) passed as
// pointer to x(1).  Note the reference passes x itself as rfftf1's work array.
int sint1(Sint& s, double* x0) {
    double* x = x0 - 1;  // 1-based
    int n = s.n;
    if (n < 2) {
        x[1] = x[1] + x[1];
    } else if (n == 2) {
        double xhold = SQRT3 * (x[1] + x[2]);
        x[2] = SQRT3 * (x[1] - x[2]);
        x[1] = xhold;
    } else {
        int np1 = n + 1;
        int ns2 = n / 2;
        double* cc = s.cc.data();  // 1-based, size n+2
        cc[1] = 0.0;
        for (int k = 1; k <= ns2; ++k) {
            int kc = np1 - k;
            double t1 = x[k] - x[kc];
            double t2 = s.was[k] * (x[k] + x[kc]);
            cc[k + 1] = t1 + t2;
            cc[kc + 1] = t2 - t1;
        }
        int modn = n % 2;
        if (modn != 0) cc[ns2 + 2] = 4.0 * x[ns2 + 1];
        if (rfftf1(s.rfft, cc + 1, x + 1) != 0) return -1;
        x[1] = 0.5 * cc[1];
        for (int i = 3; i <= n; i += 2) {
            x[i] = x[i - 2] + cc[i - 1];
            x[i - 1] = -cc[i];
        }
        if (modn == 0) x[n] = -cc[n + 1];
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Stratification, qg3p_diagnostics.F90:125-450.
void strat_l2(double rd_bcl, double h1, double h2, double* s1, double* s2) {
    double fsq_over_nsq = (h1 * h2) / (2.0 * (rd_bcl * rd_bcl));
    *s1 = fsq_over_nsq * 2.0 / (h1 * (h1 + h2));
    *s2 = fsq_over_nsq * 2.0 / (h2 * (h1 + h2));
}

void strat_l3(double rd_bcl1, double rd_bcl2, double h1, double h2, double h3, double* s1, double* s21,
              double* s22, double* s3) {
    double lambda1 = -1.0 / (rd_bcl1 * rd_bcl1);
    double lambda2 = -1.0 / (rd_bcl2 * rd_bcl2);
    double b1 = -(lambda1 + lambda2);
    double c1 = lambda1 * lambda2;
    double h[4];
    h[0] = 2.0 / (h1 * (h1 + h2));
    h[1] = 2.0 / (h2 * (h1 + h2));
    h[2] = 2.0 / (h2 * (h2 + h3));
    h[3] = 2.0 / (h3 * (h2 + h3));
    double l = h[0] * h[2] + h[0] * h[3] + h[1] * h[3];
    double a2 = l * (h[2] + h[3]);
    double b2 = -b1 * l;
    double c2 = c1 * (h[0] + h[1]);
    double f2 = (-b2 - std::sqrt(b2 * b2 - 4.0 * a2 * c2)) / (2.0 * a2);
    double f1 = (b1 - f2 * (h[2] + h[3])) / (h[0] + h[1]);
    *s1 = f1 * h[0];
    *s21 = f1 * h[1];
    *s22 = f2 * h[2];
    *s3 = f2 * h[3];
}

// s_matrix, qg3p_diagnostics.F90:342-366.  Column-major L x L.
void s_matrix(int L, const double* s1, const double* s2, double* S) {
    for (int k = 0; k < L * L; ++k) S[k] = 0.0;
    auto A = [&](int i, int j) -> double& { return S[(i - 1) + L * (j - 1)]; };
    for (int i = 1; i <= L; ++i) {
        if (i > 1) {
            A(i, i - 1) = s1[i - 1];
            if (i < L) {
                A(i, i) = -(s1[i - 1] + s2[i - 1]);
                A(i, i + 1) = s2[i - 1];
            } else {
                A(i, i) = -s1[i - 1];
            }
        } else if (i < L) {
            A(i, i) = -s2[i - 1];
            A(i, i + 1) = s2[i - 1];
        }
    }
}

// Cyclic Jacobi eigenvalue method for a symmetric n x n matrix (Golub & Van
// Loan, Matrix Computations, section 8.5).  a is destroyed; v receives the
// orthonormal eigenvectors as columns.
void jacobi_symmetric(int n, double* a, double* w, double* v) {
    auto A = [&](int i, int j) -> double& { return a[i + n * j]; };
    auto Vv = [&](int i, int j) -> double& { return v[i + n * j]; };
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) Vv(i, j) = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += A(p, q) * A(p, q);
        if (off == 0.0) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                if (A(p, q) == 0.0) continue;
                double theta = (A(q, q) - A(p, p)) / (2.0 * A(p, q));
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0);
                double s = t * c;
                for (int k = 0; k < n; ++k) {
                    double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - s * akq;
                    A(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - s * aqk;
                    A(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = Vv(k, p), vkq = Vv(k, q);
                    Vv(k, p) = c * vkp - s * vkq;
                    Vv(k, q) = s * vkp + c * vkq;
                }
            }
        }
    }
    for (int i = 0; i < n; ++i) w[i] = A(i, i);
}

// Gaussian elimination with partial pivoting; inverse of a column-major n x n
// matrix (the result dgetrf + dgetri compute in exact arithmetic).
int inverse(int n, const double* a_in, double* ainv) {
    std::vector<double> a(a_in, a_in + (size_t)n * n);
    for (int i = 0; i < n * n; ++i) ainv[i] = 0.0;
    for (int i = 0; i < n; ++i) ainv[i + n * i] = 1.0;
    auto A = [&](int i, int j) -> double& { return a[i + (size_t)n * j]; };
    auto B = [&](int i, int j) -> double& { return ainv[i + (size_t)n * j]; };
    for (int k = 0; k < n; ++k) {
        int piv = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(A(i, k)) > std::fabs(A(piv, k))) piv = i;
        if (A(piv, k) == 0.0) return -1;
        if (piv != k)
            for (int j = 0; j < n; ++j) {
                std::swap(A(k, j), A(piv, j));
                std::swap(B(k, j), B(piv, j));
            }
        double d = A(k, k);
        for (int i = k + 1; i < n; ++i) {
            double f = A(i, k) / d;
            if (f == 0.0) continue;
            for (int j = k; j < n; ++j) A(i, j) -= f * A(k, j);
            for (int j = 0; j < n; ++j) B(i, j) -= f * B(k, j);
        }
    }
    for (int k = n - 1; k >= 0; --k) {
        for (int j = 0; j < n; ++j) {
            double s = B(k, j);
            for (int m = k + 1; m < n; ++m) s -= A(k, m) * B(m, j);
            B(k, j) = s / A(k, k);
        }
    }
    return 0;
}

// Eigen-decomposition of the (non-symmetric) real tridiagonal stratification
// matrix S by symmetrisation.  S(i,i+1)*S(i+1,i) > 0 for the layer model
// (s2(i)*s1(i+1) = (f0^2/g')^2/(H_i H_{i+1})), so T = D S D^-1 with
// D = diag(d), d(i+1)/d(i) = sqrt(S(i,i+1)/S(i+1,i)) is symmetric; the
// eigenvectors of S are D^-1 times those of T, normalised to unit 2-norm as
// dgeev (lapack_interfaces.F90:159-196) returns them.
int eigen_real_tridiag(int n, const double* S, double* w, double* vec) {
    auto A = [&](int i, int j) { return S[i + n * j]; };
    std::vector<double> d(n, 1.0), T((size_t)n * n, 0.0), Q((size_t)n * n);
    for (int i = 0; i + 1 < n; ++i) {
        double up = A(i, i + 1), lo = A(i + 1, i);
        if (!(up * lo > 0.0)) {
            if (up == 0.0 && lo == 0.0) {
                d[i + 1] = d[i];
                continue;
            }
            return -1;
        }
        d[i + 1] = d[i] * std::sqrt(up / lo);
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) T[i + n * j] = d[i] * A(i, j) / d[j];
    // Exact symmetry of the off-diagonals.
    for (int i = 0; i + 1 < n; ++i) {
        double s = std::sqrt(A(i, i + 1) * A(i + 1, i));
        T[i + n * (i + 1)] = s;
        T[(i + 1) + n * i] = s;
    }
    std::vector<double> w0(n);
    jacobi_symmetric(n, T.data(), w0.data(), Q.data());
    // Eigenvalues in ascending order: the order dgeev returns for the
    // stratification matrices pinned by unittest/test_eigendecompose.F90:72-86
    // and test_stratification.F90:41-44 (most negative first).
    std::vector<int> ord(n);
    for (int j = 0; j < n; ++j) ord[j] = j;
    for (int a = 1; a < n; ++a)
        for (int b = a; b > 0 && w0[ord[b]] < w0[ord[b - 1]]; --b) std::swap(ord[b], ord[b - 1]);
    for (int jo = 0; jo < n; ++jo) {
        int j = ord[jo];
        w[jo] = w0[j];
        double nrm = 0.0;
        for (int i = 0; i < n; ++i) {
            double x = Q[i + n * j] / d[i];
            vec[i + n * jo] = x;
            nrm += x * x;
        }
        nrm = std::sqrt(nrm);
        for (int i = 0; i < n; ++i) vec[i + n * jo] /= nrm;
    }
    return 0;
}

// s_conversion_matrices + sort_barotropic, qg3p_diagnostics.F90:372-422.
int s_conversion_matrices(int L, const double* S, double* m2z, double* z2m, double* ss) {
    if (eigen_real_tridiag(L, S, ss, m2z) != 0) return -1;
    for (int i = 0; i < L; ++i) ss[i] = -ss[i];
    auto M = [&](int i, int j) -> double& { return m2z[(i - 1) + L * (j - 1)]; };
    int bt = 1;
    double min_s = ss[0];
    for (int i = 2; i <= L; ++i)
        if (ss[i - 1] < min_s) {
            bt = i;
            min_s = ss[i - 1];
        }
    // ss(2:bt_index) = ss(:bt_index - 1); ss(1) = 0
    std::vector<double> ss0(ss, ss + L);
    for (int i = 2; i <= bt; ++i) ss[i - 1] = ss0[i - 2];
    ss[0] = 0.0;
    // Array assignments evaluate their right-hand sides first.
    std::vector<double> m0(m2z, m2z + L * L);
    auto M0 = [&](int i, int j) { return m0[(i - 1) + L * (j - 1)]; };
    double m11 = M0(1, 1);
    for (int j = 2; j <= bt; ++j)
        for (int i = 1; i <= L; ++i) M(i, j) = M0(i, j - 1) / m11;
    for (int j = bt + 1; j <= L; ++j)
        for (int i = 1; i <= L; ++i) M(i, j) = M0(i, j) / m11;
    for (int i = 1; i <= L; ++i) M(i, 1) = 1.0;
    return inverse(L, m2z, z2m);
}

// ---------------------------------------------------------------------------
// Helmholtz solver cache, qg3p_helmholtz.F90:292-386 (PH1D single process).
struct HelmCache {
    Decomp d;
    Sint sint;
    std::vector<double> ss;
    // PH1D ge_fact(ii, jj) per layer (qg3p_helmholtz.F90:794-809), non-periodic.
    std::vector<std::vector<double>> ge_fact;
    int max_j = 0;
    // Periodic channel: poinit_j eig + periodic_coefficients b, c (non-PH1D
    // path, :429-610), each (ii, jj) per layer.
    std::vector<std::vector<double>> eig, pb, pc;
};

}  // namespace

struct or_helm_cache {
    HelmCache c;
};

namespace {

void helm_init(HelmCache& c, const Decomp& d, const double* ss) {
    c.d = d;
    sinti(c.sint, d.g_ii2);
    c.ss.assign(ss, ss + d.layers);
    int ii = d.ii, jj = d.jj;
    if (!d.periodic_j) {
        // allocate_h1d_c, qg3p_helmholtz.F90:794-809 (max_j = jj - 1 when p_a < 0).
        c.max_j = jj - 1;
        c.ge_fact.assign(d.layers, std::vector<double>((size_t)ii * jj, 0.0));
        double norm_fact = PI / (2.0 * (double)(ii - 1));
        std::vector<double> diag((size_t)ii + 1, 0.0);
        for (int layer = 1; layer <= d.layers; ++layer) {
            V2 g{c.ge_fact[layer - 1].data(), ii, jj};
            for (int i = 2; i <= ii - 1; ++i) {
                double s = std::sin((double)(i - 1) * norm_fact);
                diag[i] = -2.0 - c.ss[layer - 1] - 4.0 * (s * s);
                g(i, 2) = diag[i];
            }
            for (int j = 3; j <= c.max_j; ++j)
                for (int i = 2; i <= ii - 1; ++i) g(i, j) = diag[i] - 1.0 / g(i, j - 1);
            for (int j = 2; j <= c.max_j; ++j)
                for (int i = 2; i <= ii - 1; ++i) g(i, j) = 1.0 / g(i, j);
        }
    } else {
        // poinit_j, :429-469 and periodic_coefficients, :473-559.
        c.eig.assign(d.layers, std::vector<double>((size_t)ii * jj, 0.0));
        c.pb.assign(d.layers, std::vector<double>((size_t)ii * jj, 0.0));
        c.pc.assign(d.layers, std::vector<double>((size_t)ii * jj, 0.0));
        double cff = PI / (2.0 * (double)d.g_ii_int);
        for (int layer = 1; layer <= d.layers; ++layer) {
            V2 e{c.eig[layer - 1].data(), ii, jj};
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) {
                double s = std::sin((double)(i - 1) * cff);
                double v = -2.0 - c.ss[layer - 1] - 4.0 * (s * s);
                for (int j = d.l_j_min; j <= d.l_j_max; ++j) e(i, j) = v;
            }
            for (int j = 3; j <= jj - 1; ++j)
                for (int i = d.l_i_min; i <= d.l_i_max; ++i) e(i, j) = e(i, j) - 1.0 / e(i, j - 1);
            for (int j = 2; j <= jj - 1; ++j)
                for (int i = d.l_i_min; i <= d.l_i_max; ++i) e(i, j) = 1.0 / e(i, j);
            V2 b{c.pb[layer - 1].data(), ii, jj};
            V2 cc{c.pc[layer - 1].data(), ii, jj};
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) {
                double s = std::sin((double)(i - 1) * cff);
                double a = -2.0 - c.ss[layer - 1] - 4.0 * (s * s);
                b(i, 1) = a;
                b(i, 2) = 1.0;
                for (int j = 3; j <= jj - 1; ++j) b(i, j) = 0.0;
                b(i, jj) = 1.0;
                cc(i, 1) = 1.0;
                for (int j = 2; j <= jj - 2; ++j) cc(i, j) = 0.0;
                cc(i, jj - 1) = 1.0;
                cc(i, jj) = a;
            }
            for (int j = 3; j <= jj - 1; ++j)
                for (int i = d.l_i_min; i <= d.l_i_max; ++i) {
                    b(i, j) = b(i, j) - b(i, j - 1) * e(i, j - 1);
                    cc(i, j) = cc(i, j) - cc(i, j - 1) * e(i, j - 1);
                }
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) {
                b(i, jj - 1) = b(i, jj - 1) * e(i, jj - 1);
                cc(i, jj - 1) = cc(i, jj - 1) * e(i, jj - 1);
            }
            for (int j = jj - 2; j >= 2; --j)
                for (int i = d.l_i_min; i <= d.l_i_max; ++i) {
                    b(i, j) = (b(i, j) - b(i, j + 1)) * e(i, j);
                    cc(i, j) = (cc(i, j) - cc(i, j + 1)) * e(i, j);
                }
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) {
                b(i, 1) = b(i, 1) - b(i, 2);
                cc(i, 1) = cc(i, 1) - cc(i, 2);
            }
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) {
                b(i, jj) = b(i, jj) - b(i, jj - 1);
                cc(i, jj) = cc(i, jj) - cc(i, jj - 1);
            }
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) cc(i, 1) = cc(i, 1) / b(i, 1);
            for (int j = 2; j <= jj; ++j)
                for (int i = d.l_i_min; i <= d.l_i_max; ++i) cc(i, j) = cc(i, j) - cc(i, 1) * b(i, j);
        }
    }
}

// helm, qg3p_helmholtz.F90:614-769, serial.  Non-periodic: PH1D path where
// h1d reduces to ge_local (:1028-1059).  Periodic: non-PH1D Thomas
// (:715-728) followed by periodic_ge (:565-610).
int helm(HelmCache& c, double* zeta_p) {
    const Decomp& d = c.d;
    int ii = d.ii, jj = d.jj;
    V3 z{zeta_p, ii, jj, d.layers};
    double cff = 0.5 / (double)d.g_ii_int;
    for (int layer = 1; layer <= d.layers; ++layer) {
        for (int j = d.l_j_min; j <= d.l_j_max; ++j) {
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) z(i, j, layer) = cff * z(i, j, layer);
            if (sint1(c.sint, &z(d.l_i_min, j, layer)) != 0) return -1;
        }
        if (!d.periodic_j) {
            V2 g{c.ge_fact[layer - 1].data(), ii, jj};
            int max_j = c.max_j;
            for (int j = 3; j <= max_j; ++j)
                for (int i = 2; i <= ii - 1; ++i) z(i, j, layer) = z(i, j, layer) - z(i, j - 1, layer) * g(i, j - 1);
            for (int i = 2; i <= ii - 1; ++i) z(i, max_j, layer) = z(i, max_j, layer) * g(i, max_j);
            for (int j = max_j - 1; j >= 2; --j)
                for (int i = 2; i <= ii - 1; ++i) z(i, j, layer) = (z(i, j, layer) - z(i, j + 1, layer)) * g(i, j);
            for (int i = 2; i <= ii - 1; ++i) z(i, 1, layer) = 0.0;
        } else {
            V2 e{c.eig[layer - 1].data(), ii, jj};
            for (int j = 3; j <= jj - 1; ++j)
                for (int i = d.l_i_min; i <= d.l_i_max; ++i)
                    z(i, j, layer) = z(i, j, layer) - z(i, j - 1, layer) * e(i, j - 1);
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) z(i, jj - 1, layer) = z(i, jj - 1, layer) * e(i, jj - 1);
            for (int j = jj - 2; j >= 2; --j)
                for (int i = d.l_i_min; i <= d.l_i_max; ++i)
                    z(i, j, layer) = (z(i, j, layer) - z(i, j + 1, layer)) * e(i, j);
            // periodic_ge
            V2 b{c.pb[layer - 1].data(), ii, jj};
            V2 cc{c.pc[layer - 1].data(), ii, jj};
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) z(i, 1, layer) = z(i, 1, layer) - z(i, 2, layer);
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) z(i, jj, layer) = z(i, jj, layer) - z(i, jj - 1, layer);
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) z(i, 1, layer) = z(i, 1, layer) / b(i, 1);
            for (int j = 2; j <= jj; ++j)
                for (int i = d.l_i_min; i <= d.l_i_max; ++i) z(i, j, layer) = z(i, j, layer) - z(i, 1, layer) * b(i, j);
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) z(i, jj, layer) = z(i, jj, layer) / cc(i, jj);
            for (int j = jj - 1; j >= 1; --j)
                for (int i = d.l_i_min; i <= d.l_i_max; ++i) z(i, j, layer) = z(i, j, layer) - z(i, jj, layer) * cc(i, j);
        }
        for (int j = d.l_j_min; j <= d.l_j_max; ++j) {
            if (sint1(c.sint, &z(d.l_i_min, j, layer)) != 0) return -1;
            z(d.ii, j, layer) = 0.0;
        }
    }
    return 0;
}

// ---------------------------------------------------------------------------
// qg3p_laplace_bc.F90:55-86 (closed) and :128-150 (periodic).
void add_laplace_bc_rhs_layer(const Decomp& d, double bc, double bc_d, double* rhs_p) {
    V2 rhs{rhs_p, d.ii, d.jj};
    if (!d.periodic_j) {
        if (d.p_a == -1)
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) rhs(i, d.l_j_max) -= bc;
        if (d.p_c == -1)
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) rhs(i, d.l_j_min) -= bc;
        if (d.p_b == -1)
            for (int j = d.l_j_min; j <= d.l_j_max; ++j) rhs(d.l_i_min, j) -= bc;
        if (d.p_d == -1)
            for (int j = d.l_j_min; j <= d.l_j_max; ++j) rhs(d.l_i_max, j) -= bc;
    } else {
        if (d.p_b == -1)
            for (int j = d.l_j_min; j <= d.l_j_max; ++j) rhs(d.l_i_min, j) -= bc;
        if (d.p_d == -1)
            for (int j = d.l_j_min; j <= d.l_j_max; ++j) rhs(d.l_i_max, j) -= bc_d;
    }
}

// qg3p_laplace_bc.F90:193-224 (closed) and :227-251 (periodic).
void apply_dirichlet_bc_layer(const Decomp& d, double bc, double bc_d, double* z_p) {
    V2 z{z_p, d.ii, d.jj};
    if (!d.periodic_j) {
        if (d.p_a == -1)
            for (int i = 1; i <= d.ii; ++i) z(i, d.jj) = bc;
        if (d.p_c == -1)
            for (int i = 1; i <= d.ii; ++i) z(i, 1) = bc;
        if (d.p_b == -1)
            for (int j = 1; j <= d.jj; ++j) z(1, j) = bc;
        if (d.p_d == -1)
            for (int j = 1; j <= d.jj; ++j) z(d.ii, j) = bc;
    } else {
        if (d.p_b == -1)
            for (int j = 1; j <= d.jj; ++j) z(1, j) = bc;
        if (d.p_d == -1)
            for (int j = 1; j <= d.jj; ++j) z(d.ii, j) = bc_d;
    }
}

void apply_dirichlet_bc(const Decomp& d, double bc, double* z) {
    for (int l = 0; l < d.layers; ++l) apply_dirichlet_bc_layer(d, bc, bc, z + (size_t)l * d.ii * d.jj);
}

// local_integral, qg3p_diagnostics.F90:669-720.  Fortran sum() over an array
// section accumulates in array-element order.
double local_integral(const Decomp& d, const double* psi_p) {
    V2 psi{const_cast<double*>(psi_p), d.ii, d.jj};
    double integral = 0.0;
    for (int j = d.l_j_min; j <= d.l_j_max; ++j)
        for (int i = d.l_i_min; i <= d.l_i_max; ++i) integral += psi(i, j);
    if (d.p_b == -1) {
        double s = 0.0;
        for (int j = d.l_j_min; j <= d.l_j_max; ++j) s += psi(1, j);
        integral = integral + 0.5 * s;
        if (d.p_c == -1) integral = integral + 0.25 * psi(1, 1);
        if (d.p_a == -1) integral = integral + 0.25 * psi(1, d.jj);
    }
    if (d.p_d == -1) {
        double s = 0.0;
        for (int j = d.l_j_min; j <= d.l_j_max; ++j) s += psi(d.ii, j);
        integral = integral + 0.5 * s;
        if (d.p_c == -1) integral = integral + 0.25 * psi(d.ii, 1);
        if (d.p_a == -1) integral = integral + 0.25 * psi(d.ii, d.jj);
    }
    if (d.p_c == -1) {
        double s = 0.0;
        for (int i = d.l_i_min; i <= d.l_i_max; ++i) s += psi(i, 1);
        integral = integral + 0.5 * s;
    }
    if (d.p_a == -1) {
        double s = 0.0;
        for (int i = d.l_i_min; i <= d.l_i_max; ++i) s += psi(i, d.jj);
        integral = integral + 0.5 * s;
    }
    return integral;
}

double mean_layer(const Decomp& d, const double* psi) {
    return local_integral(d, psi) / (double)(d.g_ii_int * d.g_jj_int);
}

// energy, qg3p_diagnostics.F90:778-863.  psi is a full data array.
int energy(const Decomp& d, const double* h, const double* s2, const double* psi_p, double* ekin,
           double* epot_out) {
    int L = d.layers;
    V3 data{const_cast<double*>(psi_p), d.ii + 2, d.jj + 2, L};
    auto sd = [&](int i, int j, int k) -> double { return data(i + 1, j + 1, k); };
    double h_total = 0.0;
    for (int k = 0; k < L; ++k) h_total += h[k];
    std::vector<double> fac(L > 1 ? L - 1 : 1);
    for (int i = 1; i <= L - 1; ++i) fac[i - 1] = 0.5 * s2[i - 1] * h[i - 1] / h_total;
    double epot = 0.0;
    auto sq = [](double x) { return x * x; };
    for (int k = 1; k <= L - 1; ++k) {
        double f = fac[k - 1];
        for (int j = d.l_j_min; j <= d.l_j_max; ++j)
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) epot = epot + f * sq(sd(i, j, k) - sd(i, j, k + 1));
        if (d.p_c == -1) {
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) epot = epot + 0.5 * f * sq(sd(i, 1, k) - sd(i, 1, k + 1));
            if (d.p_b == -1) epot = epot + 0.25 * f * sq(sd(1, 1, k) - sd(1, 1, k + 1));
            if (d.p_d == -1) epot = epot + 0.25 * f * sq(sd(d.ii, 1, k) - sd(d.ii, 1, k + 1));
        }
        if (d.p_a == -1) {
            for (int i = d.l_i_min; i <= d.l_i_max; ++i)
                epot = epot + 0.5 * f * sq(sd(i, d.jj, k) - sd(i, d.jj, k + 1));
            if (d.p_b == -1) epot = epot + 0.25 * f * sq(sd(1, d.jj, k) - sd(1, d.jj, k + 1));
            if (d.p_d == -1) epot = epot + 0.25 * f * sq(sd(d.ii, d.jj, k) - sd(d.ii, d.jj, k + 1));
        }
        if (d.p_b == -1)
            for (int j = d.l_j_min; j <= d.l_j_max; ++j) epot = epot + 0.5 * f * sq(sd(1, j, k) - sd(1, j, k + 1));
        if (d.p_d == -1)
            for (int j = d.l_j_min; j <= d.l_j_max; ++j)
                epot = epot + 0.5 * f * sq(sd(d.ii, j, k) - sd(d.ii, j, k + 1));
    }
    for (int k = 1; k <= L; ++k) {
        double e = 0.0;
        for (int j = d.f_j_min; j <= d.fb_j_max; ++j)
            for (int i = d.f_i_min; i <= d.fb_i_max; ++i)
                e = e + 0.25 * (sq(data(i - 1, j, k) + data(i, j, k) - data(i - 1, j - 1, k) - data(i, j - 1, k)) +
                                sq(data(i, j - 1, k) + data(i, j, k) - data(i - 1, j - 1, k) - data(i - 1, j, k)));
        ekin[k - 1] = e;
    }
    double cff = 1.0 / (double)(d.g_ii_int * d.g_jj_int);
    epot = cff * epot;
    for (int k = 0; k < L; ++k) ekin[k] = 0.5 * cff * (h[k] / h_total) * ekin[k];
    *epot_out = epot;
    if (epot != epot) return -1;
    for (int k = 0; k < L; ++k)
        if (ekin[k] != ekin[k]) return -1;
    return 0;
}

}  // namespace

// ===========================================================================
// The model: state in reference layouts and the routines of qg3p_aux.F90.
struct or_model {
    Decomp d;
    or_params p;
    std::vector<double> beta, h, s1, s2, ss, m2z, z2m, wind;
    HelmCache hc;
    std::vector<double> corr;  // (ii, jj, L, 1) correction_function_mass; (ii, jj, L, 2) channel
    std::vector<double> inv_corr_a;  // channel: (2, 2, L - 1), correction_function_momentum
    std::vector<double> phi;   // working memory (ii, jj, L)
    // Prognostic fields, full data arrays (ii+2, jj+2, L); [1] is leapfrog level 2.
    std::vector<double> psi[2], rel[2], zeta[2], zeta_old[2];
    // CABARET
    std::vector<double> zeta_fi, zeta_fj, ui, uj, uimo, ujmo, flux_i, flux_j;
    std::vector<double> res, res_beta;  // (ii, jj, L) sized as ii_m x jj_m x layers
    double dt = 0, tweight_a = 0.5, tweight_u = 0.5, model_time = 0;
    int lf_count = 0;  // leapfrog sub-steps taken since initialisation
    // Time average (qg3.F90:93, 502-503, 672-680, 725): sum of dt * psi sdata.
    std::vector<double> psi_av;  // (ii, jj, L)
    double diag_time = 0, av_threshold = 0;
    bool av_on = false;
    // quad eddy covariances (qg3.F90:505-558, 683-721), in output order:
    // uu vv uu_i vv_i uv ur vr rr pr uz vz zz zr pp pz ut vt rt tt sc_ub
    // sc_vb sc_bb sc_bb_i; *_i and sc_ub, sc_vb, sc_bb_i have L - 1 layers.
    bool quad_on = false;
    std::vector<double> quad[23];
    std::vector<double> p_beta_y;  // (ii+2, L)
    // Scratch arrays the reference keeps as module-level `save` arrays.
    std::vector<double> psi_edge, zeta_fin, zeta_fjn, res_visc;

    size_t nfull() const { return (size_t)(d.ii + 2) * (d.jj + 2) * d.layers; }
    size_t nfi() const { return (size_t)(d.ii + 3) * (d.jj + 2) * d.layers; }
    size_t nfj() const { return (size_t)(d.ii + 2) * (d.jj + 3) * d.layers; }
    size_t nsd() const { return (size_t)d.ii * d.jj * d.layers; }
    V3 full(std::vector<double>& v) { return V3{v.data(), d.ii + 2, d.jj + 2, d.layers}; }
    V3 fi(std::vector<double>& v) { return V3{v.data(), d.ii + 3, d.jj + 2, d.layers}; }
    V3 fj(std::vector<double>& v) { return V3{v.data(), d.ii + 2, d.jj + 3, d.layers}; }
    V3 sdv(std::vector<double>& v) { return V3{v.data(), d.ii, d.jj, d.layers}; }
};

namespace {

double S1(const or_model& m, int l) { return m.s1[l - 1]; }
double S2(const or_model& m, int l) { return m.s2[l - 1]; }

// z_to_modes_rank2, qg3p_diagnostics.F90:534-553 (dot_product order).
void z_to_modes(const or_model& m, const double* z, double* modes) {
    int L = m.d.layers;
    size_t n = (size_t)m.d.ii * m.d.jj;
    for (size_t p = 0; p < n; ++p)
        for (int layer = 1; layer <= L; ++layer) {
            double s = 0.0;
            for (int l = 1; l <= L; ++l) s += m.z2m[(layer - 1) + L * (l - 1)] * z[p + n * (l - 1)];
            modes[p + n * (layer - 1)] = s;
        }
}

// correction_function_mass, qg3p_aux.F90:196-230.
void correction_function_mass(or_model& m) {
    const Decomp& d = m.d;
    int L = d.layers;
    m.corr.assign(m.nsd(), 1.0);
    helm(m.hc, m.corr.data());
    apply_dirichlet_bc(d, 0.0, m.corr.data());
    V3 c = m.sdv(m.corr);
    std::vector<double> mean_corr(L);
    for (int layer = 1; layer <= L; ++layer) {
        double s = 0.0;
        for (int j = d.l_j_min; j <= d.l_j_max; ++j)
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) s += c(i, j, layer);
        mean_corr[layer - 1] = s / (double)(d.g_ii_int * d.g_jj_int);
    }
    for (int layer = 1; layer <= L; ++layer) {
        double ssl = m.ss[layer - 1];
        double den = 1.0 + ssl * mean_corr[layer - 1];
        for (int j = 1; j <= d.jj; ++j)
            for (int i = 1; i <= d.ii; ++i) c(i, j, layer) = (1.0 + ssl * c(i, j, layer)) / den;
    }
}

// update_pdata (qg3p_base.F90:1887-1956) for one rank: only a channel
// (periodic j) has a halo to fill, its own first / last sdata row: halo row
// 1 <- row jj+1, halo row jj+2 <- row 2, columns 2..ii+1.
void update_pdata(or_model& m, std::vector<double>& v) {
    const Decomp& d = m.d;
    if (!d.periodic_j) return;
    V3 a = m.full(v);
    for (int l = 1; l <= d.layers; ++l)
        for (int i = 2; i <= d.ii + 1; ++i) {
            a(i, 1, l) = a(i, d.jj + 1, l);
            a(i, d.jj + 2, l) = a(i, 2, l);
        }
}

// update_flux_j (qg3p_base.F90:2964-3003) for one rank of a channel: faces
// fa_j_min <- fa_j_max - 1 and fa_j_max + 1 <- fa_j_min + 2, and with
// level_1 also fa_j_max <- fa_j_min + 1, over columns fa_i_min+1 ..
// fa_i_min+ii2.  update_flux_i has nothing to do on one rank.
void update_flux_j(or_model& m, std::vector<double>& v, bool level_1) {
    const Decomp& d = m.d;
    if (!d.periodic_j) return;
    V3 a = m.fj(v);
    for (int l = 1; l <= d.layers; ++l)
        for (int i = d.fa_i_min + 1; i <= d.fa_i_min + d.ii2; ++i) {
            a(i, d.fa_j_min, l) = a(i, d.fa_j_max - 1, l);
            a(i, d.fa_j_max + 1, l) = a(i, d.fa_j_min + 2, l);
            if (level_1) a(i, d.fa_j_max, l) = a(i, d.fa_j_min + 1, l);
        }
}

// zeta_boundary, qg3p_aux.F90:289-379: the mean relative PV of the modal
// field psi (sdata (ii, jj, L)) along the two walls i = 1 (z_b) and i = ii
// (z_d) of a channel: the wall relative vorticity of the velocity boundary
// condition and the thickness term -ss psi.
void zeta_boundary(const or_model& m, const double* psi_p, double* z_b, double* z_d) {
    const Decomp& d = m.d;
    const int L = d.layers, ii = d.ii;
    V3 psi{const_cast<double*>(psi_p), d.ii, d.jj, L};
    for (int l = 0; l < L; ++l) z_b[l] = z_d[l] = 0.0;
    switch (m.p.bc_type) {
        case OR_BC_PARTIAL_SLIP: {
            const double cff = m.p.alpha / (m.p.alpha + 3.0);
            if (d.p_b == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.l_j_min; j <= d.l_j_max; ++j)
                        z_b[l - 1] = z_b[l - 1] + cff * (-3.5 * psi(1, j, l) + 4.0 * psi(2, j, l) - 0.5 * psi(3, j, l));
            if (d.p_d == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.l_j_min; j <= d.l_j_max; ++j)
                        z_d[l - 1] = z_d[l - 1] +
                                     cff * (-3.5 * psi(ii, j, l) + 4.0 * psi(ii - 1, j, l) - 0.5 * psi(ii - 2, j, l));
            break;
        }
        case OR_BC_NO_SLIP: {
            if (d.p_b == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.l_j_min; j <= d.l_j_max; ++j)
                        z_b[l - 1] = z_b[l - 1] + 2.0 * (psi(2, j, l) - psi(1, j, l));
            if (d.p_d == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.l_j_min; j <= d.l_j_max; ++j)
                        z_d[l - 1] = z_d[l - 1] + 2.0 * (psi(ii - 1, j, l) - psi(ii, j, l));
            break;
        }
        default:  // free slip: no vorticity term
            break;
    }
    if (d.p_b == -1)
        for (int l = 1; l <= L; ++l)
            for (int j = d.l_j_min; j <= d.l_j_max; ++j) z_b[l - 1] = z_b[l - 1] - m.ss[l - 1] * psi(1, j, l);
    if (d.p_d == -1)
        for (int l = 1; l <= L; ++l)
            for (int j = d.l_j_min; j <= d.l_j_max; ++j) z_d[l - 1] = z_d[l - 1] - m.ss[l - 1] * psi(ii, j, l);
    for (int l = 0; l < L; ++l) {
        z_b[l] = z_b[l] / (double)d.g_jj_int;
        z_d[l] = z_d[l] / (double)d.g_jj_int;
    }
}

// correction_function_momentum, qg3p_aux.F90:233-285: the two channel
// correction functions (homogeneous Helmholtz solutions with psi = 1 on one
// wall and 0 on the other) and, per baroclinic mode, the inverse of the 2 x 2
// matrix of their wall PV means.
void correction_function_momentum(or_model& m) {
    const Decomp& d = m.d;
    const int L = d.layers;
    const size_t n = m.nsd();
    m.corr.assign(2 * n, 0.0);
    for (int w = 0; w < 2; ++w) {
        double* c = m.corr.data() + (size_t)w * n;
        const double bb = w == 0 ? 1.0 : 0.0, bd = w == 0 ? 0.0 : 1.0;
        for (int l = 0; l < L; ++l) add_laplace_bc_rhs_layer(d, bb, bd, c + (size_t)l * d.ii * d.jj);
        helm(m.hc, c);
        for (int l = 0; l < L; ++l) apply_dirichlet_bc_layer(d, bb, bd, c + (size_t)l * d.ii * d.jj);
    }
    std::vector<double> zb1(L), zd1(L), zb2(L), zd2(L);
    zeta_boundary(m, m.corr.data(), zb1.data(), zd1.data());
    zeta_boundary(m, m.corr.data() + n, zb2.data(), zd2.data());
    m.inv_corr_a.assign((size_t)4 * (L > 1 ? L - 1 : 1), 0.0);
    for (int mode = 2; mode <= L; ++mode) {
        // z_b(mode, :, :): rows (z_b, z_d), columns (corr 1, corr 2), column-major
        const double a[4] = {zb1[mode - 1], zd1[mode - 1], zb2[mode - 1], zd2[mode - 1]};
        inverse(2, a, m.inv_corr_a.data() + (size_t)4 * (mode - 2));
    }
}

// pv_inversion + modes_to_z_correct_mass + modes_to_z_btcu,
// qg3p_aux.F90:452-521 and qg3p_diagnostics.F90:615-635.  zeta/psi are full
// data arrays; only their sdata parts are read / written.
int pv_inversion(or_model& m, std::vector<double>& zeta, std::vector<double>& psi) {
    const Decomp& d = m.d;
    int L = d.layers, ii = d.ii, jj = d.jj;
    V3 zf = m.full(zeta), pf = m.full(psi);
    std::vector<double> zs(m.nsd());
    V3 z = m.sdv(zs);
    for (int l = 1; l <= L; ++l)
        for (int j = 1; j <= jj; ++j)
            for (int i = 1; i <= ii; ++i) z(i, j, l) = zf(i + 1, j + 1, l);
    m.phi.assign(m.nsd(), 0.0);
    z_to_modes(m, zs.data(), m.phi.data());
    if (helm(m.hc, m.phi.data()) != 0) return -3;
    apply_dirichlet_bc(d, 0.0, m.phi.data());
    if (d.periodic_j) {
        // modes_to_z_correct_momentum, qg3p_aux.F90:524-575, then modes_to_z
        // (qg3p_diagnostics.F90:570-612).
        std::vector<double> cb(L), cd(L);
        zeta_boundary(m, m.phi.data(), cb.data(), cd.data());
        V3 ph = m.sdv(m.phi);
        const size_t n = m.nsd();
        V3 c1{m.corr.data(), ii, jj, L}, c2{m.corr.data() + n, ii, jj, L};
        for (int layer = 2; layer <= L; ++layer) {
            const double* A = m.inv_corr_a.data() + (size_t)4 * (layer - 2);
            const double p1 = A[0] * cb[layer - 1] + A[2] * cd[layer - 1];
            const double p2 = A[1] * cb[layer - 1] + A[3] * cd[layer - 1];
            if (p1 != p1 || p2 != p2) return -2;  // labort("NaN psiC encountered")
            for (int j = 1; j <= jj; ++j)
                for (int i = 1; i <= ii; ++i)
                    ph(i, j, layer) = ph(i, j, layer) - p1 * c1(i, j, layer) - p2 * c2(i, j, layer);
        }
        for (int j = 1; j <= jj; ++j)
            for (int i = 1; i <= ii; ++i)
                for (int layer = 1; layer <= L; ++layer) {
                    double s = 0.0;
                    for (int mm = 1; mm <= L; ++mm) s += m.m2z[(layer - 1) + L * (mm - 1)] * ph(i, j, mm);
                    pf(i + 1, j + 1, layer) = s;
                }
        return 0;
    }
    std::vector<double> psiC(L);
    for (int l = 1; l <= L; ++l) psiC[l - 1] = mean_layer(d, m.phi.data() + (size_t)(l - 1) * ii * jj);
    for (int l = 0; l < L; ++l)
        if (psiC[l] != psiC[l]) return -2;  // labort("NaN psiC encountered")
    V3 ph = m.sdv(m.phi), c = m.sdv(m.corr);
    for (int j = 1; j <= jj; ++j)
        for (int i = 1; i <= ii; ++i)
            for (int layer = 1; layer <= L; ++layer) {
                double dot = 0.0;
                for (int mm = 2; mm <= L; ++mm)
                    dot += m.m2z[(layer - 1) + L * (mm - 1)] * (ph(i, j, mm) - psiC[mm - 1] * c(i, j, mm));
                pf(i + 1, j + 1, layer) = ph(i, j, 1) - psiC[0] + dot;
            }
    return 0;
}

// apply_rel_bc, qg3p_aux.F90:779-915.
void apply_rel_bc(or_model& m, std::vector<double>& psi_v, std::vector<double>& rel_v) {
    const Decomp& d = m.d;
    V3 psi = m.full(psi_v), rel = m.full(rel_v);
    int L = d.layers, ii = d.ii, jj = d.jj;
    switch (m.p.bc_type) {
        case OR_BC_PARTIAL_SLIP: {
            double cff = m.p.alpha / (m.p.alpha + 3.0);
            if (d.p_b == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.fa_j_min; j <= d.fa_j_max; ++j)
                        rel(2, j, l) = cff * (-3.5 * psi(2, j, l) + 4.0 * psi(3, j, l) - 0.5 * psi(4, j, l));
            if (d.p_d == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.fa_j_min; j <= d.fa_j_max; ++j)
                        rel(ii + 1, j, l) = cff * (-3.5 * psi(ii + 1, j, l) + 4.0 * psi(ii, j, l) - 0.5 * psi(ii - 1, j, l));
            if (d.p_c == -1)
                for (int l = 1; l <= L; ++l)
                    for (int i = d.fa_i_min; i <= d.fa_i_max; ++i)
                        rel(i, 2, l) = cff * (-3.5 * psi(i, 2, l) + 4.0 * psi(i, 3, l) - 0.5 * psi(i, 4, l));
            if (d.p_a == -1)
                for (int l = 1; l <= L; ++l)
                    for (int i = d.fa_i_min; i <= d.fa_i_max; ++i)
                        rel(i, jj + 1, l) = cff * (-3.5 * psi(i, jj + 1, l) + 4.0 * psi(i, jj, l) - 0.5 * psi(i, jj - 1, l));
            break;
        }
        case OR_BC_NO_SLIP: {
            if (d.p_b == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.fa_j_min; j <= d.fa_j_max; ++j) rel(2, j, l) = 2.0 * (psi(3, j, l) - psi(2, j, l));
            if (d.p_d == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.fa_j_min; j <= d.fa_j_max; ++j)
                        rel(ii + 1, j, l) = 2.0 * (psi(ii, j, l) - psi(ii + 1, j, l));
            if (d.p_c == -1)
                for (int l = 1; l <= L; ++l)
                    for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) rel(i, 2, l) = 2.0 * (psi(i, 3, l) - psi(i, 2, l));
            if (d.p_a == -1)
                for (int l = 1; l <= L; ++l)
                    for (int i = d.fa_i_min; i <= d.fa_i_max; ++i)
                        rel(i, jj + 1, l) = 2.0 * (psi(i, jj, l) - psi(i, jj + 1, l));
            break;
        }
        default: {  // OR_BC_FREE_SLIP
            if (d.p_b == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.fa_j_min; j <= d.fa_j_max; ++j) rel(2, j, l) = 0.0;
            if (d.p_d == -1)
                for (int l = 1; l <= L; ++l)
                    for (int j = d.fa_j_min; j <= d.fa_j_max; ++j) rel(ii + 1, j, l) = 0.0;
            if (d.p_c == -1)
                for (int l = 1; l <= L; ++l)
                    for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) rel(i, 2, l) = 0.0;
            if (d.p_a == -1)
                for (int l = 1; l <= L; ++l)
                    for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) rel(i, jj + 1, l) = 0.0;
        }
    }
}

// rel_from_psi, qg3p_aux.F90:579-603: the five-point Laplacian of psi on
// the interior nodes, then apply_rel_bc on the boundary.
void rel_from_psi(or_model& m, std::vector<double>& psi_v, std::vector<double>& rel_v) {
    const Decomp& d = m.d;
    V3 psi = m.full(psi_v), rel = m.full(rel_v);
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i)
                rel(i, j, l) = -4.0 * psi(i, j, l) + psi(i - 1, j, l) + psi(i, j + 1, l) + psi(i + 1, j, l) +
                               psi(i, j - 1, l);
    apply_rel_bc(m, psi_v, rel_v);
}

// rel_from_zeta_and_psi, qg3p_aux.F90:738-775.
void rel_from_zeta_and_psi(or_model& m, std::vector<double>& zeta_v, std::vector<double>& psi_v,
                           std::vector<double>& rel_v) {
    const Decomp& d = m.d;
    int L = d.layers;
    V3 zeta = m.full(zeta_v), psi = m.full(psi_v), rel = m.full(rel_v);
    if (L == 1) {
        rel_v = zeta_v;
    } else {
        for (int j = d.fa_j_min; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min; i <= d.fa_i_max; ++i)
                rel(i, j, 1) = zeta(i, j, 1) + S2(m, 1) * (psi(i, j, 1) - psi(i, j, 2));
        for (int l = 2; l <= L - 1; ++l)
            for (int j = d.fa_j_min; j <= d.fa_j_max; ++j)
                for (int i = d.fa_i_min; i <= d.fa_i_max; ++i)
                    rel(i, j, l) = zeta(i, j, l) + S1(m, l) * (psi(i, j, l) - psi(i, j, l - 1)) +
                                   S2(m, l) * (psi(i, j, l) - psi(i, j, l + 1));
        for (int j = d.fa_j_min; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min; i <= d.fa_i_max; ++i)
                rel(i, j, L) = zeta(i, j, L) + S1(m, L) * (psi(i, j, L) - psi(i, j, L - 1));
    }
    apply_rel_bc(m, psi_v, rel_v);
}

// update_zeta_bc, qg3p_aux.F90:643-734.
void update_zeta_bc(or_model& m, std::vector<double>& rel_v, std::vector<double>& psi_v,
                    std::vector<double>& zeta_v) {
    const Decomp& d = m.d;
    int L = d.layers, ii = d.ii, jj = d.jj;
    V3 zeta = m.full(zeta_v), psi = m.full(psi_v), rel = m.full(rel_v);
    auto pv = [&](int i, int j) {
        zeta(i, j, 1) = rel(i, j, 1) - S2(m, 1) * (psi(i, j, 1) - psi(i, j, 2));
        zeta(i, j, L) = rel(i, j, L) - S1(m, L) * (psi(i, j, L) - psi(i, j, L - 1));
    };
    auto pvmid = [&](int i, int j, int l) {
        zeta(i, j, l) = rel(i, j, l) - S1(m, l) * (psi(i, j, l) - psi(i, j, l - 1)) -
                        S2(m, l) * (psi(i, j, l) - psi(i, j, l + 1));
    };
    if (L == 1) {
        if (d.p_c == -1)
            for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) zeta(i, 2, 1) = rel(i, 2, 1);
        if (d.p_a == -1)
            for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) zeta(i, jj + 1, 1) = rel(i, jj + 1, 1);
        if (d.p_b == -1)
            for (int j = d.fa_j_min; j <= d.fa_j_max; ++j) zeta(2, j, 1) = rel(2, j, 1);
        if (d.p_d == -1)
            for (int j = d.fa_j_min; j <= d.fa_j_max; ++j) zeta(ii + 1, j, 1) = rel(ii + 1, j, 1);
        return;
    }
    if (d.p_c == -1) {
        for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) pv(i, 2);
        for (int l = 2; l <= L - 1; ++l)
            for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) pvmid(i, 2, l);
    }
    if (d.p_a == -1) {
        for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) pv(i, jj + 1);
        for (int l = 2; l <= L - 1; ++l)
            for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) pvmid(i, jj + 1, l);
    }
    if (d.p_b == -1) {
        for (int j = d.fa_j_min; j <= d.fa_j_max; ++j) pv(2, j);
        for (int l = 2; l <= L - 1; ++l)
            for (int j = d.fa_j_min; j <= d.fa_j_max; ++j) pvmid(2, j, l);
    }
    if (d.p_d == -1) {
        for (int j = d.fa_j_min; j <= d.fa_j_max; ++j) pv(ii + 1, j);
        for (int l = 2; l <= L - 1; ++l)
            for (int j = d.fa_j_min; j <= d.fa_j_max; ++j) pvmid(ii + 1, j, l);
    }
}

double maxabs_u(or_model& m) {
    const Decomp& d = m.d;
    V3 ui = m.fi(m.ui), uj = m.fj(m.uj);
    double a = 0.0, b = 0.0;
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max - 1; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max; ++i) a = std::fmax(a, std::fabs(ui(i, j, l)));
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max - 1; ++i) b = std::fmax(b, std::fabs(uj(i, j, l)));
    return std::fmax(a, b);
}

// cabaret_adapt_dt, qg3p_aux.F90:946-990.  fne(max_u, 0) with the test_tools
// tolerance 10*max(spacing(max_u), epsilon).
void cabaret_adapt_dt(or_model& m) {
    double max_u = maxabs_u(m);
    double old_dt = m.dt;
    double tol = 10.0 * std::fmax(std::nextafter(std::fabs(max_u), INFINITY) - std::fabs(max_u),
                                  2.220446049250313e-16);
    if (std::fabs(max_u - 0.0) > tol) {
        double dt = m.p.target_cfl / max_u;
        dt = std::fmin(std::fmin(dt, old_dt * m.p.max_dt_increase), m.p.max_dt);
        m.dt = dt;
    }
    m.tweight_a = 0.5 * m.dt / old_dt;
    m.tweight_u = m.dt / (old_dt + m.dt);
}

// cabaret_predictor, qg3p_aux.F90:993-1020.
void cabaret_predictor(or_model& m) {
    const Decomp& d = m.d;
    V3 z = m.full(m.zeta[0]), zo = m.full(m.zeta_old[0]), r = m.sdv(m.res);
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i) z(i, j, l) = zo(i, j, l) + 0.5 * m.dt * r(i - 1, j - 1, l);
}

// cabaret_beta, qg3p_aux.F90:1023-1061.
void cabaret_beta(or_model& m) {
    const Decomp& d = m.d;
    V3 z = m.full(m.zeta[0]), ui = m.fi(m.ui), rb = m.sdv(m.res_beta);
    double ta = m.tweight_a;
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.l_j_min; j <= d.l_j_max; ++j)
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) {
                double res_beta = m.dt * (0.5 * (ui(i + 2, j + 1, l) + ui(i + 1, j + 1, l)) * m.beta[l - 1]);
                z(i + 1, j + 1, l) = z(i + 1, j + 1, l) + (1.0 + ta) * res_beta - ta * rb(i, j, l);
                rb(i, j, l) = res_beta;
            }
}

// cabaret_forcing, qg3p_aux.F90:1065-1164.
void cabaret_forcing(or_model& m) {
    const Decomp& d = m.d;
    int L = d.layers;
    V3 z = m.full(m.zeta[0]), rp = m.full(m.rel[0]);
    m.res_visc.assign(m.nsd(), 0.0);
    V3 rv = m.sdv(m.res_visc);
    V2 fw{m.wind.data(), d.ii, d.jj};
    bool has_wind = !m.wind.empty();
    double dt = m.dt, nu = m.p.viscosity, vb = m.p.visc_bot;
    auto lap = [&](int i, int j, int l) {
        return -4.0 * rp(i, j, l) + rp(i - 1, j, l) + rp(i + 1, j, l) + rp(i, j - 1, l) + rp(i, j + 1, l);
    };
    if (L == 1) {
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i)
                rv(i - 1, j - 1, 1) = dt * ((has_wind ? fw(i - 1, j - 1) : 0.0) - vb * rp(i, j, 1) + nu * lap(i, j, 1));
    } else {
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i)
                rv(i - 1, j - 1, 1) = dt * ((has_wind ? fw(i - 1, j - 1) : 0.0) + nu * lap(i, j, 1));
        for (int l = 2; l <= L - 1; ++l)
            for (int j = d.f_j_min; j <= d.f_j_max; ++j)
                for (int i = d.f_i_min; i <= d.f_i_max; ++i) rv(i - 1, j - 1, l) = dt * nu * lap(i, j, l);
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i)
                rv(i - 1, j - 1, L) = dt * (-vb * rp(i, j, L) + nu * lap(i, j, L));
    }
    for (int l = 1; l <= L; ++l)
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i) z(i, j, l) = z(i, j, l) + rv(i - 1, j - 1, l);
}

// cabaret_cell_boundaries_time_integrated, qg3p_aux.F90:1235-1313.
void cabaret_cell_boundaries(or_model& m) {
    const Decomp& d = m.d;
    int L = d.layers;
    V3 psi = m.full(m.psi[0]), ui = m.fi(m.ui), uj = m.fj(m.uj), uimo = m.fi(m.uimo), ujmo = m.fj(m.ujmo);
    m.psi_edge.assign(m.nfull(), 0.0);
    V3 pe = m.full(m.psi_edge);
    double tu = m.tweight_u;
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max; ++i)
                pe(i, j, l) = 0.25 * (psi(i, j, l) + psi(i, j - 1, l) + psi(i - 1, j, l) + psi(i - 1, j - 1, l));
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max - 1; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max; ++i) {
                double uim = -pe(i, j + 1, l) + pe(i, j, l);
                ui(i, j, l) = (1.0 + tu) * uim - tu * uimo(i, j, l);
                uimo(i, j, l) = uim;
            }
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max - 1; ++i) {
                double ujm = pe(i + 1, j, l) - pe(i, j, l);
                uj(i, j, l) = (1.0 + tu) * ujm - tu * ujmo(i, j, l);
                ujmo(i, j, l) = ujm;
            }
}

// cabaret_cell_boundaries_velocity, qg3p_aux.F90:1168-1231: the face
// velocities of psi itself, without time weighting, into uimo / ujmo (the
// checkpoint pickup's use, qg3.F90:326).
void cabaret_cell_boundaries_velocity(or_model& m) {
    const Decomp& d = m.d;
    int L = d.layers;
    V3 psi = m.full(m.psi[0]), uimo = m.fi(m.uimo), ujmo = m.fj(m.ujmo);
    m.psi_edge.assign(m.nfull(), 0.0);
    V3 pe = m.full(m.psi_edge);
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max; ++i)
                pe(i, j, l) = 0.25 * (psi(i, j, l) + psi(i, j - 1, l) + psi(i - 1, j, l) + psi(i - 1, j - 1, l));
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max - 1; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max; ++i) uimo(i, j, l) = -pe(i, j + 1, l) + pe(i, j, l);
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max - 1; ++i) ujmo(i, j, l) = pe(i + 1, j, l) - pe(i, j, l);
}

// cabaret_extrapolator, qg3p_aux.F90:1317-1544.
void cabaret_extrapolator(or_model& m) {
    const Decomp& d = m.d;
    int L = d.layers;
    bool lim = m.p.limiter != 0;
    V3 zeta = m.full(m.zeta[0]), zo = m.full(m.zeta_old[0]);
    V3 ui = m.fi(m.ui), uj = m.fj(m.uj), zfi = m.fi(m.zeta_fi), zfj = m.fj(m.zeta_fj);
    m.zeta_fin.assign(m.nfull(), 0.0);
    m.zeta_fjn.assign(m.nfull(), 0.0);
    V3 fin = m.full(m.zeta_fin), fjn = m.full(m.zeta_fjn);
    double dt = m.dt;
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max - 1; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max; ++i) {
                double u1 = ui(i, j, l), fi1 = zfi(i, j, l), fi2, psi_n, psi_o, v0, u2, d_f;
                if (u1 >= 0.0) {
                    if (d.p_b >= 0 || i > d.fb_i_min + 1) {
                        u2 = ui(i - 1, j, l);
                        fi2 = zfi(i - 1, j, l);
                        v0 = (u1 + u2) / 2.0;
                        psi_n = zeta(i - 1, j, l);
                        psi_o = zo(i - 1, j, l);
                        d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi1 - fi2);
                    } else {
                        fi2 = zeta(i - 1, j, l);
                        v0 = 0.0;
                        psi_n = zeta(i - 1, j, l);
                        psi_o = zo(i - 1, j, l);
                        d_f = -(psi_n - psi_o);
                    }
                } else {
                    if (d.p_d >= 0 || i < d.fb_i_max) {
                        u2 = ui(i + 1, j, l);
                        fi2 = zfi(i + 1, j, l);
                        v0 = (u1 + u2) / 2.0;
                        psi_n = zeta(i, j, l);
                        psi_o = zo(i, j, l);
                        d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi2 - fi1);
                    } else {
                        fi2 = zeta(i, j, l);
                        v0 = 0.0;
                        psi_n = zeta(i, j, l);
                        psi_o = zo(i, j, l);
                        d_f = -(psi_n - psi_o);
                    }
                }
                double v = 2.0 * psi_n - fi2;
                if (lim) {
                    double fmax = std::fmax(std::fmax(fi1, fi2), psi_n) - d_f;
                    double fmin = std::fmin(std::fmin(fi1, fi2), psi_n) - d_f;
                    if (v > fmax) v = fmax;
                    if (v < fmin) v = fmin;
                }
                fin(i, j, l) = v;
            }
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max - 1; ++i) {
                double u1 = uj(i, j, l), fi1 = zfj(i, j, l), fi2, psi_n, psi_o, v0, u2, d_f;
                if (u1 >= 0.0) {
                    if (d.p_c >= 0 || j > d.fb_j_min + 1) {
                        u2 = uj(i, j - 1, l);
                        fi2 = zfj(i, j - 1, l);
                        v0 = (u1 + u2) / 2.0;
                        psi_n = zeta(i, j - 1, l);
                        psi_o = zo(i, j - 1, l);
                        d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi1 - fi2);
                    } else {
                        fi2 = zeta(i, j - 1, l);
                        v0 = 0.0;
                        psi_n = zeta(i, j - 1, l);
                        psi_o = zo(i, j - 1, l);
                        d_f = -(psi_n - psi_o);
                    }
                } else {
                    if (d.p_a >= 0 || j < d.fb_j_max) {
                        u2 = uj(i, j + 1, l);
                        fi2 = zfj(i, j + 1, l);
                        v0 = (u1 + u2) / 2.0;
                        psi_n = zeta(i, j, l);
                        psi_o = zo(i, j, l);
                        d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi2 - fi1);
                    } else {
                        fi2 = zeta(i, j, l);
                        v0 = 0.0;
                        psi_n = zeta(i, j, l);
                        psi_o = zo(i, j, l);
                        d_f = -(psi_n - psi_o);
                    }
                }
                double v = 2.0 * psi_n - fi2;
                if (lim) {
                    double fmax = std::fmax(std::fmax(fi1, fi2), psi_n) - d_f;
                    double fmin = std::fmin(std::fmin(fi1, fi2), psi_n) - d_f;
                    if (v > fmax) v = fmax;
                    if (v < fmin) v = fmin;
                }
                fjn(i, j, l) = v;
            }
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max - 1; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max; ++i) zfi(i, j, l) = fin(i, j, l);
    for (int l = 1; l <= L; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max - 1; ++i) zfj(i, j, l) = fjn(i, j, l);
}

// cabaret_flux, qg3p_aux.F90:1547-1594.
void cabaret_flux(or_model& m) {
    const Decomp& d = m.d;
    V3 ui = m.fi(m.ui), uj = m.fj(m.uj), zfi = m.fi(m.zeta_fi), zfj = m.fj(m.zeta_fj);
    V3 fli = m.fi(m.flux_i), flj = m.fj(m.flux_j);
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.fa_j_min + 1; j <= d.fa_j_max - 1; ++j)
            for (int i = d.fa_i_min; i <= d.fa_i_max + 1; ++i) fli(i, j, l) = ui(i, j, l) * zfi(i, j, l);
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.fa_j_min; j <= d.fa_j_max + 1; ++j)
            for (int i = d.fa_i_min + 1; i <= d.fa_i_max - 1; ++i) flj(i, j, l) = uj(i, j, l) * zfj(i, j, l);
}

// cabaret_corrector, qg3p_aux.F90:1597-1642.
void cabaret_corrector(or_model& m) {
    const Decomp& d = m.d;
    V3 z = m.full(m.zeta[0]), fli = m.fi(m.flux_i), flj = m.fj(m.flux_j), r = m.sdv(m.res);
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i) {
                r(i - 1, j - 1, l) = -(fli(i + 1, j, l) - fli(i, j, l) + flj(i, j + 1, l) - flj(i, j, l));
                z(i, j, l) = z(i, j, l) + 0.5 * m.dt * r(i - 1, j - 1, l);
            }
}

// ---- leapfrog (qg3p_aux.F90:1644-2203) ------------------------------------
// The centred flux-form Jacobian + forcing increment T*(...) at interior
// node (i, j) of layer l; used by zeta_tendency (:1790-1939, with T = dt)
// and zeta_centred (:2027-2202, with T = 2 dt).  bottom friction follows
// the default (CENTRED_BOTTOM_FRICTION undefined) rel_p_l form.
double centred_increment(or_model& m, double T, V3& psi, V3& rel, V3& rel_p, int i, int j, int l) {
    int L = m.d.layers;
    V2 by{m.p_beta_y.data(), m.d.ii + 2, L};
    V2 fw{m.wind.data(), m.d.ii, m.d.jj};
    bool has_wind = !m.wind.empty();
    double nu = m.p.viscosity, vb = m.p.visc_bot;
    auto q = [&](int a, int b) {
        // beta_y + rel + stratification coupling at (a, b) in layer l.
        double v = by(a, l) + rel(a, b, l);
        if (L > 1) {
            if (l == 1) {
                v += S2(m, 1) * psi(a, b, 2);
            } else if (l == L) {
                v += S1(m, L) * psi(a, b, L - 1);
            } else {
                v += S1(m, l) * psi(a, b, l - 1);
                v += S2(m, l) * psi(a, b, l + 1);
            }
        }
        return v;
    };
    double jac = 0.25 * ((q(i, j + 1) * (psi(i - 1, j + 1, l) - psi(i + 1, j + 1, l))) -
                         (q(i, j - 1) * (psi(i - 1, j - 1, l) - psi(i + 1, j - 1, l))) -
                         (q(i - 1, j) * (psi(i - 1, j + 1, l) - psi(i - 1, j - 1, l))) +
                         (q(i + 1, j) * (psi(i + 1, j + 1, l) - psi(i + 1, j - 1, l))));
    double lap = -4.0 * rel_p(i, j, l) + rel_p(i - 1, j, l) + rel_p(i + 1, j, l) + rel_p(i, j - 1, l) +
                 rel_p(i, j + 1, l);
    double inc;
    if (L == 1) {
        // Single layer: the reference places the bottom friction inside the
        // viscosity bracket (:1839-1842, :2063-2070).
        inc = jac + (has_wind ? fw(i - 1, j - 1) : 0.0) + nu * (lap - vb * rel_p(i, j, 1));
    } else if (l == 1) {
        inc = jac + (has_wind ? fw(i - 1, j - 1) : 0.0) + nu * lap;
    } else if (l == L) {
        inc = jac + nu * lap - vb * rel_p(i, j, L);
    } else {
        inc = jac + nu * lap;
    }
    return T * inc;
}

void zeta_forward_euler(or_model& m) {
    const Decomp& d = m.d;
    V3 psi = m.full(m.psi[0]), rel = m.full(m.rel[0]), z1 = m.full(m.zeta[0]), z2 = m.full(m.zeta[1]);
    std::vector<double> zt(m.nfull(), 0.0);
    V3 t = m.full(zt);
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i) t(i, j, l) = centred_increment(m, m.dt, psi, rel, rel, i, j, l);
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.l_j_min; j <= d.l_j_max; ++j)
            for (int i = d.l_i_min; i <= d.l_i_max; ++i) z2(i + 1, j + 1, l) = z1(i + 1, j + 1, l) + t(i + 1, j + 1, l);
}

void zeta_centred(or_model& m, int lf) {
    const Decomp& d = m.d;
    int mm = lf % 2 + 1;
    V3 psi_m = m.full(m.psi[mm - 1]), rel_m = m.full(m.rel[mm - 1]), rel_p_l = m.full(m.rel[lf - 1]);
    V3 zl = m.full(m.zeta[lf - 1]);
    double T = 2.0 * m.dt;
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i)
                zl(i, j, l) = zl(i, j, l) + centred_increment(m, T, psi_m, rel_m, rel_p_l, i, j, l);
}

// robert_asselin_filter_pdata + _rank3 with RA_DOUBLE_FILTER,
// qg3p_aux.F90:48-64, 1719-1786.
void raw_filter(or_model& m, int lf) {
    const Decomp& d = m.d;
    int mm = lf % 2 + 1;
    double w21 = 0.5 * m.p.ra_nu * m.p.ra_alpha;
    double w22 = 1.0 - 2.0 * w21;
    double w11 = -0.5 * m.p.ra_nu * (1.0 - m.p.ra_alpha);
    double w12 = -2.0 * w11;
    double w13 = 1.0 + w11;
    V3 pl = m.full(m.zeta[lf - 1]), pm = m.full(m.zeta[mm - 1]);
    V3 ol = m.full(m.zeta_old[lf - 1]), om = m.full(m.zeta_old[mm - 1]);
    for (int l = 1; l <= d.layers; ++l)
        for (int j = d.fa_j_min; j <= d.fa_j_max; ++j)
            for (int i = d.fa_i_min; i <= d.fa_i_max; ++i) {
                double lphi_l = pl(i, j, l);
                pl(i, j, l) = w11 * ol(i, j, l) + w12 * pm(i, j, l) + w13 * lphi_l;
                pm(i, j, l) = w21 * (ol(i, j, l) + lphi_l) + w22 * pm(i, j, l);
                om(i, j, l) = pm(i, j, l);
            }
}

int invert_level(or_model& m, int lv) {
    int rc = pv_inversion(m, m.zeta[lv], m.psi[lv]);
    if (rc) return rc;
    update_pdata(m, m.psi[lv]);  // qg3.F90:642-643
    rel_from_zeta_and_psi(m, m.zeta[lv], m.psi[lv], m.rel[lv]);
    update_zeta_bc(m, m.rel[lv], m.psi[lv], m.zeta[lv]);
    return 0;
}

}  // namespace

// ===========================================================================
// C API
extern "C" {

void or_strat_l2(double rd_bcl, double h1, double h2, double* s1, double* s2) { strat_l2(rd_bcl, h1, h2, s1, s2); }

void or_strat_l3(double rd_bcl1, double rd_bcl2, double h1, double h2, double h3, double* s1, double* s21,
                 double* s22, double* s3) {
    strat_l3(rd_bcl1, rd_bcl2, h1, h2, h3, s1, s21, s22, s3);
}

static int finish_strat(int L, double* s1, double* s2, double* ss, double* m2z, double* z2m) {
    std::vector<double> S((size_t)L * L);
    s_matrix(L, s1, s2, S.data());
    return s_conversion_matrices(L, S.data(), m2z, z2m, ss);
}

int or_strat_from_parameters(int L, const double* h, const double* s1_in, const double* s2_in, double l_scale,
                             double* h_out, double* s1_out, double* s2_out, double* ss, double* m2z, double* z2m) {
    if (L <= 0) return -1;
    double ls2 = l_scale * l_scale;
    for (int k = 0; k < L; ++k) {
        h_out[k] = h[k] / l_scale;
        s1_out[k] = 0.0;
        s2_out[k] = 0.0;
    }
    for (int k = 0; k < L - 1; ++k) {
        s1_out[k + 1] = ls2 * s1_in[k];
        s2_out[k] = ls2 * s2_in[k];
    }
    return finish_strat(L, s1_out, s2_out, ss, m2z, z2m);
}

int or_strat_from_rd(int L, const double* rd, const double* h, double l_scale, double* h_out, double* s1_out,
                     double* s2_out, double* ss, double* m2z, double* z2m) {
    if (L < 1 || L > 3) return -1;
    for (int k = 0; k < L; ++k) {
        s1_out[k] = 0.0;
        s2_out[k] = 0.0;
        h_out[k] = h[k] / l_scale;
    }
    double ls2 = l_scale * l_scale;
    if (L == 2) {
        strat_l2(rd[0], h[0], h[1], &s2_out[0], &s1_out[1]);
        s2_out[0] *= ls2;
        s1_out[1] *= ls2;
    } else if (L == 3) {
        strat_l3(rd[0], rd[1], h[0], h[1], h[2], &s2_out[0], &s1_out[1], &s2_out[1], &s1_out[2]);
        s2_out[0] *= ls2;
        s2_out[1] *= ls2;
        s1_out[1] *= ls2;
        s1_out[2] *= ls2;
    }
    return finish_strat(L, s1_out, s2_out, ss, m2z, z2m);
}

int or_eigen_real_tridiag(int n, const double* a, double* w, double* v) { return eigen_real_tridiag(n, a, w, v); }
int or_inverse(int n, const double* a, double* ainv) { return inverse(n, a, ainv); }

int or_solve(int n, const double* a, const double* rhs, double* x) {
    std::vector<double> ai((size_t)n * n);
    if (inverse(n, a, ai.data()) != 0) return -1;
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += ai[i + (size_t)n * k] * rhs[k];
        x[i] = s;
    }
    return 0;
}

double or_determinant(int n, const double* a_in) {
    std::vector<double> a(a_in, a_in + (size_t)n * n);
    double det = 1.0;
    for (int k = 0; k < n; ++k) {
        int piv = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(a[i + n * k]) > std::fabs(a[piv + n * k])) piv = i;
        if (a[piv + n * k] == 0.0) return 0.0;
        if (piv != k) {
            for (int j = 0; j < n; ++j) std::swap(a[k + n * j], a[piv + n * j]);
            det = -det;
        }
        det *= a[k + n * k];
        for (int i = k + 1; i < n; ++i) {
            double f = a[i + n * k] / a[k + n * k];
            for (int j = k; j < n; ++j) a[i + n * j] -= f * a[k + n * j];
        }
    }
    return det;
}

or_helm_cache* or_helm_create(int ii, int jj, int layers, const double* ss, int periodic_j) {
    if (ii < 3 || jj < 3 || layers < 1) return nullptr;
    or_helm_cache* h = new or_helm_cache;
    helm_init(h->c, make_decomp(ii, jj, layers, periodic_j != 0), ss);
    return h;
}

void or_helm_destroy(or_helm_cache* h) { delete h; }

int or_helm(or_helm_cache* h, double* zeta) { return helm(h->c, zeta); }

int or_sint(or_helm_cache* h, double* x) { return sint1(h->c.sint, x); }

void or_add_laplace_bc_rhs(int ii, int jj, int layers, int periodic_j, double bc, double bc_d, double* rhs) {
    Decomp d = make_decomp(ii, jj, layers, periodic_j != 0);
    for (int l = 0; l < layers; ++l) add_laplace_bc_rhs_layer(d, bc, bc_d, rhs + (size_t)l * ii * jj);
}

void or_apply_dirichlet_bc(int ii, int jj, int layers, int periodic_j, double bc, double bc_d, double* zeta) {
    Decomp d = make_decomp(ii, jj, layers, periodic_j != 0);
    for (int l = 0; l < layers; ++l) apply_dirichlet_bc_layer(d, bc, bc_d, zeta + (size_t)l * ii * jj);
}

double or_mean(int ii, int jj, int periodic_j, const double* psi) {
    Decomp d = make_decomp(ii, jj, 1, periodic_j != 0);
    return mean_layer(d, psi);
}

void or_energy(int ii, int jj, int layers, int periodic_j, const double* h, const double* s2, const double* psi,
               double* ekin, double* epot) {
    Decomp d = make_decomp(ii, jj, layers, periodic_j != 0);
    energy(d, h, s2, psi, ekin, epot);
}

or_model* or_model_create(const or_params* p) {
    if (!p || p->ii < 5 || p->jj < 5 || p->layers < 1) return nullptr;
    or_model* m = new or_model;
    m->p = *p;
    int L = p->layers;
    m->d = make_decomp(p->ii, p->jj, L, p->periodic_j != 0);
    m->beta.assign(p->beta, p->beta + L);
    m->h.assign(p->h, p->h + L);
    m->s1.assign(p->s1, p->s1 + L);
    m->s2.assign(p->s2, p->s2 + L);
    m->ss.assign(p->ss, p->ss + L);
    m->m2z.assign(p->m2z, p->m2z + L * L);
    m->z2m.assign(p->z2m, p->z2m + L * L);
    if (p->force_wind) m->wind.assign(p->force_wind, p->force_wind + (size_t)p->ii * p->jj);
    m->p.beta = m->p.h = m->p.s1 = m->p.s2 = m->p.ss = m->p.m2z = m->p.z2m = m->p.force_wind = nullptr;
    m->dt = p->dt;
    helm_init(m->hc, m->d, m->ss.data());
    if (m->d.periodic_j)
        correction_function_momentum(*m);
    else
        correction_function_mass(*m);
    for (int lv = 0; lv < 2; ++lv) {
        m->psi[lv].assign(m->nfull(), 0.0);
        m->rel[lv].assign(m->nfull(), 0.0);
        m->zeta[lv].assign(m->nfull(), 0.0);
        m->zeta_old[lv].assign(m->nfull(), 0.0);
    }
    m->zeta_fi.assign(m->nfi(), 0.0);
    m->ui.assign(m->nfi(), 0.0);
    m->uimo.assign(m->nfi(), 0.0);
    m->flux_i.assign(m->nfi(), 0.0);
    m->zeta_fj.assign(m->nfj(), 0.0);
    m->uj.assign(m->nfj(), 0.0);
    m->ujmo.assign(m->nfj(), 0.0);
    m->flux_j.assign(m->nfj(), 0.0);
    m->res.assign(m->nsd(), 0.0);
    m->res_beta.assign(m->nsd(), 0.0);
    // p_beta_y, qg3.F90:303-307.
    m->p_beta_y.assign((size_t)(p->ii + 2) * L, 0.0);
    for (int l = 1; l <= L; ++l)
        for (int i = 0; i <= p->ii + 1; ++i)
            m->p_beta_y[(size_t)i + (size_t)(p->ii + 2) * (l - 1)] =
                m->beta[l - 1] * (((double)p->ii + 1.0) / 2.0 - (double)i);
    return m;
}

void or_model_destroy(or_model* m) { delete m; }

int or_model_init(or_model* m, const double* zeta_ic) {
    const Decomp& d = m->d;
    int nlev = m->p.scheme == 1 ? 2 : 1;
    for (int lv = 0; lv < nlev; ++lv) {
        std::fill(m->zeta[lv].begin(), m->zeta[lv].end(), 0.0);
        V3 z = m->full(m->zeta[lv]);
        const double* src = zeta_ic + (size_t)lv * m->nsd();
        for (int l = 1; l <= d.layers; ++l)
            for (int j = 1; j <= d.jj; ++j)
                for (int i = 1; i <= d.ii; ++i)
                    z(i + 1, j + 1, l) = src[(size_t)(i - 1) + (size_t)d.ii * ((j - 1) + (size_t)d.jj * (l - 1))];
        // apply_dirichlet_bc(0, zeta) on sdata (the walls only in a channel),
        // then update(zeta) (qg3.F90:383-385).
        for (int l = 1; l <= d.layers; ++l) {
            if (!d.periodic_j)
                for (int i = 1; i <= d.ii; ++i) {
                    z(i + 1, 2, l) = 0.0;
                    z(i + 1, d.jj + 1, l) = 0.0;
                }
            for (int j = 1; j <= d.jj; ++j) {
                z(2, j + 1, l) = 0.0;
                z(d.ii + 1, j + 1, l) = 0.0;
            }
        }
        update_pdata(*m, m->zeta[lv]);
        int rc = invert_level(*m, lv);
        if (rc) return rc;
    }
    for (auto* v : {&m->zeta_fi, &m->zeta_fj, &m->ui, &m->uj, &m->uimo, &m->ujmo, &m->flux_i, &m->flux_j, &m->res,
                    &m->res_beta})
        std::fill(v->begin(), v->end(), 0.0);
    for (int lv = 0; lv < nlev; ++lv) m->zeta_old[lv] = m->zeta[lv];
    if (m->p.scheme == 0) {
        m->model_time = m->dt / 2.0;
        m->tweight_a = 0.5;
        m->tweight_u = 0.5;
    } else {
        // FORWARD_EULER_START, qg3.F90:463-497.
        m->model_time = 0.0;
        m->lf_count = 0;
        zeta_forward_euler(*m);
        update_pdata(*m, m->zeta[1]);  // qg3.F90:475
        int rc = invert_level(*m, 1);
        if (rc) return rc;
        m->zeta_old[1] = m->zeta[1];
        m->model_time += m->dt;
    }
    return 0;
}

static void accumulate_quad(or_model& m, int lv);

// psi_av += dt * psi%sdata and diagnostic_time += dt once start_time +
// model_time > max_spin (qg3.F90:672-680, 725); av_threshold holds
// max_spin - start_time.  lv: the time level just inverted (psi BLEAPFROG).
static void accumulate_average(or_model& m, int lv) {
    if (!m.av_on || !(m.model_time > m.av_threshold)) return;
    V3 psi = m.full(m.psi[lv]), av = m.sdv(m.psi_av);
    const Decomp& d = m.d;
    for (int l = 1; l <= d.layers; ++l)
        for (int j = 1; j <= d.jj; ++j)
            for (int i = 1; i <= d.ii; ++i) av(i, j, l) = av(i, j, l) + m.dt * psi(i + 1, j + 1, l);
    if (m.quad_on) accumulate_quad(m, lv);
    m.diag_time = m.diag_time + m.dt;
}

// Layers of quad accumulator q (EC_INTERFACES: L - 1).
static int quad_layers(const or_model& m, int q) {
    return (q == 2 || q == 3 || q == 19 || q == 20 || q == 22) ? m.d.layers - 1 : m.d.layers;
}

// The quad diagnostics of one step, qg3.F90:683-721: zonal_velocity,
// meridional_velocity (qg3p_diagnostics.F90:941-1107; rows / columns the
// reference never writes stay 0 as at their allocation, qg3.F90:508-512),
// interface_velocity (:1163-1194), thickness (:1197-1227), the dt-weighted
// products (add_eddy_covariance_*_scale, :1360-1427) and
// add_scaled_buoyancy_corr (:1430-1537).  The reference zeroes every
// accumulator but ut, vt, rt and tt (qg3.F90:540-558), which it leaves
// uninitialised; here all start at 0.
static void accumulate_quad(or_model& m, int lv) {
    const Decomp& d = m.d;
    const int L = d.layers, ii = d.ii, jj = d.jj;
    V3 psi = m.full(m.psi[lv]), rel = m.full(m.rel[lv]), zeta = m.full(m.zeta[lv]);
    auto sd = [&](V3& a, int i, int j, int l) -> double& { return a(i + 1, j + 1, l); };
    std::vector<double> uv(m.nsd(), 0.0), vv(m.nsd(), 0.0), tv(m.nsd(), 0.0);
    V3 u = m.sdv(uv), v = m.sdv(vv), t = m.sdv(tv);
    const double nanv = std::numeric_limits<double>::quiet_NaN();
    for (int l = 1; l <= L; ++l)
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i) u(i - 1, j - 1, l) = 0.5 * (psi(i + 1, j, l) - psi(i - 1, j, l));
    for (int l = 1; l <= L; ++l)
        for (int j = d.f_j_min; j <= d.f_j_max; ++j) {
            double w1, w2;
            if (m.p.bc_type == OR_BC_PARTIAL_SLIP) {
                w1 = sd(rel, 1, j - 1, l) / m.p.alpha;
                w2 = sd(rel, ii, j - 1, l) / m.p.alpha;
            } else if (m.p.bc_type == OR_BC_NO_SLIP) {
                w1 = w2 = 0.0;
            } else {
                w1 = w2 = nanv;
            }
            if (d.p_b == -1) u(1, j - 1, l) = w1;
            if (d.p_d == -1) u(ii, j - 1, l) = w2;
        }
    for (int l = 1; l <= L; ++l)
        for (int j = d.f_j_min; j <= d.f_j_max; ++j)
            for (int i = d.f_i_min; i <= d.f_i_max; ++i) v(i - 1, j - 1, l) = 0.5 * (psi(i, j + 1, l) - psi(i, j - 1, l));
    for (int l = 1; l <= L; ++l)
        for (int i = d.f_i_min; i <= d.f_i_max; ++i) {
            double w1, w2;
            if (m.p.bc_type == OR_BC_PARTIAL_SLIP) {
                w1 = sd(rel, i - 1, 1, l) / m.p.alpha;
                w2 = sd(rel, i - 1, jj, l) / m.p.alpha;
            } else if (m.p.bc_type == OR_BC_NO_SLIP) {
                w1 = w2 = 0.0;
            } else {
                w1 = w2 = nanv;
            }
            if (d.p_c == -1) v(i - 1, 1, l) = w1;
            if (d.p_a == -1) v(i - 1, jj, l) = w2;
        }
    if (L > 1) {
        for (int j = 1; j <= jj; ++j)
            for (int i = 1; i <= ii; ++i) {
                t(i, j, 1) = -m.s2[0] * (sd(psi, i, j, 1) - sd(psi, i, j, 2));
                t(i, j, L) = -m.s1[L - 1] * (sd(psi, i, j, L) - sd(psi, i, j, L - 1));
            }
        for (int l = 2; l <= L - 1; ++l)
            for (int j = 1; j <= jj; ++j)
                for (int i = 1; i <= ii; ++i)
                    t(i, j, l) = -m.s1[l - 1] * (sd(psi, i, j, l) - sd(psi, i, j, l - 1)) -
                                 m.s2[l - 1] * (sd(psi, i, j, l) - sd(psi, i, j, l + 1));
    }
    const double dt = m.dt;
    auto acc = [&](int q, int i, int j, int l) -> double& {
        return m.quad[q][(size_t)(i - 1) + (size_t)ii * ((size_t)(j - 1) + (size_t)jj * (size_t)(l - 1))];
    };
    for (int l = 1; l <= L; ++l)
        for (int j = 1; j <= jj; ++j)
            for (int i = 1; i <= ii; ++i) {
                const double U = u(i, j, l), Vv = v(i, j, l), R = sd(rel, i, j, l), Z = sd(zeta, i, j, l);
                const double Pp = sd(psi, i, j, l), T = t(i, j, l);
                acc(0, i, j, l) += dt * U * U;
                acc(1, i, j, l) += dt * Vv * Vv;
                acc(4, i, j, l) += dt * U * Vv;
                acc(5, i, j, l) += dt * U * R;
                acc(6, i, j, l) += dt * Vv * R;
                acc(7, i, j, l) += dt * R * R;
                acc(8, i, j, l) += dt * Pp * R;
                acc(9, i, j, l) += dt * U * Z;
                acc(10, i, j, l) += dt * Vv * Z;
                acc(11, i, j, l) += dt * Z * Z;
                acc(12, i, j, l) += dt * Z * R;
                acc(13, i, j, l) += dt * Pp * Pp;
                acc(14, i, j, l) += dt * Pp * Z;
                acc(15, i, j, l) += dt * U * T;
                acc(16, i, j, l) += dt * Vv * T;
                acc(17, i, j, l) += dt * T * R;
                acc(18, i, j, l) += dt * T * T;
            }
    for (int l = 1; l <= L - 1; ++l)
        for (int j = 1; j <= jj; ++j)
            for (int i = 1; i <= ii; ++i) {
                const double ui = 0.5 * (u(i, j, l) + u(i, j, l + 1)), vi = 0.5 * (v(i, j, l) + v(i, j, l + 1));
                acc(2, i, j, l) += dt * ui * ui;
                acc(3, i, j, l) += dt * vi * vi;
            }
    if (L == 1) return;
    for (int l = 1; l <= L - 1; ++l)
        for (int j = 1; j <= jj; ++j)
            for (int i = 1; i <= ii; ++i) {
                const double dp = sd(psi, i, j, l) - sd(psi, i, j, l + 1);
                const double sc_b = m.s2[l - 1] * m.h[l - 1] * dp;
                acc(19, i, j, l) += dt * (0.5 * (u(i, j, l + 1) + u(i, j, l)) * sc_b);
                acc(20, i, j, l) += dt * (0.5 * (v(i, j, l + 1) + v(i, j, l)) * sc_b);
                acc(22, i, j, l) += dt * (m.s2[l - 1] * m.h[l - 1] * (dp * dp) / (m.h[l - 1] + m.h[l]));
            }
    for (int j = 1; j <= jj; ++j)
        for (int i = 1; i <= ii; ++i) {
            const double a = sd(psi, i, j, 2) - sd(psi, i, j, 1);
            acc(21, i, j, 1) += dt * (0.25 * (m.s2[0] * (a * a)));
        }
    for (int l = 2; l <= L - 1; ++l)
        for (int j = 1; j <= jj; ++j)
            for (int i = 1; i <= ii; ++i) {
                const double a = sd(psi, i, j, l - 1) - sd(psi, i, j, l), b = sd(psi, i, j, l + 1) - sd(psi, i, j, l);
                acc(21, i, j, l) += dt * (0.25 * (m.s1[l - 1] * (a * a) + m.s2[l - 1] * (b * b)));
            }
    for (int j = 1; j <= jj; ++j)
        for (int i = 1; i <= ii; ++i) {
            const double a = sd(psi, i, j, L - 1) - sd(psi, i, j, L);
            acc(21, i, j, L) += dt * (0.25 * (m.s1[L - 1] * (a * a)));
        }
}

// Start (clearing the sums, qg3.F90:502-503, 540-558) or stop the time
// average; enable = 2 adds the quad eddy covariances.
void or_model_average(or_model* m, int enable, double threshold) {
    m->av_on = enable != 0;
    m->quad_on = enable == 2;
    m->av_threshold = threshold;
    m->diag_time = 0.0;
    m->psi_av.assign(m->nsd(), 0.0);
    for (int q = 0; q < 23; ++q)
        m->quad[q].assign(m->quad_on ? (size_t)m->d.ii * m->d.jj * quad_layers(*m, q) : 0, 0.0);
}

// Quad accumulator q (ii, jj, layers of q), unscaled; returns its length.
long or_model_get_quad(or_model* m, int q, double* out) {
    if (q < 0 || q >= 23 || !m->quad_on) return -1;
    if (out) std::memcpy(out, m->quad[q].data(), m->quad[q].size() * sizeof(double));
    return (long)m->quad[q].size();
}

// The summed dt * psi (ii, jj, L) and diagnostic_time.
double or_model_get_average(or_model* m, double* sum) {
    if (sum) std::memcpy(sum, m->psi_av.data(), m->psi_av.size() * sizeof(double));
    return m->diag_time;
}

// The CABARET timestep_loop body (qg3.F90:590-967) up to its data output
// and exit point (:807-934): adapt_dt, predictor, beta, inversion, rel and
// boundary PV, half the time increment, forcing, cell boundaries,
// extrapolator, flux.  The state here is what the reference's checkpoint
// holds.
int or_model_step_to_dump(or_model* m) {
    if (m->p.scheme != 0) return -1;
    if (m->p.adapt_dt) cabaret_adapt_dt(*m);
    cabaret_predictor(*m);
    cabaret_beta(*m);
    update_pdata(*m, m->zeta[0]);  // qg3.F90:610
    int rc = invert_level(*m, 0);
    if (rc) return rc;
    m->model_time += 0.5 * m->dt;
    accumulate_average(*m, 0);
    cabaret_forcing(*m);
    update_pdata(*m, m->zeta[0]);  // :786
    cabaret_cell_boundaries(*m);
    update_flux_j(*m, m->uj, true);  // :795-796 (update(ui) has no halo on one rank)
    cabaret_extrapolator(*m);
    update_flux_j(*m, m->zeta_fj, true);  // :802-803
    cabaret_flux(*m);
    return 0;
}

// The rest of the body after the exit point (qg3.F90:940-956): corrector,
// zeta_old = zeta, the second half of the time increment.
int or_model_finish_step(or_model* m) {
    if (m->p.scheme != 0) return -1;
    cabaret_corrector(*m);
    update_pdata(*m, m->zeta[0]);  // qg3.F90:945
    m->zeta_old[0] = m->zeta[0];
    m->model_time += 0.5 * m->dt;
    return 0;
}

int or_model_step(or_model* m, int nsteps) {
    for (int s = 0; s < nsteps; ++s) {
        if (m->p.scheme == 0) {
            int rc = or_model_step_to_dump(m);
            if (rc) return rc;
            or_model_finish_step(m);
        } else {
            // One DOLEAPFROG sub-step, qg3.F90:615-651.  The sub-step index
            // alternates 1, 2, 1, 2, ... from the first step after the
            // forward-Euler start.
            int lf = (m->lf_count % 2 == 0) ? 1 : 2;
            m->lf_count += 1;
            zeta_centred(*m, lf);
            update_pdata(*m, m->zeta[lf - 1]);  // qg3.F90:625
            raw_filter(*m, lf);
            int rc = invert_level(*m, lf - 1);
            if (rc) return rc;
            m->model_time += m->dt;
            accumulate_average(*m, lf - 1);
        }
    }
    return 0;
}

// START_PICKUP (qg3.F90:314-363) and the common timestep initialisation
// (:448-462) on fields already loaded with or_model_set from a checkpoint:
// CABARET: psi, zeta, ui, uj, zeta_fi, zeta_fj, res, res_beta (read by
// read_parallel_checkpoint, qg3p_io.F90:202-314) and the checkpoint's dt;
// the face velocities of psi become uimo / ujmo, flux = u * zeta_f, and the
// corrector takes zeta half a step forwards.  Leapfrog: psi, zeta of both
// levels; rel = rel_from_psi of each level.  Then zeta_old = zeta, and
// model_time = dt / 2 with tweights 0.5 (CABARET) or model_time = 0 with the
// forward-Euler start skipped (leapfrog, :461-497).
int or_model_pickup(or_model* m, double dt) {
    if (m->p.scheme == 0) {
        m->dt = dt;
        // qg3.F90:324-329: halos of psi and of the face PV (a channel's
        // only; update(zeta_fi) has no neighbour in i on one rank).
        update_pdata(*m, m->psi[0]);
        update_flux_j(*m, m->zeta_fj, false);
        cabaret_cell_boundaries_velocity(*m);
        cabaret_flux(*m);
        cabaret_corrector(*m);
        update_pdata(*m, m->zeta[0]);  // :339
        m->zeta_old[0] = m->zeta[0];
        m->model_time = m->dt / 2.0;
        m->tweight_a = 0.5;
        m->tweight_u = 0.5;
    } else {
        for (int lv = 0; lv < 2; ++lv) {
            // qg3.F90:355-361: halos of psi and zeta, rel from psi, halo of rel.
            update_pdata(*m, m->psi[lv]);
            update_pdata(*m, m->zeta[lv]);
            rel_from_psi(*m, m->psi[lv], m->rel[lv]);
            update_pdata(*m, m->rel[lv]);
            m->zeta_old[lv] = m->zeta[lv];
        }
        m->model_time = 0.0;
        m->lf_count = 0;
    }
    return 0;
}

long or_model_get(or_model* m, const char* name, double* out) {
    std::string n(name);
    std::vector<double>* v = nullptr;
    if (n == "psi") v = &m->psi[0];
    else if (n == "zeta") v = &m->zeta[0];
    else if (n == "rel") v = &m->rel[0];
    else if (n == "zeta_old") v = &m->zeta_old[0];
    else if (n == "psi2") v = &m->psi[1];
    else if (n == "zeta2") v = &m->zeta[1];
    else if (n == "rel2") v = &m->rel[1];
    else if (n == "zeta_old2") v = &m->zeta_old[1];
    else if (n == "ui") v = &m->ui;
    else if (n == "uj") v = &m->uj;
    else if (n == "uimo") v = &m->uimo;
    else if (n == "ujmo") v = &m->ujmo;
    else if (n == "zeta_fi") v = &m->zeta_fi;
    else if (n == "zeta_fj") v = &m->zeta_fj;
    else if (n == "flux_i") v = &m->flux_i;
    else if (n == "flux_j") v = &m->flux_j;
    else if (n == "res") v = &m->res;
    else if (n == "res_beta") v = &m->res_beta;
    else if (n == "corr") v = &m->corr;
    else return -1;
    if (out) std::memcpy(out, v->data(), v->size() * sizeof(double));
    return (long)v->size();
}

long or_model_set(or_model* m, const char* name, const double* in) {
    long n = or_model_get(m, name, nullptr);
    if (n < 0) return n;
    std::string s(name);
    std::vector<double>* v = nullptr;
    if (s == "psi") v = &m->psi[0];
    else if (s == "zeta") v = &m->zeta[0];
    else if (s == "rel") v = &m->rel[0];
    else if (s == "zeta_old") v = &m->zeta_old[0];
    else if (s == "psi2") v = &m->psi[1];
    else if (s == "zeta2") v = &m->zeta[1];
    else if (s == "rel2") v = &m->rel[1];
    else if (s == "zeta_old2") v = &m->zeta_old[1];
    else if (s == "ui") v = &m->ui;
    else if (s == "uj") v = &m->uj;
    else if (s == "uimo") v = &m->uimo;
    else if (s == "ujmo") v = &m->ujmo;
    else if (s == "zeta_fi") v = &m->zeta_fi;
    else if (s == "zeta_fj") v = &m->zeta_fj;
    else if (s == "flux_i") v = &m->flux_i;
    else if (s == "flux_j") v = &m->flux_j;
    else if (s == "res") v = &m->res;
    else if (s == "res_beta") v = &m->res_beta;
    else return -1;
    std::memcpy(v->data(), in, v->size() * sizeof(double));
    return n;
}

void or_model_scalars(or_model* m, double* out4) {
    out4[0] = m->dt;
    out4[1] = m->tweight_a;
    out4[2] = m->tweight_u;
    out4[3] = m->model_time;
}

int or_model_energy(or_model* m, double* ekin, double* epot) {
    int lv = m->p.scheme == 1 ? 1 : 0;  // psi BNLEAPFROG
    return energy(m->d, m->h.data(), m->s2.data(), m->psi[lv].data(), ekin, epot);
}

// cabaret_cfl, qg3p_aux.F90:920-942.
double or_model_cfl(or_model* m) { return maxabs_u(*m) * m->dt; }

int or_pv_inversion(or_model* m, const double* zeta_data, double* psi_data) {
    std::vector<double> z(zeta_data, zeta_data + m->nfull());
    std::vector<double> p(psi_data, psi_data + m->nfull());
    int rc = pv_inversion(*m, z, p);
    std::memcpy(psi_data, p.data(), p.size() * sizeof(double));
    return rc;
}

// ---------------------------------------------------------------------------
// Double-gyre driver set-up, restated from the reference's qg3 program for
// the configuration the tests and the CPU baseline run: the
// non-dimensionalisation (qg3.F90:152-168), the STRAT_INPUT stratification
// file (qg3p_io.F90:56-102: line k holds h(k), s1(k-1), s2(k)) with
// s2(k) = f0^2 / (g'_k H_k), s1(k+1) = f0^2 / (g'_k H_(k+1)), the
// stratification object (qg3p_diagnostics.F90:210-236, 342-422), tau / h(1)
// (qg3.F90:235), the boundary condition (:239-248), the wind curl (:253-271)
// and beta (:163).  Computed here from the physical parameters alone, so the
// checker does not share the product's set-up code.
int or_setup_double_gyre(const or_physical* p, or_setup* out, double* wind) {
    if (!p || !out || p->layers < 1 || p->layers > 8 || p->ii < 5 || p->jj < 5) return -1;
    std::memset(out, 0, sizeof(*out));
    const int L = p->layers;
    const double u_scale = p->u_scale > 0.0 ? p->u_scale : 1.0;
    const int g_ii_int = p->ii - 1;
    const double l_scale = p->basinscale / (double)g_ii_int;  // qg3.F90:152
    const double t_scale = l_scale / u_scale;                 // :153
    out->l_scale = l_scale;
    out->t_scale = t_scale;
    out->dt = p->dt / t_scale;                                // :155
    out->max_dt = p->max_dt > 0.0 ? p->max_dt / t_scale : 1.0e300;  // :159
    out->alpha = l_scale / p->alpha;                          // :161
    const double beta = p->beta * l_scale * l_scale / u_scale;  // :162
    out->viscosity = p->visc / (l_scale * u_scale);           // :166
    out->visc_bot = p->visc_bot * l_scale / u_scale;          // :167
    double tau = p->tau / (u_scale * u_scale * (double)g_ii_int);  // :164
    // Stratification file values (cgs): s1_in(k) = strat%s1(k+1),
    // s2_in(k) = strat%s2(k), k = 1..L-1.
    double s1_in[8] = {0}, s2_in[8] = {0};
    for (int k = 0; k < L - 1; ++k) {
        s2_in[k] = p->f0 * p->f0 / (p->gprime[k] * p->H[k]);
        s1_in[k] = p->f0 * p->f0 / (p->gprime[k] * p->H[k + 1]);
    }
    int rc = or_strat_from_parameters(L, p->H, s1_in, s2_in, l_scale, out->h, out->s1, out->s2, out->ss,
                                      out->m2z, out->z2m);
    if (rc) return rc;
    for (int k = 0; k < L; ++k) out->beta[k] = beta;
    tau = tau / out->h[0];  // qg3.F90:235
    if (p->partial_slip) {  // :239-248
        if (p->alpha >= 1.0e100) {
            out->bc_type = OR_BC_FREE_SLIP;
            out->alpha = 0.0;
        } else {
            out->bc_type = OR_BC_PARTIAL_SLIP;
        }
    } else {
        out->bc_type = OR_BC_NO_SLIP;
    }
    if (wind) {  // :253-271 (one rank: ii_0 = jj_0 = 0)
        const double pi = 3.14159265358979323846;
        const double a_wind = -1.0 * p->wind_asym, b_wind = 1.0 / p->wind_asym;
        for (int j = 1; j <= p->jj; ++j)
            for (int i = 1; i <= p->ii; ++i) {
                const double x = (double)(j - 1) / (double)(p->jj - 1) - 0.5;
                const double y = -(double)(i - 1) / (double)(p->ii - 1) + 0.5;
                const double y_mid = p->wind_shift + p->wind_tilt * x;
                double f;
                if (y < y_mid)
                    f = a_wind * std::sin(pi * (0.5 + y) / (0.5 + y_mid));
                else
                    f = b_wind * std::sin(pi * (y - y_mid) / (0.5 - y_mid));
                wind[(size_t)(i - 1) + (size_t)p->ii * (j - 1)] = tau * 2.0 * pi * f;
            }
    }
    return 0;
}

// The seeded synthetic initial PV of the benchmark workloads (the reference's
// own random_number IC is gfortran-specific, so the runs take this one as
// input): splitmix64 uniforms, Box-Muller normals in pairs, a separable
// Gaussian smoothing of standard deviation sigma cells truncated at 3 sigma
// and renormalised, times amplitude.  out: (ii, jj, L) sdata.
static uint64_t or_splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int or_make_ic(int ii, int jj, int L, unsigned long long seed, double amplitude, double sigma, double* out) {
    if (ii < 1 || jj < 1 || L < 1 || !out) return -1;
    const double pi = 3.14159265358979323846;
    const size_t plane = (size_t)ii * jj, total = plane * L;
    uint64_t s = seed * 0x2545F4914F6CDD1Dull + 0x1234567ull;
    std::vector<double> g(total);
    for (size_t k = 0; k < total; k += 2) {
        const double u1 = ((or_splitmix64(s) >> 11) + 1.0) * (1.0 / 9007199254740992.0);
        const double u2 = ((or_splitmix64(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        const double r = std::sqrt(-2.0 * std::log(u1));
        g[k] = r * std::cos(2.0 * pi * u2);
        if (k + 1 < total) g[k + 1] = r * std::sin(2.0 * pi * u2);
    }
    const int R = sigma > 0.0 ? (int)std::ceil(3.0 * sigma) : 0;
    std::vector<double> w(2 * R + 1, 1.0);
    if (R > 0) {
        double sum = 0.0;
        for (int q = -R; q <= R; ++q) sum += (w[q + R] = std::exp(-0.5 * (q * q) / (sigma * sigma)));
        for (double& v : w) v /= sum;
    }
    std::vector<double> row(plane);
    for (int l = 0; l < L; ++l) {
        double* f = g.data() + plane * l;
        if (R > 0) {
            for (int j = 0; j < jj; ++j)  // along i
                for (int i = 0; i < ii; ++i) {
                    double a = 0.0;
                    for (int q = -R; q <= R; ++q)
                        if (i + q >= 0 && i + q < ii) a += w[q + R] * f[(size_t)(i + q) + (size_t)ii * j];
                    row[(size_t)i + (size_t)ii * j] = a;
                }
            for (int j = 0; j < jj; ++j)  // along j
                for (int i = 0; i < ii; ++i) {
                    double a = 0.0;
                    for (int q = -R; q <= R; ++q)
                        if (j + q >= 0 && j + q < jj) a += w[q + R] * row[(size_t)i + (size_t)ii * (j + q)];
                    f[(size_t)i + (size_t)ii * j] = a;
                }
        }
        for (size_t k = 0; k < plane; ++k) out[plane * l + k] = amplitude * f[k];
    }
    return 0;
}

}  // extern "C"
