// Small dense complex linear algebra on the host (FP64) for GMRES-DR:
// the per-cycle least-squares and harmonic-Ritz eigenproblem of an m x m
// Hessenberg-sized matrix (m <= a few hundred).
//   - eig_smallest: Householder reduction to Hessenberg form, single-shift
//     complex QR iteration (Wilkinson shifts) to Schur form T = Z^H A Z,
//     eigenvectors of T by back substitution, mapped back by Z.
//   - lu_solve: Gaussian elimination with partial pivoting.
//   - orthonormalise: modified Gram-Schmidt with reorthogonalisation.
#include "dense.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace opem {

// column-major: a(i,j) = A[i + j*n]
bool lu_solve(int n, std::vector<cd> A, std::vector<cd>& b) {
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::abs(A[r + (size_t)c * n]) > std::abs(A[p + (size_t)c * n])) p = r;
        if (std::abs(A[p + (size_t)c * n]) == 0.0) return false;
        if (p != c) {
            for (int k = 0; k < n; ++k) std::swap(A[c + (size_t)k * n], A[p + (size_t)k * n]);
            std::swap(b[c], b[p]);
        }
        cd d = A[c + (size_t)c * n];
        for (int r = c + 1; r < n; ++r) {
            cd f = A[r + (size_t)c * n] / d;
            if (f == 0.0) continue;
            for (int k = c; k < n; ++k) A[r + (size_t)k * n] -= f * A[c + (size_t)k * n];
            b[r] -= f * b[c];
        }
    }
    for (int r = n - 1; r >= 0; --r) {
        cd s = b[r];
        for (int k = r + 1; k < n; ++k) s -= A[r + (size_t)k * n] * b[k];
        b[r] = s / A[r + (size_t)r * n];
    }
    return true;
}

// Givens rotation zeroing b in [a; b]: [c s; -conj(s) c] [a; b] = [r; 0]
static void givens(cd a, cd b, double& c, cd& s) {
    double aa = std::abs(a), bb = std::abs(b);
    if (bb == 0.0) { c = 1.0; s = 0.0; return; }
    if (aa == 0.0) { c = 0.0; s = std::conj(b) / bb; return; }
    double rho = std::hypot(aa, bb);
    c = aa / rho;
    s = (a / aa) * std::conj(b) / rho;
}

bool eig_smallest(int n, const std::vector<cd>& Ain, int k, std::vector<cd>& theta, std::vector<cd>& vecs) {
    std::vector<cd> H = Ain;   // column-major n x n
    std::vector<cd> Z((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Z[i + (size_t)i * n] = 1.0;
    auto h = [&](int i, int j) -> cd& { return H[i + (size_t)j * n]; };
    auto z = [&](int i, int j) -> cd& { return Z[i + (size_t)j * n]; };
    // Householder reduction to upper Hessenberg, accumulating Z
    std::vector<cd> v(n);
    for (int c = 0; c < n - 2; ++c) {
        double alpha2 = 0;
        for (int r = c + 1; r < n; ++r) alpha2 += std::norm(h(r, c));
        double an = std::sqrt(alpha2);
        if (an == 0.0) continue;
        cd x0 = h(c + 1, c);
        cd ph = std::abs(x0) > 0 ? x0 / std::abs(x0) : cd(1.0, 0.0);
        std::fill(v.begin(), v.end(), 0.0);
        for (int r = c + 1; r < n; ++r) v[r] = h(r, c);
        v[c + 1] += ph * an;
        double vn2 = 0;
        for (int r = c + 1; r < n; ++r) vn2 += std::norm(v[r]);
        if (vn2 == 0.0) continue;
        for (int j = 0; j < n; ++j) {
            cd s = 0;
            for (int r = c + 1; r < n; ++r) s += std::conj(v[r]) * h(r, j);
            s *= 2.0 / vn2;
            for (int r = c + 1; r < n; ++r) h(r, j) -= v[r] * s;
        }
        for (int i = 0; i < n; ++i) {
            cd s = 0;
            for (int r = c + 1; r < n; ++r) s += h(i, r) * v[r];
            s *= 2.0 / vn2;
            for (int r = c + 1; r < n; ++r) h(i, r) -= s * std::conj(v[r]);
        }
        for (int i = 0; i < n; ++i) {
            cd s = 0;
            for (int r = c + 1; r < n; ++r) s += z(i, r) * v[r];
            s *= 2.0 / vn2;
            for (int r = c + 1; r < n; ++r) z(i, r) -= s * std::conj(v[r]);
        }
        for (int r = c + 2; r < n; ++r) h(r, c) = 0.0;
    }
    // shifted QR iteration on the active window [lo, hi]
    const double eps = std::numeric_limits<double>::epsilon();
    int hi = n - 1, iter = 0, since = 0;
    std::vector<double> gc(n);
    std::vector<cd> gs(n);
    while (hi > 0) {
        if (++iter > 60 * n) return false;
        int lo = hi;
        while (lo > 0) {
            double sc = std::abs(h(lo, lo)) + std::abs(h(lo - 1, lo - 1));
            if (sc == 0.0) sc = 1.0;
            if (std::abs(h(lo, lo - 1)) <= eps * sc) { h(lo, lo - 1) = 0.0; break; }
            --lo;
        }
        if (lo == hi) { --hi; since = 0; continue; }
        // Wilkinson shift from the trailing 2x2 of the window
        cd a = h(hi - 1, hi - 1), b = h(hi - 1, hi), c = h(hi, hi - 1), d = h(hi, hi);
        cd tr = a + d, det = a * d - b * c;
        cd disc = std::sqrt(tr * tr / 4.0 - det);
        cd l1 = tr / 2.0 + disc, l2 = tr / 2.0 - disc;
        cd mu = std::abs(l1 - d) < std::abs(l2 - d) ? l1 : l2;
        if (++since % 11 == 0) mu = d + cd(std::abs(h(hi, hi - 1)), 0.0) * 0.75;   // exceptional shift
        for (int i = lo; i <= hi; ++i) h(i, i) -= mu;
        for (int i = lo; i < hi; ++i) {
            givens(h(i, i), h(i + 1, i), gc[i], gs[i]);
            for (int j = i; j < n; ++j) {
                cd x = h(i, j), y = h(i + 1, j);
                h(i, j) = gc[i] * x + gs[i] * y;
                h(i + 1, j) = -std::conj(gs[i]) * x + gc[i] * y;
            }
        }
        for (int i = lo; i < hi; ++i) {
            int rmax = std::min(hi, i + 2);
            for (int r = 0; r <= rmax; ++r) {
                cd x = h(r, i), y = h(r, i + 1);
                h(r, i) = gc[i] * x + std::conj(gs[i]) * y;
                h(r, i + 1) = -gs[i] * x + gc[i] * y;
            }
            for (int r = 0; r < n; ++r) {
                cd x = z(r, i), y = z(r, i + 1);
                z(r, i) = gc[i] * x + std::conj(gs[i]) * y;
                z(r, i + 1) = -gs[i] * x + gc[i] * y;
            }
        }
        for (int i = lo; i <= hi; ++i) h(i, i) += mu;
    }
    // eigenvalues on the diagonal; choose the k smallest in modulus
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a2, int b2) { return std::abs(h(a2, a2)) < std::abs(h(b2, b2)); });
    k = std::min(k, n);
    theta.resize(k);
    vecs.assign((size_t)n * k, 0.0);
    double tn = 0;
    for (int i = 0; i < n; ++i)
        for (int j = i; j < n; ++j) tn = std::max(tn, std::abs(h(i, j)));
    std::vector<cd> y(n);
    for (int q = 0; q < k; ++q) {
        int i = idx[q];
        cd lam = h(i, i);
        theta[q] = lam;
        std::fill(y.begin(), y.end(), 0.0);
        y[i] = 1.0;
        for (int r = i - 1; r >= 0; --r) {
            cd s = 0;
            for (int c2 = r + 1; c2 <= i; ++c2) s += h(r, c2) * y[c2];
            cd den = h(r, r) - lam;
            if (std::abs(den) < eps * tn) den = eps * tn;
            y[r] = -s / den;
        }
        double nrm = 0;
        for (int r = 0; r < n; ++r) {
            cd s = 0;
            for (int c2 = 0; c2 <= i; ++c2) s += z(r, c2) * y[c2];
            vecs[r + (size_t)q * n] = s;
            nrm += std::norm(s);
        }
        nrm = std::sqrt(nrm);
        for (int r = 0; r < n; ++r) vecs[r + (size_t)q * n] /= nrm;
    }
    return true;
}

int orthonormalise(int rows, int cols, std::vector<cd>& Q) {
    int rank = 0;
    for (int c = 0; c < cols; ++c) {
        cd* v = &Q[(size_t)c * rows];
        double n0 = 0;
        for (int r = 0; r < rows; ++r) n0 += std::norm(v[r]);
        n0 = std::sqrt(n0);
        for (int pass = 0; pass < 2; ++pass)
            for (int p = 0; p < c; ++p) {
                const cd* u = &Q[(size_t)p * rows];
                cd d = 0;
                for (int r = 0; r < rows; ++r) d += std::conj(u[r]) * v[r];
                for (int r = 0; r < rows; ++r) v[r] -= d * u[r];
            }
        double nr = 0;
        for (int r = 0; r < rows; ++r) nr += std::norm(v[r]);
        nr = std::sqrt(nr);
        if (nr <= 1e-14 * std::max(n0, 1e-300)) return rank;
        for (int r = 0; r < rows; ++r) v[r] /= nr;
        ++rank;
    }
    return rank;
}

void GivensLsq::reset(int m_, const std::vector<cd>& c) {
    m = m_;
    R.assign((size_t)(m + 1) * m, 0.0);
    g = c;
    g.resize(m + 1, 0.0);
    rots.clear();
}

static inline void rot_apply(const GivensLsq::Rot& q, cd& a, cd& b) {
    cd x = a, y = b;
    a = q.c * x + q.s * y;
    b = -std::conj(q.s) * x + q.c * y;
}

double GivensLsq::add_column(int j, const cd* col, int top) {
    cd* rc = &R[(size_t)j * (m + 1)];
    for (int i = 0; i <= top; ++i) rc[i] = col[i];
    for (int i = top + 1; i <= m; ++i) rc[i] = 0.0;
    for (const Rot& q : rots) rot_apply(q, rc[q.i1], rc[q.i2]);
    for (int r = j + 1; r <= top; ++r) {
        if (rc[r] == 0.0) continue;
        Rot q;
        q.i1 = j;
        q.i2 = r;
        double aa = std::abs(rc[j]), bb = std::abs(rc[r]);
        if (aa == 0.0) { q.c = 0.0; q.s = std::conj(rc[r]) / bb; }
        else { double rho = std::hypot(aa, bb); q.c = aa / rho; q.s = (rc[j] / aa) * std::conj(rc[r]) / rho; }
        rot_apply(q, rc[j], rc[r]);
        rc[r] = 0.0;
        rot_apply(q, g[j], g[r]);
        rots.push_back(q);
    }
    return std::abs(g[j + 1]);
}

void GivensLsq::solve(int k, std::vector<cd>& y) const {
    y.assign(k, 0.0);
    for (int i = k - 1; i >= 0; --i) {
        cd s = g[i];
        for (int c = i + 1; c < k; ++c) s -= R[i + (size_t)c * (m + 1)] * y[c];
        y[i] = s / R[i + (size_t)i * (m + 1)];
    }
}

bool gmres_dr_deflate(int m, int kd, const std::vector<cd>& Hh, const std::vector<cd>& c, const std::vector<cd>& y,
                      std::vector<cd>& Pm, std::vector<cd>& Hn, std::vector<cd>& cn) {
    const size_t ld = (size_t)m + 1;
    std::vector<cd> rc(m + 1);
    for (int i = 0; i <= m; ++i) {
        cd t = c[i];
        for (int j = 0; j < m; ++j) t -= Hh[i + (size_t)j * ld] * y[j];
        rc[i] = t;
    }
    // harmonic Ritz problem (H_m + |h_{m+1,m}|^2 H_m^{-H} e_m e_m^T) g = theta g
    std::vector<cd> Hm((size_t)m * m), HmH((size_t)m * m), f(m, 0.0);
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) {
            Hm[i + (size_t)j * m] = Hh[i + (size_t)j * ld];
            HmH[j + (size_t)i * m] = std::conj(Hh[i + (size_t)j * ld]);
        }
    f[m - 1] = 1.0;
    if (!lu_solve(m, HmH, f)) return false;
    double hm2 = std::norm(Hh[m + (size_t)(m - 1) * ld]);
    for (int i = 0; i < m; ++i) Hm[i + (size_t)(m - 1) * m] += hm2 * f[i];
    std::vector<cd> theta, gv;
    if (!eig_smallest(m, Hm, kd, theta, gv)) return false;
    Pm.assign(ld * (kd + 1), 0.0);
    for (int q = 0; q < kd; ++q)
        for (int i = 0; i < m; ++i) Pm[i + (size_t)q * ld] = gv[i + (size_t)q * m];
    for (int i = 0; i <= m; ++i) Pm[i + (size_t)kd * ld] = rc[i];
    if (orthonormalise(m + 1, kd + 1, Pm) != kd + 1) return false;
    std::vector<cd> T1(ld * kd, 0.0);
    for (int q = 0; q < kd; ++q)
        for (int j = 0; j < m; ++j) {
            cd pj = Pm[j + (size_t)q * ld];
            if (pj == 0.0) continue;
            for (int i = 0; i <= m; ++i) T1[i + (size_t)q * ld] += Hh[i + (size_t)j * ld] * pj;
        }
    Hn.assign(ld * m, 0.0);
    cn.assign(m + 1, 0.0);
    for (int q = 0; q < kd; ++q)
        for (int a = 0; a <= kd; ++a) {
            cd t = 0;
            for (int i = 0; i <= m; ++i) t += std::conj(Pm[i + (size_t)a * ld]) * T1[i + (size_t)q * ld];
            Hn[a + (size_t)q * ld] = t;
        }
    for (int a = 0; a <= kd; ++a) {
        cd t = 0;
        for (int i = 0; i <= m; ++i) t += std::conj(Pm[i + (size_t)a * ld]) * rc[i];
        cn[a] = t;
    }
    return true;
}

}  // namespace opem
