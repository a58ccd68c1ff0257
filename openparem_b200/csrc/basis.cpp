// Order-p Nedelec (first kind) basis on the reference tetrahedron.
//
// Space: ND_p = P_{p-1}^3 + x cross P~_{p-1}^3, the space of MFEM's
// ND_FECollection(p,3) used by the reference (src/OpenParEM3D/fem3D.cpp:65-66).
// Basis: dual to moment functionals on the reference tetrahedron with
// vertices v0=(0,0,0), v1=(1,0,0), v2=(0,1,0), v3=(0,0,1), which is the
// element's vertices sorted by global index:
//   edge (a,b):   int_0^1 u(v_a+s t).t P_k(2s-1) ds,            t=v_b-v_a, k<p
//   face (a,b,c): int_{unit tri} u.t_m q_r(s1,s2) ds1 ds2,       t1=v_b-v_a, t2=v_c-v_a
//   interior:     int_T u_d w_r(x) dx,                             d=x,y,z
// with q_r / w_r the degree-ordered monomials orthonormalised by the
// Cholesky factor of their exact Gram matrix.  A shared edge or face is
// parameterised from its lowest global vertex by every element touching it,
// so the assembled space is H(curl)-conforming with no sign flips.
#include "opem_internal.h"
#include "../../include/opem_b200.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>

namespace opem {

static const int EDGES[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
static const int FACES[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
static const double VERTS[4][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

double shifted_legendre(int k, double s) {
    double x = 2.0 * s - 1.0;
    if (k == 0) return 1.0;
    double p0 = 1.0, p1 = x;
    for (int n = 1; n < k; ++n) {
        double p2 = ((2.0 * n + 1.0) * x * p1 - n * p0) / (n + 1.0);
        p0 = p1;
        p1 = p2;
    }
    return p1;
}

// Legendre P_n(z) and P_{n-1}(z) by the three-term recurrence.
static void legendre_pair(int n, double z, double& pn, double& pnm1) {
    double p0 = 1.0, p1 = z;
    if (n == 0) { pn = 1.0; pnm1 = 0.0; return; }
    for (int k = 1; k < n; ++k) {
        double p2 = ((2.0 * k + 1.0) * z * p1 - k * p0) / (k + 1.0);
        p0 = p1;
        p1 = p2;
    }
    pn = p1;
    pnm1 = p0;
}

void gauss_legendre01(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));   // Newton from the asymptotic root
        double pn, pnm1, dp;
        for (int it = 0; it < 100; ++it) {
            legendre_pair(n, z, pn, pnm1);
            dp = n * (z * pn - pnm1) / (z * z - 1.0);
            double dz = pn / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        legendre_pair(n, z, pn, pnm1);
        dp = n * (z * pn - pnm1) / (z * z - 1.0);
        x[i] = 0.5 * (1.0 - z);
        w[i] = 1.0 / ((1.0 - z * z) * dp * dp);   // half of 2/((1-z^2) P_n'(z)^2)
    }
}

void tri_rule(int deg, std::vector<double>& s1, std::vector<double>& s2, std::vector<double>& w) {
    // s1 = u, s2 = (1-u) v, jacobian (1-u); Gauss-Legendre exact for deg+1 in u
    int n = (deg + 2) / 2 + 1;
    std::vector<double> x, wx;
    gauss_legendre01(n, x, wx);
    s1.clear(); s2.clear(); w.clear();
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            s1.push_back(x[i]);
            s2.push_back((1.0 - x[i]) * x[j]);
            w.push_back(wx[i] * wx[j] * (1.0 - x[i]));
        }
}

// The rule the reference's port integrals amount to: a product of fields
// interpolated at the nodes of MFEM 4.8's order-p L2 triangle (Gauss-Legendre
// basis: the nodes (o_i, o_j) / (o_i + o_j + o_{p-i-j}), i + j <= p, o the p + 1
// Gauss-Legendre points on [0, 1]) and the interpolant integrated exactly; the
// weights are the integrals of the degree-p Lagrange polynomials on the nodes
// (tangentialInnerProduct, src/OpenParEM3D/port.cpp:3463-3490; Fields::calculatePz,
// src/OpenParEM2D/fem2D.cpp:395-480, at order p - 1).  Weights sum to 1/2.
void l2_nodal_rule(int p, std::vector<double>& s1, std::vector<double>& s2, std::vector<double>& w) {
    std::vector<double> o, ow;
    gauss_legendre01(p + 1, o, ow);
    std::sort(o.begin(), o.end());
    s1.clear(); s2.clear();
    for (int j = 0; j <= p; ++j)
        for (int i = 0; i + j <= p; ++i) {
            const double d = o[i] + o[j] + o[p - i - j];
            s1.push_back(o[i] / d);
            s2.push_back(o[j] / d);
        }
    // V^T w = moments, V[node][monomial s1^a s2^b], moments a! b! / (a + b + 2)!
    const int n = (int)s1.size();
    std::vector<int> ma, mb;
    for (int a = 0; a <= p; ++a)
        for (int b = 0; a + b <= p; ++b) { ma.push_back(a); mb.push_back(b); }
    auto fact = [](int k) { double f = 1; for (int i = 2; i <= k; ++i) f *= i; return f; };
    std::vector<double> A((size_t)n * (n + 1));   // row m: V[.][m] | moment m
    for (int m = 0; m < n; ++m) {
        for (int q = 0; q < n; ++q) A[(size_t)m * (n + 1) + q] = std::pow(s1[q], ma[m]) * std::pow(s2[q], mb[m]);
        A[(size_t)m * (n + 1) + n] = fact(ma[m]) * fact(mb[m]) / fact(ma[m] + mb[m] + 2);
    }
    for (int c = 0; c < n; ++c) {   // Gaussian elimination, partial pivoting
        int pr = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[(size_t)r * (n + 1) + c]) > std::fabs(A[(size_t)pr * (n + 1) + c])) pr = r;
        if (pr != c)
            for (int k = 0; k <= n; ++k) std::swap(A[(size_t)pr * (n + 1) + k], A[(size_t)c * (n + 1) + k]);
        for (int r = c + 1; r < n; ++r) {
            const double f = A[(size_t)r * (n + 1) + c] / A[(size_t)c * (n + 1) + c];
            for (int k = c; k <= n; ++k) A[(size_t)r * (n + 1) + k] -= f * A[(size_t)c * (n + 1) + k];
        }
    }
    w.assign(n, 0.0);
    for (int r = n - 1; r >= 0; --r) {
        double s = A[(size_t)r * (n + 1) + n];
        for (int k = r + 1; k < n; ++k) s -= A[(size_t)r * (n + 1) + k] * w[k];
        w[r] = s / A[(size_t)r * (n + 1) + r];
    }
}

static void tet_rule(int deg, std::vector<double>& X, std::vector<double>& w) {
    // x = u, y = (1-u) v, z = (1-u)(1-v) t ; jacobian (1-u)^2 (1-v)
    int n = (deg + 3) / 2 + 1;
    std::vector<double> g, gw;
    gauss_legendre01(n, g, gw);
    X.clear(); w.clear();
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                double u = g[i], v = g[j], t = g[k];
                X.push_back(u);
                X.push_back((1 - u) * v);
                X.push_back((1 - u) * (1 - v) * t);
                w.push_back(gw[i] * gw[j] * gw[k] * (1 - u) * (1 - u) * (1 - v));
            }
}

static void monomials3(int P, std::vector<int>& E) {
    E.clear();
    for (int d = 0; d <= P; ++d)
        for (int a = d; a >= 0; --a)
            for (int b = d - a; b >= 0; --b) {
                E.push_back(a); E.push_back(b); E.push_back(d - a - b);
            }
}

static double fact(int n) {
    double r = 1;
    for (int i = 2; i <= n; ++i) r *= i;
    return r;
}

// Cholesky G = L L^T, returns L^{-1} (row-major n x n)
static std::vector<double> chol_inv(std::vector<double> G, int n) {
    std::vector<double> L(n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        double s = G[j * n + j];
        for (int k = 0; k < j; ++k) s -= L[j * n + k] * L[j * n + k];
        if (s <= 0) throw std::runtime_error("test-polynomial Gram matrix not positive definite");
        L[j * n + j] = std::sqrt(s);
        for (int i = j + 1; i < n; ++i) {
            double t = G[i * n + j];
            for (int k = 0; k < j; ++k) t -= L[i * n + k] * L[j * n + k];
            L[i * n + j] = t / L[j * n + j];
        }
    }
    std::vector<double> Li(n * n, 0.0);
    for (int c = 0; c < n; ++c) {
        for (int i = 0; i < n; ++i) {
            double t = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) t -= L[i * n + k] * Li[k * n + c];
            Li[i * n + c] = t / L[i * n + i];
        }
    }
    return Li;
}

std::vector<double> tri_test_polys(int P, std::vector<int>& mon2) {
    mon2.clear();
    for (int d = 0; d <= P; ++d)
        for (int i = d; i >= 0; --i) { mon2.push_back(i); mon2.push_back(d - i); }
    int n = (int)mon2.size() / 2;
    std::vector<double> G(n * n);
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
            int i = mon2[2 * a] + mon2[2 * b], j = mon2[2 * a + 1] + mon2[2 * b + 1];
            G[a * n + b] = fact(i) * fact(j) / fact(i + j + 2);
        }
    return chol_inv(G, n);
}

static std::vector<double> tet_test_polys(int P, std::vector<int>& mon3) {
    monomials3(P, mon3);
    int n = (int)mon3.size() / 3;
    std::vector<double> G(n * n);
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
            int i = mon3[3 * a] + mon3[3 * b], j = mon3[3 * a + 1] + mon3[3 * b + 1],
                k = mon3[3 * a + 2] + mon3[3 * b + 2];
            G[a * n + b] = fact(i) * fact(j) * fact(k) / fact(i + j + k + 3);
        }
    return chol_inv(G, n);
}

namespace {

struct PolyCtx {
    int P, nm;
    std::vector<int> E;
    std::map<long, int> idx;
    long key(int a, int b, int c) const { return (long)a * 10000 + b * 100 + c; }
    void init(int P_) {
        P = P_;
        monomials3(P, E);
        nm = (int)E.size() / 3;
        for (int m = 0; m < nm; ++m) idx[key(E[3 * m], E[3 * m + 1], E[3 * m + 2])] = m;
    }
    void vander(const double* x, double* V) const {
        for (int m = 0; m < nm; ++m)
            V[m] = std::pow(x[0], E[3 * m]) * std::pow(x[1], E[3 * m + 1]) * std::pow(x[2], E[3 * m + 2]);
    }
};

// evaluate vector polynomial coefficient block c (3*nm) at V
inline void evalv(const double* c, const double* V, int nm, double* out) {
    for (int d = 0; d < 3; ++d) {
        double s = 0;
        for (int m = 0; m < nm; ++m) s += c[d * nm + m] * V[m];
        out[d] = s;
    }
}

}  // namespace

static std::unique_ptr<NDRef> build_ref(int p) {
    if (p < 1 || p > 6) throw std::runtime_error("Nedelec order out of range");
    auto R = std::make_unique<NDRef>();
    R->p = p;
    int ld = 6 * p + 4 * p * (p - 1) + p * (p - 1) * (p - 2) / 2;
    R->ld = ld;
    R->ldf = 3 * p + p * (p - 1);
    PolyCtx C;
    C.init(p);
    int nm = C.nm;
    R->nmon = nm;
    R->mon = C.E;
    int dim = 3 * nm;

    // ---- spanning set of ND_p, orthonormalised by MGS with reorthogonalisation
    std::vector<std::vector<double>> span;
    for (int m = 0; m < nm; ++m) {
        int deg = C.E[3 * m] + C.E[3 * m + 1] + C.E[3 * m + 2];
        if (deg <= p - 1)
            for (int c = 0; c < 3; ++c) {
                std::vector<double> v(dim, 0.0);
                v[c * nm + m] = 1.0;
                span.push_back(v);
            }
    }
    for (int m = 0; m < nm; ++m) {
        int e[3] = {C.E[3 * m], C.E[3 * m + 1], C.E[3 * m + 2]};
        if (e[0] + e[1] + e[2] != p - 1) continue;
        for (int c = 0; c < 3; ++c) {
            // x cross (e_c m): component r = sum_s eps(r,s,c) x_s m
            std::vector<double> v(dim, 0.0);
            for (int r = 0; r < 3; ++r)
                for (int s = 0; s < 3; ++s) {
                    if (r == s || r == c || s == c) continue;
                    int eps = ((r + 1) % 3 == s) ? 1 : -1;   // (r,s,c) cyclic -> +1
                    int f[3] = {e[0], e[1], e[2]};
                    f[s] += 1;
                    v[r * nm + C.idx[C.key(f[0], f[1], f[2])]] += eps;
                }
            span.push_back(v);
        }
    }
    std::vector<std::vector<double>> Q;
    for (auto& v : span) {
        double n0 = 0;
        for (double t : v) n0 += t * t;
        n0 = std::sqrt(n0);
        for (int pass = 0; pass < 2; ++pass)
            for (auto& q : Q) {
                double d = 0;
                for (int i = 0; i < dim; ++i) d += q[i] * v[i];
                for (int i = 0; i < dim; ++i) v[i] -= d * q[i];
            }
        double nr = 0;
        for (double t : v) nr += t * t;
        nr = std::sqrt(nr);
        if (nr > 1e-9 * n0) {
            for (double& t : v) t /= nr;
            Q.push_back(v);
        }
    }
    if ((int)Q.size() != ld) throw std::runtime_error("ND_p spanning set has wrong rank");

    // ---- moment functionals W (ld x dim)
    std::vector<std::vector<double>> W;
    std::vector<double> V(nm);
    {
        std::vector<double> s, ws;
        gauss_legendre01(p + 2, s, ws);
        for (int e = 0; e < 6; ++e) {
            const double* va = VERTS[EDGES[e][0]];
            const double* vb = VERTS[EDGES[e][1]];
            double t[3] = {vb[0] - va[0], vb[1] - va[1], vb[2] - va[2]};
            for (int k = 0; k < p; ++k) {
                std::vector<double> w(dim, 0.0);
                for (size_t q = 0; q < s.size(); ++q) {
                    double x[3] = {va[0] + s[q] * t[0], va[1] + s[q] * t[1], va[2] + s[q] * t[2]};
                    C.vander(x, V.data());
                    double f = ws[q] * shifted_legendre(k, s[q]);
                    for (int d = 0; d < 3; ++d)
                        for (int m = 0; m < nm; ++m) w[d * nm + m] += f * t[d] * V[m];
                }
                W.push_back(w);
            }
        }
    }
    if (p >= 2) {
        std::vector<int> mon2;
        std::vector<double> T2 = tri_test_polys(p - 2, mon2);
        int nq2 = (int)mon2.size() / 2;
        std::vector<double> s1, s2, wq;
        tri_rule(2 * p + 2, s1, s2, wq);
        for (int f = 0; f < 4; ++f) {
            const double* va = VERTS[FACES[f][0]];
            const double* vb = VERTS[FACES[f][1]];
            const double* vc = VERTS[FACES[f][2]];
            double t1[3], t2[3];
            for (int d = 0; d < 3; ++d) { t1[d] = vb[d] - va[d]; t2[d] = vc[d] - va[d]; }
            for (int r = 0; r < nq2; ++r)
                for (int tm = 0; tm < 2; ++tm) {
                    const double* t = tm ? t2 : t1;
                    std::vector<double> w(dim, 0.0);
                    for (size_t q = 0; q < wq.size(); ++q) {
                        double x[3];
                        for (int d = 0; d < 3; ++d) x[d] = va[d] + s1[q] * t1[d] + s2[q] * t2[d];
                        C.vander(x, V.data());
                        double qv = 0;
                        for (int c = 0; c < nq2; ++c)
                            qv += T2[r * nq2 + c] * std::pow(s1[q], mon2[2 * c]) * std::pow(s2[q], mon2[2 * c + 1]);
                        double f0 = wq[q] * qv;
                        for (int d = 0; d < 3; ++d)
                            for (int m = 0; m < nm; ++m) w[d * nm + m] += f0 * t[d] * V[m];
                    }
                    W.push_back(w);
                }
        }
    }
    if (p >= 3) {
        std::vector<int> mon3;
        std::vector<double> T3 = tet_test_polys(p - 3, mon3);
        int nq3 = (int)mon3.size() / 3;
        std::vector<double> X, wq;
        tet_rule(2 * p + 2, X, wq);
        for (int r = 0; r < nq3; ++r)
            for (int d = 0; d < 3; ++d) {
                std::vector<double> w(dim, 0.0);
                for (size_t q = 0; q < wq.size(); ++q) {
                    const double* x = &X[3 * q];
                    C.vander(x, V.data());
                    double qv = 0;
                    for (int c = 0; c < nq3; ++c)
                        qv += T3[r * nq3 + c] * std::pow(x[0], mon3[3 * c]) * std::pow(x[1], mon3[3 * c + 1]) *
                              std::pow(x[2], mon3[3 * c + 2]);
                    for (int m = 0; m < nm; ++m) w[d * nm + m] += wq[q] * qv * V[m];
                }
                W.push_back(w);
            }
    }
    if ((int)W.size() != ld) throw std::runtime_error("functional count mismatch");

    // ---- D_ij = l_i(q_j); phi_k = sum_j Cc[k][j] q_j with D Cc^T = I
    std::vector<double> D(ld * ld);
    for (int i = 0; i < ld; ++i)
        for (int j = 0; j < ld; ++j) {
            double s = 0;
            for (int t = 0; t < dim; ++t) s += W[i][t] * Q[j][t];
            D[i * ld + j] = s;
        }
    // invert D by Gauss-Jordan with partial pivoting
    std::vector<double> Inv(ld * ld, 0.0);
    for (int i = 0; i < ld; ++i) Inv[i * ld + i] = 1.0;
    for (int c = 0; c < ld; ++c) {
        int piv = c;
        for (int r = c + 1; r < ld; ++r)
            if (std::fabs(D[r * ld + c]) > std::fabs(D[piv * ld + c])) piv = r;
        if (std::fabs(D[piv * ld + c]) < 1e-300) throw std::runtime_error("singular DOF matrix");
        if (piv != c)
            for (int k = 0; k < ld; ++k) {
                std::swap(D[c * ld + k], D[piv * ld + k]);
                std::swap(Inv[c * ld + k], Inv[piv * ld + k]);
            }
        double d = 1.0 / D[c * ld + c];
        for (int k = 0; k < ld; ++k) { D[c * ld + k] *= d; Inv[c * ld + k] *= d; }
        for (int r = 0; r < ld; ++r) {
            if (r == c) continue;
            double f = D[r * ld + c];
            if (f == 0.0) continue;
            for (int k = 0; k < ld; ++k) { D[r * ld + k] -= f * D[c * ld + k]; Inv[r * ld + k] -= f * Inv[c * ld + k]; }
        }
    }
    // Cc = Inv^T  -> coef[k] = sum_j Inv[j][k] Q_j
    R->coef.assign((size_t)ld * dim, 0.0);
    for (int k = 0; k < ld; ++k)
        for (int j = 0; j < ld; ++j) {
            double c = Inv[j * ld + k];
            for (int t = 0; t < dim; ++t) R->coef[(size_t)k * dim + t] += c * Q[j][t];
        }
    // curl coefficients: curl u = (dy uz - dz uy, dz ux - dx uz, dx uy - dy ux)
    std::vector<double> curl((size_t)ld * dim, 0.0);
    auto dcoef = [&](const double* c, int dir, double* out) {
        for (int m = 0; m < nm; ++m) out[m] = 0;
        for (int m = 0; m < nm; ++m) {
            int e[3] = {C.E[3 * m], C.E[3 * m + 1], C.E[3 * m + 2]};
            if (e[dir] == 0 || c[m] == 0.0) continue;
            int f[3] = {e[0], e[1], e[2]};
            f[dir] -= 1;
            out[C.idx[C.key(f[0], f[1], f[2])]] += e[dir] * c[m];
        }
    };
    std::vector<double> a(nm), b(nm);
    for (int k = 0; k < ld; ++k) {
        const double* u = &R->coef[(size_t)k * dim];
        double* cu = &curl[(size_t)k * dim];
        dcoef(u + 2 * nm, 1, a.data()); dcoef(u + 1 * nm, 2, b.data());
        for (int m = 0; m < nm; ++m) cu[0 * nm + m] = a[m] - b[m];
        dcoef(u + 0 * nm, 2, a.data()); dcoef(u + 2 * nm, 0, b.data());
        for (int m = 0; m < nm; ++m) cu[1 * nm + m] = a[m] - b[m];
        dcoef(u + 1 * nm, 0, a.data()); dcoef(u + 0 * nm, 1, b.data());
        for (int m = 0; m < nm; ++m) cu[2 * nm + m] = a[m] - b[m];
    }

    // ---- reference tensors
    std::vector<double> X, wq;
    tet_rule(2 * p + 1, X, wq);
    int nq = (int)wq.size();
    std::vector<double> PV((size_t)ld * nq * 3), CV((size_t)ld * nq * 3);
    for (int q = 0; q < nq; ++q) {
        C.vander(&X[3 * q], V.data());
        for (int k = 0; k < ld; ++k) {
            evalv(&R->coef[(size_t)k * dim], V.data(), nm, &PV[((size_t)k * nq + q) * 3]);
            evalv(&curl[(size_t)k * dim], V.data(), nm, &CV[((size_t)k * nq + q) * 3]);
        }
    }
    {   // tables for the error indicator (degree 2p+2 rule)
        std::vector<double> Xe, we;
        tet_rule(2 * p + 2, Xe, we);
        const int nqe = (int)we.size();
        R->nq_err = nqe;
        R->w_err = we;
        R->phi_err.assign((size_t)nqe * ld * 3, 0.0);
        R->curl_err.assign((size_t)nqe * ld * 3, 0.0);
        for (int q = 0; q < nqe; ++q) {
            C.vander(&Xe[3 * q], V.data());
            for (int k = 0; k < ld; ++k) {
                evalv(&R->coef[(size_t)k * dim], V.data(), nm, &R->phi_err[((size_t)q * ld + k) * 3]);
                evalv(&curl[(size_t)k * dim], V.data(), nm, &R->curl_err[((size_t)q * ld + k) * 3]);
            }
        }
    }
    static const int SA[6] = {0, 1, 2, 0, 0, 1}, SB[6] = {0, 1, 2, 1, 2, 2};
    R->Mh.assign((size_t)6 * ld * ld, 0.0);
    R->Kh.assign((size_t)6 * ld * ld, 0.0);
    R->Qh.assign((size_t)ld * ld, 0.0);
    for (int i = 0; i < ld; ++i)
        for (int j = 0; j < ld; ++j) {
            double m9[3][3] = {{0}}, k9[3][3] = {{0}}, qv = 0;
            for (int q = 0; q < nq; ++q) {
                const double* pi = &PV[((size_t)i * nq + q) * 3];
                const double* pj = &PV[((size_t)j * nq + q) * 3];
                const double* ci = &CV[((size_t)i * nq + q) * 3];
                const double* cj = &CV[((size_t)j * nq + q) * 3];
                for (int x = 0; x < 3; ++x)
                    for (int y = 0; y < 3; ++y) {
                        m9[x][y] += wq[q] * pi[x] * pj[y];
                        k9[x][y] += wq[q] * ci[x] * cj[y];
                    }
                qv += wq[q] * (pi[0] * cj[0] + pi[1] * cj[1] + pi[2] * cj[2]);
            }
            for (int s = 0; s < 6; ++s) {
                int x = SA[s], y = SB[s];
                double mv = (x == y) ? m9[x][x] : m9[x][y] + m9[y][x];
                double kv = (x == y) ? k9[x][x] : k9[x][y] + k9[y][x];
                R->Mh[((size_t)s * ld + i) * ld + j] = mv;
                R->Kh[((size_t)s * ld + i) * ld + j] = kv;
            }
            R->Qh[(size_t)i * ld + j] = qv;
        }

    // ---- face tables (exact, and with the port integrals' nodal rule: Wh)
    int ldf = R->ldf;
    std::vector<double> s1, s2, wt, n1, n2, nw;
    tri_rule(2 * p + 1, s1, s2, wt);
    l2_nodal_rule(p, n1, n2, nw);
    static const int FE[4][3] = {{0, 1, 3}, {0, 2, 4}, {1, 2, 5}, {3, 4, 5}};   // (ab, ac, bc) edges
    for (int f = 0; f < 4; ++f) {
        std::vector<int>& fd = R->face_dofs[f];
        fd.clear();
        for (int e = 0; e < 3; ++e)
            for (int k = 0; k < p; ++k) fd.push_back(FE[f][e] * p + k);
        int nfd = p * (p - 1);
        for (int k = 0; k < nfd; ++k) fd.push_back(6 * p + f * nfd + k);
        const double* va = VERTS[FACES[f][0]];
        const double* vb = VERTS[FACES[f][1]];
        const double* vc = VERTS[FACES[f][2]];
        double t1[3], t2[3], N[3];
        for (int d = 0; d < 3; ++d) { t1[d] = vb[d] - va[d]; t2[d] = vc[d] - va[d]; }
        N[0] = t1[1] * t2[2] - t1[2] * t2[1];
        N[1] = t1[2] * t2[0] - t1[0] * t2[2];
        N[2] = t1[0] * t2[1] - t1[1] * t2[0];
        int nqf = (int)wt.size();
        std::vector<double> P1((size_t)ldf * nqf), P2((size_t)ldf * nqf), CN((size_t)ldf * nqf);
        for (int q = 0; q < nqf; ++q) {
            double x[3];
            for (int d = 0; d < 3; ++d) x[d] = va[d] + s1[q] * t1[d] + s2[q] * t2[d];
            C.vander(x, V.data());
            for (int a2 = 0; a2 < ldf; ++a2) {
                double u[3], cu[3];
                evalv(&R->coef[(size_t)fd[a2] * dim], V.data(), nm, u);
                evalv(&curl[(size_t)fd[a2] * dim], V.data(), nm, cu);
                P1[(size_t)a2 * nqf + q] = u[0] * t1[0] + u[1] * t1[1] + u[2] * t1[2];
                P2[(size_t)a2 * nqf + q] = u[0] * t2[0] + u[1] * t2[1] + u[2] * t2[2];
                CN[(size_t)a2 * nqf + q] = cu[0] * N[0] + cu[1] * N[1] + cu[2] * N[2];
            }
        }
        R->Fh[f].assign((size_t)3 * ldf * ldf, 0.0);
        R->Ch[f].assign((size_t)ldf * ldf, 0.0);
        for (int i = 0; i < ldf; ++i)
            for (int j = 0; j < ldf; ++j) {
                double f11 = 0, f22 = 0, f12 = 0, cc = 0;
                for (int q = 0; q < nqf; ++q) {
                    double w = wt[q];
                    f11 += w * P1[(size_t)i * nqf + q] * P1[(size_t)j * nqf + q];
                    f22 += w * P2[(size_t)i * nqf + q] * P2[(size_t)j * nqf + q];
                    f12 += w * (P1[(size_t)i * nqf + q] * P2[(size_t)j * nqf + q] +
                                P2[(size_t)i * nqf + q] * P1[(size_t)j * nqf + q]);
                    cc += w * CN[(size_t)i * nqf + q] * CN[(size_t)j * nqf + q];
                }
                R->Fh[f][((size_t)0 * ldf + i) * ldf + j] = f11;
                R->Fh[f][((size_t)1 * ldf + i) * ldf + j] = f22;
                R->Fh[f][((size_t)2 * ldf + i) * ldf + j] = f12;
                R->Ch[f][(size_t)i * ldf + j] = cc;
            }
        // the same tangential tables with the nodal rule
        const int nqn = (int)nw.size();
        std::vector<double> W1((size_t)ldf * nqn), W2((size_t)ldf * nqn);
        for (int q = 0; q < nqn; ++q) {
            double x[3];
            for (int d = 0; d < 3; ++d) x[d] = va[d] + n1[q] * t1[d] + n2[q] * t2[d];
            C.vander(x, V.data());
            for (int a2 = 0; a2 < ldf; ++a2) {
                double u[3];
                evalv(&R->coef[(size_t)fd[a2] * dim], V.data(), nm, u);
                W1[(size_t)a2 * nqn + q] = u[0] * t1[0] + u[1] * t1[1] + u[2] * t1[2];
                W2[(size_t)a2 * nqn + q] = u[0] * t2[0] + u[1] * t2[1] + u[2] * t2[2];
            }
        }
        R->Wh[f].assign((size_t)3 * ldf * ldf, 0.0);
        for (int i = 0; i < ldf; ++i)
            for (int j = 0; j < ldf; ++j) {
                double f11 = 0, f22 = 0, f12 = 0;
                for (int q = 0; q < nqn; ++q) {
                    const double w = nw[q];
                    const double a1 = W1[(size_t)i * nqn + q], a2 = W2[(size_t)i * nqn + q];
                    const double b1 = W1[(size_t)j * nqn + q], b2 = W2[(size_t)j * nqn + q];
                    f11 += w * a1 * b1;
                    f22 += w * a2 * b2;
                    f12 += w * (a1 * b2 + a2 * b1);
                }
                R->Wh[f][((size_t)0 * ldf + i) * ldf + j] = f11;
                R->Wh[f][((size_t)1 * ldf + i) * ldf + j] = f22;
                R->Wh[f][((size_t)2 * ldf + i) * ldf + j] = f12;
            }
    }
    return R;
}

const NDRef& nd_reference(int p) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<NDRef>> cache;
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(p);
    if (it != cache.end()) return *it->second;
    auto r = build_ref(p);
    const NDRef& ref = *r;
    cache[p] = std::move(r);
    return ref;
}

}  // namespace opem

extern "C" int opem_selftest_face_tables(int p, int nodal, double* out, int64_t nout) {
    if (p < 1 || p > 8 || !out) return OPEM_ERR_ARG;
    try {
        const opem::NDRef& R = opem::nd_reference(p);
        const size_t L = (size_t)3 * R.ldf * R.ldf;
        if (nout < (int64_t)(4 * L)) return OPEM_ERR_ARG;
        for (int f = 0; f < 4; ++f) {
            const std::vector<double>& src = nodal ? R.Wh[f] : R.Fh[f];
            std::copy(src.begin(), src.end(), out + f * L);
        }
    } catch (const std::exception&) {
        return OPEM_ERR_ARG;
    }
    return OPEM_OK;
}
