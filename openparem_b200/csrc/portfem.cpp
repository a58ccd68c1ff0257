// Port modes solved on the port's own faces (host).
//
// The reference drives every port with the mode its 2D solver finds on the
// port's cross-section: OpenParEM3D writes the port faces out as a 2D mesh,
// spawns OpenParEM2D (src/OpenParEM3D/port.cpp:5081-5176), reads back the modal
// fields and metrics (load_modeMetrics, port.cpp:5302-5453) and interpolates the
// fields onto the 3D port trace (Mode::fillX, port.cpp:3234-3341).  Here the
// chain runs in-process:
//   * the 2D mesh is a conforming split of the port faces, each into nsub x nsub
//     similar triangles, with each sub-triangle's material taken from the
//     tetrahedron that owns its face;
//   * the fundamental mode comes from opem_port_mode_2d (lowest-order edge
//     elements for e_t, linear nodal e_z, PEC on the outer boundary),
//     gamma = j beta;
//   * for propagation along the outward normal n (the convention of the
//     analytic TE modes) H_t = n x (gamma e_t + grad_t e_z) / (j w mu);
//   * V = -int E . dl along the voltage path (composite 4-point Gauss on
//     16 nsub pieces), Pz = 1/2 int (E x H*) . n (edge-midpoint rule, exact for
//     the piecewise-quadratic integrand), and along the current path, where one
//     is given, I = int H . dl (the same Gauss rule per segment);
//   * Z by the port's impedance definition (OpenParEM2D Mode::calculateImpedance,
//     fem2D.cpp:1803-1824): PV V V* / (2 Pz*), VI V / I, PI 2 Pz / (I I*).
// On unsplit port faces (and at orders above 2, and for higher modes) the mode
// is solved with the order-p elements of RefSpaces2D, so it lies in the 3D trace
// space, and the chain follows the reference's 2D solver further: H_t is the
// mu-weighted L2 projection of the expression above onto the edge space (Hsolve,
// src/OpenParEM2D/Hsolve.c:454-560) and Pz integrates E_t x H_t* interpolated on
// the order-(p-1) L2 triangle (Fields::calculatePz, fem2D.cpp:395-480); the 3D
// overlaps of such a port use the order-p nodal rule (assemble.cu).
// The 3D port trace is then the moment interpolation of this field on each
// port face (engine.cu port_traces), as for the analytic modes.
#include "portfem.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>

#include "../../include/opem_b200.h"
#include "opem_internal.h"

namespace opem {

namespace {
using cd = std::complex<double>;
constexpr double MU0 = 4e-7 * M_PI;
const int LP[3][2] = {{0, 1}, {0, 2}, {1, 2}};

void unit(const double* a, double* out) {
    const double s = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (int i = 0; i < 3; ++i) out[i] = a[i] / s;
}

// n x (gx u + gy v) for complex plane components
void n_cross_plane(const double n[3], const double u[3], const double v[3], cd gx, cd gy, cd out[3]) {
    cd w[3];
    for (int i = 0; i < 3; ++i) w[i] = gx * u[i] + gy * v[i];
    out[0] = n[1] * w[2] - n[2] * w[1];
    out[1] = n[2] * w[0] - n[0] * w[2];
    out[2] = n[0] * w[1] - n[1] * w[0];
}
}  // namespace

void PortFem2D::eval_tri(int64_t t, const double X[3], cd E[3], cd Hy[3]) const {
    const double d0 = (X[0] - o[0]) * u[0] + (X[1] - o[1]) * u[1] + (X[2] - o[2]) * u[2] - P0[2 * t];
    const double d1 = (X[0] - o[0]) * v[0] + (X[1] - o[1]) * v[1] + (X[2] - o[2]) * v[2] - P0[2 * t + 1];
    const double* Ji = &Jinv[4 * t];
    const double l1 = Ji[0] * d0 + Ji[1] * d1, l2 = Ji[2] * d0 + Ji[3] * d1;
    const double lam[3] = {1 - l1 - l2, l1, l2};
    const double* gg = &g[6 * t];
    cd ex = 0.0, ey = 0.0, zx, zy;
    if (ref) {   // order-p path: unsplit faces, order >= 3, or a higher mode
        // reference bases at (l1, l2), covariant map J^-T (J^-1 = Ji row-major)
        const int nf = ref->nf, nl = ref->nl;
        std::vector<double> N(2 * nf), cu(nf), L(nl), gL(2 * nl);
        ref->nd(l1, l2, N.data(), cu.data());
        ref->h1(l1, l2, L.data(), gL.data());
        cd rx = 0.0, ry = 0.0, gx = 0.0, gy = 0.0;
        const cd* c = &ct[(size_t)nf * t];
        for (int i = 0; i < nf; ++i) { rx += c[i] * N[2 * i]; ry += c[i] * N[2 * i + 1]; }
        if (!ch.empty()) {   // H_t / y from its projection onto the edge space
            cd hx = 0.0, hy = 0.0;
            const cd* h = &ch[(size_t)nf * t];
            for (int i = 0; i < nf; ++i) { hx += h[i] * N[2 * i]; hy += h[i] * N[2 * i + 1]; }
            ex = Ji[0] * rx + Ji[2] * ry;
            ey = Ji[1] * rx + Ji[3] * ry;
            const cd px = Ji[0] * hx + Ji[2] * hy, py = Ji[1] * hx + Ji[3] * hy;
            for (int i = 0; i < 3; ++i) {
                E[i] = ex * u[i] + ey * v[i];
                Hy[i] = px * u[i] + py * v[i];
            }
            return;
        }
        const cd* z = &cz[(size_t)nl * t];
        for (int i = 0; i < nl; ++i) { gx += z[i] * gL[2 * i]; gy += z[i] * gL[2 * i + 1]; }
        ex = Ji[0] * rx + Ji[2] * ry;
        ey = Ji[1] * rx + Ji[3] * ry;
        zx = Ji[0] * gx + Ji[2] * gy;
        zy = Ji[1] * gx + Ji[3] * gy;
    } else if (order == 2) {
        // W_ab, G_ab = grad(l_a l_b) per edge, then l_2 W_01 and l_0 W_12; e_z quadratic
        zx = 0.0;
        zy = 0.0;
        for (int i = 0; i < 3; ++i) {
            const int a = LP[i][0], b = LP[i][1];
            const double wx = lam[a] * gg[2 * b] - lam[b] * gg[2 * a];
            const double wy = lam[a] * gg[2 * b + 1] - lam[b] * gg[2 * a + 1];
            const double gx = lam[a] * gg[2 * b] + lam[b] * gg[2 * a];
            const double gy = lam[a] * gg[2 * b + 1] + lam[b] * gg[2 * a + 1];
            ex += ct[8 * t + i] * wx + ct[8 * t + 3 + i] * gx;
            ey += ct[8 * t + i] * wy + ct[8 * t + 3 + i] * gy;
            zx += cz[6 * t + 3 + i] * gx + cz[6 * t + i] * gg[2 * i];
            zy += cz[6 * t + 3 + i] * gy + cz[6 * t + i] * gg[2 * i + 1];
        }
        const int FC[2][3] = {{2, 0, 1}, {0, 1, 2}};
        for (int k = 0; k < 2; ++k) {
            const int c = FC[k][0], a = FC[k][1], b = FC[k][2];
            const double wx = lam[a] * gg[2 * b] - lam[b] * gg[2 * a];
            const double wy = lam[a] * gg[2 * b + 1] - lam[b] * gg[2 * a + 1];
            ex += ct[8 * t + 6 + k] * (lam[c] * wx);
            ey += ct[8 * t + 6 + k] * (lam[c] * wy);
        }
    } else {
        for (int i = 0; i < 3; ++i) {
            const int a = LP[i][0], b = LP[i][1];
            const double nx = lam[a] * gg[2 * b] - lam[b] * gg[2 * a];
            const double ny = lam[a] * gg[2 * b + 1] - lam[b] * gg[2 * a + 1];
            ex += ce[3 * t + i] * nx;
            ey += ce[3 * t + i] * ny;
        }
        zx = gz[2 * t];
        zy = gz[2 * t + 1];
    }
    for (int i = 0; i < 3; ++i) E[i] = ex * u[i] + ey * v[i];
    // H_t / y = (mu_port / mu) n x (e_t + grad e_z / gamma)
    const cd s = mu_port / mu[t];
    n_cross_plane(n, u, v, s * (ex + zx / gamma), s * (ey + zy / gamma), Hy);
}

void PortFem2D::eval_face(int64_t f, double s1, double s2, const double X[3], cd E[3], cd Hy[3]) const {
    const int N = nsub;
    int i = (int)std::floor(N * std::max(0.0, s1));
    i = std::min(i, N - 1);
    int j = (int)std::floor(N * std::max(0.0, s2));
    j = std::min(j, N - 1 - i);
    const double fi = N * s1 - i, fj = N * s2 - j;
    const int up = (fi + fj > 1.0 && i + j <= N - 2) ? 1 : 0;
    const int64_t t = sub[(((size_t)f * (N + 1) + i) * (N + 1) + j) * 2 + up];
    eval_tri(t, X, E, Hy);
}

int64_t PortFem2D::locate(const double X[3]) const {
    const double x0 = (X[0] - o[0]) * u[0] + (X[1] - o[1]) * u[1] + (X[2] - o[2]) * u[2];
    const double x1 = (X[0] - o[0]) * v[0] + (X[1] - o[1]) * v[1] + (X[2] - o[2]) * v[2];
    int64_t best = 0;
    double bv = -1e300;
    const int64_t T = (int64_t)st.size() / 3;
    for (int64_t t = 0; t < T; ++t) {
        const double d0 = x0 - P0[2 * t], d1 = x1 - P0[2 * t + 1];
        const double* Ji = &Jinv[4 * t];
        const double l1 = Ji[0] * d0 + Ji[1] * d1, l2 = Ji[2] * d0 + Ji[3] * d1;
        const double m = std::min(1 - l1 - l2, std::min(l1, l2));
        if (m > bv) { bv = m; best = t; }
    }
    return best;
}

int port_fem2d_solve(const double* verts, int64_t nface, const int64_t* fv, const cd* eps_face, const cd* mu_face,
                     const double* desc, int nsub, int order, double freq, double mu_port, PortFem2D& M,
                     std::string& err, int zdef, const double* ipath, int npath, bool closed, int mode) {
    if (zdef < 0 || zdef > 2 || (zdef != 0 && (!ipath || npath < 2))) {
        err = "impedance definition: VI and PI need a current path of at least two points";
        return OPEM_ERR_ARG;
    }
    if (nface < 1 || nsub < 1 || nsub > 64 || order < 1 || order > 8 || !(freq > 0)) {
        err = "port mode: bad arguments";
        return OPEM_ERR_ARG;
    }
    M = PortFem2D{};
    M.nsub = nsub;
    M.order = order;
    M.nface = nface;
    M.freq = freq;
    M.mu_port = mu_port;
    for (int i = 0; i < 3; ++i) M.o[i] = desc[i];
    unit(desc + 3, M.u);
    unit(desc + 6, M.v);
    unit(desc + 9, M.n);
    const int N = nsub;
    // conforming split: corner nodes by vertex, edge nodes by (low vertex, high
    // vertex, step from the low one), interior nodes by (face, i, j)
    std::map<std::array<int64_t, 4>, int64_t> key;
    std::vector<double> X3;
    auto node = [&](const std::array<int64_t, 4>& k, const double* X) {
        auto it = key.find(k);
        if (it != key.end()) return it->second;
        const int64_t id = (int64_t)X3.size() / 3;
        key.emplace(k, id);
        X3.insert(X3.end(), X, X + 3);
        return id;
    };
    auto edge_node = [&](int64_t ga, int64_t gb, int m) {
        if (m == 0) return node({0, ga, 0, 0}, verts + 3 * ga);
        if (m == N) return node({0, gb, 0, 0}, verts + 3 * gb);
        const int64_t lo = std::min(ga, gb), hi = std::max(ga, gb);
        const int mm = ga < gb ? m : N - m;
        const double t = (double)mm / N;
        double X[3];
        for (int c = 0; c < 3; ++c) X[c] = verts[3 * lo + c] + t * (verts[3 * hi + c] - verts[3 * lo + c]);
        return node({1, lo, hi, mm}, X);
    };
    std::vector<int64_t> tris, tri_face;
    M.sub.assign((size_t)nface * (N + 1) * (N + 1) * 2, -1);
    std::vector<int64_t> ids((size_t)(N + 1) * (N + 1));
    for (int64_t f = 0; f < nface; ++f) {
        const int64_t g0 = fv[3 * f], g1 = fv[3 * f + 1], g2 = fv[3 * f + 2];
        const double *A = verts + 3 * g0, *B = verts + 3 * g1, *C = verts + 3 * g2;
        for (int i = 0; i <= N; ++i)
            for (int j = 0; j <= N - i; ++j) {
                int64_t id;
                if (j == 0) id = edge_node(g0, g1, i);
                else if (i == 0) id = edge_node(g0, g2, j);
                else if (i + j == N) id = edge_node(g1, g2, j);
                else {
                    const double ti = (double)i / N, tj = (double)j / N;
                    double X[3];
                    for (int c = 0; c < 3; ++c) X[c] = A[c] + ti * (B[c] - A[c]) + tj * (C[c] - A[c]);
                    id = node({2, f, i, j}, X);
                }
                ids[(size_t)i * (N + 1) + j] = id;
            }
        auto at = [&](int i, int j) { return ids[(size_t)i * (N + 1) + j]; };
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N - i; ++j) {
                M.sub[(((size_t)f * (N + 1) + i) * (N + 1) + j) * 2] = (int64_t)tri_face.size();
                tris.insert(tris.end(), {at(i, j), at(i + 1, j), at(i, j + 1)});
                tri_face.push_back(f);
                if (i + j <= N - 2) {
                    M.sub[(((size_t)f * (N + 1) + i) * (N + 1) + j) * 2 + 1] = (int64_t)tri_face.size();
                    tris.insert(tris.end(), {at(i + 1, j), at(i + 1, j + 1), at(i, j + 1)});
                    tri_face.push_back(f);
                }
            }
    }
    const int64_t nn = (int64_t)X3.size() / 3, T = (int64_t)tri_face.size();
    M.xy.resize(2 * nn);
    for (int64_t p = 0; p < nn; ++p) {
        const double* X = &X3[3 * p];
        const double d[3] = {X[0] - M.o[0], X[1] - M.o[1], X[2] - M.o[2]};
        M.xy[2 * p] = d[0] * M.u[0] + d[1] * M.u[1] + d[2] * M.u[2];
        M.xy[2 * p + 1] = d[0] * M.v[0] + d[1] * M.v[1] + d[2] * M.v[2];
    }
    std::vector<double> eps2(2 * T), mu2(2 * T);
    M.mu.resize(T);
    for (int64_t t = 0; t < T; ++t) {
        const cd e = eps_face[tri_face[t]], m = mu_face ? mu_face[tri_face[t]] : cd(1.0);
        eps2[2 * t] = e.real(); eps2[2 * t + 1] = e.imag();
        mu2[2 * t] = m.real(); mu2[2 * t + 1] = m.imag();
        M.mu[t] = m;
    }
    double beta[2];
    int64_t ne = 0;
    std::vector<int64_t> edges;
    std::vector<double> et, ez;
    // order-p elements of RefSpaces2D on unsplit faces (the mode then lies in the
    // 3D trace space), at orders above 2 and for higher modes; the split faces
    // keep the earlier first- and second-order solvers
    const bool use_ref = order >= 3 || mode > 0 || nsub == 1;
    if (order >= 2 || use_ref) {
        std::vector<cd> epsc(T), muc(T);
        for (int64_t t = 0; t < T; ++t) { epsc[t] = cd(eps2[2 * t], eps2[2 * t + 1]); muc[t] = M.mu[t]; }
        cd b2;
        std::vector<int64_t> st2;
        int rc;
        if (!use_ref) {
            rc = port_mode_2d_p2(nn, M.xy.data(), T, tris.data(), epsc.data(), muc.data(), freq, b2, M.ct, M.cz, st2);
        } else {
            try {
                M.ref = &ref_spaces_2d(order);
            } catch (const std::exception& e) {
                err = e.what();
                return OPEM_ERR_ARG;
            }
            rc = port_mode_2d_pp(nn, M.xy.data(), T, tris.data(), epsc.data(), muc.data(), freq, order, b2, M.ct,
                                 M.cz, st2, mode);
        }
        if (rc != OPEM_OK) { err = "port mode: 2D eigensolve failed"; return rc; }
        beta[0] = b2.real();
        beta[1] = b2.imag();
    } else {
        int rc = opem_port_mode_2d(nn, M.xy.data(), T, tris.data(), eps2.data(), mu2.data(), freq, beta, &ne, nullptr,
                                   nullptr, nullptr);
        if (rc != OPEM_OK) { err = "port mode: 2D mesh rejected"; return rc; }
        edges.resize(2 * ne);
        et.resize(2 * ne);
        ez.resize(2 * nn);
        rc = opem_port_mode_2d(nn, M.xy.data(), T, tris.data(), eps2.data(), mu2.data(), freq, beta, &ne, edges.data(),
                               et.data(), ez.data());
        if (rc != OPEM_OK) { err = "port mode: 2D eigensolve failed"; return rc; }
    }
    M.gamma = cd(-beta[1], beta[0]);   // j beta
    std::map<std::pair<int64_t, int64_t>, int64_t> eid;
    for (int64_t e = 0; e < ne; ++e) eid[{edges[2 * e], edges[2 * e + 1]}] = e;
    M.st.resize(3 * T);
    M.P0.resize(2 * T);
    M.Jinv.resize(4 * T);
    M.g.resize(6 * T);
    M.ce.resize(3 * T);
    M.gz.resize(2 * T);
    std::vector<double> area(T);
    for (int64_t t = 0; t < T; ++t) {
        int64_t s[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
        std::sort(s, s + 3);
        for (int k = 0; k < 3; ++k) M.st[3 * t + k] = s[k];
        const double* p0 = &M.xy[2 * s[0]];
        const double* p1 = &M.xy[2 * s[1]];
        const double* p2 = &M.xy[2 * s[2]];
        const double J00 = p1[0] - p0[0], J01 = p2[0] - p0[0], J10 = p1[1] - p0[1], J11 = p2[1] - p0[1];
        const double det = J00 * J11 - J01 * J10;
        area[t] = 0.5 * std::fabs(det);
        double* Ji = &M.Jinv[4 * t];
        Ji[0] = J11 / det; Ji[1] = -J01 / det; Ji[2] = -J10 / det; Ji[3] = J00 / det;
        M.P0[2 * t] = p0[0];
        M.P0[2 * t + 1] = p0[1];
        const double r[3][2] = {{-1, -1}, {1, 0}, {0, 1}};
        for (int k = 0; k < 3; ++k) {   // grad lambda_k = J^-T r_k
            M.g[6 * t + 2 * k] = Ji[0] * r[k][0] + Ji[2] * r[k][1];
            M.g[6 * t + 2 * k + 1] = Ji[1] * r[k][0] + Ji[3] * r[k][1];
        }
        if (order >= 2 || M.ref) continue;   // coefficients per triangle already (ct, cz)
        for (int i = 0; i < 3; ++i) {
            const int64_t e = eid.at({s[LP[i][0]], s[LP[i][1]]});
            M.ce[3 * t + i] = cd(et[2 * e], et[2 * e + 1]);
        }
        cd gx = 0.0, gy = 0.0;
        for (int k = 0; k < 3; ++k) {
            const cd z(ez[2 * s[k]], ez[2 * s[k] + 1]);
            gx += z * M.g[6 * t + 2 * k];
            gy += z * M.g[6 * t + 2 * k + 1];
        }
        M.gz[2 * t] = gx;
        M.gz[2 * t + 1] = gy;
    }
    // order-p path: H_t as the reference's 2D solver forms it, the mu-weighted L2
    // projection of n x (gamma e_t + grad e_z) / (j w mu) onto the edge space
    // (projected here divided by y)
    if (M.ref) {
        auto hfield = [&](int64_t t, double x, double y, cd& fx, cd& fy) {
            double X[3];
            for (int c = 0; c < 3; ++c) X[c] = M.o[c] + x * M.u[c] + y * M.v[c];
            cd E[3], Hy[3];
            M.eval_tri(t, X, E, Hy);
            fx = Hy[0] * M.u[0] + Hy[1] * M.u[1] + Hy[2] * M.u[2];
            fy = Hy[0] * M.v[0] + Hy[1] * M.v[1] + Hy[2] * M.v[2];
        };
        std::vector<cd> chp;
        const int rc = project_nd_2d(nn, M.xy.data(), T, M.st.data(), order, M.mu.data(), hfield, chp);
        if (rc != OPEM_OK) { err = "port mode: H projection failed"; return rc; }
        M.ch.swap(chp);
    }
    // V = -int E . dl along the voltage path
    {
        const double* p0 = desc + 16;
        const double* p1 = desc + 19;
        const double dl[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
        std::vector<double> x, w;
        gauss_legendre01(4, x, w);
        const int K = 16 * N;
        cd vint = 0.0;
        for (int k = 0; k < K; ++k)
            for (int q = 0; q < 4; ++q) {
                const double s = (k + x[q]) / K;
                const double X[3] = {p0[0] + s * dl[0], p0[1] + s * dl[1], p0[2] + s * dl[2]};
                cd E[3], Hy[3];
                M.eval_tri(M.locate(X), X, E, Hy);
                vint += (w[q] / K) * (E[0] * dl[0] + E[1] * dl[1] + E[2] * dl[2]);
            }
        M.V = -vint;
    }
    // Pz = 1/2 int (E x H*) . n, H = y Hy
    {
        const double w = 2 * M_PI * freq;
        const cd y = M.gamma / cd(0.0, w * MU0 * mu_port);
        // edge-midpoint rule (exact for the quadratic integrand of order 1), or
        // the degree-2p triangle rule (order p >= 2: integrand of degree 2p)
        std::vector<double> r1, r2, rw;
        if (M.ref) {
            // the reference's Pz (Fields::calculatePz, src/OpenParEM2D/fem2D.cpp:395-480):
            // E_t x H_t* interpolated on the order-(p-1) L2 triangle and integrated
            l2_nodal_rule(order - 1, r1, r2, rw);
            for (double& x : rw) x *= 6.0;
        } else if (order >= 2) {
            tri_rule(2 * order, r1, r2, rw);
            for (double& x : rw) x *= 6.0;   // weights of the midpoint form: area/3 * sum -> sum_q 2 w_q area
        } else {
            r1 = {0.5, 0.0, 0.5};
            r2 = {0.0, 0.5, 0.5};
            rw = {1.0, 1.0, 1.0};
        }
        cd pz = 0.0;
        for (int64_t t = 0; t < T; ++t) {
            cd acc = 0.0;
            const double* q0 = &M.xy[2 * M.st[3 * t]];
            const double* q1 = &M.xy[2 * M.st[3 * t + 1]];
            const double* q2 = &M.xy[2 * M.st[3 * t + 2]];
            for (size_t m = 0; m < rw.size(); ++m) {
                const double x2[2] = {q0[0] + r1[m] * (q1[0] - q0[0]) + r2[m] * (q2[0] - q0[0]),
                                      q0[1] + r1[m] * (q1[1] - q0[1]) + r2[m] * (q2[1] - q0[1])};
                double X[3];
                for (int c = 0; c < 3; ++c) X[c] = M.o[c] + x2[0] * M.u[c] + x2[1] * M.v[c];
                cd E[3], Hy[3];
                M.eval_tri(t, X, E, Hy);
                cd H[3];
                for (int c = 0; c < 3; ++c) H[c] = y * Hy[c];
                const cd cx = E[1] * std::conj(H[2]) - E[2] * std::conj(H[1]);
                const cd cy = E[2] * std::conj(H[0]) - E[0] * std::conj(H[2]);
                const cd cz = E[0] * std::conj(H[1]) - E[1] * std::conj(H[0]);
                acc += rw[m] * (cx * M.n[0] + cy * M.n[1] + cz * M.n[2]);
            }
            pz += area[t] / 3.0 * acc;
        }
        M.Pz = 0.5 * pz;
    }
    // I = int H . dl along the current path, H = y Hy
    M.I = 0.0;
    if (ipath && npath >= 2) {
        const double w = 2 * M_PI * freq;
        const cd y = M.gamma / cd(0.0, w * MU0 * mu_port);
        std::vector<double> x, wq;
        gauss_legendre01(4, x, wq);
        const int K = 16 * N;
        const int nseg = closed ? npath : npath - 1;
        cd iint = 0.0;
        for (int sgi = 0; sgi < nseg; ++sgi) {
            const double* p0 = ipath + 3 * sgi;
            const double* p1 = ipath + 3 * ((sgi + 1) % npath);
            const double dl[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
            for (int k = 0; k < K; ++k)
                for (int q = 0; q < 4; ++q) {
                    const double s = (k + x[q]) / K;
                    const double X[3] = {p0[0] + s * dl[0], p0[1] + s * dl[1], p0[2] + s * dl[2]};
                    cd E[3], Hy[3];
                    M.eval_tri(M.locate(X), X, E, Hy);
                    iint += (wq[q] / K) * (Hy[0] * dl[0] + Hy[1] * dl[1] + Hy[2] * dl[2]);
                }
        }
        M.I = y * iint;
    }
    if (zdef == OPEM_Z_VI) M.Z = M.V / M.I;
    else if (zdef == OPEM_Z_PI) M.Z = 2.0 * M.Pz / (M.I * std::conj(M.I));
    else M.Z = 0.5 * M.V * std::conj(M.V) / std::conj(M.Pz);
    if (!std::isfinite(M.Z.real()) || !std::isfinite(M.Z.imag())) {
        err = "port impedance is not finite (zero current or voltage on its path)";
        return OPEM_ERR_BREAKDOWN;
    }
    return OPEM_OK;
}

}  // namespace opem

extern "C" int opem_port_mode_faces_z(int64_t nverts, const double* verts, int64_t nface, const int64_t* face_verts,
                                      const double* eps_face, const double* mu_face, const double* desc, int nsub,
                                      int order, double freq, int definition, int npath, const double* path,
                                      int closed, int mode, double* metrics) {
    using cd = std::complex<double>;
    if (nverts < 3 || !verts || nface < 1 || !face_verts || !eps_face || !desc || !metrics) return OPEM_ERR_ARG;
    if (npath < 0 || (npath > 0 && !path) || mode < 0 || mode > 15) return OPEM_ERR_ARG;
    for (int64_t i = 0; i < 3 * nface; ++i)
        if (face_verts[i] < 0 || face_verts[i] >= nverts) return OPEM_ERR_ARG;
    std::vector<cd> eps(nface), mu(nface, cd(1.0));
    for (int64_t f = 0; f < nface; ++f) {
        eps[f] = cd(eps_face[2 * f], eps_face[2 * f + 1]);
        if (mu_face) mu[f] = cd(mu_face[2 * f], mu_face[2 * f + 1]);
    }
    opem::PortFem2D M;
    std::string err;
    int rc = opem::port_fem2d_solve(verts, nface, face_verts, eps.data(), mu.data(), desc, nsub, order, freq, mu[0].real(), M,
                                    err, definition, npath > 0 ? path : nullptr, npath, closed != 0, mode);
    if (rc != OPEM_OK) return rc;
    const cd m5[5] = {M.gamma, M.Z, M.V, M.Pz, M.I};
    for (int i = 0; i < 5; ++i) { metrics[2 * i] = m5[i].real(); metrics[2 * i + 1] = m5[i].imag(); }
    return OPEM_OK;
}

extern "C" int opem_port_mode_faces(int64_t nverts, const double* verts, int64_t nface, const int64_t* face_verts,
                                    const double* eps_face, const double* mu_face, const double* desc, int nsub,
                                    int order, double freq, double* metrics, int64_t npts, const int64_t* pt_face,
                                    const double* pt_s, double* E_out, double* Hy_out) {
    using cd = std::complex<double>;
    if (nverts < 3 || !verts || nface < 1 || !face_verts || !eps_face || !desc || !metrics) return OPEM_ERR_ARG;
    if (npts > 0 && (!pt_face || !pt_s)) return OPEM_ERR_ARG;
    for (int64_t i = 0; i < 3 * nface; ++i)
        if (face_verts[i] < 0 || face_verts[i] >= nverts) return OPEM_ERR_ARG;
    for (int64_t p = 0; p < npts; ++p)
        if (pt_face[p] < 0 || pt_face[p] >= nface) return OPEM_ERR_ARG;
    std::vector<cd> eps(nface), mu(nface, cd(1.0));
    for (int64_t f = 0; f < nface; ++f) {
        eps[f] = cd(eps_face[2 * f], eps_face[2 * f + 1]);
        if (mu_face) mu[f] = cd(mu_face[2 * f], mu_face[2 * f + 1]);
    }
    opem::PortFem2D M;
    std::string err;
    int rc = opem::port_fem2d_solve(verts, nface, face_verts, eps.data(), mu.data(), desc, nsub, order, freq, mu[0].real(), M,
                                    err);
    if (rc != OPEM_OK) return rc;
    const cd m4[4] = {M.gamma, M.Z, M.V, M.Pz};
    for (int i = 0; i < 4; ++i) { metrics[2 * i] = m4[i].real(); metrics[2 * i + 1] = m4[i].imag(); }
    for (int64_t p = 0; p < npts; ++p) {
        const int64_t f = pt_face[p];
        const double s1 = pt_s[2 * p], s2 = pt_s[2 * p + 1];
        const double* A = verts + 3 * face_verts[3 * f];
        const double* B = verts + 3 * face_verts[3 * f + 1];
        const double* C = verts + 3 * face_verts[3 * f + 2];
        double X[3];
        for (int c = 0; c < 3; ++c) X[c] = A[c] + s1 * (B[c] - A[c]) + s2 * (C[c] - A[c]);
        cd E[3], Hy[3];
        M.eval_face(f, s1, s2, X, E, Hy);
        for (int c = 0; c < 3; ++c) {
            if (E_out) { E_out[6 * p + 2 * c] = E[c].real(); E_out[6 * p + 2 * c + 1] = E[c].imag(); }
            if (Hy_out) { Hy_out[6 * p + 2 * c] = Hy[c].real(); Hy_out[6 * p + 2 * c + 1] = Hy[c].imag(); }
        }
    }
    return OPEM_OK;
}
