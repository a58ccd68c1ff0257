// Problem lifecycle, per-frequency solve and the C ABI entry points.
//
// The per-frequency flow restates the body of OpenParEM3D's driving-set loop
// (src/OpenParEM3D/OpenParEM3D.cpp:497-566):
//   for each driving set d (one driven S-port, 'single' driving set, port.cpp:7314-7356)
//     A_d = build_A(omega, d)                         fem3D.cpp:103-190
//     eliminate PEC rows/cols                          fem3D.cpp:728-729
//     x0 = driven mode trace; b = -A x0; b[P] = x0[P]; eliminate P; GMRES
//                                                      solveComplexLinearSystem.c:100-209
//     H: P h = j Q e                                   fem3D.cpp:192-225, 610-648
//     C+/C- from port overlaps                         port.cpp:3463-3568
//   S from a S = b                                     port.cpp:7499-7606
//   S <- (S + S^T)/2                                   results.cpp:401-418
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

#include "engine.h"

namespace opem {

static const double EPS0 = 8.8541878176e-12;   // src/OpenParEM3D/OpenParEM3D.cpp:216
static const double MU0 = 4e-7 * M_PI;

int64_t Problem::device_bytes() const {
    int64_t b = 0;
    b += d_verts.bytes() + d_tets.bytes() + d_region.bytes() + d_elem_dofs.bytes() + d_geo.bytes();
    b += d_rowptr.bytes() + d_cols.bytes() + d_d2e_ptr.bytes() + d_d2e_elem.bytes() + d_d2e_loc.bytes();
    b += d_K.bytes() + d_Meps.bytes() + d_Mtand.bytes() + d_Msig.bytes() + d_M1.bytes() + d_Q.bytes();
    b += f_K.bytes() + f_Meps.bytes() + f_Mtand.bytes() + f_Msig.bytes();
    b += d_elemcoef.bytes() + d_pec.bytes() + d_portmask.bytes() + d_et.bytes() + d_nxe.bytes() + d_et_x.bytes() + d_nxe_x.bytes();
    b += d_patch_ptr.bytes() + d_patch_dofs.bytes() + d_d2p_ptr.bytes() + d_d2p_idx.bytes() + d_patch_off.bytes();
    for (auto& g : groups) b += g.uslot.bytes() + g.urow.bytes() + g.ucol.bytes() + g.R.bytes() + g.brow.bytes() + g.bptr.bytes();
    return b;
}

// ---------------------------------------------------------------------------
// materials and port modes
// ---------------------------------------------------------------------------
// Temperature::get_Rs, src/OpenParEMCommon/OpenParEMmaterials.cpp:860-874
static double surface_resistance(double f, double sigma, double mu_r, double Rz) {
    double Rs = std::sqrt(M_PI * f * MU0 * mu_r / sigma);
    if (Rz == 0) return Rs;
    double r = Rz / (2 * std::sqrt(3.0) * 2 * (1 + std::sqrt(2.0)));
    double Aflat = 36 * r * r;
    double delta = std::sqrt(1 / (M_PI * f * MU0 * mu_r * sigma));
    return Rs * (1 + 84 * (M_PI * r * r / Aflat) / (1 + delta / r + delta * delta / (2 * r * r)));
}

static int port_region(const Problem& P, int k) {
    for (const BGroup& G : P.groups)
        if (G.type == OPEM_BDR_PORT && G.port == k && !G.faces.empty()) return P.topo.region[P.topo.face_owner[G.faces[0]]];
    return 0;
}

static void te_eval(const double* d, const double* X, double* E) {
    const double* o = d;
    const double* u = d + 3;
    const double* v = d + 6;
    double a = d[12], b = d[13], m = d[14], n = d[15];
    double ku = m * M_PI / a, kv = n * M_PI / b, amp = std::max(ku, kv);
    double uu = 0, vv = 0, nu = 0, nv = 0;
    for (int i = 0; i < 3; ++i) { nu += u[i] * u[i]; nv += v[i] * v[i]; }
    nu = std::sqrt(nu); nv = std::sqrt(nv);
    for (int i = 0; i < 3; ++i) { uu += (X[i] - o[i]) * u[i] / nu; vv += (X[i] - o[i]) * v[i] / nv; }
    double Eu = -(kv / amp) * std::cos(ku * uu) * std::sin(kv * vv);
    double Ev = (ku / amp) * std::sin(ku * uu) * std::cos(kv * vv);
    for (int i = 0; i < 3; ++i) E[i] = Eu * u[i] / nu + Ev * v[i] / nv;
}

static const int FV[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

bool has_fem2d_ports(const Problem& P) {
    for (int k = 0; k < P.nports && k < (int)P.modes.size(); ++k)
        if (P.modes[k].kind == 1) return true;
    return false;
}

// The 2D mode pm (P.modes[k] or an extra mode of port k) of port k's faces at
// freq, from the mode's cache or solved now.  The port faces are taken in the
// order port_traces visits them.
static std::shared_ptr<const PortFem2D> port_fem2d_pm(const Problem& P, int k, const PortMode& pm, double freq) {
    std::lock_guard<std::mutex> lk(pm.fem->mu);
    for (auto& e : pm.fem->sols)
        if (e.first == freq) return e.second;
    const Topology& T = P.topo;
    std::vector<int64_t> fv;
    std::vector<cd> eps, mu;
    const double w = 2 * M_PI * freq;
    for (const BGroup& G : P.groups) {
        if (G.type != OPEM_BDR_PORT || G.port != k) continue;
        for (int32_t f : G.faces) {
            const int t = T.face_owner[f], lf = T.face_lface[f];
            for (int c = 0; c < 3; ++c) fv.push_back(T.tets[4 * (size_t)t + FV[lf][c]]);
            const int r = T.region[t];
            eps.push_back(P.eps_r[r] * cd(1.0, -P.tand[r]) - cd(0.0, P.sigma[r] / (w * EPS0)));
            mu.push_back(cd(P.mu_r[r], 0.0));
        }
    }
    if (fv.empty()) throw OpemError(OPEM_ERR_ARG, "port without faces");
    auto sol = std::make_shared<PortFem2D>();
    std::string err;
    int rc = port_fem2d_solve(T.verts.data(), (int64_t)fv.size() / 3, fv.data(), eps.data(), mu.data(), pm.desc,
                              pm.nsub, pm.order2d, freq, mu[0].real(), *sol, err, pm.zdef,
                              pm.ipath.empty() ? nullptr : pm.ipath.data(), (int)(pm.ipath.size() / 3),
                              pm.ipath_closed, pm.mode);
    if (rc != OPEM_OK) throw OpemError(rc, err);
    pm.fem->sols.emplace_back(freq, sol);
    if (pm.fem->sols.size() > 8) pm.fem->sols.erase(pm.fem->sols.begin());
    return sol;
}

static std::shared_ptr<const PortFem2D> port_fem2d(const Problem& P, int k, double freq) {
    return port_fem2d_pm(P, k, P.modes[k], freq);
}

void sport_gamma_Z_V(const Problem& P, int s, double freq, cd& gamma, cd& Z, cd& V) {
    if (s < P.nports) {
        port_gamma_Z_V(P, s, freq, gamma, Z, V);
        return;
    }
    const ExtraMode& x = P.extra[s - P.nports];
    auto sol = port_fem2d_pm(P, x.port, x.m, freq);
    gamma = sol->gamma;
    Z = sol->Z;
    V = sol->V;
}

// Port::addPortIntegrators (src/OpenParEM3D/port.cpp:5790-5806): a port with
// several modes absorbs with the gamma of largest magnitude among them
cd robin_gamma(const Problem& P, int k, double freq) {
    cd g, Z, V;
    port_gamma_Z_V(P, k, freq, g, Z, V);
    for (int i = 0; i < (int)P.extra.size(); ++i) {
        if (P.extra[i].port != k) continue;
        cd gx;
        sport_gamma_Z_V(P, P.nports + i, freq, gx, Z, V);
        if (std::abs(gx) > std::abs(g)) g = gx;
    }
    return g;
}

void port_gamma_Z_V(const Problem& P, int k, double freq, cd& gamma, cd& Z, cd& V) {
    if (P.modes[k].kind == 1) {
        auto sol = port_fem2d(P, k, freq);
        gamma = sol->gamma;
        Z = sol->Z;
        V = sol->V;
        return;
    }
    const double* d = P.modes[k].desc;
    int r = port_region(P, k);
    double w = 2 * M_PI * freq, k0 = w * std::sqrt(MU0 * EPS0);
    cd epsc = P.eps_r[r] * cd(1.0, -P.tand[r]) - cd(0.0, P.sigma[r] / (w * EPS0));
    double mu = P.mu_r[r] * MU0;
    double a = d[12], b = d[13], m = d[14], n = d[15];
    double kc2 = std::pow(m * M_PI / a, 2) + std::pow(n * M_PI / b, 2);
    gamma = std::sqrt(cd(kc2, 0) - k0 * k0 * epsc * P.mu_r[r]);
    if (gamma.real() < 0) gamma = -gamma;
    // V = -int E.dl along the voltage path (24-point Gauss-Legendre)
    std::vector<double> s, ws;
    gauss_legendre01(24, s, ws);
    const double* p0 = d + 16;
    const double* p1 = d + 19;
    double vint = 0;
    for (size_t q = 0; q < s.size(); ++q) {
        double X[3], E[3];
        for (int i = 0; i < 3; ++i) X[i] = p0[i] + s[q] * (p1[i] - p0[i]);
        te_eval(d, X, E);
        vint += ws[q] * (E[0] * (p1[0] - p0[0]) + E[1] * (p1[1] - p0[1]) + E[2] * (p1[2] - p0[2]));
    }
    V = cd(-vint, 0);
    // Pz = 1/2 conj(gamma/(j w mu)) int |E_t|^2 dS  (H_t = gamma/(j w mu) n x E_t)
    double ku = m * M_PI / a, kv = n * M_PI / b, amp = std::max(ku, kv);
    double Ca = m > 0 ? a / 2 : a, Sa = m > 0 ? a / 2 : 0, Cb = n > 0 ? b / 2 : b, Sb = n > 0 ? b / 2 : 0;
    double I = (kv / amp) * (kv / amp) * Ca * Sb + (ku / amp) * (ku / amp) * Sa * Cb;
    cd yw = gamma / cd(0.0, w * mu);
    cd Pz = 0.5 * std::conj(yw) * I;
    Z = 0.5 * V * std::conj(V) / std::conj(Pz);
}

// Trace DOFs of a tangential field on one port (Mode::fillX's data, port.cpp:3234-3341):
// the edge and face moment functionals applied to E_t and n x E_t.
static void port_traces_fem2d(Problem& P, int k, std::vector<double>& et, std::vector<double>& nxe, double freq,
                              const PortMode* pm = nullptr);

static void port_traces(Problem& P, int k, std::vector<double>& et, std::vector<double>& nxe, double freq) {
    if (P.modes[k].kind == 1) {
        port_traces_fem2d(P, k, et, nxe, freq);
        return;
    }
    const Topology& T = P.topo;
    const NDRef& R = nd_reference(T.p);
    const int p = T.p;
    et.assign(2 * T.n, 0.0);
    nxe.assign(2 * T.n, 0.0);
    std::vector<uint8_t> cnt(T.n, 0);
    const double* d = P.modes[k].desc;
    double nrm[3] = {d[9], d[10], d[11]};
    double nn = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
    for (double& t : nrm) t /= nn;
    std::vector<double> s, ws;
    gauss_legendre01(p + 4, s, ws);
    std::vector<double> s1, s2, wt;
    tri_rule(2 * p + 4, s1, s2, wt);
    std::vector<int> mon2;
    std::vector<double> T2;
    if (p >= 2) T2 = tri_test_polys(p - 2, mon2);
    int nq2 = (int)mon2.size() / 2;
    // E_t and n x E_t of the analytic mode at X
    auto fields = [&](const double* X, cd* E, cd* NE) {
        double Er[3];
        te_eval(d, X, Er);
        for (int i = 0; i < 3; ++i) E[i] = Er[i];
        NE[0] = nrm[1] * Er[2] - nrm[2] * Er[1];
        NE[1] = nrm[2] * Er[0] - nrm[0] * Er[2];
        NE[2] = nrm[0] * Er[1] - nrm[1] * Er[0];
    };
    for (const BGroup& G : P.groups) {
        if (G.type != OPEM_BDR_PORT || G.port != k) continue;
        for (int32_t f : G.faces) {
            int t = T.face_owner[f], lf = T.face_lface[f];
            const int32_t* tv = &T.tets[4 * (size_t)t];
            const int32_t* ed = &T.elem_dofs[(size_t)t * T.ld];
            double Pv[3][3];
            for (int c = 0; c < 3; ++c)
                for (int i = 0; i < 3; ++i) Pv[c][i] = T.verts[3 * (size_t)tv[FV[lf][c]] + i];
            std::vector<cd> ve, vn;
            const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
            for (int e = 0; e < 3; ++e) {
                const int* pr = pairs[e];
                double tv3[3];
                for (int i = 0; i < 3; ++i) tv3[i] = Pv[pr[1]][i] - Pv[pr[0]][i];
                for (int kk = 0; kk < p; ++kk) {
                    cd ae = 0, an = 0;
                    for (size_t q = 0; q < s.size(); ++q) {
                        double X[3];
                        cd E[3], NE[3];
                        for (int i = 0; i < 3; ++i) X[i] = Pv[pr[0]][i] + s[q] * tv3[i];
                        fields(X, E, NE);
                        double L = shifted_legendre(kk, s[q]);
                        ae += ws[q] * L * (E[0] * tv3[0] + E[1] * tv3[1] + E[2] * tv3[2]);
                        an += ws[q] * L * (NE[0] * tv3[0] + NE[1] * tv3[1] + NE[2] * tv3[2]);
                    }
                    ve.push_back(ae);
                    vn.push_back(an);
                }
            }
            if (p >= 2) {
                double t1[3], t2[3];
                for (int i = 0; i < 3; ++i) { t1[i] = Pv[1][i] - Pv[0][i]; t2[i] = Pv[2][i] - Pv[0][i]; }
                for (int r = 0; r < nq2; ++r)
                    for (int tm = 0; tm < 2; ++tm) {
                        const double* tt = tm ? t2 : t1;
                        cd ae = 0, an = 0;
                        for (size_t q = 0; q < wt.size(); ++q) {
                            double X[3];
                            cd E[3], NE[3];
                            for (int i = 0; i < 3; ++i) X[i] = Pv[0][i] + s1[q] * t1[i] + s2[q] * t2[i];
                            fields(X, E, NE);
                            double qv = 0;
                            for (int c = 0; c < nq2; ++c)
                                qv += T2[r * nq2 + c] * std::pow(s1[q], mon2[2 * c]) * std::pow(s2[q], mon2[2 * c + 1]);
                            ae += wt[q] * qv * (E[0] * tt[0] + E[1] * tt[1] + E[2] * tt[2]);
                            an += wt[q] * qv * (NE[0] * tt[0] + NE[1] * tt[1] + NE[2] * tt[2]);
                        }
                        ve.push_back(ae);
                        vn.push_back(an);
                    }
            }
            for (int a2 = 0; a2 < T.ldf; ++a2) {
                int32_t g = ed[R.face_dofs[lf][a2]];
                et[2 * (size_t)g] += ve[a2].real();
                et[2 * (size_t)g + 1] += ve[a2].imag();
                nxe[2 * (size_t)g] += vn[a2].real();
                nxe[2 * (size_t)g + 1] += vn[a2].imag();
                cnt[g] += 1;
            }
        }
    }
    // an edge inside the port gets the mean of its two faces' moments (equal:
    // both faces evaluate the same points of a continuous field)
    for (size_t g = 0; g < cnt.size(); ++g)
        if (cnt[g] > 1)
            for (int c = 0; c < 2; ++c) {
                et[2 * g + c] /= cnt[g];
                nxe[2 * g + c] /= cnt[g];
            }
}

// Trace DOFs of a port's 2D mode: the same moment functionals as port_traces,
// integrated cell by cell over the face's split (composite rules: the mode is
// piecewise linear on the sub-triangles), E_t and H_t / y evaluated on the face
// being traced.  An edge inside the port gets the mean of its two faces'
// moments: E_t's tangential trace is the same from both sides, H_t's (a normal
// component of the edge-element field) jumps between cells.
static void port_traces_fem2d(Problem& P, int k, std::vector<double>& et, std::vector<double>& nxe, double freq,
                              const PortMode* pm) {
    const Topology& T = P.topo;
    std::shared_ptr<const PortFem2D> fem = port_fem2d_pm(P, k, pm ? *pm : P.modes[k], freq);
    const NDRef& R = nd_reference(T.p);
    const int p = T.p, N = fem->nsub;
    et.assign(2 * T.n, 0.0);
    nxe.assign(2 * T.n, 0.0);
    std::vector<uint8_t> cnt(T.n, 0);
    std::vector<double> s, ws;
    gauss_legendre01(p + 4, s, ws);
    std::vector<double> s1, s2, wt;
    tri_rule(2 * p + 4, s1, s2, wt);
    std::vector<int> mon2;
    std::vector<double> T2;
    if (p >= 2) T2 = tri_test_polys(p - 2, mon2);
    const int nq2 = (int)mon2.size() / 2;
    auto dot3 = [](const cd* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    int64_t fidx = 0;   // port-face index, in the order port_fem2d lists the faces
    for (const BGroup& G : P.groups) {
        if (G.type != OPEM_BDR_PORT || G.port != k) continue;
        for (int32_t f : G.faces) {
            const int t = T.face_owner[f], lf = T.face_lface[f];
            const int32_t* tv = &T.tets[4 * (size_t)t];
            const int32_t* ed = &T.elem_dofs[(size_t)t * T.ld];
            double Pv[3][3];
            for (int c = 0; c < 3; ++c)
                for (int i = 0; i < 3; ++i) Pv[c][i] = T.verts[3 * (size_t)tv[FV[lf][c]] + i];
            std::vector<cd> ve, vn;
            const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
            for (int e = 0; e < 3; ++e) {
                const int* pr = pairs[e];
                double tv3[3];
                for (int i = 0; i < 3; ++i) tv3[i] = Pv[pr[1]][i] - Pv[pr[0]][i];
                std::vector<cd> ae(p, 0.0), an(p, 0.0);
                for (int m = 0; m < N; ++m)
                    for (size_t q = 0; q < s.size(); ++q) {
                        const double sp = (m + s[q]) / N, wq = ws[q] / N;
                        double X[3];
                        for (int i = 0; i < 3; ++i) X[i] = Pv[pr[0]][i] + sp * tv3[i];
                        // face parameters of the edge point: (s,0), (0,s), (1-s,s)
                        const double a1 = e == 0 ? sp : (e == 1 ? 0.0 : 1.0 - sp);
                        const double a2 = e == 0 ? 0.0 : sp;
                        cd E[3], H[3];
                        fem->eval_face(fidx, a1, a2, X, E, H);
                        const cd et_ = dot3(E, tv3), hn_ = dot3(H, tv3);
                        for (int kk = 0; kk < p; ++kk) {
                            const double L = shifted_legendre(kk, sp);
                            ae[kk] += wq * L * et_;
                            an[kk] += wq * L * hn_;
                        }
                    }
                for (int kk = 0; kk < p; ++kk) { ve.push_back(ae[kk]); vn.push_back(an[kk]); }
            }
            if (p >= 2) {
                double t1[3], t2[3];
                for (int i = 0; i < 3; ++i) { t1[i] = Pv[1][i] - Pv[0][i]; t2[i] = Pv[2][i] - Pv[0][i]; }
                std::vector<cd> ae(2 * nq2, 0.0), an(2 * nq2, 0.0);
                for (int i = 0; i < N; ++i)
                    for (int j = 0; j < N - i; ++j)
                        for (int up = 0; up < 2; ++up) {
                            if (up && i + j > N - 2) continue;
                            const int64_t tri = fem->sub[(((size_t)fidx * (N + 1) + i) * (N + 1) + j) * 2 + up];
                            for (size_t q = 0; q < wt.size(); ++q) {
                                const double a1 = up ? (i + 1 - s1[q]) / N : (i + s1[q]) / N;
                                const double a2 = up ? (j + 1 - s2[q]) / N : (j + s2[q]) / N;
                                const double w = wt[q] / ((double)N * N);
                                double X[3];
                                for (int c = 0; c < 3; ++c) X[c] = Pv[0][c] + a1 * t1[c] + a2 * t2[c];
                                cd E[3], H[3];
                                fem->eval_tri(tri, X, E, H);
                                const cd e1 = dot3(E, t1), e2 = dot3(E, t2), h1 = dot3(H, t1), h2 = dot3(H, t2);
                                for (int r = 0; r < nq2; ++r) {
                                    double qv = 0;
                                    for (int c = 0; c < nq2; ++c)
                                        qv += T2[r * nq2 + c] * std::pow(a1, mon2[2 * c]) * std::pow(a2, mon2[2 * c + 1]);
                                    ae[2 * r] += w * qv * e1;
                                    ae[2 * r + 1] += w * qv * e2;
                                    an[2 * r] += w * qv * h1;
                                    an[2 * r + 1] += w * qv * h2;
                                }
                            }
                        }
                for (int r = 0; r < 2 * nq2; ++r) { ve.push_back(ae[r]); vn.push_back(an[r]); }
            }
            for (int a2 = 0; a2 < T.ldf; ++a2) {
                int32_t g = ed[R.face_dofs[lf][a2]];
                et[2 * (size_t)g] += ve[a2].real();
                et[2 * (size_t)g + 1] += ve[a2].imag();
                nxe[2 * (size_t)g] += vn[a2].real();
                nxe[2 * (size_t)g + 1] += vn[a2].imag();
                cnt[g] += 1;
            }
            ++fidx;
        }
    }
    for (size_t g = 0; g < cnt.size(); ++g)
        if (cnt[g] > 1)
            for (int c = 0; c < 2; ++c) {
                et[2 * g + c] /= cnt[g];
                nxe[2 * g + c] /= cnt[g];
            }
}

void refresh_port_traces(Problem& P, double freq) {
    if (!has_fem2d_ports(P) || P.trace_freq == freq) return;
    const int64_t n = P.topo.n;
    cudaStream_t s = P.ctx->stream;
    for (int k = 0; k < P.nports; ++k) {
        if (P.modes[k].kind != 1) continue;
        std::vector<double> et, nx;
        port_traces(P, k, et, nx, freq);
        OPEM_CUDA(cudaMemcpyAsync(P.d_et.p + (size_t)2 * n * k, et.data(), et.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
        OPEM_CUDA(cudaMemcpyAsync(P.d_nxe.p + (size_t)2 * n * k, nx.data(), nx.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
        // (pageable sources: each copy has read its buffer when it returns)
    }
    for (size_t i = 0; i < P.extra.size(); ++i) {
        std::vector<double> et, nx;
        port_traces_fem2d(P, P.extra[i].port, et, nx, freq, &P.extra[i].m);
        OPEM_CUDA(cudaMemcpyAsync(P.d_et_x.p + (size_t)2 * n * i, et.data(), et.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
        OPEM_CUDA(cudaMemcpyAsync(P.d_nxe_x.p + (size_t)2 * n * i, nx.data(), nx.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
    }
    OPEM_CUDA(cudaStreamSynchronize(s));
    P.trace_freq = freq;
}

void system_coefficients(const Problem& P, double freq, int d, VolCoef& vc, std::vector<BCoef>& bc) {
    double w = 2 * M_PI * freq, k0 = w * std::sqrt(MU0 * EPS0), k02 = k0 * k0;
    vc.c_eps = make_double2(-k02, 0);
    vc.c_tand = make_double2(0, k02);
    vc.c_sig = make_double2(0, w * MU0);
    bc.assign(P.groups.size(), BCoef{});
    for (size_t g = 0; g < P.groups.size(); ++g) {
        const BGroup& G = P.groups[g];
        BCoef c;
        std::memset(&c, 0, sizeof(c));
        if (G.type == OPEM_BDR_PORT && G.port != d) {
            const cd gamma = robin_gamma(P, G.port, freq);
            cd ig = 1.0 / gamma;
            cd ce = -k02 * ig, ct = cd(0, k02) * ig, cs = cd(0, w * MU0) * ig;
            c.c_cc = make_double2(ig.real(), ig.imag());
            c.c_eps = make_double2(ce.real(), ce.imag());
            c.c_tand = make_double2(ct.real(), ct.imag());
            c.c_sig = make_double2(cs.real(), cs.imag());
        } else if (G.type == OPEM_BDR_IMPEDANCE) {
            double Rs = surface_resistance(freq, G.sigma, G.mu_r, G.Rz);
            c.c_one = make_double2(0, w * MU0 / Rs);
        } else if (G.type == OPEM_BDR_RADIATION) {
            double eta = G.eta > 0 ? G.eta : std::sqrt(MU0 / EPS0);
            c.c_one = make_double2(0, w * MU0 / eta);
        }
        bc[g] = c;
    }
}

// a S = b  (BoundaryDatabase::calculateS); Cp/Cm indexed [driving set][S-port]
static std::vector<cd> s_matrix(int N, const std::vector<cd>& Cp, const std::vector<cd>& Cm, const std::vector<cd>& V,
                                const std::vector<cd>& Z) {
    int M = N * N;
    std::vector<cd> a((size_t)M * M, 0.0), b(M, 0.0);
    std::vector<cd> sc(N);
    for (int k = 0; k < N; ++k) sc[k] = V[k] / std::sqrt(Z[k]);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            b[i * N + j] = Cp[i * N + j] * sc[j];
            for (int k = 0; k < N; ++k) a[(size_t)(i * N + j) * M + (j * N + k)] = Cm[i * N + k] * sc[k];
        }
    // Gaussian elimination with partial pivoting
    for (int c = 0; c < M; ++c) {
        int piv = c;
        for (int r = c + 1; r < M; ++r)
            if (std::abs(a[(size_t)r * M + c]) > std::abs(a[(size_t)piv * M + c])) piv = r;
        if (piv != c) {
            for (int k = 0; k < M; ++k) std::swap(a[(size_t)c * M + k], a[(size_t)piv * M + k]);
            std::swap(b[c], b[piv]);
        }
        cd p = a[(size_t)c * M + c];
        for (int r = c + 1; r < M; ++r) {
            cd f = a[(size_t)r * M + c] / p;
            if (f == 0.0) continue;
            for (int k = c; k < M; ++k) a[(size_t)r * M + k] -= f * a[(size_t)c * M + k];
            b[r] -= f * b[c];
        }
    }
    std::vector<cd> S(M);
    for (int r = M - 1; r >= 0; --r) {
        cd s = b[r];
        for (int k = r + 1; k < M; ++k) s -= a[(size_t)r * M + k] * S[k];
        S[r] = s / a[(size_t)r * M + r];
    }
    return S;
}

__global__ void dmask_kernel(int64_t n, const uint8_t* __restrict__ pec, const uint8_t* __restrict__ pm, int d,
                             uint8_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (pec[i] || ((pm[i] >> d) & 1)) ? 1 : 0;
}

void make_dmask(Problem& P, int d, uint8_t* dm) {
    dmask_kernel<<<P.ctx->sm_count * 8, 256, 0, P.ctx->stream>>>(P.topo.n, P.d_pec.p, P.d_portmask.p, d, dm);
    ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
}

double port_mu_r(const Problem& P, int k) { return P.mu_r[port_region(P, k)]; }

std::vector<cd> s_matrix_solve(int N, const std::vector<cd>& Cp, const std::vector<cd>& Cm, const std::vector<cd>& V,
                               const std::vector<cd>& Z, bool reciprocal) {
    std::vector<cd> S = s_matrix(N, Cp, Cm, V, Z);
    if (reciprocal) {
        std::vector<cd> S2 = S;
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) S2[i * N + j] = 0.5 * (S[i * N + j] + S[j * N + i]);
        S = S2;
    }
    return S;
}

// x0 with PEC entries removed (columns of PEC dofs are zero in the eliminated A)
__global__ void lift_kernel(int64_t n, const double2* __restrict__ et, const uint8_t* __restrict__ pec,
                            double2* __restrict__ x0) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x0[i] = pec[i] ? make_double2(0, 0) : et[i];
}

__global__ void add_kernel(int64_t n, const double2* __restrict__ a, double2* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = make_double2(b[i].x + a[i].x, b[i].y + a[i].y);
}

__global__ void cscale_kernel(int64_t n, double2 s, const double2* __restrict__ x, double2* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = make_double2(s.x * x[i].x - s.y * x[i].y, s.x * x[i].y + s.y * x[i].x);
}

struct FreqResult {
    std::vector<cd> S, Zo;
    opem_solve_stats st;
};

static void solve_frequency_plain(Problem& P, double freq, const opem_solver_opts& o, FreqResult& out,
                                  bool keep_fields) {
    cudaStream_t s = P.ctx->stream;
    const int64_t n = P.topo.n, nnz = (int64_t)P.topo.cols.size();
    // S-ports: every port's first mode, then the extra modes (one driving set each)
    const int N = P.nsports();
    unsigned vg = (unsigned)(P.ctx->sm_count * 8);
    cudaEvent_t e0, e1;
    OPEM_CUDA(cudaEventCreate(&e0));
    OPEM_CUDA(cudaEventCreate(&e1));
    OPEM_CUDA(cudaEventRecord(e0, s));
    DBuf<double2> A(nnz), b(n), x(n), x0(n), h(n), bh(n), ov(4 * N * N + 4);
    DBuf<uint8_t> dm(n);
    std::vector<cd> Cp(N * N), Cm(N * N), gam(N), Z(N), V(N);
    double w = 2 * M_PI * freq;
    refresh_port_traces(P, freq);
    for (int k = 0; k < N; ++k) sport_gamma_Z_V(P, k, freq, gam[k], Z[k], V[k]);
    // trace vectors of S-port k
    auto et_of = [&](int k) {
        return k < P.nports ? reinterpret_cast<const double2*>(P.d_et.p) + (size_t)k * n
                            : reinterpret_cast<const double2*>(P.d_et_x.p) + (size_t)(k - P.nports) * n;
    };
    auto nxe_of = [&](int k) {
        return k < P.nports ? reinterpret_cast<const double2*>(P.d_nxe.p) + (size_t)k * n
                            : reinterpret_cast<const double2*>(P.d_nxe_x.p) + (size_t)(k - P.nports) * n;
    };
    out.st = opem_solve_stats{};
    out.st.converged = 1;
    if (keep_fields) { P.last_e.assign(N, {}); P.last_h.assign(N, {}); }
    for (int d = 0; d < N; ++d) {
        const int pd = sport_port(P, d);   // the port this driving set drives
        VolCoef vc;
        std::vector<BCoef> bc;
        system_coefficients(P, freq, pd, vc, bc);
        form_system_matrix(P, vc, bc, A.p);
        dmask_kernel<<<vg, 256, 0, s>>>(n, P.d_pec.p, P.d_portmask.p, pd, dm.p); ++P.ctx->launches;
        const double2* et = et_of(d);
        lift_kernel<<<vg, 256, 0, s>>>(n, et, P.d_pec.p, x0.p); ++P.ctx->launches;
        // b_F = -(A x0'')_F
        spmv_complex(P, A.p, x0.p, b.p, dm.p);
        cscale_kernel<<<vg, 256, 0, s>>>(n, make_double2(-1, 0), b.p, b.p); ++P.ctx->launches;
        OPEM_CUDA(cudaGetLastError());
        SolveResult r = solve_plain_fp64(P, A.p, dm.p, b.p, x.p, o);
        out.st.iterations += r.its;
        out.st.rnorm = std::max(out.st.rnorm, r.relres);
        if (!r.converged) out.st.converged = 0;
        if (r.code != OPEM_OK && r.code != OPEM_ERR_NOT_CONVERGED) throw OpemError(r.code, "E-field solve failed");
        // e = x_F + x0 on the driven port (identity rows keep x0 there)
        add_kernel<<<vg, 256, 0, s>>>(n, et, x.p); ++P.ctx->launches;
        // H: M1 h = (j / (w mu0)) Q_mu e
        spmv_real_complex(P, P.d_Q.p, x.p, bh.p, 0.0, 1.0 / (w * MU0));
        SolveResult rh = solve_mass_cg(P, bh.p, h.p, o.h_rtol, o.h_maxits);
        out.st.h_iterations += rh.its;
        // overlaps
        for (int k = 0; k < N; ++k) {
            const double2* etk = et_of(k);
            const double2* nxk = nxe_of(k);
            const int pk = sport_port(P, k);
            double2* o4 = ov.p + 4 * (d * N + k);
            port_overlap(P, pk, etk, x.p, o4 + 0);   // e0 = <Em, E>
            port_overlap(P, pk, etk, etk, o4 + 1);   // e2
            port_overlap(P, pk, nxk, h.p, o4 + 2);   // <n x Em, H>   (scaled below)
            port_overlap(P, pk, nxk, nxk, o4 + 3);   // <n x Em, n x Em>
        }
        if (keep_fields) {
            P.last_e[d].resize(2 * n);
            P.last_h[d].resize(2 * n);
            OPEM_CUDA(cudaMemcpyAsync(P.last_e[d].data(), x.p, n * sizeof(double2), cudaMemcpyDeviceToHost, s));
            OPEM_CUDA(cudaMemcpyAsync(P.last_h[d].data(), h.p, n * sizeof(double2), cudaMemcpyDeviceToHost, s));
        }
    }
    std::vector<double2> hov(4 * N * N);
    OPEM_CUDA(cudaMemcpyAsync(hov.data(), ov.p, hov.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
    OPEM_CUDA(cudaEventRecord(e1, s));
    OPEM_CUDA(cudaStreamSynchronize(s));
    for (int d = 0; d < N; ++d)
        for (int k = 0; k < N; ++k) {
            const double2* o4 = &hov[4 * (d * N + k)];
            // mode H_t = y n x E_t, y = gamma / (j w mu):  h0 = conj(y) <nxE, H>, h2 = |y|^2 <nxE, nxE>
            int r = port_region(P, sport_port(P, k));
            cd y = gam[k] / cd(0, w * P.mu_r[r] * MU0);
            cd e0(o4[0].x, o4[0].y), e2(o4[1].x, o4[1].y);
            cd h0 = std::conj(y) * cd(o4[2].x, o4[2].y), h2 = std::norm(y) * cd(o4[3].x, o4[3].y);
            Cp[d * N + k] = 0.5 * (e0 / e2 + h0 / h2);
            Cm[d * N + k] = 0.5 * (e0 / e2 - h0 / h2);
        }
    out.S = s_matrix(N, Cp, Cm, V, Z);
    if (o.force_reciprocal) {
        std::vector<cd> S2 = out.S;
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) S2[i * N + j] = 0.5 * (out.S[i * N + j] + out.S[j * N + i]);
        out.S = S2;
    }
    out.Zo = Z;
    float ms = 0;
    OPEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    out.st.seconds = ms * 1e-3;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// ---------------------------------------------------------------------------
// assembly driver
// ---------------------------------------------------------------------------
static void assemble_problem(Problem& P) {
    Topology& T = P.topo;
    cudaStream_t s = P.ctx->stream;
    std::string err;
    if (P.nregions == 0) {
        P.nregions = 1;
        P.eps_r = {1.0}; P.tand = {0.0}; P.sigma = {0.0}; P.mu_r = {1.0};
    }
    for (int32_t r : T.region)
        if (r < 0 || r >= P.nregions) throw OpemError(OPEM_ERR_ARG, "tet region index out of range");
    int rc = build_pattern(T, err);
    if (rc) throw OpemError(rc, err);
    // boundary classification
    std::map<int, Problem::Bdr> bmap(P.bdr.begin(), P.bdr.end());
    P.groups.clear();
    std::map<int, int> attr_group;
    std::vector<int32_t> pec_faces;
    P.nports = 0;
    for (auto& kv : bmap)
        if (kv.second.type == OPEM_BDR_PORT) P.nports = std::max(P.nports, (int)kv.second.params[0] + 1);
    if (P.nports > 8) throw OpemError(OPEM_ERR_UNSUPPORTED, "at most 8 ports");
    for (size_t b = 0; b < T.bdr_face.size(); ++b) {
        int attr = T.bdr_attr[b];
        auto it = bmap.find(attr);
        int type = it == bmap.end() ? OPEM_BDR_PMC : it->second.type;
        if (type == OPEM_BDR_PEC) { pec_faces.push_back(T.bdr_face[b]); continue; }
        if (type == OPEM_BDR_PMC) continue;
        auto g = attr_group.find(attr);
        if (g == attr_group.end()) {
            BGroup G;
            G.attr = attr;
            G.type = type;
            if (type == OPEM_BDR_PORT) G.port = (int)it->second.params[0];
            if (type == OPEM_BDR_IMPEDANCE) {
                G.sigma = it->second.params[0]; G.Rz = it->second.params[1];
                G.mu_r = it->second.params[2] > 0 ? it->second.params[2] : 1.0;
                if (!(G.sigma > 0)) throw OpemError(OPEM_ERR_ARG, "impedance boundary needs sigma > 0");
            }
            if (type == OPEM_BDR_RADIATION) G.eta = it->second.params[0];
            P.groups.push_back(std::move(G));
            g = attr_group.emplace(attr, (int)P.groups.size() - 1).first;
        }
        P.groups[g->second].faces.push_back(T.bdr_face[b]);
    }
    for (int k = 0; k < P.nports; ++k)
        if (!P.modes.size() || k >= (int)P.modes.size() || !P.modes[k].set)
            throw OpemError(OPEM_ERR_STATE, "port mode not set for port " + std::to_string(k));
    for (const ExtraMode& x : P.extra)
        if (x.port < 0 || x.port >= P.nports || P.modes[x.port].kind != 1)
            throw OpemError(OPEM_ERR_STATE, "an extra mode needs a port driven by its own 2D mode");
    // dirichlet masks
    const NDRef& R = nd_reference(T.p);
    P.h_pec.assign(T.n, 0);
    P.h_portmask.assign(T.n, 0);
    for (int32_t f : pec_faces) {
        int t = T.face_owner[f], lf = T.face_lface[f];
        for (int a = 0; a < T.ldf; ++a) P.h_pec[T.elem_dofs[(size_t)t * T.ld + R.face_dofs[lf][a]]] = 1;
    }
    P.port_dofs.assign(P.nports, {});
    for (BGroup& G : P.groups) {
        if (G.type != OPEM_BDR_PORT) continue;
        for (int32_t f : G.faces) {
            int t = T.face_owner[f], lf = T.face_lface[f];
            for (int a = 0; a < T.ldf; ++a) {
                int32_t dd = T.elem_dofs[(size_t)t * T.ld + R.face_dofs[lf][a]];
                P.h_portmask[dd] |= (uint8_t)(1u << G.port);
            }
        }
    }
    for (int64_t i = 0; i < T.n; ++i)
        for (int k = 0; k < P.nports; ++k)
            if ((P.h_portmask[i] >> k) & 1) P.port_dofs[k].push_back((int32_t)i);
    P.d_pec.upload(P.h_pec, s);
    P.d_portmask.upload(P.h_portmask, s);
    // patches
    rc = build_patches(T, P.h_pec, err);
    if (rc) throw OpemError(rc, err);
    P.npatch = (int)T.patch_ptr.size() - 1;
    P.d_patch_ptr.upload(T.patch_ptr, s);
    P.d_patch_dofs.upload(T.patch_dofs, s);
    P.d_patch_off.upload(T.patch_off, s);
    {
        std::vector<int32_t> cnt(T.n + 1, 0);
        for (int32_t dd : T.patch_dofs) cnt[dd + 1]++;
        for (int64_t i = 0; i < T.n; ++i) cnt[i + 1] += cnt[i];
        std::vector<int32_t> idx(T.patch_dofs.size()), fill(cnt.begin(), cnt.end() - 1);
        for (size_t q = 0; q < T.patch_dofs.size(); ++q) idx[fill[T.patch_dofs[q]]++] = (int32_t)q;
        P.d_d2p_ptr.upload(cnt, s);
        P.d_d2p_idx.upload(idx, s);
    }
    // operators
    assemble_volume(P);
    assemble_boundary(P);
    // port traces
    std::vector<double> et_all((size_t)2 * T.n * std::max(1, P.nports), 0.0), nx_all(et_all.size(), 0.0);
    for (int k = 0; k < P.nports; ++k) {
        if (P.modes[k].kind == 1) continue;   // 2D modes: traced per frequency (refresh_port_traces)
        std::vector<double> et, nx;
        port_traces(P, k, et, nx, 0.0);
        std::copy(et.begin(), et.end(), et_all.begin() + (size_t)2 * T.n * k);
        std::copy(nx.begin(), nx.end(), nx_all.begin() + (size_t)2 * T.n * k);
    }
    P.d_et.upload(et_all, s);
    P.d_nxe.upload(nx_all, s);
    if (!P.extra.empty()) {   // extra modes: traced per frequency as well
        std::vector<double> zx((size_t)2 * T.n * P.extra.size(), 0.0);
        P.d_et_x.upload(zx, s);
        P.d_nxe_x.upload(zx, s);
        OPEM_CUDA(cudaStreamSynchronize(s));
    }
    P.trace_freq = -1;
    for (int k = 0; k < P.nports; ++k)
        if (P.modes[k].kind == 1) P.modes[k].fem = std::make_shared<PortFemCache>();   // geometry may have changed
    for (ExtraMode& x : P.extra) x.m.fem = std::make_shared<PortFemCache>();
    OPEM_CUDA(cudaStreamSynchronize(s));
    P.assembled = true;
}

// ---------------------------------------------------------------------------
// Allocation-free assembly of A(freq, d) (opem_system_matrix_noalloc).
//
// The device staging buffer for the assembled values is this file-scope
// array instead of a cudaMalloc'd buffer.  Every GPU that loads the library
// holds it (OPEM_NOALLOC_MAX_NNZ complex doubles = 16 MiB) until the process
// exits.  In host code `g_noalloc_A` is only a host-side stand-in, not a device
// address: the device address is obtained once per device with
// cudaGetSymbolAddress and passed to the kernels.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double2 g_noalloc_A[OPEM_NOALLOC_MAX_NNZ];

static const int NOALLOC_MAX_DEVICES = 64;
static double2* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};
static std::mutex g_noalloc_mu;

// Device address of g_noalloc_A on `device` (which must be current).
static int noalloc_scratch(int device, double2** out, std::string& err) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) { err = "device index beyond the no-alloc set-up table"; return OPEM_ERR_ARG; }
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_A);
        if (e != cudaSuccess || !ptr) { err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e); return OPEM_ERR_CUDA; }
        g_noalloc_addr[device] = static_cast<double2*>(ptr);
    }
    *out = g_noalloc_addr[device];
    return OPEM_OK;
}

// system_coefficients into a fixed-size array: the port terms only need gamma.
// gamma comes from port_gamma_Z_V for every port kind, so a port driven by its
// own 2D mode (kind 1) gets the gamma of that mode, solved on the host (host
// memory only; no device allocation).  May throw OpemError from the 2D solve.
static int coefficients_fixed(const Problem& P, double freq, int d, VolCoef& vc, BCoef* bc, int cap) {
    if ((int)P.groups.size() > cap) return -1;
    double w = 2 * M_PI * freq, k0 = w * std::sqrt(MU0 * EPS0), k02 = k0 * k0;
    vc.c_eps = make_double2(-k02, 0);
    vc.c_tand = make_double2(0, k02);
    vc.c_sig = make_double2(0, w * MU0);
    for (size_t g = 0; g < P.groups.size(); ++g) {
        const BGroup& G = P.groups[g];
        BCoef c;
        std::memset(&c, 0, sizeof(c));
        if (G.type == OPEM_BDR_PORT && G.port != d) {
            const cd gamma = robin_gamma(P, G.port, freq);
            cd ig = 1.0 / gamma;
            cd ce = -k02 * ig, ct = cd(0, k02) * ig, cs = cd(0, w * MU0) * ig;
            c.c_cc = make_double2(ig.real(), ig.imag());
            c.c_eps = make_double2(ce.real(), ce.imag());
            c.c_tand = make_double2(ct.real(), ct.imag());
            c.c_sig = make_double2(cs.real(), cs.imag());
        } else if (G.type == OPEM_BDR_IMPEDANCE) {
            c.c_one = make_double2(0, w * MU0 / surface_resistance(freq, G.sigma, G.mu_r, G.Rz));
        } else if (G.type == OPEM_BDR_RADIATION) {
            double eta = G.eta > 0 ? G.eta : std::sqrt(MU0 / EPS0);
            c.c_one = make_double2(0, w * MU0 / eta);
        }
        bc[g] = c;
    }
    return (int)P.groups.size();
}

}  // namespace opem

// ===========================================================================
// C ABI
// ===========================================================================
using namespace opem;


template <class F>
static int guarded(Context* ctx, F&& f) {
    // a runtime error left by an earlier, unrelated call on this thread must not
    // be reported by this call's launch checks
    (void)cudaGetLastError();
    try {
        f();
        return OPEM_OK;
    } catch (const OpemError& e) {
        if (ctx) ctx->last_error = e.what();
        return e.code;
    } catch (const CudaError& e) {
        if (ctx) ctx->last_error = e.what();
        return OPEM_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->last_error = "host allocation failed";
        return OPEM_ERR_NOMEM;
    } catch (const std::exception& e) {
        if (ctx) ctx->last_error = e.what();
        return OPEM_ERR_ARG;
    }
}

extern "C" {

void opem_default_opts(opem_solver_opts* o) {
    if (!o) return;
    o->rtol = 1e-10;
    o->maxits = 5000;
    o->restart = 100;
    o->precision = OPEM_PREC_FP64;
    o->poly_degree = 0;
    o->force_reciprocal = 1;
    o->h_maxits = 2000;
    o->h_rtol = 1e-12;
    o->deflate = 30;
}

int opem_context_create(int device, opem_context* out) {
    if (!out) return OPEM_ERR_ARG;
    *out = nullptr;
    auto* c = new (std::nothrow) opem_context_s;
    if (!c) return OPEM_ERR_NOMEM;
    int rc = guarded(&c->c, [&] {
        int ndev = 0;
        OPEM_CUDA(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) throw OpemError(OPEM_ERR_ARG, "no such CUDA device");
        c->c.device = device;
        OPEM_CUDA(cudaSetDevice(device));
        OPEM_CUDA(cudaStreamCreateWithFlags(&c->c.stream, cudaStreamNonBlocking));
        OPEM_CUDA(cudaHostAlloc((void**)&c->c.pinned, 64 * sizeof(double), cudaHostAllocMapped));
        OPEM_CUDA(cudaDeviceGetAttribute(&c->c.sm_count, cudaDevAttrMultiProcessorCount, device));
    });
    if (rc) { delete c; return rc; }
    *out = c;
    return OPEM_OK;
}

int opem_context_destroy(opem_context ctx) {
    if (!ctx) return OPEM_ERR_ARG;
    cudaSetDevice(ctx->c.device);
    if (ctx->c.stream) cudaStreamDestroy(ctx->c.stream);
    if (ctx->c.pinned) cudaFreeHost(ctx->c.pinned);
    delete ctx;
    return OPEM_OK;
}

const char* opem_context_last_error(opem_context ctx) { return ctx ? ctx->c.last_error.c_str() : "null context"; }

int opem_problem_create(opem_context ctx, int64_t nverts, const double* verts, int64_t ntets, const int64_t* tets,
                        const int32_t* tet_region, int64_t nbdr, const int64_t* bdr_tris, const int32_t* bdr_attr,
                        int order, opem_problem* out) {
    if (!ctx || !out) return OPEM_ERR_ARG;
    *out = nullptr;
    if (order < 1 || order > 3) { ctx->c.last_error = "order must be 1..3"; return OPEM_ERR_UNSUPPORTED; }
    if (nbdr > 0 && (!bdr_tris || !bdr_attr)) return OPEM_ERR_ARG;
    auto* p = new (std::nothrow) opem_problem_s;
    if (!p) return OPEM_ERR_NOMEM;
    p->p.ctx = &ctx->c;
    p->device = ctx->c.device;
    int rc = guarded(&ctx->c, [&] {
        OPEM_CUDA(cudaSetDevice(ctx->c.device));
        std::string err;
        int r = build_topology(p->p.topo, nverts, verts, ntets, tets, tet_region, nbdr, bdr_tris, bdr_attr, order, err);
        if (r) throw OpemError(r, err);
    });
    if (rc) { delete p; return rc; }
    *out = p;
    return OPEM_OK;
}

int opem_problem_destroy(opem_problem prob) {
    if (!prob) return OPEM_ERR_ARG;
    cudaSetDevice(prob->device);   // not through the context, which may be gone
    delete prob;
    (void)cudaGetLastError();
    return OPEM_OK;
}

int opem_problem_set_regions(opem_problem prob, int nregions, const double* eps_r, const double* tand,
                             const double* sigma, const double* mu_r) {
    if (!prob || nregions <= 0 || !eps_r) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    P.nregions = nregions;
    P.eps_r.assign(eps_r, eps_r + nregions);
    P.tand.assign(nregions, 0.0);
    P.sigma.assign(nregions, 0.0);
    P.mu_r.assign(nregions, 1.0);
    if (tand) P.tand.assign(tand, tand + nregions);
    if (sigma) P.sigma.assign(sigma, sigma + nregions);
    if (mu_r) P.mu_r.assign(mu_r, mu_r + nregions);
    for (int r = 0; r < nregions; ++r)
        if (!(P.mu_r[r] > 0) || !std::isfinite(P.eps_r[r])) return OPEM_ERR_ARG;
    P.assembled = false;
    return OPEM_OK;
}

int opem_problem_set_boundary(opem_problem prob, int attr, int type, const double* params, int nparams) {
    if (!prob || attr < 1 || type < OPEM_BDR_PEC || type > OPEM_BDR_RADIATION) return OPEM_ERR_ARG;
    if (nparams < 0 || nparams > 3 || (nparams > 0 && !params)) return OPEM_ERR_ARG;
    Problem::Bdr b;
    b.type = type;
    for (int i = 0; i < nparams; ++i) b.params[i] = params[i];
    if (type == OPEM_BDR_PORT && (nparams < 1 || b.params[0] < 0 || b.params[0] > 7)) return OPEM_ERR_ARG;
    auto& v = prob->p.bdr;
    for (auto& kv : v)
        if (kv.first == attr) { kv.second = b; prob->p.assembled = false; return OPEM_OK; }
    v.push_back({attr, b});
    prob->p.assembled = false;
    return OPEM_OK;
}

int opem_problem_set_port_te(opem_problem prob, int port, const double* desc) {
    if (!prob || !desc || port < 0 || port > 7) return OPEM_ERR_ARG;
    if (!(desc[12] > 0) || !(desc[13] > 0) || desc[14] < 0 || desc[15] < 0 || (desc[14] == 0 && desc[15] == 0))
        return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if ((int)P.modes.size() <= port) P.modes.resize(port + 1);
    P.modes[port].set = true;
    P.modes[port].kind = 0;
    P.modes[port].zdef = OPEM_Z_PV;
    P.modes[port].ipath.clear();
    P.modes[port].fem.reset();
    std::memcpy(P.modes[port].desc, desc, 22 * sizeof(double));
    // the port's further modes belonged to its earlier definition
    P.extra.erase(std::remove_if(P.extra.begin(), P.extra.end(), [&](const ExtraMode& x) { return x.port == port; }),
                  P.extra.end());
    P.assembled = false;
    return OPEM_OK;
}

int opem_problem_set_port_fem2d(opem_problem prob, int port, const double* desc, int nsub, int order) {
    if (!prob || !desc || port < 0 || port > 7 || nsub < 1 || nsub > 64 || order < 1 || order > 8) return OPEM_ERR_ARG;
    for (int i = 0; i < 22; ++i)
        if (!std::isfinite(desc[i])) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if ((int)P.modes.size() <= port) P.modes.resize(port + 1);
    PortMode& m = P.modes[port];
    m.set = true;
    m.kind = 1;
    m.nsub = nsub;
    m.order2d = order;
    m.zdef = OPEM_Z_PV;
    m.ipath.clear();
    m.mode = 0;
    m.fem = std::make_shared<PortFemCache>();
    std::memcpy(m.desc, desc, 22 * sizeof(double));
    P.extra.erase(std::remove_if(P.extra.begin(), P.extra.end(), [&](const ExtraMode& x) { return x.port == port; }),
                  P.extra.end());
    P.assembled = false;
    return OPEM_OK;
}

int opem_problem_add_port_mode(opem_problem prob, int port, int mode, const double* vpath, int definition, int npath,
                               const double* path, int closed, int* sport) {
    if (!prob || !vpath || port < 0 || mode < 1 || mode > 15 || definition < OPEM_Z_PV || definition > OPEM_Z_PI ||
        npath < 0 || (npath > 0 && !path) || (definition != OPEM_Z_PV && npath < 2))
        return OPEM_ERR_ARG;
    for (int i = 0; i < 6; ++i)
        if (!std::isfinite(vpath[i])) return OPEM_ERR_ARG;
    for (int i = 0; i < 3 * npath; ++i)
        if (!std::isfinite(path[i])) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if ((int)P.modes.size() <= port || !P.modes[port].set || P.modes[port].kind != 1) return OPEM_ERR_STATE;
    if ((int)P.modes.size() + (int)P.extra.size() >= 16) return OPEM_ERR_UNSUPPORTED;
    ExtraMode x;
    x.port = port;
    x.m = P.modes[port];   // frame, split and element order of the port
    x.m.mode = mode;
    std::memcpy(x.m.desc + 16, vpath, 6 * sizeof(double));
    x.m.zdef = definition;
    x.m.ipath.assign(path ? path : nullptr, path ? path + 3 * npath : nullptr);
    x.m.ipath_closed = closed != 0;
    x.m.fem = std::make_shared<PortFemCache>();
    P.extra.push_back(std::move(x));
    if (sport) *sport = (int)P.modes.size() + (int)P.extra.size() - 1;
    P.assembled = false;
    return OPEM_OK;
}

int opem_problem_set_port_impedance(opem_problem prob, int port, int definition, int npath, const double* path,
                                    int closed) {
    if (!prob || port < 0 || definition < OPEM_Z_PV || definition > OPEM_Z_PI || npath < 0 || (npath > 0 && !path))
        return OPEM_ERR_ARG;
    if (definition != OPEM_Z_PV && npath < 2) return OPEM_ERR_ARG;
    for (int i = 0; i < 3 * npath; ++i)
        if (!std::isfinite(path[i])) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if ((int)P.modes.size() <= port || !P.modes[port].set) return OPEM_ERR_STATE;
    PortMode& m = P.modes[port];
    if (m.kind != 1) return definition == OPEM_Z_PV && npath == 0 ? OPEM_OK : OPEM_ERR_UNSUPPORTED;
    m.zdef = definition;
    m.ipath.assign(path ? path : nullptr, path ? path + 3 * npath : nullptr);
    m.ipath_closed = closed != 0;
    m.fem = std::make_shared<PortFemCache>();   // solved again with the new definition
    P.assembled = false;
    return OPEM_OK;
}

int opem_problem_assemble(opem_problem prob) {
    if (!prob) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    return guarded(P.ctx, [&] {
        OPEM_CUDA(cudaSetDevice(P.ctx->device));
        assemble_problem(P);
    });
}

int opem_problem_info(opem_problem prob, int64_t* info, int ninfo) {
    if (!prob || !info) return OPEM_ERR_ARG;
    const Problem& P = prob->p;
    const int64_t sum_s = (int64_t)P.topo.patch_dofs.size();
    const int64_t sum_s2 = P.topo.patch_off.empty() ? 0 : P.topo.patch_off.back();
    int64_t v[9] = {P.topo.n, (int64_t)P.topo.cols.size(), P.nsports(), P.npatch, P.topo.max_patch, P.topo.ld,
                    P.device_bytes(), sum_s, sum_s2};
    for (int i = 0; i < ninfo && i < 9; ++i) info[i] = v[i];
    return OPEM_OK;
}

static bool opts_ok(const opem_solver_opts* o) {
    return o && o->rtol > 0 && o->maxits > 0 && o->restart >= 2 && o->restart <= 2048 && o->h_maxits > 0 && o->h_rtol > 0 && o->deflate >= 0 && o->poly_degree >= 0 && o->poly_degree <= 32 &&
           (o->precision == OPEM_PREC_FP64 || o->precision == OPEM_PREC_MIXED);
}

int opem_solve_frequency(opem_problem prob, double freq, const opem_solver_opts* opts, double* S_out, double* Zo_out,
                         opem_solve_stats* stats) {
    if (!prob || !S_out || !(freq > 0)) return OPEM_ERR_ARG;
    opem_solver_opts o;
    opem_default_opts(&o);
    if (opts) o = *opts;
    if (!opts_ok(&o)) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if (!P.assembled) { P.ctx->last_error = "problem not assembled"; return OPEM_ERR_STATE; }
    if (o.precision == OPEM_PREC_MIXED && !P.extra.empty()) {
        P.ctx->last_error = "ports with several modes run on the FP64 path";
        return OPEM_ERR_UNSUPPORTED;
    }
    FreqResult fr;
    int rc = guarded(P.ctx, [&] {
        OPEM_CUDA(cudaSetDevice(P.ctx->device));
        if (o.precision == OPEM_PREC_MIXED) {
            std::vector<std::vector<cd>> S;
            std::vector<opem_solve_stats> st;
            solve_sweep_mixed(P, 1, &freq, o, S, st);
            fr.S = S[0];
            fr.st = st[0];
            fr.Zo.resize(P.nports);
            for (int k = 0; k < P.nports; ++k) {
                cd g, V;
                port_gamma_Z_V(P, k, freq, g, fr.Zo[k], V);
            }
        } else {
            solve_frequency_plain(P, freq, o, fr, true);
        }
    });
    if (rc) return rc;
    int N = P.nsports();
    for (int i = 0; i < N * N; ++i) { S_out[2 * i] = fr.S[i].real(); S_out[2 * i + 1] = fr.S[i].imag(); }
    if (Zo_out)
        for (int i = 0; i < N; ++i) { Zo_out[2 * i] = fr.Zo[i].real(); Zo_out[2 * i + 1] = fr.Zo[i].imag(); }
    if (stats) *stats = fr.st;
    return fr.st.converged ? OPEM_OK : OPEM_ERR_NOT_CONVERGED;
}

int opem_solve_sweep(opem_problem prob, int nfreq, const double* freqs, const opem_solver_opts* opts, double* S_out,
                     opem_solve_stats* stats) {
    if (!prob || nfreq <= 0 || !freqs || !S_out) return OPEM_ERR_ARG;
    int N = prob->p.nsports(), worst = OPEM_OK;
    if (opts && opts->precision == OPEM_PREC_MIXED) {
        Problem& P = prob->p;
        if (!P.extra.empty()) {
            P.ctx->last_error = "ports with several modes run on the FP64 path";
            return OPEM_ERR_UNSUPPORTED;
        }
        if (!opts_ok(opts)) return OPEM_ERR_ARG;
        if (!P.assembled) { P.ctx->last_error = "problem not assembled"; return OPEM_ERR_STATE; }
        for (int f = 0; f < nfreq; ++f)
            if (!(freqs[f] > 0)) return OPEM_ERR_ARG;
        std::vector<std::vector<cd>> S;
        std::vector<opem_solve_stats> st;
        int rc = guarded(P.ctx, [&] {
            OPEM_CUDA(cudaSetDevice(P.ctx->device));
            solve_sweep_mixed(P, nfreq, freqs, *opts, S, st);
        });
        if (rc) return rc;
        for (int f = 0; f < nfreq; ++f) {
            for (int i = 0; i < N * N; ++i) {
                S_out[(size_t)2 * N * N * f + 2 * i] = S[f][i].real();
                S_out[(size_t)2 * N * N * f + 2 * i + 1] = S[f][i].imag();
            }
            if (stats) stats[f] = st[f];
            if (!st[f].converged) worst = OPEM_ERR_NOT_CONVERGED;
        }
        return worst;
    }
    for (int f = 0; f < nfreq; ++f) {
        int rc = opem_solve_frequency(prob, freqs[f], opts, S_out + (size_t)2 * N * N * f, nullptr, stats ? stats + f : nullptr);
        if (rc == OPEM_ERR_NOT_CONVERGED) worst = rc;
        else if (rc) return rc;
    }
    return worst;
}

// fem3D::calculateMeshErrors marking (src/OpenParEM3D/fem3D.cpp:1321-1350): the
// floor(NE * fraction) (at least one) largest errors, largest first (ties by
// element index), and the largest error.
int opem_mesh_errors(opem_problem prob, double fraction, double* errors_out, int64_t* marked_out, int64_t max_marked,
                     int64_t* nmarked, double* max_error) {
    if (!prob || !(fraction >= 0) || !(fraction <= 1) || max_marked < 0 || (max_marked > 0 && !marked_out))
        return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if (!P.assembled) return OPEM_ERR_STATE;
    bool have = false;
    for (auto& v : P.last_h) have |= !v.empty();
    if (!have) return OPEM_ERR_STATE;
    return guarded(P.ctx, [&] {
        OPEM_CUDA(cudaSetDevice(P.ctx->device));
        const int64_t ne = P.topo.ne;
        std::vector<double> e;
        mesh_error_indicator(P, e);
        if (errors_out) std::memcpy(errors_out, e.data(), ne * sizeof(double));
        int64_t count = std::max<int64_t>(1, (int64_t)((double)ne * fraction));
        count = std::min(count, ne);
        std::vector<int64_t> idx(ne);
        for (int64_t i = 0; i < ne; ++i) idx[i] = i;
        std::partial_sort(idx.begin(), idx.begin() + count, idx.end(),
                          [&](int64_t a, int64_t b) { return e[a] > e[b] || (e[a] == e[b] && a < b); });
        for (int64_t i = 0; i < std::min(count, max_marked); ++i) marked_out[i] = idx[i];
        if (nmarked) *nmarked = count;
        if (max_error) *max_error = e[idx[0]];
    });
}

int opem_get_fields(opem_problem prob, int d, double* e_out, double* h_out) {
    if (!prob) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if (d < 0 || d >= (int)P.last_e.size() || P.last_e[d].empty()) return OPEM_ERR_STATE;
    if (e_out) std::memcpy(e_out, P.last_e[d].data(), P.last_e[d].size() * sizeof(double));
    if (h_out) std::memcpy(h_out, P.last_h[d].data(), P.last_h[d].size() * sizeof(double));
    return OPEM_OK;
}

int opem_get_operator(opem_problem prob, int which, int64_t* rowptr, int32_t* cols, double* vals) {
    if (!prob) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if (!P.assembled) return OPEM_ERR_STATE;
    return guarded(P.ctx, [&] {
        if (rowptr)
            for (size_t i = 0; i < P.topo.rowptr.size(); ++i) rowptr[i] = P.topo.rowptr[i];
        if (cols) std::memcpy(cols, P.topo.cols.data(), P.topo.cols.size() * sizeof(int32_t));
        if (vals) {
            DBuf<double>* src[6] = {&P.d_K, &P.d_Meps, &P.d_Mtand, &P.d_Msig, &P.d_M1, &P.d_Q};
            if (which < 0 || which > 5) throw OpemError(OPEM_ERR_ARG, "operator index");
            size_t nnz = P.topo.cols.size();
            if (src[which]->p == nullptr) std::memset(vals, 0, nnz * sizeof(double));
            else OPEM_CUDA(cudaMemcpy(vals, src[which]->p, nnz * sizeof(double), cudaMemcpyDeviceToHost));
        }
    });
}

int opem_get_system_matrix(opem_problem prob, double freq, int d, double* vals) {
    if (!prob || !vals || !(freq > 0)) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if (!P.assembled || d < 0 || d >= std::max(1, P.nports)) return OPEM_ERR_STATE;
    return guarded(P.ctx, [&] {
        OPEM_CUDA(cudaSetDevice(P.ctx->device));
        size_t nnz = P.topo.cols.size();
        DBuf<double2> A(nnz);
        VolCoef vc;
        std::vector<BCoef> bc;
        system_coefficients(P, freq, d, vc, bc);
        form_system_matrix(P, vc, bc, A.p);
        OPEM_CUDA(cudaStreamSynchronize(P.ctx->stream));
        OPEM_CUDA(cudaMemcpy(vals, A.p, nnz * sizeof(double2), cudaMemcpyDeviceToHost));
    });
}

int opem_context_launches(opem_context ctx, int64_t* out) {
    if (!ctx || !out) return OPEM_ERR_ARG;
    *out = ctx->c.launches;
    return OPEM_OK;
}

int opem_profile_kernels(opem_problem prob, double freq, int reps, double* out, int nout) {
    if (!prob || !out || nout < 12 || reps <= 0 || !(freq > 0)) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if (!P.assembled) return OPEM_ERR_STATE;
    return guarded(P.ctx, [&] {
        OPEM_CUDA(cudaSetDevice(P.ctx->device));
        const int64_t n = P.topo.n;
        DBuf<double2> A(P.topo.cols.size());
        DBuf<uint8_t> dm(n);
        VolCoef vc;
        std::vector<BCoef> bc;
        system_coefficients(P, freq, 0, vc, bc);
        form_system_matrix(P, vc, bc, A.p);
        dmask_kernel<<<P.ctx->sm_count * 8, 256, 0, P.ctx->stream>>>(n, P.d_pec.p, P.d_portmask.p, 0, dm.p);
        ++P.ctx->launches;
        profile_fp64(P, A.p, dm.p, reps, out);
    });
}

int opem_profile_batch_kernels(opem_problem prob, double freq, int nsys, int reps, double* out, int nout) {
    if (!prob || !out || nout < 15 || reps <= 0 || !(freq > 0) || nsys < 1 || nsys > 32) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if (!P.assembled) return OPEM_ERR_STATE;
    return guarded(P.ctx, [&] {
        OPEM_CUDA(cudaSetDevice(P.ctx->device));
        profile_batch(P, freq, nsys, reps, out, nout);
    });
}

int opem_check_block_apply(opem_problem prob, double freq, int nsys, int r0, int nd, double* out, int nout) {
    if (!prob || !out || nout < 5 || !(freq > 0) || nsys < 1 || nsys > 32 || r0 < 0 || nd < 1 || r0 + nd > nsys)
        return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if (!P.assembled) return OPEM_ERR_STATE;
    return guarded(P.ctx, [&] {
        OPEM_CUDA(cudaSetDevice(P.ctx->device));
        check_block_apply(P, freq, nsys, r0, nd, out);
    });
}

int opem_selftest_wait_timeout(opem_context ctx, int polls) {
    if (!ctx || polls < 1 || polls > (1 << 24)) return OPEM_ERR_ARG;
    int code = OPEM_OK;
    int rc = guarded(&ctx->c, [&] {
        OPEM_CUDA(cudaSetDevice(ctx->c.device));
        code = selftest_wait_timeout(ctx->c, polls);
    });
    return rc != OPEM_OK ? rc : code;
}

// No counterpart in the reference.  See include/opem_b200.h for the contract.
int opem_system_matrix_noalloc(opem_problem prob, double freq, int d, double* vals) {
    if (!prob || !vals || !(freq > 0)) return OPEM_ERR_ARG;
    Problem& P = prob->p;
    if (!P.assembled || d < 0 || d >= std::max(1, P.nports)) {
        P.ctx->last_error = "opem_system_matrix_noalloc: problem not assembled or driving set out of range";
        return OPEM_ERR_STATE;
    }
    const size_t nnz = P.topo.cols.size();
    if (nnz > (size_t)OPEM_NOALLOC_MAX_NNZ) {
        P.ctx->last_error = "opem_system_matrix_noalloc: nnz exceeds OPEM_NOALLOC_MAX_NNZ (1048576); "
                            "use opem_get_system_matrix";
        return OPEM_ERR_ARG;
    }
    const int CAP = 64;
    if ((int)P.groups.size() > CAP) {
        P.ctx->last_error = "opem_system_matrix_noalloc: more than 64 boundary groups";
        return OPEM_ERR_ARG;
    }
    return guarded(P.ctx, [&] {
        BCoef bc[CAP];
        VolCoef vc;
        coefficients_fixed(P, freq, d, vc, bc, CAP);
        OPEM_CUDA(cudaSetDevice(P.ctx->device));
        double2* scratch = nullptr;
        std::string err;
        int rc = noalloc_scratch(P.ctx->device, &scratch, err);
        if (rc) throw OpemError(rc, err);
        // combine_kernel writes every one of the nnz entries before the boundary
        // kernels add to them, so nothing left by an earlier call is read.
        form_system_matrix_n(P, vc, bc, (size_t)CAP, scratch);
        OPEM_CUDA(cudaMemcpyAsync(vals, scratch, nnz * sizeof(double2), cudaMemcpyDeviceToHost, P.ctx->stream));
        OPEM_CUDA(cudaStreamSynchronize(P.ctx->stream));
    });
}

}  // extern "C"
