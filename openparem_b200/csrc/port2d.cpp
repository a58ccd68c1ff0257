// Port eigenmode of a waveguide cross-section on the host (the modal problem
// OpenParEM3D hands to its 2D solver, src/OpenParEM3D/port.cpp:5081-5176, solved
// there by OpenParEM2D with SLEPc).  Lowest-order edge elements for the
// transverse field e_t, linear nodal elements for e_z, PEC on the outer
// boundary, per-triangle complex eps_r and mu_r.  With psi = j e_z / beta the
// problem is the symmetric pencil (Lee, Sun and Cendes, IEEE MTT 1991)
//
//     [S - k0^2 T_eps  0] x = -beta^2 [T_mu  -G; -G^T  Kz] x,
//
// and the fundamental mode (largest beta^2) is found by inverse iteration with
// the shift -k0^2 max Re(eps_r mu_r), moved onto the Rayleigh quotient once
// that has settled to ~1e-6.  The shifted matrix is factorised (twice) by
// banded LU with partial pivoting, updated column by column, after the
// narrowest of a few reverse Cuthill-McKee orderings (2D meshes keep the band
// near sqrt(n)).
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <numeric>
#include <queue>
#include <vector>

#include "../../include/opem_b200.h"
#include "dense.h"
#include "opem_internal.h"
#include "portfem.h"

namespace {

using cd = std::complex<double>;
constexpr double MU0 = 4e-7 * M_PI, EPS0 = 8.8541878176e-12;

struct Triplet { int r, c; cd v; };

// banded LU with partial pivoting (kl sub-, ku super-diagonals; ku grows by kl)
struct Banded {
    int n = 0, kl = 0, ku0 = 0, ku = 0, ld = 0;   // ku = ku0 + kl: upper band after pivoting
    std::vector<cd> a;   // column-major band storage: a[(kl + ku0 + i - j) + j * ld] (LAPACK's layout)
    std::vector<int> piv;
    cd& at(int i, int j) { return a[(size_t)(kl + ku0 + i - j) + (size_t)j * ld]; }
    void init(int n_, int kl_, int ku_) {
        n = n_; kl = kl_; ku0 = ku_; ku = ku_ + kl_; ld = 2 * kl + ku0 + 1;
        a.assign((size_t)ld * n, 0.0);
        piv.assign(n, 0);
    }
    bool factor() {
        for (int j = 0; j < n; ++j) {
            const int imax = std::min(n - 1, j + kl);
            int p = j;
            double best = std::abs(at(j, j));
            for (int i = j + 1; i <= imax; ++i)
                if (std::abs(at(i, j)) > best) { best = std::abs(at(i, j)); p = i; }
            if (!(best > 0)) return false;
            piv[j] = p;
            const int jmax = std::min(n - 1, j + ku);
            if (p != j)
                for (int k = j; k <= jmax; ++k) std::swap(at(j, k), at(p, k));
            const cd d = 1.0 / at(j, j);
            for (int i = j + 1; i <= imax; ++i) at(i, j) *= d;
            // rank-1 update column by column: within a column the band rows are contiguous
            const cd* lj = &at(j + 1, j);
            for (int k = j + 1; k <= jmax; ++k) {
                const cd u = at(j, k);
                if (u == 0.0) continue;
                cd* ck = &at(j + 1, k);
                for (int i = 0; i < imax - j; ++i) ck[i] -= lj[i] * u;
            }
        }
        return true;
    }
    void solve(std::vector<cd>& b) {
        for (int j = 0; j < n; ++j) {
            if (piv[j] != j) std::swap(b[j], b[piv[j]]);
            const int imax = std::min(n - 1, j + kl);
            for (int i = j + 1; i <= imax; ++i) b[i] -= at(i, j) * b[j];
        }
        for (int j = n - 1; j >= 0; --j) {
            b[j] /= at(j, j);
            const int imin = std::max(0, j - ku);
            for (int i = imin; i < j; ++i) b[i] -= at(i, j) * b[j];
        }
    }
};

// reverse Cuthill-McKee order of a symmetric sparsity pattern
std::vector<int> rcm(int n, const std::vector<std::vector<int>>& adj, int start = -1) {
    std::vector<int> order, deg(n);
    for (int i = 0; i < n; ++i) deg[i] = (int)adj[i].size();
    std::vector<char> seen(n, 0);
    for (int root0 = (start >= 0 ? start : 0), first = 1; root0 < n; root0 = first ? 0 : root0 + 1, first = 0) {
        if (seen[root0]) continue;
        int root = root0;   // a pseudo-peripheral start: lowest degree in the component's first BFS level set
        for (int pass = 0; pass < (first && start >= 0 ? 0 : 2); ++pass) {
            std::vector<int> lvl(n, -1);
            std::queue<int> q;
            q.push(root);
            lvl[root] = 0;
            int last = root;
            while (!q.empty()) {
                int u = q.front();
                q.pop();
                last = u;
                for (int w : adj[u])
                    if (lvl[w] < 0) { lvl[w] = lvl[u] + 1; q.push(w); }
            }
            int best = last;
            for (int i = 0; i < n; ++i)
                if (lvl[i] == lvl[last] && deg[i] < deg[best]) best = i;
            root = best;
        }
        std::queue<int> q;
        q.push(root);
        seen[root] = 1;
        while (!q.empty()) {
            int u = q.front();
            q.pop();
            order.push_back(u);
            std::vector<int> nb;
            for (int w : adj[u])
                if (!seen[w]) { seen[w] = 1; nb.push_back(w); }
            std::sort(nb.begin(), nb.end(), [&](int x, int y) { return deg[x] < deg[y]; });
            for (int w : nb) q.push(w);
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

// Fundamental eigenpair of the pencil A x = -beta^2 B x (largest beta^2) by
// The pencil's A has no e_z block, so every (0, psi) is an eigenvector with
// lam = 0: a null space as large as the e_z space, which lies between the
// propagating modes (lam < 0) and the cut-off ones (lam > 0) and captures an
// iteration about a shift below them once the wanted mode is cut off.  With the
// unknowns from nut on being psi, PsiConstraint sets psi to the solution of the
// e_z rows of B x = 0 (psi = -B_zz^-1 B_zt e_t), which every eigenvector of a
// nonzero lam satisfies; applied after every step it removes any null-space
// component.  pos: the iteration's permuted numbering.
struct PsiConstraint {
    int n = 0, nut = 0, nz = 0;
    std::vector<Triplet> Bzt;
    Banded Mz;
    std::vector<int> zpos;
    std::vector<cd> zr;
    bool init(int n_, int nut_, const std::vector<Triplet>& Bm) {
        n = n_; nut = nut_; nz = n - nut;
        if (nz <= 0) return true;
        std::vector<std::vector<int>> zadj(nz);
        for (auto& t : Bm) {
            if (t.r < nut) continue;
            if (t.c < nut) Bzt.push_back(t);
            else if (t.r != t.c) zadj[t.r - nut].push_back(t.c - nut);
        }
        for (auto& a : zadj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
        std::vector<int> zord = rcm(nz, zadj);
        zpos.assign(nz, 0);
        for (int i = 0; i < nz; ++i) zpos[zord[i]] = i;
        int zbw = 0;
        for (int i = 0; i < nz; ++i)
            for (int j : zadj[i]) zbw = std::max(zbw, std::abs(zpos[i] - zpos[j]));
        Mz.init(nz, zbw, zbw);
        for (auto& t : Bm)
            if (t.r >= nut && t.c >= nut) Mz.at(zpos[t.r - nut], zpos[t.c - nut]) += t.v;
        zr.assign(nz, 0.0);
        return Mz.factor();
    }
    void apply(cd* y, const std::vector<int>& pos) {
        if (nz <= 0) return;
        std::fill(zr.begin(), zr.end(), cd(0.0));
        for (auto& t : Bzt) zr[zpos[t.r - nut]] -= t.v * y[pos[t.c]];
        Mz.solve(zr);
        for (int i = 0; i < nz; ++i) y[pos[nut + i]] = zr[zpos[i]];
    }
};

// inverse iteration with the shift sigma: RCM ordering, banded LU of A - sigma B,
// converged when the eigenvalue has settled and the unit eigenvector stops
// moving (up to phase).  Returns an OPEM_* code; lam = -beta^2, xout unit norm
// in the caller's numbering.  nut < n: the unknowns from nut on are psi, held to
// PsiConstraint.
int solve_pencil(int n, const std::vector<Triplet>& A, const std::vector<Triplet>& Bm, double sigma, cd& lam,
                 std::vector<cd>& xout, int nut = -1) {
    // ordering and band
    std::vector<std::vector<int>> adj(n);
    for (auto* T : {&A, &Bm})
        for (auto& x : *T)
            if (x.r != x.c) adj[x.r].push_back(x.c);
    for (auto& a : adj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
    // the band of the reverse Cuthill-McKee order from the pseudo-peripheral start
    // and from a few lowest-degree starts: the narrowest one is kept (the LU costs
    // n bw^2)
    auto band = [&](const std::vector<int>& ord) {
        std::vector<int> ps(n);
        for (int i = 0; i < n; ++i) ps[ord[i]] = i;
        int b = 0;
        for (int i = 0; i < n; ++i)
            for (int j : adj[i]) b = std::max(b, std::abs(ps[i] - ps[j]));
        return b;
    };
    std::vector<int> ord = rcm(n, adj);
    int bw = band(ord);
    {
        std::vector<int> cand(n);
        for (int i = 0; i < n; ++i) cand[i] = i;
        const int K = std::min(n, 8);
        std::partial_sort(cand.begin(), cand.begin() + K, cand.end(), [&](int a, int b) {
            return adj[a].size() < adj[b].size() || (adj[a].size() == adj[b].size() && a < b);
        });
        for (int k = 0; k < K; ++k) {
            std::vector<int> o2 = rcm(n, adj, cand[k]);
            const int b2 = band(o2);
            if (b2 < bw) { bw = b2; ord.swap(o2); }
        }
    }
    std::vector<int> pos(n);
    for (int i = 0; i < n; ++i) pos[ord[i]] = i;
    Banded M;
    auto factor_at = [&](cd shift) {
        M.init(n, bw, bw);
        for (auto& x : A) M.at(pos[x.r], pos[x.c]) += x.v;
        for (auto& x : Bm) M.at(pos[x.r], pos[x.c]) -= shift * x.v;
        return M.factor();
    };
    cd shift = sigma;
    if (!factor_at(shift)) return OPEM_ERR_BREAKDOWN;
    PsiConstraint psi;
    if (nut > 0 && nut < n && !psi.init(n, nut, Bm)) return OPEM_ERR_BREAKDOWN;
    bool refreshed = false;
    // inverse iteration: y = (A - sigma B)^-1 B x; its dominant eigenvalue mu gives lambda = sigma + 1/mu
    auto Bmul = [&](const std::vector<cd>& x, std::vector<cd>& y) {
        std::fill(y.begin(), y.end(), 0.0);
        for (auto& t : Bm) y[pos[t.r]] += t.v * x[pos[t.c]];
    };
    std::vector<cd> x(n), y(n), bx(n), xold(n);
    for (int i = 0; i < n; ++i) x[i] = cd(1.0 + 0.001 * (i % 7), 0.0005 * (i % 5));
    psi.apply(x.data(), pos);
    cd lam_prev = 0;
    lam = 0;
    bool ok = false;
    int lam_done = 0;
    for (int it = 0; it < 4000; ++it) {
        xold = x;
        Bmul(x, bx);
        y = bx;
        M.solve(y);
        psi.apply(y.data(), pos);
        // Rayleigh-type estimate mu = (x^H B y) / (x^H B x), B symmetric
        std::vector<cd> by(n);
        Bmul(y, by);
        cd num = 0, den = 0;
        for (int i = 0; i < n; ++i) { num += std::conj(x[i]) * by[i]; den += std::conj(x[i]) * bx[i]; }
        double nrm = 0;
        for (auto& v : y) nrm += std::norm(v);
        nrm = std::sqrt(nrm);
        if (!(nrm > 0) || den == 0.0) return OPEM_ERR_BREAKDOWN;
        for (int i = 0; i < n; ++i) x[i] = y[i] / nrm;
        const cd mu = num / den;
        lam = shift + 1.0 / mu;
        // converged when the eigenvalue has settled and the unit eigenvector stops
        // moving (up to phase): the eigenvalue settles about twice as fast, and
        // small components such as e_z of a TE-like mode need the vector itself
        // once the eigenvalue is known to ~1e-6, move the shift onto it (one more
        // factorisation): the remaining steps then converge in a few iterations
        if (!refreshed && it > 3 && std::abs(lam - lam_prev) <= 1e-6 * std::abs(lam)) {
            refreshed = true;
            const cd s2 = lam;
            if (factor_at(s2)) {
                shift = s2;
                lam_prev = 0;
                lam_done = 0;
                continue;
            }
            if (!factor_at(shift)) return OPEM_ERR_BREAKDOWN;   // exactly singular: keep the first shift
        }
        if (it > 3 && std::abs(lam - lam_prev) <= 1e-14 * std::abs(lam)) ++lam_done;
        if (lam_done) {
            cd c = 0;
            for (int i = 0; i < n; ++i) c += std::conj(xold[i]) * x[i];
            const cd ph = std::abs(c) > 0 ? c / std::abs(c) : cd(1.0);
            double dx = 0;
            for (int i = 0; i < n; ++i) dx += std::norm(x[i] - ph * xold[i]);
            if (std::sqrt(dx) <= 1e-12 || lam_done > 20) { ok = true; break; }
        }
        lam_prev = lam;
    }
    if (!ok) return OPEM_ERR_NOT_CONVERGED;
    xout.assign(n, 0.0);
    for (int i = 0; i < n; ++i) xout[i] = x[pos[i]];
    return OPEM_OK;
}

// The k eigenpairs of A x = -beta^2 B x with the largest beta^2 (the k eigenvalues
// nearest the shift sigma, which lies below all of them) by subspace iteration on
// (A - sigma B)^-1 B with k + 2 vectors (one banded LU, RCM order as above) and
// Rayleigh-Ritz on the projected pencil: converged when every wanted Ritz pair's
// residual is below 1e-11 relative and its value has settled to 1e-13.  lam[i] = -beta_i^2 in increasing distance from sigma, X (n x k,
// column-major) the Ritz vectors in the caller's numbering.
// The unknowns from nut on are psi, held to PsiConstraint after every step, so
// cut-off modes are found too.
int solve_pencil_k(int n, const std::vector<Triplet>& A, const std::vector<Triplet>& Bm, double sigma, int k,
                   std::vector<cd>& lam, std::vector<cd>& X, int nut) {
    const int q = std::min(n, k + 2);
    if (k < 1 || k > n || nut < 1 || nut > n) return OPEM_ERR_ARG;
    std::vector<std::vector<int>> adj(n);
    for (auto* T : {&A, &Bm})
        for (auto& x : *T)
            if (x.r != x.c) adj[x.r].push_back(x.c);
    for (auto& a : adj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
    std::vector<int> ord = rcm(n, adj);
    std::vector<int> pos(n);
    for (int i = 0; i < n; ++i) pos[ord[i]] = i;
    int bw = 0;
    for (int i = 0; i < n; ++i)
        for (int j : adj[i]) bw = std::max(bw, std::abs(pos[i] - pos[j]));
    Banded M;
    M.init(n, bw, bw);
    for (auto& x : A) M.at(pos[x.r], pos[x.c]) += x.v;
    for (auto& x : Bm) M.at(pos[x.r], pos[x.c]) -= sigma * x.v;
    if (!M.factor()) return OPEM_ERR_BREAKDOWN;
    auto mul = [&](const std::vector<Triplet>& T, const cd* x, cd* y) {   // permuted numbering
        std::fill(y, y + n, cd(0.0));
        for (auto& t : T) y[pos[t.r]] += t.v * x[pos[t.c]];
    };
    PsiConstraint psi;
    if (!psi.init(n, nut, Bm)) return OPEM_ERR_BREAKDOWN;
    auto constrain = [&](cd* y) { psi.apply(y, pos); };   // y in the permuted numbering
    std::vector<cd> Y((size_t)n * q), AY((size_t)n * q), BY((size_t)n * q), tmp(n);
    for (int c = 0; c < q; ++c) {
        for (int i = 0; i < n; ++i) Y[(size_t)c * n + i] = cd(1.0 + 0.001 * ((i * (c + 3)) % 11), 0.0007 * ((i + 5 * c) % 7));
        constrain(&Y[(size_t)c * n]);
    }
    std::vector<cd> prev(k, cd(0.0));
    lam.assign(k, 0.0);
    bool ok = false;
    for (int it = 0; it < 2000 && !ok; ++it) {
        // Y <- (A - sigma B)^-1 B Y, orthonormal columns
        for (int c = 0; c < q; ++c) {
            mul(Bm, &Y[(size_t)c * n], tmp.data());
            M.solve(tmp);
            constrain(tmp.data());
            std::copy(tmp.begin(), tmp.end(), &Y[(size_t)c * n]);
        }
        if (opem::orthonormalise(n, q, Y) != q) return OPEM_ERR_BREAKDOWN;
        // projected pencil Ah z = lam Bh z -> C = Bh^-1 (Ah - sigma Bh), eigenvalues lam - sigma
        for (int c = 0; c < q; ++c) {
            mul(A, &Y[(size_t)c * n], &AY[(size_t)c * n]);
            mul(Bm, &Y[(size_t)c * n], &BY[(size_t)c * n]);
        }
        std::vector<cd> Ah((size_t)q * q), Bh((size_t)q * q);
        for (int i = 0; i < q; ++i)
            for (int j = 0; j < q; ++j) {
                cd a = 0, b = 0;
                for (int r = 0; r < n; ++r) {
                    a += std::conj(Y[(size_t)i * n + r]) * AY[(size_t)j * n + r];
                    b += std::conj(Y[(size_t)i * n + r]) * BY[(size_t)j * n + r];
                }
                Ah[i + (size_t)j * q] = a;
                Bh[i + (size_t)j * q] = b;
            }
        std::vector<cd> C((size_t)q * q);
        for (int j = 0; j < q; ++j) {
            std::vector<cd> col(q);
            for (int i = 0; i < q; ++i) col[i] = Ah[i + (size_t)j * q] - sigma * Bh[i + (size_t)j * q];
            if (!opem::lu_solve(q, Bh, col)) return OPEM_ERR_BREAKDOWN;
            for (int i = 0; i < q; ++i) C[i + (size_t)j * q] = col[i];
        }
        std::vector<cd> th, Z;
        if (!opem::eig_smallest(q, C, q, th, Z)) return OPEM_ERR_BREAKDOWN;
        std::vector<int> idx(q);
        for (int i = 0; i < q; ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](int a, int b) { return std::abs(th[a]) < std::abs(th[b]); });
        // Ritz vectors, nearest first, and their products with A and B (the same
        // combinations of AY and BY)
        std::vector<cd> Yn((size_t)n * q, 0.0), AYn((size_t)n * k, 0.0), BYn((size_t)n * k, 0.0);
        for (int c = 0; c < q; ++c)
            for (int j = 0; j < q; ++j) {
                const cd z = Z[j + (size_t)idx[c] * q];
                if (z == 0.0) continue;
                for (int r = 0; r < n; ++r) Yn[(size_t)c * n + r] += Y[(size_t)j * n + r] * z;
                if (c < k)
                    for (int r = 0; r < n; ++r) {
                        AYn[(size_t)c * n + r] += AY[(size_t)j * n + r] * z;
                        BYn[(size_t)c * n + r] += BY[(size_t)j * n + r] * z;
                    }
            }
        Y.swap(Yn);
        // converged when every wanted pair's residual |A y - lam B y| is below
        // 1e-11 of |A y| + |lam| |B y| and its value has settled to 1e-13
        bool settled = true;
        for (int i = 0; i < k; ++i) {
            lam[i] = sigma + th[idx[i]];
            double rr = 0, na = 0, nb = 0;
            for (int r = 0; r < n; ++r) {
                rr += std::norm(AYn[(size_t)i * n + r] - lam[i] * BYn[(size_t)i * n + r]);
                na += std::norm(AYn[(size_t)i * n + r]);
                nb += std::norm(BYn[(size_t)i * n + r]);
            }
            if (!(std::sqrt(rr) <= 1e-11 * (std::sqrt(na) + std::abs(lam[i]) * std::sqrt(nb)))) settled = false;
            if (!(std::abs(lam[i] - prev[i]) <= 1e-13 * std::abs(lam[i]))) settled = false;
            prev[i] = lam[i];
        }
        ok = settled && it >= 3;
    }
    if (!ok) return OPEM_ERR_NOT_CONVERGED;
    X.assign((size_t)n * k, 0.0);
    for (int c = 0; c < k; ++c) {
        double nr = 0;
        for (int r = 0; r < n; ++r) nr += std::norm(Y[(size_t)c * n + r]);
        nr = std::sqrt(nr);
        for (int i = 0; i < n; ++i) X[(size_t)c * n + i] = Y[(size_t)c * n + pos[i]] / nr;
    }
    return OPEM_OK;
}

}  // namespace

extern "C" {

int opem_port_mode_2d(int64_t nnodes, const double* xy, int64_t ntri, const int64_t* tris, const double* eps_r,
                      const double* mu_r, double freq, double* beta_out, int64_t* nedges, int64_t* edges_out,
                      double* et_out, double* ez_out) {
    if (nnodes < 3 || !xy || ntri < 1 || !tris || !eps_r || !(freq > 0) || !beta_out || !nedges) return OPEM_ERR_ARG;
    for (int64_t t = 0; t < 3 * ntri; ++t)
        if (tris[t] < 0 || tris[t] >= nnodes) return OPEM_ERR_ARG;
    const double k0 = 2 * M_PI * freq * std::sqrt(MU0 * EPS0);
    // edges: sorted vertex pairs, numbered in lexicographic order; orientation low -> high vertex
    std::map<std::pair<int64_t, int64_t>, int> eid;
    std::vector<std::array<int64_t, 3>> st(ntri);
    for (int64_t t = 0; t < ntri; ++t) {
        std::array<int64_t, 3> v = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
        std::sort(v.begin(), v.end());
        st[t] = v;
        static const int LP[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        for (auto& lp : LP) eid[{v[lp[0]], v[lp[1]]}] = 0;
    }
    int ne = 0;
    std::vector<std::pair<int64_t, int64_t>> edges;
    for (auto& kv : eid) { kv.second = ne++; edges.push_back(kv.first); }
    *nedges = ne;
    if (!et_out && !ez_out && !edges_out) return OPEM_OK;   // size query
    if (edges_out)
        for (int e = 0; e < ne; ++e) { edges_out[2 * e] = edges[e].first; edges_out[2 * e + 1] = edges[e].second; }
    // element matrices
    std::vector<Triplet> Aee, Bee, Ben, Bnn;   // A = S - k0^2 T_eps; B blocks T_mu, -G, Kz
    std::vector<int> ecount(ne, 0);
    double emax = 0;
    static const int LP[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int64_t t = 0; t < ntri; ++t) {
        const auto& v = st[t];
        double P[3][2];
        for (int k = 0; k < 3; ++k) { P[k][0] = xy[2 * v[k]]; P[k][1] = xy[2 * v[k] + 1]; }
        const double J00 = P[1][0] - P[0][0], J01 = P[2][0] - P[0][0], J10 = P[1][1] - P[0][1], J11 = P[2][1] - P[0][1];
        const double det = J00 * J11 - J01 * J10;
        if (!(std::fabs(det) > 0)) return OPEM_ERR_ARG;
        const double area = 0.5 * std::fabs(det);
        // grad lambda: rows of J^-T applied to (-1,-1), (1,0), (0,1)
        const double i00 = J11 / det, i01 = -J01 / det, i10 = -J10 / det, i11 = J00 / det;   // J^-1
        double g[3][2];
        const double r[3][2] = {{-1, -1}, {1, 0}, {0, 1}};
        for (int k = 0; k < 3; ++k) {   // grad = J^-T r
            g[k][0] = i00 * r[k][0] + i10 * r[k][1];
            g[k][1] = i01 * r[k][0] + i11 * r[k][1];
        }
        auto dotg = [&](int p, int q) { return g[p][0] * g[q][0] + g[p][1] * g[q][1]; };
        auto Mll = [&](int p, int q) { return area / 12.0 * (p == q ? 2.0 : 1.0); };
        double curl[3];
        for (int i = 0; i < 3; ++i) {
            const int a = LP[i][0], b = LP[i][1];
            curl[i] = 2.0 * (g[a][0] * g[b][1] - g[a][1] * g[b][0]);
        }
        const cd er(eps_r[2 * t], eps_r[2 * t + 1]);
        const cd mr = mu_r ? cd(mu_r[2 * t], mu_r[2 * t + 1]) : cd(1.0, 0.0);
        const cd im = 1.0 / mr;
        emax = std::max(emax, std::real(er * mr));
        int ge[3];
        for (int i = 0; i < 3; ++i) { ge[i] = eid[{v[LP[i][0]], v[LP[i][1]]}]; ++ecount[ge[i]]; }
        for (int i = 0; i < 3; ++i) {
            const int a = LP[i][0], b = LP[i][1];
            for (int j = 0; j < 3; ++j) {
                const int c = LP[j][0], d = LP[j][1];
                const double m = Mll(a, c) * dotg(b, d) - Mll(a, d) * dotg(b, c) - Mll(b, c) * dotg(a, d) + Mll(b, d) * dotg(a, c);
                Aee.push_back({ge[i], ge[j], im * curl[i] * curl[j] * area - k0 * k0 * er * m});
                Bee.push_back({ge[i], ge[j], im * m});
            }
            for (int k = 0; k < 3; ++k) {
                const double ng = area / 3.0 * ((g[b][0] - g[a][0]) * g[k][0] + (g[b][1] - g[a][1]) * g[k][1]);
                Ben.push_back({ge[i], (int)v[k], -im * ng});
            }
        }
        for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l)
                Bnn.push_back({(int)v[k], (int)v[l], im * area * dotg(k, l) - k0 * k0 * er * Mll(k, l)});
    }
    // PEC: boundary edges (in one triangle) and their nodes are removed
    std::vector<int> emap(ne, -1), nmap(nnodes, -1);
    std::vector<char> bnode(nnodes, 0);
    for (int e = 0; e < ne; ++e)
        if (ecount[e] == 1) { bnode[edges[e].first] = 1; bnode[edges[e].second] = 1; }
    int nu = 0;
    for (int e = 0; e < ne; ++e)
        if (ecount[e] != 1) emap[e] = nu++;
    const int nue = nu;
    std::vector<char> used(nnodes, 0);
    for (int64_t t = 0; t < 3 * ntri; ++t) used[tris[t]] = 1;
    for (int64_t i = 0; i < nnodes; ++i)
        if (used[i] && !bnode[i]) nmap[i] = nu++;
    const int n = nu;
    if (n == 0) return OPEM_ERR_ARG;
    // global sparse A and B in the unknown numbering
    std::vector<Triplet> A, Bm;
    for (auto& x : Aee) if (emap[x.r] >= 0 && emap[x.c] >= 0) A.push_back({emap[x.r], emap[x.c], x.v});
    for (auto& x : Bee) if (emap[x.r] >= 0 && emap[x.c] >= 0) Bm.push_back({emap[x.r], emap[x.c], x.v});
    for (auto& x : Ben)
        if (emap[x.r] >= 0 && nmap[x.c] >= 0) {
            Bm.push_back({emap[x.r], nmap[x.c], x.v});
            Bm.push_back({nmap[x.c], emap[x.r], x.v});
        }
    for (auto& x : Bnn) if (nmap[x.r] >= 0 && nmap[x.c] >= 0) Bm.push_back({nmap[x.r], nmap[x.c], x.v});
    const double sigma = -k0 * k0 * emax;
    cd lam = 0;
    std::vector<cd> xs;
    {
        int rc = solve_pencil(n, A, Bm, sigma, lam, xs);
        if (rc != OPEM_OK) return rc;
    }
    cd beta = std::sqrt(-lam);
    if (beta.real() < 0) beta = -beta;
    beta_out[0] = beta.real();
    beta_out[1] = beta.imag();
    // scale: the largest e_t coefficient becomes 1
    cd big = 0.0;
    for (int e = 0; e < ne; ++e)
        if (emap[e] >= 0 && std::abs(xs[emap[e]]) > std::abs(big)) big = xs[emap[e]];
    const cd s = std::abs(big) > 0 ? 1.0 / big : cd(1.0);
    if (et_out)
        for (int e = 0; e < ne; ++e) {
            const cd v = emap[e] >= 0 ? xs[emap[e]] * s : cd(0.0);
            et_out[2 * e] = v.real();
            et_out[2 * e + 1] = v.imag();
        }
    if (ez_out)
        for (int64_t i = 0; i < nnodes; ++i) {
            const cd v = nmap[i] >= 0 ? -cd(0, 1) * beta * xs[nmap[i]] * s : cd(0.0);   // e_z = -j beta psi
            ez_out[2 * i] = v.real();
            ez_out[2 * i + 1] = v.imag();
        }
    return OPEM_OK;
}

}  // extern "C"

namespace opem {

// Second-order elements for the same pencil (the oracle's port2d.solve_mode_p2):
// with the triangle's vertices sorted by node id and l_0..2 their barycentrics,
//   e_t: W_ab = l_a grad l_b - l_b grad l_a and G_ab = grad(l_a l_b) for the edges
//        (a,b) = (0,1), (0,2), (1,2) (shared by the edge's triangles), then the
//        face functions l_2 W_01 and l_0 W_12 (no tangential trace);
//   e_z: l_0, l_1, l_2 and the edge bubbles l_a l_b.
// Whitney functions plus edge gradients span the complete linear fields and the
// face functions complete the degree-2 first-kind space (Webb, IEEE TAP 47(8)
// 1999); grad of the quadratic nodal space lies in it, as the pencil needs.
// Element integrals by the degree-4 triangle rule (exact for these products).
// Outputs per triangle: ct (8 e_t coefficients), cz (6 e_z coefficients), st
// (the sorted vertex ids), scaled so the largest Whitney coefficient is 1.
int port_mode_2d_p2(int64_t nnodes, const double* xy, int64_t ntri, const int64_t* tris, const cd* eps_r,
                    const cd* mu_r, double freq, cd& beta, std::vector<cd>& ct, std::vector<cd>& cz,
                    std::vector<int64_t>& st) {
    if (nnodes < 3 || !xy || ntri < 1 || !tris || !eps_r || !(freq > 0)) return OPEM_ERR_ARG;
    for (int64_t t = 0; t < 3 * ntri; ++t)
        if (tris[t] < 0 || tris[t] >= nnodes) return OPEM_ERR_ARG;
    static const int LP[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    const double k0 = 2 * M_PI * freq * std::sqrt(MU0 * EPS0);
    st.resize(3 * ntri);
    std::map<std::pair<int64_t, int64_t>, int> eid;
    for (int64_t t = 0; t < ntri; ++t) {
        int64_t v[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
        std::sort(v, v + 3);
        for (int k = 0; k < 3; ++k) st[3 * t + k] = v[k];
        for (auto& lp : LP) eid[{v[lp[0]], v[lp[1]]}] = 0;
    }
    int ne = 0;
    std::vector<std::pair<int64_t, int64_t>> edges;
    for (auto& kv : eid) { kv.second = ne++; edges.push_back(kv.first); }
    // global numbering: e_t = [W (ne), G (ne), face (2 ntri)], e_z = [vertex (nnodes), bubble (ne)]
    const int64_t net = 2 * (int64_t)ne + 2 * ntri, nz = nnodes + ne;
    std::vector<int64_t> tdof(8 * ntri), zdof(6 * ntri);
    std::vector<int> ecount(ne, 0);
    for (int64_t t = 0; t < ntri; ++t) {
        for (int i = 0; i < 3; ++i) {
            const int e = eid[{st[3 * t + LP[i][0]], st[3 * t + LP[i][1]]}];
            ++ecount[e];
            tdof[8 * t + i] = e;
            tdof[8 * t + 3 + i] = ne + e;
            zdof[6 * t + i] = st[3 * t + i];
            zdof[6 * t + 3 + i] = nnodes + e;
        }
        tdof[8 * t + 6] = 2 * (int64_t)ne + 2 * t;
        tdof[8 * t + 7] = 2 * (int64_t)ne + 2 * t + 1;
    }
    std::vector<double> q1, q2, qw;
    tri_rule(4, q1, q2, qw);
    const int nq = (int)qw.size();
    std::vector<Triplet> Aee, Bee, Ben, Bnn;
    double emax = 0;
    auto cross = [](const double* a, const double* b) { return a[0] * b[1] - a[1] * b[0]; };
    for (int64_t t = 0; t < ntri; ++t) {
        const double* p0 = xy + 2 * st[3 * t];
        const double* p1 = xy + 2 * st[3 * t + 1];
        const double* p2 = xy + 2 * st[3 * t + 2];
        const double J00 = p1[0] - p0[0], J01 = p2[0] - p0[0], J10 = p1[1] - p0[1], J11 = p2[1] - p0[1];
        const double det = J00 * J11 - J01 * J10;
        if (!(std::fabs(det) > 0)) return OPEM_ERR_ARG;
        const double area = 0.5 * std::fabs(det);
        const double i00 = J11 / det, i01 = -J01 / det, i10 = -J10 / det, i11 = J00 / det;
        double g[3][2];
        const double r[3][2] = {{-1, -1}, {1, 0}, {0, 1}};
        for (int k = 0; k < 3; ++k) {
            g[k][0] = i00 * r[k][0] + i10 * r[k][1];
            g[k][1] = i01 * r[k][0] + i11 * r[k][1];
        }
        const cd er = eps_r[t], mr = mu_r ? mu_r[t] : cd(1.0), im = 1.0 / mr;
        emax = std::max(emax, std::real(er * mr));
        double M[8][8] = {}, C[8][8] = {}, Gm[8][6] = {}, Kg[6][6] = {}, Ml[6][6] = {};
        for (int q = 0; q < nq; ++q) {
            const double lam[3] = {1 - q1[q] - q2[q], q1[q], q2[q]};
            const double w = 2 * area * qw[q];
            double N[8][2], cN[8], L[6], dL[6][2];
            for (int i = 0; i < 3; ++i) {
                const int a = LP[i][0], b = LP[i][1];
                for (int c = 0; c < 2; ++c) {
                    N[i][c] = lam[a] * g[b][c] - lam[b] * g[a][c];
                    N[3 + i][c] = lam[a] * g[b][c] + lam[b] * g[a][c];
                    dL[3 + i][c] = N[3 + i][c];
                    dL[i][c] = g[i][c];
                }
                cN[i] = 2.0 * cross(g[a], g[b]);
                cN[3 + i] = 0.0;
                L[i] = lam[i];
                L[3 + i] = lam[a] * lam[b];
            }
            const int FC[2][3] = {{2, 0, 1}, {0, 1, 2}};   // (c, a, b): l_c W_ab
            for (int k = 0; k < 2; ++k) {
                const int c = FC[k][0], a = FC[k][1], b = FC[k][2];
                double W[2];
                for (int d = 0; d < 2; ++d) W[d] = lam[a] * g[b][d] - lam[b] * g[a][d];
                for (int d = 0; d < 2; ++d) N[6 + k][d] = lam[c] * W[d];
                cN[6 + k] = cross(g[c], W) + lam[c] * 2.0 * cross(g[a], g[b]);
            }
            for (int i = 0; i < 8; ++i) {
                for (int j = 0; j < 8; ++j) {
                    M[i][j] += w * (N[i][0] * N[j][0] + N[i][1] * N[j][1]);
                    C[i][j] += w * cN[i] * cN[j];
                }
                for (int j = 0; j < 6; ++j) Gm[i][j] += w * (N[i][0] * dL[j][0] + N[i][1] * dL[j][1]);
            }
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j) {
                    Kg[i][j] += w * (dL[i][0] * dL[j][0] + dL[i][1] * dL[j][1]);
                    Ml[i][j] += w * L[i] * L[j];
                }
        }
        for (int i = 0; i < 8; ++i) {
            for (int j = 0; j < 8; ++j) {
                Aee.push_back({(int)tdof[8 * t + i], (int)tdof[8 * t + j], im * C[i][j] - k0 * k0 * er * M[i][j]});
                Bee.push_back({(int)tdof[8 * t + i], (int)tdof[8 * t + j], im * M[i][j]});
            }
            for (int j = 0; j < 6; ++j) Ben.push_back({(int)tdof[8 * t + i], (int)zdof[6 * t + j], -im * Gm[i][j]});
        }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j)
                Bnn.push_back({(int)zdof[6 * t + i], (int)zdof[6 * t + j], im * Kg[i][j] - k0 * k0 * er * Ml[i][j]});
    }
    // PEC: both edge functions of boundary edges, boundary vertices and bubbles
    std::vector<int> tmap(net, -1), zmap(nz, -1);
    std::vector<char> bnode(nnodes, 0), bedge(ne, 0);
    for (int e = 0; e < ne; ++e)
        if (ecount[e] == 1) { bedge[e] = 1; bnode[edges[e].first] = 1; bnode[edges[e].second] = 1; }
    int nu = 0;
    for (int64_t i = 0; i < net; ++i) {
        const bool drop = (i < ne && bedge[i]) || (i >= ne && i < 2 * ne && bedge[i - ne]);
        if (!drop) tmap[i] = nu++;
    }
    const int nut = nu;
    std::vector<char> used(nnodes, 0);
    for (int64_t t = 0; t < 3 * ntri; ++t) used[tris[t]] = 1;
    for (int64_t i = 0; i < nz; ++i) {
        const bool drop = i < nnodes ? (!used[i] || bnode[i]) : (bool)bedge[i - nnodes];
        if (!drop) zmap[i] = nu++;
    }
    const int n = nu;
    if (nut == 0) return OPEM_ERR_ARG;
    std::vector<Triplet> A, Bm;
    for (auto& x : Aee) if (tmap[x.r] >= 0 && tmap[x.c] >= 0) A.push_back({tmap[x.r], tmap[x.c], x.v});
    for (auto& x : Bee) if (tmap[x.r] >= 0 && tmap[x.c] >= 0) Bm.push_back({tmap[x.r], tmap[x.c], x.v});
    for (auto& x : Ben)
        if (tmap[x.r] >= 0 && zmap[x.c] >= 0) {
            Bm.push_back({tmap[x.r], zmap[x.c], x.v});
            Bm.push_back({zmap[x.c], tmap[x.r], x.v});
        }
    for (auto& x : Bnn) if (zmap[x.r] >= 0 && zmap[x.c] >= 0) Bm.push_back({zmap[x.r], zmap[x.c], x.v});
    cd lam = 0;
    std::vector<cd> xs;
    int rc = solve_pencil(n, A, Bm, -k0 * k0 * emax, lam, xs);
    if (rc != OPEM_OK) return rc;
    beta = std::sqrt(-lam);
    if (beta.real() < 0) beta = -beta;
    cd big = 0.0;
    for (int e = 0; e < ne; ++e)
        if (tmap[e] >= 0 && std::abs(xs[tmap[e]]) > std::abs(big)) big = xs[tmap[e]];
    const cd sc = std::abs(big) > 0 ? 1.0 / big : cd(1.0);
    ct.assign(8 * ntri, 0.0);
    cz.assign(6 * ntri, 0.0);
    for (int64_t t = 0; t < ntri; ++t) {
        for (int i = 0; i < 8; ++i) {
            const int m = tmap[tdof[8 * t + i]];
            ct[8 * t + i] = m >= 0 ? xs[m] * sc : cd(0.0);
        }
        for (int i = 0; i < 6; ++i) {
            const int m = zmap[zdof[6 * t + i]];
            cz[6 * t + i] = m >= 0 ? -cd(0, 1) * beta * xs[m] * sc : cd(0.0);   // e_z = -j beta psi
        }
    }
    return OPEM_OK;
}

}  // namespace opem

// ---------------------------------------------------------------------------
// Order-p elements (the spaces of the reference's 2D solver at mesh.order p,
// MFEM ND_FECollection(p) and H1_FECollection(p), OpenParEM2D fem2D.cpp:2188-2191)
// ---------------------------------------------------------------------------
namespace opem {

namespace {
// inverse of a dense real n x n matrix (row-major) by Gauss-Jordan with partial pivoting
bool invert_real(int n, std::vector<double>& A) {
    std::vector<double> I((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) I[(size_t)i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[(size_t)r * n + c]) > std::fabs(A[(size_t)piv * n + c])) piv = r;
        if (!(std::fabs(A[(size_t)piv * n + c]) > 0)) return false;
        if (piv != c)
            for (int k = 0; k < n; ++k) {
                std::swap(A[(size_t)piv * n + k], A[(size_t)c * n + k]);
                std::swap(I[(size_t)piv * n + k], I[(size_t)c * n + k]);
            }
        const double d = 1.0 / A[(size_t)c * n + c];
        for (int k = 0; k < n; ++k) { A[(size_t)c * n + k] *= d; I[(size_t)c * n + k] *= d; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = A[(size_t)r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
                I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
            }
        }
    }
    A.swap(I);
    return true;
}

double ipow(double x, int a) {
    double r = 1.0;
    for (int i = 0; i < a; ++i) r *= x;
    return r;
}

RefSpaces2D build_ref_spaces(int p) {
    RefSpaces2D R;
    R.p = p;
    for (int d = 0; d <= p; ++d)
        for (int a = d; a >= 0; --a) { R.mono.push_back(a); R.mono.push_back(d - a); }
    R.nm = (int)R.mono.size() / 2;
    auto idx = [&](int a, int b) {
        for (int m = 0; m < R.nm; ++m)
            if (R.mono[2 * m] == a && R.mono[2 * m + 1] == b) return m;
        throw std::runtime_error("monomial out of range");
    };
    // spanning set of R_p: P_{p-1}^2, then (-y, x) x^a y^(p-1-a)
    std::vector<std::vector<double>> FX, FY;
    for (int d = 0; d <= p - 1; ++d)
        for (int a = d; a >= 0; --a) {
            std::vector<double> e(R.nm, 0.0), z(R.nm, 0.0);
            e[idx(a, d - a)] = 1.0;
            FX.push_back(e); FY.push_back(z);
            FX.push_back(z); FY.push_back(e);
        }
    for (int a = 0; a < p; ++a) {
        const int b = p - 1 - a;
        std::vector<double> ex(R.nm, 0.0), ey(R.nm, 0.0);
        ex[idx(a, b + 1)] = -1.0;
        ey[idx(a + 1, b)] = 1.0;
        FX.push_back(ex); FY.push_back(ey);
    }
    const int nf = (int)FX.size();
    if (nf != p * (p + 2)) throw std::runtime_error("edge space dimension");
    R.nf = nf;
    auto poly = [&](const std::vector<double>& c, double x, double y) {
        double s = 0;
        for (int m = 0; m < R.nm; ++m)
            if (c[m] != 0.0) s += c[m] * ipow(x, R.mono[2 * m]) * ipow(y, R.mono[2 * m + 1]);
        return s;
    };
    // degrees of freedom of the spanning functions: D (nf x nf), row = DOF
    std::vector<double> D((size_t)nf * nf, 0.0);
    std::vector<double> s, ws;
    gauss_legendre01(p + 2, s, ws);
    static const double VR[3][2] = {{0, 0}, {1, 0}, {0, 1}};
    static const int LPr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    int row = 0;
    for (auto& lp : LPr) {
        const double ax = VR[lp[0]][0], ay = VR[lp[0]][1];
        const double tx = VR[lp[1]][0] - ax, ty = VR[lp[1]][1] - ay;
        for (int k = 0; k < p; ++k, ++row)
            for (int j = 0; j < nf; ++j) {
                double acc = 0;
                for (size_t q = 0; q < s.size(); ++q) {
                    const double x = ax + s[q] * tx, y = ay + s[q] * ty;
                    acc += ws[q] * shifted_legendre(k, s[q]) * (poly(FX[j], x, y) * tx + poly(FY[j], x, y) * ty);
                }
                D[(size_t)row * nf + j] = acc;
            }
    }
    if (p >= 2) {
        std::vector<int> m2;
        const std::vector<double> T2 = tri_test_polys(p - 2, m2);
        const int nq2 = (int)m2.size() / 2;
        std::vector<double> q1, q2, qw;
        tri_rule(2 * p + 2, q1, q2, qw);
        for (int r = 0; r < nq2; ++r)
            for (int comp = 0; comp < 2; ++comp, ++row)
                for (int j = 0; j < nf; ++j) {
                    double acc = 0;
                    for (size_t q = 0; q < qw.size(); ++q) {
                        double tv = 0;
                        for (int c = 0; c < nq2; ++c)
                            tv += T2[(size_t)r * nq2 + c] * ipow(q1[q], m2[2 * c]) * ipow(q2[q], m2[2 * c + 1]);
                        acc += qw[q] * tv * (comp ? poly(FY[j], q1[q], q2[q]) : poly(FX[j], q1[q], q2[q]));
                    }
                    D[(size_t)row * nf + j] = acc;
                }
    }
    if (row != nf || !invert_real(nf, D)) throw std::runtime_error("edge degrees of freedom not unisolvent");
    // nodal function i = sum_j F_j Dinv[j][i]
    R.CX.assign((size_t)R.nm * nf, 0.0);
    R.CY.assign((size_t)R.nm * nf, 0.0);
    for (int j = 0; j < nf; ++j)
        for (int i = 0; i < nf; ++i) {
            const double c = D[(size_t)j * nf + i];
            if (c == 0.0) continue;
            for (int m = 0; m < R.nm; ++m) {
                R.CX[(size_t)m * nf + i] += c * FX[j][m];
                R.CY[(size_t)m * nf + i] += c * FY[j][m];
            }
        }
    // Lagrange nodes and the inverse Vandermonde
    std::vector<std::array<double, 2>> nodes = {{0, 0}, {1, 0}, {0, 1}};
    for (auto& lp : LPr)
        for (int k = 1; k < p; ++k)
            nodes.push_back({VR[lp[0]][0] + (double)k / p * (VR[lp[1]][0] - VR[lp[0]][0]),
                             VR[lp[0]][1] + (double)k / p * (VR[lp[1]][1] - VR[lp[0]][1])});
    for (int j = 1; j < p; ++j)
        for (int i = 1; i < p - j; ++i) nodes.push_back({(double)i / p, (double)j / p});
    R.nl = (int)nodes.size();
    if (R.nl != R.nm) throw std::runtime_error("Lagrange node count");
    std::vector<double> V((size_t)R.nl * R.nm);
    for (int r = 0; r < R.nl; ++r)
        for (int m = 0; m < R.nm; ++m) V[(size_t)r * R.nm + m] = ipow(nodes[r][0], R.mono[2 * m]) * ipow(nodes[r][1], R.mono[2 * m + 1]);
    if (!invert_real(R.nm, V)) throw std::runtime_error("Lagrange nodes not unisolvent");
    R.CL = V;   // (V^-1)[m][i]: coefficient of monomial m in Lagrange function i
    return R;
}
}  // namespace

void RefSpaces2D::nd(double x, double y, double* N, double* curl) const {
    for (int i = 0; i < nf; ++i) { N[2 * i] = N[2 * i + 1] = 0.0; curl[i] = 0.0; }
    for (int m = 0; m < nm; ++m) {
        const int a = mono[2 * m], b = mono[2 * m + 1];
        const double v = ipow(x, a) * ipow(y, b);
        const double dx = a > 0 ? a * ipow(x, a - 1) * ipow(y, b) : 0.0;
        const double dy = b > 0 ? b * ipow(x, a) * ipow(y, b - 1) : 0.0;
        const double* cx = &CX[(size_t)m * nf];
        const double* cy = &CY[(size_t)m * nf];
        for (int i = 0; i < nf; ++i) {
            N[2 * i] += cx[i] * v;
            N[2 * i + 1] += cy[i] * v;
            curl[i] += cy[i] * dx - cx[i] * dy;
        }
    }
}

void RefSpaces2D::h1(double x, double y, double* L, double* gL) const {
    for (int i = 0; i < nl; ++i) { L[i] = 0.0; gL[2 * i] = gL[2 * i + 1] = 0.0; }
    for (int m = 0; m < nm; ++m) {
        const int a = mono[2 * m], b = mono[2 * m + 1];
        const double v = ipow(x, a) * ipow(y, b);
        const double dx = a > 0 ? a * ipow(x, a - 1) * ipow(y, b) : 0.0;
        const double dy = b > 0 ? b * ipow(x, a) * ipow(y, b - 1) : 0.0;
        const double* c = &CL[(size_t)m * nl];
        for (int i = 0; i < nl; ++i) {
            L[i] += c[i] * v;
            gL[2 * i] += c[i] * dx;
            gL[2 * i + 1] += c[i] * dy;
        }
    }
}

const RefSpaces2D& ref_spaces_2d(int p) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<RefSpaces2D>> cache;
    if (p < 1 || p > 8) throw std::runtime_error("2D element order must be 1..8");
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(p);
    if (it == cache.end()) it = cache.emplace(p, std::make_unique<RefSpaces2D>(build_ref_spaces(p))).first;
    return *it->second;
}

}  // namespace opem

namespace opem {

int port_mode_2d_pp(int64_t nnodes, const double* xy, int64_t ntri, const int64_t* tris, const cd* eps_r,
                    const cd* mu_r, double freq, int p, cd& beta, std::vector<cd>& ct, std::vector<cd>& cz,
                    std::vector<int64_t>& st, int mode) {
    if (nnodes < 3 || !xy || ntri < 1 || !tris || !eps_r || !(freq > 0) || p < 1 || p > 8 || mode < 0 || mode > 15)
        return OPEM_ERR_ARG;
    for (int64_t t = 0; t < 3 * ntri; ++t)
        if (tris[t] < 0 || tris[t] >= nnodes) return OPEM_ERR_ARG;
    const RefSpaces2D& R = ref_spaces_2d(p);
    static const int LP[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    const double k0 = 2 * M_PI * freq * std::sqrt(MU0 * EPS0);
    st.resize(3 * ntri);
    std::map<std::pair<int64_t, int64_t>, int> eid;
    for (int64_t t = 0; t < ntri; ++t) {
        int64_t v[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
        std::sort(v, v + 3);
        for (int k = 0; k < 3; ++k) st[3 * t + k] = v[k];
        for (auto& lp : LP) eid[{v[lp[0]], v[lp[1]]}] = 0;
    }
    int ne = 0;
    std::vector<std::pair<int64_t, int64_t>> edges;
    for (auto& kv : eid) { kv.second = ne++; edges.push_back(kv.first); }
    // global numbering: e_t = [edge moments (p per edge), interior (p (p-1) per triangle)],
    // e_z = [vertex (nnodes), edge nodes (p-1 per edge), interior ((p-1)(p-2)/2 per triangle)]
    const int nf = R.nf, nl = R.nl, nint = p * (p - 1), nle = p - 1, nli = (p - 1) * (p - 2) / 2;
    const int64_t net = (int64_t)ne * p + ntri * nint, nz = nnodes + (int64_t)ne * nle + ntri * nli;
    std::vector<int64_t> tdof((size_t)nf * ntri), zdof((size_t)nl * ntri);
    std::vector<int> ecount(ne, 0);
    for (int64_t t = 0; t < ntri; ++t) {
        int64_t* td = &tdof[(size_t)nf * t];
        int64_t* zd = &zdof[(size_t)nl * t];
        for (int i = 0; i < 3; ++i) {
            const int e = eid[{st[3 * t + LP[i][0]], st[3 * t + LP[i][1]]}];
            ++ecount[e];
            for (int k = 0; k < p; ++k) td[p * i + k] = (int64_t)e * p + k;
            for (int k = 0; k < nle; ++k) zd[3 + nle * i + k] = nnodes + (int64_t)e * nle + k;
            zd[i] = st[3 * t + i];
        }
        for (int j = 0; j < nint; ++j) td[3 * p + j] = (int64_t)ne * p + t * nint + j;
        for (int j = 0; j < nli; ++j) zd[3 + 3 * nle + j] = nnodes + (int64_t)ne * nle + t * nli + j;
    }
    if (net > INT32_MAX / 2 || nz > INT32_MAX / 2) return OPEM_ERR_ARG;
    // reference bases at the quadrature points (exact for the degree-2p products)
    std::vector<double> q1, q2, qw;
    tri_rule(2 * p + 1, q1, q2, qw);
    const int nq = (int)qw.size();
    std::vector<double> Nh((size_t)nq * nf * 2), Ch((size_t)nq * nf), Lh((size_t)nq * nl), Gh((size_t)nq * nl * 2);
    for (int q = 0; q < nq; ++q) {
        R.nd(q1[q], q2[q], &Nh[(size_t)q * nf * 2], &Ch[(size_t)q * nf]);
        R.h1(q1[q], q2[q], &Lh[(size_t)q * nl], &Gh[(size_t)q * nl * 2]);
    }
    std::vector<Triplet> Aee, Bee, Ben, Bnn;
    double emax = 0;
    std::vector<double> M((size_t)nf * nf), C((size_t)nf * nf), Gm((size_t)nf * nl), Kg((size_t)nl * nl),
        Ml((size_t)nl * nl), Np((size_t)nf * 2), Gp((size_t)nl * 2);
    for (int64_t t = 0; t < ntri; ++t) {
        const double* p0 = xy + 2 * st[3 * t];
        const double* p1 = xy + 2 * st[3 * t + 1];
        const double* p2 = xy + 2 * st[3 * t + 2];
        const double J00 = p1[0] - p0[0], J01 = p2[0] - p0[0], J10 = p1[1] - p0[1], J11 = p2[1] - p0[1];
        const double det = J00 * J11 - J01 * J10;
        if (!(std::fabs(det) > 0)) return OPEM_ERR_ARG;
        // J^-T = [[J11, -J10], [-J01, J00]] / det
        const double a00 = J11 / det, a01 = -J10 / det, a10 = -J01 / det, a11 = J00 / det;
        const cd er = eps_r[t], mr = mu_r ? mu_r[t] : cd(1.0), im = 1.0 / mr;
        emax = std::max(emax, std::real(er * mr));
        std::fill(M.begin(), M.end(), 0.0);
        std::fill(C.begin(), C.end(), 0.0);
        std::fill(Gm.begin(), Gm.end(), 0.0);
        std::fill(Kg.begin(), Kg.end(), 0.0);
        std::fill(Ml.begin(), Ml.end(), 0.0);
        for (int q = 0; q < nq; ++q) {
            const double w = qw[q] * std::fabs(det);
            const double* nh = &Nh[(size_t)q * nf * 2];
            const double* ch = &Ch[(size_t)q * nf];
            const double* lh = &Lh[(size_t)q * nl];
            const double* gh = &Gh[(size_t)q * nl * 2];
            for (int i = 0; i < nf; ++i) {
                Np[2 * i] = a00 * nh[2 * i] + a01 * nh[2 * i + 1];
                Np[2 * i + 1] = a10 * nh[2 * i] + a11 * nh[2 * i + 1];
            }
            for (int i = 0; i < nl; ++i) {
                Gp[2 * i] = a00 * gh[2 * i] + a01 * gh[2 * i + 1];
                Gp[2 * i + 1] = a10 * gh[2 * i] + a11 * gh[2 * i + 1];
            }
            for (int i = 0; i < nf; ++i) {
                const double ci = ch[i] / det;
                for (int j = 0; j < nf; ++j) {
                    M[(size_t)i * nf + j] += w * (Np[2 * i] * Np[2 * j] + Np[2 * i + 1] * Np[2 * j + 1]);
                    C[(size_t)i * nf + j] += w * ci * (ch[j] / det);
                }
                for (int j = 0; j < nl; ++j)
                    Gm[(size_t)i * nl + j] += w * (Np[2 * i] * Gp[2 * j] + Np[2 * i + 1] * Gp[2 * j + 1]);
            }
            for (int i = 0; i < nl; ++i)
                for (int j = 0; j < nl; ++j) {
                    Kg[(size_t)i * nl + j] += w * (Gp[2 * i] * Gp[2 * j] + Gp[2 * i + 1] * Gp[2 * j + 1]);
                    Ml[(size_t)i * nl + j] += w * lh[i] * lh[j];
                }
        }
        const int64_t* td = &tdof[(size_t)nf * t];
        const int64_t* zd = &zdof[(size_t)nl * t];
        for (int i = 0; i < nf; ++i) {
            for (int j = 0; j < nf; ++j) {
                Aee.push_back({(int)td[i], (int)td[j], im * C[(size_t)i * nf + j] - k0 * k0 * er * M[(size_t)i * nf + j]});
                Bee.push_back({(int)td[i], (int)td[j], im * M[(size_t)i * nf + j]});
            }
            for (int j = 0; j < nl; ++j) Ben.push_back({(int)td[i], (int)zd[j], -im * Gm[(size_t)i * nl + j]});
        }
        for (int i = 0; i < nl; ++i)
            for (int j = 0; j < nl; ++j)
                Bnn.push_back({(int)zd[i], (int)zd[j], im * Kg[(size_t)i * nl + j] - k0 * k0 * er * Ml[(size_t)i * nl + j]});
    }
    // PEC: every DOF of a boundary edge (its moments, its edge nodes) and its vertices
    std::vector<int> tmap(net, -1), zmap(nz, -1);
    std::vector<char> bnode(nnodes, 0), bedge(ne, 0);
    for (int e = 0; e < ne; ++e)
        if (ecount[e] == 1) { bedge[e] = 1; bnode[edges[e].first] = 1; bnode[edges[e].second] = 1; }
    int nu = 0;
    for (int64_t i = 0; i < net; ++i) {
        const bool drop = i < (int64_t)ne * p && bedge[i / p];
        if (!drop) tmap[i] = nu++;
    }
    const int nut = nu;
    std::vector<char> used(nnodes, 0);
    for (int64_t t = 0; t < 3 * ntri; ++t) used[tris[t]] = 1;
    for (int64_t i = 0; i < nz; ++i) {
        bool drop = false;
        if (i < nnodes) drop = !used[i] || bnode[i];
        else if (i < nnodes + (int64_t)ne * nle) drop = bedge[(i - nnodes) / nle];
        if (!drop) zmap[i] = nu++;
    }
    const int n = nu;
    if (nut == 0) return OPEM_ERR_ARG;
    std::vector<Triplet> A, Bm;
    for (auto& x : Aee) if (tmap[x.r] >= 0 && tmap[x.c] >= 0) A.push_back({tmap[x.r], tmap[x.c], x.v});
    for (auto& x : Bee) if (tmap[x.r] >= 0 && tmap[x.c] >= 0) Bm.push_back({tmap[x.r], tmap[x.c], x.v});
    for (auto& x : Ben)
        if (tmap[x.r] >= 0 && zmap[x.c] >= 0) {
            Bm.push_back({tmap[x.r], zmap[x.c], x.v});
            Bm.push_back({zmap[x.c], tmap[x.r], x.v});
        }
    for (auto& x : Bnn) if (zmap[x.r] >= 0 && zmap[x.c] >= 0) Bm.push_back({zmap[x.r], zmap[x.c], x.v});
    cd lam = 0;
    std::vector<cd> xs;
    int rc;
    if (mode == 0) {
        rc = solve_pencil(n, A, Bm, -k0 * k0 * emax, lam, xs, nut);
    } else {   // the mode-th mode in decreasing beta^2
        std::vector<cd> lams, X;
        rc = solve_pencil_k(n, A, Bm, -k0 * k0 * emax, mode + 1, lams, X, nut);
        if (rc == OPEM_OK) {
            lam = lams[mode];
            xs.assign(X.begin() + (size_t)mode * n, X.begin() + (size_t)(mode + 1) * n);
        }
    }
    if (rc != OPEM_OK) return rc;
    beta = std::sqrt(-lam);
    if (beta.real() < 0) beta = -beta;
    cd big = 0.0;
    for (int64_t i = 0; i < (int64_t)ne * p; ++i)
        if (tmap[i] >= 0 && std::abs(xs[tmap[i]]) > std::abs(big)) big = xs[tmap[i]];
    const cd sc = std::abs(big) > 0 ? 1.0 / big : cd(1.0);
    ct.assign((size_t)nf * ntri, 0.0);
    cz.assign((size_t)nl * ntri, 0.0);
    for (int64_t t = 0; t < ntri; ++t) {
        for (int i = 0; i < nf; ++i) {
            const int m = tmap[tdof[(size_t)nf * t + i]];
            ct[(size_t)nf * t + i] = m >= 0 ? xs[m] * sc : cd(0.0);
        }
        for (int i = 0; i < nl; ++i) {
            const int m = zmap[zdof[(size_t)nl * t + i]];
            cz[(size_t)nl * t + i] = m >= 0 ? -cd(0, 1) * beta * xs[m] * sc : cd(0.0);   // e_z = -j beta psi
        }
    }
    return OPEM_OK;
}

int project_nd_2d(int64_t nnodes, const double* xy, int64_t ntri, const int64_t* st, int p, const cd* weight,
                  const std::function<void(int64_t, double, double, cd&, cd&)>& field, std::vector<cd>& ch) {
    if (nnodes < 3 || !xy || ntri < 1 || !st || p < 1 || p > 8 || !weight) return OPEM_ERR_ARG;
    const RefSpaces2D& R = ref_spaces_2d(p);
    static const int LP[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    // numbering: p moments per edge (edges of sorted vertex pairs), p (p-1) per triangle
    std::map<std::pair<int64_t, int64_t>, int> eid;
    for (int64_t t = 0; t < ntri; ++t)
        for (auto& lp : LP) eid[{st[3 * t + lp[0]], st[3 * t + lp[1]]}] = 0;
    int ne = 0;
    for (auto& kv : eid) kv.second = ne++;
    const int nf = R.nf, nint = p * (p - 1);
    const int64_t n = (int64_t)ne * p + ntri * nint;
    if (n > INT32_MAX / 2) return OPEM_ERR_ARG;
    std::vector<int> tdof((size_t)nf * ntri);
    for (int64_t t = 0; t < ntri; ++t) {
        for (int i = 0; i < 3; ++i) {
            const int e = eid[{st[3 * t + LP[i][0]], st[3 * t + LP[i][1]]}];
            for (int k = 0; k < p; ++k) tdof[(size_t)nf * t + p * i + k] = e * p + k;
        }
        for (int j = 0; j < nint; ++j) tdof[(size_t)nf * t + 3 * p + j] = (int)(ne * p + t * nint + j);
    }
    std::vector<double> q1, q2, qw;
    tri_rule(2 * p + 2, q1, q2, qw);
    const int nq = (int)qw.size();
    std::vector<double> Nh((size_t)nq * nf * 2), Ch((size_t)nf);
    for (int q = 0; q < nq; ++q) R.nd(q1[q], q2[q], &Nh[(size_t)q * nf * 2], Ch.data());
    std::vector<Triplet> Mt;
    Mt.reserve((size_t)ntri * nf * nf);
    std::vector<cd> rhs(n, 0.0), Ml((size_t)nf * nf);
    std::vector<double> Np((size_t)nf * 2);
    for (int64_t t = 0; t < ntri; ++t) {
        const double* p0 = xy + 2 * st[3 * t];
        const double* p1 = xy + 2 * st[3 * t + 1];
        const double* p2 = xy + 2 * st[3 * t + 2];
        const double J00 = p1[0] - p0[0], J01 = p2[0] - p0[0], J10 = p1[1] - p0[1], J11 = p2[1] - p0[1];
        const double det = J00 * J11 - J01 * J10;
        if (!(std::fabs(det) > 0)) return OPEM_ERR_ARG;
        const double a00 = J11 / det, a01 = -J10 / det, a10 = -J01 / det, a11 = J00 / det;   // J^-T
        std::fill(Ml.begin(), Ml.end(), 0.0);
        const int* td = &tdof[(size_t)nf * t];
        for (int q = 0; q < nq; ++q) {
            const cd w = qw[q] * std::fabs(det) * weight[t];
            const double* nh = &Nh[(size_t)q * nf * 2];
            for (int i = 0; i < nf; ++i) {
                Np[2 * i] = a00 * nh[2 * i] + a01 * nh[2 * i + 1];
                Np[2 * i + 1] = a10 * nh[2 * i] + a11 * nh[2 * i + 1];
            }
            cd fx, fy;
            field(t, p0[0] + q1[q] * J00 + q2[q] * J01, p0[1] + q1[q] * J10 + q2[q] * J11, fx, fy);
            for (int i = 0; i < nf; ++i) {
                rhs[td[i]] += w * (Np[2 * i] * fx + Np[2 * i + 1] * fy);
                for (int j = 0; j < nf; ++j)
                    Ml[(size_t)i * nf + j] += w * (Np[2 * i] * Np[2 * j] + Np[2 * i + 1] * Np[2 * j + 1]);
            }
        }
        for (int i = 0; i < nf; ++i)
            for (int j = 0; j < nf; ++j) Mt.push_back({td[i], td[j], Ml[(size_t)i * nf + j]});
    }
    // banded LU in reverse Cuthill-McKee order
    std::vector<std::vector<int>> adj(n);
    for (auto& x : Mt)
        if (x.r != x.c) adj[x.r].push_back(x.c);
    for (auto& a : adj) { std::sort(a.begin(), a.end()); a.erase(std::unique(a.begin(), a.end()), a.end()); }
    const std::vector<int> ord = rcm((int)n, adj);
    std::vector<int> pos(n);
    for (int64_t i = 0; i < n; ++i) pos[ord[i]] = (int)i;
    int bw = 0;
    for (int64_t i = 0; i < n; ++i)
        for (int j : adj[i]) bw = std::max(bw, std::abs(pos[i] - pos[j]));
    Banded B;
    B.init((int)n, bw, bw);
    for (auto& x : Mt) B.at(pos[x.r], pos[x.c]) += x.v;
    if (!B.factor()) return OPEM_ERR_BREAKDOWN;
    std::vector<cd> b(n);
    for (int64_t i = 0; i < n; ++i) b[pos[i]] = rhs[i];
    B.solve(b);
    ch.assign((size_t)nf * ntri, 0.0);
    for (int64_t t = 0; t < ntri; ++t)
        for (int i = 0; i < nf; ++i) ch[(size_t)nf * t + i] = b[pos[tdof[(size_t)nf * t + i]]];
    return OPEM_OK;
}

}  // namespace opem
