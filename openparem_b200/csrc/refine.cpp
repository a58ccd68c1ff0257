// Conforming refinement of marked tetrahedra (host).
//
// The reference refines the elements its error indicator marks with MFEM's
// ParMesh::GeneralRefinement (fem3D::refineMesh, src/OpenParEM3D/fem3D.cpp:
// 1426-1447) and solves again on the refined mesh.  Here the marked
// tetrahedra are bisected at their longest edge and the mesh is closed by
// longest-edge bisection (Rivara): any tetrahedron with a bisected edge is
// bisected at its own longest edge until no tetrahedron has a bisected edge.
// A tetrahedron's longest edge is also the longest edge of the two faces that
// contain it, so every face, interior or on the boundary, is split at its own
// longest edge; the boundary triangles are refined by the same rule and stay
// matched to the tetrahedra's faces.  Edge lengths are compared with a global
// tie-break on the vertex ids, so the result does not depend on the order the
// tetrahedra are visited.  The refined mesh keeps every region and boundary
// attribute; its new vertices are the edge midpoints.
#include <algorithm>
#include <array>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "../../include/opem_b200.h"

namespace {

struct Mesh {
    std::vector<double> X;                                 // 3 per vertex
    std::map<std::pair<int64_t, int64_t>, int64_t> mid;    // edge (lo, hi) -> midpoint vertex

    double len2(int64_t a, int64_t b) const {
        double s = 0;
        for (int c = 0; c < 3; ++c) {
            const double d = X[3 * a + c] - X[3 * b + c];
            s += d * d;
        }
        return s;
    }
    // strict "longer than" on edges: squared length, then the sorted vertex ids
    bool longer(int64_t a, int64_t b, int64_t c, int64_t d) const {
        const double l1 = len2(a, b), l2 = len2(c, d);
        if (l1 != l2) return l1 > l2;
        const auto k1 = std::make_pair(std::min(a, b), std::max(a, b));
        const auto k2 = std::make_pair(std::min(c, d), std::max(c, d));
        return k1 > k2;
    }
    int64_t midpoint(int64_t a, int64_t b) {
        const auto k = std::make_pair(std::min(a, b), std::max(a, b));
        auto it = mid.find(k);
        if (it != mid.end()) return it->second;
        const int64_t m = (int64_t)X.size() / 3;
        for (int c = 0; c < 3; ++c) X.push_back(0.5 * (X[3 * k.first + c] + X[3 * k.second + c]));
        mid.emplace(k, m);
        return m;
    }
    bool split(int64_t a, int64_t b) const { return mid.count({std::min(a, b), std::max(a, b)}) > 0; }
};

// longest edge (i, j) of a cell with n = 3 or 4 vertices
template <int N>
void longest(const Mesh& M, const std::array<int64_t, N>& v, int& i0, int& j0) {
    i0 = 0;
    j0 = 1;
    for (int i = 0; i < N; ++i)
        for (int j = i + 1; j < N; ++j)
            if (M.longer(v[i], v[j], v[i0], v[j0])) { i0 = i; j0 = j; }
}

template <int N>
bool has_split_edge(const Mesh& M, const std::array<int64_t, N>& v) {
    for (int i = 0; i < N; ++i)
        for (int j = i + 1; j < N; ++j)
            if (M.split(v[i], v[j])) return true;
    return false;
}

// bisection at the longest edge: the two children replace vertex j0 resp. i0 by the midpoint
template <int N>
void bisect(Mesh& M, const std::array<int64_t, N>& v, std::array<int64_t, N>& c1, std::array<int64_t, N>& c2) {
    int i0, j0;
    longest<N>(M, v, i0, j0);
    const int64_t m = M.midpoint(v[i0], v[j0]);
    c1 = v;
    c2 = v;
    c1[j0] = m;
    c2[i0] = m;
}

}  // namespace

extern "C" int opem_refine_mesh(int64_t nverts, const double* verts, int64_t ntets, const int64_t* tets,
                                const int32_t* region, int64_t nbdr, const int64_t* bdr_tris, const int32_t* bdr_attr,
                                int64_t nmarked, const int64_t* marked, int64_t* counts, double* verts_out,
                                int64_t* tets_out, int32_t* region_out, int64_t* bdr_out, int32_t* attr_out) {
    if (nverts < 4 || !verts || ntets < 1 || !tets || nbdr < 0 || (nbdr > 0 && (!bdr_tris || !bdr_attr)) ||
        nmarked < 0 || (nmarked > 0 && !marked) || !counts)
        return OPEM_ERR_ARG;
    for (int64_t i = 0; i < 4 * ntets; ++i)
        if (tets[i] < 0 || tets[i] >= nverts) return OPEM_ERR_ARG;
    for (int64_t i = 0; i < 3 * nbdr; ++i)
        if (bdr_tris[i] < 0 || bdr_tris[i] >= nverts) return OPEM_ERR_ARG;
    for (int64_t i = 0; i < nmarked; ++i)
        if (marked[i] < 0 || marked[i] >= ntets) return OPEM_ERR_ARG;
    Mesh M;
    M.X.assign(verts, verts + 3 * nverts);
    std::vector<std::array<int64_t, 4>> T(ntets);
    std::vector<int32_t> R(ntets, 0);
    for (int64_t e = 0; e < ntets; ++e) {
        for (int k = 0; k < 4; ++k) T[e][k] = tets[4 * e + k];
        if (region) R[e] = region[e];
    }
    // marked tetrahedra: one bisection each
    std::vector<char> mk(ntets, 0);
    for (int64_t i = 0; i < nmarked; ++i) mk[marked[i]] = 1;
    std::vector<std::array<int64_t, 4>> cur;
    std::vector<int32_t> curR;
    for (int64_t e = 0; e < ntets; ++e) {
        if (mk[e]) {
            std::array<int64_t, 4> a, b;
            bisect<4>(M, T[e], a, b);
            cur.push_back(a); curR.push_back(R[e]);
            cur.push_back(b); curR.push_back(R[e]);
        } else {
            cur.push_back(T[e]); curR.push_back(R[e]);
        }
    }
    // closure: bisect every tetrahedron with a bisected edge until none has one
    std::vector<std::array<int64_t, 4>> done;
    std::vector<int32_t> doneR;
    std::deque<std::pair<std::array<int64_t, 4>, int32_t>> work;
    for (size_t i = 0; i < cur.size(); ++i) work.push_back({cur[i], curR[i]});
    bool changed = true;
    while (changed) {
        changed = false;
        done.clear();
        doneR.clear();
        while (!work.empty()) {
            auto w = work.front();
            work.pop_front();
            if (has_split_edge<4>(M, w.first)) {
                std::array<int64_t, 4> a, b;
                bisect<4>(M, w.first, a, b);
                work.push_back({a, w.second});
                work.push_back({b, w.second});
                changed = true;
            } else {
                done.push_back(w.first);
                doneR.push_back(w.second);
            }
        }
        // a bisection late in the pass may have split an edge of a tetrahedron already kept
        if (changed)
            for (size_t i = 0; i < done.size(); ++i) work.push_back({done[i], doneR[i]});
    }
    // boundary triangles by the same rule
    std::vector<std::array<int64_t, 3>> B;
    std::vector<int32_t> BA;
    std::deque<std::pair<std::array<int64_t, 3>, int32_t>> bw;
    for (int64_t f = 0; f < nbdr; ++f) bw.push_back({{bdr_tris[3 * f], bdr_tris[3 * f + 1], bdr_tris[3 * f + 2]}, bdr_attr[f]});
    while (!bw.empty()) {
        auto w = bw.front();
        bw.pop_front();
        if (has_split_edge<3>(M, w.first)) {
            int i0, j0;
            longest<3>(M, w.first, i0, j0);
            if (!M.split(w.first[i0], w.first[j0])) return OPEM_ERR_MESH;   // a face not split at its longest edge
            std::array<int64_t, 3> a, b;
            bisect<3>(M, w.first, a, b);
            bw.push_back({a, w.second});
            bw.push_back({b, w.second});
        } else {
            B.push_back(w.first);
            BA.push_back(w.second);
        }
    }
    const int64_t nv = (int64_t)M.X.size() / 3, nt = (int64_t)done.size(), nb = (int64_t)B.size();
    counts[0] = nv;
    counts[1] = nt;
    counts[2] = nb;
    if (verts_out) std::memcpy(verts_out, M.X.data(), M.X.size() * sizeof(double));
    for (int64_t e = 0; e < nt; ++e) {
        if (tets_out)
            for (int k = 0; k < 4; ++k) tets_out[4 * e + k] = done[e][k];
        if (region_out) region_out[e] = doneR[e];
    }
    for (int64_t f = 0; f < nb; ++f) {
        if (bdr_out)
            for (int k = 0; k < 3; ++k) bdr_out[3 * f + k] = B[f][k];
        if (attr_out) attr_out[f] = BA[f];
    }
    return OPEM_OK;
}
