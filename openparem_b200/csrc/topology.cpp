// Mesh topology, DOF numbering, CSR pattern and vertex patches (host).
//
// Replaces the DOF bookkeeping MFEM does for ND_FECollection(p,3) on the
// reference's ParMesh (src/OpenParEM3D/fem3D.cpp:65-78) and the sparsity
// that hypre/PETSc build in hypre_ParCSRMatrixToMat (src/OpenParEM3D/csr.c:171-223).
// Global DOF order: edges (p each), faces (p(p-1) each), element interiors.
#include "opem_internal.h"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace opem {

static const int EDGES[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
static const int FACES[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

template <class K>
static void sort_unique_ids(const std::vector<K>& keys, std::vector<int32_t>& inv, int64_t& nuniq) {
    size_t m = keys.size();
    std::vector<int64_t> order(m);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });
    inv.assign(m, -1);
    int64_t u = -1;
    for (size_t i = 0; i < m; ++i) {
        if (i == 0 || keys[order[i]] != keys[order[i - 1]]) ++u;
        inv[order[i]] = (int32_t)u;
    }
    nuniq = u + 1;
}

int build_topology(Topology& T, int64_t nv, const double* verts, int64_t ne, const int64_t* tets,
                   const int32_t* region, int64_t nb, const int64_t* bdr, const int32_t* battr, int p,
                   std::string& err) {
    if (nv <= 0 || ne <= 0 || !verts || !tets) { err = "empty mesh"; return OPEM_ERR_ARG; }
    if (nv >= (1LL << 31) || ne >= (1LL << 31) / 8) { err = "mesh too large for int32 ids"; return OPEM_ERR_ARG; }
    const NDRef& R = nd_reference(p);
    T.p = p; T.ld = R.ld; T.ldf = R.ldf;
    T.nv = nv; T.ne = ne;
    T.verts.assign(verts, verts + 3 * nv);
    T.tets.resize(4 * ne);
    T.region.resize(ne);
    for (int64_t e = 0; e < ne; ++e) {
        int64_t v[4] = {tets[4 * e], tets[4 * e + 1], tets[4 * e + 2], tets[4 * e + 3]};
        for (int k = 0; k < 4; ++k)
            if (v[k] < 0 || v[k] >= nv) { err = "tet vertex id out of range"; return OPEM_ERR_MESH; }
        std::sort(v, v + 4);
        if (v[0] == v[1] || v[1] == v[2] || v[2] == v[3]) { err = "degenerate tet"; return OPEM_ERR_MESH; }
        for (int k = 0; k < 4; ++k) T.tets[4 * e + k] = (int32_t)v[k];
        T.region[e] = region ? region[e] : 0;
    }
    // edges
    std::vector<int64_t> ek(6 * ne);
    for (int64_t e = 0; e < ne; ++e)
        for (int l = 0; l < 6; ++l)
            ek[6 * e + l] = (int64_t)T.tets[4 * e + EDGES[l][0]] * nv + T.tets[4 * e + EDGES[l][1]];
    sort_unique_ids(ek, T.tet_edges, T.nE);
    // faces: key = (a*nv + b)*nv + c may overflow int64 for nv > 2^21; use pairs
    std::vector<std::pair<int64_t, int32_t>> fk(4 * ne);
    for (int64_t e = 0; e < ne; ++e)
        for (int l = 0; l < 4; ++l) {
            const int32_t* t = &T.tets[4 * e];
            fk[4 * e + l] = {(int64_t)t[FACES[l][0]] * nv + t[FACES[l][1]], t[FACES[l][2]]};
        }
    sort_unique_ids(fk, T.tet_faces, T.nF);
    T.face_owner.assign(T.nF, -1);
    T.face_lface.assign(T.nF, -1);
    for (int64_t e = 0; e < ne; ++e)
        for (int l = 0; l < 4; ++l) {
            int32_t f = T.tet_faces[4 * e + l];
            if (T.face_owner[f] < 0) { T.face_owner[f] = (int32_t)e; T.face_lface[f] = l; }
        }
    // dofs
    int nfd = p * (p - 1), nid = p * (p - 1) * (p - 2) / 2;
    int64_t base_f = T.nE * p, base_i = base_f + T.nF * nfd;
    T.n = base_i + ne * nid;
    if (T.n >= (1LL << 31)) { err = "too many dofs for int32"; return OPEM_ERR_ARG; }
    T.elem_dofs.resize((size_t)ne * T.ld);
    for (int64_t e = 0; e < ne; ++e) {
        int32_t* d = &T.elem_dofs[(size_t)e * T.ld];
        int c = 0;
        for (int l = 0; l < 6; ++l)
            for (int k = 0; k < p; ++k) d[c++] = (int32_t)(T.tet_edges[6 * e + l] * (int64_t)p + k);
        for (int l = 0; l < 4; ++l)
            for (int k = 0; k < nfd; ++k) d[c++] = (int32_t)(base_f + T.tet_faces[4 * e + l] * (int64_t)nfd + k);
        for (int k = 0; k < nid; ++k) d[c++] = (int32_t)(base_i + e * nid + k);
    }
    // boundary triangles -> faces (binary search in the sorted face keys)
    std::vector<std::pair<std::pair<int64_t, int32_t>, int32_t>> fsorted;
    fsorted.reserve(T.nF);
    for (int64_t e = 0; e < ne; ++e)
        for (int l = 0; l < 4; ++l) {
            int32_t f = T.tet_faces[4 * e + l];
            if (T.face_owner[f] == e && T.face_lface[f] == l) fsorted.push_back({fk[4 * e + l], f});
        }
    std::sort(fsorted.begin(), fsorted.end());
    T.bdr_face.resize(nb);
    T.bdr_attr.resize(nb);
    for (int64_t b = 0; b < nb; ++b) {
        int64_t v[3] = {bdr[3 * b], bdr[3 * b + 1], bdr[3 * b + 2]};
        std::sort(v, v + 3);
        std::pair<int64_t, int32_t> key = {v[0] * nv + v[1], (int32_t)v[2]};
        auto it = std::lower_bound(fsorted.begin(), fsorted.end(), std::make_pair(key, (int32_t)-1));
        if (it == fsorted.end() || it->first != key) { err = "boundary triangle is not a mesh face"; return OPEM_ERR_MESH; }
        T.bdr_face[b] = it->second;
        T.bdr_attr[b] = battr ? battr[b] : 1;
    }
    return OPEM_OK;
}

int build_pattern(Topology& T, std::string& err) {
    const int64_t n = T.n, ne = T.ne;
    const int ld = T.ld;
    // dof -> (elem, local) lists
    T.d2e_ptr.assign(n + 1, 0);
    for (size_t k = 0; k < T.elem_dofs.size(); ++k) T.d2e_ptr[T.elem_dofs[k] + 1]++;
    for (int64_t i = 0; i < n; ++i) T.d2e_ptr[i + 1] += T.d2e_ptr[i];
    T.d2e_elem.resize(T.elem_dofs.size());
    T.d2e_loc.resize(T.elem_dofs.size());
    {
        std::vector<int32_t> fill(T.d2e_ptr.begin(), T.d2e_ptr.end() - 1);
        for (int64_t e = 0; e < ne; ++e)
            for (int i = 0; i < ld; ++i) {
                int32_t d = T.elem_dofs[(size_t)e * ld + i];
                int32_t pos = fill[d]++;
                T.d2e_elem[pos] = (int32_t)e;
                T.d2e_loc[pos] = (uint8_t)i;
            }
    }
    // row patterns
    std::vector<int32_t> rowlen(n, 0);
#pragma omp parallel
    {
        std::vector<int32_t> buf;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t r = 0; r < n; ++r) {
            buf.clear();
            for (int32_t k = T.d2e_ptr[r]; k < T.d2e_ptr[r + 1]; ++k) {
                const int32_t* d = &T.elem_dofs[(size_t)T.d2e_elem[k] * ld];
                buf.insert(buf.end(), d, d + ld);
            }
            std::sort(buf.begin(), buf.end());
            rowlen[r] = (int32_t)(std::unique(buf.begin(), buf.end()) - buf.begin());
        }
    }
    T.rowptr.assign(n + 1, 0);
    int64_t nnz = 0;
    for (int64_t r = 0; r < n; ++r) {
        nnz += rowlen[r];
        if (nnz >= (1LL << 31)) { err = "nnz exceeds int32"; return OPEM_ERR_ARG; }
        T.rowptr[r + 1] = (int32_t)nnz;
    }
    T.cols.resize(nnz);
#pragma omp parallel
    {
        std::vector<int32_t> buf;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t r = 0; r < n; ++r) {
            buf.clear();
            for (int32_t k = T.d2e_ptr[r]; k < T.d2e_ptr[r + 1]; ++k) {
                const int32_t* d = &T.elem_dofs[(size_t)T.d2e_elem[k] * ld];
                buf.insert(buf.end(), d, d + ld);
            }
            std::sort(buf.begin(), buf.end());
            auto endu = std::unique(buf.begin(), buf.end());
            std::copy(buf.begin(), endu, T.cols.begin() + T.rowptr[r]);
        }
    }
    return OPEM_OK;
}

// Vertex patches (Arnold-Falk-Winther): for every vertex the dofs of its
// incident edges, faces and elements, minus PEC dofs.  Each patch's dense
// block is inverted for the overlapping block-Jacobi preconditioner.
int build_patches(Topology& T, const std::vector<uint8_t>& pec, std::string& err) {
    const int p = T.p, ld = T.ld;
    const int nfd = p * (p - 1);
    std::vector<std::vector<int32_t>> lists(T.nv);
    for (int64_t e = 0; e < T.ne; ++e) {
        const int32_t* d = &T.elem_dofs[(size_t)e * ld];
        for (int lv = 0; lv < 4; ++lv) {
            auto& L = lists[T.tets[4 * e + lv]];
            for (int le = 0; le < 6; ++le)
                if (EDGES[le][0] == lv || EDGES[le][1] == lv)
                    for (int k = 0; k < p; ++k) L.push_back(d[le * p + k]);
            for (int lf = 0; lf < 4; ++lf)
                if (FACES[lf][0] == lv || FACES[lf][1] == lv || FACES[lf][2] == lv)
                    for (int k = 0; k < nfd; ++k) L.push_back(d[6 * p + lf * nfd + k]);
            for (int k = 6 * p + 4 * nfd; k < ld; ++k) L.push_back(d[k]);
        }
    }
    T.patch_ptr.assign(1, 0);
    T.patch_dofs.clear();
    T.patch_off.assign(1, 0);
    T.max_patch = 0;
    for (int64_t v = 0; v < T.nv; ++v) {
        auto& L = lists[v];
        std::sort(L.begin(), L.end());
        L.erase(std::unique(L.begin(), L.end()), L.end());
        std::vector<int32_t> keep;
        for (int32_t d : L)
            if (!pec[d]) keep.push_back(d);
        if (keep.empty()) continue;
        T.patch_dofs.insert(T.patch_dofs.end(), keep.begin(), keep.end());
        T.patch_ptr.push_back((int32_t)T.patch_dofs.size());
        int64_t s = (int64_t)keep.size();
        T.patch_off.push_back(T.patch_off.back() + s * s);
        T.max_patch = std::max<int>(T.max_patch, (int)s);
        std::vector<int32_t>().swap(L);
    }
    (void)err;
    return OPEM_OK;
}

}  // namespace opem
