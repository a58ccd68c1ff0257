// Element-batched assembly of the frequency-independent operators.
//
// Restates the MFEM integrators the reference adds in fem3D::build_A / build_P /
// build_Q (src/OpenParEM3D/fem3D.cpp:115-123, :153-162, :195-216) and the
// boundary integrators of Port::addPortIntegrators (src/OpenParEM3D/port.cpp:5783-5875)
// and Boundary::addImpedanceIntegrator (port.cpp:1009-1041):
//   K    = sum_e (1/mu_r) int curl u_i . curl u_j        (CurlCurlIntegrator)
//   Meps = sum_e eps_r   int u_i . u_j                    (VectorFEMassIntegrator)
//   Q    = sum_e (1/mu_r) int u_i . curl u_j              (MixedVectorCurlIntegrator)
//   port / wall terms: int_F curl_s u curl_s v, int_F u_t . v_t
// On affine tetrahedra each element matrix is a 6-term combination of
// reference tensors with the element's metric, so the kernel only needs 13
// doubles of geometry per element and the reference tables in shared memory.
//
// Assembly is row-owned: one warp owns one CSR row and walks the elements
// that contain the row's DOF in a fixed order, so the sums are deterministic
// and need no atomics.
#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>

#include "engine.h"

namespace opem {

__constant__ int c_faces[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

__global__ void geo_kernel(int64_t ne, const double* __restrict__ verts, const int32_t* __restrict__ tets,
                           ElemGeo* __restrict__ geo) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    double P[4][3];
    for (int k = 0; k < 4; ++k)
        for (int d = 0; d < 3; ++d) P[k][d] = verts[3 * (int64_t)tets[4 * e + k] + d];
    double J[3][3];   // columns P1-P0, P2-P0, P3-P0
    for (int d = 0; d < 3; ++d)
        for (int c = 0; c < 3; ++c) J[d][c] = P[c + 1][d] - P[0][d];
    double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                 J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    double id = 1.0 / det;
    double Ji[3][3];
    Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
    Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
    Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
    Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
    Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
    Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
    Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
    Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
    Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    const int SA[6] = {0, 1, 2, 0, 0, 1}, SB[6] = {0, 1, 2, 1, 2, 2};
    double ad = fabs(det);
    ElemGeo g;
    for (int s = 0; s < 6; ++s) {
        int a = SA[s], b = SB[s];
        double C = J[0][a] * J[0][b] + J[1][a] * J[1][b] + J[2][a] * J[2][b];      // (J^T J)_ab
        double G = Ji[a][0] * Ji[b][0] + Ji[a][1] * Ji[b][1] + Ji[a][2] * Ji[b][2];  // (J^-1 J^-T)_ab
        g.gK[s] = C / ad;
        g.gM[s] = ad * G;
    }
    g.sgn = det > 0 ? 1.0 : -1.0;
    g.pad = det;
    geo[e] = g;
}

__device__ inline int32_t row_find(const int32_t* __restrict__ c, int32_t lo, int32_t hi, int32_t col) {
    while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (c[mid] < col) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// One warp per CSR row; LD = local dofs per element.
template <int LD>
__global__ void __launch_bounds__(256) assemble_rows_kernel(
    int64_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
    const int32_t* __restrict__ d2e_ptr, const int32_t* __restrict__ d2e_elem, const uint8_t* __restrict__ d2e_loc,
    const int32_t* __restrict__ elem_dofs, const ElemGeo* __restrict__ geo, const double* __restrict__ ecoef,
    const double* __restrict__ ref, double* __restrict__ K, double* __restrict__ Meps, double* __restrict__ Mtand,
    double* __restrict__ Msig, double* __restrict__ M1, double* __restrict__ Q) {
    extern __shared__ double sref[];   // Kh(6 LD^2) | Mh(6 LD^2) | Qh(LD^2)
    const int T = 13 * LD * LD;
    for (int t = threadIdx.x; t < T; t += blockDim.x) sref[t] = ref[t];
    __syncthreads();
    const double* Kh = sref;
    const double* Mh = sref + 6 * LD * LD;
    const double* Qh = sref + 12 * LD * LD;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
        const int32_t rs = rowptr[r], re = rowptr[r + 1];
        for (int32_t k = rs + lane; k < re; k += 32) {
            K[k] = 0; Meps[k] = 0; M1[k] = 0; Q[k] = 0;
            if (Mtand) Mtand[k] = 0;
            if (Msig) Msig[k] = 0;
        }
        __syncwarp();
        for (int32_t t = d2e_ptr[r]; t < d2e_ptr[r + 1]; ++t) {
            const int32_t e = d2e_elem[t];
            const int i = d2e_loc[t];
            const ElemGeo g = geo[e];
            const double inv_mu = ecoef[4 * e + 0], eps = ecoef[4 * e + 1], epst = ecoef[4 * e + 2], sig = ecoef[4 * e + 3];
            for (int j = lane; j < LD; j += 32) {
                const int32_t col = elem_dofs[(int64_t)e * LD + j];
                const int32_t pos = row_find(cols, rs, re, col);
                double kv = 0, mv = 0;
#pragma unroll
                for (int s = 0; s < 6; ++s) {
                    kv += g.gK[s] * Kh[(s * LD + i) * LD + j];
                    mv += g.gM[s] * Mh[(s * LD + i) * LD + j];
                }
                const double qv = Qh[i * LD + j];
                K[pos] += inv_mu * kv;
                Meps[pos] += eps * mv;
                M1[pos] += mv;
                Q[pos] += inv_mu * g.sgn * qv;
                if (Mtand) Mtand[pos] += epst * mv;
                if (Msig) Msig[pos] += sig * mv;
            }
            __syncwarp();
        }
    }
}

__global__ void elem_coef_kernel(int64_t ne, const int32_t* __restrict__ region, const double* __restrict__ mat,
                                 int nreg, double* __restrict__ ecoef) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int r = region[e];
    r = r < 0 ? 0 : (r >= nreg ? nreg - 1 : r);
    double er = mat[4 * r + 0], td = mat[4 * r + 1], sg = mat[4 * r + 2], mr = mat[4 * r + 3];
    ecoef[4 * e + 0] = 1.0 / mr;
    ecoef[4 * e + 1] = er;
    ecoef[4 * e + 2] = er * td;
    ecoef[4 * e + 3] = sg;
}

template <int LD>
static void launch_assemble(Problem& P, cudaStream_t s) {
    size_t smem = (size_t)13 * LD * LD * sizeof(double);
    auto kern = assemble_rows_kernel<LD>;
    OPEM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int bpsm = 1;
    OPEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kern, 256, smem));
    int grid = std::max(1, bpsm) * P.ctx->sm_count;
    kern<<<grid, 256, smem, s>>>(P.topo.n, P.d_rowptr.p, P.d_cols.p, P.d_d2e_ptr.p, P.d_d2e_elem.p, P.d_d2e_loc.p,
                                 P.d_elem_dofs.p, P.d_geo.p, P.d_elemcoef.p, P.d_ref.p, P.d_K.p, P.d_Meps.p,
                                 P.has_tand ? P.d_Mtand.p : nullptr, P.has_sig ? P.d_Msig.p : nullptr, P.d_M1.p, P.d_Q.p); ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
}

__global__ void to_float_kernel(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

void assemble_volume(Problem& P) {
    cudaStream_t s = P.ctx->stream;
    Topology& T = P.topo;
    const NDRef& R = nd_reference(T.p);
    const int ld = T.ld;
    P.d_verts.upload(T.verts, s);
    P.d_tets.upload(T.tets, s);
    P.d_region.upload(T.region, s);
    P.d_elem_dofs.upload(T.elem_dofs, s);
    P.d_rowptr.upload(T.rowptr, s);
    P.d_cols.upload(T.cols, s);
    P.d_d2e_ptr.upload(T.d2e_ptr, s);
    P.d_d2e_elem.upload(T.d2e_elem, s);
    P.d_d2e_loc.upload(T.d2e_loc, s);
    // reference tables
    std::vector<double> ref((size_t)13 * ld * ld);
    std::copy(R.Kh.begin(), R.Kh.end(), ref.begin());
    std::copy(R.Mh.begin(), R.Mh.end(), ref.begin() + (size_t)6 * ld * ld);
    std::copy(R.Qh.begin(), R.Qh.end(), ref.begin() + (size_t)12 * ld * ld);
    P.d_ref.upload(ref, s);
    // element geometry and material coefficients
    P.d_geo.alloc(T.ne);
    geo_kernel<<<(unsigned)((T.ne + 255) / 256), 256, 0, s>>>(T.ne, P.d_verts.p, P.d_tets.p, P.d_geo.p); ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
    std::vector<double> mat(4 * P.nregions);
    P.has_tand = P.has_sig = false;
    for (int r = 0; r < P.nregions; ++r) {
        mat[4 * r + 0] = P.eps_r[r]; mat[4 * r + 1] = P.tand[r]; mat[4 * r + 2] = P.sigma[r]; mat[4 * r + 3] = P.mu_r[r];
        if (P.tand[r] != 0.0) P.has_tand = true;
        if (P.sigma[r] != 0.0) P.has_sig = true;
    }
    DBuf<double> d_mat;
    d_mat.upload(mat, s);
    P.d_elemcoef.alloc(4 * T.ne);
    elem_coef_kernel<<<(unsigned)((T.ne + 255) / 256), 256, 0, s>>>(T.ne, P.d_region.p, d_mat.p, P.nregions, P.d_elemcoef.p); ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
    size_t nnz = T.cols.size();
    P.d_K.alloc(nnz); P.d_Meps.alloc(nnz); P.d_M1.alloc(nnz); P.d_Q.alloc(nnz);
    if (P.has_tand) P.d_Mtand.alloc(nnz); else P.d_Mtand.release();
    if (P.has_sig) P.d_Msig.alloc(nnz); else P.d_Msig.release();
    switch (ld) {
        case 6: launch_assemble<6>(P, s); break;
        case 20: launch_assemble<20>(P, s); break;
        case 45: launch_assemble<45>(P, s); break;
        default: throw OpemError(OPEM_ERR_UNSUPPORTED, "GPU assembly supports Nedelec orders 1..3");
    }
    OPEM_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------------------
// boundary groups
// ---------------------------------------------------------------------------
struct FaceGeo { double A2, gi00, gi11, gi01, w_mu, w_eps, w_tand, w_sig; int lf, pad; };

__global__ void face_geo_kernel(int nf, const int32_t* __restrict__ faces, const int32_t* __restrict__ owner,
                                const int32_t* __restrict__ lface, const int32_t* __restrict__ tets,
                                const double* __restrict__ verts, const double* __restrict__ ecoef, FaceGeo* __restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    int f = faces[k];
    int t = owner[f], lf = lface[f];
    const int32_t* tv = &tets[4 * (int64_t)t];
    double a[3], b[3], c[3];
    for (int d = 0; d < 3; ++d) {
        a[d] = verts[3 * (int64_t)tv[c_faces[lf][0]] + d];
        b[d] = verts[3 * (int64_t)tv[c_faces[lf][1]] + d];
        c[d] = verts[3 * (int64_t)tv[c_faces[lf][2]] + d];
    }
    double t1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    double t2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    double g11 = t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2];
    double g22 = t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2];
    double g12 = t1[0] * t2[0] + t1[1] * t2[1] + t1[2] * t2[2];
    double det = g11 * g22 - g12 * g12;
    double N[3] = {t1[1] * t2[2] - t1[2] * t2[1], t1[2] * t2[0] - t1[0] * t2[2], t1[0] * t2[1] - t1[1] * t2[0]};
    FaceGeo g;
    g.A2 = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
    g.gi00 = g22 / det;
    g.gi11 = g11 / det;
    g.gi01 = -g12 / det;
    g.w_mu = ecoef[4 * (int64_t)t + 0];
    g.w_eps = ecoef[4 * (int64_t)t + 1];
    g.w_tand = ecoef[4 * (int64_t)t + 2];
    g.w_sig = ecoef[4 * (int64_t)t + 3];
    g.lf = lf;
    g.pad = 0;
    out[k] = g;
}

// One thread per unique CSR slot of a group: deterministic sum of its face entries.
__global__ void boundary_reduce_kernel(int64_t nu, int ldf, const int32_t* __restrict__ uptr, const int32_t* __restrict__ uent,
                                       const FaceGeo* __restrict__ fg, const double* __restrict__ ftab, double* __restrict__ R) {
    int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (u >= nu) return;
    const int L2 = ldf * ldf;
    double cc = 0, me = 0, mt = 0, ms = 0, m1 = 0;
    for (int32_t q = uptr[u]; q < uptr[u + 1]; ++q) {
        int32_t ent = uent[q];
        int k = ent / L2, ij = ent % L2;
        const FaceGeo g = fg[k];
        const double* T = ftab + (size_t)g.lf * 4 * L2;   // F11 | F22 | F12 | C
        double bm = g.A2 * (g.gi00 * T[ij] + g.gi11 * T[L2 + ij] + g.gi01 * T[2 * L2 + ij]);
        double bc = T[3 * L2 + ij] / g.A2;
        cc += g.w_mu * bc;
        me += g.w_eps * bm;
        mt += g.w_tand * bm;
        ms += g.w_sig * bm;
        m1 += bm;
    }
    R[u] = cc; R[nu + u] = me; R[2 * nu + u] = mt; R[3 * nu + u] = ms; R[4 * nu + u] = m1;
}

void assemble_boundary(Problem& P) {
    cudaStream_t s = P.ctx->stream;
    Topology& T = P.topo;
    const NDRef& R = nd_reference(T.p);
    const int ldf = T.ldf, L2 = ldf * ldf;
    // face tables: per local face F11 | F22 | F12 | C
    std::vector<double> ftab((size_t)16 * L2);
    for (int f = 0; f < 4; ++f) {
        std::copy(R.Fh[f].begin(), R.Fh[f].end(), ftab.begin() + (size_t)f * 4 * L2);
        std::copy(R.Ch[f].begin(), R.Ch[f].end(), ftab.begin() + (size_t)f * 4 * L2 + 3 * L2);
    }
    DBuf<double> d_ftab;
    d_ftab.upload(ftab, s);
    // A port driven by its own 2D mode on unsplit faces carries the mode exactly
    // in its trace space; its overlap block (R_one, used by no system matrix of a
    // port group) takes the reference's nodal rule (tangentialInnerProduct,
    // src/OpenParEM3D/port.cpp:3463-3490): the same reduction over tables built
    // with that rule.  The Robin blocks keep exact integration.
    auto nodal_port = [&](const BGroup& G) {
        return G.type == OPEM_BDR_PORT && G.port >= 0 && G.port < (int)P.modes.size() && P.modes[G.port].kind == 1 &&
               P.modes[G.port].nsub == 1;
    };
    DBuf<double> d_wtab;
    bool any_nodal = false;
    for (const BGroup& G : P.groups) any_nodal = any_nodal || nodal_port(G);
    if (any_nodal) {
        std::vector<double> wtab = ftab;
        for (int f = 0; f < 4; ++f) std::copy(R.Wh[f].begin(), R.Wh[f].end(), wtab.begin() + (size_t)f * 4 * L2);
        d_wtab.upload(wtab, s);
    }
    DBuf<int32_t> d_owner, d_lface;
    d_owner.upload(T.face_owner, s);
    d_lface.upload(T.face_lface, s);
    for (BGroup& G : P.groups) {
        int nf = (int)G.faces.size();
        if (nf == 0) { G.nu = 0; continue; }
        // entries (face k, i, j) -> CSR slot
        std::vector<std::pair<int32_t, int32_t>> ent;   // (slot, entry)
        ent.reserve((size_t)nf * L2);
        for (int k = 0; k < nf; ++k) {
            int f = G.faces[k];
            int t = T.face_owner[f], lf = T.face_lface[f];
            const int32_t* ed = &T.elem_dofs[(size_t)t * T.ld];
            for (int i = 0; i < ldf; ++i) {
                int32_t row = ed[R.face_dofs[lf][i]];
                for (int j = 0; j < ldf; ++j) {
                    int32_t col = ed[R.face_dofs[lf][j]];
                    const int32_t* c0 = &T.cols[T.rowptr[row]];
                    const int32_t* c1 = &T.cols[T.rowptr[row + 1]];
                    const int32_t* it = std::lower_bound(c0, c1, col);
                    ent.push_back({(int32_t)(it - &T.cols[0]), k * L2 + i * ldf + j});
                }
            }
        }
        std::sort(ent.begin(), ent.end());
        std::vector<int32_t> uslot, uptr, uent, urow, ucol;
        for (size_t q = 0; q < ent.size(); ++q) {
            if (q == 0 || ent[q].first != ent[q - 1].first) { uslot.push_back(ent[q].first); uptr.push_back((int32_t)q); }
            uent.push_back(ent[q].second);
        }
        uptr.push_back((int32_t)ent.size());
        G.nu = (int64_t)uslot.size();
        // row/col of each slot
        urow.resize(G.nu);
        ucol.resize(G.nu);
        for (int64_t u = 0; u < G.nu; ++u) {
            int32_t sl = uslot[u];
            int32_t row = (int32_t)(std::upper_bound(T.rowptr.begin(), T.rowptr.end(), sl) - T.rowptr.begin() - 1);
            urow[u] = row;
            ucol[u] = T.cols[sl];
        }
        G.h_urow = urow;
        G.h_ucol = ucol;
        // boundary CSR over the rows the group touches (slots are sorted => rows sorted)
        G.h_brow.clear(); G.h_bptr.clear();
        for (int64_t u = 0; u < G.nu; ++u)
            if (u == 0 || urow[u] != urow[u - 1]) { G.h_brow.push_back(urow[u]); G.h_bptr.push_back((int32_t)u); }
        G.h_bptr.push_back((int32_t)G.nu);
        G.uslot.upload(uslot, s);
        G.urow.upload(urow, s);
        G.ucol.upload(ucol, s);
        G.brow.upload(G.h_brow, s);
        G.bptr.upload(G.h_bptr, s);
        DBuf<int32_t> d_uptr, d_uent, d_faces;
        d_uptr.upload(uptr, s);
        d_uent.upload(uent, s);
        d_faces.upload(G.faces, s);
        DBuf<FaceGeo> d_fg(nf);
        face_geo_kernel<<<(nf + 127) / 128, 128, 0, s>>>(nf, d_faces.p, d_owner.p, d_lface.p, P.d_tets.p, P.d_verts.p,
                                                         P.d_elemcoef.p, d_fg.p); ++P.ctx->launches;
        OPEM_CUDA(cudaGetLastError());
        G.R.alloc(5 * G.nu);
        boundary_reduce_kernel<<<(unsigned)((G.nu + 127) / 128), 128, 0, s>>>(G.nu, ldf, d_uptr.p, d_uent.p, d_fg.p,
                                                                             d_ftab.p, G.R.p); ++P.ctx->launches;
        OPEM_CUDA(cudaGetLastError());
        if (nodal_port(G)) {
            DBuf<double> Rn;
            Rn.alloc(5 * G.nu);
            boundary_reduce_kernel<<<(unsigned)((G.nu + 127) / 128), 128, 0, s>>>(G.nu, ldf, d_uptr.p, d_uent.p,
                                                                                 d_fg.p, d_wtab.p, Rn.p);
            ++P.ctx->launches;
            OPEM_CUDA(cudaGetLastError());
            OPEM_CUDA(cudaMemcpyAsync(G.R.p + 4 * G.nu, Rn.p + 4 * G.nu, G.nu * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s));
            OPEM_CUDA(cudaStreamSynchronize(s));
        }
        OPEM_CUDA(cudaStreamSynchronize(s));
    }
}

// ---------------------------------------------------------------------------
// system matrix A(omega, d) = K + sum c Mx + boundary groups (FP64 complex)
// ---------------------------------------------------------------------------
__global__ void combine_kernel(int64_t nnz, const double* __restrict__ K, const double* __restrict__ Me,
                               const double* __restrict__ Mt, const double* __restrict__ Ms, VolCoef c,
                               double2* __restrict__ A) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        double me = Me[k];
        double re = K[k] + c.c_eps.x * me, im = c.c_eps.y * me;
        if (Mt) { double v = Mt[k]; re += c.c_tand.x * v; im += c.c_tand.y * v; }
        if (Ms) { double v = Ms[k]; re += c.c_sig.x * v; im += c.c_sig.y * v; }
        A[k] = make_double2(re, im);
    }
}

__global__ void boundary_add_kernel(int64_t nu, const int32_t* __restrict__ uslot, const double* __restrict__ R, BCoef c,
                                    double2* __restrict__ A) {
    int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (u >= nu) return;
    double cc = R[u], me = R[nu + u], mt = R[2 * nu + u], ms = R[3 * nu + u], m1 = R[4 * nu + u];
    double2 a = A[uslot[u]];
    a.x += c.c_cc.x * cc + c.c_eps.x * me + c.c_tand.x * mt + c.c_sig.x * ms + c.c_one.x * m1;
    a.y += c.c_cc.y * cc + c.c_eps.y * me + c.c_tand.y * mt + c.c_sig.y * ms + c.c_one.y * m1;
    A[uslot[u]] = a;
}

void form_system_matrix(Problem& P, const VolCoef& vc, const std::vector<BCoef>& bc, double2* A) {
    cudaStream_t s = P.ctx->stream;
    int64_t nnz = (int64_t)P.topo.cols.size();
    combine_kernel<<<P.ctx->sm_count * 8, 256, 0, s>>>(nnz, P.d_K.p, P.d_Meps.p, P.has_tand ? P.d_Mtand.p : nullptr,
                                                       P.has_sig ? P.d_Msig.p : nullptr, vc, A); ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
    for (size_t g = 0; g < P.groups.size(); ++g) {
        BGroup& G = P.groups[g];
        if (G.nu == 0) continue;
        const BCoef& c = bc[g];
        if (c.c_cc.x == 0 && c.c_cc.y == 0 && c.c_eps.x == 0 && c.c_eps.y == 0 && c.c_tand.x == 0 && c.c_tand.y == 0 &&
            c.c_sig.x == 0 && c.c_sig.y == 0 && c.c_one.x == 0 && c.c_one.y == 0)
            continue;
        boundary_add_kernel<<<(unsigned)((G.nu + 255) / 256), 256, 0, s>>>(G.nu, G.uslot.p, G.R.p, c, A); ++P.ctx->launches;
        OPEM_CUDA(cudaGetLastError());
    }
}

// Same kernels as form_system_matrix, coefficients from a plain array (no
// host containers), for the allocation-free entry point.
void form_system_matrix_n(Problem& P, const VolCoef& vc, const BCoef* bc, size_t nb, double2* A) {
    cudaStream_t s = P.ctx->stream;
    int64_t nnz = (int64_t)P.topo.cols.size();
    combine_kernel<<<P.ctx->sm_count * 8, 256, 0, s>>>(nnz, P.d_K.p, P.d_Meps.p, P.has_tand ? P.d_Mtand.p : nullptr,
                                                       P.has_sig ? P.d_Msig.p : nullptr, vc, A);
    ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
    for (size_t g = 0; g < P.groups.size() && g < nb; ++g) {
        BGroup& G = P.groups[g];
        if (G.nu == 0) continue;
        boundary_add_kernel<<<(unsigned)((G.nu + 255) / 256), 256, 0, s>>>(G.nu, G.uslot.p, G.R.p, bc[g], A);
        ++P.ctx->launches;
        OPEM_CUDA(cudaGetLastError());
    }
}

// ---------------------------------------------------------------------------
// port overlap: out = sum_u conj(a[row_u]) R_one[u] b[col_u]  (FP64)
// Mode::calculateSplits / tangentialInnerProduct, src/OpenParEM3D/port.cpp:3463-3568
// ---------------------------------------------------------------------------
__global__ void overlap_kernel(int64_t nu, const int32_t* __restrict__ urow, const int32_t* __restrict__ ucol,
                               const double* __restrict__ Rone, const double2* __restrict__ a, const double2* __restrict__ b,
                               double2* __restrict__ out) {
    __shared__ double sre[256], sim[256];
    double re = 0, im = 0;
    for (int64_t u = threadIdx.x; u < nu; u += blockDim.x) {
        double2 p = cconjmul(a[urow[u]], b[ucol[u]]);
        double w = Rone[u];
        re += w * p.x;
        im += w * p.y;
    }
    sre[threadIdx.x] = re;
    sim[threadIdx.x] = im;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) { sre[threadIdx.x] += sre[threadIdx.x + st]; sim[threadIdx.x] += sim[threadIdx.x + st]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = make_double2(sre[0], sim[0]);
}

void port_overlap(Problem& P, int k, const double2* a, const double2* b, double2* out_dev) {
    for (BGroup& G : P.groups) {
        if (G.type != OPEM_BDR_PORT || G.port != k || G.nu == 0) continue;
        overlap_kernel<<<1, 256, 0, P.ctx->stream>>>(G.nu, G.urow.p, G.ucol.p, G.R.p + 4 * G.nu, a, b, out_dev); ++P.ctx->launches;
        OPEM_CUDA(cudaGetLastError());
        return;
    }
    throw OpemError(OPEM_ERR_STATE, "port has no faces");
}

}  // namespace opem
