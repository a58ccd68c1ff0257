// Zienkiewicz-Zhu error indicator on H and refinement marking.
//
// Restates fem3D::calculateMeshErrors (src/OpenParEM3D/fem3D.cpp:1162-1420)
// and its estimator OPEM_L2ZZErrorEstimator (:987-1154), run as the reference
// runs them (real and imaginary parts separately, norm_p = 1), on the H fields
// of the last opem_solve_frequency:
//   flux       F = (1/mu_r) curl H per tetrahedron (CurlCurlIntegrator's element
//              flux; curl of an order-p edge-element field is exact in the
//              order p-1 face-element space the reference stores it in)
//   smooth     s = L2 projection of F onto the edge elements: M1 s = Q_mu h
//              (b_i = int N_i . F is the MixedVectorCurl product the H
//              projection already uses), mass CG to 1e-12 (the reference: CG
//              with SOR, rtol 1e-12, 2000 iterations)
//   error(e)   sqrt((int_e |Re(s - F)|)^2 + (int_e |Im(s - F)|)^2)
//   merge      the larger error per element over the driving sets (:1258-1263)
//   marking    the floor(NE * fraction) (at least 1) largest errors, and the
//              largest as maxMeshError (:1321-1350)
// The element integrals use the collapsed Gauss-Legendre tet rule of degree
// 2p+2 (NDRef::w_err): the integrand is not polynomial, so the rule is part of
// the definition.
//
// Device work: the SpMV and mass CG of the H projection (krylov.cu), and
// zz_element_kernel, one warp per tetrahedron: the element's DOFs of s and h
// are gathered once into shared memory, each lane takes quadrature points,
// and the two L1 integrals are reduced across the warp.  The kernel reads
// 2 x ld complex DOFs per element (L2-resident tables for the basis); it is a
// small fraction of one driving set's solve.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "engine.h"

namespace opem {

constexpr int ZZ_WARPS = 4;   // tetrahedra per block

__global__ void __launch_bounds__(32 * ZZ_WARPS)
zz_element_kernel(int64_t ne, int ld, int nq, const double* __restrict__ verts, const int32_t* __restrict__ tets,
                  const int32_t* __restrict__ region, const double* __restrict__ inv_mu,
                  const int32_t* __restrict__ elem_dofs, const double2* __restrict__ s, const double2* __restrict__ h,
                  const double* __restrict__ w, const double* __restrict__ phi, const double* __restrict__ curl,
                  double* __restrict__ err) {
    extern __shared__ double2 zz_sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * ZZ_WARPS + warp;
    if (e >= ne) return;
    double2* se = zz_sm + (size_t)warp * 2 * ld;
    double2* he = se + ld;
    for (int i = lane; i < ld; i += 32) {
        const int32_t g = __ldg(elem_dofs + e * ld + i);
        se[i] = s[g];
        he[i] = h[g];
    }
    __syncwarp();
    // geometry: J = [P1-P0, P2-P0, P3-P0] (columns), its inverse and determinant
    double P[4][3];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const int32_t id = __ldg(tets + 4 * e + v);
#pragma unroll
        for (int c = 0; c < 3; ++c) P[v][c] = __ldg(verts + 3 * (int64_t)id + c);
    }
    double J[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) J[a][b] = P[b + 1][a] - P[0][a];
    const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                       J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                       J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    double Ji[3][3];   // inverse: adjugate / det
    Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
    Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
    Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
    Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    const double cf = __ldg(inv_mu + __ldg(region + e)) / det;   // curl N = J curl_hat N / det, over mu_r
    const double adet = fabs(det);
    double acc_re = 0, acc_im = 0;
    for (int q = lane; q < nq; q += 32) {
        double sr[3] = {0, 0, 0}, si[3] = {0, 0, 0}, cr[3] = {0, 0, 0}, ci[3] = {0, 0, 0};
        const double* pq = phi + (size_t)q * ld * 3;
        const double* cq = curl + (size_t)q * ld * 3;
        for (int i = 0; i < ld; ++i) {
            const double2 a = se[i], b = he[i];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double pv = __ldg(pq + 3 * i + c), cv = __ldg(cq + 3 * i + c);
                sr[c] += a.x * pv; si[c] += a.y * pv;
                cr[c] += b.x * cv; ci[c] += b.y * cv;
            }
        }
        double dr2 = 0, di2 = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            // s = J^-T s_hat, F = J c_hat / (det mu_r)
            const double spr = Ji[0][a] * sr[0] + Ji[1][a] * sr[1] + Ji[2][a] * sr[2];
            const double spi = Ji[0][a] * si[0] + Ji[1][a] * si[1] + Ji[2][a] * si[2];
            const double fr = cf * (J[a][0] * cr[0] + J[a][1] * cr[1] + J[a][2] * cr[2]);
            const double fi = cf * (J[a][0] * ci[0] + J[a][1] * ci[1] + J[a][2] * ci[2]);
            dr2 += (spr - fr) * (spr - fr);
            di2 += (spi - fi) * (spi - fi);
        }
        const double wq = __ldg(w + q) * adet;
        acc_re += wq * sqrt(dr2);
        acc_im += wq * sqrt(di2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc_re += __shfl_down_sync(0xffffffffu, acc_re, o);
        acc_im += __shfl_down_sync(0xffffffffu, acc_im, o);
    }
    if (lane == 0) err[e] = fmax(err[e], sqrt(acc_re * acc_re + acc_im * acc_im));
}

// Errors of the last solve's driving sets, merged per element (host vector of ne).
void mesh_error_indicator(Problem& P, std::vector<double>& out) {
    const Topology& T = P.topo;
    const NDRef& R = nd_reference(T.p);
    cudaStream_t st = P.ctx->stream;
    const int64_t n = T.n, ne = T.ne;
    DBuf<double> w, phi, cur, imu, err(ne);
    w.upload(R.w_err, st);
    phi.upload(R.phi_err, st);
    cur.upload(R.curl_err, st);
    std::vector<double> inv_mu(P.nregions);
    for (int r = 0; r < P.nregions; ++r) inv_mu[r] = 1.0 / P.mu_r[r];
    imu.upload(inv_mu, st);
    DBuf<double2> h(n), b(n), sm(n);
    OPEM_CUDA(cudaMemsetAsync(err.p, 0, ne * sizeof(double), st));
    const size_t smem = (size_t)ZZ_WARPS * 2 * T.ld * sizeof(double2);
    for (size_t d = 0; d < P.last_h.size(); ++d) {
        if (P.last_h[d].empty()) continue;
        OPEM_CUDA(cudaMemcpyAsync(h.p, P.last_h[d].data(), n * sizeof(double2), cudaMemcpyHostToDevice, st));
        spmv_real_complex(P, P.d_Q.p, h.p, b.p, 1.0, 0.0);   // b = Q_mu h = int N . curl h / mu_r
        SolveResult r = solve_mass_cg(P, b.p, sm.p, 1e-12, 2000);
        if (r.code != OPEM_OK) throw OpemError(r.code, "error indicator: mass solve failed");
        zz_element_kernel<<<(unsigned)((ne + ZZ_WARPS - 1) / ZZ_WARPS), 32 * ZZ_WARPS, smem, st>>>(
            ne, T.ld, R.nq_err, P.d_verts.p, P.d_tets.p, P.d_region.p, imu.p, P.d_elem_dofs.p, sm.p, h.p, w.p, phi.p,
            cur.p, err.p);
        ++P.ctx->launches;
        OPEM_CUDA(cudaGetLastError());
    }
    out.resize(ne);
    OPEM_CUDA(cudaMemcpyAsync(out.data(), err.p, ne * sizeof(double), cudaMemcpyDeviceToHost, st));
    OPEM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace opem
