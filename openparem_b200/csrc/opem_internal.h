// Internal declarations of the B200 solve stage (not part of the C ABI).
#pragma once
#include <cstdint>
#include <cstdio>
#include <complex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/opem_b200.h"

namespace opem {

using cd = std::complex<double>;

// ---------------------------------------------------------------------------
// Reference-element tables of the order-p Nedelec basis (host, FP64).
// The basis is the dual basis of moment degrees of freedom on the reference
// tetrahedron with vertices sorted by global index (see basis.cpp).
// ---------------------------------------------------------------------------
struct NDRef {
    int p = 0;
    int ld = 0;        // local dofs per tet
    int ldf = 0;       // dofs of one face trace: 3 edges * p + p(p-1)
    int nmon = 0;      // monomials of degree <= p
    // symmetric combinations, index s in (00,11,22,01,02,12); off-diagonal
    // entries hold T_ab + T_ba:  Mh[s][i][j], Kh[s][i][j]
    std::vector<double> Mh, Kh;   // 6*ld*ld
    std::vector<double> Qh;       // ld*ld : int phi_i . curl phi_j
    // per local face f: Fh[f] = 3*ldf*ldf in (t1t1, t2t2, t1t2+t2t1); Ch[f] = ldf*ldf
    std::vector<double> Fh[4], Ch[4];
    // Fh with the port integrals' nodal rule (l2_nodal_rule(p)) in place of exact
    // integration: the overlaps of ports driven by their own 2D modes
    std::vector<double> Wh[4];
    std::vector<int> face_dofs[4];   // ldf local dof ids per face
    std::vector<double> coef;        // ld*3*nmon basis coefficients
    std::vector<int> mon;            // nmon*3 exponents
    // values and curls of the basis at the collapsed Gauss-Legendre tet rule of
    // degree 2p+2 (the error indicator's rule): w_err[q], phi_err / curl_err [q][i][3]
    int nq_err = 0;
    std::vector<double> w_err, phi_err, curl_err;
};

// Builds (and caches) the tables for order p; throws std::runtime_error.
const NDRef& nd_reference(int p);

// Gauss-Legendre rule on [0,1] with n points.
void gauss_legendre01(int n, std::vector<double>& x, std::vector<double>& w);
// Collapsed rules exact to total degree `deg` (Gauss-Legendre in each direction).
void tri_rule(int deg, std::vector<double>& s1, std::vector<double>& s2, std::vector<double>& w);
// The nodal rule of MFEM's order-p L2 triangle (Gauss-Legendre nodes) that the
// reference's port integrals amount to; weights sum to 1/2.
void l2_nodal_rule(int p, std::vector<double>& s1, std::vector<double>& s2, std::vector<double>& w);
// Orthonormal test polynomials on the unit triangle: coefficients T (n x n) over
// monomials s1^i s2^j of degree <= P ordered by degree, i descending.
std::vector<double> tri_test_polys(int P, std::vector<int>& mon2);
double shifted_legendre(int k, double s);

// ---------------------------------------------------------------------------
// Host mesh topology and DOF numbering.
// ---------------------------------------------------------------------------
struct Topology {
    int p = 0, ld = 0, ldf = 0;
    int64_t nv = 0, ne = 0, nE = 0, nF = 0, n = 0;
    std::vector<double> verts;        // nv*3
    std::vector<int32_t> tets;        // ne*4, ascending global ids
    std::vector<int32_t> region;      // ne
    std::vector<int32_t> tet_edges;   // ne*6
    std::vector<int32_t> tet_faces;   // ne*4
    std::vector<int32_t> face_owner, face_lface;   // nF
    std::vector<int32_t> elem_dofs;   // ne*ld
    std::vector<int32_t> bdr_face;    // nb
    std::vector<int32_t> bdr_attr;    // nb
    // CSR pattern
    std::vector<int32_t> rowptr, cols;
    // dof -> (element, local index) lists
    std::vector<int32_t> d2e_ptr, d2e_elem;
    std::vector<uint8_t> d2e_loc;
    // vertex patches (block-Jacobi blocks)
    std::vector<int32_t> patch_ptr, patch_dofs;   // CSR over vertices with >=1 dof
    std::vector<int64_t> patch_off;               // offsets of s_v^2 blocks
    int max_patch = 0;
};

int build_topology(Topology& T, int64_t nv, const double* verts, int64_t ne, const int64_t* tets,
                   const int32_t* region, int64_t nb, const int64_t* bdr, const int32_t* battr,
                   int p, std::string& err);
int build_pattern(Topology& T, std::string& err);
int build_patches(Topology& T, const std::vector<uint8_t>& pec_mask, std::string& err);

}  // namespace opem
