// Port modes solved on the port's own faces (host only, internal).
#pragma once
#include <complex>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace opem {

// The fundamental mode of one port at one frequency, found on a conforming
// split of the port's faces (each face into nsub x nsub similar triangles).
// Second-order edge / quadratic nodal solve of the port pencil (port2d.cpp):
// per triangle 8 e_t and 6 e_z coefficients of the hierarchical basis and the
// sorted vertex ids.
int port_mode_2d_p2(int64_t nnodes, const double* xy, int64_t ntri, const int64_t* tris,
                    const std::complex<double>* eps_r, const std::complex<double>* mu_r, double freq,
                    std::complex<double>& beta, std::vector<std::complex<double>>& ct,
                    std::vector<std::complex<double>>& cz, std::vector<int64_t>& st);

// Nodal bases of order p on the unit triangle (x, y >= 0, x + y <= 1), with the
// triangle's vertices in increasing global order: the first-kind Nedelec space
// R_p = P_{p-1}^2 + (-y, x) P~_{p-1} (p (p+2) functions, degrees of freedom the
// edge moments against shifted Legendre L_0..L_{p-1} along each edge from its
// lower to its higher vertex, then interior moments against P_{p-2}^2) and the
// Lagrange space of degree p (equispaced nodes: vertices, edge nodes from the
// edge's lower vertex, interior), both as coefficients over the monomials
// x^a y^b of degree <= p.
struct RefSpaces2D {
    int p = 0, nm = 0, nf = 0, nl = 0;
    std::vector<int> mono;            // 2 nm exponents
    std::vector<double> CX, CY, CL;   // nm x nf, nm x nf, nm x nl (row m, column i)
    // values N (nf x 2) and scalar curls (nf) of the edge functions at (x, y)
    void nd(double x, double y, double* N, double* curl) const;
    // values (nl) and gradients (nl x 2) of the Lagrange functions at (x, y)
    void h1(double x, double y, double* L, double* gL) const;
};
const RefSpaces2D& ref_spaces_2d(int p);   // cached; throws std::runtime_error for p < 1 or p > 8

// The fundamental mode (mode 0), or the mode-th mode in decreasing beta^2
// (mode <= 15: subspace iteration over the mode + 1 leading modes), with
// order-p elements of RefSpaces2D (the spaces of the reference's 2D solver at
// mesh.order p): per triangle nf e_t and nl e_z coefficients on the reference
// bases, and the sorted vertex ids.
int port_mode_2d_pp(int64_t nnodes, const double* xy, int64_t ntri, const int64_t* tris,
                    const std::complex<double>* eps_r, const std::complex<double>* mu_r, double freq, int p,
                    std::complex<double>& beta, std::vector<std::complex<double>>& ct,
                    std::vector<std::complex<double>>& cz, std::vector<int64_t>& st, int mode = 0);

// Weighted L2 projection of a tangential field onto the order-p edge space of
// RefSpaces2D on the triangles (st: 3 sorted vertex ids per triangle; weight: one
// complex factor per triangle; no boundary condition), as the reference's 2D
// solver forms H_t (Hsolve, src/OpenParEM2D/Hsolve.c:454-560, with the mass
// matrix weighted by omega mu, fem2D.cpp:2297-2303).  field(t, x, y, fx, fy)
// gives the field at the point (x, y) of triangle t.  ch: nf coefficients per
// triangle on the reference bases.  Returns an OPEM_* code.
int project_nd_2d(int64_t nnodes, const double* xy, int64_t ntri, const int64_t* st, int p,
                  const std::complex<double>* weight,
                  const std::function<void(int64_t, double, double, std::complex<double>&, std::complex<double>&)>& field,
                  std::vector<std::complex<double>>& ch);

struct PortFem2D {
    using cd = std::complex<double>;
    int nsub = 0;
    int order = 1;                    // 2D element order (1 .. 8)
    int64_t nface = 0;
    double o[3], u[3], v[3], n[3];    // unit frame of the port plane; n = outward normal
    double freq = 0, mu_port = 1;
    cd gamma, V, Z, Pz, I;            // I: current along the current path (0 without one)
    std::vector<double> xy;           // 2D nodes
    std::vector<int64_t> st;          // 3 sorted node ids per sub-triangle
    std::vector<double> P0, Jinv, g;  // per sub-triangle: first node (2), J^-1 (4), grad lambda (3x2)
    std::vector<cd> ce, gz, mu;       // order 1: edge coefficients (3), grad e_z (2); mu_r (1)
    std::vector<cd> ct, cz;           // order 2: e_t (8) and e_z (6) coefficients; order >= 3: nf and nl
    const RefSpaces2D* ref = nullptr; // order-p path (unsplit faces, order >= 3, higher modes): the reference bases
    std::vector<cd> ch;               // order-p path: H_t / y projected onto the edge space (nf per triangle)
    std::vector<int64_t> sub;         // per face: (i, j, upper) -> sub-triangle

    // E_t and H_t / y (y = gamma / (j w mu0 mu_port)) at the 3D point X of
    // sub-triangle t
    void eval_tri(int64_t t, const double X[3], cd E[3], cd Hy[3]) const;
    // the same at X = P0 + s1 (P1 - P0) + s2 (P2 - P0) of port face f
    void eval_face(int64_t f, double s1, double s2, const double X[3], cd E[3], cd Hy[3]) const;
    // the sub-triangle a point of the port plane is deepest inside
    int64_t locate(const double X[3]) const;
};

// Builds and solves the mode.  verts: 3D vertices; face_verts: 3 vertex ids per
// port face in the face's local order; eps_face / mu_face: complex relative
// permittivity / permeability per face (from the owning tetrahedron);
// desc: the 22-double port descriptor (origin, u, v, outward normal, a, b, m, n,
// voltage path); order: 2D element order (1 or 2); mu_port: mu_r used to scale
// H_t / y; zdef: OPEM_Z_PV / VI / PI; ipath: the current path's points (xyz,
// npath of them, closed: with the segment back to the first).  Returns an
// OPEM_* code.  mode > 0: the mode-th mode in decreasing beta^2 instead of the
// fundamental one (order-p elements of RefSpaces2D for every order).
int port_fem2d_solve(const double* verts, int64_t nface, const int64_t* face_verts,
                     const std::complex<double>* eps_face, const std::complex<double>* mu_face, const double* desc,
                     int nsub, int order, double freq, double mu_port, PortFem2D& out, std::string& err,
                     int zdef = 0, const double* ipath = nullptr, int npath = 0, bool closed = true, int mode = 0);

}  // namespace opem
