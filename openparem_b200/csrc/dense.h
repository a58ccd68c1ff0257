// Small dense complex linear algebra on the host (internal).  Column-major.
#pragma once
#include <complex>
#include <vector>

namespace opem {
using cd = std::complex<double>;
// Solves A x = b in place (b <- x).  Returns false on an exactly singular pivot.
bool lu_solve(int n, std::vector<cd> A, std::vector<cd>& b);
// k eigenpairs of the n x n matrix A with the smallest |theta|; vecs is n x k, unit columns.
bool eig_smallest(int n, const std::vector<cd>& A, int k, std::vector<cd>& theta, std::vector<cd>& vecs);
// Orthonormalises the columns of Q (rows x cols) in place; returns the numerical rank.
int orthonormalise(int rows, int cols, std::vector<cd>& Q);

// Incremental QR (Givens rotations) of the (m+1) x m least-squares matrix of
// one GMRES(-DR) cycle: columns arrive one by one; the first block after a
// deflated restart may be dense.
struct GivensLsq {
    struct Rot { int i1, i2; double c; cd s; };
    int m = 0;
    std::vector<cd> R;      // (m+1) x m column-major, rotated copy of H
    std::vector<cd> g;      // rotated right-hand side
    std::vector<Rot> rots;
    void reset(int m_, const std::vector<cd>& c);
    // add column j (entries 0..top); returns the least-squares residual |g[j+1]|
    double add_column(int j, const cd* col, int top);
    // y = R[:k,:k]^-1 g[:k]
    void solve(int k, std::vector<cd>& y) const;
};

// Deflated restart of GMRES-DR (Morgan): from the cycle's (m+1) x m Hessenberg
// H (column-major, ld m+1), right-hand side c and least-squares solution y,
// builds the orthonormal (m+1) x (kd+1) basis change Pm (kd harmonic Ritz
// vectors of smallest modulus plus the residual vector) and the new
// (kd+1) x kd block Hn (returned in an (m+1) x m array) and right-hand side cn.
bool gmres_dr_deflate(int m, int kd, const std::vector<cd>& H, const std::vector<cd>& c, const std::vector<cd>& y,
                      std::vector<cd>& Pm, std::vector<cd>& Hn, std::vector<cd>& cn);
}  // namespace opem
