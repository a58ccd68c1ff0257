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
}  // namespace opem
