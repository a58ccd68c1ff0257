/* CPU kernels of the oracle's iterative FP64 solve (test and baseline
 * infrastructure, not the product): complex CSR products, vertex-patch block
 * Jacobi set-up and apply, OpenMP over rows / patches.
 *
 * The oracle's direct solve (scipy SuperLU, the reference's Cholesky/LU-
 * preconditioned KSP of solveComplexLinearSystem.c:137-168) cannot factor the
 * 681k-DOF benchmark guide in bench time; these kernels let the same FP64
 * problem be solved on the host cores by preconditioned GMRES instead
 * (oracle/cpu_solve.py).  Complex numbers are interleaved (re, im) doubles.
 * Build: gcc -O3 -march=native -fopenmp -shared -fPIC (oracle/build_cpu.py). */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } zc;

/* y = A x */
void opem_cpu_spmv(int64_t n, const int64_t* rowptr, const int32_t* cols, const zc* vals, const zc* x, zc* y) {
#pragma omp parallel for schedule(static, 1024)
    for (int64_t i = 0; i < n; ++i) {
        double re = 0, im = 0;
        for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            const zc a = vals[k], b = x[cols[k]];
            re += a.re * b.re - a.im * b.im;
            im += a.re * b.im + a.im * b.re;
        }
        y[i].re = re;
        y[i].im = im;
    }
}

/* A[row][col] from CSR (binary search in the sorted row), 0 if absent */
static zc csr_at(const int64_t* rowptr, const int32_t* cols, const zc* vals, int64_t row, int32_t col) {
    int64_t lo = rowptr[row], hi = rowptr[row + 1] - 1;
    while (lo <= hi) {
        const int64_t mid = (lo + hi) / 2;
        if (cols[mid] == col) return vals[mid];
        if (cols[mid] < col) lo = mid + 1; else hi = mid - 1;
    }
    zc z = {0, 0};
    return z;
}

/* In-place inverse of the s x s row-major complex matrix a by Gauss-Jordan with
 * partial pivoting; piv is scratch of s ints.  Returns 0, or 1 if singular. */
static int zinvert(int s, zc* a, int* piv) {
    for (int c = 0; c < s; ++c) {
        int p = c;
        double best = hypot(a[(size_t)c * s + c].re, a[(size_t)c * s + c].im);
        for (int r = c + 1; r < s; ++r) {
            const double m = hypot(a[(size_t)r * s + c].re, a[(size_t)r * s + c].im);
            if (m > best) { best = m; p = r; }
        }
        if (!(best > 0)) return 1;
        piv[c] = p;
        if (p != c)
            for (int j = 0; j < s; ++j) {
                zc t = a[(size_t)c * s + j];
                a[(size_t)c * s + j] = a[(size_t)p * s + j];
                a[(size_t)p * s + j] = t;
            }
        const zc d = a[(size_t)c * s + c];
        const double dd = d.re * d.re + d.im * d.im;
        const zc inv = {d.re / dd, -d.im / dd};
        a[(size_t)c * s + c].re = 1;
        a[(size_t)c * s + c].im = 0;
        for (int j = 0; j < s; ++j) {
            const zc v = a[(size_t)c * s + j];
            a[(size_t)c * s + j].re = v.re * inv.re - v.im * inv.im;
            a[(size_t)c * s + j].im = v.re * inv.im + v.im * inv.re;
        }
        for (int r = 0; r < s; ++r) {
            if (r == c) continue;
            const zc f = a[(size_t)r * s + c];
            if (f.re == 0 && f.im == 0) continue;
            a[(size_t)r * s + c].re = 0;
            a[(size_t)r * s + c].im = 0;
            for (int j = 0; j < s; ++j) {
                const zc v = a[(size_t)c * s + j];
                a[(size_t)r * s + j].re -= f.re * v.re - f.im * v.im;
                a[(size_t)r * s + j].im -= f.re * v.im + f.im * v.re;
            }
        }
    }
    for (int c = s - 1; c >= 0; --c)   /* undo the row swaps as column swaps */
        if (piv[c] != c)
            for (int r = 0; r < s; ++r) {
                zc t = a[(size_t)r * s + c];
                a[(size_t)r * s + c] = a[(size_t)r * s + piv[c]];
                a[(size_t)r * s + piv[c]] = t;
            }
    return 0;
}

/* Inverted patch blocks: block v = inverse of A restricted to the DOFs
 * pdofs[pptr[v] .. pptr[v+1]), stored row-major at boff[v].  Returns the
 * number of singular blocks (left as identity). */
int opem_cpu_patch_invert(int npatch, const int64_t* pptr, const int32_t* pdofs, const int64_t* boff,
                          const int64_t* rowptr, const int32_t* cols, const zc* vals, zc* blocks) {
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : bad)
    for (int v = 0; v < npatch; ++v) {
        const int64_t p0 = pptr[v];
        const int s = (int)(pptr[v + 1] - p0);
        zc* a = blocks + boff[v];
        int* piv = (int*)malloc(sizeof(int) * (size_t)(s > 0 ? s : 1));
        for (int r = 0; r < s; ++r)
            for (int c = 0; c < s; ++c) a[(size_t)r * s + c] = csr_at(rowptr, cols, vals, pdofs[p0 + r], pdofs[p0 + c]);
        if (zinvert(s, a, piv)) {
            ++bad;
            memset(a, 0, sizeof(zc) * (size_t)s * s);
            for (int r = 0; r < s; ++r) a[(size_t)r * s + r].re = 1;
        }
        free(piv);
    }
    return bad;
}

/* y = sum over patches of R_v^T B_v R_v x: per-patch products into t (patch
 * entry order), then each DOF sums its entries in the fixed order of d2p
 * (deterministic, no atomics). */
void opem_cpu_patch_apply(int npatch, const int64_t* pptr, const int32_t* pdofs, const int64_t* boff,
                          const zc* blocks, int64_t n, const int64_t* d2p_ptr, const int64_t* d2p_idx, const zc* x,
                          zc* t, zc* y) {
#pragma omp parallel for schedule(dynamic, 32)
    for (int v = 0; v < npatch; ++v) {
        const int64_t p0 = pptr[v];
        const int s = (int)(pptr[v + 1] - p0);
        const zc* a = blocks + boff[v];
        for (int r = 0; r < s; ++r) {
            double re = 0, im = 0;
            const zc* row = a + (size_t)r * s;
            for (int c = 0; c < s; ++c) {
                const zc m = row[c], b = x[pdofs[p0 + c]];
                re += m.re * b.re - m.im * b.im;
                im += m.re * b.im + m.im * b.re;
            }
            t[p0 + r].re = re;
            t[p0 + r].im = im;
        }
    }
#pragma omp parallel for schedule(static, 1024)
    for (int64_t i = 0; i < n; ++i) {
        double re = 0, im = 0;
        for (int64_t q = d2p_ptr[i]; q < d2p_ptr[i + 1]; ++q) {
            re += t[d2p_idx[q]].re;
            im += t[d2p_idx[q]].im;
        }
        y[i].re = re;
        y[i].im = im;
    }
}

/* Jacobi-preconditioned CG on the real SPD matrix M (CSR, doubles) for two
 * right-hand sides at once (the real and imaginary parts of a complex rhs):
 * x = M^{-1} b to relative residual rtol, at most maxits iterations.
 * Returns the iteration count (negative if not converged). */
int opem_cpu_cg2(int64_t n, const int64_t* rowptr, const int32_t* cols, const double* vals, const double* b0,
                 const double* b1, double rtol, int maxits, double* x0, double* x1) {
    double *r = (double*)malloc(sizeof(double) * 2 * n), *z = (double*)malloc(sizeof(double) * 2 * n);
    double *p = (double*)malloc(sizeof(double) * 2 * n), *q = (double*)malloc(sizeof(double) * 2 * n);
    double* dg = (double*)malloc(sizeof(double) * n);
    const double* b[2] = {b0, b1};
    double* x[2] = {x0, x1};
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        dg[i] = 1;
        for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (cols[k] == i && vals[k] != 0) dg[i] = 1.0 / vals[k];
    }
    double rz[2], bn[2];
    for (int c = 0; c < 2; ++c) {
        double s1 = 0, s2 = 0;
#pragma omp parallel for reduction(+ : s1, s2)
        for (int64_t i = 0; i < n; ++i) {
            x[c][i] = 0;
            r[c * n + i] = b[c][i];
            z[c * n + i] = dg[i] * b[c][i];
            p[c * n + i] = z[c * n + i];
            s1 += r[c * n + i] * z[c * n + i];
            s2 += b[c][i] * b[c][i];
        }
        rz[c] = s1;
        bn[c] = sqrt(s2);
    }
    int it = 0, done = 0, conv[2] = {bn[0] == 0, bn[1] == 0};
    for (; it < maxits && !done; ++it) {
        for (int c = 0; c < 2; ++c) {
            if (conv[c]) continue;
            double pq = 0;
#pragma omp parallel for reduction(+ : pq) schedule(static, 1024)
            for (int64_t i = 0; i < n; ++i) {
                double s = 0;
                for (int64_t k = rowptr[i]; k < rowptr[i + 1]; ++k) s += vals[k] * p[c * n + cols[k]];
                q[c * n + i] = s;
                pq += p[c * n + i] * s;
            }
            const double al = rz[c] / pq;
            double rr = 0, nrz = 0;
#pragma omp parallel for reduction(+ : rr, nrz)
            for (int64_t i = 0; i < n; ++i) {
                x[c][i] += al * p[c * n + i];
                r[c * n + i] -= al * q[c * n + i];
                z[c * n + i] = dg[i] * r[c * n + i];
                rr += r[c * n + i] * r[c * n + i];
                nrz += r[c * n + i] * z[c * n + i];
            }
            if (sqrt(rr) <= rtol * bn[c]) { conv[c] = 1; continue; }
            const double be = nrz / rz[c];
            rz[c] = nrz;
#pragma omp parallel for
            for (int64_t i = 0; i < n; ++i) p[c * n + i] = z[c * n + i] + be * p[c * n + i];
        }
        done = conv[0] && conv[1];
    }
    free(r); free(z); free(p); free(q); free(dg);
    return done ? it : -it;
}
