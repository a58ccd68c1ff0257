// GMRES Hessenberg least squares on the device (FP64), shared by the FP64
// solver (krylov.cu) and the batched sweep solver (mixed.cu) (internal).
//
// The reference's KSPGMRES (src/OpenParEM3D/solveComplexLinearSystem.c:137,
// inside PETSc) updates a Givens QR of the (m+1) x m Hessenberg matrix H one
// column per Arnoldi step and reads the residual estimate |g[j+1]| from the
// rotated right-hand side g.  Here that update runs on the device, one thread
// per system, on the H column the Gram-Schmidt kernels have just written, so
// only the residual estimates (one double per system) cross to the host per
// step; the back substitution for y at the end of a cycle writes y where the
// basis-combination kernel reads it.  After a deflated restart the first kd
// columns of H form a full (kd+1) x kd block, whose entries below the diagonal
// take kd (kd+1)/2 rotations; every later column takes one.
#pragma once
#include <cstdint>
#include <vector>

#include "engine.h"

namespace opem {

// Per-system device arrays (R systems; m columns).  A rotation (i1 < i2, c, s)
// maps rows (a, b) -> (c a + s b, -conj(s) a + c b).
struct LsqState {
    double2* Hr;      // R x (m+1) x m: the rotated copy of H (column-major, ld m+1)
    double2* g;       // R x (m+1): the rotated right-hand side
    short2* ri;       // R x maxrot: rows (i1, i2) of each rotation, in the order made
    double* rc;       // R x maxrot: cosines
    double2* rs;      // R x maxrot: sines
    int* nrot;        // R: rotations so far in the cycle
    double* est;      // R: |g[j+1]| after the last column
    int m, maxrot;
};

__host__ __device__ inline double2 cmulc(double2 a, double2 b) {   // a * conj(b)
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

__host__ __device__ inline void lsq_rot(double c, double2 s, double2& a, double2& b) {
    const double2 x = a, y = b, sy = cmul(s, y), sx = cmulc(x, s);   // s y and conj(s) x
    a = make_double2(c * x.x + sy.x, c * x.y + sy.y);
    b = make_double2(c * y.x - sx.x, c * y.y - sx.y);
}

// Adds column j of system r (entries 0..top of Hcol, zero below) to its QR:
// the earlier rotations, then new ones that zero rows j+1..top.  Returns
// |g[j+1]|.  Sets *err = 2 (and stops) if the rotation store is full.
__host__ __device__ inline double lsq_add_column(const LsqState& L, int r, int j, int top,
                                                 const double2* __restrict__ Hcol, int* __restrict__ err) {
    const int m = L.m;
    double2* rc = L.Hr + ((int64_t)r * m + j) * (m + 1);
    double2* g = L.g + (int64_t)r * (m + 1);
    short2* ri = L.ri + (int64_t)r * L.maxrot;
    double* rcs = L.rc + (int64_t)r * L.maxrot;
    double2* rsn = L.rs + (int64_t)r * L.maxrot;
    for (int i = 0; i <= m; ++i) rc[i] = i <= top ? Hcol[i] : make_double2(0, 0);
    int nr = L.nrot[r];
    for (int q = 0; q < nr; ++q) lsq_rot(rcs[q], rsn[q], rc[ri[q].x], rc[ri[q].y]);
    for (int i2 = j + 1; i2 <= top; ++i2) {
        const double2 b = rc[i2];
        if (b.x == 0.0 && b.y == 0.0) continue;
        if (nr >= L.maxrot) {
            *err = 2;
            break;
        }
        const double2 a = rc[j];
        const double aa = hypot(a.x, a.y), bb = hypot(b.x, b.y);
        double c;
        double2 s;
        if (aa == 0.0) {
            c = 0.0;
            s = make_double2(b.x / bb, -b.y / bb);
        } else {
            const double rho = hypot(aa, bb);
            c = aa / rho;
            s = cmulc(make_double2(a.x / aa, a.y / aa), b);
            s = make_double2(s.x / rho, s.y / rho);
        }
        lsq_rot(c, s, rc[j], rc[i2]);
        rc[i2] = make_double2(0, 0);
        lsq_rot(c, s, g[j], g[i2]);
        ri[nr] = make_short2((short)j, (short)i2);
        rcs[nr] = c;
        rsn[nr] = s;
        ++nr;
    }
    L.nrot[r] = nr;
    return hypot(g[j + 1].x, g[j + 1].y);
}

// y = Hr[:k,:k]^-1 g[:k] of system r (back substitution)
__host__ __device__ inline void lsq_back_subst(const LsqState& L, int r, int k, double2* __restrict__ yr) {
    const int m = L.m;
    const double2* Hr = L.Hr + (int64_t)r * m * (m + 1);
    const double2* g = L.g + (int64_t)r * (m + 1);
    for (int i = k - 1; i >= 0; --i) {
        double2 s = g[i];
        for (int c = i + 1; c < k; ++c) {
            const double2 t = cmul(Hr[i + (int64_t)c * (m + 1)], yr[c]);
            s.x -= t.x;
            s.y -= t.y;
        }
        const double2 d = Hr[i + (int64_t)i * (m + 1)];
        const double dd = d.x * d.x + d.y * d.y;
        const double2 q = cmulc(s, d);
        yr[i] = make_double2(q.x / dd, q.y / dd);
    }
}

// Device workspace and launches for R <= 32 systems.  H is the device
// Hessenberg array the Gram-Schmidt kernels write: system r's column j at
// (r m + j)(m+1).
struct LsqWork {
    int R = 0, m = 0, maxrot = 0;
    DBuf<double2> Hr, g, rs, cvec;
    DBuf<short2> ri;
    DBuf<double> rc, est;
    DBuf<int> nrot, start, err;
    DBuf<uint8_t> flags;
    void alloc(int R_, int m_, int kd, cudaStream_t s);
    LsqState state() const { return LsqState{Hr.p, g.p, ri.p, rc.p, rs.p, nrot.p, est.p, m, maxrot}; }
    // cycle start of the systems with reset[r] != 0 (host flags): g = c[r]
    // (R x (m+1)), then the first start[r] columns of H; est[r] of the systems
    // with start[r] > 0 comes back in est_out (synchronises the stream)
    void start_cycle(const std::vector<uint8_t>& reset, const std::vector<double2>& c, const std::vector<int>& start_,
                     const double2* H, cudaStream_t s, std::vector<double>& est_out);
    // column j of the systems with act[r] (device flags); est_out = est of all R
    // systems (synchronises the stream)
    void step(int j, const uint8_t* act, const double2* H, cudaStream_t s, std::vector<double>& est_out);
    // y[r] (ldy apart) for the systems with act[r] (device flags), k = ncols[r] (device)
    void solve(const int* ncols, const uint8_t* act, double2* y, int ldy, cudaStream_t s);
    // throws OPEM_ERR_BREAKDOWN if a column found the rotation store full (synchronises)
    void check(cudaStream_t s);
};

}  // namespace opem
