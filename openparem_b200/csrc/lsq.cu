// GMRES Hessenberg least squares on the device: kernels and launches (lsq.h).
#include "lsq.h"

#include <random>

#include "dense.h"

namespace opem {

namespace {

__global__ void lsq_start_kernel(int R, LsqState L, const uint8_t* __restrict__ reset, const double2* __restrict__ cvec,
                                 const int* __restrict__ start, const double2* __restrict__ H, int* __restrict__ err) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R || !reset[r]) return;
    const int m = L.m;
    for (int i = 0; i <= m; ++i) L.g[(int64_t)r * (m + 1) + i] = cvec[(int64_t)r * (m + 1) + i];
    L.nrot[r] = 0;
    const int st = start[r];
    for (int j = 0; j < st; ++j) L.est[r] = lsq_add_column(L, r, j, st, H + ((int64_t)r * m + j) * (m + 1), err);
}

__global__ void lsq_step_kernel(int R, LsqState L, int j, const uint8_t* __restrict__ act, const double2* __restrict__ H,
                                int* __restrict__ err) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R || !act[r]) return;
    L.est[r] = lsq_add_column(L, r, j, j + 1, H + ((int64_t)r * L.m + j) * (L.m + 1), err);
}

__global__ void lsq_solve_kernel(int R, LsqState L, const int* __restrict__ ncols, const uint8_t* __restrict__ act,
                                 double2* __restrict__ y, int ldy) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R || !act[r]) return;
    lsq_back_subst(L, r, ncols[r], y + (int64_t)r * ldy);
}

}  // namespace

void LsqWork::alloc(int R_, int m_, int kd, cudaStream_t s) {
    if (R_ < 1 || R_ > 32) throw OpemError(OPEM_ERR_ARG, "least squares: 1..32 systems");
    R = R_;
    m = m_;
    maxrot = kd * (kd + 1) / 2 + m + 1;   // the restart block's columns, then one per step
    Hr.alloc((size_t)R * (m + 1) * m);
    g.alloc((size_t)R * (m + 1));
    cvec.alloc((size_t)R * (m + 1));
    ri.alloc((size_t)R * maxrot);
    rc.alloc((size_t)R * maxrot);
    rs.alloc((size_t)R * maxrot);
    nrot.alloc(R);
    start.alloc(R);
    flags.alloc(R);
    err.alloc(1);
    err.zero(s);
    est.upload(std::vector<double>(R, 1.0), s);
}

void LsqWork::start_cycle(const std::vector<uint8_t>& reset, const std::vector<double2>& c, const std::vector<int>& start_,
                          const double2* H, cudaStream_t s, std::vector<double>& est_out) {
    flags.upload(reset.data(), R, s);
    cvec.upload(c.data(), (size_t)R * (m + 1), s);
    start.upload(start_.data(), R, s);
    lsq_start_kernel<<<1, 32, 0, s>>>(R, state(), flags.p, cvec.p, start.p, H, err.p);
    OPEM_CUDA(cudaGetLastError());
    std::vector<double> e(R);
    OPEM_CUDA(cudaMemcpyAsync(e.data(), est.p, R * sizeof(double), cudaMemcpyDeviceToHost, s));
    OPEM_CUDA(cudaStreamSynchronize(s));
    for (int r = 0; r < R; ++r)
        if (reset[r] && start_[r] > 0) est_out[r] = e[r];
}

void LsqWork::step(int j, const uint8_t* act, const double2* H, cudaStream_t s, std::vector<double>& est_out) {
    lsq_step_kernel<<<1, 32, 0, s>>>(R, state(), j, act, H, err.p);
    OPEM_CUDA(cudaGetLastError());
    est_out.resize(R);
    OPEM_CUDA(cudaMemcpyAsync(est_out.data(), est.p, R * sizeof(double), cudaMemcpyDeviceToHost, s));
    OPEM_CUDA(cudaStreamSynchronize(s));
}

void LsqWork::solve(const int* ncols, const uint8_t* act, double2* y, int ldy, cudaStream_t s) {
    lsq_solve_kernel<<<1, 32, 0, s>>>(R, state(), ncols, act, y, ldy);
    OPEM_CUDA(cudaGetLastError());
}

void LsqWork::check(cudaStream_t s) {
    int e = 0;
    OPEM_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    OPEM_CUDA(cudaStreamSynchronize(s));
    if (e) throw OpemError(OPEM_ERR_BREAKDOWN, "Hessenberg least squares: rotation store exhausted");
}

}  // namespace opem

// ---------------------------------------------------------------------------
// host check: the device update (the same inline functions, compiled for the
// host) against the host Givens QR (dense.cpp GivensLsq) on seeded problems
// ---------------------------------------------------------------------------
extern "C" int opem_selftest_lsq(int m, int kd, int seed, double* max_rel_diff) {
    using namespace opem;
    using cdd = std::complex<double>;
    if (m < 2 || kd < 0 || kd > m - 2 || !max_rel_diff) return OPEM_ERR_ARG;
    const int maxrot = kd * (kd + 1) / 2 + m + 1;
    std::vector<double2> Hr((size_t)(m + 1) * m), g(m + 1), rs(maxrot);
    std::vector<short2> ri(maxrot);
    std::vector<double> rc(maxrot), est(1);
    std::vector<int> nrot(1);
    int err = 0;
    const LsqState L{Hr.data(), g.data(), ri.data(), rc.data(), rs.data(), nrot.data(), est.data(), m, maxrot};
    std::mt19937 gen((unsigned)seed);
    std::normal_distribution<double> nd;
    double worst = 0;
    for (int start : {0, kd}) {
        // H: a restart block (start+1) x start, then Hessenberg columns
        std::vector<cdd> H((size_t)(m + 1) * m, 0.0), c(m + 1, 0.0);
        for (int j = 0; j < m; ++j) {
            const int top = j < start ? start : j + 1;
            for (int i = 0; i <= top; ++i) H[i + (size_t)j * (m + 1)] = cdd(nd(gen), nd(gen));
        }
        if (start == 0) c[0] = 1.5;
        else
            for (int i = 0; i <= start; ++i) c[i] = cdd(nd(gen), nd(gen));
        GivensLsq G;
        G.reset(m, c);
        for (int i = 0; i <= m; ++i) g[i] = make_double2(c[i].real(), c[i].imag());
        nrot[0] = 0;
        std::vector<double2> col(m + 1);
        for (int j = 0; j < m; ++j) {
            const int top = j < start ? start : j + 1;
            for (int i = 0; i <= m; ++i) col[i] = make_double2(H[i + (size_t)j * (m + 1)].real(), H[i + (size_t)j * (m + 1)].imag());
            const double e1 = G.add_column(j, &H[(size_t)j * (m + 1)], top);
            const double e2 = lsq_add_column(L, 0, j, top, col.data(), &err);
            worst = std::max(worst, std::fabs(e1 - e2) / std::max(1e-300, std::fabs(e1)));
            if (j >= start) {
                std::vector<cdd> y1;
                G.solve(j + 1, y1);
                std::vector<double2> y2(j + 1);
                lsq_back_subst(L, 0, j + 1, y2.data());
                for (int i = 0; i <= j; ++i)
                    worst = std::max(worst, std::abs(y1[i] - cdd(y2[i].x, y2[i].y)) / std::max(1e-300, std::abs(y1[i])));
            }
        }
    }
    *max_rel_diff = worst;
    return err ? OPEM_ERR_BREAKDOWN : OPEM_OK;
}
