// GMRES Hessenberg least squares on the device: kernels and launches (lsq.h).
#include "lsq.h"

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
