// Batched mixed-precision solve of many (frequency, driving set) systems.
//
// Same per-frequency flow as the FP64 path (the reference's driving-set loop,
// src/OpenParEM3D/OpenParEM3D.cpp:497-566) but up to RMAX systems share every
// read of the operator and of the block-Jacobi blocks:
//   outer (FP64):  r = b - A x on the FP64 operators; stop at ||r|| <= rtol ||b||
//   inner:         flexible GMRES-DR on A d = r/||r|| with FP64 Krylov bases V and
//                  Z and FP64 Arnoldi products; the preconditioner M^-1 q(A M^-1)
//                  (FP32 vertex-patch blocks, GMRES polynomial q evaluated with
//                  FP32 operators and vectors) varies per step; x += ||r|| d
//   H (FP64):      batched CG on the mass matrix, P h = j Q e
//   overlaps and S: FP64, as in the FP64 path.
// (An FP32-Krylov inner solve was measured first and dropped: FP32 vectors cap
// each inner solve's contraction of the FP64 residual near u32 * cond.)
// The Hessenberg least squares of every system runs on the device in FP64
// (lsq.cu); the deflation eigenproblem and the polynomial's roots on the host.
//
// Layouts: vectors that feed the shared-matrix kernels (SpMV, block apply) are
// interleaved, element (k, r) at k*R + r, so one row's gather for all systems
// is one contiguous segment; per-system dense work (Gram-Schmidt, basis
// updates) uses system-major vectors, system r at r*ld.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "dense.h"
#include "lsq.h"
#include "engine.h"
#include "patch_tc.h"

namespace opem {

constexpr int RMAX = 32;
static const double MU0_M = 4e-7 * M_PI;

// ---------------------------------------------------------------------------
// complex helpers for both precisions
// ---------------------------------------------------------------------------
template <class T2> struct Cx;
template <> struct Cx<float2> {
    using R = float;
    __device__ static float2 make(float a, float b) { return make_float2(a, b); }
};
template <> struct Cx<double2> {
    using R = double;
    __device__ static double2 make(double a, double b) { return make_double2(a, b); }
};

template <class T> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };

// per-system volume coefficients (A = K + ce Meps + ct Mtand + cs Msig)
template <class T2> struct VC3 { T2 ce, ct, cs; };
// per-system boundary-group coefficients
template <class T2> struct BC5 { T2 cc, ce, ct, cs, c1; };

// ---------------------------------------------------------------------------
// batched SpMV: y_il = A_r x_il for every system r; Dirichlet rows of system r
// (PEC or its driven port) are set to zero.
// ---------------------------------------------------------------------------
// T2: vector type (float2 or double2); T: matrix values, coefficients and
// accumulation.  A group of W lanes owns one row (W = 16: two rows per warp
// when R <= 16; W = 32 otherwise), lane = system.  The row's nonzeros are
// staged SPMV_CH at a time in shared memory (column index and the real
// operator values, coalesced loads), then every lane gathers its system's
// entries of x for 8 nonzeros at once and accumulates the products with each
// real operator separately (K x, Meps x, Mtand x, Msig x); the system's
// coefficients are applied once per row.
constexpr int SPMV_CH = 32;
template <class T> struct SpmvStage;
template <> struct SpmvStage<float> {
    float4 v[SPMV_CH];   // K, Meps, Mtand, Msig
    int col[SPMV_CH];
};
template <> struct SpmvStage<double> {
    double2 km[SPMV_CH];   // K, Meps
    double2 ts[SPMV_CH];   // Mtand, Msig
    int col[SPMV_CH];
};

template <class T2, class T, bool HT, bool HS, int W>
__global__ void __launch_bounds__(256) spmv_batch_kernel(
    int64_t n, int R, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols, const T* __restrict__ K,
    const T* __restrict__ Me, const T* __restrict__ Mt, const T* __restrict__ Ms,
    const VC3<typename CplxOf<T>::type>* __restrict__ coef, const T2* __restrict__ x, T2* __restrict__ y,
    const uint8_t* __restrict__ pec, const uint8_t* __restrict__ pm, const uint8_t* __restrict__ dsys) {
    constexpr int SUB = 32 / W;   // rows per warp
    __shared__ SpmvStage<T> stage[8][SUB];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int sub = lane / W, sl = lane - sub * W;
    SpmvStage<T>& st = stage[wid][sub];
    const bool act = sl < R;
    VC3<typename CplxOf<T>::type> c{};
    int d = 0;
    if (act) { c = coef[sl]; d = dsys[sl]; }
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t rb = (blockIdx.x * (int64_t)(blockDim.x >> 5) + wid) * SUB; rb < n; rb += nwarps * SUB) {
        const int64_t row = rb + sub;
        const bool rv = row < n;
        const int32_t ks = rv ? rowptr[row] : 0;
        const int len = rv ? rowptr[row + 1] - ks : 0;
        int maxlen = len;
        if (SUB == 2) maxlen = max(len, __shfl_xor_sync(0xffffffffu, len, 16));
        T kr = 0, ki = 0, mr = 0, mi = 0, tr = 0, ti = 0, sr = 0, si = 0;
        for (int c0 = 0; c0 < maxlen; c0 += SPMV_CH) {
#pragma unroll
            for (int w = 0; w < SPMV_CH / W; ++w) {
                const int e = w * W + sl;
                if (c0 + e < len) {
                    const int32_t k = ks + c0 + e;
                    st.col[e] = __ldg(cols + k);
                    if constexpr (sizeof(T) == 4) {
                        st.v[e] = make_float4(__ldg(K + k), __ldg(Me + k), HT ? __ldg(Mt + k) : 0.f,
                                              HS ? __ldg(Ms + k) : 0.f);
                    } else {
                        st.km[e] = make_double2(__ldg(K + k), __ldg(Me + k));
                        if (HT || HS) st.ts[e] = make_double2(HT ? __ldg(Mt + k) : 0.0, HS ? __ldg(Ms + k) : 0.0);
                    }
                }
            }
            __syncwarp();
            const int cnt = min(SPMV_CH, len - c0);
            if (act)
                for (int j0 = 0; j0 < cnt; j0 += 8) {
                    T2 xv[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (j0 + u < cnt) xv[u] = x[(int64_t)st.col[j0 + u] * R + sl];
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (j0 + u < cnt) {
                            const T xr = (T)xv[u].x, xi = (T)xv[u].y;
                            T kv, mv, tv = 0, sv = 0;
                            if constexpr (sizeof(T) == 4) {
                                const float4 q = st.v[j0 + u];
                                kv = q.x; mv = q.y; tv = q.z; sv = q.w;
                            } else {
                                const double2 q = st.km[j0 + u];
                                kv = q.x; mv = q.y;
                                if (HT || HS) { const double2 q2 = st.ts[j0 + u]; tv = q2.x; sv = q2.y; }
                            }
                            kr = fma(kv, xr, kr); ki = fma(kv, xi, ki);
                            mr = fma(mv, xr, mr); mi = fma(mv, xi, mi);
                            if (HT) { tr = fma(tv, xr, tr); ti = fma(tv, xi, ti); }
                            if (HS) { sr = fma(sv, xr, sr); si = fma(sv, xi, si); }
                        }
                }
            __syncwarp();
        }
        if (act && rv) {
            T re = kr + c.ce.x * mr - c.ce.y * mi, im = ki + c.ce.x * mi + c.ce.y * mr;
            if (HT) { re += c.ct.x * tr - c.ct.y * ti; im += c.ct.x * ti + c.ct.y * tr; }
            if (HS) { re += c.cs.x * sr - c.cs.y * si; im += c.cs.x * si + c.cs.y * sr; }
            const bool D = pec[row] || ((pm[row] >> d) & 1);
            y[row * R + sl] = D ? Cx<T2>::make(0, 0) : Cx<T2>::make((typename Cx<T2>::R)re, (typename Cx<T2>::R)im);
        }
    }
}

// ---------------------------------------------------------------------------
// element-by-element batched product of the volume operators (ND2: LD = 20):
//   y_r = sum_e P_e^T ( (1/mu_e) Khat_e + c_{e,r} Mhat_e ) P_e x_r,
//   c_{e,r} = c_eps,r eps_e + c_tand,r eps_e tan_d_e + c_sig,r sigma_e,
// with Khat_e = sum_s gK_s Kref_s and Mhat_e = sum_s gM_s Mref_s the element's
// geometric curl-curl and mass matrices (the same sums the CSR assembly
// forms).  The CSR product gathers R x-entries per nonzero (29M gathers of
// R*8 bytes on the 681k-DOF case, served by L2); per element the 20 DOF
// segments are gathered once and used 20 times.
// Pass 1 (ebe_elem_kernel): a group of W lanes per element (lane = system)
// builds Khat_e and Mhat_e in shared memory, gathers x_e into registers and
// writes the element's 20 x R outputs to ye.  Pass 2 (ebe_sum_kernel): every
// DOF sums its elements' entries in the fixed order of its element list (so
// the result is deterministic) and zeroes the Dirichlet rows of each system.
// ---------------------------------------------------------------------------
template <class T, int LD>
struct EbeMats {
    T K[LD * LD];
    T M[LD * LD];
};

template <class T2, class T, int LD, int W>
__global__ void __launch_bounds__(256) ebe_elem_kernel(int64_t ne, int R, const int32_t* __restrict__ edofs,
                                                       const ElemGeo* __restrict__ geo,
                                                       const double* __restrict__ ecoef, const double* __restrict__ ref,
                                                       const VC3<typename CplxOf<T>::type>* __restrict__ coef,
                                                       const T2* __restrict__ x, T2* __restrict__ ye) {
    using C2 = typename CplxOf<T>::type;
    constexpr int SUB = 32 / W;
    constexpr int LL = LD * LD;
    extern __shared__ float4 ebe_smem[];
    T* sref = reinterpret_cast<T*>(ebe_smem);                        // Kref (6 LL) | Mref (6 LL)
    EbeMats<T, LD>* mats = reinterpret_cast<EbeMats<T, LD>*>(sref + 12 * LL);   // [8 warps][SUB]
    for (int t = threadIdx.x; t < 12 * LL; t += blockDim.x) sref[t] = (T)ref[t];
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, sub = lane / W, sl = lane - sub * W;
    EbeMats<T, LD>& E = mats[wid * SUB + sub];
    const bool act = sl < R;
    VC3<C2> c{};
    if (act) c = coef[sl];
    const int64_t ngroups = (int64_t)gridDim.x * (blockDim.x >> 5) * SUB;
    for (int64_t e = (blockIdx.x * (int64_t)(blockDim.x >> 5) + wid) * SUB + sub; e - sub < ne; e += ngroups) {
        const bool ev = e < ne;
        if (ev) {
            const ElemGeo g = geo[e];
            T gk[6], gm[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) { gk[q] = (T)g.gK[q]; gm[q] = (T)g.gM[q]; }
            for (int t = sl; t < LL; t += W) {
                T kv = 0, mv = 0;
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    kv = fma(gk[q], sref[q * LL + t], kv);
                    mv = fma(gm[q], sref[(6 + q) * LL + t], mv);
                }
                E.K[t] = kv;
                E.M[t] = mv;
            }
        }
        __syncwarp();
        if (ev && act) {
            const T imu = (T)ecoef[4 * e + 0], eps = (T)ecoef[4 * e + 1], epst = (T)ecoef[4 * e + 2],
                    sig = (T)ecoef[4 * e + 3];
            const T cer = c.ce.x * eps + c.ct.x * epst + c.cs.x * sig;
            const T cei = c.ce.y * eps + c.ct.y * epst + c.cs.y * sig;
            T xr[LD], xi[LD];
#pragma unroll
            for (int j = 0; j < LD; ++j) {
                const T2 v = x[(int64_t)__ldg(edofs + e * LD + j) * R + sl];
                xr[j] = (T)v.x;
                xi[j] = (T)v.y;
            }
            T2* out = ye + (e * LD) * (int64_t)R + sl;
#pragma unroll 2
            for (int i = 0; i < LD; ++i) {
                T kr = 0, ki = 0, mr = 0, mi = 0;
#pragma unroll
                for (int j = 0; j < LD; ++j) {
                    const T kv = E.K[i * LD + j], mv = E.M[i * LD + j];
                    kr = fma(kv, xr[j], kr); ki = fma(kv, xi[j], ki);
                    mr = fma(mv, xr[j], mr); mi = fma(mv, xi[j], mi);
                }
                const T yr = imu * kr + cer * mr - cei * mi;
                const T yi = imu * ki + cer * mi + cei * mr;
                out[(int64_t)i * R] = Cx<T2>::make((typename Cx<T2>::R)yr, (typename Cx<T2>::R)yi);
            }
        }
        __syncwarp();
    }
}

template <class T2, int W>
__global__ void __launch_bounds__(256) ebe_sum_kernel(int64_t n, int R, int LD, const int32_t* __restrict__ d2e_ptr,
                                                      const int32_t* __restrict__ d2e_elem,
                                                      const uint8_t* __restrict__ d2e_loc, const T2* __restrict__ ye,
                                                      T2* __restrict__ y, const uint8_t* __restrict__ pec,
                                                      const uint8_t* __restrict__ pm, const uint8_t* __restrict__ dsys) {
    constexpr int SUB = 32 / W;
    const int lane = threadIdx.x & 31, sub = lane / W, sl = lane - sub * W;
    if (sl >= R) return;
    const int d = dsys[sl];
    const int64_t ngroups = (int64_t)gridDim.x * (blockDim.x >> 5) * SUB;
    for (int64_t row = (blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5)) * SUB + sub; row < n;
         row += ngroups) {
        typename Cx<T2>::R re = 0, im = 0;
        if (!(pec[row] || ((pm[row] >> d) & 1))) {
            const int32_t t0 = d2e_ptr[row], t1 = d2e_ptr[row + 1];
            for (int32_t t = t0; t < t1; ++t) {
                const T2 v = ye[((int64_t)d2e_elem[t] * LD + d2e_loc[t]) * R + sl];
                re += v.x;
                im += v.y;
            }
        }
        y[row * R + sl] = Cx<T2>::make(re, im);
    }
}

// boundary groups: y_il[row] += sum_u (coef . R_u) x_il[col_u] on the group's rows
template <class T2, class T>
__global__ void bnd_batch_kernel(int nrows, int R, const int32_t* __restrict__ brow, const int32_t* __restrict__ bptr,
                                 const int32_t* __restrict__ ucol, const double* __restrict__ Rg, int64_t nu,
                                 const BC5<typename CplxOf<T>::type>* __restrict__ coef, const T2* __restrict__ x,
                                 T2* __restrict__ y,
                                 const uint8_t* __restrict__ pec, const uint8_t* __restrict__ pm,
                                 const uint8_t* __restrict__ dsys) {
    int lane = threadIdx.x & 31;
    int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= nrows || lane >= R) return;
    int row = brow[i];
    int d = dsys[lane];
    if (pec[row] || ((pm[row] >> d) & 1)) return;
    BC5<typename CplxOf<T>::type> c = coef[lane];
    T re = 0, im = 0;
    for (int32_t u = bptr[i]; u < bptr[i + 1]; ++u) {
        T rcc = (T)Rg[u], re_ = (T)Rg[nu + u], rt = (T)Rg[2 * nu + u], rs = (T)Rg[3 * nu + u], r1 = (T)Rg[4 * nu + u];
        T ar = c.cc.x * rcc + c.ce.x * re_ + c.ct.x * rt + c.cs.x * rs + c.c1.x * r1;
        T ai = c.cc.y * rcc + c.ce.y * re_ + c.ct.y * rt + c.cs.y * rs + c.c1.y * r1;
        T2 xv = x[(int64_t)ucol[u] * R + lane];
        re += ar * xv.x - ai * xv.y;
        im += ar * xv.y + ai * xv.x;
    }
    T2 v = y[(int64_t)row * R + lane];
    y[(int64_t)row * R + lane] = Cx<T2>::make((typename Cx<T2>::R)(v.x + re), (typename Cx<T2>::R)(v.y + im));
}

// ---------------------------------------------------------------------------
// layout transposes through shared memory (32 rows x R systems per tile)
// ---------------------------------------------------------------------------
template <class T2> __device__ inline T2 cvt2(float2 a);
template <class T2> __device__ inline T2 cvt2(double2 a);
template <> __device__ inline float2 cvt2<float2>(float2 a) { return a; }
template <> __device__ inline float2 cvt2<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __device__ inline double2 cvt2<double2>(float2 a) { return make_double2(a.x, a.y); }
template <> __device__ inline double2 cvt2<double2>(double2 a) { return a; }

template <class T2, class O2 = T2>
__global__ void sm2il_kernel(int64_t n, int R, const T2* __restrict__ in, int64_t ld, O2* __restrict__ out) {
    __shared__ O2 tile[RMAX][33];
    int64_t k0 = (int64_t)blockIdx.x * 32;
    for (int r = threadIdx.y; r < R; r += blockDim.y) {
        int64_t k = k0 + threadIdx.x;
        if (k < n) tile[r][threadIdx.x] = cvt2<O2>(in[r * ld + k]);
    }
    __syncthreads();
    int t = threadIdx.y * blockDim.x + threadIdx.x;
    for (int e = t; e < 32 * R; e += blockDim.x * blockDim.y) {
        int kk = e / R, r = e % R;
        int64_t k = k0 + kk;
        if (k < n) out[k * R + r] = tile[r][kk];
    }
}

template <class T2, class O2 = T2>
__global__ void il2sm_kernel(int64_t n, int R, const T2* __restrict__ in, O2* __restrict__ out, int64_t ld) {
    __shared__ O2 tile[RMAX][33];
    int64_t k0 = (int64_t)blockIdx.x * 32;
    int t = threadIdx.y * blockDim.x + threadIdx.x;
    for (int e = t; e < 32 * R; e += blockDim.x * blockDim.y) {
        int kk = e / R, r = e % R;
        int64_t k = k0 + kk;
        if (k < n) tile[r][kk] = cvt2<O2>(in[k * R + r]);
    }
    __syncthreads();
    for (int r = threadIdx.y; r < R; r += blockDim.y) {
        int64_t k = k0 + threadIdx.x;
        if (k < n) out[r * ld + k] = tile[r][threadIdx.x];
    }
}

// ---------------------------------------------------------------------------
// batched vertex-patch block Jacobi (FP32 blocks), systems [r0, r0+Rd)
// ---------------------------------------------------------------------------
// ---- bulk-copy (TMA) and mbarrier helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16) completing on bar
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for phase `parity` of bar; false if it did not complete within the poll limit
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// The FP32 blocks are stored column-major per patch (element (a, b) at
// off32[v] + b*s + a; off32[v] a multiple of 16 elements).  One CTA per patch.
// The block streams through shared memory in panels of PW columns (each
// panel is contiguous in HBM) with bulk copies (TMA) into an NS-stage ring
// whose stages complete on mbarriers; thread 0 refills a stage as soon as the
// CTA has consumed it.  The driving set's systems are split into G =
// ceil(Rd / RC) groups of at most RC systems, the block rows into SA =
// ceil(s / TR) slots of TR rows (slot j holds rows j, j + SA, ...).  Work item
// i = (g, j), g = i / SA, j = i % SA, accumulates its TR rows of T = B X for the
// RC systems of group g in registers, one item per thread (the launch has at
// least SA * G threads).  The inputs X[b][group] are staged once per patch in
// shared memory and read by all threads of a warp at the same address
// (broadcast), 16 bytes at a time, each value feeding TR complex multiply-adds.
// A stage that does not complete within the poll limit sets *err and the CTA
// stops after waiting (again bounded) for its copies in flight.
// The ring shape (NS stages of PW columns, NS <= PA_NS_MAX, PW a multiple of 4)
// is a launch parameter picked per (patch size, systems) by a short timing run
// on first use (tune_ring below).
constexpr int PA_NS_MAX = 4;
// bulk copy of block panel p (columns p*PW ..) into ring stage p % NS; the size is
// rounded up to 16 bytes, so it may read 8 bytes past the block (the FP32 block
// array ends with slack)
__device__ __forceinline__ void pa_issue(int p, int NS, int PW, int s, int smax, const float2* Bv, float2* ring,
                                         uint64_t* bar) {
    const int b0 = p * PW, pw = min(PW, s - b0);
    const uint32_t bytes = (uint32_t)(((int64_t)pw * s * 8 + 15) & ~15ll);
    uint64_t* bb = &bar[p % NS];
    mbar_expect_tx(bb, bytes);
    bulk_g2s(ring + (size_t)(p % NS) * PW * smax, Bv + (int64_t)b0 * s, bytes, bb);
}

template <int RC, int TR>
__global__ void __launch_bounds__(512, TR == 1 ? 2 : 1) patch_apply1_batch_kernel(
    int npatch, int smax, int NS, int PW, const int32_t* __restrict__ pptr, const int32_t* __restrict__ pdofs,
    const int64_t* __restrict__ off32, const float2* __restrict__ B, const float2* __restrict__ x, int R, int r0, int Rd,
    float2* __restrict__ t, int* __restrict__ err, const int32_t* __restrict__ plist, int ldt) {
    constexpr int RCP = (RC + 1) & ~1;   // group stride in shared memory (16-byte aligned groups)
    constexpr int NV = RCP / 2;          // float4 loads per input row and group
    __shared__ __align__(8) uint64_t bar[PA_NS_MAX];
    extern __shared__ float4 smem4[];
    const int v = plist ? plist[blockIdx.x] : blockIdx.x;
    const int32_t p0 = pptr[v];
    const int s = pptr[v + 1] - p0;
    const int G = (Rd + RC - 1) / RC;
    const int RP = G * RCP;
    float2* ring = reinterpret_cast<float2*>(smem4);          // NS x (PW * smax)
    float2* xs = ring + (size_t)NS * PW * smax;           // s x RP
    const float2* __restrict__ Bv = B + off32[v];
    const int npanel = (s + PW - 1) / PW;
    if (threadIdx.x == 0) {
        for (int k = 0; k < NS; ++k) mbar_init(&bar[k], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int p = 0; p < min(NS, npanel); ++p) pa_issue(p, NS, PW, s, smax, Bv, ring, bar);
    // stage X (s rows x G groups) while the first panels are in flight
    const int tot = s * RP;
    for (int e0 = threadIdx.x; e0 < tot; e0 += 4 * blockDim.x) {
        int64_t src[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = e0 + u * blockDim.x;
            src[u] = -1;
            if (e < tot) {
                const int b = e / RP, c = e - b * RP, g = c / RCP, q = c - g * RCP, l = g * RC + q;
                if (q < RC && l < Rd) src[u] = (int64_t)pdofs[p0 + b] * R + r0 + l;
            }
        }
        float2 val[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) val[u] = src[u] >= 0 ? x[src[u]] : make_float2(0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (e0 + u * blockDim.x < tot) xs[e0 + u * blockDim.x] = val[u];
    }
    __syncthreads();
    const int SA = (s + TR - 1) / TR;
    const int i = threadIdx.x;
    const bool work = i < SA * G;
    const int g = work ? i / SA : 0, j = work ? i - g * SA : 0;
    const float4* __restrict__ xg = reinterpret_cast<const float4*>(xs + g * RCP);
    const int xstride = RP / 2;   // float4 per input row
    float re[TR][RC], im[TR][RC];
    int row[TR];
#pragma unroll
    for (int r = 0; r < TR; ++r) {
        row[r] = min(j + r * SA, s - 1);   // rows past the block repeat the last row (not stored)
#pragma unroll
        for (int q = 0; q < RC; ++q) { re[r][q] = 0.f; im[r][q] = 0.f; }
    }
    // Every thread waits (bounded) for the stage; whether the whole CTA goes on
    // is decided at the end-of-panel barrier by __syncthreads_or, so all threads
    // take the same branch and none leaves while others are still in a barrier.
    bool ok = true;
    int p = 0;
    for (; p < npanel; ++p) {
        const bool got = mbar_wait(&bar[p % NS], (uint32_t)((p / NS) & 1));
        const int b0 = p * PW, pw = min(PW, s - b0);
        const float2* panel = ring + (size_t)(p % NS) * PW * smax;
        if (work && got) {
            // one block column: TR row entries against the group's RC staged inputs
            auto step = [&](const float2* __restrict__ col, const float4* __restrict__ xr) {
                float2 m[TR];
#pragma unroll
                for (int r = 0; r < TR; ++r) m[r] = col[row[r]];
#pragma unroll
                for (int h = 0; h < NV; ++h) {
                    const float4 xv = xr[h];
#pragma unroll
                    for (int r = 0; r < TR; ++r) {
                        re[r][2 * h] = fmaf(m[r].x, xv.x, fmaf(-m[r].y, xv.y, re[r][2 * h]));
                        im[r][2 * h] = fmaf(m[r].x, xv.y, fmaf(m[r].y, xv.x, im[r][2 * h]));
                        if (2 * h + 1 < RC) {
                            re[r][2 * h + 1] = fmaf(m[r].x, xv.z, fmaf(-m[r].y, xv.w, re[r][2 * h + 1]));
                            im[r][2 * h + 1] = fmaf(m[r].x, xv.w, fmaf(m[r].y, xv.z, im[r][2 * h + 1]));
                        }
                    }
                }
            };
            const float2* col = panel;
            const float4* xr = xg + b0 * xstride;
            if (pw == PW) {   // full panel: no per-column test (PW is a multiple of 4)
                for (int bb = 0; bb < PW; bb += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u, col += s, xr += xstride) step(col, xr);
                }
            } else {
                for (int bb = 0; bb < pw; ++bb, col += s, xr += xstride) step(col, xr);
            }
        }
        // every thread is done with this stage; a stage that did not complete for
        // any thread stops the whole CTA
        if (__syncthreads_or(!got)) { ok = false; break; }
        if (threadIdx.x == 0 && p + NS < npanel) pa_issue(p + NS, NS, PW, s, smax, Bv, ring, bar);
    }
    if (!ok) {
        // a stage never completed: flag it and drain the copies this CTA issued (bounded)
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            for (int q = p; q < min(npanel, p + NS); ++q) mbar_wait(&bar[q % NS], (uint32_t)((q / NS) & 1));
        }
        return;
    }
    if (work) {
        const int nc = min(RC, Rd - g * RC);
#pragma unroll
        for (int r = 0; r < TR; ++r) {
            const int a = j + r * SA;
            if (a < s) {
                float2* out = t + (int64_t)(p0 + a) * ldt + g * RC;
#pragma unroll
                for (int q = 0; q < RC; ++q)
                    if (q < nc) out[q] = make_float2(re[r][q], im[r][q]);
            }
        }
    }
}

// systems per group for a driving set of Rd systems: at most 8, groups balanced
static inline int patch_rc(int Rd) {
    const int G = (Rd + 7) / 8;
    return (Rd + G - 1) / G;
}

// FP64 row-major blocks -> FP32 column-major blocks at off32 (one CTA per patch)
__global__ void blocks_to_f32_colmajor_kernel(int npatch, const int32_t* __restrict__ pptr,
                                              const int64_t* __restrict__ poff, const int64_t* __restrict__ off32,
                                              const double2* __restrict__ in, float2* __restrict__ out,
                                              const int32_t* __restrict__ plist) {
    const int v = plist ? plist[blockIdx.x] : blockIdx.x;   // plist: only the listed patches
    const int s = pptr[v + 1] - pptr[v];
    const double2* src = in + poff[v];
    float2* dst = out + off32[v];
    for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
        const int a = e / s, b = e - a * s;
        double2 val = src[e];
        dst[b * s + a] = make_float2((float)val.x, (float)val.y);
    }
}

// y[i, r] = sum over the patch entries of DOF i of t (row stride R), for every
// system r; system r belongs to driving set dsys[r] (its Dirichlet rows zero).
// One launch for all systems, every thread group reading whole R-system rows of t.
__global__ void patch_sum_all_kernel(int64_t n, const int32_t* __restrict__ d2p_ptr,
                                     const int32_t* __restrict__ d2p_idx, const float2* __restrict__ t, int R,
                                     const uint8_t* __restrict__ pec, const uint8_t* __restrict__ pm,
                                     const uint8_t* __restrict__ dsys, float2* __restrict__ y) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * R) return;
    const int64_t i = e / R;
    const int r = (int)(e - i * R);
    float re = 0.f, im = 0.f;
    if (!(pec[i] || ((pm[i] >> dsys[r]) & 1)))
        for (int32_t q = d2p_ptr[i]; q < d2p_ptr[i + 1]; ++q) {
            const float2 v = t[(int64_t)d2p_idx[q] * R + r];
            re += v.x;
            im += v.y;
        }
    y[e] = make_float2(re, im);
}

// ---------------------------------------------------------------------------
// per-system dense kernels on system-major FP32 vectors (blockIdx.y = system)
// ---------------------------------------------------------------------------
constexpr int MDT = 8;
__global__ void __launch_bounds__(256) multidot_sys_kernel(int64_t n, int nvec, const double2* __restrict__ V,
                                                            int64_t ldsys, const double2* __restrict__ w,
                                                            const uint8_t* __restrict__ act, double2* __restrict__ part) {
    int r = blockIdx.y;
    if (!act[r]) return;
    __shared__ double red[2 * MDT][8];   // [tile entry][warp]
    const double2* Vr = V + r * ldsys;
    const double2* wr = w + r * n;
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i0 = 0; i0 < nvec; i0 += MDT) {
        double re[MDT], im[MDT];
#pragma unroll
        for (int q = 0; q < MDT; ++q) { re[q] = 0; im[q] = 0; }
        for (int64_t k = lo + threadIdx.x; k < hi; k += blockDim.x) {
            double2 b = wr[k];
#pragma unroll
            for (int q = 0; q < MDT; ++q)
                if (i0 + q < nvec) {
                    double2 a = Vr[(int64_t)(i0 + q) * n + k];
                    re[q] += a.x * b.x + a.y * b.y;
                    im[q] += a.x * b.y - a.y * b.x;
                }
        }
#pragma unroll
        for (int q = 0; q < MDT; ++q)
            for (int o = 16; o > 0; o >>= 1) {
                re[q] += __shfl_down_sync(0xffffffffu, re[q], o);
                im[q] += __shfl_down_sync(0xffffffffu, im[q], o);
            }
        __syncthreads();
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < MDT; ++q) { red[2 * q][wid] = re[q]; red[2 * q + 1][wid] = im[q]; }
        __syncthreads();
        if (threadIdx.x < 2 * MDT) {
            double acc = 0;
            for (int u = 0; u < nw; ++u) acc += red[threadIdx.x][u];
            int q = threadIdx.x >> 1;
            if (i0 + q < nvec) {
                double2* o = &part[((int64_t)r * nvec + i0 + q) * gridDim.x + blockIdx.x];
                if (threadIdx.x & 1) o->y = acc; else o->x = acc;
            }
        }
    }
}

// h[r][i] = sum of partials; H[r][col][i] (+)= h
__global__ void finish_sys_kernel(int nparts, int nvec, const double2* __restrict__ part, const uint8_t* __restrict__ act,
                                  double2* __restrict__ h, double2* __restrict__ Hcol, int64_t ldH, int accumulate) {
    int i = blockIdx.x, r = blockIdx.y;
    if (!act[r]) return;
    __shared__ double sre[256], sim[256];
    double re = 0, im = 0;
    for (int c = threadIdx.x; c < nparts; c += blockDim.x) {
        double2 p = part[((int64_t)r * nvec + i) * nparts + c];
        re += p.x;
        im += p.y;
    }
    sre[threadIdx.x] = re;
    sim[threadIdx.x] = im;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) { sre[threadIdx.x] += sre[threadIdx.x + st]; sim[threadIdx.x] += sim[threadIdx.x + st]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        h[(int64_t)r * nvec + i] = make_double2(sre[0], sim[0]);
        double2* o = &Hcol[r * ldH + i];
        if (accumulate) *o = make_double2(o->x + sre[0], o->y + sim[0]);
        else *o = make_double2(sre[0], sim[0]);
    }
}

__global__ void update_sys_kernel(int64_t n, int nvec, const double2* __restrict__ V, int64_t ldsys,
                                  const double2* __restrict__ h, const uint8_t* __restrict__ act, double2* __restrict__ w) {
    int r = blockIdx.y;
    if (!act[r]) return;
    extern __shared__ double2 shd[];
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) shd[i] = h[(int64_t)r * nvec + i];
    __syncthreads();
    const double2* Vr = V + r * ldsys;
    double2* wr = w + r * n;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 acc = wr[k];
#pragma unroll 4
        for (int i = 0; i < nvec; ++i) {
            double2 v = Vr[(int64_t)i * n + k], c = shd[i];
            acc.x -= c.x * v.x - c.y * v.y;
            acc.y -= c.x * v.y + c.y * v.x;
        }
        wr[k] = acc;
    }
}

// out[r] += sum_i y[r][i] Z[r][i]
__global__ void combo_add_sys_kernel(int64_t n, const double2* __restrict__ Z, int64_t ldsys,
                                     const double2* __restrict__ y, int ldy, const int* __restrict__ ncols,
                                     const uint8_t* __restrict__ act, double2* __restrict__ out) {
    int r = blockIdx.y;
    if (!act[r]) return;
    extern __shared__ double2 shd[];
    const int nv = ncols[r];
    for (int i = threadIdx.x; i < nv; i += blockDim.x) shd[i] = y[(int64_t)r * ldy + i];
    __syncthreads();
    const double2* Zr = Z + r * ldsys;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double re = 0, im = 0;
#pragma unroll 4
        for (int i = 0; i < nv; ++i) {
            double2 v = Zr[(int64_t)i * n + k], c = shd[i];
            re += c.x * v.x - c.y * v.y;
            im += c.x * v.y + c.y * v.x;
        }
        double2 o = out[r * n + k];
        out[r * n + k] = make_double2(o.x + re, o.y + im);
    }
}

// W[r][c] = sum_i V[r][i] Q[r][i][c]  (deflated-restart basis change; Q has ldq rows)
__global__ void rotate_sys_kernel(int64_t n, int nin, int nout, const double2* __restrict__ V, int64_t ldsys,
                                  const double2* __restrict__ Q, int ldq, int64_t qstride,
                                  const uint8_t* __restrict__ act, double2* __restrict__ W, int64_t ldw) {
    int r = blockIdx.y;
    if (!act[r]) return;
    const double2* Vr = V + r * ldsys;
    const double2* Qr = Q + (int64_t)r * qstride;
    double2* Wr = W + r * ldw;
    constexpr int CH = 8;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        for (int c0 = 0; c0 < nout; c0 += CH) {
            double re[CH], im[CH];
#pragma unroll
            for (int q = 0; q < CH; ++q) { re[q] = 0; im[q] = 0; }
            for (int i = 0; i < nin; ++i) {
                double2 v = Vr[(int64_t)i * n + k];
#pragma unroll
                for (int q = 0; q < CH; ++q)
                    if (c0 + q < nout) {
                        double2 c = __ldg(&Qr[(int64_t)(c0 + q) * ldq + i]);
                        re[q] += v.x * c.x - v.y * c.y;
                        im[q] += v.x * c.y + v.y * c.x;
                    }
            }
#pragma unroll
            for (int q = 0; q < CH; ++q)
                if (c0 + q < nout) Wr[(int64_t)(c0 + q) * n + k] = make_double2(re[q], im[q]);
        }
    }
}

template <class T2>
__global__ void nrm2_sys_kernel(int64_t n, const T2* __restrict__ x, int64_t ld, const uint8_t* __restrict__ act,
                                double* __restrict__ part) {
    int r = blockIdx.y;
    __shared__ double sh[256];
    double s = 0;
    if (act[r]) {
        const T2* xr = x + r * ld;
        int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
        int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
        for (int64_t k = lo + threadIdx.x; k < hi; k += blockDim.x) {
            double a = xr[k].x, b = xr[k].y;
            s += a * a + b * b;
        }
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(int64_t)r * gridDim.x + blockIdx.x] = sh[0];
}

__global__ void nrm2_finish_kernel(int nparts, const double* __restrict__ part, double* __restrict__ out) {
    int r = blockIdx.x;
    __shared__ double sh[256];
    double s = 0;
    for (int c = threadIdx.x; c < nparts; c += blockDim.x) s += part[(int64_t)r * nparts + c];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[r] = sqrt(sh[0]);
}

// Second-pass test of classical Gram-Schmidt: after the first pass,
// |w'|^2 = |w|^2 - sum_i |h_i|^2 (Pythagoras, no extra read), and the pass is
// repeated only if |w'| < eta |w| with eta = 0.01, i.e. only when the
// projection cancelled all but 1 % of w and the first pass's result is
// dominated by rounding (the estimate is small, and the pass therefore
// repeated, exactly when cancellation makes it inaccurate).  The classical
// Daniel-Gragg-Kaufman-Stewart threshold eta = 1/sqrt(2) asked for the second
// pass at every step of the benchmark; with eta = 0.01 the Krylov step counts
// are unchanged there, and each step loses at most ~u/eta of orthogonality.
// Accuracy does not rest on it: the batched solver's FP64 outer refinement
// checks the true residual.
__global__ void reorth_decide_kernel(int R, int nvec, const double2* __restrict__ h, const double* __restrict__ nrm0,
                                     const uint8_t* __restrict__ act, uint8_t* __restrict__ act2) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        uint8_t need = 0;
        if (act[r]) {
            double s = 0;
            for (int i = 0; i < nvec; ++i) {
                const double2 v = h[(int64_t)r * nvec + i];
                s += v.x * v.x + v.y * v.y;
            }
            const double w2 = nrm0[r] * nrm0[r];
            need = (w2 - s < 1e-4 * w2) ? 1 : 0;
        }
        act2[r] = need;
    }
}

// dst[r] = src[r] / nrm[r]; also H[r][col+1] = nrm[r]
__global__ void normalize_sys_kernel(int64_t n, const double2* __restrict__ src, int64_t lds, const double* __restrict__ nrm,
                                     const uint8_t* __restrict__ act, double2* __restrict__ dst, int64_t ldd,
                                     double2* __restrict__ Hsub, int64_t ldH) {
    int r = blockIdx.y;
    if (!act[r]) return;
    double nr = nrm[r];
    if (Hsub && blockIdx.x == 0 && threadIdx.x == 0) Hsub[r * ldH] = make_double2(nr, 0);
    double inv = nr > 0 ? 1.0 / nr : 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 a = src[r * lds + k];
        dst[r * ldd + k] = make_double2(a.x * inv, a.y * inv);
    }
}

// c = a - b  (all systems, system-major FP64)
__global__ void sub_sys_kernel(int64_t n, int R, const double2* __restrict__ a, const double2* __restrict__ b,
                               double2* __restrict__ c) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * R) return;
    c[e] = make_double2(a[e].x - b[e].x, a[e].y - b[e].y);
}

// polynomial preconditioner steps on interleaved FP32 vectors, c[r] = 1/theta_i of system r:
//   y += c u   (first = 1: y = c u)
__global__ void poly_acc_kernel(int64_t cnt, int R, const float2* __restrict__ c, const float2* __restrict__ u,
                                float2* __restrict__ y, int first) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x) {
        float2 cc = c[e % R], uu = u[e];
        float2 p = make_float2(cc.x * uu.x - cc.y * uu.y, cc.x * uu.y + cc.y * uu.x);
        if (first) y[e] = p;
        else y[e] = make_float2(y[e].x + p.x, y[e].y + p.y);
    }
}
// one polynomial step in one pass: u = src - c t (src may be u), then y += cn u
__global__ void poly_step_kernel(int64_t cnt, int R, const float2* __restrict__ c, const float2* __restrict__ cn,
                                 const float2* src, const float2* __restrict__ t, float2* u, float2* __restrict__ y) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % R);
        const float2 cc = c[r], tt = t[e], ss = src[e];
        const float2 uu = make_float2(ss.x - (cc.x * tt.x - cc.y * tt.y), ss.y - (cc.x * tt.y + cc.y * tt.x));
        u[e] = uu;
        const float2 c2 = cn[r];
        const float2 p = make_float2(c2.x * uu.x - c2.y * uu.y, c2.x * uu.y + c2.y * uu.x);
        y[e] = make_float2(y[e].x + p.x, y[e].y + p.y);
    }
}

// interleaved FP32 -> FP64
__global__ void il_f2d_kernel(int64_t cnt, const float2* __restrict__ a, double2* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = make_double2(a[i].x, a[i].y);
}

// FP64 outer pieces ---------------------------------------------------------
// out[r] = a[r] * s_r  (s_r = 1/nrm[r])  and  x[r] += nrm[r] * d[r]
__global__ void scale_sys_kernel(int64_t n, const double2* __restrict__ a, const double* __restrict__ nrm,
                                 const uint8_t* __restrict__ act, double2* __restrict__ out) {
    int r = blockIdx.y;
    double inv = (act[r] && nrm[r] > 0) ? 1.0 / nrm[r] : 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 v = a[r * n + k];
        out[r * n + k] = make_double2(v.x * inv, v.y * inv);
    }
}

__global__ void refine_sys_kernel(int64_t n, const double2* __restrict__ d, const double* __restrict__ nrm,
                                  const uint8_t* __restrict__ act, double2* __restrict__ x) {
    int r = blockIdx.y;
    if (!act[r]) return;
    double sc = nrm[r];
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 a = d[r * n + k], v = x[r * n + k];
        x[r * n + k] = make_double2(v.x + sc * a.x, v.y + sc * a.y);
    }
}

// x[r] += d[r]
__global__ void add_sys_kernel(int64_t n, const double2* __restrict__ d, const uint8_t* __restrict__ act,
                               double2* __restrict__ x) {
    int r = blockIdx.y;
    if (!act[r]) return;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 a = d[r * n + k], v = x[r * n + k];
        x[r * n + k] = make_double2(v.x + a.x, v.y + a.y);
    }
}

// r = b - y (y interleaved FP64), system-major output
__global__ void resid_kernel(int64_t n, int R, const double2* __restrict__ b, const double2* __restrict__ y_il,
                             double2* __restrict__ r) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * R) return;
    int64_t k = e / R;
    int rr = (int)(e % R);
    double2 bv = b[rr * n + k], yv = y_il[e];
    r[rr * n + k] = make_double2(bv.x - yv.x, bv.y - yv.y);
}

__global__ void real_to_f32_kernel(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// x0 lift per system: x0[r] = et[port d_r] with PEC entries removed  (system-major FP64)
__global__ void lift_batch_kernel(int64_t n, const double2* __restrict__ et, const uint8_t* __restrict__ pec,
                                  const uint8_t* __restrict__ dsys, double2* __restrict__ x0) {
    int r = blockIdx.y;
    const double2* e = et + (int64_t)dsys[r] * n;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        x0[r * n + k] = pec[k] ? make_double2(0, 0) : e[k];
}

__global__ void neg_sys_kernel(int64_t n, int R, double2* __restrict__ x) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * R) return;
    x[e] = make_double2(-x[e].x, -x[e].y);
}

// e[r] = x[r] + et[port d_r]  (driven-port values on the identity rows)
__global__ void finish_e_kernel(int64_t n, const double2* __restrict__ et, const uint8_t* __restrict__ dsys,
                                double2* __restrict__ x) {
    int r = blockIdx.y;
    const double2* e = et + (int64_t)dsys[r] * n;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 v = x[r * n + k], a = e[k];
        x[r * n + k] = make_double2(v.x + a.x, v.y + a.y);
    }
}

// ---- batched CG on the mass matrix (FP64, interleaved layout) -------------
// y_il = s_r * (V x_il)  with a real CSR matrix
__global__ void __launch_bounds__(256) spmv_real_batch_kernel(int64_t n, int R, const int32_t* __restrict__ rowptr,
                                                               const int32_t* __restrict__ cols, const double* __restrict__ V,
                                                               const double2* __restrict__ x, const double2* __restrict__ sc,
                                                               double2* __restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double2 s = lane < R ? sc[lane] : make_double2(0, 0);
    for (int64_t row = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); row < n; row += warps) {
        if (lane >= R) continue;
        double re = 0, im = 0;
        for (int32_t k = rowptr[row]; k < rowptr[row + 1]; ++k) {
            double a = V[k];
            double2 xv = x[(int64_t)cols[k] * R + lane];
            re += a * xv.x;
            im += a * xv.y;
        }
        y[row * R + lane] = make_double2(s.x * re - s.y * im, s.x * im + s.y * re);
    }
}

// per-system conj-dot over interleaved vectors: part[blk][r] = sum conj(a) b
__global__ void dot_il_kernel(int64_t n, int R, const double2* __restrict__ a, const double2* __restrict__ b,
                              double2* __restrict__ part) {
    // blockDim = (32, 8): x = system lane, y = row offset
    __shared__ double sre[8][33], sim[8][33];
    int l = threadIdx.x, ty = threadIdx.y;
    double re = 0, im = 0;
    if (l < R) {
        int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
        int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
        for (int64_t k = lo + ty; k < hi; k += blockDim.y) {
            double2 x = a[k * R + l], y = b[k * R + l];
            re += x.x * y.x + x.y * y.y;
            im += x.x * y.y - x.y * y.x;
        }
    }
    sre[ty][l] = re;
    sim[ty][l] = im;
    __syncthreads();
    if (ty == 0) {
        for (int u = 1; u < blockDim.y; ++u) { re += sre[u][l]; im += sim[u][l]; }
        part[(int64_t)blockIdx.x * 32 + l] = make_double2(re, im);
    }
}

__global__ void dot_il_finish_kernel(int nparts, const double2* __restrict__ part, double2* __restrict__ out) {
    int l = threadIdx.x;   // 32 threads
    double re = 0, im = 0;
    for (int c = 0; c < nparts; ++c) { re += part[(int64_t)c * 32 + l].x; im += part[(int64_t)c * 32 + l].y; }
    out[l] = make_double2(re, im);
}

// x += a_r p; r -= a_r q  with a_r = num_r / den_r  (interleaved)
__global__ void cg_update_batch_kernel(int64_t n, int R, const double2* __restrict__ num, const double2* __restrict__ den,
                                       const uint8_t* __restrict__ act, const double2* __restrict__ p,
                                       const double2* __restrict__ q, double2* __restrict__ x, double2* __restrict__ r) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * R) return;
    int l = (int)(e % R);
    if (!act[l]) return;
    double2 an = num[l], ad = den[l];
    double dd = ad.x * ad.x + ad.y * ad.y;
    double2 a = make_double2((an.x * ad.x + an.y * ad.y) / dd, (an.y * ad.x - an.x * ad.y) / dd);
    double2 pk = p[e], qk = q[e];
    x[e] = make_double2(x[e].x + a.x * pk.x - a.y * pk.y, x[e].y + a.x * pk.y + a.y * pk.x);
    r[e] = make_double2(r[e].x - (a.x * qk.x - a.y * qk.y), r[e].y - (a.x * qk.y + a.y * qk.x));
}

__global__ void cg_dir_batch_kernel(int64_t n, int R, const double2* __restrict__ rzn, const double2* __restrict__ rzo,
                                    const uint8_t* __restrict__ act, const double2* __restrict__ z, double2* __restrict__ p) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * R) return;
    int l = (int)(e % R);
    if (!act[l]) return;
    double2 a = rzn[l], b = rzo[l];
    double dd = b.x * b.x + b.y * b.y;
    double2 be = make_double2((a.x * b.x + a.y * b.y) / dd, (a.y * b.x - a.x * b.y) / dd);
    double2 pk = p[e];
    p[e] = make_double2(z[e].x + be.x * pk.x - be.y * pk.y, z[e].y + be.x * pk.y + be.y * pk.x);
}

__global__ void dscale_batch_kernel(int64_t n, int R, const double* __restrict__ d, const double2* __restrict__ x,
                                    double2* __restrict__ y) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * R) return;
    double s = d[e / R];
    y[e] = make_double2(s * x[e].x, s * x[e].y);
}

__global__ void diag_inv_m1_kernel(int64_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                                   const double* __restrict__ A, double* __restrict__ dinv) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double d = 0;
        for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (cols[k] == i) { d = A[k]; break; }
        dinv[i] = d != 0 ? 1.0 / d : 1.0;
    }
}

// ===========================================================================
// host orchestration
// ===========================================================================
struct System {
    double freq;
    int d;   // driving set (driven port)
};

struct Batch {
    Problem& P;
    cudaStream_t s;
    int64_t n;
    int R = 0, N = 0, m = 0, kd = 0;
    std::vector<System> sys;
    // device coefficient tables
    DBuf<VC3<float2>> vc32;
    DBuf<VC3<double2>> vc64;
    std::vector<DBuf<BC5<float2>>> bc32;
    std::vector<DBuf<BC5<double2>>> bc64;
    DBuf<uint8_t> dsys, act;
    DBuf<int> err;   // set by a kernel whose bounded wait ran out
    DBuf<float2> ye32;    // element outputs of the element-by-element product (FP32 vectors)
    DBuf<double2> ye64;   // the same for FP64 vectors
    std::vector<uint8_t> h_act;
    // systems per driving set occupy lanes [r0[d], r0[d]+Rd[d])
    std::vector<int> r0, Rd;
    explicit Batch(Problem& P_) : P(P_), s(P_.ctx->stream), n(P_.topo.n) {}
    unsigned grid1(int64_t work) const { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 65535)); }
};

template <class T2> DBuf<T2>& ebe_buffer(Batch& B);
template <> DBuf<float2>& ebe_buffer<float2>(Batch& B) { return B.ye32; }
template <> DBuf<double2>& ebe_buffer<double2>(Batch& B) { return B.ye64; }

static unsigned vgrid(const Problem& P) { return (unsigned)(P.ctx->sm_count * 4); }

// blocks per system for the per-system multi-dot: about 4 CTAs per SM over the
// whole batch, but at least 16K elements per CTA so each thread streams a long
// run per tile and the per-tile reduction is amortised.
static int md_blocks_sys(int sms, int R, int64_t n) {
    int64_t by_sm = std::max<int64_t>(1, (int64_t)4 * sms / std::max(1, R));
    int64_t by_len = std::max<int64_t>(1, n / 16384);
    return (int)std::max<int64_t>(1, std::min<int64_t>({by_sm, by_len, 512}));
}

// Element-by-element volume product y_il = (K + c Meps + ...) x_il for every
// system (Dirichlet rows zeroed); returns false where it does not apply (it
// is built for 20-DOF ND2 elements), leaving the CSR product to the caller.
template <class T2, class T>
static bool ebe_volume(Batch& B, const VC3<typename CplxOf<T>::type>* vc, const T2* x_il, T2* y_il) {
    Problem& P = B.P;
    constexpr int LD = 20;
    if (P.topo.ld != LD) return false;
    const int64_t ne = (int64_t)P.topo.ne;
    DBuf<T2>& ye = ebe_buffer<T2>(B);
    const size_t need = (size_t)ne * LD * B.R;
    if (ye.n < need) ye.alloc(need);
    const int W = B.R <= 16 ? 16 : 32;
    const size_t smem = ((size_t)12 * LD * LD + (size_t)8 * (32 / W) * 2 * LD * LD) * sizeof(T);
    const int grid = P.ctx->sm_count * 4;
    if (W == 16) {
        OPEM_CUDA(cudaFuncSetAttribute(ebe_elem_kernel<T2, T, LD, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
        ebe_elem_kernel<T2, T, LD, 16><<<grid, 256, smem, B.s>>>(ne, B.R, P.d_elem_dofs.p, P.d_geo.p,
                                                                P.d_elemcoef.p, P.d_ref.p, vc, x_il, ye.p);
        ebe_sum_kernel<T2, 16><<<P.ctx->sm_count * 8, 256, 0, B.s>>>(B.n, B.R, LD, P.d_d2e_ptr.p, P.d_d2e_elem.p,
                                                                     P.d_d2e_loc.p, ye.p, y_il, P.d_pec.p,
                                                                     P.d_portmask.p, B.dsys.p);
    } else {
        OPEM_CUDA(cudaFuncSetAttribute(ebe_elem_kernel<T2, T, LD, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
        ebe_elem_kernel<T2, T, LD, 32><<<grid, 256, smem, B.s>>>(ne, B.R, P.d_elem_dofs.p, P.d_geo.p,
                                                                P.d_elemcoef.p, P.d_ref.p, vc, x_il, ye.p);
        ebe_sum_kernel<T2, 32><<<P.ctx->sm_count * 8, 256, 0, B.s>>>(B.n, B.R, LD, P.d_d2e_ptr.p, P.d_d2e_elem.p,
                                                                     P.d_d2e_loc.p, ye.p, y_il, P.d_pec.p,
                                                                     P.d_portmask.p, B.dsys.p);
    }
    P.ctx->launches += 2;
    return true;
}

template <class T2, class T>
static void spmv_batch(Batch& B, const T* K, const T* Me, const T* Mt, const T* Ms,
                       const VC3<typename CplxOf<T>::type>* vc,
                       const std::vector<const BC5<typename CplxOf<T>::type>*>& bcs, const T2* x_il, T2* y_il) {
    Problem& P = B.P;
    if (ebe_volume<T2, T>(B, vc, x_il, y_il)) {
        // boundary groups below
    } else {
    const int grid = P.ctx->sm_count * 16;
    const int32_t* rp = P.d_rowptr.p;
    const int32_t* cl = P.d_cols.p;
#define OPEM_SPMV_LAUNCH(HT_, HS_, W_)                                                                            \
    spmv_batch_kernel<T2, T, HT_, HS_, W_><<<grid, 256, 0, B.s>>>(B.n, B.R, rp, cl, K, Me, Mt, Ms, vc, x_il, y_il, \
                                                                  P.d_pec.p, P.d_portmask.p, B.dsys.p)
    if (B.R <= 16) {
        if (Mt && Ms) OPEM_SPMV_LAUNCH(true, true, 16);
        else if (Mt) OPEM_SPMV_LAUNCH(true, false, 16);
        else if (Ms) OPEM_SPMV_LAUNCH(false, true, 16);
        else OPEM_SPMV_LAUNCH(false, false, 16);
    } else {
        if (Mt && Ms) OPEM_SPMV_LAUNCH(true, true, 32);
        else if (Mt) OPEM_SPMV_LAUNCH(true, false, 32);
        else if (Ms) OPEM_SPMV_LAUNCH(false, true, 32);
        else OPEM_SPMV_LAUNCH(false, false, 32);
    }
#undef OPEM_SPMV_LAUNCH
    ++P.ctx->launches;
    }
    for (size_t g = 0; g < P.groups.size(); ++g) {
        BGroup& G = P.groups[g];
        int nrows = (int)G.h_brow.size();
        if (G.nu == 0 || nrows == 0) continue;
        bnd_batch_kernel<T2, T><<<(nrows + 7) / 8, 256, 0, B.s>>>(nrows, B.R, G.brow.p, G.bptr.p, G.ucol.p, G.R.p, G.nu,
                                                                 bcs[g], x_il, y_il, P.d_pec.p, P.d_portmask.p, B.dsys.p);
        ++P.ctx->launches;
    }
    OPEM_CUDA(cudaGetLastError());
}

template <class T2, class O2>
static void to_il(Batch& B, const T2* sm, int64_t ld, O2* il) {
    sm2il_kernel<T2, O2><<<(unsigned)((B.n + 31) / 32), dim3(32, 8), 0, B.s>>>(B.n, B.R, sm, ld, il);
    ++B.P.ctx->launches;
}
template <class T2, class O2>
static void to_sm(Batch& B, const T2* il, O2* sm, int64_t ld) {
    il2sm_kernel<T2, O2><<<(unsigned)((B.n + 31) / 32), dim3(32, 8), 0, B.s>>>(B.n, B.R, il, sm, ld);
    ++B.P.ctx->launches;
}

// FP32 block-Jacobi blocks of one driving set: column-major, block v at off32[v]
// (a multiple of 16 elements, so every block and every even column starts
// 16-byte aligned for the bulk copies), 16 elements of slack at the end.
struct PatchSet32 {
    DBuf<float2> B;
    DBuf<int64_t> off32;
};

static std::vector<int64_t> block_offsets32(const Topology& T) {
    std::vector<int64_t> off(T.patch_ptr.size() - 1);
    int64_t o = 0;
    for (size_t v = 0; v + 1 < T.patch_ptr.size(); ++v) {
        off[v] = o;
        const int64_t sz = (int64_t)(T.patch_ptr[v + 1] - T.patch_ptr[v]);
        o += (sz * sz + 15) / 16 * 16;
    }
    off.push_back(o + 16);   // total elements incl. slack
    return off;
}

// FP32 block-Jacobi blocks for driving set d at frequency f (FP64 inversion, then
// rounded).  With `port_only`, only the patches that touch a port face are built:
// the others are the same for every driving set and are read from another set.
static void build_patchset(Batch& B, double f, int d, PatchSet32& ps, bool port_only = false) {
    Problem& P = B.P;
    const int64_t nnz = (int64_t)P.topo.cols.size();
    DBuf<double2> A(nnz);
    DBuf<uint8_t> dm(B.n);
    VolCoef vc;
    std::vector<BCoef> bc;
    system_coefficients(P, f, d, vc, bc);
    form_system_matrix(P, vc, bc, A.p);
    make_dmask(P, d, dm.p);
    const int32_t* plist = port_only ? P.d_plist_port.p : nullptr;
    const int nlist = port_only ? P.n_plist_port : P.npatch;
    DBuf<double2> B64;
    patch_blocks_fp64(P, A.p, dm.p, B64, plist, port_only ? nlist : 0);
    std::vector<int64_t> off = block_offsets32(P.topo);
    ps.B.alloc((size_t)off.back());
    OPEM_CUDA(cudaMemsetAsync(ps.B.p, 0, ps.B.bytes(), B.s));
    off.pop_back();
    ps.off32.upload(off, B.s);
    if (nlist > 0) {
        blocks_to_f32_colmajor_kernel<<<nlist, 256, 0, B.s>>>(P.npatch, P.d_patch_ptr.p, P.d_patch_off.p, ps.off32.p,
                                                              B64.p, ps.B.p, plist);
        ++P.ctx->launches;
    }
    OPEM_CUDA(cudaStreamSynchronize(B.s));
}

struct Ring { int ns, pw; };

// Patches a block apply covers: plist[0..nlist) (all patches when plist is null),
// T written with row stride ldt systems (Rd when 0).
struct PatchSel {
    const int32_t* plist = nullptr;
    int nlist = 0;
    int ldt = 0;
};

template <int RC, int TR>
static void launch_patch_apply1(Problem& P, cudaStream_t s, const PatchSet32& ps, const float2* x_il, int R, int r0,
                                int Rd, float2* t, int* err, Ring ring, const PatchSel& sel) {
    const int G = (Rd + RC - 1) / RC;
    const int RCP = (RC + 1) & ~1;
    const int smax = P.topo.max_patch;
    const size_t smem = ((size_t)ring.ns * ring.pw * smax + (size_t)smax * G * RCP) * sizeof(float2);
    if (smem > 48 * 1024) {
        // per function and process-wide: always the same device-wide value, so that
        // concurrent launches with other ring shapes or patch sizes cannot lower it
        int optin = 0;
        OPEM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, P.ctx->device));
        if (smem > (size_t)optin - 1024)
            throw OpemError(OPEM_ERR_UNSUPPORTED, "vertex patch too large for the batched block apply's ring");
        OPEM_CUDA(cudaFuncSetAttribute(patch_apply1_batch_kernel<RC, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       optin - 1024));
    }
    const int items = (smax + TR - 1) / TR * G;
    const int threads = std::max(32, (items + 31) / 32 * 32);
    if (threads > 512) throw OpemError(OPEM_ERR_UNSUPPORTED, "vertex patch too large for the batched block apply");
    const int grid = sel.plist ? sel.nlist : P.npatch;
    if (grid < 1) return;
    patch_apply1_batch_kernel<RC, TR><<<grid, threads, smem, s>>>(P.npatch, smax, ring.ns, ring.pw, P.d_patch_ptr.p,
                                                                  P.d_patch_dofs.p, ps.off32.p, ps.B.p, x_il, R, r0, Rd,
                                                                  t, err, sel.plist, sel.ldt > 0 ? sel.ldt : Rd);
    OPEM_CUDA(cudaGetLastError());
    ++P.ctx->launches;
}

// Ring shape autotuner: on the first call for a (device, largest patch, systems)
// combination, every candidate shape that fits in shared memory is run once to
// warm up and twice timed (CUDA events on the caller's stream, the call's own
// inputs; the apply overwrites its output, and every shape gives bitwise the
// same result), and the fastest is kept for the life of the process.
static std::mutex g_ring_mu;
static std::map<std::tuple<int, int, int>, Ring> g_ring_choice;

template <class Launch>
static Ring tune_ring(Problem& P, cudaStream_t s, int Rd, int RC, int G, Launch&& launch) {
    const auto key = std::make_tuple(P.ctx->device, P.topo.max_patch, Rd);
    {
        std::lock_guard<std::mutex> lk(g_ring_mu);
        auto it = g_ring_choice.find(key);
        if (it != g_ring_choice.end()) return it->second;
    }
    static const Ring cands[] = {{3, 16}, {4, 8}, {2, 32}, {3, 8}, {2, 8}, {4, 4}};
    int optin = 0;
    OPEM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, P.ctx->device));
    const int RCP = (RC + 1) & ~1;
    cudaEvent_t e0, e1;
    OPEM_CUDA(cudaEventCreate(&e0));
    OPEM_CUDA(cudaEventCreate(&e1));
    Ring best{0, 0};
    float best_ms = 1e30f;
    for (const Ring& c : cands) {
        const size_t smem = ((size_t)c.ns * c.pw * P.topo.max_patch + (size_t)P.topo.max_patch * G * RCP) * 8;
        if (smem > (size_t)optin - 1024) continue;
        launch(c);
        OPEM_CUDA(cudaEventRecord(e0, s));
        launch(c);
        launch(c);
        OPEM_CUDA(cudaEventRecord(e1, s));
        OPEM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        OPEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) { best_ms = ms; best = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best.ns == 0) throw OpemError(OPEM_ERR_UNSUPPORTED, "vertex patch too large for the batched block apply");
    std::lock_guard<std::mutex> lk(g_ring_mu);
    g_ring_choice[key] = best;
    return best;
}

template <int RC, int TR>
static void launch_patch_apply1_tuned(Problem& P, cudaStream_t s, const PatchSet32& ps, const float2* x_il, int R,
                                      int r0, int Rd, float2* t, int* err, const PatchSel& sel) {
    const int G = (Rd + RC - 1) / RC;
    const Ring ring = tune_ring(P, s, Rd, RC, G, [&](Ring c) {
        launch_patch_apply1<RC, TR>(P, s, ps, x_il, R, r0, Rd, t, err, c, sel);
    });
    launch_patch_apply1<RC, TR>(P, s, ps, x_il, R, r0, Rd, t, err, ring, sel);
}

template <int TR>
static void patch_apply1_batch_tr(Problem& P, cudaStream_t s, const PatchSet32& ps, const float2* x_il, int R, int r0,
                                  int Rd, float2* t, int* err, const PatchSel& sel) {
    switch (patch_rc(Rd)) {
        case 1: launch_patch_apply1_tuned<1, TR>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
        case 2: launch_patch_apply1_tuned<2, TR>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
        case 3: launch_patch_apply1_tuned<3, TR>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
        case 4: launch_patch_apply1_tuned<4, TR>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
        case 5: launch_patch_apply1_tuned<5, TR>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
        case 6: launch_patch_apply1_tuned<6, TR>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
        case 7: launch_patch_apply1_tuned<7, TR>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
        default: launch_patch_apply1_tuned<8, TR>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
    }
}

// Block apply variants: the tensor-core kernel (patch_tc.cu) where it applies
// (patches of at most 128 DOFs, at most 32 systems) and the FP32 FMA kernel.
enum { PA_AUTO = 0, PA_FMA = 1, PA_TENSOR = 2 };

static void patch_apply1_batch_fma(Problem& P, cudaStream_t s, const PatchSet32& ps, const float2* x_il, int R, int r0,
                                   int Rd, float2* t, int* err, const PatchSel& sel);

static void patch_apply1_batch_tensor(Problem& P, cudaStream_t s, const PatchSet32& ps, const float2* x_il, int R,
                                      int r0, int Rd, float2* t, int* err, const PatchSel& sel) {
    PatchTcLaunch L;
    L.device = P.ctx->device;
    L.sm_count = P.ctx->sm_count;
    L.npatch = P.npatch;
    L.smax = P.topo.max_patch;
    L.pptr = P.d_patch_ptr.p;
    L.pdofs = P.d_patch_dofs.p;
    L.off32 = ps.off32.p;
    L.B = ps.B.p;
    L.total_f2 = (int64_t)ps.B.n;
    L.x = x_il;
    L.R = R;
    L.r0 = r0;
    L.Rd = Rd;
    L.t = t;
    L.ldt = sel.ldt;
    L.plist = sel.plist;
    L.nlist = sel.nlist;
    L.err = err;
    patch_apply1_batch_tc(L, s);
    ++P.ctx->launches;
}

// Variant chooser: on the first call for a (device, largest patch, systems)
// combination where the tensor-core kernel applies, both kernels run once to
// warm up and twice timed (CUDA events on the caller's stream, the call's own
// inputs and patches; both overwrite their output) and the faster is kept for
// the life of the process.
static std::mutex g_pa_mu;
static std::map<std::tuple<int, int, int>, int> g_pa_choice;

// OPEM_BLOCK_APPLY=tensor|fma pins the kernel (the tensor-core one only where it
// applies); unset or anything else: the first-use timing decides.  A pinned choice
// keeps profiled runs, whose serialised launches distort the timing, on the
// kernel an unprofiled run picks.
static int pinned_variant() {
    const char* e = std::getenv("OPEM_BLOCK_APPLY");
    if (!e) return PA_AUTO;
    if (!std::strcmp(e, "tensor")) return PA_TENSOR;
    if (!std::strcmp(e, "fma")) return PA_FMA;
    return PA_AUTO;
}

static int patch_apply_variant(Problem& P, cudaStream_t s, const PatchSet32& ps, const float2* x_il, int R, int r0,
                               int Rd, float2* t, int* err, const PatchSel& sel) {
    if (!patch_tc_supported(P.ctx->device, P.topo.max_patch, Rd)) return PA_FMA;
    if (pinned_variant() != PA_AUTO) return pinned_variant();
    const auto key = std::make_tuple(P.ctx->device, P.topo.max_patch, Rd);
    {
        std::lock_guard<std::mutex> lk(g_pa_mu);
        auto it = g_pa_choice.find(key);
        if (it != g_pa_choice.end()) return it->second;
    }
    cudaEvent_t e0, e1;
    OPEM_CUDA(cudaEventCreate(&e0));
    OPEM_CUDA(cudaEventCreate(&e1));
    float ms[3] = {0, 0, 0};
    for (int v = PA_FMA; v <= PA_TENSOR; ++v) {
        auto run = [&] {
            if (v == PA_TENSOR) patch_apply1_batch_tensor(P, s, ps, x_il, R, r0, Rd, t, err, sel);
            else patch_apply1_batch_fma(P, s, ps, x_il, R, r0, Rd, t, err, sel);
        };
        run();
        OPEM_CUDA(cudaEventRecord(e0, s));
        run();
        run();
        OPEM_CUDA(cudaEventRecord(e1, s));
        OPEM_CUDA(cudaEventSynchronize(e1));
        OPEM_CUDA(cudaEventElapsedTime(&ms[v], e0, e1));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int best = ms[PA_TENSOR] <= ms[PA_FMA] ? PA_TENSOR : PA_FMA;
    std::lock_guard<std::mutex> lk(g_pa_mu);
    g_pa_choice[key] = best;
    return best;
}

// t = blocks (x restricted to the patches) for systems [r0, r0+Rd) of x_il (R systems)
static void patch_apply1_batch(Problem& P, cudaStream_t s, const PatchSet32& ps, const float2* x_il, int R, int r0,
                               int Rd, float2* t, int* err, int variant = PA_AUTO, const PatchSel& sel = PatchSel{}) {
    if (variant == PA_AUTO) variant = patch_apply_variant(P, s, ps, x_il, R, r0, Rd, t, err, sel);
    if (variant == PA_TENSOR) patch_apply1_batch_tensor(P, s, ps, x_il, R, r0, Rd, t, err, sel);
    else patch_apply1_batch_fma(P, s, ps, x_il, R, r0, Rd, t, err, sel);
}

static void patch_apply1_batch_fma(Problem& P, cudaStream_t s, const PatchSet32& ps, const float2* x_il, int R, int r0,
                                   int Rd, float2* t, int* err, const PatchSel& sel) {
    int tr = 1;   // rows per thread: 1 unless the patch needs more than 512 threads
    const int G = (Rd + patch_rc(Rd) - 1) / patch_rc(Rd);
    while (tr < 4 && (P.topo.max_patch + tr - 1) / tr * G > 512) tr *= 2;   // one work item per thread
    switch (tr) {
        case 1: patch_apply1_batch_tr<1>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
        case 4: patch_apply1_batch_tr<4>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
        default: patch_apply1_batch_tr<2>(P, s, ps, x_il, R, r0, Rd, t, err, sel); break;
    }
}

// Splits the vertex patches into those with no DOF on any port face and the
// others.  The system matrices of the driving sets differ only in port terms
// (the driven port's Dirichlet rows, the other ports' boundary terms), which
// sit on port-face DOFs, so the first kind has the same inverted block for
// every driving set.
static void ensure_patch_lists(Problem& P, cudaStream_t s) {
    if (P.n_plist_shared >= 0) return;
    const Topology& T = P.topo;
    std::vector<int32_t> sh, pt;
    for (int v = 0; v < P.npatch; ++v) {
        bool port = false;
        for (int32_t q = T.patch_ptr[v]; q < T.patch_ptr[v + 1] && !port; ++q)
            port = P.h_portmask[T.patch_dofs[q]] != 0;
        (port ? pt : sh).push_back(v);
    }
    P.d_plist_shared.upload(sh, s);
    P.d_plist_port.upload(pt, s);
    OPEM_CUDA(cudaStreamSynchronize(s));
    P.n_plist_shared = (int)sh.size();
    P.n_plist_port = (int)pt.size();
}

// y = block Jacobi (x) for every system of the batch.  Patch outputs t have row
// stride R (all systems).  With more than one driving set, the patches away from
// the ports are applied once for all R systems (one block read, every system in
// the tensor-core N dimension); the port patches per driving set with its blocks.
static void patch_apply_batch(Batch& B, const std::vector<PatchSet32>& sets, DBuf<float2>& t, const float2* x_il,
                              float2* y_il) {
    Problem& P = B.P;
    const int R = B.R;
    int first = -1, active = 0;
    for (int d = 0; d < B.N; ++d)
        if (B.Rd[d] > 0) { if (first < 0) first = d; ++active; }
    if (first < 0) return;
    ensure_patch_lists(P, B.s);
    if (active > 1 && P.n_plist_shared > 0) {
        PatchSel sh;
        sh.plist = P.d_plist_shared.p;
        sh.nlist = P.n_plist_shared;
        sh.ldt = R;
        patch_apply1_batch(P, B.s, sets[first], x_il, R, 0, R, t.p, B.err.p, PA_AUTO, sh);
        if (P.n_plist_port > 0)
            for (int d = 0; d < B.N; ++d) {
                if (B.Rd[d] == 0) continue;
                PatchSel pt;
                pt.plist = P.d_plist_port.p;
                pt.nlist = P.n_plist_port;
                pt.ldt = R;
                patch_apply1_batch(P, B.s, sets[d], x_il, R, B.r0[d], B.Rd[d], t.p + B.r0[d], B.err.p, PA_AUTO, pt);
            }
    } else {
        for (int d = 0; d < B.N; ++d) {
            if (B.Rd[d] == 0) continue;
            PatchSel all;
            all.ldt = R;
            patch_apply1_batch(P, B.s, sets[d], x_il, R, B.r0[d], B.Rd[d], t.p + B.r0[d], B.err.p, PA_AUTO, all);
        }
    }
    const int64_t work = B.n * R;
    patch_sum_all_kernel<<<(unsigned)((work + 255) / 256), 256, 0, B.s>>>(
        B.n, P.d_d2p_ptr.p, P.d_d2p_idx.p, t.p, R, P.d_pec.p, P.d_portmask.p, B.dsys.p, y_il);
    ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
}

static void nrm_sys_f64(Batch& B, const double2* x, int64_t ld, DBuf<double>& part, double* out, const uint8_t* act) {
    const int nb = 64;
    nrm2_sys_kernel<double2><<<dim3(nb, B.R), 256, 0, B.s>>>(B.n, x, ld, act, part.p);
    nrm2_finish_kernel<<<B.R, 256, 0, B.s>>>(nb, part.p, out);
    B.P.ctx->launches += 2;
}

// ---------------------------------------------------------------------------
// Batched flexible GMRES-DR (FP64 Krylov, FP32 block Jacobi) on all active
// systems in lockstep:  A d = rhs.
// The preconditioned directions z_j = M^-1 v_j are stored (Z, FP64 copy of the
// FP32 block-Jacobi output), so A Z = V H holds in FP64 whatever the
// preconditioner's precision, and d = Z y.  Deflated restarts rotate both
// bases: V <- V P_{k+1}, Z <- Z P_k.
// ---------------------------------------------------------------------------
// The inner right-hand sides are normalised residuals (unit norm), so the
// inner tolerance applies to the least-squares residual estimate directly.
struct InnerWork {
    DBuf<double2> V, Z, w, w_il, z_il64, h, part, yd, Qd, W, rhs, d;
    DBuf<float2> x_il32, z_il32, t;
    DBuf<float2> pu, py, pt, pt2, pc;   // polynomial preconditioner work (interleaved FP32) and 1/theta table
    DBuf<double2> H;     // per system (m+1) x m FP64 Hessenberg
    DBuf<double> nrm, npart, nrm0;
    DBuf<uint8_t> act2;   // systems whose second Gram-Schmidt pass is needed
    DBuf<int> ncols;
    LsqWork lsq;   // the systems' Hessenberg least squares (device, FP64)
};

// Leja ordering of polynomial roots (largest first, then maximising the product of distances)
static std::vector<cd> leja(std::vector<cd> th) {
    std::vector<cd> out;
    if (th.empty()) return out;
    size_t i0 = 0;
    for (size_t i = 1; i < th.size(); ++i)
        if (std::abs(th[i]) > std::abs(th[i0])) i0 = i;
    out.push_back(th[i0]);
    th.erase(th.begin() + i0);
    while (!th.empty()) {
        size_t best = 0;
        double bv = -1;
        for (size_t i = 0; i < th.size(); ++i) {
            double lp = 0;
            for (const cd& o : out) lp += std::log(std::abs(th[i] - o) + 1e-300);
            if (lp > bv) { bv = lp; best = i; }
        }
        out.push_back(th[best]);
        th.erase(th.begin() + best);
    }
    return out;
}

// FP32 copies of the real volume operators (matrix products inside the FP32
// polynomial preconditioner; the Arnoldi products stay FP64)
static void ensure_f32_operators(Problem& P, cudaStream_t s) {
    if (P.f_K.p) return;
    const int64_t nnz = (int64_t)P.topo.cols.size();
    const unsigned g = (unsigned)(P.ctx->sm_count * 4);
    auto cvt = [&](const DBuf<double>& a, DBuf<float>& b) {
        b.alloc(nnz);
        real_to_f32_kernel<<<g, 256, 0, s>>>(nnz, a.p, b.p);
        ++P.ctx->launches;
    };
    cvt(P.d_K, P.f_K);
    cvt(P.d_Meps, P.f_Meps);
    if (P.has_tand) cvt(P.d_Mtand, P.f_Mtand);
    if (P.has_sig) cvt(P.d_Msig, P.f_Msig);
    OPEM_CUDA(cudaGetLastError());
}

static int inner_solve(Batch& B, InnerWork& W, const std::vector<PatchSet32>& sets,
                       const std::vector<const BC5<double2>*>& bc64, const std::vector<const BC5<float2>*>& bc32, const std::vector<uint8_t>& active_in,
                       double tol, int maxits, int poly_deg, int& its_out) {
    Problem& P = B.P;
    const int64_t n = B.n;
    const int R = B.R, m = B.m, kd = B.kd;
    const int64_t ldV = (int64_t)(m + 1) * n;   // per-system stride of V (m+1 vectors) and Z (m vectors, same stride)
    const int64_t ldH = (int64_t)(m + 1) * m;
    const unsigned gy = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, P.ctx->sm_count * 2));
    const int nb = md_blocks_sys(P.ctx->sm_count, R, n);
    std::vector<uint8_t> done(R), iact(R);
    for (int r = 0; r < R; ++r) done[r] = active_in[r] ? 0 : 1;
    OPEM_CUDA(cudaMemsetAsync(W.d.p, 0, W.d.bytes(), B.s));
    OPEM_CUDA(cudaMemcpyAsync(W.w.p, W.rhs.p, (size_t)n * R * sizeof(double2), cudaMemcpyDeviceToDevice, B.s));
    std::vector<std::vector<cd>> Hh(R, std::vector<cd>((size_t)(m + 1) * m)), c(R, std::vector<cd>(m + 1));
    std::vector<int> start(R, 0), ncol(R, 0);
    std::vector<char> fresh(R, 1);
    std::vector<double> beta(R, 1.0), est(R, 1.0), hnrm(R), hest(R);
    std::vector<std::vector<cd>> ys(R);
    // the Hessenberg least squares runs on the device (W.lsq); the host reads
    // the residual estimates per step, and H itself only where it forms the
    // polynomial's roots and the deflated restarts
    auto download_H = [&]() {   // W.H -> Hh of the systems still running, zero outside each column's rows
        std::vector<double2> hh((size_t)R * ldH);
        OPEM_CUDA(cudaMemcpyAsync(hh.data(), W.H.p, hh.size() * sizeof(double2), cudaMemcpyDeviceToHost, B.s));
        OPEM_CUDA(cudaStreamSynchronize(B.s));
        for (int r = 0; r < R; ++r) {
            if (done[r]) continue;
            for (int j = 0; j < m; ++j) {
                const int top = j < start[r] ? start[r] : j + 1;
                for (int i = 0; i <= m; ++i) {
                    const double2 v = i <= top && j < std::max(ncol[r], start[r]) ? hh[(size_t)r * ldH + (size_t)j * (m + 1) + i]
                                                                                  : make_double2(0, 0);
                    Hh[r][i + (size_t)j * (m + 1)] = cd(v.x, v.y);
                }
            }
        }
    };
    int its = 0;
    int npoly = 0;   // degree of the polynomial preconditioner in use (0: block Jacobi alone)
    auto upload_act = [&](const std::vector<uint8_t>& a) {
        OPEM_CUDA(cudaMemcpyAsync(B.act.p, a.data(), R, cudaMemcpyHostToDevice, B.s));
    };
    auto apply_A = [&](const double2* x_il64, double2* y_sm) {   // y = A x (FP64), via interleaved layout
        spmv_batch<double2, double>(B, P.d_K.p, P.d_Meps.p, P.has_tand ? P.d_Mtand.p : nullptr,
                                    P.has_sig ? P.d_Msig.p : nullptr, B.vc64.p, bc64, x_il64, W.w_il.p);
        to_sm(B, W.w_il.p, y_sm, n);
    };
    while (true) {
        for (int r = 0; r < R; ++r) iact[r] = (!done[r] && fresh[r]) ? 1 : 0;
        upload_act(iact);
        nrm_sys_f64(B, W.w.p, n, W.npart, W.nrm.p, B.act.p);
        normalize_sys_kernel<<<dim3(gy, R), 256, 0, B.s>>>(n, W.w.p, n, W.nrm.p, B.act.p, W.V.p, ldV, nullptr, 0);
        ++P.ctx->launches;
        OPEM_CUDA(cudaMemcpyAsync(hnrm.data(), W.nrm.p, R * sizeof(double), cudaMemcpyDeviceToHost, B.s));
        OPEM_CUDA(cudaStreamSynchronize(B.s));
        int jmin = m;
        std::vector<double2> hc0((size_t)R * (m + 1), make_double2(0, 0));
        std::vector<uint8_t> rst(R, 0);
        for (int r = 0; r < R; ++r) {
            if (done[r]) continue;
            if (fresh[r]) {
                beta[r] = hnrm[r];
                std::fill(c[r].begin(), c[r].end(), 0.0);
                c[r][0] = beta[r];
                start[r] = 0;
                if (!(beta[r] > 0)) { done[r] = 1; continue; }
            }
            rst[r] = 1;
            for (int i = 0; i <= m; ++i) hc0[(size_t)r * (m + 1) + i] = make_double2(c[r][i].real(), c[r][i].imag());
            ncol[r] = start[r];
            jmin = std::min(jmin, start[r]);
        }
        bool any = false;
        for (int r = 0; r < R; ++r) any |= !done[r];
        if (!any) break;
        // least-squares state of the cycle: g = c, the restart block's columns
        W.lsq.start_cycle(rst, hc0, start, W.H.p, B.s, est);
        ++P.ctx->launches;
        std::vector<uint8_t> cyc(R, 0);
        for (int r = 0; r < R; ++r) cyc[r] = !done[r];
        for (int j = jmin; j < m; ++j) {
            for (int r = 0; r < R; ++r) iact[r] = (cyc[r] && j >= start[r]) ? 1 : 0;
            bool anyj = false;
            for (int r = 0; r < R; ++r) anyj |= iact[r];
            if (!anyj) break;
            upload_act(iact);
            // z_j = P v_j, kept in Z (P = M^-1 for the first steps, then M^-1 q(A M^-1)
            // with the GMRES polynomial q of each system, all in FP32); w = A z_j (FP64)
            to_il(B, W.V.p + (int64_t)j * n, ldV, W.x_il32.p);
            if (npoly > 0) {
                const int64_t cnt = n * R;
                const unsigned gp = (unsigned)std::min<int64_t>((cnt + 255) / 256, P.ctx->sm_count * 16);
                // y = q(A M^-1) v with Leja-ordered roots: u_0 = v, y = u_0/theta_0, then
                // u_{i+1} = u_i - (A M^-1 u_i)/theta_i and y += u_{i+1}/theta_{i+1} in one pass
                poly_acc_kernel<<<gp, 256, 0, B.s>>>(cnt, R, W.pc.p, W.x_il32.p, W.py.p, 1);
                ++P.ctx->launches;
                for (int i = 0; i + 1 < npoly; ++i) {
                    const float2* src = i == 0 ? W.x_il32.p : W.pu.p;
                    patch_apply_batch(B, sets, W.t, src, W.pt.p);
                    spmv_batch<float2, float>(B, P.f_K.p, P.f_Meps.p, P.has_tand ? P.f_Mtand.p : nullptr,
                                              P.has_sig ? P.f_Msig.p : nullptr, B.vc32.p, bc32, W.pt.p, W.pt2.p);
                    poly_step_kernel<<<gp, 256, 0, B.s>>>(cnt, R, W.pc.p + (size_t)i * R, W.pc.p + (size_t)(i + 1) * R,
                                                          src, W.pt2.p, W.pu.p, W.py.p);
                    ++P.ctx->launches;
                }
                patch_apply_batch(B, sets, W.t, W.py.p, W.z_il32.p);
            } else {
                patch_apply_batch(B, sets, W.t, W.x_il32.p, W.z_il32.p);
            }
            to_sm(B, W.z_il32.p, W.Z.p + (int64_t)j * n, ldV);
            il_f2d_kernel<<<vgrid(P), 256, 0, B.s>>>(n * R, W.z_il32.p, W.z_il64.p);
            ++P.ctx->launches;
            apply_A(W.z_il64.p, W.w.p);
            // classical Gram-Schmidt; the second pass only for the systems whose
            // first pass cancelled all but 1 % of |w| (decided on the device)
            nrm_sys_f64(B, W.w.p, n, W.npart, W.nrm0.p, B.act.p);
            for (int pass = 0; pass < 2; ++pass) {
                const uint8_t* ap = pass == 0 ? B.act.p : W.act2.p;
                multidot_sys_kernel<<<dim3(nb, R), 256, 0, B.s>>>(n, j + 1, W.V.p, ldV, W.w.p, ap, W.part.p);
                finish_sys_kernel<<<dim3(j + 1, R), 256, 0, B.s>>>(nb, j + 1, W.part.p, ap, W.h.p,
                                                                   W.H.p + (int64_t)j * (m + 1), ldH, pass);
                update_sys_kernel<<<dim3(gy, R), 256, (j + 1) * sizeof(double2), B.s>>>(n, j + 1, W.V.p, ldV, W.h.p,
                                                                                       ap, W.w.p);
                P.ctx->launches += 3;
                if (pass == 0) {
                    reorth_decide_kernel<<<1, 32, 0, B.s>>>(R, j + 1, W.h.p, W.nrm0.p, B.act.p, W.act2.p);
                    ++P.ctx->launches;
                }
            }
            nrm_sys_f64(B, W.w.p, n, W.npart, W.nrm.p, B.act.p);
            normalize_sys_kernel<<<dim3(gy, R), 256, 0, B.s>>>(n, W.w.p, n, W.nrm.p, B.act.p,
                                                                W.V.p + (int64_t)(j + 1) * n, ldV,
                                                                W.H.p + (int64_t)j * (m + 1) + j + 1, ldH);
            ++P.ctx->launches;
            OPEM_CUDA(cudaGetLastError());
            W.lsq.step(j, B.act.p, W.H.p, B.s, hest);
            ++P.ctx->launches;
            if (P.cancel.load(std::memory_order_relaxed)) throw OpemError(OPEM_ERR_CANCELLED, "request cancelled");
            ++its;
            for (int r = 0; r < R; ++r) {
                if (!iact[r]) continue;
                est[r] = hest[r];
                ncol[r] = j + 1;
                if (!std::isfinite(est[r]) || est[r] <= tol) cyc[r] = 0;
            }
            if (poly_deg > 1 && npoly == 0 && j + 1 == poly_deg) {
                download_H();
                // harmonic Ritz values of the first poly_deg steps of every system -> GMRES polynomial roots
                const int dg = poly_deg;
                std::vector<float2> hc((size_t)dg * R, make_float2(0.f, 0.f));
                bool okall = true;
                for (int r = 0; r < R; ++r) {
                    if (done[r]) continue;
                    std::vector<cd> Hd((size_t)dg * dg), HdH((size_t)dg * dg), f(dg, 0.0);
                    for (int b2 = 0; b2 < dg; ++b2)
                        for (int a2 = 0; a2 < dg; ++a2) {
                            Hd[a2 + (size_t)b2 * dg] = Hh[r][a2 + (size_t)b2 * (m + 1)];
                            HdH[b2 + (size_t)a2 * dg] = std::conj(Hh[r][a2 + (size_t)b2 * (m + 1)]);
                        }
                    f[dg - 1] = 1.0;
                    std::vector<cd> th, gv;
                    if (!lu_solve(dg, HdH, f)) { okall = false; break; }
                    double h2 = std::norm(Hh[r][dg + (size_t)(dg - 1) * (m + 1)]);
                    for (int a2 = 0; a2 < dg; ++a2) Hd[a2 + (size_t)(dg - 1) * dg] += h2 * f[a2];
                    if (!eig_smallest(dg, Hd, dg, th, gv)) { okall = false; break; }
                    double tmax = 0;
                    for (auto& t3 : th) tmax = std::max(tmax, std::abs(t3));
                    for (auto& t3 : th)
                        if (!(std::abs(t3) > 1e-6 * tmax)) okall = false;
                    th = leja(th);
                    for (int i = 0; i < dg; ++i) {
                        cd ci = 1.0 / th[i];
                        hc[(size_t)i * R + r] = make_float2((float)ci.real(), (float)ci.imag());
                    }
                }
                if (okall) {
                    OPEM_CUDA(cudaMemcpyAsync(W.pc.p, hc.data(), hc.size() * sizeof(float2), cudaMemcpyHostToDevice, B.s));
                    npoly = dg;
                }
            }
            if (its >= maxits) break;
        }
        // d += Z y, y from the device least squares
        std::vector<int> nc(R, 0);
        int ymax = 0;
        for (int r = 0; r < R; ++r) {
            iact[r] = (!done[r] && ncol[r] > 0) ? 1 : 0;
            if (!iact[r]) continue;
            nc[r] = ncol[r];
            ymax = std::max(ymax, ncol[r]);
        }
        W.lsq.check(B.s);
        if (ymax > 0) {
            upload_act(iact);
            OPEM_CUDA(cudaMemcpyAsync(W.ncols.p, nc.data(), R * sizeof(int), cudaMemcpyHostToDevice, B.s));
            W.lsq.solve(W.ncols.p, B.act.p, W.yd.p, m, B.s);
            ++P.ctx->launches;
            combo_add_sys_kernel<<<dim3(gy, R), 256, ymax * sizeof(double2), B.s>>>(n, W.Z.p, ldV, W.yd.p, m, W.ncols.p,
                                                                                   B.act.p, W.d.p);
            ++P.ctx->launches;
        }
        bool all = true;
        for (int r = 0; r < R; ++r) {
            if (done[r]) continue;
            if (est[r] <= tol || !std::isfinite(est[r])) done[r] = 1;
            all &= (bool)done[r];
        }
        if (all || its >= maxits) break;
        // systems that cannot deflate restart from their true residual (FP64)
        bool need_fresh = false;
        for (int r = 0; r < R; ++r) need_fresh |= (!done[r] && (kd == 0 || ncol[r] < m));
        if (need_fresh) {
            to_il(B, W.d.p, n, W.z_il64.p);
            apply_A(W.z_il64.p, W.w.p);
            sub_sys_kernel<<<(unsigned)((n * R + 255) / 256), 256, 0, B.s>>>(n, R, W.rhs.p, W.w.p, W.w.p);
            ++P.ctx->launches;
        }
        // deflated restarts (host FP64, systems in parallel) from the cycle's H and y
        bool want_def = false;
        for (int r = 0; r < R; ++r) want_def |= (!done[r] && kd > 0 && ncol[r] == m);
        if (want_def) {
            download_H();
            std::vector<double2> yh((size_t)R * m);
            OPEM_CUDA(cudaMemcpyAsync(yh.data(), W.yd.p, yh.size() * sizeof(double2), cudaMemcpyDeviceToHost, B.s));
            OPEM_CUDA(cudaStreamSynchronize(B.s));
            for (int r = 0; r < R; ++r) {
                if (done[r] || ncol[r] != m) continue;
                ys[r].assign(m, 0.0);
                for (int i = 0; i < m; ++i) ys[r][i] = cd(yh[(size_t)r * m + i].x, yh[(size_t)r * m + i].y);
            }
        }
        std::vector<std::vector<cd>> Pm(R), Hn(R), cn(R);
        std::vector<char> ok(R, 0);
#pragma omp parallel for schedule(dynamic, 1)
        for (int r = 0; r < R; ++r) {
            if (done[r] || kd == 0 || ncol[r] < m) continue;
            ok[r] = gmres_dr_deflate(m, kd, Hh[r], c[r], ys[r], Pm[r], Hn[r], cn[r]) ? 1 : 0;
        }
        bool anydef = false;
        const int64_t qstride = (int64_t)(m + 1) * (kd + 1);
        std::vector<double2> Qh((size_t)R * qstride, make_double2(0, 0));
        for (int r = 0; r < R; ++r) {
            iact[r] = 0;
            fresh[r] = 1;
            if (done[r] || !ok[r]) continue;
            iact[r] = 1;
            anydef = true;
            for (size_t t2 = 0; t2 < Pm[r].size(); ++t2)
                Qh[(size_t)r * qstride + t2] = make_double2(Pm[r][t2].real(), Pm[r][t2].imag());
        }
        if (anydef) {
            upload_act(iact);
            OPEM_CUDA(cudaMemcpyAsync(W.Qd.p, Qh.data(), Qh.size() * sizeof(double2), cudaMemcpyHostToDevice, B.s));
            const int64_t ldw = (int64_t)(kd + 1) * n;
            // V <- V P_{k+1}
            rotate_sys_kernel<<<dim3(gy, R), 256, 0, B.s>>>(n, m + 1, kd + 1, W.V.p, ldV, W.Qd.p, m + 1, qstride, B.act.p,
                                                             W.W.p, ldw);
            ++P.ctx->launches;
            for (int r = 0; r < R; ++r)
                if (iact[r])
                    OPEM_CUDA(cudaMemcpyAsync(W.V.p + r * ldV, W.W.p + r * ldw, (size_t)(kd + 1) * n * sizeof(double2),
                                              cudaMemcpyDeviceToDevice, B.s));
            // Z <- Z P_k (first m rows, first kd columns of P)
            rotate_sys_kernel<<<dim3(gy, R), 256, 0, B.s>>>(n, m, kd, W.Z.p, ldV, W.Qd.p, m + 1, qstride, B.act.p, W.W.p,
                                                             ldw);
            ++P.ctx->launches;
            for (int r = 0; r < R; ++r)
                if (iact[r])
                    OPEM_CUDA(cudaMemcpyAsync(W.Z.p + r * ldV, W.W.p + r * ldw, (size_t)kd * n * sizeof(double2),
                                              cudaMemcpyDeviceToDevice, B.s));
            OPEM_CUDA(cudaStreamSynchronize(B.s));
            for (int r = 0; r < R; ++r) {
                if (!iact[r]) continue;
                // the restart block becomes the first kd columns of the next cycle's H
                std::vector<double2> hn((size_t)ldH);
                for (size_t t2 = 0; t2 < hn.size(); ++t2) hn[t2] = make_double2(Hn[r][t2].real(), Hn[r][t2].imag());
                OPEM_CUDA(cudaMemcpyAsync(W.H.p + r * ldH, hn.data(), hn.size() * sizeof(double2), cudaMemcpyHostToDevice, B.s));
                OPEM_CUDA(cudaStreamSynchronize(B.s));
                c[r] = cn[r];
                start[r] = kd;
                fresh[r] = 0;
            }
        }
    }
    its_out = its;
    return OPEM_OK;
}

// ---------------------------------------------------------------------------
// batched CG for the H projection (FP64): M1 h_r = (j/(w_r mu0)) Q e_r
// ---------------------------------------------------------------------------
static int mass_cg_batch(Batch& B, const double2* e_il, double2* h_il, double rtol, int maxits, int& its_out) {
    Problem& P = B.P;
    const int64_t n = B.n;
    const int R = B.R;
    const int64_t nR = n * R;
    DBuf<double> dinv(n);
    DBuf<double2> r(nR), z(nR), p(nR), q(nR), part((size_t)32 * 1024), sc(32), rz(32), pq(32), rzn(32);
    std::vector<double2> hsc(32, make_double2(0, 0));
    for (int i = 0; i < R; ++i) hsc[i] = make_double2(0.0, 1.0 / (2 * M_PI * B.sys[i].freq * MU0_M));
    OPEM_CUDA(cudaMemcpyAsync(sc.p, hsc.data(), 32 * sizeof(double2), cudaMemcpyHostToDevice, B.s));
    int grid = P.ctx->sm_count * 16;
    spmv_real_batch_kernel<<<grid, 256, 0, B.s>>>(n, R, P.d_rowptr.p, P.d_cols.p, P.d_Q.p, e_il, sc.p, r.p);  // r = b
    diag_inv_m1_kernel<<<vgrid(P), 256, 0, B.s>>>(n, P.d_rowptr.p, P.d_cols.p, P.d_M1.p, dinv.p);
    P.ctx->launches += 2;
    OPEM_CUDA(cudaMemsetAsync(h_il, 0, nR * sizeof(double2), B.s));
    unsigned ge = (unsigned)((nR + 255) / 256);
    const int nb = 256;
    auto dot = [&](const double2* a, const double2* b, double2* out) {
        dot_il_kernel<<<nb, dim3(32, 8), 0, B.s>>>(n, R, a, b, part.p);
        dot_il_finish_kernel<<<1, 32, 0, B.s>>>(nb, part.p, out);
        P.ctx->launches += 2;
    };
    std::vector<double2> hb(32), hr(32);
    dot(r.p, r.p, rz.p);
    OPEM_CUDA(cudaMemcpyAsync(hb.data(), rz.p, 32 * sizeof(double2), cudaMemcpyDeviceToHost, B.s));
    dscale_batch_kernel<<<ge, 256, 0, B.s>>>(n, R, dinv.p, r.p, z.p);
    OPEM_CUDA(cudaMemcpyAsync(p.p, z.p, nR * sizeof(double2), cudaMemcpyDeviceToDevice, B.s));
    dot(r.p, z.p, rz.p);
    P.ctx->launches += 3;
    OPEM_CUDA(cudaStreamSynchronize(B.s));
    std::vector<double> bn(R);
    for (int i = 0; i < R; ++i) bn[i] = std::sqrt(hb[i].x);
    std::vector<uint8_t> act(R, 1);
    for (int i = 0; i < R; ++i) act[i] = bn[i] > 0;
    OPEM_CUDA(cudaMemcpyAsync(B.act.p, act.data(), R, cudaMemcpyHostToDevice, B.s));
    DBuf<double2> one(32);
    std::vector<double2> h1(32, make_double2(1, 0));
    OPEM_CUDA(cudaMemcpyAsync(one.p, h1.data(), 32 * sizeof(double2), cudaMemcpyHostToDevice, B.s));
    int its = 0;
    while (its < maxits) {
        spmv_real_batch_kernel<<<grid, 256, 0, B.s>>>(n, R, P.d_rowptr.p, P.d_cols.p, P.d_M1.p, p.p, one.p, q.p);
        dot(p.p, q.p, pq.p);
        cg_update_batch_kernel<<<ge, 256, 0, B.s>>>(n, R, rz.p, pq.p, B.act.p, p.p, q.p, h_il, r.p);
        P.ctx->launches += 2;
        ++its;
        if (its % 10 == 0 || its >= maxits) {
            dot(r.p, r.p, rzn.p);
            OPEM_CUDA(cudaMemcpyAsync(hr.data(), rzn.p, 32 * sizeof(double2), cudaMemcpyDeviceToHost, B.s));
            OPEM_CUDA(cudaStreamSynchronize(B.s));
            bool all = true;
            for (int i = 0; i < R; ++i) {
                if (!act[i]) continue;
                double rn = std::sqrt(hr[i].x);
                if (rn <= rtol * bn[i] || !std::isfinite(rn)) act[i] = 0;
                all &= !act[i];
            }
            OPEM_CUDA(cudaMemcpyAsync(B.act.p, act.data(), R, cudaMemcpyHostToDevice, B.s));
            if (all) break;
        }
        dscale_batch_kernel<<<ge, 256, 0, B.s>>>(n, R, dinv.p, r.p, z.p);
        dot(r.p, z.p, rzn.p);
        cg_dir_batch_kernel<<<ge, 256, 0, B.s>>>(n, R, rzn.p, rz.p, B.act.p, z.p, p.p);
        OPEM_CUDA(cudaMemcpyAsync(rz.p, rzn.p, 32 * sizeof(double2), cudaMemcpyDeviceToDevice, B.s));
        P.ctx->launches += 2;
    }
    OPEM_CUDA(cudaGetLastError());
    its_out = its;
    return OPEM_OK;
}

// ---------------------------------------------------------------------------
// one batch of systems: returns Cp/Cm per system and stats
// ---------------------------------------------------------------------------
struct BatchOut {
    std::vector<cd> Cp, Cm;   // [system][port]
    int inner_its = 0, outer = 0, h_its = 0;
    double worst = 0;
    bool converged = true;
};

// Coefficient tables of the batch's systems (FP64 and FP32 copies), device pointers in bp32/bp64.
static void setup_coefficients(Batch& B, const std::vector<System>& systems, std::vector<const BC5<float2>*>& bp32,
                               std::vector<const BC5<double2>*>& bp64) {
    Problem& P = B.P;
    const int R = B.R;
    std::vector<VC3<float2>> v32(R);
    std::vector<VC3<double2>> v64(R);
    std::vector<std::vector<BC5<float2>>> b32(P.groups.size(), std::vector<BC5<float2>>(R));
    std::vector<std::vector<BC5<double2>>> b64(P.groups.size(), std::vector<BC5<double2>>(R));
    std::vector<uint8_t> ds(R);
    for (int r = 0; r < R; ++r) {
        VolCoef vc;
        std::vector<BCoef> bc;
        system_coefficients(P, systems[r].freq, systems[r].d, vc, bc);
        v64[r] = {vc.c_eps, vc.c_tand, vc.c_sig};
        v32[r] = {make_float2((float)vc.c_eps.x, (float)vc.c_eps.y), make_float2((float)vc.c_tand.x, (float)vc.c_tand.y),
                  make_float2((float)vc.c_sig.x, (float)vc.c_sig.y)};
        for (size_t g = 0; g < bc.size(); ++g) {
            const BCoef& c = bc[g];
            b64[g][r] = {c.c_cc, c.c_eps, c.c_tand, c.c_sig, c.c_one};
            auto f = [](double2 a) { return make_float2((float)a.x, (float)a.y); };
            b32[g][r] = {f(c.c_cc), f(c.c_eps), f(c.c_tand), f(c.c_sig), f(c.c_one)};
        }
        ds[r] = (uint8_t)systems[r].d;
    }
    B.vc32.upload(v32, B.s);
    B.vc64.upload(v64, B.s);
    bp32.clear();
    bp64.clear();
    B.bc32.resize(P.groups.size());
    B.bc64.resize(P.groups.size());
    for (size_t g = 0; g < P.groups.size(); ++g) {
        B.bc32[g].upload(b32[g], B.s);
        B.bc64[g].upload(b64[g], B.s);
        bp32.push_back(B.bc32[g].p);
        bp64.push_back(B.bc64[g].p);
    }
    B.dsys.upload(ds, B.s);
    B.act.alloc(RMAX);
    B.err.alloc(1);
    B.err.zero(B.s);
}

// raises if a kernel of the batch flagged a bounded wait that ran out
static void check_batch_err(Batch& B) {
    int e = 0;
    OPEM_CUDA(cudaMemcpyAsync(&e, B.err.p, sizeof(int), cudaMemcpyDeviceToHost, B.s));
    OPEM_CUDA(cudaStreamSynchronize(B.s));
    if (e) throw OpemError(OPEM_ERR_TIMEOUT, "batched block apply: a bulk-copy stage did not complete");
}

static void solve_batch(Problem& P, const std::vector<System>& systems, const opem_solver_opts& o, BatchOut& out) {
    Batch B(P);
    B.sys = systems;
    B.R = (int)systems.size();
    B.N = P.nports;
    B.m = std::max(2, o.restart);
    B.kd = std::max(0, std::min(o.deflate, B.m - 2));
    const int R = B.R, N = B.N, m = B.m, kd = B.kd;
    const int64_t n = B.n, nR = n * R;
    // systems sorted by driving set -> contiguous lanes
    B.r0.assign(N, 0);
    B.Rd.assign(N, 0);
    for (int r = 0; r < R; ++r) B.Rd[systems[r].d]++;
    for (int d = 1; d < N; ++d) B.r0[d] = B.r0[d - 1] + B.Rd[d - 1];
    for (int r = 1; r < R; ++r)
        if (systems[r].d < systems[r - 1].d) throw OpemError(OPEM_ERR_ARG, "batch systems must be ordered by driving set");
    std::vector<const BC5<float2>*> bp32;
    std::vector<const BC5<double2>*> bp64;
    setup_coefficients(B, systems, bp32, bp64);
    // block-Jacobi sets: one per driving set, at the batch's middle frequency
    std::vector<PatchSet32> sets(N);
    double fmid = 0.5 * (systems.front().freq + systems.back().freq);
    {
        double lo = 1e300, hi = 0;
        for (auto& sy : systems) { lo = std::min(lo, sy.freq); hi = std::max(hi, sy.freq); }
        fmid = 0.5 * (lo + hi);
    }
    // the first active driving set gets every block; the others only those of the
    // patches touching a port face (patch_apply_batch reads the rest from the first)
    ensure_patch_lists(P, B.s);
    int first = -1;
    for (int d = 0; d < N; ++d)
        if (B.Rd[d] > 0) {
            build_patchset(B, fmid, d, sets[d], first >= 0 && P.n_plist_shared > 0);
            if (first < 0) first = d;
        }
    // right-hand sides b_r = -(A_r x0_r) with Dirichlet rows 0  (FP64)
    DBuf<double2> x0(nR), x0_il(nR), y_il(nR), b(nR), x(nR), r64(nR);
    const unsigned gy = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, P.ctx->sm_count * 2));
    const double2* et = reinterpret_cast<const double2*>(P.d_et.p);
    lift_batch_kernel<<<dim3(gy, R), 256, 0, B.s>>>(n, et, P.d_pec.p, B.dsys.p, x0.p);
    ++P.ctx->launches;
    to_il(B, x0.p, n, x0_il.p);
    spmv_batch<double2, double>(B, P.d_K.p, P.d_Meps.p, P.has_tand ? P.d_Mtand.p : nullptr,
                                P.has_sig ? P.d_Msig.p : nullptr, B.vc64.p, bp64, x0_il.p, y_il.p);
    to_sm(B, y_il.p, b.p, n);
    neg_sys_kernel<<<(unsigned)((nR + 255) / 256), 256, 0, B.s>>>(n, R, b.p);
    ++P.ctx->launches;
    OPEM_CUDA(cudaMemsetAsync(x.p, 0, nR * sizeof(double2), B.s));
    DBuf<double> nrm(RMAX), npart((size_t)RMAX * 64);
    std::vector<uint8_t> all1(R, 1), act(R, 1);
    OPEM_CUDA(cudaMemcpyAsync(B.act.p, all1.data(), R, cudaMemcpyHostToDevice, B.s));
    nrm_sys_f64(B, b.p, n, npart, nrm.p, B.act.p);
    std::vector<double> bn(R), rn(R);
    OPEM_CUDA(cudaMemcpyAsync(bn.data(), nrm.p, R * sizeof(double), cudaMemcpyDeviceToHost, B.s));
    OPEM_CUDA(cudaStreamSynchronize(B.s));
    // inner work buffers
    InnerWork W;
    const int64_t ldV = (int64_t)(m + 1) * n;
    const int nbm = md_blocks_sys(P.ctx->sm_count, R, n);
    W.V.alloc((size_t)R * ldV);
    W.Z.alloc((size_t)R * ldV);
    W.w.alloc(nR);
    W.w_il.alloc(nR);
    W.z_il64.alloc(nR);
    W.x_il32.alloc(nR);
    W.z_il32.alloc(nR);
    W.t.alloc(P.topo.patch_dofs.size() * (size_t)R);   // patch outputs of every system (row stride R)
    W.h.alloc((size_t)R * (m + 1));
    W.part.alloc((size_t)R * (m + 1) * nbm);
    W.yd.alloc((size_t)R * m);
    W.Qd.alloc((size_t)R * (m + 1) * (kd + 1));
    W.W.alloc((size_t)R * (kd + 1) * n);
    W.rhs.alloc(nR);
    W.d.alloc(nR);
    W.H.alloc((size_t)R * (m + 1) * m);
    W.lsq.alloc(R, m, kd, B.s);
    W.nrm.alloc(RMAX);
    W.nrm0.alloc(RMAX);
    W.act2.alloc(RMAX);
    W.npart.alloc((size_t)RMAX * 64);
    W.ncols.alloc(RMAX);
    if (o.poly_degree > 1) {
        W.pu.alloc(nR);
        W.py.alloc(nR);
        W.pt.alloc(nR);
        W.pt2.alloc(nR);
        W.pc.alloc((size_t)o.poly_degree * R);
    }
    // outer FP64 refinement (normally one pass: the inner Krylov solve is FP64)
    OPEM_CUDA(cudaMemcpyAsync(r64.p, b.p, nR * sizeof(double2), cudaMemcpyDeviceToDevice, B.s));
    rn = bn;
    int outer = 0, inner_total = 0;
    for (int r = 0; r < R; ++r) act[r] = (bn[r] > 0 && rn[r] > o.rtol * bn[r]) ? 1 : 0;
    while (outer < 4) {
        bool any = false;
        for (int r = 0; r < R; ++r) any |= act[r];
        if (!any || inner_total >= o.maxits) break;
        ++outer;
        // inner tolerance relative to this step's residual, aiming at rtol ||b||
        double tol_in = 1.0;
        for (int r = 0; r < R; ++r)
            if (act[r]) tol_in = std::min(tol_in, 0.5 * o.rtol * bn[r] / rn[r]);
        tol_in = std::max(tol_in, 1e-14);
        OPEM_CUDA(cudaMemcpyAsync(B.act.p, act.data(), R, cudaMemcpyHostToDevice, B.s));
        OPEM_CUDA(cudaMemcpyAsync(nrm.p, rn.data(), R * sizeof(double), cudaMemcpyHostToDevice, B.s));
        scale_sys_kernel<<<dim3(gy, R), 256, 0, B.s>>>(n, r64.p, nrm.p, B.act.p, W.rhs.p);
        ++P.ctx->launches;
        int its = 0;
        inner_solve(B, W, sets, bp64, bp32, act, tol_in, o.maxits - inner_total, o.poly_degree, its);
        check_batch_err(B);
        inner_total += its;
        OPEM_CUDA(cudaMemcpyAsync(B.act.p, act.data(), R, cudaMemcpyHostToDevice, B.s));
        refine_sys_kernel<<<dim3(gy, R), 256, 0, B.s>>>(n, W.d.p, nrm.p, B.act.p, x.p);
        ++P.ctx->launches;
        // FP64 residual r = b - A x
        to_il(B, x.p, n, x0_il.p);
        spmv_batch<double2, double>(B, P.d_K.p, P.d_Meps.p, P.has_tand ? P.d_Mtand.p : nullptr,
                                    P.has_sig ? P.d_Msig.p : nullptr, B.vc64.p, bp64, x0_il.p, y_il.p);
        resid_kernel<<<(unsigned)((nR + 255) / 256), 256, 0, B.s>>>(n, R, b.p, y_il.p, r64.p);
        ++P.ctx->launches;
        OPEM_CUDA(cudaMemcpyAsync(B.act.p, all1.data(), R, cudaMemcpyHostToDevice, B.s));
        nrm_sys_f64(B, r64.p, n, npart, nrm.p, B.act.p);
        OPEM_CUDA(cudaMemcpyAsync(rn.data(), nrm.p, R * sizeof(double), cudaMemcpyDeviceToHost, B.s));
        OPEM_CUDA(cudaStreamSynchronize(B.s));
        for (int r = 0; r < R; ++r) act[r] = (bn[r] > 0 && rn[r] > o.rtol * bn[r] && std::isfinite(rn[r])) ? 1 : 0;
    }
    out.inner_its = inner_total;
    out.outer = outer;
    out.worst = 0;
    out.converged = true;
    for (int r = 0; r < R; ++r) {
        double rel = bn[r] > 0 ? rn[r] / bn[r] : 0;
        out.worst = std::max(out.worst, rel);
        if (!(rel <= o.rtol)) out.converged = false;
    }
    // e = x + x0 (driven port values), H projection, overlaps
    finish_e_kernel<<<dim3(gy, R), 256, 0, B.s>>>(n, et, B.dsys.p, x.p);
    ++P.ctx->launches;
    W.V.release();
    W.Z.release();
    W.W.release();
    DBuf<double2> e_il(nR), h_il(nR), h_sm(nR);
    to_il(B, x.p, n, e_il.p);
    mass_cg_batch(B, e_il.p, h_il.p, o.h_rtol, o.h_maxits, out.h_its);
    to_sm(B, h_il.p, h_sm.p, n);
    DBuf<double2> ov((size_t)4 * R * N);
    for (int r = 0; r < R; ++r)
        for (int k = 0; k < N; ++k) {
            const double2* etk = et + (size_t)k * n;
            const double2* nxk = reinterpret_cast<const double2*>(P.d_nxe.p) + (size_t)k * n;
            double2* o4 = ov.p + 4 * (r * N + k);
            port_overlap(P, k, etk, x.p + (size_t)r * n, o4 + 0);
            port_overlap(P, k, etk, etk, o4 + 1);
            port_overlap(P, k, nxk, h_sm.p + (size_t)r * n, o4 + 2);
            port_overlap(P, k, nxk, nxk, o4 + 3);
        }
    std::vector<double2> hov((size_t)4 * R * N);
    OPEM_CUDA(cudaMemcpyAsync(hov.data(), ov.p, hov.size() * sizeof(double2), cudaMemcpyDeviceToHost, B.s));
    OPEM_CUDA(cudaStreamSynchronize(B.s));
    out.Cp.assign((size_t)R * N, 0.0);
    out.Cm.assign((size_t)R * N, 0.0);
    for (int r = 0; r < R; ++r) {
        double w = 2 * M_PI * systems[r].freq;
        for (int k = 0; k < N; ++k) {
            cd gam, Z, V;
            port_gamma_Z_V(P, k, systems[r].freq, gam, Z, V);
            cd y = gam / cd(0, w * port_mu_r(P, k) * MU0_M);
            const double2* o4 = &hov[4 * (r * N + k)];
            cd e0(o4[0].x, o4[0].y), e2(o4[1].x, o4[1].y);
            cd h0 = std::conj(y) * cd(o4[2].x, o4[2].y), h2 = std::norm(y) * cd(o4[3].x, o4[3].y);
            out.Cp[(size_t)r * N + k] = 0.5 * (e0 / e2 + h0 / h2);
            out.Cm[(size_t)r * N + k] = 0.5 * (e0 / e2 - h0 / h2);
        }
    }
}

// Sweep driver: frequencies are grouped so that a batch holds F frequencies
// x N driving sets <= RMAX systems.
void solve_sweep_mixed(Problem& P, int nfreq, const double* freqs, const opem_solver_opts& o,
                       std::vector<std::vector<cd>>& S, std::vector<opem_solve_stats>& st) {
    if (!P.extra.empty()) throw OpemError(OPEM_ERR_UNSUPPORTED, "ports with several modes run on the FP64 path");
    const int N = P.nports;
    int F = std::max(1, RMAX / std::max(1, N));
    if (o.poly_degree > 1) ensure_f32_operators(P, P.ctx->stream);
    // Keep a batch's per-system Krylov storage (V and Z, FP64, (m+1) vectors each,
    // plus the rotation buffer and vectors) within half of the free device memory.
    {
        size_t freeb = 0, totb = 0;
        OPEM_CUDA(cudaMemGetInfo(&freeb, &totb));
        const int m = std::max(2, o.restart), kd = std::max(0, std::min(o.deflate, m - 2));
        const double per_sys = (double)P.topo.n * sizeof(double2) * (2.0 * (m + 1) + (kd + 1) + 16) +
                               (double)P.topo.patch_dofs.size() * sizeof(float2) +
                               (double)P.topo.ne * P.topo.ld * (sizeof(float2) + sizeof(double2));
        const double fixed = (double)P.topo.patch_off.back() * (sizeof(float2) * N + sizeof(double2));
        const double avail = P.ws_cap > 0 ? std::min(0.5 * (double)freeb, (double)P.ws_cap) : 0.5 * (double)freeb;
        int Fm = (int)std::floor((avail - fixed) / (per_sys * std::max(1, N)));
        if (Fm < 1 && P.ws_cap > 0)   // the cap is advisory: fall back to the free memory for one point
            Fm = (int)std::floor((0.5 * (double)freeb - fixed) / (per_sys * std::max(1, N)));
        if (Fm < 1) throw OpemError(OPEM_ERR_NOMEM, "not enough device memory for one batched frequency point");
        F = std::min(F, Fm);
    }
    // ports driven by their own 2D mode have traces that change with frequency:
    // one frequency point per batch, traces refreshed before it
    if (has_fem2d_ports(P)) F = 1;
    int nb = (nfreq + F - 1) / F;
    F = (nfreq + nb - 1) / nb;   // balance the batches
    S.assign(nfreq, {});
    st.assign(nfreq, opem_solve_stats{});
    // batches are contiguous in frequency and span at most 15% of their centre
    // frequency, since a batch shares one block-Jacobi set per driving set
    std::vector<int> order(nfreq);
    for (int i = 0; i < nfreq; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return freqs[a] < freqs[b]; });
    std::vector<double> fs(nfreq);
    for (int i = 0; i < nfreq; ++i) fs[i] = freqs[order[i]];
    for (int f0 = 0; f0 < nfreq;) {
        int f1 = std::min(nfreq, f0 + F);
        while (f1 - f0 > 1 && (fs[f1 - 1] - fs[f0]) > 0.15 * 0.5 * (fs[f1 - 1] + fs[f0])) --f1;
        cudaEvent_t e0, e1;
        OPEM_CUDA(cudaEventCreate(&e0));
        OPEM_CUDA(cudaEventCreate(&e1));
        OPEM_CUDA(cudaEventRecord(e0, P.ctx->stream));
        std::vector<System> sys;
        for (int d = 0; d < N; ++d)
            for (int f = f0; f < f1; ++f) sys.push_back({fs[f], d});
        refresh_port_traces(P, fs[f0]);
        BatchOut bo;
        solve_batch(P, sys, o, bo);
        if (!bo.converged && o.restart < 1024) {
            // Restart escalation: vertex-patch block Jacobi is weak on under-resolved,
            // strongly indefinite meshes, where a short restart cycle stagnates (a 26k-DOF
            // ND3 guide with an eps_r 7.6 block: GMRES-DR(100, 30) stalls for 3000 steps,
            // (300, 60) converges in 222).  Retry the batch once with a 3x longer cycle
            // and twice the deflation space if its Krylov bases fit in half of the free memory.
            opem_solver_opts o2 = o;
            o2.restart = std::min(1024, 3 * o.restart);
            o2.deflate = std::min(2 * std::max(o.deflate, 1), o2.restart - 2);
            size_t freeb = 0, totb = 0;
            OPEM_CUDA(cudaMemGetInfo(&freeb, &totb));
            const double need = (double)sys.size() * P.topo.n * sizeof(double2) *
                                (2.0 * (o2.restart + 1) + (o2.deflate + 1) + 16);
            if (need < 0.5 * (double)freeb) {
                BatchOut bo2;
                solve_batch(P, sys, o2, bo2);
                if (bo2.converged || bo2.worst < bo.worst) bo = std::move(bo2);
            }
        }
        OPEM_CUDA(cudaEventRecord(e1, P.ctx->stream));
        OPEM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        OPEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        const int nf = f1 - f0;
        for (int f = f0; f < f1; ++f) {
            std::vector<cd> Cp((size_t)N * N), Cm((size_t)N * N), V(N), Z(N);
            for (int d = 0; d < N; ++d) {
                int r = d * nf + (f - f0);
                for (int k = 0; k < N; ++k) {
                    Cp[d * N + k] = bo.Cp[(size_t)r * N + k];
                    Cm[d * N + k] = bo.Cm[(size_t)r * N + k];
                }
            }
            for (int k = 0; k < N; ++k) {
                cd g;
                port_gamma_Z_V(P, k, fs[f], g, Z[k], V[k]);
            }
            S[order[f]] = s_matrix_solve(N, Cp, Cm, V, Z, o.force_reciprocal != 0);
            opem_solve_stats& s = st[order[f]];
            s.iterations = bo.inner_its;   // lockstep iterations of the batch
            s.outer = bo.outer;
            s.h_iterations = bo.h_its;
            s.converged = bo.converged ? 1 : 0;
            s.rnorm = bo.worst;
            s.seconds = ms * 1e-3 / nf;    // the batch's device time shared by its points
        }
        f0 = f1;
    }
}


// Times the batched-path kernels in isolation (CUDA events on the context
// stream): R systems near frequency f on driving set 0.  out[3k+0] = ms per
// launch, out[3k+1] = algorithmic bytes per launch, out[3k+2] = launches for
//   k = 0  FP32 block apply (patch_apply1_batch_kernel, one driving set of R systems)
//   k = 1  batched SpMV, FP32 operators and vectors (polynomial products)
//   k = 2  batched SpMV, FP64 operators, FP32 vectors
//   k = 3  batched SpMV, FP64 operators and vectors (Arnoldi products)
//   k = 4  patch sum of the block apply (patch_sum_all_kernel)
// The SpMV entries include the boundary-group kernels of the same product.
void profile_batch(Problem& P, double f, int R, int reps, double* out, int nout) {
    if (R < 1 || R > RMAX) throw OpemError(OPEM_ERR_ARG, "profile_batch: 1 <= nsys <= 32");
    Batch B(P);
    B.R = R;
    B.N = std::max(1, P.nports);
    B.r0.assign(B.N, 0);
    B.Rd.assign(B.N, 0);
    B.Rd[0] = R;
    std::vector<System> systems(R);
    for (int r = 0; r < R; ++r) systems[r] = {f * (1.0 + 0.002 * r), 0};
    B.sys = systems;
    std::vector<const BC5<float2>*> bp32;
    std::vector<const BC5<double2>*> bp64;
    setup_coefficients(B, systems, bp32, bp64);
    ensure_f32_operators(P, B.s);
    PatchSet32 set;
    build_patchset(B, f, 0, set);
    const int64_t n = B.n, nR = n * R, nnz = (int64_t)P.topo.cols.size();
    const int64_t sum_s = (int64_t)P.topo.patch_dofs.size();
    const double sum_s2 = (double)P.topo.patch_off.back();
    DBuf<float2> x32(nR), y32(nR), t((size_t)sum_s * R);
    DBuf<double2> x64(nR), y64(nR);
    OPEM_CUDA(cudaMemsetAsync(x32.p, 0x3c, x32.bytes(), B.s));   // finite, nonzero inputs
    OPEM_CUDA(cudaMemsetAsync(x64.p, 0x3c, x64.bytes(), B.s));
    OPEM_CUDA(cudaMemsetAsync(t.p, 0, t.bytes(), B.s));
    cudaEvent_t e0, e1;
    OPEM_CUDA(cudaEventCreate(&e0));
    OPEM_CUDA(cudaEventCreate(&e1));
    auto timeit = [&](auto&& launch) {
        for (int i = 0; i < 3; ++i) launch();
        OPEM_CUDA(cudaEventRecord(e0, B.s));
        for (int i = 0; i < reps; ++i) launch();
        OPEM_CUDA(cudaEventRecord(e1, B.s));
        OPEM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        OPEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return (double)ms / reps;
    };
    const double nops = 2.0 + (P.has_tand ? 1 : 0) + (P.has_sig ? 1 : 0);
    const double csr = (double)nnz * 4 + 4.0 * (n + 1) + 2.0 * n;   // cols, rowptr, masks
    // element-by-element product (ND2): element data, x read once, element outputs
    // written and read back, DOF -> element lists, y written
    const bool ebe = P.topo.ld == 20;
    const double ne_ld = (double)P.topo.ne * P.topo.ld;
    auto ebe_bytes = [&](double vb) {
        return (double)P.topo.ne * (sizeof(ElemGeo) + 32.0) + ne_ld * 4 + nR * vb + 2.0 * ne_ld * R * vb +
               ne_ld * 5 + 4.0 * (n + 1) + 2.0 * n + nR * vb;
    };
    out[0] = timeit([&] { patch_apply1_batch(P, B.s, set, x32.p, R, 0, R, t.p, B.err.p); });
    check_batch_err(B);
    out[1] = sum_s2 * 8 + (double)sum_s * (4 + 2.0 * R * 8) + P.npatch * 12.0;
    const double* Mt = P.has_tand ? P.d_Mtand.p : nullptr;
    const double* Ms = P.has_sig ? P.d_Msig.p : nullptr;
    out[3] = timeit([&] {
        spmv_batch<float2, float>(B, P.f_K.p, P.f_Meps.p, P.has_tand ? P.f_Mtand.p : nullptr,
                                  P.has_sig ? P.f_Msig.p : nullptr, B.vc32.p, bp32, x32.p, y32.p);
    });
    out[4] = ebe ? ebe_bytes(8) : csr + nnz * 4.0 * nops + 2.0 * nR * 8;
    out[6] = timeit([&] { spmv_batch<float2, double>(B, P.d_K.p, P.d_Meps.p, Mt, Ms, B.vc64.p, bp64, x32.p, y32.p); });
    out[7] = ebe ? ebe_bytes(8) : csr + nnz * 8.0 * nops + 2.0 * nR * 8;
    out[9] = timeit([&] { spmv_batch<double2, double>(B, P.d_K.p, P.d_Meps.p, Mt, Ms, B.vc64.p, bp64, x64.p, y64.p); });
    out[10] = ebe ? ebe_bytes(16) : csr + nnz * 8.0 * nops + 2.0 * nR * 16;
    out[12] = timeit([&] {
        patch_sum_all_kernel<<<(unsigned)((nR + 255) / 256), 256, 0, B.s>>>(
            n, P.d_d2p_ptr.p, P.d_d2p_idx.p, t.p, R, P.d_pec.p, P.d_portmask.p, B.dsys.p, y32.p);
        ++P.ctx->launches;
    });
    out[13] = (double)sum_s * (R * 8 + 4) + 4.0 * (n + 1) + 2.0 * n + nR * 8.0;
    for (int k = 0; k < 5; ++k) out[3 * k + 2] = reps;
    if (nout >= 21) {   // kernels 5 and 6: the FP32 FMA and the tensor-core block apply
        out[15] = timeit([&] { patch_apply1_batch(P, B.s, set, x32.p, R, 0, R, t.p, B.err.p, PA_FMA); });
        out[16] = out[1];
        out[17] = reps;
        out[18] = -1;
        out[19] = out[1];
        out[20] = 0;
        if (patch_tc_supported(P.ctx->device, P.topo.max_patch, R)) {
            out[18] = timeit([&] { patch_apply1_batch(P, B.s, set, x32.p, R, 0, R, t.p, B.err.p, PA_TENSOR); });
            out[20] = reps;
        }
        check_batch_err(B);
    }
    OPEM_CUDA(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}


// Block-apply check: the FP32 block set of driving set 0 at f and R systems of
// deterministic inputs in [-1, 1] (interleaved, R systems) go through the FMA
// kernel and the tensor-core kernel (when it applies); both results are
// compared with an FP64 host product of the same FP32 blocks and inputs.
// out[0] = max |tensor - ref| / max |ref| (-1 when the tensor-core kernel does
// not apply), out[1] = the same for the FMA kernel, out[2] = the kernel the
// solver uses for this problem and Rd (2 tensor core, 1 FMA), out[3] =
// max |tensor - fma| / max |ref|, out[4] = 1 if a bounded wait ran out.
void check_block_apply(Problem& P, double f, int R, int r0, int Rd, double* out) {
    if (R < 1 || R > RMAX || r0 < 0 || Rd < 1 || r0 + Rd > R) throw OpemError(OPEM_ERR_ARG, "check_block_apply: systems");
    Batch B(P);
    B.R = R;
    B.N = std::max(1, P.nports);
    B.err.alloc(1);
    B.err.zero(B.s);
    PatchSet32 set;
    build_patchset(B, f, 0, set);
    const int64_t n = B.n, nR = n * R;
    const int64_t sum_s = (int64_t)P.topo.patch_dofs.size();
    std::vector<float2> hx((size_t)nR);
    uint64_t st = 0x9E3779B97F4A7C15ull;
    auto rnd = [&] {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return (float)((double)(st >> 11) * (2.0 / 9007199254740992.0) - 1.0);
    };
    for (auto& v : hx) { v.x = rnd(); v.y = rnd(); }
    DBuf<float2> x(nR), t1((size_t)sum_s * Rd), t2((size_t)sum_s * Rd);
    x.upload(hx, B.s);
    t1.zero(B.s);
    t2.zero(B.s);
    const bool tc = patch_tc_supported(P.ctx->device, P.topo.max_patch, Rd);
    patch_apply1_batch(P, B.s, set, x.p, R, r0, Rd, t1.p, B.err.p, PA_FMA);
    if (tc) patch_apply1_batch(P, B.s, set, x.p, R, r0, Rd, t2.p, B.err.p, PA_TENSOR);
    std::vector<float2> h1((size_t)sum_s * Rd), h2((size_t)sum_s * Rd), hb((size_t)set.B.n);
    std::vector<int64_t> off((size_t)P.npatch);
    int herr = 0;
    OPEM_CUDA(cudaMemcpyAsync(h1.data(), t1.p, t1.bytes(), cudaMemcpyDeviceToHost, B.s));
    OPEM_CUDA(cudaMemcpyAsync(h2.data(), t2.p, t2.bytes(), cudaMemcpyDeviceToHost, B.s));
    OPEM_CUDA(cudaMemcpyAsync(hb.data(), set.B.p, set.B.bytes(), cudaMemcpyDeviceToHost, B.s));
    OPEM_CUDA(cudaMemcpyAsync(off.data(), set.off32.p, off.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, B.s));
    OPEM_CUDA(cudaMemcpyAsync(&herr, B.err.p, sizeof(int), cudaMemcpyDeviceToHost, B.s));
    OPEM_CUDA(cudaStreamSynchronize(B.s));
    const Topology& T = P.topo;
    double scale = 0, e1 = 0, e2 = 0, e12 = 0;
    for (int v = 0; v < P.npatch; ++v) {
        const int p0 = T.patch_ptr[v], sz = T.patch_ptr[v + 1] - p0;
        const float2* Bv = hb.data() + off[v];
        for (int a = 0; a < sz; ++a)
            for (int r = 0; r < Rd; ++r) {
                double re = 0, im = 0;
                for (int b = 0; b < sz; ++b) {
                    const float2 m = Bv[(size_t)b * sz + a];
                    const float2 xv = hx[(size_t)T.patch_dofs[p0 + b] * R + r0 + r];
                    re += (double)m.x * xv.x - (double)m.y * xv.y;
                    im += (double)m.x * xv.y + (double)m.y * xv.x;
                }
                const size_t k = (size_t)(p0 + a) * Rd + r;
                scale = std::max(scale, std::hypot(re, im));
                e1 = std::max(e1, std::hypot(h1[k].x - re, h1[k].y - im));
                if (tc) {
                    e2 = std::max(e2, std::hypot(h2[k].x - re, h2[k].y - im));
                    e12 = std::max(e12, std::hypot((double)h2[k].x - h1[k].x, (double)h2[k].y - h1[k].y));
                }
            }
    }
    if (!(scale > 0)) scale = 1;
    out[0] = tc ? e2 / scale : -1.0;
    out[1] = e1 / scale;
    out[2] = patch_apply_variant(P, B.s, set, x.p, R, r0, Rd, t1.p, B.err.p, PatchSel{}) == PA_TENSOR ? 2.0 : 1.0;
    out[3] = tc ? e12 / scale : -1.0;
    out[4] = herr ? 1.0 : 0.0;
}

// Device bytes a request needs on top of what the problem holds: its operators
// if it is not assembled yet (pattern and patch sizes estimated from the DOF
// count and order), and the solve workspace (the FP64 path's system matrix,
// blocks and Krylov basis, or the batched path's per-system bases, FP32
// blocks and element buffers for one batch).
double request_bytes_estimate(const Problem& P, int nfreq, const opem_solver_opts& o) {
    const double n = (double)P.topo.n;
    const int ld = P.topo.ld;
    const double nnz = P.assembled ? (double)P.topo.cols.size() : n * (ld <= 6 ? 16 : ld <= 20 ? 43 : 85);
    const double ss2 = (P.assembled && !P.topo.patch_off.empty()) ? (double)P.topo.patch_off.back()
                                                                   : n * (ld <= 6 ? 32 : ld <= 20 ? 240 : 1100);
    const double ss = P.assembled ? (double)P.topo.patch_dofs.size() : n * (ld <= 6 ? 5 : ld <= 20 ? 6 : 7);
    const double ne = (double)P.topo.ne;
    const int N = std::max(1, P.assembled ? P.nports : 2);
    double b = 0;
    if (!P.assembled) b += nnz * 60 + n * 64 + ne * (ld * 8.0 + 160) + ss * 12;
    const int m = std::max(2, o.restart), kd = std::max(0, std::min(o.deflate, m - 2));
    b += nnz * 16 + ss2 * 16;   // one system matrix and one FP64 block set (block inversion)
    if (o.precision == OPEM_PREC_MIXED) {
        const int F = std::max(1, std::min(nfreq, RMAX / N));
        const double R = (double)F * N;
        b += nnz * 16;   // FP32 operator copies
        b += R * (n * 16.0 * (2.0 * (m + 1) + (kd + 1) + 16) + ss * 8 + ne * ld * 24.0);
        b += ss2 * 8.0 * N;
    } else {
        b += n * 16.0 * (m + 1 + 24) + ss2 * 16;
    }
    return b;
}


// Failure-detection self-test: a bounded wait on an mbarrier phase that nothing
// completes (the barrier expects one arrival and gets none) gives up after
// `polls` polls and records the timeout in *status, as the batched block apply
// does when a bulk copy never lands.
__global__ void selftest_wait_kernel(int polls, int* __restrict__ status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    bool done = false;
    for (int it = 0; it < polls && !done; ++it) done = mbar_try_wait(&bar, 0);
    __syncthreads();
    if (!done && threadIdx.x == 0) atomicExch(status, 1);
}

__global__ void selftest_touch_kernel(int* __restrict__ v) { if (threadIdx.x == 0) v[1] = 7; }

int selftest_wait_timeout(Context& C, int polls) {
    DBuf<int> st(2);
    OPEM_CUDA(cudaMemsetAsync(st.p, 0, 2 * sizeof(int), C.stream));
    selftest_wait_kernel<<<1, 32, 0, C.stream>>>(polls, st.p);
    ++C.launches;
    OPEM_CUDA(cudaGetLastError());
    selftest_touch_kernel<<<1, 32, 0, C.stream>>>(st.p);   // the context still runs kernels
    ++C.launches;
    OPEM_CUDA(cudaGetLastError());
    int h[2] = {0, 0};
    OPEM_CUDA(cudaMemcpyAsync(h, st.p, sizeof(h), cudaMemcpyDeviceToHost, C.stream));
    OPEM_CUDA(cudaStreamSynchronize(C.stream));
    if (h[1] != 7) return OPEM_ERR_CUDA;
    return h[0] == 1 ? OPEM_ERR_TIMEOUT : OPEM_ERR_STATE;
}

}  // namespace opem
