// Device-side helpers and kernel launcher declarations (internal).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace opem {

// ---- complex helpers (double2 / float2 = re, im) --------------------------
__host__ __device__ inline double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ inline double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ inline double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ inline double2 cconjmul(double2 a, double2 b) { return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }  // conj(a)*b
__host__ __device__ inline float2 cmulf(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ inline float2 cconjmulf(float2 a, float2 b) { return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }

// Per-element geometric factors written by the geometry kernel:
// gK[6] = (J^T J)_s / |det J|, gM[6] = |det J| (J^-1 J^-T)_s, sgn = sign(det J)
struct ElemGeo { double gK[6]; double gM[6]; double sgn; double pad; };

// Coefficients of one boundary group applied to one system:
// A += c_cc R_cc + c_eps R_eps + c_tand R_tand + c_sig R_sig + c_one R_one
struct BCoef { double2 c_cc, c_eps, c_tand, c_sig, c_one; };

// Sizes handed to the combine / SpMV kernels for the batched mixed path.
struct VolCoef { double2 c_eps, c_tand, c_sig; };   // A = K + c_eps Meps + c_tand Mtand + c_sig Msig

}  // namespace opem
