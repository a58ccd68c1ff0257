// Tensor-core (tcgen05) batched vertex-patch block apply (internal).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace opem {

// One launch of T = B_v X_v over every patch v for the Rd systems [r0, r0+Rd)
// of the interleaved inputs x (element (dof, r) at dof*R + r).  B holds the FP32
// column-major blocks (block v at off32[v] float2 elements, a multiple of 16;
// total_f2 elements in all, a multiple of 16).  T is written per patch entry:
// t[(pptr[v] + a) * ldt + r] (ldt = Rd when 0).  With plist, only the nlist
// patches plist[0..nlist) are applied.
struct PatchTcLaunch {
    int device = 0, sm_count = 148;
    int npatch = 0, smax = 0;
    const int32_t* pptr = nullptr;
    const int32_t* pdofs = nullptr;
    const int64_t* off32 = nullptr;
    const float2* B = nullptr;
    int64_t total_f2 = 0;
    const float2* x = nullptr;
    int R = 0, r0 = 0, Rd = 0;
    float2* t = nullptr;
    int ldt = 0;
    const int32_t* plist = nullptr;
    int nlist = 0;
    int* err = nullptr;   // set to 1 when a bounded wait ran out
};

// Whether the tensor-core kernel handles this case: a compute capability 10.0
// device, patches of at most 128 DOFs (two 128-row tiles of the real form) and
// at most 32 systems per launch.
bool patch_tc_supported(int device, int smax, int Rd);

// Launches the kernel on `stream`; throws OpemError when unsupported.
void patch_apply1_batch_tc(const PatchTcLaunch& L, cudaStream_t stream);

}  // namespace opem
