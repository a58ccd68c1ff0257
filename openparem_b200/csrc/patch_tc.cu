// Batched vertex-patch block apply on the fifth-generation tensor cores.
//
// The batched sweep solver preconditions every (frequency, driving set) system
// of a driving set with the same overlapping vertex-patch block Jacobi: for each
// patch v, T_v = B_v X_v, where B_v is the inverted s x s complex block (FP32,
// stored column-major) and X_v holds the patch's s input rows for Rd systems.
// It replaces the direct PCLU/PCCHOLESKY preconditioner of the reference's
// KSPGMRES solve (src/OpenParEM3D/solveComplexLinearSystem.c:153-161).
//
// Real form.  Column b of B_v is stored as 2s floats (re, im interleaved), so
// read as a real matrix C (2s x s) it has rows C[2a] = Re B[a,:], C[2a+1] =
// Im B[a,:].  With the inputs as one real K x N matrix [Xr | Xi] (K = s, N = 2RP,
// RP = Rd rounded up to 16 or 32), P = C [Xr | Xi] gives
//   Re T[a][r] = P[2a][r] - P[2a+1][RP + r],  Im T[a][r] = P[2a][RP + r] + P[2a+1][r].
// P is one tcgen05.mma.kind::tf32 product per 128-row tile (M = 128) and K step
// of 8.  TF32 keeps 10 mantissa bits, too few for these inverted blocks (block
// Jacobi with TF32-rounded blocks took the config-2 sweep from 66-91 Krylov
// steps per batch to 91-104, and one batch to the 3000-step limit), so both
// operands are split, hi = the value with the low 13 mantissa bits cleared (an
// exact TF32 number) and lo = value - hi (exact in FP32); the dropped lo(C) lo(X)
// term is 2^-22 relative.  The split inputs sit side by side as one K x 2N
// operand [hi(X) | lo(X)], so two products per K step, hi(C) [hi(X) | lo(X)]
// (N = 2N columns) and lo(C) hi(X) accumulated onto its first N columns, give
// P = D[:, :N] + D[:, N:] in FP32 in tensor memory.
//
// One persistent CTA per SM walks its share of the selected patches (selection
// entries blockIdx.x, + gridDim.x, ...)
// with warp-specialised roles connected by mbarriers:
//   warp 0          TMA producer (one thread): streams each patch's block in
//                   panels of KC = 16 columns (contiguous in HBM), one bulk copy
//                   (cp.async.bulk, the TMA engine) per panel into an NS-stage
//                   ring.  Bulk copies, not tensor-map boxes: with the panels
//                   seen as a 2D map of 128-byte rows, boxes of 16 rows held one
//                   CTA per SM to 2.9 TB/s in a streaming probe on B200, while one
//                   bulk copy per 12.8 KB panel reached 6.0 TB/s;
//   warp 1          MMA issuer (one thread): tcgen05.mma with A (the split block
//                   panel) in tensor memory and B (the split inputs) in shared
//                   memory, tcgen05.commit to release each stage;
//   warps 2-3, 20-23 input stager: a warp gathers chunks of the patch's X rows
//                   (one coalesced index load, then per row one coalesced load of
//                   its Rd systems, RP lanes per row, 16 loads in flight per
//                   lane), splits them and writes them in the canonical K-major
//                   (no swizzle) layout, XB buffers;
//   warps 4-7, 8-11 converter, two warpgroups taking alternate panels: reads a
//                   ring stage (thread = one of the 128 lanes of an M tile,
//                   consecutive rows, conflict-free), splits each entry into
//                   hi/lo and stores them into tensor memory with tcgen05.st
//                   (AS staging slots);
//   warps 12-19     epilogue, warpgroup E draining M tile E of each patch (both
//                   tiles at once, so the accumulators free up sooner): tcgen05.ld
//                   (AB buffers), the re/im recombination of neighbouring rows by
//                   one shuffle, and the stores of T.
// Every wait is bounded: a wait that runs out sets *err and a shared abort flag
// that stops every role; the producer then waits (bounded) for its copies in
// flight, the MMA thread for its products, and the CTA frees its tensor memory.
// The bulk copies read only this GPU's own block array; no load multicasts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "engine.h"
#include "patch_tc.h"

namespace opem {
namespace tc {

constexpr int KC = 16;        // block columns per panel
constexpr int AS = 4;         // tensor-memory staging slots for the split panel
constexpr int AB_MAX = 2;     // accumulator buffers (two for up to 16 systems, one above)
constexpr int XB = 3;         // split-input buffers
constexpr int NS_MAX = 8;     // ring stages
constexpr int THREADS = 768;
constexpr int W_TMA = 0, W_MMA = 1, W_CV = 4, W_EP = 12, W_X2 = 20;
constexpr int X_WARPS = 6, X_THREADS = 192, CV_WARPS = 4, EP_THREADS = 256;
constexpr int X_ITERS = 16;   // row loads in flight per stager lane (a chunk is 16 x (32 / RP) rows)
constexpr uint32_t POLL_LIMIT = 1u << 22;

struct Bars {
    uint64_t full[NS_MAX], empty[NS_MAX];
    uint64_t tfull[AS], tempty[AS];
    uint64_t afull[AB_MAX], aempty[AB_MAX];
    uint64_t xfull[XB], xempty[XB];
    uint64_t drain;
    uint32_t tmem_base;
    int abort;
};

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of parity `parity`; gives up (setting the abort
// flag and *err) after POLL_LIMIT polls or when another role has aborted.
__device__ __forceinline__ bool bar_wait(Bars& S, uint64_t* b, uint32_t parity, int* err) {
    for (uint32_t it = 0; it < POLL_LIMIT; ++it) {
        if (bar_try(b, parity)) return true;
        if (*(volatile int*)&S.abort) return false;
    }
    *(volatile int*)&S.abort = 1;
    atomicExch(err, 1);
    return false;
}
// The same, decided for the whole warp: warps that go on to warp-collective
// tensor-memory instructions (.sync.aligned) must take one branch together.
__device__ __forceinline__ bool bar_wait_warp(Bars& S, uint64_t* b, uint32_t parity, int* err) {
    const bool ok = bar_wait(S, b, parity, err);
    return __all_sync(0xffffffffu, ok);
}
// plain bounded wait (drains at exit): no abort test
__device__ __forceinline__ void bar_wait_drain(uint64_t* b, uint32_t parity) {
    for (uint32_t it = 0; it < POLL_LIMIT; ++it)
        if (bar_try(b, parity)) return;
}

// global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16)
// completing on mbarrier b
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     su32(dst)),
                 "l"(src), "r"(bytes), "r"(su32(b))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
          "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// D (tensor memory) (+)= A (tensor memory, 128 x 8, K-major) * B (shared memory descriptor)
__device__ __forceinline__ void umma_tf32_ts(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(b))
                 : "memory");
}

// Shared-memory matrix descriptor: canonical K-major layout without swizzle
// (8-row x 16-byte core matrices of 128 contiguous bytes), LBO = byte stride
// between core matrices along K, SBO = byte stride between 8-row groups.
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version of this architecture; base offset 0, no swizzle
    return d;
}
// Instruction descriptor: D FP32, A and B TF32, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void split_tf32(float a, uint32_t& hi, uint32_t& lo) {
    const uint32_t h = __float_as_uint(a) & 0xFFFFE000u;
    hi = h;
    lo = __float_as_uint(a - __uint_as_float(h));
}

struct Args {
    const float2* B;        // FP32 blocks (column-major, block v at off32[v])
    int nsel, MT, NS, slot_bytes, xbytes;
    const int32_t* plist;   // the patches to apply (nsel of them), or all patches when null
    int ldt;                // row stride of T in systems (>= Rd)
    uint32_t tmem_cols;
    const int32_t* pptr;
    const int32_t* pdofs;
    const int64_t* off32;
    const float2* x;
    int R, r0, Rd;
    float* t;
    int* err;
};

// Bytes of one split-input buffer [hi | lo] for patches of up to smax DOFs: K
// rows rounded up to 8, 2 x 2 RP columns of 4 bytes.
inline int xbuf_bytes(int smax, int RP) { return ((smax + 7) / 8 * 8) * (4 * RP) * 4; }
// accumulator buffers for RP (tensor memory: 4 x 2 x 32 staging + AB x 2 x 4RP columns <= 512)
__host__ __device__ constexpr int acc_buffers(int RP) { return RP <= 16 ? 2 : 1; }

template <int RP>
__global__ void __launch_bounds__(THREADS, 1) patch_apply_tc_kernel(Args g) {
    constexpr int NA = 2 * RP;   // columns of [Xr | Xi] and of P
    constexpr int NB = 2 * NA;   // columns of the split inputs [hi | lo] and of the accumulators
    constexpr int AB = acc_buffers(RP);
    __shared__ __align__(8) Bars S;
    extern __shared__ __align__(1024) unsigned char dsm_raw[];
    // the launch adds 1024 bytes so the ring can start on a 1024-byte boundary
    unsigned char* dsm = dsm_raw + ((1024u - (su32(dsm_raw) & 1023u)) & 1023u);
    unsigned char* ring = dsm;
    unsigned char* xbuf = dsm + (size_t)g.NS * g.slot_bytes;   // XB x [hi | lo]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int MT = g.MT;
    const uint32_t colD0 = (uint32_t)(AS * MT * 2 * KC);

    if (threadIdx.x == 0) {
        for (int k = 0; k < g.NS; ++k) {
            bar_init(&S.full[k], 1);
            bar_init(&S.empty[k], CV_WARPS);
        }
        for (int k = 0; k < AS; ++k) {
            bar_init(&S.tfull[k], CV_WARPS);
            bar_init(&S.tempty[k], 1);
        }
        for (int k = 0; k < AB; ++k) {
            bar_init(&S.afull[k], 1);
            bar_init(&S.aempty[k], EP_THREADS);
        }
        for (int k = 0; k < XB; ++k) {
            bar_init(&S.xfull[k], X_THREADS);
            bar_init(&S.xempty[k], 1);
        }
        bar_init(&S.drain, 1);
        S.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&S.tmem_base)),
                     "r"(g.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = S.tmem_base;

    if (warp == W_TMA) {
        if (lane == 0) {
            int gp = 0;
            bool ok = true;
            for (int k = blockIdx.x; k < g.nsel && ok; k += gridDim.x) {
                const int v = g.plist ? g.plist[k] : k;
                const int s = g.pptr[v + 1] - g.pptr[v];
                const int npan = (s + KC - 1) / KC;
                const float2* Bv = g.B + g.off32[v];
                for (int p = 0; p < npan; ++p, ++gp) {
                    const int slot = gp % g.NS;
                    if (gp >= g.NS && !bar_wait(S, &S.empty[slot], (uint32_t)(((gp / g.NS) + 1) & 1), g.err)) {
                        ok = false;
                        break;
                    }
                    // the panel's columns are contiguous; the size is rounded up to 16
                    // bytes (at most 8 bytes past the block: the array ends with slack)
                    const int b0 = p * KC, pw = min(KC, s - b0);
                    const uint32_t bytes = (uint32_t)(((int64_t)pw * s * 8 + 15) & ~15ll);
                    bar_expect_tx(&S.full[slot], bytes);
                    bulk_g2s(ring + (size_t)slot * g.slot_bytes, Bv + (int64_t)b0 * s, bytes, &S.full[slot]);
                }
            }
            // every copy issued has landed before the CTA may exit (bounded)
            for (int q = max(0, gp - g.NS); q < gp; ++q) bar_wait_drain(&S.full[q % g.NS], (uint32_t)((q / g.NS) & 1));
        }
    } else if (warp == W_MMA) {
        if (lane == 0) {
            constexpr uint32_t IDESC_W = idesc_tf32(NB), IDESC_N = idesc_tf32(NA);
            constexpr uint32_t LBO = (uint32_t)(NB / 8) * 128u, SBO = 128u;
            constexpr uint64_t KSTEP = (uint64_t)(8 * NB * 4 / 16);   // 8 K rows, in 16-byte descriptor units
            int gp = 0, i = 0;
            bool ok = true;
            for (int k = blockIdx.x; k < g.nsel && ok; k += gridDim.x, ++i) {
                const int v = g.plist ? g.plist[k] : k;
                const int s = g.pptr[v + 1] - g.pptr[v];
                const int npan = (s + KC - 1) / KC, mtv = (2 * s + 127) / 128;
                const int ab = i % AB, xb = i % XB;
                if (!bar_wait(S, &S.xfull[xb], (uint32_t)((i / XB) & 1), g.err)) break;
                if (i >= AB && !bar_wait(S, &S.aempty[ab], (uint32_t)(((i / AB) + 1) & 1), g.err)) break;
                tc_fence_after();
                const uint64_t dx0 = desc_kmajor(su32(xbuf + (size_t)xb * g.xbytes), LBO, SBO);
                const uint32_t d0 = tbase + colD0 + (uint32_t)(ab * MT * NB);
                for (int p = 0; p < npan; ++p, ++gp) {
                    const int ts = gp % AS;
                    if (!bar_wait(S, &S.tfull[ts], (uint32_t)((gp / AS) & 1), g.err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const int pw = min(KC, s - p * KC), nks = (pw + 7) / 8;
                    const uint64_t kb = (uint64_t)(2 * p) * KSTEP;   // K offset of the panel
                    const uint32_t a0 = tbase + (uint32_t)(ts * MT * 2 * KC);
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt) {
                        if (mt >= mtv) break;
                        const uint32_t d = d0 + (uint32_t)(mt * NB);
                        const uint32_t ahi = a0 + (uint32_t)(mt * 2 * KC);
#pragma unroll
                        for (int ks = 0; ks < KC / 8; ++ks) {
                            if (ks >= nks) break;
                            const uint64_t bx = dx0 + kb + ks * KSTEP;
                            const uint32_t a = ahi + 8u * ks;
                            umma_tf32_ts(d, a, bx, IDESC_W, (p > 0 || ks > 0) ? 1u : 0u);   // hi(C) [hi(X) | lo(X)]
                            umma_tf32_ts(d, a + KC, bx, IDESC_N, 1u);                     // + lo(C) hi(X)
                        }
                    }
                    umma_commit(&S.tempty[ts]);
                }
                if (!ok) break;
                umma_commit(&S.afull[ab]);
                umma_commit(&S.xempty[xb]);
            }
            // no product in flight when the CTA frees its tensor memory (bounded)
            umma_commit(&S.drain);
            bar_wait_drain(&S.drain, 0);
        }
    } else if (warp < W_CV || warp >= W_X2) {
        // input stager: X rows of the patch, split, canonical K-major layout
        const int sw = warp < W_CV ? warp - 2 : warp - W_X2 + 2;
        int i = 0;
        for (int k = blockIdx.x; k < g.nsel; k += gridDim.x, ++i) {
            const int v = g.plist ? g.plist[k] : k;
            const int xb = i % XB;
            if (i >= XB && !bar_wait(S, &S.xempty[xb], (uint32_t)(((i / XB) + 1) & 1), g.err)) break;
            const int p0 = g.pptr[v], s = g.pptr[v + 1] - p0, SP = (s + 7) / 8 * 8;
            float* xs = reinterpret_cast<float*>(xbuf + (size_t)xb * g.xbytes);
            constexpr int RPW = 32 / RP, CH = X_ITERS * RPW;   // rows per warp load, rows per chunk
            const int r = lane % RP, hg = lane / RP;
            for (int b0 = sw * CH; b0 < SP; b0 += X_WARPS * CH) {
                int mydof = -1;
                if (lane < CH && b0 + lane < s) mydof = g.pdofs[p0 + b0 + lane];
                float2 xv[X_ITERS];
#pragma unroll
                for (int j = 0; j < X_ITERS; ++j) {
                    const int dj = __shfl_sync(0xffffffffu, mydof, j * RPW + hg);
                    xv[j] = (dj >= 0 && r < g.Rd) ? g.x[(int64_t)dj * g.R + g.r0 + r] : make_float2(0.f, 0.f);
                }
#pragma unroll
                for (int j = 0; j < X_ITERS; ++j) {
                    const int b = b0 + j * RPW + hg;
                    if (b >= SP) break;
                    uint32_t h0, l0, h1, l1;
                    split_tf32(xv[j].x, h0, l0);
                    split_tf32(xv[j].y, h1, l1);
                    // element (k = b, n) of a K-major operand: core matrix (k / 4, n / 8);
                    // columns: hi re r, hi im RP + r, lo re NA + r, lo im NA + RP + r
                    const int base = (b >> 2) * (NB / 8) * 32 + (b & 3);   // in floats
                    auto at = [&](int n) { return base + (n >> 3) * 32 + (n & 7) * 4; };
                    xs[at(r)] = __uint_as_float(h0);
                    xs[at(RP + r)] = __uint_as_float(h1);
                    xs[at(NA + r)] = __uint_as_float(l0);
                    xs[at(NA + RP + r)] = __uint_as_float(l1);
                }
            }
            fence_async_smem();
            bar_arrive(&S.xfull[xb]);
        }
    } else if (warp < W_EP) {
        // converter group G takes panels gp with gp % 2 == G: ring stage -> split
        // -> tensor memory (lane quarter q)
        const int G = (warp - W_CV) >> 2, q = warp & 3, t = q * 32 + lane;
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        int gp = 0;
        bool ok = true;
        for (int k = blockIdx.x; k < g.nsel && ok; k += gridDim.x) {
            const int v = g.plist ? g.plist[k] : k;
            const int s = g.pptr[v + 1] - g.pptr[v];
            const int npan = (s + KC - 1) / KC, mtv = (2 * s + 127) / 128;
            for (int p = 0; p < npan; ++p, ++gp) {
                if ((gp & 1) != G) continue;
                const int slot = gp % g.NS, ts = gp % AS;
                if (!bar_wait_warp(S, &S.full[slot], (uint32_t)((gp / g.NS) & 1), g.err)) { ok = false; break; }
                if (gp >= AS && !bar_wait_warp(S, &S.tempty[ts], (uint32_t)(((gp / AS) + 1) & 1), g.err)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const float* panel = reinterpret_cast<const float*>(ring + (size_t)slot * g.slot_bytes);
                const int pw = min(KC, s - p * KC);
                for (int mt = 0; mt < mtv; ++mt) {
                    const int m = mt * 128 + t;
                    const bool valid = m < 2 * s;
                    const float* col = panel + m;
                    uint32_t hi[KC], lo[KC];
#pragma unroll
                    for (int kk = 0; kk < KC; ++kk) {
                        const float a = (valid && kk < pw) ? col[kk * 2 * s] : 0.f;
                        split_tf32(a, hi[kk], lo[kk]);
                    }
                    const uint32_t c = (uint32_t)((ts * MT + mt) * 2 * KC);
                    tmem_st16(tbase + lane_off + c, hi);
                    tmem_st16(tbase + lane_off + c + KC, lo);
                }
                tmem_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    bar_arrive(&S.tfull[ts]);
                    bar_arrive(&S.empty[slot]);
                }
            }
        }
    } else {
        // epilogue group E drains M tile E of each patch (lane quarter q)
        const int E = (warp - W_EP) >> 2, q = warp & 3;
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        int i = 0;
        for (int k = blockIdx.x; k < g.nsel; k += gridDim.x, ++i) {
            const int v = g.plist ? g.plist[k] : k;
            const int ab = i % AB;
            if (!bar_wait_warp(S, &S.afull[ab], (uint32_t)((i / AB) & 1), g.err)) break;
            tc_fence_after();
            const int p0 = g.pptr[v], s = g.pptr[v + 1] - p0, mtv = (2 * s + 127) / 128;
            if (E >= mtv) {
                tc_fence_before();
                bar_arrive(&S.aempty[ab]);
                continue;
            }
            const int mt = E;
            const uint32_t col = colD0 + (uint32_t)((ab * MT + mt) * NB);
            float val[RP];
#pragma unroll
            for (int h = 0; h < NA / 32; ++h) {
                uint32_t d[32], e[32];
                tmem_ld32(tbase + lane_off + col + 32u * h, d);
                tmem_ld32(tbase + lane_off + col + NA + 32u * h, e);
                tmem_wait_ld();
                // this lane holds row m of P = D[:, :NA] + D[:, NA:]: columns [0, RP)
                // = C Xr, [RP, 2RP) = C Xi; the even row of a pair needs the odd
                // row's C Xi, the odd row the even row's C Xi (one xor shuffle)
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int n = 32 * h + c;
                    const float pn = __uint_as_float(d[c]) + __uint_as_float(e[c]);
                    if (n >= RP) {
                        const float other = __shfl_xor_sync(0xffffffffu, pn, 1);
                        const int r = n - RP;
                        if (lane & 1) val[r] += other;    // Im T = P[2a][RP+r] + P[2a+1][r]
                        else val[r] -= other;             // Re T = P[2a][r] - P[2a+1][RP+r]
                    } else {
                        val[n] = pn;
                    }
                }
            }
            // the accumulator tile is read: release it before the stores
            tc_fence_before();
            bar_arrive(&S.aempty[ab]);
            const int m = mt * 128 + q * 32 + lane;
            if (m < 2 * s) {
                float* out = g.t + ((int64_t)(p0 + (m >> 1)) * g.ldt) * 2 + (lane & 1);
#pragma unroll
                for (int r = 0; r < RP; ++r)
                    if (r < g.Rd) out[2 * r] = val[r];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(g.tmem_cols) : "memory");
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
}  // namespace tc

bool patch_tc_supported(int device, int smax, int Rd) {
    if (smax < 1 || smax > 128 || Rd < 1 || Rd > 32) return false;
    int major = 0, minor = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device) != cudaSuccess) return false;
    return major == 10 && minor == 0;
}

void patch_apply1_batch_tc(const PatchTcLaunch& L, cudaStream_t stream) {
    using namespace tc;
    if (!patch_tc_supported(L.device, L.smax, L.Rd)) throw OpemError(OPEM_ERR_UNSUPPORTED, "tensor-core block apply");
    // every block and every 16-column panel starts 16-byte aligned (off32 a
    // multiple of 16 elements), and the array ends with 16 elements of slack
    if (L.total_f2 % 16 != 0 || (reinterpret_cast<uintptr_t>(L.B) & 15))
        throw OpemError(OPEM_ERR_ARG, "block array not 16-byte aligned with slack");
    const int RP = L.Rd <= 16 ? 16 : 32;
    const int MT = (2 * L.smax + 127) / 128;
    Args g;
    g.nsel = L.plist ? L.nlist : L.npatch;
    g.plist = L.plist;
    g.B = L.B;
    g.ldt = L.ldt > 0 ? L.ldt : L.Rd;
    g.MT = MT;
    g.slot_bytes = (KC * L.smax * 8 + 127) / 128 * 128;
    g.xbytes = xbuf_bytes(L.smax, RP);
    int optin = 0;
    OPEM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, L.device));
    const int dyn_max = optin - 2048;   // static barriers and the alignment slack stay below 2 KB
    const int budget = dyn_max - 1024 - XB * g.xbytes;
    g.NS = std::min(NS_MAX, budget / g.slot_bytes);
    if (g.NS < 2) throw OpemError(OPEM_ERR_UNSUPPORTED, "tensor-core block apply: shared memory");
    uint32_t cols = (uint32_t)(AS * MT * 2 * KC + acc_buffers(RP) * MT * 4 * RP), c = 32;
    while (c < cols) c <<= 1;
    g.tmem_cols = c;
    if (c > 512) throw OpemError(OPEM_ERR_UNSUPPORTED, "tensor-core block apply: tensor memory");
    g.pptr = L.pptr;
    g.pdofs = L.pdofs;
    g.off32 = L.off32;
    g.x = L.x;
    g.R = L.R;
    g.r0 = L.r0;
    g.Rd = L.Rd;
    g.t = reinterpret_cast<float*>(L.t);
    g.err = L.err;
    const size_t smem = 1024 + (size_t)g.NS * g.slot_bytes + (size_t)XB * g.xbytes;
    if (g.nsel < 1) return;
    const int grid = std::max(1, std::min(g.nsel, L.sm_count));
    // the maximum dynamic shared memory is a process-wide function attribute:
    // always the same device-wide value, so concurrent launches cannot lower it
    if (RP == 16) {
        OPEM_CUDA(cudaFuncSetAttribute(patch_apply_tc_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max));
        patch_apply_tc_kernel<16><<<grid, THREADS, smem, stream>>>(g);
    } else {
        OPEM_CUDA(cudaFuncSetAttribute(patch_apply_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max));
        patch_apply_tc_kernel<32><<<grid, THREADS, smem, stream>>>(g);
    }
    OPEM_CUDA(cudaGetLastError());
}

}  // namespace opem
