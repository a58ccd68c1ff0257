// Krylov solvers and the vertex-patch block-Jacobi preconditioner (FP64 path).
//
// Replaces the PETSc KSPGMRES solve of solveComplexLinearSystem
// (src/OpenParEM3D/solveComplexLinearSystem.c:100-209) and the mass-matrix
// solve of solveHfield (:235-315).  The reference preconditions with a sparse
// direct factorisation (PCCHOLESKY/PCLU via MUMPS); here GMRES(m) is right-
// preconditioned by overlapping vertex-patch block Jacobi (additive Schwarz
// on the dofs of each vertex star), which keeps the discrete-gradient kernel
// of curl-curl local to each block.  Orthogonalisation is classical Gram-
// Schmidt with one reorthogonalisation (CGS2).  The small (m+1) x m Hessenberg
// least-squares problem (Givens rotations, back substitution) runs on the
// device in FP64 (lsq.cu), the host reading one residual estimate per Arnoldi
// step; the harmonic Ritz eigenproblem of each restart runs on the host in
// FP64 (dense.cpp).
#include <algorithm>
#include <cmath>

#include "dense.h"
#include "engine.h"
#include "lsq.h"

namespace opem {

// ---------------------------------------------------------------------------
// SpMV
// ---------------------------------------------------------------------------
template <int TPR>
__global__ void spmv_c64_kernel(int64_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                                const double2* __restrict__ A, const double2* __restrict__ x, double2* __restrict__ y,
                                const uint8_t* __restrict__ zero_rows, double2 scale) {
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t r = t / TPR;
    int lane = (int)(t % TPR);
    double re = 0, im = 0;
    if (r < n) {
        const int32_t k1 = __ldg(rowptr + r + 1);
        int32_t k = __ldg(rowptr + r) + lane;
        // three slots of the row per lane in flight: column indices, then values and
        // gathers, then the products (rows of up to 3*TPR nonzeros take one round)
        for (; k < k1; k += 3 * TPR) {
            int32_t c[3];
            double2 a[3], v[3];
#pragma unroll
            for (int u = 0; u < 3; ++u) c[u] = (k + u * TPR < k1) ? __ldg(cols + k + u * TPR) : -1;
#pragma unroll
            for (int u = 0; u < 3; ++u)
                if (c[u] >= 0) { a[u] = __ldg(A + k + u * TPR); v[u] = __ldg(x + c[u]); }
#pragma unroll
            for (int u = 0; u < 3; ++u)
                if (c[u] >= 0) {
                    re += a[u].x * v[u].x - a[u].y * v[u].y;
                    im += a[u].x * v[u].y + a[u].y * v[u].x;
                }
        }
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o, TPR);
        im += __shfl_down_sync(0xffffffffu, im, o, TPR);
    }
    if (r < n && lane == 0) {
        if (zero_rows && zero_rows[r]) y[r] = make_double2(0, 0);
        else y[r] = make_double2(scale.x * re - scale.y * im, scale.x * im + scale.y * re);
    }
}

template <int TPR>
__global__ void spmv_rc64_kernel(int64_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                                 const double* __restrict__ A, const double2* __restrict__ x, double2* __restrict__ y,
                                 double2 scale) {
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t r = t / TPR;
    int lane = (int)(t % TPR);
    double re = 0, im = 0;
    if (r < n) {
        const int32_t k1 = __ldg(rowptr + r + 1);
        int32_t k = __ldg(rowptr + r) + lane;
        for (; k < k1; k += 3 * TPR) {   // three slots per lane in flight, as in spmv_c64_kernel
            int32_t c[3];
            double a[3];
            double2 v[3];
#pragma unroll
            for (int u = 0; u < 3; ++u) c[u] = (k + u * TPR < k1) ? __ldg(cols + k + u * TPR) : -1;
#pragma unroll
            for (int u = 0; u < 3; ++u)
                if (c[u] >= 0) { a[u] = __ldg(A + k + u * TPR); v[u] = __ldg(x + c[u]); }
#pragma unroll
            for (int u = 0; u < 3; ++u)
                if (c[u] >= 0) { re += a[u] * v[u].x; im += a[u] * v[u].y; }
        }
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o, TPR);
        im += __shfl_down_sync(0xffffffffu, im, o, TPR);
    }
    if (r < n && lane == 0) y[r] = make_double2(scale.x * re - scale.y * im, scale.x * im + scale.y * re);
}

static int tpr_for(const Problem& P) {
    double avg = (double)P.topo.cols.size() / std::max<int64_t>(1, P.topo.n);
    return avg > 48 ? 32 : (avg > 20 ? 16 : 8);
}

void spmv_complex(Problem& P, const double2* A, const double2* x, double2* y, const uint8_t* zero_rows) {
    int64_t n = P.topo.n;
    int tpr = tpr_for(P);
    int64_t threads = n * tpr;
    unsigned grid = (unsigned)((threads + 255) / 256);
    double2 one = make_double2(1, 0);
    cudaStream_t s = P.ctx->stream;
    if (tpr == 32) spmv_c64_kernel<32><<<grid, 256, 0, s>>>(n, P.d_rowptr.p, P.d_cols.p, A, x, y, zero_rows, one);
    else if (tpr == 16) spmv_c64_kernel<16><<<grid, 256, 0, s>>>(n, P.d_rowptr.p, P.d_cols.p, A, x, y, zero_rows, one);
    else spmv_c64_kernel<8><<<grid, 256, 0, s>>>(n, P.d_rowptr.p, P.d_cols.p, A, x, y, zero_rows, one);
    ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
}

void spmv_real_complex(Problem& P, const double* vals, const double2* x, double2* y, double sre, double sim) {
    int64_t n = P.topo.n;
    int tpr = tpr_for(P);
    unsigned grid = (unsigned)((n * tpr + 255) / 256);
    double2 sc = make_double2(sre, sim);
    cudaStream_t s = P.ctx->stream;
    if (tpr == 32) spmv_rc64_kernel<32><<<grid, 256, 0, s>>>(n, P.d_rowptr.p, P.d_cols.p, vals, x, y, sc);
    else if (tpr == 16) spmv_rc64_kernel<16><<<grid, 256, 0, s>>>(n, P.d_rowptr.p, P.d_cols.p, vals, x, y, sc);
    else spmv_rc64_kernel<8><<<grid, 256, 0, s>>>(n, P.d_rowptr.p, P.d_cols.p, vals, x, y, sc);
    ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// reductions (deterministic: fixed partition, fixed tree order)
// ---------------------------------------------------------------------------
constexpr int RED_BLOCKS = 512;

__device__ inline void block_sum2(double& a, double& b) {
    __shared__ double sa[32], sb[32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    int nw = blockDim.x >> 5;
    a = (threadIdx.x < nw) ? sa[threadIdx.x] : 0.0;
    b = (threadIdx.x < nw) ? sb[threadIdx.x] : 0.0;
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
}

// partial[blockIdx.y*gridDim.x + blockIdx.x] = sum over chunk of conj(V_i) w,  i = blockIdx.y
__global__ void multidot_kernel(int64_t n, const double2* __restrict__ V, int64_t ldv, const double2* __restrict__ w,
                                double2* __restrict__ partial) {
    const double2* v = V + (int64_t)blockIdx.y * ldv;
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    double re = 0, im = 0;
    for (int64_t k = lo + threadIdx.x; k < hi; k += blockDim.x) {
        double2 a = v[k], b = w[k];
        re += a.x * b.x + a.y * b.y;
        im += a.x * b.y - a.y * b.x;
    }
    block_sum2(re, im);
    if (threadIdx.x == 0) partial[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = make_double2(re, im);
}

// Tiled multi-dot: partial[i*gridDim.x + blockIdx.x] = sum over the block's
// chunk of conj(V_i) w for all i < nvec.  w's chunk is read once per tile of
// 8 vectors (L1 resident); every V_i is read exactly once.
constexpr int MD_TILE = 8;
__global__ void __launch_bounds__(256) multidot_tile_kernel(int64_t n, int nvec, const double2* __restrict__ V,
                                                             int64_t ldv, const double2* __restrict__ w,
                                                             double2* __restrict__ partial) {
    __shared__ double red[2 * MD_TILE][8];
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i0 = 0; i0 < nvec; i0 += MD_TILE) {
        double re[MD_TILE], im[MD_TILE];
#pragma unroll
        for (int q = 0; q < MD_TILE; ++q) { re[q] = 0; im[q] = 0; }
        for (int64_t k = lo + threadIdx.x; k < hi; k += blockDim.x) {
            double2 b = w[k];
#pragma unroll
            for (int q = 0; q < MD_TILE; ++q) {
                if (i0 + q < nvec) {
                    double2 a = V[(int64_t)(i0 + q) * ldv + k];
                    re[q] += a.x * b.x + a.y * b.y;
                    im[q] += a.x * b.y - a.y * b.x;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < MD_TILE; ++q)
            for (int o = 16; o > 0; o >>= 1) {
                re[q] += __shfl_down_sync(0xffffffffu, re[q], o);
                im[q] += __shfl_down_sync(0xffffffffu, im[q], o);
            }
        __syncthreads();
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < MD_TILE; ++q) { red[2 * q][wid] = re[q]; red[2 * q + 1][wid] = im[q]; }
        __syncthreads();
        if (threadIdx.x < 2 * MD_TILE) {
            double acc = 0;
            for (int u = 0; u < nw; ++u) acc += red[threadIdx.x][u];
            int q = threadIdx.x >> 1;
            if (i0 + q < nvec) {
                double2* out = &partial[(int64_t)(i0 + q) * gridDim.x + blockIdx.x];
                if (threadIdx.x & 1) out->y = acc; else out->x = acc;
            }
        }
    }
}

// h[i] = sum_c partial[i][c]; optionally accumulate into Hcol[i]
__global__ void finish_dot_kernel(int nparts, const double2* __restrict__ partial, double2* __restrict__ h,
                                  double2* __restrict__ Hcol, int accumulate) {
    int i = blockIdx.x;
    double re = 0, im = 0;
    for (int c = threadIdx.x; c < nparts; c += blockDim.x) {
        double2 p = partial[(int64_t)i * nparts + c];
        re += p.x; im += p.y;
    }
    block_sum2(re, im);
    if (threadIdx.x == 0) {
        h[i] = make_double2(re, im);
        if (Hcol) {
            if (accumulate) Hcol[i] = make_double2(Hcol[i].x + re, Hcol[i].y + im);
            else Hcol[i] = make_double2(re, im);
        }
    }
}

// w -= sum_{i<=j} h_i V_i
__global__ void cgs_update_kernel(int64_t n, int nvec, const double2* __restrict__ V, int64_t ldv,
                                  const double2* __restrict__ h, double2* __restrict__ w) {
    extern __shared__ double2 sh[];
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) sh[i] = h[i];
    __syncthreads();
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 acc = w[k];
#pragma unroll 4
        for (int i = 0; i < nvec; ++i) {
            double2 v = V[(int64_t)i * ldv + k];
            double2 c = sh[i];
            acc.x -= c.x * v.x - c.y * v.y;
            acc.y -= c.x * v.y + c.y * v.x;
        }
        w[k] = acc;
    }
}

// out = sum_i y_i V_i
__global__ void combo_kernel(int64_t n, int nvec, const double2* __restrict__ V, int64_t ldv,
                             const double2* __restrict__ y, double2* __restrict__ out) {
    extern __shared__ double2 sh[];
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) sh[i] = y[i];
    __syncthreads();
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double re = 0, im = 0;
        for (int i = 0; i < nvec; ++i) {
            double2 v = V[(int64_t)i * ldv + k];
            double2 c = sh[i];
            re += c.x * v.x - c.y * v.y;
            im += c.x * v.y + c.y * v.x;
        }
        out[k] = make_double2(re, im);
    }
}

__global__ void nrm2_partial_kernel(int64_t n, const double2* __restrict__ w, double2* __restrict__ partial) {
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    double s = 0, dummy = 0;
    for (int64_t k = lo + threadIdx.x; k < hi; k += blockDim.x) {
        double2 a = w[k];
        s += a.x * a.x + a.y * a.y;
    }
    block_sum2(s, dummy);
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(s, 0);
}

// dst = src / nrm  where nrm = sqrt(*sq) ; also writes nrm to *out (optional)
__global__ void normalize_kernel(int64_t n, const double2* __restrict__ sq, const double2* __restrict__ src,
                                 double2* __restrict__ dst, double2* __restrict__ out) {
    double nr = sqrt(sq->x);
    if (blockIdx.x == 0 && threadIdx.x == 0 && out) *out = make_double2(nr, 0);
    double inv = nr > 0 ? 1.0 / nr : 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 a = src[k];
        dst[k] = make_double2(a.x * inv, a.y * inv);
    }
}

__global__ void axpy_kernel(int64_t n, double2 a, const double2* __restrict__ x, double2* __restrict__ y) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 v = x[k];
        y[k] = make_double2(y[k].x + a.x * v.x - a.y * v.y, y[k].y + a.x * v.y + a.y * v.x);
    }
}

__global__ void sub_kernel(int64_t n, const double2* __restrict__ a, const double2* __restrict__ b, double2* __restrict__ c) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        c[k] = make_double2(a[k].x - b[k].x, a[k].y - b[k].y);
}

// Givens step j on column j of H ((m+1) x m, column-major, ld = m+1); g (m+1).
// Writes |g[j+1]| to *resid (host-mapped).
__global__ void givens_kernel(int j, int ldh, double2* __restrict__ H, double2* __restrict__ cs_sn,
                              double2* __restrict__ g, const double2* __restrict__ hnext, double* __restrict__ resid) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double2* col = H + (int64_t)j * ldh;
    col[j + 1] = *hnext;
    for (int i = 0; i < j; ++i) {
        double c = cs_sn[2 * i].x;
        double2 s = cs_sn[2 * i + 1];
        double2 a = col[i], b = col[i + 1];
        // [c s; -conj(s) c]
        double2 na = make_double2(c * a.x + s.x * b.x - s.y * b.y, c * a.y + s.x * b.y + s.y * b.x);
        double2 nb = make_double2(-(s.x * a.x + s.y * a.y) + c * b.x, -(s.x * a.y - s.y * a.x) + c * b.y);
        col[i] = na;
        col[i + 1] = nb;
    }
    double2 a = col[j], b = col[j + 1];
    double aa = hypot(a.x, a.y), bb = hypot(b.x, b.y);
    double c;
    double2 s;
    double2 r;
    if (aa == 0.0) {
        c = 0.0; s = make_double2(1, 0); r = b;
    } else {
        double rho = hypot(aa, bb);
        c = aa / rho;
        double2 ph = make_double2(a.x / aa, a.y / aa);
        // s = ph * conj(b) / rho
        s = make_double2((ph.x * b.x + ph.y * b.y) / rho, (ph.y * b.x - ph.x * b.y) / rho);
        r = make_double2(ph.x * rho, ph.y * rho);
    }
    cs_sn[2 * j] = make_double2(c, 0);
    cs_sn[2 * j + 1] = s;
    col[j] = r;
    col[j + 1] = make_double2(0, 0);
    double2 gj = g[j];
    g[j] = make_double2(c * gj.x, c * gj.y);
    g[j + 1] = make_double2(-(s.x * gj.x + s.y * gj.y), -(s.x * gj.y - s.y * gj.x));
    *resid = hypot(g[j + 1].x, g[j + 1].y);
}

// back substitution  R y = g  (R upper triangular k x k inside H)
__global__ void backsolve_kernel(int k, int ldh, const double2* __restrict__ H, const double2* __restrict__ g,
                                 double2* __restrict__ y) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = k - 1; i >= 0; --i) {
        double2 s = g[i];
        for (int c = i + 1; c < k; ++c) {
            double2 h = H[(int64_t)c * ldh + i], v = y[c];
            s.x -= h.x * v.x - h.y * v.y;
            s.y -= h.x * v.y + h.y * v.x;
        }
        double2 d = H[(int64_t)i * ldh + i];
        double den = d.x * d.x + d.y * d.y;
        y[i] = make_double2((s.x * d.x + s.y * d.y) / den, (s.y * d.x - s.x * d.y) / den);
    }
}

__global__ void set_g_kernel(int m1, double2* __restrict__ g, const double2* __restrict__ beta) {
    for (int i = threadIdx.x; i < m1; i += blockDim.x) g[i] = make_double2(i == 0 ? beta->x : 0.0, 0);
}

// ---------------------------------------------------------------------------
// vertex-patch block Jacobi
// ---------------------------------------------------------------------------
__device__ inline int32_t find_col(const int32_t* __restrict__ c, int32_t lo, int32_t hi, int32_t col) {
    int32_t h0 = hi;
    while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (c[mid] < col) lo = mid + 1; else hi = mid;
    }
    return (lo < h0 && c[lo] == col) ? lo : -1;
}

__global__ void patch_extract_kernel(int npatch, const int32_t* __restrict__ pptr, const int32_t* __restrict__ pdofs,
                                     const int64_t* __restrict__ poff, const int32_t* __restrict__ rowptr,
                                     const int32_t* __restrict__ cols, const double2* __restrict__ A,
                                     const uint8_t* __restrict__ dmask, double2* __restrict__ B,
                                     const int32_t* __restrict__ plist) {
    int v = plist ? plist[blockIdx.x] : blockIdx.x;   // plist: only the listed patches
    if (v >= npatch) return;
    int32_t p0 = pptr[v];
    int s = pptr[v + 1] - p0;
    double2* Bv = B + poff[v];
    for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
        int a = t / s, b = t % s;
        int32_t r = pdofs[p0 + a], c = pdofs[p0 + b];
        double2 val = make_double2(0, 0);
        if (dmask[r] || dmask[c]) {
            if (a == b) val = make_double2(1, 0);
        } else {
            int32_t k = find_col(cols, rowptr[r], rowptr[r + 1], c);
            if (k >= 0) val = A[k];
        }
        Bv[t] = val;
    }
}

// In-place Gauss-Jordan inversion with partial pivoting, one CTA per patch.
// The block is staged in shared memory when it fits, otherwise worked on in
// global memory (L2 resident).
__global__ void patch_invert_kernel(int npatch, const int32_t* __restrict__ pptr, const int64_t* __restrict__ poff,
                                    double2* __restrict__ B, int smem_max_s, int* __restrict__ status,
                                    const int32_t* __restrict__ plist) {
    extern __shared__ double2 sm[];
    __shared__ int piv_row;
    __shared__ double piv_abs[32];
    __shared__ int piv_idx[32];
    __shared__ int ipiv[512];
    int v = plist ? plist[blockIdx.x] : blockIdx.x;   // plist: only the listed patches
    if (v >= npatch) return;
    int s = pptr[v + 1] - pptr[v];
    double2* G = B + poff[v];
    bool use_sm = s <= smem_max_s;
    double2* M = use_sm ? sm : G;
    if (use_sm)
        for (int t = threadIdx.x; t < s * s; t += blockDim.x) M[t] = G[t];
    __syncthreads();
    for (int c = 0; c < s; ++c) {
        // pivot search over rows c..s-1
        double best = -1.0;
        int bi = c;
        for (int r = c + threadIdx.x; r < s; r += blockDim.x) {
            double2 x = M[r * s + c];
            double ax = fabs(x.x) + fabs(x.y);
            if (ax > best) { best = ax; bi = r; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double ob = __shfl_down_sync(0xffffffffu, best, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if ((threadIdx.x & 31) == 0) { piv_abs[threadIdx.x >> 5] = best; piv_idx[threadIdx.x >> 5] = bi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            int nw = blockDim.x >> 5;
            double b0 = piv_abs[0];
            int i0 = piv_idx[0];
            for (int w = 1; w < nw; ++w)
                if (piv_abs[w] > b0 || (piv_abs[w] == b0 && piv_idx[w] < i0)) { b0 = piv_abs[w]; i0 = piv_idx[w]; }
            piv_row = i0;
            if (c < 512) ipiv[c] = i0;
            if (!(b0 > 0.0)) atomicExch(status, 1);
        }
        __syncthreads();
        int pr = piv_row;
        if (pr != c)
            for (int k = threadIdx.x; k < s; k += blockDim.x) {
                double2 t0 = M[c * s + k];
                M[c * s + k] = M[pr * s + k];
                M[pr * s + k] = t0;
            }
        __syncthreads();
        double2 p = M[c * s + c];
        double den = p.x * p.x + p.y * p.y;
        double2 ip = den > 0 ? make_double2(p.x / den, -p.y / den) : make_double2(0, 0);
        __syncthreads();
        // scale pivot row (pivot entry becomes 1/p)
        for (int k = threadIdx.x; k < s; k += blockDim.x) {
            double2 x = (k == c) ? make_double2(1, 0) : M[c * s + k];
            M[c * s + k] = cmul(x, ip);
        }
        __syncthreads();
        // eliminate the other rows
        for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
            int r = t / s, k = t % s;
            if (r == c) continue;
            double2 f = M[r * s + c];
            if (k == c) continue;
            M[r * s + k] = csub(M[r * s + k], cmul(f, M[c * s + k]));
        }
        __syncthreads();
        for (int r = threadIdx.x; r < s; r += blockDim.x) {
            if (r == c) continue;
            double2 f = M[r * s + c];
            M[r * s + c] = make_double2(-(f.x * M[c * s + c].x - f.y * M[c * s + c].y),
                                        -(f.x * M[c * s + c].y + f.y * M[c * s + c].x));
        }
        __syncthreads();
    }
    // undo the row interchanges as column interchanges, last first
    for (int c = min(s, 512) - 1; c >= 0; --c) {
        int pr = ipiv[c];
        if (pr != c)
            for (int r = threadIdx.x; r < s; r += blockDim.x) {
                double2 t0 = M[r * s + c];
                M[r * s + c] = M[r * s + pr];
                M[r * s + pr] = t0;
            }
        __syncthreads();
    }
    if (use_sm)
        for (int t = threadIdx.x; t < s * s; t += blockDim.x) G[t] = M[t];
}

// phase 1: t[p0+a] = sum_b B_v[a][b] r[dofs[p0+b]]
// One CTA per patch; each warp keeps 4 block rows in flight (independent
// 16-byte loads per lane) to hide DRAM latency; lanes stride the columns so
// every row read is coalesced.
__global__ void __launch_bounds__(256) patch_apply1_kernel(int npatch, const int32_t* __restrict__ pptr,
                                                            const int32_t* __restrict__ pdofs,
                                                            const int64_t* __restrict__ poff, const double2* __restrict__ B,
                                                            const double2* __restrict__ r, double2* __restrict__ t) {
    extern __shared__ double2 rv[];
    int v = blockIdx.x;
    int32_t p0 = pptr[v];
    int s = pptr[v + 1] - p0;
    for (int a = threadIdx.x; a < s; a += blockDim.x) rv[a] = r[pdofs[p0 + a]];
    __syncthreads();
    const double2* Bv = B + poff[v];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    constexpr int RW = 4;
    for (int a0 = w * RW; a0 < s; a0 += nw * RW) {
        double re[RW], im[RW];
#pragma unroll
        for (int q = 0; q < RW; ++q) { re[q] = 0; im[q] = 0; }
        for (int b = lane; b < s; b += 32) {
            double2 x = rv[b];
#pragma unroll
            for (int q = 0; q < RW; ++q) {
                if (a0 + q < s) {
                    double2 m = __ldcs(&Bv[(int64_t)(a0 + q) * s + b]);
                    re[q] += m.x * x.x - m.y * x.y;
                    im[q] += m.x * x.y + m.y * x.x;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < RW; ++q) {
            for (int o = 16; o > 0; o >>= 1) {
                re[q] += __shfl_down_sync(0xffffffffu, re[q], o);
                im[q] += __shfl_down_sync(0xffffffffu, im[q], o);
            }
            if (lane == 0 && a0 + q < s) t[p0 + a0 + q] = make_double2(re[q], im[q]);
        }
    }
}

// phase 2: y_i = sum over the patch entries of dof i (fixed order); masked rows -> 0
__global__ void patch_apply2_kernel(int64_t n, const int32_t* __restrict__ d2p_ptr, const int32_t* __restrict__ d2p_idx,
                                    const double2* __restrict__ t, const uint8_t* __restrict__ dmask, double2* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double re = 0, im = 0;
        if (!dmask[i])
            for (int32_t q = d2p_ptr[i]; q < d2p_ptr[i + 1]; ++q) {
                double2 v = t[d2p_idx[q]];
                re += v.x; im += v.y;
            }
        y[i] = make_double2(re, im);
    }
}

__global__ void diag_inv_kernel(int64_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                                const double* __restrict__ A, double* __restrict__ dinv) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double d = 0;
        for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (cols[k] == i) { d = A[k]; break; }
        dinv[i] = d != 0 ? 1.0 / d : 1.0;
    }
}

__global__ void dscale_kernel(int64_t n, const double* __restrict__ d, const double2* __restrict__ x, double2* __restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = make_double2(d[i] * x[i].x, d[i] * x[i].y);
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
struct Red {
    DBuf<double2> part, out;
    explicit Red(int nmax) : part((size_t)nmax * RED_BLOCKS), out(nmax + 4) {}
};

static int md_blocks(const Problem& P) { return std::min(RED_BLOCKS, 2 * P.ctx->sm_count); }

static void dot_many(Problem& P, Red& R, const double2* V, int64_t ldv, int nvec, const double2* w, double2* Hcol,
                     int accumulate) {
    cudaStream_t s = P.ctx->stream;
    int64_t n = P.topo.n;
    const int nb = md_blocks(P);
    multidot_tile_kernel<<<nb, 256, 0, s>>>(n, nvec, V, ldv, w, R.part.p); ++P.ctx->launches;
    finish_dot_kernel<<<nvec, 256, 0, s>>>(nb, R.part.p, R.out.p, Hcol, accumulate); ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
}

static void nrm2_dev(Problem& P, Red& R, const double2* w, double2* sq_out) {
    cudaStream_t s = P.ctx->stream;
    nrm2_partial_kernel<<<RED_BLOCKS, 256, 0, s>>>(P.topo.n, w, R.part.p); ++P.ctx->launches;
    finish_dot_kernel<<<1, 256, 0, s>>>(RED_BLOCKS, R.part.p, sq_out, nullptr, 0); ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
}

static double read_scalar(Problem& P, const double2* dev, bool sqrt_it) {
    double2 h;
    OPEM_CUDA(cudaMemcpyAsync(&h, dev, sizeof(double2), cudaMemcpyDeviceToHost, P.ctx->stream));
    OPEM_CUDA(cudaStreamSynchronize(P.ctx->stream));
    return sqrt_it ? std::sqrt(h.x) : h.x;
}

static unsigned vgrid(const Problem& P) { return (unsigned)(P.ctx->sm_count * 8); }

struct PatchPrec {
    DBuf<double2> B, t;
    DBuf<int> status;
};

static void patch_setup(Problem& P, PatchPrec& pc, const double2* A, const uint8_t* dmask,
                        const int32_t* plist = nullptr, int nlist = 0) {
    cudaStream_t s = P.ctx->stream;
    const Topology& T = P.topo;
    size_t tot = (size_t)T.patch_off.back();
    if (pc.B.n < tot) pc.B.alloc(tot);
    if (pc.t.n < T.patch_dofs.size()) pc.t.alloc(T.patch_dofs.size());
    if (pc.status.n < 1) pc.status.alloc(1);
    pc.status.zero(s);
    const unsigned grid = plist ? (unsigned)nlist : (unsigned)P.npatch;
    if (grid == 0) return;
    patch_extract_kernel<<<grid, 256, 0, s>>>(P.npatch, P.d_patch_ptr.p, P.d_patch_dofs.p, P.d_patch_off.p,
                                              P.d_rowptr.p, P.d_cols.p, A, dmask, pc.B.p, plist); ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
    int smax = 0;
    size_t smem = 0;
    int dev_max = 0;
    OPEM_CUDA(cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, P.ctx->device));
    size_t budget = (size_t)dev_max - 4096;
    while ((size_t)(smax + 1) * (smax + 1) * sizeof(double2) <= budget) ++smax;
    smax = std::min(smax, T.max_patch);
    smem = (size_t)smax * smax * sizeof(double2);
    // the attribute is per function and process-wide: set the same device-wide value on
    // every call (concurrent problems with other patch sizes must not lower it)
    OPEM_CUDA(cudaFuncSetAttribute(patch_invert_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget));
    if (T.max_patch > 512) throw OpemError(OPEM_ERR_UNSUPPORTED, "vertex patch larger than 512 dofs");
    patch_invert_kernel<<<grid, 256, smem, s>>>(P.npatch, P.d_patch_ptr.p, P.d_patch_off.p, pc.B.p, smax, pc.status.p,
                                                plist); ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
}

// FP64 inverted vertex-patch blocks of A (for the mixed path, which rounds them to FP32).
void patch_blocks_fp64(Problem& P, const double2* A, const uint8_t* dmask, DBuf<double2>& B, const int32_t* plist,
                       int nlist) {
    PatchPrec pc;
    patch_setup(P, pc, A, dmask, plist, nlist);
    B = std::move(pc.B);
}

static void patch_apply(Problem& P, PatchPrec& pc, const double2* r, double2* y, const uint8_t* dmask) {
    cudaStream_t s = P.ctx->stream;
    size_t smem = (size_t)P.topo.max_patch * sizeof(double2);
    patch_apply1_kernel<<<P.npatch, 256, smem, s>>>(P.npatch, P.d_patch_ptr.p, P.d_patch_dofs.p, P.d_patch_off.p, pc.B.p,
                                                    r, pc.t.p); ++P.ctx->launches;
    patch_apply2_kernel<<<vgrid(P), 256, 0, s>>>(P.topo.n, P.d_d2p_ptr.p, P.d_d2p_idx.p, pc.t.p, dmask, y); ++P.ctx->launches;
    OPEM_CUDA(cudaGetLastError());
}

// W[:, c] = sum_r V[:, r] Q[r, c]  (tall-skinny basis rotation for deflated restarts).
// Q ((m+1) x (k+1), ~100 KB) is read through the read-only cache: every thread
// reads the same entries, so they are L1 broadcasts.
__global__ void basis_rotate_kernel(int64_t n, int nin, int nout, const double2* __restrict__ V, int64_t ldv,
                                    const double2* __restrict__ Q, double2* __restrict__ W, int64_t ldw) {
    constexpr int CH = 8;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        for (int c0 = 0; c0 < nout; c0 += CH) {
            double re[CH], im[CH];
#pragma unroll
            for (int q = 0; q < CH; ++q) { re[q] = 0; im[q] = 0; }
            for (int r = 0; r < nin; ++r) {
                double2 v = V[(int64_t)r * ldv + k];
#pragma unroll
                for (int q = 0; q < CH; ++q) {
                    if (c0 + q < nout) {
                        double2 c = __ldg(&Q[(c0 + q) * nin + r]);
                        re[q] += v.x * c.x - v.y * c.y;
                        im[q] += v.x * c.y + v.y * c.x;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < CH; ++q)
                if (c0 + q < nout) W[(int64_t)(c0 + q) * ldw + k] = make_double2(re[q], im[q]);
        }
    }
}


// ---------------------------------------------------------------------------
// GMRES-DR(m, k), FP64, right preconditioned by vertex-patch block Jacobi.
// Restarted GMRES (the reference's KSPGMRES) with deflated restarting: at
// each restart the k harmonic Ritz vectors of smallest modulus are kept in
// the basis (Morgan's GMRES-DR), so restarts do not throw away the slow
// modes.  k = 0 gives plain GMRES(m).  Solves the free block A_FF x_F = b_F;
// rows/cols in dmask are identity and every Krylov vector is zero there.
// The device runs the Arnoldi steps (SpMV, block Jacobi, CGS2) and the
// Hessenberg least squares; the host the per-restart harmonic-Ritz
// eigenproblem, in FP64.
// ---------------------------------------------------------------------------
SolveResult solve_plain_fp64(Problem& P, const double2* A, const uint8_t* dmask, const double2* b, double2* x,
                             const opem_solver_opts& o) {
    cudaStream_t s = P.ctx->stream;
    const int64_t n = P.topo.n;
    const int m = std::max(2, o.restart);
    const int kd = std::max(0, std::min(o.deflate, m - 2));
    SolveResult res;
    DBuf<double2> V((size_t)(m + 1) * n), w(n), z(n), H((size_t)(m + 1) * m), yd(m + 2), scal(8), Qd;
    DBuf<double2> Wd;
    if (kd > 0) { Wd.alloc((size_t)(kd + 1) * n); Qd.alloc((size_t)(m + 1) * (kd + 1)); }
    Red R(m + 2);
    PatchPrec pc;
    patch_setup(P, pc, A, dmask);
    OPEM_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double2), s));
    nrm2_dev(P, R, b, scal.p);
    double bnorm = read_scalar(P, scal.p, true);
    if (bnorm == 0.0) { res.converged = 1; return res; }
    OPEM_CUDA(cudaMemcpyAsync(w.p, b, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    std::vector<cd> Hh((size_t)(m + 1) * m, 0.0), c(m + 1, 0.0), y;
    LsqWork lsq;
    lsq.alloc(1, m, kd, s);
    DBuf<uint8_t> one;
    one.upload(std::vector<uint8_t>(1, 1), s);
    DBuf<int> ncd(1);
    double beta = bnorm;
    int start = 0, its = 0;
    bool fresh = true;
    while (true) {
        if (fresh) {
            // V0 = r / ||r||
            nrm2_dev(P, R, w.p, scal.p);
            normalize_kernel<<<vgrid(P), 256, 0, s>>>(n, scal.p, w.p, V.p, scal.p + 1);
            ++P.ctx->launches;
            std::fill(Hh.begin(), Hh.end(), 0.0);
            std::fill(c.begin(), c.end(), 0.0);
            c[0] = beta;
            start = 0;
        }
        std::vector<double2> c0(m + 1);
        for (int i = 0; i <= m; ++i) c0[i] = make_double2(c[i].real(), c[i].imag());
        std::vector<double> e1(1, 0.0);
        lsq.start_cycle(std::vector<uint8_t>(1, 1), c0, std::vector<int>(1, start), H.p, s, e1);
        ++P.ctx->launches;
        double est = e1[0];
        int ncol = start;
        for (int j = start; j < m; ++j) {
            double2* Vj = V.p + (int64_t)j * n;
            patch_apply(P, pc, Vj, z.p, dmask);
            spmv_complex(P, A, z.p, w.p, dmask);
            double2* Hcol = H.p + (int64_t)j * (m + 1);
            for (int pass = 0; pass < 2; ++pass) {
                dot_many(P, R, V.p, n, j + 1, w.p, Hcol, pass);
                cgs_update_kernel<<<vgrid(P), 256, (j + 1) * sizeof(double2), s>>>(n, j + 1, V.p, n, R.out.p, w.p);
                ++P.ctx->launches;
            }
            nrm2_dev(P, R, w.p, scal.p + 2);
            normalize_kernel<<<vgrid(P), 256, 0, s>>>(n, scal.p + 2, w.p, V.p + (int64_t)(j + 1) * n, Hcol + j + 1);
            ++P.ctx->launches;
            OPEM_CUDA(cudaGetLastError());
            lsq.step(j, one.p, H.p, s, e1);
            ++P.ctx->launches;
            if (P.cancel.load(std::memory_order_relaxed)) throw OpemError(OPEM_ERR_CANCELLED, "request cancelled");
            est = e1[0];
            ++its;
            ncol = j + 1;
            if (!std::isfinite(est)) { res.code = OPEM_ERR_BREAKDOWN; break; }
            if (est / bnorm <= o.rtol || its >= o.maxits) break;
        }
        if (res.code != OPEM_OK) break;
        // x += M^-1 (V y), y from the device least squares
        lsq.check(s);
        ncd.upload(&ncol, 1, s);
        lsq.solve(ncd.p, one.p, yd.p, m, s);
        ++P.ctx->launches;
        combo_kernel<<<vgrid(P), 256, ncol * sizeof(double2), s>>>(n, ncol, V.p, n, yd.p, w.p);
        ++P.ctx->launches;
        patch_apply(P, pc, w.p, z.p, dmask);
        axpy_kernel<<<vgrid(P), 256, 0, s>>>(n, make_double2(1, 0), z.p, x);
        ++P.ctx->launches;
        // true residual
        spmv_complex(P, A, x, z.p, dmask);
        sub_kernel<<<vgrid(P), 256, 0, s>>>(n, b, z.p, w.p);
        ++P.ctx->launches;
        nrm2_dev(P, R, w.p, scal.p);
        beta = read_scalar(P, scal.p, true);
        if (!std::isfinite(beta)) { res.code = OPEM_ERR_BREAKDOWN; break; }
        if (beta / bnorm <= o.rtol) { res.converged = 1; break; }
        if (its >= o.maxits) break;
        fresh = true;
        if (kd == 0 || ncol < m) continue;
        // ---- deflated restart (harmonic Ritz vectors of the m x m problem), from
        // the cycle's H (zero outside each column's rows) and y
        {
            std::vector<double2> hh((size_t)(m + 1) * m), yh(m);
            OPEM_CUDA(cudaMemcpyAsync(hh.data(), H.p, hh.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
            OPEM_CUDA(cudaMemcpyAsync(yh.data(), yd.p, m * sizeof(double2), cudaMemcpyDeviceToHost, s));
            OPEM_CUDA(cudaStreamSynchronize(s));
            for (int j = 0; j < m; ++j) {
                const int top = j < start ? start : j + 1;
                for (int i = 0; i <= m; ++i)
                    Hh[i + (size_t)j * (m + 1)] = i <= top ? cd(hh[i + (size_t)j * (m + 1)].x, hh[i + (size_t)j * (m + 1)].y) : cd(0.0);
            }
            y.assign(m, 0.0);
            for (int i = 0; i < m; ++i) y[i] = cd(yh[i].x, yh[i].y);
        }
        std::vector<cd> Pm, Hn, cn;
        if (!gmres_dr_deflate(m, kd, Hh, c, y, Pm, Hn, cn)) continue;
        // device: V[:, :kd+1] = V Pm
        std::vector<double2> Qh((size_t)(m + 1) * (kd + 1));
        for (size_t t = 0; t < Qh.size(); ++t) Qh[t] = make_double2(Pm[t].real(), Pm[t].imag());
        OPEM_CUDA(cudaMemcpyAsync(Qd.p, Qh.data(), Qh.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
        basis_rotate_kernel<<<vgrid(P), 256, 0, s>>>(n, m + 1, kd + 1, V.p, n, Qd.p, Wd.p, n);
        ++P.ctx->launches;
        OPEM_CUDA(cudaMemcpyAsync(V.p, Wd.p, (size_t)(kd + 1) * n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        // the restart block becomes the first kd columns of the next cycle's H
        {
            std::vector<double2> hn(Hn.size());
            for (size_t t = 0; t < hn.size(); ++t) hn[t] = make_double2(Hn[t].real(), Hn[t].imag());
            OPEM_CUDA(cudaMemcpyAsync(H.p, hn.data(), hn.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
        }
        OPEM_CUDA(cudaStreamSynchronize(s));
        c = cn;
        start = kd;
        fresh = false;
    }
    res.its = its;
    res.relres = beta / bnorm;
    if (!res.converged && res.code == OPEM_OK) res.code = OPEM_ERR_NOT_CONVERGED;
    return res;
}

// ---------------------------------------------------------------------------
// CG on the (real SPD) ND mass matrix with complex right-hand side, Jacobi
// preconditioned: P h = b  (fem3D::build_P + solveHfield).
// ---------------------------------------------------------------------------
__global__ void cg_update_kernel(int64_t n, const double2* __restrict__ alpha_num, const double2* __restrict__ alpha_den,
                                 const double2* __restrict__ p, const double2* __restrict__ q, double2* __restrict__ x,
                                 double2* __restrict__ r) {
    // alpha = rz / (p^H q)  (complex; p^H q is real for SPD)
    double2 an = *alpha_num, ad = *alpha_den;
    double den = ad.x * ad.x + ad.y * ad.y;
    double2 a = make_double2((an.x * ad.x + an.y * ad.y) / den, (an.y * ad.x - an.x * ad.y) / den);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 pk = p[k], qk = q[k];
        x[k] = make_double2(x[k].x + a.x * pk.x - a.y * pk.y, x[k].y + a.x * pk.y + a.y * pk.x);
        r[k] = make_double2(r[k].x - (a.x * qk.x - a.y * qk.y), r[k].y - (a.x * qk.y + a.y * qk.x));
    }
}

__global__ void cg_direction_kernel(int64_t n, const double2* __restrict__ rz_new, const double2* __restrict__ rz_old,
                                    const double2* __restrict__ z, double2* __restrict__ p) {
    double2 a = *rz_new, b = *rz_old;
    double den = b.x * b.x + b.y * b.y;
    double2 beta = make_double2((a.x * b.x + a.y * b.y) / den, (a.y * b.x - a.x * b.y) / den);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 pk = p[k];
        p[k] = make_double2(z[k].x + beta.x * pk.x - beta.y * pk.y, z[k].y + beta.x * pk.y + beta.y * pk.x);
    }
}

SolveResult solve_mass_cg(Problem& P, const double2* b, double2* x, double rtol, int maxits) {
    cudaStream_t s = P.ctx->stream;
    const int64_t n = P.topo.n;
    SolveResult res;
    DBuf<double> dinv(n);
    DBuf<double2> r(n), z(n), p(n), q(n), sc(8);
    Red R(4);
    diag_inv_kernel<<<vgrid(P), 256, 0, s>>>(n, P.d_rowptr.p, P.d_cols.p, P.d_M1.p, dinv.p); ++P.ctx->launches;
    OPEM_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double2), s));
    OPEM_CUDA(cudaMemcpyAsync(r.p, b, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    nrm2_dev(P, R, b, sc.p);
    double bnorm = read_scalar(P, sc.p, true);
    if (bnorm == 0) { res.converged = 1; return res; }
    dscale_kernel<<<vgrid(P), 256, 0, s>>>(n, dinv.p, r.p, z.p); ++P.ctx->launches;
    OPEM_CUDA(cudaMemcpyAsync(p.p, z.p, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    dot_many(P, R, r.p, n, 1, z.p, nullptr, 0);   // rz = r^H z
    OPEM_CUDA(cudaMemcpyAsync(sc.p + 1, R.out.p, sizeof(double2), cudaMemcpyDeviceToDevice, s));
    int its = 0;
    double rn = bnorm;
    while (its < maxits) {
        spmv_real_complex(P, P.d_M1.p, p.p, q.p, 1.0, 0.0);
        dot_many(P, R, p.p, n, 1, q.p, nullptr, 0);   // p^H q
        cg_update_kernel<<<vgrid(P), 256, 0, s>>>(n, sc.p + 1, R.out.p, p.p, q.p, x, r.p); ++P.ctx->launches;
        ++its;
        if (its % 10 == 0 || its >= maxits) {
            nrm2_dev(P, R, r.p, sc.p + 3);
            rn = read_scalar(P, sc.p + 3, true);
            if (rn / bnorm <= rtol || !std::isfinite(rn)) break;
        }
        dscale_kernel<<<vgrid(P), 256, 0, s>>>(n, dinv.p, r.p, z.p); ++P.ctx->launches;
        dot_many(P, R, r.p, n, 1, z.p, nullptr, 0);   // rz_new
        cg_direction_kernel<<<vgrid(P), 256, 0, s>>>(n, R.out.p, sc.p + 1, z.p, p.p); ++P.ctx->launches;
        OPEM_CUDA(cudaMemcpyAsync(sc.p + 1, R.out.p, sizeof(double2), cudaMemcpyDeviceToDevice, s));
    }
    OPEM_CUDA(cudaGetLastError());
    res.its = its;
    res.relres = rn / bnorm;
    res.converged = res.relres <= rtol;
    if (!std::isfinite(rn)) res.code = OPEM_ERR_BREAKDOWN;
    return res;
}

}  // namespace opem

namespace opem {

// Times the FP64-path kernels in isolation (CUDA events on the context stream).
// out[3k+0] = ms per launch, out[3k+1] = algorithmic bytes per launch, out[3k+2] = launches.
void profile_fp64(Problem& P, const double2* A, const uint8_t* dmask, int reps, double* out) {
    cudaStream_t s = P.ctx->stream;
    const int64_t n = P.topo.n, nnz = (int64_t)P.topo.cols.size();
    const int nv = 64;
    DBuf<double2> V((size_t)nv * n), w(n), z(n);
    OPEM_CUDA(cudaMemsetAsync(V.p, 0, V.bytes(), s));
    OPEM_CUDA(cudaMemsetAsync(w.p, 0, w.bytes(), s));
    Red R(nv + 2);
    PatchPrec pc;
    patch_setup(P, pc, A, dmask);
    cudaEvent_t e0, e1;
    OPEM_CUDA(cudaEventCreate(&e0));
    OPEM_CUDA(cudaEventCreate(&e1));
    double patch_sq = 0, patch_len = 0;
    for (size_t v = 0; v + 1 < P.topo.patch_ptr.size(); ++v) {
        double sz = P.topo.patch_ptr[v + 1] - P.topo.patch_ptr[v];
        patch_sq += sz * sz;
        patch_len += sz;
    }
    auto timeit = [&](auto&& launch) {
        for (int i = 0; i < 3; ++i) launch();
        OPEM_CUDA(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; ++i) launch();
        OPEM_CUDA(cudaEventRecord(e1, s));
        OPEM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        OPEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return (double)ms / reps;
    };
    size_t smem_p = (size_t)P.topo.max_patch * sizeof(double2);
    out[0] = timeit([&] { spmv_complex(P, A, V.p, w.p, dmask); });
    out[1] = (double)nnz * (16 + 4) + 4.0 * (n + 1) + n * (16.0 + 16.0 + 1.0);
    out[3] = timeit([&] {
        patch_apply1_kernel<<<P.npatch, 256, smem_p, s>>>(P.npatch, P.d_patch_ptr.p, P.d_patch_dofs.p, P.d_patch_off.p,
                                                          pc.B.p, V.p, pc.t.p);
        ++P.ctx->launches;
    });
    out[4] = patch_sq * 16 + patch_len * (4 + 16 + 16) + P.npatch * 12.0;
    out[6] = timeit([&] {
        multidot_tile_kernel<<<md_blocks(P), 256, 0, s>>>(n, nv, V.p, n, w.p, R.part.p);
        ++P.ctx->launches;
    });
    out[7] = (double)nv * n * 16 + n * 16.0;
    out[9] = timeit([&] {
        cgs_update_kernel<<<P.ctx->sm_count * 8, 256, nv * sizeof(double2), s>>>(n, nv, V.p, n, R.out.p, w.p);
        ++P.ctx->launches;
    });
    out[10] = (double)nv * n * 16 + 2.0 * n * 16;
    for (int k = 0; k < 4; ++k) out[3 * k + 2] = reps;
    OPEM_CUDA(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

}  // namespace opem
