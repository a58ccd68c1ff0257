// Host-side engine state shared by the .cu files (internal).
#pragma once
#include <atomic>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "opem_device.h"
#include "opem_internal.h"
#include "portfem.h"

namespace opem {

#define OPEM_CUDA(call)                                                                   \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};
struct OpemError : std::runtime_error {
    int code;
    OpemError(int c, const std::string& s) : std::runtime_error(s), code(c) {}
};

// RAII device buffer
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    explicit DBuf(size_t n_) { alloc(n_); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; return *this; }
    ~DBuf() { release(); }
    void alloc(size_t n_) {
        release();
        n = n_;
        if (n) {
            cudaError_t e = cudaMalloc(&p, n * sizeof(T));
            if (e != cudaSuccess) { p = nullptr; n = 0; throw OpemError(OPEM_ERR_NOMEM, "cudaMalloc failed"); }
        }
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
    void upload(const T* h, size_t cnt, cudaStream_t s) { OPEM_CUDA(cudaMemcpyAsync(p, h, cnt * sizeof(T), cudaMemcpyHostToDevice, s)); }
    void upload(const std::vector<T>& v, cudaStream_t s) { if (v.size() > n) alloc(v.size()); if (!v.empty()) upload(v.data(), v.size(), s); }
    void zero(cudaStream_t s) { if (n) OPEM_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    size_t bytes() const { return n * sizeof(T); }
};

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    double* pinned = nullptr;     // small host-mapped scratch for scalars
    int sm_count = 148;
    int64_t launches = 0;         // kernels this context has launched (bench accounting)
};

// A boundary group: every boundary triangle of one attribute that adds a
// term to A (port ABC, impedance, radiation).
struct BGroup {
    int attr = 0, type = 0, port = -1;
    double sigma = 0, Rz = 0, mu_r = 1, eta = 0;
    std::vector<int32_t> faces;            // global face ids
    int64_t nu = 0;                        // unique CSR slots
    std::vector<int32_t> h_urow, h_ucol;   // row/col of each unique slot
    DBuf<int32_t> uslot, urow, ucol;       // device
    DBuf<double> R;                        // 5*nu: cc, eps, tand, sig, one
    // boundary CSR over the group's rows (for the batched SpMV correction)
    std::vector<int32_t> h_brow, h_bptr;
    DBuf<int32_t> brow, bptr;
};

// Modes a port was solved with, per frequency (ports driven by their own 2D mode)
struct PortFemCache {
    std::mutex mu;
    std::vector<std::pair<double, std::shared_ptr<const PortFem2D>>> sols;   // most recent last
};

struct PortMode {
    bool set = false;
    double desc[26];
    int kind = 0;    // 0: analytic TE_mn (desc), 1: 2D mode of the port faces
    int nsub = 0;    // kind 1: split of each port face
    int order2d = 1; // kind 1: 2D element order
    int zdef = 0;    // kind 1: OPEM_Z_PV / VI / PI
    std::vector<double> ipath;   // kind 1: current path points (xyz)
    bool ipath_closed = true;
    int mode = 0;    // kind 1: which mode of the 2D problem, in decreasing beta^2
    std::shared_ptr<PortFemCache> fem;
};

// A further mode of a port driven by its own 2D modes: one more S-port (and
// driving set) on the same faces, as the reference's ports with several modes.
// S-ports are numbered: every port's first mode in port order, then these in
// the order they were added.
struct ExtraMode {
    int port = -1;
    PortMode m;      // kind 1, the port's frame and element order; its own mode
                     // number, voltage path (desc[16..21]) and impedance definition
};

struct Problem {
    Context* ctx = nullptr;
    Topology topo;
    int nregions = 0;
    std::vector<double> eps_r, tand, sigma, mu_r;   // per region
    struct Bdr { int type = 0; double params[3] = {0, 0, 0}; };
    std::vector<std::pair<int, Bdr>> bdr;           // attr -> type
    int nports = 0;
    std::vector<PortMode> modes;
    std::vector<ExtraMode> extra;   // further modes of ports driven by their 2D modes
    int nsports() const { return nports + (int)extra.size(); }
    double trace_freq = -1;     // frequency of the device traces of ports driven by their 2D mode
    bool assembled = false;
    int64_t ws_cap = 0;         // device bytes a batched sweep may take for its workspace (0: half of free)
    std::atomic<int> cancel{0}; // set from another thread: the solvers stop at their next Krylov step

    // device mesh/operator data
    DBuf<double> d_verts;
    DBuf<int32_t> d_tets, d_region, d_elem_dofs;
    DBuf<ElemGeo> d_geo;
    DBuf<int32_t> d_rowptr, d_cols, d_d2e_ptr, d_d2e_elem;
    DBuf<uint8_t> d_d2e_loc;
    DBuf<double> d_ref;         // Kh(6) | Mh(6) | Qh, ld*ld each
    DBuf<double> d_K, d_Meps, d_Mtand, d_Msig, d_M1, d_Q;
    DBuf<float> f_K, f_Meps, f_Mtand, f_Msig;   // FP32 copies (mixed path)
    bool has_tand = false, has_sig = false;
    DBuf<double> d_elemcoef;    // per element: inv_mu, eps, eps*tand, sigma
    std::vector<BGroup> groups;
    // Dirichlet masks
    std::vector<uint8_t> h_pec, h_portmask;
    DBuf<uint8_t> d_pec, d_portmask;
    std::vector<std::vector<int32_t>> port_dofs;   // all dofs on each port's faces
    // port mode traces (frequency-independent shapes)
    std::vector<std::vector<double>> et_trace;     // per port: n complex (only port dofs nonzero)
    std::vector<std::vector<double>> nxe_trace;    // per port: trace of n x Et
    DBuf<double> d_et, d_nxe;                      // nports * n complex
    DBuf<double> d_et_x, d_nxe_x;                  // the same for the extra modes
    // vertex patches
    DBuf<int32_t> d_patch_ptr, d_patch_dofs, d_d2p_ptr, d_d2p_idx;
    DBuf<int64_t> d_patch_off;
    int npatch = 0;
    // patches with no DOF on any port face (their blocks are the same for every
    // driving set) and the others; built on first use by the batched solver
    DBuf<int32_t> d_plist_shared, d_plist_port;
    int n_plist_shared = -1, n_plist_port = 0;
    // last fields per driving set
    std::vector<std::vector<double>> last_e, last_h;
    int64_t device_bytes() const;
};

// ---- assembly (assemble.cu)
void assemble_volume(Problem& P);
void assemble_boundary(Problem& P);
// A = K + vc.c_eps*Meps + ... plus boundary groups (FP64 complex, nnz)
void form_system_matrix(Problem& P, const VolCoef& vc, const std::vector<BCoef>& bc, double2* A);
void form_system_matrix_n(Problem& P, const VolCoef& vc, const BCoef* bc, size_t nb, double2* A);
// host: coefficients of A(freq) for driving set d
void system_coefficients(const Problem& P, double freq, int d, VolCoef& vc, std::vector<BCoef>& bc);
void port_gamma_Z_V(const Problem& P, int port, double freq, cd& gamma, cd& Z, cd& V);
// gamma, Z, V of S-port s (port modes, then the extra modes)
void sport_gamma_Z_V(const Problem& P, int s, double freq, cd& gamma, cd& Z, cd& V);
// the physical port of S-port s
inline int sport_port(const Problem& P, int s) { return s < P.nports ? s : P.extra[s - P.nports].port; }
// gamma of port k's absorbing condition: of its largest-|gamma| mode
cd robin_gamma(const Problem& P, int k, double freq);
// Re-computes the device traces of the ports driven by their own 2D mode for
// freq (no-op when there are none or they are current); synchronises the stream.
void refresh_port_traces(Problem& P, double freq);
bool has_fem2d_ports(const Problem& P);
// ZZ error indicator of the H fields kept by the last opem_solve_frequency
// (estimate.cu): per element, the larger over the driving sets.
void mesh_error_indicator(Problem& P, std::vector<double>& err);
// overlaps <a, B_port b> for port k: out = conj(a)^T R_one b over the port's slots
void port_overlap(Problem& P, int k, const double2* a, const double2* b, double2* out_dev);

// ---- krylov / preconditioner (krylov.cu)
struct SolveResult { int its = 0; int converged = 0; double relres = 0; int code = OPEM_OK; };
SolveResult solve_plain_fp64(Problem& P, const double2* A, const uint8_t* dmask_dev, const double2* b,
                             double2* x, const opem_solver_opts& o);
SolveResult solve_mass_cg(Problem& P, const double2* b, double2* x, double rtol, int maxits);
void spmv_real_complex(Problem& P, const double* vals, const double2* x, double2* y, double scale_re, double scale_im);
void spmv_complex(Problem& P, const double2* A, const double2* x, double2* y, const uint8_t* zero_rows);
void profile_fp64(Problem& P, const double2* A, const uint8_t* dmask, int reps, double* out);
void profile_batch(Problem& P, double f, int R, int reps, double* out, int nout);
void check_block_apply(Problem& P, double f, int R, int r0, int Rd, double* out);
// Inverted FP64 vertex-patch blocks of A (Dirichlet rows/columns from dmask); with
// plist, only the nlist listed patches are computed (the others are left as they are).
void patch_blocks_fp64(Problem& P, const double2* A, const uint8_t* dmask, DBuf<double2>& B,
                       const int32_t* plist = nullptr, int nlist = 0);

// ---- engine helpers shared with the mixed path (engine.cu)
void make_dmask(Problem& P, int d, uint8_t* dm);
double port_mu_r(const Problem& P, int k);
std::vector<cd> s_matrix_solve(int N, const std::vector<cd>& Cp, const std::vector<cd>& Cm, const std::vector<cd>& V,
                               const std::vector<cd>& Z, bool reciprocal);

// ---- batched mixed-precision sweep (mixed.cu)
void solve_sweep_mixed(Problem& P, int nfreq, const double* freqs, const opem_solver_opts& o,
                       std::vector<std::vector<cd>>& S, std::vector<opem_solve_stats>& st);
// device bytes a request (nfreq points with options o) needs beyond what P already holds
double request_bytes_estimate(const Problem& P, int nfreq, const opem_solver_opts& o);
// failure-detection self-test (mixed.cu): OPEM_ERR_TIMEOUT when the bounded wait ran out
int selftest_wait_timeout(Context& C, int polls);

}  // namespace opem

// opaque handles of the C ABI
struct opem_context_s { opem::Context c; };
struct opem_problem_s {
    opem::Problem p;
    int device = 0;   // the context's device, kept for teardown without the context
};
