/*
 * opem_b200.h -- C ABI of the B200-native OpenParEM3D per-frequency solve stage.
 *
 * One library (libopem_b200.so), plain pointers and sizes, no C++ or torch
 * types.  Every entry point returns an int status (OPEM_OK == 0, negative
 * on error) and never exits the process.  Output buffers are owned by the
 * caller.  One opem_context per host thread; a context owns one CUDA device
 * and one stream.
 *
 * Reference seams replaced (paths inside the OpenParEM tree):
 *   fem3D::solve                      src/OpenParEM3D/fem3D.cpp:712-799 (declared fem3D.hpp:167-168)
 *   solveComplexLinearSystem          src/OpenParEM3D/solveComplexLinearSystem.c:100-209 (extern "C" at fem3D.cpp:24-25)
 *   fem3D::build_A                    src/OpenParEM3D/fem3D.cpp:103-190
 *   fem3D::buildHgrids / solveHfield  src/OpenParEM3D/fem3D.cpp:610-648, solveComplexLinearSystem.c:235-315
 *   Mode::calculateSplits             src/OpenParEM3D/port.cpp:3524-3568
 *   BoundaryDatabase::calculateS      src/OpenParEM3D/port.cpp:7499-7606
 *   Result::forceReciprocal           src/OpenParEM3D/results.cpp:401-418
 */
#ifndef OPEM_B200_H
#define OPEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------- */
#define OPEM_OK                 0
#define OPEM_ERR_ARG          (-1)   /* bad argument (null pointer, size, index)      */
#define OPEM_ERR_CUDA         (-2)   /* a CUDA runtime call failed                     */
#define OPEM_ERR_NOMEM        (-3)   /* device or host allocation failed               */
#define OPEM_ERR_STATE        (-4)   /* call out of order (e.g. solve before assemble) */
#define OPEM_ERR_MESH         (-5)   /* inconsistent mesh (boundary face not a mesh face, degenerate tet) */
#define OPEM_ERR_NOT_CONVERGED (-6)  /* iteration limit reached; outputs hold the last iterate */
#define OPEM_ERR_BREAKDOWN    (-7)   /* NaN/Inf or Krylov breakdown                    */
#define OPEM_ERR_TIMEOUT      (-8)   /* device-side iteration/time budget exhausted    */
#define OPEM_ERR_UNSUPPORTED  (-9)   /* order or feature not built                     */
#define OPEM_ERR_CANCELLED    (-10)  /* request cancelled (serving loop)                */

/* ---- boundary types (BoundaryDatabase attributes, src/OpenParEM3D/port.cpp:6885-7026) */
#define OPEM_BDR_PEC        1   /* essential, E_t = 0 (fem3D.cpp:80-99)                      */
#define OPEM_BDR_PMC        2   /* natural, nothing added                                    */
#define OPEM_BDR_PORT       3   /* wave port; params[0] = port index                          */
#define OPEM_BDR_IMPEDANCE  4   /* surface impedance; params = {sigma S/m, Rz m, mu_r}        */
#define OPEM_BDR_RADIATION  5   /* 1st-order RBC; params[0] = wave impedance ohm (<=0: eta0)  */

/* ---- port impedance definitions (the port file's impedance_definition) ---- */
#define OPEM_Z_PV           0   /* Z = V V* / (2 Pz*)   (voltage path)                        */
#define OPEM_Z_VI           1   /* Z = V / I            (voltage and current paths)           */
#define OPEM_Z_PI           2   /* Z = 2 Pz / (I I*)    (current path)                        */

/* ---- precision modes ----------------------------------------------------- */
#define OPEM_PREC_FP64      0   /* plain FP64 GMRES (the drop-in)                             */
#define OPEM_PREC_MIXED     1   /* FP32 inner GMRES + polynomial/block-Jacobi, FP64 refinement */

typedef struct opem_context_s* opem_context;
typedef struct opem_problem_s* opem_problem;

/* Solver options (solveComplexLinearSystem.c:131-141 defaults shown in brackets). */
typedef struct {
    double rtol;          /* relative residual tolerance [1e-10]                            */
    int    maxits;        /* total inner iteration limit [5000]                              */
    int    restart;       /* GMRES restart length m, 2..2048 [100]                           */
    int    precision;     /* OPEM_PREC_FP64 or OPEM_PREC_MIXED                               */
    int    poly_degree;   /* polynomial preconditioner degree (mixed mode), 0 = none [0]     */
    int    force_reciprocal; /* S <- (S+S^T)/2 (results.cpp:401-418) [1]                      */
    int    h_maxits;      /* iteration limit of the H projection CG [2000]                    */
    double h_rtol;        /* tolerance of the H projection CG [1e-12]                         */
    int    deflate;       /* harmonic Ritz vectors kept at each GMRES restart (GMRES-DR) [30] */
} opem_solver_opts;

typedef struct {
    int    iterations;    /* inner iterations summed over driving sets                      */
    int    outer;         /* refinement (outer) steps, mixed mode                            */
    int    h_iterations;  /* CG iterations of the H projection                               */
    int    converged;     /* 1 if every driving set met rtol                                  */
    double rnorm;         /* worst final relative residual ||b-Ax||/||b|| (FP64)             */
    double seconds;       /* device time of the whole call                                    */
} opem_solve_stats;

/* ---- context ----------------------------------------------------------- */
int  opem_context_create(int device, opem_context* out);
int  opem_context_destroy(opem_context ctx);
/* Last error message of this context (static storage inside ctx). */
const char* opem_context_last_error(opem_context ctx);
void opem_default_opts(opem_solver_opts* opts);

/* ---- problem setup (fem3D::build_fe_spaces, fem3D.cpp:65-78; mesh load OpenParEM3D.cpp:284-327)
 * verts: nverts*3 doubles (m); tets: ntets*4 int64 (0-based vertex ids);
 * tet_region: ntets int32 region index; bdr_tris: nbdr*3 int64; bdr_attr: nbdr int32 (>=1).
 * order: Nedelec order p (ND_FECollection(p,3)); 1..3 are supported.          */
int  opem_problem_create(opem_context ctx, int64_t nverts, const double* verts,
                         int64_t ntets, const int64_t* tets, const int32_t* tet_region,
                         int64_t nbdr, const int64_t* bdr_tris, const int32_t* bdr_attr,
                         int order, opem_problem* out);
int  opem_problem_destroy(opem_problem prob);
/* Region materials (per-region PWConstCoefficients, OpenParEM3D.cpp:394-437): relative
 * permittivity, loss tangent, conductivity (S/m), relative permeability.          */
int  opem_problem_set_regions(opem_problem prob, int nregions, const double* eps_r,
                              const double* tand, const double* sigma, const double* mu_r);
int  opem_problem_set_boundary(opem_problem prob, int attr, int type, const double* params, int nparams);
/* Analytic rectangular TE_mn port mode (the data load_modeMetrics reads, port.cpp:5302-5453).
 * desc = {origin xyz, u-axis xyz, v-axis xyz, outward normal xyz, a, b, m, n,
 *         voltage path start xyz, voltage path end xyz}  (22 doubles).          */
int  opem_problem_set_port_te(opem_problem prob, int port, const double* desc);
/* Port driven by the fundamental mode of its own cross-section, solved at every
 * frequency on the port faces split nsub x nsub (1..64) with the materials of
 * the tetrahedra behind them (the 2D solve the reference spawns per frequency,
 * port.cpp:5081-5176).  On split faces (nsub > 1) order 1: lowest-order edge
 * elements for e_t and linear nodal e_z (opem_port_mode_2d's solve); order 2:
 * degree-2 edge elements and quadratic nodal e_z (beta converges at fourth order
 * in the split).  With nsub 1, or order 3 to 8: first-kind edge elements of order
 * p and degree-p nodal e_z, the spaces of the reference's 2D solver at
 * mesh.order p; with nsub 1 and p the 3D order the mode lies in the 3D port trace
 * space, and the port follows the reference's 2D solver further: H_t projected
 * onto the edge space, Pz and the port's overlap integrals by the nodal rules of
 * MFEM's L2 triangle.  desc as for opem_problem_set_port_te; its a, b, m, n are
 * not used.                                                                    */
int  opem_problem_set_port_fem2d(opem_problem prob, int port, const double* desc, int nsub, int order);
/* Impedance definition of a port driven by its own 2D mode (after
 * opem_problem_set_port_fem2d; the reference's impedance_definition and current
 * IntegrationPath, Mode::calculateImpedance in OpenParEM2D fem2D.cpp:1803-1824):
 * definition OPEM_Z_PV (default) | OPEM_Z_VI | OPEM_Z_PI; path: npath >= 2 points
 * (xyz) of the current integration path in the port plane, I = sum over its
 * segments of int H . dl (a closed path also takes the segment from the last
 * point back to the first).  VI and PI need the path.  The mode's sign is set by
 * its voltage, so I takes the sign of the path's orientation: as in the reference's
 * port files, orient it so that V / I is positive.  OPEM_ERR_UNSUPPORTED for a
 * port driven by an analytic TE mode.                                          */
int  opem_problem_set_port_impedance(opem_problem prob, int port, int definition, int npath, const double* path,
                                     int closed);
/* A further mode of a port driven by its own 2D mode (after
 * opem_problem_set_port_fem2d; the reference's ports with several Mode blocks):
 * mode = 1..15, the mode-th mode of the same 2D problem in decreasing beta^2,
 * with its own voltage path (vpath: start xyz, end xyz) and impedance definition
 * (definition, npath, path, closed as for opem_problem_set_port_impedance).  It
 * adds one S-port and one driving set on the same faces: S-ports are every
 * port's first mode in port order, then the added modes in the order added;
 * *sport (may be NULL) receives its 0-based S-port index.  When another port
 * drives, a port with several modes absorbs with the gamma of largest magnitude
 * among them (Port::addPortIntegrators, port.cpp:5790-5806).  Such problems solve
 * on the FP64 path: mixed precision returns OPEM_ERR_UNSUPPORTED.  Setting the
 * port again (set_port_te / set_port_fem2d) removes its added modes.
 * OPEM_ERR_STATE when the port is not driven by its own 2D mode.               */
int  opem_problem_add_port_mode(opem_problem prob, int port, int mode, const double* vpath, int definition,
                                int npath, const double* path, int closed, int* sport);
/* Builds DOF numbering, CSR pattern, vertex patches, and assembles the frequency-
 * independent operators on the device.                                         */
int  opem_problem_assemble(opem_problem prob);
/* info[0]=ndofs, [1]=nnz, [2]=S-ports (ports plus added modes), [3]=npatches, [4]=max patch size, [5]=local dofs,
 * [6]=device bytes held, [7]=sum of patch sizes, [8]=sum of squared patch sizes
 * (entries of the block-Jacobi blocks).                                         */
int  opem_problem_info(opem_problem prob, int64_t* info, int ninfo);

/* ---- the per-frequency solve (fem3D::solve + calculateSplits + calculateS) ----
 * S_out: N*N complex (interleaved re,im), N = S-ports (info[2]), row = portOut,
 * col = portIn.  Zo_out: N complex (may be NULL).  stats may be NULL.           */
int  opem_solve_frequency(opem_problem prob, double freq, const opem_solver_opts* opts,
                          double* S_out, double* Zo_out, opem_solve_stats* stats);
/* A sweep: nfreq frequencies x all driving sets in one call (batched in mixed mode).
 * S_out: nfreq*nports*nports complex.  stats: nfreq entries (may be NULL).      */
int  opem_solve_sweep(opem_problem prob, int nfreq, const double* freqs, const opem_solver_opts* opts,
                      double* S_out, opem_solve_stats* stats);
/* Zienkiewicz-Zhu error indicator on the H fields of the last
 * opem_solve_frequency (fem3D::calculateMeshErrors, fem3D.cpp:1162-1420):
 * per element sqrt((int |Re(s - F)|)^2 + (int |Im(s - F)|)^2) with F = curl H / mu_r
 * and s its L2 projection onto the edge elements, the larger over the driving
 * sets (errors_out, ne doubles, may be NULL); marked_out receives up to
 * max_marked element indices of the floor(ne * fraction) (at least 1) largest
 * errors, largest first; *nmarked that count; *max_error the largest error.
 * OPEM_ERR_STATE before a solve.                                                 */
int  opem_mesh_errors(opem_problem prob, double fraction, double* errors_out, int64_t* marked_out,
                      int64_t max_marked, int64_t* nmarked, double* max_error);
/* E and H DOF vectors (ndofs complex each, interleaved) of the last single-frequency
 * solve for driving set d (0-based).  Either pointer may be NULL.               */
int  opem_get_fields(opem_problem prob, int d, double* e_out, double* h_out);

/* ---- operator-level access (parity tests; fem3D::build_A / build_P / build_Q)
 * which: 0=K(1/mu_r) 1=M(eps_r) 2=M(eps_r tand) 3=M(sigma) 4=M(1) 5=Q(1/mu_r)
 * rowptr: ndofs+1 int64, cols: nnz int32, vals: nnz doubles. Any may be NULL.   */
int  opem_get_operator(opem_problem prob, int which, int64_t* rowptr, int32_t* cols, double* vals);
/* Complex A(freq) for driving set d (before Dirichlet handling), nnz complex.   */
int  opem_get_system_matrix(opem_problem prob, double freq, int d, double* vals);

/* ---- measurement support (no reference counterpart) -------------------------
 * Kernel launches issued by this context so far.                                */
int  opem_context_launches(opem_context ctx, int64_t* out);
/* Times the hot kernels of the FP64 path in isolation on the context stream with
 * CUDA events (A(freq) for driving set 0): reps launches each.  out receives
 * 12 doubles: {ms per launch, algorithmic bytes per launch, launches}, for
 * kernels 0 = complex CSR SpMV, 1 = vertex-patch block apply, 2 = Gram-Schmidt
 * dot products against 64 Krylov vectors, 3 = the matching vector update.       */
int  opem_profile_kernels(opem_problem prob, double freq, int reps, double* out, int nout);
/* The same for the batched sweep solver's kernels, nsys (1..32) systems near
 * freq on driving set 0; out receives 15 doubles, kernels 0 = FP32 block apply
 * for nsys systems (the kernel the solver picks), 1 = batched SpMV with FP32
 * operators and vectors, 2 = FP64 operators and FP32 vectors, 3 = FP64 operators
 * and vectors, 4 = patch sum; with nout >= 21 also 5 = the FP32 FMA block apply
 * and 6 = the tensor-core block apply (ms = -1 where it does not apply).         */
int  opem_profile_batch_kernels(opem_problem prob, double freq, int nsys, int reps, double* out, int nout);
/* Checks the batched block apply (the preconditioner that replaces the
 * reference's direct PCLU, solveComplexLinearSystem.c:153-161): the FP32 block
 * set of driving set 0 at freq, nsys interleaved systems of deterministic
 * inputs, systems [r0, r0+nd) applied by the FP32 FMA kernel and by the
 * tensor-core kernel, both compared with an FP64 host product of the same FP32
 * blocks.  out (5 doubles): [0] max error of the tensor-core kernel relative to
 * the largest result (-1 if it does not apply), [1] the same for the FMA kernel,
 * [2] the kernel the solver uses for this case (2 tensor core, 1 FMA),
 * [3] max |tensor - FMA| relative, [4] 1 if a bounded wait ran out.            */
int  opem_check_block_apply(opem_problem prob, double freq, int nsys, int r0, int nd, double* out, int nout);

/* ---- OpenParEM3D project input (project.c, mesh.cpp:449-588, port.cpp:6369-7078,
 * OpenParEMmaterials.cpp) --------------------------------------------------------
 * Reads a .proj file with its gmsh 2.2 mesh (physical volumes named after
 * materials), ports file and materials databases, and creates the problem:
 * regions and materials, exterior faces classified into ports (closed
 * rectangular Path of each Port, ordered by Sport), Boundary blocks
 * (surface_impedance with the material's conductivity and Rz,
 * perfect_electric_conductor, perfect_magnetic_conductor, radiation) and PEC for
 * every other exterior face; each port is driven by the TE10 mode of its
 * rectangle (a = the wide side) with the voltage path of its Line block.  order
 * > 0 replaces mesh.order (orders 1-3 are built).  The frequency plan
 * (point, point.refine and linear entries, sorted, duplicates removed) goes to
 * freqs (up to max_freqs) and its length to *nfreq.                            */
int  opem_project_load(opem_context ctx, const char* proj_path, int order, opem_problem* out, int* nfreq,
                       double* freqs, int max_freqs);
/* The last value of a key of a .proj file ("refinement.relative.tolerance",
 * "mesh.3D.refinement.fraction", ...), "//" comment removed, into buf (len bytes
 * with the terminator); OPEM_ERR_ARG if the file or the key is missing.         */
int  opem_project_value(const char* proj_path, const char* key, char* buf, int len);
/* The same reading without a device (host only): info[0]=vertices, [1]=tets,
 * [2]=regions, [3]=exterior faces, [4]=port faces, [5]=Boundary-block faces,
 * [6]=PEC faces, [7]=ports, [8]=frequency points, [9]=order; msg receives the
 * reason when the project cannot be read (OPEM_ERR_ARG).                       */
int  opem_project_info(const char* proj_path, int order, int64_t* info, int ninfo, double* freqs, int max_freqs,
                       char* msg, int msg_len);
/* The problem arrays opem_project_load would pass to opem_problem_create and the
 * set_* calls, on the host: counts[8] = {vertices, tets, regions, exterior faces,
 * boundary attributes, ports, frequency points, order}; then (any may be NULL)
 * verts (3 per vertex), tets (4 per tet), region (per tet), region_mat
 * (eps_r, tan_d, sigma, mu_r per region), tris (3 per face), attr (per face,
 * 1-based), bdr_type and bdr_params (3 per attribute: port index | sigma, Rz,
 * mu_r | eta), port_desc (22 per port, as opem_problem_set_port_te), port_nsub
 * (per port: 0 = analytic TE10, n > 0 = its own 2D mode with faces split n x n
 * and 2D elements of the problem's order (n = 1: the reference's own 2D problem),
 * chosen for ports whose faces see more than one material or leave part of the
 * port polygon uncovered, ports that are not rectangles and ports whose impedance
 * definition uses the current), freqs.
 * Call once with only counts to size the buffers.                              */
int  opem_project_read(const char* proj_path, int order, int64_t* counts, double* verts, int64_t* tets,
                       int32_t* region, double* region_mat, int64_t* tris, int32_t* attr, int32_t* bdr_type,
                       double* bdr_params, double* port_desc, int32_t* port_nsub, double* freqs, char* msg,
                       int msg_len);

/* Impedance definition of port `port` of a project as the reader takes it
 * (host only): definition OPEM_Z_PV / VI / PI, the current path's point count
 * and up to cap of its points (xyz), closed = 1 when the path is closed.       */
int  opem_project_port_impedance(const char* proj_path, int port, int* definition, int* closed, int* npath,
                                 double* path, int cap, char* msg, int msg_len);

/* ---- port eigenmode of a cross-section (host only; the modal problem the
 * reference hands to OpenParEM2D, port.cpp:5081-5176) ----------------------------
 * Fundamental mode of a guide with PEC walls on a triangle mesh: nodes xy
 * (2 doubles each), triangles (3 node indices each), per-triangle complex eps_r
 * and mu_r (interleaved re, im; mu_r may be NULL for 1).  Lowest-order edge
 * elements for e_t, linear nodal elements for e_z.  beta_out = beta (complex,
 * exp(-j beta z)).  Edges are the sorted vertex pairs in lexicographic order,
 * oriented from the lower to the higher node index; *nedges is their count
 * (call with edges_out, et_out and ez_out all NULL to query it).  et_out: edge
 * coefficients (2 doubles each), scaled so the largest is 1; ez_out: nodal e_z
 * (2 doubles each).  OPEM_ERR_NOT_CONVERGED if inverse iteration stalls.       */
int  opem_port_mode_2d(int64_t nnodes, const double* xy, int64_t ntri, const int64_t* tris, const double* eps_r,
                       const double* mu_r, double freq, double* beta_out, int64_t* nedges, int64_t* edges_out,
                       double* et_out, double* ez_out);
/* The mode opem_problem_set_port_fem2d uses, on the host: port faces given as
 * vertex triples (face_verts, 3 per face, in the face's local vertex order) of
 * verts (3 doubles each), eps_face / mu_face complex per face (interleaved;
 * mu_face may be NULL), desc, nsub and order as for opem_problem_set_port_fem2d.
 * metrics = {gamma, Z, V, Pz} (4 complex, interleaved).  For npts points, each
 * given as a face (pt_face) and its parameters (pt_s: s1, s2 with
 * X = P0 + s1 (P1 - P0) + s2 (P2 - P0)), E_out and Hy_out (3 complex each, may
 * be NULL) receive E_t and H_t / y, y = gamma / (j w mu0 mu_r(face 0)).        */
int  opem_port_mode_faces(int64_t nverts, const double* verts, int64_t nface, const int64_t* face_verts,
                          const double* eps_face, const double* mu_face, const double* desc, int nsub, int order,
                          double freq, double* metrics, int64_t npts, const int64_t* pt_face, const double* pt_s,
                          double* E_out, double* Hy_out);
/* The same metrics under an impedance definition (as opem_problem_set_port_impedance),
 * of mode `mode` of the cross-section in decreasing beta^2 (0 = the fundamental
 * mode; 1..15 by subspace iteration with order-`order` elements of the reference's
 * 2D spaces): metrics = {gamma, Z, V, Pz, I} (5 complex; I = 0 without a current
 * path).                                                                        */
int  opem_port_mode_faces_z(int64_t nverts, const double* verts, int64_t nface, const int64_t* face_verts,
                            const double* eps_face, const double* mu_face, const double* desc, int nsub, int order,
                            double freq, int definition, int npath, const double* path, int closed, int mode,
                            double* metrics);

/* ---- S-parameter post-processing (host only, no GPU needed) -----------------
 * Renormalises S (nports x nports complex, interleaved, row = portOut) from the
 * port impedances Zo (nports complex, as opem_solve_frequency returns them) to
 * one reference impedance zref: Z = k (I+S)(I-S)^-1 k with k = diag(sqrt(Zo)),
 * S' = (Z/zref + I)^-1 (Z/zref - I)  (Result::renormalize, results.cpp:567-580).
 * OPEM_ERR_BREAKDOWN if I-S or Z/zref+I is singular.                            */
int  opem_s_renormalize(int nports, const double* S, const double* Zo, double zref_re, double zref_im,
                        double* S_out);
/* Writes a Touchstone 1.1 file (ResultDatabase::saveTouchstone, results.cpp:1055-1208):
 * nfreq points of renormalised S (layout as opem_solve_sweep returns), reference
 * impedance zref (ohm, > 0), format "RI" | "MA" | "DB", unit "Hz" | "kHz" | "MHz" | "GHz". */
int  opem_write_touchstone(const char* path, int nfreq, const double* freqs, int nports, const double* S,
                           double zref, const char* format, const char* unit);
/* Mixed-mode conversion of S already renormalised to zref (fem3D::build_Mc_Ms with
 * conversion 1, fem3D.cpp:1586-1900; Result::SparameterConversion, results.cpp:587-630):
 * npairs differential pairs, pairs = {P1, N1, P2, N2, ...} (1-based S-ports); S-port
 * P becomes the pair's common mode (Zo = zref/2), N its differential mode
 * (Zo = 2 zref).  Zo_out (nports complex, may be NULL) receives the new impedances.  */
int  opem_s_mixed_mode(int nports, const double* S, int npairs, const int* pairs, double zref, double* S_out,
                       double* Zo_out);
/* Modal to single-ended conversion (fem3D::build_Mc_Ms with conversion 0,
 * fem3D.cpp:1586-1900; Result::SparameterConversion, results.cpp:587-630): S the
 * modal S-parameters (nports x nports complex, row = portOut), Zmode the modes'
 * impedances (nports complex), Tv and Ti (nports x nports complex, row-major) the
 * maps from single-ended line voltages / currents to modal ones, each port's block
 * on the diagonal in S-port order (the Tv, Ti a multi-conductor port's 2D solve
 * gives).  S_out: single-ended S at zref on every S-port; Zo_out (may be NULL) = zref.
 * OPEM_ERR_BREAKDOWN if Tv, Ti or Ms + Mc S is singular.                         */
int  opem_s_single_ended(int nports, const double* S, const double* Zmode, const double* Tv, const double* Ti,
                         double zref, double* S_out, double* Zo_out);
/* Line-to-modal maps of one port with n lines and n modes, the reference's "line"
 * calculation (Mode::calculateModalCurrent / calculateModalVoltage,
 * OpenParEM2D fem2D.cpp:1591-1790): I and V (n x n complex, row = mode, column =
 * line) the modes' currents on the lines' current paths and voltages on their
 * voltage paths (V may be NULL).  Ti[i][k] = sign(Re I[i][k]) scaled by
 * 0.5 (|sum sign I| + |sum I|) / |sum sign I|; a mode whose Ti[i][0] is negative is
 * flipped (flipped[i] = 1: its field, currents and voltages change sign) and its
 * row negated; Tv = (conj(Ti)^-1)^T.  Im and Vm (n complex each, may be NULL) get
 * the mode currents sum_k Ti[i][k] I[i][k] and voltages sum_k Tv[i][k] V[i][k]
 * after the flips.  flipped may be NULL.  OPEM_ERR_BREAKDOWN if a mode carries no
 * net signed current or Ti is singular.                                          */
int  opem_port_line_maps(int n, const double* I, const double* V, double* Ti, double* Tv, int* flipped, double* Im,
                         double* Vm);
/* Touchstone 2.0 (the reference's mixed-mode writer, results.cpp:1210-1372): as
 * opem_write_touchstone plus the 2.0 keywords and, with pairs, [Mixed-Mode Order]. */
int  opem_write_touchstone2(const char* path, int nfreq, const double* freqs, int nports, const double* S,
                            double zref, const char* format, const char* unit, int npairs, const int* pairs);
/* Results CSV in the reference's _results.csv layout (ResultDatabase::saveCSV,
 * results.cpp:940-1052): header keys, one "#S-port" line per port (zref <= 0:
 * "not renormalized"), S(row;col) values with the driven port (column) outer.  */
int  opem_write_results_csv(const char* path, int nfreq, const double* freqs, int nports, const double* S,
                            double zref, const char* format, const char* unit);
/* The reference's regression comparator (process3D, process3D.cpp:105-560): the
 * S-parameter test cases of test_cases_path (magS(dB) / argS(deg) with equal,
 * lessthan, greaterthan) evaluated against a results CSV, written to out_path in
 * the _test_results.csv layout and order; *ncases and *npassed (may be NULL).
 * OPEM_ERR_ARG for unreadable or malformed files, OPEM_ERR_UNSUPPORTED for
 * antenna-metric cases.                                                          */
int  opem_evaluate_test_cases(const char* test_cases_path, const char* results_csv_path, const char* out_path,
                              int* ncases, int* npassed);
/* Largest column 2-norm of S_cur^-1 (S_prev - S_cur): the reference's change of S
 * between adaptive passes (ResultDatabase::calculate_maxRelativeError,
 * results.cpp:714-768), compared with refinement.relative.tolerance.            */
int  opem_s_relative_change(int nports, const double* S_prev, const double* S_cur, double* out);

/* ---- mesh refinement (host only) ---------------------------------------------
 * Conforming refinement of the marked tetrahedra (the reference refines what its
 * error indicator marks with MFEM GeneralRefinement, fem3D::refineMesh,
 * fem3D.cpp:1426-1447): each marked tetrahedron is bisected at its longest edge
 * and the mesh closed by longest-edge bisection; regions and boundary attributes
 * carry over, boundary triangles are split to match.  counts = {vertices, tets,
 * boundary triangles} of the refined mesh; the output arrays may be NULL (size
 * query).  OPEM_ERR_MESH if a boundary triangle is not a face of the mesh.      */
int  opem_refine_mesh(int64_t nverts, const double* verts, int64_t ntets, const int64_t* tets,
                      const int32_t* region, int64_t nbdr, const int64_t* bdr_tris, const int32_t* bdr_attr,
                      int64_t nmarked, const int64_t* marked, int64_t* counts, double* verts_out,
                      int64_t* tets_out, int32_t* region_out, int64_t* bdr_out, int32_t* attr_out);

/* ---- serving loop (no counterpart in the reference: it solves one project per
 * process, OpenParEM3D.cpp:494-555) -------------------------------------------
 * A server runs solve requests from any number of caller threads on one GPU.
 * It has `slots` slot contexts (each with its own CUDA stream), so up to that
 * many requests run at once and their kernels overlap on the device.  A queued
 * request starts when a slot is free and its estimated device footprint fits
 * in hbm_budget_bytes minus the footprints of the running requests (<= 0: 90 %
 * of the free device memory at creation); it always starts when nothing runs.
 * The queue is scanned in arrival order and the first request that fits starts;
 * requests on the same problem run one after another.  Operators stay resident:
 * a problem is assembled by its first request (if the caller has not) and kept.
 * A submitted problem belongs to the server until opem_server_wait has returned
 * its request: the caller must not use or destroy it meanwhile.  Each result is
 * the same as the same request run alone (every kernel reads only its own
 * request's data; reductions are deterministic).                               */
typedef struct opem_server_s* opem_server;
int  opem_server_create(int device, int slots, int64_t hbm_budget_bytes, opem_server* out);
/* Waits for running requests; queued ones are dropped (their wait would fail).  */
int  opem_server_destroy(opem_server srv);
/* Queues nfreq frequency points of prob (the same result layout as
 * opem_solve_sweep); returns at once with the request id.                      */
int  opem_server_submit(opem_server srv, opem_problem prob, int nfreq, const double* freqs,
                        const opem_solver_opts* opts, int64_t* request_id);
/* Blocks until the request is done (timeout_s < 0: no limit; OPEM_ERR_TIMEOUT if
 * it is still queued or running when timeout_s runs out, and it can be waited
 * for again).  Then S_out (nfreq*nports*nports complex), stats (nfreq) and
 * times_out[3] = {submitted, started, finished} in seconds since the server
 * was created are filled (any may be NULL) and the request's status returned.  */
int  opem_server_wait(opem_server srv, int64_t request_id, double timeout_s, double* S_out,
                      opem_solve_stats* stats, double* times_out);
/* Cancels a request: a queued one is dropped at once, a running one stops at its
 * next Krylov step (the solvers poll a per-problem flag between steps); either way
 * its wait returns OPEM_ERR_CANCELLED.  OPEM_ERR_ARG for an unknown id, OPEM_OK
 * if the request had already finished (its result stands).                     */
int  opem_server_cancel(opem_server srv, int64_t request_id);
/* info[0]=queued, [1]=running, [2]=completed, [3]=admitted bytes, [4]=budget, [5]=slots. */
int  opem_server_info(opem_server srv, int64_t* info, int ninfo);

/* ---- failure-detection self-test (no reference counterpart) -----------------
 * Launches one kernel whose bounded mbarrier wait (the wait the batched block
 * apply uses for its bulk copies) is made to run out: it waits for a barrier
 * phase that nothing completes, gives up after `polls` polls (1..2^24), records
 * the timeout in a device status word and returns.  Returns OPEM_ERR_TIMEOUT
 * when the status word reported the timeout and the context still runs a
 * kernel afterwards, another status otherwise.                                   */
int  opem_selftest_wait_timeout(opem_context ctx, int polls);
/* Host check of the device Hessenberg least squares (no device needed): the
 * column update and back substitution the solvers run on the GPU, compiled for
 * the host, against the host Givens QR on seeded random problems of m columns,
 * a fresh cycle and one started from a deflated (kd+1) x kd block.
 * max_rel_diff: largest relative difference of residual estimates and y.     */
int  opem_selftest_lsq(int m, int kd, int seed, double* max_rel_diff);
/* Host copy of the face tables the boundary assembly uploads (no device
 * needed): for the order-p reference tetrahedron and each local face f = 0..3,
 * the tangential mass tables (t1 t1, t2 t2, t1 t2 + t2 t1; ldf x ldf each, ldf =
 * p (p + 2)) integrated exactly (nodal = 0) or with the port integrals' nodal
 * rule (nodal = 1: the rule of MFEM's order-p L2 triangle, which the overlaps of
 * ports driven by their own 2D modes use).  out: 4 * 3 * ldf * ldf doubles;
 * OPEM_ERR_ARG when nout is smaller or p is outside 1..8.                       */
int  opem_selftest_face_tables(int p, int nodal, double* out, int64_t nout);

/* ---- allocation-free assembly (no counterpart in the reference) -------------
 * For callers that cannot allocate device memory at the point of use: a
 * process whose HBM is already claimed by another allocator (a PETSc or Kokkos
 * memory pool, or a serving process that reserves its whole budget up front)
 * or a latency-critical loop that must not call cudaMalloc/cudaFree.  Like
 * opem_get_system_matrix it writes A(freq) for driving set d (before Dirichlet
 * handling, nnz complex, interleaved) into the host buffer vals, but it stages
 * the values in a static device array of OPEM_NOALLOC_MAX_NNZ complex doubles
 * (16 MiB, held by every GPU that loads the library until the process exits)
 * and calls no cudaMalloc, cudaFree or allocating library routine.
 *  - Problems with nnz > OPEM_NOALLOC_MAX_NNZ are rejected with OPEM_ERR_ARG.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress); make that first call before any stream capture.
 *  - All calls on a device share the one array: calls that overlap on the GPU
 *    (other host threads, other problems on the same device) race.  Each call
 *    overwrites every entry it reads, so nothing has to be cleared between calls. */
#define OPEM_NOALLOC_MAX_NNZ (1 << 20)
int  opem_system_matrix_noalloc(opem_problem prob, double freq, int d, double* vals);

#ifdef __cplusplus
}
#endif
#endif /* OPEM_B200_H */
