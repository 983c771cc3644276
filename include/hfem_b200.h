/*
 * hfem_b200: C ABI of the B200 (sm_100a) HDG element hot path.
 *
 * Drop-in for the serial hot path of exapde/hfem (the reference).  The
 * reference composes this path at compile/link time rather than through a
 * plugin ABI; each entry point below names the reference routine it replaces.
 * All arrays use the reference's layouts (column-major; element-major arrays
 * are npv x nc x ne etc.), all integers are 0-based int32, all reals float64.
 * Host pointers are only read/written during the call; device buffers belong
 * to the context.  Every call returns 0 on success or a negative HFEM_E_* code;
 * hfem_last_error() gives the message.  Nothing calls exit().
 */
#ifndef HFEM_B200_H
#define HFEM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hfem_ctx hfem_ctx;

enum {
    HFEM_OK = 0,
    HFEM_E_ARG = -1,         /* invalid argument or size */
    HFEM_E_UNSUPPORTED = -2, /* element shape / order without a compiled kernel */
    HFEM_E_CUDA = -3,        /* CUDA runtime error */
    HFEM_E_STATE = -4,       /* call made before the data it needs was set */
    HFEM_E_MESH = -5,        /* connectivity inconsistent (missing CSR block, bad index) */
    HFEM_E_SINGULAR = -6,    /* singular local matrix */
    HFEM_E_NOMEM = -7        /* device allocation failed */
};

/* Sizes of one problem: element (nd, npv nodes, npf nodes per face, nfe faces,
 * ngv volume and ngf face quadrature points) and mesh (ne elements, nf faces,
 * nblocks = entries of the face-to-face block CSR). */
typedef struct {
    int nd, npv, npf, nfe, ngv, ngf;
    int ne, nf, nblocks;
} hfem_dims;

/* Context on CUDA device `device`.  Replaces the struct set-up of
 * preprocessing/initializestructs.cpp:45-930 (initializeStructs). */
int hfem_create(const hfem_dims* dims, int device, hfem_ctx** out);
int hfem_destroy(hfem_ctx* ctx);
const char* hfem_last_error(const hfem_ctx* ctx);

/* Work on an existing CUDA stream (cudaStream_t passed as void*); NULL = the
 * context's own stream. */
int hfem_set_stream(hfem_ctx* ctx, void* stream);

/* Master element tables, as masterstruct holds them
 * (preprocessing/digasopre.h:109-229, written by mkmasterelement.m):
 *   shapvt ngv x npv x (nd+1), shapvg npv x ngv x (nd+1),
 *   shapvgdotshapvl npv^2 x ngv x (nd+1), shapft ngf x npf x nd,
 *   shapfg npf x ngf x nd, shapfgdotshapfc npf^2 x ngf x nd, perm npf x nfe. */
int hfem_set_master(hfem_ctx* ctx, const double* shapvt, const double* shapvg, const double* shapvgdotshapvl,
                    const double* shapft, const double* shapfg, const double* shapfgdotshapfc, const int* perm);

/* Mesh (meshstruct, digasopre.h:231-300) and the face-block CSR (sysstruct
 * ent2entStart/ent2ent, diagonal block first in every row; produced by the
 * reference's dmdserial, preprocessing/preprocessing.cpp:14):
 *   dgnodes npv x nd x ne, elcon (npf*nfe) x ne, t2f nfe x ne,
 *   ent2entStart nf+1, ent2ent nblocks.
 * Checks the connectivity the reference asserts (globalassembly.cpp:69-75). */
int hfem_set_mesh(hfem_ctx* ctx, const double* dgnodes, const int* elcon, const int* t2f,
                  const int* ent2entStart, const int* ent2ent);

/* Boundary faces of a bounded mesh (mesh.bf, app.bcm, app.bcs of the
 * reference; faceint elementassembly.cpp:1075-1246 with fbouDriver): bf[ne x
 * nfe] element-major, >= 0 interior, -(ib + 1) on boundary ib; bcm[nbnd] the
 * boundary condition types (1 free-stream far field, 2 no-slip adiabatic
 * wall, 5 Dirichlet, 6 extrapolation, 7 slip wall, as
 * application/FM/fbou.cpp on a fixed mesh);
 * bcs[nbnd x nch] their states.  The trace equations of boundary faces take
 * the boundary flux.  Call after hfem_set_mesh (which clears it). */
int hfem_set_boundary(hfem_ctx* ctx, const int* bf, int nbnd, const int* bcm, const double* bcs);

/* The equations (app.appname of the reference, initializestructs.cpp:126):
 * 1 compressible Navier-Stokes (default), 0 Euler.  Euler keeps the
 * Navier-Stokes state layout (the q slots are carried but unused): the
 * inviscid flux does not depend on q, so the element matrices equal those of
 * the reference's q-free Euler discretisation (flag_q 0, nc = ncu). */
int hfem_set_app(hfem_ctx* ctx, int appname);

/* The trace-flux stabilization tensor and the viscosity model (app.convStabMethod
 * and app.viscosityModel, initializestructs.cpp:131,134; digasopre.h:84,88).
 * conv_stab: 0 constant tau = physicsparam[5] (default), 1 Lax-Friedrichs,
 * 2 Roe (application/FM/stabilizationTensor.cpp); viscosity_model: 0 constant
 * (default), 1 Sutherland's law (application/FM/getViscosity.c).  The
 * no-slip wall's energy row takes the same tensor (its fhat), the Dirichlet
 * condition keeps physicsparam[5] as the reference's fbou does.  Other values:
 * HFEM_E_UNSUPPORTED. */
int hfem_set_models(hfem_ctx* ctx, int conv_stab, int viscosity_model);

/* Physics: physicsparam = [gamma, eps, Re, Pr, Mach, tau] (compressible
 * Navier-Stokes), tdep/fc_u/fc_q/time as appstruct (digasopre.h:7-91); the
 * equations are chosen by hfem_set_app, the stabilization and viscosity by
 * hfem_set_models. */
int hfem_set_physics(hfem_ctx* ctx, const double* physicsparam, int tdep, double fc_u, double fc_q, double time);

/* Solution state sol.UDG (npv x nc x ne), sol.UH (nch x nf*npf) and the time
 * source sol.SH (npv x nc x ne; may be NULL = zero).  Host pointers. */
int hfem_set_solution(hfem_ctx* ctx, const double* udg, const double* uh, const double* sh);
int hfem_get_solution(hfem_ctx* ctx, double* udg, double* uh);
/* Same, with device pointers already on the context's device. */
int hfem_set_solution_device(hfem_ctx* ctx, const double* udg, const double* uh, const double* sh);

/* hfem_set_solution followed by hfem_assemble, with the copies overlapped: uh
 * first, then udg and sh in `chunks` pieces of elements on a second stream; the
 * element kernel of each piece starts as soon as that piece has arrived (the
 * host arrays should be pinned for the copies to run asynchronously).  Same
 * results as the two calls.  No counterpart in the reference (its state is
 * already in host memory). */
int hfem_assemble_host(hfem_ctx* ctx, const double* udg, const double* uh, const double* sh, int chunks,
                       double* rnorm);

/* q from (u, uh) on every element.  Replaces getQ
 * (assembly/elementassembly.cpp:1414-1479) as called by solveProblem
 * (solvers/dgsolvers.cpp:464-474). */
int hfem_getq(hfem_ctx* ctx);

/* Element assembly, static condensation and scatter into the face-block
 * system Hg x = Rg; stores D^-1 Ru and D^-1 F per element.  Replaces
 * assembleLinearSystem (assembly/globalassembly.cpp:423-556) with
 * assembleElementMatrixVector (elementassembly.cpp:1481-1499),
 * schurElementMatrixVector (elementschur.cpp:331-343) and
 * mapElement2LinearSystem (globalassembly.cpp:8-161).  rnorm (may be NULL)
 * receives sqrt(sum ||Ru_e||^2 + ||sum Rh_e||^2) as sol.rNorm. */
int hfem_assemble(hfem_ctx* ctx, double* rnorm);

/* Residual norm only.  Replaces computeResidualNorm (globalassembly.cpp:618-678). */
int hfem_residual(hfem_ctx* ctx, double* rnorm);

/* Restarted GMRES on Hg x = Rg (x starts at 0), left preconditioning:
 * precond -1 none, 0 block ILU(0) in the minimum-discarded-fill order
 * (kernel/computeMDFordering.m, computeBILU0.m, applyBILU0.m; the ordering is
 * computed from the first system the context solves and kept, as the
 * reference's reuseOrdering does), 2 entity-wise block Jacobi
 * (kernel/mkBlockJacobi.m).
 * Replaces computeOrdering / computePreconditioner / gmres
 * (solvers/dgsolvers.cpp:16-20, closed in the reference; spec
 * kernel/gmres_bilu0.m).  conv: 1 converged, 0 max iterations, -1 breakdown.
 * hist (may be NULL) receives up to hist_len relative residuals. */
int hfem_gmres(hfem_ctx* ctx, int precond, int restart, double tol, int maxit, int* conv, int* iters,
               double* hist, int hist_len);

/* uh += alpha x; u += alpha (D^-1 Ru - D^-1 F x_e); q recomputed.
 * Replaces updateSol / getU (solvers/solutionupdate.cpp:6-98). */
int hfem_update(hfem_ctx* ctx, double alpha);

/* Damped Newton with line search on the assembled system.  Replaces
 * solveNonlinearProblem (solvers/dgsolvers.cpp:106-205).  rnorm_hist
 * receives the residual before each iteration and the final one
 * (up to hist_len entries); *niter the number of iterations. */
int hfem_newton(hfem_ctx* ctx, double newton_tol, int newton_maxiter, int precond, int restart, double gmres_tol,
                int gmres_maxit, double* rnorm_hist, int hist_len, int* niter, int* converged);

/* One DIRK(stages, order) time step of size dt (stages 1-3; (1,1) (1,2) (2,2)
 * (2,3) (3,3) as solvers/DIRKcoeff.cpp), each stage solved by hfem_newton.
 * Replaces one iteration of solveUnsteadyProblem (solvers/dgsolvers.cpp:221-444);
 * the context's time advances by dt.  *newton_iters (may be NULL) receives the
 * Newton iterations of all stages. */
int hfem_dirk_step(hfem_ctx* ctx, double dt, int stages, int order, double newton_tol, int newton_maxiter,
                   int precond, int restart, double gmres_tol, int gmres_maxit, int* newton_iters);

/* Arithmetic of the assembly and solve (no counterpart in the reference, which
 * is FP64 throughout).  mode 0: FP64 everywhere (default).  mode 1: the
 * element contractions (volume D = Y'Phi, F = Y'Psi and the face K, H rows)
 * in 3xTF32 split precision on the tensor cores with FP32 accumulation, the
 * two Schur GEMMs (D^-1 F and H - K D^-1 F) on the tcgen05 tensor cores in
 * TF32 with FP32 accumulation, and the preconditioner applied with FP32 factors
 * (block-Jacobi inverses, BILU0 factors).  mode 2: only the preconditioner in
 * FP32 (the Jacobian FP64, so Newton converges as in mode 0 while GMRES
 * applies FP32 factors).  mode 3: the 3xTF32 element contractions and the FP32
 * preconditioner, the Schur GEMMs in FP64 (Jacobian blocks good to about 1e-6
 * relative, so Newton keeps its FP64 iteration count).  In every mode the
 * element LU, the residuals (rnorm), the Arnoldi process and the Newton update
 * stay FP64, so Newton iterations refine the solution to the FP64 residual
 * tolerance. */
int hfem_set_precision(hfem_ctx* ctx, int mode);

/* y = Hg x with device pointers x, y (nf*bsz doubles each, on the context's
 * device), after an assembly; the matvec of GMRES without a preconditioner.
 * hfem_set_step makes duh (device, nf*bsz) the step that hfem_update applies,
 * in place of the last GMRES solution.  For drivers that run their own Krylov
 * method around the assembled system, e.g. the domain-decomposed GMRES of
 * several GPUs (matvec of the local rows, then a sum over the part
 * interfaces; solvers/pDLAK.cpp:322-357 in the reference's MPI path). */
int hfem_matvec(hfem_ctx* ctx, const double* x, double* y);
int hfem_set_step(hfem_ctx* ctx, const double* duh);

/* The BILU0 ordering in use: ordered2unordered[i] = face pivoted at step i
 * (sys.ordered2unordered of the reference).  hfem_reset_ordering makes the
 * next BILU0 solve recompute it from the current system. */
int hfem_get_ordering(hfem_ctx* ctx, int* ordered2unordered);
int hfem_reset_ordering(hfem_ctx* ctx);

/* Device memory of contexts is drawn from a per-process pool of size-class
 * blocks; a destroyed context's blocks stay cached for the next context (no
 * cudaMalloc/cudaFree, which synchronise the device, when contexts are built
 * and dropped repeatedly).  hfem_pool_trim frees the cached blocks and returns
 * how many; hfem_pool_cached_bytes reports their total.  No counterpart in
 * the reference. */
int hfem_pool_trim(void);
long long hfem_pool_cached_bytes(void);

/* Device address and length (doubles) of one of the context's buffers, with
 * the ids of hfem_download plus 8 = UDG and 9 = UH (the resident state, which
 * a caller may also write), for zero-copy use on the device after the
 * context's stream has been synchronised (done here).  The buffer belongs to
 * the context and moves when the context reallocates it.  No counterpart in
 * the reference (its arrays live in host structs). */
int hfem_device_buffer(hfem_ctx* ctx, int what, const double** ptr, size_t* count);

/* Assembly split in two for graph capture: hfem_assemble_async only enqueues
 * the kernels of hfem_assemble on the context's stream (buffers are
 * allocated first if needed); hfem_assemble_finish waits, checks the element
 * LUs and returns the residual norm.  Together they equal hfem_assemble. */
int hfem_assemble_async(hfem_ctx* ctx);
int hfem_assemble_finish(hfem_ctx* ctx, double* rnorm);

/* Batched-GEMM tilings compiled into the library (any is valid for any
 * shape); hfem_autotune times them all on the context's own operands and
 * keeps the fastest for D^-1 F and for H - K D^-1 F, or the fused kernel that
 * does both (best = {-1, -1}) when it is faster than that pair (best[2],
 * ms[2 * count] may be NULL; ms holds the pairs' timings);
 * hfem_set_gemm_tiles applies a stored choice (-1, -1: the fused kernel).
 * No counterpart in the reference (its BLAS picks its own kernels). */
int hfem_gemm_candidates(void);
int hfem_autotune(hfem_ctx* ctx, int reps, int* best, double* ms);
int hfem_set_gemm_tiles(hfem_ctx* ctx, int gemm_dinvf, int gemm_schur);

/* One CUDA graph replaying the assembly (hfem_assemble_async) of n contexts
 * on the same device, each context on its own branch; launch it on any
 * stream and call hfem_assemble_finish on each context afterwards.  The
 * contexts must not be reallocated (new mesh, larger restart) while the
 * graph is alive.  No counterpart in the reference. */
typedef struct hfem_graph hfem_graph;
int hfem_graph_capture(hfem_ctx** ctxs, int n, void* stream, hfem_graph** graph);
int hfem_graph_launch(hfem_graph* graph, void* stream);
int hfem_graph_destroy(hfem_graph* graph);

/* Several independent problems in one context (a disjoint union of meshes, so
 * element work of many requests runs in one launch; no counterpart in the
 * reference, which runs one problem per process).  eprob (ne) and fprob (nf)
 * map elements and faces to problems; params holds per problem
 * [gamma, eps, Re, Pr, Mach, tau, tdep, fc_u]. */
int hfem_set_problem_map(hfem_ctx* ctx, int nprob, const int* eprob, const int* fprob, const double* params);
/* Residual norm of each problem after hfem_assemble / hfem_residual
 * (computeResidualNorm restricted to the problem's elements and faces). */
int hfem_problem_rnorms(hfem_ctx* ctx, double* rnorm);
/* updateSol with one step length per problem (alpha[nprob], host). */
int hfem_update_problems(hfem_ctx* ctx, const double* alpha);
/* GMRES for every problem of the context at once: the algorithm of hfem_gmres
 * (kernel/gmres_bilu0.m:17-105) run per problem, with each problem's own
 * Krylov basis, Hessenberg matrix and stopping test, sharing the launches.
 * Needs a problem map whose fprob is non-decreasing with every problem owning
 * a face.  conv[nprob] and iters[nprob] as in hfem_gmres. */
int hfem_gmres_problems(hfem_ctx* ctx, int precond, int restart, double tol, int maxit, int* conv, int* iters);

/* Download device results for inspection (host buffers of the given length):
 * what = 0 Hg (nblocks*bsz^2), 1 Rg (nf*bsz), 2 Rr = sum of uncondensed Rh
 * (nf*bsz), 3 DinvRu (n*ne), 4 DinvF (n*nb*ne), 5 condensed element H
 * (nb*nb*ne), 6 condensed element Rh (nb*ne), 7 GMRES solution x (nf*bsz),
 * 10 element K (nb*n*ne), 12 element Rh before condensation (nb*ne),
 * 13 element D^-1 after an
 * assembly (n*n*ne; D itself after a residual-only pass), 14 ||Ru_e||^2 before
 * condensation (ne). */
int hfem_download(hfem_ctx* ctx, int what, double* host, size_t count);

/* Per-kernel device time (ms) accumulated since the last reset, when timing
 * is on (measurement helper, no counterpart in the reference).  names
 * receives a ';'-separated list matching ms[]; returns the number of kernels. */
int hfem_set_timing(hfem_ctx* ctx, int on);
int hfem_kernel_times(hfem_ctx* ctx, char* names, size_t names_len, double* ms, int* counts, int max_kernels);

/* Measurement helper (no counterpart in the reference): FP64 FMA throughput of
 * `device` in TFLOP/s from a burst kernel, the compute roof of this FP64 path. */
int hfem_fp64_peak(int device, double* tflops);

/* Element assembly + static condensation that allocates nothing (no
 * counterpart in the reference).  For callers that cannot call cudaMalloc:
 * programs whose device memory comes from their own caching pool (PyTorch,
 * RMM), where a raw cudaMalloc would synchronise the device and fragment the
 * pool, and serving loops that reserve HBM once and must not allocate per
 * request.  It runs the same kernels as hfem_assemble's element pass, so its
 * blocks equal that path's.  Every pointer except physicsparam (6 doubles,
 * host) is device memory on the calling thread's current device, under that
 * device's primary context (the one the CUDA runtime and PyTorch use).  The
 * caller passes all inputs -- master tables, dgnodes, elcon, udg with q, uh, sh
 * and, for a bounded mesh, bf (ne x nfe, element-major, < 0 on boundary
 * -(ib + 1)), bcm (condition types 1, 2, 5, 6 or 7 per boundary) and bcs
 * (nch states per boundary) as hfem_set_boundary takes them (bf = NULL: no
 * boundary faces); appname 1 Navier-Stokes, 0 Euler (constant tau =
 * physicsparam[5] and constant viscosity: the models of hfem_set_models are
 * not taken here) -- and all outputs, per
 * element: D (n^2; receives D^-1), DinvF (n*nb), K (nb*n), H (nb^2,
 * condensed), DinvRu (n), Rh (nb, condensed), Rh_uncondensed (nb), ru2
 * (||Ru||^2 before condensation), info (0, or 1 + pivot step of a singular D).
 * The element workspace comes from one fixed 32 MiB device array that every
 * GPU loading the library holds until exit; it bounds the element kernel's
 * grid (large element shapes run on fewer CTAs), and shapes whose per-CTA
 * workspace exceeds it are rejected with HFEM_E_ARG.  The first call on a
 * device looks up that array's address (cudaGetSymbolAddress) and sets the
 * kernels' launch attributes; make that first call before any stream capture.
 * All calls share the array and nothing in it needs to start at zero; calls
 * that overlap on the GPU (different streams or threads at once) race on it.
 * Launches on `stream` (cudaStream_t, NULL = legacy default stream) and
 * returns without synchronising. */
int hfem_condense_noalloc(const hfem_dims* dims, const double* shapvt, const double* shapvg,
                          const double* shapvgdotshapvl, const double* shapft, const double* shapfg,
                          const double* shapfgdotshapfc, const int* perm, const double* dgnodes, const int* elcon,
                          const double* udg, const double* uh, const double* sh, const double* physicsparam,
                          int tdep, double fc_u, double fc_q, const int* bf, const int* bcm, const double* bcs,
                          int appname, double* D, double* DinvF, double* K, double* H, double* DinvRu, double* Rh,
                          double* Rh_uncondensed, double* ru2, int* info, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HFEM_B200_H */
