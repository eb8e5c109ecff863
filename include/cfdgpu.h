/*
 * cfdgpu.h -- C ABI of the B200 (sm_100a) time-step library for stabilised
 * linear-element incompressible Navier-Stokes (quad4/tri3/hex8/tet4).
 *
 * The library replaces, behind plain pointers and sizes, the per-time-step
 * body of the cfdsfemmpi solver:
 *   - the element loop + PETSc assembly of StabFEM::solveFullyImplicit
 *     (src/base/StabFEM2.cpp:654-740) and the element virtual
 *     ElementBase::calcStiffnessAndResidual (src/base/ElementBase.h:87),
 *   - the SolverPetsc object (src/base/SolverPetsc.h:15-64: initialise,
 *     zeroMtx, assembleMatrixAndVectorSerial, factoriseAndSolve),
 *   - SolutionData's per-step vector algebra (src/base/SolutionData.cpp:64-91).
 * The caller keeps the reference's driver (time loop, ramp, output) and calls
 * cfdgpu_step once per time step.
 *
 * Conventions: every function returns 0 on success or a negative CFDGPU_E*
 * code; cfdgpu_last_error(h) describes the last failure on a handle.  No
 * function calls exit().  One handle per host thread; a handle owns one CUDA
 * stream and all of its device memory.  Full nodal vectors use the
 * reference's layout: index node*ndof + dof, ndof = ndim + 1 (u, v[, w], p).
 */
#ifndef CFDGPU_H
#define CFDGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define CFDGPU_OK 0
#define CFDGPU_EINVAL (-1)      /* bad argument or wrong state (SolverPetsc.cpp:205-209) */
#define CFDGPU_ECUDA (-2)       /* CUDA runtime error */
#define CFDGPU_ENEGJAC (-3)     /* negative Jacobian (reference exits, e.g. Hexa8Node.cpp:79-84) */
#define CFDGPU_EKSP (-4)        /* linear solve diverged (reference exits, SolverPetsc.cpp:264-269) */
#define CFDGPU_ENOMEM (-5)
#define CFDGPU_ENODEV (-6)      /* no CUDA device / kernels not loadable */
#define CFDGPU_ETOOBIG (-7)     /* size beyond the fixed scratch of an allocation-free entry point */

/* element types, as selected in StabFEM::prepareInputData (StabFEM.cpp:351-366) */
#define CFDGPU_TRI3 0
#define CFDGPU_QUAD4 1
#define CFDGPU_TET4 2
#define CFDGPU_HEX8 3

/* preconditioners (PETSc -pc_type names) */
#define CFDGPU_PC_NONE 0
#define CFDGPU_PC_JACOBI 1      /* inverse of the scalar diagonal */
#define CFDGPU_PC_PBJACOBI 2    /* inverse of each node's ndof x ndof diagonal block */
#define CFDGPU_PC_BJACOBI_ILU 3 /* -pc_type bjacobi -sub_pc_type ilu -sub_pc_factor_levels k
                                   (input/petsc_options_gmres.dat:2-5): block Jacobi over
                                   bjacobi_blocks contiguous node ranges, block ILU(ilu_levels)
                                   in natural order inside each range; one range = -pc_type ilu */

/* Krylov methods (PETSc -ksp_type names) */
#define CFDGPU_KSP_GMRES 0      /* KSPGMRES: classical Gram-Schmidt, left preconditioning */
#define CFDGPU_KSP_BCGS 1       /* KSPBCGS (input/petsc_options_bcgs.dat:1): BiCGStab, left preconditioning */
#define CFDGPU_KSP_PREONLY 2    /* KSPPREONLY: x = M^-1 b, one preconditioner application; with the complete
                                   factorisation (ilu_levels = -1, one block) a direct solve, as the
                                   reference's tests ask (testdata/ldc2dquad10/petsc_options.dat:1-2) */

/* precision modes */
#define CFDGPU_PREC_FP64 0      /* FP64 element kernels, matrix and Krylov solve */
#define CFDGPU_PREC_MIXED 1     /* FP64 flexible GMRES (FP64 matrix, basis, Hessenberg, residual) whose
                                   preconditioner is an FP32 BiCGStab inner solve on an FP32 copy of the
                                   tangent with the FP32 form of pc_type */

/* Mesh: borrowed host arrays, copied at create (StabFEM::readInputData,
 * StabFEM.cpp:80-264).  conn is 0-based, nElem*npElem; DBC entries are
 * 0-based (node, dof, value) triples. */
typedef struct cfdgpu_mesh {
  int ndim;
  int npElem;
  int nNode;
  int nElem;
  const double *coords;     /* nNode*ndim */
  const int32_t *conn;      /* nElem*npElem */
  int nDBC;
  const int32_t *dbc_node;
  const int32_t *dbc_dof;
  const double *dbc_value;
} cfdgpu_mesh;

/* Control parameters (StabFEM::readControlParameters, StabFEM.cpp:268-322)
 * plus the Newton settings the reference hard-codes (StabFEM2.cpp:654,749). */
typedef struct cfdgpu_control {
  double rho, mu;
  double bodyforce[3];      /* read but unused by the active elements */
  double stab[3];           /* SUPG, PSPG, LSIC factors (elemData[8..10]) */
  int tis;
  double rhoInf;
  double dt;
  double newton_tol;        /* absolute residual 2-norm, reference: 1e-8 */
  int newton_max_iter;      /* reference: 10 */
} cfdgpu_control;

/* Krylov options (PETSc option semantics: -ksp_gmres_restart, -ksp_rtol,
 * -ksp_atol, -ksp_divtol, -ksp_max_it, -pc_type). */
typedef struct cfdgpu_solver_opts {
  int restart;
  double rtol, atol, dtol;
  int max_it;
  int pc_type;
  int precision;            /* CFDGPU_PREC_* */
  int inner_restart;        /* mixed mode: FP32 BiCGStab iterations per outer flexible-GMRES step (0: 20) */
  double inner_rtol;        /* mixed mode: inner relative tolerance of those iterations (0: 1e-2) */
  int reuse_tangent;        /* 1: assemble K once per step, residual-only after (exact for this formulation) */
  double refine_rtol;       /* mixed mode: outer target ||b - A x|| <= max(refine_rtol ||b||, F) on the FP64
                               matrix, F below (0: 1e-10); restart = outer restart */
  double newton_rtol;       /* extra relative Newton test ||F_k|| <= newton_rtol ||F_0||, F_0 the iteration-0
                               residual of the constant predictor (0: off, the reference's test only) */
  int formulation;          /* CFDGPU_FORM_*: element routine (0: the reference's active semi-implicit one) */
  int ksp_type;             /* CFDGPU_KSP_* (0: GMRES) */
  int ilu_levels;           /* CFDGPU_PC_BJACOBI_ILU: level of fill k (-sub_pc_factor_levels, 0..16); -1 keeps
                               all fill: the complete block LU of each block (-pc_type lu, natural ordering) */
  int bjacobi_blocks;       /* CFDGPU_PC_BJACOBI_ILU: number of blocks (0 or 1: one block, as a serial run) */
  double refine_atol;       /* mixed mode: absolute floor F of the outer target max(refine_rtol ||b||, F)
                               (0: T/10, T the step's Newton target; < 0: no floor) */
} cfdgpu_solver_opts;

/* element formulations */
#define CFDGPU_FORM_SEMI_IMPLICIT 0   /* active "semi-implicit type B" routines; tangent reusable in a step */
#define CFDGPU_FORM_FULLY_IMPLICIT 1  /* the reference's commented-out fully-implicit routines (SUPG+PSPG, LSIC in
                                         3D, full Newton tangent); reuse_tangent is ignored */

#define CFDGPU_MAX_NEWTON 32

typedef struct cfdgpu_step_stats {
  int newton_iters;                     /* assemblies done (including the converged check) */
  int converged;                        /* residual < newton_tol within the cap */
  double norms[CFDGPU_MAX_NEWTON];      /* residual 2-norm per Newton iteration */
  int ksp_its[CFDGPU_MAX_NEWTON];       /* Krylov iterations per solve */
  int ksp_reason[CFDGPU_MAX_NEWTON];    /* PETSc-style KSPConvergedReason per solve */
  int refinements[CFDGPU_MAX_NEWTON];   /* mixed mode: outer flexible-GMRES iterations per solve */
  double ms_assembly, ms_solver, ms_total;
  int guess_used;                       /* 1: the combined initial guess was kept */
  double guess_norm, plain_norm;        /* iteration-0 residual norms of both guesses (when a guess mode is set) */
  double guess_alpha;                   /* coefficient of the first guess direction (0: constant predictor) */
  double guess_alpha2;                  /* coefficient of the second direction (0 when only one is set) */
} cfdgpu_step_stats;

typedef struct cfdgpu_handle cfdgpu_handle;

/* Replaces StabFEM::setSolver/prepareMatrixPattern (StabFEM2.cpp:10-319) and
 * SolverPetsc::initialise (SolverPetsc.cpp:30-116): copies the mesh, builds
 * the nodal-block (BSR) pattern, element colouring and element->block slot
 * map, Dirichlet sets, and allocates all device state (zero initial state,
 * SolutionData::initialise, SolutionData.cpp:16-35). */
int cfdgpu_create(const cfdgpu_mesh *mesh, const cfdgpu_control *ctrl, const cfdgpu_solver_opts *opts,
                  cfdgpu_handle **out);
int cfdgpu_destroy(cfdgpu_handle *h);
const char *cfdgpu_last_error(const cfdgpu_handle *h);

/* Replaces the body of the time loop of StabFEM::solveFullyImplicit
 * (StabFEM2.cpp:632-799): setTimeParam + timeUpdate, assignBoundaryConditions
 * with the caller's ramp factor, then the Newton loop (assembly, residual
 * norm, GMRES solve, update).  Returns CFDGPU_EKSP when a linear solve
 * diverges (the reference exits there); Newton non-convergence is reported
 * in stats->converged and is not an error (the reference continues). */
int cfdgpu_step(cfdgpu_handle *h, double timeNow, double timeFact, cfdgpu_step_stats *stats);

/* Full nodal vector soln (SolutionData::soln), host memory, nNode*ndof. */
int cfdgpu_get_solution(cfdgpu_handle *h, double *soln);
int cfdgpu_set_solution(cfdgpu_handle *h, const double *soln);
/* Device pointer of the handle's soln vector (for callers that keep data on
 * the GPU) and the handle's CUDA stream (cudaStream_t). */
int cfdgpu_device_solution(cfdgpu_handle *h, double **dptr);
int cfdgpu_stream(cfdgpu_handle *h, void **stream);
/* Overwrite the time-history vectors (solnPrev, solnDot) from host memory;
 * NULL leaves one unchanged.  solnDot becomes solnDotPrev at the next step
 * (SolutionData::timeUpdate, SolutionData.cpp:64-78). */
int cfdgpu_set_history(cfdgpu_handle *h, const double *solnPrev, const double *solnDot);
/* Copy solnPrev and solnDot to host memory (NULL skips one). */
int cfdgpu_get_history(cfdgpu_handle *h, double *solnPrev, double *solnDot);

/* Element routine parity hook (ElementBase::calcStiffnessAndResidual): for
 * the listed elements, K_e (nsize x nsize, row-major, local index
 * node*ndof+dof) and F_e from the handle's current solnPrev, solnCur and
 * solnDotCur under time scheme tis/rhoInf/dt, without lifting or Dirichlet
 * masking.  nsize = npElem*ndof.  K and F are host arrays. */
int cfdgpu_element_matrices(cfdgpu_handle *h, const int32_t *elem_ids, int n, double *K, double *F);
/* Set solnPrev, solnCur, solnDotCur directly (host arrays, nNode*ndof) and
 * the td[] vector used by element kernels (time scheme tis). */
int cfdgpu_set_element_state(cfdgpu_handle *h, const double *solnPrev, const double *solnCur,
                             const double *solnDotCur);

/* Sizes of the structures exported by cfdgpu_export_pattern. */
typedef struct cfdgpu_pattern_info {
  int nNode, nElem, npElem, ndof;
  int64_t nnzb;             /* BSR blocks */
  int ncolors;
  int nfixed;               /* distinct Dirichlet dofs */
  int nfree;                /* free dofs (reference ntotdofs_global) */
} cfdgpu_pattern_info;
int cfdgpu_pattern_info_get(cfdgpu_handle *h, cfdgpu_pattern_info *info);
/* rowptr (nNode+1), colidx (nnzb), slot (nElem*npElem*npElem; entries < 0
 * mark the first writer of a block: block = -slot-1), color (nElem),
 * color_ptr (ncolors+1), color_elems (nElem), fixed_dofs (nfixed, sorted),
 * dofmap (nNode*ndof: free index or -1, StabFEM2.cpp:57-81).  Any pointer
 * may be NULL. */
int cfdgpu_export_pattern(cfdgpu_handle *h, int32_t *rowptr, int32_t *colidx, int32_t *slot, int32_t *color,
                          int32_t *color_ptr, int32_t *color_elems, int32_t *fixed_dofs, int32_t *dofmap);

/* Host-only variant (no device, no handle): builds the same structures from
 * a mesh.  Call once with NULL arrays to get the sizes in *info, then with
 * arrays of those sizes. */
int cfdgpu_pattern_build(const cfdgpu_mesh *mesh, cfdgpu_pattern_info *info, int32_t *rowptr, int32_t *colidx,
                         int32_t *slot, int32_t *color, int32_t *color_ptr, int32_t *color_elems,
                         int32_t *fixed_dofs, int32_t *dofmap);

/* Host-only: the block ILU(k) symbolic phase of the library (the factor
 * pattern and the schedules of the persistent factorisation and triangular
 * solves) for a mesh, levels (-1: complete factorisation) and block-Jacobi
 * blocks.  Call once with NULL arrays to get the sizes, then with arrays of
 * those sizes: rowptr (nNode+1), colidx (nnzb), perm (nNode; the identity
 * unless the complete factorisation is reordered), lorder / uorder (nNode:
 * rows in level order of the lower / upper dependency DAG), lchain / uchain
 * (2 x nchains: first row, one past the last row), lchain_order /
 * uchain_order (nchains: chain ids in chain-DAG level order).  Any pointer may
 * be NULL.  Used by tests to check the schedules' invariants (every input of
 * a row or chain is handed out earlier), on which the sync-free kernels'
 * progress rests. */
typedef struct cfdgpu_ilu_info {
  int nNode;
  int64_t nnzb;              /* factor blocks */
  int nchains_l, nchains_u;
  int nlev_l, nlev_u;        /* levels of the row DAGs */
  int chain_levels_l, chain_levels_u;
} cfdgpu_ilu_info;
int cfdgpu_ilu_pattern_build(const cfdgpu_mesh *mesh, int levels, int nblocks, cfdgpu_ilu_info *info,
                             int32_t *rowptr, int32_t *colidx, int32_t *perm, int32_t *lorder, int32_t *uorder,
                             int32_t *lchain, int32_t *uchain, int32_t *lchain_order, int32_t *uchain_order);

/* Assemble (iteration-0 semantics when iter == 0: lifting included) at the
 * current state and copy the BSR values (nnzb*ndof*ndof, FP64, block
 * row-major) and the RHS (nNode*ndof) to host.  Uses the td[] of the last
 * step or of cfdgpu_set_element_state. */
int cfdgpu_assemble_export(cfdgpu_handle *h, int iter, double *bsr_vals, double *rhs);

/* Solve A x = b on the handle's last assembled matrix with the handle's
 * GMRES options; b and x are host arrays (nNode*ndof, zero at Dirichlet
 * dofs).  its/reason may be NULL. */
int cfdgpu_solve_export(cfdgpu_handle *h, const double *b, double *x, int *its, int *reason);

/* Block ILU(k) factors of the last assembled matrix (handles with
 * pc_type CFDGPU_PC_BJACOBI_ILU), for parity checks against a CPU ILU.  The
 * factor pattern is a BSR over the nodes: rowptr (nNode+1), colidx (*nnzb,
 * sorted per row), diag (nNode, position of each diagonal block); vals
 * (nnzb*ndof*ndof, row-major blocks) hold the multipliers L_ip below the
 * diagonal and U on and above it; dinv (nNode*ndof*ndof) the inverted
 * diagonal blocks of U.  Any pointer may be NULL; asking for vals or dinv
 * factorises the matrix first.  Replaces the numeric factorisation PETSc's
 * PCSetUp runs inside KSPSolve (SolverPetsc.cpp:253). */
int cfdgpu_ilu_export(cfdgpu_handle *h, int64_t *nnzb, int32_t *rowptr, int32_t *colidx, int32_t *diag, double *vals,
                      double *dinv);

/* z = M^-1 r with the handle's preconditioner, built from the last assembled
 * matrix (PCApply; host arrays of nNode*ndof, zero at Dirichlet dofs). */
int cfdgpu_pc_apply_export(cfdgpu_handle *h, const double *r, double *z);

/* True (unpreconditioned) residual of the last assembled system:
 * *norm = ||b - A x||_2 with the library's deterministic reduction.  x and b
 * are host arrays of nNode*ndof doubles (zero at Dirichlet dofs). */
int cfdgpu_true_residual(cfdgpu_handle *h, const double *x, const double *b, double *norm);

/* Allocation-free variant of cfdgpu_true_residual, for callers that may not
 * allocate device memory (code running inside another framework's memory
 * pool, or given only a stream to enqueue on).  No handle: the caller passes
 * a BSR matrix already on the device (row pointer nNode+1, column index,
 * values in nodal blocks of ndof x ndof, row-major) and device vectors x, b
 * (nNode*ndof); the kernel writes ||b - A x||_2 to the device double d_norm,
 * enqueued on `stream` (a cudaStream_t; NULL = legacy default stream).
 * ndof is 3 or 4.  Alignment: d_val, d_x and d_b 16 bytes, d_norm 8 bytes,
 * d_rowptr and d_colidx 4 bytes (the 4x4 kernel reads 16-byte vectors);
 * other pointers return CFDGPU_EINVAL before any work is enqueued.  Scratch
 * lives in a fixed array inside the library (16 MiB, held by every GPU that
 * loads the library until exit); nNode*ndof above 2,097,152 returns
 * CFDGPU_ETOOBIG.  The call allocates nothing.  Its first call on a device
 * looks up the array's device address (cudaGetSymbolAddress, with the device
 * current) and should come before any stream capture; later calls outside
 * capture look it up again, so the address stays valid after a
 * cudaDeviceReset, while calls during capture use the address found by the
 * last call outside capture.  All calls share the array: calls that overlap
 * on the GPU (different streams, or different host threads on one device)
 * race and must be serialised by the caller.  This entry point has no
 * counterpart in the reference. */
int cfdgpu_residual_norm_noalloc(int nNode, int ndof, const int32_t *d_rowptr, const int32_t *d_colidx,
                                 const double *d_val, const double *d_x, const double *d_b, double *d_norm,
                                 void *stream);

/* Timers in the reference's categories (StabFEM::printComputerTimes,
 * StabFEM.cpp:711-727), seconds: [0] pattern, [1] assembly, [2] solver,
 * [3] post-process (unused by the library), [4] total in cfdgpu_step. */
int cfdgpu_timers(cfdgpu_handle *h, double t[5]);

/* Number of kernel launches issued by this handle so far. */
int64_t cfdgpu_launch_count(cfdgpu_handle *h);

/* ---- learned Newton initial guess ------------------------------------
 * A message-passing network over the handle's node graph (hidden width 64,
 * three residual mean-aggregation layers) maps [u_n, u_n - u_{n-1}, X] to the
 * correction of the next-step increment over linear extrapolation,
 * u_{n+1} - 2 u_n + u_{n-1}; the predicted increment is u_n - u_{n-1} plus
 * that correction.  Training and inference run on the device with the
 * library's own kernels (BF16 tensor-core GEMMs, FP32 accumulation, FP32
 * Adam).  No counterpart in the reference: its Newton loop starts from the
 * previous step's solution (src/base/StabFEM2.cpp:654, SolutionData.cpp:64-78). */
typedef struct cfdgpu_mpnn cfdgpu_mpnn;
int cfdgpu_mpnn_create(cfdgpu_handle *h, uint64_t seed, cfdgpu_mpnn **out);
int cfdgpu_mpnn_destroy(cfdgpu_mpnn *m);
int cfdgpu_mpnn_num_params(cfdgpu_mpnn *m);
int cfdgpu_mpnn_get_params(cfdgpu_mpnn *m, float *p);
int cfdgpu_mpnn_set_params(cfdgpu_mpnn *m, const float *p);
/* feature scales for u_n and u_n - u_{n-1} (2*ndof values) and scales of the
 * correction target (ndof values); set before adding samples */
int cfdgpu_mpnn_set_scales(cfdgpu_mpnn *m, const float *in_scale, const float *out_scale);
/* one training sample (host arrays of nNode*ndof): u_{n-1}, u_n, u_{n+1} */
int cfdgpu_mpnn_add_sample(cfdgpu_mpnn *m, const double *u_nm1, const double *u_n, const double *u_np1);
/* Condition input channel (a per-instance scalar such as a scaled Reynolds
 * number; 0 by default): used by later samples of the network's own graph
 * and by its predictions. */
int cfdgpu_mpnn_set_condition(cfdgpu_mpnn *m, double cond);
/* A training sample (host arrays) on another handle's mesh graph, with its
 * condition value: one network's weights learn from instances of different
 * meshes.  The other mesh must have the same dofs per node and dimension and
 * at most as many nodes as the network's own; predictions always serve the
 * network's own handle (copy trained weights into a network per instance
 * with cfdgpu_mpnn_get_params / cfdgpu_mpnn_set_params). */
int cfdgpu_mpnn_add_sample_on(cfdgpu_mpnn *m, cfdgpu_handle *h, double cond, const double *u_nm1, const double *u_n,
                              const double *u_np1);
int cfdgpu_mpnn_num_samples(cfdgpu_mpnn *m);
/* masked mean-squared error of one sample and its gradient (host floats) */
int cfdgpu_mpnn_loss_grad(cfdgpu_mpnn *m, int sample, float *loss, float *grad);
/* iters Adam steps cycling over the samples; *loss_out = last loss */
int cfdgpu_mpnn_train(cfdgpu_mpnn *m, int iters, float lr, float *loss_out);
/* predicted increment (host arrays; zero at prescribed dofs) */
int cfdgpu_mpnn_predict(cfdgpu_mpnn *m, const double *u_nm1, const double *u_n, double *delta);
/* Initial-guess directions for cfdgpu_step (bit flags). */
#define CFDGPU_GUESS_NETWORK 1            /* the network's predicted increment */
#define CFDGPU_GUESS_NETWORK_VELOCITY 2   /* the same, velocity dofs only */
#define CFDGPU_GUESS_EXTRAPOLATION 4      /* u_n - u_{n-1} (linear extrapolation) */
/* Newton initial guess of cfdgpu_step: u_n + a1*d1 + a2*d2 over the selected
 * directions (at most two).  The iteration-0 residual is affine in the state,
 * so one residual evaluation per direction gives the exact minimiser of
 * ||F(u_n + a1 d1 + a2 d2)||; it is used only if it lowers the residual
 * (stats->guess_used), otherwise the step runs from the reference's constant
 * predictor.  mode 0 (or m NULL with network bits) = constant predictor. */
int cfdgpu_set_guess_mode(cfdgpu_handle *h, cfdgpu_mpnn *m, int mode);
/* cfdgpu_set_guess_mode(h, m, NETWORK | EXTRAPOLATION), or mode 0 for m = NULL */
int cfdgpu_set_guess(cfdgpu_handle *h, cfdgpu_mpnn *m);

/* Per-kernel device timing with CUDA events on the handle's stream (off by
 * default).  Kinds: */
#define CFDGPU_KIND_SPMV 0        /* BSR SpMV with the fused preconditioner (Krylov operator) */
#define CFDGPU_KIND_ELEM_K 1      /* element kernel, tangent + residual, one launch per colour */
#define CFDGPU_KIND_ELEM_F 2      /* element kernel, residual only */
#define CFDGPU_KIND_ORTHO 3       /* Gram-Schmidt multi-dot + update/norm pair */
#define CFDGPU_KIND_TRSV 4        /* block ILU triangular solves (lower + upper, one preconditioner application) */
#define CFDGPU_KIND_ILU 5         /* block ILU numeric factorisation */
#define CFDGPU_KIND_BCGS 6        /* BiCGStab vector updates and dot products of one iteration */
#define CFDGPU_KIND_COUNT 7
int cfdgpu_set_profiling(cfdgpu_handle *h, int on);
/* Totals since profiling was switched on: launches, summed device ms, and
 * summed algorithmic bytes (the minimum DRAM traffic of each launch). */
int cfdgpu_kernel_stats(cfdgpu_handle *h, int kind, int64_t *launches, double *total_ms, double *total_bytes);

/* ---- batched stepping of independent instances -----------------------
 * No counterpart in the reference (one mesh per process).  A batch owns one
 * handle per instance (each with its own mesh, control and solver options)
 * and a pool of host threads that step the instances concurrently on the
 * current device, largest first.  Each instance computes exactly what its
 * own handle would alone.  For many concurrent streams to reach the GPU
 * separately, set CUDA_DEVICE_MAX_CONNECTIONS (e.g. 32) before the process
 * creates its CUDA context. */
#define CFDGPU_BATCH_MAX 4096
#define CFDGPU_BATCH_MAX_THREADS 128
#define CFDGPU_BATCH_MAX_DEPTH 8
typedef struct cfdgpu_batch cfdgpu_batch;
/* count instances, arrays of count structs; on failure *out may still be set
 * (read cfdgpu_batch_last_error, then cfdgpu_batch_destroy) */
int cfdgpu_batch_create(int count, const cfdgpu_mesh *meshes, const cfdgpu_control *ctrls,
                        const cfdgpu_solver_opts *opts, cfdgpu_batch **out);
int cfdgpu_batch_destroy(cfdgpu_batch *b);
const char *cfdgpu_batch_last_error(cfdgpu_batch *b);
int cfdgpu_batch_size(cfdgpu_batch *b);
/* instance i's handle (get/set solution, history, timers...); owned by the batch */
cfdgpu_handle *cfdgpu_batch_handle(cfdgpu_batch *b, int i);
/* concurrency: host threads stepping instances at once; chunk: Arnoldi steps
 * per CUDA graph (1..64); depth: chunks each instance keeps enqueued beyond
 * the one whose state its thread waits for (1..8).  (0, 0, 0) = autotune:
 * the next batch steps each try one candidate, scored by wall time per GMRES
 * iteration, and the best is kept.  Results do not depend on any of them. */
int cfdgpu_batch_set_schedule(cfdgpu_batch *b, int concurrency, int chunk, int depth);
int cfdgpu_batch_get_schedule(cfdgpu_batch *b, int *concurrency, int *chunk, int *depth, int *tuned);
/* one time step of every instance: timeNow/timeFact per instance (count
 * values each); stats and latency_ms (host wall time of each instance's
 * step) per instance.  Returns the first failing instance's code. */
int cfdgpu_batch_step(cfdgpu_batch *b, const double *timeNow, const double *timeFact, cfdgpu_step_stats *stats,
                      double *latency_ms);

#ifdef __cplusplus
}
#endif

#endif /* CFDGPU_H */
