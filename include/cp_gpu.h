/*
 * cp_gpu.h -- C ABI of the B200 crystal-plasticity quadrature-point library.
 *
 * The library replaces, for a batch of quadrature points (qps) resident on one
 * GPU, the per-qp hot path of PRISMS-Plasticity's crystalPlasticity<dim> model:
 *
 *   calculatePlasticity(cellID, q, StiffnessCalFlag)
 *       src/materialModels/crystalPlasticity/calculatePlasticity.cc:13-1022
 *       (declared include/crystalPlasticity.h:77)
 *   inactive_slip_removal(...)       .../inactiveSlipRemoval.cc:4-124
 *   the inline algorithmic tangent   .../calculatePlasticity.cc:473-940
 *       (include/crystalPlasticity.h:48 declares tangent_modulus, never defined)
 *   getElementalValues(...) qp loop   .../getElementalValues.cc:127-163
 *       (pure virtual in include/ellipticBVP.h:130, override crystalPlasticity.h:78)
 *   reorient()                       .../reorient.cc:4-98
 *   history commit _iter -> _conv    .../updateAfterIncrement.cc:287-305
 *   volume averages                  .../updateAfterIncrement.cc:119-126,218-235,710-722
 *
 * Conventions
 *   - Every function returns an int status: CP_OK (0) or a negative CP_E* code;
 *     cp_last_error() gives a one-line message for the handle's last failure.
 *   - Pointers named h_* are host pointers, borrowed for the duration of the
 *     call (pageable works; page-locked memory gets the full copy bandwidth).
 *     Pointers named d_* are device pointers on the handle's GPU; those calls
 *     are asynchronous on the handle's stream unless noted.
 *   - 3x3 tensors are row-major (A[i][j] at 3*i+j); a batch of tensors is
 *     qp-major: qp k's tensor starts at 9*k.  dP/dF is dPdF[m][n][o][p] at
 *     81*k + 27*m + 9*n + 3*o + p (the reference's Tensor<4,3> dP_dF).
 *   - Voigt order everywhere is (11,22,33,23,13,12) as in vecform/matform
 *     (matrixOperations.cc:133-163).
 *   - One CUDA stream per handle; no global mutable state; calls on different
 *     handles may come from different host threads.  A handle is not
 *     re-entrant (like the reference class, which keeps scratch in members).
 *   - There is no CPU fallback: if the CUDA kernels cannot be launched the
 *     call fails with CP_E_CUDA.
 */
#ifndef CP_GPU_H
#define CP_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CP_MAX_SYSTEMS 64  /* slip + twin systems per lattice, dummy twin included */
#define CP_MAX_LATTICES 8  /* phases per handle (the reference supports up to 4) */

/* return codes */
#define CP_OK 0
#define CP_E_ARG (-1)      /* invalid argument / size */
#define CP_E_STATE (-2)    /* call out of order (e.g. cp_update before cp_bind_qps) */
#define CP_E_CUDA (-3)     /* CUDA runtime error */
#define CP_E_NOMEM (-4)    /* device or pinned allocation failed */
#define CP_E_UNSUPPORTED (-5)

/* per-qp status bits written by cp_update / cp_assemble (0 = clean) */
#define CP_QP_NONFINITE 1       /* a NaN/Inf reached P, T or dP/dF */
#define CP_QP_SINGULAR 2        /* a zero pivot in an active-set or tangent solve */
#define CP_QP_ACTIVE_OVERFLOW 4 /* potentially active set larger than the kernel's tile */
#define CP_QP_SERIES_CAP 8      /* exp / Gateaux series hit its term cap */
#define CP_QP_SLIP_SEARCH_CAP 16 /* informational: slip-search cap reached (reference truncates silently, calculatePlasticity.cc:155-158) */
#define CP_QP_ILL_CONDITIONED 32 /* informational: an active-set solve had condition > 1e12; the
                                    reference's compute_inverse_svd(0.0) result there is set by rounding */

/*
 * One lattice (phase).  Field names follow userInputParameters
 * (src/userInputParameters/userInputParameters.cc:255-323) and the per-phase
 * members loaded by multiphaseInit (multiphaseInit.cc:4-67).
 * Systems 0..n_slip-1 are slip systems, n_slip..n_slip+n_twin-1 twin systems.
 * With twinning disabled the reference appends ONE dummy twin system
 * (init.cc:37-41,178-185; userInputParameters.cc:303-311): callers build it
 * with cp_material_add_dummy_twin().
 */
typedef struct cp_material_t {
    int32_t n_slip;               /* numSlipSystems */
    int32_t n_twin;               /* numTwinSystems (1 = the dummy when twinning is off) */
    int32_t twinning_enabled;     /* enableTwinning: twin reorientation branch */
    int32_t reserved;
    double elastic_stiffness[36]; /* 6x6 Voigt, row-major: "Elastic Stiffness row 1..6" */
    double slip_normal[CP_MAX_SYSTEMS * 3];    /* n_alpha, unit length */
    double slip_direction[CP_MAX_SYSTEMS * 3]; /* m_alpha, unit length */
    double latent_hardening[CP_MAX_SYSTEMS * CP_MAX_SYSTEMS]; /* q[a][b] at a*CP_MAX_SYSTEMS+b */
    double initial_slip_resistance[CP_MAX_SYSTEMS];   /* s0 */
    double initial_hardening_modulus[CP_MAX_SYSTEMS]; /* h0 */
    double saturation_stress[CP_MAX_SYSTEMS];         /* s_s */
    double power_law_exponent[CP_MAX_SYSTEMS];        /* a */
    double kinematic_c1[CP_MAX_SYSTEMS];              /* C_1 (0 when kinematic hardening is off) */
    double kinematic_c2[CP_MAX_SYSTEMS];              /* C_2 */
    double twin_threshold_fraction;  /* twinThresholdFraction */
    double twin_saturation_factor;   /* twinSaturationFactor */
    double twin_shear;               /* twinShear ("Characteristic Twin Shear") */
} cp_material_t;

/* Numerical options (userInputParameters.cc:320-323) and execution knobs. */
typedef struct cp_options_t {
    double stress_tolerance;            /* modelStressTolerance ("Stress Tolerance") */
    int32_t max_slip_search_iterations; /* modelMaxSlipSearchIterations */
    int32_t max_solver_iterations;      /* modelMaxSolverIterations */
    int32_t enable_multiphase;          /* F_T rule, calculatePlasticity.cc:970-980 */
    int32_t device;                     /* CUDA device ordinal */
    int32_t update_variant;             /* launch shape of the sorted update: 0 = each lattice group's
                                           shape chosen by cp_autotune, or the default rule before any
                                           tuning; k in 1..CP_UPDATE_VARIANTS forces shape k-1 */
    int32_t use_graphs;                 /* 1 (cp_options_default): the launches of a cp_update_device,
                                           cp_assemble_device or cp_update_from_displacement call are
                                           captured once as a CUDA graph and replayed while the call's
                                           pointers, scalars and launch shapes repeat; 0: stream launches */
    int32_t plain_kernel;               /* 1: one thread per qp in bind order with full-size per-thread
                                           scratch (the plain FP64 drop-in, kept as a baseline);
                                           0 (default): qps sorted by potentially-active-set size each
                                           call, compact per-thread scratch */
    int32_t reference_order;            /* 1: cp_update / cp_update_device / cp_update_from_displacement
                                           evaluate calculatePlasticity in the reference's own operation
                                           order (full consistency matrix, SVD pseudo-inverse, FullMatrix
                                           inverses, no multiply-add contraction), reproducing a CPU
                                           restatement bit for bit; slow (per-qp scratch of ~6 n^2
                                           doubles, up to 2 GiB per handle).  The assembly, autotune,
                                           mixed-precision and batch calls return CP_E_UNSUPPORTED. */
} cp_options_t;

typedef struct cp_handle cp_handle;

/* Fill *opts with the reference defaults (tol 1e-9, caps 1/1, device 0). */
int cp_options_default(cp_options_t* opts);

/* Append the reference's dummy twin system to a twinning-disabled lattice:
 * CRSS 10e14, h0 1, a 0, s_s 10e15, n=(1,0,0), m=(0,1,0), zero q row/col
 * (userInputParameters.cc:303-311, init.cc:51-65,178-185). */
int cp_material_add_dummy_twin(cp_material_t* mat);

/*
 * Create a handle for n_lattices phases on opts->device.
 * Replaces the constructor + multiphaseInit: all per-lattice constants go to
 * the device once instead of being reloaded on every qp call
 * (multiphaseInit.cc:4-67 runs at calculatePlasticity.cc:17).
 */
int cp_create(const cp_material_t* lattices, int32_t n_lattices,
              const cp_options_t* opts, cp_handle** out);
void cp_destroy(cp_handle* h);
const char* cp_last_error(const cp_handle* h);

/*
 * Allocate the resident per-qp history (init.cc:198-330): Fp=Fe=I, s=s0,
 * W=0, twin/slip fractions 0, twin flag 0, rot=rotnew=rodrigues.
 * lattice_id[k] in [0, n_lattices); h_rodrigues is 3*n_qp (orientation of qp k).
 * Internally qps are grouped by lattice; all qp-indexed arrays of the API stay
 * in the caller's order.
 */
int cp_bind_qps(cp_handle* h, int64_t n_qp, const int32_t* h_lattice_id,
                const double* h_rodrigues);
int64_t cp_num_qps(const cp_handle* h);

/*
 * Batched calculatePlasticity(cellID, q, stiffness_flag) for every bound qp.
 * h_F: 9*n_qp deformation gradients.  Outputs (may be NULL when unwanted):
 * h_P (first Piola, 9*n_qp), h_T (Cauchy, 9*n_qp), h_dPdF (81*n_qp, only
 * written when stiffness_flag == 1), h_status (n_qp status bits).
 * F_e / F_r are the previous increment's volume-averaged twin quantities
 * (updateAfterIncrement.cc:719-720) used by the twin-reorientation threshold.
 * Synchronous: returns when the outputs are in host memory.  Batches above
 * 2^18 qps run in caller-order chunks whose copies overlap the other chunks'
 * kernels; page-locked host buffers get the full overlap.
 */
int cp_update(cp_handle* h, const double* h_F, int32_t stiffness_flag,
              double F_e, double F_r, double* h_P, double* h_T, double* h_dPdF,
              int32_t* h_status);

/* Same on device buffers, asynchronous on the handle's stream. */
int cp_update_device(cp_handle* h, const double* d_F, int32_t stiffness_flag,
                     double F_e, double F_r, double* d_P, double* d_T,
                     double* d_dPdF, int32_t* d_status);

/*
 * Per-qp work statistics of the last cp_update / cp_assemble (device buffer
 * kept by the handle), copied to h_stats as 8 int32 per qp:
 *   [0] potentially active systems p0, [1] final active systems p,
 *   [2] active-set removal rounds, [3] exp series terms e,
 *   [4] Gateaux series terms c (count3), [5] slip-search passes,
 *   [6] lattice id, [7] ceil(log10) of the largest condition estimate of the
 *   active-set solves (pivot ratio of the LU factors; 0 when no solve ran).
 */
int cp_get_stats(cp_handle* h, int32_t* h_stats);

/*
 * Element mesh for the fused assembly: n_cells hexahedral Q1 cells with 8
 * Gauss points each; qp k = 8*cell + q must be the bound qp of that point.
 * h_grad_N: shape-function gradients, [cell][q][node a][3] (8*8*3 doubles per
 * cell), or one cell's worth shared by all cells when uniform != 0.
 * h_JxW: [cell][q] (or [q] when uniform).  Local dof d = 3*a + c is component
 * c of node a (FESystem<FE_Q<1>,3> ordering).
 */
int cp_bind_mesh(cp_handle* h, int64_t n_cells, const double* h_grad_N,
                 const double* h_JxW, int32_t uniform);

/*
 * Batched getElementalValues (getElementalValues.cc:127-163): for every cell,
 * F = I + sum_d U_d grad N_d at each qp, calculatePlasticity(...,1), then
 * Re[d] -= gradN_d . P . JxW and Ke[d1][d2] += gradN_d1 . dPdF . gradN_d2 JxW.
 * h_U_local: 24*n_cells; outputs h_Ke 576*n_cells (row-major 24x24, not
 * symmetric), h_Re 24*n_cells.  Synchronous; chunked over cells like
 * cp_update (copies overlap the kernels of the other chunks).
 */
int cp_assemble(cp_handle* h, const double* h_U_local, double F_e, double F_r,
                double* h_Ke, double* h_Re, int32_t* h_status);
int cp_assemble_device(cp_handle* h, const double* d_U_local, double F_e,
                       double F_r, double* d_Ke, double* d_Re, int32_t* d_status);

/*
 * Mixed-precision batched getElementalValues: the same sorted FP64 update
 * (F gather, calculatePlasticity with the tangent), then the element
 * contraction Ke = sum_q B^T (JxW dP/dF) B on the tensor cores in split-BF16
 * (three bf16 terms per operand, six products) with FP32 accumulation:
 * Ke is FP32 (576 per cell, relative error ~1e-7 of the cell's largest
 * entry against the FP64 contraction), Re stays FP64 and equals
 * cp_assemble's bit for bit (getElementalValues.cc:144-162).  Needs a
 * uniform mesh (cp_bind_mesh uniform != 0) and the sorted update.  The
 * device form is asynchronous: an expired wait inside the contraction
 * (an error flag, no GPU fault) is reported by the next cp_synchronize;
 * the host form reports it itself.
 */
int cp_assemble_mixed(cp_handle* h, const double* h_U_local, double F_e, double F_r,
                      float* h_Ke, double* h_Re, int32_t* h_status);
int cp_assemble_mixed_device(cp_handle* h, const double* d_U_local, double F_e,
                             double F_r, float* d_Ke, double* d_Re, int32_t* d_status);

/*
 * Volume averages over the bound mesh after a post-pass update, as
 * updateAfterIncrement.cc:119-126,218-235,710-722 accumulates them, using the
 * F of the last cp_update (E = (F^T F - I)/2) and its Cauchy stress.
 * out[0..8] strain E (3x3 row-major), out[9..17] stress T, out[18] F_r
 * (twin fraction), out[19] F_e (twinned volume), out[20] F_s (slip), out[21]
 * volume.  Requires cp_bind_mesh (for JxW).
 */
int cp_averages(cp_handle* h, double out[22]);

/*
 * cp_averages without any device allocation.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: host codes whose device memory is
 * handed to their own pool allocator up front (a PETSc/Kokkos-style pool in
 * the FE application owns the GPU's memory), and per-increment callbacks that
 * must not pay cudaMalloc/cudaFree, which synchronise the whole device and
 * stall the caller's other streams.  cp_averages allocates its reduction
 * scratch on first use; this variant instead uses a file-scope device array
 * compiled into the library (about 2.9 MB, held on every GPU that loads the
 * library until the process exits) and calls no allocating routine.
 *
 * Same inputs, outputs and summation order as cp_averages.  Limits and rules:
 *   - at most CP_NOALLOC_AVG_MAX_QPS bound qps; larger handles get CP_E_ARG
 *     with a message naming the limit;
 *   - the first call on a handle looks up the array's device address
 *     (cudaGetSymbolAddress, with the handle's device current) and keeps it
 *     in the handle; make that first call before any stream capture (the
 *     address does not survive a device reset, which no handle survives);
 *   - every call on a device shares the one array and it keeps the last
 *     call's contents (each call writes every entry it reads, so nothing
 *     needs clearing); calls that overlap on the GPU (different handles on
 *     different streams of the same device) race on it.
 */
#define CP_NOALLOC_AVG_MAX_QPS (1 << 22)
int cp_averages_noalloc(cp_handle* h, double out[22]);

/* reorient() (reorient.cc:4-98) on all qps: updates rotnew_conv. */
int cp_reorient(cp_handle* h);

/* Commit the increment: *_conv = *_iter (updateAfterIncrement.cc:287-305).
 * In the sorted pipeline (not plain_kernel, not reference_order) the device
 * storage of each lattice group is also permuted into the order of the last
 * update's sort keys (within the chunks of the host-pointer calls); caller
 * order, cp_get_state / cp_set_state and every result are unchanged. */
int cp_commit(cp_handle* h);

/* History fields for cp_get_state / cp_set_state.  Per-qp widths: */
#define CP_FIELD_FP_CONV 0       /* 9 */
#define CP_FIELD_FE_CONV 1       /* 9 */
#define CP_FIELD_S_CONV 2        /* n_T of the qp's lattice, padded to the handle's max n_T */
#define CP_FIELD_W_CONV 3        /* same */
#define CP_FIELD_ROT_CONV 4      /* 3 */
#define CP_FIELD_ROTNEW_CONV 5   /* 3 */
#define CP_FIELD_TWINFRAC_CONV 6 /* n_twin, padded to the handle's max n_twin */
#define CP_FIELD_SLIPFRAC_CONV 7 /* n_slip, padded to the handle's max n_slip */
#define CP_FIELD_TWIN_CONV 8     /* 1 (0.0 or 1.0) */
#define CP_FIELD_ITER_OFFSET 16  /* add to get the *_iter field */
#define CP_FIELD_FP_ITER (CP_FIELD_ITER_OFFSET + CP_FIELD_FP_CONV)

/* Width (doubles per qp) of a field in cp_get_state/cp_set_state. */
int32_t cp_field_width(const cp_handle* h, int32_t field);
/* Copy a history field to/from host (h_buf: width*n_qp doubles, caller order). */
int cp_get_state(cp_handle* h, int32_t field, double* h_buf);
int cp_set_state(cp_handle* h, int32_t field, const double* h_buf);

/*
 * The Newton step's global system on the device (next to the qp path: the
 * reference's ellipticBVP::assemble, src/ellipticBVP/assemble.cc:62-90, with
 * constraints.distribute_local_to_global at :78; the Dirichlet constraints of
 * boundaryConditions.cc:453-497; solveLinearSystem.cc:10-36, PETSc BiCG with
 * a Jacobi preconditioner and tolerance relLinearSolverTolerance * ||b||).
 *
 * cp_bind_dofs: after cp_bind_mesh.  h_cell_dofs holds the 24 global dof
 * indices of every cell in local-dof order (d = 3a + c), h_constrained the
 * Dirichlet dofs.  Builds the CSR pattern of K and, per matrix entry and per
 * dof, the list of element entries that sum into it (cell order, so the
 * scatter is deterministic).  The displacement u (n_dofs) starts at zero.
 */
int cp_bind_dofs(cp_handle* h, int64_t n_dofs, const int64_t* h_cell_dofs,
                 int64_t n_constrained, const int64_t* h_constrained);
int cp_set_displacement(cp_handle* h, const double* h_u);
int cp_get_displacement(cp_handle* h, double* h_u);

#define CP_SOLVER_BICG 0     /* PETScWrappers::SolverBiCG, the reference's solver */
#define CP_SOLVER_BICGSTAB 1 /* BiCGStab (right Jacobi preconditioning) */
#define CP_PRECOND_JACOBI 0     /* PETScWrappers::PreconditionJacobi, the reference's */
#define CP_PRECOND_NODE_BLOCK 1 /* inverse of each node's 3x3 diagonal block (BiCG, precond_norm 0) */
typedef struct cp_solver_t {
    int32_t kind;           /* CP_SOLVER_* */
    int32_t max_iterations; /* "Maximum linear solver iterations" (decks: 50000) */
    double rel_tolerance;   /* "Relative linear solver tolerance": stop at ||r|| <= tol ||b|| */
    int32_t precond_norm;   /* 0: true residual ||b - K du||; 1: ||M^-1 r|| (PETSc's BiCG default) */
    int32_t check_every;    /* iterations queued between host checks of convergence (0: 8) */
    int32_t precond;        /* CP_PRECOND_* (the node blocks need the three components of every
                               node among one cell's local dofs 3a..3a+2, as cp_bind_dofs takes them) */
    int32_t kernel_mode;    /* 0: Jacobi BiCG of at most CP_PERSISTENT_MAX_DOFS dofs runs as one
                               cooperative launch that iterates to convergence, larger systems as
                               four kernels per iteration; 1: always four kernels per iteration;
                               2: one cooperative launch at any size */
    int32_t precision;      /* CP_PRECISION_FP64 (default): FP64 assembly and solve.
                               CP_PRECISION_MIXED: the element contraction on the tensor cores
                               (cp_assemble_mixed: FP32 Ke, FP64 Re), K scattered to FP32, and the
                               solve as FP64 iterative refinement (r = b - K x in FP64 products of
                               K's FP32 values, stopped at ||r|| <= rel_tolerance ||b||) around
                               FP32 Jacobi BiCG inner solves to a relative residual of
                               inner_tolerance (at most 2000 iterations each); a pass is kept when
                               it cuts ||r|| ten-fold, and the first FP32 pass that does not hands
                               the remaining passes to FP64 BiCG on the same matrix; BiCG + Jacobi
                               and the true-residual test only; needs a uniform mesh */
    int32_t max_refinements; /* CP_PRECISION_MIXED: outer refinement passes (0: 10) */
    double inner_tolerance;  /* CP_PRECISION_MIXED: relative residual of each FP32 inner solve
                               (0: 1e-5) */
} cp_solver_t;
#define CP_PRECISION_FP64 0
#define CP_PRECISION_MIXED 1
#define CP_PERSISTENT_MAX_DOFS 49152
typedef struct cp_solve_info_t {
    int32_t iterations; /* Krylov iterations to convergence (or the cap); mixed precision: all
                           inner FP32 iterations of every refinement pass */
    int32_t converged;  /* 1 if the tolerance was met */
    int32_t breakdown;  /* 1 if the method broke down (zero rho or denominator) */
    int32_t refinements; /* mixed precision: refinement passes run (0 in FP64) */
    double rhs_norm;      /* ||b|| of the condensed system */
    double residual_norm; /* the tested residual norm at exit */
    int32_t fp64_iterations; /* of 'iterations', those run in FP64 (all of them in FP64 mode; in
                               mixed precision the FP64 passes that follow an FP32 pass which
                               did not cut the residual ten-fold) */
    int32_t reserved;
} cp_solve_info_t;
int cp_solver_default(cp_solver_t* solver); /* BiCG, Jacobi, 50000, 1e-10, true residual */

/*
 * One Newton iteration on the device (solveNonLinearSystem.cc:14-81, one
 * pass): U_local gathered from u, batched getElementalValues, K and R
 * scattered, the constrained dofs' increments h_du_constrained (n_constrained
 * values in cp_bind_dofs order; NULL = zero) condensed into the system, the
 * Krylov solve, constrained dofs set to their increments (distribute), and
 * u += du.  solver NULL = cp_solver_default.  info may be NULL.
 */
int cp_newton_iteration(cp_handle* h, const double* h_du_constrained, double F_e, double F_r,
                        const cp_solver_t* solver, cp_solve_info_t* info);

/*
 * The second half of cp_newton_iteration: K and R from the element matrices
 * already in the handle's system (written by cp_batch_assemble), the
 * condensation, the Krylov solve, distribute and u += du.  FP64 only.
 */
int cp_newton_solve(cp_handle* h, const double* h_du_constrained, const cp_solver_t* solver,
                    cp_solve_info_t* info);

/*
 * The post-pass calculatePlasticity(...,0) at every qp
 * (updateAfterIncrement.cc:105) with F from the device displacement; then
 * cp_averages / cp_reorient / cp_commit as after cp_update.
 */
int cp_update_from_displacement(cp_handle* h, double F_e, double F_r);

/*
 * Launch-shape autotuner of the sorted update (no counterpart in the
 * reference).  Shapes 0-3 run one thread per qp (threads per block /
 * registers per thread):
 *   0: 256 / 255   1: 256 / 128   2: 64 / 255   3: 64 / 128
 * Shape 4 runs four lanes per qp with the active-set matrix, right-hand
 * sides and per-system vectors in shared memory, in chunks of qps with one
 * potentially-active-set size (a persistent grid of two 128-thread blocks
 * per SM); it serves max_slip_search_iterations = 1 only (otherwise calls
 * take the untuned rule's shape and the tuner skips it, median -1).  Every
 * shape gives the same bits.  The untuned rule takes 2 (FCC class) or 3 (BCC/HCP classes) for launches
 * of at most 9,472 qps and 0 above.  cp_autotune times every shape on
 * the live workload, group by group: path CP_TUNE_UPDATE runs the flag-1
 * update with d_in = F (9*n_qp, device); path CP_TUNE_ASSEMBLE runs the fused
 * assembly's update with d_in = U_local (24*n_cells, device).  Each shape
 * runs 1 + reps times (the first untimed); the update reads the _conv
 * history and writes _iter, so the repeats see the same input and leave the
 * history as one call would.  The chosen shape (cp_tune_select on the
 * timings, min_gain as there) is stored in the handle for that path and
 * used by later calls while cp_options_t.update_variant is 0.  results (may
 * be NULL) receives one row per lattice group; returns the number of groups
 * or a negative CP_E* code.  Synchronous.
 */
#define CP_UPDATE_VARIANTS 5
#define CP_TUNE_UPDATE 0
#define CP_TUNE_ASSEMBLE 1
typedef struct cp_tune_result_t {
    int32_t lattice;         /* lattice id of the group */
    int32_t chosen;          /* shape chosen, 0..CP_UPDATE_VARIANTS-1 */
    int32_t default_variant; /* the untuned rule's shape for the group */
    int32_t reserved;
    int64_t n_qp;            /* qps of the group */
    double median_ms[CP_UPDATE_VARIANTS]; /* median time of one launch per shape */
} cp_tune_result_t;
int cp_autotune(cp_handle* h, const double* d_in, int32_t path, int32_t reps, double min_gain,
                cp_tune_result_t* results, int32_t max_results);

/*
 * The autotuner's selection rule, host only: ms[v * reps + r] is repeat r of
 * shape v (non-finite or negative entries are failed launches and count as
 * missing).  Picks the shape with the smallest median (ties: the lower
 * index), but keeps default_variant unless the winner's median is below
 * (1 - min_gain) times the default's.  Returns -1 if no shape has a timing.
 */
int32_t cp_tune_select(int32_t n_variants, int32_t reps, const double* ms, int32_t default_variant,
                       double min_gain);

/* CUDA graphs captured (instantiated or updated) and launched by the handle
 * since its creation (cp_options_t.use_graphs). */
int cp_graph_stats(cp_handle* h, int64_t* captures, int64_t* launches);

/*
 * Continuous batching of independent requests (served RVE solves; no
 * counterpart in the reference, which solves one problem per process).  A
 * cp_batch is a queue on one device on which the calculatePlasticity work of
 * several handles runs as shared launches: one counting sort over all their
 * lattice groups and one update launch per lattice class (FCC / BCC / HCP
 * sized solves) over the qps of every handle, each qp with its own handle's
 * constants, history and displacement field.  Per-qp arithmetic is that of
 * the per-handle launches, so results do not depend on what shares a
 * launch.  The handles need cp_bind_dofs (the displacement u is gathered on
 * the device) and the sorted update.
 *   cp_batch_assemble: the Newton iteration's assembly at each handle's u
 *     (flag 1; Ke/Re into the handle's system); follow it with
 *     cp_newton_solve on each handle.
 *   cp_batch_post: the post-pass (flag 0) at each handle's u; follow it with
 *     cp_averages / cp_reorient / cp_commit as after
 *     cp_update_from_displacement.
 * F_e, F_r: n values, each handle's twin-rule scalars.  At most 64 handles'
 * worth of groups per launch (larger lists run as several).  Asynchronous:
 * ordered after the work already queued on each handle's stream and before
 * the work queued there afterwards.
 */
typedef struct cp_batch cp_batch;
int cp_batch_create(int32_t device, cp_batch** out);
void cp_batch_destroy(cp_batch* b);
const char* cp_batch_last_error(const cp_batch* b);
int64_t cp_batch_launches(const cp_batch* b); /* shared update launches issued so far */
int cp_batch_assemble(cp_batch* b, cp_handle* const* hs, int32_t n, const double* F_e, const double* F_r);
int cp_batch_post(cp_batch* b, cp_handle* const* hs, int32_t n, const double* F_e, const double* F_r);

/* Wait for all work queued on the handle's stream. */
int cp_synchronize(cp_handle* h);

/* Diagnostics: when enabled, every update/assembly kernel launch is
 * bracketed by CUDA events on the handle's stream; cp_get_timing returns, per
 * lattice group (internal qp groups, one per lattice present), its lattice
 * id, qp count, number of timed launches and their summed duration in ms,
 * and the number of groups.  cp_set_timing resets the accumulators. */
int cp_set_timing(cp_handle* h, int32_t enable);
int cp_get_timing(cp_handle* h, int32_t max_groups, int32_t* lattice, int64_t* count,
                  int64_t* launches, double* total_ms);
/* The same for the element-contraction launches of the assembly calls:
 * kind 0 the FP64 contraction, kind 1 the tensor-core one. */
int cp_get_contract_timing(cp_handle* h, int32_t kind, int64_t* launches, double* total_ms);

/* Diagnostics: measured FP64 FMA throughput of the device (TFLOP/s), the
 * denominator of the FP64 roofline of the qp update (no counterpart in the
 * reference). */
int cp_measure_fp64_peak(int32_t device, double* tflops);

/* Diagnostics: make the next persistent Jacobi BiCG solves (cp_solver_t
 * kernel_mode 0 on small systems, or 2) wait at most wait_seconds at each
 * grid barrier (0: the default 1 s) and, with withhold_block >= 0, have that
 * block of the solve's grid never arrive, so that every wait runs out: the
 * solve then returns CP_E_CUDA ("a grid barrier of the solve timed out") and
 * the context stays usable.  (-1, 0) restores the normal solve.  No
 * counterpart in the reference. */
int cp_debug_barrier_test(cp_handle* h, int32_t withhold_block, double wait_seconds);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their own
 * device work (input uploads, output reads) with the *_device entry points. */
void* cp_stream(cp_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* CP_GPU_H */
