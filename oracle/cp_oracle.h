/*
 * cp_oracle.h -- CPU oracle for the crystal-plasticity qp hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain FP64 C++ restatement of the
 * reference algorithm (PRISMS-Plasticity v1.5.0, src/materialModels/
 * crystalPlasticity/ *.cc), used by tests/, __graft_entry__.smoke() and the
 * bench's CPU-baseline leg as the checker.  The product (plasticity_b200/)
 * never links or calls it.
 *
 * The reference itself cannot be built here (it needs deal.II, PETSc, p4est,
 * MPI and LAPACK), so its third-party kernels are restated from their
 * published algorithms:
 *   LAPACKFullMatrix::compute_inverse_svd(0.0)  -> one-sided Jacobi SVD pseudo-inverse
 *   LAPACKFullMatrix::compute_eigenvalues_symmetric -> cyclic Jacobi eigen-solver
 *   FullMatrix::invert -> cofactor formula (n<=3), Gauss-Jordan with partial pivoting
 * Parity of the per-qp oracle with the reference is pinned at the system level
 * by the reference's golden stress-strain curves (tests/compile_tests/...).
 *
 * State layout (one lattice per call, qp-major "AoS"):
 *   Fp/Fe: 9 per qp, s/W: nT per qp, rot/rotnew: 3, twinfrac: n_twin,
 *   slipfrac: n_slip, twin flag: int32.
 */
#ifndef CP_ORACLE_H
#define CP_ORACLE_H
#include <stdint.h>
#include "../include/cp_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_state {
    int64_t n_qp;
    double *Fp_conv, *Fe_conv, *s_conv, *W_conv, *rot_conv, *rotnew_conv,
        *twinfrac_conv, *slipfrac_conv;
    int32_t* twin_conv;
    double *Fp_iter, *Fe_iter, *s_iter, *W_iter, *rot_iter, *rotnew_iter,
        *twinfrac_iter, *slipfrac_iter;
    int32_t* twin_iter;
} or_state;

/* calculatePlasticity for qps [0, n_qp): F 9*n_qp; P,T 9*n_qp (nullable);
 * dPdF 81*n_qp when flag==1 (nullable); stats 8*n_qp and status n_qp
 * (nullable; same layouts as cp_get_stats / cp_update). */
int oracle_update(const cp_material_t* mat, const cp_options_t* opt,
                  const or_state* st, const double* F, int32_t flag,
                  double F_e, double F_r, double* P, double* T, double* dPdF,
                  int32_t* stats, int32_t* status, int32_t nthreads);

/* getElementalValues for n_cells cells (qp k = 8*cell+q).  gradN: per cell
 * 8*8*3 (or shared when uniform), JxW per cell 8 (or shared).  Writes Ke
 * 576*n_cells, Re 24*n_cells, and the qp Cauchy stress / F when non-null. */
int oracle_assemble(const cp_material_t* mat, const cp_options_t* opt,
                    const or_state* st, int64_t n_cells, const double* U,
                    const double* gradN, const double* JxW, int32_t uniform,
                    double F_e, double F_r, double* Ke, double* Re,
                    int32_t* stats, int32_t* status, int32_t nthreads);

/* rotnew_conv = rotnew_iter; reorient(); rotnew_iter = rotnew_conv
 * (updateAfterIncrement.cc:287-295, reorient.cc:18-96). */
int oracle_reorient(const or_state* st, int32_t nthreads);

/* building blocks, exported for unit tests */
void oracle_odfpoint(const double r[3], double R[9]);
void oracle_elasticmoduli(const double R[9], const double C[36], double out[36]);
int oracle_matrix_exponential(const double A[9], double out[9]);
int oracle_pinv_svd(const double* A, int n, double* Ainv);
int oracle_invert(const double* A, int n, double* Ainv);
void oracle_eig_sym3(const double C[9], double evals[3], double evecs[9]);
/* the parity build's pow (exported by every build, used by the parity build) */
double oracle_parity_pow(double x, double y);

#ifdef __cplusplus
}
#endif
#endif
