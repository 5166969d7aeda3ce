// cp_solve.cuh -- the Newton step's global system on the device: scatter of
// the element matrices and residuals into one CSR matrix and vector
// (ellipticBVP::assemble, src/ellipticBVP/assemble.cc:62-90, through
// constraints.distribute_local_to_global, :78), Dirichlet condensation
// (boundaryConditions.cc:453-497 / AffineConstraints with inhomogeneities) and
// the Jacobi-preconditioned Krylov solve of solveLinearSystem.cc:10-36
// (PETScWrappers::SolverBiCG + PreconditionJacobi), restated as plain CUDA.
//
// Layout: K is CSR (row_ptr int64, col int32, values FP64), rows = global dofs.
// The Q1 pattern is structurally symmetric, so tpos[p] (the position of entry
// (j, i) for entry p = (i, j)) turns K's values into K^T's in the same pattern.  Every
// reduction is two-stage with a fixed block count and a fixed final order, so
// a solve is deterministic for a given input.
#pragma once

#include <cstdint>

namespace cp {

constexpr int SOLVE_BLOCK = 256;
// node-triple SpMV: 5 resident 256-thread blocks per SM (launch bound 48
// registers) and a grid of one wave; measured against 8 blocks of 74
// registers (3 resident) on the 32^3 dual-phase RVE: 0.130 -> 0.122 s per increment
constexpr int SPMV3_MIN_BLOCKS = 5;
constexpr int SPMV3_GRID = 148 * SPMV3_MIN_BLOCKS;
constexpr int RED_BLOCKS = 296;  // 2 x 148 SMs

// ---- gather / scatter ----------------------------------------------------

// U_local[24 c + d] = u[cell_dofs[24 c + d]]  (getElementalValues.cc:31-33)
__global__ void gather_ulocal_kernel(const double* __restrict__ u, const int64_t* __restrict__ cell_dofs,
                                     int64_t n, double* __restrict__ Ul) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) Ul[t] = u[cell_dofs[t]];
}

// value p of the global matrix = sum of its element entries, in cell order:
// src[idx[ptr[p]..ptr[p+1])] (element entry index cell*576 + 24 d1 + d2, or
// cell*24 + d for the residual)
__global__ void scatter_sum_kernel(const double* __restrict__ src, const int64_t* __restrict__ ptr,
                                   const int64_t* __restrict__ idx, int64_t n, double* __restrict__ out) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double s = 0.0;
    for (int64_t q = ptr[p]; q < ptr[p + 1]; ++q) s += src[idx[q]];
    out[p] = s;
}

// ---- condensation --------------------------------------------------------

// x[con[j]] = v[j] (v null: zero); the other entries are left as they are
__global__ void constrained_vector_kernel(const int64_t* __restrict__ con, const double* __restrict__ v,
                                          int64_t n_con, double* __restrict__ x) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n_con) x[con[j]] = v ? v[j] : 0.0;
}

// rows and columns of constrained dofs become those of the identity
// (du = the prescribed increment there); rhs of a constrained row = its value
__global__ void condense_matrix_kernel(const int64_t* __restrict__ row_ptr, const int* __restrict__ col,
                                       const unsigned char* __restrict__ cmask, int64_t n, double* __restrict__ vals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool ci = cmask[i];
    for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
        const int j = col[p];
        if (ci || cmask[j]) vals[p] = (ci && j == i) ? 1.0 : 0.0;
    }
}

// rhs = R - K dc on free rows, dc on constrained rows (K still unmodified)
__global__ void condense_rhs_kernel(const double* __restrict__ R, const double* __restrict__ Kdc,
                                    const double* __restrict__ dc, const unsigned char* __restrict__ cmask, int64_t n,
                                    double* __restrict__ rhs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rhs[i] = cmask[i] ? dc[i] : R[i] - Kdc[i];
}

// ---- sparse products (a warp per row: the row's entries load coalesced) ---

// y = K x
__global__ void spmv_kernel(const int64_t* __restrict__ row_ptr, const int* __restrict__ col,
                            const double* __restrict__ vals, const double* __restrict__ x, int64_t n,
                            double* __restrict__ y, const int* __restrict__ done) {
    if (done && *done) return;
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    double s = 0.0;
    for (int64_t p = row_ptr[row] + lane; p < row_ptr[row + 1]; p += 32)
        s += vals[p] * x[col[p]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[row] = s;
}

// ---- reductions ------------------------------------------------------------

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[SOLVE_BLOCK / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < SOLVE_BLOCK / 32; ++w) s += sh[w];
    __syncthreads();
    return s;  // valid in thread 0
}

// partial[b] = sum over the block's grid-stride share of a[i] * b[i]
__global__ void __launch_bounds__(SOLVE_BLOCK) dot_partial_kernel(const double* __restrict__ a,
                                                                  const double* __restrict__ b, int64_t n,
                                                                  double* __restrict__ partial,
                                                                  const int* __restrict__ done) {
    if (done && *done) return;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += a[i] * b[i];
    s = block_sum(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// out = sum of the RED_BLOCKS partials in a fixed order (one block)
__global__ void __launch_bounds__(SOLVE_BLOCK) dot_final_kernel(const double* __restrict__ partial,
                                                                double* __restrict__ out,
                                                                const int* __restrict__ done) {
    if (done && *done) return;
    double s = 0.0;
    for (int i = threadIdx.x; i < RED_BLOCKS; i += blockDim.x) s += partial[i];
    s = block_sum(s);
    if (threadIdx.x == 0) *out = s;
}

// ---- Krylov scalars and vector updates -------------------------------------
//
// Device scalars of one solve (sc[]):
enum SolveScalar {
    SC_RHO = 0,      // current rho
    SC_RHO_OLD,      // previous rho
    SC_DEN,          // p~ . q (BiCG) / r0 . v (BiCGStab)
    SC_RR,           // ||r||^2
    SC_BB,           // ||b||^2
    SC_ALPHA,
    SC_BETA,
    SC_OMEGA,        // BiCGStab
    SC_TS,           // t . s (BiCGStab)
    SC_TT,           // t . t (BiCGStab)
    SC_ZZ,           // ||M^-1 r||^2 (preconditioned norm)
    SC_COUNT
};

// info[]: 0 iterations done, 1 converged, 2 breakdown
// Convergence test after an iteration: ||r|| <= tol ||b|| (true residual), or
// ||M^-1 r|| <= tol ||b|| when precond_norm (the norm PETSc's BiCG tests).
__global__ void check_kernel(double* __restrict__ sc, double tol, int precond_norm, int* __restrict__ done,
                             int* __restrict__ info) {
    if (*done) return;
    info[0] += 1;
    const double rn = sqrt(precond_norm ? sc[SC_ZZ] : sc[SC_RR]);
    if (rn <= tol * sqrt(sc[SC_BB])) {
        info[1] = 1;
        *done = 1;
    }
}

// scalar bookkeeping between iterations: rho_old = rho
__global__ void shift_rho_kernel(double* __restrict__ sc, const int* __restrict__ done) {
    if (*done) return;
    sc[SC_RHO_OLD] = sc[SC_RHO];
}

// BiCGStab (right Jacobi preconditioning), van der Vorst's iteration:
// p = r + beta (p - omega v), beta = (rho / rho_old)(alpha / omega)
__global__ void bicgstab_dir_kernel(double* __restrict__ sc, const double* __restrict__ r,
                                    const double* __restrict__ v, int64_t n, int first, double* __restrict__ p,
                                    int* __restrict__ done, int* __restrict__ info) {
    if (*done) return;
    const double rho = sc[SC_RHO];
    if (rho == 0.0 || !isfinite(rho) || (!first && sc[SC_OMEGA] == 0.0)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            info[2] = 1;
            *done = 1;
        }
        return;
    }
    const double beta = first ? 0.0 : (rho / sc[SC_RHO_OLD]) * (sc[SC_ALPHA] / sc[SC_OMEGA]);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    p[i] = first ? r[i] : r[i] + beta * (p[i] - sc[SC_OMEGA] * v[i]);
}

// alpha = rho / (r0 . v); s = r - alpha v
__global__ void bicgstab_s_kernel(double* __restrict__ sc, const double* __restrict__ r,
                                  const double* __restrict__ v, int64_t n, double* __restrict__ s,
                                  int* __restrict__ done, int* __restrict__ info) {
    if (*done) return;
    const double den = sc[SC_DEN];
    if (den == 0.0 || !isfinite(den)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            info[2] = 1;
            *done = 1;
        }
        return;
    }
    const double alpha = sc[SC_RHO] / den;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) sc[SC_ALPHA] = alpha;
    if (i >= n) return;
    s[i] = r[i] - alpha * v[i];
}

// omega = (t . s) / (t . t); x += alpha p^ + omega s^; r = s - omega t
__global__ void bicgstab_x_kernel(double* __restrict__ sc, const double* __restrict__ ph,
                                  const double* __restrict__ sh, const double* __restrict__ s,
                                  const double* __restrict__ t, int64_t n, double* __restrict__ x,
                                  double* __restrict__ r, const int* __restrict__ done) {
    if (*done) return;
    const double tt = sc[SC_TT];
    const double omega = tt != 0.0 ? sc[SC_TS] / tt : 0.0;
    const double alpha = sc[SC_ALPHA];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) sc[SC_OMEGA] = omega;
    if (i >= n) return;
    x[i] += alpha * ph[i] + omega * sh[i];
    r[i] = s[i] - omega * t[i];
}

// y = a (copy)
__global__ void copy_kernel(const double* __restrict__ a, int64_t n, double* __restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = a[i];
}

// y = a .* dinv
__global__ void scale_kernel(const double* __restrict__ a, const double* __restrict__ dinv, int64_t n,
                             double* __restrict__ y, const int* __restrict__ done) {
    if (done && *done) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = a[i] * dinv[i];
}

// binv[9 b..] = inverse of node b's 3x3 diagonal block of K (entries at
// blkpos[9 b + 3 a + c]), by the adjugate; a singular or non-finite block
// falls back to the inverse of its diagonal (1 for a zero diagonal entry)
__global__ void block_setup_kernel(const double* __restrict__ vals, const int64_t* __restrict__ blkpos, int64_t nb,
                                   double* __restrict__ binv) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    double m[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) m[e] = vals[blkpos[9 * b + e]];
    const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    double* o = binv + 9 * b;
    if (det != 0.0 && isfinite(det)) {
        const double r = 1.0 / det;
        o[0] = c00 * r;
        o[1] = (m[2] * m[7] - m[1] * m[8]) * r;
        o[2] = (m[1] * m[5] - m[2] * m[4]) * r;
        o[3] = c01 * r;
        o[4] = (m[0] * m[8] - m[2] * m[6]) * r;
        o[5] = (m[2] * m[3] - m[0] * m[5]) * r;
        o[6] = c02 * r;
        o[7] = (m[1] * m[6] - m[0] * m[7]) * r;
        o[8] = (m[0] * m[4] - m[1] * m[3]) * r;
    } else {
#pragma unroll
        for (int e = 0; e < 9; ++e) o[e] = 0.0;
        o[0] = m[0] != 0.0 ? 1.0 / m[0] : 1.0;
        o[4] = m[4] != 0.0 ? 1.0 / m[4] : 1.0;
        o[8] = m[8] != 0.0 ? 1.0 / m[8] : 1.0;
    }
}

// valsT[p] = vals[tpos[p]]: the values of K^T in K's pattern
__global__ void transpose_values_kernel(const double* __restrict__ vals, const int64_t* __restrict__ tpos, int64_t nnz,
                                        double* __restrict__ valsT) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nnz) valsT[p] = vals[tpos[p]];
}

// dinv[i] = 1 / K_ii (zero diagonal -> 1, the row is then left unpreconditioned)
__global__ void jacobi_setup_kernel(const double* __restrict__ vals, const int64_t* __restrict__ diag_pos, int64_t n,
                                    double* __restrict__ dinv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = vals[diag_pos[i]];
    dinv[i] = d != 0.0 ? 1.0 / d : 1.0;
}

// u += du
__global__ void add_kernel(const double* __restrict__ du, int64_t n, double* __restrict__ u) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) u[i] += du[i];
}

// ---- fused BiCG iteration: 4 kernels, each reduction finished by the last
// block to arrive (its partial written, __threadfence, an atomic ticket; the
// last block sums the partials in block order, so the result is
// deterministic; nothing waits on another block)

// the block's partial of v into partial[blockIdx.x]; true in every thread of
// the block that finished last, which then holds sum(partial) in order in *out
__device__ __forceinline__ bool last_block_sum(double v, double* __restrict__ partial,
                                               unsigned int* __restrict__ ticket, double* __restrict__ out) {
    __shared__ bool is_last;
    const double s = block_sum(v);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = s;
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double f = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) f += ((volatile double*)partial)[b];
    f = block_sum(f);
    if (threadIdx.x == 0) {
        *out = f;
        *ticket = 0u;
    }
    return true;
}

// (1) z = r / d, z~ = r~ / d; rho = z . r~
__global__ void __launch_bounds__(SOLVE_BLOCK) fbicg_precond_kernel(
    const double* __restrict__ dinv, const double* __restrict__ r, const double* __restrict__ rt, int64_t n,
    double* __restrict__ z, double* __restrict__ zt, double* __restrict__ sc, double* __restrict__ partial,
    unsigned int* __restrict__ ticket, const int* __restrict__ done) {
    if (*done) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        const double a = r[i] * dinv[i], b = rt[i] * dinv[i];
        z[i] = a;
        zt[i] = b;
        v = a * rt[i];
    }
    last_block_sum(v, partial, ticket, sc + SC_RHO);
}

// (1, node blocks) z = B^-1 r and z~ = B^-T r~ per node (dofs blk[3 b..]);
// rho = z . r~
__global__ void __launch_bounds__(SOLVE_BLOCK) fbicg_precond_block_kernel(
    const double* __restrict__ binv, const int64_t* __restrict__ blk, const double* __restrict__ r,
    const double* __restrict__ rt, int64_t nb, double* __restrict__ z, double* __restrict__ zt,
    double* __restrict__ sc, double* __restrict__ partial, unsigned int* __restrict__ ticket,
    const int* __restrict__ done) {
    if (*done) return;
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (b < nb) {
        const int64_t g[3] = {blk[3 * b], blk[3 * b + 1], blk[3 * b + 2]};
        const double* B = binv + 9 * b;
        const double r0 = r[g[0]], r1 = r[g[1]], r2 = r[g[2]];
        const double t0 = rt[g[0]], t1 = rt[g[1]], t2 = rt[g[2]];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double za = B[3 * a] * r0 + B[3 * a + 1] * r1 + B[3 * a + 2] * r2;
            const double zta = B[a] * t0 + B[3 + a] * t1 + B[6 + a] * t2;
            z[g[a]] = za;
            zt[g[a]] = zta;
            v += za * (a == 0 ? t0 : (a == 1 ? t1 : t2));
        }
    }
    last_block_sum(v, partial, ticket, sc + SC_RHO);
}

// (2) p = z + beta p, p~ = z~ + beta p~ (beta = rho / rho_old, 0 on the first
// iteration); breakdown when rho is zero
__global__ void __launch_bounds__(SOLVE_BLOCK) fbicg_dir_kernel(
    const double* __restrict__ sc, const double* __restrict__ z, const double* __restrict__ zt, int64_t n, int first,
    double* __restrict__ p, double* __restrict__ pt, int* __restrict__ done, int* __restrict__ info) {
    if (*done) return;
    const double rho = sc[SC_RHO];
    if (rho == 0.0 || !isfinite(rho)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            info[2] = 1;
            *done = 1;
        }
        return;
    }
    const double beta = first ? 0.0 : rho / sc[SC_RHO_OLD];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // the first direction is z itself, as in the persistent solve: the old p
    // is not read (a solve that broke down may have left non-finite values)
    p[i] = first ? z[i] : z[i] + beta * p[i];
    pt[i] = first ? zt[i] : zt[i] + beta * pt[i];
}

// (3) q = K p and q~ = K^T p~ (a warp per row, both in one pass over the
// row; valsT[k] = K value of the transposed entry, gathered once per solve);
// den = p~ . q
__global__ void __launch_bounds__(SOLVE_BLOCK) fbicg_spmv_kernel(
    const int64_t* __restrict__ row_ptr, const int* __restrict__ col, const double* __restrict__ vals,
    const double* __restrict__ valsT, const double* __restrict__ p, const double* __restrict__ pt, int64_t n,
    double* __restrict__ q, double* __restrict__ qt, double* __restrict__ sc, double* __restrict__ partial,
    unsigned int* __restrict__ ticket, const int* __restrict__ done) {
    if (*done) return;
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    double v = 0.0;
    if (row < n) {
        double s = 0.0, st = 0.0;
        for (int64_t k = row_ptr[row] + lane; k < row_ptr[row + 1]; k += 32) {
            const int c = col[k];
            s += vals[k] * p[c];
            st += valsT[k] * pt[c];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            st += __shfl_xor_sync(0xffffffffu, st, o);
        }
        if (lane == 0) {
            q[row] = s;
            qt[row] = st;
            v = pt[row] * s;
        }
    }
    last_block_sum(v, partial, ticket, sc + SC_DEN);
}

// (3, node triples) the same when the three rows of every node (dofs 3t,
// 3t+1, 3t+2) share one column pattern, as a nodal vector field's stiffness
// does: a warp per node (grid-stride), each column index and p[c], p~[c]
// loaded once for the three rows.  Every row's sums run in the same order as
// in the row kernel (lane j takes entries j, j+32, ... of the row, then the
// same shuffle tree), so q and q~ are the same; den = p~ . q is summed node by
// node in a grid of fixed size.
__global__ void __launch_bounds__(SOLVE_BLOCK, SPMV3_MIN_BLOCKS) fbicg_spmv3_kernel(
    const int64_t* __restrict__ row_ptr, const int* __restrict__ col, const double* __restrict__ vals,
    const double* __restrict__ valsT, const double* __restrict__ p, const double* __restrict__ pt, int64_t n,
    double* __restrict__ q, double* __restrict__ qt, double* __restrict__ sc, double* __restrict__ partial,
    unsigned int* __restrict__ ticket, const int* __restrict__ done) {
    if (*done) return;
    const int64_t nt = n / 3;
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    double v = 0.0;
    for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nt; t += nw) {
        const int64_t k0 = row_ptr[3 * t];
        const int64_t len = row_ptr[3 * t + 1] - k0;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, u0 = 0.0, u1 = 0.0, u2 = 0.0;
        for (int64_t j = lane; j < len; j += 32) {
            const int c = col[k0 + j];
            const double pc = p[c], tc = pt[c];
            s0 += vals[k0 + j] * pc;
            s1 += vals[k0 + len + j] * pc;
            s2 += vals[k0 + 2 * len + j] * pc;
            u0 += valsT[k0 + j] * tc;
            u1 += valsT[k0 + len + j] * tc;
            u2 += valsT[k0 + 2 * len + j] * tc;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            u0 += __shfl_xor_sync(0xffffffffu, u0, o);
            u1 += __shfl_xor_sync(0xffffffffu, u1, o);
            u2 += __shfl_xor_sync(0xffffffffu, u2, o);
        }
        if (lane == 0) {
            q[3 * t] = s0;
            q[3 * t + 1] = s1;
            q[3 * t + 2] = s2;
            qt[3 * t] = u0;
            qt[3 * t + 1] = u1;
            qt[3 * t + 2] = u2;
            v += pt[3 * t] * s0 + pt[3 * t + 1] * s1 + pt[3 * t + 2] * s2;
        }
    }
    last_block_sum(v, partial, ticket, sc + SC_DEN);
}

// ---- the whole Jacobi BiCG solve in one cooperative launch -----------------
//
// For systems small enough that the four kernels of an iteration are bound by
// launch latency and host polling: one launch (cudaLaunchCooperativeKernel,
// so every block is resident) iterates to convergence, the iteration cap or a
// breakdown.  Same recurrence as the four kernels above; the phases of an
// iteration are separated by grid barriers, two per iteration:
//   [B+C] p = z + beta p, p~ = z~ + beta p~ (formed where the SpMV reads them,
//         double-buffered), q = K p, q~ = K^T p~, den = p~ . q;
//   [D] x, r, r~ updates, ||r||^2, and the next z = r / d, z~ = r~ / d,
//       rho = z . r~ (the first iteration's rho before the loop).
// A reduction writes one partial per block; after the barrier every block
// sums all partials in the same fixed order, so all blocks hold the same
// scalar and the result does not depend on timing.  Values another block
// wrote in this launch (z, z~, p, p~, q, q~, the partials) are read through L2
// (ld.global.cg), never the non-coherent or L1 paths.
//
// The barrier is a counter and a generation word.  Its wait is bounded: after
// PBICG_WAIT_NS of the global timer (or PBICG_SPIN_LIMIT polls) it raises err
// and returns, and every block leaves at its next barrier once err is set, so
// no launch can wait forever.
constexpr long long PBICG_SPIN_LIMIT = 1ll << 30;  // a backstop only: the timer ends a wait first
constexpr unsigned long long PBICG_WAIT_NS = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct PbicgArgs {
    const int64_t* row_ptr;
    const int* col;
    const double* vals;
    const double* valsT;
    const double* dinv;
    int64_t n;
    int triples;       // rows 3t..3t+2 share one column pattern
    int precond_norm;  // test ||M^-1 r|| instead of ||r||
    int max_iter;
    double tol;
    double bnorm;  // ||b||
    double *x, *r, *rt, *z, *zt, *p, *pt, *q, *qt;
    double *p2, *pt2;  // second buffers of the direction pair
    double* partial;   // 3 x gridDim.x: rho, den, ||r||^2
    unsigned* bar;     // [0] arrivals, [1] generation
    int* info;         // [0] iterations, [1] converged, [2] breakdown
    int* err;          // barrier timeout
    double* sc;        // final scalars (SC_RR / SC_ZZ)
    unsigned long long wait_ns;  // bound of one barrier wait
    int withhold;      // diagnostics: this block never arrives at a barrier (-1: none)
};

__device__ __forceinline__ bool pbicg_barrier(unsigned* bar, int* err, unsigned long long wait_ns = PBICG_WAIT_NS,
                                              int withhold = -1) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        // (a withheld block skips its arrival and waits like the others, so
        // every wait of the barrier runs out)
        if ((int)blockIdx.x != withhold && atomicAdd(bar, 1u) == gridDim.x - 1) {
            bar[0] = 0u;
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            long long spins = 0;
            while (*gen == g) {
                if (++spins > PBICG_SPIN_LIMIT || *(volatile int*)err || global_ns() - t0 > wait_ns) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int*)err == 0;
}

// sum of partial[0 .. gridDim.x) in a fixed order (the same in every block)
__device__ __forceinline__ double pbicg_allsum(const double* partial) {
    __shared__ double total;
    double f = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) f += __ldcg(partial + b);
    f = block_sum(f);
    if (threadIdx.x == 0) total = f;
    __syncthreads();
    const double t = total;
    __syncthreads();
    return t;
}

__device__ __forceinline__ void pbicg_put(double v, double* partial) {
    const double s = block_sum(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// block_sum of two values with one pass through shared memory (the same
// shuffle tree and warp order per value as block_sum)
__device__ __forceinline__ void block_sum2(double v0, double v1, double& s0, double& s1) {
    __shared__ double sh2[2][SOLVE_BLOCK / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_xor_sync(0xffffffffu, v0, o);
        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh2[0][threadIdx.x >> 5] = v0;
        sh2[1][threadIdx.x >> 5] = v1;
    }
    __syncthreads();
    s0 = 0.0;
    s1 = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < SOLVE_BLOCK / 32; ++w) {
            s0 += sh2[0][w];
            s1 += sh2[1][w];
        }
    __syncthreads();
}

// pbicg_put / pbicg_allsum for two partial rows at once
__device__ __forceinline__ void pbicg_put2(double v0, double v1, double* partial0, double* partial1) {
    double s0, s1;
    block_sum2(v0, v1, s0, s1);
    if (threadIdx.x == 0) {
        partial0[blockIdx.x] = s0;
        partial1[blockIdx.x] = s1;
    }
}
__device__ __forceinline__ void pbicg_allsum2(const double* partial0, const double* partial1, double& t0,
                                              double& t1) {
    __shared__ double total2[2];
    double f0 = 0.0, f1 = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        f0 += __ldcg(partial0 + b);
        f1 += __ldcg(partial1 + b);
    }
    double s0, s1;
    block_sum2(f0, f1, s0, s1);
    if (threadIdx.x == 0) {
        total2[0] = s0;
        total2[1] = s1;
    }
    __syncthreads();
    t0 = total2[0];
    t1 = total2[1];
    __syncthreads();
}

__global__ void __launch_bounds__(SOLVE_BLOCK) pbicg_kernel(PbicgArgs a) {
    const int64_t n = a.n;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const int64_t warp = tid >> 5, nwarps = nthreads >> 5;
    // one partial row per reduced quantity: a row is rewritten only after
    // every block has passed the barrier that follows its last read
    double* P0 = a.partial;                  // rho
    double* P1 = a.partial + gridDim.x;      // den
    double* P2 = a.partial + 2 * gridDim.x;  // ||r||^2 (or ||M^-1 r||^2)
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    // [A] of the first iteration
    {
        double v = 0.0;
        for (int64_t i = tid; i < n; i += nthreads) {
            const double zi = a.r[i] * a.dinv[i], zti = a.rt[i] * a.dinv[i];
            a.z[i] = zi;
            a.zt[i] = zti;
            v += zi * a.rt[i];
        }
        pbicg_put(v, P0);
    }
    if (!pbicg_barrier(a.bar, a.err, a.wait_ns, a.withhold)) return;
    double rho = pbicg_allsum(P0), rho_old = 1.0;
    for (int k = 0; k < a.max_iter; ++k) {
        if (rho == 0.0 || !isfinite(rho)) {
            if (lead) a.info[2] = 1;
            return;
        }
        // [B+C] the directions p = z + beta p_old, p~ = z~ + beta p~_old are
        // formed where the SpMV needs them (every warp for the columns it
        // reads, the same expression as the four-kernel iteration's), so no
        // barrier separates them from the SpMV; the owner of a row stores its
        // p, p~ into the other buffer of the pair for [D] and the next
        // iteration
        const double beta = k == 0 ? 0.0 : rho / rho_old;
        const double* po = (k & 1) ? a.p2 : a.p;
        const double* pto = (k & 1) ? a.pt2 : a.pt;
        double* pn = (k & 1) ? a.p : a.p2;
        double* ptn = (k & 1) ? a.pt : a.pt2;
        auto dir = [&](const double* zv, const double* old, int64_t c) {
            return k == 0 ? __ldcg(zv + c) : __ldcg(zv + c) + beta * __ldcg(old + c);
        };
        {
            double v = 0.0;
            if (a.triples) {
                for (int64_t t = warp; t < n / 3; t += nwarps) {
                    const int64_t k0 = a.row_ptr[3 * t];
                    const int64_t len = a.row_ptr[3 * t + 1] - k0;
                    double s0 = 0.0, s1 = 0.0, s2 = 0.0, u0 = 0.0, u1 = 0.0, u2 = 0.0;
                    for (int64_t j = lane; j < len; j += 32) {
                        const int c = a.col[k0 + j];
                        const double pc = dir(a.z, po, c), tc = dir(a.zt, pto, c);
                        s0 += a.vals[k0 + j] * pc;
                        s1 += a.vals[k0 + len + j] * pc;
                        s2 += a.vals[k0 + 2 * len + j] * pc;
                        u0 += a.valsT[k0 + j] * tc;
                        u1 += a.valsT[k0 + len + j] * tc;
                        u2 += a.valsT[k0 + 2 * len + j] * tc;
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
                        u0 += __shfl_xor_sync(0xffffffffu, u0, o);
                        u1 += __shfl_xor_sync(0xffffffffu, u1, o);
                        u2 += __shfl_xor_sync(0xffffffffu, u2, o);
                    }
                    if (lane == 0) {
                        const double t0 = dir(a.zt, pto, 3 * t), t1 = dir(a.zt, pto, 3 * t + 1),
                                     t2 = dir(a.zt, pto, 3 * t + 2);
                        pn[3 * t] = dir(a.z, po, 3 * t);
                        pn[3 * t + 1] = dir(a.z, po, 3 * t + 1);
                        pn[3 * t + 2] = dir(a.z, po, 3 * t + 2);
                        ptn[3 * t] = t0;
                        ptn[3 * t + 1] = t1;
                        ptn[3 * t + 2] = t2;
                        a.q[3 * t] = s0;
                        a.q[3 * t + 1] = s1;
                        a.q[3 * t + 2] = s2;
                        a.qt[3 * t] = u0;
                        a.qt[3 * t + 1] = u1;
                        a.qt[3 * t + 2] = u2;
                        v += t0 * s0 + t1 * s1 + t2 * s2;
                    }
                }
            } else {
                for (int64_t row = warp; row < n; row += nwarps) {
                    double s = 0.0, st = 0.0;
                    for (int64_t kk = a.row_ptr[row] + lane; kk < a.row_ptr[row + 1]; kk += 32) {
                        const int c = a.col[kk];
                        s += a.vals[kk] * dir(a.z, po, c);
                        st += a.valsT[kk] * dir(a.zt, pto, c);
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        s += __shfl_xor_sync(0xffffffffu, s, o);
                        st += __shfl_xor_sync(0xffffffffu, st, o);
                    }
                    if (lane == 0) {
                        const double tr = dir(a.zt, pto, row);
                        pn[row] = dir(a.z, po, row);
                        ptn[row] = tr;
                        a.q[row] = s;
                        a.qt[row] = st;
                        v += tr * s;
                    }
                }
            }
            pbicg_put(v, P1);
        }
        if (!pbicg_barrier(a.bar, a.err, a.wait_ns, a.withhold)) return;
        const double den = pbicg_allsum(P1);
        if (den == 0.0 || !isfinite(den)) {
            if (lead) a.info[2] = 1;
            return;
        }
        // [D] and the next [A]
        const double alpha = rho / den;
        {
            double vr = 0.0, vz = 0.0;
            for (int64_t i = tid; i < n; i += nthreads) {
                a.x[i] += alpha * __ldcg(pn + i);
                const double ri = a.r[i] - alpha * __ldcg(a.q + i);
                const double rti = a.rt[i] - alpha * __ldcg(a.qt + i);
                a.r[i] = ri;
                a.rt[i] = rti;
                const double zi = ri * a.dinv[i], zti = rti * a.dinv[i];
                a.z[i] = zi;
                a.zt[i] = zti;
                vr += a.precond_norm ? zi * zi : ri * ri;
                vz += zi * rti;
            }
            pbicg_put2(vr, vz, P2, P0);
        }
        if (!pbicg_barrier(a.bar, a.err, a.wait_ns, a.withhold)) return;
        double rr;
        rho_old = rho;
        pbicg_allsum2(P2, P0, rr, rho);
        if (lead) {
            a.info[0] = k + 1;
            a.sc[a.precond_norm ? SC_ZZ : SC_RR] = rr;
        }
        if (sqrt(rr) <= a.tol * a.bnorm) {
            if (lead) a.info[1] = 1;
            return;
        }
    }
}

// (4) x += alpha p; r -= alpha q; r~ -= alpha q~ (alpha = rho / den);
// ||r||^2 (and ||M^-1 r||^2), then the convergence test in the last block;
// rho_old = rho for the next iteration
__global__ void __launch_bounds__(SOLVE_BLOCK) fbicg_step_kernel(
    double* __restrict__ sc, const double* __restrict__ p, const double* __restrict__ q, const double* __restrict__ qt,
    const double* __restrict__ dinv, int64_t n, double tol, int precond_norm, double* __restrict__ x,
    double* __restrict__ r, double* __restrict__ rt, double* __restrict__ partial, unsigned int* __restrict__ ticket,
    int* __restrict__ done, int* __restrict__ info) {
    if (*done) return;
    const double den = sc[SC_DEN];
    if (den == 0.0 || !isfinite(den)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            info[2] = 1;
            *done = 1;
        }
        return;
    }
    const double alpha = sc[SC_RHO] / den;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        rt[i] -= alpha * qt[i];
        v = precond_norm ? (ri * dinv[i]) * (ri * dinv[i]) : ri * ri;
    }
    if (last_block_sum(v, partial, ticket, sc + (precond_norm ? SC_ZZ : SC_RR)) && threadIdx.x == 0) {
        info[0] += 1;
        const double rn = sqrt(sc[precond_norm ? SC_ZZ : SC_RR]);
        if (rn <= tol * sqrt(sc[SC_BB])) {
            info[1] = 1;
            *done = 1;
        }
        sc[SC_RHO_OLD] = sc[SC_RHO];
    }
}

}  // namespace cp
