// cp_solve32.cuh -- the mixed-precision Newton-step solve: the condensed
// system K du = b with K assembled from the FP32 tensor-core element
// matrices (cp_tc.cu), solved by FP64 iterative refinement around FP32
// Jacobi BiCG (solveLinearSystem.cc:10-36 runs PETSc BiCG + Jacobi in FP64).
//
//   x = 0, r = b (FP64)
//   repeat: solve K d = r approximately in FP32 (BiCG, Jacobi, to a relative
//           residual of the inner tolerance), x += d (FP64),
//           r = b - K x (FP64 products of K's FP32 values), until
//           ||r|| <= tol ||b||.
//
// A pass is kept when it cuts ||r|| at least ten-fold.  FP32 BiCG stagnates
// on badly conditioned steps (where FP64 Jacobi BiCG needs thousands of
// iterations); the first FP32 pass that does not cut the residual hands the
// rest of the solve to FP64 BiCG passes on the same FP32-assembled matrix.
//
// The inner iteration is the four-kernel fused BiCG of cp_solve.cuh with
// FP32 vectors and matrix values; its scalars (rho, den, alpha, beta, norms)
// are FP64 and its reductions sum FP64 partials in a fixed order, as there.
// An FP32 SpMV moves 12 bytes per non-zero (value, transposed value, column)
// against 20 in FP64.
#pragma once

#include "cp_solve.cuh"

namespace cp {

// vals32[p] = sum of the FP32 element entries of matrix entry p, summed in
// FP64 in cell order, rounded once to FP32
__global__ void scatter_sum_f32_kernel(const float* __restrict__ src, const int64_t* __restrict__ ptr,
                                       const int64_t* __restrict__ idx, int64_t n, float* __restrict__ out) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double s = 0.0;
    for (int64_t q = ptr[p]; q < ptr[p + 1]; ++q) s += (double)src[idx[q]];
    out[p] = (float)s;
}

__global__ void condense_matrix_f32_kernel(const int64_t* __restrict__ row_ptr, const int* __restrict__ col,
                                           const unsigned char* __restrict__ cmask, int64_t n,
                                           float* __restrict__ vals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool ci = cmask[i];
    for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
        const int j = col[p];
        if (ci || cmask[j]) vals[p] = (ci && j == i) ? 1.0f : 0.0f;
    }
}

__global__ void transpose_values_f32_kernel(const float* __restrict__ vals, const int64_t* __restrict__ tpos,
                                            int64_t nnz, float* __restrict__ valsT) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nnz) valsT[p] = vals[tpos[p]];
}

__global__ void jacobi_setup_f32_kernel(const float* __restrict__ vals, const int64_t* __restrict__ diag_pos,
                                        int64_t n, float* __restrict__ dinv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float d = vals[diag_pos[i]];
    dinv[i] = d != 0.0f ? 1.0f / d : 1.0f;
}

// y = K x with FP32 values and FP64 x, y (a warp per row, FP64 sums): the
// condensation's K dc and the refinement's residual r = b - K x (b non-null)
__global__ void spmv_f32_kernel(const int64_t* __restrict__ row_ptr, const int* __restrict__ col,
                                const float* __restrict__ vals, const double* __restrict__ x, int64_t n,
                                const double* __restrict__ b, double* __restrict__ y) {
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    double s = 0.0;
    for (int64_t p = row_ptr[row] + lane; p < row_ptr[row + 1]; p += 32) s += (double)vals[p] * x[col[p]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[row] = b ? b[row] - s : s;
}

// inner solve start: r32 = r~32 = r64, the inner solution d = 0
__global__ void mixed_start_kernel(const double* __restrict__ r64, int64_t n, float* __restrict__ r,
                                   float* __restrict__ rt, float* __restrict__ d) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = (float)r64[i];
    r[i] = v;
    rt[i] = v;
    d[i] = 0.0f;
}

// a refinement pass's candidate x_try = x + d (d FP32 from an FP32 inner
// solve, or FP64 from an FP64 one)
__global__ void mixed_try_kernel(const double* __restrict__ x, const float* __restrict__ d32,
                                 const double* __restrict__ d64, int64_t n, double* __restrict__ x_try) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x_try[i] = x[i] + (d32 ? (double)d32[i] : d64[i]);
}

// y = (double) x: K's FP32 values for an FP64 inner solve
__global__ void promote_f32_kernel(const float* __restrict__ x, int64_t n, double* __restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = (double)x[i];
}

// ||v||^2 of an FP32 vector into sc[slot] (the inner solve's reference norm)
__global__ void __launch_bounds__(SOLVE_BLOCK) norm2_f32_kernel(const float* __restrict__ v, int64_t n,
                                                                 double* __restrict__ sc, int slot,
                                                                 double* __restrict__ partial,
                                                                 unsigned int* __restrict__ ticket) {
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = (double)v[i];
        s += x * x;
    }
    last_block_sum(s, partial, ticket, sc + slot);
}

// (1) z = r / d, z~ = r~ / d (FP32); rho = z . r~ (FP64)
__global__ void __launch_bounds__(SOLVE_BLOCK) mbicg_precond_kernel(
    const float* __restrict__ dinv, const float* __restrict__ r, const float* __restrict__ rt, int64_t n,
    float* __restrict__ z, float* __restrict__ zt, double* __restrict__ sc, double* __restrict__ partial,
    unsigned int* __restrict__ ticket, const int* __restrict__ done) {
    if (*done) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        const float a = r[i] * dinv[i], b = rt[i] * dinv[i];
        z[i] = a;
        zt[i] = b;
        v = (double)a * (double)rt[i];
    }
    last_block_sum(v, partial, ticket, sc + SC_RHO);
}

// (2) p = z + beta p, p~ = z~ + beta p~
__global__ void __launch_bounds__(SOLVE_BLOCK) mbicg_dir_kernel(
    const double* __restrict__ sc, const float* __restrict__ z, const float* __restrict__ zt, int64_t n, int first,
    float* __restrict__ p, float* __restrict__ pt, int* __restrict__ done, int* __restrict__ info) {
    if (*done) return;
    const double rho = sc[SC_RHO];
    if (rho == 0.0 || !isfinite(rho)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            info[2] = 1;
            *done = 1;
        }
        return;
    }
    const float beta = first ? 0.0f : (float)(rho / sc[SC_RHO_OLD]);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // the first direction is z itself: the old p is never read then (it may be
    // memory no solve has written yet, and 0 * NaN would poison every pass)
    p[i] = first ? z[i] : z[i] + beta * p[i];
    pt[i] = first ? zt[i] : zt[i] + beta * pt[i];
}

// (3) q = K p, q~ = K^T p~ (FP32), a warp per row; den = p~ . q (FP64)
__global__ void __launch_bounds__(SOLVE_BLOCK) mbicg_spmv_kernel(
    const int64_t* __restrict__ row_ptr, const int* __restrict__ col, const float* __restrict__ vals,
    const float* __restrict__ valsT, const float* __restrict__ p, const float* __restrict__ pt, int64_t n,
    float* __restrict__ q, float* __restrict__ qt, double* __restrict__ sc, double* __restrict__ partial,
    unsigned int* __restrict__ ticket, const int* __restrict__ done) {
    if (*done) return;
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    double v = 0.0;
    if (row < n) {
        float s = 0.0f, st = 0.0f;
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
            v = (double)pt[row] * (double)s;
        }
    }
    last_block_sum(v, partial, ticket, sc + SC_DEN);
}

// (3, node triples) the same, a warp per node, each column index and p[c],
// p~[c] loaded once for the node's three rows
__global__ void __launch_bounds__(SOLVE_BLOCK, SPMV3_MIN_BLOCKS) mbicg_spmv3_kernel(
    const int64_t* __restrict__ row_ptr, const int* __restrict__ col, const float* __restrict__ vals,
    const float* __restrict__ valsT, const float* __restrict__ p, const float* __restrict__ pt, int64_t n,
    float* __restrict__ q, float* __restrict__ qt, double* __restrict__ sc, double* __restrict__ partial,
    unsigned int* __restrict__ ticket, const int* __restrict__ done) {
    if (*done) return;
    const int64_t nt = n / 3;
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    double v = 0.0;
    for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nt; t += nw) {
        const int64_t k0 = row_ptr[3 * t];
        const int64_t len = row_ptr[3 * t + 1] - k0;
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, u0 = 0.0f, u1 = 0.0f, u2 = 0.0f;
        for (int64_t j = lane; j < len; j += 32) {
            const int c = col[k0 + j];
            const float pc = p[c], tc = pt[c];
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
            v += (double)pt[3 * t] * s0 + (double)pt[3 * t + 1] * s1 + (double)pt[3 * t + 2] * s2;
        }
    }
    last_block_sum(v, partial, ticket, sc + SC_DEN);
}

// (4) d += alpha p; r -= alpha q; r~ -= alpha q~ (FP32); ||r||^2 (FP64) and
// the inner convergence test ||r|| <= tol ||r_start|| (sc[SC_BB] holds
// ||r_start||^2) in the last block
__global__ void __launch_bounds__(SOLVE_BLOCK) mbicg_step_kernel(
    double* __restrict__ sc, const float* __restrict__ p, const float* __restrict__ q, const float* __restrict__ qt,
    int64_t n, double tol, float* __restrict__ d, float* __restrict__ r, float* __restrict__ rt,
    double* __restrict__ partial, unsigned int* __restrict__ ticket, int* __restrict__ done, int* __restrict__ info) {
    if (*done) return;
    const double den = sc[SC_DEN];
    if (den == 0.0 || !isfinite(den)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            info[2] = 1;
            *done = 1;
        }
        return;
    }
    const float alpha = (float)(sc[SC_RHO] / den);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        d[i] += alpha * p[i];
        const float ri = r[i] - alpha * q[i];
        r[i] = ri;
        rt[i] -= alpha * qt[i];
        v = (double)ri * (double)ri;
    }
    if (last_block_sum(v, partial, ticket, sc + SC_RR) && threadIdx.x == 0) {
        info[0] += 1;
        if (sqrt(sc[SC_RR]) <= tol * sqrt(sc[SC_BB])) {
            info[1] = 1;
            *done = 1;
        }
        sc[SC_RHO_OLD] = sc[SC_RHO];
    }
}

}  // namespace cp
