// cp_kernels.cuh -- the CUDA kernels behind include/cp_gpu.h.
#pragma once

#include "cp_qp.cuh"

namespace cp {

constexpr int QP_BLOCK = 128;  // threads per block of the qp kernels (16 Q1 cells)

// calculatePlasticity for every qp of one lattice group (thread per qp).
// F, P, T, dPdF, status, stats are in the caller's qp order.
template <int NT, int PMAX>
__global__ void __launch_bounds__(QP_BLOCK) update_kernel(const LatDev* __restrict__ L, Opts o, GroupDev g,
                                                          const double* __restrict__ F, int flag, double F_e,
                                                          double F_r, double* __restrict__ P, double* __restrict__ T,
                                                          double* __restrict__ dPdF, int32_t* __restrict__ status,
                                                          int32_t* __restrict__ stats, double* __restrict__ keepF,
                                                          double* __restrict__ keepT, int lattice_id) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.count) return;
    const int64_t k = g.qp[i];
    M3 Fk;
#pragma unroll
    for (int c = 0; c < 9; ++c) Fk.a[c] = F[9 * k + c];
    double Tl[9];
    QpOut out;
    out.P = P ? P + 9 * k : nullptr;
    out.T = (T || keepT) ? Tl : nullptr;
    out.dPdF = (dPdF && flag == 1) ? dPdF + 81 * k : nullptr;
    out.scale = 1.0;
    const int st = qp_update<NT, PMAX>(*L, o, g, i, Fk, flag, F_e, F_r, out, stats ? stats + 8 * k : nullptr,
                                       lattice_id);
    if (T)
#pragma unroll
        for (int c = 0; c < 9; ++c) T[9 * k + c] = Tl[c];
    if (keepT) {
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            keepT[9 * k + c] = Tl[c];
            keepF[9 * k + c] = Fk.a[c];
        }
    }
    if (status) status[k] = st;
}

// getElementalValues for every cell of one lattice group: the 8 qps of a
// cell are 8 consecutive threads; each computes F from the cell's nodal
// displacements, runs the update with the tangent, and parks JxW*P and
// JxW*dPdF in shared memory; then thread (cell, node a) contracts rows
// 3a..3a+2 of Ke and Re (getElementalValues.cc:127-163).
template <int NT, int PMAX>
__global__ void __launch_bounds__(QP_BLOCK) assemble_kernel(const LatDev* __restrict__ L, Opts o, GroupDev g,
                                                            const double* __restrict__ U,
                                                            const double* __restrict__ gradN,
                                                            const double* __restrict__ JxW, int uniform,
                                                            double F_e, double F_r, double* __restrict__ Ke,
                                                            double* __restrict__ Re, int32_t* __restrict__ status,
                                                            int32_t* __restrict__ stats, int lattice_id) {
    extern __shared__ double smem[];
    double* sP = smem;                       // [QP_BLOCK][9]
    double* sD = smem + QP_BLOCK * 9;        // [QP_BLOCK][81]
    const int tid = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + tid;
    const bool active = i < g.count;
    int64_t k = 0, cell = 0;
    const int q = tid & 7;
    if (active) {
        k = g.qp[i];
        cell = k >> 3;
        const double* gq = (uniform ? gradN : gradN + cell * 192) + q * 24;  // [q][a][3]
        const double w = uniform ? JxW[q] : JxW[cell * 8 + q];
        const double* Uc = U + 24 * cell;
        M3 F = zero3();
        for (int d = 0; d < 24; ++d) {
            const int ci = d % 3, a = d / 3;
            const double ud = Uc[d];
#pragma unroll
            for (int j = 0; j < 3; ++j) F(ci, j) += ud * gq[a * 3 + j];
        }
        F(0, 0) += 1.0;
        F(1, 1) += 1.0;
        F(2, 2) += 1.0;
        QpOut out;
        out.P = sP + tid * 9;
        out.T = nullptr;
        out.dPdF = sD + tid * 81;
        out.scale = w;
        const int st = qp_update<NT, PMAX>(*L, o, g, i, F, 1, F_e, F_r, out, stats ? stats + 8 * k : nullptr,
                                           lattice_id);
        if (status) status[k] = st;
    }
    __syncthreads();
    if (!active) return;
    // contraction: this thread owns node a = q of its cell
    const int base = tid & ~7;
    const int a1 = q;
    const double* g0 = uniform ? gradN : gradN + cell * 192;
    double K[3][24];
    double Rl[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 24; ++c) K[r][c] = 0.0;
    for (int qq = 0; qq < 8; ++qq) {
        const double* gq = g0 + qq * 24;
        const double* Pq = sP + (base + qq) * 9;
        const double* Dq = sD + (base + qq) * 81;
        const double g1x = gq[a1 * 3], g1y = gq[a1 * 3 + 1], g1z = gq[a1 * 3 + 2];
#pragma unroll
        for (int ci = 0; ci < 3; ++ci) {
            Rl[ci] -= g1x * Pq[3 * ci] + g1y * Pq[3 * ci + 1] + g1z * Pq[3 * ci + 2];
#pragma unroll
            for (int cj = 0; cj < 3; ++cj) {
                // t_l = sum_k g1_k dPdF[ci][k][cj][l]
                double t[3];
#pragma unroll
                for (int l = 0; l < 3; ++l)
                    t[l] = g1x * Dq[27 * ci + 0 + 3 * cj + l] + g1y * Dq[27 * ci + 9 + 3 * cj + l] +
                           g1z * Dq[27 * ci + 18 + 3 * cj + l];
#pragma unroll
                for (int a2 = 0; a2 < 8; ++a2)
                    K[ci][3 * a2 + cj] += t[0] * gq[a2 * 3] + t[1] * gq[a2 * 3 + 1] + t[2] * gq[a2 * 3 + 2];
            }
        }
    }
    double* Kc = Ke + cell * 576 + (3 * a1) * 24;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 24; ++c) Kc[r * 24 + c] = K[r][c];
#pragma unroll
    for (int r = 0; r < 3; ++r) Re[cell * 24 + 3 * a1 + r] = Rl[r];
}

// history initialisation (init.cc:198-330)
__global__ void init_state_kernel(const LatDev* __restrict__ L, GroupDev g, const double* __restrict__ rod);

// reorient() for one group (reorient.cc:18-96), bracketed by the rotnew
// copies of updateAfterIncrement.cc:287 and :295.
__global__ void reorient_kernel(GroupDev g);

// per-block partial sums of the volume averages (updateAfterIncrement.cc:119-126,218-235)
__global__ void averages_partial_kernel(const LatDev* __restrict__ L, GroupDev g, const double* __restrict__ keepF,
                                        const double* __restrict__ keepT, const double* __restrict__ JxW,
                                        int uniform, double* __restrict__ partial);
__global__ void averages_final_kernel(const double* __restrict__ partial, int nblocks, double* __restrict__ out);

}  // namespace cp
