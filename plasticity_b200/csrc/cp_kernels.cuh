// cp_kernels.cuh -- the CUDA kernels behind include/cp_gpu.h.
#pragma once

#include "cp_qp2.cuh"

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
            for (int j = 0; j < 3; ++j) F(ci, j) = fmad(ud, gq[a * 3 + j], F(ci, j));
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

// ---------------------------------------------------------------- sorted pipeline
// F of caller qp k from a caller array ...
struct FromArray {
    const double* __restrict__ F;
    __device__ __forceinline__ M3 operator()(int64_t k) const {
        M3 m;
#pragma unroll
        for (int c = 0; c < 9; ++c) m.a[c] = F[9 * k + c];
        return m;
    }
    __device__ __forceinline__ double weight(int64_t) const { return 1.0; }
};
// ... or from the cell's nodal displacements (getElementalValues.cc:129-138):
// qp k is Gauss point k % 8 of cell k / 8
struct FromMesh {
    const double* __restrict__ U;
    const double* __restrict__ gradN;
    const double* __restrict__ JxW;
    int uniform;
    __device__ __forceinline__ M3 operator()(int64_t k) const {
        const int64_t cell = k >> 3;
        const int q = (int)(k & 7);
        const double* gq = (uniform ? gradN : gradN + cell * 192) + q * 24;
        const double* Uc = U + 24 * cell;
        M3 F = zero3();
        for (int d = 0; d < 24; ++d) {
            const int ci = d % 3, a = d / 3;
            const double ud = Uc[d];
#pragma unroll
            for (int j = 0; j < 3; ++j) F(ci, j) = fmad(ud, gq[a * 3 + j], F(ci, j));
        }
        F(0, 0) += 1.0;
        F(1, 1) += 1.0;
        F(2, 2) += 1.0;
        return F;
    }
    __device__ __forceinline__ double weight(int64_t k) const { return uniform ? JxW[k & 7] : JxW[k]; }
};

// ---------------------------------------------------------------- batched launches
// One lattice group of one handle in a launch shared by several handles
// (continuous batching of served requests): its constants, history, F
// source (the cell's nodal displacements), sort buffers and outputs.  The
// groups of a launch are laid out block-aligned: group k owns
// ceil(m_k / blockDim) consecutive blocks, so no block spans two groups.
struct BatchDesc {
    const LatDev* L;
    Opts o;
    GroupDev g;
    FromMesh fm;
    unsigned char* key;
    int* hist;  // SORT_BUCKETS counts, then SORT_BUCKETS offsets
    int* perm;
    int64_t m;
    double F_e, F_r;
    double* stage;  // assembly: JxW P, JxW dP/dF (null in the post-pass)
    int32_t *status, *stats;
    double *keepF, *keepT;  // post-pass: F and T kept for the averages
    int lattice_id;
};
constexpr int CP_BATCH_MAX = 48;  // groups per batched launch (the launch parameter holds them by value)
struct BatchArgs {
    int n;
    int flag;
    BatchDesc d[CP_BATCH_MAX];
};

// the group owning this block (blocks of B threads, block-aligned layout)
// and the block's index within it; -1 past the last group
__device__ __forceinline__ int batch_group_of_block(const BatchArgs& a, int B, int64_t& local_block) {
    int64_t b = blockIdx.x;
    for (int k = 0; k < a.n; ++k) {
        const int64_t nb = (a.d[k].m + B - 1) / B;
        if (b < nb) {
            local_block = b;
            return k;
        }
        b -= nb;
    }
    return -1;
}

constexpr int SORT_BUCKETS = 64;

// sort key: bucket 63 - min(p0, 63), so ascending buckets = descending p0
// (over internal qps [i0, i0 + m) of the group)
template <class FSrc>
__global__ void __launch_bounds__(QP_BLOCK) classify_kernel(const LatDev* __restrict__ L, Opts o, GroupDev g, FSrc fs,
                                                            int64_t i0, int64_t m, unsigned char* __restrict__ key,
                                                            int* __restrict__ hist) {
    __shared__ int sh[SORT_BUCKETS];
    if (threadIdx.x < SORT_BUCKETS) sh[threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = i0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < i0 + m) {
        const int p0 = count_potentially_active(*L, o, g, i, fs(g.qp[i]));
        const int b = SORT_BUCKETS - 1 - (p0 < SORT_BUCKETS - 1 ? p0 : SORT_BUCKETS - 1);
        key[i] = (unsigned char)b;
        atomicAdd(&sh[b], 1);
    }
    __syncthreads();
    if (threadIdx.x < SORT_BUCKETS && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

#ifndef CP_TEMPLATES_ONLY  // the non-template kernels are defined in cp_api.cu
// exclusive scan of the bucket counts (one warp, SORT_BUCKETS = 64)
__global__ void bucket_scan_kernel(const int* __restrict__ hist, int* __restrict__ offs) {
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int b = 0; b < SORT_BUCKETS; ++b) {
            offs[b] = acc;
            acc += hist[b];
        }
    }
}

// scatter internal indices [i0, i0 + m) into bucket order, positions 0..m-1
// of perm (block-aggregated reservations)
__global__ void __launch_bounds__(256) bucket_scatter_kernel(const unsigned char* __restrict__ key, int64_t i0,
                                                             int64_t m, int* __restrict__ offs,
                                                             int* __restrict__ perm) {
    __shared__ int cnt[SORT_BUCKETS], base[SORT_BUCKETS];
    if (threadIdx.x < SORT_BUCKETS) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = i0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int b = 0, r = 0;
    if (i < i0 + m) {
        b = key[i];
        r = atomicAdd(&cnt[b], 1);
    }
    __syncthreads();
    if (threadIdx.x < SORT_BUCKETS) base[threadIdx.x] = cnt[threadIdx.x] ? atomicAdd(&offs[threadIdx.x], cnt[threadIdx.x]) : 0;
    __syncthreads();
    if (i < i0 + m) perm[base[b] + r] = (int)i;
}

#endif

// calculatePlasticity over m qps of one group in sorted order (thread j runs
// internal qp perm[j]).  Outputs by caller index k: P/T/dPdF/status/stats; with a
// non-null 'stage' (the assembly path) JxW*P and JxW*dP/dF go to stage[90k..].
// Threads run the qps in sorted order (descending potentially-active-set
// size): consecutive threads, and so the lanes of a warp, run solves of
// similar size.  (Mixing large- and small-solve warps inside a block, sorting
// only inside 256-qp blocks, and a persistent grid-stride launch with 64-256
// resident threads per SM all measured slower.)  The launch shape (threads
// per block, registers per thread) is a template choice, see kU2Shapes in
// cp_launch.h.
//
// Block order: for the classes of at most 32 systems the blocks take the sorted
// ranges alternately from the two ends (block 2b the b-th range from the
// largest solves, block 2b+1 the b-th from the smallest), so the SMs hold a mix
// of large and small solves and their per-thread scratch shares the L2 with
// less spilling to DRAM (2^21-qp mixed workload: FCC 6.79 -> 6.63 ms, HCP 2.24
// -> 1.90 ms).  The 48-system class keeps the ranges in descending order: its
// largest solves are long enough that taking them first shortens the tail more
// (interleaved 11.94 against 11.69 ms).  Each qp's update is independent of
// which block runs it, so the order changes no result.
template <int PMAX>
__device__ __forceinline__ int64_t update2_block_range(int64_t b, int64_t nb) {
    if (PMAX > 32) return b;
    return (b & 1) ? nb - 1 - (b >> 1) : (b >> 1);
}
template <int PMAX, class FSrc>
__device__ __forceinline__ void update2_one(const LatDev& L, const Opts& o, const GroupDev& g, const FSrc& fs,
                                            int64_t i, int flag, double F_e, double F_r, double* __restrict__ P,
                                            double* __restrict__ T, double* __restrict__ dPdF,
                                            double* __restrict__ stage, int32_t* __restrict__ status,
                                            int32_t* __restrict__ stats, double* __restrict__ keepF,
                                            double* __restrict__ keepT, int lattice_id, double* d2_slot,
                                            int d2_stride) {
    const int64_t k = g.qp[i];
    const M3 F = fs(k);
    double Tl[9];
    QpOut out;
    if (stage) {
        out.P = stage + 90 * k;
        out.dPdF = stage + 90 * k + 9;
        out.scale = fs.weight(k);
    } else {
        out.P = P ? P + 9 * k : nullptr;
        out.dPdF = (dPdF && flag == 1) ? dPdF + 81 * k : nullptr;
        out.scale = 1.0;
    }
    out.T = (T || keepT) ? Tl : nullptr;
    const int st = qp_update2<PMAX>(L, o, g, i, F, flag, F_e, F_r, out, stats ? stats + 8 * k : nullptr, lattice_id,
                                    d2_slot, d2_stride);
    if (T)
#pragma unroll
        for (int c = 0; c < 9; ++c) T[9 * k + c] = Tl[c];
    if (keepT) {
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            keepT[9 * k + c] = Tl[c];
            keepF[9 * k + c] = F.a[c];
        }
    }
    if (status) status[k] = st;
}

template <int PMAX, class FSrc, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
    update2_kernel(const LatDev* __restrict__ L, Opts o, GroupDev g, FSrc fs, const int* __restrict__ perm, int64_t m,
                   int flag, double F_e, double F_r, double* __restrict__ P, double* __restrict__ T, double* __restrict__ dPdF,
                   double* __restrict__ stage, int32_t* __restrict__ status, int32_t* __restrict__ stats,
                   double* __restrict__ keepF, double* __restrict__ keepT, int lattice_id) {
    // per-thread rotated-stiffness slots, entry e of thread t at sD2[e * BLOCK + t]
    __shared__ double sD2[21 * BLOCK];
    const int64_t j = update2_block_range<PMAX>(blockIdx.x, gridDim.x) * blockDim.x + threadIdx.x;
    if (j < m)
        update2_one<PMAX>(*L, o, g, fs, perm[j], flag, F_e, F_r, P, T, dPdF, stage, status, stats, keepF, keepT,
                          lattice_id, sD2 + threadIdx.x, BLOCK);
}

// update2_kernel over the groups of several handles in one launch: thread j
// of group k's blocks runs internal qp perm_k[j] of that group (its own
// constants, history and displacement field).  Same per-qp arithmetic as the
// per-handle launch, so the results do not depend on what else shares it.
template <int PMAX, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) update2_batch_kernel(const __grid_constant__ BatchArgs a) {
    __shared__ double sD2[21 * BLOCK];
    int64_t lb = 0;
    const int k = batch_group_of_block(a, BLOCK, lb);
    if (k < 0) return;
    const BatchDesc& d = a.d[k];
    const int64_t j = lb * BLOCK + threadIdx.x;
    if (j < d.m)
        update2_one<PMAX>(*d.L, d.o, d.g, d.fm, d.perm[j], a.flag, d.F_e, d.F_r, nullptr, nullptr, nullptr, d.stage,
                          d.status, d.stats, d.keepF, d.keepT, d.lattice_id, sD2 + threadIdx.x, BLOCK);
}

#ifndef CP_TEMPLATES_ONLY
// Element contraction (getElementalValues.cc:144-162) from the staged JxW*P
// and JxW*dP/dF of the cell's 8 qps: thread (cell, node a) forms rows
// 3a..3a+2 of Ke and Re; the block's Ke leave through shared memory as one
// coalesced run.  Cells [cell_begin, cell_end) in caller order;
// CONTRACT_CELLS per block.
constexpr int CONTRACT_CELLS = 8;
__global__ void __launch_bounds__(CONTRACT_CELLS * 8) contract_kernel(const double* __restrict__ stage,
                                                                      const double* __restrict__ gradN, int uniform,
                                                                      int64_t cell_begin, int64_t cell_end,
                                                                      double* __restrict__ Ke,
                                                                      double* __restrict__ Re) {
    // one padded row per cell: the 8 threads of a cell read their own row,
    // and a row stride of 721 doubles puts the warp's 4 cells on different banks
    __shared__ double sd[CONTRACT_CELLS][8 * 90 + 1];
    const int tid = threadIdx.x;
    const int lc = tid >> 3, a1 = tid & 7;
    const int64_t cell0 = cell_begin + (int64_t)blockIdx.x * CONTRACT_CELLS;
    // cooperative, coalesced load of the block's cells' staged values
    const int64_t ncb = (cell_end - cell0) < CONTRACT_CELLS ? (cell_end - cell0) : CONTRACT_CELLS;
    const double* src = stage + cell0 * 720;
    for (int t = tid; t < ncb * 720; t += CONTRACT_CELLS * 8) sd[t / 720][t % 720] = src[t];
    __syncthreads();
    const int64_t cell = cell0 + lc;
    const bool live = cell < cell_end;
    const double* g0 = uniform ? gradN : gradN + (live ? cell : cell0) * 192;
    double K[3][24];
    double Rl[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 24; ++c) K[r][c] = 0.0;
    for (int qq = 0; qq < 8; ++qq) {
        const double* gq = g0 + qq * 24;
        const double* Pq = &sd[lc][qq * 90];
        const double* Dq = Pq + 9;
        const double g1x = gq[a1 * 3], g1y = gq[a1 * 3 + 1], g1z = gq[a1 * 3 + 2];
#pragma unroll
        for (int ci = 0; ci < 3; ++ci) {
            Rl[ci] -= g1x * Pq[3 * ci] + g1y * Pq[3 * ci + 1] + g1z * Pq[3 * ci + 2];
#pragma unroll
            for (int cj = 0; cj < 3; ++cj) {
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
    // Ke through shared memory (the staged values are no longer needed), so
    // that the block's cells, contiguous in Ke, are written coalesced
    __syncthreads();
    if (live) {
        double* Ks = &sd[lc][(3 * a1) * 24];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 24; ++c) Ks[r * 24 + c] = K[r][c];
#pragma unroll
        for (int r = 0; r < 3; ++r) Re[cell * 24 + 3 * a1 + r] = Rl[r];
    }
    __syncthreads();
    double2* dst = reinterpret_cast<double2*>(Ke + cell0 * 576);
    for (int t = tid; t < ncb * 288; t += CONTRACT_CELLS * 8) {
        const int cc = t / 288, e = t % 288;
        dst[t] = make_double2(sd[cc][2 * e], sd[cc][2 * e + 1]);
    }
}

#endif

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
