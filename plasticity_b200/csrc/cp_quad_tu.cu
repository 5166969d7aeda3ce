// cp_quad_tu.cu -- the quad form of the sorted update (cp_qp4.cuh: four lanes
// per qp, scratch in shared memory) for one lattice class and F source.
// Compiled once per (CP_TU_PMAX, CP_TU_FSRC) by plasticity_b200/build.py;
// cp_api.cu reaches it through cp_launch.h as launch shape U2_QUAD.
#define CP_TEMPLATES_ONLY
#include "cp_kernels.cuh"
#include "cp_launch.h"
#include "cp_qp4.cuh"

#if !defined(CP_TU_PMAX) || !defined(CP_TU_FSRC)
#error "compile with -DCP_TU_PMAX=<16|32|48> -DCP_TU_FSRC=<FromArray|FromMesh>"
#endif

namespace cp {

constexpr int Q4_BLOCK = 128;                 // 32 quads per block
constexpr int Q4_SMEM_BYTES = 110 * 1024;     // per-qp areas; two blocks per SM (96, 80, 64 KB: slower)
constexpr int Q4_SMEM_DOUBLES = Q4_SMEM_BYTES / 8;

template <int PMAX, class FSrc>
__device__ __forceinline__ void update4_one(const LatDev& L, const Opts& o, const GroupDev& g, const FSrc& fs, int64_t i,
                                            int flag, double F_e, double F_r, double* __restrict__ P,
                                            double* __restrict__ T, double* __restrict__ dPdF,
                                            double* __restrict__ stage, int32_t* __restrict__ status,
                                            int32_t* __restrict__ stats, double* __restrict__ keepF,
                                            double* __restrict__ keepT, int lattice_id, double* area, int cap,
                                            const Quad& q) {
    const int64_t k = g.qp[i];
    const M3 F = fs(k);
    QuadOut out;
    if (stage) {
        out.P = stage + 90 * k;
        out.dPdF = stage + 90 * k + 9;
        out.scale = fs.weight(k);
    } else {
        out.P = P ? P + 9 * k : nullptr;
        out.dPdF = (dPdF && flag == 1) ? dPdF + 81 * k : nullptr;
        out.scale = 1.0;
    }
    out.T = T ? T + 9 * k : nullptr;
    out.keepT = keepT ? keepT + 9 * k : nullptr;
    out.keepF = keepT ? keepF + 9 * k : nullptr;
    const int st = qp_update4<PMAX>(L, o, g, i, F, flag, F_e, F_r, out, stats ? stats + 8 * k : nullptr, lattice_id,
                                    area, cap, q);
    if (status && q.l == 0) status[k] = st;
}

// The sorted qps of one group in chunks: a chunk is a run of qps of one
// sort bucket (one potentially-active-set size p0), as many as the block's
// shared memory holds areas of capacity min(p0, PMAX), at most one per quad.
// All quads of a chunk start together, so the quads of a warp, running
// solves of one size, stay converged as long as their qps take the same
// number of removal rounds (qps claimed one by one as quads free up, or
// chunks per warp, measured 1.4-1.5x slower: the quads of a warp then diverge
// and their paths serialise).  The chunk table follows from the bucket
// counts and ends the counting sort left in hist (every block derives it);
// blocks take chunks blockIdx.x, blockIdx.x + gridDim.x, ... (a persistent
// grid of two blocks per SM).
template <int PMAX, class FSrc>
__global__ void __launch_bounds__(Q4_BLOCK, 2)
    update4_kernel(const LatDev* __restrict__ L, Opts o, GroupDev g, FSrc fs, const int* __restrict__ perm,
                   const int* __restrict__ hist, int flag, double F_e, double F_r, double* __restrict__ P,
                   double* __restrict__ T, double* __restrict__ dPdF, double* __restrict__ stage,
                   int32_t* __restrict__ status, int32_t* __restrict__ stats, double* __restrict__ keepF,
                   double* __restrict__ keepT, int lattice_id) {
    extern __shared__ double sm[];
    __shared__ int s_first[SORT_BUCKETS + 1], s_per[SORT_BUCKETS], s_start[SORT_BUCKETS], s_end[SORT_BUCKETS];
    const int n = L->n;
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int b = 0; b < SORT_BUCKETS; ++b) {
            const int c = hist[b], e = hist[SORT_BUCKETS + b];
            const int cap = (SORT_BUCKETS - 1 - b) < PMAX ? (SORT_BUCKETS - 1 - b) : PMAX;
            int per = Q4_SMEM_DOUBLES / quad_area_doubles(cap, n);
            if (per > Q4_BLOCK / 4) per = Q4_BLOCK / 4;
            if (per < 1) per = 1;  // unreachable: the launch checks the largest area fits
            s_first[b] = acc;
            s_per[b] = per;
            s_start[b] = e - c;
            s_end[b] = e;
            acc += (c + per - 1) / per;
        }
        s_first[SORT_BUCKETS] = acc;
    }
    __syncthreads();
    const int total = s_first[SORT_BUCKETS];
    const int lane = threadIdx.x & 31;
    const Quad q{lane & 3, 0xFu << (lane & ~3), lane & ~3};
    const int qi = threadIdx.x >> 2;
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        int b = 0;
        while (b < SORT_BUCKETS - 1 && s_first[b + 1] <= c) ++b;
        const int per = s_per[b];
        const int j0 = s_start[b] + (c - s_first[b]) * per;
        const int left = s_end[b] - j0;
        const int cnt = left < per ? left : per;
        const int cap = (SORT_BUCKETS - 1 - b) < PMAX ? (SORT_BUCKETS - 1 - b) : PMAX;
        if (qi < cnt)
            update4_one<PMAX>(*L, o, g, fs, perm[j0 + qi], flag, F_e, F_r, P, T, dPdF, stage, status, stats, keepF,
                              keepT, lattice_id, sm + (int64_t)qi * quad_area_doubles(cap, n), cap, q);
        __syncthreads();  // the next chunk lays its areas out afresh
    }
}

template <int PMAX, class FSrc>
cudaError_t launch_update4(cudaStream_t s, const U2Args& a, const FSrc& fs) {
    if (a.o.max_search != 1 || !a.hist || a.num_sms < 1) return cudaErrorInvalidValue;
    if (quad_area_doubles(PMAX, NM) > Q4_SMEM_DOUBLES) return cudaErrorInvalidValue;
    update4_kernel<PMAX, FSrc><<<2 * a.num_sms, Q4_BLOCK, Q4_SMEM_BYTES, s>>>(
        a.L, a.o, a.g, fs, a.perm, a.hist, a.flag, a.F_e, a.F_r, a.P, a.T, a.dPdF, a.stage, a.status, a.stats,
        a.keepF, a.keepT, a.lattice_id);
    return cudaGetLastError();
}

template <int PMAX, class FSrc>
cudaError_t prepare_update4() {
    return cudaFuncSetAttribute(update4_kernel<PMAX, FSrc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Q4_SMEM_BYTES);
}

template cudaError_t launch_update4<CP_TU_PMAX, CP_TU_FSRC>(cudaStream_t, const U2Args&, const CP_TU_FSRC&);
template cudaError_t prepare_update4<CP_TU_PMAX, CP_TU_FSRC>();

}  // namespace cp
