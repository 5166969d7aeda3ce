// cp_ref_tu.cu -- the reference-order update (cp_qpref.cuh): one thread per
// qp over a fixed grid, each thread with its own scratch slot in global
// memory.  plasticity_b200/build.py compiles this unit with -fmad=false, so
// every multiply and add rounds as the reference's source writes it.
#include "cp_launch.h"
#include "cp_qpref.cuh"

namespace cp {

constexpr int REF_BLOCK = 64;

__global__ void __launch_bounds__(REF_BLOCK)
    update_ref_kernel(const LatDev* __restrict__ L, Opts o, GroupDev g, const double* __restrict__ F, int flag,
                      double F_e, double F_r, double* __restrict__ P, double* __restrict__ T,
                      double* __restrict__ dPdF, int32_t* __restrict__ status, int32_t* __restrict__ stats,
                      double* __restrict__ keepF, double* __restrict__ keepT, int lattice_id, double* scratch,
                      int64_t slot, int64_t nslots) {
    // thread t owns scratch slot t and runs qps t, t + nslots, ...
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= nslots) return;
    double* w = scratch + tid * slot;
    for (int64_t i = tid; i < g.count; i += nslots) {
        const int64_t k = g.qp[i];
        double Tl[9];
        QpOut out;
        out.P = P ? P + 9 * k : nullptr;
        out.T = (T || keepT) ? Tl : nullptr;
        out.dPdF = (dPdF && flag == 1) ? dPdF + 81 * k : nullptr;
        out.scale = 1.0;
        const int st = ref::qp_update_ref(*L, o, g, i, F + 9 * k, flag, F_e, F_r, out,
                                          stats ? stats + 8 * k : nullptr, lattice_id, w);
        if (T)
            for (int c = 0; c < 9; ++c) T[9 * k + c] = Tl[c];
        if (keepT)
            for (int c = 0; c < 9; ++c) {
                keepT[9 * k + c] = Tl[c];
                keepF[9 * k + c] = F[9 * k + c];
            }
        if (status) status[k] = st;
    }
}

int64_t ref_scratch_doubles(int n) { return ref::scratch_doubles(n); }

cudaError_t launch_update_ref(cudaStream_t s, const LatDev* L, const Opts& o, const GroupDev& g, const double* F,
                              int flag, double F_e, double F_r, double* P, double* T, double* dPdF, int32_t* status,
                              int32_t* stats, double* keepF, double* keepT, int lattice_id, double* scratch,
                              int64_t slot, int64_t threads) {
    if (g.count <= 0 || threads <= 0) return cudaSuccess;
    const int64_t t = threads < g.count ? threads : g.count;
    const unsigned grid = (unsigned)((t + REF_BLOCK - 1) / REF_BLOCK);
    update_ref_kernel<<<grid, REF_BLOCK, 0, s>>>(L, o, g, F, flag, F_e, F_r, P, T, dPdF, status, stats, keepF, keepT,
                                                 lattice_id, scratch, slot, t);
    return cudaGetLastError();
}

}  // namespace cp
