// cp_batch_tu.cu -- the batched sorted update (several handles' groups of one
// lattice class in one launch) for one class, CP_TU_PMAX; compiled once per
// class by plasticity_b200/build.py.
#define CP_TEMPLATES_ONLY  // the non-template kernels live in cp_api.cu
#include "cp_kernels.cuh"
#include "cp_launch.h"

#if !defined(CP_TU_PMAX)
#error "compile with -DCP_TU_PMAX=<16|32|48>"
#endif

namespace cp {

template <int PMAX>
cudaError_t launch_update2_batch(cudaStream_t s, const BatchArgs& a, int64_t) {
    // the class's default shape for large launches: 256 threads, 255
    // registers (FCC class) or 128 (BCC/HCP classes)
    constexpr int B = 256, MB = PMAX <= 16 ? 1 : 2;
    int64_t blocks = 0;
    for (int k = 0; k < a.n; ++k) blocks += (a.d[k].m + B - 1) / B;
    if (blocks == 0) return cudaSuccess;
    update2_batch_kernel<PMAX, B, MB><<<(unsigned)blocks, B, 0, s>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_update2_batch<CP_TU_PMAX>(cudaStream_t, const BatchArgs&, int64_t);

}  // namespace cp
