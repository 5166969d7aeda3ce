// cp_update_tu.cu -- one launch shape of the sorted update for one lattice
// class and F source.  Compiled once per (CP_TU_PMAX, CP_TU_FSRC,
// CP_TU_VARIANT) by plasticity_b200/build.py, so the large kernel
// instantiations build in parallel; cp_api.cu reaches them through
// cp_launch.h.
#define CP_TEMPLATES_ONLY  // the non-template kernels live in cp_api.cu
#include "cp_kernels.cuh"
#include "cp_launch.h"

#if !defined(CP_TU_PMAX) || !defined(CP_TU_FSRC) || !defined(CP_TU_VARIANT)
#error "compile with -DCP_TU_PMAX=<16|32|48> -DCP_TU_FSRC=<FromArray|FromMesh> -DCP_TU_VARIANT=<0..3>"
#endif

namespace cp {

template <int PMAX, class FSrc, int V>
cudaError_t launch_update2_v(cudaStream_t s, const U2Args& a, const FSrc& fs) {
    constexpr int B = kU2Shapes[V].block, MB = kU2Shapes[V].min_blocks;
    const unsigned grid = (unsigned)((a.m + B - 1) / B);
    update2_kernel<PMAX, FSrc, B, MB><<<grid, B, 0, s>>>(a.L, a.o, a.g, fs, a.perm, a.m, a.flag, a.F_e, a.F_r, a.P,
                                                         a.T, a.dPdF, a.stage, a.status, a.stats, a.keepF, a.keepT,
                                                         a.lattice_id);
    return cudaGetLastError();
}

template cudaError_t launch_update2_v<CP_TU_PMAX, CP_TU_FSRC, CP_TU_VARIANT>(cudaStream_t, const U2Args&,
                                                                            const CP_TU_FSRC&);

}  // namespace cp
