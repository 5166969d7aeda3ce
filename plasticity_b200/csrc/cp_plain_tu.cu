// cp_plain_tu.cu -- the plain thread-per-qp update and fused assembly of one
// lattice class (CP_TU_NT systems, CP_TU_PMAX solve rows), compiled once per
// class by plasticity_b200/build.py.
#define CP_TEMPLATES_ONLY  // the non-template kernels live in cp_api.cu
#include "cp_kernels.cuh"
#include "cp_launch.h"

#if !defined(CP_TU_NT) || !defined(CP_TU_PMAX)
#error "compile with -DCP_TU_NT=<16|32|64> -DCP_TU_PMAX=<16|32|48>"
#endif

namespace cp {

template <int NT, int PMAX>
cudaError_t launch_update_plain(cudaStream_t s, const LatDev* L, const Opts& o, const GroupDev& g, const double* F,
                                int flag, double F_e, double F_r, double* P, double* T, double* dPdF,
                                int32_t* status, int32_t* stats, double* keepF, double* keepT, int lattice_id) {
    const unsigned grid = (unsigned)((g.count + QP_BLOCK - 1) / QP_BLOCK);
    update_kernel<NT, PMAX><<<grid, QP_BLOCK, 0, s>>>(L, o, g, F, flag, F_e, F_r, P, T, dPdF, status, stats, keepF,
                                                      keepT, lattice_id);
    return cudaGetLastError();
}

template <int NT, int PMAX>
cudaError_t launch_assemble_plain(cudaStream_t s, const LatDev* L, const Opts& o, const GroupDev& g,
                                  const double* U, const double* gradN, const double* JxW, int uniform, double F_e,
                                  double F_r, double* Ke, double* Re, int32_t* status, int32_t* stats,
                                  int lattice_id) {
    const size_t smem = (size_t)QP_BLOCK * 90 * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(assemble_kernel<NT, PMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned grid = (unsigned)((g.count + QP_BLOCK - 1) / QP_BLOCK);
    assemble_kernel<NT, PMAX><<<grid, QP_BLOCK, smem, s>>>(L, o, g, U, gradN, JxW, uniform, F_e, F_r, Ke, Re, status,
                                                           stats, lattice_id);
    return cudaGetLastError();
}

template cudaError_t launch_update_plain<CP_TU_NT, CP_TU_PMAX>(cudaStream_t, const LatDev*, const Opts&,
                                                               const GroupDev&, const double*, int, double, double,
                                                               double*, double*, double*, int32_t*, int32_t*,
                                                               double*, double*, int);
template cudaError_t launch_assemble_plain<CP_TU_NT, CP_TU_PMAX>(cudaStream_t, const LatDev*, const Opts&,
                                                                 const GroupDev&, const double*, const double*,
                                                                 const double*, int, double, double, double*,
                                                                 double*, int32_t*, int32_t*, int);

}  // namespace cp
