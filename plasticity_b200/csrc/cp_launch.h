// cp_launch.h -- host-side launchers of the per-qp kernels.
//
// The large per-qp kernels are compiled in their own translation units (one
// per lattice class, F source and launch shape; plasticity_b200/build.py
// compiles them in parallel) and reached from cp_api.cu through these
// launchers, which take plain arguments only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cp_qp.cuh"

namespace cp {

struct FromArray;
struct FromMesh;
struct BatchArgs;

// Arguments of one sorted-update launch over m qps of a lattice group
// (thread j runs internal qp perm[j]); see update2_kernel.
struct U2Args {
    const LatDev* L;
    Opts o;
    GroupDev g;
    const int* perm;
    int64_t m;
    int flag;
    double F_e, F_r;
    double *P, *T, *dPdF, *stage;
    int32_t *status, *stats;
    double *keepF, *keepT;
    int lattice_id;
    const int* hist;  // the sort's bucket counts, then bucket ends (the quad shape's chunk table)
    int num_sms;
};

// Launch shapes of the sorted update (the autotuner's choices): threads per
// block and the resident blocks per SM the registers are sized for
// (__launch_bounds__(block, min_blocks): 255 registers for 256 threads per
// SM, 128 for 512).
struct U2Shape {
    int block, min_blocks;
};
constexpr int U2_THREAD_SHAPES = 4;
constexpr U2Shape kU2Shapes[U2_THREAD_SHAPES] = {{256, 1}, {256, 2}, {64, 4}, {64, 8}};
// Shape 4: four lanes per qp with the scratch in shared memory (cp_qp4.cuh,
// one slip-search pass only).
constexpr int U2_QUAD = U2_THREAD_SHAPES;
constexpr int U2_VARIANTS = U2_THREAD_SHAPES + 1;

// Default shape without tuning: launches of at most U2_SPREAD_QPS qps (an
// RVE's or a served request's group) in 64-thread blocks spread over the SMs
// (255 registers for the FCC class, PMAX 16; 128 for the BCC/HCP classes),
// larger ones in 256-thread blocks of 255 registers, one per SM (measured per
// class on the 2^21-qp mixed workload: BCC 11.7 against 13.1 ms for two
// 128-register blocks per SM, FCC 6.6 against 8.5, HCP 2.26 against 2.27).
constexpr int64_t U2_SPREAD_QPS = 148 * 64;
inline int u2_default_variant(int pmax, int64_t m) {
    const bool small_class = pmax <= 16;
    if (m <= U2_SPREAD_QPS) return small_class ? 2 : 3;
    return 0;
}

// Sorted update, one translation unit per (PMAX, F source, variant).
template <int PMAX, class FSrc, int V>
cudaError_t launch_update2_v(cudaStream_t s, const U2Args& a, const FSrc& fs);

// The quad form of the sorted update (cp_quad_tu.cu, one translation unit per
// (PMAX, F source)); a.hist and a.num_sms must be set; max_search must be 1.
// prepare_update4 raises the kernel's shared-memory limit once per device.
template <int PMAX, class FSrc>
cudaError_t launch_update4(cudaStream_t s, const U2Args& a, const FSrc& fs);
template <int PMAX, class FSrc>
cudaError_t prepare_update4();

// Plain thread-per-qp update (F from a caller array) and plain fused assembly
// of one group, one translation unit per lattice class.
template <int NT, int PMAX>
cudaError_t launch_update_plain(cudaStream_t s, const LatDev* L, const Opts& o, const GroupDev& g, const double* F,
                                int flag, double F_e, double F_r, double* P, double* T, double* dPdF,
                                int32_t* status, int32_t* stats, double* keepF, double* keepT, int lattice_id);
template <int NT, int PMAX>
cudaError_t launch_assemble_plain(cudaStream_t s, const LatDev* L, const Opts& o, const GroupDev& g,
                                  const double* U, const double* gradN, const double* JxW, int uniform, double F_e,
                                  double F_r, double* Ke, double* Re, int32_t* status, int32_t* stats,
                                  int lattice_id);

// The reference-order update (cp_qpref.cuh, compiled without FMA contraction
// in cp_ref_tu.cu) of one group, F from a caller array: one thread per qp
// on at most 'threads' threads, thread t on scratch slot t (scratch holds
// 'threads' slots of 'slot' doubles).
int64_t ref_scratch_doubles(int n);
cudaError_t launch_update_ref(cudaStream_t s, const LatDev* L, const Opts& o, const GroupDev& g, const double* F,
                              int flag, double F_e, double F_r, double* P, double* T, double* dPdF, int32_t* status,
                              int32_t* stats, double* keepF, double* keepT, int lattice_id, double* scratch,
                              int64_t slot, int64_t threads);

// The batched sorted update (update2_batch_kernel) of one lattice class over
// the groups of several handles, in the class's default launch shape;
// cp_batch_tu.cu, one translation unit per class.
template <int PMAX>
cudaError_t launch_update2_batch(cudaStream_t s, const BatchArgs& a, int64_t total_blocks_unused = 0);

// Split-BF16 tensor-core contraction of the staged JxW dP/dF of cells
// [cell_begin, cell_end) into FP32 Ke and, from the staged JxW P, FP64 Re
// (cp_tc.cu).  gradN: the shared shape-function gradients of a uniform mesh.
// *err is raised if a wait of the kernel expired.  prepare_ke_tc sets the
// kernel's shared-memory size once per device.
cudaError_t prepare_ke_tc();
cudaError_t launch_ke_tc(cudaStream_t s, const double* stage, const double* gradN, int64_t cell_begin,
                         int64_t cell_end, float* Ke, double* Re, int* err, int num_sms);

}  // namespace cp
