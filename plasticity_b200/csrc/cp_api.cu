// cp_api.cu -- C ABI of include/cp_gpu.h: resident per-qp history on one
// GPU, kernel dispatch by lattice class, host/device entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cp_gpu.h"
#include "cp_kernels.cuh"
#include "cp_launch.h"
#include "cp_solve32.cuh"

using namespace cp;

// ---------------------------------------------------------------- kernels
namespace cp {

__global__ void init_state_kernel(const LatDev* __restrict__ L, GroupDev g, const double* __restrict__ rod) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.count) return;
    const int64_t cnt = g.count;
    const int n = L->n, ns = L->ns, nw = L->nw;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        const double v = (c == 0 || c == 4 || c == 8) ? 1.0 : 0.0;
        g.Fp_c[c * cnt + i] = v;
        g.Fe_c[c * cnt + i] = v;
        g.Fp_i[c * cnt + i] = v;
        g.Fe_i[c * cnt + i] = v;
    }
    for (int a = 0; a < n; ++a) {
        const double s0 = L->s0[a];
        g.s_c[a * cnt + i] = s0;
        g.s_i[a * cnt + i] = s0;
        g.W_c[a * cnt + i] = 0.0;
        g.W_i[a * cnt + i] = 0.0;
    }
    const int64_t k = g.qp[i];
    for (int c = 0; c < 3; ++c) {
        const double r = rod[3 * k + c];
        g.rot_c[c * cnt + i] = r;
        g.rot_i[c * cnt + i] = r;
        g.rotnew_c[c * cnt + i] = r;
        g.rotnew_i[c * cnt + i] = r;
    }
    for (int t = 0; t < nw; ++t) {
        g.tw_c[t * cnt + i] = 0.0;
        g.tw_i[t * cnt + i] = 0.0;
    }
    for (int t = 0; t < ns; ++t) {
        g.sl_c[t * cnt + i] = 0.0;
        g.sl_i[t * cnt + i] = 0.0;
    }
    g.twin_c[i] = 0;
    g.twin_i[i] = 0;
}

// symmetric 3x3 eigen-decomposition by cyclic Jacobi (columns of V are
// eigenvectors), the stand-in for LAPACK syevx of reorient.cc:35,48
__device__ void eig_sym3(const M3& C, double ev[3], M3& V) {
    M3 A = C;
    V = eye3();
    for (int sweep = 0; sweep < 50; ++sweep) {
        const double off = A(0, 1) * A(0, 1) + A(0, 2) * A(0, 2) + A(1, 2) * A(1, 2);
        const double dia = A(0, 0) * A(0, 0) + A(1, 1) * A(1, 1) + A(2, 2) * A(2, 2);
        if (off <= 1e-32 * dia || off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                const double apq = A(p, q);
                if (apq == 0.0) continue;
                const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - s * akq;
                    A(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - s * aqk;
                    A(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = V(k, p), vkq = V(k, q);
                    V(k, p) = c * vkp - s * vkq;
                    V(k, q) = s * vkp + c * vkq;
                }
            }
    }
    ev[0] = A(0, 0);
    ev[1] = A(1, 1);
    ev[2] = A(2, 2);
}

__device__ M3 polar_rotation(const M3& Fe) {
    const M3 C = mulTN(Fe, Fe);
    double ev[3];
    M3 V;
    eig_sym3(C, ev, V);
    M3 Lam = zero3();
    Lam(0, 0) = sqrt(ev[0]);
    Lam(1, 1) = sqrt(ev[1]);
    Lam(2, 2) = sqrt(ev[2]);
    const M3 U = mulNT(mul(V, Lam), V);
    return mul(Fe, inv(U));
}

__global__ void reorient_kernel(GroupDev g) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.count) return;
    const int64_t cnt = g.count;
    double rold[3];
    for (int c = 0; c < 3; ++c) rold[c] = g.rotnew_i[c * cnt + i];  // rotnew_conv = rotnew_iter
    M3 Fe_old = load_soa3(g.Fe_c, cnt, i);
    const M3 Fe_new = load_soa3(g.Fe_i, cnt, i);
    if (g.twin_c[i] != g.twin_i[i]) Fe_old = Fe_new;
    const M3 R_old = polar_rotation(Fe_old);
    const M3 R_new = polar_rotation(Fe_new);
    M3 Om = R_new;
    axpy(Om, -1.0, R_old);
    Om = mulNT(Om, R_new);
    double ov[3];
    ov[0] = -0.5 * (Om(1, 2) - Om(2, 1));
    ov[1] = 0.5 * (Om(0, 2) - Om(2, 0));
    ov[2] = -0.5 * (Om(0, 1) - Om(1, 0));
    const double dot = ov[0] * rold[0] + ov[1] * rold[1] + ov[2] * rold[2];
    double cr[3], rn[3];
    cr[0] = ov[1] * rold[2] - ov[2] * rold[1];
    cr[1] = ov[2] * rold[0] - ov[0] * rold[2];
    cr[2] = ov[0] * rold[1] - ov[1] * rold[0];
    for (int c = 0; c < 3; ++c) rn[c] = rold[c] + 0.5 * (ov[c] + dot * rold[c] + cr[c]);
    const double mx = 10000.0;
    const double nrm = sqrt(rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2]);
    if (nrm > mx)
        for (int c = 0; c < 3; ++c) rn[c] = rn[c] * mx / nrm;
    for (int c = 0; c < 3; ++c) {
        g.rotnew_c[c * cnt + i] = rn[c];
        g.rotnew_i[c * cnt + i] = rn[c];  // rotnew_iter = rotnew_conv
    }
}

constexpr int AVG_N = 22;
constexpr int AVG_BLOCK = 256;

__global__ void __launch_bounds__(AVG_BLOCK)
    averages_partial_kernel(const LatDev* __restrict__ L, GroupDev g, const double* __restrict__ keepF,
                            const double* __restrict__ keepT, const double* __restrict__ JxW, int uniform,
                            double* __restrict__ partial) {
    __shared__ double red[AVG_BLOCK / 32][AVG_N];
    // qps in bind order (the group's j-th bound qp), so the sums do not depend
    // on the internal order of the history
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v[AVG_N];
#pragma unroll
    for (int c = 0; c < AVG_N; ++c) v[c] = 0.0;
    if (j < g.count) {
        const int64_t i = g.where ? g.where[j] : j;
        const int64_t cnt = g.count;
        const int64_t k = g.qp[i];
        const double w = uniform ? JxW[k & 7] : JxW[k];
        M3 F;
#pragma unroll
        for (int c = 0; c < 9; ++c) F.a[c] = keepF[9 * k + c];
        const M3 C = mulTN(F, F);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) v[3 * a + b] = 0.5 * (C(a, b) - (a == b ? 1.0 : 0.0)) * w;
#pragma unroll
        for (int c = 0; c < 9; ++c) v[9 + c] = keepT[9 * k + c] * w;
        double fr = 0.0, fs = 0.0;
        for (int t = 0; t < L->nw; ++t) fr += g.tw_i[t * cnt + i];
        for (int t = 0; t < L->ns; ++t) fs += g.sl_i[t * cnt + i];
        v[18] = fr * w;
        v[19] = (double)g.twin_i[i] * w;
        v[20] = fs * w;
        v[21] = w;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < AVG_N; ++c) {
        double x = v[c];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if (lane == 0) red[warp][c] = x;
    }
    __syncthreads();
    if (threadIdx.x < AVG_N) {
        double s = 0.0;
        for (int wi = 0; wi < AVG_BLOCK / 32; ++wi) s += red[wi][threadIdx.x];
        partial[(int64_t)blockIdx.x * AVG_N + threadIdx.x] = s;
    }
}

__global__ void averages_final_kernel(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
    // one thread per component, fixed order: deterministic
    const int c = threadIdx.x;
    if (c >= AVG_N) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[(int64_t)b * AVG_N + c];
    out[c] = s;
}

// gather one history field of a group into caller-order rows of width w
__global__ void gather_field_kernel(const double* __restrict__ src, const int* __restrict__ isrc, int64_t cnt,
                                    const int64_t* __restrict__ qp, int comps, int width,
                                    double* __restrict__ dst) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const int64_t k = qp[i];
    for (int c = 0; c < width; ++c) {
        double v = 0.0;
        if (c < comps) v = isrc ? (double)isrc[c * cnt + i] : src[c * cnt + i];
        dst[k * width + c] = v;
    }
}
__global__ void scatter_field_kernel(double* __restrict__ dst, int* __restrict__ idst, int64_t cnt,
                                     const int64_t* __restrict__ qp, int comps, int width,
                                     const double* __restrict__ src) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const int64_t k = qp[i];
    for (int c = 0; c < comps; ++c) {
        const double v = src[k * width + c];
        if (idst)
            idst[c * cnt + i] = (int)v;
        else
            dst[c * cnt + i] = v;
    }
}

// F of every qp from the cell's nodal displacements (getElementalValues.cc:129-138),
// the same expression the sorted update evaluates inline (FromMesh), for the
// plain kernel's post-pass from the device displacement
__global__ void mesh_F_kernel(FromMesh fm, int64_t n_qp, double* __restrict__ F) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_qp) return;
    const M3 f = fm(k);
#pragma unroll
    for (int c = 0; c < 9; ++c) F[9 * k + c] = f.a[c];
}

// ---- the counting sort of several handles' groups (batched launches, see
// BatchDesc): histogram reset, classification, scan and scatter per group
__global__ void batch_hist_zero_kernel(const __grid_constant__ BatchArgs a) {
    if ((int)blockIdx.x < a.n && threadIdx.x < 2 * SORT_BUCKETS) a.d[blockIdx.x].hist[threadIdx.x] = 0;
}

__global__ void __launch_bounds__(QP_BLOCK) classify_batch_kernel(const __grid_constant__ BatchArgs a) {
    __shared__ int sh[SORT_BUCKETS];
    int64_t lb = 0;
    const int k = batch_group_of_block(a, QP_BLOCK, lb);
    if (k < 0) return;
    const BatchDesc& d = a.d[k];
    if (threadIdx.x < SORT_BUCKETS) sh[threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = lb * QP_BLOCK + threadIdx.x;
    if (i < d.m) {
        const int p0 = count_potentially_active(*d.L, d.o, d.g, i, d.fm(d.g.qp[i]));
        const int b = SORT_BUCKETS - 1 - (p0 < SORT_BUCKETS - 1 ? p0 : SORT_BUCKETS - 1);
        d.key[i] = (unsigned char)b;
        atomicAdd(&sh[b], 1);
    }
    __syncthreads();
    if (threadIdx.x < SORT_BUCKETS && sh[threadIdx.x]) atomicAdd(&d.hist[threadIdx.x], sh[threadIdx.x]);
}

__global__ void bucket_scan_batch_kernel(const __grid_constant__ BatchArgs a) {
    if ((int)blockIdx.x >= a.n || threadIdx.x != 0) return;
    int* h = a.d[blockIdx.x].hist;
    int acc = 0;
    for (int b = 0; b < SORT_BUCKETS; ++b) {
        h[SORT_BUCKETS + b] = acc;
        acc += h[b];
    }
}

__global__ void __launch_bounds__(256) bucket_scatter_batch_kernel(const __grid_constant__ BatchArgs a) {
    __shared__ int cnt[SORT_BUCKETS], base[SORT_BUCKETS];
    int64_t lb = 0;
    const int k = batch_group_of_block(a, 256, lb);
    if (k < 0) return;
    const BatchDesc& d = a.d[k];
    if (threadIdx.x < SORT_BUCKETS) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = lb * 256 + threadIdx.x;
    int b = 0, r = 0;
    if (i < d.m) {
        b = d.key[i];
        r = atomicAdd(&cnt[b], 1);
    }
    __syncthreads();
    if (threadIdx.x < SORT_BUCKETS)
        base[threadIdx.x] = cnt[threadIdx.x] ? atomicAdd(&d.hist[SORT_BUCKETS + threadIdx.x], cnt[threadIdx.x]) : 0;
    __syncthreads();
    if (i < d.m) d.perm[base[b] + r] = (int)i;
}

// FP64 FMA throughput probe: 8 independent dependent-FMA chains per thread.
__global__ void fp64_fma_probe_kernel(int iters, double seed, double* out) {
    double a[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) a[c] = seed + threadIdx.x * 1e-9 + c;
    const double m = 0.999999999, k = 1e-12;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < 8; ++c) a[c] = fma(a[c], m, k);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 8; ++c) s += a[c];
    if (s == 12345.678) out[0] = s;  // keeps the chains alive
}

}  // namespace cp

// ---------------------------------------------------------------- no-alloc averages scratch
// Device-resident scratch for cp_averages_noalloc: one row of AVG_N partial
// sums per reduction block (up to CP_NOALLOC_AVG_MAX_QPS qps, plus one spare
// block per lattice group for the per-group rounding) and one final row.
// Every GPU that loads this library holds it (about 2.9 MB) until exit.
constexpr int64_t NOALLOC_AVG_BLOCKS = CP_NOALLOC_AVG_MAX_QPS / cp::AVG_BLOCK + CP_MAX_LATTICES;
static __device__ __align__(256) double g_noalloc_avg_scratch[(NOALLOC_AVG_BLOCKS + 1) * cp::AVG_N];

// ---------------------------------------------------------------- handle
namespace {

struct Group {
    int lattice = 0;
    int nt_class = 0;  // 16, 32 or 64
    int n = 0, ns = 0, nw = 0;
    int64_t count = 0;
    int64_t* d_qp = nullptr;
    double* d_block = nullptr;  // one allocation for all double fields
    int* d_twin = nullptr;      // twin_c, twin_i
    unsigned char* d_key = nullptr;  // sort key per internal qp
    int* d_perm = nullptr;           // internal qps in sorted order
    int* d_hist = nullptr;           // SORT_BUCKETS counts, then SORT_BUCKETS offsets
    int64_t* d_qp_tmp = nullptr;     // the reordered qp map before it replaces d_qp
    int* d_where = nullptr;          // internal index of the qp bound j-th (identity until reordered)
    mutable bool sorted = false;     // d_key holds the keys of a sort since the last reorder
    int tuned[2] = {-1, -1};         // launch shape chosen by cp_autotune (F from an array / from the
                                     // mesh); -1: the default rule of u2_default_variant
    GroupDev dev{};
    std::vector<int64_t> qp_host;    // the group's caller indices in bind order (increasing): the
                                     // internal order of the sorted pipeline differs only within
                                     // the reorder segments, so chunk bounds still follow from it
};

// Host-pointer updates run in caller-order chunks so that one chunk's copies
// overlap another chunk's kernels (chunk c is a contiguous internal range of
// every group, since each group keeps its qps in caller order).
constexpr int MAX_CHUNKS = 4;
int chunks_for(int64_t n) { return n >= (1 << 20) ? 4 : (n >= (1 << 18) ? 2 : 1); }

}  // namespace

struct cp_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t s_in = nullptr, s_out = nullptr;  // host-to-device and device-to-host copies
    cudaEvent_t ev_in[MAX_CHUNKS] = {}, ev_done[MAX_CHUNKS] = {};
    cp_options_t opts{};
    Opts dopts{};
    int n_lat = 0;
    std::vector<cp_material_t> mats;
    std::vector<LatDev*> d_lat;
    int64_t n_qp = 0;
    std::vector<int32_t> lattice_of;  // host copy, caller order
    std::vector<Group> groups;
    int n_max = 0, ns_max = 0, nw_max = 0;
    // staging for host-pointer calls (caller order)
    double *d_F = nullptr, *d_P = nullptr, *d_T = nullptr, *d_dPdF = nullptr;
    int32_t* d_status = nullptr;
    size_t dPdF_cap = 0;
    int32_t* d_stats = nullptr;
    double *d_keepF = nullptr, *d_keepT = nullptr;
    bool have_post = false;
    // mesh
    int64_t n_cells = 0;
    int uniform = 1;
    double *d_gradN = nullptr, *d_JxW = nullptr;
    double *d_U = nullptr, *d_Ke = nullptr, *d_Re = nullptr;
    double* d_stage = nullptr;  // JxW*P and JxW*dP/dF per qp between update and contraction
    int num_sms = 0;
    int* d_tc_err = nullptr;    // raised by the tensor-core contraction if one of its waits expired
    // global system of the Newton step (cp_bind_dofs)
    struct System {
        int64_t n_dofs = 0, nnz = 0, n_con = 0;
        int64_t* d_cell_dofs = nullptr;         // 24 per cell
        int64_t* d_row_ptr = nullptr;           // n_dofs + 1
        int* d_col = nullptr;                   // nnz
        int64_t* d_tpos = nullptr;              // nnz: position of the transposed entry
        int64_t* d_diag = nullptr;              // n_dofs: position of the diagonal entry
        int64_t *d_kptr = nullptr, *d_kidx = nullptr;  // element-matrix contributions per entry
        int64_t *d_rptr = nullptr, *d_ridx = nullptr;  // element-residual contributions per dof
        int64_t* d_con = nullptr;               // constrained dofs
        unsigned char* d_cmask = nullptr;       // n_dofs
        double *d_vals = nullptr, *d_Ke = nullptr, *d_Re = nullptr, *d_Ul = nullptr, *d_duc = nullptr;
        double* d_valsT = nullptr;              // K^T's values in K's pattern (per solve)
        bool triples = false;                   // rows 3t..3t+2 share one column pattern
        int64_t n_blocks = 0;                   // node blocks (0: unavailable)
        int64_t *d_blk = nullptr, *d_blkpos = nullptr;  // 3 dofs / 9 entry positions per node block
        double* d_binv = nullptr;               // inverted 3x3 blocks (per solve)
        float *d_vals32 = nullptr, *d_valsT32 = nullptr;  // mixed precision: K, K^T values (FP32)
        float* d_vec32 = nullptr;               // mixed precision: MV_COUNT FP32 vectors of n_dofs
        double* d_vec = nullptr;                // n_dofs x SYS_VECS vectors
        double *d_sc = nullptr, *d_partial = nullptr;
        double* d_fpartial = nullptr;           // per-block partials of the fused iteration (n_dofs / 8 + 64)
        unsigned int* d_ticket = nullptr;       // [0..3] arrival counters of the fused reductions,
                                                // [4..6] the persistent solve's barrier and timeout flag
        int *d_done = nullptr, *d_info = nullptr;
        // a block of Krylov iterations captured as CUDA graphs (first block /
        // later blocks), for the solver settings they were captured with
        cudaGraphExec_t g_first = nullptr, g_next = nullptr;
        int g_kind = -1, g_precond = -1, g_every = 0, g_pc = -1;
        double g_tol = -1.0;
    } sys;
    // averages scratch
    double *d_avg_partial = nullptr, *d_avg_out = nullptr;
    int64_t avg_cap = 0;
    double* noalloc_scratch = nullptr;  // device address of g_noalloc_avg_scratch (cp_averages_noalloc)
    // the reference-order update's per-thread scratch (cp_options_t.reference_order)
    double* d_refscratch = nullptr;
    int64_t ref_slot = 0, ref_threads = 0;
    unsigned long long barrier_wait_ns = 0;  // cp_debug_barrier_test: 0 = the default wait
    int barrier_withhold = -1;
    // optional per-launch timing of the update/assembly kernels
    bool timing = false;
    struct Pending {
        cudaEvent_t a, b;
        int group;
    };
    std::vector<Pending> pending;
    std::vector<double> group_ms;
    std::vector<int64_t> group_launches;
    double contract_ms[2] = {0.0, 0.0};       // element contractions: [0] FP64, [1] tensor-core
    int64_t contract_launches[2] = {0, 0};
    // captured calls (cp_options_t.use_graphs): a few graphs keyed by the
    // call's kind, pointers, scalars and launch shapes, least recently used
    // replaced first
    struct GraphKey {
        int kind = -1;
        const void* p[8] = {};
        int flag = 0;
        uint64_t fe = 0, fr = 0;
        int64_t epoch = 0;  // tune_epoch at capture
        bool operator==(const GraphKey& o) const {
            if (kind != o.kind || flag != o.flag || fe != o.fe || fr != o.fr || epoch != o.epoch) return false;
            for (int i = 0; i < 8; ++i)
                if (p[i] != o.p[i]) return false;
            return true;
        }
    };
    struct GraphEntry {
        GraphKey key;
        cudaGraphExec_t exec = nullptr;
        uint64_t last_use = 0;
    };
    std::vector<GraphEntry> graphs;
    uint64_t graph_clock = 0;
    int64_t graph_captures = 0, graph_launches = 0;
    int64_t tune_epoch = 0;  // bumped whenever a group's launch shape changes
    std::string err;
};

// A batching queue: one stream on which the sorted updates of several
// handles run as shared launches (cp_batch_assemble / cp_batch_post).
struct cp_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_done = nullptr;
    std::vector<cudaEvent_t> ev_in;
    int64_t launches = 0;  // batched update launches issued
    std::string err;
};

namespace {

int fail(cp_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

int cuda_fail(cp_handle* h, cudaError_t e, const char* what) {
    return fail(h, CP_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(h, call)                                            \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

int nt_class_of(int n) { return n <= 16 ? 16 : (n <= 32 ? 32 : 64); }

void free_group(Group& g) {
    cudaFree(g.d_qp);
    cudaFree(g.d_block);
    cudaFree(g.d_twin);
    cudaFree(g.d_key);
    cudaFree(g.d_perm);
    cudaFree(g.d_hist);
    cudaFree(g.d_qp_tmp);
    cudaFree(g.d_where);
    g = Group{};
}

void free_graphs(cp_handle* h) {
    for (auto& e : h->graphs)
        if (e.exec) cudaGraphExecDestroy(e.exec);
    h->graphs.clear();
}

void free_qps(cp_handle* h) {
    free_graphs(h);
    for (auto& g : h->groups) free_group(g);
    h->groups.clear();
    cudaFree(h->d_F);
    cudaFree(h->d_P);
    cudaFree(h->d_T);
    cudaFree(h->d_dPdF);
    cudaFree(h->d_status);
    cudaFree(h->d_stats);
    cudaFree(h->d_keepF);
    cudaFree(h->d_keepT);
    h->d_F = h->d_P = h->d_T = h->d_dPdF = nullptr;
    h->d_status = nullptr;
    h->d_stats = nullptr;
    h->d_keepF = h->d_keepT = nullptr;
    h->dPdF_cap = 0;
    h->n_qp = 0;
    h->have_post = false;
}

void free_system(cp_handle* h);

void free_mesh(cp_handle* h) {
    free_graphs(h);
    free_system(h);
    cudaFree(h->d_gradN);
    cudaFree(h->d_JxW);
    cudaFree(h->d_U);
    cudaFree(h->d_Ke);
    cudaFree(h->d_Re);
    cudaFree(h->d_stage);
    h->d_gradN = h->d_JxW = h->d_U = h->d_Ke = h->d_Re = h->d_stage = nullptr;
    h->n_cells = 0;
}

// vectors of the Newton system, n_dofs doubles each, in d_vec
enum SysVec { V_U = 0, V_X, V_R, V_RHS, V_DC, V_KDC, V_RES, V_RT, V_Z, V_ZT, V_P, V_PT, V_Q, V_QT, V_DINV, V_S, V_T,
              V_PH, V_SH, SYS_VECS };

void free_system(cp_handle* h) {
    auto& y = h->sys;
    cudaFree(y.d_cell_dofs);
    cudaFree(y.d_row_ptr);
    cudaFree(y.d_col);
    cudaFree(y.d_tpos);
    cudaFree(y.d_diag);
    cudaFree(y.d_kptr);
    cudaFree(y.d_kidx);
    cudaFree(y.d_rptr);
    cudaFree(y.d_ridx);
    cudaFree(y.d_con);
    cudaFree(y.d_cmask);
    cudaFree(y.d_vals);
    cudaFree(y.d_valsT);
    cudaFree(y.d_blk);
    cudaFree(y.d_blkpos);
    cudaFree(y.d_binv);
    cudaFree(y.d_vals32);
    cudaFree(y.d_valsT32);
    cudaFree(y.d_vec32);
    cudaFree(y.d_Ke);
    cudaFree(y.d_Re);
    cudaFree(y.d_Ul);
    cudaFree(y.d_duc);
    cudaFree(y.d_vec);
    cudaFree(y.d_sc);
    cudaFree(y.d_partial);
    cudaFree(y.d_fpartial);
    cudaFree(y.d_ticket);
    cudaFree(y.d_done);
    cudaFree(y.d_info);
    if (y.g_first) cudaGraphExecDestroy(y.g_first);
    if (y.g_next) cudaGraphExecDestroy(y.g_next);
    y = cp_handle::System{};
}

// double fields of a group in the order they are carved out of d_block
int64_t group_doubles(int n, int ns, int nw, int64_t cnt) {
    return cnt * 2 * (9 + 9 + n + n + 3 + 3 + nw + ns);
}

void carve(Group& g) {
    const int64_t c = g.count;
    double* p = g.d_block;
    auto take = [&](int comps) {
        double* r = p;
        p += comps * c;
        return r;
    };
    GroupDev& d = g.dev;
    d.count = c;
    d.qp = g.d_qp;
    d.Fp_c = take(9);
    d.Fe_c = take(9);
    d.s_c = take(g.n);
    d.W_c = take(g.n);
    d.rot_c = take(3);
    d.rotnew_c = take(3);
    d.tw_c = take(g.nw);
    d.sl_c = take(g.ns);
    d.Fp_i = take(9);
    d.Fe_i = take(9);
    d.s_i = take(g.n);
    d.W_i = take(g.n);
    d.rot_i = take(3);
    d.rotnew_i = take(3);
    d.tw_i = take(g.nw);
    d.sl_i = take(g.ns);
    d.twin_c = g.d_twin;
    d.twin_i = g.d_twin + c;
    d.where = g.d_where;
}

unsigned blocks_for(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

void launch_update_plain_group(cp_handle* h, const Group& g, const double* F, int flag, double F_e, double F_r,
                               double* P, double* T, double* dPdF, int32_t* st, double* kF, double* kT) {
    switch (g.nt_class) {
        case 16:
            launch_update_plain<16, 16>(h->stream, h->d_lat[g.lattice], h->dopts, g.dev, F, flag, F_e, F_r, P, T, dPdF,
                                        st, h->d_stats, kF, kT, g.lattice);
            break;
        case 32:
            launch_update_plain<32, 32>(h->stream, h->d_lat[g.lattice], h->dopts, g.dev, F, flag, F_e, F_r, P, T, dPdF,
                                        st, h->d_stats, kF, kT, g.lattice);
            break;
        default:
            launch_update_plain<64, 48>(h->stream, h->d_lat[g.lattice], h->dopts, g.dev, F, flag, F_e, F_r, P, T, dPdF,
                                        st, h->d_stats, kF, kT, g.lattice);
            break;
    }
}

cudaError_t launch_assemble_plain_group(cp_handle* h, const Group& g, const double* U, double F_e, double F_r,
                                        double* Ke, double* Re, int32_t* st) {
    switch (g.nt_class) {
        case 16:
            return launch_assemble_plain<16, 16>(h->stream, h->d_lat[g.lattice], h->dopts, g.dev, U, h->d_gradN,
                                                 h->d_JxW, h->uniform, F_e, F_r, Ke, Re, st, h->d_stats, g.lattice);
        case 32:
            return launch_assemble_plain<32, 32>(h->stream, h->d_lat[g.lattice], h->dopts, g.dev, U, h->d_gradN,
                                                 h->d_JxW, h->uniform, F_e, F_r, Ke, Re, st, h->d_stats, g.lattice);
        default:
            return launch_assemble_plain<64, 48>(h->stream, h->d_lat[g.lattice], h->dopts, g.dev, U, h->d_gradN,
                                                 h->d_JxW, h->uniform, F_e, F_r, Ke, Re, st, h->d_stats, g.lattice);
    }
}

void timing_begin(cp_handle* h, int gi, cudaEvent_t* a) {
    if (!h->timing) return;
    cudaEventCreate(a);
    cudaEventRecord(*a, h->stream);
    (void)gi;
}
void timing_end(cp_handle* h, int gi, cudaEvent_t a) {
    if (!h->timing) return;
    cudaEvent_t b;
    cudaEventCreate(&b);
    cudaEventRecord(b, h->stream);
    h->pending.push_back({a, b, gi});
}

// Sort internal qps [i0, i0 + m) of a group by potentially-active-set size
// (descending) into positions i0.. of its permutation.
template <class FSrc>
void sort_group(cp_handle* h, const Group& g, FSrc fs, int64_t i0, int64_t m) {
    cudaMemsetAsync(g.d_hist, 0, sizeof(int) * SORT_BUCKETS, h->stream);
    g.sorted = true;
    classify_kernel<FSrc><<<blocks_for(m, QP_BLOCK), QP_BLOCK, 0, h->stream>>>(h->d_lat[g.lattice], h->dopts, g.dev,
                                                                             fs, i0, m, g.d_key, g.d_hist);
    bucket_scan_kernel<<<1, 32, 0, h->stream>>>(g.d_hist, g.d_hist + SORT_BUCKETS);
    bucket_scatter_kernel<<<blocks_for(m, 256), 256, 0, h->stream>>>(g.d_key, i0, m, g.d_hist + SORT_BUCKETS,
                                                                    g.d_perm + i0);
}

template <class FSrc>
constexpr int fsrc_path() {
    return std::is_same<FSrc, FromMesh>::value ? 1 : 0;
}

template <int PMAX, class FSrc>
cudaError_t launch_update2_shape(cudaStream_t s, const U2Args& a, const FSrc& fs, int v) {
    switch (v) {
        case 0: return launch_update2_v<PMAX, FSrc, 0>(s, a, fs);
        case 1: return launch_update2_v<PMAX, FSrc, 1>(s, a, fs);
        case 2: return launch_update2_v<PMAX, FSrc, 2>(s, a, fs);
        case 3: return launch_update2_v<PMAX, FSrc, 3>(s, a, fs);
        default: return launch_update4<PMAX, FSrc>(s, a, fs);
    }
}

// the quad kernels' shared-memory limit, for the current device
cudaError_t prepare_update4_all() {
    cudaError_t e = cudaSuccess;
    const cudaError_t r[6] = {prepare_update4<16, FromArray>(), prepare_update4<32, FromArray>(),
                              prepare_update4<48, FromArray>(), prepare_update4<16, FromMesh>(),
                              prepare_update4<32, FromMesh>(),  prepare_update4<48, FromMesh>()};
    for (cudaError_t x : r)
        if (x != cudaSuccess) e = x;
    return e;
}

// the sorted update of internal qps [i0, i0 + m) of group g (sort done) in
// launch shape v (-1: the group's tuned shape, else the default rule)
template <class FSrc>
cudaError_t launch_update2(cp_handle* h, const Group& g, FSrc fs, int64_t i0, int64_t m, int flag, double F_e,
                           double F_r, double* P, double* T, double* dPdF, double* stage, int32_t* st, double* kF,
                           double* kT, int v = -1) {
    const int pmax = g.nt_class == 16 ? 16 : (g.nt_class == 32 ? 32 : 48);
    if (v < 0 && h->opts.update_variant > 0) v = h->opts.update_variant - 1;
    if (v < 0) v = g.tuned[fsrc_path<FSrc>()];
    if (v < 0) v = u2_default_variant(pmax, m);
    if (v == U2_QUAD && h->dopts.max_search != 1) v = u2_default_variant(pmax, m);  // one slip-search pass only
    const U2Args a{h->d_lat[g.lattice], h->dopts, g.dev, g.d_perm + i0, m, flag, F_e, F_r, P, T, dPdF, stage, st,
                   h->d_stats, kF, kT, g.lattice, g.d_hist, h->num_sms};
    switch (pmax) {
        case 16: return launch_update2_shape<16>(h->stream, a, fs, v);
        case 32: return launch_update2_shape<32>(h->stream, a, fs, v);
        default: return launch_update2_shape<48>(h->stream, a, fs, v);
    }
}

// calculatePlasticity over internal qps [i0, i0 + m) of group gi (sort + update)
template <class FSrc>
void sorted_update_group(cp_handle* h, size_t gi, FSrc fs, int flag, double F_e, double F_r, double* P, double* T,
                         double* dPdF, double* stage, int32_t* st, double* kF, double* kT, int64_t i0 = 0,
                         int64_t m = -1) {
    const Group& g = h->groups[gi];
    if (m < 0) m = g.count - i0;
    if (m <= 0) return;
    sort_group(h, g, fs, i0, m);
    cudaEvent_t ev{};
    timing_begin(h, (int)gi, &ev);
    launch_update2(h, g, fs, i0, m, flag, F_e, F_r, P, T, dPdF, stage, st, kF, kT);
    timing_end(h, (int)gi, ev);
}

uint64_t bits_of(double x) {
    uint64_t u;
    std::memcpy(&u, &x, sizeof u);
    return u;
}

// Run enqueue() (the stream work of one call) through a CUDA graph captured
// for this key: captured on first use (or when the key changes: the cached
// graph is updated in place when its topology allows, else re-instantiated)
// and launched with one cudaGraphLaunch.  Without use_graphs, with launch
// timing on, or when the stream is already being captured by the caller, the
// work is enqueued directly.
template <class Enqueue>
int run_graph(cp_handle* h, const cp_handle::GraphKey& key, Enqueue enqueue) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(h, cudaStreamIsCapturing(h->stream, &cs));
    if (!h->opts.use_graphs || h->timing || cs != cudaStreamCaptureStatusNone) return enqueue();
    cp_handle::GraphEntry* hit = nullptr;
    for (auto& e : h->graphs)
        if (e.exec && e.key == key) hit = &e;
    if (!hit) {
        CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if (rc != CP_OK || e != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc != CP_OK ? rc : cuda_fail(h, e == cudaSuccess ? cudaErrorUnknown : e, "graph capture");
        }
        // a slot: an unused one, else the least recently used (updated in
        // place if the topology matches, else re-instantiated)
        constexpr size_t MAX_GRAPHS = 6;
        if (h->graphs.size() < MAX_GRAPHS) {
            h->graphs.emplace_back();
            hit = &h->graphs.back();
        } else {
            hit = &h->graphs[0];
            for (auto& x : h->graphs)
                if (x.last_use < hit->last_use) hit = &x;
        }
        bool ok = false;
        if (hit->exec) {
            cudaGraphExecUpdateResultInfo info;
            ok = cudaGraphExecUpdate(hit->exec, g, &info) == cudaSuccess;
            if (!ok) {
                cudaGetLastError();
                cudaGraphExecDestroy(hit->exec);
                hit->exec = nullptr;
            }
        }
        if (!ok) {
            const cudaError_t ei = cudaGraphInstantiate(&hit->exec, g, 0);
            if (ei != cudaSuccess) {
                hit->exec = nullptr;
                hit->key = cp_handle::GraphKey{};
                cudaGraphDestroy(g);
                return cuda_fail(h, ei, "cudaGraphInstantiate");
            }
        }
        cudaGraphDestroy(g);
        hit->key = key;
        ++h->graph_captures;
    }
    hit->last_use = ++h->graph_clock;
    CK(h, cudaGraphLaunch(hit->exec, h->stream));
    ++h->graph_launches;
    // every graph of this handle runs the sort of every lattice group, so the
    // keys of a replay are those of this call
    for (const auto& g : h->groups) g.sorted = true;
    return CP_OK;
}

// The reference-order update of every group (stream launches): one thread per
// qp on up to 64 threads per SM, each with a scratch slot of the size the
// largest lattice needs, allocated on first use and capped at 2 GiB.
int dispatch_update_ref(cp_handle* h, const double* F, int flag, double F_e, double F_r, double* P, double* T,
                        double* dPdF, int32_t* st) {
    if (!h->d_refscratch) {
        const int64_t slot = ref_scratch_doubles(h->n_max);
        int64_t threads = (int64_t)h->num_sms * 64;
        const int64_t cap = (2ll << 30) / (8 * slot);
        if (threads > cap) threads = cap < 64 ? 64 : cap;
        void* p = nullptr;
        if (cudaMalloc(&p, sizeof(double) * slot * threads) != cudaSuccess)
            return fail(h, CP_E_NOMEM, "reference_order: scratch allocation failed");
        h->d_refscratch = static_cast<double*>(p);
        h->ref_slot = slot;
        h->ref_threads = threads;
    }
    double* kF = flag == 0 ? h->d_keepF : nullptr;
    double* kT = flag == 0 ? h->d_keepT : nullptr;
    for (size_t gi = 0; gi < h->groups.size(); ++gi) {
        const auto& g = h->groups[gi];
        cudaEvent_t ev{};
        timing_begin(h, (int)gi, &ev);
        const cudaError_t e = launch_update_ref(h->stream, h->d_lat[g.lattice], h->dopts, g.dev, F, flag, F_e, F_r, P,
                                                T, dPdF, st, h->d_stats, kF, kT, g.lattice, h->d_refscratch,
                                                h->ref_slot, h->ref_threads);
        timing_end(h, (int)gi, ev);
        if (e != cudaSuccess) return cuda_fail(h, e, "update_ref_kernel");
    }
    if (flag == 0) h->have_post = true;
    return CP_OK;
}

int dispatch_update(cp_handle* h, const double* F, int flag, double F_e, double F_r, double* P, double* T,
                    double* dPdF, int32_t* st) {
    if (h->opts.reference_order) return dispatch_update_ref(h, F, flag, F_e, F_r, P, T, dPdF, st);
    if (!h->opts.plain_kernel) {
        double* kF = flag == 0 ? h->d_keepF : nullptr;
        double* kT = flag == 0 ? h->d_keepT : nullptr;
        cp_handle::GraphKey key;
        key.kind = 0;
        key.p[0] = F;
        key.p[1] = P;
        key.p[2] = T;
        key.p[3] = dPdF;
        key.p[4] = st;
        key.flag = flag;
        key.fe = bits_of(F_e);
        key.fr = bits_of(F_r);
        key.epoch = h->tune_epoch;
        const int rc = run_graph(h, key, [&]() -> int {
            for (size_t gi = 0; gi < h->groups.size(); ++gi)
                sorted_update_group(h, gi, FromArray{F}, flag, F_e, F_r, P, T, dPdF, nullptr, st, kF, kT);
            CK(h, cudaGetLastError());
            return CP_OK;
        });
        if (rc != CP_OK) return rc;
        if (flag == 0) h->have_post = true;
        return CP_OK;
    }
    double* kF = flag == 0 ? h->d_keepF : nullptr;
    double* kT = flag == 0 ? h->d_keepT : nullptr;
    for (size_t gi = 0; gi < h->groups.size(); ++gi) {
        const auto& g = h->groups[gi];
        cudaEvent_t ev{};
        timing_begin(h, (int)gi, &ev);
        launch_update_plain_group(h, g, F, flag, F_e, F_r, P, T, dPdF, st, kF, kT);
        timing_end(h, (int)gi, ev);
    }
    CK(h, cudaGetLastError());
    if (flag == 0) h->have_post = true;
    return CP_OK;
}

int check_device(cp_handle* h) {
    CK(h, cudaSetDevice(h->device));
    return CP_OK;
}

// ---------------------------------------------------------------- history order
// The sorted update reads each qp's history (structure of arrays, component c
// of internal qp i at c * count + i) at the internal indices of its sort
// order; when the internal order is the sort order, a warp's 32 qps are 32
// neighbouring indices and every history access coalesces, instead of one
// 32-byte sector per 8-byte value.  So cp_commit, which copies the _iter half
// over the _conv half anyway, also permutes each group's history (both
// halves), twin flags and qp map into the order of the keys of the last sort:
// a stable counting sort by key within each reorder segment.  The segments are
// bounded by every internal index at which a caller-order chunk of the host
// calls starts, so each chunk keeps its contiguous internal range.  Every
// kernel addresses the history by internal index and maps to the caller by
// qp[i], so no result changes.

// Stable counting sort by key of internal qps [seg[b], seg[b + 1]) (one block
// per segment, tiles of 256 in order): src[p] is the internal qp that moves to
// position p.
__global__ void __launch_bounds__(256) reorder_sort_kernel(const unsigned char* __restrict__ key,
                                                           const int* __restrict__ seg, int* __restrict__ src) {
    __shared__ int base[SORT_BUCKETS];
    __shared__ int wcnt[8][SORT_BUCKETS];
    const int lo = seg[blockIdx.x], hi = seg[blockIdx.x + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < SORT_BUCKETS) base[tid] = 0;
    __syncthreads();
    for (int i = lo + tid; i < hi; i += 256) atomicAdd(&base[key[i] < SORT_BUCKETS ? key[i] : SORT_BUCKETS - 1], 1);
    __syncthreads();
    if (tid == 0) {
        int acc = lo;
        for (int b = 0; b < SORT_BUCKETS; ++b) {
            const int c = base[b];
            base[b] = acc;
            acc += c;
        }
    }
    __syncthreads();
    for (int t0 = lo; t0 < hi; t0 += 256) {
        const int i = t0 + tid;
        const bool valid = i < hi;
        const int k = valid ? (key[i] < SORT_BUCKETS ? key[i] : SORT_BUCKETS - 1) : SORT_BUCKETS;
        for (int e = tid; e < 8 * SORT_BUCKETS; e += 256) (&wcnt[0][0])[e] = 0;
        __syncthreads();
        const unsigned same = __match_any_sync(0xffffffffu, k);
        const int rank = __popc(same & ((1u << lane) - 1u));
        if (valid && lane == __ffs(same) - 1) wcnt[warp][k] = __popc(same);
        __syncthreads();
        if (valid) {
            int off = base[k] + rank;
            for (int w = 0; w < warp; ++w) off += wcnt[w][k];
            src[off] = i;
        }
        __syncthreads();
        if (tid < SORT_BUCKETS) {
            int sum = 0;
            for (int w = 0; w < 8; ++w) sum += wcnt[w][tid];
            base[tid] += sum;
        }
        __syncthreads();
    }
}

// dst[r * count + p] = srcv[r * count + src[p]] for every row r of a field block
template <class T>
__global__ void reorder_gather_kernel(const T* __restrict__ srcv, T* __restrict__ dst, int64_t rows, int64_t count,
                                      const int* __restrict__ src) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    const int64_t from = src[p];
    for (int64_t r = 0; r < rows; ++r) dst[r * count + p] = srcv[r * count + from];
}

// inv[src[p]] = p: the new position of every old internal index ...
__global__ void reorder_inverse_kernel(const int* __restrict__ src, int64_t count, int* __restrict__ inv) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < count) inv[src[p]] = (int)p;
}
// ... and where[j] <- inv[where[j]] (a second launch, after the inverse is whole)
__global__ void reorder_where_kernel(const int* __restrict__ inv, int64_t count, int* __restrict__ where) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < count) where[j] = inv[where[j]];
}

// The internal indices at which reorder segments of group g start (with 0 and
// count): every start of a caller-order chunk of qps or of cells.
std::vector<int> reorder_segments(const cp_handle* h, const Group& g) {
    std::vector<int64_t> b{0, g.count};
    const auto& q = g.qp_host;
    const int cq = chunks_for(h->n_qp);
    for (int c = 1; c < cq; ++c)
        b.push_back(std::lower_bound(q.begin(), q.end(), h->n_qp * c / cq) - q.begin());
    if (h->n_cells > 0)
        for (int c = 1; c < cq; ++c)
            b.push_back(std::lower_bound(q.begin(), q.end(), 8 * (h->n_cells * c / cq)) - q.begin());
    std::sort(b.begin(), b.end());
    b.erase(std::unique(b.begin(), b.end()), b.end());
    return std::vector<int>(b.begin(), b.end());
}

}  // namespace

// ---------------------------------------------------------------- C ABI
extern "C" {

int cp_options_default(cp_options_t* o) {
    if (!o) return CP_E_ARG;
    std::memset(o, 0, sizeof *o);
    o->stress_tolerance = 1.0e-9;
    o->max_slip_search_iterations = 1;
    o->max_solver_iterations = 1;
    o->enable_multiphase = 0;
    o->device = 0;
    o->update_variant = 0;
    o->use_graphs = 1;
    return CP_OK;
}

int cp_material_add_dummy_twin(cp_material_t* m) {
    if (!m || m->n_slip < 1 || m->n_slip + 1 > CP_MAX_SYSTEMS) return CP_E_ARG;
    const int d = m->n_slip;
    m->n_twin = 1;
    m->twinning_enabled = 0;
    m->slip_normal[3 * d] = 1.0;
    m->slip_normal[3 * d + 1] = 0.0;
    m->slip_normal[3 * d + 2] = 0.0;
    m->slip_direction[3 * d] = 0.0;
    m->slip_direction[3 * d + 1] = 1.0;
    m->slip_direction[3 * d + 2] = 0.0;
    for (int j = 0; j < CP_MAX_SYSTEMS; ++j) {
        m->latent_hardening[d * CP_MAX_SYSTEMS + j] = 0.0;
        m->latent_hardening[j * CP_MAX_SYSTEMS + d] = 0.0;
    }
    m->initial_slip_resistance[d] = 10e14;
    m->initial_hardening_modulus[d] = 1.0;
    m->power_law_exponent[d] = 0.0;
    m->saturation_stress[d] = 10e15;
    m->kinematic_c1[d] = 0.0;
    m->kinematic_c2[d] = 0.0;
    return CP_OK;
}

int cp_create(const cp_material_t* lattices, int32_t n_lattices, const cp_options_t* opts, cp_handle** out) {
    if (!out || !lattices || n_lattices < 1 || n_lattices > CP_MAX_LATTICES) return CP_E_ARG;
    *out = nullptr;
    for (int l = 0; l < n_lattices; ++l) {
        const cp_material_t& m = lattices[l];
        if (m.n_slip < 1 || m.n_twin < 1 || m.n_slip + m.n_twin > CP_MAX_SYSTEMS) return CP_E_ARG;
    }
    cp_handle* h = new cp_handle();
    if (opts)
        h->opts = *opts;
    else
        cp_options_default(&h->opts);
    if (h->opts.max_slip_search_iterations < 0 || h->opts.max_solver_iterations < 0) {
        delete h;
        return CP_E_ARG;
    }
    h->device = h->opts.device;
    if (cudaSetDevice(h->device) != cudaSuccess || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return CP_E_CUDA;
    }
    bool ok = cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking) == cudaSuccess;
    for (int c = 0; ok && c < MAX_CHUNKS; ++c)
        ok = cudaEventCreateWithFlags(&h->ev_in[c], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&h->ev_done[c], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        cp_destroy(h);
        return CP_E_CUDA;
    }
    if (cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess ||
        prepare_ke_tc() != cudaSuccess || prepare_update4_all() != cudaSuccess ||
        cudaMalloc(&h->d_tc_err, sizeof(int)) != cudaSuccess ||
        cudaMemset(h->d_tc_err, 0, sizeof(int)) != cudaSuccess) {
        cp_destroy(h);
        return CP_E_CUDA;
    }
    h->dopts.tol = h->opts.stress_tolerance;
    h->dopts.max_search = h->opts.max_slip_search_iterations;
    h->dopts.max_solver = h->opts.max_solver_iterations;
    h->dopts.multiphase = h->opts.enable_multiphase;
    h->n_lat = n_lattices;
    h->mats.assign(lattices, lattices + n_lattices);
    for (int l = 0; l < n_lattices; ++l) {
        const cp_material_t& m = lattices[l];
        LatDev hl;
        std::memset(&hl, 0, sizeof hl);
        hl.n = m.n_slip + m.n_twin;
        hl.ns = m.n_slip;
        hl.nw = m.n_twin;
        hl.twinning = m.twinning_enabled;
        std::memcpy(hl.C, m.elastic_stiffness, sizeof hl.C);
        std::memcpy(hl.m, m.slip_direction, sizeof hl.m);
        std::memcpy(hl.nn, m.slip_normal, sizeof hl.nn);
        std::memcpy(hl.q, m.latent_hardening, sizeof hl.q);
        std::memcpy(hl.s0, m.initial_slip_resistance, sizeof hl.s0);
        std::memcpy(hl.h0, m.initial_hardening_modulus, sizeof hl.h0);
        std::memcpy(hl.ss, m.saturation_stress, sizeof hl.ss);
        std::memcpy(hl.a, m.power_law_exponent, sizeof hl.a);
        std::memcpy(hl.C1, m.kinematic_c1, sizeof hl.C1);
        std::memcpy(hl.C2, m.kinematic_c2, sizeof hl.C2);
        hl.twin_thr = m.twin_threshold_fraction;
        hl.twin_sat = m.twin_saturation_factor;
        hl.twin_shear = m.twin_shear;
        LatDev* d = nullptr;
        if (cudaMalloc(&d, sizeof(LatDev)) != cudaSuccess ||
            cudaMemcpy(d, &hl, sizeof hl, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFree(d);
            cp_destroy(h);
            return CP_E_CUDA;
        }
        h->d_lat.push_back(d);
        h->n_max = std::max(h->n_max, hl.n);
        h->ns_max = std::max(h->ns_max, hl.ns);
        h->nw_max = std::max(h->nw_max, hl.nw);
    }
    *out = h;
    return CP_OK;
}

void cp_destroy(cp_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_qps(h);
    free_mesh(h);
    cudaFree(h->d_avg_partial);
    cudaFree(h->d_avg_out);
    cudaFree(h->d_tc_err);
    cudaFree(h->d_refscratch);
    for (auto* d : h->d_lat) cudaFree(d);
    for (auto& p : h->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->s_in) cudaStreamDestroy(h->s_in);
    if (h->s_out) cudaStreamDestroy(h->s_out);
    for (int c = 0; c < MAX_CHUNKS; ++c) {
        if (h->ev_in[c]) cudaEventDestroy(h->ev_in[c]);
        if (h->ev_done[c]) cudaEventDestroy(h->ev_done[c]);
    }
    delete h;
}

const char* cp_last_error(const cp_handle* h) { return h ? h->err.c_str() : "null handle"; }

void* cp_stream(cp_handle* h) { return h ? (void*)h->stream : nullptr; }

int64_t cp_num_qps(const cp_handle* h) { return h ? h->n_qp : 0; }

int cp_bind_qps(cp_handle* h, int64_t n_qp, const int32_t* lattice_id, const double* rod) {
    if (!h) return CP_E_ARG;
    if (n_qp < 1 || !lattice_id || !rod) return fail(h, CP_E_ARG, "cp_bind_qps: bad arguments");
    if (int rc = check_device(h)) return rc;
    std::vector<std::vector<int64_t>> idx(h->n_lat);
    for (int64_t k = 0; k < n_qp; ++k) {
        const int l = lattice_id[k];
        if (l < 0 || l >= h->n_lat) return fail(h, CP_E_ARG, "cp_bind_qps: lattice id out of range");
        idx[l].push_back(k);
    }
    free_qps(h);
    free_mesh(h);
    h->n_qp = n_qp;
    h->lattice_of.assign(lattice_id, lattice_id + n_qp);
    double* d_rod = nullptr;
    CK(h, cudaMalloc(&d_rod, sizeof(double) * 3 * n_qp));
    CK(h, cudaMemcpy(d_rod, rod, sizeof(double) * 3 * n_qp, cudaMemcpyHostToDevice));
    for (int l = 0; l < h->n_lat; ++l) {
        if (idx[l].empty()) continue;
        Group g;
        g.lattice = l;
        g.ns = h->mats[l].n_slip;
        g.nw = h->mats[l].n_twin;
        g.n = g.ns + g.nw;
        g.nt_class = nt_class_of(g.n);
        g.count = (int64_t)idx[l].size();
        if (cudaMalloc(&g.d_qp, sizeof(int64_t) * g.count) != cudaSuccess ||
            cudaMalloc(&g.d_block, sizeof(double) * group_doubles(g.n, g.ns, g.nw, g.count)) != cudaSuccess ||
            cudaMalloc(&g.d_twin, sizeof(int) * 2 * g.count) != cudaSuccess ||
            cudaMalloc(&g.d_key, g.count) != cudaSuccess ||
            cudaMalloc(&g.d_perm, sizeof(int) * g.count) != cudaSuccess ||
            cudaMalloc(&g.d_hist, sizeof(int) * 2 * SORT_BUCKETS) != cudaSuccess ||
            cudaMalloc(&g.d_qp_tmp, sizeof(int64_t) * g.count) != cudaSuccess ||
            cudaMalloc(&g.d_where, sizeof(int) * g.count) != cudaSuccess ||
            cudaMemset(g.d_key, 0, g.count) != cudaSuccess) {
            free_group(g);
            cudaFree(d_rod);
            free_qps(h);
            return fail(h, CP_E_NOMEM, "cp_bind_qps: device allocation failed");
        }
        CK(h, cudaMemcpy(g.d_qp, idx[l].data(), sizeof(int64_t) * g.count, cudaMemcpyHostToDevice));
        {
            std::vector<int> iota((size_t)g.count);
            for (int64_t j = 0; j < g.count; ++j) iota[(size_t)j] = (int)j;
            CK(h, cudaMemcpy(g.d_where, iota.data(), sizeof(int) * g.count, cudaMemcpyHostToDevice));
        }
        g.qp_host = idx[l];
        carve(g);
        init_state_kernel<<<blocks_for(g.count, 256), 256, 0, h->stream>>>(h->d_lat[l], g.dev, d_rod);
        h->groups.push_back(g);
    }
    CK(h, cudaGetLastError());
    CK(h, cudaStreamSynchronize(h->stream));
    cudaFree(d_rod);
    if (cudaMalloc(&h->d_stats, sizeof(int32_t) * 8 * n_qp) != cudaSuccess ||
        cudaMalloc(&h->d_keepF, sizeof(double) * 9 * n_qp) != cudaSuccess ||
        cudaMalloc(&h->d_keepT, sizeof(double) * 9 * n_qp) != cudaSuccess)
        return fail(h, CP_E_NOMEM, "cp_bind_qps: device allocation failed");
    CK(h, cudaMemset(h->d_stats, 0, sizeof(int32_t) * 8 * n_qp));
    return CP_OK;
}

static int ensure_staging(cp_handle* h, bool need_dPdF) {
    const int64_t n = h->n_qp;
    if (!h->d_F) {
        if (cudaMalloc(&h->d_F, sizeof(double) * 9 * n) != cudaSuccess ||
            cudaMalloc(&h->d_P, sizeof(double) * 9 * n) != cudaSuccess ||
            cudaMalloc(&h->d_T, sizeof(double) * 9 * n) != cudaSuccess ||
            cudaMalloc(&h->d_status, sizeof(int32_t) * n) != cudaSuccess)
            return fail(h, CP_E_NOMEM, "staging allocation failed");
    }
    if (need_dPdF && h->dPdF_cap < (size_t)n) {
        cudaFree(h->d_dPdF);
        h->d_dPdF = nullptr;
        if (cudaMalloc(&h->d_dPdF, sizeof(double) * 81 * n) != cudaSuccess)
            return fail(h, CP_E_NOMEM, "staging allocation failed");
        h->dPdF_cap = (size_t)n;
    }
    return CP_OK;
}

int cp_update_device(cp_handle* h, const double* d_F, int32_t flag, double F_e, double F_r, double* d_P,
                     double* d_T, double* d_dPdF, int32_t* d_status) {
    if (!h) return CP_E_ARG;
    if (h->n_qp == 0) return fail(h, CP_E_STATE, "cp_update: no qps bound");
    if (!d_F || (flag != 0 && flag != 1)) return fail(h, CP_E_ARG, "cp_update: bad arguments");
    if (int rc = check_device(h)) return rc;
    return dispatch_update(h, d_F, flag, F_e, F_r, d_P, d_T, d_dPdF, d_status);
}

int cp_update(cp_handle* h, const double* h_F, int32_t flag, double F_e, double F_r, double* h_P, double* h_T,
              double* h_dPdF, int32_t* h_status) {
    if (!h) return CP_E_ARG;
    if (h->n_qp == 0) return fail(h, CP_E_STATE, "cp_update: no qps bound");
    if (!h_F || (flag != 0 && flag != 1)) return fail(h, CP_E_ARG, "cp_update: bad arguments");
    if (int rc = check_device(h)) return rc;
    if (int rc = ensure_staging(h, flag == 1 && h_dPdF)) return rc;
    const int64_t n = h->n_qp;
    double* dd = (flag == 1 && h_dPdF) ? h->d_dPdF : nullptr;
    double* dP = h_P ? h->d_P : nullptr;
    double* dT = h_T ? h->d_T : nullptr;
    if (h->opts.plain_kernel || h->opts.reference_order) {
        CK(h, cudaMemcpyAsync(h->d_F, h_F, sizeof(double) * 9 * n, cudaMemcpyHostToDevice, h->stream));
        if (int rc = dispatch_update(h, h->d_F, flag, F_e, F_r, dP, dT, dd, h->d_status)) return rc;
        if (h_P) CK(h, cudaMemcpyAsync(h_P, h->d_P, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost, h->stream));
        if (h_T) CK(h, cudaMemcpyAsync(h_T, h->d_T, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost, h->stream));
        if (dd) CK(h, cudaMemcpyAsync(h_dPdF, dd, sizeof(double) * 81 * n, cudaMemcpyDeviceToHost, h->stream));
        if (h_status)
            CK(h, cudaMemcpyAsync(h_status, h->d_status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        return CP_OK;
    }
    // chunk c: F in on s_in, the sort + update of its qps on the compute
    // stream, its outputs out on s_out while the next chunk computes
    double* kF = flag == 0 ? h->d_keepF : nullptr;
    double* kT = flag == 0 ? h->d_keepT : nullptr;
    const int C = chunks_for(n);
    for (int c = 0; c < C; ++c) {
        const int64_t k0 = n * c / C, k1 = n * (c + 1) / C, nk = k1 - k0;
        CK(h, cudaMemcpyAsync(h->d_F + 9 * k0, h_F + 9 * k0, sizeof(double) * 9 * nk, cudaMemcpyHostToDevice,
                              h->s_in));
        CK(h, cudaEventRecord(h->ev_in[c], h->s_in));
        CK(h, cudaStreamWaitEvent(h->stream, h->ev_in[c], 0));
        for (size_t gi = 0; gi < h->groups.size(); ++gi) {
            const auto& q = h->groups[gi].qp_host;
            const int64_t i0 = std::lower_bound(q.begin(), q.end(), k0) - q.begin();
            const int64_t i1 = std::lower_bound(q.begin(), q.end(), k1) - q.begin();
            sorted_update_group(h, gi, FromArray{h->d_F}, flag, F_e, F_r, dP, dT, dd, nullptr, h->d_status, kF, kT,
                                i0, i1 - i0);
        }
        CK(h, cudaGetLastError());
        CK(h, cudaEventRecord(h->ev_done[c], h->stream));
        CK(h, cudaStreamWaitEvent(h->s_out, h->ev_done[c], 0));
        if (h_P)
            CK(h, cudaMemcpyAsync(h_P + 9 * k0, h->d_P + 9 * k0, sizeof(double) * 9 * nk, cudaMemcpyDeviceToHost,
                                  h->s_out));
        if (h_T)
            CK(h, cudaMemcpyAsync(h_T + 9 * k0, h->d_T + 9 * k0, sizeof(double) * 9 * nk, cudaMemcpyDeviceToHost,
                                  h->s_out));
        if (dd)
            CK(h, cudaMemcpyAsync(h_dPdF + 81 * k0, dd + 81 * k0, sizeof(double) * 81 * nk, cudaMemcpyDeviceToHost,
                                  h->s_out));
        if (h_status)
            CK(h, cudaMemcpyAsync(h_status + k0, h->d_status + k0, sizeof(int32_t) * nk, cudaMemcpyDeviceToHost,
                                  h->s_out));
    }
    CK(h, cudaStreamSynchronize(h->s_out));
    CK(h, cudaStreamSynchronize(h->stream));
    if (flag == 0) h->have_post = true;
    return CP_OK;
}

int cp_get_stats(cp_handle* h, int32_t* h_stats) {
    if (!h || !h_stats) return CP_E_ARG;
    if (h->n_qp == 0) return fail(h, CP_E_STATE, "no qps bound");
    if (int rc = check_device(h)) return rc;
    CK(h, cudaMemcpyAsync(h_stats, h->d_stats, sizeof(int32_t) * 8 * h->n_qp, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return CP_OK;
}

int cp_bind_mesh(cp_handle* h, int64_t n_cells, const double* grad_N, const double* JxW, int32_t uniform) {
    if (!h) return CP_E_ARG;
    if (n_cells < 1 || !grad_N || !JxW) return fail(h, CP_E_ARG, "cp_bind_mesh: bad arguments");
    if (h->n_qp != 8 * n_cells) return fail(h, CP_E_STATE, "cp_bind_mesh: bound qps must be 8 per cell");
    for (int64_t c = 0; c < n_cells; ++c)
        for (int q = 1; q < 8; ++q)
            if (h->lattice_of[8 * c + q] != h->lattice_of[8 * c])
                return fail(h, CP_E_ARG, "cp_bind_mesh: the 8 qps of a cell must share a lattice");
    if (int rc = check_device(h)) return rc;
    free_mesh(h);
    const size_t ng = uniform ? 192 : (size_t)192 * n_cells, nw = uniform ? 8 : (size_t)8 * n_cells;
    if (cudaMalloc(&h->d_gradN, sizeof(double) * ng) != cudaSuccess ||
        cudaMalloc(&h->d_JxW, sizeof(double) * nw) != cudaSuccess)
        return fail(h, CP_E_NOMEM, "cp_bind_mesh: allocation failed");
    CK(h, cudaMemcpy(h->d_gradN, grad_N, sizeof(double) * ng, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(h->d_JxW, JxW, sizeof(double) * nw, cudaMemcpyHostToDevice));
    h->n_cells = n_cells;
    h->uniform = uniform ? 1 : 0;
    return CP_OK;
}

int cp_assemble_device(cp_handle* h, const double* d_U, double F_e, double F_r, double* d_Ke, double* d_Re,
                       int32_t* d_status) {
    if (!h) return CP_E_ARG;
    if (h->n_cells == 0) return fail(h, CP_E_STATE, "cp_assemble: no mesh bound");
    if (!d_U || !d_Ke || !d_Re) return fail(h, CP_E_ARG, "cp_assemble: bad arguments");
    if (h->opts.reference_order)
        return fail(h, CP_E_UNSUPPORTED, "cp_assemble: reference_order runs cp_update / cp_update_device only");
    if (int rc = check_device(h)) return rc;
    if (!h->opts.plain_kernel) {
        if (!h->d_stage && cudaMalloc(&h->d_stage, sizeof(double) * 90 * h->n_qp) != cudaSuccess)
            return fail(h, CP_E_NOMEM, "cp_assemble: staging allocation failed");
        const FromMesh fm{d_U, h->d_gradN, h->d_JxW, h->uniform};
        cp_handle::GraphKey key;
        key.kind = 1;
        key.p[0] = d_U;
        key.p[1] = d_Ke;
        key.p[2] = d_Re;
        key.p[3] = d_status;
        key.flag = 1;
        key.fe = bits_of(F_e);
        key.fr = bits_of(F_r);
        key.epoch = h->tune_epoch;
        return run_graph(h, key, [&]() -> int {
            for (size_t gi = 0; gi < h->groups.size(); ++gi)
                sorted_update_group(h, gi, fm, 1, F_e, F_r, nullptr, nullptr, nullptr, h->d_stage, d_status,
                                    nullptr, nullptr);
            cudaEvent_t ev{};
            timing_begin(h, -1, &ev);
            contract_kernel<<<blocks_for(h->n_cells, CONTRACT_CELLS), CONTRACT_CELLS * 8, 0, h->stream>>>(
                h->d_stage, h->d_gradN, h->uniform, 0, h->n_cells, d_Ke, d_Re);
            timing_end(h, -1, ev);
            CK(h, cudaGetLastError());
            return CP_OK;
        });
    }
    for (size_t gi = 0; gi < h->groups.size(); ++gi) {
        const auto& g = h->groups[gi];
        cudaEvent_t ev{};
        timing_begin(h, (int)gi, &ev);
        const cudaError_t e = launch_assemble_plain_group(h, g, d_U, F_e, F_r, d_Ke, d_Re, d_status);
        timing_end(h, (int)gi, ev);
        if (e != cudaSuccess) return cuda_fail(h, e, "assemble_kernel");
    }
    return CP_OK;
}

int cp_assemble(cp_handle* h, const double* h_U, double F_e, double F_r, double* h_Ke, double* h_Re,
                int32_t* h_status) {
    if (!h) return CP_E_ARG;
    if (h->opts.reference_order)
        return fail(h, CP_E_UNSUPPORTED, "cp_assemble: reference_order runs cp_update / cp_update_device only");
    if (h->n_cells == 0) return fail(h, CP_E_STATE, "cp_assemble: no mesh bound");
    if (!h_U || !h_Ke || !h_Re) return fail(h, CP_E_ARG, "cp_assemble: bad arguments");
    if (int rc = check_device(h)) return rc;
    if (int rc = ensure_staging(h, false)) return rc;
    const int64_t nc = h->n_cells;
    if (!h->d_U) {
        if (cudaMalloc(&h->d_U, sizeof(double) * 24 * nc) != cudaSuccess ||
            cudaMalloc(&h->d_Ke, sizeof(double) * 576 * nc) != cudaSuccess ||
            cudaMalloc(&h->d_Re, sizeof(double) * 24 * nc) != cudaSuccess)
            return fail(h, CP_E_NOMEM, "cp_assemble: allocation failed");
    }
    if (h->opts.plain_kernel) {
        CK(h, cudaMemcpyAsync(h->d_U, h_U, sizeof(double) * 24 * nc, cudaMemcpyHostToDevice, h->stream));
        if (int rc = cp_assemble_device(h, h->d_U, F_e, F_r, h->d_Ke, h->d_Re, h->d_status)) return rc;
        CK(h, cudaMemcpyAsync(h_Ke, h->d_Ke, sizeof(double) * 576 * nc, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaMemcpyAsync(h_Re, h->d_Re, sizeof(double) * 24 * nc, cudaMemcpyDeviceToHost, h->stream));
        if (h_status)
            CK(h, cudaMemcpyAsync(h_status, h->d_status, sizeof(int32_t) * h->n_qp, cudaMemcpyDeviceToHost,
                                  h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        return CP_OK;
    }
    if (!h->d_stage && cudaMalloc(&h->d_stage, sizeof(double) * 90 * h->n_qp) != cudaSuccess)
        return fail(h, CP_E_NOMEM, "cp_assemble: staging allocation failed");
    // caller-order chunks of cells (as cp_update): U in on s_in, the sorted
    // update of the chunk's qps and its contraction on the compute stream, Ke,
    // Re and status out on s_out while the next chunk computes
    const FromMesh fm{h->d_U, h->d_gradN, h->d_JxW, h->uniform};
    const int C = chunks_for(h->n_qp);
    for (int c = 0; c < C; ++c) {
        const int64_t c0 = nc * c / C, c1 = nc * (c + 1) / C, ncc = c1 - c0;
        if (ncc <= 0) continue;
        CK(h, cudaMemcpyAsync(h->d_U + 24 * c0, h_U + 24 * c0, sizeof(double) * 24 * ncc, cudaMemcpyHostToDevice,
                              h->s_in));
        CK(h, cudaEventRecord(h->ev_in[c], h->s_in));
        CK(h, cudaStreamWaitEvent(h->stream, h->ev_in[c], 0));
        for (size_t gi = 0; gi < h->groups.size(); ++gi) {
            const auto& q = h->groups[gi].qp_host;
            const int64_t i0 = std::lower_bound(q.begin(), q.end(), 8 * c0) - q.begin();
            const int64_t i1 = std::lower_bound(q.begin(), q.end(), 8 * c1) - q.begin();
            sorted_update_group(h, gi, fm, 1, F_e, F_r, nullptr, nullptr, nullptr, h->d_stage, h->d_status, nullptr,
                                nullptr, i0, i1 - i0);
        }
        contract_kernel<<<blocks_for(ncc, CONTRACT_CELLS), CONTRACT_CELLS * 8, 0, h->stream>>>(
            h->d_stage, h->d_gradN, h->uniform, c0, c1, h->d_Ke, h->d_Re);
        CK(h, cudaGetLastError());
        CK(h, cudaEventRecord(h->ev_done[c], h->stream));
        CK(h, cudaStreamWaitEvent(h->s_out, h->ev_done[c], 0));
        CK(h, cudaMemcpyAsync(h_Ke + 576 * c0, h->d_Ke + 576 * c0, sizeof(double) * 576 * ncc, cudaMemcpyDeviceToHost,
                              h->s_out));
        CK(h, cudaMemcpyAsync(h_Re + 24 * c0, h->d_Re + 24 * c0, sizeof(double) * 24 * ncc, cudaMemcpyDeviceToHost,
                              h->s_out));
        if (h_status)
            CK(h, cudaMemcpyAsync(h_status + 8 * c0, h->d_status + 8 * c0, sizeof(int32_t) * 8 * ncc,
                                  cudaMemcpyDeviceToHost, h->s_out));
    }
    CK(h, cudaStreamSynchronize(h->s_out));
    CK(h, cudaStreamSynchronize(h->stream));
    return CP_OK;
}

// reads and clears the tensor-core contraction's error flag (synchronises)
static int check_tc_error(cp_handle* h) {
    int e = 0;
    CK(h, cudaMemcpyAsync(&e, h->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (e) {
        CK(h, cudaMemsetAsync(h->d_tc_err, 0, sizeof(int), h->stream));
        return fail(h, CP_E_CUDA, "tensor-core contraction: a wait expired (results incomplete)");
    }
    return CP_OK;
}

int cp_assemble_mixed_device(cp_handle* h, const double* d_U, double F_e, double F_r, float* d_Ke, double* d_Re,
                             int32_t* d_status) {
    if (!h) return CP_E_ARG;
    if (h->n_cells == 0) return fail(h, CP_E_STATE, "cp_assemble_mixed: no mesh bound");
    if (!d_U || !d_Ke || !d_Re) return fail(h, CP_E_ARG, "cp_assemble_mixed: bad arguments");
    if (!h->uniform) return fail(h, CP_E_UNSUPPORTED, "cp_assemble_mixed: needs a uniform mesh (shared gradients)");
    if (h->opts.plain_kernel || h->opts.reference_order)
        return fail(h, CP_E_UNSUPPORTED, "cp_assemble_mixed: needs the sorted update");
    if (int rc = check_device(h)) return rc;
    if (!h->d_stage && cudaMalloc(&h->d_stage, sizeof(double) * 90 * h->n_qp) != cudaSuccess)
        return fail(h, CP_E_NOMEM, "cp_assemble_mixed: staging allocation failed");
    const FromMesh fm{d_U, h->d_gradN, h->d_JxW, h->uniform};
    cp_handle::GraphKey key;
    key.kind = 3;
    key.p[0] = d_U;
    key.p[1] = d_Ke;
    key.p[2] = d_Re;
    key.p[3] = d_status;
    key.flag = 1;
    key.fe = bits_of(F_e);
    key.fr = bits_of(F_r);
    key.epoch = h->tune_epoch;
    return run_graph(h, key, [&]() -> int {
        for (size_t gi = 0; gi < h->groups.size(); ++gi)
            sorted_update_group(h, gi, fm, 1, F_e, F_r, nullptr, nullptr, nullptr, h->d_stage, d_status, nullptr,
                                nullptr);
        CK(h, cudaGetLastError());
        cudaEvent_t ev{};
        timing_begin(h, -2, &ev);
        CK(h, launch_ke_tc(h->stream, h->d_stage, h->d_gradN, 0, h->n_cells, d_Ke, d_Re, h->d_tc_err, h->num_sms));
        timing_end(h, -2, ev);
        return CP_OK;
    });
}

int cp_assemble_mixed(cp_handle* h, const double* h_U, double F_e, double F_r, float* h_Ke, double* h_Re,
                      int32_t* h_status) {
    if (!h) return CP_E_ARG;
    if (h->n_cells == 0) return fail(h, CP_E_STATE, "cp_assemble_mixed: no mesh bound");
    if (!h_U || !h_Ke || !h_Re) return fail(h, CP_E_ARG, "cp_assemble_mixed: bad arguments");
    if (int rc = check_device(h)) return rc;
    if (int rc = ensure_staging(h, false)) return rc;
    const int64_t nc = h->n_cells;
    if (!h->d_U) {
        if (cudaMalloc(&h->d_U, sizeof(double) * 24 * nc) != cudaSuccess ||
            cudaMalloc(&h->d_Ke, sizeof(double) * 576 * nc) != cudaSuccess ||
            cudaMalloc(&h->d_Re, sizeof(double) * 24 * nc) != cudaSuccess)
            return fail(h, CP_E_NOMEM, "cp_assemble_mixed: allocation failed");
    }
    float* dK = reinterpret_cast<float*>(h->d_Ke);  // FP32 Ke in the first half of the FP64 buffer
    CK(h, cudaMemcpyAsync(h->d_U, h_U, sizeof(double) * 24 * nc, cudaMemcpyHostToDevice, h->stream));
    if (int rc = cp_assemble_mixed_device(h, h->d_U, F_e, F_r, dK, h->d_Re, h->d_status)) return rc;
    CK(h, cudaMemcpyAsync(h_Ke, dK, sizeof(float) * 576 * nc, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaMemcpyAsync(h_Re, h->d_Re, sizeof(double) * 24 * nc, cudaMemcpyDeviceToHost, h->stream));
    if (h_status)
        CK(h, cudaMemcpyAsync(h_status, h->d_status, sizeof(int32_t) * h->n_qp, cudaMemcpyDeviceToHost, h->stream));
    return check_tc_error(h);
}

int cp_averages(cp_handle* h, double out[22]) {
    if (!h || !out) return CP_E_ARG;
    if (h->n_cells == 0) return fail(h, CP_E_STATE, "cp_averages: no mesh bound (JxW needed)");
    if (!h->have_post) return fail(h, CP_E_STATE, "cp_averages: no cp_update with stiffness_flag 0 yet");
    if (int rc = check_device(h)) return rc;
    int64_t nblocks = 0;
    for (const auto& g : h->groups) nblocks += blocks_for(g.count, AVG_BLOCK);
    if (h->avg_cap < nblocks) {
        cudaFree(h->d_avg_partial);
        h->d_avg_partial = nullptr;
        if (cudaMalloc(&h->d_avg_partial, sizeof(double) * AVG_N * nblocks) != cudaSuccess)
            return fail(h, CP_E_NOMEM, "cp_averages: allocation failed");
        h->avg_cap = nblocks;
    }
    if (!h->d_avg_out && cudaMalloc(&h->d_avg_out, sizeof(double) * AVG_N) != cudaSuccess)
        return fail(h, CP_E_NOMEM, "cp_averages: allocation failed");
    int64_t off = 0;
    for (const auto& g : h->groups) {
        const unsigned nb = blocks_for(g.count, AVG_BLOCK);
        averages_partial_kernel<<<nb, AVG_BLOCK, 0, h->stream>>>(h->d_lat[g.lattice], g.dev, h->d_keepF, h->d_keepT,
                                                                 h->d_JxW, h->uniform,
                                                                 h->d_avg_partial + off * AVG_N);
        off += nb;
    }
    averages_final_kernel<<<1, 32, 0, h->stream>>>(h->d_avg_partial, (int)nblocks, h->d_avg_out);
    CK(h, cudaGetLastError());
    double sums[AVG_N];
    CK(h, cudaMemcpyAsync(sums, h->d_avg_out, sizeof sums, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    const double vol = sums[21];
    for (int c = 0; c < 21; ++c) out[c] = sums[c] / vol;
    out[21] = vol;
    return CP_OK;
}

int cp_averages_noalloc(cp_handle* h, double out[22]) {
    if (!h || !out) return CP_E_ARG;
    if (h->n_cells == 0) return fail(h, CP_E_STATE, "cp_averages_noalloc: no mesh bound (JxW needed)");
    if (!h->have_post) return fail(h, CP_E_STATE, "cp_averages_noalloc: no cp_update with stiffness_flag 0 yet");
    if (h->n_qp > (int64_t)CP_NOALLOC_AVG_MAX_QPS)
        return fail(h, CP_E_ARG, "cp_averages_noalloc: " + std::to_string(h->n_qp) +
                                     " qps exceed the static scratch limit CP_NOALLOC_AVG_MAX_QPS (" +
                                     std::to_string((int64_t)CP_NOALLOC_AVG_MAX_QPS) + "); use cp_averages");
    if (int rc = check_device(h)) return rc;
    int64_t nblocks = 0;
    for (const auto& g : h->groups) nblocks += blocks_for(g.count, AVG_BLOCK);
    if (nblocks > NOALLOC_AVG_BLOCKS) return fail(h, CP_E_ARG, "cp_averages_noalloc: scratch too small");
    // the array's device address (its host-side name is only a stand-in),
    // looked up on the handle's first call with the handle's device current
    if (!h->noalloc_scratch) {
        void* p = nullptr;
        CK(h, cudaGetSymbolAddress(&p, g_noalloc_avg_scratch));
        h->noalloc_scratch = static_cast<double*>(p);
    }
    double* scratch = h->noalloc_scratch;
    double* partial = scratch;
    double* final_row = scratch + NOALLOC_AVG_BLOCKS * AVG_N;
    // every partial row read below is written earlier in this call, so the
    // scratch needs no clearing between calls
    int64_t off = 0;
    for (const auto& g : h->groups) {
        const unsigned nb = blocks_for(g.count, AVG_BLOCK);
        averages_partial_kernel<<<nb, AVG_BLOCK, 0, h->stream>>>(h->d_lat[g.lattice], g.dev, h->d_keepF, h->d_keepT,
                                                                 h->d_JxW, h->uniform, partial + off * AVG_N);
        off += nb;
    }
    averages_final_kernel<<<1, 32, 0, h->stream>>>(partial, (int)nblocks, final_row);
    CK(h, cudaGetLastError());
    double sums[AVG_N];
    CK(h, cudaMemcpyAsync(sums, final_row, sizeof sums, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    const double vol = sums[21];
    for (int c = 0; c < 21; ++c) out[c] = sums[c] / vol;
    out[21] = vol;
    return CP_OK;
}

int cp_reorient(cp_handle* h) {
    if (!h) return CP_E_ARG;
    if (h->n_qp == 0) return fail(h, CP_E_STATE, "cp_reorient: no qps bound");
    if (int rc = check_device(h)) return rc;
    for (const auto& g : h->groups) reorient_kernel<<<blocks_for(g.count, 128), 128, 0, h->stream>>>(g.dev);
    CK(h, cudaGetLastError());
    return CP_OK;
}

int cp_commit(cp_handle* h) {
    if (!h) return CP_E_ARG;
    if (h->n_qp == 0) return fail(h, CP_E_STATE, "cp_commit: no qps bound");
    if (int rc = check_device(h)) return rc;
    const bool reorder = !h->opts.plain_kernel && !h->opts.reference_order;
    for (const auto& g : h->groups) {
        // the _iter half of the block directly follows the _conv half
        const int64_t half = group_doubles(g.n, g.ns, g.nw, g.count) / 2;
        if (reorder && g.sorted) {
            // _conv in the order of the last sort's keys, gathered from _iter
            // (the sort's permutation buffer holds the source indices), then
            // _iter, the twin flags and the qp map the same
            const std::vector<int> seg = reorder_segments(h, g);
            const int nseg = (int)seg.size() - 1;
            CK(h, cudaMemcpyAsync(g.d_hist, seg.data(), sizeof(int) * seg.size(), cudaMemcpyHostToDevice, h->stream));
            reorder_sort_kernel<<<nseg, 256, 0, h->stream>>>(g.d_key, g.d_hist, g.d_perm);
            const unsigned nb = blocks_for(g.count, 256);
            reorder_gather_kernel<double><<<nb, 256, 0, h->stream>>>(g.d_block + half, g.d_block, half / g.count,
                                                                     g.count, g.d_perm);
            reorder_gather_kernel<int><<<nb, 256, 0, h->stream>>>(g.d_twin + g.count, g.d_twin, 1, g.count,
                                                                  g.d_perm);
            reorder_gather_kernel<int64_t><<<nb, 256, 0, h->stream>>>(g.d_qp, g.d_qp_tmp, 1, g.count, g.d_perm);
            CK(h, cudaGetLastError());
            CK(h, cudaMemcpyAsync(g.d_block + half, g.d_block, sizeof(double) * half, cudaMemcpyDeviceToDevice,
                                  h->stream));
            CK(h, cudaMemcpyAsync(g.d_twin + g.count, g.d_twin, sizeof(int) * g.count, cudaMemcpyDeviceToDevice,
                                  h->stream));
            CK(h, cudaMemcpyAsync(g.d_qp, g.d_qp_tmp, sizeof(int64_t) * g.count, cudaMemcpyDeviceToDevice,
                                  h->stream));
            int* inv = reinterpret_cast<int*>(g.d_qp_tmp);  // new position of each old internal index
            reorder_inverse_kernel<<<nb, 256, 0, h->stream>>>(g.d_perm, g.count, inv);
            reorder_where_kernel<<<nb, 256, 0, h->stream>>>(inv, g.count, g.d_where);
            CK(h, cudaGetLastError());
            g.sorted = false;
            continue;
        }
        CK(h, cudaMemcpyAsync(g.d_block, g.d_block + half, sizeof(double) * half, cudaMemcpyDeviceToDevice,
                              h->stream));
        CK(h, cudaMemcpyAsync(g.d_twin, g.d_twin + g.count, sizeof(int) * g.count, cudaMemcpyDeviceToDevice,
                              h->stream));
    }
    return CP_OK;
}

static bool field_info(const cp_handle* h, const Group& g, int field, double** p, int** ip, int* comps) {
    const bool it = field >= CP_FIELD_ITER_OFFSET;
    const int f = it ? field - CP_FIELD_ITER_OFFSET : field;
    const GroupDev& d = g.dev;
    *ip = nullptr;
    *p = nullptr;
    switch (f) {
        case CP_FIELD_FP_CONV: *p = it ? d.Fp_i : d.Fp_c; *comps = 9; break;
        case CP_FIELD_FE_CONV: *p = it ? d.Fe_i : d.Fe_c; *comps = 9; break;
        case CP_FIELD_S_CONV: *p = it ? d.s_i : d.s_c; *comps = g.n; break;
        case CP_FIELD_W_CONV: *p = it ? d.W_i : d.W_c; *comps = g.n; break;
        case CP_FIELD_ROT_CONV: *p = it ? d.rot_i : d.rot_c; *comps = 3; break;
        case CP_FIELD_ROTNEW_CONV: *p = it ? d.rotnew_i : d.rotnew_c; *comps = 3; break;
        case CP_FIELD_TWINFRAC_CONV: *p = it ? d.tw_i : d.tw_c; *comps = g.nw; break;
        case CP_FIELD_SLIPFRAC_CONV: *p = it ? d.sl_i : d.sl_c; *comps = g.ns; break;
        case CP_FIELD_TWIN_CONV: *ip = it ? d.twin_i : d.twin_c; *comps = 1; break;
        default: return false;
    }
    (void)h;
    return true;
}

int32_t cp_field_width(const cp_handle* h, int32_t field) {
    if (!h) return 0;
    const int f = field >= CP_FIELD_ITER_OFFSET ? field - CP_FIELD_ITER_OFFSET : field;
    switch (f) {
        case CP_FIELD_FP_CONV:
        case CP_FIELD_FE_CONV: return 9;
        case CP_FIELD_S_CONV:
        case CP_FIELD_W_CONV: return h->n_max;
        case CP_FIELD_ROT_CONV:
        case CP_FIELD_ROTNEW_CONV: return 3;
        case CP_FIELD_TWINFRAC_CONV: return h->nw_max;
        case CP_FIELD_SLIPFRAC_CONV: return h->ns_max;
        case CP_FIELD_TWIN_CONV: return 1;
        default: return 0;
    }
}

static int state_io(cp_handle* h, int32_t field, double* hbuf, bool get) {
    if (!h || !hbuf) return CP_E_ARG;
    if (h->n_qp == 0) return fail(h, CP_E_STATE, "no qps bound");
    const int width = cp_field_width(h, field);
    if (width <= 0) return fail(h, CP_E_ARG, "unknown state field");
    if (int rc = check_device(h)) return rc;
    double* d_buf = nullptr;
    CK(h, cudaMalloc(&d_buf, sizeof(double) * width * h->n_qp));
    int rc = CP_OK;
    if (get) {
        CK(h, cudaMemsetAsync(d_buf, 0, sizeof(double) * width * h->n_qp, h->stream));
    } else {
        CK(h, cudaMemcpyAsync(d_buf, hbuf, sizeof(double) * width * h->n_qp, cudaMemcpyHostToDevice, h->stream));
    }
    for (const auto& g : h->groups) {
        double* p;
        int* ip;
        int comps;
        field_info(h, g, field, &p, &ip, &comps);
        if (get)
            gather_field_kernel<<<blocks_for(g.count, 256), 256, 0, h->stream>>>(p, ip, g.count, g.d_qp, comps,
                                                                               width, d_buf);
        else
            scatter_field_kernel<<<blocks_for(g.count, 256), 256, 0, h->stream>>>(p, ip, g.count, g.d_qp, comps,
                                                                                width, d_buf);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_fail(h, e, "state kernel");
    if (get && rc == CP_OK)
        e = cudaMemcpyAsync(hbuf, d_buf, sizeof(double) * width * h->n_qp, cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess && rc == CP_OK) rc = cuda_fail(h, e, "state copy");
    cudaStreamSynchronize(h->stream);
    cudaFree(d_buf);
    return rc;
}

int cp_get_state(cp_handle* h, int32_t field, double* h_buf) { return state_io(h, field, h_buf, true); }
int cp_set_state(cp_handle* h, int32_t field, const double* h_buf) {
    return state_io(h, field, const_cast<double*>(h_buf), false);
}

int cp_measure_fp64_peak(int32_t device, double* tflops) {
    if (!tflops) return CP_E_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return CP_E_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double* d = nullptr;
    if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return CP_E_NOMEM;
    const int threads = 256, blocks = sms * 8, iters = 1 << 15;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fp64_fma_probe_kernel<<<blocks, threads>>>(256, 1.0, d);  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        fp64_fma_probe_kernel<<<blocks, threads>>>(iters, 1.0 + rep, d);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    const cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (e != cudaSuccess) return CP_E_CUDA;
    const double flops = 2.0 * 8.0 * (double)iters * threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return CP_OK;
}

int cp_set_timing(cp_handle* h, int32_t enable) {
    if (!h) return CP_E_ARG;
    if (int rc = check_device(h)) return rc;
    CK(h, cudaStreamSynchronize(h->stream));
    for (auto& p : h->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    h->pending.clear();
    h->timing = enable != 0;
    h->group_ms.assign(h->groups.size(), 0.0);
    h->group_launches.assign(h->groups.size(), 0);
    h->contract_ms[0] = h->contract_ms[1] = 0.0;
    h->contract_launches[0] = h->contract_launches[1] = 0;
    return CP_OK;
}

int cp_get_timing(cp_handle* h, int32_t max_groups, int32_t* lattice, int64_t* count, int64_t* launches,
                  double* total_ms) {
    if (!h) return CP_E_ARG;
    if (int rc = check_device(h)) return rc;
    CK(h, cudaStreamSynchronize(h->stream));
    if (h->group_ms.size() != h->groups.size()) {
        h->group_ms.assign(h->groups.size(), 0.0);
        h->group_launches.assign(h->groups.size(), 0);
    }
    for (auto& p : h->pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p.a, p.b);
        if (p.group < 0) {  // -1: FP64 contraction, -2: tensor-core contraction
            h->contract_ms[-p.group - 1] += ms;
            h->contract_launches[-p.group - 1] += 1;
        } else {
            h->group_ms[p.group] += ms;
            h->group_launches[p.group] += 1;
        }
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    h->pending.clear();
    const int ng = (int)h->groups.size();
    for (int g = 0; g < ng && g < max_groups; ++g) {
        if (lattice) lattice[g] = h->groups[g].lattice;
        if (count) count[g] = h->groups[g].count;
        if (launches) launches[g] = h->group_launches[g];
        if (total_ms) total_ms[g] = h->group_ms[g];
    }
    return ng;
}

int cp_get_contract_timing(cp_handle* h, int32_t kind, int64_t* launches, double* total_ms) {
    if (!h || kind < 0 || kind > 1) return CP_E_ARG;
    int64_t dummy[CP_MAX_LATTICES];
    const int ng = cp_get_timing(h, 0, nullptr, dummy, nullptr, nullptr);  // folds the pending events in
    if (ng < 0) return ng;
    if (launches) *launches = h->contract_launches[kind];
    if (total_ms) *total_ms = h->contract_ms[kind];
    return CP_OK;
}

int cp_synchronize(cp_handle* h) {
    if (!h) return CP_E_ARG;
    if (int rc = check_device(h)) return rc;
    CK(h, cudaStreamSynchronize(h->stream));
    return check_tc_error(h);
}

// ---- the Newton step's global system ------------------------------------

int cp_bind_dofs(cp_handle* h, int64_t n_dofs, const int64_t* h_cell_dofs, int64_t n_constrained,
                 const int64_t* h_constrained) {
    if (!h) return CP_E_ARG;
    if (h->n_cells == 0) return fail(h, CP_E_STATE, "cp_bind_dofs: no mesh bound");
    if (n_dofs < 1 || n_dofs > INT32_MAX || !h_cell_dofs || n_constrained < 0 || (n_constrained && !h_constrained))
        return fail(h, CP_E_ARG, "cp_bind_dofs: bad arguments");
    if (int rc = check_device(h)) return rc;
    const int64_t nc = h->n_cells;
    for (int64_t t = 0; t < 24 * nc; ++t)
        if (h_cell_dofs[t] < 0 || h_cell_dofs[t] >= n_dofs)
            return fail(h, CP_E_ARG, "cp_bind_dofs: dof index out of range");
    for (int64_t c = 0; c < nc; ++c)
        for (int a = 0; a < 24; ++a)
            for (int b = a + 1; b < 24; ++b)
                if (h_cell_dofs[24 * c + a] == h_cell_dofs[24 * c + b])
                    return fail(h, CP_E_ARG, "cp_bind_dofs: repeated dof within a cell");
    std::vector<unsigned char> cmask(n_dofs, 0);
    for (int64_t j = 0; j < n_constrained; ++j) {
        if (h_constrained[j] < 0 || h_constrained[j] >= n_dofs)
            return fail(h, CP_E_ARG, "cp_bind_dofs: constrained dof out of range");
        if (cmask[h_constrained[j]]) return fail(h, CP_E_ARG, "cp_bind_dofs: constrained dof listed twice");
        cmask[h_constrained[j]] = 1;
    }
    // CSR pattern: row i holds the dofs of every cell that holds i
    std::vector<int64_t> row_ptr(n_dofs + 1, 0);
    for (int64_t t = 0; t < 24 * nc; ++t) row_ptr[h_cell_dofs[t] + 1] += 24;
    for (int64_t i = 0; i < n_dofs; ++i) row_ptr[i + 1] += row_ptr[i];
    std::vector<int> cand(row_ptr[n_dofs]);
    {
        std::vector<int64_t> fill(row_ptr.begin(), row_ptr.end() - 1);
        for (int64_t c = 0; c < nc; ++c)
            for (int a = 0; a < 24; ++a) {
                const int64_t i = h_cell_dofs[24 * c + a];
                for (int b = 0; b < 24; ++b) cand[fill[i]++] = (int)h_cell_dofs[24 * c + b];
            }
    }
    std::vector<int64_t> rp(n_dofs + 1, 0);
    std::vector<int> col;
    col.reserve(cand.size() / 2);
    for (int64_t i = 0; i < n_dofs; ++i) {
        auto b = cand.begin() + row_ptr[i], e = cand.begin() + row_ptr[i + 1];
        std::sort(b, e);
        e = std::unique(b, e);
        col.insert(col.end(), b, e);
        rp[i + 1] = (int64_t)col.size();
    }
    const int64_t nnz = (int64_t)col.size();
    // the three dofs of a node (3t, 3t+1, 3t+2) with one column pattern
    bool triples = n_dofs % 3 == 0;
    for (int64_t t = 0; triples && t < n_dofs / 3; ++t) {
        const int64_t a = rp[3 * t], len = rp[3 * t + 1] - a;
        triples = rp[3 * t + 2] - rp[3 * t + 1] == len && rp[3 * t + 3] - rp[3 * t + 2] == len;
        for (int64_t j = 0; triples && j < len; ++j)
            triples = col[a + j] == col[a + len + j] && col[a + j] == col[a + 2 * len + j];
    }
    auto find = [&](int64_t i, int j) -> int64_t {
        const auto b = col.begin() + rp[i], e = col.begin() + rp[i + 1];
        return (int64_t)(std::lower_bound(b, e, j) - col.begin());
    };
    std::vector<int64_t> tpos(nnz), diag(n_dofs);
    for (int64_t i = 0; i < n_dofs; ++i) {
        diag[i] = rp[i + 1] > rp[i] ? find(i, (int)i) : -1;
        for (int64_t p = rp[i]; p < rp[i + 1]; ++p) tpos[p] = find(col[p], (int)i);
    }
    for (int64_t i = 0; i < n_dofs; ++i)
        if (diag[i] < 0) return fail(h, CP_E_ARG, "cp_bind_dofs: a dof belongs to no cell");
    // node blocks: the three components of a node, local dofs 3a..3a+2 of a
    // cell; usable when every dof sits in exactly one such triple
    std::vector<int64_t> blk, blkpos;
    {
        std::vector<int64_t> owner(n_dofs, -1);
        bool ok = true;
        for (int64_t c = 0; c < nc && ok; ++c)
            for (int a = 0; a < 8 && ok; ++a) {
                const int64_t* g = h_cell_dofs + 24 * c + 3 * a;
                const int64_t b = owner[g[0]];
                if (b < 0) {
                    const int64_t nb = (int64_t)blk.size() / 3;
                    for (int k = 0; k < 3; ++k) {
                        if (owner[g[k]] >= 0) ok = false;
                        owner[g[k]] = nb;
                        blk.push_back(g[k]);
                    }
                } else {
                    for (int k = 0; k < 3; ++k) ok = ok && blk[3 * b + k] == g[k];
                }
            }
        if (ok)
            for (int64_t b = 0; b < (int64_t)blk.size() / 3; ++b)
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q) blkpos.push_back(find(blk[3 * b + r], (int)blk[3 * b + q]));
        else
            blk.clear();
    }
    const int64_t n_blocks = (int64_t)blk.size() / 3;
    // contributions of element entries (cell order within each entry)
    std::vector<int64_t> kptr(nnz + 1, 0), kidx(576 * nc), epos(576 * nc);
    for (int64_t c = 0; c < nc; ++c)
        for (int a = 0; a < 24; ++a)
            for (int b = 0; b < 24; ++b) {
                const int64_t p = find(h_cell_dofs[24 * c + a], (int)h_cell_dofs[24 * c + b]);
                epos[576 * c + 24 * a + b] = p;
                kptr[p + 1] += 1;
            }
    for (int64_t p = 0; p < nnz; ++p) kptr[p + 1] += kptr[p];
    {
        std::vector<int64_t> fill(kptr.begin(), kptr.end() - 1);
        for (int64_t e = 0; e < 576 * nc; ++e) kidx[fill[epos[e]]++] = e;
    }
    std::vector<int64_t> rptr(n_dofs + 1, 0), ridx(24 * nc);
    for (int64_t t = 0; t < 24 * nc; ++t) rptr[h_cell_dofs[t] + 1] += 1;
    for (int64_t i = 0; i < n_dofs; ++i) rptr[i + 1] += rptr[i];
    {
        std::vector<int64_t> fill(rptr.begin(), rptr.end() - 1);
        for (int64_t t = 0; t < 24 * nc; ++t) ridx[fill[h_cell_dofs[t]]++] = t;
    }
    free_system(h);
    auto& y = h->sys;
    y.n_dofs = n_dofs;
    y.nnz = nnz;
    y.n_con = n_constrained;
    y.n_blocks = n_blocks;
    y.triples = triples;
    if (n_blocks &&
        (cudaMalloc(&y.d_blk, sizeof(int64_t) * 3 * n_blocks) != cudaSuccess ||
         cudaMalloc(&y.d_blkpos, sizeof(int64_t) * 9 * n_blocks) != cudaSuccess ||
         cudaMalloc(&y.d_binv, sizeof(double) * 9 * n_blocks) != cudaSuccess)) {
        free_system(h);
        return fail(h, CP_E_NOMEM, "cp_bind_dofs: device allocation failed");
    }
    if (n_blocks) {
        CK(h, cudaMemcpy(y.d_blk, blk.data(), sizeof(int64_t) * 3 * n_blocks, cudaMemcpyHostToDevice));
        CK(h, cudaMemcpy(y.d_blkpos, blkpos.data(), sizeof(int64_t) * 9 * n_blocks, cudaMemcpyHostToDevice));
    }
    bool ok = cudaMalloc(&y.d_cell_dofs, sizeof(int64_t) * 24 * nc) == cudaSuccess &&
              cudaMalloc(&y.d_row_ptr, sizeof(int64_t) * (n_dofs + 1)) == cudaSuccess &&
              cudaMalloc(&y.d_col, sizeof(int) * nnz) == cudaSuccess &&
              cudaMalloc(&y.d_tpos, sizeof(int64_t) * nnz) == cudaSuccess &&
              cudaMalloc(&y.d_diag, sizeof(int64_t) * n_dofs) == cudaSuccess &&
              cudaMalloc(&y.d_kptr, sizeof(int64_t) * (nnz + 1)) == cudaSuccess &&
              cudaMalloc(&y.d_kidx, sizeof(int64_t) * 576 * nc) == cudaSuccess &&
              cudaMalloc(&y.d_rptr, sizeof(int64_t) * (n_dofs + 1)) == cudaSuccess &&
              cudaMalloc(&y.d_ridx, sizeof(int64_t) * 24 * nc) == cudaSuccess &&
              cudaMalloc(&y.d_con, sizeof(int64_t) * std::max<int64_t>(n_constrained, 1)) == cudaSuccess &&
              cudaMalloc(&y.d_cmask, n_dofs) == cudaSuccess &&
              cudaMalloc(&y.d_vals, sizeof(double) * nnz) == cudaSuccess &&
              cudaMalloc(&y.d_valsT, sizeof(double) * nnz) == cudaSuccess &&
              cudaMalloc(&y.d_Ke, sizeof(double) * 576 * nc) == cudaSuccess &&
              cudaMalloc(&y.d_Re, sizeof(double) * 24 * nc) == cudaSuccess &&
              cudaMalloc(&y.d_Ul, sizeof(double) * 24 * nc) == cudaSuccess &&
              cudaMalloc(&y.d_duc, sizeof(double) * std::max<int64_t>(n_constrained, 1)) == cudaSuccess &&
              cudaMalloc(&y.d_vec, sizeof(double) * SYS_VECS * n_dofs) == cudaSuccess &&
              cudaMalloc(&y.d_sc, sizeof(double) * SC_COUNT) == cudaSuccess &&
              cudaMalloc(&y.d_partial, sizeof(double) * RED_BLOCKS) == cudaSuccess &&
              cudaMalloc(&y.d_fpartial, sizeof(double) * (n_dofs / 8 + 64)) == cudaSuccess &&
              cudaMalloc(&y.d_ticket, sizeof(unsigned int) * 8) == cudaSuccess &&
              cudaMalloc(&y.d_done, sizeof(int)) == cudaSuccess && cudaMalloc(&y.d_info, sizeof(int) * 3) == cudaSuccess;
    if (!ok) {
        free_system(h);
        return fail(h, CP_E_NOMEM, "cp_bind_dofs: device allocation failed");
    }
    CK(h, cudaMemcpy(y.d_cell_dofs, h_cell_dofs, sizeof(int64_t) * 24 * nc, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(y.d_row_ptr, rp.data(), sizeof(int64_t) * (n_dofs + 1), cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(y.d_col, col.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(y.d_tpos, tpos.data(), sizeof(int64_t) * nnz, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(y.d_diag, diag.data(), sizeof(int64_t) * n_dofs, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(y.d_kptr, kptr.data(), sizeof(int64_t) * (nnz + 1), cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(y.d_kidx, kidx.data(), sizeof(int64_t) * 576 * nc, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(y.d_rptr, rptr.data(), sizeof(int64_t) * (n_dofs + 1), cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(y.d_ridx, ridx.data(), sizeof(int64_t) * 24 * nc, cudaMemcpyHostToDevice));
    if (n_constrained)
        CK(h, cudaMemcpy(y.d_con, h_constrained, sizeof(int64_t) * n_constrained, cudaMemcpyHostToDevice));
    CK(h, cudaMemcpy(y.d_cmask, cmask.data(), n_dofs, cudaMemcpyHostToDevice));
    CK(h, cudaMemset(y.d_vec, 0, sizeof(double) * SYS_VECS * n_dofs));
    CK(h, cudaMemset(y.d_ticket, 0, sizeof(unsigned int) * 8));
    return CP_OK;
}

int cp_set_displacement(cp_handle* h, const double* h_u) {
    if (!h || !h_u) return CP_E_ARG;
    if (!h->sys.n_dofs) return fail(h, CP_E_STATE, "cp_set_displacement: no dofs bound");
    if (int rc = check_device(h)) return rc;
    CK(h, cudaMemcpyAsync(h->sys.d_vec + V_U * h->sys.n_dofs, h_u, sizeof(double) * h->sys.n_dofs,
                          cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return CP_OK;
}

int cp_get_displacement(cp_handle* h, double* h_u) {
    if (!h || !h_u) return CP_E_ARG;
    if (!h->sys.n_dofs) return fail(h, CP_E_STATE, "cp_get_displacement: no dofs bound");
    if (int rc = check_device(h)) return rc;
    CK(h, cudaMemcpyAsync(h_u, h->sys.d_vec + V_U * h->sys.n_dofs, sizeof(double) * h->sys.n_dofs,
                          cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return CP_OK;
}

namespace {

// a = sum_i x_i y_i into sc[slot] (deterministic two-stage)
void sys_dot(cp_handle* h, const double* x, const double* y, int slot, const int* done) {
    auto& s = h->sys;
    dot_partial_kernel<<<RED_BLOCKS, SOLVE_BLOCK, 0, h->stream>>>(x, y, s.n_dofs, s.d_partial, done);
    dot_final_kernel<<<1, SOLVE_BLOCK, 0, h->stream>>>(s.d_partial, s.d_sc + slot, done);
}

void sys_spmv(cp_handle* h, const double* x, double* y, const int* done) {
    auto& s = h->sys;
    const int64_t threads = 32 * s.n_dofs;
    spmv_kernel<<<blocks_for(threads, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_row_ptr, s.d_col, s.d_vals, x,
                                                                              s.n_dofs, y, done);
}

// one Krylov iteration of the chosen method (queued, no host sync)
void krylov_iteration(cp_handle* h, const cp_solver_t& sv, bool first) {
    auto& s = h->sys;
    const int64_t n = s.n_dofs;
    const unsigned nb = blocks_for(n, SOLVE_BLOCK);
    double* V = s.d_vec;
    auto v = [&](int k) { return V + (int64_t)k * n; };
    const int* done = s.d_done;
    if (sv.kind == CP_SOLVER_BICGSTAB) {
        sys_dot(h, v(V_RT), v(V_RES), SC_RHO, done);
        bicgstab_dir_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_sc, v(V_RES), v(V_Q), n, first, v(V_P),
                                                                 s.d_done, s.d_info);
        scale_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(V_P), v(V_DINV), n, v(V_PH), done);
        sys_spmv(h, v(V_PH), v(V_Q), done);  // v
        sys_dot(h, v(V_RT), v(V_Q), SC_DEN, done);
        bicgstab_s_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_sc, v(V_RES), v(V_Q), n, v(V_S), s.d_done,
                                                               s.d_info);
        scale_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(V_S), v(V_DINV), n, v(V_SH), done);
        sys_spmv(h, v(V_SH), v(V_T), done);
        sys_dot(h, v(V_T), v(V_S), SC_TS, done);
        sys_dot(h, v(V_T), v(V_T), SC_TT, done);
        bicgstab_x_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_sc, v(V_PH), v(V_SH), v(V_S), v(V_T), n, v(V_X),
                                                               v(V_RES), done);
    } else {
        // BiCG in four kernels; the last one also tests convergence
        if (sv.precond == CP_PRECOND_NODE_BLOCK)
            fbicg_precond_block_kernel<<<blocks_for(s.n_blocks, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(
                s.d_binv, s.d_blk, v(V_RES), v(V_RT), s.n_blocks, v(V_Z), v(V_ZT), s.d_sc, s.d_fpartial,
                s.d_ticket + 0, done);
        else
            fbicg_precond_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(V_DINV), v(V_RES), v(V_RT), n, v(V_Z),
                                                                      v(V_ZT), s.d_sc, s.d_fpartial, s.d_ticket + 0,
                                                                      done);
        fbicg_dir_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_sc, v(V_Z), v(V_ZT), n, first, v(V_P), v(V_PT),
                                                              s.d_done, s.d_info);
        if (s.triples)  // a warp per node, grid of SPMV3_GRID blocks at most (<= n / 8 partials)
            fbicg_spmv3_kernel<<<(int)std::min<int64_t>(blocks_for(32 * (n / 3), SOLVE_BLOCK), SPMV3_GRID),
                                 SOLVE_BLOCK, 0, h->stream>>>(s.d_row_ptr, s.d_col, s.d_vals, s.d_valsT, v(V_P),
                                                              v(V_PT), n, v(V_Q), v(V_QT), s.d_sc, s.d_fpartial,
                                                              s.d_ticket + 1, done);
        else
            fbicg_spmv_kernel<<<blocks_for(32 * n, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(
                s.d_row_ptr, s.d_col, s.d_vals, s.d_valsT, v(V_P), v(V_PT), n, v(V_Q), v(V_QT), s.d_sc,
                s.d_fpartial, s.d_ticket + 1, done);
        fbicg_step_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_sc, v(V_P), v(V_Q), v(V_QT), v(V_DINV), n,
                                                               sv.rel_tolerance, sv.precond_norm, v(V_X), v(V_RES),
                                                               v(V_RT), s.d_fpartial, s.d_ticket + 2, s.d_done,
                                                               s.d_info);
        return;
    }
    sys_dot(h, v(V_RES), v(V_RES), SC_RR, done);
    if (sv.precond_norm) {
        scale_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(V_RES), v(V_DINV), n, v(V_Z), done);
        sys_dot(h, v(V_Z), v(V_Z), SC_ZZ, done);
    }
    check_kernel<<<1, 1, 0, h->stream>>>(s.d_sc, sv.rel_tolerance, sv.precond_norm, s.d_done, s.d_info);
    shift_rho_kernel<<<1, 1, 0, h->stream>>>(s.d_sc, done);
}

// Capture 'every' Krylov iterations as two graphs (the first block, whose
// first iteration starts the recurrences, and later blocks).  Returns false
// (plain launches are used) if capture is not possible.
bool ensure_solve_graphs(cp_handle* h, const cp_solver_t& sv, int every) {
    auto& s = h->sys;
    if (s.g_first && s.g_next && s.g_kind == sv.kind && s.g_precond == sv.precond_norm && s.g_every == every &&
        s.g_tol == sv.rel_tolerance && s.g_pc == sv.precond)
        return true;
    if (s.g_first) cudaGraphExecDestroy(s.g_first);
    if (s.g_next) cudaGraphExecDestroy(s.g_next);
    s.g_first = s.g_next = nullptr;
    for (int f = 1; f >= 0; --f) {
        if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
        for (int t = 0; t < every; ++t) krylov_iteration(h, sv, f == 1 && t == 0);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        cudaGraphExec_t ex = nullptr;
        const bool ok = e == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        if (!ok) {
            cudaGetLastError();
            return false;
        }
        (f ? s.g_first : s.g_next) = ex;
    }
    s.g_kind = sv.kind;
    s.g_precond = sv.precond_norm;
    s.g_every = every;
    s.g_tol = sv.rel_tolerance;
    s.g_pc = sv.precond;
    return true;
}

}  // namespace

namespace {

// SpMV units (nodes or rows) per block of the persistent solve's grid: one per
// warp keeps the dependent column / vector loads of the SpMV short
#ifndef CP_PBICG_UNITS_PER_BLOCK
#define CP_PBICG_UNITS_PER_BLOCK 8
#endif

// Krylov solve of the condensed system K x = rhs (FP64 values in s.d_vals,
// K^T's in s.d_valsT, the Jacobi diagonal in V_DINV) from x = 0 into V_X:
// one cooperative launch for small Jacobi BiCG systems, else four kernels
// per iteration replayed as graphs; hinfo = {iterations, converged,
// breakdown}, *bnorm_out = ||rhs||
int krylov_solve(cp_handle* h, const cp_solver_t& sv, const double* rhs, int hinfo[3], double* bnorm_out) {
    auto& s = h->sys;
    const int64_t n = s.n_dofs;
    double* V = s.d_vec;
    auto v = [&](int k) { return V + (int64_t)k * n; };
    const unsigned nb = blocks_for(n, SOLVE_BLOCK);
    // Krylov solve from x = 0: r = r~ = rhs
    CK(h, cudaMemsetAsync(v(V_X), 0, sizeof(double) * n, h->stream));
    copy_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(rhs, n, v(V_RES));
    copy_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(rhs, n, v(V_RT));
    CK(h, cudaMemsetAsync(s.d_done, 0, sizeof(int), h->stream));
    CK(h, cudaMemsetAsync(s.d_info, 0, sizeof(int) * 3, h->stream));
    CK(h, cudaMemsetAsync(s.d_sc, 0, sizeof(double) * SC_COUNT, h->stream));
    CK(h, cudaMemsetAsync(s.d_ticket, 0, sizeof(unsigned int) * 8, h->stream));
    sys_dot(h, rhs, rhs, SC_BB, nullptr);
    sys_dot(h, rhs, rhs, SC_RR, nullptr);
    if (sv.precond_norm) {
        scale_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(rhs, v(V_DINV), n, v(V_Z), nullptr);
        sys_dot(h, v(V_Z), v(V_Z), SC_ZZ, nullptr);
    }
    double sc0[SC_COUNT];
    CK(h, cudaMemcpyAsync(sc0, s.d_sc, sizeof sc0, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    hinfo[0] = hinfo[1] = hinfo[2] = 0;
    const double bnorm = std::sqrt(sc0[SC_BB]);
    *bnorm_out = bnorm;
    // one cooperative launch for the whole Jacobi BiCG solve (small systems,
    // or on request) where the device can run one
    bool persistent = sv.kind == CP_SOLVER_BICG && sv.precond == CP_PRECOND_JACOBI && sv.kernel_mode != 1 &&
                      (sv.kernel_mode == 2 || n <= CP_PERSISTENT_MAX_DOFS);
    int p_grid = 0;
    if (persistent && bnorm != 0.0) {
        int dev = 0, nsm = 0, coop = 0, per_sm = 0;
        CK(h, cudaGetDevice(&dev));
        CK(h, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CK(h, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        CK(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pbicg_kernel, SOLVE_BLOCK, 0));
        // nodes or rows, CP_PBICG_UNITS_PER_BLOCK per block, at most one block
        // per SM: the solves of other handles (concurrent requests) keep room
        // to run beside it
        const int64_t units = s.triples ? n / 3 : n;
        p_grid = (int)std::max<int64_t>(
            1, std::min<int64_t>(std::min<int64_t>((int64_t)nsm * per_sm, nsm),
                                 (units + CP_PBICG_UNITS_PER_BLOCK - 1) / CP_PBICG_UNITS_PER_BLOCK));
        persistent = coop && per_sm > 0 && 3 * (int64_t)p_grid <= n / 8 + 64;  // partials fit the scratch
    }
    if (bnorm == 0.0) {
        hinfo[1] = 1;  // du = 0 solves it
    } else if (persistent) {
        PbicgArgs pa{s.d_row_ptr, s.d_col, s.d_vals, s.d_valsT, v(V_DINV), n, s.triples ? 1 : 0,
                     sv.precond_norm, sv.max_iterations, sv.rel_tolerance, bnorm, v(V_X), v(V_RES), v(V_RT),
                     v(V_Z), v(V_ZT), v(V_P), v(V_PT), v(V_Q), v(V_QT), v(V_S), v(V_T), s.d_fpartial,
                     s.d_ticket + 4, s.d_info,
                     reinterpret_cast<int*>(s.d_ticket + 6), s.d_sc,
                     h->barrier_wait_ns ? h->barrier_wait_ns : PBICG_WAIT_NS, h->barrier_withhold};
        void* kargs[] = {&pa};
        CK(h, cudaLaunchCooperativeKernel((const void*)pbicg_kernel, dim3(p_grid), dim3(SOLVE_BLOCK), kargs, 0,
                                          h->stream));
        unsigned tk[8];
        CK(h, cudaMemcpyAsync(hinfo, s.d_info, sizeof(int) * 3, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaMemcpyAsync(tk, s.d_ticket, sizeof tk, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        if (tk[6]) return fail(h, CP_E_CUDA, "cp_newton_iteration: a grid barrier of the solve timed out");
    } else {
        const int every = sv.check_every > 0 ? sv.check_every : 8;
        const bool graphs = ensure_solve_graphs(h, sv, every);
        int queued = 0;
        while (queued < sv.max_iterations) {
            const int k = std::min(every, sv.max_iterations - queued);
            if (graphs && k == every)
                CK(h, cudaGraphLaunch(queued == 0 ? s.g_first : s.g_next, h->stream));
            else
                for (int t = 0; t < k; ++t) krylov_iteration(h, sv, queued + t == 0);
            queued += k;
            CK(h, cudaGetLastError());
            CK(h, cudaMemcpyAsync(hinfo, s.d_info, sizeof(int) * 3, cudaMemcpyDeviceToHost, h->stream));
            CK(h, cudaStreamSynchronize(h->stream));
            if (hinfo[1] || hinfo[2]) break;
        }
    }
    return CP_OK;
}

// FP32 vectors of the mixed-precision inner solve
enum MixVec { MV_R = 0, MV_RT, MV_Z, MV_ZT, MV_P, MV_PT, MV_Q, MV_QT, MV_D, MV_DINV, MV_COUNT };
constexpr double MIXED_INNER_TOL = 1e-5;  // default relative residual of an inner FP32 solve
constexpr int MIXED_INNER_CAP = 2000;      // iterations of one FP32 pass at most

// One Newton iteration with the mixed-precision assembly and solve
// (cp_solver_t.precision = CP_PRECISION_MIXED).
int mixed_newton_iteration(cp_handle* h, const cp_solver_t& sv, const double* h_duc, double F_e, double F_r,
                           cp_solve_info_t* info) {
    auto& s = h->sys;
    const int64_t n = s.n_dofs, nc = h->n_cells;
    if (!s.d_vals32) {
        if (cudaMalloc(&s.d_vals32, sizeof(float) * s.nnz) != cudaSuccess ||
            cudaMalloc(&s.d_valsT32, sizeof(float) * s.nnz) != cudaSuccess ||
            cudaMalloc(&s.d_vec32, sizeof(float) * MV_COUNT * n) != cudaSuccess) {
            cudaFree(s.d_vals32);
            cudaFree(s.d_valsT32);
            cudaFree(s.d_vec32);
            s.d_vals32 = s.d_valsT32 = s.d_vec32 = nullptr;
            return fail(h, CP_E_NOMEM, "cp_newton_iteration: mixed-precision buffers");
        }
        // the FP32 vectors start as zeros, like the FP64 ones of cp_bind_dofs
        CK(h, cudaMemsetAsync(s.d_vec32, 0, sizeof(float) * MV_COUNT * n, h->stream));
    }
    double* V = s.d_vec;
    auto v = [&](int k) { return V + (int64_t)k * n; };
    auto w = [&](int k) { return s.d_vec32 + (int64_t)k * n; };
    const unsigned nb = blocks_for(n, SOLVE_BLOCK);
    float* Ke32 = reinterpret_cast<float*>(s.d_Ke);
    gather_ulocal_kernel<<<blocks_for(24 * nc, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(v(V_U), s.d_cell_dofs,
                                                                                         24 * nc, s.d_Ul);
    if (int rc = cp_assemble_mixed_device(h, s.d_Ul, F_e, F_r, Ke32, s.d_Re, h->d_status)) return rc;
    scatter_sum_f32_kernel<<<blocks_for(s.nnz, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(Ke32, s.d_kptr, s.d_kidx,
                                                                                         s.nnz, s.d_vals32);
    scatter_sum_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_Re, s.d_rptr, s.d_ridx, n, v(V_R));
    if (s.n_con && h_duc)
        CK(h, cudaMemcpyAsync(s.d_duc, h_duc, sizeof(double) * s.n_con, cudaMemcpyHostToDevice, h->stream));
    const double* duc = (s.n_con && h_duc) ? s.d_duc : nullptr;
    CK(h, cudaMemsetAsync(v(V_DC), 0, sizeof(double) * n, h->stream));
    if (s.n_con)
        constrained_vector_kernel<<<blocks_for(s.n_con, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_con, duc,
                                                                                                  s.n_con, v(V_DC));
    spmv_f32_kernel<<<blocks_for(32 * n, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_row_ptr, s.d_col, s.d_vals32,
                                                                                   v(V_DC), n, nullptr, v(V_KDC));
    condense_rhs_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(V_R), v(V_KDC), v(V_DC), s.d_cmask, n, v(V_RHS));
    condense_matrix_f32_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_row_ptr, s.d_col, s.d_cmask, n, s.d_vals32);
    jacobi_setup_f32_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_vals32, s.d_diag, n, w(MV_DINV));
    transpose_values_f32_kernel<<<blocks_for(s.nnz, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_vals32, s.d_tpos,
                                                                                              s.nnz, s.d_valsT32);
    // refinement vectors: b in V_RHS; x and r = b - K x in V_PH / V_SH; a
    // pass's candidate x + d and its residual in V_KDC / V_DC (the roles of
    // the two pairs swap when a candidate is accepted)
    int ix = V_PH, ir = V_SH, ixt = V_KDC, irt = V_DC;
    CK(h, cudaMemsetAsync(v(ix), 0, sizeof(double) * n, h->stream));
    copy_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(V_RHS), n, v(ir));
    CK(h, cudaMemsetAsync(s.d_ticket, 0, sizeof(unsigned int) * 8, h->stream));
    CK(h, cudaMemsetAsync(s.d_sc, 0, sizeof(double) * SC_COUNT, h->stream));
    sys_dot(h, v(V_RHS), v(V_RHS), SC_BB, nullptr);
    double sc0[SC_COUNT];
    CK(h, cudaMemcpyAsync(sc0, s.d_sc, sizeof sc0, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    CK(h, cudaGetLastError());
    const double bnorm = std::sqrt(sc0[SC_BB]);
    double rnorm = bnorm;
    int total_iters = 0, iters64 = 0, passes = 0, breakdown = 0;
    bool use64 = false, have64 = false;
    const int max_passes = sv.max_refinements > 0 ? sv.max_refinements : 10;
    const int every = sv.check_every > 0 ? sv.check_every : 8;
    const double tol_in = sv.inner_tolerance > 0.0 ? sv.inner_tolerance : MIXED_INNER_TOL;
    const int cap32 = std::min(sv.max_iterations, MIXED_INNER_CAP);
    cp_solver_t sv64 = sv;
    sv64.precision = CP_PRECISION_FP64;
    while (bnorm != 0.0 && !(rnorm <= sv.rel_tolerance * bnorm) && passes < max_passes) {
        ++passes;
        int hinfo[3] = {0, 0, 0};
        if (!use64) {
            // the inner FP32 solve K d = r from d = 0
            mixed_start_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(ir), n, w(MV_R), w(MV_RT), w(MV_D));
            CK(h, cudaMemsetAsync(s.d_done, 0, sizeof(int), h->stream));
            CK(h, cudaMemsetAsync(s.d_info, 0, sizeof(int) * 3, h->stream));
            CK(h, cudaMemsetAsync(s.d_sc, 0, sizeof(double) * SC_COUNT, h->stream));
            CK(h, cudaMemsetAsync(s.d_ticket, 0, sizeof(unsigned int) * 8, h->stream));
            // (RED_BLOCKS partials: the RED_BLOCKS-sized buffer, not the fused
            // iteration's n / 8 + 64, which smaller systems would overrun)
            norm2_f32_kernel<<<RED_BLOCKS, SOLVE_BLOCK, 0, h->stream>>>(w(MV_R), n, s.d_sc, SC_BB, s.d_partial,
                                                                        s.d_ticket + 3);
            int queued = 0;
            const int* done = s.d_done;
            while (queued < cap32) {
                const int k = std::min(every, cap32 - queued);
                for (int t = 0; t < k; ++t) {
                    mbicg_precond_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(w(MV_DINV), w(MV_R), w(MV_RT), n,
                                                                            w(MV_Z), w(MV_ZT), s.d_sc, s.d_fpartial,
                                                                            s.d_ticket + 0, done);
                    mbicg_dir_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_sc, w(MV_Z), w(MV_ZT), n,
                                                                        queued + t == 0, w(MV_P), w(MV_PT), s.d_done,
                                                                        s.d_info);
                    if (s.triples)
                        mbicg_spmv3_kernel<<<(int)std::min<int64_t>(blocks_for(32 * (n / 3), SOLVE_BLOCK),
                                                                    SPMV3_GRID),
                                             SOLVE_BLOCK, 0, h->stream>>>(s.d_row_ptr, s.d_col, s.d_vals32,
                                                                          s.d_valsT32, w(MV_P), w(MV_PT), n, w(MV_Q),
                                                                          w(MV_QT), s.d_sc, s.d_fpartial,
                                                                          s.d_ticket + 1, done);
                    else
                        mbicg_spmv_kernel<<<blocks_for(32 * n, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(
                            s.d_row_ptr, s.d_col, s.d_vals32, s.d_valsT32, w(MV_P), w(MV_PT), n, w(MV_Q), w(MV_QT),
                            s.d_sc, s.d_fpartial, s.d_ticket + 1, done);
                    mbicg_step_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_sc, w(MV_P), w(MV_Q), w(MV_QT), n,
                                                                         tol_in, w(MV_D), w(MV_R), w(MV_RT),
                                                                         s.d_fpartial, s.d_ticket + 2, s.d_done,
                                                                         s.d_info);
                }
                queued += k;
                CK(h, cudaGetLastError());
                CK(h, cudaMemcpyAsync(hinfo, s.d_info, sizeof(int) * 3, cudaMemcpyDeviceToHost, h->stream));
                CK(h, cudaStreamSynchronize(h->stream));
                if (hinfo[1] || hinfo[2]) break;
            }
            total_iters += hinfo[0];
            if (hinfo[2]) breakdown = 1;
            mixed_try_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(ix), w(MV_D), nullptr, n, v(ixt));
        } else {
            // an FP64 inner solve on the same (FP32-assembled) matrix
            if (!have64) {
                promote_f32_kernel<<<blocks_for(s.nnz, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_vals32, s.nnz,
                                                                                                s.d_vals);
                promote_f32_kernel<<<blocks_for(s.nnz, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_valsT32, s.nnz,
                                                                                                s.d_valsT);
                jacobi_setup_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_vals, s.d_diag, n, v(V_DINV));
                have64 = true;
            }
            double bn = 0.0;
            if (int rc = krylov_solve(h, sv64, v(ir), hinfo, &bn)) return rc;
            total_iters += hinfo[0];
            iters64 += hinfo[0];
            if (hinfo[2]) breakdown = 1;
            mixed_try_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(ix), nullptr, v(V_X), n, v(ixt));
        }
        // the candidate's residual b - K (x + d) in FP64
        spmv_f32_kernel<<<blocks_for(32 * n, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(
            s.d_row_ptr, s.d_col, s.d_vals32, v(ixt), n, v(V_RHS), v(irt));
        sys_dot(h, v(irt), v(irt), SC_RR, nullptr);
        double rr = 0.0;
        CK(h, cudaMemcpyAsync(&rr, s.d_sc + SC_RR, sizeof rr, cudaMemcpyDeviceToHost, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
        const double rt = std::sqrt(rr);
        // accepted when it cuts the residual ten-fold (or meets the tolerance);
        // an FP32 pass that does not hands the rest of the solve to FP64 passes
        const bool good = std::isfinite(rt) && (rt <= 0.1 * rnorm || rt <= sv.rel_tolerance * bnorm);
        if (good || (use64 && std::isfinite(rt) && rt < rnorm)) {
            std::swap(ix, ixt);
            std::swap(ir, irt);
            rnorm = rt;
        } else if (use64) {
            break;  // the FP64 pass made no progress either
        }
        if (!good) use64 = true;
    }
    copy_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(ix), n, v(V_X));
    if (s.n_con)
        constrained_vector_kernel<<<blocks_for(s.n_con, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_con, duc,
                                                                                                  s.n_con, v(V_X));
    add_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(V_X), n, v(V_U));
    CK(h, cudaGetLastError());
    if (int rc = check_tc_error(h)) return rc;
    if (info) {
        info->iterations = total_iters;
        info->converged = bnorm == 0.0 || rnorm <= sv.rel_tolerance * bnorm;
        info->breakdown = breakdown;
        info->refinements = passes;
        info->fp64_iterations = iters64;
        info->rhs_norm = bnorm;
        info->residual_norm = bnorm == 0.0 ? 0.0 : rnorm;
    }
    return CP_OK;
}

}  // namespace

int cp_solver_default(cp_solver_t* sv) {
    if (!sv) return CP_E_ARG;
    sv->kind = CP_SOLVER_BICG;
    sv->max_iterations = 50000;
    sv->rel_tolerance = 1.0e-10;
    sv->precond_norm = 0;
    sv->check_every = 8;
    sv->precond = CP_PRECOND_JACOBI;
    sv->kernel_mode = 0;
    sv->precision = CP_PRECISION_FP64;
    sv->max_refinements = 0;
    sv->inner_tolerance = 0.0;
    return CP_OK;
}


// the solver settings of a Newton iteration, checked (solver NULL: defaults)
static int newton_settings(cp_handle* h, const cp_solver_t* solver, cp_solver_t* out) {
    auto& s = h->sys;
    if (!s.n_dofs) return fail(h, CP_E_STATE, "cp_newton_iteration: no dofs bound");
    cp_solver_t sv;
    if (solver)
        sv = *solver;
    else
        cp_solver_default(&sv);
    if ((sv.kind != CP_SOLVER_BICG && sv.kind != CP_SOLVER_BICGSTAB) || sv.max_iterations < 1 ||
        !(sv.rel_tolerance >= 0.0))
        return fail(h, CP_E_ARG, "cp_newton_iteration: bad solver settings");
    if (sv.precond != CP_PRECOND_JACOBI && sv.precond != CP_PRECOND_NODE_BLOCK)
        return fail(h, CP_E_ARG, "cp_newton_iteration: unknown preconditioner");
    if (sv.kernel_mode < 0 || sv.kernel_mode > 2) return fail(h, CP_E_ARG, "cp_newton_iteration: bad kernel_mode");
    if (sv.precond == CP_PRECOND_NODE_BLOCK && (sv.kind != CP_SOLVER_BICG || sv.precond_norm))
        return fail(h, CP_E_UNSUPPORTED, "cp_newton_iteration: node blocks need BiCG with the true-residual test");
    if (sv.precond == CP_PRECOND_NODE_BLOCK && !s.n_blocks)
        return fail(h, CP_E_UNSUPPORTED, "cp_newton_iteration: the dof map has no node blocks");
    if (sv.precision != CP_PRECISION_FP64 && sv.precision != CP_PRECISION_MIXED)
        return fail(h, CP_E_ARG, "cp_newton_iteration: unknown precision");
    if (sv.precision == CP_PRECISION_MIXED &&
        (sv.kind != CP_SOLVER_BICG || sv.precond != CP_PRECOND_JACOBI || sv.precond_norm || sv.max_refinements < 0 ||
         !(sv.inner_tolerance >= 0.0 && sv.inner_tolerance < 1.0)))
        return fail(h, CP_E_UNSUPPORTED, "cp_newton_iteration: mixed precision runs Jacobi BiCG, true residual");
    *out = sv;
    return CP_OK;
}

static int newton_after_assembly(cp_handle* h, const cp_solver_t& sv, const double* h_du_constrained,
                                 cp_solve_info_t* info);

int cp_newton_iteration(cp_handle* h, const double* h_du_constrained, double F_e, double F_r,
                        const cp_solver_t* solver, cp_solve_info_t* info) {
    if (!h) return CP_E_ARG;
    cp_solver_t sv;
    if (int rc = newton_settings(h, solver, &sv)) return rc;
    if (int rc = check_device(h)) return rc;
    if (int rc = ensure_staging(h, false)) return rc;
    if (sv.precision == CP_PRECISION_MIXED) return mixed_newton_iteration(h, sv, h_du_constrained, F_e, F_r, info);
    auto& s = h->sys;
    const int64_t nc = h->n_cells;
    // batched getElementalValues at the current u
    gather_ulocal_kernel<<<blocks_for(24 * nc, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(
        s.d_vec + V_U * s.n_dofs, s.d_cell_dofs, 24 * nc, s.d_Ul);
    if (int rc = cp_assemble_device(h, s.d_Ul, F_e, F_r, s.d_Ke, s.d_Re, h->d_status)) return rc;
    return newton_after_assembly(h, sv, h_du_constrained, info);
}

int cp_newton_solve(cp_handle* h, const double* h_du_constrained, const cp_solver_t* solver,
                    cp_solve_info_t* info) {
    if (!h) return CP_E_ARG;
    cp_solver_t sv;
    if (int rc = newton_settings(h, solver, &sv)) return rc;
    if (sv.precision != CP_PRECISION_FP64)
        return fail(h, CP_E_UNSUPPORTED, "cp_newton_solve: FP64 only (its Ke/Re come from cp_batch_assemble)");
    if (int rc = check_device(h)) return rc;
    if (int rc = ensure_staging(h, false)) return rc;
    return newton_after_assembly(h, sv, h_du_constrained, info);
}

// K and R from the element matrices in sys.d_Ke / d_Re, condensation, the
// Krylov solve, distribute and u += du
static int newton_after_assembly(cp_handle* h, const cp_solver_t& sv, const double* h_du_constrained,
                                 cp_solve_info_t* info) {
    auto& s = h->sys;
    const int64_t n = s.n_dofs;
    double* V = s.d_vec;
    auto v = [&](int k) { return V + (int64_t)k * n; };
    const unsigned nb = blocks_for(n, SOLVE_BLOCK);
    // K and R (distribute_local_to_global), in cell order per entry
    scatter_sum_kernel<<<blocks_for(s.nnz, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_Ke, s.d_kptr, s.d_kidx,
                                                                                     s.nnz, s.d_vals);
    scatter_sum_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_Re, s.d_rptr, s.d_ridx, n, v(V_R));
    // condensation of the prescribed increments
    if (s.n_con && h_du_constrained)
        CK(h, cudaMemcpyAsync(s.d_duc, h_du_constrained, sizeof(double) * s.n_con, cudaMemcpyHostToDevice,
                              h->stream));
    const double* duc = (s.n_con && h_du_constrained) ? s.d_duc : nullptr;
    CK(h, cudaMemsetAsync(v(V_DC), 0, sizeof(double) * n, h->stream));
    if (s.n_con)
        constrained_vector_kernel<<<blocks_for(s.n_con, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_con, duc,
                                                                                                  s.n_con, v(V_DC));
    sys_spmv(h, v(V_DC), v(V_KDC), nullptr);
    condense_rhs_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(V_R), v(V_KDC), v(V_DC), s.d_cmask, n, v(V_RHS));
    condense_matrix_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_row_ptr, s.d_col, s.d_cmask, n, s.d_vals);
    jacobi_setup_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(s.d_vals, s.d_diag, n, v(V_DINV));
    if (sv.precond == CP_PRECOND_NODE_BLOCK)
        block_setup_kernel<<<blocks_for(s.n_blocks, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_vals, s.d_blkpos,
                                                                                             s.n_blocks, s.d_binv);
    transpose_values_kernel<<<blocks_for(s.nnz, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_vals, s.d_tpos, s.nnz,
                                                                                          s.d_valsT);
    int hinfo[3] = {0, 0, 0};
    double bnorm = 0.0;
    if (int rc = krylov_solve(h, sv, v(V_RHS), hinfo, &bnorm)) return rc;
    // distribute: constrained dofs take their prescribed increments exactly
    if (s.n_con)
        constrained_vector_kernel<<<blocks_for(s.n_con, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(s.d_con, duc,
                                                                                                  s.n_con, v(V_X));
    add_kernel<<<nb, SOLVE_BLOCK, 0, h->stream>>>(v(V_X), n, v(V_U));
    CK(h, cudaGetLastError());
    double scf[SC_COUNT];
    CK(h, cudaMemcpyAsync(scf, s.d_sc, sizeof scf, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (info) {
        info->iterations = hinfo[0];
        info->converged = hinfo[1];
        info->breakdown = hinfo[2];
        info->refinements = 0;
        info->fp64_iterations = hinfo[0];
        info->rhs_norm = bnorm;
        info->residual_norm = bnorm == 0.0 ? 0.0 : std::sqrt(sv.precond_norm ? scf[SC_ZZ] : scf[SC_RR]);
    }
    return CP_OK;
}

int cp_update_from_displacement(cp_handle* h, double F_e, double F_r) {
    if (!h) return CP_E_ARG;
    auto& s = h->sys;
    if (!s.n_dofs) return fail(h, CP_E_STATE, "cp_update_from_displacement: no dofs bound");
    if (int rc = check_device(h)) return rc;
    if (int rc = ensure_staging(h, false)) return rc;
    const int64_t nc = h->n_cells;
    const FromMesh fm{s.d_Ul, h->d_gradN, h->d_JxW, h->uniform};
    if (h->opts.plain_kernel || h->opts.reference_order) {  // F of every qp first, then that update on it
        gather_ulocal_kernel<<<blocks_for(24 * nc, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(
            s.d_vec + V_U * s.n_dofs, s.d_cell_dofs, 24 * nc, s.d_Ul);
        mesh_F_kernel<<<blocks_for(h->n_qp, 256), 256, 0, h->stream>>>(fm, h->n_qp, h->d_F);
        CK(h, cudaGetLastError());
        return dispatch_update(h, h->d_F, 0, F_e, F_r, nullptr, nullptr, nullptr, h->d_status);
    }
    cp_handle::GraphKey key;
    key.kind = 2;
    key.fe = bits_of(F_e);
    key.fr = bits_of(F_r);
    key.epoch = h->tune_epoch;
    const int rc = run_graph(h, key, [&]() -> int {
        gather_ulocal_kernel<<<blocks_for(24 * nc, SOLVE_BLOCK), SOLVE_BLOCK, 0, h->stream>>>(
            s.d_vec + V_U * s.n_dofs, s.d_cell_dofs, 24 * nc, s.d_Ul);
        for (size_t gi = 0; gi < h->groups.size(); ++gi)
            sorted_update_group(h, gi, fm, 0, F_e, F_r, nullptr, nullptr, nullptr, nullptr, h->d_status, h->d_keepF,
                                h->d_keepT);
        CK(h, cudaGetLastError());
        return CP_OK;
    });
    if (rc != CP_OK) return rc;
    h->have_post = true;
    return CP_OK;
}

int32_t cp_tune_select(int32_t n_variants, int32_t reps, const double* ms, int32_t default_variant,
                       double min_gain) {
    if (n_variants < 1 || reps < 1 || !ms) return -1;
    std::vector<double> med(n_variants, 0.0);
    std::vector<bool> valid(n_variants, false);
    for (int v = 0; v < n_variants; ++v) {
        std::vector<double> x;
        for (int r = 0; r < reps; ++r) {
            const double t = ms[(int64_t)v * reps + r];
            if (std::isfinite(t) && t >= 0.0) x.push_back(t);
        }
        if (x.empty()) continue;
        std::sort(x.begin(), x.end());
        const size_t c = x.size();
        med[v] = c % 2 ? x[c / 2] : 0.5 * (x[c / 2 - 1] + x[c / 2]);
        valid[v] = true;
    }
    int best = -1;
    for (int v = 0; v < n_variants; ++v)
        if (valid[v] && (best < 0 || med[v] < med[best])) best = v;
    if (best < 0) return -1;
    if (default_variant >= 0 && default_variant < n_variants && valid[default_variant] && best != default_variant &&
        !(med[best] < (1.0 - min_gain) * med[default_variant]))
        return default_variant;
    return best;
}

int cp_autotune(cp_handle* h, const double* d_in, int32_t path, int32_t reps, double min_gain,
                cp_tune_result_t* results, int32_t max_results) {
    if (!h) return CP_E_ARG;
    if (h->n_qp == 0) return fail(h, CP_E_STATE, "cp_autotune: no qps bound");
    if (!d_in || (path != CP_TUNE_UPDATE && path != CP_TUNE_ASSEMBLE) || reps < 1 || reps > 64 ||
        !(min_gain >= 0.0 && min_gain < 1.0) || max_results < 0)
        return fail(h, CP_E_ARG, "cp_autotune: bad arguments");
    if (h->opts.plain_kernel || h->opts.reference_order)
        return fail(h, CP_E_UNSUPPORTED, "cp_autotune: the plain and reference-order updates have one launch shape");
    if (path == CP_TUNE_ASSEMBLE && h->n_cells == 0) return fail(h, CP_E_STATE, "cp_autotune: no mesh bound");
    if (int rc = check_device(h)) return rc;
    if (int rc = ensure_staging(h, path == CP_TUNE_UPDATE)) return rc;
    if (path == CP_TUNE_ASSEMBLE && !h->d_stage && cudaMalloc(&h->d_stage, sizeof(double) * 90 * h->n_qp) != cudaSuccess)
        return fail(h, CP_E_NOMEM, "cp_autotune: staging allocation failed");
    constexpr int V = U2_VARIANTS;
    std::vector<cudaEvent_t> ev(2 * V * reps, nullptr);
    for (auto& e : ev) CK(h, cudaEventCreate(&e));
    const FromArray fa{d_in};
    const FromMesh fm{d_in, h->d_gradN, h->d_JxW, h->uniform};
    int rc = CP_OK;
    const int ng = (int)h->groups.size();
    for (int gi = 0; gi < ng && rc == CP_OK; ++gi) {
        Group& g = h->groups[gi];
        const int64_t m = g.count;
        auto launch = [&](int v) {
            return path == CP_TUNE_UPDATE
                       ? launch_update2(h, g, fa, 0, m, 1, 0.0, 0.0, h->d_P, nullptr, h->d_dPdF, nullptr, h->d_status,
                                        nullptr, nullptr, v)
                       : launch_update2(h, g, fm, 0, m, 1, 0.0, 0.0, nullptr, nullptr, nullptr, h->d_stage,
                                        h->d_status, nullptr, nullptr, v);
        };
        if (path == CP_TUNE_UPDATE)
            sort_group(h, g, fa, 0, m);
        else
            sort_group(h, g, fm, 0, m);
        std::vector<double> ms(V * reps, -1.0);
        for (int v = 0; v < V && rc == CP_OK; ++v) {
            if (v == U2_QUAD && h->dopts.max_search != 1) continue;  // not applicable: no timing
            cudaError_t e = launch(v);  // untimed first launch
            for (int r = 0; r < reps && e == cudaSuccess; ++r) {
                cudaEventRecord(ev[2 * (v * reps + r)], h->stream);
                e = launch(v);
                cudaEventRecord(ev[2 * (v * reps + r) + 1], h->stream);
            }
            if (e != cudaSuccess) rc = cuda_fail(h, e, "cp_autotune: launch");
        }
        if (rc == CP_OK) {
            const cudaError_t e = cudaStreamSynchronize(h->stream);
            if (e != cudaSuccess) rc = cuda_fail(h, e, "cp_autotune: synchronize");
        }
        if (rc != CP_OK) break;
        for (int t = 0; t < V * reps; ++t) {
            float x = 0.f;
            if (cudaEventElapsedTime(&x, ev[2 * t], ev[2 * t + 1]) == cudaSuccess) ms[t] = x;
        }
        const int pmax = g.nt_class == 16 ? 16 : (g.nt_class == 32 ? 32 : 48);
        const int def = u2_default_variant(pmax, m);
        const int chosen = cp_tune_select(V, reps, ms.data(), def, min_gain);
        if (chosen >= 0) g.tuned[path] = chosen;
        if (results && gi < max_results) {
            cp_tune_result_t& out = results[gi];
            out.lattice = g.lattice;
            out.chosen = chosen;
            out.default_variant = def;
            out.reserved = 0;
            out.n_qp = m;
            for (int v = 0; v < V; ++v) {
                std::vector<double> one(ms.begin() + v * reps, ms.begin() + (v + 1) * reps);
                std::sort(one.begin(), one.end());
                out.median_ms[v] = one.size() % 2 ? one[one.size() / 2]
                                                  : 0.5 * (one[one.size() / 2 - 1] + one[one.size() / 2]);
            }
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    ++h->tune_epoch;
    return rc == CP_OK ? ng : rc;
}

int cp_debug_barrier_test(cp_handle* h, int32_t withhold_block, double wait_seconds) {
    if (!h || !(wait_seconds >= 0.0 && wait_seconds <= 60.0) || withhold_block < -1) return CP_E_ARG;
    h->barrier_withhold = withhold_block;
    h->barrier_wait_ns = (unsigned long long)(wait_seconds * 1e9);
    return CP_OK;
}

int cp_graph_stats(cp_handle* h, int64_t* captures, int64_t* launches) {
    if (!h) return CP_E_ARG;
    if (captures) *captures = h->graph_captures;
    if (launches) *launches = h->graph_launches;
    return CP_OK;
}

// ---- continuous batching across handles ------------------------------------

int cp_batch_create(int32_t device, cp_batch** out) {
    if (!out) return CP_E_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return CP_E_CUDA;
    cp_batch* b = new cp_batch();
    b->device = device;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming) != cudaSuccess) {
        cp_batch_destroy(b);
        return CP_E_CUDA;
    }
    *out = b;
    return CP_OK;
}

void cp_batch_destroy(cp_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto e : b->ev_in) cudaEventDestroy(e);
    if (b->ev_done) cudaEventDestroy(b->ev_done);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* cp_batch_last_error(const cp_batch* b) { return b ? b->err.c_str() : "null batch"; }

int64_t cp_batch_launches(const cp_batch* b) { return b ? b->launches : 0; }

static int batch_fail(cp_batch* b, int code, const std::string& msg) {
    b->err = msg;
    return code;
}

#define BCK(b, call)                                                                                  \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return batch_fail(b, CP_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// The sorted update of every lattice group of hs[0..n) at the displacement
// each handle holds (its device u, as cp_newton_iteration gathers it), as
// shared launches on the batch's stream: one counting sort over all groups
// (per group keys and buckets) and one update launch per lattice class.
// flag 1: the assembly (JxW P, JxW dP/dF staged, then each handle's
// contraction into its system's Ke/Re); flag 0: the post-pass (F and T kept
// for cp_averages).  Ordered after the work queued on each handle's stream
// and before the work queued there afterwards.
static int batch_run(cp_batch* b, cp_handle* const* hs, int32_t n, const double* F_e, const double* F_r, int flag) {
    if (!b) return CP_E_ARG;
    if (!hs || n < 1 || !F_e || !F_r) return batch_fail(b, CP_E_ARG, "cp_batch: bad arguments");
    for (int i = 0; i < n; ++i) {
        cp_handle* h = hs[i];
        if (!h) return batch_fail(b, CP_E_ARG, "cp_batch: null handle");
        if (h->device != b->device) return batch_fail(b, CP_E_ARG, "cp_batch: handle on another device");
        if (!h->sys.n_dofs) return batch_fail(b, CP_E_STATE, "cp_batch: a handle has no dofs bound");
        if (h->opts.plain_kernel || h->opts.reference_order)
            return batch_fail(b, CP_E_UNSUPPORTED, "cp_batch: needs the sorted update");
        for (int j = 0; j < i; ++j)
            if (hs[j] == h) return batch_fail(b, CP_E_ARG, "cp_batch: a handle is listed twice");
    }
    BCK(b, cudaSetDevice(b->device));
    for (int i = 0; i < n; ++i) {
        cp_handle* h = hs[i];
        if (ensure_staging(h, false)) return batch_fail(b, CP_E_NOMEM, "cp_batch: " + h->err);
        if (flag == 1 && !h->d_stage && cudaMalloc(&h->d_stage, sizeof(double) * 90 * h->n_qp) != cudaSuccess)
            return batch_fail(b, CP_E_NOMEM, "cp_batch: staging allocation failed");
    }
    while ((int)b->ev_in.size() < n) {
        cudaEvent_t e;
        BCK(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->ev_in.push_back(e);
    }
    for (int i = 0; i < n; ++i) {
        BCK(b, cudaEventRecord(b->ev_in[i], hs[i]->stream));
        BCK(b, cudaStreamWaitEvent(b->stream, b->ev_in[i], 0));
    }
    std::vector<BatchDesc> all;
    for (int i = 0; i < n; ++i) {
        cp_handle* h = hs[i];
        auto& y = h->sys;
        const int64_t nc = h->n_cells;
        gather_ulocal_kernel<<<blocks_for(24 * nc, SOLVE_BLOCK), SOLVE_BLOCK, 0, b->stream>>>(
            y.d_vec + V_U * y.n_dofs, y.d_cell_dofs, 24 * nc, y.d_Ul);
        const FromMesh fm{y.d_Ul, h->d_gradN, h->d_JxW, h->uniform};
        for (const auto& g : h->groups) {
            BatchDesc d{};
            d.L = h->d_lat[g.lattice];
            d.o = h->dopts;
            d.g = g.dev;
            d.fm = fm;
            d.key = g.d_key;
            g.sorted = true;
            d.hist = g.d_hist;
            d.perm = g.d_perm;
            d.m = g.count;
            d.F_e = F_e[i];
            d.F_r = F_r[i];
            d.stage = flag == 1 ? h->d_stage : nullptr;
            d.status = h->d_status;
            d.stats = h->d_stats;
            d.keepF = flag == 0 ? h->d_keepF : nullptr;
            d.keepT = flag == 0 ? h->d_keepT : nullptr;
            d.lattice_id = g.lattice;
            all.push_back(d);
        }
    }
    // classes: the PMAX of each group's lattice, taken from its handle
    std::vector<int> cls;
    for (int i = 0; i < n; ++i)
        for (const auto& g : hs[i]->groups) cls.push_back(g.nt_class == 16 ? 16 : (g.nt_class == 32 ? 32 : 48));
    for (size_t c0 = 0; c0 < all.size(); c0 += CP_BATCH_MAX) {
        const int cnt = (int)std::min<size_t>(CP_BATCH_MAX, all.size() - c0);
        BatchArgs a;
        a.n = cnt;
        a.flag = flag;
        int64_t b128 = 0, b256 = 0;
        for (int k = 0; k < cnt; ++k) {
            a.d[k] = all[c0 + k];
            b128 += (a.d[k].m + QP_BLOCK - 1) / QP_BLOCK;
            b256 += (a.d[k].m + 255) / 256;
        }
        batch_hist_zero_kernel<<<cnt, 2 * SORT_BUCKETS, 0, b->stream>>>(a);
        if (b128) classify_batch_kernel<<<(unsigned)b128, QP_BLOCK, 0, b->stream>>>(a);
        bucket_scan_batch_kernel<<<cnt, 32, 0, b->stream>>>(a);
        if (b256) bucket_scatter_batch_kernel<<<(unsigned)b256, 256, 0, b->stream>>>(a);
        BCK(b, cudaGetLastError());
        for (int pm : {16, 32, 48}) {
            BatchArgs u;
            u.n = 0;
            u.flag = flag;
            for (int k = 0; k < cnt; ++k)
                if (cls[c0 + k] == pm) u.d[u.n++] = all[c0 + k];
            if (!u.n) continue;
            cudaError_t e = pm == 16 ? launch_update2_batch<16>(b->stream, u)
                                     : (pm == 32 ? launch_update2_batch<32>(b->stream, u)
                                                 : launch_update2_batch<48>(b->stream, u));
            if (e != cudaSuccess) return batch_fail(b, CP_E_CUDA, std::string("batched update: ") + cudaGetErrorString(e));
            ++b->launches;
        }
    }
    for (int i = 0; i < n; ++i) {
        cp_handle* h = hs[i];
        if (flag == 1)
            contract_kernel<<<blocks_for(h->n_cells, CONTRACT_CELLS), CONTRACT_CELLS * 8, 0, b->stream>>>(
                h->d_stage, h->d_gradN, h->uniform, 0, h->n_cells, h->sys.d_Ke, h->sys.d_Re);
        else
            h->have_post = true;
    }
    BCK(b, cudaGetLastError());
    BCK(b, cudaEventRecord(b->ev_done, b->stream));
    for (int i = 0; i < n; ++i) BCK(b, cudaStreamWaitEvent(hs[i]->stream, b->ev_done, 0));
    return CP_OK;
}

int cp_batch_assemble(cp_batch* b, cp_handle* const* hs, int32_t n, const double* F_e, const double* F_r) {
    return batch_run(b, hs, n, F_e, F_r, 1);
}

int cp_batch_post(cp_batch* b, cp_handle* const* hs, int32_t n, const double* F_e, const double* F_r) {
    return batch_run(b, hs, n, F_e, F_r, 0);
}

}  // extern "C"

