// cp_tc.cu -- the element contraction of getElementalValues
// (getElementalValues.cc:144-162) on the 5th-generation tensor cores, in
// split-BF16 with FP32 accumulation (the mixed-precision assembly).
//
// For a mesh whose cells share their shape-function gradients (cp_bind_mesh
// with uniform != 0), Ke of a cell is one small GEMM against a constant:
//
//   Ke[3 a1 + i][3 a2 + j] = sum_{q,k,l} D_q[i][k][j][l] * g_q[a1][k] g_q[a2][l]
//
// with D_q = JxW_q dP/dF_q (the update's stage).  Rows m = (cell, i, j) (9 per
// cell), columns n = (a1, a2) (64), reduction t = (q, k, l) (72, padded to
// 80): C[m][n] = sum_t A[m][t] B[n][t] with A the staged tangents and
// B[n][t] = g_q[a1][k] g_q[a2][l] (one constant 64 x 72 matrix).  A tile is
// 14 cells = 126 of the 128 rows of one tcgen05.mma (M = 128, N = 64, K = 16
// per instruction).  Both operands are split into three bf16 terms
// (x = hi + mid + lo, each the bf16 rounding of what is left), and the six
// products hi.hi, hi.mid, mid.hi, hi.lo, mid.mid, lo.hi accumulate in one
// FP32 accumulator in tensor memory: relative error ~1e-7 against the FP64
// contraction.  Re stays FP64 (the Newton residual), computed from the staged
// P with the same operation order as contract_kernel, so it is bit-identical
// to the FP64 assembly's.
//
// One persistent CTA per SM (the shared memory below allows one): the
// tile's staged values (14 x 720 doubles, contiguous) arrive by one bulk copy
// (cp.async.bulk, completion on an mbarrier) issued while the previous tile
// is still in its MMA and epilogue; the 256 threads split them into the
// three bf16 operand copies in the canonical K-major layout (8-row x 16-byte
// core matrices, no swizzle); one thread issues the 30 MMAs and commits them
// to a second mbarrier; the epilogue reads the accumulator with tcgen05.ld
// (warp w reads TMEM lanes 32 (w % 4) .. +31, column half w / 4), scatters it
// into the cell-major Ke layout in shared memory and writes it out coalesced.
// Every mbarrier wait is bounded (2 s of the global timer): on expiry the
// kernel raises *err, waits (bounded) for its own bulk copy and MMAs still in
// flight, frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cp_launch.h"

namespace cp {

namespace {

constexpr int TC_CELLS = 14;
constexpr int TC_M = 128, TC_N = 64, TC_K = 80, TC_KREAL = 72;
constexpr int TC_THREADS = 256;
constexpr int TC_ROWBYTES = (TC_K / 8) * 128;               // one 8-row group of a K-major operand: 1280 B
constexpr int TC_A_BYTES = (TC_M / 8) * TC_ROWBYTES;        // 20,480
constexpr int TC_B_BYTES = (TC_N / 8) * TC_ROWBYTES;        // 10,240
constexpr int TC_IN_DOUBLES = TC_CELLS * 720;               // staged JxW P (9) + JxW dP/dF (81) per qp
constexpr int TC_OFF_IN = 0;
constexpr int TC_OFF_A = 80896;                             // 80,640 rounded up to 1 KB
constexpr int TC_OFF_B = TC_OFF_A + 3 * TC_A_BYTES;         // 142,336
constexpr int TC_OFF_KE = TC_OFF_B + 3 * TC_B_BYTES;        // 173,056
constexpr int TC_OFF_G = TC_OFF_KE + TC_CELLS * 576 * 4;    // 205,312
constexpr int TC_OFF_BAR = TC_OFF_G + 192 * 8;              // 206,848
constexpr int TC_SMEM = TC_OFF_BAR + 64;
constexpr uint32_t TC_TMEM_COLS = 64;                       // FP32 accumulator, N = 64 columns
constexpr uint64_t TC_WAIT_NS = 2000000000ull;

static_assert(TC_OFF_A >= TC_IN_DOUBLES * 8, "input staging overlaps the operands");
static_assert(TC_CELLS * 9 <= TC_M, "a tile's rows exceed the MMA's M");
static_assert(TC_SMEM <= 232448, "more shared memory than a CTA may have");

// column t = 9 q + 3 k + l of A (t < 72) -> offset of JxW dP/dF[i][k][j][l]
// of qp q in a cell's staged record, relative to that of [i][0][j][0] of qp 0
// (records of 90 doubles: 9 of JxW P, then 81 of JxW dP/dF)
__constant__ short c_tc_off[TC_KREAL] = {
#define CP_TC_OFF(q) 90 * q, 90 * q + 1, 90 * q + 2, 90 * q + 9, 90 * q + 10, 90 * q + 11, 90 * q + 18, \
                     90 * q + 19, 90 * q + 20
    CP_TC_OFF(0), CP_TC_OFF(1), CP_TC_OFF(2), CP_TC_OFF(3), CP_TC_OFF(4), CP_TC_OFF(5), CP_TC_OFF(6), CP_TC_OFF(7)
#undef CP_TC_OFF
};

// byte offset of element (r, k) of a K-major operand tile (r: M or N index)
__device__ __forceinline__ int kmajor_off(int r, int k) {
    return (r >> 3) * TC_ROWBYTES + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    return ok != 0;
}

// wait for the phase with a bound of TC_WAIT_NS of the global timer (and a
// poll-count backstop far beyond it); false on expiry
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1; it < (1u << 31); ++it) {
        if (mbar_try_wait(bar, phase)) return true;
        if ((it & 255u) == 0 && global_ns() - t0 > TC_WAIT_NS) return false;
    }
    return false;
}

// bulk copy of 'bytes' (multiple of 16, both addresses 16-byte aligned) from
// this GPU's global memory into shared memory, completing on 'bar'
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// shared-memory matrix descriptor of a K-major, unswizzled operand: core
// matrices 8 rows x 16 bytes, K-adjacent core matrices 128 B apart (leading
// byte offset), 8-row groups TC_ROWBYTES apart (stride byte offset);
// bits 46-47 = 1 (the sm_100 descriptor version), layout type 0 (no swizzle)
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(128u >> 4) << 16) |
           ((uint64_t)((uint32_t)TC_ROWBYTES >> 4) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits
// 17-22, M >> 4 at bits 24-28
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// x = hi + mid + lo, each the bf16 rounding of what the previous terms leave
__device__ __forceinline__ void split3(double x, unsigned short* h) {
    const __nv_bfloat16 a = __double2bfloat16(x);
    const double r1 = x - (double)__bfloat162float(a);
    const __nv_bfloat16 b = __double2bfloat16(r1);
    const double r2 = r1 - (double)__bfloat162float(b);
    const __nv_bfloat16 c = __double2bfloat16(r2);
    h[0] = __bfloat16_as_ushort(a);
    h[1] = __bfloat16_as_ushort(b);
    h[2] = __bfloat16_as_ushort(c);
}

__global__ void __launch_bounds__(TC_THREADS, 1)
    ke_tc_kernel(const double* __restrict__ stage, const double* __restrict__ gradN, int64_t cell_begin,
                 int64_t cell_end, float* __restrict__ Ke, double* __restrict__ Re, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    double* sIn = reinterpret_cast<double*>(smem + TC_OFF_IN);
    unsigned char* sA = smem + TC_OFF_A;
    unsigned char* sB = smem + TC_OFF_B;
    float* sKe = reinterpret_cast<float*>(smem + TC_OFF_KE);
    double* sG = reinterpret_cast<double*>(smem + TC_OFF_G);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TC_OFF_BAR);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + TC_OFF_BAR + 16);
    int* s_err = reinterpret_cast<int*>(smem + TC_OFF_BAR + 20);
    const uint32_t bar_load = smem_u32(&bars[0]), bar_mma = smem_u32(&bars[1]);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t ncell = cell_end - cell_begin;
    const int64_t ntiles = (ncell + TC_CELLS - 1) / TC_CELLS;

    if (tid == 0) {
        mbar_init(bar_load, 1);
        mbar_init(bar_mma, 1);
        *s_err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int t = tid; t < 192; t += TC_THREADS) sG[t] = gradN[t];
    // operands start zeroed: the K padding (t = 72..79) and rows 126, 127
    // of A are never written again
    for (int t = tid; t < (3 * TC_A_BYTES + 3 * TC_B_BYTES) / 16; t += TC_THREADS)
        reinterpret_cast<uint4*>(sA)[t] = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    // B[n = 8 a1 + a2][t = 9 q + 3 k + l] = g_q[a1][k] g_q[a2][l], split
    for (int e = tid; e < TC_N * TC_KREAL; e += TC_THREADS) {
        const int n = e / TC_KREAL, t = e % TC_KREAL;
        const int a1 = n >> 3, a2 = n & 7, q = t / 9, k = (t / 3) % 3, l = t % 3;
        unsigned short h[3];
        split3(sG[q * 24 + a1 * 3 + k] * sG[q * 24 + a2 * 3 + l], h);
        const int off = kmajor_off(n, t);
#pragma unroll
        for (int p = 0; p < 3; ++p) *reinterpret_cast<unsigned short*>(sB + p * TC_B_BYTES + off) = h[p];
    }
    __syncthreads();  // barrier initialisation visible before the first copy

    uint32_t load_phase = 0, mma_phase = 0;
    bool load_pending = false, mma_pending = false;  // thread 0's view of its async work
    int64_t tile = blockIdx.x;
    if (tid == 0 && tile < ntiles) {
        const int64_t c0 = cell_begin + tile * TC_CELLS;
        const int nc = (int)((cell_end - c0) < TC_CELLS ? (cell_end - c0) : TC_CELLS);
        bulk_load(smem_u32(sIn), stage + c0 * 720, (uint32_t)(nc * 720 * 8), bar_load);
        load_pending = true;
    }
    for (; tile < ntiles; tile += gridDim.x) {
        const int64_t c0 = cell_begin + tile * TC_CELLS;
        const int nc = (int)((cell_end - c0) < TC_CELLS ? (cell_end - c0) : TC_CELLS);
        if (!mbar_wait(bar_load, load_phase)) atomicOr(s_err, 1);
        __syncthreads();
        if (*s_err) break;
        load_phase ^= 1u;
        if (tid == 0) load_pending = false;
        // A[m = 9 c + 3 i + j][t = 9 q + 3 k + l] = JxW dP/dF[i][k][j][l] of qp q
        // of cell c, split.  Work item (row m, chunk kc) fills columns
        // t = 8 kc .. 8 kc + 7 of the row: one 16-byte store per bf16 term;
        // the 32 lanes of a warp take consecutive rows of one chunk, so the
        // column offsets (c_tc_off) are the same in every lane
        for (int e = tid; e < (TC_KREAL / 8) * TC_M; e += TC_THREADS) {
            const int kc = e / TC_M, m = e % TC_M;
            if (m >= 9 * nc) continue;
            const int c = m / 9, r9 = m % 9;
            const double* row = sIn + c * 720 + 9 + 27 * (r9 / 3) + 3 * (r9 % 3);
            uint32_t w[3][4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                unsigned short h0[3], h1[3];
                split3(row[c_tc_off[8 * kc + 2 * u]], h0);
                split3(row[c_tc_off[8 * kc + 2 * u + 1]], h1);
#pragma unroll
                for (int p = 0; p < 3; ++p) w[p][u] = (uint32_t)h0[p] | ((uint32_t)h1[p] << 16);
            }
            const int off = kmajor_off(m, 8 * kc);
#pragma unroll
            for (int p = 0; p < 3; ++p)
                *reinterpret_cast<uint4*>(sA + p * TC_A_BYTES + off) = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
        }
        // Re in FP64 from JxW P, in contract_kernel's order of operations
        for (int e = tid; e < nc * 24; e += TC_THREADS) {
            const int c = e / 24, r = e % 24, a1 = r / 3, ci = r % 3;
            double acc = 0.0;
            for (int qq = 0; qq < 8; ++qq) {
                const double* Pq = sIn + (c * 8 + qq) * 90;
                const double* gq = sG + qq * 24;
                acc -= gq[a1 * 3] * Pq[3 * ci] + gq[a1 * 3 + 1] * Pq[3 * ci + 1] + gq[a1 * 3 + 2] * Pq[3 * ci + 2];
            }
            Re[(c0 + c) * 24 + r] = acc;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            // the next tile's staged values stream in during this tile's MMAs and epilogue
            const int64_t nt = tile + gridDim.x;
            if (nt < ntiles) {
                const int64_t n0 = cell_begin + nt * TC_CELLS;
                const int nn = (int)((cell_end - n0) < TC_CELLS ? (cell_end - n0) : TC_CELLS);
                bulk_load(smem_u32(sIn), stage + n0 * 720, (uint32_t)(nn * 720 * 8), bar_load);
                load_pending = true;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // small products first: lo.hi, mid.mid, hi.lo, mid.hi, hi.mid, hi.hi
            const int pa[6] = {2, 1, 0, 1, 0, 0}, pb[6] = {0, 1, 2, 0, 1, 0};
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            uint32_t acc = 0u;
#pragma unroll
            for (int s = 0; s < 6; ++s)
#pragma unroll
                for (int kk = 0; kk < TC_K / 16; ++kk) {
                    mma_bf16(tmem, kmajor_desc(a0 + pa[s] * TC_A_BYTES + kk * 256),
                             kmajor_desc(b0 + pb[s] * TC_B_BYTES + kk * 256), acc);
                    acc = 1u;
                }
            mma_commit(bar_mma);
            mma_pending = true;
        }
        if (!mbar_wait(bar_mma, mma_phase)) atomicOr(s_err, 1);
        __syncthreads();
        if (*s_err) break;
        mma_phase ^= 1u;
        if (tid == 0) mma_pending = false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        {
            const int quad = warp & 3, half = warp >> 2;
            const int row = 32 * quad + lane;
            uint32_t r0[16], r1[16];
            const uint32_t taddr = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(32 * half);
            tmem_ld16(taddr, r0);
            tmem_ld16(taddr + 16, r1);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < 9 * nc) {
                const int c = row / 9, i = (row % 9) / 3, j = row % 3;
                float* kc = sKe + c * 576;
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const int n0 = 32 * half + u, n1 = n0 + 16;
                    kc[(3 * (n0 >> 3) + i) * 24 + 3 * (n0 & 7) + j] = __uint_as_float(r0[u]);
                    kc[(3 * (n1 >> 3) + i) * 24 + 3 * (n1 & 7) + j] = __uint_as_float(r1[u]);
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        {
            float4* dst = reinterpret_cast<float4*>(Ke + c0 * 576);
            const float4* src = reinterpret_cast<const float4*>(sKe);
            for (int e = tid; e < nc * 144; e += TC_THREADS) dst[e] = src[e];
        }
        __syncthreads();
    }
    // leave: on an expired wait, let this CTA's own copy and MMAs finish
    // (bounded) before its tensor memory is released
    if (tid == 0 && *s_err) {
        if (load_pending) mbar_wait(bar_load, load_phase);
        if (mma_pending) mbar_wait(bar_mma, mma_phase);
        atomicOr(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
}

}  // namespace

cudaError_t prepare_ke_tc() {
    return cudaFuncSetAttribute(ke_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
}

cudaError_t launch_ke_tc(cudaStream_t s, const double* stage, const double* gradN, int64_t cell_begin,
                         int64_t cell_end, float* Ke, double* Re, int* err, int num_sms) {
    const int64_t ntiles = (cell_end - cell_begin + TC_CELLS - 1) / TC_CELLS;
    if (ntiles <= 0) return cudaSuccess;
    // the bulk copies start at stage + 720 * cell (5,760 B per cell): 16-byte
    // alignment of every copy follows from the base's
    if (reinterpret_cast<uintptr_t>(stage) & 15u) return cudaErrorInvalidValue;
    const unsigned grid = (unsigned)(ntiles < num_sms ? ntiles : num_sms);
    ke_tc_kernel<<<grid, TC_THREADS, TC_SMEM, s>>>(stage, gradN, cell_begin, cell_end, Ke, Re, err);
    return cudaGetLastError();
}

}  // namespace cp
