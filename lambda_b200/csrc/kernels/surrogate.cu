// Thin-film surrogate: a 5 -> 64 -> 64 -> 64 -> 4 MLP (ReLU hidden layers) that maps
// (lambda, cos theta, thickness, n_film, n_substrate) of a single film between air
// and a substrate to (R_s, R_p, T_s, T_p), standing in for the transfer matrix of
// Material::thinFilmReflectance (src/scene/material.h:263-309).
//
//   k_film_labels    training/audit data: uniform samples of the input box, labelled
//                    by the FP64 transfer matrix (tmm.cuh)
//   k_train_step     forward + backward of a minibatch on CUDA cores, forward rounded
//                    to BF16 exactly as inference rounds it; per-CTA gradients are
//                    summed with atomics
//   k_adam           Adam update of the FP32 master weights
//   k_mlp_tc         inference on the 5th-generation tensor cores: one persistent CTA
//                    per SM of 5 warpgroups, BF16 weights resident in shared memory
//                    (canonical K-major layout, no swizzle), each layer's input rows
//                    and FP32 accumulators in tensor memory (tcgen05.mma with A from
//                    TMEM), tcgen05.ld / tcgen05.st epilogues (ReLU, BF16)
//   k_film_encode    the render's thin-film shade, in three kernels per bounce: the
//   k_mlp_tc         hits' four hero-wavelength queries encoded as MLP rows, the
//   k_film_scatter   tensor-core MLP over them, then the scatter; hits outside the
//                    trained domain take the exact FP32 transfer matrix in the scatter
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "buffer_policy.h"
#include "engine.h"
#include "lambda_gpu.h"
#define LAMBDA_WAVEFRONT_HELPERS_ONLY
#include "wavefront.cuh"

using namespace lambda_dev;

namespace mlp {

constexpr int kIn = LAMBDA_MLP_IN, kH = LAMBDA_MLP_HIDDEN, kOut = LAMBDA_MLP_OUT;
constexpr int kInPad = 16;   // K of layer 1 (bf16 MMA K = 16)
constexpr int kOutPad = 16;  // N of layer 4 (M = 128 needs N % 16 == 0)
constexpr int kParams = LAMBDA_MLP_PARAMS;
// parameter offsets (row-major out x in)
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH * kH;
constexpr int oW4 = oB3 + kH, oB4 = oW4 + kOut * kH;
static_assert(oB4 + kOut == kParams, "parameter layout");

constexpr int kTileM = 128;  // rows per MMA tile (TMEM lanes)
constexpr int kRowStride = 8;  // floats per input row in the staging buffer

// Byte offset of element (r, k) of a K-major bf16 operand with K columns, stored as
// 8x8 core matrices (8 rows x 16 bytes, 128 contiguous bytes): core (r/8, k/8) at
// ((r/8) * (K/8) + k/8) * 128. Consecutive core matrices along K are 128 bytes apart
// (LBO), along M/N (K/8)*128 bytes apart (SBO).
__host__ __device__ constexpr int core_offset(int r, int k, int K) {
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// Shared-memory layout of the tensor-core MLP kernels (bytes). The biases ride in
// the MMAs: every operand row carries two constant-1 columns that meet (b_hi, b_lo),
// the bias split into two BF16 parts (b_lo = bf16(b - b_hi), so b_hi + b_lo is b to
// about 2^-17 relative), and the epilogues add nothing. For layers 2-4 that product
// is one extra K step whose second core matrix (k 8..15) is the zero block.
constexpr int sW1 = 0;                           // [64][16]: W1 in k 0..4, (b1 hi, b1 lo) in k 5, 6
constexpr int sW2 = sW1 + kH * kInPad * 2;       // [64][64]
constexpr int sW3 = sW2 + kH * kH * 2;           // [64][64]
constexpr int sW4 = sW3 + kH * kH * 2;           // [16][64]
constexpr int sB2 = sW4 + kOutPad * kH * 2;      // [64][8]: (b2 hi, b2 lo, 0, ...)
constexpr int sB3 = sB2 + kH * 16;               // [64][8]
constexpr int sB4 = sB3 + kH * 16;               // [16][8]
constexpr int kPackedWeightBytes = sB4 + kOutPad * 16;  // the weight image, copied as is
constexpr int sZero = kPackedWeightBytes;        // [128][8] zeros
// A CTA runs kChains warpgroups, each with its own stream of 128-row tiles, its own
// MMA-completion mbarrier and 96 TMEM columns: a 64-column FP32 accumulator and a
// 32-column BF16 operand (the layer's input rows, two values per column). The
// weights are the only operands in shared memory.
constexpr int kChains = 5;                       // 5 x 96 + 8 columns fit the SM's 512
constexpr int sBar = sZero + kTileM * 16;        // kChains mbarriers
constexpr int sTmemSlot = sBar + 8 * kChains;
constexpr int kMlpSmem = sTmemSlot + 8;
constexpr int kMlpThreads = 128 * kChains;
constexpr int kTmemAlloc = 512;                  // the CTA's TMEM allocation (a power of two)
constexpr int tAcc = 0;                          // chain c's accumulator: columns 64c .. 64c + 63
constexpr int tOperand = 64 * kChains;           // chain c's operand: columns 320 + 32c .. + 31
constexpr int tOnes = tOperand + 32 * kChains;   // (1, 1, 0 ...) rows, 8 columns, shared by the chains
static_assert(tOnes + 8 <= kTmemAlloc, "TMEM columns");

// Input normalisation to [-1, 1] over the trained box.
struct Range {
    float lo[kIn], hi[kIn];
};

__host__ __device__ inline float normalise(float v, float lo, float hi) { return 2.0f * (v - lo) / (hi - lo) - 1.0f; }

// Input encoding of one film query (lambda, cos theta in air, thickness, n_film,
// n_sub): the film's round-trip phase 2 delta = 4 pi n_f d cos(theta_f) / lambda
// (Snell: sin theta_f = sin theta / n_f) enters as (cos 2 delta, sin 2 delta), so
// the network sees the interference term as a smooth periodic feature; the angle
// and the two indices are normalised to [-1, 1]. The wavelength and thickness
// ranges bound the trained domain (and the phase), not the encoding.
__host__ __device__ inline void encode(const float *v, const Range &rg, float *x) {
    const float c0 = v[1], nf = v[3];
    const float cf = sqrtf(fmaxf(1.0f - (1.0f - c0 * c0) / (nf * nf), 0.0f));
    const float two_delta = 4.0f * 3.14159265358979f * nf * v[2] * cf / v[0];
#ifdef __CUDA_ARCH__
    sincosf(two_delta, &x[1], &x[0]);
#else
    x[0] = std::cos(two_delta);
    x[1] = std::sin(two_delta);
#endif
    x[2] = normalise(c0, rg.lo[1], rg.hi[1]);
    x[3] = normalise(nf, rg.lo[3], rg.hi[3]);
    x[4] = normalise(v[4], rg.lo[4], rg.hi[4]);
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier primitives (PTX ISA 8.7+, sm_100a)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return uint32_t(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor: start, leading-dimension (K) and stride (M/N)
// byte offsets in 16-byte units, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(kTileM >> 4) << 24);
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Waits for phase `parity` of an mbarrier; gives up after `limit` polls and reports false.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 32 consecutive FP32 columns of this warp's 32 TMEM lanes (one per thread). The
// values are valid only after tmem_wait(), which names them as operands so that no
// use is scheduled before the wait.
__device__ __forceinline__ void tmem_ld32(uint32_t addr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr));
}

__device__ __forceinline__ void tmem_ld4(uint32_t addr, uint32_t (&r)[4]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

// Waits for this thread's outstanding tcgen05.ld; the registers passed are tied to
// the wait.
__device__ __forceinline__ void tmem_wait(uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.wait::ld.sync.aligned;"
        : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "+r"(r[8]),
          "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]),
          "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]), "+r"(r[24]),
          "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
        :
        : "memory");
}

__device__ __forceinline__ void tmem_wait(uint32_t (&r)[4]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]) : : "memory");
}

// Ties registers loaded before an earlier tmem_wait to that wait (an empty volatile
// statement after it in program order).
__device__ __forceinline__ void tmem_after_wait(uint32_t (&r)[32]) {
    asm volatile(""
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31]));
}

// ReLU and round-to-nearest BF16 of two FP32 values in one instruction; lo goes
// to the low half (the lower address, element k), hi to the high half (k + 1).
__device__ __forceinline__ uint32_t relu_bf16x2(uint32_t lo, uint32_t hi) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(__uint_as_float(hi)), "f"(__uint_as_float(lo)));
    return d;
}

// ---------------------------------------------------------------------------
// Tensor-core inference
// ---------------------------------------------------------------------------

// D (TMEM) = A (TMEM, BF16, K-major rows: row i in lane i, two K values per 32-bit
// column) x B (shared memory descriptor).
__device__ __forceinline__ void mma_bf16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "r"(tmem_a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

// 16 / 8 consecutive 32-bit columns of this warp's 32 TMEM lanes (one per thread).
__device__ __forceinline__ void tmem_st16(uint32_t addr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(addr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

__device__ __forceinline__ void tmem_st8(uint32_t addr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(addr), "r"(r[0]),
                 "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}

// Waits for this thread's outstanding tcgen05.st.
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// One lane of a converged warp (elect.sync); the MMAs are issued from a
// warp-uniform branch, so their operands stay warp-uniform.
__device__ __forceinline__ bool elect_one() {
    uint32_t leader;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "elect.sync _|p, 0xffffffff;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(leader));
    return leader != 0;
}

// Round-to-nearest BF16 of two FP32 values; lo in the low half (element k).
__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
    uint32_t d;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// Barrier of warpgroup wg (named barrier 1 + wg, 128 threads).
__device__ __forceinline__ void wg_sync(int wg) { asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory"); }

// AND of a predicate over warpgroup wg, as its barrier.
__device__ __forceinline__ bool wg_sync_and(int wg, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.b32 q, %1, 0;\n\t"
        "barrier.cta.red.and.pred p, %2, 128, q;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r)
        : "r"(uint32_t(v)), "r"(1 + wg)
        : "memory");
    return r != 0;
}

// Inference over n_rows rows, or rows_per_count * *count rows when count is given
// (a count the GPU produced, such as a bounce's thin-film hits): row i's input is
// kRowStride floats already encoded (kQueries = false) or the i-th
// lambda_film_query, encoded here (kQueries = true); out: rows x (R_s, R_p, T_s, T_p).
//
// One CTA per SM, persistent, of kChains warpgroups. Each warpgroup works through its
// own 128-row tiles, one thread per row, with every layer's input rows kept in tensor
// memory: the thread writes its row's layer-1 operand (5 features, the two
// constant-1 bias columns, zeros to K = 16) with tcgen05.st, and each hidden layer's
// epilogue reads the accumulator (tcgen05.ld), applies ReLU and BF16 rounding in one
// cvt per pair and stores the next layer's operand back with tcgen05.st. The MMAs
// (M = 128, N = 64 or 16, K = 16 each) take A from those columns and only the
// weights from shared memory, so shared-memory bandwidth, which bounds the
// operand-in-shared-memory form at N = 64, carries 24.5 KB per tile instead of about
// 140 KB. Biases ride in the MMAs: layer 1 through its two constant-1
// columns; layers 2-4 through one extra K step, (1, 1, 0 ...) rows in tensor memory
// against (b_hi, b_lo, 0 ...) rows whose second core matrix is the zero block.
// One elected lane of the warpgroup's first warp issues a layer's MMAs and commits
// them to the warpgroup's mbarrier; the next tile's input is loaded (and encoded)
// while the output layer's MMAs run. Error bit 1 is set if an MMA completion wait
// gave up after `polls` polls (LAMBDA_DEFAULT_MMA_POLLS normally); the thread then
// waits again, bounded by the default limit, for the MMAs already issued, so no TMEM
// is read or freed under a running MMA, and the warpgroup stops after the tile.
template <bool kQueries>
__global__ void __launch_bounds__(kMlpThreads, 1) k_mlp_tc(const uint4 *__restrict__ packed,
                                                          const void *__restrict__ in, int n_rows, Range rg,
                                                          float4 *__restrict__ out, int *error, uint32_t polls,
                                                          const int *count = nullptr, int rows_per_count = 0) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int rows = count ? rows_per_count * *count : n_rows;
    const int tiles = (rows + kTileM - 1) / kTileM;
    if (int(blockIdx.x) * kChains >= tiles) return;  // uniform per block, before any TMEM allocation
    const int tid = threadIdx.x, wg = tid >> 7, r = tid & 127, wi = (tid >> 5) & 3;
    for (int i = tid; i < kPackedWeightBytes / 16; i += kMlpThreads) reinterpret_cast<uint4 *>(smem)[i] = packed[i];
    for (int i = tid; i < kTileM; i += kMlpThreads) *reinterpret_cast<uint4 *>(smem + sZero + i * 16) = make_uint4(0, 0, 0, 0);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + sTmemSlot);
    if (tid < kChains) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(smem + sBar + 8 * tid)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemAlloc)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_proxy_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t base = smem_u32(smem), tmem0 = *tmem_slot;
    const uint32_t lanes = uint32_t(wi * 32) << 16;  // this warp's 32 TMEM lanes
    if (wg == 0) {
        const uint32_t ones[8] = {0x3F803F80u, 0, 0, 0, 0, 0, 0, 0};  // bf16 (1, 1), zeros
        tmem_st8(tmem0 + tOnes + lanes, ones);
        tmem_wait_st();
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t acc = tmem0 + tAcc + uint32_t(64 * wg), opnd = tmem0 + tOperand + uint32_t(32 * wg);
    const uint32_t ones = tmem0 + tOnes, bar = base + sBar + 8 * wg;
    const uint32_t id64 = instr_desc(kH), id16 = instr_desc(kOutPad);
    uint32_t phase = 0;
    auto load_row = [&](int tile, float *e) {
        const int row = tile * kTileM + r;
#pragma unroll
        for (int i = 0; i < kIn; i++) e[i] = 0.0f;
        if (tile < tiles && row < rows) {
            if constexpr (kQueries) {
                const lambda_film_query q = static_cast<const lambda_film_query *>(in)[row];
                const float v[kIn] = {q.lambda_nm, q.cos_theta, q.thickness_nm, q.n_film, q.n_sub};
                encode(v, rg, e);
            } else {
                const float *x = static_cast<const float *>(in) + size_t(row) * kRowStride;
                const float4 a = *reinterpret_cast<const float4 *>(x);
                e[0] = a.x;
                e[1] = a.y;
                e[2] = a.z;
                e[3] = a.w;
                e[4] = x[4];
            }
        }
    };
    const int stride = int(gridDim.x) * kChains;
    float e[kIn];
    load_row(blockIdx.x * kChains + wg, e);
    bool ok = true;
    for (int tile = blockIdx.x * kChains + wg; tile < tiles && ok; tile += stride) {
        const int row = tile * kTileM + r;
        {
            const uint32_t x[8] = {bf16x2(e[0], e[1]), bf16x2(e[2], e[3]), bf16x2(e[4], 1.0f), bf16x2(1.0f, 0.0f), 0, 0, 0, 0};
            tmem_st8(opnd + lanes, x);
            tmem_wait_st();
        }
        bool done = true;
        float y[kOut];
#pragma unroll 1
        for (int layer = 0; layer < 4; layer++) {
            // the operand rows are in tensor memory; one lane of warp 0 issues the MMAs
            fence_before();
            wg_sync(wg);
            const int wofs = layer == 0 ? sW1 : (layer == 1 ? sW2 : (layer == 2 ? sW3 : sW4));
            const int bofs = layer == 1 ? sB2 : (layer == 2 ? sB3 : sB4);
            const uint64_t dw = smem_desc(base + wofs, 128, layer == 0 ? 256 : 1024);
            const uint64_t db = smem_desc(base + bofs, sZero - bofs, 128);
            if (wi == 0) {
                if (elect_one()) {
                    fence_after();
                    if (layer == 0) {
                        mma_bf16_ts(acc, opnd, dw, id64, 0);
                    } else {
                        const uint32_t idesc = layer == 3 ? id16 : id64;
                        mma_bf16_ts(acc, ones, db, idesc, 0);
#pragma unroll
                        for (int kk = 0; kk < kH / 16; kk++)  // K step kk: operand columns 8kk.., weight bytes 256kk..
                            mma_bf16_ts(acc, opnd + 8 * kk, dw + 16 * kk, idesc, 1);
                    }
                    mma_commit(bar);
                }
                __syncwarp();
            }
            if (layer == 3) load_row(tile + stride, e);  // under the output layer's MMAs
            if (!mbar_wait(bar, phase, polls)) {
                done = false;
                mbar_wait(bar, phase, LAMBDA_DEFAULT_MMA_POLLS);  // drain what was issued
            }
            phase ^= 1u;
            fence_after();
            if (layer < 3) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    uint32_t a[32], x[16];
                    tmem_ld32(acc + lanes + 32 * h, a);
                    tmem_wait(a);
#pragma unroll
                    for (int i = 0; i < 16; i++) x[i] = relu_bf16x2(a[2 * i], a[2 * i + 1]);
                    tmem_st16(opnd + lanes + 16 * h, x);
                }
                tmem_wait_st();
            } else {
                uint32_t o[4];
                tmem_ld4(acc + lanes, o);
                tmem_wait(o);
#pragma unroll
                for (int i = 0; i < kOut; i++) y[i] = __uint_as_float(o[i]);
            }
        }
        ok = wg_sync_and(wg, done);
        if (ok && row < rows) out[row] = make_float4(y[0], y[1], y[2], y[3]);
    }
    if (!ok && r == 0) atomicOr(error, 2);
    // every TMEM access has completed (tcgen05 waits) before the columns are released
    fence_before();
    __syncthreads();
    fence_after();
    if (tid < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem0), "r"(kTmemAlloc) : "memory");
}

// ---------------------------------------------------------------------------
// Training
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t i, int dim) {
    return double(splitmix(seed ^ splitmix(i * 8 + uint64_t(dim))) >> 11) * (1.0 / 9007199254740992.0);
}

// Uniform samples of the input box labelled by the FP64 transfer matrix.
// x: [n][kRowStride] normalised inputs; y: [n][4] (R_s, R_p, T_s, T_p).
__global__ void k_film_labels(uint64_t seed, int64_t first, int n, Range rg, float *x, float *y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v[kIn];
    for (int d = 0; d < kIn; d++)
        v[d] = float(rg.lo[d] + (rg.hi[d] - rg.lo[d]) * uniform01(seed, uint64_t(first + i), d));
    cx<double> idx[3] = {cx<double>{1.0, 0.0}, cx<double>{double(v[3]), 0.0}, cx<double>{double(v[4]), 0.0}};
    const double d = v[2];
    const FilmResult<double> r = film_stack<double, 1>(1, idx, &d, double(v[1]), double(v[0]));
    float e[kIn];
    encode(v, rg, e);
    for (int k = 0; k < kIn; k++) x[size_t(i) * kRowStride + k] = e[k];
    for (int k = kIn; k < kRowStride; k++) x[size_t(i) * kRowStride + k] = 0.0f;
    y[size_t(i) * 4] = float(r.rs);
    y[size_t(i) * 4 + 1] = float(r.rp);
    y[size_t(i) * 4 + 2] = float(r.ts);
    y[size_t(i) * 4 + 3] = float(r.tp);
}

constexpr int kTrainRows = 64;
constexpr int kTrainThreads = 256;
// shared memory of k_train_step (floats)
constexpr int tW = 0;                          // master weights rounded to bf16 (forward copy)
constexpr int tX = tW + kParams;               // [64][5]
constexpr int tH1 = tX + kTrainRows * kIn;     // [64][64]
constexpr int tH2 = tH1 + kTrainRows * kH;
constexpr int tH3 = tH2 + kTrainRows * kH;
constexpr int tDY = tH3 + kTrainRows * kH;     // [64][4]
constexpr int tDA = tDY + kTrainRows * kOut;   // [64][64]
constexpr int tDB = tDA + kTrainRows * kH;
constexpr int tLoss = tDB + kTrainRows * kH;
constexpr int kTrainSmem = (tLoss + 8) * 4;

// Dense layer on 64 rows: out[r][o] = act(sum_i in[r][i] * W[o][i] + b[o]), rounded to bf16.
template <int NIN, int NOUT>
__device__ __forceinline__ void fwd_layer(const float *W, const float *b, const float *in, float *out, bool relu) {
    for (int e = threadIdx.x; e < kTrainRows * NOUT; e += blockDim.x) {
        const int r = e / NOUT, o = e % NOUT;
        float a = 0.0f;
#pragma unroll 8
        for (int i = 0; i < NIN; i++) a += in[r * NIN + i] * W[o * NIN + i];
        a += b[o];
        out[e] = relu ? bf16_round(fmaxf(a, 0.0f)) : a;
    }
}

// grad W[o][i] += sum_r d[r][o] * in[r][i]; grad b[o] += sum_r d[r][o]
template <int NIN, int NOUT>
__device__ __forceinline__ void grad_w(const float *d, const float *in, float *gW, float *gb) {
    for (int e = threadIdx.x; e < NOUT * NIN; e += blockDim.x) {
        const int o = e / NIN, i = e % NIN;
        float a = 0.0f;
        for (int r = 0; r < kTrainRows; r++) a += d[r * NOUT + o] * in[r * NIN + i];
        atomicAdd(&gW[e], a);
    }
    for (int o = threadIdx.x; o < NOUT; o += blockDim.x) {
        float a = 0.0f;
        for (int r = 0; r < kTrainRows; r++) a += d[r * NOUT + o];
        atomicAdd(&gb[o], a);
    }
}

// d_in[r][i] = (sum_o d[r][o] * W[o][i]) * (act[r][i] > 0)
template <int NIN, int NOUT>
__device__ __forceinline__ void back_act(const float *d, const float *W, const float *act, float *din) {
    for (int e = threadIdx.x; e < kTrainRows * NIN; e += blockDim.x) {
        const int r = e / NIN, i = e % NIN;
        float a = 0.0f;
#pragma unroll 8
        for (int o = 0; o < NOUT; o++) a += d[r * NOUT + o] * W[o * NIN + i];
        din[e] = act[e] > 0.0f ? a : 0.0f;
    }
}

// One minibatch slice of 64 rows per CTA: forward (bf16-rounded like inference),
// MSE loss over the 4 outputs, backward, gradients accumulated into `grad`.
__global__ void __launch_bounds__(kTrainThreads) k_train_step(const float *params, const float *x, const float *y,
                                                             int rows, float inv_count, float *grad, float *loss) {
    extern __shared__ float ts[];
    const int r0 = blockIdx.x * kTrainRows;
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
        const bool is_weight = !(i >= oB1 && i < oW2) && !(i >= oB2 && i < oW3) && !(i >= oB3 && i < oW4) && i < oB4;
        ts[tW + i] = is_weight ? bf16_round(params[i]) : params[i];
    }
    for (int e = threadIdx.x; e < kTrainRows * kIn; e += blockDim.x) {
        const int r = e / kIn, k = e % kIn;
        ts[tX + e] = r0 + r < rows ? bf16_round(x[size_t(r0 + r) * kRowStride + k]) : 0.0f;
    }
    __syncthreads();
    const float *W = ts + tW;
    fwd_layer<kIn, kH>(W + oW1, W + oB1, ts + tX, ts + tH1, true);
    __syncthreads();
    fwd_layer<kH, kH>(W + oW2, W + oB2, ts + tH1, ts + tH2, true);
    __syncthreads();
    fwd_layer<kH, kH>(W + oW3, W + oB3, ts + tH2, ts + tH3, true);
    __syncthreads();
    // output layer, loss and its gradient
    float lsum = 0.0f;
    for (int e = threadIdx.x; e < kTrainRows * kOut; e += blockDim.x) {
        const int r = e / kOut, o = e % kOut;
        float a = W[oB4 + o];
        for (int i = 0; i < kH; i++) a += ts[tH3 + r * kH + i] * W[oW4 + o * kH + i];
        float dy = 0.0f;
        if (r0 + r < rows) {
            const float err = a - y[size_t(r0 + r) * 4 + o];
            lsum += err * err * inv_count;
            dy = 2.0f * err * inv_count;
        }
        ts[tDY + e] = dy;
    }
    atomicAdd(loss, lsum);
    __syncthreads();
    grad_w<kH, kOut>(ts + tDY, ts + tH3, grad + oW4, grad + oB4);
    back_act<kH, kOut>(ts + tDY, W + oW4, ts + tH3, ts + tDA);
    __syncthreads();
    grad_w<kH, kH>(ts + tDA, ts + tH2, grad + oW3, grad + oB3);
    back_act<kH, kH>(ts + tDA, W + oW3, ts + tH2, ts + tDB);
    __syncthreads();
    grad_w<kH, kH>(ts + tDB, ts + tH1, grad + oW2, grad + oB2);
    back_act<kH, kH>(ts + tDB, W + oW2, ts + tH1, ts + tDA);
    __syncthreads();
    grad_w<kIn, kH>(ts + tDA, ts + tX, grad + oW1, grad + oB1);
}

__global__ void k_adam(float *p, float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1 - b1) * gi;
    const float vi = b2 * v[i] + (1 - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.0f;
}

// ---------------------------------------------------------------------------
// Render integration
// ---------------------------------------------------------------------------

struct FilmSurrogate {
    Range rg;
    float lam_lo, lam_hi, cos_lo, cos_hi, d_lo, d_hi, nf_lo, nf_hi, ns_lo, ns_hi;
};

// Inside the trained range, the grazing region where the render takes the exact
// transfer matrix because the network's error concentrates there.
__device__ __forceinline__ bool grazing_exact(float cos_theta, float n_sub) {
    return cos_theta < LAMBDA_SURROGATE_GRAZING_COS ||
           (n_sub < LAMBDA_SURROGATE_LOW_SUB_INDEX && cos_theta < LAMBDA_SURROGATE_LOW_SUB_COS);
}

// Thin-film shade with the surrogate, step 1 of 3 (k_film_encode, k_mlp_tc,
// k_film_scatter): for thin-film hit i of the bounce, the film thickness and the
// four hero-wavelength queries (lambda, cos, thickness, n_film, n_sub), encoded as
// MLP input rows 4i .. 4i + 3, and whether the surrogate's domain covers the hit.
// The domain is a single film with real indices between air (index exactly 1) and
// a substrate inside the trained box. A back-face hit (light inside the substrate)
// is mapped to the equivalent incidence from air by Snell's law, since a lossless
// stack reflects the same from both sides. Hits outside the domain or in its
// grazing region (grazing_exact), and back-face hits past the critical angle (where the transfer matrix of material.h:263-309
// does not return the physical R = 1), are left to the exact FP32 transfer matrix
// in step 3; their rows are zeros.
__global__ void __launch_bounds__(256) k_film_encode(int bounce, RenderParams rp, DeviceScene sc, PathState ps,
                                                     FilmSurrogate fs, float *__restrict__ rows,
                                                     uint8_t *__restrict__ in_domain) {
    const int n = ps.counts[queue_slot(bounce, kQFilm)];
    const int *q = ps.mat_queue[2];
    const int stride = gridDim.x * blockDim.x;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride) {
        const int p = q[idx];
        const ShadeIn s = load_shade(ps, sc, p);
        bool ok = s.m.y == 1;
        const float d = ok ? scalar_texture(sc, sc.material_props[s.m.w], s.sp.point) : 0.0f;
        const float cos_in = dot(s.nrm, -s.d);
        ok = ok && d >= fs.d_lo && d <= fs.d_hi;
        float e[kHero][kIn];
#pragma unroll
        for (int w = 0; w < kHero; w++) {
            const float lam = s.lam.v[w];
            const double2 a = cspectrum_at(sc, sc.material_props[s.m.z], lam);
            const double2 b = cspectrum_at(sc, sc.material_props[s.m.z + 1], lam);
            const double2 c = cspectrum_at(sc, sc.material_props[s.m.z + 2], lam);
            const float nf = float(b.x), ns = float(c.x);
            float c0 = cos_in;
            if (!s.front) {
                const float sin2 = ns * ns * (1 - cos_in * cos_in);
                ok = ok && sin2 < 1.0f;
                c0 = sqrtf(fmaxf(1 - sin2, 0.0f));
            }
            ok = ok && a.x == 1.0 && a.y == 0.0 && b.y == 0.0 && c.y == 0.0 && nf >= fs.nf_lo && nf <= fs.nf_hi &&
                 ns >= fs.ns_lo && ns <= fs.ns_hi && c0 >= fs.cos_lo && c0 <= fs.cos_hi && lam >= fs.lam_lo &&
                 lam <= fs.lam_hi && !grazing_exact(c0, ns);
            const float v[kIn] = {lam, c0, d, nf, ns};
            encode(v, fs.rg, e[w]);
        }
        float4 *r = reinterpret_cast<float4 *>(rows + size_t(idx) * (kHero * kRowStride));
#pragma unroll
        for (int w = 0; w < kHero; w++) {
            r[2 * w] = ok ? make_float4(e[w][0], e[w][1], e[w][2], e[w][3]) : make_float4(0, 0, 0, 0);
            r[2 * w + 1] = make_float4(ok ? e[w][4] : 0.0f, 0, 0, 0);
        }
        in_domain[idx] = ok ? 1 : 0;
    }
}

// Step 3: each hit's reflectance (R_s + R_p) / 2 at its four wavelengths from the
// MLP's outputs (or, outside the domain, the exact FP32 transfer matrix), then the
// thin-film scatter (material.h:228-261) and Russian roulette.
__global__ void __launch_bounds__(256, 3) k_film_scatter(int bounce, RenderParams rp, DeviceScene sc, PathState ps,
                                                         const float4 *__restrict__ out,
                                                         const uint8_t *__restrict__ in_domain) {
    const int n = ps.counts[queue_slot(bounce, kQFilm)];
    const int *q = ps.mat_queue[2];
    int *q_next = ps.queue[(bounce + 1) & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int idx = base + threadIdx.x;
        const bool valid = idx < n;
        bool alive = false, ok = false;
        int p = 0;
        if (valid) {
            p = q[idx];
            const ShadeIn s = load_shade(ps, sc, p);
            const float4 ff = __ldg(&sc.film_flat[s.mat]);
            ok = in_domain[idx] != 0;
            s4 R;
            if (ok) {
#pragma unroll
                for (int w = 0; w < kHero; w++) {
                    const float4 y = out[size_t(idx) * kHero + w];
                    R.v[w] = clampf((y.x + y.y) * 0.5f, 0.0f, 1.0f);
                }
            } else {
                float thick[kMaxFilmLayers];
                thin_film_thickness(sc, s, thick);
                R = thin_film_r4(sc, s.m, s.front, dot(s.nrm, -s.d), s.lam, thick, ff);
            }
            Rng rng = path_rng(ps, p);
            s4 att;
            f3 nd;
            thin_film_scatter(sc, s, R, rng, att, nd, ff);
            alive = finish_scatter(ps, s, rng, bounce, att, nd, 0, true);
        }
        const int slot = warp_push(&ps.counts[queue_slot(bounce + 1, kQActive)], alive);
        if (alive) q_next[slot] = p;
        warp_push(&ps.counts[queue_slot(bounce, kQFilmFallback)], valid && !ok);
    }
}

// Host: the FP32 parameters as the BF16 shared-memory image of the MLP kernels
// (weights in their operand layouts, each bias as a (hi, lo) pair of BF16 columns).
void pack_weights(const float *p, std::vector<uint8_t> &packed) {
    packed.assign(kPackedWeightBytes, 0);
    auto put = [&](int region, int K, int r, int k, float v) {
        const __nv_bfloat16 b = __float2bfloat16_rn(v);
        std::memcpy(&packed[region + core_offset(r, k, K)], &b, 2);
    };
    auto put_bias = [&](int region, int K, int r, int k, float v) {
        const float hi = __bfloat162float(__float2bfloat16_rn(v));
        put(region, K, r, k, hi);
        put(region, K, r, k + 1, v - hi);
    };
    for (int o = 0; o < kH; o++) {
        for (int i = 0; i < kIn; i++) put(sW1, kInPad, o, i, p[oW1 + o * kIn + i]);
        put_bias(sW1, kInPad, o, kIn, p[oB1 + o]);
    }
    for (int o = 0; o < kH; o++) {
        for (int i = 0; i < kH; i++) {
            put(sW2, kH, o, i, p[oW2 + o * kH + i]);
            put(sW3, kH, o, i, p[oW3 + o * kH + i]);
        }
        put_bias(sB2, 8, o, 0, p[oB2 + o]);
        put_bias(sB3, 8, o, 0, p[oB3 + o]);
    }
    for (int o = 0; o < kOut; o++) {
        for (int i = 0; i < kH; i++) put(sW4, kH, o, i, p[oW4 + o * kH + i]);
        put_bias(sB4, 8, o, 0, p[oB4 + o]);
    }
}

Range to_range(const lambda_film_range &r) {
    Range g;
    const float *src[kIn] = {r.lambda_nm, r.cos_theta, r.thickness_nm, r.n_film, r.n_sub};
    for (int k = 0; k < kIn; k++) {
        g.lo[k] = src[k][0];
        g.hi[k] = src[k][1];
    }
    return g;
}

bool range_ok(const lambda_film_range &r) {
    const float *src[kIn] = {r.lambda_nm, r.cos_theta, r.thickness_nm, r.n_film, r.n_sub};
    for (int k = 0; k < kIn; k++)
        if (!(src[k][1] > src[k][0]) || !std::isfinite(src[k][0]) || !std::isfinite(src[k][1])) return false;
    return r.n_film[0] > 0 && r.n_sub[0] > 0 && r.cos_theta[0] >= 0 && r.cos_theta[1] <= 1 && r.lambda_nm[0] > 0 &&
           r.thickness_nm[0] >= 0;
}

// Dynamic shared memory of the MLP kernels (below the 48 KB default today; set so
// that a larger layout needs no other change).
cudaError_t configure_mlp_kernels() {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMlpSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMlpSmem);
    return e;
}

// Grid of the MLP kernel for `tiles` 128-row tiles: one CTA per SM (each allocates
// all 512 TMEM columns), or fewer when there are fewer tiles than chains.
int mlp_grid(int64_t tiles, int sm_count) {
    return int(std::max<int64_t>(1, std::min<int64_t>((tiles + kChains - 1) / kChains, sm_count)));
}

}  // namespace mlp

using namespace mlp;

#define CK(call, what)                                          \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return ctx->cuda_fail(e_, what); \
    } while (0)

lambda_status lambda_ctx::surrogate_ready() {
    if (!has_surrogate)
        return fail(LAMBDA_ERR_INVALID_ARGUMENT, "no surrogate installed (lambda_surrogate_train or lambda_surrogate_set)");
    lambda_ctx *ctx = this;
    CK(configure_mlp_kernels(), "configure MLP kernels");
    return LAMBDA_OK;
}

namespace {

// Installs FP32 parameters: the master copy and the packed BF16 image.
lambda_status install(lambda_ctx *ctx, const float *params_host, const lambda_film_range &r) {
    std::vector<uint8_t> packed;
    pack_weights(params_host, packed);
    SurrogateBuffers &b = ctx->sbuf;
    CK(b.weights_f32.upload(params_host, kParams * sizeof(float), ctx->stream), "upload surrogate");
    CK(b.weights_bf16.reserve(packed.size()), "upload surrogate");
    CK(cudaMemcpyAsync(b.weights_bf16.ptr, packed.data(), packed.size(), cudaMemcpyHostToDevice, ctx->stream), "upload surrogate");
    CK(cudaStreamSynchronize(ctx->stream), "upload surrogate");
    ctx->surrogate_range = r;
    ctx->has_surrogate = true;
    return LAMBDA_OK;
}

// Runs the MLP over n_rows encoded rows (kQueries = false) or film queries
// (kQueries = true) on the context's stream and waits for it.
template <bool kQueries>
lambda_status run_mlp(lambda_ctx *ctx, const void *in, int n_rows, float4 *out_dev) {
    CK(configure_mlp_kernels(), "configure MLP kernels");
    CK(ctx->rbuf.error.reserve(16), "allocate flags");
    int *err = ctx->rbuf.error.as<int>();
    CK(cudaMemsetAsync(err, 0, 16, ctx->stream), "clear flags");
    const uint8_t *w = static_cast<const uint8_t *>(ctx->sbuf.weights_bf16.ptr);
    const int tiles = (n_rows + kTileM - 1) / kTileM;
    k_mlp_tc<kQueries><<<mlp_grid(tiles, ctx->sm_count), kMlpThreads, kMlpSmem, ctx->stream>>>(
        reinterpret_cast<const uint4 *>(w), in, n_rows, to_range(ctx->surrogate_range), out_dev, err,
        ctx->limits.mma_polls);
    CK(cudaGetLastError(), "launch MLP kernel");
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, ctx->stream), "read flags");
    CK(cudaStreamSynchronize(ctx->stream), "MLP inference");
    if (herr & 2) return ctx->fail(LAMBDA_ERR_TIMEOUT, "tensor-core MMA completion wait timed out");
    return LAMBDA_OK;
}

}  // namespace

int lambda_ctx::launch_shade_surrogate(int bounce, const RenderParams &rp, const DeviceScene &sc, const PathState &ps,
                                       StageProfiler *prof, cudaStream_t s) {
    FilmSurrogate fs;
    fs.rg = to_range(surrogate_range);
    fs.lam_lo = surrogate_range.lambda_nm[0];
    fs.lam_hi = surrogate_range.lambda_nm[1];
    fs.cos_lo = surrogate_range.cos_theta[0];
    fs.cos_hi = surrogate_range.cos_theta[1];
    fs.d_lo = surrogate_range.thickness_nm[0];
    fs.d_hi = surrogate_range.thickness_nm[1];
    fs.nf_lo = surrogate_range.n_film[0];
    fs.nf_hi = surrogate_range.n_film[1];
    fs.ns_lo = surrogate_range.n_sub[0];
    fs.ns_hi = surrogate_range.n_sub[1];
    const uint4 *w = static_cast<const uint4 *>(sbuf.weights_bf16.ptr);
    float *rows = rbuf.film_rows.as<float>();
    float4 *out = rbuf.film_out.as<float4>();
    uint8_t *in_domain = rbuf.film_in_domain.as<uint8_t>();
    // grids for the pass's largest thin-film queue, one hit per pixel
    const int64_t hits = std::max(1, rp.num_pixels);
    auto grid = [&](int per_sm, int block) {
        return int(std::max<int64_t>(1, std::min<int64_t>((hits + block - 1) / block, int64_t(per_sm) * sm_count)));
    };
    const int64_t tiles = (hits * kHero + kTileM - 1) / kTileM;
    if (prof) prof->begin(9);
    k_film_encode<<<grid(film_encode_ctas, 256), 256, 0, s>>>(bounce, rp, sc, ps, fs, rows, in_domain);
    if (prof) prof->end();
    if (prof) prof->begin(10);
    k_mlp_tc<false><<<mlp_grid(tiles, sm_count), kMlpThreads, kMlpSmem, s>>>(
        w, rows, 0, Range{}, out, ps.error, limits.mma_polls, ps.counts + queue_slot(bounce, kQFilm), kHero);
    if (prof) prof->end();
    if (prof) prof->begin(11);
    k_film_scatter<<<grid(film_scatter_ctas, 256), 256, 0, s>>>(bounce, rp, sc, ps, out, in_domain);
    if (prof) prof->end();
    return 3;
}

// Kernel attributes, grids and the path-state buffers of the surrogate's render
// kernels for `pixels` paths, set up before any stream capture.
lambda_status lambda_ctx::ensure_surrogate_state(int pixels) {
    lambda_ctx *ctx = this;
    CK(configure_mlp_kernels(), "configure MLP kernels");
    if (mlp_ctas_per_sm <= 0) {
        mlp_ctas_per_sm = 1;  // each CTA holds all 512 TMEM columns of its SM
        film_encode_ctas = resident_ctas((const void *)k_film_encode, device, 256, 0);
        film_scatter_ctas = resident_ctas((const void *)k_film_scatter, device, 256, 0);
    }
    const size_t P = size_t(std::max(pixels, 1));
    CK(rbuf.film_rows.reserve(P * kHero * kRowStride * sizeof(float)), "allocate surrogate rows");
    CK(rbuf.film_out.reserve(P * kHero * sizeof(float4)), "allocate surrogate rows");
    CK(rbuf.film_in_domain.reserve(P), "allocate surrogate rows");
    return LAMBDA_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" lambda_status lambda_surrogate_set(lambda_ctx *ctx, const float *params, const lambda_film_range *range) {
    if (!ctx || !params || !range) return LAMBDA_ERR_INVALID_ARGUMENT;
    if (!range_ok(*range)) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "invalid surrogate input range");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    std::vector<float> p(kParams);
    if (is_device_pointer(params)) CK(cudaMemcpy(p.data(), params, kParams * 4, cudaMemcpyDeviceToHost), "read parameters");
    else std::memcpy(p.data(), params, kParams * 4);
    for (float v : p)
        if (!std::isfinite(v)) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "non-finite surrogate parameter");
    return install(ctx, p.data(), *range);
}

extern "C" lambda_status lambda_surrogate_get(const lambda_ctx *cctx, float *params, lambda_film_range *range) {
    if (!cctx || !params) return LAMBDA_ERR_INVALID_ARGUMENT;
    lambda_ctx *ctx = const_cast<lambda_ctx *>(cctx);
    if (!ctx->has_surrogate) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "no surrogate installed");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaMemcpy(params, ctx->sbuf.weights_f32.ptr, kParams * 4, cudaMemcpyDeviceToHost), "read parameters");
    if (range) *range = ctx->surrogate_range;
    return LAMBDA_OK;
}

extern "C" lambda_status lambda_surrogate_eval(lambda_ctx *ctx, const lambda_film_query *q, int32_t n, float *out) {
    if (!ctx || n < 0 || (n > 0 && (!q || !out))) return LAMBDA_ERR_INVALID_ARGUMENT;
    if (!ctx->has_surrogate) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "no surrogate installed");
    if (n == 0) return LAMBDA_OK;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    Staging sg{ctx, {}};
    CopyBack back;
    const lambda_film_query *dq;
    float *dout;
    CK(sg.in(q, size_t(n), &dq), "stage queries");
    CK(sg.out(out, size_t(n) * 4, &dout, back), "stage results");
    lambda_status st = run_mlp<true>(ctx, dq, n, reinterpret_cast<float4 *>(dout));
    if (st != LAMBDA_OK) return st;
    return finish_staging(ctx, back);
}

namespace {

void init_params(std::vector<float> &p, uint64_t seed) {
    p.assign(kParams, 0.0f);
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
    auto uni = [&]() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return double(s >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    auto fill = [&](int off, int fan_out, int fan_in, double gain) {
        const double a = gain * std::sqrt(6.0 / fan_in);
        for (int i = 0; i < fan_out * fan_in; i++) p[off + i] = float(a * uni());
    };
    fill(oW1, kH, kIn, 1.0);
    fill(oW2, kH, kH, 1.0);
    fill(oW3, kH, kH, 1.0);
    fill(oW4, kOut, kH, 0.5);
}

}  // namespace

extern "C" lambda_status lambda_surrogate_train(lambda_ctx *ctx, const lambda_train_desc *desc,
                                                lambda_train_report *report) {
    if (!ctx || !desc) return LAMBDA_ERR_INVALID_ARGUMENT;
    const lambda_train_desc &d = *desc;
    if (d.samples < kTrainRows || d.samples > (int64_t(1) << 28) || d.epochs < 1 || d.batch < kTrainRows ||
        d.batch % kTrainRows != 0 || !(d.learning_rate > 0) || !range_ok(d.range))
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "invalid training settings");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    const Range rg = to_range(d.range);
    const int64_t N = d.samples;
    const int audit_n = 1 << 18;
    DeviceBuffer x, y, ax, ay, params, grad, m, v, loss, aout;
    CK(x.reserve(size_t(N) * kRowStride * 4), "allocate training set");
    CK(y.reserve(size_t(N) * 16), "allocate training set");
    CK(ax.reserve(size_t(audit_n) * kRowStride * 4), "allocate audit set");
    CK(ay.reserve(size_t(audit_n) * 16), "allocate audit set");
    CK(aout.reserve(size_t(audit_n) * 16), "allocate audit set");
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaEventRecord(e0, st);
    for (int64_t first = 0; first < N; first += (1 << 22)) {
        const int chunk = int(std::min<int64_t>(1 << 22, N - first));
        k_film_labels<<<(chunk + 255) / 256, 256, 0, st>>>(d.seed, first, chunk, rg, x.as<float>() + first * kRowStride,
                                                          y.as<float>() + first * 4);
    }
    k_film_labels<<<(audit_n + 255) / 256, 256, 0, st>>>(d.seed ^ 0xA5A5A5A5A5A5ull, 0, audit_n, rg, ax.as<float>(),
                                                        ay.as<float>());
    CK(cudaGetLastError(), "launch label kernel");
    cudaEventRecord(e1, st);

    std::vector<float> p;
    init_params(p, d.seed);
    CK(params.upload(p.data(), kParams * 4, st), "upload parameters");
    CK(grad.reserve(kParams * 4), "allocate gradients");
    CK(m.reserve(kParams * 4), "allocate optimiser state");
    CK(v.reserve(kParams * 4), "allocate optimiser state");
    CK(loss.reserve(64), "allocate loss");
    CK(cudaMemsetAsync(grad.ptr, 0, kParams * 4, st), "clear gradients");
    CK(cudaMemsetAsync(m.ptr, 0, kParams * 4, st), "clear optimiser state");
    CK(cudaMemsetAsync(v.ptr, 0, kParams * 4, st), "clear optimiser state");
    CK(cudaFuncSetAttribute(k_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem), "configure training kernel");
    const int64_t steps_per_epoch = (N + d.batch - 1) / d.batch;
    const int64_t total = steps_per_epoch * d.epochs;
    int64_t t = 0;
    float last_loss = 0;
    for (int ep = 0; ep < d.epochs; ep++) {
        CK(cudaMemsetAsync(loss.ptr, 0, 4, st), "clear loss");
        for (int64_t s = 0; s < steps_per_epoch; s++, t++) {
            const int64_t r0 = s * d.batch;
            const int rows = int(std::min<int64_t>(d.batch, N - r0));
            const int blocks = (rows + kTrainRows - 1) / kTrainRows;
            k_train_step<<<blocks, kTrainThreads, kTrainSmem, st>>>(params.as<float>(), x.as<float>() + r0 * kRowStride,
                                                                   y.as<float>() + r0 * 4, rows,
                                                                   1.0f / float(rows * kOut), grad.as<float>(),
                                                                   loss.as<float>());
            // cosine decay to 2% of the base rate
            const double frac = double(t) / double(std::max<int64_t>(1, total - 1));
            const float lr = float(d.learning_rate * (0.02 + 0.98 * 0.5 * (1 + std::cos(3.14159265358979 * frac))));
            const float c1 = float(1 - std::pow(0.9, double(t + 1))), c2 = float(1 - std::pow(0.999, double(t + 1)));
            k_adam<<<(kParams + 255) / 256, 256, 0, st>>>(params.as<float>(), grad.as<float>(), m.as<float>(),
                                                         v.as<float>(), kParams, lr, 0.9f, 0.999f, 1e-8f, c1, c2);
        }
        CK(cudaGetLastError(), "launch training kernels");
        float h = 0;
        CK(cudaMemcpyAsync(&h, loss.ptr, 4, cudaMemcpyDeviceToHost, st), "read loss");
        CK(cudaStreamSynchronize(st), "training");
        last_loss = h / float(steps_per_epoch);
    }
    cudaEventRecord(e2, st);
    CK(cudaMemcpyAsync(p.data(), params.ptr, kParams * 4, cudaMemcpyDeviceToHost, st), "read parameters");
    CK(cudaStreamSynchronize(st), "training");
    lambda_status s = install(ctx, p.data(), d.range);
    if (s != LAMBDA_OK) return s;
    // audit: tensor-core inference against the FP64 labels
    s = run_mlp<false>(ctx, ax.as<float>(), audit_n, aout.as<float4>());
    if (s != LAMBDA_OK) return s;
    std::vector<float> got(size_t(audit_n) * 4), want(size_t(audit_n) * 4);
    CK(cudaMemcpy(got.data(), aout.ptr, got.size() * 4, cudaMemcpyDeviceToHost), "read audit");
    CK(cudaMemcpy(want.data(), ay.ptr, want.size() * 4, cudaMemcpyDeviceToHost), "read audit");
    double mx = 0, mean = 0;
    for (size_t i = 0; i < got.size(); i++) {
        const double e = std::fabs(double(got[i]) - double(want[i]));
        mx = std::max(mx, e);
        mean += e;
    }
    mean /= double(got.size());
    if (report) {
        float lab = 0, tr = 0;
        cudaEventElapsedTime(&lab, e0, e1);
        cudaEventElapsedTime(&tr, e1, e2);
        report->label_ms = lab;
        report->train_ms = tr;
        report->final_loss = last_loss;
        report->max_abs_error = float(mx);
        report->mean_abs_error = float(mean);
        report->audit_samples = audit_n;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    for (DeviceBuffer *b : {&x, &y, &ax, &ay, &params, &grad, &m, &v, &loss, &aout}) b->release();
    return LAMBDA_OK;
}

// One training-kernel forward/backward on caller data (for gradient checks):
// x [n][5] encoded inputs, y [n][4] targets, n <= 64 * 1024; writes the mean
// squared error and its gradient w.r.t. params.
extern "C" lambda_status lambda_surrogate_grad(lambda_ctx *ctx, const float *params, const float *x, const float *y,
                                               int32_t n, float *grad_out, float *loss_out) {
    if (!ctx || !params || !x || !y || !grad_out || n <= 0 || n > (64 << 10)) return LAMBDA_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    std::vector<float> rows(size_t(n) * kRowStride, 0.0f);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < kIn; k++) rows[size_t(i) * kRowStride + k] = x[size_t(i) * kIn + k];
    DeviceBuffer dp, dx, dy, dg, dl;
    CK(dp.upload(params, kParams * 4, ctx->stream), "stage");
    CK(dx.upload(rows.data(), rows.size() * 4, ctx->stream), "stage");
    CK(dy.upload(y, size_t(n) * 16, ctx->stream), "stage");
    CK(dg.reserve(kParams * 4), "stage");
    CK(dl.reserve(16), "stage");
    CK(cudaMemsetAsync(dg.ptr, 0, kParams * 4, ctx->stream), "stage");
    CK(cudaMemsetAsync(dl.ptr, 0, 16, ctx->stream), "stage");
    CK(cudaFuncSetAttribute(k_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem), "configure training kernel");
    k_train_step<<<(n + kTrainRows - 1) / kTrainRows, kTrainThreads, kTrainSmem, ctx->stream>>>(
        dp.as<float>(), dx.as<float>(), dy.as<float>(), n, 1.0f / float(n * kOut), dg.as<float>(), dl.as<float>());
    CK(cudaGetLastError(), "launch training kernel");
    CK(cudaMemcpyAsync(grad_out, dg.ptr, kParams * 4, cudaMemcpyDeviceToHost, ctx->stream), "read gradient");
    float l = 0;
    CK(cudaMemcpyAsync(&l, dl.ptr, 4, cudaMemcpyDeviceToHost, ctx->stream), "read loss");
    CK(cudaStreamSynchronize(ctx->stream), "gradient");
    if (loss_out) *loss_out = l;
    for (DeviceBuffer *b : {&dp, &dx, &dy, &dg, &dl}) b->release();
    return LAMBDA_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free surrogate evaluation.
//
// Some callers cannot call cudaMalloc at the point where they evaluate films: a
// host renderer whose device memory belongs to its own pool allocator (a game
// engine, a DCC plug-in host) and whose render thread must not allocate, because
// cudaMalloc can synchronise the device and can fail under the host's memory
// budget. For them, lambda_surrogate_eval_static takes caller-owned device
// buffers and keeps its only scratch, the encoded network inputs, in a fixed
// array compiled into this library: kStaticMaxQueries queries (4 MiB), held by
// every GPU that loads the library until the process exits. The array is shared
// by all calls and keeps the last call's contents; calls that overlap on the GPU
// (other streams, other threads, other contexts on the same device) race on it.
// The first call on a device (and the first after a device reset) looks up the
// array's device address, which can load this library's GPU module and so
// allocate: make that call once as a warm-up, outside the region that must not
// allocate and before any stream capture.
// ---------------------------------------------------------------------------

namespace {

constexpr int kStaticMaxQueries = LAMBDA_SURROGATE_STATIC_MAX_QUERIES;
static_assert(kStaticMaxQueries == 131072, "header and library disagree");

static __device__ __align__(256) float g_static_rows[kStaticMaxQueries * mlp::kRowStride];
static __device__ __align__(256) int g_static_error[4];

// Device addresses of the two arrays, looked up once per device and CUDA context.
// In host code the array names are host-side stand-ins, never device addresses.
struct StaticScratch {
    float *rows = nullptr;
    int *error = nullptr;
    unsigned long long context_id = 0;  // the context the addresses belong to
    bool ready = false;
};
constexpr int kMaxDevices = 64;
StaticScratch g_static_scratch[kMaxDevices];
std::mutex g_static_mutex;

// Unique id of the calling thread's current CUDA context (cuCtxGetCurrent and
// cuCtxGetId, reached through the runtime's driver entry points so the library
// needs no link to libcuda), or 0 when the driver cannot tell. A device reset
// destroys the primary context and the next one gets a new id; the module is then
// loaded again at new addresses.
unsigned long long current_context_id() {
    using GetCurrent = int (*)(void **);
    using GetId = int (*)(void *, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    if (!get_current || !get_id) return 0;
    void *c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != 0 || !c || get_id(c, &id) != 0) return 0;
    return id;
}

lambda_status static_scratch(lambda_ctx *ctx, StaticScratch &out) {
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "device index too large");
    std::lock_guard<std::mutex> lock(g_static_mutex);
    StaticScratch &s = g_static_scratch[ctx->device];
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");  // the lookup is per device: this device must be current
    const unsigned long long id = current_context_id();
    // an unknown id (0) never matches, so the addresses are looked up again on every call
    if (!s.ready || id == 0 || id != s.context_id) {
        void *rows = nullptr, *err = nullptr;
        CK(cudaGetSymbolAddress(&rows, g_static_rows), "look up the static scratch array");
        CK(cudaGetSymbolAddress(&err, g_static_error), "look up the static error word");
        s.rows = static_cast<float *>(rows);
        s.error = static_cast<int *>(err);
        s.context_id = id;
        s.ready = true;
    }
    out = s;
    return LAMBDA_OK;
}

// Whether a caller-owned buffer can be read or written by this context's kernels:
// device memory of the context's GPU, or managed memory.
bool buffer_on_context_device(const void *p, int device) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return lambda_host::buffer_usable_on(int(a.type), a.device, device);
}

__global__ void k_encode_queries(const lambda_film_query *q, int n, mlp::Range rg, float *rows) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v[mlp::kIn] = {q[i].lambda_nm, q[i].cos_theta, q[i].thickness_nm, q[i].n_film, q[i].n_sub};
    float e[mlp::kIn];
    mlp::encode(v, rg, e);
    float *row = rows + size_t(i) * mlp::kRowStride;
    reinterpret_cast<float4 *>(row)[0] = make_float4(e[0], e[1], e[2], e[3]);
    reinterpret_cast<float4 *>(row)[1] = make_float4(e[4], 0.0f, 0.0f, 0.0f);
}

}  // namespace

extern "C" lambda_status lambda_surrogate_eval_static(lambda_ctx *ctx, const lambda_film_query *queries, int32_t n,
                                                      float *out) {
    if (!ctx) return LAMBDA_ERR_INVALID_ARGUMENT;
    if (n < 0 || n > kStaticMaxQueries)
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT,
                         "lambda_surrogate_eval_static: n must be in [0, 131072] (LAMBDA_SURROGATE_STATIC_MAX_QUERIES); "
                         "split larger batches into several calls");
    if (!ctx->has_surrogate) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "no surrogate installed");
    if (n == 0) return LAMBDA_OK;
    if (!queries || !out || !buffer_on_context_device(queries, ctx->device) ||
        !buffer_on_context_device(out, ctx->device))
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT,
                         "lambda_surrogate_eval_static takes device pointers only, on the context's own GPU "
                         "(or managed memory)");
    if (reinterpret_cast<uintptr_t>(out) % 16 != 0)
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "lambda_surrogate_eval_static: out must be 16-byte aligned");
    StaticScratch sc;
    lambda_status st = static_scratch(ctx, sc);  // leaves the context's device current
    if (st != LAMBDA_OK) return st;
    CK(configure_mlp_kernels(), "configure MLP kernels");
    CK(cudaMemsetAsync(sc.error, 0, sizeof(int) * 4, ctx->stream), "clear the static error word");
    k_encode_queries<<<(n + 255) / 256, 256, 0, ctx->stream>>>(queries, n, to_range(ctx->surrogate_range), sc.rows);
    const uint8_t *w = static_cast<const uint8_t *>(ctx->sbuf.weights_bf16.ptr);
    const int tiles = (n + kTileM - 1) / kTileM;
    k_mlp_tc<false><<<mlp_grid(tiles, ctx->sm_count), kMlpThreads, kMlpSmem, ctx->stream>>>(
        reinterpret_cast<const uint4 *>(w), sc.rows, n, Range{}, reinterpret_cast<float4 *>(out), sc.error,
        ctx->limits.mma_polls);
    CK(cudaGetLastError(), "launch MLP kernel");
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, sc.error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "read the static error word");
    CK(cudaStreamSynchronize(ctx->stream), "MLP inference");
    if (herr & 2) return ctx->fail(LAMBDA_ERR_TIMEOUT, "tensor-core MMA completion wait timed out");
    return LAMBDA_OK;
}
