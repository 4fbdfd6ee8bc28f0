// Merged-index contractions of the reference's extended bucket backend
// (CMKLExtendedBackend, qtensor/ProcessingFrameworks.py:41-147), whose
// native dependency ``tcontract`` (an MKL C extension) is absent from the
// reference:
//
//   qtb_contract_outer_c64  c[n,m,k] = a[n,m] * b[n,k]          (mkl_contract_complex, :60-66)
//   qtb_contract_sum_c64    C[f,m,n] = sum_k A[k,f,m] * B[k,f,n] (mkl_contract_sum, :123-130)
//
// complex64 in and out.  The contract-sum is a batch of F complex GEMMs; with
// a large summed dimension it runs on the tcgen05 tensor cores:
//   * a pre-pass splits every operand into TF32 "hi" (rounded to nearest,
//     cvt.rna.tf32.f32) and "lo" (the rounded remainder) planes of the real
//     and imaginary parts, transposed to K-major and tiled 128 (or 64) rows
//     x 16 k in the canonical no-swizzle core-matrix layout (8 rows x 16
//     bytes), zero padded to whole 32-k blocks;
//   * one CTA per (f, 128 x 64 output tile): one lane stages the eight
//     planes of each 16-k tile (8 KB of A, 4 KB of B each) into one of two
//     shared-memory stages with bulk copies (cp.async.bulk, mbarrier
//     transaction count, bounded wait), and issues tcgen05.mma kind::tf32
//     (M=128, N=64, K=8) into Re and Im accumulators in TMEM, FP32, while
//     the next tile's copy lands:
//       Re += Ar_hi Br_hi + Ar_hi Br_lo + Ar_lo Br_hi - (Ai_hi Bi_hi + Ai_hi Bi_lo + Ai_lo Bi_hi)
//       Im += Ar_hi Bi_hi + Ar_hi Bi_lo + Ar_lo Bi_hi + Ai_hi Br_hi + Ai_hi Br_lo + Ai_lo Br_hi
//     (3xTF32: Ootomo and Yokota, "Recovering single precision accuracy from
//     Tensor Cores while surpassing the FP32 theoretical peak performance",
//     IJHPCA 2022; the lo x lo term is dropped), the negative terms through
//     the instruction descriptor's negate-A bit;
//   * every 32-k block goes to one of two TMEM buffers from zero; four warps
//     read a finished buffer back (tcgen05.ld) and add it into FP32
//     registers with round-to-nearest while the next block fills the other
//     buffer, since the tensor cores' own accumulation rounds toward zero
//     (Ootomo and Yokota keep the long sum outside the tensor cores for the
//     same reason); the registers are written as complex64.
// With a small summed dimension (the reference's own buckets sum one binary
// index, K = 2) a tile would be mostly padding, and a CUDA-core kernel
// computes the same sums in FP32.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "plan.h"

namespace qtb {

// ----------------------------------------------------------------- CUDA cores
// c[n,m,k] = a[n,m] * b[n,k], one element per thread (grid-stride).
__global__ void qtb_outer_kernel(const float2* __restrict__ a, const float2* __restrict__ b,
                                 float2* __restrict__ c, uint64_t n, uint64_t m, uint64_t k) {
    const uint64_t total = n * m * k;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t kk = i % k, mm = (i / k) % m, nn = i / (k * m);
        const float2 x = a[nn * m + mm], y = b[nn * k + kk];
        c[i] = make_float2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
    }
}

// C[f,m,n] = sum_k A[k,f,m] B[k,f,n], one output per thread, FP32 sums
// over k in order.
__global__ void qtb_contract_simt_kernel(const float2* __restrict__ A, const float2* __restrict__ B,
                                         float2* __restrict__ C, uint64_t K, uint64_t F, uint64_t M,
                                         uint64_t N) {
    const uint64_t total = F * M * N;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t nn = i % N, mm = (i / N) % M, ff = i / (N * M);
        float re = 0.f, im = 0.f;
        for (uint64_t kk = 0; kk < K; ++kk) {
            const float2 x = A[(kk * F + ff) * M + mm], y = B[(kk * F + ff) * N + nn];
            re = fmaf(x.x, y.x, re);
            re = fmaf(-x.y, y.y, re);
            im = fmaf(x.x, y.y, im);
            im = fmaf(x.y, y.x, im);
        }
        C[i] = make_float2(re, im);
    }
}

// ----------------------------------------------------------------- tensor cores
constexpr uint32_t kTcM = 128;                        // output tile rows (A tile rows)
constexpr uint32_t kTcN = 64;                         // output tile columns (complex)
constexpr uint32_t kTcBRows = 2 * kTcN;               // B tile rows: [Br | Bi] or [-Bi | Br]
constexpr uint32_t kTcK = 32;                         // k per accumulation block (K padded to it)
constexpr uint32_t kTcStageK = 8;                     // k per staged tile (one MMA k step)
constexpr uint32_t kTcStages = 3;                     // shared-memory stages (two copies in flight)
constexpr uint32_t kTcStagesPerBlock = kTcK / kTcStageK;
constexpr uint32_t kTcAWords = kTcM * kTcStageK;      // 1024 x 32-bit = 4 KB per A plane and stage
constexpr uint32_t kTcBWords = kTcBRows * kTcStageK;  // 1024 x 32-bit = 4 KB per B plane and stage
constexpr uint32_t kTcPlanes = 4;                     // A: re_hi re_lo im_hi im_lo; B: B1_hi B1_lo B2_hi B2_lo
constexpr uint32_t kTcStageWords = kTcPlanes * (kTcAWords + kTcBWords);   // 32 KB per stage
constexpr uint32_t kTcChunks = kTcStageK / 4;         // 16-byte k chunks per row of a tile
constexpr uint32_t kTcEpilogueWarps = 4;              // one per 32 TMEM lanes of the 128-row tile
constexpr uint32_t kTcThreads = 32 * (kTcEpilogueWarps + 1);   // + the copy/MMA issuing warp
constexpr uint32_t kTcBufCols = 2 * kTcN;             // one accumulator buffer: Re 0..63, Im 64..127
constexpr uint32_t kTcTmemCols = 2 * kTcBufCols;      // two buffers
constexpr uint32_t kTcSpinLimit = 1u << 24;           // bounded mbarrier waits (~1 s)
constexpr int kTcStatusTimeout = 2;

// Word of element (r, k) inside a tile of kTcStageK k: core matrix (row
// group r / 8, k chunk k / 4) at (g * kTcChunks + c) * 32 words, 8 rows of
// 16 bytes each.
__device__ __forceinline__ uint32_t tc_tile_word(uint32_t r, uint32_t k) {
    return (((r >> 3) * kTcChunks + (k >> 2)) << 5) + ((r & 7u) << 2) + (k & 3u);
}

__device__ __forceinline__ uint32_t tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// TF32 hi / lo of one component: hi rounded to nearest, lo the rounded remainder.
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
    hi = tf32_round(x);
    lo = tf32_round(x - __uint_as_float(hi));
}

// Copies a staged tile (`words` 32-bit words) from shared memory to dst, 16 bytes per thread and step.
__device__ __forceinline__ void tc_write_tile(const uint32_t* s, uint32_t* dst, uint32_t words) {
    const uint4* in = reinterpret_cast<const uint4*>(s);
    uint4* out = reinterpret_cast<uint4*>(dst);
    for (uint32_t i = threadIdx.x; i < words / 4; i += blockDim.x) out[i] = in[i];
}

// A[k][f][m] (complex64, M rows) -> TF32 planes Ar_hi, Ar_lo, Ai_hi, Ai_lo
// in tiles of 128 rows x kTcStageK k, ordered (f, row tile, k tile), each
// tile's four planes consecutive, so that one bulk copy stages all four.
// One block per tile: coalesced reads of the tile's rows, the split into
// shared memory in the core-matrix layout, then one contiguous write.
__global__ void __launch_bounds__(256) qtb_tc_split_kernel(const float2* __restrict__ src,
                                                           uint32_t* __restrict__ dst, uint32_t K, uint32_t F,
                                                           uint32_t M, uint32_t Mp, uint32_t Kp) {
    __shared__ __align__(16) uint32_t s[kTcPlanes * kTcAWords];
    const uint32_t k_tiles = Kp / kTcStageK, row_tiles = Mp / kTcM;
    const uint32_t bid = blockIdx.x;
    const uint32_t kt = bid % k_tiles, rt = (bid / k_tiles) % row_tiles, f = bid / (k_tiles * row_tiles);
    for (uint32_t e = threadIdx.x; e < kTcM * kTcStageK; e += blockDim.x) {
        const uint32_t r = e % kTcM, k = e / kTcM;
        const uint32_t m = rt * kTcM + r, kk = kt * kTcStageK + k;
        const float2 v = (m < M && kk < K) ? src[((uint64_t)kk * F + f) * M + m] : make_float2(0.f, 0.f);
        uint32_t rh, rl, ih, il;
        tf32_split(v.x, rh, rl);
        tf32_split(v.y, ih, il);
        const uint32_t w = tc_tile_word(r, k);
        s[w] = rh;
        s[kTcAWords + w] = rl;
        s[2 * kTcAWords + w] = ih;
        s[3 * kTcAWords + w] = il;
    }
    __syncthreads();
    tc_write_tile(s, dst + (uint64_t)bid * kTcPlanes * kTcAWords, kTcPlanes * kTcAWords);
}

// B[k][f][n] (complex64, N columns) -> TF32 planes B1_hi, B1_lo, B2_hi,
// B2_lo in tiles of 128 rows x kTcStageK k, ordered (f, output column
// tile, k tile), each tile's four planes consecutive: in the rows of tile
// t, B1 holds Br of columns 64 t .. 64 t + 63 then their Bi, and B2 holds
// -Bi then Br (the negation is exact in TF32).  One block per tile, as for A.
__global__ void __launch_bounds__(256) qtb_tc_split_b_kernel(const float2* __restrict__ src,
                                                             uint32_t* __restrict__ dst, uint32_t K, uint32_t F,
                                                             uint32_t N, uint32_t Np, uint32_t Kp) {
    __shared__ __align__(16) uint32_t s[kTcPlanes * kTcBWords];
    const uint32_t k_tiles = Kp / kTcStageK, col_tiles = Np / kTcN;
    const uint32_t bid = blockIdx.x;
    const uint32_t kt = bid % k_tiles, t = (bid / k_tiles) % col_tiles, f = bid / (k_tiles * col_tiles);
    for (uint32_t e = threadIdx.x; e < kTcN * kTcStageK; e += blockDim.x) {
        const uint32_t j = e % kTcN, k = e / kTcN;
        const uint32_t n = t * kTcN + j, kk = kt * kTcStageK + k;
        const float2 v = (n < N && kk < K) ? src[((uint64_t)kk * F + f) * N + n] : make_float2(0.f, 0.f);
        uint32_t rh, rl, ih, il;
        tf32_split(v.x, rh, rl);
        tf32_split(v.y, ih, il);
        const uint32_t w_re = tc_tile_word(j, k);          // row j: Br (B1), -Bi (B2)
        const uint32_t w_im = tc_tile_word(j + kTcN, k);   // row 64 + j: Bi (B1), Br (B2)
        s[w_re] = rh;
        s[kTcBWords + w_re] = rl;
        s[w_im] = ih;
        s[kTcBWords + w_im] = il;
        s[2 * kTcBWords + w_re] = ih ^ 0x80000000u;
        s[3 * kTcBWords + w_re] = il ^ 0x80000000u;
        s[2 * kTcBWords + w_im] = rh;
        s[3 * kTcBWords + w_im] = rl;
    }
    __syncthreads();
    tc_write_tile(s, dst + (uint64_t)bid * kTcPlanes * kTcBWords, kTcPlanes * kTcBWords);
}

__device__ __forceinline__ uint32_t tc_smem(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor of a K-major, no-swizzle operand tile:
// start address, leading byte offset (next 16-byte k chunk: 128 B), stride
// byte offset (next 8-row group: kTcChunks chunks x 128 B), version 1.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
           ((uint64_t)(kTcChunks * 128u >> 4) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor: FP32 accumulator, TF32 A and B, both K-major,
// N = 64 (>> 3 at bit 17), M = 128 (>> 4 at bit 24); bit 13 negates A.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((kTcBRows >> 3) << 17) | ((kTcM >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// Bounded wait for the mbarrier phase `parity`; false after the limit.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
    uint32_t done = 0;
    for (uint32_t it = 0; it < kTcSpinLimit; ++it) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

// Eight 32-bit TMEM columns of this thread's lane at each of two
// addresses, one wait for both loads; the wait is in the same asm as the
// loads, so no use of the registers can be scheduled before it.
__device__ __forceinline__ void tc_ld2x8(uint32_t ta, uint32_t tb, float* a, float* b) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%16];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8,%9,%10,%11,%12,%13,%14,%15}, [%17];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(ta), "r"(tb)
        : "memory");
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        a[j] = __uint_as_float(r[j]);
        b[j] = __uint_as_float(r[8 + j]);
    }
}

__device__ __forceinline__ void tc_bulk(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// One CTA per (f, 128 x 64 tile of C), five warps.  Ap / Bp: the pre-pass
// planes, in tiles of kTcStageK k.
//   * Warp 4 (one elected lane) stages tiles with bulk copies into
//     kTcStages shared-memory stages, kTcStages - 1 tiles ahead of the
//     MMAs it issues, so that copies land while earlier tiles' MMAs run.
//     kTcStagesPerBlock tiles make one 32-k block, accumulated in one of two
//     TMEM buffers from zero.
//   * Warps 0-3 (one per 32 TMEM lanes) read a finished block's buffer
//     with tcgen05.ld and add it into FP32 registers with round-to-nearest
//     (the tensor cores' own accumulation rounds toward zero, which over a
//     long k range biases the sum: about 3e-5 relative at K = 1000), while
//     the next block's MMAs fill the other buffer.
// mbarriers: full[s] (stage s landed), empty[s] (stage s's MMAs done),
// tfull[b] (buffer b's block done), tempty[b] (buffer b read, 128
// arrivals).  Every wait is bounded; on a timeout the status word is set,
// every role stops, and the CTA waits (bounded, in phase order) for its
// copies and MMAs in flight before freeing TMEM.
__global__ void __launch_bounds__(kTcThreads, 2)
qtb_tc_contract_kernel(const uint32_t* __restrict__ Ap, const uint32_t* __restrict__ Bp, float2* __restrict__ C,
                       uint32_t F, uint32_t M, uint32_t N, uint32_t Mp, uint32_t Np, uint32_t Kp, int* status) {
    constexpr uint32_t NS = kTcStages;
    extern __shared__ __align__(1024) unsigned char smem[];
    // [stage 0: A planes x4 | B planes x4][stage 1] ..., the mbarriers, the TMEM slot
    uint32_t* stages = reinterpret_cast<uint32_t*>(smem);
    uint64_t* bars = reinterpret_cast<uint64_t*>(stages + NS * kTcStageWords);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * NS + 4);
    __shared__ volatile int s_ok;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t nt = blockIdx.x, mt = blockIdx.y, f = blockIdx.z;
    auto full = [&](uint32_t s) { return tc_smem(&bars[s]); };
    auto empty = [&](uint32_t s) { return tc_smem(&bars[NS + s]); };
    auto tfull = [&](uint32_t b) { return tc_smem(&bars[2 * NS + b]); };
    auto tempty = [&](uint32_t b) { return tc_smem(&bars[2 * NS + 2 + b]); };
    if (threadIdx.x == 0) {
        for (uint32_t i = 0; i < 2 * NS + 2; ++i)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bars[i])));
        for (uint32_t b = 0; b < 2; ++b)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tempty(b)), "r"(32 * kTcEpilogueWarps));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_ok = 1;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(tmem_slot)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;
    const uint32_t n_tiles = Kp / kTcStageK, n_blocks = Kp / kTcK;
    auto fail_once = [&]() {
        if (s_ok) atomicOr(status, kTcStatusTimeout);
        s_ok = 0;
    };
    if (warp == kTcEpilogueWarps) {
        if (lane == 0) {
            // this CTA's tiles: (f, row tile, k tile) of A, (f, column tile, k tile) of B
            const uint32_t* a_f = Ap + ((uint64_t)f * (Mp / kTcM) + mt) * n_tiles * (kTcPlanes * kTcAWords);
            const uint32_t* b_f = Bp + ((uint64_t)f * (Np / kTcN) + nt) * n_tiles * (kTcPlanes * kTcBWords);
            auto stage_a = [&](uint32_t s) { return tc_smem(stages + s * kTcStageWords); };
            auto stage_b = [&](uint32_t s) { return tc_smem(stages + s * kTcStageWords + kTcPlanes * kTcAWords); };
            auto load = [&](uint32_t i) {   // tile i into stage i % NS
                const uint32_t s = i % NS;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full(s)),
                             "r"(kTcStageWords * 4u)
                             : "memory");
                // the tile's four planes are consecutive in global memory and in the stage
                tc_bulk(stage_a(s), a_f + (uint64_t)i * kTcPlanes * kTcAWords, kTcPlanes * kTcAWords * 4u, full(s));
                tc_bulk(stage_b(s), b_f + (uint64_t)i * kTcPlanes * kTcBWords, kTcPlanes * kTcBWords * 4u, full(s));
            };
            uint32_t loaded = 0, landed = 0;   // tiles whose copies were issued, waited for
            uint32_t committed[NS] = {}, retired[NS] = {};   // empty[s] phases issued, waited for
            for (; loaded < NS - 1 && loaded < n_tiles; ++loaded) load(loaded);
            for (uint32_t i = 0; i < n_tiles && s_ok; ++i) {
                const uint32_t s = i % NS, b = i / kTcStagesPerBlock, buf = b & 1u;
                const bool block_first = i % kTcStagesPerBlock == 0;
                if (block_first && b >= 2 && !tc_wait(tempty(buf), ((b - 2) >> 1) & 1u)) {
                    fail_once();   // the epilogue has not read this buffer's previous block
                    break;
                }
                if (!tc_wait(full(s), (i / NS) & 1u)) {
                    fail_once();
                    break;
                }
                landed = i + 1;
                asm volatile("tcgen05.fence::after_thread_sync;");
                // planes: A 0 Ar_hi 1 Ar_lo 2 Ai_hi 3 Ai_lo | B 0 B1_hi 1 B1_lo 2 B2_hi 3 B2_lo with
                // B1 = [Br | Bi] and B2 = [-Bi | Br] along N, so that
                // Ar B1 + Ai B2 = [Re | Im] in the buffer's 128 columns
                const uint32_t abase = stage_a(s), bbase = stage_b(s);
                const uint32_t acc = tmem + buf * kTcBufCols;
#pragma unroll
                for (uint32_t ks = 0; ks < kTcStageK / 8; ++ks) {
                    auto da = [&](uint32_t q) { return tc_desc(abase + q * kTcAWords * 4u + ks * 256u); };
                    auto db = [&](uint32_t q) { return tc_desc(bbase + q * kTcBWords * 4u + ks * 256u); };
                    const uint32_t first = (block_first && ks == 0) ? 0u : 1u;   // a block starts from zero
                    tc_mma(acc, da(0), db(0), kTcIdesc, first);
                    tc_mma(acc, da(0), db(1), kTcIdesc, 1u);
                    tc_mma(acc, da(1), db(0), kTcIdesc, 1u);
                    tc_mma(acc, da(2), db(2), kTcIdesc, 1u);
                    tc_mma(acc, da(2), db(3), kTcIdesc, 1u);
                    tc_mma(acc, da(3), db(2), kTcIdesc, 1u);
                }
                tc_commit(empty(s));
                ++committed[s];
                if (i % kTcStagesPerBlock == kTcStagesPerBlock - 1) tc_commit(tfull(buf));
                // tile i + NS - 1 goes into the stage of tile i - 1 once that
                // tile's MMAs are done; it lands while later tiles' MMAs run
                if (loaded < n_tiles) {
                    if (i >= 1) {
                        const uint32_t sp = (i - 1) % NS;
                        if (!tc_wait(empty(sp), ((i - 1) / NS) & 1u)) {
                            fail_once();
                            break;
                        }
                        ++retired[sp];
                    }
                    load(loaded++);
                }
            }
            // nothing of this CTA may still write shared memory or TMEM when
            // it frees them: wait (bounded, in phase order) for the copies
            // issued and not waited for, and for every MMA commit
            for (uint32_t i = landed; i < loaded; ++i) tc_wait(full(i % NS), (i / NS) & 1u);
            for (uint32_t q = 0; q < NS; ++q)
                for (uint32_t u = retired[q]; u < committed[q]; ++u) tc_wait(empty(q), u & 1u);
        }
        __syncwarp();
    } else {
        float acc_re[kTcN], acc_im[kTcN];
#pragma unroll
        for (uint32_t j = 0; j < kTcN; ++j) acc_re[j] = acc_im[j] = 0.f;
        const uint32_t lane_addr = tmem + ((warp * 32u) << 16);   // this warp's 32 TMEM lanes
        for (uint32_t b = 0; b < n_blocks; ++b) {
            const uint32_t buf = b & 1u;
            if (!s_ok) break;
            if (!tc_wait(tfull(buf), (b >> 1) & 1u)) {
                fail_once();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (uint32_t c0 = 0; c0 < kTcN; c0 += 8u) {
                float vr[8], vi[8];
                tc_ld2x8(lane_addr + buf * kTcBufCols + c0, lane_addr + buf * kTcBufCols + kTcN + c0, vr, vi);
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j) {
                    acc_re[c0 + j] += vr[j];
                    acc_im[c0 + j] += vi[j];
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tempty(buf)) : "memory");
        }
        if (s_ok) {
            const uint32_t m = mt * kTcM + warp * 32u + lane;
            if (m < M) {
                float2* crow = C + ((uint64_t)f * M + m) * N;
#pragma unroll
                for (uint32_t j = 0; j < kTcN; ++j) {
                    const uint32_t n = nt * kTcN + j;
                    if (n < N) crow[n] = make_float2(acc_re[j], acc_im[j]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
}

constexpr size_t kTcSmemBytes = kTcStages * kTcStageWords * 4 + (2 * kTcStages + 4) * 8 + 16;

static uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

// Whether the contract-sum runs on the tensor cores: mode 1 never, 2
// always, 0 when the summed dimension and both tile dimensions are large
// enough for the tiles to be mostly data.
static bool use_tensor_cores(int32_t mode, int64_t K, int64_t M, int64_t N) {
    if (mode == 1) return false;
    if (mode == 2) return true;
    return K >= 32 && M >= 64 && N >= 64;
}

static int cuda_fail_c(cudaError_t e, const char* what) {
    return fail(QTB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace qtb

using namespace qtb;

extern "C" {

int qtb_contract_outer_c64(const void* a, const void* b, void* c, int64_t n, int64_t m, int64_t k,
                           void* stream) {
    if (!a || !b || !c || n < 1 || m < 1 || k < 1) return fail(QTB_ERR_ARG, "contract_outer: bad arguments");
    const uint64_t total = (uint64_t)n * m * k;
    const unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 16);
    qtb_outer_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(a), static_cast<const float2*>(b), static_cast<float2*>(c), n, m, k);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QTB_OK : cuda_fail_c(e, "contract_outer launch");
}

int qtb_contract_sum_scratch_bytes(int64_t K, int64_t F, int64_t M, int64_t N, int32_t mode, size_t* bytes) {
    if (!bytes || K < 1 || F < 1 || M < 1 || N < 1 || mode < 0 || mode > 2)
        return fail(QTB_ERR_ARG, "contract_sum_scratch_bytes: bad arguments");
    if (!use_tensor_cores(mode, K, M, N)) {
        *bytes = 16;
        return QTB_OK;
    }
    const uint64_t Kp = round_up(K, kTcK), Mp = round_up(M, kTcM), Np = round_up(N, kTcN);
    *bytes = 256 + (uint64_t)F * kTcPlanes * (Mp + 2 * Np) * Kp * 4;   // B planes hold two rows per column
    return QTB_OK;
}

int qtb_contract_sum_c64(const void* A, const void* B, void* C, int64_t K, int64_t F, int64_t M, int64_t N,
                         int32_t mode, void* scratch, size_t scratch_bytes, void* stream) {
    if (!A || !B || !C || K < 1 || F < 1 || M < 1 || N < 1 || mode < 0 || mode > 2)
        return fail(QTB_ERR_ARG, "contract_sum: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    size_t need = 0;
    int r = qtb_contract_sum_scratch_bytes(K, F, M, N, mode, &need);
    if (r) return r;
    if (!scratch || scratch_bytes < need)
        return fail(QTB_ERR_ARG, "contract_sum: scratch smaller than qtb_contract_sum_scratch_bytes");
    cudaError_t e = cudaMemsetAsync(scratch, 0, 16, st);   // status word
    if (e != cudaSuccess) return cuda_fail_c(e, "contract_sum status reset");
    if (!use_tensor_cores(mode, K, M, N)) {
        const uint64_t total = (uint64_t)F * M * N;
        const unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 16);
        qtb_contract_simt_kernel<<<blocks, 256, 0, st>>>(static_cast<const float2*>(A),
                                                         static_cast<const float2*>(B), static_cast<float2*>(C),
                                                         K, F, M, N);
        e = cudaGetLastError();
        return e == cudaSuccess ? QTB_OK : cuda_fail_c(e, "contract_sum launch");
    }
    const uint64_t Kp = round_up(K, kTcK), Mp = round_up(M, kTcM), Np = round_up(N, kTcN);
    if (Mp / kTcM > 65535 || F > 65535 || Np / kTcN > (1u << 31) || Kp > (1u << 30) ||
        (uint64_t)F * (Mp / kTcM) * (Kp / kTcStageK) >= (1ull << 31) ||
        (uint64_t)F * (Np / kTcN) * (Kp / kTcStageK) >= (1ull << 31))
        return fail(QTB_ERR_UNSUPPORTED, "contract_sum: shape beyond the tensor-core grid");
    int* status = static_cast<int*>(scratch);
    uint32_t* Ap = reinterpret_cast<uint32_t*>(static_cast<char*>(scratch) + 256);
    uint32_t* Bp = Ap + (uint64_t)F * kTcPlanes * Mp * Kp;
    const uint32_t k_tiles = (uint32_t)(Kp / kTcStageK);
    qtb_tc_split_kernel<<<(unsigned)(F * (Mp / kTcM) * k_tiles), 256, 0, st>>>(
        static_cast<const float2*>(A), Ap, (uint32_t)K, (uint32_t)F, (uint32_t)M, (uint32_t)Mp, (uint32_t)Kp);
    qtb_tc_split_b_kernel<<<(unsigned)(F * (Np / kTcN) * k_tiles), 256, 0, st>>>(
        static_cast<const float2*>(B), Bp, (uint32_t)K, (uint32_t)F, (uint32_t)N, (uint32_t)Np, (uint32_t)Kp);
    // per device and cheap: set on every call
    e = cudaFuncSetAttribute(qtb_tc_contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kTcSmemBytes);
    if (e != cudaSuccess) return cuda_fail_c(e, "contract_sum smem attribute");
    dim3 grid((unsigned)(Np / kTcN), (unsigned)(Mp / kTcM), (unsigned)F);
    qtb_tc_contract_kernel<<<grid, kTcThreads, kTcSmemBytes, st>>>(Ap, Bp, static_cast<float2*>(C), (uint32_t)F,
                                                                  (uint32_t)M, (uint32_t)N, (uint32_t)Mp,
                                                                  (uint32_t)Np, (uint32_t)Kp, status);
    e = cudaGetLastError();
    return e == cudaSuccess ? QTB_OK : cuda_fail_c(e, "contract_sum launch");
}

}  // extern "C"
