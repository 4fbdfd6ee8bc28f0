// Device code and the device-facing C ABI of libqtb.so (sm_100a).
//
//   K1  qtb_bucket_kernel    one bucket of BucketBackend.process_bucket
//                            (qtensor/ProcessingFrameworks.py:29-31,45-147):
//                            product of the bucket's tensors over the sorted
//                            union of their variables, summed over variable 0
//   K3  qtb_network_kernel   a whole edge network (bucket_elimination,
//                            Simulate.py:90-94) per CTA: the gate tensors
//                            generated from the request's angles (qtree gate
//                            tensors, OpFactory.py:44-58), the buckets in
//                            dependency phases with intermediates in shared
//                            memory (a per-CTA global arena in the
//                            allocation-free run), and in the last CTA to
//                            finish the fp64 Neumaier sum of the edge terms
//                            with the MaxCut post-processing
//                            (QAOASimulator.py:27-41); class, persistent,
//                            lean-persistent and hybrid schedules
//   K4  qtb_wide_kernel      networks too large for shared memory, in waves
//                            contracted by the whole GPU one elimination
//                            phase at a time (tile queue, bounded waits)
//   K0  qtb_table_kernel     the gate table in global memory, for plans whose
//                            table does not fit in shared memory and for
//                            wide waves
//   qtb_energy_kernel        the energy of a plain (per-bucket) run
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "plan.h"

namespace qtb {

// ----------------------------------------------------------------- helpers
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Parallel bit extract: the bits of x selected by m, packed from bit 0 up.
__device__ __forceinline__ uint32_t pext32(uint32_t x, uint32_t m) {
    uint32_t r = 0;
    for (uint32_t bit = 1; m; bit <<= 1) {
        const uint32_t low = m & (0u - m);
        if (x & low) r |= bit;
        m ^= low;
    }
    return r;
}

// Operand offset of output index j (bits below the summed bit) from the
// precompiled runs of DevIn; falls back to the bit loop for masks of more
// than kMaxRuns runs.
__device__ __forceinline__ uint32_t gather_bits(uint32_t j, const DevIn& d, uint32_t low_mask) {
    const uint32_t n = (uint32_t)(d.runs >> 60);
    if (n <= 1u) return (j >> ((uint32_t)(d.runs >> 32) & 31u)) & (uint32_t)d.runs;
    if (n == (uint32_t)kRunsFallback) return pext32(j, d.mask & low_mask);
    uint32_t off = 0, dst = 0;
#pragma unroll
    for (uint32_t r = 0; r < (uint32_t)kMaxRuns; ++r) {
        if (r < n) {
            const uint32_t rr = (uint32_t)(d.runs >> (10 * r)) & 0x3ffu;
            const uint32_t start = rr & 31u, len = rr >> 5;
            off |= ((j >> start) & ((1u << len) - 1u)) << dst;
            dst += len;
        }
    }
    return off;
}

// ----------------------------------------------------------------- K1
// Operand t of output element j: the bits of j its mask selects, gathered by
// the precompiled runs (mask, runs as in DevIn), and with the summed
// variable set, `stride[t]` further (the summed variable is the operand's
// most significant axis; stride 0 when the operand does not hold it).
struct BucketArgs {
    const float2* in[QTB_MAX_BUCKET_INPUTS];
    uint64_t runs[QTB_MAX_BUCKET_INPUTS];
    uint32_t mask[QTB_MAX_BUCKET_INPUTS];
    uint32_t stride[QTB_MAX_BUCKET_INPUTS];
    float2* out;
    int32_t k;
    int32_t w;     // output variables
    int32_t sum;
};

// Each thread contracts up to kBucketBatch output elements, one grid width
// apart (so every load stays coalesced across the warp; a bucket smaller
// than the grid gives each thread one element), operand by operand: all their
// gathers are in flight together, which a bandwidth-bound bucket needs to
// keep enough bytes moving per SM.  The operand descriptors are copied to
// shared memory once per block, so the operand loop reads them with a
// runtime index without holding all sixteen slots in registers.  Each
// element's product folds its operands left to right, as one element at a
// time would.
constexpr int kBucketBatch = 4;
constexpr int kBucketThreads = 256;

__global__ void __launch_bounds__(kBucketThreads) qtb_bucket_kernel(const BucketArgs a) {
    __shared__ const float2* s_in[QTB_MAX_BUCKET_INPUTS];
    __shared__ uint64_t s_runs[QTB_MAX_BUCKET_INPUTS];
    __shared__ uint32_t s_mask[QTB_MAX_BUCKET_INPUTS], s_stride[QTB_MAX_BUCKET_INPUTS];
    if (threadIdx.x < (uint32_t)a.k) {
        s_in[threadIdx.x] = a.in[threadIdx.x];
        s_runs[threadIdx.x] = a.runs[threadIdx.x];
        s_mask[threadIdx.x] = a.mask[threadIdx.x];
        s_stride[threadIdx.x] = a.sum ? a.stride[threadIdx.x] : 0u;
    }
    __syncthreads();
    // 32-bit indices: at most 2^31 outputs (QTB_MAX_BUCKET_VARS), and
    // base + kBucketBatch grid widths stays below 2^32
    const uint32_t n_out = 1u << a.w;
    const uint32_t low = n_out - 1u;
    const uint32_t grid = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + threadIdx.x; base < n_out; base += grid * kBucketBatch) {
        float2 p0[kBucketBatch], p1[kBucketBatch];
#pragma unroll 1
        for (int t = 0; t < a.k; ++t) {
            DevIn d;
            d.mask = s_mask[t];
            d.src = 0;
            d.runs = s_runs[t];
            const float2* __restrict__ in = s_in[t];
            const uint32_t stride = s_stride[t];
            float2 x0[kBucketBatch], x1[kBucketBatch];
#pragma unroll
            for (int i = 0; i < kBucketBatch; ++i) {
                const uint32_t jj = base + i * grid;
                x0[i] = x1[i] = make_float2(0.f, 0.f);
                if (jj < n_out) {
                    const uint32_t off = gather_bits(jj, d, low);
                    x0[i] = in[off];
                    x1[i] = stride ? in[off + stride] : x0[i];
                }
            }
#pragma unroll
            for (int i = 0; i < kBucketBatch; ++i) {
                p0[i] = t == 0 ? x0[i] : cmul(p0[i], x0[i]);
                p1[i] = t == 0 ? x1[i] : cmul(p1[i], x1[i]);
            }
        }
#pragma unroll
        for (int i = 0; i < kBucketBatch; ++i) {
            const uint32_t jj = base + i * grid;
            if (jj < n_out) a.out[jj] = a.sum ? make_float2(p0[i].x + p1[i].x, p0[i].y + p1[i].y) : p0[i];
        }
    }
}

// Grid of a bucket launch over 2^w outputs: one thread per element up to
// eight blocks for each of the 148 SMs; larger buckets give every thread up
// to kBucketBatch elements per pass of the grid-stride loop.
static unsigned bucket_blocks(int32_t w) {
    return (unsigned)std::min<uint64_t>(((1ull << w) + kBucketThreads - 1) / kBucketThreads, 148ull * 8);
}

// Gathers of operand t of a bucket over n_vars variables (variable 0 at
// mask bit n_vars - 1, summed when sum_first).
static void bucket_operand(BucketArgs* a, int t, uint32_t mask, int n_vars, int sum_first) {
    const uint32_t w = (uint32_t)(n_vars - sum_first);
    a->mask[t] = mask;
    a->runs[t] = encode_runs(mask, w);
    a->stride[t] = (sum_first && ((mask >> w) & 1u)) ? 1u << (__builtin_popcount(mask) - 1) : 0u;
}

// ----------------------------------------------------------------- K0
// Element of a gate tensor at native index bits: axis a <-> bit a of ixb.
__device__ double2 gate_value(int kind, double alpha, uint32_t ixb) {
    const double r2 = 0.70710678118654752440;
    const int ix[3] = {(int)(ixb & 1u), (int)((ixb >> 1) & 1u), (int)((ixb >> 2) & 1u)};
    double s, c;
    switch (kind) {
        case QTB_GATE_M: return make_double2(ix[0] == ix[1] ? 1.0 : 0.0, 0.0);
        case QTB_GATE_H: return make_double2((ix[0] & ix[1]) ? -r2 : r2, 0.0);
        case QTB_GATE_X: return make_double2(ix[0] != ix[1] ? 1.0 : 0.0, 0.0);
        case QTB_GATE_Y:
            if (ix[0] == ix[1]) return make_double2(0.0, 0.0);
            return make_double2(0.0, ix[0] == 0 ? -1.0 : 1.0);
        case QTB_GATE_Z: return make_double2(ix[0] ? -1.0 : 1.0, 0.0);
        case QTB_GATE_T: return ix[0] ? make_double2(r2, r2) : make_double2(1.0, 0.0);
        case QTB_GATE_CX: {
            const bool on = ix[0] ? (ix[1] != ix[2]) : (ix[1] == ix[2]);
            return make_double2(on ? 1.0 : 0.0, 0.0);
        }
        case QTB_GATE_CZ: return make_double2((ix[0] & ix[1]) ? -1.0 : 1.0, 0.0);
        case QTB_GATE_ZPHASE:
            if (!ix[0]) return make_double2(1.0, 0.0);
            sincospi(alpha, &s, &c);
            return make_double2(c, s);
        case QTB_GATE_ZZ:
            sincospi(alpha * 0.5, &s, &c);
            return ix[0] == ix[1] ? make_double2(c, -s) : make_double2(c, s);
        case QTB_GATE_XPHASE:
        case QTB_GATE_YPHASE: {
            double gs, gc;
            sincospi(alpha * 0.5, &s, &c);   // cos/sin(pi alpha / 2); also the phase g
            gc = c;
            gs = s;
            double2 m;
            if (kind == QTB_GATE_XPHASE) {
                m = ix[0] == ix[1] ? make_double2(c, 0.0) : make_double2(0.0, -s);
            } else {
                m = ix[0] == ix[1] ? make_double2(c, 0.0)
                                   : make_double2(ix[0] == 0 ? -s : s, 0.0);
            }
            return make_double2(gc * m.x - gs * m.y, gc * m.y + gs * m.x);
        }
        default: return make_double2(0.0, 0.0);
    }
}

// Fill one gate-table entry: the gate tensor for alpha = sum coef*param,
// with its sliced axes fixed to 0 and the rest transposed to sorted order.
__device__ void table_entry(const DevEntry& en, const DevTerm* terms, const double* params,
                            float2* table) {
    double alpha = 0.0;
    for (int t = 0; t < en.expr_count; ++t)
        alpha += terms[en.expr_begin + t].coef * params[terms[en.expr_begin + t].param];
    const int n = 1 << en.rank_out;
    for (int o = 0; o < n; ++o) {
        uint32_t ixb = en.sliced_value;   // sliced axes at their values
        for (int a = 0; a < en.rank_out; ++a)
            ixb |= (uint32_t)((o >> (en.rank_out - 1 - a)) & 1) << en.perm[a];
        const double2 v = gate_value(en.kind, alpha, ixb);
        table[en.off + o] = make_float2((float)v.x, (float)v.y);
    }
}

__global__ void qtb_table_kernel(const DevEntry* entries, int n_entries, const DevTerm* terms,
                                 const double* params, float2* table) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_entries; e += gridDim.x * blockDim.x)
        table_entry(entries[e], terms, params, table);
}

// ----------------------------------------------------------------- K3
// A network of a launch: its run descriptor inline (one load locates
// everything the executor needs) and where its edge term goes.
struct Job {
    DevNetRun net;
    float2* term;
    uint64_t pad;
};
static_assert(sizeof(Job) == 64, "Job layout");

// Arguments shared by every CTA of one run (all size classes).
struct RunArgs {
    const uint4* blobs;           // network blobs
    const uint4* common;          // [DevEntry x n_entries, padded to 16 B][DevTerm ...]
    uint32_t common_bytes;        // multiple of 16
    uint32_t n_entries;
    uint32_t terms_off;           // byte offset of the DevTerm array in common
    uint32_t table_elems;
    const double* params;
    const uint32_t* recs;         // element records, or null: this launch reads plan blobs only
    uint32_t recs_bytes;          // of the plan's whole record array
    uint32_t runs_bytes;          // of the plan's DevNetRun array
    const DevNetRun* runs;
    const float2* gtable;         // global gate table (kernels without a shared table)
    float2* gscratch;             // global arenas (kernels without a shared arena)
    uint32_t arena_capacity;      // elements per CTA
    uint32_t blob_capacity;       // bytes per CTA
    int* status;
    unsigned int* done;           // networks finished in this run (reset by the last one)
    unsigned int* queue;          // claims of a persistent launch (zeroed before it)
    uint32_t static_first;        // 1: a persistent CTA's first network is job blockIdx.x
    uint32_t n_jobs;              // jobs of this launch
    uint32_t total_jobs;          // networks of the run over all its launches
    const float2* terms;          // the run's edge terms, [total_jobs]
    double* energy;               // MaxCut energy of the run, or null
    double energy_groups;         // circuits (edge terms) of the run's networks
};

constexpr int kStatusArena = 1;        // network arena larger than the launch's capacity
constexpr int kStatusStageTimeout = 2; // a staging copy did not complete in time
constexpr int kStatusBlob = 4;         // network blob larger than the launch's capacity
constexpr int kStatusQueue = 8;        // persistent launch without a job queue
constexpr int kStatusWideTimeout = 16; // a wide-network step waited too long for its predecessor
constexpr uint32_t kStageSpinLimit = 1u << 25;   // about 1.5 s of polling

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// Bulk (TMA) copies global -> shared completing on the mbarrier's current
// phase (`parity`); every thread waits with a bounded spin.  Returns false
// (status word set) if the copies did not land.  stage_issue (one thread)
// starts the copies, stage_wait (every thread) waits for them, stage does
// both.
__device__ __forceinline__ void stage_issue(void* dst0, const void* src0, uint32_t bytes0, void* dst1,
                                            const void* src1, uint32_t bytes1, uint64_t* bar) {
    const uint32_t bar_a = smem_addr(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes0 + bytes1)
                 : "memory");
    if (bytes0) bulk_copy(dst0, src0, bytes0, bar_a);
    if (bytes1) bulk_copy(dst1, src1, bytes1, bar_a);
}

__device__ bool stage_wait(uint64_t* bar, uint32_t parity, int* status) {
    const uint32_t bar_a = smem_addr(bar);
    uint32_t done = 0;
    for (uint32_t it = 0; it < kStageSpinLimit; ++it) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(bar_a), "r"(parity) : "memory");
        if (done) break;
        if (it > 64) __nanosleep(32);
    }
    if (!done && threadIdx.x == 0) atomicOr(status, kStatusStageTimeout);
    return __syncthreads_and(done) != 0;
}

__device__ bool stage(void* dst0, const void* src0, uint32_t bytes0, void* dst1, const void* src1,
                      uint32_t bytes1, uint64_t* bar, uint32_t parity, int* status) {
    if (threadIdx.x == 0) stage_issue(dst0, src0, bytes0, dst1, src1, bytes1, bar);
    return stage_wait(bar, parity, status);
}

__device__ __forceinline__ void neumaier_add(double& sum, double& comp, double x) {
    const double t = sum + x;
    comp += fabs(sum) >= fabs(x) ? (sum - t) + x : (x - t) + sum;
    sum = t;
}

// Compensated fp64 sum of Re(terms) by one warp (all 32 lanes call it) in
// a fixed order -- lane l sums terms l, l + 32, ..., then a butterfly --
// then energy = (n_groups - sum) / 2.  The order does not depend on the
// launch shape, so every schedule gives the same energy for the same terms.
__device__ void reduce_energy_warp(const float2* terms, uint32_t n, double n_groups, double* energy) {
    constexpr uint32_t kBatch = 16;   // loads in flight per lane: one L2 round trip per 16 terms
    const uint32_t lane = threadIdx.x & 31u;
    double s = 0.0, c = 0.0;
    for (uint32_t base = lane; base < n; base += 32u * kBatch) {
        float x[kBatch];
#pragma unroll
        for (uint32_t j = 0; j < kBatch; ++j) x[j] = base + 32u * j < n ? __ldcg(&terms[base + 32u * j].x) : 0.f;
#pragma unroll
        for (uint32_t j = 0; j < kBatch; ++j)
            if (base + 32u * j < n) neumaier_add(s, c, (double)x[j]);
    }
    for (int off = 16; off > 0; off >>= 1) {
        const double os = __shfl_xor_sync(0xffffffffu, s, off);
        const double oc = __shfl_xor_sync(0xffffffffu, c, off);
        neumaier_add(s, c, os);
        neumaier_add(s, c, oc);
    }
    if (lane == 0) {
        *energy = (n_groups - (s + c)) * 0.5;
        // the energy may live in mapped host memory (a caller's pinned
        // buffer), read by the host once the kernel is done
        __threadfence_system();
    }
}

// The same by a whole CTA: its first warp sums, the others wait.
__device__ void reduce_energy(const float2* terms, uint32_t n, double n_groups, double* energy) {
    if (threadIdx.x < 32) reduce_energy_warp(terms, n, n_groups, energy);
    __syncthreads();
}

// The op of a phase holding flattened element g, starting from op `oi` at
// or before it (`op` holds ops[oi]).  The ops of a phase are sorted by
// non-increasing size, so jumping (g - start) >> w ops ahead never passes
// the op holding g (every op after oi has at most 2^w elements); a short
// walk over ops of smaller size finishes.  Returns the op index.
template <typename LoadOp>
__device__ __forceinline__ uint32_t find_op(uint32_t g, uint32_t oi, DevOp& op, LoadOp load) {
    const uint32_t jump = (g - op.elem_begin) >> (op.u - op.sum);
    if (jump) {
        oi += jump;
        op = load(oi);
    }
    while (g >= op.elem_begin + (1u << (op.u - op.sum))) op = load(++oi);
    return oi;
}

// The op of a phase holding element g: the last of ops lo..hi whose first
// element is at most g, by binary search (kGlobal: the ops are in global
// memory, read through the read-only path).  Networks whose arena cannot be
// in shared memory carry no chunk tables (DevPhase::chunk_off 0); their ops
// are found this way.
template <bool kGlobal>
__device__ __forceinline__ uint32_t search_op(const DevOp* ops, uint32_t lo, uint32_t hi, uint32_t g) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        const uint32_t first = kGlobal ? __ldg(&ops[mid].elem_begin) : ops[mid].elem_begin;
        if (first <= g) lo = mid;
        else hi = mid - 1u;
    }
    return lo;
}

// One output element j of op: the product of its operands gathered at j
// (and at j with the summed bit set), summed over the bucket variable.
// Operands are taken one at a time: most ops have two or three, and a fixed
// group of operand slots would issue predicated-off instructions for the
// absent ones (measured: 84 -> 68 us per N=1000 p=3 step).
template <bool kSmemTable>
__device__ __forceinline__ void compute_element(const DevOp& op, uint32_t j, const DevIn* ins,
                                                const float2* __restrict__ table,
                                                float2* __restrict__ arena) {
    const uint32_t w = op.u - op.sum;
    const uint32_t low = (1u << w) - 1u;
    const DevIn* in = ins + op.in_begin;
    float2 p0 = make_float2(1.f, 0.f), p1 = make_float2(1.f, 0.f);
    for (uint32_t t = 0; t < op.k; ++t) {
        const DevIn d = in[t];
        const uint32_t off = gather_bits(j, d, low);
        const bool tab = d.src & kSrcTable;
        const float2* base = tab ? table + (d.src & ~kSrcTable) : arena + d.src;
        const float2 x0 = (tab && !kSmemTable) ? __ldg(base + off) : base[off];
        float2 x1 = x0;
        // the summed variable is union bit w and, in an operand that has it,
        // that operand's most significant axis: a fixed stride
        if (op.sum && ((d.mask >> w) & 1u)) {
            const uint32_t stride = 1u << (__popc(d.mask) - 1);
            x1 = (tab && !kSmemTable) ? __ldg(base + off + stride) : base[off + stride];
        }
        p0 = t == 0 ? x0 : cmul(p0, x0);
        p1 = t == 0 ? x1 : cmul(p1, x1);
    }
    arena[op.dst + j] = op.sum ? make_float2(p0.x + p1.x, p0.y + p1.y) : p0;
}

// Gate table for the run's angles into shared memory: one thread per table
// element; the element's entry is found by binary search over the entries'
// offsets, the gate tensor evaluated in fp64 and rounded to complex64.
__device__ void build_table(const unsigned char* common, const RunArgs& a, float2* stable) {
    const DevEntry* entries = reinterpret_cast<const DevEntry*>(common);
    const DevTerm* terms = reinterpret_cast<const DevTerm*>(common + a.terms_off);
    for (uint32_t i = threadIdx.x; i < a.table_elems; i += blockDim.x) {
        uint32_t lo = 0, hi = a.n_entries - 1u;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (entries[mid].off <= i) lo = mid;
            else hi = mid - 1u;
        }
        const DevEntry en = entries[lo];
        double alpha = 0.0;
        for (int t = 0; t < en.expr_count; ++t)
            alpha += terms[en.expr_begin + t].coef * __ldg(a.params + terms[en.expr_begin + t].param);
        const int o = (int)(i - en.off);
        uint32_t ixb = en.sliced_value;   // sliced axes at their values
        for (int ax = 0; ax < en.rank_out; ++ax)
            ixb |= (uint32_t)((o >> (en.rank_out - 1 - ax)) & 1) << en.perm[ax];
        const double2 v = gate_value(en.kind, alpha, ixb);
        stable[i] = make_float2((float)v.x, (float)v.y);
    }
    __syncthreads();
}

// The phases of one staged network; its scalar result is returned to thread 0.
template <bool kSmemTable>
__device__ float2 contract_network(const DevNetRun& net, const unsigned char* blob,
                                   const float2* __restrict__ table, float2* __restrict__ arena) {
    const DevPhase* phases = reinterpret_cast<const DevPhase*>(blob);
    const DevOp* ops = reinterpret_cast<const DevOp*>(blob + net.n_phases * sizeof(DevPhase));
    const DevIn* ins = reinterpret_cast<const DevIn*>(blob + net.ins_off);
    // phases with more than 32 elements: all threads, a block barrier each
    for (uint32_t p = 0; p < net.tail_start; ++p) {
        const DevPhase ph = phases[p];
        const uint16_t* chunk = reinterpret_cast<const uint16_t*>(blob + ph.chunk_off);
        uint32_t oi = ph.op_first;
        DevOp op = ops[oi];
        uint32_t op_end = op.elem_begin + (1u << (op.u - op.sum));
        for (uint32_t g = threadIdx.x; g < ph.total_elems; g += blockDim.x) {
            if (g >= op_end) {
                // the chunk table names the op of g's 32-element chunk; small
                // ops may share a chunk, so step forward to the one holding g
                oi = ph.chunk_off ? chunk[g / kChunkElems]
                                  : search_op<false>(ops, ph.op_first, ph.op_first + ph.op_count - 1u, g);
                op = ops[oi];
                oi = find_op(g, oi, op, [&](uint32_t i) { return ops[i]; });
                op_end = op.elem_begin + (1u << (op.u - op.sum));
            }
            compute_element<kSmemTable>(op, g - op.elem_begin, ins, table, arena);
        }
        __syncthreads();
    }
    // the tail (every phase <= 32 elements): warp 0 alone, warp barriers
    if (threadIdx.x < 32) {
        for (uint32_t p = net.tail_start; p < net.n_phases; ++p) {
            const DevPhase ph = phases[p];
            const uint32_t g = threadIdx.x;
            if (g < ph.total_elems) {
                DevOp op = ops[ph.op_first];
                find_op(g, ph.op_first, op, [&](uint32_t i) { return ops[i]; });
                compute_element<kSmemTable>(op, g - op.elem_begin, ins, table, arena);
            }
            __syncwarp();
        }
    }
    float2 result = make_float2(0.f, 0.f);
    if (threadIdx.x == 0)
        result = (net.result_src & kSrcTable) ? table[net.result_src & ~kSrcTable] : arena[net.result_src];
    return result;
}

// ------------------------------------------- element records (see plan.h)
// Part i of n of [p, p + bytes) into L2: a hint with nothing to wait for.
// A launch whose CTAs each bring their part of the plan's small arrays
// (records, runs, jobs) into L2 at once turns every CTA's later first
// touches into L2 hits, instead of DRAM misses on the chain of dependent
// loads that starts each network (after an L2 flush, or on a new plan).
constexpr uint32_t kL2PrefetchMaxBytes = 32u << 20;
__device__ __forceinline__ void l2_prefetch_part(const void* p, uint32_t bytes, uint32_t i, uint32_t n) {
    bytes &= ~15u;
    if (p == nullptr || bytes == 0 || bytes > kL2PrefetchMaxBytes) return;
    const uint32_t part = ((bytes + n - 1u) / n + 15u) & ~15u;
    const uint64_t begin = (uint64_t)i * part;
    if (begin >= bytes) return;
    const uint32_t size = (uint32_t)min((uint64_t)part, (uint64_t)bytes - begin);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(static_cast<const char*>(p) + begin),
                 "r"(size)
                 : "memory");
}

// Header of phase p of a network's records (zero elements past the last).
struct RecHead {
    const uint32_t* rows;   // payload: row r of element g at rows[r * total + g]
    uint32_t total;
    uint32_t kmax;
};

__device__ __forceinline__ RecHead rec_head(const uint32_t* rec, uint32_t p, uint32_t n_phases) {
    if (p >= n_phases) return RecHead{rec, 0u, 0u};
    const uint2 h = __ldg(reinterpret_cast<const uint2*>(rec) + p);
    return RecHead{rec + h.x, h.y & 0xffffffu, h.y >> 24};
}

// The record words of element g (zeros past the phase or the phase's rows).
__device__ __forceinline__ void rec_load(const RecHead& h, uint32_t g, uint32_t (&w)[kRecMaxK + 1]) {
#pragma unroll
    for (uint32_t t = 0; t <= kRecMaxK; ++t)
        w[t] = (g < h.total && t <= h.kmax) ? __ldg(h.rows + (size_t)t * h.total + g) : 0u;
}

// One output element from its record: the same products, in the same
// operand order, as compute_element.
__device__ __forceinline__ void rec_element(const uint32_t (&w)[kRecMaxK + 1], float2* __restrict__ S) {
    const uint32_t d = w[0], k = (d >> 16) & 0xffu;
    float2 p0 = S[w[1] & 0xffffu], p1 = S[w[1] >> 16];
#pragma unroll
    for (uint32_t t = 2; t <= kRecMaxK; ++t)
        if (t <= k) {
            p0 = cmul(p0, S[w[t] & 0xffffu]);
            p1 = cmul(p1, S[w[t] >> 16]);
        }
    S[d & 0xffffu] = (d >> 24) ? make_float2(p0.x + p1.x, p0.y + p1.y) : p0;
}

// The phases of one network from its element records, S the shared window
// [gate table][arena].  Each thread's record of its first element of the
// next phase, and the header of the phase after, are loaded while the
// current phase computes, so the loads from L2 overlap the phase and its
// barrier instead of starting every phase.  Same phase split as
// contract_network: phases of more than 32 elements on every thread with
// block barriers, the tail on warp 0 with warp barriers.
__device__ float2 contract_records(const DevNetRun& net, const uint32_t* __restrict__ rec,
                                   float2* __restrict__ S, const float2* __restrict__ arena) {
    const uint32_t tid = threadIdx.x;
    RecHead h = rec_head(rec, 0, net.n_phases);
    RecHead h1 = rec_head(rec, 1, net.n_phases);
    uint32_t cur[kRecMaxK + 1];
    rec_load(h, tid, cur);
    for (uint32_t p = 0; p < net.n_phases; ++p) {
        const bool tail = p >= net.tail_start;
        if (tail && tid >= 32) break;
        uint32_t nxt[kRecMaxK + 1];
        rec_load(h1, tid, nxt);
        const RecHead h2 = rec_head(rec, p + 2, net.n_phases);
        if (tid < h.total) rec_element(cur, S);
        for (uint32_t g = tid + blockDim.x; g < h.total; g += blockDim.x) {
            uint32_t w[kRecMaxK + 1];
            rec_load(h, g, w);
            rec_element(w, S);
        }
        if (tail) __syncwarp();
        else __syncthreads();
        h = h1;
        h1 = h2;
#pragma unroll
        for (uint32_t t = 0; t <= kRecMaxK; ++t) cur[t] = nxt[t];
    }
    float2 result = make_float2(0.f, 0.f);
    if (tid == 0)
        result = (net.result_src & kSrcTable) ? S[net.result_src & ~kSrcTable] : arena[net.result_src];
    return result;
}

// One output element from its compact record (kRecCompact): the same
// products, in the same operand order, as compute_element.  The operand
// fields after the first come two per 32-bit word, taken a word per loop
// step, so an element costs its own operand count (a warp: the largest of
// its lanes'), not the format's seven slots, and the two operands of a
// word load together.
__device__ __forceinline__ void rec_operand(uint32_t f, const float2* __restrict__ S, float2& p0, float2& p1) {
    const uint32_t o = f & 0xfffu;
    p0 = cmul(p0, S[o]);
    p1 = cmul(p1, S[o + ((1u << (f >> 12)) >> 1)]);
}

__device__ __forceinline__ void rec_element_compact(const uint4 r, float2* __restrict__ S) {
    const uint32_t h = r.x & 0xffffu, k = ((h >> 12) & 7u) + 1u;
    const uint32_t f = r.x >> 16;
    const uint32_t o = f & 0xfffu;
    float2 p0 = S[o], p1 = S[o + ((1u << (f >> 12)) >> 1)];
    uint32_t q0 = r.y, q1 = r.z, q2 = r.w;   // operands 1-2, 3-4, 5-6
#pragma unroll 1
    for (uint32_t t = 1; t < k; t += 2) {
        rec_operand(q0 & 0xffffu, S, p0, p1);
        if (t + 1 < k) rec_operand(q0 >> 16, S, p0, p1);
        q0 = q1;
        q1 = q2;
    }
    S[h & 0xfffu] = (h >> 15) ? make_float2(p0.x + p1.x, p0.y + p1.y) : p0;
}

// Phase headers a CTA stages in shared memory for a compact-record network
// (networks with more phases read the rest from global memory).
constexpr uint32_t kRecHeadSmem = 64;

// The phases of one network from its compact records.  The phase headers
// are staged in shared memory; each thread's record of its first element
// in the next three phases is in flight while the current phase computes,
// so the loads from L2 overlap three phases and their barriers.  Same
// phase split as contract_network.
__device__ float2 contract_records_compact(const DevNetRun& net, const uint32_t* __restrict__ rec,
                                           float2* __restrict__ S, const float2* __restrict__ arena,
                                           uint2* __restrict__ s_head) {
    const uint32_t tid = threadIdx.x, np = net.n_phases;
    const uint2* ghead = reinterpret_cast<const uint2*>(rec);
    const bool staged = np <= kRecHeadSmem;
    // Phase 0's records follow the headers (rounded up to 16 bytes), so this
    // thread's first record is loaded together with the headers instead of
    // after them; the load stays inside the network's records, and the
    // record is used only if the thread has an element in phase 0.
    const uint32_t first_word = (2u * np + 3u) & ~3u;
    const uint4 r0 = first_word + 4u * (tid + 1u) <= net.rec_words
                         ? __ldg(reinterpret_cast<const uint4*>(rec + first_word) + tid)
                         : make_uint4(0u, 0u, 0u, 0u);
    if (staged)
        for (uint32_t i = tid; i < np; i += blockDim.x) s_head[i] = __ldg(ghead + i);
    __syncthreads();
    auto head = [&](uint32_t p) {
        return p >= np ? make_uint2(0u, 0u) : staged ? s_head[p] : __ldg(ghead + p);
    };
    // a phase's header and this thread's record of its first element
    struct Ahead {
        uint2 h;
        uint4 r;
    };
    auto first = [&](uint32_t p) {
        Ahead a;
        a.h = head(p);
        a.r = tid < (a.h.y & 0xffffffu) ? __ldg(reinterpret_cast<const uint4*>(rec + a.h.x) + tid)
                                         : make_uint4(0u, 0u, 0u, 0u);
        return a;
    };
    // phase q contracts from `cur` and loads phase q + 3's header and record
    // into `ahead`; four register slots rotate through an unrolled loop, so
    // nothing is moved between registers
    auto phase = [&](uint32_t q, const Ahead& cur, Ahead& ahead) -> bool {
        if (q >= np) return false;
        const bool tail = q >= net.tail_start;
        if (tail && tid >= 32) return false;
        ahead = first(q + 3);
        const uint32_t total = cur.h.y & 0xffffffu;
        if (tid < total) rec_element_compact(cur.r, S);
        for (uint32_t g = tid + blockDim.x; g < total; g += blockDim.x)
            rec_element_compact(__ldg(reinterpret_cast<const uint4*>(rec + cur.h.x) + g), S);
        if (tail) __syncwarp();
        else __syncthreads();
        return true;
    };
    Ahead ra{head(0), r0}, rb = first(1), rc = first(2), rd;
    for (uint32_t p = 0;; p += 4) {
        if (!phase(p, ra, rd)) break;
        if (!phase(p + 1, rb, ra)) break;
        if (!phase(p + 2, rc, rb)) break;
        if (!phase(p + 3, rd, rc)) break;
    }
    float2 result = make_float2(0.f, 0.f);
    if (tid == 0)
        result = (net.result_src & kSrcTable) ? S[net.result_src & ~kSrcTable] : arena[net.result_src];
    return result;
}

// Network executor.  Shared memory, in order: mbarrier (16 B), [plan-wide
// gate entries + angle terms], the network's plan blob, [gate table],
// [arena]; the bracketed parts exist when kSmemTable / kSmemArena.
//   class launch (kPersistent = false): CTA b contracts jobs[b];
//   persistent launch: every CTA builds the gate table once, then takes
//   networks from the run's queue (jobs in descending width) until it is
//   empty.
// After each network thread 0 writes its term; with a.energy set, the CTA
// that finishes the run's last network sums Re(terms) in fp64 and writes
// the energy.
//   kLean 1 (persistent, 128 threads): registers capped for 8 CTAs per SM,
//   so small networks keep twice as many in flight per SM; kLean 2 (96
//   threads, 12 CTAs per SM) for networks whose staging and arena fit a
//   twelfth of an SM, so that a run of N=1000 p=3 size is resident at once.
template <bool kSmemArena, bool kSmemTable, bool kPersistent, int kLean = 0>
__global__ void __launch_bounds__(kLean == 2 ? 96 : kLean ? 128 : (kPersistent ? 512 : 1024),
                                  kLean == 2 ? 12 : kLean ? 8 : 1) qtb_network_kernel(
    const Job* __restrict__ jobs, const RunArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    unsigned char* common = smem + 16;
    unsigned char* blob = common + (kSmemTable ? a.common_bytes : 0);
    float2* stable = reinterpret_cast<float2*>(blob + a.blob_capacity);
    unsigned char* after_table =
        blob + a.blob_capacity + (kSmemTable ? ((a.table_elems * 8u + 15u) & ~15u) : 0u);
    float2* arena = kSmemArena ? reinterpret_cast<float2*>(after_table)
                               : a.gscratch + (size_t)blockIdx.x * a.arena_capacity;
    __shared__ unsigned int s_job, is_last;
    __shared__ uint2 s_head[kSmemArena && kSmemTable ? kRecHeadSmem : 1];
    if (kPersistent && a.queue == nullptr) {   // a persistent launch needs its queue
        if (threadIdx.x == 0) atomicOr(a.status, kStatusQueue);
        return;
    }
    if (threadIdx.x == 0) {
        l2_prefetch_part(a.recs, a.recs_bytes, blockIdx.x, gridDim.x);
        l2_prefetch_part(a.runs, a.runs_bytes, blockIdx.x, gridDim.x);
        l2_prefetch_part(jobs, a.n_jobs * (uint32_t)sizeof(Job), blockIdx.x, gridDim.x);
    }
    mbar_init(bar);
    uint32_t parity = 0;
    const float2* __restrict__ table = kSmemTable ? stable : a.gtable;
    bool table_ready = !kSmemTable;
    // The plan-wide gate entries are staged once per CTA.  Their copy starts
    // before the first network is located, so that the two overlap.
    if (kSmemTable && threadIdx.x == 0) stage_issue(common, a.common, a.common_bytes, nullptr, nullptr, 0u, bar);
    for (uint32_t iter = 0;; ++iter) {
        // With static_first, a persistent CTA's first network is job
        // blockIdx.x (on a GPU of its own every CTA of the grid is resident
        // at once, so the widest jobs start together without a queue round
        // trip) and the queue counts the claims past the first gridDim.x
        // jobs.  Without it every network is claimed from the queue: where
        // other kernels share the GPU and some CTAs start late, the CTAs
        // that start first take the widest networks.
        uint32_t job_i = blockIdx.x;
        if (kPersistent && (iter > 0 || !a.static_first)) {
            if (threadIdx.x == 0) s_job = (a.static_first ? gridDim.x : 0u) + atomicAdd(a.queue, 1u);
            __syncthreads();
            job_i = s_job;
        } else if (!kPersistent && iter > 0) {
            break;
        }
        if (job_i >= a.n_jobs) {
            if (!table_ready) stage_wait(bar, parity, a.status);   // no copy left in flight
            break;
        }
        const Job job = jobs[job_i];
        const DevNetRun& net = job.net;
        // a network with element records needs no blob (shared table and
        // arena only); otherwise blob_capacity 0: the launch reads plan
        // blobs from global memory
        const bool records = kSmemArena && kSmemTable && a.recs != nullptr && net.rec_words != 0;
        const bool staged = !records && a.blob_capacity != 0;
        if (net.arena_elems > a.arena_capacity || (staged && net.blob_bytes > a.blob_capacity)) {
            if (threadIdx.x == 0)
                atomicOr(a.status, net.arena_elems > a.arena_capacity ? kStatusArena : kStatusBlob);
            if (!table_ready) stage_wait(bar, parity, a.status);
            return;
        }
        if (!table_ready) {
            if (!stage_wait(bar, parity, a.status)) return;
            parity ^= 1u;
            build_table(common, a, stable);
            table_ready = true;
        }
        if (staged) {
            if (!stage(blob, a.blobs + net.blob_off16, net.blob_bytes, nullptr, nullptr, 0u, bar, parity, a.status))
                return;
            parity ^= 1u;
        }
        const unsigned char* nblob =
            staged ? blob : reinterpret_cast<const unsigned char*>(a.blobs + net.blob_off16);
        float2 term;
        if (!records) term = contract_network<kSmemTable>(net, nblob, table, arena);
        else if (net.rec_format == kRecCompact)
            term = contract_records_compact(net, a.recs + net.rec_off, stable, arena, s_head);
        else term = contract_records(net, a.recs + net.rec_off, stable, arena);
        if (threadIdx.x == 0) {
            *job.term = term;
            if (a.energy) {
                __threadfence();
                is_last = atomicAdd(a.done, 1u) == a.total_jobs - 1u;
            }
        }
        __syncthreads();   // blob and arena are reused by the next network
        if (a.energy && is_last) {
            __threadfence();
            reduce_energy(a.terms, a.total_jobs, a.energy_groups, a.energy);
            if (threadIdx.x == 0) *a.done = 0u;   // ready for the next run
            __syncthreads();
        }
    }
}

// ----------------------------------------------------------------- K3w
// Warp-per-network executor for small networks: every warp of a persistent
// CTA takes networks from the run's queue and contracts each one alone,
// staging its blob into the warp's own shared-memory slot by one bulk copy
// (the warp's mbarrier, bounded wait) and keeping its arena in the slot
// after it.  A phase is ceil(elements / 32) rounds of the warp, lane l
// taking element 32 r + l, so the op of a round's first element is the
// phase's chunk-table entry r; phases are separated by warp barriers only.
// With no CTA barrier between dependent phases and about twelve networks
// in flight per SM, a run of small networks is bound by the warps' issue
// rate rather than by the per-phase latency of a whole CTA.  Shared memory:
// [plan-wide gate entries + angle terms][gate table] once per CTA (when
// kSmemTable), then per warp [mbarrier, 16 B][blob, blob_capacity]
// [arena, arena_capacity complex64].
constexpr int kWarpMaxThreads = 256;

__device__ __forceinline__ void warp_bar_wait(uint64_t* bar, uint32_t parity, int* status, bool* ok) {
    const uint32_t bar_a = smem_addr(bar);
    uint32_t done = 0;
    for (uint32_t it = 0; it < kStageSpinLimit; ++it) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(bar_a), "r"(parity) : "memory");
        if (done) break;
        if (it > 64) __nanosleep(32);
    }
    if (!done && (threadIdx.x & 31u) == 0) atomicOr(status, kStatusStageTimeout);
    *ok = __all_sync(0xffffffffu, done != 0);
}

// The phases of one network from its compact element records, contracted by
// one warp: lane l takes elements l, l + 32, ... of a phase, and phases are
// separated by warp barriers only.  S is the warp's window [gate table]
// [arena], the layout the records address.  Each lane's record of its first
// element in the next three phases is in flight while the current phase
// computes (a four-slot rotation through an unrolled loop, as in
// contract_records_compact), and within a phase the next record loads while
// the current element computes.  Networks of at most 32 phases keep their
// phase headers one per lane.
__device__ void warp_records_compact(const DevNetRun& net, const uint32_t* __restrict__ rec,
                                     float2* __restrict__ S, uint32_t lane) {
    const uint32_t np = net.n_phases;
    const uint2* ghead = reinterpret_cast<const uint2*>(rec);
    const uint2 mine = lane < np ? __ldg(ghead + lane) : make_uint2(0u, 0u);
    auto head = [&](uint32_t p) -> uint2 {
        if (np <= 32u) {
            uint2 h;
            h.x = __shfl_sync(0xffffffffu, mine.x, p & 31u);
            h.y = __shfl_sync(0xffffffffu, mine.y, p & 31u);
            return p < np ? h : make_uint2(0u, 0u);
        }
        return p < np ? __ldg(ghead + p) : make_uint2(0u, 0u);
    };
    struct Ahead {
        uint2 h;
        uint4 r;
    };
    auto first = [&](uint32_t p) {
        Ahead x;
        x.h = head(p);
        x.r = lane < (x.h.y & 0xffffffu) ? __ldg(reinterpret_cast<const uint4*>(rec + x.h.x) + lane)
                                          : make_uint4(0u, 0u, 0u, 0u);
        return x;
    };
    auto phase = [&](uint32_t q, const Ahead& cur, Ahead& ahead) -> bool {
        if (q >= np) return false;
        ahead = first(q + 3);
        const uint32_t total = cur.h.y & 0xffffffu;
        const uint4* prec = reinterpret_cast<const uint4*>(rec + cur.h.x);
        uint4 r = cur.r;
        for (uint32_t g = lane; g < total; g += 32u) {
            const uint4 nx = g + 32u < total ? __ldg(prec + g + 32u) : r;
            rec_element_compact(r, S);
            r = nx;
        }
        __syncwarp();
        return true;
    };
    Ahead ra = first(0), rb = first(1), rc = first(2), rd;
    for (uint32_t p = 0;; p += 4) {
        if (!phase(p, ra, rd)) break;
        if (!phase(p + 1, rb, ra)) break;
        if (!phase(p + 2, rc, rb)) break;
        if (!phase(p + 3, rd, rc)) break;
    }
}

// With a.recs set (a launch whose every network has compact element
// records, kSmemTable), a warp's slot is [mbarrier][blob_capacity][copy of
// the gate table][arena]: the records address one window [table][arena],
// so every warp keeps its own copy of the table right before its arena and
// contracts without staging the blob.
template <bool kSmemTable>
__global__ void __launch_bounds__(kWarpMaxThreads) qtb_warp_network_kernel(const Job* __restrict__ jobs,
                                                                          const RunArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (a.queue == nullptr) {
        if (threadIdx.x == 0) atomicOr(a.status, kStatusQueue);
        return;
    }
    unsigned char* common = smem;
    float2* stable = reinterpret_cast<float2*>(smem + (kSmemTable ? a.common_bytes : 0u));
    const uint32_t table_bytes = kSmemTable ? ((a.table_elems * 8u + 15u) & ~15u) : 0u;
    const bool rec_slots = kSmemTable && a.recs != nullptr;
    const uint32_t copy_bytes = rec_slots ? table_bytes : 0u;
    const uint32_t slot_bytes = 16u + a.blob_capacity + copy_bytes + 8u * a.arena_capacity;
    unsigned char* slot = smem + (kSmemTable ? a.common_bytes : 0u) + table_bytes + warp * slot_bytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(slot);
    unsigned char* blob = slot + 16;
    float2* window = reinterpret_cast<float2*>(blob + a.blob_capacity);   // the table copy (rec_slots)
    float2* arena = reinterpret_cast<float2*>(blob + a.blob_capacity + copy_bytes);
    if (kSmemTable) {
        // plan-wide gate entries and angle terms (tiny), then the table
        const uint4* src = a.common;
        uint4* dst = reinterpret_cast<uint4*>(common);
        for (uint32_t i = threadIdx.x; i < a.common_bytes / 16u; i += blockDim.x) dst[i] = __ldg(src + i);
        __syncthreads();
        build_table(common, a, stable);
        if (rec_slots)
            for (uint32_t i = threadIdx.x & 31u; i < a.table_elems; i += 32u) window[i] = stable[i];
    }
    const float2* __restrict__ table = kSmemTable ? stable : a.gtable;
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    uint32_t parity = 0;
    for (;;) {
        uint32_t job = 0;
        if (lane == 0) job = atomicAdd(a.queue, 1u);
        job = __shfl_sync(0xffffffffu, job, 0);
        if (job >= a.n_jobs) break;
        const Job jb = jobs[job];
        const DevNetRun& net = jb.net;
        const bool use_recs = rec_slots && net.rec_words != 0 && net.rec_format == kRecCompact;
        if (net.arena_elems > a.arena_capacity || (!use_recs && net.blob_bytes > a.blob_capacity)) {
            if (lane == 0) atomicOr(a.status, net.arena_elems > a.arena_capacity ? kStatusArena : kStatusBlob);
            return;
        }
        if (use_recs) {
            warp_records_compact(net, a.recs + net.rec_off, window, lane);
        } else {
            if (lane == 0) {
                // the slot was last read by this warp's generic loads
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                const uint32_t bar_a = smem_addr(bar);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(net.blob_bytes)
                             : "memory");
                bulk_copy(blob, a.blobs + net.blob_off16, net.blob_bytes, bar_a);
            }
            bool ok = false;
            warp_bar_wait(bar, parity, a.status, &ok);
            if (!ok) return;
            parity ^= 1u;
            const DevPhase* phases = reinterpret_cast<const DevPhase*>(blob);
            const DevOp* ops = reinterpret_cast<const DevOp*>(blob + net.n_phases * sizeof(DevPhase));
            const DevIn* ins = reinterpret_cast<const DevIn*>(blob + net.ins_off);
            for (uint32_t p = 0; p < net.n_phases; ++p) {
                const DevPhase ph = phases[p];
                const uint16_t* chunk = reinterpret_cast<const uint16_t*>(blob + ph.chunk_off);
                for (uint32_t r = 0; r * 32u < ph.total_elems; ++r) {
                    const uint32_t g = r * 32u + lane;
                    if (g < ph.total_elems) {
                        uint32_t oi = ph.chunk_off ? chunk[r]
                                                   : search_op<false>(ops, ph.op_first, ph.op_first + ph.op_count - 1u, g);
                        DevOp op = ops[oi];
                        find_op(g, oi, op, [&](uint32_t i) { return ops[i]; });
                        compute_element<kSmemTable>(op, g - op.elem_begin, ins, table, arena);
                    }
                }
                __syncwarp();
            }
        }
        uint32_t last = 0;
        if (lane == 0) {
            *jb.term = (net.result_src & kSrcTable) ? table[net.result_src & ~kSrcTable] : arena[net.result_src];
            if (a.energy) {
                __threadfence();
                last = atomicAdd(a.done, 1u) == a.total_jobs - 1u;
            }
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (a.energy && last) {
            __threadfence();
            reduce_energy_warp(a.terms, a.total_jobs, a.energy_groups, a.energy);
            if (lane == 0) *a.done = 0u;   // ready for the next run
        }
        __syncwarp();   // the slot is reused by the next network
    }
}

// ----------------------------------------------------------------- K4
// Wide networks (arenas too large for shared memory) are contracted by the
// whole GPU at once.  The networks of a wave advance together, one step per
// elimination phase: step s holds phase s of every wave network that has
// one, its elements concatenated (segments) and cut into tiles.  CTAs claim
// tiles in order from a queue; a tile of step s starts once every tile of
// step s-1 has finished.  A CTA only ever waits for tiles that were claimed
// before its own, i.e. by CTAs that are running, so the scheme needs no
// co-residency guarantee (no cooperative launch), and every wait is bounded.
struct WideNet {
    const DevNetRun* run;
    float2* term;
    uint64_t arena_off;     // complex64 elements into the wave's arenas
    uint64_t pad;
};

struct WideStep {
    uint32_t seg_begin;     // into the wave's segments
    uint32_t n_segs;
    uint32_t tile_begin;    // first tile of the step
    uint32_t n_tiles;
    uint32_t total_elems;
    uint32_t tile_elems;    // elements per tile of this step (a multiple of 4 x block size)
    uint32_t pad[2];
};

struct WideSeg {
    uint32_t net;           // wave-local network
    uint32_t elem_begin;    // first element of the network's phase within the step
};

struct WideArgs {
    const WideNet* nets;
    const WideStep* steps;
    const WideSeg* segs;
    unsigned int* counters;   // [0] next tile, [1 + s] finished tiles of step s (zeroed per launch)
    float2* arenas;
    uint32_t n_nets;
    uint32_t n_steps;
    uint32_t n_tiles;         // tile n_tiles (the last one) writes the wave's terms
};

static_assert(sizeof(WideNet) == 32, "WideNet layout");
static_assert(sizeof(WideStep) == 32, "WideStep layout");
constexpr uint32_t kWideSpinLimit = 1u << 23;   // about 1 s of polling
constexpr int kWideThreads = 256;
// log2 of the elements a thread has in flight: the wave kernel comes in
// two variants, 8 (3) and 4 (2) elements, chosen per plan by the autotuner
// (the smaller batch needs fewer registers and won on N=256 p=4, the larger
// on Erdos-Renyi N=400 p=3)
constexpr uint32_t kWideBatchLog = 3;
constexpr uint32_t kWideBatch = 1u << kWideBatchLog;
constexpr uint32_t kWideGroup = 1;                                  // operands per batch of loads
constexpr uint32_t kWideMinTile = kWideBatch * kWideThreads;         // 2048
constexpr uint32_t kWideMaxTile = 8 * kWideMinTile;

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait until *counter reaches need (acquire).  Returns false after
// `limit` polls, having set `flag` in *status.
__device__ bool wait_counter(const unsigned int* counter, unsigned int need, uint32_t limit, int* status,
                             int flag) {
    uint32_t it = 0;
    while (ld_acquire(counter) < need) {
        if (++it > limit) {
            atomicOr(status, flag);
            return false;
        }
        if (it > 16) __nanosleep(128);
    }
    return true;
}

__device__ __forceinline__ DevIn ldg_in(const DevIn* p) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
    DevIn d;
    d.mask = v.x;
    d.src = v.y;
    d.runs = (uint64_t)v.z | ((uint64_t)v.w << 32);
    return d;
}

__device__ __forceinline__ DevOp ldg_op(const DevOp* p) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
    DevOp o;
    o.u = (uint8_t)(v.x & 0xffu);
    o.sum = (uint8_t)((v.x >> 8) & 0xffu);
    o.k = (uint8_t)((v.x >> 16) & 0xffu);
    o.pad = 0;
    o.dst = v.y;
    o.elem_begin = v.z;
    o.in_begin = v.w;
    return o;
}

// compute_element for a network whose arena and plan live in global memory
// and are written by other CTAs: arena reads bypass L1 (ld.cg), plan and
// gate-table reads go through the read-only path.
__device__ __forceinline__ void compute_element_wide(const DevOp& op, uint32_t j, const DevIn* ins,
                                                     const float2* __restrict__ table,
                                                     float2* __restrict__ arena) {
    const uint32_t w = op.u - op.sum;
    const uint32_t low = (1u << w) - 1u;
    const DevIn* in = ins + op.in_begin;
    float2 p0 = make_float2(1.f, 0.f), p1 = make_float2(1.f, 0.f);
    for (uint32_t t0 = 0; t0 < op.k; t0 += 4) {
        DevIn d[4];
#pragma unroll
        for (int t = 0; t < 4; ++t)
            if (t0 + t < op.k) d[t] = ldg_in(in + t0 + t);
        float2 x0[4], x1[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            if (t0 + t < op.k) {
                const uint32_t off = gather_bits(j, d[t], low);
                const bool tab = d[t].src & kSrcTable;
                const float2* base = tab ? table + (d[t].src & ~kSrcTable) : arena + d[t].src;
                x0[t] = tab ? __ldg(base + off) : __ldcg(base + off);
                x1[t] = x0[t];
                if (op.sum && ((d[t].mask >> w) & 1u)) {
                    const uint32_t stride = 1u << (__popc(d[t].mask) - 1);
                    x1[t] = tab ? __ldg(base + off + stride) : __ldcg(base + off + stride);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            if (t0 + t < op.k) {
                p0 = (t0 + t == 0) ? x0[t] : cmul(p0, x0[t]);
                p1 = (t0 + t == 0) ? x1[t] : cmul(p1, x1[t]);
            }
        }
    }
    arena[op.dst + j] = op.sum ? make_float2(p0.x + p1.x, p0.y + p1.y) : p0;
}

// 2^kBatchLog elements j + 256 e of one op at once, with the kBatchLog
// bits of j from bit 8 up zero: they differ from j only in those bits, so
// each operand offset is the gathered offset of j plus the gathered offsets
// of those bits (one full gather per operand, not one per element), and the
// loads of kWideGroup operands for all elements are issued together
// (2^(kBatchLog + 1) L2 requests in flight per thread and operand).
template <uint32_t kBatchLog>
__device__ __forceinline__ void compute_elements_wide(const DevOp& op, uint32_t j, const DevIn* ins,
                                                       const float2* __restrict__ table,
                                                       float2* __restrict__ arena) {
    constexpr uint32_t kB = 1u << kBatchLog;
    const uint32_t w = op.u - op.sum;
    const uint32_t low = (1u << w) - 1u;
    const DevIn* in = ins + op.in_begin;
    float2 p0[kB], p1[kB];
#pragma unroll
    for (uint32_t e = 0; e < kB; ++e) p0[e] = p1[e] = make_float2(1.f, 0.f);
    for (uint32_t t0 = 0; t0 < op.k; t0 += kWideGroup) {
        DevIn d[kWideGroup];
#pragma unroll
        for (int t = 0; t < kWideGroup; ++t)
            if (t0 + t < op.k) d[t] = ldg_in(in + t0 + t);
        float2 x0[kWideGroup][kB], x1[kWideGroup][kB];
#pragma unroll
        for (int t = 0; t < kWideGroup; ++t) {
            if (t0 + t < op.k) {
                const bool tab = d[t].src & kSrcTable;
                const float2* base = tab ? table + (d[t].src & ~kSrcTable) : arena + d[t].src;
                const bool has_sum = op.sum && ((d[t].mask >> w) & 1u);
                const uint32_t stride_s = has_sum ? 1u << (__popc(d[t].mask) - 1) : 0u;
                const uint32_t m = d[t].mask & low;
                // bit 8 + i of j lands at operand bit popc(m below it) when m has it
                uint32_t bit_off[kBatchLog];
#pragma unroll
                for (uint32_t i = 0; i < kBatchLog; ++i)
                    bit_off[i] = ((m >> (8 + i)) & 1u) << __popc(m & ((1u << (8 + i)) - 1u));
                uint32_t off[kB];
                off[0] = gather_bits(j, d[t], low);
#pragma unroll
                for (uint32_t e = 1; e < kB; ++e) {
                    uint32_t o = off[0];
#pragma unroll
                    for (uint32_t i = 0; i < kBatchLog; ++i)
                        if ((e >> i) & 1u) o += bit_off[i];
                    off[e] = o;
                }
#pragma unroll
                for (uint32_t e = 0; e < kB; ++e) {
                    x0[t][e] = tab ? __ldg(base + off[e]) : __ldcg(base + off[e]);
                    x1[t][e] = has_sum ? (tab ? __ldg(base + off[e] + stride_s) : __ldcg(base + off[e] + stride_s))
                                       : x0[t][e];
                }
            }
        }
#pragma unroll
        for (int t = 0; t < kWideGroup; ++t) {
            if (t0 + t < op.k) {
#pragma unroll
                for (uint32_t e = 0; e < kB; ++e) {
                    p0[e] = cmul(p0[e], x0[t][e]);
                    p1[e] = cmul(p1[e], x1[t][e]);
                }
            }
        }
    }
#pragma unroll
    for (uint32_t e = 0; e < kB; ++e)
        arena[op.dst + j + e * 256u] = op.sum ? make_float2(p0[e].x + p1[e].x, p0[e].y + p1[e].y) : p0[e];
}

template <uint32_t kBatchLog>
__global__ void __launch_bounds__(kWideThreads, 2) qtb_wide_kernel(const WideArgs w, const RunArgs a) {
    constexpr uint32_t kB = 1u << kBatchLog;
    constexpr uint32_t kBatchBits = (kB - 1u) << 8;   // the bits of j above the thread index
    __shared__ uint32_t s_tile;
    __shared__ int s_ok, s_last;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(w.counters, 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t > w.n_tiles) break;
        uint32_t s = w.n_steps;   // the result tile follows the last step
        if (t < w.n_tiles) {
            uint32_t lo = 0, hi = w.n_steps - 1u;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1u) >> 1;
                if (__ldg(&w.steps[mid].tile_begin) <= t) lo = mid;
                else hi = mid - 1u;
            }
            s = lo;
        }
        if (threadIdx.x == 0) {
            s_ok = 1;
            if (s > 0 && !wait_counter(w.counters + s, __ldg(&w.steps[s - 1].n_tiles), kWideSpinLimit,
                                       a.status, kStatusWideTimeout))
                s_ok = 0;
            __threadfence();
        }
        __syncthreads();
        if (!s_ok) return;
        if (t == w.n_tiles) {
            // every step is done: the wave's terms, then the run's energy if
            // this wave finished the run's last networks
            for (uint32_t n = threadIdx.x; n < w.n_nets; n += blockDim.x) {
                const WideNet wn = w.nets[n];
                const DevNetRun net = *wn.run;
                const float2* arena = w.arenas + wn.arena_off;
                *wn.term = (net.result_src & kSrcTable) ? __ldg(a.gtable + (net.result_src & ~kSrcTable))
                                                        : __ldcg(arena + net.result_src);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                s_last = 0;
                if (a.energy) {
                    __threadfence();
                    s_last = atomicAdd(a.done, w.n_nets) == a.total_jobs - w.n_nets;
                }
            }
            __syncthreads();
            if (s_last) {
                __threadfence();
                reduce_energy(a.terms, a.total_jobs, a.energy_groups, a.energy);
                if (threadIdx.x == 0) *a.done = 0u;
            }
            break;
        }
        const WideStep st = w.steps[s];
        const uint32_t e0 = (t - st.tile_begin) * st.tile_elems;
        const uint32_t e1 = min(e0 + st.tile_elems, st.total_elems);
        // per-thread cache of the current segment and op
        uint32_t seg_lo = 1u, seg_hi = 0u, op_lo = 1u, op_hi = 0u, ph_total = 0u;
        const unsigned char* blob = nullptr;
        const DevIn* ins = nullptr;
        const DevOp* ops = nullptr;
        const uint16_t* chunk = nullptr;
        float2* arena = nullptr;
        DevOp op{};
        uint32_t op_first = 0, op_last = 0;
        const uint32_t bd = blockDim.x;
        for (uint32_t g = e0 + threadIdx.x; g < e1;) {
            if (g < seg_lo || g >= seg_hi) {
                uint32_t lo = st.seg_begin, hi = st.seg_begin + st.n_segs - 1u;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi + 1u) >> 1;
                    if (__ldg(&w.segs[mid].elem_begin) <= g) lo = mid;
                    else hi = mid - 1u;
                }
                const WideSeg sg = w.segs[lo];
                seg_lo = sg.elem_begin;
                seg_hi = lo + 1u < st.seg_begin + st.n_segs ? __ldg(&w.segs[lo + 1u].elem_begin) : st.total_elems;
                const WideNet wn = w.nets[sg.net];
                const DevNetRun net = *wn.run;
                blob = reinterpret_cast<const unsigned char*>(a.blobs + net.blob_off16);
                const DevPhase ph = reinterpret_cast<const DevPhase*>(blob)[s];
                ph_total = ph.total_elems;
                ops = reinterpret_cast<const DevOp*>(blob + net.n_phases * sizeof(DevPhase));
                ins = reinterpret_cast<const DevIn*>(blob + net.ins_off);
                chunk = ph.chunk_off ? reinterpret_cast<const uint16_t*>(blob + ph.chunk_off) : nullptr;
                arena = w.arenas + wn.arena_off;
                op_first = ph.op_first;
                op_last = ph.op_first + ph.op_count - 1u;
                op_lo = 1u;
                op_hi = 0u;
            }
            const uint32_t l = g - seg_lo;
            if (l >= ph_total) {   // padding between segments
                g += bd;
                continue;
            }
            if (l < op_lo || l >= op_hi) {
                const uint32_t oi = chunk ? __ldg(chunk + l / kChunkElems) : search_op<true>(ops, op_first, op_last, l);
                op = ldg_op(ops + oi);
                find_op(l, oi, op, [&](uint32_t i) { return ldg_op(ops + min(i, op_last)); });
                op_lo = op.elem_begin;
                op_hi = op.elem_begin + (1u << (op.u - op.sum));
            }
            // 2^kBatchLog elements of the same op that differ only in the bits
            // from bit 8 up of the op index (the common case in wide phases:
            // tiles, segments and ops start at multiples of kWideMinTile)
            const uint32_t j = l - op.elem_begin;
            if (bd == 256u && (j & kBatchBits) == 0u && g + (kB - 1) * bd < min(e1, seg_hi) &&
                l + (kB - 1) * bd < op_hi) {
                compute_elements_wide<kBatchLog>(op, j, ins, a.gtable, arena);
                g += kB * bd;
            } else {
                compute_element_wide(op, j, ins, a.gtable, arena);
                g += bd;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(w.counters + 1 + s, 1u);
        }
    }
}

// ----------------------------------------------------------------- K5
// Networks too large for shared memory but of moderate size (arenas up to
// QTB_CLUSTER_MAX_ELEMS, opt-in) can run one thread-block cluster of
// kClusterCtas CTAs each: the cluster walks the network's phases, a phase's elements cut into
// chunks of 2048 that the cluster's CTAs take in turn, and phases are
// separated by the cluster barrier (release/acquire at cluster scope, after
// a fence for the arena in global memory).  A cluster's CTAs are scheduled
// together by the hardware, so the barrier needs no flag and no co-residency
// assumption, unlike the grid-wide steps of K4; a network's critical path
// is its phase chain at cluster-barrier latency, and the networks of a run
// proceed independently.  The arena lives in global memory (read with
// ld.cg: another CTA wrote it), the plan blob is read through the read-only
// path.  A chunk that lies within one op of at least 2048 elements is
// computed with the batched loads of K4 (eight elements per thread).
struct ClusterJob {
    const DevNetRun* run;
    float2* term;
    uint64_t arena_off;     // complex64 elements into the cluster arenas
    uint64_t pad;
};
static_assert(sizeof(ClusterJob) == 32, "ClusterJob layout");
constexpr int kClusterCtas = 8;
constexpr int kClusterThreads = 256;
constexpr uint32_t kClusterChunk = 2048;                     // elements per CTA turn (8 per thread)

__global__ void __launch_bounds__(kClusterThreads) qtb_cluster_kernel(const ClusterJob* __restrict__ jobs,
                                                                      float2* __restrict__ arenas, const RunArgs a) {
    uint32_t rank, nctas;
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    asm("mov.u32 %0, %%cluster_nctarank;" : "=r"(nctas));
    __shared__ int s_last;
    const ClusterJob job = jobs[blockIdx.x / nctas];
    const DevNetRun net = *job.run;
    const unsigned char* blob = reinterpret_cast<const unsigned char*>(a.blobs + net.blob_off16);
    const DevOp* ops = reinterpret_cast<const DevOp*>(blob + net.n_phases * sizeof(DevPhase));
    const DevIn* ins = reinterpret_cast<const DevIn*>(blob + net.ins_off);
    float2* arena = arenas + job.arena_off;
    const uint32_t t = threadIdx.x;
    for (uint32_t p = 0; p < net.n_phases; ++p) {
        const uint4 pv = __ldg(reinterpret_cast<const uint4*>(blob) + p);
        const uint32_t op_first = pv.x, op_count = pv.y, total = pv.z;
        const uint32_t op_last = op_first + op_count - 1u;
        for (uint32_t base = rank * kClusterChunk; base < total; base += nctas * kClusterChunk) {
            uint32_t oi = search_op<true>(ops, op_first, op_last, base);
            DevOp op = ldg_op(ops + oi);
            const uint32_t size = 1u << (op.u - op.sum);
            if (size >= kClusterChunk && base + kClusterChunk <= total) {
                // the whole chunk lies in this op (ops start at multiples of their size)
                compute_elements_wide<kWideBatchLog>(op, base + t - op.elem_begin, ins, a.gtable, arena);
            } else {
                uint32_t op_hi = op.elem_begin + size;
#pragma unroll 1
                for (uint32_t e = 0; e < kClusterChunk / kClusterThreads; ++e) {
                    const uint32_t g = base + t + e * kClusterThreads;
                    if (g >= total) break;
                    if (g >= op_hi) {
                        oi = search_op<true>(ops, oi, op_last, g);
                        op = ldg_op(ops + oi);
                        op_hi = op.elem_begin + (1u << (op.u - op.sum));
                    }
                    compute_element_wide(op, g - op.elem_begin, ins, a.gtable, arena);
                }
            }
        }
        // every write of the phase is visible to the whole cluster before the next phase reads it
        __threadfence();
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
    if (rank != 0) return;
    if (t == 0) {
        *job.term = (net.result_src & kSrcTable) ? __ldg(a.gtable + (net.result_src & ~kSrcTable))
                                                 : __ldcg(arena + net.result_src);
        s_last = 0;
        if (a.energy) {
            __threadfence();
            s_last = atomicAdd(a.done, 1u) == a.total_jobs - 1u;
        }
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        reduce_energy(a.terms, a.total_jobs, a.energy_groups, a.energy);
        if (t == 0) *a.done = 0u;
    }
}

// ----------------------------------------------------------------- host
static int cuda_fail(cudaError_t e, const char* what) {
    return fail(QTB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define QTB_CUDA(call)                                     \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// Shared memory of one SM available to CTAs, and the per-CTA reserve.
constexpr uint32_t kSmemPerSm = 228 * 1024;
constexpr uint32_t kSmemReservePerCta = 1024;
// Resident CTAs per SM that define the shared-memory size classes (a network
// goes to the class of the most CTAs per SM its staging + arena allows).
constexpr int kClassCtas[] = {16, 12, 10, 8, 6, 5, 4, 3, 2, 1};
constexpr int kSmemClasses = (int)(sizeof(kClassCtas) / sizeof(kClassCtas[0]));
constexpr int kMaxClasses = kSmemClasses + 1;   // + the stream of the wide waves
constexpr int kLeanThreads = 128;
constexpr int kLeanCtasPerSm = 8;
constexpr int kLean12Threads = 96;
constexpr int kLean12CtasPerSm = 12;
constexpr int kWarpDefaultThreads = 128;   // warps per CTA of the warp queue x 32

struct LaunchClass {
    bool smem;
    bool persistent;        // CTAs take networks from the run's queue
    int lean;               // persistent, registers capped: 1 = 128 threads (8 CTAs per SM), 2 = 96 (12)
    bool warp;              // persistent, every warp takes networks (qtb_warp_network_kernel)
    bool records;           // networks with element records contract from them
    int grid;               // CTAs (= n_jobs unless persistent)
    uint32_t capacity;      // arena elements per CTA
    uint32_t blob_capacity; // plan-blob bytes per CTA
    int threads;
    int n_jobs;
    size_t job_offset;      // into the job buffer
    size_t scratch_offset;  // elements into scratch (classes without a shared arena)
    size_t smem_bytes;
    uint32_t slot_table;    // warp queue over element records: bytes of each warp's gate-table copy
};

// Plan-wide staging image: gate entries, padded to 16 bytes, then the angle
// terms; small enough to stage into every CTA next to its network blob.
struct CommonImage {
    std::vector<uint8_t> bytes;
    uint32_t terms_off = 0;
};

static CommonImage common_image(const qtb_plan* plan) {
    CommonImage c;
    const size_t e_bytes = plan->entries.size() * sizeof(DevEntry);
    c.terms_off = (uint32_t)((e_bytes + 15) & ~size_t(15));
    const size_t total = (c.terms_off + plan->terms.size() * sizeof(DevTerm) + 15) & ~size_t(15);
    c.bytes.assign(std::max<size_t>(total, 16), 0);
    if (e_bytes) std::memcpy(c.bytes.data(), plan->entries.data(), e_bytes);
    if (!plan->terms.empty())
        std::memcpy(c.bytes.data() + c.terms_off, plan->terms.data(), plan->terms.size() * sizeof(DevTerm));
    return c;
}

// One wave of wide networks: its tables live in RunCache::wide_buf.
struct WideWave {
    size_t nets_off, steps_off, segs_off, counters_off;   // bytes into wide_buf
    uint32_t n_nets, n_steps, n_tiles;
    int grid;
};

constexpr int kSchedClasses = 0, kSchedPersistent = 1, kSchedHybrid = 2, kSchedWarp = 3, kSchedHybrid12 = 4;

struct RunCache {
    Job* jobs = nullptr;                // class-mode jobs, persistent-mode jobs, counters
    unsigned int* done = nullptr;
    unsigned int* queue = nullptr;
    bool tuned = false;                 // schedule and block sizes chosen by the autotuner
    int schedule = 0;                   // the schedule in use (kSched*)
    std::vector<LaunchClass> classes;   // class schedule, widest first
    std::vector<LaunchClass> pclasses;  // persistent schedule
    std::vector<LaunchClass> hclasses;  // hybrid schedule: large networks as classes + lean queue
    std::vector<LaunchClass> h12classes;  // the same with the 96-thread lean queue (12 CTAs per SM)
    std::vector<LaunchClass> wclasses;  // warp schedule: large networks as classes + warp queue
    std::vector<WideWave> waves;        // wide networks (both schedules), run one after another
    int wide_batch_log = kWideBatchLog; // wave kernel variant: 2^this elements per thread in flight
    void* wide_buf = nullptr;
    size_t counters_bytes = 0;          // counters of all waves, zeroed before a run
    size_t scratch_elems = 0;           // arenas of the largest wave, then the cluster arenas
    void* cl_jobs = nullptr;            // ClusterJob per network of moderate size (K5)
    int n_cl = 0;
    int cl_ctas = 8;                    // CTAs per cluster
    size_t cl_arena_off = 0;            // elements into scratch where the cluster arenas start
    bool smem_table = true;
    double n_groups = 0.0;              // distinct circuits among the range's networks
};

}  // namespace qtb

// plan-side device state kept outside the public struct
struct qtb_plan_device {
    std::map<std::tuple<int32_t, int32_t, uintptr_t>, qtb::RunCache> runs;
    const qtb::RunCache* last = nullptr;
    bool autotune = false;
    bool timing = false;
    double kernel_ms = 0.0;
    int64_t kernel_launches = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending, spare;
    cudaStream_t aux[qtb::kMaxClasses] = {};
    cudaEvent_t fork = nullptr, join[qtb::kMaxClasses] = {};
};

namespace qtb {
static std::map<const qtb_plan*, qtb_plan_device*> g_dev;
static std::mutex g_dev_mu;

static qtb_plan_device* dev_state(const qtb_plan* p) {
    std::lock_guard<std::mutex> lock(g_dev_mu);
    auto it = g_dev.find(p);
    if (it == g_dev.end()) it = g_dev.emplace(p, new qtb_plan_device()).first;
    return it->second;
}

static const std::vector<LaunchClass>& schedule_of(const RunCache* rc) {
    return rc->schedule == kSchedPersistent ? rc->pclasses
           : rc->schedule == kSchedHybrid   ? rc->hclasses
           : rc->schedule == kSchedWarp     ? rc->wclasses
           : rc->schedule == kSchedHybrid12 ? rc->h12classes
                                            : rc->classes;
}

// Grid of the hybrid schedule's lean queue: its resident CTAs on the GPU
// less the slots the large-network CTAs (launched first) take, counted in
// lean CTAs by threads (registers) and by shared memory.
static int hybrid_lean_grid(std::vector<LaunchClass>& sched, bool smem_table);

static void free_run(RunCache* rc) {
    if (rc->jobs) cudaFree(rc->jobs);
    if (rc->wide_buf) cudaFree(rc->wide_buf);
    if (rc->cl_jobs) cudaFree(rc->cl_jobs);
    rc->jobs = nullptr;
    rc->wide_buf = nullptr;
    rc->cl_jobs = nullptr;
}

static void free_device(qtb_plan* plan) {
    DeviceBuffers& d = plan->dev;
    void* ptrs[] = {d.runs, d.blobs, d.recs, d.entries, d.table, d.status};   // terms lives in entries
    for (void* p : ptrs)
        if (p) cudaFree(p);
    d = DeviceBuffers();
    qtb_plan_device* s = dev_state(plan);
    for (auto& kv : s->runs) free_run(&kv.second);
    s->runs.clear();
    plan->uploaded = false;
}

// Kernel instantiation for a launch class.
template <bool kA, bool kT>
static void launch_one(const LaunchClass& lc, const Job* jobs, const RunArgs& a, cudaStream_t st) {
    if (lc.warp) {
        qtb_warp_network_kernel<kT><<<lc.grid, lc.threads, lc.smem_bytes, st>>>(jobs, a);
        return;
    }
    if constexpr (kA) {
        if (lc.lean == 2) {
            qtb_network_kernel<true, kT, true, 2><<<lc.grid, kLean12Threads, lc.smem_bytes, st>>>(jobs, a);
            return;
        }
        if (lc.lean) {
            qtb_network_kernel<true, kT, true, 1><<<lc.grid, kLeanThreads, lc.smem_bytes, st>>>(jobs, a);
            return;
        }
    }
    if (lc.persistent)
        qtb_network_kernel<kA, kT, true><<<lc.grid, lc.threads, lc.smem_bytes, st>>>(jobs, a);
    else
        qtb_network_kernel<kA, kT, false><<<lc.grid, lc.threads, lc.smem_bytes, st>>>(jobs, a);
}

static void launch_class(const LaunchClass& lc, bool smem_table, const Job* jobs, const RunArgs& a,
                         cudaStream_t st) {
    if (lc.smem) {
        if (smem_table) launch_one<true, true>(lc, jobs, a, st);
        else launch_one<true, false>(lc, jobs, a, st);
    } else {
        if (smem_table) launch_one<false, true>(lc, jobs, a, st);
        else launch_one<false, false>(lc, jobs, a, st);
    }
}

template <bool kA, bool kT, bool kP, int kL = 0>
static cudaError_t allow_smem() {
    return cudaFuncSetAttribute(qtb_network_kernel<kA, kT, kP, kL>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimitBytes);
}

static int allow_all_smem() {
    QTB_CUDA((allow_smem<true, true, false>()));
    QTB_CUDA((allow_smem<true, false, false>()));
    QTB_CUDA((allow_smem<false, true, false>()));
    QTB_CUDA((allow_smem<false, false, false>()));
    QTB_CUDA((allow_smem<true, true, true>()));
    QTB_CUDA((allow_smem<true, false, true>()));
    QTB_CUDA((allow_smem<false, true, true>()));
    QTB_CUDA((allow_smem<false, false, true>()));
    QTB_CUDA((allow_smem<true, true, true, 1>()));
    QTB_CUDA((allow_smem<true, false, true, 1>()));
    QTB_CUDA((allow_smem<true, true, true, 2>()));
    QTB_CUDA((allow_smem<true, false, true, 2>()));
    QTB_CUDA(cudaFuncSetAttribute(qtb_warp_network_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kSmemLimitBytes));
    QTB_CUDA(cudaFuncSetAttribute(qtb_warp_network_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kSmemLimitBytes));
    QTB_CUDA(cudaFuncSetAttribute(qtb_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    return QTB_OK;
}

// Resident CTAs of a persistent launch class on the whole GPU.
static int persistent_grid(const LaunchClass& lc, bool smem_table, int* grid) {
    int per_sm = 0, sms = 0, dev = 0;
    QTB_CUDA(cudaGetDevice(&dev));
    QTB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (lc.warp) {
        if (smem_table)
            QTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qtb_warp_network_kernel<true>,
                                                                   lc.threads, lc.smem_bytes));
        else
            QTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qtb_warp_network_kernel<false>,
                                                                   lc.threads, lc.smem_bytes));
        // enough CTAs for one warp per network
        const int warps = std::max(1, lc.threads / 32);
        *grid = std::max(1, std::min((lc.n_jobs + warps - 1) / warps, std::max(1, per_sm) * sms));
        return QTB_OK;
    } else if (lc.lean == 2) {
        if (smem_table)
            QTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, qtb_network_kernel<true, true, true, 2>, kLean12Threads, lc.smem_bytes));
        else
            QTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, qtb_network_kernel<true, false, true, 2>, kLean12Threads, lc.smem_bytes));
    } else if (lc.lean) {
        if (smem_table)
            QTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, qtb_network_kernel<true, true, true, 1>, kLeanThreads, lc.smem_bytes));
        else
            QTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, qtb_network_kernel<true, false, true, 1>, kLeanThreads, lc.smem_bytes));
    } else if (lc.smem) {
        if (smem_table)
            QTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, qtb_network_kernel<true, true, true>, lc.threads, lc.smem_bytes));
        else
            QTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, qtb_network_kernel<true, false, true>, lc.threads, lc.smem_bytes));
    } else {
        per_sm = 1;
    }
    *grid = std::max(1, std::min(lc.n_jobs, std::max(1, per_sm) * sms));
    return QTB_OK;
}

static int hybrid_lean_grid(std::vector<LaunchClass>& sched, bool smem_table) {
    LaunchClass* lean = nullptr;
    for (LaunchClass& lc : sched)
        if (lc.lean || lc.warp) lean = &lc;
    if (!lean) return QTB_OK;
    int full = 0;
    LaunchClass probe = *lean;
    probe.n_jobs = 1 << 30;
    int r = persistent_grid(probe, smem_table, &full);
    if (r) return r;
    long long taken = 0;
    for (const LaunchClass& lc : sched) {
        if (&lc == lean) continue;
        const long long by_threads = (lc.threads + lean->threads - 1) / lean->threads;
        const long long by_smem = lean->smem_bytes ? (long long)((lc.smem_bytes + lean->smem_bytes - 1) / lean->smem_bytes) : 1;
        taken += (long long)lc.n_jobs * std::max(by_threads, by_smem);
    }
    int sms = 0, dev = 0;
    QTB_CUDA(cudaGetDevice(&dev));
    QTB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long long grid = std::max<long long>(sms, (long long)full - taken);
    // a warp queue needs one warp per network at most
    const int per_cta = lean->warp ? std::max(1, lean->threads / 32) : 1;
    const long long need = (lean->n_jobs + per_cta - 1) / per_cta;
    lean->grid = (int)std::max<long long>(1, std::min<long long>(need, grid));
    return QTB_OK;
}

// Shared memory of a warp-queue launch class of `threads` threads: the
// fixed part, then one slot (mbarrier, blob, arena) per warp.
static size_t warp_slot(const LaunchClass& lc) {
    return 16 + (size_t)lc.blob_capacity + lc.slot_table + 8 * (size_t)lc.capacity;
}
static size_t warp_smem(const LaunchClass& lc, size_t fixed, int threads) {
    return fixed + (size_t)(threads / 32) * warp_slot(lc);
}

// Re-shape the warp queue of a schedule to `threads` threads per CTA (its
// shared memory and grid follow); false if that does not fit a CTA.
static bool set_warp_threads(std::vector<LaunchClass>& sched, bool smem_table, int threads, int* err) {
    *err = QTB_OK;
    for (LaunchClass& q : sched)
        if (q.warp) {
            const size_t fixed = q.smem_bytes - (size_t)(q.threads / 32) * warp_slot(q);
            const size_t smem = warp_smem(q, fixed, threads);
            if (smem > kSmemLimitBytes) return false;
            q.threads = threads;
            q.smem_bytes = smem;
        }
    *err = hybrid_lean_grid(sched, smem_table);
    return *err == QTB_OK;
}

static void destroy_streams(qtb_plan_device* s) {
    for (auto* v : {&s->pending, &s->spare})
        for (auto& e : *v) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
    s->pending.clear();
    s->spare.clear();
    for (int i = 0; i < kMaxClasses; ++i) {
        if (s->aux[i]) cudaStreamDestroy(s->aux[i]);
        if (s->join[i]) cudaEventDestroy(s->join[i]);
        s->aux[i] = nullptr;
        s->join[i] = nullptr;
    }
    if (s->fork) cudaEventDestroy(s->fork);
    s->fork = nullptr;
}

template <typename T>
static int upload_vec(const std::vector<T>& v, void** dst) {
    const size_t bytes = std::max<size_t>(16, v.size() * sizeof(T));
    QTB_CUDA(cudaMalloc(dst, bytes));
    if (!v.empty()) QTB_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return QTB_OK;
}

static int threads_for(uint32_t max_elems) {
    if (max_elems <= 128) return 64;
    if (max_elems <= 1024) return 128;
    if (max_elems <= 4096) return 256;
    if (max_elems <= 16384) return 512;
    return 1024;
}

// Default block size of a launch class (the autotuner may replace it):
// classes too small to fill the GPU trade occupancy for per-network latency.
static int class_threads(uint32_t max_elems, int n_jobs) {
    const int t = threads_for(max_elems);
    if (n_jobs <= 148) return std::max(t, max_elems >= 512 ? 1024 : 512);
    if (n_jobs <= 4 * 148) return std::max(t, 256);
    return t;
}

// Shared memory every CTA of a run needs besides its network's blob and
// arena: the mbarrier, and with a shared gate table the plan-wide entries,
// angle terms and the table itself.
static size_t fixed_smem(const qtb_plan* plan, bool smem_table) {
    if (!smem_table) return 16;
    const size_t table = ((size_t)plan->table_elems * 8 + 15) & ~size_t(15);
    return 16 + plan->common_bytes + table;
}

static uint32_t class_bound(int c) {
    const uint32_t b = kSmemPerSm / (uint32_t)kClassCtas[c] - kSmemReservePerCta;
    return std::min(b, kSmemLimitBytes);
}

// Blob bytes a network stages: none when it contracts from element records.
static uint32_t staged_blob(const DevNetRun& r, bool records) {
    return (records && r.rec_words) ? 0u : r.blob_bytes;
}

static size_t net_need(const DevNetRun& r, size_t fixed, bool records) {
    return fixed + (size_t)staged_blob(r, records) + 8 * (size_t)((r.arena_elems + 3u) & ~3u);
}

// Wide waves of a run: the networks too large for shared memory, largest
// arena first, packed into waves whose arenas fit kWideWaveBytes (a larger
// network forms a wave of its own).  Per wave: networks, steps (one per
// phase index, its segments the wave networks that have that phase) and
// tiles of kWideTileElems elements; one device buffer holds all tables.
constexpr size_t kWideWaveBytes = size_t(1) << 30;

static int build_waves(qtb_plan* plan, std::vector<int32_t> wide, int32_t first, float2* terms,
                       RunCache* rc, bool device) {
    rc->waves.clear();
    rc->counters_bytes = 0;
    if (wide.empty()) return QTB_OK;
    auto arena_of = [&](int32_t i) { return ((size_t)plan->druns[i].arena_elems + 63) & ~size_t(63); };
    std::stable_sort(wide.begin(), wide.end(), [&](int32_t x, int32_t y) { return arena_of(x) > arena_of(y); });
    const auto* runs = static_cast<const DevNetRun*>(plan->dev.runs);
    // resident CTAs size the tiles and the grid; a size-only build needs
    // neither (and may run without a device)
    int per_sm = 1, sms = 148, dev = 0;
    if (device) {
        QTB_CUDA(cudaGetDevice(&dev));
        QTB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        QTB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qtb_wide_kernel<kWideBatchLog>,
                                                               kWideThreads, 0));
        if (plan->wave_ctas_per_sm > 0) per_sm = std::min(per_sm, (int)plan->wave_ctas_per_sm);
    }
    // QTB_WIDE_TILES_PER_CTA (1..8, default 2) in the environment sets how
    // many tiles a step is cut into per resident CTA
    int tiles_per_cta = 2;
    if (const char* env = std::getenv("QTB_WIDE_TILES_PER_CTA")) {
        const int v = std::atoi(env);
        if (v >= 1 && v <= 8) tiles_per_cta = v;
    }
    std::vector<WideNet> nets;
    std::vector<WideStep> steps;
    std::vector<WideSeg> segs;
    struct Range { size_t net0, step0, seg0; };
    std::vector<Range> ranges;
    size_t pos = 0;
    while (pos < wide.size()) {
        // members of this wave
        size_t end = pos, elems = 0;
        while (end < wide.size() && (end == pos || elems + arena_of(wide[end]) <= kWideWaveBytes / 8)) {
            elems += arena_of(wide[end]);
            ++end;
        }
        if (elems >= (size_t(1) << 31))
            return fail(QTB_ERR_UNSUPPORTED, "plan_run: network arena of 2^31 elements or more");
        Range rg{nets.size(), steps.size(), segs.size()};
        WideWave wv{};
        wv.n_nets = (uint32_t)(end - pos);
        uint32_t max_phases = 0;
        size_t off = 0;
        for (size_t k = pos; k < end; ++k) {
            const int32_t i = wide[k];
            WideNet wn{};
            wn.run = runs ? runs + i : nullptr;   // null in a size-only build
            wn.term = terms + (i - first);
            wn.arena_off = off;
            off += arena_of(i);
            nets.push_back(wn);
            max_phases = std::max(max_phases, plan->druns[i].n_phases);
        }
        rc->scratch_elems = std::max(rc->scratch_elems, off);
        uint32_t tiles = 0;
        for (uint32_t ph = 0; ph < max_phases; ++ph) {
            WideStep st{};
            st.seg_begin = (uint32_t)(segs.size() - rg.seg0);
            uint32_t total = 0;
            for (size_t k = pos; k < end; ++k) {
                const Network& n = plan->nets[wide[k]];
                if (ph >= n.phases.size()) continue;
                // segments start at multiples of kWideMinTile, so that with the
                // ops of a phase sorted widest first the elements a thread
                // batches differ only in bits 8 and 9 of their op index
                total = (total + kWideMinTile - 1) & ~(kWideMinTile - 1);
                segs.push_back(WideSeg{(uint32_t)(k - pos), total});
                total += n.phases[ph].total_elems;
            }
            st.n_segs = (uint32_t)(segs.size() - rg.seg0) - st.seg_begin;
            st.total_elems = total;
            st.tile_begin = tiles;
            // about `tiles_per_cta` tiles per resident CTA, within
            // [kWideMinTile, kWideMaxTile]
            const uint32_t target = total / (uint32_t)(tiles_per_cta * std::max(1, per_sm) * sms) + 1;
            st.tile_elems = std::min(kWideMaxTile, ((target + kWideMinTile - 1) / kWideMinTile) * kWideMinTile);
            st.n_tiles = std::max(1u, (total + st.tile_elems - 1) / st.tile_elems);
            tiles += st.n_tiles;
            steps.push_back(st);
        }
        wv.n_steps = max_phases;
        wv.n_tiles = tiles;
        wv.grid = std::max(1, std::min<int>((int)tiles + 1, std::max(1, per_sm) * sms));
        rc->waves.push_back(wv);
        ranges.push_back(rg);
        pos = end;
    }
    // device image: per wave [nets][steps][segs][counters], 256-byte aligned
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t bytes = 0;
    for (size_t v = 0; v < rc->waves.size(); ++v) {
        WideWave& wv = rc->waves[v];
        const size_t n_segs = (v + 1 < ranges.size() ? ranges[v + 1].seg0 : segs.size()) - ranges[v].seg0;
        wv.nets_off = bytes;
        bytes = align(bytes + wv.n_nets * sizeof(WideNet));
        wv.steps_off = bytes;
        bytes = align(bytes + wv.n_steps * sizeof(WideStep));
        wv.segs_off = bytes;
        bytes = align(bytes + n_segs * sizeof(WideSeg));
    }
    const size_t counters0 = bytes;
    for (WideWave& wv : rc->waves) {
        wv.counters_off = bytes;
        bytes += (1 + (size_t)wv.n_steps) * sizeof(unsigned int);
    }
    rc->counters_bytes = bytes - counters0;
    if (!device) return QTB_OK;   // sizes only (qtb_plan_scratch_bytes)
    std::vector<uint8_t> image(align(bytes), 0);
    for (size_t v = 0; v < rc->waves.size(); ++v) {
        const WideWave& wv = rc->waves[v];
        const size_t n_segs = (v + 1 < ranges.size() ? ranges[v + 1].seg0 : segs.size()) - ranges[v].seg0;
        std::memcpy(image.data() + wv.nets_off, nets.data() + ranges[v].net0, wv.n_nets * sizeof(WideNet));
        std::memcpy(image.data() + wv.steps_off, steps.data() + ranges[v].step0, wv.n_steps * sizeof(WideStep));
        std::memcpy(image.data() + wv.segs_off, segs.data() + ranges[v].seg0, n_segs * sizeof(WideSeg));
    }
    QTB_CUDA(cudaMalloc(&rc->wide_buf, image.size()));
    QTB_CUDA(cudaMemcpy(rc->wide_buf, image.data(), image.size(), cudaMemcpyHostToDevice));
    return QTB_OK;
}

// Launch classes of a run: each network goes to the shared-memory class of
// the most resident CTAs per SM its staging + arena allows (networks too
// large for shared memory run as wide waves), the largest class launched
// first so its long critical path starts early.
static int build_run(qtb_plan* plan, int32_t first, int32_t count, float2* terms, RunCache* rc,
                     bool device = true) {
    rc->smem_table = plan->table_elems <= kSmemTableLimitElems;
    rc->n_groups = 0.0;
    for (int32_t i = first; i < first + count; ++i)
        if (i == first || plan->nets[i].info.group != plan->nets[i - 1].info.group) rc->n_groups += 1.0;
    const size_t fixed = fixed_smem(plan, rc->smem_table);
    // element records serve the shared-memory executors of a plan whose
    // gate table is in shared memory (the warp queue stages blobs)
    const bool recs = rc->smem_table && !plan->drecs.empty();
    std::vector<std::vector<int32_t>> members(kMaxClasses);
    for (int32_t i = first; i < first + count; ++i) {
        const DevNetRun& r = plan->druns[i];
        const size_t need = net_need(r, fixed, recs);
        int c = kSmemClasses;   // too large for shared memory: a wide wave
        for (int b = 0; b < kSmemClasses; ++b)
            if (need <= class_bound(b)) {
                c = b;
                break;
            }
        members[c].push_back(i);
    }
    // a class holds the largest blob and the largest arena of its members;
    // move members to the global class while that exceeds the CTA limit
    for (int c = 0; c < kSmemClasses; ++c) {
        auto& m = members[c];
        for (;;) {
            uint32_t blob = 0, arena = 0;
            for (int32_t i : m) {
                blob = std::max(blob, staged_blob(plan->druns[i], recs));
                arena = std::max(arena, (plan->druns[i].arena_elems + 3u) & ~3u);
            }
            if (m.empty() || fixed + blob + 8 * (size_t)arena <= kSmemLimitBytes) break;
            auto big = std::max_element(m.begin(), m.end(), [&](int32_t x, int32_t y) {
                return net_need(plan->druns[x], fixed, recs) < net_need(plan->druns[y], fixed, recs);
            });
            members[kSmemClasses].push_back(*big);
            m.erase(big);
        }
    }
    std::vector<Job> jobs;
    const auto* runs = static_cast<const DevNetRun*>(plan->dev.runs);
    auto make_class = [&](const std::vector<int32_t>& m, bool smem, bool persistent, bool with_recs = true) {
        LaunchClass lc{};
        lc.smem = smem;
        lc.persistent = persistent;
        lc.records = smem && with_recs && recs;
        lc.job_offset = jobs.size();
        lc.n_jobs = (int)m.size();
        lc.grid = lc.n_jobs;
        uint32_t cap = 4, blob = 16, maxe = 1;
        for (int32_t i : m) {
            cap = std::max(cap, plan->druns[i].arena_elems);
            blob = std::max(blob, staged_blob(plan->druns[i], lc.records));
            maxe = std::max(maxe, plan->druns[i].max_elems);
            Job j{};
            j.net = plan->druns[i];
            j.term = terms + (i - first);
            jobs.push_back(j);
        }
        lc.capacity = (cap + 3u) & ~3u;
        // a global-arena class whose largest blob does not fit shared memory
        // reads every member's blob from global memory (capacity 0)
        lc.blob_capacity = (!smem && fixed + (size_t)blob > kSmemLimitBytes) ? 0u : blob;
        blob = lc.blob_capacity;
        lc.threads = persistent ? 256 : class_threads(maxe, lc.n_jobs);
        lc.smem_bytes = fixed + (size_t)blob + (smem ? 8 * (size_t)lc.capacity : 0);
        return lc;
    };
    rc->classes.clear();
    rc->pclasses.clear();
    rc->scratch_elems = 0;
    // class schedule; networks too large for shared memory run as wide waves
    for (int c = kSmemClasses - 1; c >= 0; --c) {
        if (members[c].empty()) continue;
        rc->classes.push_back(make_class(members[c], true, false));
    }
    // persistent schedule: every shared-memory network in one queue, widest
    // (largest arena, then most phases) first
    std::vector<int32_t> all;
    for (int c = 0; c < kSmemClasses; ++c) all.insert(all.end(), members[c].begin(), members[c].end());
    std::stable_sort(all.begin(), all.end(), [&](int32_t x, int32_t y) {
        const DevNetRun& rx = plan->druns[x];
        const DevNetRun& ry = plan->druns[y];
        return rx.arena_elems != ry.arena_elems ? rx.arena_elems > ry.arena_elems
                                                : rx.n_phases > ry.n_phases;
    });
    if (!all.empty()) {
        LaunchClass lc = make_class(all, true, true);
        if (fixed + lc.blob_capacity + 8 * (size_t)lc.capacity <= kSmemLimitBytes)
            rc->pclasses.push_back(lc);   // else no single shared-memory size fits all
    }
    // hybrid schedule: networks whose staging + arena fit an eighth of an SM
    // in one lean persistent queue (kLeanCtasPerSm CTAs per SM), the others
    // as class launches (one CTA per network, more threads), launched first
    // so that their longer critical paths start early
    rc->hclasses.clear();
    rc->h12classes.clear();
    for (int variant = 1; variant <= 2; ++variant) {
        std::vector<LaunchClass>& out = variant == 1 ? rc->hclasses : rc->h12classes;
        const int lean_ctas = variant == 1 ? kLeanCtasPerSm : kLean12CtasPerSm;
        int lean_class = 0;
        while (lean_class < kSmemClasses && kClassCtas[lean_class] != lean_ctas) ++lean_class;
        const uint32_t lean_bound = class_bound(lean_class);
        std::vector<int32_t> lean, big;
        for (int32_t i : all) (net_need(plan->druns[i], fixed, recs) <= lean_bound ? lean : big).push_back(i);
        // the lean queue holds its largest blob and its largest arena at once
        for (;;) {
            uint32_t blob = 0, arena = 0;
            for (int32_t i : lean) {
                blob = std::max(blob, staged_blob(plan->druns[i], recs));
                arena = std::max(arena, (plan->druns[i].arena_elems + 3u) & ~3u);
            }
            if (lean.empty() || fixed + blob + 8 * (size_t)arena <= lean_bound) break;
            auto worst = std::max_element(lean.begin(), lean.end(), [&](int32_t x, int32_t y) {
                return net_need(plan->druns[x], fixed, recs) < net_need(plan->druns[y], fixed, recs);
            });
            big.push_back(*worst);
            lean.erase(worst);
        }
        if (!lean.empty() && !big.empty()) {
            std::vector<int> class_of(count, kSmemClasses);
            for (int c = 0; c < kSmemClasses; ++c)
                for (int32_t i : members[c]) class_of[i - first] = c;
            for (int c = kSmemClasses - 1; c >= 0; --c) {
                std::vector<int32_t> m;
                for (int32_t i : big)
                    if (class_of[i - first] == c) m.push_back(i);
                if (!m.empty()) out.push_back(make_class(m, true, false));
            }
            LaunchClass lc = make_class(lean, true, true);
            lc.lean = variant;
            lc.threads = variant == 1 ? kLeanThreads : kLean12Threads;
            out.push_back(lc);
        }
    }
    // warp schedule: the networks whose warp slot (blob + arena) is at most
    // the 95th percentile of the run's slots go to one warp queue (every
    // warp contracts its own network), the others run as class launches,
    // started first.  Networks with compact element records need no blob in
    // the slot, only a copy of the gate table before the arena; when every
    // network of the queue has them, the queue contracts from the records.
    rc->wclasses.clear();
    if (!all.empty()) {
        const size_t table_copy = ((size_t)plan->table_elems * 8 + 15) & ~size_t(15);
        auto compact = [&](int32_t i) {
            const DevNetRun& r = plan->druns[i];
            return recs && r.rec_words != 0 && r.rec_format == kRecCompact;
        };
        auto slot_of = [&](int32_t i) {
            return 16 + (compact(i) ? table_copy : (size_t)plan->druns[i].blob_bytes) +
                   8 * (size_t)((plan->druns[i].arena_elems + 3u) & ~3u);
        };
        std::vector<size_t> slots;
        for (int32_t i : all) slots.push_back(slot_of(i));
        std::sort(slots.begin(), slots.end());
        const size_t cap = std::min(slots[std::min(slots.size() - 1, slots.size() * 95 / 100)],
                                    (kSmemLimitBytes - fixed) / 2);
        std::vector<int32_t> small, large;
        for (int32_t i : all) (slot_of(i) <= cap ? small : large).push_back(i);
        if (!small.empty()) {
            std::vector<int> class_of(count, kSmemClasses);
            for (int c = 0; c < kSmemClasses; ++c)
                for (int32_t i : members[c]) class_of[i - first] = c;
            for (int c = kSmemClasses - 1; c >= 0; --c) {
                std::vector<int32_t> m;
                for (int32_t i : large)
                    if (class_of[i - first] == c) m.push_back(i);
                if (!m.empty()) rc->wclasses.push_back(make_class(m, true, false));
            }
            const bool all_compact = std::all_of(small.begin(), small.end(), compact);
            LaunchClass lc = make_class(small, true, true, all_compact);
            lc.warp = true;
            lc.slot_table = lc.records ? (uint32_t)table_copy : 0u;
            lc.threads = kWarpDefaultThreads;
            while (lc.threads > 32 && warp_smem(lc, fixed, lc.threads) > kSmemLimitBytes) lc.threads /= 2;
            lc.smem_bytes = warp_smem(lc, fixed, lc.threads);
            rc->wclasses.push_back(lc);
        }
    }
    // networks too large for shared memory run as whole-GPU waves (K4);
    // QTB_CLUSTER_MAX_ELEMS=<elements> in the environment runs those whose
    // arena is at most that as one thread-block cluster each (K5) instead.
    // Waves are the default: on N=256 p=4 and Erdos-Renyi N=400 p=3 they
    // took 0.71 and 2.06 ms, clusters of 2-16 CTAs 0.74-1.30 and 3.4-9.8 ms.
    std::vector<int32_t> wave_nets, cl_nets;
    uint64_t cl_max = 0;
    if (const char* env = std::getenv("QTB_CLUSTER_MAX_ELEMS")) cl_max = std::strtoull(env, nullptr, 10);
    for (int32_t i : members[kSmemClasses])
        (plan->druns[i].arena_elems <= cl_max ? cl_nets : wave_nets).push_back(i);
    // QTB_WIDE_BATCH=2 or 3 in the environment fixes the wave kernel variant
    // (2^this elements per thread in flight) instead of the autotuner
    if (const char* env = std::getenv("QTB_WIDE_BATCH")) {
        const int v = std::atoi(env);
        if (v == 2 || v == 3) rc->wide_batch_log = v;
    }
    // QTB_CLUSTER_CTAS (2, 4, 8 or 16) sets the CTAs per cluster
    rc->cl_ctas = kClusterCtas;
    if (const char* env = std::getenv("QTB_CLUSTER_CTAS")) {
        const int c = std::atoi(env);
        if (c == 2 || c == 4 || c == 8 || c == 16) rc->cl_ctas = c;
    }
    auto place_clusters = [&](bool on_device) -> int {
        rc->n_cl = (int)cl_nets.size();
        rc->cl_arena_off = (rc->scratch_elems + 63) & ~size_t(63);
        std::vector<ClusterJob> cj;
        size_t off = 0;
        for (int32_t i : cl_nets) {
            ClusterJob j{};
            j.run = runs ? runs + i : nullptr;
            j.term = terms + (i - first);
            j.arena_off = rc->cl_arena_off + off;
            off += ((size_t)plan->druns[i].arena_elems + 63) & ~size_t(63);
            cj.push_back(j);
        }
        if (!cj.empty()) rc->scratch_elems = rc->cl_arena_off + off;
        if (!on_device || cj.empty()) return QTB_OK;
        QTB_CUDA(cudaMalloc(&rc->cl_jobs, cj.size() * sizeof(ClusterJob)));
        QTB_CUDA(cudaMemcpy(rc->cl_jobs, cj.data(), cj.size() * sizeof(ClusterJob), cudaMemcpyHostToDevice));
        return QTB_OK;
    };
    if (!device) {
        int r = build_waves(plan, wave_nets, first, terms, rc, false);
        return r ? r : place_clusters(false);
    }
    // jobs of both schedules, then 16 bytes of counters (done, queue), zeroed
    const size_t job_bytes = jobs.size() * sizeof(Job);
    void* buf = nullptr;
    QTB_CUDA(cudaMalloc(&buf, job_bytes + 16));
    QTB_CUDA(cudaMemcpy(buf, jobs.data(), job_bytes, cudaMemcpyHostToDevice));
    QTB_CUDA(cudaMemset(static_cast<char*>(buf) + job_bytes, 0, 16));
    rc->jobs = static_cast<Job*>(buf);
    rc->done = reinterpret_cast<unsigned int*>(static_cast<char*>(buf) + job_bytes);
    rc->queue = rc->done + 1;
    for (LaunchClass& lc : rc->pclasses)
        if (lc.persistent) {
            int r = persistent_grid(lc, rc->smem_table, &lc.grid);
            if (r) return r;
        }
    if (!rc->hclasses.empty()) {
        int r = hybrid_lean_grid(rc->hclasses, rc->smem_table);
        if (r) return r;
    }
    if (!rc->h12classes.empty()) {
        int r = hybrid_lean_grid(rc->h12classes, rc->smem_table);
        if (r) return r;
    }
    if (!rc->wclasses.empty()) {
        int r = hybrid_lean_grid(rc->wclasses, rc->smem_table);
        if (r) return r;
    }
    int rw = build_waves(plan, wave_nets, first, terms, rc, true);
    return rw ? rw : place_clusters(true);
}

}  // namespace qtb

using namespace qtb;

extern "C" {

const char* qtb_version(void) { return "qtensor_b200 0.2 (sm_100a)"; }

int qtb_init(int device) {
    int n = 0;
    QTB_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(QTB_ERR_ARG, "qtb_init: no such device");
    QTB_CUDA(cudaSetDevice(device));
    int r = allow_all_smem();
    if (r) return r;
    return QTB_OK;
}

int qtb_bucket_c64(const qtb_bucket_desc* d, const void* const* inputs, void* output, void* stream) {
    if (!d || !inputs || !output) return fail(QTB_ERR_ARG, "bucket: null argument");
    if (d->n_inputs < 1 || d->n_inputs > QTB_MAX_BUCKET_INPUTS)
        return fail(QTB_ERR_ARG, "bucket: n_inputs out of range");
    if (d->n_vars < 0 || d->n_vars > QTB_MAX_BUCKET_VARS)
        return fail(QTB_ERR_ARG, "bucket: n_vars out of range");
    if ((d->sum_first != 0 && d->sum_first != 1) || (d->sum_first && d->n_vars < 1))
        return fail(QTB_ERR_ARG, "bucket: sum_first needs at least one variable");
    const uint32_t all = d->n_vars >= 32 ? 0xffffffffu : ((1u << d->n_vars) - 1u);
    BucketArgs a{};
    for (int t = 0; t < d->n_inputs; ++t) {
        if (!inputs[t]) return fail(QTB_ERR_ARG, "bucket: null input pointer");
        if (d->masks[t] & ~all) return fail(QTB_ERR_ARG, "bucket: mask names a variable outside the union");
        a.in[t] = static_cast<const float2*>(inputs[t]);
        bucket_operand(&a, t, d->masks[t], d->n_vars, d->sum_first);
    }
    a.out = static_cast<float2*>(output);
    a.k = d->n_inputs;
    a.sum = d->sum_first;
    a.w = d->n_vars - d->sum_first;
    qtb_bucket_kernel<<<bucket_blocks(a.w), kBucketThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
    QTB_CUDA(cudaGetLastError());
    return QTB_OK;
}

int qtb_plan_upload(qtb_plan* plan) {
    if (!plan) return fail(QTB_ERR_ARG, "plan_upload: null plan");
    std::lock_guard<std::mutex> lock(plan->mu);
    // the executor's shared-memory limits on the current device (qtb_init
    // does the same; a caller that skipped it still gets working launches)
    int r0 = allow_all_smem();
    if (r0) return r0;
    free_device(plan);
    ensure_images(plan);
    int r;
    if ((r = upload_vec(plan->druns, &plan->dev.runs))) return r;
    if ((r = upload_vec(plan->dblobs, &plan->dev.blobs))) return r;
    if (!plan->drecs.empty() && (r = upload_vec(plan->drecs, &plan->dev.recs))) return r;
    {
        const CommonImage c = common_image(plan);
        plan->common_bytes = (uint32_t)c.bytes.size();
        plan->common_terms_off = c.terms_off;
        if ((r = upload_vec(c.bytes, &plan->dev.entries))) return r;
        plan->dev.terms = static_cast<char*>(plan->dev.entries) + c.terms_off;
    }
    QTB_CUDA(cudaMalloc(&plan->dev.table, std::max<size_t>(16, (size_t)plan->table_elems * 8)));
    QTB_CUDA(cudaMalloc(&plan->dev.status, sizeof(int)));
    QTB_CUDA(cudaMemset(plan->dev.status, 0, sizeof(int)));
    QTB_CUDA(cudaGetDevice(&plan->device));
    plan->uploaded = true;
    return QTB_OK;
}

static int get_run(qtb_plan* plan, int32_t first, int32_t count, void* terms, RunCache** out) {
    qtb_plan_device* s = dev_state(plan);
    auto key = std::make_tuple(first, count, reinterpret_cast<uintptr_t>(terms));
    auto it = s->runs.find(key);
    if (it == s->runs.end()) {
        if (s->runs.size() >= 64) {   // callers cycling through many output buffers
            QTB_CUDA(cudaDeviceSynchronize());
            for (auto& kv : s->runs) free_run(&kv.second);
            s->runs.clear();
        }
        RunCache rc;
        int r = build_run(plan, first, count, static_cast<float2*>(terms), &rc);
        if (r) return r;
        it = s->runs.emplace(key, rc).first;
    }
    *out = &it->second;
    return QTB_OK;
}

int qtb_plan_scratch_bytes(const qtb_plan* plan_c, int32_t first, int32_t count, size_t* bytes) {
    qtb_plan* plan = const_cast<qtb_plan*>(plan_c);
    if (!plan || !bytes) return fail(QTB_ERR_ARG, "plan_scratch_bytes: bad arguments");
    if (!plan->uploaded) {
        // before upload: the same host images qtb_plan_upload builds, so that a
        // caller can budget device memory before it allocates any
        std::lock_guard<std::mutex> lock(plan->mu);
        ensure_images(plan);
        plan->common_bytes = (uint32_t)common_image(plan).bytes.size();
    }
    if (first < 0 || count < 0 || first + count > (int32_t)plan->druns.size())
        return fail(QTB_ERR_ARG, "plan_scratch_bytes: range out of bounds");
    *bytes = 0;
    if (count == 0) return QTB_OK;
    // the exact class split of this range (the same one qtb_plan_run uses)
    RunCache rc;
    int r = build_run(plan, first, count, nullptr, &rc, false);   // sizes only, no device memory
    free_run(&rc);
    if (r) return r;
    *bytes = rc.scratch_elems * sizeof(float2);
    return QTB_OK;
}

static int ensure_streams(qtb_plan_device* s);

// The wide waves of a run, one after another on st: counters zeroed, then
// one K4 launch per wave over the shared arena scratch.
static int launch_waves(const RunCache* rc, const RunArgs& base, void* scratch_dev, cudaStream_t st) {
    if (rc->n_cl > 0) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)(rc->n_cl * rc->cl_ctas));
        cfg.blockDim = dim3(kClusterThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)rc->cl_ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        QTB_CUDA(cudaLaunchKernelEx(&cfg, qtb_cluster_kernel, static_cast<const ClusterJob*>(rc->cl_jobs),
                                    static_cast<float2*>(scratch_dev), base));
    }
    if (rc->waves.empty()) return QTB_OK;
    char* buf = static_cast<char*>(rc->wide_buf);
    QTB_CUDA(cudaMemsetAsync(buf + rc->waves[0].counters_off, 0, rc->counters_bytes, st));
    for (const WideWave& wv : rc->waves) {
        WideArgs w{};
        w.nets = reinterpret_cast<const WideNet*>(buf + wv.nets_off);
        w.steps = reinterpret_cast<const WideStep*>(buf + wv.steps_off);
        w.segs = reinterpret_cast<const WideSeg*>(buf + wv.segs_off);
        w.counters = reinterpret_cast<unsigned int*>(buf + wv.counters_off);
        w.arenas = static_cast<float2*>(scratch_dev);
        w.n_nets = wv.n_nets;
        w.n_steps = wv.n_steps;
        w.n_tiles = wv.n_tiles;
        if (rc->wide_batch_log == 2) qtb_wide_kernel<2><<<wv.grid, kWideThreads, 0, st>>>(w, base);
        else qtb_wide_kernel<kWideBatchLog><<<wv.grid, kWideThreads, 0, st>>>(w, base);
        QTB_CUDA(cudaGetLastError());
    }
    return QTB_OK;
}

// Launch a schedule on st: a persistent class needs its queue zeroed first
// (a memset node when captured); several classes, and the wide waves, run
// concurrently on forked streams joined back into st.
static int launch_schedule(qtb_plan_device* s, const RunCache* rc,
                           const std::vector<LaunchClass>& sched, const RunArgs& base,
                           void* scratch_dev, cudaStream_t st, bool with_waves = true) {
    int r = ensure_streams(s);
    if (r) return r;
    for (const LaunchClass& lc : sched)
        if (lc.persistent) QTB_CUDA(cudaMemsetAsync(rc->queue, 0, sizeof(unsigned int), st));
    const bool waves = with_waves && (!rc->waves.empty() || rc->n_cl > 0);
    const bool forked = sched.size() + (waves ? 1 : 0) > 1;
    if (forked) QTB_CUDA(cudaEventRecord(s->fork, st));
    if (waves) {
        cudaStream_t ws = forked ? s->aux[kMaxClasses - 1] : st;
        if (forked) QTB_CUDA(cudaStreamWaitEvent(ws, s->fork, 0));
        if ((r = launch_waves(rc, base, scratch_dev, ws))) return r;
        if (forked) {
            QTB_CUDA(cudaEventRecord(s->join[kMaxClasses - 1], ws));
            QTB_CUDA(cudaStreamWaitEvent(st, s->join[kMaxClasses - 1], 0));
        }
    }
    for (size_t c = 0; c < sched.size(); ++c) {
        const LaunchClass& lc = sched[c];
        cudaStream_t cs = forked ? s->aux[c] : st;
        if (forked) QTB_CUDA(cudaStreamWaitEvent(cs, s->fork, 0));
        RunArgs ac = base;
        ac.queue = rc->queue;
        ac.arena_capacity = lc.capacity;
        ac.blob_capacity = lc.blob_capacity;
        ac.recs = lc.records ? base.recs : nullptr;
        ac.n_jobs = (uint32_t)lc.n_jobs;
        ac.gscratch = lc.smem ? nullptr : static_cast<float2*>(scratch_dev) + lc.scratch_offset;
        launch_class(lc, rc->smem_table, rc->jobs + lc.job_offset, ac, cs);
        QTB_CUDA(cudaGetLastError());
        if (forked) {
            QTB_CUDA(cudaEventRecord(s->join[c], cs));
            QTB_CUDA(cudaStreamWaitEvent(st, s->join[c], 0));
        }
    }
    return QTB_OK;
}

// Autotuner, on the first run of a range (energy reduction off while it
// times): each class of the class schedule is timed alone with 64..1024
// threads per CTA; then the whole class schedule and the persistent
// schedule (128/256/512 threads) are timed end to end and the faster
// schedule is kept.  Each measurement is the fastest of three launches.
static int autotune_run(qtb_plan_device* s, RunCache* rc, const RunArgs& base, void* scratch_dev,
                        cudaStream_t st) {
    static const int kCandidates[] = {64, 128, 256, 512, 1024};
    cudaEvent_t e0, e1;
    QTB_CUDA(cudaEventCreate(&e0));
    QTB_CUDA(cudaEventCreate(&e1));
    RunArgs a = base;
    a.energy = nullptr;
    const bool log = std::getenv("QTB_AUTOTUNE_LOG") != nullptr;
    auto time_it = [&](auto&& launch, float* best) -> int {
        int r = launch();   // warm-up
        if (r) return r;
        for (int rep = 0; rep < 3; ++rep) {
            QTB_CUDA(cudaEventRecord(e0, st));
            if ((r = launch())) return r;
            QTB_CUDA(cudaEventRecord(e1, st));
            QTB_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            QTB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            *best = std::min(*best, ms);
        }
        return QTB_OK;
    };
    int r;
    for (LaunchClass& lc : rc->classes) {
        int best_t = lc.threads;
        float best_ms = 1e30f;
        for (int t : kCandidates) {
            std::vector<LaunchClass> one(1, lc);
            one[0].threads = t;
            float ms = 1e30f;
            if ((r = time_it([&] { return launch_schedule(s, rc, one, a, scratch_dev, st, false); }, &ms)))
                return r;
            if (log)
                std::fprintf(stderr, "qtb autotune: class of %d networks (smem %zu B) %4d threads %.1f us\n",
                             lc.n_jobs, lc.smem_bytes, t, 1e3 * ms);
            if (ms < best_ms) {
                best_ms = ms;
                best_t = t;
            }
        }
        lc.threads = best_t;
        for (LaunchClass& pc : rc->pclasses)   // the global class is shared
            if (!pc.persistent && pc.job_offset == lc.job_offset) pc.threads = best_t;
    }
    float class_ms = 1e30f;
    if ((r = time_it([&] { return launch_schedule(s, rc, rc->classes, a, scratch_dev, st); }, &class_ms)))
        return r;
    float pers_ms = 1e30f;
    if (!rc->pclasses.empty()) {
        for (LaunchClass& pc : rc->pclasses) {
            if (!pc.persistent) continue;
            int best_t = pc.threads;
            float best = 1e30f;
            for (int t : {128, 256, 512}) {
                std::vector<LaunchClass> sched = rc->pclasses;
                for (LaunchClass& q : sched)
                    if (q.persistent) {
                        q.threads = t;
                        if ((r = persistent_grid(q, rc->smem_table, &q.grid))) return r;
                    }
                float ms = 1e30f;
                if ((r = time_it([&] { return launch_schedule(s, rc, sched, a, scratch_dev, st); }, &ms)))
                    return r;
                if (log)
                    std::fprintf(stderr, "qtb autotune: persistent schedule %4d threads %.1f us\n", t, 1e3 * ms);
                if (ms < best) {
                    best = ms;
                    best_t = t;
                }
            }
            pc.threads = best_t;
            if ((r = persistent_grid(pc, rc->smem_table, &pc.grid))) return r;
            pers_ms = best;
        }
    }
    // hybrid schedule: the large-network classes with 256..1024 threads
    float hyb_ms = 1e30f;
    int big_threads = 512;   // block size of large-network classes, as the hybrid tuning finds
    if (!rc->hclasses.empty()) {
        int best_t = 512;
        for (int t : {256, 512, 1024}) {
            std::vector<LaunchClass> sched = rc->hclasses;
            for (LaunchClass& q : sched)
                if (!q.lean) q.threads = t;
            if ((r = hybrid_lean_grid(sched, rc->smem_table))) return r;
            float ms = 1e30f;
            if ((r = time_it([&] { return launch_schedule(s, rc, sched, a, scratch_dev, st); }, &ms)))
                return r;
            if (log)
                std::fprintf(stderr, "qtb autotune: hybrid schedule, large networks %4d threads %.1f us\n", t,
                             1e3 * ms);
            if (ms < hyb_ms) {
                hyb_ms = ms;
                best_t = t;
            }
        }
        for (LaunchClass& q : rc->hclasses)
            if (!q.lean) q.threads = best_t;
        big_threads = best_t;
        if ((r = hybrid_lean_grid(rc->hclasses, rc->smem_table))) return r;
    }
    // hybrid schedule with the 96-thread lean queue (12 CTAs per SM), its
    // large-network classes at 512 or 1024 threads
    float hyb12_ms = 1e30f;
    if (!rc->h12classes.empty()) {
        int best_t = 512;
        for (int t : {512, 1024}) {
            std::vector<LaunchClass> sched = rc->h12classes;
            for (LaunchClass& q : sched)
                if (!q.lean) q.threads = t;
            if ((r = hybrid_lean_grid(sched, rc->smem_table))) return r;
            float ms = 1e30f;
            if ((r = time_it([&] { return launch_schedule(s, rc, sched, a, scratch_dev, st); }, &ms)))
                return r;
            if (log)
                std::fprintf(stderr, "qtb autotune: hybrid schedule (96-thread lean queue), large networks %4d threads %.1f us\n",
                             t, 1e3 * ms);
            if (ms < hyb12_ms) {
                hyb12_ms = ms;
                best_t = t;
            }
        }
        for (LaunchClass& q : rc->h12classes)
            if (!q.lean) q.threads = best_t;
        if ((r = hybrid_lean_grid(rc->h12classes, rc->smem_table))) return r;
    }
    // warp schedule: the warp queue with 2, 4 or 8 warps per CTA (the
    // large-network classes keep their tuned block size)
    float warp_ms = 1e30f;
    if (!rc->wclasses.empty()) {
        for (LaunchClass& q : rc->wclasses)
            if (!q.warp) q.threads = big_threads;
        int best_t = 0;
        for (int t : {64, 128, 256}) {
            std::vector<LaunchClass> sched = rc->wclasses;
            if (!set_warp_threads(sched, rc->smem_table, t, &r)) {
                if (r) return r;
                continue;
            }
            float ms = 1e30f;
            if ((r = time_it([&] { return launch_schedule(s, rc, sched, a, scratch_dev, st); }, &ms)))
                return r;
            if (log)
                std::fprintf(stderr, "qtb autotune: warp schedule %4d threads per CTA %.1f us\n", t, 1e3 * ms);
            if (ms < warp_ms) {
                warp_ms = ms;
                best_t = t;
            }
        }
        if (best_t && !set_warp_threads(rc->wclasses, rc->smem_table, best_t, &r) && r) return r;
    }
    rc->schedule = kSchedClasses;
    float best_ms = class_ms;
    if (pers_ms < best_ms) {
        rc->schedule = kSchedPersistent;
        best_ms = pers_ms;
    }
    if (hyb_ms < best_ms) {
        rc->schedule = kSchedHybrid;
        best_ms = hyb_ms;
    }
    if (warp_ms < best_ms) {
        rc->schedule = kSchedWarp;
        best_ms = warp_ms;
    }
    if (hyb12_ms < best_ms) rc->schedule = kSchedHybrid12;
    if (log) {
        // a schedule that does not apply to the plan keeps its 1e30 sentinel
        auto us = [](float ms, char* buf) {
            if (ms >= 1e29f)
                std::snprintf(buf, 24, "n/a");
            else
                std::snprintf(buf, 24, "%.1f us", 1e3 * ms);
            return buf;
        };
        char b0[24], b1[24], b2[24], b3[24], b4[24];
        std::fprintf(stderr,
                     "qtb autotune: class schedule %s, persistent %s, hybrid %s, hybrid "
                     "(96-thread lean) %s, warp %s -> %s\n",
                     us(class_ms, b0), us(pers_ms, b1), us(hyb_ms, b2), us(hyb12_ms, b3), us(warp_ms, b4),
                     rc->schedule == kSchedWarp       ? "warp"
                     : rc->schedule == kSchedHybrid12 ? "hybrid12"
                     : rc->schedule == kSchedHybrid   ? "hybrid"
                     : rc->schedule == kSchedPersistent ? "persistent"
                                                      : "classes");
    }
    // the wave kernel variant (8 or 4 elements per thread in flight), timed
    // with the chosen schedule unless QTB_WIDE_BATCH fixes it
    if (!rc->waves.empty() && !std::getenv("QTB_WIDE_BATCH")) {
        float wave_ms[2] = {1e30f, 1e30f};
        for (int v = 0; v < 2; ++v) {
            rc->wide_batch_log = v == 0 ? (int)kWideBatchLog : 2;
            if ((r = time_it([&] { return launch_schedule(s, rc, schedule_of(rc), a, scratch_dev, st); },
                             &wave_ms[v])))
                return r;
        }
        rc->wide_batch_log = wave_ms[1] < wave_ms[0] ? 2 : (int)kWideBatchLog;
        if (log)
            std::fprintf(stderr, "qtb autotune: waves with 8 elements per thread %.1f us, 4 elements %.1f us\n",
                         1e3 * wave_ms[0], 1e3 * wave_ms[1]);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    rc->tuned = true;
    return QTB_OK;
}

// QTB_SCHEDULE=persistent:<128|256|512>, hybrid:<256|512|1024> (threads of
// the large-network classes), hybrid12:<512|1024> (the same with the
// 96-thread lean queue), warp:<64|128|256> (threads per CTA of the warp
// queue) or QTB_SCHEDULE=classes in the
// environment fixes the schedule of every range without timing it, so that a
// profiler sees one chosen configuration.  Returns 1 when it applied.
static int forced_schedule(RunCache* rc, int* err) {
    *err = QTB_OK;
    const char* env = std::getenv("QTB_SCHEDULE");
    if (!env) return 0;
    if (std::strncmp(env, "persistent:", 11) == 0 && !rc->pclasses.empty()) {
        const int t = std::atoi(env + 11);
        if (t != 128 && t != 256 && t != 512) return 0;
        for (LaunchClass& q : rc->pclasses)
            if (q.persistent) {
                q.threads = t;
                if ((*err = persistent_grid(q, rc->smem_table, &q.grid))) return 0;
            }
        rc->schedule = kSchedPersistent;
    } else if (std::strncmp(env, "hybrid:", 7) == 0 && !rc->hclasses.empty()) {
        const int t = std::atoi(env + 7);
        if (t != 256 && t != 512 && t != 1024) return 0;
        for (LaunchClass& q : rc->hclasses)
            if (!q.lean) q.threads = t;
        if ((*err = hybrid_lean_grid(rc->hclasses, rc->smem_table))) return 0;
        rc->schedule = kSchedHybrid;
    } else if (std::strncmp(env, "hybrid12:", 9) == 0 && !rc->h12classes.empty()) {
        const int t = std::atoi(env + 9);
        if (t != 512 && t != 1024) return 0;
        for (LaunchClass& q : rc->h12classes)
            if (!q.lean) q.threads = t;
        if ((*err = hybrid_lean_grid(rc->h12classes, rc->smem_table))) return 0;
        rc->schedule = kSchedHybrid12;
    } else if (std::strncmp(env, "warp:", 5) == 0 && !rc->wclasses.empty()) {
        const int t = std::atoi(env + 5);
        if (t != 64 && t != 128 && t != 256) return 0;
        if (!set_warp_threads(rc->wclasses, rc->smem_table, t, err)) return 0;
        rc->schedule = kSchedWarp;
    } else if (std::strcmp(env, "classes") == 0) {
        rc->schedule = kSchedClasses;
    } else {
        return 0;
    }
    rc->tuned = true;
    return 1;
}

static int ensure_streams(qtb_plan_device* s) {
    if (s->fork) return QTB_OK;
    QTB_CUDA(cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming));
    for (int i = 0; i < kMaxClasses; ++i) {
        QTB_CUDA(cudaStreamCreateWithFlags(&s->aux[i], cudaStreamNonBlocking));
        QTB_CUDA(cudaEventCreateWithFlags(&s->join[i], cudaEventDisableTiming));
    }
    return QTB_OK;
}

int qtb_plan_run(qtb_plan* plan, int32_t first, int32_t count, const double* params_dev,
                 void* terms_dev, double* energy_dev, void* scratch_dev, void* stream) {
    if (!plan || !terms_dev || (plan->n_params > 0 && !params_dev))
        return fail(QTB_ERR_ARG, "plan_run: null argument");
    if (!plan->uploaded) return fail(QTB_ERR_ARG, "plan_run: plan not uploaded");
    if (first < 0 || count < 1 || first + count > (int32_t)plan->druns.size())
        return fail(QTB_ERR_ARG, "plan_run: network range out of bounds");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RunCache* rc = nullptr;
    int r = get_run(plan, first, count, terms_dev, &rc);
    if (r) return r;
    if (rc->scratch_elems && !scratch_dev)
        return fail(QTB_ERR_ARG, "plan_run: this range needs scratch memory (qtb_plan_scratch_bytes)");
    qtb_plan_device* s = dev_state(plan);
    if ((r = ensure_streams(s))) return r;
    RunArgs a{};
    a.blobs = static_cast<const uint4*>(plan->dev.blobs);
    a.common = static_cast<const uint4*>(plan->dev.entries);
    a.common_bytes = plan->common_bytes;
    a.n_entries = (uint32_t)plan->entries.size();
    a.terms_off = plan->common_terms_off;
    a.table_elems = plan->table_elems;
    a.params = params_dev;
    a.static_first = plan->dynamic_claims ? 0u : 1u;
    a.recs = static_cast<const uint32_t*>(plan->dev.recs);
    a.recs_bytes = (uint32_t)(plan->drecs.size() * sizeof(uint32_t));
    a.runs = static_cast<const DevNetRun*>(plan->dev.runs);
    a.runs_bytes = (uint32_t)std::min<size_t>(plan->druns.size() * sizeof(DevNetRun), 0xffffffffu);
    a.gtable = static_cast<const float2*>(plan->dev.table);
    a.status = static_cast<int*>(plan->dev.status);
    a.done = rc->done;
    a.total_jobs = (uint32_t)count;
    a.terms = static_cast<const float2*>(terms_dev);
    a.energy = energy_dev;
    a.energy_groups = rc->n_groups;
    const int n_entries = (int)plan->entries.size();
    if ((!rc->smem_table || !rc->waves.empty() || rc->n_cl > 0) && n_entries > 0) {
        qtb_table_kernel<<<(n_entries + 127) / 128, 128, 0, st>>>(
            static_cast<const DevEntry*>(plan->dev.entries), n_entries,
            static_cast<const DevTerm*>(plan->dev.terms), params_dev,
            static_cast<float2*>(plan->dev.table));
        QTB_CUDA(cudaGetLastError());
    }
    a.queue = rc->queue;
    if (!rc->tuned && forced_schedule(rc, &r) == 0 && r) return r;
    if (s->autotune && !rc->tuned) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        QTB_CUDA(cudaStreamIsCapturing(st, &cap));
        if (cap == cudaStreamCaptureStatusNone && (r = autotune_run(s, rc, a, scratch_dev, st))) return r;
    }
    s->last = rc;
    const std::vector<LaunchClass>& sched = schedule_of(rc);
    std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
    if (s->timing) {
        if (!s->spare.empty()) {
            ev = s->spare.back();
            s->spare.pop_back();
        } else {
            QTB_CUDA(cudaEventCreate(&ev.first));
            QTB_CUDA(cudaEventCreate(&ev.second));
        }
        QTB_CUDA(cudaEventRecord(ev.first, st));
    }
    if ((r = launch_schedule(s, rc, sched, a, scratch_dev, st))) return r;
    if (s->timing) {
        QTB_CUDA(cudaEventRecord(ev.second, st));
        s->pending.push_back(ev);
        s->kernel_launches += (int64_t)(sched.size() + rc->waves.size() + (rc->n_cl > 0 ? 1 : 0));
    }
    return QTB_OK;
}

// ------------------------------------------------- plain per-bucket run
}  // extern "C"

namespace qtb {

// Energy of a plain run: one CTA, the same compensated sum as the executor.
__global__ void __launch_bounds__(256) qtb_energy_kernel(const float2* terms, uint32_t n,
                                                         double n_groups, double* energy) {
    reduce_energy(terms, n, n_groups, energy);
}

// Circuits (groups) of networks [first, first+count): networks of a circuit
// are contiguous, so this counts group changes.
static int32_t count_groups(const qtb_plan* plan, int32_t first, int32_t count) {
    int32_t groups = 0, last = -1;
    for (int32_t i = first; i < first + count; ++i)
        if (plan->nets[i].info.group != last) {
            last = plan->nets[i].info.group;
            ++groups;
        }
    return groups;
}

}  // namespace qtb

extern "C" {

int qtb_plan_plain_scratch_bytes(const qtb_plan* plan, int32_t first, int32_t count, size_t* bytes) {
    if (!plan || !bytes) return fail(QTB_ERR_ARG, "plan_plain_scratch_bytes: null argument");
    if (first < 0 || count < 1 || first + count > (int32_t)plan->nets.size())
        return fail(QTB_ERR_ARG, "plan_plain_scratch_bytes: network range out of bounds");
    size_t elems = 0;
    for (int32_t i = first; i < first + count; ++i)
        elems = std::max<size_t>(elems, (size_t)plan->nets[i].info.arena_elems);
    *bytes = 8 * elems;
    return QTB_OK;
}

int qtb_plan_run_plain(qtb_plan* plan, int32_t first, int32_t count, const double* params_dev,
                       void* terms_dev, double* energy_dev, void* scratch_dev, size_t scratch_bytes,
                       void* stream) {
    if (!plan || !terms_dev || (plan->n_params > 0 && !params_dev))
        return fail(QTB_ERR_ARG, "plan_run_plain: null argument");
    if (!plan->uploaded) return fail(QTB_ERR_ARG, "plan_run_plain: plan not uploaded");
    {
        std::lock_guard<std::mutex> lock(plan->mu);
        ensure_flat(plan);   // the flattened arrays are built on first use
    }
    if (first < 0 || count < 1 || first + count > (int32_t)plan->dnets.size())
        return fail(QTB_ERR_ARG, "plan_run_plain: network range out of bounds");
    size_t need = 0;
    int r = qtb_plan_plain_scratch_bytes(plan, first, count, &need);
    if (r) return r;
    if (need > 0 && (!scratch_dev || scratch_bytes < need))
        return fail(QTB_ERR_ARG, "plan_run_plain: scratch smaller than qtb_plan_plain_scratch_bytes");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n_entries = (int)plan->entries.size();
    if (n_entries > 0) {
        qtb_table_kernel<<<(n_entries + 127) / 128, 128, 0, st>>>(
            static_cast<const DevEntry*>(plan->dev.entries), n_entries,
            static_cast<const DevTerm*>(plan->dev.terms), params_dev,
            static_cast<float2*>(plan->dev.table));
        QTB_CUDA(cudaGetLastError());
    }
    const float2* table = static_cast<const float2*>(plan->dev.table);
    float2* arena = static_cast<float2*>(scratch_dev);
    float2* terms = static_cast<float2*>(terms_dev);
    // networks run one after another on st, so they share one arena
    for (int32_t i = first; i < first + count; ++i) {
        const DevNet& net = plan->dnets[i];
        for (uint32_t o = 0; o < net.n_ops; ++o) {
            const DevOp& op = plan->dops[net.op_begin + o];
            if (op.k < 1 || op.k > QTB_MAX_BUCKET_INPUTS)
                return fail(QTB_ERR_UNSUPPORTED, "plan_run_plain: bucket of more than 16 tensors");
            BucketArgs a{};
            for (int t = 0; t < op.k; ++t) {
                const DevIn& in = plan->dins[op.in_begin + t];
                a.in[t] = (in.src & kSrcTable) ? table + (in.src & ~kSrcTable) : arena + in.src;
                bucket_operand(&a, t, in.mask, op.u, op.sum);
            }
            a.out = arena + op.dst;
            a.k = op.k;
            a.sum = op.sum;
            a.w = op.u - op.sum;
            qtb_bucket_kernel<<<bucket_blocks(a.w), kBucketThreads, 0, st>>>(a);
            QTB_CUDA(cudaGetLastError());
        }
        const float2* res = (net.result_src & kSrcTable) ? table + (net.result_src & ~kSrcTable)
                                                         : arena + net.result_src;
        QTB_CUDA(cudaMemcpyAsync(terms + (i - first), res, sizeof(float2), cudaMemcpyDeviceToDevice, st));
    }
    if (energy_dev) {
        qtb_energy_kernel<<<1, 256, 0, st>>>(terms, (uint32_t)count,
                                             (double)count_groups(plan, first, count), energy_dev);
        QTB_CUDA(cudaGetLastError());
    }
    return QTB_OK;
}

// ------------------------------------------------- failure detection self-test
}  // extern "C"

namespace qtb {

// One thread waits, with the executor's bounded wait, on a counter that
// nothing increments; it gives up after `limit` polls and reports through
// the status word, as a wide-network step whose predecessor never finishes
// would.  Only the counter word and the status word are touched.
__global__ void qtb_selftest_wait_kernel(const unsigned int* counter, uint32_t limit, int* status) {
    if (threadIdx.x == 0 && blockIdx.x == 0) wait_counter(counter, 1u, limit, status, kStatusWideTimeout);
}

}  // namespace qtb

extern "C" {

namespace qtb {
// 8-byte words from src to dst, both device-accessible (device memory, or
// pinned host memory through its device mapping).
__global__ void qtb_copy_kernel(const unsigned long long* __restrict__ src, unsigned long long* __restrict__ dst,
                                size_t words) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}
}  // namespace qtb

int qtb_host_device_pointer(void* host, void** dev) {
    if (!host || !dev) return fail(QTB_ERR_ARG, "host_device_pointer: null argument");
    QTB_CUDA(cudaHostGetDevicePointer(dev, host, 0));
    return QTB_OK;
}

int qtb_copy_c(void* dst, const void* src, size_t bytes, void* stream) {
    if (!dst || !src || bytes % 8 != 0) return fail(QTB_ERR_ARG, "copy: null pointer or size not a multiple of 8");
    if (bytes == 0) return QTB_OK;
    const size_t words = bytes / 8;
    const unsigned blocks = (unsigned)std::min<size_t>((words + 255) / 256, 1024);
    qtb_copy_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const unsigned long long*>(src), static_cast<unsigned long long*>(dst), words);
    QTB_CUDA(cudaGetLastError());
    return QTB_OK;
}

int qtb_selftest_wait_timeout(int32_t spin_limit, int32_t* status_out) {
    if (!status_out || spin_limit < 1) return fail(QTB_ERR_ARG, "selftest_wait_timeout: bad arguments");
    void* buf = nullptr;
    QTB_CUDA(cudaMalloc(&buf, 16));
    int r = QTB_OK;
    unsigned int* counter = static_cast<unsigned int*>(buf);
    int* status = reinterpret_cast<int*>(static_cast<char*>(buf) + 8);
    cudaError_t e = cudaMemset(buf, 0, 16);
    if (e == cudaSuccess) {
        qtb_selftest_wait_kernel<<<1, 32>>>(counter, (uint32_t)spin_limit, status);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(status_out, status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) r = cuda_fail(e, "selftest_wait_timeout");
    cudaFree(buf);
    return r;
}

// ------------------------------------------------- allocation-free run
}  // extern "C"

namespace qtb {

// Library-owned scratch of qtb_plan_run_noalloc: [completion counter, 256 B]
// [unused, 256 B][jobs, 16 B each, rounded to 256 B][arenas].  Host code
// must not take this symbol's address as a device pointer; the device
// address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[QTB_NOALLOC_SCRATCH_BYTES];

constexpr int kNoallocMaxDevices = 64;
static void* g_noalloc_addr[kNoallocMaxDevices] = {};
static std::mutex g_noalloc_mu;

// Jobs of a contiguous network range, written on the device.
__global__ void qtb_noalloc_jobs_kernel(Job* jobs, const DevNetRun* runs, int32_t first,
                                        int32_t count, float2* terms) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        jobs[i].net = runs[first + i];
        jobs[i].term = terms + i;
        jobs[i].pad = 0;
    }
}

// Once per device, with that device current: the scratch array's device
// address and the kernels' shared-memory limits.
static int noalloc_setup(int device, unsigned char** out) {
    if (device < 0 || device >= kNoallocMaxDevices)
        return fail(QTB_ERR_UNSUPPORTED, "run_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* ptr = nullptr;
        QTB_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        QTB_CUDA((allow_smem<false, true, false>()));
        QTB_CUDA((allow_smem<false, false, false>()));
        g_noalloc_addr[device] = ptr;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[device]);
    return QTB_OK;
}

}  // namespace qtb

extern "C" {

int qtb_plan_run_noalloc(qtb_plan* plan, int32_t first, int32_t count, const double* params_dev,
                         void* terms_dev, double* energy_dev, void* stream) {
    if (!plan || !terms_dev || (plan->n_params > 0 && !params_dev))
        return fail(QTB_ERR_ARG, "run_noalloc: null argument");
    if (!plan->uploaded) return fail(QTB_ERR_ARG, "run_noalloc: plan not uploaded");
    if (first < 0 || count < 1 || first + count > (int32_t)plan->druns.size())
        return fail(QTB_ERR_ARG, "run_noalloc: network range out of bounds");
    int device = 0;
    QTB_CUDA(cudaGetDevice(&device));
    if (device != plan->device) return fail(QTB_ERR_ARG, "run_noalloc: plan uploaded to another device");
    unsigned char* scratch = nullptr;
    int r = noalloc_setup(device, &scratch);
    if (r) return r;
    // one launch: every network of the range in a global arena slice
    const bool smem_table = plan->table_elems <= kSmemTableLimitElems;
    const size_t fixed = fixed_smem(plan, smem_table);
    uint32_t cap = 4, blob = 16, maxe = 1;
    for (int32_t i = first; i < first + count; ++i) {
        cap = std::max(cap, plan->druns[i].arena_elems);
        blob = std::max(blob, plan->druns[i].blob_bytes);
        maxe = std::max(maxe, plan->druns[i].max_elems);
    }
    cap = (cap + 3u) & ~3u;
    // a range whose largest blob does not fit shared memory reads every
    // blob from global memory (blob capacity 0), as qtb_plan_run's global
    // classes do
    if (fixed + blob > kSmemLimitBytes) blob = 0;
    const size_t smem_bytes = fixed + blob;
    const size_t jobs_off = 512;
    const size_t arenas_off = jobs_off + (((size_t)count * sizeof(Job) + 255) & ~size_t(255));
    const size_t need = arenas_off + (size_t)count * cap * sizeof(float2);
    if (need > QTB_NOALLOC_SCRATCH_BYTES)
        return fail(QTB_ERR_UNSUPPORTED,
                    "run_noalloc: " + std::to_string(count) + " networks of arena " +
                        std::to_string(cap) + " need " + std::to_string(need) +
                        " bytes of scratch, more than the static " +
                        std::to_string((size_t)QTB_NOALLOC_SCRATCH_BYTES) + "; split the range");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned int* done = reinterpret_cast<unsigned int*>(scratch);
    Job* jobs = reinterpret_cast<Job*>(scratch + jobs_off);
    float2* arenas = reinterpret_cast<float2*>(scratch + arenas_off);
    QTB_CUDA(cudaMemsetAsync(done, 0, 256, st));
    qtb_noalloc_jobs_kernel<<<(count + 255) / 256, 256, 0, st>>>(
        jobs, static_cast<const DevNetRun*>(plan->dev.runs), first, count,
        static_cast<float2*>(terms_dev));
    QTB_CUDA(cudaGetLastError());
    const int n_entries = (int)plan->entries.size();
    if (!smem_table && n_entries > 0) {
        qtb_table_kernel<<<(n_entries + 127) / 128, 128, 0, st>>>(
            static_cast<const DevEntry*>(plan->dev.entries), n_entries,
            static_cast<const DevTerm*>(plan->dev.terms), params_dev,
            static_cast<float2*>(plan->dev.table));
        QTB_CUDA(cudaGetLastError());
    }
    RunArgs a{};
    a.blobs = static_cast<const uint4*>(plan->dev.blobs);
    a.common = static_cast<const uint4*>(plan->dev.entries);
    a.common_bytes = plan->common_bytes;
    a.n_entries = (uint32_t)n_entries;
    a.terms_off = plan->common_terms_off;
    a.table_elems = plan->table_elems;
    a.params = params_dev;
    a.static_first = plan->dynamic_claims ? 0u : 1u;
    a.gtable = static_cast<const float2*>(plan->dev.table);
    a.gscratch = arenas;
    a.arena_capacity = cap;
    a.blob_capacity = blob;
    a.status = static_cast<int*>(plan->dev.status);
    a.done = done;
    a.queue = nullptr;
    a.n_jobs = (uint32_t)count;
    a.total_jobs = (uint32_t)count;
    a.terms = static_cast<const float2*>(terms_dev);
    a.energy = energy_dev;
    a.energy_groups = 0.0;
    for (int32_t i = first; i < first + count; ++i)
        if (i == first || plan->nets[i].info.group != plan->nets[i - 1].info.group) a.energy_groups += 1.0;
    const int threads = threads_for(maxe);
    if (smem_table)
        qtb_network_kernel<false, true, false><<<count, threads, smem_bytes, st>>>(jobs, a);
    else
        qtb_network_kernel<false, false, false><<<count, threads, smem_bytes, st>>>(jobs, a);
    QTB_CUDA(cudaGetLastError());
    return QTB_OK;
}

int qtb_plan_set_wave_ctas_per_sm(qtb_plan* plan, int32_t ctas) {
    if (!plan || ctas < 0) return fail(QTB_ERR_ARG, "plan_set_wave_ctas_per_sm: bad arguments");
    plan->wave_ctas_per_sm = ctas;
    return QTB_OK;
}

int qtb_plan_set_dynamic_claims(qtb_plan* plan, int32_t enable) {
    if (!plan) return fail(QTB_ERR_ARG, "plan_set_dynamic_claims: bad arguments");
    plan->dynamic_claims = enable != 0;
    return QTB_OK;
}

int qtb_plan_set_autotune(qtb_plan* plan, int32_t enable) {
    if (!plan) return fail(QTB_ERR_ARG, "plan_set_autotune: null plan");
    // QTB_AUTOTUNE=0 in the environment keeps the default block sizes (e.g.
    // under a profiler, whose serialised replays would mislead the timing)
    const char* env = std::getenv("QTB_AUTOTUNE");
    dev_state(plan)->autotune = enable != 0 && !(env && env[0] == '0');
    return QTB_OK;
}

int qtb_plan_last_launch_config(qtb_plan* plan, int32_t* out, int32_t cap, int32_t* n_classes) {
    if (!plan || !n_classes) return fail(QTB_ERR_ARG, "plan_last_launch_config: bad arguments");
    const RunCache* rc = dev_state(plan)->last;
    if (!rc) {
        *n_classes = 0;
        return QTB_OK;
    }
    const std::vector<LaunchClass>& sched = schedule_of(rc);
    *n_classes = (int32_t)(sched.size() + rc->waves.size() + (rc->n_cl > 0 ? 1 : 0));
    if (!out) return QTB_OK;
    for (int32_t c = 0; c < *n_classes && 4 * c + 3 < cap; ++c) {
        if (c < (int32_t)sched.size()) {
            const LaunchClass& lc = sched[c];
            out[4 * c] = lc.n_jobs;
            out[4 * c + 1] = lc.threads;
            out[4 * c + 2] = (int32_t)lc.smem_bytes;
            out[4 * c + 3] = (lc.smem ? 1 : 0) | (lc.persistent ? 2 : 0) | (lc.lean ? 8 : 0) | (lc.warp ? 16 : 0) |
                             (lc.lean == 2 ? 32 : 0) | (lc.records ? 128 : 0);
        } else if (c < (int32_t)(sched.size() + rc->waves.size())) {
            const WideWave& wv = rc->waves[c - sched.size()];
            out[4 * c] = (int32_t)wv.n_nets;
            out[4 * c + 1] = kWideThreads;
            out[4 * c + 2] = 0;
            out[4 * c + 3] = 4;
        } else {   // the cluster launch (one cluster of kClusterCtas CTAs per network)
            out[4 * c] = rc->n_cl;
            out[4 * c + 1] = kClusterThreads;
            out[4 * c + 2] = 0;
            out[4 * c + 3] = 64;
        }
    }
    return QTB_OK;
}

int qtb_plan_device_bytes(const qtb_plan* plan, size_t* bytes) {
    if (!plan || !bytes) return fail(QTB_ERR_ARG, "plan_device_bytes: bad arguments");
    // images qtb_plan_upload sends, gate table, jobs of both schedules
    size_t b = 0, blob = 0;
    for (const Network& n : plan->nets) {
        blob += n.phases.size() * sizeof(DevPhase) + n.ops.size() * sizeof(DevOp) +
                n.ins.size() * sizeof(DevIn) + 16;
        if (8 * (uint64_t)n.info.arena_elems <= kSmemLimitBytes)   // chunk tables
            for (const DevPhase& ph : n.phases) blob += 2 * ((ph.total_elems + kChunkElems - 1) / kChunkElems);
    }
    b += blob + plan->nets.size() * (sizeof(DevNetRun) + 2 * sizeof(Job));
    // element records (an upper bound: one copy per network, not per distinct blob)
    if (plan->records && plan->table_elems <= kSmemTableLimitElems) {
        uint64_t words = 0;
        for (const Network& n : plan->nets) {
            if (8 * (uint64_t)n.info.arena_elems > kSmemLimitBytes) continue;
            words += 2 * n.phases.size();
            for (const DevPhase& ph : n.phases) {
                uint32_t kmax = 1;
                for (uint32_t o = ph.op_first; o < ph.op_first + ph.op_count; ++o)
                    kmax = std::max<uint32_t>(kmax, n.ops[o].k);
                words += (uint64_t)(kmax + 1) * ph.total_elems;
            }
        }
        b += 4 * (size_t)std::min<uint64_t>(words, kRecMaxWords);
    }
    b += plan->entries.size() * sizeof(DevEntry) + plan->terms.size() * sizeof(DevTerm) + 64;
    b += (size_t)plan->table_elems * sizeof(float2);
    *bytes = b;
    return QTB_OK;
}

int qtb_plan_device_status(qtb_plan* plan, int32_t* status) {
    if (!plan || !status) return fail(QTB_ERR_ARG, "plan_device_status: bad arguments");
    if (!plan->uploaded) {
        *status = 0;
        return QTB_OK;
    }
    int v = 0;
    QTB_CUDA(cudaMemcpy(&v, plan->dev.status, sizeof(int), cudaMemcpyDeviceToHost));
    *status = v;
    return QTB_OK;
}

// Kernel timing of the network executor launches (CUDA events on the run's
// stream): enable, then read the accumulated milliseconds after each run.
int qtb_plan_set_timing(qtb_plan* plan, int32_t enable) {
    if (!plan) return fail(QTB_ERR_ARG, "plan_set_timing: null plan");
    qtb_plan_device* s = dev_state(plan);
    for (auto& e : s->pending) {
        cudaEventSynchronize(e.second);
        s->spare.push_back(e);
    }
    s->pending.clear();
    s->timing = enable != 0;
    s->kernel_ms = 0.0;
    s->kernel_launches = 0;
    return QTB_OK;
}

int qtb_plan_collect_timing(qtb_plan* plan, double* total_ms, int64_t* launches) {
    if (!plan || !total_ms || !launches) return fail(QTB_ERR_ARG, "plan_collect_timing: bad arguments");
    qtb_plan_device* s = dev_state(plan);
    for (auto& e : s->pending) {
        QTB_CUDA(cudaEventSynchronize(e.second));
        float ms = 0.f;
        QTB_CUDA(cudaEventElapsedTime(&ms, e.first, e.second));
        s->kernel_ms += ms;
        s->spare.push_back(e);
    }
    s->pending.clear();
    *total_ms = s->kernel_ms;
    *launches = s->kernel_launches;
    return QTB_OK;
}

int qtb_plan_destroy(qtb_plan* plan) {
    if (!plan) return QTB_OK;
    free_device(plan);
    {
        std::lock_guard<std::mutex> lock(g_dev_mu);
        auto it = g_dev.find(plan);
        if (it != g_dev.end()) {
            destroy_streams(it->second);
            delete it->second;
            g_dev.erase(it);
        }
    }
    delete plan;
    return QTB_OK;
}

}  // extern "C"
