// Internal plan structures shared by the host plan compiler (plan.cpp) and
// the device executor (qtb.cu).  Not part of the public C ABI.
#pragma once
#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/qtb.h"

namespace qtb {

// Flag on DevIn::src / DevNet::result_src: the operand lives in the gate
// table, not in the network's arena.
constexpr uint32_t kSrcTable = 0x80000000u;

// One bucket kernel of a network (device layout, 16 bytes).
struct DevOp {
    uint8_t u;          // live (binary) variables in the bucket's union
    uint8_t sum;        // 1: sum over union variable 0 (the bucket variable)
    uint8_t k;          // number of input tensors
    uint8_t pad;
    uint32_t dst;       // arena offset of the output (complex64 elements)
    uint32_t elem_begin;  // first flattened element of this op within its phase
    uint32_t in_begin;  // index of the first DevIn of this op
};

// One operand of an op: which union bits it holds, where it lives, and the
// bit gather from an output index to the operand's index precompiled as
// contiguous runs; bits 60..62 of `runs` hold the run count n.
//   n <= 1: bits 0..31 = length mask of the run, bits 32..36 = its start
//           (the gather is (j >> start) & lenmask; 0 when n == 0);
//   2 <= n <= kMaxRuns: run r (10 bits at 10*r) = start | len << 5 moves
//           bits [start, start+len) of j to the next free operand bits
//           (runs in increasing start order, packed from bit 0 up);
//   n == kRunsFallback: more runs than kMaxRuns, gather bit by bit.
struct DevIn {
    uint32_t mask;      // bit (u-1-v) set <=> union variable v is an axis
    uint32_t src;       // arena offset, or kSrcTable | gate-table offset
    uint64_t runs;
};
constexpr int kMaxRuns = 6;
constexpr uint64_t kRunsFallback = 7;

// Ops of one dependency level; a barrier follows every phase.  In a network
// blob, chunk_off is the byte offset of the phase's chunk table: for every
// 32 flattened elements, the (network-local) index of the op holding the
// chunk's first element.  Only networks whose arena can be in shared
// memory have chunk tables (chunk_off 0 otherwise).
struct DevPhase {
    uint32_t op_first;
    uint32_t op_count;
    uint32_t total_elems;
    uint32_t chunk_off;
};

// One network (edge term).
struct DevNet {
    uint32_t op_begin;
    uint32_t n_ops;
    uint32_t phase_begin;
    uint32_t n_phases;
    uint32_t arena_elems;
    uint32_t result_src;   // arena offset or kSrcTable | offset of the scalar
    uint32_t max_elems;    // largest op output (elements)
    uint32_t pad;
};

// One network as the executor reads it: its phases, ops and operands are
// one contiguous 16-byte-aligned blob [DevPhase x n_phases][DevOp x n_ops]
// [DevIn x n_ins][uint16 chunk tables of all phases, padded to 16 bytes]
// with network-local indices, staged into shared memory by one bulk copy.
struct DevNetRun {
    uint32_t blob_off16;   // blob offset in 16-byte units
    uint32_t blob_bytes;   // multiple of 16
    uint32_t n_phases;
    uint32_t ins_off;      // byte offset of the DevIn array within the blob
    uint32_t arena_elems;
    uint32_t result_src;
    uint32_t max_elems;
    uint32_t tail_start;   // phases from here on have <= 32 elements each
    uint32_t rec_off;      // first word of the network's element records
    uint32_t rec_words;    // 0: the network has no element records
    uint32_t rec_format;   // kRecWide or kRecCompact (when rec_words != 0)
    uint32_t pad1;
};

// Element records of a network (u32 words at DevNetRun::rec_off, a multiple
// of 4, in the plan's record array), for executors whose gate table and arena share one
// shared-memory window S = [gate table, padded to an even element count]
// [arena]:
//   [phase header x n_phases][phase payloads]
//   header p: word 0 = payload offset (words from rec_off),
//             word 1 = elements of the phase | (largest operand count) << 24
//   payload p, element g (kmax + 1 rows of `elements` words, row-major):
//     row 0     = S offset of the output | k << 16 | sum << 24
//     row 1 + t = operand t: S offset at the summed variable 0 (low 16 bits)
//                 and at 1 (high 16 bits; equal when the operand lacks it)
// Every offset the bit gathers of the op would compute is resolved on the
// host, so the executor only loads and multiplies.  That is the wide
// format (kRecWide).  A network whose window has at most kRecCompactWindow
// elements and whose ops have at most kRecCompactMaxK operands uses the
// compact format (kRecCompact) instead: the same headers, padded to 16
// bytes, then per phase one 16-byte record per element (element-major),
// eight 16-bit fields:
//     field 0     = S offset of the output | (k - 1) << 12 | sum << 15
//     field 1 + t = operand t: S offset at the summed variable 0 | c << 12,
//                   its offset at 1 being that + ((1 << c) >> 1)
// (c = 0 when the operand lacks the summed variable; 0 for t >= k).
constexpr uint32_t kRecWide = 1;
constexpr uint32_t kRecCompact = 2;
constexpr uint32_t kRecCompactWindow = 4096;
constexpr uint32_t kRecCompactMaxK = 7;
constexpr uint32_t kRecMaxK = 8;                    // operands per op with records
constexpr uint64_t kRecMaxWords = uint64_t(1) << 26;   // record words per plan (256 MiB)
constexpr uint32_t kSmemTableLimitElems = 2048;   // 16 KB of gate table per CTA
// Dynamic shared memory a CTA may use (B200: 227 KB per block).
constexpr uint32_t kSmemLimitBytes = 224 * 1024;

// Gate-table entry: the tensor of a gate, sliced and transposed into the
// sorted-variable layout the network reads (device layout).
struct DevEntry {
    int32_t kind;
    int32_t expr_begin;    // into the DevTerm array
    int32_t expr_count;
    uint32_t off;          // complex64 offset in the gate table
    int8_t rank_in;        // axes of the gate tensor as generated
    int8_t rank_out;       // axes kept (not sliced)
    uint8_t sliced_mask;   // native axes fixed to a value
    int8_t perm[4];        // output axis a <- native axis perm[a]
    uint8_t sliced_value;  // the values of the sliced axes (bit per native axis)
};

struct DevTerm {
    int32_t param;
    int32_t pad;
    double coef;
};

static_assert(sizeof(DevOp) == 16, "DevOp layout");
static_assert(sizeof(DevIn) == 16, "DevIn layout");
static_assert(sizeof(DevPhase) == 16, "DevPhase layout");
static_assert(sizeof(DevNet) == 32, "DevNet layout");
static_assert(sizeof(DevNetRun) == 48, "DevNetRun layout");
constexpr uint32_t kChunkElems = 32;
static_assert(sizeof(DevEntry) == 24, "DevEntry layout");
static_assert(sizeof(DevTerm) == 16, "DevTerm layout");

// Linear angle expression: sum coef_i * params[param_i], sorted by param.
using Expr = std::vector<std::pair<int32_t, double>>;

struct EntryKey {
    int32_t kind;
    Expr expr;
    int8_t rank_in;
    uint8_t sliced_mask;
    uint8_t sliced_value;
    std::vector<int8_t> perm;
    bool operator<(const EntryKey& o) const;
};

// A simplifier decision that holds only for some angles.
struct AngleCheck {
    Expr expr;
    bool must_be_small;   // true: |expr| < 1e-5 (cancelled); false: >= 1e-5 (merged)
};

// Largest network arena (complex64 elements, 16 GiB): arena offsets must
// stay below the kSrcTable flag bit, and a wide wave rounds each arena up
// to 64 elements inside 31-bit element counts.
constexpr uint64_t kMaxArenaElems = (uint64_t(1) << 31) - 64;

// Most variables sliced per circuit (2^k networks).
constexpr int kMaxSlicedVars = 16;
// Most output qubits of an amplitude batch (2^k amplitudes per circuit).
constexpr int kMaxBatchVars = 16;

struct Network {
    qtb_network_info info{};
    std::vector<int32_t> peo;          // qtree-layout variable ids
    std::vector<DevOp> ops;
    std::vector<DevIn> ins;            // src of table operands: kSrcTable | local entry id
    std::vector<DevPhase> phases;
    std::vector<EntryKey> entries;     // local gate-table entries
    std::vector<AngleCheck> checks;
    uint32_t result_src = 0;
    uint32_t max_elems = 1;
};

struct DeviceBuffers {
    void* runs = nullptr;         // DevNetRun per network
    void* blobs = nullptr;        // concatenated network blobs
    void* entries = nullptr;      // common image: gate entries then angle terms
    void* terms = nullptr;        // inside the entries allocation
    void* recs = nullptr;         // element records (u32 words)
    void* table = nullptr;        // complex64 gate table
    void* status = nullptr;       // int error word
};

}  // namespace qtb

struct qtb_plan {
    int32_t n_params = 0;
    int32_t order_trials = 0;   // extra randomized greedy orders per network
    bool share_lightcones = true;   // isomorphic lightcones share one compile
    int32_t max_width = 0;      // slice circuits whose width reaches this (0 = never)
    int32_t max_slices = 256;   // networks one sliced circuit may become
    int32_t slicing = QTB_SLICE_GREEDY;   // how sliced variables are chosen
    int32_t wave_ctas_per_sm = 0;   // resident CTAs per SM of a wide wave (0: as many as fit)
    bool dynamic_claims = false;    // persistent CTAs claim their first network from the queue too
    int32_t n_groups = 0;       // circuits added (networks of a circuit share a group)
    std::vector<qtb::Network> nets;
    // global gate table, built from the networks' local entries
    std::map<qtb::EntryKey, int32_t> entry_index;
    std::vector<qtb::DevEntry> entries;
    std::vector<qtb::DevTerm> terms;
    uint32_t table_elems = 0;
    std::vector<qtb::AngleCheck> checks;   // distinct decisions over all networks
    std::set<std::pair<bool, qtb::Expr>> check_index;
    // flattened device images
    std::vector<qtb::DevNet> dnets;
    std::vector<qtb::DevOp> dops;
    std::vector<qtb::DevIn> dins;
    std::vector<qtb::DevPhase> dphases;
    std::vector<qtb::DevNetRun> druns;
    std::vector<uint8_t> dblobs;
    std::vector<uint32_t> drecs;     // element records (DevNetRun::rec_off)
    bool records = true;             // build element records for shared-memory executors
    bool images_valid = false;       // druns, dblobs and drecs match `nets`
    bool flat_valid = false;         // dnets, dops, dins and dphases match `nets`
    uint32_t common_bytes = 0;       // staged gate entries + angle terms
    uint32_t common_terms_off = 0;
    bool uploaded = false;
    int device = -1;
    qtb::DeviceBuffers dev;
    std::mutex mu;
};

namespace qtb {
// plan.cpp
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int compile_circuit(int32_t n_qubits, const qtb_gate* gates, int32_t n_gates,
                    int32_t simplify_passes, const double* params, int32_t n_params,
                    int32_t order_trials, int32_t max_width, int32_t max_slices, int32_t slicing,
                    int32_t batch_vars, std::vector<Network>* outs, std::string* err,
                    const std::atomic<bool>* abort = nullptr);
// compile_circuit's result when `abort` was raised while it ran.
constexpr int kCompileAborted = -1;
// Canonical structural key of an edge's lightcone (see plan.cpp).
void cone_key(int32_t n_nodes, const int64_t* indptr, const int32_t* indices, int32_t u, int32_t v,
              int32_t p, std::vector<int32_t>* key);
int build_lightcone(int32_t n_nodes, const int64_t* indptr, const int32_t* indices,
                    int32_t u, int32_t v, int32_t p, int32_t composer,
                    std::vector<qtb_gate>* gates, int32_t* n_qubits, std::string* err);
void merge_network(qtb_plan* plan, Network&& net, int32_t group);
void flatten_plan(qtb_plan* plan);
// build_blobs (the executors' per-network images) unless they already
// match the networks.
void ensure_images(qtb_plan* plan);
// flatten_plan (the plain path's and the export's arrays) likewise.
void ensure_flat(qtb_plan* plan);
uint64_t encode_runs(uint32_t mask, uint32_t w);
void build_blobs(qtb_plan* plan);
int rank_of_kind(int32_t kind);
}  // namespace qtb
