/*
 * qtb.h -- C ABI of the qtensor_b200 bucket-elimination engine (libqtb.so).
 *
 * Plain pointers, sizes and integer status codes (0 = ok); no exception or
 * device trap crosses this boundary.  Device buffers are caller-owned (any
 * allocator, e.g. torch tensors' data_ptr()); the CUDA stream is passed
 * explicitly as a void* (cudaStream_t; NULL = legacy default stream).
 *
 * Reference interfaces replaced (paths within DaniloZZZ/QTensor):
 *   qtb_bucket_c64      <- BucketBackend.process_bucket
 *                          qtensor/ProcessingFrameworks.py:14-15 (NumpyBackend :29-31,
 *                          semantics restated by CMKLExtendedBackend :45-147,
 *                          tcontract.mkl_contract_complex/_sum call sites :65-66, :129-130)
 *   qtb_plan_*          <- the per-edge host graph work of
 *                          QtreeSimulator.simulate_batch qtensor/Simulate.py:66-94
 *                          (circ2buckets, OrderingOptimizer.optimize
 *                          qtensor/optimisation/Optimizer.py:65-87, reorder_buckets,
 *                          slicing) and of the DefaultQAOAComposer simplifier
 *                          qtensor/simplify_circuit/simplify_circuit.py:78-138
 *   qtb_plan_run        <- qtree.optimizer.bucket_elimination driven by
 *                          BucketBackend.process_bucket (Simulate.py:90-94), for
 *                          every edge of QAOASimulator.energy_expectation
 *                          qtensor/QAOASimulator.py:44-66 (+ _post_process_energy :27-41)
 *   qtb_plan_run_plain  <- the same, one process_bucket launch per bucket
 *   qtb_plan_add_circuit_batch <- QtreeSimulator.simulate_batch(qc, batch_vars)
 *                          qtensor/Simulate.py:66-94 (free output qubits)
 *   qtb_plan_set_max_width <- FeynmanSimulator slicing, qtensor/FeynmanSimulator.py:49-84
 *                          with SlicesOptimizer / GreedyParvars
 *   qtb_contract_*      <- tcontract.mkl_contract_complex / mkl_contract_sum of
 *                          CMKLExtendedBackend (ProcessingFrameworks.py:41-147)
 *   qtb_last_error      <- Python exceptions raised by the reference backends
 * Entry points without a counterpart in the reference are marked where they
 * are declared (allocation-free run, failure-detection self-test).
 */
#ifndef QTB_H
#define QTB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QTB_OK 0
#define QTB_ERR_ARG 1        /* invalid argument (sizes, masks, pointers) */
#define QTB_ERR_CUDA 2       /* a CUDA runtime call failed */
#define QTB_ERR_UNSUPPORTED 3
#define QTB_ERR_DEVICE 4     /* a kernel reported an error status */

#define QTB_MAX_BUCKET_INPUTS 16
#define QTB_MAX_BUCKET_VARS 31

/* ---------------------------------------------------------------- misc */
/* Library version string. */
const char* qtb_version(void);
/* Select/initialise a CUDA device; safe to call repeatedly. */
int qtb_init(int device);
/* Copy the last error message of the calling thread into buf (NUL-terminated). */
int qtb_last_error(char* buf, size_t len);

/* ------------------------------------------------- K1: one bucket (plain path)
 * All variables are binary.  The bucket's union of variables is sorted by
 * variable id; union variable 0 (the bucket variable, smallest id) is the
 * most significant bit of a row-major union index, union variable n_vars-1
 * the least significant.  Input t holds the union variables whose bits are
 * set in masks[t] (bit (n_vars-1-v) <-> union variable v), row-major in
 * increasing variable id.  The output is the product of all inputs over the
 * union, summed over union variable 0 when sum_first != 0 (then it has
 * n_vars-1 variables), row-major complex64.                               */
typedef struct {
    int32_t n_inputs;                        /* 1..QTB_MAX_BUCKET_INPUTS */
    int32_t n_vars;                          /* 0..QTB_MAX_BUCKET_VARS */
    int32_t sum_first;                       /* 0/1; needs n_vars >= 1 */
    uint32_t masks[QTB_MAX_BUCKET_INPUTS];
} qtb_bucket_desc;

/* inputs: n_inputs device pointers to complex64 arrays; output: device
 * complex64 array of 2^(n_vars - sum_first) elements. Asynchronous on stream. */
int qtb_bucket_c64(const qtb_bucket_desc* desc, const void* const* inputs,
                   void* output, void* stream);

/* ------------------------------------------------- merged-index contractions
 * The two products of the reference's extended bucket backend
 * CMKLExtendedBackend (qtensor/ProcessingFrameworks.py:41-147), whose native
 * module tcontract (an MKL extension) the reference does not ship; complex64,
 * row-major, device pointers, asynchronous on stream.
 *   qtb_contract_outer_c64  <- tcontract.mkl_contract_complex (:65-66):
 *                              c[n,m,k] = a[n,m] * b[n,k]
 *   qtb_contract_sum_c64    <- tcontract.mkl_contract_sum (:129-130):
 *                              C[f,m,n] = sum_k A[k,f,m] * B[k,f,n]
 * The contract-sum runs on the tcgen05 tensor cores (mode 2, or mode 0 when
 * K >= 32 and M, N >= 64): complex products in 3xTF32 (each operand split
 * into TF32 high and low parts), FP32 accumulation in tensor memory per
 * 32-k block, the blocks summed in FP32 registers with round-to-nearest,
 * 128 x 64 complex output tiles; else (mode 1, or mode 0 for smaller shapes) on the CUDA
 * cores in FP32.  scratch (qtb_contract_sum_scratch_bytes for the same
 * shape and mode) holds the split operands; its first 4 bytes are a status
 * word, 0 after a good run, 2 when a staging copy or the MMAs did not
 * complete within the kernel's bounded wait.                              */
int qtb_contract_outer_c64(const void* a, const void* b, void* c, int64_t n, int64_t m, int64_t k,
                           void* stream);
int qtb_contract_sum_scratch_bytes(int64_t K, int64_t F, int64_t M, int64_t N, int32_t mode, size_t* bytes);
int qtb_contract_sum_c64(const void* A, const void* B, void* C, int64_t K, int64_t F, int64_t M, int64_t N,
                         int32_t mode, void* scratch, size_t scratch_bytes, void* stream);

/* ------------------------------------------------- plan compiler (host C++) */
/* Gate kinds of a circuit given to the plan compiler. */
enum {
    QTB_GATE_M = 0, QTB_GATE_H = 1, QTB_GATE_Z = 2, QTB_GATE_X = 3,
    QTB_GATE_Y = 4, QTB_GATE_CX = 5, QTB_GATE_CZ = 6, QTB_GATE_ZPHASE = 7,
    QTB_GATE_XPHASE = 8, QTB_GATE_YPHASE = 9, QTB_GATE_ZZ = 10, QTB_GATE_T = 11
};

/* One gate.  Parametric gates have alpha = coef * params[param]; a daggered
 * parametric gate is passed with coef negated (ZZ, XPhase, YPhase, ZPhase
 * satisfy G(alpha)^+ = G(-alpha)); the other gates are their own inverse.   */
typedef struct {
    int32_t kind;
    int32_t q0;
    int32_t q1;        /* second qubit of CX/CZ/ZZ, else -1 */
    int32_t param;     /* -1 for non-parametric gates */
    double coef;
} qtb_gate;

typedef struct qtb_plan qtb_plan;   /* opaque: a set of compiled networks */

/* Per-network statistics filled by qtb_plan_network_info. */
typedef struct {
    int32_t n_qubits;
    int32_t n_vars;           /* variables of the bucket network */
    int32_t treewidth;        /* greedy width (max neighbour count), Optimizer.py:78 */
    int32_t max_rank;         /* largest tensor rank built (incl. the summed var) */
    int32_t n_ops;            /* bucket kernels executed */
    int32_t n_phases;         /* dependency levels (barriers) */
    int32_t arena_elems;      /* complex64 scratch elements */
    int32_t angle_specific;   /* 1: simplifier decisions depend on the angles */
    double alg_bytes;         /* sum over ops of 8*(sum_t 2^rank_t + 2^w) */
    double alg_flops;         /* sum over ops of 6*(k-1)*2^u + 2*2^w*sum */
    double ref_flops;         /* PerfBackend._perfect_bucket_flop summed */
    int32_t n_slices;         /* networks of its circuit (2^sliced variables) */
    int32_t group;            /* the circuit: networks of one circuit share it */
} qtb_network_info;

/* Create an empty plan for circuits with n_params angle parameters. */
int qtb_plan_create(int32_t n_params, qtb_plan** out);
int qtb_plan_destroy(qtb_plan* plan);

/* Compile <0|circuit|0> (all qubits in and out fixed to 0) as one network:
 * simplify_passes rounds of the commutation simplifier, qtree bucket layout,
 * greedy min-degree order (ket + bra variables first), reorder, slicing and
 * symbolic bucket elimination.  params (n_params doubles) are the angles the
 * simplifier's |alpha1+alpha2| < 1e-5 cancellation test sees; decisions that
 * are not structural mark the network angle-specific.  Returns its index. */
int qtb_plan_add_circuit(qtb_plan* plan, int32_t n_qubits, const qtb_gate* gates,
                         int32_t n_gates, int32_t simplify_passes,
                         const double* params, int32_t* net_index);

/* Same, building the QAOA lightcone circuit of edge (u, v) of a graph given
 * in CSR form (node ids 0..n_nodes-1): the qubits are the nodes within p hops
 * of the edge in increasing node id; layer l = 1..p acts on the radius p+1-l
 * subgraph with ZZ(2*gamma_l) on its edges (increasing (a, b), a < b) and
 * XPhase(2*beta_l) on its nodes, then Z_u Z_v, then the inverse.
 * composer: 0 = ZZ gates + simplifier run twice (DefaultQAOAComposer),
 * 1 = ZZ gates, 2 = CX-ZPhase-CX (QtreeQAOAComposer).  params = gamma[0..p),
 * beta[0..p).                                                            */
int qtb_plan_add_lightcone(qtb_plan* plan, int32_t n_nodes, const int64_t* indptr,
                           const int32_t* indices, int32_t u, int32_t v, int32_t p,
                           int32_t composer, const double* params, int32_t* net_index);

/* Compile all edges of a graph with n_threads host threads (0 = all cores);
 * edges is 2*n_edges node ids.  Edge i of the call becomes the networks of
 * group (the plan's group count before the call) + i, in edge order.     */
int qtb_plan_add_lightcones(qtb_plan* plan, int32_t n_nodes, const int64_t* indptr,
                            const int32_t* indices, const int32_t* edges, int32_t n_edges,
                            int32_t p, int32_t composer, const double* params,
                            int32_t n_threads, int32_t* first_net_index);

/* Batch of amplitudes <b|U|0> of one circuit (QtreeSimulator.simulate_batch,
 * qtensor/Simulate.py:66-94, batch_vars free output qubits): for every
 * bitstring b of qubits 0..batch_vars-1 (qubit 0 the most significant bit,
 * the order of the reference's flattened result) and the other qubits 0,
 * the circuit's network with those bra values fixed; 2^batch_vars circuits
 * (groups) *first_group.. in order, each with its slices.  batch_vars 0 is
 * qtb_plan_add_circuit (simulate / simulate_state).                       */
int qtb_plan_add_circuit_batch(qtb_plan* plan, int32_t n_qubits, const qtb_gate* gates, int32_t n_gates,
                               int32_t simplify_passes, const double* params, int32_t batch_vars,
                               int32_t* net_index, int32_t* first_group);

/* Slicing of circuits added afterwards (qtensor/FeynmanSimulator.py:49-84,
 * SlicesOptimizer qtensor/optimisation/Optimizer.py:90-159): when the
 * greedy width reaches max_width, variables of highest degree are removed
 * from the line graph (GreedyParvars, Greedy.py:78-91) until it drops
 * below; the circuit then becomes 2^k networks, one per assignment of the
 * k sliced variables, whose amplitudes sum to the circuit's.  Networks of a
 * circuit are contiguous and share qtb_network_info.group; qtb_plan_run's
 * energy counts groups, not networks.  max_width 0 (default) never slices.
 * A circuit that would need more than max_slices networks (default 256,
 * at most 2^16) fails to compile with QTB_ERR_UNSUPPORTED before any slice
 * is built, which bounds host memory and compile time per circuit.      */
int qtb_plan_set_max_width(qtb_plan* plan, int32_t max_width, int32_t max_slices);

/* How circuits added afterwards choose their sliced variables when they
 * reach max_width (results are the same; widths and slice counts differ):
 *   QTB_SLICE_GREEDY     variables of highest degree, one at a time, until
 *                        the width drops below max_width (GreedyParvars +
 *                        SlicesOptimizer, qtensor/optimisation/Greedy.py:78-91,
 *                        Optimizer.py:109-159); the default;
 *   QTB_SLICE_TREE_TRIM  TreeTrimSplitter (Optimizer.py:178-224): rounds of
 *                        int(0.2 x excess width) + 1 variables lying in the
 *                        most largest elimination cliques;
 *   QTB_SLICE_LATE       LateParOptimizer (late_parallelisation.py:30-202):
 *                        each variable sliced at the step of the elimination
 *                        order that leaves the least width; the order is the
 *                        contracted prefixes, then the rest.
 * The order search with trials still runs on the sliced graph for the
 * greedy and tree-trimming choices.                                       */
#define QTB_SLICE_GREEDY 0
#define QTB_SLICE_TREE_TRIM 1
#define QTB_SLICE_LATE 2
int qtb_plan_set_slicing(qtb_plan* plan, int32_t method);

/* Elimination-order search for networks added afterwards: 0 (default) keeps
 * the reference's greedy rule (first node of least degree); trials > 0 also
 * runs that many seeded greedy orders with random tie-breaking and keeps
 * the one of least sum over eliminations of 2^degree (the zero-temperature
 * RGreedyOptimizer, qtensor/optimisation/RGreedy.py:15-77).               */
int qtb_plan_set_order_trials(qtb_plan* plan, int32_t trials);

/* Structural sharing for qtb_plan_add_lightcones calls made afterwards
 * (enable 1, the default): edges whose lightcones are isomorphic, by a map
 * that keeps every node's distance from the edge and sends the edge's ends
 * to the edge's ends, contract to the same <Z_u Z_v>, so the first such
 * edge (in edge order) is compiled and the others copy its networks.  Each
 * edge still has networks of its own in the plan and on the device; only
 * the host compile is shared, so a shared edge's qtb_plan_network_info and
 * qtb_plan_network_peo are those of its class's first edge (the same cone,
 * numbered as that edge's).  The canonical key is compared in full, so a
 * share is never made on a hash alone.  No counterpart in the reference,
 * which compiles every edge (qtensor/QAOASimulator.py:44-66).  0 compiles
 * every edge from its own lightcone.                                     */
int qtb_plan_set_share_lightcones(qtb_plan* plan, int32_t enable);

/* Element records (enable 1, the default; set before qtb_plan_upload): for
 * every distinct network blob whose gate table fits shared memory, the
 * host resolves each output element's operand offsets (the bit gathers of
 * its bucket's index sets, qtensor/ProcessingFrameworks.py:23-37 einsum)
 * into per-element words, so that the shared-memory executors only load and
 * multiply.  Same products in the same order as without records, so the
 * terms are identical.  Costs (1 + operands) x 4 bytes per element of
 * device memory, at most 256 MiB per plan; 0 keeps the plain plan blobs. */
int qtb_plan_set_records(qtb_plan* plan, int32_t enable);

int qtb_plan_n_networks(const qtb_plan* plan, int32_t* n);
int qtb_plan_network_info(const qtb_plan* plan, int32_t net, qtb_network_info* info);
/* Elimination order of a network as variable ids of the qtree layout
 * (bra 0..nq-1, then variables in creation order), ket+bra first. */
int qtb_plan_network_peo(const qtb_plan* plan, int32_t net, int32_t* peo, int32_t cap,
                         int32_t* n);
/* Check that params keep every angle-dependent simplifier decision of the
 * plan; *valid = 0 means the plan must be recompiled for these angles.    */
int qtb_plan_check_params(const qtb_plan* plan, const double* params, int32_t* valid);

/* Host copies of the flattened plan (the arrays qtb_plan_upload sends to the
 * device), for inspection and CPU-side verification of the compiler.
 * which: 0 networks (8 x u32 each), 1 ops (16 B each), 2 operands (8 B),
 * 3 phases (16 B), 4 gate-table entries (24 B), 5 angle terms (16 B),
 * 6 per-network executor records (12 x u32), 7 the per-network plan blobs
 * (phases, ops, operands with network-local indices) the executor stages,
 * 8 the element records (u32 words; see qtb_plan_set_records).
 * Writes min(cap, size) bytes to buf (may be NULL) and the full size.     */
int qtb_plan_export(qtb_plan* plan, int32_t which, void* buf, size_t cap, size_t* size);
/* Complex64 elements of the gate table. */
int qtb_plan_table_elems(const qtb_plan* plan, int64_t* n);

/* Copy the plan to the current device (synchronous; allocates device memory
 * owned by the plan).  Must precede qtb_plan_run.                         */
int qtb_plan_upload(qtb_plan* plan);

/* Contract networks [first, first+count) of an uploaded plan on stream:
 *   params_dev  device doubles (n_params) -- the angles of this request;
 *   terms_dev   device complex64 per network (the amplitude <0|U|0>);
 *   energy_dev  device double: (groups - sum Re terms) / 2 with a compensated
 *               (Neumaier) fp64 sum over the range's networks, groups = the
 *               circuits they belong to -- the MaxCut energy when the
 *               circuits are the edge terms of one graph; may be NULL;
 *   scratch_dev device memory of qtb_plan_scratch_bytes(); may be NULL when
 *               that size is 0.  qtb_plan_scratch_bytes also works before
 *               qtb_plan_upload (host work only), for budgeting.
 * The gate table is generated on the device from params_dev.             */
int qtb_plan_scratch_bytes(const qtb_plan* plan, int32_t first, int32_t count,
                           size_t* bytes);
int qtb_plan_run(qtb_plan* plan, int32_t first, int32_t count, const double* params_dev,
                 void* terms_dev, double* energy_dev, void* scratch_dev, void* stream);

/* The plain path over the same compiled plan: every bucket of every network
 * is one launch of the qtb_bucket_c64 kernel (the drop-in backend's
 * process_bucket, qtensor/ProcessingFrameworks.py:29-31, as called by
 * bucket_elimination in QtreeSimulator.simulate_batch, Simulate.py:90-94),
 * networks one after another, intermediates in scratch_dev (global memory,
 * qtb_plan_plain_scratch_bytes(), reused by every network), the gate table
 * in global memory, then the same fp64 compensated energy as qtb_plan_run.
 * Results equal qtb_plan_run's within complex64 rounding.                 */
int qtb_plan_plain_scratch_bytes(const qtb_plan* plan, int32_t first, int32_t count,
                                 size_t* bytes);
int qtb_plan_run_plain(qtb_plan* plan, int32_t first, int32_t count, const double* params_dev,
                       void* terms_dev, double* energy_dev, void* scratch_dev,
                       size_t scratch_bytes, void* stream);

/* Schedule and block-size autotuning: when enabled, the first qtb_plan_run
 * of a network range (outside stream capture) times every launch class of
 * the class schedule (one CTA per network, networks grouped by shared
 * memory, classes concurrent) with 64..1024 threads per CTA, then the whole
 * class schedule against the persistent, hybrid (large networks as
 * classes + a lean persistent queue) and warp-per-network schedules, and
 * keeps the fastest; with wide networks it then times the wave kernel with
 * 8 and with 4 elements per thread in flight and keeps the faster; later
 * runs reuse the choices.
 * QTB_AUTOTUNE=0 in the environment keeps the default block sizes;
 * QTB_SCHEDULE and QTB_WIDE_BATCH (2 or 3) fix the schedule and the wave
 * variant.                                                               */
int qtb_plan_set_autotune(qtb_plan* plan, int32_t enable);
/* Resident CTAs per SM of the plan's wide waves (0, the default: as many
 * as fit, two).  A wave keeps its CTAs for its whole run; with 1, half of
 * every SM stays free for other streams' kernels (a server's concurrent
 * requests) while a wide request runs.  Set before a range's first run.  */
int qtb_plan_set_wave_ctas_per_sm(qtb_plan* plan, int32_t ctas);
/* How the CTAs of a persistent launch take networks.  0 (the default): a
 * CTA's first network is the job of its own index, later ones come from
 * the launch's queue; on a GPU the run has to itself every CTA is resident
 * at once, and the first networks start without a queue round trip.  1:
 * every network comes from the queue, so that where other streams' kernels
 * hold part of the GPU (a server's concurrent requests) and some CTAs start
 * late, the CTAs that run take the widest networks first.  Results are the
 * same either way.                                                        */
int qtb_plan_set_dynamic_claims(qtb_plan* plan, int32_t enable);
/* Launch classes of the plan's most recent run: 4 ints per class (networks,
 * threads per CTA, dynamic shared memory bytes, flags: 1 = shared-memory
 * arena, 2 = persistent launch taking networks from a queue, 4 = a wave of
 * wide networks contracted by the whole GPU step by step, arenas in
 * scratch, 8 = lean persistent queue (registers capped), 16 = warp-per-
 * network queue, 32 = the 96-thread lean queue, 64 = networks of moderate
 * size, one thread-block cluster each, arenas in scratch, 128 = networks
 * with element records contract from them, qtb_plan_set_records).        */
int qtb_plan_last_launch_config(qtb_plan* plan, int32_t* out, int32_t cap, int32_t* n_classes);

/* Device memory the plan holds once uploaded (images, gate table, job
 * lists), excluding the caller's terms/energy/scratch buffers.            */
int qtb_plan_device_bytes(const qtb_plan* plan, size_t* bytes);

/* Device error word of the last run on this plan (0 = ok); synchronises.
 * Bits: 1 arena larger than the launch's capacity, 2 a staging copy did not
 * complete in time, 4 plan blob larger than the launch's capacity, 8
 * persistent launch without its queue, 16 a wide-network step waited too
 * long for its predecessor.  Every device wait is bounded: a kernel that
 * gives up sets its bit and returns; no kernel traps.                      */
int qtb_plan_device_status(qtb_plan* plan, int32_t* status);

#define QTB_STATUS_WAIT_TIMEOUT 16

/* Failure-detection self-test (no counterpart in the reference): one thread
 * waits, with the executor's bounded counter wait (a wide-network step
 * waiting for its predecessor), on a counter that nothing increments; after
 * spin_limit polls it gives up and sets QTB_STATUS_WAIT_TIMEOUT in a status
 * word returned in *status_out.  Synchronous; the device stays usable.    */
int qtb_selftest_wait_timeout(int32_t spin_limit, int32_t* status_out);

/* Device pointer of pinned host memory (cudaHostGetDevicePointer), so that
 * kernels read a caller's pinned angles and write its pinned energy
 * directly: a captured call then needs no host<->device copy nodes.  No
 * counterpart in the reference.                                          */
int qtb_host_device_pointer(void* host, void** dev);
/* Copy of `bytes` (a multiple of 8) between device-accessible buffers by a
 * kernel (device memory, or pinned host memory through its device
 * pointer), asynchronous on stream.                                      */
int qtb_copy_c(void* dst, const void* src, size_t bytes, void* stream);

/* CUDA-event timing of the network-executor launches of qtb_plan_run, on
 * the run's stream.  set_timing resets the totals; collect_timing waits for
 * the recorded events and returns the accumulated milliseconds and launch
 * count.                                                                  */
int qtb_plan_set_timing(qtb_plan* plan, int32_t enable);
int qtb_plan_collect_timing(qtb_plan* plan, double* total_ms, int64_t* launches);

/* ------------------------------------------------- allocation-free run
 * No counterpart in the reference.  For callers that must not allocate
 * device memory while they run: a host framework that owns every device
 * allocation through its own pool (a cudaMalloc behind its back escapes its
 * accounting), or a process held to a fixed device-memory budget.
 * qtb_plan_run may allocate on first use of a range (job arrays, streams,
 * events) and needs caller-allocated scratch for wide networks; this entry
 * point allocates nothing.  It contracts networks [first, first+count) of an
 * already uploaded plan (qtb_plan_upload, which allocates, is a set-up step)
 * with every network's arena, the job list and the completion counter in one
 * library-owned static device array of QTB_NOALLOC_SCRATCH_BYTES, held by
 * every GPU that loads the library until the process exits.  Every network
 * runs on one CTA with its arena in that array (plan blobs too large for
 * shared memory are read from global memory), so a network too wide for
 * shared memory, which qtb_plan_run would contract with the whole GPU, runs
 * far slower here.  Results equal qtb_plan_run's.  Requests needing more than
 * the array (64 B per network plus count x the largest arena of the range x
 * 8 B, plus 512 B) fail with QTB_ERR_UNSUPPORTED and a message; split the
 * range.  The first call on a device looks up the array's device address
 * (once per device, that device current) and should come before any stream
 * capture.  Every call shares the array and it keeps the last call's
 * contents (the counter is cleared on the stream by each call): calls that
 * overlap on the GPU race, so issue them on one stream or serialise them.
 * A call also races with a qtb_plan_run of the same plan that overlaps it
 * on the GPU: both write the plan's gate table in global memory (when it
 * does not fit shared memory) and its status word.                        */
#define QTB_NOALLOC_SCRATCH_BYTES (64u << 20)
int qtb_plan_run_noalloc(qtb_plan* plan, int32_t first, int32_t count, const double* params_dev,
                         void* terms_dev, double* energy_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* QTB_H */
