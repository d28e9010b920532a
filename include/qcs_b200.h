/*
 * qcs_b200.h -- extensions of the B200 simulator beyond the RQS-SVG API.
 *
 * None of these functions exists in the reference library; each one says
 * which reference behaviour it builds on. They follow the same conventions
 * as qcs.h: return 1 on success, 0 on failure with the message passed to the
 * exception callback. Include qcs.h first.
 */
#pragma once
#include "qcs.h"

#ifdef __cplusplus
extern "C"
{
#endif

/*
 * Execution modes for gate calls (qcs_simulator_set_fusion).
 *   QCS_FUSION_PLAIN   one kernel launch per gate call, issued when the call
 *                      is made -- the reference's execution model
 *                      (src/qcs.cu:2679-2703).
 *   QCS_FUSION_GREEDY  gate calls are queued; when a result is needed (a
 *                      measurement, a state read, an event) the queue is cut
 *                      into cache-blocked passes by the greedy planner, and
 *                      each pass applies many gates in one read and one write
 *                      of the state. Every gate is still applied with its own
 *                      FP64 formula, in an order that respects dependencies.
 *   QCS_FUSION_LEARNED like GREEDY, with the pass boundaries chosen by the
 *                      dynamic-programming planner under the learned cost
 *                      model (falls back to GREEDY when no model is loaded).
 * The default is GREEDY unless the environment variable QCS_FUSION is set to
 * 0, 1 or 2.
 */
#define QCS_FUSION_PLAIN 0
#define QCS_FUSION_GREEDY 1
#define QCS_FUSION_LEARNED 2

int qcs_simulator_set_fusion(qcs_simulator *sim, int mode);
int qcs_simulator_get_fusion(const qcs_simulator *sim, int *mode);

/*
 * Amplitude precision, set before allocate_memory: 128 (complex128, the
 * reference's type and the default) or 64 (complex64: half the memory and
 * traffic, FP32 gate arithmetic). Norms, probabilities, <Z> and the sampler
 * accumulate in FP64 either way, and state transfers and saved files are
 * complex128 (the reference's file format) in both.
 */
int qcs_simulator_set_precision(qcs_simulator *sim, int amplitude_bits);
int qcs_simulator_get_precision(const qcs_simulator *sim, int *amplitude_bits);

/*
 * Pin the measurement random-number generator. The engine is
 * std::mt19937_64 seeded with a 32-bit value, as in the reference
 * (src/qcs.cu:1845-1852), so the same seed gives the same sequence of
 * uniforms as the reference's engine. Without this call the seed comes from
 * std::random_device, exactly like the reference.
 */
int qcs_simulator_set_seed(qcs_simulator *sim, uint32_t seed);

/* Complete all queued and in-flight work of the simulator. */
int qcs_simulator_synchronize(qcs_simulator *sim);

/*
 * Copy the state vector, in logical qubit order, into a host array of
 * 2 * 2^n doubles (re, im interleaved) -- the same bytes save_statevector
 * writes to its file (src/qcs.cu:2494-2543). count is the number of
 * amplitudes the buffer holds and must be at least 2^n.
 */
int qcs_simulator_get_statevector(qcs_simulator *sim, double *amplitudes, uint64_t count);

/*
 * Load a state vector given in logical qubit order (2 * 2^n doubles). This is
 * the reachable form of the reference's unreachable loader
 * (src/qcs.cu:2121-2159). Clears the measured-qubit bookkeeping.
 */
int qcs_simulator_set_statevector(qcs_simulator *sim, const double *amplitudes, uint64_t count);

/*
 * <Z_q> for every logical qubit q = 0 .. n-1, normalised by the state's norm
 * (states are not renormalised after measurement, src/qcs.cu:2654-2674).
 * expectations must hold n doubles; norm (may be NULL) receives sum |a|^2.
 * One read pass over the state, FP64 accumulation.
 */
int qcs_simulator_expectation_z(qcs_simulator *sim, double *expectations, double *norm);

/*
 * Draw num_shots bitstrings of all n qubits from the current state without
 * changing it. Shot s measures logical qubits 0, 1, ..., n-1 in that order
 * with the chain rule of measure_qubit (src/qcs.cu:2545-2677): for qubit j,
 * r = u * (P0 + P1) with u from the simulator's engine and outcome = P0 < r.
 * The uniforms are drawn from the same engine in the same order as
 * num_shots repetitions of "run circuit, measure qubits 0..n-1" would draw
 * them, so the outcomes equal the reference's bin/qcs sample loop
 * (src/qcs_main.cpp:153-193) for a circuit that ends with that measurement.
 * bitstrings[s] has bit q set when logical qubit q was measured as 1.
 * Requires n <= 64.
 */
int qcs_simulator_sample(qcs_simulator *sim, uint32_t num_shots, uint64_t *bitstrings);

/*
 * Read single amplitudes: amplitudes[2k], amplitudes[2k+1] receive the real
 * and imaginary part of the amplitude at LOGICAL index indices[k] (the index
 * save_statevector would write it at, src/qcs.cu:2494-2543), as complex128.
 * Indices must be below 2^n. For spot checks of registers too large to copy.
 */
int qcs_simulator_get_amplitudes(qcs_simulator *sim, const uint64_t *indices, uint64_t count, double *amplitudes);

/*
 * The register on the device, in logical order, for zero-copy use by other
 * GPU code: queued gates run first; if uncontrolled SWAPs (which only
 * relabel qubits in the fused modes) or a mapping left physical qubits out
 * of logical order, the amplitudes are moved in place so that physical qubit
 * q holds logical qubit q (physical SWAPs through fused passes, at most
 * n - 1 of them packed a few per pass); then the stream is synchronised.
 * *state receives the device pointer: 2^n amplitudes, (re, im) interleaved,
 * double (amplitude_bits 128) or float (64). Valid until the next call that
 * changes the simulator; writes through it are seen by later calls.
 */
int qcs_simulator_get_device_state(qcs_simulator *sim, void **state, int *amplitude_bits);

/*
 * Compare two registers of the same size on the same device, either
 * precision: <a|b> = sum over logical indices i of conj(a_i) b_i, max_i
 * |a_i - b_i|, and the squared norms <a|a>, <b|b> (FP64 accumulation, one
 * read of each register). Any output pointer may be NULL. The fidelity of the
 * two states is |<a|b>|^2 / (<a|a> <b|b>).
 */
int qcs_simulator_compare(qcs_simulator *a, qcs_simulator *b, double *overlap_re, double *overlap_im,
                          double *max_abs_diff, double *norm_a, double *norm_b);

/*
 * Counters since creation (or the last reset_stats): kernels launched by the
 * library, gates received, passes executed by the fused path, and the
 * algorithmic bytes of the gates (2 * bytes_per_amplitude * amplitudes each
 * gate can change).
 */
typedef struct qcs_b200_stats
{
    uint64_t kernel_launches;
    uint64_t gates_received;
    uint64_t gates_applied;
    uint64_t fused_passes;
    uint64_t plain_gate_kernels;
    double algorithmic_bytes;
    uint64_t tensor_passes;       /* fused passes run as tensor passes (a subset of fused_passes) */
    uint64_t tensor8_passes;      /* tensor passes of 8 x 8 stages (a subset of tensor_passes) */
    uint64_t tcgen05_passes;      /* tensor passes issued as tcgen05.mma (a subset of tensor_passes) */
    uint64_t replayed_flushes;    /* flushes launched from a kept plan: a queue seen before (the same gates,
                                     matrices bit for bit, e.g. a circuit re-run per sample), not planned again */
} qcs_b200_stats;

int qcs_simulator_get_stats(const qcs_simulator *sim, qcs_b200_stats *stats);
int qcs_simulator_reset_stats(qcs_simulator *sim);

/*
 * Kernel timing recorder. When enabled, every gate kernel the library
 * launches is bracketed by CUDA events on the simulator's stream; the sums
 * below are per kernel class since the last read. Reading synchronizes the
 * stream and clears the records. bytes = algorithmic bytes of the launches
 * (a fused pass reads and writes the whole state once).
 */
typedef struct qcs_b200_kernel_times
{
    uint64_t fused_launches;
    double fused_ms;
    double fused_bytes;
    uint64_t plain_launches;
    double plain_ms;
    double plain_bytes;
} qcs_b200_kernel_times;

int qcs_simulator_set_kernel_timing(qcs_simulator *sim, int enable);
int qcs_simulator_get_kernel_times(qcs_simulator *sim, qcs_b200_kernel_times *times);

/*
 * Planner knobs for the fused modes: the most gates one pass may carry
 * (default 256) and the number of local qubits of a pass (default 11, range
 * 9..11). 0 keeps a default. Used to tune, and to record diverse pass
 * timings for the cost model.
 */
int qcs_simulator_set_planner_options(qcs_simulator *sim, int max_gates_per_pass, int local_qubits);

/*
 * Tensor passes: a fused pass whose stages depend on few bits outside
 * themselves can run every stage as a dense complex matrix on the tensor
 * cores instead of gate by gate: 16 x 16 matrices (four qubits per stage) or
 * 8 x 8 matrices (three qubits per stage, half the tensor work per stage),
 * FP64 (DMMA) for complex128 registers, TF32 with a three-term split for
 * complex64. mode 0: never; 1 (the default): whichever of the register path
 * and the two matrix sizes the cost estimate favours; 2: 16 x 16 stages
 * wherever a pass allows them; 3: 8 x 8 stages wherever a pass allows them.
 * Results agree with the other paths to the rounding of the matrix products
 * (they replace the reference's per-pair 2x2 products, src/qcs.cu:1139-1174,
 * by products of whole stages).
 */
#define QCS_TENSOR_NEVER 0
#define QCS_TENSOR_AUTO 1
#define QCS_TENSOR_ALWAYS 2
#define QCS_TENSOR_ALWAYS_8X8 3
int qcs_simulator_set_tensor_passes(qcs_simulator *sim, int mode);
int qcs_simulator_get_tensor_passes(const qcs_simulator *sim, int *mode);

/*
 * Tensor engine of complex64 16 x 16 stages: 1 (the default) issues them as
 * tcgen05.mma with TF32 operands and FP32 accumulators in tensor memory
 * where a pass allows it (at most one local condition bit per stage); 0
 * keeps every tensor pass on warp-level mma.sync. complex128 stages always
 * run on the FP64 tensor cores through mma.sync (tcgen05 has no FP64 kind).
 * A tcgen05 pass waits on its tensor cores with a time limit; past it the
 * next call that reads results fails with a message (the register is then
 * invalid).
 */
#define QCS_TENSOR_ENGINE_MMA_SYNC 0
#define QCS_TENSOR_ENGINE_TCGEN05 1
int qcs_simulator_set_tensor_engine(qcs_simulator *sim, int engine);
int qcs_simulator_get_tensor_engine(const qcs_simulator *sim, int *engine);

/*
 * Pass timings recorded while kernel timing is enabled: for each fused pass
 * its QCS_PASS_FEATURES features and its device time in milliseconds. The
 * features: block width (1 when the pass applies its gates one by one on
 * the register path, 3 or 4 when it runs its stages as dense 8 x 8 or
 * 16 x 16 matrices on the tensor cores); blocks (the pass's stages);
 * arithmetic gates (complex multiply-adds on every amplitude); light ops
 * (diagonal phases and permutations such as X, CX, SWAP); the target-qubit
 * stride, log2 of the largest stride among the pass's local qubits (its
 * highest local qubit); log2 of the number of chunks, n - k, capped at 16.
 * Reading synchronizes, returns up to capacity records in *count and
 * clears them.
 */
#define QCS_PASS_FEATURES 6
int qcs_simulator_get_pass_records(qcs_simulator *sim, float *features, float *milliseconds, uint32_t capacity,
                                   uint32_t *count);

/*
 * Learned cost model of fused passes: an MLP 6 -> 64 -> 64 -> 1 (FP32, ReLU)
 * whose training and inference run as this library's own CUDA kernels.
 * Inputs are the pass features above; the target is log(device time per
 * amplitude in nanoseconds) = log(ms * 1e6 / 2^n). A model is trained on
 * timings of one amplitude type (complex128 or complex64). Attach a trained model to
 * a simulator and select QCS_FUSION_LEARNED to let it plan passes; measured
 * device time then decides, per gate queue, between its plan and the greedy
 * one.
 */
typedef struct qcs_b200_cost_model qcs_b200_cost_model;
#define QCS_COST_MODEL_PARAMS 4673
#define QCS_COST_MODEL_SCALING 14

int qcs_b200_cost_model_create(qcs_b200_cost_model **model, uint32_t seed);
int qcs_b200_cost_model_destroy(qcs_b200_cost_model *model);
/* Adam on mini-batches; final_loss (may be NULL) gets the mean squared error
   on the standardised training set. */
int qcs_b200_cost_model_train(qcs_b200_cost_model *model, const float *features, const float *targets,
                              uint32_t count, uint32_t epochs, uint32_t batch, float learning_rate, float *final_loss);
int qcs_b200_cost_model_predict(qcs_b200_cost_model *model, const float *features, uint32_t count, float *predictions);
/* Gradient of the mean squared error w.r.t. the parameters (layout W1[64x6],
   b1[64], W2[64x64], b2[64], W3[64], b3) for inputs and targets that are
   already standardised; loss (may be NULL) gets the loss. */
int qcs_b200_cost_model_gradients(qcs_b200_cost_model *model, const float *inputs, const float *targets,
                                  uint32_t count, float *gradients, float *loss);
/* params: QCS_COST_MODEL_PARAMS floats; scaling: input means[6], input
   deviations[6], target mean, target deviation. */
int qcs_b200_cost_model_get_params(qcs_b200_cost_model *model, float *params, float *scaling);
int qcs_b200_cost_model_set_params(qcs_b200_cost_model *model, const float *params, const float *scaling);
/* The simulator keeps a pointer (the caller keeps the model alive). */
int qcs_simulator_set_cost_model(qcs_simulator *sim, qcs_b200_cost_model *model);
/* For the last flush in learned mode: which planner ran (1 learned, 0
   greedy) and the device times the judge holds for that gate queue (ms, -1
   when not measured yet). */
int qcs_simulator_get_planner_judge(qcs_simulator *sim, int *learned_plan, double *greedy_ms, double *learned_ms);

/*
 * Batches: many independent circuits, each on its own register, run together
 * from |0..0>. Circuits with the same gates on the same qubits (parameters
 * may differ) share one plan of fused passes, and each pass runs over all of
 * them in one launch; the whole run (gate entries in, passes, <Z> of every
 * register, results out) is one CUDA graph, replayed on later runs. The first
 * run tunes the number of local qubits of each shared plan by timing the
 * candidates. The reference has no batch API: a batch replaces a host loop
 * of create / allocate_memory / gate calls / destroy per circuit.
 *
 * A gate is given by its qcs API name and parameters; its qubits are the
 * targets, then the negative controls, then the positive controls. Gates on
 * at most two targets (any number of controls) are supported; measurements
 * are not. Registers hold 9 to 30 qubits.
 */
typedef struct qcs_b200_batch qcs_b200_batch;

typedef struct qcs_b200_gate
{
    char name[16];          /* "u3", "ry", "rz", "x", "swap", "p", ... (NUL-terminated) */
    double params[4];       /* the gate's parameters in the API's order; the rest ignored */
    int16_t num_targets;
    int16_t num_negctrls;
    int16_t num_ctrls;
    int16_t reserved;       /* 0 */
    int16_t qubits[12];
} qcs_b200_gate;

typedef struct qcs_b200_batch_info
{
    uint32_t circuits;
    uint32_t groups;            /* distinct gate structures, one shared plan each */
    uint32_t passes;            /* fused passes over all groups */
    uint32_t launches_per_run;  /* kernels one run launches */
    uint64_t amplitudes;        /* over all registers */
    uint64_t parameters;        /* gate parameters over all circuits */
    double pass_bytes;          /* bytes the passes move per run: 2 x bytes/amplitude x 2^n per pass and register
                                   (the first pass of a register writes only) */
    double last_run_ms;         /* device time of the last run */
    uint32_t tensor_passes;     /* passes run as 8 x 8 tensor passes (a subset of passes) */
    uint32_t reserved;
} qcs_b200_batch_info;

/* amplitude_bits: 128 (complex128) or 64 (complex64). */
int qcs_b200_batch_create(qcs_b200_batch **batch, int amplitude_bits);
int qcs_b200_batch_destroy(qcs_b200_batch *batch);
/* Append a circuit on num_qubits; *index (may be NULL) receives its position. */
int qcs_b200_batch_add_circuit(qcs_b200_batch *batch, int num_qubits, const qcs_b200_gate *gates,
                               uint32_t num_gates, uint32_t *index);
/* Replace every gate parameter, circuit by circuit and gate by gate in the
   order given, keeping the gates: count must equal info.parameters. */
int qcs_b200_batch_set_parameters(qcs_b200_batch *batch, const double *params, uint64_t count);
/* Run every circuit from |0..0> and compute <Z_q> of every register. */
int qcs_b200_batch_run(qcs_b200_batch *batch);
/* <Z_q> of the last run, circuit by circuit (num_qubits values each). */
int qcs_b200_batch_expectation_z(qcs_b200_batch *batch, double *expectations, uint64_t count);
/* The register of one circuit after the last run (2 * 2^n doubles). */
int qcs_b200_batch_get_statevector(qcs_b200_batch *batch, uint32_t index, double *amplitudes, uint64_t count);
int qcs_b200_batch_get_info(qcs_b200_batch *batch, qcs_b200_batch_info *info);
/* Tensor passes of a batch: every group of at least 11 qubits can run its
   passes as 8 x 8 tensor passes, each register's stage matrices built on the
   GPU from its own gate entries (FP64 tensor cores for complex128, split
   TF32 for complex64). mode 0: register passes only; 1 (the default): the
   autotuner times the tensor passes beside the register passes of each
   group and keeps the faster; 2: tensor passes wherever a pass allows them.
   Takes effect at the next run (which plans the batch again). */
int qcs_b200_batch_set_tensor_passes(qcs_b200_batch *batch, int mode);

/*
 * How the fused planner (greedy mode, 11 local qubits, 256 gates per pass)
 * would run a gate list on a register of num_qubits, computed on the host
 * without a GPU: for inspecting plans and testing the planner. This entry
 * point has no counterpart in the reference library. Gates are given as in
 * a batch (any number of targets the API allows); uncontrolled SWAPs only
 * relabel qubits, as in the simulator's fused modes. kinds[] counts the ops
 * of the passes by kind:
 *    0 dense 2x2 (one gate)            1 X/CX exchange
 *    2 dense 4x4 (two targets)         3 controlled SWAP exchange
 *    4 phase                           5 diagonal on one or two targets
 *    6 term of a phase run             7 real 2x2
 *    9 phase by +-i                   10 four one-qubit gates (complex)
 *   11 four one-qubit gates (real)    12 phase run (table-fed factors)
 *   13 run of -1 phases               14 one -1 phase of such a run
 *   15 two one-qubit gates (complex)
 */
#define QCS_B200_PLAN_KINDS 24
typedef struct qcs_b200_plan_summary
{
    uint32_t passes;            /* fused passes */
    uint32_t plain_gates;       /* gates left to the one-kernel-per-gate path */
    uint32_t stages;            /* register stages over all passes */
    uint32_t ops;               /* pass ops over all passes (terms included) */
    uint32_t kinds[QCS_B200_PLAN_KINDS];
    uint64_t table_entries;     /* complex entries of the phase-run factor tables */
    uint32_t tensor_passes;     /* passes a complex128 register runs as tensor passes (automatic choice) */
    uint32_t tensor_eligible;   /* passes whose stages allow a tensor pass of 16 x 16 stages */
    uint32_t tensor_matrices;   /* stage matrices over the tensor passes */
    uint32_t tensor8_passes;    /* tensor passes of 8 x 8 stages (a subset of tensor_passes) */
} qcs_b200_plan_summary;
int qcs_b200_plan_summary_get(int num_qubits, const qcs_b200_gate *gates, uint64_t num_gates,
                              qcs_b200_plan_summary *summary);

/*
 * Allocation-free squared-norm sums of a complex128 state vector held in the
 * caller's device memory. This entry point has no counterpart in the
 * reference library.
 *
 * It is for callers that cannot let a library call cudaMalloc: code inside a
 * framework whose caching allocator owns the device memory, real-time loops
 * that cannot take an allocation's latency or failure, and paths that must
 * not synchronise the device. The caller passes the input and the output;
 * the reduction's scratch is a fixed array inside libqcs.so (168 KiB, held by
 * every GPU that loads the library until the process exits).
 *
 *   state_device  2^num_qubits complex128 amplitudes (re, im doubles),
 *                 16-byte aligned, in device memory
 *   num_qubits    1 .. 40; larger registers are rejected (the scratch is
 *                 sized for 40 qubits)
 *   sums_device   num_qubits + 1 doubles in device memory:
 *                 sums[0] = sum |a_i|^2, sums[1 + q] = sum over i with bit q
 *                 set of |a_i|^2, so <Z_q> = (sums[0] - 2 sums[1+q]) / sums[0]
 *   stream        cudaStream_t to run on (NULL: the default stream); the call
 *                 returns once the work is queued
 *
 * The first call on each device looks up the scratch array's device address
 * with that device current; make that first call before any stream capture.
 * All calls share the scratch array, so calls that overlap on the GPU race:
 * serialise them. Returns 1 on success, 0 with a message to the exception
 * callback on failure.
 */
int qcs_b200_zsums_noalloc(const double *state_device, int num_qubits, double *sums_device, void *stream);

#ifdef __cplusplus
}
#endif
