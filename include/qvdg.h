/*
 * qvdg.h — C ABI of the B200 state-vector engine (libqvdgpu.so).
 *
 * The engine replaces the CPU state-vector backend of the qvd crate
 * (qevedo-simulator 0.1.18). Every entry point names the reference function
 * or method it stands in for, as `file:line` inside the reference crate.
 *
 * Conventions (the same as the reference, src/state.rs:10-16 and
 * src/matrix.rs:3-5):
 *   - amplitude `i` has qubit `q` equal to bit `q` of `i` (qubit 0 is the
 *     least significant bit, as in Qiskit);
 *   - a gate matrix on qubits [q0, q1, ...] has index bit j = qubit qj; it is
 *     given as 2^k x 2^k complex128 values, row-major, (re, im) interleaved;
 *   - amplitudes cross the ABI in logical order as complex128 (re, im)
 *     interleaved, whatever the device precision.
 *
 * Every call returns a status and never aborts; `qvdg_last_error` gives the
 * message of the last failing call on the calling thread. A state handle is
 * used by one caller at a time (the reference takes `&mut self`). All calls
 * are synchronous from the host's point of view.
 */
#ifndef QVDG_H
#define QVDG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  QVDG_OK = 0,
  /* invalid input: qubit out of range or repeated, bad matrix shape, ...
   * (reference: assert!/panic!, src/state.rs:182-188, src/kernels.rs:511-514) */
  QVDG_ERR_INVALID = 1,
  /* device memory could not be allocated (reference: io::Error from mmap,
   * src/memory.rs:121-123) */
  QVDG_ERR_OUT_OF_MEMORY = 2,
  /* a CUDA runtime call failed; the message names it */
  QVDG_ERR_CUDA = 3,
  /* the request is valid but this build does not run it */
  QVDG_ERR_UNSUPPORTED = 4,
  /* a bounded device-side wait gave up (batched persistent launch) */
  QVDG_ERR_TIMEOUT = 5
} qvdg_status;

/* Widest dense gate a kernel applies (targets only; controls are handled by
 * restricting the index range). Reference: MAX_GATE_QUBITS, src/kernels.rs:476. */
#define QVDG_MAX_GATE_QUBITS 6
/* Widest diagonal gate (diagonals are one complex multiply per amplitude). */
#define QVDG_MAX_DIAGONAL_QUBITS 10

/* A unitary operation on logical qubits: `matrix` on `targets`, applied where
 * every control qubit holds its value. Reference: fusion::Op,
 * src/fusion.rs:15-23. */
typedef struct {
  uint32_t num_targets;
  uint32_t num_controls;
  const uint32_t* targets;        /* matrix index bit j = targets[j] */
  const uint32_t* controls;       /* control qubits */
  const uint8_t* control_values;  /* required value (0/1) of each control */
  const double* matrix;           /* 2^k x 2^k complex128, row-major */
} qvdg_op;

/* Planner choice for the staged path. */
enum { QVDG_PLANNER_GREEDY = 0, QVDG_PLANNER_LEARNED = 1 };

/* Arithmetic of the staged path's fused dense gates. FP32: CUDA-core fp32
 * complex multiply-adds. TENSOR (complex64 states): gates on 3 to 6 qubits as
 * real matrix products on the tensor cores, operands split into bf16 high and
 * low parts with fp32 accumulation (hi*hi + hi*lo + lo*hi, about 16
 * significant bits per product; diagonal and 1-2 qubit gates stay fp32). */
enum { QVDG_MATH_FP32 = 0, QVDG_MATH_TENSOR = 1, QVDG_MATH_GATES = 2, QVDG_MATH_TENSOR_PAIRS = 3 };

/* Simulator options. Reference: simulator::Options, src/simulator.rs:37-66
 * (defaults max_fused_qubits = 4, region_bits = Some(14)). */
typedef struct {
  /* Largest fused gate in qubits (1 disables fusion). */
  uint32_t max_fused_qubits;
  /* Staged execution: 0 runs one kernel per fused gate (the reference's
   * region_bits = None); 1 runs shared-memory staged tiles (the reference's
   * cache blocking, src/blocking.rs). */
  uint32_t staged;
  /* Local qubits per staged tile; 0 picks the default for the precision.
   * Small values force many stages on small states (as region_bits 1..4 do in
   * the reference's tests, tests/simulator.rs:256-285). */
  uint32_t tile_qubits;
  /* QVDG_PLANNER_GREEDY: plan with the settings given here.
   * QVDG_PLANNER_LEARNED: build every candidate setting
   * (qvdg_planner_candidates) and run the one the registered cost model
   * (qvdg_cost_model_set) predicts fastest; max_fused_qubits, staged,
   * tile_qubits and math are then only the fallback, used for complex128
   * states or when no model is registered for the current device. */
  uint32_t planner;
  /* QVDG_MATH_FP32: every gate on the CUDA cores. QVDG_MATH_TENSOR
   * (complex64 only): fused dense gates of 3-6 qubits in staged tiles, or of
   * 4-6 qubits in plain passes (staged = 0), run on the tensor cores as
   * split-bf16 products (hi*hi + hi*lo + lo*hi) accumulated in fp32.
   * QVDG_MATH_GATES: plain passes apply a fused group of 4-5 qubits member
   * gate by member gate in registers instead of as its product matrix.
   * QVDG_MATH_TENSOR_PAIRS (complex64, plain): as TENSOR, and two
   * consecutive fused 6-qubit gates without controls share one pass over
   * the state (the second applied to the first's output on chip). */
  uint32_t math;
} qvdg_options;

/* What a run did. Reference: simulator::Stats, src/simulator.rs:70-93, plus
 * the bytes each pass moved. */
typedef struct {
  uint64_t gates;       /* ops given */
  uint64_t kernels;     /* fused ops applied */
  uint64_t passes;      /* full passes over the state (stages + relabels, or one per fused op) */
  uint64_t stages;      /* staged passes */
  double gate_seconds;  /* device time of the gate work (CUDA events) */
  double bytes;         /* algorithmic HBM bytes of the gate work */
  qvdg_options settings; /* the settings the run's plan was built with (planner = GREEDY: the learned pick
                          * or the caller's own) */
} qvdg_stats;

typedef struct qvdg_state qvdg_state;

/* Fill `opt` with the reference defaults (max_fused_qubits 4, staged). */
void qvdg_default_options(qvdg_options* opt);

/* The message of the last failing call on this thread ("" if none). */
const char* qvdg_last_error(void);

/* Library version string. */
const char* qvdg_version(void);

/* The state |0...0> of `num_qubits` qubits in single (32) or double (64)
 * precision, on the current CUDA device.
 * Reference: StateVector::zero, src/state.rs:39-49. */
qvdg_status qvdg_state_create(uint32_t num_qubits, uint32_t precision_bits, qvdg_state** out);

/* Free the state and its device memory (reference: Drop of Buffer,
 * src/memory.rs:91-96). NULL is accepted. */
qvdg_status qvdg_state_destroy(qvdg_state* state);

/* Set the state to |0...0> and the identity layout. */
qvdg_status qvdg_state_zero(qvdg_state* state);

/* Number of qubits and precision of a state. */
qvdg_status qvdg_state_info(const qvdg_state* state, uint32_t* num_qubits, uint32_t* precision_bits);

/* Replace the amplitudes with `amplitudes` (2^n complex128, logical order).
 * Reference: StateVector::from_amplitudes, src/state.rs:52-63. */
qvdg_status qvdg_state_set_amplitudes(qvdg_state* state, const double* amplitudes, size_t count);

/* Copy the amplitudes out (2^n complex128, logical order).
 * Reference: StateVector::to_vec, src/state.rs:146-159. */
qvdg_status qvdg_state_get_amplitudes(const qvdg_state* state, double* amplitudes, size_t count);

/* Apply ops in order, fusing them first; fills `stats` if not NULL.
 * Reference: simulator::apply_ops, src/simulator.rs:122-147 (fusion
 * src/fusion.rs:63-170, blocking src/blocking.rs:230-302). */
qvdg_status qvdg_apply_ops(qvdg_state* state, const qvdg_op* ops, size_t num_ops,
                           const qvdg_options* options, qvdg_stats* stats);

/* Apply one unitary `matrix` (index bit j = qubits[j]) where every control
 * holds. Reference: StateVector::apply, src/state.rs:181-198. */
qvdg_status qvdg_apply(qvdg_state* state, const double* matrix, const uint32_t* qubits,
                       uint32_t num_qubits, const uint32_t* controls,
                       const uint8_t* control_values, uint32_t num_controls);

/* <psi|psi> accumulated in double precision.
 * Reference: StateVector::norm_sqr, src/state.rs:172-177. */
qvdg_status qvdg_norm_sqr(const qvdg_state* state, double* out);

/* Multiply every amplitude by `factor`. Reference: StateVector::scale,
 * src/state.rs:201-207. */
qvdg_status qvdg_scale(qvdg_state* state, double factor);

/* Probability that `qubit` measures 1, in double precision.
 * Reference: StateVector::probability_one, src/measure.rs:43-65. */
qvdg_status qvdg_probability_one(const qvdg_state* state, uint32_t qubit, double* out);

/* <Z_q> = 1 - 2 P(q = 1) for every qubit in one pass (out: num_qubits
 * values). Built on probability_one, src/measure.rs:43-65. */
qvdg_status qvdg_expect_z_all(const qvdg_state* state, double* out);

/* Probability of every basis state in logical order (2^n doubles).
 * Reference: StateVector::probabilities, src/measure.rs:25-40. */
qvdg_status qvdg_probabilities(const qvdg_state* state, double* out, size_t count);

/* Measure `qubit` with the caller's uniform draw in [0, 1), collapse the
 * state, and write the outcome (0/1).
 * Reference: StateVector::measure, src/measure.rs:68-80. */
qvdg_status qvdg_measure(qvdg_state* state, uint32_t qubit, double uniform, int32_t* outcome);

/* Reset `qubit` to |0>: measure with `uniform`, flip on outcome 1.
 * Reference: StateVector::reset, src/measure.rs:83-87. */
qvdg_status qvdg_reset(qvdg_state* state, uint32_t qubit, double uniform);

/* Draw `shots` basis-state indices (logical) from |amplitude|^2 with the
 * caller's uniforms (`shots` values in [0, 1)), in two passes over the state,
 * the outcome of each uniform bit-exact with the reference's arithmetic.
 * `out` has room for `shots` indices; `*count` receives how many were written
 * (fewer than `shots` only when rounding puts a target at the very total, as
 * in the reference). Reference: StateVector::sample_unordered,
 * src/measure.rs:104-174. */
qvdg_status qvdg_sample_unordered(const qvdg_state* state, size_t shots, const double* uniforms,
                                  uint64_t* out, size_t* count);

/* Sample `shots` outcomes as qvdg_sample_unordered does (same uniforms, same
 * outcomes) and count them by classical key on the device: bit c of a key
 * is the OR of the values measured into classical bit c over the
 * (measure_qubits[i], measure_clbits[i]) pairs, as the reference's keyed
 * counting builds it (classical bits 0..63; at most 64 distinct pairs). Distinct keys come back ascending
 * with their counts (at most `capacity`; `*num_keys` receives how many
 * there are). Reference: count_outcomes and counts_from_keys,
 * src/simulator.rs:187-230 (the formatting of keys as bitstrings stays with
 * the caller). */
qvdg_status qvdg_sample_counts(const qvdg_state* state, size_t shots, const double* uniforms,
                               const uint32_t* measure_qubits, const uint32_t* measure_clbits, size_t num_measures,
                               uint64_t* keys, uint64_t* counts, size_t capacity, size_t* num_keys);

/* <psi|P|psi> for the Pauli string P = product of paulis[i] ('X', 'Y', 'Z' or
 * 'I') on qubits[i], summed in double precision (not normalised by the
 * norm). Reference: the state-vector branch of the Qiskit Estimator,
 * python/python/qevedo/simulator/qiskit.py:584-590 (expectation of a
 * SparsePauliOp term by term). */
qvdg_status qvdg_expect_pauli(const qvdg_state* state, const uint32_t* qubits, const char* paulis, size_t count,
                              double* out);

/* Exchange physical bit positions pairwise in one pass and relabel the
 * logical qubits that lived there. Reference: StateVector::swap_physical,
 * src/state.rs:212-268 (any bit positions are allowed here). */
qvdg_status qvdg_swap_physical(qvdg_state* state, const uint32_t* pairs, uint32_t num_pairs);

/* layout[logical] = physical bit position (num_qubits values).
 * Reference: StateVector::layout, src/state.rs:93-96. */
qvdg_status qvdg_state_layout(const qvdg_state* state, uint32_t* layout);

/* Device address and byte size of the amplitude buffer (interleaved complex
 * in the state's precision, physical order), for callers that keep data on
 * the device. The pointer stays valid until the state is destroyed. The
 * caller may write through it: the state then no longer counts as |0...0>
 * (which lets runs skip work) until the next qvdg_state_zero. */
qvdg_status qvdg_state_device_buffer(const qvdg_state* state, void** pointer, size_t* bytes);

/* Block the host until the state's stream is idle. */
qvdg_status qvdg_synchronize(const qvdg_state* state);

/* A circuit planned once (fused and cut into stages) and uploaded to the
 * current device, for states of `num_qubits` qubits in `precision_bits`
 * precision with the identity layout. Executing a plan repeats the work of
 * qvdg_apply_ops without host planning. Reference: the planning half of
 * apply_ops (src/simulator.rs:122-147, src/fusion.rs:63, src/blocking.rs:230). */
typedef struct qvdg_plan qvdg_plan;

qvdg_status qvdg_plan_create(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                             const qvdg_options* options, qvdg_plan** out);

/* Free a plan (NULL is accepted). */
qvdg_status qvdg_plan_destroy(qvdg_plan* plan);

/* Gates, fused kernels, passes, stages and algorithmic bytes of a plan (as
 * run from |0...0>, whole passes counted). */
qvdg_status qvdg_plan_info(const qvdg_plan* plan, qvdg_stats* stats);

/* Apply a plan to a state of its size and precision, in any layout (the
 * execution half of apply_ops, src/simulator.rs:122-147). A tensor-core
 * plain plan may hold two fusions: the one cheapest from |0...0>, run on a
 * state still |0...0> since its last qvdg_state_zero (its first passes skip
 * the amplitudes of untouched qubits), and the one cheapest for any other
 * state. */
qvdg_status qvdg_plan_execute(qvdg_state* state, const qvdg_plan* plan, qvdg_stats* stats);

/* ---- Learned cost model ------------------------------------------------
 * No reference counterpart: the reference plans with fixed greedy rules
 * (src/fusion.rs, src/blocking.rs). Here a small MLP predicts each pass's
 * device time from QVDG_PASS_FEATURES features the planner computes per
 * pass, so a caller can compare candidate plans before running any. */
#define QVDG_PASS_FEATURES 32

/* Features of every pass the planner builds for `ops` on a `num_qubits`
 * state under `options` (host only: no device work), for a state other than
 * |0...0> (whole passes; a plan run from |0...0> may pick another fusion and
 * skips the amplitudes of untouched qubits). `out` receives at most
 * `capacity` rows of QVDG_PASS_FEATURES floats; `*num_passes` the number of
 * passes. */
qvdg_status qvdg_plan_features(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                               const qvdg_options* options, float* out, size_t capacity, size_t* num_passes);

/* The same for the program a plan runs from |0...0> (from_zero != 0): its
 * fusion, layout and pair passes (the layout search pairs more passes
 * there), each row describing the whole pass (host only). from_zero = 0 is
 * qvdg_plan_features. */
qvdg_status qvdg_plan_features_from(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                                    const qvdg_options* options, int32_t from_zero, float* out, size_t capacity,
                                    size_t* num_passes);

/* The ops a plain plan's passes apply, in order, on logical qubits (host
 * only): each fused group as its product matrix, a pass applied gate by gate
 * as its member gates. The fusion is the one a plan picks for a state
 * other than |0...0> (from_zero = 0) or for |0...0> (from_zero != 0).
 * Reference: fuse (src/fusion.rs:63-170), which returns the greedy fusion's
 * ops the same way. Op i has num_targets[i] targets and num_controls[i]
 * controls; their qubits (targets, then controls) follow one another in
 * `qubits`, with 0 for targets and the required value for controls in
 * `control_values`, and its 4^k complex entries (row-major, interleaved
 * re/im) in `matrices`. `*num_fused`, `*num_qubit_entries` and
 * `*num_matrix_doubles` receive the sizes; with `capacity` below the
 * number of ops, only the sizes are written. Plain plans only
 * (options->staged = 0). */
qvdg_status qvdg_plan_fused_ops(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                                const qvdg_options* options, int32_t from_zero, uint32_t* num_targets,
                                uint32_t* num_controls, uint32_t* qubits, uint8_t* control_values, double* matrices,
                                size_t capacity, size_t* num_fused, size_t* num_qubit_entries,
                                size_t* num_matrix_doubles);

/* Registers the cost model for the current device, replacing any earlier
 * one: an MLP of the qvdg_mlp form below with `inputs` = QVDG_PASS_FEATURES
 * and `hidden` units per hidden layer, given its `count` parameters, that
 * predicts log(seconds per 2^24 amplitudes) of a pass from its features.
 * QVDG_PLANNER_LEARNED then ranks candidate plans with it. */
qvdg_status qvdg_cost_model_set(const float* params, size_t count, uint32_t inputs, uint32_t hidden);
/* Forgets the current device's cost model (QVDG_PLANNER_LEARNED then falls
 * back to the given settings). */
qvdg_status qvdg_cost_model_clear(void);

/* The candidate settings of the learned planner for a precision, in the
 * order qvdg_plan_choose reports them: `*count` receives their number and
 * `out` at most `capacity` of them. */
qvdg_status qvdg_planner_candidates(uint32_t precision_bits, qvdg_options* out, size_t capacity, size_t* count);

/* The learned planner's choice for `ops` on a state of `num_qubits` (host
 * planning, then one forward of the cost model on the current device): the
 * chosen settings, and every candidate's predicted seconds (at most
 * `capacity`, in qvdg_planner_candidates order). from_zero != 0 scores runs
 * that start from |0...0> (zero-start passes at the share of the state they
 * move). Fails with QVDG_ERR_INVALID when no model is registered. */
qvdg_status qvdg_plan_choose(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                             int32_t from_zero, qvdg_options* chosen, double* predicted, size_t capacity,
                             size_t* num_candidates);

/* An MLP with two hidden ReLU layers of `hidden` units and one linear
 * output, trained and evaluated by this library's own CUDA kernels (fp32,
 * on the current device). Parameters, in order: W1 (hidden x inputs), b1,
 * W2 (hidden x hidden), b2, W3 (1 x hidden), b3. */
typedef struct qvdg_mlp qvdg_mlp;
qvdg_status qvdg_mlp_create(uint32_t inputs, uint32_t hidden, uint64_t seed, qvdg_mlp** out);
qvdg_status qvdg_mlp_destroy(qvdg_mlp* mlp);
/* Number of parameters; get/set copy all of them (host arrays). */
qvdg_status qvdg_mlp_num_params(const qvdg_mlp* mlp, size_t* count);
qvdg_status qvdg_mlp_get_params(const qvdg_mlp* mlp, float* params, size_t count);
qvdg_status qvdg_mlp_set_params(qvdg_mlp* mlp, const float* params, size_t count);
/* y[i] = f(x[i]) for `rows` rows of `inputs` floats. */
qvdg_status qvdg_mlp_forward(qvdg_mlp* mlp, const float* x, size_t rows, float* y);
/* Mean squared error of f(x) against `target` and its gradient with respect
 * to every parameter (`grads`: num_params floats, may be NULL). */
qvdg_status qvdg_mlp_gradients(qvdg_mlp* mlp, const float* x, const float* target, size_t rows, float* loss,
                               float* grads);
/* `epochs` passes of Adam (learning rate `lr`) over mini-batches of `batch`
 * rows in a fixed shuffled order (`seed`); `loss` receives the final
 * full-data mean squared error. */
qvdg_status qvdg_mlp_train(qvdg_mlp* mlp, const float* x, const float* target, size_t rows, uint32_t epochs,
                           uint32_t batch, float lr, uint64_t seed, float* loss);

/* ---- Batched layered circuits ------------------------------------------
 * Many small circuits of uneven width, each a stack of layers: one 2x2 gate
 * on every qubit, then an optional entangler ladder on (q, q+1) for
 * q = 0..n-2 in that order (the hardware-efficient ansatz: RY(theta) RZ(phi)
 * per qubit and a CNOT ladder). Each circuit starts from |0...0> in complex64
 * and yields <Z_q> = total - 2 P(q = 1) for every qubit, summed in double
 * precision. The whole batch runs as ONE persistent kernel launch, captured
 * once in a CUDA graph and replayed by every run. No reference counterpart:
 * per circuit it equals apply_ops (src/simulator.rs:122-147) followed by
 * probability_one for each qubit (src/measure.rs:43-65). */
enum { QVDG_ENTANGLE_NONE = 0, QVDG_ENTANGLE_CX_LADDER = 1, QVDG_ENTANGLE_CZ_LADDER = 2 };
#define QVDG_BATCH_MAX_QUBITS 24

typedef struct {
  uint32_t num_qubits;  /* 1..QVDG_BATCH_MAX_QUBITS */
  uint32_t num_layers;
  uint32_t entangler;   /* QVDG_ENTANGLE_* */
  uint32_t reserved;    /* 0 */
  /* num_layers * num_qubits 2x2 complex128 matrices, layer-major then qubit
   * (matrix of layer l, qubit q at 8 * (l * num_qubits + q) doubles),
   * row-major, (re, im) interleaved. */
  const double* gates;
} qvdg_layered_circuit;

/* Tile shape of the batched launch: 0, 0 lets the autotuner time candidate
 * shapes (tile qubits 12-14 x 128-512 threads) on a sample of the batch and
 * keep the fastest. */
typedef struct {
  uint32_t tile_qubits;
  uint32_t threads;
} qvdg_batch_options;

typedef struct {
  uint32_t tile_qubits;  /* shape in use */
  uint32_t threads;
  uint32_t ctas;         /* persistent CTAs of the launch */
  uint32_t candidates;   /* shapes the autotuner timed (0 if given) */
  uint64_t circuits;
  uint64_t outputs;      /* sum of num_qubits */
  double tune_seconds;   /* host time spent autotuning */
} qvdg_batch_summary;

typedef struct qvdg_batch qvdg_batch;

/* Upload a batch (gate matrices in complex64), pick its tile shape and
 * capture its launch in a CUDA graph, on the current device. */
qvdg_status qvdg_batch_create(const qvdg_layered_circuit* circuits, size_t count, const qvdg_batch_options* options,
                              qvdg_batch** out);
qvdg_status qvdg_batch_destroy(qvdg_batch* batch);
/* Replace every gate matrix (same packing as at creation: circuit after
 * circuit) without re-planning: the graph reads the same device buffer. */
qvdg_status qvdg_batch_set_gates(qvdg_batch* batch, const double* gates, size_t num_matrices);
/* Run the batch: `expect_z` receives info.outputs doubles, circuit after
 * circuit, qubit 0 first; `seconds` (optional) the device time of the launch. */
qvdg_status qvdg_batch_run(qvdg_batch* batch, double* expect_z, size_t count, double* seconds);
qvdg_status qvdg_batch_info(const qvdg_batch* batch, qvdg_batch_summary* info);
/* The autotuner's timings: tile qubits, threads and sample seconds of each
 * candidate shape (at most `capacity`; `*count` receives the number). */
qvdg_status qvdg_batch_tuning(const qvdg_batch* batch, uint32_t* tile_qubits, uint32_t* threads, double* seconds,
                              size_t capacity, size_t* count);

/* Record the device time of every pass of later gate runs on this state
 * (off by default; the reference's timing counters, src/simulator.rs:128-146). */
qvdg_status qvdg_set_pass_timing(qvdg_state* state, int32_t enabled);

/* Per-pass device seconds, algorithmic bytes and kind (1 staged tile pass,
 * 0 single-gate pass, 2 single-gate pass on the tensor cores, 3 the same
 * through a shared-memory stage for gates on index bits 1-3, 4 a zero-start
 * pass: run from |0...0>, it skips the amplitudes of qubits no earlier pass
 * touched, which are zero) of the last gate run; `*count` receives the
 * number of passes, at most `capacity` entries are written. */
qvdg_status qvdg_pass_times(const qvdg_state* state, double* seconds, double* bytes, int32_t* staged,
                            size_t capacity, size_t* count);

/* Make `device` the current CUDA device of the calling thread for this
 * library (states and plans are created on the current device). */
qvdg_status qvdg_set_device(int32_t device);
/* The calling thread's current CUDA device. */
qvdg_status qvdg_get_device(int32_t* device);

/* max_i |a_i - b_i| over all logical amplitudes of two states of the same
 * size (any precisions, any layouts), accumulated in double precision on the
 * device. */
qvdg_status qvdg_max_abs_diff(const qvdg_state* a, const qvdg_state* b, double* out);

/* Per-qubit probabilities of a state vector the caller keeps in its own
 * device memory, computed without allocating anything. No counterpart in
 * the reference.
 *
 * Some callers cannot let this library call cudaMalloc: a program that has
 * given nearly all of the GPU's memory to its state vector (a 34-qubit
 * complex64 state alone takes 128 GiB of the 180 GB), or one whose device
 * memory belongs to another allocator (a framework's caching pool), where
 * an allocation from here would fail or take memory the pool counts on.
 * This entry point uses a fixed scratch array of 147,744 bytes, defined
 * in the library and held on every device that loads it until the process
 * exits, and allocates no device or pinned host memory.
 *
 * `amplitudes`: 2^num_qubits interleaved complex numbers on the current
 * device (complex64 for precision_bits 32, complex128 for 64), bit q of
 * the index = qubit q. `stream`: a cudaStream_t (NULL = the default
 * stream); the call blocks until the results are in host memory.
 * Outputs: p1[q] = sum of |a_i|^2 over the indices with bit q set
 * (num_qubits values), *total = sum of all |a_i|^2, both in double
 * precision; P(q = 1) = p1[q] / *total.
 *
 * At most 35 qubits; larger states are refused (QVDG_ERR_UNSUPPORTED).
 * The first call on a device looks up the scratch array's address on that
 * device; make that first call before any stream capture. The address is
 * kept for the life of the process: a caller that resets a device
 * (cudaDeviceReset) must not call this entry point on it afterwards, as the
 * kept address would then be stale. All calls share
 * the one array, so calls that overlap on the GPU (from several threads or
 * streams) race: order them, e.g. on one stream. */
qvdg_status qvdg_bit_probabilities_noalloc(const void* amplitudes, uint32_t num_qubits, uint32_t precision_bits,
                                           void* stream, double* p1, double* total);

#ifdef __cplusplus
}
#endif

#endif /* QVDG_H */
