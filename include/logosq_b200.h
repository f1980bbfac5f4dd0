/*
 * logosq_b200.h -- C ABI of the B200 dense state-vector engine for LogosQ.
 *
 * The engine replaces the CPU dense path of LogosQ (`State` + `Gate::apply` +
 * `Circuit::execute`, plus `Observable::expectation` and
 * `GradientMethod::compute_gradient`) with hand-written sm_100a kernels.  Every
 * entry point is `extern "C"`, takes plain pointers and sizes, returns an `int`
 * status (LQ_OK on success) and never throws or aborts.  The text of the last
 * failure on the calling thread is returned by lq_last_error().
 *
 * Conventions shared with the reference:
 *   - Qubit q of an n-qubit state is bit (n-1-q) of the basis index (qubit 0 is
 *     the most significant bit), as in src/gates/utils.rs:4-7.
 *   - Amplitudes are complex numbers stored as interleaved (re, im) pairs,
 *     like ndarray::Array1<Complex64> (src/states/mod.rs:38-41).
 *   - Host buffers are owned by the caller; transfers are synchronous.
 *
 * Threading: a state handle is used by one host thread at a time (each handle
 * owns one CUDA stream); distinct handles may be used concurrently.
 */
#ifndef LOGOSQ_B200_H
#define LOGOSQ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------
 * Status codes.  The first six mirror LogosQError (src/error.rs:9-61).
 * ------------------------------------------------------------------------- */
enum {
    LQ_OK = 0,
    LQ_ERR_QUBIT_INDEX = 1,        /* InvalidQubitIndex        src/error.rs:11-13 */
    LQ_ERR_STATE_DIMENSION = 2,    /* InvalidStateDimension    src/error.rs:15-17 */
    LQ_ERR_DIMENSION_MISMATCH = 3, /* DimensionMismatch        src/error.rs:19-21 */
    LQ_ERR_GATE_MATRIX = 4,        /* InvalidGateMatrix        src/error.rs:23-28 */
    LQ_ERR_PARAM_COUNT = 5,        /* ParameterCountMismatch   src/error.rs:30-32 */
    LQ_ERR_QUBIT_MISMATCH = 6,     /* CircuitQubitMismatch     src/error.rs:34-40 */
    LQ_ERR_INVALID_ARG = 7,        /* null pointer, bad enum, bad size          */
    LQ_ERR_OOM = 8,                /* device allocation refused                 */
    LQ_ERR_CUDA = 9,               /* CUDA runtime or driver error              */
    LQ_ERR_TIMEOUT = 10,           /* a bounded device wait ran out             */
    LQ_ERR_UNSUPPORTED = 11        /* dtype / size not supported by this call   */
};

/* Amplitude storage type of a state. */
enum {
    LQ_C128 = 0, /* complex128 (2 x f64), the drop-in type (Complex64 in Rust) */
    LQ_C64 = 1   /* complex64 (2 x f32), the tensor-core precision form        */
};

/* ---------------------------------------------------------------------------
 * Gate descriptors.  One descriptor per reference gate struct / builder.
 * ------------------------------------------------------------------------- */
enum {
    LQ_GATE_H = 0,        /* HGate            src/gates/single_qubit.rs:90-113          */
    LQ_GATE_X = 1,        /* XGate            src/gates/single_qubit.rs:14-31           */
    LQ_GATE_Y = 2,        /* YGate            src/gates/single_qubit.rs:39-58 (applies -Y,
                             as the reference struct does)                               */
    LQ_GATE_Z = 3,        /* ZGate            src/gates/single_qubit.rs:67-82           */
    LQ_GATE_S = 4,        /* SGate            src/gates/single_qubit.rs:121-137         */
    LQ_GATE_T = 5,        /* TGate            src/gates/single_qubit.rs:145-161         */
    LQ_GATE_RX = 6,       /* RXGate           src/gates/parameterized.rs:48-80          */
    LQ_GATE_RY = 7,       /* RYGate           src/gates/parameterized.rs:101-133        */
    LQ_GATE_RZ = 8,       /* RZGate           src/gates/parameterized.rs:154-178        */
    LQ_GATE_PHASE = 9,    /* PhaseGate        src/gates/parameterized.rs:199-218        */
    LQ_GATE_U3 = 10,      /* U3Gate           src/gates/parameterized.rs:249-282        */
    LQ_GATE_CNOT = 11,    /* CNOTGate         src/gates/two_qubit.rs:12-31              */
    LQ_GATE_SWAP = 12,    /* SWAPGate         src/gates/two_qubit.rs:40-62              */
    LQ_GATE_CZ = 13,      /* CZGate           src/gates/two_qubit.rs:71-92              */
    LQ_GATE_CPHASE = 14,  /* CPhaseGate       src/gates/two_qubit.rs:100-134            */
    LQ_GATE_TOFFOLI = 15, /* ToffoliGate      src/gates/three_qubit.rs:13-35            */
    LQ_GATE_CRX = 16,     /* CRXGate          src/gates/parameterized.rs:311-343        */
    LQ_GATE_CRY = 17,     /* CRYGate          src/gates/parameterized.rs:368-399        */
    LQ_GATE_CRZ = 18,     /* CRZGate          src/gates/parameterized.rs:424-451        */
    LQ_GATE_CPHASE_PARAM = 19, /* CPhaseParamGate src/gates/parameterized.rs:476-499   */
    LQ_GATE_RXX = 20,     /* RXXGate          src/gates/parameterized.rs:528-580 (keeps the
                             reference's |01>/|10> block rule, see LQ_FLAG_TEXTBOOK)     */
    LQ_GATE_RYY = 21,     /* RYYGate          src/gates/parameterized.rs:604-655        */
    LQ_GATE_RZZ = 22,     /* RZZGate          src/gates/parameterized.rs:679-709        */
    LQ_GATE_MATRIX1 = 23, /* 2x2 matrix on q[0]: Circuit::h/x/y/z/s/t/r*_matrix
                             (src/circuits/single_qubit.rs:12-126), lowered from the
                             dense 2^n x 2^n MatrixGate to a single-qubit sweep          */
    LQ_GATE_MATRIX2 = 24, /* 4x4 matrix on (q[0], q[1]) with q[0] the high bit of the
                             4x4 index: Circuit::add_two_qubit_gate
                             (src/circuits/two_qubits.rs:11-82)                          */
    LQ_GATE__COUNT = 25
};

/* Descriptor flags. */
enum {
    LQ_FLAG_RENORM = 1,  /* normalize the state after this gate, as MatrixGate::apply
                            does (src/gates/mod.rs:76-93)                                */
    LQ_FLAG_TEXTBOOK = 2 /* RXX/RYY: apply the full 4x4 rotation instead of the
                            reference's loop (which skips the |01>,|10> block when
                            qubit1 < qubit2, src/gates/parameterized.rs:563-577)         */
};

/*
 * One gate.  q[] holds LogosQ qubit indices (unused entries -1): the qubit for
 * one-qubit gates, (control, target) or (qubit1, qubit2) for two-qubit gates,
 * (control1, control2, target) for Toffoli.  angle[] is (theta, phi, lambda)
 * for U3, (theta) for rotations and (angle) for CPhase.  If param[k] >= 0 the
 * angle k is taken from the caller's parameter vector instead:
 *     angle_k = theta[param[k]] * scale[k] + angle[k]
 * which is how an Ansatz (src/optimization/ansatz.rs:10-43) is described once
 * and re-bound to new parameter vectors.  m[] holds the matrix of MATRIX1
 * (2x2) and MATRIX2 (4x4) gates, row-major, interleaved (re, im).
 */
typedef struct lq_gate {
    int32_t kind;
    int32_t flags;
    int32_t q[3];
    int32_t param[3];
    double angle[3];
    double scale[3];
    double m[32];
} lq_gate;

/*
 * One Pauli string P = X^x Z^z (up to phase) with a real coefficient, the
 * packed form of PauliTerm (src/optimization/observable.rs:79-83).  xmask has
 * bit (n-1-q) set when qubit q carries X or Y; zmask when it carries Z or Y;
 * ny counts the Y factors.  Its expectation is
 *     coefficient * Re sum_i conj(psi_i) * phase(i) * psi_{i ^ xmask},
 *     phase(i) = (+-i)^ny * (-1)^popcount(i & zmask)
 * with +i under LQ_Y_REFERENCE (the convention of PauliTerm::expectation,
 * src/optimization/observable.rs:125-132) and -i under LQ_Y_TEXTBOOK.
 */
typedef struct lq_pauli_term {
    double coefficient;
    uint64_t xmask;
    uint64_t zmask;
    int32_t ny;
    int32_t reserved;
} lq_pauli_term;

enum { LQ_Y_REFERENCE = 0, LQ_Y_TEXTBOOK = 1 };

/* Execution modes of lq_apply_circuit. */
enum {
    LQ_EXEC_FUSED = 0,   /* plan the gate list into fused shared-memory block passes */
    LQ_EXEC_PER_GATE = 1 /* one sweep per gate, in order (the Gate::apply path)      */
};

typedef struct lq_state lq_state;

/* ---------------------------------------------------------------------------
 * Library / device
 * ------------------------------------------------------------------------- */
/* Text of the last error raised on this host thread ("" if none). */
const char *lq_last_error(void);
/* Library version as major*10000 + minor*100 + patch. */
int lq_version(void);
/* Number of visible CUDA devices. */
int lq_device_count(int *count);
/* Select the device that later lq_state_create calls on this thread use. */
int lq_set_device(int device);
/* Host-side cap on bytes that lq_state_create may allocate (0 = no cap).
 * Lets tests exercise LQ_ERR_OOM without exhausting a shared GPU. */
int lq_set_alloc_limit(uint64_t bytes);

/* Launch timing (no reference counterpart; used by the benchmark): when
 * enabled, CUDA events bracket every launch and lq_profile_read returns the
 * summed device time and launch count of one kernel class:
 * 0 fused block passes, 1 per-gate sweeps, 2 reductions (norm, Pauli-sum
 * expectation, inner product), 3 batched engine, 4 tensor-core blocks.  One
 * bracket per call: work a call runs inside another bracket (the norm pass of
 * a renormalising gate) counts toward the outer class.  Enabling (or
 * disabling) resets the counters. */
int lq_profile_enable(int on);
int lq_profile_read(int kernel_class, double *total_ms, long long *launches);

/* ---------------------------------------------------------------------------
 * State (src/states/mod.rs:38-141)
 * ------------------------------------------------------------------------- */
/* Allocate an n-qubit state of the given dtype, initialised to |0...0>
 * (State::zero_state, src/states/mod.rs:136-141). */
int lq_state_create(int num_qubits, int dtype, lq_state **out);
int lq_state_destroy(lq_state *s);
int lq_state_num_qubits(const lq_state *s, int *out);
int lq_state_dtype(const lq_state *s, int *out);
/* |basis> : zero_state (index 0) and one_state (index 2^n-1), src/states/mod.rs:136-150 */
int lq_state_set_basis(lq_state *s, uint64_t index);
/* plus_state, src/states/mod.rs:153-158 */
int lq_state_set_plus(lq_state *s);
/* Copy num_amplitudes (must equal 2^n) interleaved complex128 values from the
 * host (State::new without normalisation / vector_mut, src/states/mod.rs:55-133).
 * For a C64 state the values are rounded to complex64 on the device. */
int lq_state_upload(lq_state *s, const double *host, size_t num_amplitudes);
int lq_state_download(const lq_state *s, double *host, size_t num_amplitudes);
/* Same for complex64 host data (C64 states only). */
int lq_state_upload_c64(lq_state *s, const float *host, size_t num_amplitudes);
int lq_state_download_c64(const lq_state *s, float *host, size_t num_amplitudes);
/* dst <- src (same n and dtype), like State::clone. */
int lq_state_copy(lq_state *dst, const lq_state *src);
/* out <- |a> (x) |b> (State::tensor_product, src/states/mod.rs:298-314);
 * out must have n_a + n_b qubits. */
int lq_state_tensor_product(lq_state *out, const lq_state *a, const lq_state *b);
/* Wait for all work queued on the state's stream.  Returns LQ_ERR_TIMEOUT (and
 * clears the condition) when a kernel's bounded device wait ran out since the
 * last call; the handle and the CUDA context stay usable, but the amplitudes
 * that kernel was working on are undefined. */
int lq_state_synchronize(lq_state *s);
/* Failure-path check (no reference counterpart; the reference's error surface
 * is LogosQError, src/error.rs:9-64): queue one kernel on the state's stream
 * that waits on a shared-memory barrier which nothing ever completes, giving
 * up after `polls` bounded try-wait polls (1..1048576), exactly as every
 * pipeline wait in this library gives up after its own bound.  It then raises
 * the state's timeout flag and returns, so the next lq_state_synchronize
 * reports LQ_ERR_TIMEOUT.  Touches no amplitude and copies nothing. */
int lq_check_wait_timeout(lq_state *s, unsigned polls);
/* Device pointer and CUDA stream (cudaStream_t) of the state, for callers that
 * interoperate with other CUDA code.  The pointer stays owned by the handle. */
int lq_state_device_ptr(lq_state *s, void **dptr);
int lq_state_stream(lq_state *s, void **stream);

/* ---------------------------------------------------------------------------
 * Reductions (FP64 accumulation for both dtypes)
 * ------------------------------------------------------------------------- */
/* sum |a_i|^2 */
int lq_norm_sqr(const lq_state *s, double *out);
/* State::normalize (src/states/mod.rs:91-114): divide by the norm if > 1e-10. */
int lq_normalize(lq_state *s);
/* State::probabilities (src/states/mod.rs:277-279): |a_i|^2 into host[2^n]. */
int lq_probabilities(const lq_state *s, double *host, size_t len);
/* State::probability (src/states/mod.rs:288-293): 0.0 when out of range. */
int lq_probability(const lq_state *s, uint64_t basis, double *out);
/* <a|b> = sum conj(a_i) b_i (inner_product_parallel, src/states/mod.rs:350-365);
 * out[0] = re, out[1] = im. */
int lq_inner_product(const lq_state *a, const lq_state *b, double out[2]);
/* n_shots basis indices drawn from |a_i|^2 (measure / measure_shots_parallel,
 * src/states/mod.rs:180-258) with a seeded counter-based generator. */
int lq_measure_shots(const lq_state *s, uint64_t n_shots, uint64_t seed, uint64_t *host_out);
/* sum_t coefficient_t * <P_t> (PauliObservable::expectation,
 * src/optimization/observable.rs:228-232; PauliTerm::expectation :95-147).
 * per_term (optional, may be NULL) receives each term's contribution.  Terms
 * sharing an X mask are evaluated in one sweep; at most 2000 terms may share
 * one X mask (LQ_ERR_UNSUPPORTED above that). */
int lq_expectation_pauli(const lq_state *s, const lq_pauli_term *terms, int nterms,
                         int y_convention, double *out, double *per_term);

/* Pauli-sum expectation that allocates no memory (no reference counterpart).
 * For callers that cannot call cudaMalloc: code whose device memory is owned by
 * a host framework's own allocator or strict memory budget, and code that must
 * not insert the device-wide synchronisation an allocation or free can cause
 * in the middle of its stream work.  Same result as lq_expectation_pauli, but
 * the amplitudes are a caller-owned device pointer (2^num_qubits complex
 * values of dtype LQ_C128 or LQ_C64), the work runs on the caller's CUDA
 * stream (a cudaStream_t, NULL for the default stream) and all scratch lives
 * in one fixed 64 KiB device array inside this library (every GPU that loads
 * the library holds it until the process exits).  At most 1024 terms per call;
 * more returns LQ_ERR_UNSUPPORTED.  The call copies its term table from host
 * stack memory and waits for its stream, so it cannot be recorded into a CUDA
 * graph: on a capturing stream it returns LQ_ERR_UNSUPPORTED.  Calls share the
 * array: two calls whose work overlaps on the GPU race, so
 * serialise them (one stream, or synchronise between them).  The call returns
 * after the result is in *out. */
int lq_expectation_pauli_static(const void *d_amplitudes, int num_qubits, int dtype,
                                const lq_pauli_term *terms, int nterms, int y_convention,
                                void *stream, double *out);

/* ---------------------------------------------------------------------------
 * Gates (src/gates: single_qubit.rs, two_qubit.rs, three_qubit.rs,
 * parameterized.rs, matrix.rs) -- each call is one in-place sweep on the state's
 * stream, the drop-in for Gate::apply (src/gates/mod.rs:26-35).
 * ------------------------------------------------------------------------- */
/* One descriptor; theta may be NULL when no param[] index is used. */
int lq_apply_gate(lq_state *s, const lq_gate *g, const double *theta, int ntheta);
/* 2x2 matrix m (row-major, interleaved re/im) on one qubit. */
int lq_apply_matrix1(lq_state *s, int qubit, const double m[8]);
/* 2x2 matrix on target when control is |1> (CRX/CRY/CNOT family). */
int lq_apply_controlled1(lq_state *s, int control, int target, const double m[8]);
/* Diagonal gate on k <= 3 qubits: amplitude *= phases[pattern], pattern = the
 * bits of the k qubits, qubits[0] most significant; phases has 2^k complex. */
int lq_apply_diagonal(lq_state *s, int k, const int *qubits, const double *phases);
/* SWAPGate (src/gates/two_qubit.rs:40-62). */
int lq_apply_swap(lq_state *s, int qubit1, int qubit2);
/* 4x4 matrix on (qubit1, qubit2), qubit1 the high bit of the 4x4 index. */
int lq_apply_matrix2(lq_state *s, int qubit1, int qubit2, const double m[32]);
/* MatrixGate::apply (src/gates/mod.rs:76-93): a full 2^n x 2^n matrix m
 * (row-major, interleaved re/im, dim = 2^n, n <= 13) times the state, then
 * State::normalize, exactly as the reference's dense gate does. */
int lq_apply_dense(lq_state *s, const double *m, uint64_t dim);
/* Dense 2^k x 2^k matrix (k <= 4) on the listed qubits (qubits[0] the high bit
 * of the matrix index), applied by the fused shared-memory block kernel. */
int lq_apply_block(lq_state *s, int k, const int *qubits, const double *m);

/* ---------------------------------------------------------------------------
 * Circuit::execute (src/circuits/mod.rs:352-375)
 * ------------------------------------------------------------------------- */
/* Apply ops[0..nops) in order.  LQ_EXEC_FUSED groups them into fused passes
 * (each a TMA-staged shared-memory tile kernel); LQ_EXEC_PER_GATE runs one sweep
 * per gate.  circuit_qubits must equal the state's qubit count
 * (CircuitQubitMismatch, src/circuits/mod.rs:353-358). */
int lq_apply_circuit(lq_state *s, int circuit_qubits, const lq_gate *ops, int nops,
                     const double *theta, int ntheta, int mode);
/* Fusion width of lq_apply_circuit: tile bits T (5..12) of a fused pass,
 * i.e. 2^T amplitudes staged per CTA.  Chosen by the benchmark's autotuner;
 * default 11. */
int lq_set_fusion_width(int tile_bits);
int lq_get_fusion_width(int *tile_bits);
/* Host-only planning query (no device work): how lq_apply_circuit in fused
 * mode would split the gate list on an n-qubit state -- number of fused passes
 * (full-state HBM sweeps), register rounds inside them, and gates that run as
 * standalone per-gate sweeps. */
int lq_plan_circuit(int num_qubits, const lq_gate *ops, int nops, int *passes, int *rounds,
                    int *standalone);
/* Host-only dump of the fused program lq_apply_circuit would run (for tests and
 * inspection): int32 counts {steps, rounds, ops, coefficients, T}, then per
 * step int32 {fused, gate, h, round_begin, nrounds}, the round records, the op
 * records and the FP64 coefficients.  *used receives the size needed. */
int lq_plan_dump(int num_qubits, const lq_gate *ops, int nops, const double *theta, int ntheta,
                 void *buf, size_t cap, size_t *used);
/* Precision form: Circuit::execute on a complex64 state (LQ_C64, n >= 12) with
 * the gates fused into 5-qubit blocks, each applied as a complex 32 x 32 GEMM
 * on the tcgen05 tensor cores (TF32 inputs, 3xTF32 split products, FP32
 * accumulation).  Gates must act on at most 2 qubits.  *blocks / *passes
 * (optional) receive the number of 5-qubit blocks and of full-state passes.
 * FP64 is kept for lq_norm_sqr / lq_expectation_pauli on the result. */
int lq_apply_circuit_tc(lq_state *s, int circuit_qubits, const lq_gate *ops, int nops,
                        const double *theta, int ntheta, int *blocks, int *passes);
/* Statistics of the last lq_apply_circuit on this handle: number of kernel
 * launches and number of fused passes (0 in per-gate mode). */
int lq_last_circuit_stats(const lq_state *s, int *launches, int *passes);

/* ---------------------------------------------------------------------------
 * Variational calls (src/optimization/)
 * ------------------------------------------------------------------------- */
/* Energy of |0> evolved by the parameterised gate list: the objective closure
 * of VQE::run (src/optimization/vqe.rs:63-67).  work is any state handle with
 * the right qubit count; it is overwritten. */
int lq_ansatz_energy(lq_state *work, const lq_gate *ops, int nops, const double *theta,
                     int nparams, const lq_pauli_term *terms, int nterms, int y_convention,
                     double *energy);
/* ParameterShift::compute_gradient (src/optimization/gradient.rs:44-78):
 * grad_i = (E(theta + shift e_i) - E(theta - shift e_i)) / 2. */
int lq_parameter_shift(lq_state *work, const lq_gate *ops, int nops, const double *theta,
                       int nparams, const lq_pauli_term *terms, int nterms, int y_convention,
                       double shift, double *grad);
/* FiniteDifference::compute_gradient (src/optimization/gradient.rs:96-125). */
int lq_finite_difference(lq_state *work, const lq_gate *ops, int nops, const double *theta,
                         int nparams, const lq_pauli_term *terms, int nterms, int y_convention,
                         double epsilon, double *grad);

/* ---------------------------------------------------------------------------
 * Batched parameter-shift engine: all 2P+1 circuits of many VQE instances of
 * uneven qubit counts in one CUDA-graph-captured call of persistent launches.
 * ------------------------------------------------------------------------- */
typedef struct lq_vqe_instance {
    int32_t num_qubits;        /* 1..20 */
    int32_t nops;
    const lq_gate *ops;        /* parameterised ansatz (param[] indices into theta) */
    int32_t nparams;
    int32_t nterms;
    const lq_pauli_term *terms;
} lq_vqe_instance;

typedef struct lq_batch lq_batch;

/* Build the batch (copies every descriptor to the device, plans the work list
 * and captures the launch in a CUDA graph on first use). */
int lq_batch_create(const lq_vqe_instance *instances, int ninstances, lq_batch **out);
int lq_batch_destroy(lq_batch *b);
/* Total parameter count over all instances. */
int lq_batch_num_params(const lq_batch *b, int *out);
/* theta: concatenated parameter vectors (instance order).  energy[ninstances]
 * gets E(theta), grad[total params] the parameter-shift gradient. */
int lq_batch_gradients(lq_batch *b, const double *theta, double shift, double *energy,
                       double *grad);
/* Tuning of the batch: the largest qubit count kept entirely in shared memory,
 * and the fusion width (tile bits) the autotuner chose on the first
 * lq_batch_gradients call for larger instances (0 before that call). */
int lq_batch_tuning(const lq_batch *b, int *smem_max_qubits, int *tile_bits);
/* Force the fusion width (tile bits 10, 11 or 12) of the instances larger than
 * 2^12 amplitudes, or 0 to autotune again on the next lq_batch_gradients call.
 * No reference counterpart (tuning control of this engine). */
int lq_batch_set_tile_bits(lq_batch *b, int tile_bits);
/* Whether the batch shares circuit prefixes (each shifted circuit starts from
 * the unshifted circuit's state just before its parameter's first gate; off
 * when LQ_BATCH_PREFIX=0 at creation or when the checkpoints would not fit)
 * and the device bytes its checkpoints take.  No reference counterpart. */
int lq_batch_prefix_info(const lq_batch *b, int *shared, uint64_t *checkpoint_bytes);

/* ---------------------------------------------------------------------------
 * Noise models (NoiseModel::apply, src/noise/mod.rs) on complex128 states.
 * As in the reference, `qubit` here is the basis-index bit (1 << qubit), not
 * the gate convention n-1-qubit; `qubits` NULL means every qubit.
 * ------------------------------------------------------------------------- */
/* apply_x_error / apply_y_error / apply_z_error (src/noise/mod.rs:337-380):
 * pauli 1 = X, 2 = Y (the reference's -Y), 3 = Z.  DepolarizingNoise
 * (src/noise/mod.rs:60-83) draws its errors on the host and calls this. */
int lq_noise_pauli(lq_state *s, int qubit, int pauli);
/* AmplitudeDampingNoise::apply (src/noise/mod.rs:108-146): the sum over target
 * qubits of (K0 + K1) psi, K0 = |0><0| + sqrt(1-g)|1><1|, K1 = sqrt(g)|0><1|,
 * then normalised.  More than one target needs a scratch vector of 2^n
 * amplitudes (LQ_ERR_OOM if it cannot be allocated). */
int lq_noise_amplitude_damping(lq_state *s, double gamma, const int *qubits, int nqubits);
/* PhaseDampingNoise::apply (src/noise/mod.rs:173-210): |1> amplitudes of the
 * LAST target qubit scaled by sqrt(1-lambda) (each target rewrites the
 * vector), then normalised. */
int lq_noise_phase_damping(lq_state *s, double lambda, const int *qubits, int nqubits);

/* ---------------------------------------------------------------------------
 * Learned warm start.  No reference counterpart: the reference starts every
 * VQE from caller-supplied angles (VQE::run, src/optimization/vqe.rs:69-88);
 * these calls produce such angles.  A fully connected network in FP32 on the
 * device: in_dim -> hidden (x depth, GELU) -> out_dim (linear).  Parameters are
 * one flat vector, per layer W (out x in, row major) then b (out).
 * ------------------------------------------------------------------------- */
typedef struct lq_mlp lq_mlp;

/* Seeded uniform He initialisation (last layer scaled by 0.1), zero biases. */
int lq_mlp_create(int in_dim, int hidden, int depth, int out_dim, uint64_t seed, lq_mlp **out);
int lq_mlp_destroy(lq_mlp *net);
int lq_mlp_num_params(const lq_mlp *net, int64_t *out);
int lq_mlp_get_params(const lq_mlp *net, float *host, int64_t count);
int lq_mlp_set_params(lq_mlp *net, const float *host, int64_t count);
/* Gradient of the last lq_mlp_loss_grad / lq_mlp_backward call. */
int lq_mlp_get_grads(const lq_mlp *net, float *host, int64_t count);
/* y[batch x out_dim] = net(x[batch x in_dim]); host buffers. */
int lq_mlp_forward(lq_mlp *net, const float *x, int batch, float *y);
/* Periodic angle loss  L = sum(mask * (1 - cos(y - target))) / sum(mask)  and
 * dL/dparams (kept on the device for lq_mlp_adam_step). */
int lq_mlp_loss_grad(lq_mlp *net, const float *x, const float *target, const float *mask,
                     int batch, double *loss);
/* dL/dparams for a caller-supplied dL/dy[batch x out_dim] (host) at inputs x:
 * the chain rule through the network for any loss, e.g. the VQE energy with
 * dE/dtheta from lq_batch_gradients. */
int lq_mlp_backward(lq_mlp *net, const float *x, const float *dy, int batch);
/* One Adam step on the device with the last gradient (bias-corrected, step
 * count kept by the network). */
int lq_mlp_adam_step(lq_mlp *net, float lr, float beta1, float beta2, float eps);
/* Zero the Adam moments and step count (start of a new training stage). */
int lq_mlp_reset_adam(lq_mlp *net);

/* Exact ground energy of a real Pauli-sum Hamiltonian (every term with an even
 * number of Y factors, as in the XYZ chains the VQE workloads use) by FP64
 * Lanczos on the full 2^n space with full reorthogonalisation; stops when the
 * lowest Ritz value moves by less than tol.  No reference counterpart (the
 * reference has no exact solver); its energies are the yardstick for VQE. */
int lq_lanczos_ground_energy(int num_qubits, const lq_pauli_term *terms, int nterms,
                             int max_iter, double tol, uint64_t seed, double *e0, int *iters);

#ifdef __cplusplus
}
#endif

#endif /* LOGOSQ_B200_H */
