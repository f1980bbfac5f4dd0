// @generated by logosq-cuda/gen_ffi.py from include/logosq_b200.h -- do not edit.
//! Raw bindings of the B200 engine's C ABI (`include/logosq_b200.h`).
#![allow(non_camel_case_types, dead_code, clippy::missing_safety_doc)]

use std::os::raw::{c_char, c_int, c_longlong, c_uint, c_void};

pub const LQ_OK: c_int = 0;
pub const LQ_ERR_QUBIT_INDEX: c_int = 1;
pub const LQ_ERR_STATE_DIMENSION: c_int = 2;
pub const LQ_ERR_DIMENSION_MISMATCH: c_int = 3;
pub const LQ_ERR_GATE_MATRIX: c_int = 4;
pub const LQ_ERR_PARAM_COUNT: c_int = 5;
pub const LQ_ERR_QUBIT_MISMATCH: c_int = 6;
pub const LQ_ERR_INVALID_ARG: c_int = 7;
pub const LQ_ERR_OOM: c_int = 8;
pub const LQ_ERR_CUDA: c_int = 9;
pub const LQ_ERR_TIMEOUT: c_int = 10;
pub const LQ_ERR_UNSUPPORTED: c_int = 11;
pub const LQ_C128: c_int = 0;
pub const LQ_C64: c_int = 1;
pub const LQ_GATE_H: c_int = 0;
pub const LQ_GATE_X: c_int = 1;
pub const LQ_GATE_Y: c_int = 2;
pub const LQ_GATE_Z: c_int = 3;
pub const LQ_GATE_S: c_int = 4;
pub const LQ_GATE_T: c_int = 5;
pub const LQ_GATE_RX: c_int = 6;
pub const LQ_GATE_RY: c_int = 7;
pub const LQ_GATE_RZ: c_int = 8;
pub const LQ_GATE_PHASE: c_int = 9;
pub const LQ_GATE_U3: c_int = 10;
pub const LQ_GATE_CNOT: c_int = 11;
pub const LQ_GATE_SWAP: c_int = 12;
pub const LQ_GATE_CZ: c_int = 13;
pub const LQ_GATE_CPHASE: c_int = 14;
pub const LQ_GATE_TOFFOLI: c_int = 15;
pub const LQ_GATE_CRX: c_int = 16;
pub const LQ_GATE_CRY: c_int = 17;
pub const LQ_GATE_CRZ: c_int = 18;
pub const LQ_GATE_CPHASE_PARAM: c_int = 19;
pub const LQ_GATE_RXX: c_int = 20;
pub const LQ_GATE_RYY: c_int = 21;
pub const LQ_GATE_RZZ: c_int = 22;
pub const LQ_GATE_MATRIX1: c_int = 23;
pub const LQ_GATE_MATRIX2: c_int = 24;
pub const LQ_GATE__COUNT: c_int = 25;
pub const LQ_FLAG_RENORM: c_int = 1;
pub const LQ_FLAG_TEXTBOOK: c_int = 2;
pub const LQ_Y_REFERENCE: c_int = 0;
pub const LQ_Y_TEXTBOOK: c_int = 1;
pub const LQ_EXEC_FUSED: c_int = 0;
pub const LQ_EXEC_PER_GATE: c_int = 1;

#[repr(C)]
pub struct LqState {
    _opaque: [u8; 0],
}

#[repr(C)]
pub struct LqBatch {
    _opaque: [u8; 0],
}

#[repr(C)]
pub struct LqMlp {
    _opaque: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct LqGate {
    pub kind: i32,
    pub flags: i32,
    pub q: [i32; 3],
    pub param: [i32; 3],
    pub angle: [f64; 3],
    pub scale: [f64; 3],
    pub m: [f64; 32],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct LqPauliTerm {
    pub coefficient: f64,
    pub xmask: u64,
    pub zmask: u64,
    pub ny: i32,
    pub reserved: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct LqVqeInstance {
    pub num_qubits: i32,
    pub nops: i32,
    pub ops: *const LqGate,
    pub nparams: i32,
    pub nterms: i32,
    pub terms: *const LqPauliTerm,
}

extern "C" {
    pub fn lq_version() -> c_int;
    pub fn lq_device_count(count: *mut c_int) -> c_int;
    pub fn lq_set_device(device: c_int) -> c_int;
    pub fn lq_set_alloc_limit(bytes: u64) -> c_int;
    pub fn lq_profile_enable(on: c_int) -> c_int;
    pub fn lq_profile_read(kernel_class: c_int, total_ms: *mut f64, launches: *mut c_longlong) -> c_int;
    pub fn lq_state_create(num_qubits: c_int, dtype: c_int, out: *mut *mut LqState) -> c_int;
    pub fn lq_state_destroy(s: *mut LqState) -> c_int;
    pub fn lq_state_num_qubits(s: *const LqState, out: *mut c_int) -> c_int;
    pub fn lq_state_dtype(s: *const LqState, out: *mut c_int) -> c_int;
    pub fn lq_state_set_basis(s: *mut LqState, index: u64) -> c_int;
    pub fn lq_state_set_plus(s: *mut LqState) -> c_int;
    pub fn lq_state_upload(s: *mut LqState, host: *const f64, num_amplitudes: usize) -> c_int;
    pub fn lq_state_download(s: *const LqState, host: *mut f64, num_amplitudes: usize) -> c_int;
    pub fn lq_state_upload_c64(s: *mut LqState, host: *const f32, num_amplitudes: usize) -> c_int;
    pub fn lq_state_download_c64(s: *const LqState, host: *mut f32, num_amplitudes: usize) -> c_int;
    pub fn lq_state_copy(dst: *mut LqState, src: *const LqState) -> c_int;
    pub fn lq_state_tensor_product(out: *mut LqState, a: *const LqState, b: *const LqState) -> c_int;
    pub fn lq_state_synchronize(s: *mut LqState) -> c_int;
    pub fn lq_check_wait_timeout(s: *mut LqState, polls: c_uint) -> c_int;
    pub fn lq_state_device_ptr(s: *mut LqState, dptr: *mut *mut c_void) -> c_int;
    pub fn lq_state_stream(s: *mut LqState, stream: *mut *mut c_void) -> c_int;
    pub fn lq_norm_sqr(s: *const LqState, out: *mut f64) -> c_int;
    pub fn lq_normalize(s: *mut LqState) -> c_int;
    pub fn lq_probabilities(s: *const LqState, host: *mut f64, len: usize) -> c_int;
    pub fn lq_probability(s: *const LqState, basis: u64, out: *mut f64) -> c_int;
    pub fn lq_inner_product(a: *const LqState, b: *const LqState, out: *mut f64) -> c_int;
    pub fn lq_measure_shots(s: *const LqState, n_shots: u64, seed: u64, host_out: *mut u64) -> c_int;
    pub fn lq_expectation_pauli(s: *const LqState, terms: *const LqPauliTerm, nterms: c_int, y_convention: c_int, out: *mut f64, per_term: *mut f64) -> c_int;
    pub fn lq_expectation_pauli_static(d_amplitudes: *const c_void, num_qubits: c_int, dtype: c_int, terms: *const LqPauliTerm, nterms: c_int, y_convention: c_int, stream: *mut c_void, out: *mut f64) -> c_int;
    pub fn lq_apply_gate(s: *mut LqState, g: *const LqGate, theta: *const f64, ntheta: c_int) -> c_int;
    pub fn lq_apply_matrix1(s: *mut LqState, qubit: c_int, m: *const f64) -> c_int;
    pub fn lq_apply_controlled1(s: *mut LqState, control: c_int, target: c_int, m: *const f64) -> c_int;
    pub fn lq_apply_diagonal(s: *mut LqState, k: c_int, qubits: *const c_int, phases: *const f64) -> c_int;
    pub fn lq_apply_swap(s: *mut LqState, qubit1: c_int, qubit2: c_int) -> c_int;
    pub fn lq_apply_matrix2(s: *mut LqState, qubit1: c_int, qubit2: c_int, m: *const f64) -> c_int;
    pub fn lq_apply_dense(s: *mut LqState, m: *const f64, dim: u64) -> c_int;
    pub fn lq_apply_block(s: *mut LqState, k: c_int, qubits: *const c_int, m: *const f64) -> c_int;
    pub fn lq_apply_circuit(s: *mut LqState, circuit_qubits: c_int, ops: *const LqGate, nops: c_int, theta: *const f64, ntheta: c_int, mode: c_int) -> c_int;
    pub fn lq_set_fusion_width(tile_bits: c_int) -> c_int;
    pub fn lq_get_fusion_width(tile_bits: *mut c_int) -> c_int;
    pub fn lq_plan_circuit(num_qubits: c_int, ops: *const LqGate, nops: c_int, passes: *mut c_int, rounds: *mut c_int, standalone: *mut c_int) -> c_int;
    pub fn lq_plan_dump(num_qubits: c_int, ops: *const LqGate, nops: c_int, theta: *const f64, ntheta: c_int, buf: *mut c_void, cap: usize, used: *mut usize) -> c_int;
    pub fn lq_apply_circuit_tc(s: *mut LqState, circuit_qubits: c_int, ops: *const LqGate, nops: c_int, theta: *const f64, ntheta: c_int, blocks: *mut c_int, passes: *mut c_int) -> c_int;
    pub fn lq_last_circuit_stats(s: *const LqState, launches: *mut c_int, passes: *mut c_int) -> c_int;
    pub fn lq_ansatz_energy(work: *mut LqState, ops: *const LqGate, nops: c_int, theta: *const f64, nparams: c_int, terms: *const LqPauliTerm, nterms: c_int, y_convention: c_int, energy: *mut f64) -> c_int;
    pub fn lq_parameter_shift(work: *mut LqState, ops: *const LqGate, nops: c_int, theta: *const f64, nparams: c_int, terms: *const LqPauliTerm, nterms: c_int, y_convention: c_int, shift: f64, grad: *mut f64) -> c_int;
    pub fn lq_finite_difference(work: *mut LqState, ops: *const LqGate, nops: c_int, theta: *const f64, nparams: c_int, terms: *const LqPauliTerm, nterms: c_int, y_convention: c_int, epsilon: f64, grad: *mut f64) -> c_int;
    pub fn lq_batch_create(instances: *const LqVqeInstance, ninstances: c_int, out: *mut *mut LqBatch) -> c_int;
    pub fn lq_batch_destroy(b: *mut LqBatch) -> c_int;
    pub fn lq_batch_num_params(b: *const LqBatch, out: *mut c_int) -> c_int;
    pub fn lq_batch_gradients(b: *mut LqBatch, theta: *const f64, shift: f64, energy: *mut f64, grad: *mut f64) -> c_int;
    pub fn lq_batch_tuning(b: *const LqBatch, smem_max_qubits: *mut c_int, tile_bits: *mut c_int) -> c_int;
    pub fn lq_batch_set_tile_bits(b: *mut LqBatch, tile_bits: c_int) -> c_int;
    pub fn lq_batch_prefix_info(b: *const LqBatch, shared: *mut c_int, checkpoint_bytes: *mut u64) -> c_int;
    pub fn lq_noise_pauli(s: *mut LqState, qubit: c_int, pauli: c_int) -> c_int;
    pub fn lq_noise_amplitude_damping(s: *mut LqState, gamma: f64, qubits: *const c_int, nqubits: c_int) -> c_int;
    pub fn lq_noise_phase_damping(s: *mut LqState, lambda: f64, qubits: *const c_int, nqubits: c_int) -> c_int;
    pub fn lq_mlp_create(in_dim: c_int, hidden: c_int, depth: c_int, out_dim: c_int, seed: u64, out: *mut *mut LqMlp) -> c_int;
    pub fn lq_mlp_destroy(net: *mut LqMlp) -> c_int;
    pub fn lq_mlp_num_params(net: *const LqMlp, out: *mut i64) -> c_int;
    pub fn lq_mlp_get_params(net: *const LqMlp, host: *mut f32, count: i64) -> c_int;
    pub fn lq_mlp_set_params(net: *mut LqMlp, host: *const f32, count: i64) -> c_int;
    pub fn lq_mlp_get_grads(net: *const LqMlp, host: *mut f32, count: i64) -> c_int;
    pub fn lq_mlp_forward(net: *mut LqMlp, x: *const f32, batch: c_int, y: *mut f32) -> c_int;
    pub fn lq_mlp_loss_grad(net: *mut LqMlp, x: *const f32, target: *const f32, mask: *const f32, batch: c_int, loss: *mut f64) -> c_int;
    pub fn lq_mlp_backward(net: *mut LqMlp, x: *const f32, dy: *const f32, batch: c_int) -> c_int;
    pub fn lq_mlp_adam_step(net: *mut LqMlp, lr: f32, beta1: f32, beta2: f32, eps: f32) -> c_int;
    pub fn lq_mlp_reset_adam(net: *mut LqMlp) -> c_int;
    pub fn lq_lanczos_ground_energy(num_qubits: c_int, terms: *const LqPauliTerm, nterms: c_int, max_iter: c_int, tol: f64, seed: u64, e0: *mut f64, iters: *mut c_int) -> c_int;
    pub fn lq_last_error() -> *const c_char;
}
