//! logosq-cuda: LogosQ's dense state-vector path on one B200.
//!
//! `CudaState` is a device-resident `State` (src/states/mod.rs:38): the same
//! constructors, `normalize`, `probabilities`, `probability`,
//! `measure_shots_parallel`, `inner_product_parallel`, and the
//! `QuantumStateBackend` trait (src/states/backend.rs:14-60).  Gates are the
//! reference's own gate structs: `GpuGate` gives each of them its engine
//! descriptor, so `CudaState::apply_gate(&U3Gate { .. })` replaces
//! `Gate::apply` (src/gates/mod.rs:26-35) with one device sweep.  `GpuCircuit`
//! mirrors `Circuit`'s builders and submits the whole gate list at once, which
//! the engine plans into fused shared-memory passes (`Circuit::execute`,
//! src/circuits/mod.rs:352-375).  `expectation` replaces
//! `PauliObservable::expectation` (src/optimization/observable.rs:228-232) and
//! `CudaParameterShift` replaces `ParameterShift::compute_gradient`
//! (src/optimization/gradient.rs:44-78).
//!
//! Everything runs through the C ABI in `ffi` (generated from
//! include/logosq_b200.h by gen_ffi.py); there is no CPU fallback.

pub mod ffi;

use std::collections::HashMap;
use std::ffi::CStr;
use std::os::raw::c_int;
use std::ptr::{self, NonNull};

use logosq::gates::parameterized::{
    CPhaseParamGate, CRXGate, CRYGate, CRZGate, PhaseGate, RXGate, RXXGate, RYGate, RYYGate,
    RZGate, RZZGate, U3Gate,
};
use logosq::gates::single_qubit::{HGate, SGate, TGate, XGate, YGate, ZGate};
use logosq::gates::three_qubit::ToffoliGate;
use logosq::gates::two_qubit::{CNOTGate, CPhaseGate, CZGate, SWAPGate};
use logosq::optimization::observable::{Pauli, PauliObservable, PauliTerm};
use logosq::states::QuantumStateBackend;
use logosq::{LogosQError, Result, State};
use ndarray::{Array1, Array2};
use num_complex::Complex64;

// ---------------------------------------------------------------------------
// Status codes -> LogosQError
// ---------------------------------------------------------------------------

fn last_error() -> String {
    unsafe {
        let p = ffi::lq_last_error();
        if p.is_null() {
            String::new()
        } else {
            CStr::from_ptr(p).to_string_lossy().into_owned()
        }
    }
}

/// Map an engine status onto the reference's error enum (src/error.rs:9-61).
/// The engine reports qubit-index, dimension and count errors before any CUDA
/// call; those with fields the wrapper cannot know, and the engine-only codes
/// (invalid argument, out of memory, CUDA, timeout, unsupported), carry the
/// engine's message in `OptimizationError`.
fn check(rc: c_int) -> Result<()> {
    if rc == ffi::LQ_OK {
        return Ok(());
    }
    Err(LogosQError::OptimizationError { message: format!("engine status {}: {}", rc, last_error()) })
}

fn qubit_ok(q: usize, n: usize) -> Result<()> {
    if q >= n {
        return Err(LogosQError::InvalidQubitIndex { index: q, num_qubits: n });
    }
    Ok(())
}

// ---------------------------------------------------------------------------
// CudaState
// ---------------------------------------------------------------------------

/// A complex128 state vector resident in HBM, with its own CUDA stream.
pub struct CudaState {
    raw: NonNull<ffi::LqState>,
    num_qubits: usize,
}

// One host thread uses a handle at a time (the engine's threading rule);
// moving it between threads is fine.
unsafe impl Send for CudaState {}

impl Drop for CudaState {
    fn drop(&mut self) {
        unsafe {
            ffi::lq_state_destroy(self.raw.as_ptr());
        }
    }
}

impl CudaState {
    fn create(num_qubits: usize) -> Result<Self> {
        let mut p: *mut ffi::LqState = ptr::null_mut();
        check(unsafe { ffi::lq_state_create(num_qubits as c_int, ffi::LQ_C128, &mut p) })?;
        let raw = NonNull::new(p).ok_or_else(|| LogosQError::OptimizationError {
            message: "lq_state_create returned no handle".into(),
        })?;
        Ok(CudaState { raw, num_qubits })
    }

    fn ptr(&self) -> *mut ffi::LqState {
        self.raw.as_ptr()
    }

    /// |0...0> (State::zero_state, src/states/mod.rs:136-141).
    pub fn zero_state(num_qubits: usize) -> Self {
        Self::create(num_qubits).expect("device state allocation")
    }

    /// |1...1> (State::one_state, src/states/mod.rs:144-149).
    pub fn one_state(num_qubits: usize) -> Self {
        let s = Self::zero_state(num_qubits);
        let idx = if num_qubits >= 64 { u64::MAX } else { (1u64 << num_qubits) - 1 };
        check(unsafe { ffi::lq_state_set_basis(s.ptr(), idx) }).expect("set basis");
        s
    }

    /// |+...+> (State::plus_state, src/states/mod.rs:152-159).
    pub fn plus_state(num_qubits: usize) -> Self {
        let s = Self::zero_state(num_qubits);
        check(unsafe { ffi::lq_state_set_plus(s.ptr()) }).expect("set plus");
        s
    }

    /// (|00> + |11>)/sqrt(2) (State::bell_state, src/states/mod.rs:162-170).
    pub fn bell_state() -> Self {
        let h = std::f64::consts::FRAC_1_SQRT_2;
        let v = Array1::from(vec![
            Complex64::new(h, 0.0),
            Complex64::new(0.0, 0.0),
            Complex64::new(0.0, 0.0),
            Complex64::new(h, 0.0),
        ]);
        Self::new(v, Some(2)).expect("bell state")
    }

    /// State::new (src/states/mod.rs:55-75): the vector is uploaded and
    /// normalised on the device.
    pub fn new(vector: Array1<Complex64>, num_qubits: Option<usize>) -> Result<Self> {
        let len = vector.len();
        if len == 0 || !len.is_power_of_two() {
            return Err(LogosQError::InvalidStateDimension { dimension: len });
        }
        let n = num_qubits.unwrap_or(len.trailing_zeros() as usize);
        if 1usize << n != len {
            return Err(LogosQError::DimensionMismatch { expected: 1 << n, actual: len });
        }
        let mut s = Self::create(n)?;
        s.set_vector(&vector)?;
        s.normalize();
        Ok(s)
    }

    /// A device copy of a host `State`.
    pub fn from_state(state: &State) -> Result<Self> {
        let mut s = Self::create(state.num_qubits())?;
        s.set_vector(state.vector())?;
        Ok(s)
    }

    /// The amplitudes as a host `State`.
    pub fn to_state(&self) -> State {
        State::new_unchecked(self.vector(), self.num_qubits)
    }

    pub fn num_qubits(&self) -> usize {
        self.num_qubits
    }

    /// Download the amplitudes (State::vector, src/states/mod.rs:122).
    pub fn vector(&self) -> Array1<Complex64> {
        let mut v = vec![Complex64::new(0.0, 0.0); 1usize << self.num_qubits];
        check(unsafe {
            ffi::lq_state_download(self.ptr(), v.as_mut_ptr() as *mut f64, v.len())
        })
        .expect("download");
        Array1::from(v)
    }

    /// Overwrite the amplitudes (State::vector_mut, src/states/mod.rs:131-133).
    pub fn set_vector(&mut self, v: &Array1<Complex64>) -> Result<()> {
        if v.len() != 1usize << self.num_qubits {
            return Err(LogosQError::DimensionMismatch {
                expected: 1 << self.num_qubits,
                actual: v.len(),
            });
        }
        let host: Vec<Complex64> = v.iter().cloned().collect();
        check(unsafe { ffi::lq_state_upload(self.ptr(), host.as_ptr() as *const f64, host.len()) })
    }

    /// State::normalize (src/states/mod.rs:91-114).
    pub fn normalize(&mut self) {
        check(unsafe { ffi::lq_normalize(self.ptr()) }).expect("normalize");
    }

    /// State::probabilities (src/states/mod.rs:277-279).
    pub fn probabilities(&self) -> Vec<f64> {
        let mut p = vec![0.0f64; 1usize << self.num_qubits];
        check(unsafe { ffi::lq_probabilities(self.ptr(), p.as_mut_ptr(), p.len()) })
            .expect("probabilities");
        p
    }

    /// State::probability (src/states/mod.rs:288-293).
    pub fn probability(&self, basis_state: usize) -> f64 {
        let mut p = 0.0f64;
        check(unsafe { ffi::lq_probability(self.ptr(), basis_state as u64, &mut p) })
            .expect("probability");
        p
    }

    /// State::measure_shots_parallel (src/states/mod.rs:244-258): shots drawn
    /// on the device from a seeded counter-based generator, counted on the host.
    pub fn measure_shots_parallel(&self, n_shots: usize) -> HashMap<usize, usize> {
        self.measure_shots_seeded(n_shots, 0x5eed_1234_abcd_0001)
    }

    pub fn measure_shots_seeded(&self, n_shots: usize, seed: u64) -> HashMap<usize, usize> {
        let mut idx = vec![0u64; n_shots];
        check(unsafe {
            ffi::lq_measure_shots(self.ptr(), n_shots as u64, seed, idx.as_mut_ptr())
        })
        .expect("measure shots");
        let mut counts = HashMap::new();
        for i in idx {
            *counts.entry(i as usize).or_insert(0) += 1;
        }
        counts
    }

    /// State::inner_product_parallel (src/states/mod.rs:350-365).
    pub fn inner_product_parallel(&self, other: &CudaState) -> Result<Complex64> {
        if self.num_qubits != other.num_qubits {
            return Err(LogosQError::DimensionMismatch {
                expected: 1 << self.num_qubits,
                actual: 1 << other.num_qubits,
            });
        }
        let mut out = [0.0f64; 2];
        check(unsafe { ffi::lq_inner_product(self.ptr(), other.ptr(), out.as_mut_ptr()) })?;
        Ok(Complex64::new(out[0], out[1]))
    }

    /// Gate::apply of one reference gate struct: one device sweep.
    pub fn apply_gate<G: GpuGate + ?Sized>(&mut self, gate: &G) {
        let d = gate.descriptor();
        check(unsafe { ffi::lq_apply_gate(self.ptr(), &d, ptr::null(), 0) }).expect("apply gate");
    }

    /// Wait for the state's stream; reports a device wait that ran out.
    pub fn synchronize(&mut self) -> Result<()> {
        check(unsafe { ffi::lq_state_synchronize(self.ptr()) })
    }
}

fn interleave(m: &Array2<Complex64>, dim: usize) -> Result<Vec<f64>> {
    if m.shape() != [dim, dim] {
        return Err(LogosQError::InvalidGateMatrix {
            expected: vec![dim, dim],
            actual: m.shape().to_vec(),
        });
    }
    let mut out = Vec::with_capacity(2 * dim * dim);
    for r in 0..dim {
        for c in 0..dim {
            out.push(m[[r, c]].re);
            out.push(m[[r, c]].im);
        }
    }
    Ok(out)
}

/// The matrix entry points of the reference's dense `State`
/// (src/states/mod.rs:394-486): each applies its matrix on the device and then
/// renormalises, as the reference does.
impl QuantumStateBackend for CudaState {
    fn num_qubits(&self) -> usize {
        self.num_qubits
    }

    fn apply_single_qubit_matrix(&mut self, qubit: usize, matrix: &Array2<Complex64>) -> Result<()> {
        qubit_ok(qubit, self.num_qubits)?;
        let m = interleave(matrix, 2)?;
        check(unsafe { ffi::lq_apply_matrix1(self.ptr(), qubit as c_int, m.as_ptr()) })?;
        check(unsafe { ffi::lq_normalize(self.ptr()) })
    }

    fn apply_two_qubit_matrix(
        &mut self,
        control: usize,
        target: usize,
        matrix: &Array2<Complex64>,
    ) -> Result<()> {
        qubit_ok(control, self.num_qubits)?;
        qubit_ok(target, self.num_qubits)?;
        let m = interleave(matrix, 4)?;
        check(unsafe {
            ffi::lq_apply_matrix2(self.ptr(), control as c_int, target as c_int, m.as_ptr())
        })?;
        check(unsafe { ffi::lq_normalize(self.ptr()) })
    }

    /// As in the reference, the 8x8 matrix is applied to the full state.
    fn apply_three_qubit_matrix(
        &mut self,
        _q1: usize,
        _q2: usize,
        _q3: usize,
        matrix: &Array2<Complex64>,
    ) -> Result<()> {
        self.apply_full_matrix(matrix)
    }

    fn apply_full_matrix(&mut self, matrix: &Array2<Complex64>) -> Result<()> {
        let dim = 1usize << self.num_qubits;
        let m = interleave(matrix, dim)?;
        check(unsafe { ffi::lq_apply_dense(self.ptr(), m.as_ptr(), dim as u64) })?;
        check(unsafe { ffi::lq_normalize(self.ptr()) })
    }
}

// ---------------------------------------------------------------------------
// Gate descriptors for the reference's gate structs
// ---------------------------------------------------------------------------

fn desc(kind: c_int, qubits: &[usize], angles: &[f64]) -> ffi::LqGate {
    let mut g = ffi::LqGate {
        kind: kind as i32,
        flags: 0,
        q: [-1; 3],
        param: [-1; 3],
        angle: [0.0; 3],
        scale: [1.0; 3],
        m: [0.0; 32],
    };
    for (k, &q) in qubits.iter().enumerate() {
        g.q[k] = q as i32;
    }
    for (k, &a) in angles.iter().enumerate() {
        g.angle[k] = a;
    }
    g
}

/// The engine descriptor of a gate (the type-erased `Gate` trait carries no
/// parameters, so each reference gate struct provides its own).
pub trait GpuGate {
    fn descriptor(&self) -> ffi::LqGate;
}

macro_rules! one_qubit {
    ($t:ty, $k:expr) => {
        impl GpuGate for $t {
            fn descriptor(&self) -> ffi::LqGate {
                desc($k, &[self.qubit], &[])
            }
        }
    };
}
macro_rules! rotation {
    ($t:ty, $k:expr) => {
        impl GpuGate for $t {
            fn descriptor(&self) -> ffi::LqGate {
                desc($k, &[self.qubit], &[self.theta])
            }
        }
    };
}
macro_rules! controlled_rotation {
    ($t:ty, $k:expr) => {
        impl GpuGate for $t {
            fn descriptor(&self) -> ffi::LqGate {
                desc($k, &[self.control, self.target], &[self.theta])
            }
        }
    };
}
macro_rules! pair_rotation {
    ($t:ty, $k:expr) => {
        impl GpuGate for $t {
            fn descriptor(&self) -> ffi::LqGate {
                desc($k, &[self.qubit1, self.qubit2], &[self.theta])
            }
        }
    };
}

one_qubit!(HGate, ffi::LQ_GATE_H);
one_qubit!(XGate, ffi::LQ_GATE_X);
one_qubit!(YGate, ffi::LQ_GATE_Y);
one_qubit!(ZGate, ffi::LQ_GATE_Z);
one_qubit!(SGate, ffi::LQ_GATE_S);
one_qubit!(TGate, ffi::LQ_GATE_T);
rotation!(RXGate, ffi::LQ_GATE_RX);
rotation!(RYGate, ffi::LQ_GATE_RY);
rotation!(RZGate, ffi::LQ_GATE_RZ);
rotation!(PhaseGate, ffi::LQ_GATE_PHASE);
controlled_rotation!(CRXGate, ffi::LQ_GATE_CRX);
controlled_rotation!(CRYGate, ffi::LQ_GATE_CRY);
controlled_rotation!(CRZGate, ffi::LQ_GATE_CRZ);
controlled_rotation!(CPhaseParamGate, ffi::LQ_GATE_CPHASE_PARAM);
pair_rotation!(RXXGate, ffi::LQ_GATE_RXX);
pair_rotation!(RYYGate, ffi::LQ_GATE_RYY);
pair_rotation!(RZZGate, ffi::LQ_GATE_RZZ);

impl GpuGate for U3Gate {
    fn descriptor(&self) -> ffi::LqGate {
        desc(ffi::LQ_GATE_U3, &[self.qubit], &[self.theta, self.phi, self.lambda])
    }
}
impl GpuGate for CNOTGate {
    fn descriptor(&self) -> ffi::LqGate {
        desc(ffi::LQ_GATE_CNOT, &[self.control, self.target], &[])
    }
}
impl GpuGate for CZGate {
    fn descriptor(&self) -> ffi::LqGate {
        desc(ffi::LQ_GATE_CZ, &[self.control, self.target], &[])
    }
}
impl GpuGate for CPhaseGate {
    fn descriptor(&self) -> ffi::LqGate {
        desc(ffi::LQ_GATE_CPHASE, &[self.control, self.target], &[self.angle])
    }
}
impl GpuGate for SWAPGate {
    fn descriptor(&self) -> ffi::LqGate {
        desc(ffi::LQ_GATE_SWAP, &[self.qubit1, self.qubit2], &[])
    }
}
impl GpuGate for ToffoliGate {
    fn descriptor(&self) -> ffi::LqGate {
        desc(ffi::LQ_GATE_TOFFOLI, &[self.control1, self.control2, self.target], &[])
    }
}
impl GpuGate for ffi::LqGate {
    fn descriptor(&self) -> ffi::LqGate {
        *self
    }
}

// ---------------------------------------------------------------------------
// GpuCircuit: Circuit's builders, submitted as one gate list
// ---------------------------------------------------------------------------

/// A gate list with `Circuit`'s builder methods (src/circuits/parameterized.rs,
/// two_qubits.rs).  A gate may take an angle from a parameter vector
/// (`*_param` builders: angle = theta[index]), which is how an ansatz is
/// described once for `CudaParameterShift`.
#[derive(Clone, Debug, Default)]
pub struct GpuCircuit {
    ops: Vec<ffi::LqGate>,
    num_qubits: usize,
}

impl GpuCircuit {
    pub fn new(num_qubits: usize) -> Self {
        GpuCircuit { ops: Vec::new(), num_qubits }
    }
    pub fn num_qubits(&self) -> usize {
        self.num_qubits
    }
    pub fn num_operations(&self) -> usize {
        self.ops.len()
    }
    pub fn add<G: GpuGate + ?Sized>(&mut self, gate: &G) -> &mut Self {
        self.ops.push(gate.descriptor());
        self
    }
    fn push(&mut self, kind: c_int, qubits: &[usize], angles: &[f64]) -> &mut Self {
        self.ops.push(desc(kind, qubits, angles));
        self
    }
    fn push_param(&mut self, kind: c_int, qubits: &[usize], index: usize) -> &mut Self {
        let mut g = desc(kind, qubits, &[0.0]);
        g.param[0] = index as i32;
        self.ops.push(g);
        self
    }
    pub fn h(&mut self, q: usize) -> &mut Self { self.push(ffi::LQ_GATE_H, &[q], &[]) }
    pub fn x(&mut self, q: usize) -> &mut Self { self.push(ffi::LQ_GATE_X, &[q], &[]) }
    pub fn y(&mut self, q: usize) -> &mut Self { self.push(ffi::LQ_GATE_Y, &[q], &[]) }
    pub fn z(&mut self, q: usize) -> &mut Self { self.push(ffi::LQ_GATE_Z, &[q], &[]) }
    pub fn s(&mut self, q: usize) -> &mut Self { self.push(ffi::LQ_GATE_S, &[q], &[]) }
    pub fn t(&mut self, q: usize) -> &mut Self { self.push(ffi::LQ_GATE_T, &[q], &[]) }
    pub fn rx(&mut self, q: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_RX, &[q], &[theta]) }
    pub fn ry(&mut self, q: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_RY, &[q], &[theta]) }
    pub fn rz(&mut self, q: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_RZ, &[q], &[theta]) }
    pub fn phase(&mut self, q: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_PHASE, &[q], &[theta]) }
    pub fn u3(&mut self, q: usize, theta: f64, phi: f64, lambda: f64) -> &mut Self {
        self.push(ffi::LQ_GATE_U3, &[q], &[theta, phi, lambda])
    }
    pub fn cnot(&mut self, c: usize, t: usize) -> &mut Self { self.push(ffi::LQ_GATE_CNOT, &[c, t], &[]) }
    pub fn swap(&mut self, a: usize, b: usize) -> &mut Self { self.push(ffi::LQ_GATE_SWAP, &[a, b], &[]) }
    pub fn cz(&mut self, c: usize, t: usize) -> &mut Self { self.push(ffi::LQ_GATE_CZ, &[c, t], &[]) }
    pub fn cphase(&mut self, c: usize, t: usize, angle: f64) -> &mut Self {
        self.push(ffi::LQ_GATE_CPHASE, &[c, t], &[angle])
    }
    pub fn toffoli(&mut self, c1: usize, c2: usize, t: usize) -> &mut Self {
        self.push(ffi::LQ_GATE_TOFFOLI, &[c1, c2, t], &[])
    }
    pub fn crx(&mut self, c: usize, t: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_CRX, &[c, t], &[theta]) }
    pub fn cry(&mut self, c: usize, t: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_CRY, &[c, t], &[theta]) }
    pub fn crz(&mut self, c: usize, t: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_CRZ, &[c, t], &[theta]) }
    pub fn rxx(&mut self, a: usize, b: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_RXX, &[a, b], &[theta]) }
    pub fn ryy(&mut self, a: usize, b: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_RYY, &[a, b], &[theta]) }
    pub fn rzz(&mut self, a: usize, b: usize, theta: f64) -> &mut Self { self.push(ffi::LQ_GATE_RZZ, &[a, b], &[theta]) }
    pub fn rx_param(&mut self, q: usize, index: usize) -> &mut Self { self.push_param(ffi::LQ_GATE_RX, &[q], index) }
    pub fn ry_param(&mut self, q: usize, index: usize) -> &mut Self { self.push_param(ffi::LQ_GATE_RY, &[q], index) }
    pub fn rz_param(&mut self, q: usize, index: usize) -> &mut Self { self.push_param(ffi::LQ_GATE_RZ, &[q], index) }

    fn check_qubits(&self, state: &CudaState) -> Result<()> {
        if self.num_qubits != state.num_qubits() {
            return Err(LogosQError::CircuitQubitMismatch {
                circuit_qubits: self.num_qubits,
                state_qubits: state.num_qubits(),
            });
        }
        Ok(())
    }

    /// Circuit::execute (src/circuits/mod.rs:352-375): the whole list in one
    /// call, planned into fused shared-memory passes.
    pub fn execute(&self, state: &mut CudaState) -> Result<()> {
        self.execute_bound(state, &[])
    }

    /// Same, with the parameter vector the `*_param` gates read.
    pub fn execute_bound(&self, state: &mut CudaState, theta: &[f64]) -> Result<()> {
        self.check_qubits(state)?;
        check(unsafe {
            ffi::lq_apply_circuit(
                state.ptr(),
                self.num_qubits as c_int,
                self.ops.as_ptr(),
                self.ops.len() as c_int,
                if theta.is_empty() { ptr::null() } else { theta.as_ptr() },
                theta.len() as c_int,
                ffi::LQ_EXEC_FUSED,
            )
        })
    }

    /// One device sweep per gate, in order (the Gate::apply path).
    pub fn execute_per_gate(&self, state: &mut CudaState) -> Result<()> {
        self.check_qubits(state)?;
        check(unsafe {
            ffi::lq_apply_circuit(
                state.ptr(),
                self.num_qubits as c_int,
                self.ops.as_ptr(),
                self.ops.len() as c_int,
                ptr::null(),
                0,
                ffi::LQ_EXEC_PER_GATE,
            )
        })
    }
}

// ---------------------------------------------------------------------------
// Observables and gradients
// ---------------------------------------------------------------------------

/// PauliTerm (src/optimization/observable.rs:79-83) packed as X/Z bit masks
/// over basis bits (qubit q is bit n-1-q) and its Y count.
pub fn pack_term(term: &PauliTerm) -> ffi::LqPauliTerm {
    let n = term.paulis.len();
    let (mut x, mut z, mut ny) = (0u64, 0u64, 0i32);
    for (q, p) in term.paulis.iter().enumerate() {
        let bit = 1u64 << (n - 1 - q);
        match p {
            Pauli::I => {}
            Pauli::X => x |= bit,
            Pauli::Z => z |= bit,
            Pauli::Y => {
                x |= bit;
                z |= bit;
                ny += 1;
            }
        }
    }
    ffi::LqPauliTerm { coefficient: term.coefficient, xmask: x, zmask: z, ny, reserved: 0 }
}

/// PauliObservable::expectation (src/optimization/observable.rs:228-232) on
/// the device, FP64 accumulation, the reference's Y convention.
pub fn expectation(observable: &PauliObservable, state: &CudaState) -> Result<f64> {
    let terms: Vec<ffi::LqPauliTerm> = observable.terms.iter().map(pack_term).collect();
    let mut e = 0.0f64;
    check(unsafe {
        ffi::lq_expectation_pauli(
            state.ptr(),
            terms.as_ptr(),
            terms.len() as c_int,
            ffi::LQ_Y_REFERENCE,
            &mut e,
            ptr::null_mut(),
        )
    })?;
    Ok(e)
}

/// ParameterShift::compute_gradient (src/optimization/gradient.rs:44-78):
/// g_i = (E(theta + s e_i) - E(theta - s e_i)) / 2 for every parameter, with
/// the ansatz given once as a parameterised `GpuCircuit`.
pub struct CudaParameterShift {
    pub shift: f64,
}

impl Default for CudaParameterShift {
    fn default() -> Self {
        CudaParameterShift { shift: std::f64::consts::PI / 2.0 }
    }
}

impl CudaParameterShift {
    pub fn new() -> Self {
        Self::default()
    }
    pub fn with_shift(shift: f64) -> Self {
        CudaParameterShift { shift }
    }

    pub fn compute_gradient(
        &self,
        ansatz: &GpuCircuit,
        observable: &PauliObservable,
        parameters: &[f64],
    ) -> Result<Vec<f64>> {
        let mut work = CudaState::create(ansatz.num_qubits())?;
        let terms: Vec<ffi::LqPauliTerm> = observable.terms.iter().map(pack_term).collect();
        let mut grad = vec![0.0f64; parameters.len()];
        check(unsafe {
            ffi::lq_parameter_shift(
                work.ptr(),
                ansatz.ops.as_ptr(),
                ansatz.ops.len() as c_int,
                parameters.as_ptr(),
                parameters.len() as c_int,
                terms.as_ptr(),
                terms.len() as c_int,
                ffi::LQ_Y_REFERENCE,
                self.shift,
                grad.as_mut_ptr(),
            )
        })?;
        work.synchronize()?;
        Ok(grad)
    }
}
