/*
 * logosq_oracle.cpp -- CPU restatement of the LogosQ dense state-vector path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
 * baseline; it is never linked into, loaded by, or called from the product
 * library.  Only the test suite, the smoke check and the CPU-baseline leg of
 * the benchmark load it.
 *
 * The reference (zazabap/LogosQ 0.2.5) is Rust and cannot be compiled in this
 * environment (no cargo/rustc), so each loop below restates the reference loop
 * it cites, statement for statement, in C++:
 *   - complex arithmetic follows num-complex 0.4 Complex<f64> exactly:
 *       (a*b).re = a.re*b.re - a.im*b.im, (a*b).im = a.re*b.im + a.im*b.re,
 *       from_polar(r, t) = (r*cos t, r*sin t), c / f = (re/f, im/f);
 *   - the file is compiled with -ffp-contract=off, since rustc never fuses a
 *     multiply and an add into an FMA;
 *   - cos/sin come from glibc, as Rust's f64::cos/sin do on Linux.
 * Two execution modes share the per-amplitude arithmetic:
 *   faithful (threads = 1): serial wherever the reference is serial, rayon-like
 *       parallel loops where the reference uses rayon (CPhaseGate when
 *       2^n > 1024, normalize);
 *   threaded (threads > 1): every gate loop split over OpenMP threads.  Each
 *       amplitude sees the same operations in the same order, so the result is
 *       bitwise identical to faithful mode.
 * Parity pins: tests/test_oracle_golden.py checks this file against every
 * known-answer assertion of the reference's own tests for this path
 * (tests/test_circuits_dense.rs, test_gates_parameterized.rs, test_qft.rs,
 * test_optimization_observables.rs, test_optimization_gradient.rs,
 * test_parallel.rs, test_normalize.rs), against numpy matrix products, and
 * against the numpy FFT for the QFT.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

#include "../include/logosq_b200.h"

namespace {

struct C {
    double re, im;
};
inline C cmul(C a, C b) { return C{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C cadd(C a, C b) { return C{a.re + b.re, a.im + b.im}; }
inline C csub(C a, C b) { return C{a.re - b.re, a.im - b.im}; }
inline C cneg(C a) { return C{-a.re, -a.im}; }
inline C cconj(C a) { return C{a.re, -a.im}; }
inline C polar(double r, double t) { return C{r * std::cos(t), r * std::sin(t)}; }
inline C cre(double x) { return C{x, 0.0}; }

int g_threads = 1;  // 1 = faithful mode

inline int nthreads_for_loop() { return g_threads > 1 ? g_threads : 1; }

// Resolve angle k of a descriptor against the parameter vector.
inline double ang(const lq_gate *g, int k, const double *theta) {
    if (g->param[k] >= 0) return theta[g->param[k]] * g->scale[k] + g->angle[k];
    return g->angle[k];
}

// Single-qubit 2x2 sweep in the loop shape of U3Gate::apply
// (src/gates/parameterized.rs:264-281): for base step 2*stride, for offset.
// out0 = m00*a0 + m01*a1 ; out1 = m10*a0 + m11*a1 (the reference's order).
void sweep_2x2(C *v, int n, int q, C m00, C m01, C m10, C m11) {
    const uint64_t stride = 1ull << (n - 1 - q);
    const uint64_t full = 1ull << n;
    const int64_t nblocks = (int64_t)(full / (2 * stride));
#pragma omp parallel for num_threads(nthreads_for_loop()) schedule(static) if (g_threads > 1)
    for (int64_t blk = 0; blk < nblocks; ++blk) {
        const uint64_t base = (uint64_t)blk * 2 * stride;
        for (uint64_t off = 0; off < stride; ++off) {
            const uint64_t i0 = base + off, i1 = i0 + stride;
            const C a0 = v[i0], a1 = v[i1];
            v[i0] = cadd(cmul(m00, a0), cmul(m01, a1));
            v[i1] = cadd(cmul(m10, a0), cmul(m11, a1));
        }
    }
}

// Large-stride sweeps split the inner loop instead (only one block when q = 0).
void sweep_2x2_inner_parallel(C *v, int n, int q, C m00, C m01, C m10, C m11) {
    const uint64_t stride = 1ull << (n - 1 - q);
    const uint64_t full = 1ull << n;
    for (uint64_t base = 0; base < full; base += 2 * stride) {
#pragma omp parallel for num_threads(nthreads_for_loop()) schedule(static) if (g_threads > 1)
        for (int64_t off = 0; off < (int64_t)stride; ++off) {
            const uint64_t i0 = base + off, i1 = i0 + stride;
            const C a0 = v[i0], a1 = v[i1];
            v[i0] = cadd(cmul(m00, a0), cmul(m01, a1));
            v[i1] = cadd(cmul(m10, a0), cmul(m11, a1));
        }
    }
}

void apply_2x2(C *v, int n, int q, C m00, C m01, C m10, C m11) {
    const uint64_t stride = 1ull << (n - 1 - q);
    if (g_threads > 1 && (1ull << n) / (2 * stride) < (uint64_t)g_threads * 4)
        sweep_2x2_inner_parallel(v, n, q, m00, m01, m10, m11);
    else
        sweep_2x2(v, n, q, m00, m01, m10, m11);
}

// Full-index sweep with a per-index functor, split over threads in threaded mode.
template <class F>
void for_all(int n, F f, bool force_parallel = false) {
    const int64_t full = (int64_t)(1ull << n);
    const bool par = g_threads > 1 || force_parallel;
    const int nt = g_threads > 1 ? g_threads : omp_get_max_threads();
#pragma omp parallel for num_threads(nt) schedule(static) if (par)
    for (int64_t i = 0; i < full; ++i) f((uint64_t)i);
}

// MatrixGate::apply renormalises (src/gates/mod.rs:89-91): State::normalize.
void normalize(C *v, int n);

void apply_one(C *v, int n, const lq_gate *g, const double *theta) {
    const int q0 = g->q[0], q1 = g->q[1], q2 = g->q[2];
    switch (g->kind) {
    case LQ_GATE_X: {  // src/gates/single_qubit.rs:14-31: swap(idx0, idx1)
        const uint64_t stride = 1ull << (n - 1 - q0);
        for_all(n, [&](uint64_t i) {
            if ((i & stride) == 0) { C t = v[i]; v[i] = v[i + stride]; v[i + stride] = t; }
        });
        break;
    }
    case LQ_GATE_Y: {  // src/gates/single_qubit.rs:39-58: v0 = i*v1, v1 = -i*v0
        const uint64_t stride = 1ull << (n - 1 - q0);
        for_all(n, [&](uint64_t i) {
            if ((i & stride) == 0) {
                const C temp = v[i];
                v[i] = cmul(C{0.0, 1.0}, v[i + stride]);
                v[i + stride] = cmul(C{0.0, -1.0}, temp);
            }
        });
        break;
    }
    case LQ_GATE_Z: {  // src/gates/single_qubit.rs:67-82
        const uint64_t mask = 1ull << (n - 1 - q0);
        for_all(n, [&](uint64_t i) { if (i & mask) v[i] = cneg(v[i]); });
        break;
    }
    case LQ_GATE_H: {  // src/gates/single_qubit.rs:90-113: s*(a0+a1), s*(a0-a1)
        const C s = cre(1.0 / M_SQRT2);
        const uint64_t stride = 1ull << (n - 1 - q0);
        for_all(n, [&](uint64_t i) {
            if ((i & stride) == 0) {
                const C a0 = v[i], a1 = v[i + stride];
                v[i] = cmul(s, cadd(a0, a1));
                v[i + stride] = cmul(s, csub(a0, a1));
            }
        });
        break;
    }
    case LQ_GATE_S: {  // src/gates/single_qubit.rs:121-137
        const uint64_t mask = 1ull << (n - 1 - q0);
        const C ph{0.0, 1.0};
        for_all(n, [&](uint64_t i) { if (i & mask) v[i] = cmul(v[i], ph); });
        break;
    }
    case LQ_GATE_T: {  // src/gates/single_qubit.rs:145-161
        const uint64_t mask = 1ull << (n - 1 - q0);
        const C ph = polar(1.0, M_PI / 4.0);
        for_all(n, [&](uint64_t i) { if (i & mask) v[i] = cmul(v[i], ph); });
        break;
    }
    case LQ_GATE_RX: {  // src/gates/parameterized.rs:48-80
        const double th = ang(g, 0, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        apply_2x2(v, n, q0, C{c, 0.0}, C{0.0, -s}, C{0.0, -s}, C{c, 0.0});
        break;
    }
    case LQ_GATE_RY: {  // src/gates/parameterized.rs:101-133
        const double th = ang(g, 0, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        apply_2x2(v, n, q0, C{c, 0.0}, C{-s, 0.0}, C{s, 0.0}, C{c, 0.0});
        break;
    }
    case LQ_GATE_RZ: {  // src/gates/parameterized.rs:154-178
        const double th = ang(g, 0, theta);
        const C p0 = polar(1.0, -th / 2.0), p1 = polar(1.0, th / 2.0);
        const uint64_t mask = 1ull << (n - 1 - q0);
        for_all(n, [&](uint64_t i) { v[i] = cmul(v[i], (i & mask) == 0 ? p0 : p1); });
        break;
    }
    case LQ_GATE_PHASE: {  // src/gates/parameterized.rs:199-218
        const C ph = polar(1.0, ang(g, 0, theta));
        const uint64_t mask = 1ull << (n - 1 - q0);
        for_all(n, [&](uint64_t i) { if (i & mask) v[i] = cmul(v[i], ph); });
        break;
    }
    case LQ_GATE_U3: {  // src/gates/parameterized.rs:249-282
        const double th = ang(g, 0, theta), phi = ang(g, 1, theta), lam = ang(g, 2, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        const C m00 = C{c, 0.0};
        const C m01 = cneg(polar(s, lam));
        const C m10 = polar(s, phi);
        const C m11 = polar(c, phi + lam);
        apply_2x2(v, n, q0, m00, m01, m10, m11);
        break;
    }
    case LQ_GATE_CNOT: {  // src/gates/two_qubit.rs:12-31
        const uint64_t cm = 1ull << (n - 1 - q0), tm = 1ull << (n - 1 - q1);
        for_all(n, [&](uint64_t i) {
            if ((i & cm) != 0 && (i & tm) == 0) {
                const uint64_t j = i ^ tm;
                C t = v[i]; v[i] = v[j]; v[j] = t;
            }
        });
        break;
    }
    case LQ_GATE_SWAP: {  // src/gates/two_qubit.rs:40-62
        const uint64_t m1 = 1ull << (n - 1 - q0), m2 = 1ull << (n - 1 - q1);
        for_all(n, [&](uint64_t i) {
            if ((i & m1) != 0 && (i & m2) == 0) {
                const uint64_t j = i ^ m1 ^ m2;
                C t = v[i]; v[i] = v[j]; v[j] = t;
            }
        });
        break;
    }
    case LQ_GATE_CZ: {  // src/gates/two_qubit.rs:71-92
        const uint64_t both = (1ull << (n - 1 - q0)) | (1ull << (n - 1 - q1));
        for_all(n, [&](uint64_t i) { if ((i & both) == both) v[i] = cneg(v[i]); });
        break;
    }
    case LQ_GATE_CPHASE: {  // src/gates/two_qubit.rs:100-134 (rayon when 2^n > 1024)
        const uint64_t both = (1ull << (n - 1 - q0)) | (1ull << (n - 1 - q1));
        const C ph = polar(1.0, ang(g, 0, theta));
        for_all(n, [&](uint64_t i) { if ((i & both) == both) v[i] = cmul(v[i], ph); },
                (1ull << n) > 1024);
        break;
    }
    case LQ_GATE_TOFFOLI: {  // src/gates/three_qubit.rs:13-35
        const uint64_t c1 = 1ull << (n - 1 - q0), c2 = 1ull << (n - 1 - q1);
        const uint64_t tm = 1ull << (n - 1 - q2), cs = c1 | c2;
        for_all(n, [&](uint64_t i) {
            if ((i & cs) == cs && (i & tm) == 0) {
                const uint64_t j = i ^ tm;
                C t = v[i]; v[i] = v[j]; v[j] = t;
            }
        });
        break;
    }
    case LQ_GATE_CRX:    // src/gates/parameterized.rs:311-343
    case LQ_GATE_CRY: {  // src/gates/parameterized.rs:368-399
        const double th = ang(g, 0, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        C m00{c, 0.0}, m11{c, 0.0}, m01, m10;
        if (g->kind == LQ_GATE_CRX) { m01 = C{0.0, -s}; m10 = C{0.0, -s}; }
        else { m01 = C{-s, 0.0}; m10 = C{s, 0.0}; }
        const uint64_t cm = 1ull << (n - 1 - q0), tm = 1ull << (n - 1 - q1);
        for_all(n, [&](uint64_t i) {
            if ((i & cm) != 0 && (i & tm) == 0) {
                const uint64_t j = i | tm;
                const C a0 = v[i], a1 = v[j];
                v[i] = cadd(cmul(m00, a0), cmul(m01, a1));
                v[j] = cadd(cmul(m10, a0), cmul(m11, a1));
            }
        });
        break;
    }
    case LQ_GATE_CRZ: {  // src/gates/parameterized.rs:424-451
        const double th = ang(g, 0, theta);
        const uint64_t cm = 1ull << (n - 1 - q0), tm = 1ull << (n - 1 - q1);
        const C p0 = polar(1.0, -th / 2.0), p1 = polar(1.0, th / 2.0);
        for_all(n, [&](uint64_t i) {
            if ((i & cm) != 0) v[i] = cmul(v[i], (i & tm) == 0 ? p0 : p1);
        });
        break;
    }
    case LQ_GATE_CPHASE_PARAM: {  // src/gates/parameterized.rs:476-499
        const uint64_t both = (1ull << (n - 1 - q0)) | (1ull << (n - 1 - q1));
        const C ph = polar(1.0, ang(g, 0, theta));
        for_all(n, [&](uint64_t i) { if ((i & both) == both) v[i] = cmul(v[i], ph); });
        break;
    }
    case LQ_GATE_RXX:    // src/gates/parameterized.rs:528-580
    case LQ_GATE_RYY: {  // src/gates/parameterized.rs:604-655
        const double th = ang(g, 0, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        const uint64_t m1 = 1ull << (n - 1 - q0), m2 = 1ull << (n - 1 - q1);
        // |00>,|11> block: RXX uses -i s, RYY uses +i s; |01>,|10> block: -i s.
        const C off_a = g->kind == LQ_GATE_RXX ? C{0.0, -s} : C{0.0, s};
        const C off_b = C{0.0, -s};
        const C cc{c, 0.0};
        const bool textbook = (g->flags & LQ_FLAG_TEXTBOOK) != 0;
        // The loop is inherently sequential in the reference (pairs chosen by i < j);
        // each pair is visited exactly once, so a parallel split is still exact.
        for_all(n, [&](uint64_t i) {
            const bool b1 = (i & m1) != 0, b2 = (i & m2) != 0;
            if (!b1 && !b2) {
                const uint64_t j = i | m1 | m2;
                if (i < j) {
                    const C ai = v[i], aj = v[j];
                    v[i] = cadd(cmul(cc, ai), cmul(off_a, aj));
                    v[j] = cadd(cmul(off_a, ai), cmul(cc, aj));
                }
            } else if (b1 && !b2) {
                const uint64_t j = (i & ~m1) | m2;
                if (i < j || textbook) {
                    const C ai = v[i], aj = v[j];
                    v[i] = cadd(cmul(cc, ai), cmul(off_b, aj));
                    v[j] = cadd(cmul(off_b, ai), cmul(cc, aj));
                }
            }
        });
        break;
    }
    case LQ_GATE_RZZ: {  // src/gates/parameterized.rs:679-709
        const double th = ang(g, 0, theta);
        const uint64_t m1 = 1ull << (n - 1 - q0), m2 = 1ull << (n - 1 - q1);
        const C same = polar(1.0, -th / 2.0), diff = polar(1.0, th / 2.0);
        for_all(n, [&](uint64_t i) {
            const bool b1 = (i & m1) != 0, b2 = (i & m2) != 0;
            v[i] = cmul(v[i], b1 == b2 ? same : diff);
        });
        break;
    }
    case LQ_GATE_MATRIX1: {
        // Circuit::x/h/... build kron(I.., M, ..I) and apply it as a dense
        // MatrixGate (src/circuits/single_qubit.rs:12-60, src/gates/mod.rs:76-93):
        // new_i = sum_j F_ij v_j.  Only two F_ij are non-zero per row, so the
        // dense dot reduces to m[r][0]*v_{i0} + m[r][1]*v_{i1} (zeros add exactly).
        const C m00{g->m[0], g->m[1]}, m01{g->m[2], g->m[3]};
        const C m10{g->m[4], g->m[5]}, m11{g->m[6], g->m[7]};
        apply_2x2(v, n, q0, m00, m01, m10, m11);
        break;
    }
    case LQ_GATE_MATRIX2: {
        // Circuit::add_two_qubit_gate (src/circuits/two_qubits.rs:11-82).
        const uint64_t m1 = 1ull << (n - 1 - q0), m2 = 1ull << (n - 1 - q1);
        C M[4][4];
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) M[r][c] = C{g->m[(r * 4 + c) * 2], g->m[(r * 4 + c) * 2 + 1]};
        for_all(n, [&](uint64_t i) {
            if ((i & m1) == 0 && (i & m2) == 0) {
                const uint64_t idx[4] = {i, i | m2, i | m1, i | m1 | m2};
                C a[4], o[4];
                for (int r = 0; r < 4; ++r) a[r] = v[idx[r]];
                for (int r = 0; r < 4; ++r) {
                    C acc{0.0, 0.0};
                    for (int c = 0; c < 4; ++c) acc = cadd(acc, cmul(M[r][c], a[c]));
                    o[r] = acc;
                }
                for (int r = 0; r < 4; ++r) v[idx[r]] = o[r];
            }
        });
        break;
    }
    default:
        break;
    }
    if (g->flags & LQ_FLAG_RENORM) normalize(v, n);
}

// State::normalize (src/states/mod.rs:91-114): parallel sum of norm_sqr, sqrt,
// divide when > 1e-10.
void normalize(C *v, int n) {
    const int64_t full = (int64_t)(1ull << n);
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (int64_t i = 0; i < full; ++i) acc += v[i].re * v[i].re + v[i].im * v[i].im;
    const double norm = std::sqrt(acc);
    if (norm > 1e-10) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < full; ++i) v[i] = C{v[i].re / norm, v[i].im / norm};
    }
}

// PauliTerm::expectation (src/optimization/observable.rs:95-147) over the packed
// masks.  The per-index phase is built factor by factor in qubit order as the
// reference does: amplitude *= (bit ? -i : i) per Y (reference convention),
// amplitude *= -1 per Z with bit set.
double pauli_term(const C *v, int n, const lq_pauli_term *t, int yconv, const uint8_t *kind) {
    const int64_t dim = (int64_t)(1ull << n);
    C result{0.0, 0.0};
    for (int64_t ii = 0; ii < dim; ++ii) {
        const uint64_t i = (uint64_t)ii;
        C amplitude{1.0, 0.0};
        uint64_t j = i;
        for (int q = 0; q < n; ++q) {
            const uint64_t bitmask = 1ull << (n - 1 - q);
            const int bit = (i & bitmask) ? 1 : 0;
            switch (kind[q]) {
            case 1: j ^= bitmask; break;  // X
            case 2:                       // Y
                j ^= bitmask;
                if (yconv == LQ_Y_REFERENCE)
                    amplitude = cmul(amplitude, bit == 0 ? C{0.0, 1.0} : C{0.0, -1.0});
                else
                    amplitude = cmul(amplitude, bit == 0 ? C{0.0, -1.0} : C{0.0, 1.0});
                break;
            case 3:  // Z
                if (bit == 1) amplitude = cmul(amplitude, C{-1.0, 0.0});
                break;
            default: break;
            }
        }
        result = cadd(result, cmul(cmul(cconj(v[i]), amplitude), v[j]));
    }
    return t->coefficient * result.re;
}

void decode_term(const lq_pauli_term *t, int n, uint8_t *kind) {
    for (int q = 0; q < n; ++q) {
        const uint64_t b = 1ull << (n - 1 - q);
        const bool x = (t->xmask & b) != 0, z = (t->zmask & b) != 0;
        kind[q] = x && z ? 2 : x ? 1 : z ? 3 : 0;
    }
}

double observable(const C *v, int n, const lq_pauli_term *terms, int nterms, int yconv) {
    // PauliObservable::expectation (src/optimization/observable.rs:228-232):
    // terms.iter().map(expectation).sum() -- sequential sum in term order.
    std::vector<uint8_t> kind(n);
    double sum = 0.0;
    for (int t = 0; t < nterms; ++t) {
        decode_term(&terms[t], n, kind.data());
        sum += pauli_term(v, n, &terms[t], yconv, kind.data());
    }
    return sum;
}

void run_circuit(C *v, int n, const lq_gate *ops, int nops, const double *theta) {
    // Circuit::execute (src/circuits/mod.rs:352-375) without noise models.
    for (int k = 0; k < nops; ++k) apply_one(v, n, &ops[k], theta);
}

double ansatz_energy(int n, const lq_gate *ops, int nops, const double *theta,
                     const lq_pauli_term *terms, int nterms, int yconv, std::vector<C> &buf) {
    // VQE objective (src/optimization/vqe.rs:63-67): zero_state, ansatz.apply,
    // hamiltonian.expectation.
    std::fill(buf.begin(), buf.end(), C{0.0, 0.0});
    buf[0] = C{1.0, 0.0};
    run_circuit(buf.data(), n, ops, nops, theta);
    return observable(buf.data(), n, terms, nterms, yconv);
}

}  // namespace

extern "C" {

/* Thread count of every later call: 1 = faithful mode, >1 = threaded mode. */
void or_set_threads(int threads) { g_threads = threads < 1 ? 1 : threads; }
int or_get_threads(void) { return g_threads; }
int or_max_threads(void) { return omp_get_max_threads(); }

void or_apply_gate(double *psi, int n, const lq_gate *g, const double *theta) {
    apply_one(reinterpret_cast<C *>(psi), n, g, theta);
}

void or_apply_circuit(double *psi, int n, const lq_gate *ops, int nops, const double *theta) {
    run_circuit(reinterpret_cast<C *>(psi), n, ops, nops, theta);
}

void or_normalize(double *psi, int n) { normalize(reinterpret_cast<C *>(psi), n); }

double or_norm_sqr(const double *psi, int n) {
    const C *v = reinterpret_cast<const C *>(psi);
    const int64_t full = (int64_t)(1ull << n);
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (int64_t i = 0; i < full; ++i) acc += v[i].re * v[i].re + v[i].im * v[i].im;
    return acc;
}

/* State::probabilities (src/states/mod.rs:277-279): norm_sqr per amplitude. */
void or_probabilities(const double *psi, int n, double *out) {
    const C *v = reinterpret_cast<const C *>(psi);
    const uint64_t full = 1ull << n;
    for (uint64_t i = 0; i < full; ++i) out[i] = v[i].re * v[i].re + v[i].im * v[i].im;
}

/* inner_product_parallel (src/states/mod.rs:350-365): map conj(a)*b, then a
 * sequential sum in index order. */
void or_inner_product(const double *a, const double *b, int n, double *out) {
    const C *x = reinterpret_cast<const C *>(a);
    const C *y = reinterpret_cast<const C *>(b);
    const uint64_t full = 1ull << n;
    C acc{0.0, 0.0};
    for (uint64_t i = 0; i < full; ++i) acc = cadd(acc, cmul(cconj(x[i]), y[i]));
    out[0] = acc.re;
    out[1] = acc.im;
}

double or_pauli_term(const double *psi, int n, const lq_pauli_term *t, int yconv) {
    std::vector<uint8_t> kind(n);
    decode_term(t, n, kind.data());
    return pauli_term(reinterpret_cast<const C *>(psi), n, t, yconv, kind.data());
}

double or_expectation(const double *psi, int n, const lq_pauli_term *terms, int nterms, int yconv) {
    return observable(reinterpret_cast<const C *>(psi), n, terms, nterms, yconv);
}

/* xyz_heisenberg::calculate_energy_efficient (src/algorithms/xyz_heisenberg.rs:143-163)
 * with expectation_xx/yy/zz/z (:166-252), uniform couplings. */
double or_heisenberg_energy(const double *psi, int n, double jx, double jy, double jz, double h) {
    const C *v = reinterpret_cast<const C *>(psi);
    const uint64_t dim = 1ull << n;
    double energy = 0.0;
    for (int i = 0; i + 1 < n; ++i) {
        const uint64_t mi = 1ull << (n - 1 - i), mj = 1ull << (n - 2 - i);
        C xx{0.0, 0.0}, yy{0.0, 0.0};
        double zz = 0.0;
        for (uint64_t k = 0; k < dim; ++k) {
            const uint64_t f = k ^ mi ^ mj;
            xx = cadd(xx, cmul(cconj(v[k]), v[f]));
        }
        for (uint64_t k = 0; k < dim; ++k) {
            const bool bi = (k & mi) != 0, bj = (k & mj) != 0;
            const uint64_t f = k ^ mi ^ mj;
            const C pi = bi ? C{0.0, -1.0} : C{0.0, 1.0};
            const C pj = bj ? C{0.0, -1.0} : C{0.0, 1.0};
            yy = cadd(yy, cmul(cmul(cconj(v[k]), cmul(pi, pj)), v[f]));
        }
        for (uint64_t k = 0; k < dim; ++k) {
            const bool bi = (k & mi) != 0, bj = (k & mj) != 0;
            const double sign = ((int)bi + (int)bj) % 2 == 0 ? 1.0 : -1.0;
            zz += (v[k].re * v[k].re + v[k].im * v[k].im) * sign;
        }
        energy += jx * xx.re;
        energy += jy * yy.re;
        energy += jz * zz;
    }
    if (h != 0.0) {
        for (int i = 0; i < n; ++i) {
            const uint64_t mi = 1ull << (n - 1 - i);
            double z = 0.0;
            for (uint64_t k = 0; k < dim; ++k) {
                const double sign = (k & mi) ? -1.0 : 1.0;
                z += (v[k].re * v[k].re + v[k].im * v[k].im) * sign;
            }
            energy += h * z;
        }
    }
    return energy;
}

double or_ansatz_energy(int n, const lq_gate *ops, int nops, const double *theta,
                        const lq_pauli_term *terms, int nterms, int yconv) {
    std::vector<C> buf(1ull << n);
    return ansatz_energy(n, ops, nops, theta, terms, nterms, yconv, buf);
}

/* ParameterShift::compute_gradient (src/optimization/gradient.rs:44-78). */
void or_parameter_shift(int n, const lq_gate *ops, int nops, const double *theta, int nparams,
                        const lq_pauli_term *terms, int nterms, int yconv, double shift,
                        double *grad) {
    std::vector<C> buf(1ull << n);
    std::vector<double> p(theta, theta + nparams);
    for (int i = 0; i < nparams; ++i) {
        p[i] = theta[i] + shift;
        const double ep = ansatz_energy(n, ops, nops, p.data(), terms, nterms, yconv, buf);
        p[i] = theta[i] - shift;
        const double em = ansatz_energy(n, ops, nops, p.data(), terms, nterms, yconv, buf);
        p[i] = theta[i];
        grad[i] = (ep - em) / 2.0;
    }
}

/* FiniteDifference::compute_gradient (src/optimization/gradient.rs:96-125). */
void or_finite_difference(int n, const lq_gate *ops, int nops, const double *theta, int nparams,
                          const lq_pauli_term *terms, int nterms, int yconv, double eps,
                          double *grad) {
    std::vector<C> buf(1ull << n);
    std::vector<double> p(theta, theta + nparams);
    const double fx = ansatz_energy(n, ops, nops, theta, terms, nterms, yconv, buf);
    for (int i = 0; i < nparams; ++i) {
        p[i] = theta[i] + eps;
        const double fp = ansatz_energy(n, ops, nops, p.data(), terms, nterms, yconv, buf);
        p[i] = theta[i];
        grad[i] = (fp - fx) / eps;
    }
}

/* Adam::minimize (src/optimization/optimizer.rs:139-223) driving the VQE
 * objective and parameter-shift gradient (src/optimization/vqe.rs:55-100).
 * Returns the number of iterations recorded in convergence_history; params is
 * updated in place and *final_value receives f(optimal params). */
int or_vqe_adam(int n, const lq_gate *ops, int nops, double *params, int nparams,
                const lq_pauli_term *terms, int nterms, int yconv, double lr, int max_iter,
                double tol, double *history, double *final_value) {
    const double beta1 = 0.9, beta2 = 0.999, eps = 1e-8;
    std::vector<C> buf(1ull << n);
    std::vector<double> m(nparams, 0.0), v(nparams, 0.0), g(nparams);
    int hist = 0;
    bool have_prev = false;
    double prev = 0.0;
    for (int it = 1; it <= max_iter; ++it) {
        const double value = ansatz_energy(n, ops, nops, params, terms, nterms, yconv, buf);
        history[hist++] = value;
        if (have_prev && std::fabs(prev - value) < tol) break;
        prev = value;
        have_prev = true;
        or_parameter_shift(n, ops, nops, params, nparams, terms, nterms, yconv, M_PI / 2.0, g.data());
        double gn = 0.0;
        for (int i = 0; i < nparams; ++i) gn += g[i] * g[i];
        if (std::sqrt(gn) < tol) break;
        for (int i = 0; i < nparams; ++i) {
            m[i] = beta1 * m[i] + (1.0 - beta1) * g[i];
            v[i] = beta2 * v[i] + (1.0 - beta2) * g[i] * g[i];
        }
        const double mc = 1.0 / (1.0 - std::pow(beta1, it));
        const double vc = 1.0 / (1.0 - std::pow(beta2, it));
        double step_sq = 0.0;
        for (int i = 0; i < nparams; ++i) {
            const double mh = m[i] * mc, vh = v[i] * vc;
            const double step = lr * mh / (std::sqrt(vh) + eps);
            params[i] -= step;
            step_sq += step * step;
        }
        if (std::sqrt(step_sq) < tol) break;
    }
    *final_value = ansatz_energy(n, ops, nops, params, terms, nterms, yconv, buf);
    return hist;
}

/* MatrixGate::apply on a full 2^n x 2^n matrix (src/gates/mod.rs:76-93), for
 * tiny n: new = M . v (ndarray dot, row-major accumulation), then normalize. */
void or_apply_dense(double *psi, int n, const double *mat) {
    C *v = reinterpret_cast<C *>(psi);
    const uint64_t d = 1ull << n;
    std::vector<C> out(d);
    for (uint64_t r = 0; r < d; ++r) {
        C acc{0.0, 0.0};
        for (uint64_t c = 0; c < d; ++c) {
            const C mrc{mat[(r * d + c) * 2], mat[(r * d + c) * 2 + 1]};
            acc = cadd(acc, cmul(mrc, v[c]));
        }
        out[r] = acc;
    }
    for (uint64_t r = 0; r < d; ++r) v[r] = out[r];
    normalize(v, n);
}

}  // extern "C"
