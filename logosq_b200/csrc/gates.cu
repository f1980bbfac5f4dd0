// Per-gate sweeps: the drop-in for Gate::apply (src/gates/mod.rs:26-35).
//
// Every reference gate struct (src/gates/single_qubit.rs, two_qubit.rs,
// three_qubit.rs, parameterized.rs) is first reduced on the host to one of
// five canonical ops (gate_ops.h) whose coefficients are computed in FP64 with
// the reference's own formulas; one kernel per op type then sweeps the state.
//
// Memory access: amplitudes are 16-byte double2 (complex128) or 8-byte float2
// (complex64).  Single-qubit gates on a low bit (b < 5) load one amplitude per
// lane, fully coalesced, and exchange partners with warp shuffles; on higher
// bits each thread loads the two halves of a pair with 128-bit loads that are
// coalesced across the warp.  Controlled, diagonal and permutation gates only
// enumerate the amplitudes they change (bit insertion), so e.g. CPhase reads
// and writes a quarter of the state.
#include <algorithm>
#include <cmath>

#include "gate_ops.h"

namespace lq {

// ---------------------------------------------------------------------------
// Host: descriptor -> canonical op, with the reference's coefficient formulas.
// ---------------------------------------------------------------------------
double gate_angle(const lq_gate *g, int k, const double *theta) {
    if (g->param[k] >= 0) return theta[g->param[k]] * g->scale[k] + g->angle[k];
    return g->angle[k];
}

int gate_num_qubits(int kind) {
    switch (kind) {
    case LQ_GATE_CNOT: case LQ_GATE_SWAP: case LQ_GATE_CZ: case LQ_GATE_CPHASE:
    case LQ_GATE_CRX: case LQ_GATE_CRY: case LQ_GATE_CRZ: case LQ_GATE_CPHASE_PARAM:
    case LQ_GATE_RXX: case LQ_GATE_RYY: case LQ_GATE_RZZ: case LQ_GATE_MATRIX2:
        return 2;
    case LQ_GATE_TOFFOLI:
        return 3;
    default:
        return kind >= 0 && kind < LQ_GATE__COUNT ? 1 : 0;
    }
}

static int num_angles(int kind) {
    switch (kind) {
    case LQ_GATE_U3: return 3;
    case LQ_GATE_RX: case LQ_GATE_RY: case LQ_GATE_RZ: case LQ_GATE_PHASE:
    case LQ_GATE_CPHASE: case LQ_GATE_CRX: case LQ_GATE_CRY: case LQ_GATE_CRZ:
    case LQ_GATE_CPHASE_PARAM: case LQ_GATE_RXX: case LQ_GATE_RYY: case LQ_GATE_RZZ:
        return 1;
    default: return 0;
    }
}

int validate_gate(const lq_gate *g, int n, int ntheta) {
    if (!g) return set_error(LQ_ERR_INVALID_ARG, "null gate descriptor");
    const int k = gate_num_qubits(g->kind);
    if (k == 0) return set_error(LQ_ERR_INVALID_ARG, "unknown gate kind %d", g->kind);
    for (int i = 0; i < k; ++i) {
        if (g->q[i] < 0 || g->q[i] >= n)
            return set_error(LQ_ERR_QUBIT_INDEX, "Invalid qubit index: %d (must be < %d)",
                             g->q[i], n);
        for (int j = 0; j < i; ++j)
            if (g->q[i] == g->q[j])
                return set_error(LQ_ERR_INVALID_ARG, "gate kind %d uses qubit %d twice", g->kind,
                                 g->q[i]);
    }
    const int na = num_angles(g->kind);
    for (int a = 0; a < na; ++a) {
        if (g->param[a] >= ntheta)
            return set_error(LQ_ERR_PARAM_COUNT,
                             "Parameter count mismatch: expected > %d, got %d", g->param[a],
                             ntheta);
    }
    return LQ_OK;
}

int gate_class(int kind) {
    switch (kind) {
    case LQ_GATE_Z: case LQ_GATE_S: case LQ_GATE_T: case LQ_GATE_RZ: case LQ_GATE_PHASE:
    case LQ_GATE_CZ: case LQ_GATE_CPHASE: case LQ_GATE_CRZ: case LQ_GATE_CPHASE_PARAM:
    case LQ_GATE_RZZ:
        return kClassDiagonal;
    case LQ_GATE_X: case LQ_GATE_CNOT: case LQ_GATE_TOFFOLI: case LQ_GATE_SWAP:
        return kClassPermutation;
    default:
        return kClassGeneral;
    }
}

static inline void set_c(double *m, int idx, double re, double im) {
    m[2 * idx] = re;
    m[2 * idx + 1] = im;
}
static inline void polar(double r, double t, double &re, double &im) {
    re = r * std::cos(t);
    im = r * std::sin(t);
}

int make_gate_op(const lq_gate *g, const double *theta, int n, GateOp *op) {
    *op = GateOp();
    auto bit = [&](int q) { return n - 1 - q; };
    op->renorm = (g->flags & LQ_FLAG_RENORM) != 0;
    double *m = op->m;
    switch (g->kind) {
    case LQ_GATE_H: {  // single_qubit.rs:97-111: s*(a0+a1), s*(a0-a1), s = 1/sqrt(2)
        const double s = 1.0 / M_SQRT2;
        op->type = OP_M1; op->t = bit(g->q[0]);
        set_c(m, 0, s, 0); set_c(m, 1, s, 0); set_c(m, 2, s, 0); set_c(m, 3, -s, 0);
        break;
    }
    case LQ_GATE_X:
        op->type = OP_PERM1; op->t = bit(g->q[0]);
        break;
    case LQ_GATE_Y:  // single_qubit.rs:53-55: v0 = i*v1 ; v1 = -i*v0
        op->type = OP_M1; op->t = bit(g->q[0]);
        set_c(m, 0, 0, 0); set_c(m, 1, 0, 1); set_c(m, 2, 0, -1); set_c(m, 3, 0, 0);
        break;
    case LQ_GATE_Z:
        op->type = OP_DIAG; op->nfix = 1; op->fix[0] = bit(g->q[0]);
        set_c(m, 0, -1, 0);
        break;
    case LQ_GATE_S:
        op->type = OP_DIAG; op->nfix = 1; op->fix[0] = bit(g->q[0]);
        set_c(m, 0, 0, 1);
        break;
    case LQ_GATE_T: {  // single_qubit.rs:152: from_polar(1, PI/4)
        double re, im; polar(1.0, M_PI / 4.0, re, im);
        op->type = OP_DIAG; op->nfix = 1; op->fix[0] = bit(g->q[0]);
        set_c(m, 0, re, im);
        break;
    }
    case LQ_GATE_RX: {  // parameterized.rs:55-76
        const double th = gate_angle(g, 0, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        op->type = OP_M1; op->t = bit(g->q[0]);
        set_c(m, 0, c, 0); set_c(m, 1, 0, -s); set_c(m, 2, 0, -s); set_c(m, 3, c, 0);
        break;
    }
    case LQ_GATE_RY: {  // parameterized.rs:108-129
        const double th = gate_angle(g, 0, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        op->type = OP_M1; op->t = bit(g->q[0]);
        set_c(m, 0, c, 0); set_c(m, 1, -s, 0); set_c(m, 2, s, 0); set_c(m, 3, c, 0);
        break;
    }
    case LQ_GATE_RZ: {  // parameterized.rs:161-176
        const double th = gate_angle(g, 0, theta);
        double r0, i0, r1, i1;
        polar(1.0, -th / 2.0, r0, i0);
        polar(1.0, th / 2.0, r1, i1);
        op->type = OP_DIAG; op->npat = 1; op->pat[0] = bit(g->q[0]);
        set_c(m, 0, r0, i0); set_c(m, 1, r1, i1);
        break;
    }
    case LQ_GATE_PHASE: {  // parameterized.rs:204-216
        double re, im; polar(1.0, gate_angle(g, 0, theta), re, im);
        op->type = OP_DIAG; op->nfix = 1; op->fix[0] = bit(g->q[0]);
        set_c(m, 0, re, im);
        break;
    }
    case LQ_GATE_U3: {  // parameterized.rs:254-262
        const double th = gate_angle(g, 0, theta), phi = gate_angle(g, 1, theta),
                     lam = gate_angle(g, 2, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        double r, i;
        op->type = OP_M1; op->t = bit(g->q[0]);
        set_c(m, 0, c, 0);
        polar(s, lam, r, i); set_c(m, 1, -r, -i);
        polar(s, phi, r, i); set_c(m, 2, r, i);
        polar(c, phi + lam, r, i); set_c(m, 3, r, i);
        break;
    }
    case LQ_GATE_CNOT:
        op->type = OP_PERM1; op->t = bit(g->q[1]); op->nctrl = 1; op->ctrl[0] = bit(g->q[0]);
        break;
    case LQ_GATE_TOFFOLI:
        op->type = OP_PERM1; op->t = bit(g->q[2]); op->nctrl = 2;
        op->ctrl[0] = bit(g->q[0]); op->ctrl[1] = bit(g->q[1]);
        break;
    case LQ_GATE_SWAP:
        op->type = OP_SWAP; op->b0 = bit(g->q[0]); op->b1 = bit(g->q[1]);
        break;
    case LQ_GATE_CZ:
        op->type = OP_DIAG; op->nfix = 2; op->fix[0] = bit(g->q[0]); op->fix[1] = bit(g->q[1]);
        set_c(m, 0, -1, 0);
        break;
    case LQ_GATE_CPHASE:
    case LQ_GATE_CPHASE_PARAM: {  // two_qubit.rs:112 / parameterized.rs:489
        double re, im; polar(1.0, gate_angle(g, 0, theta), re, im);
        op->type = OP_DIAG; op->nfix = 2; op->fix[0] = bit(g->q[0]); op->fix[1] = bit(g->q[1]);
        set_c(m, 0, re, im);
        break;
    }
    case LQ_GATE_CRX:
    case LQ_GATE_CRY: {  // parameterized.rs:318-340 / 375-397
        const double th = gate_angle(g, 0, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        op->type = OP_M1; op->t = bit(g->q[1]); op->nctrl = 1; op->ctrl[0] = bit(g->q[0]);
        set_c(m, 0, c, 0); set_c(m, 3, c, 0);
        if (g->kind == LQ_GATE_CRX) { set_c(m, 1, 0, -s); set_c(m, 2, 0, -s); }
        else { set_c(m, 1, -s, 0); set_c(m, 2, s, 0); }
        break;
    }
    case LQ_GATE_CRZ: {  // parameterized.rs:437-449
        const double th = gate_angle(g, 0, theta);
        double r0, i0, r1, i1;
        polar(1.0, -th / 2.0, r0, i0);
        polar(1.0, th / 2.0, r1, i1);
        op->type = OP_DIAG; op->nfix = 1; op->fix[0] = bit(g->q[0]);
        op->npat = 1; op->pat[0] = bit(g->q[1]);
        set_c(m, 0, r0, i0); set_c(m, 1, r1, i1);
        break;
    }
    case LQ_GATE_RXX:
    case LQ_GATE_RYY: {  // parameterized.rs:535-578 / 611-653
        const double th = gate_angle(g, 0, theta);
        const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
        const bool textbook = (g->flags & LQ_FLAG_TEXTBOOK) != 0;
        const double offa = g->kind == LQ_GATE_RXX ? -s : s;  // |00>,|11> block (imag)
        op->type = OP_M2; op->b0 = bit(g->q[0]); op->b1 = bit(g->q[1]);
        // rows/cols: 0=|00>, 1=|01>, 2=|10>, 3=|11> (q0 high)
        for (int r = 0; r < 4; ++r) set_c(m, r * 4 + r, 1, 0);
        set_c(m, 0 * 4 + 0, c, 0); set_c(m, 3 * 4 + 3, c, 0);
        set_c(m, 0 * 4 + 3, 0, offa); set_c(m, 3 * 4 + 0, 0, offa);
        // The |10>,|01> block runs only when i < j, i.e. qubit1 > qubit2.
        if (textbook || g->q[0] > g->q[1]) {
            set_c(m, 1 * 4 + 1, c, 0); set_c(m, 2 * 4 + 2, c, 0);
            set_c(m, 1 * 4 + 2, 0, -s); set_c(m, 2 * 4 + 1, 0, -s);
        }
        break;
    }
    case LQ_GATE_RZZ: {  // parameterized.rs:692-706
        const double th = gate_angle(g, 0, theta);
        double rs, is, rd, id;
        polar(1.0, -th / 2.0, rs, is);
        polar(1.0, th / 2.0, rd, id);
        op->type = OP_DIAG; op->npat = 2; op->pat[0] = bit(g->q[1]); op->pat[1] = bit(g->q[0]);
        set_c(m, 0, rs, is); set_c(m, 1, rd, id); set_c(m, 2, rd, id); set_c(m, 3, rs, is);
        break;
    }
    case LQ_GATE_MATRIX1:
        op->type = OP_M1; op->t = bit(g->q[0]);
        for (int i = 0; i < 8; ++i) m[i] = g->m[i];
        break;
    case LQ_GATE_MATRIX2:
        op->type = OP_M2; op->b0 = bit(g->q[0]); op->b1 = bit(g->q[1]);
        for (int i = 0; i < 32; ++i) m[i] = g->m[i];
        break;
    default:
        return set_error(LQ_ERR_INVALID_ARG, "unknown gate kind %d", g->kind);
    }
    return LQ_OK;
}

// ---------------------------------------------------------------------------
// Device kernels, templated on the amplitude type (double2 / float2).
// ---------------------------------------------------------------------------
template <class A> struct RealOf;
template <> struct RealOf<double2> { using T = double; };
template <> struct RealOf<float2> { using T = float; };

template <class A>
struct M2x2 {
    typename RealOf<A>::T r[8];
};
template <class A>
struct M4x4 {
    typename RealOf<A>::T r[32];
};

__device__ __forceinline__ uint64_t insert_zero(uint64_t x, int pos) {
    const uint64_t lo = x & ((1ull << pos) - 1);
    return ((x >> pos) << (pos + 1)) | lo;
}

// out = m_a * a + m_b * b (complex), the reference's term order.
template <class A, class R>
__device__ __forceinline__ A cmac2(R ar, R ai, A a, R br, R bi, A b) {
    A o;
    o.x = (ar * a.x - ai * a.y) + (br * b.x - bi * b.y);
    o.y = (ar * a.y + ai * a.x) + (br * b.y + bi * b.x);
    return o;
}

constexpr int kItems = 2;
constexpr int kThreads = 256;

// Low target bit (b < 5): one amplitude per lane, partner by shuffle.
template <class A>
__global__ void __launch_bounds__(kThreads) k_1q_shfl(A *__restrict__ v, uint64_t N, int b,
                                                      M2x2<A> M) {
    using R = typename RealOf<A>::T;
    const uint64_t base = (uint64_t)blockIdx.x * kThreads * kItems + threadIdx.x;
    const int hi = (threadIdx.x >> b) & 1;
    const unsigned lanemask = 1u << b;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t i = base + (uint64_t)k * kThreads;
        if (i >= N) break;  // warp-uniform: N is a multiple of 32 here
        const A a = v[i];
        A p;
        p.x = __shfl_xor_sync(0xffffffffu, a.x, lanemask);
        p.y = __shfl_xor_sync(0xffffffffu, a.y, lanemask);
        A o;
        if (!hi) o = cmac2<A, R>(M.r[0], M.r[1], a, M.r[2], M.r[3], p);   // m00*a0 + m01*a1
        else o = cmac2<A, R>(M.r[4], M.r[5], p, M.r[6], M.r[7], a);       // m10*a0 + m11*a1
        v[i] = o;
    }
}

// General target bit: one pair per thread and item, 128-bit loads of both halves.
template <class A>
__global__ void __launch_bounds__(kThreads) k_1q_pair(A *__restrict__ v, uint64_t npairs, int b,
                                                      M2x2<A> M) {
    using R = typename RealOf<A>::T;
    const uint64_t base = (uint64_t)blockIdx.x * kThreads * kItems + threadIdx.x;
    const uint64_t stride = 1ull << b;
    A a0[kItems], a1[kItems];
    uint64_t i0[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t p = base + (uint64_t)k * kThreads;
        i0[k] = insert_zero(p, b);
        if (p < npairs) {
            a0[k] = v[i0[k]];
            a1[k] = v[i0[k] + stride];
        }
    }
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t p = base + (uint64_t)k * kThreads;
        if (p < npairs) {
            v[i0[k]] = cmac2<A, R>(M.r[0], M.r[1], a0[k], M.r[2], M.r[3], a1[k]);
            v[i0[k] + stride] = cmac2<A, R>(M.r[4], M.r[5], a0[k], M.r[6], M.r[7], a1[k]);
        }
    }
}

// Controlled 2x2 / controlled X: enumerate indices with all control bits 1 and
// the target bit 0.  ins[] are the inserted bit positions in ascending order and
// setmask the bits inserted as 1.
struct InsertSpec {
    int npos;
    int pos[3];
    uint64_t setmask;
};

__device__ __forceinline__ uint64_t expand(uint64_t x, const InsertSpec &s) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (k < s.npos) x = insert_zero(x, s.pos[k]);
    return x | s.setmask;
}

template <class A, bool PERM>
__global__ void __launch_bounds__(kThreads) k_ctrl1q(A *__restrict__ v, uint64_t count,
                                                     InsertSpec ins, uint64_t tmask, M2x2<A> M) {
    using R = typename RealOf<A>::T;
    const uint64_t base = (uint64_t)blockIdx.x * kThreads * kItems + threadIdx.x;
    A a0[kItems], a1[kItems];
    uint64_t i0[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t x = base + (uint64_t)k * kThreads;
        i0[k] = expand(x, ins);
        if (x < count) {
            a0[k] = v[i0[k]];
            a1[k] = v[i0[k] | tmask];
        }
    }
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t x = base + (uint64_t)k * kThreads;
        if (x < count) {
            if (PERM) {
                v[i0[k]] = a1[k];
                v[i0[k] | tmask] = a0[k];
            } else {
                v[i0[k]] = cmac2<A, R>(M.r[0], M.r[1], a0[k], M.r[2], M.r[3], a1[k]);
                v[i0[k] | tmask] = cmac2<A, R>(M.r[4], M.r[5], a0[k], M.r[6], M.r[7], a1[k]);
            }
        }
    }
}

// Diagonal: amplitude *= ph[pattern] on the indices with all fix bits set.
template <class A>
struct DiagSpec {
    InsertSpec ins;
    int npat;
    int pat[3];
    typename RealOf<A>::T ph[16];
};

template <class A>
__global__ void __launch_bounds__(kThreads) k_diag(A *__restrict__ v, uint64_t count,
                                                   DiagSpec<A> d) {
    using R = typename RealOf<A>::T;
    const uint64_t base = (uint64_t)blockIdx.x * kThreads * kItems + threadIdx.x;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t x = base + (uint64_t)k * kThreads;
        if (x < count) {
            const uint64_t i = expand(x, d.ins);
            int pattern = 0;
            if (d.npat > 0) pattern |= (int)((i >> d.pat[0]) & 1);
            if (d.npat > 1) pattern |= (int)((i >> d.pat[1]) & 1) << 1;
            if (d.npat > 2) pattern |= (int)((i >> d.pat[2]) & 1) << 2;
            const R pr = d.ph[2 * pattern], pi = d.ph[2 * pattern + 1];
            const A a = v[i];
            A o;
            o.x = a.x * pr - a.y * pi;  // a * phase (vector_slice[i] *= phase)
            o.y = a.x * pi + a.y * pr;
            v[i] = o;
        }
    }
}

template <class A>
__global__ void __launch_bounds__(kThreads) k_swap(A *__restrict__ v, uint64_t count,
                                                   InsertSpec ins, uint64_t m1, uint64_t m2) {
    const uint64_t base = (uint64_t)blockIdx.x * kThreads * kItems + threadIdx.x;
    A a[kItems], b[kItems];
    uint64_t i0[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t x = base + (uint64_t)k * kThreads;
        i0[k] = expand(x, ins);
        if (x < count) {
            a[k] = v[i0[k] | m1];
            b[k] = v[i0[k] | m2];
        }
    }
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t x = base + (uint64_t)k * kThreads;
        if (x < count) {
            v[i0[k] | m1] = b[k];
            v[i0[k] | m2] = a[k];
        }
    }
}

template <class A>
__global__ void __launch_bounds__(kThreads) k_2q(A *__restrict__ v, uint64_t count,
                                                 InsertSpec ins, uint64_t mq0, uint64_t mq1,
                                                 M4x4<A> M) {
    using R = typename RealOf<A>::T;
    const uint64_t x = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    if (x >= count) return;
    const uint64_t base = expand(x, ins);
    const uint64_t idx[4] = {base, base | mq1, base | mq0, base | mq0 | mq1};
    A a[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) a[r] = v[idx[r]];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        R ore = 0, oim = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const R mr = M.r[(r * 4 + c) * 2], mi = M.r[(r * 4 + c) * 2 + 1];
            ore += mr * a[c].x - mi * a[c].y;
            oim += mr * a[c].y + mi * a[c].x;
        }
        A o;
        o.x = ore;
        o.y = oim;
        v[idx[r]] = o;
    }
}

// MatrixGate::apply (src/gates/mod.rs:76-93): out = M . psi with a full
// 2^n x 2^n matrix, one warp per output row (small n only; O(4^n)).
__global__ void k_dense_rows(const double2 *__restrict__ M, const double2 *__restrict__ v,
                             double2 *__restrict__ out, uint64_t dim) {
    const uint64_t row = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= dim) return;
    double re = 0.0, im = 0.0;
    for (uint64_t c = lane; c < dim; c += 32) {
        const double2 m = M[row * dim + c], a = v[c];
        re += m.x * a.x - m.y * a.y;
        im += m.x * a.y + m.y * a.x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o);
        im += __shfl_down_sync(0xffffffffu, im, o);
    }
    if (lane == 0) out[row] = make_double2(re, im);
}

static inline unsigned blocks_for(uint64_t count, int per_block) {
    return (unsigned)((count + per_block - 1) / per_block);
}

static InsertSpec make_insert(std::vector<std::pair<int, int>> bits /* (pos, value) */) {
    std::sort(bits.begin(), bits.end());
    InsertSpec s{};
    s.npos = (int)bits.size();
    s.setmask = 0;
    for (int k = 0; k < s.npos; ++k) {
        s.pos[k] = bits[k].first;
        if (bits[k].second) s.setmask |= 1ull << bits[k].first;
    }
    return s;
}

template <class A>
static int launch_op_t(lq_state *s, const GateOp &op) {
    using R = typename RealOf<A>::T;
    A *v = (A *)s->d;
    const int n = s->n;
    const uint64_t N = 1ull << n;
    cudaStream_t st = s->stream;
    switch (op.type) {
    case OP_M1:
    case OP_PERM1: {
        M2x2<A> M;
        if (op.type == OP_PERM1) {
            const double x[8] = {0, 0, 1, 0, 1, 0, 0, 0};
            for (int i = 0; i < 8; ++i) M.r[i] = (R)x[i];
        } else {
            for (int i = 0; i < 8; ++i) M.r[i] = (R)op.m[i];
        }
        if (op.nctrl == 0) {
            if (op.type == OP_M1 && op.t < 5 && n >= 5) {
                k_1q_shfl<A><<<blocks_for(N, kThreads * kItems), kThreads, 0, st>>>(v, N, op.t, M);
            } else {
                k_1q_pair<A><<<blocks_for(N / 2, kThreads * kItems), kThreads, 0, st>>>(
                    v, N / 2, op.t, M);
            }
        } else {
            std::vector<std::pair<int, int>> b = {{op.t, 0}};
            for (int c = 0; c < op.nctrl; ++c) b.push_back({op.ctrl[c], 1});
            const InsertSpec ins = make_insert(b);
            const uint64_t count = N >> (1 + op.nctrl);
            const uint64_t tmask = 1ull << op.t;
            if (op.type == OP_PERM1)
                k_ctrl1q<A, true><<<blocks_for(count, kThreads * kItems), kThreads, 0, st>>>(
                    v, count, ins, tmask, M);
            else
                k_ctrl1q<A, false><<<blocks_for(count, kThreads * kItems), kThreads, 0, st>>>(
                    v, count, ins, tmask, M);
        }
        break;
    }
    case OP_DIAG: {
        DiagSpec<A> d{};
        std::vector<std::pair<int, int>> b;
        for (int c = 0; c < op.nfix; ++c) b.push_back({op.fix[c], 1});
        d.ins = make_insert(b);
        d.npat = op.npat;
        for (int i = 0; i < 3; ++i) d.pat[i] = op.pat[i];
        for (int i = 0; i < 16; ++i) d.ph[i] = (R)op.m[i];
        const uint64_t count = N >> op.nfix;
        k_diag<A><<<blocks_for(count, kThreads * kItems), kThreads, 0, st>>>(v, count, d);
        break;
    }
    case OP_SWAP: {
        const InsertSpec ins = make_insert({{op.b0, 0}, {op.b1, 0}});
        const uint64_t count = N >> 2;
        k_swap<A><<<blocks_for(count, kThreads * kItems), kThreads, 0, st>>>(
            v, count, ins, 1ull << op.b0, 1ull << op.b1);
        break;
    }
    case OP_M2: {
        M4x4<A> M;
        for (int i = 0; i < 32; ++i) M.r[i] = (R)op.m[i];
        const InsertSpec ins = make_insert({{op.b0, 0}, {op.b1, 0}});
        const uint64_t count = N >> 2;
        k_2q<A><<<blocks_for(count, kThreads), kThreads, 0, st>>>(v, count, ins, 1ull << op.b0,
                                                                   1ull << op.b1, M);
        break;
    }
    default:
        return set_error(LQ_ERR_INVALID_ARG, "unknown op type %d", op.type);
    }
    LQ_CUDA_TRY(cudaGetLastError());
    if (op.renorm) LQ_TRY(normalize_impl(s));
    return LQ_OK;
}

int launch_gate_op(lq_state *s, const GateOp &op) {
    prof_begin(s->stream, kProfGate);
    const int rc = s->dtype == LQ_C128 ? launch_op_t<double2>(s, op) : launch_op_t<float2>(s, op);
    prof_end(s->stream, kProfGate);
    return rc;
}

int apply_gate_c128(lq_state *s, const lq_gate *g, const double *theta, int ntheta,
                    int *launches) {
    LQ_TRY(validate_gate(g, s->n, ntheta));
    GateOp op;
    LQ_TRY(make_gate_op(g, theta, s->n, &op));
    LQ_TRY(launch_gate_op(s, op));
    if (launches) *launches += op.renorm ? 3 : 1;
    return LQ_OK;
}

}  // namespace lq

using namespace lq;

extern "C" {

int lq_apply_gate(lq_state *s, const lq_gate *g, const double *theta, int ntheta) {
    LQ_TRY(check_state(s));
    if (ntheta > 0 && !theta) return set_error(LQ_ERR_INVALID_ARG, "null theta");
    int l = 0;
    return apply_gate_c128(s, g, theta, ntheta, &l);
}

int lq_apply_matrix1(lq_state *s, int qubit, const double m[8]) {
    LQ_TRY(check_state(s));
    LQ_TRY(check_qubit(s, qubit));
    if (!m) return set_error(LQ_ERR_INVALID_ARG, "null matrix");
    GateOp op;
    op.type = OP_M1;
    op.t = s->n - 1 - qubit;
    for (int i = 0; i < 8; ++i) op.m[i] = m[i];
    return launch_gate_op(s, op);
}

int lq_apply_controlled1(lq_state *s, int control, int target, const double m[8]) {
    LQ_TRY(check_state(s));
    LQ_TRY(check_qubit(s, control));
    LQ_TRY(check_qubit(s, target));
    if (control == target) return set_error(LQ_ERR_INVALID_ARG, "control == target");
    if (!m) return set_error(LQ_ERR_INVALID_ARG, "null matrix");
    GateOp op;
    op.type = OP_M1;
    op.t = s->n - 1 - target;
    op.nctrl = 1;
    op.ctrl[0] = s->n - 1 - control;
    for (int i = 0; i < 8; ++i) op.m[i] = m[i];
    return launch_gate_op(s, op);
}

int lq_apply_diagonal(lq_state *s, int k, const int *qubits, const double *phases) {
    LQ_TRY(check_state(s));
    if (k < 1 || k > 3 || !qubits || !phases)
        return set_error(LQ_ERR_INVALID_ARG, "diagonal gate needs 1..3 qubits and phases");
    for (int i = 0; i < k; ++i) {
        LQ_TRY(check_qubit(s, qubits[i]));
        for (int j = 0; j < i; ++j)
            if (qubits[i] == qubits[j]) return set_error(LQ_ERR_INVALID_ARG, "repeated qubit");
    }
    GateOp op;
    op.type = OP_DIAG;
    op.npat = k;
    // pattern lsb = last qubit (qubits[0] is the most significant)
    for (int i = 0; i < k; ++i) op.pat[i] = s->n - 1 - qubits[k - 1 - i];
    for (int i = 0; i < 2 * (1 << k); ++i) op.m[i] = phases[i];
    return launch_gate_op(s, op);
}

int lq_apply_dense(lq_state *s, const double *m, uint64_t dim) {
    LQ_TRY(check_state(s));
    if (!m) return set_error(LQ_ERR_INVALID_ARG, "null matrix");
    if (s->dtype != LQ_C128) return set_error(LQ_ERR_UNSUPPORTED, "dense gates need complex128");
    if (dim != (1ull << s->n))
        return set_error(LQ_ERR_DIMENSION_MISMATCH,
                         "Matrix columns (%llu) must match state dimension (%llu)",
                         (unsigned long long)dim, (unsigned long long)(1ull << s->n));
    if (s->n > 13)
        return set_error(LQ_ERR_UNSUPPORTED, "dense 2^n x 2^n gates are limited to n <= 13");
    double2 *dm = nullptr, *tmp = nullptr;
    LQ_CUDA_TRY(cudaMallocAsync(&dm, dim * dim * 16, s->stream));
    LQ_CUDA_TRY(cudaMallocAsync(&tmp, dim * 16, s->stream));
    LQ_CUDA_TRY(cudaMemcpyAsync(dm, m, dim * dim * 16, cudaMemcpyHostToDevice, s->stream));
    k_dense_rows<<<(unsigned)((dim * 32 + 255) / 256), 256, 0, s->stream>>>(
        dm, (const double2 *)s->d, tmp, dim);
    LQ_CUDA_TRY(cudaGetLastError());
    LQ_CUDA_TRY(cudaMemcpyAsync(s->d, tmp, dim * 16, cudaMemcpyDeviceToDevice, s->stream));
    LQ_CUDA_TRY(cudaFreeAsync(dm, s->stream));
    LQ_CUDA_TRY(cudaFreeAsync(tmp, s->stream));
    LQ_TRY(normalize_impl(s));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return LQ_OK;
}

int lq_apply_swap(lq_state *s, int qubit1, int qubit2) {
    LQ_TRY(check_state(s));
    LQ_TRY(check_qubit(s, qubit1));
    LQ_TRY(check_qubit(s, qubit2));
    if (qubit1 == qubit2) return set_error(LQ_ERR_INVALID_ARG, "qubit1 == qubit2");
    GateOp op;
    op.type = OP_SWAP;
    op.b0 = s->n - 1 - qubit1;
    op.b1 = s->n - 1 - qubit2;
    return launch_gate_op(s, op);
}

int lq_apply_matrix2(lq_state *s, int qubit1, int qubit2, const double m[32]) {
    LQ_TRY(check_state(s));
    LQ_TRY(check_qubit(s, qubit1));
    LQ_TRY(check_qubit(s, qubit2));
    if (qubit1 == qubit2) return set_error(LQ_ERR_INVALID_ARG, "qubit1 == qubit2");
    if (!m) return set_error(LQ_ERR_INVALID_ARG, "null matrix");
    GateOp op;
    op.type = OP_M2;
    op.b0 = s->n - 1 - qubit1;
    op.b1 = s->n - 1 - qubit2;
    for (int i = 0; i < 32; ++i) op.m[i] = m[i];
    return launch_gate_op(s, op);
}

}  // extern "C"
