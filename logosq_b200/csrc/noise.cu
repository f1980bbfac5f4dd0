// Noise models of the reference (NoiseModel::apply, src/noise/mod.rs) on the
// device, with the reference's semantics:
//   * noise addresses index bit `qubit` (1 << qubit), unlike the gates, which
//     address bit n-1-qubit (src/noise/mod.rs:337-380);
//   * the Y error is the reference's YGate (-Y): new[bit 0] = i old[bit 1],
//     new[bit 1] = -i old[bit 0] (src/noise/mod.rs:350-368);
//   * amplitude damping sums K0 psi + K1 psi over every target qubit into one
//     fresh vector and then normalises (src/noise/mod.rs:108-146);
//   * phase damping rewrites the vector per target qubit, so only the last
//     target's damping survives, then normalises (src/noise/mod.rs:173-210).
// The Pauli errors and phase damping reuse the per-gate kernels (a
// permutation, the -Y op, a one-bit diagonal); amplitude damping on several
// qubits accumulates per-qubit 2x2 maps of the unchanged input into a scratch
// vector (one HBM sweep per target qubit).
#include <cmath>
#include <vector>

#include "gate_ops.h"

namespace lq {

// out[i] += (M psi)[i] for a real 2x2 M on index bit b.
__global__ void k_accum_m1_real(const double2 *__restrict__ psi, double2 *__restrict__ out,
                                int b, uint64_t N, double m00, double m01, double m10,
                                double m11) {
    const uint64_t bit = 1ull << b;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 a = psi[i], c = psi[i ^ bit];
        // (a0, a1) = amplitudes with the bit clear / set
        const bool set = (i & bit) != 0;
        const double2 a0 = set ? c : a, a1 = set ? a : c;
        const double r0 = set ? m10 : m00, r1 = set ? m11 : m01;
        double2 o = out[i];
        o.x += r0 * a0.x + r1 * a1.x;
        o.y += r0 * a0.y + r1 * a1.y;
        out[i] = o;
    }
}

static int noise_targets(const lq_state *s, const int *qubits, int nqubits, std::vector<int> &out) {
    out.clear();
    if (!qubits) {  // None: every qubit (src/noise/mod.rs:66-69)
        for (int q = 0; q < s->n; ++q) out.push_back(q);
        return LQ_OK;
    }
    if (nqubits < 1) return set_error(LQ_ERR_INVALID_ARG, "empty target qubit list");
    for (int k = 0; k < nqubits; ++k) {
        LQ_TRY(check_qubit(s, qubits[k]));
        out.push_back(qubits[k]);
    }
    return LQ_OK;
}

static int noise_state(const lq_state *s) {
    LQ_TRY(check_state(s));
    if (s->dtype != LQ_C128)
        return set_error(LQ_ERR_UNSUPPORTED, "noise models run on complex128 states");
    return LQ_OK;
}

}  // namespace lq

using namespace lq;

extern "C" {

int lq_noise_pauli(lq_state *s, int qubit, int pauli) {
    LQ_TRY(noise_state(s));
    LQ_TRY(check_qubit(s, qubit));
    if (pauli < 1 || pauli > 3) return set_error(LQ_ERR_INVALID_ARG, "pauli must be 1 (X), 2 (Y) or 3 (Z)");
    lq_gate g;
    memset(&g, 0, sizeof(g));
    g.kind = pauli == 1 ? LQ_GATE_X : pauli == 2 ? LQ_GATE_Y : LQ_GATE_Z;
    g.q[0] = s->n - 1 - qubit;  // gate qubit whose basis bit is `qubit`
    g.q[1] = g.q[2] = -1;
    g.param[0] = g.param[1] = g.param[2] = -1;
    GateOp op;
    LQ_TRY(make_gate_op(&g, nullptr, s->n, &op));
    return launch_gate_op(s, op);
}

int lq_noise_amplitude_damping(lq_state *s, double gamma, const int *qubits, int nqubits) {
    LQ_TRY(noise_state(s));
    if (!(gamma >= 0.0 && gamma <= 1.0))
        return set_error(LQ_ERR_INVALID_ARG, "error probability must lie in [0, 1]");
    std::vector<int> tq;
    LQ_TRY(noise_targets(s, qubits, nqubits, tq));
    const double sg = std::sqrt(gamma), s1 = std::sqrt(1.0 - gamma);
    if (tq.size() == 1) {  // K0 + K1 = [[1, sqrt(g)], [0, sqrt(1-g)]] on one bit, in place
        GateOp op;
        op.type = OP_M1;
        op.t = tq[0];
        const double m[8] = {1.0, 0.0, sg, 0.0, 0.0, 0.0, s1, 0.0};
        for (int k = 0; k < 8; ++k) op.m[k] = m[k];
        LQ_TRY(launch_gate_op(s, op));
        return normalize_impl(s);
    }
    const uint64_t N = 1ull << s->n;
    double2 *acc = nullptr;
    cudaError_t e = cudaMalloc(&acc, N * sizeof(double2));
    if (e != cudaSuccess)
        return set_error(e == cudaErrorMemoryAllocation ? LQ_ERR_OOM : LQ_ERR_CUDA, "%s",
                         cudaGetErrorString(e));
    e = cudaMemsetAsync(acc, 0, N * sizeof(double2), s->stream);
    const int grid = (int)std::min<uint64_t>(1184, (N + 255) / 256);
    for (size_t k = 0; k < tq.size() && e == cudaSuccess; ++k) {
        k_accum_m1_real<<<grid, 256, 0, s->stream>>>((const double2 *)s->d, acc, tq[k], N, 1.0, sg,
                                                      0.0, s1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->d, acc, N * sizeof(double2), cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(acc);
    if (e != cudaSuccess) return set_error(LQ_ERR_CUDA, "%s", cudaGetErrorString(e));
    return normalize_impl(s);
}

int lq_noise_phase_damping(lq_state *s, double lambda, const int *qubits, int nqubits) {
    LQ_TRY(noise_state(s));
    if (!(lambda >= 0.0 && lambda <= 1.0))
        return set_error(LQ_ERR_INVALID_ARG, "error probability must lie in [0, 1]");
    std::vector<int> tq;
    LQ_TRY(noise_targets(s, qubits, nqubits, tq));
    GateOp op;
    op.type = OP_DIAG;
    op.npat = 1;
    op.pat[0] = tq.back();  // each target rewrites the vector: the last one survives
    op.m[0] = 1.0;
    op.m[1] = 0.0;
    op.m[2] = std::sqrt(1.0 - lambda);
    op.m[3] = 0.0;
    LQ_TRY(launch_gate_op(s, op));
    return normalize_impl(s);
}

}  // extern "C"
