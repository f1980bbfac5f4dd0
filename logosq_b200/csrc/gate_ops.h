// Canonical form of one gate, shared by the per-gate kernels and the fusion
// planner.  Bit positions are basis-index bits (bit = n-1-qubit).
#pragma once

#include "lq_internal.h"

namespace lq {

enum OpType {
    OP_M1 = 0,    // 2x2 matrix on bit t (with optional controls: all ctrl bits = 1)
    OP_PERM1 = 1, // X on bit t with optional controls (CNOT, Toffoli, X): pure swap
    OP_DIAG = 2,  // amplitude *= ph[pattern] on indices whose fix bits are all 1;
                  // pattern = bits pat[0] (lsb), pat[1], pat[2] of the index
    OP_SWAP = 3,  // exchange bits b0 and b1
    OP_M2 = 4     // 4x4 matrix, row/col index = (bit b0 value)<<1 | (bit b1 value)
};

struct GateOp {
    int type = OP_M1;
    int t = -1;                  // target bit (M1 / PERM1)
    int nctrl = 0, ctrl[2] = {-1, -1};
    int npat = 0, pat[3] = {-1, -1, -1};
    int nfix = 0, fix[2] = {-1, -1};
    int b0 = -1, b1 = -1;        // SWAP / M2
    bool renorm = false;
    // Fused-path planning hints (other consumers read the op as its type says):
    // real4: an OP_M2 whose matrix is real (imaginary parts zero);
    // table: an OP_DIAG on pattern bits only, kept in the register set of the
    // round that applies it so it joins that round's diagonal table.
    bool real4 = false;
    bool table = false;
    // srot: an OP_M1 that is a scaled real rotation, [[1, -x], [x, 1]] (form 0)
    // or [[x, -1], [1, x]] (form 1) with x = m[0]; m[] holds the full real 2x2.
    bool srot = false;
    int sform = 0;
    // pairrot: an OP_M2 (real4) that is P (R'_b0 (x) R'_b1), R' scaled rotations
    // with parameters px and forms pf as above, P = pperm: 0 none, 1 CNOT
    // b0 -> b1, 2 CNOT b1 -> b0, 3 SWAP.  m[] holds the full real 4x4.
    bool pairrot = false;
    double px[2] = {0.0, 0.0};
    int pf[2] = {0, 0};
    int pperm = 0;
    double m[32] = {0};          // M1: 8 doubles; M2: 32; DIAG: ph[0..3] as 8 doubles
};

// Build the canonical op of descriptor g on an n-qubit state.
int make_gate_op(const lq_gate *g, const double *theta, int n, GateOp *op);

// Mask of all index bits the op touches (for dependency tracking).
inline uint64_t op_bits(const GateOp &o) {
    uint64_t m = 0;
    auto add = [&](int b) { if (b >= 0) m |= 1ull << b; };
    add(o.t);
    for (int i = 0; i < o.nctrl; ++i) add(o.ctrl[i]);
    for (int i = 0; i < o.npat; ++i) add(o.pat[i]);
    for (int i = 0; i < o.nfix; ++i) add(o.fix[i]);
    add(o.b0);
    add(o.b1);
    return m;
}

// Launch the per-gate kernel of op on state s (complex128 or complex64).
int launch_gate_op(lq_state *s, const GateOp &op);

}  // namespace lq
