// Host-side planner of fused passes, shared by fused.cu and batch.cu.
#pragma once

#include <vector>

#include "fused_core.cuh"
#include "gate_ops.h"

namespace lq {

struct PlannedRound {
    int rpos[4];
    std::vector<int> ops;  // indices into the pass gate list
};

struct PlannedPass {
    int h = 4;
    std::vector<int> gates;  // indices into the circuit op list (in order)
    std::vector<PlannedRound> rounds;
};

struct PlanStep {  // either a fused pass or a standalone gate
    bool fused = false;
    int gate = -1;
    PlannedPass pass;
};

// Window [0,4) U [h, h+T-4); returns passes and standalone gates in order.
std::vector<PlanStep> plan_circuit(const std::vector<GateOp> &gops, int n, int T);
// Round record (element offsets, register bit masks, thread lanes).
void fill_round(FusedRound &fr, const int rpos[4], int T, int h);
// Append the register op of gate g in a round with register positions rpos.
void encode_op(const GateOp &g, int h, int m, const int rpos[4], std::vector<FusedOp> &fops,
               std::vector<double> &coef);
// Local <-> global bit positions of the window.
inline int local_pos(int b, int h) { return b < 4 ? b : 4 + (b - h); }
inline int global_pos(int l, int h) { return l < 4 ? l : h + (l - 4); }
inline uint64_t window_mask(int h, int m) { return 0xFull | (((1ull << m) - 1) << h); }

// Fusion width used by lq_apply_circuit (tile bits T, 5..12).
int fusion_width();

}  // namespace lq
