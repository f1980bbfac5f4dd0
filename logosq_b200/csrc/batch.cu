// Batched parameter-shift engine: the 2P+1 circuits of many VQE instances
// (ParameterShift::compute_gradient, src/optimization/gradient.rs:44-78, run
// for every instance of a batch) in ONE persistent kernel launch, captured in
// a CUDA graph together with its coefficient upload and result download.
//
// Work list: one item per (instance, circuit), circuit 0 unshifted and
// circuits 2j+1 / 2j+2 with parameter j shifted by +s / -s, ordered by cost
// (largest qubit count first) and handed out through an atomic counter to
// persistent CTAs (2 per SM).  Per item a CTA simulates the circuit from
// |0...0> and reduces its FP64 energy:
//   n <= 12: the whole state lives in the CTA's shared memory (one tile);
//   n  > 12: the state lives in a per-CTA scratch slot in HBM and is swept in
//            2^T-amplitude tiles (T chosen by the autotuner) by the same fused
//            passes and register rounds as lq_apply_circuit (fused_core.cuh).
// Gate coefficients are computed on the host in FP64 with the reference
// formulas (identical to the plain path); a shifted circuit only swaps in the
// (+s / -s) coefficients of the ops bound to its parameter.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>

#include "fused_plan.h"

namespace lq {

struct BInst {
    int32_t n, T, nparams;
    int32_t pass_begin, npass;
    int32_t ewin_begin, newin;
    int32_t coef_base;  // offset of the instance's coefficient block
};

struct BPass {
    int32_t h;
    int32_t round_begin, nrounds;
    int32_t pad;
};

struct BEWin {  // energy window: groups whose X bits lie inside [0,4) U [h, h+T-4)
    int32_t h;
    int32_t group_begin, ngroups;
    int32_t pad;
};

struct BGroup {
    uint64_t xmask;
    int32_t term_begin, nterms;
};

struct BTerm {
    uint64_t z;
    double ca, cb;
};

struct BItem {
    int32_t inst;
    int32_t param;  // -1: unshifted
    int32_t sign;   // +1 / -1
    int32_t pad;
};

struct BProgram {  // device program for one fusion width
    int T = 0;
    FusedRound *rounds = nullptr;
    FusedOp *ops = nullptr;
    BPass *passes = nullptr;
    BInst *insts = nullptr;
    std::vector<BInst> h_insts;
    size_t ncoef = 0;
    // per instance: host copies needed to refresh coefficients
    std::vector<std::vector<int>> op_gate;  // fop index (instance-local) -> gate index
    std::vector<std::vector<PlanStep>> steps;
    std::vector<int> op_begin;  // first fop of each instance
    std::vector<int> nops;
};

}  // namespace lq

struct lq_batch {
    int ninst = 0;
    std::vector<int> n, nparams, param_off;
    std::vector<std::vector<lq_gate>> ops;
    std::vector<std::vector<lq_pauli_term>> terms;
    int total_params = 0;
    int maxn = 0;
    // shared device data
    lq::BEWin *ewins = nullptr;
    lq::BGroup *groups = nullptr;
    lq::BTerm *bterms = nullptr;
    lq::BItem *items = nullptr;
    int nitems = 0;
    double *coef_d = nullptr;
    double *coef_h = nullptr;  // pinned
    size_t coef_cap = 0;
    double *energy_d = nullptr;
    double *energy_h = nullptr;  // pinned
    unsigned *counter = nullptr;
    double2 *scratch = nullptr;
    size_t slot_amps = 0;
    unsigned *flag = nullptr;
    int grid = 0;
    cudaStream_t stream = nullptr;
    std::vector<lq::BProgram> progs;  // one per candidate fusion width
    int chosen = -1;                  // index into progs
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double shift_captured = 0.0;
    std::vector<double> last_tune_ms;
};

namespace lq {

constexpr int kBatchThreads = 256;
constexpr int kSmemStateMax = 12;  // states up to 2^12 amplitudes live in shared memory

__device__ __forceinline__ uint64_t insert_zero_u(uint64_t x, int pos) {
    const uint64_t lo = x & ((1ull << pos) - 1);
    return ((x >> pos) << (pos + 1)) | lo;
}

// Energy contribution of the groups of one window over the tile in smem.
__device__ double tile_energy(uint32_t tile_a, int T, int h, uint64_t tile_base,
                              const BGroup *__restrict__ groups, int g0, int ng,
                              const BTerm *__restrict__ terms, int tid, int nthr) {
    double acc = 0.0;
    const int m = T - 4;
    for (int g = g0; g < g0 + ng; ++g) {
        const BGroup gr = groups[g];
        // local X mask
        uint32_t lx = 0;
        for (int b = 0; b < 64; ++b) {
            if (!((gr.xmask >> b) & 1)) continue;
            lx |= 1u << (b < 4 ? b : 4 + (b - h));
        }
        const BTerm *tp = terms + gr.term_begin;
        if (lx == 0) {
            for (int l = tid; l < (1 << T); l += nthr) {
                const uint64_t gi = tile_base | (uint64_t)(l & 15) | ((uint64_t)(l >> 4) << h);
                double2 a;
                asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
                             : "=d"(a.x), "=d"(a.y)
                             : "r"(tile_a + ((uint32_t)swz(l) << 4)));
                double alpha = 0.0;
                for (int t = 0; t < gr.nterms; ++t)
                    alpha += ((__popcll(gi & tp[t].z) & 1) ? -tp[t].ca : tp[t].ca);
                acc += (a.x * a.x + a.y * a.y) * alpha;
            }
        } else {
            const int hb = 31 - __clz(lx);
            for (int p = tid; p < (1 << (T - 1)); p += nthr) {
                const int l = (int)insert_zero_u((uint64_t)p, hb);
                const int j = l ^ (int)lx;
                const uint64_t gi = tile_base | (uint64_t)(l & 15) | ((uint64_t)(l >> 4) << h);
                const uint64_t gj = gi ^ gr.xmask;
                double2 a, b;
                asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
                             : "=d"(a.x), "=d"(a.y)
                             : "r"(tile_a + ((uint32_t)swz(l) << 4)));
                asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
                             : "=d"(b.x), "=d"(b.y)
                             : "r"(tile_a + ((uint32_t)swz(j) << 4)));
                const double wr = a.x * b.x + a.y * b.y;
                const double wi = a.x * b.y - a.y * b.x;
                double ai = 0.0, bi = 0.0, aj = 0.0, bj = 0.0;
                for (int t = 0; t < gr.nterms; ++t) {
                    const bool si = __popcll(gi & tp[t].z) & 1, sj = __popcll(gj & tp[t].z) & 1;
                    ai += si ? -tp[t].ca : tp[t].ca;
                    bi += si ? -tp[t].cb : tp[t].cb;
                    aj += sj ? -tp[t].ca : tp[t].ca;
                    bj += sj ? -tp[t].cb : tp[t].cb;
                }
                acc += wr * ai + wi * bi + wr * aj - wi * bj;
            }
        }
        (void)m;
    }
    return acc;
}

__device__ __forceinline__ void gather_tile(uint32_t tile_a, const double2 *__restrict__ slot,
                                            int T, int h, uint64_t tile_base, int tid) {
    for (int l = tid; l < (1 << T); l += kBatchThreads) {
        const uint64_t g = tile_base | (uint64_t)(l & 15) | ((uint64_t)(l >> 4) << h);
        const double2 v = slot[g];
        asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(tile_a + ((uint32_t)swz(l) << 4)),
                     "d"(v.x), "d"(v.y)
                     : "memory");
    }
}

__device__ __forceinline__ void scatter_tile(uint32_t tile_a, double2 *__restrict__ slot, int T,
                                             int h, uint64_t tile_base, int tid) {
    for (int l = tid; l < (1 << T); l += kBatchThreads) {
        const uint64_t g = tile_base | (uint64_t)(l & 15) | ((uint64_t)(l >> 4) << h);
        double2 v;
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
                     : "=d"(v.x), "=d"(v.y)
                     : "r"(tile_a + ((uint32_t)swz(l) << 4)));
        slot[g] = v;
    }
}

__global__ void __launch_bounds__(kBatchThreads, 2)
    k_batch(const BItem *__restrict__ items, int nitems, const BInst *__restrict__ insts,
            const BPass *__restrict__ passes, const FusedRound *__restrict__ rounds,
            const FusedOp *__restrict__ ops, const double *__restrict__ coef,
            const BEWin *__restrict__ ewins, const BGroup *__restrict__ groups,
            const BTerm *__restrict__ terms, double *__restrict__ energy,
            unsigned *__restrict__ counter, double2 *__restrict__ scratch, size_t slot_amps) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t tile_a = smem_u32(base);
    __shared__ int s_item;
    __shared__ double s_red[kBatchThreads / 32];
    const int tid = threadIdx.x;
    double2 *slot = scratch + (size_t)blockIdx.x * slot_amps;

    for (;;) {
        if (tid == 0) s_item = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= nitems) break;
        const BItem item = items[it];
        const BInst in = insts[item.inst];
        const double *icoef = coef + in.coef_base;
        const int cur_p = item.param, minus = item.sign < 0;
        auto coef_of = [&](const FusedOp &op) {
            if (op.param >= 0 && op.param == cur_p)
                return icoef + op.coef_alt + (minus ? (op.type == F_M2 ? 32 : 8) : 0);
            return icoef + op.coef;
        };
        const int T = in.T;
        const int nthr = 1 << (T - 4);
        double acc = 0.0;
        if (in.n <= kSmemStateMax) {
            // whole state in shared memory: |0...0>
            for (int l = tid; l < (1 << T); l += kBatchThreads) {
                const double re = l == 0 ? 1.0 : 0.0;
                asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(tile_a +
                                                                       ((uint32_t)swz(l) << 4)),
                             "d"(re), "d"(0.0)
                             : "memory");
            }
            __syncthreads();
            for (int p = 0; p < in.npass; ++p) {
                const BPass ps = passes[in.pass_begin + p];
                for (int r = 0; r < ps.nrounds; ++r) {
                    if (tid < nthr)
                        run_round<false>(tile_a, rounds[ps.round_begin + r], ops, coef_of, 0ull,
                                         ps.h, tid);
                    __syncthreads();
                }
            }
            for (int w = 0; w < in.newin; ++w) {
                const BEWin ew = ewins[in.ewin_begin + w];
                acc += tile_energy(tile_a, T, ew.h, 0ull, groups, ew.group_begin, ew.ngroups,
                                   terms, tid, kBatchThreads);
            }
        } else {
            // state in this CTA's HBM slot, swept in tiles
            const uint64_t N = 1ull << in.n;
            for (uint64_t i = tid; i < N; i += kBatchThreads)
                slot[i] = make_double2(i == 0 ? 1.0 : 0.0, 0.0);
            __syncthreads();
            const int ntiles = 1 << (in.n - T);
            for (int p = 0; p < in.npass; ++p) {
                const BPass ps = passes[in.pass_begin + p];
                const int h = ps.h, hm = ps.h + T - 4;
                for (int t = 0; t < ntiles; ++t) {
                    const uint64_t c2 = (uint64_t)(t & ((1 << (h - 4)) - 1));
                    const uint64_t c4 = (uint64_t)(t >> (h - 4));
                    const uint64_t tb = (c2 << 4) | (c4 << hm);
                    gather_tile(tile_a, slot, T, h, tb, tid);
                    __syncthreads();
                    for (int r = 0; r < ps.nrounds; ++r) {
                        run_round<false>(tile_a, rounds[ps.round_begin + r], ops, coef_of, tb, h,
                                         tid);
                        __syncthreads();
                    }
                    scatter_tile(tile_a, slot, T, h, tb, tid);
                    __syncthreads();
                }
            }
            for (int w = 0; w < in.newin; ++w) {
                const BEWin ew = ewins[in.ewin_begin + w];
                const int h = ew.h, hm = ew.h + T - 4;
                for (int t = 0; t < ntiles; ++t) {
                    const uint64_t c2 = (uint64_t)(t & ((1 << (h - 4)) - 1));
                    const uint64_t c4 = (uint64_t)(t >> (h - 4));
                    const uint64_t tb = (c2 << 4) | (c4 << hm);
                    gather_tile(tile_a, slot, T, h, tb, tid);
                    __syncthreads();
                    acc += tile_energy(tile_a, T, h, tb, groups, ew.group_begin, ew.ngroups,
                                       terms, tid, kBatchThreads);
                    __syncthreads();
                }
            }
        }
        // block reduction of the FP64 energy (fixed order)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((tid & 31) == 0) s_red[tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            double e = 0.0;
            for (int w = 0; w < kBatchThreads / 32; ++w) e += s_red[w];
            energy[it] = e;
        }
        __syncthreads();
    }
}

static size_t batch_smem() { return (16u << kMaxT) + 2048; }

// Build the device program of every instance for fusion width Tw.
static int build_program(lq_batch *b, int Tw, BProgram &pg) {
    pg.T = Tw;
    std::vector<FusedRound> rounds;
    std::vector<FusedOp> fops;
    std::vector<BPass> passes;
    std::vector<double> dummy;
    pg.h_insts.clear();
    pg.op_gate.assign(b->ninst, {});
    pg.steps.assign(b->ninst, {});
    pg.op_begin.assign(b->ninst, 0);
    pg.nops.assign(b->ninst, 0);
    size_t coef_off = 0;
    for (int i = 0; i < b->ninst; ++i) {
        const int n = b->n[i];
        const int T = n <= kSmemStateMax ? n : std::min(Tw, n);
        std::vector<GateOp> gops(b->ops[i].size());
        std::vector<double> zeros(std::max(b->nparams[i], 1), 0.0);
        for (size_t k = 0; k < gops.size(); ++k)
            LQ_TRY(make_gate_op(&b->ops[i][k], zeros.data(), n, &gops[k]));
        std::vector<PlanStep> steps = plan_circuit(gops, n, T);
        for (auto &st : steps)
            if (!st.fused)
                return set_error(LQ_ERR_UNSUPPORTED,
                                 "instance %d: gate %d cannot be fused (batched engine needs "
                                 "every gate inside a %d-bit window)",
                                 i, st.gate, T);
        BInst in{};
        in.n = n;
        in.T = T;
        in.nparams = b->nparams[i];
        in.pass_begin = (int)passes.size();
        pg.op_begin[i] = (int)fops.size();
        std::vector<double> coef_local;
        for (auto &st : steps) {
            BPass bp{st.pass.h, (int)rounds.size(), (int)st.pass.rounds.size(), 0};
            for (auto &rd : st.pass.rounds) {
                FusedRound fr{};
                fill_round(fr, rd.rpos, T, st.pass.h);
                fr.op_begin = (int)fops.size();
                for (int k : rd.ops) {
                    const int gi = st.pass.gates[k];
                    encode_op(gops[gi], st.pass.h, T - 4, rd.rpos, fops, coef_local);
                    if (fops.back().type == F_M2 || fops.back().type >= F_BLOCK3)
                        return set_error(LQ_ERR_UNSUPPORTED,
                                         "batched engine: 4x4 gates are not supported");
                    pg.op_gate[i].push_back(gi);
                }
                fr.op_end = (int)fops.size();
                rounds.push_back(fr);
            }
            passes.push_back(bp);
        }
        in.npass = (int)passes.size() - in.pass_begin;
        pg.nops[i] = (int)fops.size() - pg.op_begin[i];
        // alternate (+s, -s) coefficient blocks for parameter-bound ops
        size_t alt = coef_local.size();
        for (int k = 0; k < pg.nops[i]; ++k) {
            FusedOp &f = fops[pg.op_begin[i] + k];
            const lq_gate &g = b->ops[i][pg.op_gate[i][k]];
            int p = -1;
            for (int a = 0; a < 3; ++a)
                if (g.param[a] >= 0) {
                    if (p >= 0 && g.param[a] != p)
                        return set_error(LQ_ERR_UNSUPPORTED,
                                         "batched engine: a gate bound to two parameters");
                    p = g.param[a];
                }
            f.param = p;
            if (p >= 0) {
                f.coef_alt = (int)alt;
                alt += 16;
            }
        }
        in.coef_base = (int)coef_off;
        coef_off += alt;
        pg.steps[i] = std::move(steps);
        pg.h_insts.push_back(in);
    }
    pg.ncoef = coef_off;
    // energy windows are shared by the programs (set in lq_batch_create)
    LQ_CUDA_TRY(cudaMalloc(&pg.rounds, sizeof(FusedRound) * std::max<size_t>(rounds.size(), 1)));
    LQ_CUDA_TRY(cudaMalloc(&pg.ops, sizeof(FusedOp) * std::max<size_t>(fops.size(), 1)));
    LQ_CUDA_TRY(cudaMalloc(&pg.passes, sizeof(BPass) * std::max<size_t>(passes.size(), 1)));
    LQ_CUDA_TRY(cudaMalloc(&pg.insts, sizeof(BInst) * pg.h_insts.size()));
    LQ_CUDA_TRY(cudaMemcpy(pg.rounds, rounds.data(), sizeof(FusedRound) * rounds.size(),
                           cudaMemcpyHostToDevice));
    LQ_CUDA_TRY(cudaMemcpy(pg.ops, fops.data(), sizeof(FusedOp) * fops.size(),
                           cudaMemcpyHostToDevice));
    LQ_CUDA_TRY(cudaMemcpy(pg.passes, passes.data(), sizeof(BPass) * passes.size(),
                           cudaMemcpyHostToDevice));
    return LQ_OK;
}

// Host FP64 coefficients of every instance for parameter vector theta.
static int fill_coefficients(lq_batch *b, BProgram &pg, const double *theta, double shift,
                             double *out) {
    for (int i = 0; i < b->ninst; ++i) {
        const int n = b->n[i];
        const double *th = theta + b->param_off[i];
        std::vector<double> tp(th, th + b->nparams[i]);
        double *blk = out + pg.h_insts[i].coef_base;
        size_t base = 0;
        size_t alt_end = 0;
        // base coefficients in encode order, then the alt blocks
        for (int k = 0; k < pg.nops[i]; ++k) {
            const lq_gate &g = b->ops[i][pg.op_gate[i][k]];
            GateOp op;
            LQ_TRY(make_gate_op(&g, tp.data(), n, &op));
            const int nc = op.type == OP_M2 ? 32 : 8;
            for (int q = 0; q < nc; ++q) blk[base + q] = (op.type == OP_PERM1 || op.type == OP_SWAP)
                                                             ? 0.0
                                                             : op.m[q];
            base += nc;
        }
        alt_end = base;
        for (int k = 0; k < pg.nops[i]; ++k) {
            const lq_gate &g = b->ops[i][pg.op_gate[i][k]];
            int p = -1;
            for (int a = 0; a < 3; ++a)
                if (g.param[a] >= 0) p = g.param[a];
            if (p < 0) continue;
            for (int sgn = 0; sgn < 2; ++sgn) {
                tp[p] = th[p] + (sgn == 0 ? shift : -shift);
                GateOp op;
                LQ_TRY(make_gate_op(&g, tp.data(), n, &op));
                for (int q = 0; q < 8; ++q) blk[alt_end + q] = op.m[q];
                alt_end += 8;
            }
            tp[p] = th[p];
        }
    }
    return LQ_OK;
}

static int launch_batch(lq_batch *b, BProgram &pg) {
    LQ_CUDA_TRY(cudaMemsetAsync(b->counter, 0, sizeof(unsigned), b->stream));
    LQ_CUDA_TRY(cudaMemcpyAsync(b->coef_d, b->coef_h, pg.ncoef * sizeof(double),
                                cudaMemcpyHostToDevice, b->stream));
    prof_begin(b->stream, kProfBatch);
    k_batch<<<b->grid, kBatchThreads, batch_smem(), b->stream>>>(
        b->items, b->nitems, pg.insts, pg.passes, pg.rounds, pg.ops, b->coef_d, b->ewins,
        b->groups, b->bterms, b->energy_d, b->counter, b->scratch, b->slot_amps);
    prof_end(b->stream, kProfBatch);
    LQ_CUDA_TRY(cudaGetLastError());
    LQ_CUDA_TRY(cudaMemcpyAsync(b->energy_h, b->energy_d, b->nitems * sizeof(double),
                                cudaMemcpyDeviceToHost, b->stream));
    return LQ_OK;
}

static void free_batch(lq_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto &pg : b->progs) {
        cudaFree(pg.rounds);
        cudaFree(pg.ops);
        cudaFree(pg.passes);
        cudaFree(pg.insts);
    }
    cudaFree(b->ewins);
    cudaFree(b->groups);
    cudaFree(b->bterms);
    cudaFree(b->items);
    cudaFree(b->coef_d);
    if (b->coef_h) cudaFreeHost(b->coef_h);
    cudaFree(b->energy_d);
    if (b->energy_h) cudaFreeHost(b->energy_h);
    cudaFree(b->counter);
    cudaFree(b->scratch);
    cudaFree(b->flag);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // namespace lq

using namespace lq;

extern "C" {

int lq_batch_create(const lq_vqe_instance *instances, int ninstances, lq_batch **out) {
    clear_error();
    if (!out || !instances || ninstances <= 0)
        return set_error(LQ_ERR_INVALID_ARG, "bad instance list");
    *out = nullptr;
    lq_batch *b = new lq_batch();
    b->ninst = ninstances;
    auto fail = [&](int rc) {
        free_batch(b);
        return rc;
    };
    for (int i = 0; i < ninstances; ++i) {
        const lq_vqe_instance &in = instances[i];
        if (in.num_qubits < 5 || in.num_qubits > 24)
            return fail(set_error(LQ_ERR_UNSUPPORTED, "instance %d: %d qubits (supported 5..24)",
                                  i, in.num_qubits));
        if (in.nops < 0 || (in.nops && !in.ops) || in.nparams < 0 || in.nterms < 0 ||
            (in.nterms && !in.terms))
            return fail(set_error(LQ_ERR_INVALID_ARG, "instance %d: bad arrays", i));
        for (int k = 0; k < in.nops; ++k) {
            int rc = validate_gate(&in.ops[k], in.num_qubits, in.nparams);
            if (rc) return fail(rc);
            if (in.ops[k].flags & LQ_FLAG_RENORM)
                return fail(set_error(LQ_ERR_UNSUPPORTED,
                                      "instance %d: renormalising gates are not batched", i));
        }
        b->n.push_back(in.num_qubits);
        b->nparams.push_back(in.nparams);
        b->param_off.push_back(b->total_params);
        b->total_params += in.nparams;
        b->maxn = std::max(b->maxn, in.num_qubits);
        b->ops.emplace_back(in.ops, in.ops + in.nops);
        b->terms.emplace_back(in.terms, in.terms + in.nterms);
    }
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(set_error(LQ_ERR_CUDA, "stream: %s", cudaGetErrorString(e)));
    // Programs for the candidate fusion widths of the tiled (n > 12) instances.
    for (int Tw : {10, 11, 12}) {
        BProgram pg;
        int rc = build_program(b, Tw, pg);
        b->progs.push_back(pg);
        if (rc) return fail(rc);
    }
    // Energy windows and term groups (shared by all programs: they only depend on
    // the instance's tile width, which is <= 12 ... windows use T of program 0 for
    // n > 12 and are rebuilt per program below when T differs).
    std::vector<BEWin> ewins;
    std::vector<BGroup> groups;
    std::vector<BTerm> bterms;
    for (size_t pi = 0; pi < b->progs.size(); ++pi) {
        BProgram &pg = b->progs[pi];
        for (int i = 0; i < b->ninst; ++i) {
            BInst &in = pg.h_insts[i];
            const int n = in.n, T = in.T, m = T - 4;
            std::map<uint64_t, std::vector<int>> byx;
            for (size_t t = 0; t < b->terms[i].size(); ++t) {
                const lq_pauli_term &pt = b->terms[i][t];
                const uint64_t lim = (1ull << n) - 1;
                if ((pt.xmask & ~lim) || (pt.zmask & ~lim))
                    return fail(set_error(LQ_ERR_QUBIT_INDEX, "instance %d term %zu", i, t));
                if (pt.ny != __builtin_popcountll(pt.xmask & pt.zmask))
                    return fail(set_error(LQ_ERR_INVALID_ARG, "instance %d term %zu: ny", i, t));
                byx[pt.xmask].push_back((int)t);
            }
            // window per group: the first h whose window holds every X bit
            std::map<int, std::vector<uint64_t>> win;
            for (auto &kv : byx) {
                int hsel = -1;
                for (int h = 4; h + m <= n; ++h)
                    if ((kv.first & ~window_mask(h, m)) == 0) {
                        hsel = h;
                        break;
                    }
                if (hsel < 0)
                    return fail(set_error(LQ_ERR_UNSUPPORTED,
                                          "instance %d: a Pauli term's X bits span more than "
                                          "one %d-bit window",
                                          i, T));
                win[hsel].push_back(kv.first);
            }
            in.ewin_begin = (int)ewins.size();
            for (auto &w : win) {
                BEWin ew{w.first, (int)groups.size(), (int)w.second.size(), 0};
                for (uint64_t x : w.second) {
                    BGroup g{x, (int)bterms.size(), (int)byx[x].size()};
                    for (int t : byx[x]) {
                        const lq_pauli_term &pt = b->terms[i][t];
                        int k = pt.ny & 3;  // reference convention: Y = +i
                        const double a = k == 0 ? 1.0 : k == 2 ? -1.0 : 0.0;
                        const double bb = k == 1 ? -1.0 : k == 3 ? 1.0 : 0.0;
                        bterms.push_back(BTerm{pt.zmask, pt.coefficient * a, pt.coefficient * bb});
                    }
                    groups.push_back(g);
                }
                ewins.push_back(ew);
            }
            in.newin = (int)ewins.size() - in.ewin_begin;
        }
        e = cudaMemcpy(pg.insts, pg.h_insts.data(), sizeof(BInst) * pg.h_insts.size(),
                       cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return fail(set_error(LQ_ERR_CUDA, "%s", cudaGetErrorString(e)));
    }
    // Work items, largest qubit count first.
    std::vector<BItem> items;
    for (int i = 0; i < b->ninst; ++i) {
        items.push_back(BItem{i, -1, 1, 0});
        for (int p = 0; p < b->nparams[i]; ++p) {
            items.push_back(BItem{i, p, 1, 0});
            items.push_back(BItem{i, p, -1, 0});
        }
    }
    std::stable_sort(items.begin(), items.end(),
                     [&](const BItem &x, const BItem &y) { return b->n[x.inst] > b->n[y.inst]; });
    b->nitems = (int)items.size();
    size_t maxcoef = 0;
    for (auto &pg : b->progs) maxcoef = std::max(maxcoef, pg.ncoef);
    b->coef_cap = std::max<size_t>(maxcoef, 1);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    b->grid = 2 * sms;
    b->slot_amps = b->maxn > kSmemStateMax ? (1ull << b->maxn) : 1;
#define LQ_B_TRY(x)                                                                 \
    do {                                                                            \
        cudaError_t _e = (x);                                                       \
        if (_e != cudaSuccess)                                                      \
            return fail(set_error(_e == cudaErrorMemoryAllocation ? LQ_ERR_OOM : LQ_ERR_CUDA, \
                                  "%s: %s", #x, cudaGetErrorString(_e)));           \
    } while (0)
    LQ_B_TRY(cudaMalloc(&b->ewins, sizeof(BEWin) * std::max<size_t>(ewins.size(), 1)));
    LQ_B_TRY(cudaMalloc(&b->groups, sizeof(BGroup) * std::max<size_t>(groups.size(), 1)));
    LQ_B_TRY(cudaMalloc(&b->bterms, sizeof(BTerm) * std::max<size_t>(bterms.size(), 1)));
    LQ_B_TRY(cudaMalloc(&b->items, sizeof(BItem) * items.size()));
    LQ_B_TRY(cudaMalloc(&b->coef_d, sizeof(double) * b->coef_cap));
    LQ_B_TRY(cudaMallocHost(&b->coef_h, sizeof(double) * b->coef_cap));
    LQ_B_TRY(cudaMalloc(&b->energy_d, sizeof(double) * b->nitems));
    LQ_B_TRY(cudaMallocHost(&b->energy_h, sizeof(double) * b->nitems));
    LQ_B_TRY(cudaMalloc(&b->counter, sizeof(unsigned)));
    LQ_B_TRY(cudaMalloc(&b->flag, sizeof(unsigned)));
    LQ_B_TRY(cudaMalloc(&b->scratch, sizeof(double2) * b->slot_amps * b->grid));
    if (!ewins.empty())
        LQ_B_TRY(cudaMemcpy(b->ewins, ewins.data(), sizeof(BEWin) * ewins.size(),
                            cudaMemcpyHostToDevice));
    if (!groups.empty())
        LQ_B_TRY(cudaMemcpy(b->groups, groups.data(), sizeof(BGroup) * groups.size(),
                            cudaMemcpyHostToDevice));
    if (!bterms.empty())
        LQ_B_TRY(cudaMemcpy(b->bterms, bterms.data(), sizeof(BTerm) * bterms.size(),
                            cudaMemcpyHostToDevice));
    LQ_B_TRY(cudaMemcpy(b->items, items.data(), sizeof(BItem) * items.size(),
                        cudaMemcpyHostToDevice));
    LQ_B_TRY(cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)batch_smem()));
#undef LQ_B_TRY
    *out = b;
    return LQ_OK;
}

int lq_batch_destroy(lq_batch *b) {
    if (!b) return LQ_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_batch(b);
    return LQ_OK;
}

int lq_batch_num_params(const lq_batch *b, int *out) {
    if (!b || !out) return set_error(LQ_ERR_INVALID_ARG, "null argument");
    *out = b->total_params;
    return LQ_OK;
}

int lq_batch_gradients(lq_batch *b, const double *theta, double shift, double *energy,
                       double *grad) {
    if (!b || !theta) return set_error(LQ_ERR_INVALID_ARG, "null argument");
    // Autotune on first use: time each candidate fusion width once, keep the fastest.
    if (b->chosen < 0) {
        b->last_tune_ms.clear();
        double best = 1e300;
        for (size_t pi = 0; pi < b->progs.size(); ++pi) {
            BProgram &pg = b->progs[pi];
            LQ_TRY(fill_coefficients(b, pg, theta, shift, b->coef_h));
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, b->stream);
            LQ_TRY(launch_batch(b, pg));
            cudaEventRecord(e1, b->stream);
            LQ_CUDA_TRY(cudaStreamSynchronize(b->stream));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            b->last_tune_ms.push_back(ms);
            if (ms < best) {
                best = ms;
                b->chosen = (int)pi;
            }
        }
    }
    BProgram &pg = b->progs[b->chosen];
    LQ_TRY(fill_coefficients(b, pg, theta, shift, b->coef_h));
    if (!b->exec) {
        // Capture [counter reset, coefficient upload, persistent kernel, energy
        // download] once; later calls relaunch the instantiated graph.
        LQ_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = launch_batch(b, pg);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return set_error(LQ_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
        b->graph = g;
        LQ_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    LQ_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(b->stream));
    // gradients (E(+s) - E(-s)) / 2 from the item energies
    std::vector<BItem> items(b->nitems);
    LQ_CUDA_TRY(cudaMemcpy(items.data(), b->items, sizeof(BItem) * b->nitems,
                           cudaMemcpyDeviceToHost));
    std::vector<double> ep(b->total_params), em(b->total_params);
    for (int k = 0; k < b->nitems; ++k) {
        const BItem &it = items[k];
        const double e = b->energy_h[k];
        if (it.param < 0) {
            if (energy) energy[it.inst] = e;
        } else if (it.sign > 0) {
            ep[b->param_off[it.inst] + it.param] = e;
        } else {
            em[b->param_off[it.inst] + it.param] = e;
        }
    }
    if (grad)
        for (int j = 0; j < b->total_params; ++j) grad[j] = (ep[j] - em[j]) / 2.0;
    return LQ_OK;
}

int lq_batch_tuning(const lq_batch *b, int *smem_max_qubits, int *threads_per_cta) {
    if (!b) return set_error(LQ_ERR_INVALID_ARG, "null batch");
    if (smem_max_qubits) *smem_max_qubits = kSmemStateMax;
    if (threads_per_cta) *threads_per_cta = b->chosen >= 0 ? b->progs[b->chosen].T : 0;
    return LQ_OK;
}

}  // extern "C"
