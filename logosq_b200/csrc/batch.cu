// Batched parameter-shift engine: the 2P+1 circuits of many VQE instances
// (ParameterShift::compute_gradient, src/optimization/gradient.rs:44-78, run
// for every instance of a batch) in one CUDA graph: coefficient upload, two
// persistent launches (base circuits, then shifted circuits from the base
// circuits' checkpoints) and result download.
//
// Work list: one item per (instance, circuit), circuit 0 unshifted and
// circuits 2j+1 / 2j+2 with parameter j shifted by +s / -s, ordered by cost
// (largest remaining work first) and handed out through an atomic counter to
// persistent CTAs (one per SM).  Per item a CTA simulates the circuit (from
// |0...0>, or from a checkpoint) and reduces its FP64 energy:
//   n <= 12: the whole state lives in the CTA's shared memory (one tile);
//   n  > 12: the state lives in a per-CTA scratch slot in HBM and is swept in
//            2^T-amplitude tiles (T chosen by the autotuner) by the same fused
//            passes and ping-pong register rounds as lq_apply_circuit
//            (fused_round.cuh).
// Gate coefficients are computed on the host in FP64 with the reference
// formulas (identical to the plain path); a shifted circuit only swaps in the
// (+s / -s) coefficients of the ops bound to its parameter.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>

#include "fused_plan.h"
#include "fused_round.cuh"

namespace lq {

struct BInst {
    int32_t n, T, nparams;
    int32_t pass_begin, npass;
    int32_t ewin_begin, newin;
    int32_t coef_base;  // offset of the instance's coefficient block
    int64_t ckpt_off;   // first amplitude of the instance's checkpoints
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
    uint32_t lx;  // X mask in tile-local bits (bits 0-3 stay, bit b >= h maps to 4 + b - h)
    int32_t pad;
};

struct BTerm {
    uint64_t z;
    double ca, cb;
    int32_t p;    // X-mask-0 group: Z bits on tile bits 8..T-1 (terms sorted by it)
    uint32_t lz;  // Z bits inside the window, in tile-local positions
};

struct BItem {
    int32_t inst;
    int32_t param;  // -1: unshifted
    int32_t sign;   // +1 / -1
    int32_t spass;  // first pass to run
    int32_t sround; // first round of that pass
    int32_t src;    // checkpoint holding the state before it (-1: |0...0>)
};

struct BProgram {  // device program for one fusion width
    int T = 0;
    FusedRound *rounds = nullptr;
    PassOp *ops = nullptr;  // op records (parameter bindings in x0 / x1, see batch_op)
    BPass *passes = nullptr;
    BInst *insts = nullptr;
    std::vector<BInst> h_insts;
    std::vector<FusedOp> h_ops;  // host copy of ops (parameter bindings)
    size_t ncoef = 0;
    // per instance: host copies needed to refresh coefficients
    // fop index (instance-local) -> the gates it applies, in order (more than one
    // for a merged run of single-qubit gates on one qubit)
    std::vector<std::vector<std::vector<int>>> op_members;
    std::vector<std::vector<PlanStep>> steps;
    std::vector<int> op_begin;  // first fop of each instance
    std::vector<int> nops;
    std::vector<BPass> h_passes;
    // per instance and parameter: the (pass, round) holding the first op bound
    // to it (pass = npass when no op is)
    std::vector<std::vector<std::pair<int, int>>> first_use;
    // work items (the base circuits first when prefixes are shared) and the
    // checkpoint index of the state after each round (-1: none kept)
    BItem *items = nullptr;
    std::vector<BItem> h_items;
    int nbase = 0;
    int32_t *rckpt = nullptr;
    std::vector<int32_t> h_rckpt;
    size_t ckpt_amps = 0;
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
    int nitems = 0;
    bool share_prefix = false;  // shifted circuits start from the base circuit's checkpoints
    double2 *ckpt = nullptr;
    size_t ckpt_amps = 0;
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
constexpr uint32_t kBatchTileBytes = 16u << kMaxT;  // one tile buffer (two per CTA)

__device__ __forceinline__ uint32_t insert_zero32(uint32_t x, int pos) {
    return ((x >> pos) << (pos + 1)) | (x & ((1u << pos) - 1));
}

__device__ __forceinline__ double2 tile_amp(uint32_t tile_a, int l) {
    double2 a;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
                 : "=d"(a.x), "=d"(a.y)
                 : "r"(tile_a + ((uint32_t)swz(l) << 4)));
    return a;
}

// c[k] <- sum_p c[p] (-1)^popcount(k & p), the 16-point Walsh-Hadamard transform.
__device__ __forceinline__ void wht16(double (&c)[16]) {
#pragma unroll
    for (int s = 1; s < 16; s <<= 1)
#pragma unroll
        for (int k = 0; k < 16; ++k)
            if (!(k & s)) {
                const double x = c[k], y = c[k | s];
                c[k] = x + y;
                c[k | s] = x - y;
            }
}

// Energy contribution of the groups of one window over the tile in smem
// (kBatchThreads threads).  A term's Z sign at global index g is the sign of
// the bits outside the window (tile_base) times the sign of the tile-local bits
// (its lz), so per-term work that depends only on the tile is done once per tile.
__device__ double tile_energy(uint32_t tile_a, int T, int h, uint64_t tile_base,
                              const BGroup *__restrict__ groups, int g0, int ng,
                              const BTerm *__restrict__ terms, int tid) {
    constexpr int nthr = kBatchThreads;
    double acc = 0.0;
    for (int g = g0; g < g0 + ng; ++g) {
        const BGroup gr = groups[g];
        const uint32_t lx = gr.lx;
        const BTerm *tp = terms + gr.term_begin;
        const int nt = gr.nterms;
        if (lx == 0 && T >= 8) {
            // Diagonal group, folded.  This thread's amplitudes l = tid + 256 k
            // (k < 2^(T-8)) differ only in tile bits 8..T-1; a term's sign is the
            // sign of the fixed bits (gfix) times (-1)^popcount(k & p), p = its Z
            // bits there.  Terms arrive sorted by p, so each thread sums them
            // into c[p] and one Walsh-Hadamard transform gives the coefficient of
            // every k: a few operations per amplitude instead of a popcount and a
            // select per term per amplitude.
            const uint64_t gfix =
                tile_base | (uint64_t)(tid & 15) | ((uint64_t)(tid >> 4) << h);
            double c[16];
            int t = 0;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                double sum = 0.0;
                for (; t < nt && tp[t].p == q; ++t)
                    sum += (__popcll(gfix & tp[t].z) & 1) ? -tp[t].ca : tp[t].ca;
                c[q] = sum;
            }
            wht16(c);
            const int nv = 1 << (T - 8);
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if (k < nv) {
                    const double2 a = tile_amp(tile_a, tid + (k << 8));
                    acc += (a.x * a.x + a.y * a.y) * c[k];
                }
        } else if (lx == 0) {
            for (int l = tid; l < (1 << T); l += nthr) {
                const double2 a = tile_amp(tile_a, l);
                double alpha = 0.0;
                for (int t = 0; t < nt; ++t) {
                    const bool sg = (__popcll(tile_base & tp[t].z) + __popc((uint32_t)l & tp[t].lz)) & 1;
                    alpha += sg ? -tp[t].ca : tp[t].ca;
                }
                acc += (a.x * a.x + a.y * a.y) * alpha;
            }
        } else {
            // Pairs (l, l ^ lx), l with bit hb clear.  The j-side sums follow from
            // the i side: a term's Z sign at j is its sign at i times (-1)^ny, and
            // ca = 0 for odd ny, cb = 0 for even ny, so aj = ai and bj = -bi.
            const int hb = 31 - __clz(lx);
            if (nt <= 2) {
                // up to two terms (XX and YY of a bond): coefficients with the
                // sign of their fixed bits, once per tile, in registers
                uint32_t lz0 = 0, lz1 = 0;
                double ca0 = 0.0, cb0 = 0.0, ca1 = 0.0, cb1 = 0.0;
                {
                    const BTerm t0 = tp[0];
                    const bool f = __popcll(tile_base & t0.z) & 1;
                    lz0 = t0.lz;
                    ca0 = f ? -t0.ca : t0.ca;
                    cb0 = f ? -t0.cb : t0.cb;
                }
                if (nt > 1) {
                    const BTerm t1 = tp[1];
                    const bool f = __popcll(tile_base & t1.z) & 1;
                    lz1 = t1.lz;
                    ca1 = f ? -t1.ca : t1.ca;
                    cb1 = f ? -t1.cb : t1.cb;
                }
                for (int p = tid; p < (1 << (T - 1)); p += nthr) {
                    const uint32_t l = insert_zero32((uint32_t)p, hb);
                    const double2 a = tile_amp(tile_a, (int)l), b = tile_amp(tile_a, (int)(l ^ lx));
                    const double wr = a.x * b.x + a.y * b.y;
                    const double wi = a.x * b.y - a.y * b.x;
                    const bool s0 = __popc(l & lz0) & 1, s1 = __popc(l & lz1) & 1;
                    const double ai = (s0 ? -ca0 : ca0) + (s1 ? -ca1 : ca1);
                    const double bi = (s0 ? -cb0 : cb0) + (s1 ? -cb1 : cb1);
                    acc += 2.0 * (wr * ai + wi * bi);
                }
            } else {
                for (int p = tid; p < (1 << (T - 1)); p += nthr) {
                    const uint32_t l = insert_zero32((uint32_t)p, hb);
                    const double2 a = tile_amp(tile_a, (int)l), b = tile_amp(tile_a, (int)(l ^ lx));
                    const double wr = a.x * b.x + a.y * b.y;
                    const double wi = a.x * b.y - a.y * b.x;
                    double ai = 0.0, bi = 0.0;
                    for (int t = 0; t < nt; ++t) {
                        const bool si =
                            (__popcll(tile_base & tp[t].z) + __popc(l & tp[t].lz)) & 1;
                        ai += si ? -tp[t].ca : tp[t].ca;
                        bi += si ? -tp[t].cb : tp[t].cb;
                    }
                    acc += 2.0 * (wr * ai + wi * bi);
                }
            }
        }
    }
    return acc;
}

// src == nullptr reads the state |0...0> without touching memory.
__device__ __forceinline__ void gather_tile(uint32_t tile_a, const double2 *__restrict__ src,
                                            int T, int h, uint64_t tile_base, int tid) {
    for (int l = tid; l < (1 << T); l += kBatchThreads) {
        const uint64_t g = tile_base | (uint64_t)(l & 15) | ((uint64_t)(l >> 4) << h);
        const double2 v = src ? src[g] : make_double2(g == 0 ? 1.0 : 0.0, 0.0);
        asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(tile_a + ((uint32_t)swz(l) << 4)),
                     "d"(v.x), "d"(v.y)
                     : "memory");
    }
}

// The same tile through cp.async (16 bytes per copy, no registers, completes at
// cp.async.wait_all), so that the next tile streams in while the current one is
// worked on; src == nullptr writes the state |0...0> directly.
__device__ __forceinline__ void gather_tile_async(uint32_t tile_a, const double2 *__restrict__ src,
                                                  int T, int h, uint64_t tile_base, int tid) {
    if (!src) {
        gather_tile(tile_a, nullptr, T, h, tile_base, tid);
        return;
    }
    for (int l = tid; l < (1 << T); l += kBatchThreads) {
        const uint64_t g = tile_base | (uint64_t)(l & 15) | ((uint64_t)(l >> 4) << h);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tile_a +
                                                                    ((uint32_t)swz(l) << 4)),
                     "l"(src + g)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
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

// One CTA per SM: the ping-pong register rounds hold two 16-amplitude arrays
// per thread (236 registers, no spills); two CTAs per SM at 128 registers
// spilled and measured slower (2480 vs 2219 ms per 256-instance gradient).
__global__ void __launch_bounds__(kBatchThreads, 1)
    k_batch(const BItem *__restrict__ items, int nitems, const BInst *__restrict__ insts,
            const BPass *__restrict__ passes, const FusedRound *__restrict__ rounds,
            const PassOp *__restrict__ ops, const double *__restrict__ coef,
            const BEWin *__restrict__ ewins, const BGroup *__restrict__ groups,
            const BTerm *__restrict__ terms, double *__restrict__ energy,
            unsigned *__restrict__ counter, double2 *__restrict__ scratch, size_t slot_amps,
            const int32_t *__restrict__ rckpt, double2 *__restrict__ ckpt) {
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
        // an op bound to the shifted parameter reads its (+s, -s) block
        auto coef_of = [&](const PassOp &op) {
            const long long u0 = __double_as_longlong(op.x0), u1 = __double_as_longlong(op.x1);
            const int p0 = (int)(unsigned)u0, p1 = (int)(unsigned)u1;
            if (p0 >= 0 && p0 == cur_p) return icoef + (int)(u0 >> 32) + (minus ? 8 : 0);
            if (p1 >= 0 && p1 == cur_p) return icoef + (int)(u1 >> 32) + (minus ? 8 : 0);
            return icoef + op.coef;
        };
        const int T = in.T;
        const int nthr = 1 << (T - 4);
        double acc = 0.0;
        // A shifted circuit shares every gate before its parameter's first op with
        // the base (unshifted) circuit: it starts at that op's (pass, round) from
        // the base circuit's checkpoint of the state just before it.  The base
        // circuit writes those checkpoints (2^n amplitudes each, natural order).
        const bool base_item = cur_p < 0;
        const size_t N = (size_t)1 << in.n;
        double2 *ck = ckpt + in.ckpt_off;
        const double2 *src = item.src >= 0 ? ck + (size_t)item.src * N : nullptr;
        // n <= 12: the whole state is one tile in shared memory; otherwise it
        // lives in this CTA's HBM slot and every pass sweeps it tile by tile.
        // One code path for both keeps a single inlined copy of the register
        // rounds (register pressure).  Only the 2^(T-4) threads that own
        // amplitudes run a round.
        const bool in_smem = in.n <= kSmemStateMax;
        // (in shared memory T = n and h = 4, so tile element l is amplitude l; a
        // state in the HBM slot is read from src by the first pass's gathers)
        if (in_smem) gather_tile(tile_a, src, T, 4, 0ull, tid);
        __syncthreads();
        const int ntiles = in_smem ? 1 : 1 << (in.n - T);
        auto tile_base = [&](int t, int h) -> uint64_t {
            if (in_smem) return 0ull;
            const uint64_t c2 = (uint64_t)(t & ((1 << (h - 4)) - 1));
            const uint64_t c4 = (uint64_t)(t >> (h - 4));
            return (c2 << 4) | (c4 << (h + T - 4));
        };
        for (int p = item.spass; p < in.npass; ++p) {
            const BPass ps = passes[in.pass_begin + p];
            const int r0 = p == item.spass ? item.sround : 0;
            // the base circuit's pass-end checkpoint takes the place of the slot
            const int cend = base_item ? rckpt[ps.round_begin + ps.nrounds - 1] : -1;
            double2 *dst = cend >= 0 ? ck + (size_t)cend * N : slot;
            // two tile buffers: tile t+1 streams in while tile t is worked on (its
            // amplitudes are disjoint from tile t's, so in-place passes are safe)
            int buf = 0;
            if (!in_smem) gather_tile_async(tile_a, src, T, ps.h, tile_base(0, ps.h), tid);
            for (int t = 0; t < ntiles; ++t) {
                const uint64_t tb = tile_base(t, ps.h);
                const uint32_t cur = tile_a + (uint32_t)buf * kBatchTileBytes;
                if (!in_smem) {
                    asm volatile("cp.async.wait_all;" ::: "memory");
                    __syncthreads();
                    if (t + 1 < ntiles)
                        gather_tile_async(tile_a + (uint32_t)(buf ^ 1) * kBatchTileBytes, src, T,
                                          ps.h, tile_base(t + 1, ps.h), tid);
                }
                for (int r = r0; r < ps.nrounds; ++r) {
                    const FusedRound &rd = rounds[ps.round_begin + r];
                    // ping-pong register round: every op reads one register array
                    // and writes the other (no moves at the op dispatch's joins)
                    if (tid < nthr) {
                        int tbase = 0;
                        for (int j = 0; j < rd.nlane; ++j) tbase |= ((tid >> j) & 1) << rd.lane[j];
                        run_round_pp_sel<0>(cur, rd, ops, coef_of, tb, ps.h, tbase);
                    }
                    __syncthreads();
                    if (base_item) {
                        const int ci = rckpt[ps.round_begin + r];
                        if (ci >= 0 && (in_smem || r + 1 < ps.nrounds)) {
                            scatter_tile(cur, ck + (size_t)ci * N, T, ps.h, tb, tid);
                            __syncthreads();
                        }
                    }
                }
                if (!in_smem) {
                    scatter_tile(cur, dst, T, ps.h, tb, tid);
                    __syncthreads();
                }
                buf ^= 1;
            }
            if (!in_smem) src = dst;
        }
        for (int w = 0; w < in.newin; ++w) {
            const BEWin ew = ewins[in.ewin_begin + w];
            int buf = 0;
            if (!in_smem) gather_tile_async(tile_a, src, T, ew.h, tile_base(0, ew.h), tid);
            for (int t = 0; t < ntiles; ++t) {
                const uint64_t tb = tile_base(t, ew.h);
                const uint32_t cur = tile_a + (uint32_t)buf * kBatchTileBytes;
                if (!in_smem) {
                    asm volatile("cp.async.wait_all;" ::: "memory");
                    __syncthreads();
                    if (t + 1 < ntiles)
                        gather_tile_async(tile_a + (uint32_t)(buf ^ 1) * kBatchTileBytes, src, T,
                                          ew.h, tile_base(t + 1, ew.h), tid);
                }
                acc += tile_energy(cur, T, ew.h, tb, groups, ew.group_begin, ew.ngroups, terms,
                                   tid);
                if (!in_smem) __syncthreads();  // before a later gather overwrites the tile
                buf ^= 1;
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

static size_t batch_smem() { return 2 * kBatchTileBytes + 2048; }

// 2x2 matrix (m00, m01, m10, m11 as re/im pairs) of an uncontrolled
// single-qubit op and the index bit it acts on; false for any other op.
static bool single_bit_matrix(const GateOp &g, int &bit, double m[8]) {
    if (g.renorm) return false;
    if ((g.type == OP_M1 || g.type == OP_PERM1) && g.nctrl == 0) {
        bit = g.t;
        if (g.type == OP_M1) {
            for (int q = 0; q < 8; ++q) m[q] = g.m[q];
        } else {
            const double x[8] = {0, 0, 1, 0, 1, 0, 0, 0};
            for (int q = 0; q < 8; ++q) m[q] = x[q];
        }
        return true;
    }
    if (g.type == OP_DIAG && g.nfix == 0 && g.npat == 1) {
        bit = g.pat[0];
        const double d[8] = {g.m[0], g.m[1], 0, 0, 0, 0, g.m[2], g.m[3]};
        for (int q = 0; q < 8; ++q) m[q] = d[q];
        return true;
    }
    return false;
}

// out = b . a (2x2 complex, re/im pairs): a is applied first.
static void mat2_mul(const double b[8], const double a[8], double out[8]) {
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) {
            double re = 0.0, im = 0.0;
            for (int k = 0; k < 2; ++k) {
                const double br = b[(r * 2 + k) * 2], bi = b[(r * 2 + k) * 2 + 1];
                const double ar = a[(k * 2 + c) * 2], ai = a[(k * 2 + c) * 2 + 1];
                re += br * ar - bi * ai;
                im += br * ai + bi * ar;
            }
            out[(r * 2 + c) * 2] = re;
            out[(r * 2 + c) * 2 + 1] = im;
        }
}

// The parameter a gate is bound to (-1: none); LQ_ERR_UNSUPPORTED for two.
static int gate_param(const lq_gate &g, int *p) {
    *p = -1;
    for (int a = 0; a < 3; ++a)
        if (g.param[a] >= 0) {
            if (*p >= 0 && g.param[a] != *p)
                return set_error(LQ_ERR_UNSUPPORTED,
                                 "batched engine: a gate bound to two parameters");
            *p = g.param[a];
        }
    return LQ_OK;
}

// Coefficients of one encoded op for angles tp: a single gate's own (8 or 32
// doubles, zeros for pure permutations), or the product of a merged run of
// single-qubit gates (8 doubles: a 2x2 for F_M1, phases (d0, d1) for F_DIAG).
static int op_coefficients(const std::vector<lq_gate> &gates, const std::vector<int> &members,
                           const double *tp, int n, double *out) {
    if (members.size() == 1) {
        GateOp op;
        LQ_TRY(make_gate_op(&gates[members[0]], tp, n, &op));
        const int nc = op.type == OP_M2 ? 32 : 8;
        for (int q = 0; q < nc; ++q)
            out[q] = (op.type == OP_PERM1 || op.type == OP_SWAP) ? 0.0 : op.m[q];
        return LQ_OK;
    }
    double acc[8] = {1, 0, 0, 0, 0, 0, 1, 0}, m[8], t[8];
    bool diag = true;
    for (int k : members) {
        GateOp op;
        LQ_TRY(make_gate_op(&gates[k], tp, n, &op));
        int bit;
        if (!single_bit_matrix(op, bit, m))
            return set_error(LQ_ERR_INVALID_ARG, "batched engine: bad merged gate");
        diag = diag && op.type == OP_DIAG;
        mat2_mul(m, acc, t);
        for (int q = 0; q < 8; ++q) acc[q] = t[q];
    }
    if (diag) {
        const double d[8] = {acc[0], acc[1], acc[6], acc[7], 0, 0, 0, 0};
        for (int q = 0; q < 8; ++q) out[q] = d[q];
    } else {
        for (int q = 0; q < 8; ++q) out[q] = acc[q];
    }
    return LQ_OK;
}

// Merge runs of uncontrolled single-qubit gates on the same qubit (no gate in
// between touches that qubit, so the run commutes into one place) into one op,
// as long as the run is bound to at most two parameters.  Returns the ops to
// plan and, per op, the gates it applies.
static int merge_single_qubit_runs(const std::vector<lq_gate> &gates, int n,
                                   std::vector<GateOp> &mops,
                                   std::vector<std::vector<int>> &members) {
    int maxp = 0;
    for (const auto &gt : gates)
        for (int a = 0; a < 3; ++a) maxp = std::max(maxp, gt.param[a] + 1);
    std::vector<double> zeros(maxp + 1, 0.0);
    std::vector<int> open(64, -1);   // per index bit: op a single-qubit gate may join
    std::vector<int> run_params;     // per op: distinct bound parameters (2 slots)
    std::vector<char> all_diag;
    mops.clear();
    members.clear();
    for (size_t k = 0; k < gates.size(); ++k) {
        GateOp g;
        LQ_TRY(make_gate_op(&gates[k], zeros.data(), n, &g));
        int p;
        LQ_TRY(gate_param(gates[k], &p));
        int bit = -1;
        double m[8];
        const bool single = single_bit_matrix(g, bit, m);
        if (single && open[bit] >= 0) {
            const int e = open[bit];
            int &p0 = run_params[2 * e], &p1 = run_params[2 * e + 1];
            const bool fits = p < 0 || p == p0 || p == p1 || p0 < 0 || p1 < 0;
            if (fits) {
                if (p >= 0 && p != p0 && p != p1) (p0 < 0 ? p0 : p1) = p;
                members[e].push_back((int)k);
                all_diag[e] = all_diag[e] && g.type == OP_DIAG;
                continue;
            }
        }
        const uint64_t bits = op_bits(g);
        for (int b = 0; b < 64; ++b)
            if ((bits >> b) & 1) open[b] = -1;
        mops.push_back(g);
        members.push_back({(int)k});
        run_params.push_back(p);
        run_params.push_back(-1);
        all_diag.push_back(g.type == OP_DIAG);
        if (single) open[bit] = (int)mops.size() - 1;
    }
    // merged runs become one 2x2 (or one diagonal) op on their qubit
    for (size_t e = 0; e < mops.size(); ++e) {
        if (members[e].size() == 1) continue;
        int bit;
        double m[8];
        single_bit_matrix(mops[e], bit, m);
        GateOp g;
        if (all_diag[e]) {
            g.type = OP_DIAG;
            g.npat = 1;
            g.pat[0] = bit;
        } else {
            g.type = OP_M1;
            g.t = bit;
        }
        LQ_TRY(op_coefficients(gates, members[e], zeros.data(), n, g.m));
        mops[e] = g;
    }
    return LQ_OK;
}

// The record of a batched op: its 2x2 / X / diagonal / swap code (the ops this
// engine plans use neither x0 nor x1), and in x0 / x1 the parameters it is bound
// to with the offsets of their (+s, -s) coefficient blocks, as int32 pairs
// (parameter, offset); parameter -1: none.
static PassOp batch_op(const FusedOp &f) {
    PassOp p = pass_op(f);
    const int32_t w[4] = {f.param, f.param >= 0 ? f.coef_alt : 0, f.param2,
                          f.param2 >= 0 ? f.coef_alt2 : 0};
    std::memcpy(&p.x0, w, 8);
    std::memcpy(&p.x1, w + 2, 8);
    return p;
}

// Build the device program of every instance for fusion width Tw.
static int build_program(lq_batch *b, int Tw, BProgram &pg) {
    pg.T = Tw;
    std::vector<FusedRound> rounds;
    std::vector<FusedOp> fops;
    std::vector<BPass> passes;
    std::vector<double> dummy;
    pg.h_insts.clear();
    pg.op_members.assign(b->ninst, {});
    pg.steps.assign(b->ninst, {});
    pg.op_begin.assign(b->ninst, 0);
    pg.nops.assign(b->ninst, 0);
    size_t coef_off = 0;
    for (int i = 0; i < b->ninst; ++i) {
        const int n = b->n[i];
        const int T = n <= kSmemStateMax ? n : std::min(Tw, n);
        std::vector<GateOp> gops;
        std::vector<std::vector<int>> members;
        LQ_TRY(merge_single_qubit_runs(b->ops[i], n, gops, members));
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
                    const int ty = fops.back().type;
                    if (!(ty == F_M1 || ty == F_M1C || ty == F_X || ty == F_XC || ty == F_DIAG ||
                          ty == F_SWAP))
                        return set_error(LQ_ERR_UNSUPPORTED,
                                         "batched engine: 4x4 gates are not supported");
                    pg.op_members[i].push_back(members[gi]);
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
            int bound[2] = {-1, -1};
            for (int gi : pg.op_members[i][k]) {
                int p;
                LQ_TRY(gate_param(b->ops[i][gi], &p));
                if (p < 0 || p == bound[0] || p == bound[1]) continue;
                if (bound[0] < 0) bound[0] = p;
                else bound[1] = p;
            }
            f.param = bound[0];
            f.param2 = bound[1];
            if (bound[0] >= 0) {
                f.coef_alt = (int)alt;
                alt += f.type == F_M2 ? 64 : 16;
            }
            if (bound[1] >= 0) {
                f.coef_alt2 = (int)alt;
                alt += 16;
            }
        }
        // first (pass, round) of each parameter's ops, in execution order
        std::vector<std::pair<int, int>> fu(b->nparams[i], {in.npass, 0});
        for (int k = 0; k < in.npass; ++k) {
            const BPass &bp = passes[in.pass_begin + k];
            for (int r = 0; r < bp.nrounds; ++r) {
                const FusedRound &fr = rounds[bp.round_begin + r];
                for (int o = fr.op_begin; o < fr.op_end; ++o)
                    for (int q : {fops[o].param, fops[o].param2})
                        if (q >= 0 && fu[q].first == in.npass) fu[q] = {k, r};
            }
        }
        pg.first_use.push_back(std::move(fu));
        in.coef_base = (int)coef_off;
        coef_off += alt;
        pg.steps[i] = std::move(steps);
        pg.h_insts.push_back(in);
    }
    pg.ncoef = coef_off;
    pg.h_ops = fops;
    pg.h_passes = passes;
    pg.h_rckpt.assign(rounds.size(), -1);
    // energy windows are shared by the programs (set in lq_batch_create)
    LQ_CUDA_TRY(cudaMalloc(&pg.rounds, sizeof(FusedRound) * std::max<size_t>(rounds.size(), 1)));
    std::vector<PassOp> pops;
    for (const FusedOp &f : fops) pops.push_back(batch_op(f));
    LQ_CUDA_TRY(cudaMalloc(&pg.ops, sizeof(PassOp) * std::max<size_t>(pops.size(), 1)));
    LQ_CUDA_TRY(cudaMalloc(&pg.passes, sizeof(BPass) * std::max<size_t>(passes.size(), 1)));
    LQ_CUDA_TRY(cudaMalloc(&pg.insts, sizeof(BInst) * pg.h_insts.size()));
    LQ_CUDA_TRY(cudaMemcpy(pg.rounds, rounds.data(), sizeof(FusedRound) * rounds.size(),
                           cudaMemcpyHostToDevice));
    LQ_CUDA_TRY(cudaMemcpy(pg.ops, pops.data(), sizeof(PassOp) * pops.size(),
                           cudaMemcpyHostToDevice));
    LQ_CUDA_TRY(cudaMemcpy(pg.passes, passes.data(), sizeof(BPass) * passes.size(),
                           cudaMemcpyHostToDevice));
    return LQ_OK;
}

// Work items and checkpoints of program pg.  Without shared prefixes every
// circuit runs from |0...0> in one launch.  With them the base circuits run
// first, in a launch of their own, keeping per instance the state just before
// each parameter's first op (after round r-1 of its pass, or after the previous
// pass); each shifted circuit then starts at that op from that checkpoint, so
// the gates before it are applied once per instance instead of once per
// circuit.  The sums are the same in the same order, so the energies are
// bitwise those of the unshared launch.
static void plan_items(lq_batch *b, BProgram &pg, bool share) {
    std::fill(pg.h_rckpt.begin(), pg.h_rckpt.end(), -1);
    pg.h_items.clear();
    std::vector<BItem> shifted;
    size_t amps = 0;
    for (int i = 0; i < b->ninst; ++i) {
        BInst &in = pg.h_insts[i];
        in.ckpt_off = (int64_t)amps;
        pg.h_items.push_back(BItem{i, -1, 1, 0, 0, -1});
        auto round_index = [&](int k, int r) {
            return pg.h_passes[in.pass_begin + k].round_begin + r;
        };
        int nck = 0;
        for (int p = 0; p < in.nparams; ++p) {
            int k = 0, r = 0, src = -1;
            const std::pair<int, int> fu = pg.first_use[i][p];
            if (share && fu.first < in.npass) {
                k = fu.first;
                r = fu.second;
                int gr = -1;
                if (r > 0)
                    gr = round_index(k, r - 1);
                else if (k > 0)
                    gr = round_index(k - 1, pg.h_passes[in.pass_begin + k - 1].nrounds - 1);
                if (gr >= 0) {
                    if (pg.h_rckpt[gr] < 0) pg.h_rckpt[gr] = nck++;
                    src = pg.h_rckpt[gr];
                }
            }
            for (int sg : {1, -1}) shifted.push_back(BItem{i, p, sg, k, r, src});
        }
        amps += (size_t)nck << in.n;
    }
    // largest remaining work first (passes carry a tile sweep each, rounds the
    // register work, the energy windows a sweep each)
    auto cost = [&](const BItem &it) {
        const BInst &in = pg.h_insts[it.inst];
        double w = 2.0 * in.newin - it.sround;
        for (int k = it.spass; k < in.npass; ++k)
            w += 4.0 + pg.h_passes[in.pass_begin + k].nrounds;
        return std::ldexp(w, in.n);
    };
    if (share) {
        std::stable_sort(pg.h_items.begin(), pg.h_items.end(), [&](const BItem &x, const BItem &y) {
            return b->n[x.inst] > b->n[y.inst];
        });
        std::stable_sort(shifted.begin(), shifted.end(),
                         [&](const BItem &x, const BItem &y) { return cost(x) > cost(y); });
        pg.nbase = (int)pg.h_items.size();
        pg.h_items.insert(pg.h_items.end(), shifted.begin(), shifted.end());
    } else {
        pg.h_items.insert(pg.h_items.end(), shifted.begin(), shifted.end());
        std::stable_sort(pg.h_items.begin(), pg.h_items.end(), [&](const BItem &x, const BItem &y) {
            return b->n[x.inst] > b->n[y.inst];
        });
        pg.nbase = 0;
    }
    pg.ckpt_amps = share ? amps : 0;
}

// Host FP64 coefficients of every instance for parameter vector theta.
static int fill_coefficients(lq_batch *b, BProgram &pg, const double *theta, double shift,
                             double *out) {
    for (int i = 0; i < b->ninst; ++i) {
        const int n = b->n[i];
        const double *th = theta + b->param_off[i];
        std::vector<double> tp(th, th + b->nparams[i]);
        double *blk = out + pg.h_insts[i].coef_base;
        // base coefficients in encode order, then the alt blocks of every
        // parameter-bound op: (+s, -s) for its first parameter, then its second
        size_t base = 0;
        for (int k = 0; k < pg.nops[i]; ++k) {
            const auto &mem = pg.op_members[i][k];
            LQ_TRY(op_coefficients(b->ops[i], mem, tp.data(), n, blk + base));
            bool m2 = false;
            if (mem.size() == 1) {
                GateOp op;
                LQ_TRY(make_gate_op(&b->ops[i][mem[0]], tp.data(), n, &op));
                m2 = op.type == OP_M2;
            }
            base += m2 ? 32 : 8;
        }
        size_t alt_end = base;
        for (int k = 0; k < pg.nops[i]; ++k) {
            const FusedOp &f = pg.h_ops[pg.op_begin[i] + k];
            const auto &mem = pg.op_members[i][k];
            for (int p : {f.param, f.param2}) {
                if (p < 0) continue;
                for (int sgn = 0; sgn < 2; ++sgn) {
                    tp[p] = th[p] + (sgn == 0 ? shift : -shift);
                    LQ_TRY(op_coefficients(b->ops[i], mem, tp.data(), n, blk + alt_end));
                    alt_end += 8;
                }
                tp[p] = th[p];
            }
        }
    }
    return LQ_OK;
}

static int launch_batch(lq_batch *b, BProgram &pg) {
    LQ_CUDA_TRY(cudaMemsetAsync(b->counter, 0, 2 * sizeof(unsigned), b->stream));
    LQ_CUDA_TRY(cudaMemcpyAsync(b->coef_d, b->coef_h, pg.ncoef * sizeof(double),
                                cudaMemcpyHostToDevice, b->stream));
    prof_begin(b->stream, kProfBatch);
    // items [0, nbase): the base circuits, which write the checkpoints that the
    // shifted circuits [nbase, nitems) start from (stream order between the two)
    const int bounds[3] = {0, pg.nbase, b->nitems};
    for (int ph = 0; ph < 2; ++ph) {
        const int i0 = bounds[ph], cnt = bounds[ph + 1] - bounds[ph];
        if (cnt <= 0) continue;
        k_batch<<<b->grid, kBatchThreads, batch_smem(), b->stream>>>(
            pg.items + i0, cnt, pg.insts, pg.passes, pg.rounds, pg.ops, b->coef_d, b->ewins,
            b->groups, b->bterms, b->energy_d + i0, b->counter + ph, b->scratch, b->slot_amps,
            pg.rckpt, b->ckpt);
        LQ_CUDA_TRY(cudaGetLastError());
    }
    prof_end(b->stream, kProfBatch);
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
        cudaFree(pg.items);
        cudaFree(pg.rckpt);
    }
    cudaFree(b->ckpt);
    cudaFree(b->ewins);
    cudaFree(b->groups);
    cudaFree(b->bterms);
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
    // Shared prefixes (LQ_BATCH_PREFIX=0 turns them off) need the checkpoints
    // of the largest program to fit next to the scratch slots.
    {
        const char *ev = getenv("LQ_BATCH_PREFIX");
        b->share_prefix = !(ev && atoi(ev) == 0);
        size_t need = 0;
        for (auto &pg : b->progs) {
            plan_items(b, pg, b->share_prefix);
            need = std::max(need, pg.ckpt_amps);
        }
        size_t freeb = 0, totalb = 0;
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const size_t slots = b->maxn > kSmemStateMax ? (size_t)nsm << b->maxn : 0;
        if (b->share_prefix && (cudaMemGetInfo(&freeb, &totalb) != cudaSuccess ||
                                (need + slots) * sizeof(double2) > freeb / 10 * 8)) {
            b->share_prefix = false;
            for (auto &pg : b->progs) plan_items(b, pg, false);
            need = 0;
        }
        b->ckpt_amps = need;
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
            // Windows: every window is one sweep of the state, so take the fewest.
            // A group's X bits above bit 3 need h in [hi - m + 1, lo] (within
            // [4, n - m]); points stabbing every such interval, chosen greedily by
            // right end, are a minimum set.  Groups with no X bit above 3 go to
            // the first window.
            struct Need {
                int a, b;
                uint64_t x;
            };
            std::vector<Need> need;
            std::vector<uint64_t> free_groups;
            for (auto &kv : byx) {
                const uint64_t up = kv.first & ~0xFull;
                if (!up) {
                    free_groups.push_back(kv.first);
                    continue;
                }
                const int lo = __builtin_ctzll(up), hi = 63 - __builtin_clzll(up);
                const int a = std::max(4, hi - m + 1), bnd = std::min(lo, n - m);
                if (a > bnd)
                    return fail(set_error(LQ_ERR_UNSUPPORTED,
                                          "instance %d: a Pauli term's X bits span more than "
                                          "one %d-bit window",
                                          i, T));
                need.push_back(Need{a, bnd, kv.first});
            }
            std::stable_sort(need.begin(), need.end(),
                             [](const Need &u, const Need &v) { return u.b < v.b; });
            std::map<int, std::vector<uint64_t>> win;
            int cur = -1;
            for (const Need &q : need) {
                if (cur < q.a) cur = q.b;
                win[cur].push_back(q.x);
            }
            const int hfree = win.empty() ? 4 : win.begin()->first;
            for (uint64_t x : free_groups) win[hfree].push_back(x);
            in.ewin_begin = (int)ewins.size();
            for (auto &w : win) {
                BEWin ew{w.first, (int)groups.size(), (int)w.second.size(), 0};
                for (uint64_t x : w.second) {
                    uint32_t lx = 0;  // the window holds every X bit (chosen above)
                    for (int bt = 0; bt < n; ++bt)
                        if ((x >> bt) & 1) lx |= 1u << (bt < 4 ? bt : 4 + (bt - w.first));
                    BGroup g{x, (int)bterms.size(), (int)byx[x].size(), lx, 0};
                    const int h = w.first;
                    const uint64_t wm = window_mask(h, m);
                    std::vector<BTerm> gt;
                    for (int t : byx[x]) {
                        const lq_pauli_term &pt = b->terms[i][t];
                        int k = pt.ny & 3;  // reference convention: Y = +i
                        const double a = k == 0 ? 1.0 : k == 2 ? -1.0 : 0.0;
                        const double bb = k == 1 ? -1.0 : k == 3 ? 1.0 : 0.0;
                        uint32_t lz = 0;  // Z bits inside the window, tile-local
                        for (int bt = 0; bt < n; ++bt)
                            if ((pt.zmask & wm) >> bt & 1) lz |= 1u << (bt < 4 ? bt : 4 + (bt - h));
                        // the diagonal group's fold index: Z bits on tile bits 8..T-1
                        const int p =
                            T >= 8 ? (int)((pt.zmask >> (h + 4)) & ((1ull << (T - 8)) - 1)) : 0;
                        gt.push_back(BTerm{pt.zmask, pt.coefficient * a, pt.coefficient * bb, p, lz});
                    }
                    if (x == 0)
                        std::stable_sort(gt.begin(), gt.end(),
                                         [](const BTerm &u, const BTerm &v) { return u.p < v.p; });
                    bterms.insert(bterms.end(), gt.begin(), gt.end());
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
    b->nitems = (int)b->progs[0].h_items.size();
    size_t maxcoef = 0;
    for (auto &pg : b->progs) maxcoef = std::max(maxcoef, pg.ncoef);
    b->coef_cap = std::max<size_t>(maxcoef, 1);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    b->grid = sms;  // one resident CTA per SM
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
    for (auto &pg : b->progs) {
        LQ_B_TRY(cudaMalloc(&pg.items, sizeof(BItem) * pg.h_items.size()));
        LQ_B_TRY(cudaMalloc(&pg.rckpt, sizeof(int32_t) * std::max<size_t>(pg.h_rckpt.size(), 1)));
        LQ_B_TRY(cudaMemcpy(pg.items, pg.h_items.data(), sizeof(BItem) * pg.h_items.size(),
                            cudaMemcpyHostToDevice));
        if (!pg.h_rckpt.empty())
            LQ_B_TRY(cudaMemcpy(pg.rckpt, pg.h_rckpt.data(), sizeof(int32_t) * pg.h_rckpt.size(),
                                cudaMemcpyHostToDevice));
    }
    LQ_B_TRY(cudaMalloc(&b->ckpt, sizeof(double2) * std::max<size_t>(b->ckpt_amps, 1)));
    LQ_B_TRY(cudaMalloc(&b->coef_d, sizeof(double) * b->coef_cap));
    LQ_B_TRY(cudaMallocHost(&b->coef_h, sizeof(double) * b->coef_cap));
    LQ_B_TRY(cudaMalloc(&b->energy_d, sizeof(double) * b->nitems));
    LQ_B_TRY(cudaMallocHost(&b->energy_h, sizeof(double) * b->nitems));
    LQ_B_TRY(cudaMalloc(&b->counter, 2 * sizeof(unsigned)));
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
    const std::vector<BItem> &items = pg.h_items;
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

int lq_batch_tuning(const lq_batch *b, int *smem_max_qubits, int *tile_bits) {
    if (!b) return set_error(LQ_ERR_INVALID_ARG, "null batch");
    if (smem_max_qubits) *smem_max_qubits = kSmemStateMax;
    if (tile_bits) *tile_bits = b->chosen >= 0 ? b->progs[b->chosen].T : 0;
    return LQ_OK;
}

int lq_batch_prefix_info(const lq_batch *b, int *shared, uint64_t *checkpoint_bytes) {
    if (!b) return set_error(LQ_ERR_INVALID_ARG, "null batch");
    if (shared) *shared = b->share_prefix ? 1 : 0;
    if (checkpoint_bytes) *checkpoint_bytes = (uint64_t)b->ckpt_amps * sizeof(double2);
    return LQ_OK;
}

int lq_batch_set_tile_bits(lq_batch *b, int tile_bits) {
    if (!b) return set_error(LQ_ERR_INVALID_ARG, "null batch");
    int pick = -1;
    for (size_t pi = 0; pi < b->progs.size(); ++pi)
        if (b->progs[pi].T == tile_bits) pick = (int)pi;
    if (tile_bits != 0 && pick < 0)
        return set_error(LQ_ERR_INVALID_ARG, "tile bits %d not among the planned widths (10-12)",
                         tile_bits);
    // the captured graph belongs to the previous choice
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->chosen = pick;  // -1: autotune again on the next lq_batch_gradients call
    return LQ_OK;
}

}  // extern "C"
