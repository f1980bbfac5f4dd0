// Fused k-qubit block passes: Circuit::execute (src/circuits/mod.rs:352-375)
// without one full-state sweep per gate.
//
// A pass owns a set W of T <= 12 index bits: the four lowest bits (so every
// global access is a 256-byte contiguous run) plus a contiguous range
// [h, h+T-4).  Each CTA stages one 2^T-amplitude tile (64 KiB of complex128 at
// T = 12) from HBM into shared memory with one TMA tensor copy (128-byte
// swizzle), applies every gate of the pass that acts inside W, and writes the
// tile back with one TMA store.  Inside the CTA the gates run in "rounds": a
// round picks four tile bits R, each thread gathers the 16 amplitudes that
// differ only in R into registers, applies all of the round's gates there, and
// scatters them back.  HBM traffic per pass is one read and one write of the
// state, however many gates the pass holds.
//
// The planner (host) picks windows greedily: at each step it chooses the h
// that lets the most not-yet-applied gates run (respecting gate order per
// bit), then splits that pass into register rounds.  Gates that fit no window
// (two-qubit gates whose bits are further apart than the window) and gates
// that renormalise run as standalone per-gate sweeps at their place in order.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "gate_ops.h"

namespace lq {

// ---------------------------------------------------------------------------
// Device program of a pass
// ---------------------------------------------------------------------------
enum FusedOpType {
    F_M1 = 0,     // 2x2 on reg bit k0, controls: reg-bit mask cm (all set)
    F_PERM1 = 1,  // X on reg bit k0, controls cm
    F_DIAG = 2,   // phases on pattern reg bits (k0 lsb, k1), fix mask cm
    F_SWAP = 3,   // swap reg bits k0, k1
    F_M2 = 4,     // 4x4, index = bit(k0)<<1 | bit(k1)
    F_BLOCK3 = 5, // 8x8 on reg bits 0..2 (matrix bit j <-> reg bit j)
    F_BLOCK4 = 6  // 16x16 on reg bits 0..3
};

struct FusedOp {
    int32_t type;
    int32_t k0, k1, npat;
    int32_t cm;       // control / fix mask over register bits
    int32_t coef;     // offset of the coefficients in the coefficient array (doubles)
};

struct FusedRound {
    int32_t rpos[4];   // tile-local bit positions of register bits 0..3
    int32_t lane[12];  // tile-local positions of thread-index bits, in order
    int32_t nlane;
    int32_t op_begin, op_end;
    int32_t pad;
};

constexpr int kMaxT = 12;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 3) & 7); }

template <int K>
__device__ __forceinline__ void reg_m1(double2 (&a)[16], int cm, const double *__restrict__ c) {
    const double m00r = c[0], m00i = c[1], m01r = c[2], m01i = c[3];
    const double m10r = c[4], m10i = c[5], m11r = c[6], m11i = c[7];
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if (e & (1 << K)) continue;
        if ((e & cm) != cm) continue;
        const double2 a0 = a[e], a1 = a[e | (1 << K)];
        double2 o0, o1;
        o0.x = (m00r * a0.x - m00i * a0.y) + (m01r * a1.x - m01i * a1.y);
        o0.y = (m00r * a0.y + m00i * a0.x) + (m01r * a1.y + m01i * a1.x);
        o1.x = (m10r * a0.x - m10i * a0.y) + (m11r * a1.x - m11i * a1.y);
        o1.y = (m10r * a0.y + m10i * a0.x) + (m11r * a1.y + m11i * a1.x);
        a[e] = o0;
        a[e | (1 << K)] = o1;
    }
}

template <int K>
__device__ __forceinline__ void reg_perm1(double2 (&a)[16], int cm) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if (e & (1 << K)) continue;
        if ((e & cm) != cm) continue;
        const double2 t = a[e];
        a[e] = a[e | (1 << K)];
        a[e | (1 << K)] = t;
    }
}

template <int K0, int K1>
__device__ __forceinline__ void reg_swap(double2 (&a)[16]) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if ((e & (1 << K0)) && !(e & (1 << K1))) {
            const int f = e ^ (1 << K0) ^ (1 << K1);
            const double2 t = a[e];
            a[e] = a[f];
            a[f] = t;
        }
    }
}

template <int K0, int K1>
__device__ __forceinline__ void reg_m2(double2 (&a)[16], const double *__restrict__ c) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if ((e & (1 << K0)) || (e & (1 << K1))) continue;
        const int idx[4] = {e, e | (1 << K1), e | (1 << K0), e | (1 << K0) | (1 << K1)};
        double2 in[4], out[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) in[r] = a[idx[r]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            double ore = 0.0, oim = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double mr = c[(r * 4 + q) * 2], mi = c[(r * 4 + q) * 2 + 1];
                ore += mr * in[q].x - mi * in[q].y;
                oim += mr * in[q].y + mi * in[q].x;
            }
            out[r] = make_double2(ore, oim);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) a[idx[r]] = out[r];
    }
}

template <int KB>
__device__ __forceinline__ void reg_block(double2 (&a)[16], const double *__restrict__ c) {
    constexpr int D = 1 << KB;
#pragma unroll
    for (int hiv = 0; hiv < 16; hiv += D) {
        double2 in[D];
#pragma unroll
        for (int q = 0; q < D; ++q) in[q] = a[hiv + q];
#pragma unroll
        for (int r = 0; r < D; ++r) {
            double ore = 0.0, oim = 0.0;
#pragma unroll
            for (int q = 0; q < D; ++q) {
                const double mr = c[(r * D + q) * 2], mi = c[(r * D + q) * 2 + 1];
                ore += mr * in[q].x - mi * in[q].y;
                oim += mr * in[q].y + mi * in[q].x;
            }
            a[hiv + r] = make_double2(ore, oim);
        }
    }
}

__device__ __forceinline__ void reg_diag(double2 (&a)[16], const FusedOp &op,
                                         const double *__restrict__ c) {
    const double p0r = c[0], p0i = c[1], p1r = c[2], p1i = c[3];
    const double p2r = c[4], p2i = c[5], p3r = c[6], p3i = c[7];
    const int k0 = op.k0, k1 = op.k1, np = op.npat, cm = op.cm;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if ((e & cm) != cm) continue;
        const int b0 = np > 0 ? (e >> k0) & 1 : 0;
        const int b1 = np > 1 ? (e >> k1) & 1 : 0;
        const double pr = b1 ? (b0 ? p3r : p2r) : (b0 ? p1r : p0r);
        const double pi = b1 ? (b0 ? p3i : p2i) : (b0 ? p1i : p0i);
        const double2 v = a[e];
        a[e] = make_double2(v.x * pr - v.y * pi, v.x * pi + v.y * pr);
    }
}

template <bool BLOCKS>
__device__ __forceinline__ void apply_fused_op(double2 (&a)[16], const FusedOp &op,
                                               const double *__restrict__ coef) {
    const double *c = coef + op.coef;
    switch (op.type) {
    case F_M1:
        switch (op.k0) {
        case 0: reg_m1<0>(a, op.cm, c); break;
        case 1: reg_m1<1>(a, op.cm, c); break;
        case 2: reg_m1<2>(a, op.cm, c); break;
        default: reg_m1<3>(a, op.cm, c); break;
        }
        break;
    case F_PERM1:
        switch (op.k0) {
        case 0: reg_perm1<0>(a, op.cm); break;
        case 1: reg_perm1<1>(a, op.cm); break;
        case 2: reg_perm1<2>(a, op.cm); break;
        default: reg_perm1<3>(a, op.cm); break;
        }
        break;
    case F_DIAG:
        reg_diag(a, op, c);
        break;
    case F_SWAP: {
        const int key = op.k0 * 4 + op.k1;
        switch (key) {
        case 1: reg_swap<0, 1>(a); break;
        case 2: reg_swap<0, 2>(a); break;
        case 3: reg_swap<0, 3>(a); break;
        case 4: reg_swap<1, 0>(a); break;
        case 6: reg_swap<1, 2>(a); break;
        case 7: reg_swap<1, 3>(a); break;
        case 8: reg_swap<2, 0>(a); break;
        case 9: reg_swap<2, 1>(a); break;
        case 11: reg_swap<2, 3>(a); break;
        case 12: reg_swap<3, 0>(a); break;
        case 13: reg_swap<3, 1>(a); break;
        default: reg_swap<3, 2>(a); break;
        }
        break;
    }
    case F_M2: {
        if constexpr (!BLOCKS) break;
        const int key = op.k0 * 4 + op.k1;
        switch (key) {
        case 1: reg_m2<0, 1>(a, c); break;
        case 2: reg_m2<0, 2>(a, c); break;
        case 3: reg_m2<0, 3>(a, c); break;
        case 4: reg_m2<1, 0>(a, c); break;
        case 6: reg_m2<1, 2>(a, c); break;
        case 7: reg_m2<1, 3>(a, c); break;
        case 8: reg_m2<2, 0>(a, c); break;
        case 9: reg_m2<2, 1>(a, c); break;
        case 11: reg_m2<2, 3>(a, c); break;
        case 12: reg_m2<3, 0>(a, c); break;
        case 13: reg_m2<3, 1>(a, c); break;
        default: reg_m2<3, 2>(a, c); break;
        }
        break;
    }
    default:
        if constexpr (BLOCKS) {
            if (op.type == F_BLOCK3) reg_block<3>(a, c);
            else reg_block<4>(a, c);
        }
        break;
    }
}

// Bounded wait on an mbarrier phase.  Returns false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < (1u << 24); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

struct TileCoords {
    int32_t h4;  // h - 4: width of the dim-2 coordinate inside blockIdx
};

// One CTA = one tile.  blockDim.x = 2^(T-4), dynamic smem = 2^T*16 + 2048.
template <bool BLOCKS>
__global__ void __launch_bounds__(256, 2)
    k_fused_pass(const __grid_constant__ CUtensorMap tmap, int T, TileCoords tc,
                 const FusedRound *__restrict__ rounds, int nrounds,
                 const FusedOp *__restrict__ ops, const double *__restrict__ coef,
                 unsigned *__restrict__ flag) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    double2 *tile = (double2 *)base;
    uint64_t *bar = (uint64_t *)(base + (16u << T));
    const uint32_t bar_a = smem_u32(bar);
    const uint32_t tile_a = smem_u32(tile);
    const int tid = threadIdx.x;

    const int32_t bid = (int32_t)blockIdx.x;
    const int32_t c2 = bid & ((1 << tc.h4) - 1);
    const int32_t c4 = bid >> tc.h4;
    const int32_t zero = 0;

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_a), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t bytes = 16u << T;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a),
                     "r"(bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(tile_a),
            "l"((uint64_t)&tmap), "r"(zero), "r"(zero), "r"(c2), "r"(zero), "r"(c4), "r"(bar_a)
            : "memory");
    }
    if (!mbar_wait(bar_a, 0)) {
        if (tid == 0) atomicOr(flag, kFlagTimeout);
        return;
    }

    for (int r = 0; r < nrounds; ++r) {
        const FusedRound &rd = rounds[r];
        // thread base index: thread bits scattered to the round's lane positions
        int tbase = 0;
        for (int j = 0; j < rd.nlane; ++j) tbase |= ((tid >> j) & 1) << rd.lane[j];
        const int p0 = 1 << rd.rpos[0], p1 = 1 << rd.rpos[1];
        const int p2 = 1 << rd.rpos[2], p3 = 1 << rd.rpos[3];
        double2 a[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const int idx = tbase | ((e & 1) ? p0 : 0) | ((e & 2) ? p1 : 0) |
                            ((e & 4) ? p2 : 0) | ((e & 8) ? p3 : 0);
            a[e] = tile[swz(idx)];
        }
        for (int o = rd.op_begin; o < rd.op_end; ++o) {
            const FusedOp op = ops[o];
            apply_fused_op<BLOCKS>(a, op, coef);
        }
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const int idx = tbase | ((e & 1) ? p0 : 0) | ((e & 2) ? p1 : 0) |
                            ((e & 4) ? p2 : 0) | ((e & 8) ? p3 : 0);
            tile[swz(idx)] = a[e];
        }
        __syncthreads();
    }
    // Make the generic-proxy writes visible to the TMA engine, then store.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
        asm volatile(
            "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group"
            " [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"((uint64_t)&tmap),
            "r"(zero), "r"(zero), "r"(c2), "r"(zero), "r"(c4), "r"(tile_a)
            : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
}

// ---------------------------------------------------------------------------
// Host: tensor maps
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// Tensor map of a complex128 state for the window [0,4) U [h, h+m):
//   dim0: 16 doubles (8 amplitudes, index bits 0-2), box 16 (=128 B, swizzle span)
//   dim1: 2  (bit 3)                                  box 2
//   dim2: 2^(h-4) (bits 4..h-1)                        box 1
//   dim3: 2^m (bits h..h+m-1)                          box 2^m
//   dim4: 2^(n-h-m) (bits h+m..n-1)                    box 1
static int make_tile_map(CUtensorMap *map, void *d, int n, int h, int m) {
    auto enc = get_encode();
    if (!enc) return set_error(LQ_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    cuuint64_t dims[5] = {16, 2, 1ull << (h - 4), 1ull << m, 1ull << (n - h - m)};
    cuuint64_t strides[4] = {128, 256, 16ull << h, 16ull << (h + m)};
    cuuint32_t box[5] = {16, 2, 1, (cuuint32_t)(1u << m), 1};
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, d, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return set_error(LQ_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) n=%d h=%d m=%d", (int)r,
                         n, h, m);
    return LQ_OK;
}

// ---------------------------------------------------------------------------
// Host: planner
// ---------------------------------------------------------------------------
struct PlannedRound {
    int rpos[4];
    std::vector<int> ops;  // indices into the pass op list
    bool block = false;
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

static inline int popc(uint64_t x) { return __builtin_popcountll(x); }

static uint64_t window_mask(int h, int m) {
    return 0xFull | (((1ull << m) - 1) << h);
}

// Local position of global bit b inside the window [0,4) U [h, h+m).
static inline int local_pos(int b, int h) { return b < 4 ? b : 4 + (b - h); }

static int choose_lanes(const int rpos[4], int T, int *lane) {
    // Thread-index bits go to the tile positions outside R.  The first three
    // should be positions whose swizzle images (p mod 3 for p < 6) differ, so
    // that 8 consecutive threads touch 8 distinct 16-byte bank groups.
    bool inR[kMaxT] = {false};
    for (int k = 0; k < 4; ++k) inR[rpos[k]] = true;
    std::vector<int> free;
    for (int p = 0; p < T; ++p)
        if (!inR[p]) free.push_back(p);
    std::vector<int> first;
    for (int res = 0; res < 3; ++res) {
        for (int p : free) {
            if (p < 6 && p % 3 == res &&
                std::find(first.begin(), first.end(), p) == first.end()) {
                first.push_back(p);
                break;
            }
        }
    }
    std::vector<int> order = first;
    for (int p : free)
        if (std::find(order.begin(), order.end(), p) == order.end()) order.push_back(p);
    for (size_t j = 0; j < order.size(); ++j) lane[j] = order[j];
    return (int)order.size();
}

static void pad_rpos(std::vector<int> &R, int T) {
    // Fill up to four register bits, preferring positions that keep one of
    // each pair (r, r+3), r < 3, outside R (see choose_lanes).
    auto conflicts = [&](int p) {
        if (p >= 6) return false;
        const int partner = p < 3 ? p + 3 : p - 3;
        return std::find(R.begin(), R.end(), partner) != R.end();
    };
    for (int pass = 0; pass < 2 && (int)R.size() < 4; ++pass) {
        for (int p = T - 1; p >= 0 && (int)R.size() < 4; --p) {
            if (std::find(R.begin(), R.end(), p) != R.end()) continue;
            if (pass == 0 && conflicts(p)) continue;
            R.push_back(p);
        }
    }
}

static std::vector<PlanStep> plan(const std::vector<GateOp> &gops, int n, int T,
                                  const std::vector<int> &order_idx) {
    const int m = T - 4;
    std::vector<PlanStep> steps;
    const int G = (int)order_idx.size();
    std::vector<char> done(G, 0);
    std::vector<uint64_t> bits(G);
    std::vector<int> nb(G);
    for (int i = 0; i < G; ++i) {
        bits[i] = op_bits(gops[order_idx[i]]);
        nb[i] = popc(bits[i]);
    }
    int remaining = G, first = 0;
    while (remaining > 0) {
        while (first < G && done[first]) ++first;
        // Best window.
        int best_h = -1, best_cnt = 0;
        for (int h = 4; h + m <= n; ++h) {
            const uint64_t W = window_mask(h, m);
            uint64_t blocked = 0;
            int cnt = 0;
            for (int i = first; i < G; ++i) {
                if (done[i]) continue;
                if ((bits[i] & ~W) == 0 && (bits[i] & blocked) == 0 &&
                    !gops[order_idx[i]].renorm && nb[i] <= 4) {
                    ++cnt;
                } else {
                    // A renormalising gate is a barrier for every bit.
                    blocked |= gops[order_idx[i]].renorm ? ~0ull : bits[i];
                    if ((blocked & ((1ull << n) - 1)) == ((1ull << n) - 1)) break;
                }
            }
            if (cnt > best_cnt) {
                best_cnt = cnt;
                best_h = h;
            }
        }
        if (best_cnt == 0) {
            PlanStep st;
            st.fused = false;
            st.gate = order_idx[first];
            steps.push_back(st);
            done[first] = 1;
            --remaining;
            continue;
        }
        PlanStep st;
        st.fused = true;
        st.pass.h = best_h;
        const uint64_t W = window_mask(best_h, m);
        uint64_t blocked = 0;
        for (int i = first; i < G; ++i) {
            if (done[i]) continue;
            if ((bits[i] & ~W) == 0 && (bits[i] & blocked) == 0 && !gops[order_idx[i]].renorm &&
                nb[i] <= 4) {
                st.pass.gates.push_back(order_idx[i]);
                done[i] = 1;
                --remaining;
            } else {
                blocked |= gops[order_idx[i]].renorm ? ~0ull : bits[i];
            }
        }
        // Rounds.
        const int P = (int)st.pass.gates.size();
        std::vector<char> sched(P, 0);
        std::vector<uint64_t> lb(P);
        for (int k = 0; k < P; ++k) {
            const uint64_t gb = op_bits(gops[st.pass.gates[k]]);
            uint64_t l = 0;
            for (int b = 0; b < n; ++b)
                if (gb >> b & 1) l |= 1ull << local_pos(b, best_h);
            lb[k] = l;
        }
        int left = P;
        while (left > 0) {
            PlannedRound rd;
            uint64_t R = 0, blk = 0;
            for (int k = 0; k < P; ++k) {
                if (sched[k]) continue;
                if ((lb[k] & blk) == 0 && popc(R | lb[k]) <= 4) {
                    R |= lb[k];
                    rd.ops.push_back(k);
                    sched[k] = 1;
                    --left;
                } else {
                    blk |= lb[k];
                }
            }
            std::vector<int> Rv;
            for (int p = 0; p < T; ++p)
                if (R >> p & 1) Rv.push_back(p);
            pad_rpos(Rv, T);
            for (int k = 0; k < 4; ++k) rd.rpos[k] = Rv[k];
            st.pass.rounds.push_back(rd);
        }
        steps.push_back(st);
    }
    return steps;
}

// Encode one gate (already part of a round with register positions rpos) as a
// register op.  lbit(b) maps a global bit to its register index.
static void encode_op(const GateOp &g, int h, const int rpos[4], std::vector<FusedOp> &fops,
                      std::vector<double> &coef) {
    auto reg = [&](int b) {
        const int lp = local_pos(b, h);
        for (int k = 0; k < 4; ++k)
            if (rpos[k] == lp) return k;
        return -1;
    };
    FusedOp f{};
    f.coef = (int)coef.size();
    switch (g.type) {
    case OP_M1:
    case OP_PERM1:
        f.type = g.type == OP_M1 ? F_M1 : F_PERM1;
        f.k0 = reg(g.t);
        f.cm = 0;
        for (int c = 0; c < g.nctrl; ++c) f.cm |= 1 << reg(g.ctrl[c]);
        if (g.type == OP_M1) coef.insert(coef.end(), g.m, g.m + 8);
        break;
    case OP_DIAG:
        f.type = F_DIAG;
        f.npat = g.npat;
        f.k0 = g.npat > 0 ? reg(g.pat[0]) : 0;
        f.k1 = g.npat > 1 ? reg(g.pat[1]) : 0;
        f.cm = 0;
        for (int c = 0; c < g.nfix; ++c) f.cm |= 1 << reg(g.fix[c]);
        coef.insert(coef.end(), g.m, g.m + 8);
        break;
    case OP_SWAP:
        f.type = F_SWAP;
        f.k0 = reg(g.b0);
        f.k1 = reg(g.b1);
        break;
    case OP_M2:
        f.type = F_M2;
        f.k0 = reg(g.b0);
        f.k1 = reg(g.b1);
        coef.insert(coef.end(), g.m, g.m + 32);
        break;
    }
    fops.push_back(f);
}

struct PassLaunch {
    int h;
    int round_begin, nrounds;
    bool extended;  // holds 4x4 ops: needs the extended kernel variant
};

int apply_circuit_impl(lq_state *s, const lq_gate *ops, int nops, const double *theta,
                       int ntheta, int mode) {
    const int n = s->n;
    s->last_launches = 0;
    s->last_passes = 0;
    std::vector<GateOp> gops(nops);
    for (int i = 0; i < nops; ++i) {
        LQ_TRY(validate_gate(&ops[i], n, ntheta));
        LQ_TRY(make_gate_op(&ops[i], theta, n, &gops[i]));
    }
    const bool can_fuse = mode == LQ_EXEC_FUSED && s->dtype == LQ_C128 && n >= 5;
    if (!can_fuse) {
        for (int i = 0; i < nops; ++i) {
            LQ_TRY(launch_gate_op(s, gops[i]));
            s->last_launches += gops[i].renorm ? 3 : 1;
        }
        return LQ_OK;
    }
    const int T = std::min(kMaxT, n);
    const int m = T - 4;
    std::vector<int> order(nops);
    for (int i = 0; i < nops; ++i) order[i] = i;
    std::vector<PlanStep> steps = plan(gops, n, T, order);

    // Encode every fused pass into one device program.
    std::vector<FusedRound> rounds;
    std::vector<FusedOp> fops;
    std::vector<double> coef;
    std::vector<PassLaunch> launches;
    for (auto &st : steps) {
        if (!st.fused) continue;
        PassLaunch pl{st.pass.h, (int)rounds.size(), (int)st.pass.rounds.size(), false};
        for (auto &rd : st.pass.rounds) {
            FusedRound fr{};
            for (int k = 0; k < 4; ++k) fr.rpos[k] = rd.rpos[k];
            fr.nlane = choose_lanes(rd.rpos, T, fr.lane);
            fr.op_begin = (int)fops.size();
            for (int k : rd.ops) {
                encode_op(gops[st.pass.gates[k]], st.pass.h, rd.rpos, fops, coef);
                if (fops.back().type == F_M2) pl.extended = true;
            }
            fr.op_end = (int)fops.size();
            rounds.push_back(fr);
        }
        launches.push_back(pl);
    }
    const size_t rb = rounds.size() * sizeof(FusedRound);
    const size_t ob = fops.size() * sizeof(FusedOp);
    const size_t cb = coef.size() * sizeof(double);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    LQ_TRY(ensure_prog(s, al(rb) + al(ob) + al(cb) + 256));
    char *dp = (char *)s->d_prog;
    FusedRound *d_rounds = (FusedRound *)dp;
    FusedOp *d_ops = (FusedOp *)(dp + al(rb));
    double *d_coef = (double *)(dp + al(rb) + al(ob));
    // The program buffer may still be read by a previous call's kernels.
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (rb) LQ_CUDA_TRY(cudaMemcpy(d_rounds, rounds.data(), rb, cudaMemcpyHostToDevice));
    if (ob) LQ_CUDA_TRY(cudaMemcpy(d_ops, fops.data(), ob, cudaMemcpyHostToDevice));
    if (cb) LQ_CUDA_TRY(cudaMemcpy(d_coef, coef.data(), cb, cudaMemcpyHostToDevice));

    static bool attr_set = false;
    const size_t smem = (16u << T) + 2048;
    if (!attr_set) {
        LQ_CUDA_TRY(cudaFuncSetAttribute(k_fused_pass<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (16 << kMaxT) + 2048));
        LQ_CUDA_TRY(cudaFuncSetAttribute(k_fused_pass<true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (16 << kMaxT) + 2048));
        attr_set = true;
    }
    size_t li = 0;
    for (auto &st : steps) {
        if (!st.fused) {
            LQ_TRY(launch_gate_op(s, gops[st.gate]));
            s->last_launches += gops[st.gate].renorm ? 3 : 1;
            continue;
        }
        const PassLaunch &pl = launches[li++];
        CUtensorMap map;
        LQ_TRY(make_tile_map(&map, s->d, n, pl.h, m));
        TileCoords tc{pl.h - 4};
        const unsigned grid = 1u << (n - T);
        prof_begin(s->stream, kProfFused);
        if (pl.extended)
            k_fused_pass<true><<<grid, 1 << (T - 4), smem, s->stream>>>(
                map, T, tc, d_rounds + pl.round_begin, pl.nrounds, d_ops, d_coef, s->d_flag);
        else
            k_fused_pass<false><<<grid, 1 << (T - 4), smem, s->stream>>>(
                map, T, tc, d_rounds + pl.round_begin, pl.nrounds, d_ops, d_coef, s->d_flag);
        prof_end(s->stream, kProfFused);
        LQ_CUDA_TRY(cudaGetLastError());
        s->last_launches += 1;
        s->last_passes += 1;
    }
    return LQ_OK;
}

static int launch_single_round(lq_state *s, int h, const FusedRound &fr, const FusedOp &fo,
                               const std::vector<double> &coef) {
    const int n = s->n;
    const int T = std::min(kMaxT, n);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t cb = coef.size() * sizeof(double);
    LQ_TRY(ensure_prog(s, al(sizeof(FusedRound)) + al(sizeof(FusedOp)) + al(cb) + 256));
    char *dp = (char *)s->d_prog;
    FusedRound *d_rounds = (FusedRound *)dp;
    FusedOp *d_ops = (FusedOp *)(dp + al(sizeof(FusedRound)));
    double *d_coef = (double *)(dp + al(sizeof(FusedRound)) + al(sizeof(FusedOp)));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    LQ_CUDA_TRY(cudaMemcpy(d_rounds, &fr, sizeof(FusedRound), cudaMemcpyHostToDevice));
    LQ_CUDA_TRY(cudaMemcpy(d_ops, &fo, sizeof(FusedOp), cudaMemcpyHostToDevice));
    LQ_CUDA_TRY(cudaMemcpy(d_coef, coef.data(), cb, cudaMemcpyHostToDevice));
    LQ_CUDA_TRY(cudaFuncSetAttribute(k_fused_pass<true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (16 << kMaxT) + 2048));
    CUtensorMap map;
    LQ_TRY(make_tile_map(&map, s->d, n, h, T - 4));
    TileCoords tc{h - 4};
    k_fused_pass<true><<<1u << (n - T), 1 << (T - 4), (16u << T) + 2048, s->stream>>>(
        map, T, tc, d_rounds, 1, d_ops, d_coef, s->d_flag);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

int apply_block_impl(lq_state *s, int k, const int *qubits, const double *m) {
    const int n = s->n;
    if (k == 1) return lq_apply_matrix1(s, qubits[0], m);
    if (k == 2) return lq_apply_matrix2(s, qubits[0], qubits[1], m);
    if (s->dtype != LQ_C128)
        return set_error(LQ_ERR_UNSUPPORTED, "block gates on complex64 states use lq_tc_*");
    if (n < 5) return set_error(LQ_ERR_UNSUPPORTED, "block gates need at least 5 qubits");
    const int T = std::min(kMaxT, n), mm = T - 4;
    int lo = n, hi = -1;
    for (int j = 0; j < k; ++j) {
        const int b = n - 1 - qubits[j];
        if (b >= 4) {
            lo = std::min(lo, b);
            hi = std::max(hi, b);
        }
    }
    int h = 4;
    if (hi >= 0) {
        h = std::max(4, std::min(lo, n - mm));
        if (hi >= h + mm)
            return set_error(LQ_ERR_UNSUPPORTED,
                             "block qubits span more than %d index bits above bit 3", mm);
    }
    std::vector<int> Rv;
    for (int j = 0; j < k; ++j) Rv.push_back(local_pos(n - 1 - qubits[k - 1 - j], h));
    pad_rpos(Rv, T);
    FusedRound fr{};
    for (int j = 0; j < 4; ++j) fr.rpos[j] = Rv[j];
    fr.nlane = choose_lanes(fr.rpos, T, fr.lane);
    fr.op_begin = 0;
    fr.op_end = 1;
    FusedOp fo{};
    fo.type = k == 3 ? F_BLOCK3 : F_BLOCK4;
    fo.coef = 0;
    std::vector<double> coef(m, m + 2 * (1 << k) * (1 << k));
    return launch_single_round(s, h, fr, fo, coef);
}

}  // namespace lq

using namespace lq;

extern "C" {

int lq_apply_circuit(lq_state *s, int circuit_qubits, const lq_gate *ops, int nops,
                     const double *theta, int ntheta, int mode) {
    LQ_TRY(check_state(s));
    if (circuit_qubits != s->n)
        return set_error(LQ_ERR_QUBIT_MISMATCH,
                         "Circuit qubit count mismatch: circuit has %d, state has %d",
                         circuit_qubits, s->n);
    if (nops < 0 || (nops > 0 && !ops)) return set_error(LQ_ERR_INVALID_ARG, "bad op list");
    if (ntheta < 0 || (ntheta > 0 && !theta)) return set_error(LQ_ERR_INVALID_ARG, "bad theta");
    if (mode != LQ_EXEC_FUSED && mode != LQ_EXEC_PER_GATE)
        return set_error(LQ_ERR_INVALID_ARG, "unknown execution mode %d", mode);
    return apply_circuit_impl(s, ops, nops, theta, ntheta, mode);
}

int lq_apply_block(lq_state *s, int k, const int *qubits, const double *m) {
    LQ_TRY(check_state(s));
    if (k < 1 || k > 4 || !qubits || !m)
        return set_error(LQ_ERR_INVALID_ARG, "block gate needs 1..4 qubits and a matrix");
    for (int i = 0; i < k; ++i) {
        LQ_TRY(check_qubit(s, qubits[i]));
        for (int j = 0; j < i; ++j)
            if (qubits[i] == qubits[j]) return set_error(LQ_ERR_INVALID_ARG, "repeated qubit");
    }
    return apply_block_impl(s, k, qubits, m);
}

int lq_plan_circuit(int num_qubits, const lq_gate *ops, int nops, int *passes, int *rounds,
                    int *standalone) {
    if (nops < 0 || (nops > 0 && !ops)) return set_error(LQ_ERR_INVALID_ARG, "bad op list");
    if (num_qubits < 5 || num_qubits > 36)
        return set_error(LQ_ERR_UNSUPPORTED, "fused planning needs 5..36 qubits");
    std::vector<GateOp> gops(nops);
    for (int i = 0; i < nops; ++i) {
        LQ_TRY(validate_gate(&ops[i], num_qubits, 1 << 30));
        static const double zero_theta[1] = {0.0};
        // Angles do not change the plan; bound parameters read theta[0].
        lq_gate g = ops[i];
        for (int k = 0; k < 3; ++k) g.param[k] = -1;
        LQ_TRY(make_gate_op(&g, zero_theta, num_qubits, &gops[i]));
    }
    const int T = std::min(kMaxT, num_qubits);
    std::vector<int> order(nops);
    for (int i = 0; i < nops; ++i) order[i] = i;
    std::vector<PlanStep> steps = plan(gops, num_qubits, T, order);
    int p = 0, r = 0, s1 = 0;
    for (auto &st : steps) {
        if (st.fused) {
            ++p;
            r += (int)st.pass.rounds.size();
        } else {
            ++s1;
        }
    }
    if (passes) *passes = p;
    if (rounds) *rounds = r;
    if (standalone) *standalone = s1;
    return LQ_OK;
}

int lq_last_circuit_stats(const lq_state *s, int *launches, int *passes) {
    LQ_TRY(check_state(s));
    if (launches) *launches = s->last_launches;
    if (passes) *passes = s->last_passes;
    return LQ_OK;
}

}  // extern "C"
