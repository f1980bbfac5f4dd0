// Fused k-qubit block passes: Circuit::execute (src/circuits/mod.rs:352-375)
// without one full-state sweep per gate.
//
// A pass owns a window W of T <= 12 index bits: the four lowest bits (so every
// global access is a 256-byte contiguous run) plus a contiguous range
// [h, h+T-4).  One CTA per tile (2^T amplitudes, 32 KiB of complex128 at
// T = 11): the tile is staged from HBM into shared memory by one TMA tensor
// copy (128-byte swizzle), every gate of the pass is applied, and the tile
// goes back by a TMA store.  HBM traffic per pass is one read and one write of
// the state, however many gates the pass holds.
//
// Inside the CTA the gates run in "rounds" (fused_core.cuh): a round picks four
// tile bits R, each thread gathers the 16 amplitudes that differ only in R
// into registers, applies the round's gates there, and scatters them back.
// Only the bits a gate mixes or permutes (its target; both bits of a SWAP or
// 4x4) must be in R.  Control bits and every bit of a diagonal gate may lie
// anywhere -- in R, elsewhere in the tile (constant per thread during a round)
// or outside the window (constant per tile during the pass): their values are
// read from the thread's global basis index.  So CNOT controls, CPhase, CZ, RZ
// and RZZ fuse into any pass that holds their target (diagonal gates need none).
//
// The planner (host) picks windows greedily: at each step it chooses the h
// that lets the most not-yet-applied gates run (respecting gate order per
// bit), then splits that pass into register rounds.  Gates whose mixed bits fit
// no window (a SWAP or 4x4 on bits further apart than the window) and gates
// that renormalise run as standalone per-gate sweeps at their place in order.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <complex>
#include <memory>
#include <mutex>

#include "fused_plan.h"
#include "fused_round.cuh"

namespace lq {

static std::atomic<int> g_fusion_width{11};
int fusion_width() { return g_fusion_width.load(); }

struct TileCoords {
    int32_t h;       // window range start (bits h .. h+m-1), h >= 4
    int32_t hm;      // h + m
    int32_t ntiles;  // 2^(n-T)
};

// One CTA per tile.  blockDim.x = 2^(T-4); dynamic smem = 2^T * 16 + 2048.
// (Measured on B200: more resident CTAs per SM beat a persistent,
// double-buffered CTA here, because the register-resident gate math needs the
// warps to hide FP64 latency more than it needs load/compute overlap.)
// MODE selects the op set: 0 = 2x2 / X / diagonal / swap, 1 = also 4x4 ops,
// 2 = also 8x8 / 16x16 block ops (more registers per mode).
template <int MODE>
__device__ __forceinline__ void fused_pass_body(const CUtensorMap &tmap, int T, TileCoords tc,
                                                const FusedRound *__restrict__ rounds,
                                                int nrounds, const FusedOp *__restrict__ ops,
                                                const double *__restrict__ coef,
                                                unsigned *__restrict__ flag) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t tile_bytes = 16u << T;
    uint64_t *bar = (uint64_t *)(base + tile_bytes);
    const uint32_t tile_a = smem_u32(base);
    const uint32_t bar_a = smem_u32(bar);
    const int tid = threadIdx.x;
    const int32_t zero = 0;
    const int tile = blockIdx.x;
    const int32_t c2 = tile & ((1 << (tc.h - 4)) - 1), c4 = tile >> (tc.h - 4);

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_a), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a),
                     "r"(tile_bytes)
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
    const uint64_t tile_base = ((uint64_t)c2 << 4) | ((uint64_t)c4 << tc.hm);
    auto coef_of = [&](const FusedOp &op) { return coef + op.coef; };
    for (int r = 0; r < nrounds; ++r) {
        run_round<MODE>(tile_a, rounds[r], ops, coef_of, tile_base, tc.h, tid);
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

// 256-thread tiles (T = 12): two CTAs per SM at 128 registers.
template <int MODE>
__global__ void __launch_bounds__(256, 2)
    k_fused_pass(const __grid_constant__ CUtensorMap tmap, int T, TileCoords tc,
                 const FusedRound *__restrict__ rounds, int nrounds,
                 const FusedOp *__restrict__ ops, const double *__restrict__ coef,
                 unsigned *__restrict__ flag) {
    fused_pass_body<MODE>(tmap, T, tc, rounds, nrounds, ops, coef, flag);
}

// 64- and 128-thread tiles (T <= 11): 168 registers per thread keep the
// register rounds free of spills; measured faster than 128 registers with more
// resident CTAs (30-qubit brickwork at T = 10: 668 vs 704 ms per step).
template <int MODE>
__global__ void __maxnreg__(168)
    k_fused_pass_narrow(const __grid_constant__ CUtensorMap tmap, int T, TileCoords tc,
                        const FusedRound *__restrict__ rounds, int nrounds,
                        const FusedOp *__restrict__ ops, const double *__restrict__ coef,
                        unsigned *__restrict__ flag) {
    fused_pass_body<MODE>(tmap, T, tc, rounds, nrounds, ops, coef, flag);
}

// Ping-pong register rounds (fused_round.cuh) over compact PassOp records;
// one CTA per tile, as k_fused_pass_narrow.
// Row length of the per-round thread-base table: the thread count, at least 8
// entries (16 bytes) so every row starts 16-byte aligned.
__host__ __device__ __forceinline__ int tb_stride(int nthreads) {
    return nthreads < 8 ? 8 : nthreads;
}

template <int MODE>
__device__ __forceinline__ void fused_pp_body(const CUtensorMap &tmap, int T, TileCoords tc,
                                              const FusedRound *__restrict__ rounds, int nrounds,
                                              const PassOp *__restrict__ ops,
                                              const double *__restrict__ coef,
                                              const uint16_t *__restrict__ tbtab,
                                              unsigned *__restrict__ flag) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t tile_bytes = 16u << T;
    uint64_t *bar = (uint64_t *)(base + tile_bytes);
    const uint32_t tile_a = smem_u32(base);
    const uint32_t bar_a = smem_u32(bar);
    const int tid = threadIdx.x;
    const int32_t zero = 0;
    const int tile = blockIdx.x;
    const int32_t c2 = tile & ((1 << (tc.h - 4)) - 1), c4 = tile >> (tc.h - 4);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_a), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a),
                     "r"(tile_bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(tile_a),
            "l"((uint64_t)&tmap), "r"(zero), "r"(zero), "r"(c2), "r"(zero), "r"(c4), "r"(bar_a)
            : "memory");
    }
    if (!mbar_wait(bar_a, 0)) {
        // leave only once the load no longer targets this CTA's shared memory
        if (tid == 0) {
            atomicOr(flag, kFlagTimeout);
            mbar_wait(bar_a, 0);
        }
        return;
    }
    const uint64_t tile_base = ((uint64_t)c2 << 4) | ((uint64_t)c4 << tc.hm);
    for (int r = 0; r < nrounds; ++r) {
        const int tbase = tbtab[r * tb_stride((int)blockDim.x) + tid];
        run_round_pp<MODE>(tile_a, rounds[r], ops, coef, tile_base, tc.h, tbase);
        __syncthreads();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
        asm volatile(
            "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group"
            " [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"((uint64_t)&tmap),
            "r"(zero), "r"(zero), "r"(c2), "r"(zero), "r"(c4), "r"(tile_a)
            : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        // shared memory is released when the CTA exits: the store must have read it
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
}

template <int MODE>
__global__ void __launch_bounds__(256, 1)
    k_fused_pp(const __grid_constant__ CUtensorMap tmap, int T, TileCoords tc,
               const FusedRound *__restrict__ rounds, int nrounds, const PassOp *__restrict__ ops,
               const double *__restrict__ coef, const uint16_t *__restrict__ tbtab,
               unsigned *__restrict__ flag) {
    fused_pp_body<MODE>(tmap, T, tc, rounds, nrounds, ops, coef, tbtab, flag);
}

// 168 registers: six 64-thread CTAs per SM at tile bits 10.  Measured on a
// 30-qubit brickwork: 481 ms per step at 168 registers (a few spills outside
// the hot ops), 540 at 192, 518 at 240 -- resident warps matter more than the
// last registers.
#ifndef LQ_PP_MAXNREG
#define LQ_PP_MAXNREG 168
#endif
template <int MODE>
__global__ void __maxnreg__(LQ_PP_MAXNREG)
    k_fused_pp_narrow(const __grid_constant__ CUtensorMap tmap, int T, TileCoords tc,
                      const FusedRound *__restrict__ rounds, int nrounds,
                      const PassOp *__restrict__ ops, const double *__restrict__ coef,
                      const uint16_t *__restrict__ tbtab, unsigned *__restrict__ flag) {
    fused_pp_body<MODE>(tmap, T, tc, rounds, nrounds, ops, coef, tbtab, flag);
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
static inline int popc(uint64_t x) { return __builtin_popcountll(x); }

// Bits an op mixes or permutes (they must sit in the register set R).
static uint64_t reg_bits(const GateOp &o) {
    switch (o.type) {
    case OP_M1:
    case OP_PERM1: return 1ull << o.t;
    case OP_SWAP:
    case OP_M2: return (1ull << o.b0) | (1ull << o.b1);
    default: {  // diagonal: free, unless it is a table factor of a real 4x4
        uint64_t m = 0;
        if (o.table)
            for (int k = 0; k < o.npat; ++k) m |= 1ull << o.pat[k];
        return m;
    }
    }
}

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

// ---------------------------------------------------------------------------
// Pair folding: (U_x (x) U_y) followed by a two-qubit gate G on bits (x, y)
// becomes ONE 4x4 op G (U_x (x) U_y).  In a U3 + CNOT layer this replaces two
// 2x2 ops and a register permutation by one 4x4 op with the same FP64 work
// and a third of the op overhead.  Runs of single-qubit gates on one bit are
// merged first.  Host FP64 products; only the fused path folds.
// ---------------------------------------------------------------------------

// Amplitude map of op g restricted to index bits {bx (hi), by (lo)} (other
// bits 0, or g touches only these): out[r*4+c] = <r| g |c>, complex.
static bool op_matrix4(const GateOp &g, int bx, int by, std::complex<double> out[16]) {
    auto bit_of = [&](int v, int b) -> int { return b == bx ? (v >> 1) & 1 : b == by ? v & 1 : -1; };
    for (int c = 0; c < 4; ++c) {
        std::complex<double> col[4] = {0, 0, 0, 0};
        switch (g.type) {
        case OP_M1:
        case OP_PERM1: {
            bool on = true;
            for (int k = 0; k < g.nctrl; ++k) {
                const int v = bit_of(c, g.ctrl[k]);
                if (v < 0) return false;
                on = on && v == 1;
            }
            const int tv = bit_of(c, g.t);
            if (tv < 0) return false;
            if (!on) {
                col[c] = 1.0;
                break;
            }
            const int tmask = g.t == bx ? 2 : 1;
            const int c0 = c & ~tmask, c1 = c | tmask;
            if (g.type == OP_PERM1) {
                col[c ^ tmask] = 1.0;
            } else {
                // column tv of the 2x2 goes to rows (t = 0, t = 1)
                col[c0] = {g.m[(0 * 2 + tv) * 2], g.m[(0 * 2 + tv) * 2 + 1]};
                col[c1] = {g.m[(1 * 2 + tv) * 2], g.m[(1 * 2 + tv) * 2 + 1]};
            }
            break;
        }
        case OP_DIAG: {
            bool on = true;
            for (int k = 0; k < g.nfix; ++k) {
                const int v = bit_of(c, g.fix[k]);
                if (v < 0) return false;
                on = on && v == 1;
            }
            int pat = 0;
            for (int k = 0; k < g.npat; ++k) {
                const int v = bit_of(c, g.pat[k]);
                if (v < 0) return false;
                pat |= v << k;
            }
            col[c] = on ? std::complex<double>(g.m[2 * pat], g.m[2 * pat + 1]) : 1.0;
            break;
        }
        case OP_SWAP: {
            if (bit_of(c, g.b0) < 0 || bit_of(c, g.b1) < 0) return false;
            const int v0 = bit_of(c, g.b0), v1 = bit_of(c, g.b1);
            int r = 0;
            r |= (g.b0 == bx ? v1 : v0) << 1;  // bit bx takes the value of its partner
            r |= (g.b0 == bx ? v0 : v1);
            col[r] = 1.0;
            break;
        }
        case OP_M2: {
            // M2 index = (bit b0) << 1 | (bit b1)
            if (bit_of(c, g.b0) < 0 || bit_of(c, g.b1) < 0) return false;
            const int ci = (bit_of(c, g.b0) << 1) | bit_of(c, g.b1);
            for (int ri = 0; ri < 4; ++ri) {
                const int vb0 = (ri >> 1) & 1, vb1 = ri & 1;
                const int r = ((g.b0 == bx ? vb0 : vb1) << 1) | (g.b0 == bx ? vb1 : vb0);
                col[r] = {g.m[(ri * 4 + ci) * 2], g.m[(ri * 4 + ci) * 2 + 1]};
            }
            break;
        }
        default: return false;
        }
        for (int r = 0; r < 4; ++r) out[r * 4 + c] = col[r];
    }
    return true;
}

// 2x2 of an uncontrolled single-qubit op and its bit; false for anything else.
static bool single_matrix(const GateOp &g, int &bit, std::complex<double> u[4]) {
    if (g.renorm) return false;
    if ((g.type == OP_M1 || g.type == OP_PERM1) && g.nctrl == 0) {
        bit = g.t;
        if (g.type == OP_M1)
            for (int k = 0; k < 4; ++k) u[k] = {g.m[2 * k], g.m[2 * k + 1]};
        else
            u[0] = 0.0, u[1] = 1.0, u[2] = 1.0, u[3] = 0.0;
        return true;
    }
    if (g.type == OP_DIAG && g.nfix == 0 && g.npat == 1) {
        bit = g.pat[0];
        u[0] = {g.m[0], g.m[1]}, u[1] = 0.0, u[2] = 0.0, u[3] = {g.m[2], g.m[3]};
        return true;
    }
    return false;
}

// ---------------------------------------------------------------------------
// Real folding.  Every 2x2 unitary has the Euler form of U3
// (src/gates/parameterized.rs:249-282):
//     U = w * diag(1, dphi) * [[c, -s], [s, c]] * diag(1, dlam),   c, s >= 0,
// so a folded pair G (U_x (x) U_y) with G a permutation times phases (CNOT,
// SWAP, CZ, CPhase, ...) becomes
//     D_out * (P * (R_x (x) R_y)) * D_in
// with a REAL 4x4 in the middle (half the FP64 work of a complex 4x4) and two
// diagonals on the pair's bits.  The diagonals of a register round are merged
// on the host into one table per run (encode_round), so a brickwork layer
// costs about 8 + 4 FP64 instructions per amplitude and pair instead of 16.
// ---------------------------------------------------------------------------
static int real_fold_mode() {  // 0: complex 4x4; 1: real 4x4; 2: scaled rotations
    static const int v = [] {
        const char *e = getenv("LQ_REAL_FOLD");
        return e ? atoi(e) : 2;
    }();
    return v;
}
static bool real_fold_enabled() { return real_fold_mode() != 0; }

struct Euler2 {
    std::complex<double> w, dphi, dlam;
    double c, s;
};

static bool euler2(const std::complex<double> u[4], Euler2 &e) {
    using cd = std::complex<double>;
    const cd a = u[0], b = u[1], cc = u[2], d = u[3];
    const double ra = std::abs(a), rb = std::abs(b), rc = std::abs(cc), rd = std::abs(d);
    if (std::abs(ra * ra + rc * rc - 1.0) > 1e-12 || std::abs(rb - rc) > 1e-12 ||
        std::abs(ra - rd) > 1e-12)
        return false;  // not unitary (e.g. a user matrix): keep the complex form
    constexpr double tiny = 1e-150;
    e.c = ra;
    e.s = rc;
    e.w = ra > tiny ? a / ra : cd(1.0, 0.0);
    if (rc > tiny && rb > tiny) {
        e.dphi = (cc / rc) * std::conj(e.w);
        e.dlam = (-b / rb) * std::conj(e.w);
    } else {
        e.dphi = 1.0;
        e.dlam = rd > tiny ? (d / rd) * std::conj(e.w) : cd(1.0, 0.0);
    }
    const cd r[4] = {e.w * e.c, -e.w * e.s * e.dlam, e.w * e.s * e.dphi,
                     e.w * e.c * e.dphi * e.dlam};
    for (int k = 0; k < 4; ++k)
        if (std::abs(r[k] - u[k]) > 1e-14) return false;
    return true;
}

// G is a permutation times phases: column c has its one non-zero in row p[c].
static bool monomial4(const std::complex<double> G[16], int p[4], std::complex<double> g[4]) {
    int used = 0;
    for (int c = 0; c < 4; ++c) {
        int row = -1;
        for (int r = 0; r < 4; ++r) {
            if (G[r * 4 + c] == std::complex<double>(0.0, 0.0)) continue;
            if (row >= 0) return false;
            row = r;
        }
        if (row < 0 || (used >> row & 1)) return false;
        used |= 1 << row;
        p[c] = row;
        g[c] = G[row * 4 + c];
    }
    return true;
}

// Scaled rotation op on bit b: R = [[c, -s], [s, c]] = sigma * R' with R' one
// FMA per component (form 0: c >= s, x = s/c, sigma = c; form 1: x = c/s,
// sigma = s).
constexpr double kMinScaledCos = 1e-3;

static GateOp scaled_rotation(int b, double c, double s, double &sigma) {
    GateOp g{};
    g.type = OP_M1;
    g.t = b;
    g.srot = true;
    double r[4];
    if (c >= kMinScaledCos) {  // x = s / c <= 1000: still one FMA per component
        const double x = s / c;
        g.sform = 0;
        sigma = c;
        r[0] = 1.0, r[1] = -x, r[2] = x, r[3] = 1.0;
    } else {
        const double x = c / s;
        g.sform = 1;
        sigma = s;
        r[0] = x, r[1] = -1.0, r[2] = 1.0, r[3] = x;
    }
    for (int k = 0; k < 4; ++k) g.m[2 * k] = r[k], g.m[2 * k + 1] = 0.0;
    return g;
}

// D_in, the real middle and D_out of G (U_x (x) U_y) on bits (bx hi, by lo),
// appended to out in time order; false when the pair does not have that form.
// Mode 2 writes the middle as two scaled rotations and the permutation (CNOT
// either way, SWAP or none) as register moves, with the rotations' scales in
// D_out; mode 1 (or any other permutation) writes it as one real 4x4.
static bool real_fold(const std::complex<double> G[16], const std::complex<double> ux[4],
                      const std::complex<double> uy[4], int bx, int by,
                      std::vector<GateOp> &out) {
    using cd = std::complex<double>;
    Euler2 ex, ey;
    int p[4];
    cd gv[4];
    if (!euler2(ux, ex) || !euler2(uy, ey) || !monomial4(G, p, gv)) return false;
    const double rx[4] = {ex.c, -ex.s, ex.s, ex.c}, ry[4] = {ey.c, -ey.s, ey.s, ey.c};
    const cd w = ex.w * ey.w;
    GateOp din{}, mid{}, dout{};
    din.type = dout.type = OP_DIAG;
    din.npat = dout.npat = 2;
    din.pat[0] = dout.pat[0] = by;  // pattern index = (bit bx) << 1 | (bit by)
    din.pat[1] = dout.pat[1] = bx;
    din.table = dout.table = true;
    for (int i = 0; i < 4; ++i) {
        const cd fi = (i & 2 ? ex.dlam : cd(1.0)) * (i & 1 ? ey.dlam : cd(1.0));
        din.m[2 * i] = fi.real();
        din.m[2 * i + 1] = fi.imag();
        const cd fo = gv[i] * (i & 2 ? ex.dphi : cd(1.0)) * (i & 1 ? ey.dphi : cd(1.0)) * w;
        dout.m[2 * p[i]] = fo.real();
        dout.m[2 * p[i] + 1] = fo.imag();
    }
    const int pc = p[0] | p[1] << 2 | p[2] << 4 | p[3] << 6;
    const int P_ID = 0 | 1 << 2 | 2 << 4 | 3 << 6, P_CX = 0 | 1 << 2 | 3 << 4 | 2 << 6,
              P_XC = 0 | 3 << 2 | 2 << 4 | 1 << 6, P_SW = 0 | 2 << 2 | 1 << 4 | 3 << 6;
    if (real_fold_mode() >= 2 && (pc == P_ID || pc == P_CX || pc == P_XC || pc == P_SW) &&
        ex.c >= kMinScaledCos && ey.c >= kMinScaledCos) {
        double sx, sy;
        const GateOp rxo = scaled_rotation(bx, ex.c, ex.s, sx);
        const GateOp ryo = scaled_rotation(by, ey.c, ey.s, sy);
        for (int i = 0; i < 8; ++i) dout.m[i] *= sx * sy;
        out.push_back(din);
        if (real_fold_mode() == 3) {  // separate ops (kept for measurement)
            out.push_back(rxo);
            out.push_back(ryo);
            if (pc == P_CX || pc == P_XC) {
                GateOp cx{};
                cx.type = OP_PERM1;
                cx.t = pc == P_CX ? by : bx;
                cx.nctrl = 1;
                cx.ctrl[0] = pc == P_CX ? bx : by;
                out.push_back(cx);
            } else if (pc == P_SW) {
                GateOp sw{};
                sw.type = OP_SWAP;
                sw.b0 = bx;
                sw.b1 = by;
                out.push_back(sw);
            }
        } else {  // one op: both rotations and the permutation
            GateOp pr{};
            pr.type = OP_M2;
            pr.real4 = true;
            pr.pairrot = true;
            pr.b0 = bx;
            pr.b1 = by;
            pr.px[0] = rxo.sform == 0 ? rxo.m[4] : rxo.m[0];
            pr.px[1] = ryo.sform == 0 ? ryo.m[4] : ryo.m[0];
            pr.pf[0] = rxo.sform;
            pr.pf[1] = ryo.sform;
            pr.pperm = pc == P_ID ? 0 : pc == P_CX ? 1 : pc == P_XC ? 2 : 3;
            // the full real matrix P (R'x (x) R'y) for every other reader of the op
            for (int c = 0; c < 4; ++c)
                for (int k = 0; k < 4; ++k) {
                    const double v = rxo.m[2 * ((c >> 1) * 2 + (k >> 1))] *
                                     ryo.m[2 * ((c & 1) * 2 + (k & 1))];
                    pr.m[2 * (p[c] * 4 + k)] = v;
                    pr.m[2 * (p[c] * 4 + k) + 1] = 0.0;
                }
            out.push_back(pr);
        }
        out.push_back(dout);
        return true;
    }
    mid.type = OP_M2;
    mid.real4 = true;
    mid.b0 = bx;
    mid.b1 = by;
    for (int c = 0; c < 4; ++c)      // row p[c] of P R is row c of R = R_x (x) R_y
        for (int k = 0; k < 4; ++k) {
            mid.m[2 * (p[c] * 4 + k)] = rx[(c >> 1) * 2 + (k >> 1)] * ry[(c & 1) * 2 + (k & 1)];
            mid.m[2 * (p[c] * 4 + k) + 1] = 0.0;
        }
    out.push_back(din);
    out.push_back(mid);
    out.push_back(dout);
    return true;
}

static void fold_pairs(std::vector<GateOp> &gops, std::vector<int> &orig, int T) {
    struct Entry {
        GateOp op;
        int orig;
        bool dead;
        bool single;
        int bit;
        std::complex<double> u[4];
    };
    std::vector<Entry> out;
    std::vector<int> open(64, -1);  // per bit: the pending single-qubit entry
    for (size_t k = 0; k < gops.size(); ++k) {
        const GateOp &g = gops[k];
        Entry e{g, (int)k, false, false, -1, {}};
        int bit;
        std::complex<double> u[4];
        if (single_matrix(g, bit, u)) {
            if (open[bit] >= 0) {  // extend the run: U_run <- u . U_run
                Entry &r = out[open[bit]];
                std::complex<double> p[4] = {u[0] * r.u[0] + u[1] * r.u[2],
                                             u[0] * r.u[1] + u[1] * r.u[3],
                                             u[2] * r.u[0] + u[3] * r.u[2],
                                             u[2] * r.u[1] + u[3] * r.u[3]};
                const bool diag = r.op.type == OP_DIAG && g.type == OP_DIAG;
                GateOp m{};
                if (diag) {
                    m.type = OP_DIAG;
                    m.npat = 1;
                    m.pat[0] = bit;
                    m.m[0] = p[0].real(), m.m[1] = p[0].imag();
                    m.m[2] = p[3].real(), m.m[3] = p[3].imag();
                } else {
                    m.type = OP_M1;
                    m.t = bit;
                    for (int q = 0; q < 4; ++q) m.m[2 * q] = p[q].real(), m.m[2 * q + 1] = p[q].imag();
                }
                r.op = m;
                r.orig = -1;
                for (int q = 0; q < 4; ++q) r.u[q] = p[q];
                continue;
            }
            e.single = true;
            e.bit = bit;
            for (int q = 0; q < 4; ++q) e.u[q] = u[q];
            out.push_back(e);
            open[bit] = (int)out.size() - 1;
            continue;
        }
        const uint64_t bits = op_bits(g);
        if (!g.renorm && popc(bits) == 2) {
            const int bx = 63 - __builtin_clzll(bits), by = __builtin_ctzll(bits);
            std::complex<double> G[16];
            // both bits must fit one window [0,4) U [h, h+T-4) (else a standalone sweep)
            const bool fits = by < 4 || bx - by < T - 4;
            if (fits && open[bx] >= 0 && open[by] >= 0 && op_matrix4(g, bx, by, G)) {
                Entry &ex = out[open[bx]], &ey = out[open[by]];
                // M = G . (U_x (x) U_y), index (bit bx) << 1 | (bit by)
                std::complex<double> K[16], M[16];
                for (int r = 0; r < 4; ++r)
                    for (int c = 0; c < 4; ++c)
                        K[r * 4 + c] = ex.u[(r >> 1) * 2 + (c >> 1)] * ey.u[(r & 1) * 2 + (c & 1)];
                for (int r = 0; r < 4; ++r)
                    for (int c = 0; c < 4; ++c) {
                        std::complex<double> s = 0.0;
                        for (int q = 0; q < 4; ++q) s += G[r * 4 + q] * K[q * 4 + c];
                        M[r * 4 + c] = s;
                    }
                ex.dead = ey.dead = true;
                std::vector<GateOp> rf;
                if (real_fold_enabled() && real_fold(G, ex.u, ey.u, bx, by, rf)) {
                    for (const GateOp &q : rf) out.push_back(Entry{q, -1, false, false, -1, {}});
                    open[bx] = open[by] = -1;
                    continue;
                }
                GateOp m{};
                m.type = OP_M2;
                m.b0 = bx;
                m.b1 = by;
                for (int q = 0; q < 16; ++q) m.m[2 * q] = M[q].real(), m.m[2 * q + 1] = M[q].imag();
                out.push_back(Entry{m, -1, false, false, -1, {}});
                open[bx] = open[by] = -1;
                continue;
            }
        }
        for (int b = 0; b < 64; ++b)
            if ((bits >> b) & 1) open[b] = -1;
        out.push_back(e);
    }
    gops.clear();
    orig.clear();
    for (auto &e : out) {
        if (e.dead) continue;
        gops.push_back(e.op);
        orig.push_back(e.orig);
    }
}

std::vector<PlanStep> plan_circuit(const std::vector<GateOp> &gops, int n, int T) {
    const int m = T - 4;
    std::vector<PlanStep> steps;
    const int G = (int)gops.size();
    const uint64_t all = (1ull << n) - 1;
    std::vector<char> done(G, 0);
    std::vector<uint64_t> bits(G), rbits(G);
    std::vector<char> fusable(G);
    for (int i = 0; i < G; ++i) {
        bits[i] = op_bits(gops[i]);
        rbits[i] = reg_bits(gops[i]);
        fusable[i] = !gops[i].renorm && popc(rbits[i]) <= 4;
    }
    int remaining = G, first = 0;
    while (remaining > 0) {
        while (first < G && done[first]) ++first;
        int best_h = -1, best_cnt = 0;
        for (int h = 4; h + m <= n; ++h) {
            const uint64_t W = window_mask(h, m);
            uint64_t blocked = 0;
            int cnt = 0;
            for (int i = first; i < G; ++i) {
                if (done[i]) continue;
                if (fusable[i] && (rbits[i] & ~W) == 0 && (bits[i] & blocked) == 0) {
                    ++cnt;
                } else {
                    // A renormalising gate is a barrier for every bit.
                    blocked |= gops[i].renorm ? all : bits[i];
                    if ((blocked & all) == all) break;
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
            st.gate = first;
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
            if (fusable[i] && (rbits[i] & ~W) == 0 && (bits[i] & blocked) == 0) {
                st.pass.gates.push_back(i);
                done[i] = 1;
                --remaining;
            } else {
                blocked |= gops[i].renorm ? all : bits[i];
                if ((blocked & all) == all) break;
            }
        }
        // Rounds: greedy, in order; an op joins the round if it is not blocked by
        // an earlier unscheduled op sharing a bit and its register bits fit R.
        const int P = (int)st.pass.gates.size();
        std::vector<char> sched(P, 0);
        std::vector<uint64_t> lreg(P), gall(P);
        for (int k = 0; k < P; ++k) {
            const int i = st.pass.gates[k];
            uint64_t l = 0;
            for (int b = 0; b < n; ++b)
                if (rbits[i] >> b & 1) l |= 1ull << local_pos(b, best_h);
            lreg[k] = l;
            gall[k] = bits[i];
        }
        int left = P;
        while (left > 0) {
            PlannedRound rd;
            uint64_t R = 0, blk = 0;
            for (int k = 0; k < P; ++k) {
                if (sched[k]) continue;
                if ((gall[k] & blk) == 0 && popc(R | lreg[k]) <= 4) {
                    R |= lreg[k];
                    rd.ops.push_back(k);
                    sched[k] = 1;
                    --left;
                } else {
                    blk |= gall[k];
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

void fill_round(FusedRound &fr, const int rpos[4], int T, int h) {
    for (int e = 0; e < 16; ++e) {
        int off = 0;
        for (int k = 0; k < 4; ++k)
            if (e >> k & 1) off |= 1 << rpos[k];
        fr.eoff[e] = swz(off) << 4;
    }
    for (int k = 0; k < 4; ++k) fr.gpos[k] = 1ull << global_pos(rpos[k], h);
    fr.nlane = choose_lanes(rpos, T, fr.lane);
}

void encode_op(const GateOp &g, int h, int m, const int rpos[4], std::vector<FusedOp> &fops,
               std::vector<double> &coef) {
    auto reg = [&](int b) {
        if (!(b < 4 || (b >= h && b < h + m))) return -1;  // outside the window
        const int lp = local_pos(b, h);
        for (int k = 0; k < 4; ++k)
            if (rpos[k] == lp) return k;
        return -1;
    };
    FusedOp f{};
    f.coef = (int)coef.size();
    f.pb0 = f.pb1 = -1;
    f.param = f.param2 = -1;
    f.coef_alt = f.coef_alt2 = -1;
    switch (g.type) {
    case OP_M1:
    case OP_PERM1: {
        f.k0 = reg(g.t);
        f.cm = 0;
        f.gmask = 0;
        for (int c = 0; c < g.nctrl; ++c) {
            const int k = reg(g.ctrl[c]);
            if (k >= 0) f.cm |= 1 << k;
            else f.gmask |= 1ull << g.ctrl[c];
        }
        if (g.type == OP_M1 && g.srot && f.cm == 0 && f.gmask == 0) {
            f.type = F_R1S;
            f.k1 = g.sform;
            coef.push_back(g.sform == 0 ? g.m[4] : g.m[0]);  // x of the form
            coef.insert(coef.end(), 7, 0.0);
        } else if (g.type == OP_M1) {
            f.type = f.cm ? F_M1C : F_M1;
            coef.insert(coef.end(), g.m, g.m + 8);
        } else {
            f.type = f.cm ? F_XC : F_X;
            coef.insert(coef.end(), 8, 0.0);
        }
        break;
    }
    case OP_DIAG:
        f.type = F_DIAG;
        f.npat = g.npat;
        f.pb0 = g.npat > 0 ? g.pat[0] : -1;
        f.pb1 = g.npat > 1 ? g.pat[1] : -1;
        f.fixmask = 0;
        for (int c = 0; c < g.nfix; ++c) f.fixmask |= 1ull << g.fix[c];
        coef.insert(coef.end(), g.m, g.m + 8);
        break;
    case OP_SWAP:
        f.type = F_SWAP;
        f.k0 = reg(g.b0);
        f.k1 = reg(g.b1);
        coef.insert(coef.end(), 8, 0.0);
        break;
    case OP_M2: {
        if (g.pairrot) {
            // F_PAIR: k0 < k1; the op's bit b0 is index bit 1 of its permutation
            int kb0 = reg(g.b0), kb1 = reg(g.b1);
            int f0 = g.pf[0], f1 = g.pf[1], perm = g.pperm;
            double x0 = g.px[0], x1 = g.px[1];
            if (kb0 > kb1) {  // roles swap: CNOT directions swap, SWAP / none stay
                std::swap(kb0, kb1);
                std::swap(f0, f1);
                std::swap(x0, x1);
                if (perm == 1 || perm == 2) perm = 3 - perm;
            }
            f.type = F_PAIR;
            f.k0 = kb0;
            f.k1 = kb1;
            f.cm = f0 | f1 << 1 | perm << 2;
            coef.push_back(x0);
            coef.push_back(x1);
            coef.insert(coef.end(), 6, 0.0);
            break;
        }
        // register bits ordered k0 < k1 (the kernel unrolls only those pairs):
        // swapping the bits swaps the two bits of the 4x4 row / column index
        const bool real = g.real4;
        f.type = real ? F_M2R : F_M2;
        int k0 = reg(g.b0), k1 = reg(g.b1);
        int sw[4] = {0, 1, 2, 3};
        if (k0 > k1) {
            std::swap(k0, k1);
            sw[1] = 2;
            sw[2] = 1;
        }
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) {
                coef.push_back(g.m[(sw[r] * 4 + sw[c]) * 2]);
                if (!real) coef.push_back(g.m[(sw[r] * 4 + sw[c]) * 2 + 1]);
            }
        f.k0 = k0;
        f.k1 = k1;
        break;
    }
    }
    fops.push_back(f);
}

struct PassLaunch {
    int h;
    int round_begin, nrounds;
    int mode;  // kernel op set the pass needs (k_fused_pass MODE)
};

static size_t fused_smem(int T) { return (16u << T) + 2048; }

static int fused_grid(int T, int ntiles) {
    (void)T;
    return ntiles;
}

static int set_smem_attrs() {
    static bool done = false;
    if (done) return LQ_OK;
    const int mx = (int)fused_smem(kMaxT);
    LQ_CUDA_TRY(cudaFuncSetAttribute(k_fused_pass<0>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    LQ_CUDA_TRY(cudaFuncSetAttribute(k_fused_pass<1>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    LQ_CUDA_TRY(cudaFuncSetAttribute(k_fused_pass<2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    LQ_CUDA_TRY(cudaFuncSetAttribute(k_fused_pass_narrow<0>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    LQ_CUDA_TRY(cudaFuncSetAttribute(k_fused_pass_narrow<1>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    LQ_CUDA_TRY(cudaFuncSetAttribute(k_fused_pass_narrow<2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    done = true;
    return LQ_OK;
}

static int pp_engine() {  // 1: ping-pong register rounds over PassOp records
    static const int v = [] {
        const char *e = getenv("LQ_FUSED_ENGINE");
        return e ? atoi(e) : 1;
    }();
    return v;
}

static int pair_index(int a, int b) {
    if (a > b) std::swap(a, b);
    static const int idx[4][4] = {{-1, 0, 1, 2}, {0, -1, 3, 4}, {1, 3, -1, 5}, {2, 4, 5, -1}};
    return idx[a][b];
}

// The kernel record of one encoded op (flat dispatch code, see PassCode).
PassOp pass_op(const FusedOp &f) {
    PassOp p{};
    p.coef = f.coef;
    p.cm = f.cm;
    p.gmask = f.gmask;
    p.fixmask = f.fixmask;
    auto packbits = [](int pb0, int pb1, int npat) {
        return (pb0 < 0 ? 0 : pb0) | (pb1 < 0 ? 0 : pb1) << 8 | npat << 16;
    };
    switch (f.type) {
    case F_M1: p.code = PC_M1 + f.k0; break;
    case F_M1C: p.code = PC_M1C + f.k0; break;
    case F_X: p.code = PC_X + f.k0; break;
    case F_XC: p.code = PC_XC + f.k0; break;
    case F_DIAG: p.code = PC_DIAG; p.bits = packbits(f.pb0, f.pb1, f.npat); break;
    case F_SWAP: p.code = PC_SWAP + pair_index(f.k0, f.k1); break;
    case F_M2: p.code = PC_M2 + pair_index(f.k0, f.k1); break;
    case F_M2R: p.code = PC_M2R + pair_index(f.k0, f.k1); break;
    case F_DTAB: p.code = PC_DTAB; p.bits = packbits(f.pb0, f.pb1, f.npat); break;
    case F_PAIR: p.code = PC_PAIR + pair_index(f.k0, f.k1) * 4 + (f.cm >> 2); p.cm = 0; break;
    case F_BLOCK3: p.code = PC_BLOCK3; break;
    default: p.code = PC_BLOCK4; break;
    }
    return p;
}

static int set_pp_attrs() {
    static bool done = false;
    if (done) return LQ_OK;
    const int mx = (int)fused_smem(kMaxT);
#define LQ_ATTR(K) LQ_CUDA_TRY(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, mx))
    LQ_ATTR(k_fused_pp<1>);
    LQ_ATTR(k_fused_pp_narrow<1>);
#undef LQ_ATTR
    done = true;
    return LQ_OK;
}

static int launch_pass_pp(lq_state *s, int T, int h, const FusedRound *d_rounds, int nrounds,
                          const PassOp *d_ops, const double *d_coef, const uint16_t *d_tb,
                          int mode) {
    const int n = s->n;
    const int m = T - 4;
    CUtensorMap map;
    LQ_TRY(make_tile_map(&map, s->d, n, h, m));
    const int ntiles = 1 << (n - T);
    TileCoords tc{h, h + m, ntiles};
    const size_t smem = fused_smem(T);
    LQ_TRY(set_pp_attrs());
    prof_begin(s->stream, kProfFused);
    const dim3 blk(1u << (T - 4));
#define LQ_FUSED_LAUNCH(K) \
    K<<<ntiles, blk, smem, s->stream>>>(map, T, tc, d_rounds, nrounds, d_ops, d_coef, d_tb, \
                                        s->d_flag)
    (void)mode;  // one op set (4x4, pair and table ops included); blocks use launch_pass
    if (T >= 12) LQ_FUSED_LAUNCH(k_fused_pp<1>);
    else LQ_FUSED_LAUNCH(k_fused_pp_narrow<1>);
#undef LQ_FUSED_LAUNCH
    prof_end(s->stream, kProfFused);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

static int launch_pass(lq_state *s, int T, int h, const FusedRound *d_rounds, int nrounds,
                       const FusedOp *d_ops, const double *d_coef, int mode) {
    const int n = s->n;
    const int m = T - 4;
    CUtensorMap map;
    LQ_TRY(make_tile_map(&map, s->d, n, h, m));
    const int ntiles = 1 << (n - T);
    TileCoords tc{h, h + m, ntiles};
    const int grid = fused_grid(T, ntiles);
    const size_t smem = fused_smem(T);
    prof_begin(s->stream, kProfFused);
    const dim3 blk(1u << (T - 4));
#define LQ_FUSED_LAUNCH(K) \
    K<<<grid, blk, smem, s->stream>>>(map, T, tc, d_rounds, nrounds, d_ops, d_coef, s->d_flag)
    if (T >= 12) {
        if (mode == 2) LQ_FUSED_LAUNCH(k_fused_pass<2>);
        else if (mode == 1) LQ_FUSED_LAUNCH(k_fused_pass<1>);
        else LQ_FUSED_LAUNCH(k_fused_pass<0>);
    } else {
        if (mode == 2) LQ_FUSED_LAUNCH(k_fused_pass_narrow<2>);
        else if (mode == 1) LQ_FUSED_LAUNCH(k_fused_pass_narrow<1>);
        else LQ_FUSED_LAUNCH(k_fused_pass_narrow<0>);
    }
#undef LQ_FUSED_LAUNCH
    prof_end(s->stream, kProfFused);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

// Encode the ops of one register round.  Diagonal gates move as early as they
// commute and each run of them becomes one F_DTAB: a phase table over the
// round's 16 register elements, the product of the run's phases, computed on
// the host.  A diagonal bit outside the register set is constant per thread
// (a thread bit of the tile, or a bit outside the window, constant per tile),
// so a table may depend on up to two such bits: one 16-entry variant per value.
// A run still open at the end of the round is carried into the next fused
// round (`carry`; `has_next` tells whether one follows with no standalone gate
// in between), where it joins that round's first table.
static void encode_round(const std::vector<GateOp> &gops, const std::vector<int> &pass_gates,
                         const PlannedRound &rd, bool has_next, int h, int T,
                         std::vector<const GateOp *> &carry, std::vector<FusedOp> &fops,
                         std::vector<double> &coef, int &mode) {
    using cd = std::complex<double>;
    const int m = T - 4;
    auto reg = [&](int b) {
        if (!(b < 4 || (b >= h && b < h + m))) return -1;
        const int lp = local_pos(b, h);
        for (int k = 0; k < 4; ++k)
            if (rd.rpos[k] == lp) return k;
        return -1;
    };
    const bool merge = real_fold_enabled();
    auto outside = [&](const GateOp &g) {  // its non-register bits, as a mask
        uint64_t o = 0;
        for (int k = 0; k < g.npat; ++k)
            if (reg(g.pat[k]) < 0) o |= 1ull << g.pat[k];
        for (int k = 0; k < g.nfix; ++k)
            if (reg(g.fix[k]) < 0) o |= 1ull << g.fix[k];
        return o;
    };
    auto table_ok = [&](const GateOp &g) {
        return merge && g.type == OP_DIAG && !g.renorm && popc(outside(g)) <= 2;
    };
    std::vector<const GateOp *> L(carry.begin(), carry.end());
    carry.clear();
    for (int k : rd.ops) {
        const GateOp &g = gops[pass_gates[k]];
        size_t pos = L.size();
        if (table_ok(g)) {
            const uint64_t b = op_bits(g);
            while (pos > 0 && !(op_bits(*L[pos - 1]) & b)) --pos;
        }
        L.insert(L.begin() + pos, &g);
    }
    std::vector<const GateOp *> pending;
    uint64_t pbits = 0, pout = 0;
    auto flush = [&]() {
        if (pending.empty()) return;
        int vb[2] = {-1, -1}, nv = 0;
        for (int b = 0; b < 64; ++b)
            if (pout >> b & 1) vb[nv++] = b;
        auto bitval = [&](int b, int e, int v) {
            const int k = reg(b);
            if (k >= 0) return (e >> k) & 1;
            return b == vb[0] ? v & 1 : (v >> 1) & 1;
        };
        FusedOp f{};
        f.type = F_DTAB;
        f.coef = (int)coef.size();
        f.npat = nv;
        f.pb0 = vb[0];
        f.pb1 = vb[1];
        f.param = f.param2 = -1;
        f.coef_alt = f.coef_alt2 = -1;
        for (int v = 0; v < (1 << nv); ++v)
            for (int e = 0; e < 16; ++e) {
                cd t = 1.0;
                for (const GateOp *g : pending) {
                    bool on = true;
                    for (int k = 0; k < g->nfix; ++k) on = on && bitval(g->fix[k], e, v);
                    if (!on) continue;
                    int pidx = 0;
                    for (int k = 0; k < g->npat; ++k) pidx |= bitval(g->pat[k], e, v) << k;
                    t *= cd(g->m[2 * pidx], g->m[2 * pidx + 1]);
                }
                coef.push_back(t.real());
                coef.push_back(t.imag());
            }
        fops.push_back(f);
        mode = std::max(mode, 1);
        pending.clear();
        pbits = pout = 0;
    };
    for (const GateOp *g : L) {
        if (table_ok(*g)) {
            const uint64_t o = outside(*g);
            if (popc(pout | o) > 2) flush();
            pending.push_back(g);
            pbits |= op_bits(*g);
            pout |= o;
            continue;
        }
        if (op_bits(*g) & pbits) flush();
        encode_op(*g, h, m, rd.rpos, fops, coef);
        const int t = fops.back().type;
        if (t == F_M2 || t == F_M2R || t == F_R1S || t == F_PAIR) mode = std::max(mode, 1);
        if (t == F_BLOCK3 || t == F_BLOCK4) mode = 2;
    }
    if (has_next && !pending.empty())
        carry = pending;
    else
        flush();
}

// Build the device program of every fused pass of `steps`.
static void encode_steps(const std::vector<PlanStep> &steps, const std::vector<GateOp> &gops,
                         int T, std::vector<FusedRound> &rounds, std::vector<FusedOp> &fops,
                         std::vector<double> &coef, std::vector<PassLaunch> &launches) {
    // diagonal runs carried forward, across rounds and into the next pass when
    // no standalone gate comes between
    std::vector<const GateOp *> carry;
    for (size_t si = 0; si < steps.size(); ++si) {
        const PlanStep &st = steps[si];
        if (!st.fused) continue;
        const bool next_pass = si + 1 < steps.size() && steps[si + 1].fused &&
                               !steps[si + 1].pass.rounds.empty();
        PassLaunch pl{st.pass.h, (int)rounds.size(), (int)st.pass.rounds.size(), 0};
        for (size_t ri = 0; ri < st.pass.rounds.size(); ++ri) {
            const PlannedRound &rd = st.pass.rounds[ri];
            const bool has_next = ri + 1 < st.pass.rounds.size() || next_pass;
            FusedRound fr{};
            fill_round(fr, rd.rpos, T, st.pass.h);
            fr.op_begin = (int)fops.size();
            encode_round(gops, st.pass.gates, rd, has_next, st.pass.h, T, carry, fops, coef,
                         pl.mode);
            fr.op_end = (int)fops.size();
            rounds.push_back(fr);
        }
        launches.push_back(pl);
    }
}

// ---------------------------------------------------------------------------
// Plan cache: the program of the last fused circuit stays in the handle's
// program buffer with its launch list, so submitting the same circuit again
// (same gates, angles and settings, compared byte for byte) launches at once:
// no planning, no upload, no synchronisation with earlier work.
// ---------------------------------------------------------------------------
struct PlanCache {
    std::vector<unsigned char> key;
    int T = 0, stride = 0;
    size_t off_ops = 0, off_coef = 0, off_tb = 0;
    struct Step {
        bool fused;
        GateOp gate;
        PassLaunch pl;
    };
    std::vector<Step> steps;
};

void free_plan_cache(lq_state *s) {
    delete static_cast<PlanCache *>(s->plan_cache);
    s->plan_cache = nullptr;
    s->prog_valid = false;
}

static std::vector<unsigned char> plan_key(const lq_gate *ops, int nops, const double *theta,
                                           int ntheta, int n, int T) {
    const int32_t hdr[6] = {n, T, nops, ntheta, real_fold_mode(), pp_engine()};
    std::vector<unsigned char> k(sizeof(hdr) + sizeof(lq_gate) * (size_t)nops +
                                 sizeof(double) * (size_t)ntheta);
    memcpy(k.data(), hdr, sizeof(hdr));
    if (nops) memcpy(k.data() + sizeof(hdr), ops, sizeof(lq_gate) * (size_t)nops);
    if (ntheta)
        memcpy(k.data() + sizeof(hdr) + sizeof(lq_gate) * (size_t)nops, theta,
               sizeof(double) * (size_t)ntheta);
    return k;
}

static int launch_cached(lq_state *s, const PlanCache &pc) {
    const char *dp = (const char *)s->d_prog;
    const FusedRound *d_rounds = (const FusedRound *)dp;
    const PassOp *d_ops = (const PassOp *)(dp + pc.off_ops);
    const double *d_coef = (const double *)(dp + pc.off_coef);
    const uint16_t *d_tb = (const uint16_t *)(dp + pc.off_tb);
    for (const auto &st : pc.steps) {
        if (!st.fused) {
            LQ_TRY(launch_gate_op(s, st.gate));
            s->last_launches += st.gate.renorm ? 3 : 1;
            continue;
        }
        LQ_TRY(launch_pass_pp(s, pc.T, st.pl.h, d_rounds + st.pl.round_begin, st.pl.nrounds, d_ops,
                              d_coef, d_tb + (size_t)st.pl.round_begin * pc.stride, st.pl.mode));
        s->last_launches += 1;
        s->last_passes += 1;
    }
    return LQ_OK;
}

int apply_circuit_impl(lq_state *s, const lq_gate *ops, int nops, const double *theta,
                       int ntheta, int mode) {
    const int n = s->n;
    s->last_launches = 0;
    s->last_passes = 0;
    for (int i = 0; i < nops; ++i) LQ_TRY(validate_gate(&ops[i], n, ntheta));
    const bool can_fuse = mode == LQ_EXEC_FUSED && s->dtype == LQ_C128 && n >= 5;
    std::vector<unsigned char> key;
    if (can_fuse && pp_engine() == 1) {
        key = plan_key(ops, nops, theta, ntheta, n, std::min(fusion_width(), n));
        const PlanCache *pc = static_cast<const PlanCache *>(s->plan_cache);
        if (s->prog_valid && pc && pc->key == key) return launch_cached(s, *pc);
    }
    std::vector<GateOp> gops(nops);
    for (int i = 0; i < nops; ++i) LQ_TRY(make_gate_op(&ops[i], theta, n, &gops[i]));
    if (!can_fuse) {
        for (int i = 0; i < nops; ++i) {
            LQ_TRY(launch_gate_op(s, gops[i]));
            s->last_launches += gops[i].renorm ? 3 : 1;
        }
        return LQ_OK;
    }
    const int T = std::min(fusion_width(), n);
    std::vector<int> orig;
    fold_pairs(gops, orig, T);
    std::vector<PlanStep> steps = plan_circuit(gops, n, T);
    std::vector<FusedRound> rounds;
    std::vector<FusedOp> fops;
    std::vector<double> coef;
    std::vector<PassLaunch> launches;
    encode_steps(steps, gops, T, rounds, fops, coef, launches);
    if (pp_engine() == 1) {
        // Kernel records, round by round: a table followed by a pair op in the
        // same round becomes one record (PC_TPAIR), so the round dispatches once.
        std::vector<PassOp> pops;
        pops.reserve(fops.size());
        for (auto &fr : rounds) {
            const int b0 = (int)pops.size();
            for (int o = fr.op_begin; o < fr.op_end; ++o) {
                const FusedOp &f = fops[o];
                PassOp p = pass_op(f);
                if (f.type == F_PAIR) {
                    p.x0 = coef[f.coef];
                    p.x1 = coef[f.coef + 1];
                }
                if (f.type == F_DTAB && o + 1 < fr.op_end && fops[o + 1].type == F_PAIR &&
                    fops[o + 1].gmask == 0 && f.gmask == 0) {
                    const FusedOp &g = fops[o + 1];
                    p.code = PC_TPAIR + pair_index(g.k0, g.k1) * 4 + (g.cm >> 2);
                    p.x0 = coef[g.coef];
                    p.x1 = coef[g.coef + 1];
                    ++o;  // the pair is part of this record
                }
                pops.push_back(p);
            }
            fr.op_begin = b0;
            fr.op_end = (int)pops.size();
        }
        // each thread's tile-local base index, per round (lanes from fill_round)
        const int nthr = 1 << (T - 4), stride = tb_stride(nthr);
        std::vector<uint16_t> tb(rounds.size() * stride, 0);
        for (size_t r = 0; r < rounds.size(); ++r)
            for (int t = 0; t < nthr; ++t) {
                int v = 0;
                for (int j = 0; j < rounds[r].nlane; ++j) v |= ((t >> j) & 1) << rounds[r].lane[j];
                tb[r * stride + t] = (uint16_t)v;
            }
        const size_t rb = rounds.size() * sizeof(FusedRound);
        const size_t ob = pops.size() * sizeof(PassOp);
        const size_t cb = coef.size() * sizeof(double);
        const size_t tbb = tb.size() * sizeof(uint16_t);
        auto al = [](size_t x) { return (x + 255) / 256 * 256; };
        LQ_TRY(ensure_prog(s, al(rb) + al(ob) + al(cb) + al(tbb) + 256));
        char *dp = (char *)s->d_prog;
        FusedRound *d_rounds = (FusedRound *)dp;
        PassOp *d_ops = (PassOp *)(dp + al(rb));
        double *d_coef = (double *)(dp + al(rb) + al(ob));
        uint16_t *d_tb = (uint16_t *)(dp + al(rb) + al(ob) + al(cb));
        // The program buffer may still be read by a previous call's kernels.
        LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
        if (rb) LQ_CUDA_TRY(cudaMemcpy(d_rounds, rounds.data(), rb, cudaMemcpyHostToDevice));
        if (ob) LQ_CUDA_TRY(cudaMemcpy(d_ops, pops.data(), ob, cudaMemcpyHostToDevice));
        if (cb) LQ_CUDA_TRY(cudaMemcpy(d_coef, coef.data(), cb, cudaMemcpyHostToDevice));
        if (tbb) LQ_CUDA_TRY(cudaMemcpy(d_tb, tb.data(), tbb, cudaMemcpyHostToDevice));
        auto pc = std::make_unique<PlanCache>();
        pc->key = std::move(key);
        pc->T = T;
        pc->stride = stride;
        pc->off_ops = (size_t)((char *)d_ops - dp);
        pc->off_coef = (size_t)((char *)d_coef - dp);
        pc->off_tb = (size_t)((char *)d_tb - dp);
        size_t li = 0;
        for (auto &st : steps) {
            if (!st.fused) pc->steps.push_back({false, gops[st.gate], PassLaunch{}});
            else pc->steps.push_back({true, GateOp{}, launches[li++]});
        }
        free_plan_cache(s);
        s->plan_cache = pc.release();
        s->prog_valid = true;
        return launch_cached(s, *static_cast<const PlanCache *>(s->plan_cache));
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
    LQ_TRY(set_smem_attrs());

    size_t li = 0;
    for (auto &st : steps) {
        if (!st.fused) {
            LQ_TRY(launch_gate_op(s, gops[st.gate]));
            s->last_launches += gops[st.gate].renorm ? 3 : 1;
            continue;
        }
        const PassLaunch &pl = launches[li++];
        LQ_TRY(launch_pass(s, T, pl.h, d_rounds + pl.round_begin, pl.nrounds, d_ops, d_coef,
                           pl.mode));
        s->last_launches += 1;
        s->last_passes += 1;
    }
    return LQ_OK;
}

int apply_block_impl(lq_state *s, int k, const int *qubits, const double *m) {
    const int n = s->n;
    if (k == 1) return lq_apply_matrix1(s, qubits[0], m);
    if (k == 2) return lq_apply_matrix2(s, qubits[0], qubits[1], m);
    if (s->dtype != LQ_C128)
        return set_error(LQ_ERR_UNSUPPORTED, "block gates need a complex128 state");
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
    int rpos[4];
    for (int j = 0; j < 4; ++j) rpos[j] = Rv[j];
    FusedRound fr{};
    fill_round(fr, rpos, T, h);
    fr.op_begin = 0;
    fr.op_end = 1;
    FusedOp fo{};
    fo.type = k == 3 ? F_BLOCK3 : F_BLOCK4;
    fo.pb0 = fo.pb1 = -1;
    fo.param = fo.coef_alt = fo.param2 = fo.coef_alt2 = -1;
    fo.coef = 0;
    const size_t cb = sizeof(double) * 2 * (1 << k) * (1 << k);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    LQ_TRY(ensure_prog(s, al(sizeof(FusedRound)) + al(sizeof(FusedOp)) + al(cb) + 256));
    char *dp = (char *)s->d_prog;
    FusedRound *d_rounds = (FusedRound *)dp;
    FusedOp *d_ops = (FusedOp *)(dp + al(sizeof(FusedRound)));
    double *d_coef = (double *)(dp + al(sizeof(FusedRound)) + al(sizeof(FusedOp)));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    LQ_CUDA_TRY(cudaMemcpy(d_rounds, &fr, sizeof(FusedRound), cudaMemcpyHostToDevice));
    LQ_CUDA_TRY(cudaMemcpy(d_ops, &fo, sizeof(FusedOp), cudaMemcpyHostToDevice));
    LQ_CUDA_TRY(cudaMemcpy(d_coef, m, cb, cudaMemcpyHostToDevice));
    LQ_TRY(set_smem_attrs());
    return launch_pass(s, T, h, d_rounds, 1, d_ops, d_coef, 2);
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

int lq_set_fusion_width(int tile_bits) {
    if (tile_bits < 5 || tile_bits > kMaxT)
        return set_error(LQ_ERR_INVALID_ARG, "fusion width must be 5..%d", kMaxT);
    g_fusion_width.store(tile_bits);
    return LQ_OK;
}

int lq_get_fusion_width(int *tile_bits) {
    if (!tile_bits) return set_error(LQ_ERR_INVALID_ARG, "null output");
    *tile_bits = fusion_width();
    return LQ_OK;
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

static int plan_for(int num_qubits, const lq_gate *ops, int nops, const double *theta,
                    int ntheta, std::vector<GateOp> &gops, std::vector<PlanStep> &steps,
                    int &T, std::vector<int> &orig) {
    if (nops < 0 || (nops > 0 && !ops)) return set_error(LQ_ERR_INVALID_ARG, "bad op list");
    if (num_qubits < 5 || num_qubits > 36)
        return set_error(LQ_ERR_UNSUPPORTED, "fused planning needs 5..36 qubits");
    gops.resize(nops);
    static const double zero_theta[1] = {0.0};
    for (int i = 0; i < nops; ++i) {
        lq_gate g = ops[i];
        if (!theta) {  // angles do not change the plan: unbind parameters
            for (int k = 0; k < 3; ++k) g.param[k] = -1;
        }
        LQ_TRY(validate_gate(&g, num_qubits, theta ? ntheta : 1 << 30));
        LQ_TRY(make_gate_op(&g, theta ? theta : zero_theta, num_qubits, &gops[i]));
    }
    T = std::min(fusion_width(), num_qubits);
    fold_pairs(gops, orig, T);
    steps = plan_circuit(gops, num_qubits, T);
    return LQ_OK;
}

int lq_plan_circuit(int num_qubits, const lq_gate *ops, int nops, int *passes, int *rounds,
                    int *standalone) {
    std::vector<GateOp> gops;
    std::vector<PlanStep> steps;
    std::vector<int> orig;
    int T;
    LQ_TRY(plan_for(num_qubits, ops, nops, nullptr, 0, gops, steps, T, orig));
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

int lq_plan_dump(int num_qubits, const lq_gate *ops, int nops, const double *theta, int ntheta,
                 void *buf, size_t cap, size_t *used) {
    // Layout (little endian): int32 counts[5] = {nsteps, nrounds, nops, ncoef, T},
    // then nsteps x int32[5] {fused, gate, h, round_begin, nrounds},
    // nrounds x FusedRound, nops x FusedOp, ncoef x double.
    std::vector<GateOp> gops;
    std::vector<PlanStep> steps;
    std::vector<int> orig;
    int T;
    LQ_TRY(plan_for(num_qubits, ops, nops, theta, ntheta, gops, steps, T, orig));
    std::vector<FusedRound> rounds;
    std::vector<FusedOp> fops;
    std::vector<double> coef;
    std::vector<PassLaunch> launches;
    encode_steps(steps, gops, T, rounds, fops, coef, launches);
    std::vector<int32_t> st_rec;
    size_t li = 0;
    for (auto &st : steps) {
        if (!st.fused) {
            // standalone steps name the caller's gate (they are never folded)
            st_rec.insert(st_rec.end(), {0, orig[st.gate], 0, 0, 0});
        } else {
            const PassLaunch &pl = launches[li++];
            st_rec.insert(st_rec.end(), {1, -1, pl.h, pl.round_begin, pl.nrounds});
        }
    }
    const int32_t counts[5] = {(int32_t)steps.size(), (int32_t)rounds.size(),
                               (int32_t)fops.size(), (int32_t)coef.size(), T};
    const size_t need = sizeof(counts) + st_rec.size() * 4 + rounds.size() * sizeof(FusedRound) +
                        fops.size() * sizeof(FusedOp) + coef.size() * 8;
    if (used) *used = need;
    if (!buf || cap < need) return set_error(LQ_ERR_INVALID_ARG, "buffer too small (%zu)", need);
    char *p = (char *)buf;
    memcpy(p, counts, sizeof(counts));
    p += sizeof(counts);
    memcpy(p, st_rec.data(), st_rec.size() * 4);
    p += st_rec.size() * 4;
    memcpy(p, rounds.data(), rounds.size() * sizeof(FusedRound));
    p += rounds.size() * sizeof(FusedRound);
    memcpy(p, fops.data(), fops.size() * sizeof(FusedOp));
    p += fops.size() * sizeof(FusedOp);
    memcpy(p, coef.data(), coef.size() * 8);
    return LQ_OK;
}

int lq_last_circuit_stats(const lq_state *s, int *launches, int *passes) {
    LQ_TRY(check_state(s));
    if (launches) *launches = s->last_launches;
    if (passes) *passes = s->last_passes;
    return LQ_OK;
}

}  // extern "C"
