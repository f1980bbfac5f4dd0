// Register rounds of the fused pass kernel, ping-pong form.
//
// A thread holds the 16 amplitudes of a round in registers (fused_core.cuh
// explains rounds).  Here every op reads one 16-element array and writes ALL
// 16 elements of the other, so each result is written straight into its final
// register: after a switch over op kinds the compiler has nothing to
// reconcile, where an in-place update needs register moves at every join (on
// B200 they were the majority of the executed instructions).  The two arrays
// alternate per op; the round ends in whichever holds the data.
//
// Ops come as compact PassOp records whose `code` is one flat dispatch index
// (pass_op_code on the host), so one indirect branch selects a fully
// specialised routine (register bits, rotation forms and permutation fixed at
// compile time).
#pragma once

#include "fused_core.cuh"

namespace lq {

struct PassOp {
    int32_t code;      // flat dispatch code (PC_* below)
    int32_t coef;      // offset of the coefficients (doubles) in the pass program
    int32_t cm;        // register control mask (M1C / XC)
    int32_t bits;      // DIAG: pb0 | pb1 << 8 | npat << 16; DTAB: variant bits, same packing
    uint64_t gmask;    // thread-level condition: global bits outside R that must be 1
    uint64_t fixmask;  // DIAG: element condition
    double x0, x1;     // PAIR: the two rotation parameters (no coefficient load)
};
static_assert(sizeof(PassOp) == 48, "PassOp layout");

// Flat codes.  Register-bit pairs (k0 < k1) are numbered
// 0:(0,1) 1:(0,2) 2:(0,3) 3:(1,2) 4:(1,3) 5:(2,3).
enum PassCode {
    PC_M1 = 0,       // + k0 (4)
    PC_M1C = 4,      // + k0 (4)
    PC_X = 8,        // + k0 (4)
    PC_XC = 12,      // + k0 (4)
    PC_DIAG = 16,    // (1)
    PC_SWAP = 17,    // + pair (6)
    PC_M2 = 23,      // + pair (6)
    PC_M2R = 29,     // + pair (6)
    PC_DTAB = 35,    // (1)
    PC_PAIR = 36,    // + pair * 4 + perm (24); both rotations in form 0
    PC_BLOCK3 = 60,
    PC_BLOCK4 = 61,
    PC_TPAIR = 62,   // + pair * 4 + perm (24): a diagonal table, then a pair op
    PC_COUNT = 86
};

__host__ __device__ constexpr int pair_k0(int p) { return p < 3 ? 0 : p < 5 ? 1 : 2; }
__host__ __device__ constexpr int pair_k1(int p) {
    return p == 0 ? 1 : p == 1 ? 2 : p == 2 ? 3 : p == 3 ? 2 : 3;
}

// ---- op routines: s = source array, d = destination array (all 16 written) --

__device__ __forceinline__ double2 cmad2(double2 m0, double2 x0, double2 m1, double2 x1) {
    // m0 * x0 + m1 * x1 (complex)
    double2 o;
    o.x = fma(-m1.y, x1.y, fma(m1.x, x1.x, fma(-m0.y, x0.y, m0.x * x0.x)));
    o.y = fma(m1.y, x1.x, fma(m1.x, x1.y, fma(m0.y, x0.x, m0.x * x0.y)));
    return o;
}

template <int K>
__device__ __forceinline__ void pp_m1(const double2 (&s)[16], double2 (&d)[16],
                                      const double *__restrict__ c, int cm) {
    const double2 m00 = make_double2(c[0], c[1]), m01 = make_double2(c[2], c[3]);
    const double2 m10 = make_double2(c[4], c[5]), m11 = make_double2(c[6], c[7]);
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if (e & (1 << K)) continue;
        const int f = e | (1 << K);
        const double2 x0 = s[e], x1 = s[f];
        if ((e & cm) == cm) {
            d[e] = cmad2(m00, x0, m01, x1);
            d[f] = cmad2(m10, x0, m11, x1);
        } else {
            d[e] = x0;
            d[f] = x1;
        }
    }
}

template <int K>
__device__ __forceinline__ void pp_x(const double2 (&s)[16], double2 (&d)[16], int cm) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if (e & (1 << K)) continue;
        const int f = e | (1 << K);
        const bool on = (e & cm) == cm;
        d[e] = on ? s[f] : s[e];
        d[f] = on ? s[e] : s[f];
    }
}

template <int K0, int K1>
__device__ __forceinline__ void pp_swap(const double2 (&s)[16], double2 (&d)[16]) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const int b0 = (e >> K0) & 1, b1 = (e >> K1) & 1;
        d[e] = b0 != b1 ? s[e ^ (1 << K0) ^ (1 << K1)] : s[e];
    }
}

// 4x4 on (K0, K1), index q = bit(K0) << 1 | bit(K1); complex (16 complex
// coefficients) or real (16 doubles).
template <int K0, int K1, bool REAL>
__device__ __forceinline__ void pp_m2(const double2 (&s)[16], double2 (&d)[16],
                                      const double *__restrict__ c) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if ((e & (1 << K0)) || (e & (1 << K1))) continue;
        const int i[4] = {e, e | (1 << K1), e | (1 << K0), e | (1 << K0) | (1 << K1)};
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            double ox = 0.0, oy = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double2 x = s[i[q]];
                if (REAL) {
                    const double m = c[r * 4 + q];
                    ox = q == 0 ? m * x.x : fma(m, x.x, ox);
                    oy = q == 0 ? m * x.y : fma(m, x.y, oy);
                } else {
                    const double mr = c[2 * (r * 4 + q)], mi = c[2 * (r * 4 + q) + 1];
                    ox = fma(-mi, x.y, q == 0 ? mr * x.x : fma(mr, x.x, ox));
                    oy = fma(mi, x.x, q == 0 ? mr * x.y : fma(mr, x.y, oy));
                }
            }
            d[i[r]] = make_double2(ox, oy);
        }
    }
}

template <int FORM>
__device__ __forceinline__ void rot_pp(double2 x0, double2 x1, double t, double2 &y0,
                                       double2 &y1) {
    if (FORM == 0) {
        y0 = make_double2(fma(-t, x1.x, x0.x), fma(-t, x1.y, x0.y));
        y1 = make_double2(fma(t, x0.x, x1.x), fma(t, x0.y, x1.y));
    } else {
        y0 = make_double2(fma(t, x0.x, -x1.x), fma(t, x0.y, -x1.y));
        y1 = make_double2(fma(t, x1.x, x0.x), fma(t, x1.y, x0.y));
    }
}

template <int K, int FORM>
__device__ __forceinline__ void pp_r1s(const double2 (&s)[16], double2 (&d)[16], double t) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if (e & (1 << K)) continue;
        rot_pp<FORM>(s[e], s[e | (1 << K)], t, d[e], d[e | (1 << K)]);
    }
}

// Folded pair in real form: rotation on K1 (x1), rotation on K0 (x0), then the
// permutation P, written as the destinations of the second level.
template <int K0, int K1, int F0, int F1, int P>
__device__ __forceinline__ void pp_pair(const double2 (&s)[16], double2 (&d)[16], double x0,
                                        double x1) {
    constexpr int perm[4][4] = {{0, 1, 2, 3}, {0, 1, 3, 2}, {0, 3, 2, 1}, {0, 2, 1, 3}};
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if ((e & (1 << K0)) || (e & (1 << K1))) continue;
        const int i[4] = {e, e | (1 << K1), e | (1 << K0), e | (1 << K0) | (1 << K1)};
        double2 v0, v1, v2, v3, z[4];
        rot_pp<F1>(s[i[0]], s[i[1]], x1, v0, v1);
        rot_pp<F1>(s[i[2]], s[i[3]], x1, v2, v3);
        rot_pp<F0>(v0, v2, x0, z[0], z[2]);
        rot_pp<F0>(v1, v3, x0, z[1], z[3]);
#pragma unroll
        for (int q = 0; q < 4; ++q) d[i[perm[P][q]]] = z[q];
    }
}

// A diagonal table (16 complex factors at c) and then a pair op, in one pass
// over the registers.
template <int K0, int K1, int P>
__device__ __forceinline__ void pp_tpair(const double2 (&s)[16], double2 (&d)[16],
                                         const double *__restrict__ c, double x0, double x1) {
    constexpr int perm[4][4] = {{0, 1, 2, 3}, {0, 1, 3, 2}, {0, 3, 2, 1}, {0, 2, 1, 3}};
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if ((e & (1 << K0)) || (e & (1 << K1))) continue;
        const int i[4] = {e, e | (1 << K1), e | (1 << K0), e | (1 << K0) | (1 << K1)};
        double2 u[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double2 p = *reinterpret_cast<const double2 *>(c + 2 * i[q]);
            const double2 v = s[i[q]];
            u[q] = make_double2(fma(-v.y, p.y, v.x * p.x), fma(v.x, p.y, v.y * p.x));
        }
        double2 v0, v1, v2, v3, z[4];
        rot_pp<0>(u[0], u[1], x1, v0, v1);
        rot_pp<0>(u[2], u[3], x1, v2, v3);
        rot_pp<0>(v0, v2, x0, z[0], z[2]);
        rot_pp<0>(v1, v3, x0, z[1], z[3]);
#pragma unroll
        for (int q = 0; q < 4; ++q) d[i[perm[P][q]]] = z[q];
    }
}

__device__ __forceinline__ void pp_dtab(const double2 (&s)[16], double2 (&d)[16],
                                        const double *__restrict__ c) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const double2 p = *reinterpret_cast<const double2 *>(c + 2 * e);
        const double2 v = s[e];
        d[e] = make_double2(fma(-v.y, p.y, v.x * p.x), fma(v.x, p.y, v.y * p.x));
    }
}

__device__ __forceinline__ void pp_diag(const double2 (&s)[16], double2 (&d)[16],
                                        const PassOp &op, const double *__restrict__ c,
                                        uint64_t gbase, const uint64_t *__restrict__ gpp) {
    const uint64_t fm = op.fixmask;
    const int npat = (op.bits >> 16) & 0xff;
    const int pb0 = op.bits & 0xff, pb1 = (op.bits >> 8) & 0xff;
    const uint64_t use0 = npat > 0 ? 1ull : 0ull, use1 = npat > 1 ? 1ull : 0ull;
    const double2 ph[4] = {make_double2(c[0], c[1]), make_double2(c[2], c[3]),
                           make_double2(c[4], c[5]), make_double2(c[6], c[7])};
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const uint64_t gi = gbase | ((e & 1) ? gpp[0] : 0ull) | ((e & 2) ? gpp[1] : 0ull) |
                            ((e & 4) ? gpp[2] : 0ull) | ((e & 8) ? gpp[3] : 0ull);
        const double2 v = s[e];
        if ((gi & fm) != fm) {
            d[e] = v;
            continue;
        }
        const int b0 = (int)((gi >> pb0) & use0), b1 = (int)((gi >> pb1) & use1);
        const double2 p = ph[b0 | (b1 << 1)];
        d[e] = make_double2(fma(-v.y, p.y, v.x * p.x), fma(v.x, p.y, v.y * p.x));
    }
}

template <int KB>
__device__ __forceinline__ void pp_block(const double2 (&s)[16], double2 (&d)[16],
                                         const double *__restrict__ c) {
    constexpr int D = 1 << KB;
#pragma unroll
    for (int hiv = 0; hiv < 16; hiv += D) {
#pragma unroll
        for (int r = 0; r < D; ++r) {
            double ore = 0.0, oim = 0.0;
#pragma unroll
            for (int q = 0; q < D; ++q) {
                const double mr = c[(r * D + q) * 2], mi = c[(r * D + q) * 2 + 1];
                ore = fma(-mi, s[hiv + q].y, fma(mr, s[hiv + q].x, ore));
                oim = fma(mi, s[hiv + q].x, fma(mr, s[hiv + q].y, oim));
            }
            d[hiv + r] = make_double2(ore, oim);
        }
    }
}

// One op, s -> d (all 16 elements written).  MODE as in fused_core.cuh (0:
// 2x2/X/diag/swap only; 1: also 4x4, pair, table and rotation ops; 2: also
// 8x8/16x16 blocks).  An op whose thread-level condition is false copies.
template <int MODE>
__device__ __forceinline__ void pp_apply(const double2 (&s)[16], double2 (&d)[16],
                                         const PassOp &op, const double *__restrict__ c,
                                         uint64_t gbase, const uint64_t *__restrict__ gp) {
    const int code = (gbase & op.gmask) == op.gmask ? op.code : -1;
    switch (code) {
#define LQ_K4(BASE, CALL) \
    case BASE + 0: CALL(0); break; case BASE + 1: CALL(1); break; \
    case BASE + 2: CALL(2); break; case BASE + 3: CALL(3); break;
#define LQ_M1(K) pp_m1<K>(s, d, c, 0)
#define LQ_M1C(K) pp_m1<K>(s, d, c, op.cm)
#define LQ_X(K) pp_x<K>(s, d, 0)
#define LQ_XC(K) pp_x<K>(s, d, op.cm)
        LQ_K4(PC_M1, LQ_M1)
        LQ_K4(PC_M1C, LQ_M1C)
        LQ_K4(PC_X, LQ_X)
        LQ_K4(PC_XC, LQ_XC)
#undef LQ_M1
#undef LQ_M1C
#undef LQ_X
#undef LQ_XC
#undef LQ_K4
    case PC_DIAG: pp_diag(s, d, op, c, gbase, gp); break;
#define LQ_P6(BASE, CALL) \
    case BASE + 0: CALL(0, 1); break; case BASE + 1: CALL(0, 2); break; \
    case BASE + 2: CALL(0, 3); break; case BASE + 3: CALL(1, 2); break; \
    case BASE + 4: CALL(1, 3); break; case BASE + 5: CALL(2, 3); break;
#define LQ_SW(A, B) pp_swap<A, B>(s, d)
        LQ_P6(PC_SWAP, LQ_SW)
#undef LQ_SW
#define LQ_M2(A, B) if constexpr (MODE >= 1) pp_m2<A, B, false>(s, d, c)
#define LQ_M2R(A, B) if constexpr (MODE >= 1) pp_m2<A, B, true>(s, d, c)
        LQ_P6(PC_M2, LQ_M2)
        LQ_P6(PC_M2R, LQ_M2R)
#undef LQ_M2
#undef LQ_M2R
#undef LQ_P6
    case PC_DTAB:
        if constexpr (MODE >= 1) {
            // up to two thread-constant bits select the table's variant
            const int nv = (op.bits >> 16) & 0xff;
            int v = 0;
            if (nv > 0) v = (int)((gbase >> (op.bits & 0xff)) & 1ull);
            if (nv > 1) v |= (int)((gbase >> ((op.bits >> 8) & 0xff)) & 1ull) << 1;
            pp_dtab(s, d, c + 32 * v);
        }
        break;
#define LQ_PR(P, Q)                                                                          \
    case PC_PAIR + P * 4 + Q:                                                                \
        if constexpr (MODE >= 1) pp_pair<pair_k0(P), pair_k1(P), 0, 0, Q>(s, d, op.x0, op.x1); \
        break;
#define LQ_PR4(P) LQ_PR(P, 0) LQ_PR(P, 1) LQ_PR(P, 2) LQ_PR(P, 3)
        LQ_PR4(0) LQ_PR4(1) LQ_PR4(2) LQ_PR4(3) LQ_PR4(4) LQ_PR4(5)
#undef LQ_PR4
#undef LQ_PR
#define LQ_TP(P, Q)                                                                    \
    case PC_TPAIR + P * 4 + Q:                                                         \
        if constexpr (MODE >= 1) {                                                     \
            const int nv = (op.bits >> 16) & 0xff;                                     \
            int v = 0;                                                                 \
            if (nv > 0) v = (int)((gbase >> (op.bits & 0xff)) & 1ull);                 \
            if (nv > 1) v |= (int)((gbase >> ((op.bits >> 8) & 0xff)) & 1ull) << 1;   \
            pp_tpair<pair_k0(P), pair_k1(P), Q>(s, d, c + 32 * v, op.x0, op.x1);        \
        }                                                                              \
        break;
#define LQ_TP4(P) LQ_TP(P, 0) LQ_TP(P, 1) LQ_TP(P, 2) LQ_TP(P, 3)
        LQ_TP4(0) LQ_TP4(1) LQ_TP4(2) LQ_TP4(3) LQ_TP4(4) LQ_TP4(5)
#undef LQ_TP4
#undef LQ_TP
    case PC_BLOCK3: if constexpr (MODE >= 2) pp_block<3>(s, d, c); break;
    case PC_BLOCK4: if constexpr (MODE >= 2) pp_block<4>(s, d, c); break;
    default:  // condition false (or an op this MODE does not hold): identity
#pragma unroll
        for (int e = 0; e < 16; ++e) d[e] = s[e];
        break;
    }
}

// One round on a tile in shared memory: gather into a, run the ops two at a
// time (a -> b, b -> a), scatter from the array holding the result.
// tbase is the thread's tile-local base index in this round (its register
// bits zero), precomputed on the host from the round's lane order.
// coef_of(op) gives the op's coefficient pointer (the batched engine swaps in
// a shifted parameter's coefficients there).
template <int MODE, class CoefOf>
__device__ __forceinline__ void run_round_pp_sel(uint32_t tile_a, const FusedRound &rd,
                                                 const PassOp *__restrict__ ops, CoefOf coef_of,
                                                 uint64_t tile_base, int h, int tbase) {
    const uint32_t sb = (uint32_t)swz(tbase) << 4;
    const uint64_t gbase = tile_base | (uint64_t)(tbase & 15) | ((uint64_t)(tbase >> 4) << h);
    // The swizzle is linear over XOR, so element e's offset is the XOR of the
    // offsets of its set register bits: four loads instead of sixteen.
    const uint32_t E0 = (uint32_t)rd.eoff[1], E1 = (uint32_t)rd.eoff[2];
    const uint32_t E2 = (uint32_t)rd.eoff[4], E3 = (uint32_t)rd.eoff[8];
    auto addr_of = [&](int e) {
        const uint32_t x = ((e & 1) ? E0 : 0u) ^ ((e & 2) ? E1 : 0u) ^ ((e & 4) ? E2 : 0u) ^
                           ((e & 8) ? E3 : 0u);
        return tile_a + (sb ^ x);
    };
    double2 a[16], b[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const uint32_t addr = addr_of(e);
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(a[e].x), "=d"(a[e].y) : "r"(addr));
    }
    const int o1 = rd.op_end;
    int o = rd.op_begin;
    for (; o + 1 < o1; o += 2) {
#ifndef LQ_PP_NO_PRELOAD
        // both records first: the second load is hidden behind the first op
        const PassOp p0 = ops[o];
        const PassOp p1 = ops[o + 1];
        pp_apply<MODE>(a, b, p0, coef_of(p0), gbase, rd.gpos);
        pp_apply<MODE>(b, a, p1, coef_of(p1), gbase, rd.gpos);
#else
        const PassOp p0 = ops[o];
        pp_apply<MODE>(a, b, p0, coef_of(p0), gbase, rd.gpos);
        const PassOp p1 = ops[o + 1];
        pp_apply<MODE>(b, a, p1, coef_of(p1), gbase, rd.gpos);
#endif
    }
    const bool odd = o < o1;
    if (odd) {
        const PassOp p0 = ops[o];
        pp_apply<MODE>(a, b, p0, coef_of(p0), gbase, rd.gpos);
    }
    if (odd) {  // two store paths: no register moves to bring b into a
#pragma unroll
        for (int e = 0; e < 16; ++e)
            asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(addr_of(e)), "d"(b[e].x),
                         "d"(b[e].y)
                         : "memory");
    } else {
#pragma unroll
        for (int e = 0; e < 16; ++e)
            asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(addr_of(e)), "d"(a[e].x),
                         "d"(a[e].y)
                         : "memory");
    }
}

template <int MODE>
__device__ __forceinline__ void run_round_pp(uint32_t tile_a, const FusedRound &rd,
                                             const PassOp *__restrict__ ops,
                                             const double *__restrict__ coef,
                                             uint64_t tile_base, int h, int tbase) {
    run_round_pp_sel<MODE>(
        tile_a, rd, ops, [coef](const PassOp &p) { return coef + p.coef; }, tile_base, h, tbase);
}

// Host: the record of an encoded op (defined with the fused planner).
PassOp pass_op(const FusedOp &f);

}  // namespace lq
