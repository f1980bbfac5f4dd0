// Register-level gate ops shared by the fused pass kernel (fused.cu) and the
// batched parameter-shift engine (batch.cu).
//
// A thread holds 16 amplitudes that differ only in four tile bits R (its
// "register bits"); each op below acts on those registers.  Ops are encoded
// by the host planner (fused.cu) as FusedOp records.
#pragma once

#include <cstdint>

#include "lq_internal.h"

namespace lq {

enum FusedOpType {
    F_M1 = 0,     // 2x2 on reg bit k0
    F_M1C = 1,    // 2x2 on reg bit k0 where the register bits cm are all 1
    F_X = 2,      // X on reg bit k0
    F_XC = 3,     // X on reg bit k0 where the register bits cm are all 1
    F_DIAG = 4,   // amplitude *= ph[pattern] where the global index bits fixmask are all 1;
                  // pattern = index bits pb0 (lsb), pb1
    F_SWAP = 5,   // swap reg bits k0, k1
    F_M2 = 6,     // 4x4, index = bit(k0)<<1 | bit(k1)
    F_BLOCK3 = 7, // 8x8 on reg bits 0..2 (matrix bit j <-> reg bit j)
    F_BLOCK4 = 8, // 16x16 on reg bits 0..3
    F_M2R = 9,    // real 4x4 (16 doubles), index = bit(k0)<<1 | bit(k1), k0 < k1
    F_DTAB = 10,  // amplitude e *= table[v][e] (16 complex per variant), e = register
                  // element index, v = values of the npat (<= 2) non-register global
                  // bits pb0 (lsb), pb1 of the thread's base index
    F_R1S = 11,   // scaled real rotation on reg bit k0, x = coef[0]:
                  // k1 = 0: [[1, -x], [x, 1]];  k1 = 1: [[x, -1], [1, x]]
    F_PAIR = 12   // scaled rotations [[1, -x], [x, 1]] on reg bits k1 (x = coef[1]) and
                  // k0 (x = coef[0]), then a permutation of the pair (cm >> 2: 0 none,
                  // 1 CNOT k0 -> k1, 2 CNOT k1 -> k0, 3 SWAP; cm bits 0-1 are 0)
};

struct FusedOp {
    int32_t type;
    int32_t k0, k1, cm;
    uint64_t gmask;    // thread-level condition: global index bits outside R, all must be 1
    uint64_t fixmask;  // F_DIAG element condition (any global bits)
    int32_t pb0, pb1;  // F_DIAG pattern bit positions (global)
    int32_t npat;
    int32_t coef;      // offset of the coefficients in the coefficient array (doubles)
    int32_t param;      // batched engine: parameter the op's angle is bound to (-1: none)
    int32_t coef_alt;   // batched engine: offset of the (+shift, -shift) coefficient pair
    int32_t param2;     // batched engine: second bound parameter of a merged op (-1: none)
    int32_t coef_alt2;  // batched engine: its (+shift, -shift) coefficient pair
};
static_assert(sizeof(FusedOp) == 64, "FusedOp layout is mirrored by the plan-dump reader");

struct FusedRound {
    int32_t eoff[16];  // swizzled byte offset of register element e relative to the thread base
    uint64_t gpos[4];  // global index mask of register bits 0..3
    int32_t lane[12];  // tile-local positions of the thread-index bits, in order
    int32_t nlane;
    int32_t op_begin, op_end;
    int32_t pad;
};

constexpr int kMaxT = 12;

// 128-byte TMA swizzle of a tile-local amplitude index: the 16-byte chunk
// (index bits 0-2) is XORed with the 128-byte row (index bits 3-5).
__host__ __device__ __forceinline__ int swz(int i) { return i ^ ((i >> 3) & 7); }

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ double2 cmul_add4(double ar, double ai, double2 x, double br,
                                             double bi, double2 y) {
    // (a * x + b * y) with one multiply and three FMAs per real output.
    double2 o;
    o.x = fma(-bi, y.y, fma(br, y.x, fma(-ai, x.y, ar * x.x)));
    o.y = fma(bi, y.x, fma(br, y.y, fma(ai, x.x, ar * x.y)));
    return o;
}

template <int K, bool CM>
__device__ __forceinline__ void reg_m1(double2 (&a)[16], int cm, const double (&c)[8]) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if (e & (1 << K)) continue;
        if (CM && (e & cm) != cm) continue;
        const double2 a0 = a[e], a1 = a[e | (1 << K)];
        a[e] = cmul_add4(c[0], c[1], a0, c[2], c[3], a1);
        a[e | (1 << K)] = cmul_add4(c[4], c[5], a0, c[6], c[7], a1);
    }
}

template <int K, bool CM>
__device__ __forceinline__ void reg_x(double2 (&a)[16], int cm) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if (e & (1 << K)) continue;
        if (CM && (e & cm) != cm) continue;
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

// 4x4 on register bits (K0, K1): four groups of four amplitudes.  The groups
// go two at a time so that each coefficient (one 16-byte load) serves two
// groups, with 16 accumulators live beside the 16 registers.
template <int K0, int K1>
__device__ __forceinline__ void reg_m2(double2 (&a)[16], const double *__restrict__ c) {
    const double2 *__restrict__ cm = reinterpret_cast<const double2 *>(c);
    int grp[4], ng = 0;
#pragma unroll
    for (int e = 0; e < 16; ++e)
        if (!(e & (1 << K0)) && !(e & (1 << K1))) grp[ng++] = e;
#pragma unroll
    for (int gp = 0; gp < 2; ++gp) {
        int idx[2][4];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int e = grp[2 * gp + s];
            idx[s][0] = e;
            idx[s][1] = e | (1 << K1);
            idx[s][2] = e | (1 << K0);
            idx[s][3] = e | (1 << K0) | (1 << K1);
        }
        double2 out[2][4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            double o0r = 0.0, o0i = 0.0, o1r = 0.0, o1i = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double2 m = cm[r * 4 + q];
                const double2 x0 = a[idx[0][q]], x1 = a[idx[1][q]];
                o0r = fma(-m.y, x0.y, fma(m.x, x0.x, o0r));
                o0i = fma(m.y, x0.x, fma(m.x, x0.y, o0i));
                o1r = fma(-m.y, x1.y, fma(m.x, x1.x, o1r));
                o1i = fma(m.y, x1.x, fma(m.x, x1.y, o1i));
            }
            out[0][r] = make_double2(o0r, o0i);
            out[1][r] = make_double2(o1r, o1i);
        }
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int r = 0; r < 4; ++r) a[idx[s][r]] = out[s][r];
    }
}

// Real 4x4 on register bits (K0, K1): a complex amplitude vector times a real
// matrix is two real matrix-vector products, half the FP64 work of a complex
// 4x4.  The 16 coefficients are read once and serve all four groups.
template <int K0, int K1>
__device__ __forceinline__ void reg_m2r(double2 (&a)[16], const double *__restrict__ c) {
    double m[16];
#pragma unroll
    for (int q = 0; q < 16; q += 2) {
        const double2 v = *reinterpret_cast<const double2 *>(c + q);
        m[q] = v.x;
        m[q + 1] = v.y;
    }
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if ((e & (1 << K0)) || (e & (1 << K1))) continue;
        const int i0 = e, i1 = e | (1 << K1), i2 = e | (1 << K0), i3 = e | (1 << K0) | (1 << K1);
        const double2 x0 = a[i0], x1 = a[i1], x2 = a[i2], x3 = a[i3];
        double2 o[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            o[r].x = fma(m[4 * r + 3], x3.x, fma(m[4 * r + 2], x2.x, fma(m[4 * r + 1], x1.x,
                                                                          m[4 * r] * x0.x)));
            o[r].y = fma(m[4 * r + 3], x3.y, fma(m[4 * r + 2], x2.y, fma(m[4 * r + 1], x1.y,
                                                                          m[4 * r] * x0.y)));
        }
        a[i0] = o[0];
        a[i1] = o[1];
        a[i2] = o[2];
        a[i3] = o[3];
    }
}

// Scaled real rotation on register bit K: one FMA per real output component,
// a quarter of a complex 2x2.  FORM 0: y0 = x0 - t x1, y1 = x1 + t x0;
// FORM 1: y0 = u x0 - x1, y1 = x0 + u x1.  (The scale the host factored out
// of the rotation travels in a diagonal table.)
template <int K, int FORM>
__device__ __forceinline__ void reg_r1s(double2 (&a)[16], double x) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if (e & (1 << K)) continue;
        const double2 x0 = a[e], x1 = a[e | (1 << K)];
        if (FORM == 0) {
            a[e] = make_double2(fma(-x, x1.x, x0.x), fma(-x, x1.y, x0.y));
            a[e | (1 << K)] = make_double2(fma(x, x0.x, x1.x), fma(x, x0.y, x1.y));
        } else {
            a[e] = make_double2(fma(x, x0.x, -x1.x), fma(x, x0.y, -x1.y));
            a[e | (1 << K)] = make_double2(fma(x, x1.x, x0.x), fma(x, x1.y, x0.y));
        }
    }
}

template <int FORM>
__device__ __forceinline__ void rot_s(double2 &y0, double2 &y1, double x) {
    const double2 x0 = y0, x1 = y1;
    if (FORM == 0) {
        y0 = make_double2(fma(-x, x1.x, x0.x), fma(-x, x1.y, x0.y));
        y1 = make_double2(fma(x, x0.x, x1.x), fma(x, x0.y, x1.y));
    } else {
        y0 = make_double2(fma(x, x0.x, -x1.x), fma(x, x0.y, -x1.y));
        y1 = make_double2(fma(x, x1.x, x0.x), fma(x, x1.y, x0.y));
    }
}

// A folded pair in real form: rotation on K1, rotation on K0, then the pair's
// permutation P written as the destination of each result (no extra moves).
// q = bit(K0) << 1 | bit(K1); P: 0 none, 1 CNOT K0->K1, 2 CNOT K1->K0, 3 SWAP.
template <int K0, int K1, int F0, int F1, int P>
__device__ __forceinline__ void reg_pair(double2 (&a)[16], double x0, double x1) {
    constexpr int perm[4][4] = {{0, 1, 2, 3}, {0, 1, 3, 2}, {0, 3, 2, 1}, {0, 2, 1, 3}};
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        if ((e & (1 << K0)) || (e & (1 << K1))) continue;
        const int i[4] = {e, e | (1 << K1), e | (1 << K0), e | (1 << K0) | (1 << K1)};
        double2 v[4] = {a[i[0]], a[i[1]], a[i[2]], a[i[3]]};
        rot_s<F1>(v[0], v[1], x1);
        rot_s<F1>(v[2], v[3], x1);
        rot_s<F0>(v[0], v[2], x0);
        rot_s<F0>(v[1], v[3], x0);
#pragma unroll
        for (int q = 0; q < 4; ++q) a[i[perm[P][q]]] = v[q];
    }
}

template <int K0, int K1>
__device__ __forceinline__ void reg_pair_dispatch(double2 (&a)[16], int code, double x0,
                                                  double x1) {
    // the planner emits both rotations in form 0; code >> 2 is the permutation
    switch (code >> 2) {
    case 0: reg_pair<K0, K1, 0, 0, 0>(a, x0, x1); break;
    case 1: reg_pair<K0, K1, 0, 0, 1>(a, x0, x1); break;
    case 2: reg_pair<K0, K1, 0, 0, 2>(a, x0, x1); break;
    default: reg_pair<K0, K1, 0, 0, 3>(a, x0, x1); break;
    }
}

// Diagonal over the register bits: one complex factor per register element,
// the product of every diagonal gate of the run (computed on the host).
__device__ __forceinline__ void reg_dtab(double2 (&a)[16], const double *__restrict__ c) {
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const double2 p = *reinterpret_cast<const double2 *>(c + 2 * e);
        const double2 v = a[e];
        a[e] = make_double2(fma(-v.y, p.y, v.x * p.x), fma(v.x, p.y, v.y * p.x));
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
                ore = fma(-mi, in[q].y, fma(mr, in[q].x, ore));
                oim = fma(mi, in[q].x, fma(mr, in[q].y, oim));
            }
            a[hiv + r] = make_double2(ore, oim);
        }
    }
}

// Diagonal op: every bit it reads comes from the element's global index
// gbase | goff(e), goff(e) = OR of gpos[k] over the set bits k of e.
__device__ __forceinline__ void reg_diag(double2 (&a)[16], const FusedOp &op,
                                         const double (&c)[8], uint64_t gbase,
                                         const uint64_t *__restrict__ gpp) {
    const uint64_t gp[4] = {gpp[0], gpp[1], gpp[2], gpp[3]};
    const uint64_t fm = op.fixmask;
    const int pb0 = op.pb0 < 0 ? 0 : op.pb0, pb1 = op.pb1 < 0 ? 0 : op.pb1;
    const uint64_t use0 = op.npat > 0 ? 1ull : 0ull, use1 = op.npat > 1 ? 1ull : 0ull;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const uint64_t gi = gbase | ((e & 1) ? gp[0] : 0ull) | ((e & 2) ? gp[1] : 0ull) |
                            ((e & 4) ? gp[2] : 0ull) | ((e & 8) ? gp[3] : 0ull);
        if ((gi & fm) != fm) continue;
        const int b0 = (int)((gi >> pb0) & use0), b1 = (int)((gi >> pb1) & use1);
        const double pr = b1 ? (b0 ? c[6] : c[4]) : (b0 ? c[2] : c[0]);
        const double pi = b1 ? (b0 ? c[7] : c[5]) : (b0 ? c[3] : c[1]);
        const double2 v = a[e];
        a[e] = make_double2(fma(-v.y, pi, v.x * pr), fma(v.x, pi, v.y * pr));
    }
}

// Apply one op.  c8 holds the op's first eight coefficients (prefetched by the
// caller); cfull points at all of them (4x4 and block ops read more).
// MODE 0: 2x2, X, diagonal and swap ops; 1: also 4x4 ops; 2: also 8x8 / 16x16
// block ops.
template <int MODE>
__device__ __forceinline__ void apply_fused_op(double2 (&a)[16], const FusedOp &op,
                                               const double (&c8)[8],
                                               const double *__restrict__ cfull, uint64_t gbase,
                                               const uint64_t *__restrict__ gp) {
    if ((gbase & op.gmask) != op.gmask) return;  // a control outside R is 0
    switch (op.type) {
    case F_M1:
        switch (op.k0) {
        case 0: reg_m1<0, false>(a, 0, c8); break;
        case 1: reg_m1<1, false>(a, 0, c8); break;
        case 2: reg_m1<2, false>(a, 0, c8); break;
        default: reg_m1<3, false>(a, 0, c8); break;
        }
        break;
    case F_M1C:
        switch (op.k0) {
        case 0: reg_m1<0, true>(a, op.cm, c8); break;
        case 1: reg_m1<1, true>(a, op.cm, c8); break;
        case 2: reg_m1<2, true>(a, op.cm, c8); break;
        default: reg_m1<3, true>(a, op.cm, c8); break;
        }
        break;
    case F_X:
        switch (op.k0) {
        case 0: reg_x<0, false>(a, 0); break;
        case 1: reg_x<1, false>(a, 0); break;
        case 2: reg_x<2, false>(a, 0); break;
        default: reg_x<3, false>(a, 0); break;
        }
        break;
    case F_XC:
        switch (op.k0) {
        case 0: reg_x<0, true>(a, op.cm); break;
        case 1: reg_x<1, true>(a, op.cm); break;
        case 2: reg_x<2, true>(a, op.cm); break;
        default: reg_x<3, true>(a, op.cm); break;
        }
        break;
    case F_DIAG:
        reg_diag(a, op, c8, gbase, gp);
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
    default:
        if constexpr (MODE >= 1) {
            if (op.type == F_M2) {
                // the encoder orders the register bits k0 < k1
                const int key = op.k0 * 4 + op.k1;
                switch (key) {
                case 1: reg_m2<0, 1>(a, cfull); break;
                case 2: reg_m2<0, 2>(a, cfull); break;
                case 3: reg_m2<0, 3>(a, cfull); break;
                case 6: reg_m2<1, 2>(a, cfull); break;
                case 7: reg_m2<1, 3>(a, cfull); break;
                default: reg_m2<2, 3>(a, cfull); break;
                }
            } else if (op.type == F_M2R) {
                const int key = op.k0 * 4 + op.k1;
                switch (key) {
                case 1: reg_m2r<0, 1>(a, cfull); break;
                case 2: reg_m2r<0, 2>(a, cfull); break;
                case 3: reg_m2r<0, 3>(a, cfull); break;
                case 6: reg_m2r<1, 2>(a, cfull); break;
                case 7: reg_m2r<1, 3>(a, cfull); break;
                default: reg_m2r<2, 3>(a, cfull); break;
                }
            } else if (op.type == F_DTAB) {
                // up to two non-register bits select one of the table's variants
                int v = 0;
                if (op.npat > 0) v = (int)((gbase >> op.pb0) & 1ull);
                if (op.npat > 1) v |= (int)((gbase >> op.pb1) & 1ull) << 1;
                reg_dtab(a, cfull + 32 * v);
            } else if (op.type == F_PAIR) {
                const double x0 = c8[0], x1 = c8[1];
                switch (op.k0 * 4 + op.k1) {
                case 1: reg_pair_dispatch<0, 1>(a, op.cm, x0, x1); break;
                case 2: reg_pair_dispatch<0, 2>(a, op.cm, x0, x1); break;
                case 3: reg_pair_dispatch<0, 3>(a, op.cm, x0, x1); break;
                case 6: reg_pair_dispatch<1, 2>(a, op.cm, x0, x1); break;
                case 7: reg_pair_dispatch<1, 3>(a, op.cm, x0, x1); break;
                default: reg_pair_dispatch<2, 3>(a, op.cm, x0, x1); break;
                }
            } else if (op.type == F_R1S) {
                const double x = c8[0];
                switch (op.k0 * 2 + op.k1) {
                case 0: reg_r1s<0, 0>(a, x); break;
                case 1: reg_r1s<0, 1>(a, x); break;
                case 2: reg_r1s<1, 0>(a, x); break;
                case 3: reg_r1s<1, 1>(a, x); break;
                case 4: reg_r1s<2, 0>(a, x); break;
                case 5: reg_r1s<2, 1>(a, x); break;
                case 6: reg_r1s<3, 0>(a, x); break;
                default: reg_r1s<3, 1>(a, x); break;
                }
            } else if constexpr (MODE >= 2) {
                if (op.type == F_BLOCK3) reg_block<3>(a, cfull);
                else reg_block<4>(a, cfull);
            }
        }
        break;
    }
}

// One round on a tile in shared memory: gather 16 registers per thread, run
// the round's ops (op descriptors and their first coefficients prefetched one
// op ahead), scatter back.  coef_of(op) returns the op's coefficient pointer.
template <int MODE, class CoefOf>
__device__ __forceinline__ void run_round(uint32_t tile_a, const FusedRound &rd,
                                          const FusedOp *__restrict__ ops, CoefOf coef_of,
                                          uint64_t tile_base, int h, int tid) {
    int tbase = 0;
    for (int j = 0; j < rd.nlane; ++j) tbase |= ((tid >> j) & 1) << rd.lane[j];
    // swizzled byte offset of the thread base (XOR-combined with the element
    // offsets; the tile address is added afterwards)
    const uint32_t sb = (uint32_t)swz(tbase) << 4;
    const uint64_t gbase = tile_base | (uint64_t)(tbase & 15) | ((uint64_t)(tbase >> 4) << h);
    double2 a[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const uint32_t addr = tile_a + (sb ^ (uint32_t)rd.eoff[e]);
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(a[e].x), "=d"(a[e].y) : "r"(addr));
    }
    if (rd.op_begin < rd.op_end) {
        FusedOp nxt = ops[rd.op_begin];
        const double *ncp = coef_of(nxt);
        double nc[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) nc[q] = ncp[q];
        for (int o = rd.op_begin; o < rd.op_end; ++o) {
            const FusedOp op = nxt;
            const double *cp = ncp;
            double cc[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) cc[q] = nc[q];
            if (o + 1 < rd.op_end) {
                nxt = ops[o + 1];
                ncp = coef_of(nxt);
#pragma unroll
                for (int q = 0; q < 8; ++q) nc[q] = ncp[q];
            }
            apply_fused_op<MODE>(a, op, cc, cp, gbase, rd.gpos);
        }
    }
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const uint32_t addr = tile_a + (sb ^ (uint32_t)rd.eoff[e]);
        asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(a[e].x), "d"(a[e].y)
                     : "memory");
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

}  // namespace lq
