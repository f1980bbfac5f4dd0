// Precision form: complex64 state, gates fused into 5-qubit blocks applied as
// complex 32x32 GEMMs on the 5th-generation tensor cores (tcgen05, TF32 inputs,
// FP32 accumulation in tensor memory) with the 3xTF32 split
//     X W ~= Xh Wh + Xh Wl + Xl Wh,   Xh = tf32(X), Xl = tf32(X - Xh).
//
// A pass owns a window of T = 12 index bits ([0,4) U [h, h+8), as the FP64
// fused passes) and applies its 5-qubit blocks to every 2^12-amplitude
// complex64 tile (32 KiB, TMA with 128-byte swizzle).  For a block on tile bits
// k0..k4 the tile is a 128 x 32 complex matrix X (rows: the other seven tile
// bits; columns: the block index).  Viewed as reals interleaved (re, im) it is
// X' (128 x 64) and the block is Y' = X' W' with the real 64 x 64 matrix
// W' = [[Re U^T, Im U^T], [-Im U^T, Re U^T]] interleaved the same way.
//
// Thread m owns GEMM row m, which is also tensor-memory lane m: it splits its
// row into TF32 hi / lo parts and writes them to tensor memory (tcgen05.st);
// one elected thread issues 3 x 8 tcgen05.mma (K = 8 each) with A read from
// tensor memory and B (W' hi / lo, prepared on the host in the swizzled K-major
// byte order and brought in by one bulk copy) from shared memory, into a
// 128-lane x 64-column FP32 accumulator; each thread reads its row back with
// tcgen05.ld and scatters it into the tile.  CTAs are persistent (two per SM:
// 97 KiB of shared memory and 256 tensor-memory columns each), prefetch their
// next tile into a second buffer and store finished tiles asynchronously.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <complex>
#include <cstring>
#include <mutex>

#include "fused_plan.h"

namespace lq {

constexpr int kTcT = 12;                  // tile bits
constexpr int kTcThreads = 128;           // thread m owns GEMM row m = TMEM lane m
constexpr uint32_t kTileBytes = 8u << kTcT;  // 32 KiB complex64 tile
constexpr uint32_t kBBytes = 64 * 64 * 4;    // 16 KiB per B part (hi / lo)
// shared memory: two tile buffers, B hi + lo, barriers
constexpr uint32_t kTcSmem = 2 * kTileBytes + 2 * kBBytes + 1024 + 128;
// tensor memory columns: D (FP32 accumulator) [0,64), A hi [64,128), A lo [128,192)
constexpr uint32_t kTmemCols = 256;
constexpr uint32_t kColD = 0, kColAh = 64, kColAl = 128;

struct TcBlock {
    int32_t k[5];     // tile-local bit of block bit j (block index bit j)
    int32_t pad[3];
    uint32_t row_bits[7];  // tile-local positions of the 7 row bits
    uint32_t pad2;
    uint64_t b_offset;  // offset (bytes) of this block's 32 KiB B image (hi then lo)
    uint32_t col_bits[32];  // tile-local index bits of block column c (its 5 bits placed)
};

static bool tc_restore_norm() {
    static const int v = [] {
        const char *e = getenv("LQ_TC_RENORM");
        return e ? atoi(e) : 1;
    }();
    return v != 0;
}

struct TcPass {
    int32_t h;
    int32_t block_begin, nblocks;
    int32_t pad;
};

__device__ __forceinline__ uint32_t tc_smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of complex64 tile element l in the TMA 128-byte-swizzled tile:
// 128-byte rows hold 16 amplitudes (bits 0-3); 16-byte chunks hold 2.
__device__ __forceinline__ uint32_t tile_off(uint32_t l) {
    const uint32_t row = l >> 4, chunk = (l & 15) >> 1;
    return row * 128 + ((chunk ^ (row & 7)) << 4) + ((l & 1) << 3);
}

// Round a finite FP32 value to TF32 (10 explicit mantissa bits), to nearest with
// ties away from zero: add half a unit of the last kept place (bit 12) to the
// IEEE bit pattern and clear the 13 dropped bits.  The pattern is
// sign-magnitude, so the same addition rounds negative values by magnitude, and
// a carry out of the mantissa steps into the next binade as rounding up should.
// Two integer operations instead of a conversion sequence that also handles
// NaN and infinity, which amplitudes (magnitude at most 1) never are.
__device__ __forceinline__ float to_tf32(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

__device__ __forceinline__ uint64_t make_sdesc(uint32_t addr, uint32_t sbo_bytes) {
    // tcgen05 shared-memory descriptor: start address >> 4 [0,14), leading
    // byte offset (unused for swizzled K-major, 1) [16,30), stride byte offset
    // >> 4 [32,46), version 1 [46,48), layout SWIZZLE_128B (2) [61,64).
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
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

// Instruction descriptor: D f32, A/B tf32, both K-major, N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, "
        "%10, %11, %12, %13, %14, %15, %16};" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
        "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
        "r"(__float_as_uint(v[15]))
        : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
        "%10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Persistent CTAs (two per SM), each walking tiles t = blockIdx.x, +gridDim.x.
// Per tile: TMA load (prefetched one tile ahead into the other buffer), then per
// 5-qubit block: B image (one bulk copy), A split into TF32 hi / lo written to
// tensor memory by the owning threads (row m = TMEM lane m), 3 x 8 tcgen05.mma
// with A from tensor memory, tcgen05.ld of the 128 x 64 FP32 result and scatter
// into the tile; finally an asynchronous TMA store, waited for only before its
// buffer is reloaded.
__global__ void __launch_bounds__(kTcThreads, 2)
    k_tc_pass(const __grid_constant__ CUtensorMap tmap, int32_t h, int32_t ntiles,
              const TcBlock *__restrict__ blocks, int nblocks,
              const unsigned char *__restrict__ bimg, unsigned *__restrict__ flag) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *tiles = base;                       // 2 x 32 KiB
    unsigned char *b_hi = tiles + 2 * kTileBytes;      // 16 KiB, then b_lo
    unsigned char *b_lo = b_hi + kBBytes;
    uint64_t *bars = (uint64_t *)(b_lo + kBBytes);     // [0],[1] tile loads, [2] B, [3] MMA
    uint32_t *tmem_slot = (uint32_t *)(bars + 4);
    int *s_abort = (int *)(tmem_slot + 1);
    const uint32_t bar_load0 = tc_smem_u32(&bars[0]);
    const uint32_t bar_b = tc_smem_u32(&bars[2]);
    const uint32_t bar_mma = tc_smem_u32(&bars[3]);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int32_t zero = 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         tc_smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < 4; ++i)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(&bars[i])),
                         "r"(1)
                         : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);

    auto issue_load = [&](int t, int buf) {
        const int32_t c1 = t & ((1 << (h - 4)) - 1), c3 = t >> (h - 4);
        const uint32_t bar = bar_load0 + 8u * buf;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(kTileBytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(tc_smem_u32(tiles + buf * kTileBytes)),
            "l"((uint64_t)&tmap), "r"(zero), "r"(c1), "r"(zero), "r"(c3), "r"(bar)
            : "memory");
    };

    // B hi + lo of block bi: one 32 KiB bulk copy of the host-prepared swizzled image
    auto issue_b = [&](int bi) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_b),
                     "r"(2 * kBBytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
            " [%0], [%1], %2, [%3];" ::"r"(tc_smem_u32(b_hi)),
            "l"((uint64_t)(bimg + blocks[bi].b_offset)), "r"(2 * kBBytes), "r"(bar_b)
            : "memory");
    };

    uint32_t load_phase[2] = {0u, 0u}, b_phase = 0u, mma_phase = 0u;
    bool load_pending[2] = {false, false};  // thread 0: a tile load not yet waited for
    bool mma_pending = false, b_pending = false;
    if (tid == 0 && (int)blockIdx.x < ntiles && nblocks > 0) {
        issue_b(0);
        b_pending = true;
    }
    int buf = 0;
    if (tid == 0 && (int)blockIdx.x < ntiles) {
        issue_load(blockIdx.x, 0);
        load_pending[0] = true;
    }
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (!tc_wait(bar_load0 + 8u * buf, load_phase[buf])) atomicExch(s_abort, 1);
        load_phase[buf] ^= 1u;
        if (tid == 0) load_pending[buf] = false;
        __syncthreads();
        if (*s_abort) break;
        const int tn = t + gridDim.x;
        if (tid == 0 && tn < ntiles) {
            // the other buffer's store (previous tile) must have left shared memory
            asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
            issue_load(tn, buf ^ 1);
            load_pending[buf ^ 1] = true;
        }
        unsigned char *tile = tiles + buf * kTileBytes;
        const uint32_t tile_a = tc_smem_u32(tile);
        for (int bi = 0; bi < nblocks; ++bi) {
            const TcBlock &blk = blocks[bi];
            // (this block's B image was requested when the previous block's MMAs
            // had finished reading the buffer, or before the first tile)
            // A row m = tid: the block's 32 complex entries, split hi / lo into TMEM
            uint32_t lbase = 0;
#pragma unroll
            for (int j = 0; j < 7; ++j) lbase |= (((uint32_t)tid >> j) & 1u) << blk.row_bits[j];
            // tile_off is linear over XOR on disjoint bits: the offset of column c is
            // the XOR of the offsets of its five block bits (five loads, not 32)
            const uint32_t rowoff = tile_off(lbase);
            const uint32_t cb0 = tile_off(1u << blk.k[0]), cb1 = tile_off(1u << blk.k[1]),
                           cb2 = tile_off(1u << blk.k[2]), cb3 = tile_off(1u << blk.k[3]),
                           cb4 = tile_off(1u << blk.k[4]);
            auto col_off = [&](int c) {
                return ((c & 1) ? cb0 : 0u) ^ ((c & 2) ? cb1 : 0u) ^ ((c & 4) ? cb2 : 0u) ^
                       ((c & 8) ? cb3 : 0u) ^ ((c & 16) ? cb4 : 0u);
            };
            // Block bit 0 on tile bit 0: columns 2c, 2c+1 share a 16-byte chunk
            // (one 128-bit access for both, and the lane bits then cover the
            // chunk slots without bank conflicts).
            const bool pair = blk.k[0] == 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float hi[16], lo[16];
#pragma unroll
                for (int c = 0; c < 8; c += 2) {
                    float4 v;
                    if (pair) {
                        v = *(const float4 *)(tile + (rowoff ^ col_off(q * 8 + c)));
                    } else {
                        const float2 v0 = *(const float2 *)(tile + (rowoff ^ col_off(q * 8 + c)));
                        const float2 v1 =
                            *(const float2 *)(tile + (rowoff ^ col_off(q * 8 + c + 1)));
                        v = make_float4(v0.x, v0.y, v1.x, v1.y);
                    }
                    const float x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const float hx = to_tf32(x[u]);
                        hi[2 * c + u] = hx;
                        lo[2 * c + u] = to_tf32(x[u] - hx);
                    }
                }
                tmem_st16(lane_base + kColAh + q * 16, hi);
                tmem_st16(lane_base + kColAl + q * 16, lo);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (tid == 0) {
                if (!tc_wait(bar_b, b_phase)) {
                    atomicExch(s_abort, 1);
                } else {
                    b_pending = false;
                    const uint32_t bh = tc_smem_u32(b_hi), bl = tc_smem_u32(b_lo);
#pragma unroll
                    for (int prod = 0; prod < 3; ++prod) {
                        // hi.Bhi + hi.Blo + lo.Bhi
                        const uint32_t acol = prod == 2 ? kColAl : kColAh;
                        const uint32_t bsrc = prod == 1 ? bl : bh;
#pragma unroll
                        for (int kk = 0; kk < 8; ++kk) {
                            const uint32_t boff = (kk >> 2) * (64 * 128) + (kk & 3) * 32;
                            const uint64_t db = make_sdesc(bsrc + boff, 1024);
                            const uint32_t acc = (prod | kk) ? 1u : 0u;
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::
                                    "r"(tmem + kColD),
                                "r"(tmem + acol + kk * 8), "l"(db), "r"(kIdesc), "r"(acc)
                                : "memory");
                        }
                    }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                        "[%0];" ::"r"(bar_mma)
                        : "memory");
                    mma_pending = true;
                }
                b_phase ^= 1u;
            }
            __syncthreads();
            if (*s_abort) break;
            // every thread decides to stop only after the barrier, so the CTA
            // leaves the loop together
            if (!tc_wait(bar_mma, mma_phase)) atomicExch(s_abort, 1);
            __syncthreads();
            if (*s_abort) break;
            mma_phase ^= 1u;
            if (tid == 0) {
                mma_pending = false;
                // the MMAs have read B: request the next block's image now, so the
                // copy overlaps this block's readback and the next block's split
                const int nb = bi + 1 < nblocks ? bi + 1 : 0;
                if (bi + 1 < nblocks || t + (int)gridDim.x < ntiles) {
                    issue_b(nb);
                    b_pending = true;
                }
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // D row m = tid back into the tile
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float d[16];
                tmem_ld16(lane_base + kColD + q * 16, d);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int c = 0; c < 8; c += 2) {
                    unsigned char *p0 = tile + (rowoff ^ col_off(q * 8 + c));
                    if (pair) {
                        *(float4 *)p0 = make_float4(d[2 * c], d[2 * c + 1], d[2 * c + 2],
                                                    d[2 * c + 3]);
                    } else {
                        *(float2 *)p0 = make_float2(d[2 * c], d[2 * c + 1]);
                        *(float2 *)(tile + (rowoff ^ col_off(q * 8 + c + 1))) =
                            make_float2(d[2 * c + 2], d[2 * c + 3]);
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
        }
        if (*s_abort) break;
        // tile -> HBM (asynchronous; waited for before this buffer is reloaded)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            const int32_t c1 = t & ((1 << (h - 4)) - 1), c3 = t >> (h - 4);
            asm volatile(
                "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group"
                " [%0, {%1, %2, %3, %4}], [%5];" ::"l"((uint64_t)&tmap),
                "r"(zero), "r"(c1), "r"(zero), "r"(c3), "r"(tile_a)
                : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
        buf ^= 1;
    }
    if (tid == 0) {
        if (*s_abort) {
            atomicOr(flag, kFlagTimeout);
            // let work in flight finish before the CTA's memory is released
            if (mma_pending) tc_wait(bar_mma, mma_phase);
            if (b_pending) tc_wait(bar_b, b_phase);
            for (int b = 0; b < 2; ++b)
                if (load_pending[b]) tc_wait(bar_load0 + 8u * b, load_phase[b]);
        }
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols)
                     : "memory");
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 tc_encode() {
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

// complex64 tile map for the window [0,4) U [h, h+8):
//   dim0: 32 floats (16 amplitudes, bits 0-3), box 32 (128 B)
//   dim1: 2^(h-4) (bits 4..h-1), box 1
//   dim2: 2^8 (bits h..h+7), box 256
//   dim3: 2^(n-h-8) (bits h+8..), box 1
static int tc_tile_map(CUtensorMap *map, void *d, int n, int h) {
    auto enc = tc_encode();
    if (!enc) return set_error(LQ_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    cuuint64_t dims[4] = {32, 1ull << (h - 4), 256, 1ull << (n - h - 8)};
    cuuint64_t strides[3] = {128, 8ull << h, 8ull << (h + 8)};
    cuuint32_t box[4] = {32, 1, 256, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, d, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return set_error(LQ_ERR_CUDA, "cuTensorMapEncodeTiled (complex64) failed (%d)", (int)r);
    return LQ_OK;
}

using cd = std::complex<double>;

// SM count of the current device (persistent grid: two CTAs per SM).
static int tc_sm_count() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(sms, 1);
}

// Apply canonical op g (global index bits) to a 32-dim vector whose block bit j
// corresponds to global bit gbit[j].
static void small_apply(const GateOp &g, const int gbit[5], cd *v) {
    auto loc = [&](int b) {
        for (int j = 0; j < 5; ++j)
            if (gbit[j] == b) return j;
        return -1;
    };
    auto c = [&](int k) { return cd(g.m[2 * k], g.m[2 * k + 1]); };
    switch (g.type) {
    case OP_M1:
    case OP_PERM1: {
        const int t = loc(g.t);
        int cm = 0;
        for (int k = 0; k < g.nctrl; ++k) cm |= 1 << loc(g.ctrl[k]);
        for (int e = 0; e < 32; ++e) {
            if ((e >> t) & 1) continue;
            if ((e & cm) != cm) continue;
            const int f = e | (1 << t);
            const cd a0 = v[e], a1 = v[f];
            if (g.type == OP_PERM1) {
                v[e] = a1;
                v[f] = a0;
            } else {
                v[e] = c(0) * a0 + c(1) * a1;
                v[f] = c(2) * a0 + c(3) * a1;
            }
        }
        break;
    }
    case OP_DIAG: {
        int fm = 0;
        for (int k = 0; k < g.nfix; ++k) fm |= 1 << loc(g.fix[k]);
        for (int e = 0; e < 32; ++e) {
            if ((e & fm) != fm) continue;
            int pat = 0;
            for (int k = 0; k < g.npat; ++k) pat |= ((e >> loc(g.pat[k])) & 1) << k;
            v[e] *= c(pat);
        }
        break;
    }
    case OP_SWAP: {
        const int a = loc(g.b0), b = loc(g.b1);
        for (int e = 0; e < 32; ++e)
            if (((e >> a) & 1) && !((e >> b) & 1)) std::swap(v[e], v[e ^ (1 << a) ^ (1 << b)]);
        break;
    }
    case OP_M2: {
        const int a = loc(g.b0), b = loc(g.b1);
        for (int e = 0; e < 32; ++e) {
            if (((e >> a) & 1) || ((e >> b) & 1)) continue;
            const int idx[4] = {e, e | (1 << b), e | (1 << a), e | (1 << a) | (1 << b)};
            cd in[4], out[4];
            for (int r = 0; r < 4; ++r) in[r] = v[idx[r]];
            for (int r = 0; r < 4; ++r) {
                out[r] = 0;
                for (int q = 0; q < 4; ++q) out[r] += cd(g.m[(r * 4 + q) * 2], g.m[(r * 4 + q) * 2 + 1]) * in[q];
            }
            for (int r = 0; r < 4; ++r) v[idx[r]] = out[r];
        }
        break;
    }
    }
}

static inline float host_tf32(double x) {
    // round-to-nearest (ties away) to a 10-bit mantissa, as cvt.rna.tf32.f32
    float f = (float)x;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) {
        u += 0x1000u;
        u &= 0xffffe000u;
    }
    memcpy(&f, &u, 4);
    return f;
}

// Swizzled byte image of B (N x K K-major, two K atoms of 64 rows x 128 B).
static void write_b_image(const double W[64][64], unsigned char *hi, unsigned char *lo) {
    for (int n = 0; n < 64; ++n)
        for (int k = 0; k < 64; ++k) {
            const int atom = k >> 5, kb = (k & 31) * 4;
            const size_t off = (size_t)atom * 64 * 128 + n * 128 + (((kb >> 4) ^ (n & 7)) << 4) +
                               (kb & 15);
            const double w = W[k][n];
            const float h = host_tf32(w);
            const float l = host_tf32(w - (double)h);
            memcpy(hi + off, &h, 4);
            memcpy(lo + off, &l, 4);
        }
}

struct TcPlan {
    std::vector<PlanStep> steps;  // fused steps reuse the window; blocks below
    std::vector<std::vector<std::vector<int>>> pass_blocks;  // per fused step: blocks of gates
    std::vector<std::vector<std::vector<int>>> block_bits;   // per step/block: 5 global bits
};

// Split each window pass into 5-bit blocks: greedy in order, a gate joins the
// open block when all its bits fit in <= 5 bits and no earlier skipped gate
// shares a bit.
static void tc_blocks(const std::vector<GateOp> &gops, const std::vector<int> &gates, int h,
                      int T, std::vector<std::vector<int>> &blocks,
                      std::vector<std::vector<int>> &bits) {
    const int P = (int)gates.size();
    std::vector<char> sched(P, 0);
    int left = P;
    while (left > 0) {
        uint64_t B = 0, blk = 0;
        std::vector<int> cur;
        for (int k = 0; k < P; ++k) {
            if (sched[k]) continue;
            const uint64_t gb = op_bits(gops[gates[k]]);
            if ((gb & blk) == 0 && __builtin_popcountll(B | gb) <= 5) {
                B |= gb;
                cur.push_back(gates[k]);
                sched[k] = 1;
                --left;
            } else {
                blk |= gb;
            }
        }
        std::vector<int> bv;
        for (int b = 0; b < 64; ++b)
            if (B >> b & 1) bv.push_back(b);
        // pad to five bits of the window
        const uint64_t W = window_mask(h, T - 4);
        for (int b = 0; b < 64 && bv.size() < 5; ++b)
            if ((W >> b & 1) && !(B >> b & 1)) bv.push_back(b);
        std::sort(bv.begin(), bv.end());
        blocks.push_back(cur);
        bits.push_back(bv);
    }
}

int apply_circuit_tc_impl(lq_state *s, const lq_gate *ops, int nops, const double *theta,
                          int ntheta, int *nblocks_out, int *npasses_out) {
    const int n = s->n;
    if (s->dtype != LQ_C64)
        return set_error(LQ_ERR_UNSUPPORTED, "the tensor-core path runs on complex64 states");
    if (n < kTcT) return set_error(LQ_ERR_UNSUPPORTED, "the tensor-core path needs >= 12 qubits");
    std::vector<GateOp> gops(nops);
    for (int i = 0; i < nops; ++i) {
        LQ_TRY(validate_gate(&ops[i], n, ntheta));
        LQ_TRY(make_gate_op(&ops[i], theta, n, &gops[i]));
        if (gops[i].renorm)
            return set_error(LQ_ERR_UNSUPPORTED, "renormalising gates are not fused on tensor cores");
    }
    // Windows: the FP64 planner with every gate required fully inside the window
    // (dense blocks cannot read controls outside it).
    std::vector<GateOp> planner_ops = gops;
    for (auto &g : planner_ops) {
        // make every bit a mixed bit for window selection: widen to a 4x4-like op
        if (g.type == OP_DIAG || g.nctrl > 0 || g.type == OP_PERM1) {
            GateOp w = g;
            w.type = OP_M2;
            const uint64_t b = op_bits(g);
            int bits[3], nb = 0;
            for (int k = 0; k < 64 && nb < 3; ++k)
                if (b >> k & 1) bits[nb++] = k;
            if (nb == 1) {
                w.type = OP_M1;
                w.t = bits[0];
                w.nctrl = 0;
            } else if (nb == 2) {
                w.b0 = bits[0];
                w.b1 = bits[1];
            } else {
                return set_error(LQ_ERR_UNSUPPORTED, "3-qubit gates are not fused on tensor cores");
            }
            w.nfix = w.npat = 0;
            g = w;
        }
    }
    std::vector<PlanStep> steps = plan_circuit(planner_ops, n, kTcT);
    std::vector<TcBlock> blocks;
    std::vector<TcPass> passes;
    std::vector<unsigned char> bimg;
    std::vector<int> step_pass(steps.size(), -1);
    for (size_t si = 0; si < steps.size(); ++si) {
        const PlanStep &st = steps[si];
        if (!st.fused) continue;
        std::vector<std::vector<int>> bl, bb;
        tc_blocks(gops, st.pass.gates, st.pass.h, kTcT, bl, bb);
        TcPass tp{st.pass.h, (int)blocks.size(), (int)bl.size(), 0};
        for (size_t b = 0; b < bl.size(); ++b) {
            int gbit[5];
            for (int j = 0; j < 5; ++j) gbit[j] = bb[b][j];
            // A block on tile bit 0 takes it as its block bit 0: columns 2c and
            // 2c+1 are then the two halves of one 16-byte chunk, read and written
            // as a pair.  U is built in this bit order, so the order is free.
            for (int j = 1; j < 5; ++j)
                if (local_pos(gbit[j], st.pass.h) == 0) std::swap(gbit[0], gbit[j]);
            // block unitary U (32 x 32): column e = product of gates on basis e
            cd U[32][32];
            for (int e = 0; e < 32; ++e) {
                cd v[32] = {};
                v[e] = 1.0;
                for (int gi : bl[b]) small_apply(gops[gi], gbit, v);
                for (int r = 0; r < 32; ++r) U[r][e] = v[r];
            }
            double W[64][64];
            for (int r = 0; r < 32; ++r)
                for (int c = 0; c < 32; ++c) {
                    W[2 * c][2 * r] = U[r][c].real();
                    W[2 * c + 1][2 * r] = -U[r][c].imag();
                    W[2 * c][2 * r + 1] = U[r][c].imag();
                    W[2 * c + 1][2 * r + 1] = U[r][c].real();
                }
            TcBlock tb{};
            for (int j = 0; j < 5; ++j) tb.k[j] = local_pos(gbit[j], st.pass.h);
            for (int c = 0; c < 32; ++c) {
                tb.col_bits[c] = 0;
                for (int j = 0; j < 5; ++j) tb.col_bits[c] |= (uint32_t)((c >> j) & 1) << tb.k[j];
            }
            // Row bits: thread m's bit j goes to tile bit row_bits[j].  The row order
            // is free (each thread writes back the row it read), so the five lane
            // bits (j < 5) take tile bits whose 8-byte bank slots in the swizzled
            // tile are linearly independent: slot(l) = (l0, l1^l4, l2^l5, l3^l6), so
            // tile bit b moves slot bit (b < 4 ? b : b - 3) for b < 7 and none above.
            // Up to 16 distinct slots per warp access = the two-wavefront minimum.
            std::vector<int> free_bits;
            for (int l = 0; l < kTcT; ++l) {
                bool inb = false;
                for (int j = 0; j < 5; ++j) inb |= tb.k[j] == l;
                if (!inb) free_bits.push_back(l);
            }
            auto slot_vec = [](int b) { return b < 7 ? 1u << (b < 4 ? b : b - 3) : 0u; };
            std::vector<int> order;
            std::vector<uint32_t> basis;  // reduced slot vectors of the chosen lane bits
            for (int b : free_bits) {
                uint32_t v = slot_vec(b);
                for (uint32_t e : basis)
                    if ((v ^ e) < v) v ^= e;
                if (v && order.size() < 5) {
                    basis.push_back(v);
                    std::sort(basis.rbegin(), basis.rend());
                    order.push_back(b);
                }
            }
            for (int b : free_bits)
                if (std::find(order.begin(), order.end(), b) == order.end()) order.push_back(b);
            for (int j = 0; j < 7; ++j) tb.row_bits[j] = (uint32_t)order[j];
            tb.b_offset = bimg.size();
            bimg.resize(bimg.size() + 2 * kBBytes);
            write_b_image(W, bimg.data() + tb.b_offset, bimg.data() + tb.b_offset + kBBytes);
            blocks.push_back(tb);
        }
        step_pass[si] = (int)passes.size();
        passes.push_back(tp);
    }
    const size_t bsz = blocks.size() * sizeof(TcBlock);
    auto al = [](size_t x) { return (x + 1023) / 1024 * 1024; };
    LQ_TRY(ensure_prog(s, al(bsz) + al(bimg.size()) + 1024));
    TcBlock *d_blocks = (TcBlock *)s->d_prog;
    unsigned char *d_bimg = (unsigned char *)s->d_prog + al(bsz);
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (bsz) LQ_CUDA_TRY(cudaMemcpy(d_blocks, blocks.data(), bsz, cudaMemcpyHostToDevice));
    if (!bimg.empty())
        LQ_CUDA_TRY(cudaMemcpy(d_bimg, bimg.data(), bimg.size(), cudaMemcpyHostToDevice));
    static bool attr = false;
    if (!attr) {
        LQ_CUDA_TRY(cudaFuncSetAttribute(k_tc_pass, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmem));
        attr = true;
    }
    // FP32 accumulation in the tensor cores rounds every block's sums toward
    // zero, which shrinks the state by a near-uniform factor per block; the
    // FP64 norm of the input is restored at the end of the circuit (one
    // reduction before, one reduction and one scaling sweep after).
    const bool restore = tc_restore_norm() && !blocks.empty();
    if (restore) LQ_TRY(norm_snapshot(s));
    int launches = 0;
    for (size_t si = 0; si < steps.size(); ++si) {
        const PlanStep &st = steps[si];
        if (!st.fused) {
            LQ_TRY(launch_gate_op(s, gops[st.gate]));
            if (restore && gops[st.gate].renorm) LQ_TRY(norm_snapshot(s));
            continue;
        }
        const TcPass &tp = passes[step_pass[si]];
        CUtensorMap map;
        LQ_TRY(tc_tile_map(&map, s->d, n, tp.h));
        const int ntiles = 1 << (n - kTcT);
        prof_begin(s->stream, kProfTc);
        k_tc_pass<<<std::min(ntiles, 2 * tc_sm_count()), kTcThreads, kTcSmem, s->stream>>>(
            map, tp.h, ntiles, d_blocks + tp.block_begin, tp.nblocks, d_bimg, s->d_flag);
        prof_end(s->stream, kProfTc);
        LQ_CUDA_TRY(cudaGetLastError());
        ++launches;
    }
    if (restore) LQ_TRY(norm_restore(s));
    if (nblocks_out) *nblocks_out = (int)blocks.size();
    if (npasses_out) *npasses_out = launches;
    return LQ_OK;
}

}  // namespace lq

using namespace lq;

extern "C" {

int lq_apply_circuit_tc(lq_state *s, int circuit_qubits, const lq_gate *ops, int nops,
                        const double *theta, int ntheta, int *blocks, int *passes) {
    LQ_TRY(check_state(s));
    if (circuit_qubits != s->n)
        return set_error(LQ_ERR_QUBIT_MISMATCH,
                         "Circuit qubit count mismatch: circuit has %d, state has %d",
                         circuit_qubits, s->n);
    if (nops < 0 || (nops > 0 && !ops)) return set_error(LQ_ERR_INVALID_ARG, "bad op list");
    if (ntheta < 0 || (ntheta > 0 && !theta)) return set_error(LQ_ERR_INVALID_ARG, "bad theta");
    return apply_circuit_tc_impl(s, ops, nops, theta, ntheta, blocks, passes);
}

}  // extern "C"
