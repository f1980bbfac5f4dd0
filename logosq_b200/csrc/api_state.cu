// State lifecycle, host<->device transfers and FP64 reductions.
//
// Reference: src/states/mod.rs (State, normalize, probabilities,
// inner_product_parallel, measure*) and src/optimization/observable.rs
// (PauliTerm::expectation, PauliObservable::expectation).

#include <algorithm>
#include <cstdarg>
#include <map>
#include <mutex>

#include "lq_internal.h"

namespace lq {

static thread_local std::string g_last_error;
static uint64_t g_alloc_limit = 0;
static std::mutex g_alloc_mu;
static uint64_t g_alloc_in_use = 0;

int set_error(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

int check_state(const lq_state *s) {
    if (!s) return set_error(LQ_ERR_INVALID_ARG, "null state handle");
    if (!s->d) return set_error(LQ_ERR_INVALID_ARG, "state handle has no device buffer");
    return LQ_OK;
}

int check_qubit(const lq_state *s, int q) {
    if (q < 0 || q >= s->n)
        return set_error(LQ_ERR_QUBIT_INDEX, "Invalid qubit index: %d (must be < %d)", q, s->n);
    return LQ_OK;
}

int ensure_prog(lq_state *s, size_t bytes) {
    s->prog_valid = false;  // the caller is about to write the buffer
    if (s->prog_cap >= bytes) return LQ_OK;
    if (s->d_prog) {
        LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
        LQ_CUDA_TRY(cudaFree(s->d_prog));
        s->d_prog = nullptr;
        s->prog_cap = 0;
    }
    size_t cap = std::max<size_t>(bytes, 1 << 16);
    LQ_CUDA_TRY(cudaMalloc(&s->d_prog, cap));
    s->prog_cap = cap;
    return LQ_OK;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// Waits, with the given bound, on an mbarrier phase that never completes (the
// barrier expects one arrival and gets none; no copy targets it), then raises
// the timeout flag: the same give-up path as the pipeline waits of the fused
// and tensor-core passes, exercised without any copy in flight.
__global__ void k_wait_probe(unsigned *__restrict__ flag, unsigned polls) {
    __shared__ __align__(8) uint64_t bar;
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(&bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t done = 0;
    for (unsigned it = 0; it < polls && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(0u)
            : "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0 && !done) atomicOr(flag, kFlagTimeout);
}

template <class A>
__device__ __forceinline__ double2 load_amp(const A *v, uint64_t i);
template <>
__device__ __forceinline__ double2 load_amp<double2>(const double2 *v, uint64_t i) {
    return v[i];
}
template <>
__device__ __forceinline__ double2 load_amp<float2>(const float2 *v, uint64_t i) {
    float2 a = v[i];
    return make_double2(a.x, a.y);
}

// Block-wide sum of NC doubles; result valid in thread 0.
template <int NC>
__device__ __forceinline__ void block_sum(double (&x)[NC], double *sh /* 32*NC */) {
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x[c] += __shfl_down_sync(0xffffffffu, x[c], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < NC; ++c) sh[warp * NC + c] = x[c];
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            x[c] = lane < nw ? sh[lane * NC + c] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x[c] += __shfl_down_sync(0xffffffffu, x[c], o);
        }
    }
}

template <class A>
__global__ void k_norm_partial(const A *__restrict__ v, uint64_t N, double *partials) {
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 a = load_amp(v, i);
        acc[0] += a.x * a.x + a.y * a.y;
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

template <class A>
__global__ void k_inner_partial(const A *__restrict__ a, const A *__restrict__ b, uint64_t N,
                                double *partials) {
    __shared__ double sh[64];
    double acc[2] = {0.0, 0.0};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 x = load_amp(a, i), y = load_amp(b, i);
        // conj(x) * y
        acc[0] += x.x * y.x + x.y * y.y;
        acc[1] += x.x * y.y - x.y * y.x;
    }
    block_sum<2>(acc, sh);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = acc[0];
        partials[2 * blockIdx.x + 1] = acc[1];
    }
}

// Sum nparts partials of NC components in a fixed order (deterministic).
template <int NC>
__global__ void k_final_sum(const double *partials, int nparts, double *out) {
    __shared__ double sh[32 * NC];
    double acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = 0.0;
    for (int p = threadIdx.x; p < nparts; p += blockDim.x)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] += partials[p * NC + c];
    block_sum<NC>(acc, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int c = 0; c < NC; ++c) out[c] = acc[c];
}

// State::normalize: divide by sqrt(norm_sqr) when the norm exceeds 1e-10.
template <class A>
__global__ void k_scale_by_norm(A *__restrict__ v, uint64_t N, const double *norm_sqr) {
    const double norm = sqrt(*norm_sqr);
    if (!(norm > 1e-10)) return;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        A a = v[i];
        a.x = a.x / norm;
        a.y = a.y / norm;
        v[i] = a;
    }
}

// v *= sqrt(target / current) (both squared norms, FP64, on the device).
template <class A>
__global__ void k_scale_to_norm(A *__restrict__ v, uint64_t N, const double *target_sq,
                                const double *current_sq) {
    if (!(*current_sq > 0.0) || !(*target_sq > 0.0)) return;
    const double f = sqrt(*target_sq / *current_sq);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        A a = v[i];
        a.x = (decltype(a.x))(a.x * f);
        a.y = (decltype(a.y))(a.y * f);
        v[i] = a;
    }
}

template <class A>
__global__ void k_set_basis(A *__restrict__ v, uint64_t N, uint64_t idx) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        A a;
        a.x = i == idx ? 1 : 0;
        a.y = 0;
        v[i] = a;
    }
}

template <class A>
__global__ void k_set_const(A *__restrict__ v, uint64_t N, double re) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        A a;
        a.x = re;
        a.y = 0;
        v[i] = a;
    }
}

// |a> (x) |b>: out[i * Nb + j] = a[i] * b[j] (src/states/mod.rs:298-314).
template <class A>
__global__ void k_kron(A *__restrict__ out, const A *__restrict__ a, const A *__restrict__ b,
                       int nb, uint64_t N) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < N;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const A x = a[k >> nb], y = b[k & ((1ull << nb) - 1)];
        A o;
        o.x = x.x * y.x - x.y * y.y;
        o.y = x.x * y.y + x.y * y.x;
        out[k] = o;
    }
}

__global__ void k_c128_to_c64(const double2 *__restrict__ src, float2 *__restrict__ dst,
                              uint64_t N) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 a = src[i];
        dst[i] = make_float2((float)a.x, (float)a.y);
    }
}

template <class A>
__global__ void k_probs(const A *__restrict__ v, double *__restrict__ p, uint64_t N) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 a = load_amp(v, i);
        p[i] = a.x * a.x + a.y * a.y;
    }
}

// Pauli-sum expectation for one group of terms sharing the same X mask.
// For every basis index i the group contributes
//     Re W_i * alpha(i) + Im W_i * beta(i),   W_i = conj(psi_i) psi_{i^x},
// with alpha(i) = sum_t c_t a_t s_t(i), beta(i) = sum_t c_t b_t s_t(i),
// s_t(i) = (-1)^popcount(i & z_t) and (a_t, b_t) the real/imag selectors of
// Re(Y^ny z) = a Re z + b Im z.  When x != 0 each unordered pair (i, i^x) is
// visited once (the i with the top bit of x clear) and adds both orientations.
struct TermCoef {
    uint64_t z;
    double ca;  // c_t * a_t
    double cb;  // c_t * b_t
};

template <class A>
__global__ void k_pauli_group(const A *__restrict__ v, int n, uint64_t xmask,
                              const TermCoef *__restrict__ tc, int nt, double *partials) {
    extern __shared__ TermCoef s_tc[];
    __shared__ double sh[32];
    for (int t = threadIdx.x; t < nt; t += blockDim.x) s_tc[t] = tc[t];
    __syncthreads();
    double acc[1] = {0.0};
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // The grid-stride loops take kU steps at a time with every load issued
    // first (kU amplitudes, or kU pairs, in flight per thread); each thread
    // still adds its steps in the same order.
    constexpr int kU = 4;
    if (xmask == 0) {
        const uint64_t N = 1ull << n;
        auto add = [&](uint64_t i, double2 a) {
            double alpha = 0.0;
            for (int t = 0; t < nt; ++t) {
                const double s = (__popcll(i & s_tc[t].z) & 1) ? -1.0 : 1.0;
                alpha += s * s_tc[t].ca;
            }
            acc[0] += (a.x * a.x + a.y * a.y) * alpha;
        };
        uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
        for (; i + (kU - 1) * stride < N; i += kU * stride) {
            double2 a[kU];
#pragma unroll
            for (int k = 0; k < kU; ++k) a[k] = load_amp(v, i + k * stride);
#pragma unroll
            for (int k = 0; k < kU; ++k) add(i + k * stride, a[k]);
        }
        for (; i < N; i += stride) add(i, load_amp(v, i));
    } else {
        const int hb = 63 - __clzll(xmask);
        const uint64_t npairs = 1ull << (n - 1);
        const uint64_t lo_mask = (1ull << hb) - 1;
        auto pair_index = [&](uint64_t p) { return ((p & ~lo_mask) << 1) | (p & lo_mask); };
        auto add = [&](uint64_t i, double2 a, double2 b) {
            // W_i = conj(a) b ; W_j = conj(W_i), j = i ^ xmask.  The j-side sums
            // follow from the i side: a term's Z sign at j is its sign at i times
            // (-1)^ny, and ca = 0 for odd ny, cb = 0 for even ny, so
            // al_j = al_i and be_j = -be_i.
            const double wr = a.x * b.x + a.y * b.y;
            const double wi = a.x * b.y - a.y * b.x;
            double al_i = 0.0, be_i = 0.0;
            for (int t = 0; t < nt; ++t) {
                const double si = (__popcll(i & s_tc[t].z) & 1) ? -1.0 : 1.0;
                al_i += si * s_tc[t].ca;
                be_i += si * s_tc[t].cb;
            }
            acc[0] += 2.0 * (wr * al_i + wi * be_i);
        };
        uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
        for (; p + (kU - 1) * stride < npairs; p += kU * stride) {
            double2 a[kU], b[kU];
#pragma unroll
            for (int k = 0; k < kU; ++k) {
                const uint64_t i = pair_index(p + k * stride);
                a[k] = load_amp(v, i);
                b[k] = load_amp(v, i ^ xmask);
            }
#pragma unroll
            for (int k = 0; k < kU; ++k) add(pair_index(p + k * stride), a[k], b[k]);
        }
        for (; p < npairs; p += stride) {
            const uint64_t i = pair_index(p);
            add(i, load_amp(v, i), load_amp(v, i ^ xmask));
        }
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

// Terms without X bits (one group, X mask 0), for states of 12 or more qubits,
// launched with 256 threads.  A block takes 4096-amplitude chunks; thread tid
// handles the 16 indices i = chunk | k << 8 | tid, k = 0..15.  A term's sign
// (-1)^popcount(i & z) is the sign of the bits the thread keeps fixed (chunk
// and tid) times (-1)^popcount(k & p), p = bits 8-11 of z.  The terms arrive
// sorted by p (pbeg[p] .. pbeg[p+1]), so each thread folds all of them into 16
// coefficients C[p], and one 16-point Walsh-Hadamard transform of C gives the
// sum of signed coefficients for all 16 k: a few operations per amplitude
// instead of a popcount and a select per term per amplitude.
template <class A>
__global__ void __launch_bounds__(256, 2)
    k_pauli_zfold(const A *__restrict__ v, int n, const TermCoef *__restrict__ tc, int nt,
                  const int *__restrict__ pbeg, double *partials) {
    extern __shared__ TermCoef s_tc[];
    __shared__ double sh[32];
    __shared__ int s_pbeg[17];
    for (int t = threadIdx.x; t < nt; t += blockDim.x) s_tc[t] = tc[t];
    if (threadIdx.x < 17) s_pbeg[threadIdx.x] = pbeg[threadIdx.x];
    __syncthreads();
    double acc[1] = {0.0};
    const uint64_t nchunks = 1ull << (n - 12);
    for (uint64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const uint64_t fixed = (c << 12) | (uint64_t)threadIdx.x;
        double pr[16];  // |a|^2 of the 16 amplitudes
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const double2 a = load_amp(v, fixed | ((uint64_t)k << 8));
            pr[k] = a.x * a.x + a.y * a.y;
        }
        double C[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            double cq = 0.0;
            for (int t = s_pbeg[q]; t < s_pbeg[q + 1]; ++t)
                cq += (__popcll(fixed & s_tc[t].z) & 1) ? -s_tc[t].ca : s_tc[t].ca;
            C[q] = cq;
        }
#pragma unroll
        for (int hs = 1; hs < 16; hs <<= 1) {
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                if (q & hs) continue;
                const double x = C[q], y = C[q | hs];
                C[q] = x + y;
                C[q | hs] = x - y;
            }
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) acc[0] += pr[k] * C[k];
    }
    block_sum<1>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// ---------------------------------------------------------------------------
// Cumulative distribution for sampling: a deterministic three-phase FP64
// inclusive scan with a fixed summation order (so a CPU restatement reproduces
// every value bit for bit).  A chunk is 1024 values = 256 threads x 4:
//   s_j    = running sum of the thread's 4 values (left to right);
//   incl_t = Kogge-Stone inclusive scan of the threads' s_3 inside each warp
//            (shuffle offsets 1, 2, 4, 8, 16);
//   W_w    = exclusive running sum of the 8 warp totals (one thread, in order);
//   cdf    = (W_w + incl_{t-1}) + s_j   (incl_{-1} = 0 at lane 0),
// and the chunk total is the chunk's last cdf value.  Chunk totals are scanned
// the same way (recursively) and added as base + value to every later chunk.
// ---------------------------------------------------------------------------
constexpr int kScanChunk = 1024;

__global__ void __launch_bounds__(256) k_probs_exact_c128(const double2 *__restrict__ v,
                                                          double *__restrict__ p, uint64_t N) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 a = v[i];
        p[i] = __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));  // no contraction
    }
}

__global__ void __launch_bounds__(256) k_probs_exact_c64(const float2 *__restrict__ v,
                                                         double *__restrict__ p, uint64_t N) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float2 a = v[i];
        const double x = a.x, y = a.y;
        p[i] = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    }
}

__global__ void __launch_bounds__(256) k_scan_chunks(const double *__restrict__ in,
                                                     double *__restrict__ out,
                                                     double *__restrict__ chunk_total,
                                                     uint64_t N) {
    __shared__ double W[8];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint64_t base = (uint64_t)blockIdx.x * kScanChunk + 4u * t;
    double s[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double x = base + j < N ? in[base + j] : 0.0;
        s[j] = j == 0 ? x : __dadd_rn(s[j - 1], x);
    }
    double incl = s[3];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = __dadd_rn(y, incl);
    }
    double excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = 0.0;
    if (lane == 31) W[warp] = incl;  // warp total
    __syncthreads();
    if (t == 0) {
        double run = 0.0;
        for (int w = 0; w < 8; ++w) {
            const double tot = W[w];
            W[w] = run;
            run = __dadd_rn(run, tot);
        }
    }
    __syncthreads();
    const double off = __dadd_rn(W[warp], excl);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double v = __dadd_rn(off, s[j]);
        if (base + j < N) out[base + j] = v;
        if (t == 255 && j == 3) chunk_total[blockIdx.x] = v;
    }
}

__global__ void k_scan_add_base(double *__restrict__ cdf, const double *__restrict__ incl_total,
                                uint64_t N) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x + kScanChunk; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = i / kScanChunk;
        cdf[i] = __dadd_rn(incl_total[c - 1], cdf[i]);
    }
}

__global__ void k_sample(const double *__restrict__ cdf, uint64_t N, uint64_t nshots,
                         uint64_t seed, uint64_t *__restrict__ out) {
    const double total = cdf[N - 1];
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nshots;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = splitmix64(seed ^ splitmix64(s));
        const double u = (double)(r >> 11) * (1.0 / 9007199254740992.0) * total;
        // first index with cdf > u
        uint64_t lo = 0, hi = N - 1;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (cdf[mid] > u) hi = mid;
            else lo = mid + 1;
        }
        out[s] = lo;
    }
}

static int red_grid(uint64_t N, int threads) {
    uint64_t g = (N + threads - 1) / threads;
    if (g > (uint64_t)kRedBlocks) g = kRedBlocks;
    if (g < 1) g = 1;
    return (int)g;
}

static int grid_for(uint64_t N, int threads) {
    uint64_t g = (N + threads - 1) / threads;
    const uint64_t cap = 148ull * 64;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

static int norm_sqr_device(const lq_state *s, double *d_out) {
    const uint64_t N = 1ull << s->n;
    const int th = 256, g = red_grid(N, th);
    prof_begin(s->stream, kProfReduce);
    if (s->dtype == LQ_C128)
        k_norm_partial<<<g, th, 0, s->stream>>>((const double2 *)s->d, N, s->d_red);
    else
        k_norm_partial<<<g, th, 0, s->stream>>>((const float2 *)s->d, N, s->d_red);
    k_final_sum<1><<<1, 256, 0, s->stream>>>(s->d_red, g, d_out);
    prof_end(s->stream, kProfReduce);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

int normalize_impl(lq_state *s) {
    double *d_norm = s->d_red + kRedBlocks * 2 * kMaxTermsPerPass - 1;
    LQ_TRY(norm_sqr_device(s, d_norm));
    const uint64_t N = 1ull << s->n;
    if (s->dtype == LQ_C128)
        k_scale_by_norm<<<grid_for(N, 256), 256, 0, s->stream>>>((double2 *)s->d, N, d_norm);
    else
        k_scale_by_norm<<<grid_for(N, 256), 256, 0, s->stream>>>((float2 *)s->d, N, d_norm);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

// FP64 norm bookkeeping of the precision form: remember the squared norm now,
// and later scale the state back to it (two slots at the end of the reduction
// scratch, clear of the partial sums and of normalize's slot).
int norm_snapshot(lq_state *s) {
    double *d_in = s->d_red + kRedBlocks * 2 * kMaxTermsPerPass - 2;
    return norm_sqr_device(s, d_in);
}

int norm_restore(lq_state *s) {
    double *d_in = s->d_red + kRedBlocks * 2 * kMaxTermsPerPass - 2;
    double *d_now = s->d_red + kRedBlocks * 2 * kMaxTermsPerPass - 3;
    LQ_TRY(norm_sqr_device(s, d_now));
    const uint64_t N = 1ull << s->n;
    if (s->dtype == LQ_C128)
        k_scale_to_norm<<<grid_for(N, 256), 256, 0, s->stream>>>((double2 *)s->d, N, d_in, d_now);
    else
        k_scale_to_norm<<<grid_for(N, 256), 256, 0, s->stream>>>((float2 *)s->d, N, d_in, d_now);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

int expectation_impl(const lq_state *s, const lq_pauli_term *terms, int nterms, int yconv,
                     double *out, double *per_term) {
    const int n = s->n;
    for (int t = 0; t < nterms; ++t) {
        const uint64_t lim = n == 64 ? ~0ull : ((1ull << n) - 1);
        if ((terms[t].xmask & ~lim) || (terms[t].zmask & ~lim))
            return set_error(LQ_ERR_QUBIT_INDEX, "Pauli term %d acts on a qubit >= %d", t, n);
        const int ny = __builtin_popcountll(terms[t].xmask & terms[t].zmask);
        if (terms[t].ny != ny)
            return set_error(LQ_ERR_INVALID_ARG,
                             "Pauli term %d: ny=%d but xmask&zmask has %d bits", t, terms[t].ny, ny);
    }
    // Re(Y^ny z) selectors: Y = +i (reference convention) or -i (textbook).
    auto selectors = [&](int ny, double &a, double &b) {
        int k = ny & 3;
        if (yconv == LQ_Y_TEXTBOOK) k = (4 - k) & 3;
        // Re(i^k (x + i y)): k=0: x ; 1: -y ; 2: -x ; 3: y
        a = k == 0 ? 1.0 : k == 2 ? -1.0 : 0.0;
        b = k == 1 ? -1.0 : k == 3 ? 1.0 : 0.0;
    };
    // Group terms by X mask (one pass over the state per group), or one group
    // per term when per-term values are requested.
    std::vector<std::pair<uint64_t, std::vector<int>>> groups;
    if (per_term) {
        for (int t = 0; t < nterms; ++t) groups.push_back({terms[t].xmask, {t}});
    } else {
        std::map<uint64_t, size_t> idx;
        for (int t = 0; t < nterms; ++t) {
            auto it = idx.find(terms[t].xmask);
            if (it == idx.end()) {
                idx[terms[t].xmask] = groups.size();
                groups.push_back({terms[t].xmask, {t}});
            } else {
                groups[it->second].second.push_back(t);
            }
        }
    }
    // A group's terms sit in the sweep's dynamic shared memory (24 bytes each,
    // 48 KB per block without an opt-in): refuse larger groups with a clear error.
    constexpr size_t kMaxGroupTerms = 2000;
    for (const auto &gr : groups)
        if (gr.second.size() > kMaxGroupTerms)
            return set_error(LQ_ERR_UNSUPPORTED,
                             "%zu Pauli terms share one X mask; at most %zu per X mask "
                             "(split the observable)",
                             gr.second.size(), kMaxGroupTerms);
    const uint64_t N = 1ull << n;
    const int th = 256;
    const int g = red_grid(std::max<uint64_t>(N / 2, 1), th);
    // The X-mask-0 group of a state with 12 or more qubits runs the folded form
    // (k_pauli_zfold): its terms sorted by bits 8-11 of the Z mask.
    int zfold = -1;
    int pbeg[17] = {0};
    if (!per_term && n >= 12) {
        for (size_t gi = 0; gi < groups.size(); ++gi)
            if (groups[gi].first == 0) zfold = (int)gi;
    }
    if (zfold >= 0) {
        auto pat = [&](int t) { return (int)((terms[t].zmask >> 8) & 15); };
        std::vector<int> &ts = groups[zfold].second;
        std::stable_sort(ts.begin(), ts.end(), [&](int x, int y) { return pat(x) < pat(y); });
        for (int q = 0; q <= 16; ++q) {
            int k = 0;
            while (k < (int)ts.size() && pat(ts[k]) < q) ++k;
            pbeg[q] = k;
        }
    }
    // Host-side packed coefficients, uploaded once per call.
    std::vector<TermCoef> tc(nterms);
    std::vector<int> offs;
    int off = 0;
    std::vector<TermCoef> packed;
    for (auto &gr : groups) {
        offs.push_back(off);
        for (int t : gr.second) {
            double a, b;
            selectors(terms[t].ny, a, b);
            packed.push_back(TermCoef{terms[t].zmask, terms[t].coefficient * a,
                                      terms[t].coefficient * b});
        }
        off += (int)gr.second.size();
    }
    lq_state *ms = const_cast<lq_state *>(s);
    const size_t coef_bytes = packed.size() * sizeof(TermCoef);
    const size_t res_bytes = groups.size() * sizeof(double);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    LQ_TRY(ensure_prog(ms, al(coef_bytes) + al(res_bytes) + sizeof(pbeg) + 256));
    TermCoef *d_tc = (TermCoef *)ms->d_prog;
    double *d_res = (double *)((char *)ms->d_prog + al(coef_bytes));
    int *d_pbeg = (int *)((char *)ms->d_prog + al(coef_bytes) + al(res_bytes));
    if (!packed.empty())
        LQ_CUDA_TRY(cudaMemcpyAsync(d_tc, packed.data(), coef_bytes, cudaMemcpyHostToDevice,
                                    s->stream));
    if (zfold >= 0)
        LQ_CUDA_TRY(cudaMemcpyAsync(d_pbeg, pbeg, sizeof(pbeg), cudaMemcpyHostToDevice,
                                    s->stream));
    prof_begin(s->stream, kProfReduce);
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const int nt = (int)groups[gi].second.size();
        const size_t shm = nt * sizeof(TermCoef);
        if ((int)gi == zfold) {
            if (s->dtype == LQ_C128)
                k_pauli_zfold<<<g, th, shm, s->stream>>>((const double2 *)s->d, n,
                                                         d_tc + offs[gi], nt, d_pbeg, s->d_red);
            else
                k_pauli_zfold<<<g, th, shm, s->stream>>>((const float2 *)s->d, n,
                                                         d_tc + offs[gi], nt, d_pbeg, s->d_red);
        } else if (s->dtype == LQ_C128) {
            k_pauli_group<<<g, th, shm, s->stream>>>((const double2 *)s->d, n, groups[gi].first,
                                                     d_tc + offs[gi], nt, s->d_red);
        } else {
            k_pauli_group<<<g, th, shm, s->stream>>>((const float2 *)s->d, n, groups[gi].first,
                                                     d_tc + offs[gi], nt, s->d_red);
        }
        k_final_sum<1><<<1, 256, 0, s->stream>>>(s->d_red, g, d_res + gi);
    }
    prof_end(s->stream, kProfReduce);
    LQ_CUDA_TRY(cudaGetLastError());
    std::vector<double> res(groups.size());
    if (!groups.empty())
        LQ_CUDA_TRY(cudaMemcpyAsync(res.data(), d_res, res_bytes, cudaMemcpyDeviceToHost,
                                    s->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    // Sum group results in term order (PauliObservable::expectation sums
    // term.expectation in order, src/optimization/observable.rs:229-231).
    double sum = 0.0;
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        sum += res[gi];
        if (per_term) per_term[groups[gi].second[0]] = res[gi];
    }
    *out = sum;
    return LQ_OK;
}

// ---------------------------------------------------------------------------
// Pauli-sum expectation that allocates nothing (lq_expectation_pauli_static).
//
// Its scratch -- the per-block partial sums, the per-group results and the
// packed term coefficients -- lives in one file-scope device array of fixed
// size instead of memory obtained from cudaMalloc.  Host code cannot hand the
// array's name to a kernel (on the host that name is only a stand-in, not a
// device address), so the device address is fetched once per device with
// cudaGetSymbolAddress and cached.
// ---------------------------------------------------------------------------
constexpr int kStaticMaxTerms = 1024;
constexpr size_t kStaticPartialBytes = sizeof(double) * kRedBlocks;
constexpr size_t kStaticResultBytes = sizeof(double) * kStaticMaxTerms;
constexpr size_t kStaticCoefBytes = sizeof(TermCoef) * kStaticMaxTerms;
constexpr size_t kStaticScratchBytes = 64 * 1024;
static_assert(kStaticPartialBytes + kStaticResultBytes + kStaticCoefBytes <= kStaticScratchBytes,
              "static scratch too small");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

static int static_scratch_address(unsigned char **out) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static unsigned char *addr[kMaxDevices] = {};
    int dev = 0;
    LQ_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(LQ_ERR_UNSUPPORTED, "device %d", dev);
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return set_error(LQ_ERR_CUDA, "cudaGetSymbolAddress(static scratch): %s",
                             cudaGetErrorString(e));
        addr[dev] = (unsigned char *)p;
    }
    *out = addr[dev];
    return LQ_OK;
}

}  // namespace lq

using namespace lq;

extern "C" {

int lq_expectation_pauli_static(const void *d_amplitudes, int num_qubits, int dtype,
                                const lq_pauli_term *terms, int nterms, int y_convention,
                                void *stream, double *out) {
    clear_error();
    if (!d_amplitudes || !out || (nterms > 0 && !terms) || nterms < 0)
        return set_error(LQ_ERR_INVALID_ARG, "null pointer or negative term count");
    if (num_qubits < 1 || num_qubits > 36)
        return set_error(LQ_ERR_STATE_DIMENSION, "num_qubits %d outside 1..36", num_qubits);
    if (dtype != LQ_C128 && dtype != LQ_C64)
        return set_error(LQ_ERR_INVALID_ARG, "unknown dtype %d", dtype);
    if (y_convention != LQ_Y_REFERENCE && y_convention != LQ_Y_TEXTBOOK)
        return set_error(LQ_ERR_INVALID_ARG, "unknown Y convention %d", y_convention);
    if (nterms > kStaticMaxTerms)
        return set_error(LQ_ERR_UNSUPPORTED,
                         "%d Pauli terms exceed the fixed scratch of this entry point "
                         "(at most %d terms; use lq_expectation_pauli)",
                         nterms, kStaticMaxTerms);
    if (nterms == 0) {
        *out = 0.0;
        return LQ_OK;
    }
    const int n = num_qubits;
    const uint64_t lim = n == 64 ? ~0ull : ((1ull << n) - 1);
    for (int t = 0; t < nterms; ++t) {
        if ((terms[t].xmask & ~lim) || (terms[t].zmask & ~lim))
            return set_error(LQ_ERR_QUBIT_INDEX, "Pauli term %d acts on a qubit >= %d", t, n);
        if (terms[t].ny != __builtin_popcountll(terms[t].xmask & terms[t].zmask))
            return set_error(LQ_ERR_INVALID_ARG, "Pauli term %d: ny does not match its masks", t);
    }
    // host-stack copies and a stream wait cannot be captured into a graph
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        LQ_CUDA_TRY(cudaStreamIsCapturing((cudaStream_t)stream, &cs));
        if (cs != cudaStreamCaptureStatusNone)
            return set_error(LQ_ERR_UNSUPPORTED,
                             "lq_expectation_pauli_static cannot run on a capturing stream");
    }
    // The scratch array is per device: the amplitudes must be on the current one.
    {
        cudaPointerAttributes pa{};
        int dev = 0;
        LQ_CUDA_TRY(cudaGetDevice(&dev));
        if (cudaPointerGetAttributes(&pa, d_amplitudes) != cudaSuccess) {
            cudaGetLastError();
            return set_error(LQ_ERR_INVALID_ARG, "d_amplitudes is not a CUDA pointer");
        }
        if (pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged)
            return set_error(LQ_ERR_INVALID_ARG, "d_amplitudes is not device memory");
        if (pa.device != dev)
            return set_error(LQ_ERR_INVALID_ARG,
                             "d_amplitudes is on device %d, the current device is %d", pa.device,
                             dev);
    }
    unsigned char *scratch = nullptr;
    LQ_TRY(static_scratch_address(&scratch));
    double *d_partials = (double *)scratch;
    double *d_results = (double *)(scratch + kStaticPartialBytes);
    TermCoef *d_coef = (TermCoef *)(scratch + kStaticPartialBytes + kStaticResultBytes);
    cudaStream_t st = (cudaStream_t)stream;

    // Group the terms by X mask with fixed-size host arrays (no heap).
    int order[kStaticMaxTerms], gbegin[kStaticMaxTerms + 1];
    uint64_t gx[kStaticMaxTerms];
    bool used[kStaticMaxTerms] = {};
    int ng = 0, k = 0;
    for (int t = 0; t < nterms; ++t) {
        if (used[t]) continue;
        gx[ng] = terms[t].xmask;
        gbegin[ng] = k;
        for (int u = t; u < nterms; ++u)
            if (!used[u] && terms[u].xmask == gx[ng]) {
                used[u] = true;
                order[k++] = u;
            }
        ++ng;
    }
    gbegin[ng] = k;
    TermCoef packed[kStaticMaxTerms];  // host stack: 24 KiB
    for (int i = 0; i < nterms; ++i) {
        const lq_pauli_term &pt = terms[order[i]];
        int q = pt.ny & 3;
        if (y_convention == LQ_Y_TEXTBOOK) q = (4 - q) & 3;
        const double a = q == 0 ? 1.0 : q == 2 ? -1.0 : 0.0;
        const double b = q == 1 ? -1.0 : q == 3 ? 1.0 : 0.0;
        packed[i] = TermCoef{pt.zmask, pt.coefficient * a, pt.coefficient * b};
    }
    LQ_CUDA_TRY(cudaMemcpyAsync(d_coef, packed, sizeof(TermCoef) * nterms,
                                cudaMemcpyHostToDevice, st));
    const uint64_t N = 1ull << n;
    const int th = 256;
    const int g = red_grid(std::max<uint64_t>(N / 2, 1), th);
    for (int gi = 0; gi < ng; ++gi) {
        const int nt = gbegin[gi + 1] - gbegin[gi];
        const size_t shm = nt * sizeof(TermCoef);
        if (dtype == LQ_C128)
            k_pauli_group<<<g, th, shm, st>>>((const double2 *)d_amplitudes, n, gx[gi],
                                              d_coef + gbegin[gi], nt, d_partials);
        else
            k_pauli_group<<<g, th, shm, st>>>((const float2 *)d_amplitudes, n, gx[gi],
                                              d_coef + gbegin[gi], nt, d_partials);
        k_final_sum<1><<<1, 256, 0, st>>>(d_partials, g, d_results + gi);
    }
    LQ_CUDA_TRY(cudaGetLastError());
    double res[kStaticMaxTerms];  // host stack: 8 KiB
    LQ_CUDA_TRY(cudaMemcpyAsync(res, d_results, sizeof(double) * ng, cudaMemcpyDeviceToHost, st));
    LQ_CUDA_TRY(cudaStreamSynchronize(st));
    double sum = 0.0;
    for (int gi = 0; gi < ng; ++gi) sum += res[gi];
    *out = sum;
    return LQ_OK;
}

const char *lq_last_error(void) { return g_last_error.c_str(); }

int lq_version(void) { return 1 * 10000 + 0 * 100 + 0; }

int lq_device_count(int *count) {
    if (!count) return set_error(LQ_ERR_INVALID_ARG, "null count");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        *count = 0;
        cudaGetLastError();
        return set_error(LQ_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    }
    *count = c;
    return LQ_OK;
}

int lq_set_device(int device) {
    LQ_CUDA_TRY(cudaSetDevice(device));
    return LQ_OK;
}

int lq_set_alloc_limit(uint64_t bytes) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    g_alloc_limit = bytes;
    return LQ_OK;
}

int lq_state_create(int num_qubits, int dtype, lq_state **out) {
    clear_error();
    if (!out) return set_error(LQ_ERR_INVALID_ARG, "null output pointer");
    *out = nullptr;
    if (dtype != LQ_C128 && dtype != LQ_C64)
        return set_error(LQ_ERR_INVALID_ARG, "unknown dtype %d", dtype);
    if (num_qubits < 1 || num_qubits > 36)
        return set_error(LQ_ERR_STATE_DIMENSION,
                         "Invalid state dimension: 2^%d (supported 1..36 qubits)", num_qubits);
    const size_t bytes = (size_t)amp_bytes(dtype) << num_qubits;
    {
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        if (g_alloc_limit && g_alloc_in_use + bytes > g_alloc_limit)
            return set_error(LQ_ERR_OOM,
                             "state of %zu bytes exceeds the allocation limit (%llu in use, "
                             "limit %llu)",
                             bytes, (unsigned long long)g_alloc_in_use,
                             (unsigned long long)g_alloc_limit);
    }
    lq_state *s = new lq_state();
    s->n = num_qubits;
    s->dtype = dtype;
    s->bytes = bytes;
    cudaGetDevice(&s->device);
    auto fail = [&](cudaError_t e, const char *what) {
        int code = e == cudaErrorMemoryAllocation ? LQ_ERR_OOM : LQ_ERR_CUDA;
        if (s->d) cudaFree(s->d);
        if (s->d_red) cudaFree(s->d_red);
        if (s->h_red) cudaFreeHost(s->h_red);
        if (s->d_flag) cudaFree(s->d_flag);
        if (s->stream) cudaStreamDestroy(s->stream);
        delete s;
        cudaGetLastError();
        return set_error(code, "%s: %s", what, cudaGetErrorString(e));
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(e, "cudaStreamCreate");
    if ((e = cudaMalloc(&s->d, bytes)) != cudaSuccess) return fail(e, "cudaMalloc(state)");
    if ((e = cudaMalloc(&s->d_red, sizeof(double) * kRedBlocks * 2 * kMaxTermsPerPass)) !=
        cudaSuccess)
        return fail(e, "cudaMalloc(reduction scratch)");
    if ((e = cudaMallocHost(&s->h_red, sizeof(double) * 64)) != cudaSuccess)
        return fail(e, "cudaMallocHost");
    if ((e = cudaMalloc(&s->d_flag, sizeof(unsigned) * 4)) != cudaSuccess)
        return fail(e, "cudaMalloc(flags)");
    if ((e = cudaMemsetAsync(s->d_flag, 0, sizeof(unsigned) * 4, s->stream)) != cudaSuccess)
        return fail(e, "cudaMemset");
    {
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        g_alloc_in_use += bytes;
    }
    *out = s;
    int rc = lq_state_set_basis(s, 0);
    if (rc != LQ_OK) {
        lq_state_destroy(s);
        *out = nullptr;
        return rc;
    }
    return LQ_OK;
}

int lq_state_destroy(lq_state *s) {
    if (!s) return LQ_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->d) {
        cudaFree(s->d);
        std::lock_guard<std::mutex> lk(g_alloc_mu);
        g_alloc_in_use -= s->bytes;
    }
    if (s->d_red) cudaFree(s->d_red);
    if (s->h_red) cudaFreeHost(s->h_red);
    if (s->d_flag) cudaFree(s->d_flag);
    if (s->d_prog) cudaFree(s->d_prog);
    free_plan_cache(s);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return LQ_OK;
}

int lq_state_num_qubits(const lq_state *s, int *out) {
    LQ_TRY(check_state(s));
    if (!out) return set_error(LQ_ERR_INVALID_ARG, "null output");
    *out = s->n;
    return LQ_OK;
}

int lq_state_dtype(const lq_state *s, int *out) {
    LQ_TRY(check_state(s));
    if (!out) return set_error(LQ_ERR_INVALID_ARG, "null output");
    *out = s->dtype;
    return LQ_OK;
}

int lq_state_set_basis(lq_state *s, uint64_t index) {
    LQ_TRY(check_state(s));
    const uint64_t N = 1ull << s->n;
    if (index >= N)
        return set_error(LQ_ERR_DIMENSION_MISMATCH, "basis index %llu >= 2^%d",
                         (unsigned long long)index, s->n);
    if (s->dtype == LQ_C128)
        k_set_basis<<<grid_for(N, 256), 256, 0, s->stream>>>((double2 *)s->d, N, index);
    else
        k_set_basis<<<grid_for(N, 256), 256, 0, s->stream>>>((float2 *)s->d, N, index);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

int lq_state_set_plus(lq_state *s) {
    LQ_TRY(check_state(s));
    const uint64_t N = 1ull << s->n;
    const double norm = 1.0 / std::sqrt((double)N);  // plus_state: 1/sqrt(size)
    if (s->dtype == LQ_C128)
        k_set_const<<<grid_for(N, 256), 256, 0, s->stream>>>((double2 *)s->d, N, norm);
    else
        k_set_const<<<grid_for(N, 256), 256, 0, s->stream>>>((float2 *)s->d, N, norm);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

int lq_state_upload(lq_state *s, const double *host, size_t num_amplitudes) {
    LQ_TRY(check_state(s));
    if (!host) return set_error(LQ_ERR_INVALID_ARG, "null host buffer");
    const uint64_t N = 1ull << s->n;
    if (num_amplitudes != N)
        return set_error(LQ_ERR_DIMENSION_MISMATCH, "Dimension mismatch: expected %llu, got %zu",
                         (unsigned long long)N, num_amplitudes);
    if (s->dtype == LQ_C128) {
        LQ_CUDA_TRY(cudaMemcpyAsync(s->d, host, N * 16, cudaMemcpyHostToDevice, s->stream));
    } else {
        // Stage in chunks through a temporary complex128 buffer.
        const uint64_t chunk = std::min<uint64_t>(N, 1ull << 24);
        double2 *tmp = nullptr;
        LQ_CUDA_TRY(cudaMallocAsync(&tmp, chunk * 16, s->stream));
        for (uint64_t o = 0; o < N; o += chunk) {
            const uint64_t c = std::min(chunk, N - o);
            LQ_CUDA_TRY(cudaMemcpyAsync(tmp, host + 2 * o, c * 16, cudaMemcpyHostToDevice,
                                        s->stream));
            k_c128_to_c64<<<grid_for(c, 256), 256, 0, s->stream>>>(tmp, (float2 *)s->d + o, c);
        }
        LQ_CUDA_TRY(cudaFreeAsync(tmp, s->stream));
    }
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return LQ_OK;
}

int lq_state_download(const lq_state *s, double *host, size_t num_amplitudes) {
    LQ_TRY(check_state(s));
    if (!host) return set_error(LQ_ERR_INVALID_ARG, "null host buffer");
    const uint64_t N = 1ull << s->n;
    if (num_amplitudes != N)
        return set_error(LQ_ERR_DIMENSION_MISMATCH, "Dimension mismatch: expected %llu, got %zu",
                         (unsigned long long)N, num_amplitudes);
    if (s->dtype == LQ_C128) {
        LQ_CUDA_TRY(cudaMemcpyAsync(host, s->d, N * 16, cudaMemcpyDeviceToHost, s->stream));
        LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    } else {
        std::vector<float> tmp(2 * N);
        LQ_CUDA_TRY(cudaMemcpyAsync(tmp.data(), s->d, N * 8, cudaMemcpyDeviceToHost, s->stream));
        LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
        for (uint64_t i = 0; i < 2 * N; ++i) host[i] = tmp[i];
    }
    return LQ_OK;
}

int lq_state_upload_c64(lq_state *s, const float *host, size_t num_amplitudes) {
    LQ_TRY(check_state(s));
    if (s->dtype != LQ_C64) return set_error(LQ_ERR_UNSUPPORTED, "state is not complex64");
    if (!host) return set_error(LQ_ERR_INVALID_ARG, "null host buffer");
    const uint64_t N = 1ull << s->n;
    if (num_amplitudes != N)
        return set_error(LQ_ERR_DIMENSION_MISMATCH, "Dimension mismatch: expected %llu, got %zu",
                         (unsigned long long)N, num_amplitudes);
    LQ_CUDA_TRY(cudaMemcpyAsync(s->d, host, N * 8, cudaMemcpyHostToDevice, s->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return LQ_OK;
}

int lq_state_download_c64(const lq_state *s, float *host, size_t num_amplitudes) {
    LQ_TRY(check_state(s));
    if (s->dtype != LQ_C64) return set_error(LQ_ERR_UNSUPPORTED, "state is not complex64");
    if (!host) return set_error(LQ_ERR_INVALID_ARG, "null host buffer");
    const uint64_t N = 1ull << s->n;
    if (num_amplitudes != N)
        return set_error(LQ_ERR_DIMENSION_MISMATCH, "Dimension mismatch: expected %llu, got %zu",
                         (unsigned long long)N, num_amplitudes);
    LQ_CUDA_TRY(cudaMemcpyAsync(host, s->d, N * 8, cudaMemcpyDeviceToHost, s->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return LQ_OK;
}

int lq_state_copy(lq_state *dst, const lq_state *src) {
    LQ_TRY(check_state(dst));
    LQ_TRY(check_state(src));
    if (dst->n != src->n || dst->dtype != src->dtype)
        return set_error(LQ_ERR_DIMENSION_MISMATCH, "Dimension mismatch: expected 2^%d, got 2^%d",
                         dst->n, src->n);
    LQ_CUDA_TRY(cudaStreamSynchronize(src->stream));
    LQ_CUDA_TRY(cudaMemcpyAsync(dst->d, src->d, dst->bytes, cudaMemcpyDeviceToDevice, dst->stream));
    return LQ_OK;
}

int lq_state_tensor_product(lq_state *out, const lq_state *a, const lq_state *b) {
    LQ_TRY(check_state(out));
    LQ_TRY(check_state(a));
    LQ_TRY(check_state(b));
    if (out->n != a->n + b->n)
        return set_error(LQ_ERR_DIMENSION_MISMATCH, "Dimension mismatch: expected 2^%d, got 2^%d",
                         a->n + b->n, out->n);
    if (out->dtype != a->dtype || a->dtype != b->dtype)
        return set_error(LQ_ERR_UNSUPPORTED, "mixed dtypes");
    LQ_CUDA_TRY(cudaStreamSynchronize(a->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(b->stream));
    const uint64_t N = 1ull << out->n;
    if (out->dtype == LQ_C128)
        k_kron<<<grid_for(N, 256), 256, 0, out->stream>>>(
            (double2 *)out->d, (const double2 *)a->d, (const double2 *)b->d, b->n, N);
    else
        k_kron<<<grid_for(N, 256), 256, 0, out->stream>>>(
            (float2 *)out->d, (const float2 *)a->d, (const float2 *)b->d, b->n, N);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

int lq_state_synchronize(lq_state *s) {
    LQ_TRY(check_state(s));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    unsigned flags = 0;
    LQ_CUDA_TRY(cudaMemcpy(&flags, s->d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (flags & kFlagTimeout) {
        cudaMemset(s->d_flag, 0, sizeof(unsigned));
        return set_error(LQ_ERR_TIMEOUT, "a bounded device wait ran out");
    }
    return LQ_OK;
}

int lq_check_wait_timeout(lq_state *s, unsigned polls) {
    LQ_TRY(check_state(s));
    if (polls < 1 || polls > (1u << 20))
        return set_error(LQ_ERR_INVALID_ARG, "polls must be 1..1048576 (got %u)", polls);
    k_wait_probe<<<1, 32, 0, s->stream>>>(s->d_flag, polls);
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

int lq_state_device_ptr(lq_state *s, void **dptr) {
    LQ_TRY(check_state(s));
    if (!dptr) return set_error(LQ_ERR_INVALID_ARG, "null output");
    *dptr = s->d;
    return LQ_OK;
}

int lq_state_stream(lq_state *s, void **stream) {
    LQ_TRY(check_state(s));
    if (!stream) return set_error(LQ_ERR_INVALID_ARG, "null output");
    *stream = (void *)s->stream;
    return LQ_OK;
}

int lq_norm_sqr(const lq_state *s, double *out) {
    LQ_TRY(check_state(s));
    if (!out) return set_error(LQ_ERR_INVALID_ARG, "null output");
    lq_state *ms = const_cast<lq_state *>(s);
    double *d_out = ms->d_red + kRedBlocks * 2 * kMaxTermsPerPass - 2;
    LQ_TRY(norm_sqr_device(s, d_out));
    LQ_CUDA_TRY(cudaMemcpyAsync(ms->h_red, d_out, sizeof(double), cudaMemcpyDeviceToHost,
                                s->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    *out = ms->h_red[0];
    return LQ_OK;
}

int lq_normalize(lq_state *s) {
    LQ_TRY(check_state(s));
    return normalize_impl(s);
}

int lq_probabilities(const lq_state *s, double *host, size_t len) {
    LQ_TRY(check_state(s));
    if (!host) return set_error(LQ_ERR_INVALID_ARG, "null host buffer");
    const uint64_t N = 1ull << s->n;
    if (len != N)
        return set_error(LQ_ERR_DIMENSION_MISMATCH, "Dimension mismatch: expected %llu, got %zu",
                         (unsigned long long)N, len);
    const uint64_t chunk = std::min<uint64_t>(N, 1ull << 24);
    double *tmp = nullptr;
    LQ_CUDA_TRY(cudaMallocAsync(&tmp, chunk * 8, s->stream));
    for (uint64_t o = 0; o < N; o += chunk) {
        const uint64_t c = std::min(chunk, N - o);
        if (s->dtype == LQ_C128)
            k_probs<<<grid_for(c, 256), 256, 0, s->stream>>>((const double2 *)s->d + o, tmp, c);
        else
            k_probs<<<grid_for(c, 256), 256, 0, s->stream>>>((const float2 *)s->d + o, tmp, c);
        LQ_CUDA_TRY(cudaMemcpyAsync(host + o, tmp, c * 8, cudaMemcpyDeviceToHost, s->stream));
    }
    LQ_CUDA_TRY(cudaFreeAsync(tmp, s->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return LQ_OK;
}

int lq_probability(const lq_state *s, uint64_t basis, double *out) {
    LQ_TRY(check_state(s));
    if (!out) return set_error(LQ_ERR_INVALID_ARG, "null output");
    if (basis >= (1ull << s->n)) {
        *out = 0.0;  // State::probability returns 0.0 out of range
        return LQ_OK;
    }
    double a[2];
    if (s->dtype == LQ_C128) {
        LQ_CUDA_TRY(cudaMemcpyAsync(a, (const double2 *)s->d + basis, 16, cudaMemcpyDeviceToHost,
                                    s->stream));
        LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    } else {
        float f[2];
        LQ_CUDA_TRY(cudaMemcpyAsync(f, (const float2 *)s->d + basis, 8, cudaMemcpyDeviceToHost,
                                    s->stream));
        LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
        a[0] = f[0];
        a[1] = f[1];
    }
    *out = a[0] * a[0] + a[1] * a[1];
    return LQ_OK;
}

int lq_inner_product(const lq_state *a, const lq_state *b, double out[2]) {
    LQ_TRY(check_state(a));
    LQ_TRY(check_state(b));
    if (!out) return set_error(LQ_ERR_INVALID_ARG, "null output");
    if (a->n != b->n)
        return set_error(LQ_ERR_DIMENSION_MISMATCH, "Dimension mismatch: expected %llu, got %llu",
                         (unsigned long long)(1ull << a->n), (unsigned long long)(1ull << b->n));
    if (a->dtype != b->dtype) return set_error(LQ_ERR_UNSUPPORTED, "mixed dtypes");
    LQ_CUDA_TRY(cudaStreamSynchronize(b->stream));
    lq_state *ma = const_cast<lq_state *>(a);
    const uint64_t N = 1ull << a->n;
    const int th = 256, g = red_grid(N, th);
    double *d_out = ma->d_red + kRedBlocks * 2 * kMaxTermsPerPass - 4;
    prof_begin(a->stream, kProfReduce);
    if (a->dtype == LQ_C128)
        k_inner_partial<<<g, th, 0, a->stream>>>((const double2 *)a->d, (const double2 *)b->d, N,
                                                 ma->d_red);
    else
        k_inner_partial<<<g, th, 0, a->stream>>>((const float2 *)a->d, (const float2 *)b->d, N,
                                                 ma->d_red);
    k_final_sum<2><<<1, 256, 0, a->stream>>>(ma->d_red, g, d_out);
    prof_end(a->stream, kProfReduce);
    LQ_CUDA_TRY(cudaGetLastError());
    LQ_CUDA_TRY(cudaMemcpyAsync(ma->h_red, d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                a->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(a->stream));
    out[0] = ma->h_red[0];
    out[1] = ma->h_red[1];
    return LQ_OK;
}

// Inclusive scan of in[0..N) into out (the fixed-order scan above); tot holds
// the chunk totals of every level (ceil(N/1024) + ceil(N/2^20) + ... doubles).
static int scan_inclusive(const double *in, double *out, double *tot, uint64_t N,
                          cudaStream_t st) {
    const uint64_t nc = (N + kScanChunk - 1) / kScanChunk;
    if (nc > 0x7fffffffull) return set_error(LQ_ERR_UNSUPPORTED, "scan too long");
    k_scan_chunks<<<(unsigned)nc, 256, 0, st>>>(in, out, tot, N);
    LQ_CUDA_TRY(cudaGetLastError());
    if (nc > 1) {
        double *incl = tot + nc;  // scanned chunk totals, in place after the totals
        LQ_TRY(scan_inclusive(tot, incl, incl + nc, nc, st));
        k_scan_add_base<<<grid_for(N, 256), 256, 0, st>>>(out, incl, N);
        LQ_CUDA_TRY(cudaGetLastError());
    }
    return LQ_OK;
}

static uint64_t scan_scratch(uint64_t N) {  // doubles needed by scan_inclusive's tot
    uint64_t need = 0;
    for (uint64_t n = N; n > 1;) {
        const uint64_t nc = (n + kScanChunk - 1) / kScanChunk;
        need += 2 * nc;
        n = nc;
    }
    return need + 2;
}

int lq_measure_shots(const lq_state *s, uint64_t n_shots, uint64_t seed, uint64_t *host_out) {
    LQ_TRY(check_state(s));
    if (!host_out && n_shots) return set_error(LQ_ERR_INVALID_ARG, "null output");
    if (n_shots == 0) return LQ_OK;
    const uint64_t N = 1ull << s->n;
    double *p = nullptr, *cdf = nullptr, *tot = nullptr;
    uint64_t *d_out = nullptr;
    LQ_CUDA_TRY(cudaMallocAsync(&p, N * 8, s->stream));
    LQ_CUDA_TRY(cudaMallocAsync(&cdf, N * 8, s->stream));
    LQ_CUDA_TRY(cudaMallocAsync(&tot, scan_scratch(N) * 8, s->stream));
    LQ_CUDA_TRY(cudaMallocAsync(&d_out, n_shots * 8, s->stream));
    if (s->dtype == LQ_C128)
        k_probs_exact_c128<<<grid_for(N, 256), 256, 0, s->stream>>>((const double2 *)s->d, p, N);
    else
        k_probs_exact_c64<<<grid_for(N, 256), 256, 0, s->stream>>>((const float2 *)s->d, p, N);
    LQ_TRY(scan_inclusive(p, cdf, tot, N, s->stream));
    k_sample<<<grid_for(n_shots, 256), 256, 0, s->stream>>>(cdf, N, n_shots, seed, d_out);
    LQ_CUDA_TRY(cudaGetLastError());
    LQ_CUDA_TRY(cudaMemcpyAsync(host_out, d_out, n_shots * 8, cudaMemcpyDeviceToHost, s->stream));
    LQ_CUDA_TRY(cudaFreeAsync(tot, s->stream));
    LQ_CUDA_TRY(cudaFreeAsync(p, s->stream));
    LQ_CUDA_TRY(cudaFreeAsync(cdf, s->stream));
    LQ_CUDA_TRY(cudaFreeAsync(d_out, s->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return LQ_OK;
}

int lq_expectation_pauli(const lq_state *s, const lq_pauli_term *terms, int nterms,
                         int y_convention, double *out, double *per_term) {
    LQ_TRY(check_state(s));
    if (!out) return set_error(LQ_ERR_INVALID_ARG, "null output");
    if (nterms < 0 || (nterms > 0 && !terms))
        return set_error(LQ_ERR_INVALID_ARG, "bad term list");
    if (y_convention != LQ_Y_REFERENCE && y_convention != LQ_Y_TEXTBOOK)
        return set_error(LQ_ERR_INVALID_ARG, "unknown Y convention %d", y_convention);
    if (nterms == 0) {
        *out = 0.0;
        return LQ_OK;
    }
    return expectation_impl(s, terms, nterms, y_convention, out, per_term);
}

}  // extern "C"
