// Learned warm start and exact ground energies.
//
// 1. A small MLP maps Hamiltonian couplings to ansatz angles: input (Jx, Jy, Jz
//    per bond, padded) + field, `depth` hidden layers of width `hidden` with
//    GELU, linear output of `out` angles.  Training and inference run on
//    hand-written FP32 kernels: a tiled SGEMM with fused bias / GELU epilogue,
//    its transposed forms for the backward pass, a periodic angle loss
//    sum(1 - cos(y - t)) over a validity mask, and Adam.
// 2. FP64 Lanczos on the full 2^n space with a Pauli-sum matrix-vector kernel
//    (textbook Pauli convention: H is real symmetric for X/Y/Z strings with an
//    even number of Y factors), full reorthogonalisation, and a host bisection
//    on the tridiagonal matrix.  This is the "exact" E0 the learned warm start
//    is judged against (the reference has no exact solver).
#include <algorithm>
#include <cmath>
#include <random>

#include "lq_internal.h"

namespace lq {

// ---------------------------------------------------------------------------
// FP32 GEMM: C[M x N] = op(A) op(B) (+ bias[N]) (+ C if accumulate), with an
// optional GELU epilogue that also stores the pre-activation Z.
//   op(A) = A (M x K, lda) or A^T (A is K x M)
//   op(B) = B (K x N, ldb) or B^T (B is N x K)
// 64 x 64 block tile, 16 x 16 threads, 4 x 4 outputs per thread, K step 16.
// ---------------------------------------------------------------------------
constexpr int GB = 64, GK = 16;

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float *__restrict__ A,
                                              int lda, const float *__restrict__ B, int ldb,
                                              float *__restrict__ Cm, int ldc,
                                              const float *__restrict__ bias, int accumulate,
                                              int gelu, float *__restrict__ Z) {
    __shared__ float As[GK][GB + 4];
    __shared__ float Bs[GK][GB + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * GB, n0 = blockIdx.x * GB;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int i = threadIdx.x; i < GK * GB; i += 256) {
            const int kk = i / GB, mm = i % GB;
            const int gm = m0 + mm, gk = k0 + kk;
            float va = 0.f;
            if (gm < M && gk < K) va = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            As[kk][mm] = va;
            const int gn = n0 + mm;
            float vb = 0.f;
            if (gn < N && gk < K) vb = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
            Bs[kk][mm] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gn = n0 + tx * 4 + j;
            if (gn >= N) continue;
            float v = acc[i][j];
            if (bias) v += bias[gn];
            if (accumulate) v += Cm[(size_t)gm * ldc + gn];
            if (gelu) {
                Z[(size_t)gm * ldc + gn] = v;
                v = 0.5f * v * (1.f + erff(v * 0.70710678118654752f));
            }
            Cm[(size_t)gm * ldc + gn] = v;
        }
    }
}

static void sgemm(cudaStream_t st, bool ta, bool tb, int M, int N, int K, const float *A, int lda,
                  const float *B, int ldb, float *Cm, int ldc, const float *bias, bool acc,
                  bool gelu, float *Z) {
    dim3 grid((N + GB - 1) / GB, (M + GB - 1) / GB);
    if (!ta && !tb)
        k_sgemm<false, false><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, Cm, ldc, bias, acc,
                                                    gelu, Z);
    else if (!ta && tb)
        k_sgemm<false, true><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, Cm, ldc, bias, acc,
                                                   gelu, Z);
    else if (ta && !tb)
        k_sgemm<true, false><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, Cm, ldc, bias, acc,
                                                   gelu, Z);
    else
        k_sgemm<true, true><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, Cm, ldc, bias, acc,
                                                  gelu, Z);
}

// dZ = dH * gelu'(Z)
__global__ void k_gelu_bwd(const float *__restrict__ Z, float *__restrict__ dH, int count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float z = Z[i];
        const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
        const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
        dH[i] *= cdf + z * pdf;
    }
}

// Periodic angle loss: sum mask * (1 - cos(y - t)) / sum(mask); dY = mask sin(y - t) / sum(mask).
__global__ void k_angle_loss(const float *__restrict__ Y, const float *__restrict__ T,
                             const float *__restrict__ Mk, float *__restrict__ dY, int count,
                             float inv_norm, double *__restrict__ loss_acc) {
    __shared__ double sh[256];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float d = Y[i] - T[i];
        const float m = Mk[i];
        acc += (double)(m * (1.f - cosf(d)));
        dY[i] = m * sinf(d) * inv_norm;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss_acc, sh[0] * inv_norm);
}

// db[n] = sum_m dY[m][n]
__global__ void k_bias_grad(const float *__restrict__ dY, float *__restrict__ db, int M, int N) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int m = 0; m < M; ++m) s += dY[(size_t)m * N + n];
    db[n] = s;
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int64_t count, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// ---------------------------------------------------------------------------
// Lanczos: y = H x for a Pauli sum (textbook convention, real H).
// For an even number of Y factors, (P x)_i = Re((-i)^ny) (-1)^popcount(i & z) x_{i ^ x}.
// ---------------------------------------------------------------------------
struct RealTerm {
    uint64_t x, z;
    double c;  // coefficient * Re((-i)^ny)
};

__global__ void k_pauli_matvec(const double *__restrict__ in, double *__restrict__ out, int n,
                               const RealTerm *__restrict__ terms, int nt) {
    extern __shared__ RealTerm s_t[];
    for (int t = threadIdx.x; t < nt; t += blockDim.x) s_t[t] = terms[t];
    __syncthreads();
    const uint64_t N = 1ull << n;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int t = 0; t < nt; ++t) {
            const double s = (__popcll(i & s_t[t].z) & 1) ? -s_t[t].c : s_t[t].c;
            acc += s * in[i ^ s_t[t].x];
        }
        out[i] = acc;
    }
}

__global__ void k_axpy(double *__restrict__ y, const double *__restrict__ x, double a, uint64_t N) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}

// partial[j * gridDim.x + b] = block b's share of <V_j, w> for j = blockIdx.y.
__global__ void k_multi_dot(const double *__restrict__ V, const double *__restrict__ w, uint64_t N,
                            double *__restrict__ partial) {
    __shared__ double sh[256];
    const double *vj = V + (size_t)blockIdx.y * N;
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x)
        acc += vj[i] * w[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = sh[0];
}

// w -= sum_j c[j] V_j   (classical Gram-Schmidt step against the Lanczos basis)
__global__ void k_multi_sub(const double *__restrict__ V, const double *__restrict__ c, int k,
                            uint64_t N, double *__restrict__ w) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        double acc = w[i];
        for (int j = 0; j < k; ++j) acc -= c[j] * V[(size_t)j * N + i];
        w[i] = acc;
    }
}

__global__ void k_scale(double *__restrict__ y, const double *__restrict__ x, double a,
                        uint64_t N) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x)
        y[i] = a * x[i];
}

// Smallest eigenvalue of the symmetric tridiagonal (alpha, beta) by bisection
// on the Sturm sequence count.
static double tridiag_min_eig(const std::vector<double> &a, const std::vector<double> &b) {
    const int k = (int)a.size();
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < k; ++i) {
        const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < k ? std::fabs(b[i]) : 0.0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    auto count_below = [&](double x) {
        int cnt = 0;
        double d = 1.0;
        for (int i = 0; i < k; ++i) {
            d = a[i] - x - (i > 0 ? b[i - 1] * b[i - 1] / d : 0.0);
            if (d == 0.0) d = -1e-300;
            if (d < 0) ++cnt;
        }
        return cnt;
    };
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (count_below(mid) >= 1) hi = mid;
        else lo = mid;
        if (hi - lo < 1e-15 * std::max(1.0, std::fabs(mid))) break;
    }
    return 0.5 * (lo + hi);
}

}  // namespace lq

struct lq_mlp {
    int in_dim = 0, hidden = 0, depth = 0, out_dim = 0;
    std::vector<int> dims;           // layer widths: in, hidden x depth, out
    std::vector<size_t> woff, boff;  // offsets in the flat parameter vector
    int64_t nparams = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // device
    int64_t adam_t = 0;
    // activations for a batch (device), capacity in rows
    int cap = 0;
    std::vector<float *> H, Z;  // H[0] = input, H[l+1] = layer l output; Z pre-activations
    float *target = nullptr, *mask = nullptr, *dA = nullptr, *dB = nullptr;
    double *loss_d = nullptr;
    cudaStream_t stream = nullptr;
};

namespace lq {

static int mlp_reserve(lq_mlp *net, int batch) {
    if (batch <= net->cap) return LQ_OK;
    for (auto p : net->H) cudaFree(p);
    for (auto p : net->Z) cudaFree(p);
    cudaFree(net->target);
    cudaFree(net->mask);
    cudaFree(net->dA);
    cudaFree(net->dB);
    net->target = net->mask = net->dA = net->dB = nullptr;
    net->cap = 0;
    net->H.assign(net->dims.size(), nullptr);
    net->Z.assign(net->dims.size(), nullptr);
    int widest = 0;
    for (size_t l = 0; l < net->dims.size(); ++l) {
        LQ_CUDA_TRY(cudaMalloc(&net->H[l], sizeof(float) * batch * net->dims[l]));
        LQ_CUDA_TRY(cudaMalloc(&net->Z[l], sizeof(float) * batch * net->dims[l]));
        widest = std::max(widest, net->dims[l]);
    }
    LQ_CUDA_TRY(cudaMalloc(&net->target, sizeof(float) * batch * net->out_dim));
    LQ_CUDA_TRY(cudaMalloc(&net->mask, sizeof(float) * batch * net->out_dim));
    LQ_CUDA_TRY(cudaMalloc(&net->dA, sizeof(float) * batch * widest));
    LQ_CUDA_TRY(cudaMalloc(&net->dB, sizeof(float) * batch * widest));
    net->cap = batch;
    return LQ_OK;
}

static int mlp_forward_dev(lq_mlp *net, int batch) {
    const int L = (int)net->dims.size() - 1;
    for (int l = 0; l < L; ++l) {
        const int K = net->dims[l], Nn = net->dims[l + 1];
        const bool last = l == L - 1;
        // H[l+1] = H[l] (batch x K) . W^T (W stored out x in) + b
        sgemm(net->stream, false, true, batch, Nn, K, net->H[l], K, net->p + net->woff[l], K,
              net->H[l + 1], Nn, net->p + net->boff[l], false, !last, net->Z[l + 1]);
    }
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

// Backward sweep from dL/dy (in net->dA, batch x out_dim) after a forward pass
// of the same batch; writes dL/dparams to net->g.
static int mlp_backward_dev(lq_mlp *net, int batch) {
    cudaStream_t st = net->stream;
    float *dY = net->dA, *dX = net->dB;
    const int L = (int)net->dims.size() - 1;
    for (int l = L - 1; l >= 0; --l) {
        const int K = net->dims[l], Nn = net->dims[l + 1];
        if (l < L - 1) {  // through the GELU of layer l's output
            k_gelu_bwd<<<std::max(1, std::min(1184, (batch * Nn + 255) / 256)), 256, 0, st>>>(
                net->Z[l + 1], dY, batch * Nn);
        }
        // dW (Nn x K) = dY^T (Nn x batch) . H[l] (batch x K)
        sgemm(st, true, false, Nn, K, batch, dY, Nn, net->H[l], K, net->g + net->woff[l], K,
              nullptr, false, false, nullptr);
        k_bias_grad<<<(Nn + 127) / 128, 128, 0, st>>>(dY, net->g + net->boff[l], batch, Nn);
        if (l > 0) {
            // dX (batch x K) = dY (batch x Nn) . W (Nn x K)
            sgemm(st, false, false, batch, K, Nn, dY, Nn, net->p + net->woff[l], K, dX, K,
                  nullptr, false, false, nullptr);
            std::swap(dY, dX);
        }
    }
    LQ_CUDA_TRY(cudaGetLastError());
    return LQ_OK;
}

}  // namespace lq

using namespace lq;

extern "C" {

int lq_mlp_create(int in_dim, int hidden, int depth, int out_dim, uint64_t seed, lq_mlp **out) {
    if (!out || in_dim < 1 || hidden < 1 || depth < 1 || out_dim < 1)
        return set_error(LQ_ERR_INVALID_ARG, "bad MLP shape");
    lq_mlp *net = new lq_mlp();
    net->in_dim = in_dim;
    net->hidden = hidden;
    net->depth = depth;
    net->out_dim = out_dim;
    net->dims.push_back(in_dim);
    for (int d = 0; d < depth; ++d) net->dims.push_back(hidden);
    net->dims.push_back(out_dim);
    size_t off = 0;
    for (size_t l = 0; l + 1 < net->dims.size(); ++l) {
        net->woff.push_back(off);
        off += (size_t)net->dims[l] * net->dims[l + 1];
        net->boff.push_back(off);
        off += net->dims[l + 1];
    }
    net->nparams = (int64_t)off;
    // He-style uniform init from a seeded generator (host), zero biases; the
    // output layer is scaled down so initial angles start near zero.
    std::vector<float> init(off, 0.f);
    std::mt19937_64 rng(seed);
    for (size_t l = 0; l + 1 < net->dims.size(); ++l) {
        const double bound =
            std::sqrt(6.0 / net->dims[l]) * (l + 2 == net->dims.size() ? 0.1 : 1.0);
        std::uniform_real_distribution<double> u(-bound, bound);
        for (size_t i = 0; i < (size_t)net->dims[l] * net->dims[l + 1]; ++i)
            init[net->woff[l] + i] = (float)u(rng);
    }
    auto fail = [&](cudaError_t e) {
        if (net->stream) cudaStreamDestroy(net->stream);
        cudaFree(net->loss_d);
        cudaFree(net->p);
        cudaFree(net->g);
        cudaFree(net->m);
        cudaFree(net->v);
        delete net;
        return set_error(e == cudaErrorMemoryAllocation ? LQ_ERR_OOM : LQ_ERR_CUDA, "%s",
                         cudaGetErrorString(e));
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking))) return fail(e);
    if ((e = cudaMalloc(&net->p, off * 4))) return fail(e);
    if ((e = cudaMalloc(&net->g, off * 4))) return fail(e);
    if ((e = cudaMalloc(&net->m, off * 4))) return fail(e);
    if ((e = cudaMalloc(&net->v, off * 4))) return fail(e);
    if ((e = cudaMalloc(&net->loss_d, sizeof(double)))) return fail(e);
    if ((e = cudaMemcpy(net->p, init.data(), off * 4, cudaMemcpyHostToDevice))) return fail(e);
    if ((e = cudaMemset(net->m, 0, off * 4)) || (e = cudaMemset(net->v, 0, off * 4)) ||
        (e = cudaMemset(net->g, 0, off * 4)))
        return fail(e);
    *out = net;
    return LQ_OK;
}

int lq_mlp_destroy(lq_mlp *net) {
    if (!net) return LQ_OK;
    cudaStreamSynchronize(net->stream);
    for (auto p : net->H) cudaFree(p);
    for (auto p : net->Z) cudaFree(p);
    cudaFree(net->target);
    cudaFree(net->mask);
    cudaFree(net->dA);
    cudaFree(net->dB);
    cudaFree(net->loss_d);
    cudaFree(net->p);
    cudaFree(net->g);
    cudaFree(net->m);
    cudaFree(net->v);
    cudaStreamDestroy(net->stream);
    delete net;
    return LQ_OK;
}

int lq_mlp_num_params(const lq_mlp *net, int64_t *out) {
    if (!net || !out) return set_error(LQ_ERR_INVALID_ARG, "null argument");
    *out = net->nparams;
    return LQ_OK;
}

int lq_mlp_get_params(const lq_mlp *net, float *host, int64_t count) {
    if (!net || !host) return set_error(LQ_ERR_INVALID_ARG, "null argument");
    if (count != net->nparams)
        return set_error(LQ_ERR_PARAM_COUNT, "Parameter count mismatch: expected %lld, got %lld",
                         (long long)net->nparams, (long long)count);
    LQ_CUDA_TRY(cudaMemcpy(host, net->p, count * 4, cudaMemcpyDeviceToHost));
    return LQ_OK;
}

int lq_mlp_set_params(lq_mlp *net, const float *host, int64_t count) {
    if (!net || !host) return set_error(LQ_ERR_INVALID_ARG, "null argument");
    if (count != net->nparams)
        return set_error(LQ_ERR_PARAM_COUNT, "Parameter count mismatch: expected %lld, got %lld",
                         (long long)net->nparams, (long long)count);
    LQ_CUDA_TRY(cudaMemcpy(net->p, host, count * 4, cudaMemcpyHostToDevice));
    return LQ_OK;
}

int lq_mlp_get_grads(const lq_mlp *net, float *host, int64_t count) {
    if (!net || !host) return set_error(LQ_ERR_INVALID_ARG, "null argument");
    if (count != net->nparams)
        return set_error(LQ_ERR_PARAM_COUNT, "Parameter count mismatch: expected %lld, got %lld",
                         (long long)net->nparams, (long long)count);
    LQ_CUDA_TRY(cudaMemcpy(host, net->g, count * 4, cudaMemcpyDeviceToHost));
    return LQ_OK;
}

int lq_mlp_forward(lq_mlp *net, const float *x, int batch, float *y) {
    if (!net || !x || !y || batch < 1) return set_error(LQ_ERR_INVALID_ARG, "bad arguments");
    LQ_TRY(mlp_reserve(net, batch));
    LQ_CUDA_TRY(cudaMemcpyAsync(net->H[0], x, sizeof(float) * batch * net->in_dim,
                                cudaMemcpyHostToDevice, net->stream));
    LQ_TRY(mlp_forward_dev(net, batch));
    LQ_CUDA_TRY(cudaMemcpyAsync(y, net->H.back(), sizeof(float) * batch * net->out_dim,
                                cudaMemcpyDeviceToHost, net->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(net->stream));
    return LQ_OK;
}

int lq_mlp_loss_grad(lq_mlp *net, const float *x, const float *target, const float *mask,
                     int batch, double *loss) {
    if (!net || !x || !target || !mask || batch < 1)
        return set_error(LQ_ERR_INVALID_ARG, "bad arguments");
    LQ_TRY(mlp_reserve(net, batch));
    cudaStream_t st = net->stream;
    const int O = net->out_dim;
    double msum = 0.0;
    for (int i = 0; i < batch * O; ++i) msum += mask[i];
    if (msum <= 0) return set_error(LQ_ERR_INVALID_ARG, "empty mask");
    LQ_CUDA_TRY(cudaMemcpyAsync(net->H[0], x, sizeof(float) * batch * net->in_dim,
                                cudaMemcpyHostToDevice, st));
    LQ_CUDA_TRY(cudaMemcpyAsync(net->target, target, sizeof(float) * batch * O,
                                cudaMemcpyHostToDevice, st));
    LQ_CUDA_TRY(cudaMemcpyAsync(net->mask, mask, sizeof(float) * batch * O,
                                cudaMemcpyHostToDevice, st));
    LQ_TRY(mlp_forward_dev(net, batch));
    LQ_CUDA_TRY(cudaMemsetAsync(net->loss_d, 0, sizeof(double), st));
    k_angle_loss<<<std::max(1, std::min(148, (batch * O + 255) / 256)), 256, 0, st>>>(
        net->H.back(), net->target, net->mask, net->dA, batch * O, (float)(1.0 / msum),
        net->loss_d);
    LQ_TRY(mlp_backward_dev(net, batch));
    double lv = 0.0;
    LQ_CUDA_TRY(cudaMemcpyAsync(&lv, net->loss_d, sizeof(double), cudaMemcpyDeviceToHost, st));
    LQ_CUDA_TRY(cudaStreamSynchronize(st));
    if (loss) *loss = lv;
    return LQ_OK;
}

int lq_mlp_backward(lq_mlp *net, const float *x, const float *dy, int batch) {
    if (!net || !x || !dy || batch < 1) return set_error(LQ_ERR_INVALID_ARG, "bad arguments");
    LQ_TRY(mlp_reserve(net, batch));
    cudaStream_t st = net->stream;
    LQ_CUDA_TRY(cudaMemcpyAsync(net->H[0], x, sizeof(float) * batch * net->in_dim,
                                cudaMemcpyHostToDevice, st));
    LQ_TRY(mlp_forward_dev(net, batch));
    LQ_CUDA_TRY(cudaMemcpyAsync(net->dA, dy, sizeof(float) * batch * net->out_dim,
                                cudaMemcpyHostToDevice, st));
    LQ_TRY(mlp_backward_dev(net, batch));
    LQ_CUDA_TRY(cudaStreamSynchronize(st));
    return LQ_OK;
}

int lq_mlp_reset_adam(lq_mlp *net) {
    if (!net) return set_error(LQ_ERR_INVALID_ARG, "null network");
    LQ_CUDA_TRY(cudaMemsetAsync(net->m, 0, net->nparams * 4, net->stream));
    LQ_CUDA_TRY(cudaMemsetAsync(net->v, 0, net->nparams * 4, net->stream));
    LQ_CUDA_TRY(cudaStreamSynchronize(net->stream));
    net->adam_t = 0;
    return LQ_OK;
}

int lq_mlp_adam_step(lq_mlp *net, float lr, float beta1, float beta2, float eps) {
    if (!net) return set_error(LQ_ERR_INVALID_ARG, "null network");
    net->adam_t += 1;
    const float c1 = 1.f / (1.f - std::pow(beta1, (float)net->adam_t));
    const float c2 = 1.f / (1.f - std::pow(beta2, (float)net->adam_t));
    k_adam<<<592, 256, 0, net->stream>>>(net->p, net->g, net->m, net->v, net->nparams, lr, beta1,
                                         beta2, eps, c1, c2);
    LQ_CUDA_TRY(cudaGetLastError());
    LQ_CUDA_TRY(cudaStreamSynchronize(net->stream));
    return LQ_OK;
}

int lq_lanczos_ground_energy(int num_qubits, const lq_pauli_term *terms, int nterms,
                             int max_iter, double tol, uint64_t seed, double *e0, int *iters) {
    if (!terms || nterms < 1 || !e0 || num_qubits < 1 || num_qubits > 26 || max_iter < 2)
        return set_error(LQ_ERR_INVALID_ARG, "bad Lanczos arguments");
    std::vector<RealTerm> rt;
    for (int t = 0; t < nterms; ++t) {
        const int ny = terms[t].ny;
        if (ny & 1)
            return set_error(LQ_ERR_UNSUPPORTED,
                             "Lanczos needs a real Hamiltonian (even number of Y per term)");
        rt.push_back(RealTerm{terms[t].xmask, terms[t].zmask,
                              terms[t].coefficient * ((ny & 3) == 2 ? -1.0 : 1.0)});
    }
    const uint64_t N = 1ull << num_qubits;
    const int kmax = (int)std::min<uint64_t>(max_iter, N);
    if ((double)(kmax + 2) * (double)N * 8.0 > 32e9)
        return set_error(LQ_ERR_OOM, "Lanczos basis of %d vectors of 2^%d doubles exceeds 32 GB",
                         kmax + 1, num_qubits);
    if (rt.size() * sizeof(RealTerm) > 48 * 1024)
        return set_error(LQ_ERR_INVALID_ARG, "too many Pauli terms for the Lanczos matvec");
    constexpr int kDotBlocks = 148;
    cudaStream_t st;
    LQ_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    double *V = nullptr, *w = nullptr, *part = nullptr, *coef = nullptr;
    RealTerm *dterms = nullptr;
    auto cleanup = [&]() {
        cudaFree(V);
        cudaFree(w);
        cudaFree(part);
        cudaFree(coef);
        cudaFree(dterms);
        cudaStreamDestroy(st);
    };
    cudaError_t e;
    if ((e = cudaMalloc(&V, sizeof(double) * N * (kmax + 1))) ||
        (e = cudaMalloc(&w, sizeof(double) * N)) ||
        (e = cudaMalloc(&part, sizeof(double) * kDotBlocks * (kmax + 1))) ||
        (e = cudaMalloc(&coef, sizeof(double) * (kmax + 1))) ||
        (e = cudaMalloc(&dterms, sizeof(RealTerm) * rt.size()))) {
        cleanup();
        return set_error(e == cudaErrorMemoryAllocation ? LQ_ERR_OOM : LQ_ERR_CUDA, "%s",
                         cudaGetErrorString(e));
    }
    if ((e = cudaMemcpy(dterms, rt.data(), sizeof(RealTerm) * rt.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess) {
        cleanup();
        return set_error(LQ_ERR_CUDA, "%s", cudaGetErrorString(e));
    }
    {  // seeded random start vector (host), normalised
        std::vector<double> v0(N);
        std::mt19937_64 rng(seed);
        std::normal_distribution<double> nd(0.0, 1.0);
        double s = 0.0;
        for (auto &x : v0) {
            x = nd(rng);
            s += x * x;
        }
        s = 1.0 / std::sqrt(s);
        for (auto &x : v0) x *= s;
        if ((e = cudaMemcpy(V, v0.data(), sizeof(double) * N, cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
            cleanup();
            return set_error(LQ_ERR_CUDA, "%s", cudaGetErrorString(e));
        }
    }
    // <V_j, x> for j < count, block partials summed on the host in a fixed order.
    std::vector<double> hpart((size_t)kDotBlocks * (kmax + 1)), hc(kmax + 1);
    cudaError_t err = cudaSuccess;  // first failure of any launch or copy below
    auto note = [&](cudaError_t r) {
        if (err == cudaSuccess && r != cudaSuccess) err = r;
    };
    auto dots = [&](const double *Vb, int count, const double *x) {
        k_multi_dot<<<dim3(kDotBlocks, count), 256, 0, st>>>(Vb, x, N, part);
        note(cudaGetLastError());
        note(cudaMemcpyAsync(hpart.data(), part, sizeof(double) * kDotBlocks * count,
                             cudaMemcpyDeviceToHost, st));
        note(cudaStreamSynchronize(st));
        for (int j = 0; j < count; ++j) {
            double s = 0.0;
            for (int b = 0; b < kDotBlocks; ++b) s += hpart[(size_t)j * kDotBlocks + b];
            hc[j] = s;
        }
    };
    const int grid = (int)std::min<uint64_t>(1184, (N + 255) / 256);
    std::vector<double> alpha, beta;
    double prev = 1e300, ev = 0.0;
    int k;
    for (k = 0; k < kmax; ++k) {
        double *vk = V + (size_t)k * N;
        k_pauli_matvec<<<grid, 256, sizeof(RealTerm) * rt.size(), st>>>(vk, w, num_qubits, dterms,
                                                                          (int)rt.size());
        dots(vk, 1, w);
        const double a = hc[0];
        alpha.push_back(a);
        k_axpy<<<grid, 256, 0, st>>>(w, vk, -a, N);
        if (k > 0) k_axpy<<<grid, 256, 0, st>>>(w, V + (size_t)(k - 1) * N, -beta[k - 1], N);
        // full reorthogonalisation against V_0..V_k, classical Gram-Schmidt twice
        for (int pass = 0; pass < 2; ++pass) {
            dots(V, k + 1, w);
            note(cudaMemcpyAsync(coef, hc.data(), sizeof(double) * (k + 1),
                                 cudaMemcpyHostToDevice, st));
            k_multi_sub<<<grid, 256, 0, st>>>(V, coef, k + 1, N, w);
        }
        dots(w, 1, w);
        const double b = std::sqrt(std::max(hc[0], 0.0));
        if (err != cudaSuccess) break;
        ev = tridiag_min_eig(alpha, beta);
        if (std::fabs(ev - prev) < tol || b < 1e-12) {
            ++k;
            break;
        }
        prev = ev;
        beta.push_back(b);
        k_scale<<<grid, 256, 0, st>>>(V + (size_t)(k + 1) * N, w, 1.0 / b, N);
    }
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = err;
    cleanup();
    if (e != cudaSuccess) return set_error(LQ_ERR_CUDA, "%s", cudaGetErrorString(e));
    *e0 = ev;
    if (iters) *iters = k;
    return LQ_OK;
}

}  // extern "C"
