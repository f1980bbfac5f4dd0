// CPU oracle for the learned warm start's network -- TEST INFRASTRUCTURE ONLY.
//
// The same fully connected network as the engine's lq_mlp_* calls, evaluated in
// FP64: in_dim -> hidden (x depth, exact GELU x * Phi(x)) -> out_dim (linear),
// flat parameters per layer W (out x in, row major) then b (out), loss
// sum(mask * (1 - cos(y - t))) / sum(mask).  Used to check the device's FP32
// forward pass and gradients; pinned itself by central finite differences in
// the CPU test suite.  There is no reference counterpart (the reference has no
// network); the definition lives in include/logosq_b200.h.
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

struct Shape {
    std::vector<int> dims;
    std::vector<size_t> woff, boff;
};

Shape make_shape(int in, int hidden, int depth, int out) {
    Shape s;
    s.dims.push_back(in);
    for (int d = 0; d < depth; ++d) s.dims.push_back(hidden);
    s.dims.push_back(out);
    size_t off = 0;
    for (size_t l = 0; l + 1 < s.dims.size(); ++l) {
        s.woff.push_back(off);
        off += (size_t)s.dims[l] * s.dims[l + 1];
        s.boff.push_back(off);
        off += s.dims[l + 1];
    }
    return s;
}

double gelu(double z) { return 0.5 * z * (1.0 + std::erf(z / std::sqrt(2.0))); }
double gelu_d(double z) {
    return 0.5 * (1.0 + std::erf(z / std::sqrt(2.0))) +
           z * std::exp(-0.5 * z * z) / std::sqrt(2.0 * M_PI);
}

}  // namespace

extern "C" {

int64_t or_mlp_num_params(int in, int hidden, int depth, int out) {
    Shape s = make_shape(in, hidden, depth, out);
    return (int64_t)(s.boff.back() + s.dims.back());
}

// y[batch x out] from the parameters (float, as the device stores them).
void or_mlp_forward(int in, int hidden, int depth, int out, const float *params, const float *x,
                    int batch, double *y) {
    Shape s = make_shape(in, hidden, depth, out);
    const int L = (int)s.dims.size() - 1;
    for (int r = 0; r < batch; ++r) {
        std::vector<double> h(x + (size_t)r * in, x + (size_t)(r + 1) * in);
        for (int l = 0; l < L; ++l) {
            const int K = s.dims[l], N = s.dims[l + 1];
            std::vector<double> o(N);
            for (int j = 0; j < N; ++j) {
                double acc = params[s.boff[l] + j];
                for (int k = 0; k < K; ++k)
                    acc += (double)params[s.woff[l] + (size_t)j * K + k] * h[k];
                o[j] = l < L - 1 ? gelu(acc) : acc;
            }
            h.swap(o);
        }
        for (int j = 0; j < out; ++j) y[(size_t)r * out + j] = h[j];
    }
}

// Loss and gradient (double) w.r.t. every parameter.
double or_mlp_loss_grad(int in, int hidden, int depth, int out, const double *params,
                        const float *x, const float *target, const float *mask, int batch,
                        double *grad) {
    Shape s = make_shape(in, hidden, depth, out);
    const int L = (int)s.dims.size() - 1;
    const size_t np = s.boff.back() + s.dims.back();
    for (size_t i = 0; i < np; ++i) grad[i] = 0.0;
    double msum = 0.0;
    for (int i = 0; i < batch * out; ++i) msum += mask[i];
    double loss = 0.0;
    for (int r = 0; r < batch; ++r) {
        std::vector<std::vector<double>> H(L + 1), Z(L + 1);
        H[0].assign(x + (size_t)r * in, x + (size_t)(r + 1) * in);
        for (int l = 0; l < L; ++l) {
            const int K = s.dims[l], N = s.dims[l + 1];
            H[l + 1].resize(N);
            Z[l + 1].resize(N);
            for (int j = 0; j < N; ++j) {
                double acc = params[s.boff[l] + j];
                for (int k = 0; k < K; ++k) acc += params[s.woff[l] + (size_t)j * K + k] * H[l][k];
                Z[l + 1][j] = acc;
                H[l + 1][j] = l < L - 1 ? gelu(acc) : acc;
            }
        }
        std::vector<double> d(out);
        for (int j = 0; j < out; ++j) {
            const double m = mask[(size_t)r * out + j];
            const double diff = H[L][j] - target[(size_t)r * out + j];
            loss += m * (1.0 - std::cos(diff)) / msum;
            d[j] = m * std::sin(diff) / msum;
        }
        for (int l = L - 1; l >= 0; --l) {
            const int K = s.dims[l], N = s.dims[l + 1];
            if (l < L - 1)
                for (int j = 0; j < N; ++j) d[j] *= gelu_d(Z[l + 1][j]);
            std::vector<double> dn(K, 0.0);
            for (int j = 0; j < N; ++j) {
                grad[s.boff[l] + j] += d[j];
                for (int k = 0; k < K; ++k) {
                    grad[s.woff[l] + (size_t)j * K + k] += d[j] * H[l][k];
                    dn[k] += d[j] * params[s.woff[l] + (size_t)j * K + k];
                }
            }
            d.swap(dn);
        }
    }
    return loss;
}

}  // extern "C"
