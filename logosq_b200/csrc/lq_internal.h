// Internal declarations shared by the translation units of liblogosq_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/logosq_b200.h"

namespace lq {

// ---------------------------------------------------------------------------
// Errors: every C entry point returns a status and records a message in a
// thread-local buffer read by lq_last_error().
// ---------------------------------------------------------------------------
int set_error(int code, const char *fmt, ...);
void clear_error();

#define LQ_CUDA_TRY(expr)                                                             \
    do {                                                                              \
        cudaError_t _e = (expr);                                                      \
        if (_e != cudaSuccess) {                                                      \
            return ::lq::set_error(_e == cudaErrorMemoryAllocation ? LQ_ERR_OOM        \
                                                                   : LQ_ERR_CUDA,      \
                                   "%s failed: %s (%s:%d)", #expr,                    \
                                   cudaGetErrorString(_e), __FILE__, __LINE__);       \
        }                                                                             \
    } while (0)

#define LQ_TRY(expr)                 \
    do {                             \
        int _rc = (expr);            \
        if (_rc != LQ_OK) return _rc; \
    } while (0)

// ---------------------------------------------------------------------------
// Device-side complex helpers (complex128 as double2, complex64 as float2).
// ---------------------------------------------------------------------------
struct Mat2 {  // 2x2 complex, row-major
    double2 m00, m01, m10, m11;
};

struct Phases4 {  // up to 4 complex phases
    double2 p[4];
};

// Reduction scratch sizes (per state handle).
constexpr int kRedBlocks = 148 * 8;   // partial slots of a two-stage reduction
constexpr int kMaxTermsPerPass = 32;  // Pauli terms accumulated per sweep

// Flag word written by kernels that wait (bounded) on a barrier.
constexpr unsigned kFlagTimeout = 1u;

}  // namespace lq

// The opaque handle of the C ABI.
struct lq_state {
    int n = 0;
    int dtype = LQ_C128;
    int device = 0;
    void *d = nullptr;        // 2^n amplitudes
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    double *d_red = nullptr;  // kRedBlocks * 2 * kMaxTermsPerPass doubles
    double *h_red = nullptr;  // pinned mirror of the final reduction results
    unsigned *d_flag = nullptr;  // timeout / error flags of waiting kernels
    // Per-handle device buffer for gate programs of fused passes.
    void *d_prog = nullptr;
    size_t prog_cap = 0;
    // Statistics of the last circuit call.
    int last_launches = 0;
    int last_passes = 0;
    // The fused program now in d_prog and its launch list, kept so that the same
    // circuit submitted again skips planning and the upload (fused.cu).  Any
    // other writer of d_prog goes through ensure_prog, which clears prog_valid.
    void *plan_cache = nullptr;
    bool prog_valid = false;
};

namespace lq {

inline size_t amp_bytes(int dtype) { return dtype == LQ_C64 ? 8 : 16; }

int check_state(const lq_state *s);
int check_qubit(const lq_state *s, int q);
int ensure_prog(lq_state *s, size_t bytes);

// gates.cu
int apply_gate_c128(lq_state *s, const lq_gate *g, const double *theta, int ntheta,
                    int *launches);
int apply_gate_c64(lq_state *s, const lq_gate *g, const double *theta, int ntheta,
                   int *launches);
int gate_num_qubits(int kind);
int validate_gate(const lq_gate *g, int n, int ntheta);
double gate_angle(const lq_gate *g, int k, const double *theta);
// Dense matrix (2^k x 2^k complex, row-major, qubit list order: q[0] high bit)
// of a gate as the reference applies it.  Returns k (number of qubits).
int gate_matrix(const lq_gate *g, const double *theta, double *m /* 2*64 doubles */);
// Classification used by the planner and the per-gate dispatcher.
enum GateClass { kClassGeneral = 0, kClassDiagonal = 1, kClassPermutation = 2 };
int gate_class(int kind);

// api_state.cu
int normalize_impl(lq_state *s);
// Record the state's FP64 squared norm; later rescale the state to it.
int norm_snapshot(lq_state *s);
int norm_restore(lq_state *s);
int expectation_impl(const lq_state *s, const lq_pauli_term *terms, int nterms, int yconv,
                     double *out, double *per_term);

// profile.cu: optional CUDA-event timing of launches, by kernel class.
enum ProfClass { kProfFused = 0, kProfGate = 1, kProfReduce = 2, kProfBatch = 3, kProfTc = 4,
                 kProfClasses = 5 };
bool prof_enabled();
// Record an event pair around a launch: call prof_begin before, prof_end after.
void prof_begin(cudaStream_t st, int cls);
void prof_end(cudaStream_t st, int cls);

// fused.cu
void free_plan_cache(lq_state *s);
int apply_circuit_impl(lq_state *s, const lq_gate *ops, int nops, const double *theta,
                       int ntheta, int mode);
int apply_block_impl(lq_state *s, int k, const int *qubits, const double *m);

}  // namespace lq
