// RT surrogate (thor_b200/csrc/surrogate.cu): network, training buffers, step hooks.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "thorx_internal.h"
#include "umma.cuh"

namespace thorx {

struct SurNet { // shapes and standardisation, passed to kernels by value
    int    nv, n_in, Kin, H, Nout;
    float *in_mean, *in_std, *out_mean, *out_std;
};

struct SurLog { // ring of logged plain-RT columns: X [cap][n_in] raw features, Y [cap][nv] K/s
    float*     X;
    float*     Y;
    long long  cap;
    long long* count; // device: columns logged so far
    long long* base;  // device: first slot of the current step, -1 when RT did not run
};

struct SurLayer {
    int            N, K;                      // padded output and input widths
    float *        W, *b, *mW, *vW, *mb, *vb; // f32 master weights and Adam moments
    float *        gW, *gb;                   // gradients (gW has max(N, 128) rows)
    __nv_bfloat16 *Wbf, *Wt;                  // bf16 [N][K] and its transpose [K][N]
};

struct Surrogate {
    SurNet             net{};
    SurLog             log{};
    SurLayer           lay[4]{};
    uint64_t           seed         = 0;
    int                Bcap         = 0; // rows of the activation buffers
    long long          adam_t       = 0;
    int                period       = 16;
    double             tol          = 0.05;
    bool               norm_fitted  = false;
    size_t             device_bytes = 0;
    std::vector<void*> allocs;
    __nv_bfloat16 *    X0 = nullptr, *dY = nullptr, *T1 = nullptr, *T2 = nullptr;
    __nv_bfloat16*     A[3]{};
    __nv_bfloat16*     dZ[2]{};
    float *            Y = nullptr, *tgt = nullptr, *dYf = nullptr;
    float*             Yt = nullptr; // inference output, transposed: [Nout][Bcap]
    __nv_bfloat16*     Gd[3]{}; // gelu'(pre-activation) of the hidden layers (training)
    float*             splitk   = nullptr; // split-K partial weight gradients
    float*             colpart  = nullptr; // column-sum partials
    static constexpr int kMaxSplits = 32;
    double*            lpart    = nullptr;
    int                lpart_n  = 0;
    unsigned int*      err      = nullptr;
    unsigned int*      stats    = nullptr; // re-checked, failed, max error (1e-6), RT columns
    uint8_t*           fallback = nullptr;

    int  init(int nv, int hidden, long long log_capacity, int batch_rows, int ncols, uint64_t seed);
    void release();
    void cast_all(cudaStream_t st);
    void forward(int B, cudaStream_t st, bool keep_z = true);
    void backward(int B, cudaStream_t st);
    void adam(float lr, cudaStream_t st);
    void fit_normalisation(long long rows, cudaStream_t st);
    void train_batch(long long nlogged, int B, float lr, cudaStream_t st);
    void load_host_batch(const float* dx, const float* dt, int B, cudaStream_t st);
    void step_features(const Geometry& g, const State& s, const RtFields& f, cudaStream_t st);
    void step_combine(const Geometry& g, const Phys& P, const State& s, const RtFields& f,
                      cudaStream_t st);
    void log_step(const Geometry& g, const State& s, const RtFields& f, cudaStream_t st);
    // the columns the plain RT ran on in surrogate mode (f.fallback, f.period), into the log
    void log_used(const Geometry& g, const State& s, const RtFields& f, cudaStream_t st);
    void gemm_n(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K,
                const umma::EpiArgs& e, cudaStream_t st);
    void gemm_wgrad(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K,
                    float* out, cudaStream_t st);
    void colsum(const float* G, int B, int N, float* db, cudaStream_t st);
    void colsum(const __nv_bfloat16* G, int B, int N, float* db, cudaStream_t st);
    void gemm_gelu_bwd(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K,
                       const umma::EpiArgs& e, cudaStream_t st);
};

} // namespace thorx
