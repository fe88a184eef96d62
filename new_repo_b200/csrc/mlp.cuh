// Learned SGS closure: 8 resolved invariants -> 64 -> 64 -> Cs^2 (GELU),
// BF16 weights with FP32 accumulation on the tcgen05 tensor cores.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace les {

constexpr int MLP_IN = 8;
constexpr int MLP_H = 64;
// flat FP32 parameter vector: W1[8][64], b1[64], W2[64][64], b2[64], w3[64], b3
constexpr int MLP_O_W1 = 0;
constexpr int MLP_O_B1 = MLP_O_W1 + MLP_IN * MLP_H;
constexpr int MLP_O_W2 = MLP_O_B1 + MLP_H;
constexpr int MLP_O_B2 = MLP_O_W2 + MLP_H * MLP_H;
constexpr int MLP_O_W3 = MLP_O_B2 + MLP_H;
constexpr int MLP_O_B3 = MLP_O_W3 + MLP_H;
constexpr int MLP_NP = MLP_O_B3 + 1;  // 4801 trainable parameters
// statistics: feature mean[8], std[8], min[8], max[8] (normalised units),
// target mean, target std, target min, max (normalised units: the output is
// clamped to the range it was trained on).  The target is the change of
// log Cs^2 over one dynamic update: Cs^2 = Cs^2_prev * exp(ymu + ysd * y).
constexpr int MLP_S_MU = 0, MLP_S_SD = 8, MLP_S_MIN = 16, MLP_S_MAX = 24, MLP_S_YMU = 32, MLP_S_YSD = 33;
constexpr int MLP_S_YMIN = 34, MLP_S_YMAX = 35;
constexpr int MLP_NS = 36;
constexpr float MLP_LOG_CS_FLOOR = -13.815510557964274f;  // log(1e-6): coefficients below are clamped

// inputs of the feature function (the state's gradients and velocity)
template <typename T>
struct MlpFeatIn {
  const T* d[9];  // dudx dudy dudz dvdx dvdy dvdz dwdx dwdy dwdz
  const T* csprev;  // Cs^2 before this update (the closure's Lagrangian memory)
  int wall_levels;  // levels 1..wall_levels keep the LASD procedure: no range flags there
  long plane;
  int nz;
  int wall;
  float dz, delta, log_delta_z0;
  // buoyant runs: d theta/dz (w nodes) and g/theta_0; feature 7 is then the
  // gradient Richardson number instead of the constant log(Delta/z0)
  const T* dtdz = nullptr;
  float beta = 0.0f;
  float cs_max = 1.0f;  // upper clip of the coefficient
};

constexpr int MLP_COLLECT_BLOCKS = 148 * 8;  // grid of both collection passes
constexpr int MLP_TRAIN_CTAS = 148;          // most CTAs of a training launch
constexpr int MLP_BLEND_BLOCKS = 4;          // blocks per level of the check's error sums

struct MlpDevice {
  float* params = nullptr;     // MLP_NP master weights
  float* stats = nullptr;      // MLP_NS
  uint16_t* img = nullptr;     // packed BF16 operand images: B1 (2 KB), B2 (8 KB), B2T (8 KB)
  float* grad = nullptr;       // MLP_NP
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* dx = nullptr;         // training features (normalised) [cap][8]
  float* dt = nullptr;         // training targets (normalised) [cap]
  float* vx = nullptr;         // validation features
  float* vt = nullptr;
  unsigned long long* counts = nullptr;  // [0] train, [1] validation
  long cap = 0;
  // fixed-order reductions (training is deterministic: no floating-point
  // atomics and no atomically assigned sample slots)
  unsigned long long* boff = nullptr;  // collection: per block (train, validation) count, then first slot
  float* gpart = nullptr;      // training: per CTA gradient [MLP_TRAIN_CTAS][MLP_NP]
  float* lpart = nullptr;      // training: per CTA loss [MLP_TRAIN_CTAS]
  float* scratch = nullptr;    // forward outputs of the host-features path
  int* colflag = nullptr;      // per (i,j) column: bit i = feature i left the training range
  int* range = nullptr;        // raw feature min[8], max[8] of the collected states (order-preserving ints)
  long plane = 0;
};

// feature transforms shared by inference and data collection
// append (features, log cs) pairs: one point in `stride` (seeded hash), every
// point of levels 1..dense_levels, the training pairs of levels 1 and 2
// wall_repeat times; the features' previous coefficient is in.csprev
template <typename T>
void mlp_collect(const MlpFeatIn<T>& in, const T* cs, MlpDevice& m, int stride, int dense_levels, int wall_repeat,
                 unsigned seed, cudaStream_t st);
template <typename T>
void mlp_infer(const MlpFeatIn<T>& in, T* cs, MlpDevice& m, unsigned* status, cudaStream_t st);
// empty the collected feature range
void mlp_reset_range(MlpDevice& m, cudaStream_t st);
// statistics of the collected raw data, then normalisation in place
void mlp_fit_stats(MlpDevice& m, cudaStream_t st);
// opt the tensor-core kernels in to their shared-memory sizes (current device)
void init_mlp_attributes();
// pack the BF16 operand images from the FP32 master weights
void mlp_pack(MlpDevice& m, cudaStream_t st);
// sample order of a training batch: row r of the batch reads sample
// (a * (off + r) + b) mod n of the buffer (a coprime to n: a permutation of
// the buffer per epoch); n = 0 reads rows in order
struct MlpPerm {
  unsigned long long a = 1, b = 0;
  long n = 0, off = 0;
};
// one optimisation pass: gradients of the mean squared error over n samples
// of a buffer (x [.][8], t [.]) into m.grad; with y_out != nullptr also
// writes the network outputs (normalised), in batch-row order.
void mlp_grad(MlpDevice& m, const float* x, const float* t, long n, float* y_out, float* loss_dev, unsigned* status,
              cudaStream_t st, MlpPerm perm = MlpPerm());
void mlp_adam(MlpDevice& m, int step, float lr, cudaStream_t st);
// number of (i,j) columns flagged out of the training range by the last
// inference; per_feature[8] (may be null) gets the columns per feature
int mlp_count_flags(MlpDevice& m, int* dcount, int* per_feature, cudaStream_t st);
// replace flagged columns of cs by cs_dyn; with check, profile[k] (host,
// nz + 2 values) gets the RMS over level k of log(cs) - log(cs_dyn), both
// floored at 1e-6 (derr: MLP_BLEND_BLOCKS * (nz + 2) device doubles)
template <typename T>
void mlp_blend(T* cs, const T* cs_dyn, MlpDevice& m, int nz, bool check, double* derr, double* profile,
               cudaStream_t st);

}  // namespace les
