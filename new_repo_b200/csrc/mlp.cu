// Learned SGS closure kernels on the sm_100a tensor cores (tcgen05).
//
// A tile is 128 points (one tensor-core M = 128 row block); each of the 128
// threads owns one point/row.  Layer 1 (K = 8 features padded to 16) and
// layer 2 (K = 64) run as tcgen05.mma with BF16 operands staged in shared
// memory and FP32 accumulators in TMEM; bias, GELU and the 64 -> 1 output
// layer run on the CUDA cores from the TMEM rows.  The training kernel adds
// the backward pass: the hidden-layer error g2 . W2^T is a third tcgen05
// GEMM, the weight gradients are row reductions accumulated per thread.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "launch.cuh"
#include "mlp.cuh"
#include "tc05.cuh"

namespace les {

namespace {
constexpr int TILE = 128;
constexpr uint32_t IDESC = tc::idesc_bf16_f32(128, 64);
// byte offsets of the packed operand images inside MlpDevice::img
constexpr int IMG_B1 = 0;           // 64 x 16  (N x K), K-major, 2 KB
constexpr int IMG_B2 = 2048;        // 64 x 64, 8 KB: B2[n][k] = W2[k][n]
constexpr int IMG_B2T = 2048 + 8192;  // 64 x 64, 8 KB: B2T[k][n] = W2[k][n]
constexpr int IMG_BYTES = 2048 + 8192 + 8192;

// byte offset of element (row, k) in a K-major no-swizzle tile whose 16-byte
// K chunks are 128 B apart and whose 8-row groups are sbo bytes apart
__host__ __device__ constexpr int kmaj_off(int row, int k, int sbo) {
  return (row >> 3) * sbo + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// GELU in its tanh form (Hendrycks & Gimpel, 2016):
//   gelu(x) = x / 2 * (1 + tanh(sqrt(2/pi) * (x + 0.044715 x^3)))
// with the hardware tanh approximation (one MUFU operation)
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float GELU_C0 = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float GELU_C1 = 0.044715f;
// x/2 (1 + t) = fma(x/2, t, x/2) with u = x (c0 + c0 c1 x^2): five FP32
// operations and one MUFU per evaluation (the epilogues are issue bound)
__device__ __forceinline__ float gelu(float x) {
  const float u = x * fmaf(GELU_C0 * GELU_C1, x * x, GELU_C0);
  const float t = tanh_fast(u);
  const float hx = 0.5f * x;
  return fmaf(hx, t, hx);
}
// the same on a pair of values with the packed FP32x2 instructions of sm_100
// (per component the rounding of the scalar form: results are bit-identical)
__device__ __forceinline__ float2 gelu2(float2 x) {
  const float2 x2 = __fmul2_rn(x, x);
  const float2 p = __ffma2_rn(make_float2(GELU_C0 * GELU_C1, GELU_C0 * GELU_C1), x2, make_float2(GELU_C0, GELU_C0));
  const float2 u = __fmul2_rn(x, p);
  const float2 t = make_float2(tanh_fast(u.x), tanh_fast(u.y));
  const float2 hx = __fmul2_rn(make_float2(0.5f, 0.5f), x);
  return __ffma2_rn(hx, t, hx);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float t = tanh_fast(GELU_C0 * fmaf(GELU_C1 * x, x * x, x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * GELU_C0 * fmaf(3.0f * GELU_C1, x * x, 1.0f);
}

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<uint16_t*>(&h);
}

// raw (transformed, not normalised) features at level k, offset o
template <typename T, bool RI = true>
__device__ __forceinline__ void raw_features(const MlpFeatIn<T>& a, long o, int k, float* t) {
  const long pl = a.plane;
  float ux, uy, uz, vx, vy, vz, wx, wy, wz;
  if (k == 1) {
    ux = float(a.d[0][o]);
    uy = float(a.d[1][o]);
    uz = a.wall ? float(a.d[2][o]) : 0.5f * float(a.d[2][o] + a.d[2][o + pl]);
    vx = float(a.d[3][o]);
    vy = float(a.d[4][o]);
    vz = a.wall ? float(a.d[5][o]) : 0.5f * float(a.d[5][o] + a.d[5][o + pl]);
    wx = 0.5f * float(a.d[6][o] + a.d[6][o + pl]);
    wy = 0.5f * float(a.d[7][o] + a.d[7][o + pl]);
    wz = float(a.d[8][o]);
  } else {
    ux = 0.5f * float(a.d[0][o] + a.d[0][o - pl]);
    uy = 0.5f * float(a.d[1][o] + a.d[1][o - pl]);
    uz = float(a.d[2][o]);
    vx = 0.5f * float(a.d[3][o] + a.d[3][o - pl]);
    vy = 0.5f * float(a.d[4][o] + a.d[4][o - pl]);
    vz = float(a.d[5][o]);
    wx = float(a.d[6][o]);
    wy = float(a.d[7][o]);
    wz = 0.5f * float(a.d[8][o] + a.d[8][o - pl]);
  }
  const float s11 = ux, s22 = vy, s33 = wz;
  const float s12 = 0.5f * (uy + vx), s13 = 0.5f * (uz + wx), s23 = 0.5f * (vz + wy);
  const float o12 = 0.5f * (uy - vx), o13 = 0.5f * (uz - wx), o23 = 0.5f * (vz - wy);
  const float ss = s11 * s11 + s22 * s22 + s33 * s33 + 2.0f * (s12 * s12 + s13 * s13 + s23 * s23);
  const float smag = sqrtf(2.0f * ss);
  const float oo = 2.0f * (o12 * o12 + o13 * o13 + o23 * o23);
  // tr(S^3) of the symmetric strain tensor
  const float r3 = s11 * s11 * s11 + s22 * s22 * s22 + s33 * s33 * s33 +
                   3.0f * (s12 * s12 * (s11 + s22) + s13 * s13 * (s11 + s33) + s23 * s23 * (s22 + s33)) +
                   6.0f * s12 * s13 * s23;
  const float z = (k == 1) ? 0.5f * a.dz : float(k - 1) * a.dz;
  t[0] = log1pf(smag);
  t[1] = log1pf(ss);
  t[2] = log1pf(oo);
  t[3] = copysignf(log1pf(fabsf(r3)), r3);
  t[4] = log1pf(z / a.delta);
  // the coefficient before this update: the Lagrangian averages of the
  // dynamic procedure relax from it (takes the slot of a gradient Richardson
  // number, which is zero without buoyancy)
  t[5] = logf(fmaxf(float(a.csprev[o]), 1e-6f));
  // vortex stretching w_i S_ij w_j (w = vorticity), Galilean invariant
  const float w1 = -2.0f * o23, w2 = 2.0f * o13, w3 = -2.0f * o12;
  const float vs = s11 * w1 * w1 + s22 * w2 * w2 + s33 * w3 * w3 +
                   2.0f * (s12 * w1 * w2 + s13 * w1 * w3 + s23 * w2 * w3);
  t[6] = copysignf(log1pf(fabsf(vs)), vs);
  if (RI && a.dtdz) {
    // gradient Richardson number g/theta_0 (d theta/dz) / |d u_h/dz|^2 at this
    // node (level 1: the wall value of d theta/dz), signed log1p
    const float ri = a.beta * float(a.dtdz[o]) / (uz * uz + vz * vz + 1e-12f);
    t[7] = copysignf(log1pf(fabsf(ri)), ri);
  } else {
    t[7] = a.log_delta_z0;
  }
}

// order-preserving float -> int map (for atomic min / max of floats)
__host__ __device__ inline int ordered_int(float f) {
  int i;
  memcpy(&i, &f, sizeof(int));
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__host__ __device__ inline float ordered_float(int i) {
  i = i >= 0 ? i : i ^ 0x7fffffff;
  float f;
  memcpy(&f, &i, sizeof(float));
  return f;
}

__device__ __forceinline__ unsigned hash32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

// --------------------------------------------------------- collection ----
// Two passes over the same grid (MLP_COLLECT_BLOCKS x 256 threads).  Pass 0
// takes the feature range of every point and counts each block's sampled
// slots (m.boff[2 b + v], v = 1 for validation); k_mlp_collect_scan turns
// the counts into each block's first slot after the pairs collected so far;
// pass 1 writes a block's pairs from there, each thread's in its own point
// order after the slots of the threads before it.  The slot of every pair
// depends on the state alone, not on the order in which the blocks run.
template <typename T>
__global__ void __launch_bounds__(256) k_mlp_collect(const MlpFeatIn<T> a, const T* cs, MlpDevice m, int stride,
                                                     int dense_levels, int wall_repeat, unsigned seed, int pass) {
  const long n = (long)(a.nz + 1) * a.plane;
  // whether point q (level k) is sampled, into which set, and how many slots
  // it takes: every point of the lowest levels, elsewhere one in `stride`
  // (seeded hash); 10 % held out; the training pairs of the two levels next
  // to the wall, where the SGS stress carries the momentum flux, repeated
  auto sample = [&](long q, int k, int& val) -> int {
    const unsigned h = hash32(unsigned(q) * 2654435761u ^ seed);
    const unsigned st = k <= dense_levels ? 1u : unsigned(stride);
    if (h % st != 0) return 0;
    val = ((h / st) % 10u) == 0u;
    return (k <= 2 && !val) ? wall_repeat : 1;
  };
  unsigned long long cnt[2] = {0, 0};
  if (pass == 0) {
    float lmin[8], lmax[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      lmin[i] = 3.0e38f;
      lmax[i] = -3.0e38f;
    }
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
      const long o = a.plane + q;
      const int k = udiv32(o, a.plane);
      float t[8];
      raw_features(a, o, k, t);  // every point: the range covers the whole state
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        lmin[i] = fminf(lmin[i], t[i]);
        lmax[i] = fmaxf(lmax[i], t[i]);
      }
      // the current coefficient is the next update's previous coefficient
      const float lcur = logf(fmaxf(float(cs[o]), 1e-6f));
      lmin[5] = fminf(lmin[5], lcur);
      lmax[5] = fmaxf(lmax[5], lcur);
      int val = 0;
      const int rep = sample(q, k, val);
      cnt[val] += rep;
    }
    // feature range of the state: warp reduction, one atomic per warp and
    // bound (min and max do not depend on the order)
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      float a0 = lmin[i], b0 = lmax[i];
      for (int off = 16; off > 0; off >>= 1) {
        a0 = fminf(a0, __shfl_down_sync(0xffffffffu, a0, off));
        b0 = fmaxf(b0, __shfl_down_sync(0xffffffffu, b0, off));
      }
      if ((threadIdx.x & 31) == 0) {
        atomicMin(&m.range[i], ordered_int(a0));
        atomicMax(&m.range[8 + i], ordered_int(b0));
      }
    }
    // the block's slot counts (integers: exact in any order)
    __shared__ unsigned long long wc[8][2];
    for (int v = 0; v < 2; ++v) {
      unsigned long long c = cnt[v];
      for (int off = 16; off > 0; off >>= 1) c += __shfl_down_sync(0xffffffffu, c, off);
      if ((threadIdx.x & 31) == 0) wc[threadIdx.x >> 5][v] = c;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      unsigned long long c = 0;
      for (int w = 0; w < int(blockDim.x >> 5); ++w) c += wc[w][threadIdx.x];
      m.boff[2 * blockIdx.x + threadIdx.x] = c;
    }
    return;
  }
  // pass 1: this thread's first slots are the block's plus the slots of the
  // threads before it
  __shared__ unsigned long long tcnt[256][2];
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    int val = 0;
    const int rep = sample(q, udiv32(a.plane + q, a.plane), val);
    cnt[val] += rep;
  }
  tcnt[threadIdx.x][0] = cnt[0];
  tcnt[threadIdx.x][1] = cnt[1];
  __syncthreads();
  unsigned long long idx[2] = {m.boff[2 * blockIdx.x], m.boff[2 * blockIdx.x + 1]};
  for (int t = 0; t < int(threadIdx.x); ++t) {
    idx[0] += tcnt[t][0];
    idx[1] += tcnt[t][1];
  }
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long o = a.plane + q;
    const int k = udiv32(o, a.plane);
    int val = 0;
    const int rep = sample(q, k, val);
    if (rep == 0) continue;
    float t[8];
    raw_features(a, o, k, t);
    // target: the change of log Cs^2 over the update (residual form: the
    // network's identity part is exact, it learns the relaxation)
    const float y = fmaxf(logf(fmaxf(float(cs[o]), 1e-30f)), MLP_LOG_CS_FLOOR) - t[5];
    for (int r = 0; r < rep; ++r) {
      if ((long)(idx[val] + r) >= m.cap) break;
      float* x = (val ? m.vx : m.dx) + (idx[val] + r) * MLP_IN;
#pragma unroll
      for (int i = 0; i < MLP_IN; ++i) x[i] = t[i];
      (val ? m.vt : m.dt)[idx[val] + r] = y;
    }
    idx[val] += rep;
  }
}

// one thread: the blocks' counts of pass 0 become their first slots, after
// the pairs already collected; m.counts gets the new totals
__global__ void k_mlp_collect_scan(MlpDevice m, int nblocks) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int v = 0; v < 2; ++v) {
    unsigned long long run = m.counts[v];
    for (int b = 0; b < nblocks; ++b) {
      const unsigned long long c = m.boff[2 * b + v];
      m.boff[2 * b + v] = run;
      run += c;
    }
    m.counts[v] = run;
  }
}

// statistics (double accumulators): sum, sum of squares, min, max of the 8
// raw features and the target, over train + validation
// part[18 b + i]: block b's sums (added on the host in block order, so the
// statistics do not depend on the order in which blocks finish)
__global__ void __launch_bounds__(128) k_mlp_stats(const float* x, const float* t, long n, double* acc,
                                                   double* part) {
  __shared__ double s[18][128];
  __shared__ float mn[9][128], mx[9][128];
  double loc[18] = {0};
  float lmin[9], lmax[9];
  for (int i = 0; i < 9; ++i) {
    lmin[i] = 3.0e38f;
    lmax[i] = -3.0e38f;
  }
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    for (int i = 0; i < 9; ++i) {
      const float v = (i < 8) ? x[q * 8 + i] : t[q];
      loc[2 * i] += v;
      loc[2 * i + 1] += double(v) * v;
      lmin[i] = fminf(lmin[i], v);
      lmax[i] = fmaxf(lmax[i], v);
    }
  }
  for (int i = 0; i < 18; ++i) s[i][threadIdx.x] = loc[i];
  for (int i = 0; i < 9; ++i) {
    mn[i][threadIdx.x] = lmin[i];
    mx[i][threadIdx.x] = lmax[i];
  }
  __syncthreads();
  if (threadIdx.x < 18) {
    double v = 0;
    for (int j = 0; j < 128; ++j) v += s[threadIdx.x][j];
    part[18 * blockIdx.x + threadIdx.x] = v;
  } else if (threadIdx.x >= 32 && threadIdx.x < 41) {
    const int i = threadIdx.x - 32;
    float a = 3.0e38f, b = -3.0e38f;
    for (int j = 0; j < 128; ++j) {
      a = fminf(a, mn[i][j]);
      b = fmaxf(b, mx[i][j]);
    }
    // order-preserving float -> int for atomic min/max
    int ia = __float_as_int(a), ib = __float_as_int(b);
    ia = ia >= 0 ? ia : ia ^ 0x7fffffff;
    ib = ib >= 0 ? ib : ib ^ 0x7fffffff;
    atomicMin(reinterpret_cast<int*>(&acc[18 + i]), ia);
    atomicMax(reinterpret_cast<int*>(&acc[27 + i]), ib);
  }
}

__global__ void k_mlp_normalize(float* x, float* t, long n, const float* stats) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    for (int i = 0; i < 8; ++i) x[q * 8 + i] = (x[q * 8 + i] - stats[MLP_S_MU + i]) / stats[MLP_S_SD + i];
    t[q] = (t[q] - stats[MLP_S_YMU]) / stats[MLP_S_YSD];
  }
}

// ---------------------------------------------------------- packing ----
__global__ void k_mlp_pack(const float* p, uint16_t* img) {
  unsigned char* base = reinterpret_cast<unsigned char*>(img);
  for (int i = threadIdx.x; i < 64 * 16; i += blockDim.x) {  // B1[n][k] = W1[k][n], k < 8
    const int n = i / 16, k = i % 16;
    const float v = (k < MLP_IN) ? p[MLP_O_W1 + k * MLP_H + n] : 0.0f;
    *reinterpret_cast<uint16_t*>(base + IMG_B1 + kmaj_off(n, k, 256)) = bf16_bits(v);
  }
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
    const int r = i / 64, c = i % 64;
    const float w = p[MLP_O_W2 + r * MLP_H + c];  // W2[k=r][n=c]
    *reinterpret_cast<uint16_t*>(base + IMG_B2 + kmaj_off(c, r, 1024)) = bf16_bits(w);   // B2[n][k]
    *reinterpret_cast<uint16_t*>(base + IMG_B2T + kmaj_off(r, c, 1024)) = bf16_bits(w);  // B2T[k][n]
  }
}

// -------------------------------------------------- shared tile layout ----
// TRAIN adds the operands of the backward GEMM (g2 . W2^T)
template <bool TRAIN>
struct __align__(1024) MlpSmemT {
  unsigned char A1[TILE * 16 * 2];                 // 4 KB  features (K-major, sbo 256)
  unsigned char A2[TILE * 64 * 2];                 // 16 KB h1 (K-major, sbo 1024)
  unsigned char B1[2048];
  unsigned char B2[8192];
  unsigned char G2[TRAIN ? TILE * 64 * 2 : 16];    // 16 KB g2 (K-major, sbo 1024)
  unsigned char B2T[TRAIN ? 8192 : 16];
  float b1[64], b2[64], w3[64];
  float stats[MLP_NS];
  float b3;
  uint64_t mbar;
  uint32_t tmem;
  int ok;
};
using InferSmem = MlpSmemT<false>;
using MlpSmem = MlpSmemT<true>;

template <bool TRAIN>
__device__ __forceinline__ void load_images(MlpSmemT<TRAIN>& S, const uint16_t* img, const float* p,
                                            const float* stats) {
  constexpr bool with_b2t = TRAIN;
  const uint4* src = reinterpret_cast<const uint4*>(img);
  uint4* d1 = reinterpret_cast<uint4*>(S.B1);
  for (int i = threadIdx.x; i < 2048 / 16; i += blockDim.x) d1[i] = src[i];
  uint4* d2 = reinterpret_cast<uint4*>(S.B2);
  for (int i = threadIdx.x; i < 8192 / 16; i += blockDim.x) d2[i] = src[2048 / 16 + i];
  if constexpr (with_b2t) {
    uint4* d3 = reinterpret_cast<uint4*>(S.B2T);
    for (int i = threadIdx.x; i < 8192 / 16; i += blockDim.x) d3[i] = src[(2048 + 8192) / 16 + i];
  }
  for (int i = threadIdx.x; i < 64; i += blockDim.x) {
    S.b1[i] = p[MLP_O_B1 + i];
    S.b2[i] = p[MLP_O_B2 + i];
    S.w3[i] = p[MLP_O_W3 + i];
  }
  for (int i = threadIdx.x; i < MLP_NS; i += blockDim.x) S.stats[i] = stats[i];
  if (threadIdx.x == 0) S.b3 = p[MLP_O_B3];
}

// two floats as a BF16 pair (round to nearest even), lo in the low half
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// write this thread's 8 normalised features as row `row` of A1
template <class S_t>
__device__ __forceinline__ void put_features(S_t& S, int row, const float* x) {
  uint4 c0, c1;
  c0.x = pack_bf16x2(x[0], x[1]);
  c0.y = pack_bf16x2(x[2], x[3]);
  c0.z = pack_bf16x2(x[4], x[5]);
  c0.w = pack_bf16x2(x[6], x[7]);
  c1 = make_uint4(0, 0, 0, 0);
  *reinterpret_cast<uint4*>(S.A1 + kmaj_off(row, 0, 256)) = c0;
  *reinterpret_cast<uint4*>(S.A1 + kmaj_off(row, 8, 256)) = c1;
}

// write 64 values as row `row` of a K-major (sbo 1024) BF16 tile
__device__ __forceinline__ void put_row64(unsigned char* tile, int row, const float* v) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    uint4 q;
    q.x = pack_bf16x2(v[8 * c + 0], v[8 * c + 1]);
    q.y = pack_bf16x2(v[8 * c + 2], v[8 * c + 3]);
    q.z = pack_bf16x2(v[8 * c + 4], v[8 * c + 5]);
    q.w = pack_bf16x2(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4*>(tile + kmaj_off(row, 8 * c, 1024)) = q;
  }
}
// write 16 values as columns 16 c .. 16 c + 15 of row `row` of a K-major (sbo 1024) BF16 tile
__device__ __forceinline__ void put16(unsigned char* tile, int row, int c, const float* v) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint4 q;
    q.x = pack_bf16x2(v[8 * h + 0], v[8 * h + 1]);
    q.y = pack_bf16x2(v[8 * h + 2], v[8 * h + 3]);
    q.z = pack_bf16x2(v[8 * h + 4], v[8 * h + 5]);
    q.w = pack_bf16x2(v[8 * h + 6], v[8 * h + 7]);
    *reinterpret_cast<uint4*>(tile + kmaj_off(row, 16 * c + 8 * h, 1024)) = q;
  }
}
__device__ __forceinline__ float tile_val(const unsigned char* tile, int row, int k, int sbo) {
  const uint16_t b = *reinterpret_cast<const uint16_t*>(tile + kmaj_off(row, k, sbo));
  return __uint_as_float(uint32_t(b) << 16);
}

// 64 TMEM columns of this thread's lane starting at column col
__device__ __forceinline__ void tmem_row64(uint32_t tbase, int col, float* v) {
  const uint32_t lane = uint32_t((threadIdx.x / 32) * 32) << 16;
#pragma unroll
  for (int j = 0; j < 4; ++j) tc::tmem_ld16(tbase + lane + uint32_t(col + 16 * j), v + 16 * j);
  tc::tmem_wait_ld();
}

// issue one tensor-core stage (thread 0) and wait for it (bounded);
// returns false (and flags the status) when the wait ran out
// stage 0: D = X . W1, 1: D = H1 . W2, 2: D = G2 . W2^T, D at TMEM column dcol
template <bool TRAIN>
__device__ __forceinline__ bool tc_stage(MlpSmemT<TRAIN>& S, uint32_t& phase, unsigned* status, int which,
                                         uint32_t dcol) {
  if (threadIdx.x == 0) {
    tc::fence_after_sync();
    const uint32_t a1 = tc::smem_u32(S.A1), a2 = tc::smem_u32(S.A2);
    const uint32_t b1 = tc::smem_u32(S.B1), b2 = tc::smem_u32(S.B2);
    if (which == 0) {
      tc::mma_bf16(S.tmem + dcol, tc::smem_desc(a1, 128, 256), tc::smem_desc(b1, 128, 256), IDESC, 0);
    } else if (which == 1) {
#pragma unroll
      for (int s = 0; s < 4; ++s)
        tc::mma_bf16(S.tmem + dcol, tc::smem_desc(a2 + 256 * s, 128, 1024), tc::smem_desc(b2 + 256 * s, 128, 1024),
                     IDESC, s > 0);
    } else if constexpr (TRAIN) {
      const uint32_t g2 = tc::smem_u32(S.G2), b2t = tc::smem_u32(S.B2T);
#pragma unroll
      for (int s = 0; s < 4; ++s)
        tc::mma_bf16(S.tmem + dcol, tc::smem_desc(g2 + 256 * s, 128, 1024), tc::smem_desc(b2t + 256 * s, 128, 1024),
                     IDESC, s > 0);
    }
    tc::mma_commit(&S.mbar);
    S.ok = tc::mbar_wait(&S.mbar, phase) ? 1 : 0;
    if (!S.ok) atomicOr(status, 16u);
  }
  phase ^= 1u;
  __syncthreads();
  tc::fence_after_sync();
  return S.ok != 0;
}

template <class S_t>
__device__ __forceinline__ void tc_setup(S_t& S, uint32_t ncols) {
  if (threadIdx.x < 32) {
    tc::tmem_alloc(&S.tmem, ncols);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    tc::mbar_init(&S.mbar, 1);
    tc::fence_mbar_init();
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}
template <class S_t>
__device__ __forceinline__ void tc_teardown(S_t& S, uint32_t ncols, uint32_t phase) {
  // after a timed-out stage, wait (bounded) for the MMA still in flight
  if (threadIdx.x == 0 && !S.ok) tc::mbar_wait(&S.mbar, phase ^ 1u);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (threadIdx.x < 32) tc::tmem_dealloc(S.tmem, ncols);
}

// ------------------------------------------------------------ inference ----
// RI: buoyant runs (feature 7 = the gradient Richardson number); the
// neutral variant is compiled without it (fewer registers, one more CTA per SM)
template <typename T, bool RI>
__global__ void __launch_bounds__(TILE, 6) k_mlp_infer(const MlpFeatIn<T> a, T* cs, MlpDevice m, unsigned* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  InferSmem& S = *reinterpret_cast<InferSmem*>(smem_raw + ((1024 - (tc::smem_u32(smem_raw) & 1023)) & 1023));
  load_images(S, m.img, m.params, m.stats);
  if (threadIdx.x == 0) S.ok = 1;
  tc_setup(S, 64);  // both layers accumulate in TMEM columns 0..63
  uint32_t phase = 0;
  const long npts = (long)(a.nz + 1) * a.plane;
  const long ntiles = (npts + TILE - 1) / TILE;
  __syncthreads();  // the statistics are in shared memory
  float inv_sd[8];  // normalisation by multiplication (the features are rounded to BF16 next)
#pragma unroll
  for (int i = 0; i < 8; ++i) inv_sd[i] = 1.0f / S.stats[MLP_S_SD + i];
  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long q = tile * TILE + threadIdx.x;
    const bool valid = q < npts;
    float x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float lprev = 0.0f;  // log Cs^2 before the update (floored)
    long o = 0;
    if (valid) {
      o = a.plane + q;
      const int k = udiv32(o, a.plane);
      float t[8];
      raw_features<T, RI>(a, o, k, t);
      int out = 0;  // bit i: feature i outside the training range (margin: 0.25 sd + 5 % of the range)
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        x[i] = (t[i] - S.stats[MLP_S_MU + i]) * inv_sd[i];
        const float mn = S.stats[MLP_S_MIN + i], mx = S.stats[MLP_S_MAX + i];
        const float margin = 0.25f + 0.05f * (mx - mn);
        if ((x[i] < mn - margin) || (x[i] > mx + margin)) out |= 1 << i;
      }
      if (out && k > a.wall_levels) atomicOr(&m.colflag[umod32(q, a.plane)], out);
      lprev = t[5];
    }
    put_features(S, threadIdx.x, x);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (!tc_stage(S, phase, status, 0, 0)) break;
    // bias and GELU two values at a time (packed FP32x2; the epilogues are
    // issue bound), 16 TMEM columns at a time (fewer live registers)
    const uint32_t tlane = uint32_t((threadIdx.x / 32) * 32) << 16;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float h[16];
      tc::tmem_ld16(S.tmem + tlane + uint32_t(16 * c), h);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; i += 2) {
        const float2 z = gelu2(
            __fadd2_rn(make_float2(h[i], h[i + 1]), make_float2(S.b1[16 * c + i], S.b1[16 * c + i + 1])));
        h[i] = z.x;
        h[i + 1] = z.y;
      }
      put16(S.A2, threadIdx.x, c, h);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (!tc_stage(S, phase, status, 1, 0)) break;
    // output layer: even and odd hidden units summed in the two lanes of a
    // packed accumulator, then added
    float2 y2 = make_float2(S.b3, 0.0f);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float h[16];
      tc::tmem_ld16(S.tmem + tlane + uint32_t(16 * c), h);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; i += 2) {
        const int k = 16 * c + i;
        const float2 g = gelu2(__fadd2_rn(make_float2(h[i], h[i + 1]), make_float2(S.b2[k], S.b2[k + 1])));
        y2 = __ffma2_rn(make_float2(S.w3[k], S.w3[k + 1]), g, y2);
      }
    }
    float y = y2.x + y2.y;
    if (valid) {
      // no extrapolation: the change is clamped to the trained range, the
      // coefficient to the range of the previous coefficients seen in training
      y = fminf(fmaxf(y, S.stats[MLP_S_YMIN]), S.stats[MLP_S_YMAX]);
      float lc = lprev + S.stats[MLP_S_YMU] + S.stats[MLP_S_YSD] * y;
      lc = fminf(fmaxf(lc, S.stats[MLP_S_MU + 5] + S.stats[MLP_S_SD + 5] * S.stats[MLP_S_MIN + 5]),
                 S.stats[MLP_S_MU + 5] + S.stats[MLP_S_SD + 5] * S.stats[MLP_S_MAX + 5]);
      cs[o] = T(fminf(fmaxf(expf(lc), 1e-24f), a.cs_max));
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  tc_teardown(S, 64, phase);
}

// ------------------------------------------------------------- training ----
// One launch: each CTA loops over tiles of samples [tile*128, +128) < n,
// forward + backward.  Gradient of L = mean_i (y_i - t_i)^2 with inv_n = 1/n.
//
// The weight gradients are one more tensor-core GEMM per tile, accumulated
// in TMEM over all of a CTA's tiles and added to m.grad once per CTA:
// D[128 x 192] += AW[128 x 128] . BW[192 x 128]^T (K = the 128 samples),
// with AW rows 0..63 = h1^T, 64..71 = x^T, 72 = ones, 73 = dy, rest zero and
// BW rows 0..63 = g2^T, 64..127 = delta1^T, 128..191 = h2^T, so that
// D[k][n] = dW2, D[64 + f][64 + k] = dW1, D[72][n] = db2, D[72][64 + k] =
// db1, D[73][128 + i] = dw3 (db3 = sum dy on the CUDA cores).  Operands are
// BF16 (the oracle rounds the same values), accumulation FP32.  The
// transposed tiles are built from the K-major sample-row tiles by 8 x 8
// transposes of core matrices (16-byte loads and stores, byte permutes).
constexpr int AW_ROWS = 128, BW_ROWS = 192, W_SBO = 2048;  // K = 128 samples: 16 chunks of 128 B per row group
constexpr uint32_t IDESC_W = tc::idesc_bf16_f32(128, 192);
constexpr uint32_t TM_Z1 = 0, TM_Z2 = 64, TM_D1 = 128, TM_W = 256;  // TMEM columns

struct TrainSmem {
  MlpSmem s;
  alignas(1024) unsigned char AW[AW_ROWS / 8 * W_SBO];   // 32 KB
  alignas(1024) unsigned char BW[BW_ROWS / 8 * W_SBO];   // 48 KB
  alignas(1024) unsigned char T64[TILE * 64 * 2];        // 16 KB sample-row staging (h2, delta1)
  float dsum[TILE / 32];
  uint64_t wbar;
};

// 8 x 8 transpose of 16-bit elements: in[r] = row r (8 values in a uint4),
// out[c] = column c
__device__ __forceinline__ void transpose8x8(const uint4* in, uint4* out) {
  uint32_t w[8][4];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    w[r][0] = in[r].x;
    w[r][1] = in[r].y;
    w[r][2] = in[r].z;
    w[r][3] = in[r].w;
  }
  uint32_t o[8][4];  // o[c][p]: column c, rows 2p and 2p + 1
#pragma unroll
  for (int c = 0; c < 8; ++c)
#pragma unroll
    for (int p = 0; p < 4; ++p)
      o[c][p] = __byte_perm(w[2 * p][c >> 1], w[2 * p + 1][c >> 1], (c & 1) ? 0x7632 : 0x5410);
#pragma unroll
  for (int c = 0; c < 8; ++c) out[c] = make_uint4(o[c][0], o[c][1], o[c][2], o[c][3]);
}

// core matrix (sample group sg, feature chunk fc) of a sample-row K-major tile
// (sbo_src) -> core matrix (feature group row0 / 8 + fc, sample chunk sg) of a
// transposed tile (sbo W_SBO)
__device__ __forceinline__ void transpose_block(const unsigned char* src, int sbo_src, unsigned char* dst, int row0,
                                                int sg, int fc) {
  uint4 in[8], out[8];
  const unsigned char* sp = src + sg * sbo_src + fc * 128;
#pragma unroll
  for (int r = 0; r < 8; ++r) in[r] = *reinterpret_cast<const uint4*>(sp + 16 * r);
  transpose8x8(in, out);
  unsigned char* dp = dst + (row0 / 8 + fc) * W_SBO + sg * 128;
#pragma unroll
  for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(dp + 16 * c) = out[c];
}

// the weight-gradient GEMM of one tile into TMEM columns TM_W.. (thread 0);
// waits (bounded) so the next tile may overwrite AW / BW
__device__ __forceinline__ bool tc_weights(TrainSmem& TS, uint32_t& wphase, unsigned* status, bool first) {
  MlpSmem& S = TS.s;
  if (threadIdx.x == 0) {
    tc::fence_after_sync();
    const uint32_t aw = tc::smem_u32(TS.AW), bw = tc::smem_u32(TS.BW);
#pragma unroll
    for (int ks = 0; ks < 8; ++ks)
      tc::mma_bf16(S.tmem + TM_W, tc::smem_desc(aw + 256 * ks, 128, W_SBO), tc::smem_desc(bw + 256 * ks, 128, W_SBO),
                   IDESC_W, (!first || ks > 0) ? 1u : 0u);
    tc::mma_commit(&TS.wbar);
    S.ok = tc::mbar_wait(&TS.wbar, wphase) ? 1 : 0;
    if (!S.ok) atomicOr(status, 16u);
  }
  wphase ^= 1u;
  __syncthreads();
  tc::fence_after_sync();
  return S.ok != 0;
}

__global__ void __launch_bounds__(TILE) k_mlp_train(MlpDevice m, const float* X, const float* Tg, long n,
                                                    float inv_n, float* y_out, float* loss, unsigned* status,
                                                    MlpPerm pm) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  TrainSmem& TS = *reinterpret_cast<TrainSmem*>(smem_raw + ((1024 - (tc::smem_u32(smem_raw) & 1023)) & 1023));
  MlpSmem& S = TS.s;
  load_images(S, m.img, m.params, m.stats);
  if (threadIdx.x == 0) {
    S.ok = 1;
    tc::mbar_init(&TS.wbar, 1);
  }
  const int tid = threadIdx.x;
  // AW rows 72..127: row 72 ones, the rest zero (row 73 is rewritten per tile)
  for (int i = tid; i < (AW_ROWS - 72) * TILE; i += TILE) {
    const int r = 72 + i / TILE, c = i % TILE;
    *reinterpret_cast<uint16_t*>(TS.AW + kmaj_off(r, c, W_SBO)) = bf16_bits(r == 72 ? 1.0f : 0.0f);
  }
  tc_setup(S, 512);  // z1, z2, delta1 (64 columns each) and the 192 weight-gradient columns
  float ab3 = 0.0f, aloss = 0.0f;
  uint32_t phase = 0, wphase = 0;
  bool first = true, wfail = false;
  const long ntiles = (n + TILE - 1) / TILE;
  const int sg = tid >> 3, fc = tid & 7;  // this thread's core matrix of the 64-wide tiles
  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long q = tile * TILE + tid;
    const bool valid = q < n;
    const long src = pm.n ? long((pm.a * (unsigned long long)(pm.off + q) + pm.b) % (unsigned long long)pm.n) : q;
    float x[8];
    for (int i = 0; i < 8; ++i) x[i] = valid ? X[src * 8 + i] : 0.0f;
    const float tg = valid ? Tg[src] : 0.0f;
    put_features(S, tid, x);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid < 16) transpose_block(S.A1, 256, TS.AW, 64, tid, 0);  // x^T -> AW rows 64..71
    if (!tc_stage(S, phase, status, 0, TM_Z1)) break;
    // the layer outputs stay in TMEM (z1 at TM_Z1, z2 at TM_Z2) and are read
    // back 16 columns at a time where they are needed, so that no 64-value
    // row is live across a stage
    const uint32_t lane = uint32_t((tid / 32) * 32) << 16;
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {  // h1 = gelu(z1 + b1)
      float v[16];
      tc::tmem_ld16(S.tmem + lane + TM_Z1 + 16 * c, v);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = gelu(v[i] + S.b1[16 * c + i]);
      put16(S.A2, tid, c, v);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    transpose_block(S.A2, 1024, TS.AW, 0, sg, fc);  // h1^T -> AW rows 0..63 (the BF16 values layer 2 uses)
    if (!tc_stage(S, phase, status, 1, TM_Z2)) break;
    float y = S.b3;
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tc::tmem_ld16(S.tmem + lane + TM_Z2 + 16 * c, v);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) y += S.w3[16 * c + i] * gelu(v[i] + S.b2[16 * c + i]);
    }
    if (y_out && valid) y_out[q] = y;
    const float dy = valid ? 2.0f * (y - tg) * inv_n : 0.0f;
    if (valid) aloss += (y - tg) * (y - tg) * inv_n;
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {  // h2 and g2 = dy w3 gelu'(z2)
      float v[16], h2[16], g2[16];
      tc::tmem_ld16(S.tmem + lane + TM_Z2 + 16 * c, v);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float z2 = v[i] + S.b2[16 * c + i];
        h2[i] = gelu(z2);
        g2[i] = dy * S.w3[16 * c + i] * gelu_grad(z2);
      }
      put16(S.G2, tid, c, g2);
      put16(TS.T64, tid, c, h2);
    }
    *reinterpret_cast<uint16_t*>(TS.AW + kmaj_off(73, tid, W_SBO)) = bf16_bits(dy);
    {  // db3: sum of dy over the tile
      float d = dy;
      for (int off = 16; off > 0; off >>= 1) d += __shfl_down_sync(0xffffffffu, d, off);
      if ((tid & 31) == 0) TS.dsum[tid >> 5] = d;
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) ab3 += (TS.dsum[0] + TS.dsum[1]) + (TS.dsum[2] + TS.dsum[3]);
    transpose_block(S.G2, 1024, TS.BW, 0, sg, fc);     // g2^T -> BW rows 0..63
    transpose_block(TS.T64, 1024, TS.BW, 128, sg, fc); // h2^T -> BW rows 128..191
    if (!tc_stage(S, phase, status, 2, TM_D1)) break;
    // delta1 = (g2 . W2^T) * gelu'(z1); h2's transpose finished before the
    // stage's barrier, so T64 is free
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      float d1[16], z1[16];
      tc::tmem_ld16(S.tmem + lane + TM_D1 + 16 * c, d1);
      tc::tmem_ld16(S.tmem + lane + TM_Z1 + 16 * c, z1);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) d1[i] *= gelu_grad(z1[i] + S.b1[16 * c + i]);
      put16(TS.T64, tid, c, d1);
    }
    __syncthreads();
    transpose_block(TS.T64, 1024, TS.BW, 64, sg, fc);  // delta1^T -> BW rows 64..127
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (!tc_weights(TS, wphase, status, first)) {
      wfail = true;
      break;
    }
    first = false;
  }
  // the weight gradients: thread r reads TMEM lane r (D row r); every warp
  // runs the same loads (tcgen05.ld is warp-collective)
  // This CTA's gradient goes to its own row of m.gpart (every entry written
  // by one thread; zeros when the CTA had no tile), summed over the CTAs in
  // a fixed order by k_mlp_grad_reduce.
  float* gp = m.gpart + (size_t)blockIdx.x * MLP_NP;
  const bool have = !first && S.ok;
  {
    float v[64];
    if (have) tmem_row64(S.tmem, TM_W, v);
    if (tid < 64)
      for (int i = 0; i < 64; ++i) gp[MLP_O_W2 + tid * MLP_H + i] = have ? v[i] : 0.0f;  // dW2[tid][.]
    else if (tid == 72)
      for (int i = 0; i < 64; ++i) gp[MLP_O_B2 + i] = have ? v[i] : 0.0f;
    if (have) tmem_row64(S.tmem, TM_W + 64, v);
    if (tid >= 64 && tid < 72)
      for (int i = 0; i < 64; ++i) gp[MLP_O_W1 + (tid - 64) * MLP_H + i] = have ? v[i] : 0.0f;  // dW1
    else if (tid == 72)
      for (int i = 0; i < 64; ++i) gp[MLP_O_B1 + i] = have ? v[i] : 0.0f;
    if (have) tmem_row64(S.tmem, TM_W + 128, v);
    if (tid == 73)
      for (int i = 0; i < 64; ++i) gp[MLP_O_W3 + i] = have ? v[i] : 0.0f;
  }
  // a weight GEMM whose wait ran out may still be in flight: wait (bounded)
  // for it before the TMEM is freed
  if (tid == 0 && !S.ok && wfail) tc::mbar_wait(&TS.wbar, wphase ^ 1u);
  tc_teardown(S, 512, phase);
  if (tid == 0) gp[MLP_O_B3] = ab3;
  for (int off = 16; off > 0; off >>= 1) aloss += __shfl_down_sync(0xffffffffu, aloss, off);
  __syncthreads();  // the last tile's reads of dsum (ab3) are done: reuse it for the warps' losses
  if ((tid & 31) == 0) TS.dsum[tid >> 5] = aloss;
  __syncthreads();
  if (tid == 0) {
    float l = 0.0f;
    for (int w = 0; w < TILE / 32; ++w) l += TS.dsum[w];
    m.lpart[blockIdx.x] = l;
  }
}

// m.grad = the sum of the CTAs' gradient rows, CTA by CTA in index order;
// *loss (when given) the same sum of their losses
__global__ void k_mlp_grad_reduce(MlpDevice m, int nctas, float* loss) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NP; i += gridDim.x * blockDim.x) {
    float g = 0.0f;
    for (int b = 0; b < nctas; ++b) g += m.gpart[(size_t)b * MLP_NP + i];
    m.grad[i] = g;
  }
  if (loss && blockIdx.x == 0 && threadIdx.x == 0) {
    float l = 0.0f;
    for (int b = 0; b < nctas; ++b) l += m.lpart[b];
    *loss = l;
  }
}

__global__ void k_mlp_adam(float* p, const float* g, float* mm, float* vv, int step, float lr) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.0f - powf(b1, float(step)), c2 = 1.0f - powf(b2, float(step));
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NP; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    mm[i] = b1 * mm[i] + (1.0f - b1) * gi;
    vv[i] = b2 * vv[i] + (1.0f - b2) * gi * gi;
    p[i] -= lr * (mm[i] / c1) / (sqrtf(vv[i] / c2) + eps);
  }
}

// out[0]: flagged columns; out[1 + i]: columns where feature i left the range
__global__ void k_mlp_count_flags(const int* flag, long plane, int* out) {
  int c[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < plane; q += (long)gridDim.x * blockDim.x) {
    const int f = flag[q];
    c[0] += f != 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) c[1 + i] += (f >> i) & 1;
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    int v = c[i];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&out[i], v);
  }
}

// blockIdx.y = level - 1; err2[k] accumulates the squared log differences of level k
template <typename T>
__global__ void k_mlp_blend(T* cs, const T* cs_dyn, const int* flag, long plane, double* err2, int check) {
  const int k = 1 + blockIdx.y;
  double e = 0.0;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < plane; p += (long)gridDim.x * blockDim.x) {
    const long o = (long)k * plane + p;
    if (check) {
      const double d = log(fmax(double(cs[o]), 1e-6)) - log(fmax(double(cs_dyn[o]), 1e-6));
      e += d * d;
    }
    if (flag[p]) cs[o] = cs_dyn[o];
  }
  if (check) {  // the block's sum, warps in order: err2[k * gridDim.x + blockIdx.x]
    __shared__ double we[8];
    for (int off = 16; off > 0; off >>= 1) e += __shfl_down_sync(0xffffffffu, e, off);
    if ((threadIdx.x & 31) == 0) we[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = 0.0;
      for (int w = 0; w < int(blockDim.x >> 5); ++w) b += we[w];
      err2[(long)k * gridDim.x + blockIdx.x] = b;
    }
  }
}

size_t infer_smem() { return sizeof(InferSmem) + 1024; }
size_t train_smem() { return sizeof(TrainSmem) + 1024; }

}  // namespace

// ------------------------------------------------------------- host side ----
template <typename T>
void mlp_collect(const MlpFeatIn<T>& in, const T* cs, MlpDevice& m, int stride, int dense_levels, int wall_repeat,
                 unsigned seed, cudaStream_t st) {
  const long n = (long)(in.nz + 1) * in.plane;
  hook_before("k_mlp_collect", double(n) * 11 * sizeof(T));
  k_mlp_collect<T><<<MLP_COLLECT_BLOCKS, 256, 0, st>>>(in, cs, m, stride, dense_levels, wall_repeat, seed, 0);
  LES_CHECK_LAUNCH();
  hook_after();
  hook_before("k_mlp_collect_scan", 32.0 * MLP_COLLECT_BLOCKS);
  k_mlp_collect_scan<<<1, 32, 0, st>>>(m, MLP_COLLECT_BLOCKS);
  LES_CHECK_LAUNCH();
  hook_after();
  hook_before("k_mlp_collect", double(n) * 11 * sizeof(T));
  k_mlp_collect<T><<<MLP_COLLECT_BLOCKS, 256, 0, st>>>(in, cs, m, stride, dense_levels, wall_repeat, seed, 1);
  LES_CHECK_LAUNCH();
  hook_after();
}

template <typename T>
void mlp_infer(const MlpFeatIn<T>& in, T* cs, MlpDevice& m, unsigned* status, cudaStream_t st) {
  LES_CUDA(cudaMemsetAsync(m.colflag, 0, sizeof(int) * m.plane, st));
  const long n = (long)(in.nz + 1) * in.plane;
  const long ntiles = (n + TILE - 1) / TILE;
  const int grid = int(std::min<long>(ntiles, 148L * 6));  // 6 CTAs per SM fit (79 registers, 32 KB, 64 TMEM columns each)
  hook_before("k_mlp_infer", double(n) * 11 * sizeof(T));
  if (in.dtdz) k_mlp_infer<T, true><<<grid, TILE, infer_smem(), st>>>(in, cs, m, status);
  else k_mlp_infer<T, false><<<grid, TILE, infer_smem(), st>>>(in, cs, m, status);
  LES_CHECK_LAUNCH();
  hook_after();
}

void init_mlp_attributes() {
  LES_CUDA(cudaFuncSetAttribute(k_mlp_infer<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)infer_smem()));
  LES_CUDA(cudaFuncSetAttribute(k_mlp_infer<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)infer_smem()));
  LES_CUDA(cudaFuncSetAttribute(k_mlp_infer<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)infer_smem()));
  LES_CUDA(cudaFuncSetAttribute(k_mlp_infer<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)infer_smem()));
  LES_CUDA(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem()));
}

void mlp_reset_range(MlpDevice& m, cudaStream_t st) {
  int rg[16];
  for (int i = 0; i < 8; ++i) {
    rg[i] = ordered_int(3.0e38f);
    rg[8 + i] = ordered_int(-3.0e38f);
  }
  LES_CUDA(cudaMemcpyAsync(m.range, rg, sizeof(rg), cudaMemcpyHostToDevice, st));
  LES_CUDA(cudaStreamSynchronize(st));
}

void mlp_pack(MlpDevice& m, cudaStream_t st) {
  hook_before("k_mlp_pack", double(MLP_NP) * 4 + IMG_BYTES);
  k_mlp_pack<<<1, 256, 0, st>>>(m.params, m.img);
  LES_CHECK_LAUNCH();
  hook_after();
}

void mlp_grad(MlpDevice& m, const float* x, const float* t, long n, float* y_out, float* loss_dev, unsigned* status,
              cudaStream_t st, MlpPerm perm) {
  const long ntiles = (n + TILE - 1) / TILE;
  const int grid = int(std::max<long>(1, std::min<long>(ntiles, (long)MLP_TRAIN_CTAS)));
  hook_before("k_mlp_train", double(n) * 36.0);
  k_mlp_train<<<grid, TILE, train_smem(), st>>>(m, x, t, n, 1.0f / float(n), y_out, loss_dev, status, perm);
  LES_CHECK_LAUNCH();
  hook_after();
  hook_before("k_mlp_grad_reduce", double(grid + 1) * MLP_NP * 4.0);
  k_mlp_grad_reduce<<<19, 256, 0, st>>>(m, grid, loss_dev);
  LES_CHECK_LAUNCH();
  hook_after();
}

void mlp_adam(MlpDevice& m, int step, float lr, cudaStream_t st) {
  hook_before("k_mlp_adam", double(MLP_NP) * 20);
  k_mlp_adam<<<19, 256, 0, st>>>(m.params, m.grad, m.adam_m, m.adam_v, step, lr);
  LES_CHECK_LAUNCH();
  hook_after();
  mlp_pack(m, st);
}

void mlp_fit_stats(MlpDevice& m, cudaStream_t st) {
  unsigned long long cnt[2];
  LES_CUDA(cudaMemcpyAsync(cnt, m.counts, sizeof(cnt), cudaMemcpyDeviceToHost, st));
  LES_CUDA(cudaStreamSynchronize(st));
  const long nt = std::min<long>((long)cnt[0], m.cap), nv = std::min<long>((long)cnt[1], m.cap);
  if (nt < 2) throw CudaError(1, "learned closure: no training data collected");
  constexpr int SB = 148;  // blocks of k_mlp_stats
  double* acc = nullptr;
  LES_CUDA(cudaMalloc(&acc, (36 + 18 * SB) * sizeof(double)));
  std::vector<double> init(36, 0.0);
  // min slots start at +max, max slots at -max (order-preserving ints)
  for (int i = 0; i < 9; ++i) {
    int big = 0x7f7fffff, neg = int(0xff7fffffu) ^ 0x7fffffff;
    std::memcpy(&init[18 + i], &big, sizeof(int));
    std::memcpy(&init[27 + i], &neg, sizeof(int));
  }
  LES_CUDA(cudaMemcpyAsync(acc, init.data(), 36 * sizeof(double), cudaMemcpyHostToDevice, st));
  k_mlp_stats<<<SB, 128, 0, st>>>(m.dx, m.dt, nt, acc, acc + 36);
  LES_CHECK_LAUNCH();
  std::vector<double> h(36 + 18 * SB);
  LES_CUDA(cudaMemcpyAsync(h.data(), acc, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  LES_CUDA(cudaStreamSynchronize(st));
  cudaFree(acc);
  for (int i = 0; i < 18; ++i) {
    h[i] = 0.0;
    for (int b = 0; b < SB; ++b) h[i] += h[36 + 18 * b + i];
  }
  // feature range: the sampled pairs and every point of the collected states
  int rg[16];
  LES_CUDA(cudaMemcpyAsync(rg, m.range, sizeof(rg), cudaMemcpyDeviceToHost, st));
  LES_CUDA(cudaStreamSynchronize(st));
  float s[MLP_NS];
  auto unorder = [](double slot) {
    int iv;
    std::memcpy(&iv, &slot, sizeof(int));
    return ordered_float(iv);
  };
  for (int i = 0; i < 9; ++i) {
    const double mean = h[2 * i] / double(nt);
    double var = h[2 * i + 1] / double(nt) - mean * mean;
    double sd = var > 1e-12 ? std::sqrt(var) : 1.0;
    float mn = unorder(h[18 + i]), mx = unorder(h[27 + i]);
    if (i < 8) {
      mn = std::min(mn, ordered_float(rg[i]));
      mx = std::max(mx, ordered_float(rg[8 + i]));
    }
    if (i < 8) {
      s[MLP_S_MU + i] = float(mean);
      s[MLP_S_SD + i] = float(sd);
      s[MLP_S_MIN + i] = float((mn - mean) / sd);
      s[MLP_S_MAX + i] = float((mx - mean) / sd);
    } else {
      s[MLP_S_YMU] = float(mean);
      s[MLP_S_YSD] = float(sd);
      s[MLP_S_YMIN] = float((mn - mean) / sd);
      s[MLP_S_YMAX] = float((mx - mean) / sd);
    }
  }
  LES_CUDA(cudaMemcpyAsync(m.stats, s, sizeof(s), cudaMemcpyHostToDevice, st));
  k_mlp_normalize<<<148 * 4, 256, 0, st>>>(m.dx, m.dt, nt, m.stats);
  LES_CHECK_LAUNCH();
  if (nv > 0) {
    k_mlp_normalize<<<148 * 4, 256, 0, st>>>(m.vx, m.vt, nv, m.stats);
    LES_CHECK_LAUNCH();
  }
  LES_CUDA(cudaStreamSynchronize(st));
}

int mlp_count_flags(MlpDevice& m, int* dcount, int* per_feature, cudaStream_t st) {
  LES_CUDA(cudaMemsetAsync(dcount, 0, 9 * sizeof(int), st));
  hook_before("k_mlp_count_flags", double(m.plane) * 4);
  k_mlp_count_flags<<<148, 256, 0, st>>>(m.colflag, m.plane, dcount);
  LES_CHECK_LAUNCH();
  hook_after();
  int h[9];
  LES_CUDA(cudaMemcpyAsync(h, dcount, sizeof(h), cudaMemcpyDeviceToHost, st));
  LES_CUDA(cudaStreamSynchronize(st));
  if (per_feature)
    for (int i = 0; i < 8; ++i) per_feature[i] = h[1 + i];
  return h[0];
}

template <typename T>
void mlp_blend(T* cs, const T* cs_dyn, MlpDevice& m, int nz, bool check, double* derr, double* profile,
               cudaStream_t st) {
  constexpr int NB = MLP_BLEND_BLOCKS;
  LES_CUDA(cudaMemsetAsync(derr, 0, sizeof(double) * NB * (nz + 2), st));
  const long n = (long)(nz + 1) * m.plane;
  hook_before("k_mlp_blend", double(n) * 3 * sizeof(T));
  k_mlp_blend<T><<<dim3(NB, nz + 1), 256, 0, st>>>(cs, cs_dyn, m.colflag, m.plane, derr, check ? 1 : 0);
  LES_CHECK_LAUNCH();
  hook_after();
  if (check) {
    std::vector<double> h((size_t)NB * (nz + 2));
    LES_CUDA(cudaMemcpyAsync(h.data(), derr, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k <= nz + 1; ++k) {
      double e = 0.0;
      for (int b = 0; b < NB; ++b) e += h[(size_t)k * NB + b];  // blocks in order
      profile[k] = std::sqrt(e / double(m.plane));
    }
  }
}
template void mlp_blend<float>(float*, const float*, MlpDevice&, int, bool, double*, double*, cudaStream_t);
template void mlp_blend<double>(double*, const double*, MlpDevice&, int, bool, double*, double*, cudaStream_t);

template void mlp_collect<float>(const MlpFeatIn<float>&, const float*, MlpDevice&, int, int, int, unsigned,
                                 cudaStream_t);
template void mlp_collect<double>(const MlpFeatIn<double>&, const double*, MlpDevice&, int, int, int, unsigned,
                                  cudaStream_t);
template void mlp_infer<float>(const MlpFeatIn<float>&, float*, MlpDevice&, unsigned*, cudaStream_t);
template void mlp_infer<double>(const MlpFeatIn<double>&, double*, MlpDevice&, unsigned*, cudaStream_t);

}  // namespace les
