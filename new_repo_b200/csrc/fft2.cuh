// Register-resident Stockham FFTs of compile-time length N = 2^a 3^b.
//
// A sequence is transformed by T = N / E lanes of one warp, each holding E
// elements in registers.  Each pass applies radix-R DFTs (R | E, R up to 32,
// evaluated in registers with compile-time twiddles) and exchanges data with
// the other T - 1 lanes through the sequence's own shared-memory slot, so a
// length-256 transform is two passes and one exchange.  Lanes of a sequence
// sit in one warp: exchanges need only __syncwarp.
//
// Layout contract (Stockham autosort): on entry lane t holds
//   v[g*R1 + r] = x[t + T*g + r*(N/R1)]      (g < E/R1, r < R1, R1 = first radix)
// and on exit
//   v[g*RL + r] = X[t + T*g + r*(N/RL)]      (RL = last radix),
// so an inverse transform whose first radix is the forward's last radix
// consumes the forward's output registers directly.
#pragma once
#include <type_traits>
#include <utility>

#include "common.cuh"

namespace les {

// ------------------------------------------------- compile-time twiddles ----
// cos/sin of 2 pi m / n from Taylor series on an argument reduced to the
// first octant (|phi| <= pi/4), with the exact octant symmetries.
constexpr double kPiCE = 3.14159265358979323846264338327950288;
constexpr double ce_sin_oct(double x) {
  double x2 = x * x, term = x, sum = x;
  for (int i = 1; i < 14; ++i) {
    term *= -x2 / double((2 * i) * (2 * i + 1));
    sum += term;
  }
  return sum;
}
constexpr double ce_cos_oct(double x) {
  double x2 = x * x, term = 1.0, sum = 1.0;
  for (int i = 1; i < 14; ++i) {
    term *= -x2 / double((2 * i - 1) * (2 * i));
    sum += term;
  }
  return sum;
}
struct CS {
  double c, s;
};
constexpr CS ce_cossin_2pi(long m, long n) {
  m %= n;
  if (m < 0) m += n;
  const long q = (8 * m) / n;
  const long r = 8 * m - q * n;
  const double phi = (kPiCE / 4.0) * (double(r) / double(n));
  const double psi = (kPiCE / 4.0) * (double(n - r) / double(n));
  switch (q) {
    case 0: return {ce_cos_oct(phi), ce_sin_oct(phi)};
    case 1: return {ce_sin_oct(psi), ce_cos_oct(psi)};
    case 2: return {-ce_sin_oct(phi), ce_cos_oct(phi)};
    case 3: return {-ce_cos_oct(psi), ce_sin_oct(psi)};
    case 4: return {-ce_cos_oct(phi), -ce_sin_oct(phi)};
    case 5: return {-ce_sin_oct(psi), -ce_cos_oct(psi)};
    case 6: return {ce_sin_oct(phi), -ce_cos_oct(phi)};
    default: return {ce_cos_oct(psi), -ce_sin_oct(psi)};
  }
}
template <int M, int R>
struct TwCE {
  static constexpr CS v = ce_cossin_2pi(M, R);
};

template <int... I, typename F>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

template <typename T>
__device__ __forceinline__ cplx<T> c_add(cplx<T> a, cplx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ cplx<T> c_sub(cplx<T> a, cplx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T>
__device__ __forceinline__ cplx<T> c_mul(cplx<T> a, cplx<T> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__device__ __forceinline__ cplx<T> c_mulc(cplx<T> a, cplx<T> b) {
  return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
// a + s b for a real s
template <typename T>
__device__ __forceinline__ cplx<T> c_axpy(cplx<T> a, T s, cplx<T> b) { return {a.x + s * b.x, a.y + s * b.y}; }
template <typename T>
__device__ __forceinline__ cplx<T> c_scl(cplx<T> a, T s) { return {a.x * s, a.y * s}; }
// componentwise a * s + b (s a pair of reals, e.g. the sign pattern (1, -1)
// of a conjugate sum)
template <typename T>
__device__ __forceinline__ cplx<T> c_fma(cplx<T> a, cplx<T> s, cplx<T> b) {
  return {a.x * s.x + b.x, a.y * s.y + b.y};
}

// FP32 complex adds on the packed FP32x2 instructions of sm_100: one
// instruction for both components, with the rounding of the scalar add,
// multiply or fused multiply-add per component (results are bit-identical
// to the scalar forms).  Complex multiplies stay scalar: their packed form
// needs the components of one operand duplicated and swapped, and the moves
// that takes cost more than the packed multiply saves.
__device__ __forceinline__ float2 f2_of(cplx<float> a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ cplx<float> c_of(float2 a) { return {a.x, a.y}; }
__device__ __forceinline__ float2 f2_sub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(r)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
template <>
__device__ __forceinline__ cplx<float> c_add<float>(cplx<float> a, cplx<float> b) {
  return c_of(__fadd2_rn(f2_of(a), f2_of(b)));
}
template <>
__device__ __forceinline__ cplx<float> c_sub<float>(cplx<float> a, cplx<float> b) {
  return c_of(f2_sub(f2_of(a), f2_of(b)));
}
template <>
__device__ __forceinline__ cplx<float> c_axpy<float>(cplx<float> a, float s, cplx<float> b) {
  return c_of(__ffma2_rn(make_float2(s, s), f2_of(b), f2_of(a)));
}
template <>
__device__ __forceinline__ cplx<float> c_scl<float>(cplx<float> a, float s) {
  return c_of(__fmul2_rn(f2_of(a), make_float2(s, s)));
}
template <>
__device__ __forceinline__ cplx<float> c_fma<float>(cplx<float> a, cplx<float> s, cplx<float> b) {
  return c_of(__ffma2_rn(f2_of(a), f2_of(s), f2_of(b)));
}

// ------------------------------------------------------ register DFTs ----
template <typename T, int R, bool INV>
struct RegDFT {
  static __device__ __forceinline__ void run(cplx<T>* v) {
    if constexpr (R == 1) {
    } else if constexpr (R == 2) {
      const cplx<T> a = v[0], b = v[1];
      v[0] = c_add(a, b);
      v[1] = c_sub(a, b);
    } else if constexpr (R == 3) {
      const T s3 = T(0.86602540378443864676372317075294);  // sqrt(3)/2
      const cplx<T> a = v[0];
      const cplx<T> t1 = c_add(v[1], v[2]), t2 = c_sub(v[1], v[2]);
      const cplx<T> m = c_axpy(a, T(-0.5), t1);
      const cplx<T> st = c_scl(t2, s3);
      const cplx<T> ist = INV ? cplx<T>{-st.y, st.x} : cplx<T>{st.y, -st.x};
      v[0] = c_add(a, t1);
      v[1] = c_add(m, ist);
      v[2] = c_sub(m, ist);
    } else if constexpr (R == 4) {
      const cplx<T> t0 = c_add(v[0], v[2]), t1 = c_sub(v[0], v[2]);
      const cplx<T> t2 = c_add(v[1], v[3]), t3 = c_sub(v[1], v[3]);
      const cplx<T> jt3 = INV ? cplx<T>{-t3.y, t3.x} : cplx<T>{t3.y, -t3.x};
      v[0] = c_add(t0, t2);
      v[2] = c_sub(t0, t2);
      v[1] = c_add(t1, jt3);
      v[3] = c_sub(t1, jt3);
    } else {
      // R = R1 * R2, n = n1 + R1 n2, k = k2 + R2 k1:
      // X[k2 + R2 k1] = sum_n1 W_R1^{n1 k1} W_R^{n1 k2} sum_n2 x[n1 + R1 n2] W_R2^{n2 k2}
      constexpr int R1 = (R % 4 == 0) ? 4 : ((R % 3 == 0) ? 3 : 2);
      constexpr int R2 = R / R1;
      static_for<R1>([&](auto n1c) {
        constexpr int n1 = decltype(n1c)::value;
        cplx<T> t[R2];
        static_for<R2>([&](auto n2c) { t[decltype(n2c)::value] = v[n1 + R1 * decltype(n2c)::value]; });
        RegDFT<T, R2, INV>::run(t);
        static_for<R2>([&](auto k2c) {
          constexpr int k2 = decltype(k2c)::value;
          constexpr int m = (n1 * k2) % R;
          if constexpr (4 * m == R) {
            // W_R^(R/4) = -i (forward) or +i (inverse): a swap
            t[k2] = INV ? cplx<T>{-t[k2].y, t[k2].x} : cplx<T>{t[k2].y, -t[k2].x};
          } else if constexpr (2 * m == R) {
            t[k2] = {-t[k2].x, -t[k2].y};
          } else if constexpr (4 * m == 3 * R) {
            t[k2] = INV ? cplx<T>{t[k2].y, -t[k2].x} : cplx<T>{-t[k2].y, t[k2].x};
          } else if constexpr (m != 0) {
            constexpr CS w = TwCE<m, R>::v;
            const cplx<T> tw = {T(w.c), INV ? T(w.s) : T(-w.s)};
            t[k2] = c_mul(t[k2], tw);
          }
          v[n1 + R1 * k2] = t[k2];
        });
      });
      cplx<T> out[R];
      static_for<R2>([&](auto k2c) {
        constexpr int k2 = decltype(k2c)::value;
        cplx<T> t[R1];
        static_for<R1>([&](auto n1c) { t[decltype(n1c)::value] = v[decltype(n1c)::value + R1 * k2]; });
        RegDFT<T, R1, INV>::run(t);
        static_for<R1>([&](auto k1c) { out[k2 + R2 * decltype(k1c)::value] = t[decltype(k1c)::value]; });
      });
      static_for<R>([&](auto ic) { v[decltype(ic)::value] = out[decltype(ic)::value]; });
    }
  }
};

// ------------------------------------------------------------- plans ----
// E = elements per lane, radices (each divides E), T = N / E lanes.
template <int N>
struct FFTPlan;
template <int E_, int... Rs>
struct PlanBase {
  static constexpr int E = E_;
};
template <> struct FFTPlan<8> : PlanBase<8, 8> {};
template <> struct FFTPlan<12> : PlanBase<12, 12> {};
template <> struct FFTPlan<16> : PlanBase<16, 16> {};
template <> struct FFTPlan<24> : PlanBase<24, 24> {};
template <> struct FFTPlan<32> : PlanBase<8, 8, 4> {};
template <> struct FFTPlan<48> : PlanBase<12, 12, 4> {};
template <> struct FFTPlan<64> : PlanBase<16, 16, 4> {};
template <> struct FFTPlan<96> : PlanBase<24, 24, 4> {};
template <> struct FFTPlan<128> : PlanBase<16, 16, 8> {};
template <> struct FFTPlan<192> : PlanBase<24, 24, 8> {};
template <> struct FFTPlan<256> : PlanBase<16, 16, 16> {};
template <> struct FFTPlan<384> : PlanBase<24, 24, 4, 4> {};
template <> struct FFTPlan<512> : PlanBase<16, 16, 16, 2> {};
template <> struct FFTPlan<768> : PlanBase<24, 24, 8, 4> {};

template <int N>
struct PlanRadices;
#define LES_PLAN(N, ...)                                   \
  template <>                                              \
  struct PlanRadices<N> {                                  \
    using seq = std::integer_sequence<int, __VA_ARGS__>;   \
  };
LES_PLAN(8, 8)
LES_PLAN(12, 12)
LES_PLAN(16, 16)
LES_PLAN(24, 24)
LES_PLAN(32, 8, 4)
LES_PLAN(48, 12, 4)
LES_PLAN(64, 16, 4)
LES_PLAN(96, 24, 4)
LES_PLAN(128, 16, 8)
LES_PLAN(192, 24, 8)
LES_PLAN(256, 16, 16)
LES_PLAN(384, 24, 4, 4)
LES_PLAN(512, 16, 16, 2)
LES_PLAN(768, 24, 8, 4)
#undef LES_PLAN

template <int First, int... Rest>
struct FirstOf {
  static constexpr int value = First;
};
template <int First, int... Rest>
struct LastOf {
  static constexpr int value = LastOf<Rest...>::value;
};
template <int First>
struct LastOf<First> {
  static constexpr int value = First;
};

template <int N>
struct Geo {
  static constexpr int E = FFTPlan<N>::E;
  static constexpr int T = N / E;
};


// Exchange layout of a sequence in its slot.  S = -1: element i at i + i/16
// (one element of padding every 16; the pass outputs are written at stride
// R, which would otherwise put a warp's lanes on a few banks).  S >= 1:
// element i at i ^ ((i >> S) & 15), a permutation within each aligned block
// of 16.  Each exchange (length N, element size ES bytes, stores of a
// radix-R pass after radices of product NS, loads of the next radix R2)
// takes the padding where that already puts a half warp (FP32 complex) or a
// quarter warp (FP64 complex) on distinct banks for both its stores and its
// loads -- its addresses differ by constants, which cost no instructions --
// and otherwise the permutation whose shift S does, found by enumerating the
// access patterns of every plan with the sequences that share a half (or
// quarter) warp at their slot_stride apart.
constexpr int exch_shift(int N, int ES, int R, int NS, int R2) {
  if (N == 32 && ES == 8 && R == 4 && NS == 1 && R2 == 8) return 2;
  if (N == 32 && ES == 8 && R == 8 && NS == 1 && R2 == 4) return 3;
  if (N == 32 && ES == 16 && R == 4 && NS == 1 && R2 == 8) return 2;
  if (N == 32 && ES == 16 && R == 8 && NS == 1 && R2 == 4) return 3;
  if (N == 48 && ES == 8 && R == 4 && NS == 1 && R2 == 12) return 2;
  if (N == 48 && ES == 8 && R == 12 && NS == 1 && R2 == 4) return 2;
  if (N == 48 && ES == 16 && R == 4 && NS == 1 && R2 == 12) return 2;
  if (N == 48 && ES == 16 && R == 12 && NS == 1 && R2 == 4) return 2;
  if (N == 64 && ES == 8 && R == 4 && NS == 1 && R2 == 16) return 2;
  if (N == 64 && ES == 8 && R == 16 && NS == 1 && R2 == 4) return -1;
  if (N == 64 && ES == 16 && R == 4 && NS == 1 && R2 == 16) return 2;
  if (N == 64 && ES == 16 && R == 16 && NS == 1 && R2 == 4) return -1;
  if (N == 96 && ES == 8 && R == 4 && NS == 1 && R2 == 24) return 2;
  if (N == 96 && ES == 8 && R == 24 && NS == 1 && R2 == 4) return 3;
  if (N == 96 && ES == 16 && R == 4 && NS == 1 && R2 == 24) return 2;
  if (N == 96 && ES == 16 && R == 24 && NS == 1 && R2 == 4) return 3;
  if (N == 128 && ES == 8 && R == 8 && NS == 1 && R2 == 16) return 3;
  if (N == 128 && ES == 8 && R == 16 && NS == 1 && R2 == 8) return -1;
  if (N == 128 && ES == 16 && R == 8 && NS == 1 && R2 == 16) return 3;
  if (N == 128 && ES == 16 && R == 16 && NS == 1 && R2 == 8) return -1;
  if (N == 192 && ES == 8 && R == 8 && NS == 1 && R2 == 24) return 3;
  if (N == 192 && ES == 8 && R == 24 && NS == 1 && R2 == 8) return 3;
  if (N == 192 && ES == 16 && R == 8 && NS == 1 && R2 == 24) return 3;
  if (N == 192 && ES == 16 && R == 24 && NS == 1 && R2 == 8) return 3;
  if (N == 256 && ES == 8 && R == 16 && NS == 1 && R2 == 16) return -1;
  if (N == 256 && ES == 16 && R == 16 && NS == 1 && R2 == 16) return -1;
  if (N == 384 && ES == 8 && R == 4 && NS == 1 && R2 == 4) return -1;
  if (N == 384 && ES == 8 && R == 4 && NS == 4 && R2 == 24) return 2;
  if (N == 384 && ES == 8 && R == 4 && NS == 24 && R2 == 4) return 3;
  if (N == 384 && ES == 8 && R == 24 && NS == 1 && R2 == 4) return 3;
  if (N == 384 && ES == 16 && R == 4 && NS == 1 && R2 == 4) return 2;
  if (N == 384 && ES == 16 && R == 4 && NS == 4 && R2 == 24) return 2;
  if (N == 384 && ES == 16 && R == 4 && NS == 24 && R2 == 4) return -1;
  if (N == 384 && ES == 16 && R == 24 && NS == 1 && R2 == 4) return 3;
  if (N == 512 && ES == 8 && R == 2 && NS == 1 && R2 == 16) return -1;
  if (N == 512 && ES == 8 && R == 16 && NS == 1 && R2 == 16) return -1;
  if (N == 512 && ES == 8 && R == 16 && NS == 2 && R2 == 16) return -1;
  if (N == 512 && ES == 8 && R == 16 && NS == 16 && R2 == 2) return -1;
  if (N == 512 && ES == 16 && R == 2 && NS == 1 && R2 == 16) return 1;
  if (N == 512 && ES == 16 && R == 16 && NS == 1 && R2 == 16) return -1;
  if (N == 512 && ES == 16 && R == 16 && NS == 2 && R2 == 16) return -1;
  if (N == 512 && ES == 16 && R == 16 && NS == 16 && R2 == 2) return -1;
  if (N == 768 && ES == 8 && R == 4 && NS == 1 && R2 == 8) return -1;
  if (N == 768 && ES == 8 && R == 8 && NS == 4 && R2 == 24) return 3;
  if (N == 768 && ES == 8 && R == 8 && NS == 24 && R2 == 4) return 3;
  if (N == 768 && ES == 8 && R == 24 && NS == 1 && R2 == 8) return 3;
  if (N == 768 && ES == 16 && R == 4 && NS == 1 && R2 == 8) return 2;
  if (N == 768 && ES == 16 && R == 8 && NS == 4 && R2 == 24) return 3;
  if (N == 768 && ES == 16 && R == 8 && NS == 24 && R2 == 4) return -1;
  if (N == 768 && ES == 16 && R == 24 && NS == 1 && R2 == 8) return 3;
  return -1;
}
template <int S>
__device__ __forceinline__ int exch_pos(int i) {
  if constexpr (S < 0) return i + (i >> 4);
  else if constexpr (S == 0) return i;
  else return i ^ ((i >> S) & 15);
}

// one pass of radix R with Ns = product of the previous radices, its
// twiddle factors at twm[OFF + (r-1) Ns + k]; then the exchange into the next
// pass's input layout (if any)
template <typename T, int N, int E, bool INV, int Ns, int OFF, int R, int... Rest>
__device__ __forceinline__ void reg_passes(cplx<T>* v, cplx<T>* seq, int t, const cplx<T>* __restrict__ twm) {
  constexpr int TL = N / E;
  constexpr int G = E / R;
#pragma unroll
  for (int g = 0; g < G; ++g) {
    if constexpr (Ns > 1) {
      const int j = t + TL * g;
      const int k = j % Ns;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const cplx<T> w = twm[OFF + (r - 1) * Ns + k];
        v[g * R + r] = INV ? c_mulc(v[g * R + r], w) : c_mul(v[g * R + r], w);
      }
    }
    RegDFT<T, R, INV>::run(v + g * R);
  }
  if constexpr (sizeof...(Rest) > 0) {
    constexpr int R2 = FirstOf<Rest...>::value;
    constexpr int G2 = E / R2;
    constexpr int SW = exch_shift(N, int(sizeof(cplx<T>)), R, Ns, R2);
    __syncwarp();
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int j = t + TL * g;
      const int k = j % Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) seq[exch_pos<SW>((j / Ns) * Ns * R + k + r * Ns)] = v[g * R + r];
    }
    __syncwarp();
#pragma unroll
    for (int g = 0; g < G2; ++g)
#pragma unroll
      for (int r = 0; r < R2; ++r) v[g * R2 + r] = seq[exch_pos<SW>(t + TL * g + r * (N / R2))];
    reg_passes<T, N, E, INV, Ns * R, OFF + (Ns > 1 ? (R - 1) * Ns : 0), Rest...>(v, seq, t, twm);
  }
}

template <typename T, int N, bool INV, int... Rs>
__device__ __forceinline__ void reg_fft_impl(cplx<T>* v, cplx<T>* seq, int t, const cplx<T>* twm,
                                             std::integer_sequence<int, Rs...>) {
  reg_passes<T, N, Geo<N>::E, INV, 1, 0, Rs...>(v, seq, t, twm);
}

// reversed radix list (the inverse runs the plan backwards)
template <typename S, typename R>
struct RevSeq;
template <int... Acc>
struct RevSeq<std::integer_sequence<int>, std::integer_sequence<int, Acc...>> {
  using type = std::integer_sequence<int, Acc...>;
};
template <int H, int... Tl, int... Acc>
struct RevSeq<std::integer_sequence<int, H, Tl...>, std::integer_sequence<int, Acc...>> {
  using type = typename RevSeq<std::integer_sequence<int, Tl...>, std::integer_sequence<int, H, Acc...>>::type;
};

template <int N, bool INV>
struct PassOrder {
  using seq = typename std::conditional<
      INV, typename RevSeq<typename PlanRadices<N>::seq, std::integer_sequence<int>>::type,
      typename PlanRadices<N>::seq>::type;
};

// ------------------------------------------------ twiddle matrices ----
// The twiddle factors of every pass after the first (radix R after radices
// of product Ns) are W^(r k N/(Ns R)) for r = 1..R-1, k = 0..Ns-1 with
// k = (lane + T g) mod Ns.  Read from a table of W^m they sit at stride
// r k, which puts the lanes of a sequence on a few banks; the matrix of a
// pass stores them as [r-1][k], so those lanes read consecutive entries.
// Matrices of all passes of a plan follow each other (twm_len entries).
template <int Ns, int R, int... Rest>
struct TwmLen {
  static constexpr int value = (Ns > 1 ? (R - 1) * Ns : 0) + TwmLen<Ns * R, Rest...>::value;
};
template <int Ns, int R>
struct TwmLen<Ns, R> {
  static constexpr int value = (Ns > 1 ? (R - 1) * Ns : 0);
};
template <int... Rs>
constexpr int twm_len_impl(std::integer_sequence<int, Rs...>) {
  return TwmLen<1, Rs...>::value;
}
template <int N, bool INV>
struct Twm {
  static constexpr int len = twm_len_impl(typename PassOrder<N, INV>::seq{});
};

// radix i of the forward plan of length N (0 past the last), for the host's
// shared-memory sizing; matches PlanRadices
__host__ __device__ constexpr int plan_radix(int N, int i) {
  switch (N) {
    case 8: return i == 0 ? 8 : 0;
    case 12: return i == 0 ? 12 : 0;
    case 16: return i == 0 ? 16 : 0;
    case 24: return i == 0 ? 24 : 0;
    case 32: return i == 0 ? 8 : (i == 1 ? 4 : 0);
    case 48: return i == 0 ? 12 : (i == 1 ? 4 : 0);
    case 64: return i == 0 ? 16 : (i == 1 ? 4 : 0);
    case 96: return i == 0 ? 24 : (i == 1 ? 4 : 0);
    case 128: return i == 0 ? 16 : (i == 1 ? 8 : 0);
    case 192: return i == 0 ? 24 : (i == 1 ? 8 : 0);
    case 256: return i == 0 ? 16 : (i == 1 ? 16 : 0);
    case 384: return i == 0 ? 24 : (i == 1 ? 4 : (i == 2 ? 4 : 0));
    case 512: return i == 0 ? 16 : (i == 1 ? 16 : (i == 2 ? 2 : 0));
    case 768: return i == 0 ? 24 : (i == 1 ? 8 : (i == 2 ? 4 : 0));
    default: return 0;
  }
}
// Distance between the shared-memory slots of consecutive sequences, in
// complex values of ES bytes: room for N + N/16 values (the padded exchange
// layout), then raised to TL (mod W), W = 128 / ES values per wavefront, when
// the TL lanes of a sequence fill less than a half (FP32) or quarter (FP64)
// warp: the W/TL sequences of one wavefront then cover disjoint banks in the
// loads, stores and splits that walk consecutive elements.  FP32 slots stay
// even (16-byte aligned: the x passes move four reals at once).
__host__ __device__ constexpr int slot_stride(int N, int ES) {
  const int TL = N / plan_radix(N, 0);
  const int W = 128 / ES;
  const int base = (N + N / 16 + 1) & ~1;
  if (TL >= W) return base;
  int want = TL % W;
  if (ES == 8 && (want & 1)) want = 2;
  return base + ((want - base % W) % W + W) % W;
}

// entries of the twiddle matrices of the forward (inv = false) or inverse
// transform of length N
__host__ __device__ constexpr int twm_len(int N, bool inv) {
  int n = 0;
  while (n < 4 && plan_radix(N, n) != 0) ++n;
  int len = 0, ns = 1;
  for (int p = 0; p < n; ++p) {
    const int r = plan_radix(N, inv ? n - 1 - p : p);
    if (p > 0) len += (r - 1) * ns;
    ns *= r;
  }
  return len;
}

template <typename T, int N, int TWS, int Ns, int OFF, int R, int... Rest>
__device__ __forceinline__ void twm_fill(const cplx<T>* __restrict__ tw, cplx<T>* twm, int tid, int nth) {
  if constexpr (Ns > 1) {
    for (int i = tid; i < (R - 1) * Ns; i += nth) {
      const int r = 1 + i / Ns, k = i % Ns;
      twm[OFF + i] = tw[(r * k * (N / (Ns * R))) * TWS];
    }
  }
  if constexpr (sizeof...(Rest) > 0)
    twm_fill<T, N, TWS, Ns * R, OFF + (Ns > 1 ? (R - 1) * Ns : 0), Rest...>(tw, twm, tid, nth);
}
template <typename T, int N, int TWS, int... Rs>
__device__ __forceinline__ void twm_build_impl(const cplx<T>* tw, cplx<T>* twm, int tid, int nth,
                                               std::integer_sequence<int, Rs...>) {
  twm_fill<T, N, TWS, 1, 0, Rs...>(tw, twm, tid, nth);
}
// Fill the matrices of the length-N transform (direction INV) from a table
// tw of exp(-2 pi i m / (N*TWS)) read at stride TWS; threads tid of nth share
// the work.  The caller synchronises before the first transform.
template <typename T, int N, bool INV, int TWS = 1>
__device__ __forceinline__ void twm_build(const cplx<T>* tw, cplx<T>* twm, int tid, int nth) {
  static_assert(Twm<N, INV>::len == twm_len(N, INV), "plan table and host sizing disagree");
  twm_build_impl<T, N, TWS>(tw, twm, tid, nth, typename PassOrder<N, INV>::seq{});
}

// The transform: v as in the layout contract above; seq is this sequence's
// shared slot of slot_stride(N, sizeof(cplx<T>)) elements (private to its T
// lanes); twm holds the twiddle matrices built by twm_build<T, N, INV>.
// Forward transforms run the plan's radices in order, inverse transforms in
// reverse order.
template <typename T, int N, bool INV>
__device__ __forceinline__ void reg_fft(cplx<T>* v, cplx<T>* seq, int t, const cplx<T>* twm) {
  reg_fft_impl<T, N, INV>(v, seq, t, twm, typename PassOrder<N, INV>::seq{});
}

template <int N, int... Rs>
constexpr int first_radix_impl(std::integer_sequence<int, Rs...>) {
  return FirstOf<Rs...>::value;
}
template <int N, int... Rs>
constexpr int last_radix_impl(std::integer_sequence<int, Rs...>) {
  return LastOf<Rs...>::value;
}
// In / out group radices of a transform: forward input layout groups of the
// plan's first radix, output groups of its last; the inverse the reverse.
template <int N, bool INV>
struct Layout {
  static constexpr int in = first_radix_impl<N>(typename PassOrder<N, INV>::seq{});
  static constexpr int out = last_radix_impl<N>(typename PassOrder<N, INV>::seq{});
};

}  // namespace les
