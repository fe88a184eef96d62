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
      const cplx<T> m = {a.x - T(0.5) * t1.x, a.y - T(0.5) * t1.y};
      const cplx<T> st = {s3 * t2.x, s3 * t2.y};
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
          if constexpr (m != 0) {
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

// Exchange slots are padded by one element every 16: the pass outputs are
// written at stride R, which would otherwise put a warp's lanes on a few
// banks.  A sequence of N elements needs N + N/16 elements of slot;
// slot_len<N>() rounds that up to even so that consecutive slots of FP32
// complex values stay 16-byte aligned (the x passes move 4 reals at once).
template <int N>
__host__ __device__ constexpr int slot_len() {
  return (N + N / 16 + 1) & ~1;
}
__device__ __forceinline__ int xpad(int i) { return i + (i >> 4); }

// one pass of radix R with Ns = product of the previous radices; then the
// exchange into the next pass's input layout (if any)
template <typename T, int N, int E, bool INV, int TWS, int Ns, int R, int... Rest>
__device__ __forceinline__ void reg_passes(cplx<T>* v, cplx<T>* seq, int t, const cplx<T>* __restrict__ tw) {
  constexpr int TL = N / E;
  constexpr int G = E / R;
#pragma unroll
  for (int g = 0; g < G; ++g) {
    if constexpr (Ns > 1) {
      const int j = t + TL * g;
      const int k = j % Ns;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const cplx<T> w = tw[(r * k * (N / (Ns * R))) * TWS];
        v[g * R + r] = INV ? c_mulc(v[g * R + r], w) : c_mul(v[g * R + r], w);
      }
    }
    RegDFT<T, R, INV>::run(v + g * R);
  }
  if constexpr (sizeof...(Rest) > 0) {
    __syncwarp();
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int j = t + TL * g;
      const int k = j % Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) seq[xpad((j / Ns) * Ns * R + k + r * Ns)] = v[g * R + r];
    }
    __syncwarp();
    constexpr int R2 = FirstOf<Rest...>::value;
    constexpr int G2 = E / R2;
#pragma unroll
    for (int g = 0; g < G2; ++g)
#pragma unroll
      for (int r = 0; r < R2; ++r) v[g * R2 + r] = seq[xpad(t + TL * g + r * (N / R2))];
    reg_passes<T, N, E, INV, TWS, Ns * R, Rest...>(v, seq, t, tw);
  }
}

template <typename T, int N, bool INV, int TWS, int... Rs>
__device__ __forceinline__ void reg_fft_impl(cplx<T>* v, cplx<T>* seq, int t, const cplx<T>* tw,
                                             std::integer_sequence<int, Rs...>) {
  reg_passes<T, N, Geo<N>::E, INV, TWS, 1, Rs...>(v, seq, t, tw);
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

// The transform: v as in the layout contract above; seq is this sequence's
// shared slot of slot_len<N>() elements (private to its T lanes); tw holds
// exp(-2 pi i m / (N*TWS)) read at stride TWS.  Forward transforms run the
// plan's radices in order, inverse transforms in reverse order.
template <typename T, int N, bool INV, int TWS = 1>
__device__ __forceinline__ void reg_fft(cplx<T>* v, cplx<T>* seq, int t, const cplx<T>* tw) {
  reg_fft_impl<T, N, INV, TWS>(v, seq, t, tw, typename PassOrder<N, INV>::seq{});
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
