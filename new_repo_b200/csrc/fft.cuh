// Shared-memory Stockham FFTs of compile-time length N = 2^a 3^b.
//
// Replaces the FFTW 1-D plans of fft_engine.f90:65-78 and
// decomp_2d_fft_2d.f90:245-323.  Every transform is unnormalised, like
// FFTW's.  A CTA transforms a batch of sequences held in shared memory; all
// threads cooperate on every radix stage (one butterfly per loop trip) and
// the stages ping-pong between two buffers (autosort, natural order out).
#pragma once
#include "common.cuh"

namespace les {

template <int REM>
struct RadixOf {
  static constexpr int value = (REM % 3 == 0) ? 3 : ((REM % 4 == 0) ? 4 : 2);
};

// Radix-R DFT of v[0..R) in registers; INV selects the +i sign.
template <typename T, int R, bool INV>
__device__ __forceinline__ void butterfly(cplx<T>* v) {
  if constexpr (R == 2) {
    cplx<T> a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    cplx<T> t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    cplx<T> t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
    // forward: -i * t3 ; inverse: +i * t3
    cplx<T> jt3 = INV ? cplx<T>{-t3.y, t3.x} : cplx<T>{t3.y, -t3.x};
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, jt3);
    v[3] = csub(t1, jt3);
  } else {  // R == 3
    const T s3 = T(0.86602540378443864676372317075294);  // sqrt(3)/2
    cplx<T> a = v[0];
    cplx<T> t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    cplx<T> m = {a.x - T(0.5) * t1.x, a.y - T(0.5) * t1.y};
    // forward: W = -1/2 - i s3 ; y1 = m - i s3 t2, y2 = m + i s3 t2
    cplx<T> st = {s3 * t2.x, s3 * t2.y};
    cplx<T> ist = INV ? cplx<T>{-st.y, st.x} : cplx<T>{st.y, -st.x};
    v[0] = cadd(a, t1);
    v[1] = cadd(m, ist);
    v[2] = csub(m, ist);
  }
}

// One Stockham pass followed by the rest (compile-time recursion on Ns).
// tw: table of exp(-2 pi i m / (N*TWS)), read at stride TWS.
template <typename T, int N, int Ns, bool INV, int TWS>
struct Stockham {
  static __device__ __forceinline__ void run(cplx<T>*& src, cplx<T>*& dst, int nseq, int sstride,
                                             const cplx<T>* __restrict__ tw) {
    if constexpr (Ns < N) {
      constexpr int R = RadixOf<N / Ns>::value;
      constexpr int NB = N / R;
      constexpr int TWSTEP = (N / (Ns * R)) * TWS;
      const int total = nseq * NB;
      for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int s = idx / NB;
        const int j = idx - s * NB;
        const int k = j % Ns;
        const cplx<T>* in = src + s * sstride;
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = in[j + r * NB];
        if constexpr (Ns > 1) {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            cplx<T> w = tw[r * k * TWSTEP];
            v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
          }
        }
        butterfly<T, R, INV>(v);
        cplx<T>* out = dst + s * sstride;
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) out[base + r * Ns] = v[r];
      }
      __syncthreads();
      cplx<T>* t = src;
      src = dst;
      dst = t;
      Stockham<T, N, Ns * R, INV, TWS>::run(src, dst, nseq, sstride, tw);
    }
  }
};

// Transform nseq sequences of length N stored at buf0 + s*sstride.  Returns
// the buffer that holds the result (buf0 or buf1).  Caller must have
// synchronised after filling buf0; the result is synchronised on return.
template <typename T, int N, bool INV, int TWS = 1>
__device__ __forceinline__ cplx<T>* fft_batch(cplx<T>* buf0, cplx<T>* buf1, int nseq, int sstride,
                                              const cplx<T>* __restrict__ tw) {
  cplx<T>* src = buf0;
  cplx<T>* dst = buf1;
  Stockham<T, N, 1, INV, TWS>::run(src, dst, nseq, sstride, tw);
  return src;
}

}  // namespace les
