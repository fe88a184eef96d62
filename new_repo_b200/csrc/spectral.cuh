// Batched horizontal 2-D real FFT passes with fused prologues/epilogues.
//
// A 2-D r2c/c2r of the reference (decomp_2d_fft_2d.f90:498-577: x r2c,
// transpose X->Y, y c2c) becomes three kernel families that work on every
// level of a field in one launch:
//
//   xfwd  : physical rows (length NX) -> half-spectrum rows, first nk modes.
//           The load step computes the transformed quantity on the fly
//           (scaling, vorticity, fine-grid products, SGS test-filter inputs).
//   ypass : columns of a spectral buffer -> y FFT (length NY) -> spectral op
//           (i*k multiply, Nyquist kill, filter, 3/2 pad or truncate) ->
//           inverse y FFT (length NYO) -> spectral buffer.  This is where the
//           2DECOMP X<->Y pencil transpose happens: columns are staged through
//           shared memory, no global transpose is ever written.
//   xinv  : half-spectrum rows -> c2r (length NX) -> fused store op
//           (plain store, rhs accumulation, stress divergence with its dz
//           term and pressure-BC layers, SGS dynamic-procedure contraction).
//
// Spectral buffers are [level][ky row][kx] with kx fastest, so the x passes
// read and write whole contiguous rows and the y pass reads C consecutive kx
// columns per row (128-byte segments).
#pragma once
#include <type_traits>

#include "common.cuh"
#include "fft2.cuh"
#include "tc05.cuh"

namespace les {

constexpr int MAXIN = 24;
constexpr int MAXOUT = 48;

// ---- asynchronous global -> shared copies (cp.async) ----
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int n = valid ? BYTES : 0;  // 0: zero fill, nothing read
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gmem), "r"(n) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(d), "l"(gmem), "n"(BYTES), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---- bulk global -> shared copies (cp.async.bulk, completion on an mbarrier) ----
// One instruction moves a whole contiguous row: both addresses 16-byte
// aligned, the size a multiple of 16.  No multicast: the destination is this
// CTA's shared memory only.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(tc::smem_u32(dst)), "l"(src), "r"(bytes), "r"(tc::smem_u32(mbar))
               : "memory");
}
// the one arrival of a stage's mbarrier, announcing the bytes its copies bring
__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(mbar)), "r"(bytes)
               : "memory");
}

// r2c split of a length-2M real row transformed as M complex values Z:
// X_k = (Z_k + conj Z_{M-k}) / 2 + W^k (Z_k - conj Z_{M-k}) / (2i), with
// wh = W^k / 2 (W = exp(-2 pi i / 2M)).  The sums with the sign pairs are
// packed FP32x2 instructions in single precision.
template <typename T>
__device__ __forceinline__ cplx<T> r2c_split(cplx<T> zk, cplx<T> zm, cplx<T> wh) {
  const cplx<T> sp = c_fma(zm, cplx<T>{T(1), T(-1)}, zk);  // Z_k + conj Z_{M-k}
  const cplx<T> dp = c_fma(zm, cplx<T>{T(-1), T(1)}, zk);  // Z_k - conj Z_{M-k}
  const cplx<T> q = {dp.y * wh.x + dp.x * wh.y, dp.y * wh.y - dp.x * wh.x};  // dp wh / i
  return c_fma(sp, cplx<T>{T(0.5), T(0.5)}, q);
}
// c2r split, the inverse of the above without the halving:
// Z_m = (X_m + conj X_{M-m}) + i W^{-m} (X_m - conj X_{M-m}).
template <typename T>
__device__ __forceinline__ cplx<T> c2r_split(cplx<T> xk, cplx<T> xm, cplx<T> w) {
  const cplx<T> s1 = c_fma(xm, cplx<T>{T(1), T(-1)}, xk);
  const cplx<T> d1 = c_fma(xm, cplx<T>{T(-1), T(1)}, xk);
  // t = d1 conj(w), held swapped as (t.y, t.x); Z = s1 + i t
  const cplx<T> ts = {d1.y * w.x - d1.x * w.y, d1.x * w.x + d1.y * w.y};
  return c_fma(ts, cplx<T>{T(-1), T(1)}, s1);
}

// r2c split and store of the first nk modes of a sequence whose FFT output
// Z sits in natural order in its slot: lane t writes modes k = t + TL i
// (i <= E: mode M, the Nyquist bin, falls on lane 0 at i = E), an unrolled
// loop with compile-time offsets; Z_M is Z_0 and the partner of mode 0 is
// Z_0 itself
template <typename T, int M, int TL, int E>
__device__ __forceinline__ void xf_split_store(const cplx<T>* seq, const cplx<T>* tw, cplx<T>* orow, int t, int nk) {
#pragma unroll
  for (int i = 0; i <= E; ++i) {
    const int k = t + TL * i;
    if (k < nk) {
      if (i == 0) orow[k] = r2c_split(seq[k], seq[k == 0 ? 0 : M - k], tw[k]);
      else if (i < E) orow[k] = r2c_split(seq[k], seq[M - k], tw[k]);
      else orow[k] = r2c_split(seq[0], seq[0], tw[M]);  // k = M (t = 0)
    }
  }
}

// ---------------------------------------------------------------- xfwd ----
enum XFOp : int {
  XF_SCALE = 0,   // field f = c0 * in[f]
  XF_CONV_IN = 1, // u,v,w scaled by -c0 and the three vorticity components (c0 scaled)
  XF_PROD = 2,    // fine-grid u x omega products (inputs on the padded grid)
  XF_LASD = 3,    // the 21 test-filter inputs of the dynamic procedure
  XF_PRESS = 4,   // field f = c0 * (in[f] / c1)   (compute_pressure.f90:138-140)
  XF_PROD_SC = 5, // fine-grid scalar advection -(u . grad theta) (inputs on the padded grid)
  XF_SCDYN = 6,   // the 19 test-filter inputs of the dynamic Prandtl model
  XF_PRESS_INC = 7,  // pressure right-hand side from the AB2 increment and div u^n
};

template <typename T>
struct XFArgs {
  int op, nf, R;
  long nrows;      // rows to process = nplanes * rows_pp
  int rows_pp;     // rows per plane of the input grid
  int plane0;      // first level
  int nk;          // modes stored per output row
  int opitch;      // complex values between output rows (>= nk; 0: nk)
  int nz;
  int wall;        // wall-law special rows at k=1
  int use_ref;     // subtract each field's value at (i,j)=(0,0) of the level
  int fluct;       // XF_LASD: form products of u, v, w minus their (0,0) values
  double ref_mul;  // refout = ref * ref_mul (the value the inverse adds back)
  T* refout[MAXIN];
  long in_pstride; // elements per plane of the input grid
  long in_rstride; // elements per row of the input grid (== NX)
  double c0, c1, c2;
  const T* in[16];
  const float* inf[16];  // FP32 inputs of an FP64 transform (in_f32 = 1)
  int in_f32;
  cplx<T>* out[MAXIN];
  long out_pstride;  // rows_pp * nk
  // staged kernel (k_xfwd_st): input rows copied per grid row, source q is
  // field sf[q] at level offset sdl[q]; scond[q]: only on the wall row (l = 1)
  int nsrc;
  int sf[16], sdl[16], scond[16];
  const cplx<T>* tw; // exp(-2 pi i m / NX), m < NX
};

// Four consecutive x points of one row, moved with 16-byte loads and stores.
template <typename T>
struct V4 {
  T e[4];
};
template <typename T>
__device__ __forceinline__ V4<T> operator+(const V4<T>& a, const V4<T>& b) {
  return {{a.e[0] + b.e[0], a.e[1] + b.e[1], a.e[2] + b.e[2], a.e[3] + b.e[3]}};
}
template <typename T>
__device__ __forceinline__ V4<T> operator-(const V4<T>& a, const V4<T>& b) {
  return {{a.e[0] - b.e[0], a.e[1] - b.e[1], a.e[2] - b.e[2], a.e[3] - b.e[3]}};
}
template <typename T>
__device__ __forceinline__ V4<T> operator*(const V4<T>& a, const V4<T>& b) {
  return {{a.e[0] * b.e[0], a.e[1] * b.e[1], a.e[2] * b.e[2], a.e[3] * b.e[3]}};
}
template <typename T>
__device__ __forceinline__ V4<T> operator*(T c, const V4<T>& b) {
  return {{c * b.e[0], c * b.e[1], c * b.e[2], c * b.e[3]}};
}
template <typename T>
__device__ __forceinline__ V4<T> operator/(const V4<T>& a, T c) {
  return {{a.e[0] / c, a.e[1] / c, a.e[2] / c, a.e[3] / c}};
}
template <typename T>
__device__ __forceinline__ V4<T> operator-(const V4<T>& a) {
  return {{-a.e[0], -a.e[1], -a.e[2], -a.e[3]}};
}

// value type V (T: one point, V4<T>: four points) loaded from S* at off
template <typename V, typename S>
struct VLd;
template <typename S>
struct VLd<float, S> {
  static __device__ __forceinline__ float ld(const S* p, long o) { return float(p[o]); }
};
template <typename S>
struct VLd<double, S> {
  static __device__ __forceinline__ double ld(const S* p, long o) { return double(p[o]); }
};
template <>
struct VLd<V4<float>, float> {
  static __device__ __forceinline__ V4<float> ld(const float* p, long o) {
    const float4 q = *reinterpret_cast<const float4*>(p + o);
    return {{q.x, q.y, q.z, q.w}};
  }
};
template <>
struct VLd<V4<double>, double> {
  static __device__ __forceinline__ V4<double> ld(const double* p, long o) {
    const double2 q0 = *reinterpret_cast<const double2*>(p + o);
    const double2 q1 = *reinterpret_cast<const double2*>(p + o + 2);
    return {{q0.x, q0.y, q1.x, q1.y}};
  }
};
template <>
struct VLd<V4<double>, float> {
  static __device__ __forceinline__ V4<double> ld(const float* p, long o) {
    const float4 q = *reinterpret_cast<const float4*>(p + o);
    return {{double(q.x), double(q.y), double(q.z), double(q.w)}};
  }
};
template <typename V, typename S>
__device__ __forceinline__ V vld(const S* p, long o) {
  return VLd<V, S>::ld(p, o);
}
// the same through the read-only data path (ld.global.nc): for inputs that
// no thread of the kernel writes; the compiler may then schedule these
// loads across shared-memory stores
template <typename V, typename S>
__device__ __forceinline__ V vldg(const S* p, long o) {
  if constexpr (std::is_same<V, V4<float>>::value && std::is_same<S, float>::value) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p + o));
    return {{q.x, q.y, q.z, q.w}};
  } else if constexpr (std::is_same<V, V4<double>>::value && std::is_same<S, double>::value) {
    const double2 q0 = __ldg(reinterpret_cast<const double2*>(p + o));
    const double2 q1 = __ldg(reinterpret_cast<const double2*>(p + o + 2));
    return {{q0.x, q0.y, q1.x, q1.y}};
  } else if constexpr (std::is_same<V, V4<double>>::value && std::is_same<S, float>::value) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p + o));
    return {{double(q.x), double(q.y), double(q.z), double(q.w)}};
  } else {
    return V(__ldg(p + o));
  }
}
template <typename T>
__device__ __forceinline__ void vst(T* p, T x) {
  *p = x;
}
__device__ __forceinline__ void vst(float* p, const V4<float>& x) {
  *reinterpret_cast<float4*>(p) = make_float4(x.e[0], x.e[1], x.e[2], x.e[3]);
}
__device__ __forceinline__ void vst(double* p, const V4<double>& x) {
  reinterpret_cast<double2*>(p)[0] = make_double2(x.e[0], x.e[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(x.e[2], x.e[3]);
}
template <typename V, typename T>
__device__ __forceinline__ V vsplat(T x) {
  if constexpr (std::is_same<V, T>::value) return x;
  else return V{{x, x, x, x}};
}

// Values of every field of op OP at level l, row j, columns i (one point for
// V = T, four for V = V4<T>; i a multiple of 4 then), stored at v + f * vs,
// minus sub[f] when SUB (the per-level references of the mixed-precision
// transforms).  The op is a template parameter so that a pass's load loop
// is compiled per op, with no dispatch per point.
template <typename T, typename V, int OP, bool SUB>
__device__ __forceinline__ void xf_load_op(const XFArgs<T>& a, int l, int j, int i, T* v, int vs, const T* sub) {
  const long off = (long)l * a.in_pstride + (long)j * a.in_rstride + i;
  auto put = [&](int f, const V& x) {
    if constexpr (SUB) vst(v + f * vs, x - vsplat<V>(sub[f]));
    else vst(v + f * vs, x);
  };
  {
    if constexpr (OP == XF_SCALE) {
      for (int f = 0; f < a.nf; ++f)
        put(f, T(a.c0) * (a.in_f32 ? vldg<V>(a.inf[f], off) : vldg<V>(a.in[f], off)));
    } else if constexpr (OP == XF_PRESS) {
      // compute_pressure.f90:138-140
      for (int f = 0; f < a.nf; ++f) {
        const V x = a.in_f32 ? vldg<V>(a.inf[f], off) : vldg<V>(a.in[f], off);
        put(f, T(a.c0) * (x / T(a.c1)));
      }
    } else if constexpr (OP == XF_CONV_IN) {
      // compute_convective_padd.f90:133-165
      const T c = T(a.c0);
      put(0, -c * vldg<V>(a.in[0], off));
      put(1, -c * vldg<V>(a.in[1], off));
      put(2, -c * vldg<V>(a.in[2], off));
      const T* dwdy = a.in[3];
      const T* dvdz = a.in[4];
      const T* dudz = a.in[5];
      const T* dwdx = a.in[6];
      const T* dvdx = a.in[7];
      const T* dudy = a.in[8];
      if (a.wall && l == 0) {
        put(3, vsplat<V>(T(0)));
        put(4, vsplat<V>(T(0)));
      } else if (a.wall && l == 1) {
        const long up = off + a.in_pstride;
        put(3, c * (T(0.5) * (vldg<V>(dwdy, off) + vldg<V>(dwdy, up)) - vldg<V>(dvdz, off)));
        put(4, c * (vldg<V>(dudz, off) - T(0.5) * (vldg<V>(dwdx, off) + vldg<V>(dwdx, up))));
      } else {
        put(3, c * (vldg<V>(dwdy, off) - vldg<V>(dvdz, off)));
        put(4, c * (vldg<V>(dudz, off) - vldg<V>(dwdx, off)));
      }
      put(5, c * (vldg<V>(dvdx, off) - vldg<V>(dudy, off)));
    } else if constexpr (OP == XF_PROD) {
      // compute_convective_padd.f90:180-249 on the fine grid; inputs are
      // ub, vb, wb, o1, o2, o3 (padded -c*u, -c*v, -c*w and vorticity).
      const T c = T(a.c0);
      const T* ub = a.in[0];
      const T* vb = a.in[1];
      const T* wb = a.in[2];
      const T* o1 = a.in[3];
      const T* o2 = a.in[4];
      const T* o3 = a.in[5];
      const long up = off + a.in_pstride;
      const long dn = off - a.in_pstride;
      const V vb0 = vldg<V>(vb, off), o30 = vldg<V>(o3, off), ub0 = vldg<V>(ub, off);
      const V wbu = vldg<V>(wb, up), o2u = vldg<V>(o2, up), o1u = vldg<V>(o1, up);
      if (l == 1) {
        put(0, c * (-vb0 * o30 + T(0.5) * wbu * o2u));
        put(1, c * (ub0 * o30 + T(0.5) * wbu * (-o1u)));
        put(2, vsplat<V>(T(0)));
      } else {
        const V wb0 = vldg<V>(wb, off), o20 = vldg<V>(o2, off), o10 = vldg<V>(o1, off);
        put(0, c * (-vb0 * o30 + T(0.5) * (wbu * o2u + wb0 * o20)));
        put(1, c * (ub0 * o30 + T(0.5) * (wb0 * (-o10) + wbu * (-o1u))));
        put(2, c * T(0.5) * ((ub0 + vldg<V>(ub, dn)) * (-o20) + (vb0 + vldg<V>(vb, dn)) * o10));
      }
    } else if constexpr (OP == XF_PROD_SC) {
      // scalar advection on the fine grid, uvp level l: inputs ub, vb, wb
      // (padded -u, -v, -w), tx, ty (padded d theta/dx, dy, uvp nodes) and
      // tz (padded d theta/dz, w nodes): ub tx + vb ty + (wb tz at l, l+1)/2
      const T c = T(a.c0);
      const long up = off + a.in_pstride;
      const V r = vldg<V>(a.in[0], off) * vldg<V>(a.in[3], off) + vldg<V>(a.in[1], off) * vldg<V>(a.in[4], off) +
                  T(0.5) * (vldg<V>(a.in[2], off) * vldg<V>(a.in[5], off) + vldg<V>(a.in[2], up) * vldg<V>(a.in[5], up));
      put(0, c * r);
    } else if constexpr (OP == XF_PRESS_INC) {
      // u* = u^n + dt (t1 r + t2 r_f), so u* / (dt t1) = u^n / (dt t1) + r +
      // (t2/t1) r_f: the increment parts (inputs 0..5: rx ry rz rfx rfy rfz)
      // and the divergence of u^n (inputs 6..8: dudx dvdy dwdz, uvp nodes)
      // over dt t1 as a fourth field; c0 = 1/(nx ny), c1 = t2/t1,
      // c2 = 1/(dt t1).  Nothing large cancels in any of the four.
      const T c = T(a.c0), r21 = T(a.c1), idt = T(a.c2);
      put(0, c * (vldg<V>(a.in[0], off) + r21 * vldg<V>(a.in[3], off)));
      put(1, c * (vldg<V>(a.in[1], off) + r21 * vldg<V>(a.in[4], off)));
      put(2, c * (vldg<V>(a.in[2], off) + r21 * vldg<V>(a.in[5], off)));
      put(3, (c * idt) * ((vldg<V>(a.in[6], off) + vldg<V>(a.in[7], off)) + vldg<V>(a.in[8], off)));
    } else if constexpr (OP == XF_SCDYN) {
      // dynamic Prandtl model on the nodes of compute_dynamic_mum
      // (compute_LagScaleDep.f90:501-520: level 1 on uvp nodes with w(2)/4,
      // levels >= 2 on w nodes).  Inputs: 0 u, 1 v, 2 w, 3 theta, 4..9 S_ij,
      // 10 |S|, 11 d theta/dx, 12 d theta/dy, 13 d theta/dz (w nodes).
      // Outputs: u, v, w, theta, u theta, v theta, w theta, S_ij (6),
      // d_j theta (3), |S| d_j theta (3).
      const long pl = a.in_pstride;
      auto at_w = [&](const T* f, long o) -> V {
        return l == 1 ? vldg<V>(f, o) : T(0.5) * (vldg<V>(f, o) + vldg<V>(f, o - pl));
      };
      V uf = at_w(a.in[0], off), vf = at_w(a.in[1], off), tf = at_w(a.in[3], off);
      V wf = l == 1 ? T(0.25) * vldg<V>(a.in[2], off + pl) : vldg<V>(a.in[2], off);
      if (a.fluct) {
        // K_j = filt(u_j theta) - filt(u_j) filt(theta) does not change when
        // per-level constants are removed from u_j and theta (the filter
        // keeps the mean); FP32 keeps the fluctuations
        const long o0 = (long)l * pl;
        auto at_w0 = [&](const T* f) -> T { return l == 1 ? f[o0] : T(0.5) * (f[o0] + f[o0 - pl]); };
        const T w0 = l == 1 ? T(0.25) * a.in[2][o0 + pl] : a.in[2][o0];
        uf = uf - vsplat<V>(at_w0(a.in[0]));
        vf = vf - vsplat<V>(at_w0(a.in[1]));
        tf = tf - vsplat<V>(at_w0(a.in[3]));
        wf = wf - vsplat<V>(w0);
      }
      put(0, uf);
      put(1, vf);
      put(2, wf);
      put(3, tf);
      put(4, uf * tf);
      put(5, vf * tf);
      put(6, wf * tf);
#pragma unroll
      for (int q = 0; q < 6; ++q) put(7 + q, vldg<V>(a.in[4 + q], off));
      const V S = vldg<V>(a.in[10], off);
      const V tx = at_w(a.in[11], off), ty = at_w(a.in[12], off), tz = vldg<V>(a.in[13], off);
      put(13, tx);
      put(14, ty);
      put(15, tz);
      put(16, S * tx);
      put(17, S * ty);
      put(18, S * tz);
    } else if constexpr (OP == XF_LASD) {
      // compute_LagScaleDep.f90:501-584: u_ft, A_ij, S_ij, |S| S_ij
      const T* u = a.in[0];
      const T* vv = a.in[1];
      const T* w = a.in[2];
      V uf, vf, wf;
      if (l == 1) {
        uf = vldg<V>(u, off);
        vf = vldg<V>(vv, off);
        wf = T(0.25) * vldg<V>(w, off + a.in_pstride);
      } else {
        const long dn = off - a.in_pstride;
        uf = T(0.5) * (vldg<V>(u, off) + vldg<V>(u, dn));
        vf = T(0.5) * (vldg<V>(vv, off) + vldg<V>(vv, dn));
        wf = vldg<V>(w, off);
      }
      if (a.fluct) {
        // L_ij = filt(u_i u_j) - filt(u_i) filt(u_j) is unchanged when a
        // per-level constant is removed from u_i; FP32 keeps the fluctuation.
        const long o0 = (long)l * a.in_pstride;
        T u0, v0, w0;
        if (l == 1) {
          u0 = u[o0];
          v0 = vv[o0];
          w0 = T(0.25) * w[o0 + a.in_pstride];
        } else {
          u0 = T(0.5) * (u[o0] + u[o0 - a.in_pstride]);
          v0 = T(0.5) * (vv[o0] + vv[o0 - a.in_pstride]);
          w0 = w[o0];
        }
        uf = uf - vsplat<V>(u0);
        vf = vf - vsplat<V>(v0);
        wf = wf - vsplat<V>(w0);
      }
      put(0, uf);
      put(1, vf);
      put(2, wf);
      put(3, uf * uf);  // A11
      put(4, uf * vf);  // A12
      put(5, uf * wf);  // A13
      put(6, vf * vf);  // A22
      put(7, vf * wf);  // A23
      put(8, wf * wf);  // A33
      const V S = vldg<V>(a.in[9], off);
#pragma unroll
      for (int q = 0; q < 6; ++q) {  // s11 s12 s13 s22 s23 s33
        const V sq = vldg<V>(a.in[3 + q], off);
        put(9 + q, sq);
        put(15 + q, S * sq);
      }
    }
  }
}

// the same with the op chosen at run time (the per-row references)
template <typename T, typename V>
__device__ __forceinline__ void xf_load(const XFArgs<T>& a, int l, int j, int i, T* v, int vs) {
  switch (a.op) {
    case XF_SCALE: xf_load_op<T, V, XF_SCALE, false>(a, l, j, i, v, vs, nullptr); break;
    case XF_CONV_IN: xf_load_op<T, V, XF_CONV_IN, false>(a, l, j, i, v, vs, nullptr); break;
    case XF_PROD: xf_load_op<T, V, XF_PROD, false>(a, l, j, i, v, vs, nullptr); break;
    case XF_LASD: xf_load_op<T, V, XF_LASD, false>(a, l, j, i, v, vs, nullptr); break;
    case XF_PRESS: xf_load_op<T, V, XF_PRESS, false>(a, l, j, i, v, vs, nullptr); break;
    case XF_PROD_SC: xf_load_op<T, V, XF_PROD_SC, false>(a, l, j, i, v, vs, nullptr); break;
    case XF_SCDYN: xf_load_op<T, V, XF_SCDYN, false>(a, l, j, i, v, vs, nullptr); break;
    case XF_PRESS_INC: xf_load_op<T, V, XF_PRESS_INC, false>(a, l, j, i, v, vs, nullptr); break;
    default: break;
  }
}

// number of sequence slots in an x pass: rounded up to whole warps
template <int M>
__host__ __device__ constexpr int seq_pad(int nseq) {
  constexpr int spw = 32 / Geo<M>::T;  // sequences per warp
  return ((nseq + spw - 1) / spw) * spw;
}

template <typename T, int NX>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? (NX <= 256 ? 4 : 3) : 2) k_xfwd(const XFArgs<T> a) {
  constexpr int M = NX / 2;
  constexpr int TL = Geo<M>::T;
  constexpr int E = Geo<M>::E;
  constexpr int RI = Layout<M, false>::in;
  constexpr int RO = Layout<M, false>::out;
  constexpr int SL = slot_stride(M, int(sizeof(cplx<T>)));  // complex values per sequence slot
  constexpr int XS = 2 * SL;         // the same slot viewed as reals
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twm = tw + NX;  // twiddle matrices of the M-point transform
  cplx<T>* buf = twm + Twm<M, false>::len;
  const int nseq = a.R * a.nf;
  const int npad = seq_pad<M>(nseq);
  T* refs = reinterpret_cast<T*>(buf + (long)npad * SL);  // R * nf per-row references
  int* rowl = reinterpret_cast<int*>(refs + a.R * a.nf);  // level of row r (-1: beyond the grid)
  int* rowj = rowl + a.R;
  for (int i = threadIdx.x; i < NX; i += blockDim.x) tw[i] = c_scl(a.tw[i], T(0.5));  // W^k / 2 for the split
  twm_build<T, M, false, 2>(a.tw, twm, threadIdx.x, blockDim.x);
  const long g0 = (long)blockIdx.x * a.R;
  for (int r = threadIdx.x; r < a.R; r += blockDim.x) {
    const long g = g0 + r;
    rowl[r] = (g < a.nrows) ? a.plane0 + udiv32(g, a.rows_pp) : -1;
    rowj[r] = (g < a.nrows) ? umod32(g, a.rows_pp) : 0;
  }
  __syncthreads();
  if (a.use_ref) {
    for (int r = threadIdx.x; r < a.R; r += blockDim.x) {
      const long g = g0 + r;
      if (g >= a.nrows) continue;
      const int l = a.plane0 + udiv32(g, a.rows_pp);
      const int j = umod32(g, a.rows_pp);
      xf_load<T, T>(a, l, 0, 0, refs + r * a.nf, 1);
      for (int f = 0; f < a.nf; ++f) {
        if (!a.refout[f]) refs[r * a.nf + f] = T(0);
        else if (j == 0) a.refout[f][l] = T(double(refs[r * a.nf + f]) * a.ref_mul);
      }
    }
    __syncthreads();
  }
  // load: four consecutive points per thread (16-byte accesses); sequence
  // s = r*nf + f holds the packed row z_m = x_{2m} + i x_{2m+1}, i.e. the
  // real row itself viewed as complex.
  T* xr = reinterpret_cast<T*>(buf);
  // the load loop is compiled per op and per reference mode (no dispatch
  // per point); references are subtracted in registers before the store
  auto load_rows = [&](auto op_c, auto ref_c) {
    constexpr int OP = decltype(op_c)::value;
    constexpr bool REF = decltype(ref_c)::value;
    for (int idx = threadIdx.x; idx < a.R * (NX / 4); idx += blockDim.x) {
      const int r = idx / (NX / 4);
      const int i = 4 * (idx - r * (NX / 4));
      T* dst = xr + (long)(r * a.nf) * XS + i;
      const int l = rowl[r];
      if (l >= 0) xf_load_op<T, V4<T>, OP, REF>(a, l, rowj[r], i, dst, XS, refs + r * a.nf);
      else
        for (int f = 0; f < a.nf; ++f) vst(dst + f * XS, vsplat<V4<T>>(T(0)));
    }
  };
  auto load_op = [&](auto op_c) {
    if (a.use_ref) load_rows(op_c, std::true_type{});
    else load_rows(op_c, std::false_type{});
  };
  switch (a.op) {
    case XF_SCALE: load_op(std::integral_constant<int, XF_SCALE>{}); break;
    case XF_CONV_IN: load_op(std::integral_constant<int, XF_CONV_IN>{}); break;
    case XF_PROD: load_op(std::integral_constant<int, XF_PROD>{}); break;
    case XF_LASD: load_op(std::integral_constant<int, XF_LASD>{}); break;
    case XF_PRESS: load_op(std::integral_constant<int, XF_PRESS>{}); break;
    case XF_PROD_SC: load_op(std::integral_constant<int, XF_PROD_SC>{}); break;
    case XF_SCDYN: load_op(std::integral_constant<int, XF_SCDYN>{}); break;
    case XF_PRESS_INC: load_op(std::integral_constant<int, XF_PRESS_INC>{}); break;
    default: break;
  }
  for (int idx = nseq * SL + threadIdx.x; idx < npad * SL; idx += blockDim.x) buf[idx] = cplx<T>{T(0), T(0)};
  __syncthreads();
  // complex FFT of length M per sequence in registers, then the r2c split
  const int lane_t = threadIdx.x % TL;
  for (int base = 0; base < npad; base += blockDim.x / TL) {
    const int s = base + threadIdx.x / TL;
    if (base + (threadIdx.x / 32) * (32 / TL) >= npad) break;  // whole warp beyond the slots
    cplx<T>* seq = buf + (long)s * SL;
    cplx<T> v[E];
#pragma unroll
    for (int g = 0; g < E / RI; ++g)
#pragma unroll
      for (int r = 0; r < RI; ++r) v[g * RI + r] = seq[lane_t + TL * g + r * (M / RI)];
    reg_fft<T, M, false>(v, seq, lane_t, twm);
    __syncwarp();
#pragma unroll
    for (int g = 0; g < E / RO; ++g)
#pragma unroll
      for (int r = 0; r < RO; ++r) seq[lane_t + TL * g + r * (M / RO)] = v[g * RO + r];
    __syncwarp();
    if (s < nseq) {
      const int r = udiv32(s, a.nf);
      const int f = s - r * a.nf;
      const int l = rowl[r];
      if (l >= 0) {
        const int j = rowj[r];
        cplx<T>* orow = a.out[f] + (long)l * a.out_pstride + (long)j * a.opitch;
        xf_split_store<T, M, TL, E>(seq, tw, orow, lane_t, a.nk);
      }
    }
  }
}

// Values of the staged ops at level l, columns i..i+3 of row r, from the
// staged input rows (rows[q] = source q of this grid row).
template <typename T, typename S>
__device__ __forceinline__ void xf_load_st(const XFArgs<T>& a, int l, const S* const* rows, int i, T* v, int vs) {
  using V = V4<T>;
  auto ld = [&](int q) { return vld<V>(rows[q], (long)i); };
  switch (a.op) {
    case XF_SCALE:
      for (int f = 0; f < a.nf; ++f) vst(v + f * vs, T(a.c0) * ld(f));
      break;
    case XF_PRESS:  // compute_pressure.f90:138-140
      for (int f = 0; f < a.nf; ++f) vst(v + f * vs, T(a.c0) * (ld(f) / T(a.c1)));
      break;
    case XF_CONV_IN: {
      // compute_convective_padd.f90:133-165; sources 0..8 = the inputs at
      // level l, 9 / 10 = dwdy / dwdx at l + 1 (wall row only)
      const T c = T(a.c0);
      vst(v + 0 * vs, -c * ld(0));
      vst(v + 1 * vs, -c * ld(1));
      vst(v + 2 * vs, -c * ld(2));
      if (a.wall && l == 0) {
        vst(v + 3 * vs, vsplat<V>(T(0)));
        vst(v + 4 * vs, vsplat<V>(T(0)));
      } else if (a.wall && l == 1) {
        vst(v + 3 * vs, c * (T(0.5) * (ld(3) + ld(9)) - ld(4)));
        vst(v + 4 * vs, c * (ld(5) - T(0.5) * (ld(6) + ld(10))));
      } else {
        vst(v + 3 * vs, c * (ld(3) - ld(4)));
        vst(v + 4 * vs, c * (ld(5) - ld(6)));
      }
      vst(v + 5 * vs, c * (ld(7) - ld(8)));
      break;
    }
    default:
      break;
  }
}

// start the copies of the staged input rows of batch `item` (one warp per
// row, 16-byte pieces)
template <typename T, typename S, int NX>
__device__ __forceinline__ void xf_issue(const XFArgs<T>& a, long item, S* stage) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  constexpr int PIECES = NX * int(sizeof(S)) / 16;
  const int nrow = a.R * a.nsrc;
  for (int s = warp; s < nrow; s += nwarps) {
    const int r = udiv32(s, a.nsrc);
    const int q = s - r * a.nsrc;
    const long g = item * a.R + r;
    const int l = a.plane0 + udiv32(g, a.rows_pp);
    const bool valid = g < a.nrows && (!a.scond[q] || (a.wall && l == 1));
    const S* base = reinterpret_cast<const S*>(std::is_same<S, T>::value ? (const void*)a.in[a.sf[q]]
                                                                          : (const void*)a.inf[a.sf[q]]);
    const S* row = valid ? base + (long)(l + a.sdl[q]) * a.in_pstride + long(umod32(g, a.rows_pp)) * a.in_rstride : base;
    S* dst = stage + (long)s * NX;
    for (int k = lane; k < PIECES; k += 32)
      cp_async<16>(reinterpret_cast<unsigned char*>(dst) + 16 * k,
                   valid ? reinterpret_cast<const unsigned char*>(row) + 16 * k
                         : reinterpret_cast<const unsigned char*>(base),
                   valid);
  }
}

// The x forward pass for the ops whose inputs are whole rows (scale,
// pressure input, convective inputs): persistent CTAs over batches of R rows,
// the input rows of the next batch copied into the other shared stage with
// cp.async while the current batch is transformed.  S: input element type.
template <typename T, int NX, typename S>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? (NX <= 256 ? 4 : 3) : 2) k_xfwd_st(const XFArgs<T> a) {
  constexpr int M = NX / 2;
  constexpr int TL = Geo<M>::T;
  constexpr int E = Geo<M>::E;
  constexpr int RI = Layout<M, false>::in;
  constexpr int RO = Layout<M, false>::out;
  constexpr int SL = slot_stride(M, int(sizeof(cplx<T>)));
  constexpr int XS = 2 * SL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twm = tw + NX;  // twiddle matrices of the M-point transform
  const int nseq = a.R * a.nf;
  const int npad = seq_pad<M>(nseq);
  S* stage0 = reinterpret_cast<S*>(twm + Twm<M, false>::len);
  S* stage1 = stage0 + (long)a.R * a.nsrc * NX;
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(stage1 + (long)a.R * a.nsrc * NX);
  T* refs = reinterpret_cast<T*>(buf + (long)npad * SL);
  int* rowl = reinterpret_cast<int*>(refs + a.R * a.nf);
  int* rowj = rowl + a.R;
  for (int i = threadIdx.x; i < NX; i += blockDim.x) tw[i] = c_scl(a.tw[i], T(0.5));  // W^k / 2 for the split
  twm_build<T, M, false, 2>(a.tw, twm, threadIdx.x, blockDim.x);
  const long nitems = (a.nrows + a.R - 1) / a.R;
  if ((long)blockIdx.x < nitems) {
    xf_issue<T, S, NX>(a, blockIdx.x, stage0);
    cp_async_commit();
  }
  int stg = 0;
  for (long item = blockIdx.x; item < nitems; item += gridDim.x) {
    const long next = item + gridDim.x;
    const S* stage = stg ? stage1 : stage0;
    if (next < nitems) {
      xf_issue<T, S, NX>(a, next, stg ? stage0 : stage1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    const long g0 = item * a.R;
    for (int r = threadIdx.x; r < a.R; r += blockDim.x) {
      const long g = g0 + r;
      rowl[r] = (g < a.nrows) ? a.plane0 + udiv32(g, a.rows_pp) : -1;
      rowj[r] = (g < a.nrows) ? umod32(g, a.rows_pp) : 0;
    }
    __syncthreads();
    if (a.use_ref) {  // per-level references: the (0,0) value of each field (from global)
      for (int r = threadIdx.x; r < a.R; r += blockDim.x) {
        const int l = rowl[r];
        if (l < 0) continue;
        xf_load<T, T>(a, l, 0, 0, refs + r * a.nf, 1);
        for (int f = 0; f < a.nf; ++f) {
          if (!a.refout[f]) refs[r * a.nf + f] = T(0);
          else if (rowj[r] == 0) a.refout[f][l] = T(double(refs[r * a.nf + f]) * a.ref_mul);
        }
      }
      __syncthreads();
    }
    T* xr = reinterpret_cast<T*>(buf);
    for (int idx = threadIdx.x; idx < a.R * (NX / 4); idx += blockDim.x) {
      const int r = idx / (NX / 4);
      const int i = 4 * (idx - r * (NX / 4));
      T* dst = xr + (long)(r * a.nf) * XS + i;
      const int l = rowl[r];
      if (l >= 0) {
        const S* rows[16];
        for (int q = 0; q < a.nsrc; ++q) rows[q] = stage + (long)(r * a.nsrc + q) * NX;
        xf_load_st<T, S>(a, l, rows, i, dst, XS);
        if (a.use_ref)
          for (int f = 0; f < a.nf; ++f) {
            const T rf = refs[r * a.nf + f];
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[f * XS + q] -= rf;
          }
      } else {
        for (int f = 0; f < a.nf; ++f) vst(dst + f * XS, vsplat<V4<T>>(T(0)));
      }
    }
    for (int idx = nseq * SL + threadIdx.x; idx < npad * SL; idx += blockDim.x) buf[idx] = cplx<T>{T(0), T(0)};
    __syncthreads();
    const int lane_t = threadIdx.x % TL;
    for (int base = 0; base < npad; base += blockDim.x / TL) {
      const int s = base + threadIdx.x / TL;
      if (base + (threadIdx.x / 32) * (32 / TL) >= npad) break;
      cplx<T>* seq = buf + (long)s * SL;
      cplx<T> v[E];
#pragma unroll
      for (int g = 0; g < E / RI; ++g)
#pragma unroll
        for (int r = 0; r < RI; ++r) v[g * RI + r] = seq[lane_t + TL * g + r * (M / RI)];
      reg_fft<T, M, false>(v, seq, lane_t, twm);
      __syncwarp();
#pragma unroll
      for (int g = 0; g < E / RO; ++g)
#pragma unroll
        for (int r = 0; r < RO; ++r) seq[lane_t + TL * g + r * (M / RO)] = v[g * RO + r];
      __syncwarp();
      if (s < nseq) {
        const int r = udiv32(s, a.nf);
        const int f = s - r * a.nf;
        const int l = rowl[r];
        if (l >= 0) {
          const int j = rowj[r];
          cplx<T>* orow = a.out[f] + (long)l * a.out_pstride + (long)j * a.opitch;
          xf_split_store<T, M, TL, E>(seq, tw, orow, lane_t, a.nk);
        }
      }
    }
    __syncthreads();
    stg ^= 1;
  }
}

// --------------------------------------------------------------- ypass ----
enum YPOp : int {
  YP_GRAD = 0,     // f -> f, i kx f, i ky f           (Nyquist killed)
  YP_DIV2 = 1,     // (fx, fy) -> i kx fx + i ky fy     (Nyquist killed)
  YP_FWDKILL = 2,  // f -> f, no inverse y transform    (Nyquist killed)
  YP_PGRAD = 3,    // p^ (already y-spectral) -> i kx p, i ky p, p
  YP_FILTER2 = 4,  // f -> G0 f, G1 f
  YP_PAD = 5,      // ny -> 3ny/2 zero padding (ky Nyquist dropped)
  YP_TRUNC = 6,    // 3ny/2 -> ny truncation (ky Nyquist zeroed)
  YP_MASK = 7,     // keep |ky| <= tt (2/3-rule truncation)
  YP_FILTER1 = 8,  // f -> G0 f
  YP_GRADY = 9,    // f -> f, i ky f                    (Nyquist killed; i kx f in the x inverse)
};

template <typename T>
struct YPArgs {
  int op, nin, nout, C, lc;  // C = 1 << lc columns per CTA
  int SI;                    // column stride of the shared stages (>= both lengths' slots)
  int ncols;           // columns processed
  int ncols1;          // columns stored for the second FILTER2 output
  int nk_in, nk_out, nk_out1;
  int ipitch, opitch, opitch1;  // complex values between rows of in / out / second out (0: the nk)
  int nplanes, ngroups;         // work items: column blocks x planes x groups
  int plane0;
  int nstage;  // input stages (set by the launcher): 2 = the next item's columns load during this one
  long in_pstride, out_pstride, out_pstride1;
  int nxh, lhx;        // base-grid Nyquist column and row length of kkx/kky/G
  int tt;              // YP_MASK: largest |ky| kept
  const cplx<T>* in[MAXIN];
  cplx<T>* out[MAXOUT];
  const T* kkx;        // [ny][lhx]
  const T* kky;
  const T* G0;         // [ny][lhx] filter kernels (include 1/(nx ny))
  const T* G1;
  const cplx<T>* tw_in;   // length NY table
  const cplx<T>* tw_out;  // length NYO table
};

// Elementwise spectral op at (kx, ky) for output q; F0/F1 are the forward
// transforms of the (up to two) input fields at that point.
template <typename T, int NY>
__device__ __forceinline__ cplx<T> yp_op(const YPArgs<T>& a, int q, int kx, int ky, cplx<T> F0, cplx<T> F1) {
  const cplx<T> zero = {T(0), T(0)};
  switch (a.op) {
    case YP_GRAD: {
      if (ky == NY / 2 || kx == a.nxh) return zero;
      if (q == 0) return F0;
      if (q == 1) return ik_mul(a.kkx[ky * a.lhx + kx], F0);
      return ik_mul(a.kky[ky * a.lhx + kx], F0);
    }
    case YP_GRADY: {
      if (ky == NY / 2 || kx == a.nxh) return zero;
      if (q == 0) return F0;
      return ik_mul(a.kky[ky * a.lhx + kx], F0);
    }
    case YP_DIV2: {
      if (ky == NY / 2 || kx == a.nxh) return zero;
      return c_add(ik_mul(a.kkx[ky * a.lhx + kx], F0), ik_mul(a.kky[ky * a.lhx + kx], F1));
    }
    case YP_FWDKILL:
      return (ky == NY / 2 || kx == a.nxh) ? zero : F0;
    case YP_PGRAD: {
      if (q == 0) return ik_mul(a.kkx[ky * a.lhx + kx], F0);
      if (q == 1) return ik_mul(a.kky[ky * a.lhx + kx], F0);
      return F0;
    }
    case YP_FILTER1:
    case YP_FILTER2: {
      const T g = (q == 0 ? a.G0 : a.G1)[ky * a.lhx + kx];
      return cplx<T>{F0.x * g, F0.y * g};
    }
    case YP_MASK:
      return (ky <= a.tt || ky >= NY - a.tt) ? F0 : zero;
    default:
      return F0;  // YP_PAD / YP_TRUNC: position remap only
  }
}

// yp_op for an op fixed at compile time, with the wavenumbers of the point
// given: kxv = kkx(kx) of the thread's column (row 0 of the table) and kyv =
// kky(ky) of the row (column 0).  The tables hold 2 pi / l times the wrapped
// index, zeroed on the Nyquist row / column only, so away from those the
// values are the table's; the kills below reproduce the zeros.
template <typename T, int NY, int OP>
__device__ __forceinline__ cplx<T> yp_op_c(const YPArgs<T>& a, int q, int kx, int ky, cplx<T> F0, T kxv, T kyv) {
  const cplx<T> zero = {T(0), T(0)};
  if constexpr (OP == YP_GRAD) {
    if (ky == NY / 2 || kx == a.nxh) return zero;
    if (q == 0) return F0;
    if (q == 1) return ik_mul(kxv, F0);
    return ik_mul(kyv, F0);
  } else if constexpr (OP == YP_GRADY) {
    if (ky == NY / 2 || kx == a.nxh) return zero;
    if (q == 0) return F0;
    return ik_mul(kyv, F0);
  } else {  // YP_PGRAD: no kill, the Nyquist row / column of the tables are zero
    if (q == 0) return ik_mul(ky == NY / 2 ? T(0) : kxv, F0);
    if (q == 1) return ik_mul(kx == a.nxh ? T(0) : kyv, F0);
    return F0;
  }
}

// y pass: start the copies of work item `item` (C columns x NY rows of every
// input field) into the shared stage `bin` ([nin][C][SI])
template <typename T, int NY>
__device__ __forceinline__ void yp_issue(const YPArgs<T>& a, long item, int ncb, cplx<T>* bin) {
  const int C = a.C, SI = a.SI;
  const int col0 = umod32(item, ncb) * C;
  const int l = a.plane0 + umod32(udiv32(item, ncb), a.nplanes);
  const int grp = udiv32(item, (long)ncb * a.nplanes);
  // thread -> fixed column c, rows ky0 + TL i: the CTA has C x TL threads,
  // so every thread copies NY / TL rows at a compile-time count and the
  // addresses advance by constant strides (an unrolled loop)
  constexpr int TL = Geo<NY>::T;
  const int c = threadIdx.x & (C - 1);
  const int ky0 = threadIdx.x >> a.lc;
  const int kx = col0 + c;
  const bool valid = kx < a.ncols;
  const long step = (long)TL * a.ipitch;
  for (int q = 0; q < a.nin; ++q) {
    const cplx<T>* base = a.in[grp * a.nin + q];
    const cplx<T>* src = valid ? base + (long)l * a.in_pstride + kx + (long)ky0 * a.ipitch : base;
    cplx<T>* dst = bin + (q * C + c) * SI + ky0;
#pragma unroll
    for (int i = 0; i < NY / TL; ++i)
      cp_async<int(sizeof(cplx<T>))>(dst + TL * i, valid ? src + i * step : base, valid);
  }
}

// FWD: forward transform only (YP_FWDKILL), compiled without the inverse so
// that it keeps fewer registers (more resident warps)
template <typename T, int NY, int NYO, bool FWD = false>
__global__ void __launch_bounds__((FWD && sizeof(T) == 8) ? 128 : 256,
                                  (FWD && sizeof(T) == 8) ? 3 : (sizeof(T) == 4 ? 2 : 1))
    k_ypass(const YPArgs<T> a) {
  constexpr int TL = Geo<NY>::T;
  static_assert(Geo<NYO>::T == TL, "pad/truncate pairs must share the lanes per sequence");
  constexpr int EI = Geo<NY>::E;
  constexpr int EO = Geo<NYO>::E;
  constexpr int FI = Layout<NY, false>::in;    // forward input groups
  constexpr int FO = Layout<NY, false>::out;   // forward output groups
  constexpr int II = Layout<NYO, true>::in;    // inverse input groups
  constexpr int IO = Layout<NYO, true>::out;   // inverse output groups
  constexpr bool SAME = (NY == NYO);
  static_assert(!SAME || FO == II, "forward output layout must feed the inverse");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* twi = reinterpret_cast<cplx<T>*>(smem_raw);  // twiddle matrices, forward NY
  cplx<T>* two = twi + Twm<NY, false>::len;                 // and inverse NYO
  const int SI = a.SI;  // >= the slots of NY and NYO
  const int C = a.C;
  T* kyrow = reinterpret_cast<T*>(two + Twm<NYO, true>::len);  // kky(ky), column 0 of the table
  cplx<T>* bin0 = reinterpret_cast<cplx<T>*>(kyrow + ((NY + 3) & ~3));  // input stage 0: [nin][C][SI]
  cplx<T>* bin1 = bin0 + (a.nstage > 1 ? a.nin * C * SI : 0);  // input stage 1 (stage 0 again when single)
  // the inverse transform, its output layout and the coalesced copy-out use
  // the first input row of each column of the current stage, free once the
  // forward transforms hold their values in registers
  static_assert(!FWD || NY == NYO, "forward-only y passes keep the length");
  twm_build<T, NY, false>(a.tw_in, twi, threadIdx.x, blockDim.x);
  if constexpr (!FWD) twm_build<T, NYO, true>(a.tw_out, two, threadIdx.x, blockDim.x);
  if (a.kky)
    for (int i = threadIdx.x; i < NY; i += blockDim.x) kyrow[i] = a.kky[(long)i * a.lhx];
  // persistent CTAs: work item = (column block, plane, group); with two
  // stages the columns of the next item are copied into the other input
  // stage asynchronously while this one is transformed, with one stage they
  // are copied after this item's last read of it (more resident CTAs where
  // shared memory limits them)
  const int ncb = (a.ncols + C - 1) / C;
  const long nitems = (long)ncb * a.nplanes * a.ngroups;
  if ((long)blockIdx.x < nitems) {
    yp_issue<T, NY>(a, blockIdx.x, ncb, bin0);
    cp_async_commit();
  }
  int stage = 0;
  for (long item = blockIdx.x; item < nitems; item += gridDim.x) {
  const long next = item + gridDim.x;
  cplx<T>* bin = stage ? bin1 : bin0;
  if (a.nstage > 1 && next < nitems) {
    yp_issue<T, NY>(a, next, ncb, stage ? bin0 : bin1);
    cp_async_commit();
    cp_async_wait<1>();
  } else {
    cp_async_wait<0>();
  }
  __syncthreads();
  const int col0 = umod32(item, ncb) * C;
  const int l = a.plane0 + umod32(udiv32(item, ncb), a.nplanes);
  const int grp = udiv32(item, (long)ncb * a.nplanes);
  const int c = threadIdx.x / TL;
  const int lt = threadIdx.x % TL;
  const int kx = col0 + c;
  // forward transform in registers; the stress divergence folds its second
  // input into w = i kx F0 + i ky F1 before the output loop
  cplx<T> f0[EI];
  cplx<T> w[EO];
  {
    cplx<T>* seq = bin + c * SI;
    if (a.op == YP_PGRAD) {
      // input is already y-spectral: load it in the inverse input layout
#pragma unroll
      for (int g = 0; g < EI / II; ++g)
#pragma unroll
        for (int r = 0; r < II; ++r) f0[g * II + r] = seq[lt + TL * g + r * (NY / II)];
    } else {
#pragma unroll
      for (int g = 0; g < EI / FI; ++g)
#pragma unroll
        for (int r = 0; r < FI; ++r) f0[g * FI + r] = seq[lt + TL * g + r * (NY / FI)];
      reg_fft<T, NY, false>(f0, seq, lt, twi);
      if constexpr (SAME) {
        if (a.op == YP_DIV2) {
          const cplx<T> zero = {T(0), T(0)};
#pragma unroll
          for (int g = 0; g < EI / FO; ++g)
#pragma unroll
            for (int r = 0; r < FO; ++r) {
              const int ky = lt + TL * g + r * (NY / FO);
              const bool kill = (ky == NY / 2) || (kx == a.nxh) || (kx >= a.ncols);
              w[g * FO + r] = kill ? zero : ik_mul(a.kkx[kx], f0[g * FO + r]);
            }
          cplx<T>* seq1 = bin + (C + c) * SI;
#pragma unroll
          for (int g = 0; g < EI / FI; ++g)
#pragma unroll
            for (int r = 0; r < FI; ++r) f0[g * FI + r] = seq1[lt + TL * g + r * (NY / FI)];
          reg_fft<T, NY, false>(f0, seq1, lt, twi);
#pragma unroll
          for (int g = 0; g < EI / FO; ++g)
#pragma unroll
            for (int r = 0; r < FO; ++r) {
              const int ky = lt + TL * g + r * (NY / FO);
              const bool kill = (ky == NY / 2) || (kx == a.nxh) || (kx >= a.ncols);
              if (!kill) w[g * FO + r] = c_add(w[g * FO + r], ik_mul(kyrow[ky], f0[g * FO + r]));
            }
        }
      }
    }
  }
  __syncwarp();  // the column's forward reads are done before its slot is rewritten
  cplx<T>* sout = bin + c * SI;
  for (int q = 0; q < a.nout; ++q) {
    if constexpr (SAME) {
      // forward output layout (groups FO) == inverse input layout; the
      // stress divergence already holds its result in w
      if constexpr (FWD) {
        // YP_FWDKILL: the killed forward output goes straight to the slot in
        // the forward output layout (groups FO)
#pragma unroll
        for (int g = 0; g < EI / FO; ++g)
#pragma unroll
          for (int r = 0; r < FO; ++r) {
            const int ky = lt + TL * g + r * (NY / FO);
            const bool kill = (ky == NY / 2) || (kx == a.nxh) || (kx >= a.ncols);
            sout[lt + TL * g + r * (NYO / FO)] = kill ? cplx<T>{T(0), T(0)} : f0[g * FO + r];
          }
      } else if (a.op != YP_DIV2) {
        // the derivative ops with the op fixed per loop (no per-element
        // dispatch) and the wavenumbers from registers / shared memory
        const T kxv = (kx < a.ncols && a.kkx) ? a.kkx[kx] : T(0);
        auto fill = [&](auto opc) {
          constexpr int OP = decltype(opc)::value;
#pragma unroll
          for (int g = 0; g < EI / FO; ++g)
#pragma unroll
            for (int r = 0; r < FO; ++r) {
              const int ky = lt + TL * g + r * (NY / FO);
              w[g * FO + r] = (kx < a.ncols) ? yp_op_c<T, NY, OP>(a, q, kx, ky, f0[g * FO + r], kxv, kyrow[ky])
                                             : cplx<T>{T(0), T(0)};
            }
        };
        if (a.op == YP_GRADY) {
          fill(std::integral_constant<int, YP_GRADY>{});
        } else if (a.op == YP_GRAD) {
          fill(std::integral_constant<int, YP_GRAD>{});
        } else if (a.op == YP_PGRAD) {
          fill(std::integral_constant<int, YP_PGRAD>{});
        } else {
#pragma unroll
          for (int g = 0; g < EI / FO; ++g)
#pragma unroll
            for (int r = 0; r < FO; ++r) {
              const int ky = lt + TL * g + r * (NY / FO);
              w[g * FO + r] = (kx < a.ncols) ? yp_op<T, NY>(a, q, kx, ky, f0[g * FO + r], f0[g * FO + r])
                                             : cplx<T>{T(0), T(0)};
            }
        }
      }
    } else {
      // 3/2 pad or truncate.  Lane lt holds the forward output at ky = lt +
      // TL m (m < EI) and the inverse wants ko = lt + TL m' (m' < EO); pad
      // and truncation map ky to ko by a shift of whole multiples of TL, so
      // the remap stays in the lane: a permutation of registers with zeros.
      // PAD: ko = ky (ky < NY/2), ky + NY/2 (ky > NY/2), ky = NY/2 dropped;
      // TRUNC: ko = ky (ky < NYO/2), ky - NYO/2 (ky > NYO), ky = NYO dropped.
      constexpr int GI = EI / FO;  // forward output: f0[g FO + r] holds m = g + r GI
      constexpr int GO = EO / II;  // inverse input: w[g II + r] wants m' = g + r GO
      const bool live = kx < a.ncols;
      static_for<EO>([&](auto mc) {
        constexpr int mo = decltype(mc)::value;
        constexpr int wi = (mo % GO) * II + mo / GO;
        constexpr bool PAD = NYO > NY;
        // source m of output m' (-1: zero), and whether lane 0 drops it
        constexpr int ms = PAD ? (mo < EI / 2 ? mo : (mo < EI ? -1 : mo - EI / 2))
                               : (mo < EO / 2 ? mo : mo + EO / 2);
        constexpr bool drop0 = PAD ? (mo == EI) : (mo == EO / 2);
        if constexpr (ms < 0) {
          w[wi] = cplx<T>{T(0), T(0)};
        } else {
          constexpr int fi = (ms % GI) * FO + ms / GI;
          const bool keep = live && !(drop0 && lt == 0);
          w[wi] = keep ? f0[fi] : cplx<T>{T(0), T(0)};
        }
      });
    }
    if constexpr (FWD) {
      // no inverse: stored above
    } else {
      reg_fft<T, NYO, true>(w, sout, lt, two);
      __syncwarp();
#pragma unroll
      for (int g = 0; g < EO / IO; ++g)
#pragma unroll
        for (int r = 0; r < IO; ++r) sout[lt + TL * g + r * (NYO / IO)] = w[g * IO + r];
    }
    __syncthreads();
    // coalesced store of output q
    const bool second = (a.op == YP_FILTER2 && q == 1);
    const int lim = second ? a.ncols1 : a.ncols;
    {
      // thread -> fixed column cc, rows ky0 + TL i (as in yp_issue)
      const int cc = threadIdx.x & (C - 1);
      const int kxx = col0 + cc;
      if (kxx < lim) {
        const int ky0 = threadIdx.x >> a.lc;
        const long opitch = second ? a.opitch1 : a.opitch;
        cplx<T>* dst = a.out[grp * a.nout + q] + (long)l * (second ? a.out_pstride1 : a.out_pstride) + kxx +
                       (long)ky0 * opitch;
        const cplx<T>* srow = bin + cc * SI + ky0;
        const long step = (long)TL * opitch;
#pragma unroll
        for (int i = 0; i < NYO / TL; ++i) dst[i * step] = srow[TL * i];
      }
    }
    __syncthreads();
  }
  if (a.nstage > 1) {
    stage ^= 1;
  } else if (next < nitems) {
    // single stage: every thread is past the last read of it (barrier above)
    yp_issue<T, NY>(a, next, ncb, bin0);
    cp_async_commit();
  }
  }
}

// ---------------------------------------------------------------- xinv ----
enum XIOp : int {
  XI_STORE = 0,  // out[f](l) = x_f for lo[f] <= l <= hi[f]
  XI_DIV = 2,    // rhs += x + dz(tz) + pf ; pressure-BC layers of the w equation
  XI_LASD = 3,   // 21 filtered fields -> L:M and M:M
  XI_WALL = 4,   // filtered u1, v1 -> u*, Neumann ghost value, wall stress
  XI_SCDYN = 5,  // 19 filtered fields of the dynamic Prandtl model -> K.X and X.X
};

template <typename T>
struct XIArgs {
  int op, nin, R;
  long nrows;
  int rows_pp;
  int plane0;
  int nk;          // modes present in the input rows (rest zero)
  int ipitch;      // complex values between input rows (>= nk; 0: nk)
  int nks;         // complex values between staged rows in shared memory (set by the launcher)
  int stage_rows;  // staged rows per stage (set by the launcher)
  int nbuf;        // input stages (set by the launcher): 2 = the next item's rows load during this one
  int merged;      // 1: each sequence is transformed in its own staged row (plain store, nstage 0)
  int nz;
  long in_pstride;
  long out_pstride;  // elements per plane of the output grid
  double c0, c1, c2, c3;
  double pf[4];
  int lo[MAXIN], hi[MAXIN];
  const cplx<T>* in[MAXIN];
  const T* refin[MAXIN];  // per-level values added back to input field f
  T* out[16];
  float* outf[16];  // FP32 outputs of an FP64 transform (out_f32 = 1, XI_STORE)
  int out_f32;
  const T* aux[8];
  const cplx<T>* tw;  // exp(-2 pi i m / NX), m < NX
  // several transforms of one staged row: nstage rows per grid row are
  // staged (0: nin); transform f reads staged row src[f] and, with dx[f],
  // multiplies it by i kx (kxr[m], the x wavenumbers, Nyquist zero) first
  int nstage;
  int src[MAXIN];
  int dx[MAXIN];
  const T* kxr;
  // set by the launcher: every output (and the plane stride) admits stores of
  // whole (x_2m, x_2m+1) pairs
  int pair_store;
  // set by the launcher: stage the spectral rows with bulk copies (every
  // input and stage row 16-byte aligned); else per-thread cp.async copies
  int bulk;
  unsigned* status;  // device status word (ST_COPY_WAIT), may be null
};

// x inverse pass: start the copies of the spectral rows of batch `item`
// (R rows x nin fields, nk values each) into the shared stage
template <typename T>
__device__ __forceinline__ void xi_issue(const XIArgs<T>& a, long item, cplx<T>* stage) {
  // one warp per row: the row address is formed once, the lanes copy its
  // nk values
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int ns = a.nstage ? a.nstage : a.nin;
  const int nrow = a.R * ns;
  for (int s = warp; s < nrow; s += nwarps) {
    const int r = s / ns;
    const int f = s - r * ns;
    const long g = item * a.R + r;
    const bool valid = g < a.nrows;
    const cplx<T>* base = a.in[f];
    const cplx<T>* row =
        valid ? base + (long)(a.plane0 + udiv32(g, a.rows_pp)) * a.in_pstride + long(umod32(g, a.rows_pp)) * a.ipitch : base;
    cplx<T>* dst = stage + (long)s * a.nks;
    for (int m = lane; m < a.nk; m += 32) cp_async<int(sizeof(cplx<T>))>(dst + m, valid ? row + m : base, valid);
  }
}

// the same with bulk copies, issued by warp 0: lane 0 announces the bytes
// of every valid row's aligned part, then each lane copies whole rows; a
// row whose addresses are not 16-byte aligned (none when the launcher set
// a.bulk) and the last value of an odd FP32 row go by plain loads and stores
// (visible after the barrier that follows the wait)
template <typename T>
__device__ __forceinline__ void xi_issue_bulk(const XIArgs<T>& a, long item, cplx<T>* stage, uint64_t* mbar) {
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  const int ns = a.nstage ? a.nstage : a.nin;
  const long rows_left = a.nrows - item * a.R;
  const int nvalid = int(rows_left < a.R ? rows_left : a.R);
  const unsigned rb = unsigned(a.nk * sizeof(cplx<T>));
  const unsigned rbulk = rb & ~15u;
  auto aligned = [&](int s) {
    const int r = udiv32(s, ns), f = s - r * ns;
    const long g = item * a.R + r;
    const cplx<T>* row = a.in[f] + (long)(a.plane0 + udiv32(g, a.rows_pp)) * a.in_pstride +
                         long(umod32(g, a.rows_pp)) * a.ipitch;
    const cplx<T>* dst = stage + (long)s * a.nks;
    return ((reinterpret_cast<uintptr_t>(row) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0;
  };
  const int nrow = nvalid * ns;
  unsigned mine = 0;
  for (int s = lane; s < nrow; s += 32)
    if (rbulk && aligned(s)) mine += rbulk;
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  // the barrier's one arrival carries every byte the copies below bring (an
  // item always has a valid row, so the phase completes)
  if (lane == 0) mbar_expect_tx(mbar, mine);
  __syncwarp();
  tc::fence_async_smem();  // earlier generic reads of this stage come first
  for (int s = lane; s < nrow; s += 32) {
    const int r = udiv32(s, ns), f = s - r * ns;
    const long g = item * a.R + r;
    const cplx<T>* row = a.in[f] + (long)(a.plane0 + udiv32(g, a.rows_pp)) * a.in_pstride +
                         long(umod32(g, a.rows_pp)) * a.ipitch;
    cplx<T>* dst = stage + (long)s * a.nks;
    int m0 = 0;
    if (rbulk && aligned(s)) {
      bulk_g2s(dst, row, rbulk, mbar);
      m0 = int(rbulk / sizeof(cplx<T>));
    }
    for (int m = m0; m < a.nk; ++m) dst[m] = row[m];
  }
}

template <typename T, int NX>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? (NX <= 256 ? 4 : 3) : 2) k_xinv(const XIArgs<T> a) {
  constexpr int M = NX / 2;
  constexpr int TL = Geo<M>::T;
  constexpr int E = Geo<M>::E;
  constexpr int RI = Layout<M, true>::in;
  constexpr int RO = Layout<M, true>::out;
  constexpr int SL = slot_stride(M, int(sizeof(cplx<T>)));  // complex values per sequence slot
  constexpr int XS = 2 * SL;         // the same slot viewed as reals
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twm = tw + NX;  // twiddle matrices of the M-point inverse transform
  const int nseq = a.R * a.nin;
  const int npad = seq_pad<M>(nseq);
  const int ns = a.nstage ? a.nstage : a.nin;        // staged rows per grid row
  // a stage holds an even number of complex values, so the sequence slots
  // after the stages keep the 16-byte alignment of their four-point accesses
  // whatever the stage count (FP32 rows of an odd nks)
  const long stage_len = ((long)a.stage_rows * a.nks + 1) & ~1L;
  cplx<T>* stage0 = twm + Twm<M, true>::len;         // input rows of a work item: [R][ns][nk]
  cplx<T>* stage1 = stage0 + (a.nbuf > 1 ? stage_len : 0L);  // stage 0 again when single
  cplx<T>* buf = stage0 + a.nbuf * stage_len;        // sequence slots (none when merged)
  int* rowl = reinterpret_cast<int*>(buf + (a.merged ? 0L : (long)npad * SL));  // level of row r (-1: beyond the grid)
  int* rowj = rowl + a.R;
  T* kxs = reinterpret_cast<T*>(rowj + a.R);          // x wavenumbers (nstage > 0)
  // one mbarrier per input stage (bulk staging)
  uint64_t* bars = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(kxs + (a.nstage ? a.nk + 2 : 0)) + 7) & ~uintptr_t(7));
  for (int i = threadIdx.x; i < NX; i += blockDim.x) tw[i] = a.tw[i];
  twm_build<T, M, true, 2>(a.tw, twm, threadIdx.x, blockDim.x);
  if (a.nstage)
    for (int i = threadIdx.x; i < a.nk; i += blockDim.x) kxs[i] = a.kxr[i];
  if (a.bulk) {
    if (threadIdx.x == 0) {
      tc::mbar_init(&bars[0], 1);
      tc::mbar_init(&bars[1], 1);
      tc::fence_mbar_init();
    }
    __syncthreads();
  }
  unsigned phase = 0;  // bit b: parity of the next completion of bars[b]
  // persistent CTAs over batches of R rows; with two stages the spectral
  // rows of the next batch are copied into the other stage while this one
  // is transformed, with one stage after this batch's last read of it
  const long nitems = (a.nrows + a.R - 1) / a.R;
  if ((long)blockIdx.x < nitems) {
    if (a.bulk) {
      xi_issue_bulk<T>(a, blockIdx.x, stage0, &bars[0]);
    } else {
      xi_issue<T>(a, blockIdx.x, stage0);
      cp_async_commit();
    }
  }
  int stg = 0;
  for (long item = blockIdx.x; item < nitems; item += gridDim.x) {
  const long next = item + gridDim.x;
  const cplx<T>* stage = stg ? stage1 : stage0;
  bool late = false;  // this thread's wait for the item's rows ran out
  if (a.bulk) {
    if (a.nbuf > 1 && next < nitems) xi_issue_bulk<T>(a, next, stg ? stage0 : stage1, &bars[stg ^ 1]);
    late = !tc::mbar_wait(&bars[stg], (phase >> stg) & 1u);
    phase ^= 1u << stg;
  } else if (a.nbuf > 1 && next < nitems) {
    xi_issue<T>(a, next, stg ? stage0 : stage1);
    cp_async_commit();
    cp_async_wait<1>();
  } else {
    cp_async_wait<0>();
  }
  const long g0 = item * a.R;
  for (int r = threadIdx.x; r < a.R; r += blockDim.x) {
    const long g = g0 + r;
    rowl[r] = (g < a.nrows) ? a.plane0 + udiv32(g, a.rows_pp) : -1;
    rowj[r] = (g < a.nrows) ? umod32(g, a.rows_pp) : 0;
  }
  if (__syncthreads_or(late)) {
    // the copies did not complete within the limit: record it, give the
    // copies in flight a last bounded wait (they write this CTA's shared
    // memory) and leave, every thread of the CTA together
    if (threadIdx.x == 0 && a.status) atomicOr(a.status, unsigned(ST_COPY_WAIT));
    tc::mbar_wait(&bars[stg], (phase >> stg) & 1u ^ 1u);
    if (a.nbuf > 1 && next < nitems) tc::mbar_wait(&bars[stg ^ 1], (phase >> (stg ^ 1)) & 1u);
    return;
  }
  // a plain store writes straight from registers; the other ops combine
  // fields per point through shared memory
  const bool direct = (a.op == XI_STORE);
  const int lane_t = threadIdx.x % TL;
  for (int base = 0; base < npad; base += blockDim.x / TL) {
    const int s = base + threadIdx.x / TL;
    if (base + (threadIdx.x / 32) * (32 / TL) >= npad) break;  // whole warp beyond the slots
    const int r = udiv32(s, a.nin);
    const int f = s - r * a.nin;
    const bool valid = (s < nseq) && (rowl[r < a.R ? r : 0] >= 0);
    int l = 0, j = 0;
    if (valid) {
      l = rowl[r];
      j = rowj[r];
    }
    // merged: the staged row of sequence s (staged rows are sequences) is its slot
    cplx<T>* seq = a.merged ? const_cast<cplx<T>*>(stage) + (long)s * a.nks : buf + (long)s * SL;
    // c2r split: Z_m = (X_m + conj X_{M-m}) + i W^{-m} (X_m - conj X_{M-m}),
    // imaginary parts of the DC and Nyquist bins ignored
    cplx<T> v[E];
    const int fs = a.nstage ? a.src[f] : f;
    const bool dxf = a.nstage && a.dx[f];
    const cplx<T>* row = valid ? stage + (long)(r * ns + fs) * a.nks : nullptr;  // the staged spectral row
    // The per-sequence choices (d/dx, whether every mode below M is present)
    // are made once here, not inside the unrolled element loop: with nk >= M
    // the partner X_{M-m} exists for every element but m = 0, which only the
    // first element of lane 0 can hold.
    auto split = [&](auto dx_c, auto full_c) {
      constexpr bool DX = decltype(dx_c)::value;
      constexpr bool FULL = decltype(full_c)::value;
#pragma unroll
      for (int gg = 0; gg < E / RI; ++gg)
#pragma unroll
        for (int rr = 0; rr < RI; ++rr) {
          const int m = lane_t + TL * gg + rr * (M / RI);
          const bool first = (gg == 0 && rr == 0);  // the only element that can hold m = 0
          cplx<T> xk, xm;
          if constexpr (FULL) {
            xk = row[m];
            xm = (first && m == 0 && a.nk == M) ? cplx<T>{T(0), T(0)} : row[M - m];
          } else {
            xk = (m < a.nk) ? row[m] : cplx<T>{T(0), T(0)};
            xm = (M - m < a.nk) ? row[M - m] : cplx<T>{T(0), T(0)};
          }
          if constexpr (DX) {  // d/dx: i kx X (compute_derivatives.f90:94-137)
            if constexpr (FULL) {
              xk = ik_mul(kxs[m], xk);
              if (!(first && m == 0 && a.nk == M)) xm = ik_mul(kxs[M - m], xm);
            } else {
              xk = (m < a.nk) ? ik_mul(kxs[m], xk) : xk;
              xm = (M - m < a.nk) ? ik_mul(kxs[M - m], xm) : xm;
            }
          }
          if (first && m == 0) {
            xk.y = T(0);
            xm.y = T(0);
          }
          v[gg * RI + rr] = c2r_split(xk, xm, tw[m]);
        }
    };
    if constexpr (sizeof(T) == 8) {
      // FP64: one generic loop (the specialised copies cost the double
      // precision kernels register spills at their 128-register budget)
#pragma unroll
      for (int gg = 0; gg < E / RI; ++gg)
#pragma unroll
        for (int rr = 0; rr < RI; ++rr) {
          const int m = lane_t + TL * gg + rr * (M / RI);
          cplx<T> z = {T(0), T(0)};
          if (valid) {
            cplx<T> xk = (m < a.nk) ? row[m] : cplx<T>{T(0), T(0)};
            cplx<T> xm = (M - m < a.nk) ? row[M - m] : cplx<T>{T(0), T(0)};
            if (dxf) {  // d/dx: i kx X (compute_derivatives.f90:94-137)
              xk = (m < a.nk) ? ik_mul(kxs[m], xk) : xk;
              xm = (M - m < a.nk) ? ik_mul(kxs[M - m], xm) : xm;
            }
            if (m == 0) {
              xk.y = T(0);
              xm.y = T(0);
            }
            z = c2r_split(xk, xm, tw[m]);
          }
          v[gg * RI + rr] = z;
        }
    } else if (!valid) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = cplx<T>{T(0), T(0)};
    } else if (a.nk >= M) {
      if (dxf) split(std::true_type{}, std::true_type{});
      else split(std::false_type{}, std::true_type{});
    } else {
      if (dxf) split(std::true_type{}, std::false_type{});
      else split(std::false_type{}, std::false_type{});
    }
    reg_fft<T, M, true>(v, seq, lane_t, twm);
    if (direct) {
      if (valid && l >= a.lo[f] && l <= a.hi[f]) {
        const T ref = a.refin[f] ? a.refin[f][l] : T(0);
        const cplx<T> ref2 = {ref, ref};
        const long off = (long)l * a.out_pstride + (long)j * NX;
        // the store form is chosen once per sequence (outside the unrolled loop)
        auto store = [&](auto form_c) {
          constexpr int FORM = decltype(form_c)::value;
#pragma unroll
          for (int gg = 0; gg < E / RO; ++gg)
#pragma unroll
            for (int rr = 0; rr < RO; ++rr) {
              const int m = lane_t + TL * gg + rr * (M / RO);
              const cplx<T> z = c_add(v[gg * RO + rr], ref2);
              if constexpr (FORM == 0) {
                *reinterpret_cast<float2*>(a.outf[f] + off + 2 * m) = make_float2(float(z.x), float(z.y));
              } else if constexpr (FORM == 1) {
                // one 8-byte (FP32) / 16-byte (FP64) store per output pair
                *reinterpret_cast<cplx<T>*>(a.out[f] + off + 2 * m) = z;
              } else {
                a.out[f][off + 2 * m] = z.x;
                a.out[f][off + 2 * m + 1] = z.y;
              }
            }
        };
        if (a.out_f32) store(std::integral_constant<int, 0>{});
        else if (a.pair_store) store(std::integral_constant<int, 1>{});
        else store(std::integral_constant<int, 2>{});
      }
    } else {
      __syncwarp();
#pragma unroll
      for (int gg = 0; gg < E / RO; ++gg)
#pragma unroll
        for (int rr = 0; rr < RO; ++rr) seq[lane_t + TL * gg + rr * (M / RO)] = v[gg * RO + rr];
    }
  }
  if (!direct) {
  __syncthreads();
  const T* xs = reinterpret_cast<const T*>(buf);  // x_i of sequence s at xs[s*XS + i]
  // four consecutive points per thread
  for (int idx = threadIdx.x; idx < a.R * (NX / 4); idx += blockDim.x) {
    const int r = idx / (NX / 4);
    const int i0 = 4 * (idx - r * (NX / 4));
    const int l = rowl[r];
    if (l < 0) continue;
    const int j = rowj[r];
    T* xw0 = const_cast<T*>(xs) + (long)(r * a.nin) * XS + i0;
    for (int f = 0; f < a.nin; ++f)  // this thread alone touches (r, i0..i0+3)
      if (a.refin[f]) {
        const T rf = a.refin[f][l];
#pragma unroll
        for (int q = 0; q < 4; ++q) xw0[f * XS + q] += rf;
      }
    if (a.op == XI_DIV) {
      // compute_derivatives.f90:544-574 + LES_engine.f90:546-551, one
      // equation per input: out[q] = rhs, aux[q] = tz, lo[q] = stag,
      // pf[q] = forcing; out[8]/out[9] = bottom/top pressure-BC layers of
      // the non-staggered (w) equation.  c0 = 1/dz.
      using V = V4<T>;
      const T rdz = T(a.c0);
      const long pl = a.out_pstride;
      const long off = (long)l * pl + (long)j * NX + i0;
      const long p2 = (long)j * NX + i0;
      for (int q = 0; q < a.nin; ++q) {
        const T* tz = a.aux[q];
        const V xq = vld<V>(static_cast<const T*>(xw0), (long)q * XS);
        if (l >= 1 && l <= a.nz) {
          const V dzq = a.lo[q] ? rdz * (vld<V>(tz, off + pl) - vld<V>(tz, off))   // ddz_w
                                : rdz * (vld<V>(tz, off) - vld<V>(tz, off - pl));  // ddz_uv
          vst(a.out[q] + off, ((vld<V>(a.out[q], off) + xq) + dzq) + vsplat<V>(T(a.pf[q])));
          if (!a.lo[q] && l == 1 && a.out[8]) vst(a.out[8] + p2, xq + dzq);
        }
        if (!a.lo[q] && l == a.nz + 1 && a.out[9]) vst(a.out[9] + p2, xq);
      }
      continue;
    }
#pragma unroll 1
    for (int q4 = 0; q4 < 4; ++q4) {
    const int i = i0 + q4;
    const long off = (long)l * a.out_pstride + (long)j * NX + i;
    const T* x = xw0 + q4;  // field f at x[f*XS]
    switch (a.op) {
      case XI_STORE: {
        for (int f = 0; f < a.nin; ++f)
          if (l >= a.lo[f] && l <= a.hi[f]) {
            if (a.out_f32) a.outf[f][off] = float(x[f * XS]);
            else a.out[f][off] = x[f * XS];
          }
        break;
      }
      case XI_LASD: {
        // compute_LagScaleDep.f90:541-594; c0 = 2 delta^2, c1 = alpha^2
        const T uf = x[0], vf = x[XS], wf = x[2 * XS];
        const T a11 = x[3 * XS] - uf * uf;
        const T a12 = x[4 * XS] - uf * vf;
        const T a13 = x[5 * XS] - uf * wf;
        const T a22 = x[6 * XS] - vf * vf;
        const T a23 = x[7 * XS] - vf * wf;
        const T a33 = x[8 * XS] - wf * wf;
        const T s11 = x[9 * XS], s12 = x[10 * XS], s13 = x[11 * XS];
        const T s22 = x[12 * XS], s23 = x[13 * XS], s33 = x[14 * XS];
        const T sft = sqrt(T(2) * (s11 * s11 + s22 * s22 + s33 * s33 +
                                   T(2) * (s12 * s12 + s13 * s13 + s23 * s23)));
        const T cst = T(a.c0), tf2 = T(a.c1);
        const T b11 = cst * (x[15 * XS] - tf2 * sft * s11);
        const T b12 = cst * (x[16 * XS] - tf2 * sft * s12);
        const T b13 = cst * (x[17 * XS] - tf2 * sft * s13);
        const T b22 = cst * (x[18 * XS] - tf2 * sft * s22);
        const T b23 = cst * (x[19 * XS] - tf2 * sft * s23);
        const T b33 = cst * (x[20 * XS] - tf2 * sft * s33);
        a.out[0][off] = a11 * b11 + a22 * b22 + a33 * b33 + T(2) * (a12 * b12 + a13 * b13 + a23 * b23);
        a.out[1][off] = b11 * b11 + b22 * b22 + b33 * b33 + T(2) * (b12 * b12 + b13 * b13 + b23 * b23);
        break;
      }
      case XI_SCDYN: {
        // K_j = filt(u_j theta) - filt(u_j) filt(theta),
        // X_j = Delta^2 (filt(|S| d_j theta) - alpha^2 |S~| filt(d_j theta));
        // c0 = Delta^2, c1 = alpha^2
        const T uf = x[0], vf = x[XS], wf = x[2 * XS], tf = x[3 * XS];
        const T k1 = x[4 * XS] - uf * tf;
        const T k2 = x[5 * XS] - vf * tf;
        const T k3 = x[6 * XS] - wf * tf;
        const T s11 = x[7 * XS], s12 = x[8 * XS], s13 = x[9 * XS];
        const T s22 = x[10 * XS], s23 = x[11 * XS], s33 = x[12 * XS];
        const T sft = sqrt(T(2) * (s11 * s11 + s22 * s22 + s33 * s33 +
                                   T(2) * (s12 * s12 + s13 * s13 + s23 * s23)));
        const T d2 = T(a.c0), tf2 = T(a.c1);
        const T x1 = d2 * (x[16 * XS] - tf2 * sft * x[13 * XS]);
        const T x2 = d2 * (x[17 * XS] - tf2 * sft * x[14 * XS]);
        const T x3 = d2 * (x[18 * XS] - tf2 * sft * x[15 * XS]);
        a.out[0][off] = k1 * x1 + k2 * x2 + k3 * x3;
        a.out[1][off] = x1 * x1 + x2 * x2 + x3 * x3;
        break;
      }
      case XI_WALL: {
        // compute_wall_law.f90:143-183, 247-251 on the filtered first level.
        // c0 = dz, c1 = 1/log-free constant unused; aux[0] = z0 plane.
        // out: u_star_avg, lbc_u, lbc_v, txz(1), tyz(1), dudz(1), dvdz(1)
        const long p2 = (long)j * NX + i;
        const double u1 = double(x[0]), v1 = double(x[XS]);
        const double uavg = sqrt(u1 * u1 + v1 * v1);
        const double dz = a.c0;
        const double ustar = KVONK * uavg / log((0.5 * dz) / double(a.aux[0][p2]));
        double bu = 0.0, bv = 0.0, tx = 0.0, ty = 0.0;
        if (uavg != 0.0) {
          bu = ustar / (0.5 * dz * KVONK) * u1 / uavg;
          bv = ustar / (0.5 * dz * KVONK) * v1 / uavg;
          tx = (ustar * ustar) * u1 / uavg;
          ty = (ustar * ustar) * v1 / uavg;
        }
        a.out[0][p2] = T(ustar);
        a.out[1][p2] = T(bu);
        a.out[2][p2] = T(bv);
        const long o1 = a.out_pstride + p2;  // level 1 of a field
        a.out[3][o1] = T(tx);
        a.out[4][o1] = T(ty);
        a.out[5][o1] = T(bu);
        a.out[6][o1] = T(bv);
        break;
      }
    }
    }
  }
  }  // the combining ops
  __syncthreads();
  if (a.nbuf > 1) {
    stg ^= 1;
  } else if (next < nitems) {
    // single stage: every thread is past the last read of it (barrier above)
    if (a.bulk) {
      xi_issue_bulk<T>(a, next, stage0, &bars[0]);
    } else {
      xi_issue<T>(a, next, stage0);
      cp_async_commit();
    }
  }
  }
}

}  // namespace les
