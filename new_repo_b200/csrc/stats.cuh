// Post-step statistics: the running sums of IO_statistics.f90 and the
// plane-averaged TKE budget of tke_budget1D.f90.  Both read the state the
// time step leaves behind and accumulate in FP64, like the reference (whose
// fields are FP64); in mixed precision the FP32 fields are widened first.
#pragma once
#include "common.cuh"

namespace les {

// ---------------------------------------------------------------------------
// io_3D_stat_averages (IO_statistics.f90:363-445): 26 running sums per point
// of levels 1..nz, stored as [26][nz][ny][nx] in the order the RAV_*_3D.dat
// file holds them (:447-488): u v w p, u2 v2 w2, u3 v3 w3, u4 v4 w4, uv uw
// vw, txx tyy tzz txy txz tyz, dudz dvdz, nu_t, sqrt(cs_opt2).
constexpr int STAT_NQ = 26;

template <typename T>
struct StatFields {
  const T *u, *v, *w, *p, *txx, *tyy, *tzz, *txy, *txz, *tyz, *dudz, *dvdz, *nut, *cs;
};

// Each product is rounded on its own (no fused multiply-add), so that the FP64
// sums equal those of the reference's expression order: x**3 = (x*x)*x,
// x**4 = (x*x)*(x*x).  uw and vw interpolate u, v to the w node; their
// first level is reset to zero on every call (:378-384).
template <typename T>
__global__ void __launch_bounds__(256) k_stat_accum(StatFields<T> f, double* __restrict__ acc, long plane, int nz) {
  const long n = (long)nz * plane;
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < n; o += (long)gridDim.x * blockDim.x) {
    const long c = o + plane;  // level 1 + o / plane of the (0..nz+1) storage
    const double u = f.u[c], v = f.v[c], w = f.w[c], p = f.p[c];
    double* a = acc + o;
    auto add = [&](int q, double x) { a[q * n] = __dadd_rn(a[q * n], x); };
    add(0, u);
    add(1, v);
    add(2, w);
    add(3, p);
    const double u2 = __dmul_rn(u, u), v2 = __dmul_rn(v, v), w2 = __dmul_rn(w, w);
    add(4, u2);
    add(5, v2);
    add(6, w2);
    add(7, __dmul_rn(u2, u));
    add(8, __dmul_rn(v2, v));
    add(9, __dmul_rn(w2, w));
    add(10, __dmul_rn(u2, u2));
    add(11, __dmul_rn(v2, v2));
    add(12, __dmul_rn(w2, w2));
    add(13, __dmul_rn(u, v));
    if (o < plane) {
      a[14 * n] = 0.0;
      a[15 * n] = 0.0;
    } else {
      const double um = __dmul_rn(0.5, __dadd_rn(double(f.u[c - plane]), u));
      const double vm = __dmul_rn(0.5, __dadd_rn(double(f.v[c - plane]), v));
      add(14, __dmul_rn(w, um));
      add(15, __dmul_rn(w, vm));
    }
    add(16, f.txx[c]);
    add(17, f.tyy[c]);
    add(18, f.tzz[c]);
    add(19, f.txy[c]);
    add(20, f.txz[c]);
    add(21, f.tyz[c]);
    add(22, f.dudz[c]);
    add(23, f.dvdz[c]);
    add(24, f.nut[c]);
    add(25, __dsqrt_rn(double(f.cs[c])));
  }
}

// io_2D_stat_averages (:316-320): running sum of the friction-velocity plane
template <typename T>
__global__ void k_plane_accum(const T* __restrict__ x, double* __restrict__ acc, long plane) {
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < plane; o += (long)gridDim.x * blockDim.x)
    acc[o] = __dadd_rn(acc[o], double(x[o]));
}

// ---------------------------------------------------------------------------
// compute_tke_budget (tke_budget1D.f90:209-390): 61 plane averages per level
// 1..nz, in the order of its avg_var calls.
constexpr int TKE_NQ = 61;

template <typename T>
struct TkeFields {
  const T *u, *v, *w, *dudx, *dudy, *dudz, *dvdx, *dvdy, *dvdz, *dwdx, *dwdy, *dwdz;
  const T *txx, *tyy, *tzz, *txy, *txz, *tyz, *cs;
  const T *c, *cx, *cy;  // the filtered "cleaned pressure" and its x, y derivatives
};

// The pointwise quantities of one point at storage offset o (level k),
// handed to put(index, value).  int_var (:424-446) interpolates w-node
// fields to the uvp node: 0.5*(f(k)+f(k+1)).  With the wall law, the first
// level of the interpolated txz, tyz and of dudz+dwdx, dvdz+dwdy is replaced
// as in :296-322.  The cs profile reads cs_opt2 one level up: the
// reference copies the (nx,ny,nz+1) array cs_opt2 into a (nx,ny,0:nz+1)
// scratch by array position (:275), so scratch level k holds level k+1.
template <typename T, typename Put>
__device__ __forceinline__ void tke_point(const TkeFields<T>& f, long o, long plane, bool k1, bool wall, double idz,
                                          Put&& put) {
  const long up = o + plane, dn = o - plane;
  auto I = [&](const T* x) { return 0.5 * (double(x[o]) + double(x[up])); };
  const double U = f.u[o], V = f.v[o];
  const double W = I(f.w);
  const double ux = f.dudx[o], uy = f.dudy[o], uz = I(f.dudz);
  const double vx = f.dvdx[o], vy = f.dvdy[o], vz = I(f.dvdz);
  const double wx = I(f.dwdx), wy = I(f.dwdy), wz = f.dwdz[o];
  put(0, U);
  put(1, V);
  put(2, W);
  put(3, ux);
  put(4, uy);
  put(5, uz);
  put(6, vx);
  put(7, vy);
  put(8, vz);
  put(9, wx);
  put(10, wy);
  put(11, wz);
  put(12, U * U);
  put(13, V * V);
  put(14, W * W);
  put(15, U * V);
  put(16, W * U);
  put(17, W * V);
  const double txx = f.txx[o], tyy = f.tyy[o], tzz = f.tzz[o], txy = f.txy[o];
  const double txzi = I(f.txz), tyzi = I(f.tyz);
  put(18, txx);
  put(19, tyy);
  put(20, tzz);
  put(21, txy);
  put(22, txzi);
  put(23, tyzi);
  put(24, double(f.cs[up]));
  put(25, (U * U) * W);
  put(26, (V * V) * W);
  put(27, (W * W) * W);
  put(28, U * (W * W));
  put(29, W * tzz);
  const bool wl = wall && k1;
  const double s3 = wl ? double(f.txz[o]) : txzi;
  const double s2 = wl ? double(f.tyz[o]) : tyzi;
  put(30, s3 * U);
  put(31, s2 * V);
  put(32, ux * txx);
  put(33, vy * tyy);
  put(34, wz * tzz);
  put(35, 0.5 * (uy + vx) * txy);
  const double s4 = wl ? double(f.dudz[o]) + 0.5 * (double(f.dwdx[o]) + double(f.dwdx[up]))
                       : 0.5 * ((double(f.dudz[o]) + double(f.dwdx[o])) + (double(f.dudz[up]) + double(f.dwdx[up])));
  const double s1 = wl ? double(f.dvdz[o]) + 0.5 * (double(f.dwdy[o]) + double(f.dwdy[up]))
                       : 0.5 * ((double(f.dvdz[o]) + double(f.dwdy[o])) + (double(f.dvdz[up]) + double(f.dwdy[up])));
  put(36, 0.5 * s4 * s3);
  put(37, 0.5 * s2 * s1);
  put(38, ux * ux);
  put(39, uy * uy);
  put(40, uz * uz);
  put(41, vx * vx);
  put(42, vy * vy);
  put(43, vz * vz);
  put(44, wx * wx);
  put(45, wy * wy);
  put(46, wz * wz);
  put(47, ux * wx);
  put(48, uy * wy);
  put(49, uz * wz);
  // pressure terms (:336-372): ddz_uv then int_var of the filtered field
  const double C = f.c[o];
  put(50, C);
  put(51, double(f.cx[o]));
  put(52, double(f.cy[o]));
  const double dz0 = idz * (C - double(f.c[dn])), dz1 = idz * (double(f.c[up]) - C);
  put(53, 0.5 * (dz0 + dz1));
  put(54, C * W);
  put(55, C * U);
  put(56, C * ux);
  put(57, C * vy);
  put(58, C * wz);
  put(59, C * wx);
  put(60, C * uz);
}

// Quantities [Q0, Q0 + NQ) of every point of level 1 + blockIdx.y, summed
// over the blockIdx.x-th share of the plane in a fixed order (per thread,
// then a shuffle tree per warp, then warps in order) -> part.
template <typename T, int Q0, int NQ>
__global__ void __launch_bounds__(256) k_tke_partial(TkeFields<T> f, double* __restrict__ part, long plane, int wall,
                                                     double idz) {
  const int k = 1 + blockIdx.y;
  const long base = (long)k * plane;
  double acc[NQ];
#pragma unroll
  for (int i = 0; i < NQ; ++i) acc[i] = 0.0;
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < plane; o += (long)gridDim.x * blockDim.x)
    tke_point(f, base + o, plane, k == 1, wall != 0, idz, [&](int q, double x) {
      if (q >= Q0 && q < Q0 + NQ) acc[q - Q0] += x;
    });
  __shared__ double red[8][NQ];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NQ; ++i) {
    double v = acc[i];
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
    if (lane == 0) red[wid][i] = v;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NQ; i += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][i];
    part[((long)blockIdx.y * gridDim.x + blockIdx.x) * TKE_NQ + Q0 + i] = s;
  }
}

// avar(q, k) += (sum of the shares) / (nx ny)  (avg_var :400-406 with
// compute_planar_average utility_tools.f90:59-92)
__global__ void k_tke_final(const double* __restrict__ part, int nch, int nz, double npts, double* __restrict__ avar) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nz * TKE_NQ; idx += gridDim.x * blockDim.x) {
    const int k0 = idx / TKE_NQ, q = idx % TKE_NQ;
    double s = 0.0;
    for (int c = 0; c < nch; ++c) s += part[((long)k0 * nch + c) * TKE_NQ + q];
    avar[(long)q * nz + k0] += s / npts;
  }
}

// The cleaned pressure p - |u|^2 / 2 of :336-343 on levels 1..nz.  Its ghost
// levels are never set by the reference's routine; on one rank scratch level
// 0 still holds cs_opt2 level 1 from the array copy of :275, and level nz+1
// is unset memory, taken here as zero.  Both reach only the dpdz profile at
// levels 1 and nz.
template <typename T>
__global__ void k_tke_cpress(const T* __restrict__ p, const T* __restrict__ u, const T* __restrict__ v,
                             const T* __restrict__ w, const T* __restrict__ cs, T* __restrict__ c, long plane, int nz) {
  const long n = (long)(nz + 2) * plane;
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < n; o += (long)gridDim.x * blockDim.x) {
    const long k = udiv32(o, plane);
    if (k == 0) {
      c[o] = cs[o + plane];
    } else if (k == nz + 1) {
      c[o] = T(0);
    } else {
      const double wm = 0.5 * (double(w[o]) + double(w[o + plane]));
      const double uu = double(u[o]), vv = double(v[o]);
      c[o] = T(double(p[o]) - 0.5 * (uu * uu + vv * vv + wm * wm));
    }
  }
}

}  // namespace les
