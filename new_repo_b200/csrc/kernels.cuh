// Pointwise, vertical and reduction kernels of the LES step.
#pragma once
#include "common.cuh"

namespace les {

// ---------------------------------------------------------------------------
// boundary conditions (boundary_condition_mpi.f90:33-63); types 0/1/2 =
// none/'drc'/'neu'.  u, v are staggered (uvp nodes), w is not.
template <typename T>
__global__ void k_set_bc(T* u, T* v, T* w, const T* lu, const T* lv, const T* lw, const T* tu, const T* tv,
                         const T* tw, int4 lt, int4 ut, long plane, int nz, T dz) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < plane; p += (long)gridDim.x * blockDim.x) {
    const long b0 = p, b1 = plane + p, t0 = (long)nz * plane + p, t1 = (long)(nz + 1) * plane + p;
    if (lt.x == 1) u[b0] = T(2) * lu[p] - u[b1];
    else if (lt.x == 2) u[b0] = u[b1] - lu[p] * dz;
    if (lt.y == 1) v[b0] = T(2) * lv[p] - v[b1];
    else if (lt.y == 2) v[b0] = v[b1] - lv[p] * dz;
    if (lt.z == 1) w[b1] = lw[p];
    if (ut.x == 1) u[t1] = T(2) * tu[p] - u[t0];
    else if (ut.x == 2) u[t1] = u[t0] + tu[p] * dz;
    if (ut.y == 1) v[t1] = T(2) * tv[p] - v[t0];
    else if (ut.y == 2) v[t1] = v[t0] + tv[p] * dz;
    if (ut.z == 1) w[t1] = tw[p];
  }
}

// ddz_uv (uvp -> w, k = 1..nz+1) for u, v and ddz_w (w -> uvp, k = 1..nz,
// top level zero) for w (compute_derivatives.f90:375-441).
// four consecutive values (16-byte aligned for FP32, 32-byte for FP64)
__device__ __forceinline__ void ld4(const float* p, float* o) {
  const float4 x = *reinterpret_cast<const float4*>(p);
  o[0] = x.x;
  o[1] = x.y;
  o[2] = x.z;
  o[3] = x.w;
}
__device__ __forceinline__ void ld4(const double* p, double* o) {
  const double2 x = reinterpret_cast<const double2*>(p)[0], y = reinterpret_cast<const double2*>(p)[1];
  o[0] = x.x;
  o[1] = x.y;
  o[2] = y.x;
  o[3] = y.y;
}
__device__ __forceinline__ void st4(float* p, const float* v) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double* v) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

template <typename T>
__global__ void k_ddz_vel(const T* u, const T* v, const T* w, T* dudz, T* dvdz, T* dwdz, long plane, int nz,
                          T rdz) {
  const long n = (long)(nz + 1) * plane;
  if (plane % 4 == 0) {  // four consecutive points (one level) per thread, vector loads and stores
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n / 4; q += (long)gridDim.x * blockDim.x) {
      const long o = plane + 4 * q;
      const int k = udiv32(o, plane);
      T a[4], b[4], r[4];
      ld4(u + o, a);
      ld4(u + o - plane, b);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = rdz * (a[i] - b[i]);
      st4(dudz + o, r);
      ld4(v + o, a);
      ld4(v + o - plane, b);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = rdz * (a[i] - b[i]);
      st4(dvdz + o, r);
      if (k <= nz) {
        ld4(w + o + plane, a);
        ld4(w + o, b);
#pragma unroll
        for (int i = 0; i < 4; ++i) r[i] = rdz * (a[i] - b[i]);
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) r[i] = T(0);
      }
      st4(dwdz + o, r);
    }
    return;
  }
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long o = plane + q;  // levels 1..nz+1
    const int k = udiv32(o, plane);
    dudz[o] = rdz * (u[o] - u[o - plane]);
    dvdz[o] = rdz * (v[o] - v[o - plane]);
    dwdz[o] = (k <= nz) ? rdz * (w[o + plane] - w[o]) : T(0);
  }
}

template <typename T>
__global__ void k_ddz(T* out, const T* f, long plane, int nz, T rdz, int w_to_uvp) {
  const long n = (long)(nz + 1) * plane;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long o = plane + q;
    const int k = udiv32(o, plane);
    if (w_to_uvp) out[o] = (k <= nz) ? rdz * (f[o + plane] - f[o]) : T(0);
    else out[o] = rdz * (f[o] - f[o - plane]);
  }
}

template <typename T>
__global__ void k_fill(T* f, long n, T val) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) f[q] = val;
}

// up to 8 plane-sized copies or fills in one launch (blockIdx.y = the op):
// the ghost-level writes of a step, which would otherwise each be a launch
template <typename T>
struct PlaneOps {
  T* dst[8];
  const T* src[8];  // null: fill with val[op]
  T val[8];
};
template <typename T>
__global__ void k_plane_ops(const PlaneOps<T> ops, long n) {
  const int op = blockIdx.y;
  T* d = ops.dst[op];
  const T* s = ops.src[op];
  const T v = ops.val[op];
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    d[q] = s ? s[q] : v;
}

template <typename T>
__global__ void k_scale(T* f, long n, T c) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) f[q] = c * f[q];
}

template <typename D, typename S>
__global__ void k_convert(D* dst, const S* src, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    dst[q] = D(src[q]);
}

// The three velocity fields in one launch: blockIdx.y selects the field.
template <typename D, typename S>
struct Convert3 {
  D* dst[3];
  const S* src[3];
};
template <typename D, typename S>
__global__ void k_convert3(const Convert3<D, S> a, long n) {
  D* __restrict__ d = a.dst[blockIdx.y];
  const S* __restrict__ s = a.src[blockIdx.y];
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) d[q] = D(s[q]);
}

template <typename T>
__global__ void k_copy(T* dst, const T* src, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) dst[q] = src[q];
}

// ---------------------------------------------------------------------------
// SGS stress (compute_sgs.f90:105-335)
template <typename T>
struct SgsArgs {
  const T* d[9];  // dudx dudy dudz dvdx dvdy dvdz dwdx dwdy dwdz
  const T* cs;
  const double* l2;  // mixing length squared per level
  T *nu, *txx, *txy, *txz, *tyy, *tyz, *tzz;
  T* sij[6];  // optional: s11 s12 s13 s22 s23 s33
  T* smag;    // optional: |S|
  int write_sij;
  int wall;
  long plane;
  int nz;
  // optional scalar SGS flux (q[0] != nullptr): pi_j = nu_theta d_j theta
  // with nu_theta = |S| (inv_prt Cs^2 l^2 + kapd[k]); pi_z(1) = -qs
  const T* dt[3];  // d theta / dx, dy (uvp nodes), dz (w nodes)
  T* q[3];         // pi_x, pi_y (uvp nodes), pi_z (w nodes)
  const double* kapd;  // Cs^2/Pr_t Delta^2 per level (dynamic model) or nullptr
  double inv_prt;      // 1 / Pr_t (constant model) or 0
  double qs;           // surface flux
};

template <typename T>
__device__ __forceinline__ void sij_at(const SgsArgs<T>& a, long o, int k, T s[6]) {
  const long pl = a.plane;
  T ux, uy, uz, vx, vy, vz, wx, wy, wz;
  if (k == 1) {
    ux = a.d[0][o];
    uy = a.d[1][o];
    if (a.wall) {
      uz = a.d[2][o];
      vz = a.d[5][o];
    } else {
      uz = T(0.5) * (a.d[2][o] + a.d[2][o + pl]);
      vz = T(0.5) * (a.d[5][o] + a.d[5][o + pl]);
    }
    vx = a.d[3][o];
    vy = a.d[4][o];
    wx = T(0.5) * (a.d[6][o] + a.d[6][o + pl]);
    wy = T(0.5) * (a.d[7][o] + a.d[7][o + pl]);
    wz = a.d[8][o];
  } else {
    ux = T(0.5) * (a.d[0][o] + a.d[0][o - pl]);
    uy = T(0.5) * (a.d[1][o] + a.d[1][o - pl]);
    uz = a.d[2][o];
    vx = T(0.5) * (a.d[3][o] + a.d[3][o - pl]);
    vy = T(0.5) * (a.d[4][o] + a.d[4][o - pl]);
    vz = a.d[5][o];
    wx = a.d[6][o];
    wy = a.d[7][o];
    wz = T(0.5) * (a.d[8][o] + a.d[8][o - pl]);
  }
  s[0] = ux;
  s[1] = T(0.5) * (uy + vx);
  s[2] = T(0.5) * (uz + wx);
  s[3] = vy;
  s[4] = T(0.5) * (vz + wy);
  s[5] = wz;
}

template <typename T>
__device__ __forceinline__ T strain_norm(const T s[6]) {
  return sqrt(T(2) * (s[0] * s[0] + s[3] * s[3] + s[5] * s[5] + T(2) * (s[1] * s[1] + s[2] * s[2] + s[4] * s[4])));
}

// sij_at for four consecutive points of one level (16-byte aligned offset),
// the same arithmetic per point: s[c][i] is component c at point o + i
template <typename T>
__device__ __forceinline__ void sij_at4(const SgsArgs<T>& a, long o, int k, T s[6][4]) {
  const long pl = a.plane;
  T d[9][4];
#pragma unroll
  for (int j = 0; j < 9; ++j) ld4(a.d[j] + o, d[j]);
  if (k == 1) {
    T e2[4], e5[4], e6[4], e7[4];
    ld4(a.d[6] + o + pl, e6);
    ld4(a.d[7] + o + pl, e7);
    if (!a.wall) {
      ld4(a.d[2] + o + pl, e2);
      ld4(a.d[5] + o + pl, e5);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const T ux = d[0][i], uy = d[1][i];
      const T uz = a.wall ? d[2][i] : T(0.5) * (d[2][i] + e2[i]);
      const T vz = a.wall ? d[5][i] : T(0.5) * (d[5][i] + e5[i]);
      const T vx = d[3][i], vy = d[4][i];
      const T wx = T(0.5) * (d[6][i] + e6[i]), wy = T(0.5) * (d[7][i] + e7[i]), wz = d[8][i];
      s[0][i] = ux;
      s[1][i] = T(0.5) * (uy + vx);
      s[2][i] = T(0.5) * (uz + wx);
      s[3][i] = vy;
      s[4][i] = T(0.5) * (vz + wy);
      s[5][i] = wz;
    }
  } else {
    T p0[4], p1[4], p3[4], p4[4], p8[4];
    ld4(a.d[0] + o - pl, p0);
    ld4(a.d[1] + o - pl, p1);
    ld4(a.d[3] + o - pl, p3);
    ld4(a.d[4] + o - pl, p4);
    ld4(a.d[8] + o - pl, p8);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const T ux = T(0.5) * (d[0][i] + p0[i]), uy = T(0.5) * (d[1][i] + p1[i]), uz = d[2][i];
      const T vx = T(0.5) * (d[3][i] + p3[i]), vy = T(0.5) * (d[4][i] + p4[i]), vz = d[5][i];
      const T wx = d[6][i], wy = d[7][i], wz = T(0.5) * (d[8][i] + p8[i]);
      s[0][i] = ux;
      s[1][i] = T(0.5) * (uy + vx);
      s[2][i] = T(0.5) * (uz + wx);
      s[3][i] = vy;
      s[4][i] = T(0.5) * (vz + wy);
      s[5][i] = wz;
    }
  }
}

// k_sgs_tau with four consecutive points per thread (plane a multiple of 4):
// grid (ceil(plane / 4 / 256), nz + 1)
template <typename T>
__global__ void k_sgs_tau4(const SgsArgs<T> a) {
  const long pl = a.plane;
  const long p = 4 * (blockIdx.x * (long)blockDim.x + threadIdx.x);
  if (p >= pl) return;
  const int k = 1 + blockIdx.y;
  const long o = (long)k * pl + p;
  T s[6][4], cs[4], nu[4], d0[4], d1[4], d3[4], d4[4], d8[4], r[4];
  sij_at4(a, o, k, s);
  ld4(a.cs + o, cs);
  T sn[4];  // |S| at this level
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const T si[6] = {s[0][i], s[1][i], s[2][i], s[3][i], s[4][i], s[5][i]};
    sn[i] = strain_norm(si);
    nu[i] = sn[i] * cs[i] * T(a.l2[k]);
  }
  st4(a.nu + o, nu);
  const bool scal = a.q[0] != nullptr;
  T nut[4];  // nu_theta at this level
  if (scal) {
    const T kd = a.kapd ? T(a.kapd[k]) : T(0);
#pragma unroll
    for (int i = 0; i < 4; ++i) nut[i] = sn[i] * (T(a.inv_prt) * cs[i] * T(a.l2[k]) + kd);
  }
  ld4(a.d[0] + o, d0);
  ld4(a.d[1] + o, d1);
  ld4(a.d[3] + o, d3);
  ld4(a.d[4] + o, d4);
  ld4(a.d[8] + o, d8);
  if (k == 1) {
#pragma unroll
    for (int i = 0; i < 4; ++i) r[i] = T(2) * nu[i] * d8[i];
    st4(a.tzz + o, r);
    st4(a.tzz + o - pl, r);  // tzz(0) = tzz(1)
#pragma unroll
    for (int i = 0; i < 4; ++i) r[i] = T(2) * nu[i] * d0[i];
    st4(a.txx + o, r);
#pragma unroll
    for (int i = 0; i < 4; ++i) r[i] = T(2) * nu[i] * T(0.5) * (d1[i] + d3[i]);
    st4(a.txy + o, r);
#pragma unroll
    for (int i = 0; i < 4; ++i) r[i] = T(2) * nu[i] * d4[i];
    st4(a.tyy + o, r);
    if (scal) {
      T t[4];
      ld4(a.dt[0] + o, t);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = nut[i] * t[i];
      st4(a.q[0] + o, r);
      ld4(a.dt[1] + o, t);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = nut[i] * t[i];
      st4(a.q[1] + o, r);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = -T(a.qs);
      st4(a.q[2] + o, r);
    }
  } else {
    if (k <= a.nz) {
      T s2[6][4], csp[4], c[4], ct[4];
      sij_at4(a, o + pl, k + 1, s2);
      ld4(a.cs + o + pl, csp);
      const T kdp = (scal && a.kapd) ? T(a.kapd[k + 1]) : T(0);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const T si[6] = {s2[0][i], s2[1][i], s2[2][i], s2[3][i], s2[4][i], s2[5][i]};
        const T snp = strain_norm(si);
        const T nukp = snp * csp[i] * T(a.l2[k + 1]);
        c[i] = T(0.5) * (nu[i] + nukp);
        if (scal) ct[i] = T(0.5) * (nut[i] + snp * (T(a.inv_prt) * csp[i] * T(a.l2[k + 1]) + kdp));
      }
      if (scal) {
        T t[4];
        ld4(a.dt[0] + o, t);
#pragma unroll
        for (int i = 0; i < 4; ++i) r[i] = ct[i] * t[i];
        st4(a.q[0] + o, r);
        ld4(a.dt[1] + o, t);
#pragma unroll
        for (int i = 0; i < 4; ++i) r[i] = ct[i] * t[i];
        st4(a.q[1] + o, r);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = T(2) * c[i] * d0[i];
      st4(a.txx + o, r);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = T(2) * c[i] * T(0.5) * (d1[i] + d3[i]);
      st4(a.txy + o, r);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = T(2) * c[i] * d4[i];
      st4(a.tyy + o, r);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = T(2) * c[i] * d8[i];
      st4(a.tzz + o, r);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) r[i] = T(2) * nu[i] * s[2][i];
    st4(a.txz + o, r);
#pragma unroll
    for (int i = 0; i < 4; ++i) r[i] = T(2) * nu[i] * s[4][i];
    st4(a.tyz + o, r);
    if (scal) {
      T t[4];
      ld4(a.dt[2] + o, t);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = nut[i] * t[i];
      st4(a.q[2] + o, r);
    }
  }
}

// S_ij and |S| on levels 1..nz+1 (written for the dynamic procedure).
template <typename T>
__global__ void k_sij(const SgsArgs<T> a) {
  const long n = (long)(a.nz + 1) * a.plane;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long o = a.plane + q;
    const int k = udiv32(o, a.plane);
    T s[6];
    sij_at(a, o, k, s);
#pragma unroll
    for (int t = 0; t < 6; ++t) a.sij[t][o] = s[t];
    a.smag[o] = strain_norm(s);
  }
}

// nu_t = |S| Cs^2 l^2 and tau_ij (compute_sgs.f90:177-242).
template <typename T>
// grid: (plane / blockDim.x, nz + 1); blockIdx.y + 1 is the level
__global__ void k_sgs_tau(const SgsArgs<T> a) {
  const long pl = a.plane;
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p < pl) {
    const int k = 1 + blockIdx.y;
    const long o = (long)k * pl + p;
    T s[6];
    sij_at(a, o, k, s);
    const T nuk = strain_norm(s) * a.cs[o] * T(a.l2[k]);
    a.nu[o] = nuk;
    if (k == 1) {
      const T tz = T(2) * nuk * a.d[8][o];
      a.txx[o] = T(2) * nuk * a.d[0][o];
      a.txy[o] = T(2) * nuk * T(0.5) * (a.d[1][o] + a.d[3][o]);
      a.tyy[o] = T(2) * nuk * a.d[4][o];
      a.tzz[o] = tz;
      a.tzz[o - pl] = tz;  // tzz(0) = tzz(1)
    } else {
      if (k <= a.nz) {
        T s2[6];
        sij_at(a, o + pl, k + 1, s2);
        const T nukp = strain_norm(s2) * a.cs[o + pl] * T(a.l2[k + 1]);
        const T c = T(0.5) * (nuk + nukp);
        a.txx[o] = T(2) * c * a.d[0][o];
        a.txy[o] = T(2) * c * T(0.5) * (a.d[1][o] + a.d[3][o]);
        a.tyy[o] = T(2) * c * a.d[4][o];
        a.tzz[o] = T(2) * c * a.d[8][o];
      }
      a.txz[o] = T(2) * nuk * s[2];
      a.tyz[o] = T(2) * nuk * s[4];
    }
  }
}

// ---------------------------------------------------------------------------
// Lagrangian scale-dependent dynamic model (compute_LagScaleDep.f90)
template <typename T>
__global__ void k_lag_accum(T* ul, T* vl, T* wl, const T* u, const T* v, const T* w, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    ul[q] = ul[q] + u[q];
    vl[q] = vl[q] + v[q];
    wl[q] = wl[q] + w[q];
  }
}

struct LagGeom {
  int nx, ny, nz;
  long plane;
  int mode;  // 0 reference 1x1 halo, 1 periodic
  double dt, dx, dy, dz, cs;
  int nlev;  // levels 1..nlev are interpolated (nz + 1: all)
};

// Offset of FF(i, j, k) of compute_interpolag_coeff (1-based i, j; level k
// in 0..nz+2) as update_halo3 (decomp_2d_custom.f90:902-1024) and the
// overrides of compute_LagScaleDep.f90:441-452 leave it.  The same for the
// four averaged fields, so a point takes its eight neighbours' offsets once.
__device__ __forceinline__ long ff_off(int i, int j, int k, const LagGeom& g) {
  if (k == 0) k = 1;
  const bool inner = (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny);
  const int ii = (i == 0) ? g.nx : ((i == g.nx + 1) ? 1 : i);
  int jj;
  if (k >= g.nz + 1) {
    if (inner) return (long)(g.nz + 1) * g.plane + (long)(j - 1) * g.nx + (i - 1);
    if (g.mode == 1) {
      jj = (j == 0) ? g.ny : ((j == g.ny + 1) ? 1 : j);
      return (long)(g.nz + 1) * g.plane + (long)(jj - 1) * g.nx + (ii - 1);
    }
    k -= 2;  // self-message halo: levels nz+1, nz+2 hold copies of nz-1, nz
  }
  if (g.mode == 1) jj = (j == 0) ? g.ny : ((j == g.ny + 1) ? 1 : j);
  else jj = (j == 0) ? 2 : ((j == g.ny + 1) ? g.ny - 1 : j);
  return (long)k * g.plane + (long)(jj - 1) * g.nx + (ii - 1);
}

// compute_interpolag_weight (:309-411) + compute_interpolag_coeff (:427-474)
// for the four F fields at once; writes the interpolated fields to Fn.
template <typename T>
__global__ void k_lag_interp(const T* ul, const T* vl, const T* wl, const T* F0, const T* F1, const T* F2,
                             const T* F3, T* N0, T* N1, T* N2, T* N3, LagGeom g) {
  // grid: (plane / blockDim.x, nlev); one point per thread, level
  // blockIdx.y + 1, and one 32-bit division for the (i, j) of the point
  const long pl = g.plane;
  const T cs = T(g.cs);
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < pl) {
    const int k = blockIdx.y + 1;
    const long o = (long)k * pl + p;
    const int jj = p / g.nx;
    const int i = p - jj * g.nx + 1;
    const int j = jj + 1;
    T uu, vv;
    if (k == 1) {
      uu = ul[o] / cs;
      vv = vl[o] / cs;
    } else {
      uu = T(0.5) * (ul[o] / cs + ul[o - pl] / cs);
      vv = T(0.5) * (vl[o] / cs + vl[o - pl] / cs);
    }
    const T xp = -uu * T(g.dt) * cs / T(g.dx);
    const T yp = -vv * T(g.dt) * cs / T(g.dy);
    T zp;
    if (k <= 2) {
      const long o2 = 2 * pl + p;
      const T w2 = wl[o2] / cs;
      T z2 = -w2 * T(g.dt) * cs / T(g.dz);
      z2 = z2 + fmin(z2, T(0));
      z2 = fmin(T(1), z2);
      z2 = fmax(T(-1), z2);
      zp = z2;
    } else {
      const T ww = wl[o] / cs;
      zp = -ww * T(g.dt) * cs / T(g.dz);
    }
    const int ax = i + (signbit(xp) ? -1 : 1);
    const int ay = j + (signbit(yp) ? -1 : 1);
    const int az = k + (signbit(zp) ? -1 : 1);
    const T cx = fabs(xp), cy = fabs(yp), cz = fabs(zp);
    const T fx = T(1) - cx, fy = T(1) - cy, fz = T(1) - cz;
    // the eight neighbours, then 32 independent loads
    const long n000 = ff_off(i, j, k, g), n00z = ff_off(i, j, az, g);
    const long n0y0 = ff_off(i, ay, k, g), n0yz = ff_off(i, ay, az, g);
    const long nx00 = ff_off(ax, j, k, g), nx0z = ff_off(ax, j, az, g);
    const long nxy0 = ff_off(ax, ay, k, g), nxyz = ff_off(ax, ay, az, g);
    const T* Fs[4] = {F0, F1, F2, F3};
    T* Ns[4] = {N0, N1, N2, N3};
    T v[4][8];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const T* __restrict__ F = Fs[t];
      v[t][0] = F[n000];
      v[t][1] = F[n00z];
      v[t][2] = F[n0y0];
      v[t][3] = F[n0yz];
      v[t][4] = F[nx00];
      v[t][5] = F[nx0z];
      v[t][6] = F[nxy0];
      v[t][7] = F[nxyz];
    }
#pragma unroll
    for (int t = 0; t < 4; ++t)
      Ns[t][o] = fx * fy * (v[t][0] * fz + v[t][1] * cz) + fx * cy * (v[t][2] * fz + v[t][3] * cz) +
                 cx * fy * (v[t][4] * fz + v[t][5] * cz) + cx * cy * (v[t][6] * fz + v[t][7] * cz);
  }
}

__device__ __forceinline__ double f32max_tiny(double x) {
  return double(fmaxf(1e-24f, float(x)));
}

// update_interpolag_coeff x2 (:607-640) and compute_dynamic_coeff (:651-707),
// including the default-REAL (float) casts of the reference's max() clips.
template <typename T>
__global__ void k_lasd_update(T* FLM, T* FMM, T* FQN, T* FNN, const T* LM, const T* MM, const T* QN, const T* NN,
                              T* cs, T* beta, int init, long plane, int nz, double opftdelta, double lagran_dt,
                              double beta_pow, const T* cs_init = nullptr, int nlev = -1, double cs_max = 0.0) {
  const long n = (long)(nlev < 0 ? nz + 1 : nlev) * plane;  // levels 1..nlev
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long o = plane + q;
    const bool top = q >= (long)nz * plane;  // level nz + 1 (o = plane + q)
    double flm, fmm, fqn, fnn;
    const double lm = LM[o], mm = MM[o], qn = QN[o], nn = NN[o];
    if (init) {
      // compute_lagscaledep.f90 initialisation: averages that imply Cs^2 = 0.03
      // (or, for the learned closure's fallback, the current coefficient)
      const double c0 = cs_init ? double(cs_init[o]) : 0.03;
      fmm = mm;
      flm = c0 * mm;
      fnn = nn;
      fqn = c0 * nn;
    } else {
      flm = FLM[o];
      fmm = FMM[o];
      fqn = FQN[o];
      fnn = FNN[o];
    }
    // 2 Delta pair
    {
      double tmp = double(fmaxf(float(flm * fmm), 1e-24f));
      tmp = opftdelta * pow(tmp, -0.125);
      tmp = f32max_tiny(tmp);
      const double dumfac = lagran_dt / tmp;
      const double epsi = dumfac / (1.0 + dumfac);
      flm = epsi * lm + (1.0 - epsi) * flm;
      fmm = epsi * mm + (1.0 - epsi) * fmm;
      flm = f32max_tiny(flm);
    }
    // 4 Delta pair
    {
      double tmp = double(fmaxf(float(fqn * fnn), 1e-24f));
      tmp = opftdelta * pow(tmp, -0.125);
      tmp = f32max_tiny(tmp);
      const double dumfac = lagran_dt / tmp;
      const double epsi = dumfac / (1.0 + dumfac);
      fqn = epsi * qn + (1.0 - epsi) * fqn;
      fnn = epsi * nn + (1.0 - epsi) * fnn;
      fqn = f32max_tiny(fqn);
    }
    FLM[o] = T(flm);
    FMM[o] = T(fmm);
    FQN[o] = T(fqn);
    FNN[o] = T(fnn);
    // coefficient: use the stored values, as the reference's arrays hold them
    const double c2 = f32max_tiny(double(T(flm)) / double(T(fmm)));
    const double c4 = f32max_tiny(double(T(fqn)) / double(T(fnn)));
    double b = (beta_pow == 1.0) ? (c4 / c2) : pow(c4 / c2, beta_pow);
    b = double(fmaxf(float(b), 0.125f));
    if (top) b = 1.0;
    beta[o] = T(b);
    const double cv = f32max_tiny(c2 / b);
    cs[o] = T(cs_max > 0.0 ? fmin(cv, cs_max) : cv);  // optional upper clip (off: the reference)
  }
}

// ---------------------------------------------------------------------------
// time advancement (LES_engine.f90:253-331)
template <typename T>
__global__ void k_ab2(T* u, T* v, T* w, const T* rx, const T* ry, const T* rz, const T* fx, const T* fy,
                      const T* fz, long plane, int nz, T dt, T t1, T t2) {
  const long n = (long)(nz + 2) * plane;
  if (plane % 4 == 0) {  // four consecutive points (one level) per thread
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n / 4; q += (long)gridDim.x * blockDim.x) {
      const long o = 4 * q;
      const int k = udiv32(o, plane);
      T x[4], r[4], f[4];
      if (k >= 1 && k <= nz) {
        T* fld[3] = {u, v, w};
        const T* rr[3] = {rx, ry, rz};
        const T* ff[3] = {fx, fy, fz};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ld4(fld[c] + o, x);
          ld4(rr[c] + o, r);
          ld4(ff[c] + o, f);
#pragma unroll
          for (int i = 0; i < 4; ++i) x[i] = x[i] + dt * (t1 * r[i] + t2 * f[i]);
          st4(fld[c] + o, x);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) x[i] = T(0);
        st4(w + o, x);  // w(0) = w(nz+1) = 0
      }
    }
    return;
  }
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < n; o += (long)gridDim.x * blockDim.x) {
    const int k = udiv32(o, plane);
    if (k >= 1 && k <= nz) {
      u[o] = u[o] + dt * (t1 * rx[o] + t2 * fx[o]);
      v[o] = v[o] + dt * (t1 * ry[o] + t2 * fy[o]);
      w[o] = w[o] + dt * (t1 * rz[o] + t2 * fz[o]);
    } else {
      w[o] = T(0);  // w(0) = w(nz+1) = 0
    }
  }
}

// projection and rhs update (LES_engine.f90:303-331), w(1) = w(nz+1) = 0.
// The w correction is formed in FP64 whatever T: dp/dz carries the mean
// vertical pressure gradient (thousands, balancing the mean shear term of
// the vertical rhs), whose FP32 product with dt would leave the same
// rounding in every point of a level -- a plane-mean w, i.e. divergence in
// the (0,0) mode, far above the FP32 rounding of w itself.
template <typename T>
__global__ void k_projection(T* u, T* v, T* w, T* rx, T* ry, T* rz, const T* dpdx, const T* dpdy, const T* dpdz,
                             long plane, int nz, double dtt_d) {
  const long n = (long)(nz + 2) * plane;
  const T dtt = T(dtt_d);
  if (plane % 4 == 0) {  // four consecutive points (one level) per thread
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n / 4; q += (long)gridDim.x * blockDim.x) {
      const long o = 4 * q;
      const int k = udiv32(o, plane);
      T x[4], d[4], r[4];
      if (k >= 1 && k <= nz) {
        T* fld[3] = {u, v, w};
        T* rr[3] = {rx, ry, rz};
        const T* dd[3] = {dpdx, dpdy, dpdz};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ld4(dd[c] + o, d);
          ld4(rr[c] + o, r);
#pragma unroll
          for (int i = 0; i < 4; ++i) r[i] = r[i] - d[i];
          st4(rr[c] + o, r);
          if (c == 2 && k == 1) {
#pragma unroll
            for (int i = 0; i < 4; ++i) x[i] = T(0);
          } else if (c == 2) {
            ld4(fld[c] + o, x);
#pragma unroll
            for (int i = 0; i < 4; ++i) x[i] = T(double(x[i]) - dtt_d * double(d[i]));
          } else {
            ld4(fld[c] + o, x);
#pragma unroll
            for (int i = 0; i < 4; ++i) x[i] = x[i] - dtt * d[i];
          }
          st4(fld[c] + o, x);
        }
      } else if (k == nz + 1) {
#pragma unroll
        for (int i = 0; i < 4; ++i) x[i] = T(0);
        st4(w + o, x);
      }
    }
    return;
  }
  for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < n; o += (long)gridDim.x * blockDim.x) {
    const int k = udiv32(o, plane);
    if (k >= 1 && k <= nz) {
      const T dz_ = dpdz[o];
      u[o] = u[o] - dtt * dpdx[o];
      v[o] = v[o] - dtt * dpdy[o];
      w[o] = (k == 1) ? T(0) : T(double(w[o]) - dtt_d * double(dz_));
      rx[o] = rx[o] - dpdx[o];
      ry[o] = ry[o] - dpdy[o];
      rz[o] = rz[o] - dz_;
    } else if (k == nz + 1) {
      w[o] = T(0);
    }
  }
}

// p = fluctuation + FP64 mean profile (mixed precision only), p(nz+1) = BOGUS
template <typename T>
__global__ void k_p_finish(T* p, const double* pmean, long plane, int nz) {
  const long top = (long)(nz + 1) * plane;
  const long t0 = blockIdx.x * (long)blockDim.x + threadIdx.x, ts = (long)gridDim.x * blockDim.x;
  for (long q = t0; q < plane; q += ts) p[top + q] = T(BOGUS);
  if (!pmean) return;
  // levels 0..nz: the FP64 mean mode added back, four consecutive points of
  // one level per thread and iteration where the plane allows
  if (plane % 4 == 0) {
    for (long q4 = t0; q4 < top / 4; q4 += ts) {
      const long o = 4 * q4;
      const double m = pmean[udiv32(o, plane)];
      T a[4];
      ld4(p + o, a);
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = T(double(a[i]) + m);
      st4(p + o, a);
    }
  } else {
    for (long o = t0; o < top; o += ts) p[o] = T(double(p[o]) + pmean[udiv32(o, plane)]);
  }
}

// ---------------------------------------------------------------------------
// pressure: one Thomas solve per (kx, ky) (compute_pressure.f90:256-305,
// 448-493, matrix of build_matrix :544-619), always in FP64.
// O: type of the pressure spectrum written (FP32 in mixed precision, whose
// inverse transforms run in FP32); its rows are opitch values apart
// G (optional): a fourth spectrum added to the right-hand side of every
// interior row (the divergence of u^n over dt tadv1 when Hx, Hy, Hz hold the
// AB2 increment only; compiled in with INC).  pm (with G): FP64 plane means per level
// (pm[f * pm_L + k]: f = 0 rz, 1 rfz, 2 dudx, 3 dvdy, 4 dwdz) from which
// the kx = ky = 0 column forms its right-hand side,
// (hz(k+1) - hz(k)) / dz + (dudx + dvdy + dwdz) idt with hz = rz + r21 rfz,
// instead of the FP32 spectra's mean coefficients.
template <typename T, typename O = T, bool INC = false>
__global__ void k_tridiag(const cplx<T>* __restrict__ Hx, const cplx<T>* __restrict__ Hy,
                          const cplx<T>* __restrict__ Hz, const cplx<T>* __restrict__ G,
                          const cplx<T>* __restrict__ bot,
                          const cplx<T>* __restrict__ top, const double* __restrict__ kkx,
                          const double* __restrict__ kky, cplx<O>* __restrict__ phat, cplx<double>* __restrict__ xs,
                          double* __restrict__ gam, double* pmean, unsigned* status, int lhx, int ny, int nz,
                          double dz, int drop_mean, int opitch, int ipitch, const double* pm = nullptr,
                          double pm_r21 = 0.0, double pm_idt = 0.0, int pm_L = 0) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ky = blockIdx.y;
  if (kx >= lhx) return;
  const long col = (long)ky * lhx + kx;  // tables and the FP64 sweep scratch
  const long sp = (long)ny * lhx;
  const long icol = (long)ky * ipitch + kx;  // input spectra (rows ipitch apart)
  const long isp = (long)ny * ipitch;
  const long ocol = (long)ky * opitch + kx;
  const long osp = (long)ny * opitch;
  if (kx == lhx - 1 || ky == ny / 2) {
    for (int l = 0; l <= nz + 1; ++l) phat[l * osp + ocol] = cplx<O>{O(0), O(0)};
    return;
  }
  const bool mean = (kx == 0 && ky == 0);
  const double a_in = 1.0 / (dz * dz);
  const double kxv = kkx[col], kyv = kky[col];
  const double b_in = -((kxv * kxv + kyv * kyv) + 2.0 / (dz * dz));
  // row 1: bottom Neumann closure (p1 - p0 = dz * bottom layer) or p0 = 0
  cplx<double> r;
  if (mean) r = {0.0, 0.0};
  else r = {double(bot[icol].x) * dz, double(bot[icol].y) * dz};
  double bet = mean ? 1.0 : -1.0;
  double cprev = mean ? 0.0 : 1.0;
  cplx<double> x = {r.x / bet, r.y / bet};
  xs[col] = x;
  bool bad = false;
  // One FP64 reciprocal per level: the recurrence multiplies by 1/bet and
  // 1/dz where the reference divides (compute_pressure.f90:473-478).  A
  // division is a long dependent instruction sequence, and with one thread
  // per system (~7 warps per SM) nothing hides its latency; the results
  // differ from dividing by rounding only (an ulp per operation).
  double ib = 1.0 / bet;
  const double idz = 1.0 / dz;
  // The levels are loaded in batches of TB: the loads of the next batch are
  // issued before the recurrence runs through the current one, so that a
  // thread keeps 2 TB levels of reads in flight (the grid holds only one
  // thread per (kx, ky), too few warps to hide DRAM latency otherwise).
  // Hz(k+1) of one level is Hz(k) of the next.
  constexpr int TB = 4;
  cplx<T> hz = Hz[isp + icol];
  cplx<T> cx[TB], cy[TB], cz[TB], cg[TB];
  auto load_fwd = [&](int k0, cplx<T>* ax, cplx<T>* ay, cplx<T>* az, cplx<T>* agg) {
#pragma unroll
    for (int j = 0; j < TB; ++j) {
      const int k = k0 + j;
      const long o = (long)k * isp + icol;
      ax[j] = (k <= nz) ? Hx[o] : cplx<T>{T(0), T(0)};
      ay[j] = (k <= nz) ? Hy[o] : cplx<T>{T(0), T(0)};
      az[j] = (k < nz) ? Hz[o + isp] : cplx<T>{T(0), T(0)};
      if constexpr (INC) agg[j] = (k <= nz) ? G[o] : cplx<T>{T(0), T(0)};
    }
  };
  load_fwd(1, cx, cy, cz, cg);
  for (int k0 = 1; k0 <= nz; k0 += TB) {
    cplx<T> nx_[TB], ny_[TB], nz_[TB], ng_[TB];
    load_fwd(k0 + TB, nx_, ny_, nz_, ng_);
#pragma unroll
    for (int j = 0; j < TB; ++j) {
      const int k = k0 + j;
      if (k <= nz) {
        const long o = (long)k * sp + col;
        const cplx<T> hx = cx[j], hy = cy[j], hzp = cz[j];
        const double sx = kxv * double(hx.x) + kyv * double(hy.x);
        const double sy = kxv * double(hx.y) + kyv * double(hy.y);
        r = {-sy + (double(hzp.x) - double(hz.x)) * idz, sx + (double(hzp.y) - double(hz.y)) * idz};
        if constexpr (INC) {
          r.x += double(cg[j].x);
          r.y += double(cg[j].y);
        }
        if (INC && mean) {
          const double hk = pm[k] + pm_r21 * pm[pm_L + k];
          const double hkp = (k < nz) ? pm[k + 1] + pm_r21 * pm[pm_L + k + 1] : 0.0;
          r = {(hkp - hk) / dz + ((pm[2 * pm_L + k] + pm[3 * pm_L + k]) + pm[4 * pm_L + k]) * pm_idt, 0.0};
        }
        const double g = cprev * ib;
        bet = b_in - a_in * g;
        bad |= (bet == 0.0);
        ib = 1.0 / bet;
        x = {(r.x - a_in * x.x) * ib, (r.y - a_in * x.y) * ib};
        gam[o] = g;
        xs[o] = x;
        cprev = a_in;
        hz = hzp;
      }
    }
#pragma unroll
    for (int j = 0; j < TB; ++j) {
      cx[j] = nx_[j];
      cy[j] = ny_[j];
      cz[j] = nz_[j];
      if constexpr (INC) cg[j] = ng_[j];
    }
  }
  {  // top row: -p(nz) + p(nz+1) = dz * top layer
    const long o = (long)(nz + 1) * sp + col;
    r = {double(top[icol].x) * dz, double(top[icol].y) * dz};
    const double g = cprev * ib;
    bet = 1.0 - (-1.0) * g;
    bad |= (bet == 0.0);
    ib = 1.0 / bet;
    x = {(r.x - (-1.0) * x.x) * ib, (r.y - (-1.0) * x.y) * ib};
    gam[o] = g;
  }
  if (bad) atomicOr(status, ST_PIVOT);
  phat[(long)(nz + 1) * osp + ocol] = cplx<O>{O(0), O(0)};
  // backward sweep, levels nz..0, batched the same way
  cplx<double> bxs[TB];
  double bg[TB];
  auto load_bwd = [&](int k0, cplx<double>* axs, double* ag) {
#pragma unroll
    for (int j = 0; j < TB; ++j) {
      const int k = k0 - j;
      const long o = (long)k * sp + col;
      axs[j] = (k >= 0) ? xs[o] : cplx<double>{0.0, 0.0};
      ag[j] = (k >= 0) ? gam[o + sp] : 0.0;
    }
  };
  load_bwd(nz, bxs, bg);
  for (int k0 = nz; k0 >= 0; k0 -= TB) {
    cplx<double> nxs[TB];
    double ng[TB];
    load_bwd(k0 - TB, nxs, ng);
#pragma unroll
    for (int j = 0; j < TB; ++j) {
      const int k = k0 - j;
      if (k >= 0) {
        x = {bxs[j].x - bg[j] * x.x, bxs[j].y - bg[j] * x.y};
        if (mean && pmean) pmean[k] = x.x;
        phat[k * osp + ocol] = (mean && drop_mean) ? cplx<O>{O(0), O(0)} : cplx<O>{O(x.x), O(x.y)};
      }
    }
#pragma unroll
    for (int j = 0; j < TB; ++j) {
      bxs[j] = nxs[j];
      bg[j] = ng[j];
    }
  }
  if (mean && pmean) pmean[nz + 1] = 0.0;
}

// ---------------------------------------------------------------------------
// running diagnostics (running_diagnostics.f90:148-305) with Neumaier sums
struct Neu {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ void merge(const Neu& o) {
    add(o.s);
    c += o.c;
  }
  __device__ __forceinline__ double val() const { return s + c; }
};

constexpr int DIAG_BLOCKS = 1184;
constexpr int DIAG_NV = 9;  // umax vmax wmax | usum vsum wsum divsum | nan | u* sum

// Per-thread partials of the diagnostics, combined in a fixed order: a
// shuffle tree within each warp (lane 0 keeps the result), then the warps in
// order.  The maxima and the NaN flag do not depend on the order; the
// compensated sums give the same bits on every run.
struct DiagAcc {
  double mx[3] = {-1234567890.0, -1234567890.0, -1234567890.0};
  Neu sum[5];  // u, v, w (uvp node), (div u)^2, u*
  double nan = 0.0;
  __device__ __forceinline__ void merge(const DiagAcc& o) {
    for (int i = 0; i < 3; ++i) mx[i] = fmax(mx[i], o.mx[i]);
    for (int i = 0; i < 5; ++i) sum[i].merge(o.sum[i]);
    nan = fmax(nan, o.nan);
  }
  __device__ __forceinline__ void warp_reduce() {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      DiagAcc o;
      for (int i = 0; i < 3; ++i) o.mx[i] = __shfl_down_sync(0xffffffffu, mx[i], off);
      for (int i = 0; i < 5; ++i) {
        o.sum[i].s = __shfl_down_sync(0xffffffffu, sum[i].s, off);
        o.sum[i].c = __shfl_down_sync(0xffffffffu, sum[i].c, off);
      }
      o.nan = __shfl_down_sync(0xffffffffu, nan, off);
      merge(o);
    }
  }
};

// block reduction of DiagAcc (blockDim.x == 256): the result is valid in thread 0
__device__ __forceinline__ void diag_block_reduce(DiagAcc& a) {
  constexpr int NW = 14;  // mx[3], sum[5] (s, c), nan
  __shared__ double wsum[8][NW];
  a.warp_reduce();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    double* r = wsum[wid];
    for (int i = 0; i < 3; ++i) r[i] = a.mx[i];
    for (int i = 0; i < 5; ++i) {
      r[3 + 2 * i] = a.sum[i].s;
      r[4 + 2 * i] = a.sum[i].c;
    }
    r[13] = a.nan;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < 8; ++w) {
      DiagAcc o;
      const double* r = wsum[w];
      for (int i = 0; i < 3; ++i) o.mx[i] = r[i];
      for (int i = 0; i < 5; ++i) {
        o.sum[i].s = r[3 + 2 * i];
        o.sum[i].c = r[4 + 2 * i];
      }
      o.nan = r[13];
      a.merge(o);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_diag_partial(const T* u, const T* v, const T* w, const T* dudx,
                                                      const T* dvdy, const T* dwdz, const T* ustar, long plane,
                                                      int nz, double* part) {
  DiagAcc a;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < plane; q += (long)gridDim.x * blockDim.x)
    a.sum[4].add(double(ustar[q]));
  const long n = (long)nz * plane;
  int nan = 0;
  auto point = [&](double uu, double vv, double ww, double wu, double dx, double dy, double dz) {
    nan |= (uu != uu) | (vv != vv) | (ww != ww);
    a.mx[0] = fmax(a.mx[0], fabs(uu));
    a.mx[1] = fmax(a.mx[1], fabs(vv));
    a.mx[2] = fmax(a.mx[2], fabs(ww));
    a.sum[0].add(uu);
    a.sum[1].add(vv);
    a.sum[2].add(0.5 * (ww + wu));
    const double dv = dx + dy + dz;
    a.sum[3].add(dv * dv);
  };
  if (plane % 4 == 0) {
    // four consecutive points per thread and iteration: all 28 loads are
    // issued (as 16-byte vectors for FP32) before the compensated sums run
    const long n4 = n / 4;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n4; q += (long)gridDim.x * blockDim.x) {
      const long o = plane + 4 * q;
      T U[4], V[4], W[4], WU[4], DX[4], DY[4], DZ[4];
      ld4(u + o, U);
      ld4(v + o, V);
      ld4(w + o, W);
      ld4(w + o + plane, WU);
      ld4(dudx + o, DX);
      ld4(dvdy + o, DY);
      ld4(dwdz + o, DZ);
      // the four points' values summed in plain FP64, then one compensated
      // addition per sum (the compensated sum is the cost, not the loads)
      double su = 0.0, sv = 0.0, sw = 0.0, sd = 0.0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double uu = U[i], vv = V[i], ww = W[i];
        nan |= (uu != uu) | (vv != vv) | (ww != ww);
        a.mx[0] = fmax(a.mx[0], fabs(uu));
        a.mx[1] = fmax(a.mx[1], fabs(vv));
        a.mx[2] = fmax(a.mx[2], fabs(ww));
        su += uu;
        sv += vv;
        sw += 0.5 * (ww + double(WU[i]));
        const double dv = double(DX[i]) + double(DY[i]) + double(DZ[i]);
        sd += dv * dv;
      }
      a.sum[0].add(su);
      a.sum[1].add(sv);
      a.sum[2].add(sw);
      a.sum[3].add(sd);
    }
  } else {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
      const long o = plane + q;
      point(u[o], v[o], w[o], w[o + plane], dudx[o], dvdy[o], dwdz[o]);
    }
  }
  a.nan = nan;
  diag_block_reduce(a);
  if (threadIdx.x == 0) {
    double* out = part + (long)blockIdx.x * DIAG_NV;
    for (int i = 0; i < 3; ++i) out[i] = a.mx[i];
    for (int q = 0; q < 4; ++q) out[3 + q] = a.sum[q].val();
    out[7] = a.nan;
    out[8] = a.sum[4].val();
  }
}

__global__ void __launch_bounds__(256) k_diag_final(const double* part, int nblocks, long plane, double dt,
                                                    double dx, double dy, double dz, double npts, double* out,
                                                    unsigned* status) {
  // fixed-order combination of the block partials (deterministic)
  DiagAcc a;
  a.mx[0] = a.mx[1] = a.mx[2] = -1e300;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    const double* q = part + (long)b * DIAG_NV;
    for (int i = 0; i < 3; ++i) a.mx[i] = fmax(a.mx[i], q[i]);
    for (int i = 0; i < 4; ++i) a.sum[i].add(q[3 + i]);
    a.sum[4].add(q[8]);
    a.nan = fmax(a.nan, q[7]);
  }
  diag_block_reduce(a);
  if (threadIdx.x == 0) {
    const double cfl = dt * (a.mx[0] / dx + a.mx[1] / dy + a.mx[2] / dz);
    const double um = a.sum[0].val() / npts, vm = a.sum[1].val() / npts, wm = a.sum[2].val() / npts;
    out[0] = cfl;
    out[1] = 0.5 * (um * um + vm * vm + wm * wm);
    out[2] = a.sum[4].val() / double(plane);
    out[3] = sqrt(a.sum[3].val() / npts);
    if (a.nan != 0.0) atomicOr(status, ST_NAN);
  }
}

// ---------------------------------------------------------------------------
// scalar transport, buoyancy and momentum forcing

// Plane means (FP64, Neumaier) of up to six fields on levels k0..k0 +
// gridDim.x - 1: one block per level, out[f * L + k].  Fixed reduction order
// (per thread, then threads in order), so repeated runs give the same bits.
template <typename T>
__global__ void k_plane_means(const T* f0, const T* f1, const T* f2, const T* f3, int nf, double* out, long plane,
                              int k0, int L, const T* f4 = nullptr, const T* f5 = nullptr) {
  const int k = k0 + blockIdx.x;
  const T* fs[6] = {f0, f1, f2, f3, f4, f5};
  __shared__ double sh[6][2][256];
  for (int f = 0; f < nf; ++f) {
    Neu a;
    const T* x = fs[f] + (long)k * plane;
    for (long p = threadIdx.x; p < plane; p += blockDim.x) a.add(double(x[p]));
    sh[f][0][threadIdx.x] = a.s;
    sh[f][1][threadIdx.x] = a.c;
  }
  __syncthreads();
  if (threadIdx.x < nf) {
    const int f = threadIdx.x;
    Neu t;
    for (int i = 0; i < blockDim.x; ++i) {
      t.add(sh[f][0][i]);
      t.add(sh[f][1][i]);
    }
    out[f * L + k] = t.val() / double(plane);
  }
}

// Plane-averaged least-squares coefficient per level k = 1..nz+1 (one block
// per level): kapd[k] = max(0, <KX> / <XX>) * scale (FP64 Neumaier sums; 0
// where <XX> = 0), the reduction of compute_DynSmag.f90:61-245 written to a
// per-level array.
template <typename T>
__global__ void k_level_ratio(const T* KX, const T* XX, double* kapd, long plane, double scale) {
  const int k = blockIdx.x + 1;
  __shared__ double sh[4][256];
  Neu a, b;
  for (long p = threadIdx.x; p < plane; p += blockDim.x) {
    a.add(double(KX[(long)k * plane + p]));
    b.add(double(XX[(long)k * plane + p]));
  }
  sh[0][threadIdx.x] = a.s;
  sh[1][threadIdx.x] = a.c;
  sh[2][threadIdx.x] = b.s;
  sh[3][threadIdx.x] = b.c;
  __syncthreads();
  if (threadIdx.x == 0) {
    Neu x, y;
    for (int i = 0; i < blockDim.x; ++i) {
      x.add(sh[0][i]);
      x.add(sh[1][i]);
      y.add(sh[2][i]);
      y.add(sh[3][i]);
    }
    const double num = x.val() / double(plane), den = y.val() / double(plane);
    const double c = (den != 0.0) ? num / den : 0.0;
    kapd[k] = fmax(0.0, c) * scale;
  }
}

// Wall value of d theta/dz (level 1): the log law of the prescribed surface
// flux, -qs / (kappa u* dz/2), zero where u* = 0.
template <typename T>
__global__ void k_scalar_wall(T* dtdz1, const T* ustar, long plane, double qs, double half_dz) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < plane; p += (long)gridDim.x * blockDim.x) {
    const double us = double(ustar[p]);
    dtdz1[p] = (us != 0.0) ? T(-qs / (KVONK * us * half_dz)) : T(0);
  }
}

// step_scalars (compute_scalars.f90:111-125): theta += dt (t1 rhs + t2 rhs_f)
// on levels 1..nz (the ghost values follow with k_scalar_bc)
template <typename T>
__global__ void k_ab2_scalar(T* th, const T* r, const T* rf, long plane, int nz, T dt, T t1, T t2) {
  const long n = (long)nz * plane;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long o = plane + q;
    th[o] = th[o] + dt * (t1 * r[o] + t2 * rf[o]);
  }
}

// Ghost values of theta (compute_scalars.f90:127-133 with a lid gradient):
// theta(0) = 0, theta(nz+1) = theta(nz) + g_top dz.
template <typename T>
__global__ void k_scalar_bc(T* th, long plane, int nz, T gdz) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < plane; p += (long)gridDim.x * blockDim.x) {
    th[p] = T(0);
    th[(long)(nz + 1) * plane + p] = th[(long)nz * plane + p] + gdz;
  }
}

// Coriolis (LES_engine.f90:553-561) and the sponge (sponge_damping.f90:131-161)
// on levels 1..nz.  mean[0*L + k], mean[1*L + k], mean[2*L + k]: plane means
// of u, v, w; sp[k]: the sponge profile on w nodes (nullptr: none).
template <typename T>
__global__ void k_forcing(T* rx, T* ry, T* rz, const T* u, const T* v, const T* w, const double* mean,
                          const double* sp, long plane, int nz, int L, T f, T ug, T vg) {
  const long n = (long)nz * plane;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long o = plane + q;
    const int k = udiv32(o, plane);
    const T uo = u[o], vo = v[o];
    T x = rx[o], y = ry[o];
    if (f != T(0)) {
      x = x + f * vo - f * vg;
      y = y - f * uo + f * ug;
    }
    if (sp) {
      const T sh = T(0.5 * (sp[k] + sp[k + 1]));
      x = x - sh * (uo - T(mean[k]));
      y = y - sh * (vo - T(mean[L + k]));
      rz[o] = rz[o] - T(sp[k]) * (w[o] - T(mean[2 * L + k]));
    }
    rx[o] = x;
    ry[o] = y;
  }
}

// Buoyancy on w nodes k = 2..nz: rz += beta (theta_w - <theta_w>),
// theta_w(k) = (theta(k) + theta(k-1)) / 2; tmean = plane means of theta.
template <typename T>
__global__ void k_buoyancy(T* rz, const T* th, const double* tmean, long plane, int nz, T beta) {
  const long n = (long)(nz - 1) * plane;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long o = 2 * plane + q;
    const int k = udiv32(o, plane);
    const T tw = T(0.5) * (th[o] + th[o - plane]);
    const T twm = T(0.5 * (tmean[k] + tmean[k - 1]));
    rz[o] = rz[o] + beta * (tw - twm);
  }
}

// ---------------------------------------------------------------------------
// pressure systems of a z-slab decomposition: the partition method.  Slab b
// of G owns rows [s_b, e_b] of every (kx, ky) column (rows 0..nz+1: the
// bottom closure row, nz interior rows, the top row; slab b holds levels
// b m + 1 .. (b+1) m, m = nz/G, plus row 0 on the first and row nz+1 on
// the last slab).  k_tri_slab_local eliminates a slab's rows with three
// right-hand sides (r, and the unit couplings -a e_first, -c e_last to the
// neighbouring slabs' boundary unknowns) into y, u, v; k_tri_slab_reduced
// solves the 2G boundary unknowns of each column (2 x 2 block Thomas);
// k_tri_slab_back forms x = y + u x_left + v x_right.  Same matrix,
// right-hand side and outputs as k_tridiag (compute_pressure.f90:256-305,
// 448-493, 544-619); only the elimination order differs.
struct SlabRows {
  int G, m, nz;
  __host__ __device__ int start(int b) const { return b == 0 ? 0 : b * m + 1; }
  __host__ __device__ int end(int b) const { return b < G - 1 ? (b + 1) * m : nz + 1; }
  __host__ __device__ int of_row(int k) const { return k == 0 ? 0 : min((k - 1) / m, G - 1); }
};

// row k of a column: coefficients (a, b, c) and the right-hand side
template <typename T>
__device__ __forceinline__ void tri_row(int k, int nz, bool mean, double a_in, double b_in, double dz, double kxv,
                                        double kyv, const cplx<T>* Hx, const cplx<T>* Hy, const cplx<T>* Hz,
                                        const cplx<T>* bot, const cplx<T>* top, long icol, long isp, double& a,
                                        double& b, double& c, cplx<double>& r) {
  if (k == 0) {
    a = 0.0;
    b = mean ? 1.0 : -1.0;
    c = mean ? 0.0 : 1.0;
    r = mean ? cplx<double>{0.0, 0.0} : cplx<double>{double(bot[icol].x) * dz, double(bot[icol].y) * dz};
  } else if (k == nz + 1) {
    a = -1.0;
    b = 1.0;
    c = 0.0;
    r = {double(top[icol].x) * dz, double(top[icol].y) * dz};
  } else {
    a = a_in;
    b = b_in;
    c = a_in;
    const long o = (long)k * isp + icol;
    const cplx<T> hx = Hx[o], hy = Hy[o], hz = Hz[o];
    const cplx<T> hzp = (k < nz) ? Hz[o + isp] : cplx<T>{T(0), T(0)};
    const double sx = kxv * double(hx.x) + kyv * double(hy.x);
    const double sy = kxv * double(hx.y) + kyv * double(hy.y);
    r = {-sy + (double(hzp.x) - double(hz.x)) / dz, sx + (double(hzp.y) - double(hz.y)) / dz};
  }
}

// grid (ceil(lhx/64), ny, G), 64 threads: one (column, slab) per thread.
// ys (complex), uu, vv: the slab's solutions at its rows; gam: scratch.
template <typename T>
__global__ void k_tri_slab_local(const cplx<T>* __restrict__ Hx, const cplx<T>* __restrict__ Hy,
                                 const cplx<T>* __restrict__ Hz, const cplx<T>* __restrict__ bot,
                                 const cplx<T>* __restrict__ top, const double* __restrict__ kkx,
                                 const double* __restrict__ kky, cplx<double>* __restrict__ ys,
                                 double* __restrict__ uu, double* __restrict__ vv, double* __restrict__ gam,
                                 unsigned* status, int lhx, int ny, int nz, double dz, int ipitch, SlabRows sr) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ky = blockIdx.y;
  const int sb = blockIdx.z;
  if (kx >= lhx || kx == lhx - 1 || ky == ny / 2) return;  // Nyquist columns: zero (k_tri_slab_back)
  const long col = (long)ky * lhx + kx, sp = (long)ny * lhx;
  const long icol = (long)ky * ipitch + kx, isp = (long)ny * ipitch;
  const bool mean = (kx == 0 && ky == 0);
  const double a_in = 1.0 / (dz * dz);
  const double kxv = kkx[col], kyv = kky[col];
  const double b_in = -((kxv * kxv + kyv * kyv) + 2.0 / (dz * dz));
  const int s = sr.start(sb), e = sr.end(sb);
  double a, b, c;
  cplx<double> r;
  tri_row<T>(s, nz, mean, a_in, b_in, dz, kxv, kyv, Hx, Hy, Hz, bot, top, icol, isp, a, b, c, r);
  double bet = b;
  bool bad = (bet == 0.0);
  cplx<double> y = {r.x / bet, r.y / bet};
  double u = (sb > 0 ? -a : 0.0) / bet;
  double cprev = c;
  double v = (e == s && sb < sr.G - 1) ? -c / bet : 0.0;
  ys[(long)s * sp + col] = y;
  uu[(long)s * sp + col] = u;
  vv[(long)s * sp + col] = v;
  for (int k = s + 1; k <= e; ++k) {
    tri_row<T>(k, nz, mean, a_in, b_in, dz, kxv, kyv, Hx, Hy, Hz, bot, top, icol, isp, a, b, c, r);
    const double g = cprev / bet;
    bet = b - a * g;
    bad |= (bet == 0.0);
    const double rv = (k == e && sb < sr.G - 1) ? -c : 0.0;
    y = {(r.x - a * y.x) / bet, (r.y - a * y.y) / bet};
    u = (0.0 - a * u) / bet;
    v = (rv - a * v) / bet;
    const long o = (long)k * sp + col;
    gam[o] = g;
    ys[o] = y;
    uu[o] = u;
    vv[o] = v;
    cprev = c;
  }
  for (int k = e - 1; k >= s; --k) {
    const long o = (long)k * sp + col;
    const double g = gam[o + sp];
    y = {ys[o].x - g * y.x, ys[o].y - g * y.y};
    u = uu[o] - g * u;
    v = vv[o] - g * v;
    ys[o] = y;
    uu[o] = u;
    vv[o] = v;
  }
  if (bad) atomicOr(status, ST_PIVOT);
}

// one column per thread: the boundary unknowns X_s^b, X_e^b of every slab
// (block Thomas over 2 x 2 blocks), written as the neighbours' values each
// slab needs: xlr[(col G + b) 2 + 0] = X_e^{b-1}, [.. + 1] = X_s^{b+1}
constexpr int MAX_SLABS = 64;
__global__ void k_tri_slab_reduced(const cplx<double>* __restrict__ ys, const double* __restrict__ uu,
                                   const double* __restrict__ vv, cplx<double>* __restrict__ xlr, unsigned* status,
                                   int lhx, int ny, SlabRows sr) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ky = blockIdx.y;
  if (kx >= lhx || kx == lhx - 1 || ky == ny / 2) return;
  const long col = (long)ky * lhx + kx, sp = (long)ny * lhx;
  const int G = sr.G;
  // forward elimination; keep the modified blocks (first column only
  // changes) and right-hand sides
  double p00[MAX_SLABS], p10[MAX_SLABS];
  cplx<double> y0[MAX_SLABS], y1[MAX_SLABS];
  bool bad = false;
  for (int b = 0; b < G; ++b) {
    const long os = (long)sr.start(b) * sp + col, oe = (long)sr.end(b) * sp + col;
    const double us = uu[os], ue = uu[oe];
    cplx<double> a0 = ys[os], a1 = ys[oe];
    double b00 = 1.0, b10 = 0.0;
    if (b > 0) {
      // p01 = 0, p11 = 1 for every modified block
      const double det = p00[b - 1];
      bad |= (det == 0.0);
      const double i10 = -p10[b - 1] / det, i11 = p00[b - 1] / det;
      const long ops = (long)sr.start(b - 1) * sp + col, ope = (long)sr.end(b - 1) * sp + col;
      const double w0 = i10 * (-vv[ops]) + i11 * (-vv[ope]);
      const cplx<double> z = {i10 * y0[b - 1].x + i11 * y1[b - 1].x, i10 * y0[b - 1].y + i11 * y1[b - 1].y};
      b00 = b00 + us * w0;
      b10 = b10 + ue * w0;
      a0 = {a0.x + us * z.x, a0.y + us * z.y};
      a1 = {a1.x + ue * z.x, a1.y + ue * z.y};
    }
    p00[b] = b00;
    p10[b] = b10;
    y0[b] = a0;
    y1[b] = a1;
  }
  cplx<double> xs_next = {0.0, 0.0};  // X_s^{b+1}
  for (int b = G - 1; b >= 0; --b) {
    cplx<double> r0 = y0[b], r1 = y1[b];
    if (b < G - 1) {
      const double vs = vv[(long)sr.start(b) * sp + col], ve = vv[(long)sr.end(b) * sp + col];
      r0 = {r0.x + vs * xs_next.x, r0.y + vs * xs_next.y};
      r1 = {r1.x + ve * xs_next.x, r1.y + ve * xs_next.y};
    }
    const double det = p00[b];  // p01 = 0, p11 = 1
    bad |= (det == 0.0);
    const cplx<double> Xs = {r0.x / det, r0.y / det};
    const cplx<double> Xe = {(-p10[b] * r0.x + p00[b] * r1.x) / det, (-p10[b] * r0.y + p00[b] * r1.y) / det};
    // slab b + 1 needs X_e^b as its left value, slab b - 1 needs X_s^b
    if (b + 1 < G) xlr[(col * G + b + 1) * 2 + 0] = Xe;
    if (b > 0) xlr[(col * G + b - 1) * 2 + 1] = Xs;
    xs_next = Xs;
  }
  xlr[(col * G + 0) * 2 + 0] = {0.0, 0.0};
  xlr[(col * G + G - 1) * 2 + 1] = {0.0, 0.0};
  if (bad) atomicOr(status, ST_PIVOT);
}

// grid (ceil(lhx/64), ny, nz + 2): x = y + u x_left + v x_right into phat
// (the outputs of k_tridiag: phat(nz+1) = 0; the mean mode kept apart in
// FP64 as pmean with drop_mean)
template <typename O>
__global__ void k_tri_slab_back(const cplx<double>* __restrict__ ys, const double* __restrict__ uu,
                                const double* __restrict__ vv, const cplx<double>* __restrict__ xlr,
                                cplx<O>* __restrict__ phat, double* pmean, int lhx, int ny, int nz, int drop_mean,
                                int opitch, SlabRows sr) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ky = blockIdx.y;
  const int k = blockIdx.z;
  if (kx >= lhx) return;
  const long col = (long)ky * lhx + kx, sp = (long)ny * lhx;
  const long oo = (long)k * ny * opitch + (long)ky * opitch + kx;
  if (kx == lhx - 1 || ky == ny / 2 || k == nz + 1) {
    phat[oo] = cplx<O>{O(0), O(0)};
    if (kx == 0 && ky == 0 && pmean && k == nz + 1) pmean[k] = 0.0;
    return;
  }
  const bool mean = (kx == 0 && ky == 0);
  const int b = sr.of_row(k);
  const long o = (long)k * sp + col;
  const cplx<double> xl = xlr[(col * sr.G + b) * 2 + 0], xr = xlr[(col * sr.G + b) * 2 + 1];
  const double u = uu[o], v = vv[o];
  const cplx<double> x = {ys[o].x + u * xl.x + v * xr.x, ys[o].y + u * xl.y + v * xr.y};
  if (mean && pmean) pmean[k] = x.x;
  phat[oo] = (mean && drop_mean) ? cplx<O>{O(0), O(0)} : cplx<O>{O(x.x), O(x.y)};
}

}  // namespace les
