// FP64 CPU restatement of the LES time step, threaded with OpenMP -- TEST AND
// BASELINE INFRASTRUCTURE ONLY.  It is the compiled form of oracle/les_oracle.py
// (same routines, same order of operations where they matter: the REAL(4)
// clips of compute_LagScaleDep.f90, the update_halo3 mirror copies of a 1x1
// process grid, the Thomas solve per (kx, ky)), used as the timed CPU
// baseline of bench.py (the host-cores port of the reference's algorithm) and
// checked against the numpy oracle by tests/test_cpu_step.py.  Nothing in the
// product path loads it.
//
// Scope: the configuration the benchmark runs -- wall law with the 2-Delta
// filtered first level (wall_filter), the Lagrangian scale-dependent dynamic
// model (dyn_LagScaleDep, reference1x1 halos), 3/2-padded convection, the
// staggered pressure solve -- plus the constant-coefficient model.
//
// Layout: fields are double[L][ny][nx] with L = nz + 2 (the Fortran
// (nx, ny, 0:nz+1) array); half spectra are complex[ny][nx/2 + 1].  FFTs are
// unnormalised in both directions (FFTW's convention) and written here: a
// mixed-radix (2, 3, 4) Stockham transform, two real rows packed into one
// complex transform for the r2c / c2r steps.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <omp.h>

namespace {

using cd = std::complex<double>;
constexpr double PI = 3.1415926535897932384626433;  // parameters_IO.f90:42
constexpr double KVONK = 0.4;
constexpr double BOGUS = -1.23456789e20;
constexpr double TF1 = 2.0, TF1_2 = 4.0, TF2 = 4.0, TF2_2 = 16.0, OPFTIME = 1.5;  // compute_LagScaleDep.f90:27-29

// ------------------------------------------------------------------ FFT ----
// Stockham autosort, decimation in frequency: a pass of radix r on blocks of
// length n (stride s, m = n / r) maps x[q + s (p + t m)] to
// y[q + s (r p + u)] = W_n^{p u} sum_t x[q + s (p + t m)] W_r^{t u}; the
// passes run until n = 1 and leave the transform in natural order.
struct Plan {
  int n = 0;
  struct Stage {
    int r, n, m, s;
    std::vector<cd> tw;  // [p][u - 1], forward sign
  };
  std::vector<Stage> st;
};

Plan make_plan(int n) {
  Plan P;
  P.n = n;
  std::vector<int> rad;
  int k = n;
  while (k % 4 == 0) { rad.push_back(4); k /= 4; }
  while (k % 2 == 0) { rad.push_back(2); k /= 2; }
  while (k % 3 == 0) { rad.push_back(3); k /= 3; }
  if (k != 1) throw std::runtime_error("FFT length must be 2^a 3^b");
  int len = n, s = 1;
  for (int r : rad) {
    Plan::Stage S;
    S.r = r;
    S.n = len;
    S.m = len / r;
    S.s = s;
    S.tw.resize((size_t)S.m * (r - 1));
    for (int p = 0; p < S.m; ++p)
      for (int u = 1; u < r; ++u) {
        const double a = -2.0 * PI * double((long)p * u % len) / double(len);
        S.tw[(size_t)p * (r - 1) + (u - 1)] = cd(std::cos(a), std::sin(a));
      }
    P.st.push_back(std::move(S));
    len /= r;
    s *= r;
  }
  return P;
}

const Plan& plan_for(int n) {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<Plan>> plans;
  std::lock_guard<std::mutex> lock(mu);
  auto it = plans.find(n);
  if (it == plans.end()) it = plans.emplace(n, std::make_unique<Plan>(make_plan(n))).first;
  return *it->second;
}

// one Stockham pass of radix R (INV: exponent sign +, conjugate twiddles),
// compiled per radix and direction so the butterfly loops carry no branches
template <int R, bool INV>
inline void fft_bfly(const cd* __restrict in, cd* __restrict out, int p, int q, int m, int s, const cd* tw) {
  constexpr double sg = INV ? 1.0 : -1.0;
  auto w = [&](int u) { return INV ? std::conj(tw[u]) : tw[u]; };
  if constexpr (R == 2) {
    const cd a = in[q + s * p], b = in[q + s * (p + m)];
    out[q + s * (2 * p)] = a + b;
    out[q + s * (2 * p + 1)] = (a - b) * w(0);
  } else if constexpr (R == 4) {
    const cd a0 = in[q + s * p], a1 = in[q + s * (p + m)], a2 = in[q + s * (p + 2 * m)],
             a3 = in[q + s * (p + 3 * m)];
    const cd t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = a1 - a3;
    const cd jt3(-sg * t3.imag(), sg * t3.real());  // sg i t3
    out[q + s * (4 * p)] = t0 + t2;
    out[q + s * (4 * p + 1)] = (t1 + jt3) * w(0);
    out[q + s * (4 * p + 2)] = (t0 - t2) * w(1);
    out[q + s * (4 * p + 3)] = (t1 - jt3) * w(2);
  } else {  // R == 3
    constexpr double s3 = 0.86602540378443864676;  // sqrt(3) / 2
    const cd a0 = in[q + s * p], a1 = in[q + s * (p + m)], a2 = in[q + s * (p + 2 * m)];
    const cd t1 = a1 + a2, t2 = a1 - a2;
    const cd mm = a0 - 0.5 * t1;
    const cd st(-sg * s3 * t2.imag(), sg * s3 * t2.real());  // sg i sqrt(3)/2 t2
    out[q + s * (3 * p)] = a0 + t1;
    out[q + s * (3 * p + 1)] = (mm + st) * w(0);
    out[q + s * (3 * p + 2)] = (mm - st) * w(1);
  }
}
template <int R, bool INV>
void fft_pass(const Plan::Stage& S, const cd* __restrict in, cd* __restrict out) {
  const int m = S.m, s = S.s;
  const cd* tw = S.tw.data();
  if (s >= m) {  // the longer of the two loops innermost
    for (int p = 0; p < m; ++p)
      for (int q = 0; q < s; ++q) fft_bfly<R, INV>(in, out, p, q, m, s, tw + (size_t)p * (R - 1));
  } else {
    for (int q = 0; q < s; ++q)
      for (int p = 0; p < m; ++p) fft_bfly<R, INV>(in, out, p, q, m, s, tw + (size_t)p * (R - 1));
  }
}

// in-place complex transform of x (work: n values); inv: exponent sign +
void cfft(const Plan& P, cd* x, cd* work, bool inv) {
  cd* in = x;
  cd* out = work;
  for (const auto& S : P.st) {
    switch (S.r * 2 + (inv ? 1 : 0)) {
      case 4: fft_pass<2, false>(S, in, out); break;
      case 5: fft_pass<2, true>(S, in, out); break;
      case 6: fft_pass<3, false>(S, in, out); break;
      case 7: fft_pass<3, true>(S, in, out); break;
      case 8: fft_pass<4, false>(S, in, out); break;
      default: fft_pass<4, true>(S, in, out); break;
    }
    std::swap(in, out);
  }
  if (in != x) std::memcpy(x, in, sizeof(cd) * P.n);
}

// real rows a, b of length n -> half spectra A, B (n/2 + 1 values each), one
// complex transform of z = a + i b
void r2c_pair(int n, const double* a, const double* b, cd* A, cd* B, cd* z, cd* work) {
  const Plan& P = plan_for(n);
  for (int i = 0; i < n; ++i) z[i] = cd(a[i], b ? b[i] : 0.0);
  cfft(P, z, work, false);
  for (int k = 0; k <= n / 2; ++k) {
    const cd zk = z[k], zm = std::conj(z[k == 0 ? 0 : n - k]);
    A[k] = 0.5 * (zk + zm);
    if (B) B[k] = cd(0.0, -0.5) * (zk - zm);
  }
}
// half spectra A, B (imaginary parts of bins 0 and n/2 ignored) -> real rows
// a, b (unnormalised inverse)
void c2r_pair(int n, const cd* A, const cd* B, double* a, double* b, cd* z, cd* work) {
  const Plan& P = plan_for(n);
  const int h = n / 2;
  // bins 0 and n/2: real parts only
  z[0] = cd(A[0].real(), B ? B[0].real() : 0.0);
  z[h] = cd(A[h].real(), B ? B[h].real() : 0.0);
  for (int k = 1; k < h; ++k) {
    const cd x = A[k], y = B ? B[k] : cd(0.0, 0.0);
    z[k] = x + cd(0.0, 1.0) * y;
    z[n - k] = std::conj(x) + cd(0.0, 1.0) * std::conj(y);
  }
  cfft(P, z, work, true);
  for (int i = 0; i < n; ++i) {
    a[i] = z[i].real();
    if (b) b[i] = z[i].imag();
  }
}

// per-thread scratch of the transforms
struct Scratch {
  std::vector<cd> z, w, col;
  std::vector<double> r0, r1;
  void need(int n) {
    if ((int)z.size() < n) {
      z.resize(n);
      w.resize(n);
      col.resize(n);
      r0.resize(n);
      r1.resize(n);
    }
  }
};
Scratch& scratch() {
  static thread_local Scratch s;
  return s;
}

// 2-D r2c of one plane (ny x nx) -> (ny x lhx): x r2c then y c2c, unnormalised
void rfft2_plane(int nx, int ny, const double* f, cd* F) {
  const int lhx = nx / 2 + 1;
  Scratch& S = scratch();
  S.need(std::max(nx, ny) + 2);
  for (int j = 0; j < ny; j += 2)
    r2c_pair(nx, f + (long)j * nx, f + (long)(j + 1) * nx, F + (long)j * lhx, F + (long)(j + 1) * lhx, S.z.data(),
             S.w.data());
  const Plan& P = plan_for(ny);
  for (int k = 0; k < lhx; ++k) {
    for (int j = 0; j < ny; ++j) S.col[j] = F[(long)j * lhx + k];
    cfft(P, S.col.data(), S.w.data(), false);
    for (int j = 0; j < ny; ++j) F[(long)j * lhx + k] = S.col[j];
  }
}
// 2-D c2r: y c2c then x c2r (F is used as scratch), unnormalised
void irfft2_plane(int nx, int ny, cd* F, double* f) {
  const int lhx = nx / 2 + 1;
  Scratch& S = scratch();
  S.need(std::max(nx, ny) + 2);
  const Plan& P = plan_for(ny);
  for (int k = 0; k < lhx; ++k) {
    for (int j = 0; j < ny; ++j) S.col[j] = F[(long)j * lhx + k];
    cfft(P, S.col.data(), S.w.data(), true);
    for (int j = 0; j < ny; ++j) F[(long)j * lhx + k] = S.col[j];
  }
  for (int j = 0; j < ny; j += 2)
    c2r_pair(nx, F + (long)j * lhx, F + (long)(j + 1) * lhx, f + (long)j * nx, f + (long)(j + 1) * nx, S.z.data(),
             S.w.data());
}

}  // namespace

namespace {

// ---------------------------------------------------------------- state ----
// field ids: the order of oracle/les_oracle.py FIELDS
enum Fid {
  U, V, W, DUDX, DUDY, DUDZ, DVDX, DVDY, DVDZ, DWDX, DWDY, DWDZ, P_, DPDX, DPDY, DPDZ, RHSX, RHSY, RHSZ, RHSX_F,
  RHSY_F, RHSZ_F, TXX, TXY, TXZ, TYY, TYZ, TZZ, CS_OPT2, NU_T, F_LM, F_MM, F_QN, F_NN, BETA, U_LAG, V_LAG, W_LAG,
  NFIELD
};
// plane ids: the order of PLANES
enum Pid { LBC_U, LBC_V, LBC_W, UBC_U, UBC_V, UBC_W, BOT_WK, TOP_WK, LBC_Z0, USTAR, NPLANE };

struct Params {
  int nx, ny, nz;
  double dt, lx, ly, lz, dx, dy, dz, z0, pfx, pfy, cs0;
  int sgs;         // 0 constant Smagorinsky, 2 Lagrangian scale-dependent dynamic
  int cs_count, dyn_init;
  int wall_model;  // 0 wall_filter, 1 wall_inst, 2 wall_homog
};

struct State {
  Params p;
  int L, lhx, lhy;
  long npl, nf, nsp;
  std::vector<double> f[NFIELD];
  std::vector<double> pl[NPLANE];
  bool f_coeff_init = false, lagran_init = false;
  int jt_total = 0;
  int lbc_typ[3] = {1, 1, 1};  // 1 Dirichlet, 2 Neumann (u, v, w)
  int ubc_typ[3] = {2, 2, 1};
  std::vector<double> kkx, kky, g2, g4;  // (ny, lhx)
  double delta, beta_pow;
  double* F(int id) { return f[id].data(); }
  double* lev(int id, int k) { return f[id].data() + (long)k * npl; }
};

std::vector<double> test_filter_kernel(const State& s, double alpha, const std::vector<double>& kk2) {
  // testfilter.f90:101-131: cutoff on kk2 rounded to REAL(4), 1/(nx ny) folded in
  const Params& p = s.p;
  std::vector<double> g((size_t)p.ny * s.lhx, 1.0 / double(p.nx * p.ny));
  const double delta = alpha * std::sqrt(p.dx * p.dy);
  const double kc2 = (PI / delta) * (PI / delta);
  for (int j = 0; j < p.ny; ++j)
    for (int i = 0; i < s.lhx; ++i) {
      const size_t q = (size_t)j * s.lhx + i;
      if (double(float(kk2[q])) >= kc2) g[q] = 0.0;
      if (i == s.lhx - 1 || j == p.ny / 2) g[q] = 0.0;
    }
  return g;
}

void init_state(State& s) {
  Params& p = s.p;
  s.L = p.nz + 2;
  s.lhx = p.nx / 2 + 1;
  s.lhy = p.ny / 2 + 1;
  s.npl = (long)p.nx * p.ny;
  s.nf = s.npl * s.L;
  s.nsp = (long)p.ny * s.lhx;
  for (auto& v : s.f) v.assign(s.nf, 0.0);
  for (auto& v : s.pl) v.assign(s.npl, 0.0);
  std::fill(s.pl[LBC_Z0].begin(), s.pl[LBC_Z0].end(), p.z0);
  std::fill(s.f[W].begin(), s.f[W].begin() + s.npl, BOGUS);
  // fft_engine.f90:97-145
  s.kkx.assign(s.nsp, 0.0);
  s.kky.assign(s.nsp, 0.0);
  std::vector<double> kk2(s.nsp);
  for (int j = 0; j < p.ny; ++j)
    for (int i = 0; i < s.lhx; ++i) {
      double kx = double(i), ky = double(((j + p.ny / 2) % p.ny) - p.ny / 2);
      if (i == s.lhx - 1 || j == s.lhy - 1) kx = ky = 0.0;
      const size_t q = (size_t)j * s.lhx + i;
      s.kkx[q] = 2.0 * PI / p.lx * kx;
      s.kky[q] = 2.0 * PI / p.ly * ky;
      kk2[q] = s.kkx[q] * s.kkx[q] + s.kky[q] * s.kky[q];
    }
  s.g2 = test_filter_kernel(s, 2.0, kk2);
  s.g4 = test_filter_kernel(s, 4.0, kk2);
  s.delta = std::pow(p.dx * p.dy * p.dz, 1.0 / 3.0);
  s.beta_pow = std::log(TF1) / (std::log(TF2) - std::log(TF1));
}

// per-thread spectral plane
std::vector<cd>& spec_buf(long n) {
  static thread_local std::vector<cd> b;
  if ((long)b.size() < n) b.resize(n);
  return b;
}
std::vector<cd>& spec_buf2(long n) {
  static thread_local std::vector<cd> b;
  if ((long)b.size() < n) b.resize(n);
  return b;
}
std::vector<double>& real_buf(long n) {
  static thread_local std::vector<double> b;
  if ((long)b.size() < n) b.resize(n);
  return b;
}

void kill_oddballs(const State& s, cd* F) {
  for (int j = 0; j < s.p.ny; ++j) F[(long)j * s.lhx + s.lhx - 1] = 0.0;
  for (int i = 0; i < s.lhx; ++i) F[(long)(s.lhy - 1) * s.lhx + i] = 0.0;
}
// i k X as the reference's (0 + i k) * X evaluates it
inline cd ik(double k, cd x) { return cd(-k * x.imag(), k * x.real()); }

// -------------------------------------------------- compute_derivatives ----
// compute_derivatives.f90:94-137, levels 0..nz+1: f is replaced by its
// Nyquist-filtered self
void grad_velocity_filt(State& s, int fid, int dx_id, int dy_id) {
  const Params& p = s.p;
  const double c = 1.0 / double(p.nx * p.ny);
#pragma omp parallel for schedule(dynamic)
  for (int k = 0; k < s.L; ++k) {
    std::vector<cd>& F = spec_buf(s.nsp);
    std::vector<cd>& G = spec_buf2(s.nsp);
    std::vector<double>& t = real_buf(s.npl);
    double* f = s.lev(fid, k);
    for (long q = 0; q < s.npl; ++q) t[q] = c * f[q];
    rfft2_plane(p.nx, p.ny, t.data(), F.data());
    kill_oddballs(s, F.data());
    for (long q = 0; q < s.nsp; ++q) G[q] = ik(s.kkx[q], F[q]);
    irfft2_plane(p.nx, p.ny, G.data(), s.lev(dx_id, k));
    for (long q = 0; q < s.nsp; ++q) G[q] = ik(s.kky[q], F[q]);
    irfft2_plane(p.nx, p.ny, G.data(), s.lev(dy_id, k));
    irfft2_plane(p.nx, p.ny, F.data(), f);
  }
}

void ddz_uv(State& s, int out, int in) {  // compute_derivatives.f90:375-400
  const double c = 1.0 / s.p.dz;
#pragma omp parallel for
  for (int k = 1; k < s.L; ++k) {
    double* o = s.lev(out, k);
    const double* a = s.lev(in, k);
    const double* b = s.lev(in, k - 1);
    for (long q = 0; q < s.npl; ++q) o[q] = c * (a[q] - b[q]);
  }
}
void ddz_w(State& s, int out, int in) {  // compute_derivatives.f90:413-441
  const double c = 1.0 / s.p.dz;
  const int nz = s.p.nz;
#pragma omp parallel for
  for (int k = 1; k <= nz; ++k) {
    double* o = s.lev(out, k);
    const double* a = s.lev(in, k + 1);
    const double* b = s.lev(in, k);
    for (long q = 0; q < s.npl; ++q) o[q] = c * (a[q] - b[q]);
  }
  std::fill(s.lev(out, nz + 1), s.lev(out, nz + 1) + s.npl, 0.0);
}

// compute_derivatives.f90:464-577: rhs(1..nz) += dx tx + dy ty + dz tz; for
// the w equation (stag false) also the bottom / top pressure-BC layers
void div_stress(State& s, int rhs, int tx, int ty, int tz, bool stag, double* bot, double* top) {
  const Params& p = s.p;
  const int nz = p.nz;
  const double c = 1.0 / double(p.nx * p.ny), rdz = 1.0 / p.dz;
#pragma omp parallel for schedule(dynamic)
  for (int k = 1; k <= nz + 1; ++k) {
    std::vector<cd>& F = spec_buf(s.nsp);
    std::vector<double>& t = real_buf(2 * s.npl);
    double* dtx = t.data();
    double* dty = t.data() + s.npl;
    for (int pass = 0; pass < 2; ++pass) {
      const double* f = s.lev(pass ? ty : tx, k);
      double* o = pass ? dty : dtx;
      for (long q = 0; q < s.npl; ++q) o[q] = c * f[q];
      rfft2_plane(p.nx, p.ny, o, F.data());
      kill_oddballs(s, F.data());
      const std::vector<double>& kv = pass ? s.kky : s.kkx;
      for (long q = 0; q < s.nsp; ++q) F[q] = ik(kv[q], F[q]);
      irfft2_plane(p.nx, p.ny, F.data(), o);
    }
    if (k <= nz) {
      double* r = s.lev(rhs, k);
      const double* z0 = s.lev(tz, k);
      for (long q = 0; q < s.npl; ++q) {
        const double dz = stag ? rdz * (s.lev(tz, k + 1)[q] - z0[q]) : rdz * (z0[q] - s.lev(tz, k - 1)[q]);
        r[q] = r[q] + dtx[q] + dty[q] + dz;
        if (!stag && k == 1 && bot) bot[q] = dtx[q] + dty[q] + dz;
      }
    } else if (!stag && top) {
      for (long q = 0; q < s.npl; ++q) top[q] = dtx[q] + dty[q];
    }
  }
  if (stag) {
    if (bot) std::fill(bot, bot + s.npl, BOGUS);
    if (top) std::fill(top, top + s.npl, BOGUS);
  }
}

// boundary_condition_mpi.f90:33-63; type 1 Dirichlet, 2 Neumann
void set_bc(State& s, bool bottom, int fid, int type, const double* bc, bool stag) {
  const int nz = s.p.nz;
  const long n = s.npl;
  const double dz = s.p.dz;
  if (bottom) {
    double* g = s.lev(fid, 0);
    double* a = s.lev(fid, 1);
    if (stag) {
      if (type == 1) for (long q = 0; q < n; ++q) g[q] = 2.0 * bc[q] - a[q];
      else if (type == 2) for (long q = 0; q < n; ++q) g[q] = a[q] - bc[q] * dz;
    } else if (type == 1) {
      for (long q = 0; q < n; ++q) a[q] = bc[q];
    }
  } else {
    double* g = s.lev(fid, nz + 1);
    double* a = s.lev(fid, nz);
    if (stag) {
      if (type == 1) for (long q = 0; q < n; ++q) g[q] = 2.0 * bc[q] - a[q];
      else if (type == 2) for (long q = 0; q < n; ++q) g[q] = a[q] + bc[q] * dz;
    } else if (type == 1) {
      for (long q = 0; q < n; ++q) g[q] = bc[q];
    }
  }
}
void apply_bcs(State& s) {
  set_bc(s, true, U, s.lbc_typ[0], s.pl[LBC_U].data(), true);
  set_bc(s, true, V, s.lbc_typ[1], s.pl[LBC_V].data(), true);
  set_bc(s, true, W, s.lbc_typ[2], s.pl[LBC_W].data(), false);
  set_bc(s, false, U, s.ubc_typ[0], s.pl[UBC_U].data(), true);
  set_bc(s, false, V, s.ubc_typ[1], s.pl[UBC_V].data(), true);
  set_bc(s, false, W, s.ubc_typ[2], s.pl[UBC_W].data(), false);
}

// ------------------------------------------------------------- wall law ----
// one plane through the 2-D cutoff filter g (testfilter.f90:197-210)
void filter_plane(const State& s, const double* f, const std::vector<double>& g, double* out) {
  std::vector<cd>& F = spec_buf(s.nsp);
  rfft2_plane(s.p.nx, s.p.ny, f, F.data());
  for (long q = 0; q < s.nsp; ++q) F[q] = F[q] * g[q];
  irfft2_plane(s.p.nx, s.p.ny, F.data(), out);
}
// u1, v1, |u| of obukhov / wallstress (compute_wall_law.f90:119-151, 210-243)
void wall_layer(State& s, std::vector<double>& u1, std::vector<double>& v1, std::vector<double>& ua) {
  const long n = s.npl;
  u1.resize(n);
  v1.resize(n);
  ua.resize(n);
  if (s.p.wall_model == 0) {
    filter_plane(s, s.lev(U, 1), s.g2, u1.data());
    filter_plane(s, s.lev(V, 1), s.g2, v1.data());
  } else if (s.p.wall_model == 1) {
    std::copy(s.lev(U, 1), s.lev(U, 1) + n, u1.begin());
    std::copy(s.lev(V, 1), s.lev(V, 1) + n, v1.begin());
  } else {
    double su = 0.0, sv = 0.0;
    for (long q = 0; q < n; ++q) { su += s.lev(U, 1)[q]; sv += s.lev(V, 1)[q]; }
    const double c = 1.0 / double(n);
    std::fill(u1.begin(), u1.end(), c * su);
    std::fill(v1.begin(), v1.end(), c * sv);
  }
  for (long q = 0; q < n; ++q) ua[q] = std::sqrt(u1[q] * u1[q] + v1[q] * v1[q]);
}
void obukhov(State& s) {  // compute_wall_law.f90:198-254 (neutral)
  std::vector<double> u1, v1, ua;
  wall_layer(s, u1, v1, ua);
  for (long q = 0; q < s.npl; ++q)
    s.pl[USTAR][q] = KVONK * ua[q] / std::log((0.5 * s.p.dz) / s.pl[LBC_Z0][q]);
}
void wallstress(State& s) {  // compute_wall_law.f90:107-185
  std::vector<double> u1, v1, ua;
  wall_layer(s, u1, v1, ua);
  const double c = 0.5 * s.p.dz * KVONK;
  for (long q = 0; q < s.npl; ++q) {
    const double us = s.pl[USTAR][q];
    const bool z = ua[q] == 0.0;
    const double bu = z ? 0.0 : us / c * u1[q] / ua[q];
    const double bv = z ? 0.0 : us / c * v1[q] / ua[q];
    s.pl[LBC_U][q] = bu;
    s.pl[LBC_V][q] = bv;
    s.lev(DUDZ, 1)[q] = bu;
    s.lev(DVDZ, 1)[q] = bv;
    s.lev(TXZ, 1)[q] = z ? 0.0 : (us * us) * u1[q] / ua[q];
    s.lev(TYZ, 1)[q] = z ? 0.0 : (us * us) * v1[q] / ua[q];
  }
}

}  // namespace

namespace {

// -------------------------------------------------------------- SGS ----
// S_ij at level k (compute_sgs.f90:260-335): uvp nodes at k = 1 (wall law),
// w nodes above; point q of the plane
struct Sij {
  double s11, s12, s13, s22, s23, s33;
};
inline Sij sij_at(State& s, int k, long q) {
  Sij r;
  if (k == 1) {
    const double ux = s.lev(DUDX, 1)[q], uy = s.lev(DUDY, 1)[q], uz = s.lev(DUDZ, 1)[q];
    const double vx = s.lev(DVDX, 1)[q], vy = s.lev(DVDY, 1)[q], vz = s.lev(DVDZ, 1)[q];
    const double wx = 0.5 * (s.lev(DWDX, 1)[q] + s.lev(DWDX, 2)[q]);
    const double wy = 0.5 * (s.lev(DWDY, 1)[q] + s.lev(DWDY, 2)[q]);
    const double wz = s.lev(DWDZ, 1)[q];
    r = {ux, 0.5 * (uy + vx), 0.5 * (uz + wx), vy, 0.5 * (vz + wy), wz};
  } else {
    const double ux = 0.5 * (s.lev(DUDX, k)[q] + s.lev(DUDX, k - 1)[q]);
    const double uy = 0.5 * (s.lev(DUDY, k)[q] + s.lev(DUDY, k - 1)[q]);
    const double uz = s.lev(DUDZ, k)[q];
    const double vx = 0.5 * (s.lev(DVDX, k)[q] + s.lev(DVDX, k - 1)[q]);
    const double vy = 0.5 * (s.lev(DVDY, k)[q] + s.lev(DVDY, k - 1)[q]);
    const double vz = s.lev(DVDZ, k)[q];
    const double wx = s.lev(DWDX, k)[q], wy = s.lev(DWDY, k)[q];
    const double wz = 0.5 * (s.lev(DWDZ, k)[q] + s.lev(DWDZ, k - 1)[q]);
    r = {ux, 0.5 * (uy + vx), 0.5 * (uz + wx), vy, 0.5 * (vz + wy), wz};
  }
  return r;
}
inline double strain_norm(const Sij& a) {
  return std::sqrt(2.0 * (a.s11 * a.s11 + a.s22 * a.s22 + a.s33 * a.s33 +
                          2.0 * (a.s12 * a.s12 + a.s13 * a.s13 + a.s23 * a.s23)));
}

inline float f32(double x) { return float(x); }
inline double f32max_tiny(double x) { return double(std::max(1e-24f, float(x))); }

// compute_LagScaleDep.f90:485-596 at one test scale, one level k: AB = L:M,
// BB = M:M (the 21 test-filtered fields of the level)
void dynamic_mum_level(State& s, int k, double tf_2, const std::vector<double>& g, double* AB, double* BB) {
  const long n = s.npl;
  const double cst = 2.0 * s.delta * s.delta;
  static thread_local std::vector<double> buf;
  if ((long)buf.size() < 22 * n) buf.resize(22 * n);
  double* uf = buf.data();
  double* vf = uf + n;
  double* wf = vf + n;
  double* A[6];
  double* Sf[6];
  double* SS[6];
  for (int i = 0; i < 6; ++i) {
    A[i] = buf.data() + (3 + i) * n;
    Sf[i] = buf.data() + (9 + i) * n;
    SS[i] = buf.data() + (15 + i) * n;
  }
  double* sft = buf.data() + 21 * n;
  for (long q = 0; q < n; ++q) {
    double u, v, w;
    if (k == 1) {
      u = s.lev(U, 1)[q];
      v = s.lev(V, 1)[q];
      w = 0.25 * s.lev(W, 2)[q];
    } else {
      u = 0.5 * (s.lev(U, k)[q] + s.lev(U, k - 1)[q]);
      v = 0.5 * (s.lev(V, k)[q] + s.lev(V, k - 1)[q]);
      w = s.lev(W, k)[q];
    }
    uf[q] = u;
    vf[q] = v;
    wf[q] = w;
    A[0][q] = u * u;
    A[1][q] = u * v;
    A[2][q] = u * w;
    A[3][q] = v * v;
    A[4][q] = v * w;
    A[5][q] = w * w;
    const Sij a = sij_at(s, k, q);
    const double S = strain_norm(a);
    const double sv[6] = {a.s11, a.s12, a.s13, a.s22, a.s23, a.s33};
    for (int i = 0; i < 6; ++i) {
      Sf[i][q] = sv[i];
      SS[i][q] = S * sv[i];
    }
  }
  // filter all 21 planes (testfilter.f90:144-184)
  std::vector<double>& t = real_buf(n);
  for (int i = 0; i < 21; ++i) {
    double* f = buf.data() + (long)i * n;
    filter_plane(s, f, g, t.data());
    std::copy(t.data(), t.data() + n, f);
  }
  for (long q = 0; q < n; ++q) {
    const double a11 = A[0][q] - uf[q] * uf[q], a12 = A[1][q] - uf[q] * vf[q], a13 = A[2][q] - uf[q] * wf[q];
    const double a22 = A[3][q] - vf[q] * vf[q], a23 = A[4][q] - vf[q] * wf[q], a33 = A[5][q] - wf[q] * wf[q];
    const double f11 = Sf[0][q], f12 = Sf[1][q], f13 = Sf[2][q], f22 = Sf[3][q], f23 = Sf[4][q], f33 = Sf[5][q];
    sft[q] = std::sqrt(2.0 * (f11 * f11 + f22 * f22 + f33 * f33 + 2.0 * (f12 * f12 + f13 * f13 + f23 * f23)));
    const double ts = tf_2 * sft[q];
    const double b11 = cst * (SS[0][q] - ts * f11), b12 = cst * (SS[1][q] - ts * f12);
    const double b13 = cst * (SS[2][q] - ts * f13), b22 = cst * (SS[3][q] - ts * f22);
    const double b23 = cst * (SS[4][q] - ts * f23), b33 = cst * (SS[5][q] - ts * f33);
    AB[q] = a11 * b11 + a22 * b22 + a33 * b33 + 2.0 * (a12 * b12 + a13 * b13 + a23 * b23);
    BB[q] = b11 * b11 + b22 * b22 + b33 * b33 + 2.0 * (b12 * b12 + b13 * b13 + b23 * b23);
  }
}

// FF of compute_interpolag_coeff (compute_LagScaleDep.f90:439-452) as
// update_halo3 (decomp_2d_custom.f90:902-1024) leaves it on a 1x1 process
// grid: mirror copies of the first / last two rows and planes (self-messages
// matched in posting order), x wrapped.  FF[(k+1)][(j+1)][(i+1)], Fortran
// k in -1..nz+2, j in -1..ny+2, i in -1..nx+2.
struct Halo {
  int nx, ny, nz;
  std::vector<double> a;
  double& at(int i, int j, int k) { return a[((long)(k + 1) * (ny + 4) + (j + 1)) * (nx + 4) + (i + 1)]; }
};
void lag_halo(State& s, const double* F, Halo& H) {
  const int nx = s.p.nx, ny = s.p.ny, nz = s.p.nz;
  H.nx = nx;
  H.ny = ny;
  H.nz = nz;
  H.a.assign((long)(nz + 4) * (ny + 4) * (nx + 4), 0.0);
  auto Fv = [&](int i, int j, int k) { return F[((long)k * ny + (j - 1)) * nx + (i - 1)]; };
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      for (int i = 1; i <= nx; ++i) H.at(i, j, k) = Fv(i, j, k);
      H.at(-1, j, k) = Fv(nx - 1, j, k);
      H.at(0, j, k) = Fv(nx, j, k);
      H.at(nx + 1, j, k) = Fv(1, j, k);
      H.at(nx + 2, j, k) = Fv(2, j, k);
    }
  // rows -1, 0 <- 1, 2 and ny+1, ny+2 <- ny-1, ny (every level, whole rows)
  for (int k = -1; k <= nz + 2; ++k)
    for (int i = -1; i <= nx + 2; ++i) {
      H.at(i, -1, k) = H.at(i, 1, k);
      H.at(i, 0, k) = H.at(i, 2, k);
      H.at(i, ny + 1, k) = H.at(i, ny - 1, k);
      H.at(i, ny + 2, k) = H.at(i, ny, k);
    }
  // planes -1, 0 <- 1, 2 and nz+1, nz+2 <- nz-1, nz
  const long pl = (long)(ny + 4) * (nx + 4);
  auto plane = [&](int k) { return H.a.data() + (long)(k + 1) * pl; };
  std::copy(plane(1), plane(1) + pl, plane(-1));
  std::copy(plane(2), plane(2) + pl, plane(0));
  std::copy(plane(nz - 1), plane(nz - 1) + pl, plane(nz + 1));
  std::copy(plane(nz), plane(nz) + pl, plane(nz + 2));
  // compute_LagScaleDep.f90:441-452
  std::copy(plane(1), plane(1) + pl, plane(0));
  std::fill(plane(-1), plane(-1) + pl, BOGUS);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      H.at(i, j, nz + 1) = Fv(i, j, nz + 1);
      H.at(i, j, nz + 2) = Fv(i, j, nz + 1);
    }
}

struct LagWeights {
  std::vector<signed char> ax, ay, az;
  std::vector<double> cx, cy, cz;  // levels 1..nz+1 flattened (k-1)*npl + q
};
// compute_LagScaleDep.f90:309-411
void interpolag_weight(State& s, LagWeights& w) {
  const Params& p = s.p;
  const int nz = p.nz;
  const long n = s.npl;
  const double cs = double(p.cs_count);
  // u_lag, v_lag to w nodes; w_lag scaled; its level 1 from level 2
  for (int comp = 0; comp < 2; ++comp) {
    double* a = s.F(comp == 0 ? U_LAG : V_LAG);
    std::vector<double> tmp(s.nf);
    for (long q = 0; q < s.nf; ++q) tmp[q] = a[q] / cs;
    for (long q = 0; q < n; ++q) a[n + q] = tmp[n + q];
    for (int k = 2; k <= nz + 1; ++k)
      for (long q = 0; q < n; ++q) a[(long)k * n + q] = 0.5 * (tmp[(long)k * n + q] + tmp[(long)(k - 1) * n + q]);
  }
  double* wl = s.F(W_LAG);
  for (long q = 0; q < s.nf; ++q) wl[q] = wl[q] / cs;
  for (long q = 0; q < n; ++q) wl[n + q] = 0.25 * wl[2 * n + q];
  const long m = (long)(nz + 1) * n;
  w.ax.resize(m); w.ay.resize(m); w.az.resize(m);
  w.cx.resize(m); w.cy.resize(m); w.cz.resize(m);
  std::vector<double> zp(m);
  for (int k = 1; k <= nz + 1; ++k)
    for (long q = 0; q < n; ++q) {
      const long o = (long)(k - 1) * n + q;
      const double xp = -s.lev(U_LAG, k)[q] * p.dt * cs / p.dx;
      const double yp = -s.lev(V_LAG, k)[q] * p.dt * cs / p.dy;
      zp[o] = -s.lev(W_LAG, k)[q] * p.dt * cs / p.dz;
      w.ax[o] = std::signbit(xp) ? -1 : 1;
      w.ay[o] = std::signbit(yp) ? -1 : 1;
      w.cx[o] = std::fabs(xp);
      w.cy[o] = std::fabs(yp);
    }
  // first-cell correction (:368-379), level 1 taken from level 2 at the end
  for (long q = 0; q < n; ++q) {
    double z1 = zp[q], z2 = zp[n + q];
    z2 = z2 + std::min(z2, 0.0);
    z1 = z1 + std::max(z1, 0.0);
    z2 = std::min(1.0, z2);
    z1 = std::min(1.0, z2);
    z2 = std::max(-1.0, z2);
    z1 = std::max(-1.0, z2);
    zp[q] = z1;
    zp[n + q] = z2;
  }
  for (long o = 0; o < m; ++o) {
    w.az[o] = std::signbit(zp[o]) ? -1 : 1;
    w.cz[o] = std::fabs(zp[o]);
  }
}
// compute_LagScaleDep.f90:427-474: trilinear upstream interpolation, levels 1..nz+1
void interpolag_coeff(State& s, int fid, const LagWeights& w) {
  Halo H;
  lag_halo(s, s.F(fid), H);
  const int nx = s.p.nx, ny = s.p.ny, nz = s.p.nz;
  double* F = s.F(fid);
#pragma omp parallel for
  for (int k = 1; k <= nz + 1; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const long q = (long)(j - 1) * nx + (i - 1);
        const long o = (long)(k - 1) * nx * ny + q;
        const int ax = i + w.ax[o], ay = j + w.ay[o], az = k + w.az[o];
        const double cx = w.cx[o], cy = w.cy[o], cz = w.cz[o];
        const double fx = 1.0 - cx, fy = 1.0 - cy, fz = 1.0 - cz;
        F[(long)k * nx * ny + q] = fx * fy * (H.at(i, j, k) * fz + H.at(i, j, az) * cz) +
                                   fx * cy * (H.at(i, ay, k) * fz + H.at(i, ay, az) * cz) +
                                   cx * fy * (H.at(ax, j, k) * fz + H.at(ax, j, az) * cz) +
                                   cx * cy * (H.at(ax, ay, k) * fz + H.at(ax, ay, az) * cz);
      }
}
// compute_LagScaleDep.f90:607-640 with the default-REAL casts of :624,626,633
void update_interpolag_coeff(State& s, int fab, int fbb, const std::vector<double>& AB,
                             const std::vector<double>& BB) {
  const double opftdelta = OPFTIME * s.delta;
  const double lagran_dt = s.p.dt * double(s.p.cs_count);
  double* Fa = s.F(fab);
  double* Fb = s.F(fbb);
#pragma omp parallel for
  for (long o = s.npl; o < s.nf; ++o) {
    double tmp = double(std::max(f32(Fa[o] * Fb[o]), 1e-24f));
    tmp = opftdelta * std::pow(tmp, -1.0 / 8.0);
    tmp = f32max_tiny(tmp);
    const double dumfac = lagran_dt / tmp;
    const double epsi = dumfac / (1.0 + dumfac);
    Fa[o] = epsi * AB[o] + (1.0 - epsi) * Fa[o];
    Fb[o] = epsi * BB[o] + (1.0 - epsi) * Fb[o];
    Fa[o] = f32max_tiny(Fa[o]);
  }
}
// compute_LagScaleDep.f90:651-707
void dynamic_coeff(State& s) {
  const int nz = s.p.nz;
#pragma omp parallel for
  for (int k = 1; k <= nz + 1; ++k)
    for (long q = 0; q < s.npl; ++q) {
      const double c2 = f32max_tiny(s.lev(F_LM, k)[q] / s.lev(F_MM, k)[q]);
      const double c4 = f32max_tiny(s.lev(F_QN, k)[q] / s.lev(F_NN, k)[q]);
      double beta = std::pow(c4 / c2, s.beta_pow);
      beta = double(std::max(f32(beta), float(1.0 / (TF1 * TF2))));
      if (k == nz + 1) beta = 1.0;
      s.lev(BETA, k)[q] = beta;
      s.lev(CS_OPT2, k)[q] = f32max_tiny(c2 / beta);
    }
}
// compute_LagScaleDep.f90:204-298
void lasd_coeff(State& s, int jt, int jtt) {
  const Params& p = s.p;
  const int nz = p.nz;
  (void)jt;
  if (jtt >= p.dyn_init)
    for (long o = 0; o < s.nf; ++o) {
      s.F(U_LAG)[o] += s.F(U)[o];
      s.F(V_LAG)[o] += s.F(V)[o];
      s.F(W_LAG)[o] += s.F(W)[o];
    }
  if (jtt < p.dyn_init) {
    std::fill(s.f[CS_OPT2].begin() + s.npl, s.f[CS_OPT2].end(), 0.03);
    return;
  }
  if (jtt % p.cs_count != 0) return;
  std::vector<double> LM(s.nf, 0.0), MM(s.nf, 0.0), QN(s.nf, 0.0), NN(s.nf, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int k = 1; k <= nz + 1; ++k) {
    const long o = (long)k * s.npl;
    dynamic_mum_level(s, k, TF1_2, s.g2, LM.data() + o, MM.data() + o);
    dynamic_mum_level(s, k, TF2_2, s.g4, QN.data() + o, NN.data() + o);
  }
  if (s.f_coeff_init) {
    LagWeights w;
    interpolag_weight(s, w);
    for (int fid : {F_LM, F_MM, F_QN, F_NN}) interpolag_coeff(s, fid, w);
  } else {
    for (long o = s.npl; o < s.nf; ++o) {
      s.F(F_MM)[o] = MM[o];
      s.F(F_LM)[o] = 0.03 * MM[o];
      s.F(F_NN)[o] = NN[o];
      s.F(F_QN)[o] = 0.03 * NN[o];
    }
    s.f_coeff_init = true;
  }
  update_interpolag_coeff(s, F_LM, F_MM, LM, MM);
  update_interpolag_coeff(s, F_QN, F_NN, QN, NN);
  dynamic_coeff(s);
  s.lagran_init = true;
  std::fill(s.f[U_LAG].begin(), s.f[U_LAG].end(), 0.0);
  std::fill(s.f[V_LAG].begin(), s.f[V_LAG].end(), 0.0);
  std::fill(s.f[W_LAG].begin(), s.f[W_LAG].end(), 0.0);
}

// compute_sgs.f90:105-247 (LES branch)
void sgs_stress(State& s, int jt, int jtt) {
  const Params& p = s.p;
  const int nz = p.nz;
  std::vector<double> lvec(nz + 2, s.delta);
  if (p.sgs == 0) {
    const double nd = 2.0;
    for (int k = 1; k <= nz + 1; ++k) {
      const double z = (k == 1) ? 0.5 * p.dz : (1 + k - 2.0) * p.dz;
      lvec[k] = std::pow(std::pow(p.cs0, nd) * std::pow(KVONK * z, -nd) + std::pow(s.delta, -nd), -1.0 / nd);
    }
    std::fill(s.f[CS_OPT2].begin() + s.npl, s.f[CS_OPT2].end(), p.cs0 * p.cs0);
  } else {
    lasd_coeff(s, jt, jtt);
  }
#pragma omp parallel for
  for (int k = 1; k <= nz + 1; ++k) {
    const double l2 = lvec[k] * lvec[k];
    for (long q = 0; q < s.npl; ++q) {
      const Sij a = sij_at(s, k, q);
      s.lev(NU_T, k)[q] = strain_norm(a) * s.lev(CS_OPT2, k)[q] * l2;
      if (k >= 2) {
        s.lev(TXZ, k)[q] = 2.0 * s.lev(NU_T, k)[q] * a.s13;
        s.lev(TYZ, k)[q] = 2.0 * s.lev(NU_T, k)[q] * a.s23;
      }
    }
  }
  // bottom layer on uvp nodes (:195-203), then levels 2..nz
#pragma omp parallel for
  for (int k = 1; k <= nz; ++k)
    for (long q = 0; q < s.npl; ++q) {
      const double nu = (k == 1) ? s.lev(NU_T, 1)[q] : 0.5 * (s.lev(NU_T, k)[q] + s.lev(NU_T, k + 1)[q]);
      s.lev(TXX, k)[q] = 2.0 * nu * s.lev(DUDX, k)[q];
      s.lev(TXY, k)[q] = 2.0 * nu * 0.5 * (s.lev(DUDY, k)[q] + s.lev(DVDX, k)[q]);
      s.lev(TYY, k)[q] = 2.0 * nu * s.lev(DVDY, k)[q];
      s.lev(TZZ, k)[q] = 2.0 * nu * s.lev(DWDZ, k)[q];
    }
  std::copy(s.lev(TZZ, 1), s.lev(TZZ, 1) + s.npl, s.lev(TZZ, 0));
}

}  // namespace

namespace {

// ------------------------------------------------- padded convection ----
// compute_convective_padd.f90:274-324: 3/2 zero padding of one level
// (x pass, then y pass): (ny, nx) -> (ny2, nx2), modes 0 .. n/2 - 1 kept
void to_big_level(const State& s, const double* in, double* out) {
  const int nx = s.p.nx, ny = s.p.ny, nx2 = 3 * nx / 2, ny2 = 3 * ny / 2;
  const int lhx = nx / 2 + 1, lhy = ny / 2 + 1;
  Scratch& S = scratch();
  S.need(std::max(nx2, ny2) + 2);
  std::vector<double>& hyb = real_buf((long)ny * nx2 + 2L * std::max(nx2, ny2));
  double* c0 = hyb.data() + (long)ny * nx2;
  double* c1 = c0 + std::max(nx2, ny2);
  const int hm = std::max(nx2, ny2) / 2 + 1;
  std::vector<cd> A(hm), B(hm), Ab(hm), Bb(hm);
  for (int j = 0; j < ny; j += 2) {
    r2c_pair(nx, in + (long)j * nx, in + (long)(j + 1) * nx, A.data(), B.data(), S.z.data(), S.w.data());
    std::fill(Ab.begin(), Ab.begin() + nx2 / 2 + 1, cd(0.0, 0.0));
    std::fill(Bb.begin(), Bb.begin() + nx2 / 2 + 1, cd(0.0, 0.0));
    for (int k = 0; k < lhx - 1; ++k) {
      Ab[k] = A[k];
      Bb[k] = B[k];
    }
    c2r_pair(nx2, Ab.data(), Bb.data(), hyb.data() + (long)j * nx2, hyb.data() + (long)(j + 1) * nx2, S.z.data(),
             S.w.data());
  }
  std::vector<double> col0(ny), col1(ny);
  for (int i = 0; i < nx2; i += 2) {
    for (int j = 0; j < ny; ++j) {
      col0[j] = hyb[(long)j * nx2 + i];
      col1[j] = hyb[(long)j * nx2 + i + 1];
    }
    r2c_pair(ny, col0.data(), col1.data(), A.data(), B.data(), S.z.data(), S.w.data());
    std::fill(Ab.begin(), Ab.begin() + ny2 / 2 + 1, cd(0.0, 0.0));
    std::fill(Bb.begin(), Bb.begin() + ny2 / 2 + 1, cd(0.0, 0.0));
    for (int k = 0; k < lhy - 1; ++k) {
      Ab[k] = A[k];
      Bb[k] = B[k];
    }
    c2r_pair(ny2, Ab.data(), Bb.data(), c0, c1, S.z.data(), S.w.data());
    for (int j = 0; j < ny2; ++j) {
      out[(long)j * nx2 + i] = c0[j];
      out[(long)j * nx2 + i + 1] = c1[j];
    }
  }
}
// compute_convective_padd.f90:337-388: fine-grid product back to (ny, nx)
void from_big_level(const State& s, const double* in, double* out) {
  const int nx = s.p.nx, ny = s.p.ny, nx2 = 3 * nx / 2, ny2 = 3 * ny / 2;
  const int lhx = nx / 2 + 1, lhy = ny / 2 + 1;
  Scratch& S = scratch();
  S.need(std::max(nx2, ny2) + 2);
  std::vector<double> hyb((long)ny * nx2), c0(ny2), c1(ny2), r0(ny), r1(ny);
  std::vector<cd> A(std::max(nx2, ny2) / 2 + 1), B(std::max(nx2, ny2) / 2 + 1), As(lhx), Bs(lhx);
  std::vector<cd> Ay(lhy), By(lhy);
  for (int i = 0; i < nx2; i += 2) {
    for (int j = 0; j < ny2; ++j) {
      c0[j] = in[(long)j * nx2 + i];
      c1[j] = in[(long)j * nx2 + i + 1];
    }
    r2c_pair(ny2, c0.data(), c1.data(), A.data(), B.data(), S.z.data(), S.w.data());
    std::fill(Ay.begin(), Ay.end(), cd(0.0, 0.0));
    std::fill(By.begin(), By.end(), cd(0.0, 0.0));
    for (int k = 0; k < lhy - 1; ++k) {
      Ay[k] = A[k];
      By[k] = B[k];
    }
    c2r_pair(ny, Ay.data(), By.data(), r0.data(), r1.data(), S.z.data(), S.w.data());
    for (int j = 0; j < ny; ++j) {
      hyb[(long)j * nx2 + i] = r0[j];
      hyb[(long)j * nx2 + i + 1] = r1[j];
    }
  }
  for (int j = 0; j < ny; j += 2) {
    r2c_pair(nx2, hyb.data() + (long)j * nx2, hyb.data() + (long)(j + 1) * nx2, A.data(), B.data(), S.z.data(),
             S.w.data());
    std::fill(As.begin(), As.end(), cd(0.0, 0.0));
    std::fill(Bs.begin(), Bs.end(), cd(0.0, 0.0));
    for (int k = 0; k < lhx - 1; ++k) {
      As[k] = A[k];
      Bs[k] = B[k];
    }
    c2r_pair(nx, As.data(), Bs.data(), out + (long)j * nx, out + (long)(j + 1) * nx, S.z.data(), S.w.data());
  }
}

// compute_convective_padd.f90:115-262: rotational form u x omega, 3/2 padding
void dealias_convec(State& s, int cxid, int cyid, int czid) {
  const Params& p = s.p;
  const int nz = p.nz, L = s.L;
  const int nx2 = 3 * p.nx / 2, ny2 = 3 * p.ny / 2;
  const long nb = (long)nx2 * ny2, n = s.npl;
  const double c0 = 1.0 / double(p.nx * p.ny);
  std::vector<double> big((size_t)6 * L * nb);
  auto B = [&](int f, int k) { return big.data() + ((long)f * L + k) * nb; };
  // fields 0..2: -c u, -c v, -c w; 3..5: c times the vorticity components
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int f = 0; f < 6; ++f)
    for (int k = 1; k < L; ++k) {
      std::vector<double> t(n);
      for (long q = 0; q < n; ++q) {
        double v;
        switch (f) {
          case 0: v = -c0 * s.lev(U, k)[q]; break;
          case 1: v = -c0 * s.lev(V, k)[q]; break;
          case 2: v = -c0 * s.lev(W, k)[q]; break;
          case 3:
            v = (k == 1) ? c0 * (0.5 * (s.lev(DWDY, 1)[q] + s.lev(DWDY, 2)[q]) - s.lev(DVDZ, 1)[q])
                         : c0 * (s.lev(DWDY, k)[q] - s.lev(DVDZ, k)[q]);
            break;
          case 4:
            v = (k == 1) ? c0 * (s.lev(DUDZ, 1)[q] - 0.5 * (s.lev(DWDX, 1)[q] + s.lev(DWDX, 2)[q]))
                         : c0 * (s.lev(DUDZ, k)[q] - s.lev(DWDX, k)[q]);
            break;
          default: v = c0 * (s.lev(DVDX, k)[q] - s.lev(DUDY, k)[q]); break;
        }
        t[q] = v;
      }
      to_big_level(s, t.data(), B(f, k));
    }
  const double c = 1.0 / double(nx2 * ny2);
  const int outs[3] = {cxid, cyid, czid};
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int comp = 0; comp < 3; ++comp)
    for (int k = 1; k <= nz; ++k) {
      std::vector<double> wk(nb);
      const double *ub = B(0, k), *vb = B(1, k), *o1 = B(3, k), *o2 = B(4, k), *o3 = B(5, k);
      const double *wbu = B(2, k + 1), *o1u = B(3, k + 1), *o2u = B(4, k + 1);
      for (long q = 0; q < nb; ++q) {
        if (comp == 0) {
          wk[q] = (k == 1) ? c * (-vb[q] * o3[q] + 0.5 * wbu[q] * o2u[q])
                           : c * (-vb[q] * o3[q] + 0.5 * (wbu[q] * o2u[q] + B(2, k)[q] * o2[q]));
        } else if (comp == 1) {
          wk[q] = (k == 1) ? c * (ub[q] * o3[q] + 0.5 * wbu[q] * (-o1u[q]))
                           : c * (ub[q] * o3[q] + 0.5 * (B(2, k)[q] * (-o1[q]) + wbu[q] * (-o1u[q])));
        } else {
          wk[q] = (k == 1) ? 0.0
                           : c * 0.5 * ((ub[q] + B(0, k - 1)[q]) * (-o2[q]) + (vb[q] + B(1, k - 1)[q]) * (o1[q]));
        }
      }
      from_big_level(s, wk.data(), s.lev(outs[comp], k));
    }
  for (int id : outs) {
    std::fill(s.lev(id, 0), s.lev(id, 0) + n, BOGUS);
    std::fill(s.lev(id, nz + 1), s.lev(id, nz + 1) + n, BOGUS);
  }
}

// ------------------------------------------------------- pressure ----
// compute_pressure.f90:116-242 with poisson_solver (:256-305), the Thomas
// solve per (kx, ky) (:448-493) and compute_press_grad (:320-372)
void press_stag_array(State& s, double tadv1) {
  const Params& p = s.p;
  const int nz = p.nz, L = s.L, ny = p.ny, lhx = s.lhx, lhy = s.lhy;
  const long n = s.npl, ns = s.nsp;
  const double c0 = 1.0 / double(p.nx * p.ny);
  std::vector<cd> H((size_t)3 * L * ns, cd(0.0, 0.0));
  auto Hs = [&](int f, int k) { return H.data() + ((long)f * L + k) * ns; };
  const double ct = c0 / tadv1;
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int f = 0; f < 3; ++f)
    for (int k = 1; k <= nz; ++k) {
      std::vector<double> t(n);
      const double* x = s.lev(f == 0 ? U : (f == 1 ? V : W), k);
      for (long q = 0; q < n; ++q) t[q] = ct * (x[q] / p.dt);
      rfft2_plane(p.nx, ny, t.data(), Hs(f, k));
      kill_oddballs(s, Hs(f, k));
    }
  double* bw = s.pl[BOT_WK].data();
  for (long q = 0; q < n; ++q) bw[q] = c0 * bw[q];
  std::vector<cd> bot(ns), top(ns);
  {
    std::vector<double> t(n);
    rfft2_plane(p.nx, ny, bw, bot.data());
    for (long q = 0; q < n; ++q) t[q] = c0 * s.pl[TOP_WK][q];
    rfft2_plane(p.nx, ny, t.data(), top.data());
  }
  kill_oddballs(s, bot.data());
  kill_oddballs(s, top.data());
  for (long q = 0; q < ns; ++q) {
    bot[q] = bot[q] * p.dz;
    top[q] = top[q] * p.dz;
  }
  // right-hand side rows 0 (bottom layer), 1..nz, nz+1 (top layer)
  std::vector<cd> r((size_t)L * ns);
  const double rdz = 1.0 / p.dz;
#pragma omp parallel for
  for (int k = 1; k <= nz; ++k)
    for (long q = 0; q < ns; ++q) {
      const cd sxy = s.kkx[q] * Hs(0, k)[q] + s.kky[q] * Hs(1, k)[q];
      const cd dz = (Hs(2, k + 1)[q] - Hs(2, k)[q]) * rdz;
      r[(long)k * ns + q] = cd(-sxy.imag(), sxy.real()) + dz;
    }
  for (long q = 0; q < ns; ++q) {
    r[q] = bot[q];
    r[(long)(nz + 1) * ns + q] = top[q];
  }
  r[0] = 0.0;
  // Thomas per column; the Nyquist row and column are left at zero
  std::vector<cd> x((size_t)L * ns, cd(0.0, 0.0));
  const double a_in = 1.0 / (p.dz * p.dz), c_in = 1.0 / (p.dz * p.dz);
#pragma omp parallel for
  for (long q = 0; q < ns; ++q) {
    const int j = int(q / lhx), i = int(q % lhx);
    if (i == lhx - 1 || j == lhy - 1) continue;
    static thread_local std::vector<double> gam;
    gam.resize(L);
    auto av = [&](int k) { return k == 0 ? (q == 0 ? 0.0 : BOGUS) : (k == nz + 1 ? -1.0 : a_in); };
    auto bv = [&](int k) {
      return k == 0 ? 1.0 * (q == 0 ? 1.0 : -1.0)
                    : (k == nz + 1 ? 1.0 : -(s.kkx[q] * s.kkx[q] + s.kky[q] * s.kky[q] + 2.0 / (p.dz * p.dz)));
    };
    auto cv = [&](int k) { return k == 0 ? (q == 0 ? 0.0 : 1.0) : (k == nz + 1 ? BOGUS : c_in); };
    double bet = bv(0);
    x[q] = r[q] * (1.0 / bet);
    for (int k = 1; k < L; ++k) {
      gam[k] = cv(k - 1) / bet;
      bet = bv(k) - av(k) * gam[k];
      x[(long)k * ns + q] = (r[(long)k * ns + q] - av(k) * x[(long)(k - 1) * ns + q]) * (1.0 / bet);
    }
    for (int k = L - 2; k >= 0; --k) x[(long)k * ns + q] = x[(long)k * ns + q] - gam[k + 1] * x[(long)(k + 1) * ns + q];
  }
  // wk: rows 0..nz from x, row nz+1 zero; gradients and the pressure
  for (long q = 0; q < ns; ++q) x[(long)(nz + 1) * ns + q] = 0.0;
#pragma omp parallel for schedule(dynamic)
  for (int k = 0; k <= nz + 1; ++k) {
    cd* X = x.data() + (long)k * ns;
    std::vector<cd>& G = spec_buf(ns);
    if (k >= 1 && k <= nz) {
      for (long q = 0; q < ns; ++q) G[q] = ik(s.kkx[q], X[q]);
      irfft2_plane(p.nx, ny, G.data(), s.lev(DPDX, k));
      for (long q = 0; q < ns; ++q) G[q] = ik(s.kky[q], X[q]);
      irfft2_plane(p.nx, ny, G.data(), s.lev(DPDY, k));
    }
    std::copy(X, X + ns, G.begin());
    irfft2_plane(p.nx, ny, G.data(), s.lev(P_, k));
  }
  std::fill(s.lev(P_, nz + 1), s.lev(P_, nz + 1) + n, BOGUS);
#pragma omp parallel for
  for (int k = 1; k <= nz; ++k)
    for (long q = 0; q < n; ++q) s.lev(DPDZ, k)[q] = rdz * (s.lev(P_, k)[q] - s.lev(P_, k - 1)[q]);
}

}  // namespace

namespace {

// ------------------------------------------------------------ the step ----
void compute_vel_grad(State& s) {  // LES_engine.f90:449-498
  grad_velocity_filt(s, U, DUDX, DUDY);
  grad_velocity_filt(s, V, DVDX, DVDY);
  grad_velocity_filt(s, W, DWDX, DWDY);
  apply_bcs(s);
  ddz_uv(s, DUDZ, U);
  ddz_uv(s, DVDZ, V);
  ddz_w(s, DWDZ, W);
}

void compute_rhs_adv(State& s) {  // LES_engine.f90:509-572
  const int nz = s.p.nz;
  const long n = s.npl;
  for (int q = 0; q < 3; ++q) {
    double* r = s.F(RHSX + q);
    double* rf = s.F(RHSX_F + q);
    std::copy(r + n, r + (long)(nz + 1) * n, rf + n);
    std::fill(r + n, r + (long)(nz + 1) * n, 0.0);
  }
  dealias_convec(s, RHSX, RHSY, RHSZ);
  div_stress(s, RHSX, TXX, TXY, TXZ, true, nullptr, nullptr);
  div_stress(s, RHSY, TXY, TYY, TYZ, true, nullptr, nullptr);
  div_stress(s, RHSZ, TXZ, TYZ, TZZ, false, s.pl[BOT_WK].data(), s.pl[TOP_WK].data());
  for (long o = n; o < (long)(nz + 1) * n; ++o) {
    s.F(RHSX)[o] = s.F(RHSX)[o] + s.p.pfx;
    s.F(RHSY)[o] = s.F(RHSY)[o] + s.p.pfy;
  }
}

// running_diagnostics.f90:148-305 -> cfl, mke, u_star, rms div u
void diagnostics(State& s, double out[4]) {
  const Params& p = s.p;
  const int nz = p.nz;
  const long n = s.npl;
  double umax = 0, vmax = 0, wmax = 0, us = 0, vs = 0, ws = 0, dsum = 0;
  for (long o = n; o < (long)(nz + 1) * n; ++o) {
    umax = std::max(umax, std::fabs(s.F(U)[o]));
    vmax = std::max(vmax, std::fabs(s.F(V)[o]));
    wmax = std::max(wmax, std::fabs(s.F(W)[o]));
    us += s.F(U)[o];
    vs += s.F(V)[o];
    ws += 0.5 * (s.F(W)[o] + s.F(W)[o + n]);
    const double d = s.F(DUDX)[o] + s.F(DVDY)[o] + s.F(DWDZ)[o];
    dsum += d * d;
  }
  const double cnt = double(p.nx) * p.ny * nz;
  out[0] = p.dt * (umax / p.dx + vmax / p.dy + wmax / p.dz);
  us /= cnt;
  vs /= cnt;
  ws /= cnt;
  out[1] = 0.5 * (us * us + vs * vs + ws * ws);
  double ust = 0.0;
  for (long q = 0; q < n; ++q) ust += s.pl[USTAR][q];
  out[2] = ust / double(n);
  out[3] = std::sqrt(dsum / cnt);
}

void les_step(State& s, double diag[4]) {  // LES_engine.f90:189-360
  const Params& p = s.p;
  const int nz = p.nz;
  const long n = s.npl;
  s.jt_total += 1;
  const int jtt = s.jt_total, jt = jtt;
  obukhov(s);
  wallstress(s);
  compute_vel_grad(s);
  sgs_stress(s, jt, jtt);
  compute_rhs_adv(s);
  const double tadv1 = (jtt == 1) ? 1.0 : 1.5;
  const double tadv2 = (jtt == 1) ? 0.0 : 1.0 - tadv1;
  for (int q = 0; q < 3; ++q) {
    double* x = s.F(U + q);
    const double* r = s.F(RHSX + q);
    const double* rf = s.F(RHSX_F + q);
#pragma omp parallel for
    for (long o = n; o < (long)(nz + 1) * n; ++o) x[o] = x[o] + p.dt * (tadv1 * r[o] + tadv2 * rf[o]);
  }
  std::fill(s.lev(W, 0), s.lev(W, 0) + n, 0.0);
  std::fill(s.lev(W, nz + 1), s.lev(W, nz + 1) + n, 0.0);
  press_stag_array(s, tadv1);
  for (int q = 0; q < 3; ++q) {
    double* x = s.F(U + q);
    double* r = s.F(RHSX + q);
    const double* g = s.F(DPDX + q);
#pragma omp parallel for
    for (long o = n; o < (long)(nz + 1) * n; ++o) {
      x[o] = x[o] - p.dt * tadv1 * g[o];
      r[o] = r[o] - g[o];
    }
  }
  std::fill(s.lev(W, 1), s.lev(W, 1) + n, 0.0);
  std::fill(s.lev(W, nz + 1), s.lev(W, nz + 1) + n, 0.0);
  apply_bcs(s);
  diagnostics(s, diag);
}

}  // namespace

// ------------------------------------------------------------- C ABI ----
// (ctypes binding in oracle/cpu_step.py)
extern "C" {

// lengths: nx, ny in 2^a 3^b (even); sgs 0 constant Smagorinsky, 2 LASD;
// wall_model 0 filter, 1 instantaneous, 2 homogeneous
void* cs_create(int nx, int ny, int nz, double dt, double lx, double ly, double lz, double z0, double pfx,
                double pfy, double cs0, int sgs, int cs_count, int dyn_init, int wall_model) {
  try {
    State* s = new State();
    Params& p = s->p;
    p.nx = nx;
    p.ny = ny;
    p.nz = nz;
    p.dt = dt;
    p.lx = lx;
    p.ly = ly;
    p.lz = lz;
    p.dx = lx / double(nx);
    p.dy = ly / double(ny);
    p.dz = lz / double(nz);
    p.z0 = z0;
    p.pfx = pfx;
    p.pfy = pfy;
    p.cs0 = cs0;
    p.sgs = sgs;
    p.cs_count = cs_count;
    p.dyn_init = dyn_init;
    p.wall_model = wall_model;
    plan_for(nx);
    plan_for(ny);
    plan_for(3 * nx / 2);
    plan_for(3 * ny / 2);
    init_state(*s);
    return s;
  } catch (...) {
    return nullptr;
  }
}
void cs_destroy(void* h) { delete static_cast<State*>(h); }
int cs_nfields(void) { return NFIELD; }
// field values, levels 0..nz+1 ((nz+2) ny nx doubles)
void cs_set_field(void* h, int id, const double* v) {
  State* s = static_cast<State*>(h);
  std::copy(v, v + s->nf, s->f[id].begin());
}
void cs_get_field(void* h, int id, double* v) {
  State* s = static_cast<State*>(h);
  std::copy(s->f[id].begin(), s->f[id].end(), v);
}
void cs_set_plane(void* h, int id, const double* v) {
  State* s = static_cast<State*>(h);
  std::copy(v, v + s->npl, s->pl[id].begin());
}
void cs_get_plane(void* h, int id, double* v) {
  State* s = static_cast<State*>(h);
  std::copy(s->pl[id].begin(), s->pl[id].end(), v);
}
// flags: f_coeff_init, lagran_init, jt_total, the lower / upper BC types
void cs_set_flags(void* h, int f_coeff_init, int lagran_init, int jt_total, const int* lbc, const int* ubc) {
  State* s = static_cast<State*>(h);
  s->f_coeff_init = f_coeff_init != 0;
  s->lagran_init = lagran_init != 0;
  s->jt_total = jt_total;
  for (int c = 0; c < 3; ++c) {
    s->lbc_typ[c] = lbc[c];
    s->ubc_typ[c] = ubc[c];
  }
}
void cs_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int cs_max_threads(void) { return omp_get_max_threads(); }
// nsteps time steps; diag: the last step's cfl, mke, u*, rms div u
int cs_step(void* h, int nsteps, double* diag) {
  try {
    State* s = static_cast<State*>(h);
    double d[4] = {0, 0, 0, 0};
    for (int i = 0; i < nsteps; ++i) les_step(*s, d);
    if (diag) std::copy(d, d + 4, diag);
    return 0;
  } catch (...) {
    return 1;
  }
}
// unnormalised 2-D r2c / c2r of ny x nx planes (the transforms under test)
void cs_rfft2(int nx, int ny, const double* f, double* F_interleaved) {
  rfft2_plane(nx, ny, f, reinterpret_cast<cd*>(F_interleaved));
}
void cs_irfft2(int nx, int ny, double* F_interleaved, double* f) {
  irfft2_plane(nx, ny, reinterpret_cast<cd*>(F_interleaved), f);
}

}  // extern "C"
