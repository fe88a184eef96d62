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

// in-place complex transform of x (work: n values); inv: exponent sign +
void cfft(const Plan& P, cd* x, cd* work, bool inv) {
  cd* in = x;
  cd* out = work;
  const double sg = inv ? 1.0 : -1.0;
  const double s3 = std::sqrt(3.0) / 2.0;
  for (const auto& S : P.st) {
    const int r = S.r, m = S.m, s = S.s;
    for (int p = 0; p < m; ++p) {
      const cd* tw = S.tw.data() + (size_t)p * (r - 1);
      if (r == 2) {
        const cd w1 = inv ? std::conj(tw[0]) : tw[0];
        for (int q = 0; q < s; ++q) {
          const cd a = in[q + s * p], b = in[q + s * (p + m)];
          out[q + s * (2 * p)] = a + b;
          out[q + s * (2 * p + 1)] = (a - b) * w1;
        }
      } else if (r == 4) {
        const cd w1 = inv ? std::conj(tw[0]) : tw[0];
        const cd w2 = inv ? std::conj(tw[1]) : tw[1];
        const cd w3 = inv ? std::conj(tw[2]) : tw[2];
        for (int q = 0; q < s; ++q) {
          const cd a0 = in[q + s * p], a1 = in[q + s * (p + m)], a2 = in[q + s * (p + 2 * m)],
                   a3 = in[q + s * (p + 3 * m)];
          const cd t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = a1 - a3;
          const cd jt3(-sg * t3.imag(), sg * t3.real());  // sg i t3
          out[q + s * (4 * p)] = t0 + t2;
          out[q + s * (4 * p + 1)] = (t1 + jt3) * w1;
          out[q + s * (4 * p + 2)] = (t0 - t2) * w2;
          out[q + s * (4 * p + 3)] = (t1 - jt3) * w3;
        }
      } else {  // r == 3
        const cd w1 = inv ? std::conj(tw[0]) : tw[0];
        const cd w2 = inv ? std::conj(tw[1]) : tw[1];
        for (int q = 0; q < s; ++q) {
          const cd a0 = in[q + s * p], a1 = in[q + s * (p + m)], a2 = in[q + s * (p + 2 * m)];
          const cd t1 = a1 + a2, t2 = a1 - a2;
          const cd mm = a0 - 0.5 * t1;
          const cd st(-sg * s3 * t2.imag(), sg * s3 * t2.real());  // sg i sqrt(3)/2 t2
          out[q + s * (3 * p)] = a0 + t1;
          out[q + s * (3 * p + 1)] = (mm + st) * w1;
          out[q + s * (3 * p + 2)] = (mm - st) * w2;
        }
      }
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
    const cd zk = z[k], zm = std::conj(z[(n - k) % n]);
    A[k] = 0.5 * (zk + zm);
    if (B) B[k] = cd(0.0, -0.5) * (zk - zm);
  }
}
// half spectra A, B (imaginary parts of bins 0 and n/2 ignored) -> real rows
// a, b (unnormalised inverse)
void c2r_pair(int n, const cd* A, const cd* B, double* a, double* b, cd* z, cd* work) {
  const Plan& P = plan_for(n);
  const int h = n / 2;
  for (int k = 0; k <= h; ++k) {
    cd x = A[k], y = B ? B[k] : cd(0.0, 0.0);
    if (k == 0 || k == h) {
      x = cd(x.real(), 0.0);
      y = cd(y.real(), 0.0);
    }
    z[k] = x + cd(0.0, 1.0) * y;
    if (k > 0 && k < h) z[n - k] = std::conj(x) + cd(0.0, 1.0) * std::conj(y);
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
