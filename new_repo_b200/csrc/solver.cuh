// Device-resident LES state and the operators of one time step.
#pragma once
#include <map>
#include <vector>
#include "../../include/lesgpu.h"
#include "common.cuh"
#include "spectral.cuh"

namespace les {

struct Grid {
  int nx, ny, nz, L, lhx, lhy, nx2, ny2;
  long plane() const { return (long)nx * ny; }
  long field() const { return plane() * L; }
};

// Per-precision interface so the C ABI can hold either instantiation.
struct SolverBase {
  les_params P{};
  Grid g{};
  cudaStream_t st = nullptr;
  bool f_coeff_init = false;
  bool lagran_init = false;
  int lbc_t[3] = {1, 1, 1};  // 'drc' until the wall law switches u,v to 'neu'
  int ubc_t[3] = {2, 2, 1};
  float timers_ms[5] = {0, 0, 0, 0, 0};
  virtual ~SolverBase() = default;
  virtual void upload(int field, const double* h, int k0, int k1) = 0;
  virtual void download(int field, double* h, int k0, int k1) = 0;
  virtual void upload_plane(int plane, const double* h) = 0;
  virtual void download_plane(int plane, double* h) = 0;
  virtual void set_initial_conditions(const double* u, const double* v, const double* w) = 0;
  virtual void grad_velocity_filt(int f, int dfdx, int dfdy) = 0;
  virtual void ddz_uv(int dfdz, int f) = 0;
  virtual void ddz_w(int dfdz, int f) = 0;
  virtual void div_stress(int rhs, int tx, int ty, int tz, int stag) = 0;
  virtual void dealias_convec(int cx, int cy, int cz) = 0;
  virtual void press_stag_array(double tadv1) = 0;
  virtual void obukhov() = 0;
  virtual void wallstress() = 0;
  virtual void sgs_stress(int jt, int jtt) = 0;
  virtual void test_filter(int f, int which) = 0;
  virtual void set_bc() = 0;
  virtual void compute_vel_grad() = 0;
  virtual void compute_rhs_adv() = 0;
  virtual void ab2(double tadv1, double tadv2) = 0;
  virtual void projection(double tadv1) = 0;
  virtual void step(int jt, int jtt) = 0;
  virtual void diagnostics(double out[4]) = 0;
  virtual unsigned status() = 0;
  virtual void read_timers() = 0;
};

SolverBase* make_solver(const les_params& p);

}  // namespace les
