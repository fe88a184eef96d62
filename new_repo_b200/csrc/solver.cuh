// Device-resident LES state and the operators of one time step.
#pragma once
#include <map>
#include <cstdio>
#include <vector>
#include "../../include/lesgpu.h"
#include "common.cuh"
#include "spectral.cuh"
#include "launch.cuh"
#include <string>

namespace les {

struct Grid {
  int nx, ny, nz, L, lhx, lhy, nx2, ny2;
  long plane() const { return (long)nx * ny; }
  long field() const { return plane() * L; }
};

// Per-precision interface so the C ABI can hold either instantiation.  It
// observes every kernel launch (LaunchHook): a launch counter, and with
// profiling on, CUDA events on the state's stream around each launch,
// labelled "<operator>/<kernel>" with the launch's algorithmic bytes.
struct SolverBase : LaunchHook {
  les_params P{};
  Grid g{};
  cudaStream_t st = nullptr;
  long launches = 0;
  std::string tag = "op";
  bool prof_on = false;
  struct Rec {
    std::string label;
    double bytes;
    cudaEvent_t a, b;
  };
  std::vector<cudaEvent_t> pool;
  size_t pool_next = 0;
  std::vector<Rec> recs;
  Rec pending;
  cudaEvent_t next_event() {
    if (pool_next >= pool.size()) {
      cudaEvent_t e;
      LES_CUDA(cudaEventCreate(&e));
      pool.push_back(e);
    }
    return pool[pool_next++];
  }
  void before(const char* kind, double bytes) override {
    ++launches;
    if (!prof_on) return;
    pending.label = tag + "/" + kind;
    pending.bytes = bytes;
    pending.a = next_event();
    LES_CUDA(cudaEventRecord(pending.a, st));
  }
  void after() override {
    if (!prof_on) return;
    pending.b = next_event();
    LES_CUDA(cudaEventRecord(pending.b, st));
    recs.push_back(pending);
  }
  void profile(bool on) {
    prof_on = on;
    recs.clear();
    pool_next = 0;
  }
  // per label: launches, total ms, bytes per launch (JSON object)
  std::string profile_report();
  // RAII operator tag
  struct Tag {
    SolverBase* s;
    std::string old;
    Tag(SolverBase* s_, const char* t) : s(s_), old(s_->tag) { s->tag = t; }
    ~Tag() { s->tag = old; }
  };
  bool f_coeff_init = false;
  bool lagran_init = false;
  int lbc_t[3] = {1, 1, 1};  // 'drc' until the wall law switches u,v to 'neu'
  int ubc_t[3] = {2, 2, 1};
  float timers_ms[5] = {0, 0, 0, 0, 0};
  ~SolverBase() override {
    if (g_hook == this) g_hook = nullptr;
    for (auto e : pool) cudaEventDestroy(e);
    for (auto e : slots)
      if (e) cudaEventDestroy(e);
  }
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
  virtual void press_from_increment(double tadv1, double tadv2) = 0;
  virtual void set_pressure_slabs(int G) = 0;
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
  // pinned-host FP64 transfers on the state's stream (converted on device in
  // mixed precision); the caller synchronises
  // learned closure (mlp.cu)
  virtual void set_sgs_model(int model) = 0;
  virtual void mlp_init(unsigned seed) = 0;
  virtual void mlp_set_params(const float* p, int n) = 0;
  virtual void mlp_get_params(float* p, int n) = 0;
  virtual void mlp_reset_data(long cap) = 0;
  virtual void mlp_collect(int stride, int dense_levels, int wall_repeat, unsigned seed) = 0;
  virtual void mlp_counts(long long* c) = 0;
  virtual void mlp_fit_stats() = 0;
  virtual void mlp_train(int epochs, int tiles_per_step, double lr, double* loss_epochs, double* val_loss) = 0;
  virtual void mlp_forward_host(const float* x, long n, float* y) = 0;
  virtual void mlp_grad_host(const float* x, const float* t, long n, float* g, float* loss) = 0;
  virtual void mlp_info(double* out) = 0;
  virtual void mlp_set_check_every(int every) = 0;
  virtual void mlp_set_wall_levels(int n) = 0;
  virtual void checkpoint_write(const char* path) = 0;
  virtual void checkpoint_read(const char* path, int with_f) = 0;
  virtual void mlp_check_profile(double* out, int n) = 0;
  virtual void upload_async(int field, const double* pinned, int k0, int k1) = 0;
  virtual void download_async(int field, double* pinned, int k0, int k1) = 0;
  virtual void diagnostics_async(double* pinned4) = 0;
  // One time step with u, v, w (levels 0..nz+1, FP64) in host memory: copies
  // in, the step, copies back, on two copy streams around the state's stream
  // (step_host in solver.cu).  The copies back of a call may still run when
  // it returns; join_copies() orders the state's stream after them and runs
  // at the start of every other entry point.
  virtual void step_host(int jt, int jtt, double* u, double* v, double* w, double* diag4) = 0;
  bool copies_pending = false;
  cudaEvent_t ev_copies = nullptr;  // recorded after a call's last copy back
  void join_copies() noexcept {
    if (!copies_pending) return;
    copies_pending = false;
    (void)cudaStreamWaitEvent(st, ev_copies, 0);
  }
  virtual void stat_init() = 0;
  virtual void stat_averages(int jt, int jtt, int start_stats, int running_period, const char* out_path) = 0;
  virtual void stat_sums(int index, double* out) = 0;
  virtual int stat_iteration_count() = 0;
  virtual void stat_spectra(int jt, int jtt, const char* out_path) = 0;
  virtual void tke_init(const char* out_path) = 0;
  virtual void tke_budget(int jt, int tke_period) = 0;
  virtual void tke_sums(double* out, int* record) = 0;
  // scalar transport, buoyancy, sponge, Coriolis
  bool scalar_on = false;
  les_scalar_params SP{};
  double sponge_frac = 0.0;
  double cs2_max = 0.0;  // optional upper clip of the dynamic coefficients (0: none, the reference)
  double coriol = 0.0, ug = 0.0, vg = 0.0;
  virtual void scalar_init(const les_scalar_params& sp) = 0;
  virtual void scalar_set_initial(const double* theta) = 0;
  virtual void scalar_kappa(double* out, int n) = 0;
  virtual void sponge_init(double frac) = 0;
  virtual bool has_field(int f) const = 0;
  // timing events on the state's stream
  cudaEvent_t slots[16] = {};
  void record_event(int i) {
    if (!slots[i]) LES_CUDA(cudaEventCreate(&slots[i]));
    LES_CUDA(cudaEventRecord(slots[i], st));
  }
  double elapsed(int a, int b) {
    if (a < 0 || b < 0 || a >= 16 || b >= 16 || !slots[a] || !slots[b]) throw CudaError(1, "event slot not recorded");
    LES_CUDA(cudaEventSynchronize(slots[b]));
    float ms = 0;
    LES_CUDA(cudaEventElapsedTime(&ms, slots[a], slots[b]));
    return ms;
  }
};

SolverBase* make_solver(const les_params& p);

}  // namespace les
