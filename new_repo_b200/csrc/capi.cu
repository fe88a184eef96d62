// extern "C" boundary of liblesgpu.so (declared in include/lesgpu.h).
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/lesgpu.h"
#include "solver.cuh"

struct les_state {
  les::SolverBase* s = nullptr;
};

namespace {
thread_local std::string g_last_error;

template <typename F>
int guard(F&& f) {
  try {
    f();
    return LES_OK;
  } catch (const les::CudaError& e) {
    g_last_error = e.what();
    return e.code ? e.code : LES_ERR_INVALID;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return LES_ERR_INVALID;
  }
}

int bad_state() {
  g_last_error = "null les_state";
  return LES_ERR_INVALID;
}
int bad_arg(const char* what) {
  g_last_error = std::string("null argument: ") + what;
  return LES_ERR_INVALID;
}
}  // namespace

// Every entry point but les_step_host first orders the state's stream after
// the copies back of an earlier les_step_host (a no-op without one).
#define STATE_OR_FAIL(s)                     \
  if (!(s) || !(s)->s) return bad_state(); \
  les::g_hook = (s)->s;                    \
  (s)->s->join_copies()

extern "C" {

const char* les_last_error(void) { return g_last_error.c_str(); }

int les_create(const les_params* p, les_state** out) {
  if (!p || !out) {
    g_last_error = "null argument";
    return LES_ERR_INVALID;
  }
  *out = nullptr;
  les::g_hook = nullptr;  // never observe launches through a previous state
  return guard([&] {
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->dt <= 0 || p->cs_count <= 0)
      throw les::CudaError(LES_ERR_INVALID, "invalid grid, dt or cs_count");
    if (p->sgs_model < LES_SGS_CST_SMAG || p->sgs_model > LES_SGS_MLP)
      throw les::CudaError(LES_ERR_INVALID, "Invalid SGS model");
    if (p->wall_model < LES_WALL_FILTER || p->wall_model > LES_WALL_HOMOG)
      throw les::CudaError(LES_ERR_INVALID, "Invalid wall law type");
    auto* st = new les_state;
    try {
      st->s = les::make_solver(*p);
    } catch (...) {
      delete st;
      throw;
    }
    *out = st;
  });
}

int les_set_precision(les_state* s, int precision) {
  STATE_OR_FAIL(s);
  return guard([&] {
    if (precision != LES_FP64 && precision != LES_MIXED) throw les::CudaError(LES_ERR_INVALID, "Invalid precision");
    les::SolverBase* old = s->s;
    if (old->P.precision == precision) return;
    if (old->P.sgs_model == LES_SGS_MLP)
      throw les::CudaError(LES_ERR_INVALID, "set the precision before selecting the learned closure");
    les_params p = old->P;
    p.precision = precision;
    std::unique_ptr<les::SolverBase> n(les::make_solver(p));
    if (old->scalar_on) n->scalar_init(old->SP);
    if (old->sponge_frac > 0.0) n->sponge_init(old->sponge_frac);
    n->coriol = old->coriol;
    n->cs2_max = old->cs2_max;
    n->ug = old->ug;
    n->vg = old->vg;
    const int nz = p.nz;
    std::vector<double> buf((size_t)(nz + 2) * p.ny * p.nx);
    for (int f = 0; f < LES_NFIELDS; ++f) {
      if (!old->has_field(f)) continue;
      old->download(f, buf.data(), 0, nz + 1);
      n->upload(f, buf.data(), 0, nz + 1);
    }
    for (int pl = 0; pl < LES_NPLANES; ++pl) {
      old->download_plane(pl, buf.data());
      n->upload_plane(pl, buf.data());
    }
    for (int c = 0; c < 3; ++c) {
      n->lbc_t[c] = old->lbc_t[c];
      n->ubc_t[c] = old->ubc_t[c];
    }
    n->f_coeff_init = old->f_coeff_init;
    n->lagran_init = old->lagran_init;
    LES_CUDA(cudaStreamSynchronize(n->st));
    if (les::g_hook == old) les::g_hook = n.get();
    s->s = n.release();
    delete old;
  });
}

int les_destroy(les_state* s) {
  if (!s) return LES_OK;
  if (les::g_hook == s->s) les::g_hook = nullptr;
  int rc = guard([&] { delete s->s; });
  delete s;
  return rc;
}

int les_upload(les_state* s, int field, const double* h, int k0, int k1) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->upload(field, h, k0, k1); });
}
int les_download(les_state* s, int field, double* h, int k0, int k1) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->download(field, h, k0, k1); });
}
int les_upload_plane(les_state* s, int plane, const double* h) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->upload_plane(plane, h); });
}
int les_download_plane(les_state* s, int plane, double* h) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->download_plane(plane, h); });
}
int les_set_initial_conditions(les_state* s, const double* u, const double* v, const double* w) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->set_initial_conditions(u, v, w); });
}
int les_set_bc_types(les_state* s, const int lbc[3], const int ubc[3]) {
  STATE_OR_FAIL(s);
  for (int i = 0; i < 3; ++i) {
    if (lbc[i] < 0 || lbc[i] > 2 || ubc[i] < 0 || ubc[i] > 2) {
      g_last_error = "bc type must be 0 (none), 1 (drc) or 2 (neu)";
      return LES_ERR_INVALID;
    }
    s->s->lbc_t[i] = lbc[i];
    s->s->ubc_t[i] = ubc[i];
  }
  return LES_OK;
}
int les_set_lagrangian_init(les_state* s, int f) {
  STATE_OR_FAIL(s);
  s->s->f_coeff_init = f != 0;
  s->s->lagran_init = f != 0;
  return LES_OK;
}
int les_get_lagrangian_init(les_state* s, int* f) {
  STATE_OR_FAIL(s);
  *f = s->s->f_coeff_init ? 1 : 0;
  return LES_OK;
}

int les_grad_velocity_filt(les_state* s, int f, int dfdx, int dfdy) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->grad_velocity_filt(f, dfdx, dfdy); });
}
int les_ddz_uv(les_state* s, int dfdz, int f) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->ddz_uv(dfdz, f); });
}
int les_ddz_w(les_state* s, int dfdz, int f) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->ddz_w(dfdz, f); });
}
int les_div_stress(les_state* s, int rhs, int tx, int ty, int tz, int stag) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->div_stress(rhs, tx, ty, tz, stag); });
}
int les_compute_dealias_convec(les_state* s, int cx, int cy, int cz) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->dealias_convec(cx, cy, cz); });
}
int les_press_stag_array(les_state* s, double tadv1) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->press_stag_array(tadv1); });
}
int les_set_pressure_slabs(les_state* s, int nslabs) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->set_pressure_slabs(nslabs); });
}
int les_press_from_increment(les_state* s, double tadv1, double tadv2) {
  STATE_OR_FAIL(s);
  if (!(tadv1 != 0.0)) return bad_arg("tadv1");
  return guard([&] { s->s->press_from_increment(tadv1, tadv2); });
}
int les_set_wall_model(les_state* s, int wall_model) {
  STATE_OR_FAIL(s);
  if (wall_model != LES_WALL_FILTER && wall_model != LES_WALL_INST && wall_model != LES_WALL_HOMOG)
    return bad_arg("wall_model");
  s->s->P.wall_model = wall_model;
  return LES_OK;
}
int les_obukhov(les_state* s) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->obukhov(); });
}
int les_wallstress(les_state* s) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->wallstress(); });
}
int les_sgs_stress(les_state* s, int jt, int jtt) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->sgs_stress(jt, jtt); });
}
int les_test_filter(les_state* s, int f, int which) {
  STATE_OR_FAIL(s);
  if (which != 2 && which != 4) {
    g_last_error = "test filter width must be 2 or 4";
    return LES_ERR_INVALID;
  }
  return guard([&] { s->s->test_filter(f, which); });
}
int les_set_bc(les_state* s) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->set_bc(); });
}
int les_compute_vel_grad(les_state* s) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->compute_vel_grad(); });
}
int les_compute_rhs_adv(les_state* s) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->compute_rhs_adv(); });
}
int les_ab2_advance(les_state* s, double t1, double t2) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->ab2(t1, t2); });
}
int les_projection(les_state* s, double t1) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->projection(t1); });
}
int les_step(les_state* s, int jt, int jtt) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->step(jt, jtt); });
}
int les_diagnostics(les_state* s, double out[4]) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->diagnostics(out); });
}
int les_get_status(les_state* s, unsigned* bits) {
  STATE_OR_FAIL(s);
  return guard([&] { *bits = s->s->status(); });
}
int les_check_status(les_state* s, unsigned* bits) {
  STATE_OR_FAIL(s);
  unsigned b = 0;
  const int rc = guard([&] { b = s->s->status(); });
  if (rc != LES_OK) return rc;
  if (bits) *bits = b;
  if (b & les::ST_NAN) {
    g_last_error = "I got a NaN";
    return LES_ERR_NUMERICAL;
  }
  if (b & les::ST_PIVOT) {
    g_last_error = "tridiag solver: error bet(i,j)=0, dividing by 0!";
    return LES_ERR_NUMERICAL;
  }
  return LES_OK;
}
int les_sync(les_state* s) {
  STATE_OR_FAIL(s);
  return guard([&] { LES_CUDA(cudaStreamSynchronize(s->s->st)); });
}
int les_profile(les_state* s, int enable) {
  STATE_OR_FAIL(s);
  return guard([&] {
    LES_CUDA(cudaStreamSynchronize(s->s->st));
    s->s->profile(enable != 0);
  });
}
int les_profile_report(les_state* s, char* buf, int buflen) {
  STATE_OR_FAIL(s);
  return guard([&] {
    const std::string r = s->s->profile_report();
    if ((int)r.size() + 1 > buflen) throw les::CudaError(LES_ERR_INVALID, "profile report buffer too small");
    std::memcpy(buf, r.c_str(), r.size() + 1);
  });
}
int les_launch_count(les_state* s, long long* n) {
  STATE_OR_FAIL(s);
  *n = s->s->launches;
  return LES_OK;
}
int les_event_record(les_state* s, int slot) {
  STATE_OR_FAIL(s);
  if (slot < 0 || slot >= 16) {
    g_last_error = "event slot must be in 0..15";
    return LES_ERR_INVALID;
  }
  return guard([&] { s->s->record_event(slot); });
}
int les_event_elapsed(les_state* s, int a, int b, double* ms) {
  STATE_OR_FAIL(s);
  return guard([&] { *ms = s->s->elapsed(a, b); });
}
int les_upload_async(les_state* s, int field, const double* pinned, int k0, int k1) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->upload_async(field, pinned, k0, k1); });
}
int les_download_async(les_state* s, int field, double* pinned, int k0, int k1) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->download_async(field, pinned, k0, k1); });
}
int les_diagnostics_async(les_state* s, double* pinned_out4) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->diagnostics_async(pinned_out4); });
}
int les_host_register(void* p, size_t bytes) {
  if (!p || bytes == 0) return bad_arg("p, bytes");
  return guard([&] { LES_CUDA(cudaHostRegister(p, bytes, cudaHostRegisterDefault)); });
}
int les_host_unregister(void* p) {
  if (!p) return bad_arg("p");
  return guard([&] { LES_CUDA(cudaHostUnregister(p)); });
}
int les_step_host(les_state* s, int jt, int jt_total, double* u, double* v, double* w, double* diag_out4) {
  if (!s || !s->s) return bad_state();
  if (!u || !v || !w) return bad_arg("u, v, w");
  les::g_hook = s->s;
  return guard([&] { s->s->step_host(jt, jt_total, u, v, w, diag_out4); });
}

int les_set_sgs_model(les_state* s, int model) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->set_sgs_model(model); });
}
int les_scalar_init(les_state* s, const les_scalar_params* sp) {
  STATE_OR_FAIL(s);
  if (!sp) return bad_arg("sp");
  return guard([&] { s->s->scalar_init(*sp); });
}
int les_scalar_set_initial(les_state* s, const double* theta) {
  STATE_OR_FAIL(s);
  if (!theta) return bad_arg("theta");
  return guard([&] { s->s->scalar_set_initial(theta); });
}
int les_scalar_kappa(les_state* s, double* out, int n) {
  STATE_OR_FAIL(s);
  if (!out) return bad_arg("out");
  return guard([&] { s->s->scalar_kappa(out, n); });
}
int les_sponge_init(les_state* s, double fraction) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->sponge_init(fraction); });
}
int les_set_cs2_max(les_state* s, double cs2_max) {
  STATE_OR_FAIL(s);
  if (!(cs2_max >= 0.0)) return bad_arg("cs2_max");
  return guard([&] { s->s->cs2_max = cs2_max; });
}
int les_set_coriolis(les_state* s, double coriol, double ug, double vg) {
  STATE_OR_FAIL(s);
  return guard([&] {
    s->s->coriol = coriol;
    s->s->ug = ug;
    s->s->vg = vg;
  });
}

int les_mlp_init(les_state* s, unsigned seed) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->mlp_init(seed); });
}
int les_mlp_set_params(les_state* s, const float* p, int n) {
  STATE_OR_FAIL(s);
  if (!p) return bad_state();
  return guard([&] { s->s->mlp_set_params(p, n); });
}
int les_mlp_get_params(les_state* s, float* p, int n) {
  STATE_OR_FAIL(s);
  if (!p) return bad_state();
  return guard([&] { s->s->mlp_get_params(p, n); });
}
int les_mlp_reset_data(les_state* s, long cap) {
  STATE_OR_FAIL(s);
  if (cap <= 0) {
    g_last_error = "learned closure: capacity must be positive";
    return LES_ERR_INVALID;
  }
  return guard([&] { s->s->mlp_reset_data(cap); });
}
int les_mlp_collect(les_state* s, int stride, int dense_levels, int wall_repeat, unsigned seed) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->mlp_collect(stride, dense_levels, wall_repeat, seed); });
}
int les_mlp_counts(les_state* s, long long out2[2]) {
  STATE_OR_FAIL(s);
  if (!out2) return bad_state();
  return guard([&] { s->s->mlp_counts(out2); });
}
int les_mlp_fit_stats(les_state* s) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->mlp_fit_stats(); });
}
int les_mlp_train(les_state* s, int epochs, int tiles_per_step, double lr, double* loss_epochs, double* val_loss) {
  STATE_OR_FAIL(s);
  if (epochs < 0 || tiles_per_step <= 0 || !(lr > 0)) {
    g_last_error = "learned closure: invalid training arguments";
    return LES_ERR_INVALID;
  }
  return guard([&] { s->s->mlp_train(epochs, tiles_per_step, lr, loss_epochs, val_loss); });
}
int les_mlp_forward(les_state* s, const float* x, long n, float* y) {
  STATE_OR_FAIL(s);
  if (!x || !y || n <= 0) {
    g_last_error = "learned closure: invalid forward arguments";
    return LES_ERR_INVALID;
  }
  return guard([&] { s->s->mlp_forward_host(x, n, y); });
}
int les_mlp_grad(les_state* s, const float* x, const float* t, long n, float* grad, float* loss) {
  STATE_OR_FAIL(s);
  if (!x || !t || !grad || !loss || n <= 0) {
    g_last_error = "learned closure: invalid gradient arguments";
    return LES_ERR_INVALID;
  }
  return guard([&] { s->s->mlp_grad_host(x, t, n, grad, loss); });
}
int les_mlp_info(les_state* s, double out12[12]) {
  STATE_OR_FAIL(s);
  if (!out12) return bad_state();
  return guard([&] { s->s->mlp_info(out12); });
}
int les_mlp_set_check_every(les_state* s, int every) {
  STATE_OR_FAIL(s);
  if (every < 0) {
    g_last_error = "learned closure: check interval must be >= 0";
    return LES_ERR_INVALID;
  }
  return guard([&] { s->s->mlp_set_check_every(every); });
}

int les_mlp_set_wall_levels(les_state* s, int nlev) {
  STATE_OR_FAIL(s);
  if (nlev < 0) {
    g_last_error = "learned closure: wall levels must be >= 0";
    return LES_ERR_INVALID;
  }
  return guard([&] { s->s->mlp_set_wall_levels(nlev); });
}

int les_mlp_check_profile(les_state* s, double* out, int n) {
  STATE_OR_FAIL(s);
  if (!out) return bad_state();
  return guard([&] { s->s->mlp_check_profile(out, n); });
}

int les_checkpoint_write(les_state* s, const char* path) {
  STATE_OR_FAIL(s);
  if (!path) return bad_state();
  return guard([&] { s->s->checkpoint_write(path); });
}
int les_checkpoint_read(les_state* s, const char* path, int lagran_init) {
  STATE_OR_FAIL(s);
  if (!path) return bad_state();
  return guard([&] { s->s->checkpoint_read(path, lagran_init); });
}

int les_stat_init(les_state* s) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->stat_init(); });
}
int les_stat_averages(les_state* s, int jt, int jt_total, int start_stats, int running_period, const char* out_path) {
  STATE_OR_FAIL(s);
  if (!out_path) return bad_arg("out_path");
  return guard([&] { s->s->stat_averages(jt, jt_total, start_stats, running_period, out_path); });
}
int les_stat_sums(les_state* s, int index, double* out) {
  STATE_OR_FAIL(s);
  if (!out) return bad_arg("out");
  return guard([&] { s->s->stat_sums(index, out); });
}
int les_stat_iterations(les_state* s, int* out) {
  STATE_OR_FAIL(s);
  if (!out) return bad_arg("out");
  return guard([&] { *out = s->s->stat_iteration_count(); });
}
int les_stat_spectra(les_state* s, int jt, int jt_total, const char* out_path) {
  STATE_OR_FAIL(s);
  if (!out_path) return bad_arg("out_path");
  return guard([&] { s->s->stat_spectra(jt, jt_total, out_path); });
}
int les_tke_init(les_state* s, const char* out_path) {
  STATE_OR_FAIL(s);
  if (!out_path) return bad_arg("out_path");
  return guard([&] { s->s->tke_init(out_path); });
}
int les_tke_budget(les_state* s, int jt, int tke_period) {
  STATE_OR_FAIL(s);
  return guard([&] { s->s->tke_budget(jt, tke_period); });
}
int les_tke_sums(les_state* s, double* out, int* record) {
  STATE_OR_FAIL(s);
  if (!out || !record) return bad_arg("out/record");
  return guard([&] { s->s->tke_sums(out, record); });
}

int les_timers(les_state* s, double out[5]) {
  STATE_OR_FAIL(s);
  return guard([&] {
    LES_CUDA(cudaStreamSynchronize(s->s->st));
    s->s->read_timers();
    for (int i = 0; i < 5; ++i) out[i] = s->s->timers_ms[i];
  });
}

}  // extern "C"
