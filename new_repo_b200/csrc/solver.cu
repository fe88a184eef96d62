// Device-resident LES state and the operator sequence of one time step
// (LES_engine.f90:189-360), for FP64 and mixed (FP32 fields) precision.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <map>
#include <memory>
#include <vector>
#include <type_traits>

#include "kernels.cuh"
#include "stats.cuh"
#include "mlp.cuh"
#include <algorithm>
#include <random>
#include "launch.cuh"
#include "solver.cuh"

namespace les {

// launch a pointwise kernel under the launch hook (count + optional events)
#define KL(kind, bytes, ...)   \
  do {                         \
    hook_before(kind, bytes);  \
    __VA_ARGS__;               \
    LES_CHECK_LAUNCH();        \
    hook_after();              \
  } while (0)

namespace {
constexpr double PI = 3.1415926535897932384626433;  // parameters_IO.f90:42
constexpr int NSPEC = 21;

int grid_for(long n, int bs = 256) {
  long g = (n + bs - 1) / bs;
  if (g > 148L * 32) g = 148L * 32;
  if (g < 1) g = 1;
  return int(g);
}

template <typename T>
T* dalloc(size_t n) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T) + 256);
  if (e != cudaSuccess) throw CudaError(3, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  LES_CUDA(cudaMemset(p, 0, n * sizeof(T) + 256));
  return reinterpret_cast<T*>(p);
}
}  // namespace

// file names of the TKE budget profiles, in the order of the avg_var calls
// of compute_tke_budget (tke_budget1D.f90:218-383)
const char* const TKE_NAMES[TKE_NQ] = {
    "u",     "v",     "w",     "dudx",  "dudy",  "dudz",     "dvdx",     "dvdy",     "dvdz",  "dwdx",  "dwdy",
    "dwdz",  "uu",    "vv",    "ww",    "uv",    "uw",       "vw",       "txx",      "tyy",   "tzz",   "txy",
    "txz",   "tyz",   "cs",    "uuw",   "vvw",   "www",      "uww",      "wtzz",     "utxz",  "vtyz",  "dxx",
    "dyy",   "dzz",   "dxy",   "dxz",   "dyz",   "dudx2",    "dudy2",    "dudz2",    "dvdx2", "dvdy2", "dvdz2",
    "dwdx2", "dwdy2", "dwdz2", "dudxdwdx", "dudydwdy", "dudzdwdz", "p", "dpdx", "dpdy", "dpdz", "pw",
    "pu",    "pdudx", "pdvdy", "pdwdz", "pdwdx", "pdudz"};

template <typename T>
class Solver final : public SolverBase {
 public:
  T* F[LES_NFIELDS] = {};
  T* PL[LES_NPLANES] = {};
  // tables
  T *kkx = nullptr, *kky = nullptr, *gt = nullptr, *gtt = nullptr;
  double *kkxd = nullptr, *kkyd = nullptr, *l2 = nullptr;
  std::map<int, cplx<T>*> tw;
  int nk2 = 1, nk4 = 1;  // kx columns with a nonzero 2Delta / 4Delta filter
  int ky2 = 0, ky4 = 0;
  double delta = 0, beta_pow = 1;
  // workspace
  cplx<T>* spec[NSPEC] = {};
  cplx<T>* spec4[NSPEC] = {};
  T* fine[6] = {};
  T* sc[15] = {};  // S, s11..s33, LM, MM, QN, NN, Fn x4
  T* refbuf[MAXIN] = {};  // per-level reference values (mixed precision)
  // FP64 spectral workspace of the pressure path in mixed precision
  cplx<double>* pspec[8] = {};
  std::map<int, cplx<double>*> twd;
  double *kkx64 = nullptr, *kky64 = nullptr;
  cplx<double>* xs = nullptr;
  double* gam = nullptr;
  double* pmean = nullptr;
  double* part = nullptr;
  double* dout = nullptr;
  unsigned* dstatus = nullptr;
  std::vector<void*> allocs;
  cudaEvent_t ev[6] = {};

  explicit Solver(const les_params& p) {
    P = p;
    g.nx = p.nx;
    g.ny = p.ny;
    g.nz = p.nz;
    g.L = p.nz + 2;
    g.lhx = p.nx / 2 + 1;
    g.lhy = p.ny / 2 + 1;
    g.nx2 = 3 * p.nx / 2;
    g.ny2 = 3 * p.ny / 2;
    if (!supported_length(p.nx) || !supported_length(p.ny) || !supported_length(g.nx2) ||
        !supported_length(g.ny2) || p.nz < 2)
      throw CudaError(1, "grid size not supported (nx, ny in {16,32,64,128,256,512}, nz >= 2)");
    // the kernels index fields and the padded fine grid with 32-bit offsets
    if ((long)(p.nz + 2) * g.nx2 * g.ny2 >= (1L << 32))
      throw CudaError(1, "grid too large: (nz + 2) * (3 nx / 2) * (3 ny / 2) must stay below 2^32 points");
    LES_CUDA(cudaSetDevice(p.device));
    LES_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (auto& e : ev) LES_CUDA(cudaEventCreate(&e));
    init_spectral_attributes();  // once per device (this one is current)
    const long nf = g.field();
    for (int i = 0; i < LES_THETA; ++i) F[i] = track(dalloc<T>(nf));  // scalar fields: les_scalar_init
    for (int i = 0; i < LES_NPLANES; ++i) PL[i] = track(dalloc<T>(g.plane()));
    build_tables();
    const long se = (long)g.L * std::max((long)g.ny * pitch(g.lhx), (long)g.ny2 * pitch(g.nx / 2));
    for (int i = 0; i < NSPEC; ++i) spec[i] = track(dalloc<cplx<T>>(se));
    for (int i = 0; i < NSPEC; ++i) spec4[i] = track(dalloc<cplx<T>>((long)g.L * g.ny * pitch(nk4)));
    const long fe = (long)g.L * g.ny2 * g.nx2;
    for (auto& f : fine) f = track(dalloc<T>(fe));
    for (auto& f : sc) f = track(dalloc<T>(nf));
    for (auto& f : refbuf) f = track(dalloc<T>(g.L));
    if (mixed())
      for (auto& f : pspec) f = track(dalloc<cplx<double>>((long)g.L * g.ny * g.lhx));
    xs = track(dalloc<cplx<double>>((long)g.L * g.ny * g.lhx));
    gam = track(dalloc<double>((long)g.L * g.ny * g.lhx));
    pmean = track(dalloc<double>(g.L));
    part = track(dalloc<double>(DIAG_BLOCKS * DIAG_NV));
    dout = track(dalloc<double>(8));
    dstatus = track(dalloc<unsigned>(4));
    // system.f90:196-198 and set_bc_surface (boundary_condition_mpi.f90:124-129)
    fill(F[LES_W], 0, 0, T(BOGUS));
    fill_plane(PL[LES_LBC_Z0], T(p.z0));
    LES_CUDA(cudaStreamSynchronize(st));
  }

  ~Solver() override {
    for (cudaStream_t s : {sh2d, sd2h, st})
      if (s) cudaStreamSynchronize(s);
    for (void* q : allocs) cudaFree(q);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : {ev_go, ev_in, ev_done, ev_copies})
      if (e) cudaEventDestroy(e);
    for (auto* v : {&ev_out, &ev_inc, &ev_cvt})
      for (auto e : *v) cudaEventDestroy(e);
    for (cudaStream_t s : {sh2d, sd2h})
      if (s) cudaStreamDestroy(s);
    if (st) cudaStreamDestroy(st);
  }

  template <typename U>
  U* track(U* q) {
    allocs.push_back(q);
    return q;
  }

  // ------------------------------------------------------------ tables ----
  void build_tables() {
    const int nx = g.nx, ny = g.ny, lhx = g.lhx, lhy = g.lhy;
    const double lx = P.lx, ly = P.ly;
    std::vector<double> hkx((long)ny * lhx), hky((long)ny * lhx), hk2((long)ny * lhx);
    // fft_engine.f90:127-143
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < lhx; ++i) {
        double kx = double(i);
        double ky = double(((j + ny / 2) % ny) - ny / 2);
        if (i == lhx - 1 || j == lhy - 1) {
          kx = 0.0;
          ky = 0.0;
        }
        kx = 2.0 * PI / lx * kx;
        ky = 2.0 * PI / ly * ky;
        hkx[(long)j * lhx + i] = kx;
        hky[(long)j * lhx + i] = ky;
        hk2[(long)j * lhx + i] = kx * kx + ky * ky;
      }
    const double dx = P.lx / double(nx), dy = P.ly / double(ny), dz = P.lz / double(g.nz);
    // testfilter.f90:101-131 (cutoff compared in default REAL)
    auto make_g = [&](double alpha, int& nkc, int& kyc) {
      std::vector<T> G((long)ny * lhx);
      const double del = alpha * std::sqrt(dx * dy);
      const double q = PI / del;
      const double kc2 = q * q;
      nkc = 1;
      kyc = 0;
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < lhx; ++i) {
          double v = 1.0 / double(nx * ny);
          if (double(float(hk2[(long)j * lhx + i])) >= kc2) v = 0.0;
          if (i == lhx - 1 || j == ny / 2) v = 0.0;
          G[(long)j * lhx + i] = T(v);
          if (v != 0.0) {
            nkc = std::max(nkc, i + 1);
            kyc = std::max(kyc, std::min(j, ny - j));
          }
        }
      return G;
    };
    auto G2 = make_g(2.0, nk2, ky2);
    auto G4 = make_g(4.0, nk4, ky4);
    std::vector<T> tkx(hkx.size()), tky(hky.size());
    for (size_t i = 0; i < hkx.size(); ++i) {
      tkx[i] = T(hkx[i]);
      tky[i] = T(hky[i]);
    }
    kkx = up(tkx);
    kky = up(tky);
    kkxd = up(hkx);
    kkyd = up(hky);
    kkx64 = kkxd;
    kky64 = kkyd;
    gt = up(G2);
    gtt = up(G4);
    delta = std::pow(dx * dy * dz, 1.0 / 3.0);  // compute_sgs.f90:144
    beta_pow = std::log(2.0) / (std::log(4.0) - std::log(2.0));
    set_mixing_length();
    for (int n : {g.nx, g.ny, g.nx2, g.ny2}) twiddles(n);
  }

  void set_mixing_length() {
    // compute_sgs.f90:143-168: l = Delta, or the wall-damped cst_Smag length
    std::vector<double> l2h(g.L, delta * delta);
    const double dz = P.lz / double(g.nz);
    if (P.sgs_model == LES_SGS_CST_SMAG) {
      const double n = 2.0;
      for (int k = 1; k <= g.nz + 1; ++k) {
        const double z = (k == 1) ? 0.5 * dz : (1 + k - 2.0) * dz;
        const double l = std::pow(std::pow(P.cs0, n) * std::pow(KVONK * z, -n) + std::pow(delta, -n), -1.0 / n);
        l2h[k] = l * l;
      }
    }
    if (!l2) l2 = track(dalloc<double>(g.L));
    LES_CUDA(cudaMemcpy(l2, l2h.data(), sizeof(double) * g.L, cudaMemcpyHostToDevice));
  }

  template <typename U>
  U* up(const std::vector<U>& h) {
    U* d = track(dalloc<U>(h.size()));
    LES_CUDA(cudaMemcpy(d, h.data(), sizeof(U) * h.size(), cudaMemcpyHostToDevice));
    return d;
  }

  const cplx<double>* twiddles64(int n) {
    auto it = twd.find(n);
    if (it != twd.end()) return it->second;
    std::vector<cplx<double>> h(n);
    for (int m = 0; m < n; ++m) {
      const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
      h[m] = cplx<double>{double(std::cos(a)), double(std::sin(a))};
    }
    cplx<double>* d = up(h);
    twd[n] = d;
    return d;
  }

  const cplx<T>* twiddles(int n) {
    auto it = tw.find(n);
    if (it != tw.end()) return it->second;
    std::vector<cplx<T>> h(n);
    for (int m = 0; m < n; ++m) {
      const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
      h[m] = cplx<T>{T(std::cos(a)), T(std::sin(a))};
    }
    cplx<T>* d = up(h);
    tw[n] = d;
    return d;
  }

  // ----------------------------------------------------------- helpers ----
  T* lev(T* f, int k) const { return f + (long)k * g.plane(); }
  void fill(T* f, int k0, int k1, T v) {
    const long n = (long)(k1 - k0 + 1) * g.plane();
    KL("k_fill", double(n) * sizeof(T), k_fill<T><<<grid_for(n), 256, 0, st>>>(lev(f, k0), n, v));
  }
  // plane-sized copies / fills batched into one launch (src null: fill)
  void plane_ops(int nops, T* const* dst, const T* const* src, const T* val) {
    PlaneOps<T> o;
    std::memset(&o, 0, sizeof(o));
    for (int i = 0; i < nops; ++i) {
      o.dst[i] = dst[i];
      o.src[i] = src ? src[i] : nullptr;
      o.val[i] = val ? val[i] : T(0);
    }
    const long n = g.plane();
    double bytes = 0.0;
    for (int i = 0; i < nops; ++i) bytes += (o.src[i] ? 2.0 : 1.0) * n * sizeof(T);
    dim3 grid(unsigned(std::min<long>(ceil_div(n, 256L), 148)), unsigned(nops));
    KL("k_plane_ops", bytes, k_plane_ops<T><<<grid, 256, 0, st>>>(o, n));
  }
  void copy(T* dst, const T* src, long n) {
    KL("k_copy", 2.0 * n * sizeof(T), k_copy<T><<<grid_for(n), 256, 0, st>>>(dst, src, n));
  }
  void fill_plane(T* f, T v) {
    KL("k_fill", double(g.plane()) * sizeof(T), k_fill<T><<<grid_for(g.plane()), 256, 0, st>>>(f, g.plane(), v));
  }

  // row pitch of the spectral buffers: whole 8-value groups (64 B in FP32),
  // so that column blocks of the y pass start on sector boundaries
  static int pitch(int nk) { return (nk + 7) & ~7; }

  XFArgs<T> xf(int op, int nf, int plane0, int nplanes, int NX, int rows_pp, int nk) {
    XFArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.op = op;
    a.nf = nf;
    a.plane0 = plane0;
    a.rows_pp = rows_pp;
    a.nrows = (long)nplanes * rows_pp;
    a.nk = nk;
    a.opitch = pitch(nk);
    a.nz = g.nz;
    a.wall = P.wall_law;
    a.in_pstride = (long)rows_pp * NX;
    a.out_pstride = (long)rows_pp * a.opitch;
    a.tw = twiddles(NX);
    return a;
  }
  YPArgs<T> yp(int op, int nin, int nout, int ncols, int nk_in, int NY, int nk_out, int NYO, int plane0) {
    YPArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.op = op;
    a.nin = nin;
    a.nout = nout;
    a.ncols = ncols;
    a.nk_in = nk_in;
    a.nk_out = nk_out;
    a.ipitch = pitch(nk_in);
    a.opitch = pitch(nk_out);
    a.in_pstride = (long)NY * a.ipitch;
    a.out_pstride = (long)NYO * a.opitch;
    a.plane0 = plane0;
    a.nxh = g.nx / 2;
    a.lhx = g.lhx;
    a.kkx = kkx;
    a.kky = kky;
    a.tw_in = twiddles(NY);
    a.tw_out = twiddles(NYO);
    return a;
  }
  XIArgs<T> xi(int op, int nin, int plane0, int nplanes, int NX, int rows_pp, int nk) {
    XIArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.op = op;
    a.nin = nin;
    a.plane0 = plane0;
    a.rows_pp = rows_pp;
    a.nrows = (long)nplanes * rows_pp;
    a.nk = nk;
    a.ipitch = pitch(nk);
    a.nz = g.nz;
    a.in_pstride = (long)rows_pp * a.ipitch;
    a.out_pstride = (long)rows_pp * NX;
    a.tw = twiddles(NX);
    a.status = dstatus;
    return a;
  }

  // ------------------------------------------------------ data movement ----
  void upload(int field, const double* h, int k0, int k1) override {
    check_field(field, k0, k1);
    const long n = (long)(k1 - k0 + 1) * g.plane();
    std::vector<T> tmp(n);
    for (long i = 0; i < n; ++i) tmp[i] = T(h[i]);
    LES_CUDA(cudaMemcpyAsync(lev(F[field], k0), tmp.data(), n * sizeof(T), cudaMemcpyHostToDevice, st));
    LES_CUDA(cudaStreamSynchronize(st));
  }
  void download(int field, double* h, int k0, int k1) override {
    check_field(field, k0, k1);
    const long n = (long)(k1 - k0 + 1) * g.plane();
    std::vector<T> tmp(n);
    LES_CUDA(cudaMemcpyAsync(tmp.data(), lev(F[field], k0), n * sizeof(T), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    for (long i = 0; i < n; ++i) h[i] = double(tmp[i]);
  }
  void upload_plane(int plane, const double* h) override {
    if (plane < 0 || plane >= LES_NPLANES) throw CudaError(1, "invalid plane id");
    std::vector<T> tmp(g.plane());
    for (long i = 0; i < g.plane(); ++i) tmp[i] = T(h[i]);
    LES_CUDA(cudaMemcpyAsync(PL[plane], tmp.data(), g.plane() * sizeof(T), cudaMemcpyHostToDevice, st));
    LES_CUDA(cudaStreamSynchronize(st));
  }
  void download_plane(int plane, double* h) override {
    if (plane < 0 || plane >= LES_NPLANES) throw CudaError(1, "invalid plane id");
    std::vector<T> tmp(g.plane());
    LES_CUDA(cudaMemcpyAsync(tmp.data(), PL[plane], g.plane() * sizeof(T), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    for (long i = 0; i < g.plane(); ++i) h[i] = double(tmp[i]);
  }
  bool has_field(int f) const override { return f >= 0 && f < LES_NFIELDS && F[f] != nullptr; }
  void check_field(int field, int k0, int k1) const {
    if (field < 0 || field >= LES_NFIELDS) throw CudaError(1, "invalid field id");
    if (!F[field]) throw CudaError(1, "field not allocated (the scalar fields need les_scalar_init)");
    if (k0 < 0 || k1 > g.nz + 1 || k1 < k0) throw CudaError(1, "invalid level range");
  }

  // ------------------------------------------------------ learned closure ----
  MlpDevice md;
  bool mlp_alloc = false, mlp_ready = false;
  long mlp_updates = 0;
  int mlp_check_every = 10;  // dynamic-procedure check every 10 updates (50 steps at cs_count 5)
  int mlp_wall_levels = 0;   // levels 1..n next to the wall keep the LASD procedure
  double mlp_last_err = -1.0;
  std::vector<double> mlp_profile;  // RMS log error per level at the last check
  int mlp_last_flags = 0;
  int mlp_feature_flags[8] = {};
  int* dcount = nullptr;
  double* derr = nullptr;
  int mlp_adam_step = 0;
  T* cs_prev = nullptr;      // Cs^2 before the current update
  bool have_prev = false;    // cs_prev holds the previous collection's coefficient

  void ensure_mlp() {
    if (mlp_alloc) return;
    md.params = track(dalloc<float>(MLP_NP));
    md.stats = track(dalloc<float>(MLP_NS));
    md.img = track(dalloc<uint16_t>(18432 / 2));
    md.grad = track(dalloc<float>(MLP_NP));
    md.adam_m = track(dalloc<float>(MLP_NP));
    md.adam_v = track(dalloc<float>(MLP_NP));
    md.colflag = track(dalloc<int>(g.plane()));
    md.range = track(dalloc<int>(16));
    md.counts = track(dalloc<unsigned long long>(2));
    md.boff = track(dalloc<unsigned long long>(2 * MLP_COLLECT_BLOCKS));
    md.gpart = track(dalloc<float>((size_t)MLP_TRAIN_CTAS * MLP_NP));
    md.lpart = track(dalloc<float>(MLP_TRAIN_CTAS));
    md.plane = g.plane();
    dcount = track(dalloc<int>(9));
    derr = track(dalloc<double>((size_t)MLP_BLEND_BLOCKS * g.L));
    mlp_profile.assign(g.L, -1.0);
    cs_prev = track(dalloc<T>(g.field()));
    init_mlp_attributes();
    mlp_alloc = true;
  }
  MlpFeatIn<T> feat_in() {
    MlpFeatIn<T> a;
    const int d[9] = {LES_DUDX, LES_DUDY, LES_DUDZ, LES_DVDX, LES_DVDY, LES_DVDZ, LES_DWDX, LES_DWDY, LES_DWDZ};
    for (int q = 0; q < 9; ++q) a.d[q] = F[d[q]];
    a.csprev = cs_prev;
    a.wall_levels = std::min(mlp_wall_levels, g.nz + 1);
    a.plane = g.plane();
    a.nz = g.nz;
    a.wall = P.wall_law;
    a.dz = float(dz());
    a.delta = float(delta);
    a.log_delta_z0 = float(std::log(delta / P.z0));
    a.cs_max = cs2_max > 0.0 ? float(std::min(cs2_max, 1.0)) : 1.0f;
    if (scalar_on && SP.buoyancy != 0.0) {
      a.dtdz = F[LES_DTDZ];
      a.beta = float(SP.buoyancy);
    }
    return a;
  }
  void set_sgs_model(int m) override {
    if (m < LES_SGS_CST_SMAG || m > LES_SGS_MLP) throw CudaError(1, "Invalid SGS model");
    P.sgs_model = m;
    set_mixing_length();
  }
  void mlp_init(unsigned seed) override {
    ensure_mlp();
    std::mt19937 rng(seed);
    std::vector<float> p(MLP_NP, 0.0f);
    auto fill_w = [&](int off, int fin, int fout) {
      std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / float(fin + fout)));
      for (int i = 0; i < fin * fout; ++i) p[off + i] = nd(rng);
    };
    fill_w(MLP_O_W1, MLP_IN, MLP_H);
    fill_w(MLP_O_W2, MLP_H, MLP_H);
    fill_w(MLP_O_W3, MLP_H, 1);
    std::vector<float> s(MLP_NS, 0.0f);
    for (int i = 0; i < 8; ++i) {
      s[MLP_S_SD + i] = 1.0f;
      s[MLP_S_MIN + i] = -1e30f;
      s[MLP_S_MAX + i] = 1e30f;
    }
    s[MLP_S_YMU] = 0.0f;  // no change of the coefficient
    s[MLP_S_YSD] = 1.0f;
    s[MLP_S_YMIN] = -1e30f;
    s[MLP_S_YMAX] = 1e30f;
    std::vector<float> all(p);
    all.insert(all.end(), s.begin(), s.end());
    mlp_set_params(all.data(), MLP_NP + MLP_NS);
    LES_CUDA(cudaMemsetAsync(md.adam_m, 0, sizeof(float) * MLP_NP, st));
    LES_CUDA(cudaMemsetAsync(md.adam_v, 0, sizeof(float) * MLP_NP, st));
    mlp_adam_step = 0;
  }
  void mlp_set_params(const float* p, int n) override {
    if (n != MLP_NP + MLP_NS) throw CudaError(1, "learned closure: expected " + std::to_string(MLP_NP + MLP_NS) + " values");
    ensure_mlp();
    LES_CUDA(cudaMemcpyAsync(md.params, p, sizeof(float) * MLP_NP, cudaMemcpyHostToDevice, st));
    LES_CUDA(cudaMemcpyAsync(md.stats, p + MLP_NP, sizeof(float) * MLP_NS, cudaMemcpyHostToDevice, st));
    mlp_pack(md, st);
    LES_CUDA(cudaStreamSynchronize(st));
    mlp_ready = true;
  }
  void mlp_get_params(float* p, int n) override {
    if (n != MLP_NP + MLP_NS) throw CudaError(1, "learned closure: expected " + std::to_string(MLP_NP + MLP_NS) + " values");
    ensure_mlp();
    LES_CUDA(cudaMemcpyAsync(p, md.params, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaMemcpyAsync(p + MLP_NP, md.stats, sizeof(float) * MLP_NS, cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
  }
  void mlp_reset_data(long cap) override {
    ensure_mlp();
    if (cap != md.cap) {
      for (float* q : {md.dx, md.dt, md.vx, md.vt})
        if (q) {
          cudaFree(q);
          allocs.erase(std::remove(allocs.begin(), allocs.end(), (void*)q), allocs.end());
        }
      md.cap = cap;
      md.dx = track(dalloc<float>(cap * MLP_IN));
      md.dt = track(dalloc<float>(cap));
      md.vx = track(dalloc<float>(cap * MLP_IN));
      md.vt = track(dalloc<float>(cap));
    }
    LES_CUDA(cudaMemsetAsync(md.counts, 0, 2 * sizeof(unsigned long long), st));
    mlp_reset_range(md, st);
  }
  void mlp_collect(int stride, int dense_levels, int wall_repeat, unsigned seed) override {
    if (!mlp_alloc || md.cap == 0) throw CudaError(1, "learned closure: call les_mlp_reset_data first");
    Tag tag_(this, "mlp");
    ensure_mlp();
    // pairs (features with the previous collection's coefficient, current
    // coefficient): collect at consecutive dynamic updates; the first call
    // only records the coefficient
    if (have_prev)
      les::mlp_collect<T>(feat_in(), F[LES_CS_OPT2], md, std::max(1, stride), dense_levels,
                          std::min(16, std::max(1, wall_repeat)), seed, st);
    copy(cs_prev, F[LES_CS_OPT2], g.field());
    have_prev = true;
  }
  void mlp_counts(long long* c) override {
    ensure_mlp();
    unsigned long long h[2];
    LES_CUDA(cudaMemcpyAsync(h, md.counts, sizeof(h), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    c[0] = std::min<long long>(h[0], md.cap);
    c[1] = std::min<long long>(h[1], md.cap);
  }
  void mlp_fit_stats() override {
    ensure_mlp();
    les::mlp_fit_stats(md, st);
  }
  void mlp_train(int epochs, int tiles_per_step, double lr, double* loss_epochs, double* val_loss) override {
    ensure_mlp();
    Tag tag_(this, "mlp_train");
    long long c[2];
    mlp_counts(c);
    const long ntr = c[0], nva = c[1];
    if (ntr < 128) throw CudaError(1, "learned closure: not enough training data");
    const long chunk = long(std::max(1, tiles_per_step)) * 128;
    const long nsteps = (ntr + chunk - 1) / chunk;
    float* dloss = nullptr;
    LES_CUDA(cudaMalloc(&dloss, (nsteps + 1) * sizeof(float)));
    std::vector<float> hl(nsteps);
    std::mt19937_64 rng(0x5eed0000ull + (unsigned long long)mlp_adam_step);
    auto gcdl = [](unsigned long long a, unsigned long long b) {
      while (b) {
        const unsigned long long t = a % b;
        a = b;
        b = t;
      }
      return a;
    };
    for (int ep = 0; ep < epochs; ++ep) {
      // a fresh permutation of the training pairs each epoch: batches mix
      // levels and collection steps
      MlpPerm pm;
      pm.n = ntr;
      do {
        pm.a = 1 + rng() % (unsigned long long)(ntr - 1);
      } while (gcdl(pm.a, (unsigned long long)ntr) != 1);
      pm.b = rng() % (unsigned long long)ntr;
      for (long s = 0; s < nsteps; ++s) {
        pm.off = s * chunk;
        const long n = std::min(chunk, ntr - pm.off);
        mlp_grad(md, md.dx, md.dt, n, nullptr, dloss + s, dstatus, st, pm);
        mlp_adam(md, ++mlp_adam_step, float(lr), st);
      }
      LES_CUDA(cudaMemcpyAsync(hl.data(), dloss, nsteps * sizeof(float), cudaMemcpyDeviceToHost, st));
      LES_CUDA(cudaStreamSynchronize(st));
      double sum = 0.0, wsum = 0.0;
      for (long s = 0; s < nsteps; ++s) {
        const double w = double(std::min(chunk, ntr - s * chunk));
        sum += w * hl[s];
        wsum += w;
      }
      if (loss_epochs) loss_epochs[ep] = sum / wsum;  // mean batch loss of the epoch
    }
    if (val_loss) {
      *val_loss = -1.0;
      if (nva > 0) {
        mlp_grad(md, md.vx, md.vt, nva, nullptr, dloss, dstatus, st);
        float h = 0;
        LES_CUDA(cudaMemcpyAsync(&h, dloss, sizeof(float), cudaMemcpyDeviceToHost, st));
        LES_CUDA(cudaStreamSynchronize(st));
        *val_loss = h;
      }
    }
    cudaFree(dloss);
    mlp_ready = true;
  }
  void mlp_forward_host(const float* x, long n, float* y) override {
    ensure_mlp();
    float *dxx = nullptr, *dtt = nullptr, *dyy = nullptr;
    LES_CUDA(cudaMalloc(&dxx, sizeof(float) * n * MLP_IN));
    LES_CUDA(cudaMalloc(&dtt, sizeof(float) * n));
    LES_CUDA(cudaMalloc(&dyy, sizeof(float) * n));
    LES_CUDA(cudaMemcpyAsync(dxx, x, sizeof(float) * n * MLP_IN, cudaMemcpyHostToDevice, st));
    LES_CUDA(cudaMemsetAsync(dtt, 0, sizeof(float) * n, st));
    mlp_grad(md, dxx, dtt, n, dyy, nullptr, dstatus, st);
    LES_CUDA(cudaMemcpyAsync(y, dyy, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    cudaFree(dxx);
    cudaFree(dtt);
    cudaFree(dyy);
  }
  void mlp_grad_host(const float* x, const float* t, long n, float* gr, float* loss) override {
    ensure_mlp();
    float *dxx = nullptr, *dtt = nullptr, *dl = nullptr;
    LES_CUDA(cudaMalloc(&dxx, sizeof(float) * n * MLP_IN));
    LES_CUDA(cudaMalloc(&dtt, sizeof(float) * n));
    LES_CUDA(cudaMalloc(&dl, sizeof(float)));
    LES_CUDA(cudaMemcpyAsync(dxx, x, sizeof(float) * n * MLP_IN, cudaMemcpyHostToDevice, st));
    LES_CUDA(cudaMemcpyAsync(dtt, t, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    LES_CUDA(cudaMemsetAsync(dl, 0, sizeof(float), st));
    mlp_grad(md, dxx, dtt, n, nullptr, dl, dstatus, st);
    LES_CUDA(cudaMemcpyAsync(gr, md.grad, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    cudaFree(dxx);
    cudaFree(dtt);
    cudaFree(dl);
  }
  void mlp_set_check_every(int every) override { mlp_check_every = every; }
  void mlp_set_wall_levels(int n) override { mlp_wall_levels = std::max(0, n); }
  void mlp_check_profile(double* out, int n) override {
    if (n < g.nz + 1) throw CudaError(1, "learned closure: profile needs nz + 1 values");
    for (int k = 1; k <= g.nz + 1; ++k) out[k - 1] = mlp_profile.empty() ? -1.0 : mlp_profile[k];
  }
  void mlp_info(double* out) override {
    out[0] = mlp_last_err;
    out[1] = mlp_last_flags;
    out[2] = double(mlp_updates);
    out[3] = mlp_ready ? 1.0 : 0.0;
    for (int i = 0; i < 8; ++i) out[4 + i] = mlp_feature_flags[i];
  }

  // Cs^2 from the learned closure at the dynamic-update cadence; columns whose
  // invariants left the training range take the dynamic procedure's value,
  // which also checks the closure every mlp_check_every updates.
  void mlp_sgs(SgsArgs<T>& a, int jtt) {
    Tag tag_(this, "mlp");
    const int nb = std::min(mlp_wall_levels, g.nz + 1);
    if (jtt < P.dyn_init) {
      fill(F[LES_CS_OPT2], 1, g.nz + 1, T(0.03));
      return;
    }
    if (jtt % P.cs_count != 0) {
      if (nb > 0) lasd(a, jtt, nb);  // Lagrangian accumulation of the wall band
      return;
    }
    if (!mlp_ready) throw CudaError(1, "learned closure has no weights (train it or load parameters)");
    copy(cs_prev, F[LES_CS_OPT2], g.field());
    have_prev = true;
    les::mlp_infer<T>(feat_in(), F[LES_CS_OPT2], md, dstatus, st);
    ++mlp_updates;
    mlp_last_flags = mlp_count_flags(md, dcount, mlp_feature_flags, st);
    const bool check = mlp_check_every > 0 && (mlp_updates % mlp_check_every) == 0;
    if (mlp_last_flags > 0 || check) {
      // one Lagrangian relaxation step of the dynamic procedure starting from
      // the coefficient before this update (the reference's F initialisation
      // with Cs^2 = cs_prev instead of 0.03), into scratch: cs -> sc[11]
      dynamic_mum(a, true);
      const long n1 = (long)(g.nz + 1) * g.plane();
      KL("k_lasd_update", 14.0 * n1 * sizeof(T),
         k_lasd_update<T><<<grid_for(n1), 256, 0, st>>>(sc[0], sc[12], sc[13], sc[14], sc[7], sc[8], sc[9], sc[10],
                                                       sc[11], sc[1], 1, g.plane(), g.nz, 1.5 * delta,
                                                       P.dt * double(P.cs_count), beta_pow, cs_prev, -1, cs2_max));
      std::vector<double> prof(g.L, 0.0);
      mlp_blend<T>(F[LES_CS_OPT2], sc[11], md, g.nz, check, derr, prof.data(), st);
      if (check) {
        // the closure's error where it is used: levels above the wall band
        double s2 = 0.0;
        int nl = 0;
        for (int k = nb + 1; k <= g.nz + 1; ++k, ++nl) s2 += prof[k] * prof[k];
        mlp_last_err = nl ? std::sqrt(s2 / nl) : 0.0;
        mlp_profile = prof;
      }
    }
    if (nb > 0) lasd(a, jtt, nb);  // the wall band: the plain procedure, Lagrangian history kept
  }

  // ------------------------------------------------------------ restart ----
  // IO_checkpoint.f90:119-256 on one rank: native FP64 records of
  // nx*ny*(nz+1) values (levels 1..nz+1, x fastest): u, v, w, rhsx, rhsy,
  // rhsz, cs_opt2, then F_LM, F_MM, F_QN, F_NN when the Lagrangian averages
  // exist (Lagran_init).
  std::vector<int> checkpoint_fields(bool with_f) const {
    std::vector<int> ids = {LES_U, LES_V, LES_W, LES_RHSX, LES_RHSY, LES_RHSZ, LES_CS_OPT2};
    if (with_f)
      for (int q : {LES_F_LM, LES_F_MM, LES_F_QN, LES_F_NN}) ids.push_back(q);
    return ids;
  }
  void checkpoint_write(const char* path) override {
    FILE* f = std::fopen(path, "wb");
    if (!f) throw CudaError(1, std::string("[checkpoint error] cannot open checkpoint file ") + path);
    const long n = (long)(g.nz + 1) * g.plane();
    std::vector<double> buf(n);
    bool ok = true;
    for (int id : checkpoint_fields(lagran_init)) {
      download(id, buf.data(), 1, g.nz + 1);
      ok = ok && std::fwrite(buf.data(), sizeof(double), n, f) == size_t(n);
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) throw CudaError(22, std::string("[checkpoint error] cannot write checkpoint file ") + path);
  }
  void checkpoint_read(const char* path, int with_f) override {
    FILE* f = std::fopen(path, "rb");
    if (!f) throw CudaError(1, std::string("[Restart error] cannot open checkpoint file ") + path);
    const long n = (long)(g.nz + 1) * g.plane();
    const auto ids = checkpoint_fields(with_f != 0);
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (bytes < long(ids.size()) * n * long(sizeof(double))) {
      std::fclose(f);
      throw CudaError(1, std::string("[Restart error] checkpoint file too short for this grid: ") + path);
    }
    std::vector<double> buf(n);
    for (int id : ids) {
      if (std::fread(buf.data(), sizeof(double), n, f) != size_t(n)) {
        std::fclose(f);
        throw CudaError(22, std::string("[Restart error] cannot read checkpoint file ") + path);
      }
      upload(id, buf.data(), 1, g.nz + 1);
    }
    std::fclose(f);
    // the Lagrangian accumulators restart empty (they are not in the file);
    // w(0) keeps its allocation value (system.f90:196-198), and the wall law
    // switches the lower u, v conditions to Neumann as after the initial
    // conditions (LES_engine.f90:160-171)
    for (int q : {LES_U_LAG, LES_V_LAG, LES_W_LAG}) fill(F[q], 0, g.nz + 1, T(0));
    fill(F[LES_W], 0, 0, T(BOGUS));
    if (P.wall_law) {
      lbc_t[0] = 2;
      lbc_t[1] = 2;
    }
    if (with_f) {  // compute_LagScaleDep.f90:66
      f_coeff_init = true;
      lagran_init = true;
    }
    LES_CUDA(cudaStreamSynchronize(st));
  }

  // --------------------------------------------------------- statistics ----
  // Running sums of IO_statistics.f90 (io_stat_init :40-250, io_stat_averages
  // :265-291, 2D :300-354, 3D :363-518) and the plane-averaged TKE budget of
  // tke_budget1D.f90 (tke_budget_init :61-160, compute_tke_budget :209-390,
  // avg_var :396-420), one rank.
  double* stat_acc = nullptr;    // [26][nz][ny][nx] running sums
  double* stat_ustar = nullptr;  // [ny][nx] running sum of u*
  int stat_iterations = 0;
  T* tke_f[3] = {};  // cleaned pressure (filtered), its x and y derivatives
  double* tke_part = nullptr;
  double* tke_avar = nullptr;  // [61][nz] running plane averages
  int tke_nch = 1, tke_ii = 1;
  std::string tke_dir;

  static std::string nine(int v) {
    char b[32];
    std::snprintf(b, sizeof b, "%09d", v);
    return b;
  }
  void write_host(const std::string& path, const std::vector<const double*>& parts, long n) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw CudaError(22, "cannot open statistics file " + path);
    bool ok = true;
    for (const double* p : parts) ok = ok && std::fwrite(p, sizeof(double), n, f) == size_t(n);
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) throw CudaError(22, "cannot write statistics file " + path);
  }
  std::vector<double> to_host(const double* d, long n) {
    std::vector<double> h(n);
    LES_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    return h;
  }

  void stat_init() override {
    const long n = (long)STAT_NQ * g.nz * g.plane();
    if (!stat_acc) {
      stat_acc = track(dalloc<double>(n));
      stat_ustar = track(dalloc<double>(g.plane()));
    } else {
      LES_CUDA(cudaMemsetAsync(stat_acc, 0, n * sizeof(double), st));
      LES_CUDA(cudaMemsetAsync(stat_ustar, 0, g.plane() * sizeof(double), st));
    }
    stat_iterations = 0;
  }
  void stat_averages(int jt, int jtt, int start_stats, int running_period, const char* out_path) override {
    (void)jt;
    if (!stat_acc) throw CudaError(1, "running statistics are not initialised (les_stat_init)");
    if (running_period <= 0) throw CudaError(1, "running_period must be positive");
    Tag tag_(this, "stats");
    const long plane = g.plane(), n = (long)g.nz * plane;
    const bool write = (jtt % running_period == 0) && jtt > start_stats;
    const std::string base = std::string(out_path) + "RAV_" + nine(jtt);
    ++stat_iterations;
    if (write) {
      FILE* f = std::fopen((base + "_info.txt").c_str(), "w");
      if (!f) throw CudaError(22, "cannot open statistics file " + base + "_info.txt");
      std::fprintf(f, "%6d%6d%6d%10d\n", g.nx, g.ny, g.nz, stat_iterations);
      if (std::fclose(f) != 0) throw CudaError(22, "cannot write statistics file " + base + "_info.txt");
      stat_iterations = 0;
    }
    KL("k_plane_accum", 20.0 * plane,
       k_plane_accum<T><<<grid_for(plane), 256, 0, st>>>(PL[LES_U_STAR_AVG], stat_ustar, plane));
    if (write) {
      const auto h = to_host(stat_ustar, plane);
      write_host(base + "_2D.dat", {h.data()}, plane);
      LES_CUDA(cudaMemsetAsync(stat_ustar, 0, plane * sizeof(double), st));
    }
    StatFields<T> sf{F[LES_U],   F[LES_V],   F[LES_W],   F[LES_P],    F[LES_TXX],  F[LES_TYY], F[LES_TZZ],
                     F[LES_TXY], F[LES_TXZ], F[LES_TYZ], F[LES_DUDZ], F[LES_DVDZ], F[LES_NU_T], F[LES_CS_OPT2]};
    KL("k_stat_accum", double(n) * (16.0 * STAT_NQ + 16.0 * sizeof(T)),
       k_stat_accum<T><<<grid_for(n), 256, 0, st>>>(sf, stat_acc, plane, g.nz));
    if (write) {
      const auto h = to_host(stat_acc, STAT_NQ * n);
      std::vector<const double*> parts;
      for (int q = 0; q < STAT_NQ; ++q) parts.push_back(h.data() + q * n);
      write_host(base + "_3D.dat", parts, n);
      LES_CUDA(cudaMemsetAsync(stat_acc, 0, STAT_NQ * n * sizeof(double), st));
    }
    LES_CUDA(cudaStreamSynchronize(st));
  }
  void stat_sums(int index, double* out) override {
    if (!stat_acc) throw CudaError(1, "running statistics are not initialised (les_stat_init)");
    if (index < 0 || index > STAT_NQ) throw CudaError(1, "statistics index out of range");
    const long n = (long)g.nz * g.plane();
    const double* src = index == STAT_NQ ? stat_ustar : stat_acc + (long)index * n;
    const long cnt = index == STAT_NQ ? g.plane() : n;
    LES_CUDA(cudaMemcpyAsync(out, src, cnt * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
  }
  int stat_iteration_count() override { return stat_iterations; }

  // io_stat_spectra (IO_statistics.f90:566-581, out :583-620): u, v, w on
  // levels 1..nz in the four fixed windows of jt_total, every 10th jt
  void stat_spectra(int jt, int jtt, const char* out_path) override {
    bool hit = false;
    for (int lo : {1500000, 1550000, 1600000, 1650000}) hit = hit || (jtt >= lo && jtt <= lo + 2000 && jt % 10 == 0);
    if (!hit) return;
    const long n = (long)g.nz * g.plane();
    std::vector<double> u(n), v(n), w(n);
    download(LES_U, u.data(), 1, g.nz);
    download(LES_V, v.data(), 1, g.nz);
    download(LES_W, w.data(), 1, g.nz);
    write_host(std::string(out_path) + "SP_" + nine(jtt) + ".dat", {u.data(), v.data(), w.data()}, n);
  }

  void tke_init(const char* out_path) override {
    tke_dir = std::string(out_path) + "ta1_profiles/";
    ::mkdir(tke_dir.c_str(), 0755);  // like the reference's system('mkdir'): an existing folder is fine
    const int per_level = std::max(1, std::min(64, (4 * 148 + g.nz - 1) / g.nz));
    tke_nch = int(std::min<long>(per_level, (g.plane() + 255) / 256));
    if (!tke_avar) {
      for (auto& f : tke_f) f = track(dalloc<T>(g.field()));
      tke_part = track(dalloc<double>((long)g.nz * 64 * TKE_NQ));
      tke_avar = track(dalloc<double>((long)TKE_NQ * g.nz));
    } else {
      LES_CUDA(cudaMemsetAsync(tke_avar, 0, (long)TKE_NQ * g.nz * sizeof(double), st));
    }
    tke_ii = 1;  // (actLaunch-1)*(nt/tke_period)+1 with actLaunch = 1
  }
  void tke_budget(int jt, int tke_period) override {
    if (!tke_avar) throw CudaError(1, "TKE budget is not initialised (les_tke_init)");
    if (tke_period <= 0) throw CudaError(1, "tke_period must be positive");
    Tag tag_(this, "tke");
    const long plane = g.plane();
    KL("k_tke_cpress", 6.0 * g.field() * sizeof(T),
       k_tke_cpress<T><<<grid_for(g.field()), 256, 0, st>>>(F[LES_P], F[LES_U], F[LES_V], F[LES_W], F[LES_CS_OPT2],
                                                             tke_f[0], plane, g.nz));
    grad_ptrs(&tke_f[0], &tke_f[1], &tke_f[2], 1);
    TkeFields<T> tf{F[LES_U],    F[LES_V],    F[LES_W],    F[LES_DUDX], F[LES_DUDY], F[LES_DUDZ],
                    F[LES_DVDX], F[LES_DVDY], F[LES_DVDZ], F[LES_DWDX], F[LES_DWDY], F[LES_DWDZ],
                    F[LES_TXX],  F[LES_TYY],  F[LES_TZZ],  F[LES_TXY],  F[LES_TXZ],  F[LES_TYZ],
                    F[LES_CS_OPT2], tke_f[0], tke_f[1], tke_f[2]};
    const dim3 grid(tke_nch, g.nz);
    const double idz = 1.0 / dz(), bytes = 26.0 * g.nz * plane * sizeof(T);
    KL("k_tke_partial", bytes, k_tke_partial<T, 0, 16><<<grid, 256, 0, st>>>(tf, tke_part, plane, P.wall_law, idz));
    KL("k_tke_partial", bytes, k_tke_partial<T, 16, 16><<<grid, 256, 0, st>>>(tf, tke_part, plane, P.wall_law, idz));
    KL("k_tke_partial", bytes, k_tke_partial<T, 32, 16><<<grid, 256, 0, st>>>(tf, tke_part, plane, P.wall_law, idz));
    KL("k_tke_partial", bytes, k_tke_partial<T, 48, 13><<<grid, 256, 0, st>>>(tf, tke_part, plane, P.wall_law, idz));
    KL("k_tke_final", 8.0 * g.nz * tke_nch * TKE_NQ,
       k_tke_final<<<grid_for((long)g.nz * TKE_NQ), 256, 0, st>>>(tke_part, tke_nch, g.nz,
                                                                 double(g.nx) * double(g.ny), tke_avar));
    if (jt % tke_period == 0) {
      // avg_var :408-418: record ii (nz FP64 values, the 4-byte record units
      // of recl = 2*nz) of <name>.out holds the sums over tke_period
      const auto h = to_host(tke_avar, (long)TKE_NQ * g.nz);
      std::vector<double> rec(g.nz);
      for (int q = 0; q < TKE_NQ; ++q) {
        for (int k = 0; k < g.nz; ++k) rec[k] = h[(long)q * g.nz + k] / double(tke_period);
        const std::string path = tke_dir + TKE_NAMES[q] + ".out";
        FILE* f = std::fopen(path.c_str(), "r+b");
        if (!f) f = std::fopen(path.c_str(), "w+b");
        if (!f) throw CudaError(22, "cannot open TKE budget file " + path);
        bool ok = std::fseek(f, long(tke_ii - 1) * g.nz * long(sizeof(double)), SEEK_SET) == 0;
        ok = ok && std::fwrite(rec.data(), sizeof(double), g.nz, f) == size_t(g.nz);
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) throw CudaError(22, "cannot write TKE budget file " + path);
      }
      LES_CUDA(cudaMemsetAsync(tke_avar, 0, (long)TKE_NQ * g.nz * sizeof(double), st));
      ++tke_ii;
    }
    LES_CUDA(cudaStreamSynchronize(st));
  }
  void tke_sums(double* out, int* record) override {
    if (!tke_avar) throw CudaError(1, "TKE budget is not initialised (les_tke_init)");
    LES_CUDA(cudaMemcpyAsync(out, tke_avar, (long)TKE_NQ * g.nz * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    *record = tke_ii;
  }

  double* staging = nullptr;  // FP64 device staging field (mixed precision transfers)
  void upload_async(int field, const double* h, int k0, int k1) override {
    check_field(field, k0, k1);
    const long n = (long)(k1 - k0 + 1) * g.plane();
    if constexpr (std::is_same<T, double>::value) {
      LES_CUDA(cudaMemcpyAsync(lev(F[field], k0), h, n * sizeof(double), cudaMemcpyHostToDevice, st));
    } else {
      if (!staging) staging = track(dalloc<double>(g.field()));
      LES_CUDA(cudaMemcpyAsync(staging, h, n * sizeof(double), cudaMemcpyHostToDevice, st));
      KL("k_convert", 12.0 * n, k_convert<T, double><<<grid_for(n), 256, 0, st>>>(lev(F[field], k0), staging, n));
    }
  }
  void download_async(int field, double* h, int k0, int k1) override {
    check_field(field, k0, k1);
    const long n = (long)(k1 - k0 + 1) * g.plane();
    if constexpr (std::is_same<T, double>::value) {
      LES_CUDA(cudaMemcpyAsync(h, lev(F[field], k0), n * sizeof(double), cudaMemcpyDeviceToHost, st));
    } else {
      if (!staging) staging = track(dalloc<double>(g.field()));
      KL("k_convert", 12.0 * n, k_convert<double, T><<<grid_for(n), 256, 0, st>>>(staging, lev(F[field], k0), n));
      LES_CUDA(cudaMemcpyAsync(h, staging, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
  }
  void diagnostics_async(double* h) override {
    diagnostics_launch();
    LES_CUDA(cudaMemcpyAsync(h, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  }

  // ------------------------------------------- step with host velocity ----
  // Copies in on sh2d, the step on st, copies back on sd2h, per chunk of
  // ~16 MB of levels.  The copy in of a chunk waits for the previous call's
  // copy back of the same chunk (same host memory; in FP64 also the same
  // device levels), so that one call's copies back and the next call's
  // copies in run at the same time, one in each direction of the link.
  // Mixed precision stages the FP64 values in device buffers (one set per
  // direction) and converts on st chunk by chunk: a chunk in as soon as it
  // has arrived, a chunk out just before its copy back.
  cudaStream_t sh2d = nullptr, sd2h = nullptr;
  cudaEvent_t ev_go = nullptr, ev_in = nullptr, ev_done = nullptr;
  std::vector<cudaEvent_t> ev_out;  // per (field, chunk): copy back done
  std::vector<cudaEvent_t> ev_inc;  // per (field, chunk): copy in done (mixed precision)
  std::vector<cudaEvent_t> ev_cvt;  // per (field, chunk): converted for the copy back (mixed)
  bool out_recorded = false;
  double* stage_in[3] = {};
  double* stage_out[3] = {};
  int chunk_lev = 0, nchunk = 0;

  void setup_host_pipe() {
    LES_CUDA(cudaStreamCreateWithFlags(&sh2d, cudaStreamNonBlocking));
    LES_CUDA(cudaStreamCreateWithFlags(&sd2h, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&ev_go, &ev_in, &ev_done, &ev_copies})
      LES_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    const long pb = g.plane() * (long)sizeof(double);
    chunk_lev = int(std::max(1L, (16L << 20) / pb));
    nchunk = (g.L + chunk_lev - 1) / chunk_lev;
    for (auto* v : {&ev_out, &ev_inc, &ev_cvt}) {
      v->assign(3 * nchunk, nullptr);
      for (auto& e : *v) LES_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (mixed())
      for (int q = 0; q < 3; ++q) {
        stage_in[q] = track(dalloc<double>(g.field()));
        stage_out[q] = track(dalloc<double>(g.field()));
      }
  }

  void step_host(int jt, int jtt, double* u, double* v, double* w, double* diag4) override {
    if (!sh2d) setup_host_pipe();
    double* h[3] = {u, v, w};
    const int fid[3] = {LES_U, LES_V, LES_W};
    constexpr bool f64 = std::is_same<T, double>::value;
    auto dev_in = [&](int q) -> double* {
      if constexpr (f64) return F[fid[q]];
      else return stage_in[q];
    };
    auto dev_out = [&](int q) -> const double* {
      if constexpr (f64) return F[fid[q]];
      else return stage_out[q];
    };
    auto chunk = [&](int c, int& k0, long& n) {
      k0 = c * chunk_lev;
      n = (long)(std::min(g.L, k0 + chunk_lev) - k0) * g.plane();
    };
    // the copies in follow everything queued on st before this call
    LES_CUDA(cudaEventRecord(ev_go, st));
    LES_CUDA(cudaStreamWaitEvent(sh2d, ev_go, 0));
    for (int q = 0; q < 3; ++q)
      for (int c = 0; c < nchunk; ++c) {
        int k0;
        long n;
        chunk(c, k0, n);
        if (out_recorded) LES_CUDA(cudaStreamWaitEvent(sh2d, ev_out[q * nchunk + c], 0));
        LES_CUDA(cudaMemcpyAsync(dev_in(q) + k0 * g.plane(), h[q] + k0 * g.plane(), n * sizeof(double),
                                 cudaMemcpyHostToDevice, sh2d));
        if constexpr (!f64) LES_CUDA(cudaEventRecord(ev_inc[q * nchunk + c], sh2d));
      }
    if constexpr (f64) {
      LES_CUDA(cudaEventRecord(ev_in, sh2d));
      LES_CUDA(cudaStreamWaitEvent(st, ev_in, 0));
    } else {
      // each chunk converted as soon as it has arrived, while the rest copy
      Tag tag_(this, "io");
      for (int q = 0; q < 3; ++q)
        for (int c = 0; c < nchunk; ++c) {
          int k0;
          long n;
          chunk(c, k0, n);
          LES_CUDA(cudaStreamWaitEvent(st, ev_inc[q * nchunk + c], 0));
          KL("k_convert", 12.0 * n, k_convert<T, double><<<grid_for(n), 256, 0, st>>>(
                                        lev(F[fid[q]], k0), stage_in[q] + k0 * g.plane(), n));
        }
    }
    step_body(jt, jtt, false);
    if constexpr (f64) {
      LES_CUDA(cudaEventRecord(ev_done, st));
      LES_CUDA(cudaStreamWaitEvent(sd2h, ev_done, 0));
    }
    for (int q = 0; q < 3; ++q)
      for (int c = 0; c < nchunk; ++c) {
        int k0;
        long n;
        chunk(c, k0, n);
        if constexpr (!f64) {  // the copy back of a chunk starts once that chunk is converted
          Tag tag_(this, "io");
          KL("k_convert", 12.0 * n, k_convert<double, T><<<grid_for(n), 256, 0, st>>>(
                                        stage_out[q] + k0 * g.plane(), lev(F[fid[q]], k0), n));
          LES_CUDA(cudaEventRecord(ev_cvt[q * nchunk + c], st));
          LES_CUDA(cudaStreamWaitEvent(sd2h, ev_cvt[q * nchunk + c], 0));
        }
        LES_CUDA(cudaMemcpyAsync(h[q] + k0 * g.plane(), dev_out(q) + k0 * g.plane(), n * sizeof(double),
                                 cudaMemcpyDeviceToHost, sd2h));
        LES_CUDA(cudaEventRecord(ev_out[q * nchunk + c], sd2h));
      }
    // the step's diagnostics, on st while the copies back run; they rewrite
    // dout, so they follow the previous call's copy of it (long done)
    if (out_recorded) LES_CUDA(cudaStreamWaitEvent(st, ev_copies, 0));
    diagnostics_launch();
    if (diag4) {
      LES_CUDA(cudaEventRecord(ev_done, st));
      LES_CUDA(cudaStreamWaitEvent(sd2h, ev_done, 0));
      LES_CUDA(cudaMemcpyAsync(diag4, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, sd2h));
    }
    out_recorded = true;
    LES_CUDA(cudaEventRecord(ev_copies, sd2h));
    copies_pending = true;
  }

  void set_initial_conditions(const double* u, const double* v, const double* w) override {
    upload(LES_U, u, 1, g.nz);
    upload(LES_V, v, 1, g.nz);
    upload(LES_W, w, 1, g.nz);
    // initial BCs with the namelist defaults: lbc 'drc' 0, ubc u,v 'neu' 0, w 'drc' 0
    const int4 lt = make_int4(1, 1, 1, 0), ut = make_int4(2, 2, 1, 0);
    for (int pl : {LES_LBC_U, LES_LBC_V, LES_LBC_W, LES_UBC_U, LES_UBC_V, LES_UBC_W}) fill_plane(PL[pl], T(0));
    launch_bc(lt, ut);
    fill(F[LES_W], 0, 0, T(BOGUS));
    if (P.wall_law) {  // LES_engine.f90:168-171
      lbc_t[0] = 2;
      lbc_t[1] = 2;
    }
    LES_CUDA(cudaStreamSynchronize(st));
  }

  void launch_bc(int4 lt, int4 ut) {
    KL("k_set_bc", 8.0 * g.plane() * sizeof(T), k_set_bc<T><<<grid_for(g.plane()), 256, 0, st>>>(F[LES_U], F[LES_V], F[LES_W], PL[LES_LBC_U], PL[LES_LBC_V],
                                                    PL[LES_LBC_W], PL[LES_UBC_U], PL[LES_UBC_V], PL[LES_UBC_W],
                                                    lt, ut, g.plane(), g.nz, T(P.lz / double(g.nz))));
  }
  void set_bc() override {
    Tag tag_(this, "bc");
    launch_bc(make_int4(lbc_t[0], lbc_t[1], lbc_t[2], 0), make_int4(ubc_t[0], ubc_t[1], ubc_t[2], 0));
  }

  double dz() const { return P.lz / double(g.nz); }
  bool mixed() const { return P.precision == LES_MIXED; }
  // Mixed precision: transform each field minus its value at (0,0) of the
  // level; refout[q] receives the value the inverse transform adds back.
  void use_refs(XFArgs<T>& a, int nf) {
    if (!mixed()) return;
    a.use_ref = 1;
    a.ref_mul = 1.0 / a.c0;
    for (int q = 0; q < nf; ++q) a.refout[q] = refbuf[q];
  }

  // ------------------------------------------------ compute_derivatives ----
  // grad_velocity_filt for up to three fields at once
  void grad_fields(const int* f, const int* dx, const int* dy, int nfld, const char* tag = "grad") {
    T *pf[3], *pdx[3], *pdy[3];
    for (int q = 0; q < nfld; ++q) {
      pf[q] = F[f[q]];
      pdx[q] = F[dx[q]];
      pdy[q] = F[dy[q]];
    }
    grad_ptrs(pf, pdx, pdy, nfld, tag);
  }
  void grad_ptrs(T* const* f, T* const* dx, T* const* dy, int nfld, const char* tag = "grad") {
    Tag tag_(this, tag);
    const int L = g.L;
    auto a = xf(XF_SCALE, nfld, 0, L, g.nx, g.ny, g.lhx);
    a.c0 = 1.0 / double(g.nx * g.ny);
    for (int q = 0; q < nfld; ++q) {
      a.in[q] = f[q];
      a.out[q] = spec[q];
    }
    use_refs(a, nfld);
    launch_xfwd<T>(g.nx, a, st);
    // y pass: F and i ky F; the x inverse forms i kx F from the staged F row
    auto b = yp(YP_GRADY, 1, 2, g.lhx, g.lhx, g.ny, g.lhx, g.ny, 0);
    for (int q = 0; q < nfld; ++q) {
      b.in[q] = spec[q];
      b.out[2 * q + 0] = spec[q];
      b.out[2 * q + 1] = spec[3 + q];
    }
    launch_ypass<T>(g.ny, g.ny, b, L, nfld, st);
    auto c = xi(XI_STORE, 3 * nfld, 0, L, g.nx, g.ny, g.lhx);
    c.nstage = 2 * nfld;
    c.kxr = kkx;  // row ky = 0 of the wavenumber table (Nyquist column zero)
    for (int q = 0; q < nfld; ++q) {
      c.in[2 * q + 0] = spec[q];
      c.in[2 * q + 1] = spec[3 + q];
      c.src[3 * q + 0] = 2 * q;
      c.src[3 * q + 1] = 2 * q;
      c.dx[3 * q + 1] = 1;
      c.src[3 * q + 2] = 2 * q + 1;
      c.out[3 * q + 0] = f[q];
      c.out[3 * q + 1] = dx[q];
      c.out[3 * q + 2] = dy[q];
    }
    for (int q = 0; q < 3 * nfld; ++q) {
      c.lo[q] = 0;
      c.hi[q] = g.nz + 1;
    }
    if (mixed())
      for (int q = 0; q < nfld; ++q) c.refin[3 * q] = refbuf[q];  // the filtered field itself
    launch_xinv<T>(g.nx, c, st);
  }
  void grad_velocity_filt(int f, int dfdx, int dfdy) override { grad_fields(&f, &dfdx, &dfdy, 1); }

  void ddz_uv(int dfdz, int f) override {
    KL("k_ddz", 2.0 * (g.nz + 1) * g.plane() * sizeof(T), k_ddz<T><<<grid_for((long)(g.nz + 1) * g.plane()), 256, 0, st>>>(F[dfdz], F[f], g.plane(), g.nz, T(1.0 / dz()), 0));
  }
  void ddz_w(int dfdz, int f) override {
    KL("k_ddz", 2.0 * (g.nz + 1) * g.plane() * sizeof(T), k_ddz<T><<<grid_for((long)(g.nz + 1) * g.plane()), 256, 0, st>>>(F[dfdz], F[f], g.plane(), g.nz, T(1.0 / dz()), 1));
  }

  void compute_vel_grad() override {
    const int f[3] = {LES_U, LES_V, LES_W};
    const int dx[3] = {LES_DUDX, LES_DVDX, LES_DWDX};
    const int dy[3] = {LES_DUDY, LES_DVDY, LES_DWDY};
    grad_fields(f, dx, dy, 3);
    set_bc();
    Tag tag_(this, "grad");
    KL("k_ddz_vel", 6.0 * (g.nz + 1) * g.plane() * sizeof(T), k_ddz_vel<T><<<grid_for((long)(g.nz + 1) * g.plane()), 256, 0, st>>>(
        F[LES_U], F[LES_V], F[LES_W], F[LES_DUDZ], F[LES_DVDZ], F[LES_DWDZ], g.plane(), g.nz, T(1.0 / dz())));
    if (scalar_on) scalar_grad();
  }

  // stress divergence of up to three equations (compute_derivatives.f90:464-577)
  struct DivEq {
    int rhs, tx, ty, tz, stag;
    double pf;
  };
  void div_eqs(const DivEq* e, int neq, bool layers, const char* tag = "divstress") {
    Tag tag_(this, tag);
    // forward transforms of the distinct tx, ty fields
    int ids[6];
    int nid = 0;
    auto slot = [&](int fid) {
      for (int q = 0; q < nid; ++q)
        if (ids[q] == fid) return q;
      ids[nid] = fid;
      return nid++;
    };
    int sx[3], sy[3];
    for (int q = 0; q < neq; ++q) {
      sx[q] = slot(e[q].tx);
      sy[q] = slot(e[q].ty);
    }
    auto a = xf(XF_SCALE, nid, 1, g.nz + 1, g.nx, g.ny, g.lhx);
    a.c0 = 1.0 / double(g.nx * g.ny);
    for (int q = 0; q < nid; ++q) {
      a.in[q] = F[ids[q]];
      a.out[q] = spec[q];
    }
    use_refs(a, nid);  // derivatives of the per-level constants vanish
    launch_xfwd<T>(g.nx, a, st);
    auto b = yp(YP_DIV2, 2, 1, g.lhx, g.lhx, g.ny, g.lhx, g.ny, 1);
    for (int q = 0; q < neq; ++q) {
      b.in[2 * q] = spec[sx[q]];
      b.in[2 * q + 1] = spec[sy[q]];
      b.out[q] = spec[6 + q];
    }
    launch_ypass<T>(g.ny, g.ny, b, g.nz + 1, neq, st);
    auto c = xi(XI_DIV, neq, 1, g.nz + 1, g.nx, g.ny, g.lhx);
    c.c0 = 1.0 / dz();
    for (int q = 0; q < neq; ++q) {
      c.in[q] = spec[6 + q];
      c.out[q] = F[e[q].rhs];
      c.aux[q] = F[e[q].tz];
      c.lo[q] = e[q].stag;
      c.pf[q] = e[q].pf;
    }
    c.out[8] = layers ? PL[LES_BOTTOM_WK_PRESS] : nullptr;
    c.out[9] = layers ? PL[LES_TOP_WK_PRESS] : nullptr;
    launch_xinv<T>(g.nx, c, st);
  }
  void div_stress(int rhs, int tx, int ty, int tz, int stag) override {
    DivEq e{rhs, tx, ty, tz, stag, 0.0};
    div_eqs(&e, 1, !stag);
    if (stag) {
      // optional layers are BOGUS for the staggered call (compute_derivatives.f90:560-574)
    }
  }

  // -------------------------------------------- compute_convective_padd ----
  void dealias_convec(int cx, int cy, int cz) override {
    Tag tag_(this, "convec");
    const int nz = g.nz;
    const bool padd = (P.dealias == LES_DEALIAS_PADD);
    const int nkin = padd ? g.nx / 2 : int(std::ceil(double(float(g.nx)) / 3.0)) - 1;
    const int FNX = padd ? g.nx2 : g.nx;
    const int FNY = padd ? g.ny2 : g.ny;
    // 1. transforms of -c u, -c v, -c w and the vorticity (levels 1..nz+1)
    auto a = xf(XF_CONV_IN, 6, 1, nz + 1, g.nx, g.ny, nkin);
    a.c0 = 1.0 / double(g.nx * g.ny);
    const int ins[9] = {LES_U, LES_V, LES_W, LES_DWDY, LES_DVDZ, LES_DUDZ, LES_DWDX, LES_DVDX, LES_DUDY};
    for (int q = 0; q < 9; ++q) a.in[q] = F[ins[q]];
    for (int q = 0; q < 6; ++q) a.out[q] = spec[q];
    use_refs(a, 6);
    launch_xfwd<T>(g.nx, a, st);
    // 2. y: pad to 3ny/2 (or 2/3-rule mask)
    if (padd) {
      auto b = yp(YP_PAD, 1, 1, nkin, nkin, g.ny, nkin, g.ny2, 1);
      for (int q = 0; q < 6; ++q) {
        b.in[q] = spec[q];
        b.out[q] = spec[6 + q];
      }
      launch_ypass<T>(g.ny, g.ny2, b, nz + 1, 6, st);
    } else {
      auto b = yp(YP_MASK, 1, 1, nkin, nkin, g.ny, nkin, g.ny, 1);
      b.tt = int(std::ceil(double(float(g.ny)) / 3.0)) - 2;
      for (int q = 0; q < 6; ++q) {
        b.in[q] = spec[q];
        b.out[q] = spec[6 + q];
      }
      launch_ypass<T>(g.ny, g.ny, b, nz + 1, 6, st);
    }
    // 3. x: c2r on the fine (or base) grid
    auto c = xi(XI_STORE, 6, 1, nz + 1, FNX, FNY, nkin);
    for (int q = 0; q < 6; ++q) {
      c.in[q] = spec[6 + q];
      c.out[q] = fine[q];
      c.lo[q] = 0;
      c.hi[q] = nz + 1;
      if (mixed()) c.refin[q] = refbuf[q];
    }
    launch_xinv<T>(FNX, c, st);
    // 4. products on the fine grid, transformed back (levels 1..nz)
    const int nkout = padd ? g.nx / 2 : int(std::ceil(double(float(2 * g.lhx)) / 3.0)) - 1;
    auto d = xf(XF_PROD, 3, 1, nz, FNX, FNY, nkout);
    d.c0 = padd ? 1.0 / double(g.nx2 * g.ny2) : 1.0 / double(g.nx * g.ny);
    for (int q = 0; q < 6; ++q) d.in[q] = fine[q];
    for (int q = 0; q < 3; ++q) d.out[q] = spec[q];
    if (mixed()) {
      d.use_ref = 1;
      d.ref_mul = 1.0 / d.c0;
      for (int q = 0; q < 3; ++q) d.refout[q] = refbuf[6 + q];
    }
    launch_xfwd<T>(FNX, d, st);
    if (padd) {
      auto e = yp(YP_TRUNC, 1, 1, nkout, nkout, g.ny2, nkout, g.ny, 1);
      for (int q = 0; q < 3; ++q) {
        e.in[q] = spec[q];
        e.out[q] = spec[3 + q];
      }
      launch_ypass<T>(g.ny2, g.ny, e, nz, 3, st);
    } else {
      auto e = yp(YP_MASK, 1, 1, nkout, nkout, g.ny, nkout, g.ny, 1);
      e.tt = int(std::ceil(double(float(2 * g.lhy)) / 3.0)) - 2;
      for (int q = 0; q < 3; ++q) {
        e.in[q] = spec[q];
        e.out[q] = spec[3 + q];
      }
      launch_ypass<T>(g.ny, g.ny, e, nz, 3, st);
    }
    auto h = xi(XI_STORE, 3, 1, nz, g.nx, g.ny, nkout);
    const int outs[3] = {cx, cy, cz};
    for (int q = 0; q < 3; ++q) {
      h.in[q] = spec[3 + q];
      h.out[q] = F[outs[q]];
      h.lo[q] = 1;
      h.hi[q] = nz;
      if (mixed()) h.refin[q] = refbuf[6 + q];
    }
    launch_xinv<T>(g.nx, h, st);
    // ghost levels of the outputs (compute_convective_padd.f90:251-259)
    if (padd) {
      T* dst[6];
      T val[6];
      for (int q = 0; q < 3; ++q) {
        dst[2 * q] = lev(F[outs[q]], 0);
        dst[2 * q + 1] = lev(F[outs[q]], nz + 1);
        val[2 * q] = val[2 * q + 1] = T(BOGUS);
      }
      plane_ops(6, dst, nullptr, val);
    } else {
      trunc_ghosts(outs);
    }
  }

  // compute_convective_trunc leaves its vorticity scratch in the ghost levels
  void trunc_ghosts(const int* outs) {
    // level 0: wall rows zeroed for cx, cy; level nz+1 and cz level 0 hold
    // c*(vorticity) of that level
    scratch_vort_level(outs, 0);
    scratch_vort_level(outs, g.nz + 1);
  }
  void scratch_vort_level(const int* outs, int k);

  // ---------------------------------------------------- compute_pressure ----
  // The pressure path transforms in S = FP64 in both precisions: its RHS
  // (div u*) is a small difference of large terms.
  template <typename S>
  XFArgs<S> xf_s(int op, int nf, int plane0, int nplanes, int nk) {
    XFArgs<S> a;
    std::memset(&a, 0, sizeof(a));
    a.op = op;
    a.nf = nf;
    a.plane0 = plane0;
    a.rows_pp = g.ny;
    a.nrows = (long)nplanes * g.ny;
    a.nk = nk;
    a.nz = g.nz;
    a.in_pstride = (long)g.ny * g.nx;
    a.out_pstride = (long)g.ny * nk;
    a.tw = twiddles64(g.nx);
    return a;
  }
  template <typename S>
  YPArgs<S> yp_s(int op, int nin, int nout, int plane0) {
    YPArgs<S> a;
    std::memset(&a, 0, sizeof(a));
    a.op = op;
    a.nin = nin;
    a.nout = nout;
    a.ncols = g.lhx;
    a.nk_in = g.lhx;
    a.nk_out = g.lhx;
    a.in_pstride = (long)g.ny * g.lhx;
    a.out_pstride = (long)g.ny * g.lhx;
    a.plane0 = plane0;
    a.nxh = g.nx / 2;
    a.lhx = g.lhx;
    a.kkx = kkx64;
    a.kky = kky64;
    a.tw_in = twiddles64(g.ny);
    a.tw_out = twiddles64(g.ny);
    return a;
  }
  template <typename S>
  XIArgs<S> xi_s(int op, int nin, int plane0, int nplanes) {
    XIArgs<S> a;
    std::memset(&a, 0, sizeof(a));
    a.op = op;
    a.nin = nin;
    a.plane0 = plane0;
    a.rows_pp = g.ny;
    a.nrows = (long)nplanes * g.ny;
    a.nk = g.lhx;
    a.nz = g.nz;
    a.in_pstride = (long)g.ny * g.lhx;
    a.out_pstride = (long)g.ny * g.nx;
    a.tw = twiddles64(g.nx);
    a.status = dstatus;
    return a;
  }
  template <typename S>
  static void set_in(XFArgs<S>& a, int q, T* f) {
    if constexpr (std::is_same<T, float>::value && std::is_same<S, double>::value) {
      a.inf[q] = f;
      a.in_f32 = 1;
    } else {
      a.in[q] = reinterpret_cast<const S*>(f);
    }
  }
  template <typename S>
  static void set_out(XIArgs<S>& a, int q, T* f) {
    if constexpr (std::is_same<T, float>::value && std::is_same<S, double>::value) {
      a.outf[q] = f;
      a.out_f32 = 1;
    } else {
      a.out[q] = reinterpret_cast<S*>(f);
    }
  }

  void press_stag_array(double tadv1) override {
    Tag tag_(this, "press");
    press_tadv1_ = tadv1;
    if (mixed()) press_impl<double>(pspec);
    else press_impl<double>(reinterpret_cast<cplx<double>**>(spec));
  }

  template <typename S>
  void press_impl(cplx<S>** sp) {
    const double tadv1 = press_tadv1_;
    const int nz = g.nz;
    const double c = 1.0 / double(g.nx * g.ny);
    // bottom/top layers (compute_pressure.f90:151-165, 196-203)
    KL("k_scale", 2.0 * g.plane() * sizeof(T), k_scale<T><<<grid_for(g.plane()), 256, 0, st>>>(PL[LES_BOTTOM_WK_PRESS], g.plane(), T(c)));
    cplx<S>* bot = sp[0];  // plane 0 of sp[0] / sp[1]
    cplx<S>* top = sp[1];
    {
      auto a = xf_s<S>(XF_SCALE, 1, 0, 1, g.lhx);
      a.c0 = 1.0;
      set_in(a, 0, PL[LES_BOTTOM_WK_PRESS]);
      a.out[0] = bot;
      launch_xfwd<S>(g.nx, a, st);
      a.c0 = c;
      set_in(a, 0, PL[LES_TOP_WK_PRESS]);
      a.out[0] = top;
      launch_xfwd<S>(g.nx, a, st);
      auto b = yp_s<S>(YP_FWDKILL, 1, 1, 0);
      b.in[0] = bot;
      b.out[0] = bot;
      b.in[1] = top;
      b.out[1] = top;
      launch_ypass<S>(g.ny, g.ny, b, 1, 2, st);
    }
    // H = FFT(u / (dt tadv1 nx ny)), Nyquist killed (levels 1..nz)
    auto a = xf_s<S>(XF_PRESS, 3, 1, nz, g.lhx);
    a.c0 = c / tadv1;
    a.c1 = P.dt;
    const int uvw[3] = {LES_U, LES_V, LES_W};
    for (int q = 0; q < 3; ++q) {
      set_in(a, q, F[uvw[q]]);
      a.out[q] = sp[2 + q];
    }
    launch_xfwd<S>(g.nx, a, st);
    auto b = yp_s<S>(YP_FWDKILL, 1, 1, 1);
    for (int q = 0; q < 3; ++q) {
      b.in[q] = sp[2 + q];
      b.out[q] = sp[2 + q];
    }
    launch_ypass<S>(g.ny, g.ny, b, nz, 3, st);
    // tridiagonal solve per (kx, ky) -> p^ in sp[5], levels 0..nz+1; in
    // mixed precision the mean mode is kept apart in FP64 (pmean)
    dim3 tg(ceil_div(g.lhx, 64), g.ny);
    if constexpr (std::is_same<T, float>::value) {
      // mixed precision: p^ leaves the FP64 solve as FP32 (its mean mode is
      // kept apart in FP64); the inverse transforms of p run in FP32 -- only
      // the forward right-hand side needs FP64, where div u* cancels
      if (pslabs > 1)
        slab_solve<S, T>(sp[2], sp[3], sp[4], bot, top, spec[0], pmean, 1, pitch(g.lhx), g.lhx);
      else
        KL("k_tridiag", 96.0 * double(g.L) * g.ny * g.lhx,
           k_tridiag<S, T><<<tg, 64, 0, st>>>(sp[2], sp[3], sp[4], nullptr, bot, top, kkxd, kkyd, spec[0], xs, gam, pmean, dstatus,
                                              g.lhx, g.ny, nz, dz(), 1, pitch(g.lhx), g.lhx));
      auto e = yp(YP_PGRAD, 1, 3, g.lhx, g.lhx, g.ny, g.lhx, g.ny, 0);
      e.in[0] = spec[0];
      e.out[0] = spec[1];
      e.out[1] = spec[2];
      e.out[2] = spec[0];
      launch_ypass<T>(g.ny, g.ny, e, g.L, 1, st);
      auto h = xi(XI_STORE, 3, 0, g.L, g.nx, g.ny, g.lhx);
      h.in[0] = spec[1];
      h.in[1] = spec[2];
      h.in[2] = spec[0];
      h.out[0] = F[LES_DPDX];
      h.out[1] = F[LES_DPDY];
      h.out[2] = F[LES_P];
      h.lo[0] = 1;
      h.hi[0] = nz;
      h.lo[1] = 1;
      h.hi[1] = nz;
      h.lo[2] = 0;
      h.hi[2] = nz + 1;
      launch_xinv<T>(g.nx, h, st);
      dpdz_only();
      KL("k_p_finish", 2.0 * g.field() * sizeof(T),
         k_p_finish<T><<<grid_for(g.field() / 4), 256, 0, st>>>(F[LES_P], pmean, g.plane(), nz));
      return;
    }
    if (pslabs > 1)
      slab_solve<S, S>(sp[2], sp[3], sp[4], bot, top, sp[5], mixed() ? pmean : nullptr, mixed() ? 1 : 0, g.lhx, g.lhx);
    else
      KL("k_tridiag", 112.0 * double(g.L) * g.ny * g.lhx, k_tridiag<S><<<tg, 64, 0, st>>>(sp[2], sp[3], sp[4], nullptr, bot, top, kkxd, kkyd, sp[5], xs, gam,
                                     mixed() ? pmean : nullptr, dstatus, g.lhx, g.ny, nz, dz(), mixed() ? 1 : 0, g.lhx, g.lhx));
    // compute_press_grad: i kx p^, i ky p^, p^ -> dpdx, dpdy (1..nz), p (0..nz+1)
    auto e = yp_s<S>(YP_PGRAD, 1, 3, 0);
    e.in[0] = sp[5];
    e.out[0] = sp[6];
    e.out[1] = sp[7];
    e.out[2] = sp[5];
    launch_ypass<S>(g.ny, g.ny, e, g.L, 1, st);
    auto h = xi_s<S>(XI_STORE, 3, 0, g.L);
    h.in[0] = sp[6];
    h.in[1] = sp[7];
    h.in[2] = sp[5];
    set_out(h, 0, F[LES_DPDX]);
    set_out(h, 1, F[LES_DPDY]);
    set_out(h, 2, F[LES_P]);
    h.lo[0] = 1;
    h.hi[0] = nz;
    h.lo[1] = 1;
    h.hi[1] = nz;
    h.lo[2] = 0;
    h.hi[2] = nz + 1;
    launch_xinv<S>(g.nx, h, st);
    // dpdz (compute_pressure.f90:359-369), then p(nz+1) = BOGUS (:353-357)
    dpdz_only();
    KL("k_p_finish", (mixed() ? 2.0 * g.field() : double(g.plane())) * sizeof(T), k_p_finish<T><<<grid_for(g.field() / 4), 256, 0, st>>>(F[LES_P], mixed() ? pmean : nullptr, g.plane(), nz));
  }
  double press_tadv1_ = 1.0;
  void dpdz_only();
  // z-slab emulation of the pressure solve: the systems solved by the
  // partition method over pslabs row blocks, as pslabs z-slab ranks would
  // (k_tri_slab_*); 1 = the single sweep of k_tridiag
  int pslabs = 1;
  double *slab_u = nullptr, *slab_v = nullptr;
  cplx<double>* slab_x = nullptr;
  int slab_x_cap = 1;
  void set_pressure_slabs(int G) override {
    if (G < 1 || G > MAX_SLABS || g.nz % G != 0 || g.nz / G < 2)
      throw CudaError(1, "pressure slabs: 1 <= G <= 64, nz a multiple of G with at least two levels per slab");
    pslabs = G;
    if (G > 1 && !slab_u) {
      const long n = (long)g.L * g.ny * g.lhx;
      slab_u = track(dalloc<double>(n));
      slab_v = track(dalloc<double>(n));
    }
    if (G > slab_x_cap) {
      slab_x = track(dalloc<cplx<double>>((long)g.ny * g.lhx * G * 2));
      slab_x_cap = G;
    }
  }
  template <typename S, typename O>
  void slab_solve(const cplx<S>* Hx, const cplx<S>* Hy, const cplx<S>* Hz, const cplx<S>* bot, const cplx<S>* top,
                  cplx<O>* phat, double* pm, int drop_mean, int opitch, int ipitch) {
    const SlabRows sr{pslabs, g.nz / pslabs, g.nz};
    const double cols = double(g.ny) * g.lhx;
    KL("k_tri_slab_local", cols * g.L * (3.0 * 2 * sizeof(S) + 40.0),
       k_tri_slab_local<S><<<dim3(ceil_div(g.lhx, 64), g.ny, pslabs), 64, 0, st>>>(
           Hx, Hy, Hz, bot, top, kkxd, kkyd, xs, slab_u, slab_v, gam, dstatus, g.lhx, g.ny, g.nz, dz(), ipitch, sr));
    KL("k_tri_slab_reduced", cols * pslabs * (2 * 32.0 + 32.0),
       k_tri_slab_reduced<<<dim3(ceil_div(g.lhx, 64), g.ny), 64, 0, st>>>(xs, slab_u, slab_v, slab_x, dstatus, g.lhx,
                                                                          g.ny, sr));
    KL("k_tri_slab_back", cols * g.L * (32.0 + 2 * sizeof(O)),
       k_tri_slab_back<O><<<dim3(ceil_div(g.lhx, 64), g.ny, g.L), 64, 0, st>>>(xs, slab_u, slab_v, slab_x, phat, pm,
                                                                               g.lhx, g.ny, g.nz, drop_mean, opitch, sr));
  }


  // press_stag_array on the state an AB2 advance left, with the right-hand
  // side formed from the increment: u* / (dt t1) = u^n / (dt t1) + r +
  // (t2/t1) r_f, and the spectral divergence of u^n is FFT(dudx + dvdy +
  // dwdz) of this step's gradients (the same Nyquist-killed derivatives the
  // reference's transform of u* forms), so rhs(k) = i kx H^x + i ky H^y +
  // (H^z(k+1) - H^z(k))/dz + FFT(div u^n)/(dt t1) with H the increments.
  // The pressure is the same in exact arithmetic; in FP32 no large value
  // cancels (u* ~ 20 against an increment of dt rhs ~ 1e-3), so the
  // transforms run in the state's precision.  Needs w(nz+1) = 0.
  void press_from_increment(double tadv1, double tadv2) override {
    Tag tag_(this, "press");
    const int nz = g.nz;
    const double c = 1.0 / double(g.nx * g.ny);
    KL("k_scale", 2.0 * g.plane() * sizeof(T), k_scale<T><<<grid_for(g.plane()), 256, 0, st>>>(PL[LES_BOTTOM_WK_PRESS], g.plane(), T(c)));
    cplx<T>* bot = spec[8];
    cplx<T>* top = spec[9];
    {
      auto a = xf(XF_SCALE, 1, 0, 1, g.nx, g.ny, g.lhx);
      a.c0 = 1.0;
      a.in[0] = PL[LES_BOTTOM_WK_PRESS];
      a.out[0] = bot;
      launch_xfwd<T>(g.nx, a, st);
      a.c0 = c;
      a.in[0] = PL[LES_TOP_WK_PRESS];
      a.out[0] = top;
      launch_xfwd<T>(g.nx, a, st);
      auto b = yp(YP_FWDKILL, 1, 1, g.lhx, g.lhx, g.ny, g.lhx, g.ny, 0);
      b.in[0] = bot;
      b.out[0] = bot;
      b.in[1] = top;
      b.out[1] = top;
      launch_ypass<T>(g.ny, g.ny, b, 1, 2, st);
    }
    auto a = xf(XF_PRESS_INC, 4, 1, nz, g.nx, g.ny, g.lhx);
    a.c0 = c;
    a.c1 = tadv2 / tadv1;
    a.c2 = 1.0 / (P.dt * tadv1);
    const int ins[9] = {LES_RHSX, LES_RHSY, LES_RHSZ, LES_RHSX_F, LES_RHSY_F, LES_RHSZ_F, LES_DUDX, LES_DVDY, LES_DWDZ};
    for (int q = 0; q < 9; ++q) a.in[q] = F[ins[q]];
    for (int q = 0; q < 4; ++q) a.out[q] = spec[2 + q];
    launch_xfwd<T>(g.nx, a, st);
    auto b = yp(YP_FWDKILL, 1, 1, g.lhx, g.lhx, g.ny, g.lhx, g.ny, 1);
    for (int q = 0; q < 4; ++q) {
      b.in[q] = spec[2 + q];
      b.out[q] = spec[2 + q];
    }
    launch_ypass<T>(g.ny, g.ny, b, nz, 4, st);
    // the mean mode's right-hand side from FP64 plane means: the plane mean of
    // rhs_z carries the mean vertical pressure gradient (thousands at the
    // wall), which an FP32 transform would round
    if (!means) means = track(dalloc<double>(6 * g.L));
    KL("k_plane_means", 5.0 * nz * g.plane() * sizeof(T),
       k_plane_means<T><<<nz, 256, 0, st>>>(F[LES_RHSZ], F[LES_RHSZ_F], F[LES_DUDX], F[LES_DVDY], 5, means, g.plane(), 1,
                                            g.L, F[LES_DWDZ]));
    dim3 tg(ceil_div(g.lhx, 64), g.ny);
    KL("k_tridiag", (4.0 * 2 * sizeof(T) + 2 * sizeof(T) + 24.0) * double(g.L) * g.ny * g.lhx,
       k_tridiag<T, T, true><<<tg, 64, 0, st>>>(spec[2], spec[3], spec[4], spec[5], bot, top, kkxd, kkyd, spec[0], xs, gam,
                                          mixed() ? pmean : nullptr, dstatus, g.lhx, g.ny, nz, dz(), mixed() ? 1 : 0,
                                          pitch(g.lhx), pitch(g.lhx), means, tadv2 / tadv1, 1.0 / (P.dt * tadv1),
                                          g.L));
    auto e = yp(YP_PGRAD, 1, 3, g.lhx, g.lhx, g.ny, g.lhx, g.ny, 0);
    e.in[0] = spec[0];
    e.out[0] = spec[1];
    e.out[1] = spec[2];
    e.out[2] = spec[0];
    launch_ypass<T>(g.ny, g.ny, e, g.L, 1, st);
    auto h = xi(XI_STORE, 3, 0, g.L, g.nx, g.ny, g.lhx);
    h.in[0] = spec[1];
    h.in[1] = spec[2];
    h.in[2] = spec[0];
    h.out[0] = F[LES_DPDX];
    h.out[1] = F[LES_DPDY];
    h.out[2] = F[LES_P];
    h.lo[0] = 1;
    h.hi[0] = nz;
    h.lo[1] = 1;
    h.hi[1] = nz;
    h.lo[2] = 0;
    h.hi[2] = nz + 1;
    launch_xinv<T>(g.nx, h, st);
    dpdz_only();
    KL("k_p_finish", (mixed() ? 2.0 * g.field() : double(g.plane())) * sizeof(T),
       k_p_finish<T><<<grid_for(g.field() / 4), 256, 0, st>>>(F[LES_P], mixed() ? pmean : nullptr, g.plane(), nz));
  }


  // ---------------------------------------------------- compute_wall_law ----
  void wall_layer() {
    Tag tag_(this, "wall");
    if (P.wall_model == LES_WALL_FILTER) {
      // get_layer_filter (utility_tools.f90:261-307) + test_filter_layer
      cplx<T>* s0 = spec[0];
      cplx<T>* s1 = spec[1];
      auto a = xf(XF_SCALE, 2, 0, 1, g.nx, g.ny, nk2);
      a.c0 = 1.0;
      a.in[0] = lev(F[LES_U], 1);
      a.in[1] = lev(F[LES_V], 1);
      a.out[0] = s0;
      a.out[1] = s1;
      use_refs(a, 2);
      launch_xfwd<T>(g.nx, a, st);
      auto b = yp(YP_FILTER1, 1, 1, nk2, nk2, g.ny, nk2, g.ny, 0);
      b.G0 = gt;
      b.in[0] = s0;
      b.out[0] = s0;
      b.in[1] = s1;
      b.out[1] = s1;
      launch_ypass<T>(g.ny, g.ny, b, 1, 2, st);
      auto c = xi(XI_WALL, 2, 0, 1, g.nx, g.ny, nk2);
      c.in[0] = s0;
      c.in[1] = s1;
      if (mixed()) {
        c.refin[0] = refbuf[0];
        c.refin[1] = refbuf[1];
      }
      c.c0 = dz();
      c.out_pstride = g.plane();
      c.aux[0] = PL[LES_LBC_Z0];
      c.out[0] = PL[LES_U_STAR_AVG];
      c.out[1] = PL[LES_LBC_U];
      c.out[2] = PL[LES_LBC_V];
      c.out[3] = F[LES_TXZ];
      c.out[4] = F[LES_TYZ];
      c.out[5] = F[LES_DUDZ];
      c.out[6] = F[LES_DVDZ];
      launch_xinv<T>(g.nx, c, st);
    } else {
      wall_plain();
    }
  }
  void wall_plain();
  void obukhov() override { wall_layer(); }
  void wallstress() override { wall_layer(); }

  // -------------------------------------------------------- compute_sgs ----
  SgsArgs<T> sgs_args() {
    SgsArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    const int d[9] = {LES_DUDX, LES_DUDY, LES_DUDZ, LES_DVDX, LES_DVDY, LES_DVDZ, LES_DWDX, LES_DWDY, LES_DWDZ};
    for (int q = 0; q < 9; ++q) a.d[q] = F[d[q]];
    a.cs = F[LES_CS_OPT2];
    a.l2 = l2;
    a.nu = F[LES_NU_T];
    a.txx = F[LES_TXX];
    a.txy = F[LES_TXY];
    a.txz = F[LES_TXZ];
    a.tyy = F[LES_TYY];
    a.tyz = F[LES_TYZ];
    a.tzz = F[LES_TZZ];
    for (int q = 0; q < 6; ++q) a.sij[q] = sc[1 + q];
    a.smag = sc[0];
    a.wall = P.wall_law;
    a.plane = g.plane();
    a.nz = g.nz;
    return a;
  }

  void sgs_stress(int jt, int jtt) override {
    Tag tag_(this, "sgs");
    const long n1 = (long)(g.nz + 1) * g.plane();
    auto a = sgs_args();
    if (P.sgs_model == LES_SGS_CST_SMAG) {
      fill(F[LES_CS_OPT2], 1, g.nz + 1, T(P.cs0 * P.cs0));
    } else if (P.sgs_model == LES_SGS_LASD) {
      lasd(a, jtt);
    } else if (P.sgs_model == LES_SGS_DYN_SMAG) {
      dynsmag(a, jt, jtt);
    } else if (P.sgs_model == LES_SGS_MLP) {
      mlp_sgs(a, jtt);
    } else {
      throw CudaError(1, "Invalid SGS model");
    }
    double sbytes = 17.0;
    if (scalar_on) {
      if (SP.sgs == LES_SCALAR_SGS_DYN && jtt >= P.dyn_init && jt % P.cs_count == 0) scalar_dynamic(a);
      a.dt[0] = F[LES_DTDX];
      a.dt[1] = F[LES_DTDY];
      a.dt[2] = F[LES_DTDZ];
      a.q[0] = F[LES_QX];
      a.q[1] = F[LES_QY];
      a.q[2] = F[LES_QZ];
      a.kapd = SP.sgs == LES_SCALAR_SGS_DYN ? kapd : nullptr;
      a.inv_prt = SP.sgs == LES_SCALAR_SGS_DYN ? 0.0 : 1.0 / SP.pr_t;
      a.qs = SP.surface_flux;
      sbytes += 6.0;
    }
    if (g.plane() % 4 == 0)
      KL("k_sgs_tau", sbytes * (g.nz + 1) * g.plane() * sizeof(T),
         k_sgs_tau4<T><<<dim3(unsigned((g.plane() / 4 + 255) / 256), unsigned(g.nz + 1)), 256, 0, st>>>(a));
    else
      KL("k_sgs_tau", 17.0 * (g.nz + 1) * g.plane() * sizeof(T),
         k_sgs_tau<T><<<dim3(unsigned((g.plane() + 255) / 256), unsigned(g.nz + 1)), 256, 0, st>>>(a));
  }

  // dynamic-procedure contractions at both test scales (compute_dynamic_mum x2)
  // nlev: levels 1..nlev (all: nz + 1)
  void dynamic_mum(SgsArgs<T>& a, bool both, int nlev = -1) {
    if (nlev < 0) nlev = g.nz + 1;
    const long n1 = (long)nlev * g.plane();
    SgsArgs<T> ab = a;
    ab.nz = nlev - 1;  // k_sij covers levels 1..nz+1 of its arguments
    KL("k_sij", 16.0 * n1 * sizeof(T), k_sij<T><<<grid_for(n1), 256, 0, st>>>(ab));
    auto x = xf(XF_LASD, 21, 1, nlev, g.nx, g.ny, nk2);
    x.in[0] = F[LES_U];
    x.in[1] = F[LES_V];
    x.in[2] = F[LES_W];
    for (int q = 0; q < 6; ++q) x.in[3 + q] = sc[1 + q];
    x.in[9] = sc[0];
    for (int q = 0; q < 21; ++q) x.out[q] = spec[q];
    x.fluct = mixed() ? 1 : 0;
    launch_xfwd<T>(g.nx, x, st);
    auto y = yp(both ? YP_FILTER2 : YP_FILTER1, 1, both ? 2 : 1, nk2, nk2, g.ny, nk2, g.ny, 1);
    y.G0 = gt;
    y.G1 = gtt;
    y.ncols1 = nk4;
    y.nk_out1 = nk4;
    y.opitch1 = pitch(nk4);
    y.out_pstride1 = (long)g.ny * y.opitch1;
    for (int q = 0; q < 21; ++q) {
      y.in[q] = spec[q];
      y.out[(both ? 2 : 1) * q] = spec[q];
      if (both) y.out[2 * q + 1] = spec4[q];
    }
    launch_ypass<T>(g.ny, g.ny, y, nlev, 21, st);
    const double cst = 2.0 * delta * delta;
    for (int sc_i = 0; sc_i < (both ? 2 : 1); ++sc_i) {
      const int nk = sc_i == 0 ? nk2 : nk4;
      auto z = xi(XI_LASD, 21, 1, nlev, g.nx, g.ny, nk);
      z.c0 = cst;
      z.c1 = sc_i == 0 ? 4.0 : 16.0;
      for (int q = 0; q < 21; ++q) z.in[q] = sc_i == 0 ? spec[q] : spec4[q];
      z.out[0] = sc[7 + 2 * sc_i];
      z.out[1] = sc[8 + 2 * sc_i];
      launch_xinv<T>(g.nx, z, st);
    }
  }

  // compute_LagScaleDep_coeff on levels 1..nlev (all: nz + 1); the learned
  // closure runs it on a band of levels next to the wall
  void lasd(SgsArgs<T>& a, int jtt, int nlev = -1) {
    Tag tag_(this, "lasd");
    const int nz = g.nz;
    if (nlev < 0) nlev = nz + 1;
    const long nacc = std::min<long>(g.field(), (long)(nlev + 1) * g.plane());  // levels 0..nlev
    if (jtt >= P.dyn_init) {
      KL("k_lag_accum", 9.0 * nacc * sizeof(T), k_lag_accum<T><<<grid_for(nacc), 256, 0, st>>>(F[LES_U_LAG], F[LES_V_LAG], F[LES_W_LAG], F[LES_U],
                                                         F[LES_V], F[LES_W], nacc));
    }
    if (jtt < P.dyn_init) {
      fill(F[LES_CS_OPT2], 1, nz + 1, T(0.03));
      return;
    }
    if (jtt % P.cs_count != 0) return;
    dynamic_mum(a, true, nlev);
    const long n1 = (long)nlev * g.plane();
    if (f_coeff_init) {
      LagGeom geo{g.nx, g.ny, nz, g.plane(), P.lag_halo, P.dt, P.lx / double(g.nx), P.ly / double(g.ny), dz(),
                  double(P.cs_count), nlev};
      KL("k_lag_interp", 11.0 * n1 * sizeof(T), k_lag_interp<T><<<dim3(unsigned((g.plane() + 255) / 256), unsigned(nlev)), 256, 0, st>>>(F[LES_U_LAG], F[LES_V_LAG], F[LES_W_LAG], F[LES_F_LM],
                                                   F[LES_F_MM], F[LES_F_QN], F[LES_F_NN], sc[11], sc[12], sc[13],
                                                   sc[14], geo));
      if (nlev == nz + 1) {
        std::swap(F[LES_F_LM], sc[11]);
        std::swap(F[LES_F_MM], sc[12]);
        std::swap(F[LES_F_QN], sc[13]);
        std::swap(F[LES_F_NN], sc[14]);
      } else {  // a band: the levels above keep their averages
        const int fl[4] = {LES_F_LM, LES_F_MM, LES_F_QN, LES_F_NN};
        for (int t = 0; t < 4; ++t) copy(lev(F[fl[t]], 1), lev(sc[11 + t], 1), n1);
      }
    }
    KL("k_lasd_update", 14.0 * n1 * sizeof(T), k_lasd_update<T><<<grid_for(n1), 256, 0, st>>>(F[LES_F_LM], F[LES_F_MM], F[LES_F_QN], F[LES_F_NN], sc[7],
                                                  sc[8], sc[9], sc[10], F[LES_CS_OPT2], F[LES_BETA],
                                                  f_coeff_init ? 0 : 1, g.plane(), nz, 1.5 * delta,
                                                  P.dt * double(P.cs_count), beta_pow, nullptr, nlev, cs2_max));
    f_coeff_init = true;
    lagran_init = true;
    for (int q : {LES_U_LAG, LES_V_LAG, LES_W_LAG}) fill(F[q], 0, std::min(nlev, nz + 1), T(0));
  }

  void dynsmag(SgsArgs<T>& a, int jt, int jtt);

  void test_filter(int f, int which) override {
    Tag tag_(this, "testfilter");
    const int nk = which == 4 ? nk4 : nk2;
    auto a = xf(XF_SCALE, 1, 1, g.nz + 1, g.nx, g.ny, nk);
    a.c0 = 1.0;
    a.in[0] = F[f];
    a.out[0] = spec[0];
    use_refs(a, 1);
    launch_xfwd<T>(g.nx, a, st);
    auto b = yp(YP_FILTER1, 1, 1, nk, nk, g.ny, nk, g.ny, 1);
    b.G0 = which == 4 ? gtt : gt;
    b.in[0] = spec[0];
    b.out[0] = spec[0];
    launch_ypass<T>(g.ny, g.ny, b, g.nz + 1, 1, st);
    auto c = xi(XI_STORE, 1, 1, g.nz + 1, g.nx, g.ny, nk);
    c.in[0] = spec[0];
    c.out[0] = F[f];
    c.lo[0] = 1;
    c.hi[0] = g.nz + 1;
    if (mixed()) c.refin[0] = refbuf[0];
    launch_xinv<T>(g.nx, c, st);
  }

  // ------------------------------------------- scalar transport (theta) ----
  double* kapd = nullptr;    // Cs^2/Pr_t * Delta^2 per level (dynamic model)
  double* means = nullptr;   // plane means: 6 x L (forcing: u, v, w, theta; pressure: five rhs fields)
  double* spong = nullptr;   // sponge profile on w nodes (L)
  void scalar_init(const les_scalar_params& sp) override {
    if (!(sp.pr_t > 0.0)) throw CudaError(1, "Invalid scalar parameters: pr_t must be positive");
    if (sp.sgs != LES_SCALAR_SGS_CONST && sp.sgs != LES_SCALAR_SGS_DYN)
      throw CudaError(1, "Invalid scalar SGS model");
    if (g.plane() % 4 != 0) throw CudaError(1, "scalar transport needs nx * ny divisible by 4");
    SP = sp;
    const long nf = g.field();
    for (int i = LES_THETA; i < LES_NFIELDS; ++i) {
      if (!F[i]) F[i] = track(dalloc<T>(nf));
      fill(F[i], 0, g.nz + 1, T(0));
    }
    if (!kapd) kapd = track(dalloc<double>(g.L));
    if (!means) means = track(dalloc<double>(6 * g.L));
    // kappa before the first dynamic update: 0.03 / Pr_t (the LASD start value over Pr_t)
    const double d2 = delta * delta;
    std::vector<double> k0(g.L, sp.sgs == LES_SCALAR_SGS_DYN ? 0.03 / sp.pr_t * d2 : 0.0);
    LES_CUDA(cudaMemcpyAsync(kapd, k0.data(), sizeof(double) * g.L, cudaMemcpyHostToDevice, st));
    scalar_on = true;
    scalar_bc();
    LES_CUDA(cudaStreamSynchronize(st));
  }
  void scalar_bc() {
    KL("k_scalar_bc", 3.0 * g.plane() * sizeof(T),
       k_scalar_bc<T><<<grid_for(g.plane()), 256, 0, st>>>(F[LES_THETA], g.plane(), g.nz, T(SP.top_gradient * dz())));
  }
  void scalar_set_initial(const double* theta) override {
    if (!scalar_on) throw CudaError(1, "scalar not initialised (les_scalar_init)");
    upload(LES_THETA, theta, 1, g.nz);
    scalar_bc();
    LES_CUDA(cudaStreamSynchronize(st));
  }
  void scalar_kappa(double* out, int n) override {
    if (!scalar_on) throw CudaError(1, "scalar not initialised (les_scalar_init)");
    if (n < g.L) throw CudaError(1, "kappa output needs nz + 2 values");
    std::vector<double> h(g.L);
    LES_CUDA(cudaMemcpyAsync(h.data(), kapd, sizeof(double) * g.L, cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    const double d2 = delta * delta;
    for (int k = 0; k < g.L; ++k) out[k] = SP.sgs == LES_SCALAR_SGS_DYN ? h[k] / d2 : 0.0;
  }
  void sponge_init(double frac) override {
    // sponge_damping.f90:61-80 on w nodes z = (k-1) dz, without the zeroing of :83
    sponge_frac = frac > 0.0 ? frac : 0.0;
    if (sponge_frac <= 0.0) return;
    if (sponge_frac >= 1.0) throw CudaError(1, "sponge layer fraction must be below 1");
    std::vector<double> h(g.L, 0.0);
    const double lz = P.lz, z_d = sponge_frac * lz;
    for (int k = 1; k <= g.nz + 1; ++k) {
      const double z = (1 + k - 2.0) * dz();
      if (z >= z_d && z <= lz) h[k] = 3.9 * 0.5 * (1.0 - std::cos(PI * (z - z_d) / (lz - z_d)));
    }
    h[g.nz + 1] = h[g.nz];
    if (!spong) spong = track(dalloc<double>(g.L));
    if (!means) means = track(dalloc<double>(6 * g.L));
    LES_CUDA(cudaMemcpy(spong, h.data(), sizeof(double) * g.L, cudaMemcpyHostToDevice));
  }

  // gradients of theta (after compute_vel_grad: the wall law's u* is current)
  void scalar_grad() {
    Tag tag_(this, "scalar");
    const int f = LES_THETA, dx = LES_DTDX, dy = LES_DTDY;
    grad_fields(&f, &dx, &dy, 1, "scalar");
    KL("k_ddz", 2.0 * (g.nz + 1) * g.plane() * sizeof(T),
       k_ddz<T><<<grid_for((long)(g.nz + 1) * g.plane()), 256, 0, st>>>(F[LES_DTDZ], F[LES_THETA], g.plane(), g.nz,
                                                                       T(1.0 / dz()), 0));
    KL("k_scalar_wall", 2.0 * g.plane() * sizeof(T),
       k_scalar_wall<T><<<grid_for(g.plane()), 256, 0, st>>>(lev(F[LES_DTDZ], 1), PL[LES_U_STAR_AVG], g.plane(),
                                                             SP.surface_flux, 0.5 * dz()));
  }

  // dynamic Prandtl model: plane-averaged Cs^2/Pr_t at the 2 Delta filter
  void scalar_dynamic(SgsArgs<T>& a) {
    Tag tag_(this, "scalar");
    const int nlev = g.nz + 1;
    const long n1 = (long)nlev * g.plane();
    SgsArgs<T> ab = a;
    KL("k_sij", 16.0 * n1 * sizeof(T), k_sij<T><<<grid_for(n1), 256, 0, st>>>(ab));
    auto x = xf(XF_SCDYN, 19, 1, nlev, g.nx, g.ny, nk2);
    x.in[0] = F[LES_U];
    x.in[1] = F[LES_V];
    x.in[2] = F[LES_W];
    x.in[3] = F[LES_THETA];
    for (int q = 0; q < 6; ++q) x.in[4 + q] = sc[1 + q];
    x.in[10] = sc[0];
    x.in[11] = F[LES_DTDX];
    x.in[12] = F[LES_DTDY];
    x.in[13] = F[LES_DTDZ];
    for (int q = 0; q < 19; ++q) x.out[q] = spec[q];
    x.fluct = mixed() ? 1 : 0;
    launch_xfwd<T>(g.nx, x, st);
    auto y = yp(YP_FILTER1, 1, 1, nk2, nk2, g.ny, nk2, g.ny, 1);
    y.G0 = gt;
    for (int q = 0; q < 19; ++q) {
      y.in[q] = spec[q];
      y.out[q] = spec[q];
    }
    launch_ypass<T>(g.ny, g.ny, y, nlev, 19, st);
    auto z = xi(XI_SCDYN, 19, 1, nlev, g.nx, g.ny, nk2);
    z.c0 = delta * delta;
    z.c1 = 4.0;
    for (int q = 0; q < 19; ++q) z.in[q] = spec[q];
    z.out[0] = sc[7];
    z.out[1] = sc[8];
    launch_xinv<T>(g.nx, z, st);
    KL("k_level_ratio", 2.0 * n1 * sizeof(T),
       k_level_ratio<T><<<nlev, 256, 0, st>>>(sc[7], sc[8], kapd, g.plane(), delta * delta));
  }

  // scalar convective term into rhs_t (levels 1..nz); the padded -u, -v, -w
  // of the momentum's convective term are still in fine[0..2]
  void scalar_convec() {
    Tag tag_(this, "scalar");
    const int nz = g.nz;
    const bool padd = (P.dealias == LES_DEALIAS_PADD);
    const int nkin = padd ? g.nx / 2 : int(std::ceil(double(float(g.nx)) / 3.0)) - 1;
    const int FNX = padd ? g.nx2 : g.nx;
    const int FNY = padd ? g.ny2 : g.ny;
    auto a = xf(XF_SCALE, 3, 1, nz + 1, g.nx, g.ny, nkin);
    a.c0 = 1.0 / double(g.nx * g.ny);
    a.in[0] = F[LES_DTDX];
    a.in[1] = F[LES_DTDY];
    a.in[2] = F[LES_DTDZ];
    for (int q = 0; q < 3; ++q) a.out[q] = spec[q];
    launch_xfwd<T>(g.nx, a, st);
    if (padd) {
      auto b = yp(YP_PAD, 1, 1, nkin, nkin, g.ny, nkin, g.ny2, 1);
      for (int q = 0; q < 3; ++q) {
        b.in[q] = spec[q];
        b.out[q] = spec[6 + q];
      }
      launch_ypass<T>(g.ny, g.ny2, b, nz + 1, 3, st);
    } else {
      auto b = yp(YP_MASK, 1, 1, nkin, nkin, g.ny, nkin, g.ny, 1);
      b.tt = int(std::ceil(double(float(g.ny)) / 3.0)) - 2;
      for (int q = 0; q < 3; ++q) {
        b.in[q] = spec[q];
        b.out[q] = spec[6 + q];
      }
      launch_ypass<T>(g.ny, g.ny, b, nz + 1, 3, st);
    }
    auto c = xi(XI_STORE, 3, 1, nz + 1, FNX, FNY, nkin);
    for (int q = 0; q < 3; ++q) {
      c.in[q] = spec[6 + q];
      c.out[q] = fine[3 + q];
      c.lo[q] = 0;
      c.hi[q] = nz + 1;
    }
    launch_xinv<T>(FNX, c, st);
    const int nkout = padd ? g.nx / 2 : int(std::ceil(double(float(2 * g.lhx)) / 3.0)) - 1;
    auto d = xf(XF_PROD_SC, 1, 1, nz, FNX, FNY, nkout);
    d.c0 = padd ? 1.0 / double(g.nx2 * g.ny2) : 1.0 / double(g.nx * g.ny);
    for (int q = 0; q < 6; ++q) d.in[q] = fine[q];
    d.out[0] = spec[0];
    launch_xfwd<T>(FNX, d, st);
    if (padd) {
      auto e = yp(YP_TRUNC, 1, 1, nkout, nkout, g.ny2, nkout, g.ny, 1);
      e.in[0] = spec[0];
      e.out[0] = spec[3];
      launch_ypass<T>(g.ny2, g.ny, e, nz, 1, st);
    } else {
      auto e = yp(YP_MASK, 1, 1, nkout, nkout, g.ny, nkout, g.ny, 1);
      e.tt = int(std::ceil(double(float(2 * g.lhy)) / 3.0)) - 2;
      e.in[0] = spec[0];
      e.out[0] = spec[3];
      launch_ypass<T>(g.ny, g.ny, e, nz, 1, st);
    }
    auto h = xi(XI_STORE, 1, 1, nz, g.nx, g.ny, nkout);
    h.in[0] = spec[3];
    h.out[0] = F[LES_RHS_T];
    h.lo[0] = 1;
    h.hi[0] = nz;
    launch_xinv<T>(g.nx, h, st);
  }

  // after the momentum right-hand side: forcing, scalar rhs, buoyancy
  void rhs_extras() {
    const int L = g.L;
    if (coriol != 0.0 || sponge_frac > 0.0) {
      Tag tag_(this, "forcing");
      if (sponge_frac > 0.0)
        KL("k_plane_means", 3.0 * g.nz * g.plane() * sizeof(T),
           k_plane_means<T><<<g.nz, 256, 0, st>>>(F[LES_U], F[LES_V], F[LES_W], nullptr, 3, means, g.plane(), 1, L));
      KL("k_forcing", 7.0 * g.nz * g.plane() * sizeof(T),
         k_forcing<T><<<grid_for((long)g.nz * g.plane()), 256, 0, st>>>(
             F[LES_RHSX], F[LES_RHSY], F[LES_RHSZ], F[LES_U], F[LES_V], F[LES_W], means,
             sponge_frac > 0.0 ? spong : nullptr, g.plane(), g.nz, L, T(coriol), T(ug), T(vg)));
    }
    if (!scalar_on) return;
    {
      Tag tag_(this, "scalar");
      // rhs_t_f = rhs_t (buffer exchange, as the momentum's)
      copy(lev(F[LES_RHS_T], 0), lev(F[LES_RHS_T_F], 0), g.plane());
      copy(lev(F[LES_RHS_T], g.nz + 1), lev(F[LES_RHS_T_F], g.nz + 1), g.plane());
      std::swap(F[LES_RHS_T], F[LES_RHS_T_F]);
    }
    scalar_convec();
    {
      DivEq e{LES_RHS_T, LES_QX, LES_QY, LES_QZ, 1, 0.0};
      div_eqs(&e, 1, false, "scalar");
    }
    if (SP.buoyancy != 0.0) {
      Tag tag_(this, "scalar");
      KL("k_plane_means", double(L) * g.plane() * sizeof(T),
         k_plane_means<T><<<L, 256, 0, st>>>(F[LES_THETA], nullptr, nullptr, nullptr, 1, means + 3 * L, g.plane(), 0, L));
      KL("k_buoyancy", 3.0 * (g.nz - 1) * g.plane() * sizeof(T),
         k_buoyancy<T><<<grid_for((long)(g.nz - 1) * g.plane()), 256, 0, st>>>(F[LES_RHSZ], F[LES_THETA], means + 3 * L,
                                                                               g.plane(), g.nz, T(SP.buoyancy)));
    }
  }

  // -------------------------------------------------------- LES_engine ----
  void compute_rhs_adv() override {
    // LES_engine.f90:516-527: rhs_f(1:nz) = rhs(1:nz); rhs = convective term.
    // The copy is a buffer exchange: the old rhs buffer becomes rhs_f after
    // taking rhs_f's ghost levels (the reference leaves those untouched), and
    // the old rhs_f buffer receives the convective term on levels 1..nz and
    // the convective routine's ghost values.
    {
      Tag tag_(this, "convec");
      const int r[3] = {LES_RHSX, LES_RHSY, LES_RHSZ}, rf[3] = {LES_RHSX_F, LES_RHSY_F, LES_RHSZ_F};
      T* dst[6];
      const T* src[6];
      for (int q = 0; q < 3; ++q) {
        dst[2 * q] = lev(F[r[q]], 0);
        src[2 * q] = lev(F[rf[q]], 0);
        dst[2 * q + 1] = lev(F[r[q]], g.nz + 1);
        src[2 * q + 1] = lev(F[rf[q]], g.nz + 1);
      }
      plane_ops(6, dst, src, nullptr);
      for (int q = 0; q < 3; ++q) std::swap(F[r[q]], F[rf[q]]);
    }
    dealias_convec(LES_RHSX, LES_RHSY, LES_RHSZ);
    DivEq e[3] = {{LES_RHSX, LES_TXX, LES_TXY, LES_TXZ, 1, P.pfx},
                  {LES_RHSY, LES_TXY, LES_TYY, LES_TYZ, 1, P.pfy},
                  {LES_RHSZ, LES_TXZ, LES_TYZ, LES_TZZ, 0, 0.0}};
    div_eqs(e, 3, true);
    rhs_extras();
  }

  void ab2(double tadv1, double tadv2) override {
    Tag tag_(this, "ab2");
    KL("k_ab2", 12.0 * g.nz * g.plane() * sizeof(T), k_ab2<T><<<grid_for(g.field()), 256, 0, st>>>(F[LES_U], F[LES_V], F[LES_W], F[LES_RHSX], F[LES_RHSY],
                                                 F[LES_RHSZ], F[LES_RHSX_F], F[LES_RHSY_F], F[LES_RHSZ_F],
                                                 g.plane(), g.nz, T(P.dt), T(tadv1), T(tadv2)));
    if (scalar_on)
    {
      KL("k_ab2_scalar", 4.0 * g.nz * g.plane() * sizeof(T),
         k_ab2_scalar<T><<<grid_for((long)g.nz * g.plane()), 256, 0, st>>>(
             F[LES_THETA], F[LES_RHS_T], F[LES_RHS_T_F], g.plane(), g.nz, T(P.dt), T(tadv1), T(tadv2)));
      scalar_bc();
    }
  }

  void projection(double tadv1) override {
    Tag tag_(this, "projection");
    // dpdz was formed by press_stag_array; this applies LES_engine.f90:303-331
    KL("k_projection", 15.0 * g.nz * g.plane() * sizeof(T), k_projection<T><<<grid_for(g.field()), 256, 0, st>>>(F[LES_U], F[LES_V], F[LES_W], F[LES_RHSX], F[LES_RHSY],
                                                        F[LES_RHSZ], F[LES_DPDX], F[LES_DPDY], F[LES_DPDZ],
                                                        g.plane(), g.nz, P.dt * tadv1));
  }

  void step(int jt, int jtt) override { step_body(jt, jtt, true); }
  // with_diag false: the caller launches the diagnostics itself (step_host,
  // after the copies back have started)
  void step_body(int jt, int jtt, bool with_diag) {
    LES_CUDA(cudaEventRecord(ev[0], st));
    if (P.wall_law) wall_layer();  // obukhov + wallstress (same filtered layer)
    compute_vel_grad();
    LES_CUDA(cudaEventRecord(ev[1], st));
    sgs_stress(jt, jtt);
    LES_CUDA(cudaEventRecord(ev[2], st));
    compute_rhs_adv();
    LES_CUDA(cudaEventRecord(ev[3], st));
    double t1, t2;
    if (jtt == 1) {
      t1 = 1.0;
      t2 = 0.0;
    } else {
      t1 = 1.5;
      t2 = 1.0 - t1;
    }
    ab2(t1, t2);
    // the reference's formulation (FP64 transforms of u* in mixed precision);
    // press_from_increment forms the same pressure in FP32 without the
    // cancellation, but its FP32 four-field y pass measured slower than the
    // FP64 three-field one at 256^3 (0.47 against 0.36 ms per step)
    press_stag_array(t1);
    LES_CUDA(cudaEventRecord(ev[4], st));
    projection(t1);
    set_bc();
    if (with_diag) diagnostics_launch();
    LES_CUDA(cudaEventRecord(ev[5], st));
    timed = true;
  }
  bool timed = false;

  void diagnostics_launch() {
    Tag tag_(this, "diag");
    KL("k_diag_partial", 6.0 * g.nz * g.plane() * sizeof(T),
       k_diag_partial<T><<<DIAG_BLOCKS, 256, 0, st>>>(F[LES_U], F[LES_V], F[LES_W], F[LES_DUDX], F[LES_DVDY],
                                                     F[LES_DWDZ], PL[LES_U_STAR_AVG], g.plane(), g.nz, part));
    KL("k_diag_final", double(DIAG_BLOCKS) * DIAG_NV * 8.0,
       k_diag_final<<<1, 256, 0, st>>>(part, DIAG_BLOCKS, g.plane(), P.dt, P.lx / double(g.nx), P.ly / double(g.ny),
                                      dz(), double(g.nx) * double(g.ny) * double(g.nz), dout, dstatus));
  }
  void diagnostics(double out[4]) override {
    diagnostics_launch();
    LES_CUDA(cudaMemcpyAsync(out, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
  }
  unsigned status() override {
    unsigned h = 0;
    LES_CUDA(cudaMemcpyAsync(&h, dstatus, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaMemsetAsync(dstatus, 0, sizeof(unsigned), st));
    LES_CUDA(cudaStreamSynchronize(st));
    return h;
  }
  void read_timers() override {
    if (!timed) return;
    LES_CUDA(cudaEventSynchronize(ev[5]));
    float ms[5];
    LES_CUDA(cudaEventElapsedTime(&ms[0], ev[0], ev[1]));
    LES_CUDA(cudaEventElapsedTime(&ms[1], ev[1], ev[2]));
    LES_CUDA(cudaEventElapsedTime(&ms[2], ev[2], ev[3]));
    LES_CUDA(cudaEventElapsedTime(&ms[3], ev[3], ev[4]));
    LES_CUDA(cudaEventElapsedTime(&ms[4], ev[0], ev[5]));
    for (int i = 0; i < 5; ++i) timers_ms[i] = ms[i];
  }
};

// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_dpdz(T* dpdz, const T* p, long plane, int nz, T rdz, const double* pmean) {
  const long n = (long)nz * plane;
  const long t0 = blockIdx.x * (long)blockDim.x + threadIdx.x, ts = (long)gridDim.x * blockDim.x;
  // p holds the fluctuation only in mixed precision (mean mode dropped from
  // the FP32 transform); the mean-mode difference is taken in FP64
  auto one = [&](T a, T b, double dm) -> T { return pmean ? T(double(rdz * (a - b)) + dm) : rdz * (a - b); };
  if (plane % 4 == 0) {  // four consecutive points of one level per thread and iteration
    for (long q4 = t0; q4 < n / 4; q4 += ts) {
      const long o = plane + 4 * q4;
      const int k = udiv32(o, plane);
      const double dm = pmean ? double(rdz) * (pmean[k] - pmean[k - 1]) : 0.0;
      T a[4], b[4], r[4];
      ld4(p + o, a);
      ld4(p + o - plane, b);
#pragma unroll
      for (int i = 0; i < 4; ++i) r[i] = one(a[i], b[i], dm);
      st4(dpdz + o, r);
    }
  } else {
    for (long q = t0; q < n; q += ts) {
      const long o = plane + q;
      const int k = udiv32(o, plane);
      dpdz[o] = one(p[o], p[o - plane], pmean ? double(rdz) * (pmean[k] - pmean[k - 1]) : 0.0);
    }
  }
}

template <typename T>
void Solver<T>::dpdz_only() {
  const bool mixed = (P.precision == LES_MIXED);
  KL("k_dpdz", 2.0 * g.nz * g.plane() * sizeof(T), k_dpdz<T><<<grid_for((long)g.nz * g.plane() / 4), 256, 0, st>>>(F[LES_DPDZ], F[LES_P], g.plane(), g.nz,
                                                             T(1.0 / dz()), mixed ? pmean : nullptr));
}

template <typename T>
__global__ void k_vort_level(T* cx, T* cy, T* cz, const T* dwdy, const T* dvdz, const T* dudz, const T* dwdx,
                             const T* dvdx, const T* dudy, long plane, int k, T c, int wall) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < plane; p += (long)gridDim.x * blockDim.x) {
    const long o = (long)k * plane + p;
    if (wall && k == 0) {
      cx[o] = T(0);
      cy[o] = T(0);
    } else {
      cx[o] = c * (dwdy[o] - dvdz[o]);
      cy[o] = c * (dudz[o] - dwdx[o]);
    }
    cz[o] = c * (dvdx[o] - dudy[o]);
  }
}

template <typename T>
void Solver<T>::scratch_vort_level(const int* outs, int k) {
  KL("k_vort_level", 9.0 * g.plane() * sizeof(T), k_vort_level<T><<<grid_for(g.plane()), 256, 0, st>>>(
      F[outs[0]], F[outs[1]], F[outs[2]], F[LES_DWDY], F[LES_DVDZ], F[LES_DUDZ], F[LES_DWDX], F[LES_DVDX],
      F[LES_DUDY], g.plane(), k, T(1.0 / double(g.nx * g.ny)), P.wall_law));
}

// wall_inst / wall_homog (compute_wall_law.f90:119-138, 210-228)
template <typename T>
__global__ void k_wall_plain(const T* u1, const T* v1, double um, double vm, int homog, const T* z0, T* ustar,
                             T* lbu, T* lbv, T* txz1, T* tyz1, T* dudz1, T* dvdz1, long plane, double dz) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < plane; p += (long)gridDim.x * blockDim.x) {
    const double uu = homog ? um : double(u1[p]);
    const double vv = homog ? vm : double(v1[p]);
    const double uavg = sqrt(uu * uu + vv * vv);
    const double us = KVONK * uavg / log((0.5 * dz) / double(z0[p]));
    double bu = 0, bv = 0, tx = 0, ty = 0;
    if (uavg != 0.0) {
      bu = us / (0.5 * dz * KVONK) * uu / uavg;
      bv = us / (0.5 * dz * KVONK) * vv / uavg;
      tx = (us * us) * uu / uavg;
      ty = (us * us) * vv / uavg;
    }
    ustar[p] = T(us);
    lbu[p] = T(bu);
    lbv[p] = T(bv);
    txz1[p] = T(tx);
    tyz1[p] = T(ty);
    dudz1[p] = T(bu);
    dvdz1[p] = T(bv);
  }
}

template <typename T>
void Solver<T>::wall_plain() {
  double um = 0, vm = 0;
  const int homog = (P.wall_model == LES_WALL_HOMOG);
  if (homog) {
    std::vector<double> h(g.plane());
    download(LES_U, h.data(), 1, 1);
    double s = 0;
    for (double x : h) s += x;
    um = (1.0 / double(g.nx * g.ny)) * s;
    download(LES_V, h.data(), 1, 1);
    s = 0;
    for (double x : h) s += x;
    vm = (1.0 / double(g.nx * g.ny)) * s;
  }
  KL("k_wall_plain", 10.0 * g.plane() * sizeof(T), k_wall_plain<T><<<grid_for(g.plane()), 256, 0, st>>>(lev(F[LES_U], 1), lev(F[LES_V], 1), um, vm, homog,
                                                       PL[LES_LBC_Z0], PL[LES_U_STAR_AVG], PL[LES_LBC_U],
                                                       PL[LES_LBC_V], lev(F[LES_TXZ], 1), lev(F[LES_TYZ], 1),
                                                       lev(F[LES_DUDZ], 1), lev(F[LES_DVDZ], 1), g.plane(), dz()));
}

// plane-averaged dynamic Smagorinsky (compute_DynSmag.f90:61-245)
template <typename T>
__global__ void k_plane_ratio(const T* LM, const T* MM, T* cs, long plane, int nz, double cs_max) {
  // one block per level k = 1..nz+1; Neumaier sums in FP64
  const int k = blockIdx.x + 1;
  __shared__ double s[4][256];
  Neu a, b;
  for (long p = threadIdx.x; p < plane; p += blockDim.x) {
    a.add(double(LM[(long)k * plane + p]));
    b.add(double(MM[(long)k * plane + p]));
  }
  s[0][threadIdx.x] = a.s;
  s[1][threadIdx.x] = a.c;
  s[2][threadIdx.x] = b.s;
  s[3][threadIdx.x] = b.c;
  __syncthreads();
  __shared__ double res;
  if (threadIdx.x == 0) {
    Neu x, y;
    for (int i = 0; i < blockDim.x; ++i) {
      x.add(s[0][i]);
      x.add(s[1][i]);
      y.add(s[2][i]);
      y.add(s[3][i]);
    }
    const double num = x.val() / double(plane), den = y.val() / double(plane);
    double c = (den != 0.0) ? num / den : 0.0;
    res = fmax(0.0, c);
    if (cs_max > 0.0) res = fmin(res, cs_max);  // optional upper clip (off: the reference)
  }
  __syncthreads();
  for (long p = threadIdx.x; p < plane; p += blockDim.x) cs[(long)k * plane + p] = T(res);
}

template <typename T>
void Solver<T>::dynsmag(SgsArgs<T>& a, int jt, int jtt) {
  if (jtt < P.dyn_init) {
    fill(F[LES_CS_OPT2], 1, g.nz + 1, T(0.03));
    return;
  }
  if (jt % P.cs_count != 0) return;
  dynamic_mum(a, false);
  KL("k_plane_ratio", 3.0 * (g.nz + 1) * g.plane() * sizeof(T), k_plane_ratio<T><<<g.nz + 1, 256, 0, st>>>(sc[7], sc[8], F[LES_CS_OPT2], g.plane(), g.nz, cs2_max));
}

std::string SolverBase::profile_report() {
  LES_CUDA(cudaStreamSynchronize(st));
  struct Acc {
    long n = 0;
    double ms = 0, bytes = 0;
  };
  std::map<std::string, Acc> acc;
  for (const auto& r : recs) {
    float ms = 0;
    LES_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    auto& x = acc[r.label];
    x.n += 1;
    x.ms += ms;
    x.bytes += r.bytes;
  }
  std::string out = "{";
  bool first = true;
  char buf[512];
  for (const auto& kv : acc) {
    std::snprintf(buf, sizeof(buf), "%s\"%s\": {\"launches\": %ld, \"ms\": %.6f, \"bytes_per_launch\": %.1f}",
                  first ? "" : ", ", kv.first.c_str(), kv.second.n, kv.second.ms, kv.second.bytes / kv.second.n);
    out += buf;
    first = false;
  }
  return out + "}";
}

SolverBase* make_solver(const les_params& p) {
  if (p.precision == LES_MIXED) return new Solver<float>(p);
  return new Solver<double>(p);
}

}  // namespace les
