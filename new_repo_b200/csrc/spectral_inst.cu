// Instantiation and launch of the spectral pass kernels for every supported
// transform length (2^a 3^b: the grid sizes 16..512 and their 3/2 padding).
#include "spectral.cuh"
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "launch.cuh"

namespace les {

thread_local LaunchHook* g_hook = nullptr;

// CTAs of `kern` resident on the current device at once; cached in a fixed
// table (no heap allocation: the allocation-free entry point launches these
// kernels too)
struct ResidentEntry {
  int dev;
  const void* kern;
  int threads;
  size_t smem;
  int n;
};
static int resident_ctas(const void* kern, int threads, size_t smem) {
  static std::mutex mu;
  static ResidentEntry table[256];
  static int used = 0;
  int dev = 0;
  LES_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  for (int i = 0; i < used; ++i) {
    const ResidentEntry& e = table[i];
    if (e.dev == dev && e.kern == kern && e.threads == threads && e.smem == smem) return e.n;
  }
  int per_sm = 0, sms = 0;
  LES_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
  LES_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int n = std::max(1, per_sm) * std::max(1, sms);
  if (used < 256) table[used++] = ResidentEntry{dev, kern, threads, smem, n};
  return n;
}


// registers per thread and the largest CTA of `kern` on the current device
// (fixed table, as above)
struct KernelLimits {
  int regs, max_threads;
};
static KernelLimits kernel_limits(const void* kern) {
  static std::mutex mu;
  static struct {
    int dev;
    const void* kern;
    KernelLimits lim;
  } table[128];
  static int used = 0;
  int dev = 0;
  LES_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  for (int i = 0; i < used; ++i)
    if (table[i].dev == dev && table[i].kern == kern) return table[i].lim;
  cudaFuncAttributes fa;
  LES_CUDA(cudaFuncGetAttributes(&fa, kern));
  const KernelLimits lim{fa.numRegs, fa.maxThreadsPerBlock};
  if (used < 128) table[used++] = {dev, kern, lim};
  return lim;
}
static int kernel_regs(const void* kern) { return kernel_limits(kern).regs; }

namespace {
constexpr int SMEM_CAP = 200 * 1024;
constexpr size_t SM_SMEM = 228 * 1024;  // shared memory per SM (1 KB of it reserved per CTA)

// Rows per work item of an x pass (256-thread CTAs, TL lanes per sequence,
// seq_per_row sequences per grid row): the count that keeps the most sequence
// slots of an SM busy -- resident CTAs (shared memory, registers) times the
// fraction of the 256 / TL slots of each pass that hold a sequence; on a tie
// the larger count (fewer items).
template <typename SmemFn>
int best_rows(const void* kern, int seq_per_row, int TL, SmemFn smem_for, int rmax = 32, double* best_score = nullptr,
              int threads = 256) {
  const int regs = kernel_regs(kern);
  const int warp_regs = ((regs * 32 + 255) / 256) * 256;
  const int by_regs = std::max(1, 65536 / (warp_regs * (threads / 32)));
  const int S = threads / TL;
  double best = -1.0;
  int best_r = 1;
  for (int R = 1; R <= rmax; ++R) {
    const size_t sm = smem_for(R);
    if (sm > SMEM_CAP) break;
    const int ctas = std::min({int(SM_SMEM / (sm + 1024)), by_regs, 2048 / threads, 32});
    if (ctas < 1) break;
    const int nseq = R * seq_per_row;
    const int passes = (nseq + S - 1) / S;
    const double score = ctas * double(nseq) / double(passes * S);
    if (score >= best - 1e-9) {
      best = score;
      best_r = R;
    }
  }
  if (best_score) *best_score = best;
  return best_r;
}

// lanes per sequence of the register FFT of length n (fft2.cuh plans)
int lanes(int n) {
  switch (n) {
    case 8: return Geo<8>::T;
    case 12: return Geo<12>::T;
    case 16: return Geo<16>::T;
    case 24: return Geo<24>::T;
    case 32: return Geo<32>::T;
    case 48: return Geo<48>::T;
    case 64: return Geo<64>::T;
    case 96: return Geo<96>::T;
    case 128: return Geo<128>::T;
    case 192: return Geo<192>::T;
    case 256: return Geo<256>::T;
    case 384: return Geo<384>::T;
    case 512: return Geo<512>::T;
    case 768: return Geo<768>::T;
    default: throw CudaError(1, "no FFT plan for length " + std::to_string(n));
  }
}
int pad_seqs(int nseq, int M) {
  const int spw = 32 / lanes(M);
  return ((nseq + spw - 1) / spw) * spw;
}
}  // namespace

bool supported_length(int n) {
  switch (n) {
    case 16: case 24: case 32: case 48: case 64: case 96: case 128:
    case 192: case 256: case 384: case 512: case 768:
      return true;
    default:
      return false;
  }
}

#define LES_LENGTHS(X) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768)

// the staged x forward pass (ops whose inputs are whole rows)
template <typename T, typename S>
static void launch_xfwd_st(int NX, XFArgs<T>& a, cudaStream_t st) {
  const int M = NX / 2;
  a.nsrc = 0;
  if (a.op == XF_CONV_IN) {
    for (int f = 0; f < 9; ++f) {
      a.sf[a.nsrc] = f;
      a.sdl[a.nsrc] = 0;
      a.scond[a.nsrc++] = 0;
    }
    for (int f : {3, 6}) {  // dwdy, dwdx one level up, read on the wall row only
      a.sf[a.nsrc] = f;
      a.sdl[a.nsrc] = 1;
      a.scond[a.nsrc++] = 1;
    }
  } else {
    for (int f = 0; f < a.nf; ++f) {
      a.sf[a.nsrc] = f;
      a.sdl[a.nsrc] = 0;
      a.scond[a.nsrc++] = 0;
    }
  }
  const int SL = slot_stride(M, int(sizeof(cplx<T>)));
  auto smem_for = [&](int R) {
    return sizeof(cplx<T>) * (NX + twm_len(M, false) + (size_t)pad_seqs(R * a.nf, M) * SL) +
           2 * sizeof(S) * (size_t)R * a.nsrc * NX +
           sizeof(T) * R * a.nf + 2 * sizeof(int) * R + 16;
  };
  void (*kern)(XFArgs<T>) = nullptr;
  switch (NX) {
#define XS_CASE(N) \
  case N: kern = k_xfwd_st<T, N, S>; break;
    LES_LENGTHS(XS_CASE)
#undef XS_CASE
    default:
      throw CudaError(1, "xfwd: unsupported transform length " + std::to_string(NX));
  }
  a.R = best_rows((const void*)kern, a.nf, lanes(M), smem_for);
  const size_t smem = smem_for(a.R);
  if (smem > SMEM_CAP) throw CudaError(1, "xfwd: shared memory request too large");
  const long nitems = ceil_div(a.nrows, a.R);
  if (nitems == 0) return;
  const int grid = int(std::min<long>(nitems, (long)resident_ctas((const void*)kern, 256, smem)));
  kern<<<grid, 256, smem, st>>>(a);
  LES_CHECK_LAUNCH();
}

template <typename T>
void launch_xfwd(int NX, XFArgs<T> a, cudaStream_t st) {
  const int M = NX / 2;
  if (a.opitch == 0) a.opitch = a.nk;
  // the staged kernel pays for its two input stages with occupancy: it wins
  // for the pressure inputs and for scalings of few fields (measured at 256^3)
  const bool staged = a.op == XF_PRESS || (a.op == XF_SCALE && a.nf <= 3);
  if (staged) {
    a.in_rstride = NX;
    static const int nin_of_op[] = {0, 9, 6, 10, 0, 6, 14, 9};
    const int nin = (a.op == XF_SCALE || a.op == XF_PRESS) ? a.nf : nin_of_op[a.op];
    const size_t isz = (a.in_f32 ? sizeof(float) : sizeof(T));
    hook_before("xfwd", double(a.nrows) * NX * nin * isz + double(a.nrows) * a.nf * a.nk * sizeof(cplx<T>));
    if (a.in_f32) {
      if constexpr (std::is_same<T, double>::value) launch_xfwd_st<T, float>(NX, a, st);
      else throw CudaError(1, "xfwd: FP32 inputs are for FP64 transforms");
    } else {
      launch_xfwd_st<T, T>(NX, a, st);
    }
    hook_after();
    return;
  }
  a.in_rstride = NX;
  const int SL = slot_stride(M, int(sizeof(cplx<T>)));
  auto smem_for = [&](int R) {
    return sizeof(cplx<T>) * (NX + twm_len(M, false) + (size_t)pad_seqs(R * a.nf, M) * SL) + sizeof(T) * R * a.nf +
           2 * sizeof(int) * R + 16;
  };
  void (*kern)(XFArgs<T>) = nullptr;
  switch (NX) {
#define XF_CASE(N) \
  case N: kern = k_xfwd<T, N>; break;
    LES_LENGTHS(XF_CASE)
#undef XF_CASE
    default:
      throw CudaError(1, "xfwd: unsupported transform length " + std::to_string(NX));
  }
  // the convective input and product passes load many inputs per point
  // straight from global memory: 128-thread CTAs (twice the CTAs per SM at
  // the same register budget) overlap one CTA's loads with the transforms of
  // others at a finer grain (measured at 256^3: 0.667 -> 0.633 ms per step);
  // the other ops keep 256 threads (the stress divergence measured slower
  // with 128: 0.236 -> 0.256 ms)
  const int XF_THREADS = (a.op == XF_CONV_IN || a.op == XF_PROD || a.op == XF_PROD_SC) ? 128 : 256;
  a.R = best_rows((const void*)kern, a.nf, lanes(M), smem_for, 32, nullptr, XF_THREADS);
  const size_t smem = smem_for(a.R);
  if (smem > SMEM_CAP) throw CudaError(1, "xfwd: shared memory request too large");
  const int grid = ceil_div(a.nrows, a.R);
  if (grid == 0) return;
  static const int nin_of_op[] = {0, 9, 6, 10, 0, 6, 14, 9};
  const int nin = (a.op == XF_SCALE || a.op == XF_PRESS) ? a.nf : nin_of_op[a.op];
  const size_t isz = (a.in_f32 ? sizeof(float) : sizeof(T));
  hook_before("xfwd", double(a.nrows) * NX * nin * isz + double(a.nrows) * a.nf * a.nk * sizeof(cplx<T>));
  kern<<<grid, XF_THREADS, smem, st>>>(a);
  LES_CHECK_LAUNCH();
  hook_after();
}

template <typename T>
void launch_xinv(int NX, XIArgs<T> a, cudaStream_t st) {
  const int M = NX / 2;
  if (a.ipitch == 0) a.ipitch = a.nk;
  a.pair_store = (a.out_pstride % 2 == 0);
  for (int f = 0; f < a.nin && f < 16; ++f)
    if (a.out[f] && reinterpret_cast<uintptr_t>(a.out[f]) % (2 * sizeof(T)) != 0) a.pair_store = 0;
  // sequence slots and one or two input stages per CTA; rows per work item
  // and stages from best_rows below
  const int SL = slot_stride(M, int(sizeof(cplx<T>)));
  const int ns = a.nstage ? a.nstage : a.nin;  // staged rows per grid row
  {
    // staged row stride: the split reads a row's modes at consecutive
    // lanes, the TL lanes of 32 / TL sequences per warp in different rows;
    // a stride of TL (mod the values per wavefront) puts those rows on
    // disjoint banks, as slot_stride does for the sequence slots
    const int W = 128 / int(sizeof(cplx<T>)), TL = lanes(M);
    a.nks = a.nk;
    if (TL < W) a.nks += ((TL % W - a.nk % W) % W + W) % W;
  }
  // a plain store with one staged row per sequence transforms each sequence
  // in its own staged row (the exchange slot is the row), which leaves room
  // for more rows per work item
  a.merged = (a.op == XI_STORE && a.nstage == 0) ? 1 : 0;
  if (a.merged) a.nks = std::max(a.nks, SL);
  auto stage_rows = [&](int R) { return a.merged ? pad_seqs(R * a.nin, M) : R * ns; };
  auto smem_nb = [&](int R, int nb) {
    return sizeof(cplx<T>) * (NX + twm_len(M, true) + nb * (((size_t)stage_rows(R) * a.nks + 1) & ~size_t(1)) +
                              (a.merged ? 0 : (size_t)pad_seqs(R * a.nin, M) * SL)) +
           2 * sizeof(int) * R + (a.nstage ? sizeof(T) * (a.nk + 2) : 0);
  };
  void (*kern)(XIArgs<T>) = nullptr;
  switch (NX) {
#define XI_CASE(N) \
  case N: kern = k_xinv<T, N>; break;
    LES_LENGTHS(XI_CASE)
#undef XI_CASE
    default:
      throw CudaError(1, "xinv: unsupported transform length " + std::to_string(NX));
  }
  // two stages unless one stage keeps strictly more sequence slots busy
  // (more resident CTAs where shared memory limits them)
  {
    double s2 = -1.0, s1 = -1.0;
    const int r2 = best_rows((const void*)kern, a.nin, lanes(M), [&](int R) { return smem_nb(R, 2); }, 32, &s2);
    const int r1 = best_rows((const void*)kern, a.nin, lanes(M), [&](int R) { return smem_nb(R, 1); }, 32, &s1);
    a.nbuf = (s1 > s2 + 1e-9) ? 1 : 2;
    a.R = (a.nbuf == 1) ? r1 : r2;
  }
  a.stage_rows = stage_rows(a.R);
  const size_t smem = smem_nb(a.R, a.nbuf);
  if (smem > SMEM_CAP) throw CudaError(1, "xinv: shared memory request too large");
  {
    // the combining ops read the sequence slots four reals at a time
    const size_t stage_len = ((size_t)a.stage_rows * a.nks + 1) & ~size_t(1);
    const size_t slots = sizeof(cplx<T>) * (NX + twm_len(M, true) + a.nbuf * stage_len);
    if (!a.merged && slots % 16 != 0) throw CudaError(1, "xinv: sequence slots not 16-byte aligned");
  }
  const long nitems = ceil_div(a.nrows, a.R);
  if (nitems == 0) return;
  const int grid = int(std::min<long>(nitems, (long)resident_ctas((const void*)kern, 256, smem)));
  {
    const size_t osz = (a.out_f32 ? sizeof(float) : sizeof(T));
    int nout = a.nin, rmw = 0;
    if (a.op == XI_DIV) { nout = a.nin; rmw = 2 * a.nin; }
    else if (a.op == XI_LASD || a.op == XI_SCDYN) nout = 2;
    else if (a.op == XI_WALL) nout = 7;
    hook_before("xinv", double(a.nrows) * ns * a.nk * sizeof(cplx<T>) + double(a.nrows) * NX * (nout + rmw) * osz);
  }
  kern<<<grid, 256, smem, st>>>(a);
  LES_CHECK_LAUNCH();
  hook_after();
}

// the y-pass kernel of a length pair; the forward-only variant exists for
// equal lengths (nullptr otherwise)
template <typename T, int A, int B>
static void (*ypass_kernel(bool fwd))(YPArgs<T>) {
  if constexpr (A == B) return fwd ? k_ypass<T, A, A, true> : k_ypass<T, A, B>;
  else return fwd ? nullptr : k_ypass<T, A, B>;
}

template <typename T>
void launch_ypass(int NY, int NYO, YPArgs<T> a, int nplanes, int ngroups, cudaStream_t st) {
  if (a.ipitch == 0) a.ipitch = a.nk_in;
  if (a.opitch == 0) a.opitch = a.nk_out;
  if (a.opitch1 == 0) a.opitch1 = a.nk_out1;
  const int TL = lanes(NY);
  if (lanes(NYO) != TL) throw CudaError(1, "ypass: length pair with different lane counts");
  // column stride of the shared stages: the load and store loops run c
  // (column) fastest and 32/C rows per warp, so a stride congruent to 32/C
  // modulo the complex values per 128-byte wavefront spreads a warp evenly
  // over the banks; room for the padded exchange layout of the longer of the
  // two transforms (the inverse runs in the first input row of each column)
  const int W = 128 / int(sizeof(cplx<T>));
  const int NL = std::max(NY, NYO);
  auto stride = [&](int C) {
    const int target = (32 / C) % W;
    const int base = NL + NL / 16;
    return base + ((target - base % W) % W + W) % W;
  };
  auto smem_for = [&](int C, int ns) {  // twiddle matrices, the ky row, ns stages of nin rows per column
    return sizeof(cplx<T>) * (twm_len(NY, false) + twm_len(NYO, true) + (size_t)C * ns * a.nin * stride(C)) +
           sizeof(T) * ((NY + 3) & ~3);
  };
  const int key = NY * 10000 + NYO;
  const bool fwd = (a.op == YP_FWDKILL);
  void (*kern)(YPArgs<T>) = nullptr;
  switch (key) {
#define YP_CASE(A, B) \
  case A * 10000 + B: kern = ypass_kernel<T, A, B>(fwd); break;
    YP_CASE(16, 16) YP_CASE(32, 32) YP_CASE(64, 64) YP_CASE(128, 128) YP_CASE(256, 256) YP_CASE(512, 512)
    YP_CASE(16, 24) YP_CASE(32, 48) YP_CASE(64, 96) YP_CASE(128, 192) YP_CASE(256, 384) YP_CASE(512, 768)
    YP_CASE(24, 16) YP_CASE(48, 32) YP_CASE(96, 64) YP_CASE(192, 128) YP_CASE(384, 256) YP_CASE(768, 512)
#undef YP_CASE
    default:
      throw CudaError(1, "ypass: unsupported length pair " + std::to_string(NY) + "->" + std::to_string(NYO));
  }
  if (!kern) throw CudaError(1, "ypass: a forward-only pass keeps the length");
  // columns per CTA (C * TL threads, at least a warp) and input stages: the
  // most busy warps per SM -- resident CTAs (shared memory, registers,
  // threads) times the warps whose columns exist; on a tie two stages (the
  // loads of the next item overlap this one), then the CTA size nearest 128
  // threads (measured at 256^3: 128-thread CTAs beat 64 and 256 at equal
  // occupancy).  One stage wins where shared memory, not registers, limits
  // the resident CTAs (the two-input stress divergence on 512-point columns).
  {
    const KernelLimits lim = kernel_limits((const void*)kern);
    const int regs = lim.regs;
    double best = -1.0;
    int best_lc = 0, best_ns = 2;
    while ((1 << best_lc) * TL < 32) ++best_lc;  // at least one full warp
    auto off128 = [&](int lc) { return std::abs(std::log2(double((1 << lc) * TL) / 128.0)); };
    for (int ns = 2; ns >= 1; --ns)
      for (int lc = 0; (1 << lc) * TL <= std::min(256, lim.max_threads); ++lc) {
        const int C = 1 << lc, threads = C * TL;
        if (threads < 32) continue;
        const size_t sm = smem_for(C, ns);
        if (sm > SMEM_CAP) break;
        const int warp_regs = ((regs * 32 + 255) / 256) * 256;
        const int by_regs = 65536 / (warp_regs * (threads / 32));
        const int ctas = std::min({int(SM_SMEM / (sm + 1024)), by_regs, 2048 / threads, 32});
        if (ctas < 1) break;
        const double busy = ctas * double(threads / 32) * std::min(1.0, double(a.ncols) / C);
        if (busy > best + 1e-9 || (busy > best - 1e-9 && ns == best_ns && off128(lc) < off128(best_lc))) {
          best = busy;
          best_lc = lc;
          best_ns = ns;
        }
      }
    a.lc = best_lc;
    a.nstage = best_ns;
  }
  a.C = 1 << a.lc;
  a.SI = stride(a.C);
  const size_t smem = smem_for(a.C, a.nstage);
  if (smem > SMEM_CAP) throw CudaError(1, "ypass: shared memory request too large");
  const int threads = a.C * TL;
  a.nplanes = nplanes;
  a.ngroups = ngroups;
  const long nitems = (long)ceil_div(a.ncols, a.C) * nplanes * ngroups;
  if (nitems == 0) return;
  // persistent grid: the CTAs that fit on the device at once
  const int grid = int(std::min<long>(nitems, (long)resident_ctas((const void*)kern, threads, smem)));
  hook_before("ypass", double(nplanes) * ngroups * a.ncols * sizeof(cplx<T>) *
                           (double(a.op == YP_PGRAD ? 1 : a.nin) * NY + double(a.nout) * NYO));
  kern<<<grid, threads, smem, st>>>(a);
  LES_CHECK_LAUNCH();
  hook_after();
}

template <typename T>
static void set_attrs() {
#define XA(N)                                                                                       \
  LES_CUDA(cudaFuncSetAttribute(k_xfwd<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP)); \
  LES_CUDA(cudaFuncSetAttribute(k_xfwd_st<T, N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP)); \
  if constexpr (std::is_same<T, double>::value)                                                       \
    LES_CUDA(cudaFuncSetAttribute(k_xfwd_st<T, N, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP)); \
  LES_CUDA(cudaFuncSetAttribute(k_xinv<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP));
  LES_LENGTHS(XA)
#undef XA
#define YA(A, B) \
  LES_CUDA(cudaFuncSetAttribute(k_ypass<T, A, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP));
#define YF(A) \
  LES_CUDA(cudaFuncSetAttribute(k_ypass<T, A, A, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP));
  YF(16) YF(32) YF(64) YF(128) YF(256) YF(512)
#undef YF
  YA(16, 16) YA(32, 32) YA(64, 64) YA(128, 128) YA(256, 256) YA(512, 512)
  YA(16, 24) YA(32, 48) YA(64, 96) YA(128, 192) YA(256, 384) YA(512, 768)
  YA(24, 16) YA(48, 32) YA(96, 64) YA(192, 128) YA(384, 256) YA(768, 512)
#undef YA
}

// cudaFuncSetAttribute applies to the current device only: done once per
// device ordinal (fixed table and a mutex, no heap allocation), so states on
// several devices of one process, and threads creating them at once, all
// launch with the shared-memory limit raised
void init_spectral_attributes() {
  static std::mutex mu;
  static bool done[256] = {};
  int dev = 0;
  LES_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) throw CudaError(1, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return;
  set_attrs<float>();
  set_attrs<double>();
  done[dev] = true;
}

template void launch_xfwd<float>(int, XFArgs<float>, cudaStream_t);
template void launch_xfwd<double>(int, XFArgs<double>, cudaStream_t);
template void launch_xinv<float>(int, XIArgs<float>, cudaStream_t);
template void launch_xinv<double>(int, XIArgs<double>, cudaStream_t);
template void launch_ypass<float>(int, int, YPArgs<float>, int, int, cudaStream_t);
template void launch_ypass<double>(int, int, YPArgs<double>, int, int, cudaStream_t);

}  // namespace les
