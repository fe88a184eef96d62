// Instantiation and launch of the y passes (k_ypass) for every supported
// length pair.
#include "spectral_launch.cuh"

#include "launch.cuh"

namespace les {

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
void set_attrs_ypass() {
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

template void launch_ypass<float>(int, int, YPArgs<float>, int, int, cudaStream_t);
template void launch_ypass<double>(int, int, YPArgs<double>, int, int, cudaStream_t);
template void set_attrs_ypass<float>();
template void set_attrs_ypass<double>();

}  // namespace les
