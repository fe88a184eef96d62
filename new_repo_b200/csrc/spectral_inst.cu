// Launch helpers of the spectral passes (occupancy and register caches,
// FFT lane counts, supported lengths) and the per-device shared-memory
// attributes of their kernels.  The kernels are instantiated and launched
// in spectral_xfwd.cu, spectral_xinv.cu and spectral_ypass.cu.
#include "spectral_launch.cuh"
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
int resident_ctas(const void* kern, int threads, size_t smem) {
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
KernelLimits kernel_limits(const void* kern) {
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

bool supported_length(int n) {
  switch (n) {
    case 16: case 24: case 32: case 48: case 64: case 96: case 128:
    case 192: case 256: case 384: case 512: case 768:
      return true;
    default:
      return false;
  }
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
  set_attrs_xfwd<float>();
  set_attrs_xfwd<double>();
  set_attrs_xinv<float>();
  set_attrs_xinv<double>();
  set_attrs_ypass<float>();
  set_attrs_ypass<double>();
  done[dev] = true;
}

}  // namespace les
