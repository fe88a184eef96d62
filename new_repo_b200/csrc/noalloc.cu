// les_grad_xy_noalloc: horizontal spectral derivatives of a device field
// with every intermediate in one fixed, file-scope device buffer.
//
// The same three spectral passes as les_grad_velocity_filt (x r2c FFT with
// the 1/(nx*ny) scaling, y pass with the ik multiplications and the Nyquist
// kill, inverse x transforms of the filtered field and both derivatives),
// launched on caller-owned device pointers.  It exists for callers that must
// not change the device memory footprint and so cannot allocate: an in-situ
// analysis hook called from a coupled model whose device memory is fully
// committed to its own fields, or code running in a process where a caching
// allocator holds the free memory, so that a cudaMalloc can fail or force the
// cache to be released.  Nothing here allocates: no cudaMalloc/cudaFree, no
// CUDA events, no host containers, no library that allocates.
//
// Scratch: g_noalloc_scratch (LES_NOALLOC_SCRATCH_BYTES) holds, 256-byte
// aligned, the wavenumber tables kkx, kky [ny][nx/2+1], the twiddle tables
// of nx and ny, and three spectra [nlev][ny][nx/2+1] (complex FP64).  Every
// call writes all of these before reading them, so nothing has to start at
// zero.  All calls in the process share the buffer of their device: two calls
// in flight at the same time on one device (different streams or host
// threads) race on it.
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/lesgpu.h"
#include "launch.cuh"

namespace les {
namespace {

constexpr size_t kScratchBytes = LES_NOALLOC_SCRATCH_BYTES;
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::atomic<unsigned char*> g_scratch_addr[kMaxDevices] = {};  // per device, set by the first call on it

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

struct ScratchLayout {
  size_t kkx, kky, twx, twy, spec[3], total;
};
ScratchLayout scratch_layout(int nx, int ny, int nlev) {
  const size_t lhx = size_t(nx / 2 + 1);
  const size_t tab = align256(sizeof(double) * size_t(ny) * lhx);
  const size_t spec = align256(sizeof(cplx<double>) * size_t(nlev) * size_t(ny) * lhx);
  ScratchLayout L;
  size_t o = 0;
  L.kkx = o;
  o += tab;
  L.kky = o;
  o += tab;
  L.twx = o;
  o += align256(sizeof(cplx<double>) * size_t(nx));
  L.twy = o;
  o += align256(sizeof(cplx<double>) * size_t(ny));
  for (int i = 0; i < 3; ++i) {
    L.spec[i] = o;
    o += spec;
  }
  L.total = o;
  return L;
}

// wavenumber tables (fft_engine.f90:127-143, Nyquist row and column zeroed)
// and the exp(-2 pi i m / n) twiddle tables, computed on the device
__global__ void k_noalloc_tables(double* kkx, double* kky, cplx<double>* twx, cplx<double>* twy, int nx, int ny,
                                 double lx, double ly) {
  const int lhx = nx / 2 + 1, lhy = ny / 2 + 1;
  const double pi = 3.14159265358979323846;
  const long n = (long)ny * lhx;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int i = int(q % lhx), j = int(q / lhx);
    double kx = double(i);
    double ky = double(((j + ny / 2) % ny) - ny / 2);
    if (i == lhx - 1 || j == lhy - 1) {
      kx = 0.0;
      ky = 0.0;
    }
    kkx[q] = 2.0 * pi / lx * kx;
    kky[q] = 2.0 * pi / ly * ky;
  }
  for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < nx + ny; m += (long)gridDim.x * blockDim.x) {
    const bool isx = m < nx;
    const int len = isx ? nx : ny;
    const int mm = int(isx ? m : m - nx);
    double s, c;
    sincospi(-2.0 * double(mm) / double(len), &s, &c);
    (isx ? twx : twy)[mm] = cplx<double>{c, s};
  }
}

// address of this device's scratch buffer; the first call on a device does
// the setup (symbol address, kernel shared-memory attributes)
int scratch_for_device(unsigned char** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw CudaError(LES_ERR_INVALID, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) throw CudaError(LES_ERR_INVALID, "device ordinal out of range");
  unsigned char* addr = g_scratch_addr[dev].load();
  if (!addr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      throw CudaError(LES_ERR_INVALID, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    init_spectral_attributes();
    addr = static_cast<unsigned char*>(p);
    g_scratch_addr[dev].store(addr);
  }
  *out = addr;
  return dev;
}

}  // namespace
}  // namespace les

namespace {
thread_local char g_noalloc_error[256];
}

extern "C" const char* les_noalloc_last_error(void) { return g_noalloc_error; }

extern "C" int les_grad_xy_noalloc(double* f, double* dfdx, double* dfdy, int nx, int ny, int nlev, double lx,
                                   double ly, void* stream) {
  using namespace les;
  g_noalloc_error[0] = '\0';
  auto fail = [](int code, const char* msg) {
    std::snprintf(g_noalloc_error, sizeof(g_noalloc_error), "%s", msg);
    return code;
  };
  if (!f || !dfdx || !dfdy) return fail(LES_ERR_INVALID, "les_grad_xy_noalloc: null field pointer");
  if ((reinterpret_cast<uintptr_t>(f) | reinterpret_cast<uintptr_t>(dfdx) | reinterpret_cast<uintptr_t>(dfdy)) & 15u)
    return fail(LES_ERR_INVALID, "les_grad_xy_noalloc: field pointers must be 16-byte aligned");
  if (nx <= 0 || ny <= 0 || nlev <= 0 || !(lx > 0) || !(ly > 0))
    return fail(LES_ERR_INVALID, "les_grad_xy_noalloc: invalid grid or domain size");
  // x: every length with a register FFT plan; y: the lengths with an
  // equal-length y pass (powers of two), checked before anything is queued
  const bool ny_ok = ny == 16 || ny == 32 || ny == 64 || ny == 128 || ny == 256 || ny == 512;
  if (!supported_length(nx) || !ny_ok)
    return fail(LES_ERR_INVALID,
                "les_grad_xy_noalloc: nx must be one of 16 24 32 48 64 96 128 192 256 384 512 768 and ny one of "
                "16 32 64 128 256 512");
  const ScratchLayout L = scratch_layout(nx, ny, nlev);
  if (L.total > kScratchBytes) {
    std::snprintf(g_noalloc_error, sizeof(g_noalloc_error),
                  "les_grad_xy_noalloc: %dx%dx%d needs %zu bytes of scratch, the static buffer holds %zu "
                  "(LES_NOALLOC_SCRATCH_BYTES)",
                  nx, ny, nlev, L.total, kScratchBytes);
    return LES_ERR_INVALID;
  }
  // launches here are not observed by a solver's profiling hook; the hook is
  // per host thread, so only states profiled on the calling thread are
  // affected, and only for the duration of this call
  LaunchHook* saved = g_hook;
  g_hook = nullptr;
  int rc = LES_OK;
  try {
    unsigned char* base = nullptr;
    scratch_for_device(&base);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* kkx = reinterpret_cast<double*>(base + L.kkx);
    double* kky = reinterpret_cast<double*>(base + L.kky);
    auto* twx = reinterpret_cast<cplx<double>*>(base + L.twx);
    auto* twy = reinterpret_cast<cplx<double>*>(base + L.twy);
    cplx<double>* sp[3];
    for (int i = 0; i < 3; ++i) sp[i] = reinterpret_cast<cplx<double>*>(base + L.spec[i]);
    const int lhx = nx / 2 + 1;
    k_noalloc_tables<<<64, 256, 0, st>>>(kkx, kky, twx, twy, nx, ny, lx, ly);
    LES_CHECK_LAUNCH();

    XFArgs<double> a;
    std::memset(&a, 0, sizeof(a));
    a.op = XF_SCALE;
    a.nf = 1;
    a.rows_pp = ny;
    a.nrows = (long)nlev * ny;
    a.nk = lhx;
    a.nz = nlev - 2;
    a.in_pstride = (long)ny * nx;
    a.out_pstride = (long)ny * lhx;
    a.tw = twx;
    a.c0 = 1.0 / double(nx * ny);
    a.in[0] = f;
    a.out[0] = sp[0];
    launch_xfwd<double>(nx, a, st);

    YPArgs<double> b;
    std::memset(&b, 0, sizeof(b));
    b.op = YP_GRAD;
    b.nin = 1;
    b.nout = 3;
    b.ncols = lhx;
    b.nk_in = lhx;
    b.nk_out = lhx;
    b.in_pstride = (long)ny * lhx;
    b.out_pstride = (long)ny * lhx;
    b.nxh = nx / 2;
    b.lhx = lhx;
    b.kkx = kkx;
    b.kky = kky;
    b.tw_in = twy;
    b.tw_out = twy;
    b.in[0] = sp[0];
    b.out[0] = sp[0];
    b.out[1] = sp[1];
    b.out[2] = sp[2];
    launch_ypass<double>(ny, ny, b, nlev, 1, st);

    XIArgs<double> c;
    std::memset(&c, 0, sizeof(c));
    c.op = XI_STORE;
    c.nin = 3;
    c.rows_pp = ny;
    c.nrows = (long)nlev * ny;
    c.nk = lhx;
    c.nz = nlev - 2;
    c.in_pstride = (long)ny * lhx;
    c.out_pstride = (long)ny * nx;
    c.tw = twx;
    for (int q = 0; q < 3; ++q) {
      c.in[q] = sp[q];
      c.lo[q] = 0;
      c.hi[q] = nlev - 1;
    }
    c.out[0] = f;
    c.out[1] = dfdx;
    c.out[2] = dfdy;
    launch_xinv<double>(nx, c, st);
  } catch (const CudaError& e) {
    std::snprintf(g_noalloc_error, sizeof(g_noalloc_error), "%s", e.what());
    rc = e.code ? e.code : LES_ERR_INVALID;
  } catch (const std::exception& e) {
    std::snprintf(g_noalloc_error, sizeof(g_noalloc_error), "%s", e.what());
    rc = LES_ERR_INVALID;
  }
  g_hook = saved;
  return rc;
}
