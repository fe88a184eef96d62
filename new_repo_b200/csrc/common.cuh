// Common definitions for the B200 LES library: complex type, field layout,
// error handling and the device status word.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <stdexcept>

namespace les {

// Sentinel used by the reference for undefined nodes (parameters_IO.f90:49).
constexpr double BOGUS = -1.23456789e20;
constexpr double KVONK = 0.4;

template <typename T>
struct __align__(2 * sizeof(T)) cplx {
  T x, y;
};

template <typename T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__device__ __forceinline__ cplx<T> cmulc(cplx<T> a, cplx<T> b) {  // a * conj(b)
  return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename T>
__device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T>
__device__ __forceinline__ cplx<T> cscale(cplx<T> a, T s) { return {a.x * s, a.y * s}; }
// i * k * a, written as (0 + i k) * (ax + i ay) the way the reference's
// eye*kkx*f_hat evaluates it.
template <typename T>
__device__ __forceinline__ cplx<T> ik_mul(T k, cplx<T> a) {
  return {T(0) * a.x - k * a.y, T(0) * a.y + k * a.x};
}

// Quotient and remainder of non-negative offsets below 2^32 (every field and
// fine-grid buffer of a supported grid; the state checks its sizes when it is
// created) in 32-bit unsigned arithmetic: a 64-bit division is a long
// software sequence on the GPU, and these sit in per-row and per-point paths.
__device__ __forceinline__ int udiv32(long n, long d) { return int(unsigned(n) / unsigned(d)); }
__device__ __forceinline__ int umod32(long n, long d) { return int(unsigned(n) % unsigned(d)); }

// Device status bits (read back by les_get_status).
enum StatusBits : unsigned {
  ST_NAN = 1u << 0,          // NaN in the velocity (LES_engine.f90:583-616)
  ST_PIVOT = 1u << 1,        // zero pivot in the tridiagonal solve (compute_pressure.f90:411-418)
  ST_MLP_RANGE = 1u << 2,    // learned closure saw inputs outside its training range
  ST_BAD_ARG = 1u << 3,      // kernel argument check failed
  ST_MLP_WAIT = 1u << 4,     // a closure kernel's tensor-core wait ran out
  ST_COPY_WAIT = 1u << 5,    // a spectral pass's bulk-copy wait ran out
};

struct CudaError : std::runtime_error {
  int code;
  CudaError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Status of a failed CUDA call: 3 (the reference's out-of-memory code) for an
// allocation failure, 4 for any other CUDA error.  Errors the CUDA runtime
// marks as sticky (a device fault: illegal address, launch failure, ...)
// leave the context unusable; the message says so.
inline int cuda_status_code(cudaError_t e) { return e == cudaErrorMemoryAllocation ? 3 : 4; }
inline bool cuda_error_is_sticky(cudaError_t e) {
  switch (e) {
    case cudaErrorIllegalAddress: case cudaErrorLaunchFailure: case cudaErrorIllegalInstruction:
    case cudaErrorMisalignedAddress: case cudaErrorInvalidAddressSpace: case cudaErrorInvalidPc:
    case cudaErrorHardwareStackError: case cudaErrorAssert: case cudaErrorLaunchTimeout:
    case cudaErrorECCUncorrectable:
      return true;
    default:
      return false;
  }
}
inline std::string cuda_error_text(const char* call, cudaError_t e) {
  std::string m = std::string(call) + ": " + cudaGetErrorString(e);
  if (cuda_error_is_sticky(e)) m += " (sticky device error: the CUDA context is lost; destroy the states and exit)";
  return m;
}

#define LES_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      throw ::les::CudaError(::les::cuda_status_code(e_), ::les::cuda_error_text(#call, e_));   \
    }                                                                                           \
  } while (0)

#define LES_CHECK_LAUNCH() LES_CUDA(cudaGetLastError())

inline int ceil_div(long a, long b) { return int((a + b - 1) / b); }

}  // namespace les
