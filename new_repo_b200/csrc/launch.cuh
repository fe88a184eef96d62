// Host-side launchers of the spectral pass kernels (spectral_inst.cu).
#pragma once
#include "spectral.cuh"

#include <string>

namespace les {

// Observer of every kernel launch: the solver counts launches and, when
// profiling, brackets each one with CUDA events on its stream.  bytes is the
// launch's compulsory (algorithmic) HBM traffic: each input read once, each
// output written once.
struct LaunchHook {
  virtual void before(const char* kind, double bytes) = 0;
  virtual void after() = 0;
  virtual ~LaunchHook() = default;
};
extern thread_local LaunchHook* g_hook;

inline void hook_before(const char* kind, double bytes) {
  if (g_hook) g_hook->before(kind, bytes);
}
inline void hook_after() {
  if (g_hook) g_hook->after();
}

bool supported_length(int n);
void init_spectral_attributes();

template <typename T>
void launch_xfwd(int NX, XFArgs<T> a, cudaStream_t st);
template <typename T>
void launch_xinv(int NX, XIArgs<T> a, cudaStream_t st);
template <typename T>
void launch_ypass(int NY, int NYO, YPArgs<T> a, int nplanes, int ngroups, cudaStream_t st);

}  // namespace les
