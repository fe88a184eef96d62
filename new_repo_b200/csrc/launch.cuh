// Host-side launchers of the spectral pass kernels (spectral_inst.cu).
#pragma once
#include "spectral.cuh"

namespace les {

bool supported_length(int n);
void init_spectral_attributes();

template <typename T>
void launch_xfwd(int NX, XFArgs<T> a, cudaStream_t st);
template <typename T>
void launch_xinv(int NX, XIArgs<T> a, cudaStream_t st);
template <typename T>
void launch_ypass(int NY, int NYO, YPArgs<T> a, int nplanes, int ngroups, cudaStream_t st);

}  // namespace les
