// Instantiation and launch of the x forward passes (k_xfwd, k_xfwd_st) for
// every supported transform length.
#include "spectral_launch.cuh"

#include "launch.cuh"

namespace les {

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
void set_attrs_xfwd() {
#define XA(N)                                                                                       \
  LES_CUDA(cudaFuncSetAttribute(k_xfwd<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP)); \
  LES_CUDA(cudaFuncSetAttribute(k_xfwd_st<T, N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP)); \
  if constexpr (std::is_same<T, double>::value)                                                       \
    LES_CUDA(cudaFuncSetAttribute(k_xfwd_st<T, N, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP));
  LES_LENGTHS(XA)
#undef XA
}

template void launch_xfwd<float>(int, XFArgs<float>, cudaStream_t);
template void launch_xfwd<double>(int, XFArgs<double>, cudaStream_t);
template void set_attrs_xfwd<float>();
template void set_attrs_xfwd<double>();

}  // namespace les
