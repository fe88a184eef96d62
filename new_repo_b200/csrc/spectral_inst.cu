// Instantiation and launch of the spectral pass kernels for every supported
// transform length (2^a 3^b: the grid sizes 16..512 and their 3/2 padding).
#include "spectral.cuh"
#include "launch.cuh"

namespace les {

thread_local LaunchHook* g_hook = nullptr;

namespace {
constexpr int SMEM_CAP = 200 * 1024;

template <typename T>
int rows_per_cta(int nseq_per_row, int M) {
  // keep one ping-pong buffer at ~48 KB so two CTAs fit on an SM
  const int target = int((48 * 1024) / sizeof(cplx<T>));
  int R = target / (nseq_per_row * M);
  if (R < 1) R = 1;
  if (R > 32) R = 32;
  return R;
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

template <typename T>
void launch_xfwd(int NX, XFArgs<T> a, cudaStream_t st) {
  const int M = NX / 2;
  a.R = rows_per_cta<T>(a.nf, M);
  a.in_rstride = NX;
  const size_t smem = sizeof(cplx<T>) * (NX + 2 * (size_t)a.R * a.nf * M) + sizeof(T) * a.R * a.nf;
  if (smem > SMEM_CAP) throw CudaError(1, "xfwd: shared memory request too large");
  const int grid = ceil_div(a.nrows, a.R);
  if (grid == 0) return;
  static const int nin_of_op[] = {0, 9, 6, 10, 0};
  const int nin = (a.op == XF_SCALE || a.op == XF_PRESS) ? a.nf : nin_of_op[a.op];
  const size_t isz = (a.in_f32 ? sizeof(float) : sizeof(T));
  hook_before("xfwd", double(a.nrows) * NX * nin * isz + double(a.nrows) * a.nf * a.nk * sizeof(cplx<T>));
  switch (NX) {
#define XF_CASE(N) \
  case N: k_xfwd<T, N><<<grid, 256, smem, st>>>(a); break;
    LES_LENGTHS(XF_CASE)
#undef XF_CASE
    default:
      throw CudaError(1, "xfwd: unsupported transform length " + std::to_string(NX));
  }
  LES_CHECK_LAUNCH();
  hook_after();
}

template <typename T>
void launch_xinv(int NX, XIArgs<T> a, cudaStream_t st) {
  const int M = NX / 2;
  a.R = rows_per_cta<T>(a.nin, M);
  const size_t smem = sizeof(cplx<T>) * (NX + 2 * (size_t)a.R * a.nin * M);
  if (smem > SMEM_CAP) throw CudaError(1, "xinv: shared memory request too large");
  const int grid = ceil_div(a.nrows, a.R);
  if (grid == 0) return;
  {
    const size_t osz = (a.out_f32 ? sizeof(float) : sizeof(T));
    int nout = a.nin, rmw = 0;
    if (a.op == XI_CONV) { nout = 6; rmw = 3; }
    else if (a.op == XI_DIV) { nout = a.nin; rmw = 2 * a.nin; }
    else if (a.op == XI_LASD) nout = 2;
    else if (a.op == XI_WALL) nout = 7;
    hook_before("xinv", double(a.nrows) * a.nin * a.nk * sizeof(cplx<T>) + double(a.nrows) * NX * (nout + rmw) * osz);
  }
  switch (NX) {
#define XI_CASE(N) \
  case N: k_xinv<T, N><<<grid, 256, smem, st>>>(a); break;
    LES_LENGTHS(XI_CASE)
#undef XI_CASE
    default:
      throw CudaError(1, "xinv: unsupported transform length " + std::to_string(NX));
  }
  LES_CHECK_LAUNCH();
  hook_after();
}

template <typename T>
void launch_ypass(int NY, int NYO, YPArgs<T> a, int nplanes, int ngroups, cudaStream_t st) {
  const int nmax = std::max(a.nin * (NY + 1), a.nout * (NYO + 1));
  const size_t per_col = 2 * (size_t)nmax * sizeof(cplx<T>);
  int lc = 4;  // up to 16 columns per CTA
  while (lc > 0 && ((size_t(1) << lc) * per_col > 96 * 1024 || (1 << lc) > 2 * a.ncols)) --lc;
  a.lc = lc;
  a.C = 1 << lc;
  const size_t smem = sizeof(cplx<T>) * (NY + NYO) + (size_t)a.C * per_col;
  if (smem > SMEM_CAP) throw CudaError(1, "ypass: shared memory request too large");
  dim3 grid(ceil_div(a.ncols, a.C), nplanes, ngroups);
  if (grid.x == 0 || nplanes == 0 || ngroups == 0) return;
  const int key = NY * 10000 + NYO;
  hook_before("ypass", double(nplanes) * ngroups * a.ncols * sizeof(cplx<T>) *
                           (double(a.op == YP_PGRAD ? 1 : a.nin) * NY + double(a.nout) * NYO));
  switch (key) {
#define YP_CASE(A, B) \
  case A * 10000 + B: k_ypass<T, A, B><<<grid, 256, smem, st>>>(a); break;
    YP_CASE(16, 16) YP_CASE(32, 32) YP_CASE(64, 64) YP_CASE(128, 128) YP_CASE(256, 256) YP_CASE(512, 512)
    YP_CASE(16, 24) YP_CASE(32, 48) YP_CASE(64, 96) YP_CASE(128, 192) YP_CASE(256, 384) YP_CASE(512, 768)
    YP_CASE(24, 16) YP_CASE(48, 32) YP_CASE(96, 64) YP_CASE(192, 128) YP_CASE(384, 256) YP_CASE(768, 512)
#undef YP_CASE
    default:
      throw CudaError(1, "ypass: unsupported length pair " + std::to_string(NY) + "->" + std::to_string(NYO));
  }
  LES_CHECK_LAUNCH();
  hook_after();
}

template <typename T>
static void set_attrs() {
#define XA(N)                                                                                       \
  LES_CUDA(cudaFuncSetAttribute(k_xfwd<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP)); \
  LES_CUDA(cudaFuncSetAttribute(k_xinv<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP));
  LES_LENGTHS(XA)
#undef XA
#define YA(A, B) \
  LES_CUDA(cudaFuncSetAttribute(k_ypass<T, A, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP));
  YA(16, 16) YA(32, 32) YA(64, 64) YA(128, 128) YA(256, 256) YA(512, 512)
  YA(16, 24) YA(32, 48) YA(64, 96) YA(128, 192) YA(256, 384) YA(512, 768)
  YA(24, 16) YA(48, 32) YA(96, 64) YA(192, 128) YA(384, 256) YA(768, 512)
#undef YA
}

void init_spectral_attributes() {
  set_attrs<float>();
  set_attrs<double>();
}

template void launch_xfwd<float>(int, XFArgs<float>, cudaStream_t);
template void launch_xfwd<double>(int, XFArgs<double>, cudaStream_t);
template void launch_xinv<float>(int, XIArgs<float>, cudaStream_t);
template void launch_xinv<double>(int, XIArgs<double>, cudaStream_t);
template void launch_ypass<float>(int, int, YPArgs<float>, int, int, cudaStream_t);
template void launch_ypass<double>(int, int, YPArgs<double>, int, int, cudaStream_t);

}  // namespace les
