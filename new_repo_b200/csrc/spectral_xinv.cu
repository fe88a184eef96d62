// Instantiation and launch of the x inverse pass (k_xinv) for every
// supported transform length.
#include "spectral_launch.cuh"

#include "launch.cuh"

namespace les {

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
  // bulk staging: one cp.async.bulk per staged row needs 16-byte aligned
  // rows in global memory (pitch and plane stride) and in the stages (stage
  // base and row stride); the kernel checks every row's addresses again and
  // copies a row that fails with plain loads
  {
    const size_t cs = sizeof(cplx<T>);
    a.bulk = ((cs * a.ipitch) % 16 == 0 && (cs * a.in_pstride) % 16 == 0 && (cs * a.nks) % 16 == 0 &&
              (cs * (NX + twm_len(M, true))) % 16 == 0 && a.nk * cs >= 16)
                 ? 1
                 : 0;
  }
  auto smem_nb = [&](int R, int nb) {
    return sizeof(cplx<T>) * (NX + twm_len(M, true) + nb * (((size_t)stage_rows(R) * a.nks + 1) & ~size_t(1)) +
                              (a.merged ? 0 : (size_t)pad_seqs(R * a.nin, M) * SL)) +
           2 * sizeof(int) * R + (a.nstage ? sizeof(T) * (a.nk + 2) : 0) + (a.bulk ? 2 * sizeof(uint64_t) + 8 : 0);
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


template <typename T>
void set_attrs_xinv() {
#define XA(N) LES_CUDA(cudaFuncSetAttribute(k_xinv<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP));
  LES_LENGTHS(XA)
#undef XA
}

template void launch_xinv<float>(int, XIArgs<float>, cudaStream_t);
template void launch_xinv<double>(int, XIArgs<double>, cudaStream_t);
template void set_attrs_xinv<float>();
template void set_attrs_xinv<double>();

}  // namespace les
