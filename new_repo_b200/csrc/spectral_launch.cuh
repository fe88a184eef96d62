// Launch helpers shared by the translation units of the spectral passes
// (spectral_xfwd.cu, spectral_xinv.cu, spectral_ypass.cu): occupancy and
// register queries with per-device caches, the rows-per-item choice of the
// x passes, the FFT lane counts and the supported lengths.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "spectral.cuh"

namespace les {

#define LES_LENGTHS(X) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768)

struct KernelLimits {
  int regs, max_threads;
};
int resident_ctas(const void* kern, int threads, size_t smem);
KernelLimits kernel_limits(const void* kern);
inline int kernel_regs(const void* kern) { return kernel_limits(kern).regs; }
int lanes(int n);
int pad_seqs(int nseq, int M);

inline constexpr int SMEM_CAP = 200 * 1024;
inline constexpr size_t SM_SMEM = 228 * 1024;  // shared memory per SM (1 KB of it reserved per CTA)

// Rows per work item of an x pass (256-thread CTAs, TL lanes per sequence,
// seq_per_row sequences per grid row): the count that keeps the most sequence
// slots of an SM busy -- resident CTAs (shared memory, registers) times the
// fraction of the 256 / TL slots of each pass that hold a sequence; on a tie
// the larger count (fewer items).
template <typename SmemFn>
inline int best_rows(const void* kern, int seq_per_row, int TL, SmemFn smem_for, int rmax = 32, double* best_score = nullptr,
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


// shared-memory limits of each family's kernels on the current device
template <typename T> void set_attrs_xfwd();
template <typename T> void set_attrs_xinv();
template <typename T> void set_attrs_ypass();

}  // namespace les
