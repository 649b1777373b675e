// fmgpu_internal.cuh -- shared definitions of the libfmgpu kernels and host code.
//
// Arithmetic contract of the FP64 path (compiled with -fmad=false, so the only
// fused multiply-adds are the explicit fma() calls):
//   row sum     acc = 0; for slot s ascending: acc = fma(a_s, x_{i+off_s}, acc)
//   residual    r_i = b_i - rowsum_i
//   reductions  DR4096: one 256-thread block per 4096-element chunk; thread t
//               owns chunk positions 2t+512m+u (m = 0..7, u = 0..1) in (m,u)
//               order; a warp butterfly then a butterfly over the 8 warp sums;
//               the last block folds the chunk sums (thread t: chunks
//               t, t+256, ... with plain adds) through the same tree.
// This fixed order makes the GPU results independent of scheduling and equal
// to a sequential restatement that follows the same order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/fmgpu.h"

namespace fmg {

constexpr int kBlock = 256;                 // threads per chunk block
constexpr int kChunk = 4096;                // elements per reduction chunk
constexpr int kPairsPerThread = kChunk / (kBlock * 2);
constexpr int kMaxLevels = 16;

// kernels launched by this library in this process (diagnostics)
extern std::atomic<long long> g_launches;

// device scalar slots of a grid (CG scalars, reduction results)
enum Scal {
  S_ALPHA = 0, S_BETA, S_LAM, S_NEGLAM, S_NEWALPHA, S_RATIO, S_RR, S_DOT, S_TMP,
  S_MFERR = 15,         // non-zero: a matrix-free operator kernel gave up waiting for a copy
  S_COUNT = 16
};

// epilogue of a chunked reduction, run by the last block on the folded value
enum Epi { EPI_STORE = 0, EPI_CG_LAMBDA = 1, EPI_CG_ALPHA = 2 };

struct Reduce {         // scratch of one chunked reduction
  double* part;         // >= number of chunks
  unsigned* counter;    // zero between reductions (reset by the last block)
  double* scal;         // grid scalar slots
  int epi;              // Epi
  int slot;             // destination slot for EPI_STORE
};

__device__ __forceinline__ long long clampi(long long j, long long N) {
  return j < 0 ? 0 : (j >= N ? N - 1 : j);
}

// Warp butterfly then butterfly over the 8 warp sums; the result is valid in
// thread 0.  smem must hold 8 doubles.  Blocks of 256 threads, 1D or (32, 8).
__device__ __forceinline__ double dr_fold256(double v, double* smem) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, o);
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;  // blocks of 256 threads, 1D or 2D
  const int warp = tid >> 5, lane = tid & 31;
  __syncthreads();  // smem may still be read by a previous fold
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  double w = 0.0;
  if (warp == 0) {
    w = lane < 8 ? smem[lane] : 0.0;
    w = w + __shfl_xor_sync(0xffffffffu, w, 4);
    w = w + __shfl_xor_sync(0xffffffffu, w, 2);
    w = w + __shfl_xor_sync(0xffffffffu, w, 1);
  }
  return w;
}

// Chunk partial -> global; the last block to finish folds all partials and
// applies the epilogue.  Must be called by all threads of a 256-thread block
// whose blockIdx.x is the chunk index and gridDim.x the chunk count.
__device__ __forceinline__ void dr_finish(double lane_sum, const Reduce& R, double* smem) {
  __shared__ bool is_last;
  double s = dr_fold256(lane_sum, smem);
  if (threadIdx.x == 0) {
    R.part[blockIdx.x] = s;
    __threadfence();
    unsigned done = atomicAdd(R.counter, 1u);
    is_last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double acc = 0.0;
  for (unsigned k = threadIdx.x; k < gridDim.x; k += kBlock) acc = acc + __ldcg(R.part + k);
  double tot = dr_fold256(acc, smem);
  if (threadIdx.x == 0) {
    double* sc = R.scal;
    switch (R.epi) {
      case EPI_CG_LAMBDA: {            // beta = (a,p); lam = alpha/beta
        double lam = sc[S_ALPHA] / tot;
        sc[S_BETA] = tot; sc[S_LAM] = lam; sc[S_NEGLAM] = -lam;
        break;
      }
      case EPI_CG_ALPHA: {             // new alpha = (q,r); ratio = new/alpha
        sc[S_NEWALPHA] = tot;
        sc[S_RATIO] = tot / sc[S_ALPHA];
        sc[S_ALPHA] = tot;
        break;
      }
      default: sc[R.slot] = tot;
    }
    *R.counter = 0u;
  }
}

inline unsigned nchunks(long long n) { return (unsigned)((n + kChunk - 1) / kChunk); }

}  // namespace fmg
