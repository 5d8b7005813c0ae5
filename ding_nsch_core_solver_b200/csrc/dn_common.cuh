// dn_common.cuh -- shared device-side types and helpers of libdn_cuda (sm_100a).
//
// Fields live on the device in the reference's Field2D layout (src/core/base/field.hpp:9-36): FP64,
// (nx'+2g) x (ny'+2g), j contiguous.  Krylov vectors are compact, row = i*ny + j (the reference's
// row_index, e.g. pressure.cpp:131).  The library is compiled with --fmad=false so that expressions
// written in the reference's operand order round exactly like the reference; hot loops that want a
// fused multiply-add ask for it explicitly.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dn_cuda.h"

namespace dn {

constexpr int kWarp = 32;
constexpr int kBlock = 256;  // threads per CTA of the persistent Krylov kernels and the field kernels

// Error codes written by device code into the handle's status word.
enum DevStatus : int {
  kDevOk = 0,
  kDevTimeout = 1,
  kDevPcgBreakdownRz0 = 2,   // "pcg preconditioner breakdown: non-positive r^T M^{-1} r"
  kDevPcgBreakdownPap = 3,   // "pcg breakdown: p^T A p is invalid"
  kDevPcgBreakdownRz = 4,    // "pcg preconditioner breakdown: non-positive new r^T M^{-1} r"
  kDevBicgRho = 5,           // "bicgstab breakdown: invalid rho"
  kDevBicgRhatV = 6,         // "bicgstab breakdown: invalid r_hat^T A M^{-1} p"
  kDevBicgTT = 7,            // "bicgstab breakdown: invalid t^T t"
  kDevBicgOmega = 8,         // "bicgstab breakdown: invalid omega"
  kDevFactorFailed = 9,      // incomplete factorization hit the pivot floor
  kDevJacobiDiverged = 10,   // "Jacobi pressure solve diverged"
};

enum PrecKind { kPrecDiag = 0, kPrecLDLT = 1, kPrecICC = 2 };

// Entry of a kernel launched with programmatic stream serialization (launch_pdl on the host): wait until the
// grids it depends on have completed and their memory is visible, then let the next grid of the stream be
// launched (its blocks wait here the same way), so that a launch overlaps its predecessor's tail instead of
// following it.  Without that launch attribute both instructions return at once.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded spin: ~2^22 polls with a short sleep, i.e. well under a few seconds, then give up.
constexpr long long kSpinLimit = 1ll << 22;

// The status buffer of a handle (or of a static solve) is [status, pad, poll limit (long long)]: every
// bounded wait gives up after that many polls (kSpinLimit when the limit is 0 or negative).
__device__ __forceinline__ long long spin_limit(const volatile int *status) {
  const long long v = *(const volatile long long *)(status + 2);
  return v > 0 ? v : kSpinLimit;
}

struct Grid {
  int nx, ny, g;
  int px, py;  // periodic flags
  double dx, dy;
};

struct BCSide {
  int type;  // dn_bc_type, already resolved by the effective_*_bc rules (operators.cpp:36-112)
  double value;
};

struct BCSet {
  BCSide p[4], u[4], v[4];
};

// A ghosted field view.
struct Fv {
  double *d;
  int nx, ny, g;  // logical interior extent (nx' x ny')
  __host__ __device__ __forceinline__ int pitch() const { return ny + 2 * g; }
  __host__ __device__ __forceinline__ double &at(int i, int j) const {
    return d[(size_t)(i + g) * (size_t)(ny + 2 * g) + (size_t)(j + g)];
  }
  __host__ __device__ __forceinline__ size_t size() const { return (size_t)(nx + 2 * g) * (size_t)(ny + 2 * g); }
};

// std::max / std::min as the reference calls them (a NaN in the first argument passes through), where the
// reference clamps values that can be NaN -- norms, pivots, denominators -- so that a non-finite state fails
// the same checks on the device as in the reference.  CUDA's fmax/fmin return the other argument instead.
__host__ __device__ __forceinline__ double max_ref(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ double min_ref(double a, double b) { return (b < a) ? b : a; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sums K values over the CTA; result valid in every thread.  `sh` holds K*kWarps doubles.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double *sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) sh[k * 32 + wid] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += sh[k * 32 + w];
    v[k] = s;
  }
  __syncthreads();
}

// Grid-wide barrier for persistent (co-resident, cooperatively launched) kernels.  Thread 0 of each CTA
// arrives on a counter and spins on a generation word with a bounded number of polls; on timeout it
// records kDevTimeout and everybody returns at the next check of *status.
struct GridBarrier {
  unsigned int *count;
  volatile unsigned int *gen;
  volatile int *status;
  unsigned int nblocks;

  __device__ __forceinline__ bool sync() const {
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned int my_gen = *gen;
      __threadfence();
      const unsigned int arrived = atomicAdd(count, 1u);
      if (arrived == nblocks - 1) {
        *count = 0u;
        __threadfence();
        atomicAdd((unsigned int *)gen, 1u);
      } else {
        long long spins = 0;
        while (*gen == my_gen) {
          ++spins;
          if (spins > spin_limit(status) || ((spins & 1023) == 0 && *status != kDevOk)) {
            atomicCAS((int *)status, kDevOk, kDevTimeout);
            break;
          }
          if (spins > 64) __nanosleep(32);
        }
      }
      __threadfence();
    }
    __syncthreads();
    return *status == kDevOk;
  }
};

// Deterministic grid reduction of K partial sums: each CTA writes its partials, crosses a barrier, then
// every CTA re-adds all partials in the same order, so every CTA holds bit-identical totals.  `parity`
// alternates between two partial buffers (each kMaxBlocks*8 doubles) so that a fast CTA writing the next
// reduction never overwrites partials a slow CTA is still reading.
constexpr int kMaxBlocks = 1024;
template <int K>
__device__ __forceinline__ bool grid_sum(double (&v)[K], double *partials_base, int &parity, double *sh,
                                         const GridBarrier &bar) {
  static_assert(K <= 8, "at most 8 values per grid reduction");
  double *partials = partials_base + (size_t)parity * kMaxBlocks * 8;
  parity ^= 1;
  block_sum<K>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) partials[(size_t)blockIdx.x * K + k] = v[k];
  }
  if (!bar.sync()) return false;
  // warp 0 re-adds the partials in a fixed order (lane-strided, then a fixed butterfly; lane 0's value is
  // used), so every CTA obtains the same bits.
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (unsigned int b = threadIdx.x; b < bar.nblocks; b += 32) s += __ldcg(&partials[(size_t)b * K + k]);
      s = warp_sum(s);
      if (threadIdx.x == 0) sh[k] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = sh[k];
  __syncthreads();
  return true;
}

}  // namespace dn
