// pcg.cuh — the device scalars of the PCG field solve and its deterministic reductions, shared by the PCG kernels
// (pcg.cu) and by the preconditioner's inverse transform (sep.cu), which folds the PCG's r·z and r·z_old into its
// epilogue.
#pragma once

#include "common.cuh"

namespace tdgl {

enum { SC_BB = 0, SC_RR, SC_RZ, SC_PAP, SC_ALPHA, SC_BETA, SC_RZ2, SC_RZOLD, SC_TOL2, SC_N };
// IC_CNT: blocks done with the current reduction; IC_LAUNCHED: iterations launched in the device-driven loop;
// IC_XDONE: the iterations (counted as IC_ITERS counts them) whose x update is done; IC_XCNT: blocks done with it
enum { IC_DONE = 0, IC_ITERS, IC_CNT, IC_LAUNCHED, IC_XDONE, IC_XCNT, IC_N };
// the solve statistics, accumulated on the device: total iterations, the last solve's, solves at maxit, loop turns,
// blocks of the tensor-core preconditioner transform whose waits ran out
enum { ST_TOTAL = 0, ST_LAST, ST_NOCONV, ST_TURNS, ST_TCWAIT, ST_N };

namespace {

__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  v = 0.0;
  if (w == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// The reductions.  mode 0: b·b; 1: r·r of the initial residual; 2: r·z (initial); 3: pAp → α, counting the
// iteration; 5: r·r → convergence flag; 4: (r·z, r·z_old) → β, rz ← r·z (flexible when f32).  (a, b) are the
// two folded sums.
__device__ void set_scalars(double a, double b, double *sc, int *ic, int mode, int flexible, double tol) {
  switch (mode) {
    case 0: sc[SC_BB] = a; break;
    case 1:   // the initial residual: already converged (with ‖b‖ = 0 too) ends the solve before its loop
      sc[SC_RR] = a;
      if (sqrt(a) <= tol * sqrt(sc[SC_BB])) ic[IC_DONE] = 1;
      break;
    case 2: sc[SC_RZ] = a; break;
    case 3: sc[SC_PAP] = a; sc[SC_ALPHA] = sc[SC_RZ] / a; ic[IC_ITERS] += 1; break;
    case 5: {
      sc[SC_RR] = a;
      if (sqrt(a) <= tol * sqrt(sc[SC_BB])) ic[IC_DONE] = 1;
      break;
    }
    case 4: {
      sc[SC_RZ2] = a;
      sc[SC_RZOLD] = b;
      sc[SC_BETA] = flexible ? (a - b) / sc[SC_RZ] : a / sc[SC_RZ];
      sc[SC_RZ] = a;
      break;
    }
  }
}

// Called by every block of a reducing kernel after thread 0 has stored the block's partials: the last block to
// arrive folds all partials in index order (the same order whichever block is last) and sets the scalars of
// `mode`, so the reduction needs no second kernel.
struct Fold {
  int mode = -1, flexible = 0;   // mode < 0: no fold
  double tol = 0.0;
  double *sc = nullptr;
  int *ic = nullptr;
  const double *bpart = nullptr;   // the second sum's partials from another kernel (nbb of them), if not null
  int nbb = 0;
};
__device__ void fold_last(const Fold &F, const double *part, double *sh) {
  if (F.mode < 0) return;
  __shared__ int last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&F.ic[IC_CNT], 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int nb = gridDim.x;
  double a = 0.0, b = 0.0;
  for (int q = threadIdx.x; q < nb; q += blockDim.x) a += __ldcg(part + q);
  if (F.bpart)
    for (int q = threadIdx.x; q < F.nbb; q += blockDim.x) b += __ldcg(F.bpart + q);
  else
    for (int q = threadIdx.x; q < nb; q += blockDim.x) b += __ldcg(part + nb + q);
  a = block_sum(a, sh);
  __syncthreads();
  b = block_sum(b, sh);
  if (threadIdx.x == 0) {
    set_scalars(a, b, F.sc, F.ic, F.mode, F.flexible, F.tol);
    F.ic[IC_CNT] = 0;
  }
}

}  // namespace

// r·z and r·z_old of the PCG folded into the preconditioner's inverse transform (which writes z): the transform reads
// r and z_old where it writes z and reduces the two sums as k_dot2 does (mode 4: β and rz).
struct DotFuse {
  const double *r[3] = {nullptr, nullptr, nullptr};
  const double *zold[3] = {nullptr, nullptr, nullptr};
  double *part = nullptr;
  Fold F;
};

}  // namespace tdgl
