// sep.cuh — what the FP32 preconditioner's plane transforms share (sep.cu: the SIMT kernel, the line solve and
// the host side; sep_tc.cu: the tensor-core kernel).
#pragma once
#include "common.cuh"
#include "pcg.cuh"

#include <vector>

namespace tdgl {

__host__ __device__ inline int rup8(int n) { return (n + 7) & ~7; }
__host__ __device__ inline int rup16(int n) { return (n + 15) & ~15; }

// One component's planes for a mirror-halved transform: plane q of the input is in[in_base + q·in_ps + (in_j0 + j)
// + in_ld·(in_k0 + k)] (j < n1, k < n2), likewise the output.
struct HalfArgs {
  const float *in;
  long long in_base, in_ps;
  int in_ld, in_j0, in_k0;
  int n1, n2;                  // points (= modes) along the row axis (y) and the column axis (z)
  const float *W1, *W2;        // SIMT: the half blocks of each axis: [E | O], row-major (in, out), rows padded to 8
  const float *T1, *T2;        // tensor cores: the half blocks as MMA operand images (tc_images), null if absent
  void *out;
  long long out_base, out_ps;
  int out_ld, out_j0, out_k0;
  int nplanes;
};
// The three components (x, y and z links) in one launch.
struct HalfMulti {
  HalfArgs c[3];
  int ncomp;
  const int *done;             // skip when the PCG has converged (null: always run)
  int dot;                     // inverse only: fold r·z and r·z_old (DotFuse) over the written points
  DotFuse df;
};

// Tensor-core operand images of the mirror half blocks of a basis B(p, m) (point p, mode m) with np points:
// E = B(p, 2m) for p, m < hS = ⌈np/2⌉ and O = B(p, 2m+1) for p, m < hD = ⌊np/2⌋.  Four images [class a][hi, lo],
// each R = rup16(hS) rows (outputs) × K = rup8(hS) columns (inputs), zero outside the block, laid out K-major
// without swizzle: element (o, i) at float (o % 8)·4 + (o / 8)·8K + (i % 4) + (i / 4)·32.  Forward (points →
// modes): element (o, i) = H_a(i, o); inverse (modes → points): H_a(o, i).  hi is the value rounded to TF32, lo the
// remainder rounded to TF32 (umma::split_tf32).
void tc_images(int np, const double *B, int ldB, std::vector<float> &fwd, std::vector<float> &inv);

// The tensor-core transform (sep_tc.cu): whether it takes planes up to n1 × n2, and the launch (one direction for
// the three components; `err` counts blocks whose tensor-core waits ran out).
extern int g_sm_count;   // SMs of the device (set by sep_create)
bool half_tc_fits(int n1, int n2);
void half_tc(Ctx *ctx, const HalfMulti &M, bool fwd, long long *err);
void half_tc_init();

}  // namespace tdgl
