// pcg.cu — the insulating-padding field solve on the device (gtdgl/src/implicit.jl:106-446).
//
// (D + aK)Δ = φₑ − θ on the coupled links by preconditioned conjugate gradients, the separable inverse of
// (I + aK) as the preconditioner (in FP32 with pcg_f32, then with the flexible β = r·(z − z_old)/rz_old), the
// warm start and the extrapolated first guess 2xₙ − xₙ₋₁ of pcg_fast (_implicit_curl_fast! :376-446), the
// zero-source update (_pcg_zero_update! :251-271), and φ = θ + (φₑ − θ)/D on the decoupled links.
//
// Iterates, residuals and dot products are FP64.  Every vector is a plane-major node-shaped array per component
// (sep.cu), zero outside the ranges, so the vector kernels are flat loops.  A·p computes the curl of p on the fly
// (no plaquette arrays).  Dot products are deterministic: a fixed grid of block partial sums reduced by one block
// in a fixed order.  The loop runs on the device: α, β and the convergence test (‖r‖ ≤ tol·‖b‖) are computed by
// the reduction kernels, and once the test passes every later kernel of the iteration returns at once; the host
// launches iterations in batches and reads the flag between batches only.
#include <algorithm>
#include <climits>
#include <cmath>

#include "common.cuh"
#include "pcg.cuh"

namespace tdgl {

Rng sep_range(const Geo &g, int ax);
void to_planes(Ctx *ctx, const double *const *a, const double *const *b, double *const *out);
void from_planes(Ctx *ctx, const double *const *in, const double *const *base, double *const *out);

static const int RED_BLOCKS = 740;   // at most 5 × 148 SMs (the stencil: five blocks per SM, launch bounds below)
static const int STR_BLOCKS = 1184;  // at most 8 × 148 SMs: full occupancy for the streaming kernels
static const int BATCH = 4;          // iterations between two reads of the convergence flag

struct PcgDev {
  double *P[3] = {}, *Q[3] = {}, *x[3] = {}, *r[3] = {}, *z[3] = {}, *b[3] = {}, *xprev[3] = {}, *zold[3] = {}, *Dp[3] = {};
  double *part = nullptr;                       // STR_BLOCKS × 2 partial sums
  double *part2 = nullptr;                      // xblocks partial sums of r·z_old (k_dot_part)
  cudaStream_t side = nullptr;                  // the x update and r·z_old beside the preconditioner
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int xblocks = 1;                              // grid of the kernels beside the preconditioner (2 per SM at most)
  double *sc = nullptr;                         // device scalars SC_*
  int *ic = nullptr;                            // device flags IC_*
  double *host_sc = nullptr;                    // pinned copies
  int *host_ic = nullptr;
  long long *stat = nullptr, *host_stat = nullptr;   // ST_* (device, pinned copy)
  long long noconv_seen = 0;                    // ST_NOCONV at the last status read
  long long tcwait_seen = 0;                    // ST_TCWAIT at the last status read
  bool warm = false, have2 = false;
  long long n;                                  // node count (per component array)
  int sblocks = STR_BLOCKS, ablocks = RED_BLOCKS;   // grids of the streaming kernels and of A·p for this size
};

namespace {
const int BS = 256;

struct Vec3 {
  double *p[3];
};
struct CVec3 {
  const double *p[3];
};
struct F3 {                  // FP32 copy of a vector (p[0] null: none)
  float *p[3];
};

// partial sums of a·b and a·c (c may be null) over the three component arrays
__global__ void __launch_bounds__(256, 8) k_dot2(CVec3 a, CVec3 b, CVec3 c, int use_c, long long n, double *part, const int *ic, Fold F) {
  if (ic && ic[IC_DONE]) return;
  __shared__ double sh[32];
  double s1 = 0.0, s2 = 0.0;
  // unrolled: the loads of several entries in flight per thread (the sums keep their order)
  for (int cc = 0; cc < 3; cc++)
#pragma unroll 2
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
      const double av = a.p[cc][t];
      s1 += av * b.p[cc][t];
      if (use_c) s2 += av * c.p[cc][t];
    }
  double r1 = block_sum(s1, sh);
  __syncthreads();
  double r2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = r1;
    part[gridDim.x + blockIdx.x] = r2;
  }
  __syncthreads();
  fold_last(F, part, sh);
}

// Q = D P + a curl curl P on the ranges (implicit.jl:212-235), the plaquette fields computed on the fly, with the
// partial sums of P·Q.  One thread per node of the box i ∈ 2..Nx, j ∈ 2..Ny, k ∈ 2..Nz (plane-major order; node
// counts fit 32 bits, checked at set-up).
struct ApplyArgs {
  const double *P[3], *D[3];
  double *Q[3];
  double sxy, sxz, syx, syz, szx, szy, dx, dy, dz, iyz, izx, ixy;
  int Nx, Ny, Nz, n2, n3;
  double *part;
  const int *ic;
  Fold F;
};

__global__ void __launch_bounds__(256, 5) k_apply(ApplyArgs A) {
  if (A.ic && A.ic[IC_DONE]) return;
  __shared__ double sh[32];
  const int Nx = A.Nx, Ny = A.Ny, Nz = A.Nz;
  const long long sj = 1, sk = A.n2, si = (long long)A.n2 * A.n3;
  const int nj = Ny - 1, nk = Nz - 1, ni = Nx - 1;
  // distinct arrays (P and D read, Q written): the compiler may keep several nodes' loads in flight, which this
  // latency-bound kernel needs (the stores to Q cannot alias the loads of P)
  const double *__restrict__ px = A.P[0], *__restrict__ py = A.P[1], *__restrict__ pz = A.P[2];
  const double *__restrict__ Dx = A.D[0], *__restrict__ Dy = A.D[1], *__restrict__ Dz = A.D[2];
  double *__restrict__ Qx = A.Q[0], *__restrict__ Qy = A.Q[1], *__restrict__ Qz = A.Q[2];
  // the plaquette areas as reciprocals: nine FP64 divisions per node were half of this kernel's instructions (the
  // operator differs from the reference's division by at most an ulp per plaquette field)
  const double iyz = A.iyz, izx = A.izx, ixy = A.ixy;
  auto at = [&](int i, int j, int k) { return (long long)(j - 1) + A.n2 * ((long long)(k - 1) + (long long)A.n3 * (i - 1)); };
  auto hx = [&](int i, int j, int k) -> double {
    if (k < 2 || k > Nz - 1 || j < 2 || j > Ny - 1 || i < 2 || i > Nx) return 0.0;
    const long long o = at(i, j, k);
    return ((pz[o + sj] - pz[o]) - py[o + sk] + py[o]) * iyz;
  };
  auto hy = [&](int i, int j, int k) -> double {
    if (k < 2 || k > Nz - 1 || j < 2 || j > Ny || i < 2 || i > Nx - 1) return 0.0;
    const long long o = at(i, j, k);
    return ((px[o + sk] - px[o]) - pz[o + si] + pz[o]) * izx;
  };
  auto hz = [&](int i, int j, int k) -> double {
    if (k < 2 || k > Nz || j < 2 || j > Ny - 1 || i < 2 || i > Nx - 1) return 0.0;
    const long long o = at(i, j, k);
    return ((py[o + si] - py[o]) - px[o + sj] + px[o]) * ixy;
  };
  double s = 0.0;
  const int n = nj * nk * ni;
#pragma unroll 2
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int j = 2 + t % nj, u = t / nj;
    const int k = 2 + u % nk, i = 2 + u / nk;
    const long long o = at(i, j, k);
    const double hx0 = hx(i, j, k), hy0 = hy(i, j, k), hz0 = hz(i, j, k);
    if (i <= Nx - 1) {
      const double q = Dx[o] * px[o] + A.sxy * (hz0 - hz(i, j - 1, k)) - A.sxz * (hy0 - hy(i, j, k - 1));
      Qx[o] = q;
      s += px[o] * q;
    }
    if (j <= Ny - 1) {
      const double q = Dy[o] * py[o] + A.syz * (hx0 - hx(i, j, k - 1)) - A.syx * (hz0 - hz(i - 1, j, k));
      Qy[o] = q;
      s += py[o] * q;
    }
    if (k <= Nz - 1) {
      const double q = Dz[o] * pz[o] + A.szx * (hy0 - hy(i - 1, j, k)) - A.szy * (hx0 - hx(i, j - 1, k));
      Qz[o] = q;
      s += pz[o] * q;
    }
  }
  const double r = block_sum(s, sh);
  if (threadIdx.x == 0) {
    A.part[blockIdx.x] = r;
    A.part[gridDim.x + blockIdx.x] = 0.0;
  }
  __syncthreads();
  fold_last(A.F, A.part, sh);
}

// r = b − Q (and its FP32 copy when given), partial r·r
__global__ void __launch_bounds__(256, 8) k_residual(Vec3 r, CVec3 b, CVec3 Q, long long n, double *part, F3 r32, Fold F) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int c = 0; c < 3; c++)
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
      const double v = b.p[c][t] - Q.p[c][t];
      r.p[c][t] = v;
      if (r32.p[0]) r32.p[c][t] = (float)v;
      s += v * v;
    }
  const double rr = block_sum(s, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rr;
    part[gridDim.x + blockIdx.x] = 0.0;
  }
  __syncthreads();
  fold_last(F, part, sh);
}

// r −= αQ (and r's FP32 copy when given), partial r·r; the convergence test folded in (x: k_update_x)
__global__ void __launch_bounds__(256, 8) k_update(Vec3 r, CVec3 Q, long long n, const double *sc, double *part, const int *ic,
                         F3 r32, Fold F) {
  if (ic[IC_DONE]) return;
  __shared__ double sh[32];
  const double alpha = sc[SC_ALPHA];
  double s = 0.0;
  for (int c = 0; c < 3; c++)
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
      const double v = r.p[c][t] - alpha * Q.p[c][t];
      r.p[c][t] = v;
      if (r32.p[0]) r32.p[c][t] = (float)v;
      s += v * v;
    }
  const double rr = block_sum(s, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rr;
    part[gridDim.x + blockIdx.x] = 0.0;
  }
  __syncthreads();
  fold_last(F, part, sh);
}

// x += αP once per iteration that ran A·p (IC_ITERS counts those; IC_XDONE is where the x updates stand), so also
// in the iteration whose r update met the tolerance and set IC_DONE.  It may run beside the preconditioner (on
// another stream): nothing there changes IC_ITERS, α, P or x.  Four entries per thread in flight.
__global__ void __launch_bounds__(256) k_update_x(Vec3 x, CVec3 P, long long n, const double *sc, int *ic) {
  __shared__ int run, last;
  const int it = ic[IC_ITERS];
  if (threadIdx.x == 0) run = ic[IC_XDONE] != it;
  __syncthreads();
  if (!run) return;
  const double alpha = sc[SC_ALPHA];
  const long long S = (long long)gridDim.x * blockDim.x;
  for (int c = 0; c < 3; c++) {
    double *__restrict__ xp = x.p[c];
    const double *__restrict__ pp = P.p[c];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; t + 3 * S < n; t += 4 * S) {
      double xv[4], pv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        xv[u] = xp[t + u * S];
        pv[u] = pp[t + u * S];
      }
#pragma unroll
      for (int u = 0; u < 4; u++) xp[t + u * S] = xv[u] + alpha * pv[u];
    }
    for (; t < n; t += S) xp[t] += alpha * pp[t];
  }
  if (threadIdx.x == 0) {   // the last block to finish records the update (every block has read IC_XDONE by then)
    __threadfence();
    last = atomicAdd(&ic[IC_XCNT], 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    ic[IC_XDONE] = it;
    ic[IC_XCNT] = 0;
  }
}

// the block partial sums of a·b into part[block], no fold (another kernel's fold takes them as its second sum)
__global__ void __launch_bounds__(256) k_dot_part(CVec3 a, CVec3 b, long long n, double *part, const int *ic) {
  if (ic[IC_DONE]) return;
  __shared__ double sh[32];
  double s = 0.0;
  for (int cc = 0; cc < 3; cc++)
#pragma unroll 2
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
      s += a.p[cc][t] * b.p[cc][t];
  const double r = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// P = z + βP (first: P = z)
__global__ void __launch_bounds__(256, 8) k_pdir(Vec3 P, CVec3 z, long long n, const double *sc, int first, const int *ic) {
  if (ic && ic[IC_DONE]) return;
  const double beta = first ? 0.0 : sc[SC_BETA];
  for (int c = 0; c < 3; c++)
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
      const double zv = z.p[c][t];
      P.p[c][t] = first ? zv : zv + beta * P.p[c][t];
    }
}

// x ← 2x − xprev, xprev ← x (pcg_fast's extrapolated guess, implicit.jl:394-398)
__global__ void __launch_bounds__(256, 8) k_extrap(Vec3 x, Vec3 xp, long long n) {
  for (int c = 0; c < 3; c++)   // per component (no 64-bit division of the flat index)
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += (long long)gridDim.x * blockDim.x) {
      const double v = x.p[c][u];
      x.p[c][u] = 2 * v - xp.p[c][u];
      xp.p[c][u] = v;
    }
}

// The first guess of a settled solve, decided on the device (implicit.jl:381-398 and _pcg_zero_update! :251-271):
// with ‖b‖ = 0 the solution is x = 0 (the extrapolation keeps xₙ as xₙ₋₁) and the solve is done; otherwise, with
// the extrapolated guess, x ← 2xₙ − xₙ₋₁ and xₙ₋₁ ← xₙ.
__global__ void __launch_bounds__(256, 8) k_guess(Vec3 x, Vec3 xp, long long n, const double *sc, int *ic, int extrap) {
  const bool zero = sc[SC_BB] == 0.0;
  if (zero && blockIdx.x == 0 && threadIdx.x == 0) ic[IC_DONE] = 1;
  if (!zero && !extrap) return;
  for (int c = 0; c < 3; c++)   // per component (no 64-bit division of the flat index)
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += (long long)gridDim.x * blockDim.x) {
      const double v = x.p[c][u];
      const double w = zero ? 0.0 : 2 * v - xp.p[c][u];   // xₙ₋₁ read before it becomes xₙ
      if (extrap) xp.p[c][u] = v;
      x.p[c][u] = w;
    }
}

// the loop's condition in a captured step: go on while the solve is not done and maxit is not reached
__global__ void k_loop_enter(cudaGraphConditionalHandle h, const int *ic, int maxit) {
  if (threadIdx.x == 0) cudaGraphSetConditional(h, (!ic[IC_DONE] && ic[IC_LAUNCHED] < maxit) ? 1u : 0u);
}
__global__ void k_loop_turn(cudaGraphConditionalHandle h, int *ic, long long *stat, int batch, int maxit) {
  if (threadIdx.x == 0) {
    ic[IC_LAUNCHED] += batch;
    stat[ST_TURNS] += 1;
    cudaGraphSetConditional(h, (!ic[IC_DONE] && ic[IC_LAUNCHED] < maxit) ? 1u : 0u);
  }
}

// the statistics of one solve (done: the zero-source update, which has no iterations)
__global__ void k_finish(const int *ic, long long *stat, int done) {
  if (threadIdx.x == 0) {
    const int it = ic[IC_ITERS];
    stat[ST_TOTAL] += it;
    stat[ST_LAST] = it;
    if (!done && !ic[IC_DONE]) stat[ST_NOCONV] += 1;
  }
}

CVec3 cv(double *const *p) {
  CVec3 v;
  for (int c = 0; c < 3; c++) v.p[c] = p[c];
  return v;
}
Vec3 vv(double *const *p) {
  Vec3 v;
  for (int c = 0; c < 3; c++) v.p[c] = p[c];
  return v;
}

Fold fold(Ctx *ctx, int mode, int flexible = 0) {
  Fold F;
  F.mode = mode;
  F.flexible = flexible;
  F.tol = ctx->P.pcg_tol;
  F.sc = ctx->pcg->sc;
  F.ic = ctx->pcg->ic;
  return F;
}
// a·b (and a·c) folded into the scalars of `mode`
void dot2(Ctx *ctx, double *const *a, double *const *b, double *const *c, bool gated, int mode, int flexible = 0) {
  PcgDev *S = ctx->pcg;
  TDGL_LAUNCH(ctx, K_PCG_DOT, (c ? 24.0 : 16.0) * 3 * S->n, k_dot2, S->sblocks, BS, 0, cv(a), cv(b), cv(c ? c : b), c ? 1 : 0, S->n,
              S->part, gated ? S->ic : nullptr, fold(ctx, mode, flexible));
}
void read_back(Ctx *ctx) {
  PcgDev *S = ctx->pcg;
  cudaMemcpyAsync(S->host_sc, S->sc, SC_N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(S->host_ic, S->ic, IC_N * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
}

void apply_A(Ctx *ctx, bool gated, int mode) {
  PcgDev *S = ctx->pcg;
  const Geo &g = ctx->g;
  const tdgl_params &Pp = ctx->P;
  ApplyArgs A;
  for (int c = 0; c < 3; c++) {
    A.P[c] = S->P[c];
    A.D[c] = S->Dp[c];
    A.Q[c] = S->Q[c];
  }
  A.sxy = Pp.sxy; A.sxz = Pp.sxz; A.syx = Pp.syx; A.syz = Pp.syz; A.szx = Pp.szx; A.szy = Pp.szy;
  A.dx = g.dx; A.dy = g.dy; A.dz = g.dz;
  A.iyz = 1.0 / (g.dy * g.dz); A.izx = 1.0 / (g.dz * g.dx); A.ixy = 1.0 / (g.dx * g.dy);
  A.Nx = g.Nx; A.Ny = g.Ny; A.Nz = g.Nz; A.n2 = g.Ny + 1; A.n3 = g.Nz + 1;
  A.part = S->part;
  A.ic = gated ? S->ic : nullptr;
  A.F = fold(ctx, mode);
  const double nbox = (double)(g.Nx - 1) * (g.Ny - 1) * (g.Nz - 1);
  TDGL_LAUNCH(ctx, K_PCG_Q, 72.0 * nbox, k_apply, S->ablocks, BS, 0, A);
}

void pdir(Ctx *ctx, double *const *z, int first, bool gated) {
  PcgDev *S = ctx->pcg;
  TDGL_LAUNCH(ctx, K_PCG_DIR, (first ? 16.0 : 24.0) * 3 * S->n, k_pdir, S->sblocks, BS, 0, vv(S->P), cv(z), S->n, S->sc,
              first, gated ? S->ic : nullptr);
}

int copy3(Ctx *ctx, double *const *dst, double *const *src) {
  for (int c = 0; c < 3; c++)
    TDGL_CUDA(cudaMemcpyAsync(dst[c], src[c], ctx->pcg->n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  return 0;
}

}  // namespace

int pcg_create(Ctx *ctx) {
  const Geo &g = ctx->g;
  PcgDev *S = new PcgDev();
  ctx->pcg = S;
  S->n = g.d.n();
  if (S->n > INT_MAX / 2) return set_err(ctx, TDGL_EINVAL, "grid too large for the PCG solve (32-bit node indices)");
  // a small grid takes fewer blocks (at least 4 entries per thread): the full grid's fixed cost of 1184 blocks and
  // their partial sums would dominate its microsecond kernels and crowd out concurrent contexts
  const long long per = (long long)BS * 4;
  S->sblocks = (int)std::min<long long>(STR_BLOCKS, std::max<long long>(1, (3 * S->n + per - 1) / per));
  const long long nbox = (long long)(g.Nx - 1) * (g.Ny - 1) * (g.Nz - 1);
  S->ablocks = (int)std::min<long long>(RED_BLOCKS, std::max<long long>(1, (nbox + per - 1) / per));
  int rc;
  double **vecs[9] = {S->P, S->Q, S->x, S->r, S->z, S->b, S->xprev, S->zold, S->Dp};
  for (int q = 0; q < 9; q++)
    for (int c = 0; c < 3; c++)
      if ((rc = dalloc(ctx, &vecs[q][c], S->n))) return rc;
  if ((rc = dalloc(ctx, &S->part, 2 * STR_BLOCKS))) return rc;
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    nsm = 148;
  // two blocks per SM at most: they fit beside a preconditioner transform block on every SM
  S->xblocks = std::min(S->sblocks, 2 * nsm);
  if ((rc = dalloc(ctx, &S->part2, S->xblocks))) return rc;
  TDGL_CUDA(cudaStreamCreateWithFlags(&S->side, cudaStreamNonBlocking));
  TDGL_CUDA(cudaEventCreateWithFlags(&S->ev_fork, cudaEventDisableTiming));
  TDGL_CUDA(cudaEventCreateWithFlags(&S->ev_join, cudaEventDisableTiming));
  if ((rc = dalloc(ctx, &S->sc, SC_N))) return rc;
  if ((rc = dalloc(ctx, &S->ic, IC_N))) return rc;
  if ((rc = dalloc(ctx, &S->stat, ST_N))) return rc;
  if (cudaMallocHost(&S->host_sc, SC_N * sizeof(double)) != cudaSuccess) return set_err(ctx, TDGL_ENOMEM, "cudaMallocHost");
  if (cudaMallocHost(&S->host_ic, IC_N * sizeof(int)) != cudaSuccess) return set_err(ctx, TDGL_ENOMEM, "cudaMallocHost");
  if (cudaMallocHost(&S->host_stat, ST_N * sizeof(long long)) != cudaSuccess) return set_err(ctx, TDGL_ENOMEM, "cudaMallocHost");
  // σ_l/σ_n on the ranges, plane-major, for A·p
  const double *D[3] = {ctx->D[0], ctx->D[1], ctx->D[2]};
  to_planes(ctx, D, nullptr, S->Dp);
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

void pcg_destroy(Ctx *ctx) {
  if (ctx->pcg) {
    if (ctx->pcg->host_sc) cudaFreeHost(ctx->pcg->host_sc);
    if (ctx->pcg->host_ic) cudaFreeHost(ctx->pcg->host_ic);
    if (ctx->pcg->host_stat) cudaFreeHost(ctx->pcg->host_stat);
    if (ctx->pcg->side) cudaStreamDestroy(ctx->pcg->side);
    if (ctx->pcg->ev_fork) cudaEventDestroy(ctx->pcg->ev_fork);
    if (ctx->pcg->ev_join) cudaEventDestroy(ctx->pcg->ev_join);
    delete ctx->pcg;
    ctx->pcg = nullptr;
  }
}

static void read_stat(Ctx *ctx) {
  PcgDev *S = ctx->pcg;
  cudaMemcpyAsync(S->host_stat, S->stat, ST_N * sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
}

int pcg_iters(Ctx *ctx, long long *total) {
  if (!ctx->pcg) {
    if (total) *total = 0;
    return 0;
  }
  read_stat(ctx);
  if (total) *total = ctx->pcg->host_stat[ST_TOTAL];
  return (int)ctx->pcg->host_stat[ST_LAST];
}

int pcg_take_status(Ctx *ctx) {
  if (!ctx->pcg) return 0;
  read_stat(ctx);
  PcgDev *S = ctx->pcg;
  const long long nc = S->host_stat[ST_NOCONV], tw = S->host_stat[ST_TCWAIT];
  const bool any = nc > S->noconv_seen, tc = tw > S->tcwait_seen;
  S->noconv_seen = nc;
  S->tcwait_seen = tw;
  if (tc) return set_err(ctx, TDGL_ECUDA, "preconditioner transform: a wait on the tensor cores ran out");
  return any ? TDGL_ENOCONV : 0;
}

long long *pcg_stat_tc(Ctx *ctx) { return ctx->pcg ? ctx->pcg->stat + ST_TCWAIT : nullptr; }

void pcg_regions(Ctx *ctx, Regions &r) {
  PcgDev *S = ctx->pcg;
  for (int c = 0; c < 3; c++) {
    r.push_back({S->x[c], S->n * sizeof(double)});
    r.push_back({S->xprev[c], S->n * sizeof(double)});
  }
}

void pcg_flags(Ctx *ctx, int *warm, int *have2, bool set) {
  PcgDev *S = ctx->pcg;
  if (set) {
    S->warm = *warm != 0;
    S->have2 = *have2 != 0;
  } else {
    *warm = S->warm;
    *have2 = S->have2;
  }
}

bool pcg_steady(Ctx *ctx) {
  PcgDev *S = ctx->pcg;
  const bool ext = (ctx->P.pcg_fast || ctx->P.pcg_f32) && ctx->P.pcg_extrap;
  return S->warm && (!ext || S->have2);
}

// One PCG iteration (implicit.jl:416-437 with the flexible β of :299-305): q = Ap, α; x, r; z = M⁻¹r; β; p.  Every
// kernel returns at once after the convergence flag is set.
static void iteration(Ctx *ctx, double *zc[3], double *zp[3], bool flex, F3 r32, bool r32_ready, double wb32) {
  PcgDev *S = ctx->pcg;
  apply_A(ctx, true, 3);
  TDGL_LAUNCH(ctx, K_PCG_UPD, (24.0 + wb32) * 3 * S->n, k_update, S->sblocks, BS, 0, vv(S->r), cv(S->Q), S->n, S->sc,
              S->part, S->ic, r32, fold(ctx, 5));
  // with TDGL_PCG_DOTFUSE=1 the FP32 preconditioner's inverse transform folds r·z and r·z_old (β) as it writes z;
  // otherwise (the default) r·z_old beside the preconditioner and r·z after it
  static const bool fuse = [] {
    const char *e = getenv("TDGL_PCG_DOTFUSE");
    return e && e[0] == '1';
  }();
  const bool fused = flex && fuse;
  // x += αP and r·z_old need nothing the preconditioner computes: they run on a second stream beside its
  // compute-bound transforms (one parallel branch of a captured loop), joined before β and the new direction.  When
  // the launches are timed one by one, the same kernels run in the same order on the one stream.
  const bool side = ctx->branches && !ctx->prof.on;
  cudaStream_t main = ctx->stream;
  if (side) {
    cudaEventRecord(S->ev_fork, main);
    cudaStreamWaitEvent(S->side, S->ev_fork, 0);
    ctx->stream = S->side;
  }
  TDGL_LAUNCH(ctx, K_PCG_XUPD, 24.0 * 3 * S->n, k_update_x, S->xblocks, BS, 0, vv(S->x), cv(S->P), S->n, S->sc, S->ic);
  if (flex && !fused)
    TDGL_LAUNCH(ctx, K_PCG_DOTS, 16.0 * 3 * S->n, k_dot_part, S->xblocks, BS, 0, cv(S->r), cv(zp), S->n, S->part2, S->ic);
  if (side) {
    ctx->stream = main;
    cudaEventRecord(S->ev_join, S->side);
  }
  DotFuse df;
  for (int c = 0; c < 3; c++) {
    df.r[c] = S->r[c];
    df.zold[c] = flex ? zp[c] : zc[c];
  }
  df.part = S->part;
  df.F = fold(ctx, 4, flex);
  const bool folded = sep_apply(ctx, S->r, zc, flex, S->ic, r32_ready, fused ? &df : nullptr);
  if (side) cudaStreamWaitEvent(main, S->ev_join, 0);
  if (!folded) {
    Fold F = fold(ctx, 4, flex);
    if (flex) {   // the second sum, r·z_old, from k_dot_part's partials
      F.bpart = S->part2;
      F.nbb = S->xblocks;
    }
    TDGL_LAUNCH(ctx, K_PCG_DOT, 16.0 * 3 * S->n, k_dot2, S->sblocks, BS, 0, cv(S->r), cv(zc), cv(zc), 0, S->n, S->part,
                S->ic, F);
  }
  pdir(ctx, zc, 0, true);
  if (flex)
    for (int c = 0; c < 3; c++) std::swap(zc[c], zp[c]);
}

// The loop of a captured step: a conditional WHILE node whose body is BATCH iterations and the kernel that updates
// the condition (the device decides when the solve is done, as the host did between batches).
static int loop_graph(Ctx *ctx, double *zc[3], double *zp[3], bool flex, F3 r32, bool r32_ready, double wb32) {
  PcgDev *S = ctx->pcg;
  const int maxit = ctx->P.pcg_maxit;
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg;
  const cudaGraphNode_t *deps;
  size_t nd;
  cudaGraphConditionalHandle h;
  TDGL_CUDA(cudaStreamGetCaptureInfo(ctx->stream, &cs, nullptr, &cg, &deps, &nd));
  TDGL_CUDA(cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault));
  TDGL_LAUNCH(ctx, K_PCG_FINAL, 0.0, k_loop_enter, 1, 32, 0, h, S->ic, maxit);
  TDGL_CUDA(cudaStreamGetCaptureInfo(ctx->stream, &cs, nullptr, &cg, &deps, &nd));
  cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};   // aggregate initialisation: the rest zero
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  TDGL_CUDA(cudaGraphAddNode(&node, cg, deps, nd, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  TDGL_CUDA(cudaStreamUpdateCaptureDependencies(ctx->stream, &node, 1, cudaStreamSetCaptureDependencies));
  cudaStream_t main = ctx->stream;
  ctx->stream = ctx->cap_stream;
  cudaError_t e = cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (int q = 0; q < BATCH; q++) iteration(ctx, zc, zp, flex, r32, r32_ready, wb32);
    TDGL_LAUNCH(ctx, K_PCG_FINAL, 0.0, k_loop_turn, 1, 32, 0, h, S->ic, S->stat, BATCH, maxit);
    cudaGraph_t out = nullptr;
    e = cudaStreamEndCapture(ctx->stream, &out);
  }
  ctx->stream = main;
  if (e != cudaSuccess) return set_err(ctx, TDGL_ECUDA, "capture of the PCG loop", e);
  return 0;
}

// A settled solve (warm start, extrapolation history present): every decision on the device, so that the same
// launches serve every step and the step can be captured.
static int pcg_settled(Ctx *ctx) {
  PcgDev *S = ctx->pcg;
  const tdgl_params &P = ctx->P;
  const bool fast = P.pcg_fast || P.pcg_f32, f32 = P.pcg_f32 != 0, ext = fast && P.pcg_extrap;
  int rc;
  to_planes(ctx, ctx->ph, ctx->th, S->b);
  scale_increment(ctx);
  dot2(ctx, S->b, S->b, nullptr, false, 0);
  TDGL_CUDA(cudaMemsetAsync(S->ic, 0, IC_N * sizeof(int), ctx->stream));
  TDGL_LAUNCH(ctx, K_PCG_EXTRAP, (ext ? 32.0 : 0.0) * 3 * S->n, k_guess, S->sblocks, BS, 0, vv(S->x), vv(S->xprev), S->n,
              S->sc, S->ic, ext ? 1 : 0);
  if ((rc = copy3(ctx, S->P, S->x))) return rc;
  apply_A(ctx, false, -1);
  F3 r32 = {{nullptr, nullptr, nullptr}};
  float *const *r32p = fast && f32 ? sep_r32(ctx) : nullptr;
  if (r32p)
    for (int c = 0; c < 3; c++) r32.p[c] = r32p[c];
  const double wb32 = r32p ? 4.0 : 0.0;
  TDGL_LAUNCH(ctx, K_PCG_RES, (24.0 + wb32) * 3 * S->n, k_residual, S->sblocks, BS, 0, vv(S->r), cv(S->b), cv(S->Q), S->n,
              S->part, r32, fold(ctx, 1));
  const bool flex = fast && f32;
  double *zc[3], *zp[3];
  for (int c = 0; c < 3; c++) {
    zc[c] = S->z[c];
    zp[c] = S->zold[c];
  }
  sep_apply(ctx, S->r, zc, flex, S->ic, r32p != nullptr);
  pdir(ctx, zc, 1, true);
  dot2(ctx, S->r, zc, nullptr, true, 2);
  if (flex)
    for (int c = 0; c < 3; c++) std::swap(zc[c], zp[c]);
  if (ctx->capturing) {
    if ((rc = loop_graph(ctx, zc, zp, flex, r32, r32p != nullptr, wb32))) return rc;
  } else {
    int launched = 0;
    while (launched < P.pcg_maxit) {
      const int nb_it = std::min(BATCH, P.pcg_maxit - launched);
      for (int q = 0; q < nb_it; q++) iteration(ctx, zc, zp, flex, r32, r32p != nullptr, wb32);
      launched += nb_it;
      read_back(ctx);
      if (S->host_ic[IC_DONE]) break;
    }
  }
  TDGL_LAUNCH(ctx, K_PCG_FINAL, 0.0, k_finish, 1, 32, 0, S->ic, S->stat, 0);
  from_planes(ctx, S->x, ctx->th, ctx->ph);
  return 0;
}

// The solve of implicit.jl:279-446.  Until the warm start has settled (the first steps, or after the carry was
// reset) the host takes the decisions of the reference's loop from read-back scalars; afterwards pcg_settled.
int pcg_implicit(Ctx *ctx) {
  if (pcg_steady(ctx)) return pcg_settled(ctx);
  PcgDev *S = ctx->pcg;
  const tdgl_params &P = ctx->P;
  const bool fast = P.pcg_fast || P.pcg_f32, f32 = P.pcg_f32 != 0;
  int rc;
  // b = φₑ − θ on the ranges, then φ = θ + (φₑ − θ)/D on every link (implicit.jl:381-388)
  to_planes(ctx, ctx->ph, ctx->th, S->b);
  scale_increment(ctx);
  dot2(ctx, S->b, S->b, nullptr, false, 0);
  TDGL_CUDA(cudaMemsetAsync(S->ic, 0, IC_N * sizeof(int), ctx->stream));
  read_back(ctx);
  const double nb = std::sqrt(S->host_sc[SC_BB]);
  if (nb == 0) {
    // _pcg_zero_update! (implicit.jl:251-271)
    if (fast) {
      if (S->warm && P.pcg_extrap) {
        if ((rc = copy3(ctx, S->xprev, S->x))) return rc;
        S->have2 = true;
      } else {
        S->have2 = false;
      }
    }
    for (int c = 0; c < 3; c++) TDGL_CUDA(cudaMemsetAsync(S->x[c], 0, S->n * sizeof(double), ctx->stream));
    S->warm = true;
    TDGL_LAUNCH(ctx, K_PCG_FINAL, 0.0, k_finish, 1, 32, 0, S->ic, S->stat, 1);
    from_planes(ctx, S->x, ctx->th, ctx->ph);
    return 0;
  }
  if (!S->warm) {
    sep_apply(ctx, S->b, S->x, false, nullptr);
    S->have2 = false;
  } else if (fast && P.pcg_extrap) {
    if (S->have2) {
      TDGL_LAUNCH(ctx, K_PCG_EXTRAP, 32.0 * 3 * S->n, k_extrap, S->sblocks, BS, 0, vv(S->x), vv(S->xprev), S->n);
    } else {
      if ((rc = copy3(ctx, S->xprev, S->x))) return rc;
      S->have2 = true;
    }
  }
  S->warm = true;
  if ((rc = copy3(ctx, S->P, S->x))) return rc;
  apply_A(ctx, false, -1);
  F3 r32 = {{nullptr, nullptr, nullptr}};
  float *const *r32p = fast && f32 ? sep_r32(ctx) : nullptr;
  if (r32p)
    for (int c = 0; c < 3; c++) r32.p[c] = r32p[c];
  const double wb32 = r32p ? 4.0 : 0.0;   // bytes per entry of the FP32 copy
  TDGL_LAUNCH(ctx, K_PCG_RES, (24.0 + wb32) * 3 * S->n, k_residual, S->sblocks, BS, 0, vv(S->r), cv(S->b), cv(S->Q), S->n,
              S->part, r32, fold(ctx, 1));
  read_back(ctx);
  const double tol = P.pcg_tol * nb;
  if (std::sqrt(S->host_sc[SC_RR]) > tol) {
    // z alternates between two buffers, so the flexible β's previous z (implicit.jl:299-305) is the other one
    const bool flex = fast && f32;
    double *zc[3], *zp[3];
    for (int c = 0; c < 3; c++) {
      zc[c] = S->z[c];
      zp[c] = S->zold[c];
    }
    sep_apply(ctx, S->r, zc, flex, nullptr, r32p != nullptr);
    pdir(ctx, zc, 1, false);
    dot2(ctx, S->r, zc, nullptr, false, 2);
    if (flex)
      for (int c = 0; c < 3; c++) std::swap(zc[c], zp[c]);
    int launched = 0;
    while (launched < P.pcg_maxit) {
      const int nb_it = std::min(BATCH, P.pcg_maxit - launched);
      for (int q = 0; q < nb_it; q++) iteration(ctx, zc, zp, flex, r32, r32p != nullptr, wb32);
      launched += nb_it;
      read_back(ctx);
      if (S->host_ic[IC_DONE]) break;
    }
  }
  TDGL_LAUNCH(ctx, K_PCG_FINAL, 0.0, k_finish, 1, 32, 0, S->ic, S->stat, 0);
  from_planes(ctx, S->x, ctx->th, ctx->ph);
  return 0;
}

bool pcg_graphable(Ctx *ctx) { return ctx->P.pcg_maxit % BATCH == 0; }

static int carry_xfer(Ctx *ctx, double *const *pm, double *host, bool up) {
  return up ? pm_from_packed_host(ctx, pm, host) : pm_to_packed_host(ctx, pm, host);
}

int pcg_set_carry(Ctx *ctx, const tdgl_carry_view *v) {
  PcgDev *S = ctx->pcg;
  int rc;
  if (v->pcg_x && (rc = carry_xfer(ctx, S->x, v->pcg_x, true))) return rc;
  if (v->pcg_xprev && (rc = carry_xfer(ctx, S->xprev, v->pcg_xprev, true))) return rc;
  S->warm = v->pcg_warm != 0;
  S->have2 = v->pcg_have2 != 0;
  return 0;
}

int pcg_get_carry(Ctx *ctx, const tdgl_carry_view *v) {
  PcgDev *S = ctx->pcg;
  int rc;
  if (v->pcg_x && (rc = carry_xfer(ctx, S->x, v->pcg_x, false))) return rc;
  if (v->pcg_xprev && (rc = carry_xfer(ctx, S->xprev, v->pcg_xprev, false))) return rc;
  const_cast<tdgl_carry_view *>(v)->pcg_warm = S->warm;
  const_cast<tdgl_carry_view *>(v)->pcg_have2 = S->have2;
  return 0;
}

}  // namespace tdgl
