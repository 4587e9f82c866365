// pcg.cu — the insulating-padding field solve on the device (gtdgl/src/implicit.jl:106-446).
//
// (D + aK)Δ = φₑ − θ on the coupled links by preconditioned conjugate gradients, the separable inverse of
// (I + aK) as the preconditioner (in FP32 with pcg_f32, then with the flexible β = r·(z − z_old)/rz_old), the
// warm start and the extrapolated first guess 2xₙ − xₙ₋₁ of pcg_fast (_implicit_curl_fast! :376-446), the
// zero-source update (_pcg_zero_update! :251-271), and φ = θ + (φₑ − θ)/D on the decoupled links.
// Iterates, residuals and dot products are FP64.  Dot products are deterministic: a fixed grid of block
// partial sums (warp shuffles, then a tree) reduced by one block in a fixed order.
#include <cmath>

#include "common.cuh"

namespace tdgl {

void sep_gather(Ctx *ctx, const double *const *a, const double *const *b, double *B);
void sep_scatter(Ctx *ctx, double *const *out, const double *const *base, const double *B);

enum { SC_BB = 0, SC_RR, SC_RZ, SC_PAP, SC_ALPHA, SC_BETA, SC_RZ2, SC_RZOLD, SC_N };
static const int RED_BLOCKS = 592;   // 4 × 148 SMs

struct PcgDev {
  double *P[3] = {}, *Q[3] = {}, *H[3] = {};   // full (node-shaped)
  double *x = nullptr, *r = nullptr, *z = nullptr, *b = nullptr, *xprev = nullptr, *zold = nullptr;   // packed ranges
  double *part = nullptr;                       // RED_BLOCKS × 2 partial sums
  double *sc = nullptr;                         // device scalars SC_*
  double *host_sc = nullptr;                    // pinned copy
  Rng rg[3];
  long long off[4];
  bool warm = false, have2 = false;
  int iters = 0;
  long long total = 0;
};

namespace {
const int BS = 256;

struct PackMap {
  Rng r[3];
  long long off[4];
  Dim d;
  __device__ __forceinline__ long long full(long long t, int &ax) const {
    ax = t >= off[1] ? (t >= off[2] ? 2 : 1) : 0;
    int i, j, k;
    rng_ijk(r[ax], t - off[ax], i, j, k);
    return d.at(i, j, k);
  }
};

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

// partial sums of a·b and (optionally) a·c over n packed entries
__global__ void k_dot2(const double *a, const double *b, const double *c, long long n, double *part) {
  __shared__ double sh[32];
  double s1 = 0.0, s2 = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    double av = a[t];
    s1 += av * b[t];
    if (c) s2 += av * c[t];
  }
  double r1 = block_sum(s1, sh);
  __syncthreads();
  double r2 = c ? block_sum(s2, sh) : 0.0;
  if (threadIdx.x == 0) {
    part[blockIdx.x] = r1;
    part[gridDim.x + blockIdx.x] = r2;
  }
}

// Reduce the partials into the scalars.  mode: 0 bb; 1 rr; 2 rz (initial); 3 pAp → α = rz/pAp;
// 4 (rz2, r·zold) → β and rz ← rz2 (flexible when f32)
__global__ void k_final(const double *part, int nb, double *sc, int mode, int flexible) {
  __shared__ double sh[32];
  double a = 0.0, b = 0.0;
  for (int q = threadIdx.x; q < nb; q += blockDim.x) {
    a += part[q];
    b += part[nb + q];
  }
  a = block_sum(a, sh);
  __syncthreads();
  b = block_sum(b, sh);
  if (threadIdx.x == 0) {
    switch (mode) {
      case 0: sc[SC_BB] = a; break;
      case 1: sc[SC_RR] = a; break;
      case 2: sc[SC_RZ] = a; break;
      case 3: sc[SC_PAP] = a; sc[SC_ALPHA] = sc[SC_RZ] / a; break;
      case 4: {
        sc[SC_RZ2] = a;
        sc[SC_RZOLD] = b;
        sc[SC_BETA] = flexible ? (a - b) / sc[SC_RZ] : a / sc[SC_RZ];
        sc[SC_RZ] = a;
        break;
      }
    }
  }
}

// b = φ − θ on the ranges and φ = θ + (φ − θ)/D on every link of the reference's arrays
struct StartArgs {
  const double *th[3], *D[3];
  double *ph[3];
  double *b;
  Rng all[3], rg[3];
  long long off[4];
  Dim d;
};
__global__ void k_start(StartArgs A) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n0 = A.all[0].n(), n1 = A.all[1].n(), n2 = A.all[2].n();
  int ax = 0;
  if (t >= n0) {
    t -= n0;
    ax = 1;
    if (t >= n1) {
      t -= n1;
      ax = 2;
      if (t >= n2) return;
    }
  }
  int i, j, k;
  rng_ijk(A.all[ax], t, i, j, k);
  const long long o = A.d.at(i, j, k);
  const double th = A.th[ax][o], ph = A.ph[ax][o];
  const Rng &r = A.rg[ax];
  int a = i - r.i0, bb = j - r.j0, c = k - r.k0;
  if (a >= 0 && a < r.ni && bb >= 0 && bb < r.nj && c >= 0 && c < r.nk)
    A.b[A.off[ax] + a + (long long)r.ni * (bb + (long long)r.nj * c)] = ph - th;
  A.ph[ax][o] = th + (ph - th) / A.D[ax][o];
}

// H = curl P on the plaquettes (implicit.jl:216-224)
struct HArgs {
  const double *P[3];
  double *H[3];
  Rng r[3];
  Dim d;
  double dx, dy, dz;
};
__global__ void k_apply_h(HArgs A) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int ax = 0;
  if (t >= A.r[0].n()) {
    t -= A.r[0].n();
    ax = 1;
    if (t >= A.r[1].n()) {
      t -= A.r[1].n();
      ax = 2;
      if (t >= A.r[2].n()) return;
    }
  }
  int i, j, k;
  rng_ijk(A.r[ax], t, i, j, k);
  const Dim d = A.d;
  const long long o = d.at(i, j, k), sx = 1, sy = d.n1, sz = (long long)d.n1 * d.n2;
  const double *px = A.P[0], *py = A.P[1], *pz = A.P[2];
  if (ax == 0) A.H[0][o] = ((pz[o + sy] - pz[o]) - py[o + sz] + py[o]) / (A.dy * A.dz);
  else if (ax == 1) A.H[1][o] = ((px[o + sz] - px[o]) - pz[o + sx] + pz[o]) / (A.dz * A.dx);
  else A.H[2][o] = ((py[o + sx] - py[o]) - px[o + sy] + px[o]) / (A.dx * A.dy);
}

// Q = D P + a curl curl P on the ranges (implicit.jl:225-235), with partial sums of P·Q
struct QArgs {
  const double *P[3], *H[3], *D[3];
  double *Q[3];
  double sxy, sxz, syx, syz, szx, szy;
  PackMap m;
  double *part;
};
__global__ void k_apply_q(QArgs A) {
  __shared__ double sh[32];
  const long long n = A.m.off[3];
  double s = 0.0;
  const Dim d = A.m.d;
  const long long sx = 1, sy = d.n1, sz = (long long)d.n1 * d.n2;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int ax;
    long long o = A.m.full(t, ax);
    const double *hx = A.H[0], *hy = A.H[1], *hz = A.H[2];
    double q;
    if (ax == 0) q = A.D[0][o] * A.P[0][o] + A.sxy * (hz[o] - hz[o - sy]) - A.sxz * (hy[o] - hy[o - sz]);
    else if (ax == 1) q = A.D[1][o] * A.P[1][o] + A.syz * (hx[o] - hx[o - sz]) - A.syx * (hz[o] - hz[o - sx]);
    else q = A.D[2][o] * A.P[2][o] + A.szx * (hy[o] - hy[o - sx]) - A.szy * (hx[o] - hx[o - sy]);
    A.Q[ax][o] = q;
    s += A.P[ax][o] * q;
  }
  double r = block_sum(s, sh);
  if (threadIdx.x == 0) {
    A.part[blockIdx.x] = r;
    A.part[gridDim.x + blockIdx.x] = 0.0;
  }
}

// r = b − Q (ranges), partial r·r
struct ResArgs {
  const double *Q[3];
  const double *b;
  double *r;
  PackMap m;
  double *part;
};
__global__ void k_residual(ResArgs A) {
  __shared__ double sh[32];
  const long long n = A.m.off[3];
  double s = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int ax;
    long long o = A.m.full(t, ax);
    double v = A.b[t] - A.Q[ax][o];
    A.r[t] = v;
    s += v * v;
  }
  double r = block_sum(s, sh);
  if (threadIdx.x == 0) {
    A.part[blockIdx.x] = r;
    A.part[gridDim.x + blockIdx.x] = 0.0;
  }
}

// x += αP, r −= αQ, partial r·r
struct UpdArgs {
  const double *P[3], *Q[3];
  double *x, *r;
  const double *sc;
  PackMap m;
  double *part;
};
__global__ void k_update(UpdArgs A) {
  __shared__ double sh[32];
  const long long n = A.m.off[3];
  const double alpha = A.sc[SC_ALPHA];
  double s = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int ax;
    long long o = A.m.full(t, ax);
    A.x[t] += alpha * A.P[ax][o];
    double v = A.r[t] - alpha * A.Q[ax][o];
    A.r[t] = v;
    s += v * v;
  }
  double r = block_sum(s, sh);
  if (threadIdx.x == 0) {
    A.part[blockIdx.x] = r;
    A.part[gridDim.x + blockIdx.x] = 0.0;
  }
}

// P = z + βP on the ranges (β = 0 and P = z for the first direction), zold = z
struct PArgs {
  double *P[3];
  const double *z;
  double *zold;
  const double *sc;
  int first;
  PackMap m;
};
__global__ void k_pdir(PArgs A) {
  const long long n = A.m.off[3];
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int ax;
  long long o = A.m.full(t, ax);
  double zv = A.z[t];
  A.P[ax][o] = A.first ? zv : zv + A.sc[SC_BETA] * A.P[ax][o];
  if (A.zold) A.zold[t] = zv;
}

// x ← 2x − xprev, xprev ← x (pcg_fast's extrapolated guess, implicit.jl:394-398)
__global__ void k_extrap(double *x, double *xp, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double v = x[t];
  x[t] = 2 * v - xp[t];
  xp[t] = v;
}

PackMap packmap(Ctx *ctx) {
  PcgDev *S = ctx->pcg;
  PackMap m;
  for (int ax = 0; ax < 3; ax++) m.r[ax] = S->rg[ax];
  for (int q = 0; q < 4; q++) m.off[q] = S->off[q];
  m.d = ctx->g.d;
  return m;
}

void dot2(Ctx *ctx, const double *a, const double *b, const double *c) {
  PcgDev *S = ctx->pcg;
  k_dot2<<<RED_BLOCKS, BS, 0, ctx->stream>>>(a, b, c, S->off[3], S->part);
  ctx->launches++;
}
void final_(Ctx *ctx, int mode, int flexible = 0) {
  PcgDev *S = ctx->pcg;
  k_final<<<1, 1024, 0, ctx->stream>>>(S->part, RED_BLOCKS, S->sc, mode, flexible);
  ctx->launches++;
}
double read_sc(Ctx *ctx, int which) {
  PcgDev *S = ctx->pcg;
  cudaMemcpyAsync(S->host_sc, S->sc, SC_N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  return S->host_sc[which];
}

void apply_A(Ctx *ctx) {
  PcgDev *S = ctx->pcg;
  const Geo &g = ctx->g;
  const tdgl_params &Pp = ctx->P;
  HArgs h;
  for (int ax = 0; ax < 3; ax++) {
    h.P[ax] = S->P[ax];
    h.H[ax] = S->H[ax];
  }
  h.r[0] = mkrng(2, g.Nx, 2, g.Ny - 1, 2, g.Nz - 1);
  h.r[1] = mkrng(2, g.Nx - 1, 2, g.Ny, 2, g.Nz - 1);
  h.r[2] = mkrng(2, g.Nx - 1, 2, g.Ny - 1, 2, g.Nz);
  h.d = g.d;
  h.dx = g.dx; h.dy = g.dy; h.dz = g.dz;
  long long nh = h.r[0].n() + h.r[1].n() + h.r[2].n();
  k_apply_h<<<nblk(nh, BS), BS, 0, ctx->stream>>>(h);
  QArgs q;
  for (int ax = 0; ax < 3; ax++) {
    q.P[ax] = S->P[ax]; q.H[ax] = S->H[ax]; q.D[ax] = ctx->D[ax]; q.Q[ax] = S->Q[ax];
  }
  q.sxy = Pp.sxy; q.sxz = Pp.sxz; q.syx = Pp.syx; q.syz = Pp.syz; q.szx = Pp.szx; q.szy = Pp.szy;
  q.m = packmap(ctx);
  q.part = S->part;
  k_apply_q<<<RED_BLOCKS, BS, 0, ctx->stream>>>(q);
  ctx->launches += 2;
}

void set_dir(Ctx *ctx, const double *z, double *zold, int first) {
  PcgDev *S = ctx->pcg;
  PArgs a;
  for (int ax = 0; ax < 3; ax++) a.P[ax] = S->P[ax];
  a.z = z;
  a.zold = zold;
  a.sc = S->sc;
  a.first = first;
  a.m = packmap(ctx);
  k_pdir<<<nblk(S->off[3], BS), BS, 0, ctx->stream>>>(a);
  ctx->launches++;
}

}  // namespace

int pcg_create(Ctx *ctx) {
  const Geo &g = ctx->g;
  PcgDev *S = new PcgDev();
  ctx->pcg = S;
  S->rg[0] = mkrng(2, g.Nx - 1, 2, g.Ny, 2, g.Nz);
  S->rg[1] = mkrng(2, g.Nx, 2, g.Ny - 1, 2, g.Nz);
  S->rg[2] = mkrng(2, g.Nx, 2, g.Ny, 2, g.Nz - 1);
  S->off[0] = 0;
  for (int ax = 0; ax < 3; ax++) S->off[ax + 1] = S->off[ax] + S->rg[ax].n();
  const long long nn = g.d.n(), nt = S->off[3];
  int rc;
  for (int ax = 0; ax < 3; ax++) {
    if ((rc = dalloc(ctx, &S->P[ax], nn))) return rc;
    if ((rc = dalloc(ctx, &S->Q[ax], nn))) return rc;
    if ((rc = dalloc(ctx, &S->H[ax], nn))) return rc;
  }
  double **vecs[6] = {&S->x, &S->r, &S->z, &S->b, &S->xprev, &S->zold};
  for (int q = 0; q < 6; q++)
    if ((rc = dalloc(ctx, vecs[q], nt))) return rc;
  if ((rc = dalloc(ctx, &S->part, 2 * RED_BLOCKS))) return rc;
  if ((rc = dalloc(ctx, &S->sc, SC_N))) return rc;
  if (cudaMallocHost(&S->host_sc, SC_N * sizeof(double)) != cudaSuccess) return set_err(ctx, TDGL_ENOMEM, "cudaMallocHost");
  return 0;
}

void pcg_destroy(Ctx *ctx) {
  if (ctx->pcg) {
    if (ctx->pcg->host_sc) cudaFreeHost(ctx->pcg->host_sc);
    delete ctx->pcg;
    ctx->pcg = nullptr;
  }
}

int pcg_iters(Ctx *ctx, long long *total) {
  if (total) *total = ctx->pcg ? ctx->pcg->total : 0;
  return ctx->pcg ? ctx->pcg->iters : 0;
}

int pcg_implicit(Ctx *ctx) {
  PcgDev *S = ctx->pcg;
  const Geo &g = ctx->g;
  const tdgl_params &P = ctx->P;
  const bool fast = P.pcg_fast || P.pcg_f32, f32 = P.pcg_f32 != 0;
  const long long nt = S->off[3];
  // b and the decoupled links
  StartArgs st;
  for (int ax = 0; ax < 3; ax++) {
    st.th[ax] = ctx->th[ax]; st.D[ax] = ctx->D[ax]; st.ph[ax] = ctx->ph[ax]; st.rg[ax] = S->rg[ax];
  }
  st.all[0] = mkrng(1, g.Nx, 1, g.Ny + 1, 1, g.Nz + 1);
  st.all[1] = mkrng(1, g.Nx + 1, 1, g.Ny, 1, g.Nz + 1);
  st.all[2] = mkrng(1, g.Nx + 1, 1, g.Ny + 1, 1, g.Nz);
  for (int q = 0; q < 4; q++) st.off[q] = S->off[q];
  st.b = S->b;
  st.d = g.d;
  long long na = st.all[0].n() + st.all[1].n() + st.all[2].n();
  k_start<<<nblk(na, BS), BS, 0, ctx->stream>>>(st);
  ctx->launches++;
  dot2(ctx, S->b, S->b, nullptr);
  final_(ctx, 0);
  const double nb = std::sqrt(read_sc(ctx, SC_BB));
  if (nb == 0) {
    // _pcg_zero_update! (implicit.jl:251-271)
    if (fast) {
      if (S->warm && P.pcg_extrap) {
        cudaMemcpyAsync(S->xprev, S->x, nt * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
        S->have2 = true;
      } else {
        S->have2 = false;
      }
    }
    cudaMemsetAsync(S->x, 0, nt * sizeof(double), ctx->stream);
    S->warm = true;
    S->iters = 0;
    const double *th[3] = {ctx->th[0], ctx->th[1], ctx->th[2]};
    sep_gather(ctx, th, nullptr, S->z);
    sep_scatter(ctx, ctx->ph, nullptr, S->z);
    return 0;
  }
  if (!S->warm) {
    sep_apply(ctx, S->b, S->x, false);
    S->have2 = false;
  } else if (fast && P.pcg_extrap) {
    if (S->have2) {
      k_extrap<<<nblk(nt, BS), BS, 0, ctx->stream>>>(S->x, S->xprev, nt);
      ctx->launches++;
    } else {
      cudaMemcpyAsync(S->xprev, S->x, nt * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
      S->have2 = true;
    }
  }
  S->warm = true;
  set_dir(ctx, S->x, nullptr, 1);
  apply_A(ctx);
  ResArgs ra;
  for (int ax = 0; ax < 3; ax++) ra.Q[ax] = S->Q[ax];
  ra.b = S->b;
  ra.r = S->r;
  ra.m = packmap(ctx);
  ra.part = S->part;
  k_residual<<<RED_BLOCKS, BS, 0, ctx->stream>>>(ra);
  ctx->launches++;
  final_(ctx, 1);
  int it = 0, status = 0;
  const double tol = P.pcg_tol * nb;
  if (std::sqrt(read_sc(ctx, SC_RR)) > tol) {
    sep_apply(ctx, S->r, S->z, fast && f32);
    set_dir(ctx, S->z, (fast && f32) ? S->zold : nullptr, 1);
    dot2(ctx, S->r, S->z, nullptr);
    final_(ctx, 2);
    bool conv = false;
    UpdArgs ua;
    for (int ax = 0; ax < 3; ax++) {
      ua.P[ax] = S->P[ax];
      ua.Q[ax] = S->Q[ax];
    }
    ua.x = S->x;
    ua.r = S->r;
    ua.sc = S->sc;
    ua.m = packmap(ctx);
    ua.part = S->part;
    while (it < P.pcg_maxit) {
      it++;
      apply_A(ctx);
      final_(ctx, 3);
      k_update<<<RED_BLOCKS, BS, 0, ctx->stream>>>(ua);
      ctx->launches++;
      final_(ctx, 1);
      if (std::sqrt(read_sc(ctx, SC_RR)) <= tol) {
        conv = true;
        break;
      }
      sep_apply(ctx, S->r, S->z, fast && f32);
      dot2(ctx, S->r, S->z, (fast && f32) ? S->zold : nullptr);
      final_(ctx, 4, fast && f32);
      set_dir(ctx, S->z, (fast && f32) ? S->zold : nullptr, 0);
    }
    if (!conv) status = TDGL_ENOCONV;
  }
  S->iters = it;
  S->total += it;
  sep_scatter(ctx, ctx->ph, ctx->th, S->x);
  return status;
}

int pcg_set_carry(Ctx *ctx, const tdgl_carry_view *v) {
  PcgDev *S = ctx->pcg;
  const size_t nb = S->off[3] * sizeof(double);
  if (v->pcg_x) TDGL_CUDA(cudaMemcpyAsync(S->x, v->pcg_x, nb, cudaMemcpyHostToDevice, ctx->stream));
  if (v->pcg_xprev) TDGL_CUDA(cudaMemcpyAsync(S->xprev, v->pcg_xprev, nb, cudaMemcpyHostToDevice, ctx->stream));
  S->warm = v->pcg_warm != 0;
  S->have2 = v->pcg_have2 != 0;
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int pcg_get_carry(Ctx *ctx, const tdgl_carry_view *v) {
  PcgDev *S = ctx->pcg;
  const size_t nb = S->off[3] * sizeof(double);
  if (v->pcg_x) TDGL_CUDA(cudaMemcpyAsync(v->pcg_x, S->x, nb, cudaMemcpyDeviceToHost, ctx->stream));
  if (v->pcg_xprev) TDGL_CUDA(cudaMemcpyAsync(v->pcg_xprev, S->xprev, nb, cudaMemcpyDeviceToHost, ctx->stream));
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  const_cast<tdgl_carry_view *>(v)->pcg_warm = S->warm;
  const_cast<tdgl_carry_view *>(v)->pcg_have2 = S->have2;
  return 0;
}

}  // namespace tdgl
