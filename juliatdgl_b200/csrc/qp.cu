// qp.cu — normal fluids per band on the device (gtdgl/src/exchange.jl; one material, no sculpted vacuum).
//
// Two bands (QPExchange): before the bands, δ = μ_π − μ_σ from the state at the start of the step (qp_potential!,
// :343-385): the source C_π/s_π − C_σ/s_σ on the nodes of the block (_conv, :303-335), the separable solve of
// σn∇²δ − λ0 δ = S on the region of δ (_qp_sep!, :271-277: the three inverse bases W along x, y, z, the division by
// σn(e_x + e_y + e_z) − λ0, the three bases V), δ on the region's nodes.  After the bands each band turns by
// e^{−iμ_µ dt}, μ_σ = −s_π δ, μ_π = s_σ δ (qp_turn!, :403-414).
// N fluids (QPExchangeN, :478-514, :533-543): R_µ = C_µ/s_µ − ΣC, the modes m_k = Σ_µ Pinv[k, µ] R_µ formed with
// the source, each mode solved as δ with its λ_k, μ_µ = Σ_k P[µ, k] m_k on the region, band µ turned by e^{−i dt μ_µ}.
//
// The region holds (Nx − 1) × nj × nk unknowns (x nodes 2..Nx; y, z nodes of the section, or of the bar with the
// insulating padding), column-major.  Each axis pass is a small dense product per line, one thread per output,
// the sum over the line in order: the oracle's arithmetic.  The potentials are functions of the state: nothing of
// them is carried.
#include "common.cuh"

namespace tdgl {

struct QpDev {
  int nm = 1;                           // modes: 1 (two bands: δ) or N (N fluids)
  double *M[TDGL_MAXB] = {};            // each mode's source, transform and solution on the region
  double *T = nullptr;                  // a work array of the region's size
  double *V[3] = {}, *W[3] = {}, *e[3] = {};
  double *mu[TDGL_MAXB] = {};           // node-shaped, zero outside the region and on the x faces: δ (two bands) or μ_µ
  int n[3] = {0, 0, 0};                 // Nx − 1, nj, nk
  int j0 = 0, k0 = 0;                   // the region's first y and z node, less one
};

namespace {

struct SrcArgs {
  const cd *G[TDGL_MAXB];
  const cd *V[3];
  const double *tau[3];
  double g[TDGL_MAXB][3], gam[TDGL_MAXB][TDGL_MAXB], s[TDGL_MAXB], Pinv[TDGL_MAXB][TDGL_MAXB], rx2, ry2, rz2;
  double *M[TDGL_MAXB];
  int N, nfluid, n1, nj, j0, k0;   // nfluid: 0 two bands (one mode, δ's source), 1 N fluids (N modes)
  Rng r;
  Dim d;
};

// _conv of band µ at node o (exchange.jl:303-335, without the drag): the link supercurrents into the node over the
// live links (τ), g along each axis, plus the Josephson exchange with the other band
__device__ __forceinline__ double conv(const SrcArgs &A, int mu, long long o, long long sy, long long sz) {
  const cd *P = A.G[mu];
  const cd p = cconj(P[o]);
  const double ax = A.tau[0][o] * cmul(cmul(p, A.V[0][o]), P[o + 1]).y +
                    A.tau[0][o - 1] * cmul(cmul(p, cconj(A.V[0][o - 1])), P[o - 1]).y;
  const double ay = A.tau[1][o] * cmul(cmul(p, A.V[1][o]), P[o + sy]).y +
                    A.tau[1][o - sy] * cmul(cmul(p, cconj(A.V[1][o - sy])), P[o - sy]).y;
  const double az = A.tau[2][o] * cmul(cmul(p, A.V[2][o]), P[o + sz]).y +
                    A.tau[2][o - sz] * cmul(cmul(p, cconj(A.V[2][o - sz])), P[o - sz]).y;
  double c = ((A.g[mu][0] * ax) * A.rx2 + (A.g[mu][1] * ay) * A.ry2) + (A.g[mu][2] * az) * A.rz2;
  for (int nu = 0; nu < A.N; nu++)
    if (nu != mu) c += A.gam[mu][nu] * cmul(p, A.G[nu][o]).y;
  return c;
}

// The modes' sources on the nodes of the block (x1..x2+1, y1..y2+1, z1..z2+1); the rest of the region stays 0.  Two
// bands: C_π/s_π − C_σ/s_σ.  N fluids: m_k = Σ_µ Pinv[k, µ] (C_µ/s_µ − ΣC), summed over µ in order from 0.
__global__ void k_qp_source(SrcArgs A) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.r.n()) return;
  int i, j, k;
  rng_ijk(A.r, t, i, j, k);
  const long long o = A.d.at(i, j, k), sy = A.d.n1, sz = (long long)A.d.n1 * A.d.n2;
  const long long q = (long long)(i - 2) + (long long)A.n1 * ((long long)(j - A.j0 - 1) + (long long)A.nj * (k - A.k0 - 1));
  if (!A.nfluid) {
    const double c1 = conv(A, 0, o, sy, sz), c2 = conv(A, 1, o, sy, sz);
    A.M[0][q] = c2 / A.s[1] - c1 / A.s[0];
    return;
  }
  double c[TDGL_MAXB], R[TDGL_MAXB];
  for (int mu = 0; mu < A.N; mu++) c[mu] = conv(A, mu, o, sy, sz);
  double C = c[0];
  for (int mu = 1; mu < A.N; mu++) C += c[mu];
  for (int mu = 0; mu < A.N; mu++) R[mu] = c[mu] / A.s[mu] - C;
  for (int kk = 0; kk < A.N; kk++) {
    double m = 0.0;
    for (int mu = 0; mu < A.N; mu++) m += A.Pinv[kk][mu] * R[mu];
    A.M[kk][q] = m;
  }
}

struct AxisArgs {
  const double *in;
  double *out;
  const double *M;              // n × n column-major, n the extent along `axis`
  int n1, n2, n3, axis;
  // div: divide by σn(e_x + e_y + e_z) − λ0 (the last forward pass); to the node-shaped δ instead of out (the last
  // inverse pass)
  int div, todelta;
  const double *e[3];
  double sigma_n, lam;
  double *delta;
  int j0, k0;
  Dim d;
};

// out[.., a, ..] = Σ_b M[a + n·b] in[.., b, ..] along the axis, b in order
__global__ void k_qp_axis(AxisArgs A) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long tot = (long long)A.n1 * A.n2 * A.n3;
  if (t >= tot) return;
  const int i = (int)(t % A.n1);
  const long long u = t / A.n1;
  const int j = (int)(u % A.n2), k = (int)(u / A.n2);
  const int a = A.axis == 0 ? i : A.axis == 1 ? j : k;
  const int n = A.axis == 0 ? A.n1 : A.axis == 1 ? A.n2 : A.n3;
  const long long st = A.axis == 0 ? 1 : A.axis == 1 ? (long long)A.n1 : (long long)A.n1 * A.n2;
  const double *in = A.in + (t - (long long)a * st);
  double acc = 0.0;
  for (int b = 0; b < n; b++) acc += A.M[a + (long long)n * b] * in[(long long)b * st];
  if (A.div) acc /= A.sigma_n * (A.e[0][i] + A.e[1][j] + A.e[2][k]) - A.lam;
  if (A.todelta)
    A.delta[A.d.at(i + 2, j + 1 + A.j0, k + 1 + A.k0)] = acc;
  else
    A.out[t] = acc;
}

// μ_µ = Σ_k P[µ, k] m_k (in order from 0) on the region's nodes (x nodes 2..Nx)
struct MuArgs {
  const double *M[TDGL_MAXB];
  double *mu[TDGL_MAXB];
  double P[TDGL_MAXB][TDGL_MAXB];
  int N, n1, nj, nk, j0, k0;
  Dim d;
};
__global__ void k_qp_mu(MuArgs A) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)A.n1 * A.nj * A.nk) return;
  const int i = (int)(t % A.n1);
  const long long u = t / A.n1;
  const int j = (int)(u % A.nj), k = (int)(u / A.nj);
  const long long o = A.d.at(i + 2, j + 1 + A.j0, k + 1 + A.k0);
  for (int mu = 0; mu < A.N; mu++) {
    double acc = 0.0;
    for (int kk = 0; kk < A.N; kk++) acc += A.P[mu][kk] * A.M[kk][t];
    A.mu[mu][o] = acc;
  }
}

// Two bands: F_µ ← F_µ e^{−i (m_µ dt) δ} with m = (−s_π, s_σ); N fluids: F_µ ← F_µ e^{−i dt μ_µ}; on the nodes the
// band update writes
struct TurnArgs {
  cd *F[TDGL_MAXB];
  const double *mu[TDGL_MAXB];
  double c[2], dt;
  int N, nfluid;
  Rng r;
  Dim d;
};
__global__ void k_qp_turn(TurnArgs A) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.r.n()) return;
  int i, j, k;
  rng_ijk(A.r, t, i, j, k);
  const long long o = A.d.at(i, j, k);
  if (!A.nfluid) {
    const double dv = A.mu[0][o];
    A.F[0][o] = cmul(A.F[0][o], ccis(-A.c[0] * dv));
    A.F[1][o] = cmul(A.F[1][o], ccis(-A.c[1] * dv));
    return;
  }
  for (int mu = 0; mu < A.N; mu++) A.F[mu][o] = cmul(A.F[mu][o], ccis(-A.dt * A.mu[mu][o]));
}

}  // namespace

int qp_create(Ctx *ctx, const tdgl_params *p) {
  const tdgl_params &P = *p;
  const Geo &g = ctx->g;
  QpDev *q = new QpDev();
  ctx->qp = q;
  q->nm = P.qp_on == 2 ? ctx->N : 1;
  q->n[0] = g.Nx - 1;
  q->n[1] = P.qp_nj;
  q->n[2] = P.qp_nk;
  q->j0 = P.qp_j0 - 1;
  q->k0 = P.qp_k0 - 1;
  const size_t nu = (size_t)q->n[0] * q->n[1] * q->n[2];
  int rc;
  if ((rc = dalloc(ctx, &q->T, nu))) return rc;
  for (int m = 0; m < q->nm; m++)
    if ((rc = dalloc(ctx, &q->M[m], nu)) || (rc = dalloc(ctx, &q->mu[m], g.d.n()))) return rc;
  const double *Vs[3] = {P.qp_Vx, P.qp_Vy, P.qp_Vz}, *Ws[3] = {P.qp_Wx, P.qp_Wy, P.qp_Wz},
               *es[3] = {P.qp_ex, P.qp_ey, P.qp_ez};
  for (int ax = 0; ax < 3; ax++) {
    const size_t nn = (size_t)q->n[ax] * q->n[ax];
    if ((rc = dalloc(ctx, &q->V[ax], nn)) || (rc = dalloc(ctx, &q->W[ax], nn)) || (rc = dalloc(ctx, &q->e[ax], q->n[ax])))
      return rc;
    TDGL_CUDA(cudaMemcpyAsync(q->V[ax], Vs[ax], nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    TDGL_CUDA(cudaMemcpyAsync(q->W[ax], Ws[ax], nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    TDGL_CUDA(cudaMemcpyAsync(q->e[ax], es[ax], q->n[ax] * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  }
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

void qp_potentials(Ctx *ctx, const double **out) {
  for (int mu = 0; mu < TDGL_MAXB; mu++) out[mu] = ctx->qp ? ctx->qp->mu[mu] : nullptr;
}

void qp_destroy(Ctx *ctx) {
  delete ctx->qp;
  ctx->qp = nullptr;
}

void qp_potential(Ctx *ctx) {
  QpDev *q = ctx->qp;
  const Geo &g = ctx->g;
  const tdgl_params &P = ctx->P;
  const long long nu = (long long)q->n[0] * q->n[1] * q->n[2];
  for (int m = 0; m < q->nm; m++) cudaMemsetAsync(q->M[m], 0, nu * sizeof(double), ctx->stream);
  SrcArgs A;
  A.N = ctx->N;
  A.nfluid = P.qp_on == 2;
  for (int mu = 0; mu < TDGL_MAXB; mu++) {
    A.G[mu] = mu < ctx->N ? ctx->G[mu] : nullptr;
    A.s[mu] = P.qp_s[mu];
    A.M[mu] = q->M[mu];
    for (int ax = 0; ax < 3; ax++) A.g[mu][ax] = P.qp_g[mu][ax];
    for (int nu2 = 0; nu2 < TDGL_MAXB; nu2++) {
      A.gam[mu][nu2] = P.qp_gamma[mu][nu2];
      A.Pinv[mu][nu2] = P.qp_Pinv[mu][nu2];
    }
  }
  for (int ax = 0; ax < 3; ax++) {
    A.V[ax] = ctx->V[ax];
    A.tau[ax] = ctx->tau[ax];
  }
  A.rx2 = 1 / (g.dx * g.dx);
  A.ry2 = 1 / (g.dy * g.dy);
  A.rz2 = 1 / (g.dz * g.dz);
  A.n1 = q->n[0];
  A.nj = q->n[1];
  A.j0 = q->j0;
  A.k0 = q->k0;
  A.r = mkrng(g.x1, g.x2 + 1, g.y1, g.y2 + 1, g.z1, g.z2 + 1);
  A.d = g.d;
  TDGL_LAUNCH(ctx, K_QP, 0.0, k_qp_source, nblk(A.r.n(), 256), 256, 0, A);
  AxisArgs X;
  X.n1 = q->n[0];
  X.n2 = q->n[1];
  X.n3 = q->n[2];
  for (int ax = 0; ax < 3; ax++) X.e[ax] = q->e[ax];
  X.sigma_n = P.qp_sigma_n;
  X.delta = q->mu[0];
  X.j0 = q->j0;
  X.k0 = q->k0;
  X.d = g.d;
  // each mode: forward M → T → M → T (the last divided), back T → M → T → M (two bands: → δ)
  for (int m = 0; m < q->nm; m++) {
    double *bufs[2] = {q->M[m], q->T};
    X.lam = P.qp_on == 2 ? P.qp_lam[m] : P.qp_lambda0;
    for (int pass = 0; pass < 6; pass++) {
      const int ax = pass % 3;
      X.in = bufs[pass % 2];
      X.out = bufs[(pass + 1) % 2];
      X.M = pass < 3 ? q->W[ax] : q->V[ax];
      X.axis = ax;
      X.div = pass == 2;
      X.todelta = pass == 5 && P.qp_on != 2;
      TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_qp_axis, nblk(nu, 256), 256, 0, X);
    }
  }
  if (P.qp_on == 2) {
    MuArgs U;
    U.N = ctx->N;
    U.n1 = q->n[0];
    U.nj = q->n[1];
    U.nk = q->n[2];
    U.j0 = q->j0;
    U.k0 = q->k0;
    U.d = g.d;
    for (int mu = 0; mu < TDGL_MAXB; mu++) {
      U.M[mu] = q->M[mu];
      U.mu[mu] = q->mu[mu];
      for (int kk = 0; kk < TDGL_MAXB; kk++) U.P[mu][kk] = P.qp_P[mu][kk];
    }
    TDGL_LAUNCH(ctx, K_QP, 8.0 * ctx->N * (ctx->N + 1) * nu, k_qp_mu, nblk(nu, 256), 256, 0, U);
  }
}

void qp_turn(Ctx *ctx) {
  QpDev *q = ctx->qp;
  const Geo &g = ctx->g;
  TurnArgs A;
  A.N = ctx->N;
  A.nfluid = ctx->P.qp_on == 2;
  A.r = mkrng(g.x1 + 1, g.x2, g.y1 + 1, g.y2, g.z1 + 1, g.z2);
  A.d = g.d;
  A.dt = ctx->P.dt;
  A.c[0] = -ctx->P.qp_s[1] * ctx->P.dt;
  A.c[1] = ctx->P.qp_s[0] * ctx->P.dt;
  for (int mu = 0; mu < TDGL_MAXB; mu++) {
    A.F[mu] = mu < ctx->N ? ctx->F[mu] : nullptr;
    A.mu[mu] = q->mu[mu];
  }
  TDGL_LAUNCH(ctx, K_QP, (40.0 * ctx->N) * A.r.n(), k_qp_turn, nblk(A.r.n(), 256), 256, 0, A);
}

}  // namespace tdgl
