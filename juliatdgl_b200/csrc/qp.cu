// qp.cu — two normal fluids on the device (gtdgl/src/exchange.jl, QPExchange: two bands, one material, no sculpted
// vacuum).  Before the bands, δ = μ_π − μ_σ from the state at the start of the step (qp_potential!, :343-385): the
// source C_π/s_π − C_σ/s_σ on the nodes of the block (_conv, :303-335), the separable solve of σn∇²δ − λ0 δ = S on
// the region of δ (_qp_sep!, :271-277: the three inverse bases W along x, y, z, the division by σn(e_x + e_y + e_z)
// − λ0, the three bases V), δ on the region's nodes.  After the bands each band turns by e^{−iμ_µ dt}, μ_σ = −s_π δ,
// μ_π = s_σ δ (qp_turn!, :403-414).
//
// The region holds (Nx − 1) × nj × nk unknowns (x nodes 2..Nx; y, z nodes of the section, or of the bar with the
// insulating padding), column-major.  Each axis pass is a small dense product per line, one thread per output,
// the sum over the line in order: the oracle's arithmetic.  δ is a function of the state: nothing of it is carried.
#include "common.cuh"

namespace tdgl {

struct QpDev {
  double *S = nullptr, *T = nullptr;    // the source, modes and solution on the region; a work array
  double *V[3] = {}, *W[3] = {}, *e[3] = {};
  double *delta = nullptr;              // δ, node-shaped: zero outside the region and on the x faces
  int n[3] = {0, 0, 0};                 // Nx − 1, nj, nk
  int j0 = 0, k0 = 0;                   // the region's first y and z node, less one
};

namespace {

struct SrcArgs {
  const cd *G[2];
  const cd *V[3];
  const double *tau[3];
  double g[2][3], gam[2], s[2], rx2, ry2, rz2;
  double *S;
  int n1, nj, j0, k0;
  Rng r;
  Dim d;
};

// _conv of band µ at node o (exchange.jl:303-335, without the drag): the link supercurrents into the node over the
// live links (τ), g along each axis, plus the Josephson exchange with the other band
__device__ __forceinline__ double conv(const SrcArgs &A, int mu, long long o, long long sy, long long sz) {
  const cd *P = A.G[mu], *Q = A.G[1 - mu];
  const cd p = cconj(P[o]);
  const double ax = A.tau[0][o] * cmul(cmul(p, A.V[0][o]), P[o + 1]).y +
                    A.tau[0][o - 1] * cmul(cmul(p, cconj(A.V[0][o - 1])), P[o - 1]).y;
  const double ay = A.tau[1][o] * cmul(cmul(p, A.V[1][o]), P[o + sy]).y +
                    A.tau[1][o - sy] * cmul(cmul(p, cconj(A.V[1][o - sy])), P[o - sy]).y;
  const double az = A.tau[2][o] * cmul(cmul(p, A.V[2][o]), P[o + sz]).y +
                    A.tau[2][o - sz] * cmul(cmul(p, cconj(A.V[2][o - sz])), P[o - sz]).y;
  double c = ((A.g[mu][0] * ax) * A.rx2 + (A.g[mu][1] * ay) * A.ry2) + (A.g[mu][2] * az) * A.rz2;
  c += A.gam[mu] * cmul(p, Q[o]).y;
  return c;
}

// S on the nodes of the block (x1..x2+1, y1..y2+1, z1..z2+1); the rest of the region stays 0
__global__ void k_qp_source(SrcArgs A) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.r.n()) return;
  int i, j, k;
  rng_ijk(A.r, t, i, j, k);
  const long long o = A.d.at(i, j, k), sy = A.d.n1, sz = (long long)A.d.n1 * A.d.n2;
  const double c1 = conv(A, 0, o, sy, sz), c2 = conv(A, 1, o, sy, sz);
  A.S[(long long)(i - 2) + (long long)A.n1 * ((long long)(j - A.j0 - 1) + (long long)A.nj * (k - A.k0 - 1))] =
      c2 / A.s[1] - c1 / A.s[0];
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
  double sigma_n, lambda0;
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
  if (A.div) acc /= A.sigma_n * (A.e[0][i] + A.e[1][j] + A.e[2][k]) - A.lambda0;
  if (A.todelta)
    A.delta[A.d.at(i + 2, j + 1 + A.j0, k + 1 + A.k0)] = acc;
  else
    A.out[t] = acc;
}

// F_µ ← F_µ e^{−i m_µ dt δ} on the nodes the band update writes (m = (−s_π, s_σ))
__global__ void k_qp_turn(cd *F0, cd *F1, const double *delta, double c0, double c1, Rng r, Dim d) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= r.n()) return;
  int i, j, k;
  rng_ijk(r, t, i, j, k);
  const long long o = d.at(i, j, k);
  const double dv = delta[o];
  F0[o] = cmul(F0[o], ccis(-c0 * dv));
  F1[o] = cmul(F1[o], ccis(-c1 * dv));
}

}  // namespace

int qp_create(Ctx *ctx, const tdgl_params *p) {
  const tdgl_params &P = *p;
  const Geo &g = ctx->g;
  QpDev *q = new QpDev();
  ctx->qp = q;
  q->n[0] = g.Nx - 1;
  q->n[1] = P.qp_nj;
  q->n[2] = P.qp_nk;
  q->j0 = P.qp_j0 - 1;
  q->k0 = P.qp_k0 - 1;
  const size_t nu = (size_t)q->n[0] * q->n[1] * q->n[2];
  int rc;
  if ((rc = dalloc(ctx, &q->S, nu)) || (rc = dalloc(ctx, &q->T, nu)) || (rc = dalloc(ctx, &q->delta, g.d.n())))
    return rc;
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

void qp_destroy(Ctx *ctx) {
  delete ctx->qp;
  ctx->qp = nullptr;
}

void qp_potential(Ctx *ctx) {
  QpDev *q = ctx->qp;
  const Geo &g = ctx->g;
  const tdgl_params &P = ctx->P;
  const long long nu = (long long)q->n[0] * q->n[1] * q->n[2];
  cudaMemsetAsync(q->S, 0, nu * sizeof(double), ctx->stream);
  SrcArgs A;
  for (int mu = 0; mu < 2; mu++) {
    A.G[mu] = ctx->G[mu];
    A.gam[mu] = P.qp_gamma[mu];
    A.s[mu] = P.qp_s[mu];
    for (int ax = 0; ax < 3; ax++) A.g[mu][ax] = P.qp_g[mu][ax];
  }
  for (int ax = 0; ax < 3; ax++) {
    A.V[ax] = ctx->V[ax];
    A.tau[ax] = ctx->tau[ax];
  }
  A.rx2 = 1 / (g.dx * g.dx);
  A.ry2 = 1 / (g.dy * g.dy);
  A.rz2 = 1 / (g.dz * g.dz);
  A.S = q->S;
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
  X.lambda0 = P.qp_lambda0;
  X.delta = q->delta;
  X.j0 = q->j0;
  X.k0 = q->k0;
  X.d = g.d;
  // forward S → T → S → T (the last divided), back T → S → T → δ
  double *bufs[2] = {q->S, q->T};
  for (int pass = 0; pass < 6; pass++) {
    const int ax = pass % 3;
    X.in = bufs[pass % 2];
    X.out = bufs[(pass + 1) % 2];
    X.M = pass < 3 ? q->W[ax] : q->V[ax];
    X.axis = ax;
    X.div = pass == 2;
    X.todelta = pass == 5;
    TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_qp_axis, nblk(nu, 256), 256, 0, X);
  }
}

void qp_turn(Ctx *ctx) {
  QpDev *q = ctx->qp;
  const Geo &g = ctx->g;
  const Rng r = mkrng(g.x1 + 1, g.x2, g.y1 + 1, g.y2, g.z1 + 1, g.z2);
  const double c0 = -ctx->P.qp_s[1] * ctx->P.dt, c1 = ctx->P.qp_s[0] * ctx->P.dt;
  TDGL_LAUNCH(ctx, K_QP, 72.0 * r.n(), k_qp_turn, nblk(r.n(), 256), 256, 0, ctx->F[0], ctx->F[1], q->delta, c0, c1, r,
              g.d);
}

}  // namespace tdgl
