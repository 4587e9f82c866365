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
#include <algorithm>

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
  // a sculpted sample: the conjugate-gradient solve of δ (QPSolve) on the conducting unknowns
  uint8_t *cond = nullptr;               // per unknown: 1 free, 0 cut, 2 held at 0
  double *cx = nullptr, *cy = nullptr, *cz = nullptr, *lamv = nullptr;   // QPVar's coefficients (null: the cut links)
  double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *part = nullptr, *sc = nullptr;
  int *ic = nullptr, *host_ic = nullptr;
  int nb = 1;                           // blocks of the reductions (fixed: the sums' order)
  long long *iters_dev = nullptr;       // CG iterations over all solves (device counter)
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
  // materials (two bands): the node map, the link weights ρ = τ·W, each material's Josephson matrix
  const uint8_t *mat;
  const MatDev *mt;
  double mg[TDGL_MAXMAT][2][2];
  int drag;                          // the drag's share of the conversion, dnu = Stepper.dragν
  double dnu[TDGL_MAXB][TDGL_MAXB];
};

// _conv of band µ at node o (exchange.jl:303-335, without the drag): the link supercurrents into the node over the
// live links (τ), g along each axis, plus the Josephson exchange with the other band
__device__ __forceinline__ double conv(const SrcArgs &A, int mu, long long o, long long sy, long long sz) {
  const cd *P = A.G[mu];
  const cd p = cconj(P[o]);
  double wxp = A.tau[0][o], wxm = A.tau[0][o - 1], wyp = A.tau[1][o], wym = A.tau[1][o - sy], wzp = A.tau[2][o],
         wzm = A.tau[2][o - sz];
  const int m = A.mat ? A.mat[o] - 1 : 0;
  if (A.mat) {   // the band's link weights ρ = τ·W (exchange.jl:359-366: _conv with mt.ρ)
    const double(*W)[TDGL_MAXMAT][TDGL_MAXMAT] = A.mt->W[mu];
    wxp *= W[0][m][A.mat[o + 1] - 1];
    wxm *= W[0][A.mat[o - 1] - 1][m];
    wyp *= W[1][m][A.mat[o + sy] - 1];
    wym *= W[1][A.mat[o - sy] - 1][m];
    wzp *= W[2][m][A.mat[o + sz] - 1];
    wzm *= W[2][A.mat[o - sz] - 1][m];
  }
  const double ax = wxp * cmul(cmul(p, A.V[0][o]), P[o + 1]).y + wxm * cmul(cmul(p, cconj(A.V[0][o - 1])), P[o - 1]).y;
  const double ay = wyp * cmul(cmul(p, A.V[1][o]), P[o + sy]).y + wym * cmul(cmul(p, cconj(A.V[1][o - sy])), P[o - sy]).y;
  const double az = wzp * cmul(cmul(p, A.V[2][o]), P[o + sz]).y + wzm * cmul(cmul(p, cconj(A.V[2][o - sz])), P[o - sz]).y;
  double c = ((A.g[mu][0] * ax) * A.rx2 + (A.g[mu][1] * ay) * A.ry2) + (A.g[mu][2] * az) * A.rz2;
  for (int nu = 0; nu < A.N; nu++) {
    if (nu == mu) continue;
    const cd *Q = A.G[nu];
    c += (A.mat ? A.mg[m][mu][nu] : A.gam[mu][nu]) * cmul(p, Q[o]).y;
    if (A.drag && A.dnu[mu][nu] != 0) {   // the drag's share (exchange.jl:327-332)
      const double qx = wxp * cmul(cmul(p, A.V[0][o]), Q[o + 1]).y + wxm * cmul(cmul(p, cconj(A.V[0][o - 1])), Q[o - 1]).y;
      const double qy = wyp * cmul(cmul(p, A.V[1][o]), Q[o + sy]).y + wym * cmul(cmul(p, cconj(A.V[1][o - sy])), Q[o - sy]).y;
      const double qz = wzp * cmul(cmul(p, A.V[2][o]), Q[o + sz]).y + wzm * cmul(cmul(p, cconj(A.V[2][o - sz])), Q[o - sz]).y;
      c += A.dnu[mu][nu] * ((qx * A.rx2 + qy * A.ry2) + qz * A.rz2);
    }
  }
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
  const int *done;              // skip once set (the conjugate-gradient solve; null: always run)
};

// out[.., a, ..] = Σ_b M[a + n·b] in[.., b, ..] along the axis, b in order
__global__ void k_qp_axis(AxisArgs A) {
  if (A.done && *A.done) return;
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

// ---- the conjugate-gradient solve of δ in a sculpted sample (_qp_cg!, exchange.jl:87-121)
// Scalars: the norm of the source, r·z, α, β and the tolerance; flags: done, iterations, the reduction's block
// counter, iterations launched (the loop's condition).  The dots use the weight 1/2 on each y and z face of the region.
enum { QC_BN = 0, QC_RZ, QC_ALPHA, QC_BETA, QC_N };
enum { QI_DONE = 0, QI_IT, QI_CNT, QI_LAUNCHED, QI_N };
const int QB = 256, QCG_BATCH = 4;

struct CgDims {
  int n1, n2, n3;
  __device__ long long n() const { return (long long)n1 * n2 * n3; }
  __device__ double w(long long t) const {
    const long long u = t / n1;
    const int j = (int)(u % n2), k = (int)(u / n2);
    return (j == 0 || j == n2 - 1 ? 0.5 : 1.0) * (k == 0 || k == n3 - 1 ? 0.5 : 1.0);
  }
};

__device__ double qb_sum(double v, double *sh) {
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

// the block partials (a, b) are in part[block], part[nb + block]; the last block folds them in order and sets the
// scalars of `mode`: 0 the source's norm (done when it is 0); 1 r·z and the test on r·r; 2 p·q → α, an iteration;
// 3 r·z and r·r → β, and the test
__device__ void cg_fold(double *part, double *sc, int *ic, int mode, double tol, int maxit, double *sh) {
  __shared__ int last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&ic[QI_CNT], 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int nb = gridDim.x;
  double a = 0.0, b = 0.0;
  for (int q = threadIdx.x; q < nb; q += blockDim.x) a += __ldcg(part + q);
  for (int q = threadIdx.x; q < nb; q += blockDim.x) b += __ldcg(part + nb + q);
  a = qb_sum(a, sh);
  __syncthreads();
  b = qb_sum(b, sh);
  if (threadIdx.x == 0) {
    if (mode == 0) {
      sc[QC_BN] = sqrt(a);
      if (sc[QC_BN] == 0) ic[QI_DONE] = 1;
    } else if (mode == 1) {
      sc[QC_RZ] = a;
      if (!(sqrt(b) > tol * sc[QC_BN])) ic[QI_DONE] = 1;
    } else if (mode == 2) {
      sc[QC_ALPHA] = sc[QC_RZ] / a;
      ic[QI_IT] += 1;
    } else {
      sc[QC_BETA] = a / sc[QC_RZ];
      sc[QC_RZ] = a;
      if (!(sqrt(b) > tol * sc[QC_BN]) || ic[QI_IT] >= maxit) ic[QI_DONE] = 1;
    }
    ic[QI_CNT] = 0;
  }
}

// S on the cut unknowns set to 0, r = −S, x = 0; ‖r‖ (weighted)
__global__ void k_cg_init(double *S, const uint8_t *cond, double *r, double *x, CgDims D, double *part, double *sc,
                          int *ic, double tol, int maxit) {
  __shared__ double sh[32];
  double a = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < D.n(); t += (long long)gridDim.x * blockDim.x) {
    if (cond[t] != 1) S[t] = 0.0;
    const double v = -S[t];
    r[t] = v;
    x[t] = 0.0;
    a += D.w(t) * v * v;
  }
  a = qb_sum(a, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = a;
    part[gridDim.x + blockIdx.x] = 0.0;
  }
  __syncthreads();
  cg_fold(part, sc, ic, 0, tol, maxit, sh);
}

// the weighted dots a·b and (with c) a·c, folded by `mode`
__global__ void k_cg_dot(const double *a, const double *b, const double *c, CgDims D, double *part, double *sc,
                         int *ic, int mode, double tol, int maxit) {
  if (ic[QI_DONE]) return;
  __shared__ double sh[32];
  double s1 = 0.0, s2 = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < D.n(); t += (long long)gridDim.x * blockDim.x) {
    const double w = D.w(t);
    s1 += w * a[t] * b[t];
    if (c) s2 += w * a[t] * c[t];
  }
  s1 = qb_sum(s1, sh);
  __syncthreads();
  s2 = qb_sum(s2, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s1;
    part[gridDim.x + blockIdx.x] = s2;
  }
  __syncthreads();
  cg_fold(part, sc, ic, mode, tol, maxit, sh);
}

// z = cond ? −z : 0 (the separable solve projected on the conducting unknowns, with the sign of A)
__global__ void k_cg_proj(double *z, const uint8_t *cond, CgDims D, const int *ic) {
  if (ic[QI_DONE]) return;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < D.n()) z[t] = cond[t] == 1 ? -z[t] : 0.0;
}

// y = −(σn∇²_c − λ) x on the unknowns (_qp_apply!, exchange.jl:52-84)
__global__ void k_cg_apply(double *y, const double *x, const uint8_t *cond, CgDims D, double ax, double ay, double az,
                           double lam, const int *ic) {
  if (ic[QI_DONE]) return;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= D.n()) return;
  const int n1 = D.n1, n2 = D.n2, n3 = D.n3;
  const int i = (int)(t % n1);
  const long long u = t / n1;
  const int j = (int)(u % n2), k = (int)(u / n2);
  const long long sj = n1, sk = (long long)n1 * n2;
  if (!cond[t]) {
    y[t] = (2 * ax + 2 * ay + 2 * az + lam) * x[t];
    return;
  }
  const double v = x[t];
  double acc = lam * v;
  acc += ax * (v - (i > 0 ? (cond[t - 1] ? x[t - 1] : v) : 0.0));
  acc += ax * (v - (i < n1 - 1 ? (cond[t + 1] ? x[t + 1] : v) : 0.0));
  if (n2 > 1) {
    if (j == 0) {
      if (cond[t + sj]) acc += 2 * ay * (v - x[t + sj]);
    } else if (j == n2 - 1) {
      if (cond[t - sj]) acc += 2 * ay * (v - x[t - sj]);
    } else {
      if (cond[t - sj]) acc += ay * (v - x[t - sj]);
      if (cond[t + sj]) acc += ay * (v - x[t + sj]);
    }
  }
  if (n3 > 1) {
    if (k == 0) {
      if (cond[t + sk]) acc += 2 * az * (v - x[t + sk]);
    } else if (k == n3 - 1) {
      if (cond[t - sk]) acc += 2 * az * (v - x[t - sk]);
    } else {
      if (cond[t - sk]) acc += az * (v - x[t - sk]);
      if (cond[t + sk]) acc += az * (v - x[t + sk]);
    }
  }
  y[t] = acc;
}

// y = −(∇·σ∇ − λ) x on the free unknowns with QPVar's coefficients (_qp_apply_var!, exchange.jl:233-256): a neighbour
// held at 0 adds its link to the diagonal, a cut one nothing; a non-free unknown is decoupled (y = d x)
struct VarCoef {
  const double *cx, *cy, *cz, *lam;
  double d;
};
__global__ void k_cg_apply_var(double *y, const double *x, const uint8_t *typ, CgDims D, VarCoef V, const int *ic) {
  if (ic[QI_DONE]) return;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= D.n()) return;
  const int n1 = D.n1, n2 = D.n2, n3 = D.n3;
  const int i = (int)(t % n1);
  const long long u = t / n1;
  const int j = (int)(u % n2), k = (int)(u / n2);
  const long long sj = n1, sk = (long long)n1 * n2;
  if (typ[t] != 1) {
    y[t] = V.d * x[t];
    return;
  }
  const double a = x[t];
  double acc = V.lam[t] * a;
  auto nb = [&](double c, long long o) { return typ[o] == 1 ? c * (a - x[o]) : typ[o] == 2 ? c * a : 0.0; };
  auto CX = [&](int ii) { return V.cx[(long long)ii + (long long)(n1 + 1) * (j + (long long)n2 * k)]; };
  auto CY = [&](int jj) { return V.cy[(long long)i + (long long)n1 * (jj + (long long)(n2 - 1) * k)]; };
  auto CZ = [&](int kk) { return V.cz[(long long)i + (long long)n1 * (j + (long long)n2 * kk)]; };
  acc += i > 0 ? nb(CX(i), t - 1) : CX(0) * a;
  acc += i < n1 - 1 ? nb(CX(i + 1), t + 1) : CX(n1) * a;
  if (n2 > 1) {
    if (j == 0) acc += 2 * nb(CY(0), t + sj);
    else if (j == n2 - 1) acc += 2 * nb(CY(n2 - 2), t - sj);
    else acc += nb(CY(j - 1), t - sj) + nb(CY(j), t + sj);
  }
  if (n3 > 1) {
    if (k == 0) acc += 2 * nb(CZ(0), t + sk);
    else if (k == n3 - 1) acc += 2 * nb(CZ(n3 - 2), t - sk);
    else acc += nb(CZ(k - 1), t - sk) + nb(CZ(k), t + sk);
  }
  y[t] = acc;
}

// op 0: dst = src; 1: dst = dst − src; 2: x += αp, r −= αq (dst = x, src = p, r, q); 3: p = z + βp (dst = p, src = z)
__global__ void k_cg_vec(int op, double *dst, const double *src, double *r, const double *q, CgDims D, const double *sc,
                         const int *ic) {
  if (ic[QI_DONE]) return;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= D.n()) return;
  if (op == 0) dst[t] = src[t];
  else if (op == 1) dst[t] = dst[t] - src[t];
  else if (op == 2) {
    const double al = sc[QC_ALPHA];
    dst[t] = dst[t] + al * src[t];
    r[t] = r[t] - al * q[t];
  } else {
    dst[t] = src[t] + sc[QC_BETA] * dst[t];
  }
}

// δ on the region's nodes from the solution x (always: x = 0 when the source was 0)
__global__ void k_cg_out(double *delta, const double *x, CgDims D, int j0, int k0, Dim d) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= D.n()) return;
  const int i = (int)(t % D.n1);
  const long long u = t / D.n1;
  const int j = (int)(u % D.n2), k = (int)(u / D.n2);
  delta[d.at(i + 2, j + 1 + j0, k + 1 + k0)] = x[t];
}

__global__ void k_cg_copy(double *dst, const double *src, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = src[t];
}

__global__ void k_cg_enter(cudaGraphConditionalHandle h, const int *ic, int maxit) {
  if (threadIdx.x == 0) cudaGraphSetConditional(h, (!ic[QI_DONE] && ic[QI_LAUNCHED] < maxit) ? 1u : 0u);
}
__global__ void k_cg_turn(cudaGraphConditionalHandle h, int *ic, int batch, int maxit) {
  if (threadIdx.x == 0) {
    ic[QI_LAUNCHED] += batch;
    cudaGraphSetConditional(h, (!ic[QI_DONE] && ic[QI_LAUNCHED] < maxit) ? 1u : 0u);
  }
}
__global__ void k_cg_count(const int *ic, long long *iters) {
  if (threadIdx.x == 0) *iters += ic[QI_IT];
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
  if (P.qp_cond) {   // a sculpted sample: the conjugate-gradient solve of δ
    q->nb = (int)std::min<long long>(4 * 148, std::max<long long>(1, ((long long)nu + 4 * QB - 1) / (4 * QB)));
    double **vs[5] = {&q->x, &q->r, &q->z, &q->p, &q->q};
    for (int v = 0; v < 5; v++)
      if ((rc = dalloc(ctx, vs[v], nu))) return rc;
    if ((rc = dalloc(ctx, &q->cond, nu)) || (rc = dalloc(ctx, &q->part, 2 * (size_t)q->nb)) ||
        (rc = dalloc(ctx, &q->sc, QC_N)) || (rc = dalloc(ctx, &q->ic, QI_N)))
      return rc;
    long long *it = nullptr;
    if ((rc = dalloc(ctx, &it, 1))) return rc;
    q->iters_dev = it;
    TDGL_CUDA(cudaMemcpyAsync(q->cond, P.qp_cond, nu, cudaMemcpyHostToDevice, ctx->stream));
    if (P.qp_cx) {   // QPVar's coefficients
      const size_t ncx = (size_t)(q->n[0] + 1) * q->n[1] * q->n[2], ncy = (size_t)q->n[0] * std::max(q->n[1] - 1, 0) * q->n[2],
                   ncz = (size_t)q->n[0] * q->n[1] * std::max(q->n[2] - 1, 0);
      if ((rc = dalloc(ctx, &q->cx, ncx)) || (rc = dalloc(ctx, &q->cy, std::max<size_t>(ncy, 1))) ||
          (rc = dalloc(ctx, &q->cz, std::max<size_t>(ncz, 1))) || (rc = dalloc(ctx, &q->lamv, nu)))
        return rc;
      TDGL_CUDA(cudaMemcpyAsync(q->cx, P.qp_cx, ncx * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      if (ncy) TDGL_CUDA(cudaMemcpyAsync(q->cy, P.qp_cy, ncy * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      if (ncz) TDGL_CUDA(cudaMemcpyAsync(q->cz, P.qp_cz, ncz * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      TDGL_CUDA(cudaMemcpyAsync(q->lamv, P.qp_lamv, nu * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    }
    if (cudaMallocHost(&q->host_ic, QI_N * sizeof(int)) != cudaSuccess) return set_err(ctx, TDGL_ENOMEM, "cudaMallocHost");
  }
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

void qp_potentials(Ctx *ctx, const double **out) {
  for (int mu = 0; mu < TDGL_MAXB; mu++) out[mu] = ctx->qp ? ctx->qp->mu[mu] : nullptr;
}

void qp_destroy(Ctx *ctx) {
  if (ctx->qp && ctx->qp->host_ic) cudaFreeHost(ctx->qp->host_ic);
  delete ctx->qp;
  ctx->qp = nullptr;
}

namespace {

// the separable solve of the region (the three W, the division with λ, the three V) from `in` to `out`, T the
// work array; skipped once the CG is done
void cg_sep(Ctx *ctx, const double *in, double *out, double lam) {
  QpDev *q = ctx->qp;
  AxisArgs X;
  X.n1 = q->n[0];
  X.n2 = q->n[1];
  X.n3 = q->n[2];
  for (int ax = 0; ax < 3; ax++) X.e[ax] = q->e[ax];
  X.sigma_n = ctx->P.qp_sigma_n;
  X.lam = lam;
  X.delta = nullptr;
  X.j0 = q->j0;
  X.k0 = q->k0;
  X.d = ctx->g.d;
  X.done = q->ic + QI_DONE;
  X.todelta = 0;
  const long long nu = (long long)X.n1 * X.n2 * X.n3;
  const double *src[6] = {in, q->T, out, q->T, out, q->T};
  double *dst[6] = {q->T, out, q->T, out, q->T, out};
  for (int pass = 0; pass < 6; pass++) {
    const int ax = pass % 3;
    X.in = src[pass];
    X.out = dst[pass];
    X.M = pass < 3 ? q->W[ax] : q->V[ax];
    X.axis = ax;
    X.div = pass == 2;
    TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_qp_axis, nblk(nu, QB), QB, 0, X);
  }
}

// one CG iteration (exchange.jl:106-116): q = A p, α; x, r; z = M⁻¹ r; β and the test; p
// y = A x: the cut links of a sculpted sample, or QPVar's variable coefficients
void cg_apply(Ctx *ctx, double *y, const double *x, const CgDims &D, double ax, double ay, double az, double lam) {
  QpDev *q = ctx->qp;
  const long long nu = (long long)D.n1 * D.n2 * D.n3;
  if (q->cx) {
    VarCoef V{q->cx, q->cy, q->cz, q->lamv, ctx->P.qp_d};
    TDGL_LAUNCH(ctx, K_QP, 72.0 * nu, k_cg_apply_var, nblk(nu, QB), QB, 0, y, x, q->cond, D, V, q->ic);
  } else {
    TDGL_LAUNCH(ctx, K_QP, 40.0 * nu, k_cg_apply, nblk(nu, QB), QB, 0, y, x, q->cond, D, ax, ay, az, lam, q->ic);
  }
}

void cg_iteration(Ctx *ctx, const CgDims &D, double ax, double ay, double az, double lam, double lsep) {
  QpDev *q = ctx->qp;
  const tdgl_params &P = ctx->P;
  const long long nu = (long long)D.n1 * D.n2 * D.n3;
  const unsigned nbl = nblk(nu, QB);
  cg_apply(ctx, q->q, q->p, D, ax, ay, az, lam);
  TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_cg_dot, q->nb, QB, 0, q->p, q->q, nullptr, D, q->part, q->sc, q->ic, 2, P.qp_tol,
              P.qp_maxit);
  TDGL_LAUNCH(ctx, K_QP, 48.0 * nu, k_cg_vec, nbl, QB, 0, 2, q->x, q->p, q->r, q->q, D, q->sc, q->ic);
  cg_sep(ctx, q->r, q->z, lsep);
  TDGL_LAUNCH(ctx, K_QP, 9.0 * nu, k_cg_proj, nbl, QB, 0, q->z, q->cond, D, q->ic);
  TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_cg_dot, q->nb, QB, 0, q->r, q->z, q->r, D, q->part, q->sc, q->ic, 3, P.qp_tol,
              P.qp_maxit);
  TDGL_LAUNCH(ctx, K_QP, 24.0 * nu, k_cg_vec, nbl, QB, 0, 3, q->p, q->z, nullptr, nullptr, D, q->sc, q->ic);
}

// _qp_cg! on the source in M[0], δ written from the solution; the loop on the device (a conditional node of a
// captured step) or, launched from the host, in batches with the done flag read between them
// (σn∇²_c − λ) x = S on the source S (overwritten; λ = max(l0, 1e-12σn)); x written to δ (two bands) or back to S
// (a mode of N fluids)
int cg_solve(Ctx *ctx, double *S, double l0, bool todelta) {
  QpDev *q = ctx->qp;
  const tdgl_params &P = ctx->P;
  const Geo &g = ctx->g;
  CgDims D{q->n[0], q->n[1], q->n[2]};
  const long long nu = (long long)D.n1 * D.n2 * D.n3;
  const unsigned nbl = nblk(nu, QB);
  const double sn = P.qp_sigma_n, ax = sn / (g.dx * g.dx), ay = sn / (g.dy * g.dy), az = sn / (g.dz * g.dz);
  // the apply's λ, and the separable preconditioner's (with QPVar the same floor, exchange.jl:381)
  const double lam = std::max(l0, 1e-12 * sn), lsep = q->cx ? lam : l0;
  TDGL_CUDA(cudaMemsetAsync(q->ic, 0, QI_N * sizeof(int), ctx->stream));
  TDGL_LAUNCH(ctx, K_QP, 24.0 * nu, k_cg_init, q->nb, QB, 0, S, q->cond, q->r, q->x, D, q->part, q->sc, q->ic,
              P.qp_tol, P.qp_maxit);
  cg_sep(ctx, q->r, q->z, lsep);
  TDGL_LAUNCH(ctx, K_QP, 9.0 * nu, k_cg_proj, nbl, QB, 0, q->z, q->cond, D, q->ic);
  TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_cg_vec, nbl, QB, 0, 0, q->x, q->z, nullptr, nullptr, D, q->sc, q->ic);
  cg_apply(ctx, q->q, q->x, D, ax, ay, az, lam);
  TDGL_LAUNCH(ctx, K_QP, 24.0 * nu, k_cg_vec, nbl, QB, 0, 1, q->r, q->q, nullptr, nullptr, D, q->sc, q->ic);
  cg_sep(ctx, q->r, q->z, lsep);
  TDGL_LAUNCH(ctx, K_QP, 9.0 * nu, k_cg_proj, nbl, QB, 0, q->z, q->cond, D, q->ic);
  TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_cg_vec, nbl, QB, 0, 0, q->p, q->z, nullptr, nullptr, D, q->sc, q->ic);
  TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_cg_dot, q->nb, QB, 0, q->r, q->z, q->r, D, q->part, q->sc, q->ic, 1, P.qp_tol,
              P.qp_maxit);
  if (ctx->capturing) {   // the loop as a conditional WHILE node, QCG_BATCH iterations per turn
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg;
    const cudaGraphNode_t *deps;
    size_t nd;
    cudaGraphConditionalHandle h;
    TDGL_CUDA(cudaStreamGetCaptureInfo(ctx->stream, &cs, nullptr, &cg, &deps, &nd));
    TDGL_CUDA(cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault));
    TDGL_LAUNCH(ctx, K_QP, 0.0, k_cg_enter, 1, 32, 0, h, q->ic, P.qp_maxit);
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
      for (int b = 0; b < QCG_BATCH; b++) cg_iteration(ctx, D, ax, ay, az, lam, lsep);
      TDGL_LAUNCH(ctx, K_QP, 0.0, k_cg_turn, 1, 32, 0, h, q->ic, QCG_BATCH, P.qp_maxit);
      cudaGraph_t out = nullptr;
      e = cudaStreamEndCapture(ctx->stream, &out);
    }
    ctx->stream = main;
    if (e != cudaSuccess) return set_err(ctx, TDGL_ECUDA, "capture of the δ solve's loop", e);
  } else {
    for (int launched = 0; launched < P.qp_maxit; launched += QCG_BATCH) {
      for (int b = 0; b < QCG_BATCH; b++) cg_iteration(ctx, D, ax, ay, az, lam, lsep);
      TDGL_CUDA(cudaMemcpyAsync(q->host_ic, q->ic, QI_N * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
      if (q->host_ic[QI_DONE]) break;
    }
  }
  TDGL_LAUNCH(ctx, K_QP, 0.0, k_cg_count, 1, 32, 0, q->ic, q->iters_dev);
  if (todelta) {
    TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_cg_out, nbl, QB, 0, q->mu[0], q->x, D, q->j0, q->k0, g.d);
  } else {   // the solution back to the source (k_cg_vec returns at once after the loop)
    TDGL_LAUNCH(ctx, K_QP, 16.0 * nu, k_cg_copy, nbl, QB, 0, S, q->x, nu);
  }
  return 0;
}

}  // namespace

long long qp_cg_iterations(Ctx *ctx) {
  if (!ctx->qp || !ctx->qp->iters_dev) return 0;
  long long v = 0;
  cudaMemcpyAsync(&v, ctx->qp->iters_dev, sizeof(v), cudaMemcpyDeviceToHost, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  return v;
}

int qp_potential(Ctx *ctx) {
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
  A.mat = ctx->mat;
  A.mt = ctx->mt;
  for (int m = 0; m < TDGL_MAXMAT; m++)
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++) A.mg[m][a][b] = P.qp_mgamma[m][a][b];
  A.drag = P.drag_on;
  for (int a = 0; a < TDGL_MAXB; a++)
    for (int b = 0; b < TDGL_MAXB; b++) A.dnu[a][b] = P.drag_nu[a][b];
  TDGL_LAUNCH(ctx, K_QP, 0.0, k_qp_source, nblk(A.r.n(), 256), 256, 0, A);
  if (q->cond && P.qp_on != 2) return cg_solve(ctx, q->M[0], P.qp_lambda0, true);
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
  X.done = nullptr;
  // each mode: forward M → T → M → T (the last divided), back T → M → T → M (two bands: → δ); in a sculpted sample
  // each mode of N fluids by conjugate gradients (with a zero source the solve returns zero, as the reference's skip)
  for (int m = 0; m < q->nm; m++) {
    if (q->cond) {
      if (int rc = cg_solve(ctx, q->M[m], P.qp_lam[m], false)) return rc;
      continue;
    }
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
  return 0;
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
