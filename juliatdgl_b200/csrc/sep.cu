// sep.cu — the exact inverse of (I + aK) on the link ranges (gtdgl/src/implicit.jl:15-104, _precond32! :346-373).
//
// K is the Yee curl-curl.  Per axis it is diagonalised by the DCT-II basis on the nodes (V) and the DST-I basis
// on the edges between them (U = D V / s); these are exactly the singular vectors _sep_bases (implicit.jl:15-22)
// takes from the SVD of the forward difference D, up to column signs that cancel in V diag V'.  Per wavevector
// the inverse is P_L + P_T/(1 + a|k|²) (implicit.jl:67-78).  The transforms are dense per line (the reference
// multiplies by the same matrices with BLAS), in FP64 for the SepSolver and in FP32 for the PCG preconditioner
// (pcg_f32), with fma accumulation.
#include <cmath>

#include "common.cuh"

namespace tdgl {

template <class T>
struct Basis {
  int n;
  T *Vt, *V, *Ut, *U, *s;   // V[i + n k], Vt = V', U[(e) + (n-1)(k-1)], Ut = U'
};

struct SepDev {
  int nx, ny, nz;
  Rng rg[3];                 // the ranges rx, ry, rz (implicit.jl:52)
  long long nr[3], ntot;
  Basis<double> bd[3];
  Basis<float> bf[3];
  double *B = nullptr, *T1 = nullptr, *T2 = nullptr;   // packed ranges (x | y | z) and two temporaries
  float *Bf = nullptr, *T1f = nullptr, *T2f = nullptr;
  long long tmax;
};

namespace {
const int BS = 256;

// out[.., o, ..] = Σ_t M(t, o) A[.., t, ..] along `axis`; dims of A: (d0, d1, d2).
// axis 0 takes Mt with Mt[o + nout t] (coalesced over o); axes 1, 2 take M with M[t + nin o].
template <class T>
__global__ void k_tx(const T *__restrict__ A, int d0, int d1, int d2, int axis, const T *__restrict__ M, int nout,
                     T *__restrict__ out) {
  int od0 = d0, od1 = d1, od2 = d2;
  if (axis == 0) od0 = nout;
  else if (axis == 1) od1 = nout;
  else od2 = nout;
  long long n = (long long)od0 * od1 * od2;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int i = (int)(t % od0);
  long long r = t / od0;
  int j = (int)(r % od1), k = (int)(r / od1);
  T s = T(0);
  if (axis == 0) {
    const T *a = A + (long long)d0 * (j + (long long)d1 * k);
    for (int q = 0; q < d0; q++) s = fma(M[i + (long long)nout * q], a[q], s);
  } else if (axis == 1) {
    const T *a = A + i + (long long)d0 * d1 * k;
    const T *m = M + (long long)d1 * j;
    for (int q = 0; q < d1; q++) s = fma(m[q], a[(long long)d0 * q], s);
  } else {
    const T *a = A + i + (long long)d0 * j;
    const T *m = M + (long long)d2 * k;
    const long long st = (long long)d0 * d1;
    for (int q = 0; q < d2; q++) s = fma(m[q], a[st * q], s);
  }
  out[t] = s;
}

// The mode solve of implicit.jl:67-78 on X (nx-1, ny, nz), Y (nx, ny-1, nz), Z (nx, ny, nz-1).
template <class T>
__global__ void k_modes(T *X, T *Y, T *Z, const T *sx, const T *sy, const T *sz, int nx, int ny, int nz, T a) {
  long long n = (long long)nx * ny * nz;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int mx = (int)(t % nx) + 1;
  long long r = t / nx;
  int my = (int)(r % ny) + 1, mz = (int)(r / ny) + 1;
  T k1 = sx[mx - 1], k2 = sy[my - 1], k3 = sz[mz - 1];
  T k2s = k1 * k1 + k2 * k2 + k3 * k3;
  if (k2s == T(0)) return;
  T *px = mx > 1 ? &X[(mx - 2) + (long long)(nx - 1) * ((my - 1) + (long long)ny * (mz - 1))] : nullptr;
  T *py = my > 1 ? &Y[(mx - 1) + (long long)nx * ((my - 2) + (long long)(ny - 1) * (mz - 1))] : nullptr;
  T *pz = mz > 1 ? &Z[(mx - 1) + (long long)nx * ((my - 1) + (long long)ny * (mz - 2))] : nullptr;
  T x1 = px ? *px : T(0), y1 = py ? *py : T(0), z1 = pz ? *pz : T(0);
  T d = (k1 * x1 + k2 * y1 + k3 * z1) / k2s;
  T f = T(1) / (T(1) + a * k2s);
  if (px) *px = k1 * d + f * (x1 - k1 * d);
  if (py) *py = k2 * d + f * (y1 - k2 * d);
  if (pz) *pz = k3 * d + f * (z1 - k3 * d);
}

// packed range arrays ↔ the full (node-shaped) link arrays
struct GatherArgs {
  const double *a[3], *b[3];   // B = a - b (b may be null)
  double *B;
  Rng r[3];
  long long off[4];
  Dim d;
};
__global__ void k_gather_diff(GatherArgs A) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.off[3]) return;
  int ax = t >= A.off[1] ? (t >= A.off[2] ? 2 : 1) : 0;
  int i, j, k;
  rng_ijk(A.r[ax], t - A.off[ax], i, j, k);
  long long o = A.d.at(i, j, k);
  A.B[t] = A.b[ax] ? A.a[ax][o] - A.b[ax][o] : A.a[ax][o];
}
struct ScatterArgs {
  double *out[3];
  const double *base[3];   // out = base + B (base may be null: out = B)
  const double *B;
  Rng r[3];
  long long off[4];
  Dim d;
};
__global__ void k_scatter_sum(ScatterArgs A) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.off[3]) return;
  int ax = t >= A.off[1] ? (t >= A.off[2] ? 2 : 1) : 0;
  int i, j, k;
  rng_ijk(A.r[ax], t - A.off[ax], i, j, k);
  long long o = A.d.at(i, j, k);
  A.out[ax][o] = A.base[ax] ? A.base[ax][o] + A.B[t] : A.B[t];
}
__global__ void k_d2f(const double *a, float *b, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) b[t] = (float)a[t];
}
__global__ void k_f2d(const float *a, double *b, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) b[t] = (double)a[t];
}

template <class T>
void upload_basis(Ctx *ctx, Basis<T> &b, int n) {
  b.n = n;
  std::vector<T> V((size_t)n * n), Vt((size_t)n * n), U((size_t)(n - 1) * (n - 1)), Ut((size_t)(n - 1) * (n - 1)), s(n);
  for (int k = 0; k < n; k++) {
    double ck = k == 0 ? std::sqrt(1.0 / n) : std::sqrt(2.0 / n);
    s[k] = (T)(2 * std::sin(M_PI * k / (2.0 * n)));
    for (int i = 0; i < n; i++) {
      double v = ck * std::cos(M_PI * k * (i + 0.5) / n);
      V[i + (size_t)n * k] = (T)v;
      Vt[k + (size_t)n * i] = (T)v;
    }
  }
  for (int k = 1; k < n; k++)
    for (int e = 0; e < n - 1; e++) {
      double u = -std::sqrt(2.0 / n) * std::sin(M_PI * k * (e + 1.0) / n);
      U[e + (size_t)(n - 1) * (k - 1)] = (T)u;
      Ut[(k - 1) + (size_t)(n - 1) * e] = (T)u;
    }
  dalloc(ctx, &b.V, V.size()); dalloc(ctx, &b.Vt, Vt.size());
  dalloc(ctx, &b.U, U.size() + 1); dalloc(ctx, &b.Ut, Ut.size() + 1); dalloc(ctx, &b.s, s.size());
  cudaMemcpyAsync(b.V, V.data(), V.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(b.Vt, Vt.data(), Vt.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(b.U, U.data(), U.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(b.Ut, Ut.data(), Ut.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(b.s, s.data(), s.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
}

template <class T>
void tx(Ctx *ctx, const T *A, int d0, int d1, int d2, int axis, const T *M, int nout, T *out) {
  int od[3] = {d0, d1, d2};
  od[axis] = nout;
  long long n = (long long)od[0] * od[1] * od[2];
  k_tx<T><<<nblk(n, BS), BS, 0, ctx->stream>>>(A, d0, d1, d2, axis, M, nout, out);
  ctx->launches++;
}

// (I + aK)^{-1} in place on the packed ranges B = (BX | BY | BZ)
template <class T>
void solve(Ctx *ctx, SepDev *S, const Basis<T> *b, T *B, T *T1, T *T2, T a) {
  const int nx = S->nx, ny = S->ny, nz = S->nz;
  T *BX = B, *BY = B + S->nr[0], *BZ = B + S->nr[0] + S->nr[1];
  // forward (implicit.jl:63-65): X by (Ux, Vy, Vz), Y by (Vx, Uy, Vz), Z by (Vx, Vy, Uz)
  tx<T>(ctx, BX, nx - 1, ny, nz, 0, b[0].Ut, nx - 1, T1);
  tx<T>(ctx, T1, nx - 1, ny, nz, 1, b[1].V, ny, T2);
  tx<T>(ctx, T2, nx - 1, ny, nz, 2, b[2].V, nz, BX);
  tx<T>(ctx, BY, nx, ny - 1, nz, 0, b[0].Vt, nx, T1);
  tx<T>(ctx, T1, nx, ny - 1, nz, 1, b[1].U, ny - 1, T2);
  tx<T>(ctx, T2, nx, ny - 1, nz, 2, b[2].V, nz, BY);
  tx<T>(ctx, BZ, nx, ny, nz - 1, 0, b[0].Vt, nx, T1);
  tx<T>(ctx, T1, nx, ny, nz - 1, 1, b[1].V, ny, T2);
  tx<T>(ctx, T2, nx, ny, nz - 1, 2, b[2].U, nz - 1, BZ);
  long long nm = (long long)nx * ny * nz;
  k_modes<T><<<nblk(nm, BS), BS, 0, ctx->stream>>>(BX, BY, BZ, b[0].s, b[1].s, b[2].s, nx, ny, nz, a);
  ctx->launches++;
  // back (implicit.jl:79-81): by the transposes
  tx<T>(ctx, BX, nx - 1, ny, nz, 0, b[0].U, nx - 1, T1);
  tx<T>(ctx, T1, nx - 1, ny, nz, 1, b[1].Vt, ny, T2);
  tx<T>(ctx, T2, nx - 1, ny, nz, 2, b[2].Vt, nz, BX);
  tx<T>(ctx, BY, nx, ny - 1, nz, 0, b[0].V, nx, T1);
  tx<T>(ctx, T1, nx, ny - 1, nz, 1, b[1].Ut, ny - 1, T2);
  tx<T>(ctx, T2, nx, ny - 1, nz, 2, b[2].Vt, nz, BY);
  tx<T>(ctx, BZ, nx, ny, nz - 1, 0, b[0].V, nx, T1);
  tx<T>(ctx, T1, nx, ny, nz - 1, 1, b[1].Vt, ny, T2);
  tx<T>(ctx, T2, nx, ny, nz - 1, 2, b[2].Ut, nz - 1, BZ);
}

}  // namespace

long long sep_nrange(Ctx *ctx, int ax) { return ctx->sep->nr[ax]; }

int sep_create(Ctx *ctx) {
  const Geo &g = ctx->g;
  SepDev *S = new SepDev();
  ctx->sep = S;
  S->nx = g.Nx - 1;
  S->ny = g.Ny - 1;
  S->nz = g.Nz - 1;
  if (S->nx < 2 || S->ny < 2 || S->nz < 2) return set_err(ctx, TDGL_EINVAL, "grid too small for the separable solve");
  S->rg[0] = mkrng(2, g.Nx - 1, 2, g.Ny, 2, g.Nz);
  S->rg[1] = mkrng(2, g.Nx, 2, g.Ny - 1, 2, g.Nz);
  S->rg[2] = mkrng(2, g.Nx, 2, g.Ny, 2, g.Nz - 1);
  S->ntot = 0;
  for (int ax = 0; ax < 3; ax++) {
    S->nr[ax] = S->rg[ax].n();
    S->ntot += S->nr[ax];
  }
  S->tmax = (long long)S->nx * S->ny * S->nz;
  int rc = 0;
  const int n[3] = {S->nx, S->ny, S->nz};
  for (int ax = 0; ax < 3; ax++) {
    upload_basis<double>(ctx, S->bd[ax], n[ax]);
    upload_basis<float>(ctx, S->bf[ax], n[ax]);
  }
  if ((rc = dalloc(ctx, &S->B, S->ntot))) return rc;
  if ((rc = dalloc(ctx, &S->T1, S->tmax))) return rc;
  if ((rc = dalloc(ctx, &S->T2, S->tmax))) return rc;
  if ((rc = dalloc(ctx, &S->Bf, S->ntot))) return rc;
  if ((rc = dalloc(ctx, &S->T1f, S->tmax))) return rc;
  if ((rc = dalloc(ctx, &S->T2f, S->tmax))) return rc;
  return 0;
}

void sep_destroy(Ctx *ctx) {
  delete ctx->sep;
  ctx->sep = nullptr;
}

// z = (I + aK)^{-1} r on packed ranges (z may alias r)
void sep_apply(Ctx *ctx, const double *r, double *z, bool f32) {
  SepDev *S = ctx->sep;
  if (f32) {
    k_d2f<<<nblk(S->ntot, BS), BS, 0, ctx->stream>>>(r, S->Bf, S->ntot);
    solve<float>(ctx, S, S->bf, S->Bf, S->T1f, S->T2f, (float)ctx->P.a_imp);
    k_f2d<<<nblk(S->ntot, BS), BS, 0, ctx->stream>>>(S->Bf, z, S->ntot);
    ctx->launches += 2;
  } else {
    if (z != r) cudaMemcpyAsync(z, r, S->ntot * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
    solve<double>(ctx, S, S->bd, z, S->T1, S->T2, ctx->P.a_imp);
  }
}

void sep_gather(Ctx *ctx, const double *const *a, const double *const *b, double *B) {
  SepDev *S = ctx->sep;
  GatherArgs A;
  for (int ax = 0; ax < 3; ax++) {
    A.a[ax] = a[ax];
    A.b[ax] = b ? b[ax] : nullptr;
    A.r[ax] = S->rg[ax];
  }
  A.off[0] = 0;
  for (int ax = 0; ax < 3; ax++) A.off[ax + 1] = A.off[ax] + S->nr[ax];
  A.B = B;
  A.d = ctx->g.d;
  k_gather_diff<<<nblk(S->ntot, BS), BS, 0, ctx->stream>>>(A);
  ctx->launches++;
}

void sep_scatter(Ctx *ctx, double *const *out, const double *const *base, const double *B) {
  SepDev *S = ctx->sep;
  ScatterArgs A;
  for (int ax = 0; ax < 3; ax++) {
    A.out[ax] = out[ax];
    A.base[ax] = base ? base[ax] : nullptr;
    A.r[ax] = S->rg[ax];
  }
  A.off[0] = 0;
  for (int ax = 0; ax < 3; ax++) A.off[ax + 1] = A.off[ax] + S->nr[ax];
  A.B = B;
  A.d = ctx->g.d;
  k_scatter_sum<<<nblk(S->ntot, BS), BS, 0, ctx->stream>>>(A);
  ctx->launches++;
}

// implicit_curl! with the SepSolver (implicit.jl:91-104)
void sep_implicit(Ctx *ctx) {
  SepDev *S = ctx->sep;
  sep_gather(ctx, ctx->ph, ctx->th, S->B);
  solve<double>(ctx, S, S->bd, S->B, S->T1, S->T2, ctx->P.a_imp);
  sep_scatter(ctx, ctx->ph, ctx->th, S->B);
}

}  // namespace tdgl
