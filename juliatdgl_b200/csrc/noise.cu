// noise.cu — thermal noise (gtdgl/src/noise.jl) and the noisy variants of the rotating frame (gtdgl/src/bands.jl).
//
// The reference draws two normals per node and band per step from a Xoshiro stream in a fixed loop order; here every
// draw is a pure function of (seed, step, stream, node) — Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11: ten
// rounds of the 4×32 multiply-xor round with the Weyl key schedule), two 53-bit uniforms, Box–Muller — so no draw
// is stored: SK-ROCK's phase kick Qθ (noise_draw!, noise.jl:101-123) is recomputed from Ψⁿ (G, untouched by the band
// update) wherever it is needed, and the kick after the bands (noise_apply!/noise_kick!, :40-66, :125-151) redraws
// the same numbers.  Streams: band µ for the order parameter, 16 + axis for the link phases (field_kick!, :183-198);
// the node is its node-shaped linear index, the step noise_step0 + the context's step count (read from the step's
// device scalars, so a captured step draws the numbers of the step it replays).
#include <cmath>

#include "common.cuh"
#include "merge.cuh"

namespace tdgl {

namespace {
const int BS = 256;
const double ROT_MIN2 = 1e-3;

__device__ __forceinline__ void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
  }
}

struct NoiseArgs {
  uint64_t seed;
  const StepScal *cur;   // the step index of the draws
  double T, dt, dV;
  int hard;
  const double *f;
  const uint8_t *mat;   // material per region (null: one material)
  const MatDev *mt;
  const uint8_t *vac;   // a sculpted sample's vacuum nodes, which take no kick (null: none)
};

// the node's material (noise.jl:113-115, 156-180): its band's γ̃² and Γ replace the band's; true where the band is absent
__device__ __forceinline__ bool node_band(const NoiseArgs &A, int mu, long long o, double &g2, double &Gam) {
  if (!A.mat) return false;
  const int m = A.mat[o] - 1;
  g2 = A.mt->full[mu][m].gamma2;
  Gam = A.mt->gam[mu][m];
  return A.mt->absent[mu][m] != 0;
}

__device__ __forceinline__ cd normals(const NoiseArgs &A, uint32_t stream, uint32_t node) {
  const uint64_t step = A.cur->noise_step;
  uint32_t w[4] = {node, (uint32_t)step, (uint32_t)(step >> 32), stream};
  philox10(w, (uint32_t)A.seed, (uint32_t)(A.seed >> 32));
  const double u1 = 1.0 - ((double)(w[0] >> 5) * 67108864.0 + (double)(w[1] >> 6)) * (1.0 / 9007199254740992.0);
  const double u2 = ((double)(w[2] >> 5) * 67108864.0 + (double)(w[3] >> 6)) * (1.0 / 9007199254740992.0);
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincos(2.0 * M_PI * u2, &s, &c);
  return mkc(r * c, r * s);
}

// Qθ of node o of band µ (noise_draw!): c √(s/Γ) Im(conj(ψ/ρ) ξ)/ρ where γ̃² > 0 and |ψ|² > ROT_MIN2, else 0
__device__ __forceinline__ double qtheta(const NoiseArgs &A, int mu, double g2, double Gam, cd psi, long long o) {
  if (A.hard && A.f[o] == 0.0) return 0.0;
  if (A.vac && A.vac[o]) return 0.0;
  if (node_band(A, mu, o, g2, Gam)) return 0.0;
  const double r2 = cabs2(psi);
  if (!(g2 > 0 && r2 > ROT_MIN2)) return 0.0;
  const double cN = sqrt(A.T * A.dt / A.dV);
  const cd xi = normals(A, (uint32_t)mu, (uint32_t)o);
  const double sk = sqrt(1 + g2 * r2), rho = sqrt(r2);
  return cN * cmul(cconj(cdivr(psi, rho)), xi).y * sqrt(sk / Gam) / rho;
}

// _sk_turn! (bands.jl:447-453): D ← X e^{i c δθ} on the interior
__device__ __forceinline__ void sk_turn_b(const Blk bk, cd * const &D, const cd * const &X, const cd * const &G, NoiseArgs const &A, int const &mu, double const &g2, double const &Gam, double const &c, Rng const &r, Dim const &d);
__global__ void k_sk_turn(cd *D, const cd *X, const cd *G, NoiseArgs A, int mu, double g2, double Gam, double c, Rng r, Dim d) { sk_turn_b(TDGL_BLK, D, X, G, A, mu, g2, Gam, c, r, d); }
TDGL_MERGEABLE(k_sk_turn, sk_turn_b, 256, 1, false);
__device__ __forceinline__ void sk_turn_b(const Blk bk, cd * const &D, const cd * const &X, const cd * const &G, NoiseArgs const &A, int const &mu, double const &g2, double const &Gam, double const &c, Rng const &r, Dim const &d) {
  const long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= r.n()) return;
  int i, j, k;
  rng_ijk(r, t, i, j, k);
  const long long o = d.at(i, j, k);
  const double q = qtheta(A, mu, g2, Gam, G[o], o);
  D[o] = q == 0.0 ? X[o] : cmul(X[o], ccis(c * q));
}

// _kwt_kick (noise.jl:78-91)
__device__ cd kwt_kick(cd F, cd psi, cd xi, double a, double cN, double dr, double g2, double Gam, double d0) {
  const double r2 = cabs2(psi), sk = sqrt(1 + g2 * r2);
  if (!(r2 > 1e-24)) return cadd(F, rmul(a, xi));
  const cd u = cdivr(psi, sqrt(r2)), w = cmul(cconj(u), xi);
  if (r2 > ROT_MIN2 && cabs2(F) > ROT_MIN2) {
    const double rho = sqrt(r2), aF = hypot(F.x, F.y);
    const double drho = cN * w.x / sqrt(Gam * sk) + d0 / (rho * (sk * sk * sk));
    const double dth = cN * w.y * sqrt(sk / Gam) / rho;
    return cmul(cdivr(F, aF), rmul(aF + drho, ccis(dth)));
  }
  return csub(cadd(F, cmul(rmul(cN, u), mkc(w.x / sqrt(Gam * sk), w.y * sqrt(sk / Gam)))),
              rmul((dr * (1 + sk * sk)) / (sk * sk * sk), psi));
}

// noise_apply! / noise_kick! of one band on the interior, after the band update
__device__ __forceinline__ void noise_after_b(const Blk bk, cd * const &F, const cd * const &G, NoiseArgs const &A, int const &mu, double const &g2b, double const &Gamb, int const &sk, Rng const &r, Dim const &d);
__global__ void k_noise_after(cd *F, const cd *G, NoiseArgs A, int mu, double g2b, double Gamb, int sk, Rng r, Dim d) { noise_after_b(TDGL_BLK, F, G, A, mu, g2b, Gamb, sk, r, d); }
TDGL_MERGEABLE(k_noise_after, noise_after_b, 256, 1, false);
__device__ __forceinline__ void noise_after_b(const Blk bk, cd * const &F, const cd * const &G, NoiseArgs const &A, int const &mu, double const &g2b, double const &Gamb, int const &sk, Rng const &r, Dim const &d) {
  const long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= r.n()) return;
  int i, j, k;
  rng_ijk(r, t, i, j, k);
  const long long o = d.at(i, j, k);
  if (A.hard && A.f[o] == 0.0) return;
  if (A.vac && A.vac[o]) return;
  double g2 = g2b, Gam = Gamb;
  if (node_band(A, mu, o, g2, Gam)) return;
  const double T = A.T, dt = A.dt, dV = A.dV, cN = sqrt(T * dt / dV), a = sqrt(T * dt / (Gam * dV));
  const cd xi = normals(A, (uint32_t)mu, (uint32_t)o);
  const cd f = F[o];
  if (g2 == 0) {
    F[o] = cadd(f, rmul(a, xi));
  } else if (sk && qtheta(A, mu, g2b, Gamb, G[o], o) != 0.0) {   // the phase went in with the stages
    const cd psi = G[o];
    const double rho = hypot(psi.x, psi.y), skk = sqrt(1 + g2 * (rho * rho));
    const cd u = cdivr(psi, rho);
    const double drho = cN * cmul(cconj(u), xi).x / sqrt(Gam * skk) + T * dt / (2 * dV * Gam) / (rho * (skk * skk * skk));
    const double aF = hypot(f.x, f.y);
    F[o] = aF > sqrt(ROT_MIN2) ? rmul((aF + drho) / aF, f) : cadd(f, rmul(drho, u));
  } else {
    F[o] = kwt_kick(f, G[o], xi, a, cN, T * dt / (2 * dV) * g2 / Gam, g2, Gam, T * dt / (2 * dV * Gam));
  }
}

// field_kick! (noise.jl:183-198) on the three link ranges
struct FKArgs {
  double *ph[3];
  const double *D[3];   // null: no conductivity per link
  double amp[3];
  Rng r[3];
  Dim d;
};
__device__ __forceinline__ void field_kick_b(const Blk bk, FKArgs const &K, NoiseArgs const &A);
__global__ void k_field_kick(FKArgs K, NoiseArgs A) { field_kick_b(TDGL_BLK, K, A); }
TDGL_MERGEABLE(k_field_kick, field_kick_b, 256, 1, false);
__device__ __forceinline__ void field_kick_b(const Blk bk, FKArgs const &K, NoiseArgs const &A) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  int ax = 0;
  if (t >= K.r[0].n()) {
    t -= K.r[0].n();
    ax = 1;
    if (t >= K.r[1].n()) {
      t -= K.r[1].n();
      ax = 2;
      if (t >= K.r[2].n()) return;
    }
  }
  int i, j, k;
  rng_ijk(K.r[ax], t, i, j, k);
  const long long o = K.d.at(i, j, k);
  const double n = normals(A, 16u + ax, (uint32_t)o).x;
  const double amp = K.D[ax] ? K.amp[ax] * sqrt(K.D[ax][o]) : K.amp[ax];
  K.ph[ax][o] += amp * n;
}

// the smoothing sweep of the frame rate (bands.jl:255-261): Ω ← Ω/2 + (Σ six neighbours of the copy T)/12
__device__ __forceinline__ void omega_smooth_b(const Blk bk, double * const &Om, const double * const &T, Rng const &r, Dim const &d);
__global__ void k_omega_smooth(double *Om, const double *T, Rng r, Dim d) { omega_smooth_b(TDGL_BLK, Om, T, r, d); }
TDGL_MERGEABLE(k_omega_smooth, omega_smooth_b, 256, 1, false);
__device__ __forceinline__ void omega_smooth_b(const Blk bk, double * const &Om, const double * const &T, Rng const &r, Dim const &d) {
  const long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= r.n()) return;
  int i, j, k;
  rng_ijk(r, t, i, j, k);
  const long long o = d.at(i, j, k), sy = d.n1, sz = (long long)d.n1 * d.n2;
  const double nb = ((T[o + 1] + T[o - 1]) + (T[o + sy] + T[o - sy])) + (T[o + sz] + T[o - sz]);
  Om[o] = 0.5 * T[o] + nb / 12;
}

// C ← C e^{−iω̂h} on the interior (the frame term as a rotation, bands.jl:262-270)
__device__ __forceinline__ void frame_rot_b(const Blk bk, cd * const &Cc, const double * const &Om, double const &h, Rng const &r, Dim const &d);
__global__ void k_frame_rot(cd *Cc, const double *Om, double h, Rng r, Dim d) { frame_rot_b(TDGL_BLK, Cc, Om, h, r, d); }
TDGL_MERGEABLE(k_frame_rot, frame_rot_b, 256, 1, false);
__device__ __forceinline__ void frame_rot_b(const Blk bk, cd * const &Cc, const double * const &Om, double const &h, Rng const &r, Dim const &d) {
  const long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= r.n()) return;
  int i, j, k;
  rng_ijk(r, t, i, j, k);
  const long long o = d.at(i, j, k);
  Cc[o] = cmul(Cc[o], ccis(-(Om[o] * h)));
}

NoiseArgs nargs(Ctx *ctx) {
  NoiseArgs A;
  A.seed = ctx->P.noise_seed;
  A.cur = ctx->ss_cur;
  A.T = ctx->P.noise_T;
  A.dt = ctx->P.dt;
  A.dV = ctx->g.dx * ctx->g.dy * ctx->g.dz;
  A.hard = ctx->P.hard;
  A.f = ctx->f;
  A.mat = ctx->mat;
  A.mt = ctx->mt;
  A.vac = ctx->vac;
  return A;
}

Rng interior(const Geo &g) { return mkrng(g.x1 + 1, g.x2, g.y1 + 1, g.y2, g.z1 + 1, g.z2); }

}  // namespace

bool skrock_band(const Ctx *ctx, int mu) {
  const tdgl_params &P = ctx->P;
  return P.noise_on && P.use_rkc[mu] && P.stages[mu] > 0 && haskwt(ctx, mu);
}

void sk_turn(Ctx *ctx, cd *D, const cd *X, int mu, double c) {
  const Rng r = interior(ctx->g);
  TDGL_LAUNCH(ctx, K_BAND, 48.0 * r.n(), k_sk_turn, nblk(r.n(), BS), BS, 0, D, X, ctx->G[mu], nargs(ctx), mu,
              ctx->P.bcs[mu].gamma2, ctx->P.noise_gamma[mu], c, r, ctx->g.d);
}

// the low-passed frame rate (Ω of the stage already stored, the faces copied): two sweeps, then C ← C e^{−iω̂h}
void frame_smooth_rot(Ctx *ctx, cd *Cc, double h) {
  const Rng r = interior(ctx->g);
  const long long n = ctx->g.d.n();
  for (int pass = 0; pass < 2; pass++) {
    cudaMemcpyAsync(ctx->Oms, ctx->Om, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);   // errors surface at the sync
    TDGL_LAUNCH(ctx, K_OMEGA, 64.0 * r.n(), k_omega_smooth, nblk(r.n(), BS), BS, 0, ctx->Om, ctx->Oms, r, ctx->g.d);
    omega_faces(ctx);
  }
  TDGL_LAUNCH(ctx, K_OMEGA, 40.0 * r.n(), k_frame_rot, nblk(r.n(), BS), BS, 0, Cc, ctx->Om, h, r, ctx->g.d);
}

void frame_rot(Ctx *ctx, cd *Cc, double h) {
  const Rng r = interior(ctx->g);
  TDGL_LAUNCH(ctx, K_OMEGA, 40.0 * r.n(), k_frame_rot, nblk(r.n(), BS), BS, 0, Cc, ctx->Om, h, r, ctx->g.d);
}

void noise_after(Ctx *ctx) {
  const Rng r = interior(ctx->g);
  for (int mu = 0; mu < ctx->N; mu++)
    TDGL_LAUNCH(ctx, K_NOISE, 56.0 * r.n(), k_noise_after, nblk(r.n(), BS), BS, 0, ctx->F[mu], ctx->G[mu], nargs(ctx), mu,
                ctx->P.bcs[mu].gamma2, ctx->P.noise_gamma[mu], skrock_band(ctx, mu) ? 1 : 0, r, ctx->g.d);
}

void field_kick(Ctx *ctx) {
  const Geo &g = ctx->g;
  const double cN = std::sqrt(ctx->P.noise_T * ctx->P.dt / (ctx->P.noise_sigma_n * g.dx * g.dy * g.dz));
  FKArgs K;
  K.r[0] = mkrng(1, g.Nx, 2, g.Ny, 2, g.Nz);
  K.r[1] = mkrng(2, g.Nx, 1, g.Ny, 2, g.Nz);
  K.r[2] = mkrng(2, g.Nx, 2, g.Ny, 1, g.Nz);
  K.amp[0] = cN * g.dx;
  K.amp[1] = cN * g.dy;
  K.amp[2] = cN * g.dz;
  for (int ax = 0; ax < 3; ax++) {   // the conductivity per link where the host gave one (uploaded at creation)
    K.ph[ax] = ctx->ph[ax];
    K.D[ax] = ctx->D[ax];
  }
  K.d = g.d;
  const long long n = K.r[0].n() + K.r[1].n() + K.r[2].n();
  TDGL_LAUNCH(ctx, K_NOISE, 24.0 * n, k_field_kick, nblk(n, BS), BS, 0, K, nargs(ctx));
}

}  // namespace tdgl
