// field.cu — the blocks of the step after the band update (gtdgl/src/field.jl).
//
//   k_current_increment  supercurrent! (:19-46) fused with field_increment! (:84-102): J on each link is computed,
//                        stored (the State carries it) and used at once for φ = θ + d1 τ J − s·Δh
//   k_scale              scale_increment! (gtdgl/src/implicit.jl:337-342)
//   k_links_curl         links! (:105-121) and curl_h! (:124-137) in one launch over their six ranges
//   k_face_h             field_bc! (:189-228) with _open_add! (gtdgl/src/openbc.jl:210-223): each face point
//                        evaluates the reference's sequence of face writes itself, so the precedence of the
//                        overlapping `.=` statements is kept without ordering the threads
//   k_advance            advance! (:248-263): G ← F on the block (θ/φ and V/U swap by pointer)
#include "common.cuh"
#include "merge.cuh"

namespace tdgl {

namespace {
const int BS = 256;

struct CurArgs {
  BandPtrs G;
  const cd *V[3];
  const double *th[3], *tau[3];
  double *J[3], *ph[3];
  const double *h[3];
  double wa[3][TDGL_MAXB];
  int N;
  double d1, sxy, sxz, syx, syz, szx, szy;
  Rng r[3];
  Dim d;
  const uint8_t *mat;   // material per region: each band's link carries w_µ ρ_µ (field.jl:48-71)
  const MatDev *mt;
  const double *dnu;    // the drag matrix ν_µν [MAXB][MAXB] (null: no drag; field.jl:73-81)
};

__device__ __forceinline__ void current_increment_b(const Blk bk, CurArgs const &A);
__global__ void k_current_increment(CurArgs A) { current_increment_b(TDGL_BLK, A); }
TDGL_MERGEABLE(k_current_increment, current_increment_b, BS, 4, false);
__device__ __forceinline__ void current_increment_b(const Blk bk, CurArgs const &A) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
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
  const long long o = d.at(i, j, k);
  const long long sx = 1, sy = d.n1, sz = (long long)d.n1 * d.n2;
  const long long s = ax == 0 ? sx : ax == 1 ? sy : sz;
  const cd v = A.V[ax][o];
  double acc;
  if (A.mat) {   // ρ_µ = τ·W[µ][ax][a][b] of the link from node a to node b
    const int a = A.mat[o] - 1, b = A.mat[o + s] - 1;
    const double tv = A.tau[ax][o];
    acc = (A.wa[ax][0] * (tv * A.mt->W[0][ax][a][b])) * cmul(cmul(cconj(A.G.p[0][o]), v), A.G.p[0][o + s]).y;
    for (int mu = 1; mu < A.N; mu++)
      acc += (A.wa[ax][mu] * (tv * A.mt->W[mu][ax][a][b])) * cmul(cmul(cconj(A.G.p[mu][o]), v), A.G.p[mu][o + s]).y;
  } else {
    acc = A.wa[ax][0] * cmul(cmul(cconj(A.G.p[0][o]), v), A.G.p[0][o + s]).y;
    for (int mu = 1; mu < A.N; mu++) acc += A.wa[ax][mu] * cmul(cmul(cconj(A.G.p[mu][o]), v), A.G.p[mu][o + s]).y;
    if (A.dnu)   // _jdrag: Σ_{µ<η} ν_µη (Im(Ψµ* V Ψη[+e]) + Im(Ψη* V Ψµ[+e]))
      for (int mu = 0; mu < A.N; mu++)
        for (int eta = mu + 1; eta < A.N; eta++) {
          const double c = A.dnu[TDGL_MAXB * mu + eta];
          if (c == 0.0) continue;
          acc += c * (cmul(cmul(cconj(A.G.p[mu][o]), v), A.G.p[eta][o + s]).y +
                      cmul(cmul(cconj(A.G.p[eta][o]), v), A.G.p[mu][o + s]).y);
        }
  }
  A.J[ax][o] = acc;
  const double *hx = A.h[0], *hy = A.h[1], *hz = A.h[2];
  double p;
  if (ax == 0)
    p = ((A.th[0][o] + (A.d1 * A.tau[0][o]) * acc) - A.sxy * (hz[o] - hz[o - sy])) + A.sxz * (hy[o] - hy[o - sz]);
  else if (ax == 1)
    p = ((A.th[1][o] + (A.d1 * A.tau[1][o]) * acc) - A.syz * (hx[o] - hx[o - sz])) + A.syx * (hz[o] - hz[o - sx]);
  else
    p = ((A.th[2][o] + (A.d1 * A.tau[2][o]) * acc) - A.szx * (hy[o] - hy[o - sx])) + A.szy * (hx[o] - hx[o - sy]);
  A.ph[ax][o] = p;
}

struct ScaleArgs {
  const double *th[3], *D[3];
  double *ph[3];
  Rng r[3];
  Dim d;
};

__device__ __forceinline__ void scale_b(const Blk bk, ScaleArgs const &A);
__global__ void k_scale(ScaleArgs A) { scale_b(TDGL_BLK, A); }
TDGL_MERGEABLE(k_scale, scale_b, BS, 1, false);
__device__ __forceinline__ void scale_b(const Blk bk, ScaleArgs const &A) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
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
  const long long o = A.d.at(i, j, k);
  A.ph[ax][o] = A.th[ax][o] + (A.ph[ax][o] - A.th[ax][o]) / A.D[ax][o];
}

struct LCArgs {
  const double *ph[3];
  cd *U[3];
  double *h[3];
  Rng r[6];
  long long off[7];
  Dim d;
  double dx, dy, dz;
};

__device__ __forceinline__ void links_curl_b(const Blk bk, LCArgs const &A);
__global__ void k_links_curl(LCArgs A) { links_curl_b(TDGL_BLK, A); }
TDGL_MERGEABLE(k_links_curl, links_curl_b, BS, 1, false);
__device__ __forceinline__ void links_curl_b(const Blk bk, LCArgs const &A) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= A.off[6]) return;
  int q = 0;
  while (t >= A.off[q + 1]) q++;
  t -= A.off[q];
  int i, j, k;
  rng_ijk(A.r[q], t, i, j, k);
  const Dim d = A.d;
  const long long o = d.at(i, j, k);
  const long long sx = 1, sy = d.n1, sz = (long long)d.n1 * d.n2;
  const double *px = A.ph[0], *py = A.ph[1], *pz = A.ph[2];
  if (q < 3) {
    A.U[q][o] = ccis(-A.ph[q][o]);
  } else if (q == 3) {
    A.h[0][o] = ((pz[o + sy] - pz[o]) - py[o + sz] + py[o]) / (A.dy * A.dz);
  } else if (q == 4) {
    A.h[1][o] = ((px[o + sz] - px[o]) - pz[o + sx] + pz[o]) / (A.dz * A.dx);
  } else {
    A.h[2][o] = ((py[o + sx] - py[o]) - px[o + sy] + px[o]) / (A.dx * A.dy);
  }
}

struct FaceArgs {
  double *h[3];
  const double *bar[6];     // hy_z, hy_y, hz_z, hz_y, hz_x, hy_x
  const double *oo[3], *on[3];
  const StepScal *cur;      // H, HJ and the ramp fraction of this step
  int bc, open;
  int Nx, Ny, Nz;
  Rng r[9];                 // per component: k faces, j faces (k inner), i faces (j, k inner)
  long long off[10];
  Dim d;
};

struct AdvArgs {
  cd *G[TDGL_MAXB];
  const cd *F[TDGL_MAXB];
  int N;
  Rng r;
  Dim d;
};

__device__ __forceinline__ void advance_b(const Blk bk, AdvArgs const &A);
__global__ void k_advance(AdvArgs A) { advance_b(TDGL_BLK, A); }
TDGL_MERGEABLE(k_advance, advance_b, BS, 1, false);
__device__ __forceinline__ void advance_b(const Blk bk, AdvArgs const &A) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= A.r.n()) return;
  int i, j, k;
  rng_ijk(A.r, t, i, j, k);
  const long long o = A.d.at(i, j, k);
  for (int mu = 0; mu < A.N; mu++) A.G[mu][o] = A.F[mu][o];
}

// Shell of a box (a, b, c) split into k faces, j faces and i faces without overlap.
void shell(int a, int b, int c, Rng *r) {
  r[0] = mkrng(1, a, 1, b, 1, 1);
  if (c > 1) r[0].nk = 2;  // k = 1 and k = c: handled through a stride below
  r[1] = mkrng(1, a, 1, 1, 2, c - 1);
  if (b > 1) r[1].nj = 2;
  r[2] = mkrng(1, 1, 2, b - 1, 2, c - 1);
  if (a > 1) r[2].ni = 2;
}

}  // namespace

// k faces etc. are enumerated as index 1 and 2 of a two-element range; map 2 to the far face.
__device__ __forceinline__ int face_of(int x, int far) { return x == 2 ? far : x; }

void supercurrent_increment(Ctx *ctx) {
  const Geo &g = ctx->g;
  const tdgl_params &P = ctx->P;
  CurArgs A;
  for (int mu = 0; mu < ctx->N; mu++) A.G.p[mu] = ctx->G[mu];
  for (int ax = 0; ax < 3; ax++) {
    A.V[ax] = ctx->V[ax]; A.th[ax] = ctx->th[ax]; A.tau[ax] = ctx->tau[ax]; A.J[ax] = ctx->J[ax];
    A.ph[ax] = ctx->ph[ax]; A.h[ax] = ctx->h[ax];
    for (int mu = 0; mu < TDGL_MAXB; mu++) A.wa[ax][mu] = P.wa[ax][mu];
  }
  A.N = ctx->N;
  A.mat = ctx->mat;
  A.mt = ctx->mt;
  A.dnu = ctx->drag_nu;
  A.d1 = P.d1; A.sxy = P.sxy; A.sxz = P.sxz; A.syx = P.syx; A.syz = P.syz; A.szx = P.szx; A.szy = P.szy;
  A.r[0] = mkrng(1, g.Nx, 2, g.Ny, 2, g.Nz);
  A.r[1] = mkrng(2, g.Nx, 1, g.Ny, 2, g.Nz);
  A.r[2] = mkrng(2, g.Nx, 2, g.Ny, 1, g.Nz);
  A.d = g.d;
  long long n = A.r[0].n() + A.r[1].n() + A.r[2].n();
  // per link: V, θ, τ in, J and φ out; per node: every band once and the three h
  const double bytes = 48.0 * n + (16.0 * ctx->N + 24.0) * (double)g.d.n();
  TDGL_LAUNCH(ctx, K_CURINC, bytes, k_current_increment, nblk(n, BS), BS, 0, A);
}

void scale_increment(Ctx *ctx) {
  const Geo &g = ctx->g;
  ScaleArgs A;
  for (int ax = 0; ax < 3; ax++) {
    A.th[ax] = ctx->th[ax]; A.D[ax] = ctx->D[ax]; A.ph[ax] = ctx->ph[ax];
  }
  // every entry of the reference's link arrays (the broadcast over the whole array)
  A.r[0] = mkrng(1, g.Nx, 1, g.Ny + 1, 1, g.Nz + 1);
  A.r[1] = mkrng(1, g.Nx + 1, 1, g.Ny, 1, g.Nz + 1);
  A.r[2] = mkrng(1, g.Nx + 1, 1, g.Ny + 1, 1, g.Nz);
  A.d = g.d;
  long long n = A.r[0].n() + A.r[1].n() + A.r[2].n();
  TDGL_LAUNCH(ctx, K_SCALE, 32.0 * n, k_scale, nblk(n, BS), BS, 0, A);
}

void links_curl(Ctx *ctx) {
  const Geo &g = ctx->g;
  LCArgs A;
  for (int ax = 0; ax < 3; ax++) {
    A.ph[ax] = ctx->ph[ax]; A.U[ax] = ctx->U[ax]; A.h[ax] = ctx->h[ax];
  }
  A.r[0] = mkrng(1, g.Nx, 2, g.Ny, 2, g.Nz);
  A.r[1] = mkrng(2, g.Nx, 1, g.Ny, 2, g.Nz);
  A.r[2] = mkrng(2, g.Nx, 2, g.Ny, 1, g.Nz);
  A.r[3] = mkrng(2, g.Nx, 2, g.Ny - 1, 2, g.Nz - 1);
  A.r[4] = mkrng(2, g.Nx - 1, 2, g.Ny, 2, g.Nz - 1);
  A.r[5] = mkrng(2, g.Nx - 1, 2, g.Ny - 1, 2, g.Nz);
  A.off[0] = 0;
  for (int q = 0; q < 6; q++) A.off[q + 1] = A.off[q] + A.r[q].n();
  A.d = g.d;
  A.dx = g.dx; A.dy = g.dy; A.dz = g.dz;
  const double nl = (double)A.off[3], nh = (double)(A.off[6] - A.off[3]);
  TDGL_LAUNCH(ctx, K_LINKSCURL, 24.0 * nl + 8.0 * nh, k_links_curl, nblk(A.off[6], BS), BS, 0, A);
}

// Face points: every point of the shell of each h array, each exactly once; each evaluates the final value of
// field_bc! (field.jl:189-228) and _open_add! (openbc.jl:210-223) at that point.
__global__ void k_face_h_shell(FaceArgs A);

void field_bc(Ctx *ctx) {
  const Geo &g = ctx->g;
  FaceArgs A;
  for (int c = 0; c < 3; c++) {
    A.h[c] = ctx->h[c];
    A.oo[c] = nullptr;
    A.on[c] = nullptr;
  }
  for (int q = 0; q < 6; q++) A.bar[q] = ctx->bar[q];
  A.cur = ctx->ss_cur;
  A.bc = ctx->P.selffield_bc;
  A.open = A.bc == TDGL_BC_OPEN;
  A.Nx = g.Nx; A.Ny = g.Ny; A.Nz = g.Nz;
  int shp[3][3] = {{g.Nx + 1, g.Ny, g.Nz}, {g.Nx, g.Ny + 1, g.Nz}, {g.Nx, g.Ny, g.Nz + 1}};
  for (int c = 0; c < 3; c++) shell(shp[c][0], shp[c][1], shp[c][2], &A.r[3 * c]);
  A.off[0] = 0;
  for (int q = 0; q < 9; q++) A.off[q + 1] = A.off[q] + A.r[q].n();
  A.d = g.d;
  if (A.open) open_face_args(ctx, A.oo, A.on);
  // the shells are described with far faces at local index 2; k_face_h_shell maps them
  TDGL_LAUNCH(ctx, K_FACEH, (A.open ? 32.0 : 16.0) * A.off[9], k_face_h_shell, nblk(A.off[9], BS), BS, 0, A);
}

__device__ __forceinline__ void face_h_shell_b(const Blk bk, FaceArgs const &A);
__global__ void k_face_h_shell(FaceArgs A) { face_h_shell_b(TDGL_BLK, A); }
TDGL_MERGEABLE(k_face_h_shell, face_h_shell_b, BS, 1, false);
__device__ __forceinline__ void face_h_shell_b(const Blk bk, FaceArgs const &A) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= A.off[9]) return;
  int q = 0;
  while (t >= A.off[q + 1]) q++;
  long long tt = t - A.off[q];
  int i, j, k;
  rng_ijk(A.r[q], tt, i, j, k);
  const int comp = q / 3, part = q % 3;
  const int Nx = A.Nx, Ny = A.Ny, Nz = A.Nz;
  const int ext[3][3] = {{Nx + 1, Ny, Nz}, {Nx, Ny + 1, Nz}, {Nx, Ny, Nz + 1}};
  if (part == 0) k = face_of(k, ext[comp][2]);
  else if (part == 1) j = face_of(j, ext[comp][1]);
  else i = face_of(i, ext[comp][0]);
  const long long o = A.d.at(i, j, k);
  const double H = A.cur->H, HJ = A.cur->HJ, fr = A.cur->open_fr;
  double v = A.h[comp][o];
  if (comp == 2) {  // hz (Nx, Ny, Nz+1)
    if (k == 1 || k == Nz + 1 || i == 1 || i == Nx || j == 1 || j == Ny) v = H;
    if (A.bc != TDGL_BC_SLAB) {
      if (k == 1 || k == Nz + 1) v = H + HJ * A.bar[2][(j - 1) + (long long)Ny * (k == 1 ? 0 : 1)];
      if (j == 1 || j == Ny) v = H + HJ * A.bar[3][(j == 1 ? 0 : 1) + 2LL * (k - 1)];
      if (i == 1 || i == Nx) v = H + HJ * A.bar[4][(j - 1) + (long long)Ny * (k - 1)];
      if (A.open) {
        double oo = A.oo[2][o], nn = A.on[2][o];
        if ((j == 1 || j == Ny) && i >= 2 && i <= Nx - 1) v += oo + fr * (nn - oo);
        if (i == 1 || i == Nx) v += oo + fr * (nn - oo);
      }
    }
  } else if (comp == 0) {  // hx (Nx+1, Ny, Nz)
    if (i == 1 || i == Nx + 1 || j == 1 || j == Ny) v = 0.0;
    if (A.open && i >= 2 && i <= Nx && (j == 1 || j == Ny || k == 1 || k == Nz)) {
      double oo = A.oo[0][o], nn = A.on[0][o];
      v = oo + fr * (nn - oo);
    }
  } else {  // hy (Nx, Ny+1, Nz)
    if (j == 1 || j == Ny + 1) v = 0.0;
    if (A.bc == TDGL_BC_SLAB) {
      if (k == 1) v = -HJ;
      if (k == Nz) v = +HJ;
    } else {
      if (k == 1 || k == Nz) v = HJ * A.bar[0][(j - 1) + (long long)(Ny + 1) * (k == 1 ? 0 : 1)];
      if (j == 1 || j == Ny + 1) v = HJ * A.bar[1][(j == 1 ? 0 : 1) + 2LL * (k - 1)];
      if (i == 1 || i == Nx) v = HJ * A.bar[5][(j - 1) + (long long)(Ny + 1) * (k - 1)];
      if (A.open) {
        double oo = A.oo[1][o], nn = A.on[1][o];
        if ((k == 1 || k == Nz) && i >= 2 && i <= Nx - 1) v += oo + fr * (nn - oo);
        if (i == 1 || i == Nx) v += oo + fr * (nn - oo);
      }
    }
  }
  A.h[comp][o] = v;
}

void advance_swap(Ctx *ctx) {
  for (int ax = 0; ax < 3; ax++) {
    std::swap(ctx->th[ax], ctx->ph[ax]);
    std::swap(ctx->V[ax], ctx->U[ax]);
  }
  ctx->parity ^= 1;
}

void advance_copy(Ctx *ctx) {
  const Geo &g = ctx->g;
  AdvArgs A;
  for (int mu = 0; mu < ctx->N; mu++) {
    A.G[mu] = ctx->G[mu];
    A.F[mu] = ctx->F[mu];
  }
  A.N = ctx->N;
  A.r = mkrng(g.x1, g.x2 + 1, g.y1, g.y2 + 1, g.z1, g.z2 + 1);
  A.d = g.d;
  TDGL_LAUNCH(ctx, K_ADVANCE, 32.0 * ctx->N * A.r.n(), k_advance, nblk(A.r.n(), BS), BS, 0, A);
  advance_swap(ctx);
}

}  // namespace tdgl
