// bands.cu — the order-parameter update of every band (gtdgl/src/bands.jl).
//
// One kernel per band stage: the gauge-link stencil of _band_row! (bands.jl:71-97) with the KWT update
// (kwt_update :135-140, kwt_update_rot :151-159), fused with the per-node epilogues that follow it in the
// reference — the rotating-frame rate or term (_frame_rate! :213-234, _frame_term! :274-286), the RKL/RKC
// combination (_combine! :425-430) and the final turn back (_frame_turn! :321-327).  Link rotations of the
// later stages (_rot!, _advance_links!, _frame_links!, _link_rate!, _rotlinks!, _rotfrac!, :292-423) run as one
// kernel over the three link ranges; the covariant Neumann ghosts (ghosts! :524-539) as three face passes in the
// reference's precedence x, y, z.
#include "common.cuh"
#include "merge.cuh"

namespace tdgl {

// The links a stage reads: the arrays as given (mode 0), or (mode 1) the rotated links of a later RKL/RKC stage of a
// rotating-frame band, V e^{iRc} with the per-step rate R (_rotlinks!, bands.jl:311-316), formed on the fly from the
// step's links where the stencil or the ghosts read them instead of from a stored copy: the same per-link formula as
// the link pass.  (_rotfrac! of a band without the frame keeps its link pass.)
struct LinkRot {
  int mode;
  double c;
  const cd *V[3], *U[3];
  const double *R[3];
};
// LR: the mode, fixed per kernel instance
template <int LR>
__device__ __forceinline__ cd link_at(const LinkRot &R, const cd *L, int ax, long long o) {
  if (LR == 0) return L[o];
  return cmul(R.V[ax][o], ccis_short(R.R[ax][o] * R.c));
}

struct StageArgs {
  cd *C;              // destination
  const cd *S;        // stage source
  BandPtrs G;         // every band at the start of the step (coupling)
  const cd *Lx, *Ly, *Lz;
  const double *f;
  tdgl_bandcoef cf;
  int mu, N, hard, rk;
  // epilogue
  int frame_rate;     // 1: first (sub)stage of a rotating-frame band: Ω from C and S, C ← C − iΩhS
  int frame_store;    // with frame_rate: store Ω only (noise: the rate is low-passed before it is applied)
  int frame_term;     // 1: later (sub)stage: C ← C − iΩhS
  int frame_rotterm;  // with frame_term: as the rotation C ← C e^{−iΩh} (noise, bands.jl:274-286)
  double h, wmax;
  double *Om;
  int combine;        // 1: C ← μC + νA
  int combine_log;    // with combine: C ← A exp(μ log(C/A)) (noise on a KWT band, bands.jl:439-445)
  double cmu, cnu;
  const cd *A;
  int turn;           // 1: C ← C e^{iΩ dt}
  double dt;
  Rng r;              // interior nodes
  Dim d;
  // material per region (bands.jl:53-68, 168-182): the node map, the tables (stage or full-step), τ for ρ
  const uint8_t *mat;
  const MatDev *mt;
  const double *tau[3];
  int mstage;
  const uint8_t *vac;   // a sculpted sample's vacuum nodes (bands.jl:103-124)
  LinkRot lr;           // how Lx, Ly, Lz are read
  const double *Th;     // the heat model's temperature field (null: none): ε = a − θ (bands.jl:33-35)
  double heat_a;
  const double *drag;   // the drag's full-step coefficients [µ][ν][x, y, z] (null: no drag), divided by ddiv
  double ddiv;          // the pass's divisor: n substeps, or the RKL/RKC weight q (_dragof, bands.jl:195-196)
};

__device__ __forceinline__ cd kwt_update(cd g, cd dd, double g2) {
  double a2 = cabs2(g);
  double q = 1 + g2 * a2;
  cd dp = rmul(sqrt(q), dd);
  return cadd(g, csub(dp, mulr(rmul(g2, g), cmul(cconj(g), dp).x / q)));
}

__device__ __forceinline__ cd kwt_update_rot(cd g, cd dd, double g2) {
  double a2 = cabs2(g);
  double q = 1 + g2 * a2;
  cd dp = rmul(sqrt(q), dd);
  cd Dl = csub(dp, mulr(rmul(g2, g), cmul(cconj(g), dp).x / q));
  if (!(a2 > 1e-24)) return cadd(g, Dl);
  double a = sqrt(a2);
  cd u = cdivr(g, a);
  cd w = cmul(cconj(u), Dl);
  return cmul(u, rmul(a + w.x, ccis(w.y / a)));
}

// _combine_log! (bands.jl:439-445): A exp(μ log(C/A)) where |A|² and |C|² exceed 1e-3, else μC + (1−μ)A.  C/A by
// the plain formula (Julia's is its robust complex division).
__device__ __forceinline__ cd combine_log(cd c, cd a, double mu) {
  if (!(cabs2(a) > 1e-3 && cabs2(c) > 1e-3)) return cadd(rmul(mu, c), rmul(1 - mu, a));
  const double dd = a.x * a.x + a.y * a.y;
  const cd z = mkc((c.x * a.x + c.y * a.y) / dd, (c.y * a.x - c.x * a.y) / dd);
  const cd w = rmul(mu, mkc(log(hypot(z.x, z.y)), atan2(z.y, z.x)));
  return cmul(a, rmul(exp(w.x), ccis(w.y)));
}

// _dif with the link weights ρ₊, ρ₋ (bands.jl:63-64): today's expression plus k((ρ₊−1)(v₊s₊−g) + (ρ₋−1)(v₋s₋−g))
__device__ __forceinline__ cd dif_mat(double rp, double rm, double k, cd vp, cd sp, cd vm, cd sm, cd g) {
  const cd a = cmul(vp, sp), b = cmul(vm, sm);
  return cadd(rmul(k, cadd(csub(a, rmul(2.0, g)), b)), rmul(k, cadd(rmul(rp - 1, csub(a, g)), rmul(rm - 1, csub(b, g)))));
}

template <bool MAT, bool VAC, int LR>
__device__ __forceinline__ void band_stage_b(const Blk bk, StageArgs const &A);
template <bool MAT, bool VAC, int LR>
__global__ void __launch_bounds__(256, (MAT || LR) ? 4 : 5) k_band_stage(StageArgs A) { band_stage_b<MAT, VAC, LR>(TDGL_BLK, A); }
#define TDGL_STAGE_MERGE(MAT, VAC, LR) \
  TDGL_MERGEABLE((k_band_stage<MAT, VAC, LR>), (band_stage_b<MAT, VAC, LR>), 256, 4, false)
TDGL_STAGE_MERGE(false, false, 0);
TDGL_STAGE_MERGE(true, false, 0);
TDGL_STAGE_MERGE(false, true, 0);
TDGL_STAGE_MERGE(true, true, 0);
TDGL_STAGE_MERGE(false, false, 1);
TDGL_STAGE_MERGE(true, false, 1);
TDGL_STAGE_MERGE(false, true, 1);
TDGL_STAGE_MERGE(true, true, 1);
template <bool MAT, bool VAC, int LR>
__device__ __forceinline__ void band_stage_b(const Blk bk, StageArgs const &A) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= A.r.n()) return;
  int i, j, k;
  rng_ijk(A.r, t, i, j, k);
  const Dim d = A.d;
  const long long o = d.at(i, j, k);
  const long long sx = 1, sy = d.n1, sz = (long long)d.n1 * d.n2;
  auto LX = [&](long long q) { return link_at<LR>(A.lr, A.Lx, 0, q); };
  auto LY = [&](long long q) { return link_at<LR>(A.lr, A.Ly, 1, q); };
  auto LZ = [&](long long q) { return link_at<LR>(A.lr, A.Lz, 2, q); };
  cd g = A.S[o];
  double fm = A.f[o];
  cd v;
  if ((VAC && A.vac[o]) || (A.hard && fm == 0.0)) {
    v = mkc(0.0, 0.0);
  } else if (VAC) {   // _band_row_vac!: each neighbour with the mask of its link (τ, or ρ = τ·W with materials)
    const int mu = A.mu, m = MAT ? A.mat[o] - 1 : 0;
    const tdgl_bandcoef &cf = MAT ? (A.mstage ? A.mt->stage[mu][m] : A.mt->full[mu][m]) : A.cf;
    double wxp = A.tau[0][o], wxm = A.tau[0][o - sx], wyp = A.tau[1][o], wym = A.tau[1][o - sy], wzp = A.tau[2][o],
           wzm = A.tau[2][o - sz];
    if (MAT) {
      const double(*W)[TDGL_MAXMAT][TDGL_MAXMAT] = A.mt->W[mu];
      wxp *= W[0][m][A.mat[o + sx] - 1];
      wxm *= W[0][A.mat[o - sx] - 1][m];
      wyp *= W[1][m][A.mat[o + sy] - 1];
      wym *= W[1][A.mat[o - sy] - 1][m];
      wzp *= W[2][m][A.mat[o + sz] - 1];
      wzm *= W[2][A.mat[o - sz] - 1][m];
    }
    cd tx = rmul(cf.kx, cadd(rmul(wxp, csub(cmul(LX(o), A.S[o + sx]), g)), rmul(wxm, csub(cmul(cconj(LX(o - sx)), A.S[o - sx]), g))));
    cd ty = rmul(cf.ky, cadd(rmul(wyp, csub(cmul(LY(o), A.S[o + sy]), g)), rmul(wym, csub(cmul(cconj(LY(o - sy)), A.S[o - sy]), g))));
    cd tz = rmul(cf.kz, cadd(rmul(wzp, csub(cmul(LZ(o), A.S[o + sz]), g)), rmul(wzm, csub(cmul(cconj(LZ(o - sz)), A.S[o - sz]), g))));
    cd acc = cadd(cadd(cadd(cadd(g, tx), ty), tz), mulr(rmul(cf.c, g), fm * cf.eps - cf.beta * cabs2(g)));
    for (int nu = 0; nu < A.N; nu++) {
      if (nu == mu) continue;
      acc = cadd(acc, rmul(cf.cpl[nu], A.G.p[nu][o]));
    }
    if (cf.gamma2 > 0) v = A.rk ? kwt_update_rot(g, csub(acc, g), cf.gamma2) : kwt_update(g, csub(acc, g), cf.gamma2);
    else v = acc;
    if (MAT && A.mt->absent[mu][m]) v = mkc(0.0, 0.0);
  } else if (MAT) {   // the node's material: its coefficients, ρ = τ·W of each link, Ψ = 0 where the band is absent
    const int m = A.mat[o] - 1, mu = A.mu;
    const tdgl_bandcoef &cf = A.mstage ? A.mt->stage[mu][m] : A.mt->full[mu][m];
    const double(*W)[TDGL_MAXMAT][TDGL_MAXMAT] = A.mt->W[mu];
    const int mxp = A.mat[o + sx] - 1, mxm = A.mat[o - sx] - 1, myp = A.mat[o + sy] - 1, mym = A.mat[o - sy] - 1,
              mzp = A.mat[o + sz] - 1, mzm = A.mat[o - sz] - 1;
    cd vxm = cconj(LX(o - sx)), vym = cconj(LY(o - sy)), vzm = cconj(LZ(o - sz));
    cd tx = dif_mat(A.tau[0][o] * W[0][m][mxp], A.tau[0][o - sx] * W[0][mxm][m], cf.kx, LX(o), A.S[o + sx], vxm,
                    A.S[o - sx], g);
    cd ty = dif_mat(A.tau[1][o] * W[1][m][myp], A.tau[1][o - sy] * W[1][mym][m], cf.ky, LY(o), A.S[o + sy], vym,
                    A.S[o - sy], g);
    cd tz = dif_mat(A.tau[2][o] * W[2][m][mzp], A.tau[2][o - sz] * W[2][mzm][m], cf.kz, LZ(o), A.S[o + sz], vzm,
                    A.S[o - sz], g);
    const double eps = A.Th ? A.mt->a[mu][m] - A.Th[o] : cf.eps;   // _anode: the material's a (bands.jl:65-66)
    cd nl = mulr(rmul(cf.c, g), fm * eps - cf.beta * cabs2(g));
    cd acc = cadd(cadd(cadd(cadd(g, tx), ty), tz), nl);
    for (int nu = 0; nu < A.N; nu++) {
      if (nu == mu) continue;
      acc = cadd(acc, rmul(cf.cpl[nu], A.G.p[nu][o]));
    }
    if (cf.gamma2 > 0) v = A.rk ? kwt_update_rot(g, csub(acc, g), cf.gamma2) : kwt_update(g, csub(acc, g), cf.gamma2);
    else v = acc;
    if (A.mt->absent[mu][m]) v = mkc(0.0, 0.0);
  } else {
    const tdgl_bandcoef &cf = A.cf;
    cd vxm = cconj(LX(o - sx)), vym = cconj(LY(o - sy)), vzm = cconj(LZ(o - sz));
    cd g2 = rmul(2.0, g);
    cd tx = rmul(cf.kx, cadd(csub(cmul(LX(o), A.S[o + sx]), g2), cmul(vxm, A.S[o - sx])));
    cd ty = rmul(cf.ky, cadd(csub(cmul(LY(o), A.S[o + sy]), g2), cmul(vym, A.S[o - sy])));
    cd tz = rmul(cf.kz, cadd(csub(cmul(LZ(o), A.S[o + sz]), g2), cmul(vzm, A.S[o - sz])));
    const double eps = A.Th ? A.heat_a - A.Th[o] : cf.eps;
    cd nl = mulr(rmul(cf.c, g), fm * eps - cf.beta * cabs2(g));
    cd acc = cadd(cadd(cadd(cadd(g, tx), ty), tz), nl);
    for (int nu = 0; nu < A.N; nu++) {
      if (nu == A.mu) continue;
      acc = cadd(acc, rmul(cf.cpl[nu], A.G.p[nu][o]));
    }
    if (A.drag)   // _drag (bands.jl:37-51): the lattice Laplacian of every other band on this pass's links
      for (int nu = 0; nu < A.N; nu++) {
        if (nu == A.mu) continue;
        const double *c3 = A.drag + 3 * (TDGL_MAXB * A.mu + nu);
        const double cx = c3[0] / A.ddiv, cy = c3[1] / A.ddiv, cz = c3[2] / A.ddiv;
        const cd *P = A.G.p[nu];
        const cd p2 = rmul(2.0, P[o]);
        const cd ex = rmul(cx, cadd(csub(cmul(LX(o), P[o + sx]), p2), cmul(vxm, P[o - sx])));
        const cd ey = rmul(cy, cadd(csub(cmul(LY(o), P[o + sy]), p2), cmul(vym, P[o - sy])));
        const cd ez = rmul(cz, cadd(csub(cmul(LZ(o), P[o + sz]), p2), cmul(vzm, P[o - sz])));
        acc = cadd(acc, cadd(cadd(ex, ey), ez));
      }
    if (cf.gamma2 > 0) v = A.rk ? kwt_update_rot(g, csub(acc, g), cf.gamma2) : kwt_update(g, csub(acc, g), cf.gamma2);
    else v = acc;
  }
  if (A.frame_rate) {
    double a2 = cabs2(g);
    double w = 0.0;
    if (a2 > 1e-3) {
      w = cmul(cconj(g), csub(v, g)).y / (a2 * A.h);
      w = w < -A.wmax ? -A.wmax : (w > A.wmax ? A.wmax : w);
    }
    A.Om[o] = w;
    if (!A.frame_store) v = cminus_i(v, w * A.h, g);
  } else if (A.frame_term) {
    v = A.frame_rotterm ? cmul(v, ccis(-(A.Om[o] * A.h))) : cminus_i(v, A.Om[o] * A.h, g);
  }
  if (A.combine) v = A.combine_log ? combine_log(v, A.A[o], A.cmu) : cadd(rmul(A.cmu, v), rmul(A.cnu, A.A[o]));
  if (A.turn) v = cmul(v, ccis(A.Om[o] * A.dt));
  A.C[o] = v;
}

// Ω on the six faces of the block copies the node inside (bands.jl:224-232), one pass per axis.
__device__ __forceinline__ void omega_face_b(const Blk bk, double * const &Om, Dim const &d, Rng const &r, int const &axis, int const &lo, int const &hi);
__global__ void k_omega_face(double *Om, Dim d, Rng r, int axis, int lo, int hi) { omega_face_b(TDGL_BLK, Om, d, r, axis, lo, hi); }
TDGL_MERGEABLE(k_omega_face, omega_face_b, 256, 1, false);
__device__ __forceinline__ void omega_face_b(const Blk bk, double * const &Om, Dim const &d, Rng const &r, int const &axis, int const &lo, int const &hi) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= r.n()) return;
  int a, b, c;
  rng_ijk(r, t, a, b, c);
  if (axis == 0) {
    Om[d.at(lo, b, c)] = Om[d.at(lo + 1, b, c)];
    Om[d.at(hi + 1, b, c)] = Om[d.at(hi, b, c)];
  } else if (axis == 1) {
    Om[d.at(a, lo, c)] = Om[d.at(a, lo + 1, c)];
    Om[d.at(a, hi + 1, c)] = Om[d.at(a, hi, c)];
  } else {
    Om[d.at(a, b, lo)] = Om[d.at(a, b, lo + 1)];
    Om[d.at(a, b, hi + 1)] = Om[d.at(a, b, hi)];
  }
}

// Covariant Neumann ghosts of one band on one pair of faces (bands.jl:524-539).
__device__ __forceinline__ void ghost_face_b(const Blk bk, cd * const &X, const cd * const &Lk, Dim const &d, Rng const &r, int const &axis, int const &lo, int const &hi, LinkRot const &lr);
__global__ void k_ghost_face(cd *X, const cd *Lk, Dim d, Rng r, int axis, int lo, int hi, LinkRot lr) { ghost_face_b(TDGL_BLK, X, Lk, d, r, axis, lo, hi, lr); }
TDGL_MERGEABLE(k_ghost_face, ghost_face_b, 256, 1, false);
__device__ __forceinline__ void ghost_face_b(const Blk bk, cd * const &X, const cd * const &Lk, Dim const &d, Rng const &r, int const &axis, int const &lo, int const &hi, LinkRot const &lr) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= r.n()) return;
  int a, b, c;
  rng_ijk(r, t, a, b, c);
  auto L = [&](long long q) {
    return lr.mode == 0 ? link_at<0>(lr, Lk, axis, q) : link_at<1>(lr, Lk, axis, q);
  };
  if (axis == 0) {
    X[d.at(lo, b, c)] = cmul(L(d.at(lo, b, c)), X[d.at(lo + 1, b, c)]);
    X[d.at(hi + 1, b, c)] = cmul(cconj(L(d.at(hi, b, c))), X[d.at(hi, b, c)]);
  } else if (axis == 1) {
    X[d.at(a, lo, c)] = cmul(L(d.at(a, lo, c)), X[d.at(a, lo + 1, c)]);
    X[d.at(a, hi + 1, c)] = cmul(cconj(L(d.at(a, hi, c))), X[d.at(a, hi, c)]);
  } else {
    X[d.at(a, b, lo)] = cmul(L(d.at(a, b, lo)), X[d.at(a, b, lo + 1)]);
    X[d.at(a, b, hi + 1)] = cmul(cconj(L(d.at(a, b, hi))), X[d.at(a, b, hi)]);
  }
}

// The three face passes of ghosts! in one launch: every point of the block's shell evaluates the writes that reach
// it in the reference's order (x faces, then y, then z).  A z-face point takes the z pass over the value the y or x
// pass left at z1+1 / z2, a y-face point (k inside) the y pass over the x pass's value, an x-face point (j, k inside)
// the x pass.  Every array value read is a node inside the block, which no pass writes, so the threads do not race;
// the products are the reference's, in its order.
struct ShellArgs {
  cd *X;
  const cd *Lx, *Ly, *Lz;
  int x1, x2, y1, y2, z1, z2;
  long long nz_face, ny_face;   // points of the two z faces; of the two y faces (k inside)
  long long n;                  // all shell points
  Dim d;
  LinkRot lr;                   // how Lx, Ly, Lz are read
};

__device__ __forceinline__ void ghost_shell_b(const Blk bk, ShellArgs const &A);
__global__ void k_ghost_shell(ShellArgs A) { ghost_shell_b(TDGL_BLK, A); }
TDGL_MERGEABLE(k_ghost_shell, ghost_shell_b, 256, 1, false);
__device__ __forceinline__ void ghost_shell_b(const Blk bk, ShellArgs const &A) {
  const long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= A.n) return;
  const Dim d = A.d;
  const int x1 = A.x1, x2 = A.x2, y1 = A.y1, y2 = A.y2, z1 = A.z1, z2 = A.z2;
  const int ni = x2 - x1 + 2, nj = y2 - y1 + 2, nk = z2 - z1;   // the block's nodes per axis; inside k
  const cd *X = A.X;
  auto lk = [&](const cd *L, int ax, long long q) {
    return A.lr.mode == 0 ? L[q] : link_at<1>(A.lr, L, ax, q);
  };
  // the value each pass writes at (i, j, k), from the values before it
  auto vx = [&](int i, int j, int k) -> cd {   // x pass (reads the inside column)
    return i == x1 ? cmul(lk(A.Lx, 0, d.at(x1, j, k)), X[d.at(x1 + 1, j, k)]) : cmul(cconj(lk(A.Lx, 0, d.at(x2, j, k))), X[d.at(x2, j, k)]);
  };
  auto after_x = [&](int i, int j, int k) -> cd { return (i == x1 || i == x2 + 1) ? vx(i, j, k) : X[d.at(i, j, k)]; };
  auto vy = [&](int i, int j, int k) -> cd {   // y pass over the x pass
    return j == y1 ? cmul(lk(A.Ly, 1, d.at(i, y1, k)), after_x(i, y1 + 1, k)) : cmul(cconj(lk(A.Ly, 1, d.at(i, y2, k))), after_x(i, y2, k));
  };
  auto after_y = [&](int i, int j, int k) -> cd { return (j == y1 || j == y2 + 1) ? vy(i, j, k) : after_x(i, j, k); };
  int i, j, k;
  cd v;
  if (t < A.nz_face) {                       // z faces: every (i, j)
    const unsigned u = (unsigned)(t / 2), w = u / (unsigned)ni;   // 32-bit: the shell has fewer than 2^31 points
    i = x1 + (int)(u - w * (unsigned)ni);
    j = y1 + (int)w;
    k = (t & 1) ? z2 + 1 : z1;
    v = k == z1 ? cmul(lk(A.Lz, 2, d.at(i, j, z1)), after_y(i, j, z1 + 1)) : cmul(cconj(lk(A.Lz, 2, d.at(i, j, z2))), after_y(i, j, z2));
  } else if (t < A.nz_face + A.ny_face) {    // y faces, k inside
    const unsigned u = (unsigned)((t - A.nz_face) / 2), w = u / (unsigned)ni;
    i = x1 + (int)(u - w * (unsigned)ni);
    k = z1 + 1 + (int)w;
    j = ((t - A.nz_face) & 1) ? y2 + 1 : y1;
    v = vy(i, j, k);
  } else {                                   // x faces, j and k inside
    const unsigned u = (unsigned)((t - A.nz_face - A.ny_face) / 2), w = u / (unsigned)(nj - 2);
    j = y1 + 1 + (int)(u - w * (unsigned)(nj - 2));
    k = z1 + 1 + (int)w;
    i = ((t - A.nz_face - A.ny_face) & 1) ? x2 + 1 : x1;
    v = vx(i, j, k);
  }
  (void)nk;
  A.X[d.at(i, j, k)] = v;
}

// Link operations over the three link ranges of the band stencil (_rx, _ry, _rz, bands.jl:349-351).
enum LinkOp { LOP_ROT_INIT = 0, LOP_ADVANCE, LOP_FRAME_LINKS, LOP_LINK_RATE, LOP_ROTLINKS, LOP_ROTFRAC };

struct LinkArgs {
  int op;
  Rng r[3];
  Dim d;
  cd *L[3], *Rl[3];
  const cd *V[3], *U[3];
  double *Rr[3];
  const double *Om;
  double par;   // n (ROT_INIT), τ (FRAME_LINKS), dt (LINK_RATE), c (ROTLINKS / ROTFRAC)
};

// The per-link formulas (bands.jl:303-310 _link_rate!, :355-369 _rot!, :409-423 _rotfrac!), shared by the step's
// link passes and by tdgl_link_rotations.  −arg q of q = V conj(U), with the short series while Re q > 0 and
// |sin| <= 0.05:
__device__ __forceinline__ double link_angle(cd v, cd u) {
  const cd q = cmul(v, cconj(u));
  const double sf = -q.y;
  return (q.x > 0 && fabs(sf) <= 0.05) ? -(sf + sf * sf * sf / 6) : cangle(q);
}
// Q^{1/n}
__device__ __forceinline__ cd link_root(cd v, cd u, double n) {
  const cd q = cmul(v, cconj(u));
  const double sf = -q.y;
  if (q.x > 0 && fabs(sf) <= 0.05) {
    const double a = (sf + sf * sf * sf / 6) / n;
    const double a2 = a * a;
    return mkc(1 - a2 / 2, -a * (1 - a2 / 6));
  }
  return ccis(cangle(q) / n);
}
// V Q^c
__device__ __forceinline__ cd link_frac(cd v, cd u, double c) {
  const cd q = cmul(v, cconj(u));
  const double sf = -q.y;
  if (q.x > 0 && fabs(sf) <= 0.05) {
    const double a = (sf + sf * sf * sf / 6) * c;
    const double a2 = a * a;
    return cmul(v, mkc(1 - a2 / 2, -a * (1 - a2 / 6)));
  }
  return cmul(v, ccis(cangle(q) * c));
}

__device__ __forceinline__ void link_op_b(const Blk bk, LinkArgs const &A);
__global__ void __launch_bounds__(256, 5) k_link_op(LinkArgs A) { link_op_b(TDGL_BLK, A); }
TDGL_MERGEABLE(k_link_op, link_op_b, 256, 1, false);
__device__ __forceinline__ void link_op_b(const Blk bk, LinkArgs const &A) {
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
  const int oi = ax == 0, oj = ax == 1, ok = ax == 2;
  switch (A.op) {
    case LOP_ROT_INIT: {
      const cd v = A.V[ax][o];
      A.L[ax][o] = v;
      A.Rl[ax][o] = link_root(v, A.U[ax][o], A.par);
      break;
    }
    case LOP_ADVANCE:
      A.L[ax][o] = cmul(A.L[ax][o], A.Rl[ax][o]);
      break;
    case LOP_FRAME_LINKS:
      A.L[ax][o] = cmul(A.L[ax][o], ccis_short((A.Om[A.d.at(i + oi, j + oj, k + ok)] - A.Om[o]) * A.par));
      break;
    case LOP_LINK_RATE:
      A.Rr[ax][o] = link_angle(A.V[ax][o], A.U[ax][o]) + (A.Om[A.d.at(i + oi, j + oj, k + ok)] - A.Om[o]) * A.par;
      break;
    case LOP_ROTLINKS:
      A.L[ax][o] = cmul(A.V[ax][o], ccis_short(A.Rr[ax][o] * A.par));
      break;
    case LOP_ROTFRAC:
      A.L[ax][o] = link_frac(A.V[ax][o], A.U[ax][o], A.par);
      break;
  }
}

__device__ __forceinline__ void copy_c_b(const Blk bk, cd * const &dst, const cd * const &src, long long const &n);
__global__ void k_copy_c(cd *dst, const cd *src, long long n) { copy_c_b(TDGL_BLK, dst, src, n); }
TDGL_MERGEABLE(k_copy_c, copy_c_b, 256, 1, false);
__device__ __forceinline__ void copy_c_b(const Blk bk, cd * const &dst, const cd * const &src, long long const &n) {
  long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = src[t];
}

namespace {

const int BS = 256;

Rng interior(const Geo &g) { return mkrng(g.x1 + 1, g.x2, g.y1 + 1, g.y2, g.z1 + 1, g.z2); }

void link_op(Ctx *ctx, int op, double par) {
  const Geo &g = ctx->g;
  LinkArgs A;
  A.op = op;
  A.r[0] = mkrng(g.x1, g.x2, g.y1, g.y2 + 1, g.z1, g.z2 + 1);
  A.r[1] = mkrng(g.x1, g.x2 + 1, g.y1, g.y2, g.z1, g.z2 + 1);
  A.r[2] = mkrng(g.x1, g.x2 + 1, g.y1, g.y2 + 1, g.z1, g.z2);
  A.d = g.d;
  for (int ax = 0; ax < 3; ax++) {
    A.L[ax] = ctx->L[ax]; A.Rl[ax] = ctx->Rl[ax]; A.V[ax] = ctx->V[ax]; A.U[ax] = ctx->U[ax]; A.Rr[ax] = ctx->Rr[ax];
  }
  A.Om = ctx->Om;
  A.par = par;
  long long n = A.r[0].n() + A.r[1].n() + A.r[2].n();
  static const double per[6] = {64, 48, 40, 48, 40, 48};   // compulsory bytes per link of each operation
  TDGL_LAUNCH(ctx, K_LINK, per[op] * n, k_link_op, nblk(n, BS), BS, 0, A);
}

StageArgs stage_base(Ctx *ctx, int mu, const tdgl_bandcoef &cf, double ddiv) {
  StageArgs A;
  memset(&A, 0, sizeof(A));
  for (int nu = 0; nu < ctx->N; nu++) A.G.p[nu] = ctx->G[nu];
  A.f = ctx->f;
  A.cf = cf;
  A.mu = mu;
  A.N = ctx->N;
  A.hard = ctx->P.hard;
  A.rk = ctx->P.noise_on;
  A.Om = ctx->Om;
  A.dt = ctx->P.dt;
  A.wmax = 0.5 / ctx->P.dt;
  A.r = interior(ctx->g);
  A.d = ctx->g.d;
  A.mat = ctx->mat;
  A.mt = ctx->mt;
  for (int ax = 0; ax < 3; ax++) A.tau[ax] = ctx->tau[ax];
  A.mstage = &cf == &ctx->P.bcs[mu];   // the stage table where the band's stage coefficients are in use
  A.vac = ctx->vac;
  A.drag = ctx->drag_c;
  A.ddiv = ddiv;
  A.Th = ctx->P.heat_on ? ctx->Th : nullptr;
  A.heat_a = ctx->P.heat_a[mu];
  return A;
}

// compulsory bytes per interior node: S, C, f, three links, the other bands, and the epilogue's A and Ω
double stage_bytes(const StageArgs &A) {
  double b = 16 + 16 + 8 + 48 + 16.0 * (A.N - 1);
  if (A.lr.mode == 1) b += 24;   // the rate R beside the links V
  if (A.combine) b += 16;
  if (A.frame_rate || A.frame_term || A.turn) b += 8;
  if (A.mat || A.vac) b += 24 + 1;   // τ along the three axes, the node's material or vacuum flag
  if (A.drag) b += 16.0 * (A.N - 1);   // the other bands' neighbours come from the cache
  return b * (double)A.r.n();
}

void launch_stage(Ctx *ctx, const StageArgs &A) {
  const long long nb = nblk(A.r.n(), BS);
  const double by = stage_bytes(A);
#define TDGL_STAGE_LAUNCH(LR)                                                                        \
  do {                                                                                               \
    if (A.vac && A.mat) TDGL_LAUNCH(ctx, K_BAND, by, (k_band_stage<true, true, LR>), nb, BS, 0, A);   \
    else if (A.vac) TDGL_LAUNCH(ctx, K_BAND, by, (k_band_stage<false, true, LR>), nb, BS, 0, A);      \
    else if (A.mat) TDGL_LAUNCH(ctx, K_BAND, by, (k_band_stage<true, false, LR>), nb, BS, 0, A);      \
    else TDGL_LAUNCH(ctx, K_BAND, by, (k_band_stage<false, false, LR>), nb, BS, 0, A);               \
  } while (0)
  if (A.lr.mode == 1) TDGL_STAGE_LAUNCH(1);
  else TDGL_STAGE_LAUNCH(0);
#undef TDGL_STAGE_LAUNCH
}

void band_euler(Ctx *ctx, int mu) {
  const bool noise = ctx->P.noise_on != 0;
  StageArgs A = stage_base(ctx, mu, ctx->P.bc[mu], 1.0);
  A.C = ctx->F[mu];
  A.S = ctx->G[mu];
  A.Lx = ctx->V[0]; A.Ly = ctx->V[1]; A.Lz = ctx->V[2];
  if (ctx->P.rotframe) {
    A.frame_rate = 1;
    A.frame_store = noise;
    A.h = ctx->P.dt;
    A.turn = !noise;
  }
  launch_stage(ctx, A);
  if (ctx->P.rotframe && noise) {   // the low-passed rate, its rotation, then the turn back (bands.jl:336-339)
    omega_faces(ctx);
    frame_smooth_rot(ctx, ctx->F[mu], ctx->P.dt);
    frame_rot(ctx, ctx->F[mu], -ctx->P.dt);
  }
}

void band_substeps(Ctx *ctx, int mu, int n) {
  const bool rot = ctx->P.rotframe != 0, ex = ctx->P.extrap != 0, noise = ctx->P.noise_on != 0;
  const cd *L[3] = {ctx->V[0], ctx->V[1], ctx->V[2]};
  if (ex) {
    link_op(ctx, LOP_ROT_INIT, (double)n);
    for (int ax = 0; ax < 3; ax++) L[ax] = ctx->L[ax];
  }
  const cd *src = ctx->G[mu];
  const double h = ctx->P.dt / n;
  for (int m = 1; m <= n; m++) {
    cd *dst = ((n - m) % 2 == 0) ? ctx->F[mu] : ctx->W;
    StageArgs A = stage_base(ctx, mu, ctx->P.bcs[mu], (double)n);
    A.C = dst;
    A.S = src;
    A.Lx = L[0]; A.Ly = L[1]; A.Lz = L[2];
    A.h = h;
    if (rot) {
      if (m == 1) {
        A.frame_rate = 1;
        A.frame_store = noise;
      } else {
        A.frame_term = 1;
        A.frame_rotterm = noise;
      }
      if (m == n) A.turn = 1;
    }
    launch_stage(ctx, A);
    if (rot && noise && m == 1) {
      omega_faces(ctx);
      frame_smooth_rot(ctx, dst, h);
    }
    if (m < n) {
      if (rot && m == 1) omega_faces(ctx);
      if (ex) link_op(ctx, LOP_ADVANCE, 0.0);
      if (rot) link_op(ctx, LOP_FRAME_LINKS, h);
      ghosts(ctx, dst, L[0], L[1], L[2]);
    }
    src = dst;
  }
}

void band_rkl(Ctx *ctx, int mu, int ns) {
  const tdgl_params &P = ctx->P;
  const bool kc = P.use_rkc[mu] != 0, rot = P.rotframe != 0, ex = P.extrap != 0, noise = P.noise_on != 0;
  const bool skq = skrock_band(ctx, mu), lg = noise && haskwt(ctx, mu);
  const double q = kc ? P.rkc_q[mu] : (double)(ns * (ns + 1) / 2);
  const double h = P.dt / q;
  const cd *L[3] = {ctx->V[0], ctx->V[1], ctx->V[2]};
  cd *buf[3] = {ctx->W, ctx->W2, ctx->F[mu]};
  const cd *A_ = ctx->G[mu], *B = ctx->G[mu];
  cd *Cc = ctx->W;
  // the links of stage j > 1 are the step's links rotated to the fraction c_{j−1} of the step, formed where the stage
  // and its ghosts read them (no stored copy)
  LinkRot lr;
  memset(&lr, 0, sizeof(lr));
  for (int ax = 0; ax < 3; ax++) {
    lr.V[ax] = ctx->V[ax];
    lr.U[ax] = ctx->U[ax];
    lr.R[ax] = ctx->Rr[ax];
  }
  for (int j = 1; j <= ns; j++) {
    Cc = buf[(j - 1) % 3];
    const cd *src = B;
    if (j == 1 && skq) {   // SK-ROCK for the phase: K₁ = E(Ψⁿ e^{iν₁δθ}) e^{i(κ₁−ν₁)δθ} (bands.jl:482-488)
      sk_turn(ctx, ctx->W2, B, mu, P.rkc_sk[mu][0]);
      ghosts(ctx, ctx->W2, L[0], L[1], L[2]);
      src = ctx->W2;
    }
    StageArgs A = stage_base(ctx, mu, P.bcs[mu], q);
    A.C = Cc;
    A.S = src;
    A.Lx = L[0]; A.Ly = L[1]; A.Lz = L[2];
    A.lr = lr;
    A.h = h;
    if (rot) {
      if (j == 1) {
        A.frame_rate = 1;
        A.frame_store = noise;
      } else {
        A.frame_term = 1;
        A.frame_rotterm = noise;
      }
    }
    if (j >= 2) {
      A.combine = 1;
      A.combine_log = lg;
      A.cmu = kc ? P.rkc_mu[mu][j - 1] : (double)(2 * j - 1) / j;
      A.cnu = kc ? P.rkc_nu[mu][j - 1] : (double)(1 - j) / j;
      A.A = A_;
    }
    const bool late_turn = j == ns && rot && j == 1 && noise;   // the turn follows the low-passed rate
    if (j == ns && rot && !late_turn) A.turn = 1;
    launch_stage(ctx, A);
    if (j == 1 && rot && noise) {
      omega_faces(ctx);
      frame_smooth_rot(ctx, Cc, h);
    }
    if (j == 1 && skq) sk_turn(ctx, Cc, Cc, mu, P.rkc_sk[mu][1] - P.rkc_sk[mu][0]);
    if (late_turn) frame_rot(ctx, Cc, -P.dt);
    if (rot && j == 1 && ex && ns > 1) {
      omega_faces(ctx);
      link_op(ctx, LOP_LINK_RATE, P.dt);
    }
    if (j < ns) {
      if (ex) {
        const double c = kc ? P.rkc_c[mu][j - 1] : (double)(j * (j + 1)) / (double)(ns * (ns + 1));
        if (rot) {
          lr.mode = 1;
          lr.c = c;
        } else {
          link_op(ctx, LOP_ROTFRAC, c);
          for (int ax = 0; ax < 3; ax++) L[ax] = ctx->L[ax];
        }
      }
      ghosts(ctx, Cc, L[0], L[1], L[2], &lr);
    }
    A_ = B;
    B = Cc;
  }
  if (Cc != ctx->F[mu]) {
    long long n = ctx->g.d.n();
    TDGL_LAUNCH(ctx, K_COPY, 32.0 * n, k_copy_c, nblk(n, BS), BS, 0, ctx->F[mu], Cc, n);
  }
}

}  // namespace

// Ω on the six faces copies the node inside (bands.jl:224-232, precedence x, y, z)
void omega_faces(Ctx *ctx) {
  const Geo &g = ctx->g;
  Rng r0 = mkrng(0, 0, g.y1 + 1, g.y2, g.z1 + 1, g.z2);
  Rng r1 = mkrng(g.x1, g.x2 + 1, 0, 0, g.z1 + 1, g.z2);
  Rng r2 = mkrng(g.x1, g.x2 + 1, g.y1, g.y2 + 1, 0, 0);
  r0.ni = 1; r1.nj = 1; r2.nk = 1;
  TDGL_LAUNCH(ctx, K_OMEGA, 32.0 * r0.n(), k_omega_face, nblk(r0.n(), BS), BS, 0, ctx->Om, g.d, r0, 0, g.x1, g.x2);
  TDGL_LAUNCH(ctx, K_OMEGA, 32.0 * r1.n(), k_omega_face, nblk(r1.n(), BS), BS, 0, ctx->Om, g.d, r1, 1, g.y1, g.y2);
  TDGL_LAUNCH(ctx, K_OMEGA, 32.0 * r2.n(), k_omega_face, nblk(r2.n(), BS), BS, 0, ctx->Om, g.d, r2, 2, g.z1, g.z2);
}

void ghosts(Ctx *ctx, cd *X, const cd *Lx, const cd *Ly, const cd *Lz, const LinkRot *lrp) {
  const Geo &g = ctx->g;
  LinkRot lr;
  memset(&lr, 0, sizeof(lr));
  if (lrp) lr = *lrp;
  if (g.x2 < g.x1 + 1 || g.y2 < g.y1 + 1 || g.z2 < g.z1 + 1) {   // a block one cell thick: the passes read ghosts
    Rng r0 = mkrng(1, 1, g.y1, g.y2 + 1, g.z1, g.z2 + 1);
    Rng r1 = mkrng(g.x1, g.x2 + 1, 1, 1, g.z1, g.z2 + 1);
    Rng r2 = mkrng(g.x1, g.x2 + 1, g.y1, g.y2 + 1, 1, 1);
    TDGL_LAUNCH(ctx, K_GHOST, 96.0 * r0.n(), k_ghost_face, nblk(r0.n(), BS), BS, 0, X, Lx, g.d, r0, 0, g.x1, g.x2, lr);
    TDGL_LAUNCH(ctx, K_GHOST, 96.0 * r1.n(), k_ghost_face, nblk(r1.n(), BS), BS, 0, X, Ly, g.d, r1, 1, g.y1, g.y2, lr);
    TDGL_LAUNCH(ctx, K_GHOST, 96.0 * r2.n(), k_ghost_face, nblk(r2.n(), BS), BS, 0, X, Lz, g.d, r2, 2, g.z1, g.z2, lr);
    return;
  }
  ShellArgs A;
  A.X = X;
  A.Lx = Lx; A.Ly = Ly; A.Lz = Lz;
  A.x1 = g.x1; A.x2 = g.x2; A.y1 = g.y1; A.y2 = g.y2; A.z1 = g.z1; A.z2 = g.z2;
  const long long ni = g.x2 - g.x1 + 2, nj = g.y2 - g.y1 + 2, nk = g.z2 - g.z1 + 2;
  A.nz_face = 2 * ni * nj;
  A.ny_face = 2 * ni * (nk - 2);
  A.n = A.nz_face + A.ny_face + 2 * (nj - 2) * (nk - 2);
  A.d = g.d;
  A.lr = lr;
  // per shell point: the point, its link and the inside value(s) it reads (up to three of each on edges)
  TDGL_LAUNCH(ctx, K_GHOST, 48.0 * A.n, k_ghost_shell, nblk(A.n, BS), BS, 0, A);
}

struct BandOut {
  cd *p[TDGL_MAXB];
};

__device__ __forceinline__ void vacuum_zero_b(const Blk bk, BandOut const &F, int const &N, const uint8_t * const &vac, long long const &n);
__global__ void k_vacuum_zero(BandOut F, int N, const uint8_t *vac, long long n) { vacuum_zero_b(TDGL_BLK, F, N, vac, n); }
TDGL_MERGEABLE(k_vacuum_zero, vacuum_zero_b, 256, 1, false);
__device__ __forceinline__ void vacuum_zero_b(const Blk bk, BandOut const &F, int const &N, const uint8_t * const &vac, long long const &n) {
  const long long t = (long long)bk.x * blockDim.x + threadIdx.x;
  if (t >= n || !vac[t]) return;
  for (int mu = 0; mu < N; mu++) F.p[mu][t] = mkc(0.0, 0.0);
}

void vacuum_zero(Ctx *ctx) {
  BandOut F;
  for (int mu = 0; mu < ctx->N; mu++) F.p[mu] = ctx->F[mu];
  const long long n = ctx->g.d.n();
  TDGL_LAUNCH(ctx, K_GHOST, 1.0 * n, k_vacuum_zero, nblk(n, BS), BS, 0, F, ctx->N, ctx->vac, n);
}

static void use_ws(Ctx *ctx, const Ctx::BandWs &w) {
  ctx->W = w.W;
  ctx->W2 = w.W2;
  ctx->Om = w.Om;
  ctx->Oms = w.Oms;
  for (int ax = 0; ax < 3; ax++) {
    ctx->L[ax] = w.L[ax];
    ctx->Rl[ax] = w.Rl[ax];
    ctx->Rr[ax] = w.Rr[ax];
  }
}

// update_bands! (bands.jl:330-346).  Each band reads the state at the start of the step (its own Ψ and, for the
// coupling and the drag, the other bands' G) and writes only its F[µ]: band µ ≥ 1 runs on its own stream with its
// own workspaces, forked from the context's stream and joined back (parallel branches of a captured step).  When the
// launches are timed one by one the bands run in order on the one stream; the results are the same.
int update_bands(Ctx *ctx) {
  const bool par = ctx->N > 1 && ctx->branches && !ctx->prof.on && ctx->bstream[1];
  cudaStream_t main = ctx->stream;
  if (par) cudaEventRecord(ctx->bev[0], main);
  for (int mu = 0; mu < ctx->N; mu++) {
    if (par && mu > 0) {
      cudaStreamWaitEvent(ctx->bstream[mu], ctx->bev[0], 0);
      ctx->stream = ctx->bstream[mu];
    }
    use_ws(ctx, ctx->bws[par ? mu : 0]);
    int n = ctx->P.nsub[mu];
    if (ctx->P.stages[mu] > 0) band_rkl(ctx, mu, ctx->P.stages[mu]);
    else if (n == 1) band_euler(ctx, mu);
    else band_substeps(ctx, mu, n);
    if (par && mu > 0) {
      cudaEventRecord(ctx->bev[mu], ctx->bstream[mu]);
      ctx->stream = main;
    }
  }
  use_ws(ctx, ctx->bws[0]);
  if (par)
    for (int mu = 1; mu < ctx->N; mu++) cudaStreamWaitEvent(main, ctx->bev[mu], 0);
  return 0;
}

}  // namespace tdgl

// ---------------------------------------------------------------------------------------------- link rotations alone
// The step's per-link rotation formulas on caller arrays (the reference drives its device kernels the same way on
// manufactured links, gpu/TDGLGPU/test/test_link_rotations.jl:21-60).
namespace {
struct RotArgs {
  int op, ax, i0, j0, k0, ni, nj, nk;
  Dim d;
  const cd *V, *U;
  const double *Om;
  double par;
  cd *L, *R;
  double *Rr;
};
__global__ void k_rotations(RotArgs A) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)A.ni * A.nj * A.nk) return;
  const int i = A.i0 + (int)(t % A.ni), j = A.j0 + (int)((t / A.ni) % A.nj), k = A.k0 + (int)(t / ((long long)A.ni * A.nj));
  const long long o = A.d.at(i, j, k);
  if (A.op == 0) {
    A.L[o] = A.V[o];
    A.R[o] = tdgl::link_root(A.V[o], A.U[o], A.par);
  } else if (A.op == 1) {
    A.L[o] = tdgl::link_frac(A.V[o], A.U[o], A.par);
  } else {
    A.Rr[o] = tdgl::link_angle(A.V[o], A.U[o]) +
              (A.Om[A.d.at(i + (A.ax == 0), j + (A.ax == 1), k + (A.ax == 2))] - A.Om[o]) * A.par;
  }
}
}  // namespace

extern "C" int tdgl_link_rotations(int32_t op, int32_t n1, int32_t n2, int32_t n3, const int32_t *rng, int32_t ax,
                                   const double *V, const double *U, const double *Om, double par, double *L, double *R) {
  if (op < 0 || op > 2 || ax < 0 || ax > 2 || n1 < 1 || n2 < 1 || n3 < 1 || !rng || !V || !U) return TDGL_EINVAL;
  if ((op == 0 && (!L || !R)) || (op == 1 && !L) || (op == 2 && (!Om || !R))) return TDGL_EINVAL;
  const int oi = ax == 0, oj = ax == 1, ok = ax == 2;
  const bool rate = op == 2;
  // every point of the range, and its neighbour along ax for the rate, lies inside the arrays
  if (rng[0] < 1 || rng[2] < 1 || rng[4] < 1 || rng[1] + (rate ? oi : 0) > n1 || rng[3] + (rate ? oj : 0) > n2 ||
      rng[5] + (rate ? ok : 0) > n3 || rng[1] < rng[0] || rng[3] < rng[2] || rng[5] < rng[4])
    return TDGL_EINVAL;
  const size_t n = (size_t)n1 * n2 * n3;
  std::vector<void *> bufs;
  auto dev = [&](size_t bytes, const void *src) -> void * {
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    bufs.push_back(p);
    if (src) cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
    else cudaMemset(p, 0, bytes);
    return p;
  };
  RotArgs A;
  A.op = op; A.ax = ax;
  A.i0 = rng[0]; A.j0 = rng[2]; A.k0 = rng[4];
  A.ni = rng[1] - rng[0] + 1; A.nj = rng[3] - rng[2] + 1; A.nk = rng[5] - rng[4] + 1;
  A.d.n1 = n1; A.d.n2 = n2; A.d.n3 = n3;
  A.par = par;
  A.V = (const cd *)dev(n * sizeof(cd), V);
  A.U = (const cd *)dev(n * sizeof(cd), U);
  A.Om = rate ? (const double *)dev(n * sizeof(double), Om) : nullptr;
  A.L = op != 2 ? (cd *)dev(n * sizeof(cd), L) : nullptr;
  A.R = op == 0 ? (cd *)dev(n * sizeof(cd), R) : nullptr;
  A.Rr = rate ? (double *)dev(n * sizeof(double), R) : nullptr;
  int rc = TDGL_OK;
  if (!A.V || !A.U || (rate && (!A.Om || !A.Rr)) || (op != 2 && !A.L) || (op == 0 && !A.R)) rc = TDGL_ENOMEM;
  if (rc == TDGL_OK) {
    const long long cnt = (long long)A.ni * A.nj * A.nk;
    k_rotations<<<(unsigned)((cnt + 255) / 256), 256>>>(A);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && A.L) e = cudaMemcpy(L, A.L, n * sizeof(cd), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && A.R) e = cudaMemcpy(R, A.R, n * sizeof(cd), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && A.Rr) e = cudaMemcpy(R, A.Rr, n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = TDGL_ECUDA;
  }
  for (void *p : bufs) cudaFree(p);
  return rc;
}
