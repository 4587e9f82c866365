// oracle.cpp — CPU restatement of the gtdgl (juliaTDGL 2) step, used ONLY as the parity checker.
//
// TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library.
// The product (juliatdgl_b200/, libtdgl_b200.so) never links or calls it.
//
// It restates, function by function and in the reference's order of floating-point operations, the step of
// gtdgl/src/step.jl:13-35:
//   bands      gtdgl/src/bands.jl   _band_row! :71-97, _drag :37-51 (with _dragof :195-196), kwt_update :135-140, kwt_update_rot :151-159,
//              _frame_rate! :213-234, _frame_term! :274-286, _cis :289, _frame_links! :292-297,
//              _link_rate! :303-310, _rotlinks! :311-316, _frame_turn! :321-327, update_bands! :330-346,
//              _rot! :355-369, _advance_links! :371-376, _band_substeps! :378-406, _rotfrac! :409-423,
//              _combine! :425-430, _band_rkl! :464-521, ghosts! :524-539
//   field      gtdgl/src/field.jl   supercurrent! :19-46, field_increment! :84-102, links! :105-121,
//              curl_h! :124-137, field_bc! :189-228, neumann! :231-245, advance! :248-263
//   implicit   gtdgl/src/implicit.jl SepSolver :15-104 (with the exact DCT-II / DST-I bases of the SVD of the
//              forward difference, to which _sep_bases :15-22 is equal up to column signs that cancel),
//              PCG :212-334, _precond32! :346-373, _implicit_curl_fast! :376-446, scale_increment! :337-342
//   open BC    gtdgl/src/openbc.jl  _lgf :95-96, OpenBC :111-136, _delta_current! :139-154, _convolve! :157-166,
//              _face_field! :169-183, open_update! :191-207, _open_add! :210-223
//   noise      gtdgl/src/noise.jl   noise_kick! :40-66, _kwt_kick :77-91, noise_draw! :101-123, noise_apply! :125-151,
//              _noise_kick_mat! :156-180, field_kick! :183-198; bands.jl _frame_rate_smooth! :243-272,
//              _combine_log! :439-445, _sk_turn! :447-453
//   vacuum     gtdgl/src/bands.jl _band_row_vac! :103-124, field.jl neumann! :235-244 (the vacuum ghosts)
//   materials  gtdgl/src/materials.jl MatField :83-114 (the link weights ρ), bands.jl _coefs/_dif :53-68 and the
//              absent bands :168-182, field.jl _supercurrent_mat! :48-71
//   terms      gtdgl/src/terms.jl heat_step! :58-130, _heat_step_mat! :134-202; exchange.jl (normal fluids per band: two
//              bands or N fluids, one material; QPSolve's CG in a sculpted sample) _conv :303-335, _qp_apply! :52-84,
//              _qp_cg! :87-121, qp_potential! :343-385 and
//              :478-514, _qp_sep! :271-277, qp_turn! :403-414 and :533-543
// Xoshiro's randn (noise.jl:28) is replaced by Philox4x32-10 normals on (seed, step, stream, node).
// FFTW's rfft/irfft (FFTW_jll 3.3.12) is replaced by a plain mixed-radix complex DFT of the same padded arrays:
// the same transform up to rounding.
//
// Build: oracle/Makefile (-O2 -fno-fast-math -ffp-contract=off, so no FMA contraction: the reference is plain
// IEEE double arithmetic without muladd).
#include "../include/tdgl_b200.h"

#include <omp.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct cd {
  double re, im;
};
inline cd C(double r, double i) { return cd{r, i}; }
inline cd operator+(cd a, cd b) { return cd{a.re + b.re, a.im + b.im}; }
inline cd operator-(cd a, cd b) { return cd{a.re - b.re, a.im - b.im}; }
inline cd operator*(cd a, cd b) { return cd{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cd operator*(double x, cd a) { return cd{x * a.re, x * a.im}; }
inline cd operator*(cd a, double x) { return cd{a.re * x, a.im * x}; }
inline cd operator/(cd a, double x) { return cd{a.re / x, a.im / x}; }
inline cd conj(cd a) { return cd{a.re, -a.im}; }
inline double abs2(cd a) { return a.re * a.re + a.im * a.im; }
inline cd cis(double x) { return cd{std::cos(x), std::sin(x)}; }
inline double angle(cd a) { return std::atan2(a.im, a.re); }
// e^{ia}: short series while |a| <= 0.05 (bands.jl:289)
inline cd cis_short(double a) {
  if (std::fabs(a) <= 0.05) {
    double a2 = a * a;
    return cd{1 - a2 / 2, a * (1 - a2 / 6)};
  }
  return cis(a);
}
// C - im*(w*h)*y  (bands.jl:221, :283): Complex{Bool} im times a real is (±0, x); the product with y then has
// real part ±0 - x*y.im and imaginary part ±0 + x*y.re.
inline cd minus_i_times(cd c, double x, cd y) { return cd{c.re - (0.0 * y.re - x * y.im), c.im - (0.0 * y.im + x * y.re)}; }

template <class T>
struct A3 {
  int n1 = 0, n2 = 0, n3 = 0;
  std::vector<T> v;
  void init(int a, int b, int c) {
    n1 = a; n2 = b; n3 = c;
    v.assign((size_t)a * b * c, T{});
  }
  // 1-based, as the reference
  T &operator()(int i, int j, int k) { return v[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (k - 1))]; }
  const T &operator()(int i, int j, int k) const {
    return v[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (k - 1))];
  }
  size_t size() const { return v.size(); }
};
typedef A3<double> R3;
typedef A3<cd> C3;
typedef A3<float> F3;

// ---------------------------------------------------------------------------------------------- FFT
void fft1(std::vector<cd> &a, int sign) {
  const int n = (int)a.size();
  if (n <= 1) return;
  int p = 2;
  while (p * p <= n && n % p) p++;
  if (n % p) p = n;
  const int m = n / p;
  std::vector<cd> out(n);
  if (p == n) {
    for (int k = 0; k < n; k++) {
      cd s{0, 0};
      for (int t = 0; t < n; t++) {
        long long e = ((long long)k * t) % n;
        double ang = sign * 2.0 * M_PI * (double)e / n;
        s = s + a[t] * cd{std::cos(ang), std::sin(ang)};
      }
      out[k] = s;
    }
    a.swap(out);
    return;
  }
  std::vector<std::vector<cd>> sub(p, std::vector<cd>(m));
  for (int r = 0; r < p; r++)
    for (int t = 0; t < m; t++) sub[r][t] = a[(size_t)t * p + r];
  for (int r = 0; r < p; r++) fft1(sub[r], sign);
  for (int q = 0; q < p; q++)
    for (int k = 0; k < m; k++) {
      int kk = k + m * q;
      cd s{0, 0};
      for (int r = 0; r < p; r++) {
        long long e = ((long long)r * kk) % n;
        double ang = sign * 2.0 * M_PI * (double)e / n;
        s = s + sub[r][k] * cd{std::cos(ang), std::sin(ang)};
      }
      out[kk] = s;
    }
  a.swap(out);
}

void fft3(C3 &A, int sign) {
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= A.n3; k++) {
    std::vector<cd> line(A.n1);
    for (int j = 1; j <= A.n2; j++) {
      for (int i = 1; i <= A.n1; i++) line[i - 1] = A(i, j, k);
      fft1(line, sign);
      for (int i = 1; i <= A.n1; i++) A(i, j, k) = line[i - 1];
    }
  }
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= A.n3; k++) {
    std::vector<cd> line(A.n2);
    for (int i = 1; i <= A.n1; i++) {
      for (int j = 1; j <= A.n2; j++) line[j - 1] = A(i, j, k);
      fft1(line, sign);
      for (int j = 1; j <= A.n2; j++) A(i, j, k) = line[j - 1];
    }
  }
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= A.n2; j++) {
    std::vector<cd> line(A.n3);
    for (int i = 1; i <= A.n1; i++) {
      for (int k = 1; k <= A.n3; k++) line[k - 1] = A(i, j, k);
      fft1(line, sign);
      for (int k = 1; k <= A.n3; k++) A(i, j, k) = line[k - 1];
    }
  }
}

// ---------------------------------------------------------------------------------------------- the separable inverse
// Basis of the SVD of the (n-1)×n forward difference D (implicit.jl:15-22): V (n×n, nodes), U ((n-1)×(n-1),
// edges), s (n, s[0] = 0).  Column-major.
struct Bases {
  int n = 0;
  std::vector<double> V, U, s, Vt, Ut;
  void make(int nn) {
    n = nn;
    V.assign((size_t)n * n, 0);
    U.assign((size_t)(n - 1) * (n - 1), 0);
    s.assign(n, 0);
    for (int k = 0; k < n; k++) {
      double ck = k == 0 ? std::sqrt(1.0 / n) : std::sqrt(2.0 / n);
      s[k] = 2 * std::sin(M_PI * k / (2.0 * n));
      for (int i = 0; i < n; i++) V[i + (size_t)n * k] = ck * std::cos(M_PI * k * (i + 0.5) / n);
    }
    for (int k = 1; k < n; k++)
      for (int e = 0; e < n - 1; e++) U[e + (size_t)(n - 1) * (k - 1)] = -std::sqrt(2.0 / n) * std::sin(M_PI * k * (e + 1.0) / n);
    Vt.resize(V.size());
    Ut.resize(U.size());
    for (int a = 0; a < n; a++)
      for (int b = 0; b < n; b++) Vt[a + (size_t)n * b] = V[b + (size_t)n * a];
    for (int a = 0; a < n - 1; a++)
      for (int b = 0; b < n - 1; b++) Ut[a + (size_t)(n - 1) * b] = U[b + (size_t)(n - 1) * a];
  }
};

// out[.., o, ..] = Σ_t M[t + nin*o] A[.., t, ..] along `axis` (0, 1, 2); dims of A: d[3].  Each output is summed over
// t in index order from zero (the plain loop of a matrix product); the loops are ordered so that the innermost one
// runs over contiguous outputs (vectorisable without reordering any sum).
template <class T>
void tx_axis(const std::vector<T> &A, const int d[3], int axis, const std::vector<T> &M, int nout, std::vector<T> &out) {
  int od[3] = {d[0], d[1], d[2]};
  od[axis] = nout;
  out.assign((size_t)od[0] * od[1] * od[2], T(0));
  const int nin = d[axis];
  if (axis == 0) {
    std::vector<T> Mt((size_t)nin * nout);   // Mt[o + nout t] = M[t + nin o]
    for (int o = 0; o < nout; o++)
      for (int t = 0; t < nin; t++) Mt[o + (size_t)nout * t] = M[t + (size_t)nin * o];
#pragma omp parallel for schedule(static)
    for (long long jk = 0; jk < (long long)d[1] * d[2]; jk++) {
      T *op = &out[(size_t)nout * jk];
      const T *ap = &A[(size_t)nin * jk];
      for (int t = 0; t < nin; t++) {
        const T at = ap[t];
        const T *mt = &Mt[(size_t)nout * t];
        for (int o = 0; o < nout; o++) op[o] += mt[o] * at;
      }
    }
  } else if (axis == 1) {
    const int n0 = d[0];
#pragma omp parallel for schedule(static)
    for (int k = 0; k < d[2]; k++)
      for (int o = 0; o < nout; o++) {
        T *op = &out[(size_t)n0 * (o + (size_t)nout * k)];
        for (int t = 0; t < nin; t++) {
          const T m = M[t + (size_t)nin * o];
          const T *ap = &A[(size_t)n0 * (t + (size_t)nin * k)];
          for (int i = 0; i < n0; i++) op[i] += m * ap[i];
        }
      }
  } else {
    const size_t pl = (size_t)d[0] * d[1];
#pragma omp parallel for schedule(static)
    for (int o = 0; o < nout; o++) {
      T *op = &out[pl * o];
      for (int t = 0; t < nin; t++) {
        const T m = M[t + (size_t)nin * o];
        const T *ap = &A[pl * t];
        for (size_t q = 0; q < pl; q++) op[q] += m * ap[q];
      }
    }
  }
}

template <class T>
struct SepT {
  int nx, ny, nz;                           // nodes per axis: Nx-1, Ny-1, Nz-1
  std::vector<T> Vx, Ux, Vy, Uy, Vz, Uz, Vxt, Uxt, Vyt, Uyt, Vzt, Uzt, sx, sy, sz;
  T a;
  void make(const Bases &bx, const Bases &by, const Bases &bz, double a_) {
    nx = bx.n; ny = by.n; nz = bz.n;
    auto cv = [](const std::vector<double> &v) { return std::vector<T>(v.begin(), v.end()); };
    Vx = cv(bx.V); Ux = cv(bx.U); Vxt = cv(bx.Vt); Uxt = cv(bx.Ut); sx = cv(bx.s);
    Vy = cv(by.V); Uy = cv(by.U); Vyt = cv(by.Vt); Uyt = cv(by.Ut); sy = cv(by.s);
    Vz = cv(bz.V); Uz = cv(bz.U); Vzt = cv(bz.Vt); Uzt = cv(bz.Ut); sz = cv(bz.s);
    a = (T)a_;
  }
  // (I + aK)^{-1} in place on BX (nx-1, ny, nz), BY (nx, ny-1, nz), BZ (nx, ny, nz-1)  (implicit.jl:62-83)
  void solve(std::vector<T> &BX, std::vector<T> &BY, std::vector<T> &BZ) {
    std::vector<T> t1, t2, X, Y, Z;
    int dX[3] = {nx - 1, ny, nz}, dY[3] = {nx, ny - 1, nz}, dZ[3] = {nx, ny, nz - 1};
    int d[3];
    // forward: X by (Ux, Vy, Vz)
    tx_axis(BX, dX, 0, Ux, nx - 1, t1); d[0] = nx - 1; d[1] = ny; d[2] = nz;
    tx_axis(t1, d, 1, Vy, ny, t2); tx_axis(t2, d, 2, Vz, nz, X);
    tx_axis(BY, dY, 0, Vx, nx, t1); d[0] = nx; d[1] = ny - 1; d[2] = nz;
    tx_axis(t1, d, 1, Uy, ny - 1, t2); tx_axis(t2, d, 2, Vz, nz, Y);
    tx_axis(BZ, dZ, 0, Vx, nx, t1); d[0] = nx; d[1] = ny; d[2] = nz - 1;
    tx_axis(t1, d, 1, Vy, ny, t2); tx_axis(t2, d, 2, Uz, nz - 1, Z);
    for (int mz = 1; mz <= nz; mz++)
      for (int my = 1; my <= ny; my++)
        for (int mx = 1; mx <= nx; mx++) {
          T k1 = sx[mx - 1], k2 = sy[my - 1], k3 = sz[mz - 1];
          T k2s = k1 * k1 + k2 * k2 + k3 * k3;
          if (k2s == 0) continue;
          T *px = mx > 1 ? &X[(mx - 2) + (size_t)(nx - 1) * ((my - 1) + (size_t)ny * (mz - 1))] : nullptr;
          T *py = my > 1 ? &Y[(mx - 1) + (size_t)nx * ((my - 2) + (size_t)(ny - 1) * (mz - 1))] : nullptr;
          T *pz = mz > 1 ? &Z[(mx - 1) + (size_t)nx * ((my - 1) + (size_t)ny * (mz - 2))] : nullptr;
          T x1 = px ? *px : T(0), y1 = py ? *py : T(0), z1 = pz ? *pz : T(0);
          T dd = (k1 * x1 + k2 * y1 + k3 * z1) / k2s;
          T f = T(1) / (T(1) + a * k2s);
          if (px) *px = k1 * dd + f * (x1 - k1 * dd);
          if (py) *py = k2 * dd + f * (y1 - k2 * dd);
          if (pz) *pz = k3 * dd + f * (z1 - k3 * dd);
        }
    // back: X by (Ux', Vy', Vz')
    d[0] = nx - 1; d[1] = ny; d[2] = nz;
    tx_axis(X, d, 0, Uxt, nx - 1, t1); tx_axis(t1, d, 1, Vyt, ny, t2); tx_axis(t2, d, 2, Vzt, nz, BX);
    d[0] = nx; d[1] = ny - 1; d[2] = nz;
    tx_axis(Y, d, 0, Vxt, nx, t1); tx_axis(t1, d, 1, Uyt, ny - 1, t2); tx_axis(t2, d, 2, Vzt, nz, BY);
    d[0] = nx; d[1] = ny; d[2] = nz - 1;
    tx_axis(Z, d, 0, Vxt, nx, t1); tx_axis(t1, d, 1, Vyt, ny, t2); tx_axis(t2, d, 2, Uzt, nz - 1, BZ);
  }
};

// ---------------------------------------------------------------------------------------------- the context
struct Range {
  int i0, i1, j0, j1, k0, k1;  // 1-based inclusive
  int n() const { return (i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1); }
};

}  // namespace

struct oracle_ctx {
  tdgl_params P;
  int N;
  int Nx, Ny, Nz, x1, x2, y1, y2, z1, z2;
  double dx, dy, dz;
  R3 f, tx, ty, tz;
  R3 D[3];
  bool haveD = false;
  std::vector<double> bar[6];
  std::vector<double> green, jbar;
  // state
  C3 G[TDGL_MAXB], F[TDGL_MAXB];
  R3 th[3], ph[3], J[3], h[3];
  C3 U[3], V[3];
  bool have_state = false;
  // workspace
  C3 W, W2, L[3], Rl[3];
  R3 Om, Oms, Rr[3];
  // separable solve
  Bases bx, by, bz;
  SepT<double> sep;
  SepT<float> sep32;
  Range rng[3];
  // PCG
  R3 Pf[3], Qf[3], Hf[3];
  std::vector<double> x[3], r[3], z[3], b[3], xprev[3], zold[3];
  bool warm = false, have2 = false;
  int iters = 0;
  long long total_iters = 0;
  // open boundary
  int open_count = -1;
  R3 o_old[3], o_new[3], o_theta[3];
  C3 o_ghat[3];
  int o_M[3][3];
  int open_recomputes = 0;
  long long steps = 0;
  // material per region (materials.jl): the node map, the tables, the link weights per band and axis
  bool haveMat = false;
  tdgl_materials M;
  std::vector<uint8_t> mat;
  R3 rho[TDGL_MAXB][3];
  bool haskwt[TDGL_MAXB] = {};
  // the heat model (terms.jl): the temperature field θ, node-shaped
  R3 Th;
  // two normal fluids (exchange.jl): δ = μ_π − μ_σ on the nodes, the 1D bases (column-major n × n) and eigenvalues
  R3 qd, qmu[TDGL_MAXB];   // δ (two bands) or the potentials μ_µ (N fluids), node-shaped
  std::vector<double> qV[3], qW[3], qe[3];
  std::vector<uint8_t> qcond;   // the CG's unknowns: 1 free, 0 cut, 2 held (empty: the separable solve)
  std::vector<double> qcx, qcy, qcz, qlamv;   // QPVar's coefficients (empty: the cut links of a sculpted sample)
  int qp_iters = 0;             // conjugate-gradient iterations of the last δ solve
  // a sculpted sample: the vacuum nodes (Masks.vac)
  bool haveVac = false;
  std::vector<uint8_t> vac;
  std::string err;
  bool isvac(int i, int j, int k) const {
    return haveVac && vac[(size_t)(i - 1) + (size_t)(Nx + 1) * ((size_t)(j - 1) + (size_t)(Ny + 1) * (size_t)(k - 1))];
  }
  int matidx(int i, int j, int k) const {   // 0-based material of node (i, j, k)
    return (int)mat[(size_t)(i - 1) + (size_t)(Nx + 1) * ((size_t)(j - 1) + (size_t)(Ny + 1) * (size_t)(k - 1))] - 1;
  }
};

namespace {

typedef oracle_ctx Ctx;

// ---------------------------------------------------------------------------------------------- bands
inline cd kwt_update(cd g, cd d, double g2) {
  double a2 = abs2(g);
  double q = 1 + g2 * a2;
  cd dp = std::sqrt(q) * d;
  return g + (dp - (g2 * g) * ((conj(g) * dp).re / q));
}

inline cd kwt_update_rot(cd g, cd d, double g2) {
  double a2 = abs2(g);
  double q = 1 + g2 * a2;
  cd dp = std::sqrt(q) * d;
  cd Dl = dp - (g2 * g) * ((conj(g) * dp).re / q);
  if (!(a2 > 1e-24)) return g + Dl;
  double a = std::sqrt(a2);
  cd u = g / a;
  cd w = conj(u) * Dl;
  return u * ((a + w.re) * cis(w.im / a));
}

// _dif with the link weights (bands.jl:63-64): today's expression plus k((ρ₊−1)(v₊s₊−g) + (ρ₋−1)(v₋s₋−g))
inline cd dif_mat(double rp, double rm, double k, cd vp, cd sp, cd vm, cd sm, cd g) {
  const cd a = vp * sp, b = vm * sm;
  return k * ((a - 2.0 * g) + b) + k * ((rp - 1) * (a - g) + (rm - 1) * (b - g));
}

// _band_pass! with materials (bands.jl:168-182): the node's coefficients from its material's table (the stage table
// when cf is the band's stage coefficients), the link weights in the diffusion, and Ψ = 0 where the band is absent
void band_pass_mat(Ctx &c, C3 &Dst, C3 &S, int mu, C3 &Lx, C3 &Ly, C3 &Lz, bool stage) {
  const bool rk = c.P.noise_on != 0;
  R3 &rx = c.rho[mu][0], &ry = c.rho[mu][1], &rz = c.rho[mu][2];
#pragma omp parallel for schedule(static)
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) {
        cd g = S(i, j, k);
        double fm = c.f(i, j, k);
        if (c.P.hard && fm == 0.0) {
          Dst(i, j, k) = C(0.0, 0.0);
          continue;
        }
        const int m = c.matidx(i, j, k);
        const tdgl_bandcoef &cf = stage ? c.M.stage[m][mu] : c.M.full[m][mu];
        cd vxm = conj(Lx(i - 1, j, k)), vym = conj(Ly(i, j - 1, k)), vzm = conj(Lz(i, j, k - 1));
        cd tx = dif_mat(rx(i, j, k), rx(i - 1, j, k), cf.kx, Lx(i, j, k), S(i + 1, j, k), vxm, S(i - 1, j, k), g);
        cd ty = dif_mat(ry(i, j, k), ry(i, j - 1, k), cf.ky, Ly(i, j, k), S(i, j + 1, k), vym, S(i, j - 1, k), g);
        cd tz = dif_mat(rz(i, j, k), rz(i, j, k - 1), cf.kz, Lz(i, j, k), S(i, j, k + 1), vzm, S(i, j, k - 1), g);
        // _epsn with _anode (bands.jl:65-66): the node's material's a − θ with the heat model
        const double eps = c.P.heat_on ? c.M.a[m][mu] - c.Th(i, j, k) : cf.eps;
        cd nl = (cf.c * g) * (fm * eps - cf.beta * abs2(g));
        cd acc = (((g + tx) + ty) + tz) + nl;
        for (int nu = 0; nu < c.N; nu++) {
          if (nu == mu) continue;
          acc = acc + cf.cpl[nu] * c.G[nu](i, j, k);
        }
        Dst(i, j, k) = cf.gamma2 > 0 ? (rk ? kwt_update_rot(g, acc - g, cf.gamma2) : kwt_update(g, acc - g, cf.gamma2)) : acc;
        if (c.M.absent[m][mu]) Dst(i, j, k) = C(0.0, 0.0);
      }
}

// _band_row_vac! (bands.jl:103-124): a vacuum node stays at Ψ = 0 and each neighbour enters with the mask of its
// link (τ; with materials ρ and the node's coefficients, and Ψ = 0 where the band is absent)
void band_pass_vac(Ctx &c, C3 &Dst, C3 &S, int mu, C3 &Lx, C3 &Ly, C3 &Lz, const tdgl_bandcoef &cf0, bool stage) {
  const bool rk = c.P.noise_on != 0;
  R3 &wx = c.haveMat ? c.rho[mu][0] : c.tx, &wy = c.haveMat ? c.rho[mu][1] : c.ty, &wz = c.haveMat ? c.rho[mu][2] : c.tz;
#pragma omp parallel for schedule(static)
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) {
        cd g = S(i, j, k);
        double fm = c.f(i, j, k);
        if (c.isvac(i, j, k) || (c.P.hard && fm == 0.0)) {
          Dst(i, j, k) = C(0.0, 0.0);
          continue;
        }
        const int m = c.haveMat ? c.matidx(i, j, k) : 0;
        const tdgl_bandcoef &cf = c.haveMat ? (stage ? c.M.stage[m][mu] : c.M.full[m][mu]) : cf0;
        cd tx = cf.kx * (wx(i, j, k) * (Lx(i, j, k) * S(i + 1, j, k) - g) + wx(i - 1, j, k) * (conj(Lx(i - 1, j, k)) * S(i - 1, j, k) - g));
        cd ty = cf.ky * (wy(i, j, k) * (Ly(i, j, k) * S(i, j + 1, k) - g) + wy(i, j - 1, k) * (conj(Ly(i, j - 1, k)) * S(i, j - 1, k) - g));
        cd tz = cf.kz * (wz(i, j, k) * (Lz(i, j, k) * S(i, j, k + 1) - g) + wz(i, j, k - 1) * (conj(Lz(i, j, k - 1)) * S(i, j, k - 1) - g));
        cd acc = (((g + tx) + ty) + tz) + (cf.c * g) * (fm * cf.eps - cf.beta * abs2(g));
        for (int nu = 0; nu < c.N; nu++) {
          if (nu == mu) continue;
          acc = acc + cf.cpl[nu] * c.G[nu](i, j, k);
        }
        Dst(i, j, k) = cf.gamma2 > 0 ? (rk ? kwt_update_rot(g, acc - g, cf.gamma2) : kwt_update(g, acc - g, cf.gamma2)) : acc;
        if (c.haveMat && c.M.absent[m][mu]) Dst(i, j, k) = C(0.0, 0.0);
      }
}

// ddiv: the pass's divisor of the drag coefficients (n substeps, or the RKL/RKC weight q; _dragof, bands.jl:195-196)
void band_pass(Ctx &c, C3 &Dst, C3 &S, int mu, C3 &Lx, C3 &Ly, C3 &Lz, const tdgl_bandcoef &cf, double ddiv) {
  if (c.haveVac) return band_pass_vac(c, Dst, S, mu, Lx, Ly, Lz, cf, &cf == &c.P.bcs[mu]);
  if (c.haveMat) return band_pass_mat(c, Dst, S, mu, Lx, Ly, Lz, &cf == &c.P.bcs[mu]);
  const bool rk = c.P.noise_on != 0;
#pragma omp parallel for schedule(static)
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) {
        cd g = S(i, j, k);
        double fm = c.f(i, j, k);
        if (c.P.hard && fm == 0.0) {
          Dst(i, j, k) = C(0.0, 0.0);
          continue;
        }
        cd vxm = conj(Lx(i - 1, j, k)), vym = conj(Ly(i, j - 1, k)), vzm = conj(Lz(i, j, k - 1));
        cd tx = cf.kx * ((Lx(i, j, k) * S(i + 1, j, k) - 2.0 * g) + vxm * S(i - 1, j, k));
        cd ty = cf.ky * ((Ly(i, j, k) * S(i, j + 1, k) - 2.0 * g) + vym * S(i, j - 1, k));
        cd tz = cf.kz * ((Lz(i, j, k) * S(i, j, k + 1) - 2.0 * g) + vzm * S(i, j, k - 1));
        // _epsn (bands.jl:33-35): with the heat model ε = a − θ at the node
        const double eps = c.P.heat_on ? c.P.heat_a[mu] - c.Th(i, j, k) : cf.eps;
        cd nl = (cf.c * g) * (fm * eps - cf.beta * abs2(g));
        cd acc = (((g + tx) + ty) + tz) + nl;
        for (int nu = 0; nu < c.N; nu++) {
          if (nu == mu) continue;
          acc = acc + cf.cpl[nu] * c.G[nu](i, j, k);
        }
        if (c.P.drag_on)   // _drag (bands.jl:37-51): the lattice Laplacian of every other band, on this pass's links
          for (int nu = 0; nu < c.N; nu++) {
            if (nu == mu) continue;
            const double cx = c.P.drag_c[mu][nu][0] / ddiv, cy = c.P.drag_c[mu][nu][1] / ddiv,
                         cz = c.P.drag_c[mu][nu][2] / ddiv;
            C3 &P = c.G[nu];
            const cd p = P(i, j, k);
            const cd ex = cx * ((Lx(i, j, k) * P(i + 1, j, k) - 2.0 * p) + vxm * P(i - 1, j, k));
            const cd ey = cy * ((Ly(i, j, k) * P(i, j + 1, k) - 2.0 * p) + vym * P(i, j - 1, k));
            const cd ez = cz * ((Lz(i, j, k) * P(i, j, k + 1) - 2.0 * p) + vzm * P(i, j, k - 1));
            acc = acc + ((ex + ey) + ez);
          }
        Dst(i, j, k) = cf.gamma2 > 0 ? (rk ? kwt_update_rot(g, acc - g, cf.gamma2) : kwt_update(g, acc - g, cf.gamma2)) : acc;
      }
}

void frame_rate(Ctx &c, C3 &Cc, C3 &Y, double h) {
  const double wmax = 0.5 / c.P.dt;
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) {
        cd y = Y(i, j, k);
        double a2 = abs2(y);
        double w = 0.0;
        if (a2 > 1e-3) {
          w = (conj(y) * (Cc(i, j, k) - y)).im / (a2 * h);
          w = w < -wmax ? -wmax : (w > wmax ? wmax : w);
        }
        c.Om(i, j, k) = w;
        Cc(i, j, k) = minus_i_times(Cc(i, j, k), w * h, y);
      }
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++) {
      c.Om(c.x1, j, k) = c.Om(c.x1 + 1, j, k);
      c.Om(c.x2 + 1, j, k) = c.Om(c.x2, j, k);
    }
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int i = c.x1; i <= c.x2 + 1; i++) {
      c.Om(i, c.y1, k) = c.Om(i, c.y1 + 1, k);
      c.Om(i, c.y2 + 1, k) = c.Om(i, c.y2, k);
    }
  for (int j = c.y1; j <= c.y2 + 1; j++)
    for (int i = c.x1; i <= c.x2 + 1; i++) {
      c.Om(i, j, c.z1) = c.Om(i, j, c.z1 + 1);
      c.Om(i, j, c.z2 + 1) = c.Om(i, j, c.z2);
    }
}

void omega_faces(Ctx &c, R3 &Om) {
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++) {
      Om(c.x1, j, k) = Om(c.x1 + 1, j, k);
      Om(c.x2 + 1, j, k) = Om(c.x2, j, k);
    }
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int i = c.x1; i <= c.x2 + 1; i++) {
      Om(i, c.y1, k) = Om(i, c.y1 + 1, k);
      Om(i, c.y2 + 1, k) = Om(i, c.y2, k);
    }
  for (int j = c.y1; j <= c.y2 + 1; j++)
    for (int i = c.x1; i <= c.x2 + 1; i++) {
      Om(i, j, c.z1) = Om(i, j, c.z1 + 1);
      Om(i, j, c.z2 + 1) = Om(i, j, c.z2);
    }
}

// With noise the frame rate is low-passed, two sweeps Ω ← Ω/2 + (Σ six neighbours)/12, and the frame term of the first
// stage is the rotation C ← C e^{−iω̂h} (bands.jl:243-272).
void frame_rate_smooth(Ctx &c, C3 &Cc, C3 &Y, double h) {
  const double wmax = 0.5 / c.P.dt;
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) {
        cd y = Y(i, j, k);
        double a2 = abs2(y);
        double w = 0.0;
        if (a2 > 1e-3) {
          w = (conj(y) * (Cc(i, j, k) - y)).im / (a2 * h);
          w = w < -wmax ? -wmax : (w > wmax ? wmax : w);
        }
        c.Om(i, j, k) = w;
      }
  omega_faces(c, c.Om);
  for (int pass = 0; pass < 2; pass++) {
    c.Oms.v = c.Om.v;
    R3 &T = c.Oms;
    for (int k = c.z1 + 1; k <= c.z2; k++)
      for (int j = c.y1 + 1; j <= c.y2; j++)
        for (int i = c.x1 + 1; i <= c.x2; i++) {
          double nb = ((T(i + 1, j, k) + T(i - 1, j, k)) + (T(i, j + 1, k) + T(i, j - 1, k))) + (T(i, j, k + 1) + T(i, j, k - 1));
          c.Om(i, j, k) = 0.5 * T(i, j, k) + nb / 12;
        }
    omega_faces(c, c.Om);
  }
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) Cc(i, j, k) = Cc(i, j, k) * cis(-(c.Om(i, j, k) * h));
}

void frame_term(Ctx &c, C3 &Cc, C3 &S, double h) {
  if (c.P.noise_on) {   // as the rotation it stands for (bands.jl:274-286)
    for (int k = c.z1 + 1; k <= c.z2; k++)
      for (int j = c.y1 + 1; j <= c.y2; j++)
        for (int i = c.x1 + 1; i <= c.x2; i++) Cc(i, j, k) = Cc(i, j, k) * cis(-(c.Om(i, j, k) * h));
    return;
  }
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) Cc(i, j, k) = minus_i_times(Cc(i, j, k), c.Om(i, j, k) * h, S(i, j, k));
}

void frame_rate_any(Ctx &c, C3 &Cc, C3 &Y, double h) {
  if (c.P.noise_on) frame_rate_smooth(c, Cc, Y, h);
  else frame_rate(c, Cc, Y, h);
}

// ---------------------------------------------------------------------------------------------- thermal noise
// The draws.  The reference draws from a Xoshiro stream in a fixed loop order (noise.jl:28-35); here every draw is a
// pure function of (seed, step, stream, node): Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11: ten rounds of
// the 4×32 multiply-xor round with the Weyl key schedule), two 53-bit uniforms, Box–Muller.  Stream µ < 8 for band
// µ, 16 + axis for the link kicks; the node is its node-shaped linear index.
const double ROT_MIN2 = 1e-3;

void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; r++) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
  }
}

// a pair of standard normals from counter {node, step, stream} under key `seed`
cd normals_at(uint64_t seed, uint64_t step, uint32_t stream, uint32_t node) {
  uint32_t w[4] = {node, (uint32_t)step, (uint32_t)(step >> 32), stream};
  philox10(w, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double u1 = 1.0 - ((double)(w[0] >> 5) * 67108864.0 + (double)(w[1] >> 6)) * (1.0 / 9007199254740992.0);
  const double u2 = ((double)(w[2] >> 5) * 67108864.0 + (double)(w[3] >> 6)) * (1.0 / 9007199254740992.0);
  const double r = std::sqrt(-2.0 * std::log(u1)), t = 2.0 * M_PI * u2;
  return cd{r * std::cos(t), r * std::sin(t)};
}

cd normals(const Ctx &c, uint32_t stream, uint32_t node) {
  return normals_at(c.P.noise_seed, (uint64_t)(c.P.noise_step0 + c.steps), stream, node);
}

uint32_t node_index(const Ctx &c, int i, int j, int k) {
  return (uint32_t)((i - 1) + (c.Nx + 1) * ((j - 1) + (c.Ny + 1) * (k - 1)));
}

// _haskwt (bands.jl:454): KWT on band µ in any material
bool haskwt(const Ctx &c, int mu) { return c.P.bcs[mu].gamma2 > 0 || c.haskwt[mu]; }

bool skrock(const Ctx &c, int mu) {
  return c.P.noise_on && c.P.use_rkc[mu] && c.P.stages[mu] > 0 && haskwt(c, mu);
}

// the Γ and γ̃² of band µ at a node (its material's, materials.jl), and whether the band is absent there
struct NodeBand {
  double Gam, g2;
  bool absent;
};
NodeBand node_band(const Ctx &c, int mu, int i, int j, int k) {
  if (!c.haveMat) return NodeBand{c.P.noise_gamma[mu], c.P.bcs[mu].gamma2, false};
  const int m = c.matidx(i, j, k);
  return NodeBand{c.M.gamma[m][mu], c.M.full[m][mu].gamma2, c.M.absent[m][mu] != 0};
}

// Qθ of noise_draw! (noise.jl:101-123): the phase kick that SK-ROCK puts into the first stage; 0 where none
double qtheta(const Ctx &c, int mu, int i, int j, int k) {
  if (c.P.hard && c.f(i, j, k) == 0.0) return 0.0;
  if (c.isvac(i, j, k)) return 0.0;
  const NodeBand nb = node_band(c, mu, i, j, k);
  if (nb.absent) return 0.0;
  const double g2 = nb.g2, Gam = nb.Gam;
  const cd psi = c.G[mu](i, j, k);
  const double r2 = abs2(psi);
  if (!(g2 > 0 && r2 > ROT_MIN2)) return 0.0;
  const double dV = c.dx * c.dy * c.dz, cN = std::sqrt(c.P.noise_T * c.P.dt / dV);
  const cd xi = normals(c, (uint32_t)mu, node_index(c, i, j, k));
  const double sk = std::sqrt(1 + g2 * r2), rho = std::sqrt(r2);
  return cN * (conj(psi / rho) * xi).im * std::sqrt(sk / Gam) / rho;
}

// _sk_turn! (bands.jl:447-453): D ← X e^{i c δθ}
void sk_turn(Ctx &c, C3 &D, C3 &X, int mu, double cc) {
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) {
        const double q = qtheta(c, mu, i, j, k);
        D(i, j, k) = q == 0.0 ? X(i, j, k) : X(i, j, k) * cis(cc * q);
      }
}

// _kwt_kick (noise.jl:78-91)
cd kwt_kick(cd F, cd psi, cd xi, double a, double cN, double dr, double g2, double Gam, double d0) {
  const double r2 = abs2(psi), sk = std::sqrt(1 + g2 * r2);
  if (!(r2 > 1e-24)) return F + a * xi;
  const cd u = psi / std::sqrt(r2), w = conj(u) * xi;
  if (r2 > ROT_MIN2 && abs2(F) > ROT_MIN2) {
    const double rho = std::sqrt(r2), aF = std::hypot(F.re, F.im);
    const double drho = cN * w.re / std::sqrt(Gam * sk) + d0 / (rho * (sk * sk * sk));
    const double dth = cN * w.im * std::sqrt(sk / Gam) / rho;
    return (F / aF) * ((aF + drho) * cis(dth));
  }
  return (F + (cN * u) * C(w.re / std::sqrt(Gam * sk), w.im * std::sqrt(sk / Gam))) -
         ((dr * (1 + sk * sk)) / (sk * sk * sk)) * psi;
}

// noise_apply! / noise_kick! (noise.jl:40-66, :125-151): the kick of every band after the band update
void noise_after(Ctx &c) {
  const double dV = c.dx * c.dy * c.dz, T = c.P.noise_T, dt = c.P.dt, cN = std::sqrt(T * dt / dV);
  for (int mu = 0; mu < c.N; mu++) {
    const bool sk = skrock(c, mu);
    C3 &F = c.F[mu];
#pragma omp parallel for schedule(static)
    for (int k = c.z1 + 1; k <= c.z2; k++)
      for (int j = c.y1 + 1; j <= c.y2; j++)
        for (int i = c.x1 + 1; i <= c.x2; i++) {
          if (c.P.hard && c.f(i, j, k) == 0.0) continue;
          if (c.isvac(i, j, k)) continue;
          const NodeBand nb = node_band(c, mu, i, j, k);   // the node's material (_noise_kick_mat!, noise.jl:156-180)
          if (nb.absent) continue;
          const double Gam = nb.Gam, g2 = nb.g2, a = std::sqrt(T * dt / (Gam * dV));
          const cd xi = normals(c, (uint32_t)mu, node_index(c, i, j, k));
          if (g2 == 0) {
            F(i, j, k) = F(i, j, k) + a * xi;
          } else if (sk && qtheta(c, mu, i, j, k) != 0.0) {   // the phase went in with the stages
            const cd psi = c.G[mu](i, j, k);
            const double rho = std::hypot(psi.re, psi.im), skk = std::sqrt(1 + g2 * (rho * rho));
            const cd u = psi / rho;
            const double drho = cN * (conj(u) * xi).re / std::sqrt(Gam * skk) + T * dt / (2 * dV * Gam) / (rho * (skk * skk * skk));
            const cd f = F(i, j, k);
            const double aF = std::hypot(f.re, f.im);
            F(i, j, k) = aF > std::sqrt(ROT_MIN2) ? f * ((aF + drho) / aF) : f + u * drho;
          } else {
            F(i, j, k) = kwt_kick(F(i, j, k), c.G[mu](i, j, k), xi, a, cN, T * dt / (2 * dV) * g2 / Gam, g2, Gam,
                                  T * dt / (2 * dV * Gam));
          }
        }
  }
}

// field_kick! (noise.jl:183-198): the link phases before the implicit solve
void field_kick(Ctx &c) {
  const double cN = std::sqrt(c.P.noise_T * c.P.dt / (c.P.noise_sigma_n * c.dx * c.dy * c.dz));
  const double ad[3] = {cN * c.dx, cN * c.dy, cN * c.dz};
  const int lo[3][3] = {{1, 2, 2}, {2, 1, 2}, {2, 2, 1}}, hi[3][3] = {{c.Nx, c.Ny, c.Nz}, {c.Nx, c.Ny, c.Nz}, {c.Nx, c.Ny, c.Nz}};
  for (int ax = 0; ax < 3; ax++)
    for (int k = lo[ax][2]; k <= hi[ax][2]; k++)
      for (int j = lo[ax][1]; j <= hi[ax][1]; j++)
        for (int i = lo[ax][0]; i <= hi[ax][0]; i++) {
          const double n = normals(c, 16u + ax, node_index(c, i, j, k)).re;
          const double amp = c.haveD ? ad[ax] * std::sqrt(c.D[ax](i, j, k)) : ad[ax];
          c.ph[ax](i, j, k) += amp * n;
        }
}

void frame_turn(Ctx &c, C3 &Fm) {
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) Fm(i, j, k) = Fm(i, j, k) * cis(c.Om(i, j, k) * c.P.dt);
}

Range rx_(const Ctx &c) { return Range{c.x1, c.x2, c.y1, c.y2 + 1, c.z1, c.z2 + 1}; }
Range ry_(const Ctx &c) { return Range{c.x1, c.x2 + 1, c.y1, c.y2, c.z1, c.z2 + 1}; }
Range rz_(const Ctx &c) { return Range{c.x1, c.x2 + 1, c.y1, c.y2 + 1, c.z1, c.z2}; }
Range lrange(const Ctx &c, int ax) { return ax == 0 ? rx_(c) : ax == 1 ? ry_(c) : rz_(c); }

// sequential over the range (the lambdas that keep a running packed index need the order)
template <class Fn>
void each(const Range &r, Fn fn) {
  for (int k = r.k0; k <= r.k1; k++)
    for (int j = r.j0; j <= r.j1; j++)
      for (int i = r.i0; i <= r.i1; i++) fn(i, j, k);
}
// parallel over k, for lambdas that depend on (i, j, k) only
template <class Fn>
void each_par(const Range &r, Fn fn) {
#pragma omp parallel for schedule(static)
  for (int k = r.k0; k <= r.k1; k++)
    for (int j = r.j0; j <= r.j1; j++)
      for (int i = r.i0; i <= r.i1; i++) fn(i, j, k);
}

void frame_links(Ctx &c, double tau) {
  for (int ax = 0; ax < 3; ax++) {
    int oi = ax == 0, oj = ax == 1, ok = ax == 2;
    each_par(lrange(c, ax), [&](int i, int j, int k) {
      c.L[ax](i, j, k) = c.L[ax](i, j, k) * cis_short((c.Om(i + oi, j + oj, k + ok) - c.Om(i, j, k)) * tau);
    });
  }
}

// The per-link formulas of the temporal link rotations (bands.jl:303-310, :355-369, :409-423), shared by the
// context passes below and by oracle_link_rotations (the manufactured inputs of test_link_rotations.jl).
// −arg q of q = V conj(U), with the short series while Re q > 0 and |sin| <= 0.05 (_link_rate!)
inline double link_angle(cd v, cd u) {
  cd q = v * conj(u);
  double sf = -q.im;
  return (q.re > 0 && std::fabs(sf) <= 0.05) ? -(sf + sf * sf * sf / 6) : angle(q);
}
// Q^{1/n} (_rot!)
inline cd link_root(cd v, cd u, double n) {
  cd q = v * conj(u);
  double sf = -q.im;
  if (q.re > 0 && std::fabs(sf) <= 0.05) {
    double a = (sf + sf * sf * sf / 6) / n;
    double a2 = a * a;
    return C(1 - a2 / 2, -a * (1 - a2 / 6));
  }
  return cis(angle(q) / n);
}
// V Q^c (_rotfrac!)
inline cd link_frac(cd v, cd u, double cc) {
  cd q = v * conj(u);
  double sf = -q.im;
  if (q.re > 0 && std::fabs(sf) <= 0.05) {
    double a = (sf + sf * sf * sf / 6) * cc;
    double a2 = a * a;
    return v * C(1 - a2 / 2, -a * (1 - a2 / 6));
  }
  return v * cis(angle(q) * cc);
}

void link_rate(Ctx &c) {
  for (int ax = 0; ax < 3; ax++) {
    int oi = ax == 0, oj = ax == 1, ok = ax == 2;
    each_par(lrange(c, ax), [&](int i, int j, int k) {
      c.Rr[ax](i, j, k) = link_angle(c.V[ax](i, j, k), c.U[ax](i, j, k)) +
                          (c.Om(i + oi, j + oj, k + ok) - c.Om(i, j, k)) * c.P.dt;
    });
  }
}

void rotlinks(Ctx &c, double cc) {
  for (int ax = 0; ax < 3; ax++)
    each_par(lrange(c, ax), [&](int i, int j, int k) { c.L[ax](i, j, k) = c.V[ax](i, j, k) * cis_short(c.Rr[ax](i, j, k) * cc); });
}

void rotfrac(Ctx &c, double cc) {
  for (int ax = 0; ax < 3; ax++)
    each_par(lrange(c, ax), [&](int i, int j, int k) { c.L[ax](i, j, k) = link_frac(c.V[ax](i, j, k), c.U[ax](i, j, k), cc); });
}

void rot_init(Ctx &c, int n) {
  for (int ax = 0; ax < 3; ax++)
    each_par(lrange(c, ax), [&](int i, int j, int k) {
      cd v = c.V[ax](i, j, k);
      c.L[ax](i, j, k) = v;
      c.Rl[ax](i, j, k) = link_root(v, c.U[ax](i, j, k), (double)n);
    });
}

void advance_links(Ctx &c) {
  for (int ax = 0; ax < 3; ax++)
    each_par(lrange(c, ax), [&](int i, int j, int k) { c.L[ax](i, j, k) = c.L[ax](i, j, k) * c.Rl[ax](i, j, k); });
}

void ghosts(Ctx &c, C3 &X, C3 &Vx, C3 &Vy, C3 &Vz) {
  for (int k = c.z1; k <= c.z2 + 1; k++)
    for (int j = c.y1; j <= c.y2 + 1; j++) {
      X(c.x1, j, k) = Vx(c.x1, j, k) * X(c.x1 + 1, j, k);
      X(c.x2 + 1, j, k) = conj(Vx(c.x2, j, k)) * X(c.x2, j, k);
    }
  for (int k = c.z1; k <= c.z2 + 1; k++)
    for (int i = c.x1; i <= c.x2 + 1; i++) {
      X(i, c.y1, k) = Vy(i, c.y1, k) * X(i, c.y1 + 1, k);
      X(i, c.y2 + 1, k) = conj(Vy(i, c.y2, k)) * X(i, c.y2, k);
    }
  for (int j = c.y1; j <= c.y2 + 1; j++)
    for (int i = c.x1; i <= c.x2 + 1; i++) {
      X(i, j, c.z1) = Vz(i, j, c.z1) * X(i, j, c.z1 + 1);
      X(i, j, c.z2 + 1) = conj(Vz(i, j, c.z2)) * X(i, j, c.z2);
    }
}

void band_substeps(Ctx &c, int mu, int n) {
  const tdgl_bandcoef &cf = c.P.bcs[mu];
  C3 &Fm = c.F[mu];
  C3 *Lx = &c.V[0], *Ly = &c.V[1], *Lz = &c.V[2];
  if (c.P.extrap) {
    rot_init(c, n);
    Lx = &c.L[0]; Ly = &c.L[1]; Lz = &c.L[2];
  }
  C3 *src = &c.G[mu];
  const bool rot = c.P.rotframe != 0;
  const double h = c.P.dt / n;
  for (int m = 1; m <= n; m++) {
    C3 *dst = ((n - m) % 2 == 0) ? &Fm : &c.W;
    band_pass(c, *dst, *src, mu, *Lx, *Ly, *Lz, cf, (double)n);
    if (rot) {
      if (m == 1) frame_rate_any(c, *dst, *src, h);
      else frame_term(c, *dst, *src, h);
    }
    if (m < n) {
      if (c.P.extrap) advance_links(c);
      if (rot) frame_links(c, h);
      ghosts(c, *dst, *Lx, *Ly, *Lz);
    }
    src = dst;
  }
  if (rot) frame_turn(c, Fm);
}

void combine(Ctx &c, C3 &Cc, C3 &A, double mu, double nu) {
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) Cc(i, j, k) = mu * Cc(i, j, k) + nu * A(i, j, k);
}

// _combine_log! (bands.jl:439-445), with noise on a KWT band: C ← A exp(μ log(C/A)), the linear combination where
// |A|² or |C|² is under ROT_MIN2.  (C/A by the plain formula; the reference's is Julia's robust complex division.)
cd clog(cd z) { return cd{std::log(std::hypot(z.re, z.im)), std::atan2(z.im, z.re)}; }
cd cexp(cd z) { return std::exp(z.re) * cis(z.im); }
cd cdiv(cd a, cd b) {
  const double d = b.re * b.re + b.im * b.im;
  return cd{(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
void combine_log(Ctx &c, C3 &Cc, C3 &A, double mu) {
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) {
        const cd a = A(i, j, k), cc = Cc(i, j, k);
        Cc(i, j, k) = abs2(a) > ROT_MIN2 && abs2(cc) > ROT_MIN2 ? a * cexp(mu * clog(cdiv(cc, a))) : mu * cc + (1 - mu) * a;
      }
}

void band_rkl(Ctx &c, int mu, int ns) {
  const tdgl_bandcoef &cf = c.P.bcs[mu];
  const bool kc = c.P.use_rkc[mu] != 0;
  const double q = kc ? c.P.rkc_q[mu] : (double)(ns * (ns + 1) / 2);
  C3 *Lx = &c.V[0], *Ly = &c.V[1], *Lz = &c.V[2];
  if (c.P.extrap) {
    for (int ax = 0; ax < 3; ax++) c.L[ax].v = c.V[ax].v;
    Lx = &c.L[0]; Ly = &c.L[1]; Lz = &c.L[2];
  }
  C3 *buf[3] = {&c.W, &c.W2, &c.F[mu]};
  const bool rot = c.P.rotframe != 0;
  const double h = c.P.dt / q;
  C3 *A = &c.G[mu], *B = &c.G[mu], *Cc = &c.W;
  const bool skq = skrock(c, mu), lg = c.P.noise_on && haskwt(c, mu);
  for (int j = 1; j <= ns; j++) {
    Cc = buf[(j - 1) % 3];
    if (j == 1 && skq) {   // SK-ROCK for the phase: K1 = E(Ψⁿ e^{iν₁δθ}) e^{i(κ₁−ν₁)δθ} (bands.jl:482-488)
      C3 &Sp = c.W2;
      const double nu1 = c.P.rkc_sk[mu][0], ka1 = c.P.rkc_sk[mu][1];
      sk_turn(c, Sp, *B, mu, nu1);
      ghosts(c, Sp, *Lx, *Ly, *Lz);
      band_pass(c, *Cc, Sp, mu, *Lx, *Ly, *Lz, cf, q);
      if (rot) frame_rate_any(c, *Cc, Sp, h);
      sk_turn(c, *Cc, *Cc, mu, ka1 - nu1);
    } else {
      band_pass(c, *Cc, *B, mu, *Lx, *Ly, *Lz, cf, q);
      if (rot) {
        if (j == 1) frame_rate_any(c, *Cc, *B, h);
        else frame_term(c, *Cc, *B, h);
      }
    }
    if (rot && j == 1 && c.P.extrap && ns > 1) link_rate(c);
    if (j >= 2) {
      double mj = kc ? c.P.rkc_mu[mu][j - 1] : (double)(2 * j - 1) / j;
      double nj = kc ? c.P.rkc_nu[mu][j - 1] : (double)(1 - j) / j;
      if (lg) combine_log(c, *Cc, *A, mj);
      else combine(c, *Cc, *A, mj, nj);
    }
    if (j < ns) {
      if (c.P.extrap) {
        double cc = kc ? c.P.rkc_c[mu][j - 1] : (double)(j * (j + 1)) / (double)(ns * (ns + 1));
        if (rot) rotlinks(c, cc);
        else rotfrac(c, cc);
      }
      ghosts(c, *Cc, *Lx, *Ly, *Lz);
    }
    A = B;
    B = Cc;
  }
  if (Cc != &c.F[mu]) c.F[mu].v = Cc->v;
  if (rot) frame_turn(c, c.F[mu]);
}

void update_bands(Ctx &c) {
  for (int mu = 0; mu < c.N; mu++) {
    int n = c.P.nsub[mu];
    if (c.P.stages[mu] > 0) {
      band_rkl(c, mu, c.P.stages[mu]);
    } else if (n == 1) {
      band_pass(c, c.F[mu], c.G[mu], mu, c.V[0], c.V[1], c.V[2], c.P.bc[mu], 1.0);
      if (c.P.rotframe) {
        frame_rate_any(c, c.F[mu], c.G[mu], c.P.dt);
        frame_turn(c, c.F[mu]);
      }
    } else {
      band_substeps(c, mu, n);
    }
  }
}

// ---------------------------------------------------------------------------------------------- field
// _supercurrent_mat! (field.jl:48-71): each band's link carries w_µ ρ_µ
void supercurrent_mat(Ctx &c) {
  auto jl = [&](int ax, cd v, int i, int j, int k, int i2, int j2, int k2) {
    double acc = (c.P.wa[ax][0] * c.rho[0][ax](i, j, k)) * ((conj(c.G[0](i, j, k)) * v) * c.G[0](i2, j2, k2)).im;
    for (int mu = 1; mu < c.N; mu++)
      acc += (c.P.wa[ax][mu] * c.rho[mu][ax](i, j, k)) * ((conj(c.G[mu](i, j, k)) * v) * c.G[mu](i2, j2, k2)).im;
    return acc;
  };
  for (int k = 2; k <= c.Nz; k++) {
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 1; i <= c.Nx; i++) c.J[0](i, j, k) = jl(0, c.V[0](i, j, k), i, j, k, i + 1, j, k);
    for (int j = 1; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx; i++) c.J[1](i, j, k) = jl(1, c.V[1](i, j, k), i, j, k, i, j + 1, k);
  }
  for (int k = 1; k <= c.Nz; k++)
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx; i++) c.J[2](i, j, k) = jl(2, c.V[2](i, j, k), i, j, k, i, j, k + 1);
}

void supercurrent(Ctx &c) {
  if (c.haveMat) return supercurrent_mat(c);
  auto jl = [&](int ax, cd v, int i, int j, int k, int i2, int j2, int k2) {
    double acc = c.P.wa[ax][0] * ((conj(c.G[0](i, j, k)) * v) * c.G[0](i2, j2, k2)).im;
    for (int mu = 1; mu < c.N; mu++) acc += c.P.wa[ax][mu] * ((conj(c.G[mu](i, j, k)) * v) * c.G[mu](i2, j2, k2)).im;
    if (c.P.drag_on)   // _jdrag (field.jl:73-81)
      for (int mu = 0; mu < c.N; mu++)
        for (int eta = mu + 1; eta < c.N; eta++) {
          const double cd_ = c.P.drag_nu[mu][eta];
          if (cd_ == 0.0) continue;
          acc += cd_ * (((conj(c.G[mu](i, j, k)) * v) * c.G[eta](i2, j2, k2)).im +
                        ((conj(c.G[eta](i, j, k)) * v) * c.G[mu](i2, j2, k2)).im);
        }
    return acc;
  };
  for (int k = 2; k <= c.Nz; k++) {
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 1; i <= c.Nx; i++) c.J[0](i, j, k) = jl(0, c.V[0](i, j, k), i, j, k, i + 1, j, k);
    for (int j = 1; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx; i++) c.J[1](i, j, k) = jl(1, c.V[1](i, j, k), i, j, k, i, j + 1, k);
  }
  for (int k = 1; k <= c.Nz; k++)
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx; i++) c.J[2](i, j, k) = jl(2, c.V[2](i, j, k), i, j, k, i, j, k + 1);
}

void field_increment(Ctx &c) {
  const tdgl_params &P = c.P;
  R3 &hx = c.h[0], &hy = c.h[1], &hz = c.h[2];
  for (int k = 2; k <= c.Nz; k++)
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 1; i <= c.Nx; i++)
        c.ph[0](i, j, k) = ((c.th[0](i, j, k) + (P.d1 * c.tx(i, j, k)) * c.J[0](i, j, k)) - P.sxy * (hz(i, j, k) - hz(i, j - 1, k))) +
                           P.sxz * (hy(i, j, k) - hy(i, j, k - 1));
  for (int k = 2; k <= c.Nz; k++)
    for (int j = 1; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx; i++)
        c.ph[1](i, j, k) = ((c.th[1](i, j, k) + (P.d1 * c.ty(i, j, k)) * c.J[1](i, j, k)) - P.syz * (hx(i, j, k) - hx(i, j, k - 1))) +
                           P.syx * (hz(i, j, k) - hz(i - 1, j, k));
  for (int k = 1; k <= c.Nz; k++)
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx; i++)
        c.ph[2](i, j, k) = ((c.th[2](i, j, k) + (P.d1 * c.tz(i, j, k)) * c.J[2](i, j, k)) - P.szx * (hy(i, j, k) - hy(i - 1, j, k))) +
                           P.szy * (hx(i, j, k) - hx(i, j - 1, k));
}

void gather_diff(Ctx &c, int ax, std::vector<double> &out) {
  const Range &r = c.rng[ax];
  out.resize(r.n());
  size_t q = 0;
  each(r, [&](int i, int j, int k) { out[q++] = c.ph[ax](i, j, k) - c.th[ax](i, j, k); });
}
void scatter_sum(Ctx &c, int ax, const std::vector<double> &x) {
  const Range &r = c.rng[ax];
  size_t q = 0;
  each(r, [&](int i, int j, int k) { c.ph[ax](i, j, k) = c.th[ax](i, j, k) + x[q++]; });
}

void implicit_sep(Ctx &c) {
  std::vector<double> B[3];
  for (int ax = 0; ax < 3; ax++) gather_diff(c, ax, B[ax]);
  c.sep.solve(B[0], B[1], B[2]);
  for (int ax = 0; ax < 3; ax++) scatter_sum(c, ax, B[ax]);
}

void scale_increment(Ctx &c) {
  for (int ax = 0; ax < 3; ax++)
    for (size_t q = 0; q < c.ph[ax].size(); q++) c.ph[ax].v[q] = c.th[ax].v[q] + (c.ph[ax].v[q] - c.th[ax].v[q]) / c.D[ax].v[q];
}

double dot(const std::vector<double> &a, const std::vector<double> &b) {
  double s = 0.0;
  for (size_t q = 0; q < a.size(); q++) s += a[q] * b[q];
  return s;
}
double dot3(const std::vector<double> *a, const std::vector<double> *b) { return dot(a[0], b[0]) + dot(a[1], b[1]) + dot(a[2], b[2]); }

void precond(Ctx &c, std::vector<double> *z, const std::vector<double> *r) {
  std::vector<double> B[3] = {r[0], r[1], r[2]};
  c.sep.solve(B[0], B[1], B[2]);
  for (int ax = 0; ax < 3; ax++) z[ax] = B[ax];
}
void precond32(Ctx &c, std::vector<double> *z, const std::vector<double> *r) {
  std::vector<float> B[3];
  for (int ax = 0; ax < 3; ax++) B[ax].assign(r[ax].begin(), r[ax].end());
  c.sep32.solve(B[0], B[1], B[2]);
  for (int ax = 0; ax < 3; ax++) z[ax].assign(B[ax].begin(), B[ax].end());
}

void scatter_full(Ctx &c, R3 *full, const std::vector<double> *v) {
  for (int ax = 0; ax < 3; ax++) {
    std::fill(full[ax].v.begin(), full[ax].v.end(), 0.0);
    size_t q = 0;
    each(c.rng[ax], [&](int i, int j, int k) { full[ax](i, j, k) = v[ax][q++]; });
  }
}
void gather_full(Ctx &c, R3 *full, int ax, std::vector<double> &out) {
  out.resize(c.rng[ax].n());
  size_t q = 0;
  each(c.rng[ax], [&](int i, int j, int k) { out[q++] = full[ax](i, j, k); });
}

void apply_A(Ctx &c) {
  const tdgl_params &P = c.P;
  R3 &px = c.Pf[0], &py = c.Pf[1], &pz = c.Pf[2];
  R3 &qx = c.Qf[0], &qy = c.Qf[1], &qz = c.Qf[2];
  R3 &hx = c.Hf[0], &hy = c.Hf[1], &hz = c.Hf[2];
  const int Nx = c.Nx, Ny = c.Ny, Nz = c.Nz;
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= Nz - 1; k++)
    for (int j = 2; j <= Ny - 1; j++)
      for (int i = 2; i <= Nx; i++) hx(i, j, k) = ((pz(i, j + 1, k) - pz(i, j, k)) - py(i, j, k + 1) + py(i, j, k)) / (c.dy * c.dz);
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= Nz - 1; k++)
    for (int j = 2; j <= Ny; j++)
      for (int i = 2; i <= Nx - 1; i++) hy(i, j, k) = ((px(i, j, k + 1) - px(i, j, k)) - pz(i + 1, j, k) + pz(i, j, k)) / (c.dz * c.dx);
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= Nz; k++)
    for (int j = 2; j <= Ny - 1; j++)
      for (int i = 2; i <= Nx - 1; i++) hz(i, j, k) = ((py(i + 1, j, k) - py(i, j, k)) - px(i, j + 1, k) + px(i, j, k)) / (c.dx * c.dy);
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= Nz; k++)
    for (int j = 2; j <= Ny; j++)
      for (int i = 2; i <= Nx - 1; i++)
        qx(i, j, k) = c.D[0](i, j, k) * px(i, j, k) + P.sxy * (hz(i, j, k) - hz(i, j - 1, k)) - P.sxz * (hy(i, j, k) - hy(i, j, k - 1));
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= Nz; k++)
    for (int j = 2; j <= Ny - 1; j++)
      for (int i = 2; i <= Nx; i++)
        qy(i, j, k) = c.D[1](i, j, k) * py(i, j, k) + P.syz * (hx(i, j, k) - hx(i, j, k - 1)) - P.syx * (hz(i, j, k) - hz(i - 1, j, k));
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= Nz - 1; k++)
    for (int j = 2; j <= Ny; j++)
      for (int i = 2; i <= Nx; i++)
        qz(i, j, k) = c.D[2](i, j, k) * pz(i, j, k) + P.szx * (hy(i, j, k) - hy(i - 1, j, k)) - P.szy * (hx(i, j, k) - hx(i, j - 1, k));
}

void pcg_zero_update(Ctx &c) {
  if (c.P.pcg_fast || c.P.pcg_f32) {
    if (c.warm && c.P.pcg_extrap) {
      for (int ax = 0; ax < 3; ax++) c.xprev[ax] = c.x[ax];
      c.have2 = true;
    } else {
      c.have2 = false;
    }
  }
  for (int ax = 0; ax < 3; ax++) std::fill(c.x[ax].begin(), c.x[ax].end(), 0.0);
  c.warm = true;
  c.iters = 0;
  for (int ax = 0; ax < 3; ax++) each(c.rng[ax], [&](int i, int j, int k) { c.ph[ax](i, j, k) = c.th[ax](i, j, k); });
}

int implicit_pcg(Ctx &c) {
  const bool fast = c.P.pcg_fast || c.P.pcg_f32;   // implicit.jl:177 (a PCGFast exists when either is set)
  const bool f32 = c.P.pcg_f32 != 0;
  for (int ax = 0; ax < 3; ax++) gather_diff(c, ax, c.b[ax]);
  scale_increment(c);
  double nb = std::sqrt(dot3(c.b, c.b));
  if (nb == 0) {
    pcg_zero_update(c);
    return 0;
  }
  if (!fast) {
    if (!c.warm) precond(c, c.x, c.b);
  } else {
    if (!c.warm) {
      precond(c, c.x, c.b);
      c.have2 = false;
    } else if (!c.P.pcg_extrap) {
    } else if (c.have2) {
      for (int ax = 0; ax < 3; ax++)
        for (size_t q = 0; q < c.x[ax].size(); q++) {
          double v = c.x[ax][q];
          c.x[ax][q] = 2 * v - c.xprev[ax][q];
          c.xprev[ax][q] = v;
        }
    } else {
      for (int ax = 0; ax < 3; ax++) c.xprev[ax] = c.x[ax];
      c.have2 = true;
    }
  }
  c.warm = true;
  scatter_full(c, c.Pf, c.x);
  apply_A(c);
  std::vector<double> q[3];
  for (int ax = 0; ax < 3; ax++) {
    gather_full(c, c.Qf, ax, q[ax]);
    c.r[ax].resize(c.b[ax].size());
    for (size_t t = 0; t < c.b[ax].size(); t++) c.r[ax][t] = c.b[ax][t] - q[ax][t];
  }
  int it = 0;
  int status = 0;
  if (nb > 0 && std::sqrt(dot3(c.r, c.r)) > c.P.pcg_tol * nb) {
    if (fast && f32) precond32(c, c.z, c.r);
    else precond(c, c.z, c.r);
    scatter_full(c, c.Pf, c.z);
    if (fast && f32)
      for (int ax = 0; ax < 3; ax++) c.zold[ax] = c.z[ax];
    double rz = dot3(c.r, c.z);
    std::vector<double> p[3];
    bool conv = false;
    while (it < c.P.pcg_maxit) {
      it++;
      apply_A(c);
      double pAp = 0.0;
      for (int ax = 0; ax < 3; ax++) {
        gather_full(c, c.Pf, ax, p[ax]);
        gather_full(c, c.Qf, ax, q[ax]);
        pAp += dot(p[ax], q[ax]);
      }
      double alpha = rz / pAp;
      for (int ax = 0; ax < 3; ax++)
        for (size_t t = 0; t < c.x[ax].size(); t++) {
          c.x[ax][t] += alpha * p[ax][t];
          c.r[ax][t] -= alpha * q[ax][t];
        }
      if (std::sqrt(dot3(c.r, c.r)) <= c.P.pcg_tol * nb) {
        conv = true;
        break;
      }
      if (fast && f32) precond32(c, c.z, c.r);
      else precond(c, c.z, c.r);
      double rz2 = dot3(c.r, c.z);
      double beta;
      if (fast && f32) {
        beta = (rz2 - dot3(c.r, c.zold)) / rz;
        for (int ax = 0; ax < 3; ax++) c.zold[ax] = c.z[ax];
      } else {
        beta = rz2 / rz;
      }
      rz = rz2;
      for (int ax = 0; ax < 3; ax++) {
        size_t t = 0;
        each(c.rng[ax], [&](int i, int j, int k) {
          c.Pf[ax](i, j, k) = c.z[ax][t] + beta * c.Pf[ax](i, j, k);
          t++;
        });
      }
    }
    if (!conv) status = TDGL_ENOCONV;
  }
  c.iters = it;
  c.total_iters += it;
  for (int ax = 0; ax < 3; ax++) scatter_sum(c, ax, c.x[ax]);
  return status;
}

void links(Ctx &c) {
  for (int k = 1; k <= c.Nz; k++) {
    if (2 <= k && k <= c.Nz) {
      for (int j = 2; j <= c.Ny; j++)
        for (int i = 1; i <= c.Nx; i++) c.U[0](i, j, k) = cis(-c.ph[0](i, j, k));
      for (int j = 1; j <= c.Ny; j++)
        for (int i = 2; i <= c.Nx; i++) c.U[1](i, j, k) = cis(-c.ph[1](i, j, k));
    }
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx; i++) c.U[2](i, j, k) = cis(-c.ph[2](i, j, k));
  }
}

void curl_h(Ctx &c) {
  R3 &px = c.ph[0], &py = c.ph[1], &pz = c.ph[2];
  for (int k = 2; k <= c.Nz - 1; k++)
    for (int j = 2; j <= c.Ny - 1; j++)
      for (int i = 2; i <= c.Nx; i++) c.h[0](i, j, k) = ((pz(i, j + 1, k) - pz(i, j, k)) - py(i, j, k + 1) + py(i, j, k)) / (c.dy * c.dz);
  for (int k = 2; k <= c.Nz - 1; k++)
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx - 1; i++) c.h[1](i, j, k) = ((px(i, j, k + 1) - px(i, j, k)) - pz(i + 1, j, k) + pz(i, j, k)) / (c.dz * c.dx);
  for (int k = 2; k <= c.Nz; k++)
    for (int j = 2; j <= c.Ny - 1; j++)
      for (int i = 2; i <= c.Nx - 1; i++) c.h[2](i, j, k) = ((py(i + 1, j, k) - py(i, j, k)) - px(i, j + 1, k) + px(i, j, k)) / (c.dx * c.dy);
}

// ---------------------------------------------------------------------------------------------- open boundary
double lgf(const Ctx &c, int i, int j, int k) {
  i = std::abs(i); j = std::abs(j); k = std::abs(k);
  const int R = c.P.open_R;
  if (std::max(i, std::max(j, k)) <= R) return c.green[i + (size_t)(R + 1) * (j + (size_t)(R + 1) * k)];
  double r2 = (double)(i * i + j * j + k * k), r = std::sqrt(r2);
  double i4 = (double)i * i * i * i, j4 = (double)j * j * j * j, k4 = (double)k * k * k * k;
  return (1 + (5 * (i4 + j4 + k4) / (r2 * r2) - 3) / (8 * r2)) / (4 * M_PI * r);
}

void open_setup(Ctx &c) {
  int sh[3][3] = {{c.Nx, c.Ny + 1, c.Nz + 1}, {c.Nx + 1, c.Ny, c.Nz + 1}, {c.Nx + 1, c.Ny + 1, c.Nz}};
  int hs[3][3] = {{c.Nx + 1, c.Ny, c.Nz}, {c.Nx, c.Ny + 1, c.Nz}, {c.Nx, c.Ny, c.Nz + 1}};
  for (int cc = 0; cc < 3; cc++) {
    for (int d = 0; d < 3; d++) c.o_M[cc][d] = 2 * sh[cc][d];
    C3 &Gh = c.o_ghat[cc];
    Gh.init(c.o_M[cc][0], c.o_M[cc][1], c.o_M[cc][2]);
    auto off = [](int a, int n) { return a <= n ? a - 1 : a - 1 - 2 * n; };
    for (int d3 = 1; d3 <= Gh.n3; d3++)
      for (int b2 = 1; b2 <= Gh.n2; b2++)
        for (int a1 = 1; a1 <= Gh.n1; a1++)
          Gh(a1, b2, d3) = C(c.P.open_fac * lgf(c, off(a1, sh[cc][0]), off(b2, sh[cc][1]), off(d3, sh[cc][2])), 0.0);
    fft3(Gh, -1);
    c.o_theta[cc].init(sh[cc][0], sh[cc][1], sh[cc][2]);
    c.o_old[cc].init(hs[cc][0], hs[cc][1], hs[cc][2]);
    c.o_new[cc].init(hs[cc][0], hs[cc][1], hs[cc][2]);
  }
}

void open_recompute(Ctx &c, double HJ) {
  const double k2 = c.P.kappa2;
  R3 &hx = c.h[0], &hy = c.h[1], &hz = c.h[2];
  C3 buf[3];
  for (int cc = 0; cc < 3; cc++) buf[cc].init(c.o_M[cc][0], c.o_M[cc][1], c.o_M[cc][2]);
  for (int k = 2; k <= c.Nz; k++)
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx - 1; i++)
        buf[0](i, j, k).re = k2 * ((hz(i, j, k) - hz(i, j - 1, k)) / c.dy - (hy(i, j, k) - hy(i, j, k - 1)) / c.dz) -
                             HJ * c.jbar[(j - 1) + (size_t)(c.Ny + 1) * (k - 1)];
  for (int k = 2; k <= c.Nz; k++)
    for (int j = 2; j <= c.Ny - 1; j++)
      for (int i = 2; i <= c.Nx; i++) buf[1](i, j, k).re = k2 * ((hx(i, j, k) - hx(i, j, k - 1)) / c.dz - (hz(i, j, k) - hz(i - 1, j, k)) / c.dx);
  for (int k = 2; k <= c.Nz - 1; k++)
    for (int j = 2; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx; i++) buf[2](i, j, k).re = k2 * ((hy(i, j, k) - hy(i - 1, j, k)) / c.dx - (hx(i, j, k) - hx(i, j - 1, k)) / c.dy);
  for (int cc = 0; cc < 3; cc++) {
    fft3(buf[cc], -1);
    for (size_t q = 0; q < buf[cc].size(); q++) buf[cc].v[q] = buf[cc].v[q] * c.o_ghat[cc].v[q];
    fft3(buf[cc], +1);
    const double inv = 1.0 / (double)buf[cc].size();
    R3 &T = c.o_theta[cc];
    for (int k = 1; k <= T.n3; k++)
      for (int j = 1; j <= T.n2; j++)
        for (int i = 1; i <= T.n1; i++) T(i, j, k) = buf[cc](i, j, k).re * inv;
  }
  // h_δ on the faces (openbc.jl:169-183)
  R3 &ftx = c.o_theta[0], &fty = c.o_theta[1], &ftz = c.o_theta[2];
  auto hzv = [&](int i, int j, int k) { return ((fty(i + 1, j, k) - fty(i, j, k)) - ftx(i, j + 1, k) + ftx(i, j, k)) / (c.dx * c.dy); };
  auto hxv = [&](int i, int j, int k) { return ((ftz(i, j + 1, k) - ftz(i, j, k)) - fty(i, j, k + 1) + fty(i, j, k)) / (c.dy * c.dz); };
  auto hyv = [&](int i, int j, int k) { return ((ftx(i, j, k + 1) - ftx(i, j, k)) - ftz(i + 1, j, k) + ftz(i, j, k)) / (c.dz * c.dx); };
  R3 &nx = c.o_new[0], &ny = c.o_new[1], &nz = c.o_new[2];
  for (int j : {1, c.Ny})
    for (int k = 1; k <= c.Nz + 1; k++)
      for (int i = 1; i <= c.Nx; i++) nz(i, j, k) = hzv(i, j, k);
  for (int j : {1, c.Ny})
    for (int k = 1; k <= c.Nz; k++)
      for (int i = 1; i <= c.Nx + 1; i++) nx(i, j, k) = hxv(i, j, k);
  for (int k : {1, c.Nz})
    for (int j = 1; j <= c.Ny + 1; j++)
      for (int i = 1; i <= c.Nx; i++) ny(i, j, k) = hyv(i, j, k);
  for (int k : {1, c.Nz})
    for (int j = 1; j <= c.Ny; j++)
      for (int i = 1; i <= c.Nx + 1; i++) nx(i, j, k) = hxv(i, j, k);
  for (int i : {1, c.Nx})
    for (int k = 1; k <= c.Nz + 1; k++)
      for (int j = 1; j <= c.Ny; j++) nz(i, j, k) = hzv(i, j, k);
  for (int i : {1, c.Nx})
    for (int k = 1; k <= c.Nz; k++)
      for (int j = 1; j <= c.Ny + 1; j++) ny(i, j, k) = hyv(i, j, k);
  c.open_recomputes++;
}

void open_update(Ctx &c, double HJ) {
  bool first = c.open_count < 0;
  c.open_count += 1;
  if (c.open_count >= c.P.open_every || first) {
    for (int cc = 0; cc < 3; cc++) c.o_old[cc].v = c.o_new[cc].v;
    open_recompute(c, HJ);
    if (first)
      for (int cc = 0; cc < 3; cc++) c.o_old[cc].v = c.o_new[cc].v;
    c.open_count = 0;
  }
}

void open_add(Ctx &c) {
  const double fr = std::min((c.open_count + 1) / (double)c.P.open_every, 1.0);
  R3 &o1 = c.o_old[0], &o2 = c.o_old[1], &o3 = c.o_old[2], &n1 = c.o_new[0], &n2 = c.o_new[1], &n3 = c.o_new[2];
  R3 &hx = c.h[0], &hy = c.h[1], &hz = c.h[2];
  for (int j : {1, c.Ny})
    for (int k = 1; k <= c.Nz + 1; k++)
      for (int i = 2; i <= c.Nx - 1; i++) hz(i, j, k) += o3(i, j, k) + fr * (n3(i, j, k) - o3(i, j, k));
  for (int j : {1, c.Ny})
    for (int k = 1; k <= c.Nz; k++)
      for (int i = 2; i <= c.Nx; i++) hx(i, j, k) = o1(i, j, k) + fr * (n1(i, j, k) - o1(i, j, k));
  for (int k : {1, c.Nz})
    for (int j = 1; j <= c.Ny + 1; j++)
      for (int i = 2; i <= c.Nx - 1; i++) hy(i, j, k) += o2(i, j, k) + fr * (n2(i, j, k) - o2(i, j, k));
  for (int k : {1, c.Nz})
    for (int j = 1; j <= c.Ny; j++)
      for (int i = 2; i <= c.Nx; i++) hx(i, j, k) = o1(i, j, k) + fr * (n1(i, j, k) - o1(i, j, k));
  for (int i : {1, c.Nx})
    for (int k = 1; k <= c.Nz + 1; k++)
      for (int j = 1; j <= c.Ny; j++) hz(i, j, k) += o3(i, j, k) + fr * (n3(i, j, k) - o3(i, j, k));
  for (int i : {1, c.Nx})
    for (int k = 1; k <= c.Nz; k++)
      for (int j = 1; j <= c.Ny + 1; j++) hy(i, j, k) += o2(i, j, k) + fr * (n2(i, j, k) - o2(i, j, k));
}

void field_bc(Ctx &c, double H, double HJ) {
  R3 &hx = c.h[0], &hy = c.h[1], &hz = c.h[2];
  const int Nx = c.Nx, Ny = c.Ny, Nz = c.Nz;
  for (int j = 1; j <= Ny; j++)
    for (int i = 1; i <= Nx; i++) hz(i, j, 1) = H, hz(i, j, Nz + 1) = H;
  for (int k = 1; k <= Nz + 1; k++)
    for (int j = 1; j <= Ny; j++) hz(1, j, k) = H, hz(Nx, j, k) = H;
  for (int k = 1; k <= Nz + 1; k++)
    for (int i = 1; i <= Nx; i++) hz(i, 1, k) = H, hz(i, Ny, k) = H;
  for (int k = 1; k <= Nz; k++)
    for (int j = 1; j <= Ny; j++) hx(1, j, k) = 0.0, hx(Nx + 1, j, k) = 0.0;
  for (int k = 1; k <= Nz; k++)
    for (int i = 1; i <= Nx + 1; i++) hx(i, 1, k) = 0.0, hx(i, Ny, k) = 0.0;
  for (int k = 1; k <= Nz; k++)
    for (int i = 1; i <= Nx; i++) hy(i, 1, k) = 0.0, hy(i, Ny + 1, k) = 0.0;
  if (c.P.selffield_bc == TDGL_BC_SLAB) {
    for (int j = 1; j <= Ny + 1; j++)
      for (int i = 1; i <= Nx; i++) hy(i, j, 1) = -HJ, hy(i, j, Nz) = +HJ;
  } else {
    const std::vector<double> &hy_z = c.bar[0], &hy_y = c.bar[1], &hz_z = c.bar[2], &hz_y = c.bar[3], &hz_x = c.bar[4], &hy_x = c.bar[5];
    int ks[2] = {1, Nz};
    for (int cc = 0; cc < 2; cc++)
      for (int j = 1; j <= Ny + 1; j++)
        for (int i = 1; i <= Nx; i++) hy(i, j, ks[cc]) = HJ * hy_z[(j - 1) + (size_t)(Ny + 1) * cc];
    int js[2] = {1, Ny + 1};
    for (int cc = 0; cc < 2; cc++)
      for (int k = 1; k <= Nz; k++)
        for (int i = 1; i <= Nx; i++) hy(i, js[cc], k) = HJ * hy_y[cc + 2 * (size_t)(k - 1)];
    int kz[2] = {1, Nz + 1};
    for (int cc = 0; cc < 2; cc++)
      for (int j = 1; j <= Ny; j++)
        for (int i = 1; i <= Nx; i++) hz(i, j, kz[cc]) = H + HJ * hz_z[(j - 1) + (size_t)Ny * cc];
    int jz[2] = {1, Ny};
    for (int cc = 0; cc < 2; cc++)
      for (int k = 1; k <= Nz + 1; k++)
        for (int i = 1; i <= Nx; i++) hz(i, jz[cc], k) = H + HJ * hz_y[cc + 2 * (size_t)(k - 1)];
    for (int i : {1, Nx})
      for (int k = 1; k <= Nz + 1; k++)
        for (int j = 1; j <= Ny; j++) hz(i, j, k) = H + HJ * hz_x[(j - 1) + (size_t)Ny * (k - 1)];
    for (int i : {1, Nx})
      for (int k = 1; k <= Nz; k++)
        for (int j = 1; j <= Ny + 1; j++) hy(i, j, k) = HJ * hy_x[(j - 1) + (size_t)(Ny + 1) * (k - 1)];
    if (c.P.selffield_bc == TDGL_BC_OPEN) open_add(c);
  }
}

void advance(Ctx &c) {
  for (int mu = 0; mu < c.N; mu++)
    for (int k = c.z1; k <= c.z2 + 1; k++)
      for (int j = c.y1; j <= c.y2 + 1; j++)
        for (int i = c.x1; i <= c.x2 + 1; i++) c.G[mu](i, j, k) = c.F[mu](i, j, k);
  for (int ax = 0; ax < 3; ax++) {
    std::swap(c.th[ax].v, c.ph[ax].v);
    std::swap(c.V[ax].v, c.U[ax].v);
  }
}

// _band_heat (terms.jl:47-52): the power band µ dissipates at a node over the step
double band_heat(double Gam, double gk, cd g, cd f, double invdt2) {
  if (gk == 0) return Gam * (abs2(f - g) * invdt2);
  const double g2 = gk * gk;
  const cd d = f - g;
  const double r = (conj(g) * d).re;
  return (Gam / std::sqrt(1 + g2 * abs2(g))) * ((abs2(d) + g2 * (r * r)) * invdt2);
}

// heat_step! (terms.jl:58-130, one material): the faces of θ copied from inside, then the in-place lexicographic
// sweep (a node reads the new θ of i−1, j−1, k−1 and the old one of i+1, j+1, k+1)
// qp_joule (exchange.jl:391-399; N fluids :516-531): the Joule heat of the normal fluids beyond σn|E|² at node
// (i, j, k), from this step's potentials; |∇·|² as the heat model takes |E|² (the mean over the two links of each axis)
double qp_joule(const Ctx &c, int i, int j, int k) {
  auto sq = [](double x) { return x * x; };
  auto grad2 = [&](const R3 &m) {
    return 0.5 * (sq(m(i + 1, j, k) - m(i, j, k)) + sq(m(i, j, k) - m(i - 1, j, k))) / (c.dx * c.dx) +
           0.5 * (sq(m(i, j + 1, k) - m(i, j, k)) + sq(m(i, j, k) - m(i, j - 1, k))) / (c.dy * c.dy) +
           0.5 * (sq(m(i, j, k + 1) - m(i, j, k)) + sq(m(i, j, k) - m(i, j, k - 1))) / (c.dz * c.dz);
  };
  const tdgl_params &P = c.P;
  if (P.qp_on == 1) return P.qp_sigma_n * P.qp_s[0] * P.qp_s[1] * grad2(c.qd) + P.qp_Gm[0][1] * sq(c.qd(i, j, k));
  double q = 0.0;
  for (int mu = 0; mu < c.N; mu++) q += P.qp_s[mu] * grad2(c.qmu[mu]);
  q *= P.qp_sigma_n;
  for (int mu = 0; mu < c.N; mu++)
    for (int nu = mu + 1; nu < c.N; nu++) q += P.qp_Gm[mu][nu] * sq(c.qmu[mu](i, j, k) - c.qmu[nu](i, j, k));
  return q;
}

void heat_step(Ctx &c) {
  R3 &T = c.Th;
  const tdgl_params &P = c.P;
  const double dt = P.dt, dx2 = c.dx * c.dx, dy2 = c.dy * c.dy, dz2 = c.dz * c.dz;
  const double gam = P.heat_gamma_bath, eta = P.heat_eta, thb = P.heat_T, den = 1 + dt * gam, invdt2 = 1 / (dt * dt);
  for (int k = c.z1; k <= c.z2 + 1; k++)
    for (int j = c.y1; j <= c.y2 + 1; j++) {
      T(c.x1, j, k) = T(c.x1 + 1, j, k);
      T(c.x2 + 1, j, k) = T(c.x2, j, k);
    }
  for (int k = c.z1; k <= c.z2 + 1; k++)
    for (int i = c.x1; i <= c.x2 + 1; i++) {
      T(i, c.y1, k) = T(i, c.y1 + 1, k);
      T(i, c.y2 + 1, k) = T(i, c.y2, k);
    }
  for (int j = c.y1; j <= c.y2 + 1; j++)
    for (int i = c.x1; i <= c.x2 + 1; i++) {
      T(i, j, c.z1) = T(i, j, c.z1 + 1);
      T(i, j, c.z2 + 1) = T(i, j, c.z2);
    }
  const int lo = c.x1 + P.heat_margin, hi = c.x2 + 1 - P.heat_margin;
  const double cx = invdt2 / dx2, cy = invdt2 / dy2, cz = invdt2 / dz2;
  // _heat_step_mat! (terms.jl:134-202): the node's Γ, γ̃ and σn; one D_T: the in-place sweep; D_T per material: the
  // neighbours of the step before (Jacobi) and the harmonic mean of the two D_T on each link
  const bool mat = c.haveMat;
  bool uni = true;
  if (mat)
    for (int m = 0; m < c.M.nmat; m++) uni = uni && c.M.heat_DT[m] == P.heat_DT;
  const R3 Rc = uni ? R3() : T;
  const R3 &R = uni ? T : Rc;
  auto hm = [](double a, double b) { return a == b ? a : 2 * a * b / (a + b); };
  for (int k = c.z1 + 1; k <= c.z2; k++)
    for (int j = c.y1 + 1; j <= c.y2; j++)
      for (int i = c.x1 + 1; i <= c.x2; i++) {
        const double q = R(i, j, k);
        const int m = mat ? c.matidx(i, j, k) : 0;
        double lap;
        if (uni) {
          lap = ((T(i + 1, j, k) - 2 * q) + T(i - 1, j, k)) / dx2 + ((T(i, j + 1, k) - 2 * q) + T(i, j - 1, k)) / dy2 +
                ((T(i, j, k + 1) - 2 * q) + T(i, j, k - 1)) / dz2;
        } else {   // the flux itself (D_T folded in): P.heat_DT · lap below is replaced
          const double *DT = c.M.heat_DT;
          const double d0 = DT[m];
          lap = (hm(d0, DT[c.matidx(i + 1, j, k)]) * (R(i + 1, j, k) - q) + hm(d0, DT[c.matidx(i - 1, j, k)]) * (R(i - 1, j, k) - q)) / dx2 +
                (hm(d0, DT[c.matidx(i, j + 1, k)]) * (R(i, j + 1, k) - q) + hm(d0, DT[c.matidx(i, j - 1, k)]) * (R(i, j - 1, k) - q)) / dy2 +
                (hm(d0, DT[c.matidx(i, j, k + 1)]) * (R(i, j, k + 1) - q) + hm(d0, DT[c.matidx(i, j, k - 1)]) * (R(i, j, k - 1) - q)) / dz2;
        }
        const double flux = uni ? P.heat_DT * lap : lap;
        const bool in = lo < i && i < hi;
        double src = 0.0;
        if (in) {
          if (mat) {
            for (int mu = 0; mu < c.N; mu++) src += band_heat(c.M.gamma[m][mu], c.M.gk[m][mu], c.G[mu](i, j, k), c.F[mu](i, j, k), invdt2);
          } else {
            src = band_heat(P.heat_Gamma[0], P.heat_gk[0], c.G[0](i, j, k), c.F[0](i, j, k), invdt2);
            for (int mu = 1; mu < c.N; mu++) src += band_heat(P.heat_Gamma[mu], P.heat_gk[mu], c.G[mu](i, j, k), c.F[mu](i, j, k), invdt2);
          }
        }
        const double sig = mat ? c.M.sigma_n[m] : P.heat_sigma_n;
        double acc;
        if (P.heat_joule) {
          double e2 = 0.0, qj = 0.0;
          if (in && c.f(i, j, k) > 0) {
            auto sq = [](double x) { return x * x; };
            if (P.qp_on) qj = qp_joule(c, i, j, k);   // terms.jl:107-108
            const double ex = 0.5 * (sq(c.th[0](i - 1, j, k) - c.ph[0](i - 1, j, k)) + sq(c.th[0](i, j, k) - c.ph[0](i, j, k))) * cx;
            const double ey = 0.5 * (sq(c.th[1](i, j - 1, k) - c.ph[1](i, j - 1, k)) + sq(c.th[1](i, j, k) - c.ph[1](i, j, k))) * cy;
            const double ez = 0.5 * (sq(c.th[2](i, j, k - 1) - c.ph[2](i, j, k - 1)) + sq(c.th[2](i, j, k) - c.ph[2](i, j, k))) * cz;
            e2 = (ex + ey) + ez;
          }
          acc = q + dt * (flux + eta * ((src + sig * e2) + qj));
        } else {
          acc = q + dt * (flux + eta * src);
        }
        double tn = (acc + dt * gam * thb) / den;
        if (tn < 0) tn = 0.0;
        else if (tn > P.heat_cap) tn = P.heat_cap;
        T(i, j, k) = tn;
      }
}

// ---------------------------------------------------------------------------------------------- two normal fluids
// _conv (exchange.jl:303-335, no drag): the conversion of band µ at node (i, j, k), the divergence of its link
// supercurrents over the live links (masks τ) plus the Josephson exchange with the other bands
// With materials (exchange.jl:359-366) the link weights are the band's ρ (τ included) and the Josephson row is that
// of the node's material.
double qp_conv(const Ctx &c, int mu, int i, int j, int k) {
  const C3 &P = c.G[mu];
  const C3 &Vx = c.V[0], &Vy = c.V[1], &Vz = c.V[2];
  const R3 &tx = c.haveMat ? c.rho[mu][0] : c.tx, &ty = c.haveMat ? c.rho[mu][1] : c.ty,
           &tz = c.haveMat ? c.rho[mu][2] : c.tz;
  const cd p = conj(P(i, j, k));
  const double gx = c.P.qp_g[mu][0], gy = c.P.qp_g[mu][1], gz = c.P.qp_g[mu][2];
  const double rx2 = 1 / (c.dx * c.dx), ry2 = 1 / (c.dy * c.dy), rz2 = 1 / (c.dz * c.dz);
  const double ax = tx(i, j, k) * (p * Vx(i, j, k) * P(i + 1, j, k)).im +
                    tx(i - 1, j, k) * (p * conj(Vx(i - 1, j, k)) * P(i - 1, j, k)).im;
  const double ay = ty(i, j, k) * (p * Vy(i, j, k) * P(i, j + 1, k)).im +
                    ty(i, j - 1, k) * (p * conj(Vy(i, j - 1, k)) * P(i, j - 1, k)).im;
  const double az = tz(i, j, k) * (p * Vz(i, j, k) * P(i, j, k + 1)).im +
                    tz(i, j, k - 1) * (p * conj(Vz(i, j, k - 1)) * P(i, j, k - 1)).im;
  double cv = ((gx * ax) * rx2 + (gy * ay) * ry2) + (gz * az) * rz2;
  const int m = c.haveMat ? c.matidx(i, j, k) : -1;
  for (int nu = 0; nu < c.N; nu++) {
    if (nu == mu) continue;
    const C3 &Q = c.G[nu];
    cv += (m >= 0 ? c.P.qp_mgamma[m][mu][nu] : c.P.qp_gamma[mu][nu]) * (p * Q(i, j, k)).im;
    if (c.P.drag_on && c.P.drag_nu[mu][nu] != 0) {   // the drag's share of the conversion (exchange.jl:327-332)
      const double qx = tx(i, j, k) * (p * Vx(i, j, k) * Q(i + 1, j, k)).im +
                        tx(i - 1, j, k) * (p * conj(Vx(i - 1, j, k)) * Q(i - 1, j, k)).im;
      const double qy = ty(i, j, k) * (p * Vy(i, j, k) * Q(i, j + 1, k)).im +
                        ty(i, j - 1, k) * (p * conj(Vy(i, j - 1, k)) * Q(i, j - 1, k)).im;
      const double qz = tz(i, j, k) * (p * Vz(i, j, k) * Q(i, j, k + 1)).im +
                        tz(i, j, k - 1) * (p * conj(Vz(i, j, k - 1)) * Q(i, j, k - 1)).im;
      cv += c.P.drag_nu[mu][nu] * ((qx * rx2 + qy * ry2) + qz * rz2);
    }
  }
  return cv;
}

// out[.., a, ..] = Σ_b M[a + n·b] A[.., b, ..] along `axis` of the n1 × n2 × n3 array A (in place; b in order)
void qp_axis(std::vector<double> &A, const int d[3], int axis, const std::vector<double> &M) {
  const int n = d[axis];
  std::vector<double> out(A.size(), 0.0);
  const size_t st = axis == 0 ? 1 : axis == 1 ? (size_t)d[0] : (size_t)d[0] * d[1];
  for (int k = 0; k < d[2]; k++)
    for (int j = 0; j < d[1]; j++)
      for (int i = 0; i < d[0]; i++) {
        const int a = axis == 0 ? i : axis == 1 ? j : k;
        const size_t o = (size_t)i + (size_t)d[0] * ((size_t)j + (size_t)d[1] * k);
        const size_t base = o - (size_t)a * st;
        double acc = 0.0;
        for (int b = 0; b < n; b++) acc += M[(size_t)a + (size_t)n * b] * A[base + (size_t)b * st];
        out[o] = acc;
      }
  A.swap(out);
}

// qp_potential! (exchange.jl:343-385, no materials, no sculpted vacuum): the source C_π/s_π − C_σ/s_σ on the nodes
// of the block, the separable solve of σn∇²δ − λ0 δ = S on the region (_qp_sep!: the three W, the division by
// σn (e_x + e_y + e_z) − λ0, the three V), then δ on the region's nodes, 0 on the x faces
// the separable solve of _qp_sep! in place: the three W, the division by σn (e_x + e_y + e_z) − λ, the three V
void qp_sep(const Ctx &c, std::vector<double> &S, const int d[3], double lam) {
  for (int ax = 0; ax < 3; ax++) qp_axis(S, d, ax, c.qW[ax]);
  for (int k = 0; k < d[2]; k++)
    for (int j = 0; j < d[1]; j++)
      for (int i = 0; i < d[0]; i++)
        S[(size_t)i + (size_t)d[0] * ((size_t)j + (size_t)d[1] * k)] /=
            c.P.qp_sigma_n * (c.qe[0][i] + c.qe[1][j] + c.qe[2][k]) - lam;
  for (int ax = 0; ax < 3; ax++) qp_axis(S, d, ax, c.qV[ax]);
}

// qp_potential! of QPExchangeN (exchange.jl:478-514, no sculpted vacuum): R_µ = C_µ/s_µ − ΣC on the nodes of the
// block, the modes M_k = Σ_µ Pinv[k, µ] R_µ, each solved with λ_k, then μ_µ = Σ_k P[µ, k] M_k on the region
void qp_cg(Ctx &c, std::vector<double> &S, const int d[3], double l0);

void qp_potential_n(Ctx &c) {
  const tdgl_params &P = c.P;
  const int N = c.N, n1 = c.Nx - 1, nj = P.qp_nj, nk = P.qp_nk, j0 = P.qp_j0 - 1, k0 = P.qp_k0 - 1;
  const int d[3] = {n1, nj, nk};
  const size_t nu = (size_t)n1 * nj * nk;
  std::vector<std::vector<double>> R(N, std::vector<double>(nu, 0.0)), M(N, std::vector<double>(nu, 0.0));
  double cv[TDGL_MAXB];
  for (int k = c.z1; k <= c.z2 + 1; k++)
    for (int j = c.y1; j <= c.y2 + 1; j++)
      for (int i = c.x1; i <= c.x2 + 1; i++) {
        for (int mu = 0; mu < N; mu++) cv[mu] = qp_conv(c, mu, i, j, k);
        double C = cv[0];
        for (int mu = 1; mu < N; mu++) C += cv[mu];
        const size_t o = (size_t)(i - 2) + (size_t)n1 * ((size_t)(j - j0 - 1) + (size_t)nj * (k - k0 - 1));
        for (int mu = 0; mu < N; mu++) R[mu][o] = cv[mu] / P.qp_s[mu] - C;
      }
  for (int kk = 0; kk < N; kk++)
    for (int mu = 0; mu < N; mu++)
      for (size_t o = 0; o < nu; o++) M[kk][o] += P.qp_Pinv[kk][mu] * R[mu][o];
  // each mode's Helmholtz problem: the separable solve, or in a sculpted sample conjugate gradients (skipped for a
  // mode without exchange and without source, exchange.jl:500-505); the iterations summed over the modes
  int its = 0;
  for (int kk = 0; kk < N; kk++) {
    if (c.qcond.empty()) {
      qp_sep(c, M[kk], d, P.qp_lam[kk]);
      continue;
    }
    double mx = 0.0;
    for (size_t o = 0; o < nu; o++) mx = std::max(mx, std::fabs(M[kk][o]));
    if (P.qp_lam[kk] > 0 || mx > 0) {
      qp_cg(c, M[kk], d, P.qp_lam[kk]);
      its += c.qp_iters;
    }
  }
  if (!c.qcond.empty()) c.qp_iters = its;
  for (int mu = 0; mu < N; mu++) {
    R3 &pot = c.qmu[mu];
    std::fill(pot.v.begin(), pot.v.end(), 0.0);
    for (int kz = 0; kz < nk; kz++)
      for (int jy = 0; jy < nj; jy++)
        for (int ix = 2; ix <= c.Nx; ix++) {
          const size_t o = (size_t)(ix - 2) + (size_t)n1 * ((size_t)jy + (size_t)nj * kz);
          double acc = 0.0;
          for (int kk = 0; kk < N; kk++) acc += P.qp_P[mu][kk] * M[kk][o];
          pot(ix, jy + 1 + j0, kz + 1 + k0) = acc;
        }
  }
}

// _qp_apply! (exchange.jl:52-84): y = −(σn∇²_c − λ) x on the unknowns: the links to a non-conducting unknown are
// cut, δ = 0 beyond the x ends, mirror ghosts on the y and z faces; a non-conducting unknown is decoupled
void qp_apply_cut(const Ctx &c, std::vector<double> &y, const std::vector<double> &x, const int d[3], double lam) {
  const int n1 = d[0], n2 = d[1], n3 = d[2];
  const double sn = c.P.qp_sigma_n, ax = sn / (c.dx * c.dx), ay = sn / (c.dy * c.dy), az = sn / (c.dz * c.dz);
  auto at = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (k - 1)); };
  auto C = [&](int i, int j, int k) { return c.qcond[at(i, j, k)] != 0; };
  auto X = [&](int i, int j, int k) { return x[at(i, j, k)]; };
  for (int k = 1; k <= n3; k++)
    for (int j = 1; j <= n2; j++)
      for (int i = 1; i <= n1; i++) {
        if (!C(i, j, k)) {
          y[at(i, j, k)] = (2 * ax + 2 * ay + 2 * az + lam) * X(i, j, k);
          continue;
        }
        const double v = X(i, j, k);
        double acc = lam * v;
        acc += ax * (v - (i > 1 ? (C(i - 1, j, k) ? X(i - 1, j, k) : v) : 0.0));
        acc += ax * (v - (i < n1 ? (C(i + 1, j, k) ? X(i + 1, j, k) : v) : 0.0));
        if (n2 > 1) {
          if (j == 1) {
            if (C(i, 2, k)) acc += 2 * ay * (v - X(i, 2, k));
          } else if (j == n2) {
            if (C(i, n2 - 1, k)) acc += 2 * ay * (v - X(i, n2 - 1, k));
          } else {
            if (C(i, j - 1, k)) acc += ay * (v - X(i, j - 1, k));
            if (C(i, j + 1, k)) acc += ay * (v - X(i, j + 1, k));
          }
        }
        if (n3 > 1) {
          if (k == 1) {
            if (C(i, j, 2)) acc += 2 * az * (v - X(i, j, 2));
          } else if (k == n3) {
            if (C(i, j, n3 - 1)) acc += 2 * az * (v - X(i, j, n3 - 1));
          } else {
            if (C(i, j, k - 1)) acc += az * (v - X(i, j, k - 1));
            if (C(i, j, k + 1)) acc += az * (v - X(i, j, k + 1));
          }
        }
        y[at(i, j, k)] = acc;
      }
}

// _qp_apply_var! (exchange.jl:233-256): y = −(∇·σ∇ − λ) x on the free unknowns with the coefficients of QPVar; a
// neighbour held at 0 adds its link to the diagonal, a cut one nothing; a non-free unknown is decoupled (y = d x)
void qp_apply_var(const Ctx &c, std::vector<double> &y, const std::vector<double> &x, const int d[3]) {
  const int n1 = d[0], n2 = d[1], n3 = d[2];
  const tdgl_params &P = c.P;
  auto at = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (k - 1)); };
  auto T = [&](int i, int j, int k) { return (int)c.qcond[at(i, j, k)]; };
  auto X = [&](int i, int j, int k) { return x[at(i, j, k)]; };
  auto CX = [&](int i, int j, int k) { return c.qcx[(size_t)(i - 1) + (size_t)(n1 + 1) * ((size_t)(j - 1) + (size_t)n2 * (k - 1))]; };
  auto CY = [&](int i, int j, int k) { return c.qcy[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)(n2 - 1) * (k - 1))]; };
  auto CZ = [&](int i, int j, int k) { return c.qcz[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (k - 1))]; };
  for (int k = 1; k <= n3; k++)
    for (int j = 1; j <= n2; j++)
      for (int i = 1; i <= n1; i++) {
        if (T(i, j, k) != 1) {
          y[at(i, j, k)] = P.qp_d * X(i, j, k);
          continue;
        }
        const double a = X(i, j, k);
        double acc = c.qlamv[at(i, j, k)] * a;
        auto nb = [&](double cc, int ii, int jj, int kk) {
          const int t = T(ii, jj, kk);
          return t == 1 ? cc * (a - X(ii, jj, kk)) : t == 2 ? cc * a : 0.0;
        };
        acc += i > 1 ? nb(CX(i, j, k), i - 1, j, k) : CX(1, j, k) * a;
        acc += i < n1 ? nb(CX(i + 1, j, k), i + 1, j, k) : CX(n1 + 1, j, k) * a;
        if (n2 > 1) {
          if (j == 1) acc += 2 * nb(CY(i, 1, k), i, 2, k);
          else if (j == n2) acc += 2 * nb(CY(i, n2 - 1, k), i, n2 - 1, k);
          else acc += nb(CY(i, j - 1, k), i, j - 1, k) + nb(CY(i, j, k), i, j + 1, k);
        }
        if (n3 > 1) {
          if (k == 1) acc += 2 * nb(CZ(i, j, 1), i, j, 2);
          else if (k == n3) acc += 2 * nb(CZ(i, j, n3 - 1), i, j, n3 - 1);
          else acc += nb(CZ(i, j, k - 1), i, j, k - 1) + nb(CZ(i, j, k), i, j, k + 1);
        }
        y[at(i, j, k)] = acc;
      }
}

// _qp_cg! (exchange.jl:87-121; with QPVar _qp_cg_var!, :258-290): (σn∇²_c − λ) x = S on the unknowns (S overwritten
// by x) by conjugate gradients in the inner product with weight 1/2 on each Neumann face, preconditioned by the
// separable solve projected on the free unknowns (with the sign that makes it positive)
void qp_cg(Ctx &c, std::vector<double> &S, const int d[3], double l0) {
  const tdgl_params &P = c.P;
  const bool var = !c.qcx.empty();
  const size_t n = S.size();
  const int n2 = d[1], n3 = d[2];
  std::vector<double> w(n), r(n), z(n), p(n), q(n), x(n);
  for (int k = 0; k < n3; k++)
    for (int j = 0; j < n2; j++)
      for (int i = 0; i < d[0]; i++)
        w[(size_t)i + (size_t)d[0] * ((size_t)j + (size_t)n2 * k)] =
            (j == 0 || j == n2 - 1 ? 0.5 : 1.0) * (k == 0 || k == n3 - 1 ? 0.5 : 1.0);
  auto wdot = [&](const std::vector<double> &a, const std::vector<double> &b) {
    double t = 0.0;
    for (size_t I = 0; I < n; I++) t += w[I] * a[I] * b[I];
    return t;
  };
  const double lam = std::max(l0, 1e-12 * P.qp_sigma_n), lsep = var ? lam : l0;
  auto apply = [&](std::vector<double> &yy, const std::vector<double> &xx) {
    if (var) qp_apply_var(c, yy, xx, d);
    else qp_apply_cut(c, yy, xx, d, lam);
  };
  for (size_t I = 0; I < n; I++)
    if (c.qcond[I] != 1) S[I] = 0.0;
  for (size_t I = 0; I < n; I++) r[I] = -S[I];
  const double bn = std::sqrt(wdot(r, r));
  if (bn == 0) {
    std::fill(S.begin(), S.end(), 0.0);
    c.qp_iters = 0;
    return;
  }
  auto prec = [&](std::vector<double> &zz, const std::vector<double> &rr) {
    zz = rr;
    qp_sep(c, zz, d, lsep);
    for (size_t I = 0; I < n; I++) zz[I] = c.qcond[I] == 1 ? -zz[I] : 0.0;
  };
  prec(z, r);
  x = z;
  apply(q, x);
  for (size_t I = 0; I < n; I++) r[I] = r[I] - q[I];
  prec(z, r);
  p = z;
  double rz = wdot(r, z);
  int it = 0;
  while (std::sqrt(wdot(r, r)) > P.qp_tol * bn && it < P.qp_maxit) {
    apply(q, p);
    const double alpha = rz / wdot(p, q);
    for (size_t I = 0; I < n; I++) x[I] = x[I] + alpha * p[I];
    for (size_t I = 0; I < n; I++) r[I] = r[I] - alpha * q[I];
    prec(z, r);
    const double rz2 = wdot(r, z);
    const double beta = rz2 / rz;
    rz = rz2;
    for (size_t I = 0; I < n; I++) p[I] = z[I] + beta * p[I];
    it++;
  }
  c.qp_iters = it;
  S = x;
}

void qp_potential(Ctx &c) {
  const tdgl_params &P = c.P;
  if (P.qp_on == 2) {
    qp_potential_n(c);
    return;
  }
  const int n1 = c.Nx - 1, nj = P.qp_nj, nk = P.qp_nk, j0 = P.qp_j0 - 1, k0 = P.qp_k0 - 1;
  const int d[3] = {n1, nj, nk};
  std::vector<double> S((size_t)n1 * nj * nk, 0.0);
  for (int k = c.z1; k <= c.z2 + 1; k++)
    for (int j = c.y1; j <= c.y2 + 1; j++)
      for (int i = c.x1; i <= c.x2 + 1; i++) {
        const double c1 = qp_conv(c, 0, i, j, k), c2 = qp_conv(c, 1, i, j, k);
        S[(size_t)(i - 2) + (size_t)n1 * ((size_t)(j - j0 - 1) + (size_t)nj * (k - k0 - 1))] = c2 / P.qp_s[1] - c1 / P.qp_s[0];
      }
  if (!c.qcond.empty()) qp_cg(c, S, d, P.qp_lambda0);
  else qp_sep(c, S, d, P.qp_lambda0);
  for (int k = 0; k < nk; k++)
    for (int j = 0; j < nj; j++) {
      c.qd(1, j + 1 + j0, k + 1 + k0) = 0.0;
      c.qd(c.Nx + 1, j + 1 + j0, k + 1 + k0) = 0.0;
      for (int i = 2; i <= c.Nx; i++) c.qd(i, j + 1 + j0, k + 1 + k0) = S[(size_t)(i - 2) + (size_t)n1 * ((size_t)j + (size_t)nj * k)];
    }
}

// qp_turn! (exchange.jl:403-414; N fluids :533-543): each band turns by e^{−iμ_µ dt} on the nodes the band update
// writes; two bands: μ_σ = −s_π δ, μ_π = s_σ δ
void qp_turn(Ctx &c) {
  if (c.P.qp_on == 2) {
    for (int mu = 0; mu < c.N; mu++)
      for (int k = c.z1 + 1; k <= c.z2; k++)
        for (int j = c.y1 + 1; j <= c.y2; j++)
          for (int i = c.x1 + 1; i <= c.x2; i++)
            c.F[mu](i, j, k) = c.F[mu](i, j, k) * cis(-c.P.dt * c.qmu[mu](i, j, k));
    return;
  }
  const double m[2] = {-c.P.qp_s[1], c.P.qp_s[0]};
  for (int mu = 0; mu < 2; mu++) {
    const double cc = m[mu] * c.P.dt;
    for (int k = c.z1 + 1; k <= c.z2; k++)
      for (int j = c.y1 + 1; j <= c.y2; j++)
        for (int i = c.x1 + 1; i <= c.x2; i++) c.F[mu](i, j, k) = c.F[mu](i, j, k) * cis(-cc * c.qd(i, j, k));
  }
}

int step(Ctx &c, double H, double HJ) {
  if (c.P.selffield_bc == TDGL_BC_OPEN) open_update(c, HJ);
  if (c.P.qp_on) qp_potential(c);
  update_bands(c);
  if (c.P.qp_on) qp_turn(c);
  if (c.P.noise_on) noise_after(c);
  supercurrent(c);
  if (c.P.heat_on) heat_step(c);
  field_increment(c);
  if (c.P.noise_on && c.P.noise_field) field_kick(c);
  int st = 0;
  if (c.P.solver == TDGL_SOLVER_SEP) implicit_sep(c);
  else if (c.P.solver == TDGL_SOLVER_PCG) st = implicit_pcg(c);
  else if (c.P.solver == TDGL_SOLVER_SCALE) scale_increment(c);
  links(c);
  curl_h(c);
  field_bc(c, H, HJ);
  for (int mu = 0; mu < c.N; mu++) ghosts(c, c.F[mu], c.U[0], c.U[1], c.U[2]);
  if (c.haveVac)   // neumann! (field.jl:235-244): the ghosts of the vacuum are vacuum too
    for (int mu = 0; mu < c.N; mu++)
      for (int k = 1; k <= c.Nz + 1; k++)
        for (int j = 1; j <= c.Ny + 1; j++)
          for (int i = 1; i <= c.Nx + 1; i++)
            if (c.isvac(i, j, k)) c.F[mu](i, j, k) = C(0.0, 0.0);
  advance(c);
  c.steps++;
  return st;
}

std::string g_err;

void copy_in(R3 &a, const double *p) { std::memcpy(a.v.data(), p, a.size() * sizeof(double)); }
void copy_in(C3 &a, const double *p) { std::memcpy(a.v.data(), p, a.size() * sizeof(cd)); }
void copy_out(const R3 &a, double *p) { std::memcpy(p, a.v.data(), a.size() * sizeof(double)); }
void copy_out(const C3 &a, double *p) { std::memcpy(p, a.v.data(), a.size() * sizeof(cd)); }

}  // namespace

extern "C" {

// the counter-based generator on its own, for known-answer and moment tests
void oracle_philox4x32_10(uint32_t *ctr, const uint32_t *key) { philox10(ctr, key[0], key[1]); }

void oracle_normals(uint64_t seed, uint64_t step, uint32_t stream, uint32_t node0, int n, double *out) {
  for (int q = 0; q < n; q++) {
    const cd z = normals_at(seed, step, stream, node0 + (uint32_t)q);
    out[2 * q] = z.re;
    out[2 * q + 1] = z.im;
  }
}

int oracle_ctx_create(const tdgl_params *p, oracle_ctx **out) {
  if (!p || !out) return TDGL_EINVAL;
  if (p->abi_version != TDGL_ABI_VERSION || p->nbands < 1 || p->nbands > TDGL_MAXB) {
    g_err = "bad abi version or band count";
    return TDGL_EINVAL;
  }
  Ctx *c = new Ctx();
  c->P = *p;
  c->N = p->nbands;
  const tdgl_grid &g = p->grid;
  c->Nx = g.Nx; c->Ny = g.Ny; c->Nz = g.Nz;
  c->x1 = g.x1; c->x2 = g.x2; c->y1 = g.y1; c->y2 = g.y2; c->z1 = g.z1; c->z2 = g.z2;
  c->dx = g.dx; c->dy = g.dy; c->dz = g.dz;
  const int n1 = g.Nx + 1, n2 = g.Ny + 1, n3 = g.Nz + 1;
  c->f.init(n1, n2, n3); c->tx.init(n1, n2, n3); c->ty.init(n1, n2, n3); c->tz.init(n1, n2, n3);
  copy_in(c->f, p->f); copy_in(c->tx, p->taux); copy_in(c->ty, p->tauy); copy_in(c->tz, p->tauz);
  if (p->vac) {
    c->haveVac = true;
    c->vac.assign(p->vac, p->vac + (size_t)n1 * n2 * n3);
  }
  if (p->materials) {   // MatField (materials.jl:83-114): the node map, the tables and the link weights ρ
    const tdgl_materials &M = *p->materials;
    if (M.nmat < 1 || M.nmat > TDGL_MAXMAT || !M.idx) {
      g_err = "bad materials";
      delete c;
      return TDGL_EINVAL;
    }
    c->haveMat = true;
    c->M = M;
    c->M.idx = nullptr;
    c->mat.assign(M.idx, M.idx + (size_t)n1 * n2 * n3);
    for (uint8_t v : c->mat)
      if (v < 1 || v > M.nmat) {
        g_err = "material index out of range";
        delete c;
        return TDGL_EINVAL;
      }
    for (int mu = 0; mu < p->nbands; mu++)
      for (int m = 0; m < M.nmat; m++) c->haskwt[mu] = c->haskwt[mu] || M.full[m][mu].gamma2 > 0;
    R3 *tau[3] = {&c->tx, &c->ty, &c->tz};
    for (int mu = 0; mu < p->nbands; mu++)
      for (int ax = 0; ax < 3; ax++) {
        R3 &r = c->rho[mu][ax];
        r.init(n1, n2, n3);
        const double m0 = M.ma[0][mu][ax];
        for (int k = 1; k <= n3; k++)
          for (int j = 1; j <= n2; j++)
            for (int i = 1; i <= n1; i++) {
              const double tv = (*tau[ax])(i, j, k);
              const int di = i + (ax == 0), dj = j + (ax == 1), dk = k + (ax == 2);
              if (di > n1 || dj > n2 || dk > n3) {   // no node across: ρ keeps τ
                r(i, j, k) = tv;
                continue;
              }
              const int a = c->matidx(i, j, k), b = c->matidx(di, dj, dk);
              const double ma = M.ma[a][mu][ax], mb = M.ma[b][mu][ax];
              const double ml = ma == mb ? ma : (ma + mb) / 2;
              const double w = (ml == m0 ? 1.0 : m0 / ml) * (a == b ? 1.0 : M.transparency[a][b]);
              r(i, j, k) = (M.absent[a][mu] || M.absent[b][mu]) ? 0.0 : tv * w;
            }
      }
  }
  int ls[3][3] = {{g.Nx, g.Ny + 1, g.Nz + 1}, {g.Nx + 1, g.Ny, g.Nz + 1}, {g.Nx + 1, g.Ny + 1, g.Nz}};
  int hs[3][3] = {{g.Nx + 1, g.Ny, g.Nz}, {g.Nx, g.Ny + 1, g.Nz}, {g.Nx, g.Ny, g.Nz + 1}};
  if (p->Dx && p->Dy && p->Dz) {
    c->haveD = true;
    const double *Ds[3] = {p->Dx, p->Dy, p->Dz};
    for (int ax = 0; ax < 3; ax++) {
      c->D[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
      copy_in(c->D[ax], Ds[ax]);
    }
  } else if (p->solver == TDGL_SOLVER_SCALE || p->solver == TDGL_SOLVER_PCG) {
    g_err = "SCALE and PCG need the link conductivity D";
    delete c;
    return TDGL_EINVAL;
  }
  if (p->selffield_bc != TDGL_BC_SLAB) {
    size_t sz[6] = {(size_t)(g.Ny + 1) * 2, (size_t)2 * g.Nz, (size_t)g.Ny * 2, (size_t)2 * (g.Nz + 1), (size_t)g.Ny * (g.Nz + 1),
                    (size_t)(g.Ny + 1) * g.Nz};
    const double *src[6] = {p->bar_hy_z, p->bar_hy_y, p->bar_hz_z, p->bar_hz_y, p->bar_hz_x, p->bar_hy_x};
    for (int q = 0; q < 6; q++) {
      if (!src[q]) {
        g_err = "bar tables missing";
        delete c;
        return TDGL_EINVAL;
      }
      c->bar[q].assign(src[q], src[q] + sz[q]);
    }
  }
  for (int mu = 0; mu < c->N; mu++) {
    c->G[mu].init(n1, n2, n3);
    c->F[mu].init(n1, n2, n3);
  }
  for (int ax = 0; ax < 3; ax++) {
    c->th[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->ph[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->J[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->U[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->V[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->L[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->Rl[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->Rr[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->h[ax].init(hs[ax][0], hs[ax][1], hs[ax][2]);
    c->Pf[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->Qf[ax].init(ls[ax][0], ls[ax][1], ls[ax][2]);
    c->Hf[ax].init(hs[ax][0], hs[ax][1], hs[ax][2]);
  }
  c->W.init(n1, n2, n3);
  c->W2.init(n1, n2, n3);
  c->Om.init(n1, n2, n3);
  if (p->qp_on) {   // exchange.jl: QPExchange's bases and δ (zero outside the region)
    if ((p->qp_on == 1 && p->nbands != 2) || p->qp_on < 1 || p->qp_on > 2 || p->qp_nj < 1 || p->qp_nk < 1 || p->qp_j0 < 1 || p->qp_k0 < 1 ||
        p->qp_j0 + p->qp_nj - 1 > g.Ny + 1 || p->qp_k0 + p->qp_nk - 1 > g.Nz + 1 || !p->qp_Vx || !p->qp_Wx ||
        !p->qp_ex || !p->qp_Vy || !p->qp_Wy || !p->qp_ey || !p->qp_Vz || !p->qp_Wz || !p->qp_ez) {
      g_err = "qp_exchange: two bands, a region inside the grid and the three bases";
      delete c;
      return TDGL_EINVAL;
    }
    const int nq[3] = {g.Nx - 1, p->qp_nj, p->qp_nk};
    const double *Vs[3] = {p->qp_Vx, p->qp_Vy, p->qp_Vz}, *Ws[3] = {p->qp_Wx, p->qp_Wy, p->qp_Wz},
                 *es[3] = {p->qp_ex, p->qp_ey, p->qp_ez};
    for (int ax = 0; ax < 3; ax++) {
      const size_t nn = (size_t)nq[ax] * nq[ax];
      c->qV[ax].assign(Vs[ax], Vs[ax] + nn);
      c->qW[ax].assign(Ws[ax], Ws[ax] + nn);
      c->qe[ax].assign(es[ax], es[ax] + nq[ax]);
    }
    c->qd.init(n1, n2, n3);
    if (p->qp_cond) c->qcond.assign(p->qp_cond, p->qp_cond + (size_t)nq[0] * nq[1] * nq[2]);
    if (p->qp_cond && p->qp_cx) {
      const size_t a = (size_t)(nq[0] + 1) * nq[1] * nq[2], b = (size_t)nq[0] * std::max(nq[1] - 1, 0) * nq[2],
                   cz = (size_t)nq[0] * nq[1] * std::max(nq[2] - 1, 0), u = (size_t)nq[0] * nq[1] * nq[2];
      c->qcx.assign(p->qp_cx, p->qp_cx + a);
      c->qcy.assign(p->qp_cy, p->qp_cy + b);
      c->qcz.assign(p->qp_cz, p->qp_cz + cz);
      c->qlamv.assign(p->qp_lamv, p->qp_lamv + u);
    }
    c->P.qp_cx = c->P.qp_cy = c->P.qp_cz = c->P.qp_lamv = nullptr;
    c->P.qp_cond = nullptr;
    if (p->qp_on == 2)
      for (int mu = 0; mu < p->nbands; mu++) c->qmu[mu].init(n1, n2, n3);
  }
  if (p->heat_on) {   // scheme.jl:403: the bath everywhere
    c->Th.init(n1, n2, n3);
    std::fill(c->Th.v.begin(), c->Th.v.end(), p->heat_T);
  }
  c->Oms.init(n1, n2, n3);
  c->rng[0] = Range{2, g.Nx - 1, 2, g.Ny, 2, g.Nz};
  c->rng[1] = Range{2, g.Nx, 2, g.Ny - 1, 2, g.Nz};
  c->rng[2] = Range{2, g.Nx, 2, g.Ny, 2, g.Nz - 1};
  if (p->solver == TDGL_SOLVER_SEP || p->solver == TDGL_SOLVER_PCG) {
    c->bx.make(g.Nx - 1);
    c->by.make(g.Ny - 1);
    c->bz.make(g.Nz - 1);
    c->sep.make(c->bx, c->by, c->bz, p->a_imp);
    c->sep32.make(c->bx, c->by, c->bz, p->a_imp);
    for (int ax = 0; ax < 3; ax++) {
      size_t n = c->rng[ax].n();
      c->x[ax].assign(n, 0); c->r[ax].assign(n, 0); c->z[ax].assign(n, 0); c->b[ax].assign(n, 0);
      c->xprev[ax].assign(n, 0); c->zold[ax].assign(n, 0);
    }
  }
  if (p->selffield_bc == TDGL_BC_OPEN) {
    if (!p->open_green || !p->open_jbar || p->open_every < 1) {
      g_err = "open boundary tables missing";
      delete c;
      return TDGL_EINVAL;
    }
    size_t gsz = (size_t)(p->open_R + 1) * (p->open_R + 1) * (p->open_R + 1);
    c->green.assign(p->open_green, p->open_green + gsz);
    c->jbar.assign(p->open_jbar, p->open_jbar + (size_t)(g.Ny + 1) * (g.Nz + 1));
    open_setup(*c);
  }
  *out = c;
  return 0;
}

int oracle_ctx_destroy(oracle_ctx *c) {
  delete c;
  return 0;
}

int oracle_upload_state(oracle_ctx *c, const tdgl_state_view *s) {
  for (int mu = 0; mu < c->N; mu++) {
    copy_in(c->G[mu], s->G[mu]);
    copy_in(c->F[mu], s->F[mu]);
  }
  for (int ax = 0; ax < 3; ax++) {
    copy_in(c->th[ax], s->th[ax]); copy_in(c->ph[ax], s->ph[ax]);
    copy_in(c->U[ax], s->U[ax]); copy_in(c->V[ax], s->V[ax]);
    copy_in(c->J[ax], s->J[ax]); copy_in(c->h[ax], s->h[ax]);
  }
  c->have_state = true;
  return 0;
}

int oracle_download_state(oracle_ctx *c, const tdgl_state_view *s) {
  for (int mu = 0; mu < c->N; mu++) {
    copy_out(c->G[mu], s->G[mu]);
    copy_out(c->F[mu], s->F[mu]);
  }
  for (int ax = 0; ax < 3; ax++) {
    copy_out(c->th[ax], s->th[ax]); copy_out(c->ph[ax], s->ph[ax]);
    copy_out(c->U[ax], s->U[ax]); copy_out(c->V[ax], s->V[ax]);
    copy_out(c->J[ax], s->J[ax]); copy_out(c->h[ax], s->h[ax]);
  }
  return 0;
}

int oracle_set_carry(oracle_ctx *c, const tdgl_carry_view *v) {
  if (c->P.solver == TDGL_SOLVER_PCG) {
    size_t off = 0;
    for (int ax = 0; ax < 3; ax++) {
      size_t n = c->rng[ax].n();
      if (v->pcg_x) std::memcpy(c->x[ax].data(), v->pcg_x + off, n * sizeof(double));
      if (v->pcg_xprev) std::memcpy(c->xprev[ax].data(), v->pcg_xprev + off, n * sizeof(double));
      off += n;
    }
    c->warm = v->pcg_warm != 0;
    c->have2 = v->pcg_have2 != 0;
  }
  if (c->P.heat_on && v->heat_theta) copy_in(c->Th, v->heat_theta);
  if (c->P.selffield_bc == TDGL_BC_OPEN) {
    c->open_count = v->open_count;
    for (int ax = 0; ax < 3; ax++) {
      if (v->open_old[ax]) copy_in(c->o_old[ax], v->open_old[ax]);
      if (v->open_new[ax]) copy_in(c->o_new[ax], v->open_new[ax]);
      if (v->open_theta[ax]) copy_in(c->o_theta[ax], v->open_theta[ax]);
    }
  }
  return 0;
}

int oracle_get_carry(oracle_ctx *c, tdgl_carry_view *v) {
  if (c->P.solver == TDGL_SOLVER_PCG) {
    size_t off = 0;
    for (int ax = 0; ax < 3; ax++) {
      size_t n = c->rng[ax].n();
      if (v->pcg_x) std::memcpy(v->pcg_x + off, c->x[ax].data(), n * sizeof(double));
      if (v->pcg_xprev) std::memcpy(v->pcg_xprev + off, c->xprev[ax].data(), n * sizeof(double));
      off += n;
    }
    v->pcg_warm = c->warm;
    v->pcg_have2 = c->have2;
  }
  if (c->P.heat_on && v->heat_theta) copy_out(c->Th, v->heat_theta);
  if (c->P.selffield_bc == TDGL_BC_OPEN) {
    v->open_count = c->open_count;
    for (int ax = 0; ax < 3; ax++) {
      if (v->open_old[ax]) copy_out(c->o_old[ax], v->open_old[ax]);
      if (v->open_new[ax]) copy_out(c->o_new[ax], v->open_new[ax]);
      if (v->open_theta[ax]) copy_out(c->o_theta[ax], v->open_theta[ax]);
    }
  }
  return 0;
}

int oracle_steps(oracle_ctx *c, int n, double H, double HJ) {
  if (!c->have_state) return TDGL_ESTATE;
  int st = 0;
  for (int q = 0; q < n; q++) {
    int r = step(*c, H, HJ);
    if (r && !st) st = r;
  }
  return st;
}

int oracle_steps_ramp(oracle_ctx *c, int n, double H, const double *HJ) {
  if (!c->have_state) return TDGL_ESTATE;
  int st = 0;
  for (int q = 0; q < n; q++) {
    int r = step(*c, H, HJ[q]);
    if (r && !st) st = r;
  }
  return st;
}

int oracle_get_stats(oracle_ctx *c, tdgl_stats *s) {
  s->steps = c->steps;
  s->pcg_last_iters = c->iters;
  s->pcg_total_iters = c->total_iters;
  s->open_recomputes = c->open_recomputes;
  s->kernel_launches_last_call = 0;
  return 0;
}

const char *oracle_last_error(void) { return g_err.c_str(); }

// δ of the two normal fluids (qp_potential!) from the context's current state, node-shaped (Nx+1)(Ny+1)(Nz+1)
int oracle_qp_delta(oracle_ctx *c, double *out) {
  if (!c || !out || c->P.qp_on != 1) return TDGL_EINVAL;
  qp_potential(*c);
  std::copy(c->qd.v.begin(), c->qd.v.end(), out);
  return 0;
}

// the conjugate-gradient iterations of the last δ solve of a sculpted sample
int oracle_qp_iters(oracle_ctx *c) { return c ? c->qp_iters : -1; }

// the potentials μ_µ of N fluids (QPExchangeN's qp_potential!) from the current state: N node-shaped arrays in turn
int oracle_qp_mu(oracle_ctx *c, double *out) {
  if (!c || !out || c->P.qp_on != 2) return TDGL_EINVAL;
  qp_potential(*c);
  for (int mu = 0; mu < c->N; mu++) std::copy(c->qmu[mu].v.begin(), c->qmu[mu].v.end(), out + mu * c->qmu[mu].v.size());
  return 0;
}

// OpenMP threads of the parallel passes (the CPU baseline is timed on every host thread and on one)
void oracle_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

// The field solve of step! alone (step.jl:26-30: implicit_curl! with the SepSolver or the PCG, or
// scale_increment!) on the uploaded θ and φ, as the reference's PCG zero-source test drives it
// (gtdgl/test/pcg_zero_fixture.jl: `TDGL.implicit_curl!(s, st.imp)`).
int oracle_field_solve(oracle_ctx *c) {
  if (!c->have_state) return TDGL_ESTATE;
  int st = 0;
  if (c->P.solver == TDGL_SOLVER_SEP) implicit_sep(*c);
  else if (c->P.solver == TDGL_SOLVER_PCG) st = implicit_pcg(*c);
  else if (c->P.solver == TDGL_SOLVER_SCALE) scale_increment(*c);
  return st;
}

// The temporal link rotations on plain column-major arrays of dims (n1, n2, n3) over the 1-based inclusive range
// rng = {i0, i1, j0, j1, k0, k1} (gtdgl/test/test_link_rotations.jl drives _rot!, _rotfrac! and _link_rate! on
// manufactured links): op 0 = _rot! (L = V, R = Q^{1/par}, complex), op 1 = _rotfrac! (L = V Q^par), op 2 =
// _link_rate! along axis ax (R real: −arg Q + (Ω[I + e_ax] − Ω[I])·par).  V, U, L and complex R interleaved.
int oracle_link_rotations(int op, int n1, int n2, int n3, const int *rng, int ax, const double *V, const double *U,
                          const double *Om, double par, double *L, double *R) {
  if (op < 0 || op > 2 || ax < 0 || ax > 2) return TDGL_EINVAL;
  const cd *v = reinterpret_cast<const cd *>(V), *u = reinterpret_cast<const cd *>(U);
  auto at = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (k - 1)); };
  const int oi = ax == 0, oj = ax == 1, ok = ax == 2;
  for (int k = rng[4]; k <= rng[5]; k++)
    for (int j = rng[2]; j <= rng[3]; j++)
      for (int i = rng[0]; i <= rng[1]; i++) {
        const size_t o = at(i, j, k);
        if (op == 0) {
          reinterpret_cast<cd *>(L)[o] = v[o];
          reinterpret_cast<cd *>(R)[o] = link_root(v[o], u[o], par);
        } else if (op == 1) {
          reinterpret_cast<cd *>(L)[o] = link_frac(v[o], u[o], par);
        } else {
          R[o] = link_angle(v[o], u[o]) + (Om[at(i + oi, j + oj, k + ok)] - Om[o]) * par;
        }
      }
  (void)n3;
  return 0;
}

// _cis (bands.jl:289) and kwt_update (bands.jl:135-140) as scalar functions (test_link_rotations.jl:29,
// test_physics.jl:50-59)
void oracle_cis_short(double a, double *out) {
  const cd z = cis_short(a);
  out[0] = z.re;
  out[1] = z.im;
}
void oracle_kwt_update(const double *g, const double *d, double g2, double *out) {
  const cd z = kwt_update(C(g[0], g[1]), C(d[0], d[1]), g2);
  out[0] = z.re;
  out[1] = z.im;
}

// (I + aK)^{-1} applied to b (the three range arrays packed x, y, z) in double (f32 = 0) or float (f32 = 1).
int oracle_sep_apply(oracle_ctx *c, double *b, int f32) {
  if (c->P.solver != TDGL_SOLVER_SEP && c->P.solver != TDGL_SOLVER_PCG) return TDGL_EINVAL;
  std::vector<double> B[3], Z[3];
  size_t off = 0;
  for (int ax = 0; ax < 3; ax++) {
    size_t n = c->rng[ax].n();
    B[ax].assign(b + off, b + off + n);
    off += n;
  }
  if (f32) precond32(*c, Z, B);
  else precond(*c, Z, B);
  off = 0;
  for (int ax = 0; ax < 3; ax++) {
    std::memcpy(b + off, Z[ax].data(), Z[ax].size() * sizeof(double));
    off += Z[ax].size();
  }
  return 0;
}

// The bar field tables (field.jl:151-180), restated independently of the host mirror, for cross-checks.
int oracle_bar_field(const tdgl_grid *g, int nq, double *hy_z, double *hy_y, double *hz_z, double *hz_y, double *hz_x, double *hy_x) {
  const int Ny = g->Ny, Nz = g->Nz, y1 = g->y1, y2 = g->y2, z1 = g->z1, z2 = g->z2;
  const double dy = g->dy, dz = g->dz;
  const double ya = (y1 - 1) * dy, yb = y2 * dy, za = (z1 - 1) * dz, zb = z2 * dz;
  const double d = (z2 - z1 + 1) * dz;
  const double cc = (-2 / d) / (2 * M_PI);
  const int ny = nq * (y2 - y1 + 1), nz = nq * (z2 - z1 + 1);
  const double hq = (yb - ya) / ny, kq = (zb - za) / nz;
  auto h = [&](double y, double z, double &oy, double &oz) {
    double hy = 0.0, hz = 0.0;
    for (int b = 1; b <= nz; b++)
      for (int a = 1; a <= ny; a++) {
        double yp = ya + (a - 0.5) * hq, zp = za + (b - 0.5) * kq;
        double r2 = (y - yp) * (y - yp) + (z - zp) * (z - zp);
        hy += -(z - zp) / r2;
        hz += (y - yp) / r2;
      }
    oy = cc * hy * hq * kq;
    oz = cc * hz * hq * kq;
  };
  auto yc = [&](int j) { return (j - 0.5) * dy; };
  auto yn = [&](int j) { return (j - 1) * dy; };
  auto zc = [&](int k) { return (k - 0.5) * dz; };
  auto zn = [&](int k) { return (k - 1) * dz; };
  double a, b;
  int kk[2] = {1, Nz};
  for (int c2 = 0; c2 < 2; c2++)
    for (int j = 1; j <= Ny + 1; j++) { h(yn(j), zc(kk[c2]), a, b); hy_z[(j - 1) + (Ny + 1) * c2] = a; }
  int jj[2] = {1, Ny + 1};
  for (int k = 1; k <= Nz; k++)
    for (int c2 = 0; c2 < 2; c2++) { h(yn(jj[c2]), zc(k), a, b); hy_y[c2 + 2 * (k - 1)] = a; }
  int kz[2] = {1, Nz + 1};
  for (int c2 = 0; c2 < 2; c2++)
    for (int j = 1; j <= Ny; j++) { h(yc(j), zn(kz[c2]), a, b); hz_z[(j - 1) + Ny * c2] = b; }
  int jz[2] = {1, Ny};
  for (int k = 1; k <= Nz + 1; k++)
    for (int c2 = 0; c2 < 2; c2++) { h(yc(jz[c2]), zn(k), a, b); hz_y[c2 + 2 * (k - 1)] = b; }
  for (int k = 1; k <= Nz + 1; k++)
    for (int j = 1; j <= Ny; j++) { h(yc(j), zn(k), a, b); hz_x[(j - 1) + Ny * (k - 1)] = b; }
  for (int k = 1; k <= Nz; k++)
    for (int j = 1; j <= Ny + 1; j++) { h(yn(j), zc(k), a, b); hy_x[(j - 1) + (Ny + 1) * (k - 1)] = a; }
  return 0;
}

}  // extern "C"
