// heat.cu — the heat model's temperature field (gtdgl/src/terms.jl: Heat, _band_heat, heat_step! with one material).
//
// The reference updates θ in place in lexicographic order: a node reads the new θ of its i−1, j−1 and k−1
// neighbours and the old θ of i+1, j+1 and k+1.  The same order on the device is a sweep over the planes
// i + j + k = s: every node of a plane depends only on the planes before it, so each plane's nodes are updated at
// once and the result is the reference's to the bit.  One block takes the whole sweep (the faces first, then the
// planes, a block barrier between them): the heat model is an optional term that no benchmark configuration uses,
// and the sweep's planes are too small to fill the GPU.
#include "common.cuh"

namespace tdgl {
namespace {

const int HT_THREADS = 1024;

struct HeatArgs {
  double *T;
  BandPtrs G, F;
  const double *th[3], *ph[3], *f;
  int N, x1, x2, y1, y2, z1, z2;
  Dim d;
  double dt, dx2, dy2, dz2, DT, gam, eta, thb, cap, sig;
  int joule, margin;
  double Gam[TDGL_MAXB], gk[TDGL_MAXB];
  // materials (_heat_step_mat!, terms.jl:134-202): the node map, each material's Γ, γ̃, σn and D_T; uni: one D_T (the
  // in-place sweep), else R holds the field of the step before and every node is updated from it (Jacobi)
  const uint8_t *mat;
  double Gm[TDGL_MAXMAT][TDGL_MAXB], gkm[TDGL_MAXMAT][TDGL_MAXB], sigm[TDGL_MAXMAT], DTm[TDGL_MAXMAT];
  int uni;
  double *R;
  // normal fluids per band (qp_joule, exchange.jl): 1 two bands (δ in qmu[0]), 2 N fluids (μ_µ); 0 none
  int qp;
  const double *qmu[TDGL_MAXB];
  double qs[TDGL_MAXB], qsig, qGm[TDGL_MAXB][TDGL_MAXB];
};

// qp_joule (exchange.jl:391-399; N fluids :516-531): the Joule heat of the normal fluids beyond σn|E|² at node o,
// from this step's potentials; |∇·|² as the heat model takes |E|² (the mean over the two links of each axis)
__device__ double qp_joule(const HeatArgs &A, long long o, long long sx, long long sy, long long sz) {
  auto grad2 = [&](const double *m) {
    const double a0 = m[o + sx] - m[o], a1 = m[o] - m[o - sx], b0 = m[o + sy] - m[o], b1 = m[o] - m[o - sy],
                 c0 = m[o + sz] - m[o], c1 = m[o] - m[o - sz];
    return 0.5 * (a0 * a0 + a1 * a1) / A.dx2 + 0.5 * (b0 * b0 + b1 * b1) / A.dy2 + 0.5 * (c0 * c0 + c1 * c1) / A.dz2;
  };
  if (A.qp == 1) {
    const double d = A.qmu[0][o];
    return A.qsig * A.qs[0] * A.qs[1] * grad2(A.qmu[0]) + A.qGm[0][1] * (d * d);
  }
  double q = 0.0;
  for (int mu = 0; mu < A.N; mu++) q += A.qs[mu] * grad2(A.qmu[mu]);
  q *= A.qsig;
  for (int mu = 0; mu < A.N; mu++)
    for (int nu = mu + 1; nu < A.N; nu++) {
      const double e = A.qmu[mu][o] - A.qmu[nu][o];
      q += A.qGm[mu][nu] * (e * e);
    }
  return q;
}

__device__ __forceinline__ double band_heat(double Gam, double gk, cd g, cd f, double invdt2) {
  if (gk == 0) return Gam * (cabs2(csub(f, g)) * invdt2);
  const double g2 = gk * gk;
  const cd d = csub(f, g);
  const double r = cmul(cconj(g), d).x;
  return (Gam / sqrt(1 + g2 * cabs2(g))) * ((cabs2(d) + g2 * (r * r)) * invdt2);
}

__global__ void __launch_bounds__(HT_THREADS) k_heat(HeatArgs A) {
  const Dim d = A.d;
  double *T = A.T;
  const int tid = threadIdx.x;
  auto at = [&](int i, int j, int k) { return d.at(i, j, k); };
  // the faces, copied from inside: x, then y (over the x faces too), then z (terms.jl:70-78)
  const int ny1 = A.y2 + 2 - A.y1, nz1 = A.z2 + 2 - A.z1, nx1 = A.x2 + 2 - A.x1;
  for (int t = tid; t < ny1 * nz1; t += HT_THREADS) {
    const int j = A.y1 + t % ny1, k = A.z1 + t / ny1;
    T[at(A.x1, j, k)] = T[at(A.x1 + 1, j, k)];
    T[at(A.x2 + 1, j, k)] = T[at(A.x2, j, k)];
  }
  __syncthreads();
  for (int t = tid; t < nx1 * nz1; t += HT_THREADS) {
    const int i = A.x1 + t % nx1, k = A.z1 + t / nx1;
    T[at(i, A.y1, k)] = T[at(i, A.y1 + 1, k)];
    T[at(i, A.y2 + 1, k)] = T[at(i, A.y2, k)];
  }
  __syncthreads();
  for (int t = tid; t < nx1 * ny1; t += HT_THREADS) {
    const int i = A.x1 + t % nx1, j = A.y1 + t / nx1;
    T[at(i, j, A.z1)] = T[at(i, j, A.z1 + 1)];
    T[at(i, j, A.z2 + 1)] = T[at(i, j, A.z2)];
  }
  __syncthreads();
  const double dt = A.dt, invdt2 = 1 / (dt * dt), den = 1 + dt * A.gam;
  const double cx = invdt2 / A.dx2, cy = invdt2 / A.dy2, cz = invdt2 / A.dz2;
  const int lo = A.x1 + A.margin, hi = A.x2 + 1 - A.margin;
  const int ny = A.y2 - A.y1, nz = A.z2 - A.z1;   // interior rows and columns
  const long long sx = 1, sy = d.n1, sz = (long long)d.n1 * d.n2;
  const double *R = A.uni ? T : A.R;
  if (!A.uni) {   // the field of the step before, faces included
    for (long long t = tid; t < d.n(); t += HT_THREADS) A.R[t] = T[t];
    __syncthreads();
  }
  auto hm = [](double a, double b) { return a == b ? a : 2 * a * b / (a + b); };
  // one D_T: the planes i + j + k = s in order (the in-place lexicographic sweep's bits); D_T per material: every node
  // from R at once (the planes are then only an order of work)
  for (int s = (A.x1 + 1) + (A.y1 + 1) + (A.z1 + 1); s <= A.x2 + A.y2 + A.z2; s++) {
    for (int t = tid; t < ny * nz; t += HT_THREADS) {
      const int j = A.y1 + 1 + t % ny, k = A.z1 + 1 + t / ny, i = s - j - k;
      if (i <= A.x1 || i > A.x2) continue;
      const long long o = at(i, j, k);
      const double q = R[o];
      const int m = A.mat ? A.mat[o] - 1 : 0;
      double flux;
      if (A.uni) {
        flux = A.DT * (((T[o + sx] - 2 * q) + T[o - sx]) / A.dx2 + ((T[o + sy] - 2 * q) + T[o - sy]) / A.dy2 +
                       ((T[o + sz] - 2 * q) + T[o - sz]) / A.dz2);
      } else {
        const double d0 = A.DTm[m];
        auto dn = [&](long long on) { return hm(d0, A.DTm[A.mat[on] - 1]); };
        flux = (dn(o + sx) * (R[o + sx] - q) + dn(o - sx) * (R[o - sx] - q)) / A.dx2 +
               (dn(o + sy) * (R[o + sy] - q) + dn(o - sy) * (R[o - sy] - q)) / A.dy2 +
               (dn(o + sz) * (R[o + sz] - q) + dn(o - sz) * (R[o - sz] - q)) / A.dz2;
      }
      const bool in = lo < i && i < hi;
      double src = 0.0;
      if (in) {
        if (A.mat) {
          for (int mu = 0; mu < A.N; mu++) src += band_heat(A.Gm[m][mu], A.gkm[m][mu], A.G.p[mu][o], A.F.p[mu][o], invdt2);
        } else {
          src = band_heat(A.Gam[0], A.gk[0], A.G.p[0][o], A.F.p[0][o], invdt2);
          for (int mu = 1; mu < A.N; mu++) src += band_heat(A.Gam[mu], A.gk[mu], A.G.p[mu][o], A.F.p[mu][o], invdt2);
        }
      }
      const double sig = A.mat ? A.sigm[m] : A.sig;
      double acc;
      if (A.joule) {
        double e2 = 0.0, qj = 0.0;
        if (in && A.f[o] > 0) {
          if (A.qp) qj = qp_joule(A, o, sx, sy, sz);   // terms.jl:107-108
          const double a0 = A.th[0][o - sx] - A.ph[0][o - sx], a1 = A.th[0][o] - A.ph[0][o];
          const double b0 = A.th[1][o - sy] - A.ph[1][o - sy], b1 = A.th[1][o] - A.ph[1][o];
          const double c0 = A.th[2][o - sz] - A.ph[2][o - sz], c1 = A.th[2][o] - A.ph[2][o];
          const double ex = 0.5 * (a0 * a0 + a1 * a1) * cx, ey = 0.5 * (b0 * b0 + b1 * b1) * cy,
                       ez = 0.5 * (c0 * c0 + c1 * c1) * cz;
          e2 = (ex + ey) + ez;
        }
        acc = q + dt * (flux + A.eta * ((src + sig * e2) + qj));
      } else {
        acc = q + dt * (flux + A.eta * src);
      }
      double tn = (acc + dt * A.gam * A.thb) / den;
      if (tn < 0) tn = 0.0;
      else if (tn > A.cap) tn = A.cap;
      T[o] = tn;
    }
    __syncthreads();
  }
}

__global__ void k_fill(double *a, double v, long long n) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    a[t] = v;
}

}  // namespace

int heat_create(Ctx *ctx, const tdgl_materials *M) {
  const long long nn = ctx->g.d.n();
  int rc;
  if ((rc = dalloc(ctx, &ctx->Th, (size_t)nn))) return rc;
  if (M) {   // each material's values; D_T per material: a second field for the Jacobi update
    HeatMat &h = ctx->hm;
    h.nmat = M->nmat;
    bool uni = true;
    for (int m = 0; m < M->nmat; m++) {
      for (int mu = 0; mu < ctx->N; mu++) {
        h.G[m][mu] = M->gamma[m][mu];
        h.gk[m][mu] = M->gk[m][mu];
      }
      h.sig[m] = M->sigma_n[m];
      h.DT[m] = M->heat_DT[m];
      uni = uni && M->heat_DT[m] == ctx->P.heat_DT;
    }
    if (!uni && (rc = dalloc(ctx, &ctx->Th2, (size_t)nn))) return rc;
  }
  TDGL_LAUNCH(ctx, K_HEAT, 8.0 * nn, k_fill, nblk(nn, 256), 256, 0, ctx->Th, ctx->P.heat_T, nn);
  return 0;
}

// heat_step! (terms.jl:58-130): after the bands, before the field increment (it reads θ − φ, the change of the link
// phases over the last step, which the fused supercurrent and field increment overwrites)
void heat_step(Ctx *ctx) {
  const tdgl_params &P = ctx->P;
  const Geo &g = ctx->g;
  HeatArgs A;
  A.T = ctx->Th;
  for (int mu = 0; mu < ctx->N; mu++) {
    A.G.p[mu] = ctx->G[mu];
    A.F.p[mu] = ctx->F[mu];
    A.Gam[mu] = P.heat_Gamma[mu];
    A.gk[mu] = P.heat_gk[mu];
  }
  for (int ax = 0; ax < 3; ax++) {
    A.th[ax] = ctx->th[ax];
    A.ph[ax] = ctx->ph[ax];
  }
  A.f = ctx->f;
  A.N = ctx->N;
  A.x1 = g.x1; A.x2 = g.x2; A.y1 = g.y1; A.y2 = g.y2; A.z1 = g.z1; A.z2 = g.z2;
  A.d = g.d;
  A.dt = P.dt;
  A.dx2 = g.dx * g.dx; A.dy2 = g.dy * g.dy; A.dz2 = g.dz * g.dz;
  A.DT = P.heat_DT; A.gam = P.heat_gamma_bath; A.eta = P.heat_eta; A.thb = P.heat_T; A.cap = P.heat_cap;
  A.sig = P.heat_sigma_n;
  A.joule = P.heat_joule;
  A.margin = P.heat_margin;
  A.mat = ctx->mat;
  A.uni = ctx->Th2 == nullptr;
  A.R = ctx->Th2;
  A.qp = P.qp_on;
  qp_potentials(ctx, A.qmu);
  A.qsig = P.qp_sigma_n;
  for (int mu = 0; mu < TDGL_MAXB; mu++) {
    A.qs[mu] = P.qp_s[mu];
    for (int nu = 0; nu < TDGL_MAXB; nu++) A.qGm[mu][nu] = P.qp_Gm[mu][nu];
  }
  for (int m = 0; m < ctx->hm.nmat; m++) {
    for (int mu = 0; mu < ctx->N; mu++) {
      A.Gm[m][mu] = ctx->hm.G[m][mu];
      A.gkm[m][mu] = ctx->hm.gk[m][mu];
    }
    A.sigm[m] = ctx->hm.sig[m];
    A.DTm[m] = ctx->hm.DT[m];
  }
  const double n = (double)(g.x2 - g.x1) * (g.y2 - g.y1) * (g.z2 - g.z1);
  TDGL_LAUNCH(ctx, K_HEAT, n * (8.0 * 8 + 32.0 * ctx->N), k_heat, 1, HT_THREADS, 0, A);
}

int heat_carry(Ctx *ctx, double *host, bool up) {
  const size_t bytes = ctx->g.d.n() * sizeof(double);
  cudaError_t e = up ? cudaMemcpyAsync(ctx->Th, host, bytes, cudaMemcpyHostToDevice, ctx->stream)
                     : cudaMemcpyAsync(host, ctx->Th, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return set_err(ctx, TDGL_ECUDA, "heat carry copy", e);
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return set_err(ctx, TDGL_ECUDA, "heat carry", e);
  return 0;
}

}  // namespace tdgl
