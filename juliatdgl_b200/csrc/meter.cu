// meter.cu — the observables of one protocol cycle, on the resident state (gtdgl/src/protocol.jl:148-189 and
// :409-453; gtdgl/src/observables.jl:48-114).
//
// After every cycle of lMax steps the ladder (protocol.jl:325-470) reads: the voltage from two plane sums of φ_x
// over the live links of the voltmeter planes (_plane_sum :148-155), θ_A (_theta_A :157-166), the path phase of
// every band along each voltmeter line (_path_phase! :168-179, then unwrapped on the host, _unwrap! :181-189), the
// per-band residual max| |Ψ| − |Ψ|prev | with max|Ψ| for the divergence guard (:432-446), max|h_z − h_z prev|
// (:447-451), and the midplane current (observables.jl:102-114); count_vortices (observables.jl:48-74) at each
// rung's close.  Here they are computed on the device and only these numbers cross to the host, so a protocol
// cycle needs no copy of the state.
//
// Maxima are exact whatever the order: they run on the bit patterns of non-negative doubles (a NaN, made positive
// by fabs, orders above +Inf, so it survives the maximum as Julia's max keeps it).  Sums use fixed-order block
// reductions (deterministic; they round differently from the reference's sequential sums).
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace tdgl {

struct MeterDev {
  int vi = 0, vo = 0, nphase = 0, nl1 = 0, nl2 = 0, imid = 0;
  unsigned char *Min = nullptr, *Mou = nullptr, *line_ok = nullptr;   // nl1 × nl2 lines (y fastest)
  double *cooper0[TDGL_MAXB] = {};   // |F_µ| on the block at the previous measurement (node-shaped)
  double *hz0 = nullptr;             // h_z at the previous measurement (node-shaped)
  double *D = nullptr;               // path phases, nphase × nl1 × nl2
  double *tline = nullptr;           // per line Σ_{vi ≤ i < vo} φ_x
  double *sums = nullptr;            // [0] vin, [1] vout, [2] ta, [3] Itot, [4] Isam, [5] Phi_enc
  unsigned long long *mx = nullptr;  // maxima as bit patterns: [µ] residual, [MAXB] amax, [MAXB + 1] diffh
  int *vort = nullptr;               // [0] Nv, [1] Nv_loop, [2] loop_ok; then nmap
  double *loop = nullptr;            // perimeter circulation (one value)
};

namespace {
const int BS = 256;
enum { S_VIN = 0, S_VOUT, S_TA, S_ITOT, S_ISAM, S_PHI, S_N };

__device__ __forceinline__ unsigned long long nbits(double v) { return (unsigned long long)__double_as_longlong(fabs(v)); }

__device__ __forceinline__ unsigned long long warp_max(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_down_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

__device__ __forceinline__ double bsum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  v = 0.0;
  if (w == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// _path_phase! (protocol.jl:168-179): D[µ][jj + nl1 kk] = Σ_{vi ≤ i < vo} angle((conj(G_µ[i]) V_x[i]) G_µ[i+1]) along
// the line (y1 + jj, z1 + kk), summed in the reference's order; and (first band's threads) the θ_A line sums.
__global__ void k_path_phase(BandPtrs Gs, const cd *Vx, const double *phx, Dim d, int y1, int z1, int nl1, int nl,
                             int vi, int vo, int nphase, double *D, double *tline) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (nphase > 0 ? nphase : 1) * nl) return;
  const int mu = t / nl, l = t - mu * nl, j = y1 + l % nl1, k = z1 + l / nl1;
  if (nphase > 0) {
    const cd *G = Gs.p[mu];
    double acc = 0.0;
    for (int i = vi; i < vo; i++) {
      const long long o = d.at(i, j, k);
      const cd w = cmul(cmul(cconj(G[o]), Vx[o]), G[o + 1]);
      acc += atan2(w.y, w.x);
    }
    D[t] = acc;
  }
  if (mu == 0) {
    double s = 0.0;
    for (int i = vi; i < vo; i++) s += phx[d.at(i, j, k)];
    tline[l] = s;
  }
}

// the sums of one cycle, one block: plane sums of φ_x (voltage), θ_A, the midplane current (observables.jl:102-114)
struct FoldArgs {
  const unsigned char *Min, *Mou, *line_ok;
  const double *phx, *tline, *hy, *hz;
  Dim d;
  int y1, y2, z1, z2, nl1, nl, vi, vo, imid, Ny, Nz;
  double ks2, dy, dz;
  double *sums;
};
__global__ void k_meter_fold(FoldArgs A) {
  __shared__ double sh[32];
  double vin = 0.0, vout = 0.0, ta = 0.0;
  for (int l = threadIdx.x; l < A.nl; l += blockDim.x) {
    const int j = A.y1 + l % A.nl1, k = A.z1 + l / A.nl1;
    if (A.Min[l]) vin += A.phx[A.d.at(A.vi, j, k)];
    if (A.Mou[l]) vout += A.phx[A.d.at(A.vo, j, k)];
    if (A.line_ok[l]) ta += A.tline[l];
  }
  double itot = 0.0, isam = 0.0;
  const int nj = A.Ny - 1, nm = nj * (A.Nz - 1);
  for (int q = threadIdx.x; q < nm; q += blockDim.x) {
    const int jj = 2 + q % nj, kk = 2 + q / nj, ii = A.imid;
    const double jx = A.ks2 * ((A.hz[A.d.at(ii, jj, kk)] - A.hz[A.d.at(ii, jj - 1, kk)]) / A.dy -
                               (A.hy[A.d.at(ii, jj, kk)] - A.hy[A.d.at(ii, jj, kk - 1)]) / A.dz);
    itot += jx;
    if (A.y1 <= jj && jj <= A.y2 + 1 && A.z1 <= kk && kk <= A.z2 + 1) isam += jx;
  }
  vin = bsum(vin, sh);
  vout = bsum(vout, sh);
  ta = bsum(ta, sh);
  itot = bsum(itot, sh);
  isam = bsum(isam, sh);
  if (threadIdx.x == 0) {
    A.sums[S_VIN] = vin;
    A.sums[S_VOUT] = vout;
    A.sums[S_TA] = ta;
    A.sums[S_ITOT] = itot * A.dy * A.dz;
    A.sums[S_ISAM] = isam * A.dy * A.dz;
  }
}

// max over the block of | |F_µ| − c0_µ | and of |F_µ|, then c0_µ ← |F_µ| (protocol.jl:432-440); init: c0_µ ← |G_µ|
struct DPtrs {
  double *p[TDGL_MAXB];
};
__global__ void k_cooper(BandPtrs Fs, DPtrs c0, int N, Rng r, Dim d, unsigned long long *mx, int init) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long res[TDGL_MAXB], am = 0ull;
  for (int mu = 0; mu < N; mu++) res[mu] = 0ull;
  if (t < r.n()) {
    int i, j, k;
    rng_ijk(r, t, i, j, k);
    const long long o = d.at(i, j, k);
    for (int mu = 0; mu < N; mu++) {
      const cd v = Fs.p[mu][o];
      const double a = hypot(v.x, v.y);
      if (!init) {
        res[mu] = nbits(a - c0.p[mu][o]);
        const unsigned long long b = nbits(a);
        am = b > am ? b : am;
      }
      c0.p[mu][o] = a;
    }
  }
  if (init) return;
  for (int mu = 0; mu < N; mu++) {
    const unsigned long long w = warp_max(res[mu]);
    if ((threadIdx.x & 31) == 0 && w) atomicMax(mx + mu, w);
  }
  am = warp_max(am);
  if ((threadIdx.x & 31) == 0 && am) atomicMax(mx + TDGL_MAXB, am);
}

// max |h_z − h_z prev| over every h_z entry (protocol.jl:447-451), then the baseline moves
__global__ void k_diffh(const double *hz, double *hz0, Rng r, Dim d, unsigned long long *mx, int init) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long m = 0ull;
  if (t < r.n()) {
    int i, j, k;
    rng_ijk(r, t, i, j, k);
    const long long o = d.at(i, j, k);
    if (!init) m = nbits(hz[o] - hz0[o]);
    hz0[o] = hz[o];
  }
  if (init) return;
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(mx + TDGL_MAXB + 1, m);
}

// count_vortices (observables.jl:48-74) on the plane kc: one thread per plaquette of the block section
struct VortArgs {
  const cd *P, *Ux, *Uy;
  const double *hz, *f;
  Dim d;
  int x1, y1, nx, ny, kc;   // nx × ny nodes of the section
  double dxdy;
  int *vort;                // [0] Nv, [3 ...] nmap
};
__device__ __forceinline__ double vdx(const VortArgs &A, int i, int j) {   // Dx[i, j], 1-based local
  const long long o = A.d.at(A.x1 - 1 + i, A.y1 - 1 + j, A.kc);
  const cd w = cmul(cmul(cconj(A.P[o]), A.Ux[o]), A.P[o + 1]);
  return atan2(w.y, w.x);
}
__device__ __forceinline__ double vdy(const VortArgs &A, int i, int j) {   // Dy[i, j]
  const long long o = A.d.at(A.x1 - 1 + i, A.y1 - 1 + j, A.kc);
  const cd w = cmul(cmul(cconj(A.P[o]), A.Uy[o]), A.P[o + A.d.n1]);
  return atan2(w.y, w.x);
}
__device__ __forceinline__ bool vmat(const VortArgs &A, int i, int j) {
  const long long o = A.d.at(A.x1 - 1 + i, A.y1 - 1 + j, A.kc);
  return A.f[o] > 1e-6 && hypot(A.P[o].x, A.P[o].y) > 1e-12;
}
__device__ __forceinline__ int vround(double w) {   // round(Int, w, RoundNearestTiesAway)
  const double a = floor(fabs(w) + 0.5);
  return (int)(w >= 0 ? a : -a);
}
__global__ void k_vort_map(VortArgs A) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x, nq = (A.nx - 1) * (A.ny - 1);
  if (t >= nq) return;
  const int i = 1 + t % (A.nx - 1), j = 1 + t / (A.nx - 1);
  const double circ = vdx(A, i, j) + vdy(A, i + 1, j) - vdx(A, i, j + 1) - vdy(A, i, j);
  const double phi = A.hz[A.d.at(A.x1 - 1 + i, A.y1 - 1 + j, A.kc)] * A.dxdy;
  const bool good = vmat(A, i, j) && vmat(A, i + 1, j) && vmat(A, i, j + 1) && vmat(A, i + 1, j + 1);
  const double w = (circ + phi) / (2 * M_PI);
  const int n = good && isfinite(w) ? vround(w) : 0;
  A.vort[3 + t] = n;
  if (n) atomicAdd(A.vort, n);
}
// the perimeter circulation (sequential sums as sumlin) and whether the perimeter runs through material
__global__ void k_vort_loop(VortArgs A, double *loop) {
  if (threadIdx.x != 0) return;
  double a = 0.0, b = 0.0, c = 0.0, e = 0.0;
  for (int i = 1; i <= A.nx - 1; i++) a += vdx(A, i, 1);
  for (int j = 1; j <= A.ny - 1; j++) b += vdy(A, A.nx, j);
  for (int i = 1; i <= A.nx - 1; i++) c += vdx(A, i, A.ny);
  for (int j = 1; j <= A.ny - 1; j++) e += vdy(A, 1, j);
  loop[0] = a + b - c - e;
  bool ok = true;
  for (int i = 1; i <= A.nx && ok; i++) ok = vmat(A, i, 1) && vmat(A, i, A.ny);
  for (int j = 1; j <= A.ny && ok; j++) ok = vmat(A, 1, j) && vmat(A, A.nx, j);
  A.vort[2] = ok ? 1 : 0;
}
// Φ_enc = Σ h_z over x1..x2, y1..y2 on kc (one block, fixed order)
__global__ void k_vort_flux(const double *hz, Dim d, int x1, int y1, int mx, int my, int kc, double *sums) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int q = threadIdx.x; q < mx * my; q += blockDim.x) s += hz[d.at(x1 + q % mx, y1 + q / mx, kc)];
  s = bsum(s, sh);
  if (threadIdx.x == 0) sums[S_PHI] = s;
}

Rng block_rng(const Geo &g) { return mkrng(g.x1, g.x2 + 1, g.y1, g.y2 + 1, g.z1, g.z2 + 1); }
Rng hz_rng(const Geo &g) { return mkrng(1, g.Nx, 1, g.Ny, 1, g.Nz + 1); }

int baselines(Ctx *ctx) {
  MeterDev *M = ctx->meter;
  const Geo &g = ctx->g;
  BandPtrs G;
  for (int mu = 0; mu < ctx->N; mu++) G.p[mu] = ctx->G[mu];
  const Rng rb = block_rng(g), rh = hz_rng(g);
  DPtrs c0;
  for (int mu = 0; mu < TDGL_MAXB; mu++) c0.p[mu] = M->cooper0[mu];
  TDGL_LAUNCH(ctx, K_METER, 24.0 * ctx->N * rb.n(), k_cooper, nblk(rb.n(), BS), BS, 0, G, c0, ctx->N, rb, g.d, M->mx, 1);
  TDGL_LAUNCH(ctx, K_METER, 16.0 * rh.n(), k_diffh, nblk(rh.n(), BS), BS, 0, ctx->h[2], M->hz0, rh, g.d, M->mx, 1);
  TDGL_CUDA(cudaGetLastError());
  return 0;
}

double from_bits(unsigned long long b) {
  double v = 0.0;
  if (b) std::memcpy(&v, &b, sizeof(v));
  return v;
}

}  // namespace

void meter_destroy(Ctx *ctx) {
  delete ctx->meter;
  ctx->meter = nullptr;
}

}  // namespace tdgl

using namespace tdgl;

extern "C" int tdgl_meter_set(tdgl_ctx *c, const tdgl_meter *m) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !m) return set_err(ctx, TDGL_EINVAL, "null argument");
  if (!ctx->have_state) return set_err(ctx, TDGL_ESTATE, "no state uploaded");
  const Geo &g = ctx->g;
  if (!(g.x1 <= m->vi && m->vi < m->vo && m->vo <= g.x2))
    return set_err(ctx, TDGL_EINVAL, "voltmeter planes: need x1 <= vi < vo <= x2");
  if (m->nphase < 0 || m->nphase > ctx->N) return set_err(ctx, TDGL_EINVAL, "nphase out of range");
  if (!m->Min || !m->Mou || !m->line_ok) return set_err(ctx, TDGL_EINVAL, "null voltmeter mask");
  if (!ctx->meter) {
    MeterDev *M = new MeterDev();
    ctx->meter = M;
    M->nl1 = g.y2 - g.y1 + 2;
    M->nl2 = g.z2 - g.z1 + 2;
    const long long nl = (long long)M->nl1 * M->nl2, nn = g.d.n();
    int rc;
    if ((rc = dalloc(ctx, &M->Min, nl)) || (rc = dalloc(ctx, &M->Mou, nl)) || (rc = dalloc(ctx, &M->line_ok, nl))) return rc;
    for (int mu = 0; mu < ctx->N; mu++)
      if ((rc = dalloc(ctx, &M->cooper0[mu], nn))) return rc;
    if ((rc = dalloc(ctx, &M->hz0, nn)) || (rc = dalloc(ctx, &M->D, (size_t)ctx->N * nl)) || (rc = dalloc(ctx, &M->tline, nl)) ||
        (rc = dalloc(ctx, &M->sums, S_N)) || (rc = dalloc(ctx, &M->mx, TDGL_MAXB + 2)) || (rc = dalloc(ctx, &M->loop, 1)))
      return rc;
    const long long nq = (long long)(g.x2 - g.x1 + 1) * (g.y2 - g.y1 + 1);
    if ((rc = dalloc(ctx, &M->vort, 3 + nq))) return rc;
  }
  MeterDev *M = ctx->meter;
  M->vi = m->vi;
  M->vo = m->vo;
  M->nphase = m->nphase;
  M->imid = (int)std::floor(std::fabs(g.Nx / 2.0) + 0.5);   // oround(Nx/2) (observables.jl:106)
  const size_t nl = (size_t)M->nl1 * M->nl2;
  TDGL_CUDA(cudaMemcpyAsync(M->Min, m->Min, nl, cudaMemcpyHostToDevice, ctx->stream));
  TDGL_CUDA(cudaMemcpyAsync(M->Mou, m->Mou, nl, cudaMemcpyHostToDevice, ctx->stream));
  TDGL_CUDA(cudaMemcpyAsync(M->line_ok, m->line_ok, nl, cudaMemcpyHostToDevice, ctx->stream));
  int rc;
  if ((rc = baselines(ctx))) return rc;
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

extern "C" int tdgl_measure(tdgl_ctx *c, tdgl_obs *out) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !out) return set_err(ctx, TDGL_EINVAL, "null argument");
  if (!ctx->meter) return set_err(ctx, TDGL_ESTATE, "tdgl_meter_set first");
  MeterDev *M = ctx->meter;
  const Geo &g = ctx->g;
  const int nl = M->nl1 * M->nl2, np = M->nphase;
  BandPtrs G, F;
  for (int mu = 0; mu < ctx->N; mu++) {
    G.p[mu] = ctx->G[mu];
    F.p[mu] = ctx->F[mu];
  }
  const long long nth = (long long)(np > 0 ? np : 1) * nl;
  TDGL_LAUNCH(ctx, K_METER, (32.0 * np + 8.0) * nl * (M->vo - M->vi), k_path_phase, nblk(nth, BS), BS, 0, G, ctx->V[0],
              ctx->ph[0], g.d, g.y1, g.z1, M->nl1, nl, M->vi, M->vo, np, M->D, M->tline);
  FoldArgs A;
  A.Min = M->Min; A.Mou = M->Mou; A.line_ok = M->line_ok;
  A.phx = ctx->ph[0]; A.tline = M->tline; A.hy = ctx->h[1]; A.hz = ctx->h[2];
  A.d = g.d;
  A.y1 = g.y1; A.y2 = g.y2; A.z1 = g.z1; A.z2 = g.z2; A.nl1 = M->nl1; A.nl = nl; A.vi = M->vi; A.vo = M->vo;
  A.imid = M->imid; A.Ny = g.Ny; A.Nz = g.Nz;
  A.ks2 = ctx->P.kappa2; A.dy = g.dy; A.dz = g.dz;
  A.sums = M->sums;
  TDGL_LAUNCH(ctx, K_METER, 24.0 * nl, k_meter_fold, 1, 1024, 0, A);
  TDGL_CUDA(cudaMemsetAsync(M->mx, 0, (TDGL_MAXB + 2) * sizeof(unsigned long long), ctx->stream));
  const Rng rb = block_rng(g), rh = hz_rng(g);
  DPtrs c0;
  for (int mu = 0; mu < TDGL_MAXB; mu++) c0.p[mu] = M->cooper0[mu];
  TDGL_LAUNCH(ctx, K_METER, 24.0 * ctx->N * rb.n(), k_cooper, nblk(rb.n(), BS), BS, 0, F, c0, ctx->N, rb, g.d, M->mx, 0);
  TDGL_LAUNCH(ctx, K_METER, 16.0 * rh.n(), k_diffh, nblk(rh.n(), BS), BS, 0, ctx->h[2], M->hz0, rh, g.d, M->mx, 0);
  double sums[S_N];
  unsigned long long mx[TDGL_MAXB + 2];
  TDGL_CUDA(cudaMemcpyAsync(sums, M->sums, sizeof(sums), cudaMemcpyDeviceToHost, ctx->stream));
  TDGL_CUDA(cudaMemcpyAsync(mx, M->mx, sizeof(mx), cudaMemcpyDeviceToHost, ctx->stream));
  for (int mu = 0; mu < np; mu++)
    if (out->D[mu])
      TDGL_CUDA(cudaMemcpyAsync(out->D[mu], M->D + (size_t)mu * nl, nl * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  out->vsum_in = sums[S_VIN];
  out->vsum_out = sums[S_VOUT];
  out->ta_sum = sums[S_TA];
  out->Itot = sums[S_ITOT];
  out->Isam = sums[S_ISAM];
  for (int mu = 0; mu < TDGL_MAXB; mu++) out->res[mu] = mu < ctx->N ? from_bits(mx[mu]) : 0.0;
  out->amax = from_bits(mx[TDGL_MAXB]);
  out->diffh = from_bits(mx[TDGL_MAXB + 1]);
  return 0;
}

extern "C" int tdgl_vortices(tdgl_ctx *c, int32_t band, int32_t kc, int32_t *Nv, int32_t *Nv_loop, int32_t *loop_ok,
                             int32_t *nmap) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !Nv || !Nv_loop || !loop_ok) return set_err(ctx, TDGL_EINVAL, "null argument");
  if (!ctx->meter) return set_err(ctx, TDGL_ESTATE, "tdgl_meter_set first");
  const Geo &g = ctx->g;
  if (band < 0 || band >= ctx->N) return set_err(ctx, TDGL_EINVAL, "band out of range");
  if (kc < 1 || kc > g.Nz + 1) return set_err(ctx, TDGL_EINVAL, "kc out of range");
  MeterDev *M = ctx->meter;
  VortArgs A;
  A.P = ctx->F[band]; A.Ux = ctx->V[0]; A.Uy = ctx->V[1]; A.hz = ctx->h[2]; A.f = ctx->f;
  A.d = g.d;
  A.x1 = g.x1; A.y1 = g.y1; A.nx = g.x2 - g.x1 + 2; A.ny = g.y2 - g.y1 + 2; A.kc = kc;
  A.dxdy = g.dx * g.dy;
  A.vort = M->vort;
  const int nq = (A.nx - 1) * (A.ny - 1);
  TDGL_CUDA(cudaMemsetAsync(M->vort, 0, 3 * sizeof(int), ctx->stream));
  TDGL_LAUNCH(ctx, K_METER, 80.0 * nq, k_vort_map, nblk(nq, BS), BS, 0, A);
  TDGL_LAUNCH(ctx, K_METER, 40.0 * (A.nx + A.ny), k_vort_loop, 1, 32, 0, A, M->loop);
  TDGL_LAUNCH(ctx, K_METER, 8.0 * nq, k_vort_flux, 1, 1024, 0, ctx->h[2], g.d, g.x1, g.y1, A.nx - 1, A.ny - 1, kc, M->sums);
  int v[3];
  double loop, phi;
  TDGL_CUDA(cudaMemcpyAsync(v, M->vort, sizeof(v), cudaMemcpyDeviceToHost, ctx->stream));
  TDGL_CUDA(cudaMemcpyAsync(&loop, M->loop, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TDGL_CUDA(cudaMemcpyAsync(&phi, M->sums + S_PHI, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (nmap) TDGL_CUDA(cudaMemcpyAsync(nmap, M->vort + 3, nq * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  *Nv = v[0];
  const double wl = (loop + phi * A.dxdy) / (2 * M_PI);
  *Nv_loop = std::isfinite(wl) ? (int)(wl >= 0 ? std::floor(wl + 0.5) : -std::floor(-wl + 0.5)) : 0;
  *loop_ok = v[2];
  return 0;
}
