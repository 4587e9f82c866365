// openbc.cu — the open boundary of the field on the device (gtdgl/src/openbc.jl).
//
// Every `every` steps: δJ = κ² ∇_h × h − HJ·J_bar on the links of the box (_delta_current! :139-154), the Hockney
// convolution θ_δ = (dx³/κ²) G ∗ δJ with the lattice Green function (_convolve! :157-166), and h_δ = ∇_h × θ_δ on the
// faces (_face_field! :169-183); in between, the faces ramp linearly from the previous h_δ to the new one
// (open_update! :191-207, _open_add! :210-223).
//
// The reference pads each link lattice to exactly twice its size for FFTW's rfft.  Hockney's method needs any
// padded length M ≥ 2n − 1 along each axis (the circular convolution then never wraps onto the box), so this file
// pads to the smallest 2^a 3^b 5^c 7^d ≥ 2n − 1 and builds the transformed Green function at that size: the same
// convolution up to rounding.  The FFTs are hand-written: batched mixed-radix Stockham passes (radices 8, 4, 2, 3,
// 5, 7) over tiles of lines held in shared memory, FP64 complex, one pass per axis.
#include <cmath>

#include "common.cuh"

namespace tdgl {

struct OpenDev {
  int M[3][3];                 // padded sizes per component
  int sh[3][3];                // link-array shapes per component
  cd *ghat[3] = {};
  cd *buf = nullptr;           // one padded work array (largest component)
  double *theta[3] = {}, *old_[3] = {}, *new_[3] = {};   // node-shaped
  double *green = nullptr;     // (R+1)^3
  int count = -1;
};

namespace {
const int BS = 256;

int smooth_at_least(int n) {
  for (int m = n;; m++) {
    int r = m;
    for (int p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) return m;
  }
}

// radices of n, largest first among powers of two (8, 4, 2), then 3, 5, 7
int radices(int n, int *R) {
  int c = 0;
  while (n % 8 == 0) { R[c++] = 8; n /= 8; }
  while (n % 4 == 0) { R[c++] = 4; n /= 4; }
  while (n % 2 == 0) { R[c++] = 2; n /= 2; }
  for (int p : {3, 5, 7})
    while (n % p == 0) { R[c++] = p; n /= p; }
  return n == 1 ? c : -1;
}

struct FftArgs {
  cd *data;
  int N;                 // line length
  int axis;
  int d0, d1, d2;        // array dims
  int Lu;                // lines span [0, Lu) of the lower of the two other axes (and nlines / Lu of the higher)
  long long nlines;
  int TL;                // lines per block
  int nst;
  int R[32];
  double sign;           // -1 forward, +1 inverse
};

// offset of the first element of line L and the element stride; the lines of an axis pass are the (u, v) of the
// other two axes (u the lower one), u ∈ [0, Lu)
__device__ __forceinline__ long long line_base(const FftArgs &A, long long L, long long &stride) {
  const long long u = L % A.Lu, v = L / A.Lu;
  if (A.axis == 0) {
    stride = 1;
    return (long long)A.d0 * (u + (long long)A.d1 * v);
  }
  if (A.axis == 1) {
    stride = A.d0;
    return u + (long long)A.d0 * A.d1 * v;
  }
  stride = (long long)A.d0 * A.d1;
  return u + (long long)A.d0 * v;
}

// Twiddles come from a table of exp(±2πi t/N), t < N, built per block: the stage twiddle exp(±2πi jm r/(Ns R)) is
// entry jm r N/(Ns R) and the R-point kernel's exp(±2πi e/R) is entry e N/R.  The table entry is sincospi of 2t/N,
// the same rational as 2 jm r/(Ns R) (or 2e/R), so it is bit-identical to evaluating the twiddle directly.  Lines
// sit N + 1 elements apart in shared memory, so the TL lines of a strided pass land on different banks.
__global__ void k_fft_lines(FftArgs A) {
  extern __shared__ cd sm[];
  const int N = A.N, TL = A.TL, NS = A.N + 1;
  cd *tw = sm, *b0 = sm + N, *b1 = sm + N + (long long)TL * NS;
  const long long L0 = (long long)blockIdx.x * TL;
  const int nl = (int)min((long long)TL, A.nlines - L0);
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    double sn, cs;
    sincospi(A.sign * 2.0 * (double)t / (double)N, &sn, &cs);
    tw[t] = mkc(cs, sn);
  }
  // load (for axis > 0 the TL lines are adjacent in memory: the inner loop over lines is coalesced)
  for (int q = threadIdx.x; q < nl * N; q += blockDim.x) {
    int l, e;
    if (A.axis == 0) { e = q % N; l = q / N; }
    else { l = q % nl; e = q / nl; }
    long long st;
    long long base = line_base(A, L0 + l, st);
    b0[(long long)l * NS + e] = A.data[base + st * e];
  }
  __syncthreads();
  int Ns = 1;
  for (int s = 0; s < A.nst; s++) {
    const int R = A.R[s];
    const int nb = N / R, ts = N / (Ns * R), tr = N / R;
    for (int q = threadIdx.x; q < nl * nb; q += blockDim.x) {
      const int l = q / nb, j = q % nb;
      const cd *in = b0 + (long long)l * NS;
      cd *out = b1 + (long long)l * NS;
      cd v[8];
      const int jm = j % Ns;
      for (int r = 0; r < R; r++) {
        cd x = in[j + r * nb];
        if (r && jm) x = cmul(x, tw[jm * r * ts]);
        v[r] = x;
      }
      cd w[8];
      for (int k = 0; k < R; k++) {
        cd acc = v[0];
        for (int r = 1; r < R; r++) acc = cadd(acc, cmul(v[r], tw[((r * k) % R) * tr]));
        w[k] = acc;
      }
      const int idxD = (j / Ns) * Ns * R + jm;
      for (int k = 0; k < R; k++) out[idxD + k * Ns] = w[k];
    }
    __syncthreads();
    cd *t = b0; b0 = b1; b1 = t;
    Ns *= R;
  }
  for (int q = threadIdx.x; q < nl * N; q += blockDim.x) {
    int l, e;
    if (A.axis == 0) { e = q % N; l = q / N; }
    else { l = q % nl; e = q / nl; }
    long long st;
    long long base = line_base(A, L0 + l, st);
    A.data[base + st * e] = b0[(long long)l * NS + e];
  }
}

// 3-D FFT of the M[0] × M[1] × M[2] array, one launch per axis.  With a box (extents b ≤ M): forward, the input is
// zero outside [0, b) on every axis, so the axes run in order 0, 1, 2 over only the lines that are not yet known
// to be zero (b1·b2, then M0·b2, then M0·M1 lines); inverse, only [0, b) of the output is kept, so the axes run in
// order 2, 1, 0 over only the lines that feed it (M0·M1, M0·b2, b1·b2).  The skipped lines hold zeros (forward) or
// values nothing reads (inverse).  Without a box every pass covers every line.
int fft3(Ctx *ctx, cd *data, const int M[3], double sign, const int *box = nullptr) {
  const int b[3] = {box ? box[0] : M[0], box ? box[1] : M[1], box ? box[2] : M[2]};
  const bool fwd = sign < 0;
  for (int q = 0; q < 3; q++) {
    const int ax = fwd ? q : 2 - q;
    FftArgs A;
    A.data = data;
    A.N = M[ax];
    A.axis = ax;
    A.d0 = M[0]; A.d1 = M[1]; A.d2 = M[2];
    // extents of the two other axes: an axis already transformed in this call is full (forward) or only needed on
    // its box (inverse); an axis not yet transformed is nonzero only on its box (forward) or still full (inverse)
    int ext[3];
    for (int a = 0; a < 3; a++) {
      const bool done = fwd ? a < ax : a > ax;
      ext[a] = fwd ? (done ? M[a] : b[a]) : (done ? b[a] : M[a]);
    }
    const int u = ax == 0 ? 1 : 0, v = ax == 2 ? 1 : 2;
    A.Lu = ext[u];
    A.nlines = (long long)ext[u] * ext[v];
    A.nst = radices(A.N, A.R);
    if (A.nst < 0) return set_err(ctx, TDGL_EINVAL, "FFT length not smooth");
    int tl = (int)(96 * 1024 / (2 * 16 * (long long)(A.N + 1)));
    A.TL = tl < 1 ? 1 : (tl > 16 ? 16 : tl);
    A.sign = sign;
    size_t smem = ((size_t)2 * A.TL * (A.N + 1) + A.N) * sizeof(cd);
    unsigned grid = (unsigned)((A.nlines + A.TL - 1) / A.TL);
    TDGL_LAUNCH(ctx, K_OPEN_FFT, 32.0 * A.N * A.nlines, k_fft_lines, grid, BS, smem, A);
  }
  return 0;
}

__device__ double lgf(const double *G, int R, int i, int j, int k) {
  i = abs(i); j = abs(j); k = abs(k);
  if (max(i, max(j, k)) <= R) return G[i + (R + 1) * (j + (R + 1) * k)];
  double r2 = (double)(i * i + j * j + k * k), r = sqrt(r2);
  double i4 = (double)i * i * i * i, j4 = (double)j * j * j * j, k4 = (double)k * k * k * k;
  return (1 + (5 * (i4 + j4 + k4) / (r2 * r2) - 3) / (8 * r2)) / (4 * M_PI * r);
}

__global__ void k_green(cd *out, int M0, int M1, int M2, int n0, int n1, int n2, const double *G, int R, double fac) {
  long long n = (long long)M0 * M1 * M2;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int a = (int)(t % M0);
  long long r = t / M0;
  int b = (int)(r % M1), c = (int)(r / M1);
  int oa = a < n0 ? a : a - M0, ob = b < n1 ? b : b - M1, oc = c < n2 ? c : c - M2;
  out[t] = mkc(fac * lgf(G, R, oa, ob, oc), 0.0);
}

// δJ into the padded buffer of component c (zero elsewhere)
struct DJArgs {
  cd *buf;
  int M0, M1;
  const double *h[3];
  const double *jbar;
  double k2, HJ, dx, dy, dz;
  int comp, Nx, Ny, Nz;
  Rng r;
  Dim d;
};
__global__ void k_delta_current(DJArgs A) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.r.n()) return;
  int i, j, k;
  rng_ijk(A.r, t, i, j, k);
  const Dim d = A.d;
  const long long o = d.at(i, j, k), sx = 1, sy = d.n1, sz = (long long)d.n1 * d.n2;
  const double *hx = A.h[0], *hy = A.h[1], *hz = A.h[2];
  double v;
  if (A.comp == 0)
    v = A.k2 * ((hz[o] - hz[o - sy]) / A.dy - (hy[o] - hy[o - sz]) / A.dz) - A.HJ * A.jbar[(j - 1) + (long long)(A.Ny + 1) * (k - 1)];
  else if (A.comp == 1)
    v = A.k2 * ((hx[o] - hx[o - sz]) / A.dz - (hz[o] - hz[o - sx]) / A.dx);
  else
    v = A.k2 * ((hy[o] - hy[o - sx]) / A.dx - (hx[o] - hx[o - sy]) / A.dy);
  A.buf[(long long)(i - 1) + (long long)A.M0 * ((j - 1) + (long long)A.M1 * (k - 1))] = mkc(v, 0.0);
}

__global__ void k_mul(cd *a, const cd *b, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) a[t] = cmul(a[t], b[t]);
}

__global__ void k_extract(double *theta, const cd *buf, int M0, int M1, Rng r, Dim d, double inv) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= r.n()) return;
  int i, j, k;
  rng_ijk(r, t, i, j, k);
  theta[d.at(i, j, k)] = buf[(long long)(i - 1) + (long long)M0 * ((j - 1) + (long long)M1 * (k - 1))].x * inv;
}

// h_δ on the tangential plaquettes of the six faces (openbc.jl:169-183)
struct FFArgs {
  const double *th[3];
  double *out[3];
  int Nx, Ny, Nz;
  double dx, dy, dz;
  Rng r[3];
  Dim d;
};
__global__ void k_face_field(FFArgs A) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  if (t >= A.r[0].n()) {
    t -= A.r[0].n();
    c = 1;
    if (t >= A.r[1].n()) {
      t -= A.r[1].n();
      c = 2;
      if (t >= A.r[2].n()) return;
    }
  }
  int i, j, k;
  rng_ijk(A.r[c], t, i, j, k);
  const Dim d = A.d;
  const long long o = d.at(i, j, k), sx = 1, sy = d.n1, sz = (long long)d.n1 * d.n2;
  const double *fx = A.th[0], *fy = A.th[1], *fz = A.th[2];
  const int Nx = A.Nx, Ny = A.Ny, Nz = A.Nz;
  if (c == 2) {  // hz on j ∈ {1, Ny} or i ∈ {1, Nx}
    if (j == 1 || j == Ny || i == 1 || i == Nx) A.out[2][o] = ((fy[o + sx] - fy[o]) - fx[o + sy] + fx[o]) / (A.dx * A.dy);
  } else if (c == 0) {  // hx on j ∈ {1, Ny} or k ∈ {1, Nz}
    if (j == 1 || j == Ny || k == 1 || k == Nz) A.out[0][o] = ((fz[o + sy] - fz[o]) - fy[o + sz] + fy[o]) / (A.dy * A.dz);
  } else {  // hy on k ∈ {1, Nz} or i ∈ {1, Nx}
    if (k == 1 || k == Nz || i == 1 || i == Nx) A.out[1][o] = ((fx[o + sz] - fx[o]) - fz[o + sx] + fz[o]) / (A.dz * A.dx);
  }
}

}  // namespace

int open_create(Ctx *ctx) {
  const Geo &g = ctx->g;
  const tdgl_params &P = ctx->P;
  OpenDev *O = new OpenDev();
  ctx->open = O;
  TDGL_CUDA(cudaFuncSetAttribute(k_fft_lines, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  int sh[3][3] = {{g.Nx, g.Ny + 1, g.Nz + 1}, {g.Nx + 1, g.Ny, g.Nz + 1}, {g.Nx + 1, g.Ny + 1, g.Nz}};
  long long maxn = 0;
  for (int c = 0; c < 3; c++)
    for (int a = 0; a < 3; a++) {
      O->sh[c][a] = sh[c][a];
      O->M[c][a] = smooth_at_least(2 * sh[c][a] - 1);
    }
  for (int c = 0; c < 3; c++) maxn = std::max(maxn, (long long)O->M[c][0] * O->M[c][1] * O->M[c][2]);
  int rc;
  size_t gsz = (size_t)(P.open_R + 1) * (P.open_R + 1) * (P.open_R + 1);
  if ((rc = dalloc(ctx, &O->green, gsz))) return rc;
  TDGL_CUDA(cudaMemcpyAsync(O->green, P.open_green, gsz * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = dalloc(ctx, &O->buf, maxn))) return rc;
  for (int c = 0; c < 3; c++) {
    long long n = (long long)O->M[c][0] * O->M[c][1] * O->M[c][2];
    if ((rc = dalloc(ctx, &O->ghat[c], n))) return rc;
    if ((rc = dalloc(ctx, &O->theta[c], g.d.n()))) return rc;
    if ((rc = dalloc(ctx, &O->old_[c], g.d.n()))) return rc;
    if ((rc = dalloc(ctx, &O->new_[c], g.d.n()))) return rc;
  }
  // the transformed Green function per link lattice (openbc.jl:119-127, at the padded size chosen here)
  for (int c = 0; c < 3; c++) {
    long long n = (long long)O->M[c][0] * O->M[c][1] * O->M[c][2];
    TDGL_LAUNCH(ctx, K_OPEN_MISC, 16.0 * n, k_green, nblk(n, BS), BS, 0, O->ghat[c], O->M[c][0], O->M[c][1], O->M[c][2], sh[c][0],
                sh[c][1], sh[c][2], O->green, P.open_R, P.open_fac);
    if ((rc = fft3(ctx, O->ghat[c], O->M[c], -1.0))) return rc;
  }
  TDGL_CUDA(cudaGetLastError());
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

void open_destroy(Ctx *ctx) {
  delete ctx->open;
  ctx->open = nullptr;
}

static int open_recompute(Ctx *ctx, double HJ) {
  OpenDev *O = ctx->open;
  const Geo &g = ctx->g;
  const tdgl_params &P = ctx->P;
  for (int c = 0; c < 3; c++) {
    const int *M = O->M[c];
    long long n = (long long)M[0] * M[1] * M[2];
    TDGL_CUDA(cudaMemsetAsync(O->buf, 0, n * sizeof(cd), ctx->stream));
    DJArgs A;
    A.buf = O->buf;
    A.M0 = M[0]; A.M1 = M[1];
    for (int q = 0; q < 3; q++) A.h[q] = ctx->h[q];
    A.jbar = ctx->jbar;
    A.k2 = P.kappa2; A.HJ = HJ; A.dx = g.dx; A.dy = g.dy; A.dz = g.dz;
    A.comp = c; A.Nx = g.Nx; A.Ny = g.Ny; A.Nz = g.Nz;
    if (c == 0) A.r = mkrng(2, g.Nx - 1, 2, g.Ny, 2, g.Nz);
    else if (c == 1) A.r = mkrng(2, g.Nx, 2, g.Ny - 1, 2, g.Nz);
    else A.r = mkrng(2, g.Nx, 2, g.Ny, 2, g.Nz - 1);
    A.d = g.d;
    TDGL_LAUNCH(ctx, K_OPEN_MISC, 40.0 * A.r.n(), k_delta_current, nblk(A.r.n(), BS), BS, 0, A);
    int rc;
    if ((rc = fft3(ctx, O->buf, M, -1.0, O->sh[c]))) return rc;
    TDGL_LAUNCH(ctx, K_OPEN_MISC, 48.0 * n, k_mul, nblk(n, BS), BS, 0, O->buf, O->ghat[c], n);
    if ((rc = fft3(ctx, O->buf, M, +1.0, O->sh[c]))) return rc;
    Rng box = mkrng(1, O->sh[c][0], 1, O->sh[c][1], 1, O->sh[c][2]);
    TDGL_LAUNCH(ctx, K_OPEN_MISC, 24.0 * box.n(), k_extract, nblk(box.n(), BS), BS, 0, O->theta[c], O->buf, M[0], M[1], box, g.d,
                1.0 / (double)n);
  }
  FFArgs F;
  for (int c = 0; c < 3; c++) {
    F.th[c] = O->theta[c];
    F.out[c] = O->new_[c];
  }
  F.Nx = g.Nx; F.Ny = g.Ny; F.Nz = g.Nz;
  F.dx = g.dx; F.dy = g.dy; F.dz = g.dz;
  F.r[0] = mkrng(1, g.Nx + 1, 1, g.Ny, 1, g.Nz);
  F.r[1] = mkrng(1, g.Nx, 1, g.Ny + 1, 1, g.Nz);
  F.r[2] = mkrng(1, g.Nx, 1, g.Ny, 1, g.Nz + 1);
  F.d = g.d;
  long long nf = F.r[0].n() + F.r[1].n() + F.r[2].n();
  TDGL_LAUNCH(ctx, K_OPEN_MISC, 16.0 * nf, k_face_field, nblk(nf, BS), BS, 0, F);
  ctx->open_recomputes++;
  return 0;
}

// open_update! (openbc.jl:191-207)
int open_update(Ctx *ctx, double HJ) {
  OpenDev *O = ctx->open;
  const bool first = O->count < 0;
  O->count += 1;
  if (O->count >= ctx->P.open_every || first) {
    const size_t nb = ctx->g.d.n() * sizeof(double);
    for (int c = 0; c < 3; c++) TDGL_CUDA(cudaMemcpyAsync(O->old_[c], O->new_[c], nb, cudaMemcpyDeviceToDevice, ctx->stream));
    int rc = open_recompute(ctx, HJ);
    if (rc) return rc;
    if (first)
      for (int c = 0; c < 3; c++) TDGL_CUDA(cudaMemcpyAsync(O->old_[c], O->new_[c], nb, cudaMemcpyDeviceToDevice, ctx->stream));
    O->count = 0;
  }
  return 0;
}

void open_face_args(Ctx *ctx, const double **oo, const double **on) {
  OpenDev *O = ctx->open;
  for (int c = 0; c < 3; c++) {
    oo[c] = O->old_[c];
    on[c] = O->new_[c];
  }
}

void open_regions(Ctx *ctx, Regions &r) {
  OpenDev *O = ctx->open;
  const size_t nb = ctx->g.d.n() * sizeof(double);
  for (int c = 0; c < 3; c++) {
    r.push_back({O->theta[c], nb});
    r.push_back({O->old_[c], nb});
    r.push_back({O->new_[c], nb});
  }
}

int *open_count_ptr(Ctx *ctx) { return &ctx->open->count; }

double open_fraction(Ctx *ctx) {
  const double f = (ctx->open->count + 1) / (double)ctx->P.open_every;
  return f < 1.0 ? f : 1.0;
}

// host (reference-shaped) ↔ device (node-shaped) copies of the ramp, through the repack helpers of api.cu
int repack_up(Ctx *ctx, double *dst, const double *src, int a, int b, int c);
int repack_down(Ctx *ctx, double *dst, const double *src, int a, int b, int c);

int open_set_carry(Ctx *ctx, const tdgl_carry_view *v) {
  OpenDev *O = ctx->open;
  const Geo &g = ctx->g;
  int hs[3][3] = {{g.Nx + 1, g.Ny, g.Nz}, {g.Nx, g.Ny + 1, g.Nz}, {g.Nx, g.Ny, g.Nz + 1}};
  O->count = v->open_count;
  for (int c = 0; c < 3; c++) {
    int rc;
    if (v->open_old[c] && (rc = repack_up(ctx, O->old_[c], v->open_old[c], hs[c][0], hs[c][1], hs[c][2]))) return rc;
    if (v->open_new[c] && (rc = repack_up(ctx, O->new_[c], v->open_new[c], hs[c][0], hs[c][1], hs[c][2]))) return rc;
    if (v->open_theta[c] && (rc = repack_up(ctx, O->theta[c], v->open_theta[c], O->sh[c][0], O->sh[c][1], O->sh[c][2]))) return rc;
  }
  return 0;
}

int open_get_carry(Ctx *ctx, const tdgl_carry_view *v) {
  OpenDev *O = ctx->open;
  const Geo &g = ctx->g;
  int hs[3][3] = {{g.Nx + 1, g.Ny, g.Nz}, {g.Nx, g.Ny + 1, g.Nz}, {g.Nx, g.Ny, g.Nz + 1}};
  const_cast<tdgl_carry_view *>(v)->open_count = O->count;
  for (int c = 0; c < 3; c++) {
    int rc;
    if (v->open_old[c] && (rc = repack_down(ctx, v->open_old[c], O->old_[c], hs[c][0], hs[c][1], hs[c][2]))) return rc;
    if (v->open_new[c] && (rc = repack_down(ctx, v->open_new[c], O->new_[c], hs[c][0], hs[c][1], hs[c][2]))) return rc;
    if (v->open_theta[c] && (rc = repack_down(ctx, v->open_theta[c], O->theta[c], O->sh[c][0], O->sh[c][1], O->sh[c][2]))) return rc;
  }
  return 0;
}

}  // namespace tdgl
