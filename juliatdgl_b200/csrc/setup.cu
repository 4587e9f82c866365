// setup.cu — device helpers for the host's one-time set-up.
//
// tdgl_bar_field: the field of the bar current on the outer faces per unit HJ (gtdgl/src/field.jl:151-180): the
// 2D Biot–Savart field of a uniform current density over the bar section, with nq×nq midpoint quadrature per
// section cell, at every face point of the six tables.  One warp per face point, the quadrature points split over
// its lanes (the reference sums them in one loop; the order of the sum is the only difference).
#include <cmath>

#include "common.cuh"

namespace {

struct BarArgs {
  int Ny, Nz;
  double ya, za, hq, kq, dy, dz, c;
  int ny, nz;           // quadrature points along y and z
  long long off[7];     // prefix sums of the six table sizes
  double *out;          // the six tables, packed
};

__global__ void k_bar(BarArgs A) {
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= A.off[6]) return;
  int t = 0;
  while (w >= A.off[t + 1]) t++;
  const long long q = w - A.off[t];
  // table t: (rows, cols) and which component; point (j, k) of the reference's 1-based indices
  double y, z;
  int comp;  // 0: hy, 1: hz
  const int Ny = A.Ny, Nz = A.Nz;
  int j, k;
  switch (t) {
    case 0: j = (int)(q % (Ny + 1)) + 1; k = (q / (Ny + 1)) == 0 ? 1 : Nz; y = (j - 1) * A.dy; z = (k - 0.5) * A.dz; comp = 0; break;
    case 1: j = (q % 2) == 0 ? 1 : Ny + 1; k = (int)(q / 2) + 1; y = (j - 1) * A.dy; z = (k - 0.5) * A.dz; comp = 0; break;
    case 2: j = (int)(q % Ny) + 1; k = (q / Ny) == 0 ? 1 : Nz + 1; y = (j - 0.5) * A.dy; z = (k - 1) * A.dz; comp = 1; break;
    case 3: j = (q % 2) == 0 ? 1 : Ny; k = (int)(q / 2) + 1; y = (j - 0.5) * A.dy; z = (k - 1) * A.dz; comp = 1; break;
    case 4: j = (int)(q % Ny) + 1; k = (int)(q / Ny) + 1; y = (j - 0.5) * A.dy; z = (k - 1) * A.dz; comp = 1; break;
    default: j = (int)(q % (Ny + 1)) + 1; k = (int)(q / (Ny + 1)) + 1; y = (j - 1) * A.dy; z = (k - 0.5) * A.dz; comp = 0; break;
  }
  double s = 0.0;
  const long long nq = (long long)A.ny * A.nz;
  for (long long p = lane; p < nq; p += 32) {
    const int a = (int)(p % A.ny) + 1, b = (int)(p / A.ny) + 1;
    const double yp = A.ya + (a - 0.5) * A.hq, zp = A.za + (b - 0.5) * A.kq;
    const double r2 = (y - yp) * (y - yp) + (z - zp) * (z - zp);
    s += comp == 0 ? -(z - zp) / r2 : (y - yp) / r2;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) A.out[w] = A.c * s * A.hq * A.kq;
}

}  // namespace

extern "C" int tdgl_bar_field(const tdgl_grid *g, int32_t nq, double *hy_z, double *hy_y, double *hz_z, double *hz_y, double *hz_x,
                              double *hy_x) {
  if (!g || nq < 1) return TDGL_EINVAL;
  BarArgs A;
  A.Ny = g->Ny;
  A.Nz = g->Nz;
  A.dy = g->dy;
  A.dz = g->dz;
  A.ya = (g->y1 - 1) * g->dy;
  const double yb = g->y2 * g->dy;
  A.za = (g->z1 - 1) * g->dz;
  const double zb = g->z2 * g->dz;
  const double d = (g->z2 - g->z1 + 1) * g->dz;
  A.c = (-2 / d) / (2 * M_PI);
  A.ny = nq * (g->y2 - g->y1 + 1);
  A.nz = nq * (g->z2 - g->z1 + 1);
  A.hq = (yb - A.ya) / A.ny;
  A.kq = (zb - A.za) / A.nz;
  const long long sz[6] = {(long long)(g->Ny + 1) * 2, 2LL * g->Nz, (long long)g->Ny * 2, 2LL * (g->Nz + 1),
                           (long long)g->Ny * (g->Nz + 1), (long long)(g->Ny + 1) * g->Nz};
  A.off[0] = 0;
  for (int t = 0; t < 6; t++) A.off[t + 1] = A.off[t] + sz[t];
  double *dev = nullptr;
  if (cudaMalloc(&dev, A.off[6] * sizeof(double)) != cudaSuccess) return TDGL_ENOMEM;
  A.out = dev;
  const long long threads = A.off[6] * 32;
  k_bar<<<(unsigned)((threads + 255) / 256), 256>>>(A);
  cudaError_t e = cudaDeviceSynchronize();
  double *outs[6] = {hy_z, hy_y, hz_z, hz_y, hz_x, hy_x};
  for (int t = 0; t < 6 && e == cudaSuccess; t++) e = cudaMemcpy(outs[t], dev + A.off[t], sz[t] * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dev);
  return e == cudaSuccess ? 0 : TDGL_ECUDA;
}
