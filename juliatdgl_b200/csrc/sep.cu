// sep.cu — the exact inverse of (I + aK) on the link ranges (gtdgl/src/implicit.jl:15-104, _precond32! :346-373).
//
// K is the Yee curl-curl.  Per axis it is diagonalised by the DCT-II basis on the nodes (V) and the DST-I basis
// on the edges between them (U = D V / s); these are exactly the singular vectors _sep_bases (implicit.jl:15-22)
// takes from the SVD of the forward difference D, up to column signs that cancel.  The reference transforms along
// x, y and z and divides per wavevector (P_L + P_T/(1 + a|k|²), implicit.jl:67-78).  Here only y and z are
// transformed (dense per line, as the reference's BLAS products); along x, (I + aK) for one (k_y, k_z) is a
// tridiagonal system that is solved directly (k_linesolve): the same inverse, with no x transform.
//
// Layout of the solver domain ("plane-major"): every vector of the field solve is a node-shaped array indexed
// j + (Ny+1)(k + (Nz+1) i) (0-based), so one x-plane is contiguous.  Mode-space ("hat") arrays are [p + P i] with
// p = my + ny·mz, P = ny·nz.  FP64 for the SepSolver, FP32 for the PCG preconditioner (pcg_f32).
#include <atomic>
#include <cmath>
#include <cstdio>

#include <algorithm>

#include "common.cuh"
#include "sep.cuh"
#include "merge.cuh"
#include "pcg.cuh"

namespace tdgl {

int g_sm_count = 0;   // SMs of the device (set by sep_create)

template <class T>
struct Basis {
  int n;
  T *V, *Vt, *U, *Ut, *s;   // V[i + n k] (node basis), Vt = V', U[e + (n-1)(k-1)] (edge basis), Ut = U'
  // the mirror-symmetric half blocks [E | O] of V (n points) and U (n − 1 points), forward ([point][mode]) and
  // inverse ([mode][point]), rows padded to a multiple of 8; FP32 only (null for FP64)
  T *HVf = nullptr, *HVi = nullptr, *HUf = nullptr, *HUi = nullptr;
  // the same half blocks as tensor-core operand images (tc_images; FP32 only)
  T *TVf = nullptr, *TVi = nullptr, *TUf = nullptr, *TUi = nullptr;
};

template <class T>
struct Work {
  T *Xh = nullptr, *Yh = nullptr, *Zh = nullptr;   // hat arrays
  double *inv = nullptr;   // the factorisation of the line solves (fixed for the run, FP64); c_i = −g·inv_i (i < n−1)
};

struct SepDev {
  int nx, ny, nz;
  long long P;               // ny·nz
  Basis<double> bd[3];
  Basis<float> bf[3];
  double *B[3] = {};         // plane-major right-hand side / solution (SepSolver)
  float *r32[3] = {};        // FP32 copy of the preconditioner's input (PCG with the FP32 preconditioner)
  bool tc = false;           // the FP32 preconditioner's plane transforms run on the tensor cores (sep_tc.cu)
  void *gtmp = nullptr;      // planes too large for one block: the first product of every plane (k_bgemm)
  float *hx = nullptr, *ho = nullptr;   // the mirror-halved FP32 transforms of large planes: X / O2 and O1 per plane
  long long hx_ps = 0, ho_ps = 0;       // their plane strides
  Work<double> wd;
  Work<float> wf;
};

namespace {
const int BS = 256;

// ---------------------------------------------------------------------------------------------- the plane transform
// out plane q: O2[jo][ko] = Σ_k (Σ_j M1t[jo + nj_out j] In[j][k]) M2t[ko + nk_out k]
// with In[j][k] = in[in_base + q in_ps + (in_j0 + j) + in_ld (in_k0 + k)] and
//      out[out_base + q out_ps + (out_j0 + jo) + out_ld (out_k0 + ko)] = O2[jo][ko].
// A block takes a chunk of jc output rows jo (jc ≤ PL_JC, a multiple of 4: the rows split evenly over the chunks)
// and up to `ppb` planes at a time (small planes: enough register tiles to keep its threads busy); every output sums
// over j, then k, in index order, whatever the chunking.
struct PlaneArgs {
  const void *in;
  long long in_base, in_ps;
  int in_ld, in_j0, in_k0, nj_in, nk_in;
  const void *M1t, *M2t;
  int nj_out, nk_out;
  void *out;
  long long out_base, out_ps;
  int out_ld, out_j0, out_k0;
  int nplanes;
  const int *done;           // skip when the PCG has converged (null: always run)
  int jc, ppb;               // k_plane: output rows per chunk, planes per pass at most
};

const int PL_JC = 48, PL_THREADS = 192, PL_PPB = 8;

__device__ __forceinline__ void ld4(float *v, const float *p) {
  const float4 t = *reinterpret_cast<const float4 *>(p);
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ld4(double *v, const double *p) {
  const double2 t0 = *reinterpret_cast<const double2 *>(p), t1 = *reinterpret_cast<const double2 *>(p + 2);
  v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y;
}
__device__ __forceinline__ void ld2(float *v, const float *p) {
  const float2 t = *reinterpret_cast<const float2 *>(p);
  v[0] = t.x; v[1] = t.y;
}
__device__ __forceinline__ void ld2(double *v, const double *p) {
  const double2 t = *reinterpret_cast<const double2 *>(p);
  v[0] = t.x; v[1] = t.y;
}
template <int TA, class T>
__device__ __forceinline__ void ldta(T *v, const T *p) {
  if constexpr (TA == 4) ld4(v, p);
  else ld2(v, p);
}
// one element, global to shared, asynchronously (all loads of a pass in flight at once)
__device__ __forceinline__ void cp_async_el(void *smem, const double *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(g)
               : "memory");
}
__device__ __forceinline__ void cp_async_el(void *smem, const float *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(g)
               : "memory");
}
__device__ __forceinline__ void cp_async_el_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__host__ __device__ inline int rup4(int n) { return (n + 3) & ~3; }

// shared memory of k_plane: the basis chunks M1 [nj_in][jc] and M2 [nk_in][KO], and per plane of a pass its input
// [nj_in][KP] and first product [KP][jc]
template <class T>
__host__ __device__ inline size_t plane_smem(int nj_in, int nk_in, int nk_out, int jc = PL_JC, int ppb = 1) {
  const int KP = rup4(nk_in), KO = rup4(nk_out);
  return sizeof(T) * ((size_t)nj_in * jc + (size_t)nk_in * KO + (size_t)ppb * ((size_t)nj_in * KP + (size_t)KP * jc));
}

// acc[a][b] += u[a] v[b] over a TA × 4 tile
template <int TA, class T>
struct Tile {
  T acc[TA][4];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int a = 0; a < TA; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] = T(0);
  }
  __device__ __forceinline__ void fma_step(const T *u, const T *v) {
#pragma unroll
    for (int a = 0; a < TA; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] = fma(u[a], v[b], acc[a][b]);
  }
};
// TA: output rows jo per register tile (tiles TA × 4).  Large planes take 4 (fewer shared loads per multiply-add);
// small ones 2, so that a pass has more tiles for the block's threads and fewer registers keep more blocks per SM.
template <class TIn, class TOut, class T, int TA>
__device__ __forceinline__ void plane_b(const Blk bk, PlaneArgs const &A);
template <class TIn, class TOut, class T, int TA>
__global__ void __launch_bounds__(PL_THREADS, TA == 2 ? 4 : 1) k_plane(PlaneArgs A) {
  plane_b<TIn, TOut, T, TA>(TDGL_BLK, A);
}
TDGL_MERGEABLE((k_plane<double, double, double, 2>), (plane_b<double, double, double, 2>), PL_THREADS, 4, true);
TDGL_MERGEABLE((k_plane<double, double, double, 4>), (plane_b<double, double, double, 4>), PL_THREADS, 1, true);
template <class TIn, class TOut, class T, int TA>
__device__ __forceinline__ void plane_b(const Blk bk, PlaneArgs const &A) {
  if (A.done && *A.done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  // planes per pass: up to A.ppb (what the shared memory holds), as many as the block's share of the planes allows
  // (a grid of one block per plane takes one plane at a time)
  // the row chunk: balanced (A.jc) for small planes; PL_JC for large ones, whose inner loops then step through
  // shared memory by a compile-time stride (immediate offsets, no address arithmetic in the issue-bound loop)
  const int KP = rup4(A.nk_in), KO = rup4(A.nk_out), JC = TA == 4 ? PL_JC : A.jc;
  const int PPB = min(A.ppb, (int)((A.nplanes + bk.nx - 1) / bk.nx));
  const int nj = A.nj_in, nk = A.nk_in;
  T *M1s = (T *)smraw;                     // [nj_in][JC]
  T *M2s = M1s + (size_t)nj * JC;          // [nk_in][KO]
  T *Ins = M2s + (size_t)nk * KO;          // PPB × [nj_in][KP]
  T *O1s = Ins + (size_t)PPB * nj * KP;    // PPB × [KP][JC]
  const int jo0 = bk.y * JC;
  const T *M1t = (const T *)A.M1t, *M2t = (const T *)A.M2t;
  const int tid = threadIdx.x;
  const int pin = nj * KP, po1 = KP * JC;   // per-plane strides of Ins and O1s
  // the block's basis chunks once, and the zero columns k >= nk_in of its input slots (never written again)
  for (int t = tid; t < nj * JC; t += PL_THREADS) {
    const int j = t / JC, jj = t % JC;
    M1s[t] = jo0 + jj < A.nj_out ? M1t[(jo0 + jj) + (long long)A.nj_out * j] : T(0);
  }
  for (int t = tid; t < nk * KO; t += PL_THREADS) {
    const int k = t / KO, ko = t % KO;
    M2s[t] = ko < A.nk_out ? M2t[ko + (long long)A.nk_out * k] : T(0);
  }
  const int kpad = KP - nk;
  for (int t = tid; t < PPB * nj * kpad; t += PL_THREADS) {
    const int pp = t / (nj * kpad), r = t % (nj * kpad);
    Ins[pp * pin + (r / kpad) * KP + nk + r % kpad] = T(0);
  }
  // then pass after pass of PPB planes (the grid may hold fewer blocks than passes)
  for (int g = bk.x; g * PPB < A.nplanes; g += bk.nx) {
    const int q0 = g * PPB, np = min(PPB, A.nplanes - q0);
    // rows k by warp, consecutive j by lane (coalesced, no index division)
    const int warp = tid >> 5, lane = tid & 31;
    for (int pk = warp; pk < np * nk; pk += PL_THREADS / 32) {
      const int pp = pk / nk, k = pk - pp * nk;
      const TIn *in = (const TIn *)A.in + A.in_base + (long long)(q0 + pp) * A.in_ps + A.in_j0 +
                      (long long)A.in_ld * (A.in_k0 + k);
      T *dst = Ins + pp * pin + k;
      for (int j = lane; j < nj; j += 32) {
        if constexpr (sizeof(TIn) == sizeof(T)) cp_async_el(dst + j * KP, (const T *)in + j);
        else dst[j * KP] = (T)in[j];
      }
    }
    if constexpr (sizeof(TIn) == sizeof(T)) cp_async_el_wait();
    __syncthreads();
    // first product: O1[k][jj] for jj < JC, k < KP (TA × 4 tiles), every plane of the pass
    const int t1 = (JC / TA) * (KP / 4);
    for (int tt = tid; tt < np * t1; tt += PL_THREADS) {
      const int pp = tt / t1, tile = tt % t1;
      const int jq = tile % (JC / TA), kq = tile / (JC / TA);
      Tile<TA, T> tl;
      tl.zero();
      const T *mp = M1s + jq * TA, *ip = Ins + pp * pin + kq * 4;
#pragma unroll 4
      for (int j = 0; j < nj; j++) {
        T mv[TA], iv[4];
        ldta<TA>(mv, mp + j * JC);
        ld4(iv, ip + j * KP);
        tl.fma_step(mv, iv);
      }
      T *o1 = O1s + pp * po1;
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int a = 0; a < TA; a++) o1[(kq * 4 + b) * JC + jq * TA + a] = tl.acc[a][b];
    }
    __syncthreads();
    // second product: O2[jj][ko] = Σ_k O1[k][jj] M2[k][ko]
    const int t2 = (JC / TA) * (KO / 4);
    for (int tt = tid; tt < np * t2; tt += PL_THREADS) {
      const int pp = tt / t2, tile = tt % t2;
      const int jq = tile % (JC / TA), kq = tile / (JC / TA);
      Tile<TA, T> tl;
      tl.zero();
      const T *op = O1s + pp * po1 + jq * TA, *mp = M2s + kq * 4;
#pragma unroll 4
      for (int k = 0; k < nk; k++) {
        T ov[TA], mv[4];
        ldta<TA>(ov, op + k * JC);
        ld4(mv, mp + k * KO);
        tl.fma_step(ov, mv);
      }
      const auto &acc = tl.acc;
      TOut *out = (TOut *)A.out + A.out_base + (long long)(q0 + pp) * A.out_ps;
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const int ko = kq * 4 + b;
        if (ko >= A.nk_out) continue;
#pragma unroll
        for (int a = 0; a < TA; a++) {
          const int jo = jo0 + jq * TA + a;
          if (jo < A.nj_out) out[(A.out_j0 + jo) + (long long)A.out_ld * (A.out_k0 + ko)] = (TOut)acc[a][b];
        }
      }
    }
    __syncthreads();   // the next pass overwrites Ins and O1s
  }
}

// The same plane transform for planes whose input does not fit one block's shared memory (k_plane keeps the whole
// input plane there): the sum over k runs in chunks of PT_K, and within a chunk the sum over j in chunks of PT_J, so
// the block holds only chunks of the input and the bases and its PL_JC × KO output rows.  First product
// O1[k][jj] = Σ_j M1[j][jo0+jj] In[j][k] (registers, 3 outputs a thread); second Acc[jj][ko] += Σ_k O1[k][jj] M2[k][ko]
// (shared memory, each thread the same outputs every chunk).  The same sums as k_plane, in chunks.
const int PT_J = 16, PT_K = 16, PT_THREADS = 256;

template <class T>
__host__ __device__ inline size_t tiled_smem(int nk_out) {
  const int KO = rup4(nk_out);
  return sizeof(T) * ((size_t)PT_J * PL_JC + (size_t)PT_J * PT_K + (size_t)PT_K * PL_JC + (size_t)PT_K * KO +
                      (size_t)PL_JC * KO);
}

template <class TIn, class TOut, class T>
__device__ __forceinline__ void plane_tiled_b(const Blk bk, PlaneArgs const &A);
template <class TIn, class TOut, class T>
__global__ void __launch_bounds__(PT_THREADS) k_plane_tiled(PlaneArgs A) {
  plane_tiled_b<TIn, TOut, T>(TDGL_BLK, A);
}
TDGL_MERGEABLE((k_plane_tiled<double, double, double>), (plane_tiled_b<double, double, double>), PT_THREADS, 1, false);
template <class TIn, class TOut, class T>
__device__ __forceinline__ void plane_tiled_b(const Blk bk, PlaneArgs const &A) {
  if (A.done && *A.done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int KO = rup4(A.nk_out);
  T *M1c = (T *)smraw;                       // [PT_J][PL_JC]
  T *Inc = M1c + PT_J * PL_JC;               // [PT_J][PT_K]
  T *O1c = Inc + PT_J * PT_K;                // [PT_K][PL_JC]
  T *M2c = O1c + PT_K * PL_JC;               // [PT_K][KO]
  T *Acc = M2c + (size_t)PT_K * KO;          // [PL_JC][KO]
  const int q = bk.x, jo0 = bk.y * PL_JC, tid = threadIdx.x;
  const TIn *in = (const TIn *)A.in + A.in_base + (long long)q * A.in_ps;
  const T *M1t = (const T *)A.M1t, *M2t = (const T *)A.M2t;
  for (int t = tid; t < PL_JC * KO; t += PT_THREADS) Acc[t] = T(0);
  // product-1 outputs of this thread: k = tid % PT_K, jj = 3 (tid / PT_K) + c (PT_THREADS = PT_K × PL_JC / 3)
  const int k1 = tid % PT_K, jj1 = 3 * (tid / PT_K);
  for (int k0 = 0; k0 < A.nk_in; k0 += PT_K) {
    T o1[3] = {T(0), T(0), T(0)};
    for (int j0 = 0; j0 < A.nj_in; j0 += PT_J) {
      __syncthreads();   // the previous chunk's readers are done (and, on the first pass, Acc is zero)
      for (int t = tid; t < PT_J * PL_JC; t += PT_THREADS) {
        const int j = t / PL_JC, jj = t % PL_JC;
        M1c[t] = (j0 + j < A.nj_in && jo0 + jj < A.nj_out) ? M1t[(jo0 + jj) + (long long)A.nj_out * (j0 + j)] : T(0);
      }
      for (int t = tid; t < PT_J * PT_K; t += PT_THREADS) {
        const int j = t / PT_K, k = t % PT_K;
        Inc[t] = (j0 + j < A.nj_in && k0 + k < A.nk_in)
                     ? (T)in[(A.in_j0 + j0 + j) + (long long)A.in_ld * (A.in_k0 + k0 + k)] : T(0);
      }
      __syncthreads();
#pragma unroll 4
      for (int j = 0; j < PT_J; j++) {
        const T x = Inc[j * PT_K + k1];
#pragma unroll
        for (int c = 0; c < 3; c++) o1[c] = fma(M1c[j * PL_JC + jj1 + c], x, o1[c]);
      }
    }
    __syncthreads();   // the previous chunk's second product has read O1c and M2c
#pragma unroll
    for (int c = 0; c < 3; c++) O1c[k1 * PL_JC + jj1 + c] = o1[c];
    for (int t = tid; t < PT_K * KO; t += PT_THREADS) {
      const int k = t / KO, ko = t % KO;
      M2c[t] = (k0 + k < A.nk_in && ko < A.nk_out) ? M2t[ko + (long long)A.nk_out * (k0 + k)] : T(0);
    }
    __syncthreads();
    for (int t = tid; t < PL_JC * KO; t += PT_THREADS) {
      const int jj = t / KO, ko = t % KO;
      T acc = Acc[t];
#pragma unroll 4
      for (int k = 0; k < PT_K; k++) acc = fma(O1c[k * PL_JC + jj], M2c[k * KO + ko], acc);
      Acc[t] = acc;
    }
  }
  __syncthreads();
  TOut *out = (TOut *)A.out + A.out_base + (long long)q * A.out_ps;
  for (int t = tid; t < PL_JC * KO; t += PT_THREADS) {
    const int jj = t / KO, ko = t % KO, jo = jo0 + jj;
    if (jo < A.nj_out && ko < A.nk_out) out[(A.out_j0 + jo) + (long long)A.out_ld * (A.out_k0 + ko)] = (TOut)Acc[t];
  }
}

// The FP32 plane transforms of the PCG preconditioner, halved by the mirror symmetry of the bases.  Both bases of
// an axis with n points (the DCT-II node basis V, the DST-I edge basis U) satisfy B[n−1−p][m] = (−1)^m B[p][m] for
// the 0-based mode index m.  So the forward transform pairs the points, S_p = x_p + x_{n−1−p} (the middle point
// alone when n is odd) for the even modes and D_p = x_p − x_{n−1−p} for the odd ones, and applies two square
// blocks E[p][m_e] = B[p][2m_e] (⌈n/2⌉ wide) and O[p][m_o] = B[p][2m_o+1] (⌊n/2⌋ wide); the inverse applies their
// transposes and unpairs, x_p = E_p + O_p, x_{n−1−p} = E_p − O_p.  Half the multiply-adds of the dense products,
// along y and along z (the same operator; the sums round differently).
//
// One persistent block per SM (8 warps, two independent halves of 4 warps) keeps the four half blocks of both
// axes in shared memory and takes the planes two at a time (one slot per half): the next pair, raw FP32, is staged by cp.async while the current pair is
// computed; the prologue forms the paired (or mode-gathered) plane X in class order (even class rows/columns
// first); the row product O1 = W1ᵀ X and the column product O2 = O1 W2 run in 8 × 8 register tiles (64 FMA per
// four 128-bit shared loads, which cost four wavefronts each; consecutive threads take consecutive column tiles); the epilogue scatters modes
// (forward) or unpairs (inverse) with coalesced row stores.  The forward input is the FP32 copy of the residual
// that the PCG update writes (the same rounding as converting here).
// Shared layout (floats): W1e [hS1][R0], W1o [hD1][R1], W2e [hS2][C0], W2o [hD2][C1], then per slot
// XO [max(n1, JP)][P32_KPAD] (X as [r][c], then O2 as [r][KS]), O1 [KP][JP], Stg [n2][n1]; hS = ⌈n/2⌉, hD = ⌊n/2⌋,
// R = C = 8⌈h/8⌉, JP = R0 + R1, KP = 8⌈n2/8⌉, KS = 4·odd ≥ C0 + C1 (conflict-free float4 rows).  The half
// blocks are stored in global memory already padded this way ([h][8⌈h/8⌉] each), so each block copies one
// contiguous image per axis with 16-byte cp.async.
const int HX_THREADS = 256, HX_HALF = HX_THREADS / 2, HX_HWARPS = HX_HALF / 32, P32_KPAD = 52;

__host__ __device__ inline int p32_ks(int KO) { return 4 * ((KO / 4) | 1); }
// column c of X sits at xsw(c) in its row: the 8-column groups of consecutive column tiles (32 bytes apart) would
// put tiles kt and kt + 4 on the same banks; columns ≥ 32 shift by 4 floats (rows have P32_KPAD = 52 ≥ 48 + 4)
__host__ __device__ inline int xsw(int c) { return c + ((c >> 5) << 2); }

struct HalfGeo {
  int hS1, hD1, hS2, hD2, R0, R1, C0, C1, JP, KP, KS, XR;
  __host__ __device__ HalfGeo(int n1, int n2) {
    hS1 = (n1 + 1) / 2; hD1 = n1 / 2; hS2 = (n2 + 1) / 2; hD2 = n2 / 2;
    R0 = rup8(hS1); R1 = rup8(hD1); C0 = rup8(hS2); C1 = rup8(hD2);
    JP = R0 + R1; KP = rup8(n2); KS = p32_ks(C0 + C1); XR = n1 > JP ? n1 : JP;
  }
  __host__ __device__ size_t wfloats() const {
    return (size_t)hS1 * R0 + (size_t)hD1 * R1 + (size_t)hS2 * C0 + (size_t)hD2 * C1;
  }
  __host__ __device__ size_t slot(int n1, int n2) const {   // one plane's XO, O1 and Stg, rounded to 16 bytes
    return ((size_t)XR * P32_KPAD + (size_t)KP * JP + (size_t)n1 * n2 + 3) & ~(size_t)3;
  }
};

size_t half_smem(int n1, int n2) {
  const HalfGeo G(n1, n2);
  return sizeof(float) * (G.wfloats() + 2 * G.slot(n1, n2));
}
bool half_fits(int n1, int n2) {
  const HalfGeo G(n1, n2);
  // 256 bytes of static shared memory (the folded dot products' block reduction) come on top of the dynamic
  return n1 >= 1 && n2 >= 1 && n2 <= 48 && G.C0 + G.C1 <= 48 && half_smem(n1, n2) + 256 <= 227 * 1024;
}

__device__ __forceinline__ void cp_async(void *smem, const float *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(g)
               : "memory");
}
__device__ __forceinline__ void cp_async(void *smem, const double *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(g)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const float *g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(g)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// FWD: points → modes (TOut = float); otherwise modes → points (TOut = double).  Inputs are FP32.  The three
// components go in one launch: planes are taken in pairs within a component, and a block's consecutive pairs may
// belong to different components (the block then loads the next component's half blocks); the shared layout is that
// of the largest geometry, so a plane of the next component can be staged while the current one is computed.
template <class TOut, bool FWD>
__global__ void __launch_bounds__(HX_THREADS, 1) k_half32(HalfMulti M) {
  if (M.done && *M.done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  int n1m = 1, n2m = 1, npairs = 0;
  for (int c = 0; c < M.ncomp; c++) {
    n1m = max(n1m, M.c[c].n1);
    n2m = max(n2m, M.c[c].n2);
    npairs += (M.c[c].nplanes + 1) / 2;
  }
  const HalfGeo Gm(n1m, n2m);
  const int tid = threadIdx.x;
  // Each half of the block (HX_HALF threads, its own named barrier) owns one plane slot and runs the planes
  // 2u + half on its own schedule, so one half's latency-bound prologue or epilogue overlaps the other half's
  // products.
  const int half = tid / HX_HALF, ht = tid % HX_HALF, lane = ht & 31, warp = ht >> 5;
  float *const W1e = (float *)smraw;
  float *const XO = W1e + Gm.wfloats() + (size_t)half * Gm.slot(n1m, n2m);
  float *const O1s = XO + (size_t)Gm.XR * P32_KPAD;
  float *const Stg = O1s + (size_t)Gm.KP * Gm.JP;
  auto hsync = [&]() { asm volatile("bar.sync %0, %1;" ::"r"(1 + half), "r"(HX_HALF) : "memory"); };
  auto locate = [&](int v, int &c) {   // pair v of the launch → (component c, pair u of that component)
    c = 0;
    while (c + 1 < M.ncomp && v >= (M.c[c].nplanes + 1) / 2) v -= (M.c[c++].nplanes + 1) / 2;
    return v;
  };
  auto stage = [&](int v) {   // this half's plane of pair v, raw, into its Stg (rows k, contiguous j)
    int c;
    const int u = locate(v, c);
    const HalfArgs &A = M.c[c];
    const int q = 2 * u + half;
    if (q >= A.nplanes) return;
    const float *in = A.in + A.in_base + (long long)q * A.in_ps + A.in_j0 + (long long)A.in_ld * A.in_k0;
    for (int k = warp; k < A.n2; k += HX_HWARPS)
      for (int j = lane; j < A.n1; j += 32) cp_async(Stg + k * A.n1 + j, in + j + (long long)A.in_ld * k);
  };
  int loaded = -1;
  double dz = 0.0, dzo = 0.0;   // r·z and r·z_old over this thread's written points (inverse with M.dot)
  for (int v = blockIdx.x; v < npairs; v += gridDim.x) {
    int ci;
    const int u = locate(v, ci);
    const HalfArgs &A = M.c[ci];
    const HalfGeo G(A.n1, A.n2);
    const int n1 = A.n1, n2 = A.n2;
    float *const W1o = W1e + (size_t)G.hS1 * G.R0;
    float *const W2e = W1o + (size_t)G.hD1 * G.R1;
    float *const W2o = W2e + (size_t)G.hS2 * G.C0;
    if (ci != loaded || v == (int)blockIdx.x) {
      __syncthreads();   // both halves are done with the previous half blocks
      if (ci != loaded) {   // the padded images of both axes (the four blocks are contiguous in shared memory)
        const int c1 = (G.hS1 * G.R0 + G.hD1 * G.R1) / 4, c2 = (G.hS2 * G.C0 + G.hD2 * G.C1) / 4;
        for (int t = tid; t < c1 + c2; t += HX_THREADS)
          cp_async16(W1e + 4 * t, t < c1 ? A.W1 + 4 * t : A.W2 + 4 * (t - c1));
        loaded = ci;
      }
      if (v == (int)blockIdx.x) stage(v);
      cp_async_wait_all();
      __syncthreads();   // the half blocks and this pair's planes are in shared memory
    }
    const int nkt = G.KP / 4, nkt8 = G.KP / 8, nrt0 = G.R0 / 8, nrt = G.JP / 8, nct0 = G.C0 / 8, nct = (G.C0 + G.C1) / 8;
    const int nq = G.hS1 * G.hS2, T1 = nrt * nkt8, T2 = nrt * nct, npad = G.KP - n2;
    const int q = 2 * u + half;
    if (q >= A.nplanes) {   // an odd component's last pair: this half only stages its next plane
      if (v + (int)gridDim.x < npairs) stage(v + gridDim.x);
      cp_async_wait_all();
      continue;
    }
    // prologue: X[r][c] in class order.  Forward: one item per mirror quadrant (p, qc), p < hS1, qc < hS2, reads
    // x at (p, qc), (p', qc), (p, qc'), (p', qc') (p' = n1−1−p, qc' = n2−1−qc; a middle point has no partner)
    // and writes its four class entries SS, SD, DS, DD.  Inverse: gathers even modes first, then odd ones.
    if (FWD) {
      for (int t = ht; t < nq; t += HX_HALF) {
        const int qc = t % G.hS2, p = t / G.hS2, pp = n1 - 1 - p, qq = n2 - 1 - qc;   // lanes along qc: no
        const bool rp = pp != p, cp = qq != qc;                                      // bank conflicts
        const float a = Stg[qc * n1 + p];
        const float b = rp ? Stg[qc * n1 + pp] : 0.f;
        const float c = cp ? Stg[qq * n1 + p] : 0.f;
        const float d = rp && cp ? Stg[qq * n1 + pp] : 0.f;
        const float s0 = a + c, s1 = b + d, d0 = a - c, d1 = b - d;
        float *x = XO + p * P32_KPAD, *xd = x + G.hS1 * P32_KPAD;
        x[xsw(qc)] = s0 + s1;
        if (cp) x[xsw(G.hS2 + qc)] = d0 + d1;
        if (rp) {
          xd[xsw(qc)] = s0 - s1;
          if (cp) xd[xsw(G.hS2 + qc)] = d0 - d1;
        }
      }
      if (npad > 0)   // zero columns n2..KP−1 (the previous O2 used them)
        for (int t = ht; t < n1 * npad; t += HX_HALF) XO[(t / npad) * P32_KPAD + xsw(n2 + t % npad)] = 0.f;
    } else {
      for (int c4 = warp; c4 < nkt; c4 += HX_HWARPS)
        for (int r = lane; r < n1; r += 32) {
          const int rb = r >= G.hS1, p = rb ? r - G.hS1 : r, m = rb ? 2 * p + 1 : 2 * p;
          float v[4];
#pragma unroll
          for (int b = 0; b < 4; b++) {
            const int c = 4 * c4 + b, cb = c >= G.hS2, qc = cb ? c - G.hS2 : c, mk = cb ? 2 * qc + 1 : 2 * qc;
            v[b] = c < n2 ? Stg[mk * n1 + m] : 0.f;
          }
          *reinterpret_cast<float4 *>(XO + r * P32_KPAD + xsw(4 * c4)) = make_float4(v[0], v[1], v[2], v[3]);
        }
    }
    hsync();
    if (v + (int)gridDim.x < npairs) stage(v + gridDim.x);
    // row product: O1[c][r_out] = Σ_{r_in of the block} W1[r_in][r_out] X[r_in][c]
    for (int tile = ht; tile < T1; tile += HX_HALF) {
      const int kt = tile % nkt8, rtg = tile / nkt8;
      const bool ob = rtg >= nrt0;
      const int rt = ob ? rtg - nrt0 : rtg, nin = ob ? G.hD1 : G.hS1, ld = ob ? G.R1 : G.R0;
      const float *mp = (ob ? W1o : W1e) + rt * 8, *ip = XO + (ob ? G.hS1 : 0) * P32_KPAD + xsw(kt * 8);
      float acc[8][8];
#pragma unroll
      for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = 0.f;
#pragma unroll 2
      for (int i = 0; i < nin; i++) {
        const float4 m0 = *reinterpret_cast<const float4 *>(mp + i * ld);
        const float4 m1 = *reinterpret_cast<const float4 *>(mp + i * ld + 4);
        const float4 x0 = *reinterpret_cast<const float4 *>(ip + i * P32_KPAD);
        const float4 x1 = *reinterpret_cast<const float4 *>(ip + i * P32_KPAD + 4);
        const float mv[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
        const float xv[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
          for (int b = 0; b < 8; b++) acc[a][b] = fmaf(mv[a], xv[b], acc[a][b]);
      }
      float *o = O1s + (ob ? G.R0 : 0) + rt * 8;
#pragma unroll
      for (int b = 0; b < 8; b++) {
        float *op = o + (kt * 8 + b) * G.JP;
        *reinterpret_cast<float4 *>(op) = make_float4(acc[0][b], acc[1][b], acc[2][b], acc[3][b]);
        *reinterpret_cast<float4 *>(op + 4) = make_float4(acc[4][b], acc[5][b], acc[6][b], acc[7][b]);
      }
    }
    hsync();
    // column product: O2[r][c_out] = Σ_{c_in of the block} O1[c_in][r] W2[c_in][c_out], into XO as [r][KS]
    for (int tile = ht; tile < T2; tile += HX_HALF) {
      const int ctg = tile % nct, rt = tile / nct;
      const bool ob = ctg >= nct0;
      const int ct = ob ? ctg - nct0 : ctg, nin = ob ? G.hD2 : G.hS2, ld = ob ? G.C1 : G.C0;
      const float *op = O1s + (ob ? G.hS2 : 0) * G.JP + rt * 8, *mp = (ob ? W2o : W2e) + ct * 8;
      float acc[8][8];
#pragma unroll
      for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = 0.f;
#pragma unroll 2
      for (int i = 0; i < nin; i++) {
        const float4 o0 = *reinterpret_cast<const float4 *>(op + i * G.JP);
        const float4 o1 = *reinterpret_cast<const float4 *>(op + i * G.JP + 4);
        const float4 w0 = *reinterpret_cast<const float4 *>(mp + i * ld);
        const float4 w1 = *reinterpret_cast<const float4 *>(mp + i * ld + 4);
        const float ov[8] = {o0.x, o0.y, o0.z, o0.w, o1.x, o1.y, o1.z, o1.w};
        const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
          for (int b = 0; b < 8; b++) acc[a][b] = fmaf(ov[a], wv[b], acc[a][b]);
      }
      float *o2 = XO + (ob ? G.C0 : 0) + ct * 8;
#pragma unroll
      for (int a = 0; a < 8; a++) {
        float *q2 = o2 + (rt * 8 + a) * G.KS;
        *reinterpret_cast<float4 *>(q2) = make_float4(acc[a][0], acc[a][1], acc[a][2], acc[a][3]);
        *reinterpret_cast<float4 *>(q2 + 4) = make_float4(acc[a][4], acc[a][5], acc[a][6], acc[a][7]);
      }
    }
    hsync();
    // epilogue: forward scatters the classes to mode order (four consecutive modes k per thread, consecutive
    // lanes on consecutive modes j); inverse unpairs one mirror quadrant (p, qc) per item into its four points
    // (consecutive lanes on consecutive p: the rows p and n1−1−p are both written contiguously)
    TOut *out = (TOut *)A.out + A.out_base + (long long)q * A.out_ps + A.out_j0 + (long long)A.out_ld * A.out_k0;
    if (FWD) {
      for (int k4 = warp; k4 < nkt; k4 += HX_HWARPS)
        for (int j = lane; j < n1; j += 32) {
          const float *o2 = XO + ((j & 1) ? G.R0 + (j >> 1) : (j >> 1)) * G.KS;
#pragma unroll
          for (int b = 0; b < 4; b++) {
            const int k = 4 * k4 + b;
            if (k >= n2) break;
            out[j + (long long)A.out_ld * k] = (TOut)o2[(k & 1) ? G.C0 + (k >> 1) : (k >> 1)];
          }
        }
    } else {
      const long long obase = out - (TOut *)A.out;   // r and z_old have z's layout
      const double *rr = M.dot ? M.df.r[ci] + obase : nullptr, *zo = M.dot ? M.df.zold[ci] + obase : nullptr;
      auto put = [&](long long at, float val) {
        const TOut zv = (TOut)val;
        out[at] = zv;
        if (M.dot) {
          const double rv = rr[at];
          dz += rv * (double)zv;
          dzo += rv * zo[at];
        }
      };
      for (int t = ht; t < nq; t += HX_HALF) {
        const int p = t % G.hS1, qc = t / G.hS1, pp = n1 - 1 - p, qq = n2 - 1 - qc;
        const bool rp = pp != p, cp = qq != qc;   // a partner exists exactly when the odd class has the index
        const float *o2 = XO + p * G.KS + qc;
        const float ee = o2[0];
        const float eo = cp ? o2[G.C0] : 0.f;
        const float oe = rp ? o2[G.R0 * G.KS] : 0.f;
        const float oo = rp && cp ? o2[G.R0 * G.KS + G.C0] : 0.f;
        const float s0 = ee + oe, s1 = eo + oo, d0 = ee - oe, d1 = eo - oo;
        const long long oq = (long long)A.out_ld * qc, oqq = (long long)A.out_ld * qq;
        put(oq + p, s0 + s1);
        if (rp) put(oq + pp, d0 + d1);
        if (cp) {
          put(oqq + p, s0 - s1);
          if (rp) put(oqq + pp, d0 - d1);
        }
      }
    }
    cp_async_wait_all();
    hsync();   // this half's next plane is staged; O2's reads are done before X is rewritten
  }
  if (!FWD && M.dot) {   // the block's partial sums, folded by the last block (pcg.cuh)
    __shared__ double sh[32];
    __syncthreads();
    const double a = block_sum(dz, sh);
    __syncthreads();
    const double b = block_sum(dzo, sh);
    if (tid == 0) {
      M.df.part[blockIdx.x] = a;
      M.df.part[gridDim.x + blockIdx.x] = b;
    }
    __syncthreads();
    fold_last(M.df.F, M.df.part, sh);
  }
}

// r32 = (float)r on the ranges' planes (the forward transform's FP32 input, when the caller has none)
__global__ void k_to_f32(const double *r, float *r32, long long n) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    r32[t] = (float)r[t];
}

// ---------------------------------------------------------------------------------------------- the line solve
// For one (my, mz) with k2 = s_y, k3 = s_z, c0 = 1 + a(k2² + k3²), (I + aK) along x reads
//   c0 X − a k2 D Y − a k3 D Z = bX (x edges),  −a k2 Dᵀ X + (I + a DᵀD + a k3²) Y − a k2 k3 Z = bY (nodes, and Z),
// D the forward difference and DᵀD the Neumann Laplacian.  Eliminating X leaves [[1+a k3², −a k2 k3],
// [−a k2 k3, 1+a k2²]] (determinant c0) times M = I + (a/c0) DᵀD on (Y, Z): one scalar tridiagonal M for both,
// solved by the Thomas algorithm, then X from Y and Z.  Empty slots (Y at my = 1, Z at mz = 1) stay zero.
// The factorisation of M per line is fixed for the run (it depends on a, k_y, k_z only): k_linefactor stores the
// pivot reciprocals inv_i = 1/(b_i − l c_{i−1}) and c_i = u_i inv_i once.
// The sweeps always run in FP64, also for the FP32 mode-space arrays of the FP32 preconditioner: M has condition
// number up to 1 + 4a/c0 (≈ 200 at a ≈ 49, the 256×128×32 ramp), so an FP32 sweep would lose ~1e-6 of relative
// accuracy on the low modes where the dense FP32 transforms of the reference's _precond32! (implicit.jl:346-373)
// keep ~3e-7.
__global__ void k_linefactor(double *inv, int nx, long long P, int ny, const double *sy, const double *sz,
                             double a) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int my = (int)(p % ny), mz = (int)(p / ny);
  const double k2 = sy[my], k3 = sz[mz];
  const double c0 = 1.0 + a * (k2 * k2 + k3 * k3);
  const double g = a / c0;
  double cprev = 0.0;
  for (int i = 0; i < nx; i++) {
    const double lo = i > 0 ? -g : 0.0, up = i < nx - 1 ? -g : 0.0;
    const double diag = 1.0 + g * ((i == 0 || i == nx - 1) ? 1.0 : 2.0);
    const double iv = 1.0 / (diag - lo * cprev);
    inv[p + P * i] = iv;
    cprev = up * iv;   // the sweeps form the same c_i = up·inv_i
  }
}

// One thread per line (lines are adjacent in memory, so every step of a sweep is a coalesced load across the warp),
// loads issued LS_U steps ahead.  For lines too long for the staged kernel below.
const int LS_U = 16;

template <class T>
__device__ __forceinline__ void linesolve_b(const Blk bk, T * const &Xh, T * const &Yh, T * const &Zh, const double * const &inv, int const &nx, long long const &P, int const &ny, const double * const &sy, const double * const &sz, double const &a, const int * const &done);
template <class T>
__global__ void __launch_bounds__(128) k_linesolve(T *Xh, T *Yh, T *Zh, const double *inv, int nx,
                                                   long long P, int ny, const double *sy, const double *sz, double a,
                                                   const int *done) {
  linesolve_b<T>(TDGL_BLK, Xh, Yh, Zh, inv, nx, P, ny, sy, sz, a, done);
}
TDGL_MERGEABLE((k_linesolve<double>), (linesolve_b<double>), 128, 1, false);
template <class T>
__device__ __forceinline__ void linesolve_b(const Blk bk, T * const &Xh, T * const &Yh, T * const &Zh, const double * const &inv, int const &nx, long long const &P, int const &ny, const double * const &sy, const double * const &sz, double const &a, const int * const &done) {
  if (done && *done) return;
  const long long p = (long long)bk.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int my = (int)(p % ny), mz = (int)(p / ny);
  const double k2 = sy[my], k3 = sz[mz];
  const double c0 = 1.0 + a * (k2 * k2 + k3 * k3);
  const double g = a / c0, fy = a * k2 / c0, fz = a * k3 / c0;
  const double pyy = (1.0 + a * k2 * k2) / c0, pyz = a * k2 * k3 / c0, pzz = (1.0 + a * k3 * k3) / c0;
  double dyp = 0.0, dzp = 0.0, bxl = 0.0;
  // forward sweep, LS_U nodes at a time: loads of a block issued before its arithmetic; the forward results go back
  // into Y and Z (rounded to T: with T = float the staged kernel, which keeps them in FP64, is the one used)
  for (int i0 = 0; i0 < nx; i0 += LS_U) {
    double xv[LS_U], yv[LS_U], zv[LS_U], iv[LS_U];
#pragma unroll
    for (int u = 0; u < LS_U; u++) {
      const int i = i0 + u;
      const long long o = p + P * i;
      xv[u] = i < nx - 1 ? (double)Xh[o] : 0.0;
      yv[u] = i < nx ? (double)Yh[o] : 0.0;
      zv[u] = i < nx ? (double)Zh[o] : 0.0;
      iv[u] = i < nx ? inv[o] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < LS_U; u++) {
      const int i = i0 + u;
      if (i >= nx) break;
      const double dtb = bxl - xv[u];
      const double byp = yv[u] + fy * dtb, bzp = zv[u] + fz * dtb;
      const double ry = pyy * byp + pyz * bzp, rz = pyz * byp + pzz * bzp;
      const double lo = i > 0 ? -g : 0.0;
      dyp = (ry - lo * dyp) * iv[u];
      dzp = (rz - lo * dzp) * iv[u];
      const long long o = p + P * i;
      Yh[o] = (T)dyp;
      Zh[o] = (T)dzp;
      bxl = xv[u];
    }
  }
  // backward sweep, and X from Y and Z
  double yn = 0.0, zn = 0.0;
  const int nb = (nx + LS_U - 1) / LS_U;
  for (int bI = nb - 1; bI >= 0; bI--) {
    const int i0 = bI * LS_U;
    double xv[LS_U], yv[LS_U], zv[LS_U], cv[LS_U];
#pragma unroll
    for (int u = 0; u < LS_U; u++) {
      const int i = i0 + u;
      const long long o = p + P * i;
      xv[u] = i < nx - 1 ? (double)Xh[o] : 0.0;
      yv[u] = i < nx ? (double)Yh[o] : 0.0;
      zv[u] = i < nx ? (double)Zh[o] : 0.0;
      cv[u] = i < nx ? (i < nx - 1 ? -g : 0.0) * inv[o] : 0.0;   // k_linefactor's c_i = up·inv_i
    }
#pragma unroll
    for (int u = LS_U - 1; u >= 0; u--) {
      const int i = i0 + u;
      if (i >= nx) continue;
      const long long o = p + P * i;
      const double y = yv[u] - cv[u] * yn, z = zv[u] - cv[u] * zn;
      if (i < nx - 1) Xh[o] = (T)((xv[u] + a * k2 * (yn - y) + a * k3 * (zn - z)) / c0);
      Yh[o] = (T)y;
      Zh[o] = (T)z;
      yn = y;
      zn = z;
    }
  }
}

// The same solve with the lines staged in shared memory: a block takes LS2_LINES consecutive lines and loads X, Y, Z
// and the factorisation with all its threads (coalesced rows, all loads in flight as cp.async), forms the
// right-hand sides in FP64, runs the two sweeps per (line, component) out of shared memory (LS2_LINES lanes per
// component), and writes Y, Z and X back with all its threads.  The arithmetic is that of k_linesolve, operation for
// operation, with every intermediate in FP64.
// Shared rows hold LS2_LINES lines and one pad entry (LS2_ROW): the sweeps' lanes walk chunks of consecutive rows,
// and an odd row length spreads them over the banks.
const int LS2_THREADS = 256, LS2_LINES = 8, LS2_ROW = LS2_LINES + 1;
template <class T>
size_t ls2_smem(int nx) {
  // x, y, z as T; the factorisation inv; for T = float also the FP64 right-hand sides of Y and Z
  return (size_t)nx * LS2_ROW * (3 * sizeof(T) + sizeof(double) + (sizeof(T) == 8 ? 0 : 2 * sizeof(double)));
}

template <class T>
__device__ __forceinline__ void linesolve_staged_b(const Blk bk, T * const &Xh, T * const &Yh, T * const &Zh, const double * const &inv, int const &nx, long long const &P, int const &ny, const double * const &sy, const double * const &sz, double const &a, const int * const &done);
template <class T>
__global__ void __launch_bounds__(LS2_THREADS) k_linesolve_staged(T *Xh, T *Yh, T *Zh, const double *inv,
                                                                  int nx, long long P, int ny, const double *sy,
                                                                  const double *sz, double a, const int *done) {
  linesolve_staged_b<T>(TDGL_BLK, Xh, Yh, Zh, inv, nx, P, ny, sy, sz, a, done);
}
TDGL_MERGEABLE((k_linesolve_staged<double>), (linesolve_staged_b<double>), LS2_THREADS, 1, false);
template <class T>
__device__ __forceinline__ void linesolve_staged_b(const Blk bk, T * const &Xh, T * const &Yh, T * const &Zh, const double * const &inv, int const &nx, long long const &P, int const &ny, const double * const &sy, const double * const &sz, double const &a, const int * const &done) {
  if (done && *done) return;
  constexpr int LB = LS2_LINES, RS = LS2_THREADS / LB, DS = LS2_ROW;
  constexpr bool F64 = sizeof(T) == 8;
  extern __shared__ __align__(16) unsigned char smraw[];
  double *ivs = (double *)smraw;   // [nx][DS]
  double *yd = ivs + (size_t)nx * DS, *zd = F64 ? nullptr : yd + (size_t)nx * DS;
  T *xs = (T *)(F64 ? yd : zd + (size_t)nx * DS);
  T *ys = xs + (size_t)nx * DS, *zs = ys + (size_t)nx * DS;
  if (F64) {   // the right-hand sides in place
    yd = (double *)ys;
    zd = (double *)zs;
  }
  const int tid = threadIdx.x, l = tid % LB, r0 = tid / LB;
  const long long p = (long long)bk.x * LB + l;
  const bool valid = p < P;
  for (int i = r0; i < nx; i += RS) {   // all loads in flight at once (cp.async), then one wait
    const long long o = p + P * i;
    const int s = i * DS + l;
    if (valid) {
      if (i < nx - 1) cp_async(xs + s, Xh + o);
      else xs[s] = T(0);
      cp_async(ys + s, Yh + o);
      cp_async(zs + s, Zh + o);
      cp_async(ivs + s, inv + o);
    } else {
      xs[s] = ys[s] = zs[s] = T(0);
      ivs[s] = 0.0;
    }
  }
  cp_async_wait_all();
  const int my = valid ? (int)(p % ny) : 0, mz = valid ? (int)(p / ny) : 0;
  const double k2 = sy[my], k3 = sz[mz];
  const double c0 = 1.0 + a * (k2 * k2 + k3 * k3);
  const double g = a / c0, fy = a * k2 / c0, fz = a * k3 / c0;
  const double pyy = (1.0 + a * k2 * k2) / c0, pyz = a * k2 * k3 / c0, pzz = (1.0 + a * k3 * k3) / c0;
  __syncthreads();
  for (int i = r0; i < nx; i += RS) {   // right-hand sides (x is only read)
    const int s = i * DS + l;
    const double dtb = (i > 0 ? (double)xs[s - DS] : 0.0) - (double)xs[s];
    const double byp = (double)ys[s] + fy * dtb, bzp = (double)zs[s] + fz * dtb;
    yd[s] = pyy * byp + pyz * bzp;
    zd[s] = pyz * byp + pzz * bzp;
  }
  __syncthreads();
  // the sweeps, one warp per (line, component): both are first-order linear recurrences, d_i = α_i d_{i−1} + β_i
  // forward (α_i = g inv_i, β_i = rhs_i inv_i) and y_i = −c_i y_{i+1} + d_i backward, so each lane composes the affine
  // maps of its chunk of ⌈nx/32⌉ nodes, a warp scan of the 32 maps gives every chunk its entry value, and the lanes
  // then run their chunks: ~2⌈nx/32⌉ + 5 dependent steps per sweep instead of nx
  {
    const int lane = tid & 31, warp = tid >> 5, C = (nx + 31) >> 5, i0 = lane * C, i1 = min(nx, i0 + C);
    for (int pr = warp; pr < 2 * LB; pr += LS2_THREADS / 32) {
      const int lp = pr % LB;
      double *v = pr < LB ? yd : zd;
      const double gl = __shfl_sync(0xffffffffu, g, lp);   // line lp's g: lane lp of every warp holds line lp
      // forward
      double A = 1.0, B = 0.0;
      for (int i = i0; i < i1; i++) {
        const int s = i * DS + lp;
        const double al = i > 0 ? gl * ivs[s] : 0.0, be = v[s] * ivs[s];
        A = al * A;
        B = al * B + be;
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double Ap = __shfl_up_sync(0xffffffffu, A, o), Bp = __shfl_up_sync(0xffffffffu, B, o);
        if (lane >= o) {
          B = A * Bp + B;
          A = A * Ap;
        }
      }
      double d = __shfl_up_sync(0xffffffffu, B, 1);
      if (lane == 0) d = 0.0;
      for (int i = i0; i < i1; i++) {
        const int s = i * DS + lp;
        const double al = i > 0 ? gl * ivs[s] : 0.0;
        d = al * d + v[s] * ivs[s];
        v[s] = d;
      }
      __syncwarp();
      // backward
      A = 1.0;
      B = 0.0;
      const double ul = -gl;   // the upper diagonal: c_i = up·inv_i (0 on the last node), as k_linefactor
      for (int i = i1 - 1; i >= i0; i--) {
        const int s = i * DS + lp;
        const double ga = -((i < nx - 1 ? ul : 0.0) * ivs[s]);
        A = ga * A;
        B = ga * B + v[s];
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double An = __shfl_down_sync(0xffffffffu, A, o), Bn = __shfl_down_sync(0xffffffffu, B, o);
        if (lane + o < 32) {
          B = A * Bn + B;
          A = A * An;
        }
      }
      double y = __shfl_down_sync(0xffffffffu, B, 1);
      if (lane == 31) y = 0.0;
      for (int i = i1 - 1; i >= i0; i--) {
        const int s = i * DS + lp;
        y = -((i < nx - 1 ? ul : 0.0) * ivs[s]) * y + v[s];
        v[s] = y;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (!valid) return;
  for (int i = r0; i < nx; i += RS) {
    const long long o = p + P * i;
    const int s = i * DS + l;
    const double y = yd[s], z = zd[s];
    if (i < nx - 1) Xh[o] = (T)(((double)xs[s] + a * k2 * (yd[s + DS] - y) + a * k3 * (zd[s + DS] - z)) / c0);
    Yh[o] = (T)y;
    Zh[o] = (T)z;
  }
}

// the FP64 bases' wave numbers s = 2 sin(πk/2n) of y and z, for both precisions
template <class T>
void linesolve(Ctx *ctx, SepDev *S, Work<T> &w, const int *done) {
  const int nx = S->nx;
  const long long P = S->P;
  const KCat cat = sizeof(T) == 8 ? K_MODES64 : K_MODES32;
  const double bytes = (6.0 * sizeof(T) + 8.0) * nx * P;   // X, Y, Z in and out; the factorisation in
  if (ls2_smem<T>(nx) <= 227 * 1024) {
    TDGL_LAUNCH(ctx, cat, bytes, k_linesolve_staged<T>, (int)((P + LS2_LINES - 1) / LS2_LINES), LS2_THREADS,
                ls2_smem<T>(nx), w.Xh, w.Yh, w.Zh, w.inv, nx, P, S->ny, S->bd[1].s, S->bd[2].s, ctx->P.a_imp,
                done);
  } else {
    TDGL_LAUNCH(ctx, cat, bytes, k_linesolve<T>, nblk(P, 128), 128, 0, w.Xh, w.Yh, w.Zh, w.inv, nx, P, S->ny,
                S->bd[1].s, S->bd[2].s, ctx->P.a_imp, done);
  }
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
  if (sizeof(T) == 4) {
    // half blocks of a basis B(p, m) with np points: E[p][me] = B(p, 2me) (p, me < ⌈np/2⌉), O[p][mo] = B(p, 2mo+1)
    // (p, mo < ⌊np/2⌋); the inverse stores the transposes
    auto halves = [&](int np, auto B, std::vector<T> &F, std::vector<T> &I) {
      const int hS = (np + 1) / 2, hD = np / 2, lS = (hS + 7) & ~7, lD = (hD + 7) & ~7;   // rows padded to 8
      F.assign((size_t)hS * lS + (size_t)hD * lD, T(0));
      I.assign(F.size(), T(0));
      for (int p = 0; p < hS; p++)
        for (int m = 0; m < hS; m++) {
          F[(size_t)p * lS + m] = B(p, 2 * m);
          I[(size_t)m * lS + p] = B(p, 2 * m);
        }
      const size_t o = (size_t)hS * lS;
      for (int p = 0; p < hD; p++)
        for (int m = 0; m < hD; m++) {
          F[o + (size_t)p * lD + m] = B(p, 2 * m + 1);
          I[o + (size_t)m * lD + p] = B(p, 2 * m + 1);
        }
    };
    std::vector<T> HVf, HVi, HUf, HUi;
    halves(n, [&](int p, int m) { return V[p + (size_t)n * m]; }, HVf, HVi);
    halves(n - 1, [&](int p, int m) { return U[p + (size_t)(n - 1) * m]; }, HUf, HUi);
    dalloc(ctx, &b.HVf, HVf.size()); dalloc(ctx, &b.HVi, HVi.size());
    dalloc(ctx, &b.HUf, HUf.size() + 1); dalloc(ctx, &b.HUi, HUi.size() + 1);
    cudaMemcpyAsync(b.HVf, HVf.data(), HVf.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(b.HVi, HVi.data(), HVi.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(b.HUf, HUf.data(), HUf.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(b.HUi, HUi.data(), HUi.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    // the tensor-core images of the same (FP32) half blocks
    std::vector<double> Bd((size_t)n * n), Ud((size_t)(n - 1) * (n - 1));
    for (size_t t = 0; t < Bd.size(); t++) Bd[t] = (double)V[t];
    for (size_t t = 0; t < Ud.size(); t++) Ud[t] = (double)U[t];
    std::vector<float> TVf, TVi, TUf, TUi;
    tc_images(n, Bd.data(), n, TVf, TVi);
    tc_images(n - 1, Ud.data(), n - 1, TUf, TUi);
    float *dst[4];
    const std::vector<float> *src[4] = {&TVf, &TVi, &TUf, &TUi};
    for (int t = 0; t < 4; t++) {
      dalloc(ctx, &dst[t], src[t]->size() + 4);
      cudaMemcpyAsync(dst[t], src[t]->data(), src[t]->size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
    }
    b.TVf = (T *)dst[0]; b.TVi = (T *)dst[1]; b.TUf = (T *)dst[2]; b.TUi = (T *)dst[3];
  }
  cudaStreamSynchronize(ctx->stream);
}


// ---------------------------------------------------------------------------------------------- large planes
// Large planes (whose one-block transform would leave at most two blocks per SM, or not fit one block) take the plane
// transform as two batched products through a plane-sized buffer in global memory (L2): T_q = M1 · In_q, then Out_q = T_q · M2ᵀ.  Each is C_q(m, n) = Σ_k A_q(m, k) B_q(k, n), the
// sum over k in index order (fma from 0), so both sums run in the order of the one-block kernel and give its bits.
// A_q(m, k) = A[a_off + a_q·q + a_m·m + a_k·k] (a_q = 0: an operand shared by the planes), likewise B and C.
// A block takes a 64 × 64 output tile of one plane: 64 threads, 8 × 8 outputs each (rows 4t_m..4t_m+3 and 32 more,
// columns likewise), 16-deep operand tiles in shared memory; several blocks per SM hide the loads.
struct BGemm {
  const void *A, *B;
  void *C;
  long long a_off, a_q, a_m, a_k, b_off, b_q, b_k, b_n, c_off, c_q, c_m, c_n;
  int M, N, K;
  const int *done;
};
const int GB_M = 64, GB_N = 64, GB_K = 16, GB_THREADS = 64, GB_LD = GB_K * GB_M / GB_THREADS;
const size_t GB_ONEBLOCK = 96 * 1024;

template <class TA_, class TB_, class TC_, class T>
__global__ void __launch_bounds__(GB_THREADS) k_bgemm(BGemm G) {
  if (G.done && *G.done) return;
  // rows padded by 4 (16-byte aligned rows; the stores of k-fastest operands fall on distinct banks but for pairs)
  __shared__ __align__(16) T As[GB_K][GB_M + 4];
  __shared__ __align__(16) T Bs[GB_K][GB_N + 4];
  const int tid = threadIdx.x, m0 = blockIdx.x * GB_M, n0 = blockIdx.y * GB_N;
  const long long q = blockIdx.z;
  const TA_ *Ap = (const TA_ *)G.A + G.a_off + q * G.a_q;
  const TB_ *Bp = (const TB_ *)G.B + G.b_off + q * G.b_q;
  // the operand loads put the unit-stride index across the threads (coalesced): element u of a thread is
  // (m, k) = (tid, u) when a_m = 1, else (tid / 16 + 4u, tid % 16); likewise B; out of range reads 0
  const bool am = G.a_m == 1, bk = G.b_k == 1;
  const int am_m = am ? tid : tid / GB_K, am_k = am ? 0 : tid % GB_K;
  const int bk_n = bk ? tid / GB_K : tid, bk_k = bk ? tid % GB_K : 0;
  const int tm = tid % 8, tn = tid / 8;
  T acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; a++)
#pragma unroll
    for (int b = 0; b < 8; b++) acc[a][b] = T(0);
  for (int k0 = 0; k0 < G.K; k0 += GB_K) {
    __syncthreads();   // the previous tile's readers are done
#pragma unroll 4
    for (int u = 0; u < GB_LD; u++) {
      const int m = am ? am_m : am_m + 4 * u, ka = am ? u : am_k;
      const int gm = m0 + m, gka = k0 + ka;
      As[ka][m] = (gm < G.M && gka < G.K) ? (T)Ap[G.a_m * gm + G.a_k * gka] : T(0);
      const int n = bk ? bk_n + 4 * u : bk_n, kb = bk ? bk_k : u;
      const int gn = n0 + n, gkb = k0 + kb;
      Bs[kb][n] = (gn < G.N && gkb < G.K) ? (T)Bp[G.b_k * gkb + G.b_n * gn] : T(0);
    }
    __syncthreads();
    const int kn = min(GB_K, G.K - k0);
    for (int k = 0; k < kn; k++) {
      T av[8], bv[8];
#pragma unroll
      for (int a = 0; a < 4; a++) {
        av[a] = As[k][4 * tm + a];
        av[4 + a] = As[k][32 + 4 * tm + a];
        bv[a] = Bs[k][4 * tn + a];
        bv[4 + a] = Bs[k][32 + 4 * tn + a];
      }
#pragma unroll
      for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
  }
  TC_ *Cp = (TC_ *)G.C + G.c_off + q * G.c_q;
#pragma unroll
  for (int a = 0; a < 8; a++) {
    const int gm = m0 + (a < 4 ? 4 * tm + a : 32 + 4 * tm + a - 4);
    if (gm >= G.M) continue;
#pragma unroll
    for (int b = 0; b < 8; b++) {
      const int gn = n0 + (b < 4 ? 4 * tn + b : 32 + 4 * tn + b - 4);
      if (gn < G.N) Cp[G.c_m * gm + G.c_n * gn] = (TC_)acc[a][b];
    }
  }
}

// the two batched products of a plane transform through the buffer `tmp` (nplanes × nj_out × nk_in of T)
template <class TIn, class TOut, class T>
void plane_gemm(Ctx *ctx, const PlaneArgs &A, T *tmp, double bytes) {
  const int cat = sizeof(T) == 8 ? K_TX64 : K_TX32;
  BGemm G1;   // T_q(jo, k) = Σ_j M1t[jo + nj_out j] In_q(j, k)
  G1.A = A.M1t; G1.a_off = 0; G1.a_q = 0; G1.a_m = 1; G1.a_k = A.nj_out;
  G1.B = A.in; G1.b_off = A.in_base + A.in_j0 + (long long)A.in_ld * A.in_k0; G1.b_q = A.in_ps; G1.b_k = 1;
  G1.b_n = A.in_ld;
  G1.C = tmp; G1.c_off = 0; G1.c_q = (long long)A.nj_out * A.nk_in; G1.c_m = 1; G1.c_n = A.nj_out;
  G1.M = A.nj_out; G1.N = A.nk_in; G1.K = A.nj_in;
  G1.done = A.done;
  dim3 g1((G1.M + GB_M - 1) / GB_M, (G1.N + GB_N - 1) / GB_N, A.nplanes);
  TDGL_LAUNCH(ctx, cat, bytes / 2, (k_bgemm<T, TIn, T, T>), g1, GB_THREADS, 0, G1);
  BGemm G2;   // Out_q(jo, ko) = Σ_k T_q(jo, k) M2t[ko + nk_out k]
  G2.A = tmp; G2.a_off = 0; G2.a_q = (long long)A.nj_out * A.nk_in; G2.a_m = 1; G2.a_k = A.nj_out;
  G2.B = A.M2t; G2.b_off = 0; G2.b_q = 0; G2.b_k = A.nk_out; G2.b_n = 1;
  G2.C = A.out; G2.c_off = A.out_base + A.out_j0 + (long long)A.out_ld * A.out_k0; G2.c_q = A.out_ps; G2.c_m = 1;
  G2.c_n = A.out_ld;
  G2.M = A.nj_out; G2.N = A.nk_out; G2.K = A.nk_in;
  G2.done = A.done;
  dim3 g2((G2.M + GB_M - 1) / GB_M, (G2.N + GB_N - 1) / GB_N, A.nplanes);
  TDGL_LAUNCH(ctx, cat, bytes / 2, (k_bgemm<T, T, TOut, T>), g2, GB_THREADS, 0, G2);
}

// The mirror-halved FP32 transforms (as k_half32) of planes too large for one block: a pass that pairs the points
// (forward) or gathers the modes in class order (inverse) into X, the row product and the column product of each
// class as batched products (k_bgemm) on the half blocks, and a pass that scatters the modes (forward) or unpairs the
// points (inverse).  Per plane: X (n1 × n2, class order, column-major), O1 (JP × n2), O2 (JP × (C0 + C1), in X's
// buffer); the products sum in k_half32's order, so the results are its.
template <bool FWD>
__global__ void k_half_in(HalfArgs A, float *X, long long xps, const double *in64, const int *done) {
  if (done && *done) return;
  const HalfGeo G(A.n1, A.n2);
  const int n1 = A.n1, n2 = A.n2;
  const long long per = FWD ? (long long)G.hS1 * G.hS2 : (long long)n1 * n2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per * A.nplanes) return;
  const long long q = t / per;
  const int e = (int)(t % per);
  float *x = X + q * xps;
  if (FWD) {   // the four points of a mirror quadrant (p, qc) → its four class entries SS, SD, DS, DD
    const double *in = in64 + A.in_base + q * A.in_ps + A.in_j0 + (long long)A.in_ld * A.in_k0;
    const int qc = e % G.hS2, p = e / G.hS2, pp = n1 - 1 - p, qq = n2 - 1 - qc;
    const bool rp = pp != p, cp = qq != qc;
    const float a = (float)in[p + (long long)A.in_ld * qc];
    const float b = rp ? (float)in[pp + (long long)A.in_ld * qc] : 0.f;
    const float c = cp ? (float)in[p + (long long)A.in_ld * qq] : 0.f;
    const float d = rp && cp ? (float)in[pp + (long long)A.in_ld * qq] : 0.f;
    const float s0 = a + c, s1 = b + d, d0 = a - c, d1 = b - d;
    x[p + (long long)n1 * qc] = s0 + s1;
    if (cp) x[p + (long long)n1 * (G.hS2 + qc)] = d0 + d1;
    if (rp) {
      x[G.hS1 + p + (long long)n1 * qc] = s0 - s1;
      if (cp) x[G.hS1 + p + (long long)n1 * (G.hS2 + qc)] = d0 - d1;
    }
  } else {     // X(r, c) = the mode of class order (r, c): even modes first
    const float *in = A.in + A.in_base + q * A.in_ps + A.in_j0 + (long long)A.in_ld * A.in_k0;
    const int r = e % n1, c = e / n1;
    const int m = r < G.hS1 ? 2 * r : 2 * (r - G.hS1) + 1, mk = c < G.hS2 ? 2 * c : 2 * (c - G.hS2) + 1;
    x[r + (long long)n1 * c] = in[m + (long long)A.in_ld * mk];
  }
}

template <bool FWD>
__global__ void k_half_out(HalfArgs A, const float *O2, long long ops, const int *done) {
  if (done && *done) return;
  const HalfGeo G(A.n1, A.n2);
  const int n1 = A.n1, n2 = A.n2, JP = G.JP;
  const long long per = FWD ? (long long)n1 * n2 : (long long)G.hS1 * G.hS2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per * A.nplanes) return;
  const long long q = t / per;
  const int e = (int)(t % per);
  const float *o2 = O2 + q * ops;
  if (FWD) {   // modes in order: row j from its class (even j: E row j/2, odd: O row R0 + j/2), likewise columns
    float *out = (float *)A.out + A.out_base + q * A.out_ps + A.out_j0 + (long long)A.out_ld * A.out_k0;
    const int j = e % n1, k = e / n1;
    const int r = (j & 1) ? G.R0 + (j >> 1) : (j >> 1), c = (k & 1) ? G.C0 + (k >> 1) : (k >> 1);
    out[j + (long long)A.out_ld * k] = o2[r + (long long)JP * c];
  } else {     // unpair one mirror quadrant (p, qc) into its four points
    double *out = (double *)A.out + A.out_base + q * A.out_ps + A.out_j0 + (long long)A.out_ld * A.out_k0;
    const int p = e % G.hS1, qc = e / G.hS1, pp = n1 - 1 - p, qq = n2 - 1 - qc;
    const bool rp = pp != p, cp = qq != qc;
    const float ee = o2[p + (long long)JP * qc];
    const float eo = cp ? o2[p + (long long)JP * (G.C0 + qc)] : 0.f;
    const float oe = rp ? o2[G.R0 + p + (long long)JP * qc] : 0.f;
    const float oo = rp && cp ? o2[G.R0 + p + (long long)JP * (G.C0 + qc)] : 0.f;
    const float s0 = ee + oe, s1 = eo + oo, d0 = ee - oe, d1 = eo - oo;
    const long long oq = (long long)A.out_ld * qc, oqq = (long long)A.out_ld * qq;
    out[oq + p] = (double)(s0 + s1);
    if (rp) out[oq + pp] = (double)(d0 + d1);
    if (cp) {
      out[oqq + p] = (double)(s0 - s1);
      if (rp) out[oqq + pp] = (double)(d0 - d1);
    }
  }
}

// The same batched product with the tile shape as template parameters: BM × BN outputs per block, TM × TN per thread
// (TM or TN = 8: two runs of 4, half a tile apart, so that the 16-byte shared loads of a quarter warp are one
// contiguous row; 6: one run).  The mirror-halved products take 48 × 96 tiles (rows ⌈n/2⌉ = 144, columns n2 = 95) and
// 96 × 48 tiles (rows JP = 288, columns 48), which divide them with almost no empty outputs; 96 threads each.
template <int BM, int BN, int TM, int TN, class T>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) k_bgemm_t(BGemm G) {
  constexpr int NT = (BM / TM) * (BN / TN), LA = GB_K * BM / NT, LB = GB_K * BN / NT;
  if (G.done && *G.done) return;
  __shared__ __align__(16) T As[GB_K][BM + 4];
  __shared__ __align__(16) T Bs[GB_K][BN + 4];
  const int tid = threadIdx.x, m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const long long q = blockIdx.z;
  const T *Ap = (const T *)G.A + G.a_off + q * G.a_q;
  const T *Bp = (const T *)G.B + G.b_off + q * G.b_q;
  static_assert(NT % BM == 0 && NT % BN == 0 && NT % GB_K == 0, "tile loads: whole rows per pass");
  const bool am = G.a_m == 1, bk = G.b_k == 1;
  // element u of this thread's loads: A (m, k) = (tid % BM, tid / BM + u NT/BM) when a_m = 1, else
  // (tid / 16 + u NT/16, tid % 16); B likewise
  const int a_m0 = am ? tid % BM : tid / GB_K, a_k0 = am ? tid / BM : tid % GB_K;
  const int a_dm = am ? 0 : NT / GB_K, a_dk = am ? NT / BM : 0;
  const int b_n0 = bk ? tid / GB_K : tid % BN, b_k0 = bk ? tid % GB_K : tid / BN;
  const int b_dn = bk ? NT / GB_K : 0, b_dk = bk ? 0 : NT / BN;
  const int tm = tid % (BM / TM), tn = tid / (BM / TM);
  auto row = [&](int a) { return TM == 8 ? (a < 4 ? 4 * tm + a : BM / 2 + 4 * tm + a - 4) : TM * tm + a; };
  auto col = [&](int b) { return TN == 8 ? (b < 4 ? 4 * tn + b : BN / 2 + 4 * tn + b - 4) : TN * tn + b; };
  T acc[TM][TN];
#pragma unroll
  for (int a = 0; a < TM; a++)
#pragma unroll
    for (int b = 0; b < TN; b++) acc[a][b] = T(0);
  for (int k0 = 0; k0 < G.K; k0 += GB_K) {
    __syncthreads();
#pragma unroll 4
    for (int u = 0; u < LA; u++) {
      const int m = a_m0 + a_dm * u, k = a_k0 + a_dk * u;
      const int gm = m0 + m, gk = k0 + k;
      As[k][m] = (gm < G.M && gk < G.K) ? Ap[G.a_m * gm + G.a_k * gk] : T(0);
    }
#pragma unroll 4
    for (int u = 0; u < LB; u++) {
      const int n = b_n0 + b_dn * u, k = b_k0 + b_dk * u;
      const int gn = n0 + n, gk = k0 + k;
      Bs[k][n] = (gn < G.N && gk < G.K) ? Bp[G.b_k * gk + G.b_n * gn] : T(0);
    }
    __syncthreads();
    const int kn = min(GB_K, G.K - k0);
    for (int k = 0; k < kn; k++) {
      T av[TM], bv[TN];
#pragma unroll
      for (int a = 0; a < TM; a++) av[a] = As[k][row(a)];
#pragma unroll
      for (int b = 0; b < TN; b++) bv[b] = Bs[k][col(b)];
#pragma unroll
      for (int a = 0; a < TM; a++)
#pragma unroll
        for (int b = 0; b < TN; b++) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
  }
  T *Cp = (T *)G.C + G.c_off + q * G.c_q;
#pragma unroll
  for (int a = 0; a < TM; a++) {
    const int gm = m0 + row(a);
    if (gm >= G.M) continue;
#pragma unroll
    for (int b = 0; b < TN; b++) {
      const int gn = n0 + col(b);
      if (gn < G.N) Cp[G.c_m * gm + G.c_n * gn] = acc[a][b];
    }
  }
}

// one component's mirror-halved transform of large planes (forward: FP64 points in; inverse: FP64 points out)
void half_gemm(Ctx *ctx, const HalfArgs &A, bool fwd, const double *in64, const int *done) {
  SepDev *S = ctx->sep;
  const HalfGeo G(A.n1, A.n2);
  const KCat cat = fwd ? K_TX32 : K_TX32I;
  const long long nin = fwd ? (long long)G.hS1 * G.hS2 * A.nplanes : (long long)A.n1 * A.n2 * A.nplanes;
  const double pts = (double)A.n1 * A.n2 * A.nplanes;
  if (fwd) TDGL_LAUNCH(ctx, cat, 12.0 * pts, k_half_in<true>, nblk(nin, 256), 256, 0, A, S->hx, S->hx_ps, in64, done);
  else TDGL_LAUNCH(ctx, cat, 8.0 * pts, k_half_in<false>, nblk(nin, 256), 256, 0, A, S->hx, S->hx_ps, nullptr, done);
  const float *W1[2] = {A.W1, A.W1 + (size_t)G.hS1 * G.R0}, *W2[2] = {A.W2, A.W2 + (size_t)G.hS2 * G.C0};
  const int h1[2] = {G.hS1, G.hD1}, R[2] = {G.R0, G.R1}, h2[2] = {G.hS2, G.hD2}, Cw[2] = {G.C0, G.C1};
  for (int a = 0; a < 2; a++) {   // row product of class a: O1(r, c) = Σ_i W1a[i][r] X(off_a + i, c)
    if (h1[a] < 1) continue;
    BGemm B;
    B.A = W1[a]; B.a_off = 0; B.a_q = 0; B.a_m = 1; B.a_k = R[a];
    B.B = S->hx; B.b_off = a ? G.hS1 : 0; B.b_q = S->hx_ps; B.b_k = 1; B.b_n = A.n1;
    B.C = S->ho; B.c_off = a ? G.R0 : 0; B.c_q = S->ho_ps; B.c_m = 1; B.c_n = G.JP;
    B.M = h1[a]; B.N = A.n2; B.K = h1[a];
    B.done = done;
    dim3 g((B.M + 47) / 48, (B.N + 95) / 96, A.nplanes);
    TDGL_LAUNCH(ctx, cat, 8.0 * pts / 2, (k_bgemm_t<48, 96, 6, 8, float>), g, 96, 0, B);
  }
  for (int b = 0; b < 2; b++) {   // column product of class b: O2(r, C_off + c) = Σ_k O1(r, off_b + k) W2b[k][c]
    if (h2[b] < 1) continue;
    BGemm B;
    B.A = S->ho; B.a_off = (long long)G.JP * (b ? G.hS2 : 0); B.a_q = S->ho_ps; B.a_m = 1; B.a_k = G.JP;
    B.B = W2[b]; B.b_off = 0; B.b_q = 0; B.b_k = Cw[b]; B.b_n = 1;
    B.C = S->hx; B.c_off = (long long)G.JP * (b ? G.C0 : 0); B.c_q = S->hx_ps; B.c_m = 1; B.c_n = G.JP;
    B.M = G.JP; B.N = h2[b]; B.K = h2[b];
    B.done = done;
    dim3 g((B.M + 95) / 96, (B.N + 47) / 48, A.nplanes);
    TDGL_LAUNCH(ctx, cat, 8.0 * pts / 2, (k_bgemm_t<96, 48, 8, 6, float>), g, 96, 0, B);
  }
  const long long nout = fwd ? (long long)A.n1 * A.n2 * A.nplanes : (long long)G.hS1 * G.hS2 * A.nplanes;
  if (fwd) TDGL_LAUNCH(ctx, cat, 8.0 * pts, k_half_out<true>, nblk(nout, 256), 256, 0, A, S->hx, S->hx_ps, done);
  else TDGL_LAUNCH(ctx, cat, 12.0 * pts, k_half_out<false>, nblk(nout, 256), 256, 0, A, S->hx, S->hx_ps, done);
}

template <class TIn, class TOut, class T>
void plane(Ctx *ctx, PlaneArgs A) {
  const double bytes = (double)A.nplanes * ((double)A.nj_in * A.nk_in * sizeof(TIn) + (double)A.nj_out * A.nk_out * sizeof(TOut));
  const int ngy = (A.nj_out + PL_JC - 1) / PL_JC;
  // planes whose one-block transform would hold more than GB_ONEBLOCK of shared memory (at most two blocks per SM)
  // take the batched products when the context has their buffer
  const size_t one = plane_smem<T>(A.nj_in, A.nk_in, A.nk_out);
  if (one > GB_ONEBLOCK && one <= 227 * 1024 && ctx->sep && ctx->sep->gtmp) {
    plane_gemm<TIn, TOut, T>(ctx, A, (T *)ctx->sep->gtmp, bytes);
  } else if (one <= 227 * 1024) {
    // the output rows split evenly over the chunks (no chunk mostly empty); room for as many planes per pass as keep
    // the threads busy (at most PL_PPB; at most 56 KB of shared memory, four blocks per SM), used when a block has
    // several planes (a merged launch gives each context fewer blocks); persistent: a block keeps its basis chunks
    // in shared memory for all its planes (about four blocks per SM in all).  Small planes take 2-row tiles.
    const bool small = A.nj_out <= 2 * PL_JC;
    A.jc = small ? rup4((A.nj_out + ngy - 1) / ngy) : PL_JC;
    const int ta = small ? 2 : 4;
    const int tiles = (A.jc / ta) * (std::max(rup4(A.nk_in), rup4(A.nk_out)) / 4);
    A.ppb = std::max(1, std::min(PL_PPB, PL_THREADS / std::max(1, tiles)));
    while (A.ppb > 1 && plane_smem<T>(A.nj_in, A.nk_in, A.nk_out, A.jc, A.ppb) > 56 * 1024) A.ppb--;
    const size_t smem = plane_smem<T>(A.nj_in, A.nk_in, A.nk_out, A.jc, A.ppb);
    const int nsm = g_sm_count > 0 ? g_sm_count : 148;
    dim3 grid(std::max(1, std::min((int)A.nplanes, (4 * nsm + ngy - 1) / ngy)), ngy);
    const int cat = sizeof(T) == 8 ? K_TX64 : K_TX32;
    if (small) TDGL_LAUNCH(ctx, cat, bytes, (k_plane<TIn, TOut, T, 2>), grid, PL_THREADS, smem, A);
    else TDGL_LAUNCH(ctx, cat, bytes, (k_plane<TIn, TOut, T, 4>), grid, PL_THREADS, smem, A);
  } else if (ctx->sep && ctx->sep->gtmp) {
    // a plane too large for one block: two batched products through a plane-sized buffer
    plane_gemm<TIn, TOut, T>(ctx, A, (T *)ctx->sep->gtmp, bytes);
  } else {
    // a plane too large for one block, without the buffer: chunked sums (sep_create checked that these fit)
    A.jc = PL_JC;
    A.ppb = 1;
    dim3 grid(A.nplanes, ngy);
    TDGL_LAUNCH(ctx, sizeof(T) == 8 ? K_TX64 : K_TX32, bytes, (k_plane_tiled<TIn, TOut, T>), grid, PT_THREADS,
                tiled_smem<T>(A.nk_out), A);
  }
}

void half_tx(Ctx *ctx, const HalfMulti &M, bool fwd) {
  const int nsm = g_sm_count > 0 ? g_sm_count : 148;
  int npairs = 0, n1m = 1, n2m = 1;
  double bytes = 0;
  for (int c = 0; c < M.ncomp; c++) {
    const HalfArgs &A = M.c[c];
    npairs += (A.nplanes + 1) / 2;
    n1m = std::max(n1m, A.n1);
    n2m = std::max(n2m, A.n2);
    bytes += (double)A.nplanes * A.n1 * A.n2 * (fwd ? 2 * sizeof(float) : sizeof(float) + sizeof(double));
  }
  const int grid = npairs < nsm ? npairs : nsm;
  if (grid <= 0) return;
  if (fwd) TDGL_LAUNCH(ctx, K_TX32, bytes, (k_half32<float, true>), grid, HX_THREADS, half_smem(n1m, n2m), M);
  else TDGL_LAUNCH(ctx, K_TX32I, bytes, (k_half32<double, false>), grid, HX_THREADS, half_smem(n1m, n2m), M);
}

template <class TIn, class TOut, class T>
void set_plane_smem() {
  smem_optin(k_plane<TIn, TOut, T, 2>);
  smem_optin(k_plane<TIn, TOut, T, 4>);
}

// z = (I + aK)^{-1} r: r and z are the three plane-major node-shaped component arrays (FP64); entries of z outside
// the ranges are not written.
template <class T>
void solve(Ctx *ctx, SepDev *S, const Basis<T> *b, Work<T> &w, const double *const *r, double *const *z, const int *done,
           const float *const *r32 = nullptr, const DotFuse *dot = nullptr) {
  const Geo &g = ctx->g;
  const int nx = S->nx, ny = S->ny, nz = S->nz;
  const long long n2 = g.Ny + 1, n3 = g.Nz + 1, ps = n2 * n3, P = S->P;
  // the ranges (implicit.jl:52) start at i = j = k = 2 (0-based plane 1, row 1, column 1)
  auto fwd = [&](const double *in, int nj, int nk, const T *M1t, const T *M2t, int njo, int nko, int jo_off, int ko_off,
                 T *hat, int nplanes) {
    PlaneArgs A;
    A.in = in; A.in_base = ps; A.in_ps = ps; A.in_ld = (int)n2; A.in_j0 = 1; A.in_k0 = 1;
    A.nj_in = nj; A.nk_in = nk;
    A.M1t = M1t; A.M2t = M2t;
    A.nj_out = njo; A.nk_out = nko;
    A.out = hat; A.out_base = 0; A.out_ps = P; A.out_ld = ny; A.out_j0 = jo_off; A.out_k0 = ko_off;
    A.nplanes = nplanes;
    A.done = done;
    plane<double, T, T>(ctx, A);
  };
  auto inv = [&](const T *hat, int nj, int nk, int j_off, int k_off, const T *M1t, const T *M2t, int njo, int nko, double *out,
                 int nplanes) {
    PlaneArgs A;
    A.in = hat; A.in_base = 0; A.in_ps = P; A.in_ld = ny; A.in_j0 = j_off; A.in_k0 = k_off;
    A.nj_in = nj; A.nk_in = nk;
    A.M1t = M1t; A.M2t = M2t;
    A.nj_out = njo; A.nk_out = nko;
    A.out = out; A.out_base = ps; A.out_ps = ps; A.out_ld = (int)n2; A.out_j0 = 1; A.out_k0 = 1;
    A.nplanes = nplanes;
    A.done = done;
    plane<T, double, T>(ctx, A);
  };
  if constexpr (sizeof(T) == 4) {
    if (r32) {   // the mirror-halved FP32 transforms: one launch per direction for the three components
      HalfMulti F, I;
      F.ncomp = I.ncomp = 3;
      F.done = I.done = done;
      F.dot = 0;
      I.dot = dot != nullptr;
      if (dot) I.df = *dot;
      const float *W1f[3] = {b[1].HVf, b[1].HUf, b[1].HVf}, *W2f[3] = {b[2].HVf, b[2].HVf, b[2].HUf};
      const float *W1i[3] = {b[1].HVi, b[1].HUi, b[1].HVi}, *W2i[3] = {b[2].HVi, b[2].HVi, b[2].HUi};
      const float *T1f[3] = {b[1].TVf, b[1].TUf, b[1].TVf}, *T2f[3] = {b[2].TVf, b[2].TVf, b[2].TUf};
      const float *T1i[3] = {b[1].TVi, b[1].TUi, b[1].TVi}, *T2i[3] = {b[2].TVi, b[2].TVi, b[2].TUi};
      T *hat[3] = {w.Xh, w.Yh, w.Zh};
      const int c1[3] = {ny, ny - 1, ny}, c2[3] = {nz, nz, nz - 1}, j0[3] = {0, 1, 0}, k0[3] = {0, 0, 1};
      const int planes[3] = {nx - 1, nx, nx};
      for (int c = 0; c < 3; c++) {
        HalfArgs &f = F.c[c], &v = I.c[c];
        f.in = r32[c]; f.in_base = ps; f.in_ps = ps; f.in_ld = (int)n2; f.in_j0 = 1; f.in_k0 = 1;
        f.out = hat[c]; f.out_base = 0; f.out_ps = P; f.out_ld = ny; f.out_j0 = j0[c]; f.out_k0 = k0[c];
        f.n1 = c1[c]; f.n2 = c2[c]; f.nplanes = planes[c]; f.W1 = W1f[c]; f.W2 = W2f[c]; f.T1 = T1f[c]; f.T2 = T2f[c];
        v.in = hat[c]; v.in_base = 0; v.in_ps = P; v.in_ld = ny; v.in_j0 = j0[c]; v.in_k0 = k0[c];
        v.out = z[c]; v.out_base = ps; v.out_ps = ps; v.out_ld = (int)n2; v.out_j0 = 1; v.out_k0 = 1;
        v.n1 = c1[c]; v.n2 = c2[c]; v.nplanes = planes[c]; v.W1 = W1i[c]; v.W2 = W2i[c]; v.T1 = T1i[c]; v.T2 = T2i[c];
      }
      if (S->tc) {
        long long *err = pcg_stat_tc(ctx);
        half_tc(ctx, F, true, err);
        linesolve<T>(ctx, S, w, done);
        half_tc(ctx, I, false, err);
      } else {
        half_tx(ctx, F, true);
        linesolve<T>(ctx, S, w, done);
        half_tx(ctx, I, false);
      }
      return;
    }
    if (S->hx) {   // planes too large for one block: the same mirror-halved transforms as batched products
      const float *W1f[3] = {b[1].HVf, b[1].HUf, b[1].HVf}, *W2f[3] = {b[2].HVf, b[2].HVf, b[2].HUf};
      const float *W1i[3] = {b[1].HVi, b[1].HUi, b[1].HVi}, *W2i[3] = {b[2].HVi, b[2].HVi, b[2].HUi};
      T *hat[3] = {w.Xh, w.Yh, w.Zh};
      const int c1[3] = {ny, ny - 1, ny}, c2[3] = {nz, nz, nz - 1}, j0[3] = {0, 1, 0}, k0[3] = {0, 0, 1};
      const int planes[3] = {nx - 1, nx, nx};
      HalfArgs f[3], v[3];
      for (int c = 0; c < 3; c++) {
        f[c] = HalfArgs();
        f[c].in = nullptr; f[c].in_base = ps; f[c].in_ps = ps; f[c].in_ld = (int)n2; f[c].in_j0 = 1; f[c].in_k0 = 1;
        f[c].out = hat[c]; f[c].out_base = 0; f[c].out_ps = P; f[c].out_ld = ny; f[c].out_j0 = j0[c]; f[c].out_k0 = k0[c];
        f[c].n1 = c1[c]; f[c].n2 = c2[c]; f[c].nplanes = planes[c]; f[c].W1 = W1f[c]; f[c].W2 = W2f[c];
        v[c] = HalfArgs();
        v[c].in = hat[c]; v[c].in_base = 0; v[c].in_ps = P; v[c].in_ld = ny; v[c].in_j0 = j0[c]; v[c].in_k0 = k0[c];
        v[c].out = z[c]; v[c].out_base = ps; v[c].out_ps = ps; v[c].out_ld = (int)n2; v[c].out_j0 = 1; v[c].out_k0 = 1;
        v[c].n1 = c1[c]; v[c].n2 = c2[c]; v[c].nplanes = planes[c]; v[c].W1 = W1i[c]; v[c].W2 = W2i[c];
      }
      for (int c = 0; c < 3; c++) half_gemm(ctx, f[c], true, r[c], done);
      linesolve<T>(ctx, S, w, done);
      for (int c = 0; c < 3; c++) half_gemm(ctx, v[c], false, nullptr, done);
      return;
    }
  }
  // forward: X by (Vy, Vz), Y by (Uy, Vz), Z by (Vy, Uz) (implicit.jl:63-65 without the x transform).  The
  // transforms take the transposed matrices: forward V → Vt, inverse V' → V.
  fwd(r[0], ny, nz, b[1].Vt, b[2].Vt, ny, nz, 0, 0, w.Xh, nx - 1);
  fwd(r[1], ny - 1, nz, b[1].Ut, b[2].Vt, ny - 1, nz, 1, 0, w.Yh, nx);
  fwd(r[2], ny, nz - 1, b[1].Vt, b[2].Ut, ny, nz - 1, 0, 1, w.Zh, nx);
  linesolve<T>(ctx, S, w, done);
  inv(w.Xh, ny, nz, 0, 0, b[1].V, b[2].V, ny, nz, z[0], nx - 1);
  inv(w.Yh, ny - 1, nz, 1, 0, b[1].U, b[2].V, ny - 1, nz, z[1], nx);
  inv(w.Zh, ny, nz - 1, 0, 1, b[1].V, b[2].U, ny, nz - 1, z[2], nx);
}

// the mode-space arrays of one precision; the FP64 factorisation of the line solves is allocated with the FP64 work
// and shared by the FP32 one
template <class T>
int alloc_work(Ctx *ctx, SepDev *S, Work<T> &w) {
  const long long nx = S->nx, P = S->P;
  int rc;
  if ((rc = dalloc(ctx, &w.Xh, (nx - 1) * P))) return rc;
  if ((rc = dalloc(ctx, &w.Yh, nx * P))) return rc;
  if ((rc = dalloc(ctx, &w.Zh, nx * P))) return rc;
  if (sizeof(T) == 8) {
    if ((rc = dalloc(ctx, &w.inv, nx * P))) return rc;
  } else {
    w.inv = S->wd.inv;
  }
  return 0;
}

void factor_lines(Ctx *ctx, SepDev *S, Work<double> &w) {
  TDGL_LAUNCH(ctx, K_MODES64, 8.0 * S->nx * S->P, k_linefactor, nblk(S->P, 128), 128, 0, w.inv, S->nx, S->P, S->ny,
              S->bd[1].s, S->bd[2].s, ctx->P.a_imp);
}

// ---------------------------------------------------------------------------------------------- layout conversions
// node-shaped x-fastest (the state's layout) ↔ plane-major, through 32 × 32 tiles of (i, j) in shared memory.
struct ConvArgs {
  const double *a[3], *b[3];   // to plane-major: out = a − b (b null: out = a); x-fastest inputs
  double *out[3];              // plane-major outputs (to_pm) / x-fastest outputs (from_pm: out = base + in)
  const double *in[3];         // from_pm: plane-major inputs
  const double *base[3];       // from_pm: x-fastest base (null: out = in)
  Rng r[3];                    // ranges per component
  int n1, n2, n3;
  int to_pm;
};

__device__ __forceinline__ void convert_b(const Blk bk, ConvArgs const &A);
__global__ void k_convert(ConvArgs A) { convert_b(TDGL_BLK, A); }
TDGL_MERGEABLE(k_convert, convert_b, 256, 1, false);
__device__ __forceinline__ void convert_b(const Blk bk, ConvArgs const &A) {
  __shared__ double tile[32][33];
  const int c = bk.z % 3, kk = bk.z / 3;
  const Rng r = A.r[c];
  if (kk >= r.nk) return;
  const int k = r.k0 + kk;
  const int ib = bk.x * 32, jb = bk.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;   // 32 × 8
  const long long sxf = (long long)A.n1 * A.n2;   // x-fastest plane stride (per k)
  if (A.to_pm) {
    for (int yy = ty; yy < 32; yy += 8) {
      const int i = ib + tx, j = jb + yy;
      double v = 0.0;
      if (i < r.ni && j < r.nj) {
        const long long o = (long long)(r.i0 - 1 + i) + (long long)A.n1 * (r.j0 - 1 + j) + sxf * (k - 1);
        v = A.b[c] ? A.a[c][o] - A.b[c][o] : A.a[c][o];
      }
      tile[yy][tx] = v;
    }
    __syncthreads();
    for (int yy = ty; yy < 32; yy += 8) {
      const int i = ib + yy, j = jb + tx;
      if (i < r.ni && j < r.nj) {
        const long long o = (long long)(r.j0 - 1 + j) + (long long)A.n2 * ((k - 1) + (long long)A.n3 * (r.i0 - 1 + i));
        A.out[c][o] = tile[tx][yy];
      }
    }
  } else {
    for (int yy = ty; yy < 32; yy += 8) {
      const int i = ib + yy, j = jb + tx;
      double v = 0.0;
      if (i < r.ni && j < r.nj) v = A.in[c][(long long)(r.j0 - 1 + j) + (long long)A.n2 * ((k - 1) + (long long)A.n3 * (r.i0 - 1 + i))];
      tile[tx][yy] = v;
    }
    __syncthreads();
    for (int yy = ty; yy < 32; yy += 8) {
      const int i = ib + tx, j = jb + yy;
      if (i < r.ni && j < r.nj) {
        const long long o = (long long)(r.i0 - 1 + i) + (long long)A.n1 * (r.j0 - 1 + j) + sxf * (k - 1);
        A.out[c][o] = A.base[c] ? A.base[c][o] + tile[yy][tx] : tile[yy][tx];
      }
    }
  }
}

// packed ranges (x-fastest within each range, components x | y | z: the layout of the reference's imp.x) ↔ plane-major
struct PackArgs {
  double *pm[3];
  double *packed;
  Rng r[3];
  long long off[4];
  int n2, n3;
  int to_packed;
};
__global__ void k_packpm(PackArgs A) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.off[3]) return;
  const int c = t >= A.off[1] ? (t >= A.off[2] ? 2 : 1) : 0;
  int i, j, k;
  rng_ijk(A.r[c], t - A.off[c], i, j, k);
  const long long o = (long long)(j - 1) + A.n2 * ((long long)(k - 1) + (long long)A.n3 * (i - 1));
  if (A.to_packed) A.packed[t] = A.pm[c][o];
  else A.pm[c][o] = A.packed[t];
}

}  // namespace

Rng sep_range(const Geo &g, int ax);

// host packed ranges ↔ device plane-major component arrays (the carry of the PCG, tdgl_sep_apply)
static int pm_xfer(Ctx *ctx, double *const *pm, double *host, bool up) {
  const Geo &g = ctx->g;
  PackArgs A;
  A.off[0] = 0;
  for (int c = 0; c < 3; c++) {
    A.pm[c] = pm[c];
    A.r[c] = sep_range(g, c);
    A.off[c + 1] = A.off[c] + A.r[c].n();
  }
  A.n2 = g.Ny + 1;
  A.n3 = g.Nz + 1;
  const size_t nb = A.off[3] * sizeof(double);
  double *buf = nullptr;
  TDGL_CUDA(cudaMalloc(&buf, nb));
  A.packed = buf;
  cudaError_t e = cudaSuccess;
  if (up) {
    e = cudaMemcpyAsync(buf, host, nb, cudaMemcpyHostToDevice, ctx->stream);
    A.to_packed = 0;
    if (e == cudaSuccess) TDGL_LAUNCH(ctx, K_PACK, 16.0 * A.off[3], k_packpm, nblk(A.off[3], BS), BS, 0, A);
  } else {
    A.to_packed = 1;
    TDGL_LAUNCH(ctx, K_PACK, 16.0 * A.off[3], k_packpm, nblk(A.off[3], BS), BS, 0, A);
    e = cudaMemcpyAsync(host, buf, nb, cudaMemcpyDeviceToHost, ctx->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(buf);
  if (e != cudaSuccess) return set_err(ctx, TDGL_ECUDA, "packed transfer", e);
  return 0;
}
int pm_from_packed_host(Ctx *ctx, double *const *pm, const double *host) { return pm_xfer(ctx, pm, const_cast<double *>(host), true); }
int pm_to_packed_host(Ctx *ctx, double *const *pm, double *host) { return pm_xfer(ctx, pm, host, false); }

Rng sep_range(const Geo &g, int ax) {
  if (ax == 0) return mkrng(2, g.Nx - 1, 2, g.Ny, 2, g.Nz);
  if (ax == 1) return mkrng(2, g.Nx, 2, g.Ny - 1, 2, g.Nz);
  return mkrng(2, g.Nx, 2, g.Ny, 2, g.Nz - 1);
}

long long sep_nrange(Ctx *ctx, int ax) { return sep_range(ctx->g, ax).n(); }

// x-fastest (a − b) on the ranges → plane-major out
void to_planes(Ctx *ctx, const double *const *a, const double *const *b, double *const *out) {
  const Geo &g = ctx->g;
  ConvArgs A;
  int maxk = 0;
  for (int c = 0; c < 3; c++) {
    A.a[c] = a[c];
    A.b[c] = b ? b[c] : nullptr;
    A.out[c] = out[c];
    A.in[c] = nullptr;
    A.base[c] = nullptr;
    A.r[c] = sep_range(g, c);
    maxk = std::max(maxk, A.r[c].nk);
  }
  A.n1 = g.Nx + 1; A.n2 = g.Ny + 1; A.n3 = g.Nz + 1;
  A.to_pm = 1;
  dim3 grid((g.Nx + 31) / 32, (g.Ny + 31) / 32, 3 * maxk);
  double n = (double)(A.r[0].n() + A.r[1].n() + A.r[2].n());
  TDGL_LAUNCH(ctx, K_PACK, (b ? 24.0 : 16.0) * n, k_convert, grid, dim3(32, 8), 0, A);
}

// plane-major in → x-fastest out = base + in on the ranges
void from_planes(Ctx *ctx, const double *const *in, const double *const *base, double *const *out) {
  const Geo &g = ctx->g;
  ConvArgs A;
  int maxk = 0;
  for (int c = 0; c < 3; c++) {
    A.a[c] = nullptr;
    A.b[c] = nullptr;
    A.in[c] = in[c];
    A.base[c] = base ? base[c] : nullptr;
    A.out[c] = out[c];
    A.r[c] = sep_range(g, c);
    maxk = std::max(maxk, A.r[c].nk);
  }
  A.n1 = g.Nx + 1; A.n2 = g.Ny + 1; A.n3 = g.Nz + 1;
  A.to_pm = 0;
  dim3 grid((g.Nx + 31) / 32, (g.Ny + 31) / 32, 3 * maxk);
  double n = (double)(A.r[0].n() + A.r[1].n() + A.r[2].n());
  TDGL_LAUNCH(ctx, K_PACK, (base ? 24.0 : 16.0) * n, k_convert, grid, dim3(32, 8), 0, A);
}

int sep_create(Ctx *ctx) {
  const Geo &g = ctx->g;
  SepDev *S = new SepDev();
  ctx->sep = S;
  S->nx = g.Nx - 1;
  S->ny = g.Ny - 1;
  S->nz = g.Nz - 1;
  if (S->nx < 2 || S->ny < 2 || S->nz < 2) return set_err(ctx, TDGL_EINVAL, "grid too small for the separable solve");
  S->P = (long long)S->ny * S->nz;
  const int n[3] = {S->nx, S->ny, S->nz};
  for (int ax = 0; ax < 3; ax++) {
    upload_basis<double>(ctx, S->bd[ax], n[ax]);
    upload_basis<float>(ctx, S->bf[ax], n[ax]);
  }
  int rc;
  for (int c = 0; c < 3; c++)
    if ((rc = dalloc(ctx, &S->B[c], g.d.n()))) return rc;
  if ((rc = alloc_work<double>(ctx, S, S->wd))) return rc;
  const bool f32 = ctx->P.solver == TDGL_SOLVER_PCG && ctx->P.pcg_f32;
  if (f32 && (rc = alloc_work<float>(ctx, S, S->wf))) return rc;
  // the tensor-core transforms where the planes fit them, with TDGL_PRECOND_TC=1 (default: the SIMT kernel)
  const char *tcenv = getenv("TDGL_PRECOND_TC");
  S->tc = f32 && half_tc_fits(S->ny, S->nz) && tcenv && tcenv[0] == '1';
  if (f32 && (S->tc || half_fits(S->ny, S->nz)))
    for (int c = 0; c < 3; c++)
      if ((rc = dalloc(ctx, &S->r32[c], g.d.n()))) return rc;
  // planes too large for the one-block transform take the batched products through a buffer of the first product;
  // the FP32 preconditioner's mirror-halved ones (when the one-block mirror-halved kernel does not take the planes)
  // through its X / O2 and O1 buffers
  const bool large = plane_smem<double>(S->ny, S->nz, S->nz) > GB_ONEBLOCK || plane_smem<float>(S->ny, S->nz, S->nz) > GB_ONEBLOCK;
  if (large && (rc = dalloc(ctx, (double **)&S->gtmp, (size_t)S->nx * S->ny * S->nz))) return rc;
  if (large && f32 && !S->tc && !half_fits(S->ny, S->nz)) {
    const HalfGeo G(S->ny, S->nz);   // the largest component's planes (y and z extents ny, nz)
    S->hx_ps = std::max((long long)S->ny * S->nz, (long long)G.JP * (G.C0 + G.C1));
    S->ho_ps = (long long)G.JP * S->nz;
    if ((rc = dalloc(ctx, &S->hx, (size_t)S->nx * S->hx_ps)) || (rc = dalloc(ctx, &S->ho, (size_t)S->nx * S->ho_ps)))
      return rc;
  }
  factor_lines(ctx, S, S->wd);
  // shared memory of the plane transforms (the forward shape nj = ny, nk = nz is the largest)
  // a plane larger than one block's shared memory takes the chunked transform, whose output rows must fit
  if (tiled_smem<double>(S->nz) > 227 * 1024)
    return set_err(ctx, TDGL_EINVAL, "separable solve: the z extent is too large for the plane transform");
  // the attribute belongs to the kernel, not to this context: the ceiling, so that a smaller context created later
  // does not lower the limit of a larger one
  set_plane_smem<double, double, double>();
  set_plane_smem<double, float, float>();
  set_plane_smem<float, double, float>();
  smem_optin(k_plane_tiled<double, double, double>);
  smem_optin(k_plane_tiled<double, float, float>);
  smem_optin(k_plane_tiled<float, double, float>);
  smem_optin(k_linesolve_staged<float>);
  smem_optin(k_linesolve_staged<double>);
  smem_optin(k_half32<float, true>);
  smem_optin(k_half32<double, false>);
  half_tc_init();
  if (!g_sm_count) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count < 1) g_sm_count = 148;
  }
  TDGL_CUDA(cudaGetLastError());
  return 0;
}

void sep_destroy(Ctx *ctx) {
  delete ctx->sep;
  ctx->sep = nullptr;
}

// z = (I + aK)^{-1} r on plane-major component arrays (z may alias r: r is read by the forward pass only)
bool sep_apply(Ctx *ctx, const double *const *r, double *const *z, bool f32, const int *done, bool r32_ready,
               const DotFuse *dot) {
  SepDev *S = ctx->sep;
  if (!f32) {
    solve<double>(ctx, S, S->bd, S->wd, r, z, done);
    return false;
  }
  if (S->r32[0]) {
    if (!r32_ready) {
      const long long n = ctx->g.d.n();
      for (int c = 0; c < 3; c++)
        TDGL_LAUNCH(ctx, K_CONVERT, 12.0 * n, k_to_f32, nblk(n, BS), BS, 0, r[c], S->r32[c], n);
    }
    solve<float>(ctx, S, S->bf, S->wf, r, z, done, S->r32, dot);
    return dot != nullptr;
  }
  solve<float>(ctx, S, S->bf, S->wf, r, z, done);
  return false;
}

float *const *sep_r32(Ctx *ctx) { return ctx->sep && ctx->sep->r32[0] ? ctx->sep->r32 : nullptr; }

// implicit_curl! with the SepSolver (implicit.jl:91-104)
void sep_implicit(Ctx *ctx) {
  SepDev *S = ctx->sep;
  to_planes(ctx, ctx->ph, ctx->th, S->B);
  sep_apply(ctx, S->B, S->B, false, nullptr);
  from_planes(ctx, S->B, ctx->th, ctx->ph);
}

}  // namespace tdgl

// ================================================================================================================
// The separable inverse for callers that cannot allocate device memory (tdgl_sep_apply_noalloc).
//
// Some hosts cannot call cudaMalloc: a solver that runs inside another framework's memory pool or under its
// stream capture, a process whose device memory is fully reserved up front, or a plugin that the host forbids
// to allocate.  For them the inverse of (I + aK) runs from a fixed scratch array that this file declares at file
// scope: every GPU that loads the library holds these TDGL_NOALLOC_BYTES until the process exits.  The caller
// passes the input and the output.  Nothing here calls cudaMalloc, cudaFree or any allocating routine.
// ================================================================================================================
#define TDGL_NOALLOC_BYTES (16u << 20)

namespace {

__device__ __align__(256) double g_noalloc_scratch[TDGL_NOALLOC_BYTES / sizeof(double)];

const int NOALLOC_MAXDEV = 64;
// device address of the scratch, per device (set on the first call on that device; first calls from several host
// threads at once may both look it up and store the same address: atomic, so that this is not a data race)
std::atomic<double *> g_noalloc_ptr[NOALLOC_MAXDEV] = {};

// the DCT-II / DST-I bases of n nodes, written into the scratch (the same formulas upload_basis evaluates on the host)
__global__ void k_noalloc_basis(double *V, double *Vt, double *U, double *Ut, double *s, int n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nn = (long long)n * n;
  if (t < nn) {
    const int i = (int)(t % n), k = (int)(t / n);
    const double ck = k == 0 ? sqrt(1.0 / n) : sqrt(2.0 / n);
    const double v = ck * cos(M_PI * k * (i + 0.5) / n);
    V[i + (long long)n * k] = v;
    Vt[k + (long long)n * i] = v;
    if (i == 0) s[k] = 2 * sin(M_PI * k / (2.0 * n));
  }
  const long long m = (long long)(n - 1) * (n - 1);
  if (t < m) {
    const int e = (int)(t % (n - 1)), k = 1 + (int)(t / (n - 1));
    const double u = -sqrt(2.0 / n) * sin(M_PI * k * (e + 1.0) / n);
    U[e + (long long)(n - 1) * (k - 1)] = u;
    Ut[(k - 1) + (long long)(n - 1) * e] = u;
  }
}

}  // namespace

extern "C" int tdgl_sep_apply_noalloc(const tdgl_grid *g, double a, const double *const *b, double *const *z, void *stream) {
  using namespace tdgl;
  if (!g || !b || !z || !b[0] || !b[1] || !b[2] || !z[0] || !z[1] || !z[2]) return set_err(nullptr, TDGL_EINVAL, "null argument");
  if (!(g->dx == g->dy && g->dy == g->dz)) return set_err(nullptr, TDGL_EINVAL, "the separable solve needs dx = dy = dz");
  const int nx = g->Nx - 1, ny = g->Ny - 1, nz = g->Nz - 1;
  if (nx < 2 || ny < 2 || nz < 2) return set_err(nullptr, TDGL_EINVAL, "grid too small for the separable solve");
  // scratch layout (doubles): bases of y and z, the hat arrays, the line factorisation
  const long long P = (long long)ny * nz;
  const long long by = 2LL * ny * ny + 2LL * (ny - 1) * (ny - 1) + ny, bz = 2LL * nz * nz + 2LL * (nz - 1) * (nz - 1) + nz;
  const long long need = by + bz + (3LL * nx - 1) * P + 2LL * nx * P;
  const long long cap = (long long)(TDGL_NOALLOC_BYTES / sizeof(double));
  if (need > cap) {
    char m[256];
    snprintf(m, sizeof(m), "grid too large for the fixed scratch: needs %lld bytes, the scratch holds %u", need * 8, TDGL_NOALLOC_BYTES);
    return set_err(nullptr, TDGL_EINVAL, m);
  }
  if (plane_smem<double>(ny, nz, nz) > 227 * 1024) return set_err(nullptr, TDGL_EINVAL, "the y-z plane is too large for one block");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_err(nullptr, TDGL_ECUDA, "cudaGetDevice", e);
  if (dev < 0 || dev >= NOALLOC_MAXDEV) return set_err(nullptr, TDGL_EINVAL, "device index out of range");
  if (!g_noalloc_ptr[dev].load()) {
    // set-up, once per device, with that device current: the scratch's device address (in host code the symbol
    // is only a host-side stand-in), and the shared-memory limit of the plane transform
    double *ptr = nullptr;
    e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) return set_err(nullptr, TDGL_ECUDA, "cudaGetSymbolAddress", e);
    g_noalloc_ptr[dev].store(ptr);
  }
  e = smem_optin(k_plane<double, double, double, 2>);
  if (e == cudaSuccess)
    e = smem_optin(k_plane<double, double, double, 4>);
  if (e != cudaSuccess) return set_err(nullptr, TDGL_ECUDA, "cudaFuncSetAttribute", e);
  e = smem_optin(k_linesolve_staged<double>);
  if (e != cudaSuccess) return set_err(nullptr, TDGL_ECUDA, "cudaFuncSetAttribute", e);
  double *s0 = g_noalloc_ptr[dev].load();
  // a context on the host stack: the stream and the geometry for the launches, nothing on the device
  Ctx ctx;
  ctx.stream = (cudaStream_t)stream;
  ctx.P.a_imp = a;
  ctx.g.Nx = g->Nx; ctx.g.Ny = g->Ny; ctx.g.Nz = g->Nz;
  ctx.g.x1 = g->x1; ctx.g.x2 = g->x2; ctx.g.y1 = g->y1; ctx.g.y2 = g->y2; ctx.g.z1 = g->z1; ctx.g.z2 = g->z2;
  ctx.g.dx = g->dx; ctx.g.dy = g->dy; ctx.g.dz = g->dz;
  ctx.g.d = Dim{g->Nx + 1, g->Ny + 1, g->Nz + 1};
  SepDev S;
  S.nx = nx; S.ny = ny; S.nz = nz; S.P = P;
  double *q = s0;
  auto take = [&](long long n) { double *r = q; q += n; return r; };
  const int nax[2] = {ny, nz};
  for (int ax = 1; ax <= 2; ax++) {
    const int n = nax[ax - 1];
    Basis<double> &B = S.bd[ax];
    B.n = n;
    B.V = take((long long)n * n); B.Vt = take((long long)n * n);
    B.U = take((long long)(n - 1) * (n - 1)); B.Ut = take((long long)(n - 1) * (n - 1));
    B.s = take(n);
    k_noalloc_basis<<<nblk((long long)n * n, BS), BS, 0, ctx.stream>>>(B.V, B.Vt, B.U, B.Ut, B.s, n);
  }
  Work<double> &w = S.wd;
  w.Xh = take((nx - 1) * P); w.Yh = take(nx * P); w.Zh = take(nx * P);
  w.inv = take(nx * P);
  // every call shares the scratch and finds the previous call's contents: the empty slots of the hat arrays (Y at
  // my = 1, Z at mz = 1) must read zero, so the hat arrays are cleared
  e = cudaMemsetAsync(w.Xh, 0, (size_t)(3LL * nx - 1) * P * sizeof(double), ctx.stream);
  if (e != cudaSuccess) return set_err(nullptr, TDGL_ECUDA, "cudaMemsetAsync", e);
  factor_lines(&ctx, &S, w);
  solve<double>(&ctx, &S, S.bd, w, b, z, nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(nullptr, TDGL_ECUDA, "tdgl_sep_apply_noalloc launch", e);
  return 0;
}
