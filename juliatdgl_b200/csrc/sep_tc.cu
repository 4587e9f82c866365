// sep_tc.cu — the FP32 preconditioner's plane transforms on the fifth-generation tensor cores (tcgen05, kind::tf32,
// three passes: hi·hi + hi·lo + lo·hi, about the accuracy of FP32 multiply-adds).  The same operator as the SIMT
// kernel k_half32 (sep.cu) and the reference's SGEMMs (gtdgl/src/implicit.jl:346-373): per x-plane, the y and z
// transforms of the mirror-halved DCT-II / DST-I bases; the sums round differently.
//
// Per plane (n1 × n2 points, mirror classes S and D along each axis: hS = ⌈n/2⌉, hD = ⌊n/2⌋):
//   prologue  the plane is paired (forward) or gathered by mode class (inverse) into X̃, split into TF32 hi and lo,
//             and stored as the B operand of the y product: per y class a, [z column n in class order][y index k];
//   y product D_a = W1_aᵀ X̃_a        (M 128 ≥ hS1 output rows, N = 2·K2 z columns, K = K1; 2 classes × 3 passes),
//             into tensor memory; rows beyond the class's size are never used;
//   split     D → D_hi, D_lo in tensor memory (the A operand of the z product, read from tensor memory);
//   z product Y_ab = D_a[:, class b] W2_b (M 128, N = NZ, K = K2; 4 blocks × 3 passes);
//   epilogue  Y is scattered to mode order (forward, FP32) or unpaired into points (inverse, FP64, with the PCG's
//             r·z and r·z_old folded in as in k_half32).
// One persistent block per SM (one component per block, a contiguous range of its planes); X̃ is double-buffered so
// the next plane's prologue runs while the tensor cores take the y product of this one.  Tensor-memory columns:
// D at 0, D_hi at 128, D_lo at 256, Y at 384 (512 allocated).
//
// Shared memory (bytes): the four y images (K1 rows each), the four z images (NZ rows each), then 2 × 4 X̃ images
// (2·K2 rows each); every operand row group is SBO = 32·K bytes.  The y product reads 128 rows of A: the rows past
// the image fall on later images or buffers of this block (the layout reserves enough), and only feed rows of D and
// Y that are never read.  Every wait on the tensor cores is bounded: a block whose wait runs out counts itself in
// `err`, waits (bounded) for its MMAs, releases its tensor memory and leaves.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sep.cuh"
#include "umma.cuh"

namespace tdgl {

void tc_images(int np, const double *B, int ldB, std::vector<float> &fwd, std::vector<float> &inv) {
  const int hS = (np + 1) / 2, hD = np / 2, K = rup8(hS), R = rup16(hS);
  const size_t img = (size_t)R * K;
  fwd.assign(4 * img, 0.f);
  inv.assign(4 * img, 0.f);
  auto rnd = [](float f) {   // to TF32, nearest (ties away), as umma::round_tf32
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u = (u + 0x1000u) & 0xFFFFE000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
  };
  auto split = [&](double x, float &hi, float &lo) {
    const float f = (float)x;
    hi = rnd(f);
    lo = rnd(f - hi);
  };
  for (int a = 0; a < 2; a++) {
    const int h = a ? hD : hS;
    for (int o = 0; o < h; o++)
      for (int i = 0; i < h; i++) {
        const size_t at = (size_t)(o % 8) * 4 + (size_t)(o / 8) * 8 * K + (i % 4) + (size_t)(i / 4) * 32;
        float hi, lo;
        split(B[i + (size_t)ldB * (2 * o + a)], hi, lo);   // forward: input point i, output mode 2o + a
        fwd[(2 * a) * img + at] = hi;
        fwd[(2 * a + 1) * img + at] = lo;
        split(B[o + (size_t)ldB * (2 * i + a)], hi, lo);   // inverse: output point o, input mode 2i + a
        inv[(2 * a) * img + at] = hi;
        inv[(2 * a + 1) * img + at] = lo;
      }
  }
}

namespace {

const int TC_THREADS = 256, TC_WAIT = 1 << 20;

struct TcLayout {
  int hS1, hD1, hS2, hD2, K1, K2, NZ, NY, sbo1, sbo2, img1, img2, imgx, gimg1, off_w2, off_x, end;
  __host__ __device__ TcLayout(int n1, int n2) {
    hS1 = (n1 + 1) / 2; hD1 = n1 / 2; hS2 = (n2 + 1) / 2; hD2 = n2 / 2;
    K1 = rup8(hS1); K2 = rup8(hS2); NZ = rup16(hS2); NY = 2 * K2;
    sbo1 = 32 * K1; sbo2 = 32 * K2;
    img1 = (K1 / 8) * sbo1;          // a y image in shared memory (its first K1 rows)
    gimg1 = 4 * rup16(hS1) * K1;     // a y image in global memory (R rows)
    img2 = (NZ / 8) * sbo2;          // a z image (NZ rows)
    imgx = (NY / 8) * sbo1;          // an X̃ image
    off_w2 = 4 * img1; off_x = off_w2 + 4 * img2; end = off_x + 8 * imgx;
    const int over = 3 * img1 + 16 * sbo1;   // the last y image read as 128 rows
    if (end < over) end = over;
  }
};

__device__ __forceinline__ void cp16(void *smem, const void *g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(g)
               : "memory");
}
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// four consecutive k of one row n of an image pair (hi, lo)
__device__ __forceinline__ void put4(unsigned char *hi, unsigned char *lo, const float (&v)[4]) {
  float h[4], l[4];
#pragma unroll
  for (int t = 0; t < 4; t++) umma::split_tf32(v[t], h[t], l[t]);
  *reinterpret_cast<float4 *>(hi) = make_float4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<float4 *>(lo) = make_float4(l[0], l[1], l[2], l[3]);
}

struct TcSplit {
  int cta0[4];      // blocks [cta0[c], cta0[c+1]) take component c
  long long *err;   // blocks whose tensor-core waits ran out (null: not counted)
};

template <class TOut, bool FWD>
__global__ void __launch_bounds__(TC_THREADS, 1) k_half_tc(HalfMulti M, TcSplit T) {
  if (M.done && *M.done) return;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint32_t tslot;
  __shared__ __align__(8) uint64_t bars[3];
  __shared__ double shred[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, quarter = warp & 3, half = warp >> 2;
  int ci = 0;
  while (ci + 1 < M.ncomp && (int)blockIdx.x >= T.cta0[ci + 1]) ci++;
  const HalfArgs &A = M.c[ci];
  const int nb = T.cta0[ci + 1] - T.cta0[ci], bi = (int)blockIdx.x - T.cta0[ci];
  const int q0 = (int)((long long)A.nplanes * bi / nb), q1 = (int)((long long)A.nplanes * (bi + 1) / nb);
  const int cnt = q1 - q0;
  double dz = 0.0, dzo = 0.0;   // r·z and r·z_old over this thread's written points (inverse with M.dot)
  if (cnt > 0) {
    const TcLayout L(A.n1, A.n2);
    const int n1 = A.n1, n2 = A.n2;
    const uint32_t sb = umma::saddr(smraw);
    const uint32_t bar_y = umma::saddr(&bars[0]), bar_z = umma::saddr(&bars[1]), bar_f = umma::saddr(&bars[2]);
    // the X̃ buffers start zero (their pads are never written); the basis images come in by cp.async
    {
      float4 *x4 = reinterpret_cast<float4 *>(smraw + L.off_x);
      for (int t = tid; t < 8 * L.imgx / 16; t += TC_THREADS) x4[t] = make_float4(0.f, 0.f, 0.f, 0.f);
      const int c1 = L.img1 / 16, c2 = L.img2 / 16;
      for (int t = tid; t < 4 * c1; t += TC_THREADS)
        cp16(smraw + (size_t)(t / c1) * L.img1 + 16 * (t % c1),
             reinterpret_cast<const unsigned char *>(A.T1) + (size_t)(t / c1) * L.gimg1 + 16 * (t % c1));
      for (int t = tid; t < 4 * c2; t += TC_THREADS)
        cp16(smraw + L.off_w2 + 16 * (size_t)t, reinterpret_cast<const unsigned char *>(A.T2) + 16 * (size_t)t);
    }
    if (tid == 0) {
      umma::mbar_init(bar_y, 1);
      umma::mbar_init(bar_z, 1);
      umma::mbar_init(bar_f, 1);
    }
    if (warp == 0) umma::tmem_alloc(umma::saddr(&tslot), 512);

    const int NP4 = (L.hS1 + 3) / 4, NQG = (L.hS2 + 7) / 8;
    const int ntask = 8 * NP4 * NQG;
    // one task: a group of four k (y) of one z column qc; lanes 8t..8t+7 take eight consecutive z columns of one
    // group: 128 contiguous bytes per store.  Its 16 loads land in v (zero outside the plane).
    auto task_load = [&](const float *in, long long ld, int u, float (&v)[16]) {
      const int l8 = u & 7, rest = u >> 3, p4 = rest % NP4, qc = 8 * (rest / NP4) + l8;
      const bool live = u < ntask && qc < L.hS2;
      if (FWD) {   // points (p, qc), (p', qc), (p, qc'), (p', qc') of each p (p' = n1−1−p, qc' = n2−1−qc)
        const int qq = n2 - 1 - qc;
        const bool cp = qq != qc;
#pragma unroll
        for (int t = 0; t < 4; t++) {
          const int p = 4 * p4 + t, pp = n1 - 1 - p;
          const bool ok = live && p < L.hS1, rp = ok && pp != p;
          v[4 * t] = ok ? in[p + ld * qc] : 0.f;
          v[4 * t + 1] = rp ? in[pp + ld * qc] : 0.f;
          v[4 * t + 2] = ok && cp ? in[p + ld * qq] : 0.f;
          v[4 * t + 3] = rp && cp ? in[pp + ld * qq] : 0.f;
        }
      } else {     // modes (2p + a, 2qc + b) of the four classes (a, b)
        const bool cD = qc < L.hD2;
        const float *r0 = in + ld * (2 * qc), *r1 = in + ld * (2 * qc + 1);
#pragma unroll
        for (int t = 0; t < 4; t++) {
          const int p = 4 * p4 + t;
          const bool rS = live && p < L.hS1, rD = live && p < L.hD1;
          v[4 * t] = rS ? r0[2 * p] : 0.f;
          v[4 * t + 1] = rD ? r0[2 * p + 1] : 0.f;
          v[4 * t + 2] = rS && cD ? r1[2 * p] : 0.f;
          v[4 * t + 3] = rD && cD ? r1[2 * p + 1] : 0.f;
        }
      }
    };
    auto task_store = [&](unsigned char *X, int u, const float (&v)[16]) {   // X: images [a][hi, lo] at (2a+hl)·imgx
      const int l8 = u & 7, rest = u >> 3, p4 = rest % NP4, qc = 8 * (rest / NP4) + l8;
      if (u >= ntask || qc >= L.hS2) return;
      const int nS = qc, nD = L.K2 + qc;
      const int oS = (nS % 8) * 16 + (nS / 8) * L.sbo1 + p4 * 128, oD = (nD % 8) * 16 + (nD / 8) * L.sbo1 + p4 * 128;
      float ss[4], sd[4], ds[4], dd[4];
      bool wD;   // the z class D column exists
      if (FWD) {   // the mirror quadrant into its four class entries
        const bool cp = n2 - 1 - qc != qc;
        wD = cp;
#pragma unroll
        for (int t = 0; t < 4; t++) {
          const int p = 4 * p4 + t;
          const bool rp = p < L.hS1 && n1 - 1 - p != p;
          const float a = v[4 * t], b = v[4 * t + 1], c = v[4 * t + 2], d = v[4 * t + 3];
          const float s0 = a + c, s1 = b + d, d0 = a - c, d1 = b - d;
          ss[t] = s0 + s1;
          sd[t] = cp ? d0 + d1 : 0.f;
          ds[t] = rp ? s0 - s1 : 0.f;
          dd[t] = rp && cp ? d0 - d1 : 0.f;
        }
      } else {
        wD = qc < L.hD2;
#pragma unroll
        for (int t = 0; t < 4; t++) {
          ss[t] = v[4 * t];
          ds[t] = v[4 * t + 1];
          sd[t] = v[4 * t + 2];
          dd[t] = v[4 * t + 3];
        }
      }
      put4(X + oS, X + L.imgx + oS, ss);
      put4(X + 2 * L.imgx + oS, X + 3 * L.imgx + oS, ds);
      if (wD) {
        put4(X + oD, X + L.imgx + oD, sd);
        put4(X + 2 * L.imgx + oD, X + 3 * L.imgx + oD, dd);
      }
    };
    auto plane_in = [&](int q) {
      return A.in + A.in_base + (long long)q * A.in_ps + A.in_j0 + (long long)A.in_ld * A.in_k0;
    };
    // plane q into X̃ buffer buf from task u0 on (the loads of two tasks go out together)
    auto prologue = [&](int q, int buf, int from) {
      unsigned char *X = smraw + L.off_x + (size_t)buf * 4 * L.imgx;
      const float *in = plane_in(q);
      for (int u0 = from; u0 < ntask; u0 += 2 * TC_THREADS) {
        float v0[16], v1[16];
        task_load(in, A.in_ld, u0, v0);
        task_load(in, A.in_ld, u0 + TC_THREADS, v1);
        task_store(X, u0, v0);
        task_store(X, u0 + TC_THREADS, v1);
      }
    };
    auto issue_y = [&](uint32_t tm, int buf) {   // D_a = W1_a X̃_a for both y classes (one thread)
      // the two classes' chains interleaved: independent accumulators keep the tensor pipe busy
      const uint32_t id = umma::idesc_tf32(128, L.NY), xb = sb + L.off_x + (uint32_t)(buf * 4 * L.imgx);
      const int ks[2] = {(L.hS1 + 7) / 8, (L.hD1 + 7) / 8};
      for (int pass = 0; pass < 3; pass++) {
        const int ah = pass == 2, bh = pass == 1;   // (hi, hi), (hi, lo), (lo, hi)
        for (int s = 0; s < ks[0]; s++)
          for (int a = 0; a < 2; a++)
            if (s < ks[a])
              umma::mma_ss(tm + a * L.NY, umma::sdesc(sb + (2 * a + ah) * L.img1 + 256 * s, 128, L.sbo1),
                           umma::sdesc(xb + (2 * a + bh) * L.imgx + 256 * s, 128, L.sbo1), id, (pass | s) ? 1u : 0u);
      }
    };
    auto issue_z = [&](uint32_t tm) {   // Y_ab = D_a[:, class b] W2_b (A from tensor memory), four chains interleaved
      const uint32_t id = umma::idesc_tf32(128, L.NZ);
      const int ks[2] = {(L.hS2 + 7) / 8, (L.hD2 + 7) / 8};
      for (int pass = 0; pass < 3; pass++) {
        const int ah = pass == 2, bh = pass == 1;
        for (int s = 0; s < ks[0]; s++)
          for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++)
              if (s < ks[b])
                umma::mma_ts(tm + 384 + (2 * a + b) * L.NZ, tm + (ah ? 256 : 128) + a * L.NY + b * L.K2 + 8 * s,
                             umma::sdesc(sb + L.off_w2 + (2 * b + bh) * L.img2 + 256 * s, 128, L.sbo2), id,
                             (pass | s) ? 1u : 0u);
      }
    };

    // the first two planes go in before the loop; plane i + 2's loads are issued right after plane i's MMAs and
    // land in X̃ after plane i's epilogue (the buffer of plane i, free once its y product is done)
    prologue(q0, 0, tid);
    if (cnt > 1) prologue(q0 + 1, 1, tid);
    cp_wait();
    umma::fence_smem_async();
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tm = tslot;
    const uint32_t lq = (uint32_t)(32 * quarter) << 16;
    const bool rows = 32 * quarter < L.hS1;   // this warp's lanes hold rows of D and Y
    if (tid == 0) {
      issue_y(tm, 0);
      umma::commit(bar_y);
    }
    bool ok = true;
    for (int i = 0; i < cnt; i++) {
      const int q = q0 + i, buf = i & 1;
      ok = umma::mbar_wait(bar_y, i & 1, TC_WAIT);
      ok = __syncthreads_and(ok);
      if (!ok) break;
      umma::fence_after();
      if (rows)   // D → D_hi, D_lo (half h of the block takes y class h), two column chunks per TMEM wait
        for (int c = half * L.NY; c < (half + 1) * L.NY; c += 32) {
          const bool two = c + 16 < (half + 1) * L.NY;
          float v[16], w[16], h[16], l[16];
          umma::ld16(tm + lq + c, v);
          if (two) umma::ld16(tm + lq + c + 16, w);
          umma::ld_wait();
#pragma unroll
          for (int t = 0; t < 16; t++) umma::split_tf32(v[t], h[t], l[t]);
          umma::st16(tm + lq + 128 + c, h);
          umma::st16(tm + lq + 256 + c, l);
          if (two) {
#pragma unroll
            for (int t = 0; t < 16; t++) umma::split_tf32(w[t], h[t], l[t]);
            umma::st16(tm + lq + 128 + c + 16, h);
            umma::st16(tm + lq + 256 + c + 16, l);
          }
        }
      umma::st_wait();
      umma::fence_smem_async();   // plane i + 1's X̃ (stored last iteration) before its y product
      umma::fence_before();
      __syncthreads();
      umma::fence_after();
      if (tid == 0) {
        issue_z(tm);
        umma::commit(bar_z);
        if (i + 1 < cnt) {
          issue_y(tm, buf ^ 1);
          umma::commit(bar_y);
        }
      }
      const bool ahead = i + 2 < cnt;
      float pv0[16], pv1[16];   // plane i + 2: the first two tasks of this thread, in flight during the epilogue
      if (ahead) {
        task_load(plane_in(q + 2), A.in_ld, tid, pv0);
        task_load(plane_in(q + 2), A.in_ld, tid + TC_THREADS, pv1);
      }
      ok = umma::mbar_wait(bar_z, i & 1, TC_WAIT);
      ok = __syncthreads_and(ok);
      if (!ok) break;
      umma::fence_after();
      TOut *out = (TOut *)A.out + A.out_base + (long long)q * A.out_ps + A.out_j0 + (long long)A.out_ld * A.out_k0;
      const long long ldo = A.out_ld;
      const int p = 32 * quarter + lane;
      if (FWD) {   // modes (2p + a, 2qc + b); half h of the block takes z class b = h
        const int b = half, h2 = b ? L.hD2 : L.hS2;
        if (rows)
          for (int c0 = 0; c0 < h2; c0 += 16) {
            float vs[16], vd[16];
            umma::ld16(tm + lq + 384 + b * L.NZ + c0, vs);
            umma::ld16(tm + lq + 384 + (2 + b) * L.NZ + c0, vd);
            umma::ld_wait();
#pragma unroll
            for (int t = 0; t < 16; t++) {
              const int qc = c0 + t;
              if (qc >= h2) break;
              TOut *o = out + ldo * (2 * qc + b) + 2 * p;
              if (p < L.hS1) o[0] = (TOut)vs[t];
              if (p < L.hD1) o[1] = (TOut)vd[t];
            }
          }
      } else {     // points: the four class entries of (p, qc) unpaired into the mirror quadrant
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
        const int pp = n1 - 1 - p;
        const bool pin = p < L.hS1, rp = pin && pp != p;
        if (rows)
          for (int c0 = 16 * half; c0 < L.hS2; c0 += 32) {
            float ee[16], eo[16], oe[16], oo[16];
            umma::ld16(tm + lq + 384 + 0 * L.NZ + c0, ee);
            umma::ld16(tm + lq + 384 + 1 * L.NZ + c0, eo);
            umma::ld16(tm + lq + 384 + 2 * L.NZ + c0, oe);
            umma::ld16(tm + lq + 384 + 3 * L.NZ + c0, oo);
            umma::ld_wait();
            if (pin)
#pragma unroll
              for (int t = 0; t < 16; t++) {
                const int qc = c0 + t, qq = n2 - 1 - qc;
                if (qc >= L.hS2) break;
                const bool cp = qq != qc;
                const float e0 = ee[t], e1 = cp ? eo[t] : 0.f, o0 = rp ? oe[t] : 0.f, o1 = rp && cp ? oo[t] : 0.f;
                const float s0 = e0 + o0, s1 = e1 + o1, d0 = e0 - o0, d1 = e1 - o1;
                const long long oq = ldo * qc, oqq = ldo * qq;
                put(oq + p, s0 + s1);
                if (rp) put(oq + pp, d0 + d1);
                if (cp) {
                  put(oqq + p, s0 - s1);
                  if (rp) put(oqq + pp, d0 - d1);
                }
              }
          }
      }
      if (ahead) {   // plane i + 2 into this plane's X̃ buffer (its y product is done)
        unsigned char *X = smraw + L.off_x + (size_t)buf * 4 * L.imgx;
        task_store(X, tid, pv0);
        task_store(X, tid + TC_THREADS, pv1);
        prologue(q + 2, buf, tid + 2 * TC_THREADS);
      }
      umma::fence_before();
    }
    if (!ok) {   // a wait ran out: count it, let this block's MMAs finish (bounded), then release
      if (tid == 0) {
        if (T.err) atomicAdd((unsigned long long *)T.err, 1ull);
        umma::commit(bar_f);
      }
      umma::mbar_wait(bar_f, 0, TC_WAIT);
    }
    umma::fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_free(tm, 512);
  }
  if (!FWD && M.dot) {   // the block's partial sums, folded by the last block (pcg.cuh)
    __syncthreads();
    const double a = block_sum(dz, shred);
    __syncthreads();
    const double b = block_sum(dzo, shred);
    if (tid == 0) {
      M.df.part[blockIdx.x] = a;
      M.df.part[gridDim.x + blockIdx.x] = b;
    }
    __syncthreads();
    fold_last(M.df.F, M.df.part, shred);
  }
}

size_t tc_smem(int n1, int n2) { return (size_t)TcLayout(n1, n2).end; }

}  // namespace

bool half_tc_fits(int n1, int n2) {
  if (n1 < 2 || n2 < 2) return false;
  const TcLayout L(n1, n2);
  // 128 tensor-memory lanes hold a y class; the z classes' D and Y blocks fit their column ranges
  return L.hS1 <= 128 && 2 * L.NY <= 128 && 4 * L.NZ <= 128 && tc_smem(n1, n2) + 1024 <= 227 * 1024;
}

void half_tc_init() {
  smem_optin(k_half_tc<float, true>);
  smem_optin(k_half_tc<double, false>);
}

void half_tc(Ctx *ctx, const HalfMulti &M, bool fwd, long long *err) {
  const int nsm = g_sm_count > 0 ? g_sm_count : 148;
  long long tot = 0;
  size_t smem = 0;
  double bytes = 0;
  for (int c = 0; c < M.ncomp; c++) {
    const HalfArgs &A = M.c[c];
    tot += A.nplanes;
    smem = std::max(smem, tc_smem(A.n1, A.n2));
    bytes += (double)A.nplanes * A.n1 * A.n2 * (fwd ? 2 * sizeof(float) : sizeof(float) + sizeof(double));
  }
  if (tot <= 0) return;
  // blocks per component in proportion to its planes, at least one each
  TcSplit T;
  T.err = err;
  const long long G = std::min<long long>(nsm, tot);
  int at = 0;
  for (int c = 0; c < 3; c++) {
    T.cta0[c] = at;
    if (c < M.ncomp && M.c[c].nplanes > 0)
      at += (int)std::max<long long>(1, std::min<long long>(M.c[c].nplanes, G * M.c[c].nplanes / tot));
  }
  T.cta0[3] = at;
  if (fwd) TDGL_LAUNCH(ctx, K_TX32, bytes, (k_half_tc<float, true>), at, TC_THREADS, smem, M, T);
  else TDGL_LAUNCH(ctx, K_TX32I, bytes, (k_half_tc<double, false>), at, TC_THREADS, smem, M, T);
}

}  // namespace tdgl
