// merge.cuh — one launch of a kernel for many contexts (the merged step of a batch).
//
// A batch whose contexts' steps launch the same kernels in the same order replays the step with one launch per
// kernel for all of them.  The merged grid is the contexts' own grids laid end to end (a context's grid, flattened
// x fastest, starts at its `start`); each block finds its context by a binary search over the starts, rebuilds the
// block index and grid it has in that context's own launch (Blk), and runs the kernel's body with that context's
// parameter record.  Every thread therefore computes what it computes in the context's own launch, and each context
// gets the bits it gets alone.
//
// The records travel as the merged kernel's parameters (up to 32 KB), in its constant bank like any kernel's
// parameters: the body reads its fields there on demand, with about the registers of the plain kernel; a batch with
// more contexts than one launch holds takes several launches.
//
// A kernel takes part by splitting into a body (`void body(const Blk, const P &...)`, indexing with the Blk) and the
// plain kernel that calls it with TDGL_BLK, and by registering the pair with TDGL_MERGEABLE.
#pragma once

#include "common.cuh"

namespace tdgl {

struct MergeSeg {
  unsigned start, gx, gy, gz;
};

// The parameters of a merged launch, passed as the kernel's own (up to 32 KB of kernel parameters): n contexts, the
// first merged block of each with its own grid, and each context's parameter record.  NCAP is as many contexts as fit.
constexpr int MERGE_PARAM_BYTES = 32000;
constexpr int merge_cap(size_t argsize) { return (int)((MERGE_PARAM_BYTES - 16) / (argsize + sizeof(MergeSeg))); }
template <class Pk, int NCAP>
struct MergeParams {
  int n;
  MergeSeg seg[NCAP];
  Pk args[NCAP];
};

// the context of this block (the last segment that starts at or before it) and the block as that context sees it
__device__ __forceinline__ Blk merged_blk(const MergeSeg *seg, int n, int &c) {
  const unsigned b = blockIdx.x;
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg[mid].start <= b) lo = mid;
    else hi = mid - 1;
  }
  c = lo;
  const MergeSeg s = seg[lo];
  const unsigned r = b - s.start;
  return Blk{r % s.gx, (r / s.gx) % s.gy, r / (s.gx * s.gy), s.gx, s.gy, s.gz};
}

template <auto BODY, class... D>
__device__ __forceinline__ void argpack_call(const Blk &bk, const ArgPack<> &, const D &...d) {
  BODY(bk, d...);
}
template <auto BODY, class H, class... T, class... D>
__device__ __forceinline__ void argpack_call(const Blk &bk, const ArgPack<H, T...> &p, const D &...d) {
  argpack_call<BODY>(bk, p.t, d..., p.h);
}

// The merged form of a kernel.  The parameter block stays in the kernel's parameter space (__grid_constant__): the
// body reads its context's record there, as the plain kernel reads its own parameters.
template <auto BODY, int MAXT, int MINB, class... P>
__global__ void __launch_bounds__(MAXT, MINB)
    k_merged(const __grid_constant__ MergeParams<ArgPack<P...>, merge_cap(sizeof(ArgPack<P...>))> t) {
  int c;
  const Blk bk = merged_blk(t.seg, t.n, c);
  argpack_call<BODY>(bk, t.args[c]);
}

void merge_register(const void *kern, MergeInfo m);

template <auto BODY, int MAXT, int MINB, class... P>
MergeInfo merge_info(void (*)(P...), bool stride_x) {
  using Pk = ArgPack<P...>;
  constexpr int cap = merge_cap(sizeof(Pk));
  static_assert(cap >= 8, "kernel parameters too large to merge");
  using MP = MergeParams<Pk, cap>;
  MergeInfo m;
  m.merged = (const void *)k_merged<BODY, MAXT, MINB, P...>;
  m.argsize = sizeof(Pk);
  m.stride_x = stride_x;
  m.cap = cap;
  m.off_seg = offsetof(MP, seg);
  m.off_args = offsetof(MP, args);
  m.param_bytes = sizeof(MP);
  return m;
}

struct MergeReg {
  MergeReg(const void *kern, MergeInfo m) { merge_register(kern, m); }
};

#define TDGL_MCAT2(a, b) a##b
#define TDGL_MCAT(a, b) TDGL_MCAT2(a, b)
// registers kernel K (plain form) with its body; MAXT, MINB: the launch bounds of the merged form; STRIDE_X: the
// body strides over blk.x (its x-grid may be resized)
#define TDGL_MERGEABLE(K, BODY, MAXT, MINB, STRIDE_X)                                              \
  static const tdgl::MergeReg TDGL_MCAT(tdgl_merge_reg_, __LINE__)((const void *)(K),              \
                                                                   tdgl::merge_info<BODY, MAXT, MINB>((K), (STRIDE_X)))

}  // namespace tdgl
