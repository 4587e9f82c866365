// common.cuh — device helpers and the context of the B200 stepper.
//
// The library is compiled with --fmad=false: the stencils keep the reference's IEEE operation order (no FMA
// contraction), so that they agree with gtdgl's CPU step to rounding of the transcendental functions only.
// Kernels that may contract (the dense line transforms of the separable solve) call fma() explicitly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/tdgl_b200.h"

typedef double2 cd;

__host__ __device__ __forceinline__ cd mkc(double r, double i) { return make_double2(r, i); }
__device__ __forceinline__ cd cadd(cd a, cd b) { return mkc(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cd csub(cd a, cd b) { return mkc(a.x - b.x, a.y - b.y); }
// Julia's Complex * Complex: (ar*br - ai*bi, ar*bi + ai*br)
__device__ __forceinline__ cd cmul(cd a, cd b) { return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ cd rmul(double s, cd a) { return mkc(s * a.x, s * a.y); }
__device__ __forceinline__ cd mulr(cd a, double s) { return mkc(a.x * s, a.y * s); }
__device__ __forceinline__ cd cdivr(cd a, double s) { return mkc(a.x / s, a.y / s); }
__device__ __forceinline__ cd cconj(cd a) { return mkc(a.x, -a.y); }
__device__ __forceinline__ double cabs2(cd a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ cd ccis(double x) {
  double s, c;
  sincos(x, &s, &c);
  return mkc(c, s);
}
__device__ __forceinline__ double cangle(cd a) { return atan2(a.y, a.x); }
// e^{ia} with the short series while |a| <= 0.05 (gtdgl/src/bands.jl:289)
__device__ __forceinline__ cd ccis_short(double a) {
  if (fabs(a) <= 0.05) {
    double a2 = a * a;
    return mkc(1 - a2 / 2, a * (1 - a2 / 6));
  }
  return ccis(a);
}
// C - im*(x)*y, with Julia's Complex{Bool}·Real product (±0, x) (gtdgl/src/bands.jl:221, :283)
__device__ __forceinline__ cd cminus_i(cd c, double x, cd y) {
  return mkc(c.x - (0.0 * y.x - x * y.y), c.y - (0.0 * y.y + x * y.x));
}

// A 3D index range, 1-based inclusive as in the reference; ni etc. are its extents.
struct Rng {
  int i0, j0, k0, ni, nj, nk;
  __host__ __device__ long long n() const { return (long long)ni * nj * nk; }
};
__host__ inline Rng mkrng(int i0, int i1, int j0, int j1, int k0, int k1) {
  Rng r;
  r.i0 = i0; r.j0 = j0; r.k0 = k0;
  r.ni = i1 >= i0 ? i1 - i0 + 1 : 0;
  r.nj = j1 >= j0 ? j1 - j0 + 1 : 0;
  r.nk = k1 >= k0 ? k1 - k0 + 1 : 0;
  return r;
}
// The point t of range r.  32-bit division (a 64-bit one is a long software sequence): every range of a context
// holds fewer than 2^31 points, which the context checks at creation.
__device__ __forceinline__ void rng_ijk(const Rng &r, long long t, int &i, int &j, int &k) {
  const unsigned u = (unsigned)t, ni = (unsigned)r.ni, nj = (unsigned)r.nj;
  const unsigned b = u / ni, c = b / nj;
  i = r.i0 + (int)(u - b * ni);
  j = r.j0 + (int)(b - c * nj);
  k = r.k0 + (int)c;
}

// Dimensions of a column-major 3D array; at(i,j,k) takes the reference's 1-based indices.
struct Dim {
  int n1, n2, n3;
  __host__ __device__ long long at(int i, int j, int k) const {
    return (long long)(i - 1) + (long long)n1 * ((long long)(j - 1) + (long long)n2 * (k - 1));
  }
  __host__ __device__ long long n() const { return (long long)n1 * n2 * n3; }
};

// Every device array (nodes, links, plaquettes) is stored with the node shape (Nx+1, Ny+1, Nz+1), so that one
// offset formula serves all of them; the reference's smaller link / plaquette shapes are the leading corner.
struct Geo {
  int Nx, Ny, Nz, x1, x2, y1, y2, z1, z2;
  double dx, dy, dz;
  Dim d;
};

struct BandPtrs {
  const cd *p[TDGL_MAXB];
};

// The block a thread works on, as its own launch sees it (blockIdx, gridDim): the hardware's in a plain launch, one
// context's share of the grid in a merged launch (merge.cuh).  Kernel bodies index with it instead of blockIdx.
struct Blk {
  unsigned x, y, z, nx, ny, nz;
};
#define TDGL_BLK (Blk{blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y, gridDim.z})

// A kernel's parameters as one trivially copyable record (the first in h, the rest in t), so that the parameters of
// many launches can sit side by side.
template <class... P>
struct ArgPack;
template <>
struct ArgPack<> {};
template <class H, class... T>
struct ArgPack<H, T...> {
  H h;
  ArgPack<T...> t;
};
inline void argpack_set(ArgPack<> &) {}
template <class H, class... T, class A, class... B>
void argpack_set(ArgPack<H, T...> &p, A &&a, B &&...b) {
  p.h = static_cast<H>(a);
  argpack_set(p.t, static_cast<B &&>(b)...);
}

// ------------------------------------------------------------------------------------------ launch helpers
static inline unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

#define TDGL_CUDA(call)                                                         \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) return tdgl::set_err(ctx, TDGL_ECUDA, #call, e_);    \
  } while (0)

namespace tdgl {

// Kernel categories of the per-launch profiler (tdgl_profile): CUDA events around every launch, with the
// algorithmic (compulsory) bytes of that launch, so that a driver can report achieved bandwidth per kernel.
enum KCat {
  K_BAND = 0, K_LINK, K_GHOST, K_OMEGA, K_CURINC, K_LINKSCURL, K_FACEH, K_ADVANCE, K_SCALE, K_TX64, K_MODES64,
  K_TX32, K_MODES32, K_CONVERT, K_PCG_START, K_PCG_H, K_PCG_Q, K_PCG_RES, K_PCG_UPD, K_PCG_DOT, K_PCG_FINAL,
  K_PCG_DIR, K_PCG_EXTRAP, K_PACK, K_OPEN_FFT, K_OPEN_MISC, K_COPY, K_METER, K_NOISE, K_TX32I, K_HEAT, K_PCG_XUPD, K_PCG_DOTS, K_QP, K_NCAT
};
extern const char *kcat_name[K_NCAT];

struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  struct Rec {
    int cat;
    cudaEvent_t a, b;
    double bytes;
  };
  std::vector<Rec> pend;
  double ms[K_NCAT] = {};
  double bytes[K_NCAT] = {};
  long long n[K_NCAT] = {};
};

// Material per region on the device (materials.jl): the tables each node reads through its material index.  The
// link weight of band µ along axis ax between materials a and b is ρ = τ·W[µ][ax][a][b], W = (m_ref/m_link)·t_ab
// (0 where the band is absent at either end), formed from the node map instead of stored per link.
struct MatDev {
  tdgl_bandcoef full[TDGL_MAXB][TDGL_MAXMAT], stage[TDGL_MAXB][TDGL_MAXMAT];
  double W[TDGL_MAXB][3][TDGL_MAXMAT][TDGL_MAXMAT];
  double gam[TDGL_MAXB][TDGL_MAXMAT];   // Γ (the noise kick)
  double a[TDGL_MAXB][TDGL_MAXMAT];     // a of each band (ε = a − θ with the heat model)
  int absent[TDGL_MAXB][TDGL_MAXMAT];
};

// The values that change from one step to the next, read by the kernels from device memory (one copy per step
// from pinned host memory), so that a step captured in a CUDA graph replays with the next step's values.
struct StepScal {
  double H, HJ;                 // applied field, self-field factor (field_bc!)
  double open_fr;               // the open boundary's ramp fraction (openbc.jl:210-223)
  unsigned long long noise_step;   // the noise stream's step index
};

// the heat model's per-material values (tdgl_materials, ABI v7), kept by the context
struct HeatMat {
  int nmat = 0;
  double G[TDGL_MAXMAT][TDGL_MAXB] = {}, gk[TDGL_MAXMAT][TDGL_MAXB] = {};
  double sig[TDGL_MAXMAT] = {}, DT[TDGL_MAXMAT] = {};
};

struct SepDev;
struct PcgDev;
struct OpenDev;
struct MeterDev;
struct QpDev;

// What a merged launch needs of a kernel (merge.cuh): its merged form, the size of its parameter record, whether
// its blocks stride over x (`for (q = blk.x; q < n; q += blk.nx)`, so that its x-grid may be resized), and the
// layout of the merged form's parameter block.
struct MergeInfo {
  const void *merged;
  size_t argsize;
  bool stride_x;
  int cap;                                  // contexts per merged launch
  size_t off_seg, off_args, param_bytes;    // layout of its parameter block (merge.cuh: MergeParams)
};
const MergeInfo *merge_lookup(const void *kern);

// The kernel launches of one captured step of a context, as a batch records them to merge them with the other
// contexts' (ok: every launch was of a kernel that has a merged form).
struct TapeRec {
  const void *kern;
  const MergeInfo *m;
  dim3 grid, block;
  size_t smem;
  std::vector<unsigned char> args;
};
struct Tape {
  bool ok = true;
  std::vector<TapeRec> recs;
};

struct Ctx {
  tdgl_params P;
  int N;
  Geo g;
  cudaStream_t stream = nullptr;
  std::string err;
  // coefficient tables
  double *f = nullptr, *tau[3] = {nullptr, nullptr, nullptr};
  double *D[3] = {nullptr, nullptr, nullptr};
  double *bar[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  double *jbar = nullptr;
  // state
  cd *G[TDGL_MAXB] = {}, *F[TDGL_MAXB] = {};
  double *th[3] = {}, *ph[3] = {}, *J[3] = {}, *h[3] = {};
  cd *U[3] = {}, *V[3] = {};
  bool have_state = false;
  // workspaces of the band stages
  cd *W = nullptr, *W2 = nullptr, *L[3] = {}, *Rl[3] = {};
  double *Th = nullptr;   // the heat model's temperature field (node-shaped; terms.jl)
  double *Th2 = nullptr;  // with D_T per material: the field of the step before (the Jacobi update)
  HeatMat hm;             // with materials: each material's Γ, γ̃, σn and D_T for the heat step
  double *drag_c = nullptr, *drag_nu = nullptr;   // the interband drag's tables ([MAXB][MAXB][3], [MAXB][MAXB])
  double *Om = nullptr, *Oms = nullptr, *Rr[3] = {};   // Oms: the copy of the frame-rate smoothing (noise)
  // The bands of a step are updated concurrently: each reads only the state at the start of the step and writes its
  // own F[µ], so band µ ≥ 1 runs on bstream[µ] (band 0 on the context's stream) with its own stage workspaces
  // (bws[µ]; the fields above point at the workspaces of the band being launched).
  struct BandWs {
    cd *W = nullptr, *W2 = nullptr, *L[3] = {}, *Rl[3] = {};
    double *Om = nullptr, *Oms = nullptr, *Rr[3] = {};
  };
  BandWs bws[TDGL_MAXB];
  cudaStream_t bstream[TDGL_MAXB] = {};
  cudaEvent_t bev[TDGL_MAXB] = {};
  // solvers
  SepDev *sep = nullptr;
  PcgDev *pcg = nullptr;
  OpenDev *open = nullptr;
  MeterDev *meter = nullptr;   // the cycle observables (meter.cu)
  QpDev *qp = nullptr;         // two normal fluids (qp.cu)
  // material per region: the node map (1-based material per node) and the tables; null for one material
  uint8_t *mat = nullptr;
  MatDev *mt = nullptr;
  bool haskwt_mat[TDGL_MAXB] = {};   // KWT on band µ in some material
  uint8_t *vac = nullptr;            // a sculpted sample: nonzero on the vacuum nodes (null: no vacuum)
  // per-step values: the device copy the kernels read, and the pinned host slots of the current call
  StepScal *ss_cur = nullptr;
  StepScal *ss_host = nullptr;
  int ss_cap = 0;
  cudaEvent_t ss_done = nullptr;   // the copies from ss_host of the last call have run
  bool ss_pending = false;
  StepScal ss_last;                // the values last copied to ss_cur (valid while ss_last_ok)
  bool ss_last_ok = false;
  // the step as a CUDA graph, one per θ/φ parity (advance! swaps them by pointer)
  bool graphs = true;
  bool branches = true;   // parallel branches inside a step (the bands side by side, the PCG's work beside its preconditioner)
  bool capturing = false;
  int parity = 0;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  cudaGraph_t graph[2] = {nullptr, nullptr};   // the captured steps, released with their executable graphs
  int glaunch[2] = {0, 0};
  cudaStream_t cap_stream = nullptr;   // captures the bodies of conditional nodes
  Tape *tape = nullptr;                // a batch records the launches of the step it captures here
  // counters
  long long steps = 0;
  int launches = 0;
  Prof prof;
  int open_recomputes = 0;
  std::vector<void *> allocs;
  size_t alloc_bytes = 0;   // device memory of the context's arrays (admission against an HBM budget)
};

int set_err(Ctx *ctx, int code, const char *what, cudaError_t e = cudaSuccess);
cudaEvent_t prof_begin(Ctx *ctx);
void prof_end(Ctx *ctx, cudaEvent_t a, int cat, double bytes);
void prof_collect(Ctx *ctx);

template <class... P, class... A>
void tape_record(Ctx *ctx, void (*kern)(P...), dim3 grid, dim3 block, size_t smem, A &&...a) {
  Tape *t = ctx->tape;
  const MergeInfo *m = merge_lookup((const void *)kern);
  if (!m) {
    t->ok = false;
    return;
  }
  ArgPack<P...> pk;
  argpack_set(pk, static_cast<A &&>(a)...);
  TapeRec r;
  r.kern = (const void *)kern;
  r.m = m;
  r.grid = grid;
  r.block = block;
  r.smem = smem;
  r.args.assign((const unsigned char *)&pk, (const unsigned char *)&pk + sizeof(pk));
  t->recs.push_back(std::move(r));
}

// Every kernel launch of the library goes through this macro: it counts the launch and, when profiling is on,
// times it with a pair of events on the context's stream; a batch capturing the step also records it.
#define TDGL_LAUNCH(ctx, cat, bytes, kern, grid, block, smem, ...)        \
  do {                                                                   \
    if ((ctx)->tape)                                                     \
      tdgl::tape_record((ctx), kern, dim3(grid), dim3(block), (size_t)(smem), __VA_ARGS__); \
    cudaEvent_t ev_a_ = tdgl::prof_begin(ctx);                           \
    kern<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);       \
    tdgl::prof_end((ctx), ev_a_, (cat), (double)(bytes));                \
    (ctx)->launches++;                                                   \
  } while (0)
// Let launches of `kern` use the device's whole opt-in shared memory per block less the kernel's own static shared
// memory (the two together may not exceed the opt-in limit, or the attribute call fails).
inline cudaError_t smem_optin(const void *kern) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kern);
  if (e != cudaSuccess) return e;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}
template <class... P>
cudaError_t smem_optin(void (*kern)(P...)) { return smem_optin((const void *)kern); }

template <class T>
int dalloc(Ctx *ctx, T **p, size_t n) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, n * sizeof(T) + 16);
  if (e != cudaSuccess) return set_err(ctx, TDGL_ENOMEM, "cudaMalloc", e);
  cudaMemsetAsync(q, 0, n * sizeof(T) + 16, ctx->stream);
  ctx->allocs.push_back(q);
  ctx->alloc_bytes += n * sizeof(T) + 16;
  *p = (T *)q;
  return 0;
}

// meter.cu
void meter_destroy(Ctx *ctx);

// _haskwt (bands.jl:454): KWT on band µ in any material
inline bool haskwt(const Ctx *ctx, int mu) { return ctx->P.bcs[mu].gamma2 > 0 || ctx->haskwt_mat[mu]; }

// noise.cu
bool skrock_band(const Ctx *ctx, int mu);
void sk_turn(Ctx *ctx, cd *D, const cd *X, int mu, double c);
void frame_smooth_rot(Ctx *ctx, cd *Cc, double h);
void frame_rot(Ctx *ctx, cd *Cc, double h);
void noise_after(Ctx *ctx);
void field_kick(Ctx *ctx);

// bands.cu
int update_bands(Ctx *ctx);
void omega_faces(Ctx *ctx);
struct LinkRot;   // bands.cu: links read as given or rotated on the fly
void ghosts(Ctx *ctx, cd *X, const cd *Lx, const cd *Ly, const cd *Lz, const LinkRot *lr = nullptr);
void vacuum_zero(Ctx *ctx);   // neumann! on a sculpted sample: F = 0 on every vacuum node, ghosts included
// field.cu
void supercurrent_increment(Ctx *ctx);
void scale_increment(Ctx *ctx);
void links_curl(Ctx *ctx);
void field_bc(Ctx *ctx);   // H, HJ and the ramp fraction from ctx->ss_cur
void advance_copy(Ctx *ctx);
void advance_swap(Ctx *ctx);          // the host half of advance!: θ↔φ and V↔U by pointer
// sep.cu
int sep_create(Ctx *ctx);
void sep_destroy(Ctx *ctx);
void sep_implicit(Ctx *ctx);
// (I + aK)^{-1} on plane-major component arrays (sep.cu); done: skip when set (the PCG's convergence flag)
struct DotFuse;   // pcg.cuh
// z = (I + aK)^{-1} r; with `dot`, the FP32 path also folds r·z and r·z_old into the PCG's scalars and returns true
// (false: the caller reduces them itself)
bool sep_apply(Ctx *ctx, const double *const *r, double *const *z, bool f32, const int *done, bool r32_ready = false,
               const DotFuse *dot = nullptr);
float *const *sep_r32(Ctx *ctx);   // the FP32 input copy the PCG writes for the FP32 preconditioner (null: none)
long long sep_nrange(Ctx *ctx, int ax);
int pm_from_packed_host(Ctx *ctx, double *const *pm, const double *host);
int pm_to_packed_host(Ctx *ctx, double *const *pm, double *host);
// heat.cu
int heat_create(Ctx *ctx, const tdgl_materials *M);
void heat_step(Ctx *ctx);
int heat_carry(Ctx *ctx, double *host, bool up);
int qp_create(Ctx *ctx, const tdgl_params *p);
void qp_destroy(Ctx *ctx);
int qp_potential(Ctx *ctx);
long long qp_cg_iterations(Ctx *ctx);   // the δ solve's CG iterations over all steps (a sculpted sample)
void qp_turn(Ctx *ctx);
void qp_potentials(Ctx *ctx, const double **out);   // δ (two bands) or μ_µ, node-shaped (null: none)
// pcg.cu
int pcg_create(Ctx *ctx);
void pcg_destroy(Ctx *ctx);
int pcg_implicit(Ctx *ctx);
int pcg_set_carry(Ctx *ctx, const tdgl_carry_view *v);
int pcg_get_carry(Ctx *ctx, const tdgl_carry_view *v);
int pcg_iters(Ctx *ctx, long long *total);
long long *pcg_stat_tc(Ctx *ctx);   // the device counter of tensor-core waits that ran out (null: no PCG)
// the device regions that carry a context's state from step to step (snapshots), and the host flags beside them
typedef std::vector<std::pair<void *, size_t>> Regions;
void pcg_regions(Ctx *ctx, Regions &r);
void pcg_flags(Ctx *ctx, int *warm, int *have2, bool set);
void open_regions(Ctx *ctx, Regions &r);
int *open_count_ptr(Ctx *ctx);
bool pcg_steady(Ctx *ctx);            // warm start settled: every later step launches the same kernels
bool pcg_graphable(Ctx *ctx);         // maxit is a whole number of loop turns (the captured loop's granularity)
int pcg_take_status(Ctx *ctx);        // TDGL_ENOCONV if a step since the last call reached maxit (syncs)
// openbc.cu
int open_create(Ctx *ctx);
void open_destroy(Ctx *ctx);
int open_update(Ctx *ctx, double HJ);
// the old/new face fields of the open boundary and this step's ramp fraction (openbc.jl:210-223)
void open_face_args(Ctx *ctx, const double **oo, const double **on);
double open_fraction(Ctx *ctx);
int open_set_carry(Ctx *ctx, const tdgl_carry_view *v);
int open_get_carry(Ctx *ctx, const tdgl_carry_view *v);

}  // namespace tdgl
