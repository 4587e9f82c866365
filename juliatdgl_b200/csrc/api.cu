// api.cu — the C-ABI of include/tdgl_b200.h: context, state transfer, and the order of one step
// (gtdgl/src/step.jl:13-35): open boundary, bands, supercurrent + increment, implicit solve, links + curl,
// field boundary, Neumann ghosts, advance.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "merge.cuh"

namespace tdgl {

static std::string g_err;

int set_err(Ctx *ctx, int code, const char *what, cudaError_t e) {
  char buf[512];
  if (e != cudaSuccess) snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  else snprintf(buf, sizeof(buf), "%s", what);
  if (ctx) ctx->err = buf;
  g_err = buf;   // the library's last error, whichever context raised it (a batch reports through it)
  return code;
}

const char *kcat_name[K_NCAT] = {"band_stage", "link_rotation", "neumann_ghosts", "frame_rate_faces", "current_increment",
                                  "links_curl", "face_field", "advance", "scale_increment", "sep_transform_f64",
                                  "sep_modes_f64", "precond_transform_f32", "precond_modes_f32", "precond_convert",
                                  "pcg_start", "pcg_curl", "pcg_apply", "pcg_residual", "pcg_update", "pcg_dot",
                                  "pcg_final", "pcg_direction", "pcg_extrap", "pack", "open_fft", "open_misc", "copy",
                                  "meter", "noise", "precond_inverse_f32", "heat", "pcg_update_x",
                                  "pcg_dot_side", "qp_exchange"};

cudaEvent_t prof_begin(Ctx *ctx) {
  Prof &p = ctx->prof;
  if (!p.on) return nullptr;
  cudaEvent_t e;
  if (!p.pool.empty()) {
    e = p.pool.back();
    p.pool.pop_back();
  } else {
    cudaEventCreate(&e);
  }
  cudaEventRecord(e, ctx->stream);
  return e;
}

void prof_end(Ctx *ctx, cudaEvent_t a, int cat, double bytes) {
  Prof &p = ctx->prof;
  if (!p.on || !a) return;
  cudaEvent_t e;
  if (!p.pool.empty()) {
    e = p.pool.back();
    p.pool.pop_back();
  } else {
    cudaEventCreate(&e);
  }
  cudaEventRecord(e, ctx->stream);
  p.pend.push_back(Prof::Rec{cat, a, e, bytes});
  if (p.pend.size() > 20000) prof_collect(ctx);
}

void prof_collect(Ctx *ctx) {
  Prof &p = ctx->prof;
  if (p.pend.empty()) return;
  cudaStreamSynchronize(ctx->stream);
  for (auto &r : p.pend) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    p.ms[r.cat] += ms;
    p.bytes[r.cat] += r.bytes;
    p.n[r.cat] += 1;
    p.pool.push_back(r.a);
    p.pool.push_back(r.b);
  }
  p.pend.clear();
}

namespace {
const int BS = 256;

// packed (a, b, c) host layout ↔ node-shaped device layout
template <class T>
__global__ void k_unpack(T *dst, const T *src, int a, int b, int c, Dim d) {
  long long n = (long long)a * b * c;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  // 32-bit division (the context holds fewer than 2^31 nodes)
  const unsigned u = (unsigned)t, r = u / (unsigned)a, k = r / (unsigned)b;
  const int i = (int)(u - r * (unsigned)a), j = (int)(r - k * (unsigned)b);
  dst[d.at(i + 1, j + 1, (int)k + 1)] = src[t];
}
template <class T>
__global__ void k_pack(T *dst, const T *src, int a, int b, int c, Dim d) {
  long long n = (long long)a * b * c;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const unsigned u = (unsigned)t, r = u / (unsigned)a, k = r / (unsigned)b;
  const int i = (int)(u - r * (unsigned)a), j = (int)(r - k * (unsigned)b);
  dst[t] = src[d.at(i + 1, j + 1, (int)k + 1)];
}

}  // namespace

struct Staging {
  void *dev = nullptr;
  size_t bytes = 0;
};
static Staging &staging(Ctx *ctx);

template <class T>
int up(Ctx *ctx, T *dst, const T *src, int a, int b, int c) {
  size_t nb = (size_t)a * b * c * sizeof(T);
  Staging &s = staging(ctx);
  TDGL_CUDA(cudaMemcpyAsync(s.dev, src, nb, cudaMemcpyHostToDevice, ctx->stream));
  long long n = (long long)a * b * c;
  TDGL_LAUNCH(ctx, K_PACK, 2.0 * nb, k_unpack<T>, nblk(n, BS), BS, 0, dst, (const T *)s.dev, a, b, c, ctx->g.d);
  TDGL_CUDA(cudaGetLastError());
  return 0;
}
template <class T>
int down(Ctx *ctx, T *dst, const T *src, int a, int b, int c) {
  size_t nb = (size_t)a * b * c * sizeof(T);
  Staging &s = staging(ctx);
  long long n = (long long)a * b * c;
  TDGL_LAUNCH(ctx, K_PACK, 2.0 * nb, k_pack<T>, nblk(n, BS), BS, 0, (T *)s.dev, src, a, b, c, ctx->g.d);
  TDGL_CUDA(cudaGetLastError());
  TDGL_CUDA(cudaMemcpyAsync(dst, s.dev, nb, cudaMemcpyDeviceToHost, ctx->stream));
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int repack_up(Ctx *ctx, double *dst, const double *src, int a, int b, int c) { return up<double>(ctx, dst, src, a, b, c); }
int repack_down(Ctx *ctx, double *dst, const double *src, int a, int b, int c) { return down<double>(ctx, dst, src, a, b, c); }

// A snapshot of everything a context carries from step to step (the state by role, so the θ/φ parity does not
// matter; the PCG warm start and extrapolation history; the open boundary's ramp), in one device buffer, with the
// host flags and the step count (the noise index).  The reference keeps the same set for its delay confirmation
// (_confirmation_snapshot / _confirmation_state!, protocol.jl:222-236).
struct Snap {
  void *dev = nullptr;
  size_t bytes = 0;
  long long steps = 0;
  int warm = 0, have2 = 0, open_count = -1;
  bool taken = false;
};

struct CtxX : Ctx {
  Staging stg;
  std::vector<Snap> snaps;
};
static Staging &staging(Ctx *ctx) { return static_cast<CtxX *>(ctx)->stg; }

static int check_params(const tdgl_params *p, char *why, size_t n) {
  auto no = [&](const char *m) {
    if (why && n) snprintf(why, n, "%s", m);
    return 0;
  };
  if (p->abi_version != TDGL_ABI_VERSION) return no("ABI version mismatch");
  if (p->nbands < 1 || p->nbands > TDGL_MAXB) return no("band count out of range");
  const tdgl_grid &g = p->grid;
  if (g.Nx < 3 || g.Ny < 3 || g.Nz < 3) return no("grid too small");
  // kernels index the points of a range with 32-bit arithmetic
  if ((double)(g.Nx + 1) * (g.Ny + 1) * (g.Nz + 1) * 3.0 >= 2147483647.0) return no("grid too large");
  if (!(g.x1 >= 2 && g.x2 + 1 <= g.Nx && g.y1 >= 2 && g.y2 + 1 <= g.Ny && g.z1 >= 2 && g.z2 + 1 <= g.Nz))
    return no("the block must have at least one padding cell on each face");
  for (int mu = 0; mu < p->nbands; mu++) {
    if (p->stages[mu] < 0 || p->stages[mu] > TDGL_MAXSTG) return no("stage count out of range");
    if (p->stages[mu] == 0 && p->nsub[mu] < 1) return no("substeps must be >= 1");
  }
  if (p->noise_on && !(p->noise_T >= 0)) return no("noise temperature must be >= 0");
  if (p->noise_on && p->noise_field && !(p->noise_sigma_n > 0)) return no("field noise needs sigma_n > 0");
  if (p->noise_on)
    for (int mu = 0; mu < p->nbands; mu++)
      if (!(p->noise_gamma[mu] > 0)) return no("noise needs Gamma > 0 per band");
  if (!p->f || !p->taux || !p->tauy || !p->tauz) return no("masks missing");
  if ((p->solver == TDGL_SOLVER_SCALE || p->solver == TDGL_SOLVER_PCG) && !(p->Dx && p->Dy && p->Dz))
    return no("link conductivity missing");
  if (p->solver < 0 || p->solver > 3) return no("unknown solver");
  if ((p->solver == TDGL_SOLVER_SEP || p->solver == TDGL_SOLVER_PCG) && !(g.dx == g.dy && g.dy == g.dz))
    return no("the implicit curl-curl needs dx = dy = dz");
  if (p->selffield_bc != TDGL_BC_SLAB &&
      !(p->bar_hy_z && p->bar_hy_y && p->bar_hz_z && p->bar_hz_y && p->bar_hz_x && p->bar_hy_x))
    return no("bar tables missing");
  if (p->selffield_bc == TDGL_BC_OPEN && (!p->open_green || !p->open_jbar || p->open_every < 1 || p->open_R < 1))
    return no("open-boundary tables missing");
  if (p->selffield_bc < 0 || p->selffield_bc > 2) return no("unknown self-field boundary");
  if (p->rotframe && !p->extrap) return no("rotframe needs extrap");
  if (p->heat_on && (p->vac || p->noise_on))   // scheme.jl:383, 428-429
    return no("the heat model is not taken with a sculpted sample or with noise");
  if (p->heat_on && !(p->heat_DT >= 0 && p->heat_cap > 0 && p->heat_margin >= 0)) return no("heat coefficients out of range");
  if (p->drag_on && (p->materials || p->vac))   // scheme.jl:384, materials.jl:75
    return no("the drag is not taken with materials or a sculpted sample");
  if (p->qp_on) {   // exchange.jl: QPExchange (two bands) or QPExchangeN; one material, no sculpted vacuum
    if (p->qp_on < 1 || p->qp_on > 2 || (p->qp_on == 1 && p->nbands != 2) || p->nbands < 2 ||
        (p->materials && p->qp_on != 1) ||
        ((p->vac || p->qp_cond) && (!p->qp_cond || !(p->qp_tol > 0) || p->qp_maxit < 1)) ||
        (p->qp_cx && (p->qp_on != 1 || !(p->qp_cond && p->qp_cy && p->qp_cz && p->qp_lamv))))
      return no("qp_exchange: two bands (or N fluids with one material); a sculpted sample with "
                "the conducting unknowns; the variable coefficients with two bands and the unknowns' types");
    if (p->qp_nj < 1 || p->qp_nk < 1 || p->qp_j0 < 1 || p->qp_k0 < 1 || p->qp_j0 + p->qp_nj - 1 > g.Ny + 1 ||
        p->qp_k0 + p->qp_nk - 1 > g.Nz + 1 || p->qp_j0 > g.y1 || p->qp_j0 + p->qp_nj - 1 < g.y2 + 1 ||
        p->qp_k0 > g.z1 || p->qp_k0 + p->qp_nk - 1 < g.z2 + 1 || g.x1 < 2 || g.x2 + 1 > g.Nx)
      return no("qp_exchange: the region of delta must hold the block inside the grid");
    if (!p->qp_Vx || !p->qp_Wx || !p->qp_ex || !p->qp_Vy || !p->qp_Wy || !p->qp_ey || !p->qp_Vz || !p->qp_Wz ||
        !p->qp_ez)
      return no("qp_exchange: bases missing");
  }
  if (p->vac && !(p->solver == TDGL_SOLVER_PCG || p->solver == TDGL_SOLVER_SCALE))
    return no("a sculpted sample needs the insulating padding (PCG or explicit with sigma per link)");
  if (const tdgl_materials *M = p->materials) {
    if (M->nmat < 1 || M->nmat > TDGL_MAXMAT) return no("material count out of range");
    if (!M->idx) return no("material map missing");
    const size_t nn = (size_t)(g.Nx + 1) * (g.Ny + 1) * (g.Nz + 1);
    for (size_t q = 0; q < nn; q++)
      if (M->idx[q] < 1 || M->idx[q] > M->nmat) return no("material index out of range");
    for (int mu = 0; mu < p->nbands; mu++)
      if (M->absent[0][mu]) return no("the first material has all its bands");
    for (int a = 0; a < M->nmat; a++) {
      for (int b = 0; b < M->nmat; b++)
        if (!(M->transparency[a][b] > 0 && M->transparency[a][b] <= 1)) return no("transparency must be in (0, 1]");
      for (int mu = 0; mu < p->nbands; mu++) {
        if (p->noise_on && !(M->gamma[a][mu] > 0)) return no("noise needs Gamma > 0 per material and band");
        for (int ax = 0; ax < 3; ax++)
          if (!(M->ma[a][mu][ax] > 0)) return no("band masses must be positive");
      }
    }
  }
  return 1;
}

// MatField's link weights without τ (materials.jl:97-110), per band, axis and pair of materials
static void mat_tables(const tdgl_materials &M, int N, MatDev *t) {
  memset(t, 0, sizeof(*t));
  for (int mu = 0; mu < N; mu++)
    for (int a = 0; a < M.nmat; a++) {
      t->full[mu][a] = M.full[a][mu];
      t->stage[mu][a] = M.stage[a][mu];
      t->gam[mu][a] = M.gamma[a][mu];
      t->a[mu][a] = M.a[a][mu];
      t->absent[mu][a] = M.absent[a][mu] != 0;
      for (int ax = 0; ax < 3; ax++) {
        const double m0 = M.ma[0][mu][ax];
        for (int b = 0; b < M.nmat; b++) {
          const double ma = M.ma[a][mu][ax], mb = M.ma[b][mu][ax];
          const double ml = ma == mb ? ma : (ma + mb) / 2;
          const double w = (ml == m0 ? 1.0 : m0 / ml) * (a == b ? 1.0 : M.transparency[a][b]);
          t->W[mu][ax][a][b] = (M.absent[a][mu] || M.absent[b][mu]) ? 0.0 : w;
        }
      }
    }
}

// Everything of step! (step.jl:13-35) after the open-boundary update, with this step's H, HJ, ramp fraction and
// noise index already in ctx->ss_cur.  The host effects (the θ/φ, V/U pointer swap and the step count) come last.
static int step_body(Ctx *ctx) {
  int rc = 0;
  if (ctx->P.qp_on && (rc = qp_potential(ctx))) return rc;   // qp_potential! (step.jl:15)
  rc = update_bands(ctx);
  if (rc) return rc;
  if (ctx->P.qp_on) qp_turn(ctx);            // qp_turn! (step.jl:19)
  if (ctx->P.noise_on) noise_after(ctx);   // noise_apply! / noise_kick! (step.jl:25)
  if (ctx->P.heat_on) heat_step(ctx);        // heat_step! (step.jl:27; reads θ − φ before the increment)
  supercurrent_increment(ctx);
  if (ctx->P.noise_on && ctx->P.noise_field) field_kick(ctx);   // field_kick! (step.jl:29)
  switch (ctx->P.solver) {
    case TDGL_SOLVER_SEP: sep_implicit(ctx); break;
    case TDGL_SOLVER_PCG: rc = pcg_implicit(ctx); break;
    case TDGL_SOLVER_SCALE: scale_increment(ctx); break;
    default: break;
  }
  if (rc) return rc;
  links_curl(ctx);
  field_bc(ctx);
  for (int mu = 0; mu < ctx->N; mu++) ghosts(ctx, ctx->F[mu], ctx->U[0], ctx->U[1], ctx->U[2]);
  if (ctx->vac) vacuum_zero(ctx);   // neumann! (field.jl:235-244)
  advance_copy(ctx);
  ctx->steps++;
  return 0;
}

// A step launches the same kernels with the same arguments as the last one of its parity once the PCG warm start
// has settled; it is then captured once per parity and replayed as one graph launch.
static bool graph_ready(Ctx *ctx) {
  if (!ctx->graphs || ctx->prof.on) return false;
  if (ctx->P.solver == TDGL_SOLVER_PCG) return pcg_steady(ctx) && pcg_graphable(ctx);
  return true;
}

static int capture_step(Ctx *ctx) {
  const int p = ctx->parity;
  cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return set_err(ctx, TDGL_ECUDA, "cudaStreamBeginCapture", e);
  ctx->capturing = true;
  const int l0 = ctx->launches;
  int rc = step_body(ctx);
  ctx->capturing = false;
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(ctx->stream, &g);
  if (rc == 0 && e != cudaSuccess) rc = set_err(ctx, TDGL_ECUDA, "cudaStreamEndCapture", e);
  if (rc == 0) {
    e = cudaGraphInstantiate(&ctx->gexec[p], g, 0);
    if (e != cudaSuccess) rc = set_err(ctx, TDGL_ECUDA, "cudaGraphInstantiate", e);
  }
  if (rc) {
    if (g) cudaGraphDestroy(g);
    ctx->graphs = false;   // the context goes on without graphs
    return rc;
  }
  ctx->graph[p] = g;
  ctx->glaunch[p] = ctx->launches - l0;
  // the captured step has not run yet: its host effects already have, so launch it now
  e = cudaGraphLaunch(ctx->gexec[p], ctx->stream);
  if (e != cudaSuccess) return set_err(ctx, TDGL_ECUDA, "cudaGraphLaunch", e);
  return 0;
}

static int step(Ctx *ctx) {
  if (!graph_ready(ctx)) return step_body(ctx);
  const int p = ctx->parity;
  if (!ctx->gexec[p]) return capture_step(ctx);
  cudaError_t e = cudaGraphLaunch(ctx->gexec[p], ctx->stream);
  if (e != cudaSuccess) return set_err(ctx, TDGL_ECUDA, "cudaGraphLaunch", e);
  ctx->launches += ctx->glaunch[p];
  advance_swap(ctx);
  ctx->steps++;
  return 0;
}

static void drop_graphs(Ctx *ctx) {
  for (int p = 0; p < 2; p++) {
    if (ctx->gexec[p]) {
      cudaGraphExecDestroy(ctx->gexec[p]);
      ctx->gexec[p] = nullptr;
    }
    if (ctx->graph[p]) {
      cudaGraphDestroy(ctx->graph[p]);
      ctx->graph[p] = nullptr;
    }
  }
}

}  // namespace tdgl

using namespace tdgl;

extern "C" {

static void state_regions(Ctx *ctx, Regions &r) {
  const size_t nn = ctx->g.d.n();
  for (int mu = 0; mu < ctx->N; mu++) {
    r.push_back({ctx->G[mu], nn * sizeof(cd)});
    r.push_back({ctx->F[mu], nn * sizeof(cd)});
  }
  for (int ax = 0; ax < 3; ax++) {
    r.push_back({ctx->th[ax], nn * sizeof(double)});
    r.push_back({ctx->ph[ax], nn * sizeof(double)});
    r.push_back({ctx->J[ax], nn * sizeof(double)});
    r.push_back({ctx->h[ax], nn * sizeof(double)});
    r.push_back({ctx->U[ax], nn * sizeof(cd)});
    r.push_back({ctx->V[ax], nn * sizeof(cd)});
  }
  if (ctx->pcg) pcg_regions(ctx, r);
  if (ctx->open) open_regions(ctx, r);
  if (ctx->Th) r.push_back({ctx->Th, nn * sizeof(double)});
}

static int snap_copy(Ctx *ctx, Snap &sn, bool take) {
  Regions r;
  state_regions(ctx, r);
  size_t off = 0;
  for (auto &q : r) {
    char *d = (char *)sn.dev + off;
    if (take) TDGL_CUDA(cudaMemcpyAsync(d, q.first, q.second, cudaMemcpyDeviceToDevice, ctx->stream));
    else TDGL_CUDA(cudaMemcpyAsync(q.first, d, q.second, cudaMemcpyDeviceToDevice, ctx->stream));
    off += (q.second + 255) & ~(size_t)255;
  }
  return 0;
}

int tdgl_snapshot_take(tdgl_ctx *c, int32_t slot) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || slot < 0 || slot > 255) return set_err(ctx, TDGL_EINVAL, "snapshot: bad slot");
  if (!ctx->have_state) return set_err(ctx, TDGL_ESTATE, "no state uploaded");
  CtxX *x = static_cast<CtxX *>(ctx);
  if ((int)x->snaps.size() <= slot) x->snaps.resize(slot + 1);
  Snap &sn = x->snaps[slot];
  if (!sn.dev) {
    Regions r;
    state_regions(ctx, r);
    size_t b = 0;
    for (auto &q : r) b += (q.second + 255) & ~(size_t)255;
    cudaError_t e = cudaMalloc(&sn.dev, b);
    if (e != cudaSuccess) return set_err(ctx, TDGL_ENOMEM, "snapshot cudaMalloc", e);
    sn.bytes = b;
  }
  int rc = snap_copy(ctx, sn, true);
  if (rc) return rc;
  sn.steps = ctx->steps;
  if (ctx->pcg) pcg_flags(ctx, &sn.warm, &sn.have2, false);
  if (ctx->open) sn.open_count = *open_count_ptr(ctx);
  sn.taken = true;
  return 0;
}

int tdgl_snapshot_restore(tdgl_ctx *c, int32_t slot) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx) return TDGL_EINVAL;
  CtxX *x = static_cast<CtxX *>(ctx);
  if (slot < 0 || slot >= (int)x->snaps.size() || !x->snaps[slot].taken) return set_err(ctx, TDGL_EINVAL, "snapshot: empty slot");
  Snap &sn = x->snaps[slot];
  int rc = snap_copy(ctx, sn, false);
  if (rc) return rc;
  ctx->steps = sn.steps;
  if (ctx->pcg) pcg_flags(ctx, &sn.warm, &sn.have2, true);
  if (ctx->open) *open_count_ptr(ctx) = sn.open_count;
  return 0;
}

int tdgl_snapshot_free(tdgl_ctx *c, int32_t slot) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx) return TDGL_EINVAL;
  CtxX *x = static_cast<CtxX *>(ctx);
  if (slot < 0 || slot >= (int)x->snaps.size()) return 0;
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  if (x->snaps[slot].dev) cudaFree(x->snaps[slot].dev);
  x->snaps[slot] = Snap();
  return 0;
}

int64_t tdgl_device_bytes(const tdgl_ctx *c) {
  const Ctx *ctx = reinterpret_cast<const Ctx *>(c);
  if (!ctx) return 0;
  const CtxX *x = static_cast<const CtxX *>(ctx);
  int64_t b = (int64_t)ctx->alloc_bytes + (int64_t)x->stg.bytes;
  for (const Snap &sn : x->snaps) b += (int64_t)sn.bytes;
  return b;
}

int tdgl_abi_version(void) { return TDGL_ABI_VERSION; }

int tdgl_supported(const tdgl_params *p, char *why, int32_t why_len) {
  if (!p) return 0;
  return check_params(p, why, why_len > 0 ? (size_t)why_len : 0);
}

const char *tdgl_last_error(const tdgl_ctx *c) {
  const Ctx *ctx = reinterpret_cast<const Ctx *>(c);
  return ctx ? ctx->err.c_str() : g_err.c_str();
}

int tdgl_ctx_destroy(tdgl_ctx *c) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx) return 0;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  drop_graphs(ctx);
  if (ctx->ss_host) cudaFreeHost(ctx->ss_host);
  if (ctx->ss_done) cudaEventDestroy(ctx->ss_done);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  for (int mu = 0; mu < TDGL_MAXB; mu++) {
    if (ctx->bstream[mu]) cudaStreamDestroy(ctx->bstream[mu]);
    if (ctx->bev[mu]) cudaEventDestroy(ctx->bev[mu]);
  }
  ctx->prof.on = false;
  for (auto &r : ctx->prof.pend) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : ctx->prof.pool) cudaEventDestroy(e);
  sep_destroy(ctx);
  pcg_destroy(ctx);
  open_destroy(ctx);
  meter_destroy(ctx);
  qp_destroy(ctx);
  for (void *q : ctx->allocs) cudaFree(q);
  CtxX *x = static_cast<CtxX *>(ctx);
  if (x->stg.dev) cudaFree(x->stg.dev);
  for (Snap &sn : x->snaps)
    if (sn.dev) cudaFree(sn.dev);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete x;
  return 0;
}

int tdgl_ctx_create(const tdgl_params *p, tdgl_ctx **out) {
  if (!p || !out) return set_err(nullptr, TDGL_EINVAL, "null argument");
  char why[256] = {0};
  if (!check_params(p, why, sizeof(why))) {
    std::string m = std::string("unsupported parameters: ") + why;
    return set_err(nullptr, TDGL_EINVAL, m.c_str());
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return set_err(nullptr, TDGL_ECUDA, "no CUDA device", e);
  CtxX *x = new CtxX();
  Ctx *ctx = x;
  ctx->P = *p;
  ctx->N = p->nbands;
  const tdgl_grid &gg = p->grid;
  Geo &g = ctx->g;
  g.Nx = gg.Nx; g.Ny = gg.Ny; g.Nz = gg.Nz;
  g.x1 = gg.x1; g.x2 = gg.x2; g.y1 = gg.y1; g.y2 = gg.y2; g.z1 = gg.z1; g.z2 = gg.z2;
  g.dx = gg.dx; g.dy = gg.dy; g.dz = gg.dz;
  g.d = Dim{gg.Nx + 1, gg.Ny + 1, gg.Nz + 1};
  // host pointers of the params are not kept
  ctx->P.f = ctx->P.taux = ctx->P.tauy = ctx->P.tauz = nullptr;
  ctx->P.Dx = ctx->P.Dy = ctx->P.Dz = nullptr;
  ctx->P.bar_hy_z = ctx->P.bar_hy_y = ctx->P.bar_hz_z = ctx->P.bar_hz_y = ctx->P.bar_hz_x = ctx->P.bar_hy_x = nullptr;
  ctx->P.open_jbar = nullptr;
  ctx->P.materials = nullptr;
  ctx->P.vac = nullptr;
  ctx->P.qp_Vx = ctx->P.qp_Wx = ctx->P.qp_ex = ctx->P.qp_Vy = ctx->P.qp_Wy = ctx->P.qp_ey = nullptr;
  ctx->P.qp_Vz = ctx->P.qp_Wz = ctx->P.qp_ez = nullptr;
  ctx->P.qp_cond = nullptr;
  ctx->P.qp_cx = ctx->P.qp_cy = ctx->P.qp_cz = ctx->P.qp_lamv = nullptr;
  int rc = 0;
  auto fail = [&](int code) {
    std::string m = ctx->err;
    tdgl_ctx_destroy(reinterpret_cast<tdgl_ctx *>(ctx));
    set_err(nullptr, code, m.c_str());
    return code;
  };
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(set_err(ctx, TDGL_ECUDA, "cudaStreamCreate", e));
  if ((e = cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(set_err(ctx, TDGL_ECUDA, "cudaStreamCreate", e));
  if ((e = cudaEventCreateWithFlags(&ctx->ss_done, cudaEventDisableTiming)) != cudaSuccess)
    return fail(set_err(ctx, TDGL_ECUDA, "cudaEventCreate", e));
  if ((rc = dalloc(ctx, &ctx->ss_cur, 1))) return fail(rc);
  const long long nn = g.d.n();
  x->stg.bytes = (size_t)nn * sizeof(cd);
  if ((e = cudaMalloc(&x->stg.dev, x->stg.bytes)) != cudaSuccess) return fail(set_err(ctx, TDGL_ENOMEM, "cudaMalloc", e));
  // masks (already node-shaped)
  if ((rc = dalloc(ctx, &ctx->f, nn))) return fail(rc);
  for (int ax = 0; ax < 3; ax++)
    if ((rc = dalloc(ctx, &ctx->tau[ax], nn))) return fail(rc);
  if ((rc = up<double>(ctx, ctx->f, p->f, g.Nx + 1, g.Ny + 1, g.Nz + 1))) return fail(rc);
  const double *taus[3] = {p->taux, p->tauy, p->tauz};
  for (int ax = 0; ax < 3; ax++)
    if ((rc = up<double>(ctx, ctx->tau[ax], taus[ax], g.Nx + 1, g.Ny + 1, g.Nz + 1))) return fail(rc);
  if (p->materials) {   // the node map is node-shaped already: a plain copy; the tables once per context
    const tdgl_materials &M = *p->materials;
    std::vector<MatDev> t(1);
    mat_tables(M, ctx->N, t.data());
    for (int mu = 0; mu < ctx->N; mu++)
      for (int a = 0; a < M.nmat; a++) ctx->haskwt_mat[mu] = ctx->haskwt_mat[mu] || M.full[a][mu].gamma2 > 0;
    if ((rc = dalloc(ctx, &ctx->mat, (size_t)nn))) return fail(rc);
    if ((rc = dalloc(ctx, &ctx->mt, 1))) return fail(rc);
    if ((e = cudaMemcpyAsync(ctx->mat, M.idx, (size_t)nn, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(set_err(ctx, TDGL_ECUDA, "material map upload", e));
    if ((e = cudaMemcpyAsync(ctx->mt, t.data(), sizeof(MatDev), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(set_err(ctx, TDGL_ECUDA, "material tables upload", e));
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(set_err(ctx, TDGL_ECUDA, "materials", e));
  }
  if (p->heat_on && (rc = heat_create(ctx, p->materials))) return fail(rc);
  if (p->qp_on && (rc = qp_create(ctx, p))) return fail(rc);
  if (p->drag_on) {   // the drag's tables (read by the band stages and the supercurrent)
    if ((rc = dalloc(ctx, &ctx->drag_c, (size_t)TDGL_MAXB * TDGL_MAXB * 3))) return fail(rc);
    if ((rc = dalloc(ctx, &ctx->drag_nu, (size_t)TDGL_MAXB * TDGL_MAXB))) return fail(rc);
    if ((e = cudaMemcpyAsync(ctx->drag_c, p->drag_c, sizeof(p->drag_c), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(ctx->drag_nu, p->drag_nu, sizeof(p->drag_nu), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(set_err(ctx, TDGL_ECUDA, "drag tables upload", e));
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(set_err(ctx, TDGL_ECUDA, "drag", e));
  }
  if (p->vac) {   // node-shaped already: a plain copy
    if ((rc = dalloc(ctx, &ctx->vac, (size_t)nn))) return fail(rc);
    if ((e = cudaMemcpyAsync(ctx->vac, p->vac, (size_t)nn, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(set_err(ctx, TDGL_ECUDA, "vacuum map upload", e));
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(set_err(ctx, TDGL_ECUDA, "vacuum", e));
  }
  int ls[3][3] = {{g.Nx, g.Ny + 1, g.Nz + 1}, {g.Nx + 1, g.Ny, g.Nz + 1}, {g.Nx + 1, g.Ny + 1, g.Nz}};
  if (p->Dx) {
    const double *Ds[3] = {p->Dx, p->Dy, p->Dz};
    for (int ax = 0; ax < 3; ax++) {
      if ((rc = dalloc(ctx, &ctx->D[ax], nn))) return fail(rc);
      if ((rc = up<double>(ctx, ctx->D[ax], Ds[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return fail(rc);
    }
  }
  if (p->selffield_bc != TDGL_BC_SLAB) {
    size_t sz[6] = {(size_t)(g.Ny + 1) * 2, (size_t)2 * g.Nz, (size_t)g.Ny * 2, (size_t)2 * (g.Nz + 1), (size_t)g.Ny * (g.Nz + 1),
                    (size_t)(g.Ny + 1) * g.Nz};
    const double *src[6] = {p->bar_hy_z, p->bar_hy_y, p->bar_hz_z, p->bar_hz_y, p->bar_hz_x, p->bar_hy_x};
    for (int q = 0; q < 6; q++) {
      if ((rc = dalloc(ctx, &ctx->bar[q], sz[q]))) return fail(rc);
      if ((e = cudaMemcpyAsync(ctx->bar[q], src[q], sz[q] * sizeof(double), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
        return fail(set_err(ctx, TDGL_ECUDA, "bar upload", e));
    }
  }
  if (p->selffield_bc == TDGL_BC_OPEN) {
    size_t n = (size_t)(g.Ny + 1) * (g.Nz + 1);
    if ((rc = dalloc(ctx, &ctx->jbar, n))) return fail(rc);
    if ((e = cudaMemcpyAsync(ctx->jbar, p->open_jbar, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(set_err(ctx, TDGL_ECUDA, "jbar upload", e));
  }
  // state and workspaces
  for (int mu = 0; mu < ctx->N; mu++) {
    if ((rc = dalloc(ctx, &ctx->G[mu], nn))) return fail(rc);
    if ((rc = dalloc(ctx, &ctx->F[mu], nn))) return fail(rc);
  }
  for (int ax = 0; ax < 3; ax++) {
    double **rs[5] = {&ctx->th[ax], &ctx->ph[ax], &ctx->J[ax], &ctx->h[ax], &ctx->Rr[ax]};
    for (int q = 0; q < 5; q++)
      if ((rc = dalloc(ctx, rs[q], nn))) return fail(rc);
    cd **cs[4] = {&ctx->U[ax], &ctx->V[ax], &ctx->L[ax], &ctx->Rl[ax]};
    for (int q = 0; q < 4; q++)
      if ((rc = dalloc(ctx, cs[q], nn))) return fail(rc);
  }
  if ((rc = dalloc(ctx, &ctx->W, nn))) return fail(rc);
  if ((rc = dalloc(ctx, &ctx->W2, nn))) return fail(rc);
  if ((rc = dalloc(ctx, &ctx->Om, nn))) return fail(rc);
  if (p->noise_on && (rc = dalloc(ctx, &ctx->Oms, nn))) return fail(rc);
  // the stage workspaces of band 0 are the ones above; bands 1.. get their own, a stream each and the fork/join
  // events (update_bands runs the bands concurrently)
  {
    Ctx::BandWs &w0 = ctx->bws[0];
    w0.W = ctx->W; w0.W2 = ctx->W2; w0.Om = ctx->Om; w0.Oms = ctx->Oms;
    for (int ax = 0; ax < 3; ax++) {
      w0.L[ax] = ctx->L[ax]; w0.Rl[ax] = ctx->Rl[ax]; w0.Rr[ax] = ctx->Rr[ax];
    }
    for (int mu = 1; mu < ctx->N; mu++) {
      Ctx::BandWs &w = ctx->bws[mu];
      if ((rc = dalloc(ctx, &w.W, nn)) || (rc = dalloc(ctx, &w.W2, nn)) || (rc = dalloc(ctx, &w.Om, nn)) ||
          (p->noise_on && (rc = dalloc(ctx, &w.Oms, nn))))
        return fail(rc);
      for (int ax = 0; ax < 3; ax++)
        if ((rc = dalloc(ctx, &w.L[ax], nn)) || (rc = dalloc(ctx, &w.Rl[ax], nn)) || (rc = dalloc(ctx, &w.Rr[ax], nn)))
          return fail(rc);
      if ((e = cudaStreamCreateWithFlags(&ctx->bstream[mu], cudaStreamNonBlocking)) != cudaSuccess)
        return fail(set_err(ctx, TDGL_ECUDA, "cudaStreamCreate", e));
    }
    for (int mu = 0; mu < ctx->N; mu++)
      if ((e = cudaEventCreateWithFlags(&ctx->bev[mu], cudaEventDisableTiming)) != cudaSuccess)
        return fail(set_err(ctx, TDGL_ECUDA, "cudaEventCreate", e));
  }
  if (p->solver == TDGL_SOLVER_SEP || p->solver == TDGL_SOLVER_PCG)
    if ((rc = sep_create(ctx))) return fail(rc);
  if (p->solver == TDGL_SOLVER_PCG)
    if ((rc = pcg_create(ctx))) return fail(rc);
  if (p->selffield_bc == TDGL_BC_OPEN)
    if ((rc = open_create(ctx))) return fail(rc);
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(set_err(ctx, TDGL_ECUDA, "set-up", e));
  *out = reinterpret_cast<tdgl_ctx *>(ctx);
  return 0;
}

int tdgl_upload_state(tdgl_ctx *c, const tdgl_state_view *s) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !s) return TDGL_EINVAL;
  const Geo &g = ctx->g;
  int ls[3][3] = {{g.Nx, g.Ny + 1, g.Nz + 1}, {g.Nx + 1, g.Ny, g.Nz + 1}, {g.Nx + 1, g.Ny + 1, g.Nz}};
  int hs[3][3] = {{g.Nx + 1, g.Ny, g.Nz}, {g.Nx, g.Ny + 1, g.Nz}, {g.Nx, g.Ny, g.Nz + 1}};
  int rc;
  for (int mu = 0; mu < ctx->N; mu++) {
    if (!s->G[mu] || !s->F[mu]) return set_err(ctx, TDGL_EINVAL, "band array missing");
    if ((rc = up<cd>(ctx, ctx->G[mu], (const cd *)s->G[mu], g.Nx + 1, g.Ny + 1, g.Nz + 1))) return rc;
    if ((rc = up<cd>(ctx, ctx->F[mu], (const cd *)s->F[mu], g.Nx + 1, g.Ny + 1, g.Nz + 1))) return rc;
  }
  for (int ax = 0; ax < 3; ax++) {
    if ((rc = up<double>(ctx, ctx->th[ax], s->th[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = up<double>(ctx, ctx->ph[ax], s->ph[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = up<cd>(ctx, ctx->U[ax], (const cd *)s->U[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = up<cd>(ctx, ctx->V[ax], (const cd *)s->V[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = up<double>(ctx, ctx->J[ax], s->J[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = up<double>(ctx, ctx->h[ax], s->h[ax], hs[ax][0], hs[ax][1], hs[ax][2]))) return rc;
  }
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->have_state = true;
  return 0;
}

int tdgl_download_state(tdgl_ctx *c, const tdgl_state_view *s) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !s) return TDGL_EINVAL;
  if (!ctx->have_state) return set_err(ctx, TDGL_ESTATE, "no state uploaded");
  const Geo &g = ctx->g;
  int ls[3][3] = {{g.Nx, g.Ny + 1, g.Nz + 1}, {g.Nx + 1, g.Ny, g.Nz + 1}, {g.Nx + 1, g.Ny + 1, g.Nz}};
  int hs[3][3] = {{g.Nx + 1, g.Ny, g.Nz}, {g.Nx, g.Ny + 1, g.Nz}, {g.Nx, g.Ny, g.Nz + 1}};
  int rc;
  for (int mu = 0; mu < ctx->N; mu++) {
    if ((rc = down<cd>(ctx, (cd *)s->G[mu], ctx->G[mu], g.Nx + 1, g.Ny + 1, g.Nz + 1))) return rc;
    if ((rc = down<cd>(ctx, (cd *)s->F[mu], ctx->F[mu], g.Nx + 1, g.Ny + 1, g.Nz + 1))) return rc;
  }
  for (int ax = 0; ax < 3; ax++) {
    if ((rc = down<double>(ctx, s->th[ax], ctx->th[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = down<double>(ctx, s->ph[ax], ctx->ph[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = down<cd>(ctx, (cd *)s->U[ax], ctx->U[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = down<cd>(ctx, (cd *)s->V[ax], ctx->V[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = down<double>(ctx, s->J[ax], ctx->J[ax], ls[ax][0], ls[ax][1], ls[ax][2]))) return rc;
    if ((rc = down<double>(ctx, s->h[ax], ctx->h[ax], hs[ax][0], hs[ax][1], hs[ax][2]))) return rc;
  }
  return 0;
}

int tdgl_set_carry(tdgl_ctx *c, const tdgl_carry_view *v) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !v) return TDGL_EINVAL;
  int rc;
  if (ctx->pcg && (rc = pcg_set_carry(ctx, v))) return rc;
  if (ctx->open && (rc = open_set_carry(ctx, v))) return rc;
  if (ctx->Th && v->heat_theta && (rc = heat_carry(ctx, v->heat_theta, true))) return rc;
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int tdgl_get_carry(tdgl_ctx *c, const tdgl_carry_view *v) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !v) return TDGL_EINVAL;
  int rc;
  if (ctx->pcg && (rc = pcg_get_carry(ctx, v))) return rc;
  if (ctx->open && (rc = open_get_carry(ctx, v))) return rc;
  if (ctx->Th && v->heat_theta && (rc = heat_carry(ctx, v->heat_theta, false))) return rc;
  return 0;
}

// pinned slots for the per-step values of a call of n steps; the slots of the previous call are reused only after
// their copies have run
static int ss_reserve(Ctx *ctx, int n) {
  if (ctx->ss_pending) {
    TDGL_CUDA(cudaEventSynchronize(ctx->ss_done));
    ctx->ss_pending = false;
  }
  if (n <= ctx->ss_cap) return 0;
  if (ctx->ss_host) cudaFreeHost(ctx->ss_host);
  ctx->ss_host = nullptr;
  ctx->ss_cap = 0;
  const int cap = std::max(n, 64);
  TDGL_CUDA(cudaMallocHost(&ctx->ss_host, (size_t)cap * sizeof(StepScal)));
  ctx->ss_cap = cap;
  return 0;
}

static int deferred_status(Ctx *ctx) {
  const int st = ctx->P.solver == TDGL_SOLVER_PCG ? pcg_take_status(ctx) : 0;
  if (st == TDGL_ENOCONV) set_err(ctx, st, "PCG reached maxit without meeting its tolerance");
  return st;
}

static int run_steps(Ctx *ctx, int32_t n, double H, const double *HJs, double HJ, bool wait) {
  if (!ctx) return TDGL_EINVAL;
  if (!ctx->have_state) return set_err(ctx, TDGL_ESTATE, "no state uploaded");
  if (n < 0) return set_err(ctx, TDGL_EINVAL, "negative step count");
  ctx->launches = 0;
  int rc = ss_reserve(ctx, n);
  if (rc) return rc;
  const bool open = ctx->P.selffield_bc == TDGL_BC_OPEN;
  for (int q = 0; q < n; q++) {
    const double hj = HJs ? HJs[q] : HJ;
    if (open && (rc = open_update(ctx, hj))) return rc;   // open_update! (step.jl:14), outside the captured step
    StepScal &v = ctx->ss_host[q];
    v.H = H;
    v.HJ = hj;
    v.open_fr = open ? open_fraction(ctx) : 0.0;
    v.noise_step = (unsigned long long)(ctx->P.noise_step0 + ctx->steps);
    // a step with the values of the last one (fixed H and HJ, no noise, no open ramp) needs no copy
    if (!ctx->ss_last_ok || memcmp(&v, &ctx->ss_last, sizeof(StepScal)) != 0) {
      TDGL_CUDA(cudaMemcpyAsync(ctx->ss_cur, &v, sizeof(StepScal), cudaMemcpyHostToDevice, ctx->stream));
      ctx->ss_last = v;
      ctx->ss_last_ok = true;
    }
    if ((rc = step(ctx))) return rc;
  }
  TDGL_CUDA(cudaEventRecord(ctx->ss_done, ctx->stream));
  ctx->ss_pending = true;
  TDGL_CUDA(cudaGetLastError());
  if (!wait) return 0;
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return deferred_status(ctx);
}

// ---------------------------------------------------------------------------------------------- batches
// Many independent contexts stepped together (uneven grids, each with its own H and HJ).  Once every context's step
// repeats (the PCG warm start settled), one step of the whole batch is captured across streams — the batch stream
// forks to every context's stream, each captures its step (its PCG loop as a conditional node of the same graph)
// and joins back — once per parity; afterwards one launch advances every context by a step, the independent
// branches running concurrently.  A context with noise gets a one-thread kernel after its step that advances its
// noise index.  A context with the open boundary takes its open update (open_update!, step.jl:14: the ramp count,
// and the recomputation when due) on its own stream before each batch step, ordered after the previous batch step
// and before the next, with that step's scalars (the ramp fraction among them) copied to its device scalars.
__device__ __forceinline__ void ss_advance_b(const Blk bk, StepScal * const &s);
__global__ void k_ss_advance(StepScal *s) { ss_advance_b(TDGL_BLK, s); }
TDGL_MERGEABLE(k_ss_advance, ss_advance_b, 32, 1, false);
__device__ __forceinline__ void ss_advance_b(const Blk bk, StepScal * const &s) {
  if (threadIdx.x == 0) s->noise_step += 1;
}

struct tdgl_batch_impl {
  std::vector<Ctx *> c;
  cudaStream_t stream = nullptr;
  std::vector<cudaEvent_t> fork, join;
  cudaEvent_t done = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};   // k = 0: the parities par0; k = 1: all flipped
  std::vector<int> par0, glaunch[2];
  // merged steps (merge.cuh): the launches each context's captured step recorded and the graph nodes it added;
  // contexts whose nodes are exactly those launches share merged launches in the batch graph
  bool merge = true;
  double merge_blocks_per_sm = 4.0;   // the x-grid of a striding kernel, over the whole merged launch
  std::vector<Tape> tape[2];
  std::vector<std::vector<cudaGraphNode_t>> added[2];
  int launches[2] = {0, 0};    // kernel launches of a step of graph k
  int mchains[2] = {0, 0};     // merged chains in graph k
  int mcontexts[2] = {0, 0};   // contexts served by them
};

static void batch_drop(tdgl_batch_impl *b) {
  for (int k = 0; k < 2; k++) {
    if (b->exec[k]) {
      cudaGraphExecDestroy(b->exec[k]);
      b->exec[k] = nullptr;
    }
    b->launches[k] = b->mchains[k] = b->mcontexts[k] = 0;
  }
}

// the nodes of the graph that stream s is capturing into
static bool capture_nodes(cudaStream_t s, std::vector<cudaGraphNode_t> &out) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  size_t n = 0;
  out.clear();
  if (cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr) != cudaSuccess || !g) return false;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return false;
  out.resize(n);
  if (n && cudaGraphGetNodes(g, out.data(), &n) != cudaSuccess) return false;
  out.resize(n);
  return true;
}

// One merged launch: the kernel's merged form over a chain's contexts, with its parameter block.
struct MergedLaunch {
  const void *fn;
  dim3 grid, block;
  size_t smem;
  std::vector<unsigned char> params;
};

// Plans the merged launches of graph k.  A context takes part when the nodes its step added to the capture are
// its recorded launches alone (all kernels with a merged form: no PCG loop, no copies).  Those with the same
// kernel sequence (kernel and block shape at every position) form a group; a group of two or more is cut into
// chains of at most as many contexts as one launch of each of its kernels holds, and each position of a chain
// becomes one merged launch.  `members` receives the contexts of each chain.
static void merge_plan(tdgl_batch_impl *b, int k, std::vector<std::vector<MergedLaunch>> &chains,
                       std::vector<std::vector<int>> &members) {
  const int nc = (int)b->c.size();
  std::vector<int> ok;
  for (int i = 0; i < nc; i++) {
    const Tape &t = b->tape[k][i];
    bool good = t.ok && !t.recs.empty() && t.recs.size() == b->added[k][i].size();
    for (size_t q = 0; good && q < b->added[k][i].size(); q++) {
      cudaGraphNodeType ty;
      good = cudaGraphNodeGetType(b->added[k][i][q], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel;
    }
    if (good) ok.push_back(i);
  }
  auto same = [&](int i, int j) {
    const auto &a = b->tape[k][i].recs, &o = b->tape[k][j].recs;
    if (a.size() != o.size()) return false;
    for (size_t p = 0; p < a.size(); p++)
      if (a[p].kern != o[p].kern || a[p].block.x != o[p].block.x || a[p].block.y != o[p].block.y ||
          a[p].block.z != o[p].block.z)
        return false;
    return true;
  };
  std::vector<std::vector<int>> groups;
  for (int i : ok) {
    bool placed = false;
    for (auto &g : groups)
      if (same(g[0], i)) {
        g.push_back(i);
        placed = true;
        break;
      }
    if (!placed) groups.push_back({i});
  }
  int nsm = 148, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    nsm = 148;
  for (const auto &g : groups) {
    if (g.size() < 2) continue;   // a context alone keeps its own launches
    const auto &recs0 = b->tape[k][g[0]].recs;
    int cap = (int)g.size();
    for (const auto &r : recs0) cap = std::min(cap, r.m->cap);
    for (size_t c0 = 0; c0 < g.size(); c0 += cap) {
      const int n = (int)std::min(g.size() - c0, (size_t)cap);
      std::vector<MergedLaunch> chain;
      bool good = n >= 2;
      for (size_t p = 0; good && p < recs0.size(); p++) {
        const MergeInfo *m = recs0[p].m;
        MergedLaunch L;
        L.fn = m->merged;
        L.block = recs0[p].block;
        L.smem = 0;
        L.params.assign(m->param_bytes, 0);
        *reinterpret_cast<int *>(L.params.data()) = n;
        // a striding kernel's x-grid: its share, by its own x-grid, of merge_blocks_per_sm × SMs, at most its own
        double gsum = 0.0;
        for (int q = 0; q < n; q++) gsum += b->tape[k][g[c0 + q]].recs[p].grid.x;
        unsigned long long start = 0;
        for (int q = 0; q < n; q++) {
          const TapeRec &r = b->tape[k][g[c0 + q]].recs[p];
          unsigned gx = r.grid.x;
          if (m->stride_x) {
            const double want = b->merge_blocks_per_sm * nsm / std::max(1u, r.grid.y * r.grid.z) * (gx / gsum);
            gx = (unsigned)std::max(1.0, std::min((double)gx, std::ceil(want)));
          }
          MergeSeg sg{(unsigned)start, gx, r.grid.y, r.grid.z};
          memcpy(L.params.data() + m->off_seg + q * sizeof(MergeSeg), &sg, sizeof(sg));
          memcpy(L.params.data() + m->off_args + q * m->argsize, r.args.data(), m->argsize);
          start += (unsigned long long)gx * r.grid.y * r.grid.z;
          L.smem = std::max(L.smem, r.smem);
        }
        L.grid = dim3((unsigned)start, 1, 1);
        good = start > 0 && start <= 0x7fffffffULL;
        if (good && L.smem > 48 * 1024) {
          // the SM's ceiling, not this launch's need: launches of the same kernel at other positions need other
          // amounts, and the attribute is the function's
          cudaFuncAttributes fa;
          good = cudaFuncGetAttributes(&fa, L.fn) == cudaSuccess && L.smem + fa.sharedSizeBytes <= 227 * 1024 &&
                 cudaFuncSetAttribute(L.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(227 * 1024 - fa.sharedSizeBytes)) == cudaSuccess;
          if (!good) cudaGetLastError();
        }
        chain.push_back(std::move(L));
      }
      if (!good) continue;   // these contexts keep their own launches
      chains.push_back(std::move(chain));
      members.emplace_back(g.begin() + c0, g.begin() + c0 + n);
    }
  }
}

// Replaces, in the captured batch graph g, the nodes of the contexts that merge by chains of merged launches.  The
// branches of the batch graph are independent (each starts at the fork and ends at the join), so a context's nodes
// can be removed without touching the others.  A chain whose nodes the graph refuses is taken out again and its
// contexts keep their own nodes; returns the CUDA error of removing a node (then the graph is unusable).
static cudaError_t batch_merge(tdgl_batch_impl *b, int k, cudaGraph_t g) {
  std::vector<std::vector<MergedLaunch>> chains;
  std::vector<std::vector<int>> members;
  if (b->merge) merge_plan(b, k, chains, members);
  int served = 0, nchains = 0;
  cudaError_t e = cudaSuccess;
  for (size_t q = 0; q < chains.size() && e == cudaSuccess; q++) {
    std::vector<cudaGraphNode_t> made;
    cudaError_t ea = cudaSuccess;
    for (auto &L : chains[q]) {
      void *args[1] = {L.params.data()};
      cudaKernelNodeParams kp = {};
      kp.func = const_cast<void *>(L.fn);
      kp.gridDim = L.grid;
      kp.blockDim = L.block;
      kp.sharedMemBytes = (unsigned)L.smem;
      kp.kernelParams = args;
      cudaGraphNode_t nd = nullptr;
      const cudaGraphNode_t *dep = made.empty() ? nullptr : &made.back();
      if ((ea = cudaGraphAddKernelNode(&nd, g, dep, dep ? 1 : 0, &kp)) != cudaSuccess) break;
      made.push_back(nd);
    }
    if (ea != cudaSuccess) {   // this chain's contexts keep their own launches
      cudaGetLastError();
      for (cudaGraphNode_t nd : made) cudaGraphDestroyNode(nd);
      continue;
    }
    for (int i : members[q]) {
      for (cudaGraphNode_t nd : b->added[k][i])
        if ((e = cudaGraphDestroyNode(nd)) != cudaSuccess) break;
      b->glaunch[k][i] = 0;
      served++;
    }
    b->glaunch[k][members[q][0]] = (int)chains[q].size();   // the chain's launches, counted on its first context
    nchains++;
  }
  for (auto &t : b->tape[k]) t = Tape();
  for (auto &a : b->added[k]) a.clear();
  b->mchains[k] = nchains;
  b->mcontexts[k] = served;
  return e;
}

// captures one step of every context as graph k and launches it (the step it captured; the host effects of the step
// have run during the capture)
static int batch_capture(tdgl_batch_impl *b, int k) {
  Ctx *c0 = b->c[0];
  const int nc = (int)b->c.size();
  if (k == 0) {
    b->par0.resize(nc);
    for (int i = 0; i < nc; i++) b->par0[i] = b->c[i]->parity;
  }
  b->glaunch[k].assign(nc, 0);
  b->tape[k].assign(nc, Tape());
  b->added[k].assign(nc, {});
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return set_err(c0, TDGL_ECUDA, "batch capture", e);
  int rc = 0;
  // every context forks from the same point and joins back only after all are captured: the branches stay
  // independent (a join before the next fork would chain them)
  if ((e = cudaEventRecord(b->fork[0], b->stream)) != cudaSuccess) rc = set_err(c0, TDGL_ECUDA, "batch fork", e);
  std::vector<cudaGraphNode_t> before, after;
  for (int i = 0; i < nc && rc == 0; i++) {
    Ctx *ctx = b->c[i];
    if ((e = cudaStreamWaitEvent(ctx->stream, b->fork[0], 0)) != cudaSuccess) {
      rc = set_err(ctx, TDGL_ECUDA, "batch fork", e);
      break;
    }
    const bool seen = b->merge && capture_nodes(ctx->stream, before);
    ctx->capturing = true;
    if (seen) ctx->tape = &b->tape[k][i];
    const int l0 = ctx->launches;
    rc = step_body(ctx);
    ctx->capturing = false;
    if (rc == 0 && ctx->P.noise_on) TDGL_LAUNCH(ctx, K_COPY, 0.0, k_ss_advance, 1, 32, 0, ctx->ss_cur);
    ctx->tape = nullptr;
    if (rc) break;
    b->glaunch[k][i] = ctx->launches - l0;
    if (seen && capture_nodes(ctx->stream, after)) {   // the nodes this context's step added
      std::sort(before.begin(), before.end());
      for (cudaGraphNode_t nd : after)
        if (!std::binary_search(before.begin(), before.end(), nd)) b->added[k][i].push_back(nd);
    } else {
      b->tape[k][i].ok = false;
    }
  }
  for (int i = 0; i < nc; i++) {   // join every stream that joined the capture, also after an error
    Ctx *ctx = b->c[i];
    if ((e = cudaEventRecord(b->join[i], ctx->stream)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(b->stream, b->join[i], 0)) != cudaSuccess) {
      if (rc == 0) rc = set_err(ctx, TDGL_ECUDA, "batch join", e);
    }
  }
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(b->stream, &g);
  if (rc == 0 && e != cudaSuccess) rc = set_err(c0, TDGL_ECUDA, "batch capture end", e);
  if (rc == 0 && (e = batch_merge(b, k, g)) != cudaSuccess) rc = set_err(c0, TDGL_ECUDA, "batch merge", e);
  if (rc == 0 && (e = cudaGraphInstantiate(&b->exec[k], g, 0)) != cudaSuccess) rc = set_err(c0, TDGL_ECUDA, "batch instantiate", e);
  if (g) cudaGraphDestroy(g);
  if (rc) return rc;
  b->launches[k] = 0;
  for (int i = 0; i < nc; i++) b->launches[k] += b->glaunch[k][i];
  if ((e = cudaGraphLaunch(b->exec[k], b->stream)) != cudaSuccess) return set_err(c0, TDGL_ECUDA, "batch launch", e);
  return 0;
}

int tdgl_batch_create(tdgl_ctx *const *ctxs, int32_t n, tdgl_batch **out) {
  if (!ctxs || n < 1 || !out) return set_err(nullptr, TDGL_EINVAL, "batch: null argument or empty batch");
  tdgl_batch_impl *b = new tdgl_batch_impl();
  for (int i = 0; i < n; i++) {
    Ctx *ctx = reinterpret_cast<Ctx *>(ctxs[i]);
    if (!ctx || !ctx->have_state || !ctx->graphs || (ctx->P.solver == TDGL_SOLVER_PCG && !pcg_graphable(ctx))) {
      delete b;
      return set_err(nullptr, TDGL_EINVAL, "batch: every context needs a state, graphs on, maxit a multiple of 4");
    }
    for (Ctx *o : b->c)
      if (o == ctx) {
        delete b;
        return set_err(nullptr, TDGL_EINVAL, "batch: a context appears twice");
      }
    b->c.push_back(ctx);
  }
  b->fork.assign(n, nullptr);
  b->join.assign(n, nullptr);
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  for (int i = 0; i < n && e == cudaSuccess; i++) {
    e = cudaEventCreateWithFlags(&b->fork[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    tdgl_batch_destroy(reinterpret_cast<tdgl_batch *>(b));
    return set_err(nullptr, TDGL_ECUDA, "batch: stream or event creation", e);
  }
  *out = reinterpret_cast<tdgl_batch *>(b);
  return 0;
}

int tdgl_batch_destroy(tdgl_batch *bb) {
  tdgl_batch_impl *b = reinterpret_cast<tdgl_batch_impl *>(bb);
  if (!b) return 0;
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop(b);
  for (auto e : b->fork)
    if (e) cudaEventDestroy(e);
  for (auto e : b->join)
    if (e) cudaEventDestroy(e);
  if (b->done) cudaEventDestroy(b->done);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return 0;
}

static int batch_launch(tdgl_batch_impl *b, int m, const double *H, const double *HJ);

int tdgl_batch_steps(tdgl_batch *bb, int32_t n, const double *H, const double *HJ, int32_t wait) {
  tdgl_batch_impl *b = reinterpret_cast<tdgl_batch_impl *>(bb);
  if (!b || !H || !HJ || n < 0) return set_err(nullptr, TDGL_EINVAL, "batch_steps: bad argument");
  const int nc = (int)b->c.size();
  int rc = 0, done = 0;
  // lockstep warm-up until every context's step repeats
  for (; done < n; done++) {
    bool ready = true;
    for (Ctx *ctx : b->c) ready = ready && graph_ready(ctx);
    if (ready) break;
    if (done >= 8) return set_err(b->c[0], TDGL_ECUDA, "batch: the steps did not settle");
    for (int i = 0; i < nc; i++)
      if ((rc = run_steps(b->c[i], 1, H[i], nullptr, HJ[i], false))) return rc;
  }
  if (done < n) {
    if ((rc = batch_launch(b, n - done, H, HJ))) return rc;
  }
  if (!wait) return 0;
  int status = 0;
  for (Ctx *ctx : b->c) {
    TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
    const int st = deferred_status(ctx);
    if (st && !status) status = st;
  }
  return status;
}

// The open update of an open-boundary context before batch step q of this call, and that step's scalars (slot q of
// its pinned scalars) into its device scalars; the batch stream then follows the context's stream.
static int batch_open_step(tdgl_batch_impl *b, int i, int q, double H, double HJ) {
  Ctx *ctx = b->c[i];
  int rc;
  if ((rc = open_update(ctx, HJ))) return rc;
  StepScal &v = ctx->ss_host[q];
  v.H = H;
  v.HJ = HJ;
  v.open_fr = open_fraction(ctx);
  v.noise_step = (unsigned long long)(ctx->P.noise_step0 + ctx->steps);
  TDGL_CUDA(cudaMemcpyAsync(ctx->ss_cur, &v, sizeof(StepScal), cudaMemcpyHostToDevice, ctx->stream));
  TDGL_CUDA(cudaEventRecord(b->fork[i], ctx->stream));
  TDGL_CUDA(cudaStreamWaitEvent(b->stream, b->fork[i], 0));
  return 0;
}

// m steps of a settled batch: captured steps first (one per parity), then graph launches
static int batch_launch(tdgl_batch_impl *b, int m, const double *H, const double *HJ) {
  const int nc = (int)b->c.size();
  int rc = 0;
  bool any_open = false;
  // this call's H, HJ and the noise index of its next step into every context's device scalars (an open-boundary
  // context: after its open update); the batch stream then follows every context's stream
  for (int i = 0; i < nc; i++) {
    Ctx *ctx = b->c[i];
    const bool open = ctx->P.selffield_bc == TDGL_BC_OPEN;
    any_open = any_open || open;
    if ((rc = ss_reserve(ctx, open ? m : 1))) return rc;
    ctx->ss_last_ok = false;   // the batch graph advances the noise index on the device
    ctx->launches = 0;
    if (open) {
      if ((rc = batch_open_step(b, i, 0, H[i], HJ[i]))) return rc;
    } else {
      StepScal &v = ctx->ss_host[0];
      v.H = H[i];
      v.HJ = HJ[i];
      v.open_fr = 0.0;
      v.noise_step = (unsigned long long)(ctx->P.noise_step0 + ctx->steps);
      TDGL_CUDA(cudaMemcpyAsync(ctx->ss_cur, &v, sizeof(StepScal), cudaMemcpyHostToDevice, ctx->stream));
      TDGL_CUDA(cudaEventRecord(b->fork[i], ctx->stream));
      TDGL_CUDA(cudaStreamWaitEvent(b->stream, b->fork[i], 0));
    }
  }
  // the batch graphs serve while every context has flipped parity together since they were captured
  if (b->exec[0])
    for (int i = 0; i < nc; i++)
      if ((b->c[i]->parity ^ b->par0[i]) != (b->c[0]->parity ^ b->par0[0])) {
        batch_drop(b);
        break;
      }
  for (int q = 0; q < m; q++) {
    if (any_open && q > 0) {
      // each open context's update waits for the previous batch step (the recomputation reads the state) and the
      // next batch step for the update
      Ctx *ctx = b->c[0];   // (the context that carries an error message)
      TDGL_CUDA(cudaEventRecord(b->done, b->stream));
      for (int i = 0; i < nc; i++) {
        ctx = b->c[i];
        if (ctx->P.selffield_bc != TDGL_BC_OPEN) continue;
        TDGL_CUDA(cudaStreamWaitEvent(ctx->stream, b->done, 0));
        if ((rc = batch_open_step(b, i, q, H[i], HJ[i]))) return rc;
      }
    }
    if (!b->exec[0]) {
      if ((rc = batch_capture(b, 0))) return rc;
    } else if (!b->exec[1] && b->c[0]->parity != b->par0[0]) {
      if ((rc = batch_capture(b, 1))) return rc;
    } else {
      const int k = b->c[0]->parity ^ b->par0[0];
      cudaError_t e = cudaGraphLaunch(b->exec[k], b->stream);
      if (e != cudaSuccess) return set_err(b->c[0], TDGL_ECUDA, "batch graph launch", e);
      for (int i = 0; i < nc; i++) {
        Ctx *ctx = b->c[i];
        ctx->launches += b->glaunch[k][i];
        advance_swap(ctx);
        ctx->steps++;
      }
    }
  }
  Ctx *ctx = b->c[0];   // (the context that carries an error message)
  TDGL_CUDA(cudaEventRecord(b->done, b->stream));
  for (Ctx *cx : b->c) {
    TDGL_CUDA(cudaStreamWaitEvent(cx->stream, b->done, 0));
    TDGL_CUDA(cudaEventRecord(cx->ss_done, cx->stream));   // the pinned scalars are free again after this
    cx->ss_pending = true;
  }
  return 0;
}

int tdgl_batch_info(const tdgl_batch *bb, int32_t *one_graph) {
  const tdgl_batch_impl *b = reinterpret_cast<const tdgl_batch_impl *>(bb);
  if (!b) return TDGL_EINVAL;
  if (one_graph) *one_graph = b->exec[0] ? 1 : 0;
  return 0;
}

int tdgl_batch_set_merge(tdgl_batch *bb, int32_t on, double blocks_per_sm) {
  tdgl_batch_impl *b = reinterpret_cast<tdgl_batch_impl *>(bb);
  if (!b || !(blocks_per_sm >= 0.0) || blocks_per_sm > 1024.0) return set_err(nullptr, TDGL_EINVAL, "batch_set_merge: bad argument");
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop(b);   // the next step captures again
  b->merge = on != 0;
  if (blocks_per_sm > 0.0) b->merge_blocks_per_sm = blocks_per_sm;
  return 0;
}

int tdgl_batch_merge_info(const tdgl_batch *bb, int32_t *contexts, int32_t *chains, int32_t *launches_per_step) {
  const tdgl_batch_impl *b = reinterpret_cast<const tdgl_batch_impl *>(bb);
  if (!b) return TDGL_EINVAL;
  if (contexts) *contexts = b->exec[0] ? b->mcontexts[0] : 0;
  if (chains) *chains = b->exec[0] ? b->mchains[0] : 0;
  if (launches_per_step) *launches_per_step = b->exec[0] ? b->launches[0] : 0;
  return 0;
}

int tdgl_steps(tdgl_ctx *c, int32_t n, double H, double HJ) { return run_steps(reinterpret_cast<Ctx *>(c), n, H, nullptr, HJ, true); }

int tdgl_steps_ramp(tdgl_ctx *c, int32_t n, double H, const double *HJ) {
  if (!HJ) return TDGL_EINVAL;
  return run_steps(reinterpret_cast<Ctx *>(c), n, H, HJ, 0.0, true);
}

int tdgl_steps_async(tdgl_ctx *c, int32_t n, double H, double HJ) { return run_steps(reinterpret_cast<Ctx *>(c), n, H, nullptr, HJ, false); }

int tdgl_sync(tdgl_ctx *c) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx) return TDGL_EINVAL;
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return deferred_status(ctx);
}

int tdgl_set_graphs(tdgl_ctx *c, int32_t on) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx) return TDGL_EINVAL;
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  drop_graphs(ctx);
  ctx->graphs = on != 0;
  return 0;
}

int tdgl_set_branches(tdgl_ctx *c, int32_t on) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx) return TDGL_EINVAL;
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  drop_graphs(ctx);
  ctx->branches = on != 0;
  return 0;
}

void *tdgl_stream(tdgl_ctx *c) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  return ctx ? (void *)ctx->stream : nullptr;
}

int tdgl_device_state(tdgl_ctx *c, tdgl_state_view *dev) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !dev) return TDGL_EINVAL;
  memset(dev, 0, sizeof(*dev));
  for (int mu = 0; mu < ctx->N; mu++) {
    dev->G[mu] = (double *)ctx->G[mu];
    dev->F[mu] = (double *)ctx->F[mu];
  }
  for (int ax = 0; ax < 3; ax++) {
    dev->th[ax] = ctx->th[ax]; dev->ph[ax] = ctx->ph[ax];
    dev->U[ax] = (double *)ctx->U[ax]; dev->V[ax] = (double *)ctx->V[ax];
    dev->J[ax] = ctx->J[ax]; dev->h[ax] = ctx->h[ax];
  }
  return 0;
}

int tdgl_field_solve(tdgl_ctx *c) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx) return TDGL_EINVAL;
  if (!ctx->have_state) return set_err(ctx, TDGL_ESTATE, "no state uploaded");
  ctx->launches = 0;
  int rc = 0;
  switch (ctx->P.solver) {
    case TDGL_SOLVER_SEP: sep_implicit(ctx); break;
    case TDGL_SOLVER_PCG: rc = pcg_implicit(ctx); break;
    case TDGL_SOLVER_SCALE: scale_increment(ctx); break;
    default: break;
  }
  if (rc) return rc;
  TDGL_CUDA(cudaStreamSynchronize(ctx->stream));
  return deferred_status(ctx);
}

int tdgl_sep_apply(tdgl_ctx *c, const double *b, double *z, int32_t f32) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !b || !z) return TDGL_EINVAL;
  if (!ctx->sep) return set_err(ctx, TDGL_EINVAL, "no separable solve in this context");
  if (f32 && !(ctx->P.solver == TDGL_SOLVER_PCG && ctx->P.pcg_f32)) return set_err(ctx, TDGL_EINVAL, "no FP32 preconditioner");
  // packed host ranges → plane-major device arrays → solve → back (through the PCG carry helpers' layout)
  const long long nn = ctx->g.d.n();
  double *d[3] = {nullptr, nullptr, nullptr};
  cudaError_t e = cudaSuccess;
  for (int q = 0; q < 3 && e == cudaSuccess; q++) {
    e = cudaMalloc(&d[q], nn * sizeof(double));
    if (e == cudaSuccess) e = cudaMemsetAsync(d[q], 0, nn * sizeof(double), ctx->stream);
  }
  if (e == cudaSuccess) {
    int rc = pm_from_packed_host(ctx, d, b);
    if (!rc) {
      sep_apply(ctx, d, d, f32 != 0, nullptr);
      rc = pm_to_packed_host(ctx, d, z);
    }
    for (int q = 0; q < 3; q++) cudaFree(d[q]);
    return rc;
  }
  for (int q = 0; q < 3; q++)
    if (d[q]) cudaFree(d[q]);
  return set_err(ctx, TDGL_ECUDA, "sep_apply", e);
}

int tdgl_profile(tdgl_ctx *c, int32_t on) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx) return TDGL_EINVAL;
  prof_collect(ctx);
  Prof &p = ctx->prof;
  for (int q = 0; q < K_NCAT; q++) {
    p.ms[q] = 0;
    p.bytes[q] = 0;
    p.n[q] = 0;
  }
  p.on = on != 0;
  return 0;
}

int tdgl_profile_read(tdgl_ctx *c, int32_t cat, const char **name, int64_t *launches, double *ms, double *bytes) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx) return TDGL_EINVAL;
  if (cat < 0) return K_NCAT;
  if (cat >= K_NCAT) return TDGL_EINVAL;
  prof_collect(ctx);
  const Prof &p = ctx->prof;
  if (name) *name = kcat_name[cat];
  if (launches) *launches = p.n[cat];
  if (ms) *ms = p.ms[cat];
  if (bytes) *bytes = p.bytes[cat];
  return 0;
}

int tdgl_get_stats(tdgl_ctx *c, tdgl_stats *out) {
  Ctx *ctx = reinterpret_cast<Ctx *>(c);
  if (!ctx || !out) return TDGL_EINVAL;
  out->steps = ctx->steps;
  long long tot = 0;
  out->pcg_last_iters = ctx->pcg ? pcg_iters(ctx, &tot) : 0;
  out->pcg_total_iters = tot;
  out->open_recomputes = ctx->open_recomputes;
  out->kernel_launches_last_call = ctx->launches;
  out->qp_cg_total_iters = qp_cg_iterations(ctx);
  return 0;
}

}  // extern "C"
