/*
 * tdgl_b200.h — C-ABI of the B200 stepper of the gtdgl (juliaTDGL 2) ladder cycle.
 *
 * The library advances the state of gtdgl's `TDGL.step!` (gtdgl/src/step.jl:13-35) n steps on one GPU.  It is
 * the device side of the accelerator hook `TDGL.STEPS[]` (gtdgl/src/protocol.jl:305-316): the host (Julia's
 * `Stepper`, or the Python mirror in juliatdgl_b200/) decides dt, the stage counts and every coefficient, as
 * gtdgl/src/scheme.jl:250-434 does, and passes them here; the library keeps the state resident in HBM between
 * calls and copies it to and from host buffers on request.
 *
 * Conventions
 *   - Arrays are column-major with the reference's shapes (i fastest), exactly the memory of Julia's
 *     Array{Float64,3} / Array{ComplexF64,3}.  Complex arrays are interleaved (re, im) doubles.
 *     Node arrays (Nx+1, Ny+1, Nz+1); x links (Nx, Ny+1, Nz+1); y links (Nx+1, Ny, Nz+1); z links
 *     (Nx+1, Ny+1, Nz); hx (Nx+1, Ny, Nz); hy (Nx, Ny+1, Nz); hz (Nx, Ny, Nz+1)   (gtdgl/src/state.jl:13-22).
 *   - Grid indices x1..z2 are the reference's 1-based block bounds (gtdgl/src/grid.jl:9-27).
 *   - Every entry point returns 0 on success or a negative TDGL_E* code; tdgl_last_error() gives the message.
 *     Calls on one context are single-threaded; contexts are independent (one CUDA stream each).
 *   - The library owns device memory; the caller owns every host buffer it passes.
 */
#ifndef TDGL_B200_H
#define TDGL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDGL_ABI_VERSION 8
#define TDGL_MAXB 8      /* bands */
#define TDGL_MAXSTG 64   /* RKL / RKC stages per band */
#define TDGL_MAXMAT 8    /* materials per region */

enum {
  TDGL_OK = 0,
  TDGL_EINVAL = -1,       /* invalid or unsupported parameters */
  TDGL_ENOMEM = -2,       /* device allocation failed */
  TDGL_ECUDA = -3,        /* CUDA runtime error */
  TDGL_ENOCONV = -4,      /* the PCG solve reached maxit without meeting its tolerance */
  TDGL_EDIVERGED = -5,    /* a non-finite value appeared in the state */
  TDGL_ESTATE = -6        /* no state uploaded yet */
};

/* field solve (gtdgl/src/step.jl:26-30) */
enum { TDGL_SOLVER_EXPLICIT = 0, TDGL_SOLVER_SCALE = 1, TDGL_SOLVER_SEP = 2, TDGL_SOLVER_PCG = 3 };
/* outer-face condition of the injected current (gtdgl/src/scheme.jl:208-214) */
enum { TDGL_BC_SLAB = 0, TDGL_BC_BAR = 1, TDGL_BC_OPEN = 2 };

typedef struct tdgl_grid {
  int32_t Nx, Ny, Nz;                 /* cells, padding included */
  int32_t x1, x2, y1, y2, z1, z2;     /* 1-based block bounds */
  double dx, dy, dz;
} tdgl_grid;

/* BandCoef (gtdgl/src/scheme.jl:21-28) */
typedef struct tdgl_bandcoef {
  double kx, ky, kz;                  /* rx/(m_x Γh), … */
  double c;                           /* dt/Γ */
  double eps;                         /* ε = a − T */
  double beta;
  double gamma2;                      /* γ̃² of KWT (0 = plain TDGL) */
  double cpl[TDGL_MAXB];              /* (dt/Γh) γ_µν */
} tdgl_bandcoef;

/* Material per region (MatField, gtdgl/src/materials.jl:28-39, built at gtdgl/src/scheme.jl:368-372): each node
 * takes the band coefficients of its material; each link of band µ the weight ρ = τ·(m_ref/m_link)·t_ab (0 where the
 * band is absent from either end), with m_link = (m_a + m_b)/2 along the link's axis, m_ref the first material's
 * mass and t_ab the transparency of the pair (materials.jl:97-110).  The library forms ρ from idx, τ and these tables
 * on the fly.  Material 1 is the Stepper's model: its entries equal bc / bcs. */
typedef struct tdgl_materials {
  int32_t nmat;                                   /* materials, 1..TDGL_MAXMAT */
  const uint8_t *idx;                             /* node array: the material of each node, 1..nmat */
  tdgl_bandcoef full[TDGL_MAXMAT][TDGL_MAXB];     /* MatField.full: full-step coefficients per material and band */
  tdgl_bandcoef stage[TDGL_MAXMAT][TDGL_MAXB];    /* MatField.stage: per (sub)stage, divided as bcs */
  double ma[TDGL_MAXMAT][TDGL_MAXB][3];           /* band masses along x, y, z (Band.ma) */
  double transparency[TDGL_MAXMAT][TDGL_MAXMAT];  /* MatField.t: symmetric, ones on the diagonal */
  int32_t absent[TDGL_MAXMAT][TDGL_MAXB];         /* MatField.absent: band µ absent from material m */
  double gamma[TDGL_MAXMAT][TDGL_MAXB];           /* Γ of each material's bands (the noise kick, noise.jl:101-180) */
  /* ABI v7, the heat model with materials (terms.jl _heat_step_mat!; bands.jl:65-66): per material the a of each
   * band (ε = a − θ), its γ̃ (the heat source), σn (the Joule heat) and D_T (MatField.a, .DT, materials.jl:37-38) */
  double a[TDGL_MAXMAT][TDGL_MAXB];
  double gk[TDGL_MAXMAT][TDGL_MAXB];
  double sigma_n[TDGL_MAXMAT];
  double heat_DT[TDGL_MAXMAT];
} tdgl_materials;

/* Everything the Stepper holds that the step reads (gtdgl/src/scheme.jl:167-198). Host pointers are read
 * during tdgl_ctx_create only. */
typedef struct tdgl_params {
  int32_t abi_version;                /* TDGL_ABI_VERSION */
  int32_t nbands;                     /* N, 1..TDGL_MAXB */
  tdgl_grid grid;
  double dt;
  int32_t nsub[TDGL_MAXB];            /* Euler substeps per band (used when stages == 0) */
  int32_t stages[TDGL_MAXB];          /* RKL1 / RKC1 stages per band (0 = Euler with nsub substeps) */
  int32_t use_rkc[TDGL_MAXB];         /* 1: the band's stages take the RKC weights below */
  double rkc_q[TDGL_MAXB];            /* RKCCoef.q */
  double rkc_mu[TDGL_MAXB][TDGL_MAXSTG];
  double rkc_nu[TDGL_MAXB][TDGL_MAXSTG];
  double rkc_c[TDGL_MAXB][TDGL_MAXSTG];
  double rkc_sk[TDGL_MAXB][2];        /* SK-ROCK weights (ν₁, κ₁) */
  tdgl_bandcoef bc[TDGL_MAXB];        /* full-step coefficients */
  tdgl_bandcoef bcs[TDGL_MAXB];       /* per (sub)stage coefficients */
  double wa[3][TDGL_MAXB];            /* supercurrent weight g_µ along x, y, z */
  /* FieldCoef (gtdgl/src/scheme.jl:149-153) */
  double d1, sxy, sxz, syx, syz, szx, szy, a_imp;
  int32_t solver;                     /* TDGL_SOLVER_* */
  int32_t selffield_bc;               /* TDGL_BC_* */
  int32_t extrap, rotframe, hard;
  /* masks, node-shaped (gtdgl/src/grid.jl:35-45) */
  const double *f, *taux, *tauy, *tauz;
  /* σ_l/σ_n per link (SCALE and PCG solvers), link-shaped; NULL otherwise */
  const double *Dx, *Dy, *Dz;
  /* bar field per unit HJ (gtdgl/src/field.jl:173-178; BAR and OPEN): (Ny+1)×2, 2×Nz, Ny×2, 2×(Nz+1),
   * Ny×(Nz+1), (Ny+1)×Nz, column-major */
  const double *bar_hy_z, *bar_hy_y, *bar_hz_z, *bar_hz_y, *bar_hz_x, *bar_hy_x;
  /* PCGSolver (gtdgl/src/implicit.jl:142-189) */
  double pcg_tol;
  int32_t pcg_maxit, pcg_fast, pcg_f32, pcg_extrap;
  /* OpenBC (gtdgl/src/openbc.jl:100-136) */
  int32_t open_every, open_R;
  double kappa2;                      /* κ² */
  double open_fac;                    /* dx³/κ² */
  const double *open_green;           /* lattice Green table, (R+1)³ column-major */
  const double *open_jbar;            /* (Ny+1)×(Nz+1) */
  /* thermal noise (gtdgl/src/noise.jl): Langevin kicks of T̃ = noise_T on every band (and on the link phases with
   * noise_field), drawn from a counter-based Philox4x32-10 stream: the two normals of (node, band) at step n are a pure
   * function of (noise_seed, noise_step0 + n, band, node), so a run continues its stream from any step. */
  int32_t noise_on, noise_field;
  double noise_T;
  uint64_t noise_seed;
  double noise_gamma[TDGL_MAXB];      /* Γ_µ of each band (model.jl:26-33) */
  double noise_sigma_n;               /* σn of the field kick (noise.jl:183-198) */
  int64_t noise_step0;                /* the stream index of this context's first step */
  const tdgl_materials *materials;    /* null: one material (Stepper.mt === nothing) */
  /* A sculpted sample (a shape with vacuum, Masks.vac after sculpt!, gtdgl/src/geometry.jl:537-557): node array,
   * nonzero on the vacuum nodes.  The band update holds them at Ψ = 0 and reads each neighbour with the mask of its
   * link (τ, or ρ with materials; bands.jl:103-124), the Neumann ghosts of the vacuum are zeroed (field.jl:235-244)
   * and the noise skips them.  Null: no vacuum. */
  const uint8_t *vac;
  /* ABI v5: the interband drag (gtdgl/src/scheme.jl:404-413; in the band equation bands.jl:37-51, in the
   * supercurrent field.jl:73-81).  drag_on = 0: none (Stepper.drag === nothing).  drag_c[µ][ν] = Stepper.drag[µ][ν],
   * the full-step coefficients (x, y, z) of band ν's lattice Laplacian in band µ's equation (a pass of n substeps or
   * an RKL/RKC stage of weight q divides them by n or q, bands.jl:195-196); drag_nu[µ][ν] = Stepper.dragν[µ][ν], the
   * symmetric drag matrix of the supercurrent.  One material without vacuum, as the reference (scheme.jl:384,
   * materials.jl:75). */
  int32_t drag_on;
  double drag_c[TDGL_MAXB][TDGL_MAXB][3];
  double drag_nu[TDGL_MAXB][TDGL_MAXB];
  /* ABI v6: the heat model (gtdgl/src/terms.jl, Heat and heat_step! with one material): the temperature field θ
   * above the bath, ε_µ = a_µ − θ in the band equation (bands.jl:33-35), θ stepped after the supercurrent by an
   * in-place lexicographic sweep (terms.jl:58-130).  heat_on = 0: none.  One material without vacuum.  θ itself
   * travels in the carry (tdgl_carry_view.heat_theta), as TDGLGPU keeps Stepper.heat.θ beside the state. */
  int32_t heat_on, heat_joule, heat_margin;
  double heat_DT, heat_gamma_bath, heat_eta, heat_cap;
  double heat_T, heat_sigma_n;            /* the bath (Model.T) and σn (the Joule heat σn|E|²) */
  double heat_a[TDGL_MAXB];               /* a_µ of each band (ε = a − θ) */
  double heat_Gamma[TDGL_MAXB], heat_gk[TDGL_MAXB];   /* Γ_µ and γ̃_µ of the heat source (_band_heat) */
  /* ABI v8: normal fluids per band (gtdgl/src/exchange.jl).  qp_on = 0: one normal fluid (Stepper.qpx === nothing).  qp_on = 1, two bands (QPExchange): each
   * step, before the bands, δ = μ_π − μ_σ solves σn∇²δ − λ0 δ = C_π/s_π − C_σ/s_σ on the region of δ (qp_potential!);
   * after the bands each band turns by e^{−iμ_µ dt}, μ_σ = −s_π δ, μ_π = s_σ δ (qp_turn!).  qp_on = 2, N fluids
   * (QPExchangeN): R_µ = C_µ/s_µ − Σ_ν C_ν, the modes m_k = Σ_µ qp_Pinv[k][µ] R_µ each solve σn∇²m_k − qp_lam[k] m_k
   * = m_k's source, μ_µ = Σ_k qp_P[µ][k] m_k, and band µ turns by e^{−i dt μ_µ}.  C_µ is the conversion of band µ
   * from the state at the start of the step (_conv).  The region of δ (or μ): x nodes 2..Nx (0 on the x faces), y
   * nodes qp_j0 .. qp_j0+qp_nj−1, z nodes qp_k0 .. qp_k0+qp_nk−1 (Neumann).  The separable solve takes the eigenbases
   * of the three 1D second differences as the reference holds them: V (columns), W = V⁻¹ and the eigenvalues e,
   * n × n column-major (x: n = Nx−1, Dirichlet; y: n = qp_nj, z: n = qp_nk, Neumann).  With the heat model's Joule
   * term the fluids add σn Σ_µ s_µ|∇μ_µ|² + Σ_{µ<ν} G_µν(μ_µ − μ_ν)² to its source (qp_joule, terms.jl:107-109). */
  int32_t qp_on;
  double qp_s[TDGL_MAXB];                 /* the shares of σn of the bands' normal fluids */
  double qp_sigma_n, qp_lambda0;          /* σn; λ0 = G (1/s_σ + 1/s_π) of the two-band form */
  double qp_g[TDGL_MAXB][3];              /* each band's stiffness along x, y, z (stiffness(b, i)) */
  double qp_gamma[TDGL_MAXB][TDGL_MAXB];  /* Model.γ (the Josephson terms of _conv) */
  double qp_P[TDGL_MAXB][TDGL_MAXB];      /* N fluids: QPExchangeN.P (μ = P m) */
  double qp_Pinv[TDGL_MAXB][TDGL_MAXB];   /* N fluids: QPExchangeN.Pinv (m = Pinv μ) */
  double qp_lam[TDGL_MAXB];               /* N fluids: QPExchangeN.λ, the eigenvalues of S⁻¹L */
  double qp_Gm[TDGL_MAXB][TDGL_MAXB];     /* the exchange conductances of the Joule heat (qp_joule, with the heat
                                             model's Joule term): QPExchangeN.Gm, or QPExchange.G in [0][1] */
  int32_t qp_j0, qp_nj, qp_k0, qp_nk;     /* the region along y and z (1-based first node, extent) */
  const double *qp_Vx, *qp_Wx, *qp_ex;    /* the 1D bases (Vx, Wx, ex of QPExchange / QPExchangeN) */
  const double *qp_Vy, *qp_Wy, *qp_ey;
  const double *qp_Vz, *qp_Wz, *qp_ez;
  /* A sculpted sample or materials whose σn, exchange or fluids differ (two bands): the unknowns of the region
   * ((Nx−1) × qp_nj × qp_nk, column-major): 1 free, 0 cut (no conductor), 2 held at δ = 0 (a one-fluid material);
   * QPSolve.cond, or QPVar.typ.  δ then solves its equation by conjugate gradients preconditioned by the separable
   * solve (_qp_cg!, _qp_cg_var!, exchange.jl:87-121, 258-290) to the relative tolerance qp_tol in at most qp_maxit
   * iterations, started cold every step.  With qp_cx (QPVar) the equation has the variable coefficients σ_l/h² of
   * the region's links (qp_cx: (Nx) × qp_nj × qp_nk, the two x ends included; qp_cy: (Nx−1) × (qp_nj−1) × qp_nk;
   * qp_cz: (Nx−1) × qp_nj × (qp_nk−1)), λ per unknown (qp_lamv) and qp_d on the decoupled unknowns; without, the
   * cut links of a sculpted sample with σn and λ0.  Null: the separable solve. */
  const uint8_t *qp_cond;
  double qp_tol;
  int32_t qp_maxit;
  const double *qp_cx, *qp_cy, *qp_cz, *qp_lamv;
  double qp_d;
  /* With materials (two bands): each material's Josephson matrix Model.γ (the terms of _conv at its nodes); the
   * link weights of _conv are the band stage's, τ·W from the node map. */
  double qp_mgamma[TDGL_MAXMAT][2][2];
} tdgl_params;

/* Host buffers of every field of `State` (gtdgl/src/state.jl:13-22). */
typedef struct tdgl_state_view {
  double *G[TDGL_MAXB], *F[TDGL_MAXB];   /* complex, node-shaped */
  double *th[3], *ph[3];                 /* θ, φ: x, y, z links */
  double *U[3], *V[3];                   /* complex links */
  double *J[3];                          /* supercurrent, links */
  double *h[3];                          /* hx, hy, hz */
} tdgl_state_view;

/* The Stepper-side state the hook must carry across cycles (gtdgl/src/protocol.jl:635-663): the PCG warm
 * start (gtdgl/src/implicit.jl:142-169; x and xprev over the ranges of the separable solve, packed per
 * component x, y, z) and the open-boundary ramp (gtdgl/src/openbc.jl:100-109; h-shaped old/new, link-shaped θ). */
typedef struct tdgl_carry_view {
  double *pcg_x;                         /* sum of the three range sizes */
  double *pcg_xprev;
  int32_t pcg_warm, pcg_have2;
  int32_t open_count;
  double *open_old[3], *open_new[3];
  double *open_theta[3];
  double *heat_theta;                    /* node-shaped temperature field (ABI v6; null: not carried) */
} tdgl_carry_view;

typedef struct tdgl_stats {
  int64_t steps;                         /* steps taken by this context */
  int32_t pcg_last_iters;                /* iterations of the last PCG solve */
  int64_t pcg_total_iters;
  int32_t open_recomputes;               /* open-boundary recomputations */
  int32_t kernel_launches_last_call;     /* kernels launched by the last tdgl_steps call */
  int64_t qp_cg_total_iters;             /* CG iterations of the two fluids' δ solve in a sculpted sample (ABI v8) */
} tdgl_stats;

typedef struct tdgl_ctx tdgl_ctx;

/* Replaces GPUStepper(st, backend) (gpu/TDGLGPU/src/TDGLGPU.jl:2039-2071 set-up): copies the coefficients,
 * masks and tables to the device and allocates the state and the workspaces. */
int tdgl_ctx_create(const tdgl_params *p, tdgl_ctx **out);
int tdgl_ctx_destroy(tdgl_ctx *ctx);

/* Replaces device_state / device_state! (gpu/TDGLGPU/src/TDGLGPU.jl:63-74): host State → device. */
int tdgl_upload_state(tdgl_ctx *ctx, const tdgl_state_view *s);
/* Replaces host_state! (gpu/TDGLGPU/src/TDGLGPU.jl:77-82): device → host State (every field). */
int tdgl_download_state(tdgl_ctx *ctx, const tdgl_state_view *s);

/* The carry of the PCG warm start and the open ramp (gpu/TDGLGPU/src/TDGLGPU.jl:2130-2135 _pcg_up!/_pcg_down!,
 * _open_up!).  NULL pointers in the view are skipped. */
int tdgl_set_carry(tdgl_ctx *ctx, const tdgl_carry_view *c);
int tdgl_get_carry(tdgl_ctx *ctx, const tdgl_carry_view *c);

/* Replaces gpu_steps!(g, gs, n; H, HJ) (gpu/TDGLGPU/src/TDGLGPU.jl:2065-2071): n steps of step!(s, st; H, HJ),
 * returning after the device has finished. */
int tdgl_steps(tdgl_ctx *ctx, int32_t n, double H, double HJ);
/* n steps with HJ[q] at step q (a current ramp); the same as n calls of tdgl_steps(ctx, 1, H, HJ[q]). */
int tdgl_steps_ramp(tdgl_ctx *ctx, int32_t n, double H, const double *HJ);
/* Enqueue n steps on the context's stream without waiting (tdgl_sync waits, and returns TDGL_ENOCONV if a PCG
 * solve of the enqueued steps reached maxit). */
int tdgl_steps_async(tdgl_ctx *ctx, int32_t n, double H, double HJ);
int tdgl_sync(tdgl_ctx *ctx);
/* Steps as CUDA graphs (default on): once a step launches the same kernels as the last one of its θ/φ parity (after
 * the PCG warm start has settled), it is captured once per parity, the PCG loop as a conditional node, and replayed
 * as one graph launch with the step's H, HJ, ramp fraction and noise index read from device memory.  The same
 * kernels run in the same order: results are identical with and without.  0 turns it off (and drops the graphs). */
int tdgl_set_graphs(tdgl_ctx *ctx, int32_t on);
/* Parallel branches inside a step (default on): the bands of a step side by side, each on its own stream, and the
 * PCG's x update and r·z_old beside its preconditioner.  They fill the GPU when one context runs alone; a caller that
 * keeps many contexts in flight at once (continuous batching) may turn them off, so that the device's queues hold
 * one chain per context.  Results are identical either way.  Drops the captured graphs. */
int tdgl_set_branches(tdgl_ctx *ctx, int32_t on);

/* Snapshots on the device (the delay confirmation of the ladder, gtdgl/src/protocol.jl:222-262: continue an earlier
 * rung from its start): a slot holds the state, the PCG warm start and extrapolation history, the open boundary's
 * ramp and the step count (the noise index).  restore puts them back; the steps that follow repeat the ones that
 * followed the take, to the bit.  Slots 0..255, allocated on first use. */
int tdgl_snapshot_take(tdgl_ctx *ctx, int32_t slot);
int tdgl_snapshot_restore(tdgl_ctx *ctx, int32_t slot);
int tdgl_snapshot_free(tdgl_ctx *ctx, int32_t slot);
/* Device memory held by the context (its arrays, staging and snapshots), for admission against an HBM budget. */
int64_t tdgl_device_bytes(const tdgl_ctx *ctx);

/* Batches (config: many uneven grids stepped together): the contexts (each with its state uploaded; graphs on)
 * advance in lockstep.  An open-boundary context takes its open update (ramp count, recomputation when due) on its
 * own stream before each batch step.  After the first steps, once each context's step is captured for both θ/φ
 * parities, one graph holds every context's step as an independent branch and one launch advances the whole
 * batch by a step; the device runs the branches concurrently.  Contexts whose steps launch only kernels (no PCG
 * loop, no copies) and the same sequence of kernels are merged: they share one launch per kernel (each block runs
 * the body of its own context's launch), so that their step is a few dozen launches whatever their number.  Each
 * context keeps its own results: a run in a batch gives the bits it gives alone, merged or not.  H[i], HJ[i]: the applied field and self-field of context i for these n steps.
 * wait = 0 returns after enqueuing (each context's stream then follows the batch). */
typedef struct tdgl_batch tdgl_batch;
int tdgl_batch_create(tdgl_ctx *const *ctxs, int32_t n, tdgl_batch **out);
int tdgl_batch_steps(tdgl_batch *batch, int32_t n, const double *H, const double *HJ, int32_t wait);
int tdgl_batch_info(const tdgl_batch *batch, int32_t *one_graph);   /* 1: one graph launch per batch step */
/* Merging on (default) or off, and the launch shape of the kernels whose blocks stride over planes: their merged
 * x-grid holds about blocks_per_sm blocks per SM in all (0: keep the current value; default 4).  The batch captures
 * its step again at the next call. */
int tdgl_batch_set_merge(tdgl_batch *batch, int32_t on, double blocks_per_sm);
/* Of the captured batch step: contexts served by merged launches; chains of merged launches (groups of contexts
 * with the same kernels, cut to what one launch holds); kernel launches of a batch step in all. */
int tdgl_batch_merge_info(const tdgl_batch *batch, int32_t *contexts, int32_t *chains, int32_t *launches_per_step);
int tdgl_batch_destroy(tdgl_batch *batch);

/* The context's CUDA stream (cudaStream_t) and the device pointers of its state (for timing with events on
 * that stream and for device-resident drivers).  Pointers stay valid until the next step swaps θ/φ and V/U. */
void *tdgl_stream(tdgl_ctx *ctx);
int tdgl_device_state(tdgl_ctx *ctx, tdgl_state_view *dev);

int tdgl_get_stats(tdgl_ctx *ctx, tdgl_stats *out);

/* Per-kernel timing (no counterpart in the reference, which times whole steps only): with profiling on, every
 * kernel launch of the context is bracketed by CUDA events on its stream and counted with its algorithmic
 * (compulsory) bytes.  tdgl_profile resets the counters; tdgl_profile_read(ctx, -1, …) returns the number of
 * kernel categories, and for 0 <= cat < that number fills the category's name, launches, milliseconds and bytes. */
int tdgl_profile(tdgl_ctx *ctx, int32_t on);

/* The field solve of step! alone on the resident θ and φ (gtdgl/src/step.jl:26-30): implicit_curl! with the
 * SepSolver or the PCG (gtdgl/src/implicit.jl:91-104, :279-334, :376-446; warm start and extrapolation as in a
 * step), or scale_increment! (:337-342); writes φ and the PCG carry.  Replaces TDGLGPU._implicit_curl!(g, sep, gs),
 * which the reference's device PCG zero-source test drives directly (gpu/TDGLGPU/test/test_pcg_zero_rhs.jl:7-16). */
int tdgl_field_solve(tdgl_ctx *ctx);

/* The temporal link rotations of the band update on caller arrays (host buffers, column-major (n1, n2, n3), complex
 * interleaved), over the 1-based inclusive range rng = {i0, i1, j0, j1, k0, k1}: op 0 = _rot! (L = V, R = Q^{1/par}),
 * op 1 = _rotfrac! (L = V Q^par), op 2 = _link_rate! along axis ax (R real, −arg Q + (Ω[I + e_ax] − Ω[I])·par), with
 * Q = V conj(U) (gtdgl/src/bands.jl:303-310, :355-369, :409-423).  The step's own link passes use the same device
 * formulas.  Replaces the reference's device rotation kernels as its test drives them (_rot_k!, _rotfrac_k!,
 * _lrate_k!, gpu/TDGLGPU/test/test_link_rotations.jl:21-60).  Allocates and synchronises: a test and set-up helper. */
int tdgl_link_rotations(int32_t op, int32_t n1, int32_t n2, int32_t n3, const int32_t *rng, int32_t ax, const double *V,
                        const double *U, const double *Om, double par, double *L, double *R);

/* (I + aK)^{-1} alone (gtdgl/src/implicit.jl:62-83 _sep_solve!; with f32 = 1, _precond32! :353-373): b and z are
 * host buffers over the three ranges of the separable solve, packed x, y, z.  For SEP and PCG contexts. */
int tdgl_sep_apply(tdgl_ctx *ctx, const double *b, double *z, int32_t f32);

/* The same FP64 inverse of (I + aK) for callers that cannot allocate device memory (a solver running inside
 * another framework's memory pool or stream capture, a process whose device memory is reserved up front, a plugin
 * forbidden to allocate).  No counterpart in the reference: it is an addition of this library.
 * It needs no context and allocates nothing: its scratch is a fixed 16 MiB array in the library's device image,
 * which every GPU that loads the library holds until the process exits.  Grids whose scratch (bases, mode-space
 * arrays, line factorisation) exceeds 16 MiB are rejected with TDGL_EINVAL (a 192×64×16-cell grid with one padding
 * cell fits).
 *   g: the grid (dx = dy = dz); a = (dt/σn) κ²/dx² (tdgl_params.a_imp);
 *   b[3], z[3]: device pointers to the x, y, z components, each a node-shaped (Nx+1)(Ny+1)(Nz+1) array in the
 *     plane-major order j + (Ny+1)(k + (Nz+1) i) (0-based); the solve reads b and writes z on the ranges of the
 *     separable solve (gtdgl/src/implicit.jl:52) and leaves the other entries of z as they were; z may equal b;
 *   stream: the cudaStream_t to run on (0: the default stream); the call returns without waiting for the device.
 * The first call on a device looks up the scratch's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  Every call shares the scratch, which keeps the previous call's contents (the call
 * clears what it needs zeroed): calls that overlap on the GPU, from two streams or two threads, race. */
int tdgl_sep_apply_noalloc(const tdgl_grid *g, double a, const double *const *b, double *const *z, void *stream);
int tdgl_profile_read(tdgl_ctx *ctx, int32_t cat, const char **name, int64_t *launches, double *ms, double *bytes);

/* The field of the bar current per unit HJ on the outer faces (gtdgl/src/field.jl:151-180), computed on the
 * device with nq×nq midpoint quadrature per section cell; out = the six tables of tdgl_params (bar_hy_z …
 * bar_hy_x) as host buffers.  Host set-up helper: the Stepper holds these tables in the reference. */
int tdgl_bar_field(const tdgl_grid *g, int32_t nq, double *hy_z, double *hy_y, double *hz_z, double *hz_y, double *hz_x,
                   double *hy_x);
/* Why the last call on ctx failed (ctx may be NULL for tdgl_ctx_create failures). */
const char *tdgl_last_error(const tdgl_ctx *ctx);
/* 1 if the parameters are supported (supported(st), gpu/TDGLGPU/src/TDGLGPU.jl:39-44); otherwise 0 and why. */
/* ---- the observables of one protocol cycle, on the resident state (gtdgl/src/protocol.jl:148-189, :409-453;
 * gtdgl/src/observables.jl:48-114).  The ladder's voltmeter: planes vi < vo (x indices, protocol.jl:341), the live
 * links of each plane and the complete lines (:342-346), as (y2−y1+2) × (z2−z1+2) column-major byte masks. */
typedef struct tdgl_meter {
  int32_t vi, vo;                     /* voltmeter planes, x1 <= vi < vo <= x2 */
  int32_t nphase;                     /* bands 1..nphase get their path phase measured (0..N) */
  const uint8_t *Min, *Mou;           /* live x links on the planes vi and vo (nonzero = live) */
  const uint8_t *line_ok;             /* lines whose links are all live between the planes */
} tdgl_meter;

typedef struct tdgl_obs {
  double *D[TDGL_MAXB];               /* host buffers, one line grid each: the path phase of band µ < nphase
                                         (_path_phase!, protocol.jl:168-179); null: not copied */
  double vsum_in, vsum_out;           /* Σ φx over Min at vi and over Mou at vo (_plane_sum, :148-155): the voltage
                                         is vsum_out/count(Mou) − vsum_in/count(Min) (:412) */
  double ta_sum;                      /* Σ over line_ok lines of Σ_{vi <= i < vo} φx: θ_A = ta_sum/count(line_ok) */
  double res[TDGL_MAXB];              /* max over the block of | |F_µ| − |F_µ| at the previous measurement | (:432-440) */
  double amax;                        /* max |F_µ| over bands and block; NaN or Inf when a value is not finite */
  double diffh;                       /* max |h_z − h_z at the previous measurement| over every h_z (:447-451) */
  double Itot, Isam;                  /* midplane_current (observables.jl:102-114) */
} tdgl_obs;

/* Sets the voltmeter and takes the baselines of res and diffh from the current state: |G_µ| on the block and h_z,
 * as the ladder does at its start (protocol.jl:360-361). */
int tdgl_meter_set(tdgl_ctx *ctx, const tdgl_meter *m);
/* The observables of the current state; moves the baselines to it (protocol.jl:409-451). */
int tdgl_measure(tdgl_ctx *ctx, tdgl_obs *out);
/* count_vortices (observables.jl:48-74) of band `band` (0-based) on the plane z = kc (1-based), from F, V and h_z:
 * Nv, the perimeter winding Nv_loop, whether the perimeter runs through material, and optionally the per-plaquette
 * map nmap ((x2−x1+1) × (y2−y1+1), column-major). */
int tdgl_vortices(tdgl_ctx *ctx, int32_t band, int32_t kc, int32_t *Nv, int32_t *Nv_loop, int32_t *loop_ok,
                  int32_t *nmap);

int tdgl_supported(const tdgl_params *p, char *why, int32_t why_len);
int tdgl_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* TDGL_B200_H */
