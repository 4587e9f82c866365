# TDGLB200.jl — the Julia side of the B200 stepper: the accelerator hook of gtdgl (`TDGL.STEPS[]`,
# gtdgl/src/protocol.jl:305-316) driving libtdgl_b200.so through `ccall`, in place of TDGLGPU
# (gpu/TDGLGPU/src/TDGLGPU.jl:2086-2144).
#
#   using TDGL, TDGLB200
#   TDGLB200.enable!()                 # fallback = :error only: the library has no CPU path
#   run_ladders(st, Js; H=H, pr=pr)    # every ladder cycle runs on the device
#
# The structs below mirror include/tdgl_b200.h field by field (ABI version 7); tests/test_julia_shim.py checks the
# field list, order and types against the C header and the Python mirror (juliatdgl_b200/abi.py).  Each cycle the
# closure copies the State up, the Stepper's carried state up (the PCG warm start and extrapolation history,
# implicit.jl:142-169; the open boundary's ramp, openbc.jl:100-109), steps, and copies both back, so that the host
# may change any of them between cycles (_pcg_reset! at a ladder's start, _pcg_back! / _open_back! around the delay
# confirmation, protocol.jl:222-262, :376) and the device follows.
module TDGLB200

using TDGL
using TDGL: State, Stepper, PCGSolver, SepSolver, lattice_green

const LIB = get(ENV, "TDGL_B200_LIB", joinpath(@__DIR__, "..", "libtdgl_b200.so"))
const ABI_VERSION = Int32(8)
const MAXB = 8
const MAXSTG = 64
const MAXMAT = 8

const SOLVER_EXPLICIT, SOLVER_SCALE, SOLVER_SEP, SOLVER_PCG = Int32(0), Int32(1), Int32(2), Int32(3)
const BC_SLAB, BC_BAR, BC_OPEN = Int32(0), Int32(1), Int32(2)
const E_NOCONV = Int32(-4)

struct Grid_t
    Nx::Int32; Ny::Int32; Nz::Int32
    x1::Int32; x2::Int32; y1::Int32; y2::Int32; z1::Int32; z2::Int32
    dx::Float64; dy::Float64; dz::Float64
end

struct BandCoef_t
    kx::Float64; ky::Float64; kz::Float64
    c::Float64
    eps::Float64
    beta::Float64
    gamma2::Float64
    cpl::NTuple{MAXB,Float64}
end

struct Materials_t
    nmat::Int32
    idx::Ptr{UInt8}
    full::NTuple{MAXMAT,NTuple{MAXB,BandCoef_t}}
    stage::NTuple{MAXMAT,NTuple{MAXB,BandCoef_t}}
    ma::NTuple{MAXMAT,NTuple{MAXB,NTuple{3,Float64}}}
    transparency::NTuple{MAXMAT,NTuple{MAXMAT,Float64}}
    absent::NTuple{MAXMAT,NTuple{MAXB,Int32}}
    gamma::NTuple{MAXMAT,NTuple{MAXB,Float64}}
    a::NTuple{MAXMAT,NTuple{MAXB,Float64}}               # st.mt.a (ε = a − θ with the heat model)
    gk::NTuple{MAXMAT,NTuple{MAXB,Float64}}              # γ̃ of each material's bands (the heat source)
    sigma_n::NTuple{MAXMAT,Float64}                      # σn of each material (the Joule heat)
    heat_DT::NTuple{MAXMAT,Float64}                      # st.mt.DT (empty without heat)
end

struct Params_t
    abi_version::Int32
    nbands::Int32
    grid::Grid_t
    dt::Float64
    nsub::NTuple{MAXB,Int32}
    stages::NTuple{MAXB,Int32}
    use_rkc::NTuple{MAXB,Int32}
    rkc_q::NTuple{MAXB,Float64}
    rkc_mu::NTuple{MAXB,NTuple{MAXSTG,Float64}}
    rkc_nu::NTuple{MAXB,NTuple{MAXSTG,Float64}}
    rkc_c::NTuple{MAXB,NTuple{MAXSTG,Float64}}
    rkc_sk::NTuple{MAXB,NTuple{2,Float64}}
    bc::NTuple{MAXB,BandCoef_t}
    bcs::NTuple{MAXB,BandCoef_t}
    wa::NTuple{3,NTuple{MAXB,Float64}}
    d1::Float64
    sxy::Float64
    sxz::Float64
    syx::Float64
    syz::Float64
    szx::Float64
    szy::Float64
    a_imp::Float64
    solver::Int32
    selffield_bc::Int32
    extrap::Int32
    rotframe::Int32
    hard::Int32
    f::Ptr{Float64}
    taux::Ptr{Float64}
    tauy::Ptr{Float64}
    tauz::Ptr{Float64}
    Dx::Ptr{Float64}
    Dy::Ptr{Float64}
    Dz::Ptr{Float64}
    bar_hy_z::Ptr{Float64}
    bar_hy_y::Ptr{Float64}
    bar_hz_z::Ptr{Float64}
    bar_hz_y::Ptr{Float64}
    bar_hz_x::Ptr{Float64}
    bar_hy_x::Ptr{Float64}
    pcg_tol::Float64
    pcg_maxit::Int32
    pcg_fast::Int32
    pcg_f32::Int32
    pcg_extrap::Int32
    open_every::Int32
    open_R::Int32
    kappa2::Float64
    open_fac::Float64
    open_green::Ptr{Float64}
    open_jbar::Ptr{Float64}
    noise_on::Int32
    noise_field::Int32
    noise_T::Float64
    noise_seed::UInt64
    noise_gamma::NTuple{MAXB,Float64}
    noise_sigma_n::Float64
    noise_step0::Int64
    materials::Ptr{Materials_t}
    vac::Ptr{UInt8}
    drag_on::Int32
    drag_c::NTuple{MAXB,NTuple{MAXB,NTuple{3,Float64}}}
    drag_nu::NTuple{MAXB,NTuple{MAXB,Float64}}
    heat_on::Int32
    heat_joule::Int32
    heat_margin::Int32
    heat_DT::Float64
    heat_gamma_bath::Float64
    heat_eta::Float64
    heat_cap::Float64
    heat_T::Float64
    heat_sigma_n::Float64
    heat_a::NTuple{MAXB,Float64}
    heat_Gamma::NTuple{MAXB,Float64}
    heat_gk::NTuple{MAXB,Float64}
    qp_on::Int32                     # normal fluids per band (exchange.jl QPExchange / QPExchangeN; ABI v8)
    qp_s::NTuple{MAXB,Float64}
    qp_sigma_n::Float64
    qp_lambda0::Float64
    qp_g::NTuple{MAXB,NTuple{3,Float64}}
    qp_gamma::NTuple{MAXB,NTuple{MAXB,Float64}}
    qp_P::NTuple{MAXB,NTuple{MAXB,Float64}}
    qp_Pinv::NTuple{MAXB,NTuple{MAXB,Float64}}
    qp_lam::NTuple{MAXB,Float64}
    qp_Gm::NTuple{MAXB,NTuple{MAXB,Float64}}
    qp_j0::Int32
    qp_nj::Int32
    qp_k0::Int32
    qp_nk::Int32
    qp_Vx::Ptr{Float64}
    qp_Wx::Ptr{Float64}
    qp_ex::Ptr{Float64}
    qp_Vy::Ptr{Float64}
    qp_Wy::Ptr{Float64}
    qp_ey::Ptr{Float64}
    qp_Vz::Ptr{Float64}
    qp_Wz::Ptr{Float64}
    qp_ez::Ptr{Float64}
    qp_cond::Ptr{UInt8}
    qp_tol::Float64
    qp_maxit::Int32
    qp_cx::Ptr{Float64}
    qp_cy::Ptr{Float64}
    qp_cz::Ptr{Float64}
    qp_lamv::Ptr{Float64}
    qp_d::Float64
    qp_mgamma::NTuple{MAXMAT,NTuple{2,NTuple{2,Float64}}}
end

struct StateView_t
    G::NTuple{MAXB,Ptr{Float64}}
    F::NTuple{MAXB,Ptr{Float64}}
    th::NTuple{3,Ptr{Float64}}
    ph::NTuple{3,Ptr{Float64}}
    U::NTuple{3,Ptr{Float64}}
    V::NTuple{3,Ptr{Float64}}
    J::NTuple{3,Ptr{Float64}}
    h::NTuple{3,Ptr{Float64}}
end

struct CarryView_t
    pcg_x::Ptr{Float64}
    pcg_xprev::Ptr{Float64}
    pcg_warm::Int32
    pcg_have2::Int32
    open_count::Int32
    open_old::NTuple{3,Ptr{Float64}}
    open_new::NTuple{3,Ptr{Float64}}
    open_theta::NTuple{3,Ptr{Float64}}
    heat_theta::Ptr{Float64}         # st.heat.θ, read and written in place (ABI v6)
end

# ---------------------------------------------------------------------------------------------- helpers
pad(t, n, z) = ntuple(i -> i <= length(t) ? t[i] : z, n)
ptr(a) = a === nothing ? Ptr{Float64}(C_NULL) : Ptr{Float64}(pointer(a))

coef(b) = BandCoef_t(b.kx, b.ky, b.kz, b.c, b.ε, b.β, b.γ2, pad(Tuple(b.cpl), MAXB, 0.0))
coef(m, a::Int) = BandCoef_t(m.kx[a], m.ky[a], m.kz[a], m.c[a], m.ε[a], m.β[a], m.γ2[a], pad(Tuple(m.cpl[a]), MAXB, 0.0))
const ZCOEF = BandCoef_t(0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, ntuple(_ -> 0.0, MAXB))

solver_of(st::Stepper) = st.imp isa PCGSolver ? SOLVER_PCG : st.imp isa SepSolver ? SOLVER_SEP :
                         st.D !== nothing ? SOLVER_SCALE : SOLVER_EXPLICIT

"""The arrays a Params_t points into (kept alive by the cache as long as the context lives)."""
mutable struct Keep
    arrays::Vector{Any}
end
keep!(k::Keep, a) = (push!(k.arrays, a); a)

"""
    params(st) -> (Params_t, Keep)

tdgl_params of a Stepper (gtdgl/src/scheme.jl:167-198), field by field; the same as pack_params in
juliatdgl_b200/abi.py.  `noise_step0`: the index of the stream's first step (the steps this Stepper has taken).
"""
function params(st::Stepper{N}; noise_step0::Integer=0) where N
    N <= MAXB || throw(ArgumentError("TDGLB200: at most $MAXB bands"))
    k = Keep(Any[])
    gr = st.grid; md = st.model; mk = st.masks; fc = st.fc
    g = Grid_t(gr.Nx, gr.Ny, gr.Nz, gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2, gr.dx, gr.dy, gr.dz)
    rk(µ) = st.rkc === nothing ? nothing : st.rkc[µ]
    any(µ -> st.rkl[µ] > MAXSTG, 1:N) && throw(ArgumentError("TDGLB200: at most $MAXSTG stages per band"))
    stagearr(f) = ntuple(µ -> µ <= N && rk(µ) !== nothing ? pad(Tuple(f(rk(µ))), MAXSTG, 0.0) : ntuple(_ -> 0.0, MAXSTG), MAXB)
    D = st.D
    bar = st.bar
    S = st.imp isa PCGSolver ? st.imp : nothing
    ob = st.open
    nz = st.noise
    green = ob === nothing ? nothing : keep!(k, lattice_green(8))
    jbar = ob === nothing ? nothing : keep!(k, ob.Jbar)
    vac = mk.vac === nothing ? nothing : keep!(k, UInt8.(mk.vac))
    mat = st.mt === nothing ? Ptr{Materials_t}(C_NULL) : materials!(k, st)
    qx = st.qpx
    qn = qx isa TDGL.QPExchangeN
    # the conjugate-gradient solve of δ: QPSolve's conducting unknowns of a sculpted sample (1 or 0) or QPVar's
    # types, as bytes; QPVar's coefficients
    qv = qx isa TDGL.QPExchange ? qx.var : nothing
    qcond = qv !== nothing ? keep!(k, UInt8.(qv.typ)) :
            qx === nothing || qx.ps.cond === nothing ? nothing : keep!(k, UInt8.(qx.ps.cond))
    mg(m, µ, ν) = st.mt !== nothing && m <= length(st.mt.models) && qx !== nothing ? st.mt.models[m].γ[µ][ν] : 0.0
    mat8(f) = ntuple(a -> ntuple(c -> qn && a <= N && c <= N ? f(a, c) : 0.0, MAXB), MAXB)
    p = Params_t(ABI_VERSION, Int32(N), g, st.dt,
        pad(Int32.(st.nsub), MAXB, Int32(0)), pad(Int32.(st.rkl), MAXB, Int32(0)),
        ntuple(µ -> Int32(µ <= N && rk(µ) !== nothing), MAXB),
        ntuple(µ -> µ <= N && rk(µ) !== nothing ? rk(µ).q : 0.0, MAXB),
        stagearr(r -> r.μ), stagearr(r -> r.ν), stagearr(r -> r.c),
        ntuple(µ -> µ <= N && rk(µ) !== nothing ? rk(µ).sk : (0.0, 0.0), MAXB),
        ntuple(µ -> µ <= N ? coef(st.bc[µ]) : ZCOEF, MAXB), ntuple(µ -> µ <= N ? coef(st.bcs[µ]) : ZCOEF, MAXB),
        ntuple(ax -> pad(st.wa[ax], MAXB, 0.0), 3),
        fc.d1, fc.sxy, fc.sxz, fc.syx, fc.syz, fc.szx, fc.szy, fc.a,
        solver_of(st), ob !== nothing ? BC_OPEN : bar !== nothing ? BC_BAR : BC_SLAB,
        Int32(st.extrap), Int32(st.rotframe), Int32(st.hard),
        ptr(mk.f), ptr(mk.τx), ptr(mk.τy), ptr(mk.τz),
        ptr(D === nothing ? nothing : D[1]), ptr(D === nothing ? nothing : D[2]), ptr(D === nothing ? nothing : D[3]),
        ptr(bar === nothing ? nothing : keep!(k, bar.hy_z)), ptr(bar === nothing ? nothing : keep!(k, bar.hy_y)),
        ptr(bar === nothing ? nothing : keep!(k, bar.hz_z)), ptr(bar === nothing ? nothing : keep!(k, bar.hz_y)),
        ptr(bar === nothing ? nothing : keep!(k, bar.hz_x)), ptr(bar === nothing ? nothing : keep!(k, bar.hy_x)),
        S === nothing ? 0.0 : S.tol, Int32(S === nothing ? 0 : S.maxit),
        Int32(S !== nothing && S.fast !== nothing), Int32(S !== nothing && S.fast !== nothing && S.fast.f32),
        Int32(S !== nothing && S.fast !== nothing && S.fast.extrap),
        Int32(ob === nothing ? 0 : ob.every), Int32(8), md.κ^2, gr.dx^3 / md.κ^2, ptr(green), ptr(jbar),
        Int32(nz !== nothing), Int32(nz !== nothing && nz.field), nz === nothing ? 0.0 : nz.T,
        nz === nothing ? UInt64(0) : nz.seed, pad(Tuple(b.Γ for b in md.bands), MAXB, 0.0), md.σn,
        Int64(noise_step0), mat, vac === nothing ? Ptr{UInt8}(C_NULL) : pointer(vac),
        Int32(st.drag !== nothing),
        ntuple(µ -> ntuple(ν -> st.drag !== nothing && µ <= N && ν <= N ? st.drag[µ][ν] : (0.0, 0.0, 0.0), MAXB), MAXB),
        ntuple(µ -> ntuple(ν -> st.dragν !== nothing && µ <= N && ν <= N ? st.dragν[µ][ν] : 0.0, MAXB), MAXB),
        Int32(st.heat !== nothing), Int32(st.heat !== nothing && st.heat.h.joule),
        Int32(st.heat === nothing ? 0 : st.heat.h.margin), st.heat === nothing ? 0.0 : st.heat.h.D_T,
        st.heat === nothing ? 0.0 : st.heat.h.gamma_bath, st.heat === nothing ? 0.0 : st.heat.h.eta,
        st.heat === nothing ? 0.0 : st.heat.h.cap, st.heat === nothing ? 0.0 : st.heat.T, md.σn,
        pad(Tuple(b.a for b in md.bands), MAXB, 0.0), pad(Tuple(b.Γ for b in md.bands), MAXB, 0.0),
        pad(Tuple(b.γkwt for b in md.bands), MAXB, 0.0),
        Int32(qx === nothing ? 0 : qn ? 2 : 1), pad(qx === nothing ? () : Tuple(qx.s), MAXB, 0.0),
        qx === nothing ? 0.0 : qx.σn, qx === nothing || qn ? 0.0 : qx.λ0,
        ntuple(µ -> ntuple(i -> qx !== nothing && µ <= N ? TDGL.stiffness(md.bands[µ], i) : 0.0, 3), MAXB),
        ntuple(µ -> ntuple(ν -> qx !== nothing && µ <= N && ν <= N ? md.γ[µ][ν] : 0.0, MAXB), MAXB),
        mat8((a, c) -> qx.P[a, c]), mat8((a, c) -> qx.Pinv[a, c]), pad(qn ? Tuple(qx.λ) : (), MAXB, 0.0),
        qn ? mat8((a, c) -> qx.Gm[a, c]) :
            ntuple(a -> ntuple(c -> qx !== nothing && a == 1 && c == 2 ? qx.G : 0.0, MAXB), MAXB),
        Int32(qx === nothing ? 0 : qx.ps.j0), Int32(qx === nothing ? 0 : size(qx.S, 2)),
        Int32(qx === nothing ? 0 : qx.ps.k0), Int32(qx === nothing ? 0 : size(qx.S, 3)),
        ptr(qx === nothing ? nothing : qx.Vx), ptr(qx === nothing ? nothing : qx.Wx), ptr(qx === nothing ? nothing : qx.ex),
        ptr(qx === nothing ? nothing : qx.Vy), ptr(qx === nothing ? nothing : qx.Wy), ptr(qx === nothing ? nothing : qx.ey),
        ptr(qx === nothing ? nothing : qx.Vz), ptr(qx === nothing ? nothing : qx.Wz), ptr(qx === nothing ? nothing : qx.ez),
        qcond === nothing ? Ptr{UInt8}(C_NULL) : pointer(qcond),
        qx === nothing ? 0.0 : qx.ps.tol, Int32(qx === nothing ? 0 : qx.ps.maxit),
        ptr(qv === nothing ? nothing : qv.cx), ptr(qv === nothing ? nothing : qv.cy),
        ptr(qv === nothing ? nothing : qv.cz), ptr(qv === nothing ? nothing : qv.λ),
        qv === nothing ? 0.0 : qx.σn * (2 / gr.dx^2 + 2 / gr.dy^2 + 2 / gr.dz^2) + qx.λ0,
        ntuple(m -> ntuple(µ -> ntuple(ν -> mg(m, µ, ν), 2), 2), MAXMAT))
    (p, k)
end

function materials!(k::Keep, st::Stepper{N}) where N
    mt = st.mt
    M = length(mt.models)
    M <= MAXMAT || throw(ArgumentError("TDGLB200: at most $MAXMAT materials"))
    idx = keep!(k, mt.idx)
    z3 = ntuple(_ -> (0.0, 0.0, 0.0), MAXB)
    m = Materials_t(Int32(M), pointer(idx),
        ntuple(a -> a <= M ? ntuple(µ -> µ <= N ? coef(mt.full[µ], a) : ZCOEF, MAXB) : ntuple(_ -> ZCOEF, MAXB), MAXMAT),
        ntuple(a -> a <= M ? ntuple(µ -> µ <= N ? coef(mt.stage[µ], a) : ZCOEF, MAXB) : ntuple(_ -> ZCOEF, MAXB), MAXMAT),
        ntuple(a -> a <= M ? ntuple(µ -> µ <= N ? Tuple(mt.models[a].bands[µ].ma) : (0.0, 0.0, 0.0), MAXB) : z3, MAXMAT),
        ntuple(a -> ntuple(b -> a <= M && b <= M ? mt.t[a, b] : 0.0, MAXMAT), MAXMAT),
        ntuple(a -> ntuple(µ -> Int32(a <= M && µ <= N && mt.absent[a, µ]), MAXB), MAXMAT),
        ntuple(a -> ntuple(µ -> a <= M && µ <= N ? mt.models[a].bands[µ].Γ : 0.0, MAXB), MAXMAT),
        ntuple(a -> ntuple(µ -> a <= M && µ <= N ? mt.a[µ][a] : 0.0, MAXB), MAXMAT),
        ntuple(a -> ntuple(µ -> a <= M && µ <= N ? mt.models[a].bands[µ].γkwt : 0.0, MAXB), MAXMAT),
        ntuple(a -> a <= M ? mt.models[a].σn : 0.0, MAXMAT),
        ntuple(a -> a <= length(mt.DT) ? mt.DT[a] : 0.0, MAXMAT))
    r = keep!(k, Ref(m))
    Base.unsafe_convert(Ptr{Materials_t}, r)
end

function view(s::State{N}) where N
    StateView_t(ntuple(µ -> µ <= N ? Ptr{Float64}(pointer(s.G[µ])) : Ptr{Float64}(C_NULL), MAXB),
                ntuple(µ -> µ <= N ? Ptr{Float64}(pointer(s.F[µ])) : Ptr{Float64}(C_NULL), MAXB),
                (ptr(s.θx), ptr(s.θy), ptr(s.θz)), (ptr(s.φx), ptr(s.φy), ptr(s.φz)),
                (ptr(s.Ux), ptr(s.Uy), ptr(s.Uz)), (ptr(s.Vx), ptr(s.Vy), ptr(s.Vz)),
                (ptr(s.Jx), ptr(s.Jy), ptr(s.Jz)), (ptr(s.hx), ptr(s.hy), ptr(s.hz)))
end

# The carry packs x and xprev over the three ranges of the separable solve (implicit.jl:52), x, y, z; the PCG keeps
# them as range-shaped arrays (S.x[c], S.fast.xprev[c]), column-major, so the packing is their concatenation.
struct Carry
    x::Vector{Float64}
    xprev::Vector{Float64}
end
Carry(S::PCGSolver) = Carry(zeros(sum(length, S.x)), zeros(sum(length, S.x)))

function carry_up!(c::Union{Nothing,Carry}, st::Stepper)
    S = st.imp isa PCGSolver ? st.imp : nothing
    ob = st.open
    if S !== nothing
        o = 0
        for q in 1:3
            n = length(S.x[q])
            copyto!(c.x, o + 1, vec(S.x[q]), 1, n)
            S.fast === nothing || copyto!(c.xprev, o + 1, vec(S.fast.xprev[q]), 1, n)
            o += n
        end
    end
    CarryView_t(S === nothing ? C_NULL : pointer(c.x), S === nothing || S.fast === nothing ? C_NULL : pointer(c.xprev),
                Int32(S !== nothing && S.warm[1]), Int32(S !== nothing && S.fast !== nothing && S.fast.have2[1]),
                Int32(ob === nothing ? -1 : ob.count),
                ob === nothing ? (C_NULL, C_NULL, C_NULL) : (ptr(ob.old[1]), ptr(ob.old[2]), ptr(ob.old[3])),
                ob === nothing ? (C_NULL, C_NULL, C_NULL) : (ptr(ob.new[1]), ptr(ob.new[2]), ptr(ob.new[3])),
                ob === nothing ? (C_NULL, C_NULL, C_NULL) : (ptr(ob.θ[1]), ptr(ob.θ[2]), ptr(ob.θ[3])),
                st.heat === nothing ? Ptr{Float64}(C_NULL) : ptr(st.heat.θ))
end

function carry_down!(st::Stepper, c::Union{Nothing,Carry}, v::CarryView_t)
    S = st.imp isa PCGSolver ? st.imp : nothing
    if S !== nothing
        o = 0
        for q in 1:3
            n = length(S.x[q])
            copyto!(vec(S.x[q]), 1, c.x, o + 1, n)
            S.fast === nothing || copyto!(vec(S.fast.xprev[q]), 1, c.xprev, o + 1, n)
            o += n
        end
        S.warm[1] = v.pcg_warm != 0
        S.fast === nothing || (S.fast.have2[1] = v.pcg_have2 != 0)
    end
    st.open === nothing || (st.open.count = Int(v.open_count))   # old/new/θ were written in place
    st
end

# ---------------------------------------------------------------------------------------------- the context cache
mutable struct Ctx
    st::Any
    ptr::Ptr{Cvoid}
    p::Base.RefValue{Params_t}
    keep::Keep
    carry::Union{Nothing,Carry}
    steps::Int                   # steps taken through the hook (the noise stream's index)
end
const _CTX = Ref{Union{Nothing,Ctx}}(nothing)

lasterr(ctx) = unsafe_string(ccall((:tdgl_last_error, LIB), Cstring, (Ptr{Cvoid},), ctx))
check(rc, ctx) = rc == 0 || error("TDGLB200: ", lasterr(ctx), " (", rc, ")")

"""supported(st) -> (ok, why): whether the library runs this Stepper's step (TDGLGPU.jl:39-44)."""
function supported(st::Stepper)
    p, k = try params(st) catch e; return (false, sprint(showerror, e)) end
    buf = zeros(UInt8, 256)
    ok = GC.@preserve k buf ccall((:tdgl_supported, LIB), Cint, (Ref{Params_t}, Ptr{UInt8}, Int32), p, buf, 256)
    (ok != 0, unsafe_string(pointer(buf)))
end

function context!(st::Stepper)
    c = _CTX[]
    c !== nothing && c.st === st && return c
    c === nothing || close!()
    ok, why = supported(st)
    ok || throw(ArgumentError("TDGLB200: unsupported configuration: $why"))
    p, k = params(st)
    pr = Ref(p)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve k check(ccall((:tdgl_ctx_create, LIB), Cint, (Ref{Params_t}, Ref{Ptr{Cvoid}}), pr, out), C_NULL)
    c = Ctx(st, out[], pr, k, st.imp isa PCGSolver ? Carry(st.imp) : nothing, 0)
    _CTX[] = c
    c
end

function close!()
    c = _CTX[]
    c === nothing && return
    ccall((:tdgl_ctx_destroy, LIB), Cint, (Ptr{Cvoid},), c.ptr)
    _CTX[] = nothing
end

"""One ladder cycle on the device: n steps of step!(s, st; H, HJ) (the body of TDGL.STEPS[])."""
function cycle!(s::State, st::Stepper, n::Int; H::Float64, HJ::Float64)
    c = context!(st)
    v = Ref(view(s))
    cv = Ref(carry_up!(c.carry, st))
    GC.@preserve s st c begin
        check(ccall((:tdgl_upload_state, LIB), Cint, (Ptr{Cvoid}, Ref{StateView_t}), c.ptr, v), c.ptr)
        check(ccall((:tdgl_set_carry, LIB), Cint, (Ptr{Cvoid}, Ref{CarryView_t}), c.ptr, cv), c.ptr)
        rc = ccall((:tdgl_steps, LIB), Cint, (Ptr{Cvoid}, Int32, Float64, Float64), c.ptr, Int32(n), H, HJ)
        rc == 0 || rc == E_NOCONV || check(rc, c.ptr)   # maxit reached: the reference's own loop goes on too
        check(ccall((:tdgl_download_state, LIB), Cint, (Ptr{Cvoid}, Ref{StateView_t}), c.ptr, v), c.ptr)
        check(ccall((:tdgl_get_carry, LIB), Cint, (Ptr{Cvoid}, Ref{CarryView_t}), c.ptr, cv), c.ptr)
    end
    carry_down!(st, c.carry, cv[])
    c.steps += n
    s
end

"""
    enable!(; fallback=:error)

Installs the device stepper in TDGL.STEPS[] (TDGLGPU.enable!, TDGLGPU.jl:2103-2111).  There is no CPU fallback:
`fallback` other than :error is an ArgumentError, and an unsupported Stepper raises at its first cycle.
"""
function enable!(; fallback::Symbol=:error)
    fallback === :error || throw(ArgumentError("TDGLB200 has no CPU fallback"))
    ccall((:tdgl_abi_version, LIB), Cint, ()) == ABI_VERSION || error("TDGLB200: the library's ABI version differs")
    TDGL.STEPS[] = (s, st, n; H, HJ) -> cycle!(s, st, n; H=Float64(H), HJ=Float64(HJ))
    nothing
end

disable!() = (TDGL.STEPS[] = nothing; close!(); nothing)

end # module
