# LatticeMatricesB200Ext.jl -- package extension of LatticeMatrices.jl that
# sends the Dirac-operator hot path of CUDA-resident fields to liblmb200
# (sm_100a kernels behind the C ABI of include/lmb200.h).
#
# NOT TESTED: no Julia toolchain was available where this file was written.
# Every ccall below binds an entry point whose behaviour is tested through the
# Python ctypes mirror (latticematrices.jl_b200/lmb200/) against the oracle;
# the Julia side is the binding a maintainer would load as a package
# extension, with weak dependencies CUDA and EnzymeCore:
#
#   [weakdeps]    CUDA, EnzymeCore
#   [extensions]  LatticeMatricesB200Ext = ["CUDA", "EnzymeCore"]
#
# What it overrides, for LatticeMatrix fields whose storage is a CuArray:
#   * mul!(C, D, psi) and mul!(C, D', psi) for WilsonDiracOperator4D,
#     WilsonDiracCloverOperator4D, StaggeredDiracOperator4D and
#     HISQDiracOperator4D (WilsonDiracCloverOperator.jl:561-601 and the
#     other operators' mul! methods);
#   * cg!(x, DdagDOp(D, tmp), b, r, p, Ap; rtol, atol, maxiter) for those
#     operators (LinearAlgebras/cg.jl:73-137), with an optional inner
#     precision (:double as the reference, :single, :half = int16 storage);
#   * mul_cached_hisq! / mul_cached_clover! (HISQFullSmearing.jl:457-466,
#     WilsonDiracCloverOperator.jl:642-651) and their Enzyme reverse rules
#     (ext/AD/HISQFullSmearing.jl:295-462,
#     ext/AD/WilsonDiracCloverOperator.jl:348-444): the link cotangent comes
#     from lmb_hisq_link_pullback / lmb_wilson_clover_link_pullback, the
#     fermion cotangent from the adjoint stencil;
#   * dSFdU(dfdU, cache, phi) (ext/LatticeMatricesEnzymeExt.jl:387-460): the
#     whole fermion force -- CG, chi = D eta, pullback -- in one call of
#     lmb_hisq_fermion_force / lmb_wilson_clover_fermion_force.
# Fields on the CPU, and operators without a native kernel, keep the
# reference's own methods.
module LatticeMatricesB200Ext

using LinearAlgebra
using CUDA
using LatticeMatrices
using LatticeMatrices: LatticeMatrix, WilsonDiracOperator4D, WilsonDiracCloverOperator4D,
    StaggeredDiracOperator4D, HISQDiracOperator4D, HISQDiracCache4D, DdagDOp, CGResult,
    mark_halo_dirty!
import LatticeMatrices: cg!, mul_cached_hisq!, mul_cached_clover!, dSFdU
import EnzymeCore
import EnzymeCore.EnzymeRules as ER

const lib = get(ENV, "LMB200_LIB", "liblmb200.so")

# ---------------------------------------------------------------------------
# the C ABI: constants and structs of include/lmb200.h
# ---------------------------------------------------------------------------
const LMB_OK = 0
const LMB_ERR_ARG = -1
const LINKS_THIN, LINKS_FAT, LINKS_LONG = 0, 1, 2
const OP_WILSON, OP_WILSON_CLOVER, OP_STAGGERED, OP_HISQ = 0, 1, 2, 3
const PRECISION = Dict(:double => 0, :single => 1, :half => 2)
const REASONS = (:converged, :maximum_iterations, :nonpositive_curvature, :numerical_breakdown)

struct CGParams
    op::Cint
    kappa::Cdouble
    csw::Cdouble
    mass::Cdouble
    naik_epsilon::Cdouble
    rtol::Cdouble
    atol::Cdouble
    maxiter::Cint
    precision::Cint
    delta::Cdouble
    check_interval::Cint
    profile::Cint
end
CGParams(op, kappa, csw, mass, eps; rtol=1e-10, atol=0.0, maxiter=5000, precision=:double, delta=0.1) =
    CGParams(op, kappa, csw, mass, eps, rtol, atol, maxiter, PRECISION[precision], delta, 0, 0)

struct CGOut
    converged::Cint
    iterations::Cint
    residual_norm::Cdouble
    relative_residual::Cdouble
    reason::Cint
    reliable_updates::Cint
    true_residual_norm::Cdouble
    dslash_ms::Cdouble
    update_ms::Cdouble
    dslash_launches::Cint
    update_launches::Cint
    kernel_launches::Clonglong
    link_reals::Cint
end
CGOut() = CGOut(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)

to_result(o::CGOut) = CGResult(o.converged != 0, Int(o.iterations), o.residual_norm,
                               o.relative_residual, REASONS[o.reason+1])

# ---------------------------------------------------------------------------
# contexts: one lmb_ctx per operator (link / clover caches, CG workspaces)
# ---------------------------------------------------------------------------
mutable struct Ctx
    h::Ptr{Cvoid}
end

function Ctx(dev::Integer)
    h = ccall((:lmb_create, lib), Ptr{Cvoid}, (Cint,), dev)
    h == C_NULL && error("lmb_create($dev) failed")
    c = Ctx(h)
    finalizer(c) do c
        c.h == C_NULL || ccall((:lmb_destroy, lib), Cvoid, (Ptr{Cvoid},), c.h)
        c.h = C_NULL
    end
    return c
end

const CONTEXTS = WeakKeyDict{Any,Ctx}()
ctx_of(owner) = get!(() -> Ctx(CUDA.deviceid(CUDA.device())), CONTEXTS, owner)

function check(c::Ctx, rc)
    rc == LMB_OK && return nothing
    msg = unsafe_string(ccall((:lmb_last_error, lib), Cstring, (Ptr{Cvoid},), c.h))
    rc == LMB_ERR_ARG && throw(ArgumentError(msg))
    error("liblmb200 error $rc: $msg")
end

stream() = CUDA.stream().handle           # every call is ordered on the task's stream
devptr(ls::LatticeMatrix) = Ptr{Cvoid}(UInt(pointer(ls.A)))
devptrs(fields) = Ptr{Cvoid}[devptr(f) for f in fields]
epochs(fields) = UInt64[f.halo_epoch.core for f in fields]
dtype_code(::Type{ComplexF64}) = Cint(0)
dtype_code(::Type{ComplexF32}) = Cint(1)

function set_geometry!(c::Ctx, psi::LatticeMatrix{4,T}) where {T}
    ph = ComplexF64.(collect(psi.phases))
    check(c, ccall((:lmb_set_geometry, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cint}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cint}, Cint),
        c.h, Cint[psi.PN...], psi.nw, real.(ph), imag.(ph), Cint[psi.coords...], dtype_code(T)))
end

function upload_links!(c::Ctx, which, links)
    check(c, ccall((:lmb_links_upload, lib), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Ptr{Cvoid}}, Ptr{UInt64}, Ptr{Cvoid}),
        c.h, which, devptrs(links), epochs(links), stream()))
end

# the process grid of a field split over MPI ranks: one NCCL communicator per
# context, its id made on rank 0 (nccl_unique_id) and broadcast by the caller
# (MPI.Bcast! in its communicator); the library exchanges the faces of the
# split dimensions, overlapped with the interior sites
function set_process_grid!(c::Ctx, psi::LatticeMatrix{4}, nccl_id::Vector{UInt8}, nranks, rank,
                           nb_minus, nb_plus)
    mask = UInt32(sum(d -> psi.dims[d] > 1 ? (1 << (d - 1)) : 0, 1:4))
    check(c, ccall((:lmb_set_process_grid, lib), Cint,
        (Ptr{Cvoid}, Ptr{UInt8}, Cint, Cint, Ptr{Cint}, Ptr{Cint}, Cuint, Ptr{Cint}, Ptr{Cint}),
        c.h, nccl_id, nranks, rank, Cint[psi.dims...], Cint[psi.coords...], mask,
        Cint[nb_minus...], Cint[nb_plus...]))
end

function nccl_unique_id()
    id = zeros(UInt8, 128)
    rc = ccall((:lmb_nccl_unique_id, lib), Cint, (Ptr{UInt8},), id)
    rc == LMB_OK || error("lmb_nccl_unique_id failed ($rc): NCCL unavailable")
    return id
end

# ---------------------------------------------------------------------------
# operators: which links, which entry point
# ---------------------------------------------------------------------------
bind!(c::Ctx, D::WilsonDiracOperator4D, psi) = (set_geometry!(c, psi); upload_links!(c, LINKS_THIN, D.U); c)
bind!(c::Ctx, D::WilsonDiracCloverOperator4D, psi) = bind!(c, D.wilson, psi)
bind!(c::Ctx, D::StaggeredDiracOperator4D, psi) = (set_geometry!(c, psi); upload_links!(c, LINKS_THIN, D.U); c)
function bind!(c::Ctx, D::HISQDiracOperator4D, psi)
    set_geometry!(c, psi)
    upload_links!(c, LINKS_FAT, D.links.fat_links)
    upload_links!(c, LINKS_LONG, D.links.long_links)
    return c
end

function apply!(C, D::WilsonDiracOperator4D, psi, dagger; precision=:double)
    c = bind!(ctx_of(D), D, psi)
    check(c, ccall((:lmb_wilson_apply, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Cint, Cint, Ptr{Cvoid}),
        c.h, devptr(C), devptr(psi), D.κ, dagger, PRECISION[precision], stream()))
    mark_halo_dirty!(C)                  # the library writes the core only
    return C
end
function apply!(C, D::WilsonDiracCloverOperator4D, psi, dagger; precision=:double)
    c = bind!(ctx_of(D), D, psi)
    check(c, ccall((:lmb_wilson_clover_apply, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Cdouble, Cint, Cint, Ptr{Cvoid}),
        c.h, devptr(C), devptr(psi), D.wilson.κ, D.cSW, dagger, PRECISION[precision], stream()))
    mark_halo_dirty!(C)
    return C
end
function apply!(C, D::StaggeredDiracOperator4D, psi, dagger; precision=:double)
    c = bind!(ctx_of(D), D, psi)
    check(c, ccall((:lmb_staggered_apply, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Cint, Cint, Ptr{Cvoid}),
        c.h, devptr(C), devptr(psi), D.mass, dagger, PRECISION[precision], stream()))
    mark_halo_dirty!(C)
    return C
end
function apply!(C, D::HISQDiracOperator4D, psi, dagger; precision=:double)
    c = bind!(ctx_of(D), D, psi)
    check(c, ccall((:lmb_hisq_apply, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Cdouble, Cint, Cint, Ptr{Cvoid}),
        c.h, devptr(C), devptr(psi), D.mass, D.naik_epsilon, dagger, PRECISION[precision], stream()))
    mark_halo_dirty!(C)
    return C
end

const NativeOp = Union{WilsonDiracOperator4D,WilsonDiracCloverOperator4D,StaggeredDiracOperator4D,HISQDiracOperator4D}

function LinearAlgebra.mul!(C::LatticeMatrix{4,T,<:CuArray}, D::NativeOp, psi::LatticeMatrix{4,T,<:CuArray}) where {T}
    return apply!(C, D, psi, 0)
end
function LinearAlgebra.mul!(C::LatticeMatrix{4,T,<:CuArray}, D::Adjoint{<:Any,<:NativeOp},
                            psi::LatticeMatrix{4,T,<:CuArray}) where {T}
    return apply!(C, parent(D), psi, 1)
end

cg_params(D::WilsonDiracOperator4D; kw...) = CGParams(OP_WILSON, D.κ, 0.0, 0.0, 0.0; kw...)
cg_params(D::WilsonDiracCloverOperator4D; kw...) = CGParams(OP_WILSON_CLOVER, D.wilson.κ, D.cSW, 0.0, 0.0; kw...)
cg_params(D::StaggeredDiracOperator4D; kw...) = CGParams(OP_STAGGERED, 0.0, 0.0, D.mass, 0.0; kw...)
cg_params(D::HISQDiracOperator4D; kw...) = CGParams(OP_HISQ, 0.0, 0.0, D.mass, D.naik_epsilon; kw...)

# cg!(x, DdagDOp(D, tmp), b, r, p, Ap): the whole solve in the library
# (r, p, Ap and the FP32 / int16 copies live in the context)
function cg!(x::LatticeMatrix{4,T,<:CuArray}, A::DdagDOp{<:NativeOp}, b::LatticeMatrix{4,T,<:CuArray},
             r, p, Ap; rtol=1e-10, atol=0.0, maxiter=5000, precision=:double, delta=0.1) where {T}
    D = A.D
    c = bind!(ctx_of(D), D, b)
    prm = Ref(cg_params(D; rtol=rtol, atol=atol, maxiter=maxiter, precision=precision, delta=delta))
    out = Ref(CGOut())
    check(c, ccall((:lmb_cg_ddagd, lib), Cint,
        (Ptr{Cvoid}, Ref{CGParams}, Ptr{Cvoid}, Ptr{Cvoid}, Ref{CGOut}, Ptr{Cvoid}),
        c.h, prm, devptr(x), devptr(b), out, stream()))
    mark_halo_dirty!(x)
    return to_result(out[])
end

# ---------------------------------------------------------------------------
# cached operators: the library keeps the smeared links / clover blocks keyed
# by thin-link pointer + halo epoch, so the refresh of
# _ensure_hisq_cache_current! / _ensure_clover_cache_current! is implicit
# ---------------------------------------------------------------------------
function smear!(c::Ctx, cache::HISQDiracCache4D, U)
    check(c, ccall((:lmb_hisq_links_from_thin, lib), Cint,
        (Ptr{Cvoid}, Ptr{Ptr{Cvoid}}, Ptr{UInt64}, Cdouble, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Cvoid}),
        c.h, devptrs(U), epochs(U), cache.operator.naik_epsilon, C_NULL, C_NULL, stream()))
end

function mul_cached_hisq!(result::LatticeMatrix{4,T,<:CuArray}, cache::HISQDiracCache4D,
                          U1::LatticeMatrix{4}, U2::LatticeMatrix{4}, U3::LatticeMatrix{4}, U4::LatticeMatrix{4},
                          psi::LatticeMatrix{4,T,<:CuArray}) where {T}
    c = ctx_of(cache)
    set_geometry!(c, psi)
    smear!(c, cache, (U1, U2, U3, U4))       # fat / long link sets of the context
    op = cache.operator
    check(c, ccall((:lmb_hisq_apply, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Cdouble, Cint, Cint, Ptr{Cvoid}),
        c.h, devptr(result), devptr(psi), op.mass, op.naik_epsilon, 0, 0, stream()))
    mark_halo_dirty!(result)
    return result
end

function mul_cached_clover!(result::LatticeMatrix{4,T,<:CuArray}, cache::WilsonDiracCloverOperator4D,
                            U1::LatticeMatrix{4}, U2::LatticeMatrix{4}, U3::LatticeMatrix{4}, U4::LatticeMatrix{4},
                            psi::LatticeMatrix{4,T,<:CuArray}) where {T}
    c = ctx_of(cache)
    set_geometry!(c, psi)
    upload_links!(c, LINKS_THIN, (U1, U2, U3, U4))   # F_mu_nu and clover blocks follow the epochs
    check(c, ccall((:lmb_wilson_clover_apply, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Cdouble, Cint, Cint, Ptr{Cvoid}),
        c.h, devptr(result), devptr(psi), cache.wilson.κ, cache.cSW, 0, 0, stream()))
    mark_halo_dirty!(result)
    return result
end

# ---------------------------------------------------------------------------
# Enzyme reverse rules
# ---------------------------------------------------------------------------
shadow(x) = x isa ER.Annotation && hasproperty(x, :dval) ? x.dval : nothing
function link_shadows(Us...)
    d = map(shadow, Us)
    n = count(s -> s isa LatticeMatrix, d)
    0 < n < 4 && throw(ArgumentError("the four links must be active together"))
    return n == 4 ? d : nothing
end

# the core of a padded field as a view (storage order NC1, NC2, X.., T..)
core(ls::LatticeMatrix{4}) = view(ls.A, :, :, ntuple(d -> ls.nw+1:ls.nw+ls.PN[d], 4)...)

# dpsi += D^+ dresult (the fermion cotangent; the adjoint stencil writes the core)
function add_adjoint_apply!(dpsi, D, dresult, psi)
    tmp = similar(psi)
    apply!(tmp, D, dresult, 1)
    core(dpsi) .+= core(tmp)
    mark_halo_dirty!(dpsi)
end

for (F, Cache, needs_nw) in ((:mul_cached_hisq!, :HISQDiracCache4D, 3),
                             (:mul_cached_clover!, :WilsonDiracCloverOperator4D, 1))
    @eval function ER.augmented_primal(cfg::ER.RevConfig, ::ER.Const{typeof($F)}, ::Type{RT},
                                       result::ER.Annotation{<:LatticeMatrix}, cache::ER.Annotation{<:$Cache},
                                       U1::ER.Annotation{<:LatticeMatrix}, U2::ER.Annotation{<:LatticeMatrix},
                                       U3::ER.Annotation{<:LatticeMatrix}, U4::ER.Annotation{<:LatticeMatrix},
                                       psi::ER.Annotation{<:LatticeMatrix}) where {RT}
        result.val.nw < $needs_nw && throw(ArgumentError(
            string("Enzyme differentiation of ", $(string(F)), " requires nw >= ", $needs_nw)))
        link_shadows(U1, U2, U3, U4)             # all four active, or none
        out = $F(result.val, cache.val, U1.val, U2.val, U3.val, U4.val, psi.val)
        primal = ER.needs_primal(cfg) ? out : nothing
        dres = ER.needs_shadow(cfg) ? shadow(result) : nothing
        # no tape: the pullback recomputes smearing levels / staples from U
        return ER.augmented_rule_return_type(cfg, RT, nothing)(primal, dres, nothing)
    end
end

function ER.reverse(cfg::ER.RevConfig, ::ER.Const{typeof(mul_cached_hisq!)}, dret, tape,
                    result::ER.Annotation{<:LatticeMatrix}, cache::ER.Annotation{<:HISQDiracCache4D},
                    U1::ER.Annotation{<:LatticeMatrix}, U2::ER.Annotation{<:LatticeMatrix},
                    U3::ER.Annotation{<:LatticeMatrix}, U4::ER.Annotation{<:LatticeMatrix},
                    psi::ER.Annotation{<:LatticeMatrix})
    none = (nothing, nothing, nothing, nothing, nothing, nothing, nothing)
    dresult = shadow(result)
    dresult isa LatticeMatrix || return none
    U = (U1.val, U2.val, U3.val, U4.val)
    dU = link_shadows(U1, U2, U3, U4)
    c = ctx_of(cache.val)
    set_geometry!(c, psi.val)
    if dU !== nothing
        any(mu -> dU[mu].A === U[mu].A, 1:4) &&
            throw(ArgumentError("mul_cached_hisq! thin-link shadow aliases its primal link"))
        # dU += d/dU Re<dresult, D_HISQ(U) psi> through Naik, level-2 Fat7 +
        # Lepage, U(3) projection and level-1 Fat7 (HISQPullback.jl:620-699)
        check(c, ccall((:lmb_hisq_link_pullback, lib), Cint,
            (Ptr{Cvoid}, Ptr{Ptr{Cvoid}}, Cdouble, Cdouble, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Ptr{Cvoid}}, Ptr{Cvoid}),
            c.h, devptrs(U), cache.val.operator.naik_epsilon, 1.0, devptr(dresult), devptr(psi.val),
            devptrs(dU), stream()))
        foreach(mark_halo_dirty!, dU)
    end
    dpsi = shadow(psi)
    if dpsi isa LatticeMatrix
        smear!(c, cache.val, U)
        add_adjoint_apply!(dpsi, cache.val.operator, dresult, psi.val)
    end
    fill!(dresult.A, zero(eltype(dresult.A)))   # the result was overwritten: its cotangent is consumed
    return none
end

function ER.reverse(cfg::ER.RevConfig, ::ER.Const{typeof(mul_cached_clover!)}, dret, tape,
                    result::ER.Annotation{<:LatticeMatrix}, cache::ER.Annotation{<:WilsonDiracCloverOperator4D},
                    U1::ER.Annotation{<:LatticeMatrix}, U2::ER.Annotation{<:LatticeMatrix},
                    U3::ER.Annotation{<:LatticeMatrix}, U4::ER.Annotation{<:LatticeMatrix},
                    psi::ER.Annotation{<:LatticeMatrix})
    none = (nothing, nothing, nothing, nothing, nothing, nothing, nothing)
    dresult = shadow(result)
    dresult isa LatticeMatrix || return none
    U = (U1.val, U2.val, U3.val, U4.val)
    dU = link_shadows(U1, U2, U3, U4)
    D = cache.val
    c = ctx_of(D)
    set_geometry!(c, psi.val)
    if dU !== nothing
        any(mu -> dU[mu].A === U[mu].A, 1:4) &&
            throw(ArgumentError("mul_cached_clover! link shadow aliases its primal link"))
        # hopping outer products and the four-leaf clover term through
        # F_mu_nu (WilsonCloverPullback.jl:342-403)
        check(c, ccall((:lmb_wilson_clover_link_pullback, lib), Cint,
            (Ptr{Cvoid}, Ptr{Ptr{Cvoid}}, Cdouble, Cdouble, Cdouble, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Ptr{Cvoid}},
             Ptr{Cvoid}),
            c.h, devptrs(U), D.wilson.κ, D.cSW, 1.0, devptr(dresult), devptr(psi.val), devptrs(dU), stream()))
        foreach(mark_halo_dirty!, dU)
    end
    dpsi = shadow(psi)
    if dpsi isa LatticeMatrix
        upload_links!(c, LINKS_THIN, U)
        tmp = similar(psi.val)
        check(c, ccall((:lmb_wilson_clover_apply, lib), Cint,
            (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Cdouble, Cint, Cint, Ptr{Cvoid}),
            c.h, devptr(tmp), devptr(dresult), D.wilson.κ, D.cSW, 1, 0, stream()))
        core(dpsi) .+= core(tmp)
        mark_halo_dirty!(dpsi)
    end
    fill!(dresult.A, zero(eltype(dresult.A)))
    return none
end

# ---------------------------------------------------------------------------
# dSFdU: dfdU += dS/dU for S = phi^+ (D^+D)^-1 phi, in one library call
# (eta = (D^+D)^-1 phi by the native CG, chi = D eta, dfdU += -2 d/dU
# Re<chi, D(U) eta>); the reference's Enzyme_derivative! accumulates into the
# shadows the same way
# ---------------------------------------------------------------------------
function dSFdU(dfdU, cache::HISQDiracCache4D, phi::LatticeMatrix{4,T,<:CuArray};
               rtol=1e-10, maxiter=5000, precision=:double) where {T}
    U = cache.cache_state.source_links   # the thin links the cache was last built from
    c = ctx_of(cache)
    set_geometry!(c, phi)
    op = cache.operator
    prm = Ref(CGParams(OP_HISQ, 0.0, 0.0, op.mass, op.naik_epsilon; rtol=rtol, maxiter=maxiter,
                       precision=precision))
    out = Ref(CGOut())
    check(c, ccall((:lmb_hisq_fermion_force, lib), Cint,
        (Ptr{Cvoid}, Ptr{Ptr{Cvoid}}, Ptr{UInt64}, Cdouble, Cdouble, Ptr{Cvoid}, Ptr{Ptr{Cvoid}},
         Ref{CGParams}, Ref{CGOut}, Ptr{Cvoid}),
        c.h, devptrs(U), epochs(U), op.mass, op.naik_epsilon, devptr(phi), devptrs(dfdU), prm, out, stream()))
    foreach(mark_halo_dirty!, dfdU)
    return to_result(out[])
end

function dSFdU(dfdU, D::WilsonDiracCloverOperator4D, phi::LatticeMatrix{4,T,<:CuArray};
               rtol=1e-10, maxiter=5000, precision=:double) where {T}
    U = D.wilson.U
    c = ctx_of(D)
    set_geometry!(c, phi)
    prm = Ref(CGParams(OP_WILSON_CLOVER, D.wilson.κ, D.cSW, 0.0, 0.0; rtol=rtol, maxiter=maxiter,
                       precision=precision))
    out = Ref(CGOut())
    check(c, ccall((:lmb_wilson_clover_fermion_force, lib), Cint,
        (Ptr{Cvoid}, Ptr{Ptr{Cvoid}}, Ptr{UInt64}, Cdouble, Cdouble, Ptr{Cvoid}, Ptr{Ptr{Cvoid}},
         Ref{CGParams}, Ref{CGOut}, Ptr{Cvoid}),
        c.h, devptrs(U), epochs(U), D.wilson.κ, D.cSW, devptr(phi), devptrs(dfdU), prm, out, stream()))
    foreach(mark_halo_dirty!, dfdU)
    return to_result(out[])
end

end # module
