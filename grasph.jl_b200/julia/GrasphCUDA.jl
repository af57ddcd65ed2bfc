# GrasphCUDA.jl — Julia binding of libgrasph_cuda.so for Grasph.jl.
#
# Adds a device-backed method of `time_integrate!` for a
# `LeapFrogTimeIntegrator` whose systems, functors and updaters are of the
# kinds the library implements, plus per-phase entry points.  Host arrays stay
# the source of truth between calls: they are uploaded when a call starts and
# written back when it ends.  Unsupported combinations raise ArgumentError;
# there is no CPU fallback inside this module (call Grasph's own method).
#
# Load after Grasph:   using Grasph; include("GrasphCUDA.jl"); using .GrasphCUDA
module GrasphCUDA

using Grasph
using StaticArrays
using HDF5

const LIB = get(ENV, "GRASPH_CUDA_LIB", joinpath(@__DIR__, "..", "libgrasph_cuda.so"))

# Constants of include/grasph_cuda.h
const GC_SYS = Dict(BasicParticleSystem => 0, FluidParticleSystem => 1,
                    StressParticleSystem => 2, ElastoPlasticParticleSystem => 3)
const GC_FIELD = (x=0, v=1, rho=2, dvdt=3, drhodt=4, p=5, stress=6, strain_rate=7,
                  vorticity=8, strain=9, strain_p=10, id=11)
const GC_WRAP_DYNAMIC = 1
const GC_WRAP_STATIC = 2
const GC_PFN_NPARAM = 6
const GC_UPD_NPARAM = 6

struct GcError <: Exception
    status::Cint
    msg::String
end

function check(ctx, st)
    st == 0 && return nothing
    msg = ctx == C_NULL ? "" : unsafe_string(ccall((:gc_last_error, LIB), Cstring, (Ptr{Cvoid},), ctx))
    st == 1 && throw(ArgumentError(msg))
    throw(GcError(st, msg))
end

pfn_kind(::Nothing) = 0
pfn_kind(::FluidPfn) = 1
pfn_kind(::CauchyFluidPfn) = 2
pfn_kind(::StrainRatePfn) = 3
pfn_kind(::StrainRateVorticityPfn) = 4
pfn_kind(::FluidSolidPfn) = 7
pfn_kind(::InterpolateFieldFn) = 8
pfn_kind(::NeighborCountFn) = 9
pfn_kind(f) = throw(ArgumentError("pairwise functor $(typeof(f)) has no device implementation"))

function pfn_params(f)
    p = [0.0, 0.0, 0.0, 2.0, NaN, NaN]
    f === nothing && return p
    if f isa FluidPfn || f isa CauchyFluidPfn || f isa FluidSolidPfn
        p[1] = f.art_visc_alpha; p[2] = f.art_visc_beta; p[3] = f.h
        f.delta === nothing || (p[5] = f.delta)
    end
    f isa FluidSolidPfn && (p[4] = typeof(f).parameters[1])
    if f isa InterpolateFieldFn
        fs, acc = typeof(f).parameters
        p[1] = Float64(reduce(|, (1 << GC_FIELD[s] for s in fs); init=0)); p[2] = acc ? 1.0 : 0.0
    end
    if f isa FluidPfn
        p[4] = typeof(f).parameters[1]
        f.epsilon === nothing || (p[6] = f.epsilon)
    end
    return p
end

upd_entry(u::ZeroFieldUpdater{S}) where {S} =
    (1, [Float64(reduce(|, (1 << GC_FIELD[s] for s in S); init=0)), 0, 0, 0, 0, 0])
upd_entry(u::TaitEOSUpdater) = (2, [u.rho0, u.gamma, 0, 0, 0, 0])
upd_entry(u::LinearEOSUpdater) = (3, [u.rho0, 0, 0, 0, 0, 0])
upd_entry(u::ElastoPlasticStressUpdater) = (4, [u.E, u.nu, u.phi, u.psi, u.cohesion, 0])
upd_entry(u::HookeLawStressUpdater) = (5, [u.E, u.nu, 0, 0, 0, 0])
function upd_entry(u::VirtualNormUpdater{S}) where {S}
    p = zeros(6)
    p[1:length(u.v_mult)] .= u.v_mult
    p[4] = Float64(reduce(|, (1 << GC_FIELD[s] for s in S); init=0))
    return (7, p)
end
upd_entry(u::PrescribedVelocityUpdater) = (8, zeros(6))
upd_entry(u) = throw(ArgumentError("state updater $(typeof(u)) has no device implementation"))

function set_updaters!(ctx, inst, handle, updaters)
    isempty(updaters) && return nothing
    lens = Cint[]; kinds = Cint[]; prm = Float64[]
    for entry in updaters
        chain = entry === nothing ? () : (entry isa Tuple ? entry : (entry,))
        push!(lens, length(chain))
        for u in chain
            k, p = upd_entry(u)
            push!(kinds, k); append!(prm, p)
        end
    end
    check(ctx, ccall((:gc_set_updaters, LIB), Cint,
                     (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cint}, Ptr{Cint}, Ptr{Cdouble}),
                     ctx, inst, handle, length(lens), lens, kinds, prm))
end

fields_of(ps) = [f for f in (:x, :v, :rho, :dvdt, :drhodt, :p, :stress, :strain_rate, :vorticity,
                               :strain, :strain_p, :id) if hasfield(typeof(ps), f)]

# The systems held on the device: the integrator's, then the virtual systems'
# sources (sorted, moved and filled on the device like the others).
function device_systems(lf)
    out = Any[ps for ps in lf.systems]
    for vps in lf.virtual_systems
        src = getfield(vps, :source)
        any(s -> s === src, out) || push!(out, src)
    end
    return out
end

# integrator kind of the C ABI (GC_INTEGRATOR_LEAPFROG / GC_INTEGRATOR_RK4)
integ_kind(::LeapFrogTimeIntegrator) = Cint(0)
integ_kind(::RK4TimeIntegrator) = Cint(1)

"""
    CudaLeapFrog(lf::Union{LeapFrogTimeIntegrator,RK4TimeIntegrator}; device=0)

A device context holding the model of `lf` (one instance), stepped with the
integrator `lf` is (LeapFrog or RK4).
"""
mutable struct CudaLeapFrog
    ctx::Ptr{Cvoid}
    lf::Union{LeapFrogTimeIntegrator,RK4TimeIntegrator}
    handles::IdDict{Any,Cint}
    inters::Vector{Cint}
end

function CudaLeapFrog(lf::Union{LeapFrogTimeIntegrator,RK4TimeIntegrator}; device::Integer=0)
    ctx = Ref{Ptr{Cvoid}}(C_NULL)
    check(C_NULL, ccall((:gc_ctx_create, LIB), Cint, (Cint, Csize_t, Ref{Ptr{Cvoid}}), device, 0, ctx))
    inst = Ref{Cint}(0)
    check(ctx[], ccall((:gc_instance_add, LIB), Cint, (Ptr{Cvoid}, Ref{Cint}), ctx[], inst))
    h = IdDict{Any,Cint}()
    for ps in lf.systems
        out = Ref{Cint}(0)
        ns = hasfield(typeof(ps), :stress) ? length(eltype(ps.stress)) : 0
        check(ctx[], ccall((:gc_add_system, LIB), Cint,
                           (Ptr{Cvoid}, Cint, Cint, Int64, Cint, Cint, Cdouble, Cdouble, Ptr{Cdouble}, Cdouble, Ref{Cint}),
                           ctx[], inst[], GC_SYS[typeof(ps).name.wrapper], ps.n, ps.ndims, ns, ps.mass, ps.c,
                           Vector{Float64}(ps.source_v), ps.source_rho, out))
        h[ps] = out[]
    end
    # virtual systems: the source becomes a system of its own, never integrated
    for vps in lf.virtual_systems
        src = getfield(vps, :source)
        if !haskey(h, src)
            out = Ref{Cint}(0)
            ns = hasfield(typeof(src), :stress) ? length(eltype(src.stress)) : 0
            check(ctx[], ccall((:gc_add_system, LIB), Cint,
                               (Ptr{Cvoid}, Cint, Cint, Int64, Cint, Cint, Cdouble, Cdouble, Ptr{Cdouble}, Cdouble,
                                Ref{Cint}),
                               ctx[], inst[], GC_SYS[typeof(src).name.wrapper], src.n, src.ndims, ns, src.mass,
                               src.c, Vector{Float64}(src.source_v), src.source_rho, out))
            h[src] = out[]
        end
        zf = typeof(vps).parameters[5]
        zmask = Cint(reduce(|, (1 << GC_FIELD[s] for s in zf); init=0))
        out = Ref{Cint}(0)
        check(ctx[], ccall((:gc_add_virtual, LIB), Cint, (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cdouble}, Ref{Cint}),
                           ctx[], inst[], h[src], zmask, Vector{Float64}(getfield(vps, :prescribed_v)), out))
        h[vps] = out[]
        set_updaters!(ctx[], inst[], h[vps], getfield(vps, :state_updater))
    end
    for ge in lf.ghosts
        g = ge.ghost
        nf = Cint[]; flds = Cint[]; mds = Cint[]
        for u in g.updaters
            if u === nothing
                push!(nf, 0)
            else
                fs, ms = typeof(u).parameters
                push!(nf, length(fs))
                for (f, m) in zip(fs, ms)
                    push!(flds, GC_FIELD[f]); push!(mds, m === nothing ? 0 : 1)
                end
            end
        end
        normals = reduce(vcat, [Vector(b.normal) for b in ge.boundaries])
        points = reduce(vcat, [Vector(b.point) for b in ge.boundaries])
        out = Ref{Cint}(0)
        check(ctx[], ccall((:gc_add_ghost, LIB), Cint,
                           (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cint}, Ptr{Cint}, Ptr{Cint}, Cint, Ptr{Cdouble},
                            Ptr{Cdouble}, Cdouble, Int64, Ref{Cint}),
                           ctx[], inst[], h[g.source], length(nf), nf, flds, mds, length(ge.boundaries),
                           normals, points, ge.cutoff, 0, out))
        h[g] = out[]
    end
    # probes (measured by measure_probes!) after the systems and virtual systems
    for pr in lf.probes
        ex = getfield(pr, :extras)
        mask = Cint(0); ns = Cint(0)
        for k in keys(ex)
            if haskey(GC_FIELD, k) && k in (:v, :rho, :p, :stress)
                mask |= Cint(1) << GC_FIELD[k]
                k === :stress && (ns = Cint(length(eltype(ex[k]))))
            else
                mask |= Cint(1) << 17  # GC_FIELD_COUNT: a NeighborCountFn array
            end
        end
        mt = getfield(pr, :mirror_target)
        pos = reduce(vcat, [Vector(p) for p in getfield(pr, :x)])
        out = Ref{Cint}(0)
        check(ctx[], ccall((:gc_add_probe, LIB), Cint,
                           (Ptr{Cvoid}, Cint, Int64, Cint, Ptr{Cdouble}, Cint, Cint, Cint, Ptr{Cdouble}, Ref{Cint}),
                           ctx[], inst[], pr.n, pr.ndims, pos, mt === nothing ? Cint(-1) : h[mt], mask, ns,
                           Vector{Float64}(getfield(pr, :prescribed_v)), out))
        h[pr] = out[]
        set_updaters!(ctx[], inst[], h[pr], getfield(pr, :state_updater))
    end
    for pi in lf.probe_interactions
        f = first(pi.pfns)
        out = Ref{Cint}(0)
        kk = pi.kernel isa CubicSplineKernel ? 0 : 1
        check(ctx[], ccall((:gc_add_probe_interaction, LIB), Cint,
                           (Ptr{Cvoid}, Cint, Cint, Cint, Cint, Cdouble, Cint, Ptr{Cdouble}, Ref{Cint}),
                           ctx[], inst[], h[pi.system_a], h[pi.system_b], kk, pi.kernel.h, pfn_kind(f),
                           pfn_params(f), out))
    end
    ints = Cint[]
    for si in lf.interactions
        b = si.system_b
        bh = Cint(-1)
        if b isa DynamicBoundarySystem || b isa StaticBoundarySystem
            if !haskey(h, b)
                out = Ref{Cint}(0)
                inner = getfield(b, :inner)
                if b isa DynamicBoundarySystem
                    check(ctx[], ccall((:gc_add_boundary, LIB), Cint,
                                       (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Cdouble, Ref{Cint}),
                                       ctx[], inst[], h[inner], GC_WRAP_DYNAMIC, Vector(b.boundary_normal),
                                       Vector(b.boundary_point), b.boundary_beta, out))
                else
                    z = zeros(ps_ndims(inner))
                    check(ctx[], ccall((:gc_add_boundary, LIB), Cint,
                                       (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Cdouble, Ref{Cint}),
                                       ctx[], inst[], h[inner], GC_WRAP_STATIC, z, z, b.lj_cutoff, out))
                end
                h[b] = out[]
            end
            bh = h[b]
        elseif b !== nothing
            bh = h[b]
        end
        kinds = Cint[pfn_kind(f) for f in si.pfns]
        prm = reduce(vcat, [pfn_params(f) for f in si.pfns])
        kk = si.kernel isa CubicSplineKernel ? 0 : 1
        out = Ref{Cint}(0)
        check(ctx[], ccall((:gc_add_interaction, LIB), Cint,
                           (Ptr{Cvoid}, Cint, Cint, Cint, Cint, Cdouble, Cint, Ptr{Cint}, Ptr{Cdouble}, Ref{Cint}),
                           ctx[], inst[], h[si.system_a], bh, kk, si.kernel.h, length(kinds), kinds, prm, out))
        push!(ints, out[])
        vf = si.vadjust_pfn
        if vf !== nothing
            vf isa XSPHPfn || throw(ArgumentError("velocity-adjust functor $(typeof(vf)) has no device implementation"))
            check(ctx[], ccall((:gc_set_velocity_adjust, LIB), Cint, (Ptr{Cvoid}, Cint, Cint, Cint, Cdouble),
                               ctx[], inst[], out[], 6, vf.epsilon))
        end
    end
    for ps in lf.systems
        isempty(ps.state_updater) && continue
        lens = Cint[]; kinds = Cint[]; prm = Float64[]
        for entry in ps.state_updater
            chain = entry === nothing ? () : (entry isa Tuple ? entry : (entry,))
            push!(lens, length(chain))
            for u in chain
                k, p = upd_entry(u)
                push!(kinds, k); append!(prm, p)
            end
        end
        check(ctx[], ccall((:gc_set_updaters, LIB), Cint,
                           (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cint}, Ptr{Cint}, Ptr{Cdouble}),
                           ctx[], inst[], h[ps], length(lens), lens, kinds, prm))
    end
    check(ctx[], ccall((:gc_set_integrator, LIB), Cint, (Ptr{Cvoid}, Cint, Cdouble), ctx[], inst[], lf.Γ))
    check(ctx[], ccall((:gc_set_integrator_kind, LIB), Cint, (Ptr{Cvoid}, Cint, Cint), ctx[], inst[],
                       integ_kind(lf)))
    check(ctx[], ccall((:gc_finalize, LIB), Cint, (Ptr{Cvoid},), ctx[]))
    cl = CudaLeapFrog(ctx[], lf, h, ints)
    finalizer(c -> ccall((:gc_ctx_destroy, LIB), Cint, (Ptr{Cvoid},), c.ctx), cl)
    return cl
end

ps_ndims(ps) = ps.ndims

function field_io!(cl::CudaLeapFrog, ps, f::Symbol, upload::Bool)
    arr = getfield(ps, f)
    fid = GC_FIELD[f]
    # the library moves Float64: a Float32 system's field goes through a
    # widened copy, rounded back to Float32 after a download
    wide = eltype(eltype(arr)) === Float32
    buf = wide ? Float64.(reinterpret(Float32, arr)) : arr
    GC.@preserve buf begin
        fn = upload ? :gc_upload_field : :gc_download_field
        st = ccall((fn, LIB), Cint, (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}, Csize_t),
                   cl.ctx, 0, cl.handles[ps], fid, pointer(buf), sizeof(buf))
        check(cl.ctx, st)
    end
    if wide && !upload
        reinterpret(Float32, arr) .= Float32.(buf)
    end
end

"""
    measure_probes!(cl::CudaLeapFrog)

The save-time probe measurement (`_measure_probes!`) on the device, then each
probe's x, id, w_sum and extras copied back in id order.
"""
function measure_probes!(cl::CudaLeapFrog)
    check(cl.ctx, ccall((:gc_measure_probes, LIB), Cint, (Ptr{Cvoid},), cl.ctx))
    for pr in cl.lf.probes
        h = cl.handles[pr]
        io(arr, fid) = GC.@preserve arr check(cl.ctx, ccall((:gc_download_field, LIB), Cint,
                                              (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}, Csize_t),
                                              cl.ctx, 0, h, fid, pointer(arr), sizeof(arr)))
        io(getfield(pr, :x), GC_FIELD.x)
        io(getfield(pr, :id), GC_FIELD.id)
        io(getfield(pr, :w_sum), 16)
        for (k, arr) in pairs(getfield(pr, :extras))
            if k in (:v, :rho, :p, :stress)
                io(arr, GC_FIELD[k])
            else
                buf = zeros(Float64, length(arr)); io(buf, 17)
                arr .= round.(eltype(arr), buf)
            end
        end
    end
    return nothing
end

function upload!(cl::CudaLeapFrog)
    for ps in device_systems(cl.lf), f in fields_of(ps)
        field_io!(cl, ps, f, true)
    end
end

function download!(cl::CudaLeapFrog)
    for ps in device_systems(cl.lf), f in fields_of(ps)
        field_io!(cl, ps, f, false)
    end
end

"""
    download_ghosts!(cl::CudaLeapFrog)

Each ghost system's current particles (generated and sorted on the device in
the last step) copied into its host arrays, resized to the device's count:
x, v, rho, idx_original, idx_boundary, normals and the copier extras.
"""
function download_ghosts!(cl::CudaLeapFrog)
    for ge in cl.lf.ghosts
        g = ge.ghost
        h = cl.handles[g]
        n = Ref{Int64}(0)
        check(cl.ctx, ccall((:gc_get_count, LIB), Cint, (Ptr{Cvoid}, Cint, Cint, Ref{Int64}), cl.ctx, 0, h, n))
        io(arr, fid) = GC.@preserve arr check(cl.ctx, ccall((:gc_download_field, LIB), Cint,
                                              (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}, Csize_t),
                                              cl.ctx, 0, h, fid, pointer(arr), sizeof(arr)))
        for (f, fid) in ((:x, GC_FIELD.x), (:v, GC_FIELD.v), (:rho, GC_FIELD.rho),
                         (:idx_original, 13), (:idx_boundary, 14), (:normals, 15))
            arr = getfield(g, f)
            resize!(arr, n[])
            n[] > 0 && io(arr, fid)
        end
        for (k, arr) in pairs(getfield(g, :extras))
            resize!(arr, n[])
            n[] > 0 && io(arr, GC_FIELD[k])
        end
    end
    return nothing
end

# _maybe_save!'s file (src/TimeIntegration.jl:520-549) from the downloaded
# state: step and sim_time attributes, one group per system, ghost system,
# virtual system and probe written by Grasph's own write_h5.
function save_h5(cl::CudaLeapFrog, output_prefix, global_step::Int, width::Int, dt)
    path = "$(output_prefix)_$(lpad(global_step, width, '0')).h5"
    d = dirname(path)
    !isempty(d) && mkpath(d)
    h5open(path, "w") do f
        HDF5.attrs(f)["step"] = global_step
        HDF5.attrs(f)["sim_time"] = Float64(global_step * dt)
        for ps in cl.lf.systems
            Grasph.write_h5(ps, create_group(f, ps.name))
        end
        for ge in cl.lf.ghosts
            Grasph.write_h5(ge.ghost, create_group(f, ge.ghost.name))
        end
        for vps in cl.lf.virtual_systems
            Grasph.write_h5(vps, create_group(f, vps.name))
        end
        for probe in cl.lf.probes
            Grasph.write_h5(probe, create_group(f, probe.name))
        end
    end
    return path
end

"""
    time_integrate!(cl::CudaLeapFrog, num_timesteps, print_interval_step,
                    save_interval_step, CFL, output_prefix; ...)

Device version of Grasph's LeapFrog `time_integrate!`
(src/TimeIntegration.jl:580).  Runs the steps on the GPU in chunks that end
at print/save boundaries, where the host arrays are refreshed and Grasph's
own `print_summary`/`write_h5` run.
"""
function Grasph.time_integrate!(cl::CudaLeapFrog, num_timesteps::Int, print_interval_step::Int,
                                save_interval_step::Int, CFL::Real, output_prefix;
                                step_offset::Int=0, output_width=nothing, kw...)
    T = typeof(cl.lf.c)
    dt = T(CFL) * cl.lf.h / cl.lf.c
    width = output_width === nothing ? ndigits(step_offset + num_timesteps) : output_width
    upload!(cl)
    done = 0
    while done < num_timesteps
        g = step_offset + done
        n = num_timesteps - done
        for iv in (print_interval_step, output_prefix === nothing ? 0 : save_interval_step)
            iv > 0 && (n = min(n, iv - g % iv))
        end
        check(cl.ctx, ccall((:gc_step, LIB), Cint, (Ptr{Cvoid}, Cint, Cdouble), cl.ctx, n, CFL))
        done += n
        g = step_offset + done
        if g % print_interval_step == 0
            download!(cl)
            foreach(print_summary, cl.lf.systems)
        end
        # _maybe_save!: probes measured, then the snapshot file
        if output_prefix !== nothing && g % save_interval_step == 0
            isempty(cl.lf.probes) || measure_probes!(cl)
            download!(cl)
            download_ghosts!(cl)
            save_h5(cl, output_prefix, g, width, dt)
        end
    end
    download!(cl)
    return nothing
end

end # module
