# MarineHydroB200: the ccall / ChainRulesCore layer through which MarineHydro.jl
# reaches libmarinehydro_b200 (include/marinehydro_b200.h).  Include it beside
# the reference's module (src/MarineHydro.jl), where `Mesh`, the Green-function
# singletons and ChainRulesCore are in scope.
#
# UNTESTED: no Julia toolchain exists on the machines this library was built and
# measured on, so this file has never been loaded; the same entry points are
# exercised through Python ctypes by the repository's tests.
module MarineHydroB200
const lib = "libmarinehydro_b200"   # or the absolute path of the .so

const MH_GF = Dict(Rankine => 1, RankineReflected => 2, RankineReflectedNegative => 4,
                   GFWu => 8, ExactGuevelDelhommeau => 16)
gf_mask(gfs) = UInt32(sum(MH_GF[typeof(g)] for g in gfs))

check(rc, ctx) = rc == 0 || throw(ErrorException(unsafe_string(
    ccall((:mh_last_error, lib), Cstring, (Ptr{Cvoid},), ctx))))

mutable struct Context
    h::Ptr{Cvoid}
    function Context(device::Integer=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:mh_ctx_create, lib), Cint, (Cint, Ref{Ptr{Cvoid}}), device, r), C_NULL)
        c = new(r[]); finalizer(x -> ccall((:mh_ctx_destroy, lib), Cint, (Ptr{Cvoid},), x.h), c)
    end
end

mutable struct DeviceMesh
    h::Ptr{Cvoid}; ctx::Context
end
function DeviceMesh(ctx::Context, mesh::MarineHydro.Mesh)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    V = Matrix{Float64}(mesh.vertices); F = Matrix{Int64}(mesh.faces)
    C = Matrix{Float64}(mesh.centers);  N = Matrix{Float64}(mesh.normals)
    A = Vector{Float64}(mesh.areas);    R = Vector{Float64}(mesh.radii)
    GC.@preserve V F C N A R check(ccall((:mh_mesh_create, lib), Cint,
        (Ptr{Cvoid}, Int64, Int64, Ptr{Float64}, Ptr{Int64}, Ptr{Float64}, Ptr{Float64},
         Ptr{Float64}, Ptr{Float64}, Ref{Ptr{Cvoid}}),
        ctx.h, size(F, 1), size(V, 1), V, F, C, N, A, R, r), ctx.h)
    m = DeviceMesh(r[], ctx)
    finalizer(x -> ccall((:mh_mesh_destroy, lib), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), x.ctx.h, x.h), m)
end

# assemble_matrices(green_functions, mesh, wavenumber; direct) -- src/matrix_assembly.jl:4-42
function assemble_matrices(ctx, gfs, mesh, k; direct=true)
    dm = DeviceMesh(ctx, mesh); n = size(mesh.faces, 1)
    S = Matrix{ComplexF64}(undef, n, n); D = similar(S)
    check(ccall((:mh_assemble_matrices, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Float64, UInt32, Cint, Ptr{ComplexF64}, Ptr{ComplexF64}),
        ctx.h, dm.h, k, gf_mask(gfs), direct, S, D), ctx.h)
    S, D
end

# solve(D, S, bc; direct) -- src/matrix_assembly.jl:105-133
function solve(ctx, D, S, bc; direct=true)
    n = size(D, 1); B = reshape(Vector{ComplexF64}(vec(bc)), n, :); phi = similar(B)
    check(ccall((:mh_solve, lib), Cint,
        (Ptr{Cvoid}, Int64, Ptr{ComplexF64}, Ptr{ComplexF64}, Ptr{ComplexF64}, Int64, Cint,
         Ptr{ComplexF64}), ctx.h, n, D, S, B, size(B, 2), direct, phi), ctx.h)
    bc isa AbstractVector ? vec(phi) : phi
end

# calculate_radiation_forces(mesh, dof, omega) -- src/waves.jl:29-37
function calculate_radiation_forces(ctx, mesh, dof, omega;
        gfs=(Rankine(), RankineReflected(), GFWu()), direct=true, precision=0)
    dm = DeviceMesh(ctx, mesh); d = Matrix{Float64}(reshape(dof, :, 3)); out = zeros(2)
    check(ccall((:mh_calculate_radiation_forces, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Int64, Float64, Float64, Float64, UInt32, Cint,
         Cint, Ptr{Float64}), ctx.h, dm.h, d, size(d, 1), omega, SETTINGS.rho, SETTINGS.g,
        gf_mask(gfs), direct, precision, out), ctx.h)
    out
end

struct BatchInfo                      # mh_batch_info
    refine_iterations::Int32
    n_fallback::Int32
    max_rel_residual::Float64
end

# compute_hydrodynamic_coefficients -- src/problems_and_results.jl:231-236
# one call per body: all dofs radiating and influenced, all headings
function hydro_batch(ctx, mesh, omegas, dofs::Vector{Matrix{Float64}}, betas;
        gfs=(Rankine(), RankineReflected(), GFWu()), direct=true, precision=1,
        tol=1e-10, max_iter=30)
    dm = DeviceMesh(ctx, mesh); nd = length(dofs); nw = length(omegas); nb = length(betas)
    D = reduce(vcat, vec.(dofs)); A = zeros(nd, nd, nw); B = zeros(nd, nd, nw)
    Fd = zeros(ComplexF64, nd, nw, nb); Fk = zeros(ComplexF64, nd, nw, nb)
    info = Ref(BatchInfo(0, 0, 0.0))
    check(ccall((:mh_hydro_batch, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Ptr{Float64},
         Float64, Float64, UInt32, Cint, Cint, Float64, Cint, Ptr{Float64}, Ptr{Float64},
         Ptr{ComplexF64}, Ptr{ComplexF64}, Ref{BatchInfo}),
        ctx.h, dm.h, nw, Vector{Float64}(omegas), nd, D, nb, Vector{Float64}(betas),
        SETTINGS.rho, SETTINGS.g, gf_mask(gfs), direct, precision, tol, max_iter, A, B, Fd, Fk,
        info), ctx.h)
    (added_mass=A, radiation_damping=B, diffraction_force=Fd, Froude_Krylov_force=Fk,
     excitation_force=Fd .+ Fk)
end

# Adjoint: the pullback of hydro_batch (replaces Zygote through assemble_matrices /
# solve / integrate_pressure, src/matrix_assembly.jl:105-133 with ImplicitAD at :120).
# Returns the cotangents of the Mesh fields, of the frequencies and of the dofs.
function hydro_batch_vjp(ctx, mesh, omegas, dofs, betas, Abar, Bbar, Fdbar, Fkbar;
        gfs=(Rankine(), RankineReflected(), GFWu()), direct=true, precision=1,
        tol=1e-10, max_iter=30)
    dm = DeviceMesh(ctx, mesh); nd = length(dofs); nw = length(omegas); nb = length(betas)
    D = reduce(vcat, vec.(dofs))
    dV = zeros(mesh.nvertices, 3); dC = zeros(mesh.nfaces, 3); dN = zeros(mesh.nfaces, 3)
    dA = zeros(mesh.nfaces); dR = zeros(mesh.nfaces); dW = zeros(nw); dD = zeros(length(D))
    info = Ref(BatchInfo(0, 0, 0.0))
    check(ccall((:mh_hydro_batch_vjp, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Ptr{Float64},
         Float64, Float64, UInt32, Cint, Cint, Float64, Cint,
         Ptr{Float64}, Ptr{Float64}, Ptr{ComplexF64}, Ptr{ComplexF64},     # output cotangents
         Ptr{Float64}, Ptr{Float64}, Ptr{ComplexF64}, Ptr{ComplexF64},     # outputs (may be C_NULL)
         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
         Ptr{Float64}, Ref{BatchInfo}),
        ctx.h, dm.h, nw, Vector{Float64}(omegas), nd, D, nb, Vector{Float64}(betas),
        SETTINGS.rho, SETTINGS.g, gf_mask(gfs), direct, precision, tol, max_iter,
        Abar, Bbar, Fdbar, Fkbar, C_NULL, C_NULL, C_NULL, C_NULL,
        dV, dC, dN, dA, dR, dW, dD, info), ctx.h)
    mesh_bar = Tangent{Mesh}(vertices=dV, centers=dC, normals=dN, areas=dA, radii=dR)
    (mesh_bar, dW, [reshape(dD[(q-1)*3*mesh.nfaces+1:q*3*mesh.nfaces], :, 3) for q in 1:nd])
end

# Meshes generated on the device (mh_mesh_hemisphere / mh_mesh_wavebot): the
# WaveBot of src/meshes.jl:458-479 and the hemispheres the paper scripts load;
# parameters (radius, cx, cy, cz) and (r1, r2, d1, d2).
function hemisphere_mesh(ctx, radius, center, ntheta, nphi)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:mh_mesh_hemisphere, lib), Cint,
        (Ptr{Cvoid}, Float64, Float64, Float64, Float64, Cint, Cint, Ref{Ptr{Cvoid}}),
        ctx.h, radius, center[1], center[2], center[3], ntheta, nphi, r), ctx.h)
    m = DeviceMesh(r[], ctx)
    finalizer(x -> ccall((:mh_mesh_destroy, lib), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), x.ctx.h, x.h), m)
end
function wavebot_mesh(ctx, r1, r2, d1, d2; n_points=(5, 10, 5), n_theta=72)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:mh_mesh_wavebot, lib), Cint,
        (Ptr{Cvoid}, Float64, Float64, Float64, Float64, Cint, Cint, Cint, Cint, Ref{Ptr{Cvoid}}),
        ctx.h, r1, r2, d1, d2, n_points[1], n_points[2], n_points[3], n_theta, r), ctx.h)
    m = DeviceMesh(r[], ctx)
    finalizer(x -> ccall((:mh_mesh_destroy, lib), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), x.ctx.h, x.h), m)
end
# The generator-parameter cotangents of a mesh cotangent (the mesh_bar of
# hydro_batch_vjp): the device replacement of the finite-difference rrules of
# paper/MeshGradients_singlebody.jl:85-167.
function mesh_param_vjp(ctx, dm::DeviceMesh, mesh_bar)
    np = Ref{Cint}(0)
    check(ccall((:mh_mesh_nparams, lib), Cint, (Ptr{Cvoid}, Ref{Cint}), dm.h, np), ctx.h)
    out = zeros(np[])
    check(ccall((:mh_mesh_param_vjp, lib), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
         Ptr{Float64}),
        ctx.h, dm.h, mesh_bar.vertices, mesh_bar.centers, mesh_bar.normals, mesh_bar.areas,
        mesh_bar.radii, out), ctx.h)
    out
end
end

# One Zygote node per batch call (ChainRulesCore):
function ChainRulesCore.rrule(::typeof(MarineHydroB200.hydro_batch), ctx, mesh, omegas, dofs, betas;
                              kw...)
    y = MarineHydroB200.hydro_batch(ctx, mesh, omegas, dofs, betas; kw...)
    function pullback(ȳ)
        mesh_bar, dW, dD = MarineHydroB200.hydro_batch_vjp(ctx, mesh, omegas, dofs, betas,
            unthunk(ȳ.added_mass), unthunk(ȳ.radiation_damping),
            unthunk(ȳ.diffraction_force) .+ unthunk(ȳ.excitation_force),
            unthunk(ȳ.Froude_Krylov_force) .+ unthunk(ȳ.excitation_force); kw...)
        (NoTangent(), NoTangent(), mesh_bar, dW, dD, NoTangent())
    end
    y, pullback
end
