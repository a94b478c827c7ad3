"""
    PartiaB200

Partia's interpolation drivers on the B200 library `libpartia_b200` (the C ABI
of `include/partia_b200.h`), as an execution backend: the same methods the
CUDA extension adds (ext/CUDAExt/KernelInterpolation/grid_interpolation/
drivers/PointSamples_driver.jl:12,44 and LineSamples_driver.jl:11,49), for
`B200ComputeBackend()`.

    using Partia, PartiaB200
    result = PointSamples_interpolation(B200ComputeBackend(), grid, input, catalog, itpSymmetric)

`StructuredGrid_interpolation` is backend-generic in Partia and reaches these
methods through `PointSamples_interpolation`.  The library path is taken
from `ENV["PARTIA_B200_LIB"]` (default `libpartia_b200.so` on the loader's
search path).

Each `InterpolationInput` gets one library context, kept while its mass
array lives: the particles and the LBVH stay on the device between calls.
A driver call on an input whose coordinates and smoothing lengths still equal
the leaves of the LBVH last built from it (`matches_lbvh_leaf_order`) replaces
only the masses, densities and columns (`psb_set_values`) instead of
rebuilding: `LinearBVH!` would permute such an input by the identity and
build the same tree.
"""
module PartiaB200

using Libdl
using Partia
using Partia: InterpolationInput, InterpolationCatalog, PointSamples, LineSamples, LinearBVH, GridBundle,
              AbstractInterpolationStrategy, itpGather, itpScatter, itpSymmetric

export B200ComputeBackend

const libpsb = get(ENV, "PARTIA_B200_LIB", "libpartia_b200.so")

"""
    B200ComputeBackend(; device = 0, precision = :fp64)

Execution backend of the B200 library.  `precision = :fp32c` selects float
pair sums with compensated accumulation (double inclusion tests and
finalisation); `:fp64` computes in double throughout.
"""
struct B200ComputeBackend <: Partia.AbstractExecutionBackend
    device::Int
    precision::Symbol
end
B200ComputeBackend(; device::Integer = 0, precision::Symbol = :fp64) = B200ComputeBackend(Int(device), precision)

# ---- C ABI -----------------------------------------------------------------

# psb_catalog (include/partia_b200.h)
struct PsbCatalog
    n_scalar::Int32
    scalar_slots::Ptr{Int32}
    scalar_shepard::Ptr{UInt8}
    n_grad::Int32
    grad_slots::Ptr{Int32}
    n_div::Int32
    div_slots::Ptr{Int32}
    n_curl::Int32
    curl_slots::Ptr{Int32}
end

const PSB_FLAG_DEVICE_PTRS = UInt32(1)
const PSB_H_NEAREST = Cint(0)
const PSB_PREC_FP64 = Cint(0)
const PSB_PREC_FP32C = Cint(1)

strategy_code(::Type{itpGather}) = Cint(0)
strategy_code(::Type{itpScatter}) = Cint(1)
strategy_code(::Type{itpSymmetric}) = Cint(2)
dtype_code(::Type{Float64}) = Cint(0)
dtype_code(::Type{Float32}) = Cint(1)
precision_code(b::B200ComputeBackend) = b.precision === :fp32c ? PSB_PREC_FP32C : PSB_PREC_FP64
# psb_kernel: the input's smoothed_kernel (InterpolationInput.jl:41-49)
kernel_code(::Partia.M4_spline) = Cint(0)
kernel_code(::Partia.M5_spline) = Cint(1)
kernel_code(::Partia.M6_spline) = Cint(2)
kernel_code(::Partia.C2_Wendland) = Cint(3)
kernel_code(::Partia.C4_Wendland) = Cint(4)
kernel_code(::Partia.C6_Wendland) = Cint(5)

"""One `psb_ctx`: particles, LBVH and scratch of one input on one GPU."""
mutable struct PsbContext
    h::Ptr{Cvoid}
    device::Int
    function PsbContext(device::Integer = 0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:psb_create, libpsb), Cint, (Ptr{Ptr{Cvoid}}, Cint), r, device)
        rc == 0 || error("libpartia_b200: psb_create failed ($rc); is a CUDA device visible?")
        ctx = new(r[], Int(device))
        finalizer(c -> ccall((:psb_destroy, libpsb), Cint, (Ptr{Cvoid},), c.h), ctx)
        return ctx
    end
end

# Negative status -> the exception Partia raises for the same condition.
function check(ctx::PsbContext, rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:psb_last_error, libpsb), Cstring, (Ptr{Cvoid},), ctx.h))
    rc == -1 && throw(ArgumentError(msg))
    rc == -2 && throw(DimensionMismatch(msg))
    error("libpartia_b200: $msg (status $rc)")
end

# InterpolationCatalog -> the C catalog's arrays (0-based column slots; the
# density-gradient slot 0 becomes -1)
function concise(catalog::InterpolationCatalog)
    cc = Partia.to_concise_catalog(catalog)
    s = Int32[x - 1 for x in cc.scalar_slots]
    sh = UInt8[b ? 1 : 0 for b in cc.scalar_snormalization]
    g = Int32[x - 1 for x in cc.grad_slots]
    d = Int32[x - 1 for t in cc.div_slots for x in t]
    c = Int32[x - 1 for t in cc.curl_slots for x in t]
    return (s, sh, g, d, c)
end

psb_catalog(s, sh, g, d, c) = Ref(PsbCatalog(length(s), pointer(s), pointer(sh), length(g), pointer(g),
                                             length(d) ÷ 3, pointer(d), length(c) ÷ 3, pointer(c)))

const LEAF_ORDER_MSG = "Provided LBVH leaf order does not match the current input ordering. " *
                       "Ensure the LBVH was built from the same Morton-reordered input."
const LINE_MODE_MSG = "LineSamples_interpolation only supports itpScatter. " *
                      "Line-integrated samples do not have a well-defined query smoothing length ha, " *
                      "so itpGather and itpSymmetric are not supported."

# ---- one context per input ---------------------------------------------------

mutable struct InputState
    ctx::PsbContext
    # copies of the Morton-ordered coordinates and smoothing lengths the
    # context's tree was built from (nothing before the first build); the tree
    # is a function of these alone
    leaf_coor::Union{Nothing,NTuple{3,Vector}}
    leaf_scale::Union{Nothing,Vector}
    kernel::Cint                      # psb_kernel the particles were set with
end

# keyed on the input's mass vector: an InterpolationInput is immutable, its arrays are not
const STATES = WeakKeyDict{AbstractVector,InputState}()
const STATES_LOCK = ReentrantLock()

function input_state(backend::B200ComputeBackend, input::InterpolationInput)
    lock(STATES_LOCK) do
        st = get(STATES, input.m, nothing)
        if st === nothing || st.ctx.device != backend.device
            st = InputState(PsbContext(backend.device), nothing, nothing, Cint(-1))
            STATES[input.m] = st
        end
        return st
    end
end

# the context holds the tree of exactly these leaves
same_leaves(st::InputState, input::InterpolationInput) =
    st.leaf_scale !== nothing && st.kernel == kernel_code(input.smoothed_kernel) &&
    all(input.coord[d] == st.leaf_coor[d] for d in 1:3) && input.h == st.leaf_scale

function record_leaves!(st::InputState, input::InterpolationInput)
    st.leaf_coor = map(copy, input.coord)
    st.leaf_scale = copy(input.h)
    st.kernel = kernel_code(input.smoothed_kernel)
    return nothing
end

function set_particles!(ctx::PsbContext, input::InterpolationInput{3,TF}) where {TF}
    cols = collect(input.quant)
    colptrs = Ptr{Cvoid}[pointer(c) for c in cols]
    GC.@preserve cols colptrs input begin
        check(ctx, ccall((:psb_set_particles, libpsb), Cint,
            (Ptr{Cvoid}, Int64, Cint, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid},
             Ptr{Cvoid}, Int32, Ptr{Ptr{Cvoid}}, Cint, UInt32),
            ctx.h, input.Npart, dtype_code(TF), input.coord[1], input.coord[2], input.coord[3],
            input.m, input.h, input.ρ, Int32(length(cols)), colptrs, kernel_code(input.smoothed_kernel),
            UInt32(0)))
    end
    return nothing
end

function set_values!(ctx::PsbContext, input::InterpolationInput)
    cols = collect(input.quant)
    colptrs = Ptr{Cvoid}[pointer(c) for c in cols]
    GC.@preserve cols colptrs input begin
        check(ctx, ccall((:psb_set_values, libpsb), Cint,
            (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int32, Ptr{Ptr{Cvoid}}, UInt32),
            ctx.h, input.m, input.ρ, Int32(length(cols)), colptrs, UInt32(0)))
    end
    return nothing
end

function build!(ctx::PsbContext, n::Integer)
    perm = Vector{Int64}(undef, n)
    check(ctx, ccall((:psb_build_lbvh, libpsb), Cint, (Ptr{Cvoid}, Ptr{Int64}, Ptr{UInt64}), ctx.h, perm, C_NULL))
    return perm
end

"""
    b200_linear_bvh!(backend, input) -> order

`LinearBVH!(input)` on the device (InterpolationInput.jl:201-221): Morton
codes, sort, Karras tree and refit run on the GPU, the device copies are
permuted, and `input`'s own arrays are permuted in place by the returned
(1-based) order, exactly as `LinearBVH!` permutes them.  A host `LinearBVH`
for the external-LBVH overloads is still Partia's `LinearBVH!(input)`; on an
input already permuted here it finds the same order (the identity).
"""
function b200_linear_bvh!(backend::B200ComputeBackend, input::InterpolationInput{3,TF}) where {TF}
    st = input_state(backend, input)
    set_particles!(st.ctx, input)
    order = build!(st.ctx, input.Npart) .+ 1
    for v in (input.coord..., input.m, input.h, input.ρ, input.quant...)
        Base.permute!(v, order)
    end
    record_leaves!(st, input)
    return order
end

# The drivers' LinearBVH!(input) (initialize_interpolation.jl:50): an input
# still equal to the leaves of the context's tree would be permuted by the
# identity and get the same tree, so only its values are replaced.
function bound_context(backend::B200ComputeBackend, input::InterpolationInput)
    st = input_state(backend, input)
    if same_leaves(st, input)
        set_values!(st.ctx, input)
    else
        b200_linear_bvh!(backend, input)
    end
    return st.ctx
end

# An external LBVH whose leaf order `input` matches (checked by the caller):
# the tree is a function of the leaves, so the context's tree is rebuilt from
# `input` only when it holds other leaves; the input is then already in
# Morton order and the build's permutation is the identity.
function bound_context(backend::B200ComputeBackend, input::InterpolationInput, ::LinearBVH)
    st = input_state(backend, input)
    if same_leaves(st, input)
        set_values!(st.ctx, input)
        return st.ctx
    end
    set_particles!(st.ctx, input)
    perm = build!(st.ctx, input.Npart)
    perm == 0:input.Npart-1 || throw(ArgumentError(LEAF_ORDER_MSG))
    record_leaves!(st, input)
    return st.ctx
end

# ---- drivers ---------------------------------------------------------------------

function run_points(backend::B200ComputeBackend, ctx::PsbContext, grid_template::PointSamples{3,TF},
                    catalog::InterpolationCatalog, strategy) where {TF}
    s, sh, g, d, c = concise(catalog)
    grids, names, _ = Partia.initialize_interpolation(Partia.CPUComputeBackend(), grid_template, catalog)
    outs = Ptr{Cvoid}[pointer(gr.grid) for gr in grids]
    x, y, z = grid_template.coor
    GC.@preserve s sh g d c grids outs grid_template begin
        cat = psb_catalog(s, sh, g, d, c)
        # hmode PSB_H_NEAREST: the nearest particle's h, Partia's driver semantics (PointSamples_kernel.jl:19)
        check(ctx, ccall((:psb_interp_points, libpsb), Cint,
            (Ptr{Cvoid}, Int64, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ptr{Cvoid}, Cint,
             Ref{PsbCatalog}, Cint, Ptr{Ptr{Cvoid}}, UInt32, Ptr{Cvoid}),
            ctx.h, length(x), x, y, z, PSB_H_NEAREST, C_NULL, strategy_code(strategy), cat,
            precision_code(backend), outs, UInt32(0), C_NULL))
    end
    return GridBundle(grids, names)
end

function run_lines(backend::B200ComputeBackend, ctx::PsbContext, grid_template::LineSamples{3,TF},
                   catalog::InterpolationCatalog) where {TF}
    s, sh, g, d, c = concise(catalog)
    grids, names, _ = Partia.initialize_interpolation(Partia.CPUComputeBackend(), grid_template, catalog)
    outs = Ptr{Cvoid}[pointer(gr.grid) for gr in grids]
    o, m = grid_template.origin, grid_template.direction
    GC.@preserve s sh g d c grids outs grid_template begin
        cat = psb_catalog(s, sh, g, d, c)
        check(ctx, ccall((:psb_interp_lines, libpsb), Cint,
            (Ptr{Cvoid}, Int64, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid},
             Cint, Ptr{Cvoid}, Cint, Ref{PsbCatalog}, Cint, Ptr{Ptr{Cvoid}}, UInt32, Ptr{Cvoid}),
            ctx.h, length(o[1]), o[1], o[2], o[3], m[1], m[2], m[3], Cint(1), C_NULL,
            strategy_code(itpScatter), cat, precision_code(backend), outs, UInt32(0), C_NULL))
    end
    return GridBundle(grids, names)
end

# PointSamples_driver.jl:12 (CUDAExt) / :34-48 (CPU)
function Partia.PointSamples_interpolation(backend::B200ComputeBackend, grid_template::PointSamples{3,TF},
        input::InterpolationInput{3,TF}, catalog::InterpolationCatalog{3,N,G,Div,C,L},
        itp_strategy::Type{S} = itpSymmetric) where {N,G,Div,C,L,TF<:AbstractFloat,S<:AbstractInterpolationStrategy}
    ctx = bound_context(backend, input)
    return run_points(backend, ctx, grid_template, catalog, itp_strategy)
end

# PointSamples_driver.jl:44 (CUDAExt) / :98-118 (CPU)
function Partia.PointSamples_interpolation(backend::B200ComputeBackend, grid_template::PointSamples{3,TF},
        input::InterpolationInput{3,TF}, LBVH::LinearBVH{3,TF}, catalog::InterpolationCatalog{3,N,G,Div,C,L},
        itp_strategy::Type{S} = itpSymmetric) where {N,G,Div,C,L,TF<:AbstractFloat,S<:AbstractInterpolationStrategy}
    Partia.matches_lbvh_leaf_order(input, LBVH) || throw(ArgumentError(LEAF_ORDER_MSG))
    ctx = bound_context(backend, input, LBVH)
    return run_points(backend, ctx, grid_template, catalog, itp_strategy)
end

# LineSamples_driver.jl:11 (CUDAExt) / :39-55 (CPU)
function Partia.LineSamples_interpolation(backend::B200ComputeBackend, grid_template::LineSamples{3,TF},
        input::InterpolationInput{3,TF}, catalog::InterpolationCatalog{3,N,0,0,0,N},
        itp_strategy::Type{S} = itpScatter) where {N,TF<:AbstractFloat,S<:AbstractInterpolationStrategy}
    itp_strategy === itpScatter || throw(ArgumentError(LINE_MODE_MSG))
    ctx = bound_context(backend, input)
    return run_lines(backend, ctx, grid_template, catalog)
end

# LineSamples_driver.jl:49 (CUDAExt) / :116-141 (CPU)
function Partia.LineSamples_interpolation(backend::B200ComputeBackend, grid_template::LineSamples{3,TF},
        input::InterpolationInput{3,TF}, LBVH::LinearBVH{3,TF}, catalog::InterpolationCatalog{3,N,0,0,0,N},
        itp_strategy::Type{S} = itpScatter) where {N,TF<:AbstractFloat,S<:AbstractInterpolationStrategy}
    itp_strategy === itpScatter || throw(ArgumentError(LINE_MODE_MSG))
    Partia.matches_lbvh_leaf_order(input, LBVH) || throw(ArgumentError(LEAF_ORDER_MSG))
    ctx = bound_context(backend, input, LBVH)
    return run_lines(backend, ctx, grid_template, catalog)
end

"""
    b200_adjoint_points(ctx, grid_template, catalog, strategy, gout) -> (gm, gx, gy, gz, gcols)

`psb_adjoint_points`: for L = Σ_k Σ_s gout[k][s] out_k(s), the gradients with
respect to the particle masses, positions and columns, in the order the
particles were given to the context (the input's order).  FP64, double
particle data; h and ρ are held fixed, and so is the nearest particle's h.
"""
function b200_adjoint_points(ctx::PsbContext, n::Integer, ncol::Integer, grid_template::PointSamples{3,Float64},
                             catalog::InterpolationCatalog, strategy, gout::Vector{Vector{Float64}})
    s, sh, g, d, c = concise(catalog)
    gm, gx, gy, gz = zeros(n), zeros(n), zeros(n), zeros(n)
    gcols = [zeros(n) for _ in 1:ncol]
    gptr = Ptr{Cvoid}[pointer(v) for v in gout]
    cptr = Ptr{Float64}[pointer(v) for v in gcols]
    x, y, z = grid_template.coor
    GC.@preserve s sh g d c gout gptr gcols cptr grid_template begin
        cat = psb_catalog(s, sh, g, d, c)
        check(ctx, ccall((:psb_adjoint_points, libpsb), Cint,
            (Ptr{Cvoid}, Int64, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ptr{Cvoid}, Cint, Ref{PsbCatalog},
             Ptr{Ptr{Cvoid}}, Ptr{Float64}, Ptr{Ptr{Float64}}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
             UInt32, Ptr{Cvoid}),
            ctx.h, length(x), x, y, z, PSB_H_NEAREST, C_NULL, strategy_code(strategy), cat,
            gptr, gm, cptr, gx, gy, gz, UInt32(0), C_NULL))
    end
    return gm, gx, gy, gz, gcols
end

end # module
