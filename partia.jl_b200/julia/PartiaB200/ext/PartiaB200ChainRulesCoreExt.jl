"""
The rrule of PointSamples_interpolation on the B200 backend: the pullback is
`psb_adjoint_points` (include/partia_b200.h), the vector-Jacobian product of
the interpolation with respect to the particle masses, positions and
quantity columns.  Smoothing lengths and densities are held fixed, and so is
the nearest particle's h (piecewise constant in the positions); their
tangents are marked not implemented.  The reference has no derivatives; this
is the ChainRulesCore form of the adjoint the library provides.

The rule is for the external-LBVH method, whose input is already in Morton
order and is not mutated: the gradients then come back in the input's own
order.  (The other method permutes its input in place, as LinearBVH! does,
which a reverse-mode rule cannot express; call `LinearBVH!(input)` first.)
"""
module PartiaB200ChainRulesCoreExt

using ChainRulesCore
using Partia
using Partia: InterpolationInput, InterpolationCatalog, PointSamples, LinearBVH, GridBundle,
              AbstractInterpolationStrategy, itpSymmetric
using PartiaB200
using PartiaB200: B200ComputeBackend, bound_context, b200_adjoint_points

function ChainRulesCore.rrule(::typeof(Partia.PointSamples_interpolation), backend::B200ComputeBackend,
        grid_template::PointSamples{3,Float64}, input::InterpolationInput{3,Float64}, LBVH::LinearBVH{3,Float64},
        catalog::InterpolationCatalog{3,N,G,Div,C,L},
        itp_strategy::Type{S} = itpSymmetric) where {N,G,Div,C,L,S<:AbstractInterpolationStrategy}
    bundle = Partia.PointSamples_interpolation(backend, grid_template, input, LBVH, catalog, itp_strategy)
    function pointsamples_pullback(Δ)
        Δb = unthunk(Δ)
        ns = length(grid_template.grid)
        # one cotangent vector per output field (zero where a field has none)
        gout = Vector{Vector{Float64}}(undef, L)
        for k in 1:L
            dk = Δb isa AbstractZero ? ZeroTangent() : unthunk(Δb.grids[k])
            gk = dk isa AbstractZero ? ZeroTangent() : unthunk(dk.grid)
            gout[k] = gk isa AbstractZero ? zeros(ns) : replace(Vector{Float64}(gk), NaN => 0.0)
        end
        ctx = bound_context(backend, input, LBVH)
        gm, gx, gy, gz, gcols = b200_adjoint_points(ctx, input.Npart, length(input.quant), grid_template,
                                                    catalog, itp_strategy, gout)
        dinput = Tangent{typeof(input)}(;
            coord = Tangent{typeof(input.coord)}(gx, gy, gz),
            m = gm,
            quant = Tangent{typeof(input.quant)}(gcols...),
            h = @not_implemented("smoothing lengths are held fixed by the adjoint"),
            ρ = @not_implemented("densities are held fixed by the adjoint"))
        return (NoTangent(), NoTangent(), NoTangent(), dinput, NoTangent(), NoTangent(), NoTangent())
    end
    return bundle, pointsamples_pullback
end

end # module
