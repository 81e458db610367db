# UncertainTeaB200Ext.jl -- the host side a maintainer adds to UncertainTea
# (shohei81/uncertaintea) to run its device path on this library's B200 kernels.
#
# It swaps in after lowering + staging (src/device/workspace.jl:88-137): the
# DeviceExecutionPlan that _lower_device_plan built (src/device/plan/lowering.jl:1360)
# and the DeviceStagingBundle of _stage_device_observations
# (src/device/staging.jl:11-39, 499) are translated into this library's kernel
# description -- one of the fixed families of include/ut_b200.h when the plan's
# steps match it, else a step program -- and every KernelAbstractions launch
# becomes a ccall into libut_b200.so.
#
# Julia is not installed in the container this library is built in, so this
# file is not executed there; tests/test_native_abi.py checks its struct
# mirrors and code tables against include/ut_b200.h, and the same C ABI is
# exercised from Python (uncertaintea_b200/_native.py) and plain C
# (tests/c_host/c_caller.c).
module UncertainTeaB200Ext

using UncertainTea, CUDA
using UncertainTea: DeviceExecutionPlan, DeviceStagingBundle, DeviceLiteralExpr, DeviceSlotExpr,
                    DevicePrimitiveExpr, DeviceObservedColumnExpr, DeviceLoopStep, DeviceDeterministicStep,
                    DeviceNoncenteredNormalChoiceStep, DeviceDiagNormalChoiceStepDyn, DeviceMvNormalChoiceStep,
                    DeviceBernoulliLogitGLMChoiceStep, DeviceBernoulliLogitGLMChoiceStepDyn,
                    DeviceBroadcastNormalChoiceStep, DeviceBernoulliLogitChoiceStep

const LIB = joinpath(@__DIR__, "..", "uncertaintea_b200", "libut_b200.so")

# ---- C struct mirrors (include/ut_b200.h), fields in header order ----------
struct UtPlanDesc                         # ut_plan_desc
    family::Int32; num_params::Int32; num_obs::Int32; num_coefs::Int32
    has_intercept::Int32; num_groups::Int32
    intercept_mu::Float64; intercept_sigma::Float64; coef_mu::Float64; coef_sigma::Float64
    mu_loc::Float64; mu_scale::Float64; tau_scale::Float64
    scale_shape::Float64; scale_rate::Float64
    prob_alpha::Float64; prob_beta::Float64
    nu_prior::Float64; nu_obs::Float64
    weibull_shape::Float64; weibull_scale::Float64
    obs_scale::Float64
end

struct UtExprNode                         # ut_expr_node
    op::Int32; a::Int32; b::Int32; reserved::Int32
    value::Float64
end

struct UtProgramStep                      # ut_program_step
    kind::Int32; dist::Int32
    arg::NTuple{4,Int32}
    value_source::Int32; obs_offset::Int32; transform::Int32; binding_slot::Int32
    count::Int32; width::Int32; body::Int32; iterator_slot::Int32; iterator_start::Int32
end

struct UtHmcBuffers                       # ut_hmc_buffers
    position::CuPtr{Float32}; gradient::CuPtr{Float32}; logjoint::CuPtr{Float32}
    inverse_mass::CuPtr{Float32}; step::CuPtr{Float32}
    accept_prob::CuPtr{Float32}; energy::CuPtr{Float32}; energy_error::CuPtr{Float32}
    accepted::CuPtr{UInt8}; divergent::CuPtr{UInt8}
    proposal::CuPtr{Float32}; endpoint_momentum::CuPtr{Float32}
end

struct UtNutsBuffers                      # ut_nuts_buffers
    position::CuPtr{Float32}; gradient::CuPtr{Float32}; logjoint::CuPtr{Float32}
    inverse_mass::CuPtr{Float32}; step::CuPtr{Float32}
    accept_prob::CuPtr{Float32}; energy::CuPtr{Float32}; energy_error::CuPtr{Float32}
    tree_depth::CuPtr{Int32}; integration_steps::CuPtr{Int32}
    divergent::CuPtr{UInt8}; moved::CuPtr{UInt8}
end

struct UtMeadsBuffers                     # ut_meads_buffers
    position::CuPtr{Float32}; gradient::CuPtr{Float32}; logjoint::CuPtr{Float32}
    momentum::CuPtr{Float32}; slice::CuPtr{Float32}
    accept_prob::CuPtr{Float32}; energy::CuPtr{Float32}; energy_error::CuPtr{Float32}
    accepted::CuPtr{UInt8}; divergent::CuPtr{UInt8}; integration_steps::CuPtr{Int32}
    fold_parameters::CuPtr{Float32}
end

# ---- codes (include/ut_b200.h) ----------------------------------------------
const UT_FAMILY_PROGRAM = Int32(8)
const UT_STEP_CHOICE = Int32(1)
const UT_STEP_DETERMINISTIC = Int32(2)
const UT_STEP_LOOP = Int32(3)
const UT_STEP_IID_NORMAL = Int32(4)
const UT_STEP_GLM_BERNOULLI_LOGIT = Int32(5)

# reference step type name => (UT_DIST_* code, argument field names in order)
const CHOICE_STEPS = Dict{Symbol,Tuple{Int32,Tuple}}(
    :DeviceNormalChoiceStep => (Int32(1), (:mu, :sigma)),
    :DeviceLognormalChoiceStep => (Int32(2), (:mu, :sigma)),
    :DeviceExponentialChoiceStep => (Int32(3), (:rate,)),
    :DeviceGammaChoiceStep => (Int32(4), (:shape, :rate)),
    :DeviceLaplaceChoiceStep => (Int32(5), (:loc, :scale)),
    :DeviceCauchyChoiceStep => (Int32(6), (:mu, :sigma)),
    :DeviceHalfNormalChoiceStep => (Int32(7), (:sigma,)),
    :DeviceHalfCauchyChoiceStep => (Int32(8), (:scale,)),
    :DeviceLogisticChoiceStep => (Int32(9), (:mu, :scale)),
    :DeviceGumbelChoiceStep => (Int32(10), (:mu, :scale)),
    :DeviceFrechetChoiceStep => (Int32(11), (:shape, :scale)),
    :DeviceRayleighChoiceStep => (Int32(12), (:scale,)),
    :DeviceInverseGaussianChoiceStep => (Int32(13), (:mu, :lambda)),
    :DeviceBetaChoiceStep => (Int32(14), (:alpha, :beta)),
    :DeviceStudentTChoiceStep => (Int32(15), (:nu, :mu, :sigma)),
    :DeviceInverseGammaChoiceStep => (Int32(16), (:shape, :scale)),
    :DeviceWeibullChoiceStep => (Int32(17), (:shape, :scale)),
    :DeviceBernoulliChoiceStep => (Int32(18), (:probability,)),
    :DeviceBernoulliLogitChoiceStep => (Int32(19), (:eta,)),
    :DevicePoissonChoiceStep => (Int32(20), (:lambda,)),
    :DeviceGeometricChoiceStep => (Int32(21), (:probability,)),
    :DeviceNegativeBinomialChoiceStep => (Int32(22), (:successes, :probability)),
    :DeviceBinomialChoiceStep => (Int32(23), (:trials, :probability)),
)

# DevicePrimitiveExpr{Op} => UT_EXPR_* (src/device/logjoint_kernel.jl:36-58)
const EXPR_OPS = Dict{Symbol,Int32}(
    :neg => 3, :+ => 4, :- => 5, :* => 6, :/ => 7, :^ => 8, :exp => 9, :log => 10, :log1p => 11, :sqrt => 12,
    :abs => 13, :min => 14, :max => 15, :sin => 16, :cos => 17, :tan => 18, :tanh => 19, :sinh => 20,
    :cosh => 21, :atan => 22, :expm1 => 23,
)

# ---- errors -----------------------------------------------------------------
function ut_check(status)
    status == 0 && return nothing
    buf = Vector{UInt8}(undef, 4096)
    ccall((:ut_last_error, LIB), Int32, (Ptr{UInt8}, Csize_t), buf, length(buf))
    msg = unsafe_string(pointer(buf))
    status in (1, 3, 4) && throw(ArgumentError(msg))       # ArgumentError
    status == 2 && throw(DimensionMismatch(msg))           # DimensionMismatch
    error(msg)
end

# ---- DeviceExecutionPlan => step program -----------------------------------
# The translation walks the plan in the reference's own order and replays its
# observation cursor (src/device/logjoint_kernel.jl:68-78: every observed
# choice consumes the next staged row; a GLM observation D + 1 rows; a loop
# its body's rows once per iteration), so each observed value, observation
# leaf and nested loop gets its row within the block of its loop depth.
# Julia slots, rows and loop ids are 1-based; the C program's are 0-based.
mutable struct ProgramBuilder
    steps::Vector{UtProgramStep}
    nodes::Vector{UtExprNode}
    num_slots::Int32
    trip_counts::Vector{Int32}
    loop_starts::Vector{Int32}
    issues::Vector{String}
end

node!(b::ProgramBuilder, op, a=0, c=0, v=0.0) =
    (push!(b.nodes, UtExprNode(Int32(op), Int32(a), Int32(c), Int32(0), Float64(v))); Int32(length(b.nodes) - 1))

lower_expr!(b::ProgramBuilder, e::DeviceLiteralExpr, depth) = node!(b, 0, 0, 0, e.value)
lower_expr!(b::ProgramBuilder, e::DeviceSlotExpr, depth) = node!(b, 1, e.slot - 1)
# covariate column of the current element block (broadcast / GLM staging)
lower_expr!(b::ProgramBuilder, e::DeviceObservedColumnExpr, depth) = node!(b, 2, e.offset, depth)
function lower_expr!(b::ProgramBuilder, e::DevicePrimitiveExpr{Op}, depth) where {Op}
    args = [lower_expr!(b, a, depth) for a in e.args]
    if Op === :- && length(args) == 1
        return node!(b, EXPR_OPS[:neg], args[1])
    elseif Op === :clamp                                   # clamp(x, lo, hi) = min(max(x, lo), hi)
        return node!(b, EXPR_OPS[:min], node!(b, EXPR_OPS[:max], args[1], args[2]), args[3])
    end
    haskey(EXPR_OPS, Op) || (push!(b.issues, "expression operation $(Op) has no device form"); return node!(b, 0))
    acc = args[1]
    length(args) == 1 && return node!(b, EXPR_OPS[Op], acc)
    for k = 2:length(args)                                 # variadic +, *, min, max fold left
        acc = node!(b, EXPR_OPS[Op], acc, args[k])
    end
    return acc
end

step!(b::ProgramBuilder; kind, dist=0, args=Int32[], value_source=-1, obs_offset=0, transform=0, binding_slot=-1,
      count=0, width=0, body=0, iterator_slot=-1, iterator_start=0) =
    push!(b.steps, UtProgramStep(Int32(kind), Int32(dist),
                                 ntuple(k -> k <= length(args) ? Int32(args[k]) : Int32(-1), 4),
                                 Int32(value_source), Int32(obs_offset), Int32(transform), Int32(binding_slot),
                                 Int32(count), Int32(width), Int32(body), Int32(iterator_slot),
                                 Int32(iterator_start)))

slot0(s) = s > 0 ? Int32(s - 1) : Int32(-1)

# Lowers steps at loop depth `depth`; `cursor` is the row within the current
# block (0-based); returns the cursor after them.
function lower_steps!(b::ProgramBuilder, steps::Tuple, depth, cursor)
    for s in steps
        cursor = lower_step!(b, s, depth, cursor)
    end
    return cursor
end

function lower_step!(b::ProgramBuilder, s, depth, cursor)
    name = nameof(typeof(s))
    if haskey(CHOICE_STEPS, name)
        dist, fields = CHOICE_STEPS[name]
        args = [lower_expr!(b, getfield(s, f), depth) for f in fields]
        if s.value_source > 0
            step!(b; kind=UT_STEP_CHOICE, dist=dist, args=args, value_source=s.value_source - 1,
                  transform=hasfield(typeof(s), :transform) ? s.transform : 0, binding_slot=slot0(s.binding_slot))
            return cursor
        end
        step!(b; kind=UT_STEP_CHOICE, dist=dist, args=args, value_source=-1, obs_offset=cursor,
              binding_slot=slot0(s.binding_slot))
        return cursor + 1
    elseif s isa DeviceNoncenteredNormalChoiceStep      # z ~ normal(0, 1) raw; binding = mu + sigma * z
        b.num_slots += 1
        z = b.num_slots - Int32(1)
        step!(b; kind=UT_STEP_CHOICE, dist=1, args=[node!(b, 0, 0, 0, 0.0), node!(b, 0, 0, 0, 1.0)],
              value_source=s.value_source - 1, binding_slot=z)
        theta = node!(b, EXPR_OPS[:+], lower_expr!(b, s.mu, depth),
                      node!(b, EXPR_OPS[:*], lower_expr!(b, s.sigma, depth), node!(b, 1, z)))
        step!(b; kind=UT_STEP_DETERMINISTIC, args=[theta], binding_slot=slot0(s.binding_slot))
        return cursor
    elseif s isa DeviceDeterministicStep
        step!(b; kind=UT_STEP_DETERMINISTIC, args=[lower_expr!(b, s.expr, depth)], binding_slot=slot0(s.binding_slot))
        return cursor
    elseif s isa DeviceDiagNormalChoiceStepDyn
        step!(b; kind=UT_STEP_IID_NORMAL, args=[lower_expr!(b, s.mu, depth), lower_expr!(b, s.sigma, depth)],
              value_source=s.value_source - 1, count=s.dimension)
        return cursor
    elseif s isa DeviceMvNormalChoiceStep               # diagonal: one scalar normal per component
        for d in eachindex(s.mu)
            args = [lower_expr!(b, s.mu[d], depth), lower_expr!(b, s.sigma[d], depth)]
            if s.value_source > 0
                step!(b; kind=UT_STEP_CHOICE, dist=1, args=args, value_source=s.value_source - 1 + d - 1)
            else
                step!(b; kind=UT_STEP_CHOICE, dist=1, args=args, obs_offset=cursor)
                cursor += 1
            end
        end
        return cursor
    elseif s isa DeviceLoopStep
        body = s.body
        # a loop whose body is only the fused GLM step is the GLM likelihood over its observations
        if length(body) == 1 && (body[1] isa DeviceBernoulliLogitGLMChoiceStepDyn ||
                                 body[1] isa DeviceBernoulliLogitGLMChoiceStep)
            g = body[1]
            D = g isa DeviceBernoulliLogitGLMChoiceStepDyn ? g.coef_length : typeof(g).parameters[1]
            n = b.trip_counts[s.loop_id]
            icpt = g.intercept isa DeviceLiteralExpr && iszero(g.intercept.value) ? Int32[] :
                   [lower_expr!(b, g.intercept, depth)]
            step!(b; kind=UT_STEP_GLM_BERNOULLI_LOGIT, args=icpt, value_source=g.coef_value_source - 1,
                  obs_offset=cursor, count=n, width=D)
            return cursor + n * (D + 1)
        end
        at = length(b.steps) + 1
        step!(b; kind=UT_STEP_LOOP)                       # patched below
        rows = lower_steps!(b, body, depth + 1, 0)
        n = b.trip_counts[s.loop_id]
        b.steps[at] = UtProgramStep(UT_STEP_LOOP, Int32(0), (Int32(-1), Int32(-1), Int32(-1), Int32(-1)),
                                    Int32(-1), Int32(cursor), Int32(0), Int32(-1), Int32(n), Int32(rows),
                                    Int32(length(b.steps) - at), slot0(s.iterator_slot),
                                    Int32(b.loop_starts[s.loop_id]))
        return cursor + n * rows
    elseif s isa DeviceBroadcastNormalChoiceStep        # element block: covariate columns, then y
        n = b.trip_counts[s.count_id]
        at = length(b.steps) + 1
        step!(b; kind=UT_STEP_LOOP)
        mu = lower_expr!(b, s.mu, depth + 1)
        sigma = lower_expr!(b, s.sigma, depth + 1)
        step!(b; kind=UT_STEP_CHOICE, dist=1, args=[mu, sigma], obs_offset=s.stride - 1)
        b.steps[at] = UtProgramStep(UT_STEP_LOOP, Int32(0), (Int32(-1), Int32(-1), Int32(-1), Int32(-1)),
                                    Int32(-1), Int32(cursor), Int32(0), Int32(-1), Int32(n), Int32(s.stride),
                                    Int32(1), Int32(-1), Int32(1))
        return cursor + n * s.stride
    end
    push!(b.issues, "plan step $(name) has no B200 form")
    return cursor
end

"""
    lower_program(plan, bundle, num_params) -> (steps, nodes, num_slots, issues)

The step program of a DeviceExecutionPlan and its staging bundle (one shared
observation column).  `issues` lists every step or expression without a
device form (the reference's device_lowering_report wording); the C library
checks the rest (ut_program_report).
"""
function lower_program(plan::DeviceExecutionPlan, bundle::DeviceStagingBundle, num_params::Integer)
    b = ProgramBuilder(UtProgramStep[], UtExprNode[], Int32(plan.slot_count), bundle.trip_counts,
                       bundle.loop_starts, String[])
    lower_steps!(b, plan.steps, 0, 0)
    return b.steps, b.nodes, b.num_slots, b.issues
end

# ---- workspace and entry points ----------------------------------------------
mutable struct B200Workspace
    handle::Ptr{Cvoid}
    P::Int
    C::Int
end

function B200Workspace(plan::DeviceExecutionPlan, bundle::DeviceStagingBundle, num_params::Integer, C::Integer)
    bundle.shared || throw(ArgumentError("per-chain observation columns are not supported; stage one shared column"))
    steps, nodes, nslots, issues = lower_program(plan, bundle, num_params)
    isempty(issues) || throw(ArgumentError("model cannot be lowered to the device path:\n  - " * join(issues, "\n  - ")))
    observed = vec(Float32.(bundle.observed[:, 1]))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    ut_check(ccall((:ut_workspace_create_program, LIB), Int32,
                   (Ptr{UtProgramStep}, Int32, Ptr{UtExprNode}, Int32, Int32, Int32, Ptr{Float32}, Int64, Int32,
                    Int32, Ref{Ptr{Cvoid}}),
                   steps, length(steps), nodes, length(nodes), nslots, num_params, observed, length(observed), C, 32,
                   h))
    ws = B200Workspace(h[], num_params, C)
    finalizer(w -> ccall((:ut_workspace_destroy, LIB), Int32, (Ptr{Cvoid},), w.handle), ws)
    return ws
end

# A plan of one of the fixed families (filled UtPlanDesc) skips the program:
# its kernels are specialised (tensor-core GLM, HBM-streaming few-chain GLM).
function B200Workspace(desc::UtPlanDesc, observed::Vector{Float32}, trip_counts::Vector{Int32},
                       loop_starts::Vector{Int32}, C::Integer)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    ut_check(ccall((:ut_workspace_create, LIB), Int32,
                   (Ref{UtPlanDesc}, Ptr{Float32}, Int64, Int64, Ptr{Int32}, Ptr{Int32}, Int32, Int32, Int32,
                    Ref{Ptr{Cvoid}}),
                   desc, observed, length(observed), 1, trip_counts, loop_starts, length(trip_counts), C, 32, h))
    ws = B200Workspace(h[], desc.num_params, C)
    finalizer(w -> ccall((:ut_workspace_destroy, LIB), Int32, (Ptr{Cvoid},), w.handle), ws)
    return ws
end

# device_batched_logjoint_gradient!(ws, params) -> (values, gradients); params P x C
function logjoint_gradient!(ws::B200Workspace, params::Matrix{Float32})
    size(params) == (ws.P, ws.C) || throw(DimensionMismatch("expected $((ws.P, ws.C)), got $(size(params))"))
    values = Vector{Float32}(undef, ws.C)
    grads = Matrix{Float32}(undef, ws.P, ws.C)
    ut_check(ccall((:ut_logjoint_gradient, LIB), Int32, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}),
                   ws.handle, params, values, grads))
    return values, grads
end

function logjoint_gradient!(ws::B200Workspace, params::CuMatrix{Float32}, values::CuVector{Float32},
                            grads::CuMatrix{Float32})
    ut_check(ccall((:ut_logjoint_gradient_device, LIB), Int32,
                   (Ptr{Cvoid}, CuPtr{Float32}, CuPtr{Float32}, CuPtr{Float32}, Ptr{Cvoid}),
                   ws.handle, params, values, grads, CUDA.stream().handle))
end

# one persistent-NUTS iteration (_device_persistent_nuts_proposals!, persistent_nuts.jl:678)
persistent_nuts_iteration!(ws::B200Workspace, bufs::UtNutsBuffers, max_depth, threshold, coord) =
    ut_check(ccall((:ut_persistent_nuts_iteration, LIB), Int32,
                   (Ptr{Cvoid}, Ref{UtNutsBuffers}, Int32, Float32, UInt32, Ptr{Cvoid}),
                   ws.handle, bufs, max_depth, threshold, coord, CUDA.stream().handle))

# one HMC / ChEES iteration (_device_leapfrog_integrate[_perchain]! + accept, hmc_kernels.jl:218-590)
hmc_iteration!(ws::B200Workspace, bufs::UtHmcBuffers, L, coord, threshold) =
    ut_check(ccall((:ut_hmc_iteration, LIB), Int32,
                   (Ptr{Cvoid}, Ref{UtHmcBuffers}, Int32, UInt32, Float32, Ptr{Cvoid}),
                   ws.handle, bufs, L, coord, threshold, CUDA.stream().handle))

end # module
