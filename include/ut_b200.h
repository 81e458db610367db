/*
 * ut_b200.h -- C ABI of the B200 (sm_100a) batched density + sampler library.
 *
 * This is the boundary a host language binds (Julia `ccall`, Python `ctypes`).
 * Every signature uses plain C types: pointers, sizes, and two plain structs.
 * No C++ or torch types cross it.
 *
 * Layout conventions (identical to UncertainTea's column-major Julia arrays):
 *   - a "P x C" matrix holds C chains, each chain's P unconstrained parameters
 *     contiguous (chain c, parameter p at index c*P + p);
 *   - a "C" vector holds one value per chain.
 *
 * Host-pointer entry points copy in, run on the current CUDA device, copy out
 * and synchronise before returning (the reference's `copyto!` + `synchronize`
 * boundary).  Entry points whose names end in `_device`, and the sampler
 * iteration entry points, take DEVICE pointers and a `cudaStream_t` passed as
 * `void*` (NULL = legacy default stream); they return once the work is queued.
 *
 * Status codes are returned by every entry point; the message of the last
 * failure on the calling thread is available through ut_last_error.
 * No entry point falls back to a CPU path.
 */
#ifndef UT_B200_H
#define UT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define UT_OK                  0
#define UT_ERR_ARGUMENT        1  /* reference: ArgumentError                    */
#define UT_ERR_DIMENSION       2  /* reference: DimensionMismatch                */
#define UT_ERR_UNSUPPORTED     3  /* model not lowerable to a kernel description */
#define UT_ERR_PRECISION       4  /* precision other than Float32 requested      */
#define UT_ERR_CUDA            5  /* a CUDA runtime call failed                  */
#define UT_ERR_NO_DEVICE       6  /* no CUDA device visible                      */
#define UT_ERR_DEVICE_TIMEOUT  7  /* a bounded in-kernel wait gave up            */

/* Largest observation count of a kernel description (and of the
 * allocation-free GLM entry point): the kernels index observations in 32-bit
 * arithmetic, and 2^30 keeps every split end in range. */
#define UT_MAX_OBS (1 << 30)

/* ---- model families a kernel description can hold ---------------------- */
/* Bernoulli-logit GLM: optional intercept ~ normal, coefficients ~ iid normal,
 * y_i ~ bernoullilogit(intercept + x_i . beta).  Lowered form of the
 * reference's DeviceBernoulliLogitGLMChoiceStepDyn + DeviceDiagNormalChoiceStepDyn
 * (src/device/plan/steps.jl:205-225, 334-340). */
#define UT_FAMILY_GLM_BERNOULLI_LOGIT        1
/* Non-centred hierarchical normal: mu ~ normal(mu_loc, mu_scale),
 * tau ~ halfcauchy(tau_scale) (log transform), z_j ~ normal(0, 1),
 * y_ij ~ normal(mu + tau * z_j, sigma_j).  Semantics of the reference's
 * `reparam=:noncentered` iid latent (docs/noncentered-reparam.md:22-36). */
#define UT_FAMILY_HIER_NORMAL_NONCENTERED    2
/* Normal location/scale with a gamma scale: mu ~ normal(mu_loc, mu_scale),
 * s ~ gamma(scale_shape, scale_rate) (log transform, log|J| = log s),
 * y_i ~ normal(mu, s) for i = 1..N.  The reference's device-lowerable
 * gaussian model (DeviceNormalChoiceStep + DeviceGammaChoiceStep + a
 * DeviceLoopStep of normal observations, src/device/plan/steps.jl:6-44,
 * 445-449; scored at src/device/logjoint_kernel.jl:105-111, 146-151). */
#define UT_FAMILY_NORMAL_LOCATION_SCALE      3
/* Bernoulli observations of a beta probability: p ~ beta(prob_alpha,
 * prob_beta) (logit transform, log|J| = -|u| - 2 log1p(exp(-|u|))),
 * z_i ~ bernoulli(p) for i = 1..N.  The reference's device-lowerable
 * bernoulli model (DeviceBetaChoiceStep with the logit transform and a loop
 * of Bernoulli observations; math.jl:161-165, 191-195, 1144-1159). */
#define UT_FAMILY_BERNOULLI_BETA             4
/* Normal observations with a lognormal log-scale and a gamma location:
 * a ~ lognormal(mu_loc, mu_scale), b ~ gamma(scale_shape, scale_rate) (both
 * log transform), y_i ~ normal(b, exp(a)) for i = 1..N.  The reference's
 * device-lowerable lognormal/gamma model (math.jl:93-97, 103-107; an
 * exp-derived scale argument). */
#define UT_FAMILY_LOGNORMAL_GAMMA_NORMAL     5
/* Heavy-tailed location with two scales: loc ~ studentt(nu_prior, mu_loc,
 * mu_scale) (identity), s ~ inversegamma(scale_shape, scale_rate) and
 * w ~ weibull(weibull_shape, weibull_scale) (both log transform),
 * y_i ~ studentt(nu_obs, loc, s + w).  The reference's device-lowerable
 * heavy-tail model (math.jl:167-186). */
#define UT_FAMILY_STUDENTT_HEAVY_TAIL        6
/* Normal location with a known observation scale: mu ~ normal(mu_loc,
 * mu_scale) (identity), y_i ~ normal(mu, obs_scale) for i = 1..N.  The
 * reference's conjugate gaussian gate model (a DeviceNormalChoiceStep and
 * normal observations with a constant scale argument; the persistent-NUTS and
 * ChEES device tests, test/uncertaintea/core/device_persistent_nuts.jl:33-38,
 * device_chees.jl:26-32). */
#define UT_FAMILY_NORMAL_KNOWN_SCALE         7

/* Fixed kernel description: what the host lowers a model's execution plan to
 * (reference: DeviceExecutionPlan, src/device/plan/steps.jl:482-489, produced
 * by _lower_device_plan, src/device/plan/lowering.jl:1360).  Parameter rows:
 *   GLM : [intercept (if has_intercept)] then num_coefs coefficients;
 *   HIER: [mu, log(tau), z_1 .. z_J];
 *   NLS : [mu, log(s)];
 *   BB  : [logit(p)];
 *   LGN : [log(a), log(b)];
 *   HT  : [loc, log(s), log(w)];
 *   NKS : [mu]. */
typedef struct ut_plan_desc {
    int32_t family;          /* UT_FAMILY_*                                   */
    int32_t num_params;      /* P, unconstrained parameter count              */
    int32_t num_obs;         /* N, observations                               */
    int32_t num_coefs;       /* GLM: D covariates                             */
    int32_t has_intercept;   /* GLM: 1 if an intercept row leads the params   */
    int32_t num_groups;      /* HIER: J groups                                */
    double intercept_mu;     /* GLM: intercept ~ normal(intercept_mu, ...)    */
    double intercept_sigma;
    double coef_mu;          /* GLM: beta_d ~ normal(coef_mu, coef_sigma)     */
    double coef_sigma;
    double mu_loc;           /* HIER: mu ~ normal(mu_loc, mu_scale)           */
    double mu_scale;
    double tau_scale;        /* HIER: tau ~ halfcauchy(tau_scale)             */
    double scale_shape;      /* NLS: s ~ gamma(scale_shape, scale_rate)       */
    double scale_rate;       /*      (mu uses mu_loc / mu_scale)              */
    double prob_alpha;       /* BB: p ~ beta(prob_alpha, prob_beta)           */
    double prob_beta;
    double nu_prior;         /* HT: loc ~ studentt(nu_prior, mu_loc, mu_scale) */
    double nu_obs;           /*     y ~ studentt(nu_obs, loc, s + w)          */
    double weibull_shape;    /*     w ~ weibull(weibull_shape, weibull_scale) */
    double weibull_scale;    /*     (s uses scale_shape / scale_rate)         */
    double obs_scale;        /* NKS: y ~ normal(mu, obs_scale)                */
} ut_plan_desc;

typedef struct ut_workspace ut_workspace;

/* ---- library / errors -------------------------------------------------- */
const char* ut_version(void);
/* Copies the last error message of this thread into buf (NUL-terminated,
 * truncated to len) and returns its full length. */
int32_t ut_last_error(char* buf, size_t len);
/* Number of visible CUDA devices (0 when none). */
int32_t ut_device_count(void);

/* ---- lowering report ----------------------------------------------------
 * reference: device_lowering_report (src/device/workspace.jl:24-35).
 * Returns UT_OK when the description is supported, else UT_ERR_UNSUPPORTED
 * with the issue list written to `issues`. */
int32_t ut_lowering_report(const ut_plan_desc* plan, char* issues, size_t len);

/* ---- workspace ------------------------------------------------------------
 * reference: DeviceBatchedWorkspace(model, C; backend, precision, args,
 * constraints) (src/device/workspace.jl:71-137).  `observed` is the staged
 * observation buffer, one shared column (reference DeviceStagingBundle,
 * src/device/staging.jl:11-39):
 *   GLM : observed_rows = N*(D+1): per observation the D covariates then y;
 *   HIER: observed_rows = N + J:  the N y values group after group, then the
 *         J fixed sigma_j; trip_counts[j] = n_j and loop_starts[j] = first row
 *         of group j (num_loops = J);
 *   NLS : observed_rows = N: the y values (no loops are passed);
 *   BB  : observed_rows = N: the z values;
 *   LGN : observed_rows = N: the y values;
 *   HT  : observed_rows = N: the y values.
 * precision_bits must be 32 (Float32); anything else is UT_ERR_PRECISION. */
int32_t ut_workspace_create(const ut_plan_desc* plan,
                            const float* observed, int64_t observed_rows, int64_t observed_cols,
                            const int32_t* trip_counts, const int32_t* loop_starts, int32_t num_loops,
                            int32_t batch_size, int32_t precision_bits,
                            ut_workspace** out);
int32_t ut_workspace_destroy(ut_workspace* ws);
int32_t ut_workspace_info(const ut_workspace* ws, int32_t* num_params, int32_t* batch_size);
/* Which kernel family evaluates this workspace's density: 1 = one warp per
 * chain (observation data staged in shared memory), 2 = CUDA-core
 * observation-tiled GEMM path, 3 = tensor-core (tcgen05, 3xTF32) path,
 * 4 = HBM-streaming path for a few chains (C <= 16, GLM with P % 4 == 0 and
 * P <= 128). */
int32_t ut_workspace_path(const ut_workspace* ws);

/* ---- composable kernel description: the step program -----------------------
 * reference: the step tuple of DeviceExecutionPlan (src/device/plan/steps.jl:
 * 6-489) that _lower_device_plan produces (src/device/plan/lowering.jl:1360),
 * walked by _device_logjoint_kernel! (src/device/logjoint_kernel.jl:724) and
 * _device_gradient_kernel! (src/device/gradient_kernel.jl:1124).  Where a
 * model matches none of the fixed families above, the host passes its plan
 * step by step: choice steps (a distribution, argument expressions, a value
 * that is a latent parameter row or a staged observation, a transform, a
 * binding slot), deterministic steps, loops, the iid normal vector prior
 * (DeviceDiagNormalChoiceStepDyn, steps.jl:334-340) and the fused
 * Bernoulli-logit GLM likelihood (DeviceBernoulliLogitGLMChoiceStep[Dyn],
 * steps.jl:181-225).  The logjoint and its full gradient come from one pass.
 *
 * Observations: the staged buffer is read in blocks.  The top level is one
 * block (row 0 ..); a loop's iteration t is the block that starts at row
 * `obs_offset + t * width` of the enclosing block; an observed value, an
 * observation leaf of an expression and a nested loop each name their row in
 * the block of their own loop depth, so the host fixes every row statically
 * (the reference's cursor, src/device/logjoint_kernel.jl:68-78, 620-634).
 * Slots (0 .. num_slots-1) hold the values of bindings and iterators, as the
 * reference's `slots` buffer; parameters rows are 0-based. */
#define UT_FAMILY_PROGRAM 8

#define UT_STEP_CHOICE              1  /* value ~ dist(args...)                         */
#define UT_STEP_DETERMINISTIC       2  /* slot = expression (DeviceDeterministicStep)   */
#define UT_STEP_LOOP                3  /* `count` iterations of the next `body` steps    */
#define UT_STEP_IID_NORMAL          4  /* `count` latent rows ~ normal(arg0, arg1)      */
#define UT_STEP_GLM_BERNOULLI_LOGIT 5  /* `count` observations, each `width` covariates
                                        * then y ~ bernoullilogit(arg0 + x . beta), beta
                                        * = `width` latent rows from value_source       */

/* Distributions of UT_STEP_CHOICE; the argument order is the reference step's
 * field order (math.jl:88-300).  Values of 18-23 must be observed. */
#define UT_DIST_NORMAL             1  /* mu, sigma          */
#define UT_DIST_LOGNORMAL          2  /* mu, sigma          */
#define UT_DIST_EXPONENTIAL        3  /* rate               */
#define UT_DIST_GAMMA              4  /* shape, rate        */
#define UT_DIST_LAPLACE            5  /* loc, scale         */
#define UT_DIST_CAUCHY             6  /* mu, sigma          */
#define UT_DIST_HALFNORMAL         7  /* sigma              */
#define UT_DIST_HALFCAUCHY         8  /* scale              */
#define UT_DIST_LOGISTIC           9  /* mu, scale          */
#define UT_DIST_GUMBEL            10  /* mu, scale          */
#define UT_DIST_FRECHET           11  /* shape, scale       */
#define UT_DIST_RAYLEIGH          12  /* scale              */
#define UT_DIST_INVERSEGAUSSIAN   13  /* mu, lambda         */
#define UT_DIST_BETA              14  /* alpha, beta        */
#define UT_DIST_STUDENTT          15  /* nu, mu, sigma      */
#define UT_DIST_INVERSEGAMMA      16  /* shape, scale       */
#define UT_DIST_WEIBULL           17  /* shape, scale       */
#define UT_DIST_BERNOULLI         18  /* p                  */
#define UT_DIST_BERNOULLI_LOGIT   19  /* eta                */
#define UT_DIST_POISSON           20  /* lambda             */
#define UT_DIST_GEOMETRIC         21  /* p                  */
#define UT_DIST_NEGATIVE_BINOMIAL 22  /* successes, p       */
#define UT_DIST_BINOMIAL          23  /* trials, p          */

/* Transforms of a latent scalar value (math.jl:1137-1159). */
#define UT_TRANSFORM_IDENTITY 0
#define UT_TRANSFORM_LOG      1       /* value = exp(u), log|J| = u                    */
#define UT_TRANSFORM_LOGIT    2       /* value = logistic(u), log|J| = -|u| - 2 log1p(exp(-|u|)) */

/* Expression nodes (reference DeviceLiteralExpr / DeviceSlotExpr /
 * DevicePrimitiveExpr / DeviceObservedColumnExpr, src/device/plan/exprs.jl).
 * An operand `a` / `b` is the index of an earlier node. */
#define UT_EXPR_LITERAL  0   /* `value`                                                     */
#define UT_EXPR_SLOT     1   /* slot `a`                                                    */
#define UT_EXPR_OBS      2   /* observation row `a` of the block at loop depth `b` (0 = top) */
#define UT_EXPR_NEG      3
#define UT_EXPR_ADD      4
#define UT_EXPR_SUB      5
#define UT_EXPR_MUL      6
#define UT_EXPR_DIV      7
#define UT_EXPR_POW      8
#define UT_EXPR_EXP      9
#define UT_EXPR_LOG     10
#define UT_EXPR_LOG1P   11
#define UT_EXPR_SQRT    12
#define UT_EXPR_ABS     13
#define UT_EXPR_MIN     14
#define UT_EXPR_MAX     15
#define UT_EXPR_SIN     16
#define UT_EXPR_COS     17
#define UT_EXPR_TAN     18
#define UT_EXPR_TANH    19
#define UT_EXPR_SINH    20
#define UT_EXPR_COSH    21
#define UT_EXPR_ATAN    22
#define UT_EXPR_EXPM1   23

typedef struct ut_expr_node {
    int32_t op;            /* UT_EXPR_*                                           */
    int32_t a;             /* operand node / slot / observation row               */
    int32_t b;             /* operand node / loop depth of an observation row     */
    int32_t reserved;      /* 0                                                   */
    double value;          /* UT_EXPR_LITERAL                                     */
} ut_expr_node;

typedef struct ut_program_step {
    int32_t kind;          /* UT_STEP_*                                                  */
    int32_t dist;          /* UT_STEP_CHOICE: UT_DIST_*                                  */
    int32_t arg[4];        /* root node of each argument expression, -1 = none          */
    int32_t value_source;  /* >= 0: first parameter row of a latent value; -1: observed */
    int32_t obs_offset;    /* row of an observed value / of a loop's first block         */
    int32_t transform;     /* UT_TRANSFORM_* of a latent scalar choice                   */
    int32_t binding_slot;  /* slot that receives the value, -1 = none                    */
    int32_t count;         /* LOOP: iterations; IID_NORMAL: rows; GLM: observations      */
    int32_t width;         /* LOOP: rows per iteration block; GLM: covariates            */
    int32_t body;          /* LOOP: number of following steps in its body (nested too)   */
    int32_t iterator_slot; /* LOOP: slot holding iterator_start + t, -1 = none           */
    int32_t iterator_start;
} ut_program_step;

/* Checks a step program (the device_lowering_report of a program): UT_OK or
 * UT_ERR_UNSUPPORTED with the issues.  observed_rows = the staged rows. */
int32_t ut_program_report(const ut_program_step* steps, int32_t num_steps, const ut_expr_node* nodes,
                          int32_t num_nodes, int32_t num_slots, int32_t num_params, int64_t observed_rows,
                          char* issues, size_t len);
/* A workspace over a step program (DeviceBatchedWorkspace of a model outside
 * the fixed families); every other workspace entry point and every sampler
 * accepts it.  Parameters: 1 <= P <= 256, every row read by exactly one
 * latent step. */
int32_t ut_workspace_create_program(const ut_program_step* steps, int32_t num_steps, const ut_expr_node* nodes,
                                    int32_t num_nodes, int32_t num_slots, int32_t num_params,
                                    const float* observed, int64_t observed_rows, int32_t batch_size,
                                    int32_t precision_bits, ut_workspace** out);
/* Synchronises the workspace's work and reports the sticky device error word:
 * UT_ERR_DEVICE_TIMEOUT when a bounded in-kernel wait gave up since the last
 * check (the word is cleared by this call), else UT_OK.  Until it is cleared,
 * kernels that wait on barriers return early instead of waiting. */
int32_t ut_workspace_check(ut_workspace* ws, void* stream);

/* ---- batched density ------------------------------------------------------
 * reference: device_batched_logjoint! (src/device/workspace.jl:276-307) and
 * device_batched_logjoint_gradient! (src/device/api.jl:82-107).
 * Host buffers: params P x C, totals C, gradients P x C. */
int32_t ut_logjoint(ut_workspace* ws, const float* params, float* totals);
int32_t ut_logjoint_gradient(ut_workspace* ws, const float* params, float* totals, float* gradients);
/* Same computations on device-resident buffers (the kernel launch sites of
 * src/device/workspace.jl:290-301 and src/device/tiled_gradient.jl:292-390). */
int32_t ut_logjoint_device(ut_workspace* ws, const float* d_params, float* d_totals, void* stream);
int32_t ut_logjoint_gradient_device(ut_workspace* ws, const float* d_params, float* d_totals,
                                    float* d_gradients, void* stream);

/* ---- Philox4x32-10 stream ---------------------------------------------------
 * reference: philox4x32 (src/device/rng.jl:95-119), device_rand_uniform
 * (:165-174), device_rand_normal (:196-219).  Host buffers; computed on the
 * GPU.  keys: n x 2, counters: n x 4, out: n x 4 words. */
int32_t ut_philox4x32(const uint32_t* keys, const uint32_t* counters, int64_t n, uint32_t* out);
/* out[i] = device_rand_{uniform,normal}(Float32, chain, iteration, stream, draw_start + i) */
int32_t ut_rand_uniform(uint32_t chain, uint32_t iteration, uint32_t stream, uint32_t draw_start,
                        int64_t n, float* out);
int32_t ut_rand_normal(uint32_t chain, uint32_t iteration, uint32_t stream, uint32_t draw_start,
                       int64_t n, float* out);

/* ---- samplers (device buffers) -------------------------------------------- */
/* Per-iteration buffers of one HMC / ChEES iteration.  position, gradient and
 * logjoint hold the chains' current state and are updated in place with the
 * accepted proposal. */
typedef struct ut_hmc_buffers {
    float* position;            /* P x C in/out                                  */
    float* gradient;            /* P x C in/out                                  */
    float* logjoint;            /* C in/out                                      */
    const float* inverse_mass;  /* P   shared diagonal inverse mass              */
    const float* step;          /* C   per-chain step size                       */
    float* accept_prob;         /* C out                                         */
    float* energy;              /* C out: Hamiltonian of the retained state      */
    float* energy_error;        /* C out: H(proposal) - H(current), +Inf invalid */
    uint8_t* accepted;          /* C out                                         */
    uint8_t* divergent;         /* C out                                         */
    float* proposal;            /* P x C out (optional, NULL): proposal position */
    float* endpoint_momentum;   /* P x C out (optional, NULL): negated end momentum */
} ut_hmc_buffers;

/* One batched HMC iteration: Philox momentum (stream 0, draw = parameter),
 * H0, leapfrog trajectory of num_leapfrog_steps steps, H1, and the
 * Metropolis accept with a Philox uniform (stream 4, draw 0), applied on
 * device.  reference: the per-iteration body of _run_device_batched_hmc
 * (src/device/hmc_kernels.jl:517-590), leapfrog as
 * _device_leapfrog_integrate_perchain! (:255-287). */
int32_t ut_hmc_iteration(ut_workspace* ws, const ut_hmc_buffers* buf, int32_t num_leapfrog_steps,
                         uint32_t iteration_coord, float divergence_threshold, void* stream);

/* One ChEES-HMC iteration: ut_hmc_iteration with this iteration's jittered
 * step count, keeping the proposal position and the negated endpoint momentum
 * on the device for ut_chees_reduce; both optional outputs of `buf` are
 * required.  reference: the per-iteration device body of
 * _run_device_batched_chees (src/device/chees_kernels.jl:375-474). */
int32_t ut_chees_iteration(ut_workspace* ws, const ut_hmc_buffers* buf, int32_t num_leapfrog_steps,
                           uint32_t iteration_coord, float divergence_threshold, void* stream);

/* One-step leapfrog probe used by the reasonable-step-size search: from the
 * current state, with momentum drawn at `iteration_coord`, integrate one step
 * of size trial_step[c] and write log_accept_ratio[c] = H0 - H1 (-Inf when
 * invalid).  The state is left unchanged.  reference:
 * _batched_reasonable_log_accept_ratio! (src/inference/nuts/adaptation.jl:389-425). */
int32_t ut_leapfrog_probe(ut_workspace* ws, const float* d_position, const float* d_gradient,
                          const float* d_logjoint, const float* d_inverse_mass, const float* d_trial_step,
                          uint32_t iteration_coord, float* d_log_accept_ratio, void* stream);

/* Per-iteration buffers of one persistent NUTS iteration. */
typedef struct ut_nuts_buffers {
    float* position;            /* P x C in/out: replaced by the proposal when moved */
    float* gradient;            /* P x C in/out                                  */
    float* logjoint;            /* C in/out                                      */
    const float* inverse_mass;  /* P                                             */
    const float* step;          /* C                                             */
    float* accept_prob;         /* C out  (reference out_real[1, :])             */
    float* energy;              /* C out  (out_real[2, :], proposal energy)      */
    float* energy_error;        /* C out  (out_real[3, :])                       */
    int32_t* tree_depth;        /* C out  (out_int[1, :])                        */
    int32_t* integration_steps; /* C out  (out_int[2, :])                        */
    uint8_t* divergent;         /* C out                                         */
    uint8_t* moved;             /* C out                                         */
} ut_nuts_buffers;

/* One persistent multinomial-NUTS iteration for every chain in ONE launch.
 * reference: _device_persistent_nuts_proposals! (src/device/persistent_nuts.jl:678-761)
 * running _persist_nuts_chain! (:226-491); Philox streams 0-3 as at :70-73. */
int32_t ut_persistent_nuts_iteration(ut_workspace* ws, const ut_nuts_buffers* buf,
                                     int32_t max_tree_depth, float divergence_threshold,
                                     uint32_t iteration_coord, void* stream);

/* One lockstep ("masked") NUTS iteration for any workspace, including those
 * whose gradient is a batched all-chains kernel (the large GLM): every chain's
 * tree is advanced one leaf per step between batched gradient evaluations, with
 * the tree decisions and Philox draws of ut_persistent_nuts_iteration (so the
 * two give the same trees where both apply).  Synchronises `stream` every 16
 * leaves to stop once every tree is complete.  P <= 256, max_tree_depth <= 16.
 * reference: the masked lockstep device tree (src/device/nuts_kernels.jl:61-600). */
int32_t ut_lockstep_nuts_iteration(ut_workspace* ws, const ut_nuts_buffers* buf, int32_t max_tree_depth,
                                   float divergence_threshold, uint32_t iteration_coord, void* stream);

/* Per-iteration buffers of MEADS (device pointers). */
typedef struct ut_meads_buffers {
    float* position;            /* P x C in/out                                   */
    float* gradient;            /* P x C in/out                                   */
    float* logjoint;            /* C in/out                                       */
    float* momentum;            /* P x C in/out: persistent whitened momentum     */
    float* slice;               /* C in/out: persistent slice variable in [-1, 1) */
    float* accept_prob;         /* C out (1 for the skipped fold)                 */
    float* energy;              /* C out: -logjoint + |momentum|^2 / 2            */
    float* energy_error;        /* C out (0 for the skipped fold)                 */
    uint8_t* accepted;          /* C out                                          */
    uint8_t* divergent;         /* C out                                          */
    int32_t* integration_steps; /* C out: 1, or 0 for the skipped fold            */
    float* fold_parameters;     /* optional K x 4 out: step, alpha, delta, 0      */
} ut_meads_buffers;

/* Initial MEADS state: momentum ~ N(0, I) from Philox stream 0 and slice
 * u = 2 U - 1 from stream 4, at (chain, iteration_coord).
 * reference: batched_meads (src/inference/api_batched_meads.jl:285-296). */
int32_t ut_meads_init(ut_workspace* ws, const ut_meads_buffers* buf, uint32_t iteration_coord, void* stream);

/* One MEADS iteration for every chain: per-fold ensemble statistics of the
 * neighbour fold (mean, std, trace-ratio eigenvalue estimates of the whitened
 * states and gradients) -> step size, damping, slice drift; partial momentum
 * refresh (Philox stream 0), one leapfrog step with inverse mass std^2, the
 * persistent-slice accept; the fold (iteration - 1) mod num_folds is left
 * unchanged.  iteration >= 1; num_chains >= 2 * num_folds; P <= 544.
 * reference: batched_meads (src/inference/api_batched_meads.jl:170-547),
 * _meads_fold_parameters! (:89-153), _meads_max_eig (:48-78); the reference
 * runs it on the host only. */
int32_t ut_meads_iteration(ut_workspace* ws, const ut_meads_buffers* buf, int32_t num_folds, int32_t iteration,
                           float divergence_threshold, uint32_t iteration_coord, void* stream);

/* One mean-field ADVI step over the workspace's batch of M particles
 * (batch_size = M): draws eps[j, p] from the Philox stream at coordinate
 * (particle j, iteration_coord, stream 5, parameter p), writes the particles
 * location + scale * eps to d_particles (M x P), their logjoints to d_values (M)
 * and gradients to d_gradients (M x P), and reduces
 *   d_location_gradient[p] = mean_j grad[j, p],
 *   d_scale_gradient[p]    = mean_j grad[j, p] * scale[p] * eps[j, p].
 * Device pointers; queued on `stream`.  reference: the device ADVI inner loop
 * _run_device_batched_advi (src/device/advi_kernels.jl:45-209) with its
 * reduction _device_advi_reduce! (:15-38); the reference draws eps on the host. */
int32_t ut_advi_step(ut_workspace* ws, const float* d_location, const float* d_scale, uint32_t iteration_coord,
                     float* d_particles, float* d_values, float* d_gradients, float* d_location_gradient,
                     float* d_scale_gradient, void* stream);

/* ChEES cross-chain trajectory statistics, reduced on device.
 * reference: _chees_trajectory_update! (src/inference/api_batched_chees.jl:158-228),
 * device passes _device_chees_proposal_mean! / _device_chees_endpoint_terms!
 * (src/device/chees_kernels.jl:67-106).  Writes the two host doubles
 * out[0] = gradient_numerator, out[1] = acceptance_denominator and synchronises. */
int32_t ut_chees_reduce(ut_workspace* ws, const float* d_initials, const float* d_proposals,
                        const float* d_endpoint_momentum, const float* d_accept_prob,
                        const uint8_t* d_divergent, const float* d_inverse_mass,
                        double* out, void* stream);

/* ---- warmup adaptation on device ------------------------------------------
 * Pooled running-variance update over the C chains' positions, chain after
 * chain in index order (Welford with the early-window clip), for the
 * windowed diagonal mass adaptation.  reference: _update_running_variance!
 * (src/inference/nuts/adaptation.jl:170-209) with _running_variance_sample!
 * (:83-101) and the clip constants of src/inference/data_types.jl:189-193.
 * d_state: double[2P + 3] = mean(P), m2(P), count, weight_sum,
 * weight_square_sum (updated in place); d_weights: C doubles in [0, 1]
 * (a zero weight skips the chain). */
int32_t ut_running_variance_update(const float* d_positions, const double* d_weights, int32_t num_params,
                                   int32_t num_chains, double* d_state, int32_t window_length, void* stream);

/* One warmup iteration's adaptation on the device, so warmup copies nothing to
 * the host between mass-window ends.  reference: the per-iteration
 * warmup_update! of src/inference/warmup.jl:262-326 / 371-470: the running-
 * variance weights of src/inference/nuts/adaptation.jl:225-260 into d_weights
 * (C doubles; NULL skips them), the window progress taken from
 * d_variance_state (the ut_running_variance_update state, its count at
 * [2P]) and window_length; and with adapt_step, one dual-averaging update
 * (adaptation.jl:1-28) of d_dual -- per chain (per_chain = 1, C x 5 doubles)
 * with each chain's statistic (0 when divergent), or shared (5 doubles) with
 * the mean statistic over the chains (hmc_support.jl:635-652) -- writing the
 * new step sizes to d_step (C floats).  Dual-averaging state: mu, log step,
 * log step average, hbar, iteration. */
int32_t ut_warmup_adapt(const float* d_accept_prob, const uint8_t* d_accepted, const uint8_t* d_divergent,
                        int32_t num_chains, int32_t num_params, const double* d_variance_state,
                        int32_t window_length, double* d_weights, double* d_dual, int32_t per_chain,
                        int32_t adapt_step, double target_accept, float* d_step, void* stream);
/* The warmup's final step sizes exp(log step average) into d_step (C floats). */
int32_t ut_dual_averaging_final(const double* d_dual, int32_t num_chains, int32_t per_chain, float* d_step,
                                void* stream);

/* ---- allocation-free GLM logjoint + gradient ------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they need a gradient (a host whose device memory all comes from
 * its own pool or a fixed budget, or a latency-critical loop that cannot take
 * the synchronisation cudaMalloc / cudaFree may imply): the Bernoulli-logit GLM
 * logjoint and gradient of C chains with every buffer supplied by the caller
 * on the device and no device memory allocated.
 *   d_design   : N x P row-major design matrix (a leading column of ones when
 *                has_intercept = 1, then the covariates)
 *   d_y        : N outcomes in {0, 1}
 *   d_params   : C x P chain-major parameters;  d_totals: C;  d_gradients: C x P
 * Scratch memory is a fixed 16 MiB device array owned by the library (held by
 * every GPU that uses it until exit): C * (P + 1) may be at most 4,194,304,
 * and 1 <= N <= UT_MAX_OBS; other sizes are rejected with UT_ERR_ARGUMENT.
 * The first call on a device performs a one-time set-up for that device, and
 * with CUDA's lazy module loading that first call is also when the 16 MiB and
 * the module's code are committed on the device: a host that reserves its
 * whole memory budget at start-up should make one call per device first (and
 * before any stream capture).  All calls share the array, so calls that
 * overlap on the GPU race: serialise them.  Returns once the work is queued
 * on `stream`. */
int32_t ut_glm_logjoint_gradient_noalloc(const float* d_design, const float* d_y, int64_t num_obs,
                                         int32_t num_params, int32_t has_intercept, double intercept_mu,
                                         double intercept_sigma, double coef_mu, double coef_sigma,
                                         const float* d_params, int32_t num_chains, float* d_totals,
                                         float* d_gradients, void* stream);

/* ---- learned gradient surrogate ------------------------------------------ */
/* No counterpart in the reference.  An MLP  P -> 256 -> 256 -> P  with SiLU
 * hidden layers maps an unconstrained position to an approximation of the
 * logjoint gradient.  Weights are FP32 (updated by Adam); the matmuls run in
 * BF16 with FP32 accumulation.  Inputs are normalised per coordinate as
 * (theta - in_mean) / in_scale and outputs de-normalised as
 * y * out_scale + out_mean.  It is trained on (theta, gradient) pairs that an
 * exact sampler produced (typically its warmup) and then drives leapfrog
 * trajectories whose Metropolis accept uses the exact logjoint, so the target
 * distribution stays exact.  1 <= P <= 128.
 *
 * Weight layout (one flat FP32 array; Pp = P rounded up to 16; entries at
 * row or column index >= P are zero and stay zero):
 *   W1 [256][Pp], b1 [256], W2 [256][256], b2 [256], W3 [Pp][256], b3 [Pp]. */
typedef struct ut_surrogate ut_surrogate;

/* Allocates the weights on the current device, initialised as
 * U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from Philox (key = (seed, layer)), zero
 * biases, identity normalisation. */
int32_t ut_surrogate_create(int32_t num_params, uint32_t seed, ut_surrogate** out);
int32_t ut_surrogate_destroy(ut_surrogate* s);
/* Length of the flat weight array. */
int32_t ut_surrogate_num_weights(const ut_surrogate* s, int64_t* out);
/* Host copies of the FP32 weights.  set_weights also resets the Adam state. */
int32_t ut_surrogate_get_weights(const ut_surrogate* s, float* out, int64_t n);
int32_t ut_surrogate_set_weights(ut_surrogate* s, const float* in, int64_t n);
/* Normalisation as 4*P host floats: in_mean, in_scale, out_mean, out_scale. */
int32_t ut_surrogate_get_normalization(const ut_surrogate* s, float* out);
int32_t ut_surrogate_set_normalization(ut_surrogate* s, const float* in);
/* Sets the normalisation to the per-coordinate means and standard deviations
 * of num_pairs device pairs (d_theta, d_gradient: num_pairs x P each). */
int32_t ut_surrogate_fit_normalization(ut_surrogate* s, const float* d_theta, const float* d_gradient,
                                       int64_t num_pairs, void* stream);
/* num_steps Adam steps (beta1 0.9, beta2 0.999, eps 1e-8) on the mean squared
 * error between the normalised network output and the normalised gradient,
 * loss = sum over batch rows and coordinates of (y - t)^2 / batch.  The
 * learning rate goes geometrically from learning_rate to final_learning_rate.
 * Step k uses the pair rows d_batch_index[k*batch .. k*batch+batch) when
 * d_batch_index is given (indices outside [0, num_pairs) are skipped and
 * reported by ut_surrogate_check), else rows drawn uniformly with
 * replacement from Philox (key = (seed, Adam step count)).  d_losses
 * (optional, num_steps floats) receives each step's loss.  1 <= batch <= 65536. */
int32_t ut_surrogate_train(ut_surrogate* s, const float* d_theta, const float* d_gradient, int64_t num_pairs,
                           const int32_t* d_batch_index, int32_t batch, int32_t num_steps, float learning_rate,
                           float final_learning_rate, uint32_t seed, float* d_losses, void* stream);
/* The loss of one batch and its gradient with respect to the weights (flat
 * layout above), without updating anything. */
int32_t ut_surrogate_loss_gradient(ut_surrogate* s, const float* d_theta, const float* d_gradient, int64_t num_pairs,
                                   const int32_t* d_batch_index, int32_t batch, float* d_weight_gradient,
                                   float* d_loss, void* stream);
/* Surrogate gradient at n positions: d_out (n x P) = network(d_theta). */
int32_t ut_surrogate_gradient(const ut_surrogate* s, const float* d_theta, int64_t n, float* d_out, void* stream);
/* Synchronises `stream` and reports batch indices that were out of range. */
int32_t ut_surrogate_check(ut_surrogate* s, void* stream);

/* One batched HMC iteration whose leapfrog kicks all use the surrogate
 * gradient (at the start, at every intermediate point and at the end), with
 * the Metropolis accept on the exact logjoint of the workspace's model: the
 * leapfrog map of any position-only force field is volume-preserving and
 * reversible, so the chain keeps the exact target.  Same momentum and accept
 * Philox streams and the same buffers as ut_hmc_iteration, except that
 * buf->gradient is neither read nor written (recompute it with
 * ut_logjoint_gradient_device before an exact iteration).  Per iteration: L+1
 * surrogate evaluations and one logjoint-only evaluation of the model. */
int32_t ut_surrogate_hmc_iteration(ut_workspace* ws, const ut_surrogate* s, const ut_hmc_buffers* buf,
                                   int32_t num_leapfrog_steps, uint32_t iteration_coord,
                                   float divergence_threshold, void* stream);

/* ---- uneven batching: many hierarchical models in one batched launch ------ */
/* No counterpart in the reference.  A batch of independent non-centred
 * hierarchical normal models (UT_FAMILY_HIER_NORMAL_NONCENTERED), each with
 * its own groups, group sizes, priors and chain count, sampled together by
 * batched persistent NUTS: one launch per parameter-slot class per iteration
 * (the classes run concurrently), per-model step-size and diagonal-mass
 * adaptation on the device, and the iterations replayed from a captured CUDA
 * graph.  State layout: model m's chains own the C_m x P_m chain-major block
 * starting at state_offsets[m] of the position / gradient / draw arrays, its
 * per-chain entries start at chain_offsets[m], its inverse mass at
 * param_offsets[m]. */
typedef struct ut_multi ut_multi;

/* Device pointers into a batch's state (owned by the batch). */
typedef struct ut_multi_view {
    float* position;            /* state_floats                                  */
    float* gradient;            /* state_floats                                  */
    float* logjoint;            /* total_chains                                  */
    float* step;                /* total_chains                                  */
    float* inverse_mass;        /* param_floats                                  */
    float* accept_prob;         /* total_chains, last iteration                  */
    int32_t* tree_depth;        /* total_chains, last iteration                  */
    int32_t* integration_steps; /* total_chains, last iteration                  */
    uint8_t* divergent;         /* total_chains, last iteration                  */
    float* draws;               /* draws_capacity x state_floats                 */
    float* draw_accept;         /* draws_capacity x total_chains                 */
    int32_t* draw_tree_depth;   /* draws_capacity x total_chains                 */
    uint8_t* draw_divergent;    /* draws_capacity x total_chains                 */
    int32_t* iteration;         /* iterations run since ut_multi_begin           */
    int64_t state_floats;
    int64_t total_chains;
    int64_t param_floats;
    int32_t draws_capacity;
} ut_multi_view;

/* plans[m]: the model's kernel description (num_params = num_groups + 2 <=
 * 544).  observed: the models' staged blocks one after another, model m's at
 * observed_offsets[m] (num_models + 1 entries), each num_obs y values group
 * after group then num_groups sigma values.  trip_counts / loop_starts: every
 * model's num_groups entries one model after another, loop_starts relative to
 * the model's own block.  chains[m]: chain count of model m. */
int32_t ut_multi_create(int32_t num_models, const ut_plan_desc* plans, const float* observed,
                        const int64_t* observed_offsets, const int32_t* trip_counts, const int32_t* loop_starts,
                        const int32_t* chains, int32_t max_tree_depth, ut_multi** out);
int32_t ut_multi_destroy(ut_multi* mm);
/* Offsets of every model (num_models + 1 entries each; any may be NULL). */
int32_t ut_multi_layout(const ut_multi* mm, int64_t* state_offsets, int64_t* chain_offsets, int64_t* param_offsets);
/* Per slot-count class (8 entries each; any may be NULL): slots per lane K
 * (models with P <= 32 K), models, chains, chains per CTA and the staging
 * limit in bytes (a model's data is staged in shared memory when it fits). */
int32_t ut_multi_class_info(const ut_multi* mm, int32_t* slot_counts, int32_t* num_models, int64_t* num_chains,
                            int32_t* chains_per_block, int32_t* stage_limit_bytes);
/* Sets one class's launch configuration: 1..4 chains per CTA, staging limit 0..204800 bytes. */
int32_t ut_multi_configure(ut_multi* mm, int32_t klass, int32_t chains_per_block, int32_t stage_limit_bytes);
/* Copies state_floats device positions in and evaluates logjoint + gradient there. */
int32_t ut_multi_set_positions(ut_multi* mm, const float* d_positions, void* stream);
/* Starts a run: iteration counter 0, unit inverse masses, every step size
 * initial_step, warmup_actions[i] for warmup iteration i (bit 0: add the
 * model's non-divergent positions to its Welford window, bit 1: the window
 * ends and sets the model's inverse mass, bit 2: final step sizes), and room
 * for draws_capacity sampling draws.  Warmup adapts as the reference's default
 * batched NUTS: every chain searches a reasonable step size at the first
 * iteration and after every window (one momentum draw at Philox coordinate
 * seed + 2^31 + iteration), then dual-averages it towards target_accept on its
 * own accept statistic (0 when divergent).  The Philox iteration coordinate of
 * iteration i is seed + i. */
int32_t ut_multi_begin(ut_multi* mm, int32_t num_warmup, int32_t num_samples, uint32_t seed, float target_accept,
                       float initial_step, float divergence_threshold, const uint8_t* warmup_actions,
                       int32_t draws_capacity);
/* Runs the next num_iterations iterations (warmup first, then sampling, whose
 * positions are recorded as draws), from a captured CUDA graph when
 * use_graph != 0.  Ordered after prior work on `stream`; later work on
 * `stream` waits for it. */
int32_t ut_multi_run(ut_multi* mm, int32_t num_iterations, int32_t use_graph, void* stream);
/* Autotuner: for every class, times each (chains per CTA in {1, 2, 4}) x
 * (staging off / on) candidate on the next iteration from the current state
 * (restored after every trial; results do not depend on the choice) and
 * keeps the fastest.  timings_ms (optional, 8 x 6 floats): class k's
 * candidate (w, s) at [6 k + 2 w + s], -1 for empty classes.  Synchronises. */
int32_t ut_multi_autotune(ut_multi* mm, int32_t trials, float* timings_ms, void* stream);
/* Max split R-hat over each model's parameters from its first num_draws
 * recorded draws (d_out: num_models floats). */
int32_t ut_multi_split_rhat(ut_multi* mm, int32_t num_draws, float* d_out, void* stream);
/* Per-model stopping: stopped[m] != 0 (host array of num_models bytes) makes
 * the following iterations skip model m's chains -- their positions, steps and
 * adaptation state stay as they are -- so the batch's work goes to the models
 * still running.  The draw buffer keeps recording every model; a stopped
 * model's later draws repeat its last state and are not its samples.  Reset
 * to all-running by ut_multi_begin.  No counterpart in the reference. */
int32_t ut_multi_set_stopped(ut_multi* mm, const uint8_t* stopped, void* stream);
int32_t ut_multi_buffers(const ut_multi* mm, ut_multi_view* view);

#ifdef __cplusplus
}
#endif

#endif /* UT_B200_H */
