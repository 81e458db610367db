// ut_program.cuh -- the composable kernel description (step program): a host
// compiler that checks a program and folds its deterministic bindings into the
// expressions that read them, and a warp-per-chain device interpreter that
// returns the logjoint and its full gradient in one pass.
//
// The reference walks its DeviceExecutionPlan step tuple once per chain thread
// for the value (src/device/logjoint_kernel.jl:724) and once per (parameter,
// chain) thread with scalar forward-mode duals for the gradient
// (src/device/gradient_kernel.jl:1124).  Here one warp owns a chain: the 32
// lanes share the top-level steps, split the iterations of every top-level loop
// among themselves, and the gradient is reverse mode -- each choice term's
// partial derivatives flow back through its argument expressions into
// per-lane adjoints of the latent bindings, which are summed over the lanes
// in a fixed order at the end (deterministic, no atomics).  A latent value's
// gradient is then the adjoint of its binding times the transform's
// derivative plus the log-Jacobian's derivative.
//
// Compiled form: deterministic steps vanish (their expressions are copied into
// every reader), an observed binding becomes an observation leaf, a loop
// iterator becomes an iterator leaf, so the only slots left on the device are
// latent values.  Every argument expression is a contiguous run of nodes in
// evaluation order ending at its root.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "ut_common.cuh"

namespace ut {

constexpr int kProgMaxExprNodes = 48;   // nodes of one argument expression after inlining
constexpr int kProgMaxDepth = 4;        // loop nesting
constexpr int kProgMaxSlots = 64;       // latent bindings on the device
constexpr int kProgMaxParams = 256;
constexpr int kProgMaxSteps = 1024;
constexpr int kProgExprIter = 100;      // compiled-only leaf: iterator of the loop at depth a

struct PStep {
    int kind, dist, tr, vs, off, slot, count, width, body, istart, depth;
    int afirst[4], aroot[4];  // node range of each argument, aroot < 0: none
};

struct PNode {
    int op, a, b, dep;  // dep: the value depends on a latent slot (its adjoint matters)
    float v;
};

struct ProgModel {
    const PStep* steps;
    const PNode* nodes;
    const float* obs;
    int nsteps, nnodes, nslots, nobs, P;
    int pp;  // parameters rounded up to 32 (per-warp scratch layout)
};

// ---------------------------------------------------------------------------
// host compiler
// ---------------------------------------------------------------------------
__host__ __device__ inline int prog_dist_nargs(int d) {
    switch (d) {
        case UT_DIST_EXPONENTIAL: case UT_DIST_HALFNORMAL: case UT_DIST_HALFCAUCHY: case UT_DIST_RAYLEIGH:
        case UT_DIST_BERNOULLI: case UT_DIST_BERNOULLI_LOGIT: case UT_DIST_POISSON: case UT_DIST_GEOMETRIC:
            return 1;
        case UT_DIST_STUDENTT:
            return 3;
        default:
            return (d >= UT_DIST_NORMAL && d <= UT_DIST_BINOMIAL) ? 2 : -1;
    }
}

__host__ __device__ inline bool prog_dist_discrete(int d) { return d >= UT_DIST_BERNOULLI && d <= UT_DIST_BINOMIAL; }

inline int prog_op_arity(int op) {
    switch (op) {
        case UT_EXPR_LITERAL: case UT_EXPR_SLOT: case UT_EXPR_OBS: return 0;
        case UT_EXPR_ADD: case UT_EXPR_SUB: case UT_EXPR_MUL: case UT_EXPR_DIV: case UT_EXPR_POW:
        case UT_EXPR_MIN: case UT_EXPR_MAX:
            return 2;
        default:
            return (op >= UT_EXPR_NEG && op <= UT_EXPR_EXPM1) ? 1 : -1;
    }
}

struct ProgCompiled {
    std::vector<PStep> steps;
    std::vector<PNode> nodes;
    int nslots = 0;
    int P = 0;
};

class ProgCompiler {
  public:
    ProgCompiler(const ut_program_step* s, int ns, const ut_expr_node* n, int nn, int nslots, int P, int64_t rows)
        : in_(s), ns_(ns), nd_(n), nn_(nn), nslots_(nslots), P_(P), rows_(rows) {}

    // Empty string on success; else one issue per line.
    std::string run(ProgCompiled* out) {
        if (!in_ || ns_ < 1) add("a program needs at least one step");
        if (ns_ > kProgMaxSteps) add("a program has at most 1024 steps");
        if (nn_ < 0 || (nn_ > 0 && !nd_)) add("null or negative expression node list");
        if (nslots_ < 0 || nslots_ > 4096) add("num_slots must be in 0..4096");
        if (P_ < 1 || P_ > kProgMaxParams) add("num_params must be in 1..256");
        if (rows_ < 0 || rows_ > UT_MAX_OBS) add("observed_rows must be in 0..2^30");
        if (!issues_.empty()) return issues_;
        for (int i = 0; i < nn_; ++i) check_node(i);
        if (!issues_.empty()) return issues_;
        env_.assign(nslots_, Def());
        covered_.assign(P_, 0);
        int pc = 0;
        compile_block(pc, ns_, 0, rows_);
        for (const auto& gr : glm_rows_)
            for (int r = gr.first; r < gr.first + gr.second; ++r)
                if (covered_[r] == 0) {
                    add("GLM coefficient row " + std::to_string(r) + " is not a latent value");
                    break;
                }
        for (int r = 0; r < P_; ++r)
            if (covered_[r] != 1) {
                add("parameter row " + std::to_string(r) + (covered_[r] ? " is read by more than one latent step"
                                                                         : " is read by no latent step"));
                break;
            }
        if (devslots_ > kProgMaxSlots) add("a program has at most 64 latent scalar values");
        if (!issues_.empty()) return issues_;
        out->steps = steps_;
        out->nodes = nodes_;
        out->nslots = devslots_;
        out->P = P_;
        return issues_;
    }

  private:
    struct Def {
        int state = 0;          // 0 unwritten, 1 defined
        int depth = 0;          // loop depth of its definition
        std::vector<PNode> t;   // self-contained compiled tree, root last
    };

    const ut_program_step* in_;
    int ns_;
    const ut_expr_node* nd_;
    int nn_, nslots_, P_;
    int64_t rows_;
    std::string issues_;
    std::vector<Def> env_;
    std::vector<int> covered_;
    std::vector<PStep> steps_;
    std::vector<PNode> nodes_;
    std::vector<int64_t> blocks_;  // rows of the observation block at each loop depth
    std::vector<std::pair<int, int>> glm_rows_;  // (first row, count) read by GLM steps
    int devslots_ = 0;

    void add(const std::string& m) {
        if (issues_.size() > 2000) return;
        issues_ += (issues_.empty() ? "" : "\n") + m;
    }

    void check_node(int i) {
        const ut_expr_node& e = nd_[i];
        const int ar = prog_op_arity(e.op);
        const std::string at = "expression node " + std::to_string(i);
        if (ar < 0) { add(at + ": unknown operation " + std::to_string(e.op)); return; }
        if (ar >= 1 && (e.a < 0 || e.a >= i)) add(at + ": operand a must be an earlier node");
        if (ar == 2 && (e.b < 0 || e.b >= i)) add(at + ": operand b must be an earlier node");
        if (e.op == UT_EXPR_SLOT && (e.a < 0 || e.a >= nslots_)) add(at + ": slot out of range");
        if (e.op == UT_EXPR_OBS && (e.a < 0 || e.b < 0 || e.b > kProgMaxDepth)) add(at + ": bad observation row");
        if (e.op == UT_EXPR_LITERAL && !std::isfinite(e.value)) add(at + ": non-finite literal");
    }

    // Copies the expression rooted at input node r into `t` (post order),
    // substituting slot definitions; returns false (with an issue) on error.
    bool emit(int r, int depth, std::vector<PNode>& t, const std::string& where) {
        if (r < 0 || r >= nn_) { add(where + ": expression root out of range"); return false; }
        const ut_expr_node& e = nd_[r];
        const int ar = prog_op_arity(e.op);
        if (e.op == UT_EXPR_SLOT) {
            const Def& d = env_[e.a];
            if (d.state == 0) {
                add(where + ": slot " + std::to_string(e.a) + " is read before it is written");
                return false;
            }
            if (d.depth > depth) {
                add(where + ": slot " + std::to_string(e.a) + " is bound inside a loop and read outside it");
                return false;
            }
            const int base = (int)t.size();
            for (PNode n : d.t) {
                if (prog_op_arity(n.op) >= 1) n.a += base;
                if (prog_op_arity(n.op) == 2) n.b += base;
                t.push_back(n);
            }
        } else if (e.op == UT_EXPR_OBS) {
            if (e.b > depth) { add(where + ": observation leaf of a deeper loop"); return false; }
            if ((int64_t)e.a >= blocks_[e.b]) { add(where + ": observation leaf outside its block"); return false; }
            t.push_back(PNode{UT_EXPR_OBS, e.a, e.b, 0, 0.0f});
        } else if (e.op == UT_EXPR_LITERAL) {
            t.push_back(PNode{UT_EXPR_LITERAL, 0, 0, 0, (float)e.value});
        } else {
            if (!emit(e.a, depth, t, where)) return false;
            const int ia = (int)t.size() - 1;
            int ib = -1;
            if (ar == 2) {
                if (!emit(e.b, depth, t, where)) return false;
                ib = (int)t.size() - 1;
            }
            PNode n{e.op, ia, ib < 0 ? 0 : ib, t[ia].dep | (ib >= 0 ? t[ib].dep : 0), 0.0f};
            t.push_back(n);
        }
        if ((int)t.size() > kProgMaxExprNodes) {
            add(where + ": an argument expression has more than 48 nodes after its bindings are inlined");
            return false;
        }
        return true;
    }

    // Appends an argument's compiled nodes to the program's node list.
    bool arg(int r, int depth, PStep& ps, int j, const std::string& where) {
        std::vector<PNode> t;
        if (!emit(r, depth, t, where)) return false;
        const int base = (int)nodes_.size();
        for (PNode n : t) {
            if (prog_op_arity(n.op) >= 1) n.a += base;
            if (prog_op_arity(n.op) == 2) n.b += base;
            nodes_.push_back(n);
        }
        ps.afirst[j] = base;
        ps.aroot[j] = (int)nodes_.size() - 1;
        return true;
    }

    void bind(int slot, int depth, std::vector<PNode> t, const std::string& where) {
        if (slot < 0) return;
        if (slot >= nslots_) { add(where + ": binding slot out of range"); return; }
        env_[slot].state = 1;
        env_[slot].depth = depth;
        env_[slot].t = std::move(t);
    }

    bool claim_rows(int vs, int n, const std::string& where) {
        if (vs < 0 || n < 1 || (int64_t)vs + n > P_) { add(where + ": parameter rows out of range"); return false; }
        for (int r = vs; r < vs + n; ++r) covered_[r] += 1;
        return true;
    }

    // Compiles steps [pc, end) at loop depth `depth` whose block holds `block` rows.
    void compile_block(int& pc, int end, int depth, int64_t block) {
        blocks_.resize(depth + 1);
        blocks_[depth] = block;
        while (pc < end && issues_.size() < 2000) {
            const ut_program_step& s = in_[pc];
            const std::string where = "step " + std::to_string(pc);
            PStep ps{};
            ps.kind = s.kind;
            ps.depth = depth;
            for (int j = 0; j < 4; ++j) ps.afirst[j] = ps.aroot[j] = -1;
            if (s.kind == UT_STEP_DETERMINISTIC) {
                std::vector<PNode> t;
                if (s.binding_slot < 0) add(where + ": a deterministic step needs a binding slot");
                else if (emit(s.arg[0], depth, t, where)) bind(s.binding_slot, depth, std::move(t), where);
                ++pc;
                continue;
            }
            if (s.kind == UT_STEP_CHOICE) {
                const int na = prog_dist_nargs(s.dist);
                if (na < 0) { add(where + ": unknown distribution " + std::to_string(s.dist)); ++pc; continue; }
                ps.dist = s.dist;
                bool ok = true;
                for (int j = 0; j < na && ok; ++j) ok = arg(s.arg[j], depth, ps, j, where);
                if (!ok) { ++pc; continue; }
                if (s.value_source >= 0) {
                    if (depth > 0) add(where + ": a latent choice inside a loop is not supported");
                    if (prog_dist_discrete(s.dist)) add(where + ": a discrete distribution's value must be observed");
                    if (s.transform < UT_TRANSFORM_IDENTITY || s.transform > UT_TRANSFORM_LOGIT)
                        add(where + ": unknown transform");
                    if (!claim_rows(s.value_source, 1, where)) { ++pc; continue; }
                    ps.vs = s.value_source;
                    ps.tr = s.transform;
                    ps.slot = devslots_++;
                    std::vector<PNode> t{PNode{UT_EXPR_SLOT, ps.slot, 0, 1, 0.0f}};
                    bind(s.binding_slot, depth, std::move(t), where);
                } else {
                    if (s.obs_offset < 0 || s.obs_offset >= block) { add(where + ": observed row outside its block"); ++pc; continue; }
                    ps.vs = -1;
                    ps.off = s.obs_offset;
                    std::vector<PNode> t{PNode{UT_EXPR_OBS, s.obs_offset, depth, 0, 0.0f}};
                    bind(s.binding_slot, depth, std::move(t), where);
                }
                steps_.push_back(ps);
                ++pc;
                continue;
            }
            if (s.kind == UT_STEP_IID_NORMAL) {
                if (depth > 0) add(where + ": an iid normal vector prior inside a loop is not supported");
                if (s.binding_slot >= 0) add(where + ": a vector value has no scalar binding (binding_slot must be -1)");
                bool ok = arg(s.arg[0], depth, ps, 0, where) && arg(s.arg[1], depth, ps, 1, where);
                if (ok && claim_rows(s.value_source, s.count, where)) {
                    ps.vs = s.value_source;
                    ps.count = s.count;
                    steps_.push_back(ps);
                }
                ++pc;
                continue;
            }
            if (s.kind == UT_STEP_GLM_BERNOULLI_LOGIT) {
                if (depth > 0) add(where + ": the fused GLM step is a top-level step");
                if (s.width < 1 || s.count < 0) { add(where + ": GLM needs covariates >= 1 and observations >= 0"); ++pc; continue; }
                if (s.obs_offset < 0 || (int64_t)s.obs_offset + (int64_t)s.count * (s.width + 1) > block)
                    add(where + ": GLM observation rows outside the staged buffer");
                bool ok = true;
                if (s.arg[0] >= 0) ok = arg(s.arg[0], depth, ps, 0, where);
                // the coefficients are read here; a latent step (their prior) owns the rows
                if (s.value_source < 0 || (int64_t)s.value_source + s.width > P_) {
                    add(where + ": GLM coefficient rows out of range");
                    ok = false;
                }
                if (ok) glm_rows_.push_back({s.value_source, s.width});
                if (ok) {
                    ps.vs = s.value_source;
                    ps.count = s.count;
                    ps.width = s.width;
                    ps.off = s.obs_offset;
                    steps_.push_back(ps);
                }
                ++pc;
                continue;
            }
            if (s.kind == UT_STEP_LOOP) {
                if (depth + 1 > kProgMaxDepth) { add(where + ": loops nest at most 4 deep"); ++pc; continue; }
                if (s.count < 0 || s.width < 0 || s.body < 0 || (int64_t)pc + 1 + s.body > end) {
                    add(where + ": loop count, width or body out of range");
                    ++pc;
                    continue;
                }
                if (s.count > 0 && (s.obs_offset < 0 || (int64_t)s.obs_offset + (int64_t)s.count * s.width > block)) {
                    add(where + ": loop blocks outside the enclosing block");
                    ++pc;
                    continue;
                }
                const std::vector<Def> saved = env_;
                if (s.iterator_slot >= 0) {
                    std::vector<PNode> t{PNode{kProgExprIter, depth + 1, 0, 0, 0.0f}};
                    bind(s.iterator_slot, depth + 1, std::move(t), where);
                }
                ps.count = s.count;
                ps.width = s.width;
                ps.off = s.obs_offset;
                ps.istart = s.iterator_start;
                const size_t at = steps_.size();
                steps_.push_back(ps);
                int inner = pc + 1;
                compile_block(inner, pc + 1 + s.body, depth + 1, s.width);
                steps_[at].body = (int)(steps_.size() - at - 1);
                env_ = saved;  // bindings of the body do not outlive it
                pc = pc + 1 + s.body;
                continue;
            }
            add(where + ": unknown step kind " + std::to_string(s.kind));
            ++pc;
        }
    }
};

// ---------------------------------------------------------------------------
// device math
// ---------------------------------------------------------------------------
// digamma: recurrence psi(x) = psi(x + 1) - 1/x up to x >= 6, then the
// asymptotic series psi(x) ~ ln x - 1/(2x) - sum_k B_2k / (2k x^2k) with the
// Bernoulli numbers B_2 .. B_8 (1/6, -1/30, 1/42, -1/30).
__host__ __device__ __forceinline__ float prog_digamma(float x) {
    float acc = 0.0f;
    for (int i = 0; i < 8 && x < 6.0f; ++i) {
        acc -= 1.0f / x;
        x += 1.0f;
    }
    const float r = 1.0f / x, r2 = r * r;
    const float series = r2 * (1.0f / 12.0f - r2 * (1.0f / 120.0f - r2 * (1.0f / 252.0f - r2 * (1.0f / 240.0f))));
    return acc + logf(x) - 0.5f * r - series;
}

// loggamma(x + 1/2) - loggamma(x), large-x safe (math.jl:80-86, crossover 12 in Float32).
__host__ __device__ __forceinline__ float prog_lgamma_half_ratio(float x) {
    if (x > 12.0f)
        return x * log1pf(1.0f / (2.0f * x)) + 0.5f * logf(x) - 0.5f + (1.0f / (x + 0.5f) - 1.0f / x) / 12.0f;
    return lgammaf(x + 0.5f) - lgammaf(x);
}

constexpr float kProgHalfLog2Pi = 0.9189385332046727f;
constexpr float kProgLogPi = 1.1447298858494002f;
constexpr float kProgLog2 = 0.6931471805599453f;

// Log-density of one choice term (math.jl:88-300) and its partials with
// respect to the arguments (da) and the value (dx), which are only written
// when `grad`.
__host__ __device__ float prog_dist(int dist, const float* a, float x, bool grad, float* da, float& dx) {
    const float ninf = -INFINITY;
    float lp = 0.0f;
    da[0] = da[1] = da[2] = 0.0f;
    dx = 0.0f;
    switch (dist) {
        case UT_DIST_NORMAL: {
            const float z = (x - a[0]) / a[1];
            lp = -logf(a[1]) - kProgHalfLog2Pi - 0.5f * z * z;
            if (grad) { da[0] = z / a[1]; da[1] = (z * z - 1.0f) / a[1]; dx = -z / a[1]; }
        } break;
        case UT_DIST_LOGNORMAL: {
            const float lx = logf(x), z = (lx - a[0]) / a[1];
            lp = x >= FLT_MIN ? -logf(a[1]) - kProgHalfLog2Pi - 0.5f * z * z - lx : ninf;
            if (grad) { da[0] = z / a[1]; da[1] = (z * z - 1.0f) / a[1]; dx = (-z / a[1] - 1.0f) / x; }
        } break;
        case UT_DIST_EXPONENTIAL:
            lp = x >= 0.0f ? logf(a[0]) - a[0] * x : ninf;
            if (grad) { da[0] = 1.0f / a[0] - x; dx = -a[0]; }
            break;
        case UT_DIST_GAMMA: {
            const float lx = logf(x), lr = logf(a[1]);
            lp = x >= FLT_MIN ? a[0] * lr - lgammaf(a[0]) + (a[0] - 1.0f) * lx - a[1] * x : ninf;
            if (grad) { da[0] = lr - prog_digamma(a[0]) + lx; da[1] = a[0] / a[1] - x; dx = (a[0] - 1.0f) / x - a[1]; }
        } break;
        case UT_DIST_LAPLACE: {
            const float d = x - a[0], ad = fabsf(d), sg = d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f);
            lp = -logf(2.0f * a[1]) - ad / a[1];
            if (grad) { da[0] = sg / a[1]; da[1] = -1.0f / a[1] + ad / (a[1] * a[1]); dx = -sg / a[1]; }
        } break;
        case UT_DIST_CAUCHY: {
            const float z = (x - a[0]) / a[1], w = 2.0f * z / (a[1] * (1.0f + z * z));
            lp = -kProgLogPi - logf(a[1]) - log1pf(z * z);
            if (grad) { da[0] = w; da[1] = -1.0f / a[1] + w * z; dx = -w; }
        } break;
        case UT_DIST_HALFNORMAL: {
            const float z = x / a[0];
            lp = x >= 0.0f ? kProgLog2 - logf(a[0]) - kProgHalfLog2Pi - 0.5f * z * z : ninf;
            if (grad) { da[0] = (z * z - 1.0f) / a[0]; dx = -z / a[0]; }
        } break;
        case UT_DIST_HALFCAUCHY: {
            const float z = x / a[0], w = 2.0f * z / (a[0] * (1.0f + z * z));
            lp = x >= 0.0f ? kProgLog2 - kProgLogPi - logf(a[0]) - log1pf(z * z) : ninf;
            if (grad) { da[0] = -1.0f / a[0] + w * z; dx = -w; }
        } break;
        case UT_DIST_LOGISTIC: {
            const float z = (x - a[0]) / a[1], az = fabsf(z);
            lp = -logf(a[1]) - az - 2.0f * log1pf(expf(-az));
            if (grad) {
                const float th = tanhf(0.5f * z);
                da[0] = th / a[1]; da[1] = (-1.0f + z * th) / a[1]; dx = -th / a[1];
            }
        } break;
        case UT_DIST_GUMBEL: {
            const float z = (x - a[0]) / a[1], e = expf(-z);
            lp = -logf(a[1]) - z - e;
            if (grad) { da[0] = (1.0f - e) / a[1]; da[1] = (-1.0f + z * (1.0f - e)) / a[1]; dx = (e - 1.0f) / a[1]; }
        } break;
        case UT_DIST_FRECHET: {
            const float lz = logf(x) - logf(a[1]), w = expf(-a[0] * lz);
            lp = x >= FLT_MIN ? logf(a[0]) - logf(a[1]) - (1.0f + a[0]) * lz - w : ninf;
            if (grad) {
                da[0] = 1.0f / a[0] - lz + lz * w;
                da[1] = a[0] * (1.0f - w) / a[1];
                dx = (-(1.0f + a[0]) + a[0] * w) / x;
            }
        } break;
        case UT_DIST_RAYLEIGH: {
            lp = x >= FLT_MIN ? logf(x) - 2.0f * logf(a[0]) - x * x / (2.0f * a[0] * a[0]) : ninf;
            if (grad) { da[0] = -2.0f / a[0] + x * x / (a[0] * a[0] * a[0]); dx = 1.0f / x - x / (a[0] * a[0]); }
        } break;
        case UT_DIST_INVERSEGAUSSIAN: {
            const float mu = a[0], lam = a[1], d = x - mu;
            lp = x >= FLT_MIN ? 0.5f * logf(lam) - kProgHalfLog2Pi - 1.5f * logf(x) - lam * d * d / (2.0f * mu * mu * x)
                              : ninf;
            if (grad) {
                da[0] = lam * d / (mu * mu * mu);
                da[1] = 0.5f / lam - d * d / (2.0f * mu * mu * x);
                dx = -1.5f / x - lam * (2.0f * d * x - d * d) / (2.0f * mu * mu * x * x);
            }
        } break;
        case UT_DIST_BETA: {
            const float lx = logf(x), l1x = log1pf(-x);
            const float lb = lgammaf(a[0]) + lgammaf(a[1]) - lgammaf(a[0] + a[1]);
            lp = (x > 0.0f && x < 1.0f) ? (a[0] - 1.0f) * lx + (a[1] - 1.0f) * l1x - lb : ninf;
            if (grad) {
                const float ps = prog_digamma(a[0] + a[1]);
                da[0] = lx - prog_digamma(a[0]) + ps;
                da[1] = l1x - prog_digamma(a[1]) + ps;
                dx = (a[0] - 1.0f) / x - (a[1] - 1.0f) / (1.0f - x);
            }
        } break;
        case UT_DIST_STUDENTT: {
            const float nu = a[0], z = (x - a[1]) / a[2], q = z * z / nu;
            lp = prog_lgamma_half_ratio(0.5f * nu) - 0.5f * (logf(nu) + kProgLogPi) - logf(a[2]) -
                 0.5f * (nu + 1.0f) * log1pf(q);
            if (grad) {
                const float w = (nu + 1.0f) * z / (a[2] * (nu + z * z));
                da[0] = 0.5f * (prog_digamma(0.5f * (nu + 1.0f)) - prog_digamma(0.5f * nu)) - 0.5f / nu -
                        0.5f * log1pf(q) + 0.5f * (nu + 1.0f) * z * z / (nu * (nu + z * z));
                da[1] = w;
                da[2] = -1.0f / a[2] + w * z;
                dx = -w;
            }
        } break;
        case UT_DIST_INVERSEGAMMA: {
            const float lx = logf(x);
            lp = x >= FLT_MIN ? a[0] * logf(a[1]) - lgammaf(a[0]) - (a[0] + 1.0f) * lx - a[1] / x : ninf;
            if (grad) {
                da[0] = logf(a[1]) - prog_digamma(a[0]) - lx;
                da[1] = a[0] / a[1] - 1.0f / x;
                dx = -(a[0] + 1.0f) / x + a[1] / (x * x);
            }
        } break;
        case UT_DIST_WEIBULL: {
            const float k = a[0], lam = a[1], ll = logf(x) - logf(lam), t = expf(k * ll);
            if (x >= FLT_MIN) lp = logf(k) + (k - 1.0f) * logf(x) - k * logf(lam) - t;
            else if (x == 0.0f) lp = k < 1.0f ? INFINITY : (k == 1.0f ? -logf(lam) : ninf);
            else lp = ninf;
            if (grad) { da[0] = 1.0f / k + ll - t * ll; da[1] = (-k + k * t) / lam; dx = (k - 1.0f - k * t) / x; }
        } break;
        case UT_DIST_BERNOULLI: {
            const bool one = x > 0.5f, sup = (x == 0.0f) | (x == 1.0f);
            lp = sup ? (one ? logf(a[0]) : log1pf(-a[0])) : ninf;
            if (grad) da[0] = one ? 1.0f / a[0] : -1.0f / (1.0f - a[0]);
        } break;
        case UT_DIST_BERNOULLI_LOGIT: {
            const float eta = a[0], e = expf(-fabsf(eta));
            const float lpe = fmaxf(eta, 0.0f) + log1pf(e);
            const bool sup = (x == 0.0f) | (x == 1.0f);
            lp = sup ? x * eta - lpe : ninf;
            if (grad) da[0] = x - (eta >= 0.0f ? 1.0f / (1.0f + e) : e / (1.0f + e));
        } break;
        case UT_DIST_POISSON: {
            const float k = rintf(x);
            lp = (x >= 0.0f && x == k) ? k * logf(a[0]) - a[0] - lgammaf(k + 1.0f) : ninf;
            if (grad) da[0] = k / a[0] - 1.0f;
        } break;
        case UT_DIST_GEOMETRIC: {
            const float k = rintf(x);
            lp = (x >= 0.0f && x == k) ? logf(a[0]) + (k > 0.0f ? k * log1pf(-a[0]) : 0.0f) : ninf;
            if (grad) da[0] = 1.0f / a[0] - (k > 0.0f ? k / (1.0f - a[0]) : 0.0f);
        } break;
        case UT_DIST_NEGATIVE_BINOMIAL: {
            const float k = rintf(x), r = a[0], p = a[1];
            lp = (x >= 0.0f && x == k) ? lgammaf(k + r) - lgammaf(r) - lgammaf(k + 1.0f) + r * logf(p) +
                                             (k > 0.0f ? k * log1pf(-p) : 0.0f)
                                       : ninf;
            if (grad) {
                da[0] = prog_digamma(k + r) - prog_digamma(r) + logf(p);
                da[1] = r / p - (k > 0.0f ? k / (1.0f - p) : 0.0f);
            }
        } break;
        case UT_DIST_BINOMIAL: {
            const float n = rintf(a[0]), k = rintf(x), p = a[1];
            const bool sup = (x == k) & (a[0] == n) & (k >= 0.0f) & (n >= 0.0f) & (k <= n);
            lp = sup ? lgammaf(n + 1.0f) - lgammaf(k + 1.0f) - lgammaf(n - k + 1.0f) +
                           (k > 0.0f ? k * logf(p) : 0.0f) + (k < n ? (n - k) * log1pf(-p) : 0.0f)
                     : ninf;
            if (grad) da[1] = (k > 0.0f ? k / p : 0.0f) - (k < n ? (n - k) / (1.0f - p) : 0.0f);
        } break;
        default:
            lp = NAN;
    }
    return lp;
}

// Latent transform (math.jl:1144-1159): value, log|J|, d value/du, d log|J|/du.
__host__ __device__ __forceinline__ float prog_transform(int tr, float u, float& lad, float& dxdu, float& dlad) {
    if (tr == UT_TRANSFORM_LOG) {
        const float x = expf(u);
        lad = u; dxdu = x; dlad = 1.0f;
        return x;
    }
    if (tr == UT_TRANSFORM_LOGIT) {
        const float x = 1.0f / (1.0f + expf(-u)), m = fabsf(u);
        lad = -m - 2.0f * log1pf(expf(-m));
        dxdu = x * (1.0f - x);
        dlad = -tanhf(0.5f * u);
        return x;
    }
    lad = 0.0f; dxdu = 1.0f; dlad = 0.0f;
    return u;
}

// Per-lane evaluation context: the block base row and iteration of each loop depth.
struct ProgCtx {
    int base[kProgMaxDepth + 1];
    int iter[kProgMaxDepth + 1];   // iterator value (start + t)
};

__device__ __forceinline__ float prog_unary(int op, float x) {
    switch (op) {
        case UT_EXPR_NEG: return -x;
        case UT_EXPR_EXP: return expf(x);
        case UT_EXPR_LOG: return logf(x);
        case UT_EXPR_LOG1P: return log1pf(x);
        case UT_EXPR_SQRT: return sqrtf(x);
        case UT_EXPR_ABS: return fabsf(x);
        case UT_EXPR_SIN: return sinf(x);
        case UT_EXPR_COS: return cosf(x);
        case UT_EXPR_TAN: return tanf(x);
        case UT_EXPR_TANH: return tanhf(x);
        case UT_EXPR_SINH: return sinhf(x);
        case UT_EXPR_COSH: return coshf(x);
        case UT_EXPR_ATAN: return atanf(x);
        default: return expm1f(x);
    }
}

// d op(x) / dx given x and y = op(x)
__device__ __forceinline__ float prog_unary_d(int op, float x, float y) {
    switch (op) {
        case UT_EXPR_NEG: return -1.0f;
        case UT_EXPR_EXP: return y;
        case UT_EXPR_LOG: return 1.0f / x;
        case UT_EXPR_LOG1P: return 1.0f / (1.0f + x);
        case UT_EXPR_SQRT: return 0.5f / y;
        case UT_EXPR_ABS: return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f);
        case UT_EXPR_SIN: return cosf(x);
        case UT_EXPR_COS: return -sinf(x);
        case UT_EXPR_TAN: return 1.0f + y * y;
        case UT_EXPR_TANH: return 1.0f - y * y;
        case UT_EXPR_SINH: return coshf(x);
        case UT_EXPR_COSH: return sinhf(x);
        case UT_EXPR_ATAN: return 1.0f / (1.0f + x * x);
        default: return y + 1.0f;  // expm1
    }
}

// Evaluates nodes [first, root] into v[0 .. root-first].
__device__ float prog_eval(const PNode* nodes, int first, int root, float* v, const float* sv, const float* obs,
                           const ProgCtx& cx) {
    for (int i = first; i <= root; ++i) {
        const PNode n = nodes[i];
        float r;
        switch (n.op) {
            case UT_EXPR_LITERAL: r = n.v; break;
            case UT_EXPR_SLOT: r = sv[n.a]; break;
            case UT_EXPR_OBS: r = obs[cx.base[n.b] + n.a]; break;
            case kProgExprIter: r = (float)cx.iter[n.a]; break;
            case UT_EXPR_ADD: r = v[n.a - first] + v[n.b - first]; break;
            case UT_EXPR_SUB: r = v[n.a - first] - v[n.b - first]; break;
            case UT_EXPR_MUL: r = v[n.a - first] * v[n.b - first]; break;
            case UT_EXPR_DIV: r = v[n.a - first] / v[n.b - first]; break;
            case UT_EXPR_POW: r = powf(v[n.a - first], v[n.b - first]); break;
            case UT_EXPR_MIN: r = fminf(v[n.a - first], v[n.b - first]); break;
            case UT_EXPR_MAX: r = fmaxf(v[n.a - first], v[n.b - first]); break;
            default: r = prog_unary(n.op, v[n.a - first]);
        }
        v[i - first] = r;
    }
    return v[root - first];
}

// Reverse pass over one evaluated expression: adjoint `g` of its root flows to
// the latent slots it reads, added into adj[slot * 33] (the caller's column).
__device__ void prog_backprop(const PNode* nodes, int first, int root, const float* v, float g, float* adj) {
    float w[kProgMaxExprNodes];
    for (int i = 0; i <= root - first; ++i) w[i] = 0.0f;
    w[root - first] = g;
    for (int i = root; i >= first; --i) {
        const PNode n = nodes[i];
        const float wi = w[i - first];
        if (!n.dep || wi == 0.0f) continue;
        const int ia = n.a - first, ib = n.b - first;
        switch (n.op) {
            case UT_EXPR_SLOT: adj[n.a * 33] += wi; break;
            case UT_EXPR_ADD: w[ia] += wi; w[ib] += wi; break;
            case UT_EXPR_SUB: w[ia] += wi; w[ib] -= wi; break;
            case UT_EXPR_MUL: w[ia] += wi * v[ib]; w[ib] += wi * v[ia]; break;
            case UT_EXPR_DIV: w[ia] += wi / v[ib]; w[ib] -= wi * v[i - first] / v[ib]; break;
            case UT_EXPR_POW:
                if (nodes[n.a].dep) w[ia] += wi * v[ib] * powf(v[ia], v[ib] - 1.0f);
                if (nodes[n.b].dep) w[ib] += wi * v[i - first] * logf(v[ia]);
                break;
            case UT_EXPR_MIN: if (v[ia] <= v[ib]) w[ia] += wi; else w[ib] += wi; break;
            case UT_EXPR_MAX: if (v[ia] >= v[ib]) w[ia] += wi; else w[ib] += wi; break;
            case UT_EXPR_LITERAL: case UT_EXPR_OBS: case kProgExprIter: break;
            default: w[ia] += wi * prog_unary_d(n.op, v[ia], v[i - first]);
        }
    }
}

// One choice term with value x: its log-density; with `grad`, the argument
// adjoints are added into adj (the caller's lane column) and d lp / dx returned.
__device__ float prog_choice(const ProgModel& m, const PStep& s, float x, const float* sv, const ProgCtx& cx, bool grad,
                             float* adj, float& dx) {
    float v[3][kProgMaxExprNodes];
    float a[3] = {0.0f, 0.0f, 0.0f}, da[3];
    const int na = prog_dist_nargs(s.dist);
    for (int j = 0; j < na; ++j) a[j] = prog_eval(m.nodes, s.afirst[j], s.aroot[j], v[j], sv, m.obs, cx);
    const float lp = prog_dist(s.dist, a, x, grad, da, dx);
    if (grad)
        for (int j = 0; j < na; ++j)
            if (m.nodes[s.aroot[j]].dep) prog_backprop(m.nodes, s.afirst[j], s.aroot[j], v[j], da[j], adj);
    return lp;
}

// Per-warp scratch (floats): qs[pp] parameters, gs[pp] gradient, sv[64] slot
// values, adj[nslots * 33] per-lane slot adjoints (lane column, stride 33).
__host__ __device__ inline int prog_scratch_floats(int P, int nslots) {
    const int pp = ((P + 31) / 32) * 32;
    return ((2 * pp + kProgMaxSlots + 33 * nslots + 31) / 32) * 32;
}

template <int K>
__device__ float prog_lj_grad(const ProgModel& m, const float (&q)[K], float (&g)[K], float* scratch, bool want_grad) {
    const int lane = threadIdx.x & 31;
    float* qs = scratch;
    float* gs = scratch + m.pp;
    float* sv = gs + m.pp;
    float* adj = sv + kProgMaxSlots;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int p = lane + 32 * k;
        if (p < m.P) { qs[p] = q[k]; gs[p] = 0.0f; }
    }
    for (int i = lane; i < 33 * m.nslots; i += 32) adj[i] = 0.0f;
    __syncwarp();
    float* my = adj + lane;  // this lane's adjoint column
    float lj = 0.0f;
    ProgCtx cx;
    cx.base[0] = 0;
    cx.iter[0] = 0;
    int pc = 0;
    while (pc < m.nsteps) {
        const PStep s = m.steps[pc];
        if (s.kind == UT_STEP_CHOICE) {
            float x, lad = 0.0f, dxdu, dlad;
            if (s.vs >= 0) {
                x = prog_transform(s.tr, qs[s.vs], lad, dxdu, dlad);
                if (lane == 0) sv[s.slot] = x;
                __syncwarp();
            } else {
                x = m.obs[s.off];
            }
            float dx;
            // every lane evaluates the term; lane 0 keeps it
            const float lp = prog_choice(m, s, x, sv, cx, want_grad && lane == 0, my, dx);
            if (lane == 0) {
                lj += lp + lad;
                if (want_grad && s.vs >= 0) my[s.slot * 33] += dx;
            }
            ++pc;
        } else if (s.kind == UT_STEP_IID_NORMAL) {
            float v[2][kProgMaxExprNodes];
            const float mu = prog_eval(m.nodes, s.afirst[0], s.aroot[0], v[0], sv, m.obs, cx);
            const float sg = prog_eval(m.nodes, s.afirst[1], s.aroot[1], v[1], sv, m.obs, cx);
            float dmu = 0.0f, dsg = 0.0f;
            const float inv = 1.0f / sg, lsg = logf(sg);
            for (int d = lane; d < s.count; d += 32) {
                const float z = (qs[s.vs + d] - mu) * inv;
                lj += -lsg - kProgHalfLog2Pi - 0.5f * z * z;
                if (want_grad) {
                    gs[s.vs + d] -= z * inv;
                    dmu += z * inv;
                    dsg += (z * z - 1.0f) * inv;
                }
            }
            if (want_grad) {
                if (m.nodes[s.aroot[0]].dep) prog_backprop(m.nodes, s.afirst[0], s.aroot[0], v[0], dmu, my);
                if (m.nodes[s.aroot[1]].dep) prog_backprop(m.nodes, s.afirst[1], s.aroot[1], v[1], dsg, my);
            }
            ++pc;
        } else if (s.kind == UT_STEP_GLM_BERNOULLI_LOGIT) {
            // lane = covariate: per observation a warp dot product, then every lane
            // adds the residual times its covariates into its coefficient rows
            float v[kProgMaxExprNodes];
            const float icpt = s.aroot[0] >= 0 ? prog_eval(m.nodes, s.afirst[0], s.aroot[0], v, sv, m.obs, cx) : 0.0f;
            const int F = s.width;
            float racc = 0.0f, ll = 0.0f;
            for (int i = 0; i < s.count; ++i) {
                const float* row = m.obs + s.off + (size_t)i * (F + 1);
                float part = 0.0f;
                for (int d = lane; d < F; d += 32) part = fmaf(qs[s.vs + d], row[d], part);
                const float eta = icpt + warp_sum(part);
                const float y = row[F];
                const float e = expf(-fabsf(eta));
                const bool sup = (y == 0.0f) | (y == 1.0f);
                ll += sup ? y * eta - (fmaxf(eta, 0.0f) + log1pf(e)) : -INFINITY;
                if (want_grad) {
                    const float r = y - (eta >= 0.0f ? 1.0f / (1.0f + e) : e / (1.0f + e));
                    racc += r;
                    for (int d = lane; d < F; d += 32) gs[s.vs + d] = fmaf(r, row[d], gs[s.vs + d]);
                }
            }
            if (lane == 0) {
                lj += ll;
                if (want_grad && s.aroot[0] >= 0 && m.nodes[s.aroot[0]].dep)
                    prog_backprop(m.nodes, s.afirst[0], s.aroot[0], v, racc, my);
            }
            ++pc;
        } else {  // UT_STEP_LOOP at the top level: lanes take its iterations
            const int end = pc + 1 + s.body;
            for (int t = lane; t < s.count; t += 32) {
                int li[kProgMaxDepth + 1], it[kProgMaxDepth + 1];
                int depth = 1;
                li[1] = pc;
                it[1] = t;
                cx.base[1] = s.off + t * s.width;
                cx.iter[1] = s.istart + t;
                int ip = pc + 1;
                while (true) {
                    const PStep& L = m.steps[li[depth]];
                    if (ip == li[depth] + 1 + L.body) {
                        if (depth == 1) break;
                        if (++it[depth] < L.count) {
                            cx.base[depth] = cx.base[depth - 1] + L.off + it[depth] * L.width;
                            cx.iter[depth] = L.istart + it[depth];
                            ip = li[depth] + 1;
                        } else {
                            --depth;  // ip already points past the finished loop's body
                        }
                        continue;
                    }
                    const PStep b = m.steps[ip];
                    if (b.kind == UT_STEP_LOOP) {
                        if (b.count == 0) { ip += 1 + b.body; continue; }
                        ++depth;
                        li[depth] = ip;
                        it[depth] = 0;
                        cx.base[depth] = cx.base[depth - 1] + b.off;
                        cx.iter[depth] = b.istart;
                        ++ip;
                        continue;
                    }
                    // an observed choice of the body
                    float dx;
                    lj += prog_choice(m, b, m.obs[cx.base[depth] + b.off], sv, cx, want_grad, my, dx);
                    ++ip;
                }
            }
            pc = end;
        }
    }
    lj = warp_sum(lj);
    if (want_grad) {
        __syncwarp();
        // slot adjoints: lane s sums slot s's 33-stride row in lane order
        for (int sl = lane; sl < m.nslots; sl += 32) {
            float acc = 0.0f;
            for (int j = 0; j < 32; ++j) acc += adj[sl * 33 + j];
            adj[sl * 33 + 32] = acc;
        }
        __syncwarp();
        // latent scalar values: gradient of the unconstrained row
        for (int k = lane; k < m.nsteps; k += 32) {
            const PStep s = m.steps[k];
            if (s.kind == UT_STEP_CHOICE && s.vs >= 0) {
                float lad, dxdu, dlad;
                prog_transform(s.tr, qs[s.vs], lad, dxdu, dlad);
                gs[s.vs] += adj[s.slot * 33 + 32] * dxdu + dlad;  // a GLM step may have added to the row
            }
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int p = lane + 32 * k;
            g[k] = p < m.P ? gs[p] : 0.0f;
        }
    }
    __syncwarp();
    return lj;
}

}  // namespace ut
