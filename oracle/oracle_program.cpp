// oracle_program.cpp -- CPU restatement of the reference's device plan walk for
// a step program (include/ut_b200.h, UT_FAMILY_PROGRAM).  TEST INFRASTRUCTURE
// ONLY: the parity tests load it as the oracle; the product library never
// links, loads or calls it.
//
// It follows the reference's interpreter, not the B200 kernel: the steps are
// walked in order with a slots array written by choice bindings,
// deterministic steps and loop iterators (src/device/logjoint_kernel.jl:
// 60-78, 614-634, 700-720), loops walk their body once per iteration over the
// iteration's block of staged rows, and the gradient is forward mode with a
// scalar dual seeded on one parameter row per pass, as the reference's
// gradient kernel does per (parameter, chain) thread
// (src/device/gradient_kernel.jl:1116-1145, src/device/dual.jl:17-153).
// The densities restate src/device/math.jl:88-300 and the transforms
// math.jl:1137-1159, in float64.  Parity of this restatement is pinned by
// closed forms (scipy densities) and central finite differences in the CPU
// tests, not by reference outputs (Julia is not available here).
#include "oracle_program.h"

#include <cfloat>
#include <cmath>
#include <limits>

namespace oracle_program {

Program& current() {
    static Program p;
    return p;
}

namespace {

// Forward-mode dual seeded on one parameter row: value v, derivative d, and m,
// the sum of the magnitudes of every contribution to d (each operation adds
// |partial| x |operand's m| instead of partial x operand's d).  m is the scale
// of the rounding error of an evaluation of d, cancellation included.
struct Dual {
    double v, d, m;
};
inline Dual C(double v) { return {v, 0.0, 0.0}; }
inline Dual un(double v, double dv, const Dual& a) { return {v, dv * a.d, std::fabs(dv) * a.m}; }
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d, a.m + b.m}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d, a.m + b.m}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d, a.m}; }
inline Dual operator*(Dual a, Dual b) {
    return {a.v * b.v, a.d * b.v + a.v * b.d, a.m * std::fabs(b.v) + std::fabs(a.v) * b.m};
}
inline Dual operator/(Dual a, Dual b) {
    return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v),
            a.m / std::fabs(b.v) + std::fabs(a.v) * b.m / (b.v * b.v)};
}
inline Dual operator+(Dual a, double b) { return {a.v + b, a.d, a.m}; }
inline Dual operator-(Dual a, double b) { return {a.v - b, a.d, a.m}; }
inline Dual operator-(double a, Dual b) { return {a - b.v, -b.d, b.m}; }
inline Dual operator*(double a, Dual b) { return {a * b.v, a * b.d, std::fabs(a) * b.m}; }
inline Dual operator/(Dual a, double b) { return {a.v / b, a.d / b, a.m / std::fabs(b)}; }
inline Dual dlog(Dual a) { return un(std::log(a.v), 1.0 / a.v, a); }
inline Dual dexp(Dual a) { const double e = std::exp(a.v); return un(e, e, a); }
inline Dual dlog1p(Dual a) { return un(std::log1p(a.v), 1.0 / (1.0 + a.v), a); }
inline Dual dsqrt(Dual a) { const double s = std::sqrt(a.v); return un(s, 0.5 / s, a); }
inline Dual dabs(Dual a) { return a.v < 0 ? -a : a; }
inline Dual dsin(Dual a) { return un(std::sin(a.v), std::cos(a.v), a); }
inline Dual dcos(Dual a) { return un(std::cos(a.v), -std::sin(a.v), a); }
inline Dual dtan(Dual a) { const double t = std::tan(a.v); return un(t, 1.0 + t * t, a); }
inline Dual dtanh(Dual a) { const double t = std::tanh(a.v); return un(t, 1.0 - t * t, a); }
inline Dual dsinh(Dual a) { return un(std::sinh(a.v), std::cosh(a.v), a); }
inline Dual dcosh(Dual a) { return un(std::cosh(a.v), std::sinh(a.v), a); }
inline Dual datan(Dual a) { return un(std::atan(a.v), 1.0 / (1.0 + a.v * a.v), a); }
inline Dual dexpm1(Dual a) { return un(std::expm1(a.v), std::exp(a.v), a); }
inline Dual dpow(Dual a, Dual b) {
    const double p = std::pow(a.v, b.v);
    const double pa = b.v * std::pow(a.v, b.v - 1.0);
    double d = pa * a.d, m = std::fabs(pa) * a.m;
    if (b.d != 0.0 || b.m != 0.0) {
        const double pb = p * std::log(a.v);
        d += pb * b.d;
        m += std::fabs(pb) * b.m;
    }
    return {p, d, m};
}
inline Dual dmin(Dual a, Dual b) { return a.v <= b.v ? a : b; }
inline Dual dmax(Dual a, Dual b) { return a.v >= b.v ? a : b; }

// digamma by upward recurrence to x >= 10 and the asymptotic series
// ln x - 1/(2x) - sum_{k=1..6} B_2k / (2k x^2k).
double digamma(double x) {
    double acc = 0.0;
    while (x < 10.0) {
        acc -= 1.0 / x;
        x += 1.0;
    }
    const double r = 1.0 / x, r2 = r * r;
    const double s = r2 * (1.0 / 12 - r2 * (1.0 / 120 - r2 * (1.0 / 252 - r2 * (1.0 / 240 - r2 * (1.0 / 132 -
                                                                                                      r2 * (691.0 / 32760))))));
    return acc + std::log(x) - 0.5 * r - s;
}
inline Dual dlgamma(Dual a) { return un(std::lgamma(a.v), digamma(a.v), a); }

const double kNegInf = -std::numeric_limits<double>::infinity();
const double kHalfLog2Pi = 0.9189385332046727;  // math.jl:90
const double kLogPi = 1.1447298858494002;       // math.jl:113
const double kLog2 = 0.6931471805599453;

inline bool positive_normal(Dual x) { return x.v >= DBL_MIN; }  // math.jl:59-66
inline Dual sel(bool c, Dual a, double b) { return c ? a : C(b); }

// loggamma(x + 1/2) - loggamma(x) (math.jl:80-86; crossover 1200 in Float64)
Dual lgamma_half_ratio(Dual x) {
    if (x.v > 1200.0)
        return x * dlog1p(C(1.0) / (2.0 * x)) + dlog(x) / 2.0 - 0.5 + (C(1.0) / (x + 0.5) - C(1.0) / x) / 12.0;
    return dlgamma(x + 0.5) - dlgamma(x);
}

// math.jl:88-300
Dual logpdf(int dist, const Dual* a, Dual x) {
    switch (dist) {
        case UT_DIST_NORMAL: {  // math.jl:88-91
            const Dual z = (x - a[0]) / a[1];
            return -dlog(a[1]) - kHalfLog2Pi - z * z / 2.0;
        }
        case UT_DIST_LOGNORMAL: {  // :93-97
            const Dual lx = dlog(x), z = (lx - a[0]) / a[1];
            return sel(positive_normal(x), -dlog(a[1]) - kHalfLog2Pi - z * z / 2.0 - lx, kNegInf);
        }
        case UT_DIST_EXPONENTIAL:  // :99-101
            return sel(x.v >= 0.0, dlog(a[0]) - a[0] * x, kNegInf);
        case UT_DIST_GAMMA:  // :103-107
            return sel(positive_normal(x), a[0] * dlog(a[1]) - dlgamma(a[0]) + (a[0] - 1.0) * dlog(x) - a[1] * x, kNegInf);
        case UT_DIST_LAPLACE:  // :109-111
            return -dlog(2.0 * a[1]) - dabs(x - a[0]) / a[1];
        case UT_DIST_CAUCHY: {  // :115-118
            const Dual z = (x - a[0]) / a[1];
            return -dlog(a[1]) - kLogPi - dlog1p(z * z);
        }
        case UT_DIST_HALFNORMAL: {  // :120-124
            const Dual z = x / a[0];
            return sel(x.v >= 0.0, -dlog(a[0]) + kLog2 - kHalfLog2Pi - z * z / 2.0, kNegInf);
        }
        case UT_DIST_HALFCAUCHY: {  // :126-130
            const Dual z = x / a[0];
            return sel(x.v >= 0.0, -dlog(a[0]) + (kLog2 - kLogPi) - dlog1p(z * z), kNegInf);
        }
        case UT_DIST_LOGISTIC: {  // :132-136
            const Dual z = (x - a[0]) / a[1], az = dabs(z);
            return -dlog(a[1]) - az - 2.0 * dlog1p(dexp(-az));
        }
        case UT_DIST_GUMBEL: {  // :138-141
            const Dual z = (x - a[0]) / a[1];
            return -dlog(a[1]) - z - dexp(-z);
        }
        case UT_DIST_FRECHET: {  // :144-148
            const Dual lz = dlog(x) - dlog(a[1]);
            return sel(positive_normal(x), dlog(a[0]) - dlog(a[1]) - (a[0] + 1.0) * lz - dexp(-(a[0] * lz)), kNegInf);
        }
        case UT_DIST_RAYLEIGH:  // :150-153
            return sel(positive_normal(x), dlog(x) - 2.0 * dlog(a[0]) - x * x / (2.0 * a[0] * a[0]), kNegInf);
        case UT_DIST_INVERSEGAUSSIAN: {  // :155-159
            const Dual d = x - a[0];
            return sel(positive_normal(x),
                       0.5 * dlog(a[1]) - kHalfLog2Pi - 1.5 * dlog(x) - a[1] * d * d / (2.0 * a[0] * a[0] * x), kNegInf);
        }
        case UT_DIST_BETA: {  // :161-165
            const Dual lb = dlgamma(a[0]) + dlgamma(a[1]) - dlgamma(a[0] + a[1]);
            return sel(x.v > 0.0 && x.v < 1.0, (a[0] - 1.0) * dlog(x) + (a[1] - 1.0) * dlog1p(-x) - lb, kNegInf);
        }
        case UT_DIST_STUDENTT: {  // :167-173
            const Dual z = (x - a[1]) / a[2];
            return lgamma_half_ratio(a[0] / 2.0) - (dlog(a[0]) + kLogPi) / 2.0 - dlog(a[2]) -
                   (a[0] + 1.0) * dlog1p(z * z / a[0]) / 2.0;
        }
        case UT_DIST_INVERSEGAMMA:  // :175-179
            return sel(positive_normal(x),
                       a[0] * dlog(a[1]) - dlgamma(a[0]) - (a[0] + 1.0) * dlog(x) - a[1] / x, kNegInf);
        case UT_DIST_WEIBULL: {  // :181-186
            if (positive_normal(x))
                return dlog(a[0]) + (a[0] - 1.0) * dlog(x) - a[0] * dlog(a[1]) - dexp(a[0] * (dlog(x) - dlog(a[1])));
            if (x.v == 0.0) {
                if (a[0].v < 1.0) return C(std::numeric_limits<double>::infinity());
                return a[0].v == 1.0 ? -dlog(a[1]) : C(kNegInf);
            }
            return C(kNegInf);
        }
        case UT_DIST_BERNOULLI: {  // :191-195
            const bool sup = x.v == 0.0 || x.v == 1.0;
            return sel(sup, x.v > 0.5 ? dlog(a[0]) : dlog1p(-a[0]), kNegInf);
        }
        case UT_DIST_BERNOULLI_LOGIT: {  // :202-217
            const Dual eta = a[0];
            const Dual lpe = eta.v > 0.0 ? eta + dlog1p(dexp(-eta)) : dlog1p(dexp(eta));
            const bool sup = x.v == 0.0 || x.v == 1.0;
            return sel(sup, x * eta - lpe, kNegInf);
        }
        case UT_DIST_POISSON: {  // :230-235
            const double k = std::round(x.v);
            const bool ok = x.v >= 0.0 && x.v == k;
            return sel(ok, k * dlog(a[0]) - a[0] - std::lgamma(k + 1.0), kNegInf);
        }
        case UT_DIST_GEOMETRIC: {  // :281-285
            const double k = std::round(x.v);
            const bool ok = x.v >= 0.0 && x.v == k;
            return sel(ok, dlog(a[0]) + (k > 0.0 ? k * dlog1p(-a[0]) : C(0.0)), kNegInf);
        }
        case UT_DIST_NEGATIVE_BINOMIAL: {  // :287-294
            const double k = std::round(x.v);
            const bool ok = x.v >= 0.0 && x.v == k;
            const Dual base = dlgamma(a[0] + k) - dlgamma(a[0]) - std::lgamma(k + 1.0) + a[0] * dlog(a[1]) +
                              (k > 0.0 ? k * dlog1p(-a[1]) : C(0.0));
            return sel(ok, base, kNegInf);
        }
        case UT_DIST_BINOMIAL: {  // :261-279 (trials from the first argument)
            const double n = std::round(a[0].v), k = std::round(x.v);
            const bool ok = x.v == k && a[0].v == n && k >= 0.0 && n >= 0.0 && k <= n;
            const double lc = std::lgamma(n + 1.0) - std::lgamma(k + 1.0) - std::lgamma(n - k + 1.0);
            const Dual base = C(lc) + (k > 0.0 ? k * dlog(a[1]) : C(0.0)) + (k < n ? (n - k) * dlog1p(-a[1]) : C(0.0));
            return sel(ok, base, kNegInf);
        }
        default:
            return C(std::numeric_limits<double>::quiet_NaN());
    }
}

// math.jl:1144-1159: (constrained value, log|J|)
Dual transform(int tr, Dual u, Dual& lad) {
    if (tr == UT_TRANSFORM_LOG) {
        lad = u;
        return dexp(u);
    }
    if (tr == UT_TRANSFORM_LOGIT) {
        const Dual c = C(1.0) / (C(1.0) + dexp(-u)), m = dabs(u);
        lad = -m - 2.0 * dlog1p(dexp(-m));
        return c;
    }
    lad = C(0.0);
    return u;
}

struct Walker {
    const Program& p;
    const std::vector<double>& obs;
    const Dual* q;
    std::vector<Dual> slots;
    std::vector<long long> base;   // block base row per loop depth

    Dual eval(int i) {
        const ut_expr_node& n = p.nodes[i];
        switch (n.op) {
            case UT_EXPR_LITERAL: return C(n.value);
            case UT_EXPR_SLOT: return slots[n.a];
            case UT_EXPR_OBS: return C(obs[base[n.b] + n.a]);
            case UT_EXPR_NEG: return -eval(n.a);
            case UT_EXPR_ADD: return eval(n.a) + eval(n.b);
            case UT_EXPR_SUB: return eval(n.a) - eval(n.b);
            case UT_EXPR_MUL: return eval(n.a) * eval(n.b);
            case UT_EXPR_DIV: return eval(n.a) / eval(n.b);
            case UT_EXPR_POW: return dpow(eval(n.a), eval(n.b));
            case UT_EXPR_EXP: return dexp(eval(n.a));
            case UT_EXPR_LOG: return dlog(eval(n.a));
            case UT_EXPR_LOG1P: return dlog1p(eval(n.a));
            case UT_EXPR_SQRT: return dsqrt(eval(n.a));
            case UT_EXPR_ABS: return dabs(eval(n.a));
            case UT_EXPR_MIN: return dmin(eval(n.a), eval(n.b));
            case UT_EXPR_MAX: return dmax(eval(n.a), eval(n.b));
            case UT_EXPR_SIN: return dsin(eval(n.a));
            case UT_EXPR_COS: return dcos(eval(n.a));
            case UT_EXPR_TAN: return dtan(eval(n.a));
            case UT_EXPR_TANH: return dtanh(eval(n.a));
            case UT_EXPR_SINH: return dsinh(eval(n.a));
            case UT_EXPR_COSH: return dcosh(eval(n.a));
            case UT_EXPR_ATAN: return datan(eval(n.a));
            default: return dexpm1(eval(n.a));
        }
    }

    void bind(int slot, Dual v) {
        if (slot >= 0) slots[slot] = v;
    }

    // Walks steps [i, end) at loop depth `depth`; returns their log-density.
    Dual walk(int i, int end, int depth) {
        Dual total = C(0.0);
        while (i < end) {
            const ut_program_step& s = p.steps[i];
            switch (s.kind) {
                case UT_STEP_DETERMINISTIC:
                    bind(s.binding_slot, eval(s.arg[0]));
                    ++i;
                    break;
                case UT_STEP_CHOICE: {
                    Dual a[4];
                    const int na = s.dist == UT_DIST_STUDENTT ? 3 : (s.arg[1] >= 0 ? 2 : 1);
                    for (int j = 0; j < na; ++j) a[j] = eval(s.arg[j]);
                    Dual x, lad = C(0.0);
                    if (s.value_source >= 0) x = transform(s.transform, q[s.value_source], lad);
                    else x = C(obs[base[depth] + s.obs_offset]);
                    bind(s.binding_slot, x);
                    total = total + logpdf(s.dist, a, x) + lad;
                    ++i;
                    break;
                }
                case UT_STEP_IID_NORMAL: {  // DeviceDiagNormalChoiceStepDyn (logjoint_kernel.jl:514-533)
                    const Dual mu = eval(s.arg[0]), sg = eval(s.arg[1]);
                    Dual a[2] = {mu, sg};
                    for (int d = 0; d < s.count; ++d) total = total + logpdf(UT_DIST_NORMAL, a, q[s.value_source + d]);
                    ++i;
                    break;
                }
                case UT_STEP_GLM_BERNOULLI_LOGIT: {  // logjoint_kernel.jl:378-399
                    const Dual icpt = s.arg[0] >= 0 ? eval(s.arg[0]) : C(0.0);
                    const int F = s.width;
                    for (int k = 0; k < s.count; ++k) {
                        const long long row = base[depth] + s.obs_offset + (long long)k * (F + 1);
                        Dual eta = icpt;
                        for (int d = 0; d < F; ++d) eta = eta + q[s.value_source + d] * C(obs[row + d]);
                        Dual a[1] = {eta};
                        total = total + logpdf(UT_DIST_BERNOULLI_LOGIT, a, C(obs[row + F]));
                    }
                    ++i;
                    break;
                }
                case UT_STEP_LOOP: {  // logjoint_kernel.jl:620-634
                    const int body_end = i + 1 + s.body;
                    if ((int)base.size() < depth + 2) base.resize(depth + 2);
                    for (int t = 0; t < s.count; ++t) {
                        base[depth + 1] = base[depth] + s.obs_offset + (long long)t * s.width;
                        bind(s.iterator_slot, C((double)(s.iterator_start + t)));
                        total = total + walk(i + 1, body_end, depth + 1);
                    }
                    i = body_end;
                    break;
                }
                default:
                    return C(std::numeric_limits<double>::quiet_NaN());
            }
        }
        return total;
    }
};

}  // namespace

double logjoint_grad(const Program& prog, const std::vector<double>& obs, const double* q, double* g, double* mag) {
    const int P = prog.P;
    std::vector<Dual> qd(P);
    double value = 0.0;
    const bool seed = g || mag;
    const int passes = seed ? P : 1;
    for (int s = 0; s < passes; ++s) {
        for (int r = 0; r < P; ++r) qd[r] = {q[r], (seed && r == s) ? 1.0 : 0.0, (seed && r == s) ? 1.0 : 0.0};
        Walker w{prog, obs, qd.data(), std::vector<Dual>(std::max(prog.nslots, 1)), std::vector<long long>(1, 0)};
        const Dual t = w.walk(0, (int)prog.steps.size(), 0);
        value = t.v;
        if (g) g[s] = t.d;
        if (mag) mag[s] = t.m;
    }
    return value;
}

}  // namespace oracle_program
