/* A plain C host of the B200 library, bound through include/ut_b200.h alone:
 * what a non-Python caller (the reference's Julia ccall shim, a C service)
 * sees at the boundary.  Without a device it exercises the host-side contract:
 * version string, lowering report with its issue list, the workspace's
 * argument validation and the no-device error.  With a device it also
 * evaluates a two-observation logistic regression and checks the logjoint and
 * gradient against the closed form.  Exit status 0 = every check held. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "ut_b200.h"

static int failures = 0;

#define CHECK(cond, what)                                   \
    do {                                                    \
        if (!(cond)) {                                      \
            fprintf(stderr, "FAILED: %s\n", what);          \
            failures++;                                     \
        }                                                   \
    } while (0)

static double log1p_exp(double x) { return x > 0 ? x + log1p(exp(-x)) : log1p(exp(x)); }

int main(void) {
    char buf[512];
    CHECK(ut_version() != NULL && strlen(ut_version()) > 0, "version string");

    /* y_i ~ bernoullilogit(x_i . beta), beta ~ normal(0, 1), D = 2, N = 2 */
    ut_plan_desc plan;
    memset(&plan, 0, sizeof plan);
    plan.family = UT_FAMILY_GLM_BERNOULLI_LOGIT;
    plan.num_params = 2;
    plan.num_obs = 2;
    plan.num_coefs = 2;
    plan.coef_mu = 0.0;
    plan.coef_sigma = 1.0;
    plan.intercept_sigma = 1.0;
    CHECK(ut_lowering_report(&plan, buf, sizeof buf) == UT_OK, "GLM description lowers");

    ut_plan_desc bad = plan;
    bad.coef_sigma = 0.0;
    CHECK(ut_lowering_report(&bad, buf, sizeof buf) == UT_ERR_UNSUPPORTED, "bad prior scale is unsupported");
    CHECK(strstr(buf, "coefficient prior scale") != NULL, "issue list names the prior scale");

    /* staged rows: per observation the D covariates then y */
    const float observed[6] = {0.5f, -1.0f, 1.0f, /**/ -0.3f, 0.8f, 0.0f};
    ut_workspace* ws = NULL;
    CHECK(ut_workspace_create(&plan, observed, 6, 1, NULL, NULL, 0, 3, 64, &ws) == UT_ERR_PRECISION,
          "Float64 is refused");
    CHECK(ut_workspace_create(&plan, observed, 5, 1, NULL, NULL, 0, 3, 32, &ws) == UT_ERR_DIMENSION,
          "wrong staged row count is a dimension error");
    CHECK(ut_workspace_info(NULL, NULL, NULL) == UT_ERR_ARGUMENT, "null handle");
    ut_last_error(buf, sizeof buf);
    CHECK(strstr(buf, "null workspace handle") != NULL, "last error names the null handle");

    int32_t rc = ut_workspace_create(&plan, observed, 6, 1, NULL, NULL, 0, 3, 32, &ws);
    if (ut_device_count() == 0) {
        CHECK(rc == UT_ERR_NO_DEVICE && ws == NULL, "no device: no workspace, no CPU fallback");
    } else {
        CHECK(rc == UT_OK && ws != NULL, "workspace created");
        if (rc == UT_OK) {
            /* params P x C column-major: chain c's two coefficients are contiguous */
            const float params[6] = {0.2f, -0.4f, 1.0f, 0.5f, -0.7f, 0.1f};
            float totals[3], grads[6];
            CHECK(ut_logjoint_gradient(ws, params, totals, grads) == UT_OK, "logjoint_gradient");
            for (int c = 0; c < 3; ++c) {
                const double b0 = params[2 * c], b1 = params[2 * c + 1];
                double lj = -0.5 * (b0 * b0 + b1 * b1) - log(2.0 * M_PI), g0 = -b0, g1 = -b1;
                for (int i = 0; i < 2; ++i) {
                    const double x0 = observed[3 * i], x1 = observed[3 * i + 1], y = observed[3 * i + 2];
                    const double eta = x0 * b0 + x1 * b1, p = 1.0 / (1.0 + exp(-eta));
                    lj += y * eta - log1p_exp(eta);
                    g0 += (y - p) * x0;
                    g1 += (y - p) * x1;
                }
                CHECK(fabs(totals[c] - lj) <= 1e-5 * fabs(lj), "logjoint matches the closed form");
                CHECK(fabs(grads[2 * c] - g0) <= 1e-5 && fabs(grads[2 * c + 1] - g1) <= 1e-5,
                      "gradient matches the closed form");
            }
            CHECK(ut_workspace_destroy(ws) == UT_OK, "destroy");
        }
    }
    if (failures == 0) printf("c_caller: all checks passed (%s)\n", ut_device_count() ? "device" : "no device");
    return failures == 0 ? 0 : 1;
}
