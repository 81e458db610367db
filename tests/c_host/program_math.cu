// program_math.cu -- host build of the step program's distribution and
// transform arithmetic (uncertaintea_b200/csrc/ut_program.cuh), so the CPU
// tests can check the device formulas' values and partial derivatives
// without a GPU.  Test harness only.
#include "../../include/ut_b200.h"
#include "../../uncertaintea_b200/csrc/ut_program.cuh"

extern "C" float prog_dist_host(int dist, const float* a, float x, float* da, float* dx) {
    float d = 0.0f;
    const float lp = ut::prog_dist(dist, a, x, true, da, d);
    *dx = d;
    return lp;
}

extern "C" float prog_digamma_host(float x) { return ut::prog_digamma(x); }

extern "C" float prog_transform_host(int tr, float u, float* lad, float* dxdu, float* dlad) {
    return ut::prog_transform(tr, u, *lad, *dxdu, *dlad);
}
