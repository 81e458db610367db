// ut_tc_glm.cuh -- tensor-core (tcgen05, 3xTF32) GLM logjoint + gradient.
// Placeholder until the sm_100a kernel lands: `enabled` stays false and the
// CUDA-core tiled kernel serves the large-N path.
#pragma once

#include <cuda_runtime.h>
#include <vector>

namespace ut {

struct TcGlmPlan {
    bool enabled = false;
};

inline const char* tc_glm_last_error() { return ""; }

inline int tc_glm_setup(TcGlmPlan& plan, const float*, const float*, int, int, int, int, float, float, float, float,
                        int, std::vector<void*>*) {
    plan.enabled = false;
    return 0;
}

inline cudaError_t tc_glm_launch(const TcGlmPlan&, const float*, float*, float*, cudaStream_t) {
    return cudaErrorNotSupported;
}

}  // namespace ut
