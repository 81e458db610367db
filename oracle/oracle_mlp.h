// oracle_mlp.h -- CPU restatement of the project's learned gradient surrogate
// (the MLP  P -> 256 -> 256 -> P  with SiLU hidden layers).  TEST
// INFRASTRUCTURE ONLY.  The surrogate has no counterpart in the reference; this
// restatement follows the rounding points of uncertaintea_b200/csrc/ut_mlp.cuh
// (BF16 operands, wide accumulation) when bf16 != 0, and plain FP64 otherwise.
#pragma once

#include <cstdint>

namespace oracle_mlp {

constexpr int kH = 256;

struct Layout {
    int P, Pp;
    int64_t w1, b1, w2, b2, w3, b3, total;
    static Layout make(int P);
};

// Surrogate gradient at n positions x (n x P) -> out (n x P).
void forward(const float* params, const float* norm, int P, const float* x, int64_t n, float* out, int bf16);

// The same network with its (rounded) weights prepared once; operator() maps
// one position (P floats) to its surrogate gradient.  Safe to call from
// several threads at once.
class Evaluator {
  public:
    Evaluator(const float* params, const float* norm, int P, int bf16);
    ~Evaluator();
    Evaluator(const Evaluator&) = delete;
    Evaluator& operator=(const Evaluator&) = delete;
    void operator()(const float* theta, float* out) const;

  private:
    struct Impl;
    Impl* impl_;
};

}  // namespace oracle_mlp
