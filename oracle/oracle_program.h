// oracle_program.h -- CPU restatement of the reference's device plan walk for a
// step program (TEST INFRASTRUCTURE ONLY; see oracle_program.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "../include/ut_b200.h"

namespace oracle_program {

struct Program {
    std::vector<ut_program_step> steps;
    std::vector<ut_expr_node> nodes;
    int nslots = 0;
    int P = 0;
};

// The program the next model built with family UT_FAMILY_PROGRAM uses.
Program& current();

// Logjoint (and, when g != nullptr, its gradient) of one chain in float64,
// the gradient by forward-mode duals, one pass per parameter row.  With mag,
// also the gradient magnitude: per row, the sum of the magnitudes of every
// contribution to the derivative (each operation's |partial| times its
// operand's magnitude), the scale of the FP32 rounding error of the gradient.
double logjoint_grad(const Program& prog, const std::vector<double>& obs, const double* q, double* g,
                     double* mag = nullptr);

}  // namespace oracle_program
