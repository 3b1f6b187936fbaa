// mg.hpp -- geometric multigrid preconditioner and the mixed-precision solve.
#pragma once
#include "problem.hpp"

namespace icb
{
/// GMG-preconditioned CG in FP64 (precision ICB_FP64) or FP32 inner GMG-PCG
/// inside FP64 defect correction (precision ICB_MIXED).
int solve_multigrid(icb_problem p, const icb_solve_opts &o, const double *b,
                    icb_solve_info *info);
} // namespace icb
