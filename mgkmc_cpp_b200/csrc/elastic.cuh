// Linear-elastic simulation driver (main.cpp:418-869) over the GPU LS solver.
#pragma once
#include <string>

#include "../../include/mgkmc_b200.h"

namespace mgk {

// Runs the whole proportional-loading schedule; macro_out (nullable) gets
// (n_steps + 1) rows of {eps_macro, sig_macro} (row-major DxD each),
// ls_iters_out (nullable) the LS iterations summed over every solve.
mgk_status elastic_run(const mgk_le_params& p, const double* E, const double* nu, double* macro_out, int* ls_iters_out,
                       std::string* err);

}  // namespace mgk
