// The correlated-field generator on the GPU (see fieldgen.cu).
#pragma once

namespace mgk {

// generate_correlated_field_cpp (material_generator.hpp:130-258) into
// out_host (N values); throws on CUDA errors and unsupported axis lengths.
void correlated_field(int dim, int nx, int ny, int nz, double mean, double sd, double corr, bool has_min, double cmin,
                      bool has_max, double cmax, int seed, double* out_host);

}  // namespace mgk
