// ASCII VTU (VTK XML unstructured hexahedra) output with the reference's
// layout and number formatting (vtu_writer.hpp:23-395).
#pragma once
#include <string>

namespace mgk {

// eps, sig, eps_plastic: N row-major DxD tensors (eps_plastic may be null);
// soft: N x 2 (g_p, g_t) or null; E, nu: N values.  D = 2 writes an nz = 1
// slab with the 2x2 block embedded in 3x3 (export_to_vtu_2d, :368-395).
// Throws std::runtime_error when the file cannot be opened (:183-186).
void write_vtu_fields(const std::string& filename, int D, int nx, int ny, int nz, const double* eps, const double* sig,
                      const double* E, const double* nu, double pixel, const double* eps_plastic, const double* soft);

}  // namespace mgk
