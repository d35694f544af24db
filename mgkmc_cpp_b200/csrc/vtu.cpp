// VTU writer: element-centred displacement reconstruction
// (reconstruct_displacement_element_centered, vtu_writer.hpp:23-168) and the
// ASCII file layout of export_to_vtu (:171-366).  Values go through a default
// std::ostream (6 significant digits), as in the reference, so the text is the
// same for the same numbers.
#include "vtu.h"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <stdexcept>
#include <vector>

namespace mgk {

namespace {

struct T3 {
    double a[9];  // row-major 3x3
    double operator()(int i, int j) const { return a[i * 3 + j]; }
};

static std::vector<T3> embed(int D, const double* src, size_t N) {
    std::vector<T3> out(N);
    for (size_t v = 0; v < N; ++v) {
        for (int k = 0; k < 9; ++k) out[v].a[k] = 0.0;
        for (int i = 0; i < D; ++i)
            for (int j = 0; j < D; ++j) out[v].a[i * 3 + j] = src[v * D * D + i * D + j];
    }
    return out;
}

// sqrt(c * |dev(t)|^2) with the squared norm summed in column-major storage order
static double vm(const T3& t, double c) {
    double tr = (t(0, 0) + t(1, 1)) + t(2, 2);
    double s = 0.0;
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double d = t(i, j) - (i == j ? 1.0 : 0.0) * (tr / 3.0);
            s += d * d;
        }
    return std::sqrt(c * s);
}

}  // namespace

void write_vtu_fields(const std::string& filename, int D, int nx, int ny, int nz, const double* eps2, const double* sig2,
                      const double* E, const double* nu, double pixel, const double* epsp2, const double* soft) {
    const size_t N = (size_t)nx * ny * nz;
    std::vector<T3> eps = embed(D, eps2, N), sig = embed(D, sig2, N);
    std::vector<T3> epsp;
    if (epsp2) epsp = embed(D, epsp2, N);
    std::ofstream fs(filename);
    if (!fs.is_open()) throw std::runtime_error("Failed to open VTU file for writing: " + filename);
    const int Nx = nx + 1, Ny = ny + 1, Nz = nz + 1;
    const long num_points = (long)Nx * Ny * Nz;
    const long num_cells = (long)N;
    fs << "<?xml version=\"1.0\"?>\n";
    fs << "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    fs << "  <UnstructuredGrid>\n";
    fs << "    <Piece NumberOfPoints=\"" << num_points << "\" NumberOfCells=\"" << num_cells << "\">\n";
    // displacement by axis-wise integration of the strain (vtu_writer.hpp:42-165)
    std::vector<double> u(3 * num_points, 0.0);
    auto node = [&](int i, int j, int k) { return ((long)i * Ny * Nz + (long)j * Nz + k); };
    auto elem = [&](int i, int j, int k) { return ((long)i * ny * nz + (long)j * nz + k); };
    for (int i = 1; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k)
                u[3 * node(i, j, k)] = u[3 * node(i - 1, j, k)] + eps[elem(i - 1, std::min(j, ny - 1), std::min(k, nz - 1))](0, 0) * pixel;
    for (int j = 1; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i)
            for (int k = 0; k < Nz; ++k)
                u[3 * node(i, j, k) + 1] = u[3 * node(i, j - 1, k) + 1] + eps[elem(std::min(i, nx - 1), j - 1, std::min(k, nz - 1))](1, 1) * pixel;
    for (int k = 1; k < Nz; ++k)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                u[3 * node(i, j, k) + 2] = u[3 * node(i, j, k - 1) + 2] + eps[elem(std::min(i, nx - 1), std::min(j, ny - 1), k - 1)](2, 2) * pixel;
    for (int j = 1; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i)
            for (int k = 0; k < Nz; ++k) u[3 * node(i, j, k)] += 0.5 * eps[elem(std::min(i, nx - 1), j - 1, std::min(k, nz - 1))](0, 1) * pixel;
    for (int k = 1; k < Nz; ++k)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j) u[3 * node(i, j, k)] += 0.5 * eps[elem(std::min(i, nx - 1), std::min(j, ny - 1), k - 1)](0, 2) * pixel;
    for (int i = 1; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) u[3 * node(i, j, k) + 1] += 0.5 * eps[elem(i - 1, std::min(j, ny - 1), std::min(k, nz - 1))](0, 1) * pixel;
    for (int k = 1; k < Nz; ++k)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j) u[3 * node(i, j, k) + 1] += 0.5 * eps[elem(std::min(i, nx - 1), std::min(j, ny - 1), k - 1)](1, 2) * pixel;
    for (int i = 1; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) u[3 * node(i, j, k) + 2] += 0.5 * eps[elem(i - 1, std::min(j, ny - 1), std::min(k, nz - 1))](0, 2) * pixel;
    for (int j = 1; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i)
            for (int k = 0; k < Nz; ++k) u[3 * node(i, j, k) + 2] += 0.5 * eps[elem(std::min(i, nx - 1), j - 1, std::min(k, nz - 1))](1, 2) * pixel;
    double u0[3] = {0, 0, 0};
    for (int j = 0; j < Ny; ++j)
        for (int k = 0; k < Nz; ++k)
            for (int c = 0; c < 3; ++c) u0[c] += u[3 * node(0, j, k) + c];
    for (int c = 0; c < 3; ++c) u0[c] /= (Ny * Nz);
    for (long i = 0; i < num_points; ++i)
        for (int c = 0; c < 3; ++c) u[3 * i + c] -= u0[c];
    fs << "      <PointData Vectors=\"displacement\">\n";
    fs << "        <DataArray type=\"Float64\" Name=\"displacement\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    for (long i = 0; i < num_points; ++i) fs << u[3 * i] << " " << u[3 * i + 1] << " " << u[3 * i + 2] << "\n";
    fs << "        </DataArray>\n";
    fs << "      </PointData>\n";
    fs << "      <CellData>\n";
    auto scalar = [&](const char* name, auto get) {
        fs << "        <DataArray type=\"Float64\" Name=\"" << name << "\" format=\"ascii\">\n";
        for (long i = 0; i < num_cells; ++i) fs << get(i) << (i % 10 == 9 || i == num_cells - 1 ? "\n" : " ");
        fs << "        </DataArray>\n";
    };
    scalar("E", [&](long i) { return E[i]; });
    scalar("nu", [&](long i) { return nu[i]; });
    static const int ci[6] = {0, 1, 2, 0, 0, 1}, cj[6] = {0, 1, 2, 1, 2, 2};
    static const char* en[6] = {"eps_xx", "eps_yy", "eps_zz", "eps_xy", "eps_xz", "eps_yz"};
    static const char* sn[6] = {"sig_xx", "sig_yy", "sig_zz", "sig_xy", "sig_xz", "sig_yz"};
    static const char* pn[6] = {"eps_plastic_xx", "eps_plastic_yy", "eps_plastic_zz", "eps_plastic_xy", "eps_plastic_xz", "eps_plastic_yz"};
    for (int c = 0; c < 6; ++c) scalar(en[c], [&](long i) { return eps[i](ci[c], cj[c]); });
    scalar("eps_vm", [&](long i) { return vm(eps[i], 2.0 / 3.0); });
    for (int c = 0; c < 6; ++c) scalar(sn[c], [&](long i) { return sig[i](ci[c], cj[c]); });
    scalar("sig_vm", [&](long i) { return vm(sig[i], 1.5); });
    if (!epsp.empty()) {
        for (int c = 0; c < 6; ++c) scalar(pn[c], [&](long i) { return epsp[i](ci[c], cj[c]); });
        scalar("eps_plastic_vm", [&](long i) { return vm(epsp[i], 2.0 / 3.0); });
    }
    if (soft) {
        scalar("g_p", [&](long i) { return soft[2 * i]; });
        scalar("g_t", [&](long i) { return soft[2 * i + 1]; });
    }
    fs << "      </CellData>\n";
    fs << "      <Points>\n";
    fs << "        <DataArray type=\"Float64\" Name=\"Points\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    for (int i = 0; i <= nx; ++i)
        for (int j = 0; j <= ny; ++j)
            for (int k = 0; k <= nz; ++k) fs << i * pixel << " " << j * pixel << " " << k * pixel << "\n";
    fs << "        </DataArray>\n";
    fs << "      </Points>\n";
    fs << "      <Cells>\n";
    fs << "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n";
    const int NYZ = (ny + 1) * (nz + 1), NZ = nz + 1;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int n0 = i * NYZ + j * NZ + k, n1 = n0 + 1, n2 = n0 + NZ, n3 = n2 + 1, n4 = n0 + NYZ, n5 = n4 + 1, n6 = n4 + NZ, n7 = n6 + 1;
                fs << n0 << " " << n1 << " " << n3 << " " << n2 << " " << n4 << " " << n5 << " " << n7 << " " << n6 << "\n";
            }
    fs << "        </DataArray>\n";
    fs << "        <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n";
    for (long i = 1; i <= num_cells; ++i) fs << i * 8 << (i % 10 == 0 || i == num_cells ? "\n" : " ");
    fs << "        </DataArray>\n";
    fs << "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
    for (long i = 1; i <= num_cells; ++i) fs << 12 << (i % 10 == 0 || i == num_cells ? "\n" : " ");
    fs << "        </DataArray>\n";
    fs << "      </Cells>\n";
    fs << "    </Piece>\n";
    fs << "  </UnstructuredGrid>\n";
    fs << "</VTKFile>\n";
}

}  // namespace mgk
