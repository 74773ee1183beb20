// Helpers shared by the host-mirror translation units: the C-ABI status check,
// the conversion of a reference unit cell to the C-ABI descriptor, and the
// far-field sums on the GPU (plain FP64 form) for lists of aperture cells.
#pragma once
#include <vector>

#include "celeris.hpp"
#include "celeris_b200.h"

namespace celeris {
namespace detail {

// Throws std::invalid_argument for CELERIS_ERR_INVALID_ARG, std::runtime_error otherwise.
void check(int status, const char* what);
// Smallest signed difference of two angles, in (-pi, pi].
double angle_diff(double a, double b);
celeris_rcwa_cell to_cell(const Material& incident, const RectCell2D& L, const Material& substrate, double px,
                          double py, double wl, double theta, double phi, int Mx, int My, int grid,
                          bool force_laurent);
Rcwa2DResult from_result(const celeris_rcwa_result& r);

struct Cell {
    double x, y;
    cdouble t;
};
// |E|^2 on the n x n grid centred at (cx, cy), half-width W, plane z.
std::vector<double> psf_gpu(const std::vector<Cell>& cells, double cx, double cy, double z, double k, int n,
                            double W);
// |E|^2 on an x-z slice (y = 0): row = z, column = x.
std::vector<double> zx_gpu(const std::vector<Cell>& cells, double xmin, double xmax, int nx, double zmin,
                           double zmax, int nz, double k);

}  // namespace detail
}  // namespace celeris
