// ORACLE - test infrastructure only (the checker and the timed CPU baseline).
//
// A C-ABI shim over the REFERENCE's own CPU far-field, compiled together with
// the reference sources where they lie (src/celeris/analysis/focal.cpp,
// design/metalens.cpp, design/phase_profile.cpp, materials/material.cpp) by
// oracle/Makefile into oracle/_ref/libref_farfield.so. No reference source is
// copied into this repository. Built without CELERIS_USE_CUDA_KERNELS, so
// celeris::propagate_pillars runs its FP64 std::async row loop
// (focal.cpp:205-238) on all host threads.
#include <complex>
#include <thread>
#include <vector>

#include "celeris/analysis/focal.hpp"

#define REF_API extern "C" __attribute__((visibility("default")))

// |E|^2 on the n x n grid via celeris::propagate_pillars (focal.hpp:52-56).
REF_API int ref_propagate_pillars(const double* px, const double* py, const double* pt, int npil,
                                  double cx, double cy, double z, double wavelength_um, int n,
                                  double half_window_um, double* out) {
    std::vector<double> X(px, px + npil), Y(py, py + npil);
    std::vector<std::complex<double>> T(static_cast<size_t>(npil));
    for (int i = 0; i < npil; ++i) T[i] = std::complex<double>(pt[2 * i], pt[2 * i + 1]);
    celeris::PsfMap m = celeris::propagate_pillars(X, Y, T, cx, cy, z, wavelength_um, n, half_window_um);
    for (size_t i = 0; i < m.intensity.size(); ++i) out[i] = m.intensity[i];
    return static_cast<int>(m.intensity.size());
}

// Host threads the reference's parallel_rows uses (focal.cpp:21).
REF_API int ref_hardware_threads() {
    unsigned hw = std::thread::hardware_concurrency();
    return hw == 0 ? 1 : static_cast<int>(hw);
}
