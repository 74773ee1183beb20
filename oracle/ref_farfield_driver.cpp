// ORACLE - test infrastructure only (the checker and the timed CPU baseline).
//
// A C-ABI shim over the REFERENCE's own CPU far-field and its callers, compiled
// together with the reference sources where they lie (src/celeris/analysis/
// focal.cpp, field.cpp, throughfocus.cpp, design/metalens.cpp,
// design/phase_profile.cpp, materials/material.cpp) by oracle/Makefile into
// oracle/_ref/libref_farfield.so. No reference source is copied into this
// repository. Built without CELERIS_USE_CUDA_KERNELS, so celeris::
// propagate_pillars runs its FP64 std::async row loop (focal.cpp:205-238) on all
// host threads, and the field / through-focus analyses take their CPU loops.
#include <complex>
#include <thread>
#include <vector>

#include "celeris/analysis/chromatic.hpp"
#include "celeris/analysis/field.hpp"
#include "celeris/analysis/tolerance.hpp"
#include "celeris/analysis/focal.hpp"
#include "celeris/analysis/throughfocus.hpp"

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

// ---- the reference's analyses on a lens given as plain arrays -----------------------
namespace {
celeris::MetalensDesign make_lens(int n_cells, double period_um, const double* fill_map) {
    celeris::MetalensDesign d{};
    d.n_cells = n_cells;
    d.period_um = period_um;
    d.fill_map.assign(fill_map, fill_map + static_cast<size_t>(n_cells) * n_cells);
    return d;
}
celeris::UnitCellLibrary make_lib(double period_um, double wavelength_um, double thickness_um, int nlib,
                                  const double* fill, const double* phase, const double* amp) {
    celeris::UnitCellLibrary l{};
    l.period_um = period_um;
    l.wavelength_um = wavelength_um;
    l.thickness_um = thickness_um;
    l.fill.assign(fill, fill + nlib);
    l.phase.assign(phase, phase + nlib);
    l.amplitude.assign(amp, amp + nlib);
    return l;
}
}  // namespace

// throughfocus.cpp: z_out[161], I_out[161] (normalized), scal = {z_peak, dof}.
REF_API int ref_through_focus(int n_cells, double period_um, const double* fill_map, int nlib, const double* lfill,
                              const double* lphase, const double* lamp, double lib_wl, double f, double wl, double D,
                              float* z_out, float* I_out, double* scal) {
    const auto lens = make_lens(n_cells, period_um, fill_map);
    const auto lib = make_lib(period_um, lib_wl, 0.0, nlib, lfill, lphase, lamp);
    const celeris::ThroughFocus tf = celeris::analyze_through_focus(lens, lib, f, wl, D);
    for (size_t i = 0; i < tf.z_um.size(); ++i) {
        z_out[i] = tf.z_um[i];
        I_out[i] = tf.intensity[i];
    }
    scal[0] = tf.z_peak_um;
    scal[1] = tf.dof_um;
    return static_cast<int>(tf.z_um.size());
}

// field.cpp analyze_field_of_view: out[3 * nang] = {angle, rel_strehl, spot_shift}.
REF_API int ref_field_of_view(int n_cells, double period_um, const double* fill_map, int nlib, const double* lfill,
                              const double* lphase, const double* lamp, double lib_wl, double f, double wl, double D,
                              const double* angles, int nang, double* out) {
    const auto lens = make_lens(n_cells, period_um, fill_map);
    const auto lib = make_lib(period_um, lib_wl, 0.0, nlib, lfill, lphase, lamp);
    const auto pts = celeris::analyze_field_of_view(lens, lib, f, wl, D, std::vector<double>(angles, angles + nang));
    for (size_t i = 0; i < pts.size(); ++i) {
        out[3 * i] = pts[i].angle_deg;
        out[3 * i + 1] = pts[i].rel_strehl;
        out[3 * i + 2] = pts[i].spot_shift_um;
    }
    return static_cast<int>(pts.size());
}

// field.cpp analyze_wide_fov: out[3 * nang].
REF_API int ref_wide_fov(int n_cells, double period_um, const double* fill_map, int nlib, const double* lfill,
                         const double* lphase, const double* lamp, double lib_wl, double f, double wl, double D_lens,
                         double D_stop, double stop_dist, const double* angles, int nang, double* out) {
    const auto lens = make_lens(n_cells, period_um, fill_map);
    const auto lib = make_lib(period_um, lib_wl, 0.0, nlib, lfill, lphase, lamp);
    const auto pts = celeris::analyze_wide_fov(lens, lib, f, wl, D_lens, D_stop, stop_dist,
                                               std::vector<double>(angles, angles + nang));
    for (size_t i = 0; i < pts.size(); ++i) {
        out[3 * i] = pts[i].angle_deg;
        out[3 * i + 1] = pts[i].rel_strehl;
        out[3 * i + 2] = pts[i].spot_shift_um;
    }
    return static_cast<int>(pts.size());
}

// field.cpp analyze_field_grid: out[7 * n * n] = {tx, ty, rel_strehl, fwhm_x, fwhm_y, cx, cy} row-major.
REF_API int ref_field_grid(int n_cells, double period_um, const double* fill_map, int nlib, const double* lfill,
                           const double* lphase, const double* lamp, double lib_wl, double f, double wl, double D,
                           double max_angle_deg, int n_half, int psf_n, double* out) {
    const auto lens = make_lens(n_cells, period_um, fill_map);
    const auto lib = make_lib(period_um, lib_wl, 0.0, nlib, lfill, lphase, lamp);
    const celeris::FieldGrid g = celeris::analyze_field_grid(lens, lib, f, wl, D, max_angle_deg, n_half, psf_n);
    for (size_t i = 0; i < g.points.size(); ++i) {
        const auto& p = g.points[i];
        const double v[7] = {p.theta_x_deg, p.theta_y_deg, p.rel_strehl, p.fwhm_x_um, p.fwhm_y_um, p.cx_um, p.cy_um};
        for (int q = 0; q < 7; ++q) out[7 * i + q] = v[q];
    }
    return static_cast<int>(g.points.size());
}

// celeris::analyze_chromatic (chromatic.cpp, CPU): per wavelength (lambda, z of the
// on-axis peak, peak relative to the design point); returns the count.
REF_API int ref_chromatic(int n_cells, double period_um, const double* fill_map, int nlib, const double* lfill,
                          const double* lphase, const double* lamp, double lib_wl, double f, double wl, double D,
                          double lam_min, double lam_max, int n, double* out) {
    const auto lens = make_lens(n_cells, period_um, fill_map);
    const auto lib = make_lib(period_um, lib_wl, 0.0, nlib, lfill, lphase, lamp);
    const auto pts = celeris::analyze_chromatic(lens, lib, f, wl, D, lam_min, lam_max, n);
    for (size_t i = 0; i < pts.size(); ++i) {
        out[3 * i] = pts[i].wavelength_um;
        out[3 * i + 1] = pts[i].focal_length_um;
        out[3 * i + 2] = pts[i].rel_peak;
    }
    return static_cast<int>(pts.size());
}

// celeris::analyze_tolerance (tolerance.cpp, CPU): rows (sigma, mean, std, worst Strehl).
REF_API int ref_tolerance(int n_cells, double period_um, const double* fill_map, int nlib, const double* lfill,
                          const double* lphase, const double* lamp, double lib_wl, double f, double wl, double D,
                          const double* sigmas, int nsig, int trials, unsigned seed, double* out) {
    const auto lens = make_lens(n_cells, period_um, fill_map);
    const auto lib = make_lib(period_um, lib_wl, 0.0, nlib, lfill, lphase, lamp);
    const auto r = celeris::analyze_tolerance(lens, lib, f, wl, D, std::vector<double>(sigmas, sigmas + nsig),
                                              trials, seed);
    for (size_t i = 0; i < r.size(); ++i) {
        out[4 * i] = r[i].sigma_nm;
        out[4 * i + 1] = r[i].mean_strehl;
        out[4 * i + 2] = r[i].std_strehl;
        out[4 * i + 3] = r[i].worst_strehl;
    }
    return static_cast<int>(r.size());
}
