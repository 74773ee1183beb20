// ORACLE - test infrastructure only (the checker).
//
// A C-ABI shim over the REFERENCE's own library builders, designs and on-axis
// focus checks (src/celeris/design/achromatic.cpp, pb_achromatic.cpp,
// polar_metalens.cpp, pb_metalens.cpp, system_opt.cpp, metalens.cpp,
// analysis/polarization.cpp, focal.cpp), compiled from the sources where they lie by
// oracle/Makefile into oracle/_ref/libref_library.so. The reference's RCWA
// (rcwa2d.cpp) needs Eigen, which is absent, so this file supplies
// celeris::solve_rcwa_2d itself: it forwards every solve to a callback that the
// test registers (the numpy restatement oracle/rcwa.py). The builders' own
// loops, grids, unwrapping, slopes, filters, designs and z scans are the
// reference's code; only the cell solve is the oracle's.
#include <complex>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "celeris/design/achromatic.hpp"
#include "celeris/design/metalens.hpp"
#include "celeris/design/optimize.hpp"
#include "celeris/design/pb_achromatic.hpp"
#include "celeris/design/pb_metalens.hpp"
#include "celeris/design/system_opt.hpp"
#include "celeris/analysis/polarization.hpp"
#include "celeris/design/polar_metalens.hpp"
#include "celeris/rcwa/rcwa2d.hpp"

#define REF_API extern "C" __attribute__((visibility("default")))

using cd = std::complex<double>;

// in: n_inc(2) n_sub(2) px py wl theta phi Ex0(2) Ey0(2) Mx My nl, then per layer
//     eps_pillar(2) eps_bg(2) fill_x fill_y thickness shape shape_param rotation (10)
// out: R T sum_de de_t0 de_r0 tx0(2) ty0(2)
typedef int (*rcwa_callback)(const double* in, int nin, double* out);
static rcwa_callback g_rcwa = nullptr;
static std::mutex g_mu;

REF_API void ref_set_rcwa_callback(rcwa_callback cb) { g_rcwa = cb; }

namespace celeris {
Rcwa2DResult solve_rcwa_2d(const Material& incident, const Rcwa2DStack& stack, const Material& substrate,
                           double wavelength_um, double theta_rad, double phi_rad, cdouble Ex0, cdouble Ey0, int Mx,
                           int My, std::vector<OrderEfficiency>* orders_out) {
    if (!g_rcwa) throw std::runtime_error("no RCWA callback registered");
    if (orders_out) throw std::runtime_error("orders_out is not forwarded");
    const cd ni = incident.index(wavelength_um), ns = substrate.index(wavelength_um);
    std::vector<double> in = {ni.real(), ni.imag(), ns.real(), ns.imag(), stack.period_x_um, stack.period_y_um,
                              wavelength_um, theta_rad, phi_rad, Ex0.real(), Ex0.imag(), Ey0.real(), Ey0.imag(),
                              (double)Mx, (double)My, (double)stack.layers.size()};
    for (const RectCell2D& L : stack.layers) {
        const cd ep = L.pillar.permittivity(wavelength_um), eb = L.background.permittivity(wavelength_um);
        const double v[10] = {ep.real(), ep.imag(), eb.real(), eb.imag(), L.fill_x, L.fill_y, L.thickness_um,
                              (double)static_cast<int>(L.shape), L.shape_param, L.rotation_rad};
        in.insert(in.end(), v, v + 10);
    }
    double out[9] = {0};
    {
        std::lock_guard<std::mutex> lk(g_mu);  // one solve at a time through the callback
        if (g_rcwa(in.data(), static_cast<int>(in.size()), out) != 0) throw std::runtime_error("RCWA callback failed");
    }
    return Rcwa2DResult{out[0], out[1], out[2], out[3], out[4], cd(out[5], out[6]), cd(out[7], out[8])};
}
}  // namespace celeris

namespace {
celeris::Material mat(const double* n) { return celeris::Material::constant(cd(n[0], n[1]), "m"); }
}  // namespace

// Materials are constant indices, each given as (re, im): mats = pillar, background, incident, substrate.
// specs: 5 doubles each (shape, fill_x, fill_y, thickness, shape_param).
// out_atoms: per atom 3 + 2 nb doubles (phase0, group delay, mean amplitude, phase[nb], amplitude[nb]).
// out_meta: center_index, gd_min, gd_max.
REF_API int ref_build_dispersive_library_from_specs(const double* mats, double period_um, const double* band, int nb,
                                                    double center_um, const double* specs, int nspec, int M,
                                                    double* out_atoms, double* out_meta) {
    std::vector<celeris::MetaAtomSpec> sp(nspec);
    for (int i = 0; i < nspec; ++i) {
        const double* s = specs + 5 * i;
        sp[i] = {static_cast<celeris::MetaShape>(static_cast<int>(s[0])), s[1], s[2], s[3], s[4]};
    }
    const auto lib = celeris::build_dispersive_library_from_specs(mat(mats), mat(mats + 2), mat(mats + 4),
                                                                  mat(mats + 6), period_um,
                                                                  std::vector<double>(band, band + nb), center_um,
                                                                  sp, M);
    for (int i = 0; i < nspec; ++i) {
        double* o = out_atoms + (size_t)i * (3 + 2 * nb);
        const auto& a = lib.atoms[i];
        o[0] = a.phase0_rad;
        o[1] = a.group_delay_fs;
        o[2] = a.mean_amplitude;
        for (int j = 0; j < nb; ++j) {
            o[3 + j] = a.phase_rad[j];
            o[3 + nb + j] = a.amplitude[j];
        }
    }
    out_meta[0] = lib.center_index;
    out_meta[1] = lib.gd_min_fs;
    out_meta[2] = lib.gd_max_fs;
    return 0;
}

// Same output layout for the fill x height grid; returns the atom count.
REF_API int ref_build_dispersive_library(const double* mats, double period_um, const double* band, int nb,
                                         double center_um, double fill_min, double fill_max, int n_fills,
                                         double thick_lo, double thick_hi, int n_heights, int M, double* out_atoms,
                                         double* out_meta) {
    const auto lib = celeris::build_dispersive_library(mat(mats), mat(mats + 2), mat(mats + 4), mat(mats + 6),
                                                       period_um, std::vector<double>(band, band + nb), center_um,
                                                       fill_min, fill_max, n_fills, thick_lo, thick_hi, n_heights, M);
    for (size_t i = 0; i < lib.atoms.size(); ++i) {
        double* o = out_atoms + i * (3 + 2 * nb);
        const auto& a = lib.atoms[i];
        o[0] = a.phase0_rad;
        o[1] = a.group_delay_fs;
        o[2] = a.mean_amplitude;
        for (int j = 0; j < nb; ++j) {
            o[3 + j] = a.phase_rad[j];
            o[3 + nb + j] = a.amplitude[j];
        }
    }
    out_meta[0] = lib.center_index;
    out_meta[1] = lib.gd_min_fs;
    out_meta[2] = lib.gd_max_fs;
    return static_cast<int>(lib.atoms.size());
}

// PB library: per kept atom 7 + 2 nb doubles (fill_x, fill_y, phase0, group delay,
// mean amplitude, mean conversion, retardance, cross[nb] as re, im); returns the kept count.
REF_API int ref_build_dispersive_pb_library(const double* mats, double period_um, const double* band, int nb,
                                            double center_um, double fill_min, double fill_max, int n_fills,
                                            double thickness_um, int M, double min_amplitude, double* out_atoms,
                                            double* out_meta) {
    const auto lib = celeris::build_dispersive_pb_library(mat(mats), mat(mats + 2), mat(mats + 4), mat(mats + 6),
                                                          period_um, std::vector<double>(band, band + nb), center_um,
                                                          fill_min, fill_max, n_fills, thickness_um, M,
                                                          min_amplitude);
    for (size_t i = 0; i < lib.atoms.size(); ++i) {
        double* o = out_atoms + i * (7 + 2 * nb);
        const auto& a = lib.atoms[i];
        const double v[7] = {a.fill_x, a.fill_y, a.phase0_rad, a.group_delay_fs, a.mean_amplitude, a.mean_conversion,
                             a.retardance_center_deg};
        for (int k = 0; k < 7; ++k) o[k] = v[k];
        for (int j = 0; j < nb; ++j) {
            o[7 + 2 * j] = a.cross[j].real();
            o[8 + 2 * j] = a.cross[j].imag();
        }
    }
    out_meta[0] = lib.center_index;
    out_meta[1] = lib.gd_min_fs;
    out_meta[2] = lib.gd_max_fs;
    return static_cast<int>(lib.atoms.size());
}

// Polarization library: 6 doubles per cell (fill_x, fill_y, phase_x, phase_y, amp_x, amp_y).
REF_API int ref_build_polarization_library(const double* mats, double period_um, double wavelength_um,
                                           double thickness_um, double fill_min, double fill_max, int n_samples,
                                           int M, double* out) {
    const auto lib = celeris::build_polarization_library(mat(mats), mat(mats + 2), mat(mats + 4), mat(mats + 6),
                                                         period_um, wavelength_um, thickness_um, fill_min, fill_max,
                                                         n_samples, M);
    for (size_t i = 0; i < lib.cells.size(); ++i) {
        const auto& c = lib.cells[i];
        const double v[6] = {c.fill_x, c.fill_y, c.phase_x, c.phase_y, c.amp_x, c.amp_y};
        for (int k = 0; k < 6; ++k) out[6 * i + k] = v[k];
    }
    return static_cast<int>(lib.cells.size());
}

// Stack library: layers as (pillar n(2), background n(2), fill_x, fill_y, thickness, shape, shape_param)
// with constant indices; out: fill, phase, amplitude [n_samples each].
REF_API int ref_build_unit_cell_library_stack(const double* layers, int nl, double px, double py, int active,
                                              const double* n_inc, const double* n_sub, double wavelength_um,
                                              double fill_min, double fill_max, int n_samples, int M, double* fill,
                                              double* phase, double* amp) {
    celeris::Rcwa2DStack st{px, py, {}};
    for (int l = 0; l < nl; ++l) {
        const double* v = layers + 9 * l;
        st.layers.push_back(celeris::RectCell2D{mat(v), mat(v + 2), v[4], v[5], v[6],
                                                static_cast<celeris::MetaShape>(static_cast<int>(v[7])), v[8]});
    }
    const auto lib = celeris::build_unit_cell_library_stack(st, active, mat(n_inc), mat(n_sub), wavelength_um,
                                                            fill_min, fill_max, n_samples, M);
    for (int i = 0; i < n_samples; ++i) {
        fill[i] = lib.fill[i];
        phase[i] = lib.phase[i];
        amp[i] = lib.amplitude[i];
    }
    return 0;
}

// Dispersive library given as arrays (atoms: fill, thickness, phase0, group delay, mean amplitude,
// phase[nb], amplitude[nb] = 5 + 2 nb doubles) -> design_achromatic_metalens, then
// verify_achromatic_focus. out_idx: n_cells^2 atom indices; out_metrics: rms phase, rms gd, mean amp,
// required span, available span, coverage; out_focus: per band (wavelength, focal length, rel_peak).
REF_API int ref_achromatic_design_verify(double period_um, const double* band, int nb, double center_um,
                                         int center_index, double gd_min, double gd_max, const double* atoms,
                                         int natoms, double f_um, double d_um, double gd_weight, double amp_weight,
                                         int* out_idx, double* out_metrics, double* out_focus) {
    celeris::DispersiveLibrary lib;
    lib.wavelengths_um.assign(band, band + nb);
    lib.center_wavelength_um = center_um;
    lib.center_index = center_index;
    lib.period_um = period_um;
    lib.gd_min_fs = gd_min;
    lib.gd_max_fs = gd_max;
    for (int i = 0; i < natoms; ++i) {
        const double* a = atoms + (size_t)i * (5 + 2 * nb);
        celeris::DispersiveAtom at;
        at.fill = at.fill_x = at.fill_y = a[0];
        at.thickness_um = a[1];
        at.phase0_rad = a[2];
        at.group_delay_fs = a[3];
        at.mean_amplitude = a[4];
        at.phase_rad.assign(a + 5, a + 5 + nb);
        at.amplitude.assign(a + 5 + nb, a + 5 + 2 * nb);
        lib.atoms.push_back(at);
    }
    const auto d = celeris::design_achromatic_metalens(lib, f_um, d_um, gd_weight, amp_weight);
    for (size_t i = 0; i < d.atom_index.size(); ++i) out_idx[i] = d.atom_index[i];
    const double m[6] = {d.rms_phase_error_deg, d.rms_group_delay_error_fs, d.mean_amplitude,
                         d.required_gd_span_fs, d.available_gd_span_fs, d.gd_coverage};
    for (int k = 0; k < 6; ++k) out_metrics[k] = m[k];
    const auto fp = celeris::verify_achromatic_focus(lib, d);
    for (size_t j = 0; j < fp.size(); ++j) {
        out_focus[3 * j] = fp[j].wavelength_um;
        out_focus[3 * j + 1] = fp[j].focal_length_um;
        out_focus[3 * j + 2] = fp[j].rel_peak;
    }
    return d.n_cells;
}

// PB library as arrays (atoms: fill_x, fill_y, phase0, group delay, mean amplitude, mean conversion,
// cross[nb] as re, im = 6 + 2 nb doubles) -> design_pb_achromatic_metalens + verify_pb_achromatic_focus.
// out_rot: per-site rotation; out_metrics: rms phase, rms gd, mean amp, mean conversion, coverage.
REF_API int ref_pb_design_verify(double period_um, double thickness_um, const double* band, int nb, double center_um,
                                 int center_index, double gd_min, double gd_max, const double* atoms, int natoms,
                                 double f_um, double d_um, int handedness, double gd_weight, double amp_weight,
                                 int* out_idx, double* out_rot, double* out_metrics, double* out_focus) {
    celeris::DispersivePbLibrary lib;
    lib.wavelengths_um.assign(band, band + nb);
    lib.center_wavelength_um = center_um;
    lib.center_index = center_index;
    lib.period_um = period_um;
    lib.thickness_um = thickness_um;
    lib.gd_min_fs = gd_min;
    lib.gd_max_fs = gd_max;
    for (int i = 0; i < natoms; ++i) {
        const double* a = atoms + (size_t)i * (6 + 2 * nb);
        celeris::DispersivePbAtom at;
        at.fill_x = a[0];
        at.fill_y = a[1];
        at.thickness_um = thickness_um;
        at.phase0_rad = a[2];
        at.group_delay_fs = a[3];
        at.mean_amplitude = a[4];
        at.mean_conversion = a[5];
        for (int j = 0; j < nb; ++j) at.cross.push_back(cd(a[6 + 2 * j], a[7 + 2 * j]));
        lib.atoms.push_back(at);
    }
    const auto d = celeris::design_pb_achromatic_metalens(lib, f_um, d_um, handedness, gd_weight, amp_weight);
    for (size_t i = 0; i < d.atom_index.size(); ++i) {
        out_idx[i] = d.atom_index[i];
        out_rot[i] = d.rotation_rad[i];
    }
    const double m[5] = {d.rms_phase_error_deg, d.rms_group_delay_error_fs, d.mean_amplitude, d.mean_conversion,
                         d.gd_coverage};
    for (int k = 0; k < 5; ++k) out_metrics[k] = m[k];
    const auto fp = celeris::verify_pb_achromatic_focus(lib, d);
    for (size_t j = 0; j < fp.size(); ++j) {
        out_focus[3 * j] = fp[j].wavelength_um;
        out_focus[3 * j + 1] = fp[j].focal_length_um;
        out_focus[3 * j + 2] = fp[j].rel_peak;
    }
    return d.n_cells;
}

// Polarization library as arrays (6 doubles per cell) -> design_polarization_metalens.
// out_fill: n^2 (fill_x, fill_y); out_metrics: rms x, rms y, mean amp x, mean amp y.
REF_API int ref_polarization_design(double period_um, double wavelength_um, const double* cells, int ncells,
                                    double fx_um, double fy_um, double d_um, double amp_weight, double* out_fill,
                                    double* out_metrics) {
    celeris::PolarizationLibrary lib;
    lib.period_um = period_um;
    lib.wavelength_um = wavelength_um;
    for (int i = 0; i < ncells; ++i) {
        const double* c = cells + 6 * i;
        lib.cells.push_back({c[0], c[1], c[2], c[3], c[4], c[5]});
    }
    const auto d = celeris::design_polarization_metalens(lib, fx_um, fy_um, d_um, amp_weight);
    for (size_t i = 0; i < d.fill_x.size(); ++i) {
        out_fill[2 * i] = d.fill_x[i];
        out_fill[2 * i + 1] = d.fill_y[i];
    }
    const double m[4] = {d.rms_phase_error_x_deg, d.rms_phase_error_y_deg, d.mean_amp_x, d.mean_amp_y};
    for (int k = 0; k < 4; ++k) out_metrics[k] = m[k];
    return d.n_cells;
}

// Rectangle cell with constant indices: mats = pillar, background, incident, substrate (re, im each).
// solve_jones: out = xx, xy, yx, yy (re, im each).
REF_API int ref_solve_jones(const double* mats, double period_um, double fill_x, double fill_y, double thickness_um,
                            double rotation_rad, double wavelength_um, int M, double* out) {
    celeris::RectCell2D cell{mat(mats), mat(mats + 2), fill_x, fill_y, thickness_um, celeris::MetaShape::Rectangle,
                             0.5, rotation_rad};
    const celeris::Rcwa2DStack st{period_um, period_um, {cell}};
    const auto J = celeris::solve_jones(mat(mats + 4), st, mat(mats + 6), wavelength_um, M);
    const cd v[4] = {J.xx, J.xy, J.yx, J.yy};
    for (int i = 0; i < 4; ++i) {
        out[2 * i] = v[i].real();
        out[2 * i + 1] = v[i].imag();
    }
    return 0;
}

// find_hwp_atom: out = fill_x, fill_y, thickness, t_x (2), t_y (2), retardance, efficiency.
REF_API int ref_find_hwp_atom(const double* mats, double period_um, double wavelength_um, double thickness_um,
                              double fill_min, double fill_max, int n_samples, int M, double* out) {
    const auto a = celeris::find_hwp_atom(mat(mats), mat(mats + 2), mat(mats + 4), mat(mats + 6), period_um,
                                          wavelength_um, thickness_um, fill_min, fill_max, n_samples, M);
    const double v[9] = {a.fill_x, a.fill_y, a.thickness_um, a.t_x.real(), a.t_x.imag(), a.t_y.real(),
                         a.t_y.imag(), a.retardance_deg, a.conversion_efficiency};
    for (int i = 0; i < 9; ++i) out[i] = v[i];
    return 0;
}

// verify_pb_phase for an atom (fill_x, fill_y, thickness): 4 doubles per rotation.
REF_API int ref_verify_pb_phase(const double* mats, double period_um, double wavelength_um, double fill_x,
                                double fill_y, double thickness_um, const double* rot, int nrot, int M, double* out) {
    celeris::HwpAtom a;
    a.fill_x = fill_x;
    a.fill_y = fill_y;
    a.thickness_um = thickness_um;
    const auto pts = celeris::verify_pb_phase(mat(mats), mat(mats + 2), mat(mats + 4), mat(mats + 6), period_um,
                                              wavelength_um, a, std::vector<double>(rot, rot + nrot), M);
    for (int i = 0; i < nrot; ++i) {
        const double v[4] = {pts[i].rotation_deg, pts[i].cross_phase_deg, pts[i].conversion_eff,
                             pts[i].copol_leakage};
        for (int k = 0; k < 4; ++k) out[4 * i + k] = v[k];
    }
    return 0;
}

// design_pb_metalens (focusing) for an atom given by t_x, t_y: out_rot n^2, out_t n^2 (re, im),
// out_metrics = rms phase error, conversion efficiency; returns n.
REF_API int ref_design_pb_metalens(const double* tx, const double* ty, double period_um, double wavelength_um,
                                   double f_um, double d_um, int handedness, double* out_rot, double* out_t,
                                   double* out_metrics) {
    celeris::HwpAtom a;
    a.t_x = cd(tx[0], tx[1]);
    a.t_y = cd(ty[0], ty[1]);
    const auto d = celeris::design_pb_metalens(a, period_um, wavelength_um, f_um, d_um, handedness);
    for (size_t i = 0; i < d.rotation_rad.size(); ++i) {
        out_rot[i] = d.rotation_rad[i];
        out_t[2 * i] = d.t_cross[i].real();
        out_t[2 * i + 1] = d.t_cross[i].imag();
    }
    out_metrics[0] = d.rms_phase_error_deg;
    out_metrics[1] = d.conversion_efficiency;
    return d.n_cells;
}

// analyze_birefringence: 7 doubles per sample.
REF_API int ref_analyze_birefringence(const double* mats, double period_um, double wavelength_um,
                                      double thickness_um, double fill_y, double fill_min, double fill_max,
                                      int n_samples, int M, double* out) {
    const auto pts = celeris::analyze_birefringence(mat(mats), mat(mats + 2), mat(mats + 4), mat(mats + 6),
                                                    period_um, wavelength_um, thickness_um, fill_y, fill_min,
                                                    fill_max, n_samples, M);
    for (size_t i = 0; i < pts.size(); ++i) {
        const auto& p = pts[i];
        const double v[7] = {p.fill_x, p.fill_y, p.phase_x_deg, p.phase_y_deg, p.retardance_deg, p.tx, p.ty};
        for (int k = 0; k < 7; ++k) out[7 * i + k] = v[k];
    }
    return static_cast<int>(pts.size());
}

// optimize_system: out = period, thickness, strehl, mean amplitude, merit.
REF_API int ref_optimize_system(const double* mats, double f_um, double d_um, double wavelength_um, double p_lo,
                                double p_hi, double t_lo, double t_hi, int grid, int M, int fill_samples,
                                double eff_weight, double* out) {
    const auto r = celeris::optimize_system(mat(mats), mat(mats + 2), mat(mats + 4), mat(mats + 6), f_um, d_um,
                                            wavelength_um, p_lo, p_hi, t_lo, t_hi, grid, M, fill_samples, eff_weight,
                                            nullptr);
    const double v[5] = {r.period_um, r.thickness_um, r.strehl, r.mean_amplitude, r.merit};
    for (int k = 0; k < 5; ++k) out[k] = v[k];
    return 0;
}

// optimize_pillar (optimize.cpp:22-86): the reference's central differences and
// Adam over (fill, thickness), every cell solve forwarded to the oracle.
// mats = pillar, background, incident, substrate (re, im each).
// out: fill, thickness_um, achieved_phase_rad, achieved_amplitude, loss, iterations.
REF_API int ref_optimize_pillar(const double* mats, double period_um, double wavelength_um, double target_phase_rad,
                                double amplitude_weight, int M, double fill0, double thickness0, int max_iters,
                                double* out) {
    const celeris::PillarTarget tgt{wavelength_um, target_phase_rad, amplitude_weight};
    const auto r = celeris::optimize_pillar(mat(mats), mat(mats + 2), mat(mats + 4), mat(mats + 6), period_um, tgt, M,
                                            fill0, thickness0, max_iters);
    out[0] = r.fill;
    out[1] = r.thickness_um;
    out[2] = r.achieved_phase_rad;
    out[3] = r.achieved_amplitude;
    out[4] = r.loss;
    out[5] = r.iterations;
    return 0;
}
