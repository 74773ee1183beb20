// Library builders of the reference that sweep unit cells through solve_rcwa_2d,
// and the designs and on-axis focus checks built on them. Every sweep here is ONE
// batched GPU call (celeris_rcwa_batch / celeris_rcwa_stack_batch): a cell's X and
// Y transmissions come from one eigensolve, where the reference runs one or two
// full solves per (atom, wavelength) on std::async workers.
//
//   build_unit_cell_library_stack   design/metalens.cpp:71-110
//   dispersive libraries            design/achromatic.cpp:54-192 (specs, fill x height, single etch)
//   design_achromatic_metalens      design/achromatic.cpp:194-283
//   verify_achromatic_focus         design/achromatic.cpp:285-339 (200-point on-axis z scans)
//   dispersive PB library           design/pb_achromatic.cpp:47-154
//   design / verify (PB)            design/pb_achromatic.cpp:156-300
//   polarization library / design   design/polar_metalens.cpp:23-121
//   Jones / HWP atom / PB check      design/pb_metalens.cpp:36-104 (rotated atoms in one batch)
//   PB metalens design              design/pb_metalens.cpp:106-151
//   birefringence sweep             analysis/polarization.cpp:23-60
//   system optimisation             design/system_opt.cpp:9-43 (all grid libraries in one batch)
//
// The selection costs, grids and reductions follow the reference's formulas so
// that the libraries and designs are the reference's for the same solver output.
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "celeris.hpp"
#include "detail.hpp"

namespace celeris {
using namespace detail;

namespace {

constexpr double kCUmPerFs = 0.299792458;  // c in um / fs: omega in rad / fs

// Remove 2 pi jumps between consecutive samples (achromatic.cpp:27-35).
void unwrap_phase(std::vector<double>& p) {
    for (size_t i = 1; i < p.size(); ++i) {
        double d = p[i] - p[i - 1];
        while (d > pi) {
            p[i] -= 2.0 * pi;
            d -= 2.0 * pi;
        }
        while (d < -pi) {
            p[i] += 2.0 * pi;
            d += 2.0 * pi;
        }
    }
}

// Least-squares slope of y against x (achromatic.cpp:38-50).
double slope_lsq(const std::vector<double>& x, const std::vector<double>& y) {
    const size_t n = x.size();
    if (n < 2) return 0.0;
    double mx = 0.0, my = 0.0;
    for (size_t i = 0; i < n; ++i) {
        mx += x[i];
        my += y[i];
    }
    mx /= n;
    my /= n;
    double sxy = 0.0, sxx = 0.0;
    for (size_t i = 0; i < n; ++i) {
        sxy += (x[i] - mx) * (y[i] - my);
        sxx += (x[i] - mx) * (x[i] - mx);
    }
    return sxx != 0.0 ? sxy / sxx : 0.0;
}

// Band sample nearest the centre wavelength (first on ties).
int nearest_index(const std::vector<double>& band, double center) {
    int best = 0;
    double bd = std::abs(band[0] - center);
    for (int j = 1; j < static_cast<int>(band.size()); ++j) {
        const double d = std::abs(band[j] - center);
        if (d < bd) {
            bd = d;
            best = j;
        }
    }
    return best;
}

std::vector<double> band_omegas(const std::vector<double>& band) {
    std::vector<double> w(band.size());
    for (size_t j = 0; j < band.size(); ++j) w[j] = 2.0 * pi * kCUmPerFs / band[j];
    return w;
}

double fill_on_grid(double lo, double hi, int i, int n) { return n <= 1 ? lo : lo + (hi - lo) * i / (n - 1); }

// X and Y results of single-layer cells, one batched call.
std::vector<celeris_rcwa_result> solve_batch(const std::vector<celeris_rcwa_cell>& cc, const char* what) {
    std::vector<celeris_rcwa_result> r(2 * cc.size());
    if (!cc.empty()) check(celeris_rcwa_batch(cc.data(), static_cast<int>(cc.size()), r.data(), nullptr), what);
    return r;
}

cdouble tx_of(const celeris_rcwa_result& r) { return cdouble(r.tx0[0], r.tx0[1]); }
cdouble ty_of(const celeris_rcwa_result& r) { return cdouble(r.ty0[0], r.ty0[1]); }

void gd_range(const std::vector<double>& gd, double& lo, double& hi) {
    lo = hi = gd.empty() ? 0.0 : gd[0];
    for (double g : gd) {
        lo = std::min(lo, g);
        hi = std::max(hi, g);
    }
}

// Aperture sites of an n x n design inside the circular stop (achromatic.cpp:293-302).
struct Site {
    double x, y;
    size_t off;
};
std::vector<Site> aperture_sites(int n_cells, double p, double diameter_um) {
    const double c = (n_cells - 1) / 2.0, R = diameter_um / 2.0;
    std::vector<Site> s;
    for (int iy = 0; iy < n_cells; ++iy)
        for (int ix = 0; ix < n_cells; ++ix) {
            const double x = (ix - c) * p, y = (iy - c) * p;
            if (std::sqrt(x * x + y * y) > R) continue;
            s.push_back({x, y, static_cast<size_t>(iy) * n_cells + ix});
        }
    return s;
}

// On-axis |E|^2 at one z and the first maximum of a 200-point scan over
// [0.4 f, 1.8 f] (achromatic.cpp:318-337), both on the GPU far field.
double on_axis_at(const std::vector<Cell>& cells, double z, double k) {
    if (cells.empty()) return 0.0;
    return zx_gpu(cells, 0.0, 0.0, 2, z, z, 2, k)[0];
}
void focus_scan(const std::vector<Cell>& cells, double f, double k, double& best_z, double& best_I) {
    constexpr int NZ = 200;
    const double zlo = 0.4 * f, zhi = 1.8 * f;
    best_z = f;
    best_I = -1.0;
    if (cells.empty()) {
        best_I = 0.0;
        return;
    }
    const std::vector<double> I = zx_gpu(cells, 0.0, 0.0, 2, zlo, zhi, NZ, k);
    for (int q = 0; q < NZ; ++q) {
        const double v = I[static_cast<size_t>(q) * 2];
        if (v > best_I) {
            best_I = v;
            best_z = zlo + (zhi - zlo) * q / (NZ - 1);
        }
    }
}

}  // namespace

// ---- stack library (metalens.cpp:71-110) -------------------------------------------------
UnitCellLibrary build_unit_cell_library_stack(Rcwa2DStack stack, int active_layer, const Material& incident,
                                              const Material& substrate, double wavelength_um, double fill_min,
                                              double fill_max, int n_samples, int M) {
    UnitCellLibrary lib;
    lib.period_um = stack.period_x_um;
    lib.wavelength_um = wavelength_um;
    const int nl = static_cast<int>(stack.layers.size());
    const bool active = active_layer >= 0 && active_layer < nl;
    lib.thickness_um = active ? stack.layers[active_layer].thickness_um : 0.0;
    if (n_samples <= 0) return lib;
    if (nl == 0) throw std::invalid_argument("build_unit_cell_library_stack: stack has no layers");
    std::vector<celeris_rcwa_cell> cc;
    std::vector<int> start(1, 0);
    lib.fill.resize(n_samples);
    for (int i = 0; i < n_samples; ++i) {
        const double f = fill_min + (fill_max - fill_min) * i / (n_samples - 1);
        lib.fill[i] = f;
        for (int l = 0; l < nl; ++l) {
            RectCell2D L = stack.layers[l];
            if (active && l == active_layer) L.fill_x = L.fill_y = f;
            cc.push_back(to_cell(incident, L, substrate, stack.period_x_um, stack.period_y_um, wavelength_um, 0.0,
                                 0.0, M, M, 0, false));
        }
        start.push_back(static_cast<int>(cc.size()));
    }
    std::vector<celeris_rcwa_result> r(2 * static_cast<size_t>(n_samples));
    if (nl == 1)
        check(celeris_rcwa_batch(cc.data(), n_samples, r.data(), nullptr), "build_unit_cell_library_stack");
    else
        check(celeris_rcwa_stack_batch(cc.data(), start.data(), n_samples, r.data(), nullptr),
              "build_unit_cell_library_stack");
    lib.phase.resize(n_samples);
    lib.amplitude.resize(n_samples);
    for (int i = 0; i < n_samples; ++i) {  // X polarization (Ex0 = 1)
        lib.phase[i] = std::arg(tx_of(r[2 * i]));
        lib.amplitude[i] = std::abs(tx_of(r[2 * i]));
    }
    return lib;
}

// ---- dispersive libraries (achromatic.cpp:54-192) ------------------------------------------
DispersiveLibrary build_dispersive_library_from_specs(const Material& pillar, const Material& background,
                                                      const Material& incident, const Material& substrate,
                                                      double period_um, const std::vector<double>& band_wavelengths_um,
                                                      double center_wavelength_um,
                                                      const std::vector<MetaAtomSpec>& specs, int M) {
    if (band_wavelengths_um.empty()) throw std::invalid_argument("build_dispersive_library: empty band");
    DispersiveLibrary lib;
    lib.wavelengths_um = band_wavelengths_um;
    lib.center_wavelength_um = center_wavelength_um;
    lib.period_um = period_um;
    const int nb = static_cast<int>(band_wavelengths_um.size());
    lib.center_index = nearest_index(band_wavelengths_um, center_wavelength_um);
    const std::vector<double> omega = band_omegas(band_wavelengths_um);
    // every (atom, band sample) cell in one batch: cell index = atom * nb + j
    std::vector<celeris_rcwa_cell> cc;
    cc.reserve(specs.size() * nb);
    for (const MetaAtomSpec& s : specs)
        for (int j = 0; j < nb; ++j) {
            RectCell2D L{pillar, background, s.fill_x, s.fill_y, s.thickness_um, s.shape, s.shape_param};
            cc.push_back(to_cell(incident, L, substrate, period_um, period_um, band_wavelengths_um[j], 0.0, 0.0, M,
                                 M, 0, false));
        }
    const std::vector<celeris_rcwa_result> r = solve_batch(cc, "build_dispersive_library");
    lib.atoms.resize(specs.size());
    std::vector<double> gd(specs.size());
    for (size_t a = 0; a < specs.size(); ++a) {
        const MetaAtomSpec& s = specs[a];
        DispersiveAtom& at = lib.atoms[a];
        at.fill = std::max(s.fill_x, s.fill_y);
        at.thickness_um = s.thickness_um;
        at.shape = s.shape;
        at.fill_x = s.fill_x;
        at.fill_y = s.fill_y;
        at.shape_param = s.shape_param;
        at.phase_rad.resize(nb);
        at.amplitude.resize(nb);
        double amp = 0.0;
        for (int j = 0; j < nb; ++j) {
            const cdouble t = tx_of(r[2 * (a * nb + j)]);  // X polarization
            at.phase_rad[j] = std::arg(t);
            at.amplitude[j] = std::abs(t);
            amp += at.amplitude[j];
        }
        at.phase0_rad = at.phase_rad[lib.center_index];
        at.mean_amplitude = amp / nb;
        std::vector<double> ph = at.phase_rad;
        unwrap_phase(ph);
        at.group_delay_fs = slope_lsq(omega, ph);
        gd[a] = at.group_delay_fs;
    }
    gd_range(gd, lib.gd_min_fs, lib.gd_max_fs);
    return lib;
}

DispersiveLibrary build_dispersive_library(const Material& pillar, const Material& background,
                                           const Material& incident, const Material& substrate, double period_um,
                                           const std::vector<double>& band_wavelengths_um,
                                           double center_wavelength_um, double fill_min, double fill_max,
                                           int n_fills, double thick_lo, double thick_hi, int n_heights, int M) {
    const int nh = std::max(1, n_heights);
    std::vector<MetaAtomSpec> specs;
    for (int ih = 0; ih < nh; ++ih) {  // height outer, fill inner (achromatic.cpp:143-150)
        const double h = nh == 1 ? thick_lo : thick_lo + (thick_hi - thick_lo) * ih / (nh - 1);
        for (int i = 0; i < n_fills; ++i) {
            const double f = fill_on_grid(fill_min, fill_max, i, n_fills);
            specs.push_back({MetaShape::Rectangle, f, f, h, 0.5});
        }
    }
    DispersiveLibrary lib = build_dispersive_library_from_specs(pillar, background, incident, substrate, period_um,
                                                                band_wavelengths_um, center_wavelength_um, specs, M);
    lib.n_fill = n_fills;
    lib.n_height = nh;
    return lib;
}

DispersiveLibrary build_single_etch_library(const Material& pillar, const Material& background,
                                            const Material& incident, const Material& substrate, double period_um,
                                            const std::vector<double>& band_wavelengths_um,
                                            double center_wavelength_um, double fill_min, double fill_max,
                                            int n_fills, double thickness_um, int M) {
    // one etch depth; square, circle, three cross arm widths, two ring bores per fill
    std::vector<MetaAtomSpec> specs;
    for (int i = 0; i < n_fills; ++i) {
        const double f = fill_on_grid(fill_min, fill_max, i, n_fills);
        specs.push_back({MetaShape::Rectangle, f, f, thickness_um, 0.5});
        specs.push_back({MetaShape::Ellipse, f, f, thickness_um, 0.5});
        for (double arm : {0.3, 0.5, 0.7}) specs.push_back({MetaShape::Cross, f, f, thickness_um, arm});
        for (double bore : {0.4, 0.6}) specs.push_back({MetaShape::Ring, f, f, thickness_um, bore});
    }
    DispersiveLibrary lib = build_dispersive_library_from_specs(pillar, background, incident, substrate, period_um,
                                                                band_wavelengths_um, center_wavelength_um, specs, M);
    lib.n_fill = n_fills;
    lib.n_height = 1;
    return lib;
}

AchromaticDesign design_achromatic_metalens(const DispersiveLibrary& lib, double focal_length_um,
                                            double diameter_um, double gd_weight, double amplitude_weight) {
    const double p = lib.period_um, f = focal_length_um, R = diameter_um / 2.0;
    const double k0 = 2.0 * pi / lib.center_wavelength_um;
    const int n = std::max(1, static_cast<int>(std::round(diameter_um / p)));
    const double c = (n - 1) / 2.0;
    AchromaticDesign d;
    d.n_cells = n;
    d.period_um = p;
    d.center_wavelength_um = lib.center_wavelength_um;
    d.focal_length_um = f;
    d.diameter_um = diameter_um;
    const size_t nn = static_cast<size_t>(n) * n;
    d.atom_index.resize(nn);
    d.fill_map.resize(nn);
    d.thickness_map.resize(nn);
    // group-delay budget over the aperture, centred in the library's range
    const double span = (std::sqrt(R * R + f * f) - f) / kCUmPerFs;
    const double gd_ref = 0.5 * (lib.gd_min_fs + lib.gd_max_fs) + 0.5 * span;
    // group-delay error -> phase error at the band edge
    double dw_half = 0.0;
    if (lib.wavelengths_um.size() >= 2)
        dw_half = 0.5 * std::abs(2.0 * pi * kCUmPerFs / lib.wavelengths_um.front() -
                                 2.0 * pi * kCUmPerFs / lib.wavelengths_um.back());
    double e_ph = 0.0, e_gd = 0.0, amp = 0.0, hmin = 0.0, hmax = 0.0;
    int cnt = 0;
    for (int iy = 0; iy < n; ++iy)
        for (int ix = 0; ix < n; ++ix) {
            const double x = (ix - c) * p, y = (iy - c) * p, r = std::sqrt(x * x + y * y);
            const double sag = std::sqrt(r * r + f * f) - f;
            const double tgt_ph = -k0 * sag, tgt_gd = -sag / kCUmPerFs + gd_ref;
            int best = 0;
            double best_cost = 1e300;
            for (int q = 0; q < static_cast<int>(lib.atoms.size()); ++q) {
                const DispersiveAtom& a = lib.atoms[q];
                const double dphi = angle_diff(a.phase0_rad, tgt_ph);
                const double dgd = (a.group_delay_fs - tgt_gd) * dw_half;
                const double dam = 1.0 - a.mean_amplitude;
                const double cost = dphi * dphi + gd_weight * dgd * dgd + amplitude_weight * dam * dam;
                if (cost < best_cost) {
                    best_cost = cost;
                    best = q;
                }
            }
            const DispersiveAtom& a = lib.atoms[best];
            const size_t off = static_cast<size_t>(iy) * n + ix;
            d.atom_index[off] = best;
            d.fill_map[off] = a.fill;
            d.thickness_map[off] = a.thickness_um;
            const double ephi = angle_diff(a.phase0_rad, tgt_ph), egd = a.group_delay_fs - tgt_gd;
            e_ph += ephi * ephi;
            e_gd += egd * egd;
            amp += a.mean_amplitude;
            if (cnt == 0) {
                hmin = hmax = a.thickness_um;
            } else {
                hmin = std::min(hmin, a.thickness_um);
                hmax = std::max(hmax, a.thickness_um);
            }
            ++cnt;
        }
    d.rms_phase_error_deg = std::sqrt(e_ph / cnt) * 180.0 / pi;
    d.rms_group_delay_error_fs = std::sqrt(e_gd / cnt);
    d.mean_amplitude = amp / cnt;
    d.required_gd_span_fs = span;
    d.available_gd_span_fs = lib.gd_max_fs - lib.gd_min_fs;
    d.gd_coverage = span > 1e-12 ? d.available_gd_span_fs / span : 1.0;
    d.min_height_um = hmin;
    d.max_height_um = hmax;
    d.single_height = (hmax - hmin) < 1e-9;
    return d;
}

std::vector<AchromaticFocalPoint> verify_achromatic_focus(const DispersiveLibrary& lib,
                                                          const AchromaticDesign& design) {
    const std::vector<Site> sites = aperture_sites(design.n_cells, design.period_um, design.diameter_um);
    auto cells_at = [&](int j) {
        std::vector<Cell> cells;
        cells.reserve(sites.size());
        for (const Site& s : sites) {
            const DispersiveAtom& a = lib.atoms[design.atom_index[s.off]];
            cells.push_back({s.x, s.y, std::polar(a.amplitude[j], a.phase_rad[j])});
        }
        return cells;
    };
    const double peak0 = on_axis_at(cells_at(lib.center_index), design.focal_length_um,
                                    2.0 * pi / lib.center_wavelength_um);
    std::vector<AchromaticFocalPoint> out;
    for (int j = 0; j < static_cast<int>(lib.wavelengths_um.size()); ++j) {
        const double lam = lib.wavelengths_um[j];
        double z, I;
        focus_scan(cells_at(j), design.focal_length_um, 2.0 * pi / lam, z, I);
        out.push_back({lam, z, peak0 > 0 ? I / peak0 : 0.0});
    }
    return out;
}

MetalensDesign to_metalens_design(const AchromaticDesign& d) {
    MetalensDesign m;
    m.n_cells = d.n_cells;
    m.period_um = d.period_um;
    m.fill_map = d.fill_map;
    m.rms_phase_error_deg = d.rms_phase_error_deg;
    m.mean_amplitude = d.mean_amplitude;
    return m;
}

// ---- dispersive Pancharatnam-Berry library (pb_achromatic.cpp:47-154) ------------------------
DispersivePbLibrary build_dispersive_pb_library(const Material& pillar, const Material& background,
                                                const Material& incident, const Material& substrate,
                                                double period_um, const std::vector<double>& band_wavelengths_um,
                                                double center_wavelength_um, double fill_min, double fill_max,
                                                int n_fills, double thickness_um, int M, double min_amplitude) {
    if (band_wavelengths_um.empty()) throw std::invalid_argument("build_dispersive_pb_library: empty band");
    DispersivePbLibrary lib;
    lib.wavelengths_um = band_wavelengths_um;
    lib.center_wavelength_um = center_wavelength_um;
    lib.period_um = period_um;
    lib.thickness_um = thickness_um;
    lib.n_fill = n_fills;
    const int nb = static_cast<int>(band_wavelengths_um.size());
    lib.center_index = nearest_index(band_wavelengths_um, center_wavelength_um);
    const std::vector<double> omega = band_omegas(band_wavelengths_um);
    // (fill_x, fill_y) grid, fill_y outer; both polarizations of a cell from one solve
    const int na = std::max(0, n_fills) * std::max(0, n_fills);
    std::vector<celeris_rcwa_cell> cc;
    cc.reserve(static_cast<size_t>(na) * nb);
    for (int iy = 0; iy < n_fills; ++iy)
        for (int ix = 0; ix < n_fills; ++ix)
            for (int j = 0; j < nb; ++j) {
                RectCell2D L{pillar, background, fill_on_grid(fill_min, fill_max, ix, n_fills),
                             fill_on_grid(fill_min, fill_max, iy, n_fills), thickness_um, MetaShape::Rectangle, 0.5};
                cc.push_back(to_cell(incident, L, substrate, period_um, period_um, band_wavelengths_um[j], 0.0, 0.0,
                                     M, M, 0, false));
            }
    const std::vector<celeris_rcwa_result> r = solve_batch(cc, "build_dispersive_pb_library");
    std::vector<DispersivePbAtom> atoms(na);
    for (int a = 0; a < na; ++a) {
        DispersivePbAtom& at = atoms[a];
        at.fill_x = fill_on_grid(fill_min, fill_max, a % n_fills, n_fills);
        at.fill_y = fill_on_grid(fill_min, fill_max, a / n_fills, n_fills);
        at.thickness_um = thickness_um;
        at.cross.resize(nb);
        std::vector<double> ph(nb);
        double amp = 0.0, conv = 0.0;
        for (int j = 0; j < nb; ++j) {
            const size_t cell = static_cast<size_t>(a) * nb + j;
            const cdouble tx = tx_of(r[2 * cell]), ty = ty_of(r[2 * cell + 1]);  // X: Ex0 = 1; Y: Ey0 = 1
            const cdouble acr = (tx - ty) / 2.0;  // spin-flip amplitude of an axis-aligned rectangle
            at.cross[j] = acr;
            ph[j] = std::arg(acr);
            amp += std::abs(acr);
            conv += std::norm(acr);
            if (j == lib.center_index) at.retardance_center_deg = angle_diff(std::arg(tx), std::arg(ty)) * 180.0 / pi;
        }
        at.phase0_rad = ph[lib.center_index];
        at.mean_amplitude = amp / nb;
        at.mean_conversion = conv / nb;
        unwrap_phase(ph);
        at.group_delay_fs = slope_lsq(omega, ph);
    }
    // drop weakly birefringent atoms, but never all of them
    std::vector<DispersivePbAtom> kept;
    for (const DispersivePbAtom& at : atoms)
        if (at.mean_amplitude >= min_amplitude) kept.push_back(at);
    lib.atoms = kept.empty() ? std::move(atoms) : std::move(kept);
    std::vector<double> gd;
    for (const DispersivePbAtom& at : lib.atoms) gd.push_back(at.group_delay_fs);
    gd_range(gd, lib.gd_min_fs, lib.gd_max_fs);
    return lib;
}

PbAchromaticDesign design_pb_achromatic_metalens(const DispersivePbLibrary& lib, double focal_length_um,
                                                 double diameter_um, int handedness, double gd_weight,
                                                 double amplitude_weight) {
    const double p = lib.period_um, f = focal_length_um, R = diameter_um / 2.0;
    const double k0 = 2.0 * pi / lib.center_wavelength_um;
    const int n = std::max(1, static_cast<int>(std::round(diameter_um / p)));
    const double c = (n - 1) / 2.0;
    handedness = handedness >= 0 ? 1 : -1;
    PbAchromaticDesign d;
    d.n_cells = n;
    d.period_um = p;
    d.thickness_um = lib.thickness_um;
    d.handedness = handedness;
    d.center_wavelength_um = lib.center_wavelength_um;
    d.focal_length_um = f;
    d.diameter_um = diameter_um;
    const size_t nn = static_cast<size_t>(n) * n;
    d.atom_index.resize(nn);
    d.rotation_rad.resize(nn);
    d.fill_x_map.resize(nn);
    d.fill_y_map.resize(nn);
    const double span = (std::sqrt(R * R + f * f) - f) / kCUmPerFs;
    const double gd_ref = 0.5 * (lib.gd_min_fs + lib.gd_max_fs) + 0.5 * span;
    double dw_half = 0.0;
    if (lib.wavelengths_um.size() >= 2)
        dw_half = 0.5 * std::abs(2.0 * pi * kCUmPerFs / lib.wavelengths_um.front() -
                                 2.0 * pi * kCUmPerFs / lib.wavelengths_um.back());
    double e_ph = 0.0, e_gd = 0.0, amp = 0.0, conv = 0.0;
    int cnt = 0;
    for (int iy = 0; iy < n; ++iy)
        for (int ix = 0; ix < n; ++ix) {
            const double x = (ix - c) * p, y = (iy - c) * p, r = std::sqrt(x * x + y * y);
            const double sag = std::sqrt(r * r + f * f) - f;
            const double tgt_ph = -k0 * sag, tgt_gd = -sag / kCUmPerFs + gd_ref;
            // the rotation sets the base phase exactly, so only group delay and conversion are scored
            int best = 0;
            double best_cost = 1e300;
            for (int q = 0; q < static_cast<int>(lib.atoms.size()); ++q) {
                const DispersivePbAtom& a = lib.atoms[q];
                const double dgd = (a.group_delay_fs - tgt_gd) * dw_half;
                const double dam = 1.0 - a.mean_amplitude;
                const double cost = gd_weight * dgd * dgd + amplitude_weight * dam * dam;
                if (cost < best_cost) {
                    best_cost = cost;
                    best = q;
                }
            }
            const DispersivePbAtom& a = lib.atoms[best];
            const double phi_geo = tgt_ph - a.phase0_rad;  // phi_geo = -2 handedness theta
            const size_t off = static_cast<size_t>(iy) * n + ix;
            d.atom_index[off] = best;
            d.rotation_rad[off] = -handedness * phi_geo / 2.0;
            d.fill_x_map[off] = a.fill_x;
            d.fill_y_map[off] = a.fill_y;
            const double ephi = angle_diff(a.phase0_rad + phi_geo, tgt_ph), egd = a.group_delay_fs - tgt_gd;
            e_ph += ephi * ephi;
            e_gd += egd * egd;
            amp += a.mean_amplitude;
            conv += a.mean_conversion;
            ++cnt;
        }
    d.rms_phase_error_deg = std::sqrt(e_ph / cnt) * 180.0 / pi;
    d.rms_group_delay_error_fs = std::sqrt(e_gd / cnt);
    d.mean_amplitude = amp / cnt;
    d.mean_conversion = conv / cnt;
    d.required_gd_span_fs = span;
    d.available_gd_span_fs = lib.gd_max_fs - lib.gd_min_fs;
    d.gd_coverage = span > 1e-12 ? d.available_gd_span_fs / span : 1.0;
    return d;
}

std::vector<AchromaticFocalPoint> verify_pb_achromatic_focus(const DispersivePbLibrary& lib,
                                                             const PbAchromaticDesign& design) {
    const std::vector<Site> sites = aperture_sites(design.n_cells, design.period_um, design.diameter_um);
    auto cells_at = [&](int j) {
        std::vector<Cell> cells;
        cells.reserve(sites.size());
        for (const Site& s : sites) {
            const double phi_geo = -2.0 * design.handedness * design.rotation_rad[s.off];
            cells.push_back({s.x, s.y, lib.atoms[design.atom_index[s.off]].cross[j] * std::polar(1.0, phi_geo)});
        }
        return cells;
    };
    const double peak0 = on_axis_at(cells_at(lib.center_index), design.focal_length_um,
                                    2.0 * pi / lib.center_wavelength_um);
    std::vector<AchromaticFocalPoint> out;
    for (int j = 0; j < static_cast<int>(lib.wavelengths_um.size()); ++j) {
        const double lam = lib.wavelengths_um[j];
        double z, I;
        focus_scan(cells_at(j), design.focal_length_um, 2.0 * pi / lam, z, I);
        out.push_back({lam, z, peak0 > 0 ? I / peak0 : 0.0});
    }
    return out;
}

// ---- polarization library and design (polar_metalens.cpp:23-121) ---------------------------
int PolarizationLibrary::lookup(double target_x, double target_y, double amplitude_weight) const {
    int best = 0;
    double best_cost = 1e300;
    for (int i = 0; i < static_cast<int>(cells.size()); ++i) {
        const PolarCell& c = cells[i];
        const double dx = angle_diff(c.phase_x, target_x), dy = angle_diff(c.phase_y, target_y);
        const double ax = 1.0 - c.amp_x, ay = 1.0 - c.amp_y;
        const double cost = dx * dx + dy * dy + amplitude_weight * (ax * ax + ay * ay);
        if (cost < best_cost) {
            best_cost = cost;
            best = i;
        }
    }
    return best;
}

PolarizationLibrary build_polarization_library(const Material& pillar, const Material& background,
                                               const Material& incident, const Material& substrate,
                                               double period_um, double wavelength_um, double thickness_um,
                                               double fill_min, double fill_max, int n_samples, int M) {
    PolarizationLibrary lib;
    lib.period_um = period_um;
    lib.wavelength_um = wavelength_um;
    lib.thickness_um = thickness_um;
    const int total = std::max(0, n_samples) * std::max(0, n_samples);
    std::vector<celeris_rcwa_cell> cc(total);
    lib.cells.resize(total);
    for (int i = 0; i < total; ++i) {  // i = iy * n + ix
        const double fx = fill_min + (fill_max - fill_min) * (i % n_samples) / (n_samples - 1);
        const double fy = fill_min + (fill_max - fill_min) * (i / n_samples) / (n_samples - 1);
        lib.cells[i].fill_x = fx;
        lib.cells[i].fill_y = fy;
        RectCell2D L{pillar, background, fx, fy, thickness_um};
        cc[i] = to_cell(incident, L, substrate, period_um, period_um, wavelength_um, 0.0, 0.0, M, M, 0, false);
    }
    const std::vector<celeris_rcwa_result> r = solve_batch(cc, "build_polarization_library");
    for (int i = 0; i < total; ++i) {
        const cdouble tx = tx_of(r[2 * i]), ty = ty_of(r[2 * i + 1]);
        PolarCell& c = lib.cells[i];
        c.phase_x = std::arg(tx);
        c.phase_y = std::arg(ty);
        c.amp_x = std::abs(tx);
        c.amp_y = std::abs(ty);
    }
    return lib;
}

PolarMetalensDesign design_polarization_metalens(const PolarizationLibrary& lib, double focal_x_um,
                                                 double focal_y_um, double diameter_um, double amplitude_weight) {
    const double p = lib.period_um, lam = lib.wavelength_um;
    const int n = std::max(1, static_cast<int>(std::round(diameter_um / p)));
    const double c = (n - 1) / 2.0;
    PolarMetalensDesign d;
    d.n_cells = n;
    d.period_um = p;
    const size_t nn = static_cast<size_t>(n) * n;
    d.fill_x.resize(nn);
    d.fill_y.resize(nn);
    d.t_x.resize(nn);
    d.t_y.resize(nn);
    auto hyperbolic = [&](double r, double f) { return -(2.0 * pi / lam) * (std::sqrt(r * r + f * f) - f); };
    double ex2 = 0.0, ey2 = 0.0, ax = 0.0, ay = 0.0;
    int cnt = 0;
    for (int iy = 0; iy < n; ++iy)
        for (int ix = 0; ix < n; ++ix) {
            const double x = (ix - c) * p, y = (iy - c) * p, r = std::sqrt(x * x + y * y);
            const double tx = hyperbolic(r, focal_x_um), ty = hyperbolic(r, focal_y_um);
            const PolarCell& pc = lib.cells[lib.lookup(tx, ty, amplitude_weight)];
            const size_t off = static_cast<size_t>(iy) * n + ix;
            d.fill_x[off] = pc.fill_x;
            d.fill_y[off] = pc.fill_y;
            d.t_x[off] = std::polar(pc.amp_x, pc.phase_x);
            d.t_y[off] = std::polar(pc.amp_y, pc.phase_y);
            const double ex = angle_diff(pc.phase_x, tx), ey = angle_diff(pc.phase_y, ty);
            ex2 += ex * ex;
            ey2 += ey * ey;
            ax += pc.amp_x;
            ay += pc.amp_y;
            ++cnt;
        }
    if (cnt) {
        d.rms_phase_error_x_deg = std::sqrt(ex2 / cnt) * 180.0 / pi;
        d.rms_phase_error_y_deg = std::sqrt(ey2 / cnt) * 180.0 / pi;
        d.mean_amp_x = ax / cnt;
        d.mean_amp_y = ay / cnt;
    }
    return d;
}

// ---- Jones matrices and the Pancharatnam-Berry metalens (pb_metalens.cpp) -----------------
namespace {
double wrap_angle(double a) {
    while (a > pi) a -= 2.0 * pi;
    while (a <= -pi) a += 2.0 * pi;
    return a;
}
// (co, cross) circular amplitudes of J applied to right-circular input
// (pb_metalens.cpp:19-33): e_R = (x - i y)/sqrt2, e_L = (x + i y)/sqrt2.
void circular_parts(const JonesMatrix& J, cdouble& co, cdouble& cross) {
    const cdouble I(0.0, 1.0);
    const double r = 1.0 / std::sqrt(2.0);
    const cdouble ex = (J.xx - I * J.xy) * r, ey = (J.yx - I * J.yy) * r;
    co = (ex + I * ey) * r;
    cross = (ex - I * ey) * r;
}
// Columns of the Jones matrix: X (Ex0 = 1) and Y (Ey0 = 1) results of one solve.
JonesMatrix jones_of(const celeris_rcwa_result& rx, const celeris_rcwa_result& ry) {
    return {tx_of(rx), tx_of(ry), ty_of(rx), ty_of(ry)};
}
}  // namespace

JonesMatrix solve_jones(const Material& incident, const Rcwa2DStack& stack, const Material& substrate,
                        double wavelength_um, int M) {
    if (stack.layers.empty()) throw std::invalid_argument("solve_jones: stack has no layers");
    std::vector<celeris_rcwa_cell> cc;
    for (const RectCell2D& L : stack.layers)
        cc.push_back(to_cell(incident, L, substrate, stack.period_x_um, stack.period_y_um, wavelength_um, 0.0, 0.0,
                             M, M, 0, false));
    std::vector<celeris_rcwa_result> r(2);
    if (cc.size() == 1) {
        check(celeris_rcwa_batch(cc.data(), 1, r.data(), nullptr), "solve_jones");
    } else {
        const int start[2] = {0, static_cast<int>(cc.size())};
        check(celeris_rcwa_stack_batch(cc.data(), start, 1, r.data(), nullptr), "solve_jones");
    }
    return jones_of(r[0], r[1]);
}

HwpAtom find_hwp_atom(const Material& pillar, const Material& background, const Material& incident,
                      const Material& substrate, double period_um, double wavelength_um, double thickness_um,
                      double fill_min, double fill_max, int n_samples, int M) {
    const PolarizationLibrary lib = build_polarization_library(pillar, background, incident, substrate, period_um,
                                                               wavelength_um, thickness_um, fill_min, fill_max,
                                                               n_samples, M);
    HwpAtom best;
    double best_eff = -1.0;
    for (const PolarCell& c : lib.cells) {
        const cdouble tx = std::polar(c.amp_x, c.phase_x), ty = std::polar(c.amp_y, c.phase_y);
        const double eff = std::norm(tx - ty) / 4.0;  // spin-flip conversion |t_x - t_y|^2 / 4
        if (eff > best_eff) {
            best_eff = eff;
            best.fill_x = c.fill_x;
            best.fill_y = c.fill_y;
            best.thickness_um = thickness_um;
            best.t_x = tx;
            best.t_y = ty;
            best.retardance_deg = wrap_angle(c.phase_x - c.phase_y) * 180.0 / pi;
            best.conversion_efficiency = eff;
        }
    }
    return best;
}

std::vector<PbVerifyPoint> verify_pb_phase(const Material& pillar, const Material& background,
                                           const Material& incident, const Material& substrate, double period_um,
                                           double wavelength_um, const HwpAtom& atom,
                                           const std::vector<double>& rotations_rad, int M) {
    std::vector<celeris_rcwa_cell> cc;
    for (double rot : rotations_rad) {
        RectCell2D L{pillar, background, atom.fill_x, atom.fill_y, atom.thickness_um, MetaShape::Rectangle, 0.5,
                     rot};
        cc.push_back(to_cell(incident, L, substrate, period_um, period_um, wavelength_um, 0.0, 0.0, M, M, 0, false));
    }
    const std::vector<celeris_rcwa_result> r = solve_batch(cc, "verify_pb_phase");
    std::vector<PbVerifyPoint> out(rotations_rad.size());
    for (size_t i = 0; i < rotations_rad.size(); ++i) {
        cdouble co, cross;
        circular_parts(jones_of(r[2 * i], r[2 * i + 1]), co, cross);
        out[i] = {rotations_rad[i] * 180.0 / pi, std::arg(cross) * 180.0 / pi, std::norm(cross), std::norm(co)};
    }
    return out;
}

PbMetalensDesign design_pb_metalens(const HwpAtom& atom, double period_um, double wavelength_um,
                                    const PhaseProfile& profile, double diameter_um, int handedness) {
    const int n = std::max(1, static_cast<int>(std::round(diameter_um / period_um)));
    const double c = (n - 1) / 2.0;
    PbMetalensDesign d;
    d.n_cells = n;
    d.period_um = period_um;
    d.atom = atom;
    const size_t nn = static_cast<size_t>(n) * n;
    d.rotation_rad.resize(nn);
    d.t_cross.resize(nn);
    // geometric phase on the cross output: -2 handedness theta; the atom's own
    // spin-flip amplitude is a global piston
    const cdouble a0 = (atom.t_x - atom.t_y) / 2.0;
    const double piston = std::arg(a0);
    double e2 = 0.0;
    int cnt = 0;
    for (int iy = 0; iy < n; ++iy)
        for (int ix = 0; ix < n; ++ix) {
            const double x = (ix - c) * period_um, y = (iy - c) * period_um;
            const double phi = phase_profile_value(profile, x, y, wavelength_um);
            const size_t off = static_cast<size_t>(iy) * n + ix;
            d.rotation_rad[off] = -handedness * phi / 2.0;
            d.t_cross[off] = a0 * std::polar(1.0, phi);
            const double err = wrap_angle(std::arg(d.t_cross[off]) - phi - piston);
            e2 += err * err;
            ++cnt;
        }
    if (cnt) d.rms_phase_error_deg = std::sqrt(e2 / cnt) * 180.0 / pi;
    d.conversion_efficiency = std::norm(a0);
    return d;
}

PbMetalensDesign design_pb_metalens(const HwpAtom& atom, double period_um, double wavelength_um,
                                    double focal_length_um, double diameter_um, int handedness) {
    PhaseProfile p;
    p.kind = PhaseProfileKind::Focusing;
    p.focal_length_um = focal_length_um;
    return design_pb_metalens(atom, period_um, wavelength_um, p, diameter_um, handedness);
}

// ---- birefringence sweep (analysis/polarization.cpp) ------------------------------------------
std::vector<BirefringencePoint> analyze_birefringence(const Material& pillar, const Material& background,
                                                      const Material& incident, const Material& substrate,
                                                      double period_um, double wavelength_um, double thickness_um,
                                                      double fill_y, double fill_min, double fill_max,
                                                      int n_samples, int M) {
    const int ns = std::max(0, n_samples);
    std::vector<celeris_rcwa_cell> cc(ns);
    std::vector<double> fx(ns);
    for (int i = 0; i < ns; ++i) {
        fx[i] = fill_min + (fill_max - fill_min) * i / (n_samples - 1);
        RectCell2D L{pillar, background, fx[i], fill_y, thickness_um};
        cc[i] = to_cell(incident, L, substrate, period_um, period_um, wavelength_um, 0.0, 0.0, M, M, 0, false);
    }
    const std::vector<celeris_rcwa_result> r = solve_batch(cc, "analyze_birefringence");
    auto deg = [](double a) { return wrap_angle(a) * 180.0 / pi; };
    std::vector<BirefringencePoint> out(ns);
    for (int i = 0; i < ns; ++i) {
        const cdouble tx = tx_of(r[2 * i]), ty = ty_of(r[2 * i + 1]);  // co-pol of X and of Y input
        out[i] = {fx[i], fill_y, deg(std::arg(tx)), deg(std::arg(ty)), deg(std::arg(tx) - std::arg(ty)),
                  std::abs(tx), std::abs(ty)};
    }
    return out;
}

// ---- period x thickness system optimisation (design/system_opt.cpp) ---------------------------
SystemOptResult optimize_system(const Material& pillar, const Material& background, const Material& incident,
                                const Material& substrate, double focal_um, double diameter_um,
                                double wavelength_um, double period_lo, double period_hi, double thick_lo,
                                double thick_hi, int grid, int M, int fill_samples, double efficiency_weight,
                                const std::function<void(float)>& progress) {
    grid = std::max(2, grid);
    const int nf = std::max(0, fill_samples);
    // every grid point's library sweep (fill 0.08 .. 0.92) in one batched call
    std::vector<celeris_rcwa_cell> cc;
    cc.reserve(static_cast<size_t>(grid) * grid * nf);
    auto period_at = [&](int ip) { return period_lo + (period_hi - period_lo) * ip / (grid - 1); };
    auto thick_at = [&](int it) { return thick_lo + (thick_hi - thick_lo) * it / (grid - 1); };
    for (int ip = 0; ip < grid; ++ip)
        for (int it = 0; it < grid; ++it)
            for (int i = 0; i < nf; ++i) {
                const double f = 0.08 + (0.92 - 0.08) * i / (nf - 1);
                RectCell2D L{pillar, background, f, f, thick_at(it), MetaShape::Rectangle, 0.5};
                cc.push_back(to_cell(incident, L, substrate, period_at(ip), period_at(ip), wavelength_um, 0.0, 0.0,
                                     M, M, 0, false));
            }
    const std::vector<celeris_rcwa_result> r = solve_batch(cc, "optimize_system");
    SystemOptResult best{period_lo, thick_lo, 0, 0, -1};
    int done = 0, k = 0;
    for (int ip = 0; ip < grid; ++ip)
        for (int it = 0; it < grid; ++it) {
            UnitCellLibrary lib;
            lib.period_um = period_at(ip);
            lib.wavelength_um = wavelength_um;
            lib.thickness_um = thick_at(it);
            for (int i = 0; i < nf; ++i, ++k) {
                const cdouble t = tx_of(r[2 * static_cast<size_t>(k)]);
                lib.fill.push_back(0.08 + (0.92 - 0.08) * i / (nf - 1));
                lib.phase.push_back(std::arg(t));
                lib.amplitude.push_back(std::abs(t));
            }
            const MetalensDesign lens = design_metalens(lib, focal_um, diameter_um);
            const FocalAnalysis foc = analyze_focus(lens, lib, focal_um, wavelength_um, diameter_um);
            const double merit = foc.strehl + efficiency_weight * lens.mean_amplitude;
            if (merit > best.merit) best = {lib.period_um, lib.thickness_um, foc.strehl, lens.mean_amplitude, merit};
            if (progress) progress(static_cast<float>(++done) / (grid * grid));
        }
    return best;
}

}  // namespace celeris
