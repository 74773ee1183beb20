// C++ host mirror of the reference's celeris:: interface for the hot path.
//
// Same names, argument meaning and error behaviour as the reference headers
// (src/celeris/core.hpp, materials/material.hpp, rcwa/rcwa2d.hpp,
// design/metalens.hpp, design/phase_profile.hpp, design/optimize.hpp,
// analysis/focal.hpp, cuda/propagate.hpp), so a caller switches by relinking.
// Every far-field and RCWA evaluation goes through the C ABI in
// include/celeris_b200.h (sm_100a kernels); there is no CPU fallback, and a
// non-zero status becomes std::runtime_error (std::invalid_argument where the
// reference throws it).
#pragma once

#include <array>
#include <complex>
#include <functional>
#include <string>
#include <vector>

namespace celeris {

using cdouble = std::complex<double>;
inline constexpr double pi = 3.14159265358979323846;
enum class Pol { TE, TM };

// ---- materials (material.hpp:19-66) -------------------------------------------
class Material {
public:
    Material(std::function<cdouble(double)> dispersion, std::string name);
    cdouble index(double wavelength_um) const { return dispersion_(wavelength_um); }
    cdouble permittivity(double wavelength_um) const {
        const cdouble n = index(wavelength_um);
        return n * n;
    }
    const std::string& name() const { return name_; }
    static Material constant(cdouble n, std::string name = "constant");
    static Material sellmeier(std::vector<std::array<double, 2>> bc_terms, std::string name = "sellmeier");
    static Material sellmeier_ri_formula1(std::vector<double> coeffs, std::string name = "formula1");
    static Material tabulated(std::vector<double> wavelength_um, std::vector<double> n, std::vector<double> k,
                              std::string name = "tabulated");

private:
    std::function<cdouble(double)> dispersion_;
    std::string name_;
};

namespace materials {
const Material& air();
const Material& bk7();
const Material& fused_silica();
const Material& silicon_nitride();
}  // namespace materials

// ---- 2D RCWA (rcwa2d.hpp:26-124) ------------------------------------------------
enum class MetaShape { Rectangle, Ellipse, Cross, Ring };

struct RectCell2D {
    Material pillar;
    Material background;
    double fill_x;
    double fill_y;
    double thickness_um;
    MetaShape shape = MetaShape::Rectangle;
    double shape_param = 0.5;
    double rotation_rad = 0.0;
    bool is_plain_rect() const { return shape == MetaShape::Rectangle && rotation_rad == 0.0; }
    static RectCell2D homogeneous(Material m, double thickness_um) {
        return RectCell2D{m, m, 1.0, 1.0, thickness_um, MetaShape::Rectangle, 0.5};
    }
};

struct Rcwa2DStack {
    double period_x_um;
    double period_y_um;
    std::vector<RectCell2D> layers;
};

struct Rcwa2DResult {
    double R, T, sum_de, de_t0, de_r0;
    cdouble tx0, ty0;
};

struct OrderEfficiency {
    int p, q;
    double de_t;
    double de_r;
    bool prop_t;
    bool prop_r;
};

// eig.hpp:25 with plain containers: A (n x n, column-major) -> eigenvalues and
// unit-norm right eigenvectors (column-major), on the GPU eigen-stages.
void eig_general(const std::vector<cdouble>& A, int n, std::vector<cdouble>& evals, std::vector<cdouble>& evecs);

// Patterned layers between the incident and substrate half-spaces; layers[0]
// is next to the incident side (rcwa2d.cpp:361-364). orders_out (optional)
// receives every order's efficiencies (rcwa2d.cpp:464-485).
Rcwa2DResult solve_rcwa_2d(const Material& incident, const Rcwa2DStack& stack, const Material& substrate,
                           double wavelength_um, double theta_rad, double phi_rad, cdouble Ex0, cdouble Ey0,
                           int Mx, int My, std::vector<OrderEfficiency>* orders_out = nullptr);

// Energy budget of one meta-atom (analysis/efficiency.hpp:18-44).
struct EfficiencyBudget {
    double reflection, transmission, absorption;
    double t_zero, r_zero, t_stray, r_stray;
    int n_prop_t, n_prop_r;
    std::vector<OrderEfficiency> orders;  // sorted by transmitted power, descending
};
EfficiencyBudget analyze_efficiency(const Material& incident, const Material& pillar, const Material& background,
                                    const Material& substrate, double period_x_um, double period_y_um, double fill_x,
                                    double fill_y, double thickness_um, double wavelength_um, cdouble Ex0,
                                    cdouble Ey0, int M, MetaShape shape = MetaShape::Rectangle,
                                    double shape_param = 0.5);

// New: both polarizations of many uneven cells in one batched launch sequence
// (multi-layer stacks go through the stack batch).
struct CellSpec {
    Rcwa2DStack stack;
    Material incident;
    Material substrate;
    double wavelength_um;
    int M;
    int grid = 0;             // Laurent raster size (0: reference rule)
    bool force_laurent = false;
};
std::vector<std::array<Rcwa2DResult, 2>> solve_rcwa_2d_batch(const std::vector<CellSpec>& cells);

// ---- phase profiles (phase_profile.hpp) -----------------------------------------
enum class PhaseProfileKind { Focusing, Quadratic, Vortex, Deflector, Axicon, Freeform };
struct PhaseProfile {
    PhaseProfileKind kind = PhaseProfileKind::Focusing;
    double focal_length_um = 50.0;
    int topological_charge = 1;
    double deflect_deg = 10.0;
    double deflect_azimuth_deg = 0.0;
    double axicon_deg = 5.0;
    std::vector<double> freeform_phase_rad;
    int freeform_n = 0;
    double freeform_extent_um = 0.0;
};
double phase_profile_value(const PhaseProfile& profile, double x, double y, double wavelength_um);
PhaseProfile load_freeform_phase(const std::string& path, double extent_um);

// ---- unit-cell library and lens design (metalens.hpp:21-135) ----------------------
struct UnitCellLibrary {
    double period_um = 0, wavelength_um = 0, thickness_um = 0;
    std::vector<double> fill, phase, amplitude;
    double phase_span() const;
    double coverage() const;
    int lookup(double target_phase_rad) const;
    int lookup_weighted(double target_phase_rad, double amplitude_weight) const;
    cdouble transmission_for_fill(double fill) const;
};

UnitCellLibrary build_unit_cell_library(const Material& pillar, const Material& background,
                                        const Material& incident, const Material& substrate, double period_um,
                                        double wavelength_um, double thickness_um, double fill_min,
                                        double fill_max, int n_samples, int M,
                                        MetaShape shape = MetaShape::Rectangle, double shape_param = 0.5);

struct HeightSweepEntry {
    double thickness_um, coverage_deg, mean_transmittance;
};
struct HeightOptResult {
    double best_thickness_um = 0, coverage_deg = 0, mean_transmittance = 0;
    bool reached_target = false;
    double coverage_target_deg = 0;
    std::vector<HeightSweepEntry> sweep;
    UnitCellLibrary best_library;
};
HeightOptResult optimize_height_for_2pi(const Material& pillar, const Material& background,
                                        const Material& incident, const Material& substrate, double period_um,
                                        double wavelength_um, double thick_lo, double thick_hi, int n_heights,
                                        double fill_min, double fill_max, int fill_samples, int M,
                                        double coverage_target_deg = 330.0,
                                        MetaShape shape = MetaShape::Rectangle, double shape_param = 0.5);

struct MetalensDesign {
    int n_cells = 0;
    double period_um = 0;
    std::vector<double> fill_map;
    double rms_phase_error_deg = 0;
    double mean_amplitude = 0;
};
MetalensDesign design_metalens(const UnitCellLibrary& lib, const PhaseProfile& profile, double diameter_um,
                               double amplitude_weight = 0.25);
MetalensDesign design_metalens(const UnitCellLibrary& lib, double focal_length_um, double diameter_um,
                               double amplitude_weight = 0.25);

// ---- library builders on the batched RCWA and their on-axis checks ------------------------
// design/metalens.cpp:71-110: one layer of a multi-layer stack swept in fill.
UnitCellLibrary build_unit_cell_library_stack(Rcwa2DStack stack, int active_layer, const Material& incident,
                                              const Material& substrate, double wavelength_um, double fill_min,
                                              double fill_max, int n_samples, int M);

// design/achromatic.hpp:33-161
struct DispersiveAtom {
    double fill = 0;
    double thickness_um = 0;
    MetaShape shape = MetaShape::Rectangle;
    double fill_x = 0, fill_y = 0;
    double shape_param = 0.5;
    double phase0_rad = 0;       // phase at the centre wavelength
    double group_delay_fs = 0;   // least-squares d(phase)/d(omega) over the band
    double mean_amplitude = 0;
    std::vector<double> phase_rad;
    std::vector<double> amplitude;
};
struct MetaAtomSpec {
    MetaShape shape = MetaShape::Rectangle;
    double fill_x = 0.5;
    double fill_y = 0.5;
    double thickness_um = 0.6;
    double shape_param = 0.5;
};
struct DispersiveLibrary {
    std::vector<double> wavelengths_um;
    double center_wavelength_um = 0;
    int center_index = 0;
    double period_um = 0;
    int n_fill = 0, n_height = 0;
    std::vector<DispersiveAtom> atoms;
    double gd_min_fs = 0, gd_max_fs = 0;
};
DispersiveLibrary build_dispersive_library_from_specs(const Material& pillar, const Material& background,
                                                      const Material& incident, const Material& substrate,
                                                      double period_um, const std::vector<double>& band_wavelengths_um,
                                                      double center_wavelength_um,
                                                      const std::vector<MetaAtomSpec>& specs, int M);
DispersiveLibrary build_dispersive_library(const Material& pillar, const Material& background,
                                           const Material& incident, const Material& substrate, double period_um,
                                           const std::vector<double>& band_wavelengths_um,
                                           double center_wavelength_um, double fill_min, double fill_max,
                                           int n_fills, double thick_lo, double thick_hi, int n_heights, int M);
DispersiveLibrary build_single_etch_library(const Material& pillar, const Material& background,
                                            const Material& incident, const Material& substrate, double period_um,
                                            const std::vector<double>& band_wavelengths_um,
                                            double center_wavelength_um, double fill_min, double fill_max,
                                            int n_fills, double thickness_um, int M);
struct AchromaticDesign {
    int n_cells = 0;
    double period_um = 0;
    std::vector<int> atom_index;
    std::vector<double> fill_map;
    std::vector<double> thickness_map;
    double center_wavelength_um = 0;
    double focal_length_um = 0;
    double diameter_um = 0;
    double rms_phase_error_deg = 0;
    double rms_group_delay_error_fs = 0;
    double mean_amplitude = 0;
    double required_gd_span_fs = 0;
    double available_gd_span_fs = 0;
    double gd_coverage = 0;
    bool single_height = true;
    double min_height_um = 0, max_height_um = 0;
};
AchromaticDesign design_achromatic_metalens(const DispersiveLibrary& lib, double focal_length_um,
                                            double diameter_um, double gd_weight = 1.0,
                                            double amplitude_weight = 0.25);
struct AchromaticFocalPoint {
    double wavelength_um;
    double focal_length_um;
    double rel_peak;
};
// On-axis focus search per band sample: 200-point z scans on the GPU far field.
std::vector<AchromaticFocalPoint> verify_achromatic_focus(const DispersiveLibrary& lib,
                                                          const AchromaticDesign& design);
MetalensDesign to_metalens_design(const AchromaticDesign& d);

// design/pb_achromatic.hpp:40-121
struct DispersivePbAtom {
    double fill_x = 0, fill_y = 0;
    double thickness_um = 0;
    double phase0_rad = 0;
    double group_delay_fs = 0;
    double mean_amplitude = 0;
    double mean_conversion = 0;
    double retardance_center_deg = 0;
    std::vector<cdouble> cross;  // (t_x - t_y) / 2 per band sample
};
struct DispersivePbLibrary {
    std::vector<double> wavelengths_um;
    double center_wavelength_um = 0;
    int center_index = 0;
    double period_um = 0;
    double thickness_um = 0;
    int n_fill = 0;
    std::vector<DispersivePbAtom> atoms;
    double gd_min_fs = 0, gd_max_fs = 0;
};
DispersivePbLibrary build_dispersive_pb_library(const Material& pillar, const Material& background,
                                                const Material& incident, const Material& substrate,
                                                double period_um, const std::vector<double>& band_wavelengths_um,
                                                double center_wavelength_um, double fill_min, double fill_max,
                                                int n_fills, double thickness_um, int M, double min_amplitude = 0.30);
struct PbAchromaticDesign {
    int n_cells = 0;
    double period_um = 0;
    double thickness_um = 0;
    int handedness = +1;
    std::vector<int> atom_index;
    std::vector<double> rotation_rad;
    std::vector<double> fill_x_map;
    std::vector<double> fill_y_map;
    double center_wavelength_um = 0;
    double focal_length_um = 0;
    double diameter_um = 0;
    double rms_phase_error_deg = 0;
    double rms_group_delay_error_fs = 0;
    double mean_amplitude = 0;
    double mean_conversion = 0;
    double required_gd_span_fs = 0;
    double available_gd_span_fs = 0;
    double gd_coverage = 0;
};
PbAchromaticDesign design_pb_achromatic_metalens(const DispersivePbLibrary& lib, double focal_length_um,
                                                 double diameter_um, int handedness = +1, double gd_weight = 1.0,
                                                 double amplitude_weight = 0.25);
std::vector<AchromaticFocalPoint> verify_pb_achromatic_focus(const DispersivePbLibrary& lib,
                                                             const PbAchromaticDesign& design);

// design/polar_metalens.hpp:17-60
struct PolarCell {
    double fill_x, fill_y;
    double phase_x, phase_y;
    double amp_x, amp_y;
};
struct PolarizationLibrary {
    double period_um = 0, wavelength_um = 0, thickness_um = 0;
    std::vector<PolarCell> cells;
    int lookup(double target_x, double target_y, double amplitude_weight = 0.0) const;
};
PolarizationLibrary build_polarization_library(const Material& pillar, const Material& background,
                                               const Material& incident, const Material& substrate,
                                               double period_um, double wavelength_um, double thickness_um,
                                               double fill_min, double fill_max, int n_samples, int M);
struct PolarMetalensDesign {
    int n_cells = 0;
    double period_um = 0;
    std::vector<double> fill_x;
    std::vector<double> fill_y;
    std::vector<cdouble> t_x;
    std::vector<cdouble> t_y;
    double rms_phase_error_x_deg = 0, rms_phase_error_y_deg = 0;
    double mean_amp_x = 0, mean_amp_y = 0;
};
PolarMetalensDesign design_polarization_metalens(const PolarizationLibrary& lib, double focal_x_um,
                                                 double focal_y_um, double diameter_um,
                                                 double amplitude_weight = 0.25);

// design/pb_metalens.hpp:13-70: Jones matrix of a cell, the half-wave-plate atom
// search, the rotated-atom check and the geometric-phase (PB) metalens.
struct JonesMatrix {
    cdouble xx, xy, yx, yy;
};
JonesMatrix solve_jones(const Material& incident, const Rcwa2DStack& stack, const Material& substrate,
                        double wavelength_um, int M);
struct HwpAtom {
    double fill_x = 0, fill_y = 0;
    double thickness_um = 0;
    cdouble t_x = 0, t_y = 0;
    double retardance_deg = 0;
    double conversion_efficiency = 0;
};
HwpAtom find_hwp_atom(const Material& pillar, const Material& background, const Material& incident,
                      const Material& substrate, double period_um, double wavelength_um, double thickness_um,
                      double fill_min, double fill_max, int n_samples, int M);
struct PbVerifyPoint {
    double rotation_deg;
    double cross_phase_deg;
    double conversion_eff;
    double copol_leakage;
};
std::vector<PbVerifyPoint> verify_pb_phase(const Material& pillar, const Material& background,
                                           const Material& incident, const Material& substrate, double period_um,
                                           double wavelength_um, const HwpAtom& atom,
                                           const std::vector<double>& rotations_rad, int M);
struct PbMetalensDesign {
    int n_cells = 0;
    double period_um = 0;
    HwpAtom atom;
    std::vector<double> rotation_rad;
    std::vector<cdouble> t_cross;
    double rms_phase_error_deg = 0;
    double conversion_efficiency = 0;
};
PbMetalensDesign design_pb_metalens(const HwpAtom& atom, double period_um, double wavelength_um,
                                    const PhaseProfile& profile, double diameter_um, int handedness = +1);
PbMetalensDesign design_pb_metalens(const HwpAtom& atom, double period_um, double wavelength_um,
                                    double focal_length_um, double diameter_um, int handedness = +1);

// analysis/polarization.hpp:14-36: x / y phase and retardance of a fill_x sweep.
struct BirefringencePoint {
    double fill_x, fill_y;
    double phase_x_deg, phase_y_deg, retardance_deg;
    double tx, ty;
};
std::vector<BirefringencePoint> analyze_birefringence(const Material& pillar, const Material& background,
                                                      const Material& incident, const Material& substrate,
                                                      double period_um, double wavelength_um, double thickness_um,
                                                      double fill_y, double fill_min, double fill_max,
                                                      int n_samples, int M);

// design/system_opt.hpp:12-31: period x thickness grid search on Strehl and
// efficiency; every grid point's library comes from ONE batched RCWA call.
struct SystemOptResult {
    double period_um;
    double thickness_um;
    double strehl;
    double mean_amplitude;
    double merit;
};
SystemOptResult optimize_system(const Material& pillar, const Material& background, const Material& incident,
                                const Material& substrate, double focal_um, double diameter_um,
                                double wavelength_um, double period_lo, double period_hi, double thick_lo,
                                double thick_hi, int grid, int M, int fill_samples, double efficiency_weight,
                                const std::function<void(float)>& progress);

// ---- reference inverse-design gradient (optimize.hpp) --------------------------------
struct PillarTarget {
    double wavelength_um, target_phase_rad, amplitude_weight;
};
struct OptimizedPillar {
    double fill, thickness_um, achieved_phase_rad, achieved_amplitude, loss;
    int iterations;
};
OptimizedPillar optimize_pillar(const Material& pillar, const Material& background, const Material& incident,
                                const Material& substrate, double period_um, const PillarTarget& target, int M,
                                double fill0, double thickness0, int max_iters);

// ---- focal-plane analysis (focal.hpp:16-72) ------------------------------------------
struct FocalAnalysis {
    double strehl, phase_strehl, fwhm_um, diffraction_limit_um, encircled_energy;
};
struct PsfMap {
    int n;
    double half_window_um;
    std::vector<double> intensity;
};
FocalAnalysis analyze_focus(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                            double wavelength_um, double diameter_um);
PsfMap compute_psf(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                   double wavelength_um, double diameter_um, int n, double half_window_um);
PsfMap propagate_pillars(const std::vector<double>& px, const std::vector<double>& py,
                         const std::vector<cdouble>& t, double cx, double cy, double z, double wavelength_um,
                         int n, double half_window_um);
struct FieldPsf {
    PsfMap psf;
    double angle_deg, cx_um, rel_strehl;
};
FieldPsf compute_psf_field(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                           double wavelength_um, double diameter_um, double angle_deg, int n,
                           double half_window_um, double on_axis_peak = 0.0);

// ---- fabrication tolerance (tolerance.hpp:12-27) ------------------------------------------
// Monte-Carlo Strehl under Gaussian pillar-size errors: the reference's seeds,
// generator (std::mt19937) and std::normal_distribution, each trial one GPU
// focal analysis.
struct ToleranceResult {
    double sigma_nm, mean_strehl, std_strehl, worst_strehl;
};
std::vector<ToleranceResult> analyze_tolerance(const MetalensDesign& lens, const UnitCellLibrary& lib,
                                               double focal_length_um, double wavelength_um, double diameter_um,
                                               const std::vector<double>& sigmas_nm, int trials, unsigned seed);

// ---- through-focus and off-axis analyses (callers of the far field) ----------------------
// chromatic.hpp:10-34: on-axis focus search (120 z samples around f0 lambda0 / lambda)
// per wavelength; the dispersive form rebuilds the library at every wavelength.
struct ChromaticPoint {
    double wavelength_um;
    double focal_length_um;
    double rel_peak;
};
std::vector<ChromaticPoint> analyze_chromatic(const MetalensDesign& lens, const UnitCellLibrary& lib,
                                              double design_focal, double design_wavelength, double diameter,
                                              double lambda_min, double lambda_max, int n);
std::vector<ChromaticPoint> analyze_chromatic_dispersive(const MetalensDesign& lens,
                                                         const std::function<UnitCellLibrary(double)>& build_lib_at,
                                                         double design_focal, double design_wavelength,
                                                         double diameter, double lambda_min, double lambda_max,
                                                         int n);

// throughfocus.hpp:13-35: on-axis z scan (161 points) + x-z caustic (201 x 201 on the GPU).
struct ThroughFocus {
    std::vector<float> z_um;
    std::vector<float> intensity;
    double z_peak_um = 0;
    double dof_um = 0;
    int caustic_nx = 0, caustic_nz = 0;
    double caustic_xmin = 0, caustic_xmax = 0;
    double caustic_zmin = 0, caustic_zmax = 0;
    std::vector<float> caustic;
};
ThroughFocus analyze_through_focus(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                                   double wavelength_um, double diameter_um);

// field.hpp:9-47: tilted-illumination focal spots.
struct FieldPoint {
    double angle_deg;
    double rel_strehl;
    double spot_shift_um;
};
std::vector<FieldPoint> analyze_field_of_view(const MetalensDesign& lens, const UnitCellLibrary& lib,
                                              double focal_length_um, double wavelength_um, double diameter_um,
                                              const std::vector<double>& angles_deg);
std::vector<FieldPoint> analyze_wide_fov(const MetalensDesign& lens, const UnitCellLibrary& lib,
                                         double focal_length_um, double wavelength_um, double lens_diameter_um,
                                         double stop_diameter_um, double stop_distance_um,
                                         const std::vector<double>& angles_deg);
struct FieldGridPoint {
    double theta_x_deg, theta_y_deg;
    double rel_strehl;
    double fwhm_x_um, fwhm_y_um;
    double cx_um, cy_um;
};
struct FieldGrid {
    int n = 0;
    double max_angle_deg = 0;
    std::vector<FieldGridPoint> points;
};
FieldGrid analyze_field_grid(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                             double wavelength_um, double diameter_um, double max_angle_deg, int n_half, int psf_n);

namespace cuda {
bool available();
const char* device_name();
bool propagate_psf(const double* px, const double* py, const std::complex<double>* pt, int npil, double cx,
                   double cy, double z, double k, int n, double half_window, double* out);
bool propagate_zx(const double* px, const double* py, const std::complex<double>* pt, int npil, double xmin,
                  double xmax, int nx, double zmin, double zmax, int nz, double k, double* out);
// cuda/eigensolve.hpp:14-31: general complex eigendecomposition (column-major);
// `streams` is accepted for the signature and unused (the batch is one launch
// sequence, one CTA per matrix).
bool geev(const std::complex<double>* A, int n, std::complex<double>* w, std::complex<double>* vr);
bool geev_batched(const std::complex<double>* As, int n, int batch, std::complex<double>* ws,
                  std::complex<double>* vrs, int streams = 4);
}  // namespace cuda

}  // namespace celeris
