// Host logic of the celeris:: mirror. The arithmetic of the hot path is on
// the GPU behind the C ABI; what stays here is the reference's host-side glue
// (materials, aperture assembly, library lookup, lens design, focal metrics),
// written to the same specifications:
//   materials        material.cpp:13-81, database.cpp:12-46
//   solve_rcwa_2d    rcwa2d.cpp:209-222 argument checks, then celeris_solve_rcwa_2d (one
//                    layer) or celeris_solve_rcwa_2d_stack (several layers)
//   library sweep    metalens.cpp:122-163 (one batched GPU launch sequence)
//   lookup / design  metalens.cpp:14-69, 112-120, 230-272
//   height sweep     metalens.cpp:165-228
//   optimize_pillar  optimize.cpp:22-86 (central differences + Adam; the four
//                    perturbed solves per step are one GPU batch)
//   focal analysis   focal.cpp:32-146 (metrics), 148-203, 205-238, 240-311
#include "celeris.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <random>
#include <sstream>
#include <stdexcept>

#include "celeris_b200.h"
#include "detail.hpp"

namespace celeris {
namespace detail {

void check(int status, const char* what) {
    if (status == CELERIS_OK) return;
    std::string msg = std::string(what) + ": " + celeris_last_error();
    if (status == CELERIS_ERR_INVALID_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

double angle_diff(double a, double b) {
    double d = a - b;
    while (d > pi) d -= 2.0 * pi;
    while (d <= -pi) d += 2.0 * pi;
    return d;
}

celeris_rcwa_cell to_cell(const Material& incident, const RectCell2D& L, const Material& substrate,
                          double px, double py, double wl, double theta, double phi, int Mx, int My, int grid,
                          bool force_laurent) {
    celeris_rcwa_cell c{};
    c.period_x_um = px;
    c.period_y_um = py;
    c.wavelength_um = wl;
    c.theta_rad = theta;
    c.phi_rad = phi;
    const cdouble ni = incident.index(wl), ns = substrate.index(wl);
    const cdouble ep = L.pillar.permittivity(wl), eb = L.background.permittivity(wl);
    c.n_inc[0] = ni.real();
    c.n_inc[1] = ni.imag();
    c.n_sub[0] = ns.real();
    c.n_sub[1] = ns.imag();
    c.eps_pillar[0] = ep.real();
    c.eps_pillar[1] = ep.imag();
    c.eps_bg[0] = eb.real();
    c.eps_bg[1] = eb.imag();
    c.fill_x = L.fill_x;
    c.fill_y = L.fill_y;
    c.thickness_um = L.thickness_um;
    c.shape_param = L.shape_param;
    c.rotation_rad = L.rotation_rad;
    c.shape = static_cast<int>(L.shape);
    c.Mx = Mx;
    c.My = My;
    c.grid = grid;
    c.force_laurent = force_laurent ? 1 : 0;
    return c;
}

Rcwa2DResult from_result(const celeris_rcwa_result& r) {
    return Rcwa2DResult{r.R, r.T, r.sum_de, r.de_t0, r.de_r0, cdouble(r.tx0[0], r.tx0[1]),
                        cdouble(r.ty0[0], r.ty0[1])};
}

// |E|^2 of the plain FP64 form on the n x n grid (the GPU kernel).
std::vector<double> psf_gpu(const std::vector<Cell>& cells, double cx, double cy, double z, double k, int n,
                            double W) {
    std::vector<double> px(cells.size()), py(cells.size()), pt(2 * cells.size());
    for (size_t c = 0; c < cells.size(); ++c) {
        px[c] = cells[c].x;
        py[c] = cells[c].y;
        pt[2 * c] = cells[c].t.real();
        pt[2 * c + 1] = cells[c].t.imag();
    }
    std::vector<double> out(static_cast<size_t>(n) * n, 0.0);
    check(celeris_propagate_psf(px.data(), py.data(), pt.data(), static_cast<int>(cells.size()), cx, cy, z, k, n,
                                W, out.data()),
          "propagate_psf");
    return out;
}

// |E|^2 on an x-z slice (y = 0) of the plain FP64 form: row = z, column = x.
std::vector<double> zx_gpu(const std::vector<Cell>& cells, double xmin, double xmax, int nx, double zmin,
                           double zmax, int nz, double k) {
    std::vector<double> px(cells.size()), py(cells.size()), pt(2 * cells.size());
    for (size_t c = 0; c < cells.size(); ++c) {
        px[c] = cells[c].x;
        py[c] = cells[c].y;
        pt[2 * c] = cells[c].t.real();
        pt[2 * c + 1] = cells[c].t.imag();
    }
    std::vector<double> out(static_cast<size_t>(nx) * nz, 0.0);
    if (cells.empty()) return out;
    check(celeris_propagate_zx(px.data(), py.data(), pt.data(), static_cast<int>(cells.size()), xmin, xmax, nx,
                               zmin, zmax, nz, k, out.data()),
          "propagate_zx");
    return out;
}

}  // namespace detail

namespace {
using namespace detail;

std::vector<Cell> aperture_cells(const MetalensDesign& lens, const UnitCellLibrary& lib, double diameter_um,
                                 double k_tilt_sin = 0.0) {
    // focal.cpp:156-164 (circular aperture mask, nearest-fill transmission)
    const double p = lens.period_um;
    const double center = (lens.n_cells - 1) / 2.0;
    const double R_ap = diameter_um / 2.0;
    std::vector<Cell> cells;
    for (int iy = 0; iy < lens.n_cells; ++iy)
        for (int ix = 0; ix < lens.n_cells; ++ix) {
            const double x = (ix - center) * p, y = (iy - center) * p;
            if (std::sqrt(x * x + y * y) > R_ap) continue;
            const double fill = lens.fill_map[static_cast<size_t>(iy) * lens.n_cells + ix];
            cdouble t = lib.transmission_for_fill(fill);
            if (k_tilt_sin != 0.0) t *= std::polar(1.0, k_tilt_sin * x);
            cells.push_back({x, y, t});
        }
    return cells;
}

// Peak |E|^2 and the x of its pixel on an NG x NG grid centred at (xc, 0): the
// search of field.cpp:48-75 / 106-134 (first maximum in row-major order, strict >).
std::pair<double, double> peak_on_grid(const std::vector<Cell>& cells, double xc, double W, double z, double k) {
    constexpr int NG = 81;
    double best = 0.0, best_x = xc;
    if (cells.empty()) return {best, best_x};
    const std::vector<double> I = psf_gpu(cells, xc, 0.0, z, k, NG, W);
    const double step = 2.0 * W / (NG - 1);
    for (int j = 0; j < NG; ++j)
        for (int i = 0; i < NG; ++i) {
            const double v = I[static_cast<size_t>(j) * NG + i];
            if (v > best) {
                best = v;
                best_x = (xc - W) + i * step;
            }
        }
    return {best, best_x};
}

}  // namespace
using namespace detail;

// ---- materials ---------------------------------------------------------------------
Material::Material(std::function<cdouble(double)> dispersion, std::string name)
    : dispersion_(std::move(dispersion)), name_(std::move(name)) {}

Material Material::constant(cdouble n, std::string name) {
    return Material([n](double) { return n; }, std::move(name));
}

Material Material::sellmeier(std::vector<std::array<double, 2>> bc, std::string name) {
    return Material(
        [bc = std::move(bc)](double wl) {
            const double l2 = wl * wl;
            double n2 = 1.0;
            for (const auto& t : bc) n2 += t[0] * l2 / (l2 - t[1]);
            return cdouble(std::sqrt(n2), 0.0);
        },
        std::move(name));
}

Material Material::sellmeier_ri_formula1(std::vector<double> c, std::string name) {
    if (c.empty() || c.size() % 2 == 0)
        throw std::invalid_argument("Material::sellmeier_ri_formula1: need c0 + (strength, resonance) pairs");
    return Material(
        [c = std::move(c)](double wl) {
            const double l2 = wl * wl;
            double n2 = 1.0 + c[0];
            for (size_t i = 1; i + 1 < c.size(); i += 2) n2 += c[i] * l2 / (l2 - c[i + 1] * c[i + 1]);
            return cdouble(std::sqrt(n2), 0.0);
        },
        std::move(name));
}

Material Material::tabulated(std::vector<double> wl, std::vector<double> n, std::vector<double> k,
                             std::string name) {
    if (wl.size() < 2 || wl.size() != n.size() || n.size() != k.size())
        throw std::invalid_argument("Material::tabulated: need matching arrays of length >= 2");
    if (!std::is_sorted(wl.begin(), wl.end()))
        throw std::invalid_argument("Material::tabulated: wavelengths must be ascending");
    return Material(
        [wl = std::move(wl), n = std::move(n), k = std::move(k)](double q) {
            if (q <= wl.front()) return cdouble(n.front(), k.front());
            if (q >= wl.back()) return cdouble(n.back(), k.back());
            const size_t i = static_cast<size_t>(std::lower_bound(wl.begin(), wl.end(), q) - wl.begin());
            const double t = (q - wl[i - 1]) / (wl[i] - wl[i - 1]);
            return cdouble(n[i - 1] + t * (n[i] - n[i - 1]), k[i - 1] + t * (k[i] - k[i - 1]));
        },
        std::move(name));
}

namespace materials {
const Material& air() {
    static const Material m = Material::constant(cdouble(1.0, 0.0), "air");
    return m;
}
const Material& bk7() {  // Schott N-BK7 Sellmeier {B, C (um^2)}
    static const Material m = Material::sellmeier(
        {{{1.03961212, 0.00600069867}, {0.231792344, 0.0200179144}, {1.01046945, 103.560653}}}, "N-BK7");
    return m;
}
const Material& fused_silica() {  // Malitson 1965
    static const Material m = Material::sellmeier({{{0.6961663, 0.0684043 * 0.0684043},
                                                    {0.4079426, 0.1162414 * 0.1162414},
                                                    {0.8974794, 9.896161 * 9.896161}}},
                                                  "fused-silica");
    return m;
}
const Material& silicon_nitride() {  // Luke et al. 2015
    static const Material m =
        Material::sellmeier({{{3.0249, 0.1353406 * 0.1353406}, {40314.0, 1239.842 * 1239.842}}}, "Si3N4");
    return m;
}
}  // namespace materials

// ---- RCWA ------------------------------------------------------------------------------
Rcwa2DResult solve_rcwa_2d(const Material& incident, const Rcwa2DStack& stack, const Material& substrate,
                           double wavelength_um, double theta_rad, double phi_rad, cdouble Ex0, cdouble Ey0,
                           int Mx, int My, std::vector<OrderEfficiency>* orders_out) {
    if (Mx < 0 || My < 0) throw std::invalid_argument("M must be >= 0");
    if (stack.layers.empty()) throw std::invalid_argument("solve_rcwa_2d: stack has no layers");
    std::vector<celeris_rcwa_cell> cc;
    cc.reserve(stack.layers.size());
    for (const RectCell2D& L : stack.layers)
        cc.push_back(to_cell(incident, L, substrate, stack.period_x_um, stack.period_y_um, wavelength_um, theta_rad,
                             phi_rad, Mx, My, 0, false));
    const double ex[2] = {Ex0.real(), Ex0.imag()}, ey[2] = {Ey0.real(), Ey0.imag()};
    celeris_rcwa_result r{};
    if (orders_out) {
        const int N = (2 * Mx + 1) * (2 * My + 1);
        std::vector<celeris_rcwa_order> o(N);
        check(celeris_solve_rcwa_2d_orders(cc.data(), static_cast<int>(cc.size()), ex, ey, &r, o.data(), N),
              "solve_rcwa_2d");
        orders_out->clear();
        orders_out->reserve(N);
        for (const celeris_rcwa_order& x : o)
            orders_out->push_back(OrderEfficiency{x.p, x.q, x.de_t, x.de_r, x.prop_t != 0, x.prop_r != 0});
    } else if (cc.size() == 1)
        check(celeris_solve_rcwa_2d(&cc[0], ex, ey, &r), "solve_rcwa_2d");
    else
        check(celeris_solve_rcwa_2d_stack(cc.data(), static_cast<int>(cc.size()), ex, ey, &r), "solve_rcwa_2d");
    return from_result(r);
}

void eig_general(const std::vector<cdouble>& A, int n, std::vector<cdouble>& evals, std::vector<cdouble>& evecs) {
    if (n < 1 || A.size() != static_cast<size_t>(n) * n)
        throw std::invalid_argument("eig_general: A must hold n * n entries, n >= 1");
    evals.assign(n, cdouble(0.0, 0.0));
    evecs.assign(static_cast<size_t>(n) * n, cdouble(0.0, 0.0));
    check(celeris_eig_general(reinterpret_cast<const double*>(A.data()), n, reinterpret_cast<double*>(evals.data()),
                              reinterpret_cast<double*>(evecs.data())),
          "eig_general");
}

// analysis/efficiency.cpp:7-46: one solve with orders, then the budget.
EfficiencyBudget analyze_efficiency(const Material& incident, const Material& pillar, const Material& background,
                                    const Material& substrate, double period_x_um, double period_y_um, double fill_x,
                                    double fill_y, double thickness_um, double wavelength_um, cdouble Ex0,
                                    cdouble Ey0, int M, MetaShape shape, double shape_param) {
    RectCell2D cell{pillar, background, fill_x, fill_y, thickness_um, shape, shape_param};
    Rcwa2DStack stack{period_x_um, period_y_um, {cell}};
    std::vector<OrderEfficiency> orders;
    const Rcwa2DResult r =
        solve_rcwa_2d(incident, stack, substrate, wavelength_um, 0.0, 0.0, Ex0, Ey0, M, M, &orders);
    EfficiencyBudget b{};
    b.reflection = r.R;
    b.transmission = r.T;
    b.absorption = std::max(0.0, 1.0 - r.R - r.T);
    b.t_zero = r.de_t0;
    b.r_zero = r.de_r0;
    b.t_stray = std::max(0.0, r.T - r.de_t0);
    b.r_stray = std::max(0.0, r.R - r.de_r0);
    for (const OrderEfficiency& o : orders) {
        b.n_prop_t += o.prop_t ? 1 : 0;
        b.n_prop_r += o.prop_r ? 1 : 0;
    }
    std::sort(orders.begin(), orders.end(),
              [](const OrderEfficiency& a, const OrderEfficiency& c) { return a.de_t > c.de_t; });
    b.orders = std::move(orders);
    return b;
}

std::vector<std::array<Rcwa2DResult, 2>> solve_rcwa_2d_batch(const std::vector<CellSpec>& cells) {
    std::vector<celeris_rcwa_cell> cc;
    std::vector<int> start(1, 0);
    bool multi = false;
    for (const CellSpec& s : cells) {
        if (s.stack.layers.empty()) throw std::invalid_argument("solve_rcwa_2d_batch: stack has no layers");
        multi = multi || s.stack.layers.size() > 1;
        for (const RectCell2D& L : s.stack.layers)
            cc.push_back(to_cell(s.incident, L, s.substrate, s.stack.period_x_um, s.stack.period_y_um,
                                 s.wavelength_um, 0.0, 0.0, s.M, s.M, s.grid, s.force_laurent));
        start.push_back(static_cast<int>(cc.size()));
    }
    const int ns = static_cast<int>(cells.size());
    std::vector<celeris_rcwa_result> r(2 * cells.size());
    std::vector<int> info(cells.size());
    if (multi)
        check(celeris_rcwa_stack_batch(cc.data(), start.data(), ns, r.data(), info.data()), "rcwa_stack_batch");
    else
        check(celeris_rcwa_batch(cc.data(), ns, r.data(), info.data()), "rcwa_batch");
    std::vector<std::array<Rcwa2DResult, 2>> out(cells.size());
    for (size_t i = 0; i < cells.size(); ++i) out[i] = {from_result(r[2 * i]), from_result(r[2 * i + 1])};
    return out;
}

// ---- phase profiles ---------------------------------------------------------------------
namespace {
double sample_freeform(const PhaseProfile& p, double x, double y) {
    const int n = p.freeform_n;
    if (n <= 0 || p.freeform_extent_um <= 0.0 || static_cast<int>(p.freeform_phase_rad.size()) < n * n)
        return 0.0;
    if (n == 1) return p.freeform_phase_rad[0];
    const double W = p.freeform_extent_um;
    const double gx = std::clamp((x / W + 0.5) * (n - 1), 0.0, static_cast<double>(n - 1));
    const double gy = std::clamp((y / W + 0.5) * (n - 1), 0.0, static_cast<double>(n - 1));
    const int x0 = static_cast<int>(std::floor(gx)), y0 = static_cast<int>(std::floor(gy));
    const int x1 = std::min(x0 + 1, n - 1), y1 = std::min(y0 + 1, n - 1);
    const double fx = gx - x0, fy = gy - y0;
    auto at = [&](int ix, int iy) { return p.freeform_phase_rad[static_cast<size_t>(iy) * n + ix]; };
    const double top = at(x0, y0) * (1 - fx) + at(x1, y0) * fx;
    const double bot = at(x0, y1) * (1 - fx) + at(x1, y1) * fx;
    return top * (1 - fy) + bot * fy;
}
}  // namespace

double phase_profile_value(const PhaseProfile& p, double x, double y, double wavelength_um) {
    const double k = 2.0 * pi / wavelength_um;
    const double r = std::sqrt(x * x + y * y);
    const double f = p.focal_length_um;
    switch (p.kind) {
        case PhaseProfileKind::Focusing:
            return -k * (std::sqrt(r * r + f * f) - f);
        case PhaseProfileKind::Quadratic:
            return -k * r * r / (2.0 * f);
        case PhaseProfileKind::Vortex: {
            double phi = p.topological_charge * std::atan2(y, x);
            if (f > 0.0) phi += -k * (std::sqrt(r * r + f * f) - f);
            return phi;
        }
        case PhaseProfileKind::Deflector: {
            const double a = p.deflect_deg * pi / 180.0, az = p.deflect_azimuth_deg * pi / 180.0;
            return k * std::sin(a) * (x * std::cos(az) + y * std::sin(az));
        }
        case PhaseProfileKind::Axicon:
            return -k * std::sin(p.axicon_deg * pi / 180.0) * r;
        case PhaseProfileKind::Freeform:
            return sample_freeform(p, x, y);
    }
    return 0.0;
}

PhaseProfile load_freeform_phase(const std::string& path, double extent_um) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open freeform phase file: " + path);
    std::vector<double> vals;
    std::string line;
    while (std::getline(f, line)) {
        const size_t h = line.find('#');
        if (h != std::string::npos) line.resize(h);
        std::istringstream ss(line);
        for (double v; ss >> v;) vals.push_back(v);
    }
    if (vals.empty()) throw std::runtime_error("freeform phase file is empty: " + path);
    const int n = static_cast<int>(std::llround(std::sqrt(static_cast<double>(vals.size()))));
    if (static_cast<size_t>(n) * n != vals.size())
        throw std::runtime_error("freeform phase file is not a square grid: " + path);
    if (extent_um <= 0.0) throw std::runtime_error("freeform phase extent must be positive");
    PhaseProfile p;
    p.kind = PhaseProfileKind::Freeform;
    p.freeform_phase_rad = std::move(vals);
    p.freeform_n = n;
    p.freeform_extent_um = extent_um;
    return p;
}

// ---- library --------------------------------------------------------------------------
double UnitCellLibrary::phase_span() const {
    if (phase.empty()) return 0.0;
    const auto mm = std::minmax_element(phase.begin(), phase.end());
    return *mm.second - *mm.first;
}

double UnitCellLibrary::coverage() const {
    const int n = static_cast<int>(phase.size());
    if (n < 2) return 0.0;
    std::vector<double> p(phase.begin(), phase.end());
    for (double& v : p) {
        while (v < 0.0) v += 2.0 * pi;
        while (v >= 2.0 * pi) v -= 2.0 * pi;
    }
    std::sort(p.begin(), p.end());
    double gap = 0.0;
    for (int i = 1; i < n; ++i) gap = std::max(gap, p[i] - p[i - 1]);
    gap = std::max(gap, (p[0] + 2.0 * pi) - p[n - 1]);
    return 2.0 * pi - gap;
}

int UnitCellLibrary::lookup(double target) const {
    int best = 0;
    double be = std::abs(angle_diff(phase[0], target));
    for (int i = 1; i < static_cast<int>(phase.size()); ++i) {
        const double e = std::abs(angle_diff(phase[i], target));
        if (e < be) {
            be = e;
            best = i;
        }
    }
    return best;
}

int UnitCellLibrary::lookup_weighted(double target, double w) const {
    int best = 0;
    double bc = 1e300;
    for (int i = 0; i < static_cast<int>(phase.size()); ++i) {
        const double dphi = angle_diff(phase[i], target), damp = 1.0 - amplitude[i];
        const double cost = dphi * dphi + w * damp * damp;
        if (cost < bc) {
            bc = cost;
            best = i;
        }
    }
    return best;
}

cdouble UnitCellLibrary::transmission_for_fill(double f) const {
    int best = 0;
    double bd = std::abs(fill[0] - f);
    for (int i = 1; i < static_cast<int>(fill.size()); ++i) {
        const double d = std::abs(fill[i] - f);
        if (d < bd) {
            bd = d;
            best = i;
        }
    }
    return std::polar(amplitude[best], phase[best]);
}

UnitCellLibrary build_unit_cell_library(const Material& pillar, const Material& background,
                                        const Material& incident, const Material& substrate, double period_um,
                                        double wavelength_um, double thickness_um, double fill_min,
                                        double fill_max, int n_samples, int M, MetaShape shape,
                                        double shape_param) {
    UnitCellLibrary lib;
    lib.period_um = period_um;
    lib.wavelength_um = wavelength_um;
    lib.thickness_um = thickness_um;
    if (n_samples <= 0) return lib;
    std::vector<celeris_rcwa_cell> cc(n_samples);
    lib.fill.resize(n_samples);
    for (int i = 0; i < n_samples; ++i) {
        const double f = fill_min + (fill_max - fill_min) * i / (n_samples - 1);  // metalens.cpp:142
        lib.fill[i] = f;
        RectCell2D L{pillar, background, f, f, thickness_um, shape, shape_param};
        cc[i] = to_cell(incident, L, substrate, period_um, period_um, wavelength_um, 0.0, 0.0, M, M, 0, false);
    }
    std::vector<celeris_rcwa_result> r(2 * n_samples);
    check(celeris_rcwa_batch(cc.data(), n_samples, r.data(), nullptr), "build_unit_cell_library");
    lib.phase.resize(n_samples);
    lib.amplitude.resize(n_samples);
    for (int i = 0; i < n_samples; ++i) {  // X polarization (Ex0 = 1), metalens.cpp:146-150
        const cdouble t(r[2 * i].tx0[0], r[2 * i].tx0[1]);
        lib.phase[i] = std::arg(t);
        lib.amplitude[i] = std::abs(t);
    }
    return lib;
}

HeightOptResult optimize_height_for_2pi(const Material& pillar, const Material& background,
                                        const Material& incident, const Material& substrate, double period_um,
                                        double wavelength_um, double thick_lo, double thick_hi, int n_heights,
                                        double fill_min, double fill_max, int fill_samples, int M,
                                        double coverage_target_deg, MetaShape shape, double shape_param) {
    n_heights = std::max(2, n_heights);
    HeightOptResult res;
    res.coverage_target_deg = coverage_target_deg;
    std::vector<UnitCellLibrary> libs;
    double best_cov = 0.0;
    for (int i = 0; i < n_heights; ++i) {
        const double h = thick_lo + (thick_hi - thick_lo) * i / (n_heights - 1);
        UnitCellLibrary lib = build_unit_cell_library(pillar, background, incident, substrate, period_um,
                                                      wavelength_um, h, fill_min, fill_max, fill_samples, M,
                                                      shape, shape_param);
        double s = 0.0;
        for (double a : lib.amplitude) s += a * a;
        const double mt = lib.amplitude.empty() ? 0.0 : s / lib.amplitude.size();
        const double cov = lib.coverage() * 180.0 / pi;
        res.sweep.push_back({h, cov, mt});
        best_cov = std::max(best_cov, cov);
        libs.push_back(std::move(lib));
    }
    // selection rule of metalens.cpp:207-227
    const double tol = 12.0;
    const bool any = best_cov >= coverage_target_deg - 1e-9;
    const double floor_deg = any ? coverage_target_deg : best_cov - tol;
    int bi = 0;
    double bT = -1.0;
    for (int i = 0; i < n_heights; ++i) {
        if (res.sweep[i].coverage_deg < floor_deg - 1e-9) continue;
        if (res.sweep[i].mean_transmittance > bT + 1e-12) {
            bT = res.sweep[i].mean_transmittance;
            bi = i;
        }
    }
    res.best_thickness_um = res.sweep[bi].thickness_um;
    res.coverage_deg = res.sweep[bi].coverage_deg;
    res.mean_transmittance = res.sweep[bi].mean_transmittance;
    res.reached_target = res.coverage_deg >= coverage_target_deg - 1e-9;
    res.best_library = std::move(libs[bi]);
    return res;
}

MetalensDesign design_metalens(const UnitCellLibrary& lib, const PhaseProfile& profile, double diameter_um,
                               double amplitude_weight) {
    const double p = lib.period_um, lambda = lib.wavelength_um;
    const int n = std::max(1, static_cast<int>(std::round(diameter_um / p)));
    const double center = (n - 1) / 2.0;
    MetalensDesign d;
    d.n_cells = n;
    d.period_um = p;
    d.fill_map.resize(static_cast<size_t>(n) * n);
    double sq = 0.0, amp = 0.0;
    int count = 0;
    for (int iy = 0; iy < n; ++iy)
        for (int ix = 0; ix < n; ++ix) {
            const double x = (ix - center) * p, y = (iy - center) * p;
            const double target = phase_profile_value(profile, x, y, lambda);
            const int idx = lib.lookup_weighted(target, amplitude_weight);
            d.fill_map[static_cast<size_t>(iy) * n + ix] = lib.fill[idx];
            const double e = angle_diff(lib.phase[idx], target);
            sq += e * e;
            amp += lib.amplitude[idx];
            ++count;
        }
    d.rms_phase_error_deg = std::sqrt(sq / count) * 180.0 / pi;
    d.mean_amplitude = amp / count;
    return d;
}

MetalensDesign design_metalens(const UnitCellLibrary& lib, double focal_length_um, double diameter_um,
                               double amplitude_weight) {
    PhaseProfile prof;
    prof.kind = PhaseProfileKind::Focusing;
    prof.focal_length_um = focal_length_um;
    return design_metalens(lib, prof, diameter_um, amplitude_weight);
}

// ---- optimize_pillar ------------------------------------------------------------------------
OptimizedPillar optimize_pillar(const Material& pillar, const Material& background, const Material& incident,
                                const Material& substrate, double period_um, const PillarTarget& target, int M,
                                double fill0, double thickness0, int max_iters) {
    const std::array<double, 2> lo{0.08, 0.20}, hi{0.92, 1.00};
    std::array<double, 2> x{std::clamp(fill0, lo[0], hi[0]), std::clamp(thickness0, lo[1], hi[1])};
    auto cell_of = [&](const std::array<double, 2>& v) {
        RectCell2D L{pillar, background, v[0], v[0], v[1]};
        return to_cell(incident, L, substrate, period_um, period_um, target.wavelength_um, 0.0, 0.0, M, M, 0,
                       false);
    };
    auto loss_of = [&](const celeris_rcwa_result& r) {
        const cdouble t(r.tx0[0], r.tx0[1]);
        const double dphi = angle_diff(std::arg(t), target.target_phase_rad);
        const double damp = 1.0 - std::abs(t);
        return dphi * dphi + target.amplitude_weight * damp * damp;
    };
    auto solve = [&](const std::vector<std::array<double, 2>>& pts) {
        std::vector<celeris_rcwa_cell> cc;
        for (const auto& v : pts) cc.push_back(cell_of(v));
        std::vector<celeris_rcwa_result> r(2 * cc.size());
        check(celeris_rcwa_batch(cc.data(), static_cast<int>(cc.size()), r.data(), nullptr), "optimize_pillar");
        std::vector<celeris_rcwa_result> xpol(cc.size());
        for (size_t i = 0; i < cc.size(); ++i) xpol[i] = r[2 * i];
        return xpol;
    };
    std::array<double, 2> m{0, 0}, v2{0, 0};
    const double b1 = 0.9, b2 = 0.999, eps = 1e-8;
    const std::array<double, 2> lr{0.04, 0.04}, h{5e-3, 5e-3};  // optimize.cpp:50-52
    std::array<double, 2> best = x;
    double best_loss = loss_of(solve({x})[0]);
    for (int t = 1; t <= max_iters; ++t) {
        std::array<std::array<double, 2>, 2> xp{x, x}, xm{x, x};
        for (int k = 0; k < 2; ++k) {
            xp[k][k] = std::clamp(x[k] + h[k], lo[k], hi[k]);
            xm[k][k] = std::clamp(x[k] - h[k], lo[k], hi[k]);
        }
        const auto r = solve({xp[0], xm[0], xp[1], xm[1]});  // the four central-difference solves
        std::array<double, 2> g{(loss_of(r[0]) - loss_of(r[1])) / (xp[0][0] - xm[0][0]),
                                (loss_of(r[2]) - loss_of(r[3])) / (xp[1][1] - xm[1][1])};
        for (int k = 0; k < 2; ++k) {
            m[k] = b1 * m[k] + (1 - b1) * g[k];
            v2[k] = b2 * v2[k] + (1 - b2) * g[k] * g[k];
            const double mh = m[k] / (1 - std::pow(b1, t)), vh = v2[k] / (1 - std::pow(b2, t));
            x[k] = std::clamp(x[k] - lr[k] * mh / (std::sqrt(vh) + eps), lo[k], hi[k]);
        }
        const double l = loss_of(solve({x})[0]);
        if (l < best_loss) {
            best_loss = l;
            best = x;
        }
    }
    const celeris_rcwa_result r = solve({best})[0];
    const cdouble t(r.tx0[0], r.tx0[1]);
    return {best[0], best[1], std::arg(t), std::abs(t), best_loss, max_iters};
}

// ---- focal analysis -----------------------------------------------------------------------------
FocalAnalysis analyze_focus(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                            double wavelength_um, double diameter_um) {
    const double k = 2.0 * pi / wavelength_um;
    std::vector<Cell> cells = aperture_cells(lens, lib, diameter_um);
    const double dl = wavelength_um * focal_length_um / diameter_um;  // focal.cpp:61-64
    const double W = std::max(6.0 * dl, 4.0);
    const int NG = 121;
    const double step = 2.0 * W / (NG - 1);
    const std::vector<double> I = psf_gpu(cells, 0.0, 0.0, focal_length_um, k, NG, W);
    const double peak = *std::max_element(I.begin(), I.end());
    // ideal lens at the focal centre: |t| = 1, ideal phase (focal.cpp:104); on
    // the GPU as the centre pixel of a 3 x 3 grid with step W' (exactly 0).
    std::vector<Cell> ideal = cells;
    for (Cell& c : ideal) {
        const double r = std::sqrt(c.x * c.x + c.y * c.y);
        c.t = std::polar(1.0, -k * (std::sqrt(r * r + focal_length_um * focal_length_um) - focal_length_um));
    }
    const std::vector<double> I3 = psf_gpu(ideal, 0.0, 0.0, focal_length_um, k, 3, 1.0);
    const double peak_ideal = I3[4];
    double amp = 0.0;  // same-amplitude in-phase peak (focal.cpp:109-115)
    for (const Cell& c : cells)
        amp += std::abs(c.t) / std::sqrt(c.x * c.x + c.y * c.y + focal_length_um * focal_length_um);
    const double peak_same = amp * amp;
    const int cr = NG / 2;
    const double half = peak / 2.0;
    int lo = -1, hi = -1;
    for (int i = 0; i < NG; ++i) {
        const double v = I[static_cast<size_t>(cr) * NG + i];
        if (v >= half) {
            if (lo < 0) lo = i;
            hi = i;
        }
    }
    const double fwhm = (hi > lo && lo >= 0) ? (hi - lo) * step : 0.0;
    const double r_null = 1.22 * dl;
    double in = 0.0, total = 0.0;
    for (int j = 0; j < NG; ++j) {
        const double fy = -W + j * step;
        for (int i = 0; i < NG; ++i) {
            const double fx = -W + i * step;
            const double v = I[static_cast<size_t>(j) * NG + i];
            total += v;
            if (std::sqrt(fx * fx + fy * fy) <= r_null) in += v;
        }
    }
    FocalAnalysis out;
    out.strehl = peak_ideal > 0 ? peak / peak_ideal : 0.0;
    out.phase_strehl = peak_same > 0 ? peak / peak_same : 0.0;
    out.fwhm_um = fwhm;
    out.diffraction_limit_um = dl;
    out.encircled_energy = total > 0 ? in / total : 0.0;
    return out;
}

PsfMap compute_psf(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                   double wavelength_um, double diameter_um, int n, double half_window_um) {
    const double k = 2.0 * pi / wavelength_um;
    PsfMap m{n, half_window_um, {}};
    if (n <= 0) return m;
    m.intensity = psf_gpu(aperture_cells(lens, lib, diameter_um), 0.0, 0.0, focal_length_um, k, n, half_window_um);
    return m;
}

PsfMap propagate_pillars(const std::vector<double>& px, const std::vector<double>& py,
                         const std::vector<cdouble>& t, double cx, double cy, double z, double wavelength_um,
                         int n, double half_window_um) {
    PsfMap m{n, half_window_um, {}};
    const double k = 2.0 * pi / wavelength_um;
    const int npil = static_cast<int>(px.size());
    if (npil == 0 || n <= 0) {  // focal.cpp:216
        m.intensity.assign(static_cast<size_t>(std::max(n, 0)) * std::max(n, 0), 0.0);
        return m;
    }
    if (py.size() != px.size() || t.size() != px.size())
        throw std::invalid_argument("propagate_pillars: px, py, t lengths differ");
    m.intensity.assign(static_cast<size_t>(n) * n, 0.0);
    check(celeris_propagate_psf(px.data(), py.data(), reinterpret_cast<const double*>(t.data()), npil, cx, cy, z,
                                k, n, half_window_um, m.intensity.data()),
          "propagate_pillars");
    return m;
}

FieldPsf compute_psf_field(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                           double wavelength_um, double diameter_um, double angle_deg, int n,
                           double half_window_um, double on_axis_peak) {
    const double k = 2.0 * pi / wavelength_um;
    const double theta = angle_deg * pi / 180.0;
    std::vector<Cell> cells = aperture_cells(lens, lib, diameter_um, k * std::sin(theta));
    const double cx = focal_length_um * std::tan(theta);  // focal.cpp:264
    FieldPsf out;
    out.angle_deg = angle_deg;
    out.cx_um = cx;
    out.psf = PsfMap{n, half_window_um, {}};
    // the reference samples fx around cx but fy around 0 (focal.cpp:292-295)
    out.psf.intensity = psf_gpu(cells, cx, 0.0, focal_length_um, k, n, half_window_um);
    double peak = 0.0;
    for (double v : out.psf.intensity) peak = std::max(peak, v);
    out.rel_strehl = on_axis_peak > 0 ? peak / on_axis_peak : 1.0;
    return out;
}

// ---- through-focus (throughfocus.cpp:15-135) -------------------------------------------------
// ---- fabrication tolerance (tolerance.cpp) --------------------------------------------------
std::vector<ToleranceResult> analyze_tolerance(const MetalensDesign& lens, const UnitCellLibrary& lib,
                                               double focal_length_um, double wavelength_um, double diameter_um,
                                               const std::vector<double>& sigmas_nm, int trials, unsigned seed) {
    std::vector<ToleranceResult> out;
    for (double sigma_nm : sigmas_nm) {
        const double sigma_fill = (sigma_nm / 1000.0) / lens.period_um;  // CD error -> fill fraction
        const int n = std::max(1, trials);
        double sum = 0.0, sum2 = 0.0, worst = 1e300;
        for (int t = 0; t < n; ++t) {
            // per-trial stream as tolerance.cpp:26-31
            std::mt19937 rng(seed + static_cast<unsigned>(t) * 7919u + static_cast<unsigned>(sigma_nm * 13.0));
            std::normal_distribution<double> g(0.0, sigma_fill);
            MetalensDesign perturbed = lens;
            for (double& f : perturbed.fill_map) f = std::clamp(f + g(rng), 0.05, 0.95);
            const double s = analyze_focus(perturbed, lib, focal_length_um, wavelength_um, diameter_um).strehl;
            sum += s;
            sum2 += s * s;
            worst = std::min(worst, s);
        }
        const double mean = sum / n;
        out.push_back({sigma_nm, mean, std::sqrt(std::max(0.0, sum2 / n - mean * mean)), worst});
    }
    return out;
}

// ---- chromatic focal shift (chromatic.cpp) -------------------------------------------------
namespace {
// First maximum of a 120-point on-axis scan over [0.55, 1.6] x f0 lambda0 / lambda
// (chromatic.cpp:46-56), on the GPU far field.
ChromaticPoint chromatic_point(const std::vector<Cell>& cells, double design_focal, double design_wavelength,
                               double lam, double design_peak) {
    constexpr int NZ = 120;
    const double k = 2.0 * pi / lam;
    const double expected = design_focal * design_wavelength / lam;
    const double zlo = 0.55 * expected, zhi = 1.6 * expected;
    double best_z = expected, best_I = -1.0;
    if (!cells.empty()) {
        const std::vector<double> I = zx_gpu(cells, 0.0, 0.0, 2, zlo, zhi, NZ, k);
        for (int j = 0; j < NZ; ++j) {
            const double v = I[static_cast<size_t>(j) * 2];
            if (v > best_I) {
                best_I = v;
                best_z = zlo + (zhi - zlo) * j / (NZ - 1);
            }
        }
    } else {
        best_I = 0.0;
    }
    return {lam, best_z, design_peak > 0 ? best_I / design_peak : 0.0};
}
double on_axis_peak(const std::vector<Cell>& cells, double z, double k) {
    return cells.empty() ? 0.0 : zx_gpu(cells, 0.0, 0.0, 2, z, z, 2, k)[0];
}
}  // namespace

std::vector<ChromaticPoint> analyze_chromatic(const MetalensDesign& lens, const UnitCellLibrary& lib,
                                              double design_focal, double design_wavelength, double diameter,
                                              double lambda_min, double lambda_max, int n) {
    const std::vector<Cell> cells = aperture_cells(lens, lib, diameter);
    const double peak0 = on_axis_peak(cells, design_focal, 2.0 * pi / design_wavelength);
    std::vector<ChromaticPoint> out;
    for (int i = 0; i < n; ++i) {
        const double lam = lambda_min + (lambda_max - lambda_min) * i / (n - 1);
        out.push_back(chromatic_point(cells, design_focal, design_wavelength, lam, peak0));
    }
    return out;
}

std::vector<ChromaticPoint> analyze_chromatic_dispersive(const MetalensDesign& lens,
                                                         const std::function<UnitCellLibrary(double)>& build_lib_at,
                                                         double design_focal, double design_wavelength,
                                                         double diameter, double lambda_min, double lambda_max,
                                                         int n) {
    // the aperture is fixed by the design; each wavelength's library sets the transmissions
    const double peak0 =
        on_axis_peak(aperture_cells(lens, build_lib_at(design_wavelength), diameter), design_focal,
                     2.0 * pi / design_wavelength);
    std::vector<ChromaticPoint> out;
    for (int i = 0; i < n; ++i) {
        const double lam = lambda_min + (lambda_max - lambda_min) * i / (n - 1);
        const std::vector<Cell> cells = aperture_cells(lens, build_lib_at(lam), diameter);
        out.push_back(chromatic_point(cells, design_focal, design_wavelength, lam, peak0));
    }
    return out;
}

ThroughFocus analyze_through_focus(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                                   double wavelength_um, double diameter_um) {
    const double R = diameter_um / 2.0;
    const double k = 2.0 * pi / wavelength_um;
    const std::vector<Cell> cells = aperture_cells(lens, lib, diameter_um);
    // scan window around the nominal focus, widened for low NA (throughfocus.cpp:45-49)
    const double na = std::sin(std::atan(R / focal_length_um));
    const double half = std::max(2.0 * wavelength_um / (na * na + 1e-6), 0.25 * focal_length_um);
    const double zlo = std::max(0.1 * focal_length_um, focal_length_um - half);
    const double zhi = focal_length_um + half;
    const int N = 161;
    ThroughFocus tf;
    // on-axis intensities: an x-z slice with both columns at x = 0
    const std::vector<double> onaxis = zx_gpu(cells, 0.0, 0.0, 2, zlo, zhi, N, k);
    std::vector<double> I(N);
    double peak = 0.0;
    for (int i = 0; i < N; ++i) {
        I[i] = onaxis[static_cast<size_t>(i) * 2];
        peak = std::max(peak, I[i]);
        tf.z_um.push_back(static_cast<float>(zlo + (zhi - zlo) * i / (N - 1)));
    }
    if (peak <= 0) peak = 1;
    int ipk = 0;
    for (int i = 0; i < N; ++i) {
        tf.intensity.push_back(static_cast<float>(I[i] / peak));
        if (I[i] > I[ipk]) ipk = i;
    }
    tf.z_peak_um = tf.z_um[ipk];
    const double half_lvl = peak / 2.0;  // depth of focus: axial FWHM (throughfocus.cpp:70-75)
    int lo = -1, hi = -1;
    for (int i = 0; i < N; ++i)
        if (I[i] >= half_lvl) {
            if (lo < 0) lo = i;
            hi = i;
        }
    tf.dof_um = (hi > lo && lo >= 0) ? (tf.z_um[hi] - tf.z_um[lo]) : 0.0;
    // x-z caustic on the GPU grid of the reference (201 x 201, throughfocus.cpp:80-100)
    const double dl = wavelength_um * focal_length_um / std::max(diameter_um, 1e-6);
    const double Wx = std::max(8.0 * dl, 3.0);
    tf.caustic_xmin = -Wx;
    tf.caustic_xmax = Wx;
    tf.caustic_zmin = zlo;
    tf.caustic_zmax = zhi;
    tf.caustic_nx = tf.caustic_nz = 201;
    const std::vector<double> cmap = zx_gpu(cells, -Wx, Wx, 201, zlo, zhi, 201, k);
    double cpeak = 0.0;
    for (double v : cmap) cpeak = std::max(cpeak, v);
    if (cpeak <= 0) cpeak = 1.0;
    tf.caustic.resize(cmap.size());
    for (size_t i = 0; i < cmap.size(); ++i) tf.caustic[i] = static_cast<float>(cmap[i] / cpeak);
    return tf;
}

// ---- off-axis analyses (field.cpp) --------------------------------------------------------------
std::vector<FieldPoint> analyze_field_of_view(const MetalensDesign& lens, const UnitCellLibrary& lib,
                                              double focal_length_um, double wavelength_um, double diameter_um,
                                              const std::vector<double>& angles_deg) {
    const double k = 2.0 * pi / wavelength_um;
    const double dl = wavelength_um * focal_length_um / diameter_um;
    // peak within the window spanning the f sin and f tan spot predictions (field.cpp:35-57)
    auto peak_near = [&](double theta, double xc) {
        const double s = std::sin(theta);
        const double W = std::max(3.0 * dl, 2.0) + std::abs(focal_length_um * std::tan(theta) - focal_length_um * s);
        return peak_on_grid(aperture_cells(lens, lib, diameter_um, k * s), xc, W, focal_length_um, k);
    };
    const double on_axis_peak = peak_near(0.0, 0.0).first;
    std::vector<FieldPoint> out;
    for (double ang : angles_deg) {
        const double theta = ang * pi / 180.0;
        const auto pk = peak_near(theta, focal_length_um * std::tan(theta));
        out.push_back({ang, on_axis_peak > 0 ? pk.first / on_axis_peak : 0.0, pk.second});
    }
    return out;
}

std::vector<FieldPoint> analyze_wide_fov(const MetalensDesign& lens, const UnitCellLibrary& lib,
                                         double focal_length_um, double wavelength_um, double lens_diameter_um,
                                         double stop_diameter_um, double stop_distance_um,
                                         const std::vector<double>& angles_deg) {
    const double k = 2.0 * pi / wavelength_um;
    const double R_stop = stop_diameter_um / 2.0;
    const double dl_stop = wavelength_um * focal_length_um / stop_diameter_um;
    const std::vector<Cell> all = aperture_cells(lens, lib, lens_diameter_um);
    // only the cells under the decentred stop patch are lit (field.cpp:101-134)
    auto peak = [&](double theta, double x_patch) {
        const double s = std::sin(theta);
        const double x_sin = focal_length_um * s, x_tan = focal_length_um * std::tan(theta);
        const double xc = 0.5 * (x_sin + x_tan);
        const double W = std::max(3.0 * dl_stop, 2.0) + 0.5 * std::abs(x_tan - x_sin);
        std::vector<Cell> lit;
        for (const Cell& c : all) {
            const double dx = c.x - x_patch, dy = c.y;
            if (dx * dx + dy * dy > R_stop * R_stop) continue;
            lit.push_back({c.x, c.y, c.t * std::polar(1.0, k * s * c.x)});
        }
        return peak_on_grid(lit, xc, W, focal_length_um, k);
    };
    const double on_axis_peak = peak(0.0, 0.0).first;
    std::vector<FieldPoint> out;
    for (double ang : angles_deg) {
        const double theta = ang * pi / 180.0;
        const auto pk = peak(theta, stop_distance_um * std::tan(theta));
        out.push_back({ang, on_axis_peak > 0 ? pk.first / on_axis_peak : 0.0, pk.second});
    }
    return out;
}

FieldGrid analyze_field_grid(const MetalensDesign& lens, const UnitCellLibrary& lib, double focal_length_um,
                             double wavelength_um, double diameter_um, double max_angle_deg, int n_half, int psf_n) {
    const double k = 2.0 * pi / wavelength_um;
    const double dl = wavelength_um * focal_length_um / diameter_um;  // field.cpp:178-181
    const double W = std::max(6.0 * dl, 4.0);
    const double step = 2.0 * W / (psf_n - 1);
    struct Spot {
        double peak, fwhm_x, fwhm_y;
    };
    // peak and tangential/sagittal FWHM of one tilted-illumination PSF (field.cpp:183-211)
    auto spot_at = [&](double tx, double ty, double cx, double cy) -> Spot {
        std::vector<Cell> cells = aperture_cells(lens, lib, diameter_um);
        const double sx = std::sin(tx), sy = std::sin(ty);
        for (Cell& c : cells) c.t *= std::polar(1.0, k * (sx * c.x + sy * c.y));
        const std::vector<double> I = psf_gpu(cells, cx, cy, focal_length_um, k, psf_n, W);
        int pix = 0, piy = 0;
        double best = -1.0;
        for (int j = 0; j < psf_n; ++j)
            for (int i = 0; i < psf_n; ++i) {
                const double v = I[static_cast<size_t>(j) * psf_n + i];
                if (v > best) {
                    best = v;
                    pix = i;
                    piy = j;
                }
            }
        const double half = best / 2.0;
        auto fwhm_along = [&](bool horizontal) {
            int lo = -1, hi = -1;
            for (int s = 0; s < psf_n; ++s) {
                const size_t idx = horizontal ? static_cast<size_t>(piy) * psf_n + s : static_cast<size_t>(s) * psf_n + pix;
                if (I[idx] >= half) {
                    if (lo < 0) lo = s;
                    hi = s;
                }
            }
            return (hi > lo && lo >= 0) ? (hi - lo) * step : 0.0;
        };
        return {best, fwhm_along(true), fwhm_along(false)};
    };
    const Spot on_axis = spot_at(0.0, 0.0, 0.0, 0.0);
    const double ref = on_axis.peak > 0 ? on_axis.peak : 1.0;
    FieldGrid g;
    g.n = 2 * n_half + 1;
    g.max_angle_deg = max_angle_deg;
    g.points.reserve(static_cast<size_t>(g.n) * g.n);
    for (int jy = -n_half; jy <= n_half; ++jy) {
        const double ang_y = n_half > 0 ? max_angle_deg * jy / n_half : 0.0;
        const double ty = ang_y * pi / 180.0;
        for (int jx = -n_half; jx <= n_half; ++jx) {
            const double ang_x = n_half > 0 ? max_angle_deg * jx / n_half : 0.0;
            const double tx = ang_x * pi / 180.0;
            const double cx = focal_length_um * std::tan(tx), cy = focal_length_um * std::tan(ty);
            const Spot s = spot_at(tx, ty, cx, cy);
            g.points.push_back({ang_x, ang_y, s.peak / ref, s.fwhm_x, s.fwhm_y, cx, cy});
        }
    }
    return g;
}

namespace cuda {
bool available() { return celeris_available() != 0; }
const char* device_name() { return celeris_device_name(); }
bool propagate_psf(const double* px, const double* py, const std::complex<double>* pt, int npil, double cx,
                   double cy, double z, double k, int n, double half_window, double* out) {
    if (npil <= 0 || n <= 0) return false;  // propagate.cu:139
    return celeris_propagate_psf(px, py, reinterpret_cast<const double*>(pt), npil, cx, cy, z, k, n, half_window,
                                 out) == CELERIS_OK;
}
bool propagate_zx(const double* px, const double* py, const std::complex<double>* pt, int npil, double xmin,
                  double xmax, int nx, double zmin, double zmax, int nz, double k, double* out) {
    if (npil <= 0 || nx <= 1 || nz <= 1) return false;  // propagate.cu:201
    return celeris_propagate_zx(px, py, reinterpret_cast<const double*>(pt), npil, xmin, xmax, nx, zmin, zmax, nz,
                                k, out) == CELERIS_OK;
}
bool geev(const std::complex<double>* A, int n, std::complex<double>* w, std::complex<double>* vr) {
    return celeris_eig_general(reinterpret_cast<const double*>(A), n, reinterpret_cast<double*>(w),
                               reinterpret_cast<double*>(vr)) == CELERIS_OK;
}
bool geev_batched(const std::complex<double>* As, int n, int batch, std::complex<double>* ws,
                  std::complex<double>* vrs, int /*streams*/) {
    return celeris_eig_general_batch(reinterpret_cast<const double*>(As), n, batch, reinterpret_cast<double*>(ws),
                                     reinterpret_cast<double*>(vrs), nullptr) == CELERIS_OK;
}
}  // namespace cuda

}  // namespace celeris
