// pybind11 module `_celeris`: the reference's Python surface for the hot path
// (bindings/python/celeris_module.cpp:54-439 names and arguments), over the C++
// host mirror in celeris.hpp. Maps are returned as numpy arrays like the
// reference (PsfMap.intensity, MetalensDesign.fill_map).
#include <pybind11/complex.h>
#include <pybind11/functional.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "celeris.hpp"

namespace py = pybind11;
using namespace celeris;

static py::array_t<double> to_2d(const std::vector<double>& v, int rows, int cols) {
    py::array_t<double> a({rows, cols});
    std::copy(v.begin(), v.end(), a.mutable_data());
    return a;
}

static std::vector<double> from_square(const py::array_t<double>& arr, int& n) {
    auto buf = py::array_t<double, py::array::c_style | py::array::forcecast>(arr);
    if (buf.ndim() != 2 || buf.shape(0) != buf.shape(1))
        throw std::runtime_error("freeform phase map must be a square 2D array");
    n = static_cast<int>(buf.shape(0));
    return std::vector<double>(buf.data(), buf.data() + static_cast<size_t>(n) * n);
}

PYBIND11_MODULE(_celeris, m) {
    m.doc() = "CELERIS hot path on B200 (sm_100a kernels behind a C ABI): far-field RS sum and 2D RCWA.";

    py::enum_<Pol>(m, "Pol").value("TE", Pol::TE).value("TM", Pol::TM);
    py::enum_<MetaShape>(m, "MetaShape")
        .value("Rectangle", MetaShape::Rectangle)
        .value("Ellipse", MetaShape::Ellipse)
        .value("Cross", MetaShape::Cross)
        .value("Ring", MetaShape::Ring);
    py::enum_<PhaseProfileKind>(m, "PhaseProfileKind")
        .value("Focusing", PhaseProfileKind::Focusing)
        .value("Quadratic", PhaseProfileKind::Quadratic)
        .value("Vortex", PhaseProfileKind::Vortex)
        .value("Deflector", PhaseProfileKind::Deflector)
        .value("Axicon", PhaseProfileKind::Axicon)
        .value("Freeform", PhaseProfileKind::Freeform);

    py::class_<Material>(m, "Material")
        .def_static("constant", &Material::constant, py::arg("n"), py::arg("name") = "constant")
        .def_static("sellmeier", &Material::sellmeier, py::arg("bc_terms"), py::arg("name") = "sellmeier")
        .def_static("tabulated", &Material::tabulated, py::arg("wavelength_um"), py::arg("n"), py::arg("k"),
                    py::arg("name") = "tabulated")
        .def("index", &Material::index, py::arg("wavelength_um"))
        .def("permittivity", &Material::permittivity, py::arg("wavelength_um"))
        .def_property_readonly("name", &Material::name)
        .def("__repr__", [](const Material& x) { return "<celeris.Material '" + x.name() + "'>"; });

    auto mats = m.def_submodule("materials", "Built-in published materials.");
    mats.def("air", [] { return materials::air(); });
    mats.def("bk7", [] { return materials::bk7(); });
    mats.def("fused_silica", [] { return materials::fused_silica(); });
    mats.def("silicon_nitride", [] { return materials::silicon_nitride(); });

    py::class_<RectCell2D>(m, "RectCell2D")
        .def(py::init([](Material pillar, Material background, double fx, double fy, double h, MetaShape shape,
                         double param) { return RectCell2D{pillar, background, fx, fy, h, shape, param}; }),
             py::arg("pillar"), py::arg("background"), py::arg("fill_x"), py::arg("fill_y"),
             py::arg("thickness_um"), py::arg("shape") = MetaShape::Rectangle, py::arg("shape_param") = 0.5)
        .def_static("homogeneous", &RectCell2D::homogeneous, py::arg("material"), py::arg("thickness_um"))
        .def_readwrite("pillar", &RectCell2D::pillar)
        .def_readwrite("background", &RectCell2D::background)
        .def_readwrite("fill_x", &RectCell2D::fill_x)
        .def_readwrite("fill_y", &RectCell2D::fill_y)
        .def_readwrite("thickness_um", &RectCell2D::thickness_um)
        .def_readwrite("shape", &RectCell2D::shape)
        .def_readwrite("shape_param", &RectCell2D::shape_param)
        .def_readwrite("rotation_rad", &RectCell2D::rotation_rad);

    py::class_<Rcwa2DStack>(m, "Rcwa2DStack")
        .def(py::init([](double px, double py_, std::vector<RectCell2D> layers) {
                 return Rcwa2DStack{px, py_, std::move(layers)};
             }),
             py::arg("period_x_um"), py::arg("period_y_um"), py::arg("layers"))
        .def_readwrite("period_x_um", &Rcwa2DStack::period_x_um)
        .def_readwrite("period_y_um", &Rcwa2DStack::period_y_um)
        .def_readwrite("layers", &Rcwa2DStack::layers);

    py::class_<Rcwa2DResult>(m, "Rcwa2DResult")
        .def_readonly("R", &Rcwa2DResult::R)
        .def_readonly("T", &Rcwa2DResult::T)
        .def_readonly("sum_de", &Rcwa2DResult::sum_de)
        .def_readonly("de_t0", &Rcwa2DResult::de_t0)
        .def_readonly("de_r0", &Rcwa2DResult::de_r0)
        .def_readonly("tx0", &Rcwa2DResult::tx0)
        .def_readonly("ty0", &Rcwa2DResult::ty0);

    m.def("solve_rcwa_2d",
          [](const Material& inc, const Rcwa2DStack& st, const Material& sub, double wl, double th, double ph,
             cdouble ex, cdouble ey, int Mx, int My) { return solve_rcwa_2d(inc, st, sub, wl, th, ph, ex, ey, Mx, My); },
          py::arg("incident"), py::arg("stack"), py::arg("substrate"), py::arg("wavelength_um"),
          py::arg("theta_rad"), py::arg("phi_rad"), py::arg("Ex0"), py::arg("Ey0"), py::arg("Mx"), py::arg("My"));
    m.def(
        "eig_general",
        [](py::array_t<std::complex<double>, py::array::f_style | py::array::forcecast> A) {
            if (A.ndim() != 2 || A.shape(0) != A.shape(1)) throw std::invalid_argument("eig_general: square matrix");
            const int n = static_cast<int>(A.shape(0));
            std::vector<cdouble> a(A.data(), A.data() + static_cast<size_t>(n) * n), vals, vecs;
            eig_general(a, n, vals, vecs);
            py::array_t<std::complex<double>> ev(n);
            std::copy(vals.begin(), vals.end(), ev.mutable_data());
            py::array_t<std::complex<double>, py::array::f_style> V({n, n});
            std::copy(vecs.begin(), vecs.end(), V.mutable_data());
            return py::make_tuple(ev, V);
        },
        py::arg("A"));
    py::class_<OrderEfficiency>(m, "OrderEfficiency")
        .def_readonly("p", &OrderEfficiency::p)
        .def_readonly("q", &OrderEfficiency::q)
        .def_readonly("de_t", &OrderEfficiency::de_t)
        .def_readonly("de_r", &OrderEfficiency::de_r)
        .def_readonly("prop_t", &OrderEfficiency::prop_t)
        .def_readonly("prop_r", &OrderEfficiency::prop_r);
    m.def("solve_rcwa_2d_orders",
          [](const Material& inc, const Rcwa2DStack& st, const Material& sub, double wl, double th, double ph,
             cdouble ex, cdouble ey, int Mx, int My) {
              std::vector<OrderEfficiency> o;
              Rcwa2DResult r = solve_rcwa_2d(inc, st, sub, wl, th, ph, ex, ey, Mx, My, &o);
              return py::make_tuple(r, o);
          },
          py::arg("incident"), py::arg("stack"), py::arg("substrate"), py::arg("wavelength_um"),
          py::arg("theta_rad"), py::arg("phi_rad"), py::arg("Ex0"), py::arg("Ey0"), py::arg("Mx"), py::arg("My"));
    py::class_<EfficiencyBudget>(m, "EfficiencyBudget")
        .def_readonly("reflection", &EfficiencyBudget::reflection)
        .def_readonly("transmission", &EfficiencyBudget::transmission)
        .def_readonly("absorption", &EfficiencyBudget::absorption)
        .def_readonly("t_zero", &EfficiencyBudget::t_zero)
        .def_readonly("r_zero", &EfficiencyBudget::r_zero)
        .def_readonly("t_stray", &EfficiencyBudget::t_stray)
        .def_readonly("r_stray", &EfficiencyBudget::r_stray)
        .def_readonly("n_prop_t", &EfficiencyBudget::n_prop_t)
        .def_readonly("n_prop_r", &EfficiencyBudget::n_prop_r)
        .def_readonly("orders", &EfficiencyBudget::orders);
    m.def("analyze_efficiency", &analyze_efficiency, py::arg("incident"), py::arg("pillar"), py::arg("background"),
          py::arg("substrate"), py::arg("period_x_um"), py::arg("period_y_um"), py::arg("fill_x"), py::arg("fill_y"),
          py::arg("thickness_um"), py::arg("wavelength_um"), py::arg("Ex0"), py::arg("Ey0"), py::arg("M"),
          py::arg("shape") = MetaShape::Rectangle, py::arg("shape_param") = 0.5);

    py::class_<UnitCellLibrary>(m, "UnitCellLibrary")
        .def(py::init<>())
        .def_readwrite("period_um", &UnitCellLibrary::period_um)
        .def_readwrite("wavelength_um", &UnitCellLibrary::wavelength_um)
        .def_readwrite("thickness_um", &UnitCellLibrary::thickness_um)
        .def_readwrite("fill", &UnitCellLibrary::fill)
        .def_readwrite("phase", &UnitCellLibrary::phase)
        .def_readwrite("amplitude", &UnitCellLibrary::amplitude)
        .def("phase_span", &UnitCellLibrary::phase_span)
        .def("coverage", &UnitCellLibrary::coverage)
        .def("lookup", &UnitCellLibrary::lookup, py::arg("target_phase_rad"))
        .def("lookup_weighted", &UnitCellLibrary::lookup_weighted, py::arg("target_phase_rad"),
             py::arg("amplitude_weight"))
        .def("transmission_for_fill", &UnitCellLibrary::transmission_for_fill, py::arg("fill"));

    m.def("build_unit_cell_library", &build_unit_cell_library, py::arg("pillar"), py::arg("background"),
          py::arg("incident"), py::arg("substrate"), py::arg("period_um"), py::arg("wavelength_um"),
          py::arg("thickness_um"), py::arg("fill_min"), py::arg("fill_max"), py::arg("n_samples"), py::arg("M"),
          py::arg("shape") = MetaShape::Rectangle, py::arg("shape_param") = 0.5);

    py::class_<HeightSweepEntry>(m, "HeightSweepEntry")
        .def_readonly("thickness_um", &HeightSweepEntry::thickness_um)
        .def_readonly("coverage_deg", &HeightSweepEntry::coverage_deg)
        .def_readonly("mean_transmittance", &HeightSweepEntry::mean_transmittance);
    py::class_<HeightOptResult>(m, "HeightOptResult")
        .def_readonly("best_thickness_um", &HeightOptResult::best_thickness_um)
        .def_readonly("coverage_deg", &HeightOptResult::coverage_deg)
        .def_readonly("mean_transmittance", &HeightOptResult::mean_transmittance)
        .def_readonly("reached_target", &HeightOptResult::reached_target)
        .def_readonly("coverage_target_deg", &HeightOptResult::coverage_target_deg)
        .def_readonly("sweep", &HeightOptResult::sweep)
        .def_readonly("best_library", &HeightOptResult::best_library);
    m.def("optimize_height_for_2pi", &optimize_height_for_2pi, py::arg("pillar"), py::arg("background"),
          py::arg("incident"), py::arg("substrate"), py::arg("period_um"), py::arg("wavelength_um"),
          py::arg("thick_lo"), py::arg("thick_hi"), py::arg("n_heights"), py::arg("fill_min"), py::arg("fill_max"),
          py::arg("fill_samples"), py::arg("M"), py::arg("coverage_target_deg") = 330.0,
          py::arg("shape") = MetaShape::Rectangle, py::arg("shape_param") = 0.5);

    py::class_<MetalensDesign>(m, "MetalensDesign")
        .def_readonly("n_cells", &MetalensDesign::n_cells)
        .def_readonly("period_um", &MetalensDesign::period_um)
        .def_readonly("rms_phase_error_deg", &MetalensDesign::rms_phase_error_deg)
        .def_readonly("mean_amplitude", &MetalensDesign::mean_amplitude)
        .def_property_readonly("fill_map",
                               [](const MetalensDesign& d) { return to_2d(d.fill_map, d.n_cells, d.n_cells); });

    py::class_<PhaseProfile>(m, "PhaseProfile")
        .def(py::init<>())
        .def_readwrite("kind", &PhaseProfile::kind)
        .def_readwrite("focal_length_um", &PhaseProfile::focal_length_um)
        .def_readwrite("topological_charge", &PhaseProfile::topological_charge)
        .def_readwrite("deflect_deg", &PhaseProfile::deflect_deg)
        .def_readwrite("deflect_azimuth_deg", &PhaseProfile::deflect_azimuth_deg)
        .def_readwrite("axicon_deg", &PhaseProfile::axicon_deg)
        .def_readwrite("freeform_n", &PhaseProfile::freeform_n)
        .def_readwrite("freeform_extent_um", &PhaseProfile::freeform_extent_um)
        .def_property(
            "freeform_phase",
            [](const PhaseProfile& p) { return to_2d(p.freeform_phase_rad, p.freeform_n, p.freeform_n); },
            [](PhaseProfile& p, const py::array_t<double>& a) {
                int n = 0;
                p.freeform_phase_rad = from_square(a, n);
                p.freeform_n = n;
            })
        .def_static("focusing",
                    [](double f) {
                        PhaseProfile p;
                        p.kind = PhaseProfileKind::Focusing;
                        p.focal_length_um = f;
                        return p;
                    },
                    py::arg("focal_length_um"));
    m.def("phase_profile_value", &phase_profile_value, py::arg("profile"), py::arg("x"), py::arg("y"),
          py::arg("wavelength_um"));
    m.def("load_freeform_phase", &load_freeform_phase, py::arg("path"), py::arg("extent_um"));
    m.def("design_metalens", py::overload_cast<const UnitCellLibrary&, double, double, double>(&design_metalens),
          py::arg("lib"), py::arg("focal_length_um"), py::arg("diameter_um"), py::arg("amplitude_weight") = 0.25);
    m.def("design_metalens",
          py::overload_cast<const UnitCellLibrary&, const PhaseProfile&, double, double>(&design_metalens),
          py::arg("lib"), py::arg("profile"), py::arg("diameter_um"), py::arg("amplitude_weight") = 0.25);

    py::class_<PillarTarget>(m, "PillarTarget")
        .def(py::init([](double wl, double ph, double w) { return PillarTarget{wl, ph, w}; }),
             py::arg("wavelength_um"), py::arg("target_phase_rad"), py::arg("amplitude_weight") = 0.25)
        .def_readwrite("wavelength_um", &PillarTarget::wavelength_um)
        .def_readwrite("target_phase_rad", &PillarTarget::target_phase_rad)
        .def_readwrite("amplitude_weight", &PillarTarget::amplitude_weight);
    py::class_<OptimizedPillar>(m, "OptimizedPillar")
        .def_readonly("fill", &OptimizedPillar::fill)
        .def_readonly("thickness_um", &OptimizedPillar::thickness_um)
        .def_readonly("achieved_phase_rad", &OptimizedPillar::achieved_phase_rad)
        .def_readonly("achieved_amplitude", &OptimizedPillar::achieved_amplitude)
        .def_readonly("loss", &OptimizedPillar::loss)
        .def_readonly("iterations", &OptimizedPillar::iterations);
    m.def("optimize_pillar", &optimize_pillar, py::arg("pillar"), py::arg("background"), py::arg("incident"),
          py::arg("substrate"), py::arg("period_um"), py::arg("target"), py::arg("M"), py::arg("fill0"),
          py::arg("thickness0"), py::arg("max_iters"));

    py::class_<FocalAnalysis>(m, "FocalAnalysis")
        .def_readonly("strehl", &FocalAnalysis::strehl)
        .def_readonly("phase_strehl", &FocalAnalysis::phase_strehl)
        .def_readonly("fwhm_um", &FocalAnalysis::fwhm_um)
        .def_readonly("diffraction_limit_um", &FocalAnalysis::diffraction_limit_um)
        .def_readonly("encircled_energy", &FocalAnalysis::encircled_energy);
    m.def("analyze_focus", &analyze_focus, py::arg("lens"), py::arg("lib"), py::arg("focal_length_um"),
          py::arg("wavelength_um"), py::arg("diameter_um"));

    py::class_<PsfMap>(m, "PsfMap")
        .def_readonly("n", &PsfMap::n)
        .def_readonly("half_window_um", &PsfMap::half_window_um)
        .def_property_readonly("intensity", [](const PsfMap& p) { return to_2d(p.intensity, p.n, p.n); });
    m.def("compute_psf", &compute_psf, py::arg("lens"), py::arg("lib"), py::arg("focal_length_um"),
          py::arg("wavelength_um"), py::arg("diameter_um"), py::arg("n"), py::arg("half_window_um"));
    m.def("propagate_pillars", &propagate_pillars, py::arg("px"), py::arg("py"), py::arg("t"), py::arg("cx"),
          py::arg("cy"), py::arg("z"), py::arg("wavelength_um"), py::arg("n"), py::arg("half_window_um"));

    py::class_<FieldPsf>(m, "FieldPsf")
        .def_readonly("psf", &FieldPsf::psf)
        .def_readonly("angle_deg", &FieldPsf::angle_deg)
        .def_readonly("cx_um", &FieldPsf::cx_um)
        .def_readonly("rel_strehl", &FieldPsf::rel_strehl);
    m.def("compute_psf_field", &compute_psf_field, py::arg("lens"), py::arg("lib"), py::arg("focal_length_um"),
          py::arg("wavelength_um"), py::arg("diameter_um"), py::arg("angle_deg"), py::arg("n"),
          py::arg("half_window_um"), py::arg("on_axis_peak") = 0.0);

    py::class_<ThroughFocus>(m, "ThroughFocus")
        .def_property_readonly("z_um", [](const ThroughFocus& t) { return py::array_t<float>(t.z_um.size(), t.z_um.data()); })
        .def_property_readonly("intensity",
                               [](const ThroughFocus& t) { return py::array_t<float>(t.intensity.size(), t.intensity.data()); })
        .def_readonly("z_peak_um", &ThroughFocus::z_peak_um)
        .def_readonly("dof_um", &ThroughFocus::dof_um)
        .def_readonly("caustic_nx", &ThroughFocus::caustic_nx)
        .def_readonly("caustic_nz", &ThroughFocus::caustic_nz)
        .def_readonly("caustic_xmin", &ThroughFocus::caustic_xmin)
        .def_readonly("caustic_xmax", &ThroughFocus::caustic_xmax)
        .def_readonly("caustic_zmin", &ThroughFocus::caustic_zmin)
        .def_readonly("caustic_zmax", &ThroughFocus::caustic_zmax)
        .def_property_readonly("caustic", [](const ThroughFocus& t) {
            py::array_t<float> a({t.caustic_nz, t.caustic_nx});
            std::copy(t.caustic.begin(), t.caustic.end(), a.mutable_data());
            return a;
        });
    m.def("analyze_through_focus", &analyze_through_focus, py::arg("lens"), py::arg("lib"),
          py::arg("focal_length_um"), py::arg("wavelength_um"), py::arg("diameter_um"));

    py::class_<ToleranceResult>(m, "ToleranceResult")
        .def_readonly("sigma_nm", &ToleranceResult::sigma_nm)
        .def_readonly("mean_strehl", &ToleranceResult::mean_strehl)
        .def_readonly("std_strehl", &ToleranceResult::std_strehl)
        .def_readonly("worst_strehl", &ToleranceResult::worst_strehl);
    m.def("analyze_tolerance", &analyze_tolerance, py::arg("lens"), py::arg("lib"), py::arg("focal_length_um"),
          py::arg("wavelength_um"), py::arg("diameter_um"), py::arg("sigmas_nm"), py::arg("trials"),
          py::arg("seed"));
    py::class_<ChromaticPoint>(m, "ChromaticPoint")
        .def_readonly("wavelength_um", &ChromaticPoint::wavelength_um)
        .def_readonly("focal_length_um", &ChromaticPoint::focal_length_um)
        .def_readonly("rel_peak", &ChromaticPoint::rel_peak);
    m.def("analyze_chromatic", &analyze_chromatic, py::arg("lens"), py::arg("lib"), py::arg("design_focal"),
          py::arg("design_wavelength"), py::arg("diameter"), py::arg("lambda_min"), py::arg("lambda_max"),
          py::arg("n"));
    m.def("analyze_chromatic_dispersive", &analyze_chromatic_dispersive, py::arg("lens"), py::arg("build_lib_at"),
          py::arg("design_focal"), py::arg("design_wavelength"), py::arg("diameter"), py::arg("lambda_min"),
          py::arg("lambda_max"), py::arg("n"));
    py::class_<FieldPoint>(m, "FieldPoint")
        .def_readonly("angle_deg", &FieldPoint::angle_deg)
        .def_readonly("rel_strehl", &FieldPoint::rel_strehl)
        .def_readonly("spot_shift_um", &FieldPoint::spot_shift_um);
    m.def("analyze_field_of_view", &analyze_field_of_view, py::arg("lens"), py::arg("lib"),
          py::arg("focal_length_um"), py::arg("wavelength_um"), py::arg("diameter_um"), py::arg("angles_deg"));
    m.def("analyze_wide_fov", &analyze_wide_fov, py::arg("lens"), py::arg("lib"), py::arg("focal_length_um"),
          py::arg("wavelength_um"), py::arg("lens_diameter_um"), py::arg("stop_diameter_um"),
          py::arg("stop_distance_um"), py::arg("angles_deg"));
    py::class_<FieldGridPoint>(m, "FieldGridPoint")
        .def_readonly("theta_x_deg", &FieldGridPoint::theta_x_deg)
        .def_readonly("theta_y_deg", &FieldGridPoint::theta_y_deg)
        .def_readonly("rel_strehl", &FieldGridPoint::rel_strehl)
        .def_readonly("fwhm_x_um", &FieldGridPoint::fwhm_x_um)
        .def_readonly("fwhm_y_um", &FieldGridPoint::fwhm_y_um)
        .def_readonly("cx_um", &FieldGridPoint::cx_um)
        .def_readonly("cy_um", &FieldGridPoint::cy_um);
    py::class_<FieldGrid>(m, "FieldGrid")
        .def_readonly("n", &FieldGrid::n)
        .def_readonly("max_angle_deg", &FieldGrid::max_angle_deg)
        .def_readonly("points", &FieldGrid::points);
    m.def("analyze_field_grid", &analyze_field_grid, py::arg("lens"), py::arg("lib"), py::arg("focal_length_um"),
          py::arg("wavelength_um"), py::arg("diameter_um"), py::arg("max_angle_deg"), py::arg("n_half"),
          py::arg("psf_n"));

    // ---- library builders on the batched RCWA, designs and on-axis checks
    m.def("build_unit_cell_library_stack", &build_unit_cell_library_stack, py::arg("stack"), py::arg("active_layer"),
          py::arg("incident"), py::arg("substrate"), py::arg("wavelength_um"), py::arg("fill_min"),
          py::arg("fill_max"), py::arg("n_samples"), py::arg("M"));
    py::class_<MetaAtomSpec>(m, "MetaAtomSpec")
        .def(py::init([](MetaShape shape, double fx, double fy, double h, double sp) {
                 return MetaAtomSpec{shape, fx, fy, h, sp};
             }),
             py::arg("shape") = MetaShape::Rectangle, py::arg("fill_x") = 0.5, py::arg("fill_y") = 0.5,
             py::arg("thickness_um") = 0.6, py::arg("shape_param") = 0.5)
        .def_readwrite("shape", &MetaAtomSpec::shape)
        .def_readwrite("fill_x", &MetaAtomSpec::fill_x)
        .def_readwrite("fill_y", &MetaAtomSpec::fill_y)
        .def_readwrite("thickness_um", &MetaAtomSpec::thickness_um)
        .def_readwrite("shape_param", &MetaAtomSpec::shape_param);
    py::class_<DispersiveAtom>(m, "DispersiveAtom")
        .def(py::init<>())
        .def_readwrite("fill", &DispersiveAtom::fill)
        .def_readwrite("thickness_um", &DispersiveAtom::thickness_um)
        .def_readwrite("shape", &DispersiveAtom::shape)
        .def_readwrite("fill_x", &DispersiveAtom::fill_x)
        .def_readwrite("fill_y", &DispersiveAtom::fill_y)
        .def_readwrite("shape_param", &DispersiveAtom::shape_param)
        .def_readwrite("phase0_rad", &DispersiveAtom::phase0_rad)
        .def_readwrite("group_delay_fs", &DispersiveAtom::group_delay_fs)
        .def_readwrite("mean_amplitude", &DispersiveAtom::mean_amplitude)
        .def_readwrite("phase_rad", &DispersiveAtom::phase_rad)
        .def_readwrite("amplitude", &DispersiveAtom::amplitude);
    py::class_<DispersiveLibrary>(m, "DispersiveLibrary")
        .def(py::init<>())
        .def_readwrite("wavelengths_um", &DispersiveLibrary::wavelengths_um)
        .def_readwrite("center_wavelength_um", &DispersiveLibrary::center_wavelength_um)
        .def_readwrite("center_index", &DispersiveLibrary::center_index)
        .def_readwrite("period_um", &DispersiveLibrary::period_um)
        .def_readwrite("n_fill", &DispersiveLibrary::n_fill)
        .def_readwrite("n_height", &DispersiveLibrary::n_height)
        .def_readwrite("atoms", &DispersiveLibrary::atoms)
        .def_readwrite("gd_min_fs", &DispersiveLibrary::gd_min_fs)
        .def_readwrite("gd_max_fs", &DispersiveLibrary::gd_max_fs);
    m.def("build_dispersive_library_from_specs", &build_dispersive_library_from_specs, py::arg("pillar"),
          py::arg("background"), py::arg("incident"), py::arg("substrate"), py::arg("period_um"),
          py::arg("band_wavelengths_um"), py::arg("center_wavelength_um"), py::arg("specs"), py::arg("M"));
    m.def("build_dispersive_library", &build_dispersive_library, py::arg("pillar"), py::arg("background"),
          py::arg("incident"), py::arg("substrate"), py::arg("period_um"), py::arg("band_wavelengths_um"),
          py::arg("center_wavelength_um"), py::arg("fill_min"), py::arg("fill_max"), py::arg("n_fills"),
          py::arg("thick_lo"), py::arg("thick_hi"), py::arg("n_heights"), py::arg("M"));
    m.def("build_single_etch_library", &build_single_etch_library, py::arg("pillar"), py::arg("background"),
          py::arg("incident"), py::arg("substrate"), py::arg("period_um"), py::arg("band_wavelengths_um"),
          py::arg("center_wavelength_um"), py::arg("fill_min"), py::arg("fill_max"), py::arg("n_fills"),
          py::arg("thickness_um"), py::arg("M"));
    py::class_<AchromaticDesign>(m, "AchromaticDesign")
        .def(py::init<>())
        .def_readwrite("n_cells", &AchromaticDesign::n_cells)
        .def_readwrite("period_um", &AchromaticDesign::period_um)
        .def_readwrite("atom_index", &AchromaticDesign::atom_index)
        .def_readwrite("fill_map", &AchromaticDesign::fill_map)
        .def_readwrite("thickness_map", &AchromaticDesign::thickness_map)
        .def_readwrite("center_wavelength_um", &AchromaticDesign::center_wavelength_um)
        .def_readwrite("focal_length_um", &AchromaticDesign::focal_length_um)
        .def_readwrite("diameter_um", &AchromaticDesign::diameter_um)
        .def_readwrite("rms_phase_error_deg", &AchromaticDesign::rms_phase_error_deg)
        .def_readwrite("rms_group_delay_error_fs", &AchromaticDesign::rms_group_delay_error_fs)
        .def_readwrite("mean_amplitude", &AchromaticDesign::mean_amplitude)
        .def_readwrite("required_gd_span_fs", &AchromaticDesign::required_gd_span_fs)
        .def_readwrite("available_gd_span_fs", &AchromaticDesign::available_gd_span_fs)
        .def_readwrite("gd_coverage", &AchromaticDesign::gd_coverage)
        .def_readwrite("single_height", &AchromaticDesign::single_height)
        .def_readwrite("min_height_um", &AchromaticDesign::min_height_um)
        .def_readwrite("max_height_um", &AchromaticDesign::max_height_um);
    m.def("design_achromatic_metalens", &design_achromatic_metalens, py::arg("lib"), py::arg("focal_length_um"),
          py::arg("diameter_um"), py::arg("gd_weight") = 1.0, py::arg("amplitude_weight") = 0.25);
    py::class_<AchromaticFocalPoint>(m, "AchromaticFocalPoint")
        .def_readonly("wavelength_um", &AchromaticFocalPoint::wavelength_um)
        .def_readonly("focal_length_um", &AchromaticFocalPoint::focal_length_um)
        .def_readonly("rel_peak", &AchromaticFocalPoint::rel_peak);
    m.def("verify_achromatic_focus", &verify_achromatic_focus, py::arg("lib"), py::arg("design"));
    m.def("to_metalens_design", &to_metalens_design, py::arg("design"));
    py::class_<DispersivePbAtom>(m, "DispersivePbAtom")
        .def(py::init<>())
        .def_readwrite("fill_x", &DispersivePbAtom::fill_x)
        .def_readwrite("fill_y", &DispersivePbAtom::fill_y)
        .def_readwrite("thickness_um", &DispersivePbAtom::thickness_um)
        .def_readwrite("phase0_rad", &DispersivePbAtom::phase0_rad)
        .def_readwrite("group_delay_fs", &DispersivePbAtom::group_delay_fs)
        .def_readwrite("mean_amplitude", &DispersivePbAtom::mean_amplitude)
        .def_readwrite("mean_conversion", &DispersivePbAtom::mean_conversion)
        .def_readwrite("retardance_center_deg", &DispersivePbAtom::retardance_center_deg)
        .def_readwrite("cross", &DispersivePbAtom::cross);
    py::class_<DispersivePbLibrary>(m, "DispersivePbLibrary")
        .def(py::init<>())
        .def_readwrite("wavelengths_um", &DispersivePbLibrary::wavelengths_um)
        .def_readwrite("center_wavelength_um", &DispersivePbLibrary::center_wavelength_um)
        .def_readwrite("center_index", &DispersivePbLibrary::center_index)
        .def_readwrite("period_um", &DispersivePbLibrary::period_um)
        .def_readwrite("thickness_um", &DispersivePbLibrary::thickness_um)
        .def_readwrite("n_fill", &DispersivePbLibrary::n_fill)
        .def_readwrite("atoms", &DispersivePbLibrary::atoms)
        .def_readwrite("gd_min_fs", &DispersivePbLibrary::gd_min_fs)
        .def_readwrite("gd_max_fs", &DispersivePbLibrary::gd_max_fs);
    m.def("build_dispersive_pb_library", &build_dispersive_pb_library, py::arg("pillar"), py::arg("background"),
          py::arg("incident"), py::arg("substrate"), py::arg("period_um"), py::arg("band_wavelengths_um"),
          py::arg("center_wavelength_um"), py::arg("fill_min"), py::arg("fill_max"), py::arg("n_fills"),
          py::arg("thickness_um"), py::arg("M"), py::arg("min_amplitude") = 0.30);
    py::class_<PbAchromaticDesign>(m, "PbAchromaticDesign")
        .def(py::init<>())
        .def_readwrite("n_cells", &PbAchromaticDesign::n_cells)
        .def_readwrite("period_um", &PbAchromaticDesign::period_um)
        .def_readwrite("thickness_um", &PbAchromaticDesign::thickness_um)
        .def_readwrite("handedness", &PbAchromaticDesign::handedness)
        .def_readwrite("atom_index", &PbAchromaticDesign::atom_index)
        .def_readwrite("rotation_rad", &PbAchromaticDesign::rotation_rad)
        .def_readwrite("fill_x_map", &PbAchromaticDesign::fill_x_map)
        .def_readwrite("fill_y_map", &PbAchromaticDesign::fill_y_map)
        .def_readwrite("center_wavelength_um", &PbAchromaticDesign::center_wavelength_um)
        .def_readwrite("focal_length_um", &PbAchromaticDesign::focal_length_um)
        .def_readwrite("diameter_um", &PbAchromaticDesign::diameter_um)
        .def_readwrite("rms_phase_error_deg", &PbAchromaticDesign::rms_phase_error_deg)
        .def_readwrite("rms_group_delay_error_fs", &PbAchromaticDesign::rms_group_delay_error_fs)
        .def_readwrite("mean_amplitude", &PbAchromaticDesign::mean_amplitude)
        .def_readwrite("mean_conversion", &PbAchromaticDesign::mean_conversion)
        .def_readwrite("required_gd_span_fs", &PbAchromaticDesign::required_gd_span_fs)
        .def_readwrite("available_gd_span_fs", &PbAchromaticDesign::available_gd_span_fs)
        .def_readwrite("gd_coverage", &PbAchromaticDesign::gd_coverage);
    m.def("design_pb_achromatic_metalens", &design_pb_achromatic_metalens, py::arg("lib"),
          py::arg("focal_length_um"), py::arg("diameter_um"), py::arg("handedness") = 1, py::arg("gd_weight") = 1.0,
          py::arg("amplitude_weight") = 0.25);
    m.def("verify_pb_achromatic_focus", &verify_pb_achromatic_focus, py::arg("lib"), py::arg("design"));
    py::class_<PolarCell>(m, "PolarCell")
        .def(py::init<>())
        .def_readwrite("fill_x", &PolarCell::fill_x)
        .def_readwrite("fill_y", &PolarCell::fill_y)
        .def_readwrite("phase_x", &PolarCell::phase_x)
        .def_readwrite("phase_y", &PolarCell::phase_y)
        .def_readwrite("amp_x", &PolarCell::amp_x)
        .def_readwrite("amp_y", &PolarCell::amp_y);
    py::class_<PolarizationLibrary>(m, "PolarizationLibrary")
        .def(py::init<>())
        .def_readwrite("period_um", &PolarizationLibrary::period_um)
        .def_readwrite("wavelength_um", &PolarizationLibrary::wavelength_um)
        .def_readwrite("thickness_um", &PolarizationLibrary::thickness_um)
        .def_readwrite("cells", &PolarizationLibrary::cells)
        .def("lookup", &PolarizationLibrary::lookup, py::arg("target_x"), py::arg("target_y"),
             py::arg("amplitude_weight") = 0.0);
    m.def("build_polarization_library", &build_polarization_library, py::arg("pillar"), py::arg("background"),
          py::arg("incident"), py::arg("substrate"), py::arg("period_um"), py::arg("wavelength_um"),
          py::arg("thickness_um"), py::arg("fill_min"), py::arg("fill_max"), py::arg("n_samples"), py::arg("M"));
    py::class_<PolarMetalensDesign>(m, "PolarMetalensDesign")
        .def_readonly("n_cells", &PolarMetalensDesign::n_cells)
        .def_readonly("period_um", &PolarMetalensDesign::period_um)
        .def_readonly("fill_x", &PolarMetalensDesign::fill_x)
        .def_readonly("fill_y", &PolarMetalensDesign::fill_y)
        .def_readonly("t_x", &PolarMetalensDesign::t_x)
        .def_readonly("t_y", &PolarMetalensDesign::t_y)
        .def_readonly("rms_phase_error_x_deg", &PolarMetalensDesign::rms_phase_error_x_deg)
        .def_readonly("rms_phase_error_y_deg", &PolarMetalensDesign::rms_phase_error_y_deg)
        .def_readonly("mean_amp_x", &PolarMetalensDesign::mean_amp_x)
        .def_readonly("mean_amp_y", &PolarMetalensDesign::mean_amp_y);
    m.def("design_polarization_metalens", &design_polarization_metalens, py::arg("lib"), py::arg("focal_x_um"),
          py::arg("focal_y_um"), py::arg("diameter_um"), py::arg("amplitude_weight") = 0.25);

    py::class_<JonesMatrix>(m, "JonesMatrix")
        .def_readonly("xx", &JonesMatrix::xx)
        .def_readonly("xy", &JonesMatrix::xy)
        .def_readonly("yx", &JonesMatrix::yx)
        .def_readonly("yy", &JonesMatrix::yy);
    m.def("solve_jones", &solve_jones, py::arg("incident"), py::arg("stack"), py::arg("substrate"),
          py::arg("wavelength_um"), py::arg("M"));
    py::class_<HwpAtom>(m, "HwpAtom")
        .def(py::init<>())
        .def_readwrite("fill_x", &HwpAtom::fill_x)
        .def_readwrite("fill_y", &HwpAtom::fill_y)
        .def_readwrite("thickness_um", &HwpAtom::thickness_um)
        .def_readwrite("t_x", &HwpAtom::t_x)
        .def_readwrite("t_y", &HwpAtom::t_y)
        .def_readwrite("retardance_deg", &HwpAtom::retardance_deg)
        .def_readwrite("conversion_efficiency", &HwpAtom::conversion_efficiency);
    m.def("find_hwp_atom", &find_hwp_atom, py::arg("pillar"), py::arg("background"), py::arg("incident"),
          py::arg("substrate"), py::arg("period_um"), py::arg("wavelength_um"), py::arg("thickness_um"),
          py::arg("fill_min"), py::arg("fill_max"), py::arg("n_samples"), py::arg("M"));
    py::class_<PbVerifyPoint>(m, "PbVerifyPoint")
        .def_readonly("rotation_deg", &PbVerifyPoint::rotation_deg)
        .def_readonly("cross_phase_deg", &PbVerifyPoint::cross_phase_deg)
        .def_readonly("conversion_eff", &PbVerifyPoint::conversion_eff)
        .def_readonly("copol_leakage", &PbVerifyPoint::copol_leakage);
    m.def("verify_pb_phase", &verify_pb_phase, py::arg("pillar"), py::arg("background"), py::arg("incident"),
          py::arg("substrate"), py::arg("period_um"), py::arg("wavelength_um"), py::arg("atom"),
          py::arg("rotations_rad"), py::arg("M"));
    py::class_<PbMetalensDesign>(m, "PbMetalensDesign")
        .def_readonly("n_cells", &PbMetalensDesign::n_cells)
        .def_readonly("period_um", &PbMetalensDesign::period_um)
        .def_readonly("atom", &PbMetalensDesign::atom)
        .def_readonly("rotation_rad", &PbMetalensDesign::rotation_rad)
        .def_readonly("t_cross", &PbMetalensDesign::t_cross)
        .def_readonly("rms_phase_error_deg", &PbMetalensDesign::rms_phase_error_deg)
        .def_readonly("conversion_efficiency", &PbMetalensDesign::conversion_efficiency);
    m.def("design_pb_metalens",
          py::overload_cast<const HwpAtom&, double, double, const PhaseProfile&, double, int>(&design_pb_metalens),
          py::arg("atom"), py::arg("period_um"), py::arg("wavelength_um"), py::arg("profile"), py::arg("diameter_um"),
          py::arg("handedness") = 1);
    m.def("design_pb_metalens",
          py::overload_cast<const HwpAtom&, double, double, double, double, int>(&design_pb_metalens),
          py::arg("atom"), py::arg("period_um"), py::arg("wavelength_um"), py::arg("focal_length_um"),
          py::arg("diameter_um"), py::arg("handedness") = 1);
    py::class_<BirefringencePoint>(m, "BirefringencePoint")
        .def_readonly("fill_x", &BirefringencePoint::fill_x)
        .def_readonly("fill_y", &BirefringencePoint::fill_y)
        .def_readonly("phase_x_deg", &BirefringencePoint::phase_x_deg)
        .def_readonly("phase_y_deg", &BirefringencePoint::phase_y_deg)
        .def_readonly("retardance_deg", &BirefringencePoint::retardance_deg)
        .def_readonly("tx", &BirefringencePoint::tx)
        .def_readonly("ty", &BirefringencePoint::ty);
    m.def("analyze_birefringence", &analyze_birefringence, py::arg("pillar"), py::arg("background"),
          py::arg("incident"), py::arg("substrate"), py::arg("period_um"), py::arg("wavelength_um"),
          py::arg("thickness_um"), py::arg("fill_y"), py::arg("fill_min"), py::arg("fill_max"), py::arg("n_samples"),
          py::arg("M"));
    py::class_<SystemOptResult>(m, "SystemOptResult")
        .def_readonly("period_um", &SystemOptResult::period_um)
        .def_readonly("thickness_um", &SystemOptResult::thickness_um)
        .def_readonly("strehl", &SystemOptResult::strehl)
        .def_readonly("mean_amplitude", &SystemOptResult::mean_amplitude)
        .def_readonly("merit", &SystemOptResult::merit);
    m.def("optimize_system", &optimize_system, py::arg("pillar"), py::arg("background"), py::arg("incident"),
          py::arg("substrate"), py::arg("focal_um"), py::arg("diameter_um"), py::arg("wavelength_um"),
          py::arg("period_lo"), py::arg("period_hi"), py::arg("thick_lo"), py::arg("thick_hi"), py::arg("grid"),
          py::arg("M"), py::arg("fill_samples"), py::arg("efficiency_weight"),
          py::arg("progress") = std::function<void(float)>());

    m.def(
        "cuda_geev_batched",
        [](py::array_t<std::complex<double>, py::array::c_style | py::array::forcecast> As) {
            // As: [batch, n, n] with each matrix column-major (the reference's layout)
            if (As.ndim() != 3 || As.shape(1) != As.shape(2)) throw std::invalid_argument("[batch, n, n] expected");
            const int batch = static_cast<int>(As.shape(0)), n = static_cast<int>(As.shape(1));
            py::array_t<std::complex<double>> w({batch, n}), vr({batch, n, n});
            const bool ok = cuda::geev_batched(As.data(), n, batch, w.mutable_data(), vr.mutable_data());
            return py::make_tuple(ok, w, vr);
        },
        py::arg("As"));
    m.def("cuda_available", &cuda::available);
    m.def("cuda_device_name", &cuda::device_name);
}
