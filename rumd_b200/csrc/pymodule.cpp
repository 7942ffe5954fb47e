// pybind11 module `_rumd`: the Python surface RUMD builds with SWIG
// (Swig/rumd.i, Sample.i, Potentials.i, Integrators.i) for the LJ/NVT path,
// over the C++ classes in rumd/rumd_classes.h.  RUMD_Error maps to
// RuntimeError and RUMD_cudaResourceError to ValueError (Swig/rumd.i:41-53).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "rumd/rumd_classes.h"
#include "rumd_b200.h"

namespace py = pybind11;
using namespace rumd;

namespace {

py::array_t<float> to_nx3(const std::vector<float>& v4, size_t n) {
  py::array_t<float> out({(py::ssize_t)n, (py::ssize_t)3});
  auto m = out.mutable_unchecked<2>();
  for (size_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) m(i, d) = v4[4 * i + d];
  return out;
}

py::array_t<float> to_nx4(const std::vector<float>& v4, size_t n) {
  py::array_t<float> out({(py::ssize_t)n, (py::ssize_t)4});
  std::memcpy(out.mutable_data(), v4.data(), n * 4 * sizeof(float));
  return out;
}

std::vector<float> flat3(py::array_t<float, py::array::c_style | py::array::forcecast> a, size_t n) {
  if (a.ndim() != 2 || (size_t)a.shape(0) != n || a.shape(1) != 3)
    throw py::value_error("expected an array of shape (N, 3)");
  return std::vector<float>(a.data(), a.data() + 3 * n);
}

}  // namespace

PYBIND11_MODULE(_rumd, m) {
  m.doc() = "RUMD class surface (Sample, Pot_LJ_12_6, IntegratorNVT, ...) on the rumd_b200 engine";
  static py::exception<RUMD_Error> err(m, "RUMD_Error", PyExc_RuntimeError);
  static py::exception<RUMD_cudaResourceError> rerr(m, "RUMD_cudaResourceError", PyExc_ValueError);
  py::register_exception_translator([](std::exception_ptr p) {
    try {
      if (p) std::rethrow_exception(p);
    } catch (const RUMD_cudaResourceError& e) {
      PyErr_SetString(PyExc_ValueError, e.what());
    } catch (const RUMD_Error& e) {
      PyErr_SetString(PyExc_RuntimeError, e.what());
    }
  });

  py::class_<Potential>(m, "Potential")
      .def("GetID_String", &Potential::GetID_String)
      .def("SetVerbose", &Potential::SetVerbose)
      .def("IsMolecularPotential", &Potential::IsMolecularPotential)
      .def("GetPotentialEnergy", &Potential::GetPotentialEnergy)
      .def("CalcF", &Potential::CalcF, py::arg("initialize") = true, py::arg("calc_stresses") = false);

  py::class_<PairPotential, Potential> pp(m, "PairPotential");
  py::enum_<PairPotential::CutoffMethod>(pp, "CutoffMethod")
      .value("NS", PairPotential::NS)
      .value("SP", PairPotential::SP)
      .value("SF", PairPotential::SF)
      .export_values();
  pp.def("GetPotentialParameter", &PairPotential::GetPotentialParameter)
      .def("GetPotentialParameters", &PairPotential::GetPotentialParameters)
      .def("SetNbListSkin", &PairPotential::SetNbListSkin)
      .def("GetNbListSkin", &PairPotential::GetNbListSkin)
      .def("SetNB_Method", &PairPotential::SetNB_Method)
      .def("GetNB_Method", &PairPotential::GetNB_Method)
      .def("SetNbMaxNumNbrs", &PairPotential::SetNbMaxNumNbrs)
      .def("GetMaxCutoff", &PairPotential::GetMaxCutoff)
      .def("GetCutoffMethod", &PairPotential::GetCutoffMethod)
      .def("GetActualMaxNumNbrs", &PairPotential::GetActualMaxNumNbrs)
      .def("SetAssumeNewton3", &PairPotential::SetAssumeNewton3)
      .def("ParamTable", &PairPotential::ParamTable);
  m.attr("NoShift") = py::cast(PairPotential::NS);
  m.attr("ShiftedPotential") = py::cast(PairPotential::SP);
  m.attr("ShiftedForce") = py::cast(PairPotential::SF);
  m.def("NumberOfPairPotentialParameters", []() { return 12; });

  py::class_<Pot_IPL_12_6, PairPotential>(m, "Pot_IPL_12_6")
      .def(py::init<PairPotential::CutoffMethod>(), py::arg("cutoff_method"))
      .def("SetParams", &Pot_IPL_12_6::SetParams, py::arg("i"), py::arg("j"), py::arg("A12"), py::arg("A6"),
           py::arg("Rcut"));
  py::class_<Pot_LJ_12_6, Pot_IPL_12_6>(m, "Pot_LJ_12_6")
      .def(py::init<PairPotential::CutoffMethod>(), py::arg("cutoff_method"))
      .def("SetParams", &Pot_LJ_12_6::SetParams, py::arg("i"), py::arg("j"), py::arg("Sigma"), py::arg("Epsilon"),
           py::arg("Rcut"));
  py::class_<Pot_LJ_12_6_smooth_2_4, PairPotential>(m, "Pot_LJ_12_6_smooth_2_4")
      .def(py::init<PairPotential::CutoffMethod>(), py::arg("cutoff_method"))
      .def("SetParams", &Pot_LJ_12_6_smooth_2_4::SetParams, py::arg("i"), py::arg("j"), py::arg("Sigma"),
           py::arg("Epsilon"), py::arg("Rcut"));
  py::class_<Pot_IPL_n, PairPotential>(m, "Pot_IPL_n")
      .def(py::init<float, PairPotential::CutoffMethod>(), py::arg("n"), py::arg("cutoff_method"))
      .def("SetParams", &Pot_IPL_n::SetParams, py::arg("i"), py::arg("j"), py::arg("Sigma"), py::arg("Epsilon"),
           py::arg("Rcut"))
      .def("GetExponent", &Pot_IPL_n::GetExponent);

  py::class_<Integrator>(m, "Integrator")
      .def("Integrate", &Integrator::Integrate)
      .def("GetKineticEnergy", &Integrator::GetKineticEnergy, py::arg("copy") = true)
      .def("SetMomentumToZero", &Integrator::SetMomentumToZero)
      .def("GetTimeStep", &Integrator::GetTimeStep)
      .def("SetTimeStep", &Integrator::SetTimeStep)
      .def("RequiresStress", &Integrator::RequiresStress)
      .def("GetID_String", &Integrator::GetID_String);
  py::class_<IntegratorNVT, Integrator>(m, "IntegratorNVT")
      .def(py::init<float, double, double>(), py::arg("timeStep"), py::arg("targetTemperature"),
           py::arg("thermostatRelaxationTime"))
      .def(py::init<float>(), py::arg("timeStep"))
      .def("GetInfoString", &IntegratorNVT::GetInfoString, py::arg("precision") = 6)
      .def("InitializeFromInfoString", &IntegratorNVT::InitializeFromInfoString, py::arg("infoStr"),
           py::arg("verbose") = true)
      .def("SetRelaxationTime", &IntegratorNVT::SetRelaxationTime)
      .def("SetTargetTemperature", &IntegratorNVT::SetTargetTemperature, py::arg("T"), py::arg("reset") = false)
      .def("SetThermostatState", &IntegratorNVT::SetThermostatState)
      .def("SetThermostatOn", &IntegratorNVT::SetThermostatOn, py::arg("on") = true)
      .def("SetThermostatOnParticleType", &IntegratorNVT::SetThermostatOnParticleType)
      .def("SetTemperatureChangePerTimeStep", &IntegratorNVT::SetTemperatureChangePerTimeStep)
      .def("GetRelaxationTime", &IntegratorNVT::GetRelaxationTime)
      .def("GetTargetTemperature", &IntegratorNVT::GetTargetTemperature)
      .def("GetThermostatState", &IntegratorNVT::GetThermostatState)
      .def("GetThermostatOn", &IntegratorNVT::GetThermostatOn);
  py::class_<IntegratorNVE, IntegratorNVT>(m, "IntegratorNVE").def(py::init<float>(), py::arg("timeStep"));

  py::class_<Sample>(m, "Sample")
      .def(py::init<unsigned, unsigned>(), py::arg("pb") = 0, py::arg("tp") = 0)
      .def("ReadConf", &Sample::ReadConf, py::arg("filename"), py::arg("init_itg") = false)
      .def("WriteConf", [](Sample& s, const std::string& f, const std::string&) { s.WriteConf(f); }, py::arg("filename"),
           py::arg("mode") = "w")
      .def("SetConfiguration",
           [](Sample& s, py::array_t<float, py::array::c_style | py::array::forcecast> pos, std::vector<int> types,
              std::vector<float> box, std::vector<float> masses, py::object vel, py::object images) {
             size_t n = types.size();
             std::vector<float> v3, p3 = flat3(pos, n);
             std::vector<int> i3;
             if (!vel.is_none()) v3 = flat3(vel.cast<py::array_t<float, py::array::c_style | py::array::forcecast>>(), n);
             if (!images.is_none()) {
               auto a = images.cast<py::array_t<int, py::array::c_style | py::array::forcecast>>();
               i3.assign(a.data(), a.data() + 3 * n);
             }
             s.SetConfiguration(p3, types, box, masses, v3, i3);
           },
           py::arg("positions"), py::arg("types"), py::arg("box"), py::arg("masses") = std::vector<float>{1.f},
           py::arg("velocities") = py::none(), py::arg("images") = py::none())
      .def("SetPotential", &Sample::SetPotential, py::keep_alive<1, 2>())
      .def("AddPotential", &Sample::AddPotential, py::keep_alive<1, 2>())
      .def("GetPotentials", &Sample::GetPotentials, py::return_value_policy::reference)
      .def("SetIntegrator", &Sample::SetIntegrator, py::keep_alive<1, 2>())
      .def("GetIntegrator", &Sample::GetIntegrator, py::return_value_policy::reference)
      .def("CalcF", &Sample::CalcF, py::arg("calc_stresses") = false)
      .def("Run", &Sample::Run, py::arg("nsteps"), py::arg("reset_interval") = 100,
           py::call_guard<py::gil_scoped_release>())
      .def("GetPotentialEnergy", &Sample::GetPotentialEnergy, py::arg("copy") = true)
      .def("GetVirial", &Sample::GetVirial, py::arg("copy") = true)
      .def("GetStress", &Sample::GetStress, py::arg("copy") = true)
      .def("SetIncludeKineticStress", &Sample::SetIncludeKineticStress)
      .def("GetNumberOfParticles", &Sample::GetNumberOfParticles)
      .def("GetNumberOfTypes", &Sample::GetNumberOfTypes)
      .def("GetNumberThisType", &Sample::GetNumberThisType)
      .def("GetMass", &Sample::GetMass)
      .def("SetMass", &Sample::SetMass)
      .def("GetNumberOfDOFs", &Sample::GetNumberOfDOFs)
      .def("GetBoxLengths", &Sample::GetBoxLengths)
      .def("GetVolume", &Sample::GetVolume)
      .def("SetPB_TP", &Sample::SetPB_TP)
      .def("GetParticlesPerBlock", &Sample::GetParticlesPerBlock)
      .def("GetThreadsPerParticle", &Sample::GetThreadsPerParticle)
      .def("SetVerbose", &Sample::SetVerbose)
      .def("GetPositions", [](const Sample& s) { return to_nx3(s.GetField(B2MD_FIELD_POS), s.GetNumberOfParticles()); })
      .def("GetVelocities", [](const Sample& s) { return to_nx3(s.GetField(B2MD_FIELD_VEL), s.GetNumberOfParticles()); })
      .def("GetForces", [](const Sample& s) { return to_nx3(s.GetField(B2MD_FIELD_FORCE), s.GetNumberOfParticles()); })
      .def("GetPotentialEnergies",
           [](const Sample& s) {
             auto f = s.GetField(B2MD_FIELD_FORCE);
             std::vector<float> u(s.GetNumberOfParticles());
             for (size_t i = 0; i < u.size(); ++i) u[i] = f[4 * i + 3];
             return u;
           })
      .def("GetVirials",
           [](const Sample& s) {
             auto w = s.GetField(B2MD_FIELD_VIRIAL);
             std::vector<float> v(s.GetNumberOfParticles());
             for (size_t i = 0; i < v.size(); ++i) v[i] = w[4 * i + 3];
             return v;
           })
      .def("GetField4", [](const Sample& s, int field) { return to_nx4(s.GetField(field), s.GetNumberOfParticles()); })
      .def("GetImages",
           [](const Sample& s) {
             auto im = s.GetImages();
             py::array_t<int> out({(py::ssize_t)s.GetNumberOfParticles(), (py::ssize_t)3});
             std::memcpy(out.mutable_data(), im.data(), im.size() * sizeof(int));
             return out;
           })
      .def("GetTypes", &Sample::GetTypes)
      .def("SetPositions", [](Sample& s, py::array_t<float, py::array::c_style | py::array::forcecast> a) {
        s.SetPositions(flat3(a, s.GetNumberOfParticles()));
      })
      .def("SetVelocities", [](Sample& s, py::array_t<float, py::array::c_style | py::array::forcecast> a) {
        s.SetVelocities(flat3(a, s.GetNumberOfParticles()));
      })
      .def("GetStats", &Sample::Stats)
      .def("SetEnergyLog", &Sample::SetEnergyLog, py::arg("interval"), py::arg("capacity"))
      .def("GetEnergyLog",
           [](const Sample& s) {
             auto v = s.GetEnergyLog();
             py::array_t<double> out({(py::ssize_t)(v.size() / 5), (py::ssize_t)5});
             if (!v.empty()) std::memcpy(out.mutable_data(), v.data(), v.size() * sizeof(double));
             return out;
           })
      .def("ExportNeighborList",
           [](const Sample& s, int max_nbrs) {
             std::vector<unsigned> c, l;
             s.ExportNeighborList(c, l, max_nbrs);
             py::array_t<unsigned> lc((py::ssize_t)c.size()), ll({(py::ssize_t)c.size(), (py::ssize_t)max_nbrs});
             std::memcpy(lc.mutable_data(), c.data(), c.size() * sizeof(unsigned));
             std::memcpy(ll.mutable_data(), l.data(), l.size() * sizeof(unsigned));
             return py::make_tuple(lc, ll);
           })
      .def("ExportSortIndex", &Sample::ExportSortIndex);
}
