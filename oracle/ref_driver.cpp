// Test infrastructure, not product code: runs a scene through the UNMODIFIED
// reference library (EMinsight/XFDTD_CORE's own src/**, compiled against the
// project's xtensor subset into oracle/_ref by oracle/build_ref.py) and writes
// what it computed as .npy files, so that the oracle restatement and the GPU
// engine can be pinned against the reference itself.
//
//   xfd_ref_driver SCENE_TEXT OUT_DIR [--steps N] [--threads C]
//                  [--far-field N_THETA PHI] [--time-only] [--coefficients]
//
// The scene text is the line format xfdtd_core_b200/scene.py writes (one
// object / source / boundary / monitor per line).  Every line is turned into
// the reference API calls a user program makes (as in the reference's
// test/src/examples/*.cpp): Simulation(dl, dl, dl, cfl, ThreadConfig{1, 1, C}),
// addObject / addWaveformSource / addBoundary / addMonitor / addNF2FF, then
// Simulation::run(n).  Outputs in OUT_DIR:
//   ex.npy .. hz.npy          the fields after the run (Simulation::emf())
//   <movie>/NNNNN.npy         movie frames, written by the reference's MovieMonitor
//   <field_time>/<name>.npy   written by the reference's FieldTimeMonitor::output
//   fd/<sub>/...              NFFFTFrequencyDomain::processFarField (with --far-field)
//   fd/power.npy              NFFFTFrequencyDomain::outputRadiationPower
//   line/<name>.npy           VoltageMonitor / CurrentMonitor::output
//   network/s<ji>.npy         Network::output (with frequencies.npy)
//   time.txt                  "run_s steps update_s" then one line per step with
//                             its seconds: Simulation::run's wall time, and the
//                             time loop alone (UpdateStart .. UpdateEnd) and each
//                             step (NextStep to NextStep) from a SimulationFlagVisitor
//                             (with --time-only nothing else is written)
//   coef/<name>.npy           with --coefficients: the 18 update-coefficient
//                             arrays (cexe .. chzey) as the run left them
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>
#include <xtensor/xnpy.hpp>

#include "xfdtd/boundary/pml.h"
#include "xfdtd/object/thin_wire.h"
#include "xfdtd/shape/cylinder.h"
#include "xfdtd/common/constant.h"
#include "xfdtd/common/type_define.h"
#include "xfdtd/coordinate_system/coordinate_system.h"
#include "xfdtd/electromagnetic_field/electromagnetic_field.h"
#include "xfdtd/material/dispersive_material.h"
#include "xfdtd/material/material.h"
#include "xfdtd/monitor/field_monitor.h"
#include "xfdtd/monitor/field_time_monitor.h"
#include "xfdtd/monitor/movie_monitor.h"
#include "xfdtd/nffft/nffft_frequency_domain.h"
#include "xfdtd/monitor/current_monitor.h"
#include "xfdtd/monitor/voltage_monitor.h"
#include "xfdtd/network/network.h"
#include "xfdtd/network/port.h"
#include "xfdtd/object/lumped_element/capacitor.h"
#include "xfdtd/object/lumped_element/current_source.h"
#include "xfdtd/object/lumped_element/inductor.h"
#include "xfdtd/object/lumped_element/resistor.h"
#include "xfdtd/object/lumped_element/voltage_source.h"
#include "xfdtd/object/object.h"
#include "xfdtd/parallel/parallelized_config.h"
#include "xfdtd/shape/cube.h"
#include "xfdtd/shape/sphere.h"
#include "xfdtd/calculation_param/calculation_param.h"
#include "xfdtd/simulation/simulation.h"
#include "xfdtd/simulation/simulation_flag.h"
#include "xfdtd/waveform/waveform.h"
#include "xfdtd/waveform_source/tfsf_3d.h"

namespace {

[[noreturn]] void die(const std::string& msg) {
  std::cerr << "xfd_ref_driver: " << msg << "\n";
  std::exit(2);
}

double num(const std::string& s) {
  if (s == "inf") return std::numeric_limits<double>::infinity();
  return std::stod(s);
}

xfdtd::Axis::Direction direction(const std::string& d) {
  using D = xfdtd::Axis::Direction;
  if (d == "XN") return D::XN;
  if (d == "XP") return D::XP;
  if (d == "YN") return D::YN;
  if (d == "YP") return D::YP;
  if (d == "ZN") return D::ZN;
  if (d == "ZP") return D::ZP;
  die("bad direction " + d);
}

xfdtd::EMF::Field field(const std::string& f) {
  using F = xfdtd::EMF::Field;
  if (f == "EX") return F::EX;
  if (f == "EY") return F::EY;
  if (f == "EZ") return F::EZ;
  if (f == "HX") return F::HX;
  if (f == "HY") return F::HY;
  if (f == "HZ") return F::HZ;
  die("bad field " + f);
}

std::unique_ptr<xfdtd::Cube> cube_at(const std::vector<std::string>& t, std::size_t i) {
  return std::make_unique<xfdtd::Cube>(xfdtd::Vector{num(t[i]), num(t[i + 1]), num(t[i + 2])},
                                       xfdtd::Vector{num(t[i + 3]), num(t[i + 4]), num(t[i + 5])});
}

// "gaussian tau t0 amp" | "cosgauss tau t0 freq amp"; returns the waveform and
// the number of tokens it used.
std::unique_ptr<xfdtd::Waveform> waveform_at(const std::vector<std::string>& t, std::size_t i,
                                             std::size_t* used) {
  if (t[i] == "gaussian") {
    *used = 4;
    return xfdtd::Waveform::gaussian(num(t[i + 1]), num(t[i + 2]), num(t[i + 3]));
  }
  if (t[i] == "cosgauss") {
    *used = 5;
    return xfdtd::Waveform::cosineModulatedGaussian(num(t[i + 1]), num(t[i + 2]), num(t[i + 3]),
                                                    num(t[i + 4]));
  }
  die("bad waveform " + t[i]);
}

xfdtd::Array1D<xfdtd::Real> arr1(const std::vector<double>& v) {
  xfdtd::Array1D<xfdtd::Real> a = xfdtd::Array1D<xfdtd::Real>::from_shape({v.size()});
  for (std::size_t q = 0; q < v.size(); ++q) a(q) = v[q];
  return a;
}

// Material tokens from t[i]: "simple eps mu se sm" | "drude eps_inf P (wp g)*P"
// | "debye eps_inf P (eps_s tau)*P" | "mlorentz eps_inf P (a0 a1 b0 b1 b2)*P".
std::unique_ptr<xfdtd::Material> material_at(const std::string& name,
                                             const std::vector<std::string>& t, std::size_t i) {
  const std::string& k = t[i];
  if (k == "simple")
    return std::make_unique<xfdtd::Material>(
        name, xfdtd::ElectroMagneticProperty{num(t[i + 1]), num(t[i + 2]), num(t[i + 3]),
                                             num(t[i + 4])});
  const double eps_inf = num(t[i + 1]);
  const std::size_t P = (std::size_t)std::stoul(t[i + 2]);
  const std::size_t w = k == "mlorentz" ? 5 : 2;
  std::vector<std::vector<double>> col(w);
  for (std::size_t p = 0; p < P; ++p)
    for (std::size_t c = 0; c < w; ++c) col[c].push_back(num(t[i + 3 + p * w + c]));
  if (k == "drude") return xfdtd::DrudeMedium::makeDrudeMedium(name, eps_inf, arr1(col[0]), arr1(col[1]));
  if (k == "debye") return xfdtd::DebyeMedium::makeDebyeMedium(name, eps_inf, arr1(col[0]), arr1(col[1]));
  if (k == "mlorentz")
    return xfdtd::MLorentzMaterial::makeMLorentz(name, eps_inf, arr1(col[0]), arr1(col[1]),
                                                 arr1(col[2]), arr1(col[3]), arr1(col[4]));
  die("bad material " + k);
}

// Records when the time loop starts and ends and when each step ends (the
// master domain sends these flags, src/domain/domain.cpp:80-137).
class StepClock : public xfdtd::SimulationFlagVisitor {
 public:
  using clock = std::chrono::steady_clock;
  void initStep(xfdtd::SimulationInitFlag flag) override {
    if (flag == xfdtd::SimulationInitFlag::UpdateStart) {
      start = clock::now();
      last = start;
    } else if (flag == xfdtd::SimulationInitFlag::UpdateEnd) {
      end = clock::now();
    }
  }
  void iteratorStep(xfdtd::SimulationIteratorFlag flag, xfdtd::Index, xfdtd::Index,
                    xfdtd::Index) override {
    if (flag != xfdtd::SimulationIteratorFlag::NextStep) return;
    const auto now = clock::now();
    step_s.push_back(std::chrono::duration<double>(now - last).count());
    last = now;
  }
  clock::time_point start{}, last{}, end{};
  std::vector<double> step_s;
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) die("usage: xfd_ref_driver SCENE OUT_DIR [--steps N] [--threads C] "
                    "[--far-field N_THETA PHI] [--time-only]");
  const std::string scene_path = argv[1];
  const std::filesystem::path out = argv[2];
  long long steps_override = -1;
  int threads = 1;
  int n_theta = 0;
  double ff_phi = 0.0;
  bool time_only = false, coefficients = false;
  for (int a = 3; a < argc; ++a) {
    const std::string o = argv[a];
    if (o == "--steps" && a + 1 < argc) steps_override = std::stoll(argv[++a]);
    else if (o == "--threads" && a + 1 < argc) threads = std::stoi(argv[++a]);
    else if (o == "--far-field" && a + 2 < argc) {
      n_theta = std::stoi(argv[++a]);
      ff_phi = std::stod(argv[++a]);
    } else if (o == "--time-only") time_only = true;
    else if (o == "--coefficients") coefficients = true;
    else die("unknown option " + o);
  }
  std::filesystem::create_directories(out);

  std::ifstream in(scene_path);
  if (!in) die("cannot read " + scene_path);
  std::vector<std::vector<std::string>> lines;
  for (std::string ln; std::getline(in, ln);) {
    std::istringstream ss(ln);
    std::vector<std::string> t;
    for (std::string w; ss >> w;) t.push_back(w);
    if (!t.empty()) lines.push_back(t);
  }
  double dl[3] = {0, 0, 0}, cfl = 0;
  long long steps = 0;
  for (const auto& t : lines) {
    if (t[0] == "grid") {
      for (int q = 0; q < 3; ++q) dl[q] = num(t[1 + q]);
      cfl = num(t[4]);
    } else if (t[0] == "steps") {
      steps = std::stoll(t[1]);
    }
  }
  if (steps_override >= 0) steps = steps_override;
  if (cfl <= 0) die("no grid line");

  xfdtd::Simulation s{dl[0], dl[1], dl[2], cfl, xfdtd::ThreadConfig{1, 1, threads}};
  std::shared_ptr<xfdtd::NFFFTFrequencyDomain> nf2ff;
  std::vector<std::shared_ptr<xfdtd::FieldTimeMonitor>> time_monitors;
  std::map<std::string, std::shared_ptr<xfdtd::VoltageMonitor>> v_monitors;
  std::map<std::string, std::shared_ptr<xfdtd::CurrentMonitor>> c_monitors;
  std::vector<std::shared_ptr<xfdtd::Port>> ports;
  std::vector<double> net_freqs;
  bool have_network = false;
  auto xyz = [](const std::string& a) {
    if (a == "X") return xfdtd::Axis::XYZ::X;
    if (a == "Y") return xfdtd::Axis::XYZ::Y;
    if (a != "Z") die("bad axis " + a);
    return xfdtd::Axis::XYZ::Z;
  };
  for (const auto& t : lines) {
    const std::string& k = t[0];
    if (k == "xfdtd-scene" || k == "name" || k == "grid" || k == "steps") continue;
    if (k == "object") {
      std::unique_ptr<xfdtd::Shape> shape;
      std::size_t mi = 0;
      if (t[2] == "cube") {
        shape = cube_at(t, 3);
        mi = 9;
      } else if (t[2] == "sphere") {
        shape = std::make_unique<xfdtd::Sphere>(xfdtd::Vector{num(t[3]), num(t[4]), num(t[5])},
                                                num(t[6]));
        mi = 7;
      } else {
        die("bad shape " + t[2]);
      }
      s.addObject(std::make_shared<xfdtd::Object>(t[1], std::move(shape), material_at(t[1], t, mi)));
    } else if (k == "thin_wire") {
      if (t.size() != 8 || (t[7] != "X" && t[7] != "Y" && t[7] != "Z"))
        die("bad thin_wire line");
      const xfdtd::Axis axis = t[7] == "X" ? xfdtd::Axis::XP
                               : t[7] == "Y" ? xfdtd::Axis::YP : xfdtd::Axis::ZP;
      s.addObject(std::make_shared<xfdtd::ThinWire>(
          t[1], std::make_unique<xfdtd::Cylinder>(
                    xfdtd::Vector{num(t[2]), num(t[3]), num(t[4])}, num(t[5]), num(t[6]), axis)));
    } else if (k == "current_source" || k == "voltage_source") {
      std::size_t used = 0;
      auto w = waveform_at(t, 10, &used);
      if (k == "current_source")
        s.addObject(std::make_shared<xfdtd::CurrentSource>(t[1], cube_at(t, 2), direction(t[8]),
                                                           num(t[9]), std::move(w)));
      else
        s.addObject(std::make_shared<xfdtd::VoltageSource>(t[1], cube_at(t, 2), direction(t[8]),
                                                           num(t[9]), std::move(w)));
    } else if (k == "pml") {
      s.addBoundary(std::make_shared<xfdtd::PML>(std::stoi(t[1]), direction(t[2]),
                                                 std::stoi(t[3]), num(t[4]), num(t[5]),
                                                 num(t[6]), num(t[7])));
    } else if (k == "tfsf3d") {
      std::size_t used = 0;
      auto w = waveform_at(t, 7, &used);
      s.addWaveformSource(std::make_shared<xfdtd::TFSF3D>(
          (xfdtd::Index)std::stoul(t[1]), (xfdtd::Index)std::stoul(t[2]),
          (xfdtd::Index)std::stoul(t[3]), num(t[4]), num(t[5]), num(t[6]), std::move(w)));
    } else if (k == "movie") {
      s.addMonitor(std::make_shared<xfdtd::MovieMonitor>(
          std::make_unique<xfdtd::FieldMonitor>(cube_at(t, 3), field(t[2]), "", ""),
          (std::size_t)std::stoul(t[9]), t[1], (out / t[1]).string()));
    } else if (k == "field_time") {
      auto m = std::make_shared<xfdtd::FieldTimeMonitor>(t[1], cube_at(t, 3),
                                                         (out / "field_time").string(),
                                                         field(t[2]));
      time_monitors.push_back(m);
      s.addMonitor(m);
    } else if (k == "nf2ff_fd") {
      const std::size_t nfq = (std::size_t)std::stoul(t[4]);
      std::vector<double> f;
      for (std::size_t q = 0; q < nfq; ++q) f.push_back(num(t[5 + q]));
      nf2ff = std::make_shared<xfdtd::NFFFTFrequencyDomain>(
          (xfdtd::Index)std::stoul(t[1]), (xfdtd::Index)std::stoul(t[2]),
          (xfdtd::Index)std::stoul(t[3]), arr1(f), (out / "fd").string());
      s.addNF2FF(nf2ff);
    } else if (k == "resistor" || k == "capacitor" || k == "inductor") {
      if (t.size() != 10) die("bad " + k + " line");
      if (k == "resistor")
        s.addObject(std::make_shared<xfdtd::Resistor>(t[1], cube_at(t, 2), xyz(t[8]), num(t[9])));
      else if (k == "capacitor")
        s.addObject(std::make_shared<xfdtd::Capacitor>(t[1], cube_at(t, 2), xyz(t[8]), num(t[9])));
      else
        s.addObject(std::make_shared<xfdtd::Inductor>(t[1], cube_at(t, 2), xyz(t[8]), num(t[9])));
    } else if (k == "voltage_monitor" || k == "current_monitor") {
      if (t.size() != 9) die("bad " + k + " line");
      const std::string dir = (out / "line").string();
      if (k == "voltage_monitor") {
        auto m = std::make_shared<xfdtd::VoltageMonitor>(t[1], cube_at(t, 2), direction(t[8]), dir);
        v_monitors[t[1]] = m;
        s.addMonitor(m);
      } else {
        auto m = std::make_shared<xfdtd::CurrentMonitor>(t[1], cube_at(t, 2), direction(t[8]), dir);
        c_monitors[t[1]] = m;
        s.addMonitor(m);
      }
    } else if (k == "network") {
      const std::size_t n = (std::size_t)std::stoul(t[1]);
      if (t.size() != 2 + n) die("bad network line");
      for (std::size_t q = 0; q < n; ++q) net_freqs.push_back(num(t[2 + q]));
      have_network = true;
    } else if (k == "port") {
      if (t.size() != 7 || !c_monitors.count(t[5]) || !v_monitors.count(t[6]))
        die("bad port line");
      ports.push_back(std::make_shared<xfdtd::Port>(
          (std::size_t)std::stoul(t[1]), t[2] == "1", std::complex<double>{num(t[3]), num(t[4])},
          c_monitors[t[5]], v_monitors[t[6]]));
    } else {
      die("scene line '" + k + "' is not supported by the reference driver");
    }
  }
  std::shared_ptr<xfdtd::Network> network;
  if (have_network) {
    network = std::make_shared<xfdtd::Network>(ports, arr1(net_freqs), (out / "network").string());
    s.addNetwork(network);
  }

  auto step_clock = std::make_shared<StepClock>();
  s.addVisitor(step_clock);
  const auto t0 = std::chrono::steady_clock::now();
  s.run((xfdtd::Index)steps);
  const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  {
    std::ofstream f(out / "time.txt");
    f.precision(17);
    f << el << " " << steps << " "
      << std::chrono::duration<double>(step_clock->end - step_clock->start).count() << "\n";
    for (double v : step_clock->step_s) f << v << "\n";
  }
  if (time_only) return 0;

  const auto& emf = s.emf();
  xt::dump_npy((out / "ex.npy").string(), emf->ex());
  xt::dump_npy((out / "ey.npy").string(), emf->ey());
  xt::dump_npy((out / "ez.npy").string(), emf->ez());
  xt::dump_npy((out / "hx.npy").string(), emf->hx());
  xt::dump_npy((out / "hy.npy").string(), emf->hy());
  xt::dump_npy((out / "hz.npy").string(), emf->hz());
  for (auto& m : time_monitors) m->output();
  for (auto& [n, m] : v_monitors) m->output();
  for (auto& [n, m] : c_monitors) m->output();
  if (network) network->output();
  if (coefficients) {
    const auto& c = s.calculationParam()->fdtdCoefficient();
    const auto d = out / "coef";
    std::filesystem::create_directories(d);
    auto put = [&](const char* n, const auto& a) { xt::dump_npy((d / n).string() + ".npy", a); };
    put("cexe", c->cexe()); put("cexhy", c->cexhy()); put("cexhz", c->cexhz());
    put("ceye", c->ceye()); put("ceyhz", c->ceyhz()); put("ceyhx", c->ceyhx());
    put("ceze", c->ceze()); put("cezhx", c->cezhx()); put("cezhy", c->cezhy());
    put("chxh", c->chxh()); put("chxey", c->chxey()); put("chxez", c->chxez());
    put("chyh", c->chyh()); put("chyez", c->chyez()); put("chyex", c->chyex());
    put("chzh", c->chzh()); put("chzex", c->chzex()); put("chzey", c->chzey());
  }
  if (nf2ff) {  // NFFFTFrequencyDomain::outputRadiationPower -> fd/power.npy
    nf2ff->setOutputDir((out / "fd").string());
    nf2ff->outputRadiationPower();
  }
  if (nf2ff && n_theta > 0) {
    nf2ff->setOutputDir((out / "fd").string());
    nf2ff->processFarField(
        xt::linspace<xfdtd::Real>(-xfdtd::constant::PI, xfdtd::constant::PI, n_theta), ff_phi,
        "ff");
  }
  return 0;
}
