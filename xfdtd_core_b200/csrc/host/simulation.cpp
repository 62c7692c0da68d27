// xfdtd::Simulation on the B200 engine.
//
// Simulation::init restates, in FP64 on the host, the reference's set-up of
// the 3-D FDTD path and hands the result to the engine C ABI:
//   grid generation        src/grid_space/grid_space_generator.cpp:16-217,
//                          src/grid_space/grid_space.cpp:517-544
//   time step              src/calculation_param/time_param.cpp:10-13
//   painting               src/object/object.cpp:114-198 (cell centre inside,
//                          last object wins)
//   edge/face averaging    src/calculation_param/calculation_param.cpp:43-168
//   Yee coefficients       calculation_param.cpp:170-264
//   lumped elements        src/object/lumped_element/{current_source,voltage_source,
//                          resistor,capacitor,inductor}.cpp (init, coefficients)
//   CPML grading / kappa   src/boundary/pml.cpp:98-244, 286-633
//   TFSF incident grid     src/waveform_source/tfsf.cpp:36-302
//   ADE coefficients       src/material/ade_method/{m_lor,drude,debye}_ade_method.cpp
//   NF2FF surfaces/phasors src/nffft/nffft.cpp:88-245, nffft_fd_data.cpp:65-76
//   NF2FF far field        src/nffft/nffft_fd_data_process.cpp:15-144 (on the GPU)
// Instead of 18 full-grid coefficient arrays the engine receives a table of
// material classes (the (ca, cb) pair of each component, keyed by the
// materials of the 2x2x2 cells around a lattice node) plus a uint16 class per
// node, and per-axis curl factors 1/(d*kappa).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <limits>
#include <map>
#include <numeric>
#include <set>
#include <sstream>
#include <unordered_map>

#include "xfd_engine.h"
#include "xfdtd/xfdtd.h"

namespace xfdtd {

using constant::C_0;
using constant::EPSILON_0;
using constant::MU_0;
using constant::PI;

// ------------------------------------------------------------ shapes
static bool floatLE(Real lhs, Real rhs, Real eps) {
  // floatCompare(lhs, rhs, LessEqual, eps) (src/include/util/float_compare.h:20-42)
  return std::abs(lhs - rhs) <= eps ? true : lhs < rhs;
}

bool Cube::isInside(Real x, Real y, Real z, Real eps) const {
  // Cube::isInside (src/shape/cube.cpp:58-73)
  return floatLE(_origin.x(), x, eps) && floatLE(x, _end.x(), eps) &&
         floatLE(_origin.y(), y, eps) && floatLE(y, _end.y(), eps) &&
         floatLE(_origin.z(), z, eps) && floatLE(z, _end.z(), eps);
}

bool Sphere::isInside(Real x, Real y, Real z, Real eps) const {
  // Sphere::isInside (src/shape/sphere.cpp:29-32)
  const Real dx = x - _center.x(), dy = y - _center.y(), dz = z - _center.z();
  return floatLE(std::sqrt(dx * dx + dy * dy + dz * dz), _radius, eps);
}

std::unique_ptr<Cube> Sphere::wrappedCube() const {
  // Sphere::wrappedCube (src/shape/sphere.cpp:34-37)
  return std::make_unique<Cube>(_center - Vector{_radius, _radius, _radius},
                                Vector{_radius * 2, _radius * 2, _radius * 2});
}

Cylinder::Cylinder(Vector center, Real radius, Real height, Axis axis)
    : _center{center}, _radius{radius}, _height{height}, _axis{axis} {
  // Cylinder::Cylinder (src/shape/cylinder.cpp:13-26)
  if (_radius < 0) throw XFDTDException("Cylinder radius must be positive");
  if (_height < 0) throw XFDTDException("Cylinder height must be positive");
}

std::unique_ptr<Cube> Cylinder::wrappedCube() const {
  // Cylinder::wrappedCube (src/shape/cylinder.cpp:72-98): height along the
  // axis, 2 r across, centred on `center`.
  const int w = _axis.axisIndex();
  if (w < 0) throw XFDTDException("Cylinder axis is not supported");
  Real o[3], sz[3];
  for (int a = 0; a < 3; ++a) {
    const Real half = a == w ? _height / 2 : _radius;
    o[a] = _center(a) - half;
    sz[a] = 2 * half;
  }
  return std::make_unique<Cube>(Vector{o[0], o[1], o[2]}, Vector{sz[0], sz[1], sz[2]});
}

bool Cylinder::isInside(Real x, Real y, Real z, Real eps) const {
  // Cylinder::isInside (src/shape/cylinder.cpp:44-66): inside the wrapped
  // cube and within the radius of the axis line (floatCompare's default
  // tolerance, 1e-8, on the distance).
  if (!wrappedCube()->isInside(x, y, z, eps)) return false;
  const int w = _axis.axisIndex();
  const Real p[3] = {x, y, z};
  const int u = (w + 1) % 3, v = (w + 2) % 3;
  const Real du = p[u] - _center(u), dv = p[v] - _center(v);
  // the reference orders the two transverse axes (y, z), (x, z), (x, y)
  const Real dis = w == 1 ? std::sqrt(std::pow(dv, 2) + std::pow(du, 2))
                          : std::sqrt(std::pow(du, 2) + std::pow(dv, 2));
  return floatLE(dis, _radius, 1e-8);
}

ElectroMagneticProperty::ElectroMagneticProperty(Real eps_r, Real mu_r, Real sigma_e,
                                                 Real sigma_m)
    : _eps_r{eps_r},
      _mu_r{mu_r},
      _sigma_e{sigma_e == 0 ? constant::SIGMA_E_ZERO_APPROX : sigma_e},
      _sigma_m{sigma_m == 0 ? constant::SIGMA_M_ZERO_APPROX : sigma_m} {}

// --------------------------------------------------------- voxel object
namespace {
Real meanOf(const std::vector<Real>& v) {
  Real s = 0;
  for (Real x : v) s += x;
  return v.empty() ? 1 : s / (Real)v.size();
}
}  // namespace

VoxelObject::VoxelObject(std::string name, std::unique_ptr<Cube> cube, std::array<Index, 3> dims,
                         std::vector<Real> eps_r, Real mu_r, Real sigma_e)
    : Object{name, std::move(cube),
             std::make_shared<Material>(name, ElectroMagneticProperty{meanOf(eps_r), mu_r,
                                                                      sigma_e, 0})},
      _dims{dims},
      _eps_r{std::move(eps_r)},
      _mu_r{mu_r},
      _sigma_e{sigma_e == 0 ? constant::SIGMA_E_ZERO_APPROX : sigma_e} {
  if (dims[0] == 0 || dims[1] == 0 || dims[2] == 0 ||
      _eps_r.size() != dims[0] * dims[1] * dims[2])
    throw XFDTDException("VoxelObject: eps_r does not match dims");
}

// --------------------------------------------------------- materials
std::unique_ptr<DrudeMedium> DrudeMedium::makeDrudeMedium(std::string_view name, Real eps_inf,
                                                          Array1D<Real> omega_p,
                                                          Array1D<Real> gamma) {
  // DrudeEqDecision: a0 = wp^2, a1 = 0, b0 = 0, b1 = gamma, b2 = 1
  // (src/material/dispersive_material_equation.cpp:49-54)
  std::vector<std::array<Real, 5>> poles;
  std::vector<std::array<Real, 2>> native;
  for (Index p = 0; p < omega_p.size(); ++p) {
    poles.push_back({omega_p[p] * omega_p[p], 0.0, 0.0, gamma[p], 1.0});
    native.push_back({omega_p[p], gamma[p]});
  }
  return std::make_unique<DrudeMedium>(name, eps_inf, Kind::Drude, poles, native);
}

std::unique_ptr<DebyeMedium> DebyeMedium::makeDebyeMedium(std::string_view name, Real eps_inf,
                                                          Array1D<Real> eps_static,
                                                          Array1D<Real> tau) {
  // DebyeEqDecision: a0 = eps_s - eps_inf, a1 = 0, b0 = 1, b1 = tau, b2 = 0
  // (dispersive_material_equation.cpp:43-47)
  std::vector<std::array<Real, 5>> poles;
  std::vector<std::array<Real, 2>> native;
  for (Index p = 0; p < eps_static.size(); ++p) {
    poles.push_back({eps_static[p] - eps_inf, 0.0, 1.0, tau[p], 0.0});
    native.push_back({eps_static[p], tau[p]});
  }
  return std::make_unique<DebyeMedium>(name, eps_inf, Kind::Debye, poles, native);
}

std::unique_ptr<MLorentzMaterial> MLorentzMaterial::makeMLorentz(
    std::string_view name, Real eps_inf, Array1D<Real> a0, Array1D<Real> a1, Array1D<Real> b0,
    Array1D<Real> b1, Array1D<Real> b2) {
  if (a1.size() != a0.size() || b0.size() != a0.size() || b1.size() != a0.size() ||
      b2.size() != a0.size())
    throw XFDTDException("Modified Lorentz Model paramater doesn't have same size.");
  std::vector<std::array<Real, 5>> poles;
  std::vector<std::array<Real, 2>> native;
  for (Index p = 0; p < a0.size(); ++p) {
    poles.push_back({a0[p], a1[p], b0[p], b1[p], b2[p]});
    native.push_back({0.0, 0.0});
  }
  return std::make_unique<MLorentzMaterial>(name, eps_inf, Kind::MLorentz, poles, native);
}

std::complex<Real> LinearDispersiveMaterial::susceptibility(Real freq, Index p) const {
  const auto& c = _poles.at(p);  // a0 a1 b0 b1 b2
  const std::complex<Real> jw = constant::II * (static_cast<Real>(2.0) * constant::PI * freq);
  return (c[1] * jw + c[0]) / (c[4] * jw * jw + c[3] * jw + c[2]);
}

Array1D<std::complex<Real>> LinearDispersiveMaterial::relativePermittivity(
    const Array1D<Real>& freq) const {
  auto out = Array1D<std::complex<Real>>::from_shape({freq.size()});
  for (std::size_t q = 0; q < freq.size(); ++q) {
    std::complex<Real> sum{0, 0};
    for (Index p = 0; p < numPoles(); ++p) sum += susceptibility(freq(q), p);
    out(q) = _eps_inf + sum;
  }
  return out;
}

// ---------------------------------------------------------- waveform
std::unique_ptr<Waveform> Waveform::gaussian(Real tau, Real t_0, Real amplitude) {
  return std::make_unique<Waveform>(
      [tau, t_0](Real t) { return std::exp(-std::pow((t - t_0) / tau, 2)); }, amplitude);
}

std::unique_ptr<Waveform> Waveform::cosineModulatedGaussian(Real tau, Real t_0, Real frequency,
                                                            Real amplitude) {
  return std::make_unique<Waveform>(
      [tau, t_0, frequency](Real t) {
        return std::exp(-std::pow((t - t_0) / tau, 2)) *
               std::cos(2 * constant::PI * frequency * (t - t_0));
      },
      amplitude);
}

std::unique_ptr<Waveform> Waveform::sine(Real frequency, Real amplitude) {
  return std::make_unique<Waveform>(
      [frequency](Real t) { return std::sin(2 * constant::PI * frequency * t); }, amplitude);
}

// src/waveform/waveform.cpp:47-101
std::unique_ptr<Waveform> Waveform::cosine(Real frequency, Real amplitude) {
  return std::make_unique<Waveform>(
      [frequency](Real t) { return std::cos(2 * constant::PI * frequency * t); }, amplitude);
}

std::unique_ptr<Waveform> Waveform::square(Real frequency, Real amplitude) {
  return std::make_unique<Waveform>(
      [frequency](Real t) { return std::copysign(1.0, std::sin(2 * constant::PI * frequency * t)); },
      amplitude);
}

std::unique_ptr<Waveform> Waveform::triangle(Real frequency, Real /*amplitude*/) {
  return std::make_unique<Waveform>([frequency](Real t) {
    return std::asin(std::sin(2 * constant::PI * frequency * t)) * 2 / constant::PI;
  });
}

std::unique_ptr<Waveform> Waveform::sawtooth(Real frequency, Real amplitude) {
  return std::make_unique<Waveform>(
      [frequency](Real t) { return 2 * std::fmod(frequency * t, 1.0) - 1; }, amplitude);
}

std::unique_ptr<Waveform> Waveform::step(Real t_0, Real amplitude) {
  return std::make_unique<Waveform>([t_0](Real t) { return static_cast<Real>(t >= t_0); },
                                    amplitude);
}

void Waveform::init(const std::vector<Real>& time) {
  // Waveform::init (src/waveform/waveform.cpp:28-34)
  std::vector<Real> v(time.size());
  for (std::size_t i = 0; i < time.size(); ++i) v[i] = amplitude() * _f(time[i]);
  _value = Array1D<Real>(xt::adapt(v));
  _time = Array1D<Real>(xt::adapt(time));
}

// --------------------------------------------------------- helpers
namespace {

std::vector<Real> linspace(Real a, Real b, std::size_t n) {
  // xt::linspace with endpoint: a + i*step, the last sample exactly b.
  std::vector<Real> v(n);
  if (n == 1) {
    v[0] = a;
    return v;
  }
  const Real step = (b - a) / static_cast<Real>(n - 1);
  for (std::size_t i = 0; i < n; ++i) v[i] = a + step * static_cast<Real>(i);
  v[n - 1] = b;
  return v;
}

std::size_t nearestNode(const std::vector<Real>& nodes, Real x) {
  // argmin |e_node - x| (src/grid_space/grid_space.cpp:505-515); first on ties.
  std::size_t best = 0;
  Real bd = std::abs(nodes[0] - x);
  for (std::size_t i = 1; i < nodes.size(); ++i) {
    const Real d = std::abs(nodes[i] - x);
    if (d < bd) {
      bd = d;
      best = i;
    }
  }
  return best;
}

constexpr uint16_t kNoCell = 0xFFFF;

struct ClassKey {
  uint16_t m[8];
  uint8_t flags;
  bool operator==(const ClassKey& o) const {
    return flags == o.flags && std::memcmp(m, o.m, sizeof m) == 0;
  }
};

struct ClassKeyHash {
  std::size_t operator()(const ClassKey& k) const {
    uint64_t a, b;
    std::memcpy(&a, k.m, 8);
    std::memcpy(&b, k.m + 4, 8);
    uint64_t h = a * 0x9E3779B97F4A7C15ULL ^ (b + 0x632BE59BD9B4E019ULL + (a << 6) + (a >> 2));
    return static_cast<std::size_t>(h ^ (uint64_t)k.flags * 0xC2B2AE3D27D4EB4FULL);
  }
};

struct MatP {
  Real eps, mu, se, sm;
};

void checkStatus(xfd_engine* e, int st, const char* what) {
  if (st != 0) {
    std::ostringstream os;
    os << what << " failed (" << st << "): " << xfd_last_error(e);
    throw XFDTDException(os.str());
  }
}

}  // namespace

// ------------------------------------------------------------- impl
struct Simulation::Impl {
  std::vector<Real> e_node[3], h_node[3], e_size[3], h_size[3];
  Real min_d[3]{};
  std::vector<uint16_t> cell;  // painter index per cell (nx*ny*nz)
  std::vector<const Material*> painters;
  std::vector<MatP> mat;
  std::vector<double> table;    // classes x 12
  std::vector<uint16_t> lattice_class;
  std::vector<Real> fe[3], fh[3];
  struct SlabH {
    int axis, neg, n, e_start, h_start;
    std::vector<Real> a_e, b_e, a_h, b_h, kappa_e, kappa_h;
  };
  std::vector<SlabH> slabs;
  struct MovieH {
    MovieMonitor* mon;
    int id;
    int s[3], e[3];
  };
  std::vector<MovieH> movies;
  struct ProbeH {
    FieldTimeMonitor* mon;
    int id;  // engine movie id, -1 when the box is empty
  };
  std::vector<ProbeH> probes;
  NFFFTFrequencyDomain* nf2ff = nullptr;
  // E coefficient overrides of the nodes around VoxelObjects: the node, the
  // averaged eps (absolute) and sigma of its edge, its (ca, cb), and the
  // voxel (object index, flat voxel index; -1: not a voxel) of each cell of
  // the average with the cell's weight in it.
  struct OvrE {
    int32_t node[3];
    int32_t comp;
    double eps, sig, ca, cb;
    int vobj[4];
    int64_t voxel[4];
    double w;
  };
  std::vector<OvrE> ovr;
  // ThinWire H coefficient factors: (lattice node, H component) -> the
  // factors on its two curl-term coefficients (che_a, che_b).
  std::map<std::pair<Index, int>, std::array<double, 2>> hterm;
  // TFSF set-up kept for inspection (Simulation::tfsfTables)
  std::vector<double> tf_e_inc, tf_h_inc, tf_p_int[3], tf_p_half[3];
  int tf_aux = 0;
  bool initialised = false;
};

Simulation::Simulation(Real dx, Real dy, Real dz, Real cfl, ThreadConfig)
    : _dl{dx, dy, dz}, _cfl{cfl}, _impl{std::make_unique<Impl>()} {}

Simulation::~Simulation() {
  for (auto& nf : _nffts)
    if (nf) nf->_engine = nullptr;
  if (_engine) xfd_destroy(_engine);
}

void Simulation::addObject(std::shared_ptr<Object> o) { _objects.push_back(std::move(o)); }
void Simulation::addBoundary(std::shared_ptr<Boundary> b) { _boundaries.push_back(std::move(b)); }
void Simulation::addWaveformSource(std::shared_ptr<WaveformSource> s) {
  _sources.push_back(std::move(s));
}
void Simulation::addMonitor(std::shared_ptr<Monitor> m) { _monitors.push_back(std::move(m)); }
void Simulation::addNF2FF(std::shared_ptr<NFFFTTimeDomain> n) { _nffts_td.push_back(std::move(n)); }
void Simulation::addNetwork(std::shared_ptr<Network> n) { _networks.push_back(std::move(n)); }
void Simulation::addNF2FF(std::shared_ptr<NFFFTFrequencyDomain> n) {
  _nffts.push_back(std::move(n));
}

void Simulation::addVisitor(std::shared_ptr<SimulationFlagVisitor> v) {
  if (v) _visitors.push_back(std::move(v));
}
void Simulation::addDefaultVisitor() {
  _visitors.push_back(std::make_shared<DefaultSimulationFlagVisitor>());
}

void Simulation::run(Index time_step) {
  auto flag = [&](SimulationInitFlag f) {
    for (auto& v : _visitors) v->initStep(f);
  };
  flag(SimulationInitFlag::SimulationStart);
  flag(SimulationInitFlag::InitStart);
  init(time_step);
  flag(SimulationInitFlag::InitEnd);
  flag(SimulationInitFlag::UpdateStart);
  if (_visitors.empty()) {
    advance(time_step);
  } else {
    // Chunks of the engine's graph length; a visitor sees NextStep after each
    // (the engine is synchronised there, so the step it reports is done).
    const Index start = 0, end = time_step;
    for (Index t = 0; t < time_step;) {
      const Index n = std::min<Index>((Index)std::max<long long>(_chunk, 1), time_step - t);
      advance(n);
      checkStatus(_engine, xfd_sync(_engine), "xfd_sync");
      t += n;
      for (auto& v : _visitors) v->iteratorStep(SimulationIteratorFlag::NextStep, t, start, end);
    }
  }
  finish();
  flag(SimulationInitFlag::UpdateEnd);
  flag(SimulationInitFlag::SimulationEnd);
}

void DefaultSimulationFlagVisitor::initStep(SimulationInitFlag flag) {
  using clk = std::chrono::steady_clock;
  const double now = std::chrono::duration<double>(clk::now().time_since_epoch()).count();
  switch (flag) {
    case SimulationInitFlag::SimulationStart:
      std::fprintf(stderr, "Simulation start\n");
      break;
    case SimulationInitFlag::InitStart:
      _t_init = now;
      std::fprintf(stderr, "Simulation init start\n");
      break;
    case SimulationInitFlag::InitEnd:
      std::fprintf(stderr, "Simulation init end\nElapsed time: %.3f s\n", now - _t_init);
      break;
    case SimulationInitFlag::UpdateStart:
      _t_update = now;
      std::fprintf(stderr, "Simulation update start\n");
      break;
    case SimulationInitFlag::UpdateEnd:
      std::fprintf(stderr, "Simulation update end\nElapsed time: %.3f s\n", now - _t_update);
      break;
    case SimulationInitFlag::SimulationEnd:
      std::fprintf(stderr, "Simulation end\n");
      break;
  }
}

void DefaultSimulationFlagVisitor::iteratorStep(SimulationIteratorFlag flag, Index cur, Index start,
                                                Index end) {
  if (flag != SimulationIteratorFlag::NextStep || end <= start) return;
  const Index percent = (cur - start) * 100 / (end - start);
  if (percent == _last_percent) return;
  _last_percent = percent;
  std::fprintf(stderr, "\rProgress: %zu%% (%zu/%zu)%s", (size_t)percent, (size_t)(cur - start),
               (size_t)(end - start), cur >= end ? "\n" : "");
}

void Simulation::init(Index time_step) {
  if (_objects.empty()) throw XFDTDException("No object is added");
  Impl& I = *_impl;
  I = Impl{};
  if (_engine) {
    xfd_destroy(_engine);
    _engine = nullptr;
  }
  _steps = time_step;

  // ---------------------------------------------------------------- grid
  Real lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = std::numeric_limits<Real>::max();
    hi[a] = std::numeric_limits<Real>::lowest();
  }
  for (const auto& o : _objects) {  // Shape::makeWrappedCube (src/shape/shape.cpp:8-38)
    auto c = o->shape()->wrappedCube();
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], c->origin()(a));
      hi[a] = std::max(hi[a], c->end()(a));
    }
  }
  {
    Cube dom{Vector{lo[0], lo[1], lo[2]}, Vector{hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]}};
    Real mn[3] = {dom.origin().x(), dom.origin().y(), dom.origin().z()};
    Real mx[3] = {dom.end().x(), dom.end().y(), dom.end().z()};
    for (const auto& b : _boundaries) {  // extendDomain (grid_space_generator.cpp:36-99)
      auto p = std::dynamic_pointer_cast<PML>(b);
      if (!p || p->thickness() < 0) continue;
      const int a = Axis::axisOf(p->direction());
      if (Axis::negative(p->direction())) mn[a] -= p->thickness() * _dl[a];
      else mx[a] += p->thickness() * _dl[a];
    }
    Cube ext{Vector{mn[0], mn[1], mn[2]}, Vector{mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]}};
    for (int a = 0; a < 3; ++a) {  // generateGridSpace3D (:183-217)
      const Real l0 = ext.origin()(a), l1 = ext.end()(a);
      const auto na = static_cast<Index>(std::round((l1 - l0) / _dl[a]));
      if (na <= 1) throw XFDTDException("GridSpace is too small");
      const Real top = l0 + _dl[a] * na;
      I.e_node[a] = linspace(l0, l0 + (top - l0), na + 1);
      _n[a] = na;
      auto& e = I.e_node[a];
      I.h_node[a].resize(na);
      I.e_size[a].resize(na);
      for (Index i = 0; i < na; ++i) {
        I.h_node[a][i] = (e[i] + e[i + 1]) / 2;
        I.e_size[a][i] = e[i + 1] - e[i];
      }
      std::vector<Real> tmp;
      tmp.push_back(e.front() - _dl[a] / 2);
      tmp.insert(tmp.end(), I.h_node[a].begin(), I.h_node[a].end());
      tmp.push_back(e.back() + _dl[a] / 2);
      I.h_size[a].resize(na + 1);
      for (Index i = 0; i <= na; ++i) I.h_size[a][i] = tmp[i + 1] - tmp[i];
      I.min_d[a] = *std::min_element(I.e_size[a].begin(), I.e_size[a].end());
    }
  }
  const Index nx = _n[0], ny = _n[1], nz = _n[2];
  _dt = _cfl / (C_0 * std::sqrt(1.0 / (I.min_d[0] * I.min_d[0]) +
                                1.0 / (I.min_d[1] * I.min_d[1]) +
                                1.0 / (I.min_d[2] * I.min_d[2])));
  const Real dt = _dt;
  _calc = std::make_shared<CalculationParam>(std::make_unique<TimeParam>(dt, time_step, 0));
  const Real eps_tol = std::min({I.min_d[0], I.min_d[1], I.min_d[2]}) / 1000;
  if (_objects.size() >= kNoCell) throw XFDTDException("too many objects");

  // ------------------------------------------------------------ painting
  I.cell.assign(nx * ny * nz, 0);
  for (std::size_t idx = 0; idx < _objects.size(); ++idx) {
    const auto& o = _objects[idx];
    I.painters.push_back(o->material().get());
    const auto& mp = o->material()->emProperty();
    if (o->material()->dispersion()) {
      auto air = ElectroMagneticProperty::air();
      I.mat.push_back({air.epsilon(), air.mu(), air.sigmaE(), air.sigmaM()});
    } else {
      I.mat.push_back({mp.epsilon(), mp.mu(), mp.sigmaE(), mp.sigmaM()});
    }
    if (std::dynamic_pointer_cast<PecPlane>(o)) continue;  // paints no cells
    // Only cells whose centre lies within the wrapped cube (+ tolerance) can
    // test inside; the reference tests every cell with the same predicate.
    auto wc = o->shape()->wrappedCube();
    Index r0[3], r1[3];
    for (int a = 0; a < 3; ++a) {
      const auto& hn = I.h_node[a];
      const Real a0 = wc->origin()(a) - 2 * eps_tol, a1 = wc->end()(a) + 2 * eps_tol;
      r0[a] = std::lower_bound(hn.begin(), hn.end(), a0) - hn.begin();
      r1[a] = std::upper_bound(hn.begin(), hn.end(), a1) - hn.begin();
    }
    const Shape* sh = o->shape().get();
#pragma omp parallel for schedule(static)
    for (Index i = r0[0]; i < r1[0]; ++i)
      for (Index j = r0[1]; j < r1[1]; ++j)
        for (Index k = r0[2]; k < r1[2]; ++k)
          if (sh->isInside(I.h_node[0][i], I.h_node[1][j], I.h_node[2][k], eps_tol))
            I.cell[(i * ny + j) * nz + k] = static_cast<uint16_t>(idx);
  }

  // ------------------------------------------------------ material classes
  const MatP def{EPSILON_0, MU_0, constant::SIGMA_E_ZERO_APPROX, constant::SIGMA_M_ZERO_APPROX};
  // Beside each class row: the averaged (eps, sigma_e) of Ex, Ey, Ez, from
  // which later coefficient changes (PEC planes, lumped elements) start, as
  // the reference's start from its eps / sigma arrays.
  std::vector<double> class_es;
  auto classRow = [&](const ClassKey& key, double* row, double* es) {
    auto P = [&](int a, int b, int c) -> const MatP& {
      const uint16_t m = key.m[a * 4 + b * 2 + c];
      return m == kNoCell ? def : I.mat[m];
    };
    const bool ig = key.flags & 1, il = key.flags & 2, jg = key.flags & 4, jl = key.flags & 8,
               kg = key.flags & 16, kl = key.flags & 32;
    auto eCoef = [&](Real eps, Real sig, double* out) {
      out[0] = (2 * eps - dt * sig) / (2 * eps + dt * sig);
      out[1] = (2 * dt) / (2 * eps + sig * dt);
      es[out - row] = eps;
      es[out - row + 1] = sig;
    };
    auto hCoef = [&](Real mu, Real sig, double* out) {
      out[0] = (2 * mu - dt * sig) / (2 * mu + dt * sig);
      out[1] = (2 * dt) / (2 * mu + sig * dt);
    };
    auto avg4 = [](Real a, Real b, Real c, Real d) { return 0.25 * (((a + b) + c) + d); };
    auto harm = [](Real a, Real b) { return 2 * a * b / (a + b); };
    std::fill(row, row + 12, 0.0);
    std::fill(es, es + 6, 0.0);
    // Ex(i, j, k): cells (i, j-1..j, k-1..k)
    if (il) {
      if (jg && jl && kg && kl) {
        eCoef(avg4(P(1, 1, 1).eps, P(1, 0, 1).eps, P(1, 1, 0).eps, P(1, 0, 0).eps),
              avg4(P(1, 1, 1).se, P(1, 0, 1).se, P(1, 1, 0).se, P(1, 0, 0).se), row + 0);
      } else if (jl && kl) {
        eCoef(P(1, 1, 1).eps, P(1, 1, 1).se, row + 0);
      } else {
        eCoef(def.eps, def.se, row + 0);
      }
    }
    // Ey(i, j, k): cells (i-1..i, j, k-1..k)
    if (jl) {
      if (ig && il && kg && kl) {
        eCoef(avg4(P(1, 1, 1).eps, P(0, 1, 1).eps, P(1, 1, 0).eps, P(0, 1, 0).eps),
              avg4(P(1, 1, 1).se, P(0, 1, 1).se, P(1, 1, 0).se, P(0, 1, 0).se), row + 2);
      } else if (il && kl) {
        eCoef(P(1, 1, 1).eps, P(1, 1, 1).se, row + 2);
      } else {
        eCoef(def.eps, def.se, row + 2);
      }
    }
    // Ez(i, j, k): cells (i-1..i, j-1..j, k)
    if (kl) {
      if (ig && il && jg && jl) {
        eCoef(avg4(P(1, 1, 1).eps, P(0, 1, 1).eps, P(1, 0, 1).eps, P(0, 0, 1).eps),
              avg4(P(1, 1, 1).se, P(0, 1, 1).se, P(1, 0, 1).se, P(0, 0, 1).se), row + 4);
      } else if (il && jl) {
        eCoef(P(1, 1, 1).eps, P(1, 1, 1).se, row + 4);
      } else {
        eCoef(def.eps, def.se, row + 4);
      }
    }
    // Hx(i, j, k): cells (i-1..i, j, k), harmonic mean
    if (jl && kl) {
      if (ig && il) {
        hCoef(harm(P(1, 1, 1).mu, P(0, 1, 1).mu), harm(P(1, 1, 1).sm, P(0, 1, 1).sm), row + 6);
      } else if (il) {
        hCoef(P(1, 1, 1).mu, P(1, 1, 1).sm, row + 6);
      } else {
        hCoef(def.mu, def.sm, row + 6);
      }
    }
    // Hy(i, j, k): cells (i, j-1..j, k)
    if (il && kl) {
      if (jg && jl) {
        hCoef(harm(P(1, 1, 1).mu, P(1, 0, 1).mu), harm(P(1, 1, 1).sm, P(1, 0, 1).sm), row + 8);
      } else if (jl) {
        hCoef(P(1, 1, 1).mu, P(1, 1, 1).sm, row + 8);
      } else {
        hCoef(def.mu, def.sm, row + 8);
      }
    }
    // Hz(i, j, k): cells (i, j, k-1..k)
    if (il && jl) {
      if (kg && kl) {
        hCoef(harm(P(1, 1, 1).mu, P(1, 1, 0).mu), harm(P(1, 1, 1).sm, P(1, 1, 0).sm), row + 10);
      } else if (kl) {
        hCoef(P(1, 1, 1).mu, P(1, 1, 1).sm, row + 10);
      } else {
        hCoef(def.mu, def.sm, row + 10);
      }
    }
  };
  const Index NX = nx + 1, NY = ny + 1, NZ = nz + 1;
  I.lattice_class.assign(NX * NY * NZ, 0);
  {
    std::unordered_map<ClassKey, uint16_t, ClassKeyHash> ids;
    ClassKey last{};
    uint16_t last_id = 0;
    bool have_last = false;
    for (Index i = 0; i < NX; ++i)
      for (Index j = 0; j < NY; ++j)
        for (Index k = 0; k < NZ; ++k) {
          ClassKey key{};
          key.flags = (i >= 1) | ((i < nx) << 1) | ((j >= 1) << 2) | ((j < ny) << 3) |
                      ((k >= 1) << 4) | ((k < nz) << 5);
          for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
              for (int c = 0; c < 2; ++c) {
                const long ci = (long)i - 1 + a, cj = (long)j - 1 + b, ck = (long)k - 1 + c;
                uint16_t m = kNoCell;
                if (ci >= 0 && ci < (long)nx && cj >= 0 && cj < (long)ny && ck >= 0 &&
                    ck < (long)nz)
                  m = I.cell[((Index)ci * ny + cj) * nz + ck];
                key.m[a * 4 + b * 2 + c] = m;
              }
          uint16_t id;
          if (have_last && key == last) {
            id = last_id;
          } else {
            auto it = ids.find(key);
            if (it == ids.end()) {
              if (ids.size() >= 65535) throw XFDTDException("more than 65535 material classes");
              id = static_cast<uint16_t>(ids.size());
              ids.emplace(key, id);
              I.table.resize(I.table.size() + 12);
              class_es.resize(class_es.size() + 6);
              classRow(key, I.table.data() + 12 * id, class_es.data() + 6 * id);
            } else {
              id = it->second;
            }
            last = key;
            last_id = id;
            have_last = true;
          }
          I.lattice_class[(i * NY + j) * NZ + k] = id;
        }
  }
  // Overrides create new classes: (base class, override tag) -> class.
  std::map<std::pair<uint16_t, int>, uint16_t> override_ids;
  auto overrideClass = [&](Index node, int tag,
                           const std::function<void(double*, double*)>& edit) {
    const uint16_t base = I.lattice_class[node];
    auto key = std::make_pair(base, tag);
    auto it = override_ids.find(key);
    if (it != override_ids.end()) {
      I.lattice_class[node] = it->second;
      return;
    }
    const std::size_t n_cls = I.table.size() / 12;
    if (n_cls >= 65535) throw XFDTDException("more than 65535 material classes");
    std::vector<double> row(I.table.begin() + 12 * base, I.table.begin() + 12 * base + 12);
    std::vector<double> es(class_es.begin() + 6 * base, class_es.begin() + 6 * base + 6);
    edit(row.data(), es.data());
    I.table.insert(I.table.end(), row.begin(), row.end());
    class_es.insert(class_es.end(), es.begin(), es.end());
    override_ids.emplace(key, static_cast<uint16_t>(n_cls));
    I.lattice_class[node] = static_cast<uint16_t>(n_cls);
  };
  auto lat = [&](Index i, Index j, Index k) { return (i * NY + j) * NZ + k; };

  // ------------------------------------------- lumped elements, object order
  // CurrentSource / VoltageSource / Resistor / Capacitor / Inductor ::init and
  // ::correctUpdateCoefficient (src/object/lumped_element/current_source.cpp:40-165,
  // voltage_source.cpp:47-163, resistor.cpp:27-127, capacitor.cpp:16-112,
  // inductor.cpp:23-105).  Per node: the cell sizes across (da, db) and along
  // (dc) the axis give beta; (2 eps + dt sigma) and (2 eps - dt sigma) come
  // from the (ca, cb) of the node's material class, so that a later element on
  // the same node replaces an earlier one, as the reference recomputes from
  // eps and sigma.
  struct CsH {
    int comp;
    int s[3], e[3];
    std::vector<double> coff, wave;
  };
  struct IndH {
    int comp;
    int s[3], e[3];
    std::vector<double> cecjc, cjcec;
  };
  struct LumpBox {
    int comp;
    int s[3], e[3];
  };
  std::vector<CsH> current_sources;
  std::vector<IndH> inductors;
  std::vector<LumpBox> lumped_boxes;
  std::map<Index, uint16_t> material_class;
  int override_tag = 0;
  // PecPlane::correctMaterialSpace (src/object/lumped_element/pec_plane.cpp:12-66),
  // applied after the averaging (src/simulation/simulation.cpp:628-635): the
  // PEC sigma_e on the plane's two tangential E components; eps unchanged.
  for (const auto& o : _objects) {
    auto pp = std::dynamic_pointer_cast<PecPlane>(o);
    if (!pp) continue;
    const Cube* cube = dynamic_cast<const Cube*>(pp->shape().get());
    if (!cube) throw XFDTDException("a PecPlane needs a Cube");
    Index gs[3], ge[3];
    for (int a = 0; a < 3; ++a) {
      gs[a] = nearestNode(I.e_node[a], cube->origin()(a));
      ge[a] = nearestNode(I.e_node[a], cube->end()(a));
    }
    int p = -1;
    for (int a = 0; a < 3 && p < 0; ++a)
      if (gs[a] == ge[a]) p = a;
    if (p < 0) throw XFDTDException(o->name() + " PecPlane is not a plane!");
    const Real sig_pec = pp->material()->emProperty().sigmaE();
    for (int c : {(p + 1) % 3, (p + 2) % 3}) {
      Index s[3], e[3];
      for (int a = 0; a < 3; ++a) {
        s[a] = gs[a];
        e[a] = a == p ? gs[a] + 1 : (a == c ? ge[a] : ge[a] + 1);
      }
      for (Index i = s[0]; i < e[0]; ++i)
        for (Index j = s[1]; j < e[1]; ++j)
          for (Index k = s[2]; k < e[2]; ++k)
            overrideClass(lat(i, j, k), -1 - c, [&](double* rw, double* es) {
              const Real eps = es[2 * c];
              rw[2 * c] = (2 * eps - dt * sig_pec) / (2 * eps + dt * sig_pec);
              rw[2 * c + 1] = (2 * dt) / (2 * eps + sig_pec * dt);
              es[2 * c + 1] = sig_pec;
            });
    }
  }
  // ThinWire::init and ::correctUpdateCoefficient (src/object/thin_wire.cpp:12-133)
  auto thinWire = [&](const ThinWire& tw) {
    const auto* cyl = dynamic_cast<const Cylinder*>(tw.shape().get());
    if (!cyl) throw XFDTDException("ThinWire::init: shape is not Cylinder");
    const int w = cyl->axis().axisIndex();
    if (w < 0) throw XFDTDException("ThinWire::init: invalid axis");
    const Real r = cyl->radius();
    const Real dx = _dl[0], dy = _dl[1], dz = _dl[2];
    const int u = (w + 1) % 3, v = (w + 2) % 3;
    if (!(r < _dl[u] / 2 && r < _dl[v] / 2))
      throw XFDTDException("ThinWire::init: wire is not thin enough");
    auto wc = cyl->wrappedCube();
    Index gs[3], ge[3];
    for (int a = 0; a < 3; ++a) {
      gs[a] = nearestNode(I.e_node[a], wc->origin()(a));
      ge[a] = nearestNode(I.e_node[a], wc->end()(a));
    }
    // E along the wire on its nodes: ce = ceh_a = ceh_b = 0.
    const int tag = override_tag++;
    for (Index t = gs[w]; t < ge[w]; ++t) {
      Index x[3];
      x[w] = t;
      x[u] = gs[u];
      x[v] = gs[v];
      overrideClass(lat(x[0], x[1], x[2]), tag, [&](double* rw, double*) {
        rw[2 * w] = 0;
        rw[2 * w + 1] = 0;
      });
    }
    // H coefficients next to the wire: (component, term a/b, node box, factor).
    auto scale = [&](int c, int term, Index i0, Index i1, Index j0, Index j1, Index k0, Index k1,
                     Real f) {
      for (Index i = i0; i < i1; ++i)
        for (Index j = j0; j < j1; ++j)
          for (Index k = k0; k < k1; ++k) {
            if (i >= _n[0] || j >= _n[1] || k >= _n[2])
              throw XFDTDException("ThinWire " + tw.name() + " reaches the domain's far faces");
            auto it = I.hterm.emplace(std::make_pair(lat(i, j, k), c),
                                      std::array<double, 2>{1.0, 1.0}).first;
            it->second[term] *= f;
          }
    };
    const Index is = gs[0], ie = ge[0], js = gs[1], je = ge[1], ks = gs[2], ke = ge[2];
    if (w == 0) {
      const Real khy = dz * std::atan(dy / dy) / dy;
      const Real khz = dy * std::atan(dz / dy) / dz;
      if (ks < 1 || js < 1) throw XFDTDException("ThinWire on the domain's faces");
      scale(1, 1, is, ie, js, js + 1, ks - 1, ks + 1, khy * 2 / std::log(dz / r));  // chyex
      scale(2, 0, is, ie, js - 1, js + 1, ks, ks + 1, khz * 2 / std::log(dy / r));  // chzex
    } else if (w == 1) {
      const Real khz = dx * std::atan(dz / dx) / dz;
      const Real khx = dz * std::atan(dx / dz) / dx;
      if (is < 1 || ks < 1) throw XFDTDException("ThinWire on the domain's faces");
      scale(2, 1, is - 1, is + 1, js, je, ks, ks + 1, khz * 2 / std::log(dx / r));  // chzey
      scale(0, 0, is, is + 1, js, je, ks - 1, ks + 1, khx * 2 / std::log(dz / r));  // chxey
    } else {
      const Real khx = dy * std::atan(dx / dy) / dx;
      const Real khy = dx * std::atan(dy / dx) / dy;
      if (is < 1 || js < 1) throw XFDTDException("ThinWire on the domain's faces");
      scale(0, 0, is, is + 1, js - 1, js + 1, ks, ke, khx * 2 / std::log(dy / r));  // chxey
      scale(1, 1, is - 1, is + 1, js, js + 1, ks, ke, khy * 2 / std::log(dx / r));  // chyex
    }
  };
  for (const auto& o : _objects) {
    if (auto tw = std::dynamic_pointer_cast<ThinWire>(o)) {
      thinWire(*tw);
      continue;
    }
    auto le = std::dynamic_pointer_cast<LumpedElement>(o);
    if (!le) continue;
    auto cs = std::dynamic_pointer_cast<CurrentSource>(o);
    auto vs = std::dynamic_pointer_cast<VoltageSource>(o);
    auto res = std::dynamic_pointer_cast<Resistor>(o);
    auto cap = std::dynamic_pointer_cast<Capacitor>(o);
    auto ind = std::dynamic_pointer_cast<Inductor>(o);
    const Cube* cube = dynamic_cast<const Cube*>(le->shape().get());
    if (!cube) throw XFDTDException("a lumped element needs a Cube");
    const int ax = static_cast<int>(le->xyz());
    const int A = (ax + 1) % 3, B = (ax + 2) % 3;
    Index gs[3], ge[3];
    for (int a = 0; a < 3; ++a) {
      gs[a] = nearestNode(I.e_node[a], cube->origin()(a));
      ge[a] = nearestNode(I.e_node[a], cube->end()(a));
    }
    LumpBox box;
    box.comp = ax;
    for (int a = 0; a < 3; ++a) {  // LumpedElement::rangeX/Y/Z
      box.s[a] = (int)gs[a];
      box.e[a] = (int)(a == ax ? ge[a] : ge[a] + 1);
    }
    lumped_boxes.push_back(box);
    const Index na = ge[A] - gs[A] + 1, nb = ge[B] - gs[B] + 1, nc = ge[ax] - gs[ax];
    // rf / cf / inf lambdas of the element's init, in the reference's order
    Real factor = 0, amp = 0;
    if (cs) {
      factor = cs->resistance() * na * nb / nc;
      amp = cs->waveform()->amplitude() / (na * nb);
      if (Axis::negative(cs->direction())) amp *= -1;
    } else if (vs) {
      factor = vs->resistance() * na * nb / nc;
      amp = vs->waveform()->amplitude() / nc;
      if (Axis::negative(vs->direction())) amp *= -1;
    } else if (res) {
      factor = res->resistance() * na * nb / nc;
    } else if (cap) {
      factor = cap->capacitance() * nc / (nc * nb);
    } else if (ind) {
      factor = ind->inductance() * na * nb / nc;
    } else {
      throw XFDTDException("unknown lumped element " + o->name());
    }
    CsH h;
    IndH hi;
    h.comp = hi.comp = ax;
    std::copy(box.s, box.s + 3, h.s);
    std::copy(box.e, box.e + 3, h.e);
    std::copy(box.s, box.s + 3, hi.s);
    std::copy(box.e, box.e + 3, hi.e);
    for (int i = box.s[0]; i < box.e[0]; ++i)
      for (int j = box.s[1]; j < box.e[1]; ++j)
        for (int k = box.s[2]; k < box.e[2]; ++k) {
          const int x[3] = {i, j, k};
          auto dsize = [&](int a) { return a == ax ? I.e_size[a][x[a]] : I.h_size[a][x[a]]; };
          const Real da = dsize(A), db = dsize(B), dc = dsize(ax);
          const Index node = lat(i, j, k);
          const uint16_t mat = material_class.emplace(node, I.lattice_class[node]).first->second;
          const Real eps = class_es[6 * mat + 2 * ax], sig = class_es[6 * mat + 2 * ax + 1];
          if (ind) {
            hi.cecjc.push_back(-(2 * dt) / (2 * eps + dt * sig));
            hi.cjcec.push_back(dt * dc / (factor * da * db));
            continue;
          }
          Real beta, ca;
          if (vs) {
            beta = dt * dc / (da * db * factor);
          } else if (cap) {
            beta = 2 * factor * dc / (da * db);
          } else {
            beta = (dt * dc) / (factor * da * db);
          }
          const Real den_b = 2 * eps + dt * sig + beta;
          ca = cap ? (2 * eps - dt * sig + beta) / den_b : (2 * eps - dt * sig - beta) / den_b;
          const Real cb = 2 * dt / den_b;
          if (cs) h.coff.push_back(-2 * dt / (den_b * (db * da)) * amp);
          if (vs) h.coff.push_back(-2 * dt / (den_b * (da * db * factor)) * amp);
          overrideClass(node, override_tag++, [&](double* rw, double*) {
            rw[2 * ax] = ca;
            rw[2 * ax + 1] = cb;
          });
        }
    if (cs || vs) {
      std::vector<Real> h_time = linspace((0 + 0.5) * dt, (0 + _steps + 0.5) * dt, _steps);
      const auto& w = cs ? cs->waveform() : vs->waveform();
      w->init(h_time);
      h.wave.assign(w->value().begin(), w->value().end());
      current_sources.push_back(std::move(h));
    }
    if (ind) inductors.push_back(std::move(hi));
  }

  // --------------------------------------------------------------- CPML
  std::vector<Real> ke[3], kh[3];
  for (int a = 0; a < 3; ++a) {
    ke[a].assign(_n[a] + 1, 1.0);
    kh[a].assign(_n[a], 1.0);
  }
  for (const auto& b : _boundaries) {
    auto p = std::dynamic_pointer_cast<PML>(b);
    if (!p) continue;
    Impl::SlabH S;
    S.axis = Axis::axisOf(p->direction());
    S.neg = Axis::negative(p->direction());
    S.n = std::abs(p->thickness());
    const int m = S.axis;
    if (S.n == 0) continue;
    S.e_start = S.neg ? 1 : (int)_n[m] - S.n;
    S.h_start = S.neg ? 0 : (int)_n[m] - S.n;
    const int n = S.n;
    std::vector<Real> gh(I.h_size[m].begin() + S.e_start, I.h_size[m].begin() + S.e_start + n);
    std::vector<Real> ge(I.e_size[m].begin() + S.h_start, I.e_size[m].begin() + S.h_start + n);
    auto rho = [&](const std::vector<Real>& size, Real frac) {
      // PML::calculateRhoE / calculateRhoM (src/boundary/pml.cpp:564-606)
      std::vector<Real> d(n);
      d[0] = size[0] - frac * size[0];
      Real sum = 0;
      for (int i = 1; i < n; ++i) {
        sum += size[i - 1];
        d[i] = sum + (size[i] - frac * size[i]);
      }
      sum += size[n - 1];
      if (S.neg) std::reverse(d.begin(), d.end());
      for (auto& v : d) v /= sum;
      return d;
    };
    const int order = p->order();
    const Real e2m = MU_0 / EPSILON_0;
    const Real smax_e =
        p->sigmaRatio() * (order + 1) / (150 * PI * *std::min_element(gh.begin(), gh.end()));
    const Real smax_m = p->sigmaRatio() * (order + 1) /
                        (150 * PI * *std::min_element(ge.begin(), ge.end())) * e2m;
    auto re = rho(gh, 0.75), rm = rho(ge, 0.25);
    S.a_e.resize(n);
    S.b_e.resize(n);
    S.a_h.resize(n);
    S.b_h.resize(n);
    S.kappa_e.resize(n);
    S.kappa_h.resize(n);
    for (int l = 0; l < n; ++l) {
      const Real sig_e = smax_e * std::pow(re[l], order);
      const Real alp_e = p->alphaMin() + (p->alphaMax() - p->alphaMin()) * (1 - re[l]);
      const Real kap_e = 1 + (p->kappaMax() - 1) * std::pow(re[l], order);
      S.b_e[l] = std::exp((-dt / EPSILON_0) * (sig_e / kap_e + alp_e));
      S.a_e[l] = (S.b_e[l] - 1) * sig_e / ((sig_e + kap_e * alp_e) * kap_e * gh[l]);
      S.kappa_e[l] = kap_e;
      const Real sig_m = smax_m * std::pow(rm[l], order);
      const Real alp_m = (p->alphaMin() + (p->alphaMax() - p->alphaMin()) * (1 - rm[l])) * e2m;
      const Real kap_h = 1 + (p->kappaMax() - 1) * std::pow(rm[l], order);
      S.b_h[l] = std::exp((-dt / MU_0) * (sig_m / kap_h + alp_m));
      S.a_h[l] = (S.b_h[l] - 1) * sig_m / ((sig_m + kap_h * alp_m) * kap_h * ge[l]);
      S.kappa_h[l] = kap_h;
      ke[m][S.e_start + l] = kap_e;
      kh[m][S.h_start + l] = kap_h;
    }
    I.slabs.push_back(std::move(S));
  }
  for (int a = 0; a < 3; ++a) {
    I.fe[a].resize(_n[a] + 1);
    I.fh[a].resize(_n[a]);
    for (Index x = 0; x <= _n[a]; ++x) I.fe[a][x] = 1.0 / (I.h_size[a][x] * ke[a][x]);
    for (Index x = 0; x < _n[a]; ++x) I.fh[a][x] = 1.0 / (I.e_size[a][x] * kh[a][x]);
  }

  // ---------------------------------------------------------------- ADE
  std::vector<const LinearDispersiveMaterial*> disp;
  for (auto* m : I.painters)
    if (m->dispersion()) disp.push_back(dynamic_cast<const LinearDispersiveMaterial*>(m));
  int ade_kind = -1;
  int num_pole = 0;
  std::vector<double> ade_coef;
  std::vector<uint8_t> ade_comp, ade_mat;
  std::vector<int32_t> ade_node;
  if (!disp.empty()) {
    bool d_drude = false, d_debye = false, d_lor = false;
    for (auto* m : disp) {
      if (!m) throw XFDTDException("dispersive material is not a LinearDispersiveMaterial");
      num_pole = std::max<int>(num_pole, (int)m->numPoles());
      d_drude |= m->kind() == LinearDispersiveMaterial::Kind::Drude;
      d_debye |= m->kind() == LinearDispersiveMaterial::Kind::Debye;
      d_lor |= m->kind() == LinearDispersiveMaterial::Kind::MLorentz;
    }
    // Simulation::buildDispersiveSpace storage choice (simulation.cpp:800-818)
    ade_kind = (d_drude && !d_debye && !d_lor) ? 1 : (!d_drude && d_debye && !d_lor) ? 2 : 0;
    // Per painter: ADE material slot, coefficients, overwritten (ca, cb).
    std::vector<int> slot(I.painters.size(), -1);
    std::vector<std::array<double, 2>> e_coef;
    const int stride = 2 + 7 * num_pole;
    for (std::size_t pi = 0; pi < I.painters.size(); ++pi) {
      auto* m = dynamic_cast<const LinearDispersiveMaterial*>(I.painters[pi]);
      if (!m || !m->dispersion()) continue;
      if (slot.size() > 0 && (int)e_coef.size() >= 256)
        throw XFDTDException("more than 256 dispersive objects");
      slot[pi] = (int)e_coef.size();
      std::vector<double> c(stride, 0.0);
      const Real eps_inf = m->epsilonInf();
      const Real sigma = m->emProperty().sigmaE();
      const int P = (int)m->numPoles();
      if (ade_kind == 0) {
        // MLorentzADEMethodStorage::correctCoeff (m_lor_ade_method.cpp:66-159)
        std::vector<Real> a(P), bb(P), cc(P), d(P), e(P), f(P);
        for (int p = 0; p < P; ++p) {
          const auto& q = m->pole(p);
          const Real a0 = q[0], a1 = q[1], b0 = q[2], b1 = q[3], b2 = q[4];
          a[p] = (a1 * EPSILON_0 / (dt * dt)) + (0.5 * a0 * EPSILON_0 / dt);
          bb[p] = (-2 * a1 * EPSILON_0) / (dt * dt);
          cc[p] = (a1 * EPSILON_0 / (dt * dt)) - (0.5 * a0 * EPSILON_0 / dt);
          d[p] = (2 * b2 / (dt * dt)) - b0;
          e[p] = (-b2 / (dt * dt)) + (b1 / (2 * dt));
          f[p] = (b2 / (dt * dt)) + (b1 / (2 * dt));
        }
        Real sum_a = 0, sum_b = 0, sum_c = 0;
        for (int p = 0; p < P; ++p) sum_a += a[p] / f[p];
        for (int p = 0; p < P; ++p) sum_b += bb[p] / f[p];
        for (int p = 0; p < P; ++p) sum_c += cc[p] / f[p];
        const Real temp = (eps_inf * EPSILON_0) / dt + 0.5 * sum_a + 0.5 * sigma;
        c[0] = -1 / temp;
        c[1] = -0.5 * sum_c / temp;
        for (int p = 0; p < P; ++p) {
          double* pc = &c[2 + 7 * p];
          pc[0] = d[p] / f[p];
          pc[1] = e[p] / f[p];
          pc[2] = a[p] / f[p];
          pc[3] = bb[p] / f[p];
          pc[4] = cc[p] / f[p];
          pc[5] = 0.5 * (1 + d[p] / f[p]);
          pc[6] = 0.5 * (e[p] / f[p]);
        }
        e_coef.push_back({((eps_inf * EPSILON_0) / dt - 0.5 * sum_b - 0.5 * sigma) / temp,
                          1 / temp});
      } else if (ade_kind == 1) {
        // DrudeADEMethodStorage::correctCoeff (drude_ade_method.cpp:61-133)
        Real sum_beta = 0;
        std::vector<Real> kk(P), beta(P);
        for (int p = 0; p < P; ++p) {
          const Real wp = m->native(p)[0], g = m->native(p)[1];
          kk[p] = (1 - g * dt / 2) / (1 + g * dt / 2);
          beta[p] = (EPSILON_0 * wp * wp * dt / 2) / (1 + g * dt / 2);
        }
        for (int p = 0; p < P; ++p) sum_beta += beta[p];
        const Real a = (2 * EPSILON_0 * eps_inf - dt * sum_beta - dt * sigma) /
                       (2 * EPSILON_0 * eps_inf - dt * sum_beta + dt * sigma);
        const Real b = (2 * dt) / (2 * EPSILON_0 * eps_inf - dt * sum_beta + dt * sigma);
        c[0] = -b;
        for (int p = 0; p < P; ++p) {
          c[2 + 7 * p + 0] = kk[p];
          c[2 + 7 * p + 3] = beta[p];
          c[2 + 7 * p + 5] = 0.5 * (1 + kk[p]);
        }
        e_coef.push_back({a, b});
      } else {
        // DebyeADEMethodStorage::correctCoeff (debye_ade_method.cpp:47-122)
        Real sum_beta = 0;
        std::vector<Real> kk(P), beta(P);
        for (int p = 0; p < P; ++p) {
          const Real es = m->native(p)[0], tau = m->native(p)[1];
          kk[p] = (2 * tau - dt) / (2 * tau + dt);
          beta[p] = (2 * EPSILON_0 * (es - eps_inf) * dt) / (2 * tau + dt);
        }
        for (int p = 0; p < P; ++p) sum_beta += beta[p];
        const Real a = (2 * EPSILON_0 * eps_inf + sum_beta - dt * sigma) /
                       (2 * EPSILON_0 * eps_inf + sum_beta + dt * sigma);
        const Real b = (2 * dt) / (2 * EPSILON_0 * eps_inf + sum_beta + dt * sigma);
        c[0] = -b;
        for (int p = 0; p < P; ++p) {
          c[2 + 7 * p + 0] = kk[p];
          c[2 + 7 * p + 3] = beta[p] / dt;
          c[2 + 7 * p + 5] = 0.5 * (1 + kk[p]);
        }
        e_coef.push_back({a, b});
      }
      ade_coef.insert(ade_coef.end(), c.begin(), c.end());
    }
    // CPML E layers per axis: dispersive cells there are not supported.
    std::vector<char> in_pml[3];
    for (int a = 0; a < 3; ++a) in_pml[a].assign(_n[a] + 1, 0);
    for (const auto& S : I.slabs)
      for (int l = 0; l < S.n; ++l) in_pml[S.axis][S.e_start + l] = 1;
    for (Index i = 0; i < nx; ++i)
      for (Index j = 0; j < ny; ++j)
        for (Index k = 0; k < nz; ++k) {
          const uint16_t pm = I.cell[(i * ny + j) * nz + k];
          if (slot[pm] < 0) continue;
          if (in_pml[0][i] || in_pml[1][j] || in_pml[2][k])
            throw XFDTDException(
                "a dispersive object reaches into the CPML; this engine keeps ADE media out of "
                "the absorbing layers");
          const auto& ec = e_coef[slot[pm]];
          // Object::handleDispersion -> correctCoeff overwrites Ex, Ey, Ez at (i,j,k).
          overrideClass(lat(i, j, k), 1000000 + slot[pm], [&](double* rw, double*) {
            for (int c = 0; c < 3; ++c) {
              rw[2 * c] = ec[0];
              rw[2 * c + 1] = ec[1];
            }
          });
          const Index x[3] = {i, j, k};
          for (int c = 0; c < 3; ++c) {
            if (x[(c + 1) % 3] < 1 || x[(c + 2) % 3] < 1) continue;  // E update ranges
            ade_comp.push_back((uint8_t)c);
            ade_node.push_back((int32_t)i);
            ade_node.push_back((int32_t)j);
            ade_node.push_back((int32_t)k);
            ade_mat.push_back((uint8_t)slot[pm]);
          }
        }
  }

  // ------------------------------------------- voxel objects: E overrides
  {
    std::vector<const VoxelObject*> vox;
    std::vector<int> painter_vobj(_objects.size(), -1);
    for (std::size_t idx = 0; idx < _objects.size(); ++idx)
      if (auto v = dynamic_cast<const VoxelObject*>(_objects[idx].get())) {
        painter_vobj[idx] = (int)vox.size();
        vox.push_back(v);
      }
    I.ovr.clear();
    if (!vox.empty()) {
      // Voxel of a painted cell: the voxel holding the cell centre.
      auto voxelOf = [&](Index ci, Index cj, Index ck, int& vo) -> int64_t {
        vo = -1;
        const uint16_t pm = I.cell[(ci * ny + cj) * nz + ck];
        if (pm >= painter_vobj.size() || painter_vobj[pm] < 0) return -1;
        vo = painter_vobj[pm];
        const VoxelObject* v = vox[(std::size_t)vo];
        const Cube* cube = static_cast<const Cube*>(v->shape().get());
        const Index x[3] = {ci, cj, ck};
        int64_t flat = 0;
        for (int a = 0; a < 3; ++a) {
          const Real w = cube->size()(a) / (Real)v->dims()[a];
          auto q = (int64_t)std::floor((I.h_node[a][x[a]] - cube->origin()(a)) / w);
          q = std::max<int64_t>(0, std::min<int64_t>(q, (int64_t)v->dims()[a] - 1));
          flat = flat * (int64_t)v->dims()[a] + q;
        }
        return flat;
      };
      // Bounding box of the voxel cells.
      Index lo[3] = {nx, ny, nz}, hi[3] = {0, 0, 0};
      bool any = false;
      for (Index i = 0; i < nx; ++i)
        for (Index j = 0; j < ny; ++j)
          for (Index k = 0; k < nz; ++k) {
            const uint16_t pm = I.cell[(i * ny + j) * nz + k];
            if (pm >= painter_vobj.size() || painter_vobj[pm] < 0) continue;
            any = true;
            const Index x[3] = {i, j, k};
            for (int a = 0; a < 3; ++a) {
              lo[a] = std::min(lo[a], x[a]);
              hi[a] = std::max(hi[a], x[a] + 1);
            }
          }
      if (any) {
        std::vector<char> e_pml[3];
        for (int a = 0; a < 3; ++a) e_pml[a].assign(_n[a] + 1, 0);
        for (const auto& S : I.slabs)
          for (int l = 0; l < S.n; ++l) e_pml[S.axis][S.e_start + l] = 1;
        int tf_lo[3] = {-1, -1, -1}, tf_hi[3] = {-1, -1, -1};
        for (const auto& src : _sources)
          if (auto t = std::dynamic_pointer_cast<TFSF3D>(src)) {
            const Index org[3] = {t->x(), t->y(), t->z()};
            for (int a = 0; a < 3; ++a) {
              tf_lo[a] = (int)org[a];
              tf_hi[a] = (int)(_n[a] - org[a]);
            }
          }
        auto cellMat = [&](Index ci, Index cj, Index ck, int& vo, int64_t& vx) -> MatP {
          vx = voxelOf(ci, cj, ck, vo);
          if (vx >= 0) {
            const VoxelObject* v = vox[(std::size_t)vo];
            return MatP{v->epsR()[(std::size_t)vx] * EPSILON_0, 0, v->sigmaE(), 0};
          }
          return I.mat[I.cell[(ci * ny + cj) * nz + ck]];
        };
        for (Index i = lo[0]; i <= std::min(hi[0], nx); ++i)
          for (Index j = lo[1]; j <= std::min(hi[1], ny); ++j)
            for (Index k = lo[2]; k <= std::min(hi[2], nz); ++k)
              for (int c = 0; c < 3; ++c) {
                const Index x[3] = {i, j, k};
                const Index n3[3] = {nx, ny, nz};
                if (x[c] >= n3[c]) continue;  // component out of range
                const int A = (c + 1) % 3, B = (c + 2) % 3;
                // The four cells of the edge average, in the order of the
                // class rows: (x), (x - e_A), (x - e_B), (x - e_A - e_B) for Ex
                // (A = y, B = z); Ey, Ez by the same rule on their axes.
                const bool full = x[A] >= 1 && x[A] < n3[A] && x[B] >= 1 && x[B] < n3[B];
                if (!full) continue;
                Index cells[4][3];
                for (int q = 0; q < 4; ++q)
                  for (int a = 0; a < 3; ++a) cells[q][a] = x[a];
                // Ex: P(1,1,1) P(1,0,1) P(1,1,0) P(1,0,0); Ey: P(1,1,1) P(0,1,1)
                // P(1,1,0) P(0,1,0); Ez: P(1,1,1) P(0,1,1) P(1,0,1) P(0,0,1).
                const int first = c == 0 ? 1 : 0;   // axis stepped by cells 1 and 3
                const int second = c == 2 ? 1 : 2;  // axis stepped by cells 2 and 3
                cells[1][first] -= 1;
                cells[2][second] -= 1;
                cells[3][first] -= 1;
                cells[3][second] -= 1;
                Impl::OvrE o{};
                bool touches = false;
                MatP m[4];
                for (int q = 0; q < 4; ++q) {
                  m[q] = cellMat(cells[q][0], cells[q][1], cells[q][2], o.vobj[q], o.voxel[q]);
                  if (o.voxel[q] >= 0) touches = true;
                }
                if (!touches) continue;
                for (int a = 0; a < 3; ++a)
                  if (e_pml[a][x[a]] && a != c)
                    throw XFDTDException("a VoxelObject reaches into the CPML");
                for (int m2 = 0; m2 < 3 && tf_lo[0] >= 0; ++m2) {
                  const long long xm = (long long)x[m2];
                  if (xm != tf_lo[m2] && xm != tf_hi[m2]) continue;
                  bool within = true;
                  for (int a = 0; a < 3; ++a)
                    if (a != m2)
                      within = within && (long long)x[a] >= tf_lo[a] && (long long)x[a] <= tf_hi[a];
                  if (within) throw XFDTDException("a VoxelObject touches a TFSF face");
                }
                for (const auto& h : lumped_boxes)
                  if (h.comp == c && i >= (Index)h.s[0] && i < (Index)h.e[0] &&
                      j >= (Index)h.s[1] && j < (Index)h.e[1] && k >= (Index)h.s[2] &&
                      k < (Index)h.e[2])
                    throw XFDTDException("a VoxelObject touches a lumped element");
                for (int q = 0; q < 4; ++q) {
                  const uint16_t pm = I.cell[(cells[q][0] * ny + cells[q][1]) * nz + cells[q][2]];
                  if (I.painters[pm]->dispersion())
                    throw XFDTDException("a VoxelObject borders a dispersive object");
                }
                auto avg4 = [](Real a, Real b, Real cc, Real d) {
                  return 0.25 * (((a + b) + cc) + d);
                };
                o.eps = avg4(m[0].eps, m[1].eps, m[2].eps, m[3].eps);
                o.sig = avg4(m[0].se, m[1].se, m[2].se, m[3].se);
                o.ca = (2 * o.eps - dt * o.sig) / (2 * o.eps + dt * o.sig);
                o.cb = (2 * dt) / (2 * o.eps + o.sig * dt);
                o.w = 0.25;
                o.node[0] = (int32_t)i;
                o.node[1] = (int32_t)j;
                o.node[2] = (int32_t)k;
                o.comp = c;
                I.ovr.push_back(o);
              }
      }
    }
  }

  if (!_use_engine) {
    setupTfsf(nullptr);
    I.initialised = true;
    return;
  }
  // ------------------------------------------------------------- engine
  xfd_grid_desc g{};
  g.nx = (int32_t)nx;
  g.ny = (int32_t)ny;
  g.nz = (int32_t)nz;
  g.precision = _precision == Precision::FP64 ? XFD_FP64 : XFD_FP32;
  g.n_steps = (int64_t)_steps;
  g.dt = dt;
  g.device = 0;
  if (xfd_create(&g, &_engine) != XFD_OK)
    throw XFDTDException(std::string("xfd_create failed: ") + xfd_last_error(nullptr));
  xfd_engine* E = _engine;
  for (const auto& [name, value] : _engine_options)
    checkStatus(E, xfd_set_option(E, name.c_str(), value), "xfd_set_option");
  checkStatus(E, xfd_set_material_classes(E, I.table.data(), (int32_t)(I.table.size() / 12),
                                          I.lattice_class.data()),
              "xfd_set_material_classes");
  if (!I.ovr.empty()) {
    std::vector<int32_t> on, oc;
    std::vector<double> oa, ob;
    for (const auto& o : I.ovr) {
      on.insert(on.end(), o.node, o.node + 3);
      oc.push_back(o.comp);
      oa.push_back(o.ca);
      ob.push_back(o.cb);
    }
    checkStatus(E, xfd_set_e_overrides(E, (int64_t)oc.size(), on.data(), oc.data(), oa.data(),
                                       ob.data()),
                "xfd_set_e_overrides");
  }
  if (!I.hterm.empty()) {
    // The scaled coefficient minus the one the class table applies.
    std::vector<int32_t> hn, hc;
    std::vector<double> ha, hb;
    for (const auto& [key, f] : I.hterm) {
      const Index node = key.first;
      const int c = key.second, ta = (c + 1) % 3, tb = (c + 2) % 3;
      const Index x[3] = {node / (NY * NZ), (node / NZ) % NY, node % NZ};
      const double cb = I.table[12 * I.lattice_class[node] + 6 + 2 * c + 1];
      const double che_a = cb * I.fh[tb][x[tb]], che_b = -cb * I.fh[ta][x[ta]];
      for (int a = 0; a < 3; ++a) hn.push_back((int32_t)x[a]);
      hc.push_back(c);
      ha.push_back(f[0] * che_a - che_a);
      hb.push_back(f[1] * che_b - che_b);
    }
    checkStatus(E, xfd_set_h_term_overrides(E, (int64_t)hc.size(), hn.data(), hc.data(),
                                            ha.data(), hb.data()),
                "xfd_set_h_term_overrides");
  }
  const double* fe[3] = {I.fe[0].data(), I.fe[1].data(), I.fe[2].data()};
  const double* fh[3] = {I.fh[0].data(), I.fh[1].data(), I.fh[2].data()};
  checkStatus(E, xfd_set_curl_factors(E, fe, fh), "xfd_set_curl_factors");
  for (const auto& S : I.slabs) {
    xfd_cpml_slab s{S.axis, S.neg, S.n, S.e_start, S.h_start,
                    S.a_e.data(), S.b_e.data(), S.a_h.data(), S.b_h.data()};
    checkStatus(E, xfd_add_cpml(E, &s), "xfd_add_cpml");
  }
  for (const auto& h : current_sources)
    checkStatus(E, xfd_add_current_source(E, h.comp, h.s, h.e, h.coff.data(), h.wave.data()),
                "xfd_add_current_source");
  for (const auto& h : inductors)
    checkStatus(E, xfd_add_inductor(E, h.comp, h.s, h.e, h.cecjc.data(), h.cjcec.data()),
                "xfd_add_inductor");
  if (ade_kind >= 0) {
    xfd_ade_desc a{ade_kind, num_pole, (int32_t)(ade_coef.size() / (2 + 7 * num_pole)),
                   ade_coef.data(), (int64_t)ade_comp.size(), ade_comp.data(), ade_node.data(),
                   ade_mat.data()};
    checkStatus(E, xfd_set_ade(E, &a), "xfd_set_ade");
  }
  setupTfsf(E);
  setupNf2ff(E);
  setupNf2ffTd(E);
  // Movie monitors (FieldMonitor box with the +1 origin shift at index 0,
  // src/monitor/field_monitor.cpp:17-67).
  for (const auto& mon : _monitors) {
    auto mv = std::dynamic_pointer_cast<MovieMonitor>(mon);
    if (!mv) continue;
    const Shape* sh = mv->frame()->shape().get();
    auto wc = sh->wrappedCube();
    Impl::MovieH h{mv.get(), -1, {}, {}};
    for (int a = 0; a < 3; ++a) {
      int s = (int)nearestNode(I.e_node[a], wc->origin()(a));
      int e = (int)nearestNode(I.e_node[a], wc->end()(a));
      int size = e - s;
      if (s == 0) {
        s += 1;
        size -= 1;
      }
      h.s[a] = s;
      h.e[a] = s + size;
    }
    checkStatus(E, xfd_add_movie(E, static_cast<int32_t>(mv->frame()->field()), h.s, h.e,
                                 (int32_t)mv->frameInterval(), &h.id),
                "xfd_add_movie");
    mv->setFrameShape({(std::size_t)(h.e[0] - h.s[0]), (std::size_t)(h.e[1] - h.s[1]),
                       (std::size_t)(h.e[2] - h.s[2])});
    I.movies.push_back(h);
  }
  // Voltage and current monitors as weighted probes.
  for (const auto& mon : _monitors) {
    if (auto vm = std::dynamic_pointer_cast<VoltageMonitor>(mon)) {
      std::vector<int32_t> comp, node;
      std::vector<double> w;
      voltageProbe(*vm, comp, node, w);
      checkStatus(E, xfd_add_probe(E, (int64_t)comp.size(), comp.data(), node.data(), w.data(),
                                   &vm->_probe),
                  "xfd_add_probe");
      vm->_time = linspace((0 + 1) * dt, (0 + _steps) * dt, _steps);
      vm->_data.assign(_steps, 0.0);
    } else if (auto cm = std::dynamic_pointer_cast<CurrentMonitor>(mon)) {
      std::vector<int32_t> comp, node;
      std::vector<double> w;
      currentProbe(*cm, comp, node, w);
      checkStatus(E, xfd_add_probe(E, (int64_t)comp.size(), comp.data(), node.data(), w.data(),
                                   &cm->_probe),
                  "xfd_add_probe");
      cm->_time = linspace((0 + 0.5) * dt, (0 + _steps + 0.5) * dt, _steps);
      cm->_data.assign(_steps, 0.0);
    }
  }
  // Network::init (src/network/network.cpp:32-45).
  for (const auto& n : _networks) n->init(dt);
  // Field time monitors: the last node of the shifted box, every step.
  for (const auto& mon : _monitors) {
    auto ft = std::dynamic_pointer_cast<FieldTimeMonitor>(mon);
    if (!ft) continue;
    Impl::ProbeH p{ft.get(), -1};
    int s[3], e[3];
    bool empty = false;
    for (int a = 0; a < 3; ++a) {
      int o = (int)nearestNode(I.e_node[a], ft->cube()->origin()(a));
      int en = (int)nearestNode(I.e_node[a], ft->cube()->end()(a));
      int size = en - o;
      if (o == 0) {
        o += 1;
        size -= 1;
      }
      if (size <= 0) empty = true;
      s[a] = o + size - 1;
      e[a] = o + size;
    }
    if (!empty)
      checkStatus(E, xfd_add_movie(E, static_cast<int32_t>(ft->field()), s, e, 1, &p.id),
                  "xfd_add_movie");
    const bool is_e = static_cast<int>(ft->field()) < 3;
    ft->timeMutable() = is_e ? linspace((0 + 1) * dt, (0 + _steps) * dt, _steps)
                             : linspace((0 + 0.5) * dt, (0 + _steps + 0.5) * dt, _steps);
    ft->dataMutable().assign(_steps, 0.0);
    I.probes.push_back(p);
  }
  I.initialised = true;
}

void Simulation::setEngineOption(const std::string& name, long long value) {
  if (_engine) checkStatus(_engine, xfd_set_option(_engine, name.c_str(), value), "xfd_set_option");
  _engine_options.emplace_back(name, value);
  if (name == "graph_chunk") _chunk = value;
}

void Simulation::advance(Index n) {
  if (!_impl->initialised || !_engine) throw XFDTDException("Simulation not initialised");
  checkStatus(_engine, xfd_run(_engine, (int64_t)n), "xfd_run");
  if (_calc) _calc->timeParam()->setCurrentTimeStep((std::size_t)xfd_current_step(_engine));
}

void Simulation::finish() {
  if (!_engine) throw XFDTDException("Simulation not initialised");
  Impl& I = *_impl;
  checkStatus(_engine, xfd_sync(_engine), "xfd_sync");
  // Fields back into the host EMF.
  const Index n[3] = {_n[0], _n[1], _n[2]};
  for (int c = 0; c < 6; ++c) {
    Index s[3];
    for (int d = 0; d < 3; ++d) {
      const bool along = (d == c % 3);
      s[d] = (c < 3) ? (along ? n[d] : n[d] + 1) : (along ? n[d] + 1 : n[d]);
    }
    _emf._f[c] = Array3D<Real>::from_shape({(std::size_t)s[0], (std::size_t)s[1], (std::size_t)s[2]});
    if (_precision == Precision::FP64) {
      checkStatus(_engine, xfd_download_field(_engine, c, _emf._f[c].data()), "download");
    } else {
      std::vector<float> tmp(_emf._f[c].size());
      checkStatus(_engine, xfd_download_field(_engine, c, tmp.data()), "download");
      std::copy(tmp.begin(), tmp.end(), _emf._f[c].data());
    }
  }
  for (auto& h : I.movies) {
    int64_t frames = 0;
    checkStatus(_engine, xfd_get_movie_frames(_engine, h.id, nullptr, 0, &frames), "movie");
    const std::size_t per = (std::size_t)(h.e[0] - h.s[0]) * (h.e[1] - h.s[1]) * (h.e[2] - h.s[2]);
    const std::size_t w = _precision == Precision::FP64 ? 8 : 4;
    std::vector<char> buf((std::size_t)frames * per * w);
    checkStatus(_engine, xfd_get_movie_frames(_engine, h.id, buf.data(), (int64_t)buf.size(),
                                              &frames),
                "movie");
    auto& out = h.mon->framesMutable();
    out.assign((std::size_t)frames, std::vector<Real>(per));
    for (int64_t f = 0; f < frames; ++f)
      for (std::size_t q = 0; q < per; ++q)
        out[f][q] = (w == 8) ? reinterpret_cast<double*>(buf.data())[f * per + q]
                             : reinterpret_cast<float*>(buf.data())[f * per + q];
    // The frames on disk, as the reference's MovieMonitor::update writes them
    // during its run (src/monitor/movie_monitor.cpp:26-34, 58-63): one
    // <outputDir>/<step, 5 digits>.npy per frame, the monitor box in (i, j, k).
    if (!h.mon->outputDir().empty()) {
      const std::filesystem::path dir{h.mon->outputDir()};
      std::filesystem::create_directories(dir);
      const std::size_t sx = (std::size_t)(h.e[0] - h.s[0]), sy = (std::size_t)(h.e[1] - h.s[1]),
                        sz = (std::size_t)(h.e[2] - h.s[2]);
      for (std::size_t f = 0; f < out.size(); ++f) {
        auto a = Array3D<Real>::from_shape({sx, sy, sz});
        std::copy(out[f].begin(), out[f].end(), a.data());
        std::ostringstream nm;
        nm << std::setw(5) << std::setfill('0') << f * h.mon->frameInterval();
        xt::dump_npy((dir / (nm.str() + ".npy")).string(), a);
      }
    }
  }
  for (auto& p : I.probes) {
    if (p.id < 0) continue;
    int64_t frames = 0;
    checkStatus(_engine, xfd_get_movie_frames(_engine, p.id, nullptr, 0, &frames), "probe");
    const std::size_t w = _precision == Precision::FP64 ? 8 : 4;
    std::vector<char> buf((std::size_t)frames * w);
    checkStatus(_engine, xfd_get_movie_frames(_engine, p.id, buf.data(), (int64_t)buf.size(),
                                              &frames),
                "probe");
    auto& d = p.mon->dataMutable();
    for (int64_t f = 0; f < frames && f < (int64_t)d.size(); ++f)
      d[f] = (w == 8) ? reinterpret_cast<double*>(buf.data())[f]
                      : reinterpret_cast<float*>(buf.data())[f];
  }
  for (const auto& mon : _monitors) {
    std::vector<Real>* d = nullptr;
    int id = -1;
    if (auto vm = std::dynamic_pointer_cast<VoltageMonitor>(mon)) {
      d = &vm->_data;
      id = vm->_probe;
    } else if (auto cm = std::dynamic_pointer_cast<CurrentMonitor>(mon)) {
      d = &cm->_data;
      id = cm->_probe;
    }
    if (!d || id < 0) continue;
    int64_t cnt = 0;
    checkStatus(_engine, xfd_get_probe(_engine, id, nullptr, 0, &cnt), "probe");
    d->assign((std::size_t)cnt, 0.0);
    checkStatus(_engine, xfd_get_probe(_engine, id, d->data(), cnt, &cnt), "probe");
  }
  if (!_nffts_td.empty()) {
    int64_t cnt = 0;
    checkStatus(_engine, xfd_get_nf2ff_td(_engine, nullptr, 0, &cnt), "nf2ff_td");
    auto& td = *_nffts_td[0];
    td._raw.assign((std::size_t)cnt, 0.0);
    checkStatus(_engine, xfd_get_nf2ff_td(_engine, td._raw.data(), cnt, &cnt), "nf2ff_td");
    td._c_dt = C_0 * _dt;
  }
  if (I.nf2ff) {
    int64_t cnt = 0;
    checkStatus(_engine, xfd_get_nf2ff(_engine, nullptr, 0, &cnt), "nf2ff");
    std::vector<double> raw(2 * (std::size_t)cnt);
    checkStatus(_engine, xfd_get_nf2ff(_engine, raw.data(), cnt, &cnt), "nf2ff");
    auto& acc = I.nf2ff->surfaceCurrentsMutable();
    acc.resize((std::size_t)cnt);
    for (int64_t q = 0; q < cnt; ++q) acc[q] = {raw[2 * q], raw[2 * q + 1]};
  }
}

std::vector<std::vector<Real>> Simulation::coefficientArrays() const {
  const Impl& I = *_impl;
  if (!I.initialised) throw XFDTDException("Simulation not initialised");
  const Index n[3] = {_n[0], _n[1], _n[2]};
  const Index NY = n[1] + 1, NZ = n[2] + 1;
  std::vector<std::vector<Real>> out;
  for (int h = 0; h < 2; ++h)
    for (int c = 0; c < 3; ++c) {
      Index s[3];
      for (int d = 0; d < 3; ++d) {
        const bool along = (d == c);
        s[d] = (h == 0) ? (along ? n[d] : n[d] + 1) : (along ? n[d] + 1 : n[d]);
      }
      const int ta = (c + 1) % 3, tb = (c + 2) % 3;
      std::vector<Real> c0(s[0] * s[1] * s[2]), ca(c0.size()), cb(c0.size());
      for (Index i = 0; i < s[0]; ++i)
        for (Index j = 0; j < s[1]; ++j)
          for (Index k = 0; k < s[2]; ++k) {
            const Index x[3] = {i, j, k};
            const double* row = &I.table[12 * I.lattice_class[(i * NY + j) * NZ + k]];
            const Real a = row[6 * h + 2 * c], b = row[6 * h + 2 * c + 1];
            const Index q = (i * s[1] + j) * s[2] + k;
            c0[q] = a;
            if (h == 0) {  // ceh_a = -cb fe_b, ceh_b = cb fe_a
              ca[q] = -b * I.fe[tb][x[tb]];
              cb[q] = b * I.fe[ta][x[ta]];
            } else {       // che_a = cb fh_b, che_b = -cb fh_a
              ca[q] = b * I.fh[tb][x[tb]];
              cb[q] = -b * I.fh[ta][x[ta]];
            }
          }
      if (h == 1)
        for (const auto& [key, f] : I.hterm) {
          if (key.second != c) continue;
          const Index node = key.first;
          const Index x[3] = {node / (NY * NZ), (node / NZ) % NY, node % NZ};
          const Index q = (x[0] * s[1] + x[1]) * s[2] + x[2];
          ca[q] *= f[0];
          cb[q] *= f[1];
        }
      if (h == 0)
        for (const auto& o : I.ovr) {
          if (o.comp != c) continue;
          const Index x[3] = {(Index)o.node[0], (Index)o.node[1], (Index)o.node[2]};
          const Index q = (x[0] * s[1] + x[1]) * s[2] + x[2];
          c0[q] = o.ca;
          ca[q] = -o.cb * I.fe[tb][x[tb]];
          cb[q] = o.cb * I.fe[ta][x[ta]];
        }
      out.push_back(std::move(c0));
      out.push_back(std::move(ca));
      out.push_back(std::move(cb));
    }
  return out;
}

// ------------------------------------------------------------ adjoint
namespace {
struct DftCtx {
  double dt, omega;
  int64_t t0;
};

// J = sum_p |F_p|^2, F_p = dt sum_n E^n(p) exp(-i omega t_n), t_n = (t0 + n + 1) dt;
// dJ/dE^n(p) = 2 dt Re(conj(F_p) exp(-i omega t_n)).
int32_t dftPower(void* user, int64_t N, int64_t P, const double* rec, double* drec,
                 double* value) {
  const auto* c = static_cast<const DftCtx*>(user);
  std::vector<double> fr((std::size_t)P, 0.0), fi((std::size_t)P, 0.0);
  std::vector<double> pr((std::size_t)N), pi((std::size_t)N);
  for (int64_t n = 0; n < N; ++n) {
    const double ph = c->omega * (double)(c->t0 + n + 1) * c->dt;
    pr[(std::size_t)n] = c->dt * std::cos(ph);
    pi[(std::size_t)n] = -c->dt * std::sin(ph);
  }
  for (int64_t n = 0; n < N; ++n)
    for (int64_t p = 0; p < P; ++p) {
      fr[(std::size_t)p] += rec[n * P + p] * pr[(std::size_t)n];
      fi[(std::size_t)p] += rec[n * P + p] * pi[(std::size_t)n];
    }
  double J = 0;
  for (int64_t p = 0; p < P; ++p) J += fr[(std::size_t)p] * fr[(std::size_t)p] + fi[(std::size_t)p] * fi[(std::size_t)p];
  for (int64_t n = 0; n < N; ++n)
    for (int64_t p = 0; p < P; ++p)
      drec[n * P + p] = 2 * (fr[(std::size_t)p] * pr[(std::size_t)n] + fi[(std::size_t)p] * pi[(std::size_t)n]);
  *value = J;
  return 0;
}
}  // namespace

Real Simulation::dftPowerObjective(Index n_steps, int field, const std::array<int, 3>& box_s,
                                   const std::array<int, 3>& box_e, Real freq,
                                   std::vector<Real>* grad, int voxel_object,
                                   Index checkpoint_interval) {
  Impl& I = *_impl;
  if (!I.initialised || !_engine) throw XFDTDException("Simulation not initialised");
  DftCtx ctx{_dt, 2 * PI * freq, (int64_t)xfd_current_step(_engine)};
  xfd_adjoint_desc d{};
  d.n_steps = (int64_t)n_steps;
  d.checkpoint_interval = (int32_t)std::max<Index>(1, checkpoint_interval);
  d.forward_only = grad ? 0 : 1;
  d.obj_field = field;
  for (int a = 0; a < 3; ++a) {
    d.obj_s[a] = box_s[a];
    d.obj_e[a] = box_e[a];
  }
  d.objective = &dftPower;
  d.user = &ctx;
  double J = 0;
  if (!grad) {
    checkStatus(_engine, xfd_adjoint_run(_engine, &d, &J, nullptr), "xfd_adjoint_run");
    return J;
  }
  // The design box: every overridden node (of any voxel object).
  const VoxelObject* vo = nullptr;
  int count = 0;
  for (const auto& o : _objects)
    if (auto v = dynamic_cast<const VoxelObject*>(o.get())) {
      if (count == voxel_object) vo = v;
      ++count;
    }
  if (!vo || I.ovr.empty()) throw XFDTDException("no such VoxelObject on the grid");
  int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
  for (const auto& o : I.ovr)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], o.node[a]);
      hi[a] = std::max(hi[a], o.node[a] + 1);
    }
  for (int a = 0; a < 3; ++a) {
    d.design_s[a] = lo[a];
    d.design_e[a] = hi[a];
  }
  const int64_t nd = (int64_t)(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
  std::vector<double> sens((std::size_t)(6 * nd), 0.0);
  checkStatus(_engine, xfd_adjoint_run(_engine, &d, &J, sens.data()), "xfd_adjoint_run");
  grad->assign(vo->epsR().size(), 0.0);
  const Real dt = _dt;
  for (const auto& o : I.ovr) {
    const int64_t p = ((int64_t)(o.node[0] - lo[0]) * (hi[1] - lo[1]) + (o.node[1] - lo[1])) *
                          (hi[2] - lo[2]) +
                      (o.node[2] - lo[2]);
    const double s0 = sens[(std::size_t)(o.comp * nd + p)];
    const double s1 = sens[(std::size_t)((3 + o.comp) * nd + p)];
    // ca = (2 eps - sig dt) / (2 eps + sig dt), cb = 2 dt / (2 eps + sig dt)
    const double den = 2 * o.eps + o.sig * dt;
    const double dca = 4 * o.sig * dt / (den * den);
    const double dcb_cb = -2 / den;
    const double dj = (dca - o.ca * dcb_cb) * s0 + dcb_cb * s1;  // dJ/d(edge eps)
    for (int q = 0; q < 4; ++q)
      if (o.voxel[q] >= 0 && o.vobj[q] == voxel_object)
        (*grad)[(std::size_t)o.voxel[q]] += o.w * EPSILON_0 * dj;
  }
  return J;
}

void Simulation::setupTfsf(xfd_engine* E) {
  std::shared_ptr<TFSF3D> t;
  for (const auto& s : _sources) {
    if (auto p = std::dynamic_pointer_cast<TFSF3D>(s)) {
      if (t) throw XFDTDException("only one TFSF3D source is supported");
      t = p;
    } else {
      throw XFDTDException("unsupported waveform source (TFSF3D only)");
    }
  }
  if (!t) return;
  const Real dt = _dt;
  const Index org[3] = {t->x(), t->y(), t->z()};
  Index size[3];
  for (int a = 0; a < 3; ++a) {
    if (2 * org[a] >= _n[a]) throw XFDTDException("TFSF box is empty");
    size[a] = _n[a] - 2 * org[a];
  }
  // TFSF ctor / initTransform (src/waveform_source/tfsf.cpp:14-30, 231-254)
  const Real st = std::sin(t->theta()), ct = std::cos(t->theta());
  const Real sp = std::sin(t->phi()), cp = std::cos(t->phi());
  const Real ss = std::sin(t->psi()), cs = std::cos(t->psi());
  const Real k[3] = {st * cp, st * sp, ct};
  const Real va[3] = {-sp, ct * cp, st * cp}, vb[3] = {cp, ct * sp, st * sp},
             vc[3] = {0, -st, ct}, ke[3] = {ss, cs, 0};
  auto dot = [](const Real* x, const Real* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
  const Real te[3] = {dot(va, ke), dot(vb, ke), dot(vc, ke)};
  const Real th[3] = {k[1] * te[2] - k[2] * te[1], k[2] * te[0] - k[0] * te[2],
                      k[0] * te[1] - k[1] * te[0]};
  // TFSF::defaultInit (tfsf.cpp:118-175)
  const Real ratio = 1 / std::sqrt(std::pow(st, 4) * (std::pow(cp, 4) + std::pow(sp, 4)) +
                                   std::pow(ct, 4));
  const auto aux = static_cast<Index>(
      std::ceil(ratio * (std::sqrt(std::pow(size[0], 2) + std::pow(size[1], 2) +
                                   std::pow(size[2], 2)))) + 4 + 1);
  // calculateProjection / calculateInjectPostion (tfsf.cpp:256-340)
  std::vector<Real> p_int[3], p_half[3];
  for (int a = 0; a < 3; ++a) {
    const Real inj = k[a] >= 0 ? (Real)org[a] : (Real)(org[a] + size[a]);
    const Real inc = inj - (2 * k[a] / ratio);
    for (Index i = 0; i < size[a] + 1; ++i)
      p_int[a].push_back(((Real)i + (Real)org[a] - inc) * k[a] * ratio);
    for (Index i = 0; i < size[a] + 2; ++i)
      p_half[a].push_back(((Real)i + (Real)org[a] - inc - 0.5) * k[a] * ratio);
  }
  const Real scaled_dl = _dl[2] / ratio;
  const Real ceie = 1, chih = 1;
  const Real ceih = -(dt / (EPSILON_0 * scaled_dl));
  const Real chie = -(dt / (MU_0 * scaled_dl));
  const Real abc0 = (C_0 * dt - scaled_dl) / (C_0 * dt + scaled_dl);
  const Real abc1 = 2 * scaled_dl / (C_0 * dt + scaled_dl);
  // initTimeDependentVariable (tfsf.cpp:36-78): source sampled at eTime - dt.
  const Index nt = _steps;
  std::vector<Real> e_time = linspace((0 + 1) * dt, (0 + nt) * dt, nt);
  for (auto& v : e_time) v -= dt;
  t->waveform()->init(e_time);
  const auto& src = t->waveform()->value();
  const Index nl = aux - 1;
  std::vector<Real> e_inc(nt * aux, 0.0), h_inc(nt * nl, 0.0);
  auto E_ = [&](Index tt, Index l) -> Real& { return e_inc[tt * aux + l]; };
  auto H_ = [&](Index tt, Index l) -> Real& { return h_inc[tt * nl + l]; };
  if (nt > 0) {
    E_(0, 0) = src[0];
    for (Index l = 1; l < nl; ++l) H_(0, l) = chih * H_(0, l) + chie * (E_(0, l + 1) - E_(0, l));
  }
  for (Index tt = 1; tt < nt; ++tt) {
    for (Index l = 1; l < nl; ++l) {
      E_(tt, 0) = src[tt];
      E_(tt, l) = ceie * E_(tt - 1, l) + ceih * (H_(tt - 1, l) - H_(tt - 1, l - 1));
    }
    const Real ep2 = (tt < 2) ? 0.0 : E_(tt - 2, nl - 1);
    const Real el2 = (tt < 2) ? 0.0 : E_(tt - 2, nl);
    E_(tt, nl) = -ep2 + abc0 * (E_(tt, nl - 1) + el2) + abc1 * (E_(tt - 1, nl) + E_(tt - 1, nl - 1));
    for (Index l = 0; l < nl; ++l) H_(tt, l) = chih * H_(tt - 1, l) + chie * (E_(tt, l + 1) - E_(tt, l));
  }
  xfd_tfsf_desc d{};
  for (int a = 0; a < 3; ++a) {
    d.box_s[a] = (int32_t)org[a];
    d.box_e[a] = (int32_t)(org[a] + size[a]);
    d.p_int[a] = p_int[a].data();
    d.p_half[a] = p_half[a].data();
    d.ca[a] = dt / (EPSILON_0 * _dl[a]);  // TFSF::cax..caz (tfsf.cpp:177-205)
    d.cb[a] = dt / (MU_0 * _dl[a]);
    d.te[a] = te[a];
    d.th[a] = th[a];
  }
  d.aux = (int32_t)aux;
  d.e_inc = e_inc.data();
  d.h_inc = h_inc.data();
  if (E) checkStatus(E, xfd_set_tfsf(E, &d), "xfd_set_tfsf");
  auto& I = *_impl;
  I.tf_aux = (int)aux;
  for (int a = 0; a < 3; ++a) {
    I.tf_p_int[a] = p_int[a];
    I.tf_p_half[a] = p_half[a];
  }
  I.tf_e_inc = std::move(e_inc);
  I.tf_h_inc = std::move(h_inc);
}

Simulation::TfsfTables Simulation::tfsfTables() const {
  const Impl& I = *_impl;
  TfsfTables t;
  t.aux = I.tf_aux;
  t.e_inc = I.tf_e_inc;
  t.h_inc = I.tf_h_inc;
  for (int a = 0; a < 3; ++a) {
    t.p_int[a] = I.tf_p_int[a];
    t.p_half[a] = I.tf_p_half[a];
  }
  return t;
}

void Simulation::setupNf2ff(xfd_engine* E) {
  if (_nffts.empty()) return;
  if (_nffts.size() > 1) throw XFDTDException("one NFFFTFrequencyDomain per simulation");
  auto& nf = *_nffts[0];
  _impl->nf2ff = &nf;
  const auto d = nf.distance();
  // NFFFT::initGlobal / makeNodeAxisTask (src/nffft/nffft.cpp:88-245), one domain.
  xfd_nf2ff_desc desc{};
  for (int face = 0; face < 6; ++face) {
    const int m = face / 2;
    const bool positive = face % 2;
    int s[3], e[3];
    for (int a = 0; a < 3; ++a) {
      s[a] = (int)d[a];
      e[a] = (int)(_n[a] - d[a]);
    }
    const int c = positive ? e[m] : s[m];
    bool valid = positive ? (c < (int)_n[m]) : (c > 1);
    s[m] = c;
    e[m] = c + 1;
    for (int a = 0; a < 3; ++a) {
      if (a == m) continue;
      if (s[a] <= 0) s[a] = 1;
      if (e[a] >= (int)_n[a]) e[a] = (int)_n[a] - 1;
      if (e[a] <= s[a]) valid = false;
    }
    for (int a = 0; a < 3; ++a) {
      desc.task_s[face][a] = valid ? s[a] : 0;
      desc.task_e[face][a] = valid ? e[a] : 0;
      nf.faces[face][a] = desc.task_s[face][a];
      nf.faces[face][3 + a] = desc.task_e[face][a];
    }
  }
  const auto& freqs = nf.frequencies();
  const Index nt = _steps;
  const Real dt = _dt;
  std::vector<double> te(freqs.size() * nt * 2), th(freqs.size() * nt * 2);
  for (Index f = 0; f < freqs.size(); ++f)
    for (Index t = 0; t < nt; ++t) {
      // dt * exp(-j 2 pi f (t+1) dt), dt * exp(-j 2 pi f (t+1/2) dt)
      const Real ae = (-2.0 * PI) * ((freqs[f] * (Real)(t + 1)) * dt);
      const Real ah = (-2.0 * PI) * ((freqs[f] * ((Real)t + 0.5)) * dt);
      te[(f * nt + t) * 2] = dt * std::cos(ae);
      te[(f * nt + t) * 2 + 1] = dt * std::sin(ae);
      th[(f * nt + t) * 2] = dt * std::cos(ah);
      th[(f * nt + t) * 2 + 1] = dt * std::sin(ah);
    }
  desc.n_freq = (int32_t)freqs.size();
  desc.batch = 64;
  desc.te = te.data();
  desc.th = th.data();
  // The reference adds each step's term once per frequency plane
  // (nffft_frequency_domain.cpp:45-53).
  desc.scale = (double)freqs.size();
  checkStatus(E, xfd_set_nf2ff(E, &desc), "xfd_set_nf2ff");
  // Grid geometry for the far-field transform (GridSpace e/h nodes, e sizes).
  nf._engine = E;
  for (int a = 0; a < 3; ++a) {
    nf._node_e[a] = _impl->e_node[a];
    nf._node_h[a] = _impl->h_node[a];
    nf._size_e[a] = _impl->e_size[a];
  }
}

}  // namespace xfdtd

namespace xfdtd {

// NFFFT::initGlobal / makeNodeAxisTask (src/nffft/nffft.cpp:88-245), one
// domain: the six Huygens faces [s, e) of a box `d` cells inside the grid
// (all zero when a face is not valid).
static void huygensFaces(const Index n[3], const std::array<Index, 3>& d, int s_out[6][3],
                         int e_out[6][3]) {
  for (int face = 0; face < 6; ++face) {
    const int m = face / 2;
    const bool positive = face % 2;
    int s[3], e[3];
    for (int a = 0; a < 3; ++a) {
      s[a] = (int)d[a];
      e[a] = (int)(n[a] - d[a]);
    }
    const int c = positive ? e[m] : s[m];
    bool valid = positive ? (c < (int)n[m]) : (c > 1);
    s[m] = c;
    e[m] = c + 1;
    for (int a = 0; a < 3; ++a) {
      if (a == m) continue;
      if (s[a] <= 0) s[a] = 1;
      if (e[a] >= (int)n[a]) e[a] = (int)n[a] - 1;
      if (e[a] <= s[a]) valid = false;
    }
    for (int a = 0; a < 3; ++a) {
      s_out[face][a] = valid ? s[a] : 0;
      e_out[face][a] = valid ? e[a] : 0;
    }
  }
}

// ---------------------------------------------------------------- probes
namespace {
struct IRange {
  long long s, e;
  bool valid() const { return s < e; }
};
}  // namespace

// VoltageMonitor::init (src/monitor/voltage_monitor.cpp:17-180), one domain
// (node task = global task, lower corner 0, upper corner n): the a and b
// ranges of the cube's grid box extended by one node and kept off the domain
// edges, the c range as is; weight -h_c / (na nb) per node, negated for a
// negative direction (coff, :150-180).
void Simulation::voltageProbe(const VoltageMonitor& m, std::vector<int32_t>& comp,
                              std::vector<int32_t>& node, std::vector<double>& w) const {
  const Impl& I = *_impl;
  const int c = Axis::axisOf(m.direction()), a = (c + 1) % 3, b = (c + 2) % 3;
  long long o[3], e[3];
  for (int q = 0; q < 3; ++q) {
    o[q] = (long long)nearestNode(I.e_node[q], m.cube()->origin()(q));
    e[q] = (long long)nearestNode(I.e_node[q], m.cube()->end()(q));
  }
  auto clamp = [&](int ax, IRange r) {
    if (r.s <= 0) r.s = 1;
    if ((long long)_n[ax] <= r.e) r.e = (long long)_n[ax] - 1;
    return r;
  };
  IRange r[3];
  r[a] = clamp(a, IRange{o[a], e[a] + 1});
  r[b] = clamp(b, IRange{o[b], e[b] + 1});
  r[c] = IRange{o[c], e[c]};
  if (!r[0].valid() || !r[1].valid() || !r[2].valid())
    throw XFDTDException(m.name() + " globalTask is not valid");
  const long long nab = (r[a].e - r[a].s) * (r[b].e - r[b].s);
  for (long long i = r[0].s; i < r[0].e; ++i)
    for (long long j = r[1].s; j < r[1].e; ++j)
      for (long long k = r[2].s; k < r[2].e; ++k) {
        const long long x[3] = {i, j, k};
        double coff = -I.h_size[c][(std::size_t)x[c]] / (double)(std::size_t)nab;
        if (Axis::negative(m.direction())) coff *= -1.0;
        comp.push_back(c);
        node.push_back((int32_t)i);
        node.push_back((int32_t)j);
        node.push_back((int32_t)k);
        w.push_back(coff);
      }
}

// CurrentMonitor::init / update (src/monitor/current_monitor.cpp:17-379), one
// domain: the loop of H around the cube's face on its last node plane along
// the direction c, sides kept off the domain edges (make_ranges, :128-150).
void Simulation::currentProbe(const CurrentMonitor& m, std::vector<int32_t>& comp,
                              std::vector<int32_t>& node, std::vector<double>& w) const {
  const Impl& I = *_impl;
  const int c = Axis::axisOf(m.direction()), a = (c + 1) % 3, b = (c + 2) % 3;
  long long o[3], e[3];
  for (int q = 0; q < 3; ++q) {
    o[q] = (long long)nearestNode(I.e_node[q], m.cube()->origin()(q));
    e[q] = (long long)nearestNode(I.e_node[q], m.cube()->end()(q));
  }
  const long long n[3] = {(long long)_n[0], (long long)_n[1], (long long)_n[2]};
  if (e[c] == 0) throw XFDTDException("CurrentMonitor::init(): global_c_e is 0");
  if (o[a] == 0 || e[a] == n[a] || o[b] == 0 || e[b] == n[b])
    throw XFDTDException("CurrentMonitor::init(): global range is invalid");
  long long lo[3], hi[3];  // node task
  lo[a] = o[a];
  hi[a] = e[a];
  lo[b] = o[b];
  hi[b] = e[b];
  lo[c] = e[c] - 1;
  hi[c] = e[c];
  auto make_ranges = [](long long b_start, long long b_end, long long n_b, long long n_a,
                        long long start, long long end) {
    if (start <= 0) start = 1;
    end = end + 1;
    if (n_a <= end) end = n_a - 1;
    IRange rn{0, 0}, rp{0, 0};
    if (b_start != 0 && b_start != n_b - 1 && b_start != n_b) rn = IRange{start, end};
    if (b_end != n_b && b_end != n_b - 1 && b_end != 0) rp = IRange{start, end};
    return std::pair<IRange, IRange>{rn, rp};
  };
  const auto [ha_bn, ha_bp] = make_ranges(lo[b], hi[b], n[b], n[a], lo[a], hi[a]);
  const auto [hb_an, hb_ap] = make_ranges(lo[a], hi[a], n[a], n[b], lo[b], hi[b]);
  const double positive = Axis::negative(m.direction()) ? -1.0 : 1.0;
  // H_a along a at b = lo_b - 1 (+) and b = hi_b (-); H_b along b at
  // a = lo_a - 1 (-) and a = hi_a (+); all on the plane c = hi_c - 1.
  auto add = [&](int comp_axis, long long x[3], double weight) {
    comp.push_back(3 + comp_axis);
    for (int q = 0; q < 3; ++q) node.push_back((int32_t)x[q]);
    w.push_back(positive * weight);
  };
  long long x[3];
  x[c] = hi[c] - 1;
  for (long long v = ha_bn.s; ha_bn.valid() && v < ha_bn.e; ++v) {
    x[a] = v;
    x[b] = lo[b] - 1;
    add(a, x, I.e_size[a][(std::size_t)v]);
  }
  for (long long v = ha_bp.s; ha_bp.valid() && v < ha_bp.e; ++v) {
    x[a] = v;
    x[b] = hi[b];
    add(a, x, -I.e_size[a][(std::size_t)v]);
  }
  for (long long v = hb_an.s; hb_an.valid() && v < hb_an.e; ++v) {
    x[b] = v;
    x[a] = lo[a] - 1;
    add(b, x, -I.e_size[b][(std::size_t)v]);
  }
  for (long long v = hb_ap.s; hb_ap.valid() && v < hb_ap.e; ++v) {
    x[b] = v;
    x[a] = hi[a];
    add(b, x, I.e_size[b][(std::size_t)v]);
  }
}

namespace {
void writeTimeNpy(const std::string& dir, const std::string& name, const std::vector<Real>& t,
                  const std::vector<Real>& d) {
  namespace fs = std::filesystem;
  const fs::path root(dir.empty() ? "." : dir);
  fs::create_directories(root);
  std::ostringstream hdr;
  hdr << "{'descr': '<f8', 'fortran_order': False, 'shape': (2, " << t.size() << "), }";
  std::string h = hdr.str();
  const std::size_t total = 10 + h.size() + 1;
  h.append((64 - total % 64) % 64, ' ');
  h.push_back('\n');
  std::ofstream f((root / (name + ".npy")).string(), std::ios::binary);
  if (!f) throw XFDTDException("cannot write " + name + ".npy");
  f.write("\x93NUMPY\x01\x00", 8);
  const uint16_t len = static_cast<uint16_t>(h.size());
  f.write(reinterpret_cast<const char*>(&len), 2);
  f.write(h.data(), (std::streamsize)h.size());
  f.write(reinterpret_cast<const char*>(t.data()), (std::streamsize)(t.size() * sizeof(Real)));
  f.write(reinterpret_cast<const char*>(d.data()), (std::streamsize)(d.size() * sizeof(Real)));
}
}  // namespace

void VoltageMonitor::output() const {
  if (_probe >= 0) writeTimeNpy(outputDir(), name(), _time, _data);
}
void CurrentMonitor::output() const {
  if (_probe >= 0) writeTimeNpy(outputDir(), name(), _time, _data);
}

// NFFFTTimeDomain::initTimeDependentVariable / distanceRange and the per-point
// terms of TDPlaneData::update (src/nffft/nfffft_time_domain.cpp:49-78,
// 414-479; src/include/nffft/nffft_td_data.h:22-46, 169-240, 338-362).
void Simulation::setupNf2ffTd(xfd_engine* E) {
  if (_nffts_td.empty()) return;
  if (_nffts_td.size() > 1) throw XFDTDException("one NFFFTTimeDomain per simulation");
  const Impl& I = *_impl;
  auto& td = *_nffts_td[0];
  xfd_nf2ff_td_desc desc{};
  huygensFaces(_n, td.distance(), desc.task_s, desc.task_e);
  const Vector ru = td.observationDirection();
  // Point positions: e node along the face normal, h nodes across it.
  std::vector<Real> proj, ds;
  for (int face = 0; face < 6; ++face) {
    const int m = face / 2;
    const int* s = desc.task_s[face];
    const int* e = desc.task_e[face];
    for (int i = s[0]; i < e[0]; ++i)
      for (int j = s[1]; j < e[1]; ++j)
        for (int k = s[2]; k < e[2]; ++k) {
          const int x[3] = {i, j, k};
          Real r[3];
          for (int a = 0; a < 3; ++a) r[a] = a == m ? I.e_node[a][x[a]] : I.h_node[a][x[a]];
          proj.push_back(r[0] * ru(0) + r[1] * ru(1) + r[2] * ru(2));
          const int A = (m + 1) % 3, B = (m + 2) % 3;
          ds.push_back(I.e_size[A][x[A]] * I.e_size[B][x[B]]);
        }
  }
  if (proj.empty()) return;  // the reference's valid() is false: nothing recorded
  const Real lo = *std::min_element(proj.begin(), proj.end());
  const Real hi = *std::max_element(proj.begin(), proj.end());
  const Real dt = _dt;
  std::vector<Real> delay(proj.size());
  for (std::size_t q = 0; q < proj.size(); ++q) delay[q] = (hi - proj[q]) / (C_0 * dt);
  const Real aux = (hi - lo) / (C_0 * dt);
  desc.n_bins = (int64_t)((Index)std::ceil(aux) + _steps + 4);
  desc.delay = delay.data();
  desc.ds = ds.data();
  checkStatus(E, xfd_set_nf2ff_td(E, &desc), "xfd_set_nf2ff_td");
}

Vector NFFFTTimeDomain::observationDirection() const {
  return Vector{std::sin(_theta) * std::cos(_phi), std::sin(_theta) * std::sin(_phi),
                std::cos(_theta)};
}

Array1D<Real> NFFFTTimeDomain::scaled(int q) const {
  if (_raw.empty()) return Array1D<Real>::from_shape({std::size_t{0}});
  const std::size_t n = _raw.size() / 6;
  const Real den = _c_dt * 4 * PI;
  std::vector<Real> v(n);
  for (std::size_t b = 0; b < n; ++b) v[b] = _raw[q * n + b] / den;
  return Array1D<Real>(xt::adapt(v));
}

std::array<std::vector<Real>, 4> NFFFTTimeDomain::farField() const {
  std::array<std::vector<Real>, 4> out;
  if (_raw.empty()) return out;
  const auto wx_ = wx(), wy_ = wy(), wz_ = wz(), ux_ = ux(), uy_ = uy(), uz_ = uz();
  const Real ct = std::cos(_theta), st = std::sin(_theta), cp = std::cos(_phi),
             sp = std::sin(_phi);
  const std::size_t n = wx_.size();
  for (auto& v : out) v.resize(n);
  for (std::size_t b = 0; b < n; ++b) {
    out[0][b] = wx_[b] * ct * cp + wy_[b] * ct * sp - wz_[b] * st;
    out[1][b] = -wx_[b] * sp + wy_[b] * cp;
    out[2][b] = ux_[b] * ct * cp + uy_[b] * ct * sp - uz_[b] * st;
    out[3][b] = -ux_[b] * sp + uy_[b] * cp;
  }
  return out;
}

namespace {
void writeRealNpy(const std::string& path, const std::vector<Real>& v) {
  std::ostringstream hdr;
  hdr << "{'descr': '<f8', 'fortran_order': False, 'shape': (" << v.size() << ",), }";
  std::string h = hdr.str();
  const std::size_t total = 10 + h.size() + 1;
  h.append((64 - total % 64) % 64, ' ');
  h.push_back('\n');
  std::ofstream f(path, std::ios::binary);
  if (!f) throw XFDTDException("cannot write " + path);
  f.write("\x93NUMPY\x01\x00", 8);
  const uint16_t len = static_cast<uint16_t>(h.size());
  f.write(reinterpret_cast<const char*>(&len), 2);
  f.write(h.data(), (std::streamsize)h.size());
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(Real)));
}
}  // namespace

void NFFFTTimeDomain::processFarField() const {
  if (_raw.empty()) return;
  namespace fs = std::filesystem;
  const fs::path dir(_output_dir.empty() ? "." : _output_dir);
  fs::create_directories(dir);
  const auto ff = farField();
  static const char* names[4] = {"w_theta.npy", "w_phi.npy", "u_theta.npy", "u_phi.npy"};
  for (int q = 0; q < 4; ++q) writeRealNpy((dir / names[q]).string(), ff[q]);
}

}  // namespace xfdtd

// ---------------------------------------------------------------- far field
namespace xfdtd {

std::vector<std::complex<Real>> NFFFTFrequencyDomain::farField(const Array1D<Real>& theta,
                                                               const Array1D<Real>& phi,
                                                               const Vector& origin) const {
  if (theta.size() == 0 || phi.size() == 0) throw XFDTDException("Invalid theta or phi size");
  if (theta.size() != 1 && phi.size() != 1)
    throw XFDTDException("There must be only one theta or phi");
  if (!_engine) throw XFDTDException("far field: the simulation of this NF2FF is not running");
  // The angle list of the reference's broadcast of theta against phi.
  const std::size_t n = theta.size() * phi.size();
  std::vector<double> th(n), ph(n);
  for (std::size_t q = 0; q < n; ++q) {
    th[q] = theta.size() == 1 ? theta[0] : theta[q];
    ph[q] = phi.size() == 1 ? phi[0] : phi[q];
  }
  xfd_far_field_desc d{};
  d.n_angles = (int32_t)n;
  d.theta = th.data();
  d.phi = ph.data();
  d.n_freq = (int32_t)_freqs.size();
  d.freqs = _freqs.data();
  d.origin[0] = origin.x();
  d.origin[1] = origin.y();
  d.origin[2] = origin.z();
  for (int a = 0; a < 3; ++a) {
    d.node_e[a] = _node_e[a].data();
    d.node_h[a] = _node_h[a].data();
    d.size_e[a] = _size_e[a].data();
  }
  std::vector<std::complex<Real>> out(_freqs.size() * 4 * n);
  const int st = xfd_nf2ff_far_field(_engine, &d, reinterpret_cast<double*>(out.data()),
                                     (int64_t)out.size());
  if (st != XFD_OK)
    throw XFDTDException(std::string("xfd_nf2ff_far_field: ") + xfd_last_error(_engine));
  return out;
}

namespace {
void writeComplexNpy(const std::string& path, const std::complex<Real>* data, std::size_t n) {
  std::ostringstream hdr;
  hdr << "{'descr': '<c16', 'fortran_order': False, 'shape': (" << n << ",), }";
  std::string h = hdr.str();
  const std::size_t total = 10 + h.size() + 1;
  h.append((64 - total % 64) % 64, ' ');
  h.push_back('\n');
  std::ofstream f(path, std::ios::binary);
  if (!f) throw XFDTDException("cannot write " + path);
  f.write("\x93NUMPY\x01\x00", 8);
  const uint16_t len = static_cast<uint16_t>(h.size());
  f.write(reinterpret_cast<const char*>(&len), 2);
  f.write(h.data(), (std::streamsize)h.size());
  f.write(reinterpret_cast<const char*>(data), (std::streamsize)(n * sizeof(std::complex<Real>)));
}
}  // namespace

void NFFFTFrequencyDomain::processFarField(const Array1D<Real>& theta, const Array1D<Real>& phi,
                                           const std::string& sub_dir,
                                           const Vector& origin) const {
  const auto data = farField(theta, phi, origin);
  const std::size_t n = theta.size() * phi.size();
  const std::filesystem::path dir = std::filesystem::path(_output_dir) / sub_dir;
  std::filesystem::create_directories(dir);
  static const char* names[4] = {"_a_theta.npy", "_f_phi.npy", "_a_phi.npy", "_f_theta.npy"};
  for (std::size_t f = 0; f < _freqs.size(); ++f) {
    std::ostringstream ss;
    ss << std::fixed << std::setprecision(2) << _freqs[f] / 1e9 << "GHz";
    for (int r = 0; r < 4; ++r)
      writeComplexNpy((dir / (ss.str() + names[r])).string(), data.data() + (f * 4 + r) * n, n);
  }
}

void NFFFTFrequencyDomain::processFarField(const Array1D<Real>& theta, Real phi,
                                           const std::string& sub_dir,
                                           const Vector& origin) const {
  processFarField(theta, Array1D<Real>{phi}, sub_dir, origin);
}

void NFFFTFrequencyDomain::processFarField(Real theta, const Array1D<Real>& phi,
                                           const std::string& sub_dir,
                                           const Vector& origin) const {
  processFarField(Array1D<Real>{theta}, phi, sub_dir, origin);
}

std::vector<Real> NFFFTFrequencyDomain::radiationPower() const {
  const std::size_t nf = _freqs.size();
  std::size_t per_freq = 0, count[6];
  for (int f = 0; f < 6; ++f) {
    count[f] = 1;
    for (int a = 0; a < 3; ++a) count[f] *= (std::size_t)std::max(0, faces[f][3 + a] - faces[f][a]);
    per_freq += 4 * count[f];
  }
  if (nf == 0 || _acc.size() != nf * per_freq)
    throw XFDTDException("radiation power: no surface currents (run the simulation first)");
  std::vector<Real> out(nf);
  for (std::size_t q = 0; q < nf; ++q) {
    const std::complex<Real>* base = _acc.data() + q * per_freq;
    std::complex<Real> total{0.0};
    for (int f = 0; f < 6; ++f) {
      const int m = f / 2, A = (m + 1) % 3, B = (m + 2) % 3;
      const std::size_t n = count[f];
      const std::complex<Real>*ja = base, *jb = base + n, *ma = base + 2 * n, *mb = base + 3 * n;
      base += 4 * n;
      if (n == 0) continue;
      std::complex<Real> face{0.0};
      std::size_t p = 0;
      for (int i = faces[f][0]; i < faces[f][3]; ++i)
        for (int j = faces[f][1]; j < faces[f][4]; ++j)
          for (int k = faces[f][2]; k < faces[f][5]; ++k, ++p) {
            const int x[3] = {i, j, k};
            // ds: the E-cell sizes across the face (y z, z x, x y)
            const Real ds = _size_e[A][x[A]] * _size_e[B][x[B]];
            face += ds * (std::conj(ja[p]) * mb[p] - std::conj(jb[p]) * ma[p]);
          }
      total += (f % 2 == 0 ? -1.0 : 1.0) * face;
    }
    out[q] = 0.5 * std::real(total);
  }
  return out;
}

void NFFFTFrequencyDomain::outputRadiationPower() const {
  const auto power = radiationPower();
  const std::size_t n = power.size();
  auto data = Array2D<Real>::from_shape({2, n});
  for (std::size_t q = 0; q < n; ++q) {
    data(0, q) = _freqs[q];
    data(1, q) = power[q];
  }
  std::filesystem::create_directories(_output_dir.empty() ? "." : _output_dir);
  xt::dump_npy((std::filesystem::path(_output_dir) / "power.npy").string(), data);
}

// ---------------------------------------------------------------- network
namespace {
// dft (include/xfdtd/util/dft.h:9-26):
// X(f) = dt sum_n x_n exp(-j 2 pi f t_n), t_n = (n + 1) dt + shift.
std::vector<std::complex<Real>> timeDft(const std::vector<Real>& x, Real dt,
                                        const Array1D<Real>& freqs, Real shift) {
  std::vector<std::complex<Real>> out(freqs.size());
#pragma omp parallel for schedule(static)
  for (std::size_t q = 0; q < freqs.size(); ++q) {
    std::complex<Real> sum{0.0, 0.0};
    for (std::size_t n = 0; n < x.size(); ++n) {
      const Real t = (n + 1) * dt + shift;
      const Real ph = -2 * constant::PI * freqs[q] * t;
      sum += x[n] * std::complex<Real>(std::cos(ph), std::sin(ph));
    }
    out[q] = sum * dt;
  }
  return out;
}
}  // namespace

void Port::calculateSParameters(const Array1D<Real>& frequencies) {
  if (!_current_monitor || !_voltage_monitor || _current_monitor->data().empty() ||
      _voltage_monitor->data().empty())
    throw XFDTDException(
        "Port: Monitor is not valid. Please make sure you had add monitor to the simulation.");
  const Real dt = _dt;
  const std::complex<Real> z = _impedance;
  const Real k = std::sqrt(std::real(z));
  const auto i = timeDft(_current_monitor->data(), dt, frequencies, -1.5 * dt);
  const auto v = timeDft(_voltage_monitor->data(), dt, frequencies, 0.0);
  _a.resize(frequencies.size());
  _b.resize(frequencies.size());
  for (std::size_t q = 0; q < frequencies.size(); ++q) {
    _a[q] = Real{0.5} * (v[q] + z * i[q]) / k;
    _b[q] = Real{0.5} * (v[q] - std::conj(z) * i[q]) / k;
  }
}

void Network::init(Real dt) {
  std::set<std::size_t> seen;
  for (const auto& p : _ports) {
    p->init(dt);
    if (!seen.insert(p->index()).second) throw XFDTDException("Port index must be unique");
  }
}

void Network::compute() {
  for (auto& p : _ports) p->calculateSParameters(_frequencies);
  for (const auto& pi : _ports) {
    if (!pi->isSource()) continue;
    for (const auto& pj : _ports) {
      std::vector<std::complex<Real>> s(_frequencies.size());
      for (std::size_t q = 0; q < s.size(); ++q) s[q] = pj->b()[q] / pi->a()[q];
      _s_parameters[(int)(pj->index() * 10 + pi->index())] = std::move(s);
    }
  }
}

void Network::output() {
  compute();
  const std::filesystem::path out(_output_dir);
  std::filesystem::create_directories(out);
  for (const auto& [key, s] : _s_parameters)
    writeComplexNpy((out / ("s" + std::to_string(key) + ".npy")).string(), s.data(), s.size());
  writeRealNpy((out / "frequencies.npy").string(),
               std::vector<Real>(_frequencies.begin(), _frequencies.end()));
}

}  // namespace xfdtd
