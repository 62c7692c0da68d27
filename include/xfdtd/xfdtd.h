// xfdtd.h -- C++20 public API of the B200 host library (libxfdtd_host.so).
//
// Source-compatible subset of EMinsight/XFDTD_CORE's user API for the 3-D
// FDTD path: the same class names, constructor arguments and call sequence
// (include/xfdtd/simulation/simulation.h:37-155 and friends), so that a
// reference user program that builds a Simulation from Objects, PML
// boundaries, a TFSF3D source, CurrentSources, MovieMonitors and an
// NFFFTFrequencyDomain runs unchanged, with Simulation::run(n) executing the
// time loop on a B200 through the engine C ABI (xfd_engine.h).
//
// Deliberate differences, each documented at the member:
// * ThreadConfig is accepted and ignored (the time loop runs on the GPU).
// * The xt:: containers, builders and .npy writer come from the xtensor subset
//   in include/xtensor_subset (xtensor itself is not needed).
// * MPI is not used: MpiSupport keeps its calls and runs them as one rank.
// * Flag visitors are told about the time loop at the boundaries of the
//   engine's step chunks, not at every step.
// * Precision is chosen per Simulation (FP64 default, FP32 form optional)
//   instead of at build time (CMake XFDTD_CORE_SINGLE_PRECISION).
#pragma once

#include <array>
#include <cmath>
#include <complex>
#include <map>
#include <cstdint>
#include <cstdlib>
#include <functional>
#include <initializer_list>
#include <limits>
#include <memory>
#include <numbers>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "../xtensor_subset/xtensor/xt_core.hpp"

struct xfd_engine;

namespace xfdtd {

using Real = double;
using Index = std::size_t;

// ----------------------------------------------------------------- arrays
// The reference's array types (include/xfdtd/common/type_define.h:18-31):
// xtensor containers, here from the xtensor subset shipped beside this
// header (include/xtensor_subset; programs add it to their include path to
// use <xtensor/...> themselves).
template <typename T>
using Array1D = xt::xtensor<T, 1>;
template <typename T>
using Array2D = xt::xtensor<T, 2>;
template <typename T>
using Array3D = xt::xtensor<T, 3>;
template <typename T>
using Array4D = xt::xtensor<T, 4>;
template <typename T>
using Array = xt::xarray<T>;

// ------------------------------------------------------------- constants
// include/xfdtd/common/constant.h:11-18
namespace constant {
inline constexpr Real PI{std::numbers::pi_v<Real>};
inline constexpr Real EPSILON_0{8.854187817e-12};
inline constexpr Real MU_0{4 * PI * 1e-7};
inline const Real C_0{1 / std::sqrt(EPSILON_0 * MU_0)};
inline const Real Z_0{std::sqrt(MU_0 / EPSILON_0)};
inline constexpr Real SIGMA_E_ZERO_APPROX{1e-20};
inline constexpr Real SIGMA_M_ZERO_APPROX{1e-20};
inline constexpr Real INF{std::numeric_limits<Real>::infinity()};
inline constexpr Real NEG_INF{-std::numeric_limits<Real>::infinity()};
inline constexpr std::complex<Real> II{0.0, 1.0};
}  // namespace constant

class XFDTDException : public std::runtime_error {
 public:
  explicit XFDTDException(const std::string& m) : std::runtime_error(m) {}
};

// --------------------------------------------------------------- geometry
class Vector {
 public:
  Vector() = default;
  Vector(Real x, Real y, Real z) : _d{x, y, z} {}
  Real x() const { return _d[0]; }
  Real y() const { return _d[1]; }
  Real z() const { return _d[2]; }
  Real operator()(int a) const { return _d[a]; }
  Vector operator+(const Vector& o) const { return {x() + o.x(), y() + o.y(), z() + o.z()}; }
  Vector operator-(const Vector& o) const { return {x() - o.x(), y() - o.y(), z() - o.z()}; }
  Vector operator*(Real f) const { return {x() * f, y() * f, z() * f}; }
  Vector operator/(Real f) const { return {x() / f, y() / f, z() / f}; }
  bool operator==(const Vector& o) const { return _d == o._d; }
  bool operator!=(const Vector& o) const { return !(*this == o); }

 private:
  std::array<Real, 3> _d{0, 0, 0};
};

/// A unit vector along a coordinate axis, and the axis / direction enums
/// (include/xfdtd/coordinate_system/coordinate_system.h:93-170,
/// src/coordinate_system/asix.cpp).
class Axis : public Vector {
 public:
  enum class XYZ { X = 0, Y = 1, Z = 2 };
  enum class Direction { XN, XP, YN, YP, ZN, ZP };
  explicit Axis(const Vector& direction) : Vector{direction} {}
  bool operator==(const Axis& rhs) const { return Vector::operator==(rhs); }
  bool operator!=(const Axis& rhs) const { return !(*this == rhs); }
  bool operator==(Direction d) const { return *this == fromDirectionToAxis(d); }
  bool operator!=(Direction d) const { return !(*this == d); }
  /// True for both directions along the axis.
  bool operator==(XYZ c) const {
    const int a = static_cast<int>(c);
    return std::abs((*this)(a)) == 1 && (*this)((a + 1) % 3) == 0 && (*this)((a + 2) % 3) == 0;
  }
  bool operator!=(XYZ c) const { return !(*this == c); }
  static const Axis XN, XP, YN, YP, ZN, ZP;
  static Axis fromDirectionToAxis(Direction d) {
    const int a = axisOf(d);
    const Real s = negative(d) ? -1 : 1;
    return Axis{Vector{a == 0 ? s : 0, a == 1 ? s : 0, a == 2 ? s : 0}};
  }
  static XYZ fromDirectionToXYZ(Direction d) { return static_cast<XYZ>(axisOf(d)); }
  template <Direction d>
  static constexpr XYZ fromDirectionToXYZ() {
    return static_cast<XYZ>(static_cast<int>(d) / 2);
  }
  static constexpr XYZ tangentialAAxis(XYZ c) {
    return static_cast<XYZ>((static_cast<int>(c) + 1) % 3);
  }
  static constexpr XYZ tangentialBAxis(XYZ c) {
    return static_cast<XYZ>((static_cast<int>(c) + 2) % 3);
  }
  static bool directionNegative(Direction d) { return negative(d); }
  static bool directionPositive(Direction d) { return !negative(d); }
  template <Direction d>
  static constexpr bool directionNegative() { return static_cast<int>(d) % 2 == 0; }
  template <Direction d>
  static constexpr bool directionPositive() { return static_cast<int>(d) % 2 == 1; }
  static std::string toString(Direction d) {
    static const char* n[6] = {"XN", "XP", "YN", "YP", "ZN", "ZP"};
    return n[static_cast<int>(d)];
  }
  static std::string toString(XYZ c) {
    static const char* n[3] = {"X", "Y", "Z"};
    return n[static_cast<int>(c)];
  }
  /// The axis (0, 1, 2) of a direction, and whether it points down that axis.
  static int axisOf(Direction d) { return static_cast<int>(d) / 2; }
  static bool negative(Direction d) { return static_cast<int>(d) % 2 == 0; }
  /// The axis of this unit vector (0, 1, 2), or -1 when it is not along one.
  int axisIndex() const {
    for (int a = 0; a < 3; ++a)
      if (*this == static_cast<XYZ>(a)) return a;
    return -1;
  }
};
inline const Axis Axis::XN{Vector{-1, 0, 0}};
inline const Axis Axis::XP{Vector{1, 0, 0}};
inline const Axis Axis::YN{Vector{0, -1, 0}};
inline const Axis Axis::YP{Vector{0, 1, 0}};
inline const Axis Axis::ZN{Vector{0, 0, -1}};
inline const Axis Axis::ZP{Vector{0, 0, 1}};

class Cube;

class Shape {
 public:
  virtual ~Shape() = default;
  virtual bool isInside(Real x, Real y, Real z, Real eps) const = 0;
  virtual std::unique_ptr<Cube> wrappedCube() const = 0;
  virtual std::unique_ptr<Shape> clone() const = 0;
};

/// Cube(origin, size); end = origin + size (src/shape/cube.cpp).
class Cube : public Shape {
 public:
  Cube(Vector origin, Vector size) : _origin{origin}, _size{size}, _end{origin + size} {}
  bool isInside(Real x, Real y, Real z, Real eps) const override;
  std::unique_ptr<Cube> wrappedCube() const override { return std::make_unique<Cube>(*this); }
  std::unique_ptr<Shape> clone() const override { return std::make_unique<Cube>(*this); }
  const Vector& origin() const { return _origin; }
  const Vector& size() const { return _size; }
  const Vector& end() const { return _end; }
  Vector center() const { return _origin + _size / 2; }
  Real centerX() const { return center().x(); }
  Real centerY() const { return center().y(); }
  Real centerZ() const { return center().z(); }

 private:
  Vector _origin, _size, _end;
};

class Sphere : public Shape {
 public:
  Sphere(Vector center, Real radius) : _center{center}, _radius{radius} {}
  bool isInside(Real x, Real y, Real z, Real eps) const override;
  std::unique_ptr<Cube> wrappedCube() const override;
  std::unique_ptr<Shape> clone() const override { return std::make_unique<Sphere>(*this); }
  const Vector& center() const { return _center; }
  Real radius() const { return _radius; }

 private:
  Vector _center;
  Real _radius;
};

/// Cylinder(center, radius, height, axis) (src/shape/cylinder.cpp): the
/// points of its wrapped cube within `radius` of the axis line through
/// `center`.
class Cylinder : public Shape {
 public:
  Cylinder(Vector center, Real radius, Real height, Axis axis);
  bool isInside(Real x, Real y, Real z, Real eps) const override;
  std::unique_ptr<Cube> wrappedCube() const override;
  std::unique_ptr<Shape> clone() const override { return std::make_unique<Cylinder>(*this); }
  Vector center() const { return _center; }
  Real radius() const { return _radius; }
  Real height() const { return _height; }
  Axis axis() const { return _axis; }

 private:
  Vector _center;
  Real _radius, _height;
  Axis _axis;
};

// -------------------------------------------------------------- materials
/// ElectroMagneticProperty(eps_r, mu_r, sigma_e, sigma_m); zero conductivities
/// become 1e-20 (src/material/material.cpp:11-26).
class ElectroMagneticProperty {
 public:
  ElectroMagneticProperty(Real eps_r = 1, Real mu_r = 1, Real sigma_e = 0, Real sigma_m = 0);
  static ElectroMagneticProperty air() { return {1, 1, 0, 0}; }
  /// ElectroMagneticProperty::pec (src/material/material.cpp:32-34).
  static ElectroMagneticProperty pec() { return {1, 1, 1e10, 0}; }
  Real epsilonR() const { return _eps_r; }
  Real muR() const { return _mu_r; }
  Real sigmaE() const { return _sigma_e; }
  Real sigmaM() const { return _sigma_m; }
  Real epsilon() const { return _eps_r * constant::EPSILON_0; }
  Real mu() const { return _mu_r * constant::MU_0; }
  std::string toString() const {
    return "ElectroMagneticProperty{epsilon_r: " + std::to_string(_eps_r) +
           ", mu_r: " + std::to_string(_mu_r) + ", sigma_e: " + std::to_string(_sigma_e) +
           ", sigma_m: " + std::to_string(_sigma_m) + "}";
  }

 private:
  Real _eps_r, _mu_r, _sigma_e, _sigma_m;
};

class Material {
 public:
  Material(std::string_view name, ElectroMagneticProperty emp, bool dispersion = false)
      : _name{name}, _emp{emp}, _dispersion{dispersion} {}
  virtual ~Material() = default;
  static std::unique_ptr<Material> createAir() {
    return std::make_unique<Material>("air", ElectroMagneticProperty::air());
  }
  static std::unique_ptr<Material> createPec() {
    return std::make_unique<Material>("pec", ElectroMagneticProperty::pec());
  }
  const std::string& name() const { return _name; }
  const ElectroMagneticProperty& emProperty() const { return _emp; }
  bool dispersion() const { return _dispersion; }
  virtual std::string toString() const {
    return "Material{name: " + _name + ", em_property: " + _emp.toString() +
           ", dispersion: " + std::to_string(static_cast<int>(_dispersion)) + "}";
  }

 private:
  std::string _name;
  ElectroMagneticProperty _emp;
  bool _dispersion;
};

/// Linear dispersive medium in modified-Lorentz form with per-pole
/// (a0, a1, b0, b1, b2) (src/material/dispersive_material_equation.cpp:15-54).
class LinearDispersiveMaterial : public Material {
 public:
  enum class Kind { Drude, Debye, MLorentz };
  LinearDispersiveMaterial(std::string_view name, Real eps_inf, Kind kind,
                           std::vector<std::array<Real, 5>> poles,
                           std::vector<std::array<Real, 2>> native)
      : Material{name, ElectroMagneticProperty::air(), true},
        _eps_inf{eps_inf},
        _kind{kind},
        _poles{std::move(poles)},
        _native{std::move(native)} {}
  Real epsilonInf() const { return _eps_inf; }
  Kind kind() const { return _kind; }
  Index numPoles() const { return _poles.size(); }
  /// (a0, a1, b0, b1, b2) of pole p.
  const std::array<Real, 5>& pole(Index p) const { return _poles[p]; }
  /// Drude (omega_p, gamma) or Debye (eps_static, tau) of pole p.
  const std::array<Real, 2>& native(Index p) const { return _native[p]; }
  /// chi_p(f) = (a1 jw + a0) / (b2 (jw)^2 + b1 jw + b0), w = 2 pi f
  /// (MLorentzEqDecision::susceptibility,
  /// src/material/dispersive_material_equation.cpp:35-41).
  std::complex<Real> susceptibility(Real freq, Index p) const;
  /// eps_inf + sum_p chi_p(f) per frequency
  /// (LinearDispersiveMaterial::relativePermittivity,
  /// src/material/dipersive_material.cpp:31-41).
  Array1D<std::complex<Real>> relativePermittivity(const Array1D<Real>& freq) const;

 private:
  Real _eps_inf;
  Kind _kind;
  std::vector<std::array<Real, 5>> _poles;
  std::vector<std::array<Real, 2>> _native;
};

class DrudeMedium : public LinearDispersiveMaterial {
 public:
  using LinearDispersiveMaterial::LinearDispersiveMaterial;
  static std::unique_ptr<DrudeMedium> makeDrudeMedium(std::string_view name, Real eps_inf,
                                                      Array1D<Real> omega_p,
                                                      Array1D<Real> gamma);
};

class DebyeMedium : public LinearDispersiveMaterial {
 public:
  using LinearDispersiveMaterial::LinearDispersiveMaterial;
  static std::unique_ptr<DebyeMedium> makeDebyeMedium(std::string_view name, Real eps_inf,
                                                      Array1D<Real> eps_static,
                                                      Array1D<Real> tau);
};

class MLorentzMaterial : public LinearDispersiveMaterial {
 public:
  using LinearDispersiveMaterial::LinearDispersiveMaterial;
  static std::unique_ptr<MLorentzMaterial> makeMLorentz(std::string_view name, Real eps_inf,
                                                        Array1D<Real> a0, Array1D<Real> a1,
                                                        Array1D<Real> b0, Array1D<Real> b1,
                                                        Array1D<Real> b2);
};
using LorentzMedium = MLorentzMaterial;

// --------------------------------------------------------------- waveform
/// Waveform sampled once per run (src/waveform/waveform.cpp).
class Waveform {
 public:
  Waveform(std::function<Real(Real)> f, Real amplitude = 1.0)
      : _f{std::move(f)}, _amplitude{amplitude} {}
  static std::unique_ptr<Waveform> gaussian(Real tau, Real t_0, Real amplitude = 1.0);
  static std::unique_ptr<Waveform> cosineModulatedGaussian(Real tau, Real t_0, Real frequency,
                                                           Real amplitude = 1.0);
  static std::unique_ptr<Waveform> sine(Real frequency, Real amplitude = 1.0);
  static std::unique_ptr<Waveform> cosine(Real frequency, Real amplitude = 1.0);
  static std::unique_ptr<Waveform> square(Real frequency, Real amplitude = 1.0);
  /// As in the reference, the triangle wave keeps amplitude 1 whatever is
  /// passed (src/waveform/waveform.cpp:64-70).
  static std::unique_ptr<Waveform> triangle(Real frequency, Real amplitude = 1.0);
  static std::unique_ptr<Waveform> sawtooth(Real frequency, Real amplitude = 1.0);
  /// 1 from t_0 on, 0 before.
  static std::unique_ptr<Waveform> step(Real t_0, Real amplitude = 1.0);
  Real amplitude() const { return _amplitude; }
  Real operator()(Real t) const { return _f(t); }
  void init(const std::vector<Real>& time);
  const Array1D<Real>& value() const { return _value; }
  const Array1D<Real>& time() const { return _time; }

 private:
  std::function<Real(Real)> _f;
  Real _amplitude;
  Array1D<Real> _value, _time;
};

// ---------------------------------------------------------------- objects
class Object {
 public:
  Object(std::string name, std::unique_ptr<Shape> shape, std::unique_ptr<Material> material)
      : _name{std::move(name)}, _shape{std::move(shape)}, _material{std::move(material)} {}
  Object(std::string name, std::unique_ptr<Shape> shape, std::shared_ptr<Material> material)
      : _name{std::move(name)}, _shape{std::move(shape)}, _material{std::move(material)} {}
  virtual ~Object() = default;
  const std::string& name() const { return _name; }
  const std::unique_ptr<Shape>& shape() const { return _shape; }
  const std::shared_ptr<Material>& material() const { return _material; }

 private:
  std::string _name;
  std::unique_ptr<Shape> _shape;
  std::shared_ptr<Material> _material;
};

/// A block of per-voxel relative permittivities: the Cube divided into
/// dims[0] x dims[1] x dims[2] voxels (eps_r in C order, the last index
/// fastest); a cell whose centre lies in the Cube is painted, as for any
/// object, and takes the eps_r of the voxel holding its centre, with the
/// common mu_r and sigma_e.  This is the reference's extension point for
/// per-cell materials -- an Object subclass overriding correctMaterialSpace
/// (include/xfdtd/object/object.h:47) -- as a class of this library: the E
/// nodes whose averaging cells include a voxel get their own coefficients
/// (xfd_set_e_overrides), so any number of distinct voxel values costs no
/// material classes.  The voxels must stay clear of CPML layers, TFSF faces
/// and lumped sources.
class VoxelObject : public Object {
 public:
  VoxelObject(std::string name, std::unique_ptr<Cube> cube, std::array<Index, 3> dims,
              std::vector<Real> eps_r, Real mu_r = 1, Real sigma_e = 0);
  const std::array<Index, 3>& dims() const { return _dims; }
  const std::vector<Real>& epsR() const { return _eps_r; }
  Real muR() const { return _mu_r; }
  Real sigmaE() const { return _sigma_e; }

 private:
  std::array<Index, 3> _dims;
  std::vector<Real> _eps_r;
  Real _mu_r, _sigma_e;
};

/// Zero-thickness PEC sheet (src/object/lumped_element/pec_plane.cpp:9-66):
/// paints no cells; after the edge averaging its two tangential E components
/// on the plane take the PEC sigma_e.  The Cube must be flat on one axis.
class PecPlane : public Object {
 public:
  PecPlane(std::string name, std::unique_ptr<Cube> cube)
      : Object{std::move(name), std::move(cube), Material::createPec()} {}
};

/// Thin wire along a Cylinder's axis (src/object/thin_wire.cpp:9-152): air,
/// painted like any object; on a uniform grid with the radius below half the
/// cell on both transverse axes, the E component along the wire on the
/// wire's nodes is held at zero, and the H coefficients next to the wire that
/// the reference scales by k 2 / ln(d / r) (chyex, chzex for an x wire;
/// chzey, chxey for y; chxey, chyex for z -- the reference's choice) take
/// that factor.  Coefficient changes apply in object order with the lumped
/// elements'.
class ThinWire : public Object {
 public:
  ThinWire(const std::string& name, std::unique_ptr<Cylinder> shape)
      : Object{name, std::move(shape), Material::createAir()} {}
};

/// Lumped element on a Cube of E nodes along one axis
/// (include/xfdtd/object/lumped_element/lumped_element.h:19-104): the E_xyz
/// nodes of the Cube's grid box, its end included on the two other axes.
/// Elements change their nodes' E coefficients in the order they were added
/// (the last one on a node wins, each computed from the node's material).
class LumpedElement : public Object {
 public:
  LumpedElement(std::string name, std::unique_ptr<Cube> cube, Axis::XYZ xyz,
                std::unique_ptr<Material> material = Material::createAir())
      : Object{std::move(name), std::move(cube), std::move(material)}, _xyz{xyz} {}
  Axis::XYZ xyz() const { return _xyz; }

 private:
  Axis::XYZ _xyz;
};

/// Lumped current source on a Cube of E nodes along its direction
/// (src/object/lumped_element/current_source.cpp).  Resistance 0 becomes 1e-20;
/// an infinite resistance leaves the E coefficients unchanged (beta = 0).
class CurrentSource : public LumpedElement {
 public:
  CurrentSource(std::string name, std::unique_ptr<Cube> cube, Axis::Direction direction,
                Real resistance, std::unique_ptr<Waveform> waveform,
                std::unique_ptr<Material> material = Material::createAir())
      : LumpedElement{std::move(name), std::move(cube),
                      static_cast<Axis::XYZ>(Axis::axisOf(direction)), std::move(material)},
        _direction{direction},
        _resistance{resistance == 0 ? 1e-20 : resistance},
        _waveform{std::move(waveform)} {}
  Axis::Direction direction() const { return _direction; }
  Real resistance() const { return _resistance; }
  const std::unique_ptr<Waveform>& waveform() const { return _waveform; }

 private:
  Axis::Direction _direction;
  Real _resistance;
  std::unique_ptr<Waveform> _waveform;
};

/// Lumped voltage source with an internal resistance
/// (src/object/lumped_element/voltage_source.cpp:15-177): the amplitude is
/// split over the nodes along the axis, the resistance over the node count.
/// Resistance 0 becomes 1e-20.
class VoltageSource : public LumpedElement {
 public:
  VoltageSource(std::string name, std::unique_ptr<Cube> cube, Axis::Direction direction,
                Real resistance, std::unique_ptr<Waveform> waveform,
                std::unique_ptr<Material> material = Material::createAir())
      : LumpedElement{std::move(name), std::move(cube),
                      static_cast<Axis::XYZ>(Axis::axisOf(direction)), std::move(material)},
        _direction{direction},
        _resistance{resistance == 0 ? 1e-20 : resistance},
        _waveform{std::move(waveform)} {}
  Axis::Direction direction() const { return _direction; }
  Real resistance() const { return _resistance; }
  const std::unique_ptr<Waveform>& waveform() const { return _waveform; }

 private:
  Axis::Direction _direction;
  Real _resistance;
  std::unique_ptr<Waveform> _waveform;
};

/// Lumped resistor (src/object/lumped_element/resistor.cpp:12-131): E
/// coefficients only.  Resistance 0 becomes 1e-10.
class Resistor : public LumpedElement {
 public:
  Resistor(std::string name, std::unique_ptr<Cube> cube, Axis::XYZ xyz, Real resistance,
           std::unique_ptr<Material> material = Material::createAir())
      : LumpedElement{std::move(name), std::move(cube), xyz, std::move(material)},
        _resistance{resistance == 0 ? 1e-10 : resistance} {}
  Real resistance() const { return _resistance; }

 private:
  Real _resistance;
};

/// Lumped capacitor (src/object/lumped_element/capacitor.cpp:8-116): E
/// coefficients only.
class Capacitor : public LumpedElement {
 public:
  Capacitor(std::string name, std::unique_ptr<Cube> cube, Axis::XYZ xyz, Real capacitance,
            std::unique_ptr<Material> material = Material::createAir())
      : LumpedElement{std::move(name), std::move(cube), xyz, std::move(material)},
        _capacitance{capacitance} {}
  Real capacitance() const { return _capacitance; }

 private:
  Real _capacitance;
};

/// Lumped inductor (src/object/lumped_element/inductor.cpp:12-137): a
/// current state per node, advanced after every E update.  Inductance 0
/// becomes 1e-10.
class Inductor : public LumpedElement {
 public:
  Inductor(std::string name, std::unique_ptr<Cube> cube, Axis::XYZ xyz, Real inductance,
           std::unique_ptr<Material> material = Material::createAir())
      : LumpedElement{std::move(name), std::move(cube), xyz, std::move(material)},
        _inductance{inductance == 0 ? 1e-10 : inductance} {}
  Real inductance() const { return _inductance; }

 private:
  Real _inductance;
};

// --------------------------------------------------------------- boundary
class Boundary {
 public:
  virtual ~Boundary() = default;
};

/// CPML boundary (include/xfdtd/boundary/pml.h:19-21).
class PML : public Boundary {
 public:
  PML(int thickness, Axis::Direction direction, int order = 4, Real sigma_ratio = 1,
      Real alpha_min = 0, Real alpha_max = 0.05, Real kappa_max = 10)
      : _thickness{thickness},
        _direction{direction},
        _order{order},
        _sigma_ratio{sigma_ratio},
        _alpha_min{alpha_min},
        _alpha_max{alpha_max},
        _kappa_max{kappa_max} {}
  int thickness() const { return _thickness; }
  Axis::Direction direction() const { return _direction; }
  int order() const { return _order; }
  Real sigmaRatio() const { return _sigma_ratio; }
  Real alphaMin() const { return _alpha_min; }
  Real alphaMax() const { return _alpha_max; }
  Real kappaMax() const { return _kappa_max; }

 private:
  int _thickness;
  Axis::Direction _direction;
  int _order;
  Real _sigma_ratio, _alpha_min, _alpha_max, _kappa_max;
};

// --------------------------------------------------------- waveform source
class WaveformSource {
 public:
  explicit WaveformSource(std::unique_ptr<Waveform> w) : _waveform{std::move(w)} {}
  virtual ~WaveformSource() = default;
  const std::unique_ptr<Waveform>& waveform() const { return _waveform; }

 private:
  std::unique_ptr<Waveform> _waveform;
};

/// TFSF3D(x, y, z, theta, phi, psi, waveform): the total-field box starts x, y,
/// z cells from the grid faces (src/waveform_source/tfsf.cpp:118-175).
class TFSF3D : public WaveformSource {
 public:
  TFSF3D(std::size_t x, std::size_t y, std::size_t z, Real theta, Real phi, Real psi,
         std::unique_ptr<Waveform> waveform)
      : WaveformSource{std::move(waveform)}, _x{x}, _y{y}, _z{z}, _theta{theta}, _phi{phi},
        _psi{psi} {}
  std::size_t x() const { return _x; }
  std::size_t y() const { return _y; }
  std::size_t z() const { return _z; }
  Real theta() const { return _theta; }
  Real phi() const { return _phi; }
  Real psi() const { return _psi; }

 private:
  std::size_t _x, _y, _z;
  Real _theta, _phi, _psi;
};

// --------------------------------------------------------------- monitors
struct EMF {
  enum class Field { EX, EY, EZ, HX, HY, HZ };
  Array3D<Real>& field(Field f) { return _f[static_cast<int>(f)]; }
  const Array3D<Real>& field(Field f) const { return _f[static_cast<int>(f)]; }
  Array3D<Real>& ex() { return _f[0]; }
  Array3D<Real>& ey() { return _f[1]; }
  Array3D<Real>& ez() { return _f[2]; }
  Array3D<Real>& hx() { return _f[3]; }
  Array3D<Real>& hy() { return _f[4]; }
  Array3D<Real>& hz() { return _f[5]; }
  std::array<Array3D<Real>, 6> _f;
};

class Monitor {
 public:
  Monitor(std::string name, std::string output_dir)
      : _name{std::move(name)}, _output_dir{std::move(output_dir)} {}
  virtual ~Monitor() = default;
  const std::string& name() const { return _name; }
  const std::string& outputDir() const { return _output_dir; }
  void setOutputDir(std::string d) { _output_dir = std::move(d); }

 private:
  std::string _name, _output_dir;
};

class FieldMonitor : public Monitor {
 public:
  FieldMonitor(std::unique_ptr<Shape> shape, EMF::Field field, std::string name = "",
               std::string output_dir = "")
      : Monitor{std::move(name), std::move(output_dir)}, _shape{std::move(shape)},
        _field{field} {}
  const std::unique_ptr<Shape>& shape() const { return _shape; }
  EMF::Field field() const { return _field; }

 private:
  std::unique_ptr<Shape> _shape;
  EMF::Field _field;
};

/// MovieMonitor(frame, interval, name, dir): frame every `interval` steps from
/// step 0, written as <dir>/<frame index, 5 digits>.npy
/// (src/monitor/movie_monitor.cpp:26-34).
class MovieMonitor : public Monitor {
 public:
  MovieMonitor(std::unique_ptr<FieldMonitor> frame, std::size_t interval, std::string name,
               std::string output_dir)
      : Monitor{std::move(name), std::move(output_dir)}, _frame{std::move(frame)},
        _interval{interval} {}
  const std::unique_ptr<FieldMonitor>& frame() const { return _frame; }
  std::size_t frameInterval() const { return _interval; }
  /// Frames recorded by the last run, each the monitor box in (i, j, k) order.
  const std::vector<std::vector<Real>>& frames() const { return _frames; }
  std::array<std::size_t, 3> frameShape() const { return _shape; }
  std::vector<std::vector<Real>>& framesMutable() { return _frames; }
  void setFrameShape(std::array<std::size_t, 3> s) { _shape = s; }

 private:
  std::unique_ptr<FieldMonitor> _frame;
  std::size_t _interval;
  std::vector<std::vector<Real>> _frames;
  std::array<std::size_t, 3> _shape{0, 0, 0};
};

/// FieldTimeMonitor(name, cube, dir, field): every step, the field at the last
/// node of the cube's node box (the reference's update loop overwrites the
/// sample node by node, src/monitor/field_time_monitor.cpp:81-95).  After run,
/// time() holds the E or H time axis and data() the samples.
class FieldTimeMonitor : public Monitor {
 public:
  FieldTimeMonitor(std::string name, std::unique_ptr<Cube> cube, std::string output_dir,
                   EMF::Field field)
      : Monitor{std::move(name), std::move(output_dir)}, _cube{std::move(cube)}, _field{field} {}
  const std::unique_ptr<Cube>& cube() const { return _cube; }
  EMF::Field field() const { return _field; }
  const std::vector<Real>& time() const { return _time; }
  const std::vector<Real>& data() const { return _data; }
  std::vector<Real>& timeMutable() { return _time; }
  std::vector<Real>& dataMutable() { return _data; }

 private:
  std::unique_ptr<Cube> _cube;
  EMF::Field _field;
  std::vector<Real> _time, _data;
};

/// Voltage along `direction` across the cube's node box, every step
/// (src/monitor/voltage_monitor.cpp:17-235): the E component along the
/// direction, weighted by -h_c / (na nb) over the box (a, b extended by one
/// node and kept off the domain edges), sign flipped for a negative
/// direction.  time() = E times; output() writes <outputDir>/<name>.npy, a
/// (2, n_steps) array [time; data] (TimeMonitor::output, time_monitor.cpp:9-18).
class VoltageMonitor : public Monitor {
 public:
  VoltageMonitor(std::string name, std::unique_ptr<Cube> cube, Axis::Direction direction,
                 std::string output_dir = "")
      : Monitor{std::move(name), std::move(output_dir)},
        _cube{std::move(cube)},
        _direction{direction} {}
  const std::unique_ptr<Cube>& cube() const { return _cube; }
  Axis::Direction direction() const { return _direction; }
  const std::vector<Real>& time() const { return _time; }
  const std::vector<Real>& data() const { return _data; }
  void output() const;

 private:
  friend class Simulation;
  std::unique_ptr<Cube> _cube;
  Axis::Direction _direction;
  std::vector<Real> _time, _data;
  int _probe = -1;
};

/// Current through the cube's face normal to `direction`, every step: the
/// loop integral of H around it on the last node plane along the direction
/// (src/monitor/current_monitor.cpp:17-379).  time() = H times; output() as
/// for VoltageMonitor.
class CurrentMonitor : public Monitor {
 public:
  CurrentMonitor(std::string name, std::unique_ptr<Cube> cube, Axis::Direction direction,
                 std::string output_dir = "")
      : Monitor{std::move(name), std::move(output_dir)},
        _cube{std::move(cube)},
        _direction{direction} {}
  const std::unique_ptr<Cube>& cube() const { return _cube; }
  Axis::Direction direction() const { return _direction; }
  const std::vector<Real>& time() const { return _time; }
  const std::vector<Real>& data() const { return _data; }
  void output() const;

 private:
  friend class Simulation;
  std::unique_ptr<Cube> _cube;
  Axis::Direction _direction;
  std::vector<Real> _time, _data;
  int _probe = -1;
};

// ---------------------------------------------------------------- network
/// One port of a Network (include/xfdtd/network/port.h:15-70,
/// src/network/port.cpp:10-130): a current and a voltage monitor and a
/// reference impedance z.  calculateSParameters takes the DFTs
/// I(f) = dt sum_n i_n exp(-j 2 pi f ((n+1) dt - 1.5 dt)) and
/// V(f) = dt sum_n v_n exp(-j 2 pi f (n+1) dt) of the two series and forms the
/// power waves a = (V + z I) / (2 sqrt(Re z)), b = (V - conj(z) I) / (2 sqrt(Re z)).
class Port {
 public:
  Port(std::size_t index, bool is_source, std::complex<Real> impedance,
       std::shared_ptr<CurrentMonitor> current_monitor,
       std::shared_ptr<VoltageMonitor> voltage_monitor)
      : _index{index},
        _is_source{is_source},
        _impedance{impedance},
        _current_monitor{std::move(current_monitor)},
        _voltage_monitor{std::move(voltage_monitor)} {}
  std::size_t index() const { return _index; }
  bool isSource() const { return _is_source; }
  std::complex<Real> impedance() const { return _impedance; }
  const std::shared_ptr<CurrentMonitor>& currentMonitor() const { return _current_monitor; }
  const std::shared_ptr<VoltageMonitor>& voltageMonitor() const { return _voltage_monitor; }
  const std::vector<std::complex<Real>>& a() const { return _a; }
  const std::vector<std::complex<Real>>& b() const { return _b; }
  void init(Real dt) { _dt = dt; }
  void calculateSParameters(const Array1D<Real>& frequencies);

 private:
  std::size_t _index;
  bool _is_source;
  std::complex<Real> _impedance;
  std::shared_ptr<CurrentMonitor> _current_monitor;
  std::shared_ptr<VoltageMonitor> _voltage_monitor;
  Real _dt = 0;
  std::vector<std::complex<Real>> _a, _b;
};

/// S-parameters of a set of ports (include/xfdtd/network/network.h:21-70,
/// src/network/network.cpp:12-84).  output() computes every port's waves and
/// S[10 j + i] = b_j / a_i for each source port i, and writes
/// <output_dir>/s<10 j + i>.npy (complex128) and frequencies.npy.
class Network {
 public:
  Network() = default;
  explicit Network(std::string output_dir) : _output_dir{std::move(output_dir)} {}
  Network(std::vector<std::shared_ptr<Port>> ports, Array1D<Real> frequencies,
          std::string output_dir)
      : _ports{std::move(ports)},
        _frequencies{std::move(frequencies)},
        _output_dir{std::move(output_dir)} {}
  void addPort(std::shared_ptr<Port> port) { _ports.emplace_back(std::move(port)); }
  void setFrequencies(Array1D<Real> frequencies) { _frequencies = std::move(frequencies); }
  void setOutputDir(std::string output_dir) { _output_dir = std::move(output_dir); }
  /// Port::init for every port; port indices must be unique.
  void init(Real dt);
  /// The waves of every port and the S-parameters, without writing files.
  void compute();
  /// compute(), then the .npy files.
  void output();
  const std::vector<std::shared_ptr<Port>>& ports() const { return _ports; }
  const Array1D<Real>& frequencies() const { return _frequencies; }
  const std::map<int, std::vector<std::complex<Real>>>& sParameters() const {
    return _s_parameters;
  }

 private:
  std::vector<std::shared_ptr<Port>> _ports;
  Array1D<Real> _frequencies;
  std::string _output_dir;
  std::map<int, std::vector<std::complex<Real>>> _s_parameters;
};

// ------------------------------------------------------------------ NF2FF
/// Frequency-domain NF2FF on a Huygens box `distance` cells inside the grid
/// faces (src/nffft/nffft_frequency_domain.cpp).  After run() the surface
/// currents are available per frequency and face.
class NFFFTFrequencyDomain {
 public:
  NFFFTFrequencyDomain(Index dx, Index dy, Index dz, Array1D<Real> freqs,
                       std::string output_dir = "")
      : _d{dx, dy, dz}, _freqs{std::move(freqs)}, _output_dir{std::move(output_dir)} {}
  std::array<Index, 3> distance() const { return _d; }
  const Array1D<Real>& frequencies() const { return _freqs; }
  const std::string& outputDir() const { return _output_dir; }
  void setOutputDir(std::string d) { _output_dir = std::move(d); }
  /// J/M accumulators laid out [freq][face XN..ZP][ja jb ma mb][face nodes].
  const std::vector<std::complex<Real>>& surfaceCurrents() const { return _acc; }
  std::vector<std::complex<Real>>& surfaceCurrentsMutable() { return _acc; }
  /// Face node boxes [s, e) in global indices (empty when invalid).
  std::array<std::array<int, 6>, 6> faces{};

  /// Far-field potentials of the surface currents, computed on the GPU:
  /// laid out [frequency][a_theta, f_phi, a_phi, f_theta][angle] over the
  /// angles theta x phi, one of which must hold a single value
  /// (FDPlaneData::getPotential, src/nffft/nffft_fd_data_process.cpp:15-144).
  /// Needs the simulation that ran this NF2FF to be alive.
  std::vector<std::complex<Real>> farField(const Array1D<Real>& theta, const Array1D<Real>& phi,
                                           const Vector& origin = Vector{0, 0, 0}) const;
  /// processFarField (nffft_frequency_domain.h:35-62): writes, per
  /// frequency, <outputDir>/<sub_dir>/<f in GHz, 2 decimals>GHz_{a_theta,
  /// f_phi,a_phi,f_theta}.npy (complex128, one value per angle).
  void processFarField(const Array1D<Real>& theta, Real phi, const std::string& sub_dir,
                       const Vector& origin = Vector{0, 0, 0}) const;
  void processFarField(Real theta, const Array1D<Real>& phi, const std::string& sub_dir,
                       const Vector& origin = Vector{0, 0, 0}) const;
  void processFarField(const Array1D<Real>& theta, const Array1D<Real>& phi,
                       const std::string& sub_dir, const Vector& origin) const;
  /// Radiated power per frequency, 0.5 Re sum over the faces of
  /// (+-) sum ds (conj(J_a) M_b - conj(J_b) M_a) (FDPlaneData::power and
  /// calculatePower, src/nffft/nffft_fd_data_process.cpp:38-190).
  std::vector<Real> radiationPower() const;
  /// Writes <outputDir>/power.npy: the 2 x n_freq stack of the frequencies and
  /// radiationPower() (NFFFTFrequencyDomain::outputRadiationPower,
  /// src/nffft/nffft_frequency_domain.cpp:67-100).
  void outputRadiationPower() const;

 private:
  friend class Simulation;
  std::array<Index, 3> _d;
  Array1D<Real> _freqs;
  std::string _output_dir;
  std::vector<std::complex<Real>> _acc;
  xfd_engine* _engine = nullptr;  // set while the owning Simulation lives
  std::array<std::vector<Real>, 3> _node_e, _node_h, _size_e;  // grid, per axis
};

/// Time-domain near-to-far-field transform for one observation direction
/// (include/xfdtd/nffft/nffft_time_domain.h:23-86): the Huygens box `distance`
/// cells inside the domain, retarded-time potentials accumulated on the GPU
/// every step (xfd_set_nf2ff_td).
class NFFFTTimeDomain {
 public:
  NFFFTTimeDomain(Index dx, Index dy, Index dz, Real theta, Real phi)
      : _d{dx, dy, dz}, _theta{theta}, _phi{phi} {}
  NFFFTTimeDomain(Index dx, Index dy, Index dz, std::string_view output_dir, Real theta,
                  Real phi)
      : _d{dx, dy, dz}, _output_dir{output_dir}, _theta{theta}, _phi{phi} {}
  std::array<Index, 3> distance() const { return _d; }
  const std::string& outputDir() const { return _output_dir; }
  void setOutputDir(std::string d) { _output_dir = std::move(d); }
  Real theta() const { return _theta; }
  Real phi() const { return _phi; }
  /// (sin theta cos phi, sin theta sin phi, cos theta)
  Vector observationDirection() const;
  /// Potentials over the retarded-time bins, divided by (c dt 4 pi)
  /// (NFFFTTimeDomain::wx..uz, src/nffft/nfffft_time_domain.cpp:481-509).
  Array1D<Real> wx() const { return scaled(0); }
  Array1D<Real> wy() const { return scaled(1); }
  Array1D<Real> wz() const { return scaled(2); }
  Array1D<Real> ux() const { return scaled(3); }
  Array1D<Real> uy() const { return scaled(4); }
  Array1D<Real> uz() const { return scaled(5); }
  /// Writes w_theta.npy, w_phi.npy, u_theta.npy, u_phi.npy (float64, one
  /// value per bin) into outputDir() (NFFFTTimeDomain::processFarField,
  /// src/nffft/nfffft_time_domain.cpp:98-160).
  void processFarField() const;
  /// The four far-field series of processFarField, in that order.
  std::array<std::vector<Real>, 4> farField() const;

 private:
  friend class Simulation;
  Array1D<Real> scaled(int q) const;
  std::array<Index, 3> _d;
  std::string _output_dir;
  Real _theta, _phi;
  std::vector<Real> _raw;  // 6 x n_bins sums: W_x W_y W_z U_x U_y U_z
  Real _c_dt = 0;
};

/// The time axis of a run (include/xfdtd/calculation_param/time_param.h,
/// src/calculation_param/time_param.cpp): dt, the number of steps, the
/// first step, and the E / H sample times of every step.
class TimeParam {
 public:
  /// cfl / (c sqrt(1/dx^2 + 1/dy^2 + 1/dz^2)), and its 2-D and 1-D forms.
  static Real calculateDt(Real cfl, Real dx, Real dy, Real dz) {
    return cfl / (constant::C_0 * std::sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz)));
  }
  static Real calculateDt(Real cfl, Real dx, Real dy) {
    return cfl / (constant::C_0 * std::sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy)));
  }
  static Real calculateDt(Real cfl, Real dz) {
    return cfl / (constant::C_0 * std::sqrt(1.0 / (dz * dz)));
  }
  TimeParam(Real dt, std::size_t size, std::size_t start_time_step = 0)
      : _dt{dt}, _start{start_time_step}, _size{size}, _current{start_time_step} {}
  Real dt() const { return _dt; }
  std::size_t startTimeStep() const { return _start; }
  std::size_t size() const { return _size; }
  std::size_t endTimeStep() const { return _start + _size; }
  std::size_t currentTimeStep() const { return _current; }
  std::size_t remainingTimeStep() const { return _start + _size - _current; }
  void nextStep() { ++_current; }
  void setCurrentTimeStep(std::size_t t) { _current = t; }
  void setDt(Real dt) { _dt = dt; }
  /// linspace((start + 1) dt, (start + size) dt, size)
  Array1D<Real> eTime() const {
    return xt::linspace<Real>((_start + 1) * _dt, (_start + _size) * _dt, _size);
  }
  /// linspace((start + 0.5) dt, (start + size + 0.5) dt, size)
  Array1D<Real> hTime() const {
    return xt::linspace<Real>((_start + 0.5) * _dt, (_start + _size + 0.5) * _dt, _size);
  }

 private:
  Real _dt;
  std::size_t _start, _size, _current;
};

/// The parameters of a run the reference's objects read
/// (include/xfdtd/calculation_param/calculation_param.h:26-60): here the
/// time axis.  The update coefficients live on the GPU as a class table
/// (Simulation::coefficientArrays gives the reference's 18 arrays).
class CalculationParam {
 public:
  explicit CalculationParam(std::unique_ptr<TimeParam> time_param)
      : _time_param{std::move(time_param)} {}
  const std::unique_ptr<TimeParam>& timeParam() const { return _time_param; }
  std::unique_ptr<TimeParam>& timeParam() { return _time_param; }

 private:
  std::unique_ptr<TimeParam> _time_param;
};

class ThreadConfig {
 public:
  ThreadConfig(std::size_t x = 1, std::size_t y = 1, std::size_t z = 1) : _n{x, y, z} {}

 private:
  std::array<std::size_t, 3> _n;
};

/// MPI decomposition of the reference (include/xfdtd/parallel/mpi_support.h).
/// This library runs one simulation on one GPU and does not use MPI: the calls
/// reference programs make are kept and behave as on a single rank.
class MpiSupport {
 public:
  /// False: this library is not built with MPI (the reference's answer when
  /// it is compiled without it, mpi_support.h:27-30).
  static bool init(int /*argc*/ = 0, char** /*argv*/ = nullptr) { return false; }
  static bool setMpiParallelDim(int /*nx*/, int /*ny*/, int /*nz*/) { return true; }
  static int globalRank() { return 0; }
  static int globalSize() { return 1; }
  static MpiSupport& instance(int /*argc*/ = 0, char** /*argv*/ = nullptr) {
    static MpiSupport s;
    return s;
  }
  bool isRoot() const { return true; }
  int rank() const { return 0; }
  int size() const { return 1; }
  void barrier() const {}
  /// Ends the process with the code, as MPI_Abort does for one rank.
  [[noreturn]] void abort(int error_code) const { std::exit(error_code); }
};

// ------------------------------------------------------- flag visitors
/// include/xfdtd/simulation/simulation_flag.h:8-31.
enum class SimulationInitFlag { SimulationStart, SimulationEnd, InitStart, InitEnd, UpdateStart, UpdateEnd };
enum class SimulationIteratorFlag { UpdateHSStart, UpdateHSEnd, UpdateEStart, UpdateEEnd, NextStep };

class SimulationFlagVisitor {
 public:
  virtual ~SimulationFlagVisitor() = default;
  virtual void initStep(SimulationInitFlag flag) = 0;
  virtual void iteratorStep(SimulationIteratorFlag flag, Index cur, Index start, Index end) = 0;
};

/// Prints the phases and their elapsed times to stderr, and the progress of
/// the time loop (the reference's DefaultSimulationFlagVisitor,
/// src/simulation/simulation.cpp:157-280).
class DefaultSimulationFlagVisitor : public SimulationFlagVisitor {
 public:
  void initStep(SimulationInitFlag flag) override;
  void iteratorStep(SimulationIteratorFlag flag, Index cur, Index start, Index end) override;

 private:
  double _t_init = 0, _t_update = 0;
  Index _last_percent = 101;
};

enum class Precision { FP64 = 0, FP32 = 1 };

// ------------------------------------------------------------- Simulation
class Simulation {
 public:
  /// Simulation(dx, dy, dz, cfl, thread_config) -- thread_config is accepted
  /// and ignored: the time loop runs on the GPU.
  Simulation(Real dx, Real dy, Real dz, Real cfl, ThreadConfig thread_config = {1, 1, 1});
  ~Simulation();
  Simulation(const Simulation&) = delete;
  Simulation& operator=(const Simulation&) = delete;

  void addObject(std::shared_ptr<Object> object);
  void addBoundary(std::shared_ptr<Boundary> boundary);
  void addWaveformSource(std::shared_ptr<WaveformSource> source);
  void addMonitor(std::shared_ptr<Monitor> monitor);
  void addNF2FF(std::shared_ptr<NFFFTFrequencyDomain> nffft);
  void addNF2FF(std::shared_ptr<NFFFTTimeDomain> nffft);
  void addNetwork(std::shared_ptr<Network> network);
  /// Flag visitors (include/xfdtd/simulation/simulation.h:66-68): told
  /// SimulationStart / InitStart / InitEnd / UpdateStart / UpdateEnd /
  /// SimulationEnd, and NextStep (with the current, first and last step) at
  /// the end of every chunk of steps the engine runs as one graph (32 steps
  /// unless the "graph_chunk" option says otherwise) rather than every step.
  void addVisitor(std::shared_ptr<SimulationFlagVisitor> visitor);
  void addDefaultVisitor();

  /// One process, one GPU: always the root, rank 0 of 1.
  bool isRoot() const { return true; }
  int myRank() const { return 0; }
  int numNode() const { return 1; }
  int numThread() const { return 1; }

  /// Builds the grid and coefficients, runs `time_step` steps on the GPU and
  /// copies fields, movie frames and NF2FF currents back to the host.
  void run(Index time_step);

  /// Set-up only (grid, coefficients, engine upload) for `time_step` steps;
  /// run() calls it.  Exposed so that a caller can time the steps alone.
  void init(Index time_step);
  /// Advances `n` steps of an initialised simulation (asynchronous).
  void advance(Index n);
  /// Waits for the GPU and copies the outputs back (what run() does last).
  void finish();

  void setPrecision(Precision p) { _precision = p; }
  /// With false, init() stops after the host set-up (grid, classes, curl
  /// factors, CPML, ADE) and creates no engine: for checking the set-up
  /// arithmetic on a machine without a GPU.
  void setEngineEnabled(bool on) { _use_engine = on; }
  /// Engine option (xfd_set_option: "graph", "graph_chunk", "kernel",
  /// "ichunk"), applied when the engine is created, or at once if it exists.
  void setEngineOption(const std::string& name, long long value);
  Precision precision() const { return _precision; }

  const EMF& emf() const { return _emf; }
  Real dt() const { return _dt; }
  /// The run's time axis once init() or run() has set it up (null before):
  /// dt, the step count and the current step, which advances with the run.
  const std::shared_ptr<CalculationParam>& calculationParam() const { return _calc; }
  std::array<Index, 3> gridSize() const { return {_n[0], _n[1], _n[2]}; }
  xfd_engine* engine() const { return _engine; }

  /// The 18 Yee coefficient arrays as the engine applies them (class table x
  /// curl factors), in the reference shapes; order cexe cexhy cexhz ceye
  /// ceyhz ceyhx ceze cezhx cezhy chxh chxey chxez chyh chyez chyex chzh
  /// chzex chzey.  For checking the set-up against the reference's formulas.
  std::vector<std::vector<Real>> coefficientArrays() const;

  /// The TFSF3D set-up handed to the engine: the 1-D incident grid for every
  /// step (e_inc: steps x aux, h_inc: steps x (aux-1)) and the projections.
  struct TfsfTables {
    int aux = 0;
    std::vector<Real> e_inc, h_inc, p_int[3], p_half[3];
  };
  TfsfTables tfsfTables() const;

  /// Objective J = sum_p |F_p|^2 over the E_field nodes p of the node box
  /// [box_s, box_e), F_p = dt sum_n E^n(p) exp(-i 2 pi freq t_n) over the
  /// next n_steps steps (t_n = n dt, E^n the field after step n).  With
  /// `grad`, also dJ/deps_r of every voxel of the VoxelObject `voxel_object`
  /// (its index among the simulation's VoxelObjects), by the discrete
  /// adjoint (xfd_adjoint_run) with the forward state saved every
  /// `checkpoint_interval` steps; grad is resized to the voxel count (C
  /// order).  Advances the simulation n_steps either way.
  /// No counterpart in the reference (no gradient path).
  Real dftPowerObjective(Index n_steps, int field, const std::array<int, 3>& box_s,
                         const std::array<int, 3>& box_e, Real freq,
                         std::vector<Real>* grad = nullptr, int voxel_object = 0,
                         Index checkpoint_interval = 250);

  struct Impl;

 private:
  void setupTfsf(xfd_engine* e);
  void setupNf2ff(xfd_engine* e);
  void setupNf2ffTd(xfd_engine* e);
  void voltageProbe(const VoltageMonitor& m, std::vector<int32_t>& comp, std::vector<int32_t>& node,
                    std::vector<double>& w) const;
  void currentProbe(const CurrentMonitor& m, std::vector<int32_t>& comp, std::vector<int32_t>& node,
                    std::vector<double>& w) const;

  Real _dl[3];
  Real _cfl;
  Precision _precision = Precision::FP64;
  bool _use_engine = true;
  std::vector<std::pair<std::string, long long>> _engine_options;
  std::vector<std::shared_ptr<Object>> _objects;
  std::vector<std::shared_ptr<Boundary>> _boundaries;
  std::vector<std::shared_ptr<WaveformSource>> _sources;
  std::vector<std::shared_ptr<Monitor>> _monitors;
  std::vector<std::shared_ptr<NFFFTFrequencyDomain>> _nffts;
  std::vector<std::shared_ptr<NFFFTTimeDomain>> _nffts_td;
  std::vector<std::shared_ptr<Network>> _networks;
  std::vector<std::shared_ptr<SimulationFlagVisitor>> _visitors;
  long long _chunk = 32;  // steps per visitor NextStep (the engine's graph chunk)
  std::shared_ptr<CalculationParam> _calc;
  EMF _emf;
  Real _dt = 0;
  Index _n[3] = {0, 0, 0};
  Index _steps = 0;
  xfd_engine* _engine = nullptr;
  std::unique_ptr<Impl> _impl;
};

}  // namespace xfdtd
