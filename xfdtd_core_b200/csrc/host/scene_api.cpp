// Scene-file front end of the host library: parses the line format of
// xfdtd_core_b200.scene.Scene into the xfdtd:: API calls a reference user
// program makes, and exposes the Simulation through the C entry points of
// xfdtd_host.h.
#include <cmath>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "xfd_engine.h"
#include "xfdtd/xfdtd.h"
#include "xfdtd_host.h"

using namespace xfdtd;

namespace {

thread_local std::string g_err;

Axis::Direction parseDir(const std::string& s) {
  static const char* names[6] = {"XN", "XP", "YN", "YP", "ZN", "ZP"};
  for (int i = 0; i < 6; ++i)
    if (s == names[i]) return static_cast<Axis::Direction>(i);
  throw XFDTDException("bad direction '" + s + "'");
}

EMF::Field parseField(const std::string& s) {
  static const char* names[6] = {"EX", "EY", "EZ", "HX", "HY", "HZ"};
  for (int i = 0; i < 6; ++i)
    if (s == names[i]) return static_cast<EMF::Field>(i);
  throw XFDTDException("bad field '" + s + "'");
}

double num(std::istringstream& in) {
  std::string tok;
  if (!(in >> tok)) throw XFDTDException("unexpected end of line");
  char* end = nullptr;
  const double v = std::strtod(tok.c_str(), &end);
  if (end == tok.c_str() || *end != '\0') throw XFDTDException("bad number '" + tok + "'");
  return v;
}

std::unique_ptr<Waveform> parseWaveform(std::istringstream& in) {
  std::string kind;
  in >> kind;
  if (kind == "gaussian") {
    const double tau = num(in), t0 = num(in), amp = num(in);
    return Waveform::gaussian(tau, t0, amp);
  }
  if (kind == "cosgauss") {
    const double tau = num(in), t0 = num(in), f = num(in), amp = num(in);
    return Waveform::cosineModulatedGaussian(tau, t0, f, amp);
  }
  throw XFDTDException("bad waveform '" + kind + "'");
}

std::shared_ptr<Material> parseMaterial(std::istringstream& in, const std::string& name) {
  std::string kind;
  in >> kind;
  if (kind == "simple") {
    const double er = num(in), mr = num(in), se = num(in), sm = num(in);
    return std::make_shared<Material>(name, ElectroMagneticProperty{er, mr, se, sm});
  }
  const double eps_inf = num(in);
  const int P = static_cast<int>(num(in));
  if (kind == "drude" || kind == "debye") {
    std::vector<Real> x, y;
    for (int p = 0; p < P; ++p) {
      x.push_back(num(in));
      y.push_back(num(in));
    }
    if (kind == "drude")
      return DrudeMedium::makeDrudeMedium(name, eps_inf, Array1D<Real>(xt::adapt(x)), Array1D<Real>(xt::adapt(y)));
    return DebyeMedium::makeDebyeMedium(name, eps_inf, Array1D<Real>(xt::adapt(x)), Array1D<Real>(xt::adapt(y)));
  }
  if (kind == "mlorentz") {
    std::vector<Real> v[5];
    for (int p = 0; p < P; ++p)
      for (int q = 0; q < 5; ++q) v[q].push_back(num(in));
    return MLorentzMaterial::makeMLorentz(name, eps_inf, Array1D<Real>(xt::adapt(v[0])), Array1D<Real>(xt::adapt(v[1])),
                                          Array1D<Real>(xt::adapt(v[2])), Array1D<Real>(xt::adapt(v[3])),
                                          Array1D<Real>(xt::adapt(v[4])));
  }
  throw XFDTDException("bad material '" + kind + "'");
}

void writeNpy(const std::string& path, const std::vector<double>& data,
              const std::vector<std::size_t>& shape) {
  std::ostringstream hdr;
  hdr << "{'descr': '<f8', 'fortran_order': False, 'shape': (";
  for (std::size_t i = 0; i < shape.size(); ++i) hdr << shape[i] << (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
  hdr << "), }";
  std::string h = hdr.str();
  const std::size_t total = 10 + h.size() + 1;
  h.append((64 - total % 64) % 64, ' ');
  h.push_back('\n');
  std::ofstream f(path, std::ios::binary);
  if (!f) throw XFDTDException("cannot write " + path);
  const char magic[] = "\x93NUMPY\x01\x00";
  f.write(magic, 8);
  const uint16_t len = static_cast<uint16_t>(h.size());
  f.write(reinterpret_cast<const char*>(&len), 2);
  f.write(h.data(), (std::streamsize)h.size());
  f.write(reinterpret_cast<const char*>(data.data()), (std::streamsize)(data.size() * 8));
}

}  // namespace

struct xfdtd_scene {
  std::unique_ptr<Simulation> sim;
  std::vector<std::shared_ptr<MovieMonitor>> movies;
  std::vector<std::shared_ptr<FieldTimeMonitor>> probes;
  std::vector<std::shared_ptr<VoltageMonitor>> voltages;
  std::vector<std::shared_ptr<CurrentMonitor>> currents;
  std::shared_ptr<NFFFTFrequencyDomain> nf2ff;
  std::shared_ptr<NFFFTTimeDomain> nf2ff_td;
  std::shared_ptr<Network> network;
  int64_t steps = 0;
  bool finished = false;
};

static xfdtd_scene* buildScene(const char* path, int32_t precision) {
  std::ifstream f(path);
  if (!f) throw XFDTDException(std::string("cannot open scene file ") + path);
  auto sc = std::make_unique<xfdtd_scene>();
  std::string line;
  double dl[3] = {0, 0, 0}, cfl = 0;
  bool have_grid = false;
  std::vector<std::string> body;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream in(line);
    std::string kw;
    in >> kw;
    if (kw == "grid") {
      dl[0] = num(in);
      dl[1] = num(in);
      dl[2] = num(in);
      cfl = num(in);
      have_grid = true;
    } else if (kw == "steps") {
      sc->steps = static_cast<int64_t>(num(in));
    } else if (kw == "xfdtd-scene" || kw == "name") {
      continue;
    } else {
      body.push_back(line);
    }
  }
  if (!have_grid) throw XFDTDException("scene has no grid line");
  sc->sim = std::make_unique<Simulation>(dl[0], dl[1], dl[2], cfl, ThreadConfig{1, 1, 1});
  sc->sim->setPrecision((precision & 0xFF) == 1 ? Precision::FP32 : Precision::FP64);
  sc->sim->setEngineEnabled((precision & XFDTD_SCENE_NO_ENGINE) == 0);
  for (const auto& l : body) {
    std::istringstream in(l);
    std::string kw, name;
    in >> kw;
    if (kw == "object") {
      std::string shape;
      in >> name >> shape;
      std::unique_ptr<Shape> sh;
      if (shape == "cube") {
        const double ox = num(in), oy = num(in), oz = num(in), sx = num(in), sy = num(in),
                     sz = num(in);
        sh = std::make_unique<Cube>(Vector{ox, oy, oz}, Vector{sx, sy, sz});
      } else if (shape == "sphere") {
        const double cx = num(in), cy = num(in), cz = num(in), r = num(in);
        sh = std::make_unique<Sphere>(Vector{cx, cy, cz}, r);
      } else {
        throw XFDTDException("bad shape '" + shape + "'");
      }
      auto mat = parseMaterial(in, name);
      sc->sim->addObject(std::make_shared<Object>(name, std::move(sh), mat));
    } else if (kw == "thin_wire") {
      in >> name;
      const double cx = num(in), cy = num(in), cz = num(in), r = num(in), h = num(in);
      std::string ax;
      in >> ax;
      const Axis axis = ax == "X" ? Axis::XP : ax == "Y" ? Axis::YP : ax == "Z" ? Axis::ZP
                        : throw XFDTDException("bad thin-wire axis '" + ax + "'");
      sc->sim->addObject(std::make_shared<ThinWire>(
          name, std::make_unique<Cylinder>(Vector{cx, cy, cz}, r, h, axis)));
    } else if (kw == "voxels") {
      in >> name;
      const double ox = num(in), oy = num(in), oz = num(in), sx = num(in), sy = num(in),
                   sz = num(in);
      std::array<Index, 3> dims;
      for (int a = 0; a < 3; ++a) {
        const double v = num(in);
        if (v < 1) throw XFDTDException("bad voxel count");
        dims[a] = (Index)v;
      }
      const double mu_r = num(in), sigma_e = num(in);
      std::vector<Real> eps(dims[0] * dims[1] * dims[2]);
      for (auto& v : eps) v = num(in);
      sc->sim->addObject(std::make_shared<VoxelObject>(
          name, std::make_unique<Cube>(Vector{ox, oy, oz}, Vector{sx, sy, sz}), dims,
          std::move(eps), mu_r, sigma_e));
    } else if (kw == "voltage_monitor" || kw == "current_monitor") {
      in >> name;
      const double ox = num(in), oy = num(in), oz = num(in), sx = num(in), sy = num(in),
                   sz = num(in);
      std::string dir;
      in >> dir;
      auto cube = std::make_unique<Cube>(Vector{ox, oy, oz}, Vector{sx, sy, sz});
      if (kw == "voltage_monitor") {
        auto m = std::make_shared<VoltageMonitor>(name, std::move(cube), parseDir(dir));
        sc->voltages.push_back(m);
        sc->sim->addMonitor(m);
      } else {
        auto m = std::make_shared<CurrentMonitor>(name, std::move(cube), parseDir(dir));
        sc->currents.push_back(m);
        sc->sim->addMonitor(m);
      }
    } else if (kw == "current_source" || kw == "voltage_source") {
      in >> name;
      const double ox = num(in), oy = num(in), oz = num(in), sx = num(in), sy = num(in),
                   sz = num(in);
      std::string dir;
      in >> dir;
      const double r = num(in);
      auto w = parseWaveform(in);
      auto cube = std::make_unique<Cube>(Vector{ox, oy, oz}, Vector{sx, sy, sz});
      if (kw == "current_source")
        sc->sim->addObject(
            std::make_shared<CurrentSource>(name, std::move(cube), parseDir(dir), r, std::move(w)));
      else
        sc->sim->addObject(
            std::make_shared<VoltageSource>(name, std::move(cube), parseDir(dir), r, std::move(w)));
    } else if (kw == "network") {
      if (sc->network) throw XFDTDException("one network per scene");
      const auto nf = static_cast<std::size_t>(num(in));
      std::vector<Real> fr(nf);
      for (auto& v : fr) v = num(in);
      sc->network = std::make_shared<Network>(std::vector<std::shared_ptr<Port>>{},
                                              Array1D<Real>(xt::adapt(fr)), "");
      sc->sim->addNetwork(sc->network);
    } else if (kw == "port") {
      if (!sc->network) throw XFDTDException("port before network");
      const auto index = static_cast<std::size_t>(num(in));
      const bool src = num(in) != 0;
      const double zr = num(in), zi = num(in);
      std::string cname, vname;
      in >> cname >> vname;
      std::shared_ptr<CurrentMonitor> cm;
      std::shared_ptr<VoltageMonitor> vm;
      for (const auto& c : sc->currents)
        if (c->name() == cname) cm = c;
      for (const auto& v : sc->voltages)
        if (v->name() == vname) vm = v;
      if (!cm || !vm) throw XFDTDException("port monitors " + cname + " / " + vname + " not found");
      sc->network->addPort(std::make_shared<Port>(index, src, std::complex<Real>(zr, zi), cm, vm));
    } else if (kw == "pec_plane") {
      in >> name;
      const double ox = num(in), oy = num(in), oz = num(in), sx = num(in), sy = num(in),
                   sz = num(in);
      sc->sim->addObject(std::make_shared<PecPlane>(
          name, std::make_unique<Cube>(Vector{ox, oy, oz}, Vector{sx, sy, sz})));
    } else if (kw == "resistor" || kw == "capacitor" || kw == "inductor") {
      in >> name;
      const double ox = num(in), oy = num(in), oz = num(in), sx = num(in), sy = num(in),
                   sz = num(in);
      std::string axis;
      in >> axis;
      if (axis != "X" && axis != "Y" && axis != "Z") throw XFDTDException("bad axis " + axis);
      const auto xyz = static_cast<Axis::XYZ>(axis[0] - 'X');
      const double v = num(in);
      auto cube = std::make_unique<Cube>(Vector{ox, oy, oz}, Vector{sx, sy, sz});
      if (kw == "resistor")
        sc->sim->addObject(std::make_shared<Resistor>(name, std::move(cube), xyz, v));
      else if (kw == "capacitor")
        sc->sim->addObject(std::make_shared<Capacitor>(name, std::move(cube), xyz, v));
      else
        sc->sim->addObject(std::make_shared<Inductor>(name, std::move(cube), xyz, v));
    } else if (kw == "pml") {
      const int t = static_cast<int>(num(in));
      std::string dir;
      in >> dir;
      const int order = static_cast<int>(num(in));
      const double sr = num(in), amin = num(in), amax = num(in), kmax = num(in);
      sc->sim->addBoundary(std::make_shared<PML>(t, parseDir(dir), order, sr, amin, amax, kmax));
    } else if (kw == "tfsf3d") {
      const auto x = static_cast<std::size_t>(num(in)), y = static_cast<std::size_t>(num(in)),
                 z = static_cast<std::size_t>(num(in));
      const double th = num(in), ph = num(in), ps = num(in);
      sc->sim->addWaveformSource(std::make_shared<TFSF3D>(x, y, z, th, ph, ps, parseWaveform(in)));
    } else if (kw == "movie") {
      std::string field;
      in >> name >> field;
      const double ox = num(in), oy = num(in), oz = num(in), sx = num(in), sy = num(in),
                   sz = num(in);
      const auto interval = static_cast<std::size_t>(num(in));
      auto fm = std::make_unique<FieldMonitor>(
          std::make_unique<Cube>(Vector{ox, oy, oz}, Vector{sx, sy, sz}), parseField(field));
      // no output directory: the scene's frames are written by
      // xfdtd_scene_write_outputs under the directory it is given
      auto mv = std::make_shared<MovieMonitor>(std::move(fm), interval, name, "");
      sc->movies.push_back(mv);
      sc->sim->addMonitor(mv);
    } else if (kw == "field_time") {
      std::string field;
      in >> name >> field;
      const double ox = num(in), oy = num(in), oz = num(in), sx = num(in), sy = num(in),
                   sz = num(in);
      auto ft = std::make_shared<FieldTimeMonitor>(
          name, std::make_unique<Cube>(Vector{ox, oy, oz}, Vector{sx, sy, sz}), name,
          parseField(field));
      sc->probes.push_back(ft);
      sc->sim->addMonitor(ft);
    } else if (kw == "nf2ff_fd") {
      const auto dx = static_cast<Index>(num(in)), dy = static_cast<Index>(num(in)),
                 dz = static_cast<Index>(num(in));
      const int nf = static_cast<int>(num(in));
      std::vector<Real> fr;
      for (int q = 0; q < nf; ++q) fr.push_back(num(in));
      sc->nf2ff = std::make_shared<NFFFTFrequencyDomain>(dx, dy, dz, Array1D<Real>(xt::adapt(fr)));
      sc->sim->addNF2FF(sc->nf2ff);
    } else if (kw == "nf2ff_td") {
      const auto dx = static_cast<Index>(num(in)), dy = static_cast<Index>(num(in)),
                 dz = static_cast<Index>(num(in));
      const double theta = num(in), phi = num(in);
      sc->nf2ff_td = std::make_shared<NFFFTTimeDomain>(dx, dy, dz, theta, phi);
      sc->sim->addNF2FF(sc->nf2ff_td);
    } else {
      throw XFDTDException("unknown scene line: " + l);
    }
  }
  sc->sim->init(static_cast<Index>(sc->steps));
  return sc.release();
}

#define HOST_TRY(...)                   \
  try {                                 \
    __VA_ARGS__;                        \
    return 0;                           \
  } catch (const std::exception& ex) {  \
    g_err = ex.what();                  \
    return 1;                           \
  }

extern "C" {

int xfdtd_scene_open(const char* path, int32_t precision, xfdtd_scene** out) {
  HOST_TRY({
    if (!path || !out) throw XFDTDException("null argument");
    *out = buildScene(path, precision);
  })
}

void xfdtd_scene_close(xfdtd_scene* s) { delete s; }

const char* xfdtd_host_last_error(void) { return g_err.c_str(); }

struct xfd_engine* xfdtd_scene_engine(xfdtd_scene* s) { return s ? s->sim->engine() : nullptr; }

int xfdtd_scene_set_engine_option(xfdtd_scene* s, const char* name, int64_t value) {
  HOST_TRY({
    if (!s || !name) throw XFDTDException("null argument");
    s->sim->setEngineOption(name, (long long)value);
  });
}

int xfdtd_scene_info(xfdtd_scene* s, int32_t n[3], double* dt, int64_t* steps) {
  HOST_TRY({
    if (!s) throw XFDTDException("null scene");
    auto g = s->sim->gridSize();
    if (n)
      for (int a = 0; a < 3; ++a) n[a] = (int32_t)g[a];
    if (dt) *dt = s->sim->dt();
    if (steps) *steps = s->steps;
  })
}

int xfdtd_scene_advance(xfdtd_scene* s, int64_t n) {
  HOST_TRY({
    if (!s) throw XFDTDException("null scene");
    s->sim->advance(static_cast<Index>(n));
    s->finished = false;
  })
}

int xfdtd_scene_finish(xfdtd_scene* s) {
  HOST_TRY({
    if (!s) throw XFDTDException("null scene");
    s->sim->finish();
    s->finished = true;
  })
}

int xfdtd_scene_coefficients(xfdtd_scene* s, double* const out[18]) {
  HOST_TRY({
    if (!s || !out) throw XFDTDException("null argument");
    auto arrs = s->sim->coefficientArrays();
    for (int q = 0; q < 18; ++q) std::memcpy(out[q], arrs[q].data(), arrs[q].size() * 8);
  })
}

int xfdtd_scene_tfsf(xfdtd_scene* s, double* e_inc, double* h_inc, double* const p_int[3],
                     double* const p_half[3], int32_t* aux) {
  HOST_TRY({
    if (!s) throw XFDTDException("null scene");
    const auto t = s->sim->tfsfTables();
    if (aux) *aux = t.aux;
    if (e_inc) std::memcpy(e_inc, t.e_inc.data(), t.e_inc.size() * 8);
    if (h_inc) std::memcpy(h_inc, t.h_inc.data(), t.h_inc.size() * 8);
    for (int a = 0; a < 3; ++a) {
      if (p_int && p_int[a]) std::memcpy(p_int[a], t.p_int[a].data(), t.p_int[a].size() * 8);
      if (p_half && p_half[a]) std::memcpy(p_half[a], t.p_half[a].data(), t.p_half[a].size() * 8);
    }
  })
}

int xfdtd_scene_field(xfdtd_scene* s, int32_t comp, double* out) {
  HOST_TRY({
    if (!s || !out || comp < 0 || comp > 5) throw XFDTDException("bad argument");
    if (!s->finished) throw XFDTDException("call xfdtd_scene_finish first");
    const auto& a = s->sim->emf().field(static_cast<EMF::Field>(comp));
    std::memcpy(out, a.data(), a.size() * 8);
  })
}

int xfdtd_scene_movie(xfdtd_scene* s, int32_t index, double* out, int64_t capacity,
                      int64_t* n_frames, int32_t shape[3]) {
  HOST_TRY({
    if (!s || index < 0 || index >= (int32_t)s->movies.size())
      throw XFDTDException("bad movie index");
    if (!s->finished) throw XFDTDException("call xfdtd_scene_finish first");
    const auto& mv = s->movies[index];
    const auto& fr = mv->frames();
    const auto shp = mv->frameShape();
    if (n_frames) *n_frames = (int64_t)fr.size();
    if (shape)
      for (int a = 0; a < 3; ++a) shape[a] = (int32_t)shp[a];
    if (out) {
      const std::size_t per = shp[0] * shp[1] * shp[2];
      if ((std::size_t)capacity < per * fr.size()) throw XFDTDException("buffer too small");
      for (std::size_t q = 0; q < fr.size(); ++q) std::memcpy(out + q * per, fr[q].data(), per * 8);
    }
  })
}

int xfdtd_scene_field_time(xfdtd_scene* s, int32_t index, double* out, int64_t capacity,
                           int64_t* count) {
  HOST_TRY({
    if (!s || index < 0 || index >= (int32_t)s->probes.size())
      throw XFDTDException("bad field time monitor index");
    if (!s->finished) throw XFDTDException("call xfdtd_scene_finish first");
    const auto& p = s->probes[index];
    const std::size_t n = p->data().size();
    if (count) *count = (int64_t)n;
    if (out) {
      if ((std::size_t)capacity < 2 * n) throw XFDTDException("buffer too small");
      std::memcpy(out, p->time().data(), n * 8);
      std::memcpy(out + n, p->data().data(), n * 8);
    }
  })
}

int xfdtd_scene_nf2ff(xfdtd_scene* s, double* out, int64_t capacity, int64_t* count) {
  HOST_TRY({
    if (!s || !s->nf2ff) throw XFDTDException("scene has no NF2FF");
    if (!s->finished) throw XFDTDException("call xfdtd_scene_finish first");
    const auto& acc = s->nf2ff->surfaceCurrents();
    if (count) *count = (int64_t)acc.size();
    if (out) {
      if ((std::size_t)capacity < acc.size()) throw XFDTDException("buffer too small");
      for (std::size_t q = 0; q < acc.size(); ++q) {
        out[2 * q] = acc[q].real();
        out[2 * q + 1] = acc[q].imag();
      }
    }
  })
}

int xfdtd_scene_far_field(xfdtd_scene* s, int32_t n_theta, const double* theta, int32_t n_phi,
                          const double* phi, const double origin[3], double* out,
                          int64_t capacity, int64_t* count, const char* dir,
                          const char* sub_dir) {
  HOST_TRY({
    if (!s || !s->nf2ff) throw XFDTDException("scene has no NF2FF");
    if (!s->finished) throw XFDTDException("call xfdtd_scene_finish first");
    if (!theta || !phi || n_theta < 1 || n_phi < 1) throw XFDTDException("bad angles");
    Array1D<Real> th(xt::adapt(std::vector<Real>(theta, theta + n_theta)));
    Array1D<Real> ph(xt::adapt(std::vector<Real>(phi, phi + n_phi)));
    const Vector o = origin ? Vector{origin[0], origin[1], origin[2]} : Vector{0, 0, 0};
    const auto data = s->nf2ff->farField(th, ph, o);
    if (count) *count = (int64_t)data.size();
    if (out) {
      if ((std::size_t)capacity < data.size()) throw XFDTDException("buffer too small");
      for (std::size_t q = 0; q < data.size(); ++q) {
        out[2 * q] = data[q].real();
        out[2 * q + 1] = data[q].imag();
      }
    }
    if (sub_dir) {
      if (dir) s->nf2ff->setOutputDir(dir);
      s->nf2ff->processFarField(th, ph, sub_dir, o);
    }
  })
}

int xfdtd_scene_dft_objective(xfdtd_scene* s, int64_t n_steps, int32_t field,
                              const int32_t box_s[3], const int32_t box_e[3], double freq,
                              int32_t voxel_object, int32_t checkpoint_interval, double* value,
                              double* grad, int64_t capacity) {
  HOST_TRY({
    if (!s || !value || !box_s || !box_e) throw XFDTDException("null argument");
    const std::array<int, 3> bs{box_s[0], box_s[1], box_s[2]}, be{box_e[0], box_e[1], box_e[2]};
    if (!grad) {
      *value = s->sim->dftPowerObjective((Index)n_steps, field, bs, be, freq);
    } else {
      std::vector<Real> g;
      *value = s->sim->dftPowerObjective((Index)n_steps, field, bs, be, freq, &g, voxel_object,
                                         (Index)checkpoint_interval);
      if ((std::size_t)capacity < g.size()) throw XFDTDException("gradient buffer too small");
      std::copy(g.begin(), g.end(), grad);
    }
    s->finished = false;
  })
}

int xfdtd_scene_write_outputs(xfdtd_scene* s, const char* dir) {
  HOST_TRY({
    if (!s || !dir) throw XFDTDException("null argument");
    if (!s->finished) throw XFDTDException("call xfdtd_scene_finish first");
    namespace fs = std::filesystem;
    const fs::path root(dir);
    fs::create_directories(root / "fields");
    static const char* names[6] = {"EX", "EY", "EZ", "HX", "HY", "HZ"};
    for (int c = 0; c < 6; ++c) {
      const auto& a = s->sim->emf().field(static_cast<EMF::Field>(c));
      std::vector<double> v(a.data(), a.data() + a.size());
      writeNpy((root / "fields" / (std::string(names[c]) + ".npy")).string(), v,
               {a.shape()[0], a.shape()[1], a.shape()[2]});
    }
    for (const auto& mv : s->movies) {
      const fs::path d = root / mv->name();
      fs::create_directories(d);
      const auto shp = mv->frameShape();
      for (std::size_t q = 0; q < mv->frames().size(); ++q) {
        std::ostringstream nm;  // MovieMonitor::formatFrameCount: the step, 5 digits
        nm << std::setw(5) << std::setfill('0') << q * mv->frameInterval();
        writeNpy((d / (nm.str() + ".npy")).string(), mv->frames()[q], {shp[0], shp[1], shp[2]});
      }
    }
    for (const auto& p : s->probes) {  // TimeMonitor::output: [time; data]
      const fs::path d = root / p->name();
      fs::create_directories(d);
      std::vector<double> v(p->time().begin(), p->time().end());
      v.insert(v.end(), p->data().begin(), p->data().end());
      writeNpy((d / (p->name() + ".npy")).string(), v, {2, p->data().size()});
    }
    if (s->nf2ff) {
      const auto& acc = s->nf2ff->surfaceCurrents();
      std::vector<double> v;
      for (const auto& z : acc) {
        v.push_back(z.real());
        v.push_back(z.imag());
      }
      writeNpy((root / "nf2ff.npy").string(), v, {acc.size(), 2});
    }
    if (s->nf2ff_td) {
      s->nf2ff_td->setOutputDir((root / "nf2ff_td").string());
      s->nf2ff_td->processFarField();
    }
    for (const auto& m : s->voltages) {
      m->setOutputDir((root / "monitors").string());
      m->output();
    }
    for (const auto& m : s->currents) {
      m->setOutputDir((root / "monitors").string());
      m->output();
    }
    if (s->network) {
      s->network->setOutputDir((root / "network").string());
      s->network->output();
    }
  })
}

int xfdtd_scene_s_parameter(xfdtd_scene* s, int32_t key, double* out, int64_t capacity,
                            int64_t* count) {
  HOST_TRY({
    if (!s || !count) throw XFDTDException("null argument");
    if (!s->network) throw XFDTDException("scene has no network");
    if (!s->finished) throw XFDTDException("call xfdtd_scene_finish first");
    s->network->compute();
    const auto& m = s->network->sParameters();
    auto it = m.find(key);
    if (it == m.end()) throw XFDTDException("no S-parameter " + std::to_string(key));
    *count = (int64_t)(2 * it->second.size());
    if (out) {
      if (capacity < *count) throw XFDTDException("buffer too small");
      for (std::size_t q = 0; q < it->second.size(); ++q) {
        out[2 * q] = it->second[q].real();
        out[2 * q + 1] = it->second[q].imag();
      }
    }
  })
}

int xfdtd_scene_line_monitor(xfdtd_scene* s, int32_t kind, int32_t index, double* out,
                             int64_t capacity, int64_t* count) {
  HOST_TRY({
    if (!s || !count) throw XFDTDException("null argument");
    if (!s->finished) throw XFDTDException("call xfdtd_scene_finish first");
    const std::vector<Real>* t = nullptr;
    const std::vector<Real>* d = nullptr;
    if (kind == 0 && index >= 0 && index < (int32_t)s->voltages.size()) {
      t = &s->voltages[(std::size_t)index]->time();
      d = &s->voltages[(std::size_t)index]->data();
    } else if (kind == 1 && index >= 0 && index < (int32_t)s->currents.size()) {
      t = &s->currents[(std::size_t)index]->time();
      d = &s->currents[(std::size_t)index]->data();
    } else {
      throw XFDTDException("no such voltage/current monitor");
    }
    *count = (int64_t)(t->size() + d->size());
    if (out) {
      if (capacity < *count) throw XFDTDException("buffer too small");
      std::copy(t->begin(), t->end(), out);
      std::copy(d->begin(), d->end(), out + t->size());
    }
  })
}

int xfdtd_scene_nf2ff_td(xfdtd_scene* s, double* out, int64_t capacity, int64_t* count) {
  HOST_TRY({
    if (!s || !s->nf2ff_td) throw XFDTDException("scene has no time-domain NF2FF");
    if (!s->finished) throw XFDTDException("call xfdtd_scene_finish first");
    const auto ff = s->nf2ff_td->farField();
    const std::size_t n = ff[0].size();
    if (count) *count = (int64_t)(4 * n);
    if (out) {
      if ((std::size_t)capacity < 4 * n) throw XFDTDException("buffer too small");
      for (int q = 0; q < 4; ++q) std::copy(ff[q].begin(), ff[q].end(), out + q * n);
    }
  })
}

}  // extern "C"
