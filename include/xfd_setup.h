/* Set-up helpers for handing a reference Simulation's coefficients to the
 * engine (include/xfd_engine.h), header-only C++17.
 *
 * The reference keeps 18 full-grid update-coefficient arrays
 * (FDTDUpdateCoefficient, include/xfdtd/calculation_param/fdtd_update_coefficient.h:102-121,
 * filled by CalculationParam::calculateCoefficient,
 * src/calculation_param/calculation_param.cpp:170-264, and patched by the
 * objects' correctUpdateCoefficient).  The engine takes a table of material
 * classes -- per class the (ca, cb) of Ex Ey Ez Hx Hy Hz -- a uint16 class per
 * lattice node, and per-axis curl factors:
 *   ceh_a(c) = -cb_c fe[b][x_b],  ceh_b(c) = cb_c fe[a][x_a]   (E_c, a = c+1, b = c+2)
 *   che_a(c) =  cb_c fh[b][x_b],  che_b(c) = -cb_c fh[a][x_a]  (H_c)
 * buildCurlFactors forms fe, fh from the grid's cell sizes and the CPML kappa;
 * buildClasses factors the 18 arrays into classes with those factors.  A
 * coefficient whose two curl terms the reference scales differently (a
 * ThinWire's H coefficients) is no single cb: buildClasses reports it in
 * `max_residual` and xfd_set_h_term_overrides carries the difference. */
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <unordered_map>
#include <vector>

namespace xfd_setup {

/* fe[a][x] = 1 / (h_size[a][x] kappa_e[a][x]) over the nodes x = 0..n[a],
 * fh[a][x] = 1 / (e_size[a][x] kappa_h[a][x]) over the cells x = 0..n[a]-1:
 * h_size / e_size are the reference GridSpace's hSize / eSize per axis
 * (src/grid_space/grid_space.cpp), kappa the CPML kappa of the E / H layers
 * (PML::_kappa_e / _kappa_h over the layers, 1 elsewhere; null: 1). */
inline void buildCurlFactors(const int n[3], const double* const h_size[3],
                             const double* const e_size[3], const double* const kappa_e[3],
                             const double* const kappa_h[3], std::vector<double> fe[3],
                             std::vector<double> fh[3]) {
  for (int a = 0; a < 3; ++a) {
    fe[a].assign((size_t)n[a] + 1, 0.0);
    fh[a].assign((size_t)n[a], 0.0);
    for (int x = 0; x <= n[a]; ++x)
      fe[a][(size_t)x] = 1.0 / (h_size[a][x] * (kappa_e && kappa_e[a] ? kappa_e[a][x] : 1.0));
    for (int x = 0; x < n[a]; ++x)
      fh[a][(size_t)x] = 1.0 / (e_size[a][x] * (kappa_h && kappa_h[a] ? kappa_h[a][x] : 1.0));
  }
}

namespace detail {
struct RowHash {
  size_t operator()(const std::array<double, 12>& r) const {
    uint64_t h = 1469598103934665603ULL;
    for (double v : r) {
      uint64_t b;
      std::memcpy(&b, &v, 8);
      h = (h ^ b) * 1099511628211ULL;
    }
    return (size_t)h;
  }
};
struct RowEq {
  bool operator()(const std::array<double, 12>& a, const std::array<double, 12>& b) const {
    return std::memcmp(a.data(), b.data(), sizeof(double) * 12) == 0;
  }
};
}  // namespace detail

/* coef[18]: the reference arrays in the order cexe cexhy cexhz ceye ceyhz
 * ceyhx ceze cezhx cezhy chxh chxey chxez chyh chyez chyex chzh chzex chzey,
 * each C-ordered in its reference shape (E_c: n[c] along c, n+1 across; H_c:
 * n+1 along c, n across).  Per lattice node (nx+1) x (ny+1) x (nz+1) the
 * class row holds, for each component whose array has the node, its (ca, cb)
 * with cb = ceh_b / fe[a][x_a] (E) or -che_b / fh[a][x_a] (H); zero where the
 * array does not reach.  Equal rows share a class (bitwise).  Returns the
 * class count (table gets 12 doubles per class, node_class one entry per
 * node, k fastest); throws std::runtime_error above 65535 classes.
 * max_residual (optional): the largest relative difference between a
 * reference coefficient and the class value times its curl factor over both
 * curl terms -- 0 up to rounding when every coefficient factors. */
inline int buildClasses(const int n[3], const double* const coef[18],
                        const std::vector<double> fe[3], const std::vector<double> fh[3],
                        std::vector<double>& table, std::vector<uint16_t>& node_class,
                        double* max_residual = nullptr) {
  const size_t NX = (size_t)n[0] + 1, NY = (size_t)n[1] + 1, NZ = (size_t)n[2] + 1;
  node_class.assign(NX * NY * NZ, 0);
  table.clear();
  std::unordered_map<std::array<double, 12>, uint16_t, detail::RowHash, detail::RowEq> ids;
  double worst = 0.0;
  for (size_t i = 0; i < NX; ++i)
    for (size_t j = 0; j < NY; ++j)
      for (size_t k = 0; k < NZ; ++k) {
        const size_t x[3] = {i, j, k};
        std::array<double, 12> row{};
        for (int h = 0; h < 2; ++h)
          for (int c = 0; c < 3; ++c) {
            size_t s[3];
            bool in = true;
            for (int d = 0; d < 3; ++d) {
              const bool along = d == c;
              s[d] = (size_t)n[d] + ((h == 0) == along ? 0 : 1);
              in = in && x[d] < s[d];
            }
            if (!in) continue;
            const size_t q = (x[0] * s[1] + x[1]) * s[2] + x[2];
            const int a = (c + 1) % 3, b = (c + 2) % 3;
            const double* base = coef[9 * h + 3 * c];
            const double ca = base[q];
            const double cha = coef[9 * h + 3 * c + 1][q], chb = coef[9 * h + 3 * c + 2][q];
            const std::vector<double>* f = h == 0 ? fe : fh;
            const double cb = h == 0 ? chb / f[a][x[a]] : -chb / f[a][x[a]];
            row[(size_t)(6 * h + 2 * c)] = ca;
            row[(size_t)(6 * h + 2 * c + 1)] = cb;
            // the other curl term, from the same cb
            const double other = h == 0 ? -cb * f[b][x[b]] : cb * f[b][x[b]];
            const double back = h == 0 ? cb * f[a][x[a]] : -cb * f[a][x[a]];
            const double scale = std::fmax(std::fabs(cha), std::fabs(chb));
            if (scale > 0) {
              worst = std::fmax(worst, std::fabs(other - cha) / scale);
              worst = std::fmax(worst, std::fabs(back - chb) / scale);
            }
          }
        auto it = ids.find(row);
        uint16_t id;
        if (it == ids.end()) {
          if (ids.size() >= 65535) throw std::runtime_error("more than 65535 material classes");
          id = (uint16_t)ids.size();
          ids.emplace(row, id);
          table.insert(table.end(), row.begin(), row.end());
        } else {
          id = it->second;
        }
        node_class[(i * NY + j) * NZ + k] = id;
      }
  if (max_residual) *max_residual = worst;
  return (int)ids.size();
}

}  // namespace xfd_setup
