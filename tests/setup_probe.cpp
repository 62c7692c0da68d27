// Test wrapper of include/xfd_setup.h: C entry points for ctypes
// (tests/test_setup_helpers.py compiles it next to the test's temporary files).
#include "xfd_setup.h"

extern "C" int probe_build_classes(const int* n, const double* const* coef,
                                   const double* const* fe_in, const double* const* fh_in,
                                   double* table, long long table_cap, uint16_t* node_class,
                                   double* max_residual) {
  std::vector<double> fe[3], fh[3];
  for (int a = 0; a < 3; ++a) {
    fe[a].assign(fe_in[a], fe_in[a] + n[a] + 1);
    fh[a].assign(fh_in[a], fh_in[a] + n[a]);
  }
  std::vector<double> t;
  std::vector<uint16_t> nc;
  const int k = xfd_setup::buildClasses(n, coef, fe, fh, t, nc, max_residual);
  if ((long long)t.size() > table_cap) return -1;
  std::copy(t.begin(), t.end(), table);
  std::copy(nc.begin(), nc.end(), node_class);
  return k;
}

extern "C" void probe_curl_factors(const int* n, const double* const* h_size,
                                   const double* const* e_size, const double* const* kappa_e,
                                   const double* const* kappa_h, double* const* fe_out,
                                   double* const* fh_out) {
  std::vector<double> fe[3], fh[3];
  xfd_setup::buildCurlFactors(n, h_size, e_size, kappa_e, kappa_h, fe, fh);
  for (int a = 0; a < 3; ++a) {
    std::copy(fe[a].begin(), fe[a].end(), fe_out[a]);
    std::copy(fh[a].begin(), fh[a].end(), fh_out[a]);
  }
}
