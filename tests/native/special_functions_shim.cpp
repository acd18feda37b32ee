// Test shim: compiles the engine's host FMM table source and the oracle's
// FMM restatement into one test library and exposes their special
// functions (scaled modified spherical Bessel i_n, associated Legendre
// functions) and the engine's generated interaction list through extern "C"
// wrappers, so the tests can compare them with scipy and with the
// reference's own code.  Built by tests/native/__init__.py; not part of the product.
#include "../../beep3_b200/csrc/fmm_tables.cpp"
#include "../../oracle/fmm_oracle.cpp"

#include <algorithm>

extern "C" {

// engine: b[n] = i_n(x) / scal^n, n = 0..nb
void shim_engine_bessel_in(double scal, double x, int nb, double* b) { bp::bessel_in(scal, x, nb, b); }

// engine: y[tri(n, m)] = scal^n P_n^m(x), x > 1
void shim_engine_legendre_gt1(int nmax, double scal, double x, double* y) {
  std::vector<double> v;
  bp::legendre_gt1(nmax, scal, x, v);
  std::copy(v.begin(), v.end(), y);
}

// engine: its generated interaction list, 7 ints per entry (child ids
// 0-based); returns the count
int shim_engine_interaction_list(int32_t* out) {
  const std::vector<bp::RawInteraction> l = bp::interaction_table();
  if (out)
    for (size_t k = 0; k < l.size(); ++k) {
      const int32_t v[7] = {l[k].nb, l[k].dir, l[k].targ, l[k].src, l[k].dx, l[k].dy, l[k].dz};
      for (int c = 0; c < 7; ++c) out[7 * k + c] = v[c];
    }
  return (int)l.size();
}

// oracle: the same i_n
void shim_oracle_i_n(double scal, double x, int nb, double* b) { i_n(scal, x, nb, b); }

// oracle: y[tri(n, m)] = P_n^m(x), |x| <= 1, Condon-Shortley phase
void shim_oracle_lgndr(int nmax, double x, double* y) {
  std::vector<double> v;
  lgndr(nmax, x, v);
  std::copy(v.begin(), v.end(), y);
}

// oracle: y[tri(n, m)] = scal^n P_n^m(x), x > 1
void shim_oracle_lgndrgt1(int nmax, double scal, double x, double* y) {
  std::vector<double> v;
  lgndrgt1(nmax, scal, x, v);
  std::copy(v.begin(), v.end(), y);
}
}
