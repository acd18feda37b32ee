// ORACLE -- test infrastructure only.
//
// CPU restatement of libBEEP's BEM matvec path, used by tests/, by the
// smoke check and by bench.py's CPU-baseline leg as the checker and as the
// timed CPU reference.  It is never part of the product: the beep3_b200
// package neither imports nor links it.
//
// Restated functions (reference file:line):
//   near_pair<T>       evaluate_local_BEM_kernels<T>   src/bem/bem_kernels.h:134-251
//   singular<T>        singular_BEM_kernels<T>         src/bem/bem_kernels.h:18-132
//   fGC / hGC          fGeometricCorrection etc.       src/bem/bem_kernels.cpp:123-136
//   precalc            BEEP::precalc_neighbour_interactions  src/beep/beep.cpp:768-956
//                      (singular diagonal + cached LocalIntegrations per leaf)
//   nf_apply           BEEP::evaluate_local_neighbours / evaluate_local_contributions
//                      src/beep/beep.cpp:1049-1062, src/bem/local_integrations.h:123-130
//   gmres              BEEP::gmres                     src/beep/beep.cpp:1262-1483
//   rhs                BEEP::set_rhs (direct sum)      src/beep/beep.cpp:1124-1260
//   energy_coef        Mesh::init_energy_precalcs (+ renormalise) src/bem/mesh.cpp:730-925
// The far field (FMM) lives in fmm_oracle.cpp.
//
// Precision: "ref" mode (fp32 = 1) mirrors the reference CPU build: quad
// points stored as float (QuadPointT<float>, src/bem/quad_point.h:231), the
// near-field kernel instantiated with float and cached as float
// (src/bem/local_integrations.h:17-25, :107), the singular kernel in float
// (src/beep/beep.cpp:836-840).  "exact" mode (fp32 = 0) does the same in
// FP64.  Sums are applied in FP64 in both modes.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

constexpr double ONE_OVER_4PI = 1.0 / (4.0 * M_PI);

template <typename T>
struct Pt {
  T x, y, z, nx, ny, nz, w;
};

template <typename T>
std::vector<Pt<T>> points(const double* p, int count) {
  std::vector<Pt<T>> out(count);
  for (int k = 0; k < count; ++k)
    out[k] = {(T)p[7 * k], (T)p[7 * k + 1], (T)p[7 * k + 2], (T)p[7 * k + 3], (T)p[7 * k + 4], (T)p[7 * k + 5],
              (T)p[7 * k + 6]};
  return out;
}

// One collocation/quadrature point pair, literally as in the reference loop
// body (gd, ud vectors; gdd, udd 3x3 matrices).
template <typename T, typename K>
inline void kernel_terms(const Pt<T>& s, const Pt<T>& q, K kappa, T inv_eps, T& A, T& B, T& C, T& D) {
  const T sigm = (T)1e-9;
  T wt = q.w;
  T dx[3] = {q.x - s.x, q.y - s.y, q.z - s.z};
  T nrm[3] = {q.nx, q.ny, q.nz};
  T n0[3] = {s.nx, s.ny, s.nz};
  T r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
  if (std::fabs(r2) < sigm) return;
  T r = std::sqrt(r2);
  T ir2 = (T)(1.0 / r2);
  T ir = (T)(1.0 / r);
  T ir3 = ir2 * ir;
  T ir4 = ir2 * ir2;
  T ir5 = ir4 * ir;
  T gr0 = (T)ONE_OVER_4PI;
  T gr1 = gr0 * ir;
  T gr3 = gr0 * ir3;
  T ur0 = (T)(std::exp(-kappa * r) * ONE_OVER_4PI);
  T ur1 = ur0 * ir;
  T ur2 = ur0 * ir2;
  T ur3 = ur0 * ir3;
  T ur3ur2 = (T)(ur3 + kappa * ur2);
  T gd[3], ud[3];
  for (int k = 0; k < 3; ++k) {
    gd[k] = -dx[k] * gr3;
    ud[k] = -dx[k] * ur3ur2;
  }
  A += wt * (gr1 - ur1);
  T bb = 0, cc = 0;
  for (int k = 0; k < 3; ++k) {
    bb += nrm[k] * (inv_eps * gd[k] - ud[k]);
    cc += n0[k] * (gd[k] - ud[k] * inv_eps);
  }
  B += wt * bb;
  C += -wt * cc;
  if (kappa != 0) {
    T gr5 = gr0 * ir5;
    T ur4 = ur0 * ir4;
    T ur5 = ur0 * ir5;
    T pur4ur3 = (T)(kappa * (3.0 * ur4 + kappa * ur3) + 3.0 * ur5);
    T gdd[3][3], udd[3][3];
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) {
        T kron = (j == k) ? (T)1.0 : (T)0.0;
        T dxjk = dx[j] * dx[k];
        gdd[j][k] = (T)(3.0 * dxjk * gr5 - kron * gr3);
        udd[j][k] = dxjk * pur4ur3 - kron * ur3ur2;
      }
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) D -= wt * n0[k] * nrm[j] * (gdd[j][k] - udd[j][k]);
  }
}

// evaluate_local_BEM_kernels<T> (src/bem/bem_kernels.h:134-251)
template <typename T>
void near_pair(T kappa, const std::vector<Pt<T>>& qual, const std::vector<Pt<T>>& quad, double targ_eps, T out[4]) {
  T inv_eps = (T)(1.0 / targ_eps);
  T Ao = 0, Bo = 0, Co = 0, Do = 0;
  for (const auto& s : qual) {
    T A = 0, B = 0, C = 0, D = 0;
    for (const auto& q : quad) kernel_terms<T, T>(s, q, kappa, inv_eps, A, B, C, D);
    T qw = s.w;
    Ao += A * qw;
    Bo += B * qw;
    Co += C * qw;
    Do += D * qw;
  }
  Do *= inv_eps;
  out[0] = Ao;
  out[1] = Bo;
  out[2] = Co;
  out[3] = Do;
}

// singular_BEM_kernels<T>(double kappa, ...) (src/bem/bem_kernels.h:18-132)
template <typename T>
void singular(double kappa, const std::vector<Pt<T>>& g, double eps, T out[4]) {
  T inv_eps = (T)(1.0 / eps);
  T Ao = 0, Bo = 0, Co = 0, Do = 0, norm = 0;
  for (size_t a = 0; a < g.size(); ++a) {
    const auto& s = g[a];
    norm += s.w;
    T A = 0, B = 0, C = 0, D = 0;
    for (size_t b = 0; b < g.size(); ++b) kernel_terms<T, double>(s, g[b], kappa, inv_eps, A, B, C, D);
    T qw = s.w;
    Ao += A * qw;
    Bo += B * qw;
    Co += C * qw;
    Do += D * qw;
  }
  Ao /= norm;
  Bo /= norm;
  Co /= norm;
  Do *= inv_eps / norm;
  out[0] = Ao;
  out[1] = Bo;
  out[2] = Co;
  out[3] = Do;
}

double fGC(double gc, double eps) { return (1.0 - gc) + gc / eps; }
double hGC(double gc, double eps) { return gc + (1.0 - gc) / eps; }

}  // namespace

struct OrNear {
  int n = 0;
  // LocalIntegrations records: (src, targ, A, B, C, D); coefficient values
  // are float in ref mode, double in exact mode (both stored as double).
  std::vector<int32_t> src, targ;
  std::vector<double> coef;  // 4 per record
  // records [row_begin[i], row_end[i]) after the n diagonal records are
  // row i's: a patch is a row of exactly one leaf, whose block is row-major
  std::vector<int64_t> row_begin, row_end;
};

extern "C" {

void or_pair_coefficients(const OrPatches* P, int npairs, const int32_t* I, const int32_t* J, double kappa, int fp32,
                          double* out) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int k = 0; k < npairs; ++k) {
    int i = I[k], j = J[k];
    if (i == j) {
      for (int c = 0; c < 4; ++c) out[4 * k + c] = 0.0;
      continue;
    }
    int qs = P->qual_off[i], qe = P->qual_off[i + 1];
    int ps = P->quad_off[j], pe = P->quad_off[j + 1];
    if (fp32) {
      auto qual = points<float>(P->qual + 7 * (size_t)qs, qe - qs);
      auto quad = points<float>(P->quad + 7 * (size_t)ps, pe - ps);
      float o[4];
      near_pair<float>((float)kappa, qual, quad, P->eps[j], o);
      for (int c = 0; c < 4; ++c) out[4 * k + c] = o[c];
    } else {
      auto qual = points<double>(P->qual + 7 * (size_t)qs, qe - qs);
      auto quad = points<double>(P->quad + 7 * (size_t)ps, pe - ps);
      double o[4];
      near_pair<double>(kappa, qual, quad, P->eps[j], o);
      for (int c = 0; c < 4; ++c) out[4 * k + c] = o[c];
    }
  }
}

void or_singular(const OrPatches* P, double kappa, int fp32, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < P->n; ++i) {
    int gs = P->gal_off[i], ge = P->gal_off[i + 1];
    double o[4];
    if (fp32) {
      auto g = points<float>(P->gal + 7 * (size_t)gs, ge - gs);
      float f[4];
      singular<float>(kappa, g, P->eps[i], f);
      for (int c = 0; c < 4; ++c) o[c] = f[c];
      // LocalIntegrations::set stores float values (src/beep/beep.cpp:836-842)
      out[4 * i + 0] = (float)o[0];
      out[4 * i + 1] = (float)(o[1] + fGC(P->gc[i], P->eps[i]));
      out[4 * i + 2] = (float)(o[2] - hGC(P->gc[i], P->eps[i]));
      out[4 * i + 3] = (float)o[3];
    } else {
      auto g = points<double>(P->gal + 7 * (size_t)gs, ge - gs);
      singular<double>(kappa, g, P->eps[i], o);
      out[4 * i + 0] = o[0];
      out[4 * i + 1] = o[1] + fGC(P->gc[i], P->eps[i]);
      out[4 * i + 2] = o[2] - hGC(P->gc[i], P->eps[i]);
      out[4 * i + 3] = o[3];
    }
  }
}

// Cached near field over the leaves of a tree: for every leaf, rows = its
// contents, cols = contents of its existing neighbours in order 0..26
// (Octree::get_neighbourhood_contents, src/fmm/octree.h:618-650).
OrNear* or_near_create(const OrPatches* P, const OrTree* T, double kappa, int fp32) {
  auto nf = new OrNear();
  nf->n = P->n;
  // singular diagonal records first (src/beep/beep.cpp:780-843)
  std::vector<double> diag(4 * (size_t)P->n);
  or_singular(P, kappa, fp32, diag.data());
  for (int i = 0; i < P->n; ++i) {
    nf->src.push_back(i);
    nf->targ.push_back(i);
    for (int c = 0; c < 4; ++c) nf->coef.push_back(diag[4 * i + c]);
  }
  for (int k = 0; k < T->n_nodes; ++k) {
    const int32_t* info = T->info + 18 * (size_t)k;
    int flags = info[4], cstart = info[6], ccount = info[7];
    if (!(flags & 2) || ccount == 0) continue;
    std::vector<int32_t> cols;
    for (int nb = 0; nb < 27; ++nb) {
      int m = T->neighbours[27 * (size_t)k + nb];
      if (m < 0) continue;
      const int32_t* mi = T->info + 18 * (size_t)m;
      for (int c = 0; c < mi[7]; ++c) cols.push_back(T->contents[mi[6] + c]);
    }
    for (int r = 0; r < ccount; ++r) {
      int i = T->contents[cstart + r];
      nf->row_begin.resize(P->n, 0);
      nf->row_end.resize(P->n, 0);
      nf->row_begin[i] = (int64_t)nf->src.size();
      for (int32_t j : cols) {
        nf->src.push_back(i);
        nf->targ.push_back(j);
      }
      nf->row_end[i] = (int64_t)nf->src.size();
    }
  }
  nf->row_begin.resize(P->n, 0);
  nf->row_end.resize(P->n, 0);
  size_t total = nf->src.size() - P->n;
  nf->coef.resize(4 * nf->src.size());
  or_pair_coefficients(P, (int)total, nf->src.data() + P->n, nf->targ.data() + P->n, kappa, fp32,
                       nf->coef.data() + 4 * (size_t)P->n);
  return nf;
}

void or_near_destroy(OrNear* nf) { delete nf; }

int64_t or_near_count(const OrNear* nf) { return (int64_t)nf->src.size(); }

// y_f[src] += B f[targ] - A h[targ] ; y_h[src] += D f[targ] - C h[targ]
// (src/bem/local_integrations.h:123-130); y is overwritten.
//
// The reference streams its cached records serially (CACHE_GPU_RESULTS is
// defined in the CPU build, src/beep/beep.h:71, so evaluate_local_neighbours
// runs only the loop at src/beep/beep.cpp:1049-1062).  Here rows run in
// parallel, each row summing its diagonal record and then its block in the
// serial loop's order, so the result is the serial result bit for bit.
void or_near_apply(const OrNear* nf, const double* x, double* y) {
  const int n = nf->n;
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    const double* d = &nf->coef[4 * (size_t)i];
    double yf = d[1] * x[i] - d[0] * x[n + i];
    double yh = d[3] * x[i] - d[2] * x[n + i];
    for (int64_t k = nf->row_begin[i]; k < nf->row_end[i]; ++k) {
      const double* c = &nf->coef[4 * k];
      const int j = nf->targ[k];
      yf += c[1] * x[j] - c[0] * x[n + j];
      yh += c[3] * x[j] - c[2] * x[n + j];
    }
    y[i] = yf;
    y[n + i] = yh;
  }
}

// Coulomb potential and field of charges at points; per-point weights give
// the per-patch sums of BEEP::set_rhs (scale 1/(4 pi eps_solvent)) or of the
// energy precalcs (scale 1/(4 pi)).  out_a = sum w phi, out_b = sum w grad phi . n
void or_point_sums(int n_patches, const int32_t* off, const double* pts, const double* xyzq, int nc, double scale,
                   double* out_a, double* out_b) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n_patches; ++i) {
    double a = 0, b = 0;
    for (int p = off[i]; p < off[i + 1]; ++p) {
      const double* q = pts + 7 * (size_t)p;
      double phi = 0, g[3] = {0, 0, 0};
      for (int c = 0; c < nc; ++c) {
        double d[3] = {q[0] - xyzq[4 * c], q[1] - xyzq[4 * c + 1], q[2] - xyzq[4 * c + 2]};
        double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        if (d2 <= 2.220446049250313e-16) continue;
        double r = std::sqrt(d2);
        double pt = xyzq[4 * c + 3] / r;
        double ft = -pt / d2;
        phi += pt;
        for (int k = 0; k < 3; ++k) g[k] += ft * d[k];
      }
      a += q[6] * phi;
      b += q[6] * (g[0] * q[3] + g[1] * q[4] + g[2] * q[5]);
    }
    out_a[i] = a * scale;
    out_b[i] = b * scale;
  }
}

// GMRES exactly as BEEP::gmres (src/beep/beep.cpp:1262-1483), generic in the
// matvec; restart <= 0 gives the reference's single cycle.
int or_gmres(or_matvec_fn mv, void* user, int n2, const double* b, double* x, double tol, int max_iters, int restart,
             double* rel_resid) {
  const int m = (restart > 0 && restart < max_iters) ? restart : max_iters;
  std::vector<double> V((size_t)n2 * (m + 1)), U((size_t)m * (m + 1) / 2), r(n2), y(m + 1), c(m), s(m);
  auto near0 = [](double l) { return l == 0 ? 2.2250738585072014e-308 : l; };
  auto nrm2 = [&](const double* v) {
    double acc = 0;
    for (int i = 0; i < n2; ++i) acc += v[i] * v[i];
    return std::sqrt(acc);
  };
  const double nrm2b = nrm2(b);
  int total = 0;
  double last = 0;
  while (true) {
    std::fill(U.begin(), U.end(), 0.0);
    mv(user, x, r.data());
    for (int i = 0; i < n2; ++i) r[i] -= b[i];
    double beta = nrm2(r.data());
    for (int i = 0; i < n2; ++i) V[i] = r[i] / near0(beta);
    y[0] = beta;
    int j = 0, uij = 0;
    const int cycle = std::min(m, max_iters - total);
    do {
      int u0j = uij;
      double* vj = &V[(size_t)n2 * j];
      double* w = &V[(size_t)n2 * (j + 1)];
      mv(user, vj, w);
      for (int k = 0; k <= j; ++k) {
        double acc = 0;
        const double* vk = &V[(size_t)n2 * k];
        for (int i = 0; i < n2; ++i) acc += vk[i] * w[i];
        U[u0j + k] = acc;
      }
      for (int k = 0; k <= j; ++k) {
        const double* vk = &V[(size_t)n2 * k];
        const double uk = U[u0j + k];
        for (int i = 0; i < n2; ++i) w[i] -= vk[i] * uk;
      }
      double h = nrm2(w);
      for (int i = 0; i < n2; ++i) w[i] /= near0(h);
      for (int i = 0; i < j; ++i) {
        double tmp = c[i] * U[uij] - s[i] * U[uij + 1];
        U[uij + 1] = s[i] * U[uij] + c[i] * U[uij + 1];
        U[uij] = tmp;
        ++uij;
      }
      double rd = U[uij];
      double dd = std::sqrt(rd * rd + h * h);
      c[j] = rd / near0(dd);
      s[j] = -h / near0(dd);
      U[uij] = dd;
      ++uij;
      y[j + 1] = s[j] * y[j];
      y[j] = c[j] * y[j];
      ++j;
      last = std::fabs(y[j]);
    } while (j < cycle && last > tol * nrm2b);
    double su = 0, sy = 0;
    for (int k = 0; k < uij; ++k) su += std::fabs(U[k]);
    for (int k = 0; k < j; ++k) sy += std::fabs(y[k]);
    if (!(su == 0 && sy == 0)) {
      for (int i = j - 1; i >= 0; --i) {
        double t = y[i];
        for (int k = i + 1; k < j; ++k) t -= U[(size_t)k * (k + 1) / 2 + i] * y[k];
        y[i] = t / U[(size_t)i * (i + 1) / 2 + i];
      }
    }
    for (int k = 0; k < j; ++k) {
      const double* vk = &V[(size_t)n2 * k];
      for (int i = 0; i < n2; ++i) x[i] -= vk[i] * y[k];
    }
    total += j;
    if (last <= tol * nrm2b || total >= max_iters || restart <= 0) break;
  }
  if (rel_resid) *rel_resid = nrm2b > 0 ? last / nrm2b : 0.0;
  return total;
}

}  // extern "C"
