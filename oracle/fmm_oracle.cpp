// ORACLE -- test infrastructure only.
//
// CPU restatement of libBEEP's 12-channel screened-Coulomb plane-wave FMM,
// the far field of the BEM matvec (FMM_BEM_Octree<NT, NL, ..>::solve,
// src/fmm/fmm_bem_hybrid.h:183-279), over a tree given as input.
//
// Restated functions (reference file:line):
//   get_scale                 src/fmm/fmm_globals.h:63-70
//   bnlcft, yhfstrtn, yhfrmini, yhrotgen   src/fmm/fmm_globals.h:72-368
//   level globals (quadrature tables, numphys adjustment, fexp*, rlsc,
//     xs/ys/zs, shift coefficients)        src/fmm/fmm_globals.h:372-1100
//   i_n (scaled modified spherical Bessel)   src/fmm/fmm_math_funcs.h:24-113
//     -- the reference calls Cody's RIBESL for I_{n+1/2}; here i_n is
//        computed by Miller's backward recurrence normalised with
//        i_0 = sinh(x)/x (same values to rounding)
//   lgndr, lgndrgt1            src/fmm/fmm_math_funcs.h:115-207
//   yformmp (P2M)              src/fmm/fmm.h:1426-1570
//   ympshift (M2M), ylcshift (L2L)  src/fmm/fmm.h:1718-2051
//   ympoletoexp, yftophys, convert_mp_to_exp  src/fmm/fmm.h:1143-1388, :2065-2096
//   translate_up_wave / translate_down_wave   src/fmm/fmm.h:1596-1715
//   yphystof, yexptolocal, pw_to_local        src/fmm/fmm.h:894-1141, :2098-2157
//   rotate_ztoy / ztox / ytoz                 src/fmm/fmm.h:2159-2359
//   convert_mpole_to_six_planewaves, convert_and_add_accumulated_planewaves
//                                              src/fmm/fmm.h:2363-2426
//   interaction list semantics                 src/fmm/fmm_octree.h:90-227
//     (the 1512-entry table of src/fmm/interaction_list.h is generated from
//      its rule: source = child of a non-self neighbour of the parent,
//      target = child of the parent, |offset| >= 2 on some axis; direction
//      along the axis of the largest |offset|, ties to z, then y, then x --
//      equal to the stored table entry for entry)
//   evaluate_local_expansion_at_xyz (12-way, potential, field, Hessian)
//                                              src/fmm/fmm.h:40-415, :696-892
//   FMM_results_to_BEM                         src/bem/bem_kernels.cpp:12-121
//   charges of a node patch                     src/bem/node_patch.h:339-394
// Everything in FP64.
#include <algorithm>
#include <cassert>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "oracle.h"

namespace {

using cd = std::complex<double>;
constexpr double PI = 3.14159265358979323846;
constexpr double PRECIS = 2.220446049250313e-16;
const cd IMA(0.0, 1.0);

inline int tri(int n, int m) { return m + n * (n + 1) / 2; }

// ---------------------------------------------------------------- special functions
// b[n] = i_n(x) / scal^n, n = 0..nb (src/fmm/fmm_math_funcs.h:24-113)
void i_n(double scal, double x, int nb, double* b) {
  const double ensig = 1e-4, enmten = 1e-300;
  const double inv_scal = 1.0 / scal;
  if (x <= ensig) {
    double xscal = x * inv_scal;
    double term1 = 1.0, term2 = 0.5 * x * x;
    b[0] = term1 * (1.0 + term2 / 3.0);
    for (int i = 1; i <= nb; ++i) {
      term1 *= xscal / double(2 * i + 1);
      if (term1 <= enmten) term1 = 0.0;
      b[i] = term1 * (1.0 + term2 / double(2 * i + 3));
    }
    return;
  }
  if (x > 100.0) {
    for (int i = 0; i <= nb; ++i) b[i] = 0.0;
    return;
  }
  // Miller's algorithm: i_{n-1} = i_{n+1} + (2n+1)/x i_n downwards from a
  // start well above nb, normalised with i_0(x) = sinh(x)/x.
  const int start = nb + 30 + (int)(2.0 * x);
  std::vector<double> v(start + 2, 0.0);
  v[start + 1] = 0.0;
  v[start] = 1e-300;
  for (int n = start; n >= 1; --n) {
    v[n - 1] = v[n + 1] + (2.0 * n + 1.0) / x * v[n];
    if (v[n - 1] > 1e250) {  // rescale to avoid overflow
      for (int k = n - 1; k <= start + 1; ++k) v[k] *= 1e-250;
    }
  }
  const double i0 = std::sinh(x) / x;
  const double norm = i0 / v[0];
  double constant = 1.0;
  for (int i = 0; i <= nb; ++i) {
    b[i] = v[i] * norm * constant;
    constant *= inv_scal;
    if (std::fabs(b[i]) <= enmten) constant = 0.0;
  }
}

// Associated Legendre P_n^m(x), Condon-Shortley phase (src/fmm/fmm_math_funcs.h:115-141)
void lgndr(int nmax, double x, std::vector<double>& y) {
  y.assign((nmax + 1) * (nmax + 2) / 2, 0.0);
  double u = -std::sqrt(1.0 - x * x);
  y[tri(0, 0)] = 1.0;
  for (int m = 0; m <= nmax; ++m) {
    if (m > 0) y[tri(m, m)] = y[tri(m - 1, m - 1)] * u * double(2 * m - 1);
    if (m < nmax) y[tri(m + 1, m)] = double(2 * m + 1) * x * y[tri(m, m)];
    for (int n = m + 2; n <= nmax; ++n)
      y[tri(n, m)] = ((2.0 * n - 1.0) * x * y[tri(n - 1, m)] - double(n + m - 1) * y[tri(n - 2, m)]) / double(n - m);
  }
}

// Scaled Legendre functions for x > 1 (src/fmm/fmm_math_funcs.h:143-207)
void lgndrgt1(int nmax, double scal, double x, std::vector<double>& y) {
  y.assign((nmax + 1) * (nmax + 2) / 2, 0.0);
  double v = scal * x, w = scal * scal, u = std::sqrt(x * x - 1.0) * scal;
  y[tri(0, 0)] = 1.0;
  for (int m = 0; m <= nmax; ++m) {
    if (m > 0) y[tri(m, m)] = y[tri(m - 1, m - 1)] * u * double(2 * m - 1);
    if (m < nmax) y[tri(m + 1, m)] = double(2 * m + 1) * v * y[tri(m, m)];
    for (int n = m + 2; n <= nmax; ++n)
      y[tri(n, m)] = ((2.0 * n - 1.0) * v * y[tri(n - 1, m)] - double(n + m - 1) * w * y[tri(n - 2, m)]) / double(n - m);
  }
}

// ---------------------------------------------------------------- global tables
struct Rot {
  int nt = 0;
  std::vector<double> d;
  void init(int n) {
    nt = n;
    d.assign((size_t)(nt + 1) * (nt + 1) * (2 * nt + 1), 0.0);
  }
  double& operator()(int l, int mp, int m) { return d[((size_t)l * (nt + 1) + mp) * (2 * nt + 1) + (m + nt)]; }
  double operator()(int l, int mp, int m) const { return d[((size_t)l * (nt + 1) + mp) * (2 * nt + 1) + (m + nt)]; }
};

struct Globals {
  int nt;
  Rot rdpi2, rdmpi2, rdsq3, rdmsq3;
  std::vector<double> scale_factors;  // tri(l, m)

  explicit Globals(int NT) : nt(NT) {
    const int nc = 4 * NT;
    std::vector<double> c((size_t)(nc + 1) * (nc + 1), 0.0);
    auto C_ = [&](int n, int m) -> double& { return c[(size_t)n * (nc + 1) + m]; };
    for (int n = 0; n <= nc; ++n) C_(n, 0) = 1.0;
    for (int m = 1; m <= nc; ++m) {
      C_(m, m) = 1.0;
      for (int n = m + 1; n <= nc; ++n) C_(n, m) = C_(n - 1, m) + C_(n - 1, m - 1);
    }
    for (int m = 1; m <= nc; ++m)
      for (int n = m + 1; n <= nc; ++n) C_(n, m) = std::sqrt(C_(n, m));
    auto sqc = [&](int n, int m) { return C_(n, m); };
    auto fstrtn = [&](Rot& d, double theta) {
      d.init(NT);
      const double precis = 1.0e-19, ww = 0.7071067811865476;
      double ct = std::cos(theta);
      if (std::fabs(ct) <= precis) ct = 0.0;
      double st = std::sin(-theta);
      if (std::fabs(st) <= precis) st = 0.0;
      double hst = ww * st, ctp = ww * (1.0 + ct), ctn = -ww * (1.0 - ct);
      d(0, 0, 0) = 1.0;
      for (int ij = 1; ij <= NT; ++ij) {
        for (int im = -ij; im <= -1; ++im) {
          d(ij, 0, im) = -sqc(ij - im, 2) * d(ij - 1, 0, im + 1);
          if (im > (1 - ij)) d(ij, 0, im) = d(ij, 0, im) + sqc(ij + im, 2) * d(ij - 1, 0, im - 1);
          d(ij, 0, im) = d(ij, 0, im) * hst;
          if (im > -ij) d(ij, 0, im) = d(ij, 0, im) + d(ij - 1, 0, im) * ct * sqc(ij + im, 1) * sqc(ij - im, 1);
          d(ij, 0, im) = d(ij, 0, im) / ij;
        }
        d(ij, 0, 0) = d(ij - 1, 0, 0) * ct;
        if (ij > 1) d(ij, 0, 0) = d(ij, 0, 0) + hst * sqc(ij, 2) * (d(ij - 1, 0, -1) + d(ij - 1, 0, 1)) / ij;
        for (int im = 1; im <= ij; ++im) {
          d(ij, 0, im) = -sqc(ij + im, 2) * d(ij - 1, 0, im - 1);
          if (im < (ij - 1)) d(ij, 0, im) = d(ij, 0, im) + sqc(ij - im, 2) * d(ij - 1, 0, im + 1);
          d(ij, 0, im) = d(ij, 0, im) * hst;
          if (im < ij) d(ij, 0, im) = d(ij, 0, im) + d(ij - 1, 0, im) * ct * sqc(ij + im, 1) * sqc(ij - im, 1);
          d(ij, 0, im) = d(ij, 0, im) / ij;
        }
        for (int imp = 1; imp <= ij; ++imp) {
          for (int im = -ij; im <= -1; ++im) {
            d(ij, imp, im) = d(ij - 1, imp - 1, im + 1) * ctn * sqc(ij - im, 2);
            if (im > (1 - ij)) d(ij, imp, im) = d(ij, imp, im) - d(ij - 1, imp - 1, im - 1) * ctp * sqc(ij + im, 2);
            if (im > -ij)
              d(ij, imp, im) = d(ij, imp, im) + d(ij - 1, imp - 1, im) * st * sqc(ij + im, 1) * sqc(ij - im, 1);
            d(ij, imp, im) = d(ij, imp, im) * ww / sqc(ij + imp, 2);
          }
          d(ij, imp, 0) = ij * st * d(ij - 1, imp - 1, 0);
          if (ij > 1)
            d(ij, imp, 0) =
                d(ij, imp, 0) - sqc(ij, 2) * (d(ij - 1, imp - 1, -1) * ctp + d(ij - 1, imp - 1, 1) * ctn);
          d(ij, imp, 0) = d(ij, imp, 0) * ww / sqc(ij + imp, 2);
          for (int im = 1; im <= ij; ++im) {
            d(ij, imp, im) = d(ij - 1, imp - 1, im - 1) * ctp * sqc(ij + im, 2);
            if (im < (ij - 1)) d(ij, imp, im) = d(ij, imp, im) - d(ij - 1, imp - 1, im + 1) * ctn * sqc(ij - im, 2);
            if (im < ij)
              d(ij, imp, im) = d(ij, imp, im) + d(ij - 1, imp - 1, im) * st * sqc(ij + im, 1) * sqc(ij - im, 1);
            d(ij, imp, im) = d(ij, imp, im) * ww / sqc(ij + imp, 2);
          }
        }
      }
      std::vector<double> f(2 * NT + 1);
      f[0] = 1.0;
      for (int n = 1; n <= 2 * NT; ++n) f[n] = f[n - 1] * double(n);
      for (int n = 0; n <= NT; ++n)
        for (int m = 0; m <= n; ++m)
          for (int mp = -n; mp <= n; ++mp) {
            int a = std::abs(mp);
            d(n, m, mp) = d(n, m, mp) * std::sqrt(f[n + m] / f[n + a] * f[n - a] / f[n - m]);
          }
    };
    fstrtn(rdpi2, PI / 2.0);
    fstrtn(rdmpi2, -PI / 2.0);
    fstrtn(rdsq3, std::acos(std::sqrt(3.0) / 3.0));
    fstrtn(rdmsq3, std::acos(-std::sqrt(3.0) / 3.0));
    std::vector<double> f(2 * NT + 1);
    f[0] = 1.0;
    for (int l = 1; l <= 2 * NT; ++l) f[l] = f[l - 1] * double(l);
    scale_factors.assign((NT + 1) * (NT + 2) / 2, 0.0);
    for (int l = 0; l <= NT; ++l)
      for (int m = 0; m <= l; ++m) scale_factors[tri(l, m)] = f[l - m] / f[l + m] * double(2 * l + 1);
  }
};

double get_scale(double beta, double edge, int level) {
  double s = beta * edge;
  if (s >= 1.0) s = 1.0;
  return s / (double)(1u << level);
}

// Yarvin-Rokhlin quadrature for the exponential representation of the
// Yukawa kernel (published tables, src/fmm/fmm_globals.h:495-577) and the
// Fourier/physical mode counts (src/fmm/fmm_globals.h:580-708).
void quadrature(int NT, std::vector<double>& x, std::vector<double>& w, std::vector<int>& numfour,
                std::vector<int>& numphys) {
  if (NT == 9) {
    x = {.099273996739714473469540223504736787, .47725674637049431137114652301534079,
         1.0553366138218296388373573790886439,  1.7675934335400844688024335482623428,
         2.5734262935147067530294862081063911,  3.4482433920158257478760788217186928,
         4.3768098355472631055818055756390095,  5.3489575720546005399569367000367492,
         6.3576578531337464283978988532908261};
    w = {.24776441819008371281185532097879332, .49188566500464336872511239562300034,
         .65378749137677805158830324216978624, .76433038408784093054038066838984378,
         .84376180565628111640563702167128213, .90445883985098263213586733400006779,
         .9537861313683345665381807521043811,  .99670261613218547047665651916759089,
         1.0429422730252668749528766056755558};
    numfour = {2, 4, 4, 6, 6, 4, 6, 4, 2};
    numphys = {4, 8, 12, 16, 20, 20, 24, 8, 2};
  } else if (NT == 18) {
    x = {.052788527661177607475107009804560221, .26949859838931256028615734976483509,
         .6322035317468939208396250251098536,   1.1130756427760852833586113774799742,
         1.6893949614021379623807206371566281,  2.3437620046953044905535534780938178,
         3.0626998290780611533534738555317745,  3.8356294126529686394633245072327554,
         4.6542473432156272750148673367220908,  5.5120938659358147404532246582675725,
         6.4042126837727888499784967279992998,  7.3268800190617540124549122992902994,
         8.2774009925823861522076185792684555,  9.2539718060248947750778825138695538,
         10.255602723746401139237605093512684,  11.282088297877740146191172243561596,
         12.334067909676926788620221486780792,  13.414920240172401477707353478763252};
    w = {.13438265914335215112096477696468355, .29457752727395436487256574764614925,
         .42607819361148618897416895379137713, .53189220776549905878027857397682965,
         .61787306245538586857435348065337166, .68863156078905074508611505734734237,
         .74749099381426187260757387775811367, .79699192718599998208617307682288811,
         .83917454386997591964103548889397644, .8757009228374531550898041132313665,
         .90792943590067498593754180546966381, .93698393742461816291466902839601971,
         .96382546688788062194674921556725167, .98932985769673820186653756536543369,
         1.0143828459791703888726033255807124, 1.0400365437416452252250564924906939,
         1.0681548926956736522697610780596733, 1.1090758097553685690428437737864442};
    numfour = {4, 6, 6, 8, 8, 8, 10, 10, 10, 10, 12, 12, 12, 12, 12, 12, 8, 2};
    numphys = {6, 8, 12, 16, 20, 26, 30, 34, 38, 44, 48, 52, 56, 60, 60, 52, 4, 2};
  } else {
    throw std::invalid_argument("FMM order must be 9 or 18");
  }
}

struct LevelGlobals {
  int nt, nl;
  double scale, betascal;
  std::vector<double> nodes, weights;
  std::vector<int> numfour, numphys;
  int nexptot = 0, nexptotp = 0, fsize = 0;
  std::vector<cd> fexpe, fexpo, fexpback;
  std::vector<cd> xs, ys;    // [3][nexptotp]
  std::vector<double> zs;    // [3][nexptotp]
  std::vector<double> rlsc;  // [tri(n,m)][nl]
  std::vector<double> mpshift, lcshift;  // [m][a][b], (nt+1)^3

  double& RL(int n, int m, int l) { return rlsc[(size_t)tri(n, m) * nl + l]; }
  double RL(int n, int m, int l) const { return rlsc[(size_t)tri(n, m) * nl + l]; }
  size_t S3(int m, int a, int b) const { return ((size_t)m * (nt + 1) + a) * (nt + 1) + b; }

  LevelGlobals(int NT, double beta, int level, double edge) : nt(NT) {
    scale = get_scale(beta, edge, level);
    double level_edge = edge / (double)(1u << level);
    betascal = beta * level_edge / 2.0;
    mpshift.assign((size_t)(nt + 1) * (nt + 1) * (nt + 1), 0.0);
    lcshift = mpshift;
    shift_coefficients(true, scale, beta, std::sqrt(3.0) * level_edge / 2.0, mpshift);
    quadrature(NT, nodes, weights, numfour, numphys);
    nl = (int)nodes.size();
    for (int i = 0; i < nl; ++i) {
      double li = nodes[i];
      double uu = std::sqrt(li * li + 2.0 * li * scale / 2.0);
      int indd = i, mmax = numphys[i];
      for (int jj = i; jj < nl; ++jj) {
        if (uu <= nodes[jj])
          indd = jj;
        else if (numphys[jj] > mmax)
          mmax = numphys[jj];
      }
      numphys[i] = mmax > numphys[indd] ? mmax : numphys[indd];
    }
    for (int i = 0; i < nl; ++i) {
      nexptot += numfour[i];
      nexptotp += numphys[i];
    }
    nexptotp /= 2;
    for (int i = 0; i < nl; ++i) fsize += numfour[i] * numphys[i];
    fsize /= 2;
    // ymkfexp (src/fmm/fmm_globals.h:802-897)
    for (int i = 0; i < nl; ++i) {
      int na = numphys[i], na2 = na / 2;
      double ha = 2.0 * PI / na;
      for (int j = 0; j < na2; ++j) {
        double alpha = ha * j;
        for (int mm = 2; mm <= numfour[i]; mm += 2) fexpe.push_back(std::exp(IMA * double(mm - 1) * alpha));
        for (int mm = 3; mm <= numfour[i]; mm += 2) fexpo.push_back(std::exp(IMA * double(mm - 1) * alpha));
      }
    }
    for (int i = 0; i < nl; ++i) {
      int na = numphys[i], na2 = na / 2;
      double ha = 2.0 * PI / na;
      for (int mm = 3; mm <= numfour[i]; mm += 2)
        for (int j = 0; j < na2; ++j) fexpback.push_back(std::exp(-IMA * double(mm - 1) * (ha * j)));
      for (int mm = 2; mm <= numfour[i]; mm += 2)
        for (int j = 0; j < na2; ++j) fexpback.push_back(std::exp(-IMA * double(mm - 1) * (ha * j)));
    }
    // yrlscini (src/fmm/fmm_globals.h:1045-1098)
    rlsc.assign((size_t)(nt + 1) * (nt + 2) / 2 * nl, 0.0);
    std::vector<double> tmp;
    for (int l = 0; l < nl; ++l) {
      double ul = nodes[l] / betascal + 1.0;
      lgndrgt1(nt, scale / 2.0, ul, tmp);
      for (int i = 0; i <= nt; ++i)
        for (int j = 0; j <= i; ++j) RL(i, j, l) = tmp[tri(i, j)];
    }
    // ymkexps (src/fmm/fmm_globals.h:711-800)
    xs.assign(3 * (size_t)nexptotp, cd(0));
    ys = xs;
    zs.assign(3 * (size_t)nexptotp, 0.0);
    int ntot = 0;
    for (int l = 0; l < nl; ++l) {
      double w1 = nodes[l] + betascal;
      double w2 = std::sqrt(nodes[l] * (nodes[l] + betascal * 2.0));
      double hu = 2.0 * PI / double(numphys[l]);
      for (int mth = 0; mth < numphys[l] / 2; ++mth) {
        double u = hu * mth;
        int c = ntot + mth;
        zs[c] = std::exp(-w1);
        zs[nexptotp + c] = zs[c] * zs[c];
        zs[2 * nexptotp + c] = zs[nexptotp + c] * zs[c];
        xs[c] = std::exp(IMA * w2 * std::cos(u));
        xs[nexptotp + c] = xs[c] * xs[c];
        xs[2 * nexptotp + c] = xs[nexptotp + c] * xs[c];
        ys[c] = std::exp(IMA * w2 * std::sin(u));
        ys[nexptotp + c] = ys[c] * ys[c];
        ys[2 * nexptotp + c] = ys[nexptotp + c] * ys[c];
      }
      ntot += numphys[l] / 2;
    }
    shift_coefficients(false, scale, beta, std::sqrt(3.0) * level_edge / 4.0, lcshift);
  }

  // ympshiftcoef (multipole=true) / ylcshftcoef (src/fmm/fmm_globals.h:919-1043)
  void shift_coefficients(bool multipole, double scal, double beta, double r0, std::vector<double>& c0) const {
    std::vector<double> f(2 * nt + 1);
    f[0] = 1.0;
    for (int n = 1; n <= 2 * nt; ++n) f[n] = f[n - 1] * double(n);
    double r0k = r0 * beta;
    std::vector<double> bj(2 * nt + 2);
    i_n(r0k, r0k, 2 * nt, bj.data());
    for (int m = 0; m <= nt; ++m)
      for (int nd = m; nd <= nt; ++nd)
        for (int n = m; n <= nt; ++n) {
          double acc = 0.0;
          int upper = (n <= nd) ? n : nd;
          for (int k = m; k <= upper; ++k) {
            double premult;
            if (multipole)
              premult = std::pow(scal, n - nd) * std::pow(2.0, -nd - k) * (((nd + n) % 2 == 0) ? 1.0 : -1.0);
            else
              premult = std::pow(scal, nd - n) * std::pow(2.0, -nd - k);
            double fac = double(2 * nd + 1) * f[nd - m] / f[k + m] * f[n + m] * f[2 * k] / f[k] / f[k - m] / f[nd - k] /
                         f[n - k];
            acc += premult * fac * bj[nd + n - k] * std::pow(r0k, nd + n - 2 * k);
          }
          c0[S3(m, nd, n)] = acc;
        }
  }
};

using Expansion = std::vector<cd>;  // tri(n, m), n <= nt

// ---------------------------------------------------------------- operators
// rotation application shared by ympshift / ylcshift / rotate_* :
// out(l, m) = in(l, 0) rd(l, 0, m) + sum_{mp>=1} in(l, mp) rd(l, mp, m) + conj(in(l, mp)) rd(l, mp, -m)
void rotate_apply(int nt, const Expansion& in, Expansion& out, const Rot& rd) {
  for (int l = 0; l <= nt; ++l)
    for (int m = 0; m <= l; ++m) {
      cd v = in[tri(l, 0)] * rd(l, 0, m);
      for (int mp = 1; mp <= l; ++mp) v = v + in[tri(l, mp)] * rd(l, mp, m) + std::conj(in[tri(l, mp)]) * rd(l, mp, -m);
      out[tri(l, m)] = v;
    }
}

// ympshift / ylcshift (src/fmm/fmm.h:1718-2051); shift coefficients dc(m, n, n')
void shift(int nt, int ifl, bool multipole, const Expansion& in, Expansion& out, const std::vector<double>& dc,
           const LevelGlobals& G, const Rot& rd) {
  const double arg = std::sqrt(2.0) / 2.0;
  cd e1;
  if (multipole) {
    if (ifl == 4 || ifl == 8) e1 = cd(-arg, arg);
    else if (ifl == 3 || ifl == 7) e1 = cd(arg, arg);
    else if (ifl == 1 || ifl == 5) e1 = cd(arg, -arg);
    else e1 = cd(-arg, -arg);
  } else {
    if (ifl == 4 || ifl == 8) e1 = cd(arg, -arg);
    else if (ifl == 3 || ifl == 7) e1 = cd(-arg, -arg);
    else if (ifl == 1 || ifl == 5) e1 = cd(-arg, arg);
    else e1 = cd(arg, arg);
  }
  std::vector<cd> ephi(nt + 3);
  ephi[0] = 1.0;
  ephi[1] = e1;
  for (int l = 1; l <= nt + 1; ++l) ephi[l + 1] = ephi[l] * ephi[1];
  Expansion w1(in.size()), w2(in.size());
  for (int l = 0; l <= nt; ++l)
    for (int m = 0; m <= l; ++m) w1[tri(l, m)] = std::conj(ephi[m]) * in[tri(l, m)];
  rotate_apply(nt, w1, w2, rd);
  for (int n = 0; n <= nt; ++n)
    for (int m = 0; m <= n; ++m) {
      cd v = 0.0;
      for (int nd = m; nd <= nt; ++nd) v += w2[tri(nd, m)] * dc[G.S3(m, n, nd)];
      w1[tri(n, m)] = v;
    }
  for (int l = 0; l <= nt; ++l) {
    for (int m = 0; m <= l; m += 2) {
      cd v = w1[tri(l, 0)] * rd(l, 0, m);
      for (int mp = 1; mp <= l; mp += 2) v = v - (w1[tri(l, mp)] * rd(l, mp, m) + std::conj(w1[tri(l, mp)]) * rd(l, mp, -m));
      for (int mp = 2; mp <= l; mp += 2) v = v + (w1[tri(l, mp)] * rd(l, mp, m) + std::conj(w1[tri(l, mp)]) * rd(l, mp, -m));
      w2[tri(l, m)] = v;
    }
    for (int m = 1; m <= l; m += 2) {
      cd v = -w1[tri(l, 0)] * rd(l, 0, m);
      for (int mp = 1; mp <= l; mp += 2) v = v + (w1[tri(l, mp)] * rd(l, mp, m) + std::conj(w1[tri(l, mp)]) * rd(l, mp, -m));
      for (int mp = 2; mp <= l; mp += 2) v = v - (w1[tri(l, mp)] * rd(l, mp, m) + std::conj(w1[tri(l, mp)]) * rd(l, mp, -m));
      w2[tri(l, m)] = v;
    }
  }
  for (int l = 0; l <= nt; ++l)
    for (int m = 0; m <= l; ++m) out[tri(l, m)] += ephi[m] * w2[tri(l, m)];
}

void rotate_ztoy(int nt, const Expansion& mp, Expansion& out, const Rot& rdminus) {
  Expansion w(mp.size());
  cd e = 1.0;
  std::vector<cd> ephi(nt + 1);
  for (int m = 0; m <= nt; ++m) {
    ephi[m] = e;
    e *= cd(0.0, -1.0);
  }
  for (int l = 0; l <= nt; ++l)
    for (int m = 0; m <= l; ++m) w[tri(l, m)] = ephi[m] * mp[tri(l, m)];
  rotate_apply(nt, w, out, rdminus);
}

void rotate_ytoz(int nt, const Expansion& mp, Expansion& out, const Rot& rdplus) {
  Expansion w(mp.size());
  rotate_apply(nt, mp, w, rdplus);
  cd e = 1.0;
  for (int m = 0; m <= nt; ++m) {
    for (int l = m; l <= nt; ++l) out[tri(l, m)] = e * w[tri(l, m)];
    e *= cd(0.0, 1.0);
  }
}

// ympoletoexp + yftophys: multipole -> up/down physical plane waves
void mp_to_exp(const LevelGlobals& G, const Expansion& mp, cd* up_phys, cd* dn_phys) {
  const int nt = G.nt, nl = G.nl;
  std::vector<cd> mup(G.nexptot), mdn(G.nexptot);
  int ntot = 0;
  for (int l = 0; l < nl; ++l) {
    double sgn = -1.0;
    for (int mth = 0; mth < G.numfour[l]; ++mth) {
      int cur = ntot + mth;
      cd z1 = 0.0, z2 = 0.0;
      sgn = -sgn;
      for (int nm = mth; nm <= nt; nm += 2) z1 += G.RL(nm, mth, l) * mp[tri(nm, mth)];
      for (int nm = mth + 1; nm <= nt; nm += 2) z2 += G.RL(nm, mth, l) * mp[tri(nm, mth)];
      mup[cur] = z1 + z2;
      mdn[cur] = sgn * (z1 - z2);
    }
    ntot += G.numfour[l];
  }
  auto ftophys = [&](const std::vector<cd>& mf, cd* phys) {
    int nftot = 0, nptot = 0, nexte = 0, nexto = 0;
    for (int i = 0; i < nl; ++i) {
      for (int iv = 0; iv < G.numphys[i] / 2; ++iv) {
        cd val = mf[nftot];
        int sgn = -2;
        for (int mm = 1; mm < G.numfour[i]; mm += 2) {
          sgn = -sgn;
          double r = sgn * std::real(G.fexpe[nexte] * mf[nftot + mm]);
          nexte++;
          val.imag(val.imag() + r);
        }
        sgn = 2;
        for (int mm = 2; mm < G.numfour[i]; mm += 2) {
          sgn = -sgn;
          double r = sgn * std::real(G.fexpo[nexto] * mf[nftot + mm]);
          nexto++;
          val.real(val.real() + r);
        }
        phys[nptot + iv] = val;
      }
      nftot += G.numfour[i];
      nptot += G.numphys[i] / 2;
    }
  };
  ftophys(mup, up_phys);
  ftophys(mdn, dn_phys);
}

// yphystof + yexptolocal: up/down physical waves -> local expansion
void exp_to_local(const LevelGlobals& G, const std::vector<double>& sfac, const cd* up, const cd* dn,
                  Expansion& local) {
  const int nt = G.nt, nl = G.nl;
  auto phystof = [&](const cd* phys, std::vector<cd>& mf) {
    mf.assign(G.nexptot, cd(0));
    int next = 0, nftot = 0, nptot = 0;
    for (int i = 0; i < nl; ++i) {
      int na = G.numphys[i], na2 = na / 2;
      cd v = 0.0;
      for (int iv = 0; iv < na2; ++iv) v += 2.0 * std::real(phys[nptot + iv]);
      mf[nftot] = v / double(na);
      for (int mm = 3; mm <= G.numfour[i]; mm += 2) {
        cd s = 0.0;
        for (int iv = 0; iv < na2; ++iv) {
          double rt = 2.0 * std::real(phys[nptot + iv]);
          s += G.fexpback[next] * rt;
          next++;
        }
        mf[nftot + mm - 1] = s / double(na);
      }
      for (int mm = 2; mm <= G.numfour[i]; mm += 2) {
        cd s = 0.0;
        for (int iv = 0; iv < na2; ++iv) {
          cd zt(0.0, 2.0 * std::imag(phys[nptot + iv]));
          s += G.fexpback[next] * zt;
          next++;
        }
        mf[nftot + mm - 1] = s / double(na);
      }
      nftot += G.numfour[i];
      nptot += G.numphys[i] / 2;
    }
  };
  std::vector<cd> fu, fd;
  phystof(up, fu);
  phystof(dn, fd);
  std::vector<cd> zeye(nt + 1);
  zeye[0] = 1.0;
  for (int i = 1; i <= nt; ++i) zeye[i] = zeye[i - 1] * IMA;
  std::fill(local.begin(), local.end(), cd(0));
  std::vector<cd> plus(G.nexptot), minus(G.nexptot);
  for (int k = 0; k < G.nexptot; ++k) {
    plus[k] = fd[k] + fu[k];
    minus[k] = fd[k] - fu[k];
  }
  int ntot = 0;
  for (int l = 0; l < nl; ++l) {
    for (int nm = 0; nm <= nt; nm += 2) {
      int mmax = G.numfour[l] - 1 > nm ? nm : G.numfour[l] - 1;
      for (int mth = 0; mth <= mmax; ++mth) local[tri(nm, mth)] += G.RL(nm, mth, l) * G.weights[l] * plus[ntot + mth];
    }
    for (int nm = 1; nm <= nt; nm += 2) {
      int mmax = G.numfour[l] - 1 > nm ? nm : G.numfour[l] - 1;
      for (int mth = 0; mth <= mmax; ++mth) local[tri(nm, mth)] += G.RL(nm, mth, l) * G.weights[l] * minus[ntot + mth];
    }
    ntot += G.numfour[l];
  }
  double rscale = PI / (G.betascal * 2.0);
  for (int nm = 0; nm <= nt; ++nm)
    for (int mth = 0; mth <= nm; ++mth) local[tri(nm, mth)] *= zeye[mth] * rscale * sfac[tri(nm, mth)];
}

// translate_up_wave / translate_down_wave (src/fmm/fmm.h:1596-1715)
void translate(const LevelGlobals& G, bool up, const cd* wave, cd* target, int dx, int dy, int dz) {
  const int np = G.nexptotp;
  for (int i = 0; i < np; ++i) {
    double tr = 1.0;
    cd t;
    if (up) {
      if (dz > 0) tr = G.zs[(size_t)(dz - 1) * np + i];
      t = cd(tr, 0.0);
      if (dy > 0) t *= G.ys[(size_t)(dy - 1) * np + i];
      else if (dy < 0) t *= std::conj(G.ys[(size_t)(-dy - 1) * np + i]);
      if (dx > 0) t *= G.xs[(size_t)(dx - 1) * np + i];
      else if (dx < 0) t *= std::conj(G.xs[(size_t)(-dx - 1) * np + i]);
      if (dz < 0) t /= G.zs[(size_t)(-dz - 1) * np + i];
    } else {
      if (dz < 0) tr = G.zs[(size_t)(-dz - 1) * np + i];
      t = cd(tr, 0.0);
      if (dy > 0) t *= std::conj(G.ys[(size_t)(dy - 1) * np + i]);
      else if (dy < 0) t *= G.ys[(size_t)(-dy - 1) * np + i];
      if (dx > 0) t *= std::conj(G.xs[(size_t)(dx - 1) * np + i]);
      else if (dx < 0) t *= G.xs[(size_t)(-dx - 1) * np + i];
    }
    target[i] += wave[i] * t;
  }
}

// ---------------------------------------------------------------- evaluation
// potential / gradient / Hessian of one local expansion at r (relative to
// the expansion centre), following evaluate_local_expansion_at_xyz.
struct EvalCache {
  int nt;
  std::vector<cd> q;    // (nt+3)^2 [n][m], m >= 0
  std::vector<cd> gq;   // [3][(nt+2)^2]
  std::vector<cd> g2q;  // [3][3][(nt+1)^2]
};

void eval_terms(int NT, double beta, double scale, double d, double ctheta, const std::vector<cd>& ephi,
                EvalCache& E) {
  const int N2 = NT + 2;
  std::vector<double> bi(NT + 4);
  i_n(scale, d * beta, NT + 2, bi.data());
  std::vector<double> p;
  lgndr(N2, ctheta, p);
  const int Wq = NT + 3;
  E.q.assign((size_t)Wq * Wq, cd(0));
  auto Q = [&](int n, int m) -> cd& { return E.q[(size_t)n * Wq + m]; };
  for (int n = 0; n <= N2; ++n)
    for (int m = 0; m <= n; ++m) Q(n, m) = (n == 0) ? cd(bi[0]) : bi[n] * p[tri(n, m)] * ephi[m];
  const double inv_scale = 1.0 / scale;
  // grad_q over n <= NT+1 (src/fmm/fmm.h:128-208)
  const int Wg = NT + 2;
  E.gq.assign(3 * (size_t)Wg * Wg, cd(0));
  auto GQ = [&](int c, int n, int m) -> cd& { return E.gq[((size_t)c * Wg + n) * Wg + m]; };
  auto grad_of = [&](auto&& src, int n, int m, double sc, double isc, cd out[3]) {
    cd left[3], right[3];
    if (n == 0 && m == 0) {
      left[0] = left[1] = left[2] = 0.0;
      right[0] = -std::conj(src(1, 1)) * sc;
      right[1] = -src(1, 0) * sc;
      right[2] = src(1, 1) * sc;
    } else if (n == 1 && m == 0) {
      left[0] = 0.0;
      left[1] = src(0, 0) * isc;
      left[2] = 0.0;
      right[0] = -std::conj(src(2, 1)) * sc;
      right[1] = -2.0 * src(2, 0) * sc;
      right[2] = src(2, 1) * sc;
    } else if (m == 0) {
      left[0] = -std::conj(src(n - 1, 1)) * isc;
      left[1] = src(n - 1, 0) * double(n) * isc;
      left[2] = src(n - 1, 1) * isc;
      right[0] = -std::conj(src(n + 1, 1)) * sc;
      right[1] = -double(n + 1) * src(n + 1, 0) * sc;
      right[2] = src(n + 1, 1) * sc;
    } else if (n == 1 && m == 1) {
      left[0] = 2.0 * src(0, 0) * isc;
      left[1] = left[2] = 0.0;
      right[0] = 2.0 * src(2, 0) * sc;
      right[1] = -src(2, 1) * sc;
      right[2] = src(2, 2) * sc;
    } else if (m == n) {
      left[0] = src(n - 1, n - 1) * (double((n + n - 1) * (n + n)) * isc);
      left[1] = left[2] = 0.0;
      right[0] = src(n + 1, n - 1) * 2.0 * sc;
      right[1] = -src(n + 1, n) * sc;
      right[2] = src(n + 1, n + 1) * sc;
    } else if (m == n - 1) {
      left[0] = src(n - 1, n - 2) * (double((n + m - 1) * (n + m)) * isc);
      left[1] = src(n - 1, n - 1) * (double(n + m) * isc);
      left[2] = 0.0;
      right[0] = src(n + 1, m - 1) * (6.0 * sc);
      right[1] = -src(n + 1, m) * (2.0 * sc);
      right[2] = src(n + 1, m + 1) * sc;
    } else {
      left[0] = src(n - 1, m - 1) * (double((n + m - 1) * (n + m)) * isc);
      left[1] = src(n - 1, m) * (double(n + m) * isc);
      left[2] = src(n - 1, m + 1) * isc;
      right[0] = src(n + 1, m - 1) * ((double(n - m + 1) * (n - m + 2)) * sc);
      right[1] = -src(n + 1, m) * (double(n - m + 1) * sc);
      right[2] = src(n + 1, m + 1) * sc;
    }
    const double pre = -0.5 / double(2 * n + 1);
    out[0] = pre * beta * ((left[0] - right[0]) - (left[2] - right[2]));
    out[1] = cd(0, pre * beta) * ((left[0] - right[0]) + (left[2] - right[2]));
    out[2] = pre * beta * -2.0 * (left[1] - right[1]);
  };
  for (int n = 0; n <= NT + 1; ++n)
    for (int m = 0; m <= n; ++m) {
      cd o[3];
      grad_of([&](int a, int b) -> cd { return Q(a, b); }, n, m, scale, inv_scale, o);
      for (int c = 0; c < 3; ++c) GQ(c, n, m) = o[c];
    }
  const int Wh = NT + 1;
  E.g2q.assign(9 * (size_t)Wh * Wh, cd(0));
  for (int i = 0; i < 3; ++i)
    for (int n = 0; n <= NT; ++n)
      for (int m = 0; m <= n; ++m) {
        cd o[3];
        grad_of([&](int a, int b) -> cd { return GQ(i, a, b); }, n, m, scale, inv_scale, o);
        for (int c = 0; c < 3; ++c) E.g2q[(((size_t)c * 3 + i) * Wh + n) * Wh + m] = o[c];
      }
}

// 12-way evaluation and FMM_results_to_BEM for one target
void eval_patch(int NT, double beta, double beta0, double scale, double scale0, const double* xyz, const double* c0,
                const std::vector<Expansion>& loc12, const double* nrm, double& f_out, double& h_out) {
  double r[3] = {xyz[0] - c0[0], xyz[1] - c0[1], xyz[2] - c0[2]};
  double proj = r[0] * r[0] + r[1] * r[1];
  double rr = proj + r[2] * r[2];
  proj = std::sqrt(proj);
  double d = std::sqrt(rr);
  double ct = (d <= PRECIS) ? 0.0 : r[2] / d;
  std::vector<cd> ephi(NT + 5);
  ephi[0] = 1.0;
  ephi[1] = (proj <= PRECIS * d) ? cd(1.0) : cd(r[0] / proj, r[1] / proj);
  for (int i = 1; i <= NT + 2; ++i) ephi[i + 1] = ephi[i] * ephi[1];
  double pot[12], fld[3][12], f2[3][3][12];
  EvalCache E;
  const int Wq = NT + 3, Wg = NT + 2, Wh = NT + 1;
  for (int ch = 0; ch < 12; ++ch) {
    const double b = ch >= 8 ? beta0 : beta;
    const double s = ch >= 8 ? scale0 : scale;
    if (ch == 0 || (ch == 8 && beta0 != beta)) eval_terms(NT, b, s, d, ct, ephi, E);
    const Expansion& L = loc12[ch];
    double p = 0, fx = 0, fy = 0, fz = 0, h2[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    auto accum = [&](int n, int m) {
      const cd lv = L[tri(n, m)];
      p += std::real(E.q[(size_t)n * Wq + m] * lv);
      fx += std::real(E.gq[((size_t)0 * Wg + n) * Wg + m] * lv);
      fy += std::real(E.gq[((size_t)1 * Wg + n) * Wg + m] * lv);
      fz += std::real(E.gq[((size_t)2 * Wg + n) * Wg + m] * lv);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) h2[i][j] += std::real(E.g2q[(((size_t)i * 3 + j) * Wh + n) * Wh + m] * lv);
    };
    for (int n = 0; n <= NT; ++n)
      for (int m = 1; m <= n; ++m) accum(n, m);
    p *= 2.0;
    fx *= 2.0;
    fy *= 2.0;
    fz *= 2.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) h2[j][i] *= 2.0;
    for (int n = 0; n <= NT; ++n) accum(n, 0);
    const double tb = b * (2.0 / PI);
    pot[ch] = p * tb;
    fld[0][ch] = fx * tb;
    fld[1][ch] = fy * tb;
    fld[2][ch] = fz * tb;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) f2[i][j][ch] = h2[i][j] * tb;
  }
  // FMM_results_to_BEM (src/bem/bem_kernels.cpp:12-121, active branch)
  double fa = 0, ha = 0;
  fa += fld[0][0] + fld[1][1] + fld[2][2];
  double hc = 0;
  for (int j = 0; j < 3; ++j) {
    hc += (f2[j][0][4] + f2[0][j][4]) * nrm[j];
    hc += (f2[j][1][5] + f2[1][j][5]) * nrm[j];
    hc += (f2[j][2][6] + f2[2][j][6]) * nrm[j];
  }
  ha += hc / 2.0;
  fa += pot[3];
  ha += fld[0][7] * nrm[0] + fld[1][7] * nrm[1] + fld[2][7] * nrm[2];
  fa -= fld[0][8] + fld[1][9] + fld[2][10];
  hc = 0;
  for (int j = 0; j < 3; ++j) {
    hc += (f2[j][0][8] + f2[0][j][8]) * nrm[j];
    hc += (f2[j][1][9] + f2[1][j][9]) * nrm[j];
    hc += (f2[j][2][10] + f2[2][j][10]) * nrm[j];
  }
  ha -= hc / 2.0;
  fa -= pot[11];
  ha -= fld[0][11] * nrm[0] + fld[1][11] * nrm[1] + fld[2][11] * nrm[2];
  const double one_over_4pi = 1.0 / (4.0 * PI);
  f_out += fa * one_over_4pi;
  h_out += ha * one_over_4pi;
}

// BasicNodePatch::get_fmm_charge_equiv (src/bem/node_patch.h:339-394)
void patch_charges(const OrPatches* P, int i, double f, double h, double q[12]) {
  const double a = P->area[i], e = P->eps[i];
  const double* n = P->normal + 3 * (size_t)i;
  q[0] = a * f * n[0];
  q[1] = a * f * n[1];
  q[2] = a * f * n[2];
  q[3] = a * h;
  q[4] = a * f * n[0] / e;
  q[5] = a * f * n[1] / e;
  q[6] = a * f * n[2] / e;
  q[7] = a * h / e;
  q[8] = a * f * n[0] / e;
  q[9] = a * f * n[1] / e;
  q[10] = a * f * n[2] / e;
  q[11] = a * h;
}

// The 189 well-separated (source child of a non-self parent neighbour,
// target child) pairs per target, with their plane-wave direction.
struct Interaction {
  int nb, dir, targ, src, dx, dy, dz;
};
enum { UP = 0, DOWN = 1, NORTH = 2, SOUTH = 3, EAST = 4, WEST = 5 };

std::vector<Interaction> interaction_list() {
  std::vector<Interaction> out;
  for (int nb = 0; nb < 27; ++nb) {
    if (nb == 13) continue;
    int pz = nb / 9 - 1, py = (nb % 9) / 3 - 1, px = nb % 3 - 1;
    for (int t = 1; t <= 8; ++t) {
      int tx = (t - 1) & 1, ty = ((t - 1) >> 1) & 1, tz = (t - 1) >> 2;
      for (int s = 1; s <= 8; ++s) {
        int sx = 2 * px + ((s - 1) & 1), sy = 2 * py + (((s - 1) >> 1) & 1), sz = 2 * pz + ((s - 1) >> 2);
        int dx = tx - sx, dy = ty - sy, dz = tz - sz;
        const int m = std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz)));
        if (m < 2) continue;
        // the axis of the largest separation, ties to z, then y, then x
        int dir;
        if (std::abs(dz) == m) dir = dz > 0 ? UP : DOWN;
        else if (std::abs(dy) == m) dir = dy > 0 ? NORTH : SOUTH;
        else dir = dx > 0 ? EAST : WEST;
        out.push_back({nb, dir, t, s, dx, dy, dz});
      }
    }
  }
  return out;
}

}  // namespace

// ---------------------------------------------------------------- driver
struct OrFmm {
  const OrPatches* P;
  int NT;
  int n_nodes, n_levels;
  double beta, beta0, edge;
  std::vector<int32_t> info, neigh, contents;
  std::vector<double> geom;  // [n][4] centre xyz, edge
  Globals G;
  std::vector<LevelGlobals> LG, LG0;  // per level, beta and beta0
  std::vector<Interaction> ilist;
  OrFmm(const OrPatches* p, const OrTree* t, int nt, double b, double b0, double e)
      : P(p), NT(nt), n_nodes(t->n_nodes), n_levels(t->n_levels), beta(b), beta0(b0), edge(e), G(nt) {
    info.assign(t->info, t->info + 18 * (size_t)n_nodes);
    neigh.assign(t->neighbours, t->neighbours + 27 * (size_t)n_nodes);
    contents.assign(t->contents, t->contents + t->n_contents);
    geom.assign(t->geom, t->geom + 4 * (size_t)n_nodes);
    if (beta < beta0) beta = beta0;  // src/fmm/fmm_bem_hybrid.h:187
    for (int l = 0; l < n_levels; ++l) {
      LG.emplace_back(NT, beta, l, edge);
      LG0.emplace_back(NT, beta0, l, edge);
    }
    ilist = interaction_list();
  }
  const int32_t* I(int k) const { return &info[18 * (size_t)k]; }
};

extern "C" {

// The oracle's interaction list, 7 ints per entry (neighbour, direction,
// target child 1..8, source child 1..8, dx, dy, dz); returns the count and
// fills out when it is not null.
int or_interaction_list(int32_t* out) {
  const std::vector<Interaction> l = interaction_list();
  if (out)
    for (size_t k = 0; k < l.size(); ++k) {
      const int32_t v[7] = {l[k].nb, (int32_t)l[k].dir, l[k].targ, l[k].src, l[k].dx, l[k].dy, l[k].dz};
      for (int c = 0; c < 7; ++c) out[7 * k + c] = v[c];
    }
  return (int)l.size();
}

OrFmm* or_fmm_create(const OrPatches* P, const OrTree* T, double kappa, double beta0, double edge, int nterms) {
  return new OrFmm(P, T, nterms, kappa, beta0, edge);
}

void or_fmm_destroy(OrFmm* F) { delete F; }

// y (2N) += far field of x (FMM_BEM_Octree::solve, src/fmm/fmm_bem_hybrid.h:183-279)
void or_fmm_apply(OrFmm* F, const double* x, double* y) {
  const OrPatches* P = F->P;
  const int n = P->n, NT = F->NT, nn = F->n_nodes;
  const int bottom = F->n_levels - 1;
  if (bottom < 2) return;
  const size_t esz = (size_t)(NT + 1) * (NT + 2) / 2;
  // per node 12 multipoles and 12 locals
  std::vector<std::vector<Expansion>> M(nn), Lc(nn);
  for (int k = 0; k < nn; ++k) {
    M[k].assign(12, Expansion(esz, cd(0)));
    Lc[k].assign(12, Expansion(esz, cd(0)));
  }
  auto level_of = [&](int k) { return F->I(k)[0]; };
  auto flags = [&](int k) { return F->I(k)[4]; };
  auto count = [&](int k) { return F->I(k)[7]; };
  auto child = [&](int k, int c) { return F->I(k)[10 + c - 1]; };
  // P2M at non-empty childless nodes (src/fmm/fmm_bem_hybrid.h:282-335);
  // nodes in parallel as the reference's patches (src/fmm/fmm.h:1550)
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < nn; ++k) {
    if ((flags(k) & 1) || count(k) == 0) continue;
    std::vector<double> p;
    const int lev = level_of(k);
    const double* c0 = &F->geom[4 * (size_t)k];
    const int cs = F->I(k)[6], cc = count(k);
    for (int half = 0; half < 2; ++half) {
      const double b = half ? F->beta0 : F->beta;
      const double sc = get_scale(b, F->edge, lev);
      const int ch0 = half ? 8 : 0, ch1 = half ? 12 : 8;
      for (int t = 0; t < cc; ++t) {
        const int i = F->contents[cs + t];
        const double* pt = P->centroid + 3 * (size_t)i;
        double r[3] = {pt[0] - c0[0], pt[1] - c0[1], pt[2] - c0[2]};
        double proj = r[0] * r[0] + r[1] * r[1];
        double rr = proj + r[2] * r[2];
        proj = std::sqrt(proj);
        double d = std::sqrt(rr);
        double ct = (d <= PRECIS) ? 1.0 : r[2] / d;
        std::vector<cd> ephi(NT + 1);
        ephi[0] = (proj <= PRECIS * d) ? cd(1.0) : cd(r[0] / proj, -r[1] / proj);
        for (int e = 1; e < NT; ++e) ephi[e] = ephi[e - 1] * ephi[0];
        std::vector<double> bi(NT + 2);
        i_n(sc, d * b, NT, bi.data());
        lgndr(NT, ct, p);
        Expansion mp(esz, cd(0));
        mp[0] = bi[0];
        for (int l = 1; l <= NT; ++l) {
          mp[tri(l, 0)] = p[tri(l, 0)] * bi[l] * F->G.scale_factors[tri(l, 0)];
          for (int m = 1; m <= l; ++m) mp[tri(l, m)] = (bi[l] * F->G.scale_factors[tri(l, m)] * p[tri(l, m)]) * ephi[m - 1];
        }
        double q[12];
        patch_charges(P, i, x[i], x[n + i], q);
        for (int ch = ch0; ch < ch1; ++ch)
          for (size_t e = 0; e < esz; ++e) M[k][ch][e] += mp[e] * q[ch];
      }
    }
  }
  // M2M upward (src/fmm/fmm_bem_hybrid.h:337-410).  Parents in parallel
  // (the reference runs ympshift's channels in parallel, src/fmm/fmm.h:1801);
  // each parent takes its children in node order, as the serial loop does.
  for (int lev = bottom; lev > 0; --lev) {
    std::vector<int> parents;
    std::vector<std::vector<int>> kids(nn);
    for (int k = 0; k < nn; ++k) {
      if (level_of(k) != lev || count(k) == 0) continue;
      const int par = F->I(k)[5];
      if (kids[par].empty()) parents.push_back(par);
      kids[par].push_back(k);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int pi = 0; pi < (int)parents.size(); ++pi) {
      const int par = parents[pi];
      for (int k : kids[par]) {
        const int32_t* ik = F->I(k);
        int id = 1 + (ik[1] & 1) + 2 * (ik[2] & 1) + 4 * (ik[3] & 1);
        const Rot& rd = (id > 4) ? F->G.rdmsq3 : F->G.rdsq3;
        for (int ch = 0; ch < 12; ++ch) {
          const LevelGlobals& LGl = ch < 8 ? F->LG[lev] : F->LG0[lev];
          shift(NT, id, true, M[k][ch], M[par][ch], LGl.mpshift, LGl, rd);
        }
      }
    }
  }
  // downward pass: interaction lists (src/fmm/fmm_bem_hybrid.h:458-581)
  for (int lev = 0; lev < bottom; ++lev) {
    const LevelGlobals& A = F->LG[lev];
    const LevelGlobals& B = F->LG0[lev];
    const int npA = A.nexptotp, npB = B.nexptotp;
    // waves[node][dir][ch] for non-empty nodes at lev+1
    std::vector<std::vector<cd>> waves(nn);
    // multipole -> six plane waves per node in parallel (src/fmm/fmm.h:2376)
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < nn; ++k) {
      if (level_of(k) != lev + 1 || count(k) == 0) continue;
      waves[k].assign(6 * 12 * (size_t)std::max(npA, npB), cd(0));
      const size_t W = std::max(npA, npB);
      for (int ch = 0; ch < 12; ++ch) {
        const LevelGlobals& G = ch < 8 ? A : B;
        Expansion rot(esz);
        auto wp = [&](int dir) { return &waves[k][((size_t)dir * 12 + ch) * W]; };
        mp_to_exp(G, M[k][ch], wp(UP), wp(DOWN));
        rotate_ztoy(NT, M[k][ch], rot, F->G.rdmpi2);
        mp_to_exp(G, rot, wp(NORTH), wp(SOUTH));
        rotate_apply(NT, M[k][ch], rot, F->G.rdpi2);
        mp_to_exp(G, rot, wp(EAST), wp(WEST));
      }
    }
    const size_t W = std::max(npA, npB);
    // interaction lists and wave -> local conversion per parent in parallel
    // (src/fmm/fmm_octree.h:169, src/fmm/fmm.h:1616, :1676, :2407); a parent
    // writes only its own children's locals
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < nn; ++k) {
      if (level_of(k) != lev) continue;
      if ((flags(k) & 2) || (flags(k) & 4)) continue;  // leaf or shadow
      // targets: existing non-shadow children
      bool targs[8];
      for (int c = 1; c <= 8; ++c) {
        int ck = child(k, c);
        targs[c - 1] = ck >= 0 && !(flags(ck) & 4);
      }
      std::vector<cd> acc(6 * 8 * 12 * W, cd(0));
      for (const Interaction& it : F->ilist) {
        if (!targs[it.targ - 1]) continue;
        int nbk = F->neigh[27 * (size_t)k + it.nb];
        if (nbk < 0 || count(nbk) == 0) continue;
        int sk = child(nbk, it.src);
        if (sk < 0 || count(sk) == 0) continue;
        int a, bb, c;
        bool up;
        switch (it.dir) {
          case UP: a = it.dx; bb = it.dy; c = it.dz; up = true; break;
          case NORTH: a = it.dz; bb = it.dx; c = it.dy; up = true; break;
          case EAST: a = -it.dz; bb = it.dy; c = it.dx; up = true; break;
          case DOWN: a = it.dx; bb = it.dy; c = it.dz; up = false; break;
          case SOUTH: a = it.dz; bb = it.dx; c = it.dy; up = false; break;
          default: a = -it.dz; bb = it.dy; c = it.dx; up = false; break;
        }
        for (int ch = 0; ch < 12; ++ch) {
          const LevelGlobals& G = ch < 8 ? A : B;
          const cd* src = &waves[sk][((size_t)it.dir * 12 + ch) * W];
          cd* dst = &acc[(((size_t)it.dir * 8 + (it.targ - 1)) * 12 + ch) * W];
          translate(G, up, src, dst, a, bb, c);
        }
      }
      for (int c = 1; c <= 8; ++c) {
        int ck = child(k, c);
        if (ck < 0 || (flags(ck) & 4)) continue;
        for (int ch = 0; ch < 12; ++ch) {
          const LevelGlobals& G = ch < 8 ? A : B;
          auto ap = [&](int dir) { return &acc[(((size_t)dir * 8 + (c - 1)) * 12 + ch) * W]; };
          Expansion lo(esz), ro(esz);
          exp_to_local(G, F->G.scale_factors, ap(UP), ap(DOWN), lo);
          for (size_t e = 0; e < esz; ++e) Lc[ck][ch][e] += lo[e];
          exp_to_local(G, F->G.scale_factors, ap(NORTH), ap(SOUTH), lo);
          rotate_ytoz(NT, lo, ro, F->G.rdpi2);
          for (size_t e = 0; e < esz; ++e) Lc[ck][ch][e] += ro[e];
          exp_to_local(G, F->G.scale_factors, ap(EAST), ap(WEST), lo);
          rotate_apply(NT, lo, ro, F->G.rdmpi2);
          for (size_t e = 0; e < esz; ++e) Lc[ck][ch][e] += ro[e];
        }
      }
    }
  }
  // L2L (src/fmm/fmm_bem_hybrid.h:412-439, :86-124), parents in parallel
  // (each child has one parent)
  for (int lev = 0; lev < bottom; ++lev) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < nn; ++k) {
      if (level_of(k) != lev) continue;
      if (!(flags(k) & 1) || (flags(k) & 2)) continue;  // has children and not leaf
      for (int c = 1; c <= 8; ++c) {
        int ck = child(k, c);
        if (ck < 0 || count(ck) == 0 || (flags(ck) & 4)) continue;
        const Rot& rd = (c > 4) ? F->G.rdsq3 : F->G.rdmsq3;
        for (int ch = 0; ch < 12; ++ch) {
          const LevelGlobals& G = ch < 8 ? F->LG[lev] : F->LG0[lev];
          shift(NT, c, false, Lc[k][ch], Lc[ck][ch], G.lcshift, G, rd);
        }
      }
    }
  }
  // L2P at leaf patch centroids (src/fmm/fmm_bem_hybrid.h:583-642; the
  // reference's patches in parallel, :606), leaves in parallel
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < nn; ++k) {
    if (!(flags(k) & 2)) continue;
    const int lev = level_of(k);
    const double s = get_scale(F->beta, F->edge, lev), s0 = get_scale(F->beta0, F->edge, lev);
    const double* c0 = &F->geom[4 * (size_t)k];
    const int cs = F->I(k)[6], cc = count(k);
    for (int t = 0; t < cc; ++t) {
      const int i = F->contents[cs + t];
      eval_patch(NT, F->beta, F->beta0, s, s0, P->centroid + 3 * (size_t)i, c0, Lc[k], P->normal + 3 * (size_t)i,
                 y[i], y[n + i]);
    }
  }
}

// Direct 12-channel far field over explicit (target, source) pairs, the sum
// the FMM approximates: y[t] += FMM_results_to_BEM of the screened /
// pseudo-Laplace potentials, fields and Hessians at target centroids.
// Pairs of one target must be contiguous and no target may appear in two
// runs; runs are summed in parallel, each in pair order.
void or_fmm_direct(const OrPatches* P, double kappa, double beta0, int npairs, const int32_t* T, const int32_t* S,
                   const double* x, double* y) {
  std::vector<int> runs;
  for (int k = 0; k < npairs; ++k)
    if (k == 0 || T[k] != T[k - 1]) runs.push_back(k);
  runs.push_back(npairs);
  const int n_runs = (int)runs.size() - 1;
  const int n = P->n;
  const double beta = kappa < beta0 ? beta0 : kappa;
#pragma omp parallel for schedule(dynamic, 1)
  for (int ri = 0; ri < n_runs; ++ri)
  for (int k = runs[ri]; k < runs[ri + 1]; ++k) {
    const int t = T[k], s = S[k];
    double q[12];
    patch_charges(P, s, x[s], x[n + s], q);
    const double* pt = P->centroid + 3 * (size_t)t;
    const double* ps = P->centroid + 3 * (size_t)s;
    double d[3] = {pt[0] - ps[0], pt[1] - ps[1], pt[2] - ps[2]};
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r = std::sqrt(r2);
    double pot[12], fld[3][12], f2[3][3][12];
    for (int ch = 0; ch < 12; ++ch) {
      const double b = ch >= 8 ? beta0 : beta;
      const double e = std::exp(-b * r);
      const double ph = q[ch] * e / r;
      const double g1 = -q[ch] * e * (1.0 + b * r) / (r2 * r);
      const double g2 = q[ch] * e * (3.0 + 3.0 * b * r + b * b * r2) / (r2 * r2 * r);
      pot[ch] = ph;
      for (int a = 0; a < 3; ++a) {
        fld[a][ch] = g1 * d[a];
        for (int c = 0; c < 3; ++c) f2[a][c][ch] = g2 * d[a] * d[c] + (a == c ? g1 : 0.0);
      }
    }
    const double* nrm = P->normal + 3 * (size_t)t;
    double fa = fld[0][0] + fld[1][1] + fld[2][2] + pot[3] - (fld[0][8] + fld[1][9] + fld[2][10]) - pot[11];
    double hc = 0, hc0 = 0;
    for (int j = 0; j < 3; ++j) {
      hc += (f2[j][0][4] + f2[0][j][4]) * nrm[j] + (f2[j][1][5] + f2[1][j][5]) * nrm[j] +
            (f2[j][2][6] + f2[2][j][6]) * nrm[j];
      hc0 += (f2[j][0][8] + f2[0][j][8]) * nrm[j] + (f2[j][1][9] + f2[1][j][9]) * nrm[j] +
             (f2[j][2][10] + f2[2][j][10]) * nrm[j];
    }
    double ha = hc / 2.0 + (fld[0][7] * nrm[0] + fld[1][7] * nrm[1] + fld[2][7] * nrm[2]) - hc0 / 2.0 -
                (fld[0][11] * nrm[0] + fld[1][11] * nrm[1] + fld[2][11] * nrm[2]);
    y[t] += fa / (4.0 * PI);
    y[n + t] += ha / (4.0 * PI);
  }
}

}  // extern "C"
