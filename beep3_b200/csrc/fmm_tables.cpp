// Host precomputation of the plane-wave FMM tables (FP64), uploaded once per
// problem.  The tables and their generation follow the reference:
//   rotation matrices d(l, m', m) for angles +-pi/2 and +-acos(1/sqrt 3)
//     (FMM_Globals::yhrotgen / bnlcft / yhfstrtn, src/fmm/fmm_globals.h:72-368)
//   scale factors (l-m)!/(l+m)! (2l+1)          (yhfrmini, :98-118)
//   per level and screening constant: scale, Yarvin-Rokhlin nodes/weights
//     and mode counts with the numphys adjustment, Fourier<->physical
//     exponentials, scaled Legendre functions rlsc, diagonal translation
//     factors xs/ys/zs, multipole and local z-shift coefficients
//     (Level_Dependent_FMM_Globals, :372-1100)
//   scaled modified spherical Bessel functions i_n (fmm_math_funcs.h:24-113;
//     computed here by Miller's backward recurrence normalised with
//     i_0 = sinh(x)/x where the reference calls Cody's RIBESL).
#include "fmm_tables.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <stdexcept>

namespace bp {

static const double kPi = 3.14159265358979323846;

void bessel_in(double scal, double x, int nb, double* b) {
  const double ensig = 1e-4, enmten = 1e-300;
  const double inv_scal = 1.0 / scal;
  if (x <= ensig) {
    const double xs = x * inv_scal, t2 = 0.5 * x * x;
    double t1 = 1.0;
    b[0] = 1.0 + t2 / 3.0;
    for (int i = 1; i <= nb; ++i) {
      t1 *= xs / double(2 * i + 1);
      if (t1 <= enmten) t1 = 0.0;
      b[i] = t1 * (1.0 + t2 / double(2 * i + 3));
    }
    return;
  }
  if (x > 100.0) {
    for (int i = 0; i <= nb; ++i) b[i] = 0.0;
    return;
  }
  const int top = nb + 30 + (int)(2.0 * x);
  std::vector<double> v(top + 2, 0.0);
  v[top] = 1e-300;
  for (int n = top; n >= 1; --n) {
    v[n - 1] = v[n + 1] + (2.0 * n + 1.0) / x * v[n];
    if (v[n - 1] > 1e250)
      for (int k = n - 1; k <= top + 1; ++k) v[k] *= 1e-250;
  }
  const double norm = (std::sinh(x) / x) / v[0];
  double c = 1.0;
  for (int i = 0; i <= nb; ++i) {
    b[i] = v[i] * norm * c;
    c *= inv_scal;
    if (std::fabs(b[i]) <= enmten) c = 0.0;
  }
}

// Source = child of a non-self neighbour of the parent, target = child of
// the parent, separated by >= 2 child boxes along some axis.  The wave
// travels along the axis of the largest separation, ties going to z, then
// y, then x (UP/DOWN, NORTH/SOUTH, EAST/WEST by its sign): that is the
// direction of every entry of the reference's table (checked against the
// table itself by the tests), and it keeps the sideways offsets of a wave
// small.  Child ids are 0-based here (the reference's are 1..8): bit 0 x,
// bit 1 y, bit 2 z.
std::vector<RawInteraction> interaction_table() {
  std::vector<RawInteraction> out;
  for (int nb = 0; nb < 27; ++nb) {
    if (nb == 13) continue;
    const int pz = nb / 9 - 1, py = (nb % 9) / 3 - 1, px = nb % 3 - 1;
    for (int t = 0; t < 8; ++t) {
      const int tx = t & 1, ty = (t >> 1) & 1, tz = t >> 2;
      for (int s = 0; s < 8; ++s) {
        const int sx = 2 * px + (s & 1), sy = 2 * py + ((s >> 1) & 1), sz = 2 * pz + (s >> 2);
        const int dx = tx - sx, dy = ty - sy, dz = tz - sz;
        const int m = std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz)));
        if (m < 2) continue;
        int dir;
        if (std::abs(dz) == m) dir = dz > 0 ? 0 : 1;
        else if (std::abs(dy) == m) dir = dy > 0 ? 2 : 3;
        else dir = dx > 0 ? 4 : 5;
        out.push_back({nb, dir, t, s, dx, dy, dz});
      }
    }
  }
  return out;
}

double fmm_scale(double beta, double edge, int level) {
  double s = beta * edge;
  if (s >= 1.0) s = 1.0;
  return s / (double)(1ull << level);
}

namespace {

// d(l, mp, m) of a rotation by theta about the y axis, scaled as in the reference
void rotation(int nt, double theta, std::vector<double>& out) {
  const int nc = 4 * nt;
  std::vector<double> c((size_t)(nc + 1) * (nc + 1), 0.0);
  auto C = [&](int n, int m) -> double& { return c[(size_t)n * (nc + 1) + m]; };
  for (int n = 0; n <= nc; ++n) C(n, 0) = 1.0;
  for (int m = 1; m <= nc; ++m) {
    C(m, m) = 1.0;
    for (int n = m + 1; n <= nc; ++n) C(n, m) = C(n - 1, m) + C(n - 1, m - 1);
  }
  for (int m = 1; m <= nc; ++m)
    for (int n = m + 1; n <= nc; ++n) C(n, m) = std::sqrt(C(n, m));
  out.assign((size_t)(nt + 1) * (nt + 1) * (2 * nt + 1), 0.0);
  auto d = [&](int l, int mp, int m) -> double& { return out[((size_t)l * (nt + 1) + mp) * (2 * nt + 1) + m + nt]; };
  const double ww = 0.7071067811865476;
  double ct = std::cos(theta), st = std::sin(-theta);
  if (std::fabs(ct) <= 1e-19) ct = 0.0;
  if (std::fabs(st) <= 1e-19) st = 0.0;
  const double hs = ww * st, cp = ww * (1.0 + ct), cn = -ww * (1.0 - ct);
  d(0, 0, 0) = 1.0;
  for (int j = 1; j <= nt; ++j) {
    for (int m = -j; m <= -1; ++m) {
      double v = -C(j - m, 2) * d(j - 1, 0, m + 1);
      if (m > 1 - j) v += C(j + m, 2) * d(j - 1, 0, m - 1);
      v *= hs;
      if (m > -j) v += d(j - 1, 0, m) * ct * C(j + m, 1) * C(j - m, 1);
      d(j, 0, m) = v / j;
    }
    double v0 = d(j - 1, 0, 0) * ct;
    if (j > 1) v0 += hs * C(j, 2) * (d(j - 1, 0, -1) + d(j - 1, 0, 1)) / j;
    d(j, 0, 0) = v0;
    for (int m = 1; m <= j; ++m) {
      double v = -C(j + m, 2) * d(j - 1, 0, m - 1);
      if (m < j - 1) v += C(j - m, 2) * d(j - 1, 0, m + 1);
      v *= hs;
      if (m < j) v += d(j - 1, 0, m) * ct * C(j + m, 1) * C(j - m, 1);
      d(j, 0, m) = v / j;
    }
    for (int mp = 1; mp <= j; ++mp) {
      for (int m = -j; m <= -1; ++m) {
        double v = d(j - 1, mp - 1, m + 1) * cn * C(j - m, 2);
        if (m > 1 - j) v -= d(j - 1, mp - 1, m - 1) * cp * C(j + m, 2);
        if (m > -j) v += d(j - 1, mp - 1, m) * st * C(j + m, 1) * C(j - m, 1);
        d(j, mp, m) = v * ww / C(j + mp, 2);
      }
      double v = j * st * d(j - 1, mp - 1, 0);
      if (j > 1) v -= C(j, 2) * (d(j - 1, mp - 1, -1) * cp + d(j - 1, mp - 1, 1) * cn);
      d(j, mp, 0) = v * ww / C(j + mp, 2);
      for (int m = 1; m <= j; ++m) {
        double w = d(j - 1, mp - 1, m - 1) * cp * C(j + m, 2);
        if (m < j - 1) w -= d(j - 1, mp - 1, m + 1) * cn * C(j - m, 2);
        if (m < j) w += d(j - 1, mp - 1, m) * st * C(j + m, 1) * C(j - m, 1);
        d(j, mp, m) = w * ww / C(j + mp, 2);
      }
    }
  }
  std::vector<double> f(2 * nt + 1);
  f[0] = 1.0;
  for (int n = 1; n <= 2 * nt; ++n) f[n] = f[n - 1] * n;
  for (int n = 0; n <= nt; ++n)
    for (int m = 0; m <= n; ++m)
      for (int mp = -n; mp <= n; ++mp) {
        const int a = mp < 0 ? -mp : mp;
        d(n, m, mp) *= std::sqrt(f[n + m] / f[n + a] * f[n - a] / f[n - m]);
      }
}

void legendre_gt1(int nmax, double scal, double x, std::vector<double>& y) {
  y.assign((size_t)(nmax + 1) * (nmax + 2) / 2, 0.0);
  const double v = scal * x, w = scal * scal, u = std::sqrt(x * x - 1.0) * scal;
  auto T = [](int n, int m) { return m + n * (n + 1) / 2; };
  y[0] = 1.0;
  for (int m = 0; m <= nmax; ++m) {
    if (m > 0) y[T(m, m)] = y[T(m - 1, m - 1)] * u * double(2 * m - 1);
    if (m < nmax) y[T(m + 1, m)] = double(2 * m + 1) * v * y[T(m, m)];
    for (int n = m + 2; n <= nmax; ++n)
      y[T(n, m)] = ((2.0 * n - 1.0) * v * y[T(n - 1, m)] - double(n + m - 1) * w * y[T(n - 2, m)]) / double(n - m);
  }
}

}  // namespace

void yarvin_rokhlin(int nt, std::vector<double>& x, std::vector<double>& w, std::vector<int>& numfour,
                    std::vector<int>& numphys) {
  if (nt == 9) {
    x = {.099273996739714473469540223504736787, .47725674637049431137114652301534079,
         1.0553366138218296388373573790886439, 1.7675934335400844688024335482623428,
         2.5734262935147067530294862081063911, 3.4482433920158257478760788217186928,
         4.3768098355472631055818055756390095, 5.3489575720546005399569367000367492,
         6.3576578531337464283978988532908261};
    w = {.24776441819008371281185532097879332, .49188566500464336872511239562300034,
         .65378749137677805158830324216978624, .76433038408784093054038066838984378,
         .84376180565628111640563702167128213, .90445883985098263213586733400006779,
         .9537861313683345665381807521043811, .99670261613218547047665651916759089,
         1.0429422730252668749528766056755558};
    numfour = {2, 4, 4, 6, 6, 4, 6, 4, 2};
    numphys = {4, 8, 12, 16, 20, 20, 24, 8, 2};
  } else if (nt == 18) {
    x = {.052788527661177607475107009804560221, .26949859838931256028615734976483509,
         .6322035317468939208396250251098536, 1.1130756427760852833586113774799742,
         1.6893949614021379623807206371566281, 2.3437620046953044905535534780938178,
         3.0626998290780611533534738555317745, 3.8356294126529686394633245072327554,
         4.6542473432156272750148673367220908, 5.5120938659358147404532246582675725,
         6.4042126837727888499784967279992998, 7.3268800190617540124549122992902994,
         8.2774009925823861522076185792684555, 9.2539718060248947750778825138695538,
         10.255602723746401139237605093512684, 11.282088297877740146191172243561596,
         12.334067909676926788620221486780792, 13.414920240172401477707353478763252};
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

void GlobalTables::build(int nterms) {
  nt = nterms;
  rotation(nt, kPi / 2.0, rdpi2);
  rotation(nt, -kPi / 2.0, rdmpi2);
  rotation(nt, std::acos(std::sqrt(3.0) / 3.0), rdsq3);
  rotation(nt, std::acos(-std::sqrt(3.0) / 3.0), rdmsq3);
  std::vector<double> f(2 * nt + 1);
  f[0] = 1.0;
  for (int l = 1; l <= 2 * nt; ++l) f[l] = f[l - 1] * l;
  scale_factors.assign((size_t)(nt + 1) * (nt + 2) / 2, 0.0);
  for (int l = 0; l <= nt; ++l)
    for (int m = 0; m <= l; ++m) scale_factors[m + l * (l + 1) / 2] = f[l - m] / f[l + m] * double(2 * l + 1);
}

static void shift_coefficients(int nt, bool multipole, double scal, double beta, double r0, std::vector<double>& c) {
  std::vector<double> f(2 * nt + 1);
  f[0] = 1.0;
  for (int n = 1; n <= 2 * nt; ++n) f[n] = f[n - 1] * n;
  const double r0k = r0 * beta;
  std::vector<double> bj(2 * nt + 2);
  bessel_in(r0k, r0k, 2 * nt, bj.data());
  c.assign((size_t)(nt + 1) * (nt + 1) * (nt + 1), 0.0);
  for (int m = 0; m <= nt; ++m)
    for (int a = m; a <= nt; ++a)
      for (int b = m; b <= nt; ++b) {
        double acc = 0.0;
        const int up = b <= a ? b : a;
        for (int k = m; k <= up; ++k) {
          const double pre = multipole ? std::pow(scal, b - a) * std::pow(2.0, -a - k) * (((a + b) % 2 == 0) ? 1.0 : -1.0)
                                       : std::pow(scal, a - b) * std::pow(2.0, -a - k);
          const double fac =
              double(2 * a + 1) * f[a - m] / f[k + m] * f[b + m] * f[2 * k] / f[k] / f[k - m] / f[a - k] / f[b - k];
          acc += pre * fac * bj[a + b - k] * std::pow(r0k, a + b - 2 * k);
        }
        c[((size_t)m * (nt + 1) + a) * (nt + 1) + b] = acc;
      }
}

void LevelTables::build(int nterms, double beta, int level, double edge) {
  nt = nterms;
  scale = fmm_scale(beta, edge, level);
  const double ledge = edge / (double)(1ull << level);
  betascal = beta * ledge / 2.0;
  yarvin_rokhlin(nt, nodes, weights, numfour, numphys);
  nl = (int)nodes.size();
  for (int i = 0; i < nl; ++i) {
    const double li = nodes[i];
    const double uu = std::sqrt(li * li + 2.0 * li * scale / 2.0);
    int indd = i, mmax = numphys[i];
    for (int j = i; j < nl; ++j) {
      if (uu <= nodes[j])
        indd = j;
      else if (numphys[j] > mmax)
        mmax = numphys[j];
    }
    numphys[i] = mmax > numphys[indd] ? mmax : numphys[indd];
  }
  nexptot = nexptotp = 0;
  for (int i = 0; i < nl; ++i) {
    nexptot += numfour[i];
    nexptotp += numphys[i];
  }
  nexptotp /= 2;
  fexpe.clear();
  fexpo.clear();
  fexpback.clear();
  for (int i = 0; i < nl; ++i) {
    const int na2 = numphys[i] / 2;
    const double ha = 2.0 * kPi / numphys[i];
    for (int j = 0; j < na2; ++j) {
      for (int mm = 2; mm <= numfour[i]; mm += 2) fexpe.push_back(std::polar(1.0, double(mm - 1) * ha * j));
      for (int mm = 3; mm <= numfour[i]; mm += 2) fexpo.push_back(std::polar(1.0, double(mm - 1) * ha * j));
    }
  }
  for (int i = 0; i < nl; ++i) {
    const int na2 = numphys[i] / 2;
    const double ha = 2.0 * kPi / numphys[i];
    for (int mm = 3; mm <= numfour[i]; mm += 2)
      for (int j = 0; j < na2; ++j) fexpback.push_back(std::polar(1.0, -double(mm - 1) * ha * j));
    for (int mm = 2; mm <= numfour[i]; mm += 2)
      for (int j = 0; j < na2; ++j) fexpback.push_back(std::polar(1.0, -double(mm - 1) * ha * j));
  }
  const int E = (nt + 1) * (nt + 2) / 2;
  rlsc.assign((size_t)E * nl, 0.0);
  std::vector<double> tmp;
  for (int l = 0; l < nl; ++l) {
    legendre_gt1(nt, scale / 2.0, nodes[l] / betascal + 1.0, tmp);
    for (int e = 0; e < E; ++e) rlsc[(size_t)e * nl + l] = tmp[e];
  }
  xs.assign(3 * (size_t)nexptotp, 0.0);
  ys = xs;
  zs.assign(3 * (size_t)nexptotp, 0.0);
  int ntot = 0;
  for (int l = 0; l < nl; ++l) {
    const double w1 = nodes[l] + betascal;
    const double w2 = std::sqrt(nodes[l] * (nodes[l] + betascal * 2.0));
    const double hu = 2.0 * kPi / double(numphys[l]);
    for (int mth = 0; mth < numphys[l] / 2; ++mth) {
      const int c = ntot + mth;
      const double u = hu * mth;
      zs[c] = std::exp(-w1);
      zs[nexptotp + c] = zs[c] * zs[c];
      zs[2 * nexptotp + c] = zs[nexptotp + c] * zs[c];
      xs[c] = std::polar(1.0, w2 * std::cos(u));
      xs[nexptotp + c] = xs[c] * xs[c];
      xs[2 * nexptotp + c] = xs[nexptotp + c] * xs[c];
      ys[c] = std::polar(1.0, w2 * std::sin(u));
      ys[nexptotp + c] = ys[c] * ys[c];
      ys[2 * nexptotp + c] = ys[nexptotp + c] * ys[c];
    }
    ntot += numphys[l] / 2;
  }
  shift_coefficients(nt, true, scale, beta, std::sqrt(3.0) * ledge / 2.0, mpshift);
  shift_coefficients(nt, false, scale, beta, std::sqrt(3.0) * ledge / 4.0, lcshift);
}

}  // namespace bp
