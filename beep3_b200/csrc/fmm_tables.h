// Plane-wave FMM tables computed on the host in FP64 (see fmm_tables.cpp).
#pragma once

#include <complex>
#include <vector>

namespace bp {

using cplx = std::complex<double>;

// i_n(x) / scal^n for n = 0..nb
void bessel_in(double scal, double x, int nb, double* b);

// One entry of the plane-wave interaction list of a parent node: the source
// is child `src` (0..7) of neighbour `nb` (0..26, 13 = the parent itself) of
// the parent, the target child `targ` (0..7) of the parent, (dx, dy, dz) the
// target's offset from the source in child boxes, dir the wave direction
// (0 up, 1 down, 2 north, 3 south, 4 east, 5 west).
struct RawInteraction {
  int nb, dir, targ, src, dx, dy, dz;
};
// The 1512 entries of the reference's table (src/fmm/interaction_list.h),
// generated from its rule instead of stored.
std::vector<RawInteraction> interaction_table();
// min(beta * edge, 1) / 2^level
double fmm_scale(double beta, double edge, int level);
void yarvin_rokhlin(int nt, std::vector<double>& x, std::vector<double>& w, std::vector<int>& numfour,
                    std::vector<int>& numphys);

struct GlobalTables {
  int nt = 0;
  // d(l, mp, m) at ((l*(nt+1) + mp)*(2nt+1) + m + nt)
  std::vector<double> rdpi2, rdmpi2, rdsq3, rdmsq3;
  std::vector<double> scale_factors;  // [tri(l, m)]
  void build(int nterms);
};

struct LevelTables {
  int nt = 0, nl = 0, nexptot = 0, nexptotp = 0;
  double scale = 0, betascal = 0;
  std::vector<double> nodes, weights;
  std::vector<int> numfour, numphys;
  std::vector<cplx> fexpe, fexpo, fexpback;
  std::vector<double> rlsc;        // [tri(n, m)][nl]
  std::vector<cplx> xs, ys;        // [3][nexptotp]
  std::vector<double> zs;          // [3][nexptotp]
  std::vector<double> mpshift;     // [m][a][b], multipole z-shift (child -> parent)
  std::vector<double> lcshift;     // [m][a][b], local z-shift (parent -> child)
  void build(int nterms, double beta, int level, double edge);
};

}  // namespace bp
