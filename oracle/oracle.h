// ORACLE -- test infrastructure only (see oracle.cpp).
#pragma once
#include <cstdint>

extern "C" {

struct OrPatches {
  int32_t n;
  const double* centroid;  // [n][3]
  const double* normal;    // [n][3]
  const double* area;      // [n]
  const double* eps;       // [n] dielectric ratio eps_solvent / eps_protein
  const double* gc;        // [n]
  const int32_t* qual_off;
  const double* qual;      // [.][7]
  const int32_t* quad_off;
  const double* quad;
  const int32_t* gal_off;
  const double* gal;
};

struct OrTree {
  int32_t n_nodes;
  int32_t n_levels;
  const int32_t* info;        // [n][18] as exported by bp_problem_tree
  const double* geom;         // [n][4] centre xyz, edge
  const int32_t* neighbours;  // [n][27] same-level neighbour node ids or -1
  const int32_t* contents;    // every node's patch ids, node after node
  int64_t n_contents;
};

struct OrNear;
typedef void (*or_matvec_fn)(void* user, const double* x, double* y);

void or_pair_coefficients(const OrPatches* P, int npairs, const int32_t* I, const int32_t* J, double kappa, int fp32,
                          double* out);
void or_singular(const OrPatches* P, double kappa, int fp32, double* out);
OrNear* or_near_create(const OrPatches* P, const OrTree* T, double kappa, int fp32);
void or_near_destroy(OrNear* nf);
int64_t or_near_count(const OrNear* nf);
void or_near_apply(const OrNear* nf, const double* x, double* y);
void or_point_sums(int n_patches, const int32_t* off, const double* pts, const double* xyzq, int nc, double scale,
                   double* out_a, double* out_b);
struct OrFmm;
OrFmm* or_fmm_create(const OrPatches* P, const OrTree* T, double kappa, double beta0, double edge, int nterms);
void or_fmm_destroy(OrFmm* F);
void or_fmm_apply(OrFmm* F, const double* x, double* y);
int or_interaction_list(int32_t* out);
void or_fmm_direct(const OrPatches* P, double kappa, double beta0, int npairs, const int32_t* T, const int32_t* S,
                   const double* x, double* y);
int or_gmres(or_matvec_fn mv, void* user, int n2, const double* b, double* x, double tol, int max_iters, int restart,
             double* rel_resid);
}
