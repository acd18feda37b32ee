// PN / PNG1 surface patches shared by the host preparation (geometry.cpp)
// and the device mesh generator (mesh_gen.cu): vector helpers, triangle
// rules, the PNG1 control net and its point / normal / Jacobian, the curved
// area by subdivision, and the constant-basis points of a node patch.  Every
// function is the same code on both sides; the device side is compiled
// without fused multiply-adds, so both produce the same bits.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define BP_HD __host__ __device__
#else
#define BP_HD
#endif

namespace bp {
namespace pn {

struct V3 {
  double x, y, z;
};
BP_HD inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
BP_HD inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
BP_HD inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
BP_HD inline V3 operator*(double s, V3 a) { return {a.x * s, a.y * s, a.z * s}; }
BP_HD inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
BP_HD inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
BP_HD inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
BP_HD inline double len2(V3 a) { return dot(a, a); }
BP_HD inline double len(V3 a) { return sqrt(len2(a)); }
BP_HD inline V3 unit(V3 a) { return a / len(a); }
BP_HD inline bool same(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// Triangle rules on the unit parametric triangle, weights summing to one
// (src/bem/triangle.h:75-94).  Values of published symmetric rules (the
// 7-point digits as the reference truncates them, so that the point lists
// are its own).  n = 0 for an order without a rule.
struct Rule {
  int n;
  double x[7], y[7], w[7];
};
BP_HD inline Rule get_rule(int order) {
  Rule r{};
  auto set = [&r](int k, double x, double y, double w) {
    r.x[k] = x;
    r.y[k] = y;
    r.w[k] = w;
  };
  switch (order) {
    case 1:
      r.n = 1;
      set(0, 1. / 3., 1. / 3., 1.);
      break;
    case 4:
      r.n = 4;
      set(0, 1. / 3., 1. / 3., -0.56250000);
      set(1, 0.2, 0.6, 0.520833333333);
      set(2, 0.6, 0.2, 0.520833333333);
      set(3, 0.2, 0.2, 0.520833333333);
      break;
    case 6:
      r.n = 6;
      set(0, 0.659027622374092, 0.231933368553031, 1. / 6.);
      set(1, 0.659027622374092, 0.109039009072877, 1. / 6.);
      set(2, 0.231933368553031, 0.659027622374092, 1. / 6.);
      set(3, 0.231933368553031, 0.109039009072877, 1. / 6.);
      set(4, 0.109039009072877, 0.659027622374092, 1. / 6.);
      set(5, 0.109039009072877, 0.231933368553031, 1. / 6.);
      break;
    case 7:
      r.n = 7;
      set(0, 1. / 3., 1. / 3., 0.225);
      set(1, 0.05971587, 0.47014206, 0.132394153333333);
      set(2, 0.47014206, 0.05971587, 0.132394153333333);
      set(3, 0.47014206, 0.47014206, 0.132394153333333);
      set(4, 0.79742698, 0.10128650, 0.125939186666666);
      set(5, 0.10128650, 0.79742698, 0.125939186666666);
      set(6, 0.10128650, 0.10128650, 0.125939186666666);
      break;
    default:
      r.n = 0;
  }
  return r;
}

struct Tri {
  int vi[3];
  V3 v1, v2, v3;
  V3 n1, n2, n3;
  V3 n12{0, 0, 0}, n23{0, 0, 0}, n31{0, 0, 0};
  double planar_area;
  V3 planar_normal;
  bool curved = false;
  double curved_area = 0.0;

  // Two versions of one control point; blend(p, s) weights them (1-s)^2 : s^2.
  struct Pair {
    V3 a, b;
  };
  enum { E210, E120, E201, E021, E102, E012 };  // edge control points
  V3 b300, b030, b003;                          // corners
  Pair edge[6];
  Pair centre[3];  // edges v1-v2, v2-v3, v3-v1

  BP_HD static V3 blend(const Pair& p, double s) {
    const double x = 1.0 - s, xx = x * x, ss = s * s;
    return (xx * p.a + ss * p.b) / (ss + xx);
  }
  // edge control points: 210 / 120 blend along v, 201 / 102 along u,
  // 021 / 012 along w
  BP_HD V3 b210(double, double v, double) const { return blend(edge[E210], v); }
  BP_HD V3 b120(double, double v, double) const { return blend(edge[E120], v); }
  BP_HD V3 b201(double u, double, double) const { return blend(edge[E201], u); }
  BP_HD V3 b102(double u, double, double) const { return blend(edge[E102], u); }
  BP_HD V3 b021(double, double, double w) const { return blend(edge[E021], w); }
  BP_HD V3 b012(double, double, double w) const { return blend(edge[E012], w); }
  // centre control point: per edge, its pair weighted by the edge's two
  // barycentrics; the corners are nudged by 1e-6 so that no weight is 0/0
  BP_HD V3 b111(double u, double v, double w) const {
    const double eps = 1e-6;
    u += eps; v += eps; w += eps;
    double tot = u + v + w;
    u /= tot; v /= tot; w /= tot;
    double den = (u * v + u * w + v * w);
    double pre1 = u * w / den;
    V3 t1 = (1. - u) * w * centre[0].a + (1. - w) * u * centre[0].b;
    double d1 = w + u - (2. * u * w);
    double pre2 = u * v / den;
    V3 t2 = (1. - v) * u * centre[1].a + (1. - u) * v * centre[1].b;
    double d2 = u + v - (2. * u * v);
    double pre3 = v * w / den;
    V3 t3 = (1. - w) * v * centre[2].a + (1. - v) * w * centre[2].b;
    double d3 = w + v - (2. * v * w);
    return t1 * (pre1 / d1) + t2 * (pre2 / d2) + t3 * (pre3 / d3);
  }

  BP_HD V3 point(double u, double v) const {
    double w = 1.0 - u - v;
    if (!curved) return w * v1 + u * v2 + v * v3;
    return b300 * w * w * w + b030 * u * u * u + b003 * v * v * v + b210(u, v, w) * 3 * w * w * u +
           b120(u, v, w) * 3 * w * u * u + b201(u, v, w) * 3 * w * w * v + b021(u, v, w) * 3 * u * u * v +
           b102(u, v, w) * 3 * w * v * v + b012(u, v, w) * 3 * u * v * v + b111(u, v, w) * 6 * w * u * v;
  }
  BP_HD V3 dU(double u, double v, double w) const {
    return b030 * 3 * u * u - b300 * 3 * w * w + b120(u, v, w) * (6 * u * w - 3 * u * u) +
           b021(u, v, w) * 6 * u * v - b102(u, v, w) * 3 * v * v + b012(u, v, w) * 3 * v * v +
           b210(u, v, w) * (3 * w * w - 6 * w * u) - b201(u, v, w) * 6 * w * v +
           b111(u, v, w) * (6 * w * v - 6 * u * v);
  }
  BP_HD V3 dV(double u, double v, double w) const {
    return b003 * 3 * v * v - b300 * 3 * w * w - b120(u, v, w) * 3 * u * u + b021(u, v, w) * 3 * u * u +
           b102(u, v, w) * (6 * v * w - 3 * v * v) + b012(u, v, w) * 6 * v * u - b210(u, v, w) * 6 * w * u +
           b201(u, v, w) * (3 * w * w - 6 * w * v) + b111(u, v, w) * (6 * w * u - 6 * u * v);
  }
  BP_HD double jacobian(double u, double v) const {
    if (!curved) return 2.0 * planar_area;
    double w = 1.0 - u - v;
    V3 du = dU(u, v, w), dv = dV(u, v, w);
    double E = len2(du), F = dot(du, dv), G = len2(dv);
    return sqrt(E * G - F * F);
  }
  BP_HD V3 normal(double u, double v) const {
    if (!curved) return planar_normal;
    double w = 1.0 - u - v;
    return unit(cross(dU(u, v, w), dV(u, v, w)));
  }
};

struct BT {  // a plain planar triangle (vertices + planar normal)
  V3 v1, v2, v3, pn;
  BP_HD BT(V3 a, V3 b, V3 c) : v1(a), v2(b), v3(c) { pn = unit(cross(b - a, c - a)); }
};

// src/bem/png1.h:26-55
BP_HD inline void affine_between_planes(const BT& t1, const BT& t2, V3& t1_v3_in_t2, V3& t2_v3_in_t1) {
  V3 o1 = t1.v1, x1 = t1.v2 - o1;
  double s1 = len(x1);
  x1 = unit(x1);
  V3 y1 = unit(cross(t1.pn, x1));
  double dx1 = dot(t1.v3 - o1, x1), dy1 = dot(t1.v3 - o1, y1);
  V3 o2 = t2.v1, x2 = t2.v2 - o2;
  double s2 = len(x2);
  x2 = unit(x2);
  V3 y2 = unit(cross(t2.pn, x2));
  double dx2 = dot(t2.v3 - o2, x2), dy2 = dot(t2.v3 - o2, y2);
  t1_v3_in_t2 = o2 + (x2 * dx1 + y2 * dy1) * s2 / s1;
  t2_v3_in_t1 = o1 + (x1 * dx2 + y1 * dy2) * s1 / s2;
}

// src/bem/png1.h:57-78
BP_HD inline V3 affine_to_edge(const BT& t1, V3 a, V3 b, V3 nrm) {
  V3 x1 = t1.v2 - t1.v1;
  double s1 = len(x1);
  x1 = unit(x1);
  V3 y1 = unit(cross(t1.pn, x1));
  V3 rel = t1.v3 - t1.v1;
  double dx = dot(rel, x1), dy = dot(rel, y1);
  V3 x2 = b - a;
  double s2 = len(x2);
  x2 = unit(x2);
  V3 y2 = unit(cross(nrm, x2));
  return a + (x2 * dx + y2 * dy) * s2 / s1;
}

// src/bem/png1.h:118-123
BP_HD inline V3 project_and_rescale(V3 pt, V3 in_plane, V3 n) {
  V3 proj = pt + n * dot(n, in_plane - pt);
  V3 dir = unit(proj - in_plane);
  return in_plane + dir * (len(in_plane - pt) / 3.0);
}

// PNG1 control net of a triangle from its corner normals and the normals of
// its edge neighbours (src/bem/png1.h:80-160).  Each edge control point is
// the projection of the far corner of its edge into a corner's tangent
// plane (its version in that corner's plane) or that version carried into
// the tangent plane of the edge's other end by the affine map between the
// two corner triangles; the centre pairs are the corner triangles mapped
// onto each edge in the plane halfway between the triangle and its
// neighbour.
BP_HD inline void init_pn(Tri& t) {
  using P = Tri;
  t.curved = true;
  t.b300 = t.v1; t.b030 = t.v2; t.b003 = t.v3;
  Tri::Pair* e = t.edge;
  // versions in the tangent plane of the corner next to the control point
  e[P::E210].a = project_and_rescale(t.v2, t.v1, t.n1);
  e[P::E201].a = project_and_rescale(t.v3, t.v1, t.n1);
  e[P::E120].a = project_and_rescale(t.v1, t.v2, t.n2);
  e[P::E021].a = project_and_rescale(t.v3, t.v2, t.n2);
  e[P::E102].a = project_and_rescale(t.v1, t.v3, t.n3);
  e[P::E012].a = project_and_rescale(t.v2, t.v3, t.n3);
  // corner triangles of the control net, and the versions carried to the
  // other corner of each edge
  const BT c1(t.b300, e[P::E210].a, e[P::E201].a), c2(t.b030, e[P::E021].a, e[P::E120].a),
      c3(t.b003, e[P::E102].a, e[P::E012].a);
  affine_between_planes(c1, BT(e[P::E120].a, t.b030, e[P::E021].a), e[P::E021].b, e[P::E201].b);
  affine_between_planes(c2, BT(e[P::E012].a, t.b003, e[P::E102].a), e[P::E102].b, e[P::E120].b);
  affine_between_planes(c3, BT(e[P::E201].a, t.b300, e[P::E210].a), e[P::E210].b, e[P::E012].b);
  // centre pairs: the corner triangles on each side of an edge mapped onto
  // it in the plane halfway between the triangle and its edge neighbour
  const V3 Nt = t.planar_normal;
  const V3 a12 = unit(Nt + t.n12), a23 = unit(Nt + t.n23), a31 = unit(Nt + t.n31);
  t.centre[0].a = affine_to_edge(c1, e[P::E210].a, e[P::E120].a, a12);
  t.centre[0].b = affine_to_edge(BT(e[P::E120].a, t.b030, e[P::E021].a), e[P::E210].a, e[P::E120].a, a12);
  t.centre[1].a = affine_to_edge(c2, e[P::E021].a, e[P::E012].a, a23);
  t.centre[1].b = affine_to_edge(BT(e[P::E012].a, t.b003, e[P::E102].a), e[P::E021].a, e[P::E012].a, a23);
  t.centre[2].a = affine_to_edge(c3, e[P::E102].a, e[P::E201].a, a31);
  t.centre[2].b = affine_to_edge(BT(e[P::E201].a, t.b300, e[P::E210].a), e[P::E102].a, e[P::E201].a, a31);
}

// Curved area by successive subdivision until the increase falls below a
// relative tolerance (src/bem/png1.h:272-368).  Only the area is kept.
BP_HD inline double subdivided_area(const Tri& t, unsigned nsub) {
  double area = 0;
  double inc = 1.0 / (1 + nsub);
  for (unsigned vctr = 0; vctr <= nsub; ++vctr) {
    double u1 = 0.0, v1 = vctr * inc;
    double u3 = u1, v3 = v1 + inc;
    double w3 = 1.0 - u3 - v3;
    double w2 = w3, v2 = v1, u2 = 1.0 - w2 - v2;
    unsigned row = 2 * (nsub - vctr) + 1;
    while (row) {
      V3 a = t.point(u1, v1), b = t.point(u2, v2), c = t.point(u3, v3);
      area += 0.5 * len(cross(b - a, c - a));
      --row;
      double v4 = v3, u4 = u2;
      if (row) {
        V3 d = t.point(u4, v4);
        area += 0.5 * len(cross(d - b, c - b));
        --row;
        u1 = u2; v1 = v2;
        u3 = u4; v3 = v4;
        w3 = 1.0 - u3 - v3;
        w2 = w3; v2 = v1; u2 = 1.0 - w2 - v2;
      }
    }
  }
  return area;
}

BP_HD inline double curved_area(const Tri& t) {
  const double tol = 1e-6 * t.planar_area;
  unsigned n = 1;
  double a1 = subdivided_area(t, n), a2 = 0;
  while (true) {
    a2 = subdivided_area(t, ++n);
    if ((a2 - a1) <= tol) break;
    if (n > 5) break;
    a1 = a2;
  }
  return a2;
}

// Constant-basis points of triangle t for the patch centred on vertex `ref`
// (src/bem/triangle.h:388-475 with the subdivides=0 parametric rule of
// :232-330), emitted as emit(point, normal, weight).  Every parametric
// sub-triangle is 1/6 of the unit triangle so a parametric weight is
// rule_w/6 before the surface Jacobian.  False when ref is not a vertex of t.
template <typename Emit>
BP_HD inline bool constant_basis_points(const Tri& t, V3 ref, const Rule& rule, Emit&& emit) {
  const double c3 = 1. / 3.;
  V3 centre{c3, c3, c3}, origin, mid1, mid2;
  if (same(ref, t.v1)) {
    origin = {0, 0, 1}; mid1 = {0.5, 0, 0.5}; mid2 = {0, 0.5, 0.5};
  } else if (same(ref, t.v2)) {
    origin = {1, 0, 0}; mid1 = {0.5, 0.5, 0}; mid2 = {0.5, 0, 0.5};
  } else if (same(ref, t.v3)) {
    origin = {0, 1, 0}; mid1 = {0, 0.5, 0.5}; mid2 = {0.5, 0.5, 0};
  } else {
    return false;
  }
  const BT subs[2] = {BT(centre, origin, mid1), BT(mid2, origin, centre)};
  const double norm = 2.0 / sqrt(3.0);
  for (int si = 0; si < 2; ++si) {
    const BT& s = subs[si];
    double sub_area = 0.5 * len(cross(s.v2 - s.v1, s.v3 - s.v1));
    for (int k = 0; k < rule.n; ++k) {
      // point on the unit barycentric triangle is (u, v, 1-u-v); map through
      // the sub-triangle: w*v1 + u*v2 + v*v3
      double u = rule.x[k], v = rule.y[k];
      double w = 1.0 - u - v;
      V3 q = w * s.v1 + u * s.v2 + v * s.v3;
      double wt = (rule.w[k] * sub_area) * norm;
      wt *= t.jacobian(q.x, q.y) / 2.0;
      emit(t.point(q.x, q.y), t.normal(q.x, q.y), wt);
    }
  }
  return true;
}

}  // namespace pn
}  // namespace bp
