// Device generation of a mesh's node patches and point lists from a closed
// triangulated surface: the PN / PNG1 surface construction and the
// constant-basis quadrature of libBEEP's mesh preparation
// (Mesh::create_bezier_triangles / create_node_patches,
// src/bem/mesh.cpp:1632-1652; PNG1_Triangle, src/bem/png1.h:20-330;
// Triangle point generation, src/bem/triangle.h:232-475; BasicNodePatch,
// src/bem/node_patch.cpp:55-130, :198-273).  The topology (vertex normals,
// edge neighbours, anticlockwise triangle rings) is built on the host; then
//   pn_triangle_kernel  one thread per triangle: control net and curved area
//   pn_patch_kernel     one thread per node patch (vertex): its galerkin
//                       points and from them the patch centroid, normal and
//                       area; its qualocation and quadrature points
// write the device mesh's SoA point lists directly.  The surface math is
// pn_surface.h, the code the host preparation runs; this file is compiled
// without fused multiply-adds, so the points are bitwise the host's.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "engine.h"
#include "pn_surface.h"
#include "surface_topology.h"

namespace bp {
namespace {

using namespace pn;

__global__ void pn_triangle_kernel(int nt, Tri* __restrict__ T, int planar, double* __restrict__ curved) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  Tri tr = T[t];
  if (!planar) init_pn(tr);
  tr.curved_area = planar ? tr.planar_area : curved_area(tr);
  T[t] = tr;
  curved[t] = tr.curved_area;
}

// point k of a 7-array SoA list of stride n: x y z nx ny nz w
__device__ __forceinline__ void store_point(double* soa, int n, int k, V3 p, V3 nv, double w) {
  soa[k] = p.x;
  soa[(size_t)n + k] = p.y;
  soa[2 * (size_t)n + k] = p.z;
  soa[3 * (size_t)n + k] = nv.x;
  soa[4 * (size_t)n + k] = nv.y;
  soa[5 * (size_t)n + k] = nv.z;
  soa[6 * (size_t)n + k] = w;
}

// A node patch's points, in the order of the host preparation: galerkin
// points (4-point rule over the ring) give the area, the normal (the mean
// of the points' normals weighted by their weights) and the centroid; the
// qualocation points are the centroid (rule 0) or a rule over the ring with
// weights divided by the area; the quadrature points the centroid with the
// area as weight (rule 0) or a rule over the ring.
__global__ void pn_patch_kernel(int nv, const V3* __restrict__ V, const Tri* __restrict__ T,
                                const int32_t* __restrict__ ring_off, const int32_t* __restrict__ ring, int qual_rule,
                                int quad_rule, const int32_t* __restrict__ qual_off, double* __restrict__ qual, int nq,
                                const int32_t* __restrict__ quad_off, double* __restrict__ quad, int nd,
                                const int32_t* __restrict__ gal_off, double* __restrict__ gal, int ng,
                                double* __restrict__ centroid, double* __restrict__ normal, double* __restrict__ area,
                                int* __restrict__ bad) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const V3 ref = V[v];
  const int r0 = ring_off[v], r1 = ring_off[v + 1];
  const Rule gl4 = get_rule(4);
  V3 alt{0, 0, 0}, cen{0, 0, 0};
  double a = 0;
  int k = gal_off[v];
  bool ok = true;
  for (int r = r0; r < r1; ++r)
    ok = ok && constant_basis_points(T[ring[r]], ref, gl4, [&](V3 p, V3 n, double w) {
           store_point(gal, ng, k++, p, n, w);
           alt = alt + n * w;
           a += w;
           cen = cen + p * w;
         });
  const V3 nrm = unit(alt);
  cen = cen / a;
  k = qual_off[v];
  if (qual_rule == 0) {
    store_point(qual, nq, k, cen, nrm, 1.0);
  } else {
    const Rule rq = get_rule(qual_rule);
    for (int r = r0; r < r1; ++r)
      ok = ok && constant_basis_points(T[ring[r]], ref, rq,
                                       [&](V3 p, V3 n, double w) { store_point(qual, nq, k++, p, n, w / a); });
  }
  k = quad_off[v];
  if (quad_rule == 0) {
    store_point(quad, nd, k, cen, nrm, a);
  } else {
    const Rule rd = get_rule(quad_rule);
    for (int r = r0; r < r1; ++r)
      ok = ok && constant_basis_points(T[ring[r]], ref, rd,
                                       [&](V3 p, V3 n, double w) { store_point(quad, nd, k++, p, n, w); });
  }
  centroid[3 * (size_t)v] = cen.x;
  centroid[3 * (size_t)v + 1] = cen.y;
  centroid[3 * (size_t)v + 2] = cen.z;
  normal[3 * (size_t)v] = nrm.x;
  normal[3 * (size_t)v + 1] = nrm.y;
  normal[3 * (size_t)v + 2] = nrm.z;
  area[v] = a;
  if (!ok || !isfinite(a) || !isfinite(nrm.x)) atomicOr(bad, 1);
}

// CSR offsets of a point list: per vertex 2 points per rule point per ring
// triangle, or one point (rule 0)
std::vector<int32_t> point_offsets(const SurfaceTopology& topo, int rule_n) {
  std::vector<int32_t> off(1, 0);
  const int nv = (int)topo.vertices.size();
  long long total = 0;
  for (int v = 0; v < nv; ++v) {
    const int ring = topo.ring_off[v + 1] - topo.ring_off[v];
    total += rule_n == 0 ? 1 : 2LL * rule_n * ring;
    if (total > (1LL << 31) - 1) throw std::invalid_argument("too many points");
    off.push_back((int32_t)total);
  }
  return off;
}

}  // namespace
}  // namespace bp

using namespace bp;

extern "C" BP_API int32_t bp_mesh_create_from_surface(bp_ctx ctx, int32_t n_vertices, const double* vertices,
                                                      const double* vertex_normals, int32_t n_triangles,
                                                      const int32_t* triangles, int32_t planar, int32_t qual_rule,
                                                      int32_t quad_rule, const double centre[3], bp_mesh* out,
                                                      double* totals) {
  return guarded_engine([&]() -> int32_t {
    Ctx* c = reinterpret_cast<Ctx*>(ctx);
    if (!c || !vertices || !triangles || !centre || !out || n_vertices <= 0 || n_triangles <= 0)
      return fail(BP_ERR_INVALID, "bp_mesh_create_from_surface: bad argument");
    for (int r : {qual_rule, quad_rule})
      if (r != 0 && pn::get_rule(r).n == 0)
        return fail(BP_ERR_INVALID, "bp_mesh_create_from_surface: unsupported triangle rule " + std::to_string(r));
    for (long long i = 0; i < 3LL * n_vertices; ++i)
      if (!std::isfinite(vertices[i]) || (vertex_normals && !std::isfinite(vertex_normals[i])))
        return fail(BP_ERR_INVALID, "bp_mesh_create_from_surface: non-finite vertex data");
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(centre[k])) return fail(BP_ERR_INVALID, "bp_mesh_create_from_surface: non-finite centre");
    int dev_prev = -1;
    cudaGetDevice(&dev_prev);
    if (dev_prev != c->device) BP_CUDA(cudaSetDevice(c->device));
    struct Restore {
      int d;
      ~Restore() {
        if (d >= 0) cudaSetDevice(d);
      }
    } restore{dev_prev != c->device ? dev_prev : -1};
    SurfaceTopology topo;
    build_topology(n_vertices, vertices, vertex_normals, n_triangles, triangles, topo);
    const int nv = n_vertices, nt = n_triangles;
    auto m = std::make_unique<DevMesh>();
    m->ctx = c;
    m->live.attach(c->live_meshes);
    m->n = nv;
    for (int k = 0; k < 3; ++k) m->centre[k] = centre[k];
    m->h_qual_off = point_offsets(topo, qual_rule == 0 ? 0 : pn::get_rule(qual_rule).n);
    m->h_quad_off = point_offsets(topo, quad_rule == 0 ? 0 : pn::get_rule(quad_rule).n);
    m->h_gal_off = point_offsets(topo, 4);
    m->n_qual_pts = m->h_qual_off.back();
    m->n_quad_pts = m->h_quad_off.back();
    m->n_gal_pts = m->h_gal_off.back();
    cudaStream_t st = c->stream;
    DevBuf dV = upload(c, topo.vertices), dT = upload(c, topo.tris), d_ring_off = upload(c, topo.ring_off),
           d_ring = upload(c, topo.ring), d_qo = upload(c, m->h_qual_off), d_do = upload(c, m->h_quad_off),
           d_go = upload(c, m->h_gal_off);
    DevBuf d_curved(c, sizeof(double) * (size_t)nt), d_patch(c, sizeof(double) * 7 * (size_t)nv), d_bad(c, sizeof(int));
    m->d_qual.alloc(c, sizeof(double) * 7 * (size_t)m->n_qual_pts);
    m->d_quad.alloc(c, sizeof(double) * 7 * (size_t)m->n_quad_pts);
    m->d_gal.alloc(c, sizeof(double) * 7 * (size_t)m->n_gal_pts);
    BP_CUDA(cudaMemsetAsync(d_bad.get(), 0, sizeof(int), st));
    pn_triangle_kernel<<<(nt + 127) / 128, 128, 0, st>>>(nt, dT.as<pn::Tri>(), planar ? 1 : 0, d_curved.as<double>());
    BP_LAUNCH_CHECK();
    double* cen = d_patch.as<double>();
    pn_patch_kernel<<<(nv + 127) / 128, 128, 0, st>>>(
        nv, dV.as<pn::V3>(), dT.as<pn::Tri>(), d_ring_off.as<int32_t>(), d_ring.as<int32_t>(), qual_rule, quad_rule,
        d_qo.as<int32_t>(), m->d_qual.as<double>(), m->n_qual_pts, d_do.as<int32_t>(), m->d_quad.as<double>(),
        m->n_quad_pts, d_go.as<int32_t>(), m->d_gal.as<double>(), m->n_gal_pts, cen, cen + 3 * (size_t)nv,
        cen + 6 * (size_t)nv, d_bad.as<int>());
    BP_LAUNCH_CHECK();
    std::vector<double> h_patch(7 * (size_t)nv), h_curved(nt);
    int h_bad = 0;
    BP_CUDA(cudaMemcpyAsync(h_patch.data(), cen, sizeof(double) * h_patch.size(), cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaMemcpyAsync(h_curved.data(), d_curved.get(), sizeof(double) * nt, cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaMemcpyAsync(&h_bad, d_bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    if (h_bad) return fail(BP_ERR_INVALID, "bp_mesh_create_from_surface: degenerate surface (non-finite patch data)");
    m->h_centroid.assign(h_patch.begin(), h_patch.begin() + 3 * (size_t)nv);
    m->h_normal.assign(h_patch.begin() + 3 * (size_t)nv, h_patch.begin() + 6 * (size_t)nv);
    m->h_area.assign(h_patch.begin() + 6 * (size_t)nv, h_patch.end());
    m->h_gc.assign(nv, 0.5);
    if (totals) {
      double curved = 0, flat = 0;
      for (int t = 0; t < nt; ++t) {
        curved += h_curved[t];
        flat += topo.tris[t].planar_area;
      }
      totals[0] = curved;
      totals[1] = flat;
    }
    *out = reinterpret_cast<bp_mesh>(m.release());
    return BP_OK;
  });
}
