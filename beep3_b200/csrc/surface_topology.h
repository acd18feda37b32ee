// Host-side topology of a closed triangulated surface, shared by the host
// preparation (geometry.cpp) and the device mesh generator (mesh_gen.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "pn_surface.h"

namespace bp {

struct SurfaceTopology {
  std::vector<pn::V3> vertices;
  // per triangle: vertices, planar area and normal, vertex normals (given
  // unit normals, else the area-weighted mean of the adjacent planar
  // normals, src/bem/vertex.cpp:79-122) and the planar normals of its edge
  // neighbours (src/bem/mesh.cpp:996-1003); no control net yet
  std::vector<pn::Tri> tris;
  // per vertex its triangles in anticlockwise ring order
  // (src/bem/vertex.cpp:124-176): ring[ring_off[v] .. ring_off[v + 1])
  std::vector<int32_t> ring_off, ring;
};

// Throws std::invalid_argument for an index out of range, an edge without
// exactly two triangles, or a vertex without triangles.
void build_topology(int nv, const double* verts, const double* vnormals, int nt, const int32_t* tris,
                    SurfaceTopology& out);

}  // namespace bp
