// Host BVH construction for the device meshes. It builds the node array of the
// reference's BVH::build (bvh/bvh.cpp:115-193): bounds of the triangles in the
// range, leaves of at most 4 triangles, a split on the longest axis at the
// midpoint of the triangle centroids, std::partition of the index range (whose
// element order the later splits and the leaf contents depend on), a split in
// half when all centroids fall on one side, and post-order emission so the root
// is the last node. Identical arrays mean identical traversal order on the GPU,
// hence bit-exact hit triangle ids.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "host.h"

namespace mupsi {
namespace {

struct Builder {
  const float* v;
  const int32_t* f;
  std::vector<uint32_t>& idx;
  std::vector<HostNode>& nodes;

  float centroid(uint32_t ti, int axis) const {
    const int32_t* t = f + 3 * (int64_t)ti;
    return (v[3 * (int64_t)t[0] + axis] + v[3 * (int64_t)t[1] + axis] + v[3 * (int64_t)t[2] + axis]) / 3.0f;
  }

  uint32_t build(uint32_t begin, uint32_t end) {
    uint32_t count = end - begin;
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = begin; i < end; ++i) {
      const int32_t* t = f + 3 * (int64_t)idx[i];
      float tmn[3] = {INFINITY, INFINITY, INFINITY}, tmx[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a) {
          float p = v[3 * (int64_t)t[c] + a];
          tmn[a] = std::min(tmn[a], p);
          tmx[a] = std::max(tmx[a], p);
        }
      for (int a = 0; a < 3; ++a) {
        mn[a] = std::min(mn[a], tmn[a]);
        mx[a] = std::max(mx[a], tmx[a]);
      }
    }
    if (count <= 4) {
      HostNode n;
      std::copy(mn, mn + 3, n.mn);
      std::copy(mx, mx + 3, n.mx);
      n.left = begin;
      n.right = count | 0x80000000u;
      nodes.push_back(n);
      return (uint32_t)nodes.size() - 1;
    }
    float d[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
    int axis = (d[0] > d[1] && d[0] > d[2]) ? 0 : (d[1] > d[2] ? 1 : 2);
    float smin = INFINITY, smax = -INFINITY;
    for (uint32_t i = begin; i < end; ++i) {
      float c = centroid(idx[i], axis);
      smin = std::min(smin, c);
      smax = std::max(smax, c);
    }
    float split = (smin + smax) * 0.5f;
    auto mid = std::partition(idx.begin() + begin, idx.begin() + end,
                              [&](uint32_t ti) { return centroid(ti, axis) < split; });
    uint32_t m = (uint32_t)(mid - idx.begin());
    if (m == begin || m == end) m = begin + count / 2;
    uint32_t l = build(begin, m);
    uint32_t r = build(m, end);
    HostNode n;
    std::copy(mn, mn + 3, n.mn);
    std::copy(mx, mx + 3, n.mx);
    n.left = l;
    n.right = r;
    nodes.push_back(n);
    return (uint32_t)nodes.size() - 1;
  }
};

}  // namespace

uint32_t build_bvh(const float* verts, const int32_t* faces, int64_t num_faces, std::vector<HostNode>& nodes,
                   std::vector<uint32_t>& tri_idx) {
  nodes.clear();
  tri_idx.resize(num_faces);
  if (num_faces == 0) return 0;
  for (int64_t i = 0; i < num_faces; ++i) tri_idx[i] = (uint32_t)i;
  nodes.reserve(2 * num_faces);
  Builder b{verts, faces, tri_idx, nodes};
  return b.build(0, (uint32_t)num_faces);
}

}  // namespace mupsi
