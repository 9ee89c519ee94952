// Rays, spheres, BVH traversal, camera and BSDF sampling on the device.
// Each routine follows the reference function cited beside it operation for
// operation (the library is built without FMA contraction), so hit triangle ids
// and BVH results are bit-exact and the float results equal the reference's.
#pragma once
#include "dmath.cuh"

#define LEAF_FLAG 0x80000000u
#define BVH_STACK 64  // the reference's fixed traversal stack (bvh.cpp:201)

// BVH::Node: AABB (min, max) + left/right|LEAF_FLAG, 32 bytes (bvh/bvh.h:26-36)
struct __align__(16) BNode {
  float mn[3];
  float mx[3];
  uint32_t left, right;
};

struct Ray {
  v3 o, d;
  float nt, ft;
};
// Ray(origin, direction) normalizes the direction (geometry/ray.h:12)
MD Ray make_ray(v3 o, v3 d) {
  Ray r;
  r.o = o;
  r.d = normalized(d);
  r.nt = 0.0f;
  r.ft = 3.402823466e+38f;  // FLT_MAX
  return r;
}

// Device view of one mesh and its BVH (primitives/mesh.h, bvh/bvh.h)
struct DMesh {
  const BNode* nodes;
  const uint32_t* tri_idx;
  // the triangles in leaf order (entry i is triangle tri_idx[i]): 3 float4 per
  // entry holding its three vertices and, in the last word but two, its id, so a
  // leaf reads its triangles with independent 16-byte loads instead of
  // index -> face -> vertex chains
  const float4* soup;
  const int32_t* faces;   // [F*3]
  const float* verts;     // [V*3]
  const float* face_n;    // [F*3]
  const float* vert_n;    // nullable [V*3]
  const float* cdf;       // area CDF [F]
  int64_t num_nodes, num_faces;
  uint32_t root;
  uint32_t occl_start;    // first node of BVH::occluded: occl_ref as the reference, or root
  uint32_t occl_ref;      // device position of the reference's node 0 (its post-order first leaf)
  float total_area;
  m4 T, Tinv;
  int identity;           // Tinv.isIdentity()
  int normal_identity;    // normal transform (Tinv^T 3x3) is identity
  // nullable: BVH work counters (instrumentation), kBvhCountSlots pairs of
  // (nodes loaded, triangles tested); set only while a scene counts its work
  unsigned long long* count;
  // nullable: the same tree four wide (WNode), for the closest-point queries
  // whose answer does not depend on the tree's shape (bvh_closest_lowtie)
  const float4* wide;
  uint32_t wide_root;
};

// A node of the four-wide tree: the boxes of up to four children of the
// binary tree (two or three of its levels collapsed), as 16-byte rows
// lo.x[4], lo.y[4], lo.z[4], hi.x[4], hi.y[4], hi.z[4], child[4], unused[4]:
// one 128-byte read per visit. child: a node index, or W_LEAF | count << 28 |
// first leaf-order slot; an unused slot has an empty box (lo = +inf, hi = -inf).
constexpr uint32_t W_LEAF = 0x80000000u;
constexpr int kWideRows = 8;  // float4 rows per node

// BVH work tallies of one traversal: every node load (32 bytes) and every
// triangle tested (its 48-byte leaf-order record). CNT = false
// compiles to nothing; the counted copies of the traversals run only while a
// scene's profiling asks for BVH counts (the uncounted code is unchanged).
constexpr int kBvhCountSlots = 64;
template <bool CNT>
struct BvhTally {
  MD void node(uint32_t = 1) {}
  MD void tri() {}
  MD void flush(const DMesh&) {}
};
template <>
struct BvhTally<true> {
  uint32_t n = 0, t = 0;
  MD void node(uint32_t k = 1) { n += k; }
  MD void tri() { ++t; }
  MD void flush(const DMesh& m) {
    if (m.count && (n | t)) {  // spread over slots: fewer same-address atomics
      unsigned long long* c = m.count + 2 * (blockIdx.x % kBvhCountSlots);
      atomicAdd(c, (unsigned long long)n);
      atomicAdd(c + 1, (unsigned long long)t);
    }
    n = t = 0;
  }
};

MD v3 vert(const DMesh& m, int32_t i) { return ld3(m.verts + 3 * (int64_t)i); }
// Leaf-order entry i: the triangle's id and vertices (the same floats as
// verts[faces[3 id + k]]).
MD uint32_t leaf_tri(const DMesh& m, uint32_t i, v3& a, v3& b, v3& c) {
  const float4* q = m.soup + 3 * (int64_t)i;
  const float4 x = __ldg(q), y = __ldg(q + 1), z = __ldg(q + 2);
  a = mk3(x.x, x.y, x.z);
  b = mk3(x.w, y.x, y.y);
  c = mk3(y.z, y.w, z.x);
  return __float_as_uint(z.y);
}

// AABB::intersect slab test (bvh/boudingbox.cpp:6-38)
MD bool aabb_hit(const BNode& b, const Ray& r) {
  float tmin = -INFINITY, tmax = INFINITY;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float d = get(r.d, a), o = get(r.o, a);
    if (fabsf(d) > 1e-8f) {
      float t1 = (b.mn[a] - o) / d;
      float t2 = (b.mx[a] - o) / d;
      tmin = fmax_std(tmin, fmin_std(t1, t2));
      tmax = fmin_std(tmax, fmax_std(t1, t2));
    } else if (o < b.mn[a] || o > b.mx[a]) {
      return false;
    }
  }
  return tmax >= tmin && tmax >= r.nt && tmin <= r.ft;
}

// Moller-Trumbore (bvh.cpp:82-111)
MD bool ray_tri(const Ray& r, v3 v0, v3 v1, v3 v2, float& t, float& u, float& v) {
  v3 e1 = v1 - v0, e2 = v2 - v0;
  v3 h = cross(r.d, e2);
  float a = dot(e1, h);
  if (fabsf(a) < 1e-8f) return false;
  float f = 1.0f / a;
  v3 s = r.o - v0;
  u = f * dot(s, h);
  if (u < 0.0f || u > 1.0f) return false;
  v3 q = cross(s, e1);
  v = f * dot(r.d, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  t = f * dot(e2, q);
  return t > r.nt && t < r.ft;
}

MD BNode load_node(const BNode* nodes, uint32_t i) {
  const float4* p = reinterpret_cast<const float4*>(nodes + i);
  float4 a = __ldg(p), b = __ldg(p + 1);
  BNode n;
  n.mn[0] = a.x;
  n.mn[1] = a.y;
  n.mn[2] = a.z;
  n.mx[0] = a.w;
  n.mx[1] = b.x;
  n.mx[2] = b.y;
  n.left = __float_as_uint(b.z);
  n.right = __float_as_uint(b.w);
  return n;
}
// The device node array keeps every inner node's two children side by side
// at (left, left + 1) with left even (mesh upload re-lays the reference's
// post-order array out breadth first): one 64-byte read loads both.
MD BNode unpack_node(float4 a, float4 b) {
  BNode n;
  n.mn[0] = a.x;
  n.mn[1] = a.y;
  n.mn[2] = a.z;
  n.mx[0] = a.w;
  n.mx[1] = b.x;
  n.mx[2] = b.y;
  n.left = __float_as_uint(b.z);
  n.right = __float_as_uint(b.w);
  return n;
}
MD void load_pair(const BNode* nodes, uint32_t left, BNode& l, BNode& r) {
  const float4* p = reinterpret_cast<const float4*>(nodes + left);
  const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
  l = unpack_node(a, b);
  r = unpack_node(c, d);
}
MD int node_axis(const BNode& b) {
  float d0 = b.mx[0] - b.mn[0], d1 = b.mx[1] - b.mn[1], d2 = b.mx[2] - b.mn[2];
  return (d0 > d1 && d0 > d2) ? 0 : (d1 > d2 ? 1 : 2);
}
MD float node_centroid(const BNode& b, int a) { return (b.mn[a] + b.mx[a]) * 0.5f; }

// BVH::intersect (bvh.cpp:197-250): closest hit, front-to-back by child centroid
// along the parent's longest axis; narrows r.ft. `overflow` is set if the
// traversal would exceed the reference's 64-entry stack.
template <bool CNT = false>
MD bool bvh_intersect_inl(const DMesh& m, Ray& r, uint32_t& tri, float& uu, float& vv, bool& overflow) {
  if (m.num_nodes == 0) return false;
  BvhTally<CNT> tl;
  bool hit = false;
  uint32_t st[BVH_STACK];
  int sp = 0;
  st[sp++] = m.root;
  while (sp > 0) {
    BNode nd = load_node(m.nodes, st[--sp]);
    tl.node();
    if (!aabb_hit(nd, r)) continue;
    if (nd.right & LEAF_FLAG) {
      uint32_t start = nd.left, cnt = nd.right & ~LEAF_FLAG;
      for (uint32_t i = start; i < start + cnt; ++i) {
        tl.tri();
        v3 a, b, c;
        const uint32_t ti = leaf_tri(m, i, a, b, c);
        float t, u, v;
        if (ray_tri(r, a, b, c, t, u, v)) {
          r.ft = t;
          tri = ti;
          uu = u;
          vv = v;
          hit = true;
        }
      }
    } else {
      BNode ln, rn;
      load_pair(m.nodes, nd.left, ln, rn);
      tl.node(2);
      int axis = node_axis(nd);
      float lc = node_centroid(ln, axis), rc = node_centroid(rn, axis);
      bool near_first = (get(r.d, axis) > 0) ? (lc < rc) : (lc > rc);
      if (sp + 2 > BVH_STACK) {
        overflow = true;
        tl.flush(m);
        return hit;
      }
      st[sp++] = near_first ? nd.right : nd.left;
      st[sp++] = near_first ? nd.left : nd.right;
    }
  }
  tl.flush(m);
  return hit;
}

// BVH::occluded (bvh.cpp:254-300). The reference starts this traversal at node 0,
// which is the first leaf of the post-order array, not the root (bvh.cpp:259);
// that behaviour is the default so shadow rays agree with the reference, and
// MUPSI_OCCLUSION_ROOT (occl_start = root) switches to the full traversal.
MD bool bvh_occluded(const DMesh& m, const Ray& r, bool& overflow) {
  if (m.num_nodes == 0) return false;
  uint32_t st[BVH_STACK];
  int sp = 0;
  st[sp++] = m.occl_start;
  while (sp > 0) {
    BNode nd = load_node(m.nodes, st[--sp]);
    if (!aabb_hit(nd, r)) continue;
    if (nd.right & LEAF_FLAG) {
      uint32_t start = nd.left, cnt = nd.right & ~LEAF_FLAG;
      for (uint32_t i = start; i < start + cnt; ++i) {
        v3 a, b, c;
        leaf_tri(m, i, a, b, c);
        float t, u, v;
        if (ray_tri(r, a, b, c, t, u, v)) return true;
      }
    } else {
      BNode ln, rn;
      load_pair(m.nodes, nd.left, ln, rn);
      int axis = node_axis(nd);
      float lc = node_centroid(ln, axis), rc = node_centroid(rn, axis);
      bool near_first = (get(r.d, axis) > 0) ? (lc < rc) : (lc > rc);
      if (sp + 2 > BVH_STACK) {
        overflow = true;
        return false;
      }
      st[sp++] = near_first ? nd.right : nd.left;
      st[sp++] = near_first ? nd.left : nd.right;
    }
  }
  return false;
}

// std::max({a, 0, b}) as max_element over the list
MD float max3_il(float a, float b, float c) {
  float m = a;
  if (m < b) m = b;
  if (m < c) m = c;
  return m;
}
// dist2ToAABB (bvh.cpp:20-25)
MD float dist2_aabb(v3 p, const BNode& b) {
  float dx = max3_il(b.mn[0] - p.x, 0.0f, p.x - b.mx[0]);
  float dy = max3_il(b.mn[1] - p.y, 0.0f, p.y - b.mx[1]);
  float dz = max3_il(b.mn[2] - p.z, 0.0f, p.z - b.mx[2]);
  return dx * dx + dy * dy + dz * dz;
}
// dist2ToLine (bvh.cpp:27-40)
MD float dist2_line(v3 p, v3 a, v3 b, v3& out) {
  v3 ab = b - a, ap = p - a;
  if (sqn(ab) < 1e-6f) {
    out = a;
    return sqn(ap);
  }
  float d = dot(ap, ab);
  float t = d / sqn(ab);
  t = t < 0.0f ? 0.0f : (1.0f < t ? 1.0f : t);
  v3 proj = a + t * ab;
  out = proj;
  return sqn(p - proj);
}
// dist2ToTriangle (bvh.cpp:42-80)
MD float dist2_tri(v3 p, v3 a, v3 b, v3 c, v3& out) {
  v3 e1 = a - b, e2 = a - c;
  v3 n = cross(e1, e2);
  if (sqn(n) < 1e-6f) {
    out = a;
    return sqn(p - a);
  }
  n = normalized(n);
  float dp = dot(p - a, n);
  v3 pj = p - dp * n;
  v3 ab = -e1, bc = c - b, ca = e2;
  v3 c1 = cross(ab, pj - a), c2 = cross(bc, pj - b), c3 = cross(ca, pj - c);
  if (dot(c1, n) >= 0 && dot(c2, n) >= 0 && dot(c3, n) >= 0) {
    out = pj;
    return dp * dp;
  }
  float mn = INFINITY, d;
  v3 tmp;
  if ((d = dist2_line(p, a, b, tmp)) < mn) {
    mn = d;
    out = tmp;
  }
  if ((d = dist2_line(p, b, c, tmp)) < mn) {
    mn = d;
    out = tmp;
  }
  if ((d = dist2_line(p, c, a, tmp)) < mn) {
    mn = d;
    out = tmp;
  }
  return mn;
}
// BVH::closest (bvh.cpp:302-353): returns sqrt of the squared distance.
// best_init (FLT_MAX in the reference) may be any value above the true squared
// distance: boxes farther than it are pruned from the start and the same
// minimum is found (`found` reports whether a triangle beat best_init).
// LOWTIE: prune only boxes strictly farther than the best and take the lowest
// triangle index among equal distances, the rule of the lane-group query
// (bvh_closest_group): the same triangle and closest point as that query for
// any group size. Without it the reference's rule (first found wins).
template <bool CNT = false, bool LOWTIE = false>
MD float bvh_closest_inl(const DMesh& m, v3 p, uint32_t& tri, v3& q, bool& overflow,
                         float best_init = 3.402823466e+38f, bool* found = nullptr) {
  if (m.num_nodes == 0) return 0.0f;
  BvhTally<CNT> tl;
  uint32_t st[BVH_STACK];
  int sp = 0;
  st[sp++] = m.root;
  float best = best_init;
  if (found) *found = false;
  uint32_t btri = 0xffffffffu;
  // a box is kept while its distance is below the best (at or below it: LOWTIE)
  auto keep = [&](float db) { return LOWTIE ? !(db > best) : db < best; };
  while (sp > 0) {
    BNode nd = load_node(m.nodes, st[--sp]);
    tl.node();
    if (!keep(dist2_aabb(p, nd))) continue;
    if (nd.right & LEAF_FLAG) {
      uint32_t start = nd.left, cnt = nd.right & ~LEAF_FLAG;
      for (uint32_t i = start; i < start + cnt; ++i) {
        tl.tri();
        v3 a, b, c, tmp;
        const uint32_t ti = leaf_tri(m, i, a, b, c);
        float d = dist2_tri(p, a, b, c, tmp);
        if (d < best || (LOWTIE && d == best && d < best_init && ti < btri)) {
          best = d;
          tri = ti;
          btri = ti;
          q = tmp;
          if (found) *found = true;
        }
      }
    } else {
      BNode ln, rn;
      load_pair(m.nodes, nd.left, ln, rn);
      tl.node(2);
      float dl = dist2_aabb(p, ln), dr = dist2_aabb(p, rn);
      if (sp + 2 > BVH_STACK) {
        overflow = true;
        break;
      }
      if (dl < dr) {
        if (keep(dr)) st[sp++] = nd.right;
        if (keep(dl)) st[sp++] = nd.left;
      } else {
        if (keep(dl)) st[sp++] = nd.left;
        if (keep(dr)) st[sp++] = nd.right;
      }
    }
  }
  tl.flush(m);
  return sqrtf(best);
}

// BVH::closest over the four-wide tree with the lane-group rule (LOWTIE of
// bvh_closest_inl): boxes farther than the best are pruned, equal ones kept,
// and among triangles at the best distance the lowest index wins, so the
// triangle and point found do not depend on the tree's shape: they are the
// binary tree's. Its boxes are the binary tree's boxes, with the same
// distance arithmetic. Stack entries carry their box distance, so a popped
// entry is pruned without reloading its node.
template <bool CNT = false>
MD float bvh4_closest_inl(const DMesh& m, v3 p, uint32_t& tri, v3& q, bool& overflow, float best_init, bool* found) {
  BvhTally<CNT> tl;
  uint32_t sr[BVH_STACK];
  float sd[BVH_STACK];
  int sp = 0;
  sr[0] = m.wide_root;
  sd[0] = 0.0f;
  sp = 1;
  float best = best_init;
  if (found) *found = false;
  uint32_t btri = 0xffffffffu;
  while (sp > 0) {
    --sp;
    const uint32_t ref = sr[sp];
    if (sd[sp] > best) continue;
    if (ref & W_LEAF) {
      const uint32_t start = ref & 0x0fffffffu, cnt = (ref >> 28) & 7u;
      for (uint32_t i = start; i < start + cnt; ++i) {
        tl.tri();
        v3 a, b, c, tmp;
        const uint32_t ti = leaf_tri(m, i, a, b, c);
        const float d = dist2_tri(p, a, b, c, tmp);
        if (d < best || (d == best && d < best_init && ti < btri)) {
          best = d;
          tri = ti;
          btri = ti;
          q = tmp;
          if (found) *found = true;
        }
      }
      continue;
    }
    const float4* np = m.wide + (size_t)kWideRows * ref;
    const float4 lx = __ldg(np), ly = __ldg(np + 1), lz = __ldg(np + 2);
    const float4 hx = __ldg(np + 3), hy = __ldg(np + 4), hz = __ldg(np + 5);
    const uint4 ch = __ldg(reinterpret_cast<const uint4*>(np + 6));
    tl.node(4);
    // the four children's distances, as dist2_aabb forms them
    auto d2 = [&](float ax, float ay, float az, float bx, float by, float bz) {
      const float dx = max3_il(ax - p.x, 0.0f, p.x - bx);
      const float dy = max3_il(ay - p.y, 0.0f, p.y - by);
      const float dz = max3_il(az - p.z, 0.0f, p.z - bz);
      return dx * dx + dy * dy + dz * dz;
    };
    float dd[4] = {d2(lx.x, ly.x, lz.x, hx.x, hy.x, hz.x), d2(lx.y, ly.y, lz.y, hx.y, hy.y, hz.y),
                   d2(lx.z, ly.z, lz.z, hx.z, hy.z, hz.z), d2(lx.w, ly.w, lz.w, hx.w, hy.w, hz.w)};
    uint32_t cr[4] = {ch.x, ch.y, ch.z, ch.w};
    // kept children pushed farthest first, so the nearest is popped next
    // (a sorting network on the four; pruned ones sort to the end as +inf)
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (dd[k] > best) dd[k] = INFINITY;
    auto cs = [&](int a, int b) {
      if (dd[b] > dd[a]) {
        const float t = dd[a];
        dd[a] = dd[b];
        dd[b] = t;
        const uint32_t u = cr[a];
        cr[a] = cr[b];
        cr[b] = u;
      }
    };
    cs(0, 1);
    cs(2, 3);
    cs(0, 2);
    cs(1, 3);
    cs(1, 2);
    if (sp + 4 > BVH_STACK) {
      overflow = true;
      break;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (dd[k] != INFINITY) {
        sr[sp] = cr[k];
        sd[sp] = dd[k];
        ++sp;
      }
  }
  tl.flush(m);
  return sqrtf(best);
}

// The traversals out of line: every kernel carries one copy of each instead of
// one per query site. The mesh-mean march, whose warps otherwise stall on
// instruction fetch, renders a level-6 mesh at 512x512x4 in 227 ms instead of
// 358; the field march's sphere tracer keeps them inline (_inl: 224 ms
// against 304 ms out of line for its mesh SDF).
// The counted copies (bvh_*_counted) run instead while m.count is set.
static __device__ __noinline__ bool bvh_intersect_counted(const DMesh& m, Ray& r, uint32_t& tri, float& uu,
                                                          float& vv, bool& overflow) {
  return bvh_intersect_inl<true>(m, r, tri, uu, vv, overflow);
}
static __device__ __noinline__ float bvh_closest_counted(const DMesh& m, v3 p, uint32_t& tri, v3& q, bool& overflow,
                                                         float best_init, bool* found) {
  return bvh_closest_inl<true>(m, p, tri, q, overflow, best_init, found);
}
static __device__ __noinline__ bool bvh_intersect(const DMesh& m, Ray& r, uint32_t& tri, float& uu, float& vv,
                                                  bool& overflow) {
  if (m.count) return bvh_intersect_counted(m, r, tri, uu, vv, overflow);
  return bvh_intersect_inl(m, r, tri, uu, vv, overflow);
}
static __device__ __noinline__ float bvh_closest(const DMesh& m, v3 p, uint32_t& tri, v3& q, bool& overflow,
                                                 float best_init = 3.402823466e+38f, bool* found = nullptr) {
  if (m.count) return bvh_closest_counted(m, p, tri, q, overflow, best_init, found);
  return bvh_closest_inl(m, p, tri, q, overflow, best_init, found);
}
// One lane's closest-point query with the lane-group rule (LOWTIE).
// (The four-wide tree when the mesh has one: the same triangle and point.)
static __device__ __noinline__ float bvh_closest_lowtie(const DMesh& m, v3 p, uint32_t& tri, v3& q, bool& overflow,
                                                        float best_init, bool* found) {
  if (m.wide) {
    if (m.count) return bvh4_closest_inl<true>(m, p, tri, q, overflow, best_init, found);
    return bvh4_closest_inl<false>(m, p, tri, q, overflow, best_init, found);
  }
  if (m.count) return bvh_closest_inl<true, true>(m, p, tri, q, overflow, best_init, found);
  return bvh_closest_inl<false, true>(m, p, tri, q, overflow, best_init, found);
}

// Mesh::inside (mesh.cpp:341-362): parity of crossings of a +x ray from p,
// repeating BVH::intersect with nearT = last t + 1e-4 until a miss.
// INL: the inline traversal (the field march).
template <bool INL = false>
MD bool mesh_inside(const DMesh& m, v3 p, bool& overflow) {
  v3 pl = apply4(m.Tinv, p);
  Ray r = make_ray(pl, mk3(1.0f, 0.0f, 0.0f));
  uint32_t tri;
  float u, v;
  int hits = 0;
  auto isect = [&]() { return INL ? bvh_intersect_inl(m, r, tri, u, v, overflow) : bvh_intersect(m, r, tri, u, v, overflow); };
  if (isect()) {
    ++hits;
    // each crossing strictly increases nearT, so the loop ends; the cap guards
    // against a corrupted mesh only
    for (int guard = 0; r.ft < INFINITY && guard < (1 << 20); ++guard) {
      r.nt = r.ft + 1e-4f;
      r.ft = INFINITY;
      if (!isect()) break;
      ++hits;
    }
  }
  return (hits % 2) == 1;
}
// Mesh::distToPoint (mesh.cpp:325-339): world-space distance to the closest point
template <bool INL = false>
MD float mesh_dist(const DMesh& m, v3 p, uint32_t& tri, v3& q, bool& overflow) {
  v3 pl = apply4(m.Tinv, p);
  v3 ql = mk3(0, 0, 0);
  if (INL)
    bvh_closest_inl(m, pl, tri, ql, overflow);
  else
    bvh_closest(m, pl, tri, ql, overflow);
  q = apply4(m.T, ql);
  return norm3(q - p);
}

// Number of surface crossings of the segment o + d t, t in (t0, t1), counted
// as Mesh::inside counts them along its +x ray (the next search starts 1e-4
// past the previous hit). For a closed mesh an odd count flips inside/outside.
MD int segment_crossings(const DMesh& m, v3 o, v3 d, float t0, float t1, bool& overflow) {
  Ray r;
  r.o = o;
  r.d = d;
  r.nt = t0;
  r.ft = t1;
  uint32_t tri;
  float u, v;
  int n = 0;
  for (int guard = 0; guard < 64; ++guard) {
    if (!bvh_intersect(m, r, tri, u, v, overflow)) break;
    ++n;
    r.nt = r.ft + 1e-4f;
    r.ft = t1;
    if (!(r.nt < r.ft)) break;
  }
  return n;
}

// intersectUnitSphere (sphere.cpp:11-30)
MD float unit_sphere(float nt, float ft, v3 O, v3 D) {
  float a = sqn(D), b = dot(O, D), c = sqn(O) - 1.0f;
  float disc = b * b - a * c;
  if (disc < 0.0f) return -1.0f;
  float sq = sqrtf(disc);
  float t = (-b - sq) / a;
  if (t > nt && t < ft) return t;
  t = (-b + sq) / a;
  if (t > nt && t < ft) return t;
  return -1.0f;
}

// TangentFrame(n) (math/sample.h:21-32)
struct Frame {
  v3 n, t, b;
};
MD Frame make_frame(v3 nn) {
  Frame f;
  f.n = normalized(nn);
  float sign = copysignf(1.0f, f.n.z);
  float a = -1.0f / (sign + f.n.z);
  float b = f.n.x * f.n.y * a;
  f.t = normalized(mk3(1.0f + sign * f.n.x * f.n.x * a, sign * b, -sign * f.n.x));
  f.b = normalized(mk3(b, sign + f.n.y * f.n.y * a, -f.n.y));
  return f;
}
MD v3 to_global(const Frame& f, v3 p) { return (f.t * p.x + f.b * p.y) + f.n * p.z; }
