// Host-side helpers shared by the library's translation units: error state,
// launch accounting, device buffers, kernel parameters and transforms.
#pragma once
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mupsi_gpu.h"

namespace mupsi {

struct HostNode {
  float mn[3];
  float mx[3];
  uint32_t left, right;
};
static_assert(sizeof(HostNode) == 32, "BVH node is 32 bytes");

uint32_t build_bvh(const float* verts, const int32_t* faces, int64_t num_faces, std::vector<HostNode>& nodes,
                   std::vector<uint32_t>& tri_idx);

// thread-local last error message; returns `code` for `return fail(...)`
int fail(int code, const std::string& msg);
void clear_error();
void count_launch(int n = 1);

// 4x4 column-major matrices for the primitives' Translation*Scaling transforms.
struct HostM4 {
  float m[16];
};
HostM4 translate_scale(const float t[3], float s);
// Inverse by cofactors over the determinant, the rounding sequence the oracle's
// Eigen shim uses for Matrix4f::inverse().
HostM4 inverse4(const HostM4& a);
bool is_identity4(const HostM4& a);
bool is_identity3(const HostM4& a);

}  // namespace mupsi

#define MUPSI_CUDA(call)                                                                     \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return ::mupsi::fail(e_ == cudaErrorMemoryAllocation ? MUPSI_ERR_OOM : MUPSI_ERR_CUDA, \
                           std::string(#call) + ": " + cudaGetErrorString(e_));              \
  } while (0)
