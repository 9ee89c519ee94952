// OBJ reader with Mesh::fetchFrom's rules (primitives/mesh.cpp:20-136): v, vn,
// vt (optional third coordinate read and dropped) and triangular f records in
// the v, v/vt, v//vn and v/vt/vn forms with 1-based or negative (relative)
// indices; an absent vt index maps to texcoord 0; faces of other sizes and
// other record types are skipped. Numbers are read with the same stream
// extractions (std::istringstream >> float, std::stoi) as the reference, so a
// file parses to the same bits; a failed float extraction yields 0, as the
// reference's stream does.
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "host.h"

using namespace mupsi;

namespace {

template <typename T>
T* copy_out(const std::vector<T>& v) {
  if (v.empty()) return nullptr;
  T* p = static_cast<T*>(std::malloc(v.size() * sizeof(T)));
  if (p) std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}

// normIdx (mesh.cpp:99-103): 1-based -> 0-based, negative counts back from `count`
uint32_t norm_idx(int idx, size_t count) {
  if (idx > 0) return static_cast<uint32_t>(idx - 1);
  if (idx < 0) return static_cast<uint32_t>(static_cast<int>(count) + idx);
  return 0u;
}

}  // namespace

extern "C" {

int mupsi_obj_load(const char* path, mupsi_obj* out) {
  clear_error();
  if (!path || !out) return fail(MUPSI_ERR_INVALID, "null argument");
  std::memset(out, 0, sizeof *out);
  std::ifstream file(path);
  if (!file.is_open()) return fail(MUPSI_ERR_INVALID, std::string("cannot open ") + path);
  std::vector<float> v, vn, vt;
  std::vector<int32_t> f, ft;
  std::string line;
  try {
    while (std::getline(file, line)) {
      if (!line.empty() && line.back() == '\r') line.pop_back();
      if (line.empty() || line[0] == '#') continue;
      std::istringstream iss(line);
      std::string type;
      iss >> type;
      if (type == "v" || type == "vn") {
        float x, y, z;
        iss >> x >> y >> z;
        std::vector<float>& dst = type == "v" ? v : vn;
        dst.push_back(x);
        dst.push_back(y);
        dst.push_back(z);
      } else if (type == "vt") {
        float a, b, w = 0;
        iss >> a >> b;
        if (iss >> w) {
        }
        vt.push_back(a);
        vt.push_back(b);
      } else if (type == "f") {
        uint32_t vi3[3], ti3[3];
        int nv = 0;
        std::string spec;
        while (iss >> spec) {
          int vi = 0, vti = 0;
          const size_t s1 = spec.find('/');
          if (s1 == std::string::npos) {
            vi = std::stoi(spec);
          } else {
            vi = std::stoi(spec.substr(0, s1));
            const size_t s2 = spec.find('/', s1 + 1);
            if (s2 == std::string::npos)
              vti = std::stoi(spec.substr(s1 + 1));
            else if (s1 + 1 != s2)
              vti = std::stoi(spec.substr(s1 + 1, s2 - s1 - 1));
            // a normal index after the second slash is parsed by the reference and unused
          }
          if (nv < 3) {
            vi3[nv] = norm_idx(vi, v.size() / 3);
            ti3[nv] = norm_idx(vti, vt.size() / 2);
          }
          ++nv;
        }
        if (nv != 3) continue;  // faces with < 3 or > 3 vertices are skipped
        for (int c = 0; c < 3; ++c) {
          f.push_back(static_cast<int32_t>(vi3[c]));
          ft.push_back(static_cast<int32_t>(ti3[c]));
        }
      }
    }
  } catch (const std::exception& e) {  // std::stoi on a malformed index (the reference throws too)
    return fail(MUPSI_ERR_INVALID, std::string(path) + ": bad face index: " + e.what());
  }
  if (v.empty() || f.empty()) return fail(MUPSI_ERR_INVALID, std::string(path) + ": no valid geometry");
  const int64_t nvtx = (int64_t)(v.size() / 3), nt = (int64_t)(vt.size() / 2);
  for (int32_t i : f)
    if (i < 0 || i >= nvtx) return fail(MUPSI_ERR_INVALID, std::string(path) + ": vertex index out of range");
  if (nt > 0)
    for (int32_t i : ft)
      if (i < 0 || i >= nt) return fail(MUPSI_ERR_INVALID, std::string(path) + ": texcoord index out of range");
  out->num_vertices = nvtx;
  out->num_faces = (int64_t)(f.size() / 3);
  out->num_normals = (int64_t)(vn.size() / 3);
  out->num_texcoords = nt;
  out->vertices = copy_out(v);
  out->faces = copy_out(f);
  out->normals = copy_out(vn);
  out->texcoords = copy_out(vt);
  out->face_texcoords = nt > 0 ? copy_out(ft) : nullptr;
  if (!out->vertices || !out->faces || (out->num_normals && !out->normals) || (nt && !out->texcoords)) {
    mupsi_obj_free(out);
    return fail(MUPSI_ERR_INVALID, "out of host memory");
  }
  return MUPSI_OK;
}

void mupsi_obj_free(mupsi_obj* obj) {
  if (!obj) return;
  std::free(obj->vertices);
  std::free(obj->faces);
  std::free(obj->normals);
  std::free(obj->texcoords);
  std::free(obj->face_texcoords);
  std::memset(obj, 0, sizeof *obj);
}

}  // extern "C"
