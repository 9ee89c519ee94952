// OpenCV stand-in for the CPU oracle (test infrastructure). Only the handful of
// types the reference's image IO names exist; images are kept in memory, imwrite
// writes nothing and imread returns an empty image (the oracle never loads
// bitmaps: skies are constant and meshes carry no textures in the test scenes).
#ifndef MUPSI_ORACLE_CV_STUB_CORE
#define MUPSI_ORACLE_CV_STUB_CORE
#include <cstdint>
#include <string>
#include <vector>
#define CV_8UC3 16
#define CV_32FC3 21
namespace cv {
template <typename T, int N>
struct Vec {
  T v[N];
  Vec() : v{} {}
  Vec(T a, T b, T c) : v{a, b, c} {}
  T& operator[](int i) { return v[i]; }
};
typedef Vec<float, 3> Vec3f;
typedef Vec<unsigned char, 3> Vec3b;
class Mat {
 public:
  int rows = 0, cols = 0, type_ = 0;
  std::vector<unsigned char> buf;
  Mat() = default;
  Mat(int r, int c, int type) : rows(r), cols(c), type_(type) {
    buf.resize((size_t)r * c * (type == CV_32FC3 ? 12 : 3));
  }
  bool empty() const { return rows == 0 || cols == 0; }
  template <typename T>
  T& at(int r, int c) { return reinterpret_cast<T*>(buf.data())[(size_t)r * cols + c]; }
  template <typename T>
  T* ptr(int r) { return reinterpret_cast<T*>(buf.data()) + (size_t)r * cols * 3; }
};
enum { IMREAD_COLOR = 1, IMREAD_ANYDEPTH = 2, COLOR_BGR2RGB = 4 };
inline bool imwrite(const std::string&, const Mat&) { return false; }
inline Mat imread(const std::string&, int = IMREAD_COLOR) { return Mat(); }
inline void cvtColor(const Mat& src, Mat& dst, int) { dst = src; }
}  // namespace cv
#endif
