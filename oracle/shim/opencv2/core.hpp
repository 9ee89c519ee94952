// OpenCV stand-in for the CPU oracle (test infrastructure). Only the handful of
// types the reference's image IO names exist. imwrite writes nothing; imread
// reads two project-defined raw formats and nothing else: a text header
// "MUPSI_RGBF <width> <height>\n" followed by width * height * 3 little-endian
// float32 values (read only with IMREAD_ANYDEPTH, as a float image), or
// "MUPSI_RGB8 <width> <height>\n" followed by width * height * 3 bytes (an
// 8-bit image); rows from the top, RGB. The tests write skydrome and albedo
// images this way. The pixels come back already in RGB order and cvtColor is a
// copy, so the reference's BGR-to-RGB conversion leaves them as written.
#ifndef MUPSI_ORACLE_CV_STUB_CORE
#define MUPSI_ORACLE_CV_STUB_CORE
#include <cstdint>
#include <cstdio>
#include <cstring>
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
// The raw formats above.
inline Mat imread(const std::string& path, int flags = IMREAD_COLOR) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return Mat();
  char magic[16] = {0};
  int w = 0, h = 0;
  if (std::fscanf(f, "%15s %d %d", magic, &w, &h) != 3 || w <= 0 || h <= 0 || w > (1 << 15) || h > (1 << 15) ||
      std::fgetc(f) != '\n') {
    std::fclose(f);
    return Mat();
  }
  int type;
  if (std::strcmp(magic, "MUPSI_RGBF") == 0 && (flags & IMREAD_ANYDEPTH))
    type = CV_32FC3;
  else if (std::strcmp(magic, "MUPSI_RGB8") == 0)
    type = CV_8UC3;
  else {
    std::fclose(f);
    return Mat();
  }
  Mat m(h, w, type);
  const size_t got = std::fread(m.buf.data(), 1, m.buf.size(), f);
  std::fclose(f);
  if (got != m.buf.size()) return Mat();
  return m;
}
inline void cvtColor(const Mat& src, Mat& dst, int) { dst = src; }
}  // namespace cv
#endif
