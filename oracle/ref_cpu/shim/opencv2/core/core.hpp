// Minimal stand-in for OpenCV's cv::Mat (absent here), used ONLY to compile
// the reference's kernel sources for the CPU: a dense row-major buffer with
// at<T>(row, col), enough for the image helpers those files define.
#pragma once
#include <cstddef>
#include <memory>
#include <vector>
#define CV_8UC1 0
#define CV_8UC3 16
#define CV_16UC1 2
#define CV_32FC1 5
#define CV_32FC3 21
namespace cv {
template <class T, int N>
struct Vec {
  T v[N];
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
};
typedef Vec<unsigned char, 3> Vec3b;
typedef Vec<float, 3> Vec3f;
class Mat {
 public:
  int rows = 0, cols = 0, type_ = 0;
  std::shared_ptr<std::vector<unsigned char>> buf;
  static size_t elem(int t) {
    switch (t) {
      case CV_8UC1: return 1;
      case CV_8UC3: return 3;
      case CV_16UC1: return 2;
      case CV_32FC1: return 4;
      case CV_32FC3: return 12;
    }
    return 16;
  }
  Mat() {}
  Mat(int r, int c, int t)
      : rows(r), cols(c), type_(t),
        buf(std::make_shared<std::vector<unsigned char>>((size_t)r * c * elem(t))) {}
  int type() const { return type_; }
  template <class T>
  T& at(int i, int j) {
    return reinterpret_cast<T*>(buf->data())[(size_t)i * cols + j];
  }
  template <class T>
  const T& at(int i, int j) const {
    return reinterpret_cast<const T*>(buf->data())[(size_t)i * cols + j];
  }
};
}  // namespace cv
