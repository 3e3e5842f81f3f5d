// Test-only stand-in for the subset of OpenCV's C++ core that the reference's
// resample tool uses (src/resample/src/mrcimg/mrc2img.cpp,
// src/resample/src/main/main.cpp): single-channel float matrices with
// shared storage, copies, and the statistics the tool takes.  OpenCV itself
// is not available here; this lets the unmodified resample sources build as
// the oracle.  Not part of the product.
#pragma once

// Standard headers OpenCV's core header brings in, which the tool's sources
// rely on.
#include <algorithm>
#include <cassert>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#define CV_32F 5
#define CV_32FC1 CV_32F

namespace cv {

struct Size {
  int width = 0, height = 0;
  Size() = default;
  Size(int w, int h) : width(w), height(h) {}
};

struct Scalar {
  double val[4] = {0, 0, 0, 0};
  double operator[](int i) const { return val[i]; }
};

// Matrix of `rows` x `cols` floats (the only element type the tool uses),
// rows `step` bytes apart; copies share the storage, as OpenCV's do.
class Mat {
 public:
  int rows = 0, cols = 0;
  size_t step = 0;
  unsigned char *data = nullptr;

  Mat() = default;
  Mat(int r, int c, int type) { create(r, c, type); }
  Mat(Size s, int type) { create(s.height, s.width, type); }

  void create(int r, int c, int type) {
    type_ = type;
    rows = r;
    cols = c;
    step = (size_t)c * sizeof(float);
    buf_ = std::make_shared<std::vector<float>>((size_t)r * c, 0.f);
    data = reinterpret_cast<unsigned char *>(buf_->data());
  }
  static Mat zeros(Size s, int type) { return Mat(s, type); }
  Size size() const { return Size(cols, rows); }
  int type() const { return type_; }
  bool empty() const { return data == nullptr || rows == 0 || cols == 0; }
  unsigned char *ptr(int y = 0) { return data + (size_t)y * step; }
  const unsigned char *ptr(int y = 0) const { return data + (size_t)y * step; }
  template <typename T>
  T &at(int y, int x) {
    return reinterpret_cast<T *>(ptr(y))[x];
  }
  template <typename T>
  const T &at(int y, int x) const {
    return reinterpret_cast<const T *>(ptr(y))[x];
  }
  Mat clone() const {
    Mat m;
    if (!empty()) {
      m.create(rows, cols, type_);
      std::memcpy(m.data, data, (size_t)rows * step);
    }
    return m;
  }
  void copyTo(Mat &m) const { m = clone(); }

 private:
  int type_ = CV_32F;
  std::shared_ptr<std::vector<float>> buf_;
};

// Smallest and largest element.
inline void minMaxLoc(const Mat &m, double *lo, double *hi, void * = nullptr,
                      void * = nullptr) {
  double a = 0, b = 0;
  for (int y = 0; y < m.rows; ++y)
    for (int x = 0; x < m.cols; ++x) {
      const double v = m.at<float>(y, x);
      if ((y == 0 && x == 0) || v < a) a = v;
      if ((y == 0 && x == 0) || v > b) b = v;
    }
  if (lo) *lo = a;
  if (hi) *hi = b;
}

// Mean of the elements (channel 0).
inline Scalar mean(const Mat &m) {
  Scalar s;
  double acc = 0;
  for (int y = 0; y < m.rows; ++y)
    for (int x = 0; x < m.cols; ++x) acc += m.at<float>(y, x);
  s.val[0] = m.rows && m.cols ? acc / ((double)m.rows * m.cols) : 0.0;
  return s;
}

}  // namespace cv
