// Test-only stand-in for <opencv2/opencv.hpp> as the reference's resample
// tool uses it: core.hpp's matrices plus area resampling (cv::resize with
// INTER_AREA).  Not part of the product.
#pragma once

#include <cmath>
#include <vector>

#include "opencv2/core.hpp"

namespace cv {

enum { INTER_NEAREST = 0, INTER_LINEAR = 1, INTER_CUBIC = 2, INTER_AREA = 3 };

namespace shim_detail {
// Area resampling along one axis, as OpenCV documents INTER_AREA for
// shrinking: destination sample i covers the source interval
// [i s, (i + 1) s) with s = n_src / n_dst, and averages the source samples
// weighted by their overlap with it (whole samples inside, fractions at the
// two ends).  Returns the first source index and the weights.
inline void area_weights(int n_src, int n_dst, int i, int *first, std::vector<double> *w) {
  const double s = (double)n_src / n_dst;
  const double a = i * s, b = (i + 1) * s;
  int k0 = (int)std::floor(a), k1 = (int)std::ceil(b);
  if (k1 > n_src) k1 = n_src;
  w->clear();
  *first = k0;
  for (int k = k0; k < k1; ++k) {
    const double lo = k > a ? (double)k : a, hi = k + 1 < b ? (double)(k + 1) : b;
    w->push_back(hi > lo ? (hi - lo) / s : 0.0);
  }
}
}  // namespace shim_detail

// Only INTER_AREA shrinking is provided (the one use in the tool).
inline void resize(const Mat &src, Mat &dst, Size dsize, double = 0, double = 0,
                   int interpolation = INTER_LINEAR) {
  (void)interpolation;
  Mat out(dsize.height, dsize.width, src.type());
  std::vector<double> wx, wy;
  for (int j = 0; j < dsize.height; ++j) {
    int y0;
    shim_detail::area_weights(src.rows, dsize.height, j, &y0, &wy);
    for (int i = 0; i < dsize.width; ++i) {
      int x0;
      shim_detail::area_weights(src.cols, dsize.width, i, &x0, &wx);
      double acc = 0;
      for (size_t b = 0; b < wy.size(); ++b) {
        double r = 0;
        for (size_t a = 0; a < wx.size(); ++a) r += wx[a] * src.at<float>(y0 + (int)b, x0 + (int)a);
        acc += wy[b] * r;
      }
      out.at<float>(j, i) = (float)acc;
    }
  }
  dst = out;
}

}  // namespace cv
