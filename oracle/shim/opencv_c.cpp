// Test-only definitions of the OpenCV 1.x C-API names declared in
// shim/opencv4/opencv2/core/core_c.h, so that the reference's FBP filter
// (filter/filter_prj.cpp FileterProjectionSymmetrize, modes 0/1 of
// ApplyFilterInplace) runs unmodified in the oracle.  Oracle infrastructure.
//
// Only what those modes use: single-channel float images and matrices,
// image regions of interest, sub-rect matrix views, copies, flips, zeroing,
// repeat, element access, and row DFTs of real data.  A forward row DFT of
// length N stores the spectrum in OpenCV's packed layout for real input --
// Re0, Re1, Im1, Re2, Im2, ..., with Re(N/2) last when N is even -- and the
// inverse reads it back (CV_DXT_SCALE divides by N).  The DFTs are evaluated
// directly in double precision from a twiddle table and rounded to float
// once, so the result is the exact transform (OpenCV's own float FFT differs
// from it by its rounding only).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "opencv4/opencv2/core/core_c.h"

namespace {

[[noreturn]] void fail(const char *what) {
  fprintf(stderr, "oracle OpenCV shim: %s\n", what);
  abort();
}

bool is_mat(const CvArr *a) {
  return (reinterpret_cast<const CvMat *>(a)->type & 0xFFFF0000) == ORC_MAT_MAGIC;
}

// A float matrix view: rows x cols, row stride in floats.
struct View {
  float *p;
  int rows, cols, step;
  float &at(int r, int c) const { return p[(size_t)r * step + c]; }
};

View view(const CvArr *a) {
  if (is_mat(a)) {
    const CvMat *m = reinterpret_cast<const CvMat *>(a);
    if ((m->type & 0xFFFF) != CV_32FC1) fail("only CV_32FC1 matrices are supported");
    return View{m->data.fl, m->rows, m->cols, m->step / (int)sizeof(float)};
  }
  const IplImage *im = reinterpret_cast<const IplImage *>(a);
  if (im->depth != IPL_DEPTH_32F || im->nChannels != 1) fail("only 32F one-channel images");
  float *base = reinterpret_cast<float *>(im->imageData);
  const int step = im->widthStep / (int)sizeof(float);
  if (im->roi)
    return View{base + (size_t)im->roi->yOffset * step + im->roi->xOffset, im->roi->height,
                im->roi->width, step};
  return View{base, im->height, im->width, step};
}

void same_size(const View &a, const View &b, const char *who) {
  if (a.rows != b.rows || a.cols != b.cols) fail(who);
}

// Real DFT of x[0..n) into OpenCV's packed layout out[0..n), or the inverse.
void row_dft(const float *in, float *out, int n, bool inverse, bool scale,
             const std::vector<double> &c, const std::vector<double> &s) {
  std::vector<double> acc(n, 0.0);
  if (!inverse) {
    // X_k = sum_m x_m e^{-2 pi i k m / n}, k = 0 .. n/2
    for (int k = 0; k <= n / 2; ++k) {
      double re = 0, im = 0;
      for (int m = 0; m < n; ++m) {
        const int j = (int)(((long long)k * m) % n);
        re += (double)in[m] * c[j];
        im -= (double)in[m] * s[j];
      }
      if (k == 0) {
        acc[0] = re;
      } else if (2 * k == n) {
        acc[n - 1] = re;
      } else {
        acc[2 * k - 1] = re;
        acc[2 * k] = im;
      }
    }
  } else {
    // x_m = sum_k X_k e^{+2 pi i k m / n} with X_{n-k} = conj(X_k)
    const int kmax = (n % 2 == 0) ? n / 2 - 1 : (n - 1) / 2;
    for (int m = 0; m < n; ++m) {
      double v = in[0];
      for (int k = 1; k <= kmax; ++k) {
        const int j = (int)(((long long)k * m) % n);
        v += 2.0 * ((double)in[2 * k - 1] * c[j] - (double)in[2 * k] * s[j]);
      }
      if (n % 2 == 0) v += (double)in[n - 1] * ((m % 2) ? -1.0 : 1.0);
      acc[m] = scale ? v / n : v;
    }
  }
  for (int i = 0; i < n; ++i) out[i] = (float)acc[i];
}

}  // namespace

CvMat *cvCreateMatHeader(int rows, int cols, int type) {
  CvMat *m = new CvMat();
  m->type = ORC_MAT_MAGIC | type;
  m->step = cols * (int)sizeof(float);
  m->rows = rows;
  m->cols = cols;
  m->data.ptr = nullptr;
  m->refcount = nullptr;  // non-null: the header owns its data
  return m;
}

CvMat *cvCreateMat(int rows, int cols, int type) {
  CvMat *m = cvCreateMatHeader(rows, cols, type);
  m->data.fl = static_cast<float *>(calloc((size_t)rows * cols, sizeof(float)));
  m->refcount = &m->hdr_refcount;
  return m;
}

void cvSetData(CvArr *arr, void *data, int step) {
  if (is_mat(arr)) {
    CvMat *m = reinterpret_cast<CvMat *>(arr);
    m->data.ptr = static_cast<unsigned char *>(data);
    m->step = step;
  } else {
    IplImage *im = reinterpret_cast<IplImage *>(arr);
    im->imageData = im->imageDataOrigin = static_cast<char *>(data);
    im->widthStep = step;
    im->imageSize = step * im->height;
  }
}

void cvReleaseMat(CvMat **mat) {
  if (!mat || !*mat) return;
  if ((*mat)->refcount) free((*mat)->data.ptr);
  delete *mat;
  *mat = nullptr;
}

IplImage *cvCreateImageHeader(CvSize size, int depth, int channels) {
  IplImage *im = new IplImage();
  im->nSize = (int)sizeof(IplImage);
  im->nChannels = channels;
  im->depth = depth;
  im->width = size.width;
  im->height = size.height;
  im->widthStep = size.width * channels * (int)sizeof(float);
  im->roi = nullptr;
  im->imageData = im->imageDataOrigin = nullptr;
  return im;
}

IplImage *cvCreateImage(CvSize size, int depth, int channels) {
  IplImage *im = cvCreateImageHeader(size, depth, channels);
  im->imageSize = im->widthStep * size.height;
  im->imageData = im->imageDataOrigin = static_cast<char *>(calloc(im->imageSize, 1));
  im->ID = 1;  // owns its data
  return im;
}

void cvReleaseImageHeader(IplImage **image) {
  if (!image || !*image) return;
  delete (*image)->roi;
  delete *image;
  *image = nullptr;
}

void cvReleaseImage(IplImage **image) {
  if (!image || !*image) return;
  if ((*image)->ID == 1) free((*image)->imageDataOrigin);
  cvReleaseImageHeader(image);
}

void cvSetImageROI(IplImage *image, CvRect rect) {
  if (!image->roi) image->roi = new IplROI();
  image->roi->coi = 0;
  image->roi->xOffset = rect.x;
  image->roi->yOffset = rect.y;
  image->roi->width = rect.width;
  image->roi->height = rect.height;
}

void cvResetImageROI(IplImage *image) {
  delete image->roi;
  image->roi = nullptr;
}

void cvCopy(const CvArr *src, CvArr *dst, const CvArr *mask) {
  if (mask) fail("cvCopy with a mask");
  const View a = view(src), b = view(dst);
  same_size(a, b, "cvCopy: sizes differ");
  for (int r = 0; r < a.rows; ++r)
    memmove(&b.at(r, 0), &a.at(r, 0), sizeof(float) * (size_t)a.cols);
}

void cvSetZero(CvArr *arr) {
  const View v = view(arr);
  for (int r = 0; r < v.rows; ++r) memset(&v.at(r, 0), 0, sizeof(float) * (size_t)v.cols);
}

void cvZero(CvArr *arr) { cvSetZero(arr); }

void cvFlip(const CvArr *src, CvArr *dst, int flip_mode) {
  const View a = view(src), b = view(dst);
  same_size(a, b, "cvFlip: sizes differ");
  std::vector<float> t((size_t)a.rows * a.cols);
  for (int r = 0; r < a.rows; ++r)
    for (int c = 0; c < a.cols; ++c) t[(size_t)r * a.cols + c] = a.at(r, c);
  for (int r = 0; r < a.rows; ++r)
    for (int c = 0; c < a.cols; ++c) {
      const int sr = flip_mode <= 0 ? a.rows - 1 - r : r;  // 0: about x, <0: both
      const int sc = flip_mode != 0 ? a.cols - 1 - c : c;  // >0: about y
      b.at(r, c) = t[(size_t)sr * a.cols + sc];
    }
}

CvMat *cvGetSubRect(const CvArr *arr, CvMat *submat, CvRect rect) {
  const View v = view(arr);
  if (rect.x < 0 || rect.y < 0 || rect.width < 0 || rect.height < 0 ||
      rect.x + rect.width > v.cols || rect.y + rect.height > v.rows)
    fail("cvGetSubRect: rectangle outside the array");
  submat->type = ORC_MAT_MAGIC | CV_32FC1;
  submat->step = v.step * (int)sizeof(float);
  submat->refcount = nullptr;
  submat->hdr_refcount = 0;
  submat->data.fl = v.p + (size_t)rect.y * v.step + rect.x;
  submat->rows = rect.height;
  submat->cols = rect.width;
  return submat;
}

int cvGetOptimalDFTSize(int size0) {
  for (int n = size0 < 1 ? 1 : size0;; ++n) {
    int r = n;
    while (r % 2 == 0) r /= 2;
    while (r % 3 == 0) r /= 3;
    while (r % 5 == 0) r /= 5;
    if (r == 1) return n;
  }
}

void cvDFT(const CvArr *src, CvArr *dst, int flags, int nonzero_rows) {
  if (!(flags & CV_DXT_ROWS)) fail("cvDFT: only row transforms (CV_DXT_ROWS)");
  const View a = view(src), b = view(dst);
  same_size(a, b, "cvDFT: sizes differ");
  const bool inverse = (flags & CV_DXT_INVERSE) != 0, scale = (flags & CV_DXT_SCALE) != 0;
  const int n = a.cols;
  std::vector<double> c(n), s(n);
  for (int j = 0; j < n; ++j) {
    c[j] = cos(2.0 * M_PI * j / n);
    s[j] = sin(2.0 * M_PI * j / n);
  }
  // Rows past nonzero_rows: zero input (forward) or outputs of no interest
  // (inverse); both give zero rows here.
  const int live = nonzero_rows > 0 && nonzero_rows < a.rows ? nonzero_rows : a.rows;
  std::vector<float> in(n), out(n);
  for (int r = 0; r < a.rows; ++r) {
    if (r >= live) {
      memset(&b.at(r, 0), 0, sizeof(float) * (size_t)n);
      continue;
    }
    for (int i = 0; i < n; ++i) in[i] = a.at(r, i);
    row_dft(in.data(), out.data(), n, inverse, scale, c, s);
    for (int i = 0; i < n; ++i) b.at(r, i) = out[i];
  }
}

void cvMulSpectrums(const CvArr *a, const CvArr *b, CvArr *dst, int flags) {
  if (!(flags & CV_DXT_ROWS) || (flags & ~CV_DXT_ROWS)) fail("cvMulSpectrums: rows only");
  const View x = view(a), y = view(b), z = view(dst);
  same_size(x, y, "cvMulSpectrums: sizes differ");
  same_size(x, z, "cvMulSpectrums: sizes differ");
  const int n = x.cols;
  for (int r = 0; r < x.rows; ++r) {
    // packed real spectra: element 0 (and n-1 for even n) real, then pairs
    z.at(r, 0) = x.at(r, 0) * y.at(r, 0);
    const int last = (n % 2 == 0) ? n - 2 : n - 1;
    for (int i = 1; i < last; i += 2) {
      const float ar = x.at(r, i), ai = x.at(r, i + 1), br = y.at(r, i), bi = y.at(r, i + 1);
      z.at(r, i) = ar * br - ai * bi;
      z.at(r, i + 1) = ar * bi + ai * br;
    }
    if (n % 2 == 0 && n > 1) z.at(r, n - 1) = x.at(r, n - 1) * y.at(r, n - 1);
  }
}

void cvRepeat(const CvArr *src, CvArr *dst) {
  const View a = view(src), b = view(dst);
  for (int r = 0; r < b.rows; ++r)
    for (int c = 0; c < b.cols; ++c) b.at(r, c) = a.at(r % a.rows, c % a.cols);
}

CvScalar cvGet2D(const CvArr *arr, int idx0, int idx1) {
  CvScalar s = {{0, 0, 0, 0}};
  s.val[0] = view(arr).at(idx0, idx1);
  return s;
}

double cvGetReal2D(const CvArr *arr, int idx0, int idx1) { return view(arr).at(idx0, idx1); }

void cvmSet(CvMat *mat, int row, int col, double value) { view(mat).at(row, col) = (float)value; }

double cvmGet(const CvMat *mat, int row, int col) { return view(mat).at(row, col); }
