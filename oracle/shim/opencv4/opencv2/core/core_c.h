/* Test-only declarations of the OpenCV 1.x C-API names used by the reference
 * filter source (filter/filter_prj.cpp), for its FBP filter modes 0/1.  The
 * definitions (shim/opencv_c.cpp) implement the single-channel float subset
 * those modes use -- images and matrices with regions of interest, sub-rect
 * views, flips, copies, row DFTs in OpenCV's packed real-spectrum layout and
 * their products -- with the DFTs evaluated exactly in double precision.
 * Oracle infrastructure only. */
#ifndef ORACLE_SHIM_OPENCV_CORE_C_H
#define ORACLE_SHIM_OPENCV_CORE_C_H

typedef void CvArr;
typedef struct CvRect { int x, y, width, height; } CvRect;
typedef struct CvSize { int width, height; } CvSize;
typedef struct CvScalar { double val[4]; } CvScalar;
/* `type` carries ORC_MAT_MAGIC in its high 16 bits, which tells a matrix
 * from an image (whose first field, nSize, is small). */
typedef struct CvMat {
  int type, step;
  int *refcount, hdr_refcount;
  union { unsigned char *ptr; float *fl; double *db; } data;
  int rows, cols;
} CvMat;
typedef struct IplROI { int coi, xOffset, yOffset, width, height; } IplROI;
typedef struct IplImage {
  int nSize, ID, nChannels, alphaChannel, depth;
  char colorModel[4], channelSeq[4];
  int dataOrder, origin, align, width, height;
  IplROI *roi;
  void *maskROI, *imageId, *tileInfo;
  int imageSize;
  char *imageData;
  int widthStep;
  int BorderMode[4], BorderConst[4];
  char *imageDataOrigin;
} IplImage;

#define ORC_MAT_MAGIC 0x42420000
#define IPL_DEPTH_32F 32
#define IPL_DEPTH_64F 64
#define CV_32FC1 5
#define CV_DXT_FORWARD 0
#define CV_DXT_INVERSE 1
#define CV_DXT_SCALE 2
#define CV_DXT_INV_SCALE 3
#define CV_DXT_ROWS 4

static inline CvRect cvRect(int x, int y, int w, int h) {
  CvRect r = {x, y, w, h};
  return r;
}
static inline CvSize cvSize(int w, int h) {
  CvSize s = {w, h};
  return s;
}

CvMat *cvCreateMatHeader(int rows, int cols, int type);
CvMat *cvCreateMat(int rows, int cols, int type);
void cvSetData(CvArr *arr, void *data, int step);
void cvReleaseMat(CvMat **mat);
IplImage *cvCreateImage(CvSize size, int depth, int channels);
IplImage *cvCreateImageHeader(CvSize size, int depth, int channels);
void cvReleaseImage(IplImage **image);
void cvReleaseImageHeader(IplImage **image);
void cvSetImageROI(IplImage *image, CvRect rect);
void cvResetImageROI(IplImage *image);
void cvCopy(const CvArr *src, CvArr *dst, const CvArr *mask);
void cvSetZero(CvArr *arr);
void cvZero(CvArr *arr);
void cvFlip(const CvArr *src, CvArr *dst, int flip_mode);
CvMat *cvGetSubRect(const CvArr *arr, CvMat *submat, CvRect rect);
int cvGetOptimalDFTSize(int size0);
void cvDFT(const CvArr *src, CvArr *dst, int flags, int nonzero_rows);
void cvMulSpectrums(const CvArr *a, const CvArr *b, CvArr *dst, int flags);
void cvRepeat(const CvArr *src, CvArr *dst);
CvScalar cvGet2D(const CvArr *arr, int idx0, int idx1);
double cvGetReal2D(const CvArr *arr, int idx0, int idx1);
void cvmSet(CvMat *mat, int row, int col, double value);
double cvmGet(const CvMat *mat, int row, int col);

#endif
