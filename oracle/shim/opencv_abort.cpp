// Abort-if-called definitions of the OpenCV names declared in
// shim/opencv4/opencv2/core/core_c.h.  The oracle only runs the WBP filter
// (mode 2), which never reaches OpenCV; reaching one of these is a bug.
#include <stdio.h>
#include <stdlib.h>

#include "opencv4/opencv2/core/core_c.h"

#define ORACLE_ABORT(name)                                                   \
  do {                                                                       \
    fprintf(stderr, "oracle shim: OpenCV %s is not available\n", name);     \
    abort();                                                                 \
  } while (0)

CvMat *cvCreateMatHeader(int, int, int) { ORACLE_ABORT("cvCreateMatHeader"); }
CvMat *cvCreateMat(int, int, int) { ORACLE_ABORT("cvCreateMat"); }
void cvSetData(CvArr *, void *, int) { ORACLE_ABORT("cvSetData"); }
void cvReleaseMat(CvMat **) { ORACLE_ABORT("cvReleaseMat"); }
IplImage *cvCreateImage(CvSize, int, int) { ORACLE_ABORT("cvCreateImage"); }
IplImage *cvCreateImageHeader(CvSize, int, int) {
  ORACLE_ABORT("cvCreateImageHeader");
}
void cvReleaseImage(IplImage **) { ORACLE_ABORT("cvReleaseImage"); }
void cvReleaseImageHeader(IplImage **) { ORACLE_ABORT("cvReleaseImageHeader"); }
void cvSetImageROI(IplImage *, CvRect) { ORACLE_ABORT("cvSetImageROI"); }
void cvResetImageROI(IplImage *) { ORACLE_ABORT("cvResetImageROI"); }
void cvCopy(const CvArr *, CvArr *, const CvArr *) { ORACLE_ABORT("cvCopy"); }
void cvSetZero(CvArr *) { ORACLE_ABORT("cvSetZero"); }
void cvZero(CvArr *) { ORACLE_ABORT("cvZero"); }
void cvFlip(const CvArr *, CvArr *, int) { ORACLE_ABORT("cvFlip"); }
CvMat *cvGetSubRect(const CvArr *, CvMat *, CvRect) {
  ORACLE_ABORT("cvGetSubRect");
}
int cvGetOptimalDFTSize(int) { ORACLE_ABORT("cvGetOptimalDFTSize"); }
void cvDFT(const CvArr *, CvArr *, int, int) { ORACLE_ABORT("cvDFT"); }
void cvMulSpectrums(const CvArr *, const CvArr *, CvArr *, int) {
  ORACLE_ABORT("cvMulSpectrums");
}
void cvRepeat(const CvArr *, CvArr *) { ORACLE_ABORT("cvRepeat"); }
CvScalar cvGet2D(const CvArr *, int, int) { ORACLE_ABORT("cvGet2D"); }
double cvGetReal2D(const CvArr *, int, int) { ORACLE_ABORT("cvGetReal2D"); }
void cvmSet(CvMat *, int, int, double) { ORACLE_ABORT("cvmSet"); }
double cvmGet(const CvMat *, int, int) { ORACLE_ABORT("cvmGet"); }
