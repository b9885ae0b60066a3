// Stand-in for the OpenCV 1.x C types the reference's image classes name:
// CvMat with a float data view, CvArr.  The oracle's harness defines the
// image classes' out-of-line members over host arrays.
#pragma once
typedef void CvArr;
struct CvMat {
    int type, step;
    int* refcount;
    int hdr_refcount;
    union {
        unsigned char* ptr;
        short* s;
        int* i;
        float* fl;
        double* db;
    } data;
    int rows, cols;
};
