/*
 * mkl_dfti.h -- stand-in for the MKL DFTI interface used by the reference
 * (complex double, 1D, strided, out of place).  See mkl.h for the scope.
 */
#pragma once
#include "mkl.h"

enum DFTI_CONFIG_VALUE_STANDIN {
    DFTI_NO_ERROR = 0,
    DFTI_SINGLE = 35,
    DFTI_DOUBLE = 36,
    DFTI_COMPLEX = 32,
    DFTI_REAL = 33,
    DFTI_INPLACE = 43,
    DFTI_NOT_INPLACE = 44,
    DFTI_COMPLEX_COMPLEX = 39,
    DFTI_COMPLEX_REAL = 40,
    DFTI_PLACEMENT = 11,
    DFTI_FORWARD_SCALE = 4,
    DFTI_BACKWARD_SCALE = 5,
    DFTI_INPUT_STRIDES = 12,
    DFTI_OUTPUT_STRIDES = 13,
    DFTI_CONJUGATE_EVEN_STORAGE = 10,
    DFTI_NUMBER_OF_TRANSFORMS = 7,
    DFTI_INPUT_DISTANCE = 14,
    DFTI_OUTPUT_DISTANCE = 15
};

struct DFTI_DESCRIPTOR_STANDIN;
typedef struct DFTI_DESCRIPTOR_STANDIN *DFTI_DESCRIPTOR_HANDLE;

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *h, int precision, int domain, MKL_LONG dimension, ...);
MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE h, int param, ...);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void *in, ...);
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE h, void *in, ...);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *h);
