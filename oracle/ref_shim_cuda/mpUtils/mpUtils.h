/* TEST INFRASTRUCTURE ONLY: see mpCuda.h in this directory. */
#ifndef GSPH_REF_SHIM_CUDA_MPUTILS_H
#define GSPH_REF_SHIM_CUDA_MPUTILS_H
#include "mpCuda.h"
#endif
