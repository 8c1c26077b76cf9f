// Driver-API stream type of the CPU emulation of CUDA (test infrastructure; see cuda_runtime.h).
#pragma once
#include "cuda_runtime.h"
typedef struct CUstream_st* CUstream;
