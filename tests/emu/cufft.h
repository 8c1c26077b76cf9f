// cuFFT result codes for sources built against the CPU emulation of CUDA (test infrastructure;
// see cuda_runtime.h).  No transform is provided: the builds that include this name the codes only.
#pragma once
typedef enum cufftResult_t {
    CUFFT_SUCCESS = 0,
    CUFFT_INVALID_PLAN = 1,
    CUFFT_ALLOC_FAILED = 2,
    CUFFT_INVALID_TYPE = 3,
    CUFFT_INVALID_VALUE = 4,
    CUFFT_INTERNAL_ERROR = 5,
    CUFFT_EXEC_FAILED = 6,
    CUFFT_SETUP_FAILED = 7,
    CUFFT_INVALID_SIZE = 8
} cufftResult;
