// Mathematical constants of CUDA's math_constants.h that sources built against the CPU emulation
// of CUDA name (test infrastructure; see cuda_runtime.h).
#pragma once
#define CUDART_PI 3.1415926535897931e+0
