// CPU ORACLE — test infrastructure. Stand-in for the CUDA driver header when
// the reference's kernels are compiled as host C++ (oracle/ref_kernels.cpp).
#pragma once
#include "cuda_runtime.h"
