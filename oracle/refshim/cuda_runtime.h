// CPU ORACLE — test infrastructure. Stand-in for the CUDA runtime header when
// the reference's kernels are compiled as host C++ (oracle/ref_kernels.cpp):
// the reference headers name only the stream and event handle types.
#pragma once
#include <cstdint>
typedef struct ICEMPM_CUstream_st* cudaStream_t;
typedef struct ICEMPM_CUevent_st* cudaEvent_t;
