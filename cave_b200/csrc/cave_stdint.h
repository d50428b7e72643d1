// cave_stdint.h -- fixed-width integer types for every compiler that sees the device headers:
// nvcc and the host compiler take them from <cstdint>; NVRTC (the run-time compiler of the
// rule-specialised tick kernel) has no standard library headers, so they are declared here.
#pragma once
#ifdef __CUDACC_RTC__
typedef signed char int8_t;
typedef short int16_t;
typedef int int32_t;
typedef long long int64_t;
typedef unsigned char uint8_t;
typedef unsigned short uint16_t;
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
#else
#include <cstdint>
#endif
