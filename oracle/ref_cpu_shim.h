// ref_cpu_shim.h - lets the reference's generated CUDA kernel source compile as host C++.
//
// Oracle infrastructure only: oracle/ref_capture.py compiles each captured reference kernel
// (the text GQIS hands to NVRTC) once with nvcc for sm_100a and once with g++ through this
// header, so the reference's own arithmetic can produce golden outputs without a GPU.
// Device qualifiers become inline host functions; blockIdx/threadIdx are thread-local values
// set by the generated host launcher for every (block, thread) pair.
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
#define __restrict__ __restrict

struct float2 { float x, y; };
struct double2 { double x, y; };
struct int2 { int x, y; };
static inline float2 make_float2(float x, float y) { float2 r = {x, y}; return r; }
static inline double2 make_double2(double x, double y) { double2 r = {x, y}; return r; }
static inline int2 make_int2(int x, int y) { int2 r = {x, y}; return r; }
static inline float __int_as_float(int i) { float f; memcpy(&f, &i, sizeof f); return f; }

struct gq_uint3 { unsigned x, y, z; };
static thread_local gq_uint3 threadIdx, blockIdx;
static thread_local gq_uint3 blockDim;
