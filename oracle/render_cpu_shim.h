// render_cpu_shim.h - lets the reference renderer's CUDA kernel text compile as host C++.
//
// Oracle infrastructure only (tests/golden/make_render_golden.py): the kernels phase_bin,
// phase_finalize and display_rgba of the reference's Examples/fast_gpu_render.py are compiled by
// g++ with this header and run one (block, thread) at a time, which gives their arithmetic on the
// CPU; atomics become plain read-modify-writes. Compile with -ffp-contract=off.
#pragma once
#include "ref_cpu_shim.h"

#include <math.h>

struct float4 { float x, y, z, w; };
struct uchar4 { unsigned char x, y, z, w; };
static inline float4 make_float4(float x, float y, float z, float w) { float4 r = {x, y, z, w}; return r; }
static inline uchar4 make_uchar4(unsigned char x, unsigned char y, unsigned char z, unsigned char w) {
    uchar4 r = {x, y, z, w};
    return r;
}
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
static inline unsigned atomicAdd(unsigned* p, unsigned v) { unsigned o = *p; *p = o + v; return o; }
static inline float atomicAdd(float* p, float v) { float o = *p; *p = o + v; return o; }
