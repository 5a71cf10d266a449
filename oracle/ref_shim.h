/*
 * Host shim for compiling the reference's own force kernels as plain C++ (the
 * checker of the oracle; test infrastructure only, never part of the product).
 *
 * oracle/refbuild.py extracts the reference's functions unmodified into
 * oracle/_ref/src/ref_pieces{32,64}.inc; this header supplies what its translation
 * unit (src/fenzi.cu with src/globals.h, src/defs.h) would have supplied on the GPU:
 *   - CUDA qualifiers as nothing, the vector types float2/3/4 and int2/3/4, and the
 *     thread coordinates (one host loop iteration = one GPU thread);
 *   - texture fetches tex1Dfetch(tex, i) as reads of plain host arrays;
 *   - the __constant__ device symbols the kernels read (src/globals.h:590-685) as
 *     host globals, set by oracle/ref_harness.cpp;
 *   - the GPU intrinsics as host arithmetic: __fdividef(a, b) = a / b,
 *     rsqrtf(x) = rsqrt(x) = 1 / sqrt(x).
 * FZREF_VARIANT 64 compiles every `float` of the reference's statements as double
 * (with the literal suffixes dropped by the extractor) and maps the float math calls
 * to their double forms, so the reference's formulas can be compared with the FP64
 * oracle to rounding level; FZREF_VARIANT 32 keeps the reference's FP32 arithmetic.
 * The reference's own macro definitions it needs (src/defs.in.h: the __my_* helpers,
 * CC and the Ewald constants, NBPART/BPART, NBXMOD, the feature switches) are
 * extracted from src/defs.in.h by the recipe into ref_defs{32,64}.inc.
 */
#ifndef FZREF_SHIM_H
#define FZREF_SHIM_H
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#if FZREF_VARIANT == 64
typedef double fzref_real;
#else
typedef float fzref_real;
#endif

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __constant__
#define HOSTDEVICE static inline

struct float2 { fzref_real x, y; };
struct float3 { fzref_real x, y, z; };
struct float4 { fzref_real x, y, z, w; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct int4 { int x, y, z, w; };
typedef float2 cufftComplex;

static inline float2 make_float2(fzref_real x, fzref_real y) { return float2{x, y}; }
static inline float3 make_float3(fzref_real x, fzref_real y, fzref_real z) { return float3{x, y, z}; }
static inline float4 make_float4(fzref_real x, fzref_real y, fzref_real z, fzref_real w) {
  return float4{x, y, z, w};
}

/* thread coordinates of the host loop that stands for a launch */
struct fzref_dim3 { unsigned x, y, z; };
extern fzref_dim3 threadIdx, blockIdx, blockDim, gridDim;

#define tex1Dfetch(tex, i) ((tex)[(i)])
/* host-side CUDA runtime calls of InitDeviceConstants: symbols and "device" buffers
 * are host arrays here, texture binding and error checks do nothing */
#define cudaMemcpyToSymbol(sym, src, bytes) memcpy((void*)&(sym), (src), (bytes))
#define cudaMemcpy(dst, src, bytes, kind) memcpy((dst), (src), (bytes))
#define cudaMemcpyHostToDevice 0
#define cudaBindTexture(...) 0
#define checkCUDAError(msg) ((void)0)

#if FZREF_VARIANT == 64
static inline double __fdividef(double a, double b) { return a / b; }
static inline double rsqrtf(double x) { return 1.0 / std::sqrt(x); }
static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
#define sqrtf sqrt
#define acosf acos
#define sinf sin
#define cosf cos
#define asinf asin
#define expf exp
#define erff erf
#define erfcf erfc
#define copysignf copysign
#else
static inline float __fdividef(float a, float b) { return a / b; }
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
static inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
#endif

/* src/globals.h:590-685 constant symbols read by the kernels compiled here */
extern fzref_real beta, betaSqr, cutoffd, Cutond, Swcoeff1d, Swcoeff2d, Swcoeff3d;
extern int WorkgroupSized, num_types_presentd, Angle_Countd, Dihed_Countd, Improper_Countd;
extern float4 boxH;
/* texture references (src/globals.h:760-794) as host arrays */
extern const float4* texcrd;
extern const int* textype;
extern const float2* texprm1_4;
extern const float2* texnbfixprm;

#endif
