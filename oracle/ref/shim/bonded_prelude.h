/* ORACLE build shim (test infrastructure only), force-included when compiling
 * the engine's bonded-force headers as host code: CUDA qualifiers become empty
 * and the binary32 intrinsics their IEEE host equivalents (__logf, a fast
 * approximation on the GPU, becomes logf). */
#ifndef ORACLE_BONDED_PRELUDE_H
#define ORACLE_BONDED_PRELUDE_H
#include <cmath>
#include <cstdio>
#include <cstdlib>
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
static inline float __fdiv_rn(float a, float b) { return a / b; }
static inline float __frcp_rn(float a) { return 1.f / a; }
static inline float __logf(float a) { return logf(a); }
#endif
