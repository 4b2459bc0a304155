/* ORACLE build shim (test infrastructure only), force-included when compiling
 * the engine's non-bonded pair functions (NonBondedInteraction.h, built with
 * DEVICE_CODE) as host code: the CUDA runtime header supplies the vector types
 * the engine's defines use, and the binary32 intrinsics become their IEEE host
 * equivalents (__cosf, __sinf, __logf and __expf, fast approximations on the
 * GPU, become cosf, sinf, logf and expf). */
#ifndef ORACLE_NB_PRELUDE_H
#define ORACLE_NB_PRELUDE_H
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
static inline float __fdiv_rn(float a, float b) { return a / b; }
static inline float __frcp_rn(float a) { return 1.f / a; }
static inline float __logf(float a) { return logf(a); }
static inline float __cosf(float a) { return cosf(a); }
static inline float __sinf(float a) { return sinf(a); }
static inline float __expf(float a) { return expf(a); }
#endif
