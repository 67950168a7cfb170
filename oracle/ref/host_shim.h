/* Host shim that lets the reference's own transport kernel source
 * (MCGPU-PET_kernel.cu + MCGPU-PET.h) compile as plain host C++ with g++.
 *
 * TEST INFRASTRUCTURE ONLY.  It is force-included (g++ -include) in front of
 * the reference files where they lie; the resulting library under oracle/_ref
 * is the timed CPU baseline ("reference" kind) and a pin for the C
 * restatement in oracle/mcpet_oracle.c.  The product never links it.
 *
 * Semantics mirrored from CUDA:
 *   - __float2int_rd takes a float, so a double argument is first rounded to
 *     float exactly as the device call does, then floored.
 *   - __double2ull_rn / __float2ull_rn round to nearest and saturate to
 *     [0, 2^64-1] with NaN -> 0, like cvt.rni.u64.
 *   - atomicAdd is a relaxed host atomic; the address of the last few atomic
 *     targets of each host thread is recorded so a harness can recover the
 *     sinogram bin an event was tallied into.
 */
#pragma once
#include <math.h>
#include <stdint.h>
#include <limits.h>
#include <stdio.h>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ static thread_local
#define __forceinline__ inline

struct shim_dim3 { unsigned int x, y, z; };
extern thread_local shim_dim3 threadIdx, blockIdx, blockDim, gridDim;

static inline void __syncthreads(void) {}

static inline int __float2int_rd(float x) { return (int)floorf(x); }
static inline float __int2float_rn(int x) { return (float)x; }
static inline double __int2double_rn(int x) { return (double)x; }
static inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }

static inline unsigned long long shim_sat_u64(double r) {
  if (!(r == r)) return 0ull;              /* NaN */
  if (r <= 0.0) return 0ull;
  if (r >= 18446744073709551616.0) return ULLONG_MAX;
  return (unsigned long long)r;
}
static inline unsigned long long __double2ull_rn(double x) { return shim_sat_u64(nearbyint(x)); }
static inline unsigned long long __float2ull_rn(float x) { return shim_sat_u64(nearbyint((double)x)); }

/* Per-host-thread record of atomic targets (for index harnesses). */
#define SHIM_MAX_CAPTURE 8
extern thread_local void* shim_capture[SHIM_MAX_CAPTURE];
extern thread_local int shim_ncapture;
static inline void shim_record(void* p) {
  if (shim_ncapture < SHIM_MAX_CAPTURE) shim_capture[shim_ncapture++] = p;
}
static inline int atomicAdd(int* p, int v) {
  shim_record(p);
  return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}
static inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
  shim_record(p);
  return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}
