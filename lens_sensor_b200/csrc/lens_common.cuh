// Shared device helpers of the lens_sensor_b200 FDTD kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lens_fdtd.h"

#define LENS_HD __device__ __forceinline__

// Index of profile entry i inside its psi strip array, or -1 outside the strips.
// Strips hold the leading `lo` and trailing `hi` entries of a length-n profile.
LENS_HD int strip_of(int i, int lo, int hi, int n) {
    return i < lo ? i : (i >= n - hi ? lo + (i - (n - hi)) : -1);
}

// Compensated (Kahan) complex accumulation: a = (sum.re, sum.im, carry.re, carry.im).
LENS_HD void kahan_reg(float4 &a, float re, float im) {
    float y = re - a.z;
    float t = a.x + y;
    a.z = (t - a.x) - y;
    a.x = t;
    y = im - a.w;
    t = a.y + y;
    a.w = (t - a.y) - y;
    a.y = t;
}

LENS_HD void kahan_add(float4 *p, float re, float im) {
    float4 a = *p;
    float y = re - a.z;
    float t = a.x + y;
    a.z = (t - a.x) - y;
    a.x = t;
    y = im - a.w;
    t = a.y + y;
    a.w = (t - a.y) - y;
    a.y = t;
    *p = a;
}

LENS_HD double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Add v (per thread) to *acc with one atomic per warp.  All 32 lanes must call.
LENS_HD void warp_atomic_add(double *acc, double v) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(acc, v);
}

// Host-side argument helpers.
static inline bool lens_profile_ok(const LensProfile &p, int n) {
    return p.b && p.c && p.ik && p.n == n && p.lo >= 0 && p.hi >= 0 && p.lo + p.hi <= n;
}

// A psi array must be present wherever its profile has a strip.
static inline bool lens_psi_ok(const LensProfile &p, const void *psi) { return p.lo + p.hi == 0 || psi; }

static inline bool lens_table_ok(const LensStepTable *t, int n0, int nsteps) {
    return t && t->wt && t->env && n0 >= t->t0 && (n0 + nsteps) <= (t->t0 + t->n_table);
}

static inline int lens_cuda_status(void) {
    return cudaGetLastError() == cudaSuccess ? LENS_OK : LENS_ERR_CUDA;
}
