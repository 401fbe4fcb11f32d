// Precision policy for the simulation kernels.
//
// The production build computes gates, currents and the Hines solve in FP32
// (the GPU's fast SFU paths: ex2 / lg2 / rcp), keeps membrane voltage as a
// Kahan-compensated FP32 pair, and accumulates junction sums in FP64.  The
// FP64 build of the same kernel template is the GPU-side oracle run and uses
// the correctly rounded double-precision library functions throughout.
#pragma once
#ifdef __CUDACC_RTC__  // runtime compilation (NVRTC): no host headers
typedef unsigned char uint8_t;
typedef signed char int8_t;
typedef unsigned short uint16_t;
typedef short int16_t;
typedef unsigned int uint32_t;
typedef int int32_t;
typedef unsigned long long uint64_t;
typedef long long int64_t;
#else
#include <cuda_runtime.h>
#include <stdint.h>
#endif

#define NGPU_HD __host__ __device__ __forceinline__

namespace ngpu {

template <typename R> struct Math;

// FP32 uses the SFU approximations on the device; a host build (tests only)
// falls back to the C library.
template <> struct Math<float> {
#ifdef __CUDA_ARCH__
    static NGPU_HD float ex(float x) { return __expf(x); }
    static NGPU_HD float lg(float x) { return __logf(x); }
    static NGPU_HD float dv(float a, float b) { return __fdividef(a, b); }
    static NGPU_HD float rc(float a) { return __fdividef(1.0f, a); }
    static NGPU_HD float pw(float a, float b) { return __powf(a, b); }
    // exp(x) - 1: series below |x| = 1e-2 (truncation < x^5/120), where exp(x) - 1 cancels
    static NGPU_HD float em1(float x) {
        if (fabsf(x) < 1e-2f) return x * (1.0f + x * (0.5f + x * (0.16666667f + x * 0.041666668f)));
        return __expf(x) - 1.0f;
    }
#else
    static NGPU_HD float ex(float x) { return expf(x); }
    static NGPU_HD float lg(float x) { return logf(x); }
    static NGPU_HD float dv(float a, float b) { return a / b; }
    static NGPU_HD float rc(float a) { return 1.0f / a; }
    static NGPU_HD float pw(float a, float b) { return powf(a, b); }
    static NGPU_HD float em1(float x) { return expm1f(x); }
#endif
    // 1 - exp(-z) for z >= 0 without the cancellation 1 - exp(-z) suffers in
    // FP32 when z = dt/tau is small (slow gates, Ca decay): below z = 1/32 the
    // alternating Taylor series z - z^2/2 + z^3/6 - z^4/24 has truncation
    // error < z^5/120 < 3e-10 relative.
    static NGPU_HD float one_minus_exp_neg(float z) {
        if (z < 0.03125f) {
            return z * (1.0f - z * (0.5f - z * (0.16666667f - z * 0.041666668f)));
        }
        return 1.0f - ex(-z);
    }
};

template <> struct Math<double> {
    static NGPU_HD double ex(double x) { return exp(x); }
    static NGPU_HD double lg(double x) { return log(x); }
    static NGPU_HD double dv(double a, double b) { return a / b; }
    static NGPU_HD double rc(double a) { return 1.0 / a; }
    static NGPU_HD double pw(double a, double b) { return pow(a, b); }
    static NGPU_HD double em1(double x) { return expm1(x); }
    static NGPU_HD double one_minus_exp_neg(double z) { return -expm1(-z); }
};

// cnexp update of a first-order gate: x += (1 - exp(-dt/tau)) (xinf - x).
template <typename R>
NGPU_HD R cnexp(R x, R xinf, R tau, R dt) {
    return x + Math<R>::one_minus_exp_neg(Math<R>::dv(dt, tau)) * (xinf - x);
}

// Physical constants shared by the generated channel libraries.
constexpr double kFaraday = 96485.309;
constexpr double kDefCai = 5.e-5;
constexpr double kDefCao = 2.;
__host__ __device__ constexpr double ktf_of(double celsius) {
    return 1000. * 8.3134 * (celsius + 273.15) / kFaraday;
}

}  // namespace ngpu
