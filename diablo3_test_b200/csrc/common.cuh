// Shared device helpers: complex arithmetic on double2/float2 and the
// precision traits used by every kernel of libdiablo_gpu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DI __device__ __forceinline__
#define HDI __host__ __device__ __forceinline__

// ---- complex arithmetic -------------------------------------------------
HDI double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
HDI double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
HDI double2 operator-(double2 a) { return make_double2(-a.x, -a.y); }
HDI double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
HDI float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
HDI float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
HDI float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
HDI float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }

HDI double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
HDI float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
HDI double2 conj(double2 a) { return make_double2(a.x, -a.y); }
HDI float2 conj(float2 a) { return make_float2(a.x, -a.y); }
// i * a
HDI double2 mul_i(double2 a) { return make_double2(-a.y, a.x); }
HDI float2 mul_i(float2 a) { return make_float2(-a.y, a.x); }
// (0, k) * a, the reference's cikx(i)*a with cikx = ci*kx (for/fft.f90:217)
HDI double2 mul_ik(double k, double2 a) { return make_double2(-k * a.y, k * a.x); }
HDI float2 mul_ik(float k, float2 a) { return make_float2(-k * a.y, k * a.x); }

// ---- precision traits -------------------------------------------------------
template <typename T> struct CT;
template <> struct CT<double> {
  typedef double2 C;
  HDI static double2 mk(double x, double y) { return make_double2(x, y); }
};
template <> struct CT<float> {
  typedef float2 C;
  HDI static float2 mk(float x, float y) { return make_float2(x, y); }
};

template <typename C> struct CReal;
template <> struct CReal<double2> { typedef double R; };
template <> struct CReal<float2> { typedef float R; };

// conversions between storage and compute precision
HDI double2 to_c2(double2 a, double2*) { return a; }
HDI float2 to_c2(double2 a, float2*) { return make_float2((float)a.x, (float)a.y); }
HDI double2 to_c2(float2 a, double2*) { return make_double2(a.x, a.y); }
HDI float2 to_c2(float2 a, float2*) { return a; }
template <typename CTo, typename CFrom> HDI CTo cvt(CFrom a) { return to_c2(a, (CTo*)nullptr); }

template <typename C> HDI C czero() { C z; z.x = 0; z.y = 0; return z; }

// fields of the dynamic Smagorinsky model's Germano/Lilly contraction
// (k_dyn_prep builds them, the LES work arrays hold them)
#define DYN_NF 21
