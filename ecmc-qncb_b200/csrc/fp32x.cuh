// fp32x.cuh — the FP32 arithmetic types of the kernels.
//
// f1 holds one FP32 value.  Every operator is one IEEE round-to-nearest operation (__fadd_rn,
// __fmul_rn, __fmaf_rn): a multiply and an add are fused only where the source says fma(),
// never by the compiler.  The FP32 kernels compute in f1, so every kernel that shares a piece
// of arithmetic (single-lattice, batched, slab, fused-measurement) rounds it alike, whatever
// the compiler makes of the code around it, and the multiply-adds are the ones written.
//
// Division, square root and reciprocal square root use the FP32 library forms (the
// approximate ones under -prec-div=false / -prec-sqrt=false).
#pragma once
#include <cuda_runtime.h>
#include <type_traits>

namespace qcb {

// The library forms for double (and float), visible next to the f1 overloads below, so
// that calls inside this namespace with those types still resolve to them.
using ::fma;
using ::fmax;
using ::sqrt;

struct f1 {
  float v;
  f1() = default;
  __host__ __device__ constexpr f1(float x) : v(x) {}
  __host__ __device__ constexpr f1(double x) : v((float)x) {}
  __host__ __device__ constexpr f1(int x) : v((float)x) {}
  __host__ __device__ explicit operator double() const { return (double)v; }
  __host__ __device__ explicit operator float() const { return v; }
};

__device__ __forceinline__ f1 operator+(f1 a, f1 b) { return f1(__fadd_rn(a.v, b.v)); }
__device__ __forceinline__ f1 operator-(f1 a, f1 b) { return f1(__fsub_rn(a.v, b.v)); }
__device__ __forceinline__ f1 operator*(f1 a, f1 b) { return f1(__fmul_rn(a.v, b.v)); }
__device__ __forceinline__ f1 operator/(f1 a, f1 b) { return f1(a.v / b.v); }
__device__ __forceinline__ f1 operator-(f1 a) { return f1(-a.v); }
__device__ __forceinline__ f1& operator+=(f1& a, f1 b) { return a = a + b; }
__device__ __forceinline__ f1& operator-=(f1& a, f1 b) { return a = a - b; }
__device__ __forceinline__ bool operator<(f1 a, f1 b) { return a.v < b.v; }
__device__ __forceinline__ bool operator<=(f1 a, f1 b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>(f1 a, f1 b) { return a.v > b.v; }
__device__ __forceinline__ bool operator>=(f1 a, f1 b) { return a.v >= b.v; }
__device__ __forceinline__ f1 fma(f1 a, f1 b, f1 c) { return f1(__fmaf_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ f1 sqrt(f1 a) { return f1(sqrtf(a.v)); }
__device__ __forceinline__ f1 rsqrt_r(f1 a) { return f1(rsqrtf(a.v)); }
__device__ __forceinline__ f1 fmax(f1 a, f1 b) { return f1(fmaxf(a.v, b.v)); }

// FP32 arithmetic types (f1, and plain float where it remains).
template <typename R>
struct is_fp32 : std::false_type {};
template <>
struct is_fp32<float> : std::true_type {};
template <>
struct is_fp32<f1> : std::true_type {};

// Arithmetic type of the kernels for storage type S: FP64 storage computes in double, FP32
// storage in f1.
template <typename S>
struct ArithOf {
  typedef S type;
};
template <>
struct ArithOf<float> {
  typedef f1 type;
};
template <typename S>
using arith_t = typename ArithOf<S>::type;

}  // namespace qcb
