// su3.cuh — device-side complex / 3x3 complex matrix arithmetic for the SU(3) kernels.
//
// The reference carries this arithmetic in Eigen::Matrix<std::complex<double>,3,3,RowMajor>
// (src/su3/utils.h:12); here it is plain register arrays so that the compiler keeps every
// element in registers.  R is the arithmetic type: double, or the explicitly rounded FP32
// type f1 (fp32x.cuh), for which every multiply-add is the fma() written here.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp32x.cuh"

namespace qcb {

template <typename R>
struct cx {
  R re, im;
};

template <typename R>
__device__ __forceinline__ cx<R> mk(R re, R im) {
  cx<R> c;
  c.re = re;
  c.im = im;
  return c;
}
template <typename R>
__device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) { return mk(a.re + b.re, a.im + b.im); }
template <typename R>
__device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) { return mk(a.re - b.re, a.im - b.im); }
template <typename R>
__device__ __forceinline__ cx<R> operator*(cx<R> a, cx<R> b) {
  return mk(fma(a.re, b.re, -(a.im * b.im)), fma(a.re, b.im, a.im * b.re));
}
template <typename R>
__device__ __forceinline__ cx<R> operator*(R s, cx<R> a) { return mk(s * a.re, s * a.im); }
template <typename R>
__device__ __forceinline__ cx<R> conj(cx<R> a) { return mk(a.re, -a.im); }
// acc - a*b
template <typename R>
__device__ __forceinline__ cx<R> cfms(cx<R> a, cx<R> b, cx<R> acc) {
  acc.re = fma(-a.re, b.re, acc.re);
  acc.re = fma(a.im, b.im, acc.re);
  acc.im = fma(-a.re, b.im, acc.im);
  acc.im = fma(-a.im, b.re, acc.im);
  return acc;
}
// acc + a*b
template <typename R>
__device__ __forceinline__ cx<R> cfma(cx<R> a, cx<R> b, cx<R> acc) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(-a.im, b.im, acc.re);
  acc.im = fma(a.re, b.im, acc.im);
  acc.im = fma(a.im, b.re, acc.im);
  return acc;
}
// acc + conj(a)*b
template <typename R>
__device__ __forceinline__ cx<R> cfma_cn(cx<R> a, cx<R> b, cx<R> acc) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(a.im, b.im, acc.re);
  acc.im = fma(a.re, b.im, acc.im);
  acc.im = fma(-a.im, b.re, acc.im);
  return acc;
}
// acc + a*conj(b)
template <typename R>
__device__ __forceinline__ cx<R> cfma_nc(cx<R> a, cx<R> b, cx<R> acc) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(a.im, b.im, acc.re);
  acc.im = fma(-a.re, b.im, acc.im);
  acc.im = fma(a.im, b.re, acc.im);
  return acc;
}
// acc + conj(a)*conj(b)
template <typename R>
__device__ __forceinline__ cx<R> cfma_cc(cx<R> a, cx<R> b, cx<R> acc) {
  acc.re = fma(a.re, b.re, acc.re);
  acc.re = fma(-a.im, b.im, acc.re);
  acc.im = fma(-a.re, b.im, acc.im);
  acc.im = fma(-a.im, b.re, acc.im);
  return acc;
}

template <typename R>
struct m3 {
  cx<R> e[3][3];
};

template <typename R>
__device__ __forceinline__ void set_zero(m3<R>& a) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) a.e[i][j] = mk<R>(0, 0);
}
template <typename R>
__device__ __forceinline__ void set_identity(m3<R>& a) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) a.e[i][j] = mk<R>(i == j ? R(1) : R(0), 0);
}

// c = a * b
template <typename R>
__device__ __forceinline__ m3<R> mul_nn(const m3<R>& a, const m3<R>& b) {
  m3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = a.e[i][0] * b.e[0][j];
      s = cfma(a.e[i][1], b.e[1][j], s);
      s = cfma(a.e[i][2], b.e[2][j], s);
      c.e[i][j] = s;
    }
  return c;
}
// c = a * b^dagger
template <typename R>
__device__ __forceinline__ m3<R> mul_na(const m3<R>& a, const m3<R>& b) {
  m3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = mk<R>(0, 0);
      s = cfma_nc(a.e[i][0], b.e[j][0], s);
      s = cfma_nc(a.e[i][1], b.e[j][1], s);
      s = cfma_nc(a.e[i][2], b.e[j][2], s);
      c.e[i][j] = s;
    }
  return c;
}
// c = a^dagger * b
template <typename R>
__device__ __forceinline__ m3<R> mul_an(const m3<R>& a, const m3<R>& b) {
  m3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = mk<R>(0, 0);
      s = cfma_cn(a.e[0][i], b.e[0][j], s);
      s = cfma_cn(a.e[1][i], b.e[1][j], s);
      s = cfma_cn(a.e[2][i], b.e[2][j], s);
      c.e[i][j] = s;
    }
  return c;
}
// c = a^dagger * b^dagger
template <typename R>
__device__ __forceinline__ m3<R> mul_aa(const m3<R>& a, const m3<R>& b) {
  m3<R> c;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = mk<R>(0, 0);
      s = cfma_cc(a.e[0][i], b.e[j][0], s);
      s = cfma_cc(a.e[1][i], b.e[j][1], s);
      s = cfma_cc(a.e[2][i], b.e[j][2], s);
      c.e[i][j] = s;
    }
  return c;
}
// acc += a * b
template <typename R>
__device__ __forceinline__ void acc_nn(m3<R>& acc, const m3<R>& a, const m3<R>& b) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = acc.e[i][j];
      s = cfma(a.e[i][0], b.e[0][j], s);
      s = cfma(a.e[i][1], b.e[1][j], s);
      s = cfma(a.e[i][2], b.e[2][j], s);
      acc.e[i][j] = s;
    }
}
// acc += a * b^dagger
template <typename R>
__device__ __forceinline__ void acc_na(m3<R>& acc, const m3<R>& a, const m3<R>& b) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = acc.e[i][j];
      s = cfma_nc(a.e[i][0], b.e[j][0], s);
      s = cfma_nc(a.e[i][1], b.e[j][1], s);
      s = cfma_nc(a.e[i][2], b.e[j][2], s);
      acc.e[i][j] = s;
    }
}
// acc += a^dagger * b
template <typename R>
__device__ __forceinline__ void acc_an(m3<R>& acc, const m3<R>& a, const m3<R>& b) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = acc.e[i][j];
      s = cfma_cn(a.e[0][i], b.e[0][j], s);
      s = cfma_cn(a.e[1][i], b.e[1][j], s);
      s = cfma_cn(a.e[2][i], b.e[2][j], s);
      acc.e[i][j] = s;
    }
}
// acc += a^dagger * b^dagger
template <typename R>
__device__ __forceinline__ void acc_aa(m3<R>& acc, const m3<R>& a, const m3<R>& b) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = acc.e[i][j];
      s = cfma_cc(a.e[0][i], b.e[j][0], s);
      s = cfma_cc(a.e[1][i], b.e[j][1], s);
      s = cfma_cc(a.e[2][i], b.e[j][2], s);
      acc.e[i][j] = s;
    }
}
// Rows 0 and 1 of a * b^dagger (only rows 0 and 1 of a are read; row 2 of c is unset).
template <typename R>
__device__ __forceinline__ m3<R> mul_na_rows01(const m3<R>& a, const m3<R>& b) {
  m3<R> c;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = mk<R>(0, 0);
      s = cfma_nc(a.e[i][0], b.e[j][0], s);
      s = cfma_nc(a.e[i][1], b.e[j][1], s);
      s = cfma_nc(a.e[i][2], b.e[j][2], s);
      c.e[i][j] = s;
    }
  return c;
}
// Rows 0 and 1 of a * b (only rows 0 and 1 of a are read; row 2 of c is unset).
template <typename R>
__device__ __forceinline__ m3<R> mul_nn_rows01(const m3<R>& a, const m3<R>& b) {
  m3<R> c;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> s = a.e[i][0] * b.e[0][j];
      s = cfma(a.e[i][1], b.e[1][j], s);
      s = cfma(a.e[i][2], b.e[2][j], s);
      c.e[i][j] = s;
    }
  return c;
}
// acc += w; acc += w^dagger
template <typename R>
__device__ __forceinline__ void add_m3(m3<R>& acc, const m3<R>& w) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) acc.e[i][j] = acc.e[i][j] + w.e[i][j];
}
template <typename R>
__device__ __forceinline__ void add_m3_adj(m3<R>& acc, const m3<R>& w) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) acc.e[i][j] = acc.e[i][j] + conj(w.e[j][i]);
}
// Re tr(a * b)
template <typename R>
__device__ __forceinline__ R re_tr_nn(const m3<R>& a, const m3<R>& b) {
  R s = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) s = fma(a.e[i][k].re, b.e[k][i].re, fma(-a.e[i][k].im, b.e[k][i].im, s));
  return s;
}
// Re tr(a * b^dagger) = sum_ij Re(a_ij conj(b_ij))
template <typename R>
__device__ __forceinline__ R re_tr_na(const m3<R>& a, const m3<R>& b) {
  R s = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) s = fma(a.e[i][j].re, b.e[i][j].re, fma(a.e[i][j].im, b.e[i][j].im, s));
  return s;
}

// conj(a b - c d), four multiply-adds per component.
template <typename R>
__device__ __forceinline__ cx<R> conj_diff(cx<R> a, cx<R> b, cx<R> c, cx<R> d) {
  // Re(ab - cd) = a.re b.re - a.im b.im - c.re d.re + c.im d.im
  // -Im(ab - cd) = -a.re b.im - a.im b.re + c.re d.im + c.im d.re
  return mk(fma(a.re, b.re, fma(-a.im, b.im, fma(-c.re, d.re, c.im * d.im))),
            fma(-a.re, b.im, fma(-a.im, b.re, fma(c.re, d.im, c.im * d.re))));
}

// Third row of an SU(3) matrix from its first two: r2 = conj(r0 x r1).
template <typename R>
__device__ __forceinline__ void reconstruct_row2(m3<R>& u) {
  u.e[2][0] = conj_diff(u.e[0][1], u.e[1][2], u.e[0][2], u.e[1][1]);
  u.e[2][1] = conj_diff(u.e[0][2], u.e[1][0], u.e[0][0], u.e[1][2]);
  u.e[2][2] = conj_diff(u.e[0][0], u.e[1][1], u.e[0][1], u.e[1][0]);
}

__device__ __forceinline__ double rsqrt_r(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }

// Gram-Schmidt on rows 0 and 1, then row 2 = conj(row0 x row1), in the arithmetic of R.
template <typename R>
__device__ __forceinline__ void reunitarize_rows(m3<R>& u) {
  R n0 = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j) n0 = fma(u.e[0][j].re, u.e[0][j].re, fma(u.e[0][j].im, u.e[0][j].im, n0));
  R inv0 = rsqrt_r(n0);
#pragma unroll
  for (int j = 0; j < 3; ++j) u.e[0][j] = inv0 * u.e[0][j];
  // <r0, r1> = sum conj(r0_j) r1_j
  cx<R> d = mk<R>(0, 0);
#pragma unroll
  for (int j = 0; j < 3; ++j) d = cfma_cn(u.e[0][j], u.e[1][j], d);
#pragma unroll
  for (int j = 0; j < 3; ++j) u.e[1][j] = cfms(d, u.e[0][j], u.e[1][j]);
  R n1 = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j) n1 = fma(u.e[1][j].re, u.e[1][j].re, fma(u.e[1][j].im, u.e[1][j].im, n1));
  R inv1 = rsqrt_r(n1);
#pragma unroll
  for (int j = 0; j < 3; ++j) u.e[1][j] = inv1 * u.e[1][j];
  reconstruct_row2(u);
}

template <typename R2, typename R>
__device__ __forceinline__ m3<R2> convert(const m3<R>& a) {
  m3<R2> b;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) b.e[i][j] = mk<R2>(R2(a.e[i][j].re), R2(a.e[i][j].im));
  return b;
}

// ---- su(3) algebra elements: traceless anti-Hermitian, 8 reals ----------------------
// a[0], a[1]: imaginary parts of the diagonal entries 0 and 1 (entry 2 = -(a0+a1));
// a[2..7]: (re, im) of the upper off-diagonal entries (0,1), (0,2), (1,2).
template <typename R>
struct alg8 {
  R a[8];
};

template <typename R>
__device__ __forceinline__ alg8<R> alg_from_ta(const m3<R>& m) {
  alg8<R> z;
  z.a[0] = m.e[0][0].im;
  z.a[1] = m.e[1][1].im;
  z.a[2] = m.e[0][1].re;
  z.a[3] = m.e[0][1].im;
  z.a[4] = m.e[0][2].re;
  z.a[5] = m.e[0][2].im;
  z.a[6] = m.e[1][2].re;
  z.a[7] = m.e[1][2].im;
  return z;
}
template <typename R>
__device__ __forceinline__ m3<R> alg_to_m3(const alg8<R>& z) {
  m3<R> m;
  m.e[0][0] = mk<R>(0, z.a[0]);
  m.e[1][1] = mk<R>(0, z.a[1]);
  m.e[2][2] = mk<R>(0, -(z.a[0] + z.a[1]));
  m.e[0][1] = mk<R>(z.a[2], z.a[3]);
  m.e[0][2] = mk<R>(z.a[4], z.a[5]);
  m.e[1][2] = mk<R>(z.a[6], z.a[7]);
  m.e[1][0] = mk<R>(-z.a[2], z.a[3]);
  m.e[2][0] = mk<R>(-z.a[4], z.a[5]);
  m.e[2][1] = mk<R>(-z.a[6], z.a[7]);
  return m;
}

// Traceless anti-Hermitian projection (A - A^dagger)/2 - tr/3, returned as 8 reals.
// Reference: proj_lie_su3 (src/su3/utils.cpp:130-134).
template <typename R>
__device__ __forceinline__ alg8<R> proj_ta(const m3<R>& m) {
  alg8<R> z;
  R d0 = m.e[0][0].im, d1 = m.e[1][1].im, d2 = m.e[2][2].im;
  R tr3 = (d0 + d1 + d2) * R(1.0 / 3.0);
  z.a[0] = d0 - tr3;
  z.a[1] = d1 - tr3;
  z.a[2] = R(0.5) * (m.e[0][1].re - m.e[1][0].re);
  z.a[3] = R(0.5) * (m.e[0][1].im + m.e[1][0].im);
  z.a[4] = R(0.5) * (m.e[0][2].re - m.e[2][0].re);
  z.a[5] = R(0.5) * (m.e[0][2].im + m.e[2][0].im);
  z.a[6] = R(0.5) * (m.e[1][2].re - m.e[2][1].re);
  z.a[7] = R(0.5) * (m.e[1][2].im + m.e[2][1].im);
  return z;
}

// exp(X) for X in su(3) by Luescher's Cayley-Hamilton / Horner recursion with N = 18
// Taylor terms (reference: exp_su3_luscher, src/su3/utils.cpp:145-193):
// exp(X) = q0 + q1 X + q2 X^2.  The invariants t = -tr(X^2)/2, d = Re(i det X) and the
// coefficients q0, q1, q2 are always evaluated in FP64 (exp_coef64, from the 8 reals of X);
// the matrix X and the result are in R.
__device__ __forceinline__ void exp_coef64(const double (&xa)[8], double (&q)[6]) {
  double d0 = xa[0], d1 = xa[1], d2 = -(xa[0] + xa[1]);
  double ar = xa[2], ai = xa[3];  // X01
  double br = xa[4], bi = xa[5];  // X02
  double cr = xa[6], ci = xa[7];  // X12
  // t = -1/2 tr X^2 = 1/2 sum_ij |X_ij|^2 for anti-Hermitian X.
  double t = 0.5 * (d0 * d0 + d1 * d1 + d2 * d2) + (ar * ar + ai * ai + br * br + bi * bi + cr * cr + ci * ci);
  // det X with X = [[i d0, a, b], [-a*, i d1, c], [-b*, -c*, i d2]]:
  // det = i d0 (i d1 i d2 + |c|^2) - a (-a* i d2 + c b*) + b (a* c* + i d1 b*)
  // d = Re(i det X) = -Im(det X).
  // i d0 * (-d1 d2 + |c|^2)  -> imaginary part d0 (|c|^2 - d1 d2)
  double im_det = d0 * (cr * cr + ci * ci - d1 * d2);
  // -a * (-a* i d2) = i d2 |a|^2 -> imaginary part d2 |a|^2
  im_det += d2 * (ar * ar + ai * ai);
  // -a * c * b*: im part of -(a c conj(b))
  {
    double acr = ar * cr - ai * ci, aci = ar * ci + ai * cr;  // a*c
    double pim = aci * br - acr * bi;                         // Im((a c) conj(b))
    im_det -= pim;
    // b * a* * c*: Im(b conj(a) conj(c)) = Im(conj(a c conj(b))) = -pim
    im_det += -pim;
  }
  // b * i d1 b* = i d1 |b|^2
  im_det += d1 * (br * br + bi * bi);
  double dd = -im_det;
  // Horner recursion over n = N-1..0 with c_n = 1/n!.
  const int N = 18;
  double cn[N + 1];
  cn[0] = 1.0;
#pragma unroll
  for (int n = 1; n <= N; ++n) cn[n] = cn[n - 1] / double(n);
  double q0r = cn[N], q0i = 0.0, q1r = 0.0, q1i = 0.0, q2r = 0.0, q2i = 0.0;
#pragma unroll
  for (int n = N - 1; n >= 0; --n) {
    // q0' = c_n - i d q2 ; q1' = q0 - t q2 ; q2' = q1
    double n0r = cn[n] + dd * q2i, n0i = -dd * q2r;
    double n1r = q0r - t * q2r, n1i = q0i - t * q2i;
    q2r = q1r;
    q2i = q1i;
    q0r = n0r;
    q0i = n0i;
    q1r = n1r;
    q1i = n1i;
  }
  q[0] = q0r;
  q[1] = q0i;
  q[2] = q1r;
  q[3] = q1i;
  q[4] = q2r;
  q[5] = q2i;
}

// q0, q1, q2 of exp(X) in R.
template <typename R>
__device__ __forceinline__ void exp_coef(const alg8<R>& x, cx<R>& q0, cx<R>& q1, cx<R>& q2) {
  double xa[8], q[6];
#pragma unroll
  for (int k = 0; k < 8; ++k) xa[k] = (double)x.a[k];
  exp_coef64(xa, q);
  q0 = mk<R>(R(q[0]), R(q[1]));
  q1 = mk<R>(R(q[2]), R(q[3]));
  q2 = mk<R>(R(q[4]), R(q[5]));
}

// Returns exp(X).
template <typename R>
__device__ __forceinline__ m3<R> exp_su3(const alg8<R>& x) {
  cx<R> q0, q1, q2;
  exp_coef(x, q0, q1, q2);
  m3<R> X = alg_to_m3(x);
  // X^2 is Hermitian (X^dag = -X); its entries in closed form from the 8 reals
  // (d2 = -d0 - d1; a = X01, b = X02, c = X12):
  //   (X^2)_kk = -(d_k^2 + sum of |off-diagonal|^2 in row k),
  //   (X^2)_01 = -i d2 a - b c*, (X^2)_02 = -i d1 b + a c, (X^2)_12 = -i d0 c - a* b.
  m3<R> X2;
  {
    const R D0 = x.a[0], D1 = x.a[1], D2 = -(x.a[0] + x.a[1]);
    const R Ar = x.a[2], Ai = x.a[3], Br = x.a[4], Bi = x.a[5], Cr = x.a[6], Ci = x.a[7];
    const R na = fma(Ar, Ar, Ai * Ai), nb = fma(Br, Br, Bi * Bi), nc = fma(Cr, Cr, Ci * Ci);
    X2.e[0][0] = mk<R>(-fma(D0, D0, na + nb), R(0));
    X2.e[1][1] = mk<R>(-fma(D1, D1, na + nc), R(0));
    X2.e[2][2] = mk<R>(-fma(D2, D2, nb + nc), R(0));
    // s01 = (D2 Ai - Br Cr - Bi Ci, -D2 Ar - Bi Cr + Br Ci)
    const cx<R> s01 = mk<R>(fma(D2, Ai, fma(-Br, Cr, -(Bi * Ci))), fma(-D2, Ar, fma(-Bi, Cr, Br * Ci)));
    // s02 = (D1 Bi + Ar Cr - Ai Ci, -D1 Br + Ar Ci + Ai Cr)
    const cx<R> s02 = mk<R>(fma(D1, Bi, fma(Ar, Cr, -(Ai * Ci))), fma(-D1, Br, fma(Ar, Ci, Ai * Cr)));
    // s12 = (D0 Ci - Ar Br - Ai Bi, -D0 Cr - Ar Bi + Ai Br)
    const cx<R> s12 = mk<R>(fma(D0, Ci, fma(-Ar, Br, -(Ai * Bi))), fma(-D0, Cr, fma(-Ar, Bi, Ai * Br)));
    X2.e[0][1] = s01;
    X2.e[0][2] = s02;
    X2.e[1][2] = s12;
    X2.e[1][0] = conj(s01);
    X2.e[2][0] = conj(s02);
    X2.e[2][1] = conj(s12);
  }
  m3<R> E;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cx<R> v;
      if (i == j) {
        // X_ii = i d_i is imaginary and (X^2)_ii real: the products with their zero parts
        // (which leave the sums unchanged) are left out
        v = mk<R>(fma(q2.re, X2.e[i][i].re, -(q1.im * X.e[i][i].im)), fma(q2.im, X2.e[i][i].re, q1.re * X.e[i][i].im));
        v = v + q0;
      } else {
        v = q1 * X.e[i][j];
        v = cfma(q2, X2.e[i][j], v);
      }
      E.e[i][j] = v;
    }
  return E;
}

}  // namespace qcb
