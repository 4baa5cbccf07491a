// k_ecmc.cu — event-chain Monte Carlo: every l_core^4 block runs its own persistent chain,
// on one, three or six lanes of a warp, all chains of the lattice in one launch.
//
// The reference runs one chain per MPI rank (mpi::ecmccb::sample_persistant,
// src/ecmc/ecmc_mpi_cb.cpp:496-637) on a padded block whose halo and low faces are frozen
// (src/geometry/GeometryCB.cpp:33-56).  Every link a chain reads outside its own active
// links is frozen in the block that owns it, so no chain ever reads a link that another
// chain writes, and the chains of all blocks can run at the same time.  Links are read and
// written in an FP64 array-of-structures copy of the lattice (one link = 9 consecutive
// double2, 144 contiguous bytes): a chain touches scattered links, and a contiguous link
// costs 5 DRAM sectors where the structure-of-arrays layout costs 9.
//
// Random numbers: chain c's k-th uniform is Philox4x32-10 with counter (k_lo, k_hi, c,
// ECMC_CHAIN) and key seed.  Each chain has its own set of near-identity elements, as each
// rank of the reference has, renewed at the start of every call and whenever its set_counter
// (lifts since the last renewal) is a multiple of 10000 at the top of the event loop
// (ecmc_mpi_cb.cpp:560-566); the set is never stored: element pair p of generation gen comes
// from counters (3p + j, c, call, ECMC_SETC ^ gen), j < 3, when a lift picks it.  The
// arithmetic is the reference's up to the order of the floating-point operations (products
// streamed by rows, dS as a trace against R diag(1, -1, 0) R^dagger), so the CPU oracle, drawing from the same counters, takes the
// same events with links equal to rounding.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "ecmc.h"
#include "philox.cuh"
#include "su3.cuh"

namespace qcb {
namespace {

constexpr uint32_t ECMC_CHAIN = 0xECEC0001u, ECMC_SETC = 0xECE50000u;
constexpr uint64_t ECMC_MAX_EVENTS = 1ull << 26;
constexpr double PI = 3.141592653589793;  // the double nearest pi
// Sample kernel blocks: two warps.  Register caps: none (255 per thread), or ECMC_CAPPED
// blocks of 64 threads per SM (168 per thread).
constexpr int ECMC_WARPS = 2, ECMC_CAPPED = 6;

typedef m3<double> M;
typedef cx<double> Z;

// The file is compiled without automatic contraction (-fmad=false) and the products of the
// event loop use these explicit fused multiply-adds, so that every instantiation of the
// sample kernel (one, three or six lanes per chain) rounds every operation the same way.
__device__ __forceinline__ Z cmul(Z a, Z b) { return mk(fma(a.re, b.re, -(a.im * b.im)), fma(a.re, b.im, a.im * b.re)); }
// acc + a b
__device__ __forceinline__ Z cfma(Z a, Z b, Z acc) {
  return mk(fma(a.re, b.re, fma(-a.im, b.im, acc.re)), fma(a.re, b.im, fma(a.im, b.re, acc.im)));
}
// a0 b0 + a1 b1 + a2 b2
__device__ __forceinline__ Z cdot3(Z a0, Z b0, Z a1, Z b1, Z a2, Z b2) { return cfma(a2, b2, cfma(a1, b1, cmul(a0, b0))); }

// Uniform in (0, 1) from two 32-bit words: (top 53 bits of hi:lo + 1/2) 2^-53.
__device__ __forceinline__ double u53(uint32_t lo, uint32_t hi) {
  const uint64_t x = ((((uint64_t)hi) << 32) | lo) >> 11;
  return ((double)x + 0.5) * 1.1102230246251565e-16;
}

// The k-th uniform of chain `chain` (one copy of the Philox rounds in the kernel: the
// generator has two dozen call sites, and inlining each one overflowed the instruction cache).
__device__ __noinline__ double chain_uniform(uint32_t chain, uint32_t k0, uint32_t k1, uint64_t k) {
  u32x4 c;
  c.v[0] = (uint32_t)k;
  c.v[1] = (uint32_t)(k >> 32);
  c.v[2] = chain;
  c.v[3] = ECMC_CHAIN;
  const u32x4 r = philox4x32_10(c, k0, k1);
  return u53(r.v[0], r.v[1]);
}

struct Stream {
  uint32_t chain, k0, k1;
  uint64_t n;
  __device__ __forceinline__ double uni() { return chain_uniform(chain, k0, k1, n++); }
};

// SU(3) from 12 standard normals: rows 0, 1 complex Gaussian, Gram-Schmidt, row 2 =
// conj(row0 x row1) (Haar-distributed).
__device__ M haar_from_normals(const double n[12]) {
  Z r0[3], r1[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    r0[j] = mk(n[2 * j], n[2 * j + 1]);
    r1[j] = mk(n[6 + 2 * j], n[6 + 2 * j + 1]);
  }
  const double s0 = sqrt(r0[0].re * r0[0].re + r0[0].im * r0[0].im + r0[1].re * r0[1].re + r0[1].im * r0[1].im +
                         r0[2].re * r0[2].re + r0[2].im * r0[2].im);
#pragma unroll
  for (int j = 0; j < 3; ++j) r0[j] = mk(r0[j].re / s0, r0[j].im / s0);
  Z d = conj(r0[0]) * r1[0] + conj(r0[1]) * r1[1] + conj(r0[2]) * r1[2];
#pragma unroll
  for (int j = 0; j < 3; ++j) r1[j] = r1[j] - d * r0[j];
  const double s1 = sqrt(r1[0].re * r1[0].re + r1[0].im * r1[0].im + r1[1].re * r1[1].re + r1[1].im * r1[1].im +
                         r1[2].re * r1[2].re + r1[2].im * r1[2].im);
#pragma unroll
  for (int j = 0; j < 3; ++j) r1[j] = mk(r1[j].re / s1, r1[j].im / s1);
  M u;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    u.e[0][j] = r0[j];
    u.e[1][j] = r1[j];
  }
  u.e[2][0] = conj(r0[1] * r1[2] - r0[2] * r1[1]);
  u.e[2][1] = conj(r0[2] * r1[0] - r0[0] * r1[2]);
  u.e[2][2] = conj(r0[0] * r1[1] - r0[1] * r1[0]);
  return u;
}

// random_su3 (src/su3/utils.cpp:13-30), redrawn: Haar SU(3) from 6 Box-Muller pairs (not
// inlined: it runs at initialisation and at R refreshes only).
__device__ __noinline__ M haar(Stream& g) {
  double n[12];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double u1 = g.uni(), u2 = g.uni();
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincos(2 * PI * u2, &sn, &cs);
    n[2 * k] = rad * cs;
    n[2 * k + 1] = rad * sn;
  }
  return haar_from_normals(n);
}

// The block of one chain: local coordinates lc (in [-1, l] for every link a chain at an
// active link reads; -1 and l are the neighbouring blocks' faces, the reference's halo) sit
// at stored site b_d l + lc_d - cum_d (mod L_d), with base_d = b_d l - cum_d in
// (-L_d, L_d - l].
struct Block {
  int L[4], base[4], l;
  __device__ __forceinline__ uint32_t site(const int lc[4]) const {
    uint32_t s = 0;
#pragma unroll
    for (int d = 3; d >= 0; --d) {
      int c = base[d] + lc[d];
      if (c < 0) c += L[d];
      else if (c >= L[d]) c -= L[d];
      // a chain only leaves [-1, l] after a lift onto a frozen link, which takes a rounding
      // accident in the lift's tower sampling; the full reduction keeps any position in bounds
      if ((unsigned)c >= (unsigned)L[d]) c = ((c % L[d]) + L[d]) % L[d];
      s = s * (uint32_t)L[d] + (uint32_t)c;
    }
    return s;
  }
  // GeometryCB::is_frozen in block-local terms: the halo (outside [0, l)) and the links
  // leaving local coordinate 0 in a direction d != mu.
  __device__ __forceinline__ bool frozen(const int lc[4], int mu) const {
    bool f = false;
#pragma unroll
    for (int d = 0; d < 4; ++d) f = f || lc[d] < 0 || lc[d] >= l || (d != mu && lc[d] == 0);
    return f;
  }
};

__device__ __forceinline__ void shifted(const int a[4], int d1, int s1, int d2, int s2, int out[4]) {
#pragma unroll
  for (int d = 0; d < 4; ++d) out[d] = a[d] + (d == d1 ? s1 : 0) + (d == d2 ? s2 : 0);
}

// solve_reject_fast (src/ecmc/ecmc_mpi_cb.h:59-94): along U(theta) = R diag(e^{i eps theta},
// e^{-i eps theta}, 1) R^dagger U one staple's action is A cos(theta) + eps B sin(theta) +
// const; the angle at which the integral of its derivative's positive part reaches gamma.
// The reference forms theta = phi + asin(alpha) with phi = atan2(-A, B); here the same angle
// is one atan2 of (sin, cos)(phi + asin(alpha)), from cos phi = B / R, sin phi = -A / R and
// cos asin(alpha) = sqrt(1 - alpha^2), and phi's quadrant test (phi < pi/2 or > 3pi/2) is
// B > 0; R = hypot(A, B) and 1 / R come from one rsqrt of A^2 + B^2 (A and B are of order
// beta, far from overflow), and gamma / (2 R) is a product.  Exact in real arithmetic; the
// forms differ in rounding, and in the branch taken only where B / |A| is below the rounding
// of phi.
__device__ double solve_reject(double A, double B, double gamma, int eps) {
  if (eps == -1) B = -B;
  const double R2 = fma(A, A, B * B), invR = rsqrt(R2), R = R2 * invR, period = 2.0 * R;
  const double disc = floor(gamma * (0.5 * invR));
  gamma -= disc * period;
  const double p1 = R - A;
  double alpha;
  if (B > 0.0)
    alpha = (gamma > p1) ? (gamma - p1) * invR - 1.0 : (gamma + A) * invR;
  else
    alpha = gamma * invR - 1.0;
  alpha = alpha > 1.0 ? 1.0 : (alpha < -1.0 ? -1.0 : alpha);
  const double ca = sqrt(fma(-alpha, alpha, 1.0)), sp = -A * invR, cp = B * invR;
  double theta = atan2(fma(sp, ca, cp * alpha), fma(cp, ca, -(sp * alpha)));
  if (theta < 0.0) theta += 2.0 * PI;
  return theta + 2.0 * PI * disc;
}

// compute_reject_angles_fast (ecmc_mpi_cb.cpp:197-246) for one staple S, T = R^dagger U:
// P = T S R; A = -(beta/3) Re(P00 + P11), B = -(beta/3) Im(P11 - P00).  Only P00 and P11
// are needed, so S is never formed: a forward staple is S = X W^+ (W = U_nu(x) U_mu(x+nu),
// X = U_nu(x+mu)) and P_ii = (T_i. X) . (W^+ R)_.i; a backward staple is S = W^+ D
// (W = U_mu(x-nu) U_nu(x+mu-nu), D = U_nu(x-nu)) and P_ii = (T_i. W^+) . (D R)_.i.
__device__ __forceinline__ double reject_from(Z P00, Z P11, double beta, double gamma, int eps) {
  const double br = -(beta / 3.0);
  return solve_reject((P00.re + P11.re) * br, (P11.im - P00.im) * br, gamma, eps);
}

// compute_ds (ecmc_mpi_cb.cpp:263-274), Im[(R^dagger P R)_00 - (R^dagger P R)_11], as
// Im tr(P Q) with the Hermitian Q = R diag(1, -1, 0) R^dagger formed once per lift.
struct Herm {
  double d[3];  // real diagonal
  Z o[3];       // Q01, Q02, Q12 (Q10 = conj Q01, ...)
};
// Q from columns 0 and 1 of R (or of the proposal S R).
__device__ __forceinline__ Herm ds_matrix_cols(const Z c0[3], const Z c1[3]) {
  Herm q;
#pragma unroll
  for (int m = 0; m < 3; ++m)
    q.d[m] = fma(c0[m].re, c0[m].re, c0[m].im * c0[m].im) - fma(c1[m].re, c1[m].re, c1[m].im * c1[m].im);
  q.o[0] = cfma(c0[0], conj(c0[1]), cmul(mk(-c1[0].re, -c1[0].im), conj(c1[1])));
  q.o[1] = cfma(c0[0], conj(c0[2]), cmul(mk(-c1[0].re, -c1[0].im), conj(c1[2])));
  q.o[2] = cfma(c0[1], conj(c0[2]), cmul(mk(-c1[1].re, -c1[1].im), conj(c1[2])));
  return q;
}
__device__ __forceinline__ Herm ds_matrix(const M& R) {
  const Z c0[3] = {R.e[0][0], R.e[1][0], R.e[2][0]}, c1[3] = {R.e[0][1], R.e[1][1], R.e[2][1]};
  return ds_matrix_cols(c0, c1);
}
__device__ __forceinline__ int dsign(double x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

// ---- row streaming: a product is formed one row at a time, so that only one full
// matrix and a row or two are held in registers (a full FP64 SU(3) matrix is 36 registers)
__device__ __forceinline__ void ld_row(const double2* L, uint32_t s, int mu, int row, Z out[3]) {
  const double2* q = L + ((size_t)s * 4 + (size_t)mu) * 9 + 3 * row;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double2 v = q[c];
    out[c] = mk(v.x, v.y);
  }
}
// out_c = sum_a v_a M_ac
__device__ __forceinline__ void vmul(const Z v[3], const M& m, Z out[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) out[c] = cdot3(v[0], m.e[0][c], v[1], m.e[1][c], v[2], m.e[2][c]);
}
// Q_km of the Hermitian Q
__device__ __forceinline__ Z qel(const Herm& q, int k, int m) {
  if (k == m) return mk(q.d[k], 0.0);
  const int i = (k + m == 1) ? 0 : (k + m == 2 ? 1 : 2);
  return k < m ? q.o[i] : conj(q.o[i]);
}
// row m's share of Im tr(X Q): sum_k Im(X_mk Q_km)
__device__ __forceinline__ double im_row_q(const Z r[3], const Herm& q, int m) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const Z a = qel(q, k, m);
    s = fma(r[k].re, a.im, fma(r[k].im, a.re, s));
  }
  return s;
}


// Link i of lift plaquette (fwd, nu) at local coordinates out, direction returned
// (GeometryCB.cpp:58-90): 0 = (x, mu); forward 1 = (x+mu, nu), 2 = (x+nu, mu), 3 = (x, nu);
// backward 1 = (x+mu-nu, nu), 2 = (x-nu, mu), 3 = (x-nu, nu).
__device__ __forceinline__ int lift_link(int i, bool fwd, const int lc[4], int mu, int nu, int out[4]) {
  switch (i) {
    case 0: shifted(lc, -1, 0, -1, 0, out); return mu;
    case 1: shifted(lc, mu, 1, fwd ? -1 : nu, fwd ? 0 : -1, out); return nu;
    case 2: shifted(lc, nu, fwd ? 1 : -1, -1, 0, out); return mu;
    default: shifted(lc, fwd ? -1 : nu, fwd ? 0 : -1, -1, 0, out); return nu;
  }
}


// The lift's plaquette (lift_improved_fast, ecmc_mpi_cb.cpp:277-337) as F0 F1 F2 F3 with
// F0 = U0, F2 = U2^+ and, forward, F1 = U1, F3 = U3^+ or, backward, F1 = U1^+, F3 = U3.  The
// P of each link of the reference is a cyclic rotation rot_s = F_s F_s+1 F_s+2 F_s+3 or the
// adjoint of one, so every dS is +-Im tr(Q rot_s) for s = 0, 3 and X (1 forward, 2 backward):
// forward P0 = rot0, P1 = rot1, P2 = rot3^+, P3 = rot0^+; backward P0 = rot0, P1 = rot2^+,
// P2 = rot3^+, P3 = rot3.  One call forms one rot_s as (F_s F_s+1)(F_s+2 F_s+3), by rows,
// and returns (Im tr(Q rot_s), Im tr(Qn rot_s)) for the current Q and the proposal's Qn.
// With several lanes per chain, lanes 0, 1, 2 form rot0, rotX, rot3 at once; with one, the
// lane makes the three calls in turn: the same operations either way.  Not inlined: the
// products would otherwise share the event loop's register budget.
struct Factor {
  uint32_t site;
  int dir;
  bool dag;
};
__device__ __forceinline__ Factor lift_factor(int f, uint32_t x, uint32_t s1, uint32_t s2, uint32_t s3, int mu, int nu,
                                              bool fwd) {
  f &= 3;
  Factor r;
  r.site = f == 0 ? x : (f == 1 ? s1 : (f == 2 ? s2 : s3));
  r.dir = (f & 1) ? nu : mu;
  r.dag = f == 0 ? false : (f == 1 ? !fwd : (f == 2 ? true : fwd));
  return r;
}
// row m of F (U, or U^+ whose row m is the conjugated column m of U)
__device__ __forceinline__ void ld_row_f(const double2* L, const Factor& f, int m, Z out[3]) {
  const double2* q = L + ((size_t)f.site * 4 + (size_t)f.dir) * 9;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double2 v = q[f.dag ? 3 * c + m : 3 * m + c];
    out[c] = mk(v.x, f.dag ? -v.y : v.y);
  }
}
__device__ __noinline__ double2 lift_trace_lane(const double2* L, Factor fa, Factor fb, Factor fc, Factor fd, Herm q,
                                                Herm qn) {
  M D, P, B;
#pragma unroll
  for (int m = 0; m < 3; ++m) ld_row_f(L, fd, m, D.e[m]);
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    Z r[3];
    ld_row_f(L, fc, m, r);
    vmul(r, D, P.e[m]);
  }
#pragma unroll
  for (int m = 0; m < 3; ++m) ld_row_f(L, fb, m, B.e[m]);
  double t = 0.0, n = 0.0;
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    Z r[3], u[3], w[3];
    ld_row_f(L, fa, m, r);
    vmul(r, B, u);
    vmul(u, P, w);
    t += im_row_q(w, q, m);
    n += im_row_q(w, qn, m);
  }
  return make_double2(t, n);
}

// su2_quaternion_to_su3 (src/su3/utils.cpp:33-45) of (x0, x1, x2, x3) in subgroup (i, j).
__device__ M embed(const double x[4], int i, int j) {
  M X;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) X.e[a][b] = mk(0.0, 0.0);
  const int k = 3 - i - j;
  X.e[k][k] = mk(1.0, 0.0);
  X.e[i][i] = mk(x[0], x[3]);
  X.e[j][j] = mk(x[0], -x[3]);
  X.e[i][j] = mk(x[2], x[1]);
  X.e[j][i] = mk(-x[2], x[1]);
  return X;
}

// q (9 double2) = element iset of a chain's set (ecmc_set / random_SU3_epsilon,
// src/su3/utils.cpp:66-127: set[0] = 1, set[2p+1] = the product of (sqrt(1 - eps^2), eps r/|r|)
// embedded in (0,1), (0,2), (1,2) with r uniform in (-1/2, 1/2)^3, set[2p+2] = its adjoint),
// generation gen of chain c in call `call`; r from three Philox calls (3p + j, c, call,
// ECMC_SETC ^ gen).  Each embedding multiplies from the right and changes two columns only;
// skipping the exact zeros and ones of the embedded matrix leaves every rounding as in the
// full 3x3 product.
// Four words of the set's counter stream (one out-of-line copy of the Philox rounds).
__device__ __noinline__ void set_words(u32x4* w, uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t k0,
                                       uint32_t k1) {
  u32x4 cc;
  cc.v[0] = a;
  cc.v[1] = b;
  cc.v[2] = c;
  cc.v[3] = d;
  *w = philox4x32_10(cc, k0, k1);
}

__device__ __noinline__ void set_elem(double2* q, double eps, uint32_t k0, uint32_t k1, uint32_t c, uint32_t call,
                                      uint32_t gen, int iset) {
  M Mx;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) Mx.e[a][b] = mk(a == b ? 1.0 : 0.0, 0.0);
  if (iset != 0) {
    const uint32_t p = (uint32_t)(iset - 1) >> 1;
    double r[12];
    u32x4 w[3];
#pragma unroll 1
    for (uint32_t j = 0; j < 3; ++j) set_words(&w[j], 3 * p + j, c, call, ECMC_SETC ^ (gen & 0xFFFFu), k0, k1);
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int t = 0; t < 4; ++t) r[4 * j + t] = ((double)w[j].v[t] + 0.5) * 2.3283064365386963e-10 - 0.5;
    const int sub[3][2] = {{0, 1}, {0, 2}, {1, 2}};
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const double norm = sqrt(r[3 * s] * r[3 * s] + r[3 * s + 1] * r[3 * s + 1] + r[3 * s + 2] * r[3 * s + 2]);
      const double x0 = sqrt(1 - eps * eps), x1 = eps * r[3 * s] / norm, x2 = eps * r[3 * s + 1] / norm,
                   x3 = eps * r[3 * s + 2] / norm;
      const int i = sub[s][0], j = sub[s][1];
      const Z Eii = mk(x0, x3), Ejj = mk(x0, -x3), Eij = mk(x2, x1), Eji = mk(-x2, x1);
#pragma unroll
      for (int row = 0; row < 3; ++row) {
        const Z a = Mx.e[row][i], b = Mx.e[row][j];
        Mx.e[row][i] = cfma(b, Eji, cmul(a, Eii));
        Mx.e[row][j] = cfma(b, Ejj, cmul(a, Eij));
      }
    }
  }
  const bool adj = iset != 0 && (iset & 1) == 0;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const Z v = adj ? mk(Mx.e[k % 3][k / 3].re, -Mx.e[k % 3][k / 3].im) : Mx.e[k / 3][k % 3];
    q[k] = make_double2(v.re, v.im);
  }
}

// sample_persistant (ecmc_mpi_cb.cpp:496-637) for chain c: events until it has travelled
// theta_sample; the chain record persists across calls.  GROUP lanes of one warp (1, 3 or
// 6) run a chain together: each computes its share of the six staples and, with three or
// more, lanes 0-2 one product each of a lift; all of them carry the chain's state and take
// the same branches, so the group never diverges.  Every lane stores the updated link (the
// same values), so each lane's later loads see its own stores and no barrier is needed.
template <int GROUP, int MINB>
__global__ void __launch_bounds__(ECMC_WARPS * 32, MINB) k_ecmc_sample(EcmcLaunch a) {
  static_assert(GROUP == 1 || GROUP == 3 || GROUP == 6, "a chain's lanes split its six staples evenly");
  constexpr int PER_WARP = 32 / GROUP;  // chains per warp; 32 % GROUP lanes stay idle
  const int lane = threadIdx.x & 31, slot = lane / GROUP, sub = lane - slot * GROUP, lane0 = slot * GROUP;
  const uint32_t c = (blockIdx.x * ECMC_WARPS + (threadIdx.x >> 5)) * PER_WARP + slot;
  if (slot >= PER_WARP || c >= a.n_chains) return;
  const unsigned gmask = GROUP == 1 ? (1u << lane) : (((1u << GROUP) - 1u) << lane0);
  qcb_ecmc_chain& rec = a.chains[c];
  Block blk;
  blk.l = a.l;
  {
    uint32_t q = c;
#pragma unroll
    for (int d = 3; d >= 0; --d) {
      const int b = (int)(q % (uint32_t)a.nb[d]);
      q /= (uint32_t)a.nb[d];
      blk.L[d] = a.L[d];
      blk.base[d] = b * a.l - a.cum[d];
    }
  }
  Stream g;
  g.chain = c;
  g.k0 = a.k0;
  g.k1 = a.k1;
  g.n = rec.draws;
  const int l = a.l;
  double2* links = a.links;
  int set_counter = rec.initialized ? rec.set_counter : 0;
  uint32_t set_gen = 0;  // renewed at the start of every call
  int lc[4], mu, eps;
  double th_site, th_R, tr_site, tr_R;
  uint64_t events, lifts, revs = rec.revs;
  int status = 0;  // the record keeps the bits of the latest call
  M R;
  if (!rec.initialized) {
    // random_site (ecmc_mpi_cb.cpp:359-367): local coordinates 1 .. l-2 (padded 2 .. L-1)
#pragma unroll
    for (int d = 0; d < 4; ++d) lc[d] = 1 + (int)(g.uni() * (double)(l - 2));
    mu = (int)(g.uni() * 4.0);
    eps = g.uni() < 0.5 ? -1 : 1;
    R = haar(g);
    th_site = a.poisson ? -log(g.uni()) * a.theta_refresh_site : a.theta_refresh_site;
    th_R = a.poisson ? -log(g.uni()) * a.theta_refresh_R : a.theta_refresh_R;
    tr_site = tr_R = 0.0;
    events = lifts = 0;
  } else {
#pragma unroll
    for (int d = 0; d < 4; ++d) lc[d] = rec.site[d];
    mu = rec.mu;
    eps = rec.epsilon;
#pragma unroll
    for (int k = 0; k < 9; ++k) R.e[k / 3][k % 3] = mk(rec.R[2 * k], rec.R[2 * k + 1]);
    th_site = rec.theta_refresh_site;
    th_R = rec.theta_refresh_R;
    tr_site = rec.travelled_site;
    tr_R = rec.travelled_R;
    events = rec.events;
    lifts = rec.lifts;
  }
  const double theta_sample = a.poisson ? -log(g.uni()) * a.theta_sample : a.theta_sample;
  double tr_sample = 0.0;

#pragma unroll 1
  for (uint64_t ev = 0;; ++ev) {
    if (ev >= ECMC_MAX_EVENTS) {
      status |= 2;
      break;
    }
    if (set_counter % 10000 == 0) {  // the chain's set is renewed
      ++set_gen;
      set_counter = 0;
    }
    const uint32_t x = blk.site(lc);
    // rows 0 and 1 of T = R^dagger U: all the reject angles need
    M T;
#pragma unroll
    for (int j2 = 0; j2 < 3; ++j2) T.e[0][j2] = T.e[1][j2] = mk(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Z ur[3];
      ld_row(links, x, mu, c, ur);
#pragma unroll
      for (int j2 = 0; j2 < 3; ++j2) {
        T.e[0][j2] = cfma(conj(R.e[c][0]), ur[j2], T.e[0][j2]);
        T.e[1][j2] = cfma(conj(R.e[c][1]), ur[j2], T.e[1][j2]);
      }
    }
    // compute_list_staples (ecmc_mpi_cb.cpp:12-36): for each nu != mu, forward then backward;
    // lane `sub` of the chain's group computes staples sub, sub + GROUP, ...; the angles are
    // then taken in staple order, keeping the first minimum.  Staple k draws the event's
    // uniform number k.
    double best = 0.0;
    int j = 0;
#pragma unroll 1
    for (int t = 0; t < 6 / GROUP; ++t) {
      const int k = sub + t * GROUP;
      const int nu = (k >> 1) + ((k >> 1) >= mu ? 1 : 0);
      const bool fwd = (k & 1) == 0;
      // Forward S = X W^+ (X = U_nu(x+mu), W = U_nu(x) U_mu(x+nu)); backward S = W^+ D
      // (W = U_mu(x-nu) U_nu(x+mu-nu), D = U_nu(x-nu)).  With E = X or D, Tt = T E forward or
      // T backward, and (E'R) = R forward or D R backward, both are
      // P_ii = sum_r (Tt W^+)_ir (E'R)_ri, and (Tt W^+)_ir = sum_m conj(W1_rm) (Tt W2^+)_im
      // for W = W1 W2: one code path for both orientations, streaming every link by rows.
      int q4[4];
      shifted(lc, fwd ? mu : nu, fwd ? 1 : -1, -1, 0, q4);
      const uint32_t se = blk.site(q4);
      shifted(lc, nu, fwd ? 1 : -1, fwd ? -1 : mu, fwd ? 0 : 1, q4);
      const uint32_t s2 = blk.site(q4);
      const int d2 = fwd ? mu : nu;
      shifted(lc, nu, fwd ? 0 : -1, -1, 0, q4);
      const uint32_t s1 = blk.site(q4);
      const int d1 = fwd ? nu : mu;
      // With one lane per chain every lane of a warp is at the same staple, so the orientation
      // is a branch; with more, the two orientations run as one instruction stream.
      const bool fwd_math = GROUP == 1 ? fwd : true;
      Z g0[3], g1[3];  // rows 0 and 1 of Tt
      if (fwd_math) {
#pragma unroll
        for (int c2 = 0; c2 < 3; ++c2) g0[c2] = g1[c2] = mk(0.0, 0.0);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          Z er[3];
          ld_row(links, se, nu, r, er);
#pragma unroll
          for (int c2 = 0; c2 < 3; ++c2) {
            const Z e = fwd ? er[c2] : mk(r == c2 ? 1.0 : 0.0, 0.0);
            g0[c2] = cfma(T.e[0][r], e, g0[c2]);
            g1[c2] = cfma(T.e[1][r], e, g1[c2]);
          }
        }
      } else {
#pragma unroll
        for (int c2 = 0; c2 < 3; ++c2) g0[c2] = T.e[0][c2], g1[c2] = T.e[1][c2];
      }
      Z h0[3], h1[3];  // rows 0 and 1 of Tt W2^+
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        Z w2[3];
        ld_row(links, s2, d2, m, w2);
        h0[m] = cdot3(g0[0], conj(w2[0]), g0[1], conj(w2[1]), g0[2], conj(w2[2]));
        h1[m] = cdot3(g1[0], conj(w2[0]), g1[1], conj(w2[1]), g1[2], conj(w2[2]));
      }
      Z P00 = mk(0.0, 0.0), P11 = mk(0.0, 0.0);
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        Z w1[3];
        ld_row(links, s1, d1, r, w1);
        const Z y0 = cdot3(conj(w1[0]), h0[0], conj(w1[1]), h0[1], conj(w1[2]), h0[2]);
        const Z y1 = cdot3(conj(w1[0]), h1[0], conj(w1[1]), h1[1], conj(w1[2]), h1[2]);
        Z z0 = R.e[r][0], z1 = R.e[r][1];
        if (GROUP > 1 || !fwd) {
          Z er[3];
          ld_row(links, se, nu, r, er);
          const Z e0 = cdot3(er[0], R.e[0][0], er[1], R.e[1][0], er[2], R.e[2][0]);
          const Z e1 = cdot3(er[0], R.e[0][1], er[1], R.e[1][1], er[2], R.e[2][1]);
          z0 = fwd ? z0 : e0;
          z1 = fwd ? z1 : e1;
        }
        P00 = cfma(y0, z0, P00);
        P11 = cfma(y1, z1, P11);
      }
      const double rej = reject_from(P00, P11, a.beta, -log(chain_uniform(g.chain, g.k0, g.k1, g.n + k)), eps);
#pragma unroll
      for (int q = 0; q < GROUP; ++q) {
        const double rq = GROUP == 1 ? rej : __shfl_sync(gmask, rej, lane0 + q);
        const int kq = t * GROUP + q;
        if (kq == 0 || rq < best) best = rq, j = kq;
      }
    }
    g.n += 6;
    const double d_sample = theta_sample - tr_sample;
    const double d_site = th_site - tr_site;
    const double d_R = th_R - tr_R;
    // std::min({...}) returns the first smallest; a non-finite step stops the chain
    double step = best;
    if (d_sample < step) step = d_sample;
    if (d_site < step) step = d_site;
    if (d_R < step) step = d_R;
    if (!isfinite(step)) {
      status |= 1;
      break;
    }
    const int kind = (step == d_sample) ? 0 : (step == d_site) ? 1 : (step == d_R) ? 2 : 3;
    // update (ecmc_mpi_cb.cpp:340-356): U <- R diag(e^{i xi}, e^{-i xi}, 1) R^dagger U, the
    // rows of T = R^dagger U: 0 and 1 from above, 2 from U; written row by row
    {
      double sn, cs;
      sincos((double)eps * step, &sn, &cs);
      Z t2[3] = {mk(0.0, 0.0), mk(0.0, 0.0), mk(0.0, 0.0)};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Z ur[3];
        ld_row(links, x, mu, c, ur);
#pragma unroll
        for (int j2 = 0; j2 < 3; ++j2) t2[j2] = cfma(conj(R.e[c][2]), ur[j2], t2[j2]);
      }
      const Z ep = mk(cs, sn), em = mk(cs, -sn);
      double2* q = links + ((size_t)x * 4 + (size_t)mu) * 9;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const Z r0 = cmul(R.e[i][0], ep), r1 = cmul(R.e[i][1], em), r2 = R.e[i][2];
#pragma unroll
        for (int j2 = 0; j2 < 3; ++j2) {
          const Z v = cdot3(r0, T.e[0][j2], r1, T.e[1][j2], r2, t2[j2]);
          q[3 * i + j2] = make_double2(v.re, v.im);
        }
      }
      ++events;
    }
    if (kind == 0) {
      tr_site += d_sample;
      tr_R += d_sample;
      break;
    } else if (kind == 1) {
      tr_sample += d_site;
      tr_R += d_site;
      tr_site = 0.0;
      if (a.poisson) th_site = -log(g.uni()) * a.theta_refresh_site;
#pragma unroll
      for (int d = 0; d < 4; ++d) lc[d] = 1 + (int)(g.uni() * (double)(l - 2));
      mu = (int)(g.uni() * 4.0);
      eps = g.uni() < 0.5 ? -1 : 1;
    } else if (kind == 2) {
      tr_sample += d_R;
      tr_site += d_R;
      tr_R = 0.0;
      if (a.poisson) th_R = -log(g.uni()) * a.theta_refresh_R;
      R = haar(g);
    } else {
      tr_sample += best;
      tr_site += best;
      tr_R += best;
      // lift_improved_fast (ecmc_mpi_cb.cpp:277-337) on plaquette j
      const int nu = (j >> 1) + ((j >> 1) >= mu ? 1 : 0);
      const bool fwd = (j & 1) == 0;
      int t4[4];
      lift_link(1, fwd, lc, mu, nu, t4);
      const uint32_t s1 = blk.site(t4);
      const bool f1 = blk.frozen(t4, nu);
      lift_link(2, fwd, lc, mu, nu, t4);
      const uint32_t s2 = blk.site(t4);
      const bool f2 = blk.frozen(t4, mu);
      lift_link(3, fwd, lc, mu, nu, t4);
      const uint32_t s3 = blk.site(t4);
      const bool f3 = blk.frozen(t4, nu);
      // selectVariable's uniform and the set index, in the reference's order, before the
      // plaquette: the proposal R_new = S R is known in advance and its dS rides along
      const double r = g.uni();
      const int iset = (int)(g.uni() * (double)ECMC_SET_SIZE);
      // the picked element, formed once into the chain's slot (every lane of the chain writes
      // the same values and reads back its own writes)
      double2* sq = a.sx + (size_t)c * 9;
      set_elem(sq, a.epsilon_set, a.k0, a.k1, c, a.call, set_gen, iset);
      Herm Qn;
      {
        Z c0[3], c1[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          const double2 s0 = sq[3 * m], s1v = sq[3 * m + 1], s2v = sq[3 * m + 2];
          const Z a0 = mk(s0.x, s0.y), a1 = mk(s1v.x, s1v.y), a2 = mk(s2v.x, s2v.y);
          c0[m] = cdot3(a0, R.e[0][0], a1, R.e[1][0], a2, R.e[2][0]);
          c1[m] = cdot3(a0, R.e[0][1], a1, R.e[1][1], a2, R.e[2][1]);
        }
        Qn = ds_matrix_cols(c0, c1);
      }
      // traces of rot0, rotX, rot3 against Q (tq) and Qn (tn)
      double tq[3], tn[3];
      const Herm Q = ds_matrix(R);
      if (GROUP >= 3) {
        const int i3 = sub % 3, r0 = i3 == 0 ? 0 : (i3 == 1 ? (fwd ? 1 : 2) : 3);
        const double2 v = lift_trace_lane(links, lift_factor(r0, x, s1, s2, s3, mu, nu, fwd),
                                          lift_factor(r0 + 1, x, s1, s2, s3, mu, nu, fwd),
                                          lift_factor(r0 + 2, x, s1, s2, s3, mu, nu, fwd),
                                          lift_factor(r0 + 3, x, s1, s2, s3, mu, nu, fwd), Q, Qn);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          tq[q] = __shfl_sync(gmask, v.x, lane0 + q);
          tn[q] = __shfl_sync(gmask, v.y, lane0 + q);
        }
      } else {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int r0 = q == 0 ? 0 : (q == 1 ? (fwd ? 1 : 2) : 3);
          const double2 v = lift_trace_lane(links, lift_factor(r0, x, s1, s2, s3, mu, nu, fwd),
                                            lift_factor(r0 + 1, x, s1, s2, s3, mu, nu, fwd),
                                            lift_factor(r0 + 2, x, s1, s2, s3, mu, nu, fwd),
                                            lift_factor(r0 + 3, x, s1, s2, s3, mu, nu, fwd), Q, Qn);
          tq[q] = v.x;
          tn[q] = v.y;
        }
      }
      // dS of each candidate (0 for frozen links) under R and under R_new
      const double ds0 = tq[0], dn0 = tn[0];
      const double ds1 = f1 ? 0.0 : (fwd ? tq[1] : -tq[1]), dn1 = fwd ? tn[1] : -tn[1];
      const double ds2 = f2 ? 0.0 : -tq[2], dn2 = -tn[2];
      const double ds3 = f3 ? 0.0 : (fwd ? -tq[0] : tq[2]), dn3 = fwd ? -tn[0] : tn[2];
      const double a0 = fabs(ds0), a1 = fabs(ds1), a2 = fabs(ds2), a3 = fabs(ds3);
      const double sum = a0 + a1 + a2 + a3;
      const double p0 = a0 / sum, p1 = a1 / sum, p2 = a2 / sum;
      // selectVariable (ecmc_mpi_cb.cpp:252-260)
      const int idx = r < p0 ? 0 : (r < p0 + p1 ? 1 : (r < p0 + p1 + p2 ? 2 : 3));
      const double ds_old = idx == 0 ? ds0 : idx == 1 ? ds1 : idx == 2 ? ds2 : ds3;
      const double ds_new = idx == 0 ? dn0 : idx == 1 ? dn1 : idx == 2 ? dn2 : dn3;
      int new_eps = -dsign(ds_old);
      bool take = fabs(ds_old) < fabs(ds_new);
      if (!take) take = g.uni() < fabs(ds_new) / fabs(ds_old);
      if (take) {
        M Sx;
#pragma unroll
        for (int cc = 0; cc < 9; ++cc) {
          const double2 v = sq[cc];
          Sx.e[cc / 3][cc % 3] = mk(v.x, v.y);
        }
        M Rn;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j2 = 0; j2 < 3; ++j2)
            Rn.e[i][j2] = cdot3(Sx.e[i][0], R.e[0][j2], Sx.e[i][1], R.e[1][j2], Sx.e[i][2], R.e[2][j2]);
        R = Rn;
        new_eps = -dsign(ds_new);
      }
      const int nmu = lift_link(idx, fwd, lc, mu, nu, t4);
      const bool same = t4[0] == lc[0] && t4[1] == lc[1] && t4[2] == lc[2] && t4[3] == lc[3];
      revs += same ? 1 : 0;
      ++lifts;
      ++set_counter;
#pragma unroll
      for (int d = 0; d < 4; ++d) lc[d] = t4[d];
      mu = nmu;
      eps = new_eps;
    }
  }
  if (sub != 0) return;
#pragma unroll
  for (int d = 0; d < 4; ++d) rec.site[d] = lc[d];
  rec.mu = mu;
  rec.epsilon = eps;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    rec.R[2 * k] = R.e[k / 3][k % 3].re;
    rec.R[2 * k + 1] = R.e[k / 3][k % 3].im;
  }
  rec.theta_refresh_site = th_site;
  rec.theta_refresh_R = th_R;
  rec.travelled_site = tr_site;
  rec.travelled_R = tr_R;
  rec.draws = g.n;
  rec.events = events;
  rec.lifts = lifts;
  rec.revs = revs;
  rec.initialized = 1;
  rec.set_counter = set_counter;
  rec.status = status;
  if (status) atomicOr(a.status, (uint32_t)status);
}

__global__ void k_ecmc_counters(qcb_ecmc_chain* chains, uint32_t n, unsigned long long* out, int reset) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long e = 0, l = 0, r = 0;
  if (c < n) {
    e = chains[c].events;
    l = chains[c].lifts;
    r = chains[c].revs;
    if (reset) chains[c].events = chains[c].lifts = chains[c].revs = 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    l += __shfl_down_sync(0xffffffffu, l, o);
    r += __shfl_down_sync(0xffffffffu, r, o);
  }
  if ((threadIdx.x & 31) == 0 && (e | l | r)) {
    atomicAdd(&out[0], e);
    atomicAdd(&out[1], l);
    atomicAdd(&out[2], r);
  }
}

}  // namespace


namespace {

template <int GROUP, int MINB>
cudaError_t launch_sample(const EcmcLaunch& a, cudaStream_t s) {
  const uint32_t per_block = ECMC_WARPS * (32 / GROUP);
  k_ecmc_sample<GROUP, MINB><<<(a.n_chains + per_block - 1) / per_block, ECMC_WARPS * 32, 0, s>>>(a);
  return cudaGetLastError();
}

// Chains resident on the device at once for the kernel of GROUP lanes per chain.
template <int GROUP, int MINB>
uint32_t resident_chains() {
  int dev = 0, sms = 0, blocks = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_ecmc_sample<GROUP, MINB>, ECMC_WARPS * 32, 0) !=
          cudaSuccess)
    return 0;
  return (uint32_t)sms * (uint32_t)blocks * ECMC_WARPS * (32 / GROUP);
}

}  // namespace

// A call lasts about as long as its number of waves of resident chains, each chain taking a
// similar number of events, so shape k is expected to run at rate_k n / (cap_k ceil(n / cap_k)),
// rate_k being its event rate with the device full.  The rates are the ones measured on B200
// (1e8 events/s, reference default budgets, 8192 to 65536 chains); the capacities come from
// the occupancy calculator.  Among equal estimates the earlier shape wins.  The capacities are
// computed once per device, for the device current at the call (callers make the lattice's
// device current first).
int ecmc_layout(uint32_t n_chains, int lanes) {
  struct Shape {
    int layout, lanes;
    uint32_t cap;
    double rate;
  };
  constexpr int MAX_DEVICES = 64;
  static std::mutex mu;
  static bool filled[MAX_DEVICES] = {};
  static Shape table[MAX_DEVICES][4];
  if (lanes == 1) return ECMC_LAYOUT_1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) dev = 0;
  Shape shapes[4];
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!filled[dev]) {
      const Shape t[4] = {
          {ECMC_LAYOUT_6, 6, resident_chains<6, 1>(), 2.9},
          {ECMC_LAYOUT_6C, 6, resident_chains<6, ECMC_CAPPED>(), 3.3},
          {ECMC_LAYOUT_3, 3, resident_chains<3, 1>(), 3.1},
          {ECMC_LAYOUT_3C, 3, resident_chains<3, ECMC_CAPPED>(), 3.6},
      };
      for (int k = 0; k < 4; ++k) table[dev][k] = t[k];
      filled[dev] = true;
    }
    for (int k = 0; k < 4; ++k) shapes[k] = table[dev][k];
  }
  int best = lanes == 3 ? ECMC_LAYOUT_3C : ECMC_LAYOUT_6;
  double best_rate = -1.0;
  for (const Shape& sh : shapes) {
    if ((lanes != 0 && sh.lanes != lanes) || sh.cap == 0) continue;
    const double waves = (double)((n_chains + sh.cap - 1) / sh.cap);
    const double r = sh.rate * (double)n_chains / ((double)sh.cap * (waves < 1.0 ? 1.0 : waves));
    if (r > best_rate) best_rate = r, best = sh.layout;
  }
  return best;
}

cudaError_t launch_ecmc_sample(const EcmcLaunch& a, int layout, cudaStream_t s) {
  switch (layout) {
    case ECMC_LAYOUT_1: return launch_sample<1, 1>(a, s);
    case ECMC_LAYOUT_3: return launch_sample<3, 1>(a, s);
    case ECMC_LAYOUT_3C: return launch_sample<3, ECMC_CAPPED>(a, s);
    case ECMC_LAYOUT_6: return launch_sample<6, 1>(a, s);
    case ECMC_LAYOUT_6C: return launch_sample<6, ECMC_CAPPED>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_ecmc_counters(qcb_ecmc_chain* chains, uint32_t n, unsigned long long* out, int reset,
                                 cudaStream_t s) {
  k_ecmc_counters<<<(n + 127) / 128, 128, 0, s>>>(chains, n, out, reset);
  return cudaGetLastError();
}

}  // namespace qcb
