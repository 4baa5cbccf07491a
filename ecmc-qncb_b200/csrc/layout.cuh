// layout.cuh — lattice geometry and the parity-split structure-of-arrays link layout.
//
// The reference stores links array-of-structures with a one-site halo,
// links[((site*4 + mu)*9 + i*3 + j)] over an (L+2)^4 padded block
// (src/gauge/GaugeField.h:27-56, src/geometry/GeometryCB.h:24-26), with a 64-bit neighbour
// table (src/geometry/GeometryCB.cpp:10-31).  Here the lattice is periodic with no halo, and
// neighbours come from integer arithmetic on the coordinates.
//
// Site order: full lexicographic index s = x + Lx*(y + Ly*(z + Lz*t)) (x fastest, as in
// the reference and in ILDG).  Parity p = (x+y+z+t) & 1.  Because Lx is even, the
// checkerboard index i = s >> 1 is unique within a parity.
//
// Storage: for each (mu, parity) block, each link is NR reals (18: full 3x3 complex; 12:
// rows 0 and 1, row 2 = conj(row0 x row1)) split into NC "chunks" of a vector type
// (double2 / float4 / float2), each chunk stored as its own array over i.  Chunk c of link
// (mu, p, i) lives at index ((mu*2 + p)*NC + c)*stride + i, so a warp of consecutive i
// issues fully coalesced 8- or 16-byte loads.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "su3.cuh"

namespace qcb {

struct Geom {
  int L[4];      // extents x, y, z, t
  int Lxh;       // Lx / 2
  int str[4];    // full-index strides 1, Lx, Lx*Ly, Lx*Ly*Lz
  uint32_t V;    // volume
  uint32_t Vh;   // V / 2
  uint32_t stride;  // allocation stride of one chunk array (>= Vh, multiple of 64)
  uint32_t rcp[3];  // floor(2^32 / d) for d = Lxh, Ly, Lz (0xFFFFFFFF for d = 1)
  // Slab of a larger lattice (domain decomposition along t): the sites with local time
  // tlo .. thi are the slab's own, the slices outside are halo copies of the neighbours'.
  // Random-number link ids and the normalisation of the observables use the global volume
  // Vg and the global site index s + soff (mod 2^32).  A whole lattice has tlo = 0,
  // thi = Lt - 1, Vg = V, soff = 0.
  int tlo, thi;
  uint32_t Vg;
  uint32_t soff;
};

__device__ __forceinline__ bool own_site(const Geom& g, int t) { return t >= g.tlo && t <= g.thi; }

// Global site index of local full index s, periodic in the global time (halo slices of the
// first and last slab wrap around; volumes are below 2^30, so the signed view is exact).
__device__ __forceinline__ uint32_t global_site(const Geom& g, uint32_t s) {
  int32_t gs = (int32_t)(s + g.soff);
  if (gs < 0) gs += (int32_t)g.Vg;
  else if ((uint32_t)gs >= g.Vg) gs -= (int32_t)g.Vg;
  return (uint32_t)gs;
}

// n / d and n % d by multiply-high with r = rcp of d: the estimate umulhi(n, r) is q or
// q - 1 for every 32-bit n, so one correction step makes it exact.
__device__ __forceinline__ uint32_t divmod_rcp(uint32_t n, uint32_t d, uint32_t r, uint32_t* rem) {
  uint32_t q = __umulhi(n, r);
  uint32_t m = n - q * d;
  if (m >= d) {
    ++q;
    m -= d;
  }
  *rem = m;
  return q;
}

struct Coord {
  int c[4];
  uint32_t s;  // full index
};

// Coordinates of checkerboard site (parity p, index i).
__device__ __forceinline__ Coord cb_coord(const Geom& g, int p, uint32_t i) {
  Coord r;
  uint32_t m;
  const uint32_t q = divmod_rcp(i, (uint32_t)g.Lxh, g.rcp[0], &m);
  const int xh = (int)m;
  const uint32_t q2 = divmod_rcp(q, (uint32_t)g.L[1], g.rcp[1], &m);
  r.c[1] = (int)m;
  const uint32_t q3 = divmod_rcp(q2, (uint32_t)g.L[2], g.rcp[2], &m);
  r.c[2] = (int)m;
  r.c[3] = (int)q3;
  r.c[0] = 2 * xh + ((p + r.c[1] + r.c[2] + r.c[3]) & 1);
  r.s = (uint32_t)r.c[0] + (uint32_t)g.L[0] * q;
  return r;
}

// Full index of the neighbour of site s (coordinates c) displaced by d (+1/-1) in
// direction mu, with periodic wrap.
__device__ __forceinline__ uint32_t nb_full(const Geom& g, const Coord& x, int mu, int d) {
  int cm = x.c[mu] + d;
  int32_t off = d * g.str[mu];
  if (cm >= g.L[mu]) off -= g.L[mu] * g.str[mu];
  if (cm < 0) off += g.L[mu] * g.str[mu];
  return (uint32_t)((int32_t)x.s + off);
}

// Full index of x + d1*mu1 + d2*mu2 (mu1 != mu2).
__device__ __forceinline__ uint32_t nb2_full(const Geom& g, const Coord& x, int mu1, int d1, int mu2,
                                             int d2) {
  int32_t off = 0;
  int c1 = x.c[mu1] + d1;
  off += d1 * g.str[mu1];
  if (c1 >= g.L[mu1]) off -= g.L[mu1] * g.str[mu1];
  if (c1 < 0) off += g.L[mu1] * g.str[mu1];
  int c2 = x.c[mu2] + d2;
  off += d2 * g.str[mu2];
  if (c2 >= g.L[mu2]) off -= g.L[mu2] * g.str[mu2];
  if (c2 < 0) off += g.L[mu2] * g.str[mu2];
  return (uint32_t)((int32_t)x.s + off);
}

// Parity of a full index is known from the displacement parity; the checkerboard index
// is s >> 1.
__device__ __forceinline__ uint32_t cb_index(uint32_t s) { return s >> 1; }

// ---- storage traits ------------------------------------------------------------------
template <typename S, int NR>
struct Store;

template <>
struct Store<double, 18> {
  typedef double2 V;
  static constexpr int NC = 9;
};
template <>
struct Store<double, 12> {
  typedef double2 V;
  static constexpr int NC = 6;
};
template <>
struct Store<float, 18> {
  typedef float2 V;
  static constexpr int NC = 9;
};
template <>
struct Store<float, 12> {
  typedef float4 V;
  static constexpr int NC = 3;
};

// Load path of a link read.  LD_RO: read-only data path (__ldg), for kernels that never
// read links written earlier in the same launch.  LD_CG: L2-coherent loads (__ldcg), for
// persistent kernels whose blocks read links other blocks wrote in the same launch.
// (Ordinary L1-cached loads in the persistent kernels, after thread 0's acquire and a block
// barrier, returned stale links: the batch-versus-single bit-identity test failed with them.)
enum : int { LD_RO = 0, LD_CG = 1 };

template <int LM, typename V>
__device__ __forceinline__ V ldv(const V* p) {
  if (LM == LD_RO) return __ldg(p);
  return __ldcg(p);
}

template <typename S, int NR, int LM = LD_RO>
struct Links {
  typedef typename Store<S, NR>::V V;
  static constexpr int NC = Store<S, NR>::NC;
  static constexpr int NREAL = NR;
  V* p;
  uint32_t stride;

  __device__ __forceinline__ size_t idx(int mu, int par, int c, uint32_t i) const {
    return ((size_t)((mu * 2 + par) * NC + c)) * stride + i;
  }

  // Load link (mu, par, i) as an m3<R> (row 2 rebuilt for 12-real storage).
  template <typename R>
  __device__ __forceinline__ m3<R> load(int mu, int par, uint32_t i) const {
    m3<R> u;
    if constexpr (sizeof(V) == 4 * sizeof(S)) {
      // FP32 12-real: three float4 chunks (e00,e01), (e02,e10), (e11,e12).
      const V a = ldv<LM>(&p[idx(mu, par, 0, i)]);
      const V b = ldv<LM>(&p[idx(mu, par, 1, i)]);
      const V c = ldv<LM>(&p[idx(mu, par, 2, i)]);
      u.e[0][0] = mk<R>(R(a.x), R(a.y));
      u.e[0][1] = mk<R>(R(a.z), R(a.w));
      u.e[0][2] = mk<R>(R(b.x), R(b.y));
      u.e[1][0] = mk<R>(R(b.z), R(b.w));
      u.e[1][1] = mk<R>(R(c.x), R(c.y));
      u.e[1][2] = mk<R>(R(c.z), R(c.w));
    } else {
      // 2-component chunks: chunk c = element c of the row-major 3x3.
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const V v = ldv<LM>(&p[idx(mu, par, c, i)]);
        u.e[c / 3][c % 3] = mk<R>(R(v.x), R(v.y));
      }
    }
    if (NR == 12) reconstruct_row2(u);
    return u;
  }

  // Rows 0 and 1 of link (mu, par, i) only; row 2 is left unset.  For 12-real storage this
  // is the stored data with no reconstruction, for products whose row 2 is rebuilt after.
  template <typename R>
  __device__ __forceinline__ m3<R> load_rows01(int mu, int par, uint32_t i) const {
    m3<R> u;
    if constexpr (sizeof(V) == 4 * sizeof(S)) {
      const V a = ldv<LM>(&p[idx(mu, par, 0, i)]);
      const V b = ldv<LM>(&p[idx(mu, par, 1, i)]);
      const V c = ldv<LM>(&p[idx(mu, par, 2, i)]);
      u.e[0][0] = mk<R>(R(a.x), R(a.y));
      u.e[0][1] = mk<R>(R(a.z), R(a.w));
      u.e[0][2] = mk<R>(R(b.x), R(b.y));
      u.e[1][0] = mk<R>(R(b.z), R(b.w));
      u.e[1][1] = mk<R>(R(c.x), R(c.y));
      u.e[1][2] = mk<R>(R(c.z), R(c.w));
    } else {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const V v = ldv<LM>(&p[idx(mu, par, c, i)]);
        u.e[c / 3][c % 3] = mk<R>(R(v.x), R(v.y));
      }
    }
    return u;
  }

  template <typename R>
  __device__ __forceinline__ void store(int mu, int par, uint32_t i, const m3<R>& u) const {
    if constexpr (sizeof(V) == 4 * sizeof(S)) {
      V a, b, c;
      a.x = S(u.e[0][0].re), a.y = S(u.e[0][0].im), a.z = S(u.e[0][1].re), a.w = S(u.e[0][1].im);
      b.x = S(u.e[0][2].re), b.y = S(u.e[0][2].im), b.z = S(u.e[1][0].re), b.w = S(u.e[1][0].im);
      c.x = S(u.e[1][1].re), c.y = S(u.e[1][1].im), c.z = S(u.e[1][2].re), c.w = S(u.e[1][2].im);
      p[idx(mu, par, 0, i)] = a;
      p[idx(mu, par, 1, i)] = b;
      p[idx(mu, par, 2, i)] = c;
    } else {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        V v;
        v.x = S(u.e[c / 3][c % 3].re);
        v.y = S(u.e[c / 3][c % 3].im);
        p[idx(mu, par, c, i)] = v;
      }
    }
  }
};

// ---- su(3) algebra field (flow accumulator): 8 reals per link --------------------------
template <typename S>
struct AlgStore;
template <>
struct AlgStore<double> {
  typedef double2 V;
  static constexpr int NC = 4;
};
template <>
struct AlgStore<float> {
  typedef float4 V;
  static constexpr int NC = 2;
};

template <typename S, int LM = LD_RO>
struct AlgField {
  typedef typename AlgStore<S>::V V;
  static constexpr int NC = AlgStore<S>::NC;
  V* p;
  uint32_t stride;
  __device__ __forceinline__ size_t idx(int mu, int par, int c, uint32_t i) const {
    return ((size_t)((mu * 2 + par) * NC + c)) * stride + i;
  }
  template <typename R>
  __device__ __forceinline__ alg8<R> load(int mu, int par, uint32_t i) const {
    alg8<R> z;
    const S* q;
    V v[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) v[c] = (LM == LD_CG) ? __ldcg(&p[idx(mu, par, c, i)]) : p[idx(mu, par, c, i)];
    q = reinterpret_cast<const S*>(v);
#pragma unroll
    for (int k = 0; k < 8; ++k) z.a[k] = R(q[k]);
    return z;
  }
  template <typename R>
  __device__ __forceinline__ void store(int mu, int par, uint32_t i, const alg8<R>& z) const {
    V v[NC];
    S* q = reinterpret_cast<S*>(v);
#pragma unroll
    for (int k = 0; k < 8; ++k) q[k] = S(z.a[k]);
#pragma unroll
    for (int c = 0; c < NC; ++c) p[idx(mu, par, c, i)] = v[c];
  }
};

}  // namespace qcb
