// flow_site.cuh — one fused Wilson-flow RK3 stage for the four links of one site (shared by the
// single-lattice site kernel and the persistent batched kernel).
//
// Reference: GradientFlow (src/flow/gradient_flow.cpp:15-114); the stage arithmetic of each
// link is that of flow_link.cuh, with the work grouped by site.
//
// The four links U_mu(x), mu = 0..3, are updated in turn, so the links around x are read
// while they are in L1/L2, and the product that the forward staples of U_mu(x) and U_nu(x)
// share is formed once: with
//   T_{mu nu} = U_nu(x+mu) U_mu(x+nu)^dagger,
// the forward staple of U_mu(x) in plane nu is T_{mu nu} U_nu(x)^dagger and that of U_nu(x)
// in plane mu is T_{mu nu}^dagger U_mu(x)^dagger.  T_{mu nu} (mu < nu) is formed while U_mu(x)
// is updated and kept in shared memory (private to the thread) until U_nu(x) uses it: the six
// products of a site need four slots at most (slot 0: T01, then T12; slot 1: T02, then T23;
// slot 2: T03; slot 3: T13), because the planes are visited with nu ascending.  The direction
// and plane loops are not unrolled: one code body serves every (mu, nu).
#pragma once
#include "flow_link.cuh"

namespace qcb {

constexpr int FS_THREADS = 128;  // slot stride: blocks of at most this many threads

// Slot of T_{a b}, a < b, as 4-bit fields indexed by 4a + b.
__device__ __forceinline__ int t_slot(int a, int b) {
  constexpr unsigned long long tbl = (0ull << 4) | (1ull << 8) | (2ull << 12) | (0ull << 24) | (3ull << 28) | (1ull << 44);
  return (int)((tbl >> (4 * (4 * a + b))) & 0xF);
}

template <typename R, int TS>
struct TSlots {
  R* base;  // [4][TS][FS_THREADS]
  __device__ __forceinline__ R* at(int slot, int k) const { return base + (slot * TS + k) * FS_THREADS + threadIdx.x; }
  __device__ __forceinline__ void put(int slot, const m3<R>& t) const {
#pragma unroll
    for (int r = 0; r < TS / 6; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        *at(slot, 6 * r + 2 * c) = t.e[r][c].re;
        *at(slot, 6 * r + 2 * c + 1) = t.e[r][c].im;
      }
  }
  __device__ __forceinline__ m3<R> get(int slot) const {
    m3<R> t;
#pragma unroll
    for (int r = 0; r < TS / 6; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) t.e[r][c] = mk<R>(*at(slot, 6 * r + 2 * c), *at(slot, 6 * r + 2 * c + 1));
    if (TS == 12) reconstruct_row2(t);
    return t;
  }
};

// Row 2 of the site's own links U_nu(x), nu = 0..3 (12-real): rebuilt once, in the first
// direction's pass over the site (mu = 0 uses all four as full matrices), and read back for the
// later directions.  [4][6][FS_THREADS] after the T slots.
template <typename R>
struct Row2Cache {
  R* base;
  __device__ __forceinline__ R* at(int nu, int k) const { return base + (nu * 6 + k) * FS_THREADS + threadIdx.x; }
  // U_nu(x) as a full matrix from its stored rows: row 2 rebuilt and kept when `first`, read
  // back otherwise.
  template <typename F>
  __device__ __forceinline__ m3<R> load(const F& f, int nu, int par, uint32_t i, bool first) const {
    m3<R> u = f.template load_rows01<R>(nu, par, i);
    if (first) {
      reconstruct_row2(u);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        *at(nu, 2 * c) = u.e[2][c].re;
        *at(nu, 2 * c + 1) = u.e[2][c].im;
      }
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) u.e[2][c] = mk<R>(*at(nu, 2 * c), *at(nu, 2 * c + 1));
    }
    return u;
  }
};

// Shared-memory bytes of the T slots of a block (and, for 12-real, the row-2 cache).
template <typename R, int NR>
constexpr size_t flow_site_smem() {
  return (size_t)4 * (NR == 12 ? 12 : 18) * FS_THREADS * sizeof(R) + (NR == 12 ? (size_t)4 * 6 * FS_THREADS * sizeof(R) : 0);
}

// Stage `stage` (1, 2, 3) of the four links of site x = (par, i): src -> dst.
template <typename F, typename ACC, typename R, int NR>
__device__ __forceinline__ void flow_site(const Geom& g, const F& src, const F& dst, const ACC& acc, R eps, int stage,
                                          int par, uint32_t i, R* slot_mem) {
  constexpr int TS = NR == 12 ? 12 : 18;
  const TSlots<R, TS> slots{slot_mem};
  const Row2Cache<R> own{slot_mem + 4 * TS * FS_THREADS};
  const int opp = par ^ 1;
  const Coord x = cb_coord(g, par, i);
  if (!own_site(g, x.c[3])) return;  // halo slice of a slab
  const NbOff o = nb_offsets(g, x);
#pragma unroll 1
  for (int mu = 0; mu < 4; ++mu) {
    const int32_t upmu = sel4(o.up, mu);
    const uint32_t ixmu = cb_index((uint32_t)((int32_t)x.s + upmu));
    m3<R> A;
    set_zero(A);
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
      const int nu = k + (k >= mu);
      const int32_t upnu = sel4(o.up, nu), dnnu = sel4(o.dn, nu);
      const uint32_t ixnu = cb_index((uint32_t)((int32_t)x.s + upnu));
      const uint32_t ixmnu = cb_index((uint32_t)((int32_t)x.s + dnnu));
      const uint32_t ixmunu = cb_index((uint32_t)((int32_t)x.s + upmu + dnnu));
      // forward: T_{mu nu} U_nu(x)^dagger, T shared with the plane's other link
      // 12-real: the forward term W is in SU(3); only its rows 0 and 1 are multiplied out
      // (T U_nu(x)^dag from T's rows 0, 1; for nu < mu, W = U_nu(x) T from U_nu(x)'s stored
      // rows, A += W^dag) and its row 2 is rebuilt
      if constexpr (NR == 12) {
        if (nu > mu) {
          const m3<R> U0 = src.template load_rows01<R>(nu, opp, ixmu);
          const m3<R> U1 = src.template load<R>(mu, opp, ixnu);
          const m3<R> T = mul_na_rows01(U0, U1);
          slots.put(t_slot(mu, nu), T);
          const m3<R> U2 = own.load(src, nu, par, i, mu == 0);
          m3<R> W = mul_na_rows01(T, U2);
          reconstruct_row2(W);
          add_m3(A, W);
        } else {
          const m3<R> T = slots.get(t_slot(nu, mu));
          const m3<R> U2 = src.template load_rows01<R>(nu, par, i);
          m3<R> W = mul_nn_rows01(U2, T);
          reconstruct_row2(W);
          add_m3_adj(A, W);
        }
      } else {
        const m3<R> U2 = src.template load<R>(nu, par, i);
        if (nu > mu) {
          m3<R> T = mul_na(src.template load<R>(nu, opp, ixmu), src.template load<R>(mu, opp, ixnu));
          slots.put(t_slot(mu, nu), T);
          acc_na(A, T, U2);
        } else {
          const m3<R> T = slots.get(t_slot(nu, mu));  // T_{nu mu} = T_{mu nu}^dagger
          acc_aa(A, T, U2);
        }
      }
      // backward: (U_mu(x-nu) U_nu(x+mu-nu))^dagger U_nu(x-nu)
      if constexpr (NR == 12) {
        const m3<R> V1 = src.template load_rows01<R>(mu, opp, ixmnu);
        const m3<R> V0 = src.template load<R>(nu, par, ixmunu);
        m3<R> P = mul_nn_rows01(V1, V0);
        reconstruct_row2(P);
        const m3<R> V2 = src.template load<R>(nu, opp, ixmnu);
        acc_an(A, P, V2);
      } else {
        const m3<R> V0 = src.template load<R>(nu, par, ixmunu);
        const m3<R> V1 = src.template load<R>(mu, opp, ixmnu);
        const m3<R> P = mul_aa(V0, V1);
        const m3<R> V2 = src.template load<R>(nu, opp, ixmnu);
        acc_nn(A, P, V2);
      }
    }
    m3<R> U;
    if constexpr (NR == 12)
      U = own.load(src, mu, par, i, mu == 0);
    else
      U = src.template load<R>(mu, par, i);
    alg8<R> Z = proj_ta(mul_nn(U, A));
#pragma unroll
    for (int q = 0; q < 8; ++q) Z.a[q] = -Z.a[q];
    alg8<R> X;
    if (stage == 1) {
      const R c = R(0.25) * eps;
#pragma unroll
      for (int q = 0; q < 8; ++q) X.a[q] = c * Z.a[q];
      acc.template store<R>(mu, par, i, Z);
    } else {
      const alg8<R> Z0 = acc.template load<R>(mu, par, i);
      if (stage == 2) {
        const R c1 = R(8.0 / 9.0) * eps, c0 = R(17.0 / 36.0) * eps;
        alg8<R> N;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          X.a[q] = fma(c1, Z.a[q], -(c0 * Z0.a[q]));
          N.a[q] = fma(R(8.0 / 9.0), Z.a[q], -(R(17.0 / 36.0) * Z0.a[q]));
        }
        acc.template store<R>(mu, par, i, N);
      } else {
        const R c1 = R(0.75) * eps;
#pragma unroll
        for (int q = 0; q < 8; ++q) X.a[q] = fma(c1, Z.a[q], -(eps * Z0.a[q]));
      }
    }
    const m3<R> E = exp_su3(X);
    m3<R> Un = flow_product<F, R>(E, U);
    flow_reunit<R>(Un, stage);
    dst.template store<R>(mu, par, i, Un);
  }
}

}  // namespace qcb
