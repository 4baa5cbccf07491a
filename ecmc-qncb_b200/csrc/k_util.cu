// k_util.cu — start configurations, layout conversion, reunitarisation, gauge transform.
#include "dispatch.cuh"
#include "philox.cuh"

namespace qcb {

Geom make_geom(const int dims[4]) {
  Geom g;
  for (int d = 0; d < 4; ++d) g.L[d] = dims[d];
  g.Lxh = dims[0] / 2;
  g.str[0] = 1;
  g.str[1] = dims[0];
  g.str[2] = dims[0] * dims[1];
  g.str[3] = dims[0] * dims[1] * dims[2];
  g.V = (uint32_t)dims[0] * (uint32_t)dims[1] * (uint32_t)dims[2] * (uint32_t)dims[3];
  g.Vh = g.V / 2;
  g.stride = (g.Vh + 63u) & ~63u;
  const uint32_t dv[3] = {(uint32_t)g.Lxh, (uint32_t)dims[1], (uint32_t)dims[2]};
  for (int k = 0; k < 3; ++k) g.rcp[k] = dv[k] == 1 ? 0xFFFFFFFFu : (uint32_t)((1ull << 32) / dv[k]);
  g.tlo = 0;
  g.thi = dims[3] - 1;
  g.Vg = g.V;
  g.soff = 0;
  return g;
}

Geom make_slab_geom(const int global_dims[4], int t0, int tl) {
  const int local[4] = {global_dims[0], global_dims[1], global_dims[2], tl + 2};
  Geom g = make_geom(local);
  g.tlo = 1;
  g.thi = tl;
  g.Vg = (uint32_t)global_dims[0] * (uint32_t)global_dims[1] * (uint32_t)global_dims[2] * (uint32_t)global_dims[3];
  // local time 1 is global time t0: global index = local index + (t0 - 1) str[3] (mod 2^32)
  g.soff = (uint32_t)((int64_t)(t0 - 1) * (int64_t)g.str[3]);
  return g;
}

size_t link_bytes(const Geom& g, int prec, int nr) {
  const size_t per = (prec == QCB_PREC_FP64 ? 8 : 4) * (size_t)nr;
  return per * 8 * (size_t)g.stride;
}
size_t alg_bytes(const Geom& g, int prec) { return (prec == QCB_PREC_FP64 ? 8 : 4) * 8 * 8 * (size_t)g.stride; }

template <typename S, int NR>
static Links<S, NR> links_of(const LatDev& L) {
  Links<S, NR> f;
  f.p = reinterpret_cast<typename Links<S, NR>::V*>(L.links);
  f.stride = L.g.stride;
  return f;
}

// ---- cold start ----------------------------------------------------------------------
template <typename S, int NR>
__global__ void k_cold(Geom g, Links<S, NR> f) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  m3<double> one;
  set_identity(one);
#pragma unroll
  for (int b = 0; b < 8; ++b) f.template store<double>(b >> 1, b & 1, i, one);
}
template <typename S, int NR>
static cudaError_t cold_impl(const LatDev& L, cudaStream_t s, int block) {
  k_cold<S, NR><<<grid_for(L.g.Vh, block), block, 0, s>>>(L.g, links_of<S, NR>(L));
  return cudaGetLastError();
}
cudaError_t launch_cold(const LatDev& L, cudaStream_t s, int block) {
  if (block <= 0) block = 256;
  QCB_DISPATCH_STORE(L, cold_impl, L, s, block);
}

// ---- Haar-random SU(3) from the Philox stream ------------------------------------------
// Rows 0 and 1 are complex Gaussian vectors (Box-Muller), orthonormalised by Gram-Schmidt;
// row 2 = conj(row0 x row1).  Gram-Schmidt of Gaussian rows is the phase-fixed QR of
// Mezzadri (2007), so the matrix is exactly Haar-distributed on SU(3).  The reference
// (random_su3, src/su3/utils.cpp:13-30) uses a Householder QR without phase fixing.
// Always computed in FP64; `tag` selects the counter domain, `id` the matrix.
__device__ __forceinline__ m3<double> haar_su3(uint32_t id, uint32_t tag, uint32_t k0, uint32_t k1) {
  double n[12];
#pragma unroll
  for (int call = 0; call < 3; ++call) {
    u32x4 c;
    c.v[0] = id;
    c.v[1] = 0u;
    c.v[2] = tag;
    c.v[3] = (uint32_t)call;
    u32x4 r = philox4x32_10(c, k0, k1);
#pragma unroll
    for (int pr = 0; pr < 2; ++pr) {
      double u1 = u01<double>(r.v[2 * pr]);
      double u2 = u01<double>(r.v[2 * pr + 1]);
      double rad = sqrt(-2.0 * log(u1));
      double sn, cs;
      sincospi(2.0 * u2, &sn, &cs);
      n[call * 4 + pr * 2 + 0] = rad * cs;
      n[call * 4 + pr * 2 + 1] = rad * sn;
    }
  }
  m3<double> u;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    u.e[0][j] = mk<double>(n[2 * j], n[2 * j + 1]);
    u.e[1][j] = mk<double>(n[6 + 2 * j], n[6 + 2 * j + 1]);
  }
  reunitarize_rows(u);
  return u;
}

template <typename S, int NR>
__global__ void k_hot(Geom g, Links<S, NR> f, uint32_t k0, uint32_t k1) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
#pragma unroll 1
  for (int b = 0; b < 8; ++b) {
    const int mu = b >> 1, par = b & 1;
    const Coord x = cb_coord(g, par, i);
    const uint32_t link = (uint32_t)mu * g.Vg + global_site(g, x.s);
    f.template store<double>(mu, par, i, haar_su3(link, RNG_DOMAIN_HOT, k0, k1));
  }
}
template <typename S, int NR>
static cudaError_t hot_impl(const LatDev& L, uint64_t seed, cudaStream_t s, int block) {
  k_hot<S, NR><<<grid_for(L.g.Vh, block), block, 0, s>>>(L.g, links_of<S, NR>(L), (uint32_t)seed,
                                                          (uint32_t)(seed >> 32));
  return cudaGetLastError();
}
cudaError_t launch_hot(const LatDev& L, uint64_t seed, cudaStream_t s, int block) {
  if (block <= 0) block = 128;
  QCB_DISPATCH_STORE(L, hot_impl, L, seed, s, block);
}

// ---- random gauge transformation --------------------------------------------------------
// U_mu(x) -> G(x) U_mu(x) G(x+mu)^dagger (GaugeField::gauge_transform,
// src/gauge/GaugeField.cpp:100-114); G(x) is recomputed from the stream wherever needed,
// so no G field is stored.  Arithmetic in FP64.
template <typename S, int NR>
__global__ void k_gauge(Geom g, Links<S, NR> f, uint32_t k0, uint32_t k1) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  const int mu = blockIdx.y >> 1, par = blockIdx.y & 1;
  const Coord x = cb_coord(g, par, i);
  uint32_t xf;
  switch (mu) {
    case 0: xf = nb_full(g, x, 0, +1); break;
    case 1: xf = nb_full(g, x, 1, +1); break;
    case 2: xf = nb_full(g, x, 2, +1); break;
    default: xf = nb_full(g, x, 3, +1); break;
  }
  const m3<double> Gx = haar_su3(x.s, RNG_DOMAIN_GAUGE, k0, k1);
  const m3<double> Gy = haar_su3(xf, RNG_DOMAIN_GAUGE, k0, k1);
  const m3<double> U = f.template load<double>(mu, par, i);
  f.template store<double>(mu, par, i, mul_na(mul_nn(Gx, U), Gy));
}
template <typename S, int NR>
static cudaError_t gauge_impl(const LatDev& L, uint64_t seed, cudaStream_t s, int block) {
  k_gauge<S, NR><<<dim3(grid_for(L.g.Vh, block), 8), block, 0, s>>>(L.g, links_of<S, NR>(L), (uint32_t)seed,
                                                                     (uint32_t)(seed >> 32));
  return cudaGetLastError();
}
cudaError_t launch_gauge_transform(const LatDev& L, uint64_t seed, cudaStream_t s, int block) {
  if (block <= 0) block = 128;
  QCB_DISPATCH_STORE(L, gauge_impl, L, seed, s, block);
}

// ---- reunitarisation --------------------------------------------------------------------
template <typename S, int NR>
__global__ void k_reunit(Geom g, Links<S, NR> f) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  const int mu = blockIdx.y >> 1, par = blockIdx.y & 1;
  m3<double> U = f.template load<double>(mu, par, i);
  reunitarize_rows(U);
  f.template store<double>(mu, par, i, U);
}
template <typename S, int NR>
static cudaError_t reunit_impl(const LatDev& L, cudaStream_t s, int block) {
  k_reunit<S, NR><<<dim3(grid_for(L.g.Vh, block), 8), block, 0, s>>>(L.g, links_of<S, NR>(L));
  return cudaGetLastError();
}
cudaError_t launch_reunitarize(const LatDev& L, cudaStream_t s, int block) {
  if (block <= 0) block = 256;
  QCB_DISPATCH_STORE(L, reunit_impl, L, s, block);
}

// ---- AoS (ILDG order) <-> SoA ------------------------------------------------------------
__device__ __forceinline__ double bswap_d(double v) {
  unsigned long long b = __double_as_longlong(v);
  unsigned int lo = (unsigned int)b, hi = (unsigned int)(b >> 32);
  lo = __byte_perm(lo, 0, 0x0123);
  hi = __byte_perm(hi, 0, 0x0123);
  return __longlong_as_double(((unsigned long long)lo << 32) | hi);
}

// One thread per (site of the chunk, mu), blocks of AOS_BLOCK threads.  The AoS side of a
// block is one contiguous run of AOS_BLOCK links (144 bytes each), moved between global and
// shared memory in 16-byte chunks by consecutive threads (coalesced); each thread then
// converts its own link.  aos points at the chunk's first site, site0 (16-byte aligned).
constexpr int AOS_BLOCK = 128;

__device__ __forceinline__ int site_parity(const Geom& g, uint32_t s) {
  uint32_t r = s;
  const int x = (int)(r % (uint32_t)g.L[0]);
  r /= (uint32_t)g.L[0];
  const int y = (int)(r % (uint32_t)g.L[1]);
  r /= (uint32_t)g.L[1];
  const int z = (int)(r % (uint32_t)g.L[2]);
  const int tt = (int)(r / (uint32_t)g.L[2]);
  return (x + y + z + tt) & 1;
}

template <typename S, int NR>
__global__ void __launch_bounds__(AOS_BLOCK) k_aos_to_soa(Geom g, Links<S, NR> f, const double* __restrict__ aos,
                                                          uint32_t site0, uint32_t nsites, int bswap) {
  __shared__ double2 sm[AOS_BLOCK * 9];
  const uint64_t t0 = (uint64_t)blockIdx.x * AOS_BLOCK, nlinks = (uint64_t)nsites * 4;
  const uint32_t nl = (uint32_t)min((uint64_t)AOS_BLOCK, nlinks - t0);
  const double2* src = reinterpret_cast<const double2*>(aos) + t0 * 9;
  for (uint32_t c = threadIdx.x; c < nl * 9; c += AOS_BLOCK) sm[c] = src[c];
  __syncthreads();
  if (threadIdx.x >= nl) return;
  const uint64_t t = t0 + threadIdx.x;
  const uint32_t sl = (uint32_t)(t >> 2);
  const int mu = (int)(t & 3);
  const uint32_t s = site0 + sl;
  m3<double> u;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double2 v = sm[threadIdx.x * 9 + k];
    double re = v.x, im = v.y;
    if (bswap) {
      re = bswap_d(re);
      im = bswap_d(im);
    }
    u.e[k / 3][k % 3] = mk<double>(re, im);
  }
  f.template store<double>(mu, site_parity(g, s), s >> 1, u);
}

template <typename S, int NR>
__global__ void __launch_bounds__(AOS_BLOCK) k_soa_to_aos(Geom g, Links<S, NR> f, double* __restrict__ aos,
                                                          uint32_t site0, uint32_t nsites, int bswap) {
  __shared__ double2 sm[AOS_BLOCK * 9];
  const uint64_t t0 = (uint64_t)blockIdx.x * AOS_BLOCK, nlinks = (uint64_t)nsites * 4;
  const uint32_t nl = (uint32_t)min((uint64_t)AOS_BLOCK, nlinks - t0);
  if (threadIdx.x < nl) {
    const uint64_t t = t0 + threadIdx.x;
    const uint32_t sl = (uint32_t)(t >> 2);
    const int mu = (int)(t & 3);
    const uint32_t s = site0 + sl;
    const m3<double> u = f.template load<double>(mu, site_parity(g, s), s >> 1);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double re = u.e[k / 3][k % 3].re, im = u.e[k / 3][k % 3].im;
      if (bswap) {
        re = bswap_d(re);
        im = bswap_d(im);
      }
      sm[threadIdx.x * 9 + k] = make_double2(re, im);
    }
  }
  __syncthreads();
  double2* dst = reinterpret_cast<double2*>(aos) + t0 * 9;
  for (uint32_t c = threadIdx.x; c < nl * 9; c += AOS_BLOCK) dst[c] = sm[c];
}

template <typename S, int NR>
static cudaError_t a2s_impl(const LatDev& L, const double* aos, uint32_t site0, uint32_t nsites, int bswap,
                            cudaStream_t s, int) {
  k_aos_to_soa<S, NR><<<grid_for((uint64_t)nsites * 4, AOS_BLOCK), AOS_BLOCK, 0, s>>>(L.g, links_of<S, NR>(L), aos,
                                                                                     site0, nsites, bswap);
  return cudaGetLastError();
}
template <typename S, int NR>
static cudaError_t s2a_impl(const LatDev& L, double* aos, uint32_t site0, uint32_t nsites, int bswap,
                            cudaStream_t s, int) {
  k_soa_to_aos<S, NR><<<grid_for((uint64_t)nsites * 4, AOS_BLOCK), AOS_BLOCK, 0, s>>>(L.g, links_of<S, NR>(L), aos,
                                                                                     site0, nsites, bswap);
  return cudaGetLastError();
}
cudaError_t launch_aos_to_soa(const LatDev& L, const double* aos, uint32_t site0, uint32_t nsites, int bswap,
                              cudaStream_t s, int block) {
  if (block <= 0) block = 256;
  if ((uint64_t)site0 + nsites > L.g.V) return cudaErrorInvalidValue;
  QCB_DISPATCH_STORE(L, a2s_impl, L, aos, site0, nsites, bswap, s, block);
}
cudaError_t launch_soa_to_aos(const LatDev& L, double* aos, uint32_t site0, uint32_t nsites, int bswap,
                              cudaStream_t s, int block) {
  if (block <= 0) block = 256;
  if ((uint64_t)site0 + nsites > L.g.V) return cudaErrorInvalidValue;
  QCB_DISPATCH_STORE(L, s2a_impl, L, aos, site0, nsites, bswap, s, block);
}

// ---- precision / storage conversion ---------------------------------------------------
template <typename SD, int ND, typename SS, int NS>
__global__ void k_convert(Geom g, Links<SD, ND> d, Links<SS, NS> src) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  const int mu = blockIdx.y >> 1, par = blockIdx.y & 1;
  d.template store<double>(mu, par, i, src.template load<double>(mu, par, i));
}
template <typename SD, int ND>
static cudaError_t convert_dst(const LatDev& D, const LatDev& Sr, cudaStream_t s, int block) {
  dim3 grid(grid_for(D.g.Vh, block), 8);
  switch (Sr.prec * 100 + Sr.nr) {
    case QCB_PREC_FP64 * 100 + 18:
      k_convert<SD, ND, double, 18><<<grid, block, 0, s>>>(D.g, links_of<SD, ND>(D), links_of<double, 18>(Sr));
      break;
    case QCB_PREC_FP64 * 100 + 12:
      k_convert<SD, ND, double, 12><<<grid, block, 0, s>>>(D.g, links_of<SD, ND>(D), links_of<double, 12>(Sr));
      break;
    case QCB_PREC_FP32 * 100 + 18:
      k_convert<SD, ND, float, 18><<<grid, block, 0, s>>>(D.g, links_of<SD, ND>(D), links_of<float, 18>(Sr));
      break;
    case QCB_PREC_FP32 * 100 + 12:
      k_convert<SD, ND, float, 12><<<grid, block, 0, s>>>(D.g, links_of<SD, ND>(D), links_of<float, 12>(Sr));
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
cudaError_t launch_convert(const LatDev& dst, const LatDev& src, cudaStream_t s, int block) {
  if (block <= 0) block = 256;
  QCB_DISPATCH_STORE(dst, convert_dst, dst, src, s, block);
}

// ---- translation ---------------------------------------------------------------------
// dst(x) = src(x - sh) for every link: the reference's random shift of the whole field
// (src/mpi/Shift.cpp:109-186) on one device.  sh[d] in [0, L_d).  Links are copied in the
// storage type, bit for bit.
template <typename S, int NR>
__global__ void k_translate(Geom g, Links<S, NR> d, Links<S, NR> src, int4 sh) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  const int mu = blockIdx.y >> 1, par = blockIdx.y & 1;
  const Coord x = cb_coord(g, par, i);
  const int shv[4] = {sh.x, sh.y, sh.z, sh.w};
  uint32_t s = 0;
  int ps = 0;
#pragma unroll
  for (int k = 3; k >= 0; --k) {
    int y = x.c[k] - shv[k];
    if (y < 0) y += g.L[k];
    s = s * (uint32_t)g.L[k] + (uint32_t)y;
    ps += y;
  }
  d.template store<S>(mu, par, i, src.template load<S>(mu, ps & 1, s >> 1));
}
template <typename S, int NR>
static cudaError_t translate_impl(const LatDev& D, const LatDev& Sr, int4 sh, cudaStream_t s, int block) {
  dim3 grid(grid_for(D.g.Vh, block), 8);
  k_translate<S, NR><<<grid, block, 0, s>>>(D.g, links_of<S, NR>(D), links_of<S, NR>(Sr), sh);
  return cudaGetLastError();
}
cudaError_t launch_translate(const LatDev& dst, const LatDev& src, const int shift[4], cudaStream_t s, int block) {
  if (block <= 0) block = 256;
  if (dst.prec != src.prec || dst.nr != src.nr || dst.links == src.links) return cudaErrorInvalidValue;
  for (int d = 0; d < 4; ++d)
    if (dst.g.L[d] != src.g.L[d] || shift[d] < 0 || shift[d] >= dst.g.L[d]) return cudaErrorInvalidValue;
  const int4 sh = make_int4(shift[0], shift[1], shift[2], shift[3]);
  QCB_DISPATCH_STORE(dst, translate_impl, dst, src, sh, s, block);
}

}  // namespace qcb
