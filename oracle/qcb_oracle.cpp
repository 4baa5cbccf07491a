// qcb_oracle.cpp — FP64 CPU restatement of the ECMC-QNCB heatbath / plaquette / Wilson-flow
// path.  TEST INFRASTRUCTURE ONLY: it is the checker for the CUDA library, and the timed
// CPU baseline.  Nothing in the product links or calls it.
//
// PARITY UNPINNED: the reference cannot be compiled here (it needs MPI, Eigen3 and c-lime,
// none of which is installed) and it ships no tests, golden vectors or fixtures.  This
// restatement follows the reference source line by line (citations below, paths relative
// to the reference project) and is checked against known answers instead: the C++
// standard's mt19937_64 known value, the Philox4x32-10 known-answer vectors, scipy's expm,
// cold-start values and gauge/translation invariance.
//
// Field layout: array-of-structures over the periodic lattice without halo, in ILDG order:
//   links[((s*4 + mu)*9 + i*3 + j)], s = x + Lx*(y + Ly*(z + Lz*t))
// which is the reference's GaugeField layout (src/gauge/GaugeField.h:27,49-56) with the
// one-site halo removed.  On a single rank the halo holds copies of the periodic
// neighbours, and the frozen-link mask guarantees that every halo link read during a sweep
// is a copy of a frozen link (src/geometry/GeometryCB.cpp:33-56), so periodic indexing
// reproduces the single-rank reference exactly.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <random>
#include <vector>

namespace orc {

using C = std::complex<double>;

struct M3 {
  C a[9];
  C& operator()(int i, int j) { return a[i * 3 + j]; }
  const C& operator()(int i, int j) const { return a[i * 3 + j]; }
};

static M3 zero() {
  M3 m;
  for (auto& v : m.a) v = 0.0;
  return m;
}
static M3 ident() {
  M3 m = zero();
  m(0, 0) = m(1, 1) = m(2, 2) = 1.0;
  return m;
}
static M3 mul(const M3& x, const M3& y) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r(i, j) = x(i, 0) * y(0, j) + x(i, 1) * y(1, j) + x(i, 2) * y(2, j);
  return r;
}
static M3 adj(const M3& x) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r(i, j) = std::conj(x(j, i));
  return r;
}
static M3 add(const M3& x, const M3& y) {
  M3 r;
  for (int k = 0; k < 9; ++k) r.a[k] = x.a[k] + y.a[k];
  return r;
}
static M3 sub(const M3& x, const M3& y) {
  M3 r;
  for (int k = 0; k < 9; ++k) r.a[k] = x.a[k] - y.a[k];
  return r;
}
static M3 scale(C s, const M3& x) {
  M3 r;
  for (int k = 0; k < 9; ++k) r.a[k] = s * x.a[k];
  return r;
}
static C trace(const M3& x) { return x(0, 0) + x(1, 1) + x(2, 2); }
// Cofactor expansion along the first column.
static C det(const M3& m) {
  return m(0, 0) * (m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1)) - m(1, 0) * (m(0, 1) * m(2, 2) - m(0, 2) * m(2, 1)) +
         m(2, 0) * (m(0, 1) * m(1, 2) - m(0, 2) * m(1, 1));
}
static double sqnorm(const M3& m) {
  double s = 0;
  for (auto& v : m.a) s += std::norm(v);
  return s;
}

struct Lat {
  int L[4];
  size_t V;
  C* u;  // borrowed, 36*V complex
  // Optional neighbour table (borrowed): nbt[8 s + 2 mu + 0] = s + mu, [.. + 1] = s - mu.  The
  // reference keeps such a table (src/geometry/GeometryCB.cpp:10-31); it only replaces the
  // division-based lookup below, so results are the same bit for bit with or without it.
  const uint32_t* nbt = nullptr;
  size_t idx(int x, int y, int z, int t) const {
    return (size_t)x + (size_t)L[0] * ((size_t)y + (size_t)L[1] * ((size_t)z + (size_t)L[2] * (size_t)t));
  }
  void coords(size_t s, int c[4]) const {
    c[0] = (int)(s % L[0]);
    s /= L[0];
    c[1] = (int)(s % L[1]);
    s /= L[1];
    c[2] = (int)(s % L[2]);
    c[3] = (int)(s / L[2]);
  }
  // neighbour of s displaced by d (+1 / -1) in direction mu (periodic)
  size_t nb(size_t s, int mu, int d) const {
    if (nbt) return nbt[8 * s + 2 * mu + (d > 0 ? 0 : 1)];
    int c[4];
    coords(s, c);
    c[mu] = (c[mu] + d + L[mu]) % L[mu];
    return idx(c[0], c[1], c[2], c[3]);
  }
  M3 get(size_t s, int mu) const {
    M3 m;
    memcpy(m.a, u + (s * 4 + mu) * 9, sizeof m.a);
    return m;
  }
  void set(size_t s, int mu, const M3& m) { memcpy(u + (s * 4 + mu) * 9, m.a, sizeof m.a); }
};

static Lat make(double* aos, const int dims[4]) {
  Lat l;
  for (int d = 0; d < 4; ++d) l.L[d] = dims[d];
  l.V = (size_t)dims[0] * dims[1] * dims[2] * dims[3];
  l.u = reinterpret_cast<C*>(aos);
  return l;
}

// Fills the neighbour table of lattice f (8 entries per site) and attaches it to f.
static void attach_nb_table(Lat& f, std::vector<uint32_t>& tab) {
  tab.resize(8 * f.V);
  for (size_t s = 0; s < f.V; ++s)
    for (int mu = 0; mu < 4; ++mu) {
      tab[8 * s + 2 * mu] = (uint32_t)f.nb(s, mu, +1);
      tab[8 * s + 2 * mu + 1] = (uint32_t)f.nb(s, mu, -1);
    }
  f.nbt = tab.data();
}

// GaugeField::compute_staple (src/gauge/GaugeField.cpp:74-97)
static M3 staple(const Lat& f, size_t x, int mu) {
  M3 st = zero();
  size_t xmu = f.nb(x, mu, +1);
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    size_t xnu = f.nb(x, nu, +1);
    M3 U0 = f.get(xmu, nu), U1 = f.get(xnu, mu), U2 = f.get(x, nu);
    st = add(st, mul(U0, adj(mul(U2, U1))));
    size_t xmunu = f.nb(xmu, nu, -1);
    size_t xmnu = f.nb(x, nu, -1);
    M3 V0 = f.get(xmunu, nu), V1 = f.get(xmnu, mu), V2 = f.get(xmnu, nu);
    st = add(st, mul(adj(mul(V1, V0)), V2));
  }
  return st;
}

// mean_plaquette_local (src/observables/observables_mpi.cpp:8-29)
static double plaquette_sum(const Lat& f) {
  double sum = 0.0;
  for (size_t s = 0; s < f.V; ++s)
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        M3 U1 = f.get(s, mu);
        M3 U2 = f.get(f.nb(s, mu, +1), nu);
        M3 U3 = adj(f.get(f.nb(s, nu, +1), mu));
        M3 U4 = adj(f.get(s, nu));
        sum += trace(mul(mul(mul(U1, U2), U3), U4)).real() / 3.0;
      }
  return sum;
}

// clover_site (observables_mpi.cpp:61-85)
static M3 clover(const Lat& f, size_t x, int mu, int nu) {
  size_t xpmu = f.nb(x, mu, +1), xpnu = f.nb(x, nu, +1), xmmu = f.nb(x, mu, -1), xmnu = f.nb(x, nu, -1);
  size_t xmmupnu = f.nb(xmmu, nu, +1), xmmumnu = f.nb(xmmu, nu, -1), xpmumnu = f.nb(xpmu, nu, -1);
  M3 c = zero();
  c = add(c, mul(mul(mul(f.get(x, mu), f.get(xpmu, nu)), adj(f.get(xpnu, mu))), adj(f.get(x, nu))));
  c = add(c, mul(mul(mul(f.get(x, nu), adj(f.get(xmmupnu, mu))), adj(f.get(xmmu, nu))), f.get(xmmu, mu)));
  c = add(c, mul(mul(mul(adj(f.get(xmmu, mu)), adj(f.get(xmmumnu, nu))), f.get(xmmumnu, mu)), f.get(xmnu, nu)));
  c = add(c, mul(mul(mul(adj(f.get(xmnu, nu)), f.get(xmnu, mu)), f.get(xpmumnu, nu)), adj(f.get(x, mu))));
  M3 F = sub(c, adj(c));
  return scale(0.125, F);
}

// local_q_e_clover (observables_mpi.cpp:88-107) and topo_q_e_clover (:110-127)
static void topo_qe(const Lat& f, double* q_tot, double* e_tot) {
  double q = 0.0, e = 0.0;
  for (size_t s = 0; s < f.V; ++s) {
    M3 F01 = clover(f, s, 0, 1), F02 = clover(f, s, 0, 2), F03 = clover(f, s, 0, 3);
    M3 F12 = clover(f, s, 1, 2), F13 = clover(f, s, 1, 3), F23 = clover(f, s, 2, 3);
    double ql = trace(mul(F01, F23)).real() - trace(mul(F02, F13)).real() + trace(mul(F03, F12)).real();
    double el = 0.5 * (sqnorm(F01) + sqnorm(F02) + sqnorm(F03) + sqnorm(F12) + sqnorm(F13) + sqnorm(F23));
    q += ql * (1.0 / (4.0 * M_PI * M_PI));
    e += el;
  }
  *q_tot = q;
  *e_tot = e;
}

// proj_lie_su3 (src/su3/utils.cpp:130-134)
static void proj_lie(M3& A) {
  M3 B = scale(0.5, sub(A, adj(A)));
  C tr = trace(B) / 3.0;
  A = sub(B, scale(tr, ident()));
}

// exp_su3_luscher (src/su3/utils.cpp:145-193)
static M3 exp_luscher(const M3& Z, double coeff) {
  const C I(0.0, 1.0);
  M3 X = scale(coeff, Z);
  M3 X2 = mul(X, X);
  double t = -0.5 * trace(X2).real();
  double d = (I * det(X)).real();
  const int N = 18;
  double c[N + 1];
  c[0] = 1.0;
  for (int n = 1; n <= N; ++n) c[n] = c[n - 1] / (double)n;
  C q0 = c[N], q1 = 0.0, q2 = 0.0;
  for (int n = N - 1; n >= 0; --n) {
    C q0n = c[n] - I * d * q2;
    C q1n = q0 - t * q2;
    C q2n = q1;
    q0 = q0n;
    q1 = q1n;
    q2 = q2n;
  }
  return add(add(scale(q0, ident()), scale(q1, X)), scale(q2, X2));
}

// GradientFlow (src/flow/gradient_flow.cpp:10-128) on a lattice without halo.
struct Flow {
  Lat* f;
  double eps;
  std::vector<C> f0, f1;  // force_0, force_1
  void force(std::vector<C>& out) {  // compute_force (:15-34)
    for (size_t s = 0; s < f->V; ++s)
      for (int mu = 0; mu < 4; ++mu) {
        M3 st = staple(*f, s, mu);
        M3 tmp = mul(scale(-1.0, f->get(s, mu)), st);
        proj_lie(tmp);
        memcpy(&out[(s * 4 + mu) * 9], tmp.a, sizeof tmp.a);
      }
  }
  M3 at(const std::vector<C>& v, size_t s, int mu) const {
    M3 m;
    memcpy(m.a, &v[(s * 4 + mu) * 9], sizeof m.a);
    return m;
  }
  void rk3_step() {  // rk3_step (:117-128)
    f0.resize(f->V * 36);
    f1.resize(f->V * 36);
    force(f0);
    for (size_t s = 0; s < f->V; ++s)  // compute_w1 (:37-53)
      for (int mu = 0; mu < 4; ++mu) f->set(s, mu, mul(exp_luscher(at(f0, s, mu), 0.25 * eps), f->get(s, mu)));
    force(f1);
    for (size_t s = 0; s < f->V; ++s)  // compute_w2 (:56-74)
      for (int mu = 0; mu < 4; ++mu) {
        M3 Z = sub(scale((8.0 / 9.0) * eps, at(f1, s, mu)), scale((17.0 / 36.0) * eps, at(f0, s, mu)));
        f->set(s, mu, mul(exp_luscher(Z, 1.0), f->get(s, mu)));
      }
    for (size_t s = 0; s < f->V; ++s)  // replace_force_0 (:77-93)
      for (int mu = 0; mu < 4; ++mu) {
        M3 tmp = sub(scale(8.0 / 9.0, at(f1, s, mu)), scale(17.0 / 36.0, at(f0, s, mu)));
        memcpy(&f0[(s * 4 + mu) * 9], tmp.a, sizeof tmp.a);
      }
    force(f1);
    for (size_t s = 0; s < f->V; ++s)  // compute_w3 (:96-114)
      for (int mu = 0; mu < 4; ++mu) {
        M3 Z = sub(scale(0.75 * eps, at(f1, s, mu)), scale(eps, at(f0, s, mu)));
        f->set(s, mu, mul(exp_luscher(Z, 1.0), f->get(s, mu)));
      }
  }
};

// ---- SU(2) helpers (src/su3/utils.cpp:33-63) -----------------------------------------
struct Q4 {
  double v[4];
};
static M3 su2_quaternion_to_su3(const Q4& q, int i, int j) {
  M3 X = zero();
  int k = 3 - i - j;
  X(k, k) = 1.0;
  X(i, i) = C(q.v[0], q.v[3]);
  X(j, j) = C(q.v[0], -q.v[3]);
  X(i, j) = C(q.v[2], q.v[1]);
  X(j, i) = C(-q.v[2], q.v[1]);
  return X;
}
// quaternion of the 2x2 block [[w00, w01], [w10, w11]]
static Q4 su2_to_quaternion(C w00, C w01, C w10, C w11) {
  return {{(w00 + w11).real() / 2.0, (w01 + w10).imag() / 2.0, (w01 - w10).real() / 2.0, (w00 - w11).imag() / 2.0}};
}
static Q4 qmult(const Q4& q, const Q4& p) {
  return {{q.v[0] * p.v[0] - q.v[1] * p.v[1] - q.v[2] * p.v[2] - q.v[3] * p.v[3],
           q.v[0] * p.v[1] + q.v[1] * p.v[0] + q.v[2] * p.v[3] - q.v[3] * p.v[2],
           q.v[0] * p.v[2] - q.v[1] * p.v[3] + q.v[2] * p.v[0] + q.v[3] * p.v[1],
           q.v[0] * p.v[3] + q.v[1] * p.v[2] - q.v[2] * p.v[1] + q.v[3] * p.v[0]}};
}
static Q4 qadj(const Q4& q) { return {{q.v[0], -q.v[1], -q.v[2], -q.v[3]}}; }

// ---- reference heatbath with std::mt19937_64 (src/heatbath/heatbath.cpp:8-44) ----------
static Q4 generate_su2_kp(double beta, double k, std::mt19937_64& rng) {
  std::uniform_real_distribution<double> dist(0, 1);
  double alpha = beta * k * 2.0 / 3.0;
  double a0;
  while (true) {
    double delta = dist(rng);
    double r1 = dist(rng);
    double r2 = dist(rng);
    double r3 = dist(rng);
    double lambda_sq = -0.5 / alpha * (log(r1) + pow(cos(2 * M_PI * r2), 2) * log(r3));
    if (delta * delta <= 1.0 - lambda_sq) {
      a0 = 1.0 - 2.0 * lambda_sq;
      break;
    }
  }
  double r_spatial = sqrt(1.0 - a0 * a0);
  double phi = 2.0 * M_PI * dist(rng);
  double cos_theta = 2.0 * dist(rng) - 1.0;
  double sin_theta = sqrt(1.0 - cos_theta * cos_theta);
  return {{a0, r_spatial * sin_theta * cos(phi), r_spatial * sin_theta * sin(phi), r_spatial * cos_theta}};
}
static Q4 su2_step(double beta, const Q4& w, std::mt19937_64& rng) {
  double k = sqrt(w.v[0] * w.v[0] + w.v[1] * w.v[1] + w.v[2] * w.v[2] + w.v[3] * w.v[3]);
  Q4 v = {{w.v[0] / k, w.v[1] / k, w.v[2] / k, w.v[3] / k}};
  Q4 x = generate_su2_kp(beta, k, rng);
  return qmult(x, qadj(v));
}
// mpi::heatbathcb::hit (src/heatbath/heatbath_mpi.cpp:11-34)
static void hit_ref(Lat& f, size_t s, int mu, double beta, std::mt19937_64& rng) {
  M3 A = staple(f, s, mu);
  const int sub[3][2] = {{0, 1}, {1, 2}, {0, 2}};
  for (int g = 0; g < 3; ++g) {
    int i = sub[g][0], j = sub[g][1];
    M3 W = mul(f.get(s, mu), A);
    Q4 wq = su2_to_quaternion(W(i, i), W(i, j), W(j, i), W(j, j));
    Q4 r = su2_step(beta, wq, rng);
    f.set(s, mu, mul(su2_quaternion_to_su3(r, i, j), f.get(s, mu)));
  }
}

// Frozen links on one rank (src/geometry/GeometryCB.cpp:33-56): link (c, mu) with
// c_d == 1 (1-based, i.e. 0 here) for some d != mu.
static bool frozen(const int c[4], int mu) {
  for (int d = 0; d < 4; ++d)
    if (d != mu && c[d] == 0) return true;
  return false;
}

// mpi::heatbathcb::sweep (heatbath_mpi.cpp:37-56): lexicographic t, z, y, x, mu order.
static void sweep_ref(Lat& f, double beta, int n_hits, std::mt19937_64& rng) {
  for (size_t s = 0; s < f.V; ++s) {
    int c[4];
    f.coords(s, c);
    for (int mu = 0; mu < 4; ++mu)
      if (!frozen(c, mu))
        for (int h = 0; h < n_hits; ++h) hit_ref(f, s, mu, beta, rng);
  }
}

// mpi::shift::random_shift on one rank (src/mpi/Shift.cpp:109-186):
// new(c) = old(c - s), periodic, with s drawn in x, y, z, t order.
static void random_shift(Lat& f, std::mt19937_64& rng, std::vector<C>& tmp) {
  std::uniform_int_distribution<int> rand_l_shift(0, f.L[0] - 1);
  int sh[4];
  sh[0] = rand_l_shift(rng);
  sh[1] = rand_l_shift(rng);
  sh[2] = rand_l_shift(rng);
  sh[3] = rand_l_shift(rng);
  tmp.assign(f.u, f.u + f.V * 36);
  for (size_t s = 0; s < f.V; ++s) {
    int c[4];
    f.coords(s, c);
    int o[4];
    for (int d = 0; d < 4; ++d) o[d] = ((c[d] - sh[d]) % f.L[d] + f.L[d]) % f.L[d];
    size_t so = f.idx(o[0], o[1], o[2], o[3]);
    memcpy(f.u + s * 36, &tmp[so * 36], 36 * sizeof(C));
  }
}

// random_su3 (src/su3/utils.cpp:13-30): complex Gaussian 3x3, Householder QR (LAPACK /
// Eigen convention: beta = -sign(Re c0) |x|, tau = conj((beta - c0)/beta), Q = H0^* H1^* H2^*),
// then Q / det(Q)^(1/3).
static M3 random_su3_ref(std::mt19937_64& rng) {
  std::normal_distribution<double> gauss(0.0, 1.0);
  M3 z;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) z(i, j) = C(gauss(rng), gauss(rng));
  C tau[3];
  M3 a = z;
  for (int k = 0; k < 3; ++k) {
    double tail = 0.0;
    for (int i = k + 1; i < 3; ++i) tail += std::norm(a(i, k));
    C c0 = a(k, k);
    const double tol = std::numeric_limits<double>::min();
    double beta;
    if (tail <= tol && std::norm(c0.imag()) <= tol) {
      tau[k] = 0.0;
      beta = c0.real();
      for (int i = k + 1; i < 3; ++i) a(i, k) = 0.0;
    } else {
      beta = sqrt(std::norm(c0) + tail);
      if (c0.real() >= 0.0) beta = -beta;
      for (int i = k + 1; i < 3; ++i) a(i, k) = a(i, k) / (c0 - beta);
      tau[k] = std::conj((beta - c0) / beta);
    }
    a(k, k) = beta;
    // apply (I - tau v v^*) to the trailing columns, v = [1, a(k+1..,k)]
    for (int j = k + 1; j < 3; ++j) {
      C w = a(k, j);
      for (int i = k + 1; i < 3; ++i) w += std::conj(a(i, k)) * a(i, j);
      a(k, j) -= tau[k] * w;
      for (int i = k + 1; i < 3; ++i) a(i, j) -= tau[k] * a(i, k) * w;
    }
  }
  // Q = G0 G1 G2 with G_k = I - conj(tau_k) v_k v_k^*, accumulated from the right.
  M3 Q = ident();
  for (int k = 2; k >= 0; --k) {
    C h = std::conj(tau[k]);
    for (int j = 0; j < 3; ++j) {
      C w = Q(k, j);
      for (int i = k + 1; i < 3; ++i) w += std::conj(a(i, k)) * Q(i, j);
      Q(k, j) -= h * w;
      for (int i = k + 1; i < 3; ++i) Q(i, j) -= h * a(i, k) * w;
    }
  }
  C dq = det(Q);
  C root = std::pow(dq, 1.0 / 3.0);
  return scale(1.0 / root, Q);
}

// ---- Philox4x32-10 (Salmon et al., SC'11) and the library's checkerboard heatbath -----
struct P4 {
  uint32_t v[4];
};
static P4 philox(P4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c.v[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c.v[2];
    P4 n;
    n.v[0] = (uint32_t)(p1 >> 32) ^ c.v[1] ^ k0;
    n.v[1] = (uint32_t)p1;
    n.v[2] = (uint32_t)(p0 >> 32) ^ c.v[3] ^ k1;
    n.v[3] = (uint32_t)p0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}
static double u01(uint32_t w) { return ((double)w + 0.5) * 2.3283064365386963e-10; }

static const uint32_t KP_CAP = 4096;

// One subgroup update with Philox draws keyed (link, sweep, hsg, attempt); same
// arithmetic as the reference su2_step / generate_su2_kp.  Returns false at the cap.
static bool cb_subgroup(M3& U, const M3& A, int i, int j, double beta, uint32_t link, uint32_t sweep, uint32_t hsg,
                        uint32_t k0, uint32_t k1) {
  M3 W = mul(U, A);
  Q4 w = su2_to_quaternion(W(i, i), W(i, j), W(j, i), W(j, j));
  double k = sqrt(w.v[0] * w.v[0] + w.v[1] * w.v[1] + w.v[2] * w.v[2] + w.v[3] * w.v[3]);
  Q4 v = {{w.v[0] / k, w.v[1] / k, w.v[2] / k, w.v[3] / k}};
  double alpha = beta * k * 2.0 / 3.0;
  double a0 = 0;
  bool ok = false;
  for (uint32_t att = 0; att < KP_CAP; ++att) {
    P4 r = philox({{link, sweep, hsg, att}}, k0, k1);
    double delta = u01(r.v[0]), r1 = u01(r.v[1]), r2 = u01(r.v[2]), r3 = u01(r.v[3]);
    double cs = cos(2 * M_PI * r2);
    double lambda_sq = -0.5 / alpha * (log(r1) + cs * cs * log(r3));
    if (delta * delta <= 1.0 - lambda_sq) {
      a0 = 1.0 - 2.0 * lambda_sq;
      ok = true;
      break;
    }
  }
  if (!ok) return false;
  P4 r = philox({{link, sweep, hsg, 0xFFFFFFFFu}}, k0, k1);
  double phi = 2.0 * M_PI * u01(r.v[0]);
  double cos_theta = 2.0 * u01(r.v[1]) - 1.0;
  double sin_theta = sqrt(std::max(0.0, 1.0 - cos_theta * cos_theta));
  double rs = sqrt(std::max(0.0, 1.0 - a0 * a0));
  Q4 x = {{a0, rs * sin_theta * cos(phi), rs * sin_theta * sin(phi), rs * cos_theta}};
  Q4 q = qmult(x, qadj(v));
  U = mul(su2_quaternion_to_su3(q, i, j), U);
  return true;
}

// Frozen-link mask of the reference's block decomposition after a cumulative translation
// `shift` of the field: the reference moves the field by s (new(c) = old(c - s)) and freezes
// the links of local coordinate 0 in every direction d != mu of each L_core block
// (src/geometry/GeometryCB.cpp:33-56).  In the frame of the untranslated field that is
// link (c, mu) with (c_d + s_d) % lcore == 0 for some d != mu.
static bool frozen_shifted(const int c[4], int mu, int lcore, const int* shift) {
  for (int d = 0; d < 4; ++d)
    if (d != mu && (c[d] + shift[d]) % lcore == 0) return true;
  return false;
}

// Library schedule: checkerboard passes (mu, parity), Philox draws keyed by the link.  With
// lcore > 0, the links frozen by frozen_shifted(., lcore, shift) are left unchanged.
static uint64_t heatbath_cb(Lat& f, double beta, int n_sweeps, int n_hits, uint64_t seed, uint64_t sweep_offset,
                            int lcore = 0, const int* shift = nullptr) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  uint64_t fails = 0;
  for (int sw = 0; sw < n_sweeps; ++sw) {
    const uint32_t sweep = (uint32_t)(sweep_offset + (uint64_t)sw);
    for (int mu = 0; mu < 4; ++mu)
      for (int par = 0; par < 2; ++par)
        for (size_t s = 0; s < f.V; ++s) {
          int c[4];
          f.coords(s, c);
          if (((c[0] + c[1] + c[2] + c[3]) & 1) != par) continue;
          if (lcore > 0 && frozen_shifted(c, mu, lcore, shift)) continue;
          M3 A = staple(f, s, mu);
          M3 U = f.get(s, mu);
          const uint32_t link = (uint32_t)mu * (uint32_t)f.V + (uint32_t)s;
          for (int h = 0; h < n_hits; ++h) {
            const uint32_t hb = (uint32_t)h << 2;
            fails += !cb_subgroup(U, A, 0, 1, beta, link, sweep, hb | 0u, k0, k1);
            fails += !cb_subgroup(U, A, 1, 2, beta, link, sweep, hb | 1u, k0, k1);
            fails += !cb_subgroup(U, A, 0, 2, beta, link, sweep, hb | 2u, k0, k1);
          }
          f.set(s, mu, U);
        }
  }
  return fails;
}

// SU(3) matrix from 12 standard normals: rows 0, 1 complex Gaussian, Gram-Schmidt,
// row 2 = conj(row0 x row1) (Haar-distributed).
static M3 haar_from_normals(const double n[12]) {
  C r0[3], r1[3];
  for (int j = 0; j < 3; ++j) {
    r0[j] = C(n[2 * j], n[2 * j + 1]);
    r1[j] = C(n[6 + 2 * j], n[6 + 2 * j + 1]);
  }
  double n0 = std::norm(r0[0]) + std::norm(r0[1]) + std::norm(r0[2]);
  for (auto& v : r0) v /= sqrt(n0);
  C d = std::conj(r0[0]) * r1[0] + std::conj(r0[1]) * r1[1] + std::conj(r0[2]) * r1[2];
  for (int j = 0; j < 3; ++j) r1[j] -= d * r0[j];
  double n1 = std::norm(r1[0]) + std::norm(r1[1]) + std::norm(r1[2]);
  for (auto& v : r1) v /= sqrt(n1);
  M3 u;
  for (int j = 0; j < 3; ++j) {
    u(0, j) = r0[j];
    u(1, j) = r1[j];
  }
  u(2, 0) = std::conj(r0[1] * r1[2] - r0[2] * r1[1]);
  u(2, 1) = std::conj(r0[2] * r1[0] - r0[0] * r1[2]);
  u(2, 2) = std::conj(r0[0] * r1[1] - r0[1] * r1[0]);
  return u;
}

// Haar SU(3) from the Philox stream: 12 normals by Box-Muller from counters (id, 0, tag, call).
static M3 haar_philox(uint32_t id, uint32_t tag, uint32_t k0, uint32_t k1) {
  double n[12];
  for (int call = 0; call < 3; ++call) {
    P4 r = philox({{id, 0u, tag, (uint32_t)call}}, k0, k1);
    for (int pr = 0; pr < 2; ++pr) {
      double u1 = u01(r.v[2 * pr]), u2 = u01(r.v[2 * pr + 1]);
      double rad = sqrt(-2.0 * log(u1));
      n[call * 4 + pr * 2 + 0] = rad * cos(2 * M_PI * u2);
      n[call * 4 + pr * 2 + 1] = rad * sin(2 * M_PI * u2);
    }
  }
  return haar_from_normals(n);
}

const uint32_t DOMAIN_HOT = 0x80000000u, DOMAIN_GAUGE = 0x90000000u;

// Reference-schedule chain state (one rank): lattice + mt19937_64.
struct RefChain {
  int dims[4];
  std::vector<C> links;
  std::mt19937_64 rng;
  std::vector<C> tmp;
  std::vector<uint32_t> nbtab;
  Lat lat() {
    Lat l;
    for (int d = 0; d < 4; ++d) l.L[d] = dims[d];
    l.V = (size_t)dims[0] * dims[1] * dims[2] * dims[3];
    l.u = links.data();
    if (nbtab.empty()) attach_nb_table(l, nbtab);
    l.nbt = nbtab.data();
    return l;
  }
};

// ---- event-chain Monte Carlo (src/ecmc/ecmc_mpi_cb.cpp, src/su3/utils.cpp) ----------------
// Library form of mpi::ecmccb::sample_persistant (ecmc_mpi_cb.cpp:496-637): the lattice is
// cut into blocks of edge l_core (one per MPI rank in the reference) and every block runs
// its own persistent chain.  The chains are independent: the links a chain reads outside its
// own active links are frozen in their owners' blocks (GeometryCB.cpp:33-56).  Randomness:
// chain c's k-th uniform comes from Philox4x32-10 with counter (k_lo, k_hi, c, ECMC_CHAIN) and
// key = seed.  Each chain has its own set of SU(3) elements near the identity (ecmc_set), as
// each rank of the reference has: renewed at the start of every call and whenever the chain's
// set_counter (lifts since the last renewal) reaches a multiple of 10000 at the top of the event
// loop (ecmc_mpi_cb.cpp:560-566).  Element pair p of generation gen of chain c in call `call`
// comes from counters (3p + j, c, call, ECMC_SETC ^ gen), j < 3, so the set is never stored.
const uint32_t ECMC_CHAIN = 0xECEC0001u, ECMC_SET = 0xECEC0002u, ECMC_SETC = 0xECE50000u;
const int ECMC_SET_SIZE = 10001;  // sample_persistant's set (ecmc_mpi_cb.cpp:560)
const uint64_t ECMC_MAX_EVENTS = 1ull << 26;

// Same layout as qcb_ecmc_chain in the library's C header.
struct EcmcChain {
  double R[18];
  double theta_refresh_site, theta_refresh_R;
  double travelled_site, travelled_R;
  uint64_t draws, events, lifts, revs;
  int32_t site[4];
  int32_t mu, epsilon, initialized, status;
  int32_t set_counter;  // lifts since the chain's set was last renewed (mod 10000)
  int32_t pad[3];
};
static_assert(sizeof(EcmcChain) == 256, "chain record is 256 bytes");

struct EcmcParams {
  double beta, theta_sample, theta_refresh_site, theta_refresh_R, epsilon_set;
  int poisson, l_core;
};

// Uniform in (0, 1) from two 32-bit words: (top 53 bits of hi:lo + 1/2) 2^-53.
static double u53(uint32_t lo, uint32_t hi) {
  const uint64_t x = ((((uint64_t)hi) << 32) | lo) >> 11;
  return ((double)x + 0.5) * 1.1102230246251565e-16;
}

struct EcmcStream {
  uint32_t chain, k0, k1;
  uint64_t* draws;
  double uni() {
    const uint64_t n = (*draws)++;
    P4 r = philox({{(uint32_t)n, (uint32_t)(n >> 32), chain, ECMC_CHAIN}}, k0, k1);
    return u53(r.v[0], r.v[1]);
  }
  // random_su3 (src/su3/utils.cpp:13-30) redrawn: Haar SU(3) from 12 Box-Muller normals.
  M3 haar() {
    double n[12];
    for (int k = 0; k < 6; ++k) {
      const double u1 = uni(), u2 = uni();
      const double rad = sqrt(-2.0 * log(u1));
      n[2 * k] = rad * cos(2 * M_PI * u2);
      n[2 * k + 1] = rad * sin(2 * M_PI * u2);
    }
    return haar_from_normals(n);
  }
};

// random_SU3_epsilon (src/su3/utils.cpp:66-105): product of the SU(2) elements
// (sqrt(1 - eps^2), eps r/|r|) embedded in subgroups (0,1), (0,2), (1,2), r from (-1/2, 1/2)^3.
static M3 su3_near_identity(double eps, const double r[9]) {
  static const int sub[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  M3 M = ident();
  for (int s = 0; s < 3; ++s) {
    const double r1 = r[3 * s], r2 = r[3 * s + 1], r3 = r[3 * s + 2];
    const double norm = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
    Q4 x = {{sqrt(1 - eps * eps), eps * r1 / norm, eps * r2 / norm, eps * r3 / norm}};
    M = mul(M, su2_quaternion_to_su3(x, sub[s][0], sub[s][1]));
  }
  return M;
}

// solve_reject_fast (ecmc_mpi_cb.h:59-94): along U(theta) = R diag(e^{i eps theta},
// e^{-i eps theta}, 1) R^dagger U one staple's action is A cos(theta) + eps B sin(theta) + const;
// returns the angle at which the integral of the positive part of its derivative reaches gamma.
static double solve_reject(double A, double B, double gamma, int eps) {
  if (eps == -1) B = -B;
  const double R = hypot(A, B), invR = 1.0 / R, period = 2.0 * R;
  const double disc = floor(gamma / period);
  gamma -= disc * period;
  double phi = atan2(-A, B);
  if (phi < 0.0) phi += 2.0 * M_PI;
  const double p1 = R - A;
  double alpha;
  if (phi < M_PI * 0.5 || phi > M_PI * 1.5)
    alpha = (gamma > p1) ? (gamma - p1) * invR - 1.0 : (gamma + A) * invR;
  else
    alpha = gamma * invR - 1.0;
  alpha = alpha > 1.0 ? 1.0 : (alpha < -1.0 ? -1.0 : alpha);
  double theta = phi + asin(alpha);
  if (theta < 0.0) theta += 2.0 * M_PI;
  if (theta >= 2.0 * M_PI) theta -= 2.0 * M_PI;
  return theta + 2.0 * M_PI * disc;
}

// compute_reject_angles_fast (ecmc_mpi_cb.cpp:197-246), one staple S with T = R^dagger U:
// P = T S R, A = -(beta/3) Re(P00 + P11), B = -(beta/3) Im(P11 - P00).
static double reject_angle(const M3& T, const M3& S, const M3& R, double beta, double gamma, int eps) {
  C m0[3], m1[3];
  for (int c = 0; c < 3; ++c) {
    m0[c] = T(0, 0) * S(0, c) + T(0, 1) * S(1, c) + T(0, 2) * S(2, c);
    m1[c] = T(1, 0) * S(0, c) + T(1, 1) * S(1, c) + T(1, 2) * S(2, c);
  }
  const C P00 = m0[0] * R(0, 0) + m0[1] * R(1, 0) + m0[2] * R(2, 0);
  const C P11 = m1[0] * R(0, 1) + m1[1] * R(1, 1) + m1[2] * R(2, 1);
  const double br = -(beta / 3.0);
  return solve_reject((P00.real() + P11.real()) * br, (P11.imag() - P00.imag()) * br, gamma, eps);
}

// compute_ds (ecmc_mpi_cb.cpp:263-274): Im[(R^dagger P R)_00 - (R^dagger P R)_11].
static double compute_ds(const M3& P, const M3& R) {
  M3 M = mul(P, R);
  C res = 0.0;
  for (int k = 0; k < 3; ++k) {
    res += std::conj(R(k, 0)) * M(k, 0);
    res -= std::conj(R(k, 1)) * M(k, 1);
  }
  return res.imag();
}

static int dsign(double x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

// One chain's block: block coordinates b, the lattice, and the cumulative shift of the
// field's frame.  Local coordinates lc (each in [-1, l]; -1 and l are the neighbours' faces,
// the reference's halo) map to the stored site b_d l + lc_d - cum_d (mod L_d).
struct EcmcBlock {
  Lat* f;
  int l, b[4], cum[4];
  size_t site(const int lc[4]) const {
    int c[4];
    for (int d = 0; d < 4; ++d) c[d] = ((b[d] * l + lc[d] - cum[d]) % f->L[d] + f->L[d]) % f->L[d];
    return f->idx(c[0], c[1], c[2], c[3]);
  }
  M3 get(const int lc[4], int mu) const { return f->get(site(lc), mu); }
  // GeometryCB::is_frozen in block-local terms: the halo (outside [0, l)) and the links
  // leaving local coordinate 0 in a direction d != mu.
  bool frozen(const int lc[4], int mu) const {
    for (int d = 0; d < 4; ++d)
      if (lc[d] < 0 || lc[d] >= l || (d != mu && lc[d] == 0)) return true;
    return false;
  }
};

static void shifted(const int a[4], int d1, int s1, int d2, int s2, int out[4]) {
  for (int d = 0; d < 4; ++d) out[d] = a[d];
  if (d1 >= 0) out[d1] += s1;
  if (d2 >= 0) out[d2] += s2;
}

// Element iset of a chain's set (ecmc_set, src/su3/utils.cpp:119-127: set[0] = 1,
// set[2p+1] = random_SU3_epsilon, set[2p+2] = its adjoint) for generation gen of chain c in
// call `call`, drawn from the counters of element pair p.
static M3 ecmc_set_elem(double eps, uint32_t k0, uint32_t k1, uint32_t chain, uint32_t call, uint32_t gen, int iset) {
  if (iset == 0) return ident();
  const uint32_t pidx = (uint32_t)(iset - 1) >> 1;
  double r[12];
  for (uint32_t j = 0; j < 3; ++j) {
    P4 w = philox({{3 * pidx + j, chain, call, ECMC_SETC ^ (gen & 0xFFFFu)}}, k0, k1);
    for (int t = 0; t < 4; ++t) r[4 * j + t] = ((double)w.v[t] + 0.5) * 2.3283064365386963e-10 - 0.5;
  }
  const M3 M = su3_near_identity(eps, r);
  return (iset & 1) ? M : adj(M);
}

// The random draws of one chain, two policies.  LibDraws: the library's counter-based stream
// (Philox) and the chain's own set, renewed as the reference renews its rank's set.  RefDraws
// (below): the reference's std::mt19937_64 with its std:: distributions and its own stored
// set, regenerated as the reference does.
struct LibDraws {
  EcmcStream g;
  double eps_set;
  uint32_t call;
  int32_t* set_counter;
  uint32_t gen;
  int l;
  // random_site (ecmc_mpi_cb.cpp:359-367): local coordinates 1 .. l-2 (padded 2 .. L-1)
  void site(int lc[4]) {
    for (int d = 0; d < 4; ++d) lc[d] = 1 + (int)(g.uni() * (double)(l - 2));
  }
  int dir() { return (int)(g.uni() * 4.0); }
  int sense() { return g.uni() < 0.5 ? -1 : 1; }
  M3 haar() { return g.haar(); }
  double expo(double mean) { return -log(g.uni()) * mean; }
  double gamma() { return -log(g.uni()); }
  double uniform() { return g.uni(); }
  int set_index() { return (int)(g.uni() * (double)ECMC_SET_SIZE); }
  M3 set_elem(int i) const { return ecmc_set_elem(eps_set, g.k0, g.k1, g.chain, call, gen, i); }
  void call_start() { gen = 0; }
  void loop_start() {
    if (*set_counter % 10000 == 0) {
      ++gen;
      *set_counter = 0;
    }
  }
  void on_lift() { ++*set_counter; }
};

// sample_persistant (ecmc_mpi_cb.cpp:496-637) for one chain: events until the chain has
// travelled theta_sample; the state persists across calls, the chain's set of near-identity
// elements is renewed at every call and every 10000 lifts.
template <class D>
static void ecmc_chain(const EcmcBlock& blk, const EcmcParams& p, D& g, EcmcChain& st) {
  Lat& f = *blk.f;
  st.status = 0;  // the record keeps the bits of the latest call
  M3 R;
  if (!st.initialized) {
    g.site(st.site);
    st.mu = g.dir();
    st.epsilon = g.sense();
    R = g.haar();
    st.theta_refresh_site = p.poisson ? g.expo(p.theta_refresh_site) : p.theta_refresh_site;
    st.theta_refresh_R = p.poisson ? g.expo(p.theta_refresh_R) : p.theta_refresh_R;
    st.travelled_site = st.travelled_R = 0.0;
    st.events = st.lifts = 0;
    st.initialized = 1;
  } else {
    memcpy(R.a, st.R, sizeof R.a);
  }
  const double theta_sample = p.poisson ? g.expo(p.theta_sample) : p.theta_sample;
  g.call_start();
  double trav_sample = 0.0;
  int lc[4] = {st.site[0], st.site[1], st.site[2], st.site[3]};
  int mu = st.mu, eps = st.epsilon;
  for (uint64_t ev = 0;; ++ev) {
    if (ev >= ECMC_MAX_EVENTS) {
      st.status |= 2;
      break;
    }
    g.loop_start();
    const size_t x = blk.site(lc);
    const M3 U = f.get(x, mu);
    const M3 T = mul(adj(R), U);
    // compute_list_staples (ecmc_mpi_cb.cpp:12-36): for each nu != mu, forward then backward
    double best = 0.0;
    int j = 0, k = 0;
    for (int nu = 0; nu < 4; ++nu) {
      if (nu == mu) continue;
      int a[4], c[4], d[4], e[4];
      shifted(lc, mu, 1, -1, 0, a);   // x+mu
      shifted(lc, nu, 1, -1, 0, c);   // x+nu
      shifted(lc, mu, 1, nu, -1, d);  // x+mu-nu
      shifted(lc, nu, -1, -1, 0, e);  // x-nu
      M3 S = mul(blk.get(a, nu), adj(mul(f.get(x, nu), blk.get(c, mu))));
      double rej = reject_angle(T, S, R, p.beta, g.gamma(), eps);
      if (k == 0 || rej < best) best = rej, j = k;
      ++k;
      S = mul(adj(mul(blk.get(e, mu), blk.get(d, nu))), blk.get(e, nu));
      rej = reject_angle(T, S, R, p.beta, g.gamma(), eps);
      if (rej < best) best = rej, j = k;
      ++k;
    }
    const double d_sample = theta_sample - trav_sample;
    const double d_site = st.theta_refresh_site - st.travelled_site;
    const double d_R = st.theta_refresh_R - st.travelled_R;
    const double step = std::min({best, d_sample, d_site, d_R});
    if (!std::isfinite(step)) {
      st.status |= 1;
      break;
    }
    // update (ecmc_mpi_cb.cpp:340-356): U <- R diag(e^{i xi}, e^{-i xi}, 1) R^dagger U, xi = eps theta
    auto update = [&](double theta) {
      const double xi = eps * theta, cs = cos(xi), sn = sin(xi);
      M3 T2 = T;
      for (int cc = 0; cc < 3; ++cc) {
        T2(0, cc) *= C(cs, sn);
        T2(1, cc) *= C(cs, -sn);
      }
      f.set(x, mu, mul(R, T2));
      st.events++;
    };
    if (step == d_sample) {
      update(d_sample);
      st.travelled_site += d_sample;
      st.travelled_R += d_sample;
      break;
    } else if (step == d_site) {
      update(d_site);
      trav_sample += d_site;
      st.travelled_R += d_site;
      st.travelled_site = 0.0;
      if (p.poisson) st.theta_refresh_site = g.expo(p.theta_refresh_site);
      g.site(lc);
      mu = g.dir();
      eps = g.sense();
    } else if (step == d_R) {
      update(d_R);
      trav_sample += d_R;
      st.travelled_site += d_R;
      st.travelled_R = 0.0;
      if (p.poisson) st.theta_refresh_R = g.expo(p.theta_refresh_R);
      R = g.haar();
    } else {
      update(best);
      trav_sample += best;
      st.travelled_site += best;
      st.travelled_R += best;
      // lift_improved_fast (ecmc_mpi_cb.cpp:277-337) on plaquette j; its links
      // (GeometryCB.cpp:58-90): 0 = (x, mu); forward 1 = (x+mu, nu), 2 = (x+nu, mu),
      // 3 = (x, nu); backward 1 = (x+mu-nu, nu), 2 = (x-nu, mu), 3 = (x-nu, nu).
      int nu = 0;
      for (int q = 0, n = 0; q < 4; ++q)
        if (q != mu) {
          if (n == j / 2) nu = q;
          ++n;
        }
      const bool fwd = (j % 2) == 0;
      int lk[4][4], ld[4] = {mu, nu, mu, nu};
      shifted(lc, -1, 0, -1, 0, lk[0]);
      if (fwd) {
        shifted(lc, mu, 1, -1, 0, lk[1]);
        shifted(lc, nu, 1, -1, 0, lk[2]);
        shifted(lc, -1, 0, -1, 0, lk[3]);
      } else {
        shifted(lc, mu, 1, nu, -1, lk[1]);
        shifted(lc, nu, -1, -1, 0, lk[2]);
        shifted(lc, nu, -1, -1, 0, lk[3]);
      }
      const M3 U0 = f.get(x, mu), U1 = blk.get(lk[1], nu), U2 = blk.get(lk[2], mu), U3 = blk.get(lk[3], nu);
      M3 P[4];
      if (fwd) {
        const M3 U01 = mul(U0, U1), U32 = mul(U3, U2);
        P[0] = mul(U01, adj(U32));
        P[1] = mul(mul(U1, adj(U32)), U0);
        P[2] = mul(mul(U2, adj(U01)), U3);
        P[3] = adj(P[0]);
      } else {
        const M3 U21 = mul(U2, U1), Tb = mul(U0, adj(U21));
        P[0] = mul(Tb, U3);
        P[1] = mul(mul(mul(U1, adj(U0)), adj(U3)), U2);
        P[3] = mul(U3, Tb);
        P[2] = adj(P[3]);
      }
      double ab[4], sum = 0.0;
      int sg[4];
      for (int i = 0; i < 4; ++i) {
        const double ds = blk.frozen(lk[i], ld[i]) ? 0.0 : compute_ds(P[i], R);
        sg[i] = dsign(ds);
        ab[i] = fabs(ds);
        sum += ab[i];
      }
      double pr[4];
      for (int i = 0; i < 4; ++i) pr[i] = ab[i] / sum;
      // selectVariable (ecmc_mpi_cb.cpp:252-260)
      const double r = g.uniform();
      const int idx = r < pr[0] ? 0 : (r < pr[0] + pr[1] ? 1 : (r < pr[0] + pr[1] + pr[2] ? 2 : 3));
      const int iset = g.set_index();
      const M3 Rn = mul(g.set_elem(iset), R);
      const double ds_old = sg[idx] * ab[idx];
      const double ds_new = compute_ds(P[idx], Rn);
      int new_eps = -sg[idx];
      if (fabs(ds_old) < fabs(ds_new)) {
        R = Rn;
        new_eps = -dsign(ds_new);
      } else if (g.uniform() < fabs(ds_new) / fabs(ds_old)) {
        R = Rn;
        new_eps = -dsign(ds_new);
      }
      bool same = true;
      for (int d = 0; d < 4; ++d) same = same && (lk[idx][d] == lc[d]);
      st.revs += same ? 1 : 0;
      st.lifts++;
      g.on_lift();
      for (int d = 0; d < 4; ++d) lc[d] = lk[idx][d];
      mu = ld[idx];
      eps = new_eps;
    }
  }
  for (int d = 0; d < 4; ++d) st.site[d] = lc[d];
  st.mu = mu;
  st.epsilon = eps;
  memcpy(st.R, R.a, sizeof R.a);
}


// The reference's own draws (one MPI rank, std::mt19937_64 rng(seed + rank)): the static
// distributions of sample_persistant, random_site, lift_improved_fast and
// compute_reject_angles_fast (ecmc_mpi_cb.cpp:197-567), random_su3 by Householder QR
// (utils.cpp:13-30), and the rank's set of 10001 elements regenerated at the start of every
// call and whenever set_counter % 10000 == 0 at the top of the event loop (:560-566).
struct RefDraws {
  std::mt19937_64* rng;
  int l;
  double eps_set;
  std::vector<M3>* set;
  uint64_t* set_counter;
  std::uniform_int_distribution<int> coord, rdir, reps;
  std::uniform_real_distribution<double> unif01;
  RefDraws(std::mt19937_64* r, int l_, double e, std::vector<M3>* s, uint64_t* sc)
      : rng(r), l(l_), eps_set(e), set(s), set_counter(sc), coord(2, l_ - 1), rdir(0, 3), reps(0, 1), unif01(0.0, 1.0) {}
  void site(int lc[4]) {
    for (int d = 0; d < 4; ++d) lc[d] = coord(*rng) - 1;  // padded x, y, z, t -> local
  }
  int dir() { return rdir(*rng); }
  int sense() { return 2 * reps(*rng) - 1; }
  M3 haar() { return random_su3_ref(*rng); }
  double expo(double mean) { return std::exponential_distribution<double>(1.0 / mean)(*rng); }
  double gamma() { return -std::log(unif01(*rng)); }
  double uniform() { return unif01(*rng); }
  int set_index() { return (int)std::uniform_int_distribution<size_t>(0, set->size() - 1)(*rng); }
  const M3& set_elem(int i) const { return (*set)[i]; }
  // ecmc_set with random_SU3_epsilon (utils.cpp:66-127): 9 uniforms in (-1/2, 1/2) per pair
  void regenerate() {
    std::uniform_real_distribution<double> u(-0.5, 0.5);
    set->assign(ECMC_SET_SIZE, ident());
    for (int pidx = 0; pidx < (ECMC_SET_SIZE - 1) / 2; ++pidx) {
      double r[9];
      for (int d = 0; d < 9; ++d) r[d] = u(*rng);
      (*set)[2 * pidx + 1] = su3_near_identity(eps_set, r);
      (*set)[2 * pidx + 2] = adj((*set)[2 * pidx + 1]);
    }
  }
  void call_start() { regenerate(); }
  void loop_start() {
    if (*set_counter % 10000 == 0) {
      regenerate();
      *set_counter = 0;
    }
  }
  void on_lift() { ++*set_counter; }
};

// generate_ecmc_cb on one rank (n_core_dims = 1, src/bin/gauge_ecmc_ncb.cpp:20-269): the
// lattice is one L^4 block with frozen faces; each shift is random_shift (field moved) then
// sample_persistant.
struct RefEcmcRun {
  int dims[4];
  std::vector<C> links, tmp;
  std::mt19937_64 rng;
  EcmcParams p;
  EcmcChain st;
  std::vector<M3> set;
  uint64_t set_counter = 0;
  Lat lat() {
    Lat l;
    for (int d = 0; d < 4; ++d) l.L[d] = dims[d];
    l.V = (size_t)dims[0] * dims[1] * dims[2] * dims[3];
    l.u = links.data();
    return l;
  }
  void shift_and_sample() {
    Lat f = lat();
    random_shift(f, rng, tmp);
    RefDraws g(&rng, p.l_core, p.epsilon_set, &set, &set_counter);
    EcmcBlock blk;
    blk.f = &f;
    blk.l = p.l_core;
    for (int d = 0; d < 4; ++d) blk.b[d] = blk.cum[d] = 0;
    ecmc_chain(blk, p, g, st);
  }
};

}  // namespace orc

using namespace orc;

extern "C" {

int orc_plaquette(const double* aos, const int dims[4], double* out) {
  Lat f = make(const_cast<double*>(aos), dims);
  *out = plaquette_sum(f) / (6.0 * (double)f.V);
  return 0;
}

int orc_topo_qe(const double* aos, const int dims[4], double* q, double* e) {
  Lat f = make(const_cast<double*>(aos), dims);
  double qt, et;
  topo_qe(f, &qt, &et);
  *q = qt;
  *e = et / (double)f.V;
  return 0;
}

// topo_charge_flowed (observables_mpi.cpp:153-178) on a copy of aos.
int orc_flow_measure(const double* aos, const int dims[4], double eps, int n_steps_gf, int n_rk_steps, double* tQE) {
  size_t V = (size_t)dims[0] * dims[1] * dims[2] * dims[3];
  std::vector<double> copy(aos, aos + V * 72);
  Lat f = make(copy.data(), dims);
  std::vector<uint32_t> tab;
  attach_nb_table(f, tab);
  Flow gf{&f, eps, {}, {}};
  double t = 0.0;
  for (int st = 0; st < n_steps_gf; st++) {
    double q, e;
    topo_qe(f, &q, &e);
    tQE[3 * st] = t;
    tQE[3 * st + 1] = q;
    tQE[3 * st + 2] = e / (double)V;
    for (int r = 0; r < n_rk_steps; r++) {
      gf.rk3_step();
      t += eps;
    }
  }
  return 0;
}

int orc_flow_steps(double* aos, const int dims[4], double eps, int n) {
  Lat f = make(aos, dims);
  std::vector<uint32_t> tab;
  attach_nb_table(f, tab);
  Flow gf{&f, eps, {}, {}};
  for (int r = 0; r < n; ++r) gf.rk3_step();
  return 0;
}

int orc_staple(const double* aos, const int dims[4], long site, int mu, double* out18) {
  Lat f = make(const_cast<double*>(aos), dims);
  M3 a = staple(f, (size_t)site, mu);
  memcpy(out18, a.a, sizeof a.a);
  return 0;
}

int orc_exp_su3(const double* z18, double coeff, double* out18) {
  M3 z;
  memcpy(z.a, z18, sizeof z.a);
  M3 r = exp_luscher(z, coeff);
  memcpy(out18, r.a, sizeof r.a);
  return 0;
}

int orc_proj_lie(const double* a18, double* out18) {
  M3 a;
  memcpy(a.a, a18, sizeof a.a);
  proj_lie(a);
  memcpy(out18, a.a, sizeof a.a);
  return 0;
}

int orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  P4 r = philox({{ctr[0], ctr[1], ctr[2], ctr[3]}}, key[0], key[1]);
  memcpy(out, r.v, sizeof r.v);
  return 0;
}

uint64_t orc_mt19937_64_nth(uint64_t seed, int n) {
  std::mt19937_64 g(seed);
  uint64_t v = 0;
  for (int k = 0; k < n; ++k) v = g();
  return v;
}

// Library schedule (checkerboard, Philox) restated in FP64; returns KP cap hits.
uint64_t orc_heatbath_cb(double* aos, const int dims[4], double beta, int n_sweeps, int n_hits, uint64_t seed,
                         uint64_t sweep_offset) {
  Lat f = make(aos, dims);
  return heatbath_cb(f, beta, n_sweeps, n_hits, seed, sweep_offset);
}

// The same with the reference's frozen links of L_core blocks after a cumulative shift.
uint64_t orc_heatbath_cb_frozen(double* aos, const int dims[4], double beta, int n_sweeps, int n_hits, uint64_t seed,
                                uint64_t sweep_offset, int lcore, const int shift[4]) {
  Lat f = make(aos, dims);
  int sh[4];
  for (int d = 0; d < 4; ++d) sh[d] = ((shift[d] % lcore) + lcore) % lcore;
  return heatbath_cb(f, beta, n_sweeps, n_hits, seed, sweep_offset, lcore, sh);
}

// The first n shift vectors of mpi::shift::random_shift (src/mpi/Shift.cpp:163-172): four
// draws of uniform_int_distribution<int>(0, L - 1) from std::mt19937_64(seed) per shift.
int orc_shift_sequence(uint64_t seed, int L, int n, int* out) {
  std::mt19937_64 rng(seed);
  std::uniform_int_distribution<int> d(0, L - 1);
  for (int k = 0; k < 4 * n; ++k) out[k] = d(rng);
  return 0;
}

int orc_hot_start_philox(double* aos, const int dims[4], uint64_t seed) {
  Lat f = make(aos, dims);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (size_t s = 0; s < f.V; ++s)
    for (int mu = 0; mu < 4; ++mu) f.set(s, mu, haar_philox((uint32_t)mu * (uint32_t)f.V + (uint32_t)s, DOMAIN_HOT, k0, k1));
  return 0;
}

int orc_gauge_transform_philox(double* aos, const int dims[4], uint64_t seed) {
  Lat f = make(aos, dims);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  std::vector<C> out(f.V * 36);
  for (size_t s = 0; s < f.V; ++s)
    for (int mu = 0; mu < 4; ++mu) {
      M3 G = haar_philox((uint32_t)s, DOMAIN_GAUGE, k0, k1);
      M3 Gy = haar_philox((uint32_t)f.nb(s, mu, +1), DOMAIN_GAUGE, k0, k1);
      M3 r = mul(mul(G, f.get(s, mu)), adj(Gy));
      memcpy(&out[(s * 4 + mu) * 9], r.a, sizeof r.a);
    }
  memcpy(f.u, out.data(), out.size() * sizeof(C));
  return 0;
}

// Kennedy-Pendleton sampler of the reference with mt19937_64 (for distribution tests).
int orc_kp_samples(double beta, double k, int n, uint64_t seed, double* a0) {
  std::mt19937_64 rng(seed);
  for (int i = 0; i < n; ++i) a0[i] = generate_su2_kp(beta, k, rng).v[0];
  return 0;
}

// ---- reference-schedule chain (frozen links + random shift, mt19937_64) ---------------
// generate_hb_cb (src/bin/gauge_hb_ncb.cpp:18-179) for one rank (n_core_dims = 1).
void* orc_ref_create(int L, int seed, int cold_start) {
  RefChain* c = new RefChain();
  for (int d = 0; d < 4; ++d) c->dims[d] = L;
  size_t V = (size_t)L * L * L * L;
  c->links.assign(V * 36, C(0.0, 0.0));
  c->rng.seed((uint64_t)(int64_t)seed + 0);  // rp.seed + topo.rank
  Lat f = c->lat();
  for (size_t s = 0; s < V; ++s)
    for (int mu = 0; mu < 4; ++mu) f.set(s, mu, ident());
  if (!cold_start)  // GaugeField::hot_start (GaugeField.cpp:10-20), t, z, y, x, mu order
    for (size_t s = 0; s < V; ++s)
      for (int mu = 0; mu < 4; ++mu) f.set(s, mu, random_su3_ref(c->rng));
  return c;
}

void orc_ref_destroy(void* h) { delete static_cast<RefChain*>(h); }

// n_shift iterations of: random_shift, N_sweeps sweeps, plaquette -> plaq[i].
int orc_ref_run(void* h, double beta, int n_shift, int n_sweeps, int n_hits, double* plaq) {
  RefChain* c = static_cast<RefChain*>(h);
  Lat f = c->lat();
  for (int i = 0; i < n_shift; ++i) {
    random_shift(f, c->rng, c->tmp);
    for (int s = 0; s < n_sweeps; ++s) sweep_ref(f, beta, n_hits, c->rng);
    if (plaq) plaq[i] = plaquette_sum(f) / (6.0 * (double)f.V);
  }
  return 0;
}

// Sweeps only (no shift, no measurement): for timing the reference update rate.
int orc_ref_sweeps(void* h, double beta, int n_sweeps, int n_hits) {
  RefChain* c = static_cast<RefChain*>(h);
  Lat f = c->lat();
  for (int s = 0; s < n_sweeps; ++s) sweep_ref(f, beta, n_hits, c->rng);
  return 0;
}

int orc_ref_get_links(void* h, double* aos) {
  RefChain* c = static_cast<RefChain*>(h);
  memcpy(aos, c->links.data(), c->links.size() * sizeof(C));
  return 0;
}
int orc_ref_set_links(void* h, const double* aos) {
  RefChain* c = static_cast<RefChain*>(h);
  memcpy(c->links.data(), aos, c->links.size() * sizeof(C));
  return 0;
}

// ---- event-chain Monte Carlo --------------------------------------------------------------
int orc_ecmc_solve_reject(double A, double B, double gamma, int eps, double* out) {
  *out = solve_reject(A, B, gamma, eps);
  return 0;
}

int orc_ecmc_compute_ds(const double* p18, const double* r18, double* out) {
  M3 P, R;
  memcpy(P.a, p18, sizeof P.a);
  memcpy(R.a, r18, sizeof R.a);
  *out = compute_ds(P, R);
  return 0;
}

// The whole set (ECMC_SET_SIZE matrices of 18 doubles) of generation gen of chain `chain` in
// call `call`.
int orc_ecmc_set(double eps, uint64_t seed, uint32_t chain, uint64_t call, uint32_t gen, double* out) {
  for (int i = 0; i < ECMC_SET_SIZE; ++i) {
    const M3 m = ecmc_set_elem(eps, (uint32_t)seed, (uint32_t)(seed >> 32), chain, (uint32_t)call, gen, i);
    memcpy(out + 18 * i, m.a, sizeof m.a);
  }
  return 0;
}

// One sample call of every chain.  dp = {beta, theta_sample, theta_refresh_site,
// theta_refresh_R, epsilon_set}, ip = {poisson, l_core}; cum = cumulative shift of the field's
// frame; chains = prod(dims / l_core) records, chain id ((bx nby + by) nbz + bz) nbt + bt.
int orc_ecmc_sample(double* aos, const int dims[4], const double dp[5], const int ip[2], uint64_t seed, uint64_t call,
                    const int cum[4], void* chains) {
  Lat f = make(aos, dims);
  EcmcParams p{dp[0], dp[1], dp[2], dp[3], dp[4], ip[0], ip[1]};
  const int l = p.l_core;
  int nb[4];
  for (int d = 0; d < 4; ++d) {
    if (l < 3 || dims[d] % l) return 1;
    nb[d] = dims[d] / l;
  }
  EcmcChain* st = static_cast<EcmcChain*>(chains);
  EcmcBlock blk;
  blk.f = &f;
  blk.l = l;
  for (int d = 0; d < 4; ++d) blk.cum[d] = ((cum[d] % dims[d]) + dims[d]) % dims[d];
  uint32_t id = 0;
  for (int bx = 0; bx < nb[0]; ++bx)
    for (int by = 0; by < nb[1]; ++by)
      for (int bz = 0; bz < nb[2]; ++bz)
        for (int bt = 0; bt < nb[3]; ++bt, ++id) {
          blk.b[0] = bx, blk.b[1] = by, blk.b[2] = bz, blk.b[3] = bt;
          if (!st[id].initialized) st[id].set_counter = 0;
          LibDraws g{EcmcStream{id, (uint32_t)seed, (uint32_t)(seed >> 32), &st[id].draws}, p.epsilon_set,
                     (uint32_t)call, &st[id].set_counter, 0u, l};
          ecmc_chain(blk, p, g, st[id]);
        }
  return 0;
}

// generate_ecmc_cb on one rank with the reference's generator: create (cold or hot start
// with random_su3 per link), then n_shift x (random_shift + sample_persistant) with the
// plaquette after each shift; counters out[0..2] = events, lifts, same-site lifts so far.
void* orc_ecmc_ref_create(int L, int seed, int cold_start, const double dp[5], const int ip[2]) {
  RefEcmcRun* r = new RefEcmcRun();
  for (int d = 0; d < 4; ++d) r->dims[d] = L;
  const size_t V = (size_t)L * L * L * L;
  r->links.assign(V * 36, C(0.0, 0.0));
  r->rng.seed((uint64_t)(int64_t)seed + 0);  // rp.seed + topo.rank
  r->p = EcmcParams{dp[0], dp[1], dp[2], dp[3], dp[4], ip[0], L};
  (void)ip[1];
  memset(&r->st, 0, sizeof r->st);
  Lat f = r->lat();
  for (size_t s = 0; s < V; ++s)
    for (int mu = 0; mu < 4; ++mu) f.set(s, mu, ident());
  if (!cold_start)
    for (size_t s = 0; s < V; ++s)
      for (int mu = 0; mu < 4; ++mu) f.set(s, mu, random_su3_ref(r->rng));
  return r;
}

void orc_ecmc_ref_destroy(void* h) { delete static_cast<RefEcmcRun*>(h); }

int orc_ecmc_ref_run(void* h, int n_shift, double* plaq, uint64_t* counters) {
  RefEcmcRun* r = static_cast<RefEcmcRun*>(h);
  for (int i = 0; i < n_shift; ++i) {
    r->shift_and_sample();
    if (plaq) {
      Lat f = r->lat();
      plaq[i] = plaquette_sum(f) / (6.0 * (double)f.V);
    }
  }
  if (counters) {
    counters[0] = r->st.events;
    counters[1] = r->st.lifts;
    counters[2] = r->st.revs;
  }
  return 0;
}

int orc_ecmc_ref_get_links(void* h, double* aos) {
  RefEcmcRun* r = static_cast<RefEcmcRun*>(h);
  memcpy(aos, r->links.data(), r->links.size() * sizeof(C));
  return 0;
}
int orc_ecmc_ref_set_links(void* h, const double* aos) {
  RefEcmcRun* r = static_cast<RefEcmcRun*>(h);
  memcpy(r->links.data(), aos, r->links.size() * sizeof(C));
  return 0;
}

}  // extern "C"
