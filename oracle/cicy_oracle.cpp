// cicy_oracle.cpp -- FP64 CPU restatement of the reference's Tian-Yau and Schoen metric solves.
//
// TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline), linked into
// oracle/liboracle.so beside cy3_oracle.cpp and never into the product library.
//
// Reference files (crate substrate_sm_derivation/cy3_solver), cited below as
//   CS = src/cicy_sampler.rs, TY = src/route34/ty_metric.rs, GB = src/route34/groebner.rs,
//   HP = src/route34/donaldson_h_pair_sum.rs, SM = src/route34/schoen_metric.rs,
//   QT = src/quotient.rs, SS = src/route34/schoen_sampler.rs, ZP = src/route34/z3xz3_projector.rs.
//
// Third-party dependencies of the path that are absent from the reference tree, with the
// versions pinned by its Cargo.lock, restated here from their published algorithms:
//   * rand_core 0.9.5  SeedableRng::seed_from_u64: the 32-byte seed is filled with eight
//     PCG-XSH-RR 32-bit outputs of an LCG state started at the u64 seed (O'Neill 2014);
//   * rand_chacha 0.9.0 ChaCha8Rng: the ChaCha stream cipher with 8 rounds (Bernstein 2008),
//     64-bit block counter and 64-bit stream id (0), keystream read as little-endian u32
//     words, a u64 being (word[2i+1] << 32) | word[2i];
//   * rand 0.9.4  StandardUniform f64 = (u64 >> 11) * 2^-53; Open01 = the float with 52
//     fraction bits (u64 >> 12) and exponent 0, minus (1 - eps/2);
//   * rand_distr 0.5.1 StandardNormal: the ZIGNOR ziggurat (Marsaglia & Tsang 2000, Doornik
//     2005) with 256 strips, r = 3.6541528853610088, v = 0.00492867323399, the strip table
//     x_0 = v/f(r), x_1 = r, x_i = f^-1(v/x_{i-1} + f(x_{i-1})), x_256 = 0, f(x) = exp(-x^2/2),
//     the tables stored to 18 decimals; one u64 per try: 8 low bits pick the strip, the top
//     52 bits a uniform in [-1, 1); tail by Marsaglia's exponential method;
//   * num-complex 0.4.6  Complex64: (a+bi)(c+di) = (ac-bd) + (ad+bc)i, division by
//     c^2+d^2 without scaling, norm = hypot;
//   * pwos-math linalg::invert: LU with partial pivoting and per-column solves (the same
//     restatement as orc_invert_real in cy3_oracle.cpp).
// Arithmetic is operation for operation (build with -ffp-contract=off, no fast-math); the
// determinism records of the reference (tests/data/p5_10_determinism_golden.json) pin it.

#include <algorithm>
#include <array>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

namespace {

// Per-item work spread over threads (rayon stand-in); every result is per item, so the
// values do not depend on the thread count.
template <class F>
void par_for(size_t n, F&& f) {
  unsigned t = std::thread::hardware_concurrency();
  if (const char* e = std::getenv("CY3_ORACLE_THREADS")) t = (unsigned)std::max(1, std::atoi(e));
  if (t <= 1 || n < 64) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> th;
  for (unsigned q = 0; q < t; ++q)
    th.emplace_back([&] {
      for (;;) {
        size_t i0 = next.fetch_add(16);
        if (i0 >= n) break;
        for (size_t i = i0; i < std::min(n, i0 + 16); ++i) f(i);
      }
    });
  for (auto& x : th) x.join();
}

// ---------------------------------------------------------------------------------------
// num-complex arithmetic
// ---------------------------------------------------------------------------------------
struct Cx {
  double re, im;
};
inline Cx cx(double r, double i = 0.0) { return Cx{r, i}; }
inline Cx operator+(Cx a, Cx b) { return Cx{a.re + b.re, a.im + b.im}; }
inline Cx operator-(Cx a, Cx b) { return Cx{a.re - b.re, a.im - b.im}; }
inline Cx operator-(Cx a) { return Cx{-a.re, -a.im}; }
inline Cx operator*(Cx a, Cx b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cx operator/(Cx a, Cx b) {
  double n = b.re * b.re + b.im * b.im;
  return Cx{(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}
inline Cx divr(Cx a, double r) { return Cx{a.re / r, a.im / r}; }
inline Cx conj(Cx a) { return Cx{a.re, -a.im}; }
inline double norm(Cx a) { return std::hypot(a.re, a.im); }
inline double norm_sqr(Cx a) { return a.re * a.re + a.im * a.im; }
inline void operator+=(Cx& a, Cx b) { a = a + b; }
inline void operator-=(Cx& a, Cx b) { a = a - b; }
inline void operator*=(Cx& a, Cx b) { a = a * b; }

constexpr int NC = 8;   // ambient coordinates (CS:154)
constexpr int NH = 3;   // defining polynomials (CS:151)
constexpr int NF = 3;   // complex dimension (CS:162)

// ---------------------------------------------------------------------------------------
// ChaCha8Rng::seed_from_u64 and the three distributions
// ---------------------------------------------------------------------------------------
inline uint32_t rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

void chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]) {
  uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                    key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                    (uint32_t)counter, (uint32_t)(counter >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
  uint32_t x[16];
  std::memcpy(x, s, sizeof x);
#define QR(a, b, c, d)           \
  x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 16); \
  x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 12); \
  x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 8);  \
  x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 7);
  for (int r = 0; r < rounds; r += 2) {
    QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
    QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
  }
#undef QR
  for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

void pcg_seed_key(uint64_t state, uint32_t key[8]) {
  const uint64_t MUL = 6364136223846793005ull, INC = 11634580456017665027ull;
  for (int i = 0; i < 8; ++i) {
    state = state * MUL + INC;
    uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
    uint32_t rot = (uint32_t)(state >> 59);
    key[i] = (xs >> rot) | (xs << ((32 - rot) & 31));
  }
}

struct Rng {
  uint32_t key[8];
  uint64_t block = 0;
  uint32_t buf[64];
  int idx = 64;
  explicit Rng(uint64_t seed) { pcg_seed_key(seed, key); }
  uint64_t next_u64() {
    if (idx >= 64) {
      for (int b = 0; b < 4; ++b) chacha_block(key, block + b, 0, 8, buf + 16 * b);
      block += 4;
      idx = 0;
    }
    uint64_t lo = buf[idx], hi = buf[idx + 1];
    idx += 2;
    return (hi << 32) | lo;
  }
};

inline double from_bits(uint64_t b) {
  double d;
  std::memcpy(&d, &b, 8);
  return d;
}
inline double uniform53(Rng& r) { return (double)(r.next_u64() >> 11) * (1.0 / 9007199254740992.0); }
inline double open01(Rng& r) {
  return from_bits((r.next_u64() >> 12) | (1023ull << 52)) - (1.0 - 2.220446049250313e-16 / 2.0);
}

struct Zig {
  double x[257], f[257], r;
  Zig() {
    const double R = 3.6541528853610088, V = 0.00492867323399;
    auto fn = [](double t) { return std::exp(-t * t / 2.0); };
    auto finv = [](double y) { return std::sqrt(-2.0 * std::log(y)); };
    double xv[257], fv[257];
    xv[0] = V / fn(R);
    xv[1] = R;
    for (int i = 2; i < 256; ++i) xv[i] = finv(V / xv[i - 1] + fn(xv[i - 1]));
    xv[256] = 0.0;
    for (int i = 0; i <= 256; ++i) fv[i] = fn(xv[i]);
    char b[64];
    for (int i = 0; i <= 256; ++i) {
      std::snprintf(b, sizeof b, "%.18f", xv[i]);
      x[i] = std::strtod(b, nullptr);
      std::snprintf(b, sizeof b, "%.18f", fv[i]);
      f[i] = std::strtod(b, nullptr);
    }
    std::snprintf(b, sizeof b, "%.18f", R);
    r = std::strtod(b, nullptr);
  }
};
const Zig& zig() {
  static Zig z;
  return z;
}

double normal(Rng& rng) {
  const Zig& Z = zig();
  for (;;) {
    uint64_t bits = rng.next_u64();
    int i = (int)(bits & 0xff);
    double u = from_bits((bits >> 12) | (1024ull << 52)) - 3.0;
    double x = u * Z.x[i];
    if (std::fabs(x) < Z.x[i + 1]) return x;
    if (i == 0) {
      double xt = 1.0, yt = 0.0;
      while (-2.0 * yt < xt * xt) {
        double x_ = open01(rng);
        double y_ = open01(rng);
        xt = std::log(x_) / Z.r;
        yt = std::log(y_);
      }
      return u < 0.0 ? xt - Z.r : Z.r - xt;
    }
    if (Z.f[i + 1] + (Z.f[i] - Z.f[i + 1]) * uniform53(rng) < std::exp(-x * x / 2.0)) return x;
  }
}

// gaussian_unit_sphere_c8 (CS:883-899)
void unit_sphere(Rng& rng, Cx v[NC]) {
  double sq = 0.0;
  for (int k = 0; k < NC; ++k) {
    double re = normal(rng);
    double im = normal(rng);
    v[k] = cx(re, im);
    sq += re * re + im * im;
  }
  double n = std::sqrt(sq);
  if (n > 0.0)
    for (int k = 0; k < NC; ++k) v[k] = divr(v[k], n);
}

// ---------------------------------------------------------------------------------------
// The Tian-Yau triple (CS:236-283): f1 = sum z_i^3, f2 = sum w_i^3, f3 = sum z_i w_i.
// Polynomials are sparse (coefficient 1, exponent vector) lists as in the reference.
// ---------------------------------------------------------------------------------------
struct Term {
  Cx c;
  int e[NC];
};
struct Triple {
  std::vector<Term> f[NH];
  Triple() {
    for (int i = 0; i < 4; ++i) {
      Term t{cx(1.0), {0}};
      std::memset(t.e, 0, sizeof t.e);
      t.e[i] = 3;
      f[0].push_back(t);
      std::memset(t.e, 0, sizeof t.e);
      t.e[4 + i] = 3;
      f[1].push_back(t);
      std::memset(t.e, 0, sizeof t.e);
      t.e[i] = 1;
      t.e[4 + i] = 1;
      f[2].push_back(t);
    }
  }
};
const Triple& triple() {
  static Triple t;
  return t;
}

// eval_monomial (CS:298-314)
Cx eval_monomial(const Cx x[NC], const int e[NC]) {
  Cx acc = cx(1.0);
  for (int k = 0; k < NC; ++k) {
    if (e[k] == 0) continue;
    Cx p = x[k];
    for (int q = 1; q < e[k]; ++q) p *= x[k];
    acc *= p;
  }
  return acc;
}
Cx eval_poly(const std::vector<Term>& f, const Cx x[NC]) {
  Cx s = cx(0.0);
  for (const Term& t : f) s += t.c * eval_monomial(x, t.e);
  return s;
}
// poly_partial (CS:326-344)
Cx poly_partial(const std::vector<Term>& f, const Cx x[NC], int k) {
  Cx s = cx(0.0);
  for (const Term& t : f) {
    if (t.e[k] == 0) continue;
    int e[NC];
    std::memcpy(e, t.e, sizeof e);
    e[k] -= 1;
    Cx m = eval_monomial(x, e);
    s += t.c * cx((double)t.e[k]) * m;
  }
  return s;
}
void eval3(const Cx x[NC], Cx f[NH]) {
  for (int i = 0; i < NH; ++i) f[i] = eval_poly(triple().f[i], x);
}
// jacobian (CS:274-282): row-major NH x NC
void jacobian(const Cx x[NC], Cx j[NH * NC]) {
  for (int k = 0; k < NC; ++k)
    for (int i = 0; i < NH; ++i) j[i * NC + k] = poly_partial(triple().f[i], x, k);
}

// det_complex_lu (CS:959-996)
Cx det_lu(const Cx* m, int n) {
  Cx a[16];
  for (int i = 0; i < n * n; ++i) a[i] = m[i];
  Cx det = cx(1.0);
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = norm(a[k * n + k]);
    for (int p = k + 1; p < n; ++p) {
      double v = norm(a[p * n + k]);
      if (v > best) {
        best = v;
        piv = p;
      }
    }
    if (best == 0.0) return cx(0.0);
    if (piv != k) {
      for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[piv * n + j]);
      det = -det;
    }
    Cx pv = a[k * n + k];
    det *= pv;
    Cx ip = cx(1.0) / pv;
    for (int i = k + 1; i < n; ++i) {
      Cx fct = a[i * n + k] * ip;
      for (int j = k + 1; j < n; ++j) {
        Cx lhs = a[i * n + j];
        Cx rhs = fct * a[k * n + j];
        a[i * n + j] = lhs - rhs;
      }
      a[i * n + k] = cx(0.0);
    }
  }
  return det;
}

// inv_n (CS:1000-1058) and invert_n_complex (TY:2030-2082), the same Gauss-Jordan steps
bool inv_gj(const Cx* m, int n, Cx* out) {
  const int cols = 2 * n;
  Cx a[3 * 6];
  for (int i = 0; i < n * cols; ++i) a[i] = cx(0.0);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) a[i * cols + j] = m[i * n + j];
    a[i * cols + n + i] = cx(1.0);
  }
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = norm(a[k * cols + k]);
    for (int p = k + 1; p < n; ++p) {
      double v = norm(a[p * cols + k]);
      if (v > best) {
        best = v;
        piv = p;
      }
    }
    if (best < 1.0e-30) return false;
    if (piv != k)
      for (int j = 0; j < cols; ++j) std::swap(a[k * cols + j], a[piv * cols + j]);
    Cx ip = cx(1.0) / a[k * cols + k];
    for (int j = 0; j < cols; ++j) a[k * cols + j] *= ip;
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      Cx fct = a[i * cols + k];
      if (norm(fct) == 0.0) continue;
      for (int j = 0; j < cols; ++j) {
        Cx v = a[k * cols + j] * fct;
        a[i * cols + j] -= v;
      }
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) out[i * n + j] = a[i * cols + n + j];
  return true;
}

// residual_norm, line_eval (CS:852-878)
double residual_norm(const Cx f[NH]) {
  double s = 0.0;
  for (int i = 0; i < NH; ++i) s += norm_sqr(f[i]);
  return std::sqrt(s);
}
void line_eval(const Cx p[NC], const Cx d[NH][NC], const Cx t[NH], Cx x[NC]) {
  for (int k = 0; k < NC; ++k) x[k] = p[k];
  for (int j = 0; j < NH; ++j)
    for (int k = 0; k < NC; ++k) x[k] += t[j] * d[j][k];
}

// newton_solve_line (CS:771-850): Newton on t in C^3 with Armijo back-tracking.
bool newton_line(const Cx p[NC], const Cx d[NH][NC], Cx t[NH], Cx x[NC], double* res_out) {
  const int max_iter = 64;
  const double tol = 1.0e-8;
  line_eval(p, d, t, x);
  Cx f[NH];
  eval3(x, f);
  double res = residual_norm(f);
  for (int it = 0; it < max_iter; ++it) {
    if (res < tol) {
      *res_out = res;
      return true;
    }
    Cx jx[NH * NC];
    jacobian(x, jx);
    Cx m[NH * NH];
    for (int i = 0; i < NH; ++i)
      for (int j = 0; j < NH; ++j) {
        Cx s = cx(0.0);
        for (int k = 0; k < NC; ++k) s += jx[i * NC + k] * d[j][k];
        m[i * NH + j] = s;
      }
    if (norm(det_lu(m, NH)) < 1.0e-30) {
      *res_out = res;
      return false;
    }
    Cx mi[NH * NH];
    if (!inv_gj(m, NH, mi)) {
      *res_out = res;
      return false;
    }
    Cx dt[NH];
    for (int r = 0; r < NH; ++r) {
      Cx s = cx(0.0);
      for (int c = 0; c < NH; ++c) s += mi[r * NH + c] * f[c];
      dt[r] = -s;
    }
    double step = 1.0;
    bool accepted = false;
    for (int q = 0; q < 32; ++q) {
      Cx tt[NH];
      for (int r = 0; r < NH; ++r) tt[r] = t[r] + cx(step) * dt[r];
      Cx xt[NC], ft[NH];
      line_eval(p, d, tt, xt);
      eval3(xt, ft);
      double rt = residual_norm(ft);
      if (rt < (1.0 - 1.0e-4 * step) * res) {
        for (int r = 0; r < NH; ++r) t[r] = tt[r];
        for (int k = 0; k < NC; ++k) x[k] = xt[k];
        for (int i = 0; i < NH; ++i) f[i] = ft[i];
        res = rt;
        accepted = true;
        break;
      }
      step *= 0.5;
    }
    if (!accepted) {
      *res_out = res;
      return false;
    }
  }
  *res_out = res;
  return res < tol;
}

int argmax4(const Cx* v) {
  int best = 0;
  double ba = -1.0;
  for (int i = 0; i < 4; ++i) {
    double a = norm(v[i]);
    if (a > ba) {
      ba = a;
      best = i;
    }
  }
  return ba > 0.0 ? best : -1;
}

// pick_elimination_columns (CS:920-956) and the same greedy pick of TY:1944-1966
bool pick_elim(const Cx jac[NH * NC], int zi, int wi, int elim[NH]) {
  bool taken[NC] = {false};
  taken[zi] = true;
  taken[4 + wi] = true;
  for (int i = 0; i < NH; ++i) {
    int bk = -1;
    double ba = -1.0;
    for (int k = 0; k < NC; ++k) {
      if (taken[k]) continue;
      double a = norm(jac[i * NC + k]);
      if (a > ba) {
        ba = a;
        bk = k;
      }
    }
    if (bk < 0 || ba <= 0.0) return false;
    elim[i] = bk;
    taken[bk] = true;
  }
  return true;
}

struct TyPt {
  Cx x[NC];      // z then w, each factor divided by its largest coordinate
  Cx omega;      // 1 / det J_elim
  double weight; // |omega|^2 / det g_pb, later normalised
  int zi, wi;
};

// post_process_solved_point (CS:452-590)
bool post_process(const Cx xin[NC], TyPt* out) {
  Cx z[4] = {xin[0], xin[1], xin[2], xin[3]};
  Cx w[4] = {xin[4], xin[5], xin[6], xin[7]};
  int zi = argmax4(z), wi = argmax4(w);
  if (zi < 0 || wi < 0) return false;
  Cx zs = z[zi], ws = w[wi];
  const double EPS = 2.220446049250313e-16;
  if (norm(zs) < EPS || norm(ws) < EPS) return false;
  for (int i = 0; i < 4; ++i) z[i] = z[i] / zs;
  for (int i = 0; i < 4; ++i) w[i] = w[i] / ws;
  int near_one = 0;
  for (int i = 0; i < 4; ++i)
    if (norm(z[i] - cx(1.0)) < 1.0e-8) ++near_one;
  for (int i = 0; i < 4; ++i)
    if (norm(w[i] - cx(1.0)) < 1.0e-8) ++near_one;
  if (near_one > 2) return false;
  Cx xr[NC] = {z[0], z[1], z[2], z[3], w[0], w[1], w[2], w[3]};
  Cx jac[NH * NC];
  jacobian(xr, jac);
  int el[NH];
  if (!pick_elim(jac, zi, wi, el)) return false;
  Cx om[NH * NH];
  for (int i = 0; i < NH; ++i)
    for (int k = 0; k < NH; ++k) om[i * NH + k] = jac[i * NC + el[k]];
  Cx det_om = det_lu(om, NH);
  if (norm(det_om) < EPS) return false;
  Cx omega = cx(1.0) / det_om;
  bool elimd[NC] = {false};
  elimd[zi] = true;
  elimd[4 + wi] = true;
  for (int k = 0; k < NH; ++k) elimd[el[k]] = true;
  int fr[NC], nf = 0;
  for (int k = 0; k < NC; ++k)
    if (!elimd[k]) fr[nf++] = k;
  if (nf != NF) return false;
  Cx jpb[NF * NC];
  for (int i = 0; i < NF * NC; ++i) jpb[i] = cx(0.0);
  for (int a = 0; a < NF; ++a) jpb[a * NC + fr[a]] = cx(1.0);
  Cx oi[NH * NH];
  if (!inv_gj(om, NH, oi)) return false;
  for (int a = 0; a < NF; ++a) {
    Cx b[NH];
    for (int i = 0; i < NH; ++i) b[i] = jac[i * NC + fr[a]];
    for (int r = 0; r < NH; ++r) {
      Cx e = cx(0.0);
      for (int c = 0; c < NH; ++c) e += oi[r * NH + c] * b[c];
      jpb[a * NC + el[r]] = -e;
    }
  }
  // fs_metric_block (CS:1064-1126)
  Cx g[NC * NC];
  for (int i = 0; i < NC * NC; ++i) g[i] = cx(0.0);
  for (int f = 0; f < 2; ++f) {
    const Cx* v = f == 0 ? z : w;
    int pi = f == 0 ? zi : wi;
    double nv = 0.0;
    for (int k = 0; k < 4; ++k)
      if (k != pi) nv += norm_sqr(v[k]);
    double den = (1.0 + nv) * (1.0 + nv);
    for (int a = 0; a < 4; ++a) {
      if (a == pi) continue;
      for (int b = 0; b < 4; ++b) {
        if (b == pi) continue;
        double kron = a == b ? 1.0 : 0.0;
        Cx num = cx(1.0 + nv) * cx(kron) - v[a] * conj(v[b]);
        g[(4 * f + a) * NC + 4 * f + b] = num / cx(den);
      }
    }
  }
  // pullback_metric (CS:1129-1152)
  Cx tmp[NF * NC], gpb[NF * NF];
  for (int a = 0; a < NF; ++a)
    for (int b = 0; b < NC; ++b) {
      Cx s = cx(0.0);
      for (int k = 0; k < NC; ++k) s += jpb[a * NC + k] * g[k * NC + b];
      tmp[a * NC + b] = s;
    }
  for (int a = 0; a < NF; ++a)
    for (int b = 0; b < NF; ++b) {
      Cx s = cx(0.0);
      for (int k = 0; k < NC; ++k) s += tmp[a * NC + k] * conj(jpb[b * NC + k]);
      gpb[a * NF + b] = s;
    }
  double det_g = det_lu(gpb, NF).re;
  if (!std::isfinite(det_g) || std::fabs(det_g) < 1.0e-300) return false;
  double weight = norm_sqr(omega) / det_g;
  if (!std::isfinite(weight) || weight <= 0.0) return false;
  for (int k = 0; k < NC; ++k) out->x[k] = xr[k];
  out->omega = omega;
  out->weight = weight;
  out->zi = zi;
  out->wi = wi;
  return true;
}

// sample_one (CS:409-447)
bool sample_one(Rng& rng, TyPt* out) {
  Cx p[NC], d[NH][NC];
  unit_sphere(rng, p);
  for (int j = 0; j < NH; ++j) unit_sphere(rng, d[j]);
  bool have = false;
  Cx best[NC];
  double best_res = INFINITY;
  for (int att = 0; att < 4; ++att) {
    Cx t[NH];
    for (int j = 0; j < NH; ++j) {
      double re = normal(rng);
      double im = normal(rng);
      t[j] = cx(re, im);
    }
    Cx x[NC];
    double res;
    bool conv = newton_line(p, d, t, x, &res);
    if (conv && res < best_res) {
      best_res = res;
      for (int k = 0; k < NC; ++k) best[k] = x[k];
      have = true;
      if (res < 1.0e-8) break;
    }
  }
  if (!have || best_res >= 1.0e-8) return false;
  return post_process(best, out);
}

// ---------------------------------------------------------------------------------------
// Groebner basis (GB:470-656): Buchberger over f64 coefficients in the deg-lex order with
// z0 > ... > z3 > w0 > ... > w3, pairs processed in rounds against a snapshot of the basis,
// product criterion, terms below 1e-12 dropped.  Only the leading monomials are used: the
// standard monomials of R/I are the monomials that no leading monomial divides.
// ---------------------------------------------------------------------------------------
using Mono = std::array<int, NC>;
struct GPoly {
  std::vector<std::pair<double, Mono>> t;  // sorted, leading term first
};
int deglex_cmp(const Mono& a, const Mono& b) {
  int da = 0, db = 0;
  for (int k = 0; k < NC; ++k) {
    da += a[k];
    db += b[k];
  }
  if (da != db) return da < db ? -1 : 1;
  for (int k = 0; k < NC; ++k)
    if (a[k] != b[k]) return a[k] < b[k] ? -1 : 1;
  return 0;
}
GPoly make_poly(std::vector<std::pair<double, Mono>> terms) {
  // from_terms: sort by plain lex, collapse equal exponents, drop |c| <= 1e-12, sort by order
  std::sort(terms.begin(), terms.end(), [](const auto& a, const auto& b) { return a.second < b.second; });
  std::vector<std::pair<double, Mono>> col;
  for (auto& tm : terms) {
    if (!col.empty() && col.back().second == tm.second)
      col.back().first += tm.first;
    else
      col.push_back(tm);
  }
  GPoly p;
  for (auto& tm : col)
    if (std::fabs(tm.first) > 1.0e-12) p.t.push_back(tm);
  std::stable_sort(p.t.begin(), p.t.end(),
                   [](const auto& a, const auto& b) { return deglex_cmp(a.second, b.second) > 0; });
  return p;
}
GPoly poly_sub_scaled(const GPoly& a, const GPoly& b, double c, const Mono& e) {
  std::vector<std::pair<double, Mono>> terms(a.t);
  for (auto& tm : b.t) {
    Mono m;
    for (int k = 0; k < NC; ++k) m[k] = tm.second[k] + e[k];
    terms.push_back({-(tm.first * c), m});
  }
  return make_poly(terms);
}
bool divides(const Mono& d, const Mono& m) {
  for (int k = 0; k < NC; ++k)
    if (d[k] > m[k]) return false;
  return true;
}
GPoly s_poly(const GPoly& f, const GPoly& g) {
  Mono l, af, ag;
  for (int k = 0; k < NC; ++k) {
    l[k] = std::max(f.t[0].second[k], g.t[0].second[k]);
    af[k] = l[k] - f.t[0].second[k];
    ag[k] = l[k] - g.t[0].second[k];
  }
  std::vector<std::pair<double, Mono>> terms;
  double cf = 1.0 / f.t[0].first, cg = 1.0 / g.t[0].first;
  for (auto& tm : f.t) {
    Mono m;
    for (int k = 0; k < NC; ++k) m[k] = tm.second[k] + af[k];
    terms.push_back({tm.first * cf, m});
  }
  for (auto& tm : g.t) {
    Mono m;
    for (int k = 0; k < NC; ++k) m[k] = tm.second[k] + ag[k];
    terms.push_back({-(tm.first * cg), m});
  }
  return make_poly(terms);
}
GPoly remainder(GPoly p, const std::vector<GPoly>& basis) {
  std::vector<std::pair<double, Mono>> rem;
  while (!p.t.empty()) {
    const Mono lm = p.t[0].second;
    double lc = p.t[0].first;
    bool done = false;
    for (const GPoly& g : basis) {
      if (g.t.empty() || !divides(g.t[0].second, lm)) continue;
      Mono al;
      for (int k = 0; k < NC; ++k) al[k] = lm[k] - g.t[0].second[k];
      p = poly_sub_scaled(p, g, lc / g.t[0].first, al);
      done = true;
      break;
    }
    if (!done) {
      rem.push_back(p.t[0]);
      p.t.erase(p.t.begin());
    }
  }
  return make_poly(rem);
}

std::vector<Mono> groebner_lms(const std::vector<std::vector<std::pair<double, Mono>>>& gens) {
  std::vector<GPoly> g;
  for (const auto& terms : gens) g.push_back(make_poly(terms));
  std::vector<std::pair<int, int>> pairs;
  for (int i = 0; i < (int)g.size(); ++i)
    for (int j = i + 1; j < (int)g.size(); ++j) pairs.push_back({i, j});
  while (!pairs.empty()) {
    std::vector<std::pair<int, int>> active;
    for (auto& pr : pairs) {
      const Mono &a = g[pr.first].t[0].second, &b = g[pr.second].t[0].second;
      bool disjoint = true;
      for (int k = 0; k < NC; ++k)
        if (a[k] > 0 && b[k] > 0) disjoint = false;
      if (!disjoint) active.push_back(pr);
    }
    pairs.clear();
    if (active.empty()) break;
    std::vector<GPoly> snap = g;
    for (auto& pr : active) {
      GPoly s = s_poly(snap[pr.first], snap[pr.second]);
      if (s.t.empty()) continue;
      GPoly r = remainder(s, snap);
      if (r.t.empty()) continue;
      int ni = (int)g.size();
      for (int k = 0; k < ni; ++k) pairs.push_back({k, ni});
      g.push_back(r);
    }
  }
  // minimal leading monomials (GB:556-600)
  std::vector<Mono> lms;
  for (size_t i = 0; i < g.size(); ++i) {
    const Mono& li = g[i].t[0].second;
    bool redundant = false;
    for (size_t j = 0; j < g.size() && !redundant; ++j) {
      if (i == j) continue;
      const Mono& lj = g[j].t[0].second;
      if (divides(lj, li) && (lj != li || j < i)) redundant = true;
    }
    if (!redundant) lms.push_back(li);
  }
  std::sort(lms.begin(), lms.end(), [](const Mono& a, const Mono& b) { return deglex_cmp(a, b) > 0; });
  return lms;
}
// ty_generators (GB:665-703): the Tian-Yau triple with unit coefficients
const std::vector<Mono>& ty_lms() {
  static std::vector<Mono> lms = [] {
    std::vector<std::vector<std::pair<double, Mono>>> gens;
    for (int i = 0; i < NH; ++i) {
      std::vector<std::pair<double, Mono>> terms;
      for (const Term& t : triple().f[i]) {
        Mono m;
        for (int k = 0; k < NC; ++k) m[k] = t.e[k];
        terms.push_back({1.0, m});
      }
      gens.push_back(terms);
    }
    return groebner_lms(gens);
  }();
  return lms;
}

// build_ty_invariant_reduced_basis (TY:870-888) over enumerate_bigraded_kk_monomials (TY:790-818)
std::vector<Mono> ty_basis(int k) {
  std::vector<std::array<int, 4>> zm;
  for (int a0 = 0; a0 <= k; ++a0)
    for (int a1 = 0; a1 <= k - a0; ++a1)
      for (int a2 = 0; a2 <= k - a0 - a1; ++a2) zm.push_back({a0, a1, a2, k - a0 - a1 - a2});
  std::vector<Mono> out;
  const auto& lms = ty_lms();
  for (auto& zz : zm)
    for (auto& ww : zm) {
      Mono m = {zz[0], zz[1], zz[2], zz[3], ww[0], ww[1], ww[2], ww[3]};
      if ((m[1] + 2 * m[2] + m[5] + 2 * m[6]) % 3 != 0) continue;  // z3_character (QT:55-57)
      bool in_ideal = false;
      for (auto& l : lms)
        if (divides(l, m)) {
          in_ideal = true;
          break;
        }
      if (!in_ideal) out.push_back(m);
    }
  return out;
}

// ---------------------------------------------------------------------------------------
// Sections, Donaldson iteration and sigma (TY:890-1400, 1402-1470, 1788-2030)
// ---------------------------------------------------------------------------------------
void sections_at(const Cx x[NC], const std::vector<Mono>& basis, int kmax, double* vals, double* ders) {
  const int st = kmax + 1;
  std::vector<Cx> pw((size_t)NC * st);
  for (int k = 0; k < NC; ++k) {
    pw[k * st] = cx(1.0);
    for (int e = 1; e < st; ++e) pw[k * st + e] = pw[k * st + e - 1] * x[k];
  }
  const int N = (int)basis.size();
  for (int a = 0; a < N; ++a) {
    Cx acc = cx(1.0);
    for (int k = 0; k < NC; ++k) acc *= pw[k * st + basis[a][k]];
    vals[2 * a] = acc.re;
    vals[2 * a + 1] = acc.im;
  }
  if (!ders) return;
  for (int k = 0; k < NC; ++k)
    for (int a = 0; a < N; ++a) {
      const Mono& m = basis[a];
      Cx acc = cx(0.0);
      if (m[k] != 0) {
        acc = cx((double)m[k]);
        acc *= pw[k * st + m[k] - 1];
        for (int j = 0; j < NC; ++j)
          if (j != k) acc *= pw[j * st + m[j]];
      }
      ders[(size_t)k * 2 * N + 2 * a] = acc.re;
      ders[(size_t)k * 2 * N + 2 * a + 1] = acc.im;
    }
}

// hermitian_quadratic_form (TY:1870-1900): (u^dagger H v)
inline void hqf(const double* hr, const double* hi, int N, const double* u, const double* v, double* ore,
                double* oim) {
  double sr = 0.0, si = 0.0;
  for (int a = 0; a < N; ++a) {
    double vr_ = 0.0, vi_ = 0.0;
    for (int b = 0; b < N; ++b) {
      double h_r = hr[a * N + b], h_i = hi[a * N + b];
      double vr = v[2 * b], vi = v[2 * b + 1];
      vr_ += h_r * vr - h_i * vi;
      vi_ += h_r * vi + h_i * vr;
    }
    double ur = u[2 * a], ui = u[2 * a + 1];
    sr += ur * vr_ + ui * vi_;
    si += ur * vi_ - ui * vr_;
  }
  *ore = sr;
  *oim = si;
}

// ty_affine_chart_frame (TY:1929-2017)
bool chart_frame(const TyPt& pt, Cx frame[NF][NC]) {
  Cx jac[NH * NC];
  jacobian(pt.x, jac);
  int el[NH];
  if (!pick_elim(jac, pt.zi, pt.wi, el)) return false;
  bool taken[NC] = {false};
  taken[pt.zi] = true;
  taken[4 + pt.wi] = true;
  for (int i = 0; i < NH; ++i) taken[el[i]] = true;
  int fr[NF], nf = 0;
  for (int k = 0; k < NC; ++k)
    if (!taken[k]) {
      if (nf >= NF) return false;
      fr[nf++] = k;
    }
  if (nf != NF) return false;
  Cx je[NH * NH], ji[NH * NH];
  for (int i = 0; i < NH; ++i)
    for (int c = 0; c < NH; ++c) je[i * NH + c] = jac[i * NC + el[c]];
  if (!inv_gj(je, NH, ji)) return false;
  for (int a = 0; a < NF; ++a)
    for (int k = 0; k < NC; ++k) frame[a][k] = cx(0.0);
  for (int a = 0; a < NF; ++a) {
    frame[a][fr[a]] = cx(1.0);
    Cx b[NH];
    for (int i = 0; i < NH; ++i) b[i] = jac[i * NC + fr[a]];
    for (int c = 0; c < NH; ++c) {
      Cx e = cx(0.0);
      for (int i = 0; i < NH; ++i) e += ji[c * NH + i] * b[i];
      frame[a][el[c]] = -e;
    }
  }
  return true;
}

double eta_from_frame(bool frame_ok, const Cx fr[NF][NC], const double* s, const double* d, const double* hr,
                      const double* hi, int N, double omega_sq);

// compute_eta_at_point (TY:1788-1866)
double eta_at(const TyPt& pt, const double* s, const double* d, const double* hr, const double* hi, int N,
              double omega_sq) {
  Cx fr[NF][NC];
  const bool ok = chart_frame(pt, fr);
  return eta_from_frame(ok, fr, s, d, hr, hi, N, omega_sq);
}

// the per-point part of compute_eta_at_point (TY:1788-1866, SM:2092-2160) given the chart frame
double eta_from_frame(bool frame_ok, const Cx fr[NF][NC], const double* s, const double* d, const double* hr,
                      const double* hi, int N, double omega_sq) {
  if (!std::isfinite(omega_sq) || omega_sq <= 0.0) return NAN;
  const size_t tn = 2 * (size_t)N;
  double kv, dum;
  hqf(hr, hi, N, s, s, &kv, &dum);
  double ks = std::fmax(kv, 1.0e-30);
  Cx dk[NC];
  for (int i = 0; i < NC; ++i) {
    double re, im;
    hqf(hr, hi, N, s, d + i * tn, &re, &im);
    dk[i] = cx(re, im);
  }
  Cx ga[NC][NC];
  for (int i = 0; i < NC; ++i)
    for (int j = 0; j < NC; ++j) {
      double re, im;
      hqf(hr, hi, N, d + j * tn, d + i * tn, &re, &im);
      Cx t1 = divr(cx(re, im), ks);
      Cx t2 = divr(dk[i] * conj(dk[j]), ks * ks);
      ga[i][j] = t1 - t2;
    }
  if (!frame_ok) return NAN;
  Cx gt[NF][NF];
  for (int a = 0; a < NF; ++a)
    for (int b = 0; b < NF; ++b) {
      Cx acc = cx(0.0);
      for (int i = 0; i < NC; ++i) {
        Cx tc = conj(fr[a][i]);
        Cx row = cx(0.0);
        for (int j = 0; j < NC; ++j) row += ga[i][j] * fr[b][j];
        acc += tc * row;
      }
      gt[a][b] = acc;
    }
  // det_3x3_complex (TY:1902-1908)
  Cx m1 = gt[1][1] * gt[2][2] - gt[1][2] * gt[2][1];
  Cx m2 = gt[1][0] * gt[2][2] - gt[1][2] * gt[2][0];
  Cx m3 = gt[1][0] * gt[2][1] - gt[1][1] * gt[2][0];
  double det = (gt[0][0] * m1 - gt[0][1] * m2 + gt[0][2] * m3).re;
  if (!std::isfinite(det) || std::fabs(det) < 1.0e-30) return NAN;
  return std::fabs(det) / omega_sq;
}

// compute_sigma reduction (TY:1438-1468)
double sigma_reduce(const double* eta, const double* w, size_t P) {
  double tw = 0.0, we = 0.0;
  size_t cnt = 0;
  for (size_t p = 0; p < P; ++p) {
    if (!std::isfinite(eta[p]) || eta[p] <= 0.0 || !std::isfinite(w[p]) || w[p] <= 0.0) continue;
    tw += w[p];
    we += w[p] * eta[p];
    ++cnt;
  }
  if (cnt == 0 || tw < 1.0e-30) return NAN;
  double kappa = we / tw;
  if (std::fabs(kappa) < 1.0e-30) return NAN;
  double sq = 0.0;
  for (size_t p = 0; p < P; ++p) {
    if (!std::isfinite(eta[p]) || eta[p] <= 0.0 || !std::isfinite(w[p]) || w[p] <= 0.0) continue;
    double r = eta[p] / kappa - 1.0;
    sq += w[p] * r * r;
  }
  return sq / tw;
}

// LU with partial pivoting + per-column solves (pwos-math linalg::invert); also reports whether
// every pivot of U is finite and at least the smallest normal double (TY:1255-1296).
int lu_invert(const std::vector<double>& a_in, int n, std::vector<double>& inv, bool* tiny_pivot) {
  std::vector<double> a(a_in);
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = std::fabs(a[(size_t)k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      double v = std::fabs(a[(size_t)i * n + k]);
      if (v > best) {
        best = v;
        piv = i;
      }
    }
    if (!(best > 0.0) || !std::isfinite(best)) return -1;
    if (piv != k) {
      for (int j = 0; j < n; ++j) std::swap(a[(size_t)k * n + j], a[(size_t)piv * n + j]);
      std::swap(perm[k], perm[piv]);
    }
    double d = a[(size_t)k * n + k];
    for (int i = k + 1; i < n; ++i) {
      double f = a[(size_t)i * n + k] / d;
      a[(size_t)i * n + k] = f;
      if (f != 0.0)
        for (int j = k + 1; j < n; ++j) a[(size_t)i * n + j] -= f * a[(size_t)k * n + j];
    }
  }
  *tiny_pivot = false;
  for (int i = 0; i < n; ++i) {
    double pv = a[(size_t)i * n + i];
    if (!std::isfinite(pv) || std::fabs(pv) < 2.2250738585072014e-308) *tiny_pivot = true;
  }
  inv.assign((size_t)n * n, 0.0);
  std::vector<double> col(n);
  for (int c = 0; c < n; ++c) {
    for (int i = 0; i < n; ++i) col[i] = perm[i] == c ? 1.0 : 0.0;
    for (int i = 0; i < n; ++i) {
      double s = col[i];
      for (int j = 0; j < i; ++j) s -= a[(size_t)i * n + j] * col[j];
      col[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = col[i];
      for (int j = i + 1; j < n; ++j) s -= a[(size_t)i * n + j] * col[j];
      col[i] = s / a[(size_t)i * n + i];
    }
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + c] = col[i];
  }
  return 0;
}

// donaldson_iteration_impl, CPU branch (TY:1062-1370), with the 256-lane pairwise T sum of
// HP:97-160.  h_re/h_im are N x N row-major (upper-index metric); returns the residual.
double donaldson_iteration(const double* S, const double* w, size_t P, int N, double* h_re, double* h_im,
                           double alpha) {
  const size_t tn = 2 * (size_t)N;
  std::vector<double> kv(P);
  par_for(P, [&](size_t p) {
    const double* s = S + p * tn;
    double k = 0.0;
    for (int a = 0; a < N; ++a) {
      double sar = s[2 * a], sai = s[2 * a + 1];
      for (int b = 0; b < N; ++b) {
        double sbr = s[2 * b], sbi = s[2 * b + 1];
        double hr = h_re[a * N + b], hi = h_im[a * N + b];
        k += hr * (sar * sbr + sai * sbi) + hi * (sar * sbi - sai * sbr);
      }
    }
    kv[p] = std::fmax(k, 1.0e-30);
  });
  const size_t NN = (size_t)N * N;
  std::vector<double> pr(2 * NN);
  par_for((size_t)N, [&](size_t a_) {
    const int a = (int)a_;
    for (int b = 0; b < N; ++b) {
      double lre[256], lim[256];
      for (int t = 0; t < 256; ++t) {
        double ar = 0.0, ai = 0.0;
        for (size_t p = t; p < P; p += 256) {
          double wp = w[p], kp = kv[p];
          if (std::isfinite(wp) && wp > 0.0 && std::isfinite(kp) && kp > 0.0) {
            const double* s = S + p * tn;
            double sar = s[2 * a], sai = s[2 * a + 1], sbr = s[2 * b], sbi = s[2 * b + 1];
            double fct = wp / kp;
            ar += fct * (sar * sbr + sai * sbi);
            ai += fct * (sar * sbi - sai * sbr);
          }
        }
        lre[t] = ar;
        lim[t] = ai;
      }
      for (int st = 128; st > 0; st >>= 1)
        for (int t = 0; t < st; ++t) {
          lre[t] += lre[t + st];
          lim[t] += lim[t + st];
        }
      pr[2 * ((size_t)a * N + b)] = lre[0];
      pr[2 * ((size_t)a * N + b) + 1] = lim[0];
    }
  });
  double wsum = 0.0;
  for (size_t p = 0; p < P; ++p) wsum += w[p];
  if (!(wsum > 1.0e-30)) return NAN;
  double inv_w = 1.0 / wsum;
  std::vector<double> nr(NN), ni(NN);
  for (size_t i = 0; i < NN; ++i) {
    nr[i] = pr[2 * i] * inv_w;
    ni[i] = pr[2 * i + 1] * inv_w;
  }
  for (int a = 0; a < N; ++a)
    for (int b = a + 1; b < N; ++b) {
      double ar = 0.5 * (nr[a * N + b] + nr[b * N + a]);
      nr[a * N + b] = ar;
      nr[b * N + a] = ar;
      double ai = 0.5 * (ni[a * N + b] - ni[b * N + a]);
      ni[a * N + b] = ai;
      ni[b * N + a] = -ai;
    }
  for (int a = 0; a < N; ++a) ni[a * N + a] = 0.0;
  auto renorm = [&](std::vector<double>& r, std::vector<double>& i) {
    double tr = 0.0;
    for (int a = 0; a < N; ++a) tr += r[a * N + a];
    if (std::fabs(tr) > 1.0e-30) {
      double sc = (double)N / tr;
      for (auto& v : r) v *= sc;
      for (auto& v : i) v *= sc;
    }
  };
  renorm(nr, ni);
  const int tw = 2 * N;
  std::vector<double> blk((size_t)tw * tw), binv;
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b) {
      double hr = nr[a * N + b], hi = ni[a * N + b];
      blk[(size_t)(2 * a) * tw + 2 * b] = hr;
      blk[(size_t)(2 * a) * tw + 2 * b + 1] = -hi;
      blk[(size_t)(2 * a + 1) * tw + 2 * b] = hi;
      blk[(size_t)(2 * a + 1) * tw + 2 * b + 1] = hr;
    }
  bool tiny = false;
  if (lu_invert(blk, tw, binv, &tiny) != 0 || tiny) return NAN;  // h kept (TY:1309-1323)
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b) {
      double mrr = binv[(size_t)(2 * a) * tw + 2 * b], mri = binv[(size_t)(2 * a) * tw + 2 * b + 1];
      double mir = binv[(size_t)(2 * a + 1) * tw + 2 * b], mii = binv[(size_t)(2 * a + 1) * tw + 2 * b + 1];
      if (!std::isfinite(mrr) || !std::isfinite(mri) || !std::isfinite(mir) || !std::isfinite(mii)) return NAN;
      nr[a * N + b] = 0.5 * (mrr + mii);
      ni[a * N + b] = 0.5 * (mir - mri);
    }
  renorm(nr, ni);
  double al = std::min(std::max(alpha, 1.0e-6), 1.0);
  double dsq = 0.0;
  for (size_t i = 0; i < NN; ++i) {
    double dr = nr[i] - h_re[i], di = ni[i] - h_im[i];
    dsq += dr * dr + di * di;
    h_re[i] = al * nr[i] + (1.0 - al) * h_re[i];
    h_im[i] = al * ni[i] + (1.0 - al) * h_im[i];
  }
  return std::sqrt(dsq);
}

struct TyData {
  std::vector<TyPt> pts;
  std::vector<double> w, om2;
  std::vector<Mono> basis;
  int kmax = 0;
  std::vector<double> S, D;  // values [P][2N], derivatives [P][8][2N]
};

void build_sections(TyData& td, bool derivs) {
  const size_t P = td.pts.size();
  const int N = (int)td.basis.size();
  td.kmax = 0;
  for (auto& m : td.basis)
    for (int k = 0; k < NC; ++k) td.kmax = std::max(td.kmax, m[k]);
  td.S.assign(P * 2 * N, 0.0);
  if (derivs) td.D.assign(P * NC * 2 * N, 0.0);
  par_for(P, [&](size_t p) {
    sections_at(td.pts[p].x, td.basis, td.kmax, td.S.data() + p * 2 * N,
                derivs ? td.D.data() + p * NC * 2 * N : nullptr);
  });
}

double sigma_of(const TyData& td, const double* hr, const double* hi, double* eta_out) {
  const size_t P = td.pts.size();
  const int N = (int)td.basis.size();
  std::vector<double> eta(P);
  par_for(P, [&](size_t p) {
    eta[p] = eta_at(td.pts[p], td.S.data() + p * 2 * N, td.D.data() + p * NC * 2 * N, hr, hi, N, td.om2[p]);
  });
  if (eta_out) std::copy(eta.begin(), eta.end(), eta_out);
  return sigma_reduce(eta.data(), td.w.data(), P);
}

// sample_batch (CS:600-627) followed by apply_z3_quotient (CS:758-763); `gpu_stream` draws the
// per-line inputs the way sample_batch_gpu does (CS:640-740: max(4n, 64) lines of one Newton
// attempt each, the first n accepted in line order) with the Newton steps of newton_solve_line.
std::vector<TyPt> sample(uint64_t seed, size_t n, bool gpu_stream, bool z3) {
  Rng rng(seed);
  std::vector<TyPt> out;
  if (!gpu_stream) {
    size_t max_total = std::max(n * 64, (size_t)1024), att = 0;
    while (out.size() < n && att < max_total) {
      ++att;
      TyPt pt;
      if (sample_one(rng, &pt)) out.push_back(pt);
    }
  } else {
    size_t lines = std::max(n * 4, (size_t)64);
    for (size_t l = 0; l < lines; ++l) {
      Cx p[NC], d[NH][NC], t[NH];
      unit_sphere(rng, p);
      for (int j = 0; j < NH; ++j) unit_sphere(rng, d[j]);
      for (int j = 0; j < NH; ++j) {
        double re = normal(rng);
        double im = normal(rng);
        t[j] = cx(re, im);
      }
      if (out.size() >= n) continue;
      Cx x[NC];
      double res;
      if (!newton_line(p, d, t, x, &res)) continue;
      TyPt pt;
      if (post_process(x, &pt)) out.push_back(pt);
    }
  }
  double sum = 0.0;
  for (auto& p : out) sum += p.weight;
  if (std::isfinite(sum) && sum > 0.0)
    for (auto& p : out) p.weight /= sum;
  if (z3) {
    const double inv_k = 1.0 / 3.0;
    for (auto& p : out) p.weight *= inv_k;
  }
  return out;
}

void export_points(const std::vector<TyPt>& pts, double* coords, double* omega, double* weight, int* zw) {
  for (size_t p = 0; p < pts.size(); ++p) {
    for (int k = 0; k < NC; ++k) {
      coords[p * 16 + 2 * k] = pts[p].x[k].re;
      coords[p * 16 + 2 * k + 1] = pts[p].x[k].im;
    }
    if (omega) {
      omega[2 * p] = pts[p].omega.re;
      omega[2 * p + 1] = pts[p].omega.im;
    }
    if (weight) weight[p] = pts[p].weight;
    if (zw) {
      zw[2 * p] = pts[p].zi;
      zw[2 * p + 1] = pts[p].wi;
    }
  }
}

// TyPoint's patch indices (TY:483-484): argmax of |coord| over each factor of the rescaled point
void patch_indices(TyPt& pt) {
  int zi = 0, wi = 0;
  double bz = -1.0, bw = -1.0;
  for (int q = 0; q < 4; ++q) {
    double a = norm(pt.x[q]);
    if (a > bz) {
      bz = a;
      zi = q;
    }
    double b = norm(pt.x[4 + q]);
    if (b > bw) {
      bw = b;
      wi = q;
    }
  }
  pt.zi = zi;
  pt.wi = wi;
}

TyData import_points(const double* coords, const double* omega_sq, const double* weight, size_t P, int k) {
  TyData td;
  td.pts.resize(P);
  td.w.assign(weight, weight + P);
  td.om2.assign(omega_sq, omega_sq + P);
  for (size_t p = 0; p < P; ++p) {
    for (int q = 0; q < NC; ++q) td.pts[p].x[q] = cx(coords[p * 16 + 2 * q], coords[p * 16 + 2 * q + 1]);
    patch_indices(td.pts[p]);
    td.pts[p].weight = weight[p];
  }
  td.basis = ty_basis(k);
  return td;
}


// ---------------------------------------------------------------------------------------
// Schoen (SS, SM, ZP): the Z/3 x Z/3 quotient of the complete intersection in CP^2 x CP^2 x CP^1,
// coordinates x_0..x_2, y_0..y_2, t_0, t_1 (SS:99-133), sampler polynomials (SS:188-216)
//   F1 = (x0^3 + x1^3 + x2^3) t0 + x0 x1 x2 t1,  F2 = (y0^3 + y1^3 + y2^3) t1 + y0 y1 y2 t0
// ---------------------------------------------------------------------------------------
constexpr int SNH = 2;
const int S_LO[3] = {0, 3, 6}, S_HI[3] = {3, 6, 8};

struct SchoenPolys {
  std::vector<Term> f[SNH];
  SchoenPolys() {
    for (int q = 0; q < 2; ++q) {
      const int b = q == 0 ? 0 : 3, tc = q == 0 ? 6 : 7, to = q == 0 ? 7 : 6;
      for (int k = 0; k < 3; ++k) {
        Term t{cx(1.0), {0}};
        std::memset(t.e, 0, sizeof t.e);
        t.e[b + k] = 3;
        t.e[tc] = 1;
        f[q].push_back(t);
      }
      Term t{cx(1.0), {0}};
      std::memset(t.e, 0, sizeof t.e);
      t.e[b] = t.e[b + 1] = t.e[b + 2] = 1;
      t.e[to] = 1;
      f[q].push_back(t);
    }
  }
};
const SchoenPolys& spolys() {
  static SchoenPolys p;
  return p;
}
void s_eval(const Cx x[NC], Cx f[SNH]) {
  for (int i = 0; i < SNH; ++i) f[i] = eval_poly(spolys().f[i], x);
}
void s_jacobian(const Cx x[NC], Cx j[SNH * NC]) {
  for (int k = 0; k < NC; ++k)
    for (int i = 0; i < SNH; ++i) j[i * NC + k] = poly_partial(spolys().f[i], x, k);
}
double s_residual(const Cx f[SNH]) {
  double s = 0.0;
  for (int i = 0; i < SNH; ++i) s += norm_sqr(f[i]);
  return std::sqrt(s);
}
void s_line(const Cx p[NC], const Cx d[SNH][NC], const Cx t[SNH], Cx x[NC]) {
  for (int k = 0; k < NC; ++k) x[k] = p[k];
  for (int j = 0; j < SNH; ++j)
    for (int k = 0; k < NC; ++k) x[k] += t[j] * d[j][k];
}

// newton_solve_line (SS:642-700): as the Tian-Yau one without the determinant pre-check
bool s_newton(const Cx p[NC], const Cx d[SNH][NC], Cx t[SNH], Cx x[NC], double* res_out) {
  const double tol = 1.0e-8;
  s_line(p, d, t, x);
  Cx f[SNH];
  s_eval(x, f);
  double res = s_residual(f);
  for (int it = 0; it < 64; ++it) {
    if (res < tol) {
      *res_out = res;
      return true;
    }
    Cx jx[SNH * NC], m[SNH * SNH], mi[SNH * SNH];
    s_jacobian(x, jx);
    for (int i = 0; i < SNH; ++i)
      for (int j = 0; j < SNH; ++j) {
        Cx sm = cx(0.0);
        for (int k = 0; k < NC; ++k) sm += jx[i * NC + k] * d[j][k];
        m[i * SNH + j] = sm;
      }
    if (!inv_gj(m, SNH, mi)) {
      *res_out = res;
      return false;
    }
    Cx dt[SNH];
    for (int r = 0; r < SNH; ++r) {
      Cx sm = cx(0.0);
      for (int c = 0; c < SNH; ++c) sm += mi[r * SNH + c] * f[c];
      dt[r] = -sm;
    }
    double step = 1.0;
    bool accepted = false;
    for (int q = 0; q < 32; ++q) {
      Cx tt[SNH], xt[NC], ft[SNH];
      for (int r = 0; r < SNH; ++r) tt[r] = t[r] + cx(step) * dt[r];
      s_line(p, d, tt, xt);
      s_eval(xt, ft);
      const double rt = s_residual(ft);
      if (rt < (1.0 - 1.0e-4 * step) * res) {
        for (int r = 0; r < SNH; ++r) t[r] = tt[r];
        for (int k = 0; k < NC; ++k) x[k] = xt[k];
        for (int i = 0; i < SNH; ++i) f[i] = ft[i];
        res = rt;
        accepted = true;
        break;
      }
      step *= 0.5;
    }
    if (!accepted) {
      *res_out = res;
      return false;
    }
  }
  *res_out = res;
  return res < tol;
}

struct SPt {
  Cx x[NC];
  Cx omega;
  double weight;
  int patch[3];  // absolute coordinate index of each factor's largest coordinate
};

int argmax_range(const Cx* v, int lo, int hi) {
  int best = lo;
  double ba = -1.0;
  for (int k = lo; k < hi; ++k) {
    const double a = norm(v[k]);
    if (a > ba) {
      ba = a;
      best = k;
    }
  }
  return ba > 0.0 ? best : -1;
}

// pick_elimination_columns (SS:868-900)
bool s_pick_elim(const Cx jac[SNH * NC], const int patch[3], int el[SNH]) {
  bool taken[NC] = {false};
  for (int f = 0; f < 3; ++f) taken[patch[f]] = true;
  for (int i = 0; i < SNH; ++i) {
    int bk = -1;
    double ba = -1.0;
    for (int k = 0; k < NC; ++k) {
      if (taken[k]) continue;
      const double a = norm(jac[i * NC + k]);
      if (a > ba) {
        ba = a;
        bk = k;
      }
    }
    if (bk < 0 || ba <= 0.0) return false;
    el[i] = bk;
    taken[bk] = true;
  }
  return true;
}

// post_process_solved_point (SS:716-850)
bool s_post_process(const Cx xin[NC], SPt* out) {
  int patch[3];
  for (int f = 0; f < 3; ++f) {
    patch[f] = argmax_range(xin, S_LO[f], S_HI[f]);
    if (patch[f] < 0) return false;
  }
  const double EPS = 2.220446049250313e-16;
  for (int f = 0; f < 3; ++f)
    if (norm(xin[patch[f]]) < EPS) return false;
  Cx xr[NC];
  for (int f = 0; f < 3; ++f) {
    const Cx sc = xin[patch[f]];
    for (int k = S_LO[f]; k < S_HI[f]; ++k) xr[k] = xin[k] / sc;
  }
  int near_one = 0;
  for (int k = 0; k < NC; ++k)
    if (norm(xr[k] - cx(1.0)) < 1.0e-8) ++near_one;
  if (near_one > 3) return false;
  Cx jac[SNH * NC];
  s_jacobian(xr, jac);
  int el[SNH];
  if (!s_pick_elim(jac, patch, el)) return false;
  Cx om[SNH * SNH];
  for (int i = 0; i < SNH; ++i)
    for (int k = 0; k < SNH; ++k) om[i * SNH + k] = jac[i * NC + el[k]];
  const Cx det_om = det_lu(om, SNH);
  if (norm(det_om) < EPS) return false;
  const Cx omega = cx(1.0) / det_om;
  bool elimd[NC] = {false};
  for (int f = 0; f < 3; ++f) elimd[patch[f]] = true;
  for (int k = 0; k < SNH; ++k) elimd[el[k]] = true;
  int fr[NC], nf = 0;
  for (int k = 0; k < NC; ++k)
    if (!elimd[k]) {
      if (nf >= NF) return false;
      fr[nf++] = k;
    }
  if (nf != NF) return false;
  Cx jpb[NF * NC];
  for (int i = 0; i < NF * NC; ++i) jpb[i] = cx(0.0);
  for (int a = 0; a < NF; ++a) jpb[a * NC + fr[a]] = cx(1.0);
  Cx oi[SNH * SNH];
  if (!inv_gj(om, SNH, oi)) return false;
  for (int a = 0; a < NF; ++a) {
    Cx b[SNH];
    for (int i = 0; i < SNH; ++i) b[i] = jac[i * NC + fr[a]];
    for (int r = 0; r < SNH; ++r) {
      Cx e = cx(0.0);
      for (int c = 0; c < SNH; ++c) e += oi[r * SNH + c] * b[c];
      jpb[a * NC + el[r]] = -e;
    }
  }
  // fs_metric_three_blocks (SS:1090-1135)
  Cx g[NC * NC];
  for (int i = 0; i < NC * NC; ++i) g[i] = cx(0.0);
  for (int f = 0; f < 3; ++f) {
    double nz = 0.0;
    for (int k = S_LO[f]; k < S_HI[f]; ++k)
      if (k != patch[f]) nz += norm_sqr(xr[k]);
    const double den = (1.0 + nz) * (1.0 + nz);
    for (int a = S_LO[f]; a < S_HI[f]; ++a) {
      if (a == patch[f]) continue;
      for (int b = S_LO[f]; b < S_HI[f]; ++b) {
        if (b == patch[f]) continue;
        const double kron = a == b ? 1.0 : 0.0;
        const Cx num = cx(1.0 + nz) * cx(kron) - xr[a] * conj(xr[b]);
        g[a * NC + b] = num / cx(den);
      }
    }
  }
  Cx tmp[NF * NC], gpb[NF * NF];
  for (int a = 0; a < NF; ++a)
    for (int b = 0; b < NC; ++b) {
      Cx sm = cx(0.0);
      for (int k = 0; k < NC; ++k) sm += jpb[a * NC + k] * g[k * NC + b];
      tmp[a * NC + b] = sm;
    }
  for (int a = 0; a < NF; ++a)
    for (int b = 0; b < NF; ++b) {
      Cx sm = cx(0.0);
      for (int k = 0; k < NC; ++k) sm += tmp[a * NC + k] * conj(jpb[b * NC + k]);
      gpb[a * NF + b] = sm;
    }
  const double det_g = det_lu(gpb, NF).re;
  if (!std::isfinite(det_g) || std::fabs(det_g) < 1.0e-300) return false;
  const double weight = norm_sqr(omega) / det_g;
  if (!std::isfinite(weight) || weight <= 0.0) return false;
  for (int k = 0; k < NC; ++k) out->x[k] = xr[k];
  out->omega = omega;
  out->weight = weight;
  return true;
}

// sample_one (SS:429-480)
bool s_sample_one(Rng& rng, SPt* out) {
  Cx p[NC], d[SNH][NC];
  unit_sphere(rng, p);
  for (int j = 0; j < SNH; ++j) unit_sphere(rng, d[j]);
  bool have = false;
  Cx best[NC];
  double best_res = INFINITY;
  for (int att = 0; att < 4; ++att) {
    Cx t[SNH];
    for (int j = 0; j < SNH; ++j) {
      const double re = normal(rng);
      const double im = normal(rng);
      t[j] = cx(re, im);
    }
    Cx x[NC];
    double res;
    const bool conv = s_newton(p, d, t, x, &res);
    if (conv && res < best_res) {
      best_res = res;
      for (int k = 0; k < NC; ++k) best[k] = x[k];
      have = true;
      if (res < 1.0e-8) break;
    }
  }
  if (!have || best_res >= 1.0e-8) return false;
  return s_post_process(best, out);
}

// SchoenMetricPoint's patch indices (SM:1132-1150): argmax over each factor of the rescaled point
void s_patch_indices(SPt& pt) {
  for (int f = 0; f < 3; ++f) {
    int best = S_LO[f];
    double ba = -1.0;
    for (int k = S_LO[f]; k < S_HI[f]; ++k) {
      const double a = norm(pt.x[k]);
      if (a > ba) {
        ba = a;
        best = k;
      }
    }
    pt.patch[f] = best;
  }
}

// sample_points (SS:482-503) with normalise_weights (SS:1177-1185, w *= 1/sum) and apply_z3xz3_quotient
// (SS:555-560); `gpu_stream` draws one Newton attempt per line (52 draws: origin, two directions, t) and keeps
// the first n accepted lines, the layout of the device sampler
std::vector<SPt> s_sample(uint64_t seed, size_t n, bool gpu_stream, bool quotient) {
  Rng rng(seed);
  std::vector<SPt> out;
  if (!gpu_stream) {
    size_t max_total = std::max(n * 64, (size_t)1024), att = 0;
    while (out.size() < n && att < max_total) {
      ++att;
      SPt pt;
      if (s_sample_one(rng, &pt)) out.push_back(pt);
    }
  } else {
    const size_t lines = std::max(n * 4, (size_t)64);
    for (size_t l = 0; l < lines && out.size() < n; ++l) {
      Cx p[NC], d[SNH][NC], t[SNH];
      unit_sphere(rng, p);
      for (int j = 0; j < SNH; ++j) unit_sphere(rng, d[j]);
      for (int j = 0; j < SNH; ++j) {
        const double re = normal(rng);
        const double im = normal(rng);
        t[j] = cx(re, im);
      }
      Cx x[NC];
      double res;
      if (!s_newton(p, d, t, x, &res)) continue;
      SPt pt;
      if (s_post_process(x, &pt)) out.push_back(pt);
    }
  }
  double sum = 0.0;
  for (auto& q : out) sum += q.weight;
  if (std::isfinite(sum) && sum > 0.0) {
    const double inv = 1.0 / sum;
    for (auto& q : out) q.weight *= inv;
  }
  if (quotient) {
    const double inv_k = 1.0 / 9.0;
    for (auto& q : out) q.weight *= inv_k;
  }
  for (auto& q : out) s_patch_indices(q);
  return out;
}

// schoen_generators (GB:705-738): the ideal the basis is reduced by (sign pattern + - - on the t_1 terms)
const std::vector<Mono>& schoen_lms() {
  static std::vector<Mono> lms = [] {
    std::vector<std::vector<std::pair<double, Mono>>> gens(2);
    for (int q = 0; q < 2; ++q)
      for (int k = 0; k < 3; ++k) {
        Mono e{};
        e[3 * q + k] = 3;
        e[6] = 1;
        gens[q].push_back({1.0, e});
        Mono e2{};
        e2[3 * q + k] = 3;
        e2[7] = 1;
        gens[q].push_back({k == 0 ? 1.0 : -1.0, e2});
      }
    return groebner_lms(gens);
  }();
  return lms;
}

// build_schoen_invariant_reduced_basis (SM:1185-1210) over enumerate_bidegree_monomials (ZP:298-315),
// Gamma-invariance = alpha (m1 + 2 m2 + m4 + 2 m5) mod 3 == 0 and beta m7 mod 3 == 0 (ZP:100-186)
std::vector<Mono> s_basis(int dx, int dy, int dt) {
  std::vector<Mono> out;
  const auto& lms = schoen_lms();
  for (int a0 = 0; a0 <= dx; ++a0)
    for (int a1 = 0; a1 <= dx - a0; ++a1)
      for (int b0 = 0; b0 <= dy; ++b0)
        for (int b1 = 0; b1 <= dy - b0; ++b1)
          for (int c0 = 0; c0 <= dt; ++c0) {
            Mono m = {a0, a1, dx - a0 - a1, b0, b1, dy - b0 - b1, c0, dt - c0};
            if ((m[1] + 2 * m[2] + m[4] + 2 * m[5]) % 3 != 0 || m[7] % 3 != 0) continue;
            bool in_ideal = false;
            for (auto& l : lms)
              if (divides(l, m)) {
                in_ideal = true;
                break;
              }
            if (!in_ideal) out.push_back(m);
          }
  return out;
}

// schoen_affine_chart_frame (SM:2202-2270)
bool s_chart_frame(const SPt& pt, Cx frame[NF][NC]) {
  Cx jac[SNH * NC];
  s_jacobian(pt.x, jac);
  int el[SNH];
  if (!s_pick_elim(jac, pt.patch, el)) return false;
  bool taken[NC] = {false};
  for (int f = 0; f < 3; ++f) taken[pt.patch[f]] = true;
  for (int i = 0; i < SNH; ++i) taken[el[i]] = true;
  int fr[NF], nf = 0;
  for (int k = 0; k < NC; ++k)
    if (!taken[k]) {
      if (nf >= NF) return false;
      fr[nf++] = k;
    }
  if (nf != NF) return false;
  Cx je[SNH * SNH], ji[SNH * SNH];
  for (int i = 0; i < SNH; ++i)
    for (int c = 0; c < SNH; ++c) je[i * SNH + c] = jac[i * NC + el[c]];
  if (!inv_gj(je, SNH, ji)) return false;
  for (int a = 0; a < NF; ++a)
    for (int k = 0; k < NC; ++k) frame[a][k] = cx(0.0);
  for (int a = 0; a < NF; ++a) {
    frame[a][fr[a]] = cx(1.0);
    Cx b[SNH];
    for (int i = 0; i < SNH; ++i) b[i] = jac[i * NC + fr[a]];
    for (int c = 0; c < SNH; ++c) {
      Cx e = cx(0.0);
      for (int i = 0; i < SNH; ++i) e += ji[c * SNH + i] * b[i];
      frame[a][el[c]] = -e;
    }
  }
  return true;
}

struct SData {
  std::vector<SPt> pts;
  std::vector<double> w, om2;
  std::vector<Mono> basis;
  std::vector<double> S, D;
};

void s_build(SData& sd) {
  const size_t P = sd.pts.size();
  const int N = (int)sd.basis.size();
  int kmax = 0;
  for (auto& m : sd.basis)
    for (int k = 0; k < NC; ++k) kmax = std::max(kmax, m[k]);
  sd.S.assign(P * 2 * N, 0.0);
  sd.D.assign(P * NC * 2 * N, 0.0);
  par_for(P, [&](size_t p) { sections_at(sd.pts[p].x, sd.basis, kmax, sd.S.data() + p * 2 * N, sd.D.data() + p * NC * 2 * N); });
}

double s_sigma(const SData& sd, const double* hr, const double* hi, double* eta_out) {
  const size_t P = sd.pts.size();
  const int N = (int)sd.basis.size();
  std::vector<double> eta(P);
  par_for(P, [&](size_t p) {
    Cx fr[NF][NC];
    const bool ok = s_chart_frame(sd.pts[p], fr);
    eta[p] = eta_from_frame(ok, fr, sd.S.data() + p * 2 * N, sd.D.data() + p * NC * 2 * N, hr, hi, N, sd.om2[p]);
  });
  if (eta_out) std::copy(eta.begin(), eta.end(), eta_out);
  return sigma_reduce(eta.data(), sd.w.data(), P);
}

SData s_import(const double* coords, const double* omega_sq, const double* weight, size_t P, int dx, int dy, int dt) {
  SData sd;
  sd.pts.resize(P);
  sd.w.assign(weight, weight + P);
  sd.om2.assign(omega_sq, omega_sq + P);
  for (size_t p = 0; p < P; ++p) {
    for (int q = 0; q < NC; ++q) sd.pts[p].x[q] = cx(coords[p * 16 + 2 * q], coords[p * 16 + 2 * q + 1]);
    s_patch_indices(sd.pts[p]);
    sd.pts[p].weight = weight[p];
  }
  sd.basis = s_basis(dx, dy, dt);
  return sd;
}
// The balancing loop of solve_ty_metric / solve_schoen_metric (TY:555-720, SM:830-1000) on a section table:
// damping (static, or the adaptive ramp of SM:571-625), the min-residual snapshot and catastrophe guard,
// sigma after every iteration through `sig`.  Fills rec / histories / h as orc_ty_solve documents.
template <class SigmaFn>
int solve_loop(const double* S, const double* w, size_t P, int N, SigmaFn sig, bool adaptive, int max_iter, double tol,
               double* rec, double* sig_hist, double* res_hist, int hist_cap, double* h_re, double* h_im,
               size_t h_cap) {
  const size_t NN = (size_t)N * N;
  std::vector<double> hr(NN, 0.0), hi(NN, 0.0);
  for (int a = 0; a < N; ++a) hr[a * N + a] = 1.0;
  double alpha = adaptive ? 0.3 : 1.0, a_min = 0.05, a_max = 1.0, last_res = INFINITY;
  int streak = 0;
  int eff_iter = adaptive ? max_iter * std::max(7, 2) : max_iter;
  double sig_fs = sig(hr.data(), hi.data());
  double min_res = INFINITY, final_res = INFINITY;
  std::vector<double> mhr = hr, mhi = hi;
  int min_it = 0, bad = 0, iters = 0;
  std::vector<double> sh, rh;
  for (int it = 0; it < eff_iter; ++it) {
    double res = donaldson_iteration(S, w, P, N, hr.data(), hi.data(), alpha);
    if (adaptive) {
      if (std::isfinite(res)) {
        if (std::isfinite(last_res)) {
          if (res < 0.95 * last_res) {
            if (++streak >= 3) {
              alpha = std::min(alpha * 1.5, a_max);
              streak = 0;
            }
          } else if (res > 1.05 * last_res) {
            alpha = std::max(alpha * 0.7, a_min);
            streak = 0;
          }
        }
      }
      last_res = res;
    }
    if (!std::isfinite(res)) {
      if (std::isfinite(min_res)) {
        hr = mhr;
        hi = mhi;
        rh.push_back(min_res);
        sh.push_back(sig(hr.data(), hi.data()));
        final_res = min_res;
        iters = min_it;
        break;
      }
      return -3;
    }
    rh.push_back(res);
    sh.push_back(sig(hr.data(), hi.data()));
    final_res = res;
    iters = it + 1;
    if (res < min_res) {
      min_res = res;
      mhr = hr;
      mhi = hi;
      min_it = iters;
      bad = 0;
    } else if (std::isfinite(min_res) && min_res < 1.0e-2 && res > 100.0 * min_res) {
      if (++bad >= 5) {
        hr = mhr;
        hi = mhi;
        rh.push_back(min_res);
        sh.push_back(sig(hr.data(), hi.data()));
        final_res = min_res;
        iters = min_it;
        break;
      }
    } else {
      bad = 0;
    }
    if (res < tol) break;
  }
  rec[0] = (double)P;
  rec[1] = (double)N;
  rec[2] = (double)iters;
  rec[3] = sig_fs;
  rec[4] = sh.empty() ? NAN : sh.back();
  rec[5] = final_res;
  for (int i = 0; i < (int)sh.size() && i < hist_cap; ++i) {
    sig_hist[i] = sh[i];
    res_hist[i] = rh[i];
  }
  if (h_re && NN <= h_cap) {
    std::copy(hr.begin(), hr.end(), h_re);
    std::copy(hi.begin(), hi.end(), h_im);
  }
  return (int)sh.size();
}


// adam_refine_sigma_ty (TY:1488-1583; the Schoen loop is the same): finite-difference Adam on sigma^2 over the
// 2 N^2 real parameters of h, each perturbation followed by renormalise_h_trace_ty (TY:1585-1600).
template <class SigmaFn>
int fd_adam(SigmaFn sig, int N, double* hr, double* hi, int max_iters, double lr, double eps, double tol,
            double* hist, int cap) {
  const size_t NN = (size_t)N * N, nd = 2 * NN;
  const double b1 = 0.9, b2 = 0.999, ea = 1.0e-8;
  std::vector<double> m(nd, 0.0), v(nd, 0.0), sr(NN), si(NN), g(nd);
  auto renorm = [&](double* r, double* i) {
    double tr = 0.0;
    for (int a = 0; a < N; ++a) tr += r[(size_t)a * N + a];
    if (std::fabs(tr) > 1.0e-30) {
      const double sc = (double)N / tr;
      for (size_t q = 0; q < NN; ++q) r[q] *= sc;
      for (size_t q = 0; q < NN; ++q) i[q] *= sc;
    }
  };
  auto powi = [](double a, int b) {
    double r = 1.0;
    for (;;) {
      if (b & 1) r *= a;
      b /= 2;
      if (b == 0) break;
      a *= a;
    }
    return r;
  };
  int nh = 0, t = 0;
  double prev = INFINITY;
  for (int it = 0; it < max_iters; ++it) {
    std::copy(hr, hr + NN, sr.begin());
    std::copy(hi, hi + NN, si.begin());
    const double sb = sig(hr, hi);
    if (!std::isfinite(sb)) break;
    if (nh < cap) hist[nh] = sb;
    ++nh;
    if (t > 0 && std::isfinite(prev) && prev > 0.0 && (prev - sb) < tol * prev) break;
    const double sq = sb * sb;
    std::fill(g.begin(), g.end(), 0.0);
    for (int a = 0; a < N; ++a)
      for (int b = 0; b < N; ++b) {
        std::copy(sr.begin(), sr.end(), hr);
        std::copy(si.begin(), si.end(), hi);
        if (a == b)
          hr[(size_t)a * N + a] += eps;
        else {
          hr[(size_t)a * N + b] += eps;
          hr[(size_t)b * N + a] += eps;
        }
        renorm(hr, hi);
        const double sp = sig(hr, hi);
        if (std::isfinite(sp)) g[(size_t)a * N + b] = (sp * sp - sq) / eps;
      }
    for (int a = 0; a < N; ++a)
      for (int b = a + 1; b < N; ++b) {
        std::copy(sr.begin(), sr.end(), hr);
        std::copy(si.begin(), si.end(), hi);
        hi[(size_t)a * N + b] += eps;
        hi[(size_t)b * N + a] -= eps;
        renorm(hr, hi);
        const double sp = sig(hr, hi);
        if (std::isfinite(sp)) g[NN + (size_t)a * N + b] = (sp * sp - sq) / eps;
      }
    std::copy(sr.begin(), sr.end(), hr);
    std::copy(si.begin(), si.end(), hi);
    ++t;
    const double bc1 = 1.0 - powi(b1, t), bc2 = 1.0 - powi(b2, t);
    const double scale = lr * (std::sqrt(bc2) / bc1);
    for (size_t q = 0; q < NN; ++q) {
      m[q] = b1 * m[q] + (1.0 - b1) * g[q];
      v[q] = b2 * v[q] + (1.0 - b2) * g[q] * g[q];
      hr[q] -= scale * m[q] / (std::sqrt(v[q]) + ea);
    }
    for (int a = 0; a < N; ++a)
      for (int b = a + 1; b < N; ++b) {
        const double avg = 0.5 * (hr[(size_t)a * N + b] + hr[(size_t)b * N + a]);
        hr[(size_t)a * N + b] = avg;
        hr[(size_t)b * N + a] = avg;
      }
    for (int a = 0; a < N; ++a)
      for (int b = a + 1; b < N; ++b) {
        const size_t q = NN + (size_t)a * N + b;
        m[q] = b1 * m[q] + (1.0 - b1) * g[q];
        v[q] = b2 * v[q] + (1.0 - b2) * g[q] * g[q];
        const double upd = scale * m[q] / (std::sqrt(v[q]) + ea);
        hi[(size_t)a * N + b] -= upd;
        hi[(size_t)b * N + a] += upd;
      }
    for (int a = 0; a < N; ++a) hi[(size_t)a * N + a] = 0.0;
    renorm(hr, hi);
    prev = sb;
  }
  const double sf = sig(hr, hi);
  if (std::isfinite(sf)) {
    if (nh < cap) hist[nh] = sf;
    ++nh;
  }
  return nh;
}

}  // namespace

extern "C" {

// ChaCha block with a given round count (20 rounds = ChaCha20, for checking the core against
// an independent implementation), 64-bit counter, stream id 0.
void orc_ty_chacha_block(const uint32_t* key, uint64_t counter, int rounds, uint32_t* out) {
  chacha_block(key, counter, 0, rounds, out);
}

void orc_ty_seed_key(uint64_t seed, uint32_t* key) { pcg_seed_key(seed, key); }

void orc_ty_rng_u64(uint64_t seed, size_t n, uint64_t* out) {
  Rng r(seed);
  for (size_t i = 0; i < n; ++i) out[i] = r.next_u64();
}

void orc_ty_normals(uint64_t seed, size_t n, double* out) {
  Rng r(seed);
  for (size_t i = 0; i < n; ++i) out[i] = normal(r);
}

// The rendered ziggurat tables (x[257], f[257]) and r.
void orc_ty_zig_tables(double* x, double* f, double* r) {
  const Zig& z = zig();
  std::memcpy(x, z.x, sizeof z.x);
  std::memcpy(f, z.f, sizeof z.f);
  *r = z.r;
}

// Samples up to n points; coords [n][8] complex interleaved (each factor rescaled by its largest
// coordinate), omega [n] complex, weight [n], zw [n][2] patch indices.  Returns the count.
size_t orc_ty_sample(uint64_t seed, size_t n, int gpu_stream, int z3, double* coords, double* omega,
                     double* weight, int* zw) {
  std::vector<TyPt> pts = sample(seed, n, gpu_stream != 0, z3 != 0);
  export_points(pts, coords, omega, weight, zw);
  return pts.size();
}

// One post-processed line solution (x as 8 complex); returns 1 and fills the outputs, or 0.
int orc_ty_post_process(const double* x_in, double* coords, double* omega, double* weight, int* zw) {
  Cx x[NC];
  for (int k = 0; k < NC; ++k) x[k] = cx(x_in[2 * k], x_in[2 * k + 1]);
  TyPt pt;
  if (!post_process(x, &pt)) return 0;
  std::vector<TyPt> v(1, pt);
  export_points(v, coords, omega, weight, zw);
  return 1;
}

// Leading monomials of the reduced Groebner basis; returns the count (fills up to cap).
int orc_ty_groebner_lms(int* out, int cap) {
  const auto& l = ty_lms();
  for (int i = 0; i < (int)l.size() && i < cap; ++i)
    for (int k = 0; k < NC; ++k) out[i * NC + k] = l[i][k];
  return (int)l.size();
}

// Invariant, ideal-reduced basis at bidegree (k, k); returns the count (fills up to cap).
int orc_ty_basis(int k, int* out, int cap) {
  std::vector<Mono> b = ty_basis(k);
  for (int i = 0; i < (int)b.size() && i < cap; ++i)
    for (int q = 0; q < NC; ++q) out[i * NC + q] = b[i][q];
  return (int)b.size();
}

// Section values [P][2N] and derivatives [P][8][2N] (derivs may be NULL).
void orc_ty_sections(const double* coords, size_t P, const int* basis, int N, double* vals, double* ders) {
  std::vector<Mono> b(N);
  int kmax = 0;
  for (int a = 0; a < N; ++a)
    for (int q = 0; q < NC; ++q) {
      b[a][q] = basis[a * NC + q];
      kmax = std::max(kmax, b[a][q]);
    }
  for (size_t p = 0; p < P; ++p) {
    Cx x[NC];
    for (int q = 0; q < NC; ++q) x[q] = cx(coords[p * 16 + 2 * q], coords[p * 16 + 2 * q + 1]);
    sections_at(x, b, kmax, vals + p * 2 * N, ders ? ders + p * NC * 2 * N : nullptr);
  }
}

// Tangent frames [P][3][8] complex (NaN where the chart fails), from coords and patch indices.
void orc_ty_frames(const double* coords, const int* zw, size_t P, double* out) {
  for (size_t p = 0; p < P; ++p) {
    TyPt pt;
    for (int q = 0; q < NC; ++q) pt.x[q] = cx(coords[p * 16 + 2 * q], coords[p * 16 + 2 * q + 1]);
    pt.zi = zw[2 * p];
    pt.wi = zw[2 * p + 1];
    Cx fr[NF][NC];
    bool ok = chart_frame(pt, fr);
    for (int a = 0; a < NF; ++a)
      for (int q = 0; q < NC; ++q) {
        out[p * 48 + a * 16 + 2 * q] = ok ? fr[a][q].re : NAN;
        out[p * 48 + a * 16 + 2 * q + 1] = ok ? fr[a][q].im : NAN;
      }
  }
}

// One Donaldson iteration on section values [P][2N]; h_re/h_im N x N updated in place.
double orc_ty_donaldson_step(const double* vals, const double* w, size_t P, int N, double* h_re, double* h_im,
                             double alpha) {
  return donaldson_iteration(vals, w, P, N, h_re, h_im, alpha);
}

// sigma on points (coords, omega_sq, weight) at bidegree k for the metric (h_re, h_im); eta [P] out.
double orc_ty_sigma(const double* coords, const double* omega_sq, const double* weight, size_t P, int k,
                    const double* h_re, const double* h_im, double* eta) {
  TyData td = import_points(coords, omega_sq, weight, P, k);
  build_sections(td, true);
  return sigma_of(td, h_re, h_im, eta);
}

// solve_ty_metric (TY:461-760) with the reference's default damping (static 1 for k < 4, the
// adaptive ramp 0.3 / 0.05 / 1.0 of SM:571-625 otherwise), no Tikhonov shift, no Adam.
// rec = {n_points, n_basis, iterations, sigma_fs_identity, sigma_final, final_residual};
// sig_hist / res_hist (capacity hist_cap) get the per-iteration sigma and residual;
// h_re/h_im (N x N, capacity h_cap entries each) get the final metric.  Returns 0, or a
// negative code: -1 too few points, -2 empty basis, -3 non-finite residual before any
// snapshot.
int orc_ty_solve(int k, size_t n_sample, int max_iter, double tol, uint64_t seed, double* rec, double* sig_hist,
                 double* res_hist, int hist_cap, double* h_re, double* h_im, size_t h_cap) {
  TyData td;
  td.pts = sample(seed, n_sample, false, true);
  if (td.pts.size() < n_sample / 2) return -1;
  for (auto& p : td.pts) {
    patch_indices(p);
    td.w.push_back(p.weight);
    td.om2.push_back(norm_sqr(p.omega));
  }
  td.basis = ty_basis(k);
  const int N = (int)td.basis.size();
  if (N == 0) return -2;
  build_sections(td, true);
  return solve_loop(td.S.data(), td.w.data(), td.pts.size(), N,
                    [&](const double* hr, const double* hi) { return sigma_of(td, hr, hi, nullptr); }, k >= 4,
                    max_iter, tol, rec, sig_hist, res_hist, hist_cap, h_re, h_im, h_cap);
}

// Schoen entry points: coords [n][16] (x_0..x_2, y_0..y_2, t_0, t_1 rescaled), omega [n] complex, weight [n],
// patch [n][3] absolute indices.  Returns the count.
size_t orc_schoen_sample(uint64_t seed, size_t n, int gpu_stream, int quotient, double* coords, double* omega,
                         double* weight, int* patch) {
  std::vector<SPt> pts = s_sample(seed, n, gpu_stream != 0, quotient != 0);
  for (size_t p = 0; p < pts.size(); ++p) {
    for (int k = 0; k < NC; ++k) {
      coords[p * 16 + 2 * k] = pts[p].x[k].re;
      coords[p * 16 + 2 * k + 1] = pts[p].x[k].im;
    }
    if (omega) {
      omega[2 * p] = pts[p].omega.re;
      omega[2 * p + 1] = pts[p].omega.im;
    }
    if (weight) weight[p] = pts[p].weight;
    if (patch)
      for (int f = 0; f < 3; ++f) patch[3 * p + f] = pts[p].patch[f];
  }
  return pts.size();
}

int orc_schoen_groebner_lms(int* out, int cap) {
  const auto& l = schoen_lms();
  for (int i = 0; i < (int)l.size() && i < cap; ++i)
    for (int k = 0; k < NC; ++k) out[i * NC + k] = l[i][k];
  return (int)l.size();
}

int orc_schoen_basis(int dx, int dy, int dt, int* out, int cap) {
  std::vector<Mono> b = s_basis(dx, dy, dt);
  for (int i = 0; i < (int)b.size() && i < cap; ++i)
    for (int q = 0; q < NC; ++q) out[i * NC + q] = b[i][q];
  return (int)b.size();
}

void orc_schoen_frames(const double* coords, size_t P, double* out) {
  for (size_t p = 0; p < P; ++p) {
    SPt pt;
    for (int q = 0; q < NC; ++q) pt.x[q] = cx(coords[p * 16 + 2 * q], coords[p * 16 + 2 * q + 1]);
    s_patch_indices(pt);
    Cx fr[NF][NC];
    const bool ok = s_chart_frame(pt, fr);
    for (int a = 0; a < NF; ++a)
      for (int q = 0; q < NC; ++q) {
        out[p * 48 + a * 16 + 2 * q] = ok ? fr[a][q].re : NAN;
        out[p * 48 + a * 16 + 2 * q + 1] = ok ? fr[a][q].im : NAN;
      }
  }
}

double orc_schoen_sigma(const double* coords, const double* omega_sq, const double* weight, size_t P, int dx, int dy,
                        int dt, const double* h_re, const double* h_im, double* eta) {
  SData sd = s_import(coords, omega_sq, weight, P, dx, dy, dt);
  s_build(sd);
  return s_sigma(sd, h_re, h_im, eta);
}

// solve_schoen_metric (SM:766-1000) with the reference's default damping (adaptive when dx + dy + dt >= 10,
// SM:649-665), no Tikhonov shift, no Adam; outputs as orc_ty_solve.
int orc_schoen_solve(int dx, int dy, int dt, size_t n_sample, int max_iter, double tol, uint64_t seed, double* rec,
                     double* sig_hist, double* res_hist, int hist_cap, double* h_re, double* h_im, size_t h_cap) {
  SData sd;
  sd.pts = s_sample(seed, n_sample, false, true);
  if (sd.pts.size() < n_sample / 2) return -1;
  for (auto& q : sd.pts) {
    sd.w.push_back(q.weight);
    sd.om2.push_back(norm_sqr(q.omega));
  }
  sd.basis = s_basis(dx, dy, dt);
  const int N = (int)sd.basis.size();
  if (N == 0) return -2;
  s_build(sd);
  return solve_loop(sd.S.data(), sd.w.data(), sd.pts.size(), N,
                    [&](const double* hr, const double* hi) { return s_sigma(sd, hr, hi, nullptr); },
                    dx + dy + dt >= 10, max_iter, tol, rec, sig_hist, res_hist, hist_cap, h_re, h_im, h_cap);
}


// FD-Adam sigma refinement on points (coords, omega_sq, weight) for geometry 0 (Tian-Yau, degree d[0]) or 1
// (Schoen, d[0..2]) from (h_re, h_im), updated in place; history [cap]; returns its length.
int orc_cicy_adam_refine(int geom, const int* d, const double* coords, const double* omega_sq, const double* weight,
                         size_t P, double* h_re, double* h_im, int max_iters, double lr, double fd_step, double tol,
                         double* hist, int cap) {
  if (geom == 0) {
    TyData td = import_points(coords, omega_sq, weight, P, d[0]);
    build_sections(td, true);
    return fd_adam([&](const double* r, const double* i) { return sigma_of(td, r, i, nullptr); },
                   (int)td.basis.size(), h_re, h_im, max_iters, lr, fd_step, tol, hist, cap);
  }
  SData sd = s_import(coords, omega_sq, weight, P, d[0], d[1], d[2]);
  s_build(sd);
  return fd_adam([&](const double* r, const double* i) { return s_sigma(sd, r, i, nullptr); }, (int)sd.basis.size(),
                 h_re, h_im, max_iters, lr, fd_step, tol, hist, cap);
}

}  // extern "C"
