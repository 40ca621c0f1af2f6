// ORACLE — TEST INFRASTRUCTURE ONLY. Nothing in the product links, loads or calls this file; only the
// tests, the smoke check and bench.py's CPU-baseline leg do, as the checker and the timed CPU reference.
//
// A CPU restatement, in C++, of the Integrity engine's SPH giant-impact step (sean-reid/BotheadStudios,
// project `integrity-engine`). The reference is Rust + WGSL run through wgpu; it cannot be compiled here
// (no Rust toolchain) and its GPU path needs a graphics API that does not exist on these machines, so each
// function below restates the reference's arithmetic from its source and cites the file:line it follows.
//
// Two precisions are restated on purpose:
//   * f32 "GPU-parity" functions follow the WGSL kernels' operation order (shaders/sph_step.wgsl,
//     shaders/bh_gravity.wgsl). They are compiled with -ffp-contract=off so a product kernel that uses the
//     same single-rounding operations reproduces integer/quantised outputs (Morton codes, permutation,
//     tree topology, neighbour sets) bit for bit and float outputs to the last few ulps.
//   * f64 functions follow the CPU physics of record (crates/engine/src/hydrostatic.rs, eos.rs, bhtree.rs,
//     neighbors.rs, atmosphere.rs) and the f64 verifier (tools/sph-verify/src/main.rs). HydroBody::step is
//     also the timed CPU baseline (single thread = the reference; an OpenMP gather variant for all cores).
//
// Parity pinning: the reference ships no golden-vector files. This oracle is pinned against the reference's
// own known-answer tests (exact EOS parameters, EOS invariants, Barnes-Hut theta bounds, the neighbour-grid
// pair-set identity, bbox/Morton exactness and coincident-point codes, Karras tree structure, root COM,
// and the sph-verify force and 50-step integration bounds); see tests/test_oracle_pins.py.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#include <chrono>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr float kPiF = 3.14159265359f;  // sph_step.wgsl:20

// ---------------------------------------------------------------------------------------------------
// Tillotson EOS. f64 form: crates/engine/src/eos.rs:52-96. f32 form: shaders/sph_step.wgsl:78-100.
// The f64 parameter block is [rho0, a, b, A, B, E0, E_iv, E_cv, alpha, beta].
// The f32 block is the 48-byte SphEos layout (gpu_sph.rs:42; sph_step.wgsl:43):
// [rho0, a, b, A, B, E0, E_iv, E_cv, alpha, beta, _p0, _p1].
// ---------------------------------------------------------------------------------------------------
double pressure64(const double* e, double rho, double u) {
  // eos.rs:52-69 (pressure), :71-74 (p_compressed), :77-83 (p_expanded)
  const double rho0 = e[0], a = e[1], b = e[2], A = e[3], B = e[4], e0 = e[5], eiv = e[6], ecv = e[7],
               al = e[8], be = e[9];
  rho = std::max(rho, 1.0e-9);
  const double eta = rho / rho0;
  const double mu = eta - 1.0;
  const double omega_c = u / (e0 * eta * eta) + 1.0;
  const double pc = (a + b / omega_c) * rho * u + A * mu + B * mu * mu;
  if (eta >= 1.0 || u <= eiv) return pc;
  const double omega_e = u / (e0 * eta * eta) + 1.0;
  const double z = rho0 / rho - 1.0;
  const double pe = a * rho * u + (b * rho * u / omega_e + A * mu * std::exp(-be * z)) * std::exp(-al * z * z);
  if (u >= ecv) return pe;
  return ((u - eiv) * pe + (ecv - u) * pc) / (ecv - eiv);
}

// eos.rs:88-96: central differences with dρ = 1e-4 ρ and du = 1e-4|u| + 1.
double sound_speed_sq64(const double* e, double rho, double u) {
  rho = std::max(rho, 1.0e-9);
  const double dr = rho * 1.0e-4;
  const double du = std::fabs(u) * 1.0e-4 + 1.0;
  const double dpdr = (pressure64(e, rho + dr, u) - pressure64(e, rho - dr, u)) / (2.0 * dr);
  const double dpdu = (pressure64(e, rho, u + du) - pressure64(e, rho, u - du)) / (2.0 * du);
  const double p = pressure64(e, rho, u);
  return std::max(dpdr + p / (rho * rho) * dpdu, 0.0);
}

// tools/sph-verify/src/main.rs:97-105: the f64 restatement that follows the WGSL 1e-3 steps.
double sound_speed64_wgsl(const double* e, double rho, double u, double du_floor) {
  const double r = std::max(rho, 1.0e-9);
  const double dr = r * 1.0e-3;
  const double dp = (pressure64(e, r + dr, u) - pressure64(e, r - dr, u)) / (2.0 * dr);
  const double du = std::fabs(u) * 1.0e-3 + du_floor;
  const double dpu = (pressure64(e, r, u + du) - pressure64(e, r, u - du)) / (2.0 * du);
  const double pp = pressure64(e, r, u);
  return std::sqrt(std::max(dp + pp / (r * r) * dpu, 0.0));
}

// sph_step.wgsl:78-89. rho_floor is 1e-9 in the reference's SI units.
float pressure32(const float* e, float rho, float u, float rho_floor) {
  const float r = std::max(rho, rho_floor);
  const float eta = r / e[0];
  const float mu = eta - 1.0f;
  const float omega = u / (e[5] * eta * eta) + 1.0f;
  const float p_c = (e[1] + e[2] / omega) * r * u + e[3] * mu + e[4] * mu * mu;
  if (eta >= 1.0f || u <= e[6]) return p_c;
  const float z = e[0] / r - 1.0f;
  const float p_e = e[1] * r * u + (e[2] * r * u / omega + e[3] * mu * std::exp(-e[9] * z)) * std::exp(-e[8] * z * z);
  if (u >= e[7]) return p_e;
  return ((u - e[6]) * p_e + (e[7] - u) * p_c) / (e[7] - e[6]);
}

// sph_step.wgsl:90-100. du_floor is the "+ 1.0" (J/kg) of dfdu, rho_floor the 1e-9 of max(rho, 1e-9).
float sound_speed32(const float* e, float rho, float u, float du_floor, float rho_floor) {
  const float r = std::max(rho, rho_floor);
  const float dr = r * 1.0e-3f;
  const float dp = (pressure32(e, r + dr, u, rho_floor) - pressure32(e, r - dr, u, rho_floor)) / (2.0f * dr);
  const float p = pressure32(e, r, u, rho_floor);
  const float du = std::fabs(u) * 1.0e-3f + du_floor;
  const float dfdu = (pressure32(e, r, u + du, rho_floor) - pressure32(e, r, u - du, rho_floor)) / (2.0f * du);
  return std::sqrt(std::max(dp + p / (r * r) * dfdu, 0.0f));
}

// ---------------------------------------------------------------------------------------------------
// SPH kernels. Cubic spline with support radius h: f64 atmosphere.rs:39-62, f32 sph_step.wgsl:64-77.
// Wendland C2 (Wendland 1995; Dehnen & Aly 2012, MNRAS 425, Table 1) written from the formula with the
// same support-radius-h convention: W = 21/(2π h³)(1-q)^4(1+4q), dW/dr = 21/(2π h³)·(-20 q (1-q)^3)/h.
// ---------------------------------------------------------------------------------------------------
double w_cubic64(double r, double h) {  // atmosphere.rs:39-49
  const double q = r / h;
  const double sigma = 8.0 / (kPi * h * h * h);
  if (q < 0.5) return sigma * (6.0 * (q * q * q - q * q) + 1.0);
  if (q < 1.0) return sigma * 2.0 * (1.0 - q) * (1.0 - q) * (1.0 - q);
  return 0.0;
}
double dw_cubic64(double r, double h) {  // atmosphere.rs:52-62
  const double q = r / h;
  const double sigma = 8.0 / (kPi * h * h * h * h);
  if (q < 0.5) return sigma * (18.0 * q * q - 12.0 * q);
  if (q < 1.0) return sigma * -6.0 * (1.0 - q) * (1.0 - q);
  return 0.0;
}
double w_cubic64_verify(double r, double h) {  // tools/sph-verify/src/main.rs:70-74
  const double q = r / h;
  const double sig = 8.0 / (kPi * h * h * h);
  if (q < 0.5) return sig * (1.0 - 6.0 * q * q + 6.0 * q * q * q);
  if (q < 1.0) { const double t = 1.0 - q; return sig * 2.0 * t * t * t; }
  return 0.0;
}
double dw_cubic64_verify(double r, double h) {  // tools/sph-verify/src/main.rs:75-79
  const double q = r / h;
  const double sig = 8.0 / (kPi * h * h * h);
  if (q < 0.5) return sig * (-12.0 * q + 18.0 * q * q) / h;
  if (q < 1.0) { const double t = 1.0 - q; return sig * (-6.0 * t * t) / h; }
  return 0.0;
}
double w_wendland64(double r, double h) {
  const double q = r / h;
  if (q >= 1.0) return 0.0;
  const double t = 1.0 - q;
  return 21.0 / (2.0 * kPi * h * h * h) * t * t * t * t * (1.0 + 4.0 * q);
}
double dw_wendland64(double r, double h) {
  const double q = r / h;
  if (q >= 1.0) return 0.0;
  const double t = 1.0 - q;
  return 21.0 / (2.0 * kPi * h * h * h) * (-20.0 * q * t * t * t) / h;
}
float w_cubic32(float r, float h) {  // sph_step.wgsl:64-70
  const float q = r / h;
  const float sig = 8.0f / (kPiF * h * h * h);
  if (q < 0.5f) return sig * (1.0f - 6.0f * q * q + 6.0f * q * q * q);
  if (q < 1.0f) { const float t = 1.0f - q; return sig * 2.0f * t * t * t; }
  return 0.0f;
}
float dw_cubic32(float r, float h) {  // sph_step.wgsl:71-77
  const float q = r / h;
  const float sig = 8.0f / (kPiF * h * h * h);
  if (q < 0.5f) return sig * (-12.0f * q + 18.0f * q * q) / h;
  if (q < 1.0f) { const float t = 1.0f - q; return sig * (-6.0f * t * t) / h; }
  return 0.0f;
}
float w_wendland32(float r, float h) {
  const float q = r / h;
  if (q >= 1.0f) return 0.0f;
  const float t = 1.0f - q;
  return 21.0f / (2.0f * kPiF * h * h * h) * t * t * t * t * (1.0f + 4.0f * q);
}
float dw_wendland32(float r, float h) {
  const float q = r / h;
  if (q >= 1.0f) return 0.0f;
  const float t = 1.0f - q;
  return 21.0f / (2.0f * kPiF * h * h * h) * (-20.0f * q * t * t * t) / h;
}
inline float kern_w32(int kind, float r, float h) { return kind == 1 ? w_wendland32(r, h) : w_cubic32(r, h); }
inline float kern_dw32(int kind, float r, float h) { return kind == 1 ? dw_wendland32(r, h) : dw_cubic32(r, h); }

// Pair distance exactly as the product computes it: single-rounded products and sums, left to right, then
// an IEEE square root (the WGSL `length(pi.pos - pj.pos)` of sph_step.wgsl:141 with no contraction).
inline float pair_r32(const float* pi, const float* pj) {
  const float dx = pi[0] - pj[0], dy = pi[1] - pj[1], dz = pi[2] - pj[2];
  return std::sqrt((dx * dx + dy * dy) + dz * dz);
}

// ---------------------------------------------------------------------------------------------------
// Morton codes (bh_gravity.wgsl:49-108; CPU twin gpu_gravity.rs:336-357,495-502).
// ---------------------------------------------------------------------------------------------------
uint32_t expand_bits(uint32_t v) {  // bh_gravity.wgsl:82-89
  v &= 0x000003ffu;
  v = (v * 0x00010001u) & 0xff0000ffu;
  v = (v * 0x00000101u) & 0x0f00f00fu;
  v = (v * 0x00000011u) & 0xc30c30c3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
uint32_t morton32(const float* p, const float* lo, const float* hi) {  // bh_gravity.wgsl:91-98,105
  uint32_t q[3];
  for (int k = 0; k < 3; ++k) {
    const float ext = std::max(hi[k] - lo[k], 1.0e-30f);
    float u = (p[k] - lo[k]) / ext;
    u = std::min(std::max(u, 0.0f), 1.0f);
    float f = std::floor(u * 1024.0f);
    f = std::min(std::max(f, 0.0f), 1023.0f);
    q[k] = static_cast<uint32_t>(f);
  }
  return expand_bits(q[0]) * 4u + expand_bits(q[1]) * 2u + expand_bits(q[2]);
}

inline int clz32(uint32_t x) { return x == 0 ? 32 : __builtin_clz(x); }

// Karras δ with the index tiebreak, bh_gravity.wgsl:114-120.
inline int kdelta(const uint32_t* codes, int L, int i, int j) {
  if (j < 0 || j >= L) return -1;
  const uint32_t ci = codes[i], cj = codes[j];
  if (ci == cj) return 32 + clz32(static_cast<uint32_t>(i) ^ static_cast<uint32_t>(j));
  return clz32(ci ^ cj);
}

// One internal node of the Karras build, bh_gravity.wgsl:135-184. Returns (left, right).
// exact_dups = 0 reproduces the reference; 1 splits runs of equal codes on the index-extended key
// (Karras 2012 §4), which the reference's midpoint split does not always agree with.
void karras_node(const uint32_t* codes, int L, int i, uint32_t* left, uint32_t* right, int exact_dups) {
  const int d = kdelta(codes, L, i, i + 1) > kdelta(codes, L, i, i - 1) ? 1 : -1;
  const int dmin = kdelta(codes, L, i, i - d);
  int lmax = 2;
  while (kdelta(codes, L, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (kdelta(codes, L, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int first = std::min(i, j), last = std::max(i, j);
  int split = first;
  const uint32_t fc = codes[first], lc = codes[last];
  if (fc == lc && !exact_dups) {
    split = (first + last) >> 1;
  } else if (fc == lc) {
    const int cpfx = kdelta(codes, L, first, last);
    int step = last - first;
    for (;;) {
      step = (step + 1) >> 1;
      const int ns = split + step;
      if (ns < last && kdelta(codes, L, first, ns) > cpfx) split = ns;
      if (step <= 1) break;
    }
  } else {
    const int cpfx = clz32(fc ^ lc);
    int step = last - first;
    for (;;) {
      step = (step + 1) >> 1;
      const int ns = split + step;
      if (ns < last && clz32(fc ^ codes[ns]) > cpfx) split = ns;
      if (step <= 1) break;
    }
  }
  const bool ll = (split == first), rl = (split + 1 == last);
  *left = ll ? static_cast<uint32_t>((L - 1) + split) : static_cast<uint32_t>(split);
  *right = rl ? static_cast<uint32_t>((L - 1) + split + 1) : static_cast<uint32_t>(split + 1);
}

// ---------------------------------------------------------------------------------------------------
// Uniform cell list used only to enumerate candidate pairs; the neighbour predicate is always exact.
// ---------------------------------------------------------------------------------------------------
struct CellList {
  double cell = 1.0;
  std::vector<int64_t> keys;     // sorted cell keys
  std::vector<int> start, order;  // order[] = particle indices sorted by cell key (stable)
  static int64_t pack(int64_t x, int64_t y, int64_t z) {
    return ((x + (1 << 20)) << 42) | ((y + (1 << 20)) << 21) | (z + (1 << 20));
  }
  template <class GetPos>
  void build(int n, double cell_size, GetPos pos) {
    cell = std::max(cell_size, 1.0e-30);
    std::vector<int64_t> k(n);
    for (int i = 0; i < n; ++i) {
      double p[3];
      pos(i, p);
      k[i] = pack((int64_t)std::floor(p[0] / cell), (int64_t)std::floor(p[1] / cell), (int64_t)std::floor(p[2] / cell));
    }
    order.resize(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return k[a] < k[b]; });
    keys.clear();
    start.clear();
    for (int s = 0; s < n; ++s) {
      if (s == 0 || k[order[s]] != k[order[s - 1]]) {
        keys.push_back(k[order[s]]);
        start.push_back(s);
      }
    }
    start.push_back(n);
  }
  // Calls f(j) for every particle in the 27 cells around point p.
  template <class F>
  void around(const double* p, F f) const {
    const int64_t cx = (int64_t)std::floor(p[0] / cell), cy = (int64_t)std::floor(p[1] / cell),
                  cz = (int64_t)std::floor(p[2] / cell);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int64_t key = pack(cx + dx, cy + dy, cz + dz);
          auto it = std::lower_bound(keys.begin(), keys.end(), key);
          if (it == keys.end() || *it != key) continue;
          const size_t c = it - keys.begin();
          for (int s = start[c]; s < start[c + 1]; ++s) f(order[s]);
        }
  }
};

// ---------------------------------------------------------------------------------------------------
// f64 Barnes-Hut octree, crates/engine/src/bhtree.rs:21-190 (BRUTE_BELOW 1024, MAX_DEPTH 28, MAC
// (2·half)/dist < θ with dist = sqrt(|d|²+ε²)).
// ---------------------------------------------------------------------------------------------------
struct OctNode {
  double center[3], half, com[3], mass;
  int children[8];
  int leaf_begin, leaf_end;  // into OctTree::leaf_idx; empty range = internal
};
struct OctTree {
  std::vector<OctNode> nodes;
  std::vector<int> leaf_idx;
  double theta = 0.5, soft2 = 0.0, G = 6.674e-11;
  int n = 0;
  const double* pos = nullptr;
  const double* mass = nullptr;

  int build_node(std::vector<int>& idx, const double* c, double half, int depth) {
    const int id = (int)nodes.size();
    double m = 0.0, com[3] = {0, 0, 0};
    for (int i : idx) {
      m += mass[i];
      for (int k = 0; k < 3; ++k) com[k] += pos[3 * i + k] * mass[i];
    }
    OctNode nd;
    for (int k = 0; k < 3; ++k) {
      nd.center[k] = c[k];
      nd.com[k] = m > 0.0 ? com[k] / m : c[k];
    }
    nd.half = half;
    nd.mass = m;
    for (int o = 0; o < 8; ++o) nd.children[o] = -1;
    nd.leaf_begin = nd.leaf_end = 0;
    nodes.push_back(nd);
    if (idx.size() <= 1 || depth >= 28) {
      nodes[id].leaf_begin = (int)leaf_idx.size();
      leaf_idx.insert(leaf_idx.end(), idx.begin(), idx.end());
      nodes[id].leaf_end = (int)leaf_idx.size();
      return id;
    }
    std::vector<int> oct[8];
    for (int i : idx) {
      const double* p = pos + 3 * i;
      const int o = (p[0] >= c[0] ? 1 : 0) | (p[1] >= c[1] ? 2 : 0) | (p[2] >= c[2] ? 4 : 0);
      oct[o].push_back(i);
    }
    idx.clear();
    idx.shrink_to_fit();
    const double ch = half * 0.5;
    for (int o = 0; o < 8; ++o) {
      if (oct[o].empty()) continue;
      const double cc[3] = {c[0] + ((o & 1) ? ch : -ch), c[1] + ((o & 2) ? ch : -ch), c[2] + ((o & 4) ? ch : -ch)};
      const int cid = build_node(oct[o], cc, ch, depth + 1);
      nodes[id].children[o] = cid;
    }
    return id;
  }
  void build(const double* p, const double* m, int n_, double th, double soft, double g) {
    pos = p; mass = m; n = n_; theta = th; soft2 = soft * soft; G = g;
    nodes.clear(); leaf_idx.clear();
    if (n < 1024) return;  // BRUTE_BELOW
    double lo[3], hi[3];
    for (int k = 0; k < 3; ++k) lo[k] = hi[k] = p[k];
    for (int i = 1; i < n; ++i)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], p[3 * i + k]);
        hi[k] = std::max(hi[k], p[3 * i + k]);
      }
    double c[3], ext = 0.0;
    for (int k = 0; k < 3; ++k) { c[k] = (lo[k] + hi[k]) * 0.5; ext = std::max(ext, hi[k] - lo[k]); }
    const double half = std::max(ext * 0.5, 1.0e-9) * 1.0001;
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
    nodes.reserve(2 * (size_t)n);
    build_node(all, c, half, 0);
  }
  void accel_on(int i, int node, double* a) const {
    const OctNode& nd = nodes[node];
    const double* pi = pos + 3 * i;
    if (nd.leaf_end > nd.leaf_begin) {
      for (int s = nd.leaf_begin; s < nd.leaf_end; ++s) {
        const int j = leaf_idx[s];
        if (j == i) continue;
        const double d[3] = {pos[3 * j] - pi[0], pos[3 * j + 1] - pi[1], pos[3 * j + 2] - pi[2]};
        const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + soft2;
        const double g = G * mass[j] / (r2 * std::sqrt(r2));
        for (int k = 0; k < 3; ++k) a[k] += d[k] * g;
      }
      return;
    }
    const double d[3] = {nd.com[0] - pi[0], nd.com[1] - pi[1], nd.com[2] - pi[2]};
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + soft2;
    const double dist = std::sqrt(r2);
    if ((2.0 * nd.half) / dist < theta) {
      const double g = G * nd.mass / (r2 * dist);
      for (int k = 0; k < 3; ++k) a[k] += d[k] * g;
      return;
    }
    for (int o = 0; o < 8; ++o)
      if (nd.children[o] >= 0) {
        double b[3] = {0, 0, 0};
        accel_on(i, nd.children[o], b);
        for (int k = 0; k < 3; ++k) a[k] += b[k];
      }
  }
  void accelerations(double* acc, int nthreads) const {
    if (nodes.empty()) {  // brute force, bhtree.rs:118-131
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
      for (int i = 0; i < n; ++i) {
        double a[3] = {0, 0, 0};
        for (int j = 0; j < n; ++j) {
          if (i == j) continue;
          const double d[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1], pos[3 * j + 2] - pos[3 * i + 2]};
          const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + soft2;
          const double g = G * mass[j] / (r2 * std::sqrt(r2));
          for (int k = 0; k < 3; ++k) a[k] += d[k] * g;
        }
        for (int k = 0; k < 3; ++k) acc[3 * i + k] = a[k];
      }
      return;
    }
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
    for (int i = 0; i < n; ++i) {
      double a[3] = {0, 0, 0};
      accel_on(i, 0, a);
      for (int k = 0; k < 3; ++k) acc[3 * i + k] = a[k];
    }
  }
};

// ---------------------------------------------------------------------------------------------------
// HydroBody (crates/engine/src/hydrostatic.rs:241-374): the f64 CPU path of record and the timed baseline.
// ---------------------------------------------------------------------------------------------------
struct Hydro {
  int n = 0, n_eos = 0;
  std::vector<double> pos, vel, mass, u, h, rho, eos;  // eos: n_eos × 10
  std::vector<int> mat;
  double softening = 0.0, G = 6.674e-11, theta = 0.5, av_alpha = 1.0, av_beta = 2.0;
  int kernel = 0;  // 0 cubic spline (reference), 1 Wendland C2

  double W(double r, double hh) const { return kernel == 1 ? w_wendland64(r, hh) : w_cubic64(r, hh); }
  double dW(double r, double hh) const { return kernel == 1 ? dw_wendland64(r, hh) : dw_cubic64(r, hh); }
  double hmax() const { double m = 0.0; for (double x : h) m = std::max(m, x); return m; }

  // compute_density, hydrostatic.rs:241-256. Single thread: the reference's symmetric i<j pair loop over
  // the NeighborGrid (neighbors.rs:60-85). Multi-thread: a per-i gather over the same 27-cell candidates.
  void compute_density(int nthreads) {
    rho.assign(n, 0.0);
    for (int i = 0; i < n; ++i) rho[i] = mass[i] * W(0.0, h[i]);
    if (n < 512) {  // neighbors.rs:23 BRUTE_BELOW: all i<j pairs
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) density_pair(i, j);
      return;
    }
    CellList cl;
    cl.build(n, hmax(), [&](int i, double* p) { for (int k = 0; k < 3; ++k) p[k] = pos[3 * i + k]; });
    if (nthreads <= 1) {
      for (int i = 0; i < n; ++i) cl.around(&pos[3 * i], [&](int j) { if (j > i) density_pair(i, j); });
    } else {
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
      for (int i = 0; i < n; ++i) {
        double acc = 0.0;
        cl.around(&pos[3 * i], [&](int j) {
          if (j == i) return;
          const double r = dist(i, j), hij = 0.5 * (h[i] + h[j]);
          if (r < hij) acc += mass[j] * W(r, hij);
        });
        rho[i] += acc;
      }
    }
  }
  double dist(int i, int j) const {
    const double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
    return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  }
  void density_pair(int i, int j) {
    const double r = dist(i, j), hij = 0.5 * (h[i] + h[j]);
    if (r < hij) {
      const double w = W(r, hij);
      rho[i] += mass[j] * w;
      rho[j] += mass[i] * w;
    }
  }

  // Pressure and sound speed of every particle (eos.rs:52-96), once per force evaluation.
  void eos_all(int nthreads, std::vector<double>& p, std::vector<double>& c) const {
    p.resize(n);
    c.resize(n);
#pragma omp parallel for num_threads(std::max(nthreads, 1))
    for (int i = 0; i < n; ++i) {
      const double* e = &eos[10 * (size_t)mat[i]];
      p[i] = pressure64(e, rho[i], u[i]);
      c[i] = std::sqrt(sound_speed_sq64(e, rho[i], u[i]));
    }
  }
  // The pair terms of forces_and_dudt (hydrostatic.rs:300-340): pressure + Monaghan AV + du/dt of the pair
  // (i, j), added to i and, when aj is given, with the opposite sign to j.
  bool pair_terms(int i, int j, const std::vector<double>& p, const std::vector<double>& c, double* ai, double& dui,
                  double* aj, double& duj) const {
    const double dpos[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
    const double r = std::sqrt(dpos[0] * dpos[0] + dpos[1] * dpos[1] + dpos[2] * dpos[2]);
    const double hij = 0.5 * (h[i] + h[j]);
    if (r >= hij || r < 1.0e-9) return false;
    const double dvel[3] = {vel[3 * i] - vel[3 * j], vel[3 * i + 1] - vel[3 * j + 1], vel[3 * i + 2] - vel[3 * j + 2]};
    const double vr = dvel[0] * dpos[0] + dvel[1] * dpos[1] + dvel[2] * dpos[2];
    double pi_ij = 0.0;
    if (vr < 0.0) {
      const double mu = hij * vr / (r * r + 0.01 * hij * hij);
      const double c_bar = 0.5 * (c[i] + c[j]);
      const double rho_bar = 0.5 * (rho[i] + rho[j]);
      pi_ij = (-av_alpha * c_bar * mu + av_beta * mu * mu) / rho_bar;
    }
    const double coeff = p[i] / (rho[i] * rho[i]) + p[j] / (rho[j] * rho[j]) + pi_ij;
    const double dw = dW(r, hij);
    const double grad[3] = {dpos[0] / r * dw, dpos[1] / r * dw, dpos[2] / r * dw};
    const double vdg = dvel[0] * grad[0] + dvel[1] * grad[1] + dvel[2] * grad[2];
    for (int k = 0; k < 3; ++k) { ai[k] += grad[k] * (-coeff * mass[j]); if (aj) aj[k] += grad[k] * (coeff * mass[i]); }
    dui += 0.5 * mass[j] * coeff * vdg;
    duj += 0.5 * mass[i] * coeff * vdg;
    return true;
  }

  // forces_and_dudt, hydrostatic.rs:300-340: BH gravity + pressure + Monaghan AV + du/dt.
  void forces(std::vector<double>& acc, std::vector<double>& dudt, int nthreads) {
    acc.assign(3 * (size_t)n, 0.0);
    dudt.assign(n, 0.0);
    OctTree bh;
    bh.build(pos.data(), mass.data(), n, theta, softening, G);
    bh.accelerations(acc.data(), std::max(nthreads, 1));
    std::vector<double> p, c;
    eos_all(nthreads, p, c);
    if (n < 512) {
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) pair_terms(i, j, p, c, &acc[3 * i], dudt[i], &acc[3 * j], dudt[j]);
      return;
    }
    CellList cl;
    cl.build(n, hmax(), [&](int i, double* q) { for (int k = 0; k < 3; ++k) q[k] = pos[3 * i + k]; });
    if (nthreads <= 1) {
      for (int i = 0; i < n; ++i)
        cl.around(&pos[3 * i], [&](int j) { if (j > i) pair_terms(i, j, p, c, &acc[3 * i], dudt[i], &acc[3 * j], dudt[j]); });
    } else {
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
      for (int i = 0; i < n; ++i) {
        double ai[3] = {0, 0, 0}, dui = 0.0, dummy = 0.0;
        cl.around(&pos[3 * i], [&](int j) { if (j != i) pair_terms(i, j, p, c, ai, dui, nullptr, dummy); });
        for (int k = 0; k < 3; ++k) acc[3 * i + k] += ai[k];
        dudt[i] += dui;
      }
    }
  }

  // One force evaluation of the single-threaded path (the reference's own: symmetric i < j pair loops over
  // the neighbour grid, a per-particle octree walk) timed at full size with its per-particle loops run over
  // every `stride`-th block of 512 consecutive particles only (blocks keep the cache reuse that consecutive,
  // spatially close particles give the full loops). t[0] = seconds of the parts that run in full (grid and
  // octree builds, the EOS of every particle), t[1] = seconds of the sampled loops (density pairs, gravity
  // walks, force pairs). A full evaluation takes about t[0] + stride · t[1]. The state is left unchanged.
  void eval_sampled(int stride, double* t) {
    constexpr int kBlock = 512;
    auto sampled = [&](auto&& f) {
      for (int b0 = 0; b0 < n; b0 += kBlock * stride)
        for (int i = b0; i < std::min(b0 + kBlock, n); ++i) f(i);
    };
    using clk = std::chrono::steady_clock;
    auto sec = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
    std::vector<double> rho_s(n);
    auto t0 = clk::now();
    for (int i = 0; i < n; ++i) rho_s[i] = mass[i] * W(0.0, h[i]);
    CellList cl;
    cl.build(n, hmax(), [&](int i, double* q) { for (int k = 0; k < 3; ++k) q[k] = pos[3 * i + k]; });
    auto t1 = clk::now();
    sampled([&](int i) {
      cl.around(&pos[3 * i], [&](int j) {
        if (j <= i) return;
        const double r = dist(i, j), hij = 0.5 * (h[i] + h[j]);
        if (r < hij) {
          const double w = W(r, hij);
          rho_s[i] += mass[j] * w;
          rho_s[j] += mass[i] * w;
        }
      });
    });
    auto t2 = clk::now();
    OctTree bh;
    bh.build(pos.data(), mass.data(), n, theta, softening, G);
    auto t3 = clk::now();
    std::vector<double> acc(3 * (size_t)n, 0.0), dudt(n, 0.0);
    sampled([&](int i) { bh.accel_on(i, 0, &acc[3 * i]); });
    auto t4 = clk::now();
    std::vector<double> p, c;
    eos_all(1, p, c);
    CellList cl2;
    cl2.build(n, hmax(), [&](int i, double* q) { for (int k = 0; k < 3; ++k) q[k] = pos[3 * i + k]; });
    auto t5 = clk::now();
    sampled([&](int i) {
      cl2.around(&pos[3 * i], [&](int j) { if (j > i) pair_terms(i, j, p, c, &acc[3 * i], dudt[i], &acc[3 * j], dudt[j]); });
    });
    auto t6 = clk::now();
    t[0] = sec(t0, t1) + sec(t2, t3) + sec(t4, t5);
    t[1] = sec(t1, t2) + sec(t3, t4) + sec(t5, t6);
  }

  // step, hydrostatic.rs:345-359 (KDK, two force evaluations, u clamped at 0).
  void step(double dt, int nthreads) {
    std::vector<double> a, du;
    compute_density(nthreads);
    forces(a, du, nthreads);
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) vel[3 * i + k] += a[3 * i + k] * (0.5 * dt);
      u[i] = std::max(u[i] + du[i] * (0.5 * dt), 0.0);
      for (int k = 0; k < 3; ++k) pos[3 * i + k] += vel[3 * i + k] * dt;
    }
    compute_density(nthreads);
    forces(a, du, nthreads);
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) vel[3 * i + k] += a[3 * i + k] * (0.5 * dt);
      u[i] = std::max(u[i] + du[i] * (0.5 * dt), 0.0);
    }
  }
  // courant_dt, hydrostatic.rs:366-374 (assumes compute_density ran).
  double courant_dt(double cfl, double sig_floor) const {
    double dtm = INFINITY;
    for (int i = 0; i < n; ++i) {
      const double c = std::sqrt(sound_speed_sq64(&eos[10 * (size_t)mat[i]], rho[i], u[i]));
      const double vv = std::sqrt(vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] + vel[3 * i + 2] * vel[3 * i + 2]);
      dtm = std::min(dtm, h[i] / std::max(c + vv, sig_floor));
    }
    return cfl * dtm;
  }
};

// ---------------------------------------------------------------------------------------------------
// f32 SPH restatement of sph_step.wgsl cs_density (:120-149) and the SPH half of cs_forces (:153-211).
// The neighbour SET is the reference's exact set {j != i : r < ½(h_i+h_j)} (the grid with its
// cell-membership guard enumerates exactly this set, sph_step.wgsl:136-143); the sum runs over j ascending.
// ---------------------------------------------------------------------------------------------------
void neighbour_sets32(const float* pos4, int n, std::vector<std::vector<int>>& nb) {
  nb.assign(n, {});
  float hm = 0.0f;
  for (int i = 0; i < n; ++i) hm = std::max(hm, pos4[4 * i + 3]);
  CellList cl;
  cl.build(n, (double)hm * (1.0 + 1.0e-6), [&](int i, double* p) { for (int k = 0; k < 3; ++k) p[k] = pos4[4 * i + k]; });
  for (int i = 0; i < n; ++i) {
    double p[3] = {pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2]};
    cl.around(p, [&](int j) {
      if (j == i) return;
      const float r = pair_r32(&pos4[4 * i], &pos4[4 * j]);
      const float hij = 0.5f * (pos4[4 * i + 3] + pos4[4 * j + 3]);
      if (r < hij) nb[i].push_back(j);
    });
    std::sort(nb[i].begin(), nb[i].end());
  }
}

}  // namespace

// =====================================================================================================
// C ABI of the oracle (loaded by oracle/__init__.py through ctypes).
// =====================================================================================================
extern "C" {

int orc_version() { return 1; }

double orc_pressure64(const double* e, double rho, double u) { return pressure64(e, rho, u); }
double orc_sound_speed_sq64(const double* e, double rho, double u) { return sound_speed_sq64(e, rho, u); }
double orc_sound_speed64_wgsl(const double* e, double rho, double u, double du_floor) {
  return sound_speed64_wgsl(e, rho, u, du_floor);
}
float orc_pressure32(const float* e, float rho, float u, float rho_floor) { return pressure32(e, rho, u, rho_floor); }
float orc_sound_speed32(const float* e, float rho, float u, float du_floor, float rho_floor) {
  return sound_speed32(e, rho, u, du_floor, rho_floor);
}
// Per-particle EOS over a material table (n_eos × 12 floats): P and c as sph_step.wgsl:158-159.
void orc_eos32(const float* eos12, const uint32_t* mat, const float* rho, const float* u, int n, float du_floor,
               float rho_floor, float* P, float* c) {
  for (int i = 0; i < n; ++i) {
    const float* e = eos12 + 12 * (size_t)mat[i];
    P[i] = pressure32(e, rho[i], u[i], rho_floor);
    c[i] = sound_speed32(e, rho[i], u[i], du_floor, rho_floor);
  }
}

double orc_w64(int kind, double r, double h) { return kind == 1 ? w_wendland64(r, h) : w_cubic64(r, h); }
double orc_dw64(int kind, double r, double h) { return kind == 1 ? dw_wendland64(r, h) : dw_cubic64(r, h); }
float orc_w32(int kind, float r, float h) { return kern_w32(kind, r, h); }
float orc_dw32(int kind, float r, float h) { return kern_dw32(kind, r, h); }

// ---- Morton / sort / Karras / moments / traversal (bh_gravity.wgsl, gpu_gravity.rs) -----------------
void orc_bbox32(const float* pos4, int n, float* lo, float* hi) {  // cs_bbox, bh_gravity.wgsl:68-78
  for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], pos4[4 * i + k]);
      hi[k] = std::max(hi[k], pos4[4 * i + k]);
    }
}
void orc_morton32(const float* pos4, int n, const float* lo, const float* hi, uint32_t* codes) {
  for (int i = 0; i < n; ++i) codes[i] = morton32(&pos4[4 * i], lo, hi);
}
// gpu_gravity.rs:360 / gpu-bh-verify main.rs:383: sort the (code, index) pairs.
void orc_sort_code_index(const uint32_t* codes, int n, uint32_t* order, uint32_t* sorted_codes) {
  std::vector<uint32_t> o(n);
  std::iota(o.begin(), o.end(), 0u);
  std::sort(o.begin(), o.end(), [&](uint32_t a, uint32_t b) { return codes[a] != codes[b] ? codes[a] < codes[b] : a < b; });
  for (int t = 0; t < n; ++t) { order[t] = o[t]; sorted_codes[t] = codes[o[t]]; }
}
// Cluster codes (gpu_gravity.rs:366) + Karras internal nodes (cs_tree). parent[] as cs_tree_reset/cs_tree.
void orc_karras(const uint32_t* leaf_codes, int L, uint32_t* left, uint32_t* right, uint32_t* parent,
                int exact_dups) {
  const int nn = 2 * L - 1;
  for (int i = 0; i < nn; ++i) parent[i] = 0xffffffffu;
  for (int i = 0; i < L - 1; ++i) {
    karras_node(leaf_codes, L, i, &left[i], &right[i], exact_dups);
    parent[left[i]] = (uint32_t)i;
    parent[right[i]] = (uint32_t)i;
  }
}
// Structural check of gpu-bh-verify main.rs:420-459 (verify_tree): 1 = valid.
int orc_verify_tree(const uint32_t* left, const uint32_t* right, const uint32_t* parent, int L) {
  if (L == 1) return 1;
  const int ni = L - 1, nn = 2 * L - 1;
  if (parent[0] != 0xffffffffu) return 0;
  std::vector<int> visited(nn, 0);
  std::vector<int> st{0};
  int leaves = 0, internals = 0;
  while (!st.empty()) {
    const int idx = st.back();
    st.pop_back();
    if (idx >= nn) return 0;
    if (++visited[idx] > 1) return 0;
    if (idx >= ni) { ++leaves; continue; }
    ++internals;
    const int l = (int)left[idx], r = (int)right[idx];
    if (l >= nn || r >= nn) return 0;
    if ((int)parent[l] != idx || (int)parent[r] != idx) return 0;
    st.push_back(l);
    st.push_back(r);
  }
  return (leaves == L && internals == ni) ? 1 : 0;
}
// Bottom-up moments: leaf bucket sums (bh_gravity.wgsl:205-222) and the mass-weighted merge (:229-238).
// Node arrays are float4 per node: com4 = (com.xyz, mass), bmin4/bmax4 = (xyz, 0).
void orc_moments32(const float* sb4, int n, int K, int L, const uint32_t* left, const uint32_t* right,
                   float* com4, float* bmin4, float* bmax4) {
  const int leaf0 = L - 1;
  for (int c = 0; c < L; ++c) {
    const int li = leaf0 + c, s0 = c * K, s1 = std::min(s0 + K, n);
    float m = 0.0f, mx[3] = {0, 0, 0}, lo[3] = {1.0e30f, 1.0e30f, 1.0e30f}, hi[3] = {-1.0e30f, -1.0e30f, -1.0e30f};
    for (int s = s0; s < s1; ++s) {
      const float* b = &sb4[4 * s];
      m += b[3];
      for (int k = 0; k < 3; ++k) {
        mx[k] += b[k] * b[3];
        lo[k] = std::min(lo[k], b[k]);
        hi[k] = std::max(hi[k], b[k]);
      }
    }
    for (int k = 0; k < 3; ++k) {
      com4[4 * li + k] = m > 0.0f ? mx[k] / m : 0.0f;
      bmin4[4 * li + k] = lo[k];
      bmax4[4 * li + k] = hi[k];
    }
    com4[4 * li + 3] = m;
    bmin4[4 * li + 3] = 0.0f;
    bmax4[4 * li + 3] = 0.0f;
  }
  if (L < 2) return;
  // Post-order over internal nodes (children before parents).
  std::vector<int> post;
  post.reserve(L);
  std::vector<std::pair<int, int>> st{{0, 0}};
  while (!st.empty()) {
    auto& [node, state] = st.back();
    if (node >= leaf0) { st.pop_back(); continue; }
    if (state == 0) { state = 1; st.push_back({(int)left[node], 0}); }
    else if (state == 1) { state = 2; st.push_back({(int)right[node], 0}); }
    else { post.push_back(node); st.pop_back(); }
  }
  for (int node : post) {
    const int l = (int)left[node], r = (int)right[node];
    const float* cl = &com4[4 * l];
    const float* cr = &com4[4 * r];
    const float m = cl[3] + cr[3];
    for (int k = 0; k < 3; ++k) {
      com4[4 * node + k] = m > 0.0f ? (cl[k] * cl[3] + cr[k] * cr[3]) / m : 0.0f;
      bmin4[4 * node + k] = std::min(bmin4[4 * l + k], bmin4[4 * r + k]);
      bmax4[4 * node + k] = std::max(bmax4[4 * l + k], bmax4[4 * r + k]);
    }
    com4[4 * node + 3] = m;
    bmin4[4 * node + 3] = 0.0f;
    bmax4[4 * node + 3] = 0.0f;
  }
}
// cs_gravity_bh, bh_gravity.wgsl:338-394: per-particle stack walk in sorted space, written to
// acc4[order[t]]. Returns the number of dropped pushes (the reference's silent MAX_STACK guard).
int orc_gravity_bh32(const float* sb4, int n, int K, int L, const uint32_t* left, const uint32_t* right,
                     const float* com4, const float* bmin4, const float* bmax4, const uint32_t* order, float theta,
                     float soft2, float G, float* acc4) {
  const uint32_t leaf0 = (uint32_t)(L - 1);
  int dropped = 0;
  for (int t = 0; t < n; ++t) {
    const float* pi = &sb4[4 * t];
    float a[3] = {0, 0, 0};
    uint32_t stack[64];
    int sp = 0;
    stack[sp++] = 0u;
    while (sp > 0) {
      const uint32_t ni = stack[--sp];
      if (ni >= leaf0) {
        const int c = (int)(ni - leaf0), s0 = c * K, s1 = std::min(s0 + K, n);
        for (int s = s0; s < s1; ++s) {
          if (s == t) continue;
          const float* bj = &sb4[4 * s];
          const float d[3] = {bj[0] - pi[0], bj[1] - pi[1], bj[2] - pi[2]};
          const float r2 = ((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]) + soft2;
          const float g = G * bj[3] / (r2 * std::sqrt(r2));
          for (int k = 0; k < 3; ++k) a[k] = a[k] + d[k] * g;
        }
        continue;
      }
      const float* cm = &com4[4 * ni];
      const float* bl = &bmin4[4 * ni];
      const float* bh = &bmax4[4 * ni];
      const float d[3] = {cm[0] - pi[0], cm[1] - pi[1], cm[2] - pi[2]};
      const float r2 = ((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]) + soft2;
      const float dist = std::sqrt(r2);
      const float e[3] = {bh[0] - bl[0], bh[1] - bl[1], bh[2] - bl[2]};
      const float size = std::sqrt((e[0] * e[0] + e[1] * e[1]) + e[2] * e[2]);
      const float cd[3] = {0.5f * (bl[0] + bh[0]) - cm[0], 0.5f * (bl[1] + bh[1]) - cm[1], 0.5f * (bl[2] + bh[2]) - cm[2]};
      const float delta = std::sqrt((cd[0] * cd[0] + cd[1] * cd[1]) + cd[2] * cd[2]);
      if (dist >= size / theta + delta) {
        const float g = G * cm[3] / (r2 * dist);
        for (int k = 0; k < 3; ++k) a[k] = a[k] + d[k] * g;
        continue;
      }
      if (sp + 2 <= 64) {
        stack[sp++] = left[ni];
        stack[sp++] = right[ni];
      } else {
        ++dropped;
      }
    }
    for (int k = 0; k < 3; ++k) acc4[4 * order[t] + k] = a[k];
    acc4[4 * order[t] + 3] = 0.0f;
  }
  return dropped;
}
// Softened direct sum in f32 (the leaf form r2·sqrt(r2), bh_gravity.wgsl:365-366).
void orc_gravity_direct32(const float* b4, int n, float soft2, float G, float* acc4) {
  for (int i = 0; i < n; ++i) {
    float a[3] = {0, 0, 0};
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const float d[3] = {b4[4 * j] - b4[4 * i], b4[4 * j + 1] - b4[4 * i + 1], b4[4 * j + 2] - b4[4 * i + 2]};
      const float r2 = ((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]) + soft2;
      const float g = G * b4[4 * j + 3] / (r2 * std::sqrt(r2));
      for (int k = 0; k < 3; ++k) a[k] = a[k] + d[k] * g;
    }
    for (int k = 0; k < 3; ++k) acc4[4 * i + k] = a[k];
    acc4[4 * i + 3] = 0.0f;
  }
}
// f64 softened direct sum on a subset of targets (gpu-bh-verify main.rs:140-158; bhtree.rs:119-131).
void orc_gravity_direct64(const double* pos3, const double* mass, int n, const int* targets, int nt, double soft,
                          double G, double* acc3, int nthreads) {
  const double s2 = soft * soft;
#pragma omp parallel for schedule(dynamic, 16) num_threads(std::max(nthreads, 1))
  for (int q = 0; q < nt; ++q) {
    const int i = targets ? targets[q] : q;
    double a[3] = {0, 0, 0};
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const double d[3] = {pos3[3 * j] - pos3[3 * i], pos3[3 * j + 1] - pos3[3 * i + 1], pos3[3 * j + 2] - pos3[3 * i + 2]};
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + s2;
      const double g = G * mass[j] / (r2 * std::sqrt(r2));
      for (int k = 0; k < 3; ++k) a[k] += d[k] * g;
    }
    for (int k = 0; k < 3; ++k) acc3[3 * q + k] = a[k];
  }
}
// f64 octree Barnes-Hut (bhtree.rs). Returns the node count (0 = brute-force mode below 1024 bodies).
int orc_bhtree64(const double* pos3, const double* mass, int n, double theta, double soft, double G, double* acc3,
                 int nthreads) {
  OctTree t;
  t.build(pos3, mass, n, theta, soft, G);
  t.accelerations(acc3, std::max(nthreads, 1));
  return (int)t.nodes.size();
}

// ---- neighbour sets and f32 SPH (sph_step.wgsl) ------------------------------------------------------
// Exact neighbour sets, ascending per particle. Returns the total number of entries written, or -1 if a
// particle has more than `cap` neighbours.
long long orc_neighbours32(const float* pos4, int n, uint32_t* counts, uint32_t* lists, int cap) {
  std::vector<std::vector<int>> nb;
  neighbour_sets32(pos4, n, nb);
  long long total = 0;
  for (int i = 0; i < n; ++i) {
    counts[i] = (uint32_t)nb[i].size();
    if ((int)nb[i].size() > cap) return -1;
    for (size_t k = 0; k < nb[i].size(); ++k) lists[(size_t)i * cap + k] = (uint32_t)nb[i][k];
    total += (long long)nb[i].size();
  }
  return total;
}
// cs_density, sph_step.wgsl:120-149: rho_i = m_i W(0,h_i) + Σ_{j in set} m_j W(r, h_ij).
void orc_density32(const float* pos4, const float* mass, int n, int kernel, float* rho) {
  std::vector<std::vector<int>> nb;
  neighbour_sets32(pos4, n, nb);
  for (int i = 0; i < n; ++i) {
    float r_i = mass[i] * kern_w32(kernel, 0.0f, pos4[4 * i + 3]);
    for (int j : nb[i]) {
      const float r = pair_r32(&pos4[4 * i], &pos4[4 * j]);
      const float hij = 0.5f * (pos4[4 * i + 3] + pos4[4 * j + 3]);
      r_i += mass[j] * kern_w32(kernel, r, hij);
    }
    rho[i] = r_i;
  }
}
// The SPH half of cs_forces, sph_step.wgsl:171-210 (pressure + Monaghan AV + du/dt), with P and c taken
// per particle (the reference recomputes the same pure function per pair, :188-190). out4 = (a.xyz, du/dt).
void orc_sph_forces32(const float* pos4, const float* vel4, const float* mass, const float* rho, const float* P,
                      const float* c, int n, float av_alpha, float av_beta, float r_min, int kernel, float* out4) {
  std::vector<std::vector<int>> nb;
  neighbour_sets32(pos4, n, nb);
  for (int i = 0; i < n; ++i) {
    float a[3] = {0, 0, 0}, de = 0.0f;
    const float* pi = &pos4[4 * i];
    const float* vi = &vel4[4 * i];
    for (int j : nb[i]) {
      const float* pj = &pos4[4 * j];
      const float* vj = &vel4[4 * j];
      const float dpos[3] = {pi[0] - pj[0], pi[1] - pj[1], pi[2] - pj[2]};
      const float r = std::sqrt((dpos[0] * dpos[0] + dpos[1] * dpos[1]) + dpos[2] * dpos[2]);
      const float hij = 0.5f * (pi[3] + pj[3]);
      if (!(r < hij && r > r_min)) continue;
      const float dvel[3] = {vi[0] - vj[0], vi[1] - vj[1], vi[2] - vj[2]};
      const float vr = (dvel[0] * dpos[0] + dvel[1] * dpos[1]) + dvel[2] * dpos[2];
      float pi_ij = 0.0f;
      if (vr < 0.0f) {
        const float mu = hij * vr / (r * r + 0.01f * hij * hij);
        const float c_bar = 0.5f * (c[i] + c[j]);
        const float rho_bar = 0.5f * (rho[i] + rho[j]);
        pi_ij = (-av_alpha * c_bar * mu + av_beta * mu * mu) / rho_bar;
      }
      const float coeff = P[i] / (rho[i] * rho[i]) + P[j] / (rho[j] * rho[j]) + pi_ij;
      const float dw = kern_dw32(kernel, r, hij);
      const float grad[3] = {dpos[0] / r * dw, dpos[1] / r * dw, dpos[2] / r * dw};
      for (int k = 0; k < 3; ++k) a[k] += grad[k] * (-coeff * mass[j]);
      de += 0.5f * mass[j] * coeff * ((dvel[0] * grad[0] + dvel[1] * grad[1]) + dvel[2] * grad[2]);
    }
    for (int k = 0; k < 3; ++k) out4[4 * i + k] = a[k];
    out4[4 * i + 3] = de;
  }
}

}  // extern "C"

// ---- smoothing-length solve (no reference counterpart: the reference keeps h fixed, hydrostatic.rs:59-61) --
// The density is the reference's symmetric sum (sph_step.wgsl:120-149: self term m_i W(0,h_i), pairs r < h_ij
// with h_ij = ½(h_i+h_j)); the solve drives f(h_i) = ρ_i(h) − m_i(η/h_i)³ to zero by Newton–Raphson (Price
// 2012, J. Comput. Phys. 231, §3.2.1), with ∂ρ_i/∂h_i = m_i ∂W(0,h_i)/∂h + Σ_j m_j ½ ∂W(r,h_ij)/∂h (h_ij moves
// by ½ dh_i). W = σ(h) f(q), σ = c/h³, q = r/h ⇒ ∂W/∂h = −(σ/h)(3f + q f'(q)), written from the formula.
// Every particle steps from the same iterate (Jacobi). A step is limited to ±20 % and to the box the
// neighbour-list skin allows around the smoothing length h0 the list was built with:
// h ≤ h0(1+skin)·0.999 and h ≥ h0/((1+skin)·1.001).
// orc_h_solve32 runs a fixed number of such steps in f32 and then the density pass at the final h (the
// product's sequence); orc_h_solve64 iterates in f64 until the iterate settles (the converged solution).
// ---------------------------------------------------------------------------------------------------
namespace {
template <typename T>
T kern_f(int kind, T q, T& fp) {  // f(q), f'(q) of the two kernels (support radius h)
  fp = T(0);
  if (q >= T(1)) return T(0);
  if (kind == 1) {
    const T t = T(1) - q, t3 = t * t * t;
    fp = T(-20) * q * t3;
    return t3 * t * (T(1) + T(4) * q);
  }
  if (q < T(0.5)) {
    fp = T(-12) * q + T(18) * q * q;
    return T(1) - T(6) * q * q + T(6) * q * q * q;
  }
  const T t = T(1) - q;
  fp = T(-6) * t * t;
  return T(2) * t * t * t;
}
template <typename T>
void kern_w_dwdh(int kind, T r, T h, T& w, T& dwdh) {
  const T c = kind == 1 ? T(21) / (T(2) * T(kPi)) : T(8) / T(kPi);
  const T q = r / h;
  T fp;
  const T f = kern_f<T>(kind, q, fp);
  const T sig = c / (h * h * h);
  w = sig * f;
  dwdh = -(sig / h) * (T(3) * f + q * fp);
}
template <typename T>
T h_newton_step(T h, T m, T rho, T drho, T eta, T h0, T skin, T& res) {
  const T rt = m * (eta * eta * eta) / (h * h * h);
  const T f = rho - rt;
  res = std::fabs(f) / std::max(rho, T(1e-30));
  const T fp = drho + T(3) * rt / h;
  const T dh = std::fabs(fp) > T(0) ? -f / fp : T(0);
  T hn = h + dh;
  if (!(hn == hn)) hn = h;
  hn = std::min(std::max(hn, T(0.8) * h), T(1.2) * h);
  hn = std::min(hn, h0 * (T(1) + skin) * T(0.999));
  hn = std::max(hn, h0 / ((T(1) + skin) * T(1.001)));
  return hn;
}
// Candidate pairs of the solve: everything within the largest h_ij the skin allows, exact test per pass.
template <typename T>
void hsolve_candidates(const T* pos, int stride, const T* h0, int n, T skin, std::vector<std::vector<int>>& cand) {
  T hm = T(0);
  for (int i = 0; i < n; ++i) hm = std::max(hm, h0[i]);
  const double reach = (double)hm * (1.0 + (double)skin) * (1.0 + 1.0e-6);
  CellList cl;
  cl.build(n, reach, [&](int i, double* p) { for (int k = 0; k < 3; ++k) p[k] = (double)pos[stride * i + k]; });
  cand.assign(n, {});
  for (int i = 0; i < n; ++i) {
    double p[3] = {(double)pos[stride * i], (double)pos[stride * i + 1], (double)pos[stride * i + 2]};
    cl.around(p, [&](int j) {
      if (j == i) return;
      double d2 = 0.0;
      for (int k = 0; k < 3; ++k) {
        const double d = (double)pos[stride * i + k] - (double)pos[stride * j + k];
        d2 += d * d;
      }
      if (d2 < reach * reach) cand[i].push_back(j);
    });
    std::sort(cand[i].begin(), cand[i].end());
  }
}
// ρ_i, ∂ρ_i/∂h_i at the current h over the candidates (f32: the product's single-rounded pair distance).
template <typename T>
void hsolve_sums(const T* pos, int stride, const T* mass, const T* h, int i, int kind,
                 const std::vector<int>& cand, T& rho, T& drho) {
  T w, dwdh;
  kern_w_dwdh<T>(kind, T(0), h[i], w, dwdh);
  rho = mass[i] * w;
  drho = mass[i] * dwdh;
  for (int j : cand) {
    const T dx = pos[stride * i] - pos[stride * j], dy = pos[stride * i + 1] - pos[stride * j + 1],
            dz = pos[stride * i + 2] - pos[stride * j + 2];
    const T r = std::sqrt((dx * dx + dy * dy) + dz * dz);
    const T hij = T(0.5) * (h[i] + h[j]);
    if (!(r < hij)) continue;
    kern_w_dwdh<T>(kind, r, hij, w, dwdh);
    rho += mass[j] * w;
    drho += mass[j] * T(0.5) * dwdh;
  }
}
}  // namespace

extern "C" {
// f32: `iters` Jacobi-Newton steps from h0 = pos4[.w], then the density at the final h. h_out, rho_out,
// res_out (relative residual |ρ − m(η/h)³|/ρ at the final h) per particle. Returns the largest residual.
float orc_h_solve32(const float* pos4, const float* mass, int n, int kernel, float eta, float skin, int iters,
                    float* h_out, float* rho_out, float* res_out) {
  std::vector<float> h0(n), h(n), hn(n);
  for (int i = 0; i < n; ++i) h0[i] = h[i] = pos4[4 * i + 3];
  std::vector<std::vector<int>> cand;
  hsolve_candidates<float>(pos4, 4, h0.data(), n, skin, cand);
  for (int it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
      float rho, drho, res;
      hsolve_sums<float>(pos4, 4, mass, h.data(), i, kernel, cand[i], rho, drho);
      hn[i] = h_newton_step<float>(h[i], mass[i], rho, drho, eta, h0[i], skin, res);
    }
    h.swap(hn);
  }
  float rmax = 0.0f;
  for (int i = 0; i < n; ++i) {
    float rho, drho;
    hsolve_sums<float>(pos4, 4, mass, h.data(), i, kernel, cand[i], rho, drho);
    const float rt = mass[i] * (eta * eta * eta) / (h[i] * h[i] * h[i]);
    const float res = std::fabs(rho - rt) / std::max(rho, 1e-30f);
    h_out[i] = h[i];
    rho_out[i] = rho;
    res_out[i] = res;
    rmax = std::max(rmax, res);
  }
  return rmax;
}
// f64: Jacobi-Newton from h0 until no smoothing length moves by more than step_tol (relative) in a step, or
// max_iter steps. The clamps make a fixed point of the limited iteration the solution (a particle held at
// its skin bound stops moving). Returns the steps taken (max_iter + 1 when it did not settle); h_out, rho_out
// and res_out (the relative residual at h_out) per particle.
int orc_h_solve64(const double* pos3, const double* h0, const double* mass, int n, int kernel, double eta,
                  double skin, double step_tol, int max_iter, double* h_out, double* rho_out, double* res_out) {
  std::vector<double> h(h0, h0 + n), hn(n);
  std::vector<std::vector<int>> cand;
  hsolve_candidates<double>(pos3, 3, h0, n, skin, cand);
  int it = 0;
  bool settled = false;
  for (; it <= max_iter; ++it) {
    double move = 0.0;
#pragma omp parallel for schedule(dynamic, 256) reduction(max : move)
    for (int i = 0; i < n; ++i) {
      double rho, drho;
      hsolve_sums<double>(pos3, 3, mass, h.data(), i, kernel, cand[i], rho, drho);
      hn[i] = h_newton_step<double>(h[i], mass[i], rho, drho, eta, h0[i], skin, res_out[i]);
      rho_out[i] = rho;
      move = std::max(move, std::fabs(hn[i] - h[i]) / h[i]);
    }
    if (move <= step_tol) {
      settled = true;
      break;
    }
    if (it < max_iter) h.swap(hn);
  }
  for (int i = 0; i < n; ++i) h_out[i] = h[i];
  return settled ? it : max_iter + 1;
}

// cs_relax, sph_step.wgsl:245-257, in f32: a_cf = ω²(x, y, 0); v = (v + (a + a_cf)·dt)·damp; x = x + v·dt.
// pos4/vel4 are updated in place (h and u untouched); acc4 = (a.xyz, du/dt) of the evaluation at x.
void orc_relax32(float* pos4, float* vel4, const float* acc4, int n, float dt, float damp, float omega) {
  const float w2 = omega * omega;
  for (int i = 0; i < n; ++i) {
    float* p = pos4 + 4 * i;
    float* v = vel4 + 4 * i;
    const float* a = acc4 + 4 * i;
    const float cf[3] = {w2 * p[0], w2 * p[1], 0.0f};
    for (int k = 0; k < 3; ++k) {
      v[k] = (v[k] + (a[k] + cf[k]) * dt) * damp;
      p[k] = p[k] + v[k] * dt;
    }
  }
}

// cs_signal, sph_step.wgsl:263-269: signal_i = h_i / max(c_i + |v_i|, floor) (the shader's floor is 1 m/s);
// the adaptive dt is cfl · min_i signal_i (the host reduction of impact-run main.rs:345-356).
void orc_signal32(const float* pos4, const float* vel4, const float* c, int n, float floor, float* sig) {
  for (int i = 0; i < n; ++i) {
    const float* v = vel4 + 4 * i;
    const float vmag = std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
    sig[i] = pos4[4 * i + 3] / std::max(c[i] + vmag, floor);
  }
}

// ---- f64 verifier physics (tools/sph-verify/src/main.rs:106-251) ----------------------------------
// cpu_forces: O(N²) density, direct gravity (pow form) and SPH/AV/du-dt with P,c per pair (1e-3 steps).
void orc_cpu_forces64(const double* pos3, const double* vel3, const double* h, const double* mass, const double* u,
                      const int* mat, int n, const double* eos10, double soft, double G, double av_alpha,
                      double av_beta, double du_floor, int kernel, double* rho, double* acc3, double* dudt) {
  auto W = [&](double r, double hh) { return kernel == 1 ? w_wendland64(r, hh) : w_cubic64_verify(r, hh); };
  auto dW = [&](double r, double hh) { return kernel == 1 ? dw_wendland64(r, hh) : dw_cubic64_verify(r, hh); };
  for (int i = 0; i < n; ++i) {
    rho[i] = mass[i] * W(0.0, h[i]);
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      const double d[3] = {pos3[3 * i] - pos3[3 * j], pos3[3 * i + 1] - pos3[3 * j + 1], pos3[3 * i + 2] - pos3[3 * j + 2]};
      const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      const double hij = 0.5 * (h[i] + h[j]);
      if (r < hij) rho[i] += mass[j] * W(r, hij);
    }
  }
  const double s2 = soft * soft;
  std::vector<double> P(n), C(n);
  for (int i = 0; i < n; ++i) {
    const double* e = eos10 + 10 * (size_t)mat[i];
    P[i] = pressure64(e, rho[i], u[i]);
    C[i] = sound_speed64_wgsl(e, rho[i], u[i], du_floor);
  }
  for (int i = 0; i < n; ++i) {
    double a[3] = {0, 0, 0}, de = 0.0;
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      const double d[3] = {pos3[3 * j] - pos3[3 * i], pos3[3 * j + 1] - pos3[3 * i + 1], pos3[3 * j + 2] - pos3[3 * i + 2]};
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const double g = G * mass[j] / std::pow(r2 + s2, 1.5);
      for (int k = 0; k < 3; ++k) a[k] += d[k] * g;
      const double r = std::sqrt(r2);
      const double hij = 0.5 * (h[i] + h[j]);
      if (r < hij && r > 1.0e-9) {
        const double dvel[3] = {vel3[3 * i] - vel3[3 * j], vel3[3 * i + 1] - vel3[3 * j + 1], vel3[3 * i + 2] - vel3[3 * j + 2]};
        const double dpos[3] = {-d[0], -d[1], -d[2]};
        const double vr = dvel[0] * dpos[0] + dvel[1] * dpos[1] + dvel[2] * dpos[2];
        double pi_ij = 0.0;
        if (vr < 0.0) {
          const double mu = hij * vr / (r * r + 0.01 * hij * hij);
          pi_ij = (-av_alpha * 0.5 * (C[i] + C[j]) * mu + av_beta * mu * mu) / (0.5 * (rho[i] + rho[j]));
        }
        const double coeff = P[i] / (rho[i] * rho[i]) + P[j] / (rho[j] * rho[j]) + pi_ij;
        const double dwdr = dW(r, hij);
        const double grad[3] = {dpos[0] / r * dwdr, dpos[1] / r * dwdr, dpos[2] / r * dwdr};
        for (int k = 0; k < 3; ++k) a[k] += grad[k] * (-coeff * mass[j]);
        de += 0.5 * mass[j] * coeff * (dvel[0] * grad[0] + dvel[1] * grad[1] + dvel[2] * grad[2]);
      }
    }
    for (int k = 0; k < 3; ++k) acc3[3 * i + k] = a[k];
    dudt[i] = de;
  }
}
// CpuState::step × steps (tools/sph-verify/src/main.rs:237-250), state updated in place.
void orc_cpu_kdk64(double* pos3, double* vel3, const double* h, const double* mass, double* u, const int* mat, int n,
                   const double* eos10, double soft, double G, double av_alpha, double av_beta, double du_floor,
                   int kernel, double dt, int steps) {
  std::vector<double> rho(n), a(3 * (size_t)n), du(n);
  for (int s = 0; s < steps; ++s) {
    orc_cpu_forces64(pos3, vel3, h, mass, u, mat, n, eos10, soft, G, av_alpha, av_beta, du_floor, kernel, rho.data(), a.data(), du.data());
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) vel3[3 * i + k] += a[3 * i + k] * 0.5 * dt;
      u[i] = std::max(u[i] + du[i] * 0.5 * dt, 0.0);
      for (int k = 0; k < 3; ++k) pos3[3 * i + k] += vel3[3 * i + k] * dt;
    }
    orc_cpu_forces64(pos3, vel3, h, mass, u, mat, n, eos10, soft, G, av_alpha, av_beta, du_floor, kernel, rho.data(), a.data(), du.data());
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) vel3[3 * i + k] += a[3 * i + k] * 0.5 * dt;
      u[i] = std::max(u[i] + du[i] * 0.5 * dt, 0.0);
    }
  }
}

// ---- HydroBody handle (the timed CPU path) --------------------------------------------------------
void* orc_hydro_new(int n, const double* pos3, const double* vel3, const double* mass, const double* u,
                    const double* h, const int* mat, const double* eos10, int n_eos, double softening, double G,
                    double theta, double av_alpha, double av_beta, int kernel) {
  Hydro* hb = new Hydro();
  hb->n = n;
  hb->n_eos = n_eos;
  hb->pos.assign(pos3, pos3 + 3 * (size_t)n);
  hb->vel.assign(vel3, vel3 + 3 * (size_t)n);
  hb->mass.assign(mass, mass + n);
  hb->u.assign(u, u + n);
  hb->h.assign(h, h + n);
  hb->mat.assign(mat, mat + n);
  hb->eos.assign(eos10, eos10 + 10 * (size_t)n_eos);
  hb->softening = softening;
  hb->G = G;
  hb->theta = theta;
  hb->av_alpha = av_alpha;
  hb->av_beta = av_beta;
  hb->kernel = kernel;
  hb->rho.assign(n, 0.0);
  return hb;
}
void orc_hydro_free(void* p) { delete static_cast<Hydro*>(p); }
void orc_hydro_step(void* p, double dt, int nthreads) { static_cast<Hydro*>(p)->step(dt, nthreads); }
void orc_hydro_density(void* p, int nthreads) { static_cast<Hydro*>(p)->compute_density(nthreads); }
void orc_hydro_forces(void* p, double* acc3, double* dudt, int nthreads) {
  Hydro* hb = static_cast<Hydro*>(p);
  std::vector<double> a, du;
  hb->forces(a, du, nthreads);
  std::memcpy(acc3, a.data(), sizeof(double) * a.size());
  std::memcpy(dudt, du.data(), sizeof(double) * du.size());
}
void orc_hydro_eval_sampled(void* p, int stride, double* t) { static_cast<Hydro*>(p)->eval_sampled(std::max(stride, 1), t); }
double orc_hydro_courant_dt(void* p, double cfl, double sig_floor) { return static_cast<Hydro*>(p)->courant_dt(cfl, sig_floor); }
void orc_hydro_get(void* p, double* pos3, double* vel3, double* u, double* rho) {
  Hydro* hb = static_cast<Hydro*>(p);
  if (pos3) std::memcpy(pos3, hb->pos.data(), sizeof(double) * hb->pos.size());
  if (vel3) std::memcpy(vel3, hb->vel.data(), sizeof(double) * hb->vel.size());
  if (u) std::memcpy(u, hb->u.data(), sizeof(double) * hb->u.size());
  if (rho) std::memcpy(rho, hb->rho.data(), sizeof(double) * hb->rho.size());
}
int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ---- conservation sums (gpu_sph.rs:628-649; tools/impact-run/src/main.rs:195-205,528-536) ----------
// out[0..2] = KE, IE, PE (PE O(N²) softened, skipped when with_pe == 0); out[3..5] = linear momentum;
// out[6..8] = angular momentum about the origin.
void orc_conservation64(const double* pos3, const double* vel3, const double* mass, const double* u, int n,
                        double soft, double G, int with_pe, double* out) {
  double ke = 0, ie = 0, pe = 0, p[3] = {0, 0, 0}, L[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i) {
    const double* x = pos3 + 3 * i;
    const double* v = vel3 + 3 * i;
    ke += 0.5 * mass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    ie += mass[i] * u[i];
    for (int k = 0; k < 3; ++k) p[k] += mass[i] * v[k];
    L[0] += mass[i] * (x[1] * v[2] - x[2] * v[1]);
    L[1] += mass[i] * (x[2] * v[0] - x[0] * v[2]);
    L[2] += mass[i] * (x[0] * v[1] - x[1] * v[0]);
  }
  if (with_pe) {
    const double s2 = soft * soft;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) {
        const double d[3] = {pos3[3 * i] - pos3[3 * j], pos3[3 * i + 1] - pos3[3 * j + 1], pos3[3 * i + 2] - pos3[3 * j + 2]};
        pe -= G * mass[i] * mass[j] / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + s2);
      }
  }
  out[0] = ke; out[1] = ie; out[2] = pe;
  for (int k = 0; k < 3; ++k) { out[3 + k] = p[k]; out[6 + k] = L[k]; }
}

// ---- granular contact (shaders/particle_step.wgsl:140-211 contact_accel, :273-336 cs_forces, :477-530
// cs_integrate; the ground scene's terrain, drag, cooling and settle counter in orc_dem_ground_step32) -------
// params: [c_stiffness, c_normal_damp, c_friction, c_tangent_damp, c_cohesion, dt, gx, gy, gz]
// accum16 per grain: force.xyz, headroom, s_diag.xyz, 0, s_off.xyz (xy, xz, yz), 0, sv_nbr.xyz, 0
static const float kDemTheta = 0.70f;                       // particle_step.wgsl:125
static const float kDemCohRange = 0.15f;                    // particle_step.wgsl:163
static void dem_contact32(const float* pi, const float* vi, float ri, const float* pj, const float* vj, float rj,
                          const float* prm, float* acc) {
  const float d[3] = {pi[0] - pj[0], pi[1] - pj[1], pi[2] - pj[2]};
  const float dist = std::sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
  const float touch = ri + rj;
  if (dist >= touch + kDemCohRange || dist < 1.0e-9f) return;
  const float nrm[3] = {d[0] / dist, d[1] / dist, d[2] / dist};
  const float overlap = touch - dist;
  const float vr[3] = {vi[0] - vj[0], vi[1] - vj[1], vi[2] - vj[2]};
  const float v_n = (vr[0] * nrm[0] + vr[1] * nrm[1]) + vr[2] * nrm[2];
  const float f_rep = prm[0] * std::max(overlap, 0.0f);
  const float sep = std::max(-overlap, 0.0f);
  const float f_coh = prm[4] * std::min(std::max(1.0f - sep / kDemCohRange, 0.0f), 1.0f);
  const float normal_load = f_rep + f_coh;
  const float vt[3] = {vr[0] - nrm[0] * v_n, vr[1] - nrm[1] * v_n, vr[2] - nrm[2] * v_n};
  const float vt_mag = std::sqrt((vt[0] * vt[0] + vt[1] * vt[1]) + vt[2] * vt[2]);
  float at[3] = {0, 0, 0};
  if (vt_mag > 1.0e-9f) {
    const float mag = std::min(std::min(prm[3] * vt_mag, prm[2] * normal_load), vt_mag / prm[5]);
    for (int k = 0; k < 3; ++k) at[k] = -(vt[k] / vt_mag) * mag;
  }
  for (int k = 0; k < 3; ++k) acc[k] += nrm[k] * (f_rep - f_coh) + at[k];
  if (overlap > 0.0f) {
    const float dt = prm[5];
    const float g = kDemTheta * kDemTheta * dt * dt * prm[0] + kDemTheta * dt * prm[1];
    acc[4] += g * nrm[0] * nrm[0];
    acc[5] += g * nrm[1] * nrm[1];
    acc[6] += g * nrm[2] * nrm[2];
    acc[8] += g * (nrm[0] * nrm[1]);
    acc[9] += g * (nrm[0] * nrm[2]);
    acc[10] += g * (nrm[1] * nrm[2]);
    const float ndv = (nrm[0] * vj[0] + nrm[1] * vj[1]) + nrm[2] * vj[2];
    for (int k = 0; k < 3; ++k) acc[12 + k] += g * ndv * nrm[k];
  }
}
void orc_dem_contacts32(const float* pos3, const float* vel3, const float* radius, int n, const float* prm,
                        float* accum16) {
  for (int i = 0; i < n; ++i) {
    float* acc = accum16 + 16 * (size_t)i;
    for (int k = 0; k < 16; ++k) acc[k] = 0.0f;
    acc[3] = 1.0e30f;
    for (int j = 0; j < n; ++j)
      if (j != i) dem_contact32(&pos3[3 * i], &vel3[3 * i], radius[i], &pos3[3 * j], &vel3[3 * j], radius[j], prm, acc);
  }
}
// cs_integrate's directional trapezoidal solve (I+S)v' = v − ρSv + (1/θ)Σ S_c v_j + dt·a; x += dt(v+v')/2.
void orc_dem_integrate32(float* pos3, float* vel3, const float* accum16, int n, const float* prm) {
  const float rho_t = (1.0f - kDemTheta) / kDemTheta, dt = prm[5];
  for (int i = 0; i < n; ++i) {
    const float* a = accum16 + 16 * (size_t)i;
    float* v = vel3 + 3 * i;
    const float acc[3] = {prm[6] + a[0], prm[7] + a[1], prm[8] + a[2]};
    const float sdx = a[4], sdy = a[5], sdz = a[6], sxy = a[8], sxz = a[9], syz = a[10];
    const float sv[3] = {sdx * v[0] + sxy * v[1] + sxz * v[2], sxy * v[0] + sdy * v[1] + syz * v[2],
                         sxz * v[0] + syz * v[1] + sdz * v[2]};
    float rhs[3];
    for (int k = 0; k < 3; ++k) rhs[k] = v[k] - rho_t * sv[k] + (1.0f / kDemTheta) * a[12 + k] + acc[k] * dt;
    const float m00 = 1.0f + sdx, m11 = 1.0f + sdy, m22 = 1.0f + sdz, m01 = sxy, m02 = sxz, m12 = syz;
    const float c00 = m11 * m22 - m12 * m12, c01 = m02 * m12 - m01 * m22, c02 = m01 * m12 - m02 * m11;
    const float c11 = m00 * m22 - m02 * m02, c12 = m01 * m02 - m00 * m12, c22 = m00 * m11 - m01 * m01;
    const float inv_det = 1.0f / (m00 * c00 + m01 * c01 + m02 * c02);
    const float vn[3] = {(c00 * rhs[0] + c01 * rhs[1] + c02 * rhs[2]) * inv_det,
                         (c01 * rhs[0] + c11 * rhs[1] + c12 * rhs[2]) * inv_det,
                         (c02 * rhs[0] + c12 * rhs[1] + c22 * rhs[2]) * inv_det};
    for (int k = 0; k < 3; ++k) {
      pos3[3 * i + k] = pos3[3 * i + k] + (v[k] + vn[k]) * (0.5f * dt);
      v[k] = vn[k];
    }
  }
}

}  // extern "C"

namespace {

// ---------------------------------------------------------------------------------------------------
// Learned smoothing-length MLP (no reference counterpart): 8 → 64 → 64 → 1 with GELU, the FP64 statement of
// the product's BF16-operand / FP32-accumulate kernels. Parameter block (floats):
//   W1[8][64] b1[64] W2[64][64] b2[64] W3[64] b3 | x_mean[8] x_scale[8] y_mean y_scale
// (W[i][o] row-major by input). x' = (x − x_mean)·x_scale; z1 = x'W1 + b1; a1 = gelu(z1); z2 = a1W2 + b2;
// a2 = gelu(z2); y = a2·W3 + b3; the output is y·y_scale + y_mean. With `bf16` set, every tensor-core operand
// is rounded to bfloat16 where the kernels round it: W1, W2, W3, x', a1 (forward); and in the backward pass
// dz2 (for both dW2 and da1) and dz1 (for dW1). Gradients are of the mean squared error on the normalised
// target (t − y_mean)/y_scale with respect to the first 4801 (trainable) parameters, rounding treated as
// the identity (straight-through).
// ---------------------------------------------------------------------------------------------------
constexpr int kMlpIn = 8, kMlpH = 64;
constexpr int kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpIn * kMlpH, kMlpW2 = kMlpB1 + kMlpH, kMlpB2 = kMlpW2 + kMlpH * kMlpH,
              kMlpW3 = kMlpB2 + kMlpH, kMlpB3 = kMlpW3 + kMlpH, kMlpTrain = kMlpB3 + 1, kMlpXm = kMlpTrain,
              kMlpXs = kMlpXm + kMlpIn, kMlpYm = kMlpXs + kMlpIn, kMlpYs = kMlpYm + 1, kMlpTotal = kMlpYs + 1;

double bf16_round(double v) {
  // to float, then to the nearest bfloat16 (ties to even), as __float2bfloat16_rn does on a float
  float f = (float)v;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u = (u + 0x7fffu + ((u >> 16) & 1u)) & 0xffff0000u;
  std::memcpy(&f, &u, 4);
  return (double)f;
}
double gelu(double z) { return 0.5 * z * (1.0 + std::erf(z / std::sqrt(2.0))); }
double gelu_d(double z) {
  return 0.5 * (1.0 + std::erf(z / std::sqrt(2.0))) + z * std::exp(-0.5 * z * z) / std::sqrt(2.0 * kPi);
}

struct MlpFwd {
  double x[kMlpIn], z1[kMlpH], a1[kMlpH], z2[kMlpH], a2[kMlpH], y;
};

void mlp_forward1(const float* P, const float* xin, bool bf, MlpFwd& f) {
  auto R = [&](double v) { return bf ? bf16_round(v) : v; };
  for (int i = 0; i < kMlpIn; ++i) f.x[i] = R(((double)xin[i] - P[kMlpXm + i]) * P[kMlpXs + i]);
  for (int o = 0; o < kMlpH; ++o) {
    double z = 0.0;
    for (int i = 0; i < kMlpIn; ++i) z += f.x[i] * R(P[kMlpW1 + i * kMlpH + o]);
    f.z1[o] = z + P[kMlpB1 + o];
    f.a1[o] = R(gelu(f.z1[o]));
  }
  for (int o = 0; o < kMlpH; ++o) {
    double z = 0.0;
    for (int i = 0; i < kMlpH; ++i) z += f.a1[i] * R(P[kMlpW2 + i * kMlpH + o]);
    f.z2[o] = z + P[kMlpB2 + o];
    f.a2[o] = gelu(f.z2[o]);
  }
  double y = 0.0;
  for (int i = 0; i < kMlpH; ++i) y += f.a2[i] * R(P[kMlpW3 + i]);
  f.y = y + P[kMlpB3];
}

}  // namespace

extern "C" {

int orc_mlp_param_count(int trainable) { return trainable ? kMlpTrain : kMlpTotal; }

// Δlog h proposals (de-normalised network outputs) for n feature rows x[n][8].
void orc_mlp_forward(const float* P, const float* x, int n, int bf, double* out) {
  for (int s = 0; s < n; ++s) {
    MlpFwd f;
    mlp_forward1(P, x + (size_t)s * kMlpIn, bf != 0, f);
    out[s] = f.y * P[kMlpYs] + P[kMlpYm];
  }
}

// Mean-squared-error loss on the normalised targets and its gradient w.r.t. the trainable parameters.
double orc_mlp_grad(const float* P, const float* x, const float* t, int n, int bf, double* grad) {
  const bool B = bf != 0;
  auto R = [&](double v) { return B ? bf16_round(v) : v; };
  std::fill(grad, grad + kMlpTrain, 0.0);
  double loss = 0.0;
  double w2[kMlpH * kMlpH], w3[kMlpH];
  for (int k = 0; k < kMlpH * kMlpH; ++k) w2[k] = R(P[kMlpW2 + k]);
  for (int k = 0; k < kMlpH; ++k) w3[k] = R(P[kMlpW3 + k]);
  for (int s = 0; s < n; ++s) {
    MlpFwd f;
    mlp_forward1(P, x + (size_t)s * kMlpIn, B, f);
    const double tn = ((double)t[s] - P[kMlpYm]) / P[kMlpYs];
    const double e = f.y - tn;
    loss += e * e;
    const double dy = 2.0 * e / n;
    grad[kMlpB3] += dy;
    double dz2[kMlpH], dz2r[kMlpH];
    for (int j = 0; j < kMlpH; ++j) {
      grad[kMlpW3 + j] += dy * f.a2[j];
      dz2[j] = dy * w3[j] * gelu_d(f.z2[j]);
      dz2r[j] = R(dz2[j]);
      grad[kMlpB2 + j] += dz2[j];
    }
    for (int i = 0; i < kMlpH; ++i)
      for (int j = 0; j < kMlpH; ++j) grad[kMlpW2 + i * kMlpH + j] += f.a1[i] * dz2r[j];
    for (int i = 0; i < kMlpH; ++i) {
      double da1 = 0.0;
      for (int j = 0; j < kMlpH; ++j) da1 += dz2r[j] * w2[i * kMlpH + j];
      const double dz1 = da1 * gelu_d(f.z1[i]);
      grad[kMlpB1 + i] += dz1;
      const double dz1r = R(dz1);
      for (int k = 0; k < kMlpIn; ++k) grad[kMlpW1 + k * kMlpH + i] += f.x[k] * dz1r;
    }
  }
  return loss / n;
}

}  // extern "C"

namespace {

// ---------------------------------------------------------------------------------------------------
// Disk measurement and the Moon candidate, in the reference's two forms:
//   variant 0: tools/impact-run/src/main.rs:732-878 (`measure`, `moon_candidate`) with `sum_oi` (:195),
//              `com` (:207) and `perigee` (:232);
//   variant 1: crates/engine/src/gpu_sph.rs:399-469 (`disk_stats_json`) with accretion.rs:73-160
//              (`find_clumps`) and orbit.rs:91-116 (`is_bound`, `perigee`).
// Provenance decides target vs impactor (prov 0 = the target; the tool's index test i < n_earth agrees with
// it for the tool's particle layout). The union-find partition does not depend on the pair order, so the
// tool's O(k²) loop stands in for the engine's grid pairs.
// ---------------------------------------------------------------------------------------------------
double sum_oi(std::vector<double>& t) {
  std::sort(t.begin(), t.end(), [](double a, double b) { return std::fabs(a) < std::fabs(b); });
  double s = 0.0, c = 0.0;
  for (double x : t) {
    const double y = x - c, z = s + y;
    c = (z - s) - y;
    s = z;
  }
  return s;
}

// 0 = escapes, 1 = disk (periapsis beyond the remnant), 2 = remnant
int classify(int variant, const double p[3], const double v[3], double mu, double r_rem) {
  const double r = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
  const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  const double h[3] = {p[1] * v[2] - p[2] * v[1], p[2] * v[0] - p[0] * v[2], p[0] * v[1] - p[1] * v[0]};
  const double h2 = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
  if (variant == 0) {  // main.rs:232-247: r = 0 is Some(0); energy >= 0 is None
    if (r == 0.0) return 2;
    const double energy = 0.5 * v2 - mu / r;
    if (energy >= 0.0) return 0;
    const double a = -mu / (2.0 * energy);
    const double e = std::sqrt(std::max(1.0 + 2.0 * energy * h2 / (mu * mu), 0.0));
    return a * (1.0 - e) > r_rem ? 1 : 2;
  }
  // orbit.rs:91-116: bound needs r > 0; the bound periapsis uses |h|·|h|
  if (!(r > 0.0 && 0.5 * v2 - mu / r < 0.0)) return 0;
  const double energy = 0.5 * v2 - mu / r;
  const double hl = std::sqrt(h2);
  const double e = std::sqrt(std::max(1.0 + 2.0 * energy * hl * hl / (mu * mu), 0.0));
  const double a = -mu / (2.0 * energy);
  return a * (1.0 - e) > r_rem ? 1 : 2;
}

}  // namespace

extern "C" {

// P48 particles (x y z h vx vy vz u mass mat rho prov) of one impact. The reference's constants are
// parameters: remnant_frac 0.85, link_factor 2, roche 2.44, and for variant 0 rho_fallback 2700 and a pair
// distance floor of 1 m, for variant 1 a pair softening of 1e4 m. out[16]: earth_frac, disk, e_disk, t_disk,
// e_rem, t_rem, e_esc, t_esc, r_remnant, m_remnant, clump_kg, clump_earth_frac, clump_n, n_clumps, n_bound, n_disk.
void orc_measure_disk(const float* P, int n, int variant, double G, double remnant_frac, double link_factor,
                      double roche, double rho_fallback, double pe_floor, double pe_soft, double* out) {
  auto f = [&](int i, int k) { return P[12 * (size_t)i + k]; };
  auto prov = [&](int i) { uint32_t u; std::memcpy(&u, &P[12 * (size_t)i + 11], 4); return u; };
  std::fill(out, out + 16, 0.0);
  if (n == 0) return;
  double m_total = 0.0, com[3] = {0.0, 0.0, 0.0}, vcom[3] = {0.0, 0.0, 0.0};
  if (variant == 0) {
    std::vector<double> mv(n), vx(n), vy(n), vz(n);
    for (int i = 0; i < n; ++i) {
      const double m = f(i, 8);
      mv[i] = m;
      vx[i] = (double)f(i, 4) * m;
      vy[i] = (double)f(i, 5) * m;
      vz[i] = (double)f(i, 6) * m;
    }
    m_total = sum_oi(mv);
    double mm = 0.0;
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) com[k] += (double)f(i, k) * (double)f(i, 8);
      mm += (double)f(i, 8);
    }
    for (int k = 0; k < 3; ++k) com[k] /= mm;
    vcom[0] = sum_oi(vx) / m_total;
    vcom[1] = sum_oi(vy) / m_total;
    vcom[2] = sum_oi(vz) / m_total;
  } else {
    for (int i = 0; i < n; ++i) m_total += (double)f(i, 8);
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) {
        com[k] += (double)f(i, k) * (double)f(i, 8);
        vcom[k] += (double)f(i, 4 + k) * (double)f(i, 8);
      }
    for (int k = 0; k < 3; ++k) {
      com[k] /= m_total;
      vcom[k] /= m_total;
    }
  }
  std::vector<std::pair<double, double>> radii(n);
  for (int i = 0; i < n; ++i) {
    const double d[3] = {(double)f(i, 0) - com[0], (double)f(i, 1) - com[1], (double)f(i, 2) - com[2]};
    radii[i] = {std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), (double)f(i, 8)};
  }
  std::stable_sort(radii.begin(), radii.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  double cum = 0.0, r_rem = radii.back().first, m_rem = m_total;
  for (const auto& rm : radii) {
    cum += rm.second;
    if (cum >= remnant_frac * m_total) {
      r_rem = rm.first;
      m_rem = cum;
      break;
    }
  }
  const double mu = G * m_rem;
  std::vector<double> cat[6];  // e_disk, t_disk, e_rem, t_rem, e_esc, t_esc
  std::vector<int> disk;
  for (int i = 0; i < n; ++i) {
    const double rp[3] = {(double)f(i, 0) - com[0], (double)f(i, 1) - com[1], (double)f(i, 2) - com[2]};
    const double rv[3] = {(double)f(i, 4) - vcom[0], (double)f(i, 5) - vcom[1], (double)f(i, 6) - vcom[2]};
    const int c = classify(variant, rp, rv, mu, r_rem);
    const int slot = (c == 1 ? 0 : c == 2 ? 2 : 4) + (prov(i) == 0u ? 0 : 1);
    cat[slot].push_back((double)f(i, 8));
    if (c == 1) disk.push_back(i);
  }
  double sums[6];
  for (int k = 0; k < 6; ++k) sums[k] = sum_oi(cat[k]);
  const double dk = sums[0] + sums[1];
  out[0] = dk > 0.0 ? 100.0 * sums[0] / dk : 0.0;
  out[1] = dk;
  for (int k = 0; k < 6; ++k) out[2 + k] = sums[k];
  out[8] = r_rem;
  out[9] = m_rem;
  out[15] = (double)disk.size();
  const int k = (int)disk.size();
  if (k < 2) return;
  // friends-of-friends over the disk particles, linking length = link_factor × mean smoothing length (of the
  // disk in variant 0, of every particle in variant 1)
  double mean_h = 0.0;
  if (variant == 0) {
    for (int i : disk) mean_h += (double)f(i, 3);
    mean_h /= k;
  } else {
    for (int i = 0; i < n; ++i) mean_h += (double)f(i, 3);
    mean_h /= n;
  }
  const double link = link_factor * mean_h, link2 = link * link;
  auto dist2 = [&](int ia, int ib) {
    double d2 = 0.0;
    for (int c = 0; c < 3; ++c) {
      // variant 0 subtracts in f32 and widens; variant 1 widens and subtracts in f64
      const double dd = variant == 0 ? (double)(f(ia, c) - f(ib, c)) : (double)f(ia, c) - (double)f(ib, c);
      d2 += dd * dd;
    }
    return d2;
  };
  std::vector<int> parent(k);
  std::iota(parent.begin(), parent.end(), 0);
  auto find = [&](int i) {
    int r = i;
    while (parent[r] != r) r = parent[r];
    while (parent[i] != r) {
      const int nx = parent[i];
      parent[i] = r;
      i = nx;
    }
    return r;
  };
#pragma omp parallel for schedule(dynamic, 64)
  for (int a = 0; a < k; ++a)
    for (int b = a + 1; b < k; ++b)
      if (dist2(disk[a], disk[b]) <= link2) {
#pragma omp critical(orc_fof)
        {
          const int ra = find(a), rb = find(b);
          if (ra != rb) parent[ra] = rb;
        }
      }
  std::vector<std::vector<int>> groups(k);
  for (int a = 0; a < k; ++a) groups[find(a)].push_back(disk[a]);
  const double rho_rem = m_rem / (4.0 / 3.0 * kPi * r_rem * r_rem * r_rem);
  double best_m = 0.0, best_e = 0.0;
  int best_n = 0, n_bound = 0, n_clumps = 0;
  for (const auto& mem : groups) {
    if (mem.size() < 2) continue;
    double m = 0.0, cv[3] = {0, 0, 0}, cp[3] = {0, 0, 0}, vol = 0.0;
    for (int i : mem) m += (double)f(i, 8);
    if (variant == 1 && m <= 0.0) continue;  // accretion.rs:121
    ++n_clumps;
    for (int i : mem) {
      for (int c = 0; c < 3; ++c) {
        cv[c] += (double)f(i, 4 + c) * (double)f(i, 8);
        cp[c] += (double)f(i, c) * (double)f(i, 8);
      }
      const double rho = variant == 0 ? (double)f(i, 10) : (double)std::max(f(i, 10), 1.0f);
      vol += (double)f(i, 8) / rho;
    }
    for (int c = 0; c < 3; ++c) {
      cv[c] /= m;
      cp[c] /= m;
    }
    const double rho_c = vol > 0.0 ? m / vol : rho_fallback;
    double ke = 0.0, pe = 0.0;
    for (int i : mem) {
      const double dv[3] = {(double)f(i, 4) - cv[0], (double)f(i, 5) - cv[1], (double)f(i, 6) - cv[2]};
      ke += 0.5 * (double)f(i, 8) * (dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    }
    const double s2 = pe_soft * pe_soft;
#pragma omp parallel for reduction(+ : pe) schedule(dynamic, 16) if (mem.size() > 512)
    for (size_t a = 0; a < mem.size(); ++a)
      for (size_t b = a + 1; b < mem.size(); ++b) {
        const double d2 = dist2(mem[a], mem[b]);
        const double r = variant == 0 ? std::max(std::sqrt(d2), pe_floor) : std::sqrt(d2 + s2);
        pe -= G * (double)f(mem[a], 8) * (double)f(mem[b], 8) / r;
      }
    const bool bound = ke + pe < 0.0;
    const double d_roche = roche * r_rem * std::cbrt(rho_rem / rho_c);
    const double dist = std::sqrt((cp[0] - com[0]) * (cp[0] - com[0]) + (cp[1] - com[1]) * (cp[1] - com[1]) +
                                  (cp[2] - com[2]) * (cp[2] - com[2]));
    if (bound) ++n_bound;
    if (bound && dist > d_roche && m > best_m) {
      best_m = m;
      best_e = 0.0;
      for (int i : mem)
        if (prov(i) == 0u) best_e += (double)f(i, 8);
      best_n = (int)mem.size();
    }
  }
  out[10] = best_m;
  out[11] = best_m > 0.0 ? 100.0 * best_e / best_m : 0.0;
  out[12] = best_n;
  out[13] = n_clumps;
  out[14] = n_bound;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------
// Relaxed-body assembly: gpu_sph.rs:260-293 (`body_bulk`) and :309-339 (`assemble_from_relaxed_n`).
// ---------------------------------------------------------------------------------------------------
static void orc_bulk_impl(const float* P, int n, uint32_t prov, double* out5) {
  auto f = [&](int i, int k) { return P[12 * (size_t)i + k]; };
  auto pv = [&](int i) { uint32_t u; std::memcpy(&u, &P[12 * (size_t)i + 11], 4); return u; };
  std::vector<int> ps;
  for (int i = 0; i < n; ++i)
    if (pv(i) == prov) ps.push_back(i);
  double m = 0.0;
  for (int i : ps) m += (double)f(i, 8);
  auto com = [&](const std::vector<int>& sel, double c[3]) {
    double mm = 0.0;
    for (int i : sel) mm += (double)f(i, 8);
    c[0] = c[1] = c[2] = 0.0;
    if (mm <= 0.0) return;
    for (int i : sel)
      for (int k = 0; k < 3; ++k) c[k] += (double)f(i, k) * (double)f(i, 8);
    for (int k = 0; k < 3; ++k) c[k] /= mm;
  };
  auto dist = [&](int i, const double c[3]) {
    const double d[3] = {(double)f(i, 0) - c[0], (double)f(i, 1) - c[1], (double)f(i, 2) - c[2]};
    return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  };
  auto bulk_radius = [&](const std::vector<int>& sel, const double c[3]) {
    double mm = 0.0;
    for (int i : sel) mm += (double)f(i, 8);
    std::vector<std::pair<double, double>> rr;
    for (int i : sel) rr.push_back({dist(i, c), (double)f(i, 8)});
    std::stable_sort(rr.begin(), rr.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    double cum = 0.0, r = 0.0;
    for (const auto& x : rr) {
      cum += x.second;
      r = x.first;
      if (cum >= 0.98 * mm) break;
    }
    return r;
  };
  double c[3];
  com(ps, c);
  double r = bulk_radius(ps, c);
  for (int it = 0; it < 2; ++it) {
    std::vector<int> keep;
    for (int i : ps)
      if (dist(i, c) <= 1.5 * r) keep.push_back(i);
    if (keep.empty()) break;
    com(keep, c);
    r = bulk_radius(keep, c);
  }
  out5[0] = c[0];
  out5[1] = c[1];
  out5[2] = c[2];
  out5[3] = m;
  out5[4] = r;
}

extern "C" {

void orc_body_bulk(const float* P, int n, uint32_t prov, double* out5) { orc_bulk_impl(P, n, prov, out5); }

// placements: np × {offset xyz, vel xyz, spin xyz}. out: room for n records; returns the kept count.
int orc_assemble(const float* P, int n, const double* pl, int np, float* out, float* softening, float* dt) {
  std::vector<double> coms((size_t)np * 3);
  for (int k = 0; k < np; ++k) {
    double b[5];
    orc_bulk_impl(P, n, (uint32_t)k, b);
    for (int j = 0; j < 3; ++j) coms[k * 3 + j] = b[j];
  }
  int m = 0;
  float min_h = INFINITY;
  for (int i = 0; i < n; ++i) {
    const float* p = P + 12 * (size_t)i;
    uint32_t prov;
    std::memcpy(&prov, &p[11], 4);
    if (prov >= (uint32_t)np) continue;
    const double* o = pl + 9 * prov;
    const double l[3] = {(double)p[0] - coms[prov * 3], (double)p[1] - coms[prov * 3 + 1],
                         (double)p[2] - coms[prov * 3 + 2]};
    const double q[3] = {l[0] + o[0], l[1] + o[1], l[2] + o[2]};
    const double* w = o + 6;
    const double v[3] = {o[3] + (w[1] * l[2] - l[1] * w[2]), o[4] + (w[2] * l[0] - l[2] * w[0]),
                         o[5] + (w[0] * l[1] - l[0] * w[1])};
    float* r = out + 12 * (size_t)m++;
    std::memcpy(r, p, 48);
    for (int k = 0; k < 3; ++k) {
      r[k] = (float)q[k];
      r[4 + k] = (float)v[k];
    }
    min_h = std::min(min_h, p[3]);
  }
  double vmax = 0.0;
  for (int k = 0; k < np; ++k) {
    const double* v = pl + 9 * k + 3;
    vmax = std::max(vmax, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
  }
  *softening = 0.25f * min_h;
  *dt = (float)(0.01 * (double)min_h / (20000.0 + vmax));
  return m;
}

}  // extern "C"

// ---- the ground scene: particle_step.wgsl:338-452 (terrain_top/_h/_surface, terrain_resolve), :282-336
// (headroom), :477-576 (cs_integrate with cooling, drag, terrain contact, settle counter, incandescence) -----
struct OrcGround {
  float cx, cy, cz, air_rho, drag_cd, specific_heat, cool_rate;
  const int* hf;
  int w, d;
};
static float orc_terrain_top(const OrcGround& g, int cx, int cz) {
  const int x = std::min(std::max(cx, 0), g.w - 1), z = std::min(std::max(cz, 0), g.d - 1);
  return ((float)g.hf[z * g.w + x] - g.cy) - 0.5f;
}
static float orc_mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
static void orc_terrain_surface(const OrcGround& g, float px, float pz, float s[3]) {
  const float vx = px + g.cx, vz = pz + g.cz;
  const int cx = (int)std::floor(vx), cz = (int)std::floor(vz);
  const float h00 = orc_terrain_top(g, cx, cz), h10 = orc_terrain_top(g, cx + 1, cz);
  const float h01 = orc_terrain_top(g, cx, cz + 1), h11 = orc_terrain_top(g, cx + 1, cz + 1);
  const float fx = vx - (float)cx, fz = vz - (float)cz;
  s[0] = orc_mix(orc_mix(h00, h10, fx), orc_mix(h01, h11, fx), fz);
  s[1] = orc_mix(h10 - h00, h11 - h01, fz);
  s[2] = orc_mix(h01 - h00, h11 - h10, fx);
}
static void orc_terrain_normal(const float s[3], float n[3]) {
  const float nx = -s[1], nz = -s[2];
  const float l = std::sqrt((nx * nx + 1.0f * 1.0f) + nz * nz);
  n[0] = nx / l;
  n[1] = 1.0f / l;
  n[2] = nz / l;
}

extern "C" {

// One substep of the ground scene for n grains (f32, as the shader). ground[7] = center xyz, air_rho, drag_cd,
// specific_heat, cool_rate; hf = w × d heights or null. rho = grain densities; u, resting, emission3 updated.
void orc_dem_ground_step32(float* pos3, float* vel3, const float* radius, const float* rho, float* u,
                           float* resting, float* emission3, int n, const float* prm, const float* ground,
                           const int* hf, int w, int d) {
  const OrcGround g{ground[0], ground[1], ground[2], ground[3], ground[4], ground[5], ground[6], hf, w, d};
  std::vector<float> acc((size_t)n * 16, 0.0f);
  for (int i = 0; i < n; ++i) {
    float* a = &acc[16 * (size_t)i];
    a[3] = 1.0e30f;
    float tn[3] = {0.0f, 1.0f, 0.0f};
    if (hf) {
      float s[3];
      orc_terrain_surface(g, pos3[3 * i], pos3[3 * i + 2], s);
      orc_terrain_normal(s, tn);
    }
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      dem_contact32(&pos3[3 * i], &vel3[3 * i], radius[i], &pos3[3 * j], &vel3[3 * j], radius[j], prm, a);
      if (hf) {
        const float dj[3] = {pos3[3 * j] - pos3[3 * i], pos3[3 * j + 1] - pos3[3 * i + 1],
                             pos3[3 * j + 2] - pos3[3 * i + 2]};
        if ((dj[0] * tn[0] + dj[1] * tn[1]) + dj[2] * tn[2] > 0.0f)
          a[3] = std::min(a[3], std::max(std::sqrt((dj[0] * dj[0] + dj[1] * dj[1]) + dj[2] * dj[2]) -
                                             (radius[i] + radius[j]), 0.0f));
      }
    }
  }
  const float rho_t = (1.0f - kDemTheta) / kDemTheta, dt = prm[5];
  for (int i = 0; i < n; ++i) {
    const float* a = &acc[16 * (size_t)i];
    float* v = vel3 + 3 * i;
    float* p = pos3 + 3 * i;
    const float u_amb = g.specific_heat * 300.0f;
    u[i] = u_amb + (u[i] - u_amb) * std::exp(-g.cool_rate * dt);
    float ax[3] = {prm[6] + a[0], prm[7] + a[1], prm[8] + a[2]};
    const float sp = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (g.air_rho > 0.0f && sp > 1.0e-9f) {
      const float s_grain = std::max(2.0f * radius[i], 1.0e-6f);
      const float a_drag = 0.5f * g.air_rho * sp * sp * g.drag_cd / (std::max(rho[i], 1.0e-6f) * s_grain);
      for (int k = 0; k < 3; ++k) ax[k] -= (a_drag / sp) * v[k];
    }
    const float sdx = a[4], sdy = a[5], sdz = a[6], sxy = a[8], sxz = a[9], syz = a[10];
    const float sv[3] = {sdx * v[0] + sxy * v[1] + sxz * v[2], sxy * v[0] + sdy * v[1] + syz * v[2],
                         sxz * v[0] + syz * v[1] + sdz * v[2]};
    float rhs[3];
    for (int k = 0; k < 3; ++k) rhs[k] = v[k] - rho_t * sv[k] + (1.0f / kDemTheta) * a[12 + k] + ax[k] * dt;
    const float m00 = 1.0f + sdx, m11 = 1.0f + sdy, m22 = 1.0f + sdz, m01 = sxy, m02 = sxz, m12 = syz;
    const float c00 = m11 * m22 - m12 * m12, c01 = m02 * m12 - m01 * m22, c02 = m01 * m12 - m02 * m11;
    const float c11 = m00 * m22 - m02 * m02, c12 = m01 * m02 - m00 * m12, c22 = m00 * m11 - m01 * m01;
    const float inv_det = 1.0f / (m00 * c00 + m01 * c01 + m02 * c02);
    float vn[3] = {(c00 * rhs[0] + c01 * rhs[1] + c02 * rhs[2]) * inv_det,
                   (c01 * rhs[0] + c11 * rhs[1] + c12 * rhs[2]) * inv_det,
                   (c02 * rhs[0] + c12 * rhs[1] + c22 * rhs[2]) * inv_det};
    float q[3];
    for (int k = 0; k < 3; ++k) q[k] = p[k] + (v[k] + vn[k]) * (0.5f * dt);
    float rest = 0.0f;
    if (hf) {
      float s[3];
      orc_terrain_surface(g, q[0], q[2], s);
      const float pen = s[0] - (q[1] - radius[i]);
      if (pen > 0.0f) {
        float nn[3];
        orc_terrain_normal(s, nn);
        const float vdn = vn[0] * nn[0] + vn[1] * nn[1] + vn[2] * nn[2];
        float jn = 0.0f;
        if (vdn < 0.0f) {
          jn = -vdn;
          for (int k = 0; k < 3; ++k) vn[k] += jn * nn[k];
        }
        const float vd = vn[0] * nn[0] + vn[1] * nn[1] + vn[2] * nn[2];
        const float t[3] = {vn[0] - vd * nn[0], vn[1] - vd * nn[1], vn[2] - vd * nn[2]};
        const float vt = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        if (vt > 1.0e-9f) {
          const float dv = std::min(prm[2] * jn, vt);
          for (int k = 0; k < 3; ++k) vn[k] -= (t[k] / vt) * dv;
        }
        const float dp = std::min(std::min(pen, 0.01f), a[3]);
        for (int k = 0; k < 3; ++k) q[k] += dp * nn[k];
      }
      float s2[3];
      orc_terrain_surface(g, q[0], q[2], s2);
      rest = q[1] - radius[i] <= s2[0] + 0.1f ? resting[i] + 1.0f : 0.0f;
    }
    resting[i] = rest;
    for (int k = 0; k < 3; ++k) {
      p[k] = q[k];
      v[k] = vn[k];
    }
    const float temp = u[i] / std::max(g.specific_heat, 1.0f);
    float* e = emission3 + 3 * i;
    e[0] = e[1] = e[2] = 0.0f;
    if (temp > 800.0f) {
      const float x = temp - 800.0f;
      const float inten = std::min(std::max(x / 2200.0f, 0.0f), 4.0f);
      const float gg = std::min(std::max(x / 2200.0f, 0.0f), 1.0f);
      const float bb = std::min(std::max((temp - 2600.0f) / 2400.0f, 0.0f), 1.0f);
      e[0] = inten;
      e[1] = gg * inten;
      e[2] = bb * inten;
    }
  }
}

}  // extern "C"
