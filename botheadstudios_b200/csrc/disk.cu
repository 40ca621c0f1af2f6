// Disk measurement and the Moon candidate of one impact, on the device.
//
// The reference measures a finished impact on the host in two places: the impact-run tool
// (tools/impact-run/src/main.rs:732-878, `measure` + `moon_candidate`) and the engine's HUD statistics
// (crates/engine/src/gpu_sph.rs:399-469, `disk_stats_json` + accretion.rs:73-160 `find_clumps`). Both:
//   1. mass, centre of mass and bulk velocity of the impact;
//   2. the remnant radius: the smallest radius about the centre of mass enclosing 85 % of the mass (radius
//      sort + running sum);
//   3. each particle's two-body orbit about the remnant: escaping, remnant (periapsis inside it) or disk;
//   4. friends-of-friends over the disk particles with a linking length of twice the mean smoothing length
//      (the tool: an O(k²) pair loop; the engine: a cell grid), union-find;
//   5. per clump of two or more: mass, centre of mass and velocity, volume, internal kinetic energy and the
//      pairwise self-potential (O(s²)); bound when KE + PE < 0; outside the fluid Roche limit
//      2.44 R (ρ_remnant / ρ_clump)^(1/3); the Moon candidate is the heaviest bound clump outside it.
//
// Here every step is a kernel over the impact's particle range of the state (already contiguous per impact):
// deterministic two-pass f64 reductions; the radius sort is the tree's 8-bit LSD radix sort over the exact
// f64 bit patterns of the radii; the 85 % crossing is a block prefix over tile masses, then over the crossing
// tile's particles; classification writes per-block partials and an order-preserving compaction of the disk;
// the friends-of-friends search sorts the disk by a lexicographic cell key (cell edge just above the linking
// length, so every linked pair lies in the 3 × 3 column of z-runs around a particle), and one warp per
// particle scans its partners and unites linked pairs with a lock-free union-find (hooking the larger root
// under the smaller with atomicCAS, path halving; parent[i] <= i always, so every walk ends); clumps are
// contiguous after a radix sort by root; one block per clump sums its moments; the self-potential is split
// into 128 × 128 tile pairs of the clump's pair triangle, each summed in f64 by one block, then reduced per
// clump in a fixed order. The per-particle arithmetic that decides a classification (radii, periapsis, pair
// distances) is written with explicitly rounded operations in the reference's order; the sums differ from
// the reference's sequential ones only in association. Two host reads size the work: the disk count and the
// number of self-potential tile pairs.
#include <cstdint>
#include <cstring>

#include "sph_kernels.cuh"

namespace sphb {

struct DiskWork {
  int cap = 0;
  void* base = nullptr;
  unsigned long long* keys[2] = {nullptr, nullptr};
  unsigned* vals[2] = {nullptr, nullptr};
  unsigned* hist = nullptr;
  unsigned* tot = nullptr;
  double* part = nullptr;   // [kDmBlocks][kDmVals] block partials
  double* tsum = nullptr;   // [tiles] mass of each radius-sorted tile
  double* scal = nullptr;   // [S_COUNT]
  unsigned* cnt = nullptr;  // [C_COUNT]
  unsigned* bcnt = nullptr; // [kDmBlocks] disk particles per block, then their output offsets
  unsigned char* cat = nullptr;  // [cap] category of each particle
  float4* pm = nullptr;                  // [cap] x, y, z, mass of the points whose radii are sorted
  float4* dpos[2] = {nullptr, nullptr};  // disk particles: x, y, z, h
  float4* dvel[2] = {nullptr, nullptr};  // vx, vy, vz, mass
  float2* drp[2] = {nullptr, nullptr};   // rho, prov bits
  unsigned* parent = nullptr;  // [cap] union-find forest over the cell-sorted disk
  unsigned* gcnt = nullptr;    // [cap] members per root
  uint4* clump = nullptr;      // [cap/2+1] first member, members, root, units
  unsigned long long* uoff = nullptr;  // [cap/2+2] first self-potential unit of each clump
  double* cstat = nullptr;     // [cap/2+1][8] mass, com xyz, volume, target mass, internal KE, Σ m m / r
  double* upe = nullptr;       // [upe_cap] unit sums Σ m_a m_b / r (grown on demand)
  unsigned long long upe_cap = 0;
  double* out = nullptr;       // [16]
  double* bb = nullptr;        // [16] body bulk: centre, radius, new centre, new mass, new radius + mass, mass
  double* place = nullptr;     // [kMaxPlacements][12] offset, vel, spin, centre of each source body
};

namespace {

// The 48-byte exchange record (SphParticle, gpu_sph.rs:28).
struct P48x {
  float px, py, pz, h, vx, vy, vz, u, mass;
  unsigned mat;
  float rho;
  unsigned prov;
};
static_assert(sizeof(P48x) == 48, "48-byte particle");

constexpr int kDmThreads = 256;
constexpr int kDmBlocks = 592;  // 4 × 148 SMs; block b reduces the b-th contiguous chunk of the impact
constexpr int kDmVals = 8;
constexpr int kPeRows = 128;    // particles per self-potential row
constexpr int kTile = 2048;     // radius-sorted tile of the crossing walk (the radix sort's tile)
constexpr unsigned kCellBias = 1u << 20, kCellMax = (1u << 21) - 1u;
constexpr int kUnionTries = 1 << 16;
constexpr unsigned long long kMaxUnits = 1ull << 28;  // self-potential tile pairs (2 GB of partial sums)
constexpr double kPiD = 3.14159265358979323846;
constexpr unsigned kMaxPlacements = 256;

enum { S_M = 0, S_COM = 1, S_VCOM = 4, S_RREM = 7, S_MREM = 8, S_LINK = 9, S_RHOREM = 10, S_CAT = 11, S_COUNT = 24 };
enum { C_NDISK = 0, C_NCLUMP = 1, C_SEL = 2, C_ERR = 3, C_UNITS64 = 4, C_MINH = 6, C_COUNT = 8 };  // u64 in 4-5
// body-bulk slots: the current centre and radius, the latest selection's centre and mass, its crossing radius
// and running mass, the mass of every particle of the body
enum { BB_C = 0, BB_R = 3, BB_CN = 4, BB_MN = 7, BB_RN = 8, BB_M = 10 };

// Sum kDmVals doubles over the block in a fixed order (warp trees, then warps in order). Thread 0 gets them.
__device__ __forceinline__ void block_sum(double* v, double (*s)[kDmVals]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kDmVals; ++k) {
    const double x = warp_sum(v[k]);
    if (lane == 0) s[w][k] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < kDmVals; ++k) {
      double a = 0.0;
      for (int j = 0; j < nw; ++j) a += s[j][k];
      v[k] = a;
    }
  }
  __syncthreads();
}

// Sum of nb partials of value k over a warp, fixed order.
__device__ __forceinline__ double warp_sum_column(const double* part, int nb, int k) {
  double a = 0.0;
  for (int b = (int)(threadIdx.x & 31); b < nb; b += 32) a += part[b * kDmVals + k];
  return warp_sum(a);
}

__device__ __forceinline__ double dsq3(double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// The particle's position as the 48-byte exchange record holds it (f32 of the f64 master).
__device__ __forceinline__ float3 pos_f32(const State& st, unsigned t) {
  return make_float3((float)st.x[t], (float)st.y[t], (float)st.z[t]);
}

// ---- 1. mass, centre of mass, bulk velocity ----------------------------------------------------------
__global__ void __launch_bounds__(kDmThreads) k_dm_moments(State st, unsigned off, unsigned m, unsigned chunk,
                                                           double* __restrict__ part, float4* __restrict__ pm) {
  __shared__ double s[kDmThreads / 32][kDmVals];
  double a[kDmVals] = {0, 0, 0, 0, 0, 0, 0, 0};
  const unsigned b0 = blockIdx.x * chunk, b1 = min(m, b0 + chunk);
  for (unsigned i = b0 + threadIdx.x; i < b1; i += kDmThreads) {
    const unsigned t = off + i;
    const float3 p = pos_f32(st, t);
    const float4 v = st.vel_u[t];
    const double mm = st.mass[t];
    pm[i] = make_float4(p.x, p.y, p.z, st.mass[t]);  // positions and masses for the remnant radius
    a[0] += mm;
    a[1] += (double)p.x * mm;  // f32 × f32 products are exact in f64
    a[2] += (double)p.y * mm;
    a[3] += (double)p.z * mm;
    a[4] += (double)v.x * mm;
    a[5] += (double)v.y * mm;
    a[6] += (double)v.z * mm;
    a[7] += (double)st.pos_h[t].w;
  }
  block_sum(a, s);
  if (threadIdx.x == 0)
    for (int k = 0; k < kDmVals; ++k) part[blockIdx.x * kDmVals + k] = a[k];
}

__global__ void k_dm_moments_final(const double* __restrict__ part, int nb, double* __restrict__ scal) {
  __shared__ double t[kDmVals];
  const int w = threadIdx.x >> 5;
  const double v = warp_sum_column(part, nb, w);
  if ((threadIdx.x & 31) == 0) t[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    const double M = t[0];
    scal[S_M] = M;
    for (int k = 0; k < 3; ++k) {
      scal[S_COM + k] = t[1 + k] / M;
      scal[S_VCOM + k] = t[4 + k] / M;
    }
    scal[S_CAT + 7] = t[7];  // Σ h over every particle (the engine's linking length)
  }
}

// ---- 2. radii about a centre, their sort, the mass-fraction crossing ------------------------------------
// Shared by the remnant radius (85 % of an impact's mass) and the bulk radius of a body (98 %). pm holds the
// points' f32 positions and masses; the radius is the exact f64 distance from the centre.
__global__ void k_dm_radius(const float4* __restrict__ pm, unsigned m, const double* __restrict__ centre,
                            unsigned long long* __restrict__ keys, unsigned* __restrict__ vals) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const float4 p = pm[i];
  const double dx = __dsub_rn((double)p.x, centre[0]), dy = __dsub_rn((double)p.y, centre[1]),
               dz = __dsub_rn((double)p.z, centre[2]);
  const double r = __dsqrt_rn(dsq3(dx, dy, dz));
  keys[i] = (unsigned long long)__double_as_longlong(r);  // r >= 0: the bit pattern orders like the value
  vals[i] = i;
}

__global__ void __launch_bounds__(kDmThreads) k_dm_tile_mass(const float4* __restrict__ pm, unsigned m,
                                                             const unsigned* __restrict__ order,
                                                             double* __restrict__ tsum) {
  __shared__ double s[kDmThreads / 32][kDmVals];
  double a[kDmVals] = {0, 0, 0, 0, 0, 0, 0, 0};
  const unsigned b0 = blockIdx.x * kTile, b1 = min(m, b0 + kTile);
  for (unsigned i = b0 + threadIdx.x; i < b1; i += kDmThreads) a[0] += (double)pm[order[i]].w;
  block_sum(a, s);
  if (threadIdx.x == 0) tsum[blockIdx.x] = a[0];
}

// Block-wide exclusive scan of one double per thread (fixed association). Returns the block total in `total`.
__device__ __forceinline__ double block_exclusive_scan_d(double v, double* s_warp, double& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  double incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double t = __shfl_up_sync(SPH_FULL_MASK, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[w] = incl;
  __syncthreads();
  if (w == 0) {
    const double x = lane < nw ? s_warp[lane] : 0.0;
    double xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double t = __shfl_up_sync(SPH_FULL_MASK, xi, o);
      if (lane >= o) xi += t;
    }
    if (lane < nw) s_warp[lane] = xi - x;
    if (lane == 31) s_warp[32] = xi;
  }
  __syncthreads();
  const double res = s_warp[w] + incl - v;
  total = s_warp[32];
  __syncthreads();
  return res;
}

// The mass-fraction crossing in radius order: a prefix over the tile masses finds the crossing tile, a prefix
// over its points (two per thread) the first one whose running mass reaches frac·(*total). out[0] = its
// radius, out[1] = the running mass there (the last radius and the total when rounding keeps the sum short).
// One block of 1024 threads.
__global__ void __launch_bounds__(1024) k_dm_cross(const float4* __restrict__ pm, unsigned m, int tiles,
                                                   const unsigned long long* __restrict__ keys,
                                                   const unsigned* __restrict__ order, const double* __restrict__ tsum,
                                                   const double* __restrict__ total_mass, double frac,
                                                   double* __restrict__ out) {
  __shared__ double s_warp[33];
  __shared__ unsigned s_tile, s_idx;
  __shared__ double s_base, s_cum;
  const double M = *total_mass, thr = frac * M;
  const unsigned per = ((unsigned)tiles + blockDim.x - 1) / blockDim.x, t0 = threadIdx.x * per;
  double local = 0.0;
  for (unsigned k = 0; k < per; ++k)
    if (t0 + k < (unsigned)tiles) local += tsum[t0 + k];
  if (threadIdx.x == 0) {
    s_tile = 0xffffffffu;
    s_idx = 0xffffffffu;
  }
  double total;
  double cum = block_exclusive_scan_d(local, s_warp, total);  // synchronises, so s_tile is initialised
  unsigned mine = 0xffffffffu;
  for (unsigned k = 0; k < per && t0 + k < (unsigned)tiles; ++k) {
    if (cum + tsum[t0 + k] >= thr) {
      mine = t0 + k;
      atomicMin(&s_tile, mine);
      break;
    }
    cum += tsum[t0 + k];
  }
  __syncthreads();
  // the crossing tile is the first crossing of its owner's run, so the owner's running mass is its base
  if (mine != 0xffffffffu && mine == s_tile) s_base = cum;
  if (threadIdx.x == 0 && s_tile == 0xffffffffu) s_base = total;
  __syncthreads();
  // walk the particles from the crossing tile on (normally within it; rounding may push it to the next)
  double base = s_base;
  for (unsigned start = (s_tile == 0xffffffffu ? (unsigned)tiles : s_tile) * kTile; start < m; start += kTile) {
    const unsigned i0 = start + 2u * threadIdx.x;
    const double v0 = i0 < m ? (double)pm[order[i0]].w : 0.0;
    const double v1 = i0 + 1u < m ? (double)pm[order[i0 + 1u]].w : 0.0;
    double tile_total;
    const double ex = block_exclusive_scan_d(v0 + v1, s_warp, tile_total);
    const double c0 = base + ex + v0, c1 = c0 + v1;
    if (i0 < m && c0 >= thr) atomicMin(&s_idx, i0);
    else if (i0 + 1u < m && c1 >= thr) atomicMin(&s_idx, i0 + 1u);
    __syncthreads();
    if (s_idx != 0xffffffffu) {
      if (threadIdx.x == (s_idx - start) >> 1) s_cum = s_idx == i0 ? c0 : c1;
      break;
    }
    base += tile_total;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r_rem = __longlong_as_double((long long)keys[m - 1]), m_rem = M;
    if (s_idx != 0xffffffffu) {
      r_rem = __longlong_as_double((long long)keys[s_idx]);
      m_rem = s_cum;
    }
    out[0] = r_rem;
    out[1] = m_rem;
  }
}

// ---- 3. orbit classification ----------------------------------------------------------------------------
// 0 escapes, 1 disk, 2 remnant: main.rs:232-247 (variant 0) or orbit.rs:91-116 (variant 1).
__device__ __forceinline__ int classify(int variant, double px, double py, double pz, double vx, double vy,
                                        double vz, double mu, double r_rem) {
  const double r = __dsqrt_rn(dsq3(px, py, pz));
  const double v2 = dsq3(vx, vy, vz);
  const double hx = __dsub_rn(__dmul_rn(py, vz), __dmul_rn(pz, vy));
  const double hy = __dsub_rn(__dmul_rn(pz, vx), __dmul_rn(px, vz));
  const double hz = __dsub_rn(__dmul_rn(px, vy), __dmul_rn(py, vx));
  const double h2 = dsq3(hx, hy, hz);
  if (variant == 0 && r == 0.0) return 2;
  if (variant == 1 && !(r > 0.0)) return 0;
  const double energy = __dsub_rn(__dmul_rn(0.5, v2), __ddiv_rn(mu, r));
  if (energy >= 0.0) return 0;
  const double hl = __dsqrt_rn(h2);  // variant 1 multiplies by |h| twice: ((2E·|h|)·|h|)/μ²
  const double num = variant == 0 ? __dmul_rn(__dmul_rn(2.0, energy), h2)
                                  : __dmul_rn(__dmul_rn(__dmul_rn(2.0, energy), hl), hl);
  const double q = __ddiv_rn(num, __dmul_rn(mu, mu));
  const double e = __dsqrt_rn(fmax(__dadd_rn(1.0, q), 0.0));
  const double a = __ddiv_rn(-mu, __dmul_rn(2.0, energy));
  return __dmul_rn(a, __dsub_rn(1.0, e)) > r_rem ? 1 : 2;
}

// Categories: 0 target disk, 1 impactor disk, 2 target remnant, 3 impactor remnant, 4/5 escaping.
__global__ void __launch_bounds__(kDmThreads) k_dm_classify(State st, unsigned off, unsigned m, unsigned chunk,
                                                            int variant, double G, const double* __restrict__ scal,
                                                            unsigned char* __restrict__ cat,
                                                            double* __restrict__ part, unsigned* __restrict__ bcnt) {
  __shared__ double s[kDmThreads / 32][kDmVals];
  double a[kDmVals] = {0, 0, 0, 0, 0, 0, 0, 0};
  const double cx = scal[S_COM], cy = scal[S_COM + 1], cz = scal[S_COM + 2];
  const double ux = scal[S_VCOM], uy = scal[S_VCOM + 1], uz = scal[S_VCOM + 2];
  const double mu = G * scal[S_MREM], r_rem = scal[S_RREM];
  const unsigned b0 = blockIdx.x * chunk, b1 = min(m, b0 + chunk);
  unsigned ndisk = 0;
  for (unsigned base = b0; base < b1; base += kDmThreads) {
    const unsigned i = base + threadIdx.x;
    int is_disk = 0;
    if (i < b1) {
      const unsigned t = off + i;
      const float3 p = pos_f32(st, t);
      const float4 v = st.vel_u[t];
      const int c = classify(variant, __dsub_rn((double)p.x, cx), __dsub_rn((double)p.y, cy),
                             __dsub_rn((double)p.z, cz), __dsub_rn((double)v.x, ux), __dsub_rn((double)v.y, uy),
                             __dsub_rn((double)v.z, uz), mu, r_rem);
      const int k = (c == 1 ? 0 : c == 2 ? 2 : 4) + (st.prov[t] == 0u ? 0 : 1);
      cat[i] = (unsigned char)k;
      const double mm = st.mass[t];
#pragma unroll
      for (int j = 0; j < 6; ++j) a[j] += j == k ? mm : 0.0;
      if (c == 1) a[6] += (double)st.pos_h[t].w;
      is_disk = c == 1;
    }
    ndisk += (unsigned)__syncthreads_count(is_disk);
  }
  block_sum(a, s);
  if (threadIdx.x == 0) {
    for (int k = 0; k < kDmVals; ++k) part[blockIdx.x * kDmVals + k] = a[k];
    bcnt[blockIdx.x] = ndisk;
  }
}

__global__ void __launch_bounds__(1024) k_dm_classify_final(const double* __restrict__ part, int nb, unsigned m,
                                                            int variant, double link_factor,
                                                            unsigned* __restrict__ bcnt, double* __restrict__ scal,
                                                            unsigned* __restrict__ cnt, double* __restrict__ out) {
  __shared__ unsigned s_warp[33];
  __shared__ double t[kDmVals];
  const int w = threadIdx.x >> 5;
  if (w < kDmVals) {
    const double v = warp_sum_column(part, nb, w);
    if ((threadIdx.x & 31) == 0) t[w] = v;
  }
  unsigned total;
  const unsigned c = threadIdx.x < (unsigned)nb ? bcnt[threadIdx.x] : 0u;
  const unsigned o = block_exclusive_scan(c, s_warp, total);  // synchronises the block
  if (threadIdx.x < (unsigned)nb) bcnt[threadIdx.x] = o;
  if (threadIdx.x == 0) {
    cnt[C_NDISK] = total;
    const double r_rem = scal[S_RREM];
    scal[S_RHOREM] = scal[S_MREM] / (4.0 / 3.0 * kPiD * (r_rem * r_rem * r_rem));
    for (int k = 0; k < 6; ++k) scal[S_CAT + k] = t[k];
    const double mean_h = variant == 0 ? (total ? t[6] / (double)total : 0.0) : scal[S_CAT + 7] / (double)m;
    scal[S_LINK] = link_factor * mean_h;
    const double disk = t[0] + t[1];
    out[0] = disk > 0.0 ? 100.0 * t[0] / disk : 0.0;
    out[1] = disk;
    for (int k = 0; k < 6; ++k) out[2 + k] = t[k];
    out[8] = scal[S_RREM];
    out[9] = scal[S_MREM];
    for (int k = 10; k < 15; ++k) out[k] = 0.0;
    out[15] = (double)total;
  }
}

// ---- 4. friends-of-friends over the disk ----------------------------------------------------------------
__device__ __forceinline__ unsigned cell_coord(double x, double c, double inv_cs) {
  const double q = floor((x - c) * inv_cs) + (double)kCellBias;
  if (!(q > 0.0)) return 0u;  // clamping only merges far cells: linked pairs stay within one cell per axis
  return q >= (double)kCellMax ? kCellMax : (unsigned)q;
}
__device__ __forceinline__ unsigned long long cell_key(unsigned ix, unsigned iy, unsigned iz) {
  return ((unsigned long long)ix << 42) | ((unsigned long long)iy << 21) | (unsigned long long)iz;
}

// Order-preserving compaction of the disk particles (block b writes from its offset in chunk order).
__global__ void __launch_bounds__(kDmThreads) k_dm_compact(State st, const float* __restrict__ rho, unsigned off,
                                                           unsigned m, unsigned chunk,
                                                           const unsigned char* __restrict__ cat,
                                                           const unsigned* __restrict__ boff,
                                                           const double* __restrict__ scal, float4* __restrict__ dpos,
                                                           float4* __restrict__ dvel, float2* __restrict__ drp,
                                                           unsigned long long* __restrict__ keys,
                                                           unsigned* __restrict__ vals) {
  __shared__ unsigned s_warp[33];
  const double cx = scal[S_COM], cy = scal[S_COM + 1], cz = scal[S_COM + 2];
  // cell edge just above the linking length: a linked pair differs by at most one cell per axis even after
  // the f32 subtraction of the tool's distance
  const double inv_cs = 1.0 / (scal[S_LINK] * (1.0 + 0x1p-20));
  const unsigned b0 = blockIdx.x * chunk, b1 = min(m, b0 + chunk);
  unsigned run = boff[blockIdx.x];
  for (unsigned base = b0; base < b1; base += kDmThreads) {
    const unsigned i = base + threadIdx.x;
    const unsigned f = (i < b1 && cat[i] < 2) ? 1u : 0u;
    unsigned total;
    const unsigned o = run + block_exclusive_scan(f, s_warp, total);
    if (f) {
      const unsigned t = off + i;
      const float3 p = pos_f32(st, t);
      const float4 v = st.vel_u[t];
      dpos[o] = make_float4(p.x, p.y, p.z, st.pos_h[t].w);
      dvel[o] = make_float4(v.x, v.y, v.z, st.mass[t]);
      drp[o] = make_float2(rho[t], __uint_as_float(st.prov[t]));
      keys[o] = cell_key(cell_coord(p.x, cx, inv_cs), cell_coord(p.y, cy, inv_cs), cell_coord(p.z, cz, inv_cs));
      vals[o] = o;
    }
    run += total;
  }
}

__global__ void k_dm_gather(unsigned n, const unsigned* __restrict__ order, const float4* __restrict__ p0,
                            const float4* __restrict__ v0, const float2* __restrict__ r0, float4* __restrict__ p1,
                            float4* __restrict__ v1, float2* __restrict__ r1, unsigned* __restrict__ parent,
                            unsigned* __restrict__ gcnt) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned j = order[i];
  p1[i] = p0[j];
  v1[i] = v0[j];
  r1[i] = r0[j];
  if (parent) {
    parent[i] = i;
    gcnt[i] = 0u;
  }
}

// Root of x with path halving. parent[v] <= v for every v and the walk strictly decreases, so it ends.
__device__ __forceinline__ unsigned uf_find(unsigned* parent, unsigned x) {
  volatile unsigned* p = parent;
  unsigned nx = p[x];
  while (nx != x) {
    const unsigned nn = p[nx];
    if (nn != nx) p[x] = nn;  // nn is an ancestor of x
    x = nx;
    nx = nn;
  }
  return x;
}

__device__ __forceinline__ bool uf_unite(unsigned* parent, unsigned a, unsigned b) {
  for (int k = 0; k < kUnionTries; ++k) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return true;
    const unsigned hi = a > b ? a : b, lo = a > b ? b : a;
    if (atomicCAS(&parent[hi], hi, lo) == hi) return true;  // a failed hook means hi gained a parent
  }
  return false;
}

__device__ __forceinline__ double pair_d2(int variant, float4 a, float4 b) {
  if (variant == 0)  // main.rs:823: f32 difference, widened, squared
    return dsq3((double)__fsub_rn(a.x, b.x), (double)__fsub_rn(a.y, b.y), (double)__fsub_rn(a.z, b.z));
  return dsq3(__dsub_rn((double)a.x, (double)b.x), __dsub_rn((double)a.y, (double)b.y),
              __dsub_rn((double)a.z, (double)b.z));
}

__device__ __forceinline__ unsigned lower_bound_u64(const unsigned long long* k, unsigned n, unsigned long long x) {
  unsigned lo = 0, hi = n;
  while (lo < hi) {
    const unsigned mid = (lo + hi) >> 1;
    if (k[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// One warp per particle a: lanes 0-8 find the nine (x, y) columns' z-runs in the sorted cell keys, then the
// warp scans each run's partners after a, 32 at a time; a linked partner whose root differs from a's is united.
__global__ void __launch_bounds__(kDmThreads) k_dm_link(unsigned n, int variant,
                                                        const unsigned long long* __restrict__ skeys,
                                                        const float4* __restrict__ dpos,
                                                        const double* __restrict__ scal,
                                                        unsigned* __restrict__ parent, unsigned* __restrict__ cnt) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  const double link = scal[S_LINK], link2 = link * link;
  bool ok = true;
  for (unsigned a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a + 1u < n; a += nwarps) {
    const unsigned long long ka = skeys[a], knext = skeys[a + 1u];
    const unsigned ix = (unsigned)(ka >> 42), iy = (unsigned)(ka >> 21) & kCellMax, iz = (unsigned)ka & kCellMax;
    unsigned j0 = 0, j1 = 0;
    if (lane < 9u) {
      const int cx = (int)ix + (int)(lane / 3u) - 1, cy = (int)iy + (int)(lane % 3u) - 1;
      if (cx >= 0 && cx <= (int)kCellMax && cy >= 0 && cy <= (int)kCellMax) {
        const unsigned long long lo = cell_key((unsigned)cx, (unsigned)cy, iz ? iz - 1u : 0u);
        const unsigned long long hi = cell_key((unsigned)cx, (unsigned)cy, iz < kCellMax ? iz + 1u : kCellMax);
        if (hi >= knext) {  // partners come after a in the order, so each pair is tested once
          j0 = max(lower_bound_u64(skeys, n, lo), a + 1u);
          j1 = lower_bound_u64(skeys, n, hi + 1ull);
        }
      }
    }
    const float4 pa = dpos[a];
    const unsigned ra = uf_find(parent, a);
    for (int c = 0; c < 9; ++c) {
      const unsigned b0 = __shfl_sync(SPH_FULL_MASK, j0, c), b1 = __shfl_sync(SPH_FULL_MASK, j1, c);
      for (unsigned j = b0 + lane; j < b1; j += 32u)
        if (pair_d2(variant, pa, dpos[j]) <= link2) {
          const unsigned rb = uf_find(parent, j);
          // equal roots: already one group (a root never stops being one while its group is unmerged)
          if (rb != ra) ok &= uf_unite(parent, ra, rb);
        }
    }
  }
  if (!ok) atomicOr(&cnt[C_ERR], 1u);
}

__global__ void k_dm_roots(unsigned n, unsigned* __restrict__ parent, unsigned* __restrict__ gcnt,
                           unsigned long long* __restrict__ keys, unsigned* __restrict__ vals) {
  const unsigned a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const unsigned r = uf_find(parent, a);  // the smallest index of a's group
  atomicAdd(&gcnt[r], 1u);
  keys[a] = r;
  vals[a] = a;
}

// ---- 5. clumps ------------------------------------------------------------------------------------------
__global__ void k_dm_clumps(unsigned n, const unsigned long long* __restrict__ skeys,
                            const unsigned* __restrict__ gcnt, uint4* __restrict__ clump,
                            unsigned* __restrict__ cnt) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned r = (unsigned)skeys[i];
  if (i > 0 && (unsigned)skeys[i - 1] == r) return;
  const unsigned s = gcnt[r];
  if (s < 2u) return;
  const unsigned c = atomicAdd(&cnt[C_NCLUMP], 1u);
  clump[c] = make_uint4(i, s, r, 0u);
}

// One block per clump: mass, centre of mass, volume, target mass, then the internal kinetic energy.
__global__ void __launch_bounds__(kDmThreads) k_dm_clump_stats(const unsigned* __restrict__ cnt,
                                                               const uint4* __restrict__ clump, int variant,
                                                               const float4* __restrict__ dpos,
                                                               const float4* __restrict__ dvel,
                                                               const float2* __restrict__ drp,
                                                               double* __restrict__ cstat) {
  __shared__ double s[kDmThreads / 32][kDmVals];
  __shared__ double s_cv[3];
  const unsigned ncl = cnt[C_NCLUMP];
  for (unsigned c = blockIdx.x; c < ncl; c += gridDim.x) {
    const uint4 cl = clump[c];
    double a[kDmVals] = {0, 0, 0, 0, 0, 0, 0, 0}, b[kDmVals] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (unsigned j = threadIdx.x; j < cl.y; j += kDmThreads) {
      const unsigned t = cl.x + j;
      const float4 p = dpos[t], v = dvel[t];
      const float2 rp = drp[t];
      const double mm = v.w;
      a[0] += mm;
      a[1] += (double)v.x * mm;
      a[2] += (double)v.y * mm;
      a[3] += (double)v.z * mm;
      a[4] += (double)p.x * mm;
      a[5] += (double)p.y * mm;
      a[6] += (double)p.z * mm;
      const double rho = variant == 0 ? (double)rp.x : (double)fmaxf(rp.x, 1.0f);  // gpu_sph.rs:450
      a[7] += mm / rho;
      b[0] += __float_as_uint(rp.y) == 0u ? mm : 0.0;
    }
    block_sum(a, s);
    block_sum(b, s);
    if (threadIdx.x == 0) {
      for (int k = 0; k < 3; ++k) s_cv[k] = a[1 + k] / a[0];
      double* o = cstat + (size_t)c * 8;
      o[0] = a[0];
      o[1] = a[4] / a[0];
      o[2] = a[5] / a[0];
      o[3] = a[6] / a[0];
      o[4] = a[7];
      o[5] = b[0];
    }
    __syncthreads();
    double k3[kDmVals] = {0, 0, 0, 0, 0, 0, 0, 0};
    const double cvx = s_cv[0], cvy = s_cv[1], cvz = s_cv[2];
    for (unsigned j = threadIdx.x; j < cl.y; j += kDmThreads) {
      const float4 v = dvel[cl.x + j];
      k3[0] += 0.5 * (double)v.w * dsq3((double)v.x - cvx, (double)v.y - cvy, (double)v.z - cvz);
    }
    block_sum(k3, s);
    if (threadIdx.x == 0) cstat[(size_t)c * 8 + 6] = k3[0];
  }
}

// Self-potential units: the 128 × 128 tile pairs (i >= j) of a clump's lower pair triangle, T(T+1)/2 for
// T = ceil(members / 128). Exclusive 64-bit prefix over the clumps; the total goes to cnt[C_UNITS64..+1].
__device__ __forceinline__ unsigned long long clump_units(unsigned members) {
  const unsigned long long t = (members + kPeRows - 1) / kPeRows;
  return t * (t + 1ull) / 2ull;
}

__global__ void __launch_bounds__(1024) k_dm_unit_scan(unsigned* __restrict__ cnt, const uint4* __restrict__ clump,
                                                       unsigned long long* __restrict__ uoff) {
  __shared__ unsigned long long s_warp[33];
  const unsigned ncl = cnt[C_NCLUMP];
  const unsigned per = (ncl + blockDim.x - 1) / blockDim.x;
  const unsigned c0 = threadIdx.x * per;
  unsigned long long sum = 0;
  for (unsigned k = 0; k < per; ++k)
    if (c0 + k < ncl) sum += clump_units(clump[c0 + k].y);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  unsigned long long incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long t = __shfl_up_sync(SPH_FULL_MASK, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[w] = incl;
  __syncthreads();
  if (w == 0) {
    const unsigned long long x = lane < nw ? s_warp[lane] : 0ull;
    unsigned long long xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long t = __shfl_up_sync(SPH_FULL_MASK, xi, o);
      if (lane >= o) xi += t;
    }
    if (lane < nw) s_warp[lane] = xi - x;
    if (lane == 31) s_warp[32] = xi;
  }
  __syncthreads();
  unsigned long long run = s_warp[w] + incl - sum;
  for (unsigned k = 0; k < per; ++k)
    if (c0 + k < ncl) {
      uoff[c0 + k] = run;
      run += clump_units(clump[c0 + k].y);
    }
  if (threadIdx.x == 0) {
    uoff[ncl] = s_warp[32];
    *reinterpret_cast<unsigned long long*>(cnt + C_UNITS64) = s_warp[32];
  }
}

// One 128 × 128 tile pair of a clump per unit: row tile j (thread t owns member a = 128 j + t) against column
// tile i >= j staged in shared memory; on the diagonal only b > a. upe[unit] = Σ_a m_a Σ_b m_b / r_ab with the
// reference's pair distance (floored, variant 0; softened, variant 1).
__global__ void __launch_bounds__(kPeRows) k_dm_pe(const unsigned* __restrict__ cnt, const uint4* __restrict__ clump,
                                                   const unsigned long long* __restrict__ uoff, int variant,
                                                   double floor_r, double soft2, const float4* __restrict__ dpos,
                                                   const float4* __restrict__ dvel, double* __restrict__ upe) {
  __shared__ float4 sp[kPeRows];
  __shared__ double s_red[kPeRows / 32];
  const unsigned ncl = cnt[C_NCLUMP];
  const unsigned long long units = *reinterpret_cast<const unsigned long long*>(cnt + C_UNITS64);
  for (unsigned long long u = blockIdx.x; u < units; u += gridDim.x) {
    unsigned lo = 0, hi = ncl;  // the clump holding unit u: the last c with uoff[c] <= u
    while (hi - lo > 1) {
      const unsigned mid = (lo + hi) >> 1;
      if (uoff[mid] <= u) lo = mid;
      else hi = mid;
    }
    const uint4 cl = clump[lo];
    const unsigned long long k = u - uoff[lo];
    unsigned long long ti = (unsigned long long)((sqrt(8.0 * (double)k + 1.0) - 1.0) * 0.5);
    while (ti > 0 && ti * (ti + 1ull) / 2ull > k) --ti;            // the estimate is off by at most one
    while ((ti + 1ull) * (ti + 2ull) / 2ull <= k) ++ti;
    const unsigned i = (unsigned)ti, j = (unsigned)(k - ti * (ti + 1ull) / 2ull);
    const unsigned ia = j * kPeRows + threadIdx.x, ib = i * kPeRows + threadIdx.x;
    __syncthreads();  // the previous unit's readers are done with sp
    if (ib < cl.y) {
      float4 q = dpos[cl.x + ib];
      q.w = dvel[cl.x + ib].w;
      sp[threadIdx.x] = q;
    }
    __syncthreads();
    double acc = 0.0;
    if (ia < cl.y) {
      const float4 pa = dpos[cl.x + ia];
      const unsigned nb = min((unsigned)kPeRows, cl.y - i * kPeRows);
      double row = 0.0;
      // 1 / max(r, floor) = min(1/r, 1/floor) and 1 / sqrt(r² + s²) from one f64 reciprocal square root
      // (within an ulp of the divided form): the pair loop is bound by f64 issue, and this halves it
      const double inv_floor = 1.0 / floor_r;
      for (unsigned jj = i == j ? threadIdx.x + 1u : 0u; jj < nb; ++jj) {
        const float4 q = sp[jj];
        const double d2 = pair_d2(variant, pa, q);
        const double ir = variant == 0 ? fmin(rsqrt(d2), inv_floor) : rsqrt(__dadd_rn(d2, soft2));
        row += (double)q.w * ir;
      }
      acc = (double)dvel[cl.x + ia].w * row;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kPeRows / 32; ++w) t += s_red[w];
      upe[u] = t;
    }
  }
}

// One block per clump: its self-potential sum Σ_units, in a fixed order, into cstat[c][7].
__global__ void __launch_bounds__(kDmThreads) k_dm_pe_reduce(const unsigned* __restrict__ cnt,
                                                             const unsigned long long* __restrict__ uoff,
                                                             const double* __restrict__ upe,
                                                             double* __restrict__ cstat) {
  __shared__ double s[kDmThreads / 32][kDmVals];
  const unsigned ncl = cnt[C_NCLUMP];
  for (unsigned c = blockIdx.x; c < ncl; c += gridDim.x) {
    double a[kDmVals] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (unsigned long long u = uoff[c] + threadIdx.x; u < uoff[c + 1]; u += kDmThreads) a[0] += upe[u];
    block_sum(a, s);
    if (threadIdx.x == 0) cstat[(size_t)c * 8 + 7] = a[0];
  }
}

// Boundness, the Roche gate and the heaviest bound clump outside it (ties: the smaller root).
__global__ void __launch_bounds__(kDmThreads) k_dm_select(const unsigned* __restrict__ cnt,
                                                          const uint4* __restrict__ clump,
                                                          const double* __restrict__ cstat,
                                                          const double* __restrict__ scal, int variant, double G,
                                                          double roche, double rho_fallback, double* __restrict__ out) {
  __shared__ double s_m[kDmThreads], s_e[kDmThreads];
  __shared__ unsigned s_root[kDmThreads], s_n[kDmThreads], s_bound[kDmThreads], s_cl[kDmThreads];
  const unsigned ncl = cnt[C_NCLUMP];
  const double cx = scal[S_COM], cy = scal[S_COM + 1], cz = scal[S_COM + 2];
  const double r_rem = scal[S_RREM], rho_rem = scal[S_RHOREM];
  double bm = 0.0, be = 0.0;
  unsigned broot = 0xffffffffu, bn = 0, nb = 0, nc = 0;
  for (unsigned c = threadIdx.x; c < ncl; c += blockDim.x) {
    const double* st = cstat + (size_t)c * 8;
    const double M = st[0];
    if (variant == 1 && !(M > 0.0)) continue;  // accretion.rs:121 skips massless groups
    ++nc;
    const double pe = -G * st[7];
    const bool bound = st[6] + pe < 0.0;
    const double rho_c = st[4] > 0.0 ? M / st[4] : rho_fallback;
    const double d_roche = roche * r_rem * cbrt(rho_rem / rho_c);
    const double dx = st[1] - cx, dy = st[2] - cy, dz = st[3] - cz;
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    nb += bound ? 1u : 0u;
    const uint4 cl = clump[c];
    if (bound && dist > d_roche && (M > bm || (M == bm && M > 0.0 && cl.z < broot))) {
      bm = M;
      be = st[5];
      broot = cl.z;
      bn = cl.y;
    }
  }
  s_m[threadIdx.x] = bm;
  s_e[threadIdx.x] = be;
  s_root[threadIdx.x] = broot;
  s_n[threadIdx.x] = bn;
  s_bound[threadIdx.x] = nb;
  s_cl[threadIdx.x] = nc;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kDmThreads; ++k) {
      nb += s_bound[k];
      nc += s_cl[k];
      if (s_m[k] > bm || (s_m[k] == bm && s_m[k] > 0.0 && s_root[k] < broot)) {
        bm = s_m[k];
        be = s_e[k];
        broot = s_root[k];
        bn = s_n[k];
      }
    }
    out[10] = bm;
    out[11] = bm > 0.0 ? 100.0 * be / bm : 0.0;
    out[12] = (double)bn;
    out[13] = (double)nc;
    out[14] = (double)nb;
  }
}


// ---------------------------------------------------------------------------------------------------------
// Relaxed-body assembly: body_bulk (gpu_sph.rs:260-293) and assemble_from_relaxed_n (gpu_sph.rs:309-339).
// A body's bulk: the centre of mass of its particles, the radius holding 98 % of their mass about it, then twice
// the same over the particles within 1.5 × that radius of that centre (stray particles left by the relaxation
// do not drag the centre). The assembly recentres each source body (prov k) on its bulk centre, places it at
// offset k moving at vel k + spin k × (r − centre), keeps every other field, and drops particles whose prov has
// no placement.
// ---------------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool bb_take(const State& st, unsigned t, unsigned prov, int clip,
                                        const double* __restrict__ bb) {
  if (st.prov[t] != prov) return false;
  if (!clip) return true;
  const float3 p = pos_f32(st, t);
  const double r = __dsqrt_rn(dsq3(__dsub_rn((double)p.x, bb[BB_C]), __dsub_rn((double)p.y, bb[BB_C + 1]),
                                   __dsub_rn((double)p.z, bb[BB_C + 2])));
  return r <= 1.5 * bb[BB_R];
}

__global__ void __launch_bounds__(kDmThreads) k_bb_count(State st, unsigned n, unsigned chunk, unsigned prov,
                                                         int clip, const double* __restrict__ bb,
                                                         double* __restrict__ part, unsigned* __restrict__ bcnt) {
  __shared__ double s[kDmThreads / 32][kDmVals];
  double a[kDmVals] = {0, 0, 0, 0, 0, 0, 0, 0};
  const unsigned b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  unsigned cnt = 0;
  for (unsigned base = b0; base < b1; base += kDmThreads) {
    const unsigned t = base + threadIdx.x;
    const bool take = t < b1 && bb_take(st, t, prov, clip, bb);
    if (take) {
      const float3 p = pos_f32(st, t);
      const double mm = st.mass[t];
      a[0] += mm;
      a[1] += (double)p.x * mm;
      a[2] += (double)p.y * mm;
      a[3] += (double)p.z * mm;
    }
    cnt += (unsigned)__syncthreads_count(take);
  }
  block_sum(a, s);
  if (threadIdx.x == 0) {
    for (int k = 0; k < kDmVals; ++k) part[blockIdx.x * kDmVals + k] = a[k];
    bcnt[blockIdx.x] = cnt;
  }
}

// Sums of the selection (centre of mass, zero for a massless one: gpu_sph.rs:266) and the block offsets.
__global__ void __launch_bounds__(1024) k_bb_scan(const double* __restrict__ part, int nb, int first,
                                                  unsigned* __restrict__ bcnt, double* __restrict__ bb,
                                                  unsigned* __restrict__ cnt) {
  __shared__ unsigned s_warp[33];
  __shared__ double t[kDmVals];
  const int w = threadIdx.x >> 5;
  if (w < 4) {
    const double v = warp_sum_column(part, nb, w);
    if ((threadIdx.x & 31) == 0) t[w] = v;
  }
  unsigned total;
  const unsigned c = threadIdx.x < (unsigned)nb ? bcnt[threadIdx.x] : 0u;
  const unsigned o = block_exclusive_scan(c, s_warp, total);
  if (threadIdx.x < (unsigned)nb) bcnt[threadIdx.x] = o;
  if (threadIdx.x == 0) {
    cnt[C_SEL] = total;
    const double mm = t[0];
    for (int k = 0; k < 3; ++k) bb[BB_CN + k] = mm > 0.0 ? t[1 + k] / mm : 0.0;
    bb[BB_MN] = mm;
    if (first) bb[BB_M] = mm;
  }
}

__global__ void __launch_bounds__(kDmThreads) k_bb_write(State st, unsigned n, unsigned chunk, unsigned prov,
                                                         int clip, const double* __restrict__ bb,
                                                         const unsigned* __restrict__ boff, float4* __restrict__ pm) {
  __shared__ unsigned s_warp[33];
  const unsigned b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  unsigned run = boff[blockIdx.x];
  for (unsigned base = b0; base < b1; base += kDmThreads) {
    const unsigned t = base + threadIdx.x;
    const unsigned f = (t < b1 && bb_take(st, t, prov, clip, bb)) ? 1u : 0u;
    unsigned total;
    const unsigned o = run + block_exclusive_scan(f, s_warp, total);
    if (f) {
      const float3 p = pos_f32(st, t);
      pm[o] = make_float4(p.x, p.y, p.z, st.mass[t]);
    }
    run += total;
  }
}

__global__ void k_bb_commit(double* __restrict__ bb) {
  for (int k = 0; k < 3; ++k) bb[BB_C + k] = bb[BB_CN + k];
  bb[BB_R] = bb[BB_RN];
}

// Assembly: count the kept particles per block (original order), then write them transformed.
__global__ void __launch_bounds__(kDmThreads) k_asm_count(const P48x* __restrict__ aos, unsigned n, unsigned chunk,
                                                          unsigned np, unsigned* __restrict__ bcnt) {
  const unsigned b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  unsigned cnt = 0;
  for (unsigned base = b0; base < b1; base += kDmThreads) {
    const unsigned i = base + threadIdx.x;
    cnt += (unsigned)__syncthreads_count(i < b1 && aos[i].prov < np);
  }
  if (threadIdx.x == 0) bcnt[blockIdx.x] = cnt;
}

__global__ void __launch_bounds__(1024) k_u32_offsets(unsigned* __restrict__ bcnt, int nb, unsigned* __restrict__ total_out) {
  __shared__ unsigned s_warp[33];
  unsigned total;
  const unsigned c = threadIdx.x < (unsigned)nb ? bcnt[threadIdx.x] : 0u;
  const unsigned o = block_exclusive_scan(c, s_warp, total);
  if (threadIdx.x < (unsigned)nb) bcnt[threadIdx.x] = o;
  if (threadIdx.x == 0) *total_out = total;
}

__global__ void __launch_bounds__(kDmThreads) k_asm_write(const P48x* __restrict__ aos, unsigned n, unsigned chunk,
                                                          unsigned np, const double* __restrict__ place,
                                                          const unsigned* __restrict__ boff, P48x* __restrict__ dst,
                                                          unsigned* __restrict__ minh_key) {
  __shared__ unsigned s_warp[33];
  const unsigned b0 = blockIdx.x * chunk, b1 = min(n, b0 + chunk);
  unsigned run = boff[blockIdx.x];
  unsigned hk = 0xffffffffu;
  for (unsigned base = b0; base < b1; base += kDmThreads) {
    const unsigned i = base + threadIdx.x;
    P48x p;
    unsigned f = 0u;
    if (i < b1) {
      p = aos[i];
      f = p.prov < np ? 1u : 0u;
    }
    unsigned total;
    const unsigned o = run + block_exclusive_scan(f, s_warp, total);
    if (f) {
      const double* pl = place + (size_t)p.prov * 12;  // offset, vel, spin, centre
      const double lx = __dsub_rn((double)p.px, pl[9]), ly = __dsub_rn((double)p.py, pl[10]),
                   lz = __dsub_rn((double)p.pz, pl[11]);
      const double qx = __dadd_rn(lx, pl[0]), qy = __dadd_rn(ly, pl[1]), qz = __dadd_rn(lz, pl[2]);
      const double sx = pl[6], sy = pl[7], sz = pl[8];
      const double vx = __dadd_rn(pl[3], __dsub_rn(__dmul_rn(sy, lz), __dmul_rn(ly, sz)));
      const double vy = __dadd_rn(pl[4], __dsub_rn(__dmul_rn(sz, lx), __dmul_rn(lz, sx)));
      const double vz = __dadd_rn(pl[5], __dsub_rn(__dmul_rn(sx, ly), __dmul_rn(lx, sy)));
      P48x q = p;
      q.px = (float)qx;
      q.py = (float)qy;
      q.pz = (float)qz;
      q.vx = (float)vx;
      q.vy = (float)vy;
      q.vz = (float)vz;
      dst[o] = q;
      hk = min(hk, float_key(p.h));
    }
    run += total;
  }
  hk = warp_min(hk);
  if ((threadIdx.x & 31) == 0 && hk != 0xffffffffu) atomicMin(minh_key, hk);
}

int bits_of(unsigned v) {
  int b = 0;
  while (b < 32 && (v >> b)) ++b;
  return b;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Carve the workspace for m particles from one allocation.
bool work_reserve(DiskWork* w, int m) {
  if (w->cap >= m && w->base) return true;
  if (w->base) cudaFree(w->base);
  w->base = nullptr;
  w->cap = 0;
  const size_t n = (size_t)(m < 1 ? 1 : m), half = n / 2 + 2, tiles = radix_tiles((int)n);
  size_t sz = 0;
  auto take = [&](size_t bytes) {
    const size_t o = sz;
    sz += align256(bytes);
    return o;
  };
  const size_t o_k0 = take(8 * n), o_k1 = take(8 * n), o_v0 = take(4 * n), o_v1 = take(4 * n);
  const size_t o_hist = take(4 * 256 * tiles), o_tot = take(4 * 256), o_part = take(8 * kDmBlocks * kDmVals);
  const size_t o_tsum = take(8 * tiles), o_scal = take(8 * S_COUNT), o_cnt = take(4 * C_COUNT);
  const size_t o_bcnt = take(4 * kDmBlocks), o_cat = take(n);
  const size_t o_pm = take(16 * n), o_p0 = take(16 * n), o_p1 = take(16 * n), o_u0 = take(16 * n), o_u1 = take(16 * n);
  const size_t o_r0 = take(8 * n), o_r1 = take(8 * n), o_par = take(4 * n), o_g = take(4 * n);
  const size_t o_cl = take(16 * half), o_uo = take(8 * (half + 1)), o_cs = take(64 * half);
  const size_t o_out = take(8 * 16), o_bb = take(8 * 16), o_pl = take(8 * 12 * kMaxPlacements);
  void* base = nullptr;
  if (cudaMalloc(&base, sz) != cudaSuccess) return false;
  char* b = (char*)base;
  w->base = base;
  w->cap = (int)n;
  w->keys[0] = (unsigned long long*)(b + o_k0);
  w->keys[1] = (unsigned long long*)(b + o_k1);
  w->vals[0] = (unsigned*)(b + o_v0);
  w->vals[1] = (unsigned*)(b + o_v1);
  w->hist = (unsigned*)(b + o_hist);
  w->tot = (unsigned*)(b + o_tot);
  w->part = (double*)(b + o_part);
  w->tsum = (double*)(b + o_tsum);
  w->scal = (double*)(b + o_scal);
  w->cnt = (unsigned*)(b + o_cnt);
  w->bcnt = (unsigned*)(b + o_bcnt);
  w->cat = (unsigned char*)(b + o_cat);
  w->pm = (float4*)(b + o_pm);
  w->dpos[0] = (float4*)(b + o_p0);
  w->dpos[1] = (float4*)(b + o_p1);
  w->dvel[0] = (float4*)(b + o_u0);
  w->dvel[1] = (float4*)(b + o_u1);
  w->drp[0] = (float2*)(b + o_r0);
  w->drp[1] = (float2*)(b + o_r1);
  w->parent = (unsigned*)(b + o_par);
  w->gcnt = (unsigned*)(b + o_g);
  w->clump = (uint4*)(b + o_cl);
  w->uoff = (unsigned long long*)(b + o_uo);
  w->cstat = (double*)(b + o_cs);
  w->out = (double*)(b + o_out);
  w->bb = (double*)(b + o_bb);
  w->place = (double*)(b + o_pl);
  return true;
}

// Radius of the point whose running mass, in radius order about `centre`, first reaches frac·(*total)
// (out[0]) and that running mass (out[1]); every pointer is device memory; n >= 1.
int launch_radius_crossing(DiskWork* w, const float4* pm, unsigned n, const double* centre, const double* total,
                           double frac, double* out, cudaStream_t s) {
  k_dm_radius<<<(n + 255) / 256, 256, 0, s>>>(pm, n, centre, w->keys[0], w->vals[0]);
  int src = 0;
  int L = 1 + launch_radix_sort(w->keys, w->vals, (int)n, 64, w->hist, w->tot, src, s);
  const int tiles = (int)((n + kTile - 1) / kTile);
  k_dm_tile_mass<<<tiles, kDmThreads, 0, s>>>(pm, n, w->vals[src], w->tsum);
  k_dm_cross<<<1, 1024, 0, s>>>(pm, n, tiles, w->keys[src], w->vals[src], w->tsum, total, frac, out);
  return L + 2;
}

}  // namespace

void disk_work_free(DiskWork* w) {
  if (!w) return;
  if (w->base) cudaFree(w->base);
  if (w->upe) cudaFree(w->upe);
  delete w;
}

int disk_measure(const Dev& d, unsigned off, unsigned m, const DiskCfg& c, DiskWork*& w, double* out,
                 unsigned long long* launches, const char** err, cudaStream_t s) {
  std::memset(out, 0, 16 * sizeof(double));
  *launches = 0;
  if (m == 0) return 0;
  if (!w) w = new DiskWork();
  if (!work_reserve(w, (int)m)) {
    *err = "disk measure: workspace allocation failed";
    return -3;
  }
  const State& st = d.s();
  unsigned long long L = 0;
  const unsigned chunk = ((m + kDmBlocks - 1) / kDmBlocks + kDmThreads - 1) / kDmThreads * kDmThreads;
  const int nb = (int)((m + chunk - 1) / chunk);
  cudaMemsetAsync(w->cnt, 0, 4 * C_COUNT, s);
  k_dm_moments<<<nb, kDmThreads, 0, s>>>(st, off, m, chunk, w->part, w->pm);
  k_dm_moments_final<<<1, kDmThreads, 0, s>>>(w->part, nb, w->scal);
  L += 2;
  L += launch_radius_crossing(w, w->pm, m, w->scal + S_COM, w->scal + S_M, c.remnant_frac, w->scal + S_RREM, s);
  k_dm_classify<<<nb, kDmThreads, 0, s>>>(st, off, m, chunk, c.variant, c.G, w->scal, w->cat, w->part, w->bcnt);
  k_dm_classify_final<<<1, 1024, 0, s>>>(w->part, nb, m, c.variant, c.link_factor, w->bcnt, w->scal, w->cnt, w->out);
  L += 2;
  unsigned nd = 0;
  cudaMemcpyAsync(&nd, w->cnt + C_NDISK, 4, cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return -2;
  }
  int src = 0;
  if (nd >= 2) {
    k_dm_compact<<<nb, kDmThreads, 0, s>>>(st, d.rho, off, m, chunk, w->cat, w->bcnt, w->scal, w->dpos[0],
                                           w->dvel[0], w->drp[0], w->keys[0], w->vals[0]);
    L += 1;
    L += launch_radix_sort(w->keys, w->vals, (int)nd, 63, w->hist, w->tot, src, s);
    const unsigned gb = (nd + 255) / 256;
    k_dm_gather<<<gb, 256, 0, s>>>(nd, w->vals[src], w->dpos[0], w->dvel[0], w->drp[0], w->dpos[1], w->dvel[1],
                                   w->drp[1], w->parent, w->gcnt);
    const unsigned lb = (nd + 7) / 8;  // one warp per particle, grid-strided over at most 16 blocks per SM
    k_dm_link<<<lb < 2368u ? lb : 2368u, kDmThreads, 0, s>>>(nd, c.variant, w->keys[src], w->dpos[1], w->scal,
                                                             w->parent, w->cnt);
    k_dm_roots<<<gb, 256, 0, s>>>(nd, w->parent, w->gcnt, w->keys[0], w->vals[0]);
    L += 3;
    L += launch_radix_sort(w->keys, w->vals, (int)nd, bits_of(nd), w->hist, w->tot, src, s);
    k_dm_gather<<<gb, 256, 0, s>>>(nd, w->vals[src], w->dpos[1], w->dvel[1], w->drp[1], w->dpos[0], w->dvel[0],
                                   w->drp[0], nullptr, nullptr);
    k_dm_clumps<<<gb, 256, 0, s>>>(nd, w->keys[src], w->gcnt, w->clump, w->cnt);
    const unsigned cb = nd / 2 < 1184u ? nd / 2 : 1184u;  // clumps <= nd / 2; blocks stride over them
    k_dm_clump_stats<<<cb, kDmThreads, 0, s>>>(w->cnt, w->clump, c.variant, w->dpos[0], w->dvel[0], w->drp[0],
                                               w->cstat);
    k_dm_unit_scan<<<1, 1024, 0, s>>>(w->cnt, w->clump, w->uoff);
    L += 4;
    // the self-potential's unit count sizes its partial sums: read it back once
    unsigned long long units = 0;
    cudaMemcpyAsync(&units, w->cnt + C_UNITS64, 8, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      *err = cudaGetErrorString(e);
      return -2;
    }
    if (units > kMaxUnits) {
      *err = "disk measure: a clump's self-potential needs more than 2^28 tile pairs (a clump of ~3M particles)";
      return -5;
    }
    if (units > w->upe_cap) {
      if (w->upe) cudaFree(w->upe);
      w->upe = nullptr;
      w->upe_cap = 0;
      const unsigned long long cap = units + units / 2 + 1024;
      if (cudaMalloc(&w->upe, 8 * cap) != cudaSuccess) {
        *err = "disk measure: self-potential workspace allocation failed";
        return -3;
      }
      w->upe_cap = cap;
    }
    if (units) {
      const unsigned pb = units < 4736ull ? (unsigned)units : 4736u;  // 32 blocks per SM, grid-strided
      k_dm_pe<<<pb, kPeRows, 0, s>>>(w->cnt, w->clump, w->uoff, c.variant, c.pe_floor, c.pe_soft * c.pe_soft,
                                     w->dpos[0], w->dvel[0], w->upe);
      k_dm_pe_reduce<<<cb, kDmThreads, 0, s>>>(w->cnt, w->uoff, w->upe, w->cstat);
      L += 2;
    }
    k_dm_select<<<1, kDmThreads, 0, s>>>(w->cnt, w->clump, w->cstat, w->scal, c.variant, c.G, c.roche,
                                         c.rho_fallback, w->out);
    L += 1;
  }
  unsigned flags[C_COUNT];
  cudaMemcpyAsync(out, w->out, 16 * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(flags, w->cnt, sizeof(flags), cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return -2;
  }
  *launches = L;
  if (flags[C_ERR]) {
    *err = "disk measure: a union-find hook gave up after its retry limit";
    return -5;
  }
  return 0;
}


namespace {

int reserve_or_fail(DiskWork*& w, unsigned m, const char** err) {
  if (!w) w = new DiskWork();
  if (!work_reserve(w, (int)(m ? m : 1u))) {
    *err = "body measurement: workspace allocation failed";
    return -3;
  }
  return 0;
}

int sync_or_fail(cudaStream_t s, const char** err) {
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return -2;
  }
  return 0;
}

// body_bulk of one provenance into w->bb; on return out5 = {cx, cy, cz, mass, radius} (host).
int body_bulk_impl(const Dev& d, unsigned prov, DiskWork* w, double* out5, unsigned long long* L,
                   const char** err, cudaStream_t s) {
  const unsigned n = (unsigned)d.n;
  const State& st = d.s();
  const unsigned chunk = ((n + kDmBlocks - 1) / kDmBlocks + kDmThreads - 1) / kDmThreads * kDmThreads;
  const int nb = (int)((n + chunk - 1) / chunk);
  cudaMemsetAsync(w->bb, 0, 16 * sizeof(double), s);
  for (int round = 0; round < 3; ++round) {
    const int clip = round > 0;
    k_bb_count<<<nb, kDmThreads, 0, s>>>(st, n, chunk, prov, clip, w->bb, w->part, w->bcnt);
    k_bb_scan<<<1, 1024, 0, s>>>(w->part, nb, round == 0, w->bcnt, w->bb, w->cnt);
    unsigned sel = 0;
    cudaMemcpyAsync(&sel, w->cnt + C_SEL, 4, cudaMemcpyDeviceToHost, s);
    *L += 2;
    if (int rc = sync_or_fail(s, err)) return rc;
    if (sel == 0) break;  // nothing of this body (round 0), or nothing inside the clip sphere: keep the last
    k_bb_write<<<nb, kDmThreads, 0, s>>>(st, n, chunk, prov, clip, w->bb, w->bcnt, w->pm);
    *L += 1 + launch_radius_crossing(w, w->pm, sel, w->bb + BB_CN, w->bb + BB_MN, 0.98, w->bb + BB_RN, s);
    k_bb_commit<<<1, 1, 0, s>>>(w->bb);
    *L += 1;
  }
  double bb[16];
  cudaMemcpyAsync(bb, w->bb, sizeof(bb), cudaMemcpyDeviceToHost, s);
  if (int rc = sync_or_fail(s, err)) return rc;
  out5[0] = bb[BB_C];
  out5[1] = bb[BB_C + 1];
  out5[2] = bb[BB_C + 2];
  out5[3] = bb[BB_M];
  out5[4] = bb[BB_R];
  return 0;
}

}  // namespace

int body_bulk(const Dev& d, unsigned prov, DiskWork*& w, double* out5, unsigned long long* launches,
              const char** err, cudaStream_t s) {
  *launches = 0;
  for (int k = 0; k < 5; ++k) out5[k] = 0.0;
  if (d.n == 0) return 0;
  if (int rc = reserve_or_fail(w, (unsigned)d.n, err)) return rc;
  return body_bulk_impl(d, prov, w, out5, launches, err, s);
}

int assemble_n(const Dev& d, const double* placements, unsigned np, void* dst, unsigned* n_out, float* min_h,
               DiskWork*& w, unsigned long long* launches, const char** err, cudaStream_t s) {
  *launches = 0;
  *n_out = 0;
  *min_h = __builtin_inff();
  if (np > kMaxPlacements) {
    *err = "assemble: at most 256 placements";
    return -1;
  }
  const unsigned n = (unsigned)d.n;
  if (n == 0 || np == 0) return 0;
  if (int rc = reserve_or_fail(w, n, err)) return rc;
  unsigned long long L = 0;
  double place[kMaxPlacements * 12];
  for (unsigned k = 0; k < np; ++k) {
    double bulk[5];
    if (int rc = body_bulk_impl(d, k, w, bulk, &L, err, s)) return rc;
    for (int j = 0; j < 9; ++j) place[k * 12 + j] = placements[k * 9 + j];
    for (int j = 0; j < 3; ++j) place[k * 12 + 9 + j] = bulk[j];
  }
  cudaMemcpyAsync(w->place, place, sizeof(double) * 12 * np, cudaMemcpyHostToDevice, s);
  launch_to_aos(d, s);  // the state in original order, as the 48-byte records the reference assembles from
  const unsigned chunk = ((n + kDmBlocks - 1) / kDmBlocks + kDmThreads - 1) / kDmThreads * kDmThreads;
  const int nb = (int)((n + chunk - 1) / chunk);
  cudaMemsetAsync(w->cnt + C_MINH, 0xff, 4, s);
  k_asm_count<<<nb, kDmThreads, 0, s>>>((const P48x*)d.aos, n, chunk, np, w->bcnt);
  k_u32_offsets<<<1, 1024, 0, s>>>(w->bcnt, nb, w->cnt + C_SEL);
  k_asm_write<<<nb, kDmThreads, 0, s>>>((const P48x*)d.aos, n, chunk, np, w->place, w->bcnt, (P48x*)dst,
                                        w->cnt + C_MINH);
  L += 4;
  unsigned cnts[C_COUNT];
  cudaMemcpyAsync(cnts, w->cnt, sizeof(cnts), cudaMemcpyDeviceToHost, s);
  if (int rc = sync_or_fail(s, err)) return rc;
  *n_out = cnts[C_SEL];
  if (cnts[C_MINH] != 0xffffffffu) {  // the order-preserving key back to the float
    const unsigned k = cnts[C_MINH];
    const unsigned b = (k >> 31) ? (k ^ 0x80000000u) : ~k;
    std::memcpy(min_h, &b, 4);
  }
  *launches = L;
  return 0;
}

}  // namespace sphb
