// Fused LBVH group walk: Barnes-Hut gravity (group MAC, monopole + optional quadrupole) and the SPH
// neighbour lists in ONE traversal per warp.
//
// A warp owns 32 Morton-consecutive particles (its "group") and walks the tree with a LIFO stack in shared
// memory, popping up to 32 nodes at a time (one per lane) so node loads overlap instead of serialising.
// Each popped node is classified for the whole group:
//   * accepted  — the MAC sqrt(d²+ε²) >= side/θ + |centre−COM| (the node's largest side, as the reference's
//                 CPU octree measures it, bhtree.rs:181, with the δ term of bh_gravity.wgsl:382) holds for the
//                 nearest point of the group's bounding box, hence for every particle of the group, and the
//                 node's box is outside the SPH reach: appended to the multipole list;
//   * leaf      — appended to the near list (pairwise gravity + the neighbour test) when some particle of the
//                 group can reach it with its own smoothing length (a per-lane test after the group test),
//                 otherwise to the far list (pairwise gravity only); with half leaves a far leaf is queued, and
//                 a later pass classifies the halves of up to 32 queued leaves at once (each half a multipole,
//                 a term of the group's local expansion, or 8 pairwise sources);
//   * opened    — children pushed (ballot + popc compaction).
// Accepted nodes far from the group (beyond r_group/θ_L) go into the group's local expansion instead of the
// per-particle multipole list.
// Nodes whose box lies within ½(h_group,max + h_node,max) of the group are always opened, so every leaf
// that can hold an SPH neighbour reaches the direct list: the neighbour set {j != i : r_ij < h_ij} is
// complete. Without a skin (fixed h) the test is the reference predicate, single-rounded, so the set is
// identical to it (sph_step.wgsl:141-143); with a skin the list is a candidate set that contains it.
// Lists are flushed through shared memory in chunks of 32 sources (the next chunk's loads issued before the
// current chunk is evaluated); every lane then runs the chunk against its own particle with no dependent loads.
// The interaction loops take the staged sources two at a time with the packed FP32x2 add/multiply/fma of sm_100
// (each half rounded as the scalar operation); their reciprocal square roots are the bare special-function
// operation.
#include <type_traits>

#include "sph_kernels.cuh"

namespace sphb {

constexpr int TW_STACK = 1280;  // per-warp node stack
constexpr int TW_LIST = 96;     // per-warp list capacity (a pop adds <= 64 entries; flushed above 32)
constexpr int TW_WARPS_PER_SM = 24;  // resident walk warps per SM (80 registers, ~8.4 KB shared each)

// Per-block shared memory of a W-warp walk block (the traversal tile: W groups of 32 particles).
template <int W>
struct WalkSmem {
  unsigned stack[W][TW_STACK];
  unsigned m2p[W][TW_LIST];
  unsigned m2l[W][TW_LIST];   // accepted nodes far from the group: into the group's local expansion
  unsigned p2p[W][TW_LIST];   // near leaves: pairwise gravity + neighbour predicate
  unsigned p2f[W][TW_LIST];   // far leaves: pairwise gravity only
  unsigned hl[W][TW_LIST];    // far leaves queued for the classification of their halves
  float4 src[W][32];   // staged sources: x, y, z, m
  float4 q0[W][32];    // staged quadrupoles
  float2 q1[W][32];
  float2 sh[W][32];    // staged source index (bits) and smoothing length (direct list)
};

// Compensated accumulator for the precision mode.
struct Acc3 {
  float x = 0.f, y = 0.f, z = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
  template <bool KAHAN>
  __device__ __forceinline__ void add(float ax, float ay, float az) {
    if (KAHAN) {
      float yy = ax - cx, t = x + yy;
      cx = (t - x) - yy;
      x = t;
      yy = ay - cy;
      t = y + yy;
      cy = (t - y) - yy;
      y = t;
      yy = az - cz;
      t = z + yy;
      cz = (t - z) - yy;
      z = t;
    } else {
      x += ax;
      y += ay;
      z += az;
    }
  }
};

// ---- the group's local expansion --------------------------------------------------------------------------
// An accepted node far from the group (|COM − z| >= r_g/θ_L, z the centre of the group's box and r_g its
// half-diagonal) does not go through a per-particle multipole evaluation: its potential is expanded about z,
//   φ(z + y) ≈ φ0 + g·y + ½ yᵀH y + ⅙ T:yyy,   a(z + y) = −(g + H y + ½ T:yy),
// with the monopole to third order and the quadrupole to second order in y (Cartesian Taylor coefficients of
// the softened 1/R; R² = |u|² + ε², u = COM − z, e = u/R so that Q·e stays in f32 range in SI units). Each lane
// expands a different node, the warp sums the 20 coefficients (lane k ends up holding coefficient k), and each
// particle evaluates the expansion once. Coefficient order: φ0; g x, y, z; H xx, yy, zz, xy, xz, yz;
// T xxx, yyy, zzz, xxy, xxz, xyy, yyz, xzz, yzz, xyz.
constexpr int kLocal = 20;

template <bool QUAD>
__device__ __forceinline__ void local_coeffs(float4 c, float4 q0, float2 q1, float G, float zx, float zy, float zz,
                                             float soft2, float v[32]) {
  const float ux = c.x - zx, uy = c.y - zy, uz = c.z - zz;
  const float iR = rsqrt_ftz(fmaf(ux, ux, fmaf(uy, uy, fmaf(uz, uz, soft2))));
  const float ex = ux * iR, ey = uy * iR, ez = uz * iR;
  const float s0 = G * c.w * iR, s1 = s0 * iR, s2 = s1 * iR, s3 = s2 * iR;
  const float xx = ex * ex, yy = ey * ey, zz2 = ez * ez;
  v[0] = -s0;
  v[1] = -s1 * ex;
  v[2] = -s1 * ey;
  v[3] = -s1 * ez;
  v[4] = -s2 * fmaf(3.0f, xx, -1.0f);
  v[5] = -s2 * fmaf(3.0f, yy, -1.0f);
  v[6] = -s2 * fmaf(3.0f, zz2, -1.0f);
  const float m3s2 = -3.0f * s2;
  v[7] = m3s2 * ex * ey;
  v[8] = m3s2 * ex * ez;
  v[9] = m3s2 * ey * ez;
  const float ax = fmaf(-15.0f, xx, 3.0f), ay = fmaf(-15.0f, yy, 3.0f), az = fmaf(-15.0f, zz2, 3.0f);
  v[10] = s3 * ex * (ax + 6.0f);
  v[11] = s3 * ey * (ay + 6.0f);
  v[12] = s3 * ez * (az + 6.0f);
  v[13] = s3 * ey * ax;  // xxy
  v[14] = s3 * ez * ax;  // xxz
  v[15] = s3 * ex * ay;  // xyy
  v[16] = s3 * ez * ay;  // yyz
  v[17] = s3 * ex * az;  // xzz
  v[18] = s3 * ey * az;  // yzz
  v[19] = -15.0f * s3 * ex * ey * ez;
  if (QUAD) {
    // q = G·Q (traceless, about the COM): φ = −½ eQe/R³; g = (Qe − 5/2 eQe e)/R⁴;
    // H = −(Q − 5(Qe eᵀ + e Qeᵀ) − 5/2 eQe I + 35/2 eQe e eᵀ)/R⁵
    const float qxx = G * q0.x, qyy = G * q0.y, qzz = G * q0.z, qxy = G * q0.w, qxz = G * q1.x, qyz = G * q1.y;
    const float Qx = fmaf(qxx, ex, fmaf(qxy, ey, qxz * ez));
    const float Qy = fmaf(qxy, ex, fmaf(qyy, ey, qyz * ez));
    const float Qz = fmaf(qxz, ex, fmaf(qyz, ey, qzz * ez));
    const float eQe = fmaf(ex, Qx, fmaf(ey, Qy, ez * Qz));
    const float iR2 = iR * iR, iR3 = iR2 * iR, iR4 = iR2 * iR2, iR5 = iR4 * iR;
    v[0] = fmaf(-0.5f * eQe, iR3, v[0]);
    const float k25 = 2.5f * eQe;
    v[1] = fmaf(iR4, fmaf(-k25, ex, Qx), v[1]);
    v[2] = fmaf(iR4, fmaf(-k25, ey, Qy), v[2]);
    v[3] = fmaf(iR4, fmaf(-k25, ez, Qz), v[3]);
    const float k175 = 17.5f * eQe;
    v[4] = fmaf(-iR5, fmaf(k175, xx, fmaf(-10.0f * Qx, ex, qxx - k25)), v[4]);
    v[5] = fmaf(-iR5, fmaf(k175, yy, fmaf(-10.0f * Qy, ey, qyy - k25)), v[5]);
    v[6] = fmaf(-iR5, fmaf(k175, zz2, fmaf(-10.0f * Qz, ez, qzz - k25)), v[6]);
    v[7] = fmaf(-iR5, fmaf(k175 * ex, ey, fmaf(-5.0f, fmaf(Qx, ey, Qy * ex), qxy)), v[7]);
    v[8] = fmaf(-iR5, fmaf(k175 * ex, ez, fmaf(-5.0f, fmaf(Qx, ez, Qz * ex), qxz)), v[8]);
    v[9] = fmaf(-iR5, fmaf(k175 * ey, ez, fmaf(-5.0f, fmaf(Qy, ez, Qz * ey), qyz)), v[9]);
  }
}

// Sums v[0..31] over the warp in 31 shuffles: lane k returns the total of v[k] (recursive halving: at each
// step a lane keeps the half of its values whose index bit matches its lane bit and adds its partner's copy).
__device__ __forceinline__ float warp_transpose_sum32(float v[32]) {
  const unsigned lane = threadIdx.x & 31u;
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    const bool up = (lane & (unsigned)off) != 0u;
#pragma unroll
    for (int k = 0; k < off; ++k) {
      const float send = up ? v[k] : v[k + off];
      const float keep = up ? v[k + off] : v[k];
      v[k] = keep + __shfl_xor_sync(SPH_FULL_MASK, send, off);
    }
  }
  return v[0];
}

// The expansion at offset y from its centre: a += −(g + H y + ½ T:yy), φ += φ0 + g·y + ½ yHy + ⅙ T:yyy.
template <bool PHI>
__device__ __forceinline__ void local_eval(const float cf[kLocal], float yx, float yy, float yz, float& ax,
                                           float& ay, float& az, float& phi) {
  const float hx = fmaf(cf[4], yx, fmaf(cf[7], yy, cf[8] * yz));
  const float hy = fmaf(cf[7], yx, fmaf(cf[5], yy, cf[9] * yz));
  const float hz = fmaf(cf[8], yx, fmaf(cf[9], yy, cf[6] * yz));
  const float xx = 0.5f * yx * yx, yy2 = 0.5f * yy * yy, zz = 0.5f * yz * yz;
  const float xy = yx * yy, xz = yx * yz, yz2 = yy * yz;
  const float tx = fmaf(cf[10], xx, fmaf(cf[15], yy2, fmaf(cf[17], zz, fmaf(cf[13], xy, fmaf(cf[14], xz, cf[19] * yz2)))));
  const float ty = fmaf(cf[13], xx, fmaf(cf[11], yy2, fmaf(cf[18], zz, fmaf(cf[15], xy, fmaf(cf[19], xz, cf[16] * yz2)))));
  const float tz = fmaf(cf[14], xx, fmaf(cf[16], yy2, fmaf(cf[12], zz, fmaf(cf[19], xy, fmaf(cf[17], xz, cf[18] * yz2)))));
  ax = -(cf[1] + hx + tx);
  ay = -(cf[2] + hy + ty);
  az = -(cf[3] + hz + tz);
  if (PHI) {
    // ⅙ T:yyy = ⅓ (y · (½ T:yy)), ½ yHy = ½ y·(H y)
    const float third = 1.0f / 3.0f;
    phi += cf[0] + fmaf(cf[1], yx, fmaf(cf[2], yy, cf[3] * yz)) + 0.5f * fmaf(yx, hx, fmaf(yy, hy, yz * hz)) +
           third * fmaf(yx, tx, fmaf(yy, ty, yz * tz));
  }
}

// What a gravity walk writes: the acceleration alone (a step's walk: the KDK integrator needs no potential),
// the acceleration and the potential φ, or φ alone (into .w of the gravity record, for the energy diagnostic
// of a state whose step walk left it out).
enum { kWalkAcc = 0, kWalkAccPhi = 1, kWalkPhi = 2 };

template <int W, bool GRAV, bool QUAD, bool NBR, bool HILO, int OUT>
__global__ void __launch_bounds__(W * 32, TW_WARPS_PER_SM / W) k_tree_walk(
    const float4* __restrict__ body, const float4* __restrict__ pos_h, const double* __restrict__ x64,
    const double* __restrict__ y64, const double* __restrict__ z64, int K, int L,
    const unsigned* __restrict__ leaf_start, const unsigned long long* __restrict__ leaf_codes,
    const Seg* __restrict__ segs, const unsigned* __restrict__ left, const unsigned* __restrict__ right,
    const float4* __restrict__ ncom, const float4* __restrict__ nbmin, const float4* __restrict__ nbmax, const float4* __restrict__ nq0,
    const float4* __restrict__ nq1, DevParams* P, float4* __restrict__ gout, unsigned* __restrict__ nbr,
    unsigned* __restrict__ nbr_cnt, unsigned cap, float skin, float* __restrict__ h0,
    const uint2* __restrict__ groups, const unsigned* __restrict__ ngroups, int stack_cap, float local_theta,
    int half, const float4* __restrict__ hcom, const float4* __restrict__ hq0, const float2* __restrict__ hq1,
    const float2* __restrict__ hrc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WalkSmem<W>& S = *reinterpret_cast<WalkSmem<W>*>(smem_raw);
  const int w = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const int warp = blockIdx.x * W + w;
  if (warp >= (int)*ngroups) return;
  // this warp's group: a run of <= 32 Morton-consecutive particles of one impact (leaves g.x..g.y); the walk
  // starts at that impact's root
  const uint2 grp = groups[warp];
  const int s0 = (int)leaf_start[grp.x], s1 = (int)leaf_start[grp.y + 1];
  const Seg& sgr = segs[(unsigned)(leaf_codes[grp.x] >> 30)];
  const unsigned root = sgr.root;
  const int t = s0 + (int)lane;
  const bool in_group = t < s1;
  const int tl = in_group ? t : s0;
  const float4 pi = pos_h[tl];  // x, y, z, h (same f32 coordinates as body)
  float xlo = 0.f, ylo = 0.f, zlo = 0.f;
  if (HILO && in_group) {
    xlo = (float)(x64[t] - (double)pi.x);
    ylo = (float)(y64[t] - (double)pi.y);
    zlo = (float)(z64[t] - (double)pi.z);
  }
  if (NBR && in_group && h0) h0[t] = pi.w;
  // Split the group where consecutive particles are far apart (a leaf bucket of K consecutive Morton
  // particles can straddle a jump of the curve, e.g. between two bodies): each part walks with its own
  // compact box, so one straddling bucket cannot turn the walk into an all-pairs sum. The cut is at gaps above
  // 6 h: a part costs one more traversal of the tree, and splitting closer (3 h) cut 15 % of the groups into
  // parts whose boxes overlap nearly as much as the whole group's did (walk 6 % slower on 1M and 4M impacts).
  const float px = __shfl_up_sync(SPH_FULL_MASK, pi.x, 1), py = __shfl_up_sync(SPH_FULL_MASK, pi.y, 1),
              pz = __shfl_up_sync(SPH_FULL_MASK, pi.z, 1), ph_ = __shfl_up_sync(SPH_FULL_MASK, pi.w, 1);
  const float gap2 = (pi.x - px) * (pi.x - px) + (pi.y - py) * (pi.y - py) + (pi.z - pz) * (pi.z - pz);
  const float hm = 6.0f * fmaxf(pi.w, ph_);
  const unsigned brk = __ballot_sync(SPH_FULL_MASK, lane > 0 && in_group && gap2 > hm * hm);
  const int nparts = __popc(brk) + 1;
  const int mypart = __popc(brk & ((2u << lane) - 1u));
  // a negative skin: the impact's current smoothing-length skin (device-maintained)
  if (NBR && skin < 0.0f) skin = sgr.skin;
  const float grow = (1.0f + skin) * (1.0f + 1.0e-5f);
  // the conservative neighbour test of a list with a skin: lim = ½(h_i + h_j)(1 + skin)(1 + 2^-19)
  const float lim_j = 0.5f * (1.0f + skin) * (1.0f + 1.9073486e-6f);
  const float lim_i = pi.w * lim_j;
  const float G = P->G, soft2 = sgr.soft2;
  const unsigned leaf0 = (unsigned)(L - 1);
  const unsigned lt = (1u << lane) - 1u;
  // staging of the pairwise lists: entries of K (near) or K/2 (far, when far leaves are split into halves)
  // sources, 32/K entries per 32-source chunk; K is a power of two in the group walk, so shifts, not divisions
  const int ksh = 31 - __clz(K);
  const int kfsh = half > 0 ? ksh - 1 : ksh;
  const int near_per = 32 >> ksh, near_li = (int)lane >> ksh, near_off = (int)lane & (K - 1);
  const int far_per = 32 >> kfsh, far_li = (int)lane >> kfsh, far_off = (int)lane & ((1 << kfsh) - 1);

  Acc3 acc;
  float phi = 0.f;
  // the packed sums of the far, near and multipole loops (two sources per FP32x2 instruction: half x for the
  // first source of each pair, half y for the second), folded into acc at the end
  float2 fx2 = make_float2(0.f, 0.f), fy2 = fx2, fz2 = fx2, fphi2 = fx2;
  unsigned cnt = 0;
  unsigned overflow = 0;
  unsigned* stack = S.stack[w];
  // per-warp counters, 32-bit (a warp's totals stay far below 2^32); the device totals are 64-bit
  unsigned st_visits = 0, st_pops = 0, st_m2p = 0, st_p2p = 0, st_m2l = 0, st_slots = 0;

  for (int part = 0; part < nparts; ++part) {
  const bool valid = in_group && mypart == part;
  const float big = 3.0e38f;
  const float gx0 = warp_min(valid ? pi.x : big), gy0 = warp_min(valid ? pi.y : big),
              gz0 = warp_min(valid ? pi.z : big);
  const float gx1 = warp_max(valid ? pi.x : -big), gy1 = warp_max(valid ? pi.y : -big),
              gz1 = warp_max(valid ? pi.z : -big);
  const float ghmax = warp_max(valid ? pi.w : 0.0f);
  // the part's local expansion: centre z, and the distance beyond which an accepted node's COM joins it
  const float zx = 0.5f * (gx0 + gx1), zy = 0.5f * (gy0 + gy1), zz = 0.5f * (gz0 + gz1);
  const float rg2 = 0.25f * ((gx1 - gx0) * (gx1 - gx0) + (gy1 - gy0) * (gy1 - gy0) + (gz1 - gz0) * (gz1 - gz0));
  const float far2 = (GRAV && local_theta > 0.0f) ? rg2 / (local_theta * local_theta) : big;
  float loc = 0.0f;  // lane k < kLocal: coefficient k of the part's expansion
  int sp = 1, nm = 0, np = 0, nf = 0, nl = 0;
  if (lane == 0) stack[0] = root;
  __syncwarp();

  // ---- far leaves: branch-free pairwise gravity, 32 staged sources per pass ---------------------------
  // The next chunk's sources are loaded into registers before this chunk is evaluated, so the gather
  // overlaps the arithmetic.
  // the part's interactions (counters of the walk statistics): multipole nodes, expanded nodes, pairwise
  // slots the lanes run (partial leaves padded) and the real sources among them
  unsigned part_m2p = 0, part_p2p = 0, part_m2l = 0, part_src = 0;
  auto far_source = [&](int base, int count, bool& real) {
    const int per = far_per, li = far_li, off = far_off;
    float4 src = make_float4(3.0e18f, 3.0e18f, 3.0e18f, 0.0f);  // padding: massless and far away
    real = false;
    if (li < min(per, count - base)) {
      const unsigned e = S.p2f[w][base + li];  // first source << 5 | (sources − 1)
      if (off <= (int)(e & 31u)) {
        src = body[(e >> 5) + off];
        real = true;
      }
    }
    return src;
  };
  // Without hi/lo coordinates the chunk is staged as 16 source pairs, (x₀ x₁ y₀ y₁) and (z₀ z₁ m₀ m₁) in two
  // consecutive float4, and each pair is evaluated with the packed FP32x2 operations of sm_100 (add, multiply
  // and fused multiply-add on two lanes of a register pair, each rounded as its scalar form): one instruction
  // does both sources' arithmetic, the reciprocal square roots stay scalar.
  auto flush_far = [&](int count) {
    const int per = far_per;
    part_p2p += (unsigned)count << kfsh;
    bool nreal;
    float4 nxt = far_source(0, count, nreal);
    for (int base = 0; base < count; base += per) {
      float4 src = nxt;
      part_src += __popc(__ballot_sync(SPH_FULL_MASK, nreal));
      if (base + per < count) nxt = far_source(base + per, count, nreal);
      src.w *= G;
      if (HILO) {
        S.src[w][lane] = src;
      } else {
        float* f = reinterpret_cast<float*>(&S.src[w][0]) + 8 * (lane >> 1) + (lane & 1u);
        f[0] = src.x;
        f[2] = src.y;
        f[4] = src.z;
        f[6] = src.w;
      }
      __syncwarp();
      if (valid && !HILO) {
        const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y),
                     npz = make_float2(-pi.z, -pi.z), s2 = make_float2(soft2, soft2);
#pragma unroll 4
        for (int k = 0; k < 16; ++k) {
          const float4 xy = S.src[w][2 * k], zm = S.src[w][2 * k + 1];
          const float2 dx = __fadd2_rn(make_float2(xy.x, xy.y), npx);
          const float2 dy = __fadd2_rn(make_float2(xy.z, xy.w), npy);
          const float2 dz = __fadd2_rn(make_float2(zm.x, zm.y), npz);
          const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, s2)));
          const float2 rinv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
          const float2 gm = __fmul2_rn(make_float2(zm.z, zm.w), rinv);
          const float2 g = __fmul2_rn(__fmul2_rn(gm, rinv), rinv);
          fx2 = __ffma2_rn(g, dx, fx2);
          fy2 = __ffma2_rn(g, dy, fy2);
          fz2 = __ffma2_rn(g, dz, fz2);
          if (OUT != kWalkAcc) fphi2 = __fadd2_rn(fphi2, make_float2(-gm.x, -gm.y));
        }
      }
      if (valid && HILO) {
#pragma unroll 4
        for (int k = 0; k < 32; ++k) {
          const float4 bj = S.src[w][k];
          float dx = bj.x - pi.x, dy = bj.y - pi.y, dz = bj.z - pi.z;
          if (HILO) { dx -= xlo; dy -= ylo; dz -= zlo; }
          const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, soft2)));
          const float rinv = rsqrt_ftz(r2);
          const float gm = bj.w * rinv;
          const float g = gm * rinv * rinv;
          acc.add<HILO>(g * dx, g * dy, g * dz);
          if (OUT != kWalkAcc) phi -= gm;
        }
      }
      __syncwarp();
    }
  };

  // A multipole-list entry: a node index, or a half leaf (bit 31 set, index 2·leaf + half).
  auto load_multipole = [&](unsigned e, float4& c, float4& q0, float2& q1) {
    q0 = make_float4(0.f, 0.f, 0.f, 0.f);
    q1 = make_float2(0.f, 0.f);
    if (e & 0x80000000u) {
      const unsigned hi = e & 0x7fffffffu;
      c = hcom[hi];
      if (QUAD) {
        q0 = hq0[hi];
        q1 = hq1[hi];
      }
    } else {
      c = ncom[e];
      if (QUAD) {
        q0 = nq0[e];
        const float4 b = nq1[e];
        q1 = make_float2(b.x, b.y);
      }
    }
  };

  // ---- far multipoles: each lane expands its own node about z, the warp sums the coefficients -------------
  auto flush_m2l = [&](int count) {
    for (int base = 0; base < count; base += 32) {
      float v[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) v[k] = 0.0f;
      if ((int)lane < count - base) {
        float4 c, q0;
        float2 q1;
        load_multipole(S.m2l[w][base + lane], c, q0, q1);
        local_coeffs<QUAD>(c, q0, q1, G, zx, zy, zz, soft2, v);
      }
      loc += warp_transpose_sum32(v);
    }
  };

  // ---- multipole list: stage 32 nodes in shared memory, then every lane applies them -------------------
  // Without hi/lo coordinates the nodes are staged in pairs, (x₀ x₁ y₀ y₁)(z₀ z₁ m₀ m₁) in src,
  // (Qxx Qyy)(Qzz Qxy) pairs in q0 and (Qxz Qyz) pairs in q1, and evaluated two at a time with the packed
  // FP32x2 operations; an odd chunk is padded with a massless node far away.
  auto flush_m2p = [&](int count) {
    for (int base = 0; base < count; base += 32) {
      const int m = min(32, count - base);
      if (HILO) {
        if ((int)lane < m) {
          // staged with G folded in: (com, G·M) and G·Q
          float4 c, q;
          float2 b;
          load_multipole(S.m2p[w][base + lane], c, q, b);
          c.w *= G;
          S.src[w][lane] = c;
          if (QUAD) {
            S.q0[w][lane] = make_float4(G * q.x, G * q.y, G * q.z, G * q.w);
            S.q1[w][lane] = make_float2(G * b.x, G * b.y);
          }
        }
      } else if ((int)lane < ((m + 1) & ~1)) {
        float4 c = make_float4(3.0e18f, 3.0e18f, 3.0e18f, 0.0f), q = make_float4(0.f, 0.f, 0.f, 0.f);
        float2 b = make_float2(0.f, 0.f);
        if ((int)lane < m) load_multipole(S.m2p[w][base + lane], c, q, b);
        float* f = reinterpret_cast<float*>(&S.src[w][0]) + 8 * (lane >> 1) + (lane & 1u);
        f[0] = c.x;
        f[2] = c.y;
        f[4] = c.z;
        f[6] = G * c.w;
        if (QUAD) {
          float* g0 = reinterpret_cast<float*>(&S.q0[w][0]) + 8 * (lane >> 1) + (lane & 1u);
          g0[0] = G * q.x;
          g0[2] = G * q.y;
          g0[4] = G * q.z;
          g0[6] = G * q.w;
          float* g1 = reinterpret_cast<float*>(&S.q1[w][0]) + 4 * (lane >> 1) + (lane & 1u);
          g1[0] = G * b.x;
          g1[2] = G * b.y;
        }
      }
      __syncwarp();
      if (valid && !HILO) {
        const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y),
                     npz = make_float2(-pi.z, -pi.z), s2 = make_float2(soft2, soft2);
        const float4* q1p = reinterpret_cast<const float4*>(&S.q1[w][0]);
        const int mp = (m + 1) >> 1;
        for (int k = 0; k < mp; ++k) {
          const float4 xy = S.src[w][2 * k], zm = S.src[w][2 * k + 1];
          const float2 dx = __fadd2_rn(make_float2(xy.x, xy.y), npx);
          const float2 dy = __fadd2_rn(make_float2(xy.z, xy.w), npy);
          const float2 dz = __fadd2_rn(make_float2(zm.x, zm.y), npz);
          const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, s2)));
          const float2 rinv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
          const float2 rinv2 = __fmul2_rn(rinv, rinv);
          const float2 mm = make_float2(zm.z, zm.w);
          const float2 gm = __fmul2_rn(mm, rinv);  // G M / R
          const float2 g = __fmul2_rn(gm, rinv2);  // G M / R³
          if (QUAD) {
            // as the scalar form below: a = d (G M/R³ + 5/2 eᵀQe/R⁵) − Q e/R⁴, φ = −G M/R − ½ eᵀQe/R³
            const float4 qa = S.q0[w][2 * k], qb = S.q0[w][2 * k + 1], qc = q1p[k];
            const float2 qxx = make_float2(qa.x, qa.y), qyy = make_float2(qa.z, qa.w);
            const float2 qzz = make_float2(qb.x, qb.y), qxy = make_float2(qb.z, qb.w);
            const float2 qxz = make_float2(qc.x, qc.y), qyz = make_float2(qc.z, qc.w);
            const float2 ex = __fmul2_rn(dx, rinv), ey = __fmul2_rn(dy, rinv), ez = __fmul2_rn(dz, rinv);
            const float2 Qex = __ffma2_rn(qxz, ez, __ffma2_rn(qxy, ey, __fmul2_rn(qxx, ex)));
            const float2 Qey = __ffma2_rn(qyz, ez, __ffma2_rn(qyy, ey, __fmul2_rn(qxy, ex)));
            const float2 Qez = __ffma2_rn(qzz, ez, __ffma2_rn(qyz, ey, __fmul2_rn(qxz, ex)));
            const float2 eQe = __ffma2_rn(ez, Qez, __ffma2_rn(ey, Qey, __fmul2_rn(ex, Qex)));
            const float2 rinv4 = __fmul2_rn(rinv2, rinv2);
            const float2 nr4 = make_float2(-rinv4.x, -rinv4.y);
            const float2 c1 = __ffma2_rn(__fmul2_rn(make_float2(2.5f, 2.5f), eQe), __fmul2_rn(rinv4, rinv), g);
            fx2 = __ffma2_rn(nr4, Qex, __ffma2_rn(c1, dx, fx2));
            fy2 = __ffma2_rn(nr4, Qey, __ffma2_rn(c1, dy, fy2));
            fz2 = __ffma2_rn(nr4, Qez, __ffma2_rn(c1, dz, fz2));
            if (OUT != kWalkAcc) {
              const float2 t = __ffma2_rn(__fmul2_rn(make_float2(0.5f, 0.5f), eQe), rinv2, mm);
              fphi2 = __ffma2_rn(make_float2(-t.x, -t.y), rinv, fphi2);
            }
          } else {
            fx2 = __ffma2_rn(g, dx, fx2);
            fy2 = __ffma2_rn(g, dy, fy2);
            fz2 = __ffma2_rn(g, dz, fz2);
            if (OUT != kWalkAcc) fphi2 = __fadd2_rn(fphi2, make_float2(-gm.x, -gm.y));
          }
        }
      }
      if (valid && HILO) {
        for (int k = 0; k < m; ++k) {
          const float4 c = S.src[w][k];
          float dx = c.x - pi.x, dy = c.y - pi.y, dz = c.z - pi.z;
          if (HILO) { dx -= xlo; dy -= ylo; dz -= zlo; }
          const float r2 = dx * dx + dy * dy + dz * dz + soft2;
          const float rinv = rsqrt_ftz(r2);
          const float rinv2 = rinv * rinv;
          const float gm = c.w * rinv;           // G M / R
          const float g = gm * rinv2;            // G M / R³
          if (QUAD) {
            // a = G M d/R³ + (G/R⁴)(5/2 (eᵀQe) e − Q e), e = d/R (unit vector: Q·e and eᵀQe stay in f32 range
            // in SI units) = d (G M/R³ + 5/2 eᵀQe/R⁵) − Q e/R⁴;  φ = −G M/R − ½ eᵀQe/R³
            const float4 a0 = S.q0[w][k];
            const float2 a1 = S.q1[w][k];
            const float ex = dx * rinv, ey = dy * rinv, ez = dz * rinv;
            const float Qex = a0.x * ex + a0.w * ey + a1.x * ez;
            const float Qey = a0.w * ex + a0.y * ey + a1.y * ez;
            const float Qez = a1.x * ex + a1.y * ey + a0.z * ez;
            const float eQe = ex * Qex + ey * Qey + ez * Qez;
            const float rinv4 = rinv2 * rinv2;
            const float c1 = fmaf(2.5f * eQe, rinv4 * rinv, g);
            if (HILO) {
              acc.add<HILO>(c1 * dx - rinv4 * Qex, c1 * dy - rinv4 * Qey, c1 * dz - rinv4 * Qez);
            } else {  // two fused multiply-adds per axis straight into the sums
              acc.x = fmaf(-rinv4, Qex, fmaf(c1, dx, acc.x));
              acc.y = fmaf(-rinv4, Qey, fmaf(c1, dy, acc.y));
              acc.z = fmaf(-rinv4, Qez, fmaf(c1, dz, acc.z));
            }
            if (OUT != kWalkAcc) phi = fmaf(-fmaf(0.5f * eQe, rinv2, c.w), rinv, phi);
          } else {
            acc.add<HILO>(g * dx, g * dy, g * dz);
            if (OUT != kWalkAcc) phi -= gm;
          }
        }
      }
      __syncwarp();
    }
  };

  // ---- direct list: leaves of <= K sources (K divides 32), 32 sources per chunk ------------------------
  auto near_source = [&](int base, int count, float4& src, float& hsrc) {
    const int per = near_per, li = near_li, off = near_off;  // leaves per chunk, this lane's leaf and source
    int sidx = -1;
    if (li < min(per, count - base)) {
      const unsigned e = S.p2p[w][base + li];  // first source << 5 | (sources − 1)
      if (off <= (int)(e & 31u)) sidx = (int)(e >> 5) + off;
    }
    src = make_float4(3.0e18f, 3.0e18f, 3.0e18f, 0.0f);  // padding: massless and far away
    hsrc = 0.0f;
    if (sidx >= 0) {
      src = body[sidx];
      if (NBR) hsrc = pos_h[sidx].w;
    }
    return sidx;
  };
  // The neighbour test and the append of one source that passed it (the list keeps the chunk's order).
  // (the particle's first list slot once, entries 32 apart: the interleaved layout of nbr_slot)
  unsigned* const nlst = NBR ? nbr + nbr_slot((unsigned)t, 0u, cap) : nullptr;
  auto near_append = [&](bool inside, int s) {
    if (inside) {
      if (cnt < cap) nlst[(size_t)cnt * 32u] = (unsigned)s;
      ++cnt;
    }
  };
  // Without hi/lo coordinates: sources in pairs, as in the far loop (the pair (x₀ x₁ y₀ y₁)(z₀ z₁ m₀ m₁) and
  // (index₀ index₁ h₀ h₁)); every packed operation rounds as its scalar form, so the distances and the
  // predicate are those of the scalar loop below, source by source.
  auto near_pairs = [&](auto loose) {
    const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y), npz = make_float2(-pi.z, -pi.z);
    const float2 s2 = make_float2(soft2, soft2);
    const float4* shp = reinterpret_cast<const float4*>(&S.sh[w][0]);
#pragma unroll 2
    for (int k = 0; k < 16; ++k) {
      const float4 xy = S.src[w][2 * k], zm = S.src[w][2 * k + 1], sh = shp[k];
      const int sa = __float_as_int(sh.x), sb = __float_as_int(sh.y);
      const bool oa = sa != t, ob = sb != t;
      const float2 dx = __fadd2_rn(make_float2(xy.x, xy.y), npx);
      const float2 dy = __fadd2_rn(make_float2(xy.z, xy.w), npy);
      const float2 dz = __fadd2_rn(make_float2(zm.x, zm.y), npz);
      float2 dd;
      if constexpr (decltype(loose)::value) dd = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
      else dd = __fadd2_rn(__fadd2_rn(__fmul2_rn(dx, dx), __fmul2_rn(dy, dy)), __fmul2_rn(dz, dz));
      if (NBR) {
        bool ia, ib;
        if constexpr (decltype(loose)::value) {
          const float2 lim = __ffma2_rn(make_float2(sh.z, sh.w), make_float2(lim_j, lim_j), make_float2(lim_i, lim_i));
          const float2 l2 = __fmul2_rn(lim, lim);
          ia = dd.x < l2.x;
          ib = dd.y < l2.y;
        } else {
          const float2 lim = __fmul2_rn(make_float2(0.5f, 0.5f), __fadd2_rn(make_float2(pi.w, pi.w), make_float2(sh.z, sh.w)));
          const float2 q = __fmul2_rn(lim, lim);
          const float2 qlo = __fmul2_rn(q, make_float2(1.0f - 1.9073486e-6f, 1.0f - 1.9073486e-6f));
          const float2 qhi = __fmul2_rn(q, make_float2(1.0f + 1.9073486e-6f, 1.0f + 1.9073486e-6f));
          ia = dd.x < qlo.x;
          if (!ia && !(dd.x > qhi.x)) ia = fsqrt(dd.x) < lim.x;
          ib = dd.y < qlo.y;
          if (!ib && !(dd.y > qhi.y)) ib = fsqrt(dd.y) < lim.y;
        }
        near_append(oa && ia, sa);
        near_append(ob && ib, sb);
      }
      if (GRAV) {
        // the particle itself (d = 0) gets r² = 1: a finite g times a zero offset adds nothing
        const float2 r2s = __fadd2_rn(dd, s2);
        const float2 r2 = make_float2(oa ? r2s.x : 1.0f, ob ? r2s.y : 1.0f);
        const float2 rinv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
        const float2 gm = __fmul2_rn(make_float2(zm.z, zm.w), rinv);
        const float2 g = __fmul2_rn(__fmul2_rn(gm, rinv), rinv);
        fx2 = __ffma2_rn(g, dx, fx2);
        fy2 = __ffma2_rn(g, dy, fy2);
        fz2 = __ffma2_rn(g, dz, fz2);
        if (OUT != kWalkAcc) fphi2 = __fadd2_rn(fphi2, make_float2(oa ? -gm.x : 0.0f, ob ? -gm.y : 0.0f));
      }
    }
  };
  auto near_sources = [&](auto loose) {
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const float2 shk = S.sh[w][k];
      const int s = __float_as_int(shk.x);
      // padding (s = −1) sits massless at 3e18: it passes no neighbour test and adds no gravity
      const bool other = s != t;
      const float4 bj = S.src[w][k];
      const float dx = fsub(bj.x, pi.x), dy = fsub(bj.y, pi.y), dz = fsub(bj.z, pi.z);
      // the exact predicate needs the single-rounded distance; the conservative one's 2^-19 margin is far above
      // the few ulp a fused form differs by
      const float dd = decltype(loose)::value ? fmaf(dz, dz, fmaf(dy, dy, dx * dx)) : dot3_exact(dx, dy, dz);
      if (NBR && other) {
        bool inside;
        if constexpr (decltype(loose)::value) {
          const float lim = fmaf(shk.y, lim_j, lim_i);
          inside = dd < lim * lim;
        } else {
          const float lim = fmul(0.5f, fadd(pi.w, shk.y));
          // sqrt_rn(dd) < lim, decided without the square root outside a 2^-19 band around lim²:
          // dd < lim²(1-2^-19) ⇒ √dd < lim − 2 ulp(lim); dd > lim²(1+2^-19) ⇒ √dd > lim + 2 ulp(lim)
          const float q = fmul(lim, lim);
          inside = dd < fmul(q, 1.0f - 1.9073486e-6f);
          if (!inside && !(dd > fmul(q, 1.0f + 1.9073486e-6f))) inside = fsqrt(dd) < lim;
        }
        near_append(inside, s);
      }
      if (GRAV) {
        float ex = dx, ey = dy, ez = dz, d2 = dd;
        if (HILO) {
          ex -= xlo;
          ey -= ylo;
          ez -= zlo;
          d2 = ex * ex + ey * ey + ez * ez;
        }
        // the particle itself (d = 0) gets r² = 1: a finite g times a zero offset adds nothing (with hi/lo
        // coordinates its offset is −lo, so there the mass is masked)
        const float r2 = other ? d2 + soft2 : 1.0f;
        const float rinv = rsqrt_ftz(r2);
        const float gm = (HILO && !other) ? 0.0f : bj.w * rinv;
        const float g = gm * rinv * rinv;
        acc.add<HILO>(g * ex, g * ey, g * ez);
        if (OUT != kWalkAcc && other) phi -= gm;
      }
    }
  };
  auto flush_p2p = [&](int count) {
    const int per = near_per;  // leaves per chunk
    float4 nsrc;
    float nh;
    part_p2p += (unsigned)count << ksh;
    int nidx = near_source(0, count, nsrc, nh);
    for (int base = 0; base < count; base += per) {
      float4 src = nsrc;
      const float hsrc = nh;
      const int sidx = nidx;
      part_src += __popc(__ballot_sync(SPH_FULL_MASK, sidx >= 0));
      if (base + per < count) nidx = near_source(base + per, count, nsrc, nh);
      src.w *= G;
      if (HILO) {
        S.src[w][lane] = src;
        S.sh[w][lane] = make_float2(__int_as_float(sidx), hsrc);
      } else {
        float* f = reinterpret_cast<float*>(&S.src[w][0]) + 8 * (lane >> 1) + (lane & 1u);
        f[0] = src.x;
        f[2] = src.y;
        f[4] = src.z;
        f[6] = src.w;
        float* e = reinterpret_cast<float*>(&S.sh[w][0]) + 4 * (lane >> 1) + (lane & 1u);
        e[0] = __int_as_float(sidx);
        e[2] = hsrc;
      }
      __syncwarp();
      if (valid && !HILO) {
        if (NBR && skin > 0.0f) near_pairs(std::true_type{});
        else near_pairs(std::false_type{});
      }
      if (valid && HILO) {
        // A list built with a skin is a candidate set: the gather kernels keep r < h_ij at the current h,
        // and the smoothing-length solve holds h below h0·(1 + skin)·0.999, so every superset of the exact
        // predicate gives the same sums in the same order. With a skin the test is therefore a conservative
        // one (lim padded by 2^-19, more than the rounding of either form); without one (fixed h) it is the
        // reference's exact predicate.
        if (NBR && skin > 0.0f) near_sources(std::true_type{});
        else near_sources(std::false_type{});
      }
      __syncwarp();
    }
  };

  const unsigned nvalid = __popc(__ballot_sync(SPH_FULL_MASK, valid));
  // One pass per pop; the pass after the stack empties flushes what the lists still hold, so that every flush
  // loop has one call site (the walk's hot code is instruction-cache bound: a second inlined copy of each flush
  // loop measurably stalled instruction fetch). With half leaves a pass is of one of two kinds: a pop of up to
  // 32 nodes, whose far leaves are queued (S.hl), or a batch of up to 32 queued far leaves whose halves are
  // classified, one leaf per lane. Classifying halves in the pop that found the leaf ran that code once per pop
  // with a few lanes active; batched, it runs once per 32 leaves.
  int nq = 0;  // far leaves queued for the half classification
  for (;;) {
  const bool halves = GRAV && half > 0 && (nq >= 32 || (sp == 0 && nq > 0));
  const bool done = sp == 0 && nq == 0;
  if (!done) {
    // Entries of this lane: a node for the multipole lists (m0 per particle, l0 into the group's expansion), a
    // near leaf, a far leaf (or, with half leaves, a far leaf queued), and in a batch of queued leaves up to
    // two of each kind, one per half: a half accepted as a multipole when the MAC holds for its own moments,
    // else its <= half sources go to the far list.
    bool m0 = false, m1 = false, l0 = false, l1 = false, f0 = false, f1 = false, near_leaf = false, open = false,
         queue = false;
    unsigned v0 = 0u, v1 = 0u;                      // multipole entries
    unsigned fe0 = 0u, fe1 = 0u;                    // far entries: first << 5 | (count − 1)
    unsigned ls0 = 0u, ls1 = 1u;                    // a leaf's source range
    unsigned lc = 0u, rc = 0u;                      // an internal node's children, loaded alongside its box
    unsigned node = 0u;
    if (halves) {
      const int take = min(nq, 32);
      nq -= take;
      const bool have = (int)lane < take;
      const unsigned cl = have ? S.hl[w][nq + (int)lane] : 0u;
      __syncwarp();
      if (have) {
        ls0 = leaf_start[cl];
        ls1 = leaf_start[cl + 1];
        const unsigned mid = ls0 + (unsigned)half;
        const float2 rch = hrc[cl];
        const unsigned nh = ls1 > mid ? 2u : 1u;
        const float4 hA = hcom[2u * cl], hB = hcom[2u * cl + 1u];
        unsigned hf = 0u;  // bit b: half b passes the MAC; bit 2 + b: ... and lies far enough for the expansion
#pragma unroll 1
        for (unsigned b = 0; b < nh; ++b) {
          const float4 hc = b ? hB : hA;
          const float ddx = fmaxf(fmaxf(gx0 - hc.x, hc.x - gx1), 0.0f);
          const float ddy = fmaxf(fmaxf(gy0 - hc.y, hc.y - gy1), 0.0f);
          const float ddz = fmaxf(fmaxf(gz0 - hc.z, hc.z - gz1), 0.0f);
          const float ro = (b ? rch.y : rch.x) * 1.00001f;
          const bool mac_h = ddx * ddx + ddy * ddy + ddz * ddz + soft2 >= ro * ro;
          const float ux = hc.x - zx, uy = hc.y - zy, uz = hc.z - zz;
          const bool far_h = ux * ux + uy * uy + uz * uz >= far2;
          hf |= (mac_h ? 1u : 0u) << b;
          hf |= (mac_h && far_h ? 1u : 0u) << (2u + b);
        }
        m0 = (hf & 5u) == 1u;
        l0 = (hf & 4u) != 0u;
        f0 = (hf & 1u) == 0u;
        v0 = 0x80000000u | (2u * cl);
        fe0 = (ls0 << 5) | (min(ls1, mid) - ls0 - 1u);
        if (nh == 2u) {
          m1 = (hf & 10u) == 2u;
          l1 = (hf & 8u) != 0u;
          f1 = (hf & 2u) == 0u;
          v1 = 0x80000000u | (2u * cl + 1u);
          fe1 = (mid << 5) | (ls1 - mid - 1u);
        }
      }
    } else {
      const int take = min(sp, 32);
      sp -= take;
      st_visits += take;
      ++st_pops;
      const bool have = (int)lane < take;
      node = have ? stack[sp + lane] : 0u;
      __syncwarp();
      bool acc_node = false, leaf = false, far_l = false;
      float4 lbl = make_float4(0.f, 0.f, 0.f, 0.f), lbh = lbl;  // the node's box (and max h), for the lane test
      if (have) {
        const float4 bl = nbmin[node], bh = nbmax[node];
        lbl = bl;
        lbh = bh;
        const bool is_leaf = node >= leaf0;
        if (is_leaf) {
          ls0 = leaf_start[node - leaf0];
          ls1 = leaf_start[node - leaf0 + 1];
        } else {
          lc = left[node];
          rc = right[node];
        }
        bool near = false;
        {
          // SPH reach (or, for gravity alone, plain overlap with the group box so that a group's own leaves
          // take the careful path that skips self-pairs)
          const float reach = NBR ? 0.5f * (ghmax + bl.w) * grow : 0.0f;
          near = (bl.x - reach <= gx1) && (bh.x + reach >= gx0) && (bl.y - reach <= gy1) &&
                 (bh.y + reach >= gy0) && (bl.z - reach <= gz1) && (bh.z + reach >= gz0);
        }
        bool mac = false;
        if (GRAV) {
          // leaves carry their own moments and may be accepted as well
          const float4 c = ncom[node];
          // distance from the COM to the nearest point of the group box
          const float ddx = fmaxf(fmaxf(gx0 - c.x, c.x - gx1), 0.0f);
          const float ddy = fmaxf(fmaxf(gy0 - c.y, c.y - gy1), 0.0f);
          const float ddz = fmaxf(fmaxf(gz0 - c.z, c.z - gz1), 0.0f);
          // sqrt(d² + ε²) >= r_open, compared squared (both sides are non-negative; no square root per node)
          const float ro = bh.w * 1.00001f;
          mac = ddx * ddx + ddy * ddy + ddz * ddz + soft2 >= ro * ro;
          const float ux = c.x - zx, uy = c.y - zy, uz = c.z - zz;
          far_l = ux * ux + uy * uy + uz * uz >= far2;
        }
        if (mac && !near) acc_node = true;
        else if (is_leaf) leaf = GRAV || near;
        else open = GRAV || (NBR && near);
        if (is_leaf && ls1 <= ls0) acc_node = leaf = false;  // an empty leaf (none are built) adds nothing
        near_leaf = leaf && near;
      }
      if (NBR && GRAV) {
        // A leaf near the group box may still be out of every particle's own reach: then it can hold no
        // neighbour and takes the cheaper far path. The test is conservative (reach with the list's skin and a
        // margin), and a leaf holding a particle of the part is at distance 0, so self-pairs stay on the near
        // path.
        const unsigned cand = __ballot_sync(SPH_FULL_MASK, near_leaf);
        unsigned keep = 0;
        for (unsigned b = cand; b; b &= b - 1) {
          const int k = __ffs(b) - 1;
          const float x0 = __shfl_sync(SPH_FULL_MASK, lbl.x, k), y0 = __shfl_sync(SPH_FULL_MASK, lbl.y, k),
                      z0 = __shfl_sync(SPH_FULL_MASK, lbl.z, k), hm = __shfl_sync(SPH_FULL_MASK, lbl.w, k);
          const float x1 = __shfl_sync(SPH_FULL_MASK, lbh.x, k), y1 = __shfl_sync(SPH_FULL_MASK, lbh.y, k),
                      z1 = __shfl_sync(SPH_FULL_MASK, lbh.z, k);
          const float ex = fmaxf(fmaxf(x0 - pi.x, pi.x - x1), 0.0f),
                      ey = fmaxf(fmaxf(y0 - pi.y, pi.y - y1), 0.0f),
                      ez = fmaxf(fmaxf(z0 - pi.z, pi.z - z1), 0.0f);
          const float r = 0.5f * (pi.w + hm) * grow * 1.0001f;
          if (__any_sync(SPH_FULL_MASK, valid && ex * ex + ey * ey + ez * ez <= r * r)) keep |= 1u << k;
        }
        if (near_leaf && !((keep >> lane) & 1u)) near_leaf = false;
      }
      m0 = acc_node && !far_l;
      l0 = acc_node && far_l;
      v0 = node;
      const bool far_leaf = leaf && !near_leaf;
      queue = GRAV && half > 0 && far_leaf;  // its halves are classified in a later batch
      f0 = far_leaf && !queue;
      fe0 = (ls0 << 5) | min(ls1 - ls0 - 1u, 31u);
    }
    const unsigned bm0 = __ballot_sync(SPH_FULL_MASK, m0), bm1 = __ballot_sync(SPH_FULL_MASK, m1);
    const unsigned bl0 = __ballot_sync(SPH_FULL_MASK, l0), bl1 = __ballot_sync(SPH_FULL_MASK, l1);
    const unsigned bf0 = __ballot_sync(SPH_FULL_MASK, f0), bf1 = __ballot_sync(SPH_FULL_MASK, f1);
    const unsigned bo = __ballot_sync(SPH_FULL_MASK, open);
    const unsigned bn = __ballot_sync(SPH_FULL_MASK, near_leaf);
    const unsigned bq = __ballot_sync(SPH_FULL_MASK, queue);
    if (queue) S.hl[w][nq + __popc(bq & lt)] = node - leaf0;
    nq += __popc(bq);
    // two entries per lane: lanes below this one come first, then this lane's first and second entry
    if (m0 || m1) {
      const int k = nm + __popc(bm0 & lt) + __popc(bm1 & lt);
      if (m0) S.m2p[w][k] = v0;
      if (m1) S.m2p[w][k + (m0 ? 1 : 0)] = v1;
    }
    if (l0 || l1) {
      const int k = nl + __popc(bl0 & lt) + __popc(bl1 & lt);
      if (l0) S.m2l[w][k] = v0;
      if (l1) S.m2l[w][k + (l0 ? 1 : 0)] = v1;
    }
    if (f0 || f1) {
      const int k = nf + __popc(bf0 & lt) + __popc(bf1 & lt);
      if (f0) S.p2f[w][k] = fe0;
      if (f1) S.p2f[w][k + (f0 ? 1 : 0)] = fe1;
    }
    // list entries carry the leaf's source range (capacity <= 2^26 particles, leaves <= 32 sources)
    if (near_leaf) S.p2p[w][np + __popc(bn & lt)] = (ls0 << 5) | min(ls1 - ls0 - 1u, 31u);
    const int no = __popc(bo);
    if (sp + 2 * no <= stack_cap) {
      if (open) {
        const int r = sp + 2 * __popc(bo & lt);
        stack[r] = lc;
        stack[r + 1] = rc;
      }
      sp += 2 * no;
    } else if (no) {
      overflow = 1;
    }
    nm += __popc(bm0) + __popc(bm1);
    nl += __popc(bl0) + __popc(bl1);
    np += __popc(bn);
    nf += __popc(bf0) + __popc(bf1);
    part_m2p += __popc(bm0) + __popc(bm1);
    part_m2l += __popc(bl0) + __popc(bl1);
  }  // !done
    __syncwarp();
    if (nm > TW_LIST - 64 || (done && nm)) {
      flush_m2p(nm);
      nm = 0;
    }
    if (nl > TW_LIST - 64 || (done && nl)) {
      flush_m2l(nl);
      nl = 0;
    }
    if (np > TW_LIST - 64 || (done && np)) {
      flush_p2p(np);
      np = 0;
    }
    if (nf > TW_LIST - 64 || (done && nf)) {
      flush_far(nf);
      nf = 0;
    }
    if (done) break;
  }
  if (GRAV && part_m2l) {
    // the part's expansion (lane k holds coefficient k) evaluated by every particle of the part
    float cf[kLocal];
#pragma unroll
    for (int k = 0; k < kLocal; ++k) cf[k] = __shfl_sync(SPH_FULL_MASK, loc, k);
    if (valid) {
      float yx = pi.x - zx, yy = pi.y - zy, yz = pi.z - zz;
      if (HILO) { yx += xlo; yy += ylo; yz += zlo; }
      float lx, ly, lz;
      local_eval<OUT != kWalkAcc>(cf, yx, yy, yz, lx, ly, lz, phi);
      acc.add<HILO>(lx, ly, lz);
    }
  }
  st_m2p += part_m2p * nvalid;                             // node × particle interactions
  st_m2l += part_m2l;                                      // nodes expanded about a part's centre
  st_p2p += part_src * nvalid;                             // source particles × particles
  st_slots += part_p2p * nvalid;                           // ... counting the slots the lanes ran
  }  // parts

  if (in_group && GRAV) {
    if (!HILO) {
      acc.add<false>(fx2.x + fx2.y, fy2.x + fy2.y, fz2.x + fz2.y);
      phi += fphi2.x + fphi2.y;
    }
    if (OUT == kWalkPhi) reinterpret_cast<float*>(gout)[4 * (size_t)t + 3] = phi;
    else gout[t] = make_float4(acc.x, acc.y, acc.z, OUT == kWalkAccPhi ? phi : 0.0f);
  }
  if (NBR) {
    if (in_group) nbr_cnt[t] = cnt;
    const unsigned wmax = warp_max(in_group ? cnt : 0u);
    if (lane == 0) {
      atomicMax(&P->max_nbr_seen, wmax);
      if (wmax > cap) atomicOr(&P->flags, kFlagNbrOverflow);
    }
  }
  if (overflow && lane == 0) atomicOr(&P->flags, kFlagStackOverflow);
  if (lane == 0 && OUT != kWalkPhi) {  // a diagnostic's potential walk is not a step's walk
    atomicAdd(&P->stat_visits, (unsigned long long)st_visits);
    atomicAdd(&P->stat_pops, (unsigned long long)st_pops);
    atomicAdd(&P->stat_m2p, (unsigned long long)st_m2p);
    atomicAdd(&P->stat_p2p, (unsigned long long)st_p2p);
    atomicAdd(&P->stat_m2l, (unsigned long long)st_m2l);
    atomicAdd(&P->stat_p2p_slots, (unsigned long long)st_slots);
  }
}

template <int W, bool GRAV, bool QUAD, bool NBR, bool HILO, int OUT>
static void walk(const Dev& d, const Cfg& c, cudaStream_t s) {
  const int warps = d.L;  // upper bound on the number of groups
  const int blocks = (warps + W - 1) / W;
  const size_t smem = sizeof(WalkSmem<W>);
  static std::atomic<unsigned long long> attr{0};
  smem_limit_per_device(k_tree_walk<W, GRAV, QUAD, NBR, HILO, OUT>, (int)smem, attr);
  const State& st = d.s();
  k_tree_walk<W, GRAV, QUAD, NBR, HILO, OUT><<<blocks, W * 32, smem, s>>>(
      d.body, st.pos_h, st.x, st.y, st.z, d.K, d.L, d.leaf_start, d.leaf_codes, d.segs, d.left, d.right, d.ncom,
      d.nbmin, d.nbmax, d.nq0, d.nq1, d.P, d.grav, d.nbr, d.nbr_cnt, d.nbr_cap, c.h_solve ? -1.0f : c.nbr_skin,
      d.h0, d.groups, d.ngroups, c.walk_stack > 0 && c.walk_stack < TW_STACK ? c.walk_stack : TW_STACK,
      GRAV ? c.local_theta : 0.0f, GRAV ? half_leaf(d, c) : 0, d.hcom, d.hq0, d.hq1, d.hrc);
}

// Gravity (group MAC) fused with the neighbour lists; the traversal tile (warps per block) is a tuning choice.
template <bool QUAD, int OUT>
static void walk_fused(const Dev& d, const Cfg& c, cudaStream_t s) {
  if (c.hilo) {
    walk<4, true, QUAD, true, true, OUT>(d, c, s);
    return;
  }
  switch (c.walk_warps) {
    case 4: walk<4, true, QUAD, true, false, OUT>(d, c, s); break;
    case 8: walk<8, true, QUAD, true, false, OUT>(d, c, s); break;
    default: walk<2, true, QUAD, true, false, OUT>(d, c, s); break;
  }
}

int launch_walk(const Dev& d, const Cfg& c, bool potential, cudaStream_t s) {
  if (potential) {
    if (c.quad) walk_fused<true, kWalkAccPhi>(d, c, s);
    else walk_fused<false, kWalkAccPhi>(d, c, s);
  } else {
    if (c.quad) walk_fused<true, kWalkAcc>(d, c, s);
    else walk_fused<false, kWalkAcc>(d, c, s);
  }
  return 1;
}

// The potential alone, into .w of the gravity record, on the tree of the last evaluation (the energy
// diagnostic after steps whose walks left it out). The group MAC and quadrupoles of the step's walk; without
// the neighbour lists a node is near only when it overlaps the part's box.
int launch_potential(const Dev& d, const Cfg& c, cudaStream_t s) {
  if (c.hilo) {
    if (c.quad) walk<4, true, true, false, true, kWalkPhi>(d, c, s);
    else walk<4, true, false, false, true, kWalkPhi>(d, c, s);
  } else {
    if (c.quad) walk<4, true, true, false, false, kWalkPhi>(d, c, s);
    else walk<4, true, false, false, false, kWalkPhi>(d, c, s);
  }
  return 1;
}

// Gravity only (group MAC), for point sets without SPH.
int launch_gravity_group(const Dev& d, const Cfg& c, cudaStream_t s) {
  if (c.quad) walk<4, true, true, false, false, kWalkAccPhi>(d, c, s);
  else walk<4, true, false, false, false, kWalkAccPhi>(d, c, s);
  return 1;
}

// Neighbour lists only (when gravity is not the tree).
int launch_neighbours(const Dev& d, const Cfg& c, cudaStream_t s) {
  walk<4, false, false, true, false, kWalkAcc>(d, c, s);
  return 1;
}

}  // namespace sphb
