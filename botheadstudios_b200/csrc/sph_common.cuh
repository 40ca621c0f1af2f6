// Shared device helpers and the internal device-state layout of the SPH giant-impact step.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#define SPH_FULL_MASK 0xffffffffu
#define SPH_NO_PARENT 0xffffffffu

namespace sphb {

constexpr int kWarp = 32;
constexpr int kMaxMaterials = 16;   // gpu_sph.rs:113 MAX_MATERIALS
constexpr int kTravStack = 64;      // bh_gravity.wgsl:336 MAX_STACK
constexpr float kPiF = 3.14159265359f;  // sph_step.wgsl:20

// Device-side error/overflow flags (bit set, never cleared by kernels).
enum : unsigned { kFlagNbrOverflow = 1u, kFlagStackOverflow = 2u, kFlagCandOverflow = 4u, kFlagTensorTimeout = 8u };

// Material row as in SphEos48 (Tillotson, 12 floats).
struct Eos {
  float rho0, a, b, cap_a, cap_b, e0, e_iv, e_cv, alpha, beta, p0, p1;
};

// Physics scalars read by the kernels from device memory (so a captured graph sees host updates). The
// per-impact quantities (dt, time, softening, bounding box, Courant signal) live in the segment table.
struct DevParams {
  double dt_fixed;    // host-set dt (sph_set_dt)
  float av_alpha, av_beta;
  float damp, omega;
  float G;            // f32 G for the force kernels
  float theta;
  float cfl;
  float rho_floor, du_floor, r_min, sig_floor;
  float progress;     // host-set fraction of the run completed (a learned-h input)
  float skin_narrow;  // neighbour-list skin of a rebuild after a converged smoothing-length solve
  float skin_wide;    // ... after an upload, or after a solve that ended far from converged
  float skin_reset;   // residual above which the next rebuild takes the wide skin
  unsigned pad0;
  // ---- maintained by the device from here on --------------------------------------------------------
  unsigned flags;         // kFlag* bits
  unsigned max_nbr_seen;
  unsigned steps;
  unsigned h_iters_used;
  float h_residual;
  unsigned pad1;
  unsigned h_accepted;    // learned h: particles whose proposal passed the first residual check (last solve)
  unsigned pad;
  // walk statistics, accumulated once per warp: node visits, 32-wide pops, multipole and pairwise
  // interactions (particle × node, particle × source particle)
  unsigned long long stat_visits, stat_pops, stat_m2p, stat_p2p;
  unsigned long long stat_m2l;        // accepted nodes taken into a group's local expansion (per node and part)
  unsigned long long stat_p2p_slots;  // pairwise slots evaluated: every leaf counted as leaf_size sources
};

// ---- approximate reciprocal square root, reciprocal and division on the special-function unit alone ------
// The .ftz forms flush subnormal operands and results to zero, so they compile to the bare unit operation; the
// operands they get here are never subnormal (softened squared distances, squared pair distances of distinct
// particles, smoothing lengths, densities). Each result is within 2 ulp of the exact one.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float div_ftz(float a, float b) {
  float y;
  asm("div.approx.ftz.f32 %0, %1, %2;" : "=f"(y) : "f"(a), "f"(b));
  return y;
}

// ---- exact single-rounding arithmetic (no FMA contraction) -----------------------------------------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }
// ((x·x + y·y) + z·z) rounded after each operation.
__device__ __forceinline__ float dot3_exact(float x, float y, float z) {
  return fadd(fadd(fmul(x, x), fmul(y, y)), fmul(z, z));
}

// Order-preserving float <-> u32 keys (bh_gravity.wgsl:49-57).
__device__ __forceinline__ unsigned float_key(float f) {
  unsigned k = __float_as_uint(f);
  return (k >> 31) ? ~k : (k ^ 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned k) {
  return (k >> 31) ? __uint_as_float(k ^ 0x80000000u) : __uint_as_float(~k);
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(SPH_FULL_MASK, v, o));
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(SPH_FULL_MASK, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(SPH_FULL_MASK, v, o);
  return v;
}

// Spread 10 bits to 30 (bh_gravity.wgsl:82-89).
__device__ __forceinline__ unsigned expand_bits(unsigned v) {
  v &= 0x000003ffu;
  v = (v * 0x00010001u) & 0xff0000ffu;
  v = (v * 0x00000101u) & 0x0f00f00fu;
  v = (v * 0x00000011u) & 0xc30c30c3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

// ---- SPH kernels with support radius h: the reference's cubic spline (sph_step.wgsl:64-77) and Wendland C2 --
// W(r, h) = σ(h) f(q) with q = r/h and σ = c/h³ (c = 8/π cubic, 21/(2π) Wendland C2), so
// ∂W/∂r = σ f'(q)/h and ∂W/∂h = −(σ/h)(3f + q f'(q)) (the h-derivative drives the smoothing-length Newton step).
// Evaluated from one approximate reciprocal of h (within 2 ulp), every other term a product: the reference's
// per-call divisions (q = r/h, σ = 8/(π h³), f'/h) give the same values to a few ulp at a fraction of the
// instructions, which is what the gather kernels (density, smoothing-length solve, forces) spend per pair.
template <int KERNEL>
__device__ __forceinline__ void kern_pair(float r, float h, float& w, float& dwdr, float& dwdh) {
  const float ih = rcp_ftz(h);
  const float q = r * ih;
  float f = 0.0f, fp = 0.0f;
  if (KERNEL == 1) {
    if (q < 1.0f) {
      const float t = 1.0f - q, t3 = t * t * t;
      f = t3 * t * (1.0f + 4.0f * q);
      fp = -20.0f * q * t3;
    }
  } else if (q < 0.5f) {
    f = 1.0f - 6.0f * q * q + 6.0f * q * q * q;
    fp = -12.0f * q + 18.0f * q * q;
  } else if (q < 1.0f) {
    const float t = 1.0f - q;
    f = 2.0f * t * t * t;
    fp = -6.0f * t * t;
  }
  const float c = KERNEL == 1 ? 3.34225380f : 2.54647909f;  // 21/(2π), 8/π
  const float sig = c * ih * ih * ih;
  const float sih = sig * ih;
  w = sig * f;
  dwdr = sih * fp;
  dwdh = -sih * (3.0f * f + q * fp);
}

// The same kernel with the support test folded into the polynomial: t = max(1 − q, 0) (and, for the cubic
// spline, s = max(½ − q, 0), f = 2t³ − 8s³, which is 1 − 6q² + 6q³ below q = ½), so every term vanishes for
// q ≥ 1 and the gather loops evaluate a pair without a branch. Equal to kern_pair to a few ulp inside the
// support.
template <int KERNEL>
__device__ __forceinline__ void kern_pair_bf(float r, float h, float& w, float& dwdr, float& dwdh) {
  const float ih = rcp_ftz(h);
  const float q = r * ih;
  const float t = fmaxf(1.0f - q, 0.0f);
  float f, fp;
  if (KERNEL == 1) {
    const float t3 = t * t * t;
    f = t3 * t * (1.0f + 4.0f * q);
    fp = -20.0f * q * t3;
  } else {
    const float u = fmaxf(0.5f - q, 0.0f);
    const float t2 = t * t, u2 = u * u;
    f = 2.0f * t2 * t - 8.0f * u2 * u;
    fp = 24.0f * u2 - 6.0f * t2;
  }
  const float c = KERNEL == 1 ? 3.34225380f : 2.54647909f;
  const float sig = c * ih * ih * ih;
  const float sih = sig * ih;
  w = sig * f;
  dwdr = sih * fp;
  dwdh = -sih * (3.0f * f + q * fp);
}

// ---- Tillotson EOS in f32 (sph_step.wgsl:78-100), SI guards carried as parameters --------------------
__device__ __forceinline__ float tillotson_p(const Eos& e, float rho, float u, float rho_floor) {
  const float r = fmaxf(rho, rho_floor);
  const float eta = r / e.rho0;
  const float mu = eta - 1.0f;
  const float omega = u / (e.e0 * eta * eta) + 1.0f;
  const float p_c = (e.a + e.b / omega) * r * u + e.cap_a * mu + e.cap_b * mu * mu;
  if (eta >= 1.0f || u <= e.e_iv) return p_c;
  const float z = e.rho0 / r - 1.0f;
  const float p_e = e.a * r * u + (e.b * r * u / omega + e.cap_a * mu * expf(-e.beta * z)) * expf(-e.alpha * z * z);
  if (u >= e.e_cv) return p_e;
  return ((u - e.e_iv) * p_e + (e.e_cv - u) * p_c) / (e.e_cv - e.e_iv);
}
__device__ __forceinline__ float tillotson_c(const Eos& e, float rho, float u, float du_floor, float rho_floor) {
  const float r = fmaxf(rho, rho_floor);
  const float dr = r * 1.0e-3f;
  const float dp = (tillotson_p(e, r + dr, u, rho_floor) - tillotson_p(e, r - dr, u, rho_floor)) / (2.0f * dr);
  const float p = tillotson_p(e, r, u, rho_floor);
  const float du = fabsf(u) * 1.0e-3f + du_floor;
  const float dfdu = (tillotson_p(e, r, u + du, rho_floor) - tillotson_p(e, r, u - du, rho_floor)) / (2.0f * du);
  return sqrtf(fmaxf(dp + p / (r * r) * dfdu, 0.0f));
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024). Returns the block total.
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* s_warp, unsigned& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  unsigned incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(SPH_FULL_MASK, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[w] = incl;
  __syncthreads();
  if (w == 0) {
    unsigned x = lane < nw ? s_warp[lane] : 0u;
    unsigned xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(SPH_FULL_MASK, xi, o);
      if (lane >= o) xi += t;
    }
    if (lane < nw) s_warp[lane] = xi - x;
    if (lane == 31) s_warp[32] = xi;
  }
  __syncthreads();
  const unsigned res = s_warp[w] + incl - v;
  total = s_warp[32];
  __syncthreads();
  return res;
}

// Interleaved neighbour-list slot: warp-group g = t/32 owns a [cap][32] block so that entry k of all 32
// lanes is one 128-byte line.
__device__ __forceinline__ size_t nbr_slot(unsigned t, unsigned k, unsigned cap) {
  return ((size_t)(t >> 5) * cap + k) * 32u + (t & 31u);
}

}  // namespace sphb
