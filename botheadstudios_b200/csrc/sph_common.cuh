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
enum : unsigned { kFlagNbrOverflow = 1u, kFlagStackOverflow = 2u, kFlagCandOverflow = 4u };

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
  unsigned pad0;
  // ---- maintained by the device from here on --------------------------------------------------------
  unsigned flags;         // kFlag* bits
  unsigned max_nbr_seen;
  unsigned steps;
  unsigned h_iters_used;
  float h_residual;
  unsigned h_residual_bits;
  unsigned h_accepted;    // learned h: particles whose proposal passed the first residual check (last solve)
  unsigned pad;
  // walk statistics, accumulated once per warp: node visits, 32-wide pops, multipole and pairwise
  // interactions (particle × source pairs)
  unsigned long long stat_visits, stat_pops, stat_m2p, stat_p2p;
};

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

// ---- SPH kernels with support radius h (sph_step.wgsl:64-77; Wendland C2 from its formula) ----------
__device__ __forceinline__ float w_cubic(float r, float h) {
  const float q = r / h;
  const float sig = 8.0f / (kPiF * h * h * h);
  if (q < 0.5f) return sig * (1.0f - 6.0f * q * q + 6.0f * q * q * q);
  if (q < 1.0f) { const float t = 1.0f - q; return sig * 2.0f * t * t * t; }
  return 0.0f;
}
__device__ __forceinline__ float dw_cubic(float r, float h) {
  const float q = r / h;
  const float sig = 8.0f / (kPiF * h * h * h);
  if (q < 0.5f) return sig * (-12.0f * q + 18.0f * q * q) / h;
  if (q < 1.0f) { const float t = 1.0f - q; return sig * (-6.0f * t * t) / h; }
  return 0.0f;
}
__device__ __forceinline__ float w_wendland(float r, float h) {
  const float q = r / h;
  if (q >= 1.0f) return 0.0f;
  const float t = 1.0f - q;
  return 21.0f / (2.0f * kPiF * h * h * h) * t * t * t * t * (1.0f + 4.0f * q);
}
__device__ __forceinline__ float dw_wendland(float r, float h) {
  const float q = r / h;
  if (q >= 1.0f) return 0.0f;
  const float t = 1.0f - q;
  return 21.0f / (2.0f * kPiF * h * h * h) * (-20.0f * q * t * t * t) / h;
}
// ∂W/∂h at fixed r (for the smoothing-length Newton step).
__device__ __forceinline__ float dwdh_cubic(float r, float h) {
  // W = σ(h) f(q), σ ∝ h⁻³, q = r/h  ⇒  ∂W/∂h = -(3W + q·∂W/∂q·σ)/h = -(3W + r·dW/dr)/h
  return -(3.0f * w_cubic(r, h) + r * dw_cubic(r, h)) / h;
}
__device__ __forceinline__ float dwdh_wendland(float r, float h) {
  return -(3.0f * w_wendland(r, h) + r * dw_wendland(r, h)) / h;
}
template <int KERNEL>
__device__ __forceinline__ float kern_w(float r, float h) { return KERNEL == 1 ? w_wendland(r, h) : w_cubic(r, h); }
template <int KERNEL>
__device__ __forceinline__ float kern_dw(float r, float h) { return KERNEL == 1 ? dw_wendland(r, h) : dw_cubic(r, h); }
template <int KERNEL>
__device__ __forceinline__ float kern_dwdh(float r, float h) {
  return KERNEL == 1 ? dwdh_wendland(r, h) : dwdh_cubic(r, h);
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

// Interleaved neighbour-list slot: warp-group g = t/32 owns a [cap][32] block so that entry k of all 32
// lanes is one 128-byte line.
__device__ __forceinline__ size_t nbr_slot(unsigned t, unsigned k, unsigned cap) {
  return ((size_t)(t >> 5) * cap + k) * 32u + (t & 31u);
}

}  // namespace sphb
