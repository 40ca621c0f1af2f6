// Barnes-Hut gravity over the LBVH, warp-cooperative.
//
// Reference: cs_gravity_bh, shaders/bh_gravity.wgsl:338-394 — one thread per sorted particle walks the tree
// with a private stack, accepts a node when sqrt(|d|²+ε²) >= diag/θ + |centre − COM|, descends otherwise
// (push left, push right), and sums leaf buckets directly (skipping itself).
//
// B200 form: a warp walks ONE shared depth-first stack for its 32 Morton-consecutive particles. Each stack
// entry carries the lane mask of the particles that still need that subtree. At an internal node every
// lane in the mask evaluates the reference MAC for its own particle; accepting lanes apply the node's
// multipole, and the children are pushed once with the ballot of the lanes that opened it. The node record
// is one broadcast load per warp instead of 32. Because the shared stack visits nodes in the same
// depth-first, right-child-first order as the reference's private stack, and a lane takes part in exactly
// the nodes its own walk would visit, every lane accumulates the same terms in the same order as the
// reference thread would — the monopole result is bit-identical to the reference's per-particle walk.
// Optional: quadrupole moments (traceless, about the COM) and node-relative hi/lo + compensated sums.
#include "sph_kernels.cuh"

namespace sphb {

constexpr int GR_WARPS = 4;  // warps per block

// Kahan-style compensated accumulator (used by the precision mode).
struct Comp3 {
  float s[3] = {0.f, 0.f, 0.f}, c[3] = {0.f, 0.f, 0.f};
  __device__ __forceinline__ void add(int k, float v) {
    const float y = v - c[k];
    const float t = s[k] + y;
    c[k] = (t - s[k]) - y;
    s[k] = t;
  }
};

template <bool QUAD, bool HILO>
__global__ void __launch_bounds__(GR_WARPS * 32) k_gravity_tree(
    const float4* __restrict__ body, const double* __restrict__ x64, const double* __restrict__ y64,
    const double* __restrict__ z64, int n, int L, const unsigned* __restrict__ leaf_start,
    const unsigned* __restrict__ seg, const Seg* __restrict__ segs, const unsigned* __restrict__ left,
    const unsigned* __restrict__ right, const float4* __restrict__ ncom, const float4* __restrict__ nbmax,
    const float4* __restrict__ nq0, const float4* __restrict__ nq1, const DevParams* __restrict__ P,
    float4* __restrict__ out, int stack_cap) {
  __shared__ uint2 s_stack[GR_WARPS][kTravStack];
  const int wib = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const int warp = blockIdx.x * GR_WARPS + wib;
  const int t = warp * 32 + (int)lane;
  if (warp * 32 >= n) return;  // whole warp out of range
  const bool valid = t < n;
  const float4 pi = valid ? body[t] : make_float4(0.f, 0.f, 0.f, 0.f);
  // hi/lo split of the f64 master position (precision mode): x = hi + lo exactly to ~2^-48
  float xlo = 0.f, ylo = 0.f, zlo = 0.f;
  if (HILO && valid) {
    xlo = (float)(x64[t] - (double)pi.x);
    ylo = (float)(y64[t] - (double)pi.y);
    zlo = (float)(z64[t] - (double)pi.z);
  }
  const unsigned sg = valid ? seg[t] : kNoSeg;
  const float G = P->G, soft2 = valid ? segs[sg].soft2 : 0.0f;
  const unsigned leaf0 = (unsigned)(L - 1);
  float ax = 0.f, ay = 0.f, az = 0.f, phi = 0.f;
  Comp3 acc;
  uint2* stack = s_stack[wib];
  int sp = 0;
  // one start entry per impact present in the warp: that impact's root with the mask of its lanes (a lane
  // sees only its own impact's entry, so its walk is the one it would take alone)
  unsigned todo = __ballot_sync(SPH_FULL_MASK, valid);
  while (todo) {
    const unsigned s = __shfl_sync(SPH_FULL_MASK, sg, __ffs(todo) - 1);
    const unsigned m = __ballot_sync(SPH_FULL_MASK, valid && sg == s);
    if (lane == 0) stack[sp] = make_uint2(segs[s].root, m);
    ++sp;
    todo &= ~m;
  }
  __syncwarp();
  unsigned overflow = 0;
  while (sp > 0) {
    --sp;
    const uint2 e = stack[sp];
    const unsigned node = e.x, mask = e.y;
    const bool in = (mask >> lane) & 1u;
    if (node >= leaf0) {
      // leaf bucket: exact pairwise sum over its <= K sorted particles, skipping self
      const int c = (int)(node - leaf0);
      const int s0 = (int)leaf_start[c], s1 = (int)leaf_start[c + 1];
      if (in) {
        for (int s = s0; s < s1; ++s) {
          if (s == t) continue;
          const float4 bj = body[s];
          float dx = fsub(bj.x, pi.x), dy = fsub(bj.y, pi.y), dz = fsub(bj.z, pi.z);
          if (HILO) {
            dx = dx - xlo;
            dy = dy - ylo;
            dz = dz - zlo;
          }
          const float r2 = fadd(dot3_exact(dx, dy, dz), soft2);
          const float rr = fsqrt(r2);
          const float g = fdiv(fmul(G, bj.w), fmul(r2, rr));
          if (HILO) {
            acc.add(0, dx * g);
            acc.add(1, dy * g);
            acc.add(2, dz * g);
          } else {
            ax = fadd(ax, fmul(dx, g));
            ay = fadd(ay, fmul(dy, g));
            az = fadd(az, fmul(dz, g));
          }
          phi -= G * bj.w / rr;
        }
      }
      __syncwarp();
      continue;
    }
    const float4 cm = ncom[node];
    const float rc = nbmax[node].w;
    bool open = false;
    if (in) {
      float dx = fsub(cm.x, pi.x), dy = fsub(cm.y, pi.y), dz = fsub(cm.z, pi.z);
      if (HILO) {
        dx = dx - xlo;
        dy = dy - ylo;
        dz = dz - zlo;
      }
      const float r2 = fadd(dot3_exact(dx, dy, dz), soft2);
      const float dist = fsqrt(r2);
      if (dist >= rc) {
        const float g = fdiv(fmul(G, cm.w), fmul(r2, dist));
        float qx = 0.f, qy = 0.f, qz = 0.f;
        if (QUAD) {
          // a_quad = G [ -Q·d / R^5 + 5/2 (dᵀQd) d / R^7 ]  (d = COM − x, R² = |d|² + ε²), evaluated
          // with the unit vector e = d/R so that Q·e and eᵀQe stay in f32 range in SI units:
          // a_quad = (G/R⁴) [ 5/2 (eᵀQe) e − Q·e ].
          const float4 a0 = nq0[node], a1 = nq1[node];
          const float rinv = 1.0f / dist;
          const float ex = dx * rinv, ey = dy * rinv, ez = dz * rinv;
          const float Qex = a0.x * ex + a0.w * ey + a1.x * ez;
          const float Qey = a0.w * ex + a0.y * ey + a1.y * ez;
          const float Qez = a1.x * ex + a1.y * ey + a0.z * ez;
          const float eQe = ex * Qex + ey * Qey + ez * Qez;
          const float inv2 = 1.0f / r2;
          const float f = 2.5f * eQe;
          qx = ((f * ex - Qex) * inv2) * (G * inv2);
          qy = ((f * ey - Qey) * inv2) * (G * inv2);
          qz = ((f * ez - Qez) * inv2) * (G * inv2);
          phi -= ((0.5f * eQe * inv2) * G) * rinv;
        }
        if (HILO) {
          acc.add(0, dx * g + qx);
          acc.add(1, dy * g + qy);
          acc.add(2, dz * g + qz);
        } else {
          ax = fadd(ax, fmul(dx, g));
          ay = fadd(ay, fmul(dy, g));
          az = fadd(az, fmul(dz, g));
          if (QUAD) {
            ax += qx;
            ay += qy;
            az += qz;
          }
        }
        phi -= G * cm.w / dist;
      } else {
        open = true;
      }
    }
    const unsigned om = __ballot_sync(SPH_FULL_MASK, open);
    if (om) {
      if (sp + 2 <= stack_cap) {
        if (lane == 0) {
          stack[sp] = make_uint2(left[node], om);
          stack[sp + 1] = make_uint2(right[node], om);
        }
        sp += 2;
      } else {
        overflow = 1;  // the reference silently drops these children; we drop them and raise a flag
      }
    }
    __syncwarp();
  }
  if (overflow && lane == 0) atomicOr((unsigned*)&P->flags, kFlagStackOverflow);
  if (valid) {
    if (HILO) out[t] = make_float4(acc.s[0], acc.s[1], acc.s[2], phi);
    else out[t] = make_float4(ax, ay, az, phi);
  }
}

int launch_gravity_tree(const Dev& d, const Cfg& c, cudaStream_t s) {
  const int warps = (d.n + 31) / 32;
  const int blocks = (warps + GR_WARPS - 1) / GR_WARPS;
  const State& st = d.s();
#define GRAV_ARGS                                                                                           \
  d.body, st.x, st.y, st.z, d.n, d.L, d.leaf_start, st.seg, d.segs, d.left, d.right, d.ncom, d.nbmax, d.nq0, d.nq1, \
      d.P, d.grav, c.walk_stack > 0 && c.walk_stack < kTravStack ? c.walk_stack : kTravStack
  if (c.quad) {
    if (c.hilo) k_gravity_tree<true, true><<<blocks, GR_WARPS * 32, 0, s>>>(GRAV_ARGS);
    else k_gravity_tree<true, false><<<blocks, GR_WARPS * 32, 0, s>>>(GRAV_ARGS);
  } else {
    if (c.hilo) k_gravity_tree<false, true><<<blocks, GR_WARPS * 32, 0, s>>>(GRAV_ARGS);
    else k_gravity_tree<false, false><<<blocks, GR_WARPS * 32, 0, s>>>(GRAV_ARGS);
  }
#undef GRAV_ARGS
  return 1;
}

// ---------------------------------------------------------------------------------------------------
// Direct softened sum (the reference's cs_forces gravity loop, sph_step.wgsl:163-169, in the r²·sqrt(r²)
// form of bh_gravity.wgsl:366), shared-memory tiled.
// ---------------------------------------------------------------------------------------------------
constexpr int DS_TILE = 256;

__global__ void __launch_bounds__(DS_TILE) k_gravity_direct(const float4* __restrict__ body,
                                                           const unsigned* __restrict__ seg, int n,
                                                           const Seg* __restrict__ segs,
                                                           const DevParams* __restrict__ P,
                                                           float4* __restrict__ out) {
  __shared__ float4 s_b[DS_TILE];
  const int i = blockIdx.x * DS_TILE + threadIdx.x;
  // sources: the impacts of this block's targets (sorted order keeps impacts contiguous); each target sums
  // over its own impact only
  const int b0 = blockIdx.x * DS_TILE, b1 = min(b0 + DS_TILE, n) - 1;
  const int j0 = (int)segs[seg[b0]].off, j1 = (int)segs[seg[b1] + 1].off;
  const unsigned sg = i < n ? seg[i] : seg[b0];
  const int m0 = (int)segs[sg].off, m1 = (int)segs[sg + 1].off;
  const float4 pi = i < n ? body[i] : make_float4(0, 0, 0, 0);
  const float G = P->G, soft2 = segs[sg].soft2;
  float ax = 0, ay = 0, az = 0, phi = 0;
  for (int base = j0; base < j1; base += DS_TILE) {
    const int j = base + threadIdx.x;
    s_b[threadIdx.x] = j < j1 ? body[j] : make_float4(0, 0, 0, 0);
    __syncthreads();
    const int cnt = min(DS_TILE, j1 - base);
    for (int k = 0; k < cnt; ++k) {
      const int jj = base + k;
      if (jj == i || jj < m0 || jj >= m1) continue;
      const float4 bj = s_b[k];
      const float dx = bj.x - pi.x, dy = bj.y - pi.y, dz = bj.z - pi.z;
      const float r2 = dx * dx + dy * dy + dz * dz + soft2;
      const float rinv = rsqrtf(r2);
      const float g = G * bj.w * rinv * rinv * rinv;
      ax += dx * g;
      ay += dy * g;
      az += dz * g;
      phi -= G * bj.w * rinv;
    }
    __syncthreads();
  }
  if (i < n) out[i] = make_float4(ax, ay, az, phi);
}

int launch_gravity_direct(const Dev& d, cudaStream_t s) {
  k_gravity_direct<<<(d.n + DS_TILE - 1) / DS_TILE, DS_TILE, 0, s>>>(d.body, d.s().seg, d.n, d.segs, d.P, d.grav);
  return 1;
}

// FP64 softened direct sum for a subset of targets (the precision oracle of the tree).
constexpr int D64_TILE = 128;
__global__ void __launch_bounds__(D64_TILE) k_gravity_direct64(const double* __restrict__ pos3,
                                                              const double* __restrict__ mass, int n,
                                                              const unsigned* __restrict__ targets, int nt,
                                                              double soft2, double G, double* __restrict__ acc3) {
  __shared__ double s_p[D64_TILE][4];
  const int q = blockIdx.x * D64_TILE + threadIdx.x;
  const int i = q < nt ? (targets ? (int)targets[q] : q) : -1;
  double xi = 0, yi = 0, zi = 0;
  if (i >= 0) {
    xi = pos3[3 * (size_t)i];
    yi = pos3[3 * (size_t)i + 1];
    zi = pos3[3 * (size_t)i + 2];
  }
  double ax = 0, ay = 0, az = 0;
  for (int base = 0; base < n; base += D64_TILE) {
    const int j = base + threadIdx.x;
    if (j < n) {
      s_p[threadIdx.x][0] = pos3[3 * (size_t)j];
      s_p[threadIdx.x][1] = pos3[3 * (size_t)j + 1];
      s_p[threadIdx.x][2] = pos3[3 * (size_t)j + 2];
      s_p[threadIdx.x][3] = mass[j];
    }
    __syncthreads();
    const int cnt = min(D64_TILE, n - base);
    for (int k = 0; k < cnt; ++k) {
      if (base + k == i) continue;
      const double dx = s_p[k][0] - xi, dy = s_p[k][1] - yi, dz = s_p[k][2] - zi;
      const double r2 = dx * dx + dy * dy + dz * dz + soft2;
      const double g = G * s_p[k][3] / (r2 * sqrt(r2));
      ax += dx * g;
      ay += dy * g;
      az += dz * g;
    }
    __syncthreads();
  }
  if (q < nt) {
    acc3[3 * (size_t)q] = ax;
    acc3[3 * (size_t)q + 1] = ay;
    acc3[3 * (size_t)q + 2] = az;
  }
}

int launch_gravity_direct64(const double* pos3, const double* mass, int n, const unsigned* targets, int nt,
                             double soft2, double G, double* acc3, cudaStream_t s) {
  k_gravity_direct64<<<(nt + D64_TILE - 1) / D64_TILE, D64_TILE, 0, s>>>(pos3, mass, n, targets, nt, soft2, G,
                                                                         acc3);
  return 1;
}

}  // namespace sphb
