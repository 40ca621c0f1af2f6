// SPH on B200: neighbour lists from the LBVH, density + Tillotson EOS, smoothing-length solve, pressure +
// Monaghan AV + du/dt forces with the Courant signal reduction fused in, KDK leapfrog with f64 positions
// (bbox reduction fused into the drift), damped relaxation, exchange-format conversion and FP64 sums.
//
// Reference: shaders/sph_step.wgsl (cs_density :120-149, cs_forces :153-211, cs_kick_drift :221-228,
// cs_kick :232-237, cs_relax :245-257, cs_signal :263-269). The reference finds neighbours with a spatial
// hash over 27 cells plus a cell-membership guard; the set it produces is exactly {j != i : r_ij < h_ij},
// h_ij = ½(h_i + h_j). Here that set is enumerated once per tree build by a warp-cooperative walk of the
// LBVH (node AABBs carry the subtree's max h) and stored as interleaved per-particle lists; r_ij is
// computed with single-rounded operations so the set is bit-identical to the reference predicate.
#include "sph_kernels.cuh"

namespace sphb {

// Pair distance in the gather kernels from one reciprocal square root (MUFU, within 2 ulp): the sums they
// form are continuous at the support edge (W and ∇W vanish at q = 1), so a pair whose r rounds across h_ij
// changes nothing, and the exact predicate is needed only where the neighbour set is decided (the walk).
__device__ __forceinline__ float pair_r(float4 a, float4 b, float& rinv) {
  const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  const float dd = dx * dx + dy * dy + dz * dz;
  rinv = rsqrt_ftz(dd);
  return dd > 0.0f ? dd * rinv : 0.0f;
}
__device__ __forceinline__ float pair_h(float hi, float hj) { return fmul(0.5f, fadd(hi, hj)); }

// The gather kernels walk a particle's list kGather entries at a time: all of a chunk's indices are loaded,
// then all of its neighbour records, before any is used, so each thread keeps kGather gathers in flight
// instead of one dependent chain; the next chunk's indices are requested before this chunk's records, so the
// list stream (HBM) overlaps the record gathers (mostly L1/L2) and the arithmetic. `lst` is the particle's
// first list slot (entries 32 apart, interleaved); slots past the count read the sentinel record `sent` (a
// massless particle outside every support), so a pair is evaluated without testing the count or the support
// (kern_pair_bf vanishes outside it). The lists are read once per pass and streamed past the cache
// (evict-first), so they do not push the neighbours' records out of L2.
constexpr int kGather = 4;
template <int G>
__device__ __forceinline__ void list_chunk(const unsigned* __restrict__ lst, unsigned k0, unsigned c, unsigned sent,
                                           unsigned j[G]) {
#pragma unroll
  for (int u = 0; u < G; ++u) j[u] = k0 + u < c ? __ldcs(&lst[(size_t)(k0 + u) * 32u]) : sent;
}
// Records of the chunk whose indices are in `jn` (k0 = its first slot); jn2 holds the next chunk's indices.
// On return jn holds the next chunk's and jn2 the one after it: the list stays two chunks ahead of the records.
__device__ __forceinline__ void gather_pos_mass(const State& st, const unsigned* __restrict__ lst, unsigned k0,
                                                unsigned c, unsigned sent, unsigned jn[kGather],
                                                unsigned jn2[kGather], float4 pj[kGather], float mj[kGather]) {
  unsigned j[kGather];
#pragma unroll
  for (int u = 0; u < kGather; ++u) {
    j[u] = jn[u];
    jn[u] = jn2[u];
  }
  list_chunk<kGather>(lst, k0 + 2 * kGather, c, sent, jn2);
#pragma unroll
  for (int u = 0; u < kGather; ++u) {
    pj[u] = st.pos_h[j[u]];
    mj[u] = st.mass[j[u]];
  }
}

// ---------------------------------------------------------------------------------------------------
// Density (cs_density) with the EOS fused: rho_i = m_i W(0,h_i) + Σ m_j W(r, h_ij) over r < h_ij, then
// P(rho,u), c(rho,u) and the per-particle force record (m, rho, P/rho², c). The reference re-evaluates P_j
// and c_j for every pair (sph_step.wgsl:188-190); they are pure functions of (rho_j, u_j, mat_j), so one
// evaluation per particle gives the same values.
// ---------------------------------------------------------------------------------------------------
__device__ __forceinline__ float4 eos_record(const Eos* __restrict__ eos, unsigned mat, float m, float rho,
                                             float u, const DevParams* P) {
  const Eos e = eos[mat];
  const float p = tillotson_p(e, rho, u, P->rho_floor);
  const float c = tillotson_c(e, rho, u, P->du_floor, P->rho_floor);
  return make_float4(m, rho, p / (rho * rho), c);
}

template <int KERNEL>
__global__ void k_density_eos(int n, State st, const unsigned* __restrict__ nbr,
                              const unsigned* __restrict__ nbr_cnt, unsigned cap, unsigned sent,
                              const Eos* __restrict__ eos, const DevParams* __restrict__ P,
                              float* __restrict__ rho, float4* __restrict__ fdata) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float4 pi = st.pos_h[t];
  const float m = st.mass[t];
  float w, dwdr, dwdh;
  kern_pair<KERNEL>(0.0f, pi.w, w, dwdr, dwdh);
  float r_i = m * w;
  const unsigned c = min(nbr_cnt[t], cap);
  const unsigned* lst = nbr + nbr_slot((unsigned)t, 0u, cap);
  unsigned jn[kGather], jn2[kGather];
  list_chunk<kGather>(lst, 0u, c, sent, jn);
  list_chunk<kGather>(lst, kGather, c, sent, jn2);
  for (unsigned k0 = 0; k0 < c; k0 += kGather) {
    float4 pj[kGather];
    float mj[kGather];
    gather_pos_mass(st, lst, k0, c, sent, jn, jn2, pj, mj);
#pragma unroll
    for (int u = 0; u < kGather; ++u) {
      float ri;
      const float r = pair_r(pi, pj[u], ri);
      kern_pair_bf<KERNEL>(r, pair_h(pi.w, pj[u].w), w, dwdr, dwdh);
      r_i += mj[u] * w;
    }
  }
  rho[t] = r_i;
  fdata[t] = eos_record(eos, st.mat[t], m, r_i, st.vel_u[t].w, P);
}

int launch_density_eos(const Dev& d, const Cfg& c, cudaStream_t s) {
  const int blocks = (d.n + c.blk - 1) / c.blk;
  if (c.kernel == 1)
    k_density_eos<1><<<blocks, c.blk, 0, s>>>(d.n, d.s(), d.nbr, d.nbr_cnt, d.nbr_cap, d.sent, d.eos, d.P, d.rho,
                                              d.fdata);
  else
    k_density_eos<0><<<blocks, c.blk, 0, s>>>(d.n, d.s(), d.nbr, d.nbr_cnt, d.nbr_cap, d.sent, d.eos, d.P, d.rho,
                                              d.fdata);
  return 1;
}

__global__ void k_eos_only(int n, State st, const float* __restrict__ rho, const Eos* __restrict__ eos,
                           const DevParams* __restrict__ P, float4* __restrict__ fdata) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  fdata[t] = eos_record(eos, st.mat[t], st.mass[t], rho[t], st.vel_u[t].w, P);
}
int launch_eos_only(const Dev& d, cudaStream_t s) {
  k_eos_only<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, d.s(), d.rho, d.eos, d.P, d.fdata);
  return 1;
}

// ---------------------------------------------------------------------------------------------------
// Smoothing-length solve (new; the reference keeps h fixed, hydrostatic.rs:59-61). Jacobi-Newton on
// f(h_i) = rho_i(h) − m_i (η/h_i)³ with rho_i from the reference's symmetric form (h_ij = ½(h_i+h_j)),
// ∂rho_i/∂h_i = m_i ∂W(0,h_i)/∂h + Σ_j m_j ½ ∂W(r,h_ij)/∂h (Price 2012, J. Comput. Phys. 231, §3.2.1).
// h may move inside the list's skin only; the residual |f|/rho is reduced to a device maximum.
// ---------------------------------------------------------------------------------------------------
// ρ_i and ∂ρ_i/∂h_i at the particle's current h over its neighbour list (the density sum of k_density_eos,
// same terms in the same order).
template <int KERNEL>
__device__ __forceinline__ void h_sums(int t, const State& st, const unsigned* __restrict__ nbr,
                                       const unsigned* __restrict__ nbr_cnt, unsigned cap, unsigned sent,
                                       float& rho, float& drho) {
  const float4 pi = st.pos_h[t];
  const float m = st.mass[t];
  const float h = pi.w;
  float w, dwdr, dwdh;
  kern_pair<KERNEL>(0.0f, h, w, dwdr, dwdh);
  rho = m * w;
  const float dself = m * dwdh;
  float dsum = 0.0f;  // Σ m_j ∂W/∂h_ij; ∂h_ij/∂h_i = ½ is applied once
  const unsigned c = min(nbr_cnt[t], cap);
  const unsigned* lst = nbr + nbr_slot((unsigned)t, 0u, cap);
  unsigned jn[kGather], jn2[kGather];
  list_chunk<kGather>(lst, 0u, c, sent, jn);
  list_chunk<kGather>(lst, kGather, c, sent, jn2);
  for (unsigned k0 = 0; k0 < c; k0 += kGather) {
    float4 pj[kGather];
    float mj[kGather];
    gather_pos_mass(st, lst, k0, c, sent, jn, jn2, pj, mj);
#pragma unroll
    for (int u = 0; u < kGather; ++u) {
      float ri;
      const float r = pair_r(pi, pj[u], ri);
      kern_pair_bf<KERNEL>(r, pair_h(h, pj[u].w), w, dwdr, dwdh);
      rho += mj[u] * w;
      dsum += mj[u] * dwdh;
    }
  }
  drho = dself + 0.5f * dsum;
}

// The Newton update of h from the residual f = ρ − m(η/h)³, limited to ±20 % and to the list's skin. `res`
// is the relative residual |f|/ρ; `drel` the relative density change the unlimited Newton step would make
// (|∂ρ/∂h · Δh|/ρ), the density error that is left when h stops here.
__device__ __forceinline__ float h_newton(float h, float m, float rho, float drho, float eta, float h0, float skin,
                                          float& res, float& drel) {
  const float e3 = eta * eta * eta;
  const float rt = m * e3 / (h * h * h);
  const float f = rho - rt;
  res = fabsf(f) / fmaxf(rho, 1.0e-30f);
  const float fp = drho + 3.0f * rt / h;
  const float dh = fabsf(fp) > 0.0f ? -f / fp : 0.0f;
  drel = fabsf(drho * dh) / fmaxf(rho, 1.0e-30f);
  float hn = h + dh;
  if (!(hn == hn)) hn = h;  // NaN guard
  hn = fminf(fmaxf(hn, 0.8f * h), 1.2f * h);
  hn = fminf(hn, h0 * (1.0f + skin) * 0.999f);
  hn = fmaxf(hn, h0 / ((1.0f + skin) * 1.001f));
  return hn;
}

template <int KERNEL>
__global__ void k_h_iter(int n, State st, const unsigned* __restrict__ nbr, const unsigned* __restrict__ nbr_cnt,
                         unsigned cap, unsigned sent, const float* __restrict__ h0, float eta, DevParams* P, Seg* __restrict__ segs,
                         float* __restrict__ hnew, int last, const Eos* __restrict__ eos, float* __restrict__ rho_out,
                         float4* __restrict__ fdata) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  float res = 0.0f;
  const unsigned sg = t < n ? st.seg[t] : kNoSeg;
  if (t < n) {
    float rho, drho;
    h_sums<KERNEL>(t, st, nbr, nbr_cnt, cap, sent, rho, drho);
    const float m = st.mass[t], h = st.pos_h[t].w;
    float drel;
    float hn = h_newton(h, m, rho, drho, eta, h0[t], segs[sg].skin, res, drel);
    if (last) {
      // the final pass is the density pass: same sum, same order as k_density_eos
      rho_out[t] = rho;
      fdata[t] = eos_record(eos, st.mat[t], m, rho, st.vel_u[t].w, P);
      hn = h;
    }
    hnew[t] = hn;
  }
  seg_res_max(segs, sg, res);
}

constexpr float kDensityTolFraction = 0.25f;

// Learned h: check the proposed (or current) h of every listed particle. A particle whose relative density
// residual is within tolerance (or that is on its last pass) is final: its density and EOS record are
// written. Any other takes a Newton step (into hnew) and is appended to the next list. `list` null = all n.
template <int KERNEL>
__global__ void k_h_check(int n, const unsigned* __restrict__ list, const unsigned* __restrict__ list_n, State st,
                          const unsigned* __restrict__ nbr, const unsigned* __restrict__ nbr_cnt, unsigned cap,
                          unsigned sent, const float* __restrict__ h0, float eta, float tol, DevParams* P, Seg* __restrict__ segs,
                          float* __restrict__ hnew, unsigned* __restrict__ next, unsigned* __restrict__ next_n,
                          int last, const Eos* __restrict__ eos, float* __restrict__ rho_out,
                          float4* __restrict__ fdata) {
  const int count = list ? (int)*list_n : n;
  const int lane = threadIdx.x & 31;
  unsigned acc = 0;
  // whole warps step together (the append and the residual maximum below are warp-collective)
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < count; base += gridDim.x * blockDim.x) {
    const int i = base + lane;
    bool pend = false;
    int t = -1;
    unsigned sg = kNoSeg;
    float fres = 0.0f;
    if (i < count) {
      t = list ? (int)list[i] : i;
      float rho, drho, res, drel;
      h_sums<KERNEL>(t, st, nbr, nbr_cnt, cap, sent, rho, drho);
      const float m = st.mass[t], h = st.pos_h[t].w;
      const unsigned s = st.seg[t];
      const float hn = h_newton(h, m, rho, drho, eta, h0[t], segs[s].skin, res, drel);
      // accepted: residual within tolerance and a density that one more step would move by < tol/4 (near a
      // surface ρ depends strongly on h, and a small residual alone can leave a larger density error)
      if ((res <= tol && drel <= kDensityTolFraction * tol) || last) {
        rho_out[t] = rho;
        fdata[t] = eos_record(eos, st.mat[t], m, rho, st.vel_u[t].w, P);
        sg = s;
        fres = res;
        if (!list && res <= tol) ++acc;
      } else {
        hnew[t] = hn;
        pend = true;
      }
    }
    seg_res_max(segs, sg, fres);
    const unsigned bal = __ballot_sync(SPH_FULL_MASK, pend);
    unsigned at = 0;
    if (lane == 0 && bal) at = atomicAdd(next_n, (unsigned)__popc(bal));
    at = __shfl_sync(SPH_FULL_MASK, at, 0);
    if (pend) next[at + __popc(bal & ((1u << lane) - 1u))] = (unsigned)t;
  }
  acc += __shfl_xor_sync(SPH_FULL_MASK, acc, 16);
  acc += __shfl_xor_sync(SPH_FULL_MASK, acc, 8);
  acc += __shfl_xor_sync(SPH_FULL_MASK, acc, 4);
  acc += __shfl_xor_sync(SPH_FULL_MASK, acc, 2);
  acc += __shfl_xor_sync(SPH_FULL_MASK, acc, 1);
  if (lane == 0 && acc) atomicAdd(&P->h_accepted, acc);
}

__global__ void k_h_commit_list(const unsigned* __restrict__ list, const unsigned* __restrict__ list_n, State st,
                                const float* __restrict__ hnew) {
  const int count = (int)*list_n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const unsigned t = list[i];
    st.pos_h[t].w = hnew[t];
  }
}

__global__ void k_h_commit(int n, State st, const float* __restrict__ hnew) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) st.pos_h[t].w = hnew[t];
}
__global__ void k_h_reset(DevParams* P, Seg* segs, int nseg, int iters) {
  if (threadIdx.x < nseg) segs[threadIdx.x].res_bits = 0u;
  if (threadIdx.x == 0) {
    P->h_iters_used = (unsigned)iters;
    P->h_accepted = 0u;
  }
}
// The solve's residual maximum (over all impacts); and each impact's next skin: wide while some particle of it
// is still far from its smoothing length (right after an upload, or a shock), narrow once every one is near it.
__global__ void k_h_publish(DevParams* P, Seg* segs, int nseg) {
  __shared__ float s_max[kMaxSegments / 32];
  float r = 0.0f;
  if (threadIdx.x < nseg) {
    r = __uint_as_float(segs[threadIdx.x].res_bits);
    segs[threadIdx.x].skin = r > P->skin_reset ? P->skin_wide : P->skin_narrow;
  }
  r = warp_max(r);
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = 0.0f;
    for (int k = 0; k < kMaxSegments / 32; ++k) m = fmaxf(m, s_max[k]);
    P->h_residual = m;
  }
}

int launch_h_solve(const Dev& d, const Cfg& c, cudaStream_t s) {
  const int blocks = (d.n + c.blk - 1) / c.blk;
  for (int it = 0; it <= c.h_iters; ++it) {
    const int last = it == c.h_iters;
    k_h_reset<<<1, kMaxSegments, 0, s>>>(d.P, d.segs, d.nseg, c.h_iters);
    if (c.kernel == 1)
      k_h_iter<1><<<blocks, c.blk, 0, s>>>(d.n, d.s(), d.nbr, d.nbr_cnt, d.nbr_cap, d.sent, d.h0, c.h_eta, d.P, d.segs, d.hnew,
                                          last, d.eos, d.rho, d.fdata);
    else
      k_h_iter<0><<<blocks, c.blk, 0, s>>>(d.n, d.s(), d.nbr, d.nbr_cnt, d.nbr_cap, d.sent, d.h0, c.h_eta, d.P, d.segs, d.hnew,
                                          last, d.eos, d.rho, d.fdata);
    if (!last) k_h_commit<<<blocks, c.blk, 0, s>>>(d.n, d.s(), d.hnew);
  }
  k_h_publish<<<1, kMaxSegments, 0, s>>>(d.P, d.segs, d.nseg);
  return (c.h_iters + 1) * 2 + c.h_iters + 1;
}

// Learned h: the proposals written into pos_h.w before the tree build are checked in one pass over all
// particles; only the rejected ones iterate (Jacobi-Newton over their own lists), at most h_iters times,
// the last pass writing density and EOS whatever the residual. The residual maximum covers every particle.
int launch_h_learned(const Dev& d, const Cfg& c, cudaStream_t s) {
  const int full = (d.n + c.blk - 1) / c.blk;
  const int part = full < 148 * 8 ? full : 148 * 8;
  k_h_reset<<<1, kMaxSegments, 0, s>>>(d.P, d.segs, d.nseg, c.h_iters);
  cudaMemsetAsync(d.pend_n, 0, 2 * sizeof(unsigned), s);
  int launches = 2;
#define HC_ARGS(list, ln, nx, nxn, last)                                                                   \
  d.n, list, ln, d.s(), d.nbr, d.nbr_cnt, d.nbr_cap, d.sent, d.h0, c.h_eta, c.h_tol, d.P, d.segs, d.hnew, nx, nxn, last, \
      d.eos, d.rho, d.fdata
  if (c.kernel == 1)
    k_h_check<1><<<full, c.blk, 0, s>>>(HC_ARGS(nullptr, nullptr, d.pend[0], d.pend_n, c.h_iters == 0 ? 1 : 0));
  else
    k_h_check<0><<<full, c.blk, 0, s>>>(HC_ARGS(nullptr, nullptr, d.pend[0], d.pend_n, c.h_iters == 0 ? 1 : 0));
  ++launches;
  for (int it = 1; it <= c.h_iters; ++it) {
    const int a = (it - 1) & 1, b = it & 1;
    k_h_commit_list<<<part, 256, 0, s>>>(d.pend[a], d.pend_n + a, d.s(), d.hnew);
    cudaMemsetAsync(d.pend_n + b, 0, sizeof(unsigned), s);
    const int last = it == c.h_iters ? 1 : 0;
    if (c.kernel == 1)
      k_h_check<1><<<part, c.blk, 0, s>>>(HC_ARGS(d.pend[a], d.pend_n + a, d.pend[b], d.pend_n + b, last));
    else
      k_h_check<0><<<part, c.blk, 0, s>>>(HC_ARGS(d.pend[a], d.pend_n + a, d.pend[b], d.pend_n + b, last));
    launches += 3;
  }
#undef HC_ARGS
  k_h_publish<<<1, kMaxSegments, 0, s>>>(d.P, d.segs, d.nseg);
  return launches + 1;
}

// ---------------------------------------------------------------------------------------------------
// Forces (the SPH half of cs_forces, sph_step.wgsl:170-210) + gravity + the Courant signal (cs_signal
// :263-269) reduced to each impact's minimum with one atomic per warp (per lane in a warp that straddles two
// impacts).
// ---------------------------------------------------------------------------------------------------
constexpr int kForceGather = 2;  // neighbours of a force chunk (three records each)

template <int KERNEL, bool GRAV, bool DIVV>
__global__ void k_forces(int n, State st, const float4* __restrict__ fdata, const unsigned* __restrict__ nbr,
                         const unsigned* __restrict__ nbr_cnt, unsigned cap, unsigned sent,
                         const float4* __restrict__ grav, const DevParams* __restrict__ P, Seg* __restrict__ segs,
                         float4* __restrict__ acc, float* __restrict__ divv) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  float sig = __int_as_float(0x7f800000);
  const unsigned sg = t < n ? st.seg[t] : kNoSeg;
  if (t < n) {
    const float4 pi = st.pos_h[t];
    const float4 vi = st.vel_u[t];
    const float4 fi = fdata[t];
    const float alpha = P->av_alpha, beta = P->av_beta, r_min = P->r_min;
    float ax = 0.f, ay = 0.f, az = 0.f, de = 0.f, dv = 0.f;
    const unsigned c = min(nbr_cnt[t], cap);
    const unsigned* lst = nbr + nbr_slot((unsigned)t, 0u, cap);
    unsigned jn[kForceGather], jn2[kForceGather];
    list_chunk<kForceGather>(lst, 0u, c, sent, jn);
    list_chunk<kForceGather>(lst, kForceGather, c, sent, jn2);
    for (unsigned k0 = 0; k0 < c; k0 += kForceGather) {
      // a chunk's positions, velocities and force records in flight together, the indices of the two chunks
      // after it requested ahead of them (one chunk ahead left the loads waiting on the list stream)
      unsigned jj[kForceGather];
      float4 pjs[kForceGather], vjs[kForceGather], fjs[kForceGather];
#pragma unroll
      for (int u = 0; u < kForceGather; ++u) {
        jj[u] = jn[u];
        jn[u] = jn2[u];
      }
      list_chunk<kForceGather>(lst, k0 + 2 * kForceGather, c, sent, jn2);
#pragma unroll
      for (int u = 0; u < kForceGather; ++u) {
        pjs[u] = st.pos_h[jj[u]];
        vjs[u] = st.vel_u[jj[u]];
        fjs[u] = fdata[jj[u]];
      }
      // Branch-free pair: outside the support (and for the sentinel) ∇W = 0; pairs closer than r_min are
      // left out as the reference leaves them out (∇W zeroed); a receding pair (v_ij·r_ij ≥ 0) has μ = 0 and
      // so no viscosity.
#pragma unroll
      for (int u = 0; u < kForceGather; ++u) {
        const float4 pj = pjs[u];
        const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const float dd = dx * dx + dy * dy + dz * dz;
        const float rinv = rsqrt_ftz(dd);
        const float r = dd > 0.0f ? dd * rinv : 0.0f;
        const float hij = pair_h(pi.w, pj.w);
        const float4 vj = vjs[u];
        const float4 fj = fjs[u];
        const float vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
        const float vr = vx * dx + vy * dy + vz * dz;
        // approximate reciprocals (within 2 ulp): both denominators are positive and far from the limits
        const float mu = hij * fminf(vr, 0.0f) * rcp_ftz(dd + 0.01f * hij * hij);
        const float c_bar = 0.5f * (fi.w + fj.w);
        const float pij = (beta * mu - alpha * c_bar) * mu * rcp_ftz(0.5f * (fi.y + fj.y));
        const float coeff = fi.z + fj.z + pij;
        float w, dw, dwdh;
        kern_pair_bf<KERNEL>(r, hij, w, dw, dwdh);
        const float dwr = r > r_min ? dw * rinv : 0.0f;  // ∇_i W = (dx/r) ∂W/∂r
        const float gx = dx * dwr, gy = dy * dwr, gz = dz * dwr;
        const float s = -coeff * fj.x;
        ax += gx * s;
        ay += gy * s;
        az += gz * s;
        const float vg = vx * gx + vy * gy + vz * gz;
        de += 0.5f * fj.x * coeff * vg;
        if (DIVV) dv += fj.x * vg;
      }
    }
    if (GRAV) {
      const float4 g = grav[t];
      ax += g.x;
      ay += g.y;
      az += g.z;
    }
    acc[t] = make_float4(ax, ay, az, de);
    if (DIVV) divv[t] = -dv / fi.y;  // ∇·v_i = −(1/ρ_i) Σ_j m_j v_ij·∇_i W_ij (a learned-h input)
    const float vmag = sqrtf(vi.x * vi.x + vi.y * vi.y + vi.z * vi.z);
    sig = pi.w / fmaxf(fi.w + vmag, P->sig_floor);
  }
  const unsigned wlo = warp_min(sg), whi = warp_max(sg == kNoSeg ? 0u : sg);
  if (wlo == kNoSeg) return;
  if (wlo == whi) {
    sig = warp_min(sig);
    if ((threadIdx.x & 31) == 0 && sig < __int_as_float(0x7f800000))
      atomicMin(&segs[wlo].sig_bits, __float_as_uint(sig));
  } else if (sg != kNoSeg && sig < __int_as_float(0x7f800000)) {
    atomicMin(&segs[sg].sig_bits, __float_as_uint(sig));
  }
}

int launch_forces(const Dev& d, const Cfg& c, cudaStream_t s) {
  const int blocks = (d.n + c.blk - 1) / c.blk;
  const bool g = c.gravity != 2;
#define FARGS d.n, d.s(), d.fdata, d.nbr, d.nbr_cnt, d.nbr_cap, d.sent, d.grav, d.P, d.segs, d.acc, d.divv
  if (c.divv) {
    if (c.kernel == 1) {
      if (g) k_forces<1, true, true><<<blocks, c.blk, 0, s>>>(FARGS);
      else k_forces<1, false, true><<<blocks, c.blk, 0, s>>>(FARGS);
    } else {
      if (g) k_forces<0, true, true><<<blocks, c.blk, 0, s>>>(FARGS);
      else k_forces<0, false, true><<<blocks, c.blk, 0, s>>>(FARGS);
    }
  } else if (c.kernel == 1) {
    if (g) k_forces<1, true, false><<<blocks, c.blk, 0, s>>>(FARGS);
    else k_forces<1, false, false><<<blocks, c.blk, 0, s>>>(FARGS);
  } else {
    if (g) k_forces<0, true, false><<<blocks, c.blk, 0, s>>>(FARGS);
    else k_forces<0, false, false><<<blocks, c.blk, 0, s>>>(FARGS);
  }
#undef FARGS
  return 1;
}

// ---------------------------------------------------------------------------------------------------
// Step control, per impact: dt = cfl·min signal (or the fixed dt), simulated time, reset of the reductions.
// ---------------------------------------------------------------------------------------------------
__global__ void k_finalize_dt(DevParams* P, Seg* segs, int nseg) {
  const int k = threadIdx.x;
  if (k == 0) P->steps += 1u;
  if (k >= nseg) return;
  Seg& S = segs[k];
  double dt = P->dt_fixed;
  if (P->cfl > 0.0f && S.sig_bits != 0x7f800000u) dt = (double)P->cfl * (double)__uint_as_float(S.sig_bits);
  S.dt = dt;
  S.time += dt;
  S.sig_bits = 0x7f800000u;
  for (int a = 0; a < 3; ++a) {
    S.bbox[a] = 0xffffffffu;
    S.bbox[3 + a] = 0u;
  }
}
int launch_finalize_dt(const Dev& d, cudaStream_t s) {
  k_finalize_dt<<<1, kMaxSegments, 0, s>>>(d.P, d.segs, d.nseg);
  return 1;
}

// First half-kick and drift (cs_kick_drift): v += a·dt/2, u = max(u + du·dt/2, 0), x += v·dt in f64 with
// the particle's impact dt, plus each impact's bounding box of the new positions for the next Morton pass.
__global__ void k_kick_drift(int n, State st, const float4* __restrict__ acc, Seg* segs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
  unsigned sg = kNoSeg;
  if (t < n) {
    sg = st.seg[t];
    const double dt = segs[sg].dt;
    const float hdt = (float)(0.5 * dt);
    const float4 a = acc[t];
    float4 v = st.vel_u[t];
    v.x = v.x + a.x * hdt;
    v.y = v.y + a.y * hdt;
    v.z = v.z + a.z * hdt;
    v.w = fmaxf(v.w + a.w * hdt, 0.0f);
    st.vel_u[t] = v;
    const double x = st.x[t] + (double)v.x * dt, y = st.y[t] + (double)v.y * dt, z = st.z[t] + (double)v.z * dt;
    st.x[t] = x;
    st.y[t] = y;
    st.z[t] = z;
    float4 p = st.pos_h[t];
    p.x = (float)x;
    p.y = (float)y;
    p.z = (float)z;
    st.pos_h[t] = p;
    lo[0] = hi[0] = float_key(p.x);
    lo[1] = hi[1] = float_key(p.y);
    lo[2] = hi[2] = float_key(p.z);
  }
  seg_bbox_commit(lo, hi, sg, segs);
}
int launch_kick_drift(const Dev& d, cudaStream_t s) {
  k_kick_drift<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, d.s(), d.acc, d.segs);
  return 1;
}

// Final half-kick (cs_kick) with the EOS record refreshed for the new u (density is unchanged).
__global__ void k_kick(int n, State st, const float4* __restrict__ acc, const float* __restrict__ rho,
                       const Eos* __restrict__ eos, const DevParams* __restrict__ P, const Seg* __restrict__ segs,
                       float4* __restrict__ fdata) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float hdt = (float)(0.5 * segs[st.seg[t]].dt);
  const float4 a = acc[t];
  float4 v = st.vel_u[t];
  v.x = v.x + a.x * hdt;
  v.y = v.y + a.y * hdt;
  v.z = v.z + a.z * hdt;
  v.w = fmaxf(v.w + a.w * hdt, 0.0f);
  st.vel_u[t] = v;
  fdata[t] = eos_record(eos, st.mat[t], st.mass[t], rho[t], v.w, P);
}
int launch_kick(const Dev& d, cudaStream_t s) {
  k_kick<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, d.s(), d.acc, d.rho, d.eos, d.P, d.segs, d.fdata);
  return 1;
}

// Damped relaxation (cs_relax, sph_step.wgsl:245-257): v = (v + (a + ω²(x,y,0))·dt)·damp; x += v·dt.
__global__ void k_relax(int n, State st, const float4* __restrict__ acc, DevParams* P) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double dt = P->dt_fixed;
  const float fdt = (float)dt;
  const float w2 = P->omega * P->omega;
  const float4 a = acc[t];
  float4 p = st.pos_h[t];
  float4 v = st.vel_u[t];
  v.x = (v.x + (a.x + w2 * p.x) * fdt) * P->damp;
  v.y = (v.y + (a.y + w2 * p.y) * fdt) * P->damp;
  v.z = (v.z + a.z * fdt) * P->damp;
  st.vel_u[t] = v;
  const double x = st.x[t] + (double)v.x * dt, y = st.y[t] + (double)v.y * dt, z = st.z[t] + (double)v.z * dt;
  st.x[t] = x;
  st.y[t] = y;
  st.z[t] = z;
  p.x = (float)x;
  p.y = (float)y;
  p.z = (float)z;
  st.pos_h[t] = p;
}
int launch_relax(const Dev& d, cudaStream_t s) { k_relax<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, d.s(), d.acc, d.P);  return 1; }

// ---------------------------------------------------------------------------------------------------
// 48-byte exchange layout (gpu_sph.rs:28) <-> internal state.
// ---------------------------------------------------------------------------------------------------
struct P48 {
  float px, py, pz, h, vx, vy, vz, u, mass;
  unsigned mat;
  float rho;
  unsigned prov;
};
static_assert(sizeof(P48) == 48, "SphParticle48 is 48 bytes");

__global__ void k_from_aos(int n, const P48* __restrict__ aos, const Seg* __restrict__ segs, int nseg, State st,
                           float* __restrict__ rho) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int lo = 0, hi = nseg - 1;  // the impact holding slot i: last segment starting at or before it
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].off <= (unsigned)i) lo = mid;
    else hi = mid - 1;
  }
  st.seg[i] = (unsigned)lo;
  const P48 p = aos[i];
  st.pos_h[i] = make_float4(p.px, p.py, p.pz, p.h);
  st.vel_u[i] = make_float4(p.vx, p.vy, p.vz, p.u);
  st.x[i] = (double)p.px;
  st.y[i] = (double)p.py;
  st.z[i] = (double)p.pz;
  st.mass[i] = p.mass;
  st.mat[i] = p.mat;
  st.prov[i] = p.prov;
  st.id[i] = (unsigned)i;
  rho[i] = p.rho;
}
int launch_from_aos(const Dev& d, cudaStream_t s) {
  k_from_aos<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, (const P48*)d.aos, d.segs, d.nseg, d.s(), d.rho);
  return 1;
}

// Upload validation on the device (the host would walk every record): the first particle whose material is
// outside the table or that has a non-finite field, a non-positive h or a negative mass.
__global__ void k_validate_aos(int n, const P48* __restrict__ aos, unsigned ne, unsigned* __restrict__ first_bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const P48 p = aos[i];
  const bool ok = p.mat < ne && isfinite(p.px) && isfinite(p.py) && isfinite(p.pz) && isfinite(p.vx) &&
                  isfinite(p.vy) && isfinite(p.vz) && isfinite(p.u) && isfinite(p.mass) && p.h > 0.0f &&
                  isfinite(p.h) && p.mass >= 0.0f;
  if (!ok) atomicMin(first_bad, (unsigned)i);
}
int launch_validate_aos(const Dev& d, int n, unsigned ne, unsigned* first_bad, cudaStream_t s) {
  k_validate_aos<<<(n + 255) / 256, 256, 0, s>>>(n, (const P48*)d.aos, ne, first_bad);
  return 1;
}

__global__ void k_to_aos(int n, State st, const float* __restrict__ rho, P48* __restrict__ aos) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float4 p = st.pos_h[t];
  const float4 v = st.vel_u[t];
  P48 o;
  o.px = (float)st.x[t];
  o.py = (float)st.y[t];
  o.pz = (float)st.z[t];
  o.h = p.w;
  o.vx = v.x;
  o.vy = v.y;
  o.vz = v.z;
  o.u = v.w;
  o.mass = st.mass[t];
  o.mat = st.mat[t];
  o.rho = rho[t];
  o.prov = st.prov[t];
  aos[st.id[t]] = o;
}
int launch_to_aos(const Dev& d, cudaStream_t s) {
  k_to_aos<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, d.s(), d.rho, (P48*)d.aos);
  return 1;
}

// ---------------------------------------------------------------------------------------------------
// FP64 conservation sums, deterministic two-pass reduction: [mass, KE, IE, PE, p.xyz, L.xyz].
// ---------------------------------------------------------------------------------------------------
constexpr int DG_VALS = 10;
__global__ void k_diag_partial(int n, State st, const float4* __restrict__ grav, double* __restrict__ part) {
  double v[DG_VALS];
#pragma unroll
  for (int k = 0; k < DG_VALS; ++k) v[k] = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const double m = st.mass[t];
    const float4 vu = st.vel_u[t];
    const double vx = vu.x, vy = vu.y, vz = vu.z;
    const double x = st.x[t], y = st.y[t], z = st.z[t];
    v[0] += m;
    v[1] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
    v[2] += m * (double)vu.w;
    v[3] += grav ? 0.5 * m * (double)grav[t].w : 0.0;
    v[4] += m * vx;
    v[5] += m * vy;
    v[6] += m * vz;
    v[7] += m * (y * vz - z * vy);
    v[8] += m * (z * vx - x * vz);
    v[9] += m * (x * vy - y * vx);
  }
  __shared__ double s[DG_VALS][8];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < DG_VALS; ++k) {
    const double r = warp_sum(v[k]);
    if (lane == 0) s[k][w] = r;
  }
  __syncthreads();
  if (threadIdx.x < DG_VALS) {
    double r = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += s[threadIdx.x][k];
    part[blockIdx.x * 16 + threadIdx.x] = r;
  }
}
__global__ void k_diag_final(const double* __restrict__ part, int blocks, double* __restrict__ out) {
  if (threadIdx.x < DG_VALS) {
    double r = 0.0;
    for (int b = 0; b < blocks; ++b) r += part[b * 16 + threadIdx.x];
    out[threadIdx.x] = r;
  }
}
int launch_diag(const Dev& d, cudaStream_t s, double* out16) {
  k_diag_partial<<<d.diag_blocks, 256, 0, s>>>(d.n, d.s(), d.grav, d.diag_part);
  k_diag_final<<<1, 32, 0, s>>>(d.diag_part, d.diag_blocks, out16);
  return 2;
}

}  // namespace sphb
