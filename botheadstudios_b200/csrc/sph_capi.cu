// Host side of the C ABI (include/sph_b200.h): the context that owns device memory, the CUDA stream and
// the dispatch order of one KDK step. It mirrors the engine's GpuSph (crates/engine/src/gpu_sph.rs:742-922)
// and ParticleStore (gpu_store.rs): capacity clamping on upload, enqueue-only stepping, a two-phase
// non-blocking readback. Errors are status codes; nothing throws across the boundary.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include <chrono>
#include <thread>

#include "../../include/sph_b200.h"
#include "mlp.cuh"
#include "sph_kernels.cuh"

using namespace sphb;

struct sph_ctx {
  sph_config cfg{};
  Cfg kc{};
  Dev d{};
  Dev g{};                 // lazily allocated gravity-only state for sph_gravity
  bool g_alloc = false;
  cudaStream_t stream = nullptr;
  uint32_t capacity = 0;
  uint32_t n_eos = 0;
  bool uploaded = false;
  bool fresh = false;      // tree, neighbours, density, EOS and gravity are valid for the current positions
  bool evaluated = false;  // the tree, sorted state and gravity record are those of an evaluation of this state
  bool phi_valid = false;  // the gravity record's .w holds the potential of that evaluation
  // captured steady KDK sequence (two substeps), one per parity of the state double buffer
  cudaGraphExec_t kdk_graph[2] = {nullptr, nullptr};
  unsigned long long kdk_graph_launches = 0;  // kernels in one replay
  // learned smoothing lengths
  float* mlp_params = nullptr;  // [SPH_MLP_PARAMS] FP32 on the device
  MlpPacked* mlp_w = nullptr;
  bool mlp_rec = false;
  float* mlp_feat = nullptr;    // [cap][8] recorded features (original order)
  float* mlp_dh = nullptr;      // [cap] recorded Δlog h
  bool proposed = false;        // pos_h.w holds proposals for the next rebuild
  DevParams hp{};          // host copy of the host-owned fields
  void* pinned_aos = nullptr;
  cudaEvent_t rb_event = nullptr;
  bool rb_inflight = false;
  uint32_t rb_n = 0;
  double* d_diag = nullptr;
  unsigned* d_flag = nullptr;  // upload validation: the first invalid particle
  DiskWork* disk = nullptr;  // disk-measurement workspace (allocated by the first measurement)
  std::string err;
  int device = 0;
  std::vector<void*> allocs;
  // profiling
  bool prof_on = false;
  unsigned long long launches = 0;
  struct Rec { int ph; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  double prof_ms[SPH_PHASE_COUNT] = {0};
  unsigned long long prof_calls[SPH_PHASE_COUNT] = {0};
};

namespace {

// Neighbour-list skin after an upload or an unconverged smoothing-length solve (h may move up to 15 % per
// rebuild); the configured h_skin applies once every particle is near its smoothing length.
constexpr float kSkinWide = 0.15f;

sph_status cuda_fail(sph_ctx* c, cudaError_t e, const char* what) {
  if (c) {
    c->err = std::string(what) + ": " + cudaGetErrorString(e);
  }
  return e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA;
}
#define CK(call)                                                       \
  do {                                                                 \
    cudaError_t _e = (call);                                           \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call);           \
  } while (0)

template <typename T>
sph_status dalloc(sph_ctx* ctx, T** p, size_t count) {
  void* q = nullptr;
  const size_t bytes = count * sizeof(T) > 0 ? count * sizeof(T) : 16;
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
  ctx->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return SPH_OK;
}
#define ALLOC(ptr, count)                                              \
  do {                                                                 \
    sph_status _s = dalloc(ctx, &(ptr), (count));                      \
    if (_s != SPH_OK) return _s;                                       \
  } while (0)

sph_status alloc_dev(sph_ctx* ctx, Dev& d, uint32_t cap, uint32_t K, uint32_t nbr_cap, bool sph) {
  d.cap = (int)cap;
  d.K = (int)K;
  const size_t capw = ((size_t)cap + 31) / 32 * 32;
  // leaves: ceil(n_k / K) per impact, at most ceil(cap / K) + one partial leaf per extra impact
  const size_t Lmax = ((size_t)cap + K - 1) / K + kMaxSegments;
  const size_t nodes = 2 * Lmax;
  for (int b = 0; b < 2; ++b) {
    State& s = d.st[b];
    ALLOC(s.pos_h, capw + 32);  // + the sentinel record at index capw (the gather kernels' list filler)
    ALLOC(s.vel_u, capw + 32);
    ALLOC(s.x, capw);
    ALLOC(s.y, capw);
    ALLOC(s.z, capw);
    ALLOC(s.mass, capw + 32);
    ALLOC(s.mat, capw);
    ALLOC(s.prov, capw);
    ALLOC(s.id, capw);
    ALLOC(s.seg, capw);
    ALLOC(d.keys[b], capw);
    ALLOC(d.vals[b], capw);
  }
  ALLOC(d.body, capw);
  d.rs_tiles_cap = (int)radix_tiles((int)cap);
  ALLOC(d.rs_hist, 256 * (size_t)(d.rs_tiles_cap > 0 ? d.rs_tiles_cap : 1));
  ALLOC(d.rs_tot, 256);
  ALLOC(d.leaf_codes, Lmax);
  ALLOC(d.leaf_start, Lmax + 1);
  ALLOC(d.segs, (size_t)kMaxSegments + 1);
  ALLOC(d.left, Lmax);
  ALLOC(d.right, Lmax);
  ALLOC(d.parent, nodes);
  ALLOC(d.counters, Lmax);
  ALLOC(d.ncom, nodes);
  ALLOC(d.nbmin, nodes);
  ALLOC(d.nbmax, nodes);
  ALLOC(d.nq0, nodes);
  ALLOC(d.nq1, nodes);
  ALLOC(d.hcom, 2 * Lmax);
  ALLOC(d.hq0, 2 * Lmax);
  ALLOC(d.hq1, 2 * Lmax);
  ALLOC(d.hrc, Lmax);
  ALLOC(d.grav, capw);
  ALLOC(d.groups, Lmax);
  ALLOC(d.ngroups, 1);
  ALLOC(d.P, 1);
  if (sph) {
    d.nbr_cap = nbr_cap;
    ALLOC(d.nbr, capw * nbr_cap);
    ALLOC(d.nbr_cnt, capw);
    ALLOC(d.rho, capw);
    ALLOC(d.fdata, capw + 32);
    ALLOC(d.acc, capw);
    ALLOC(d.hnew, capw);
    ALLOC(d.h0, capw);
    ALLOC(d.divv, capw);
    ALLOC(d.pend[0], capw);
    ALLOC(d.pend[1], capw);
    ALLOC(d.pend_n, 2);
    ALLOC(d.eos, kMaxMaterials);
    d.diag_blocks = 148 * 2;
    ALLOC(d.diag_part, (size_t)d.diag_blocks * 16);
    uint8_t* aos = nullptr;
    ALLOC(aos, capw * 48);
    d.aos = aos;
    // The sentinel particle: massless, at rest, h = 0 and 1e18 m out on every axis, so it lies outside every
    // support (W, ∇W = 0) and its terms vanish; its force record (m 0, ρ 1, P/ρ² 0, c 0) keeps the AV finite.
    // The permutation and the passes write indices below n only, so it stays as written here.
    d.sent = (unsigned)capw;
    const float4 far = make_float4(1.0e18f, 1.0e18f, 1.0e18f, 0.0f), zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 rec = make_float4(0.0f, 1.0f, 0.0f, 0.0f);
    const float zm = 0.0f;
    for (int b = 0; b < 2; ++b) {
      CK(cudaMemcpy(d.st[b].pos_h + capw, &far, sizeof(far), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(d.st[b].vel_u + capw, &zero4, sizeof(zero4), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(d.st[b].mass + capw, &zm, sizeof(zm), cudaMemcpyHostToDevice));
    }
    CK(cudaMemcpy(d.fdata + capw, &rec, sizeof(rec), cudaMemcpyHostToDevice));
  }
  return SPH_OK;
}

int bits_for(uint32_t n) {
  int b = 1;
  while (b < 32 && (1ull << b) < (unsigned long long)n) ++b;
  return b;
}

cudaEvent_t pool_get(sph_ctx* ctx) {
  if (!ctx->pool.empty()) {
    cudaEvent_t e = ctx->pool.back();
    ctx->pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Runs `f` (which returns the number of kernels it launched) as phase `ph`, bracketed by events when
// profiling is on.
template <typename F>
void phase(sph_ctx* ctx, int ph, F&& f) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (ctx->prof_on) {
    a = pool_get(ctx);
    b = pool_get(ctx);
    cudaEventRecord(a, ctx->stream);
  }
  ctx->launches += (unsigned long long)f();
  if (ctx->prof_on) {
    cudaEventRecord(b, ctx->stream);
    ctx->recs.push_back({ph, a, b});
  }
}

// Push the host-owned DevParams fields (the block before the device-maintained reductions and counters).
sph_status push_params(sph_ctx* ctx, Dev& d) {
  const size_t bytes = offsetof(DevParams, flags);
  CK(cudaMemcpyAsync(d.P, &ctx->hp, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return SPH_OK;
}

sph_status init_params(sph_ctx* ctx, Dev& d) {
  DevParams p{};
  p = ctx->hp;
  p.flags = 0;
  p.max_nbr_seen = 0;
  p.steps = 0;
  CK(cudaMemcpyAsync(d.P, &p, sizeof(DevParams), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SPH_OK;
}

bool fused_walk(const sph_ctx* ctx) {
  return ctx->kc.gravity == SPH_GRAVITY_TREE && ctx->kc.mac == SPH_MAC_GROUP;
}

// One tree build + everything that depends only on positions (and h): sort, LBVH, gravity, neighbour
// lists, the smoothing-length solve, density and the EOS record. `potential`: the fused walk also sums the
// potential φ (the energy diagnostic's); a KDK step's walks leave it out (the reference computes the
// potential energy on demand, not in the step: gpu_sph.rs:628), and sph_diag fills it in when asked.
sph_status rebuild(sph_ctx* ctx, bool need_bbox, bool potential) {
  Dev& d = ctx->d;
  cudaStream_t s = ctx->stream;
  const Cfg& c = ctx->kc;
  phase(ctx, SPH_PHASE_SORT, [&] { return (need_bbox ? launch_bbox(d, s) : 0) + launch_sort_permute(d, s); });
  phase(ctx, SPH_PHASE_TREE, [&] { return launch_tree(d, c, ctx->cfg.theta, s); });
  const bool fused = fused_walk(ctx);
  ctx->evaluated = true;
  ctx->phi_valid = !fused || potential;  // the other gravity paths always write φ (or zero without gravity)
  phase(ctx, SPH_PHASE_GRAVITY, [&] {
    if (fused) return launch_walk(d, c, potential, s);  // gravity + neighbour lists in one walk
    if (c.gravity == SPH_GRAVITY_TREE) return launch_gravity_tree(d, c, s);
    if (c.gravity == SPH_GRAVITY_DIRECT) return launch_gravity_direct(d, s);
    cudaMemsetAsync(d.grav, 0, sizeof(float4) * (size_t)d.n, s);
    return 0;
  });
  if (!fused) phase(ctx, SPH_PHASE_NEIGHBOURS, [&] { return launch_neighbours(d, c, s); });
  // with the smoothing-length solve, its final (residual) pass is the density + EOS pass; learned h checks
  // the proposals written before this rebuild and iterates only the rejected particles
  const bool learned = c.learned && ctx->proposed;
  ctx->proposed = false;
  if (c.h_solve)
    phase(ctx, SPH_PHASE_HSOLVE, [&] { return learned ? launch_h_learned(d, c, s) : launch_h_solve(d, c, s); });
  else phase(ctx, SPH_PHASE_DENSITY, [&] { return launch_density_eos(d, c, s); });
  CK(cudaGetLastError());
  return SPH_OK;
}

void forces(sph_ctx* ctx) {
  phase(ctx, SPH_PHASE_FORCES, [&] { return launch_forces(ctx->d, ctx->kc, ctx->stream); });
}

sph_status check_ready(sph_ctx* ctx) {
  if (!ctx) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (!ctx->uploaded || ctx->d.n == 0) {
    ctx->err = "no particles uploaded";
    return SPH_ERR_STATE;
  }
  return SPH_OK;
}

void drop_graphs(sph_ctx* ctx) {
  for (auto& g : ctx->kdk_graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

// Upload of `nimp` impacts (particles [off[k], off[k+1]) of `particles`, softening soft[k]); the impacts
// are already validated as non-empty and within capacity. `on_device`: the particles are device memory
// produced by the library itself (the assembly), so they skip the host validation, and eos == nullptr keeps
// the material table.
sph_status upload_impl(sph_ctx* ctx, const SphParticle48* particles, const uint32_t* off, uint32_t nimp,
                       const SphEos48* eos, uint32_t n_eos, const float* soft, bool on_device = false) {
  cudaSetDevice(ctx->device);
  sph_status ret = SPH_OK;
  const uint32_t nu = nimp ? off[nimp] : 0u;
  const bool keep_eos = on_device && !eos;
  uint32_t ne = keep_eos ? ctx->n_eos : n_eos;
  if (ne > (uint32_t)kMaxMaterials) {
    ne = kMaxMaterials;
    ret = SPH_CLAMPED;
  }
  for (uint32_t k = 0; k < nimp; ++k)
    if (!std::isfinite(soft[k]) || soft[k] < 0.0f) {
      ctx->err = "impact " + std::to_string(k) + " has a negative or non-finite softening";
      return SPH_ERR_INVALID;
    }
  CK(cudaStreamSynchronize(ctx->stream));
  // the records go to the exchange buffer first and are checked there, before any state changes
  Dev& dv = ctx->d;
  if (nu)
    CK(cudaMemcpyAsync(dv.aos, particles, (size_t)nu * 48,
                       on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
  if (nu && !on_device) {
    unsigned bad = 0xffffffffu;
    CK(cudaMemsetAsync(ctx->d_flag, 0xff, sizeof(unsigned), ctx->stream));
    launch_validate_aos(dv, (int)nu, ne, ctx->d_flag, ctx->stream);
    CK(cudaMemcpyAsync(&bad, ctx->d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (bad != 0xffffffffu) {
      ctx->err = "particle " + std::to_string(bad) + " has a material outside the table or a non-finite field";
      return SPH_ERR_INVALID;
    }
  }
  drop_graphs(ctx);
  Dev& d = ctx->d;
  d.n = (int)nu;
  d.cur = 0;
  d.nseg = nimp ? (int)nimp : 1;
  d.segbits = nimp > 1 ? bits_for(nimp) : 0;
  // segment table: each impact's leaves are K-particle buckets from its first particle
  std::vector<Seg> table((size_t)d.nseg + 1);
  uint32_t L = 0;
  for (uint32_t k = 0; k <= nimp; ++k) {
    Seg& g = table[k];
    std::memset(&g, 0, sizeof(g));
    g.off = k < nimp ? off[k] : nu;
    g.loff = L;
    g.sig_bits = 0x7f800000u;
    for (int a = 0; a < 3; ++a) g.bbox[a] = 0xffffffffu;
    g.soft2 = k < nimp ? soft[k] * soft[k] : 0.0f;
    g.skin = ctx->hp.skin_wide;  // new positions: the first rebuild's solve gets the wide skin
    g.dt = ctx->hp.dt_fixed;
    if (k < nimp) L += (off[k + 1] - off[k] + (uint32_t)d.K - 1) / (uint32_t)d.K;
  }
  d.L = (int)L;
  ctx->n_eos = ne;
  if (!keep_eos) {
    Eos etab[kMaxMaterials];
    std::memset(etab, 0, sizeof(etab));
    if (ne) std::memcpy(etab, eos, (size_t)ne * sizeof(Eos));
    CK(cudaMemcpyAsync(d.eos, etab, sizeof(etab), cudaMemcpyHostToDevice, ctx->stream));
  }
  CK(cudaMemcpyAsync(d.segs, table.data(), table.size() * sizeof(Seg), cudaMemcpyHostToDevice, ctx->stream));
  sph_status st = push_params(ctx, d);
  if (st != SPH_OK) return st;
  if (nu) {
    launch_from_aos(d, ctx->stream);
    launch_segments(d, ctx->stream);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->uploaded = true;
  ctx->fresh = false;
  ctx->evaluated = false;
  ctx->phi_valid = false;
  return ret;
}

// One KDK substep from a fresh state (tree, gravity, neighbours and density valid for the positions). It
// rebuilds once, so it flips the state double buffer.
sph_status kdk_steady(sph_ctx* ctx) {
  Dev& d = ctx->d;
  cudaStream_t s = ctx->stream;
  forces(ctx);
  phase(ctx, SPH_PHASE_INTEGRATE, [&] { return launch_finalize_dt(d, s) + launch_kick_drift(d, s); });
  if (ctx->kc.learned || ctx->mlp_rec) {
    // the network's Δlog h from the state at the start of the drift (counted with the smoothing-length phase)
    const MlpFeatureArgs fa{ctx->kc.h_eta, ctx->cfg.h_neighbours};
    phase(ctx, SPH_PHASE_HSOLVE, [&] {
      return launch_mlp_propose(d, ctx->mlp_w, fa, d.divv, ctx->mlp_rec ? ctx->mlp_feat : nullptr,
                                ctx->mlp_rec ? ctx->mlp_dh : nullptr, ctx->kc.learned != 0, s);
    });
    ctx->proposed = ctx->kc.learned != 0;
  }
  sph_status st = rebuild(ctx, false, false);
  if (st != SPH_OK) return st;
  forces(ctx);
  phase(ctx, SPH_PHASE_INTEGRATE, [&] { return launch_kick(d, s); });
  return SPH_OK;
}

// The potential φ of the last evaluation, when its walk left it out: one potential-only walk over that
// evaluation's tree (the positions have not moved since: a KDK step ends with a kick). Enqueued on the stream.
void ensure_potential(sph_ctx* ctx) {
  if (ctx->phi_valid || !ctx->evaluated || !ctx->d.n) return;
  ctx->launches += launch_potential(ctx->d, ctx->kc, ctx->stream);
  ctx->phi_valid = true;
}

// Two steady substeps as one CUDA graph launch. Two substeps flip the double buffer twice, so a graph
// captured with the buffer in one parity replays from that parity; one graph per parity is kept until the
// next upload. Everything the kernels read that the host may change between replays (dt, AV, omega) is in
// device memory, and every launch shape depends only on the uploaded particle and leaf counts.
sph_status kdk_graph_launch(sph_ctx* ctx) {
  Dev& d = ctx->d;
  const int par = d.cur;
  cudaStream_t s = ctx->stream;
  if (!ctx->kdk_graph[par]) {
    const unsigned long long l0 = ctx->launches;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    sph_status st = kdk_steady(ctx);
    if (st == SPH_OK) st = kdk_steady(ctx);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    if (st != SPH_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return cuda_fail(ctx, ei, "cudaGraphInstantiate");
    ctx->kdk_graph[par] = ex;
    ctx->kdk_graph_launches = ctx->launches - l0;
    ctx->launches = l0;  // capture launched nothing
  }
  CK(cudaGraphLaunch(ctx->kdk_graph[par], s));
  ctx->launches += ctx->kdk_graph_launches;
  return SPH_OK;
}

}  // namespace

extern "C" {

const char* sph_status_string(sph_status s) {
  switch (s) {
    case SPH_OK: return "ok";
    case SPH_CLAMPED: return "clamped to capacity";
    case SPH_NOT_READY: return "not ready";
    case SPH_ERR_INVALID: return "invalid argument";
    case SPH_ERR_CUDA: return "CUDA error";
    case SPH_ERR_OOM: return "out of device memory";
    case SPH_ERR_TIMEOUT: return "timeout";
    case SPH_ERR_OVERFLOW: return "device capacity overflow";
    case SPH_ERR_STATE: return "call out of order";
  }
  return "unknown status";
}

sph_status sph_config_default(sph_config* cfg) {
  if (!cfg) return SPH_ERR_INVALID;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->G = 6.674e-11;          // sph_step.wgsl:21
  cfg->theta = 0.5f;           // gpu_gravity.rs:55
  cfg->leaf_size = 1;          // gpu_gravity.rs:61
  cfg->kernel = SPH_KERNEL_CUBIC;
  cfg->gravity = SPH_GRAVITY_TREE;
  cfg->multipole = SPH_MULTIPOLE_MONOPOLE;
  cfg->precision = SPH_PRECISION_F32;
  cfg->h_mode = SPH_H_FIXED;
  cfg->h_neighbours = 64.0f;
  cfg->h_tol = 1.0e-3f;
  cfg->h_iters = 3;
  cfg->max_neighbours = 256;   // the offline driver's deep buckets (tools/impact-run/src/main.rs:77)
  cfg->cfl = 0.0f;
  cfg->rho_floor = 1.0e-9f;
  cfg->du_floor = 1.0f;
  cfg->r_min = 1.0e-9f;
  cfg->sig_floor = 1.0f;
  cfg->device = -1;
  cfg->local_theta = kLocalThetaDefault;
  return SPH_OK;
}

sph_status sph_create(const sph_config* cfg, uint32_t capacity, sph_ctx** out) {
  if (!cfg || !out) return SPH_ERR_INVALID;
  *out = nullptr;
  if (cfg->leaf_size < 1 || cfg->leaf_size > 32 || !(cfg->theta > 0.0f) || cfg->kernel > 1 || cfg->gravity > 2 ||
      cfg->multipole > 1 || cfg->precision > 1 || cfg->h_mode > 2 || cfg->max_neighbours < 1 ||
      cfg->max_neighbours > 4096 || capacity > (1u << 26) || cfg->mac > 1 ||
      (cfg->block_threads != 0 && (cfg->block_threads < 64 || cfg->block_threads > 1024 || cfg->block_threads % 32)) ||
      (cfg->walk_warps != 0 && cfg->walk_warps != 2 && cfg->walk_warps != 4 && cfg->walk_warps != 8) ||
      !(cfg->h_skin >= 0.0f && cfg->h_skin <= 0.5f) || !(cfg->local_theta >= 0.0f && cfg->local_theta < 1.0f) ||
      (cfg->mac == SPH_MAC_GROUP && (cfg->leaf_size & (cfg->leaf_size - 1)) != 0))
    return SPH_ERR_INVALID;
  sph_ctx* ctx = new (std::nothrow) sph_ctx();
  if (!ctx) return SPH_ERR_OOM;
  ctx->cfg = *cfg;
  ctx->capacity = capacity < 1 ? 1 : capacity;  // GpuSph::new: capacity.max(1)
  ctx->kc.kernel = (int)cfg->kernel;
  ctx->kc.gravity = (int)cfg->gravity;
  ctx->kc.quad = cfg->multipole == SPH_MULTIPOLE_QUADRUPOLE;
  ctx->kc.hilo = cfg->precision == SPH_PRECISION_HILO;
  ctx->kc.h_solve = cfg->h_mode == SPH_H_SOLVE || cfg->h_mode == SPH_H_LEARNED;
  ctx->kc.learned = cfg->h_mode == SPH_H_LEARNED;
  ctx->kc.divv = ctx->kc.learned;
  ctx->kc.h_eta = std::cbrt(3.0f * cfg->h_neighbours / (4.0f * 3.14159265358979f));
  ctx->kc.h_tol = cfg->h_tol;
  ctx->kc.h_iters = (int)cfg->h_iters;
  ctx->kc.walk_stack = (int)std::min<uint32_t>(cfg->walk_stack, 1u << 20);
  ctx->kc.local_theta = cfg->local_theta;
  ctx->kc.skin = ctx->kc.h_solve ? (cfg->h_skin > 0.0f ? cfg->h_skin : 0.05f) : 0.0f;
  ctx->kc.mac = (int)cfg->mac;
  ctx->kc.blk = cfg->block_threads ? (int)cfg->block_threads : 256;
  ctx->kc.walk_warps = cfg->walk_warps ? (int)cfg->walk_warps : 2;
  if (cfg->device >= 0) {
    cudaError_t de = cudaSetDevice(cfg->device);
    if (de != cudaSuccess) {
      delete ctx;
      return SPH_ERR_INVALID;
    }
  }
  cudaGetDevice(&ctx->device);
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    sph_status st = cuda_fail(ctx, e, "cudaStreamCreate");
    delete ctx;
    return st;
  }
  sph_status st = alloc_dev(ctx, ctx->d, ctx->capacity, cfg->leaf_size, cfg->max_neighbours, true);
  if (st == SPH_OK) {
    e = cudaMallocHost(&ctx->pinned_aos, (size_t)ctx->capacity * 48);
    if (e != cudaSuccess) st = cuda_fail(ctx, e, "cudaMallocHost");
  }
  if (st == SPH_OK) {
    e = cudaEventCreateWithFlags(&ctx->rb_event, cudaEventDisableTiming);
    if (e != cudaSuccess) st = cuda_fail(ctx, e, "cudaEventCreate");
  }
  if (st == SPH_OK) st = dalloc(ctx, &ctx->d_diag, 16);
  if (st == SPH_OK) st = dalloc(ctx, &ctx->d_flag, 1);
  if (st == SPH_OK) st = dalloc(ctx, &ctx->mlp_params, (size_t)MLP_TOTAL);
  if (st == SPH_OK) st = dalloc(ctx, &ctx->mlp_w, 1);
  if (st == SPH_OK) {
    // the zero network: Δlog h = 0 (unit scales so that the normalisation is well defined)
    std::vector<float> z(MLP_TOTAL, 0.0f);
    for (int k = 0; k < MLP_IN; ++k) z[MLP_XS + k] = 1.0f;
    z[MLP_YS] = 1.0f;
    cudaError_t e2 = cudaMemcpy(ctx->mlp_params, z.data(), z.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e2 == cudaSuccess) {
      launch_mlp_pack(ctx->mlp_params, ctx->mlp_w, ctx->stream);
      e2 = cudaStreamSynchronize(ctx->stream);
    }
    if (e2 != cudaSuccess) st = cuda_fail(ctx, e2, "mlp init");
  }
  if (st == SPH_OK) {
    DevParams& p = ctx->hp;
    std::memset(&p, 0, sizeof(p));
    p.dt_fixed = 0.0;
    p.av_alpha = 1.0f;  // gpu_sph.rs:833 SphParams defaults
    p.av_beta = 2.0f;
    p.damp = 1.0f;
    p.omega = 0.0f;
    p.G = (float)cfg->G;
    p.theta = cfg->theta;
    p.cfl = cfg->cfl;
    p.rho_floor = cfg->rho_floor;
    p.du_floor = cfg->du_floor;
    p.r_min = cfg->r_min;
    p.sig_floor = cfg->sig_floor;
    p.skin_narrow = ctx->kc.skin;
    p.skin_wide = ctx->kc.skin > kSkinWide ? ctx->kc.skin : kSkinWide;
    p.skin_reset = 10.0f * cfg->h_tol;
    st = init_params(ctx, ctx->d);
  }
  if (st != SPH_OK) {
    sph_destroy(ctx);
    return st;
  }
  *out = ctx;
  return SPH_OK;
}

void sph_destroy(sph_ctx* ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& r : ctx->recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (cudaEvent_t e : ctx->pool) cudaEventDestroy(e);
  drop_graphs(ctx);
  disk_work_free(ctx->disk);
  for (void* p : ctx->allocs) cudaFree(p);
  if (ctx->pinned_aos) cudaFreeHost(ctx->pinned_aos);
  if (ctx->rb_event) cudaEventDestroy(ctx->rb_event);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

sph_status sph_upload(sph_ctx* ctx, const SphParticle48* particles, uint32_t n, const SphEos48* eos, uint32_t n_eos,
                      float softening) {
  if (!ctx || (!particles && n) || (!eos && n_eos)) return SPH_ERR_INVALID;
  if (!std::isfinite(softening) || softening < 0.0f) return SPH_ERR_INVALID;
  sph_status ret = SPH_OK;
  uint32_t nu = n;
  if (nu > ctx->capacity) {
    nu = ctx->capacity;
    ret = SPH_CLAMPED;
  }
  const uint32_t off[2] = {0u, nu};
  const sph_status st = upload_impl(ctx, particles, off, nu ? 1u : 0u, eos, n_eos, &softening);
  return st == SPH_OK ? ret : st;
}

sph_status sph_upload_batch(sph_ctx* ctx, const SphParticle48* particles, const uint32_t* offsets,
                            uint32_t n_impacts, const SphEos48* eos, uint32_t n_eos, const float* softening) {
  if (!ctx || !particles || !offsets || !softening || (!eos && n_eos)) return SPH_ERR_INVALID;
  if (n_impacts < 1 || n_impacts > (uint32_t)kMaxSegments || offsets[0] != 0u) {
    ctx->err = "sph_upload_batch: need 1..256 impacts and offsets[0] = 0";
    return SPH_ERR_INVALID;
  }
  for (uint32_t k = 0; k < n_impacts; ++k)
    if (offsets[k + 1] <= offsets[k]) {
      ctx->err = "sph_upload_batch: impact " + std::to_string(k) + " is empty or the offsets decrease";
      return SPH_ERR_INVALID;
    }
  if (offsets[n_impacts] > ctx->capacity) {
    ctx->err = "sph_upload_batch: the batch holds more particles than the context capacity";
    return SPH_ERR_INVALID;
  }
  return upload_impl(ctx, particles, offsets, n_impacts, eos, n_eos, softening);
}

sph_status sph_set_dt(sph_ctx* ctx, double dt, float damp) {
  if (!ctx || !std::isfinite(dt) || dt < 0.0 || !std::isfinite(damp)) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  ctx->hp.dt_fixed = dt;
  ctx->hp.damp = damp;
  return push_params(ctx, ctx->d);
}

sph_status sph_set_av(sph_ctx* ctx, float alpha, float beta) {
  if (!ctx || !std::isfinite(alpha) || !std::isfinite(beta)) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  ctx->hp.av_alpha = alpha;
  ctx->hp.av_beta = beta;
  return push_params(ctx, ctx->d);
}

sph_status sph_set_omega(sph_ctx* ctx, float omega) {
  if (!ctx || !std::isfinite(omega)) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  ctx->hp.omega = omega;
  return push_params(ctx, ctx->d);
}

sph_status sph_eval_forces(sph_ctx* ctx) {
  sph_status st = check_ready(ctx);
  if (st != SPH_OK) return st;
  st = rebuild(ctx, true, true);
  if (st != SPH_OK) return st;
  forces(ctx);
  CK(cudaGetLastError());
  ctx->fresh = true;
  return SPH_OK;
}

sph_status sph_step_kdk(sph_ctx* ctx, uint32_t substeps) {
  sph_status st = check_ready(ctx);
  if (st != SPH_OK) return st;
  const bool graphs = ctx->cfg.graph != 0 && !ctx->prof_on;
  for (uint32_t k = 0; k < substeps;) {
    // eval 1 at x_n (the tree, gravity and density of the previous eval 2 are still exact: a kick moves no
    // particle), then dt, the half-kick + drift, eval 2 at x_{n+1}, the final half-kick.
    if (!ctx->fresh) {
      st = rebuild(ctx, true, false);
      if (st != SPH_OK) return st;
      ctx->fresh = true;
    }
    if (graphs && substeps - k >= 2) {
      st = kdk_graph_launch(ctx);
      if (st != SPH_OK) return st;
      k += 2;
      continue;
    }
    st = kdk_steady(ctx);
    if (st != SPH_OK) return st;
    ++k;
  }
  // graph replays run the captured walks without passing through rebuild(): mark the potential stale here
  if (substeps && fused_walk(ctx)) ctx->phi_valid = false;
  CK(cudaGetLastError());
  return SPH_OK;
}

sph_status sph_step_relax(sph_ctx* ctx, uint32_t steps) {
  sph_status st = check_ready(ctx);
  if (st != SPH_OK) return st;
  for (uint32_t k = 0; k < steps; ++k) {
    // the relaxation moves the particles after this evaluation: its walk sums the potential
    st = rebuild(ctx, true, true);
    if (st != SPH_OK) return st;
    forces(ctx);
    phase(ctx, SPH_PHASE_INTEGRATE, [&] { return launch_relax(ctx->d, ctx->stream); });
    ctx->fresh = false;
  }
  CK(cudaGetLastError());
  return SPH_OK;
}

sph_status sph_readback_begin(sph_ctx* ctx) {
  if (!ctx) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->rb_inflight || ctx->d.n == 0) return SPH_OK;  // gpu_store.rs: no-op if empty or in flight
  launch_to_aos(ctx->d, ctx->stream);
  CK(cudaMemcpyAsync(ctx->pinned_aos, ctx->d.aos, (size_t)ctx->d.n * 48, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaEventRecord(ctx->rb_event, ctx->stream));
  ctx->rb_inflight = true;
  ctx->rb_n = (uint32_t)ctx->d.n;
  return SPH_OK;
}

sph_status sph_readback_take(sph_ctx* ctx, SphParticle48* out, uint32_t cap, uint32_t* n_out, int* ready) {
  if (!ctx || !out || !n_out || !ready) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  *ready = 0;
  *n_out = 0;
  if (!ctx->rb_inflight) return SPH_NOT_READY;
  cudaError_t e = cudaEventQuery(ctx->rb_event);
  if (e == cudaErrorNotReady) return SPH_NOT_READY;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaEventQuery");
  const uint32_t m = ctx->rb_n < cap ? ctx->rb_n : cap;
  std::memcpy(out, ctx->pinned_aos, (size_t)m * 48);
  *n_out = m;
  *ready = 1;
  ctx->rb_inflight = false;
  return m < ctx->rb_n ? SPH_CLAMPED : SPH_OK;
}

sph_status sph_readback_into(sph_ctx* ctx, SphParticle48* out, uint32_t cap, uint32_t* n_out) {
  if (!ctx || !out || !n_out) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  *n_out = 0;
  const uint32_t m = (uint32_t)ctx->d.n < cap ? (uint32_t)ctx->d.n : cap;
  if (m) {
    launch_to_aos(ctx->d, ctx->stream);
    CK(cudaMemcpyAsync(out, ctx->d.aos, (size_t)m * 48, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  *n_out = m;
  return m < (uint32_t)ctx->d.n ? SPH_CLAMPED : SPH_OK;
}

sph_status sph_sync(sph_ctx* ctx, uint32_t timeout_ms) {
  if (!ctx) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (timeout_ms == 0) {
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
  }
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(ctx->stream);
    if (e == cudaSuccess) return SPH_OK;
    if (e != cudaErrorNotReady) return cuda_fail(ctx, e, "cudaStreamQuery");
    if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms)) {
      ctx->err = "sph_sync timed out";
      return SPH_ERR_TIMEOUT;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

uint32_t sph_count(const sph_ctx* ctx) { return ctx ? (uint32_t)ctx->d.n : 0u; }

sph_status sph_particle_buffer(sph_ctx* ctx, void** device_ptr) {
  if (!ctx || !device_ptr) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->d.n) launch_to_aos(ctx->d, ctx->stream);
  CK(cudaGetLastError());
  *device_ptr = ctx->d.aos;
  return SPH_OK;
}

void* sph_stream(sph_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
const char* sph_last_error(const sph_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

sph_status sph_body_bulk(sph_ctx* ctx, uint32_t prov, double centre[3], double* mass, double* radius) {
  if (!ctx || !centre || !mass || !radius) return SPH_ERR_INVALID;
  if (!ctx->uploaded) {
    ctx->err = "sph_body_bulk: nothing uploaded";
    return SPH_ERR_STATE;
  }
  cudaSetDevice(ctx->device);
  double v[5];
  unsigned long long launches = 0;
  const char* msg = "";
  const int rc = body_bulk(ctx->d, prov, ctx->disk, v, &launches, &msg, ctx->stream);
  ctx->launches += launches;
  if (rc) {
    ctx->err = msg;
    return (sph_status)rc;
  }
  for (int k = 0; k < 3; ++k) centre[k] = v[k];
  *mass = v[3];
  *radius = v[4];
  return SPH_OK;
}

sph_status sph_assemble(sph_ctx* ctx, const sph_placement* placements, uint32_t n_placements, float* softening,
                        float* dt) {
  if (!ctx || (!placements && n_placements) || !softening || !dt) return SPH_ERR_INVALID;
  if (!ctx->uploaded) {
    ctx->err = "sph_assemble: nothing uploaded";
    return SPH_ERR_STATE;
  }
  if (n_placements > (uint32_t)kMaxSegments) {
    ctx->err = "sph_assemble: at most 256 placements";
    return SPH_ERR_INVALID;
  }
  for (uint32_t k = 0; k < n_placements; ++k)
    for (int j = 0; j < 3; ++j)
      if (!std::isfinite(placements[k].offset[j]) || !std::isfinite(placements[k].vel[j]) ||
          !std::isfinite(placements[k].spin[j])) {
        ctx->err = "sph_assemble: placement " + std::to_string(k) + " has a non-finite component";
        return SPH_ERR_INVALID;
      }
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  const uint32_t n = (uint32_t)ctx->d.n;
  void* dst = nullptr;
  if (n) CK(cudaMalloc(&dst, (size_t)n * 48));
  std::vector<double> pl((size_t)n_placements * 9);
  for (uint32_t k = 0; k < n_placements; ++k)
    for (int j = 0; j < 3; ++j) {
      pl[k * 9 + j] = placements[k].offset[j];
      pl[k * 9 + 3 + j] = placements[k].vel[j];
      pl[k * 9 + 6 + j] = placements[k].spin[j];
    }
  unsigned n_out = 0;
  float min_h = 0.0f;
  unsigned long long launches = 0;
  const char* msg = "";
  int rc = assemble_n(ctx->d, pl.data(), n_placements, dst, &n_out, &min_h, ctx->disk, &launches, &msg,
                      ctx->stream);
  ctx->launches += launches;
  sph_status st = SPH_OK;
  if (rc) {
    ctx->err = msg;
    st = (sph_status)rc;
  } else if (n_out == 0) {
    ctx->err = "sph_assemble: no particle's prov has a placement";
    st = SPH_ERR_INVALID;
  } else {
    // gpu_sph.rs:334-338: softening = a quarter of the finest h, dt shock-safe against the fastest approach
    const float soft = 0.25f * min_h;
    double vmax = 0.0;
    for (uint32_t k = 0; k < n_placements; ++k) {
      const double* v = placements[k].vel;
      vmax = std::max(vmax, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    }
    *softening = soft;
    *dt = (float)(0.01 * (double)min_h / (20000.0 + vmax));
    const uint32_t off[2] = {0u, n_out};
    st = upload_impl(ctx, (const SphParticle48*)dst, off, 1u, nullptr, 0u, &soft, true);
  }
  if (dst) cudaFree(dst);
  return st;
}

sph_status sph_measure_default(sph_measure_cfg* cfg) {
  if (!cfg) return SPH_ERR_INVALID;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->remnant_frac = 0.85;   // main.rs:744
  cfg->link_factor = 2.0;     // main.rs:810
  cfg->roche = 2.44;          // main.rs:840
  cfg->rho_fallback = 2700.0; // main.rs:836
  cfg->pe_floor = 1.0;        // main.rs:846
  cfg->pe_softening = 1.0e4;  // gpu_sph.rs:458
  return SPH_OK;
}

sph_status sph_measure_disk(sph_ctx* ctx, uint32_t impact, const sph_measure_cfg* cfg, sph_disk_measure* out) {
  if (!ctx || !cfg || !out) return SPH_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  if (!ctx->uploaded) {
    ctx->err = "sph_measure_disk: nothing uploaded";
    return SPH_ERR_STATE;
  }
  if (impact >= (uint32_t)ctx->d.nseg) {
    ctx->err = "sph_measure_disk: impact " + std::to_string(impact) + " is outside the batch";
    return SPH_ERR_INVALID;
  }
  if (cfg->variant < 0 || cfg->variant > 1 || !(cfg->remnant_frac > 0.0 && cfg->remnant_frac <= 1.0) ||
      !(cfg->link_factor > 0.0) || !(cfg->roche >= 0.0) || !std::isfinite(cfg->G) || cfg->G < 0.0 ||
      !(cfg->pe_floor >= 0.0) || !(cfg->pe_softening >= 0.0)) {
    ctx->err = "sph_measure_disk: variant 0|1, remnant_frac in (0, 1], link_factor > 0, non-negative constants";
    return SPH_ERR_INVALID;
  }
  cudaSetDevice(ctx->device);
  Seg seg[2];
  CK(cudaMemcpyAsync(seg, ctx->d.segs + impact, 2 * sizeof(Seg), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const unsigned off = seg[0].off, m = seg[1].off - off;  // the table closes with entry nseg (off = n)
  const DiskCfg dc{cfg->variant, cfg->G != 0.0 ? cfg->G : ctx->cfg.G, cfg->remnant_frac, cfg->link_factor,
                   cfg->roche, cfg->rho_fallback, cfg->pe_floor, cfg->pe_softening};
  double v[16];
  unsigned long long launches = 0;
  const char* msg = "";
  const int rc = disk_measure(ctx->d, off, m, dc, ctx->disk, v, &launches, &msg, ctx->stream);
  ctx->launches += launches;
  if (rc) {
    ctx->err = msg;
    return (sph_status)rc;
  }
  out->earth_frac = v[0];
  out->disk_mass = v[1];
  out->disk_target = v[2];
  out->disk_impactor = v[3];
  out->remnant_target = v[4];
  out->remnant_impactor = v[5];
  out->escaped_target = v[6];
  out->escaped_impactor = v[7];
  out->r_remnant = v[8];
  out->m_remnant = v[9];
  out->clump_mass = v[10];
  out->clump_target_frac = v[11];
  out->clump_n = (uint32_t)v[12];
  out->n_clumps = (uint32_t)v[13];
  out->n_bound = (uint32_t)v[14];
  out->n_disk = (uint32_t)v[15];
  return SPH_OK;
}

sph_status sph_diag(sph_ctx* ctx, sph_diag_out* out) {
  if (!ctx || !out) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  std::memset(out, 0, sizeof(*out));
  ensure_potential(ctx);
  if (ctx->d.n) launch_diag(ctx->d, ctx->stream, ctx->d_diag);
  double v[16] = {0};
  DevParams p;
  Seg s0;
  std::memset(&s0, 0, sizeof(s0));
  if (ctx->d.n) CK(cudaMemcpyAsync(v, ctx->d_diag, sizeof(v), cudaMemcpyDeviceToHost, ctx->stream));
  if (ctx->uploaded) CK(cudaMemcpyAsync(&s0, ctx->d.segs, sizeof(Seg), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&p, ctx->d.P, sizeof(p), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  out->mass = v[0];
  out->kinetic = v[1];
  out->internal = v[2];
  out->potential = v[3];
  for (int k = 0; k < 3; ++k) {
    out->momentum[k] = v[4 + k];
    out->angular_momentum[k] = v[7 + k];
  }
  out->dt = s0.dt;
  out->time = s0.time;
  out->steps = p.steps;
  out->max_neighbours_seen = p.max_nbr_seen;
  out->overflow_flags = p.flags;
  out->h_iterations = p.h_iters_used;
  out->h_residual = p.h_residual;
  out->h_accepted = p.h_accepted;
  out->walk_nodes = p.stat_visits;
  out->walk_pops = p.stat_pops;
  out->m2p_interactions = p.stat_m2p;
  out->p2p_interactions = p.stat_p2p;
  out->local_expansions = p.stat_m2l;
  out->p2p_slots = p.stat_p2p_slots;
  if (p.flags & (kFlagNbrOverflow | kFlagStackOverflow)) {
    ctx->err = "device capacity overflow (flags " + std::to_string(p.flags) + ")";
    return SPH_ERR_OVERFLOW;
  }
  return SPH_OK;
}

sph_status sph_inspect(sph_ctx* ctx, uint32_t what, void* host_out, size_t bytes) {
  if (!ctx || !host_out) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (what == SPH_Q_ACC_GRAV) ensure_potential(ctx);
  CK(cudaStreamSynchronize(ctx->stream));
  Dev& d = ctx->d;
  const size_t n = (size_t)d.n, L = (size_t)d.L;
  const size_t nn = L ? 2 * L - 1 : 0;
  auto need = [&](size_t b) { return bytes >= b; };
  std::vector<unsigned> ids;
  auto load_ids = [&]() -> sph_status {
    ids.resize(n);
    CK(cudaMemcpy(ids.data(), d.s().id, n * 4, cudaMemcpyDeviceToHost));
    return SPH_OK;
  };
  auto scatter = [&](const void* dev, size_t elem) -> sph_status {
    if (!need(n * elem)) return SPH_ERR_INVALID;
    std::vector<char> tmp(n * elem);
    CK(cudaMemcpy(tmp.data(), dev, n * elem, cudaMemcpyDeviceToHost));
    sph_status st = load_ids();
    if (st != SPH_OK) return st;
    for (size_t t = 0; t < n; ++t) std::memcpy((char*)host_out + ids[t] * elem, tmp.data() + t * elem, elem);
    return SPH_OK;
  };
  switch (what) {
    case SPH_Q_BBOX: {
      // as many impacts as the buffer holds
      const size_t m = std::min(bytes / 24, (size_t)d.nseg);
      if (m == 0) return SPH_ERR_INVALID;
      std::vector<Seg> tab(m);
      CK(cudaMemcpy(tab.data(), d.segs, m * sizeof(Seg), cudaMemcpyDeviceToHost));
      float* f = (float*)host_out;
      for (size_t g = 0; g < m; ++g)
        for (int k = 0; k < 6; ++k) {
          const unsigned key = tab[g].bbox[k];
          unsigned bits = (key >> 31) ? (key ^ 0x80000000u) : ~key;
          std::memcpy(&f[6 * g + k], &bits, 4);
        }
      return SPH_OK;
    }
    case SPH_Q_CODES: {
      if (!need(n * 4)) return SPH_ERR_INVALID;
      std::vector<unsigned long long> k(n);
      CK(cudaMemcpy(k.data(), d.keys[0], n * 8, cudaMemcpyDeviceToHost));
      for (size_t t = 0; t < n; ++t) ((unsigned*)host_out)[t] = (unsigned)(k[t] & 0x3fffffffu);
      return SPH_OK;
    }
    case SPH_Q_IMPACT_DT:
    case SPH_Q_IMPACT_TIME: {
      const size_t m = (size_t)d.nseg;
      if (!need(m * 8)) return SPH_ERR_INVALID;
      std::vector<Seg> tab(m);
      CK(cudaMemcpy(tab.data(), d.segs, m * sizeof(Seg), cudaMemcpyDeviceToHost));
      for (size_t g = 0; g < m; ++g) ((double*)host_out)[g] = what == SPH_Q_IMPACT_DT ? tab[g].dt : tab[g].time;
      return SPH_OK;
    }
    case SPH_Q_ORDER:
      if (!need(n * 4)) return SPH_ERR_INVALID;
      CK(cudaMemcpy(host_out, d.s().id, n * 4, cudaMemcpyDeviceToHost));
      return SPH_OK;
    case SPH_Q_LEFT:
    case SPH_Q_RIGHT:
      if (!need((L ? L - 1 : 0) * 4)) return SPH_ERR_INVALID;
      if (L > 1) CK(cudaMemcpy(host_out, what == SPH_Q_LEFT ? d.left : d.right, (L - 1) * 4, cudaMemcpyDeviceToHost));
      return SPH_OK;
    case SPH_Q_PARENT:
      if (!need(nn * 4)) return SPH_ERR_INVALID;
      CK(cudaMemcpy(host_out, d.parent, nn * 4, cudaMemcpyDeviceToHost));
      return SPH_OK;
    case SPH_Q_NODE_COM:
    case SPH_Q_NODE_BMIN:
    case SPH_Q_NODE_BMAX: {
      if (!need(nn * 16)) return SPH_ERR_INVALID;
      const float4* src = what == SPH_Q_NODE_COM ? d.ncom : (what == SPH_Q_NODE_BMIN ? d.nbmin : d.nbmax);
      CK(cudaMemcpy(host_out, src, nn * 16, cudaMemcpyDeviceToHost));
      return SPH_OK;
    }
    case SPH_Q_NBR_COUNT:
      return scatter(d.nbr_cnt, 4);
    case SPH_Q_NBR_LIST: {
      const size_t cap = d.nbr_cap;
      if (!need(n * cap * 4)) return SPH_ERR_INVALID;
      const size_t groups = (n + 31) / 32;
      std::vector<unsigned> lst(groups * cap * 32), cnt(n);
      CK(cudaMemcpy(lst.data(), d.nbr, lst.size() * 4, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(cnt.data(), d.nbr_cnt, n * 4, cudaMemcpyDeviceToHost));
      sph_status st = load_ids();
      if (st != SPH_OK) return st;
      unsigned* o = (unsigned*)host_out;
      std::memset(o, 0xff, n * cap * 4);
      for (size_t t = 0; t < n; ++t) {
        const size_t c = cnt[t] < cap ? cnt[t] : cap;
        for (size_t k = 0; k < c; ++k) o[ids[t] * cap + k] = ids[lst[((t >> 5) * cap + k) * 32 + (t & 31)]];
      }
      return SPH_OK;
    }
    case SPH_Q_RHO:
      return scatter(d.rho, 4);
    case SPH_Q_PRESSURE:
    case SPH_Q_SOUND: {
      if (!need(n * 4)) return SPH_ERR_INVALID;
      std::vector<float4> f(n);
      CK(cudaMemcpy(f.data(), d.fdata, n * 16, cudaMemcpyDeviceToHost));
      sph_status st = load_ids();
      if (st != SPH_OK) return st;
      for (size_t t = 0; t < n; ++t) {
        const float v = what == SPH_Q_PRESSURE ? f[t].z * (f[t].y * f[t].y) : f[t].w;
        ((float*)host_out)[ids[t]] = v;
      }
      return SPH_OK;
    }
    case SPH_Q_ACC_SPH: {
      // total acceleration minus gravity = the SPH part
      if (!need(n * 16)) return SPH_ERR_INVALID;
      std::vector<float4> a(n), g(n);
      CK(cudaMemcpy(a.data(), d.acc, n * 16, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(g.data(), d.grav, n * 16, cudaMemcpyDeviceToHost));
      sph_status st = load_ids();
      if (st != SPH_OK) return st;
      const bool sub = ctx->kc.gravity != SPH_GRAVITY_NONE;
      for (size_t t = 0; t < n; ++t) {
        float4 v = a[t];
        if (sub) {
          v.x -= g[t].x;
          v.y -= g[t].y;
          v.z -= g[t].z;
        }
        ((float4*)host_out)[ids[t]] = v;
      }
      return SPH_OK;
    }
    case SPH_Q_ACC_GRAV:
      return scatter(d.grav, 16);
    case SPH_Q_H: {
      if (!need(n * 4)) return SPH_ERR_INVALID;
      std::vector<float4> p(n);
      CK(cudaMemcpy(p.data(), d.s().pos_h, n * 16, cudaMemcpyDeviceToHost));
      sph_status st = load_ids();
      if (st != SPH_OK) return st;
      for (size_t t = 0; t < n; ++t) ((float*)host_out)[ids[t]] = p[t].w;
      return SPH_OK;
    }
    case SPH_Q_N_LEAVES:
      if (!need(4)) return SPH_ERR_INVALID;
      *(unsigned*)host_out = (unsigned)L;
      return SPH_OK;
  }
  return SPH_ERR_INVALID;
}

sph_status sph_profile_enable(sph_ctx* ctx, int on) {
  if (!ctx) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  for (auto& r : ctx->recs) {
    ctx->pool.push_back(r.a);
    ctx->pool.push_back(r.b);
  }
  ctx->recs.clear();
  for (int k = 0; k < SPH_PHASE_COUNT; ++k) {
    ctx->prof_ms[k] = 0.0;
    ctx->prof_calls[k] = 0;
  }
  ctx->launches = 0;
  ctx->prof_on = on != 0;
  return SPH_OK;
}

sph_status sph_profile_read(sph_ctx* ctx, sph_profile* out) {
  if (!ctx || !out) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  for (auto& r : ctx->recs) {
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, r.a, r.b));
    ctx->prof_ms[r.ph] += ms;
    ctx->prof_calls[r.ph] += 1;
    ctx->pool.push_back(r.a);
    ctx->pool.push_back(r.b);
  }
  ctx->recs.clear();
  for (int k = 0; k < SPH_PHASE_COUNT; ++k) {
    out->ms[k] = ctx->prof_ms[k];
    out->calls[k] = ctx->prof_calls[k];
  }
  out->kernel_launches = ctx->launches;
  return SPH_OK;
}

sph_status sph_gravity(sph_ctx* ctx, const double* pos3, const double* mass, uint32_t n, double softening,
                       uint32_t gravity_mode, double* acc3) {
  if (!ctx || (!pos3 && n) || (!mass && n) || (!acc3 && n) || gravity_mode > 1) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (n > ctx->capacity) {
    ctx->err = "sph_gravity: more points than the context capacity";
    return SPH_ERR_INVALID;
  }
  if (n == 0) return SPH_OK;
  if (!ctx->g_alloc) {
    sph_status st = alloc_dev(ctx, ctx->g, ctx->capacity, ctx->cfg.leaf_size, 0, false);
    if (st != SPH_OK) return st;
    ctx->g_alloc = true;
  }
  Dev& g = ctx->g;
  g.n = (int)n;
  g.cur = 0;
  g.L = (int)((n + g.K - 1) / g.K);
  g.nseg = 1;
  g.segbits = 0;
  std::vector<float4> ph(n);
  std::vector<double> xs(n), ys(n), zs(n);
  std::vector<float> ms(n);
  std::vector<unsigned> ids(n);
  for (uint32_t i = 0; i < n; ++i) {
    ph[i] = make_float4((float)pos3[3 * i], (float)pos3[3 * i + 1], (float)pos3[3 * i + 2], 0.0f);
    xs[i] = pos3[3 * i];
    ys[i] = pos3[3 * i + 1];
    zs[i] = pos3[3 * i + 2];
    ms[i] = (float)mass[i];
    ids[i] = i;
  }
  cudaStream_t s = ctx->stream;
  const State& st0 = g.st[0];
  CK(cudaMemcpyAsync(st0.pos_h, ph.data(), n * 16, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(st0.x, xs.data(), n * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(st0.y, ys.data(), n * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(st0.z, zs.data(), n * 8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(st0.mass, ms.data(), n * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(st0.id, ids.data(), n * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(st0.vel_u, 0, n * 16, s));
  CK(cudaMemsetAsync(st0.mat, 0, n * 4, s));
  CK(cudaMemsetAsync(st0.prov, 0, n * 4, s));
  CK(cudaMemsetAsync(st0.seg, 0, n * 4, s));
  DevParams p = ctx->hp;
  CK(cudaMemcpyAsync(g.P, &p, sizeof(p), cudaMemcpyHostToDevice, s));
  launch_segments_single(g, (float)softening * (float)softening, 0.0, s);
  launch_bbox(g, s);
  launch_sort_permute(g, s);
  if (gravity_mode == SPH_GRAVITY_TREE) {
    launch_tree(g, ctx->kc, ctx->cfg.theta, s);
    if (ctx->kc.mac == SPH_MAC_GROUP) launch_gravity_group(g, ctx->kc, s);
    else launch_gravity_tree(g, ctx->kc, s);
  } else {
    launch_gravity_direct(g, s);
  }
  CK(cudaGetLastError());
  std::vector<float4> acc(n);
  std::vector<unsigned> sid(n);
  CK(cudaMemcpyAsync(acc.data(), g.grav, n * 16, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(sid.data(), g.s().id, n * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (uint32_t t = 0; t < n; ++t) {
    acc3[3 * sid[t]] = acc[t].x;
    acc3[3 * sid[t] + 1] = acc[t].y;
    acc3[3 * sid[t] + 2] = acc[t].z;
  }
  return SPH_OK;
}

sph_status sph_gravity_direct64(sph_ctx* ctx, const double* pos3, const double* mass, uint32_t n,
                                const uint32_t* targets, uint32_t n_targets, double softening, double* acc3) {
  if (!ctx || !pos3 || !mass || !acc3 || n == 0) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  const uint32_t nt = targets ? n_targets : n;
  if (targets)
    for (uint32_t q = 0; q < nt; ++q)
      if (targets[q] >= n) return SPH_ERR_INVALID;
  double *dp = nullptr, *dm = nullptr, *da = nullptr;
  unsigned* dt = nullptr;
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMallocAsync(&dp, (size_t)n * 24, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&dm, (size_t)n * 8, s);
  if (e == cudaSuccess) e = cudaMallocAsync(&da, (size_t)nt * 24, s);
  if (e == cudaSuccess && targets) e = cudaMallocAsync(&dt, (size_t)nt * 4, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, pos3, (size_t)n * 24, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dm, mass, (size_t)n * 8, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && targets) e = cudaMemcpyAsync(dt, targets, (size_t)nt * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    launch_gravity_direct64(dp, dm, (int)n, dt, (int)nt, softening * softening, ctx->cfg.G, da, s);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(acc3, da, (size_t)nt * 24, cudaMemcpyDeviceToHost, s);
  if (dp) cudaFreeAsync(dp, s);
  if (dm) cudaFreeAsync(dm, s);
  if (da) cudaFreeAsync(da, s);
  if (dt) cudaFreeAsync(dt, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "sph_gravity_direct64");
  return SPH_OK;
}

sph_status sph_mlp_set(sph_ctx* ctx, const float* params, uint32_t count) {
  if (!ctx || !params || count != (uint32_t)MLP_TOTAL) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  for (uint32_t k = 0; k < count; ++k)
    if (!std::isfinite(params[k])) {
      ctx->err = "sph_mlp_set: parameter " + std::to_string(k) + " is not finite";
      return SPH_ERR_INVALID;
    }
  CK(cudaMemcpyAsync(ctx->mlp_params, params, count * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  launch_mlp_pack(ctx->mlp_params, ctx->mlp_w, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return SPH_OK;
}

sph_status sph_mlp_record(sph_ctx* ctx, int on) {
  if (!ctx) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  if (on && !ctx->mlp_feat) {
    sph_status st = dalloc(ctx, &ctx->mlp_feat, (size_t)ctx->capacity * MLP_IN);
    if (st == SPH_OK) st = dalloc(ctx, &ctx->mlp_dh, (size_t)ctx->capacity);
    if (st != SPH_OK) return st;
  }
  if (ctx->mlp_rec != (on != 0)) drop_graphs(ctx);  // the captured steps hold the recording pointers
  ctx->mlp_rec = on != 0;
  ctx->kc.divv = ctx->kc.learned || ctx->mlp_rec;
  return SPH_OK;
}

sph_status sph_mlp_features(sph_ctx* ctx, float* features, float* dlogh, uint32_t cap) {
  if (!ctx) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (!ctx->mlp_feat) {
    ctx->err = "sph_mlp_features: recording was never enabled";
    return SPH_ERR_STATE;
  }
  const uint32_t n = (uint32_t)ctx->d.n < cap ? (uint32_t)ctx->d.n : cap;
  if (features && n)
    CK(cudaMemcpyAsync(features, ctx->mlp_feat, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyDeviceToHost,
                       ctx->stream));
  if (dlogh && n)
    CK(cudaMemcpyAsync(dlogh, ctx->mlp_dh, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return n < (uint32_t)ctx->d.n ? SPH_CLAMPED : SPH_OK;
}

sph_status sph_set_progress(sph_ctx* ctx, float fraction) {
  if (!ctx || !std::isfinite(fraction)) return SPH_ERR_INVALID;
  cudaSetDevice(ctx->device);
  ctx->hp.progress = fraction;
  return push_params(ctx, ctx->d);
}

}  // extern "C"

// ---- granular contact context ---------------------------------------------------------------------------
// A grain set rides on an SPH context's sorted state, tree and neighbour lists (h = 2r + COH_RANGE); the
// 80-byte grain records stay resident in original order and receive positions/velocities on readback.
struct sph_dem {
  sph_ctx* base = nullptr;
  DemParams p{};
  int* terrain = nullptr;   // [wd][ww] heightfield (device), owned
  bool stepped = false;     // a substep ran since the last replace (the glow is then the integrator's)
  void* grains = nullptr;   // [cap] SphGrain80, original order
  float4* acc = nullptr;    // [cap][4] contact sums of the last substep (sorted order)
  uint32_t capacity = 0;
};

extern "C" {

sph_status sph_dem_create(uint32_t capacity, int32_t device, sph_dem** out) {
  if (!out) return SPH_ERR_INVALID;
  *out = nullptr;
  sph_config cfg;
  sph_config_default(&cfg);
  cfg.leaf_size = 8;
  cfg.gravity = SPH_GRAVITY_NONE;
  cfg.mac = SPH_MAC_GROUP;
  cfg.max_neighbours = 64;
  cfg.device = device;
  sph_dem* dem = new (std::nothrow) sph_dem();
  if (!dem) return SPH_ERR_OOM;
  sph_status st = sph_create(&cfg, capacity, &dem->base);
  if (st != SPH_OK) {
    delete dem;
    return st;
  }
  sph_ctx* ctx = dem->base;
  ctx->kc.nbr_skin = 1.0e-5f;  // contact candidates: a superset of the exact cut applied per pair
  dem->capacity = ctx->capacity;
  const size_t capw = ((size_t)dem->capacity + 31) / 32 * 32;
  uint8_t* g = nullptr;
  st = dalloc(ctx, &g, capw * 80);
  if (st == SPH_OK) st = dalloc(ctx, &dem->acc, capw * 4);
  if (st != SPH_OK) {
    sph_dem_destroy(dem);
    return st;
  }
  dem->grains = g;
  dem->p.dt = 1.0f / 60.0f;
  dem->p.gy = -9.81f;
  *out = dem;
  return SPH_OK;
}

void sph_dem_destroy(sph_dem* dem) {
  if (!dem) return;
  if (dem->terrain) {
    cudaSetDevice(dem->base->device);
    cudaStreamSynchronize(dem->base->stream);
    cudaFree(dem->terrain);
  }
  sph_destroy(dem->base);
  delete dem;
}

uint32_t sph_dem_count(const sph_dem* dem) { return dem ? (uint32_t)dem->base->d.n : 0u; }

sph_status sph_dem_set_params(sph_dem* dem, const sph_dem_params* p) {
  if (!dem || !p || !(p->dt > 0.0f) || !std::isfinite(p->dt)) return SPH_ERR_INVALID;
  DemParams& q = dem->p;
  q.gx = p->gravity[0];
  q.gy = p->gravity[1];
  q.gz = p->gravity[2];
  q.dt = p->dt;
  q.stiffness = p->c_stiffness;
  q.normal_damp = p->c_normal_damp;
  q.friction = p->c_friction;
  q.tangent_damp = p->c_tangent_damp;
  q.cohesion = p->c_cohesion;
  return SPH_OK;
}

sph_status sph_dem_set_ground(sph_dem* dem, const sph_dem_ground* g) {
  if (!dem || !g) return SPH_ERR_INVALID;
  const float v[7] = {g->center[0], g->center[1], g->center[2], g->air_rho, g->drag_cd, g->specific_heat,
                      g->cool_rate};
  for (float x : v)
    if (!std::isfinite(x)) return SPH_ERR_INVALID;
  if (g->air_rho < 0.0f || g->drag_cd < 0.0f || g->specific_heat < 0.0f || g->cool_rate < 0.0f)
    return SPH_ERR_INVALID;
  DemParams& q = dem->p;
  q.cx = g->center[0];
  q.cy = g->center[1];
  q.cz = g->center[2];
  q.air_rho = g->air_rho;
  q.drag_cd = g->drag_cd;
  q.specific_heat = g->specific_heat;
  q.cool_rate = g->cool_rate;
  return SPH_OK;
}

sph_status sph_dem_set_terrain(sph_dem* dem, const int32_t* heights, uint32_t w, uint32_t d) {
  if (!dem || ((w || d) && (!heights || !w || !d))) return SPH_ERR_INVALID;
  sph_ctx* ctx = dem->base;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->stream));
  if (dem->terrain) cudaFree(dem->terrain);
  dem->terrain = nullptr;
  dem->p.hf = nullptr;
  dem->p.ww = dem->p.wd = 0;
  if (!w) return SPH_OK;
  CK(cudaMalloc(&dem->terrain, sizeof(int) * (size_t)w * d));
  CK(cudaMemcpy(dem->terrain, heights, sizeof(int) * (size_t)w * d, cudaMemcpyHostToDevice));
  dem->p.hf = dem->terrain;
  dem->p.ww = w;
  dem->p.wd = d;
  return SPH_OK;
}

sph_status sph_dem_replace(sph_dem* dem, const SphGrain80* grains, uint32_t n) {
  if (!dem || (!grains && n)) return SPH_ERR_INVALID;
  sph_ctx* ctx = dem->base;
  cudaSetDevice(ctx->device);
  sph_status ret = SPH_OK;
  if (n > dem->capacity) {
    n = dem->capacity;
    ret = SPH_CLAMPED;
  }
  for (uint32_t i = 0; i < n; ++i) {
    const SphGrain80& g = grains[i];
    if (!std::isfinite(g.offset[0]) || !std::isfinite(g.offset[1]) || !std::isfinite(g.offset[2]) ||
        !std::isfinite(g.vel[0]) || !std::isfinite(g.vel[1]) || !std::isfinite(g.vel[2]) || !(g.radius > 0.0f) ||
        !std::isfinite(g.radius)) {
      ctx->err = "grain " + std::to_string(i) + " has a non-finite field or a non-positive radius";
      return SPH_ERR_INVALID;
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  Dev& d = ctx->d;
  d.n = (int)n;
  d.cur = 0;
  d.L = n ? (int)((n + d.K - 1) / d.K) : 0;
  d.nseg = 1;
  d.segbits = 0;
  dem->stepped = false;
  if (n) {
    CK(cudaMemcpyAsync(dem->grains, grains, (size_t)n * 80, cudaMemcpyHostToDevice, ctx->stream));
    launch_dem_load(d, dem->grains, ctx->stream);
    launch_segments_single(d, 0.0f, 0.0, ctx->stream);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->uploaded = true;
  ctx->fresh = false;
  ctx->evaluated = false;
  ctx->phi_valid = false;
  return ret;
}

sph_status sph_dem_step(sph_dem* dem, uint32_t substeps) {
  if (!dem) return SPH_ERR_INVALID;
  sph_ctx* ctx = dem->base;
  sph_status st = check_ready(ctx);
  if (st != SPH_OK) return st;
  Dev& d = ctx->d;
  cudaStream_t s = ctx->stream;
  for (uint32_t k = 0; k < substeps; ++k) {
    phase(ctx, SPH_PHASE_SORT, [&] { return launch_bbox(d, s) + launch_sort_permute(d, s); });
    phase(ctx, SPH_PHASE_TREE, [&] { return launch_tree(d, ctx->kc, ctx->cfg.theta, s); });
    phase(ctx, SPH_PHASE_NEIGHBOURS, [&] { return launch_neighbours(d, ctx->kc, s); });
    phase(ctx, SPH_PHASE_FORCES, [&] { return launch_dem_contacts(d, dem->p, dem->acc, s); });
    phase(ctx, SPH_PHASE_INTEGRATE, [&] { return launch_dem_integrate(d, dem->p, dem->acc, s); });
  }
  if (substeps) dem->stepped = true;
  CK(cudaGetLastError());
  return SPH_OK;
}

sph_status sph_dem_readback(sph_dem* dem, SphGrain80* out, uint32_t cap, uint32_t* n_out) {
  if (!dem || !out || !n_out) return SPH_ERR_INVALID;
  sph_ctx* ctx = dem->base;
  cudaSetDevice(ctx->device);
  const uint32_t n = (uint32_t)ctx->d.n;
  const uint32_t m = n < cap ? n : cap;
  *n_out = 0;
  if (n) launch_dem_store(ctx->d, dem->p, dem->stepped, dem->grains, ctx->stream);
  if (m) CK(cudaMemcpyAsync(out, dem->grains, (size_t)m * 80, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *n_out = m;
  return m < n ? SPH_CLAMPED : SPH_OK;
}

sph_status sph_dem_contacts(sph_dem* dem, float* out16, size_t bytes) {
  if (!dem || !out16) return SPH_ERR_INVALID;
  sph_ctx* ctx = dem->base;
  cudaSetDevice(ctx->device);
  const size_t n = (size_t)ctx->d.n;
  if (bytes < n * 64) return SPH_ERR_INVALID;
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<float4> a(4 * n);
  std::vector<unsigned> ids(n);
  CK(cudaMemcpy(a.data(), dem->acc, n * 64, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ids.data(), ctx->d.s().id, n * 4, cudaMemcpyDeviceToHost));
  for (size_t t = 0; t < n; ++t) std::memcpy(out16 + 16 * (size_t)ids[t], &a[4 * t], 64);
  return SPH_OK;
}

}  // extern "C"
