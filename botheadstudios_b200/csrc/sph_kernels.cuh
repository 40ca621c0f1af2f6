// Internal device layout and host-side launchers of the SPH step kernels (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>

#include "sph_common.cuh"

namespace sphb {

// Raises a kernel's dynamic shared-memory limit on the calling thread's current device, once per device: the
// attribute belongs to the device, so contexts on several GPUs in one process each need it. `done` holds one
// bit per device ordinal (below 64); two threads racing here both set the same value, which is harmless.
template <typename Kernel>
inline void smem_limit_per_device(Kernel kernel, int bytes, std::atomic<unsigned long long>& done) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess)
    done.fetch_or(bit, std::memory_order_release);
}

// Particle state, structure-of-arrays, kept in Morton (LBVH leaf) order between force evaluations.
// `id` is the particle's original index (its slot in the 48-byte exchange array).
struct State {
  float4* pos_h = nullptr;  // x, y, z (f32 copy of the f64 master), h
  float4* vel_u = nullptr;  // vx, vy, vz, u
  double* x = nullptr;      // f64 master positions
  double* y = nullptr;
  double* z = nullptr;
  float* mass = nullptr;
  unsigned* mat = nullptr;
  unsigned* prov = nullptr;
  unsigned* id = nullptr;
  unsigned* seg = nullptr;  // impact (segment) of the particle in a batch; 0 for a single impact
};

// A batch holds up to kMaxSegments independent impacts ("segments"). Sorted particles of segment k are
// [segs[k].off, segs[k+1].off) and its leaves [segs[k].loff, segs[k+1].loff): a leaf holds <= K particles and
// never crosses a segment boundary, so each segment is one subtree of the LBVH (its root in segs[k].root).
// Entry nseg closes the ranges (off = n, loff = L). One impact is the batch of one segment.
constexpr int kMaxSegments = 256;  // 8 sort-key bits above the 30-bit Morton code
struct Seg {
  unsigned off, loff;   // first sorted particle, first leaf
  unsigned root;        // LBVH node spanning exactly this segment (rebuilt with the tree)
  unsigned sig_bits;    // atomicMin target: bits of the segment's minimum Courant signal
  unsigned bbox[6];     // order-preserving keys of lo.xyz, hi.xyz (bh_gravity.wgsl:49-57)
  float soft2;          // softening² of this impact
  unsigned pad;         // first walk group of the impact
  unsigned res_bits;    // atomicMax target: the impact's smoothing-length residual maximum (float bits)
  float skin;           // neighbour-list skin of the impact's next rebuild (smoothing-length solve)
  double dt;            // dt of the current step
  double time;          // simulated time
};
static_assert(sizeof(Seg) == 72, "Seg is one 72-byte record");
constexpr unsigned kNoSeg = 0xffffffffu;

// Reduce per-thread boxes (order-preserving keys, identity values when the thread holds no point) into the
// segment table. Particles are contiguous per segment, so almost every block lies in one segment and commits
// with one atomic per axis; a block that straddles segments commits per warp (warps inside one segment) or
// per thread. `sg` is the thread's segment, kNoSeg when it holds no point. All threads of the block call it.
__device__ __forceinline__ void seg_bbox_commit(unsigned lo[3], unsigned hi[3], unsigned sg, Seg* segs) {
  __shared__ unsigned s_lo[3][32], s_hi[3][32], s_sg[2][32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const unsigned wmin = warp_min(sg), wmax = warp_max(sg == kNoSeg ? 0u : sg);
  if (lane == 0) {
    s_sg[0][w] = wmin;
    s_sg[1][w] = wmax;
  }
  __syncthreads();
  unsigned bmin = kNoSeg, bmax = 0u;
  for (int k = 0; k < nw; ++k) {
    bmin = min(bmin, s_sg[0][k]);
    bmax = max(bmax, s_sg[1][k]);
  }
  if (bmin == kNoSeg) return;  // block-uniform: no point in this block
  if (bmin == bmax) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = warp_min(lo[k]);
      hi[k] = warp_max(hi[k]);
      if (lane == 0) { s_lo[k][w] = lo[k]; s_hi[k][w] = hi[k]; }
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        unsigned a = lane < nw ? s_lo[k][lane] : 0xffffffffu;
        unsigned b = lane < nw ? s_hi[k][lane] : 0u;
        a = warp_min(a);
        b = warp_max(b);
        if (lane == 0) {
          atomicMin(&segs[bmin].bbox[k], a);
          atomicMax(&segs[bmin].bbox[3 + k], b);
        }
      }
    }
    return;
  }
  if (wmin == kNoSeg) return;
  if (wmin == wmax) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const unsigned a = warp_min(lo[k]), b = warp_max(hi[k]);
      if (lane == 0) {
        atomicMin(&segs[wmin].bbox[k], a);
        atomicMax(&segs[wmin].bbox[3 + k], b);
      }
    }
  } else if (sg != kNoSeg) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      atomicMin(&segs[sg].bbox[k], lo[k]);
      atomicMax(&segs[sg].bbox[3 + k], hi[k]);
    }
  }
}

// Maximum of non-negative per-thread values into each thread's segment (res_bits): one atomic per warp when
// the warp lies in one segment. `sg` = kNoSeg for a thread without a value. All lanes of the warp call it.
__device__ __forceinline__ void seg_res_max(Seg* segs, unsigned sg, float v) {
  const unsigned lo = warp_min(sg), hi = warp_max(sg == kNoSeg ? 0u : sg);
  if (lo == kNoSeg) return;
  if (lo == hi) {
    const float m = warp_max(sg == kNoSeg ? 0.0f : v);
    if ((threadIdx.x & 31) == 0) atomicMax(&segs[lo].res_bits, __float_as_uint(m));
  } else if (sg != kNoSeg) {
    atomicMax(&segs[sg].res_bits, __float_as_uint(v));
  }
}

struct Dev {
  int n = 0, cap = 0;
  unsigned sent = 0;  // index of the sentinel record (the gather kernels' list filler), past the capacity
  int K = 1;        // leaf size
  int L = 0;        // number of leaves
  State st[2];
  int cur = 0;
  float4* body = nullptr;  // x, y, z, m in sorted order (gravity sources)
  unsigned long long* keys[2] = {nullptr, nullptr};
  unsigned* vals[2] = {nullptr, nullptr};
  unsigned* rs_hist = nullptr;  // [256][tiles]
  unsigned* rs_tot = nullptr;   // [256]
  int rs_tiles_cap = 0;
  int nseg = 1;
  int segbits = 0;                 // sort-key bits of the segment index (0 for one segment)
  Seg* segs = nullptr;             // [kMaxSegments + 1]
  unsigned* leaf_start = nullptr;  // [L+1] first sorted particle of each leaf
  unsigned long long* leaf_codes = nullptr;  // segment << 30 | Morton code of each leaf's first particle
  unsigned* left = nullptr;     // [L-1]
  unsigned* right = nullptr;    // [L-1]
  unsigned* parent = nullptr;   // [2L-1]
  unsigned* counters = nullptr; // [L-1] climb arrival counters
  float4* ncom = nullptr;       // [2L-1] com.xyz, mass
  float4* nbmin = nullptr;      // [2L-1] bmin.xyz, max h
  float4* nbmax = nullptr;      // [2L-1] bmax.xyz, opening radius
  float4* nq0 = nullptr;        // [2L-1] Qxx, Qyy, Qzz, Qxy
  float4* nq1 = nullptr;        // [2L-1] Qxz, Qyz, 0, 0
  // Half-leaf moments (group walk, leaves of >= 16 particles): leaf c's particles [s, s + K/2) and [s + K/2, e)
  // as two multipoles, entries 2c and 2c + 1, for far leaves the walk splits
  float4* hcom = nullptr;       // [2L] com.xyz, mass
  float4* hq0 = nullptr;        // [2L] Qxx, Qyy, Qzz, Qxy
  float2* hq1 = nullptr;        // [2L] Qxz, Qyz
  float2* hrc = nullptr;        // [L] opening radii of the two halves (size/θ + |centre − COM|)
  uint2* groups = nullptr;      // [L] walk groups: (first leaf, last leaf) of runs of 32/K leaves of one impact
  unsigned* ngroups = nullptr;  // [1] number of groups
  unsigned* nbr = nullptr;      // interleaved neighbour lists [n/32][nbr_cap][32]
  unsigned* nbr_cnt = nullptr;  // [n]
  unsigned nbr_cap = 0;
  float* rho = nullptr;         // [n]
  float4* fdata = nullptr;      // [n] mass, rho, P/rho², c
  float4* grav = nullptr;       // [n] gravity acc.xyz, potential
  float4* acc = nullptr;        // [n] total acc.xyz, du/dt
  float* hnew = nullptr;        // [n] smoothing-length solve scratch
  float* h0 = nullptr;          // [n] smoothing length when the neighbour list was built
  float* divv = nullptr;        // [n] velocity divergence from the force pass (a learned-h input)
  unsigned* pend[2] = {nullptr, nullptr};  // learned h: particles still iterating (two alternating lists)
  unsigned* pend_n = nullptr;   // [2] list lengths
  Eos* eos = nullptr;           // [16]
  DevParams* P = nullptr;
  double* diag_part = nullptr;  // [blocks][16]
  int diag_blocks = 0;
  void* aos = nullptr;          // [cap] 48-byte exchange buffer (original order)
  const State& s() const { return st[cur]; }
};

// The group walk's local-expansion opening parameter (r_group / distance) that sph_config_default sets.
// Measured on the 1M impact (θ = 0.6, quadrupoles): 0.3 cuts the walk 12 % and moves the gravity error against
// FP64 direct sums from 3.8e-4 to 4.8e-4 RMS.
constexpr float kLocalThetaDefault = 0.3f;

struct Cfg {
  int kernel = 0;       // 0 cubic, 1 Wendland C2
  int gravity = 0;      // 0 tree, 1 direct, 2 none
  int quad = 0;         // quadrupole moments
  int hilo = 0;         // node-relative hi/lo + compensated sums
  int h_solve = 0;
  float h_eta = 0.0f;   // h = h_eta (m/ρ)^(1/3)
  float h_tol = 1.0e-3f;
  int h_iters = 4;
  float skin = 0.0f;    // neighbour-list radius inflation (h-solve)
  int mac = 0;          // 0 group walk, 1 per-particle reference walk
  float nbr_skin = 0.0f;  // list inflation without the h-solve (grain contacts: a superset, cut exactly later)
  int blk = 256;        // threads per block of the per-particle gather kernels (density, h-solve, forces)
  int walk_warps = 2;   // warps per block of the fused walk (2, 4 or 8)
  int learned = 0;      // smoothing lengths proposed by the MLP, checked, iterated only where rejected
  int divv = 0;         // the force pass also writes ∇·v (the learned proposal or its recording needs it)
  int walk_stack = 0;   // traversal-stack limit of the walks (0: their full stacks); for testing the overflow path
  float local_theta = 0.0f;  // group walk: accepted nodes beyond r_group/local_theta join the local expansion
};

// Grain contact constants (the reference's GpuStepParams subset used by the contact law and solve).
struct DemParams {
  float gx, gy, gz, dt;
  float stiffness, normal_damp, friction, tangent_damp, cohesion;
  // the ground scene (particle_step.wgsl Params): heightfield frame, medium, thermal relaxation
  float cx, cy, cz;
  float air_rho, drag_cd, specific_heat, cool_rate;
  const int* hf = nullptr;  // [wd][ww] column tops (voxel units), nullptr without a terrain
  unsigned ww = 0, wd = 0;
};
int launch_dem_load(const Dev& d, const void* grains, cudaStream_t s);
int launch_dem_store(const Dev& d, const DemParams& p, bool stepped, void* grains, cudaStream_t s);
int launch_dem_contacts(const Dev& d, const DemParams& p, float4* acc, cudaStream_t s);
int launch_dem_integrate(const Dev& d, const DemParams& p, const float4* acc, cudaStream_t s);

// ---- segments and tree -----------------------------------------------------------------------------
int launch_segments(const Dev& d, cudaStream_t s);        // leaf_start from the segment table
int launch_segments_single(const Dev& d, float soft2, double dt, cudaStream_t s);  // one segment, on the device
int launch_bbox(const Dev& d, cudaStream_t s);
int launch_sort_permute(Dev& d, cudaStream_t s);      // keys → radix sort → permute (swaps d.cur)
int launch_tree(const Dev& d, const Cfg& c, float theta, cudaStream_t s);  // Karras + moments
// particles per half leaf the group walk splits far leaves into (0: leaves are not split)
int half_leaf(const Dev& d, const Cfg& c);
size_t radix_tiles(int n);
// stable LSD radix sort of (keys, vals) on the low `bits` key bits; the result lands in buffer `src`
int launch_radix_sort(unsigned long long* keys[2], unsigned* vals[2], int n, int bits, unsigned* hist,
                      unsigned* tot, int& src, cudaStream_t s);

// ---- gravity ---------------------------------------------------------------------------------------
int launch_gravity_tree(const Dev& d, const Cfg& c, cudaStream_t s);
int launch_gravity_direct(const Dev& d, cudaStream_t s);
int launch_gravity_direct64(const double* pos3, const double* mass, int n, const unsigned* targets, int nt,
                             double soft2, double G, double* acc3, cudaStream_t s);

// ---- SPH -------------------------------------------------------------------------------------------
int launch_neighbours(const Dev& d, const Cfg& c, cudaStream_t s);      // neighbour lists only
// group-MAC gravity + neighbour lists; potential: also the potential φ (the steps' walks leave it out)
int launch_walk(const Dev& d, const Cfg& c, bool potential, cudaStream_t s);
int launch_potential(const Dev& d, const Cfg& c, cudaStream_t s);      // φ alone on the current tree
int launch_gravity_group(const Dev& d, const Cfg& c, cudaStream_t s);   // group-MAC gravity only
int launch_density_eos(const Dev& d, const Cfg& c, cudaStream_t s);
int launch_h_solve(const Dev& d, const Cfg& c, cudaStream_t s);
int launch_h_learned(const Dev& d, const Cfg& c, cudaStream_t s);   // check proposals, iterate the rejected
int launch_eos_only(const Dev& d, cudaStream_t s);
int launch_forces(const Dev& d, const Cfg& c, cudaStream_t s);
int launch_finalize_dt(const Dev& d, cudaStream_t s);
int launch_kick_drift(const Dev& d, cudaStream_t s);
int launch_kick(const Dev& d, cudaStream_t s);
int launch_relax(const Dev& d, cudaStream_t s);
int launch_from_aos(const Dev& d, cudaStream_t s);
int launch_to_aos(const Dev& d, cudaStream_t s);
// first invalid record of the n 48-byte particles in d.aos into *first_bad (left at 0xffffffff when all pass)
int launch_validate_aos(const Dev& d, int n, unsigned ne, unsigned* first_bad, cudaStream_t s);
int launch_diag(const Dev& d, cudaStream_t s, double* out16);

// ---- disk measurement and the Moon candidate (disk.cu) ------------------------------------------------
struct DiskCfg {
  int variant;          // 0: the impact-run tool's measure, 1: the engine's disk statistics
  double G, remnant_frac, link_factor, roche, rho_fallback, pe_floor, pe_soft;
};
struct DiskWork;        // device workspace, grown on demand
void disk_work_free(DiskWork* w);
// Measures the sorted particles [off, off + m) of the current state into out[16] (host memory; the call
// synchronises the stream). Returns 0, or a negative status with a message in *err. *launches counts kernels.
int disk_measure(const Dev& d, unsigned off, unsigned m, const DiskCfg& c, DiskWork*& w, double* out,
                 unsigned long long* launches, const char** err, cudaStream_t s);
// body_bulk (gpu_sph.rs:260-293) of the state's particles with provenance `prov`: out5 = centre xyz, mass,
// 98 %-mass radius (host memory; synchronises the stream).
int body_bulk(const Dev& d, unsigned prov, DiskWork*& w, double* out5, unsigned long long* launches,
              const char** err, cudaStream_t s);
// assemble_from_relaxed_n (gpu_sph.rs:309-339): placements = np × {offset xyz, vel xyz, spin xyz} (host);
// writes the kept particles, transformed, in original order into dst (device, room for d.n records) and returns
// their count and smallest h. Overwrites d.aos.
int assemble_n(const Dev& d, const double* placements, unsigned np, void* dst, unsigned* n_out, float* min_h,
               DiskWork*& w, unsigned long long* launches, const char** err, cudaStream_t s);

}  // namespace sphb
