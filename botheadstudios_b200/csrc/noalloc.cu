// Tree gravity of a point set that allocates no memory.
//
// Some callers cannot allocate device memory when they need a force evaluation: a real-time frame loop where
// cudaMalloc/cudaFree would synchronise the whole device and stall the frame, or a host engine whose device
// memory is reserved up front by its own allocator and hands plug-ins only the buffers it owns. For them,
// sph_gravity_tree_noalloc runs the same LBVH pipeline as the context path (bbox, Morton keys, radix sort,
// Karras, moments, group-MAC walk) with every scratch buffer carved out of one fixed array in device
// memory, compiled into the library. The caller passes device pointers for the input points and the output
// accelerations. The array holds at most kNoAllocMaxPoints points; every GPU that loads the library keeps it
// for the life of the process.
#include <cuda.h>  // driver-API types only (CUcontext, CUresult); the functions come from the runtime's lookup

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/sph_b200.h"
#include "sph_kernels.cuh"

namespace sphb {
namespace {

constexpr uint32_t kNoAllocMaxPoints = 65536;
constexpr uint32_t kNoAllocMinLeaf = 8;  // bounds the node arrays: at most kNoAllocMaxPoints / 8 leaves
constexpr size_t kAlign = 256;

constexpr size_t up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Byte size of every buffer of the pipeline for kNoAllocMaxPoints points and leaves of >= kNoAllocMinLeaf.
constexpr size_t scratch_bytes() {
  const size_t n = kNoAllocMaxPoints;
  const size_t L = n / kNoAllocMinLeaf;
  const size_t nodes = 2 * L;
  const size_t tiles = (n + 2047) / 2048;
  size_t b = 0;
  b += 2 * (up(16 * n) + up(16 * n) + 3 * up(8 * n) + 5 * up(4 * n));  // two particle states
  b += 2 * up(8 * n) + 2 * up(4 * n);                                  // sort keys and values
  b += up(16 * n) + up(16 * n);                                        // bodies, accelerations
  b += up(4 * 256 * tiles) + up(4 * 256);                              // radix histograms
  b += up(8 * L) + 3 * up(4 * L) + up(8 * L) + up(4);                  // leaf codes, left/right/counters, groups
  b += up(4 * (L + 1)) + up(2 * sizeof(Seg));                          // leaf starts, segment table
  b += up(4 * nodes) + 5 * up(16 * nodes);                             // parents, node records
  b += 2 * up(16 * L) + 2 * up(8 * L);                                 // half-leaf moments (leaves of >= 16)
  b += up(sizeof(DevParams));
  return b;
}
constexpr size_t kScratchBytes = scratch_bytes();

// The scratch array. In host code `g_noalloc_scratch` names a host-side stand-in, not device memory: its
// device address comes from cudaGetSymbolAddress, looked up once per device context.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The address is cached per device together with the unique id of the context it was looked up in. A
// cudaDeviceReset (or another context on the same device) loads the module again at another address; its
// context id differs, so the next call looks the address up again instead of using a stale one. The cache is
// read and written under a mutex: several host threads may make their first call at the same time.
constexpr int kMaxDevices = 64;
struct ScratchSlot {
  unsigned long long ctx_id = 0;  // 0: no lookup yet (driver context ids start at 1)
  void* addr = nullptr;
};
ScratchSlot g_scratch[kMaxDevices];
std::mutex g_scratch_mu;

using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);
struct CtxFns {
  PfnCtxGetCurrent get_current = nullptr;
  PfnCtxGetId get_id = nullptr;
};
// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry-point lookup (no link against libcuda).
const CtxFns& ctx_fns() {
  static const CtxFns fns = [] {
    CtxFns f;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      f.get_current = reinterpret_cast<PfnCtxGetCurrent>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      f.get_id = reinterpret_cast<PfnCtxGetId>(p);
    return f;
  }();
  return fns;
}

// Id of the calling thread's current context, 0 when there is none (or the driver cannot say).
unsigned long long current_ctx_id() {
  const CtxFns& f = ctx_fns();
  if (!f.get_current || !f.get_id) return 0;
  CUcontext c = nullptr;
  if (f.get_current(&c) != CUDA_SUCCESS || !c) return 0;
  unsigned long long id = 0;
  return f.get_id(c, &id) == CUDA_SUCCESS ? id : 0;
}

// Device address of the scratch array for the current device and context. The lookup runs with the device
// current, on the first call in each context; during a stream capture no lookup is made (the capture must
// come after a first call in the same context). Returns nullptr with *status set on failure.
void* scratch_address(int dev, cudaStream_t s, sph_status* status) {
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    *status = SPH_ERR_CUDA;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  ScratchSlot& slot = g_scratch[dev];
  unsigned long long id = current_ctx_id();
  if (slot.addr && id != 0 && slot.ctx_id == id) return slot.addr;
  if (cap != cudaStreamCaptureStatusNone) {
    *status = SPH_ERR_STATE;  // first call in this context inside a capture: nothing may be looked up here
    return nullptr;
  }
  void* ptr = nullptr;
  if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) {
    *status = SPH_ERR_CUDA;
    return nullptr;
  }
  if (id == 0) id = current_ctx_id();  // the lookup made the device's primary context current
  if (id == 0) {
    // without a context id a cached address could go stale unseen: use the fresh lookup, cache nothing
    slot = ScratchSlot{};
    return ptr;
  }
  slot.ctx_id = id;
  slot.addr = ptr;
  return ptr;
}

template <typename T>
T* carve(unsigned char*& p, size_t count) {
  T* r = reinterpret_cast<T*>(p);
  p += up(sizeof(T) * count);
  return r;
}

Dev carve_dev(unsigned char* base, uint32_t K) {
  const size_t n = kNoAllocMaxPoints;
  const size_t L = n / kNoAllocMinLeaf;
  const size_t nodes = 2 * L;
  unsigned char* p = base;
  Dev d;
  d.cap = (int)n;
  d.K = (int)K;
  for (int b = 0; b < 2; ++b) {
    State& s = d.st[b];
    s.pos_h = carve<float4>(p, n);
    s.vel_u = carve<float4>(p, n);
    s.x = carve<double>(p, n);
    s.y = carve<double>(p, n);
    s.z = carve<double>(p, n);
    s.mass = carve<float>(p, n);
    s.mat = carve<unsigned>(p, n);
    s.prov = carve<unsigned>(p, n);
    s.id = carve<unsigned>(p, n);
    s.seg = carve<unsigned>(p, n);
  }
  d.keys[0] = carve<unsigned long long>(p, n);
  d.keys[1] = carve<unsigned long long>(p, n);
  d.vals[0] = carve<unsigned>(p, n);
  d.vals[1] = carve<unsigned>(p, n);
  d.body = carve<float4>(p, n);
  d.grav = carve<float4>(p, n);
  d.rs_tiles_cap = (int)((n + 2047) / 2048);
  d.rs_hist = carve<unsigned>(p, 256 * (size_t)d.rs_tiles_cap);
  d.rs_tot = carve<unsigned>(p, 256);
  d.leaf_codes = carve<unsigned long long>(p, L);
  d.left = carve<unsigned>(p, L);
  d.right = carve<unsigned>(p, L);
  d.counters = carve<unsigned>(p, L);
  d.groups = carve<uint2>(p, L);
  d.ngroups = carve<unsigned>(p, 1);
  d.leaf_start = carve<unsigned>(p, L + 1);
  d.segs = carve<Seg>(p, 2);
  d.parent = carve<unsigned>(p, nodes);
  d.ncom = carve<float4>(p, nodes);
  d.nbmin = carve<float4>(p, nodes);
  d.nbmax = carve<float4>(p, nodes);
  d.nq0 = carve<float4>(p, nodes);
  d.nq1 = carve<float4>(p, nodes);
  // half leaves exist for leaves of >= 16 points, so 2 · (n / 16) entries, which the n / 8 of L covers
  d.hcom = carve<float4>(p, L);
  d.hq0 = carve<float4>(p, L);
  d.hq1 = carve<float2>(p, L);
  d.hrc = carve<float2>(p, L);
  d.P = carve<DevParams>(p, 1);
  return d;
}

// Everything the walk reads from DevParams, written on the device (no host copy), counters cleared.
__global__ void k_noalloc_params(DevParams* P, float G, float theta) {
  DevParams p;
  memset(&p, 0, sizeof(p));
  p.G = G;
  p.theta = theta;
  *P = p;
}

__global__ void k_noalloc_load(const float4* __restrict__ in, int n, State st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 b = in[i];
  st.pos_h[i] = make_float4(b.x, b.y, b.z, 0.0f);
  st.vel_u[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  st.x[i] = (double)b.x;
  st.y[i] = (double)b.y;
  st.z[i] = (double)b.z;
  st.mass[i] = b.w;
  st.mat[i] = 0u;
  st.prov[i] = 0u;
  st.id[i] = (unsigned)i;
  st.seg[i] = 0u;
}

// The results in input order. If the walk's traversal stack overflowed (it then skips subtrees), every
// output is NaN: the caller has no context whose flags it could read, so the result itself says it is invalid.
__global__ void k_noalloc_store(int n, const unsigned* __restrict__ id, const float4* __restrict__ grav,
                                const DevParams* __restrict__ P, float4* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float nan = __int_as_float(0x7fc00000);
  out[id[t]] = (P->flags & kFlagStackOverflow) ? make_float4(nan, nan, nan, nan) : grav[t];
}

}  // namespace
}  // namespace sphb

using namespace sphb;

extern "C" sph_status sph_gravity_tree_noalloc(const void* d_bodies4, uint32_t n, double G, float softening,
                                               float theta, uint32_t leaf_size, uint32_t multipole, void* d_acc4,
                                               void* stream) {
  if (!d_bodies4 || !d_acc4 || n == 0 || !(theta > 0.0f) || !(softening >= 0.0f) || multipole > 1) {
    return SPH_ERR_INVALID;
  }
  // the kernels read and write whole float4 records
  if (((uintptr_t)d_bodies4 | (uintptr_t)d_acc4) & 15u) return SPH_ERR_INVALID;
  if (n > kNoAllocMaxPoints) return SPH_ERR_INVALID;  // beyond the fixed scratch array
  if (leaf_size < kNoAllocMinLeaf || leaf_size > 32 || (leaf_size & (leaf_size - 1)) != 0) return SPH_ERR_INVALID;
  // an error left pending by the caller's own earlier work is not this call's to report or to clear
  if (cudaPeekAtLastError() != cudaSuccess) return SPH_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SPH_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Set-up, once per device context with that device current: the device address of the scratch array.
  sph_status st = SPH_OK;
  void* base = scratch_address(dev, s, &st);
  if (!base) return st;
  Dev d = carve_dev(static_cast<unsigned char*>(base), leaf_size);
  d.n = (int)n;
  d.cur = 0;
  d.L = (int)((n + leaf_size - 1) / leaf_size);
  Cfg c;
  c.quad = (int)multipole;
  c.mac = SPH_MAC_GROUP;
  c.local_theta = kLocalThetaDefault;  // the walk sph_gravity runs with the default configuration
  k_noalloc_params<<<1, 1, 0, s>>>(d.P, (float)G, theta);
  k_noalloc_load<<<(n + 255) / 256, 256, 0, s>>>(static_cast<const float4*>(d_bodies4), (int)n, d.st[0]);
  launch_segments_single(d, softening * softening, 0.0, s);
  launch_bbox(d, s);
  launch_sort_permute(d, s);
  launch_tree(d, c, theta, s);
  launch_gravity_group(d, c, s);
  k_noalloc_store<<<(n + 255) / 256, 256, 0, s>>>((int)n, d.s().id, d.grav, d.P, static_cast<float4*>(d_acc4));
  // no error was pending on entry, so one pending now comes from these launches: report it (and clear it)
  return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}
