// Learned smoothing-length MLP on the tensor cores: 8 → 64 → 64 → 1 with GELU, BF16 operands and FP32
// accumulation. Inference (the in-step proposal and the standalone forward) and training both run on tcgen05:
// M = 128 × N = 64 tcgen05.mma tiles issued by one thread, operands in shared memory in the canonical
// no-swizzle K-major layout, accumulators in tensor memory (see the inference and training sections). Training
// computes the weight gradients as tcgen05 GEMMs over a tile's 128 samples; Adam updates an FP32 master copy.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/sph_b200.h"
#include "mlp.cuh"

namespace sphb {

namespace {

constexpr int ROWS = 128;
// Largest proposed change of log h: an outlier proposal stays within reach of the fallback's Newton steps
// (±20 % each, inside the list skin around the proposal).
constexpr float kMaxStep = 0.03f;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * expf(-0.5f * z * z) * 0.39894228040143268f;
}

// ---- feature definition (the solver's state at the start of the step's drift) ---------------------------
__device__ __forceinline__ void features(int t, const State& st, const float* __restrict__ rho,
                                         const unsigned* __restrict__ cnt, const float4* __restrict__ acc,
                                         const float4* __restrict__ fdata, const float* __restrict__ divv,
                                         const Eos* __restrict__ eos, const Seg* __restrict__ segs,
                                         const DevParams* __restrict__ P, const MlpFeatureArgs& fa,
                                         float f[MLP_IN]) {
  const float4 p = st.pos_h[t];
  const float m = st.mass[t];
  const float r = fmaxf(rho[t], 1.0e-30f);
  const unsigned mat = st.mat[t];
  const float rho0 = eos[mat].rho0, e_iv = eos[mat].e_iv;
  const float heq = fa.eta * cbrtf(m / r);
  const float dt = (float)segs[st.seg[t]].dt;
  const float4 a = acc[t];
  const float c = fmaxf(fdata[t].w, P->sig_floor);  // the Courant signal's floor keeps c² > 0
  f[0] = logf(p.w / heq);                                                      // log h relative to h(rho)
  f[1] = logf(r / rho0);                                                       // log rho / rho0
  f[2] = divv[t] * dt;                                                         // div v over the step
  f[3] = (float)cnt[t] / fa.n_target;                                          // neighbours / target
  f[4] = log1pf(sqrtf(a.x * a.x + a.y * a.y + a.z * a.z) * p.w / (c * c));     // |a| h / c²
  f[5] = (float)mat;                                                           // material
  f[6] = log1pf(fmaxf(st.vel_u[t].w, 0.0f) / e_iv);                            // u / E_iv
  f[7] = P->progress;                                                          // step fraction
}

// ---- inference on the 5th-generation tensor cores (tcgen05) ---------------------------------------------
// A CTA of 128 threads holds 128 rows. Each thread writes its row of x' (layer 1) or of a1 (layer 2) into
// shared memory in the canonical no-swizzle K-major layout (8-row × 16-byte core matrices; core matrices
// adjacent along K are 128 B apart, 8-row groups K·16 B apart); one thread issues tcgen05.mma (BF16 × BF16 →
// FP32, M = 128, N = 64, K = 16 per instruction) with the weights as the K-major B operand, and commits to an
// mbarrier. The accumulators live in tensor memory: row r of D is TMEM lane r, so after the barrier every
// thread reads its own row (tcgen05.ld 32x32b) and applies bias, GELU and the next layer's input rounding,
// and the 64 → 1 output layer is a per-thread dot product. Every barrier wait is bounded: on a timeout the
// CTA stops issuing, raises an error flag, waits (bounded) for what it issued and frees its tensor memory.
constexpr int TC_COLS = 128;            // TMEM columns per CTA: D1 [0, 64), D2 [64, 128)
constexpr int TC_SMEM = 56 * 1024;      // dynamic shared memory per CTA: at most 4 CTAs (4 × 128 of 512 columns)
constexpr unsigned kTcSpin = 1u << 16;  // barrier polls before giving up
constexpr uint32_t kTcIdesc = (1u << 4)            // D: FP32
                              | (1u << 7)          // A: BF16
                              | (1u << 10)         // B: BF16 (A and B K-major: bits 15, 16 clear)
                              | ((64u >> 3) << 17) // N = 64
                              | ((128u >> 4) << 24);  // M = 128

struct TcSmem {
  __nv_bfloat16 a1[ROWS * 16];      // x' rows (K = 16, inputs 8..15 zero)
  __nv_bfloat16 a2[ROWS * MLP_H];   // a1 rows (K = 64)
  __nv_bfloat16 w1[MLP_H * 16];     // W1ᵀ [out][in] (K = 16)
  __nv_bfloat16 w2[MLP_H * MLP_H];  // W2ᵀ [out][in] (K = 64)
  float b1[MLP_H], b2[MLP_H], w3[MLP_H];
  unsigned long long mbar;
  unsigned tmem;
  int ok;
};
static_assert(sizeof(TcSmem) <= TC_SMEM, "tcgen05 tile fits its shared memory");

// element offset of (row r, k) in a K-major no-swizzle operand with K columns
__device__ __forceinline__ int cm(int r, int k, int K) { return (r >> 3) * (K * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7); }
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// shared-memory matrix descriptor: start, leading (K) and stride (8-row) byte offsets, sm100 version bits, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
               :: "r"(d), "l"(a), "l"(b), "r"(kTcIdesc), "r"(acc) : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(mbar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (unsigned i = 0; i < kTcSpin; ++i) {
    uint32_t done;
    asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}
// 16 consecutive FP32 columns of this warp's 32 TMEM lanes (one per thread)
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ uint4 pack8(const float f[8]) {
  __nv_bfloat162 h[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
  return *reinterpret_cast<uint4*>(h);
}

// CTA set-up: tensor memory, the barrier, the weights in the operand layout.
__device__ void tc_setup(TcSmem& S, const MlpPacked* __restrict__ W) {
  for (int i = threadIdx.x; i < MLP_H * 16; i += ROWS) S.w1[cm(i >> 4, i & 15, 16)] = W->w1t[i];
  for (int i = threadIdx.x; i < MLP_H * MLP_H; i += ROWS) S.w2[cm(i >> 6, i & 63, 64)] = W->w2t[i];
  for (int i = threadIdx.x; i < MLP_H; i += ROWS) {
    S.b1[i] = W->b1[i];
    S.b2[i] = W->b2[i];
    S.w3[i] = W->w3[i];
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&S.mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    S.ok = 1;
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&S.tmem)), "r"(TC_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// One 128-row tile: this thread's normalised inputs in, its y (before b3) out (NaN after a barrier timeout).
__device__ float tc_tile(TcSmem& S, const float xq[MLP_IN], uint32_t& phase) {
  const int r = threadIdx.x, w = r >> 5;
  const uint32_t mbar = smem_u32(&S.mbar);
  const uint32_t trow = S.tmem + ((uint32_t)(w * 32) << 16);
  const float zero8[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  *reinterpret_cast<uint4*>(S.a1 + cm(r, 0, 16)) = pack8(xq);
  *reinterpret_cast<uint4*>(S.a1 + cm(r, 8, 16)) = pack8(zero8);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (!S.ok) return __int_as_float(0x7fc00000);
  if (r == 0) {
    tc_mma(S.tmem, umma_desc(smem_u32(S.a1), 128, 256), umma_desc(smem_u32(S.w1), 128, 256), 0u);
    tc_commit(mbar);
  }
  // on a timeout `phase` keeps the parity of the commit still outstanding, for the tear-down to wait on
  bool got = mbar_wait(mbar, phase);
  if (!__syncthreads_and(got)) {
    if (r == 0) S.ok = 0;
    return __int_as_float(0x7fc00000);
  }
  phase ^= 1u;
  tc_fence_after();
  // layer 1 → GELU → a1 (bf16) row
  float z[64];
#pragma unroll
  for (int c = 0; c < 4; ++c) tc_ld16(trow + 16 * c, z + 16 * c);
  tc_wait_ld();
#pragma unroll
  for (int kb = 0; kb < 8; ++kb) {
    float h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = gelu(z[8 * kb + i] + S.b1[8 * kb + i]);
    *reinterpret_cast<uint4*>(S.a2 + cm(r, 8 * kb, 64)) = pack8(h);
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (r == 0) {
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
      tc_mma(S.tmem + 64, umma_desc(smem_u32(S.a2) + 256 * kt, 128, 1024), umma_desc(smem_u32(S.w2) + 256 * kt, 128, 1024),
             kt > 0 ? 1u : 0u);
    tc_commit(mbar);
  }
  got = mbar_wait(mbar, phase);
  if (!__syncthreads_and(got)) {
    if (r == 0) S.ok = 0;
    return __int_as_float(0x7fc00000);
  }
  phase ^= 1u;
  tc_fence_after();
#pragma unroll
  for (int c = 0; c < 4; ++c) tc_ld16(trow + 64 + 16 * c, z + 16 * c);
  tc_wait_ld();
  float y = 0.0f;
#pragma unroll
  for (int j = 0; j < MLP_H; ++j) y += gelu(z[j] + S.b2[j]) * S.w3[j];
  tc_fence_before();
  return y;
}

// CTA tear-down: after a timeout, wait (bounded) for the last commit; then free the tensor memory.
__device__ bool tc_teardown(TcSmem& S, uint32_t phase) {
  const bool failed = !S.ok;
  if (failed) mbar_wait(smem_u32(&S.mbar), phase);  // what was issued before the timeout, if anything
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(S.tmem), "r"(TC_COLS) : "memory");
  return !failed;
}

__device__ __forceinline__ void normalise(const float f[MLP_IN], const MlpPacked* W, float xq[MLP_IN]) {
#pragma unroll
  for (int k = 0; k < MLP_IN; ++k) xq[k] = (f[k] - W->xm[k]) * W->xs[k];
}

__global__ void __launch_bounds__(ROWS) k_mlp_propose(int n, State st, const float* __restrict__ rho,
                                                     const unsigned* __restrict__ cnt,
                                                     const float4* __restrict__ acc,
                                                     const float4* __restrict__ fdata,
                                                     const float* __restrict__ divv, const Eos* __restrict__ eos,
                                                     const Seg* __restrict__ segs, DevParams* __restrict__ P,
                                                     MlpFeatureArgs fa, const MlpPacked* __restrict__ W,
                                                     float* __restrict__ rec, float* __restrict__ dh, int apply) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(tc_raw);
  tc_setup(S, W);
  const float b3 = W->b3, ym = W->ym, ys = W->ys;
  uint32_t phase = 0;
  const int r = threadIdx.x;
  for (int base = blockIdx.x * ROWS; base < n; base += gridDim.x * ROWS) {
    const int t = base + r;
    float f[MLP_IN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, xq[MLP_IN];
    if (t < n) features(t, st, rho, cnt, acc, fdata, divv, eos, segs, P, fa, f);
    normalise(f, W, xq);
    const float y = tc_tile(S, xq, phase);
    if (t < n) {
      // the network gives log(h_next / h(rho)); the step from the current h subtracts log(h / h(rho)) = f[0],
      // so a residual left by the previous solve is corrected whatever the network learned
      const float d = (y + b3) * ys + ym - f[0];
      const float dc = d == d ? fminf(fmaxf(d, -kMaxStep), kMaxStep) : 0.0f;  // no proposal from a NaN
      if (apply) st.pos_h[t].w = st.pos_h[t].w * expf(dc);
      if (rec) {
        const unsigned id = st.id[t];
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) rec[(size_t)id * MLP_IN + k] = f[k];
        dh[id] = d;
      }
    }
  }
  if (!tc_teardown(S, phase) && threadIdx.x == 0) atomicOr(&P->flags, kFlagTensorTimeout);
}

__global__ void __launch_bounds__(ROWS) k_mlp_forward(const MlpPacked* __restrict__ W, const float* __restrict__ x,
                                                     int n, float* __restrict__ out, unsigned* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(tc_raw);
  tc_setup(S, W);
  uint32_t phase = 0;
  const int r = threadIdx.x;
  for (int base = blockIdx.x * ROWS; base < n; base += gridDim.x * ROWS) {
    const int t = base + r;
    float f[MLP_IN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, xq[MLP_IN];
    if (t < n)
#pragma unroll
      for (int k = 0; k < MLP_IN; ++k) f[k] = x[(size_t)t * MLP_IN + k];
    normalise(f, W, xq);
    const float y = tc_tile(S, xq, phase);
    if (t < n) out[t] = (y + W->b3) * W->ys + W->ym;
  }
  if (!tc_teardown(S, phase) && threadIdx.x == 0) atomicOr(err, 1u);
}

// ---- training on tcgen05: forward + backward of one 128-sample tile ----------------------------------------
// The same tiles as inference (M = 128 × N = 64, BF16 × BF16 → FP32 in tensor memory, one issuing thread,
// bounded mbarrier waits), five MMA groups per tile: the two forward layers (D1 = x'·W1ᵀ, D2 = a1·W2ᵀ), then
// da1 = dz2·W2 (D3) together with dW2 = a1ᵀ·dz2 (D4), then dW1 = x'ᵀ·dz1 (D5, in D1's columns). The weight
// gradients contract over the tile's 128 samples (K = 128); their M (64 inputs of layer 2, 16 padded inputs of
// layer 1) is padded to the instruction's 128 rows, whose extra rows are read from the operand buffer's unused
// rows and never used. Thread r owns sample r: it writes its rows of every A/B operand (the transposed ones
// column r), reads its row of each accumulator, and the bias and W3 gradients are column sums in shared memory.
constexpr int TT_COLS = 256;  // TMEM columns: D1 [0, 64) (then D5), D2 [64, 128), D3 [128, 192), D4 [192, 256)

struct TrainTcSmem {
  __nv_bfloat16 xa[ROWS * 16];       // x' [row][k], K = 16 (A of layer 1)
  __nv_bfloat16 ha[ROWS * MLP_H];    // a1 [row][i], K = 64 (A of layer 2)
  __nv_bfloat16 w1[MLP_H * 16];      // W1ᵀ [out][k] (B of layer 1)
  __nv_bfloat16 w2t[MLP_H * MLP_H];  // W2ᵀ [out][i] (B of layer 2)
  __nv_bfloat16 w2b[MLP_H * MLP_H];  // W2 [i][out] (B of da1 = dz2 W2: N = i, K = out)
  __nv_bfloat16 dza[ROWS * MLP_H];   // dz2 [row][out], K = 64 (A of da1)
  __nv_bfloat16 gta[ROWS * ROWS];    // a1ᵀ [i][row] then x'ᵀ [k][row], K = 128 (A of the weight gradients)
  __nv_bfloat16 gtb[MLP_H * ROWS];   // dz2ᵀ [out][row] then dz1ᵀ [i][row], K = 128 (B of the weight gradients)
  float z1[ROWS * MLP_H];            // z1, then dz1 (FP32)
  float z2[ROWS * MLP_H];            // z2 (FP32)
  float dy[ROWS];
  unsigned long long mbar;
  unsigned tmem;
  int ok;
};

// Issue (thread 0) the MMAs of `fn`, commit to the barrier, wait (bounded) for them; false on a timeout.
template <typename F>
__device__ bool tt_run(TrainTcSmem& S, uint32_t& phase, F fn) {
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (!S.ok) return false;
  const uint32_t mbar = smem_u32(&S.mbar);
  if (threadIdx.x == 0) {
    fn();
    tc_commit(mbar);
  }
  const bool got = mbar_wait(mbar, phase);
  if (!__syncthreads_and(got)) {
    if (threadIdx.x == 0) S.ok = 0;
    return false;
  }
  phase ^= 1u;
  tc_fence_after();
  return true;
}

// 64 FP32 accumulator columns of this thread's row (TMEM lane = row).
__device__ __forceinline__ void tt_row(const TrainTcSmem& S, uint32_t col, float v[64]) {
  const uint32_t t = S.tmem + ((uint32_t)((threadIdx.x >> 5) * 32) << 16) + col;
#pragma unroll
  for (int c = 0; c < 4; ++c) tc_ld16(t + 16 * c, v + 16 * c);
  tc_wait_ld();
}

__global__ void __launch_bounds__(ROWS) k_mlp_train_tc(const MlpPacked* __restrict__ W, const float* __restrict__ x,
                                                      const float* __restrict__ tgt, const unsigned* __restrict__ idx,
                                                      int m, float denom, float* __restrict__ grad,
                                                      float* __restrict__ loss, unsigned* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tt_raw[];
  TrainTcSmem& S = *reinterpret_cast<TrainTcSmem*>(tt_raw);
  const int r = threadIdx.x, lane = r & 31;
  // weights in the K-major operand layout
  for (int i = r; i < MLP_H * 16; i += ROWS) S.w1[cm(i >> 4, i & 15, 16)] = W->w1t[i];
  for (int i = r; i < MLP_H * MLP_H; i += ROWS) {
    S.w2t[cm(i >> 6, i & 63, 64)] = W->w2t[i];  // [out][in]: row out, K = in
    S.w2b[cm(i >> 6, i & 63, 64)] = W->w2[i];   // [in][out]: row in, K = out
  }
  if (r == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&S.mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    S.ok = 1;
  }
  if (r < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&S.tmem)), "r"(TT_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // this thread's sample: normalised inputs (rows past m carry dy = 0 and add nothing)
  const int s = blockIdx.x * ROWS + r;
  const bool valid = s < m;
  float f[MLP_IN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, xq[MLP_IN];
  float tn = 0.0f;
  if (valid) {
    const unsigned j = idx[s];
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) f[k] = x[(size_t)j * MLP_IN + k];
    tn = (tgt[j] - W->ym) / W->ys;
  }
  normalise(f, W, xq);
  const float zero8[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  *reinterpret_cast<uint4*>(S.xa + cm(r, 0, 16)) = pack8(xq);
  *reinterpret_cast<uint4*>(S.xa + cm(r, 8, 16)) = pack8(zero8);
  uint32_t phase = 0;
  const uint32_t xa = smem_u32(S.xa), ha = smem_u32(S.ha), w1 = smem_u32(S.w1), w2t = smem_u32(S.w2t);
  const uint32_t w2b = smem_u32(S.w2b), dza = smem_u32(S.dza), gta = smem_u32(S.gta), gtb = smem_u32(S.gtb);
  float v[64];
  // ---- layer 1: z1 = x'·W1ᵀ + b1, a1 = GELU(z1) (bf16 rows for layer 2, bf16 columns for dW2) -------------
  if (tt_run(S, phase, [&] { tc_mma(S.tmem, umma_desc(xa, 128, 256), umma_desc(w1, 128, 256), 0u); })) {
    tt_row(S, 0, v);
#pragma unroll
    for (int kb = 0; kb < 8; ++kb) {
      float h[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float z = v[8 * kb + i] + W->b1[8 * kb + i];
        S.z1[r * MLP_H + 8 * kb + i] = z;
        h[i] = gelu(z);
      }
      const uint4 hp = pack8(h);
      *reinterpret_cast<uint4*>(S.ha + cm(r, 8 * kb, 64)) = hp;
      const __nv_bfloat16* hb = reinterpret_cast<const __nv_bfloat16*>(&hp);
#pragma unroll
      for (int i = 0; i < 8; ++i) S.gta[cm(8 * kb + i, r, ROWS)] = hb[i];
    }
  }
  // ---- layer 2 and the output: y = Σ GELU(z2)·w3 + b3, dy, dz2 = dy·w3·GELU'(z2) --------------------------
  if (tt_run(S, phase, [&] {
        for (int kt = 0; kt < 4; ++kt)
          tc_mma(S.tmem + 64, umma_desc(ha + 256 * kt, 128, 1024), umma_desc(w2t + 256 * kt, 128, 1024), kt > 0 ? 1u : 0u);
      })) {
    tt_row(S, 64, v);
    float y = 0.0f;
#pragma unroll
    for (int o = 0; o < MLP_H; ++o) {
      v[o] += W->b2[o];
      S.z2[r * MLP_H + o] = v[o];
      y += gelu(v[o]) * W->w3[o];
    }
    const float e = valid ? (y + W->b3 - tn) : 0.0f;
    const float dy = 2.0f * e / denom;
    S.dy[r] = dy;
    float e2 = e * e;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e2 += __shfl_xor_sync(SPH_FULL_MASK, e2, o);
    if (lane == 0) atomicAdd(loss, e2);
#pragma unroll
    for (int ob = 0; ob < 8; ++ob) {
      float dz[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) dz[i] = dy * W->w3[8 * ob + i] * gelu_d(v[8 * ob + i]);
      const uint4 dp = pack8(dz);
      *reinterpret_cast<uint4*>(S.dza + cm(r, 8 * ob, 64)) = dp;
      const __nv_bfloat16* db = reinterpret_cast<const __nv_bfloat16*>(&dp);
#pragma unroll
      for (int i = 0; i < 8; ++i) S.gtb[cm(8 * ob + i, r, ROWS)] = db[i];
    }
  }
  // ---- da1 = dz2·W2 (D3) and dW2 = a1ᵀ·dz2 (D4, rows 0..63) -------------------------------------------------
  if (tt_run(S, phase, [&] {
        for (int kt = 0; kt < 4; ++kt)
          tc_mma(S.tmem + 128, umma_desc(dza + 256 * kt, 128, 1024), umma_desc(w2b + 256 * kt, 128, 1024),
                 kt > 0 ? 1u : 0u);
        for (int kt = 0; kt < 8; ++kt)
          tc_mma(S.tmem + 192, umma_desc(gta + 256 * kt, 128, 2048), umma_desc(gtb + 256 * kt, 128, 2048),
                 kt > 0 ? 1u : 0u);
      })) {
    if (r < MLP_H) {  // warps 0 and 1: the rows of dW2 (input i = r)
      tt_row(S, 192, v);
#pragma unroll 8
      for (int o = 0; o < MLP_H; ++o) atomicAdd(&grad[MLP_W2 + r * MLP_H + o], v[o]);
    }
    tt_row(S, 128, v);
#pragma unroll
    for (int i = 0; i < MLP_H; ++i) {
      const float dz = v[i] * gelu_d(S.z1[r * MLP_H + i]);
      S.z1[r * MLP_H + i] = dz;
      S.gtb[cm(i, r, ROWS)] = __float2bfloat16_rn(dz);
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) S.gta[cm(k, r, ROWS)] = S.xa[cm(r, k, 16)];
  }
  // ---- dW1 = x'ᵀ·dz1 (D5 in D1's columns, rows k < 8) --------------------------------------------------------
  if (tt_run(S, phase, [&] {
        for (int kt = 0; kt < 8; ++kt)
          tc_mma(S.tmem, umma_desc(gta + 256 * kt, 128, 2048), umma_desc(gtb + 256 * kt, 128, 2048), kt > 0 ? 1u : 0u);
      })) {
    if (r < 32) {
      tt_row(S, 0, v);
      if (r < MLP_IN)
#pragma unroll 8
        for (int i = 0; i < MLP_H; ++i) atomicAdd(&grad[MLP_W1 + r * MLP_H + i], v[i]);
    }
  }
  // ---- the bias and W3 gradients: column sums over the tile ---------------------------------------------------
  __syncthreads();
  if (S.ok) {
    const int col = r & 63, half = r >> 6;
    float gw3 = 0.f, gb2 = 0.f, gb1 = 0.f;
    for (int rr = half * 64; rr < half * 64 + 64; ++rr) {
      const float z = S.z2[rr * MLP_H + col], d = S.dy[rr];
      gw3 += d * gelu(z);
      gb2 += d * W->w3[col] * gelu_d(z);
      gb1 += S.z1[rr * MLP_H + col];
    }
    atomicAdd(&grad[MLP_W3 + col], gw3);
    atomicAdd(&grad[MLP_B2 + col], gb2);
    atomicAdd(&grad[MLP_B1 + col], gb1);
    if (r == 0) {
      float gb3 = 0.f;
      for (int rr = 0; rr < ROWS; ++rr) gb3 += S.dy[rr];
      atomicAdd(&grad[MLP_B3], gb3);
    }
  }
  // ---- tear-down: after a timeout wait (bounded) for what was issued, then free the tensor memory -------------
  const bool failed = !S.ok;
  if (failed) mbar_wait(smem_u32(&S.mbar), phase);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (r < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(S.tmem), "r"(TT_COLS) : "memory");
  if (failed && r == 0) atomicOr(err, 1u);
}

__global__ void k_mlp_pack(const float* __restrict__ P, MlpPacked* __restrict__ o) {
  for (int i = threadIdx.x; i < MLP_H * 16; i += blockDim.x) {
    const int out = i >> 4, in = i & 15;
    o->w1t[i] = __float2bfloat16_rn(in < MLP_IN ? P[MLP_W1 + in * MLP_H + out] : 0.0f);
  }
  for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) {
    const int out = i >> 6, in = i & 63;
    o->w2t[i] = __float2bfloat16_rn(P[MLP_W2 + in * MLP_H + out]);
    o->w2[i] = __float2bfloat16_rn(P[MLP_W2 + i]);
  }
  for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
    o->w3[i] = __bfloat162float(__float2bfloat16_rn(P[MLP_W3 + i]));
    o->b1[i] = P[MLP_B1 + i];
    o->b2[i] = P[MLP_B2 + i];
  }
  if (threadIdx.x < MLP_IN) {
    o->xm[threadIdx.x] = P[MLP_XM + threadIdx.x];
    o->xs[threadIdx.x] = P[MLP_XS + threadIdx.x];
  }
  if (threadIdx.x == 0) {
    o->b3 = P[MLP_B3];
    o->ym = P[MLP_YM];
    o->ys = P[MLP_YS];
  }
}

__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float wd, float c1,
                           float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= MLP_TRAIN) return;
  const float gi = g[i] + wd * p[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

int propose_grid() {  // 4 blocks per SM of the current device
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms * 4;
}

}  // namespace

int launch_mlp_pack(const float* params, MlpPacked* out, cudaStream_t s) {
  k_mlp_pack<<<1, 256, 0, s>>>(params, out);
  return 1;
}

int launch_mlp_propose(const Dev& d, const MlpPacked* w, const MlpFeatureArgs& fa, const float* divv, float* rec,
                       float* dh, bool apply, cudaStream_t s) {
  static std::atomic<unsigned long long> attr{0};
  smem_limit_per_device(k_mlp_propose, TC_SMEM, attr);
  const int tiles = (d.n + ROWS - 1) / ROWS;
  const int cap = propose_grid();
  const int grid = tiles < cap ? tiles : cap;
  k_mlp_propose<<<grid, ROWS, TC_SMEM, s>>>(d.n, d.s(), d.rho, d.nbr_cnt, d.acc, d.fdata, divv, d.eos, d.segs, d.P, fa,
                                      w, rec, dh, apply ? 1 : 0);
  return 1;
}

int launch_mlp_forward(const MlpPacked* w, const float* x, int n, float* out, unsigned* err, cudaStream_t s) {
  static std::atomic<unsigned long long> attr{0};
  smem_limit_per_device(k_mlp_forward, TC_SMEM, attr);
  const int tiles = (n + ROWS - 1) / ROWS;
  const int cap = propose_grid();
  const int grid = tiles < cap ? tiles : cap;
  k_mlp_forward<<<grid, ROWS, TC_SMEM, s>>>(w, x, n, out, err);
  return 1;
}

int launch_mlp_train_batch(const MlpPacked* w, const float* x, const float* t, const unsigned* idx, int m,
                           float denom, float* grad, float* loss, unsigned* err, cudaStream_t s) {
  static std::atomic<unsigned long long> attr{0};
  smem_limit_per_device(k_mlp_train_tc, (int)sizeof(TrainTcSmem), attr);
  k_mlp_train_tc<<<(m + ROWS - 1) / ROWS, ROWS, sizeof(TrainTcSmem), s>>>(w, x, t, idx, m, denom, grad, loss, err);
  return 1;
}

int launch_mlp_adam(float* params, const float* grad, float* m, float* v, int step, float lr, float b1, float b2,
                    float eps, float wd, cudaStream_t s) {
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_mlp_adam<<<(MLP_TRAIN + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr, b1, b2, eps, wd, c1, c2);
  return 1;
}

}  // namespace sphb

// ---- the network on its own (host arrays, blocking, the calling thread's current device) ------------------
using namespace sphb;

namespace {

struct DevBuf {
  std::vector<void*> ptrs;
  cudaError_t err = cudaSuccess;
  template <typename T>
  T* get(size_t count) {
    void* p = nullptr;
    if (err == cudaSuccess) err = cudaMalloc(&p, count * sizeof(T) > 0 ? count * sizeof(T) : 16);
    if (err == cudaSuccess) ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  ~DevBuf() {
    for (void* p : ptrs) cudaFree(p);
  }
};

sph_status status_of(cudaError_t e) {
  if (e == cudaSuccess) return SPH_OK;
  return e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

sph_status sph_mlp_forward(const float* params, const float* x, uint32_t n, float* out) {
  if (!params || (!x && n) || (!out && n)) return SPH_ERR_INVALID;
  if (n == 0) return SPH_OK;
  DevBuf b;
  float* dp = b.get<float>(MLP_TOTAL);
  MlpPacked* w = b.get<MlpPacked>(1);
  float* dx = b.get<float>((size_t)n * MLP_IN);
  float* dy = b.get<float>(n);
  unsigned* flag = b.get<unsigned>(1);
  if (b.err != cudaSuccess) return status_of(b.err);
  cudaError_t e = cudaMemcpy(dp, params, MLP_TOTAL * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(flag, 0, sizeof(unsigned));
  if (e != cudaSuccess) return status_of(e);
  launch_mlp_pack(dp, w, 0);
  launch_mlp_forward(w, dx, (int)n, dy, flag, 0);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(out, dy, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  unsigned timeout = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&timeout, flag, sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && timeout) return SPH_ERR_TIMEOUT;
  return status_of(e);
}

sph_status sph_mlp_grad(const float* params, const float* x, const float* t, uint32_t n, float* grad, float* loss) {
  if (!params || !x || !t || !grad || !loss || n == 0) return SPH_ERR_INVALID;
  DevBuf b;
  float* dp = b.get<float>(MLP_TOTAL);
  MlpPacked* w = b.get<MlpPacked>(1);
  float* dx = b.get<float>((size_t)n * MLP_IN);
  float* dt = b.get<float>(n);
  unsigned* idx = b.get<unsigned>(n);
  float* dg = b.get<float>(MLP_TRAIN + 1);  // gradient, then the summed squared error
  unsigned* flag = b.get<unsigned>(1);
  if (b.err != cudaSuccess) return status_of(b.err);
  std::vector<unsigned> id(n);
  for (uint32_t i = 0; i < n; ++i) id[i] = i;
  cudaError_t e = cudaMemcpy(dp, params, MLP_TOTAL * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dt, t, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(idx, id.data(), (size_t)n * sizeof(unsigned), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dg, 0, (MLP_TRAIN + 1) * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(flag, 0, sizeof(unsigned));
  if (e != cudaSuccess) return status_of(e);
  launch_mlp_pack(dp, w, 0);
  launch_mlp_train_batch(w, dx, dt, idx, (int)n, (float)n, dg, dg + MLP_TRAIN, flag, 0);
  e = cudaGetLastError();
  std::vector<float> h(MLP_TRAIN + 1);
  if (e == cudaSuccess) e = cudaMemcpy(h.data(), dg, h.size() * sizeof(float), cudaMemcpyDeviceToHost);
  unsigned timeout = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&timeout, flag, sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return status_of(e);
  if (timeout) return SPH_ERR_TIMEOUT;
  std::memcpy(grad, h.data(), MLP_TRAIN * sizeof(float));
  *loss = h[MLP_TRAIN] / (float)n;
  return SPH_OK;
}

sph_status sph_mlp_train(float* params, const float* x, const float* t, uint32_t n, const sph_mlp_train_cfg* cfg,
                         float* loss_per_epoch) {
  if (!params || !x || !t || !cfg || n == 0 || cfg->batch == 0 || !(cfg->lr > 0.0f)) return SPH_ERR_INVALID;
  DevBuf b;
  float* dp = b.get<float>(MLP_TOTAL);
  MlpPacked* w = b.get<MlpPacked>(1);
  float* dx = b.get<float>((size_t)n * MLP_IN);
  float* dt = b.get<float>(n);
  unsigned* idx = b.get<unsigned>(n);
  float* dg = b.get<float>(MLP_TRAIN + 1);
  float* dm = b.get<float>(MLP_TRAIN);
  float* dv = b.get<float>(MLP_TRAIN);
  float* dl = b.get<float>(1);
  unsigned* flag = b.get<unsigned>(1);
  if (b.err != cudaSuccess) return status_of(b.err);
  cudaError_t e = cudaMemcpy(dp, params, MLP_TOTAL * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dt, t, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dm, 0, MLP_TRAIN * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(dv, 0, MLP_TRAIN * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(flag, 0, sizeof(unsigned));
  if (e != cudaSuccess) return status_of(e);
  std::vector<unsigned> perm(n);
  for (uint32_t i = 0; i < n; ++i) perm[i] = i;
  uint64_t rs = cfg->seed * 0x2545F4914F6CDD1Dull + 1;
  const float b1 = cfg->beta1 > 0.0f ? cfg->beta1 : 0.9f, b2 = cfg->beta2 > 0.0f ? cfg->beta2 : 0.999f;
  const float eps = cfg->eps > 0.0f ? cfg->eps : 1.0e-8f;
  int step = 0;
  launch_mlp_pack(dp, w, 0);
  for (uint32_t ep = 0; ep < cfg->epochs; ++ep) {
    for (uint32_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[splitmix(rs) % (i + 1)]);  // Fisher-Yates
    e = cudaMemcpy(idx, perm.data(), (size_t)n * sizeof(unsigned), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dl, 0, sizeof(float));
    if (e != cudaSuccess) return status_of(e);
    for (uint32_t off = 0; off < n; off += cfg->batch) {
      const uint32_t m = n - off < cfg->batch ? n - off : cfg->batch;
      cudaMemsetAsync(dg, 0, MLP_TRAIN * sizeof(float), 0);
      launch_mlp_train_batch(w, dx, dt, idx + off, (int)m, (float)m, dg, dl, flag, 0);
      launch_mlp_adam(dp, dg, dm, dv, ++step, cfg->lr, b1, b2, eps, cfg->weight_decay, 0);
      launch_mlp_pack(dp, w, 0);
    }
    float l = 0.0f;
    unsigned timeout = 0;
    e = cudaMemcpy(&l, dl, sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&timeout, flag, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return status_of(e);
    if (timeout) return SPH_ERR_TIMEOUT;
    if (loss_per_epoch) loss_per_epoch[ep] = l / (float)n;
  }
  e = cudaMemcpy(params, dp, MLP_TRAIN * sizeof(float), cudaMemcpyDeviceToHost);
  return status_of(e);
}

}  // extern "C"
