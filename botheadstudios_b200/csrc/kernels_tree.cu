// LBVH construction on B200: bounding box → 30-bit Morton keys → LSD radix sort → state permutation →
// Karras internal nodes → single-pass bottom-up moments.
//
// Reference: shaders/bh_gravity.wgsl (cs_bbox :68, cs_morton :100, cs_tree :135, cs_com :201) and the CPU
// sort of crates/engine/src/gpu_gravity.rs:336-368. The sort order is (Morton code, original index), made
// exact by a stable radix sort of the codes laid out in original-index order, so the permutation, the leaf
// codes and the Karras topology are bit-identical to the reference's. A batch of impacts prefixes the code with the impact
// (segment) index: every impact is quantised in its own box, sorted into its own contiguous range and
// built into its own subtree, exactly as if it were alone.
#include <cuda/atomic>

#include "sph_kernels.cuh"

namespace sphb {

// ---------------------------------------------------------------------------------------------------
// Segment table set-up: the first particle of every leaf (leaves are K-particle buckets counted from the
// start of their segment; the last bucket of a segment may be partial).
// ---------------------------------------------------------------------------------------------------
__global__ void k_leaf_start(const Seg* __restrict__ segs, int nseg, int K, int L, int n,
                             unsigned* __restrict__ leaf_start) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > L) return;
  if (c == L) {
    leaf_start[L] = (unsigned)n;
    return;
  }
  int lo = 0, hi = nseg - 1;  // last segment whose first leaf is <= c
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].loff <= (unsigned)c) lo = mid;
    else hi = mid - 1;
  }
  leaf_start[c] = segs[lo].off + (unsigned)(c - (int)segs[lo].loff) * (unsigned)K;
}

int launch_segments(const Dev& d, cudaStream_t s) {
  k_leaf_start<<<(d.L + 1 + 255) / 256, 256, 0, s>>>(d.segs, d.nseg, d.K, d.L, d.n, d.leaf_start);
  return 1;
}

__global__ void k_segments_single(Seg* segs, int n, int L, float soft2, double dt) {
  Seg a;
  a.off = 0u;
  a.loff = 0u;
  a.root = 0u;
  a.sig_bits = 0x7f800000u;
  for (int k = 0; k < 3; ++k) {
    a.bbox[k] = 0xffffffffu;
    a.bbox[3 + k] = 0u;
  }
  a.soft2 = soft2;
  a.pad = 0u;
  a.res_bits = 0u;
  a.skin = 0.0f;
  a.dt = dt;
  a.time = 0.0;
  segs[0] = a;
  Seg e = a;
  e.off = (unsigned)n;
  e.loff = (unsigned)L;
  segs[1] = e;
}

int launch_segments_single(const Dev& d, float soft2, double dt, cudaStream_t s) {
  k_segments_single<<<1, 1, 0, s>>>(d.segs, d.n, d.L, soft2, dt);
  return 1 + launch_segments(d, s);
}

// ---------------------------------------------------------------------------------------------------
// Bounding box per segment (cs_bbox): order-preserving u32 keys, reduced per block (seg_bbox_commit).
// ---------------------------------------------------------------------------------------------------
__global__ void k_bbox_reset(Seg* segs, int nseg) {
  const int k = threadIdx.x;
  if (k >= nseg) return;
  for (int a = 0; a < 3; ++a) {
    segs[k].bbox[a] = 0xffffffffu;
    segs[k].bbox[3 + a] = 0u;
  }
}

__global__ void k_bbox(const float4* __restrict__ pos, const unsigned* __restrict__ seg, int n, Seg* segs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
  unsigned sg = kNoSeg;
  if (i < n) {
    const float4 p = pos[i];
    lo[0] = hi[0] = float_key(p.x);
    lo[1] = hi[1] = float_key(p.y);
    lo[2] = hi[2] = float_key(p.z);
    sg = seg[i];
  }
  seg_bbox_commit(lo, hi, sg, segs);
}

int launch_bbox(const Dev& d, cudaStream_t s) {
  k_bbox_reset<<<1, kMaxSegments, 0, s>>>(d.segs, d.nseg);
  k_bbox<<<(d.n + 255) / 256, 256, 0, s>>>(d.s().pos_h, d.s().seg, d.n, d.segs);
  return 2;
}

// ---------------------------------------------------------------------------------------------------
// Morton keys (cs_morton, bh_gravity.wgsl:91-108) with IEEE division, no contraction, each particle
// quantised in its own segment's box. The sort order is (segment, code, original index): each key
// segment << 30 | code is written at its particle's original index, so a stable sort on the key alone leaves
// equal keys in index order (30 + segment bits instead of 30 + segment + index bits: 4 passes, not 7, at 1M).
// ---------------------------------------------------------------------------------------------------
__global__ void k_keys(const float4* __restrict__ pos, const unsigned* __restrict__ id,
                       const unsigned* __restrict__ seg, int n, const Seg* __restrict__ segs,
                       unsigned long long* __restrict__ keys, unsigned* __restrict__ vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned sg = seg[i];
  const unsigned* bb = segs[sg].bbox;
  float lo[3], ext[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    lo[k] = key_float(bb[k]);
    ext[k] = fmaxf(fsub(key_float(bb[3 + k]), lo[k]), 1.0e-30f);
  }
  const float4 p = pos[i];
  const float pc[3] = {p.x, p.y, p.z};
  unsigned q[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float u = fdiv(fsub(pc[k], lo[k]), ext[k]);
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    float f = floorf(fmul(u, 1024.0f));
    f = fminf(fmaxf(f, 0.0f), 1023.0f);
    q[k] = (unsigned)f;
  }
  const unsigned code = expand_bits(q[0]) * 4u + expand_bits(q[1]) * 2u + expand_bits(q[2]);
  const unsigned o = id[i];  // a permutation of [0, n)
  keys[o] = ((unsigned long long)sg << 30) | code;
  vals[o] = (unsigned)i;
}

// ---------------------------------------------------------------------------------------------------
// LSD radix sort, 8-bit digits, reduce-then-scan (no inter-block waits): upsweep histograms per tile,
// per-digit scans over tiles, stable downsweep (warp match_any ranking, staged through shared memory).
// ---------------------------------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 2048 keys per tile
constexpr int RS_WARPS = RS_THREADS / 32;

size_t radix_tiles(int n) { return (size_t)((n + RS_TILE - 1) / RS_TILE); }

__global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(const unsigned long long* __restrict__ keys, int n,
                                                           int shift, unsigned* __restrict__ hist, int T) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * RS_TILE;
#pragma unroll
  for (int it = 0; it < RS_ITEMS; ++it) {
    const int idx = base + it * RS_THREADS + threadIdx.x;
    if (idx < n) atomicAdd(&h[(unsigned)(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * T + blockIdx.x] = h[threadIdx.x];
}

// One block per digit: exclusive scan of hist[d][0..T) in place; tot[d] = sum.
__global__ void __launch_bounds__(1024) k_rs_scan(unsigned* __restrict__ hist, unsigned* __restrict__ tot, int T) {
  __shared__ unsigned s_warp[33];
  unsigned* h = hist + (size_t)blockIdx.x * T;
  const int per = (T + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per;
  unsigned sum = 0;
  for (int i = 0; i < per; ++i)
    if (b0 + i < T) sum += h[b0 + i];
  unsigned total;
  unsigned run = block_exclusive_scan(sum, s_warp, total);
  for (int i = 0; i < per; ++i)
    if (b0 + i < T) {
      const unsigned v = h[b0 + i];
      h[b0 + i] = run;
      run += v;
    }
  if (threadIdx.x == 0) tot[blockIdx.x] = total;
}

__global__ void __launch_bounds__(RS_THREADS) k_rs_downsweep(const unsigned long long* __restrict__ kin,
                                                             const unsigned* __restrict__ vin,
                                                             unsigned long long* __restrict__ kout,
                                                             unsigned* __restrict__ vout, int n, int shift,
                                                             const unsigned* __restrict__ hist,
                                                             const unsigned* __restrict__ tot, int T) {
  __shared__ unsigned long long s_keys[RS_TILE];
  __shared__ unsigned s_vals[RS_TILE];
  __shared__ unsigned s_wcnt[RS_WARPS][256];
  __shared__ unsigned s_gbin[256];     // global output start of digit d for this tile
  __shared__ unsigned s_bstart[256];   // start of digit d inside the tile
  __shared__ unsigned s_warp[33];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int base = blockIdx.x * RS_TILE;

  // global digit starts: exclusive scan of the digit totals + this tile's prefix
  unsigned total;
  const unsigned dstart = block_exclusive_scan(tot[tid], s_warp, total);
  s_gbin[tid] = dstart + hist[tid * T + blockIdx.x];
#pragma unroll
  for (int k = 0; k < RS_WARPS; ++k) s_wcnt[k][tid] = 0;
  __syncthreads();

  unsigned long long key[RS_ITEMS];
  unsigned val[RS_ITEMS], dig[RS_ITEMS], loc[RS_ITEMS];
  const unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int it = 0; it < RS_ITEMS; ++it) {
    const int idx = base + (w * RS_ITEMS + it) * 32 + lane;
    const bool ok = idx < n;
    key[it] = ok ? kin[idx] : 0ull;
    val[it] = ok ? vin[idx] : 0u;
    const unsigned d = ok ? ((unsigned)(key[it] >> shift) & 255u) : 256u;
    dig[it] = d;
    const unsigned peers = __match_any_sync(SPH_FULL_MASK, d);
    const int leader = __ffs(peers) - 1;
    unsigned old = 0;
    if (lane == leader && ok) {
      old = s_wcnt[w][d];
      s_wcnt[w][d] = old + __popc(peers);
    }
    old = __shfl_sync(SPH_FULL_MASK, old, leader);
    loc[it] = old + __popc(peers & lt_mask);
    __syncwarp();
  }
  __syncthreads();
  // per digit: exclusive prefix over warps, then over digits within the tile
  {
    unsigned run = 0;
#pragma unroll
    for (int k = 0; k < RS_WARPS; ++k) {
      const unsigned c = s_wcnt[k][tid];
      s_wcnt[k][tid] = run;
      run += c;
    }
    unsigned t2;
    s_bstart[tid] = block_exclusive_scan(run, s_warp, t2);
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < RS_ITEMS; ++it) {
    if (dig[it] < 256u) {
      const unsigned p = s_bstart[dig[it]] + s_wcnt[w][dig[it]] + loc[it];
      s_keys[p] = key[it];
      s_vals[p] = val[it];
    }
  }
  __syncthreads();
  const int cnt = min(RS_TILE, n - base);
  for (int i = tid; i < cnt; i += RS_THREADS) {
    const unsigned long long k = s_keys[i];
    const unsigned d = (unsigned)(k >> shift) & 255u;
    const unsigned g = s_gbin[d] + (unsigned)i - s_bstart[d];
    kout[g] = k;
    vout[g] = s_vals[i];
  }
}

// ---------------------------------------------------------------------------------------------------
// Permutation of the particle state into the new order; leaf cluster codes (gpu_gravity.rs:366).
// ---------------------------------------------------------------------------------------------------
__global__ void k_permute(int n, int L, const unsigned* __restrict__ order,
                          const unsigned long long* __restrict__ skeys, const unsigned* __restrict__ leaf_start,
                          State in, State out, float4* __restrict__ body,
                          unsigned long long* __restrict__ leaf_codes) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const unsigned o = order[t];
  const float4 p = in.pos_h[o];
  const float m = in.mass[o];
  out.pos_h[t] = p;
  out.vel_u[t] = in.vel_u[o];
  out.x[t] = in.x[o];
  out.y[t] = in.y[o];
  out.z[t] = in.z[o];
  out.mass[t] = m;
  out.mat[t] = in.mat[o];
  out.prov[t] = in.prov[o];
  out.id[t] = in.id[o];
  out.seg[t] = in.seg[o];
  body[t] = make_float4(p.x, p.y, p.z, m);
  if (t < L) leaf_codes[t] = skeys[leaf_start[t]];
}

int launch_sort_permute(Dev& d, cudaStream_t s) {
  const int n = d.n;
  const int threads = 256;
  const int blocks = (n + threads - 1) / threads;
  const State& in = d.st[d.cur];
  k_keys<<<blocks, threads, 0, s>>>(in.pos_h, in.id, in.seg, n, d.segs, d.keys[0], d.vals[0]);
  const int T = (int)radix_tiles(n);
  const int total_bits = 30 + d.segbits;
  const int passes = (total_bits + 7) / 8;
  int src = 0;
  for (int shift = 0; shift < total_bits; shift += 8) {
    k_rs_upsweep<<<T, RS_THREADS, 0, s>>>(d.keys[src], n, shift, d.rs_hist, T);
    k_rs_scan<<<256, 1024, 0, s>>>(d.rs_hist, d.rs_tot, T);
    k_rs_downsweep<<<T, RS_THREADS, 0, s>>>(d.keys[src], d.vals[src], d.keys[src ^ 1], d.vals[src ^ 1], n, shift,
                                             d.rs_hist, d.rs_tot, T);
    src ^= 1;
  }
  // vals[src] = old slot of each sorted position; keys[src] = sorted keys
  const State& out = d.st[d.cur ^ 1];
  k_permute<<<blocks, threads, 0, s>>>(n, d.L, d.vals[src], d.keys[src], d.leaf_start, in, out, d.body,
                                       d.leaf_codes);
  d.cur ^= 1;
  // keep the sorted keys in keys[0] for inspection
  if (src != 0) cudaMemcpyAsync(d.keys[0], d.keys[src], sizeof(unsigned long long) * n, cudaMemcpyDeviceToDevice, s);
  return 2 + 3 * passes;
}

// Stable LSD radix sort of n (key, value) pairs on the low `bits` key bits, ping-ponging between buf 0 and 1.
// Returns the buffer holding the result in `src`; hist holds 256 × radix_tiles(n) counters.
int launch_radix_sort(unsigned long long* keys[2], unsigned* vals[2], int n, int bits, unsigned* hist,
                      unsigned* tot, int& src, cudaStream_t s) {
  src = 0;
  if (n <= 1) return 0;
  const int T = (int)radix_tiles(n);
  int launches = 0;
  for (int shift = 0; shift < bits; shift += 8) {
    k_rs_upsweep<<<T, RS_THREADS, 0, s>>>(keys[src], n, shift, hist, T);
    k_rs_scan<<<256, 1024, 0, s>>>(hist, tot, T);
    k_rs_downsweep<<<T, RS_THREADS, 0, s>>>(keys[src], vals[src], keys[src ^ 1], vals[src ^ 1], n, shift, hist,
                                             tot, T);
    src ^= 1;
    launches += 3;
  }
  return launches;
}

// ---------------------------------------------------------------------------------------------------
// Karras 2012 internal nodes over the leaf cluster codes (cs_tree, bh_gravity.wgsl:114-184).
// ---------------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned code_seg(unsigned long long c) { return (unsigned)(c >> 30); }

// Leaf codes are segment << 30 | Morton code: one impact's leaves share the top bits, so each impact is one
// subtree. Equal codes (always within one impact) are told apart by the leaf index counted from the impact's
// first leaf, so an impact's subtree is the tree it would get alone. With one segment every delta is the
// reference's plus 32 (bh_gravity.wgsl:114-120), which leaves every comparison unchanged.
__device__ __forceinline__ int kdelta(const unsigned long long* __restrict__ codes, const Seg* __restrict__ segs,
                                      int L, int i, int j) {
  if (j < 0 || j >= L) return -1;
  const unsigned long long ci = codes[i], cj = codes[j];
  if (ci == cj) {
    const unsigned base = segs[code_seg(ci)].loff;
    return 64 + __clz(((unsigned)i - base) ^ ((unsigned)j - base));
  }
  return __clzll(ci ^ cj);
}

// Leaves [first, last] are exactly one segment.
__device__ __forceinline__ bool whole_segment(const unsigned long long* __restrict__ codes, int L, int first,
                                              int last) {
  const unsigned sg = code_seg(codes[first]);
  return code_seg(codes[last]) == sg && (first == 0 || code_seg(codes[first - 1]) != sg) &&
         (last == L - 1 || code_seg(codes[last + 1]) != sg);
}

__global__ void k_karras(const unsigned long long* __restrict__ codes, int L, unsigned* __restrict__ left,
                         unsigned* __restrict__ right, unsigned* __restrict__ parent,
                         Seg* __restrict__ segs, int exact_dups) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L - 1) return;
  const int d = kdelta(codes, segs, L, i, i + 1) > kdelta(codes, segs, L, i, i - 1) ? 1 : -1;
  const int dmin = kdelta(codes, segs, L, i, i - d);
  int lmax = 2;
  while (kdelta(codes, segs, L, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (kdelta(codes, segs, L, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int first = min(i, j), last = max(i, j);
  int split = first;
  const unsigned long long fc = codes[first], lc = codes[last];
  if (fc == lc && !exact_dups) {
    // the reference's split of a run of equal codes (bh_gravity.wgsl:159-160); it can disagree with the
    // index-extended ranges the children compute for themselves, so such trees may be invalid
    split = (first + last) >> 1;
  } else if (fc == lc) {
    // Karras 2012 §4: index-extended keys — binary search on the common prefix of the indices
    const int cpfx = kdelta(codes, segs, L, first, last);
    int step = last - first;
    for (;;) {
      step = (step + 1) >> 1;
      const int ns = split + step;
      if (ns < last && kdelta(codes, segs, L, first, ns) > cpfx) split = ns;
      if (step <= 1) break;
    }
  } else {
    const int cpfx = __clzll(fc ^ lc);
    int step = last - first;
    for (;;) {
      step = (step + 1) >> 1;
      const int ns = split + step;
      if (ns < last && __clzll(fc ^ codes[ns]) > cpfx) split = ns;
      if (step <= 1) break;
    }
  }
  const unsigned lidx = (split == first) ? (unsigned)(L - 1 + split) : (unsigned)split;
  const unsigned ridx = (split + 1 == last) ? (unsigned)(L - 1 + split + 1) : (unsigned)(split + 1);
  left[i] = lidx;
  right[i] = ridx;
  parent[lidx] = (unsigned)i;
  parent[ridx] = (unsigned)i;
  // segment roots: the node spanning exactly one impact (a leaf when the impact has one leaf)
  if (whole_segment(codes, L, first, last)) segs[code_seg(fc)].root = (unsigned)i;
  if (split == first && whole_segment(codes, L, first, first)) segs[code_seg(fc)].root = lidx;
  if (split + 1 == last && whole_segment(codes, L, last, last)) segs[code_seg(lc)].root = ridx;
}

// Walk groups: each impact's leaves in consecutive runs of `per` (= 32/K) leaves, so a warp holds 32
// Morton-consecutive particles of one impact (the walk splits a run where consecutive particles are far
// apart). Against maximal LBVH subtrees of <= 32 particles (which left ~22 % of the lanes idle) this is
// 10 % faster at 1M with the same gravity error. Group offsets per impact go to Seg::pad (serial over <= 256 impacts), then one thread per leaf
// writes the group its run starts.
__global__ void k_group_offsets(Seg* segs, int nseg, int per, unsigned* ngroups) {
  if (threadIdx.x != 0) return;
  unsigned g = 0;
  for (int k = 0; k < nseg; ++k) {
    segs[k].pad = g;
    g += (segs[k + 1].loff - segs[k].loff + per - 1) / per;
  }
  segs[nseg].pad = g;
  *ngroups = g;
}

__global__ void k_run_groups(const Seg* __restrict__ segs, int nseg, int per, int L, uint2* __restrict__ groups) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L) return;
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].loff <= (unsigned)c) lo = mid;
    else hi = mid - 1;
  }
  const unsigned local = (unsigned)c - segs[lo].loff;
  if (local % per) return;
  const unsigned last = min((unsigned)c + per - 1, segs[lo + 1].loff - 1);
  groups[segs[lo].pad + local / per] = make_uint2((unsigned)c, last);
}

__global__ void k_single_leaf_root(Seg* segs) { segs[0].root = 0u; }

// ---------------------------------------------------------------------------------------------------
// Bottom-up moments (cs_com, bh_gravity.wgsl:201-241), single pass: each leaf thread sums its bucket, then
// climbs; the first child to arrive at a parent stops, the second merges. The arrival counter is an
// acq_rel device-scope atomic, so the second arrival sees the sibling's node data (the ordering that WGSL
// could not express and that made the reference fall back to a 33-dispatch sweep). The climb is bounded
// by the tree height; nothing waits.
// Node data: com.xyz/mass (mass-weighted merge, same f32 operations as the reference), AABB with the
// subtree's max smoothing length, the opening radius size/θ + |centre − COM| (size: the largest side for the
// group walk, the diagonal for the reference's per-particle walk) and, optionally, the
// traceless quadrupole about the COM (parallel-axis merge).
// ---------------------------------------------------------------------------------------------------
template <bool QUAD>
__global__ void k_leaf_climb(const float4* __restrict__ body, const float4* __restrict__ pos_h,
                             const unsigned* __restrict__ leaf_start, int L, const unsigned* __restrict__ left, const unsigned* __restrict__ right,
                             const unsigned* __restrict__ parent, unsigned* __restrict__ counters,
                             float4* __restrict__ ncom, float4* __restrict__ nbmin, float4* __restrict__ nbmax,
                             float4* __restrict__ nq0, float4* __restrict__ nq1, float theta, int side_mac,
                             int half, float4* __restrict__ hcom, float4* __restrict__ hq0,
                             float2* __restrict__ hq1, float2* __restrict__ hrc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L) return;
  const int li = L - 1 + c;
  const int s0 = (int)leaf_start[c], s1 = (int)leaf_start[c + 1];
  float m = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f, hmax = 0.0f;
  float lo[3] = {1.0e30f, 1.0e30f, 1.0e30f}, hi[3] = {-1.0e30f, -1.0e30f, -1.0e30f};
  for (int s = s0; s < s1; ++s) {
    const float4 b = body[s];
    m = fadd(m, b.w);
    mx = fadd(mx, fmul(b.x, b.w));
    my = fadd(my, fmul(b.y, b.w));
    mz = fadd(mz, fmul(b.z, b.w));
    lo[0] = fminf(lo[0], b.x); lo[1] = fminf(lo[1], b.y); lo[2] = fminf(lo[2], b.z);
    hi[0] = fmaxf(hi[0], b.x); hi[1] = fmaxf(hi[1], b.y); hi[2] = fmaxf(hi[2], b.z);
    hmax = fmaxf(hmax, pos_h[s].w);
  }
  float4 com = make_float4(m > 0.0f ? fdiv(mx, m) : 0.0f, m > 0.0f ? fdiv(my, m) : 0.0f,
                           m > 0.0f ? fdiv(mz, m) : 0.0f, m);
  {
    const float ex = fsub(hi[0], lo[0]), ey = fsub(hi[1], lo[1]), ez = fsub(hi[2], lo[2]);
    const float size = side_mac ? fmaxf(fmaxf(ex, ey), ez) : fsqrt(dot3_exact(ex, ey, ez));
    const float cx = fsub(fmul(0.5f, fadd(lo[0], hi[0])), com.x), cy = fsub(fmul(0.5f, fadd(lo[1], hi[1])), com.y),
                cz = fsub(fmul(0.5f, fadd(lo[2], hi[2])), com.z);
    const float rc = fadd(fdiv(size, theta), fsqrt(dot3_exact(cx, cy, cz)));
    ncom[li] = com;
    nbmin[li] = make_float4(lo[0], lo[1], lo[2], hmax);
    nbmax[li] = make_float4(hi[0], hi[1], hi[2], rc);
  }
  if (half > 0) {
    // the leaf's two halves as multipoles of their own (the far field of the group walk): COM, mass, the
    // traceless quadrupole about that COM, and the opening radius largest side/θ + |centre − COM|
    float rcs[2] = {0.0f, 0.0f};
    for (int b = 0; b < 2; ++b) {
      const int a0 = s0 + b * half, a1 = min(s0 + (b + 1) * half, s1);
      float hm = 0.0f, hx = 0.0f, hy = 0.0f, hz = 0.0f;
      float l3[3] = {1.0e30f, 1.0e30f, 1.0e30f}, u3[3] = {-1.0e30f, -1.0e30f, -1.0e30f};
      for (int s = a0; s < a1; ++s) {
        const float4 q = body[s];
        hm += q.w;
        hx = fmaf(q.x, q.w, hx);
        hy = fmaf(q.y, q.w, hy);
        hz = fmaf(q.z, q.w, hz);
        l3[0] = fminf(l3[0], q.x); l3[1] = fminf(l3[1], q.y); l3[2] = fminf(l3[2], q.z);
        u3[0] = fmaxf(u3[0], q.x); u3[1] = fmaxf(u3[1], q.y); u3[2] = fmaxf(u3[2], q.z);
      }
      const float inv = hm > 0.0f ? 1.0f / hm : 0.0f;
      const float4 hc = make_float4(hx * inv, hy * inv, hz * inv, hm);
      if (a1 > a0) {
        const float ex = u3[0] - l3[0], ey = u3[1] - l3[1], ez = u3[2] - l3[2];
        const float size = fmaxf(fmaxf(ex, ey), ez);
        const float cx = 0.5f * (l3[0] + u3[0]) - hc.x, cy = 0.5f * (l3[1] + u3[1]) - hc.y,
                    cz = 0.5f * (l3[2] + u3[2]) - hc.z;
        rcs[b] = size / theta + sqrtf(cx * cx + cy * cy + cz * cz);
      }
      float qxx = 0, qyy = 0, qzz = 0, qxy = 0, qxz = 0, qyz = 0;
      if (QUAD) {
        for (int s = a0; s < a1; ++s) {
          const float4 q = body[s];
          const float dx = q.x - hc.x, dy = q.y - hc.y, dz = q.z - hc.z;
          const float r2 = dx * dx + dy * dy + dz * dz;
          qxx += q.w * (3.0f * dx * dx - r2);
          qyy += q.w * (3.0f * dy * dy - r2);
          qzz += q.w * (3.0f * dz * dz - r2);
          qxy += q.w * 3.0f * dx * dy;
          qxz += q.w * 3.0f * dx * dz;
          qyz += q.w * 3.0f * dy * dz;
        }
      }
      hcom[2 * c + b] = hc;
      hq0[2 * c + b] = make_float4(qxx, qyy, qzz, qxy);
      hq1[2 * c + b] = make_float2(qxz, qyz);
    }
    hrc[c] = make_float2(rcs[0], rcs[1]);
  }
  if (QUAD) {
    float qxx = 0, qyy = 0, qzz = 0, qxy = 0, qxz = 0, qyz = 0;
    for (int s = s0; s < s1; ++s) {
      const float4 b = body[s];
      const float dx = b.x - com.x, dy = b.y - com.y, dz = b.z - com.z;
      const float r2 = dx * dx + dy * dy + dz * dz;
      qxx += b.w * (3.0f * dx * dx - r2);
      qyy += b.w * (3.0f * dy * dy - r2);
      qzz += b.w * (3.0f * dz * dz - r2);
      qxy += b.w * 3.0f * dx * dy;
      qxz += b.w * 3.0f * dx * dz;
      qyz += b.w * 3.0f * dy * dz;
    }
    nq0[li] = make_float4(qxx, qyy, qzz, qxy);
    nq1[li] = make_float4(qxz, qyz, 0.0f, 0.0f);
  }
  unsigned node = parent[li];
  while (node != SPH_NO_PARENT) {
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(counters[node]);
    const unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
    if (arrived == 0u) return;  // the sibling subtree finishes this node
    const unsigned l = left[node], r = right[node];
    const float4 cl = __ldcg(&ncom[l]), cr = __ldcg(&ncom[r]);
    const float4 ll = __ldcg(&nbmin[l]), rl = __ldcg(&nbmin[r]);
    const float4 lh = __ldcg(&nbmax[l]), rh = __ldcg(&nbmax[r]);
    const float mm = fadd(cl.w, cr.w);
    const float4 pc = make_float4(mm > 0.0f ? fdiv(fadd(fmul(cl.x, cl.w), fmul(cr.x, cr.w)), mm) : 0.0f,
                                  mm > 0.0f ? fdiv(fadd(fmul(cl.y, cl.w), fmul(cr.y, cr.w)), mm) : 0.0f,
                                  mm > 0.0f ? fdiv(fadd(fmul(cl.z, cl.w), fmul(cr.z, cr.w)), mm) : 0.0f, mm);
    const float bl[3] = {fminf(ll.x, rl.x), fminf(ll.y, rl.y), fminf(ll.z, rl.z)};
    const float bh[3] = {fmaxf(lh.x, rh.x), fmaxf(lh.y, rh.y), fmaxf(lh.z, rh.z)};
    const float ex = fsub(bh[0], bl[0]), ey = fsub(bh[1], bl[1]), ez = fsub(bh[2], bl[2]);
    const float size = side_mac ? fmaxf(fmaxf(ex, ey), ez) : fsqrt(dot3_exact(ex, ey, ez));
    const float cx = fsub(fmul(0.5f, fadd(bl[0], bh[0])), pc.x), cy = fsub(fmul(0.5f, fadd(bl[1], bh[1])), pc.y),
                cz = fsub(fmul(0.5f, fadd(bl[2], bh[2])), pc.z);
    const float rc = fadd(fdiv(size, theta), fsqrt(dot3_exact(cx, cy, cz)));
    ncom[node] = pc;
    nbmin[node] = make_float4(bl[0], bl[1], bl[2], fmaxf(ll.w, rl.w));
    nbmax[node] = make_float4(bh[0], bh[1], bh[2], rc);
    if (QUAD) {
      float4 q0 = make_float4(0, 0, 0, 0), q1 = make_float4(0, 0, 0, 0);
      const float4 cc[2] = {cl, cr};
      const unsigned ch[2] = {l, r};
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const float4 a0 = __ldcg(&nq0[ch[k]]), a1 = __ldcg(&nq1[ch[k]]);
        const float sx = cc[k].x - pc.x, sy = cc[k].y - pc.y, sz = cc[k].z - pc.z, w = cc[k].w;
        const float s2 = sx * sx + sy * sy + sz * sz;
        q0.x += a0.x + w * (3.0f * sx * sx - s2);
        q0.y += a0.y + w * (3.0f * sy * sy - s2);
        q0.z += a0.z + w * (3.0f * sz * sz - s2);
        q0.w += a0.w + w * 3.0f * sx * sy;
        q1.x += a1.x + w * 3.0f * sx * sz;
        q1.y += a1.y + w * 3.0f * sy * sz;
      }
      nq0[node] = q0;
      nq1[node] = q1;
    }
    node = parent[node];
  }
}

int launch_tree(const Dev& d, const Cfg& c, float theta, cudaStream_t s) {
  const int L = d.L;
  cudaMemsetAsync(d.parent, 0xff, sizeof(unsigned) * (2 * (size_t)L - 1), s);
  cudaMemsetAsync(d.ngroups, 0, sizeof(unsigned), s);
  if (L > 1) {
    cudaMemsetAsync(d.counters, 0, sizeof(unsigned) * (L - 1), s);
    k_karras<<<(L - 1 + 255) / 256, 256, 0, s>>>(d.leaf_codes, L, d.left, d.right, d.parent, d.segs,
                                                  c.mac == 0 ? 1 : 0);
  } else {
    k_single_leaf_root<<<1, 1, 0, s>>>(d.segs);
  }
  k_group_offsets<<<1, 32, 0, s>>>(d.segs, d.nseg, 32 / d.K, d.ngroups);
  k_run_groups<<<(L + 255) / 256, 256, 0, s>>>(d.segs, d.nseg, 32 / d.K, L, d.groups);
  const State& st = d.s();
  const int side_mac = c.mac == 0 ? 1 : 0;
  const int half = half_leaf(d, c);
  if (c.quad)
    k_leaf_climb<true><<<(L + 127) / 128, 128, 0, s>>>(d.body, st.pos_h, d.leaf_start, L, d.left, d.right, d.parent,
                                                       d.counters, d.ncom, d.nbmin, d.nbmax, d.nq0, d.nq1, theta,
                                                       side_mac, half, d.hcom, d.hq0, d.hq1, d.hrc);
  else
    k_leaf_climb<false><<<(L + 127) / 128, 128, 0, s>>>(d.body, st.pos_h, d.leaf_start, L, d.left, d.right, d.parent,
                                                        d.counters, d.ncom, d.nbmin, d.nbmax, d.nq0, d.nq1, theta,
                                                        side_mac, half, d.hcom, d.hq0, d.hq1, d.hrc);
  return 2;
}

// Far leaves are split in the group walk when a half holds at least 8 particles: one quadrupole evaluation
// (~50 instructions) then replaces 8 pairwise ones (~14 each); halves of 4 would not pay.
int half_leaf(const Dev& d, const Cfg& c) {
  return (c.mac == 0 && c.gravity == 0 && d.K >= 16 && d.hcom) ? d.K / 2 : 0;
}

}  // namespace sphb
