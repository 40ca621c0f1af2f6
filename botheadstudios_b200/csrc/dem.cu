// Granular (DEM) contact on B200: the contact law and the θ-implicit velocity solve of the reference's GPU
// grain pipeline (shaders/particle_step.wgsl: contact_accel :167-211, cs_forces :273-336, cs_integrate
// :477-530), on the same Morton sort / LBVH / neighbour-list machinery as the SPH step. The reference finds
// contacts with a hierarchical spatial hash whose buckets it sorts for determinism (cs_grid_sort :229-249);
// here every grain's contact candidates come from the tree walk with h = 2r + COH_RANGE (so that
// ½(h_i + h_j) = r_i + r_j + COH_RANGE is the reach), and the contact kernel applies the reference's exact
// cut. The ground scene's terrain heightfield contact, air drag, cooling, settle counter and incandescence
// (cs_integrate :477-576, terrain_* :338-452) run in the integrate kernel; the render expansion (cs_expand,
// 8 draw-only sub-cubes per grain) is not built. Grain density rides in the state's material slot and the
// settle counter in its provenance slot (both as float bits), so the sort carries them with the grain.
#include "sph_kernels.cuh"

namespace sphb {

constexpr float kDemTheta = 0.70f;   // particle_step.wgsl:125
constexpr float kDemCohRange = 0.15f;  // particle_step.wgsl:163

struct G80 {  // particle_step.wgsl:127-137 Particle (80 bytes)
  float ox, oy, oz, u, vx, vy, vz, resting, cr, cg, cb, material, er, eg, eb, rho, radius, p0, p1, p2;
};
static_assert(sizeof(G80) == 80, "grain layout is 80 bytes");

__global__ void k_dem_load(int n, const G80* __restrict__ in, State st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const G80 g = in[i];
  st.pos_h[i] = make_float4(g.ox, g.oy, g.oz, 2.0f * g.radius + kDemCohRange);
  st.vel_u[i] = make_float4(g.vx, g.vy, g.vz, g.u);
  st.x[i] = (double)g.ox;
  st.y[i] = (double)g.oy;
  st.z[i] = (double)g.oz;
  st.mass[i] = g.radius;  // the grain radius rides in the mass slot (grains carry no mass in the law)
  st.mat[i] = __float_as_uint(g.rho);       // drag reads the grain's own density
  st.prov[i] = __float_as_uint(g.resting);  // grounded-substep counter
  st.id[i] = (unsigned)i;
  st.seg[i] = 0u;
}

// particle_step.wgsl:106-118: temperature from u = c·T, and the glow of a hot grain.
__device__ __forceinline__ float3 incandescence(float t) {
  if (t <= 800.0f) return make_float3(0.f, 0.f, 0.f);
  const float x = t - 800.0f;
  const float intensity = fminf(fmaxf(x / 2200.0f, 0.0f), 4.0f);
  const float gg = fminf(fmaxf(x / 2200.0f, 0.0f), 1.0f);
  const float bb = fminf(fmaxf((t - 2600.0f) / 2400.0f, 0.0f), 1.0f);
  return make_float3(intensity, gg * intensity, bb * intensity);
}

__global__ void k_dem_store(int n, State st, DemParams p, int stepped, G80* __restrict__ io) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  G80* g = io + st.id[t];
  const float4 v = st.vel_u[t];
  g->ox = (float)st.x[t];
  g->oy = (float)st.y[t];
  g->oz = (float)st.z[t];
  g->vx = v.x;
  g->vy = v.y;
  g->vz = v.z;
  g->u = v.w;
  g->resting = __uint_as_float(st.prov[t]);
  if (stepped) {  // cs_integrate writes the glow of the grain's current temperature every substep
    const float3 e = incandescence(v.w / fmaxf(p.specific_heat, 1.0f));
    g->er = e.x;
    g->eg = e.y;
    g->eb = e.z;
  }
}

// ---- terrain (particle_step.wgsl:338-452) -----------------------------------------------------------------
// A column top in centred coordinates, clamped to the heightfield's edge (flat beyond it).
__device__ __forceinline__ float terrain_top(const DemParams& p, int cx, int cz) {
  const int x = min(max(cx, 0), (int)p.ww - 1), z = min(max(cz, 0), (int)p.wd - 1);
  return fsub(fsub((float)p.hf[(unsigned)z * p.ww + (unsigned)x], p.cy), 0.5f);
}
__device__ __forceinline__ float mixf(float a, float b, float t) { return fadd(fmul(a, fsub(1.0f, t)), fmul(b, t)); }
// The bilinear surface height and its horizontal gradient (h, ∂h/∂x, ∂h/∂z) below a position.
__device__ __forceinline__ float3 terrain_surface(const DemParams& p, float px, float pz) {
  const float vx = fadd(px, p.cx), vz = fadd(pz, p.cz);
  const int cx = (int)floorf(vx), cz = (int)floorf(vz);
  const float h00 = terrain_top(p, cx, cz), h10 = terrain_top(p, cx + 1, cz);
  const float h01 = terrain_top(p, cx, cz + 1), h11 = terrain_top(p, cx + 1, cz + 1);
  const float fx = fsub(vx, (float)cx), fz = fsub(vz, (float)cz);
  return make_float3(mixf(mixf(h00, h10, fx), mixf(h01, h11, fx), fz), mixf(fsub(h10, h00), fsub(h11, h01), fz),
                     mixf(fsub(h01, h00), fsub(h11, h10), fx));
}
// The outward surface normal (−∂h/∂x, 1, −∂h/∂z), normalised.
__device__ __forceinline__ float3 terrain_normal(float3 s) {
  const float nx = -s.y, nz = -s.z;
  const float l = fsqrt(dot3_exact(nx, 1.0f, nz));
  return make_float3(fdiv(nx, l), fdiv(1.0f, l), fdiv(nz, l));
}

// One grain pair (contact_accel, particle_step.wgsl:167-211): acceleration on i, the implicit-solve tensor
// g·n⊗n of a compressed contact and the neighbour coupling g(n·v_j)n.
__device__ __forceinline__ void dem_pair(float4 pi, float4 vi, float ri, float4 pj, float4 vj, float rj,
                                         const DemParams& p, float4& f, float4& sd, float4& so, float4& sv) {
  const float dx = fsub(pi.x, pj.x), dy = fsub(pi.y, pj.y), dz = fsub(pi.z, pj.z);
  const float dist = fsqrt(dot3_exact(dx, dy, dz));
  const float touch = ri + rj;
  if (dist >= touch + kDemCohRange || dist < 1.0e-9f) return;
  const float nx = dx / dist, ny = dy / dist, nz = dz / dist;
  const float overlap = touch - dist;
  const float vrx = vi.x - vj.x, vry = vi.y - vj.y, vrz = vi.z - vj.z;
  const float v_n = vrx * nx + vry * ny + vrz * nz;
  const float f_rep = p.stiffness * fmaxf(overlap, 0.0f);
  const float sep = fmaxf(-overlap, 0.0f);
  const float f_coh = p.cohesion * fminf(fmaxf(1.0f - sep / kDemCohRange, 0.0f), 1.0f);
  const float normal_load = f_rep + f_coh;
  const float vtx = vrx - nx * v_n, vty = vry - ny * v_n, vtz = vrz - nz * v_n;
  const float vt_mag = sqrtf(vtx * vtx + vty * vty + vtz * vtz);
  float atx = 0.f, aty = 0.f, atz = 0.f;
  if (vt_mag > 1.0e-9f) {
    const float mag = fminf(fminf(p.tangent_damp * vt_mag, p.friction * normal_load), vt_mag / p.dt);
    atx = -(vtx / vt_mag) * mag;
    aty = -(vty / vt_mag) * mag;
    atz = -(vtz / vt_mag) * mag;
  }
  const float fn = f_rep - f_coh;
  f.x += nx * fn + atx;
  f.y += ny * fn + aty;
  f.z += nz * fn + atz;
  if (overlap > 0.0f) {
    const float g = kDemTheta * kDemTheta * p.dt * p.dt * p.stiffness + kDemTheta * p.dt * p.normal_damp;
    sd.x += g * nx * nx;
    sd.y += g * ny * ny;
    sd.z += g * nz * nz;
    so.x += g * (nx * ny);
    so.y += g * (nx * nz);
    so.z += g * (ny * nz);
    const float ndv = nx * vj.x + ny * vj.y + nz * vj.z;
    sv.x += g * ndv * nx;
    sv.y += g * ndv * ny;
    sv.z += g * ndv * nz;
  }
}

// cs_forces (:273-336) for grain-grain contacts: gather over the candidate list. Output per grain: 4 float4
// (force + headroom, s_diag, s_off, sv_nbr) — the reference's Accum record.
__global__ void k_dem_contacts(int n, State st, const unsigned* __restrict__ nbr, const unsigned* __restrict__ cnt,
                               unsigned cap, DemParams p, float4* __restrict__ acc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float4 pi = st.pos_h[t], vi = st.vel_u[t];
  const float ri = st.mass[t];
  float4 f = make_float4(0.f, 0.f, 0.f, 1.0e30f), sd = make_float4(0.f, 0.f, 0.f, 0.f),
         so = make_float4(0.f, 0.f, 0.f, 0.f), sv = make_float4(0.f, 0.f, 0.f, 0.f);
  const unsigned c = min(cnt[t], cap);
  // headroom (particle_step.wgsl:282-336): the free gap to the nearest grain ahead along the terrain normal.
  // Only gaps below the 1 cm projection cap matter, and those grains are all contact candidates.
  const bool terrain = p.hf != nullptr;
  const float3 tn = terrain ? terrain_normal(terrain_surface(p, pi.x, pi.z)) : make_float3(0.f, 1.f, 0.f);
  for (unsigned k = 0; k < c; ++k) {
    const unsigned j = nbr[nbr_slot((unsigned)t, k, cap)];
    const float4 pj = st.pos_h[j];
    const float rj = st.mass[j];
    dem_pair(pi, vi, ri, pj, st.vel_u[j], rj, p, f, sd, so, sv);
    if (terrain) {
      const float dx = fsub(pj.x, pi.x), dy = fsub(pj.y, pi.y), dz = fsub(pj.z, pi.z);
      if (fadd(fadd(fmul(dx, tn.x), fmul(dy, tn.y)), fmul(dz, tn.z)) > 0.0f)
        f.w = fminf(f.w, fmaxf(fsub(fsqrt(dot3_exact(dx, dy, dz)), fadd(ri, rj)), 0.0f));
    }
  }
  acc[4 * (size_t)t + 0] = f;
  acc[4 * (size_t)t + 1] = sd;
  acc[4 * (size_t)t + 2] = so;
  acc[4 * (size_t)t + 3] = sv;
}

// cs_integrate's directional trapezoidal solve (:477-530): (I+S)v' = v − ρSv + (1/θ)ΣS_c v_j + dt·a,
// x += dt(v + v')/2 (f64 master positions).
// Per-substep cap of the terrain's position projection (particle_step.wgsl:395).
constexpr float kMaxSurfaceCorrection = 0.01f;

__global__ void k_dem_integrate(int n, State st, const float4* __restrict__ acc, DemParams p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float4 f = acc[4 * (size_t)t], sd = acc[4 * (size_t)t + 1], so = acc[4 * (size_t)t + 2],
               svn = acc[4 * (size_t)t + 3];
  float4 v = st.vel_u[t];
  // Newton cooling toward c·300 K, in energy
  const float u_amb = p.specific_heat * 300.0f;
  v.w = u_amb + (v.w - u_amb) * expf(-p.cool_rate * p.dt);
  const float rho_t = (1.0f - kDemTheta) / kDemTheta;
  float ax = p.gx + f.x, ay = p.gy + f.y, az = p.gz + f.z;
  const float r_self = st.mass[t];
  // aerodynamic drag a = ½ ρ_air v² C_d / (ρ_grain s), s = 2r, opposing the motion
  const float sp = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
  if (p.air_rho > 0.0f && sp > 1.0e-9f) {
    const float s_grain = fmaxf(2.0f * r_self, 1.0e-6f);
    const float a_drag = 0.5f * p.air_rho * sp * sp * p.drag_cd / (fmaxf(__uint_as_float(st.mat[t]), 1.0e-6f) * s_grain);
    ax -= (a_drag / sp) * v.x;
    ay -= (a_drag / sp) * v.y;
    az -= (a_drag / sp) * v.z;
  }
  const float sx = sd.x * v.x + so.x * v.y + so.y * v.z;
  const float sy = so.x * v.x + sd.y * v.y + so.z * v.z;
  const float sz = so.y * v.x + so.z * v.y + sd.z * v.z;
  const float rx = v.x - rho_t * sx + (1.0f / kDemTheta) * svn.x + ax * p.dt;
  const float ry = v.y - rho_t * sy + (1.0f / kDemTheta) * svn.y + ay * p.dt;
  const float rz = v.z - rho_t * sz + (1.0f / kDemTheta) * svn.z + az * p.dt;
  const float m00 = 1.0f + sd.x, m11 = 1.0f + sd.y, m22 = 1.0f + sd.z, m01 = so.x, m02 = so.y, m12 = so.z;
  const float c00 = m11 * m22 - m12 * m12, c01 = m02 * m12 - m01 * m22, c02 = m01 * m12 - m02 * m11;
  const float c11 = m00 * m22 - m02 * m02, c12 = m01 * m02 - m00 * m12, c22 = m00 * m11 - m01 * m01;
  const float inv_det = 1.0f / (m00 * c00 + m01 * c01 + m02 * c02);
  float nx = (c00 * rx + c01 * ry + c02 * rz) * inv_det;
  float ny = (c01 * rx + c11 * ry + c12 * rz) * inv_det;
  float nz = (c02 * rx + c12 * ry + c22 * rz) * inv_det;
  const double hdt = 0.5 * (double)p.dt;
  double x = st.x[t] + (double)(v.x + nx) * hdt, y = st.y[t] + (double)(v.y + ny) * hdt,
         z = st.z[t] + (double)(v.z + nz) * hdt;
  float resting = 0.0f;
  if (p.hf) {
    // terrain contact as a constraint that can only remove kinetic energy (terrain_resolve, :425-452)
    const float3 s = terrain_surface(p, (float)x, (float)z);
    const float pen = fsub(s.x, fsub((float)y, r_self));
    if (pen > 0.0f) {
      const float3 nn = terrain_normal(s);
      const float vn = nx * nn.x + ny * nn.y + nz * nn.z;
      float jn = 0.0f;
      if (vn < 0.0f) {
        jn = -vn;
        nx += jn * nn.x;
        ny += jn * nn.y;
        nz += jn * nn.z;
      }
      const float vd = nx * nn.x + ny * nn.y + nz * nn.z;
      const float tx = nx - vd * nn.x, ty = ny - vd * nn.y, tz = nz - vd * nn.z;
      const float vt = sqrtf(tx * tx + ty * ty + tz * tz);
      if (vt > 1.0e-9f) {
        const float dv = fminf(p.friction * jn, vt);
        nx -= (tx / vt) * dv;
        ny -= (ty / vt) * dv;
        nz -= (tz / vt) * dv;
      }
      const float dp = fminf(fminf(pen, kMaxSurfaceCorrection), f.w);
      x += (double)(dp * nn.x);
      y += (double)(dp * nn.y);
      z += (double)(dp * nn.z);
    }
    // grounded substeps (the settle counter, :565-573)
    const float fy = (float)y;
    resting = fsub(fy, r_self) <= fadd(terrain_surface(p, (float)x, (float)z).x, 0.1f)
                  ? __uint_as_float(st.prov[t]) + 1.0f : 0.0f;
  }
  st.prov[t] = __float_as_uint(resting);
  st.x[t] = x;
  st.y[t] = y;
  st.z[t] = z;
  float4 ph = st.pos_h[t];
  ph.x = (float)x;
  ph.y = (float)y;
  ph.z = (float)z;
  st.pos_h[t] = ph;
  v.x = nx;
  v.y = ny;
  v.z = nz;
  st.vel_u[t] = v;
}

int launch_dem_load(const Dev& d, const void* grains, cudaStream_t s) {
  k_dem_load<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, static_cast<const G80*>(grains), d.st[d.cur]);
  return 1;
}
int launch_dem_store(const Dev& d, const DemParams& p, bool stepped, void* grains, cudaStream_t s) {
  k_dem_store<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, d.s(), p, stepped ? 1 : 0, static_cast<G80*>(grains));
  return 1;
}
int launch_dem_contacts(const Dev& d, const DemParams& p, float4* acc, cudaStream_t s) {
  k_dem_contacts<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, d.s(), d.nbr, d.nbr_cnt, d.nbr_cap, p, acc);
  return 1;
}
int launch_dem_integrate(const Dev& d, const DemParams& p, const float4* acc, cudaStream_t s) {
  k_dem_integrate<<<(d.n + 255) / 256, 256, 0, s>>>(d.n, d.s(), acc, p);
  return 1;
}

}  // namespace sphb
