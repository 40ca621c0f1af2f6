/* sph_b200.h — C ABI of the B200-native SPH giant-impact step.
 *
 * A drop-in for the Integrity engine's GPU SPH path (sean-reid/BotheadStudios, project integrity-engine).
 * The entry points replace the engine's `GpuSph` surface (crates/engine/src/gpu_sph.rs:742-922) and its
 * gravity host (crates/engine/src/gpu_gravity.rs:181-230, 532-607). Every function is `extern "C"`, takes
 * plain pointers and sizes, never throws and returns an sph_status. A context is owned by one thread at a
 * time (the reference's GpuSph is single-owner); each context has its own CUDA stream.
 *
 * Units are the caller's: the reference runs in SI with G = 6.674e-11; the configuration carries G and the
 * SI-valued guards of the reference shaders (density floor, sound-speed step floor, coincident-pair cut and
 * signal-speed floor) so that G = 1 code units behave the same way.
 */
#ifndef SPH_B200_H
#define SPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The 48-byte particle exchange layout: gpu_sph.rs:25-37 `SphParticle` == sph_step.wgsl:38 `Particle`. */
typedef struct SphParticle48 {
  float pos[3];
  float h;
  float vel[3];
  float u;
  float mass;
  uint32_t mat;
  float rho;
  uint32_t prov;
} SphParticle48;

/* The 48-byte material row: gpu_sph.rs:39-56 `SphEos` == sph_step.wgsl:43 `Eos` (Tillotson, SI). */
typedef struct SphEos48 {
  float rho0, a, b, cap_a;
  float cap_b, e0, e_iv, e_cv;
  float alpha, beta, _p0, _p1;
} SphEos48;

/* Status codes. No exception or abort crosses this boundary. */
typedef enum sph_status {
  SPH_OK = 0,
  SPH_CLAMPED = 1,          /* upload held more particles/materials than capacity: the excess was dropped */
  SPH_ERR_INVALID = -1,     /* bad argument (null pointer, size, material index, NaN input) */
  SPH_ERR_CUDA = -2,        /* a CUDA runtime call failed; see sph_last_error() */
  SPH_ERR_OOM = -3,         /* device allocation failed */
  SPH_ERR_TIMEOUT = -4,     /* sph_sync timed out, or a bounded device wait gave up */
  SPH_ERR_OVERFLOW = -5,    /* a device-side capacity was exceeded (neighbour list, traversal stack) */
  SPH_ERR_STATE = -6,       /* call out of order (e.g. stepping before upload) */
  SPH_NOT_READY = 2         /* readback in flight, not finished yet (sph_readback_take with ready=0) */
} sph_status;

enum { SPH_KERNEL_CUBIC = 0, SPH_KERNEL_WENDLAND_C2 = 1 };
enum { SPH_GRAVITY_TREE = 0, SPH_GRAVITY_DIRECT = 1, SPH_GRAVITY_NONE = 2 };
enum { SPH_MULTIPOLE_MONOPOLE = 0, SPH_MULTIPOLE_QUADRUPOLE = 1 };
enum { SPH_H_FIXED = 0, SPH_H_SOLVE = 1, SPH_H_LEARNED = 2 };
enum { SPH_PRECISION_F32 = 0, SPH_PRECISION_HILO = 1 };

/* Solver configuration. sph_config_default() fills the reference's values (SI, cubic spline, monopole
 * Barnes-Hut at θ = 0.5 with one particle per leaf, fixed h, α = 1, β = 2). */
typedef struct sph_config {
  double G;               /* gravitational constant in the caller's units */
  float theta;            /* Barnes-Hut opening angle; MAC: sqrt(d²+ε²) >= diag/θ + |centre-COM| */
  uint32_t leaf_size;     /* particles per LBVH leaf bucket (1..32) */
  uint32_t kernel;        /* SPH_KERNEL_* (support radius h in both) */
  uint32_t gravity;       /* SPH_GRAVITY_* */
  uint32_t multipole;     /* SPH_MULTIPOLE_* */
  uint32_t precision;     /* SPH_PRECISION_*: HILO = node-relative hi/lo coordinates + compensated sums */
  uint32_t h_mode;        /* SPH_H_*: FIXED keeps the uploaded h (the reference); SOLVE iterates h; LEARNED
                             checks the MLP's proposal and iterates only where it is rejected (sph_mlp_set) */
  float h_neighbours;     /* SOLVE: target neighbour count inside the support radius */
  float h_tol;            /* SOLVE: relative density residual that ends the iteration */
  uint32_t h_iters;       /* SOLVE: maximum Newton iterations per force evaluation */
  uint32_t max_neighbours;/* per-particle neighbour-list capacity */
  float cfl;              /* > 0: adaptive dt = cfl·min h/max(c+|v|, sig_floor) each step; 0: fixed dt */
  float rho_floor;        /* sph_step.wgsl:79  max(rho, 1e-9)   (SI value 1e-9) */
  float du_floor;         /* sph_step.wgsl:91  |u|·1e-3 + 1     (SI value 1)    */
  float r_min;            /* sph_step.wgsl:187 r > 1e-9         (SI value 1e-9) */
  float sig_floor;        /* sph_step.wgsl:268 max(c+|v|, 1)    (SI value 1)    */
  int32_t device;         /* CUDA device ordinal of the context; -1 = the calling thread's current device */
  uint32_t mac;           /* SPH_MAC_*: GROUP (default) or PARTICLE (the reference's per-particle walk) */
  uint32_t graph;         /* nonzero: sph_step_kdk captures its steady two-substep sequence once in a CUDA graph
                             and replays it (phase timing is not recorded for replayed substeps) */
  uint32_t block_threads; /* threads per block of the density, h-solve and force kernels: 64..1024, a multiple of
                             32; 0 = 256 */
  uint32_t walk_warps;    /* warps per block of the fused gravity + neighbour walk: 2, 4 or 8; 0 = 2 */
  float h_skin;           /* SOLVE/LEARNED: neighbour lists are built at h·(1 + h_skin) and h moves at most that far
                             per rebuild, once the previous solve converged (residual <= 10·h_tol); after an
                             upload or an unconverged solve the skin is 0.15. 0 = 0.05 (at most 0.5) */
  uint32_t walk_stack;    /* traversal-stack entries a walk may use (per warp in GROUP mode, 1,280 there; per
                             particle in PARTICLE mode, 64 there as in bh_gravity.wgsl:336); 0 = all of them. A
                             smaller limit is for testing the overflow path: children that do not fit are
                             skipped and SPH_ERR_OVERFLOW is raised through sph_diag (the reference drops them
                             silently, bh_gravity.wgsl:388-391) */
  float local_theta;      /* GROUP mode: an accepted node whose COM lies beyond r_g/local_theta of the group's
                             box centre (r_g: the box's half-diagonal) is not evaluated per particle but expanded
                             once about the centre (monopole to third, quadrupole to second order in the offset)
                             and the expansion is evaluated per particle; 0 = every accepted node per particle.
                             sph_config_default: 0.3 */
} sph_config;

/* Barnes-Hut acceptance. PARTICLE: each particle walks with the GPU reference's MAC
 * sqrt(d²+ε²) >= diag/θ + δ (bh_gravity.wgsl:382; diag = AABB diagonal, δ = |centre − COM|), reproducing
 * cs_gravity_bh bit for bit, and uses the reference's split for runs of equal Morton codes.
 * GROUP: a warp takes a group of <= 32 Morton-consecutive particles of one impact (whole leaves; split into
 * parts where consecutive particles are more than 6 h apart) and accepts a node only when
 * sqrt(d_box²+ε²) >= side/θ + δ holds for the nearest point of the part's bounding box, so it holds for
 * every particle of the part. θ here measures the node's largest side, as in the reference's CPU octree
 * (bhtree.rs:181, (2·half)/dist < θ), with Barnes' δ term added; at equal θ this is looser than the diagonal
 * form. Leaves may be accepted as multipoles. The same walk gathers the SPH neighbour candidates, and runs
 * of equal Morton codes are split on the index-extended key (always a valid tree). leaf_size must be a power
 * of two. */
enum { SPH_MAC_GROUP = 0, SPH_MAC_PARTICLE = 1 };

/* Diagnostics: FP64 device sums over the live particles (gpu_sph.rs:628-649 total_energy;
 * tools/impact-run/src/main.rs:528-536 angular momentum), plus device-side flags. */
typedef struct sph_diag_out {
  double kinetic, internal, potential;   /* ½ Σ m_i φ_i with φ from the tree gravity of the last evaluation
                                            (KDK steps leave φ out of their walks, as the reference's step
                                            does; sph_diag then sums it in one potential-only walk) */
  double momentum[3];
  double angular_momentum[3];            /* about the origin */
  double mass;
  double dt;                             /* the dt of the last step (adaptive or fixed; impact 0 of a batch) */
  double time;                           /* simulated time accumulated by sph_step_kdk (impact 0 of a batch) */
  uint32_t steps;
  uint32_t max_neighbours_seen;
  uint32_t overflow_flags;               /* bit0 neighbour list, bit1 traversal stack */
  uint32_t h_iterations;                 /* SOLVE: iterations used by the last force evaluation */
  float h_residual;                      /* SOLVE: max relative density residual after the last solve */
  uint32_t h_accepted;                   /* LEARNED: particles whose proposed h passed the first check (last
                                            solve) */
  /* cumulative tree-walk counters of the steps' walks (GROUP mode): nodes visited, 32-wide pops,
   * particle × multipole and particle × source-particle interactions */
  uint64_t walk_nodes, walk_pops, m2p_interactions, p2p_interactions;
  uint64_t local_expansions;             /* accepted nodes expanded about a group's centre (one per node and
                                            group part) */
  uint64_t p2p_slots;                    /* pairwise slots the lanes ran: p2p_interactions with every leaf
                                            counted as leaf_size sources (the padding of partial leaves) */
} sph_diag_out;

typedef struct sph_ctx sph_ctx;

/* Fill `cfg` with the reference's defaults. */
sph_status sph_config_default(sph_config* cfg);

/* GpuSph::new (gpu_sph.rs:767): allocate a context for up to `capacity` particles on the current device. */
sph_status sph_create(const sph_config* cfg, uint32_t capacity, sph_ctx** out);
void sph_destroy(sph_ctx* ctx);

/* GpuSph::upload (gpu_sph.rs:839-851): copy particles (AoS, host) and the material table in. Like the
 * reference's ParticleStore::replace it keeps the first `capacity` particles and the first 16 materials,
 * and then returns SPH_CLAMPED. A particle whose mat is outside the table is SPH_ERR_INVALID. The next step
 * rebuilds everything from the uploaded state. */
sph_status sph_upload(sph_ctx* ctx, const SphParticle48* particles, uint32_t n, const SphEos48* eos,
                      uint32_t n_eos, float softening);

/* Batched impacts. No counterpart in the reference: its offline driver runs impacts one after another
 * (tools/impact-run/src/main.rs:645-671). Uploads `n_impacts` independent impacts as one particle array,
 * impact k being particles [offsets[k], offsets[k+1]) with softening softening[k]. Every phase of a step
 * then runs as one launch over all impacts. Impacts never interact: each is quantised in its own box, sorted
 * into its own range and built into its own subtree, so its neighbours and gravity come from itself alone,
 * and each advances with its own adaptive dt (SPH_Q_IMPACT_DT). An impact gets the same result as a context
 * that holds it alone. Particles keep their batch index (readback order). Requires 1 <= n_impacts <=
 * SPH_MAX_IMPACTS, offsets[0] = 0, every impact non-empty, and offsets[n_impacts] <= capacity: an impact is
 * never clamped. sph_upload is the batch of one impact. */
#define SPH_MAX_IMPACTS 256
sph_status sph_upload_batch(sph_ctx* ctx, const SphParticle48* particles, const uint32_t* offsets,
                            uint32_t n_impacts, const SphEos48* eos, uint32_t n_eos, const float* softening);

/* GpuSph::set_dt (gpu_sph.rs:855-859) and set_av (:865-869); SphParams.omega (gpu_sph.rs:60-79). */
sph_status sph_set_dt(sph_ctx* ctx, double dt, float damp);
sph_status sph_set_av(sph_ctx* ctx, float alpha, float beta);
sph_status sph_set_omega(sph_ctx* ctx, float omega);

/* GpuSph::encode_kdk (gpu_sph.rs:901-908): enqueue `substeps` KDK leapfrog steps (two force evaluations
 * each, u clamped at 0) on the context's stream and return without waiting. */
sph_status sph_step_kdk(sph_ctx* ctx, uint32_t substeps);
/* GpuSph::encode_relax (gpu_sph.rs:893-898): enqueue damped relaxation steps (one evaluation each). */
sph_status sph_step_relax(sph_ctx* ctx, uint32_t steps);
/* One force evaluation on the current state without integrating (the verifier's run_gpu). */
sph_status sph_eval_forces(sph_ctx* ctx);

/* ParticleStore::begin_readback / take_readback (gpu_store.rs:126-213): a two-phase, non-blocking copy of
 * the live particles (AoS, original order) to host memory the caller owns. Only one readback is in
 * flight; take returns SPH_NOT_READY with *ready = 0 until it lands. */
sph_status sph_readback_begin(sph_ctx* ctx);
sph_status sph_readback_take(sph_ctx* ctx, SphParticle48* out, uint32_t cap, uint32_t* n_out, int* ready);

/* Blocking readback straight into caller memory (pinned memory gets a direct DMA): the live particles in
 * original order. Same data as begin/take, without the library's staging copy. */
sph_status sph_readback_into(sph_ctx* ctx, SphParticle48* out, uint32_t cap, uint32_t* n_out);

/* Wait for all enqueued work (timeout_ms = 0 waits without limit). */
sph_status sph_sync(sph_ctx* ctx, uint32_t timeout_ms);
uint32_t sph_count(const sph_ctx* ctx);
/* GpuSph::particle_buffer (gpu_sph.rs:876): a device buffer holding the live particles in the 48-byte
 * layout in original order, refreshed by this call (the headless stand-in for the render vertex buffer). */
sph_status sph_particle_buffer(sph_ctx* ctx, void** device_ptr);
sph_status sph_diag(sph_ctx* ctx, sph_diag_out* out);

/* ---- relaxed-body assembly (gpu_sph.rs:260-339) ------------------------------------------------------------
 * body_bulk (gpu_sph.rs:260-293): the centre of mass of the particles with provenance `prov`, the radius holding
 * 98 % of their mass about it, then twice again over the particles within 1.5 × that radius of that centre (so
 * the strays a relaxation leaves do not drag the centre); also the body's total mass. */
sph_status sph_body_bulk(sph_ctx* ctx, uint32_t prov, double centre[3], double* mass, double* radius);

/* BodyPlacement (gpu_sph.rs:297-302): where source body prov = k goes, its bulk velocity and angular velocity. */
typedef struct sph_placement {
  double offset[3];
  double vel[3];
  double spin[3];   /* ω (rad/s, any axis): v = vel + ω × (r − centre) */
} sph_placement;

/* assemble_from_relaxed_n (gpu_sph.rs:309-339) on the context's state (the relaxed bodies, typically after
 * sph_step_relax): each particle of prov k < n_placements is recentred on its body's bulk centre, moved to
 * placements[k].offset and given placements[k].vel + spin × (r − centre); particles of other provenance are
 * dropped; the rest of the record is kept. The result replaces the state as one impact (original order of the
 * kept particles, the material table kept) with the returned softening (a quarter of the smallest h); *dt is the
 * reference's shock-safe step 0.01 h_min / (20 km/s + the fastest placement speed), for sph_set_dt. At most 256
 * placements; SPH_ERR_INVALID when no particle is kept. */
sph_status sph_assemble(sph_ctx* ctx, const sph_placement* placements, uint32_t n_placements, float* softening,
                        float* dt);

/* ---- disk measurement and the Moon candidate of one impact ------------------------------------------------
 * Replaces the host measurement of a finished impact: variant 0 follows the impact-run tool
 * (tools/impact-run/src/main.rs:732-878, `measure` + `moon_candidate`), variant 1 the engine's statistics
 * (crates/engine/src/gpu_sph.rs:399-469 `disk_stats_json` + accretion.rs:73-160 `find_clumps`). The remnant
 * is the sphere about the centre of mass holding remnant_frac of the mass; each particle's two-body orbit
 * about it is escaping, remnant (periapsis inside) or disk; friends-of-friends over the disk with a linking
 * length of link_factor × the mean smoothing length (of the disk in variant 0, of every particle in variant
 * 1); the Moon candidate is the heaviest self-bound clump (internal KE + pairwise PE < 0, two or more
 * members) beyond the fluid Roche limit roche × R (ρ_remnant/ρ_clump)^(1/3). Provenance 0 is the target. */
typedef struct sph_measure_cfg {
  int32_t variant;         /* 0: the impact-run tool, 1: the engine's disk statistics */
  int32_t reserved;
  double G;                /* 0: the context's G */
  double remnant_frac;     /* 0.85 */
  double link_factor;      /* 2 */
  double roche;            /* 2.44 */
  double rho_fallback;     /* variant 0: clump density when its volume sum is zero (2700) */
  double pe_floor;         /* variant 0: pair distance floor of the self-potential (1 m) */
  double pe_softening;     /* variant 1: pair softening of the self-potential (1e4 m) */
} sph_measure_cfg;

typedef struct sph_disk_measure {
  double earth_frac;                          /* % of the disk mass from the target (prov 0) */
  double disk_mass, disk_target, disk_impactor;
  double remnant_target, remnant_impactor;
  double escaped_target, escaped_impactor;
  double r_remnant, m_remnant;
  double clump_mass;                          /* the Moon candidate, 0 when there is none */
  double clump_target_frac;                   /* % of the candidate's mass from the target */
  uint32_t clump_n;                           /* its particles */
  uint32_t n_clumps;                          /* disk groups of two or more particles */
  uint32_t n_bound;                           /* ... of which self-bound */
  uint32_t n_disk;                            /* disk particles */
} sph_disk_measure;

sph_status sph_measure_default(sph_measure_cfg* cfg);
/* Measures impact `impact` (0 for a single upload) of the current state. Synchronises the context's stream. */
sph_status sph_measure_disk(sph_ctx* ctx, uint32_t impact, const sph_measure_cfg* cfg, sph_disk_measure* out);
/* The context's CUDA stream (cudaStream_t), for callers that order their own work after the step. */
void* sph_stream(sph_ctx* ctx);
const char* sph_last_error(const sph_ctx* ctx);
const char* sph_status_string(sph_status s);

/* Inspection of one force evaluation's intermediates, for staged verification (the checks of
 * tools/gpu-bh-verify/src/main.rs and tools/sph-verify/src/main.rs). Sorted-space arrays come back in
 * Morton order; per-particle physical quantities come back in original particle order. */
enum {
  SPH_Q_BBOX = 0,        /* float[6·n_impacts] lo.xyz, hi.xyz of each impact (cs_bbox) */
  SPH_Q_CODES = 1,       /* uint32[n]  sorted Morton codes (each in its impact's box; impacts in order) */
  SPH_Q_ORDER = 2,       /* uint32[n]  original index at each sorted position (the sort permutation) */
  SPH_Q_LEFT = 3,        /* uint32[L-1] */
  SPH_Q_RIGHT = 4,       /* uint32[L-1] */
  SPH_Q_PARENT = 5,      /* uint32[2L-1] */
  SPH_Q_NODE_COM = 6,    /* float4[2L-1] com.xyz, mass */
  SPH_Q_NODE_BMIN = 7,   /* float4[2L-1] bmin.xyz, max h */
  SPH_Q_NODE_BMAX = 8,   /* float4[2L-1] bmax.xyz, opening radius size/θ+δ (size: largest side in GROUP mode,
                            diagonal in PARTICLE mode) */
  SPH_Q_NBR_COUNT = 9,   /* uint32[n]  neighbours of each particle (original order) */
  SPH_Q_NBR_LIST = 10,   /* uint32[n*max_neighbours] original indices, row i = particle i, unsorted */
  SPH_Q_RHO = 11,        /* float[n] */
  SPH_Q_PRESSURE = 12,   /* float[n] */
  SPH_Q_SOUND = 13,      /* float[n] */
  SPH_Q_ACC_SPH = 14,    /* float4[n]  SPH acceleration xyz, du/dt */
  SPH_Q_ACC_GRAV = 15,   /* float4[n]  gravity acceleration xyz, potential (filled in on demand, as sph_diag) */
  SPH_Q_H = 16,          /* float[n]   smoothing lengths */
  SPH_Q_N_LEAVES = 17,   /* uint32[1]  L */
  SPH_Q_IMPACT_DT = 18,  /* double[n_impacts] dt of each impact's last step */
  SPH_Q_IMPACT_TIME = 19 /* double[n_impacts] simulated time of each impact */
};
sph_status sph_inspect(sph_ctx* ctx, uint32_t what, void* host_out, size_t bytes);

/* Per-phase device timing (CUDA events recorded on the context's stream around each phase; the reference
 * has none: gpu_sph.rs:879 passes `timestamp_writes: None`) and the count of kernels the library launched. */
enum {
  SPH_PHASE_SORT = 0,        /* bbox, Morton keys, radix sort, state permutation */
  SPH_PHASE_TREE = 1,        /* Karras internal nodes + bottom-up moments */
  SPH_PHASE_GRAVITY = 2,     /* Barnes-Hut traversal or direct sum */
  SPH_PHASE_NEIGHBOURS = 3,  /* neighbour lists */
  SPH_PHASE_HSOLVE = 4,      /* smoothing-length iterations */
  SPH_PHASE_DENSITY = 5,     /* density + EOS */
  SPH_PHASE_FORCES = 6,      /* pressure + AV + du/dt (+ Courant signal) */
  SPH_PHASE_INTEGRATE = 7,   /* dt, kicks, drift, relaxation */
  SPH_PHASE_COUNT = 8
};
typedef struct sph_profile {
  double ms[SPH_PHASE_COUNT];
  uint64_t calls[SPH_PHASE_COUNT];
  uint64_t kernel_launches;  /* kernels launched since sph_profile_enable (counted whether or not timing is on) */
} sph_profile;
/* on != 0 starts recording phase events; any call resets the accumulators and the launch count. */
sph_status sph_profile_enable(sph_ctx* ctx, int on);
/* Waits for the stream, then reports the accumulated phase times since the last enable. */
sph_status sph_profile_read(sph_ctx* ctx, sph_profile* out);

/* GravityField::accelerations (gpu_gravity.rs:556) / cs_gravity_bh: softened self-gravity of a point set
 * through the LBVH (gravity = SPH_GRAVITY_TREE) or the direct sum, using the context's G, θ, leaf size and
 * multipole settings. Host arrays; acc3 receives the accelerations in input order. */
sph_status sph_gravity(sph_ctx* ctx, const double* pos3, const double* mass, uint32_t n, double softening,
                       uint32_t gravity_mode, double* acc3);

/* FP64 softened direct sum on a subset of targets against all n sources, on the device (the precision
 * oracle of the gravity tree). targets may be NULL (all particles). */
sph_status sph_gravity_direct64(sph_ctx* ctx, const double* pos3, const double* mass, uint32_t n,
                                const uint32_t* targets, uint32_t n_targets, double softening, double* acc3);

/* ---- Granular (DEM) contact: GpuParticles (crates/engine/src/gpu_particles.rs:46-325) over the grain
 * pipeline of shaders/particle_step.wgsl (contact_accel :167-211, cs_forces :273-336, the implicit velocity
 * solve of cs_integrate :477-530), plus the ground scene of cs_integrate :338-576 (terrain contact, air drag,
 * cooling: sph_dem_set_ground, sph_dem_set_terrain). The draw-only sub-cube expansion (cs_expand) is
 * rendering and is not part of this path. */
/* particle_step.wgsl:127-137 `Particle` (80 bytes). */
typedef struct SphGrain80 {
  float offset[3];
  float u;
  float vel[3];
  float resting;
  float color[3];
  float material;
  float emission[3];
  float rho;
  float radius;
  float _p0, _p1, _p2;
} SphGrain80;
/* The contact constants of GpuStepParams (particle_step.wgsl:1-25) this path uses: per-mass stiffness (1/s²),
 * normal damping (1/s), Coulomb μ, tangential damping (1/s), cohesion (1/s²), substep dt, gravity. */
typedef struct sph_dem_params {
  float gravity[3];
  float dt;
  float c_stiffness, c_normal_damp, c_friction, c_tangent_damp, c_cohesion;
  float reserved[3];
} sph_dem_params;
typedef struct sph_dem sph_dem;
/* GpuParticles::new (gpu_particles.rs:67). */
sph_status sph_dem_create(uint32_t capacity, int32_t device, sph_dem** out);
void sph_dem_destroy(sph_dem* dem);
/* GpuParticles::replace (:325): clamps to capacity (SPH_CLAMPED). */
sph_status sph_dem_replace(sph_dem* dem, const SphGrain80* grains, uint32_t n);
/* GpuParticles::set_params (:304). */
sph_status sph_dem_set_params(sph_dem* dem, const sph_dem_params* p);
/* The ground scene's medium and thermal constants (particle_step.wgsl:16-50 Params: center, air_rho,
 * drag_cd, specific_heat, cool_rate). All zero (the default) is vacuum without cooling. */
typedef struct sph_dem_ground {
  float center[3];       /* world.center(): centred coordinates + center = the heightfield's voxel coordinates */
  float air_rho;         /* kg/m³ (0 = vacuum: no drag) */
  float drag_cd;         /* drag coefficient */
  float specific_heat;   /* J/(kg K): u = c·T; grains cool toward c·300 K */
  float cool_rate;       /* 1/s */
  float reserved;
} sph_dem_ground;
sph_status sph_dem_set_ground(sph_dem* dem, const sph_dem_ground* g);
/* The terrain (binding 2 of particle_step.wgsl): a w × d heightfield of column tops in voxel units, row-major
 * heights[z·w + x]; copied to the device. w = d = 0 removes it. With a terrain, each substep resolves terrain
 * contact as the reference's non-injecting constraint (cs_integrate :477-576: into-surface velocity removed,
 * Coulomb friction bounded by μ·Jn, a velocity-free position projection capped at 1 cm and by the headroom to
 * the grain resting above) and counts grounded substeps in `resting`; without one, `resting` stays 0. */
sph_status sph_dem_set_terrain(sph_dem* dem, const int32_t* heights, uint32_t w, uint32_t d);
/* GpuParticles::dispatch (:255): `substeps` × (contact gather, implicit velocity solve, drift, then drag,
 * cooling and terrain contact as set above). */
sph_status sph_dem_step(sph_dem* dem, uint32_t substeps);
/* begin_readback/take_readback (:314-320), blocking: the grains in original order. */
sph_status sph_dem_readback(sph_dem* dem, SphGrain80* out, uint32_t cap, uint32_t* n_out);
/* The contact sums of the last substep (the reference's Accum: force.xyz, headroom, s_diag.xyz, 0,
 * s_off.xyz, 0, sv_nbr.xyz, 0 — 16 floats per grain, original order), for verification. */
sph_status sph_dem_contacts(sph_dem* dem, float* out16, size_t bytes);
uint32_t sph_dem_count(const sph_dem* dem);

/* Tree gravity of a point set that allocates no memory (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory at the point where they need forces: a real-time frame
 * loop, where cudaMalloc/cudaFree would synchronise the device and stall the frame, or a host engine that
 * reserves all device memory with its own allocator and hands a plug-in only the buffers it owns. The caller
 * passes DEVICE pointers: d_bodies4 = n float4 (x, y, z, mass), d_acc4 = n float4 output (acceleration xyz,
 * potential), in input order. The work is enqueued on `stream` (a cudaStream_t; NULL = the default stream)
 * on the calling thread's current device; the result is ready when that stream reaches this point.
 * Same walk as sph_gravity with SPH_MAC_GROUP (side-based θ, Barnes' δ, quadrupole if multipole = 1).
 * Limits: n <= 65536 and leaf_size in {8, 16, 32}; larger n returns SPH_ERR_INVALID. Both pointers must be
 * 16-byte aligned (SPH_ERR_INVALID otherwise). All scratch lives in one fixed array compiled into the library
 * (about 15 MB, held by every GPU that loads the library until the process exits). The first call in each
 * device context (and the first after a cudaDeviceReset) looks up that array's device address; make that
 * first call before any stream capture (a first call inside a capture returns SPH_ERR_STATE). Every call
 * uses the same array, so calls whose work overlaps on the GPU (different streams, or different host threads
 * on one device) race and corrupt each other's results: order them on one stream. If the traversal stack
 * (1,280 nodes per warp) overflows, every output is NaN. A CUDA error already pending on the calling thread
 * is left in place and returns SPH_ERR_CUDA before any work is enqueued. */
sph_status sph_gravity_tree_noalloc(const void* d_bodies4, uint32_t n, double G, float softening, float theta,
                                    uint32_t leaf_size, uint32_t multipole, void* d_acc4, void* stream);

/* ---- Learned smoothing lengths (no counterpart in the reference, which keeps h fixed: hydrostatic.rs:59-61).
 * A small MLP, 8 → 64 → 64 → 1 with GELU, proposes each particle's Δlog h for the coming step from its state
 * at the start of the drift: log(h/h(ρ)) with h(ρ) = η(m/ρ)^(1/3), log(ρ/ρ0), ∇·v·dt, neighbours / target,
 * log(1 + |a| h / c²), material, log(1 + u/E_iv) and the run's progress (sph_set_progress). In h_mode
 * SPH_H_LEARNED the proposal (limited to ±0.03 in log h) replaces h before the tree build; one pass then checks
 * every particle: it is accepted when its density residual |ρ − m(η/h)³|/ρ is within h_tol and the density
 * change one more Newton step would make is within h_tol/4; only the rejected particles take the Newton
 * iterations (at most h_iters). The network runs on the tensor cores with BF16 weights and activations
 * and FP32 accumulation. Parameter block (SPH_MLP_PARAMS floats): W1[8][64] b1[64] W2[64][64] b2[64] W3[64]
 * b3 (the SPH_MLP_TRAINABLE weights; W[i][o] by input row) then x_mean[8] x_scale[8] y_mean y_scale
 * (x' = (x − x_mean)·x_scale). The network's output y·y_scale + y_mean is log(h_next/h(ρ)); the proposal is
 * Δlog h = that − log(h/h(ρ)) (the first input), so the residual a previous solve left is undone whatever the
 * network learned. A new context holds the zero network (the proposal h(ρ)). */
#define SPH_MLP_PARAMS 4819
#define SPH_MLP_TRAINABLE 4801
sph_status sph_mlp_set(sph_ctx* ctx, const float* params, uint32_t count);
/* on != 0: every KDK step also keeps its 8 features per particle and the network's Δlog h (original order),
 * for sph_mlp_features; the training data of the learned h. */
sph_status sph_mlp_record(sph_ctx* ctx, int on);
/* The last recorded step: features[n][8] and dlogh[n] (either may be NULL), cap = rows the buffers hold. */
sph_status sph_mlp_features(sph_ctx* ctx, float* features, float* dlogh, uint32_t cap);
/* The fraction of the run completed (the eighth input); read by the device at each step. */
sph_status sph_set_progress(sph_ctx* ctx, float fraction);

/* The network on its own, on the calling thread's current device (host arrays, blocking). */
typedef struct sph_mlp_train_cfg {
  uint32_t epochs;        /* passes over the samples */
  uint32_t batch;         /* samples per Adam step */
  float lr, beta1, beta2, eps, weight_decay;
  uint32_t seed;          /* sample shuffling */
} sph_mlp_train_cfg;
/* Δlog h of feature rows x[n][8]. */
sph_status sph_mlp_forward(const float* params, const float* x, uint32_t n, float* out);
/* Mean squared error on the normalised targets (t − y_mean)/y_scale over all n rows and its gradient w.r.t.
 * the SPH_MLP_TRAINABLE weights (FP32 sums of the BF16 tensor-core products). */
sph_status sph_mlp_grad(const float* params, const float* x, const float* t, uint32_t n, float* grad,
                        float* loss);
/* Adam on minibatches of (x, t); params is updated in place (its normalisation entries are kept);
 * loss_per_epoch (may be NULL) receives each epoch's mean training loss. */
sph_status sph_mlp_train(float* params, const float* x, const float* t, uint32_t n, const sph_mlp_train_cfg* cfg,
                         float* loss_per_epoch);

#ifdef __cplusplus
}
#endif
#endif /* SPH_B200_H */
