/*
 * sphgpu.h -- C ABI of the B200 (sm_100a) SPH particle hot path.
 *
 * One handle = one SPH scene resident in GPU memory (fluid phases + static
 * boundary particles), driven through the reference's solver step
 * semantics.  Plain pointers and sizes only; caller arrays are borrowed for
 * the duration of a call and never retained.  All functions return 0 on
 * success or a negative SPHGPU_E* code; sphgpu_last_error() gives the text.
 *
 * Reference interfaces this replaces (Artemisaturn/GRAPHICS, Source/):
 *   SphBase::runOneStep / sphStep         SphBase.h:395,411; SphBase.cpp:348-354
 *   DFSPH::sphStep                         DFSPH.h:35;  DFSPH.cpp:9-75
 *   WcSph::sphStep                         WcSph.h:50;  WcSph.cpp:23-96
 *   PciSph::sphStep                        PciSph.h:39; PciSph.cpp:31-94
 *   IISph_M::sphStep                       IISph_M.h:35; IISph_M.cpp:10-75
 *   IISph::sphStep (volume form)           IISph.h:35;   IISph.cpp:14-99
 *   SphBase::neighbourSearch               SphBase.h:673; SphBase.cpp:849-960
 *   m_Fluids / m_Solids particle arrays    SphBase.h:650-651, getters :513-541
 *   m_TH thresholds                        SphBase.h:546-583
 *   m_EC error counters                    SphBase.h:586-592
 */
#ifndef SPHGPU_H_
#define SPHGPU_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPHGPU_ABI_VERSION 3

/* error codes */
#define SPHGPU_OK 0
#define SPHGPU_EINVAL (-1)              /* bad argument / state */
#define SPHGPU_ENOMEM (-2)              /* device allocation failed */
#define SPHGPU_ECUDA (-3)               /* CUDA runtime error */
#define SPHGPU_EMAXITER (-4)            /* a solver loop hit its iteration cap */
#define SPHGPU_ENAN (-5)                /* non-finite particle state */
#define SPHGPU_ENEIGHBOUR_OVERFLOW (-6) /* a particle had more neighbours than the cap */
#define SPHGPU_EOUT_OF_DOMAIN (-7)      /* particles left [spaceMin, spaceMax] and were removed */
#define SPHGPU_ENOTIMPL (-8)

/* solvers (reference classes) */
#define SPHGPU_WCSPH 0   /* WcSph   */
#define SPHGPU_PCISPH 1  /* PciSph  */
#define SPHGPU_IISPH_M 2 /* IISph_M */
#define SPHGPU_DFSPH 3   /* DFSPH   */
#define SPHGPU_IISPH 4   /* IISph: divergence-free + constant-volume loops, per-pair h */

/* step status bits (SphStepStats.status) */
#define SPHGPU_STATUS_MAXITER_DENSITY 1u
#define SPHGPU_STATUS_MAXITER_DIVERGENCE 2u
#define SPHGPU_STATUS_NAN 4u
#define SPHGPU_STATUS_NEIGHBOUR_OVERFLOW 8u
#define SPHGPU_STATUS_OUT_OF_DOMAIN 16u
#define SPHGPU_STATUS_ZERO_DISTANCE 32u
#define SPHGPU_STATUS_SOLID_OUTSIDE 64u  /* a dynamic solid's particle left the grid */

typedef struct sphgpu_scene* sphgpu_t;

/* Scene parameters: the m_TH fields the hot path reads (SphBase.h:546-583),
 * plus the solver controls the reference hard-codes. */
typedef struct SphParams {
    float spacing_r;       /* m_TH.spacing_r: particle mass = rho0 * spacing_r^3 */
    float smoothRadius_h;  /* m_TH.smoothRadius_h: kernel support; ker h = /2 */
    float particle_d;      /* FluidParticle::d / BoundaryParticle::d (all particles) */
    float dt;              /* m_TH.dt (fixed step; initial step when cfl != 0) */
    float gravity[3];      /* m_TH.gravity_g */
    float spaceMin[3];     /* m_TH.spaceMin */
    float spaceMax[3];     /* m_TH.spaceMax */
    float soundSpeed_cs;   /* m_TH.soundSpeed_cs */
    float nu;              /* m_TH.nu: DFSPH / IISPH_M viscosity */
    float densityErro_eta; /* m_TH.densityErro_eta (PCISPH) */
    float boundary_visc;   /* SphSolid::viscosity_alpha of the walls */
    int max_neighbours;    /* NeigbStr::maxNeigbNum, reference 48 (<= 128) */
    /* DFSPH controls (reference values in brackets) */
    double df_density_goal;    /* mean (rho_adv/rho0 - 1) goal [1e-4, DFSPH.cpp:225] */
    int df_density_min_iter;   /* [2, DFSPH.cpp:229] */
    int df_density_max_iter;   /* [none in the reference] */
    double df_div_goal_abs;    /* >0: absolute mean Drho/Dt goal [2.5, DFSPH.cpp:762] */
    double df_div_goal_rel;    /* used if abs <= 0: mean(Drho/Dt)*dt/rho0 */
    int df_div_min_iter;       /* [1, DFSPH.cpp:765] */
    int df_div_max_iter;       /* loop breaks when it > this [30, DFSPH.cpp:764,772] */
    /* adaptive time step (not in the reference): dt = cfl*d/max|v| in FP64 */
    int cfl;
    float cfl_factor, dt_max, dt_min;
    /* WCSPH */
    float wc_gamma;            /* Tait exponent [7, WcSph.h:34] */
    /* PCISPH (PciSph.h:35, PciSph.cpp:114-123) */
    int pci_min_iter, pci_max_iter;
    /* IISPH_M (IISph_M.cpp:280-358) */
    float ii_omega;            /* relaxation [0.5] */
    float ii_eta_rel;          /* relative avg density error [0.001] */
    int ii_min_iter, ii_max_iter;
    /* learned warm start for the DFSPH density solve (0 = plain method) */
    int warm_start;
    /* fraction of the predicted stiffness applied before the loop: the loop
     * only pushes particles apart (rho_adv >= rho0 clamp, DFSPH.cpp:620-623),
     * so an over-prediction cannot be undone and is kept below 1 */
    float ws_scale;
    /* IISPH_M reproductions of the reference's loop bookkeeping (0 = the
     * method as published; bits may be combined):
     *   1  running error sums never reset between iterations, and the
     *      two-iteration minimum counted in particle updates
     *      (IISph_M.cpp:283-284, 350)
     *   2  velocity update v += a_p dt without the advection acceleration,
     *      as updateFluids built with -DIISPH does (SphBase.cpp:387-389);
     *      otherwise v = v_adv + a_p dt */
    int ii_compat;
    /* IISph, volume form (IISph.cpp): kinematic viscosity of fluid and of
     * boundary particles [0.1, FluidParticle / BoundaryParticle::
     * kinematicViscosity, SphBase.h:100,181]; constant-volume loop: goal on
     * the mean relative volume error, min / max iterations [1e-4, 3, 100,
     * IISph.cpp:550-555]; divergence-free loop: goal on mean(div) * dt,
     * min / max [1e-3, 2, 50, IISph.cpp:1223-1227].  A loop stops once its
     * iteration count exceeds max (the reference breaks when it > max). */
    float iv_kvisc, iv_kvisc_b;
    float iv_cv_goal, iv_div_goal;
    int iv_cv_min_iter, iv_cv_max_iter, iv_div_min_iter, iv_div_max_iter;
    /* DFSPH vorticity options, m_TH.enable_vortex (DFSPH.cpp:233-553,
     * 913-1022): 0 off; 1 TRRV (vorticity, its transport dOmega, velocity
     * refined through a Rankine vortex with weight vort_alpha = m_TH.alpha);
     * 2 micropolar (angular velocity carried per particle, m_TH.zeta,
     * m_TH.nu_t); 3 stream-function correction (vorticity lost over the step
     * put back through a stream function).  Single fluid phase. */
    int enable_vortex;
    float vort_alpha, vort_zeta, vort_nu_t;
    /* WCSPH surface tension and adhesion (WcSph.cpp:188-211, 300-311):
     * m_TH.h (the surface kernel's radius and the normal's scale), m_TH.r
     * (cohesion and curvature), m_TH.bt (adhesion); all 0 = the plain
     * method */
    float th_h, th_r, th_bt;
    int reserved[5];
} SphParams;

/* Per-step statistics (replaces m_EC and the CALL_TIME log rows). */
typedef struct SphStepStats {
    int n_fluid;                 /* active fluid particles after the step */
    int iter_density;            /* constant-density / pressure loop iterations
                                    (IISph: constant-volume, summed over phases) */
    int iter_divergence;         /* divergence-free loop iterations (IISph: summed over phases) */
    int removed;                 /* particles removed (outside the domain) */
    double err_density;          /* final FP64 error of the density loop (IISph: mean
                                    relative volume error, last phase) */
    double err_divergence;       /* final FP64 error of the divergence loop (IISph:
                                    mean divergence * dt, last phase) */
    double dt;                   /* step length used */
    uint32_t status;             /* SPHGPU_STATUS_* bits */
    int neighbour_overflow;      /* pairs dropped by the cap (m_EC.tooManyNeigb) */
    int zero_distance;           /* zero-distance pairs (m_EC.zeroDis) */
    int max_neighbours_seen;
    double mean_neighbours;
    int total_iter_density;      /* summed over the steps of this call */
    int total_iter_divergence;
    int steps;
    int reserved[5];
} SphStepStats;

int sphgpu_abi_version(void);

/* Reference-valued defaults (DFSPH/WcSph constructors, SphBase.cpp:210-225). */
int sphgpu_params_default(SphParams* p);

/* Scene lifetime.  device = CUDA ordinal; max_fluid = capacity of the fluid
 * arrays (particles can be added up to it). */
int sphgpu_create(const SphParams* p, int device, int max_fluid, sphgpu_t* out);
int sphgpu_destroy(sphgpu_t h);
int sphgpu_set_params(sphgpu_t h, const SphParams* p);

/* Static boundary particles (a static rigid SphSolid per solid_id, or one
 * solid if solid_id is NULL).  volume == NULL: compute the Akinci volume as
 * SphBase::prepareSolidPartWeight does (SphBase.cpp:766-813) before fluid is
 * present.  Replaces any previous boundary. */
int sphgpu_set_boundary(sphgpu_t h, int n, const float* xyz, const int* solid_id, const float* volume);

/* Append a fluid phase (SphWithIO::addFluidCuboid(newFluid=true)).  vel may be
 * NULL.  Returns the phase index (>= 0) or an error. */
int sphgpu_add_fluid(sphgpu_t h, int n, const float* xyz, const float* vel, float rho0, float visc_alpha);

/* Number of active fluid particles. */
int sphgpu_num_fluid(sphgpu_t h);

/* Advance nsteps steps of `solver`; blocks until done and fills *stats
 * (may be NULL).  Returns SPHGPU_EMAXITER / ENAN / ... after completing the
 * steps if the corresponding status bit was raised (the state is kept). */
int sphgpu_step(sphgpu_t h, int solver, int nsteps, SphStepStats* stats);

/* Same, but only enqueues the work on the scene's stream and returns; the
 * statistics of the last step become available after sphgpu_synchronize(). */
int sphgpu_step_async(sphgpu_t h, int solver, int nsteps);
int sphgpu_synchronize(sphgpu_t h, SphStepStats* stats);

/* Host-buffer round trip for one step (the drop-in path, where the host
 * arrays stay authoritative): upload xyz/vel (n*3 floats, reference order),
 * run one step, download positions and velocities into xyz_out/vel_out.
 * When the device state ended a DFSPH step (lists valid, no particle ever
 * removed), the upload is compared with it on the device: velocities are
 * taken as given, and the neighbour search runs again only if a position
 * differs -- handing back the previous output costs the transfers only.  In
 * that case, with graphs on, the positions the step's integration produces
 * are copied into xyz_out while its neighbour search and divergence loop
 * still run (pinned xyz_out makes the copy overlap; a step that removes
 * particles writes both outputs again afterwards).  With both outputs wanted,
 * graphs on, no vorticity option and no kappa-sum recording, the step is
 * speculative: its first part (forces, density loop, integrated positions)
 * runs on the device state while a second stream copies xyz/vel in and
 * compares them with that state bit for bit; the re-sorting second part
 * starts only if they are equal, otherwise the step runs again from the
 * uploaded state (same results either way; pinned xyz/vel make the upload
 * overlap; xyz_out may be xyz and vel_out vel). */
int sphgpu_step_host(sphgpu_t h, int solver, const float* xyz, const float* vel, float* xyz_out,
                     float* vel_out, SphStepStats* stats);

/* Fluid fields in reference order (phase by phase, each in insertion order).
 * field: "position","velocity" (n*3); "density","DFalpha","DFkappa",
 * "DFkappaV","density_adv","divergenceDeviation","presure" (n);
 * "vel_adv","acce_adv","acceleration" (n*3);
 * PCISPH: "pos_prediction","acce_pressure" (n*3);
 * IISPH_M: "dii","sum_dijpj","ii_vel_adv","acce_presure" (n*3),
 *          "aii","p_l","rho_adv" (n);
 * IISph: "advectionAcceleration","advectionVelocity","acce_presure" (n*3),
 *        "sphDensity","VF_gamma","VF_sphVolume","VF_alpha","VF_kappa",
 *        "VF_kappaV","VF_advectionVolume","VF_divergenceDeviation" (n);
 * learned warm start: "kappa_warm" (n), "ws_features" (n*16, the network's
 * normalised inputs of the last step);
 * DFSPH vorticity options (n*3): "omega", "dOmega" (TRRV), "angular_velocity"
 * (micropolar), "n0Vorticity", "deltaVorticity", "psi" (stream function);
 * "phase" (n, fluid phase index), "scene" (n, batch scene index).
 * Returns the count written.
 * set: "position","velocity","density" (the density the next PCISPH /
 * IISPH_M step's non-pressure forces read), "DFalpha". */
int sphgpu_get_fluid(sphgpu_t h, const char* field, float* out);
int sphgpu_set_fluid(sphgpu_t h, const char* field, const float* in);
/* Boundary fields in reference order (solid by solid): "position" (n*3),
 * "volume"; with a dynamic solid also "velocity" (n*3, the rigid velocity
 * updatePaticles gives), "force" (n*3, the last DFSPH step's boundary force)
 * and "kerSumFromSelf"; after an IISph step also "VF_gamma","VF_sphVolume",
 * "VF_alpha","VF_kappa","VF_kappaV","VF_advectionVolume",
 * "VF_divergenceDeviation". */
int sphgpu_get_boundary(sphgpu_t h, const char* field, float* out);

/* Particle output in the reference's .pos format (write_fluid_particles,
 * fUtility.h:254-303; Demo-Main.cpp:250-251 writes one file per phase and
 * frame): line 1 names the scene log file (log_name), line 2 the components,
 * line 3 the frame number and fluid index, line 4 the particle count, then
 * per particle of fluid phase `phase`, in the reference's order, the chosen
 * components as float32 in the reference's fixed component order: "position"
 * (3), "velocity" (3), "density" (1), "presure" (1), "acceleration" (3);
 * components = any of those words (NULL: "position", the reference's default
 * WRITE_PARTICLE_position).  Returns the particle count written. */
int sphgpu_write_pos(sphgpu_t h, const char* path, int phase, const char* components, const char* log_name);
/* read_fluid_particles (fUtility.h:486-510): the particle count of a .pos
 * file; with out != NULL also its records (max_floats = capacity of out in
 * floats), the component mask line (mask, mask_len) and the frame number.
 * Needs no GPU. */
long long sphgpu_read_pos(const char* path, float* out, long long max_floats, char* mask, int mask_len, int* frame);

/* Checkpoint / resume (no counterpart in the reference, whose restart is a
 * .pos re-import): save a single scene -- parameters, walls with their
 * volumes and solid ids, every fluid particle with the state the solvers
 * carry between steps (warm-start history, PCISPH / IISPH_M / IISph carried
 * values), frame and step length -- and load it into a new handle on
 * `device`.  Stepping the loaded handle continues the saved run bit for bit.
 * An attached warm-start network is not part of the snapshot. */
int sphgpu_save_snapshot(sphgpu_t h, const char* path);
int sphgpu_load_snapshot(const char* path, int device, sphgpu_t* out);

/* Dynamic rigid solids (DFSPH).  The reference couples rigid bodies to the
 * fluid through Bullet (SphWithBullet::updateSolids, SphWithBullet.cpp:
 * 180-224, called from DFSPH::sphStep, DFSPH.cpp:54): each step accumulates a
 * force on every boundary particle (DFSPH.cpp:681-691, 723-737, 1334-1359),
 * joins it per dynamic solid into a force and a torque about the centre of
 * mass (SphSolid::rigidForceJoin, SphBase.cpp:131-143), lets Bullet advance
 * the bodies, and moves the boundary particles with the new transforms
 * (SphSolid::updatePaticles, SphBase.cpp:95-128) before the neighbour
 * search.  Here the per-particle work runs on the device; the rigid-body
 * world stays with the caller and exchanges one force, torque and state per
 * solid and step. */

/* The state Bullet reports for a rigid body (SphSolid::updatePaticles,
 * SphWithBullet.cpp:302-317). */
typedef struct SphRigidState {
    float transform[16];       /* btTransform::getOpenGLMatrix: column-major, [12..14] = origin */
    float center_of_mass[3];   /* btRigidBody::getCenterOfMassPosition */
    float linear_velocity[3];
    float angular_velocity[3];
} SphRigidState;

/* The rigid-body world's step (applyCentralForce / applyTorque /
 * stepSimulation, SphWithBullet.cpp:185-210): called once per DFSPH step,
 * after the density loop and before the neighbour search, on the thread that
 * called sphgpu_step, with each dynamic solid's joined force and torque (3
 * FP64 values per solid; solids in the order they were made dynamic) and the
 * step length.  It advances the bodies and writes their new states into
 * states[0 .. nsolids-1], which hold the current ones on entry.  A nonzero
 * return makes the step call fail with SPHGPU_EINVAL once the step is done. */
typedef int (*sphgpu_rigid_fn)(void* user, int nsolids, const int* solid_ids, const double* force,
                               const double* torque, double dt, SphRigidState* states);

/* Make solid `solid_id` (as given to sphgpu_set_boundary) a dynamic rigid
 * body (SphSolid(dynamic = true, RIGIDBODY), SphBase.h:326-331): inner_xyz =
 * the body-frame positions of its particles (SphSolid::innerPositions), 3
 * floats per particle in the order set_boundary received them; state = its
 * initial state.  As SphWithBullet::addSolid does (SphWithBullet.cpp:
 * 101-136), the particles are placed at once and every boundary particle's
 * kerSumFromSelf and volume recomputed (prepareSolidPartWeight).  Single
 * scenes and the DFSPH solver. */
int sphgpu_set_solid_dynamic(sphgpu_t h, int solid_id, const float* inner_xyz, const SphRigidState* state);
/* fn = NULL removes the callback; the bodies then keep the state last set
 * with sphgpu_set_solid_state, which moves the particles at the next step's
 * updateSolids point (or the next "neighbourSearch" stage). */
int sphgpu_set_rigid_callback(sphgpu_t h, sphgpu_rigid_fn fn, void* user);
int sphgpu_set_solid_state(sphgpu_t h, int solid_id, const SphRigidState* state);
int sphgpu_get_solid_state(sphgpu_t h, int solid_id, SphRigidState* state);
/* rigidForceJoin of the last DFSPH step (or "DF_constantDensitySolverSecond"
 * stage): the solid's total force and its torque about the centre of mass of
 * its state at that step, summed in FP64. */
int sphgpu_get_solid_force(sphgpu_t h, int solid_id, double force[3], double torque[3]);

/* Surface reconstruction (the reference's surface_field and marchingCubes,
 * driven by its re.c: surface_setup, surface_aniso, marchingCubes).
 *
 * sphgpu_surface_create: surface_field::surface_setup(min, max, r_p, r_h,
 *   cell_size) (surface_field.cpp:8-41): the field grid spans
 *   [min - 0.75 r_h, max + 0.75 r_h] with nodes every cell_size; particles
 *   must lie in [min, max].
 * sphgpu_surface_field: surface_isotro (aniso = 0, surface_field.cpp:43-75)
 *   or surface_aniso (aniso = 1, :83-176) of n positions (3 floats each, host
 *   memory, or device memory when on_device != 0).  Nodes hold the sum over
 *   particles of det(G) W(|G (x - c)|) (W: the reference's cubic spline of
 *   radius r_h times r_p^3).  SPHGPU_EOUT_OF_DOMAIN if a particle lies
 *   outside the neighbour grid (the field is still computed).
 * sphgpu_surface_get_field / set_field: the grid (x fastest, then y, z;
 *   get_grid_min / get_grid_num / get_cell_size via sphgpu_surface_grid).
 * sphgpu_surface_mesh: marchingCubes(result, iso, field, grid_min, grid_num,
 *   cell) (marching_cubes.cpp:45-120): triangles of 9 floats (3 vertices)
 *   into out (capacity max_tris triangles; NULL to count), in cube order (z,
 *   y, x, x fastest); returns the triangle count.  ref_rows = 1 pairs the
 *   node rows as the reference's row caches do (cube y spans rows
 *   max(y-1, 0) and y, so its first row of cubes is flat and the mesh sits
 *   one cell higher along y) and accumulates the cube corners' coordinates
 *   as its loops do; ref_rows = 0 takes rows y and y + 1 and corners at
 *   min + i * cell.  The case table is this library's (sphgpu_mc_table): it
 *   cuts the same polygons out of every cube case as the reference's and
 *   may split them along other diagonals.
 * sphgpu_mc_table: that table (ntri[256]; tri[256 * 16] edge ids, -1 after
 *   the last triangle; cube numbering of marching_cubes.cpp:9-31).  Needs no
 *   GPU. */
typedef struct sphgpu_surface* sphgpu_surface_t;
int sphgpu_surface_create(const double* min3, const double* max3, double r_p, double r_h, double cell_size,
                          int device, sphgpu_surface_t* out);
int sphgpu_surface_destroy(sphgpu_surface_t s);
int sphgpu_surface_grid(sphgpu_surface_t s, double* min3, int* num3, double* cell);
int sphgpu_surface_field(sphgpu_surface_t s, int aniso, const float* xyz, int n, int on_device);
int sphgpu_surface_get_field(sphgpu_surface_t s, float* out);
int sphgpu_surface_set_field(sphgpu_surface_t s, const float* in);
long long sphgpu_surface_mesh(sphgpu_surface_t s, float iso, int ref_rows, float* out, long long max_tris);
void* sphgpu_surface_stream(sphgpu_surface_t s);
int sphgpu_surface_last_error(sphgpu_surface_t s, char* buf, int len);
/* Work counters (no reference counterpart): the (tile, particle) pairs of
 * the last field (each particle listed under every 8 x 16 x 16-node tile its
 * node box touches), the number of tiles, and this handle's kernel launches
 * so far.  Any pointer may be NULL. */
int sphgpu_surface_stats(sphgpu_surface_t s, long long* n_pairs, int* n_tiles, long long* kernels);
int sphgpu_mc_table(int* ntri, signed char* tri);

/* Stage-level entry points (parity tests run "given state S, call stage X"):
 *   "neighbourSearch"                 grid + neighbour lists (+ rho/alpha)
 *   "DF_constantDensitySolverFirst"   rho, alpha            (DFSPH.cpp:84-193)
 *   "DF_forceExceptPressure"          a_adv                 (DFSPH.cpp:1419-1475)
 *   "DF_constantDensitySolverSecond"  forces+density loop+integrate (:195-738)
 *   "DF_divergenceFreeSolver"         divergence loop       (:740-1024)
 *   "updateSolids"                    the rigid callback on the last forces
 *                                     (SphWithBullet.cpp:180-224)
 *   "wc_computePressure", "wc_computeForce"                 (WcSph.cpp:99-462)
 *   IISph: "VF_prepareAttribute" (neighbour lists of fluid and boundary
 *   particles, sphDensity, gamma, sphVolume, alpha; IISph.cpp:100-545),
 *   "advectionStep" (:1505-1570), "VF_divergenceFreeSolver" (:1219-1456),
 *   "VF_constantVolumeSolver" (:546-815), "iv_updateFluids"
 *   (SphBase.cpp:377-402 with -DIISPH)
 */
int sphgpu_stage(sphgpu_t h, const char* name, SphStepStats* stats);

/* Neighbour lists in the reference's encoding, per fluid particle in
 * reference order: counts[n]; t/idx[n*cap] = PartIdx (t<0: fluid phase -t-1,
 * t>0: solid t-1; i = index in that phase/solid), list order as
 * SphBase::neighbourSearch produces it.  Returns cap. */
int sphgpu_get_neighbours(sphgpu_t h, int* counts, int* t, int* idx);
/* Reference cell index (SpaceGridStruct::gridOfPos) per fluid particle. */
int sphgpu_get_cells(sphgpu_t h, long long* cell);

/* CUDA stream (cudaStream_t) of the scene. */
void* sphgpu_stream(sphgpu_t h);

/* Timing of the last sphgpu_step/step_async call measured with CUDA events on
 * the scene's stream: per-kernel-class accumulated milliseconds and launch
 * counts.  names/ms/launches arrays of length cap; returns entries written. */
int sphgpu_profile(sphgpu_t h, int enable);
int sphgpu_profile_read(sphgpu_t h, char* names, int name_len, double* ms, int* launches, int cap);

/* ---------------- learned warm start (no reference counterpart) ----------------
 * A BF16 MLP (16 -> 64 -> 64 -> 1, GELU; FP32 master weights) that predicts the
 * per-particle total stiffness kappa the DFSPH constant-density loop
 * (DFSPH.cpp:566-700) applies, applied once before the unmodified loop.  Parameter vector
 * (FP32, SPHGPU_MLP_NPARAM): W1[16][64] b1[64] W2[64][64] b2[64] W3[64] b3.
 * norm[34]: feature mean[16], 1/std[16], label mean, 1/std. */
#define SPHGPU_MLP_NPARAM 5313
typedef struct sphgpu_mlp* sphgpu_mlp_t;
int sphgpu_mlp_create(int device, int dataset_cap, uint64_t seed, sphgpu_mlp_t* out);
int sphgpu_mlp_destroy(sphgpu_mlp_t m);
int sphgpu_mlp_set_params(sphgpu_mlp_t m, const float* params);
int sphgpu_mlp_get_params(sphgpu_mlp_t m, float* params);
int sphgpu_mlp_set_norm(sphgpu_mlp_t m, const float* norm);
int sphgpu_mlp_get_norm(sphgpu_mlp_t m, float* norm);
int sphgpu_mlp_dataset_size(sphgpu_mlp_t m);
int sphgpu_mlp_dataset_set(sphgpu_mlp_t m, const float* X, const float* y, int n);
int sphgpu_mlp_dataset_get(sphgpu_mlp_t m, float* X, float* y, int max_n);
int sphgpu_mlp_dataset_shuffle(sphgpu_mlp_t m, uint64_t seed);
int sphgpu_mlp_train(sphgpu_mlp_t m, int epochs, int batch, float lr, float* loss_per_epoch);
int sphgpu_mlp_gradient(sphgpu_mlp_t m, const float* X, const float* y, int n, float* grad, float* loss);
int sphgpu_mlp_predict(sphgpu_mlp_t m, const float* X, float* y, int n);
/* mode 0: detach; 1: apply the warm start every DFSPH step; 2: record
 * (features, converged stiffness) of every record_every-th particle into the
 * network's dataset (plain solver, no warm start); 3: the classic warm start
 * (previous step's stiffness, no network) for comparison. */
int sphgpu_attach_warm_start(sphgpu_t h, sphgpu_mlp_t m, int mode, int record_every);

/* Copy of the last error message. */
int sphgpu_last_error(sphgpu_t h, char* buf, int len);

/* Autotuner (no reference counterpart): times the DFSPH step kernels at 64,
 * 128 and 256 threads per block on this scene (steps_per_candidate real
 * steps per candidate; the scene advances by 3x that) and keeps the fastest
 * block size per kernel class (forces, sweep A, sweep B, neighbour build).
 * report (may be NULL) receives a JSON summary of the timings. */
int sphgpu_autotune(sphgpu_t h, int solver, int steps_per_candidate, char* report, int report_len);

/* ---------------- batch of independent scenes (no reference counterpart) ----------------
 * Many DFSPH scenes of uneven size in one handle: one set of arrays, one
 * neighbour search and one launch per sweep for all of them, each scene with
 * its own box and grid, its own CFL step and its own loop convergence (a
 * converged scene stops iterating while the others continue).  All scenes
 * share the SphParams (kernel, rest density, goals); space_min/space_max
 * give each scene's box (3 floats per scene).  The handle is used with the
 * ordinary calls (sphgpu_step, sphgpu_get_fluid, ...); fluid is returned
 * scene by scene (see sphgpu_batch_scene_range).  Plain DFSPH only. */
int sphgpu_batch_create(const SphParams* p, int nscenes, const float* space_min, const float* space_max, int device,
                        int max_fluid, sphgpu_t* out);
int sphgpu_batch_num_scenes(sphgpu_t h);
/* walls of every scene: scene[i] = scene index of boundary particle i */
int sphgpu_batch_set_boundary(sphgpu_t h, int n, const float* xyz, const int* scene);
/* fluid particles with their scene indices (scenes in increasing order
 * across calls; one rest density and viscosity for the whole batch) */
int sphgpu_batch_add_fluid(sphgpu_t h, int n, const float* xyz, const float* vel, const int* scene, float rho0,
                           float visc_alpha);
/* per-scene statistics of the last step (iterations, errors, dt, status);
 * returns the number of scenes written (<= cap) */
int sphgpu_batch_stats(sphgpu_t h, SphStepStats* out, int cap);
/* the scene's particles are [first, first + count) of sphgpu_get_fluid's output */
int sphgpu_batch_scene_range(sphgpu_t h, int scene, int* first, int* count);

/* CFL time step from velocities that already live on the device, without
 * allocating anything (no counterpart in the reference, whose dt is fixed).
 * It is the in-step rule of sphgpu_step with cfl != 0:
 *   vmax = max |v| in FP64,  dt = clamp(cfl_factor * d / vmax, dt_min, dt_max)
 * (dt_max when vmax = 0), for callers that step their own particle arrays
 * and may not allocate device memory between steps: hosts that hand all
 * device memory to one pool up front, or run under a fixed memory budget.
 *   vel       device pointer to n records of `stride` floats (x, y, z first;
 *             stride >= 3, e.g. 4 for float4)
 *   dt_out    device pointer to one float, written with dt
 *   vmax_out  device pointer to one double (or NULL), written with vmax
 *   stream    cudaStream_t to run on (NULL: the legacy default stream)
 * The scratch is a file-scope device array of one FP64 partial per block of
 * 2048 velocities (32 KB) plus a ticket that is zero at load time and that
 * every call leaves at zero, so n is limited to SPHGPU_NOALLOC_MAX_N;
 * larger n is rejected with SPHGPU_EINVAL before any GPU work.  The first
 * call on a device (with that device current) looks up the scratch address
 * once (cudaGetSymbolAddress); make it before any stream capture.  The
 * address is kept for the life of the process: after cudaDeviceReset on a
 * device the library module is loaded anew and the kept address is stale,
 * so do not use this entry point on a device that has been reset.  All calls
 * on one device share the scratch: calls that overlap in time (other
 * streams, other threads) race on it and must be serialised by the caller.
 * A velocity with a non-finite component makes vmax and dt NaN (the step is
 * not silently computed from the other particles); n = 0 gives vmax = 0 and
 * dt = dt_max.  Launch errors are reported with cudaPeekAtLastError, so an
 * earlier error of other work is returned as SPHGPU_ECUDA but not cleared.
 * Returns 0, SPHGPU_EINVAL or SPHGPU_ECUDA. */
#define SPHGPU_NOALLOC_MAX_N 8388608
int sphgpu_cfl_dt_noalloc(const float* vel, int n, int stride, float cfl_factor, float d, float dt_max,
                          float dt_min, float* dt_out, double* vmax_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SPHGPU_H_ */
