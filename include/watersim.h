/*
 * watersim.h — C ABI of libwatersim.so, the B200 (sm_100a) implementation of
 * WaterSim's FLIP/MAC substep.
 *
 * The boundary replaces the FluidSolver object of the reference
 * (js/solver.js): its constructor options, public knobs, typed-array fields,
 * step()/_substep() drivers and interaction helpers. Each entry point below
 * names the reference interface it stands in for.
 *
 * Conventions
 *  - Every call returns a ws_status: 0 = OK, negative = error (and WS_BUSY,
 *    positive, from ws_step_async). The message of
 *    the last error on a handle is available from ws_last_error(). Nothing
 *    aborts or traps; device-side faults (NaN, index out of range, a bounded
 *    wait that ran out) are latched in a device status word and reported by
 *    the next call that synchronises.
 *  - Host pointers are owned by the caller and read or written only during
 *    the call. Device memory is owned by the handle.
 *  - One CUDA stream per handle (ws_get_stream); with the learned warm start
 *    on, the pressure stage forks the SOR list build onto a second, internal
 *    stream and joins it back before the solve, so all of a call's work is
 *    still ordered after earlier work on the handle's stream and before later
 *    work on it. Calls on one handle must be serialised by
 *    the caller (a frame started by ws_step_async holds the handle until it
 *    is collected; other calls meanwhile return WS_ERR_BUSY). There is no
 *    global mutable state, so different handles may be used from different
 *    threads.
 *  - Storage is float32 for particle and grid fields, uint8 for flags and
 *    cell types — the layouts of the reference's typed arrays.
 *  - Only the sphere-planet world (mode 'sphere' with voxel terrain) of the
 *    reference is implemented.
 */
#ifndef WATERSIM_H
#define WATERSIM_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t ws_status;
#define WS_OK            0
#define WS_ERR_INVALID  -1   /* bad argument or handle */
#define WS_ERR_CUDA     -2   /* a CUDA runtime call failed */
#define WS_ERR_NOMEM    -3   /* device or host allocation failed */
#define WS_ERR_STATE    -4   /* call out of order (e.g. no terrain yet) */
#define WS_ERR_DEVICE   -5   /* a kernel latched a fault (NaN, out of range) */
#define WS_ERR_TIMEOUT  -6   /* a bounded device-side wait ran out */
#define WS_ERR_RANGE    -7   /* size beyond a documented maximum */
#define WS_ERR_BUSY     -8   /* an asynchronous step (ws_step_async) is in flight on the handle */
#define WS_BUSY          1   /* ws_step_async: the previous frame is still running; nothing started */

typedef struct ws_handle ws_handle;

/* Grid and capacity — the FluidSolver constructor options nx, ny, nz, dx
 * (js/solver.js:45-53) plus the particle capacity (_allocParticles,
 * js/solver.js:218-231) and the CUDA device ordinal. */
typedef struct {
  int32_t nx, ny, nz;
  int32_t capacity;       /* particle capacity */
  double dx;
  double coreR;           /* opts.coreR (js/solver.js:81) */
  double bumpiness;       /* opts.bumpiness (js/solver.js:138) */
  double targetParticles; /* opts.targetParticles (js/solver.js:75) */
  uint32_t terrainSeed;   /* opts.terrainSeed (js/solver.js:137) */
  int32_t device;
} ws_config;

/* Public knobs of FluidSolver (js/solver.js:55-193), copied on every
 * ws_set_params. The last block selects solver strategy:
 *   sorRedBlack  must be 1 (red-black SOR is the device order);
 *   sorTol > 0   iterates to ||b - A q|| / ||b|| <= sorTol, FP64 residual
 *                checked every sorCheckEvery iterations, at most sorMaxIters;
 *                sorTol <= 0 runs pressureIters iterations like the reference;
 *   viscJacobi / extrapJacobi must be 1 (the device order of the two
 *                in-place passes of the reference);
 *   p2gCellOrder 1 scatters P2G over the particles sorted by cell (a
 *                counting sort by cell each substep, then one block per
 *                4^3 brick summing in shared memory and one atomic per
 *                touched face); 0 (default) in particle index order with
 *                one atomic per particle and face, faster on B200. */
typedef struct {
  int32_t substeps;
  int32_t pressureIters;
  double cfl, pic, gravity, viscosity, omega, maxSpeed;
  double vorticity, currents, shadeCool;
  double sunActivity, evapIntensity, atmosphereH;
  int32_t ceilReflect;     /* 0 'linear', 1 'quadratic', 2 'exponential' */
  int32_t hasSun;          /* sunPos != null */
  double sunPos[3];
  double heatK, Tamb, cloudT, cloudP, rainT, rainLiftAge, snowT, meltT;
  int32_t spinOn;
  int32_t thermalOn;       /* run the ~25 Hz thermal tick and frame passes in ws_step */
  int32_t sorRedBlack;
  int32_t sorCheckEvery;
  double sorTol;
  int32_t sorMaxIters;
  int32_t viscJacobi;
  int32_t extrapJacobi;
  int32_t p2gCellOrder;
} ws_params;

/* Scalar state and counters of FluidSolver (js/solver.js:81-214, RNG states
 * :151-153), plus solve diagnostics. */
typedef struct {
  double coreR, oceanR, spacing, particleVolume, iso, waterTopY;
  double umax, dtLast, simTime, gRamp, heatAcc;
  double targetParticles, landFrac, bumpiness;
  double sorRelRes;        /* FP64 relative residual after the last solve */
  uint32_t evS, cfS, bfS, stirS;
  uint32_t terrainSeed;
  int32_t nP, capacity;
  int32_t airborneCount, vaporCount, nightVaporCount, evapCount, substepsLast, nFluid;
  int32_t sorIters;        /* iterations run by the last solve */
  int32_t sorPath;         /* solve path of the last solve: 1 grid-wide colour lists, 2 cluster-resident
                              colour lists, 3 temporal-blocked on every SM (shared-memory regions),
                              4 owned bricks in global memory on every SM (regions too large) */
} ws_scalars;

/* Named fields — the typed arrays of FluidSolver (js/solver.js:94-129). */
typedef enum {
  WS_F_PX = 0, WS_F_PY, WS_F_PZ, WS_F_PVX, WS_F_PVY, WS_F_PVZ,      /* float32, capacity */
  WS_F_PT, WS_F_PAIR, WS_F_PLIGHT, WS_F_PWX, WS_F_PWY, WS_F_PWZ, WS_F_PPH,
  WS_F_PFLAG, WS_F_PCOOL, WS_F_PDEPTH,                               /* uint8, capacity */
  WS_F_CELLTYPE,                                                     /* uint8, nCells */
  WS_F_Q,                                                            /* float32, nCells (cellPhi == q) */
  WS_F_RHS,                                                          /* float32, nCells */
  WS_F_U, WS_F_V, WS_F_W,                                            /* float32, uN / vN / wN */
  WS_F_UO, WS_F_VO, WS_F_WO,                                         /* float32 snapshot */
  WS_F_UW, WS_F_VW, WS_F_WW,                                         /* float32 P2G weights */
  WS_F_VALIDU, WS_F_VALIDV, WS_F_VALIDW,                             /* uint8 */
  WS_F_DENS,                                                         /* float32, (nx+1)(ny+1)(nz+1) */
  WS_F_COUNT
} ws_field;

/* Terrain (the `terrain` object of generateTerrain, js/solver.js:499-504):
 * voxel rock mask and radius field on an n^3 lattice of spacing dv. */
typedef struct {
  int32_t n;
  double dv, Rsl, Rlo, Rhi, landFrac;
  const uint8_t* solid;    /* n^3 */
  const float* R;          /* n^3 */
} ws_terrain;

/* ---- lifetime: new FluidSolver(opts) (js/solver.js:45-216). The grid needs
 *      at least 4 cells along each axis, dx > 0 and capacity >= 1
 *      (WS_ERR_INVALID otherwise) and at most 2^29 cells (WS_ERR_RANGE); these
 *      are checked before any device call. Every entry point answers a NULL
 *      handle with WS_ERR_INVALID. */
ws_status ws_create(const ws_config* cfg, ws_handle** out);
ws_status ws_destroy(ws_handle* h);
const char* ws_last_error(const ws_handle* h);
const char* ws_version(void);

/* ---- knobs: assignments to the public fields (js/solver.js:55-193) */
ws_status ws_set_params(ws_handle* h, const ws_params* p);
ws_status ws_get_params(const ws_handle* h, ws_params* p);
ws_status ws_default_params(ws_params* p);
ws_status ws_set_scalars(ws_handle* h, const ws_scalars* s);
ws_status ws_get_scalars(ws_handle* h, ws_scalars* s);

/* ---- world setup: generateTerrain (js/solver.js:272-508) and
 *      resetWater/_resetWaterSphere (js/solver.js:611-731); terrain can also
 *      be supplied (the same `s.terrain` assignment the reference tests use) */
ws_status ws_generate_terrain(ws_handle* h, uint32_t seed, double seaLevel);
ws_status ws_upload_terrain(ws_handle* h, const ws_terrain* t);
ws_status ws_download_terrain(ws_handle* h, uint8_t* solid, float* R, double meta[4]);
ws_status ws_water_volume(ws_handle* h, double depth, double* volume);
ws_status ws_reset_water(ws_handle* h, double depth);

/* ---- field transfer: the typed arrays (js/solver.js:94-129). count is the
 *      element count to copy from element 0; ws_set_nparticles sets nP. */
ws_status ws_upload_field(ws_handle* h, ws_field f, const void* host, int64_t count);
ws_status ws_download_field(ws_handle* h, ws_field f, void* host, int64_t count);
ws_status ws_field_info(const ws_handle* h, ws_field f, int64_t* count, int32_t* elem_bytes);
ws_status ws_set_nparticles(ws_handle* h, int32_t nP);

/* ---- particle state in one call: the readback/upload GpuSim does around a
 *      frame (js/gpu/gpusim.js:568-650). field[f] is the host buffer of
 *      particle field f (WS_F_PX..WS_F_PDEPTH, element type as listed
 *      above) or NULL to skip it; count elements from element 0 move per
 *      field. Pinned buffers copy at full link speed.
 *      The fields no substep reads or writes (WS_F_PLIGHT, WS_F_PDEPTH,
 *      WS_F_PPH, and WS_F_PT while no vapour parcel can exist) move on a
 *      second stream beside the substeps: ws_upload_state returns once the
 *      other fields are on the device and keeps reading those buffers until
 *      the next call into the library other than ws_substep or
 *      ws_download_state, so the caller leaves them unchanged until then;
 *      ws_download_state copies them without waiting for the substeps when
 *      only substeps ran since the last upload or download, and returns
 *      with every buffer written. Every other entry point orders its work
 *      after these copies. */
#define WS_NUM_PARTICLE_FIELDS 16
typedef struct {
  int64_t count;
  void* field[WS_NUM_PARTICLE_FIELDS];
} ws_host_arrays;
ws_status ws_upload_state(ws_handle* h, const ws_host_arrays* a);
ws_status ws_download_state(ws_handle* h, const ws_host_arrays* a);

/* ---- surface mesh: MarchingTetrahedra.build (js/surface.js:66-177) of the
 *      current density field (run ws_stage(WS_STAGE_SPLAT) first) at iso, into a
 *      device buffer the handle owns: `vertices` vertices (a triangle per 3), each
 *      with a float position and a float unit normal (3 floats each), in the
 *      reference's emission order; volume is its FP64 signed-volume integral.
 *      ws_surface_device returns the device pointers (valid until the next
 *      ws_surface_mesh) for a consumer on the same GPU; ws_surface_download
 *      copies them to host buffers of at least `vertices` vertices. */
ws_status ws_surface_mesh(ws_handle* h, double iso, int64_t* vertices, double* volume);
ws_status ws_surface_download(ws_handle* h, float* pos, float* nrm, int64_t max_vertices);
ws_status ws_surface_device(ws_handle* h, const float** pos, const float** nrm, int64_t* vertices);

/* ---- metaball skin: Metaballs.build (js/surface.js:203-284). Every liquid
 *      particle adds the kernel (1 - d²/R²)² to the corners of an (m+1)³ lattice
 *      over the box, m = max(6, round(nx·detail)) (detail clamped to 0.5..1.6;
 *      NaN or <= 0 means 1), R = (1.6 + 2.2·tension)·spacing in lattice cells
 *      (tension clamped to 0..1, NaN means 0.5); the field is contoured at
 *      1.5·((1.6 + 2.2·tension)/1.6)^1.5 by the marching-tets mesher into a
 *      device buffer the handle owns (separate from the surface mesh). The
 *      field accumulates in FP64 and is stored as float. ws_metaball_field
 *      copies the last build's corner field (capacity >= (m+1)³ floats; NULL
 *      field returns m only). */
ws_status ws_metaball_mesh(ws_handle* h, double tension, double detail, int64_t* vertices, double* volume);
ws_status ws_metaball_download(ws_handle* h, float* pos, float* nrm, int64_t max_vertices);
ws_status ws_metaball_device(ws_handle* h, const float** pos, const float** nrm, int64_t* vertices);
ws_status ws_metaball_field(ws_handle* h, float* field, int64_t capacity, int32_t* m);

/* ---- render-side particle prep: WaterScene.updateParticles
 *      (js/scene.js:1595-1922) on the current particles. Each particle joins
 *      one draw class (0 liquid beads, 1 spray/rain, 2 vapour, 3 cloud,
 *      4 snow) or is culled, gets the scene's colour for it, and the draw list
 *      is sorted far to near (64 buckets of squared camera distance, stable,
 *      classes in the order above inside a bucket) into device buffers the
 *      handle owns: per point a float position (3), colour (3), alpha, size
 *      and sprite tile. counts[5] receives the class counts (the scene's
 *      _classCounts), *points their sum. The solver side (spacing, spinOn,
 *      the box centre) comes from the handle. ws_render_device returns the
 *      device pointers (valid until the next ws_render_particles);
 *      ws_render_download copies them to host buffers of max_points points
 *      (NULL skips an attribute). */
typedef struct ws_render_opts {
  int32_t show;           /* updateParticles' show argument */
  int32_t beadsMode;      /* liquid drawn as flat circles (setBeadsMode) */
  int32_t metaballMode;   /* liquid drawn by the metaball skin instead */
  int32_t spinColor;      /* colour = globally normalised spin velocity */
  int32_t cloudSprite;    /* cloudSpriteMode and its image loaded: tile 5, else 3 */
  int32_t planetLit;      /* day/night shading (scene oceanR > 0) */
  int32_t sortOn;         /* camera known: sort far to near */
  int32_t useLight;       /* solver exposure mirror present (else hemisphere) */
  int32_t useDepth;       /* solver depth mirror present (night-side bead cull) */
  int32_t useTemp;        /* temperature mirror present (else 0.32) */
  double waterOpa;        /* water-surface opacity (beads) */
  double pOpa;            /* spray/atmosphere opacity */
  double wScale;          /* world scale of vapour/cloud sprites (0 = 1) */
  double waterColor[3];   /* water hue, linear rgb */
  double sunDir[3];       /* unit sun direction, planet-local frame */
  double cam[3];          /* camera position, planet-local frame */
} ws_render_opts;
ws_status ws_render_particles(ws_handle* h, const ws_render_opts* o, int32_t counts[5], int64_t* points);
ws_status ws_render_download(ws_handle* h, float* pos, float* col, float* alpha, float* size, float* sprite,
                             int64_t max_points);
ws_status ws_render_device(ws_handle* h, const float** pos, const float** col, const float** alpha,
                           const float** size, const float** sprite, int64_t* points);

/* ---- snapshot / restore of the whole solver state (resume, or shipping
 *      state between processes). A versioned host blob: knobs, scalars and
 *      RNG streams, the particle fields (nP each), the pressure warm start q,
 *      the terrain and the balls; grid fields are rebuilt by the next substep. Call with
 *      buf == NULL to get the size. Restore needs a handle of the same grid
 *      and a capacity of at least the stored nP. No reference counterpart
 *      beyond the typed arrays themselves (js/solver.js:94-129). */
ws_status ws_snapshot(ws_handle* h, void* buf, int64_t capacity, int64_t* size);
ws_status ws_restore(ws_handle* h, const void* buf, int64_t size);

/* ---- balls: addBall (js/solver.js:3910-3912). Each ball is a rigid sphere
 *      coupled to the fluid every substep as the reference's _substep does
 *      (:2568-2624): rasterised as a moving solid whose cells carry its
 *      velocity (_rasterizeStatic :918-938, _applyBC :1153-1170), particles
 *      pushed out of it after _markFluidCells and after advection
 *      (_pushBallsChunk :1009-1026), then integrated (_updateBalls
 *      :2344-2564: waterline from the surrounding liquid, Archimedes cap,
 *      drag, added mass, terrain contact, domain shell, ball-ball contacts).
 *      resetWater drops them. ws_get_balls copies up to max balls and sets
 *      *count to the number held; ws_set_balls replaces the list (count 0
 *      clears it). At most WS_MAX_BALLS. */
#define WS_MAX_BALLS 64
typedef struct {
  double x, y, z, vx, vy, vz, r, rho, submerged;
} ws_ball;
ws_status ws_add_ball(ws_handle* h, double x, double y, double z, double r, double rho);
ws_status ws_get_balls(ws_handle* h, ws_ball* out, int32_t max, int32_t* count);
ws_status ws_set_balls(ws_handle* h, const ws_ball* in, int32_t count);

/* ---- drivers: step(dtFrame) == _stepSync (js/solver.js:2663-2700) and
 *      _substep(dt) (js/solver.js:2568-2624) */
ws_status ws_step(ws_handle* h, double dtFrame);

/* ---- asynchronous frame step: GpuSim.step's non-blocking contract
 *      (js/gpu/gpusim.js:328-339). ws_step_async starts ws_step(dtFrame) on a
 *      worker thread the handle owns and returns at once: WS_OK when the frame
 *      started, WS_BUSY (nothing started) while the previous frame still runs.
 *      ws_step_poll sets *done and, once done, returns the frame's status;
 *      ws_step_wait blocks until the frame ends and returns its status. While
 *      a frame is in flight every other call on the handle returns
 *      WS_ERR_BUSY; ws_destroy waits for the frame first. */
ws_status ws_step_async(ws_handle* h, double dtFrame);
ws_status ws_step_poll(ws_handle* h, int32_t* done);
ws_status ws_step_wait(ws_handle* h);
ws_status ws_substep(ws_handle* h, double dt);

/* ---- single stages, for tests (the private methods the reference tests
 *      call one at a time, test/phase.test.js, test/optimization.test.js).
 *      Stage ids follow the substep order. */
typedef enum {
  WS_STAGE_CLEAR_RASTER = 0,  /* u..wW.fill(0) + _rasterizeStatic      :2569-2572, :865 */
  WS_STAGE_MARK_FLUID,        /* _markFluidCells                        :945 */
  WS_STAGE_P2G,               /* _p2g + _p2gNormalizeFace + _applyBC + snapshot  :1030-1171, :2579 */
  WS_STAGE_FORCES,            /* _viscosity + _applyPlanetGravity + _applyBC     :1259, :2656, :1130 */
  WS_STAGE_PRESSURE,          /* _pressureSolve                         :1312 */
  WS_STAGE_PROJECT,           /* _project                               :1417 */
  WS_STAGE_VORTICITY,         /* _vorticityConfinement                  :1454 */
  WS_STAGE_CLAMP,             /* _clampUmSlice -> umax                  :2629 */
  WS_STAGE_EXTRAPOLATE,       /* _extrapolate                           :1562 */
  WS_STAGE_G2P_ADVECT,        /* _g2p + _advect                         :1639-2292 */
  WS_STAGE_HEAT,              /* _updateHeat                            :2715 */
  WS_STAGE_EVAPORATION,       /* _updateEvaporation                     :3008 */
  WS_STAGE_PHASE,             /* _updatePhaseChanges                    :3152 */
  WS_STAGE_PUSH_SURFACE,      /* _pushSurfaceParticles                  :3486 */
  WS_STAGE_SPLAT,             /* splatDensity                           :3785 */
  WS_STAGE_VAPOR_COLLISIONS,  /* _vaporCollisions                       :3345 */
  WS_STAGE_ICE_CONTACTS,      /* _iceContacts                           :3290 */
  WS_STAGE_CURRENTS,          /* _updateCurrents (uses the scalar simTime) :3658 */
  WS_STAGE_COUNT
} ws_stage_id;
ws_status ws_stage(ws_handle* h, int32_t stage, double dt);

/* ---- reductions (FP64 on the device) */
ws_status ws_residual(ws_handle* h, double* relres);               /* ||b-Aq||/||b|| over fluid cells */
ws_status ws_mt_volume(ws_handle* h, double iso, double* volume, int64_t* vertexCount);
                                                                    /* MarchingTetrahedra.build volume, js/surface.js:66-177 */
ws_status ws_autotune_iso(ws_handle* h, double* iso);              /* autotuneIso, js/solver.js:3838 */
ws_status ws_census(ws_handle* h, double fractions[3]);            /* earthCensus, js/main.js:176 */
ws_status ws_kinetic_energy(ws_handle* h, double* ke);             /* kineticEnergy, js/solver.js:3914 */

/* ---- interactions (js/solver.js:3852-3908) and the seeded Gaussian stir
 *      kick of the 128^3 planet workload (no reference counterpart) */
ws_status ws_apply_impulse_sphere(ws_handle* h, double cx, double cy, double cz, double R,
                                  double fx, double fy, double fz);
ws_status ws_stir_at(ws_handle* h, double cx, double cy, double cz, double vx, double vy,
                     double vz, double R, double dt);
ws_status ws_stir_gaussian(ws_handle* h, double sigma, double peak);
/* waveImpulse(dvx) (js/solver.js:3866-3892), sphere mode: a tide bulge in a
 * random direction, every particle on that side pushed radially by
 * dvx * pr^3 * (0.7 + 0.3 rnd) (pr the cosine to the bulge direction). The
 * reference draws from Math.random(); here the draws come from the seeded
 * stir stream (stirS): two for the direction, then draw p + 1 of the
 * following stream for particle p (every particle takes one), so the call is
 * reproducible; stirS advances by nP + 2 draws. */
ws_status ws_wave_impulse(ws_handle* h, double dvx);
/* dryLandFraction() (js/solver.js:3593-3623): the fraction of 1200
 * golden-angle rays whose rock surface stands above sea level with no fluid
 * cell on it, from the current cell types; 0 without terrain. */
ws_status ws_dry_land_fraction(ws_handle* h, double* fraction);
/* sampleVel(x, y, z) (js/solver.js:811-854) at n points: xyz holds n
 * (x, y, z) host doubles, uvw receives n (u, v, w) host doubles, the
 * trilinear MAC sample of the current face velocities. */
ws_status ws_sample_vel(ws_handle* h, const double* xyz, int64_t n, double* uvw);
/* terrainRadiusAt(x, y, z) (js/solver.js:512-535) at n points: the
 * trilinear terrain radius field (coreR without terrain), n host doubles. */
ws_status ws_terrain_radius_at(ws_handle* h, const double* xyz, int64_t n, double* radius);
/* oceanPoint(minDepth) (js/solver.js:591-608): a point over an ocean column
 * deeper than minDepth (0 -> 0.12), halfway between the terrain surface and
 * sea level; the deepest of 64 tries otherwise. Draws from the seeded stir
 * stream (two per try made) instead of Math.random(). WS_ERR_STATE without
 * terrain. xyz receives three host doubles. */
ws_status ws_ocean_point(ws_handle* h, double minDepth, double* xyz);

/* ---- timing / synchronisation helpers */
/* Times `reps` back-to-back launches of one kernel group on the handle's
 * stream with CUDA events and returns the mean duration of one launch in
 * microseconds. Runs on the current state (timing only; the state advances
 * as if the kernels ran). kernel: 0 one red-black SOR iteration (two
 * launches, reported per launch), 1 P2G scatter in particle index order (one
 * atomic per particle and face; the substep uses 12), 2 fused G2P + advection,
 * 3 faces pass 1 (normalise + BC + snapshot), 4 forces pass, 5 projection,
 * 6 one whole SOR solve of pressureIters iterations on the default path
 * (reported per solve), 7 the same solve on the colour-list path (cluster-
 * resident or grid-wide, whichever the lists fit; list build included),
 * 8..11 passes 3, 4, 5 and the extrapolation over the active-brick list of
 * the last substep, as a substep runs them, 12 P2G in cell order from scratch
 * (count per cell, prefix sum, particle ids scattered into cell order, per-
 * cell sums with one atomic per touched face; every brick visited), reported
 * per whole P2G. */
ws_status ws_time_kernel(ws_handle* h, int32_t kernel, int32_t reps, double* us_per_launch);
ws_status ws_synchronize(ws_handle* h);
/* Failure-detection check (no counterpart in the reference, whose solver
 * has no device waits): one device thread waits for a status word that
 * nothing ever sets, with the same bounded wait the pressure solve uses
 * between its CTAs, limited to `polls` polls (1..1e8; about 1 us each). The
 * wait runs out, latches the timeout bit, and the call returns
 * WS_ERR_TIMEOUT exactly as a timed-out solve reports it; the handle and
 * its CUDA context stay usable. */
ws_status ws_probe_wait(ws_handle* h, int64_t polls);
ws_status ws_get_stream(ws_handle* h, void** cuda_stream);
ws_status ws_launch_count(ws_handle* h, int64_t* launches);        /* kernels this handle launched */

/* ---- allocation-free FP64 residual (no counterpart in the reference)
 * For callers that cannot let a library allocate device memory: a host that
 * owns every GPU buffer through its own allocator, or a frame loop where a
 * cudaMalloc/cudaFree would synchronise the device. Needs no handle (creating
 * one allocates): computes ||b - A q||_2 / ||b||_2 over the interior fluid
 * cells of the caller's own device buffers q, rhs (float32, nx*ny*nz) and
 * cellType (uint8), with A, b the pressure system of _pressureSolve, and
 * writes the double to the caller's device pointer relres, on `stream`
 * (a cudaStream_t, or NULL). Calls no cudaMalloc/cudaFree: its scratch is a
 * fixed 128 KB device array in the library, so grids above 128^3 cells
 * (2,097,152) return WS_ERR_RANGE. All calls on a device share that array;
 * calls that overlap on the GPU race. Every call looks the array's address up
 * on the current device (cudaGetSymbolAddress, which allocates nothing), in
 * the runtime's current (primary) context, so a context re-created after
 * cudaDeviceReset is handled; the first call on a device also loads the
 * library's device code there and should come before any stream capture.
 * Each launch is checked through its own return code (WS_ERR_CUDA when one
 * fails); an earlier, unrelated error pending on the calling thread is
 * neither cleared nor reported as this call's. */
ws_status ws_residual_noalloc(int32_t nx, int32_t ny, int32_t nz, const float* q, const float* rhs,
                              const uint8_t* cellType, double* relres, void* stream);

/* ---- learned warm start of the pressure solve. No counterpart in the
 *      reference: its _pressureSolve (js/solver.js:1312-1410) starts SOR
 *      from the previous substep's q. A 3-level 3D U-Net (16/32/64
 *      channels, 3x3x3 convolutions, BF16 weights and activations, FP32
 *      accumulation on the tensor cores) maps the residual of the previous
 *      q, r0 = b - A q_prev scaled by its RMS sigma, and the cell types to
 *      the change of q over the solve; with the warm start on, every solve
 *      starts from q_prev + sigma * G * net(...) at fluid cells and SOR
 *      continues to the same tolerance, so the network only changes how
 *      many iterations the solve takes. Training pairs (input, converged
 *      q - q_prev) come from the plain solver's own solves. */
typedef struct {
  int32_t pairs_stored, pairs_capacity;  /* pairs recorded so far; ring size */
  int64_t train_steps;                   /* Adam steps taken */
  int64_t num_weights;                   /* FP32 parameters (weights, biases, head) */
  double gain;                           /* output scale G (0 until set) */
  double last_loss;                      /* mean loss of the last ws_unet_train call */
  int32_t enabled, collecting;
} ws_unet_info;
/* allocate the network on first use and (re)initialise its weights (He
 * normal from seed, zero biases) and Adam state; 3 levels (16/32/64) */
ws_status ws_unet_init(ws_handle* h, uint32_t seed);
/* the same with 3 or 4 levels (4: 16/32/64/128 channels, bottleneck at an
 * eighth of the grid); a depth different from the current network's
 * replaces it (its stored pairs included) */
ws_status ws_unet_init_levels(ws_handle* h, uint32_t seed, int32_t levels);
/* capacity > 0: record one pair per solve into a ring of that many pairs;
 * 0: stop recording (pairs are kept). A pair keeps the active 8x16x8
 * level-0 tiles only (9 bytes per voxel of those tiles): every tile fits
 * when the grid has at most 2048 tiles, else a slot holds 1.5x the active
 * tiles of the cell types at the first call, and a solve with more active
 * tiles than that is not recorded. */
ws_status ws_unet_collect(ws_handle* h, int32_t capacity);
/* on != 0: every solve starts from the network's prediction */
ws_status ws_unet_enable(ws_handle* h, int32_t on);
/* steps Adam steps (beta 0.9/0.999) of batch pairs drawn from the ring with
 * a seeded generator; mean squared error over fluid cells of the target
 * scaled by 1/G. The first call sets G to the RMS of the stored targets. */
ws_status ws_unet_train(ws_handle* h, int32_t steps, int32_t batch, double lr, uint32_t seed,
                        double* mean_loss);
ws_status ws_unet_get_info(ws_handle* h, ws_unet_info* out);
/* the FP32 parameters, flat: per layer W[cout][cin][27] then b[cout], in
 * the order e0a e0b e1a e1b ba bb d1a d1b d0a d0b, then head w[16], b */
ws_status ws_unet_get_weights(ws_handle* h, float* host, int64_t count);
ws_status ws_unet_set_weights(ws_handle* h, const float* host, int64_t count);
ws_status ws_unet_set_gain(ws_handle* h, double gain);
/* one stored pair: r0 / sigma (float), cell types (uint8), target
 * (q - q_prev) / sigma (float), each nx*ny*nz; any pointer may be NULL */
ws_status ws_unet_get_pair(ws_handle* h, int32_t idx, float* r0n, uint8_t* types, float* target);
ws_status ws_unet_put_pair(ws_handle* h, const float* r0n, const uint8_t* types, const float* target);
/* network output (before the gain) at every cell of pair idx, 0 outside
 * active tiles; and the loss gradient of one pair, flat like the weights */
ws_status ws_unet_forward_pair(ws_handle* h, int32_t idx, float* out);
ws_status ws_unet_grad_pair(ws_handle* h, int32_t idx, float* grads, double* loss);
/* after the forces stage: sets up the pressure system and returns the
 * relative residual of the previous q and of the predicted q (q is left
 * at the prediction) */
ws_status ws_unet_probe(ws_handle* h, double* relres_prev, double* relres_pred);
/* mean device time in ms of `what`: 0 the prediction (writes q), 1 one
 * training step of batch 1 at learning rate 0 */
ws_status ws_unet_time(ws_handle* h, int32_t what, int32_t reps, double* ms);
/* data-parallel training across processes (one per GPU): accumulate the
 * gradients of `samples` stored pairs drawn with `seed` (no update; returns
 * the loss summed over them), expose the FP32 gradient buffer (device
 * pointer, num_weights floats, owned by the handle) so the caller can sum it
 * over the ranks in place, then apply one Adam step with the summed
 * gradients divided by total_samples (the batch of all ranks). Ranks that
 * start from the same ws_unet_init seed and the same gain stay identical. */
ws_status ws_unet_accumulate(ws_handle* h, int32_t samples, uint32_t seed, double* loss_sum);
ws_status ws_unet_grads(ws_handle* h, void** device_ptr, int64_t* count);
ws_status ws_unet_apply(ws_handle* h, double lr, int32_t total_samples);
/* the network's FP32 weights, output gain and Adam state as a host blob
 * (buf == NULL: size query), and back (same layout; ws_unet_init first) */
ws_status ws_unet_save(ws_handle* h, void* buf, int64_t capacity, int64_t* size);
ws_status ws_unet_load(ws_handle* h, const void* buf, int64_t size);

#ifdef __cplusplus
}
#endif
#endif
