/*
 * ws_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of WaterSim's FluidSolver (js/solver.js, js/surface.js,
 * js/main.js earthCensus) used as the parity checker for the CUDA library.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it; the product library never links or calls it.
 *
 * Two builds come from one source:
 *   liboracle_js.so   storage float, arithmetic double — the JS semantics
 *                     (Float32Array storage, double arithmetic).
 *   liboracle_f64.so  storage double — the FP64 oracle the per-field error
 *                     reports are measured against.
 *
 * Parity status: the reference is JavaScript and no JS engine exists on
 * this machine, so no value of the oracle is checked against a live run of
 * solver.js ("parity unpinned" for raw numbers). The oracle is pinned to the
 * reference's own invariant and known-answer tests (test/optimization.test.js,
 * test/surface.test.js, test/phase.test.js, test/solver.test.js), ported in
 * tests/test_oracle_*.py.
 */
#ifndef WS_ORACLE_H
#define WS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Knobs: the public tunables of FluidSolver (js/solver.js:55-193) plus the
 * ordering switches that select the device-side order of the three
 * order-dependent passes. Field order matches ws_params in
 * include/watersim.h so one ctypes layout serves both. */
typedef struct {
  int32_t substeps;
  int32_t pressureIters;
  double cfl, pic, gravity, viscosity, omega, maxSpeed;
  double vorticity, currents, shadeCool;
  double sunActivity, evapIntensity, atmosphereH;
  int32_t ceilReflect;          /* 0 linear, 1 quadratic, 2 exponential */
  int32_t hasSun;
  double sunPos[3];
  double heatK, Tamb, cloudT, cloudP, rainT, rainLiftAge, snowT, meltT;
  int32_t spinOn;
  int32_t thermalOn;            /* runs the ~25 Hz thermal tick + phase passes in step() */
  /* pressure: 0 = lexicographic SOR (reference), 1 = red-black SOR */
  int32_t sorRedBlack;
  int32_t sorCheckEvery;        /* residual check cadence (iterations) in tolerance mode */
  double sorTol;                /* >0: iterate to relative residual <= sorTol */
  int32_t sorMaxIters;          /* cap in tolerance mode */
  int32_t viscJacobi;           /* 0 = in-place (reference), 1 = Jacobi */
  int32_t extrapJacobi;         /* 0 = in-place (reference), 1 = Jacobi */
  int32_t p2gCellOrder;         /* accepted, no effect: the oracle's P2G is one serial sum */
} or_params;

typedef struct {
  double coreR, oceanR, spacing, particleVolume, iso, waterTopY;
  double umax, dtLast, simTime, gRamp, heatAcc;
  double targetParticles, landFrac, bumpiness;
  double sorRelRes;             /* relative residual after the last solve (FP64) */
  uint32_t evS, cfS, bfS, stirS;
  uint32_t terrainSeed;
  int32_t nP, capacity;
  int32_t airborneCount, vaporCount, nightVaporCount, evapCount, substepsLast, nFluid;
  int32_t sorIters;             /* iterations run by the last solve */
  int32_t sorPath;              /* always 0 on the CPU */
} or_scalars;

typedef struct or_solver or_solver;

or_solver* or_create(int nx, int ny, int nz, double dx, double coreR,
                     uint32_t terrainSeed, double bumpiness, double targetParticles);
void   or_destroy(or_solver*);
int    or_storage_bytes(void);                 /* 4 (float) or 8 (double) */
void   or_get_params(const or_solver*, or_params*);
void   or_set_params(or_solver*, const or_params*);
void   or_get_scalars(const or_solver*, or_scalars*);
void   or_set_scalars(or_solver*, const or_scalars*);
/* Named array access: returns the pointer, writes element count and the
 * element kind (0 u8, 1 i32, 2 storage real, 3 f64). */
void*  or_array(or_solver*, const char* name, int64_t* count, int* kind);
int    or_alloc_particles(or_solver*, int cap);
/* terrain: generate (js/solver.js:272-508) or load an existing one */
void   or_generate_terrain(or_solver*, uint32_t seed, double seaLevel);
int    or_load_terrain(or_solver*, int n, double dv, const uint8_t* solid, const void* R,
                       double Rsl, double Rlo, double Rhi, double landFrac);
double or_water_volume_mc(or_solver*, double depth);
void   or_reset_water(or_solver*, double depth);
void   or_build_planet_gravity(or_solver*);

/* frame and substep drivers */
void   or_step(or_solver*, double dtFrame);
void   or_substep(or_solver*, double dt);

/* individual stages (same semantics as the JS methods) */
void   or_clear_faces(or_solver*);
void   or_rasterize_static(or_solver*);
void   or_mark_fluid(or_solver*);
void   or_p2g(or_solver*);
void   or_apply_bc(or_solver*);
void   or_snapshot_old(or_solver*);
void   or_viscosity(or_solver*, double dt);
void   or_planet_gravity(or_solver*, double dt);
void   or_pressure_solve(or_solver*);
double or_residual(or_solver*);                /* FP64 ||b-Aq||/||b|| over fluid cells */
void   or_project(or_solver*);
void   or_vorticity(or_solver*, double dt);
double or_clamp_um(or_solver*);
void   or_extrapolate(or_solver*);
void   or_g2p(or_solver*, double dt);
void   or_advect(or_solver*, double dt);
void   or_update_heat(or_solver*, double dt);
void   or_update_evaporation(or_solver*, double dt);
void   or_update_currents(or_solver*, double dt);
void   or_update_phase(or_solver*, double dt);
void   or_vapor_collisions(or_solver*);
void   or_ice_contacts(or_solver*);
void   or_push_surface(or_solver*);
void   or_splat_density(or_solver*);
double or_mt_volume(or_solver*, double iso, int64_t* triCount);
double or_autotune_iso(or_solver*);
void   or_census(or_solver*, double out[3]);   /* liquid, ice, vapour fractions */
double or_kinetic_energy(or_solver*);
double or_dry_land_fraction(or_solver*);
void   or_sample_vel(or_solver*, double x, double y, double z, double out[3]);
double or_sample_face(or_solver*, int comp, double x, double y, double z);
double or_terrain_radius_at(or_solver*, double x, double y, double z);
int    or_rock_cell_at(or_solver*, double x, double y, double z);
/* interactions (js/solver.js:3852-3908) and the seeded Gaussian stir */
void   or_apply_impulse_sphere(or_solver*, double cx, double cy, double cz, double R,
                               double fx, double fy, double fz);
void   or_stir_at(or_solver*, double cx, double cy, double cz, double vx, double vy,
                  double vz, double R, double dt);
void   or_stir_gaussian(or_solver*, double sigma, double peak);
void   or_wave_impulse(or_solver*, double dvx);
void   or_ocean_point(or_solver*, double minDepth, double out[3]);
/* standalone marching-tets volume over an external corner field (js/surface.js:66-177) */
double or_mt_volume_field(const void* dens, int nx, int ny, int nz, double dx, double iso,
                          int64_t* triCount);
/* the same build with the emitted vertices: pos and nrm hold 3 floats per
 * vertex (at most maxVerts vertices); returns the volume */
/* balls: each ball is 9 doubles x y z vx vy vz r rho submerged */
int or_add_ball(or_solver* s, double x, double y, double z, double r, double rho);
int or_get_balls(or_solver* s, double* out, int max);
int or_set_balls(or_solver* s, const double* in, int count);
void or_push_balls(or_solver* s);
void or_update_balls(or_solver* s, double dt);
double or_mt_mesh_field(const void* dens, int nx, int ny, int nz, double dx, double iso, float* pos, float* nrm,
                        int64_t maxVerts, int64_t* vertCount);
int or_metaball_field(int nP, const float* px, const float* py, const float* pz, const uint8_t* fl, int nx, double dx,
                      double spacing, double tension, double detail, float* field, double* mdx_out, double* iso_out,
                      double* R_out);

#ifdef __cplusplus
}
#endif
#endif
