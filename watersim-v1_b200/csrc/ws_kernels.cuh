// ws_kernels.cuh — kernel parameter blocks and launcher declarations.
#pragma once
#include "ws_internal.cuh"

struct AdvectParams {
  double dt, dtLast, pic, maxSpeed, gravity, oceanR, coreR, atmosphereH;
  double rainTe, rainLiftAge;
  double windS[3];
  int ceilReflect;
};

struct HeatParams {
  int hasSun;
  double sun[3];
  double sunActivity, Tamb, shadeCool, heatK, coreR;
};

struct PhaseParams {
  double cloudT, cloudP, rainT, snowT, meltT, rainLiftAge, cloudBase, dt;
  int spinOn;
  uint32_t tick;
};

// ---- ws_grid.cu
void launch_static_types(const Dims& d, const TerrainDev& t, double coreR, uint8_t* st, cudaStream_t s);
void launch_gravity_geometry(const Dims& d, double oceanR, float* g, cudaStream_t s);
void launch_clear_raster(const Dims& d, const GridDev& g, DevStatus* st, bool clearAcc, cudaStream_t s);
// the substep's face and cell passes over the active-brick list (ws_grid.cu)
cudaError_t launch_brick_activity(const BrickSet& B, cudaStream_t s);
void launch_clear_acc_bricks(const Dims& d, const GridDev& g, const BrickSet& B, cudaStream_t s);
void launch_faces_normalize_bc_bricks(const Dims& d, const GridDev& g, const BrickSet& B, cudaStream_t s);
void launch_faces_forces_bricks(const Dims& d, const GridDev& g, const BrickSet& B, double coef, int viscOn, double dt,
                                double gs, cudaStream_t s);
void launch_project_bricks(const Dims& d, const GridDev& g, const BrickSet& B, int doClamp, double maxSpeed,
                           DevStatus* st, cudaStream_t s);
void launch_extrapolate_bricks(const Dims& d, const GridDev& g, const BrickSet& B, cudaStream_t s);
void launch_pressure_setup_bricks(const Dims& d, const GridDev& g, uint8_t* diag8, double omega, DevStatus* st,
                                  const BrickSet& B, cudaStream_t s);
// cs: count every particle P2G will scatter in its cell (null: mark only)
void launch_mark_fluid(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t,
                       double oceanR, double coreR, const CellSort* cs, DevStatus* st, cudaStream_t s);
void launch_p2g(const Dims& d, const GridDev& g, const PartsDev& P, DevStatus* st, cudaStream_t s);
size_t cell_sort_scratch_bytes(long long nKeys);
int launch_p2g_sorted(const Dims& d, const GridDev& g, const PartsDev& P, const CellSort& cs, const BrickSet& B,
                      bool binned, void* scratch, size_t scratchBytes, DevStatus* st, cudaStream_t s);
void launch_faces_normalize_bc(const Dims& d, const GridDev& g, cudaStream_t s);
void launch_faces_forces(const Dims& d, const GridDev& g, double coef, int viscOn, double dt, double gs, cudaStream_t s);
void launch_pressure_setup(const Dims& d, const GridDev& g, uint8_t* diag8, double omega, DevStatus* st, int* sorCounts,
                           cudaStream_t s);
void launch_sor_color(const Dims& d, const GridDev& g, int color, double om1, cudaStream_t s);
int residual_blocks(const Dims& d);
void launch_residual(const Dims& d, const GridDev& g, const uint8_t* diag8, double2* partials,
                     DevStatus* st, double* hostMirror, cudaStream_t s);
void launch_project(const Dims& d, const GridDev& g, int doClamp, double maxSpeed, DevStatus* st, cudaStream_t s);
void launch_clamp_umax(const Dims& d, const GridDev& g, double maxSpeed, DevStatus* st, cudaStream_t s);
void launch_vorticity(const Dims& d, const GridDev& g, double eps, double dt, cudaStream_t s);
void launch_extrapolate(const Dims& d, const GridDev& g, cudaStream_t s);
void launch_extract_weight(const Dims& d, const float2* acc, float* out, long long off, long long n, cudaStream_t s);

// ---- ws_particles.cu
void launch_g2p_advect(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t,
                       const AdvectParams& ap, DevStatus* st, cudaStream_t s);
void launch_compact(const uint8_t* fl, int nP, int mode, int* blockCounts, int* out, int* total, cudaStream_t s);
void launch_vapor_advect(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t, const AdvectParams& ap,
                         const int* vIdx, const int* nV, uint32_t* rng, DevStatus* st, cudaStream_t s);
void launch_impulse_sphere(const PartsDev& P, double cx, double cy, double cz, double R, double fx, double fy, double fz, cudaStream_t s);
void launch_stir_at(const PartsDev& P, double cx, double cy, double cz, double vx, double vy, double vz, double R, double dt, cudaStream_t s);
void launch_stir_gaussian(const PartsDev& P, double pcx, double pcy, double pcz, double tx, double ty, double tz,
                          double sigma, double peak, cudaStream_t s);

// ---- ws_frame.cu
void launch_heat(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t, const HeatParams& hp,
                 double dt, int* cnt, double* sumT, double* change, cudaStream_t s);
// Evaporation (exact _evS stream): prepare (flags, compaction, thresholds) once,
// then passes over the candidates from t0 until no irregular kick is reported.
struct EvapScratch {
  long long* thr; uint32_t* b; int* ejP; uint32_t* ejS;
  double* wsum; int* L; int* Ew; unsigned short* table;
};
size_t evaporation_scratch_bytes(int capacity);   // <= contacts_scratch_bytes: the two share one buffer
EvapScratch evap_carve(void* base, int capacity);
void launch_evap_prepare(const Dims& d, const GridDev& g, const PartsDev& P, double freezeT, double rate, double dt,
                         uint8_t* cand, int* blockCounts, int* list, int* nC, const EvapScratch& es, cudaStream_t s);
void launch_evap_pass(int nP, const int* list, const int* nC, const EvapScratch& es, int t0, int eoff,
                      const uint32_t* sStart, DevStatus* st, cudaStream_t s);
void launch_evap_apply(const Dims& d, const GridDev& g, const PartsDev& P, double freezeT, const EvapScratch& es,
                       int nEj, cudaStream_t s);
uint32_t evap_kick_end(uint32_t s);
void launch_phase(const Dims& d, const GridDev& g, const PartsDev& P, const PhaseParams& pp, int* cnt, cudaStream_t s);
void launch_push_surface(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t,
                         double oceanR, double coreR, double atmosphereH, cudaStream_t s);
void launch_splat(const Dims& d, const GridDev& g, const PartsDev& P, double spacing, cudaStream_t s);
void launch_currents(const Dims& d, const PartsDev& P, const CurrField& F, double simTime, double strength,
                     double oceanR, double coreR, double dt, cudaStream_t s);
// scratch: mt_scratch_bytes(d.nCells) bytes (the straddling-cell list)
size_t mt_scratch_bytes(long long nCells);
void launch_mt_volume(const Dims& d, const float* dens, double iso, double2* partials, double* out, void* scratch,
                      cudaStream_t s);
// the marching-tets mesh after launch_mt_volume at the same iso and scratch
// (which leave the cell list and its per-chunk vertex counts): vertices in
// build order
void launch_mt_mesh(const Dims& d, const float* dens, double iso, const double2* partials, long long* offs,
                    long long maxVerts, float* pos, float* nrm, void* scratch, cudaStream_t s);
// render-side particle prep: classify, bucket-sort far to near, emit the
// draw list (ws_render.cu); counts land in the first five scratch words
// balls (ws_balls.cu): moving-solid raster (after the static raster),
// particle push-out, and the per-substep histogram + integration
void launch_ball_raster(const Dims& d, uint8_t* type, float* sv, bool clearSv, const double* balls, int nb,
                        const GridDev& g, cudaStream_t s);
void launch_ball_push(const PartsDev& P, const double* balls, int nb, cudaStream_t s);
void launch_ball_update(const Dims& d, const float* vel, const TerrainDev& t, const PartsDev& P, double* balls, int nb,
                        int* hist, float* surfY, const BallEnv& env, double dt, cudaStream_t s);
// Metaballs.build's corner field on an (m+1)^3 lattice of spacing mdx
// (FP64 accumulation, float result); 1 or 2 launches
void launch_metaball_field(const PartsDev& P, int m, double mdx, double R2, int rad, double* acc, float* field,
                           cudaStream_t s);
size_t render_scratch_bytes(long long capacity);
void launch_render_particles(const RenderCfg& c, const PartsDev& P, void* scratch, RenderOut o, cudaStream_t s);
void launch_particle_reduce(const PartsDev& P, int mode, double mp, double* partials, double* out, cudaStream_t s);

// ---- ws_queries.cu
void launch_wave_impulse(const Dims& d, const PartsDev& P, const double dir[3], uint32_t s0, double dvx, cudaStream_t s);
void launch_dry_land(const Dims& d, const TerrainDev& t, const uint8_t* type, double oceanR, int* dry, cudaStream_t s);
void launch_sample_vel(const Dims& d, const float* vel, const double* xyz, long long n, double* out, cudaStream_t s);
void launch_terrain_radius(const TerrainDev& t, double coreR, const double* xyz, long long n, double* out,
                           cudaStream_t s);
void launch_ocean_point(const Dims& d, const TerrainDev& t, double coreR, double oceanR, double need, uint32_t s0,
                        double* out, cudaStream_t s);

// ---- ws_sor.cu (colour lists) and ws_sor_tb.cu (temporal blocking on every SM)
cudaError_t sor_init(void** statePtr, const Dims& d, int device);
void sor_free(void* statePtr);
// the colour lists the list paths need (nothing when the temporal-blocked
// solve is the default: it builds its own plan)
cudaError_t launch_sor_lists(void* state, const Dims& d, const GridDev& g, const uint8_t* diag8, cudaStream_t s);
cudaError_t launch_sor_run(void* state, const Dims& d, const GridDev& g, const uint8_t* diag8, double omega,
                           int iters, int check, double tol, int* err, int** outIters, double** outRel, int** outPath,
                           cudaStream_t s);
cudaError_t launch_sor_solve(void* statePtr, const Dims& d, const GridDev& g, const uint8_t* diag8, double omega,
                             int iters, int check, double tol, int* err, int** outIters, double** outRel,
                             int** outPath, cudaStream_t s);
cudaError_t launch_sor_solve_lists(void* statePtr, const Dims& d, const GridDev& g, const uint8_t* diag8, double omega,
                                   int iters, int check, double tol, int* err, int** outIters, double** outRel,
                                   int** outPath, cudaStream_t s);
// per-256-cell-block colour counts the pressure setup fills for the list build
int* sor_block_counts(void* state);
int sor_solve_launches(void* state);
int sor_list_solve_launches(void* state);
// whether the default solve is the temporal-blocked one (it needs no per-block colour counts)
bool sor_uses_tb(void* state);

// ---- ws_contacts.cu
void launch_vapor_collisions(const Dims& d, const PartsDev& P, double spacing, double oceanR, int spinOn,
                             int hasSun, const double* sunRel, void* scratch, size_t scratchBytes,
                             DevStatus* st, cudaStream_t s);
void launch_ice_contacts(const PartsDev& P, double spacing, void* scratch, size_t scratchBytes, cudaStream_t s);
size_t contacts_scratch_bytes(int capacity, int rows);   // rows: ny * nz of the grid
