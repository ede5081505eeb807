// ws_api.cu — the C ABI of libwatersim (include/watersim.h): handle
// lifetime, device memory, the substep and frame drivers, field transfer and
// world setup. One CUDA stream per handle; no global mutable state.
#include "ws_kernels.cuh"
#include "ws_terrain.h"
#include "ws_unet.cuh"
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <new>
#include <atomic>
#include <thread>

// a marching-tets mesh in device memory: vertices (pos, nrm: 3 floats each),
// the per-block emission offsets, both grown on demand
struct MeshBuf {
  float *pos = nullptr, *nrm = nullptr;
  long long* offs = nullptr;
  long long cap = 0, offsCap = 0, verts = 0;
};

struct ws_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;          // the SOR list build beside the learned warm start
  cudaEvent_t evFork = nullptr, evJoin = nullptr;
  // host copies of the particle fields no substep kernel reads or writes
  // (ws_upload_state / ws_download_state) run on their own stream beside the
  // substep; every other entry point joins them into the main stream first
  cudaStream_t copyStream = nullptr;
  cudaEvent_t evCopy = nullptr, evMain = nullptr;
  bool copyPending = false;             // copies on copyStream not yet joined
  bool mainTouched = true;              // main-stream work other than substeps since the last full sync
  Dims d{};
  ws_params P{};
  ws_scalars S{};
  std::string err;
  int capacity = 0;
  long long launches = 0;
  // grid
  uint8_t *type = nullptr, *staticTypes = nullptr, *valid = nullptr, *diag8 = nullptr;
  float *vel = nullptr, *velO = nullptr, *gvel = nullptr, *q = nullptr, *rhs = nullptr, *pw = nullptr;
  float *vort = nullptr, *dens = nullptr;
  float2* acc = nullptr;
  // particles
  PartsDev parts{};
  // terrain
  uint8_t* tsolid = nullptr;
  float* tR = nullptr;
  TerrainDev terr{};
  wsterrain::Terrain hostTerrain;
  bool hasTerrain = false;
  // status, reductions, scratch
  DevStatus* st = nullptr;
  DevStatus* stHost = nullptr;          // pinned
  double2* partials = nullptr;
  int partialsCap = 0;
  double* red = nullptr;                // device reduction outputs
  double* redHost = nullptr;            // pinned
  uint32_t* rng = nullptr;              // device: cfS, bfS, evS
  int *blockCounts = nullptr, *list = nullptr, *listCount = nullptr;
  uint8_t* cand = nullptr;
  int* cellCnt = nullptr;
  double *cellSum = nullptr, *cellChange = nullptr;
  void* contactScratch = nullptr;       // allocated on first contact pass
  void* mtScratch = nullptr;            // straddling-cell list of the marching tets, grown on demand
  double* queryBuf = nullptr;           // point queries (sampleVel, terrainRadiusAt), allocated on first use
  size_t mtScratchBytes = 0;
  void* sor = nullptr;                  // persistent SOR solver state (ws_sor.cu)
  // the substep's face and cell passes run over the active 4^3 bricks
  BrickSet bricks{};
  CellSort csort{};                     // the particles sorted by cell for P2G
  void* csortCub = nullptr;             // prefix-sum scratch
  size_t csortCubBytes = 0;
  bool tbSetup = false;                 // the pressure setup may run over bricks (the solve needs no block counts)
  // substep graph: the kernel sequence of one substep captured once and
  // replayed while its launch parameters stay the same
  cudaGraphExec_t gexec = nullptr;
  bool graphDisabled = false;
  long long graphLaunches = 0;
  struct { double dt, gsA, coreR, oceanR, spacing; int vapor, nP, unet, balls, clearSv; ws_params P; } gsig{};
  bool substepPending = false;          // status of an asynchronous substep not yet pulled
  bool vaporPossible = false;
  double oceanRGeom = -1;               // oceanR the gravity geometry was built for
  // subsurface current lattice, allocated on first use
  CurrField curr{};
  double* currWaves = nullptr;
  // surface mesh and metaball skin (marching tets) in device memory, grown on demand
  // balls (addBall): device state (9 doubles each), solid-velocity field
  // (3 x nCells), histogram scratch and waterlines; allocated with the first ball
  double* balls = nullptr;
  float* sv = nullptr;
  int* ballHist = nullptr;
  float* ballSurf = nullptr;
  int nBalls = 0;
  bool hadSolidVelocity = false;
  // asynchronous frame step (ws_step_async): worker thread, in-flight flag, result
  std::thread asyncThread;
  std::atomic<int> asyncRunning{0};
  ws_status asyncResult = WS_OK;
  MeshBuf surf{}, mball{};
  // metaball corner field: FP64 accumulator and its float copy, (m+1)^3 corners
  double* mbAcc = nullptr;
  float* mbField = nullptr;
  double2* mbPartials = nullptr;
  long long mbCorners = 0, mbCells = 0;
  int mbM = 0;
  // render-side particle prep: sorted draw list + scratch, sized for capacity
  RenderOut rdr{};
  void* rdrScratch = nullptr;
  long long rdrPoints = 0;
  // learned warm start of the pressure solve (ws_unet.cu)
  unet::Net* net = nullptr;
  bool unetOn = false;                  // predict q before every solve
  bool unetCollect = false;             // store (input, converged q) pairs from every solve
};

static float bits_to_float(unsigned u) { float f; std::memcpy(&f, &u, sizeof(f)); return f; }

#define WS_TRY(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return fail_cuda(h, e_, #call); } while (0)

static ws_status fail(ws_handle* h, ws_status code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}
static ws_status fail_cuda(ws_handle* h, cudaError_t e, const char* what) {
  return fail(h, WS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
static void collect_async(ws_handle* h);
// A captured substep holds buffer pointers and scalars by value: state changes
// that move either (terrain buffers, scalars, balls) drop it.
static void drop_graph(ws_handle* h) {
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
}
static ws_status check_launch(ws_handle* h, int n) {
  h->launches += n;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(h, e, "kernel launch");
  return WS_OK;
}

static GridDev grid_of(ws_handle* h) {
  GridDev g;
  g.type = h->type; g.staticTypes = h->staticTypes; g.vel = h->vel; g.velO = h->velO; g.acc = h->acc;
  g.valid = h->valid; g.gvel = h->gvel; g.q = h->q; g.rhs = h->rhs; g.pw = h->pw;
  long long N = h->d.nCells;
  g.vfx = h->vort; g.vfy = h->vort + N; g.vfz = h->vort + 2 * N; g.omg = h->vort + 3 * N;
  g.omx = h->vort + 4 * N; g.omy = h->vort + 5 * N; g.omz = h->vort + 6 * N;
  g.dens = h->dens;
  g.sv = h->sv;
  g.seed = h->bricks.seed; g.nbx = h->bricks.nbx; g.nby = h->bricks.nby;
  return g;
}
// the next substep processes every brick (after a caller or a single stage wrote grid fields)
static void force_full_pass(ws_handle* h) {
  if (h->bricks.forceAll) cudaMemsetAsync(h->bricks.forceAll, 1, sizeof(int), h->stream);
  // the cell counts start from zero again (an interrupted substep may have left some)
  if (h->csort.count) {
    const size_t nKeys = 64 * (size_t)h->bricks.nbx * h->bricks.nby * h->bricks.nbz;
    cudaMemsetAsync(h->csort.count, 0, sizeof(int) * (nKeys + 1), h->stream);
  }
}
static PartsDev parts_of(ws_handle* h) { PartsDev P = h->parts; P.nP = h->S.nP; return P; }

// Fields no substep kernel reads or writes: the light and depth channels and
// the phase, and the temperature while no vapour parcel can exist (only the
// vapour pass reads it). Their copies may run beside the substep.
static bool substep_free(const ws_handle* h, int f) {
  return f == WS_F_PLIGHT || f == WS_F_PDEPTH || f == WS_F_PPH || (f == WS_F_PT && !h->vaporPossible);
}
// pending copies of substep-free fields into the main stream (every entry
// point but ws_substep and the state copies calls it first)
static void join_copies(ws_handle* h) {
  if (!h) return;
  if (h->copyPending && cudaEventRecord(h->evCopy, h->copyStream) == cudaSuccess)
    cudaStreamWaitEvent(h->stream, h->evCopy, 0);
  h->copyPending = false;
  h->mainTouched = true;
}

extern "C" const char* ws_version(void) { return "watersim-b200 0.1 (sm_100a)"; }

extern "C" const char* ws_last_error(const ws_handle* h) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return "an asynchronous step is in flight";
  if (!h) return "null handle";
  return h->err.c_str();
}

extern "C" ws_status ws_default_params(ws_params* p) {
  if (!p) return WS_ERR_INVALID;
  std::memset(p, 0, sizeof(*p));
  // library defaults of FluidSolver, js/solver.js:56-193
  p->substeps = 1; p->cfl = 3.0; p->pic = 0.15; p->gravity = 9.81; p->viscosity = 5e-4;
  p->pressureIters = 20; p->omega = 1.55; p->maxSpeed = 3.2;
  p->vorticity = 0; p->currents = 0; p->shadeCool = 0.035;
  p->sunActivity = 0; p->evapIntensity = 0.05; p->atmosphereH = 0.35; p->ceilReflect = 0;
  p->hasSun = 0; p->heatK = 0.6; p->Tamb = 0.32;
  p->cloudT = 0.34; p->cloudP = 0.35; p->rainT = 0.22; p->rainLiftAge = 0.4; p->snowT = 0.10;
  p->meltT = 0.10 * 1.05; p->spinOn = 0; p->thermalOn = 1;
  // device order of the order-dependent passes
  p->sorRedBlack = 1; p->sorCheckEvery = 10; p->sorTol = 0; p->sorMaxIters = 10000;
  p->viscJacobi = 1; p->extrapJacobi = 1; p->p2gCellOrder = 0;
  return WS_OK;
}

static void free_all(ws_handle* h) {
  void* bufs[] = { h->type, h->staticTypes, h->valid, h->diag8, h->vel, h->velO, h->gvel, h->q, h->rhs, h->pw,
                   h->vort, h->dens, h->acc, h->tsolid, h->tR, h->st, h->partials, h->red, h->rng,
                   h->blockCounts, h->list, h->listCount, h->cand, h->cellCnt, h->cellSum, h->cellChange,
                   h->parts.px, h->parts.py, h->parts.pz, h->parts.pvx, h->parts.pvy, h->parts.pvz, h->parts.pT,
                   h->parts.pAir, h->parts.pLight, h->parts.pWx, h->parts.pWy, h->parts.pWz, h->parts.pPh,
                   h->parts.pflag, h->parts.pcool, h->parts.pDepth };
  for (void* b : bufs) if (b) cudaFree(b);
  if (h->contactScratch) cudaFree(h->contactScratch);
  if (h->mtScratch) cudaFree(h->mtScratch);
  if (h->queryBuf) cudaFree(h->queryBuf);
  {
    void* bb[] = { h->bricks.seed, h->bricks.act, h->bricks.proc, h->bricks.list, h->bricks.count, h->bricks.forceAll,
                   h->csort.count, h->csort.start, h->csort.pcell, h->csort.pslot,
                   h->csort.perm, h->csortCub };
    for (void* b : bb) if (b) cudaFree(b);
  }
  if (h->sor) sor_free(h->sor);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->net) { h->net->destroy(); delete h->net; }
  if (h->curr.cfx) { cudaFree(h->curr.cfx); cudaFree(h->curr.cfy); cudaFree(h->curr.cfz); }
  if (h->currWaves) cudaFree(h->currWaves);
  for (MeshBuf* mb : { &h->surf, &h->mball })
    for (void* b : { (void*)mb->pos, (void*)mb->nrm, (void*)mb->offs }) if (b) cudaFree(b);
  for (void* b : { (void*)h->mbAcc, (void*)h->mbField, (void*)h->mbPartials }) if (b) cudaFree(b);
  for (void* b : { (void*)h->balls, (void*)h->sv, (void*)h->ballHist, (void*)h->ballSurf }) if (b) cudaFree(b);
  for (float* b : { h->rdr.pos, h->rdr.col, h->rdr.alpha, h->rdr.size, h->rdr.sprite }) if (b) cudaFree(b);
  if (h->rdrScratch) cudaFree(h->rdrScratch);
  if (h->stHost) cudaFreeHost(h->stHost);
  if (h->redHost) cudaFreeHost(h->redHost);
  if (h->evFork) cudaEventDestroy(h->evFork);
  if (h->evJoin) cudaEventDestroy(h->evJoin);
  if (h->evCopy) cudaEventDestroy(h->evCopy);
  if (h->evMain) cudaEventDestroy(h->evMain);
  if (h->copyStream) cudaStreamDestroy(h->copyStream);
  if (h->side) cudaStreamDestroy(h->side);
  if (h->stream) cudaStreamDestroy(h->stream);
}

template <typename T>
static cudaError_t dalloc(T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
  if (e == cudaSuccess) e = cudaMemset(*p, 0, sizeof(T) * (count ? count : 1));
  return e;
}

extern "C" ws_status ws_create(const ws_config* cfg, ws_handle** out) {
  if (!cfg || !out) return WS_ERR_INVALID;
  *out = nullptr;
  if (cfg->nx < 4 || cfg->ny < 4 || cfg->nz < 4 || !(cfg->dx > 0) || cfg->capacity < 1) return WS_ERR_INVALID;
  if ((long long)cfg->nx * cfg->ny * cfg->nz > (1LL << 31) / 4) return WS_ERR_RANGE;
  ws_handle* h = new (std::nothrow) ws_handle();
  if (!h) return WS_ERR_NOMEM;
  h->device = cfg->device;
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) { ws_status r = fail_cuda(h, e, "cudaSetDevice"); delete h; return r; }
  e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->evJoin, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->copyStream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->evCopy, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->evMain, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    ws_status r = fail_cuda(h, e, "cudaStreamCreate");
    if (h->evFork) cudaEventDestroy(h->evFork);
    if (h->evJoin) cudaEventDestroy(h->evJoin);
    if (h->evCopy) cudaEventDestroy(h->evCopy);
    if (h->evMain) cudaEventDestroy(h->evMain);
    if (h->copyStream) cudaStreamDestroy(h->copyStream);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h; return r;
  }
  Dims& d = h->d;
  d.nx = cfg->nx; d.ny = cfg->ny; d.nz = cfg->nz; d.dx = cfg->dx;
  d.W = d.nx * d.dx; d.H = d.ny * d.dx; d.D = d.nz * d.dx;
  d.cx = d.W / 2; d.cy = d.H / 2; d.cz = d.D / 2;
  d.domainR = 0.5 * std::min(std::min(d.W, d.H), d.D) - d.dx;
  d.nCells = (long long)d.nx * d.ny * d.nz;
  dims_fastdiv(d);
  d.uN = (long long)(d.nx + 1) * d.ny * d.nz; d.vN = (long long)d.nx * (d.ny + 1) * d.nz;
  d.wN = (long long)d.nx * d.ny * (d.nz + 1); d.F = d.uN + d.vN + d.wN;
  h->capacity = cfg->capacity;
  ws_default_params(&h->P);
  ws_scalars& S = h->S;
  S.coreR = cfg->coreR; S.spacing = d.dx * 0.5; S.particleVolume = S.spacing * S.spacing * S.spacing;
  S.iso = 1.8; S.waterTopY = d.dx + 1; S.gRamp = 1e9;
  S.evS = 0x51ab3c77u; S.cfS = 0x2f6e2b1u; S.bfS = 0x7f4a7c15u; S.stirS = 0x2545f491u;
  S.terrainSeed = cfg->terrainSeed ? cfg->terrainSeed : 20260114u;
  S.bumpiness = cfg->bumpiness < 0 ? 0 : (cfg->bumpiness > 2.5 ? 2.5 : cfg->bumpiness);
  S.targetParticles = cfg->targetParticles > 0 ? cfg->targetParticles : 110000;
  S.capacity = cfg->capacity;
  long long N = d.nCells, F = d.F, P = cfg->capacity;
  long long ND = (long long)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
#define AL(ptr, n) if ((e = dalloc(&(ptr), (size_t)(n))) != cudaSuccess) { ws_status r = fail_cuda(h, e, "cudaMalloc"); free_all(h); delete h; return r; }
  AL(h->type, N) AL(h->staticTypes, N) AL(h->diag8, N) AL(h->valid, F)
  AL(h->vel, F) AL(h->velO, F) AL(h->gvel, F) AL(h->acc, F)
  AL(h->q, N) AL(h->rhs, N) AL(h->pw, N) AL(h->vort, 7 * N) AL(h->dens, ND)
  AL(h->st, 1) AL(h->red, 8) AL(h->rng, 4)
  AL(h->cellCnt, N) AL(h->cellSum, N) AL(h->cellChange, N)
  PartsDev& pp = h->parts;
  AL(pp.px, P) AL(pp.py, P) AL(pp.pz, P) AL(pp.pvx, P) AL(pp.pvy, P) AL(pp.pvz, P)
  AL(pp.pT, P) AL(pp.pAir, P) AL(pp.pLight, P) AL(pp.pWx, P) AL(pp.pWy, P) AL(pp.pWz, P) AL(pp.pPh, P)
  AL(pp.pflag, P) AL(pp.pcool, P) AL(pp.pDepth, P)
  long long nb = (P + 255) / 256 + 1;
  AL(h->blockCounts, nb) AL(h->list, P) AL(h->listCount, 1) AL(h->cand, P)
  long long partN = std::max((long long)grid_for(N, 128) + 1, (long long)(3 * nb));
  AL(h->partials, partN)
  if ((e = sor_init(&h->sor, h->d, cfg->device)) != cudaSuccess) { ws_status r = fail_cuda(h, e, "SOR state"); free_all(h); delete h; return r; }
  h->partialsCap = (int)partN;
  h->tbSetup = sor_uses_tb(h->sor);
  {
    BrickSet& B = h->bricks;
    B.nbx = (d.nx + 3) / 4; B.nby = (d.ny + 3) / 4; B.nbz = (d.nz + 3) / 4;
    B.dnbx = fastdiv_make((unsigned)B.nbx); B.dnby = fastdiv_make((unsigned)B.nby);
    const long long nB = (long long)B.nbx * B.nby * B.nbz;
    AL(B.seed, nB) AL(B.act, nB) AL(B.proc, nB) AL(B.list, nB) AL(B.count, 1) AL(B.forceAll, 1)
    CellSort& cs = h->csort;
    AL(cs.count, 64 * nB + 1) AL(cs.start, 64 * nB + 1) AL(cs.pcell, P) AL(cs.pslot, P) AL(cs.perm, P)
    cs.cap = (int)P;
    h->csortCubBytes = cell_sort_scratch_bytes(64 * nB);
    if ((e = cudaMalloc(&h->csortCub, h->csortCubBytes)) != cudaSuccess) { ws_status r = fail_cuda(h, e, "cudaMalloc"); free_all(h); delete h; return r; }
    const int one = 1;
    if ((e = cudaMemset(B.seed, 0, (size_t)nB)) != cudaSuccess || (e = cudaMemset(B.act, 0, (size_t)nB)) != cudaSuccess ||
        (e = cudaMemset(B.count, 0, sizeof(int))) != cudaSuccess ||
        (e = cudaMemcpy(B.forceAll, &one, sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess) {
      ws_status r = fail_cuda(h, e, "brick state"); free_all(h); delete h; return r;
    }
  }
#undef AL
  if ((e = cudaMallocHost(&h->stHost, sizeof(DevStatus))) != cudaSuccess ||
      (e = cudaMallocHost(&h->redHost, sizeof(double) * 8)) != cudaSuccess) {
    ws_status r = fail_cuda(h, e, "cudaMallocHost"); free_all(h); delete h; return r;
  }
  std::memset(h->stHost, 0, sizeof(DevStatus));
  uint32_t rng0[4] = { S.cfS, S.bfS, S.evS, 0 };
  cudaMemcpy(h->rng, rng0, sizeof(rng0), cudaMemcpyHostToDevice);
  // static types without terrain (the shell only) until a terrain arrives
  h->terr = TerrainDev{}; h->terr.has = 0;
  launch_static_types(d, h->terr, S.coreR, h->staticTypes, h->stream);
  e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) { ws_status r = fail_cuda(h, e, "init"); free_all(h); delete h; return r; }
  *out = h;
  return WS_OK;
}

extern "C" ws_status ws_destroy(ws_handle* h) {
  if (!h) return WS_ERR_INVALID;
  collect_async(h);
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->copyStream) cudaStreamSynchronize(h->copyStream);
  free_all(h);
  delete h;
  return WS_OK;
}

extern "C" ws_status ws_set_params(ws_handle* h, const ws_params* p) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  if (!h || !p) return WS_ERR_INVALID;
  if (!p->sorRedBlack || !p->viscJacobi || !p->extrapJacobi)
    return fail(h, WS_ERR_INVALID, "the device path runs red-black SOR and Jacobi viscosity/extrapolation "
                                   "(sorRedBlack, viscJacobi and extrapJacobi must be 1)");
  h->P = *p;
  return WS_OK;
}
extern "C" ws_status ws_get_params(const ws_handle* h, ws_params* p) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  if (!h || !p) return WS_ERR_INVALID;
  *p = h->P;
  return WS_OK;
}

static void pull_substep(ws_handle* h);
static ws_status sync_status(ws_handle* h) {
  WS_TRY(cudaMemcpyAsync(h->stHost, h->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  if (h->substepPending) { pull_substep(h); h->substepPending = false; }
  if (h->stHost->err) {
    int ebits = h->stHost->err;
    cudaMemsetAsync(&h->st->err, 0, sizeof(int), h->stream);
    if (ebits & WS_DERR_TIMEOUT) return fail(h, WS_ERR_TIMEOUT, "a bounded device wait ran out");
    if (ebits & WS_DERR_NAN)
      return fail(h, WS_ERR_DEVICE, "device fault latched: a particle with a NaN or infinite position or velocity");
    return fail(h, WS_ERR_DEVICE, "device fault latched: a particle outside the domain box (range)");
  }
  return WS_OK;
}

static ws_status ensure_gravity(ws_handle* h) {
  if (h->oceanRGeom != h->S.oceanR) {
    launch_gravity_geometry(h->d, h->S.oceanR, h->gvel, h->stream);
    h->oceanRGeom = h->S.oceanR;
    return check_launch(h, 1);
  }
  return WS_OK;
}

extern "C" ws_status ws_get_scalars(ws_handle* h, ws_scalars* s) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !s) return WS_ERR_INVALID;
  ws_status st0 = sync_status(h); if (st0) return st0;
  uint32_t rng[4];
  WS_TRY(cudaMemcpyAsync(rng, h->rng, sizeof(rng), cudaMemcpyDeviceToHost, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  h->S.cfS = rng[0]; h->S.bfS = rng[1]; h->S.evS = rng[2];
  *s = h->S;
  return WS_OK;
}
extern "C" ws_status ws_set_scalars(ws_handle* h, const ws_scalars* s) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !s) return WS_ERR_INVALID;
  if (s->nP < 0 || s->nP > h->capacity) return fail(h, WS_ERR_RANGE, "nP exceeds the particle capacity");
  int cap = h->capacity;
  h->S = *s;
  h->S.capacity = cap;
  uint32_t rng[4] = { s->cfS, s->bfS, s->evS, 0 };
  WS_TRY(cudaMemcpyAsync(h->rng, rng, sizeof(rng), cudaMemcpyHostToDevice, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  return ensure_gravity(h);
}
extern "C" ws_status ws_set_nparticles(ws_handle* h, int32_t nP) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  if (nP < 0 || nP > h->capacity) return fail(h, WS_ERR_RANGE, "nP exceeds the particle capacity");
  h->S.nP = nP;
  return WS_OK;
}

// ------------------------------------------------------------ fields
// true if any byte is a steam (2) or cloud (3) flag: eight bytes per test,
// (b & 0xFE) == 2 <=> b in {2, 3}, with the classic has-zero-byte trick
static bool any_vapor_flag(const uint8_t* fl, int64_t n) {
  const uint64_t ones = 0x0101010101010101ull, highs = 0x8080808080808080ull;
  const uint64_t mask = 0xFEFEFEFEFEFEFEFEull, two = 0x0202020202020202ull;
  int64_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t x; std::memcpy(&x, fl + i, 8);
    uint64_t y = (x & mask) ^ two;
    if ((y - ones) & ~y & highs) return true;
  }
  for (; i < n; i++) if ((fl[i] & 0xFE) == 2) return true;
  return false;
}

struct FieldRef { void* ptr; long long count; int elem; int kind; };   // kind 1: weights view, 2: valid view
static bool field_ref(ws_handle* h, ws_field f, FieldRef& r) {
  const Dims& d = h->d; PartsDev& p = h->parts; long long P = h->capacity;
  long long ND = (long long)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
  r.kind = 0;
  switch (f) {
    case WS_F_PX: r = {p.px, P, 4, 0}; return true;
    case WS_F_PY: r = {p.py, P, 4, 0}; return true;
    case WS_F_PZ: r = {p.pz, P, 4, 0}; return true;
    case WS_F_PVX: r = {p.pvx, P, 4, 0}; return true;
    case WS_F_PVY: r = {p.pvy, P, 4, 0}; return true;
    case WS_F_PVZ: r = {p.pvz, P, 4, 0}; return true;
    case WS_F_PT: r = {p.pT, P, 4, 0}; return true;
    case WS_F_PAIR: r = {p.pAir, P, 4, 0}; return true;
    case WS_F_PLIGHT: r = {p.pLight, P, 4, 0}; return true;
    case WS_F_PWX: r = {p.pWx, P, 4, 0}; return true;
    case WS_F_PWY: r = {p.pWy, P, 4, 0}; return true;
    case WS_F_PWZ: r = {p.pWz, P, 4, 0}; return true;
    case WS_F_PPH: r = {p.pPh, P, 4, 0}; return true;
    case WS_F_PFLAG: r = {p.pflag, P, 1, 0}; return true;
    case WS_F_PCOOL: r = {p.pcool, P, 1, 0}; return true;
    case WS_F_PDEPTH: r = {p.pDepth, P, 1, 0}; return true;
    case WS_F_CELLTYPE: r = {h->type, d.nCells, 1, 0}; return true;
    case WS_F_Q: r = {h->q, d.nCells, 4, 0}; return true;
    case WS_F_RHS: r = {h->rhs, d.nCells, 4, 0}; return true;
    case WS_F_U: r = {h->vel, d.uN, 4, 0}; return true;
    case WS_F_V: r = {h->vel + d.uN, d.vN, 4, 0}; return true;
    case WS_F_W: r = {h->vel + d.uN + d.vN, d.wN, 4, 0}; return true;
    case WS_F_UO: r = {h->velO, d.uN, 4, 0}; return true;
    case WS_F_VO: r = {h->velO + d.uN, d.vN, 4, 0}; return true;
    case WS_F_WO: r = {h->velO + d.uN + d.vN, d.wN, 4, 0}; return true;
    case WS_F_UW: r = {(void*)0, d.uN, 4, 1}; return true;
    case WS_F_VW: r = {(void*)d.uN, d.vN, 4, 1}; return true;
    case WS_F_WW: r = {(void*)(d.uN + d.vN), d.wN, 4, 1}; return true;
    case WS_F_VALIDU: r = {h->valid, d.uN, 1, 2}; return true;
    case WS_F_VALIDV: r = {h->valid + d.uN, d.vN, 1, 2}; return true;
    case WS_F_VALIDW: r = {h->valid + d.uN + d.vN, d.wN, 1, 2}; return true;
    case WS_F_DENS: r = {h->dens, ND, 4, 0}; return true;
    default: return false;
  }
}
extern "C" ws_status ws_field_info(const ws_handle* hc, ws_field f, int64_t* count, int32_t* elem) {
  if (hc && hc->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  ws_handle* h = const_cast<ws_handle*>(hc);
  if (!h) return WS_ERR_INVALID;
  FieldRef r;
  if (!field_ref(h, f, r)) return fail(h, WS_ERR_INVALID, "unknown field");
  if (count) *count = r.count;
  if (elem) *elem = r.elem;
  return WS_OK;
}
extern "C" ws_status ws_upload_field(ws_handle* h, ws_field f, const void* host, int64_t count) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || (!host && count)) return WS_ERR_INVALID;
  FieldRef r;
  if (!field_ref(h, f, r)) return fail(h, WS_ERR_INVALID, "unknown field");
  if (count < 0 || count > r.count) return fail(h, WS_ERR_RANGE, "count exceeds the field size");
  if (r.kind != 0) return fail(h, WS_ERR_INVALID, "derived field is read-only");
  WS_TRY(cudaMemcpyAsync(r.ptr, host, (size_t)count * r.elem, cudaMemcpyHostToDevice, h->stream));
  if (f >= WS_F_CELLTYPE) force_full_pass(h);          // a grid field: rewrite every brick next substep
  WS_TRY(cudaStreamSynchronize(h->stream));
  if (f == WS_F_PFLAG && !h->vaporPossible && any_vapor_flag((const uint8_t*)host, count))
    h->vaporPossible = true;
  return WS_OK;
}
extern "C" ws_status ws_download_field(ws_handle* h, ws_field f, void* host, int64_t count) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || (!host && count)) return WS_ERR_INVALID;
  FieldRef r;
  if (!field_ref(h, f, r)) return fail(h, WS_ERR_INVALID, "unknown field");
  if (count < 0 || count > r.count) return fail(h, WS_ERR_RANGE, "count exceeds the field size");
  if (r.kind == 1) {
    float* tmp = (float*)h->cellChange;                   // 8 N bytes >= 4 * (component face count)
    if ((long long)count * 4 > h->d.nCells * 8) return fail(h, WS_ERR_RANGE, "weights view too large");
    launch_extract_weight(h->d, h->acc, tmp, (long long)(size_t)r.ptr, count, h->stream);
    ws_status s = check_launch(h, 1); if (s) return s;
    WS_TRY(cudaMemcpyAsync(host, tmp, (size_t)count * 4, cudaMemcpyDeviceToHost, h->stream));
  } else {
    WS_TRY(cudaMemcpyAsync(host, r.ptr, (size_t)count * r.elem, cudaMemcpyDeviceToHost, h->stream));
  }
  WS_TRY(cudaStreamSynchronize(h->stream));
  if (r.kind == 2) { uint8_t* v = (uint8_t*)host; for (int64_t i = 0; i < count; i++) if (v[i] == 2) v[i] = 1; }
  return WS_OK;
}

// one queued copy per particle field, one synchronisation for all of them
// Upload: the substep's fields on the main stream, which returns once they
// are on the device; the substep-free fields on the copy stream, after any
// main-stream work still reading them, left running beside the next
// substeps. Download: the substep's fields after the main stream's work;
// the substep-free fields, when only substeps ran since the last full sync,
// straight away on the copy stream (no substep changes them); both streams
// are synchronised before returning.
static ws_status state_copy(ws_handle* h, const ws_host_arrays* a, bool up) {
  if (!h || !a) return WS_ERR_INVALID;
  if (a->count < 0 || a->count > h->capacity) return fail(h, WS_ERR_RANGE, "count exceeds the particle capacity");
  if (up && a->field[WS_F_PFLAG] && !h->vaporPossible &&
      any_vapor_flag((const uint8_t*)a->field[WS_F_PFLAG], a->count))
    h->vaporPossible = true;
  const bool beside = up || !h->mainTouched;
  if (beside && h->mainTouched) {                 // copy stream after main-stream work that may use the fields
    WS_TRY(cudaEventRecord(h->evMain, h->stream));
    WS_TRY(cudaStreamWaitEvent(h->copyStream, h->evMain, 0));
  }
  for (int f = 0; f < WS_NUM_PARTICLE_FIELDS; f++) {
    if (!a->field[f]) continue;
    FieldRef r;
    field_ref(h, (ws_field)f, r);
    size_t bytes = (size_t)a->count * r.elem;
    cudaStream_t st = beside && substep_free(h, f) ? h->copyStream : h->stream;
    if (up) WS_TRY(cudaMemcpyAsync(r.ptr, a->field[f], bytes, cudaMemcpyHostToDevice, st));
    else WS_TRY(cudaMemcpyAsync(a->field[f], r.ptr, bytes, cudaMemcpyDeviceToHost, st));
  }
  WS_TRY(cudaStreamSynchronize(h->stream));
  if (up) {
    h->copyPending = true;
    h->mainTouched = false;
  } else {
    WS_TRY(cudaStreamSynchronize(h->copyStream));
    h->copyPending = false;
    h->mainTouched = false;
  }
  return WS_OK;
}
extern "C" ws_status ws_upload_state(ws_handle* h, const ws_host_arrays* a) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY; return state_copy(h, a, true); }
extern "C" ws_status ws_download_state(ws_handle* h, const ws_host_arrays* a) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  return state_copy(h, a, false);
}

// ------------------------------------------------------------ terrain + fill
static ws_status terrain_to_device(ws_handle* h) {
  const wsterrain::Terrain& T = h->hostTerrain;
  long long n3 = (long long)T.n * T.n * T.n;
  // A terrain of the same lattice size reuses the device buffers; the captured
  // substep graph, which holds the terrain by value, survives when nothing it
  // holds changes (the case of a snapshot restored onto its own planet).
  const bool reuse = h->tsolid && h->tR && h->terr.has && h->terr.n == T.n;
  if (!reuse) {
    drop_graph(h);
    if (h->tsolid) { cudaFree(h->tsolid); h->tsolid = nullptr; }
    if (h->tR) { cudaFree(h->tR); h->tR = nullptr; }
    WS_TRY(cudaMalloc(&h->tsolid, (size_t)n3));
    WS_TRY(cudaMalloc(&h->tR, sizeof(float) * (size_t)n3));
  }
  WS_TRY(cudaMemcpyAsync(h->tsolid, T.solid.data(), (size_t)n3, cudaMemcpyHostToDevice, h->stream));
  WS_TRY(cudaMemcpyAsync(h->tR, T.R.data(), sizeof(float) * (size_t)n3, cudaMemcpyHostToDevice, h->stream));
  const TerrainDev before = h->terr;
  TerrainDev& t = h->terr;
  t.n = T.n; t.has = 1; t.dv = T.dv; t.Rsl = T.Rsl; t.Rlo = T.Rlo; t.Rhi = T.Rhi;
  t.Rlo2 = T.Rlo * T.Rlo; t.Rhi2 = T.Rhi * T.Rhi; t.solid = h->tsolid; t.R = h->tR;
  t.rdv = 1.0 / T.dv; t.dvPow2 = is_pow2(T.dv) ? 1 : 0;
  if (reuse && std::memcmp(&before, &t, sizeof(TerrainDev)) != 0) drop_graph(h);
  h->S.landFrac = T.landFrac;
  h->hasTerrain = true;
  launch_static_types(h->d, t, h->S.coreR, h->staticTypes, h->stream);
  ws_status s = check_launch(h, 1); if (s) return s;
  WS_TRY(cudaStreamSynchronize(h->stream));
  return WS_OK;
}

extern "C" ws_status ws_generate_terrain(ws_handle* h, uint32_t seed, double seaLevel) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  wsterrain::GenInput in{seed, h->S.coreR, seaLevel, h->S.bumpiness, h->d.dx, h->d.cx, h->d.cy, h->d.cz, h->d.nx, h->stream};
  int r = wsterrain::generate(in, h->hostTerrain, h->err);
  if (r) return r;
  h->launches += 1;
  return terrain_to_device(h);
}

extern "C" ws_status ws_upload_terrain(ws_handle* h, const ws_terrain* t) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !t || t->n < 2 || !t->solid || !t->R) return WS_ERR_INVALID;
  force_full_pass(h);                            // the static cell types change
  wsterrain::Terrain& T = h->hostTerrain;
  long long n3 = (long long)t->n * t->n * t->n;
  T.n = t->n; T.dv = t->dv; T.Rsl = t->Rsl; T.Rlo = t->Rlo; T.Rhi = t->Rhi; T.landFrac = t->landFrac;
  T.solid.assign(t->solid, t->solid + n3);
  T.R.assign(t->R, t->R + n3);
  return terrain_to_device(h);
}

extern "C" ws_status ws_download_terrain(ws_handle* h, uint8_t* solid, float* R, double meta[4]) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  if (!h->hasTerrain) return fail(h, WS_ERR_STATE, "no terrain");
  const wsterrain::Terrain& T = h->hostTerrain;
  size_t n3 = (size_t)T.n * T.n * T.n;
  if (solid) std::memcpy(solid, T.solid.data(), n3);
  if (R) std::memcpy(R, T.R.data(), n3 * sizeof(float));
  if (meta) { meta[0] = T.n; meta[1] = T.Rlo; meta[2] = T.Rhi; meta[3] = T.landFrac; }
  return WS_OK;
}

static wsterrain::FillInput fill_input(ws_handle* h, double depth) {
  wsterrain::FillInput in;
  in.seed = h->S.terrainSeed; in.nx = h->d.nx; in.ny = h->d.ny; in.nz = h->d.nz;
  in.dx = h->d.dx; in.cx = h->d.cx; in.cy = h->d.cy; in.cz = h->d.cz;
  in.coreR = h->S.coreR; in.depth = depth; in.targetParticles = h->S.targetParticles; in.capacity = h->capacity;
  return in;
}

extern "C" ws_status ws_water_volume(ws_handle* h, double depth, double* volume) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !volume) return WS_ERR_INVALID;
  if (!h->hasTerrain) return fail(h, WS_ERR_STATE, "no terrain");
  *volume = wsterrain::water_volume(h->hostTerrain, fill_input(h, depth));
  return WS_OK;
}

static ws_status splat_and_iso(ws_handle* h);

// _resetWaterSphere, js/solver.js:651-731
extern "C" ws_status ws_reset_water(ws_handle* h, double depth) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  double R2 = h->S.coreR + depth;
  h->S.oceanR = R2;
  h->nBalls = 0;                                 // resetWater drops the balls (js/solver.js:612, 652)
  force_full_pass(h);
  if (!h->hasTerrain) { ws_status s = ws_generate_terrain(h, h->S.terrainSeed, R2); if (s) return s; }
  wsterrain::FillOutput fo;
  wsterrain::fill(h->hostTerrain, fill_input(h, depth), fo);
  int n = (int)fo.px.size();
  h->S.spacing = fo.spacing; h->S.particleVolume = fo.spacing * fo.spacing * fo.spacing;
  PartsDev& p = h->parts;
  size_t P = (size_t)h->capacity;
  WS_TRY(cudaMemcpyAsync(p.px, fo.px.data(), sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
  WS_TRY(cudaMemcpyAsync(p.py, fo.py.data(), sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
  WS_TRY(cudaMemcpyAsync(p.pz, fo.pz.data(), sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
  WS_TRY(cudaMemsetAsync(p.pvx, 0, sizeof(float) * n, h->stream));
  WS_TRY(cudaMemsetAsync(p.pvy, 0, sizeof(float) * n, h->stream));
  WS_TRY(cudaMemsetAsync(p.pvz, 0, sizeof(float) * n, h->stream));
  WS_TRY(cudaMemsetAsync(p.pflag, 0, (size_t)n, h->stream));
  WS_TRY(cudaMemsetAsync(p.pcool, 0, (size_t)n, h->stream));
  WS_TRY(cudaMemsetAsync(p.pAir, 0, sizeof(float) * P, h->stream));
  std::vector<float> tamb((size_t)n, (float)h->P.Tamb);
  WS_TRY(cudaMemcpyAsync(p.pT, tamb.data(), sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
  WS_TRY(cudaMemsetAsync(h->q, 0, sizeof(float) * h->d.nCells, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  h->S.nP = n;
  h->S.heatAcc = 0; h->S.vaporCount = h->S.nightVaporCount = 0;
  h->S.waterTopY = h->d.cy + R2;
  h->vaporPossible = false;
  ws_status s = ensure_gravity(h); if (s) return s;
  h->S.gRamp = 0;
  s = splat_and_iso(h); if (s) return s;
  h->S.umax = 0; h->S.airborneCount = 0;
  return WS_OK;
}

// ------------------------------------------------------------ reductions
static ws_status mt_scratch(ws_handle* h, long long nCells, void** out) {
  const size_t need = mt_scratch_bytes(nCells);
  if (need > h->mtScratchBytes) {
    if (h->mtScratch) cudaFree(h->mtScratch);
    h->mtScratch = nullptr; h->mtScratchBytes = 0;
    WS_TRY(cudaMalloc(&h->mtScratch, need));
    h->mtScratchBytes = need;
  }
  *out = h->mtScratch;
  return WS_OK;
}
static ws_status mt_volume(ws_handle* h, double iso, double* vol, int64_t* cnt) {
  if ((long long)grid_for(h->d.nCells, 128) > h->partialsCap) return fail(h, WS_ERR_RANGE, "partials too small");
  void* scr = nullptr;
  ws_status s = mt_scratch(h, h->d.nCells, &scr); if (s) return s;
  launch_mt_volume(h->d, h->dens, iso, h->partials, h->red, scr, h->stream);
  s = check_launch(h, 6); if (s) return s;
  WS_TRY(cudaMemcpyAsync(h->redHost, h->red, sizeof(double) * 2, cudaMemcpyDeviceToHost, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  if (vol) *vol = std::fabs(h->redHost[0]);
  if (cnt) *cnt = (int64_t)llround(h->redHost[1]);
  return WS_OK;
}
extern "C" ws_status ws_mt_volume(ws_handle* h, double iso, double* volume, int64_t* vertexCount) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  return mt_volume(h, iso, volume, vertexCount);
}
// autotuneIso, js/solver.js:3838-3849
static ws_status autotune(ws_handle* h, double* iso) {
  double Vt = h->S.nP * h->S.particleVolume, lo = 0.3, hi = 3.0;
  for (int it = 0; it < 8; it++) {
    double mid = 0.5 * (lo + hi), vol; int64_t cnt;
    ws_status s = mt_volume(h, mid, &vol, &cnt); if (s) return s;
    if (cnt > 900000 || vol > Vt) lo = mid; else hi = mid;
  }
  *iso = 0.5 * (lo + hi);
  return WS_OK;
}
extern "C" ws_status ws_autotune_iso(ws_handle* h, double* iso) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !iso) return WS_ERR_INVALID;
  return autotune(h, iso);
}
static ws_status splat_and_iso(ws_handle* h) {
  launch_splat(h->d, grid_of(h), parts_of(h), h->S.spacing, h->stream);
  ws_status s = check_launch(h, 1); if (s) return s;
  double iso;
  s = autotune(h, &iso); if (s) return s;
  h->S.iso = iso;
  return WS_OK;
}
static ws_status particle_reduce(ws_handle* h, int mode, double mp, double out[3]) {
  launch_particle_reduce(parts_of(h), mode, mp, (double*)h->partials, h->red, h->stream);
  ws_status s = check_launch(h, 2); if (s) return s;
  WS_TRY(cudaMemcpyAsync(h->redHost, h->red, sizeof(double) * 3, cudaMemcpyDeviceToHost, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  out[0] = h->redHost[0]; out[1] = h->redHost[1]; out[2] = h->redHost[2];
  return WS_OK;
}
extern "C" ws_status ws_kinetic_energy(ws_handle* h, double* ke) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !ke) return WS_ERR_INVALID;
  double o[3];
  ws_status s = particle_reduce(h, 0, 1000 * h->S.particleVolume, o); if (s) return s;
  *ke = o[0];
  return WS_OK;
}
// earthCensus, js/main.js:176-186: counts are exact, fractions in FP64
extern "C" ws_status ws_census(ws_handle* h, double fr[3]) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !fr) return WS_ERR_INVALID;
  double o[3];
  ws_status s = particle_reduce(h, 1, 0, o); if (s) return s;
  double tot = o[0] + o[1] + o[2];
  if (tot > 0) { fr[0] = o[0] / tot; fr[1] = o[1] / tot; fr[2] = o[2] / tot; } else fr[0] = fr[1] = fr[2] = 0;
  return WS_OK;
}
extern "C" ws_status ws_residual(ws_handle* h, double* relres) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !relres) return WS_ERR_INVALID;
  launch_residual(h->d, grid_of(h), h->diag8, h->partials, h->st, nullptr, h->stream);
  ws_status s = check_launch(h, 2); if (s) return s;
  s = sync_status(h); if (s) return s;
  *relres = h->stHost->relres;
  return WS_OK;
}

// ------------------------------------------------------------ substep stages
static AdvectParams advect_params(ws_handle* h, double dt) {
  AdvectParams a;
  a.dt = dt; a.dtLast = h->S.dtLast; a.pic = h->P.pic; a.maxSpeed = h->P.maxSpeed; a.gravity = h->P.gravity;
  a.oceanR = h->S.oceanR; a.coreR = h->S.coreR; a.atmosphereH = h->P.atmosphereH;
  double rainTe = std::min(h->P.rainT, h->P.cloudT - 0.02); if (rainTe < 0) rainTe = 0;
  a.rainTe = rainTe; a.rainLiftAge = h->P.rainLiftAge; a.ceilReflect = h->P.ceilReflect;
  a.windS[0] = 1; a.windS[1] = 0; a.windS[2] = 0;
  if (h->P.hasSun) {
    double sx = h->P.sunPos[0] - h->d.cx, sy = h->P.sunPos[1] - h->d.cy, sz = h->P.sunPos[2] - h->d.cz;
    double L = std::sqrt(sx * sx + sy * sy + sz * sz); if (L == 0) L = 1;
    a.windS[0] = sx / L; a.windS[1] = sy / L; a.windS[2] = sz / L;
  }
  return a;
}

// Stages take `bricks`: inside a whole substep the face and cell passes run
// over the active-brick list; a stage called on its own runs over the whole
// grid and forces the next substep to process every brick.
static ws_status stage_clear_raster(ws_handle* h, bool bricks = false) {
  launch_clear_raster(h->d, grid_of(h), h->st, !bricks, h->stream);
  if (bricks) launch_clear_acc_bricks(h->d, grid_of(h), h->bricks, h->stream);
  return check_launch(h, bricks ? 2 : 1);
}
// bricks: the substep's own pipeline, where (with p2gCellOrder) the mark
// pass also counts the particles per cell for the cell-ordered P2G
static ws_status stage_mark(ws_handle* h, bool bricks = false) {
  launch_mark_fluid(h->d, grid_of(h), parts_of(h), h->terr, h->S.oceanR, h->S.coreR,
                    bricks && h->P.p2gCellOrder ? &h->csort : nullptr, h->st, h->stream);
  ws_status s = check_launch(h, 1); if (s) return s;
  if (bricks) {
    cudaError_t e = launch_brick_activity(h->bricks, h->stream);
    if (e != cudaSuccess) return fail_cuda(h, e, "active bricks");
    s = check_launch(h, 1); if (s) return s;
  }
  return WS_OK;
}
// P2G in particle index order, or (p2gCellOrder) in cell order: with bricks
// the mark pass counted and the brick list is current; the stage-wise call
// counts here and visits every brick
static ws_status stage_p2g(ws_handle* h, bool bricks = false) {
  int n = 1;
  if (h->P.p2gCellOrder) {
    n = launch_p2g_sorted(h->d, grid_of(h), parts_of(h), h->csort, h->bricks, bricks, h->csortCub, h->csortCubBytes,
                          h->st, h->stream);
    if (n < 0) return fail_cuda(h, cudaGetLastError(), "cell sort");
  } else {
    launch_p2g(h->d, grid_of(h), parts_of(h), h->st, h->stream);
  }
  if (bricks) launch_faces_normalize_bc_bricks(h->d, grid_of(h), h->bricks, h->stream);
  else launch_faces_normalize_bc(h->d, grid_of(h), h->stream);
  return check_launch(h, n + 1);
}
// planet gravity ramp, js/solver.js:2656-2662: the applied scale of this
// substep (0 = no gravity), advancing the ramp timer
static double gravity_scale(ws_handle* h, double dt) {
  double gs = h->S.gRamp / 1.5; if (gs > 1) gs = 1;
  h->S.gRamp += dt;
  return gs > 0 ? gs * h->P.gravity : 0;
}
static ws_status stage_forces(ws_handle* h, double dt, double gsA, bool bricks = false) {
  double nu = h->P.viscosity;
  double coef = std::min(nu * dt / (h->d.dx * h->d.dx), 0.24);
  int viscOn = nu > 1e-6;
  if (bricks) launch_faces_forces_bricks(h->d, grid_of(h), h->bricks, coef, viscOn, dt, gsA, h->stream);
  else launch_faces_forces(h->d, grid_of(h), coef, viscOn, dt, gsA, h->stream);
  return check_launch(h, 1);
}
// _pressureSolve: setup (diag, rhs, q = 0 off the fluid) then the whole SOR
// solve in one persistent cooperative launch (ws_sor.cu). Iteration count and
// FP64 residual land in the status word and are read at the next sync.
static ws_status stage_pressure(ws_handle* h, bool bricks = false) {
  GridDev g = grid_of(h);
  // the colour-list solves need the setup's per-block counts over the whole grid
  if (bricks && h->tbSetup) launch_pressure_setup_bricks(h->d, g, h->diag8, h->P.omega, h->st, h->bricks, h->stream);
  else launch_pressure_setup(h->d, g, h->diag8, h->P.omega, h->st, sor_block_counts(h->sor), h->stream);
  ws_status s = check_launch(h, 1); if (s) return s;
  bool tolMode = h->P.sorTol > 0;
  int iters = tolMode ? h->P.sorMaxIters : h->P.pressureIters;
  int check = tolMode ? (h->P.sorCheckEvery > 0 ? h->P.sorCheckEvery : 1) : 0;
  int* dIters = nullptr; double* dRel = nullptr; int* dPath = nullptr;
  cudaError_t e;
  if (h->net && h->unetCollect) {
    if ((e = h->net->collect_pre(h->q, h->rhs, h->diag8, h->type, h->stream)) != cudaSuccess)
      return fail_cuda(h, e, "warm-start pair (before the solve)");
  }
  if (h->net && h->unetOn) {
    // the colour lists on the side stream while the network predicts q (they do not read q)
    WS_TRY(cudaEventRecord(h->evFork, h->stream));
    // From here on every exit joins the side stream back into the main one,
    // so a capture in progress ends with no unjoined stream and reports the
    // first error rather than an unjoined-capture one.
    struct SideJoin {
      ws_handle* h; bool armed;
      ~SideJoin() {
        if (armed && cudaEventRecord(h->evJoin, h->side) == cudaSuccess) cudaStreamWaitEvent(h->stream, h->evJoin, 0);
      }
    } join{ h, true };
    WS_TRY(cudaStreamWaitEvent(h->side, h->evFork, 0));
    if ((e = launch_sor_lists(h->sor, h->d, g, h->diag8, h->side)) != cudaSuccess) return fail_cuda(h, e, "SOR lists");
    WS_TRY(cudaEventRecord(h->evJoin, h->side));
    if ((e = h->net->predict(h->q, h->rhs, h->diag8, h->type, h->stream)) != cudaSuccess)
      return fail_cuda(h, e, "learned warm start");
    h->launches += 23;
    join.armed = false;
    WS_TRY(cudaStreamWaitEvent(h->stream, h->evJoin, 0));
    e = launch_sor_run(h->sor, h->d, g, h->diag8, h->P.omega, iters, check, h->P.sorTol, &h->st->err, &dIters, &dRel,
                       &dPath, h->stream);
  } else {
    e = launch_sor_solve(h->sor, h->d, g, h->diag8, h->P.omega, iters, check, h->P.sorTol,
                         &h->st->err, &dIters, &dRel, &dPath, h->stream);
  }
  if (e != cudaSuccess) return fail_cuda(h, e, "SOR solve launch");
  s = check_launch(h, sor_solve_launches(h->sor)); if (s) return s;
  WS_TRY(cudaMemcpyAsync(&h->st->sorIters, dIters, sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
  WS_TRY(cudaMemcpyAsync(&h->st->relres, dRel, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  WS_TRY(cudaMemcpyAsync(&h->st->pad2, dPath, sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
  if (h->net && h->unetCollect) {
    if ((e = h->net->collect_post(h->q, h->stream)) != cudaSuccess) return fail_cuda(h, e, "warm-start pair (after the solve)");
  }
  return WS_OK;
}
// solve diagnostics, valid after a sync_status that followed stage_pressure
static void pressure_diagnostics(ws_handle* h) {
  h->S.sorIters = h->stHost->sorIters;
  h->S.sorRelRes = h->stHost->relres;
  h->S.nFluid = h->stHost->nFluid;
  h->S.sorPath = h->stHost->pad2;
}
// counters of the last substep (umax, airborne, solve diagnostics)
static void pull_substep(ws_handle* h) {
  pressure_diagnostics(h);
  h->S.umax = (double)bits_to_float(h->stHost->umaxBits);
  h->S.airborneCount = h->stHost->airborne;
}
static ws_status stage_project(ws_handle* h, bool clampToo, bool bricks = false) {
  if (bricks) launch_project_bricks(h->d, grid_of(h), h->bricks, clampToo ? 1 : 0, h->P.maxSpeed, h->st, h->stream);
  else launch_project(h->d, grid_of(h), clampToo ? 1 : 0, h->P.maxSpeed, h->st, h->stream);
  return check_launch(h, 1);
}
static ws_status stage_vorticity(ws_handle* h, double dt) {
  if (!(h->P.vorticity > 0)) return WS_OK;
  launch_vorticity(h->d, grid_of(h), h->P.vorticity, dt, h->stream);
  return check_launch(h, 3);
}
static ws_status stage_clamp(ws_handle* h) {
  launch_clamp_umax(h->d, grid_of(h), h->P.maxSpeed, h->st, h->stream);
  return check_launch(h, 1);
}
static ws_status stage_extrapolate(ws_handle* h, bool bricks = false) {
  if (bricks) launch_extrapolate_bricks(h->d, grid_of(h), h->bricks, h->stream);
  else launch_extrapolate(h->d, grid_of(h), h->stream);
  return check_launch(h, 1);
}
static ws_status stage_g2p_advect(ws_handle* h, double dt) {
  AdvectParams ap = advect_params(h, dt);
  launch_g2p_advect(h->d, grid_of(h), parts_of(h), h->terr, ap, h->st, h->stream);
  ws_status s = check_launch(h, 1); if (s) return s;
  if (h->vaporPossible && h->S.nP > 0) {
    launch_compact(h->parts.pflag, h->S.nP, 0, h->blockCounts, h->list, h->listCount, h->stream);
    launch_vapor_advect(h->d, grid_of(h), parts_of(h), h->terr, ap, h->list, h->listCount, h->rng, h->st, h->stream);
    s = check_launch(h, 4); if (s) return s;
  }
  return WS_OK;
}

// _substep, js/solver.js:2568-2624
// _substep, js/solver.js:2568-2624: the kernels of one substep, enqueued
// without any host synchronisation (capturable into a CUDA graph)
static ws_status enqueue_substep(ws_handle* h, double dt, double gsA) {
  ws_status s;
  if ((s = stage_clear_raster(h, true))) return s;
  if (h->sv && (h->nBalls || h->hadSolidVelocity)) {      // balls become moving solids
    launch_ball_raster(h->d, h->type, h->sv, true, h->balls, h->nBalls, grid_of(h), h->stream);
    if ((s = check_launch(h, h->nBalls ? 1 : 0))) return s;
  }
  if ((s = stage_mark(h, true))) return s;
  if (h->nBalls) {
    launch_ball_push(parts_of(h), h->balls, h->nBalls, h->stream);
    if ((s = check_launch(h, h->S.nP ? 1 : 0))) return s;
  }
  if ((s = stage_p2g(h, true))) return s;
  if ((s = stage_forces(h, dt, gsA, true))) return s;
  if ((s = stage_pressure(h, true))) return s;
  bool vort = h->P.vorticity > 0;
  if ((s = stage_project(h, !vort, true))) return s;
  if (vort) { if ((s = stage_vorticity(h, dt))) return s; if ((s = stage_clamp(h))) return s; }
  if ((s = stage_extrapolate(h, true))) return s;
  if ((s = stage_g2p_advect(h, dt))) return s;
  if (h->nBalls) {                                        // _advect's push, then _updateBalls
    launch_ball_push(parts_of(h), h->balls, h->nBalls, h->stream);
    BallEnv env{ h->S.coreR, h->S.oceanR, h->P.gravity };
    launch_ball_update(h->d, h->vel, h->terr, parts_of(h), h->balls, h->nBalls, h->ballHist, h->ballSurf, env, dt,
                       h->stream);
    if ((s = check_launch(h, (h->S.nP ? 3 : 1) + (h->nBalls > 1 ? 1 : 0)))) return s;
  }
  return WS_OK;
}
// Captures the substep into a graph; on any capture failure the handle
// falls back to direct launches for good (same kernels, same order).
static bool capture_substep(ws_handle* h, double dt, double gsA) {
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  long long l0 = h->launches;
  if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError(); h->graphDisabled = true; return false;
  }
  ws_status s = enqueue_substep(h, dt, gsA);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (s != WS_OK || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError(); h->graphDisabled = true; h->launches = l0; return false;
  }
  e = cudaGraphInstantiate(&h->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { cudaGetLastError(); h->gexec = nullptr; h->graphDisabled = true; h->launches = l0; return false; }
  h->graphLaunches = h->launches - l0;
  h->launches = l0;
  return true;
}
static ws_status substep(ws_handle* h, double dt) {
  ws_status s = ensure_gravity(h); if (s) return s;
  double gsA = gravity_scale(h, dt);
  bool vapor = h->vaporPossible && h->S.nP > 0;
  // pair collection writes a new slot each substep: those substeps run uncaptured
  const bool collect = h->net && h->unetCollect;
  const int clearSv = (h->sv && (h->nBalls || h->hadSolidVelocity)) ? 1 : 0;
  bool same = !collect && h->gexec && h->gsig.dt == dt && h->gsig.gsA == gsA && h->gsig.vapor == (int)vapor &&
              h->gsig.nP == h->S.nP && h->gsig.unet == (int)h->unetOn && h->gsig.balls == h->nBalls &&
              h->gsig.clearSv == clearSv && h->gsig.coreR == h->S.coreR && h->gsig.oceanR == h->S.oceanR &&
              h->gsig.spacing == h->S.spacing && std::memcmp(&h->gsig.P, &h->P, sizeof(ws_params)) == 0;
  if (!same && !collect && !h->graphDisabled && capture_substep(h, dt, gsA)) {
    h->gsig.dt = dt; h->gsig.gsA = gsA; h->gsig.vapor = (int)vapor; h->gsig.nP = h->S.nP; h->gsig.P = h->P;
    h->gsig.unet = (int)h->unetOn; h->gsig.balls = h->nBalls; h->gsig.clearSv = clearSv;
    h->gsig.coreR = h->S.coreR; h->gsig.oceanR = h->S.oceanR; h->gsig.spacing = h->S.spacing;
    same = true;
  }
  if (same) {
    WS_TRY(cudaGraphLaunch(h->gexec, h->stream));
    h->launches += h->graphLaunches;
  } else {
    if ((s = enqueue_substep(h, dt, gsA))) return s;
  }
  h->S.dtLast = dt;
  h->hadSolidVelocity = h->nBalls > 0;
  h->substepPending = true;           // umax, counts and solve diagnostics are pulled at the next sync
  return WS_OK;
}

extern "C" ws_status ws_substep(ws_handle* h, double dt) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  if (!h || !(dt > 0)) return WS_ERR_INVALID;
  if (!h->hasTerrain) return fail(h, WS_ERR_STATE, "no terrain: call ws_generate_terrain or ws_upload_terrain");
  cudaSetDevice(h->device);
  return substep(h, dt);
}

// ------------------------------------------------------------ frame passes
// _updateCurrents, js/solver.js:3658-3665: the nine waves of _buildCurrWaves
// (:3634-3656, fixed seed 1234567, the LCG of the reference in doubles) are
// built once; field and relaxation run on the device each tick
static ws_status currents(ws_handle* h, double dt) {
  if (!(h->P.currents > 0)) return WS_OK;
  CurrField& F = h->curr;
  if (!F.cfx) {
    F.gnx = h->d.nx / 4 + 2; F.gny = h->d.ny / 4 + 2; F.gnz = h->d.nz / 4 + 2; F.sx = h->d.dx * 4;
    const size_t gN = (size_t)F.gnx * F.gny * F.gnz;
    WS_TRY(cudaMalloc(&F.cfx, sizeof(float) * gN));
    WS_TRY(cudaMalloc(&F.cfy, sizeof(float) * gN));
    WS_TRY(cudaMalloc(&F.cfz, sizeof(float) * gN));
    double w[45], seed = 1234567;
    const double K[3] = { 1.5, 4.0, 9.0 }, amp[3] = { 0.10, 0.085, 0.05 }, dr[3] = { 0.021, 0.05, 0.11 };
    for (int o = 0; o < 3; o++) {
      for (int c = 0; c < 3; c++) {
        double r3[3];
        for (int q = 0; q < 3; q++) { seed = std::fmod(seed * 1664525 + 1013904223, 4294967296.0); r3[q] = seed / 4294967296.0 * 2 - 1; }
        double L = std::sqrt(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]); if (L == 0) L = 1;
        double* wv = w + (o * 3 + c) * 5;
        wv[0] = r3[0] / L * K[o]; wv[1] = r3[1] / L * K[o]; wv[2] = r3[2] / L * K[o]; wv[3] = amp[o] / K[o];
        seed = std::fmod(seed * 1664525 + 1013904223, 4294967296.0);
        wv[4] = seed / 4294967296.0 * 6.283;
      }
      F.drift[o] = dr[o];
    }
    WS_TRY(cudaMalloc(&h->currWaves, sizeof(w)));
    WS_TRY(cudaMemcpy(h->currWaves, w, sizeof(w), cudaMemcpyHostToDevice));
    F.w = h->currWaves;
  }
  launch_currents(h->d, parts_of(h), F, h->S.simTime, h->P.currents, h->S.oceanR, h->S.coreR, dt, h->stream);
  return check_launch(h, 2);
}
static ws_status heat(ws_handle* h, double dt) {
  HeatParams hp;
  hp.hasSun = h->P.hasSun; hp.sun[0] = h->P.sunPos[0]; hp.sun[1] = h->P.sunPos[1]; hp.sun[2] = h->P.sunPos[2];
  hp.sunActivity = h->P.sunActivity; hp.Tamb = h->P.Tamb; hp.shadeCool = h->P.shadeCool; hp.heatK = h->P.heatK;
  hp.coreR = h->S.coreR;
  launch_heat(h->d, grid_of(h), parts_of(h), h->terr, hp, dt, h->cellCnt, h->cellSum, h->cellChange, h->stream);
  return check_launch(h, hp.heatK > 0 ? 5 : 2);
}
static ws_status contact_scratch(ws_handle* h) {
  if (h->contactScratch) return WS_OK;
  WS_TRY(cudaMalloc(&h->contactScratch, contacts_scratch_bytes(h->capacity, h->d.ny * h->d.nz)));
  return WS_OK;
}
static ws_status evaporation(ws_handle* h, double dt) {
  if (h->P.sunActivity <= 0 || h->P.evapIntensity <= 0) return WS_OK;
  double freezeT = std::max(h->P.meltT, h->P.snowT * 1.05);
  double rate = h->P.sunActivity * h->P.evapIntensity;
  if (evaporation_scratch_bytes(h->capacity) > contacts_scratch_bytes(h->capacity, h->d.ny * h->d.nz))
    return fail(h, WS_ERR_STATE, "evaporation scratch exceeds the shared contact scratch");
  ws_status s = contact_scratch(h); if (s) return s;
  uint32_t* evS = h->rng + 2;
  if (h->S.nP <= 0) { h->S.evapCount = 0; return WS_OK; }
  const EvapScratch es = evap_carve(h->contactScratch, h->capacity);
  launch_evap_prepare(h->d, grid_of(h), parts_of(h), freezeT, rate, dt, h->cand, h->blockCounts, h->list,
                      h->listCount, es, h->stream);
  s = check_launch(h, 5); if (s) return s;
  // Passes: one, unless a kick's u1 retry shifted the stream (about one kick in 10^9).
  int t0 = 0, eoff = 0, total = 0;
  const uint32_t* sStart = evS;
  for (;;) {
    launch_evap_pass(h->S.nP, h->list, h->listCount, es, t0, eoff, sStart, h->st, h->stream);
    s = check_launch(h, 5); if (s) return s;
    s = sync_status(h); if (s) return s;
    const DevStatus& hs = *h->stHost;
    if (hs.evIrr == ~0ull) {
      total = eoff + hs.evNEj;
      WS_TRY(cudaMemcpyAsync(evS, &h->st->evSEnd, sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream));
      break;
    }
    const int e = (int)(hs.evIrr >> 32), tr = (int)(hs.evIrr & 0xffffffffu), nC = hs.evNC;
    uint32_t q = 0;
    WS_TRY(cudaMemcpyAsync(&q, es.ejS + eoff + e, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    WS_TRY(cudaStreamSynchronize(h->stream));
    q = evap_kick_end(q);
    eoff += e + 1; t0 += tr + 1;
    if (t0 >= nC) {
      total = eoff;
      WS_TRY(cudaMemcpyAsync(evS, &q, sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
      WS_TRY(cudaStreamSynchronize(h->stream));
      break;
    }
    WS_TRY(cudaMemcpyAsync(&h->st->evSStart, &q, sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
    WS_TRY(cudaStreamSynchronize(h->stream));
    sStart = &h->st->evSStart;
  }
  launch_evap_apply(h->d, grid_of(h), parts_of(h), freezeT, es, total, h->stream);
  s = check_launch(h, total > 0 ? 1 : 0); if (s) return s;
  h->S.evapCount = total;
  if (total > 0) h->vaporPossible = true;
  return WS_OK;
}
static ws_status phase(ws_handle* h, double dt) {
  PhaseParams pp;
  double cloudT = h->P.cloudT;
  double rainT = std::min(h->P.rainT, cloudT - 0.02); if (rainT < 0) rainT = 0;
  double snowT = std::min(h->P.snowT, rainT - 0.02); if (snowT < 0) snowT = 0;
  pp.cloudT = cloudT; pp.cloudP = h->P.cloudP; pp.rainT = rainT; pp.snowT = snowT;
  pp.meltT = h->P.meltT > snowT * 1.05 ? h->P.meltT : snowT * 1.05;
  pp.rainLiftAge = h->P.rainLiftAge; pp.cloudBase = h->S.oceanR + 0.3 * h->P.atmosphereH;
  pp.dt = dt; pp.spinOn = h->P.spinOn; pp.tick = (uint32_t)(int)(h->S.simTime * 60);
  launch_phase(h->d, grid_of(h), parts_of(h), pp, h->cellCnt, h->stream);
  return check_launch(h, pp.spinOn && dt > 0 ? 3 : 2);
}
static ws_status push_surface(ws_handle* h) {
  launch_push_surface(h->d, grid_of(h), parts_of(h), h->terr, h->S.oceanR, h->S.coreR, h->P.atmosphereH, h->stream);
  return check_launch(h, 1);
}
static ws_status vapor_collisions(ws_handle* h) {
  double sunRel[3] = { h->P.sunPos[0] - h->d.cx, h->P.sunPos[1] - h->d.cy, h->P.sunPos[2] - h->d.cz };
  ws_status s0 = contact_scratch(h); if (s0) return s0;
  launch_vapor_collisions(h->d, parts_of(h), h->S.spacing, h->S.oceanR, h->P.spinOn, h->P.hasSun, sunRel,
                          h->contactScratch, contacts_scratch_bytes(h->capacity, h->d.ny * h->d.nz), h->st, h->stream);
  // the census lands in the status word; the caller reads it at its next
  // synchronisation (no kernel after this in the frame writes it)
  return check_launch(h, 1);
}
static void pull_vapor_census(ws_handle* h) {
  h->S.vaporCount = h->stHost->vaporCount; h->S.nightVaporCount = h->stHost->nightVapor;
}
static ws_status ice_contacts(ws_handle* h) {
  ws_status s0 = contact_scratch(h); if (s0) return s0;
  launch_ice_contacts(parts_of(h), h->S.spacing, h->contactScratch, contacts_scratch_bytes(h->capacity, h->d.ny * h->d.nz), h->stream);
  return check_launch(h, 1);
}

// _stepSync, js/solver.js:2670-2700
static ws_status step_frame(ws_handle* h, double dtFrame) {
  if (!h->hasTerrain) return fail(h, WS_ERR_STATE, "no terrain");
  cudaSetDevice(h->device);
  ws_status s;
  h->S.simTime += dtFrame;
  if (h->P.thermalOn && h->capacity > 1) {
    h->S.heatAcc = h->S.heatAcc + dtFrame;
    if (h->S.heatAcc >= 1.0 / 25) {
      double dtTick = std::min(h->S.heatAcc, 1.0 / 12);
      if ((s = heat(h, dtTick))) return s;
      if (h->P.sunActivity > 0) { if ((s = evaporation(h, dtTick))) return s; }
      if (h->P.currents > 0) { if ((s = currents(h, dtTick))) return s; }
      h->S.heatAcc = 0;
    }
  }
  double remaining = dtFrame; int guard = 0, nSub = 0;
  double base = dtFrame / std::max(1, h->P.substeps);
  // the grid clamp keeps umax <= 1.1 maxSpeed, so when even that speed leaves
  // the CFL term above min(base, 1/100) the substep dt needs no readback
  bool cflFree = (h->P.cfl * h->d.dx) / std::max(1.1 * h->P.maxSpeed, 0.08) >= std::min(base, 1.0 / 100);
  while (remaining > 1e-6 && guard < 10) {
    if (!cflFree && h->substepPending) { if ((s = sync_status(h))) return s; }
    double dt = std::min(std::min(base, (h->P.cfl * h->d.dx) / std::max(h->S.umax, 0.08)), 1.0 / 100);
    if (dt < 1e-5) dt = 1e-5;
    if ((s = substep(h, dt))) return s;
    remaining -= dt; guard++; nSub++;
  }
  h->S.substepsLast = nSub;
  if (h->P.thermalOn) {
    if ((s = vapor_collisions(h))) return s;
    if ((s = phase(h, dtFrame))) return s;
    if ((s = ice_contacts(h))) return s;
  }
  if ((s = push_surface(h))) return s;
  if ((s = sync_status(h))) return s;
  if (h->P.thermalOn) pull_vapor_census(h);
  return WS_OK;
}
extern "C" ws_status ws_step(ws_handle* h, double dtFrame) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !(dtFrame > 0)) return WS_ERR_INVALID;
  return step_frame(h, dtFrame);
}

// GpuSim.step's non-blocking contract (js/gpu/gpusim.js:328-339): the frame
// runs on a worker thread; a call while the previous frame is still running
// starts nothing (WS_BUSY, as GpuSim returns while _busy). ws_step_poll and
// ws_step_wait collect the frame's status; until then every other call on the
// handle returns WS_ERR_BUSY.
static void collect_async(ws_handle* h) {
  if (h->asyncThread.joinable()) h->asyncThread.join();
}
extern "C" ws_status ws_step_async(ws_handle* h, double dtFrame) {
  if (!h || !(dtFrame > 0)) return WS_ERR_INVALID;
  if (h->asyncRunning.load(std::memory_order_acquire)) return WS_BUSY;
  collect_async(h);
  h->asyncResult = WS_OK;
  h->asyncRunning.store(1, std::memory_order_release);
  try {
    h->asyncThread = std::thread([h, dtFrame] {
      ws_status s = step_frame(h, dtFrame);
      h->asyncResult = s;
      h->asyncRunning.store(0, std::memory_order_release);
    });
  } catch (...) {
    h->asyncRunning.store(0, std::memory_order_release);
    return fail(h, WS_ERR_NOMEM, "cannot start the step thread");
  }
  return WS_OK;
}
extern "C" ws_status ws_step_poll(ws_handle* h, int32_t* done) {
  if (!h || !done) return WS_ERR_INVALID;
  if (h->asyncRunning.load(std::memory_order_acquire)) { *done = 0; return WS_OK; }
  collect_async(h);
  *done = 1;
  return h->asyncResult;
}
extern "C" ws_status ws_step_wait(ws_handle* h) {
  if (!h) return WS_ERR_INVALID;
  collect_async(h);
  return h->asyncResult;
}

extern "C" ws_status ws_stage(ws_handle* h, int32_t stage, double dt) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  ws_status s = WS_OK;
  force_full_pass(h);                            // a stage alone runs over the whole grid
  switch (stage) {
    case WS_STAGE_CLEAR_RASTER: s = stage_clear_raster(h); break;
    case WS_STAGE_MARK_FLUID: s = stage_mark(h); break;
    case WS_STAGE_P2G: s = stage_p2g(h); break;
    case WS_STAGE_FORCES:
      s = ensure_gravity(h); if (s) return s;
      s = stage_forces(h, dt, gravity_scale(h, dt)); break;
    case WS_STAGE_PRESSURE:
      s = stage_pressure(h); if (s) return s;
      s = sync_status(h); if (s) return s;
      pressure_diagnostics(h);
      return WS_OK;
    case WS_STAGE_PROJECT: s = stage_project(h, false); break;
    case WS_STAGE_VORTICITY: s = stage_vorticity(h, dt); break;
    case WS_STAGE_CLAMP:
      s = stage_clamp(h); if (s) return s;
      s = sync_status(h); if (s) return s;
      h->S.umax = (double)bits_to_float(h->stHost->umaxBits);
      return WS_OK;
    case WS_STAGE_EXTRAPOLATE: s = stage_extrapolate(h); break;
    case WS_STAGE_G2P_ADVECT:
      s = stage_g2p_advect(h, dt); if (s) return s;
      s = sync_status(h); if (s) return s;
      h->S.airborneCount = h->stHost->airborne; h->S.dtLast = dt;
      return WS_OK;
    case WS_STAGE_HEAT: s = heat(h, dt); break;
    case WS_STAGE_EVAPORATION: s = evaporation(h, dt); break;
    case WS_STAGE_PHASE: s = phase(h, dt); break;
    case WS_STAGE_PUSH_SURFACE: s = push_surface(h); break;
    case WS_STAGE_SPLAT:
      launch_splat(h->d, grid_of(h), parts_of(h), h->S.spacing, h->stream);
      s = check_launch(h, 1); break;
    case WS_STAGE_VAPOR_COLLISIONS: s = vapor_collisions(h); break;
    case WS_STAGE_ICE_CONTACTS: s = ice_contacts(h); break;
    case WS_STAGE_CURRENTS: s = currents(h, dt); break;
    default: return fail(h, WS_ERR_INVALID, "unknown stage");
  }
  if (s) return s;
  if ((s = sync_status(h))) return s;
  if (stage == WS_STAGE_VAPOR_COLLISIONS) pull_vapor_census(h);
  return WS_OK;
}

// ------------------------------------------------------------ balls
// addBall (js/solver.js:3910-3912) and the ball list the app reads back
// (x y z vx vy vz r rho submerged, js/main.js:713 and the scene's ball meshes)
static_assert(WS_MAX_BALLS == WS_MAX_BALLS_DEV && sizeof(ws_ball) == 9 * sizeof(double), "ball layout");
static ws_status ensure_balls(ws_handle* h) {
  if (h->balls) return WS_OK;
  const size_t N = (size_t)h->d.nCells;
  WS_TRY(cudaMalloc(&h->balls, sizeof(ws_ball) * WS_MAX_BALLS));
  WS_TRY(cudaMalloc(&h->sv, sizeof(float) * 3 * N));
  WS_TRY(cudaMalloc(&h->ballHist, sizeof(int) * (WS_MAX_BALLS * 24 + WS_MAX_BALLS)));
  WS_TRY(cudaMalloc(&h->ballSurf, sizeof(float) * WS_MAX_BALLS));
  WS_TRY(cudaMemsetAsync(h->sv, 0, sizeof(float) * 3 * N, h->stream));
  WS_TRY(cudaMemsetAsync(h->ballHist, 0, sizeof(int) * (WS_MAX_BALLS * 24 + WS_MAX_BALLS), h->stream));
  drop_graph(h);                                 // the BC kernels now read the solid-velocity field
  return WS_OK;
}
extern "C" ws_status ws_add_ball(ws_handle* h, double x, double y, double z, double r, double rho) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  if (!(r > 0) || !(rho > 0)) return fail(h, WS_ERR_INVALID, "ball radius and density must be positive");
  if (h->nBalls >= WS_MAX_BALLS) return fail(h, WS_ERR_RANGE, "too many balls");
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  if ((s = ensure_balls(h))) return s;
  ws_ball b{ x, y, z, 0, 0, 0, r, rho, 0 };
  WS_TRY(cudaMemcpyAsync(h->balls + 9 * h->nBalls, &b, sizeof(b), cudaMemcpyHostToDevice, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  h->nBalls++;
  return WS_OK;
}
extern "C" ws_status ws_get_balls(ws_handle* h, ws_ball* out, int32_t max, int32_t* count) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !count || (max > 0 && !out)) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  *count = h->nBalls;
  const int n = std::min(max, h->nBalls);
  if (n > 0) WS_TRY(cudaMemcpy(out, h->balls, sizeof(ws_ball) * (size_t)n, cudaMemcpyDeviceToHost));
  return WS_OK;
}
extern "C" ws_status ws_set_balls(ws_handle* h, const ws_ball* in, int32_t count) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || count < 0 || (count > 0 && !in)) return WS_ERR_INVALID;
  if (count > WS_MAX_BALLS) return fail(h, WS_ERR_RANGE, "too many balls");
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  if (count > 0) {
    if ((s = ensure_balls(h))) return s;
    WS_TRY(cudaMemcpyAsync(h->balls, in, sizeof(ws_ball) * (size_t)count, cudaMemcpyHostToDevice, h->stream));
    WS_TRY(cudaStreamSynchronize(h->stream));
  }
  h->nBalls = count;
  return WS_OK;
}

// ------------------------------------------------------------ interactions
extern "C" ws_status ws_apply_impulse_sphere(ws_handle* h, double cx, double cy, double cz, double R,
                                             double fx, double fy, double fz) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  launch_impulse_sphere(parts_of(h), cx, cy, cz, R, fx, fy, fz, h->stream);
  ws_status s = check_launch(h, 1); if (s) return s;
  return sync_status(h);
}
extern "C" ws_status ws_stir_at(ws_handle* h, double cx, double cy, double cz, double vx, double vy,
                                double vz, double R, double dt) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  launch_stir_at(parts_of(h), cx, cy, cz, vx, vy, vz, R, dt, h->stream);
  ws_status s = check_launch(h, 1); if (s) return s;
  return sync_status(h);
}
// waveImpulse (js/solver.js:3866-3892), sphere mode, on the seeded stir
// stream: theta and phi of the bulge direction, then one draw per particle.
extern "C" ws_status ws_wave_impulse(ws_handle* h, double dvx) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !std::isfinite(dvx)) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  uint32_t st = h->S.stirS;
  st = lcg_next(st); const double th = st / 4294967296.0 * M_PI * 2;
  st = lcg_next(st); const double ph = std::acos(2 * (st / 4294967296.0) - 1);
  const double dir[3] = { std::sin(ph) * std::cos(th), std::cos(ph), std::sin(ph) * std::sin(th) };
  launch_wave_impulse(h->d, parts_of(h), dir, st, dvx, h->stream);
  h->S.stirS = lcg_jump(st, (uint32_t)h->S.nP);
  ws_status s = check_launch(h, 1); if (s) return s;
  return sync_status(h);
}
// dryLandFraction (js/solver.js:3593-3623) of the current cell types; 0
// without terrain, as the reference
extern "C" ws_status ws_dry_land_fraction(ws_handle* h, double* out) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !out) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  if (!h->terr.has) { *out = 0; return WS_OK; }
  int* dry = reinterpret_cast<int*>(h->red);
  launch_dry_land(h->d, h->terr, h->type, h->S.oceanR, dry, h->stream);
  ws_status s = check_launch(h, 1); if (s) return s;
  int n = 0;
  WS_TRY(cudaMemcpyAsync(&n, dry, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if ((s = sync_status(h))) return s;
  *out = n / 1200.0;
  return WS_OK;
}
// points: n (x, y, z) triples of host doubles -> n results; staged through
// the handle's scratch in chunks of kQueryChunk points
static const long long kQueryChunk = 1 << 16;
static ws_status query_points(ws_handle* h, const double* xyz, int64_t n, double* out, int perPoint, int kind) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || n < 0 || (n > 0 && (!xyz || !out))) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  if (!h->queryBuf) WS_TRY(cudaMalloc(&h->queryBuf, sizeof(double) * 6 * kQueryChunk));
  double* din = h->queryBuf;
  double* dout = h->queryBuf + 3 * kQueryChunk;
  for (long long b = 0; b < n; b += kQueryChunk) {
    const long long m = std::min<long long>(kQueryChunk, n - b);
    WS_TRY(cudaMemcpyAsync(din, xyz + 3 * b, sizeof(double) * 3 * m, cudaMemcpyHostToDevice, h->stream));
    if (kind == 0) launch_sample_vel(h->d, h->vel, din, m, dout, h->stream);
    else launch_terrain_radius(h->terr, h->S.coreR, din, m, dout, h->stream);
    ws_status s = check_launch(h, 1); if (s) return s;
    WS_TRY(cudaMemcpyAsync(out + perPoint * b, dout, sizeof(double) * perPoint * m, cudaMemcpyDeviceToHost, h->stream));
  }
  return sync_status(h);
}
// sampleVel (js/solver.js:811-854) at n points: u, v, w per point
extern "C" ws_status ws_sample_vel(ws_handle* h, const double* xyz, int64_t n, double* uvw) {
  return query_points(h, xyz, n, uvw, 3, 0);
}
// terrainRadiusAt (js/solver.js:512-535) at n points
extern "C" ws_status ws_terrain_radius_at(ws_handle* h, const double* xyz, int64_t n, double* radius) {
  return query_points(h, xyz, n, radius, 1, 1);
}
// oceanPoint (js/solver.js:591-608) on the seeded stir stream
extern "C" ws_status ws_ocean_point(ws_handle* h, double minDepth, double* xyz) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !xyz) return WS_ERR_INVALID;
  if (!h->terr.has) return fail(h, WS_ERR_STATE, "oceanPoint needs terrain");
  cudaSetDevice(h->device);
  const double need = minDepth ? minDepth : 0.12;            // `minDepth || 0.12`
  double* dout = reinterpret_cast<double*>(h->red);
  launch_ocean_point(h->d, h->terr, h->S.coreR, h->S.oceanR, need, h->S.stirS, dout, h->stream);
  ws_status s = check_launch(h, 1); if (s) return s;
  double r[4];
  WS_TRY(cudaMemcpyAsync(r, dout, sizeof r, cudaMemcpyDeviceToHost, h->stream));
  if ((s = sync_status(h))) return s;
  xyz[0] = r[0]; xyz[1] = r[1]; xyz[2] = r[2];
  h->S.stirS = lcg_jump(h->S.stirS, 2u * (uint32_t)r[3]);
  return WS_OK;
}

// Seeded Gaussian stir kick: the draw order (u1, theta, phi from stirS) and
// the tangent construction are part of the workload definition.
extern "C" ws_status ws_stir_gaussian(ws_handle* h, double sigma, double peak) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !(sigma > 0)) return WS_ERR_INVALID;
  uint32_t st = h->S.stirS;
  st = lcg_next(st); double u1 = st / 4294967296.0 * 2 - 1;
  st = lcg_next(st); double th = st / 4294967296.0 * 6.283185307179586;
  st = lcg_next(st); double ph = st / 4294967296.0 * 6.283185307179586;
  h->S.stirS = st;
  double sq = std::sqrt(1 - u1 * u1);
  double dxn = sq * std::cos(th), dyn = u1, dzn = sq * std::sin(th);
  double ax = 0, ay = 1, az = 0;
  if (std::fabs(dyn) > 0.9) { ax = 1; ay = 0; }
  double e1x = dyn * az - dzn * ay, e1y = dzn * ax - dxn * az, e1z = dxn * ay - dyn * ax;
  double e1l = std::sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
  e1x /= e1l; e1y /= e1l; e1z /= e1l;
  double e2x = dyn * e1z - dzn * e1y, e2y = dzn * e1x - dxn * e1z, e2z = dxn * e1y - dyn * e1x;
  double cph = std::cos(ph), sph = std::sin(ph);
  double tx = cph * e1x + sph * e2x, ty = cph * e1y + sph * e2y, tz = cph * e1z + sph * e2z;
  double R = h->S.oceanR;
  launch_stir_gaussian(parts_of(h), h->d.cx + dxn * R, h->d.cy + dyn * R, h->d.cz + dzn * R, tx, ty, tz, sigma, peak, h->stream);
  return check_launch(h, 1);
}

extern "C" ws_status ws_synchronize(ws_handle* h) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  return sync_status(h);
}
extern "C" ws_status ws_get_stream(ws_handle* h, void** s) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !s) return WS_ERR_INVALID;
  *s = (void*)h->stream;
  return WS_OK;
}
extern "C" ws_status ws_launch_count(ws_handle* h, int64_t* n) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !n) return WS_ERR_INVALID;
  *n = h->launches;
  return WS_OK;
}

// One device thread waits, with the library's bounded wait, for a status
// word that nothing sets (DevStatus::pad stays zero).
__global__ void k_probe_wait(DevStatus* st, long long polls) {
  bounded_wait_geq(reinterpret_cast<const unsigned*>(&st->pad), 1u, polls, &st->err);
}
extern "C" ws_status ws_probe_wait(ws_handle* h, int64_t polls) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || polls < 1 || polls > 100000000) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  k_probe_wait<<<1, 1, 0, h->stream>>>(h->st, (long long)polls);
  s = check_launch(h, 1); if (s) return s;
  return sync_status(h);
}

extern "C" ws_status ws_time_kernel(ws_handle* h, int32_t kernel, int32_t reps, double* us) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !us || reps < 1) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  force_full_pass(h);
  cudaEvent_t e0, e1;
  WS_TRY(cudaEventCreate(&e0));
  WS_TRY(cudaEventCreate(&e1));
  GridDev g = grid_of(h);
  int perRep = 1;
  WS_TRY(cudaEventRecord(e0, h->stream));
  for (int r = 0; r < reps; r++) {
    switch (kernel) {
      case 0: launch_sor_color(h->d, g, 0, 1 - h->P.omega, h->stream);
              launch_sor_color(h->d, g, 1, 1 - h->P.omega, h->stream); perRep = 2; break;
      case 1: launch_p2g(h->d, g, parts_of(h), h->st, h->stream); break;
      case 2: { AdvectParams ap = advect_params(h, h->S.dtLast > 0 ? h->S.dtLast : 0.01);
                launch_g2p_advect(h->d, g, parts_of(h), h->terr, ap, h->st, h->stream); } break;
      case 3: launch_faces_normalize_bc(h->d, g, h->stream); break;
      case 4: launch_faces_forces(h->d, g, 5e-6, 1, 0.01, 9.81, h->stream); break;
      case 5: launch_project(h->d, g, 1, h->P.maxSpeed, h->st, h->stream); break;
      case 6: { int* di; double* dr; int* dp;
                cudaError_t e6 = launch_sor_solve(h->sor, h->d, g, h->diag8, h->P.omega, h->P.pressureIters, 0, 0,
                                                  &h->st->err, &di, &dr, &dp, h->stream);
                if (e6 != cudaSuccess) { cudaEventDestroy(e0); cudaEventDestroy(e1); return fail_cuda(h, e6, "SOR solve"); }
                h->launches += sor_solve_launches(h->sor) - 1; } break;   // list build; timed per whole solve
      case 8: launch_faces_normalize_bc_bricks(h->d, g, h->bricks, h->stream); break;
      case 9: launch_faces_forces_bricks(h->d, g, h->bricks, 5e-6, 1, 0.01, 9.81, h->stream); break;
      case 10: launch_project_bricks(h->d, g, h->bricks, 1, h->P.maxSpeed, h->st, h->stream); break;
      case 11: launch_extrapolate_bricks(h->d, g, h->bricks, h->stream); break;
      case 12: { const int n12 = launch_p2g_sorted(h->d, g, parts_of(h), h->csort, h->bricks, false, h->csortCub,
                                                   h->csortCubBytes, h->st, h->stream);
                 if (n12 < 0) { cudaEventDestroy(e0); cudaEventDestroy(e1); return fail_cuda(h, cudaGetLastError(), "cell sort"); }
                 h->launches += n12 - 1; } break;
      case 7: { int* di; double* dr; int* dp;
                cudaError_t e7 = launch_sor_solve_lists(h->sor, h->d, g, h->diag8, h->P.omega, h->P.pressureIters, 0, 0,
                                                        &h->st->err, &di, &dr, &dp, h->stream);
                if (e7 != cudaSuccess) { cudaEventDestroy(e0); cudaEventDestroy(e1); return fail_cuda(h, e7, "SOR solve"); }
                h->launches += sor_list_solve_launches(h->sor) - 1; } break;
      default: cudaEventDestroy(e0); cudaEventDestroy(e1); return fail(h, WS_ERR_INVALID, "unknown kernel id");
    }
  }
  WS_TRY(cudaEventRecord(e1, h->stream));
  ws_status s = check_launch(h, reps * perRep); if (s) return s;
  WS_TRY(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0); cudaEventDestroy(e1);
  *us = 1000.0 * ms / (reps * perRep);
  return sync_status(h);
}

// ------------------------------------------------------------ learned warm start
static ws_status net_ready(ws_handle* h) {
  if (!h) return WS_ERR_INVALID;
  if (!h->net) return fail(h, WS_ERR_STATE, "warm-start network not initialised: call ws_unet_init");
  cudaSetDevice(h->device);
  return sync_status(h);
}
extern "C" ws_status ws_unet_init_levels(ws_handle* h, uint32_t seed, int32_t levels) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  if (levels < 3 || levels > unet::kMaxLevels) return fail(h, WS_ERR_INVALID, "levels must be 3 or 4");
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  if (h->net && h->net->levels != levels) {        // a different depth: a new network (its pairs go too)
    h->unetOn = false; h->unetCollect = false;
    h->net->destroy(); delete h->net; h->net = nullptr;
    h->gsig.unet = -1;                             // recapture the substep graph
  }
  if (!h->net) {
    h->net = new (std::nothrow) unet::Net();
    if (!h->net) return fail(h, WS_ERR_NOMEM, "warm-start network");
    cudaError_t e = h->net->create(h->d, levels);
    if (e != cudaSuccess) { h->net->destroy(); delete h->net; h->net = nullptr; return fail_cuda(h, e, "warm-start network buffers"); }
  }
  WS_TRY(h->net->init_weights(seed, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  return WS_OK;
}
extern "C" ws_status ws_unet_init(ws_handle* h, uint32_t seed) { return ws_unet_init_levels(h, seed, 3); }
extern "C" ws_status ws_unet_collect(ws_handle* h, int32_t capacity) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (capacity < 0) return fail(h, WS_ERR_RANGE, "negative pair capacity");
  if (capacity > 0) {
    cudaError_t e = h->net->reserve_pairs(capacity, h->type, h->stream);
    if (e != cudaSuccess) return fail_cuda(h, e, "pair store");
  }
  h->unetCollect = capacity > 0;
  return WS_OK;
}
extern "C" ws_status ws_unet_enable(ws_handle* h, int32_t on) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (on && !(h->net->gain > 0)) return fail(h, WS_ERR_STATE, "network has no output gain: train it or call ws_unet_set_gain");
  h->unetOn = on != 0;
  return WS_OK;
}
extern "C" ws_status ws_unet_train(ws_handle* h, int32_t steps, int32_t batch, double lr, uint32_t seed,
                                   double* mean_loss) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (h->net->pairsStored <= 0) return fail(h, WS_ERR_STATE, "no training pairs stored");
  if (steps < 0 || batch < 1 || !(lr >= 0)) return fail(h, WS_ERR_INVALID, "bad training arguments");
  cudaError_t e = h->net->train(steps, batch, lr, seed, mean_loss, h->stream);
  if (e != cudaSuccess) return fail_cuda(h, e, "warm-start training");
  int derr = 0;
  WS_TRY(cudaMemcpy(&derr, h->net->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (derr) return fail(h, WS_ERR_TIMEOUT, "tensor-core convolution timed out");
  return WS_OK;
}
extern "C" ws_status ws_unet_get_info(ws_handle* h, ws_unet_info* out) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !out) return WS_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  if (!h->net) return WS_OK;
  out->pairs_stored = h->net->pairsStored; out->pairs_capacity = h->net->pairCap;
  out->train_steps = h->net->trainSteps; out->num_weights = h->net->nparams;
  out->gain = h->net->gain; out->last_loss = h->net->lastLoss;
  out->enabled = h->unetOn; out->collecting = h->unetCollect;
  return WS_OK;
}
extern "C" ws_status ws_unet_get_weights(ws_handle* h, float* host, int64_t count) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!host || count != h->net->nparams) return fail(h, WS_ERR_RANGE, "weight count mismatch");
  WS_TRY(cudaMemcpy(host, h->net->params, sizeof(float) * count, cudaMemcpyDeviceToHost));
  return WS_OK;
}
extern "C" ws_status ws_unet_set_weights(ws_handle* h, const float* host, int64_t count) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!host || count != h->net->nparams) return fail(h, WS_ERR_RANGE, "weight count mismatch");
  WS_TRY(h->net->set_weights(host, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  return WS_OK;
}
extern "C" ws_status ws_unet_set_gain(ws_handle* h, double gain) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!(gain > 0)) return fail(h, WS_ERR_INVALID, "gain must be positive");
  WS_TRY(h->net->set_gain(gain, h->stream));
  return WS_OK;
}
extern "C" ws_status ws_unet_get_pair(ws_handle* h, int32_t idx, float* r0n, uint8_t* types, float* target) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  unet::Net& n = *h->net;
  if (idx < 0 || idx >= n.stored()) return fail(h, WS_ERR_RANGE, "pair index");
  WS_TRY(n.get_pair(idx, r0n, types, target, h->stream));
  return WS_OK;
}
extern "C" ws_status ws_unet_put_pair(ws_handle* h, const float* r0n, const uint8_t* types, const float* target) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  unet::Net& n = *h->net;
  if (!r0n || !types || !target) return WS_ERR_INVALID;
  cudaError_t e = n.put_pair(r0n, types, target, h->stream);
  if (e == cudaErrorInvalidValue) return fail(h, WS_ERR_RANGE, "the pair has more active tiles than a pair slot holds");
  if (e != cudaSuccess) return fail_cuda(h, e, "pair store");
  return WS_OK;
}
extern "C" ws_status ws_unet_forward_pair(ws_handle* h, int32_t idx, float* out) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!out || idx < 0 || idx >= std::min(h->net->pairsStored, h->net->pairCap)) return fail(h, WS_ERR_RANGE, "pair index");
  WS_TRY(h->net->forward_pair(idx, out, h->stream));
  return WS_OK;
}
extern "C" ws_status ws_unet_grad_pair(ws_handle* h, int32_t idx, float* grads, double* loss) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!grads || idx < 0 || idx >= std::min(h->net->pairsStored, h->net->pairCap)) return fail(h, WS_ERR_RANGE, "pair index");
  WS_TRY(h->net->grad_pair(idx, grads, loss, h->stream));
  return WS_OK;
}
// relative residual of q before and after the prediction, on the pressure
// system of the current face velocities (call after the forces stage)
extern "C" ws_status ws_unet_probe(ws_handle* h, double* relres_prev, double* relres_pred) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!(h->net->gain > 0)) return fail(h, WS_ERR_STATE, "network has no output gain");
  GridDev g = grid_of(h);
  launch_pressure_setup(h->d, g, h->diag8, h->P.omega, h->st, sor_block_counts(h->sor), h->stream);
  if ((s = check_launch(h, 1))) return s;
  launch_residual(h->d, g, h->diag8, h->partials, h->st, nullptr, h->stream);
  if ((s = check_launch(h, 2))) return s;
  if ((s = sync_status(h))) return s;
  if (relres_prev) *relres_prev = h->stHost->relres;
  WS_TRY(h->net->predict(h->q, h->rhs, h->diag8, h->type, h->stream));
  launch_residual(h->d, g, h->diag8, h->partials, h->st, nullptr, h->stream);
  if ((s = check_launch(h, 2))) return s;
  if ((s = sync_status(h))) return s;
  if (relres_pred) *relres_pred = h->stHost->relres;
  return WS_OK;
}
// device time of `what`: 0 the prediction on the current pressure system
// (writes q), 1 one training step on a stored pair (batch 1, learning rate 0)
extern "C" ws_status ws_unet_time(ws_handle* h, int32_t what, int32_t reps, double* ms) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!ms || reps < 1 || what < 0 || what > 1) return WS_ERR_INVALID;
  if (what == 1 && h->net->pairsStored <= 0) return fail(h, WS_ERR_STATE, "no training pairs stored");
  cudaEvent_t a, b;
  WS_TRY(cudaEventCreate(&a)); WS_TRY(cudaEventCreate(&b));
  WS_TRY(cudaEventRecord(a, h->stream));
  for (int r = 0; r < reps; r++) {
    cudaError_t e = what == 0 ? h->net->predict(h->q, h->rhs, h->diag8, h->type, h->stream)
                              : h->net->train(1, 1, 0.0, 7u + r, nullptr, h->stream);
    if (e != cudaSuccess) { cudaEventDestroy(a); cudaEventDestroy(b); return fail_cuda(h, e, "warm-start timing"); }
  }
  WS_TRY(cudaEventRecord(b, h->stream));
  WS_TRY(cudaEventSynchronize(b));
  float t = 0;
  cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a); cudaEventDestroy(b);
  *ms = t / reps;
  return WS_OK;
}

// ---- data-parallel training: each rank accumulates the gradients of its own
// samples, the caller sums the FP32 gradient buffer over the ranks (an
// all-reduce on its communicator), then every rank applies the same step
extern "C" ws_status ws_unet_accumulate(ws_handle* h, int32_t samples, uint32_t seed, double* loss_sum) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (h->net->pairsStored <= 0) return fail(h, WS_ERR_STATE, "no training pairs stored");
  if (samples < 1) return fail(h, WS_ERR_INVALID, "samples must be positive");
  WS_TRY(h->net->accumulate(samples, seed, h->stream));
  double L = 0;
  WS_TRY(h->net->loss_sum(&L, h->stream));
  if (loss_sum) *loss_sum = L;
  return WS_OK;
}
extern "C" ws_status ws_unet_grads(ws_handle* h, void** device_ptr, int64_t* count) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!device_ptr || !count) return WS_ERR_INVALID;
  *device_ptr = h->net->grads;
  *count = h->net->nparams;
  return WS_OK;
}
extern "C" ws_status ws_unet_apply(ws_handle* h, double lr, int32_t total_samples) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (total_samples < 1 || !(lr >= 0)) return fail(h, WS_ERR_INVALID, "bad learning rate or sample count");
  WS_TRY(h->net->apply(lr, total_samples, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  return WS_OK;
}

// ------------------------------------------------------------ snapshot / restore
// A self-describing host blob of the whole solver state: header, knobs,
// scalars (RNG streams included), the 16 particle fields (nP each), the
// pressure q (the next solve's warm start) and the terrain. Grid fields are
// rebuilt from the particles by the next substep, so they are not stored.
namespace {
constexpr char kSnapMagic[8] = { 'W', 'S', 'S', 'N', 'A', 'P', '0', '1' };
struct SnapHeader {
  char magic[8];
  uint32_t version, headerBytes;
  int32_t nx, ny, nz, nP, terrainN, nBalls;     // nBalls: 0 in version 1
  double dx;
  int64_t totalBytes;
  double Rsl, Rlo, Rhi, landFrac, dv;
};
int64_t snap_bytes(const ws_handle* h, int terrainN) {
  const int64_t nP = h->S.nP, N = h->d.nCells, n3 = (int64_t)terrainN * terrainN * terrainN;
  return (int64_t)sizeof(SnapHeader) + (int64_t)sizeof(ws_params) + (int64_t)sizeof(ws_scalars) +
         nP * (13 * 4 + 3) + N * 4 + n3 * 5 + (int64_t)h->nBalls * (int64_t)sizeof(ws_ball);
}
}  // namespace

extern "C" ws_status ws_snapshot(ws_handle* h, void* buf, int64_t capacity, int64_t* size) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !size) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  const int tn = h->hasTerrain ? h->hostTerrain.n : 0;
  const int64_t need = snap_bytes(h, tn);
  *size = need;
  if (!buf) return WS_OK;                              // size query
  if (capacity < need) return fail(h, WS_ERR_RANGE, "snapshot buffer too small");
  unsigned char* p = (unsigned char*)buf;
  SnapHeader hd{};
  std::memcpy(hd.magic, kSnapMagic, 8);
  hd.version = 2; hd.headerBytes = sizeof(SnapHeader);
  hd.nx = h->d.nx; hd.ny = h->d.ny; hd.nz = h->d.nz; hd.nP = h->S.nP; hd.terrainN = tn; hd.dx = h->d.dx;
  hd.nBalls = h->nBalls;
  hd.totalBytes = need;
  if (tn) { const auto& T = h->hostTerrain; hd.Rsl = T.Rsl; hd.Rlo = T.Rlo; hd.Rhi = T.Rhi; hd.landFrac = T.landFrac; hd.dv = T.dv; }
  std::memcpy(p, &hd, sizeof hd); p += sizeof hd;
  std::memcpy(p, &h->P, sizeof(ws_params)); p += sizeof(ws_params);
  std::memcpy(p, &h->S, sizeof(ws_scalars)); p += sizeof(ws_scalars);
  const int64_t nP = h->S.nP;
  for (int f = WS_F_PX; f <= WS_F_PDEPTH; f++) {
    FieldRef r; field_ref(h, (ws_field)f, r);
    WS_TRY(cudaMemcpyAsync(p, r.ptr, (size_t)(nP * r.elem), cudaMemcpyDeviceToHost, h->stream));
    p += nP * r.elem;
  }
  WS_TRY(cudaMemcpyAsync(p, h->q, sizeof(float) * (size_t)h->d.nCells, cudaMemcpyDeviceToHost, h->stream));
  p += 4 * h->d.nCells;
  WS_TRY(cudaStreamSynchronize(h->stream));
  if (tn) {
    const auto& T = h->hostTerrain;
    const size_t n3 = (size_t)tn * tn * tn;
    std::memcpy(p, T.solid.data(), n3); p += n3;
    std::memcpy(p, T.R.data(), 4 * n3); p += 4 * n3;
  }
  if (h->nBalls) WS_TRY(cudaMemcpy(p, h->balls, sizeof(ws_ball) * (size_t)h->nBalls, cudaMemcpyDeviceToHost));
  return WS_OK;
}

extern "C" ws_status ws_restore(ws_handle* h, const void* buf, int64_t size) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !buf) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  if (size < (int64_t)sizeof(SnapHeader)) return fail(h, WS_ERR_INVALID, "not a snapshot");
  force_full_pass(h);                            // q and the terrain come back
  SnapHeader hd;
  std::memcpy(&hd, buf, sizeof hd);
  if (std::memcmp(hd.magic, kSnapMagic, 8) != 0 || (hd.version != 1 && hd.version != 2) ||
      hd.headerBytes != sizeof(SnapHeader))
    return fail(h, WS_ERR_INVALID, "not a version-1 or -2 snapshot");
  if (hd.nBalls < 0 || hd.nBalls > WS_MAX_BALLS || (hd.version == 1 && hd.nBalls != 0))
    return fail(h, WS_ERR_INVALID, "bad ball count");
  if (hd.nx != h->d.nx || hd.ny != h->d.ny || hd.nz != h->d.nz || hd.dx != h->d.dx)
    return fail(h, WS_ERR_INVALID, "snapshot grid differs from this handle's");
  if (hd.nP < 0 || hd.nP > h->capacity) return fail(h, WS_ERR_RANGE, "snapshot holds more particles than the capacity");
  if (hd.terrainN < 0 || hd.terrainN > 4096) return fail(h, WS_ERR_INVALID, "bad terrain size");
  // the knobs and scalars follow the header: a blob cut short before them is refused before they are read
  if (size < (int64_t)(sizeof hd + sizeof(ws_params) + sizeof(ws_scalars)))
    return fail(h, WS_ERR_INVALID, "snapshot size mismatch");
  ws_scalars S;
  std::memcpy(&S, (const unsigned char*)buf + sizeof hd + sizeof(ws_params), sizeof S);
  const int64_t nP = hd.nP, N = h->d.nCells, n3 = (int64_t)hd.terrainN * hd.terrainN * hd.terrainN;
  const int64_t need = (int64_t)sizeof hd + (int64_t)sizeof(ws_params) + (int64_t)sizeof(ws_scalars) +
                       nP * (13 * 4 + 3) + N * 4 + n3 * 5 + (int64_t)hd.nBalls * (int64_t)sizeof(ws_ball);
  if (size != need || hd.totalBytes != need || S.nP != hd.nP) return fail(h, WS_ERR_INVALID, "snapshot size mismatch");
  const unsigned char* p = (const unsigned char*)buf + sizeof hd;
  const unsigned char* fields = p + sizeof(ws_params) + sizeof(ws_scalars);
  const unsigned char* qp = fields + nP * (13 * 4 + 3);
  if (hd.terrainN) {
    ws_terrain t;
    t.n = hd.terrainN; t.dv = hd.dv; t.Rsl = hd.Rsl; t.Rlo = hd.Rlo; t.Rhi = hd.Rhi; t.landFrac = hd.landFrac;
    t.solid = qp + 4 * N;
    t.R = (const float*)(qp + 4 * N + n3);
    if ((s = ws_upload_terrain(h, &t))) return s;
  }
  if ((s = ws_set_params(h, (const ws_params*)p))) return s;
  if ((s = ws_set_scalars(h, &S))) return s;
  ws_host_arrays a{};
  a.count = nP;
  const unsigned char* f = fields;
  for (int k = WS_F_PX; k <= WS_F_PDEPTH; k++) {
    a.field[k] = const_cast<unsigned char*>(f);
    f += nP * (k <= WS_F_PPH ? 4 : 1);
  }
  if ((s = ws_upload_state(h, &a))) return s;
  WS_TRY(cudaMemcpyAsync(h->q, qp, sizeof(float) * (size_t)N, cudaMemcpyHostToDevice, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  // the balls (version 2) follow the terrain; their solid cells are rebuilt
  // by the next substep's raster
  return ws_set_balls(h, (const ws_ball*)(qp + 4 * N + n3 * 5), hd.nBalls);
}

// network blob: header, gain, Adam step count, then params, Adam m and v (FP32)
extern "C" ws_status ws_unet_save(ws_handle* h, void* buf, int64_t capacity, int64_t* size) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!size) return WS_ERR_INVALID;
  const int64_t n = h->net->nparams, need = 8 + 8 + 8 + 8 + 3 * 4 * n;
  *size = need;
  if (!buf) return WS_OK;
  if (capacity < need) return fail(h, WS_ERR_RANGE, "network buffer too small");
  unsigned char* p = (unsigned char*)buf;
  std::memcpy(p, "WSUNET01", 8); p += 8;
  std::memcpy(p, &n, 8); p += 8;
  std::memcpy(p, &h->net->gain, 8); p += 8;
  const int64_t steps = h->net->adamStep;
  std::memcpy(p, &steps, 8); p += 8;
  WS_TRY(cudaMemcpy(p, h->net->params, 4 * n, cudaMemcpyDeviceToHost)); p += 4 * n;
  WS_TRY(cudaMemcpy(p, h->net->adm, 4 * n, cudaMemcpyDeviceToHost)); p += 4 * n;
  WS_TRY(cudaMemcpy(p, h->net->adv, 4 * n, cudaMemcpyDeviceToHost));
  return WS_OK;
}
extern "C" ws_status ws_unet_load(ws_handle* h, const void* buf, int64_t size) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  ws_status s = net_ready(h); if (s) return s;
  if (!buf) return WS_ERR_INVALID;
  const int64_t n = h->net->nparams;
  if (size != 32 + 12 * n || std::memcmp(buf, "WSUNET01", 8) != 0) return fail(h, WS_ERR_INVALID, "not a network of this layout");
  const unsigned char* p = (const unsigned char*)buf + 8;
  int64_t n2, steps; double gain;
  std::memcpy(&n2, p, 8); std::memcpy(&gain, p + 8, 8); std::memcpy(&steps, p + 16, 8);
  if (n2 != n) return fail(h, WS_ERR_INVALID, "parameter count differs");
  p += 24;
  WS_TRY(cudaMemcpy(h->net->adm, p + 4 * n, 4 * n, cudaMemcpyHostToDevice));
  WS_TRY(cudaMemcpy(h->net->adv, p + 8 * n, 4 * n, cudaMemcpyHostToDevice));
  WS_TRY(h->net->set_weights((const float*)p, h->stream));
  h->net->adamStep = (int)steps;
  if (gain > 0) WS_TRY(h->net->set_gain(gain, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  return WS_OK;
}

// ------------------------------------------------------------ surface mesh
// MarchingTetrahedra.build (js/surface.js:66-177) of a corner field on the
// lattice dd into mb, vertices in the reference's emission order. partials
// holds grid_for(dd.nCells, 128) + 1 entries; the volume pass leaves the
// per-block vertex counts there for the emission scan.
static ws_status mt_build(ws_handle* h, const Dims& dd, const float* field, double iso, double2* partials, MeshBuf& mb,
                          int64_t* vertices, double* volume) {
  const long long nb = grid_for(dd.nCells, 128);
  void* scr = nullptr;
  ws_status s = mt_scratch(h, dd.nCells, &scr); if (s) return s;
  launch_mt_volume(dd, field, iso, partials, h->red, scr, h->stream);
  s = check_launch(h, 6); if (s) return s;
  WS_TRY(cudaMemcpyAsync(h->redHost, h->red, sizeof(double) * 2, cudaMemcpyDeviceToHost, h->stream));
  WS_TRY(cudaStreamSynchronize(h->stream));
  const double vol = std::fabs(h->redHost[0]);
  const long long cnt = llround(h->redHost[1]);
  if (nb + 1 > mb.offsCap) {
    if (mb.offs) cudaFree(mb.offs);
    mb.offs = nullptr; mb.offsCap = 0;
    WS_TRY(cudaMalloc(&mb.offs, sizeof(long long) * (size_t)(nb + 1)));
    mb.offsCap = nb + 1;
  }
  if (cnt > mb.cap) {
    long long cap = std::max<long long>(cnt + cnt / 4, 1 << 16);
    if (mb.pos) cudaFree(mb.pos);
    if (mb.nrm) cudaFree(mb.nrm);
    mb.pos = nullptr; mb.nrm = nullptr; mb.cap = 0;
    WS_TRY(cudaMalloc(&mb.pos, sizeof(float) * 3 * (size_t)cap));
    WS_TRY(cudaMalloc(&mb.nrm, sizeof(float) * 3 * (size_t)cap));
    mb.cap = cap;
  }
  launch_mt_mesh(dd, field, iso, partials, mb.offs, mb.cap, mb.pos, mb.nrm, scr, h->stream);
  if ((s = check_launch(h, 2))) return s;
  WS_TRY(cudaStreamSynchronize(h->stream));
  mb.verts = cnt;
  if (vertices) *vertices = cnt;
  if (volume) *volume = vol;
  return WS_OK;
}
static ws_status mesh_download(ws_handle* h, const MeshBuf& mb, float* pos, float* nrm, int64_t max_vertices) {
  if (max_vertices < mb.verts) return fail(h, WS_ERR_RANGE, "buffers hold fewer vertices than the mesh");
  if (pos && mb.verts) WS_TRY(cudaMemcpy(pos, mb.pos, sizeof(float) * 3 * (size_t)mb.verts, cudaMemcpyDeviceToHost));
  if (nrm && mb.verts) WS_TRY(cudaMemcpy(nrm, mb.nrm, sizeof(float) * 3 * (size_t)mb.verts, cudaMemcpyDeviceToHost));
  return WS_OK;
}

// the current density field (ws_stage SPLAT / splatDensity) at iso
extern "C" ws_status ws_surface_mesh(ws_handle* h, double iso, int64_t* vertices, double* volume) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  if ((long long)grid_for(h->d.nCells, 128) + 1 > h->partialsCap) return fail(h, WS_ERR_RANGE, "partials too small");
  return mt_build(h, h->d, h->dens, iso, h->partials, h->surf, vertices, volume);
}
extern "C" ws_status ws_surface_download(ws_handle* h, float* pos, float* nrm, int64_t max_vertices) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  return mesh_download(h, h->surf, pos, nrm, max_vertices);
}
extern "C" ws_status ws_surface_device(ws_handle* h, const float** pos, const float** nrm, int64_t* vertices) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !pos || !nrm || !vertices) return WS_ERR_INVALID;
  *pos = h->surf.pos; *nrm = h->surf.nrm; *vertices = h->surf.verts;
  return WS_OK;
}

// ------------------------------------------------------------ metaballs
// Metaballs.build (js/surface.js:203-284): lattice size, spacing, kernel
// radius and contour level from tension and the detail factor, as
// metaballKernelCells / metaballIso / buildMetaballs compute them
static double js_round(double x) { double r = std::floor(x); return (x - r >= 0.5) ? r + 1 : r; }
extern "C" ws_status ws_metaball_mesh(ws_handle* h, double tension, double detail, int64_t* vertices, double* volume) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  double f = 1;
  if (std::isfinite(detail) && detail > 0) f = detail < 0.5 ? 0.5 : (detail > 1.6 ? 1.6 : detail);
  const int nx = h->d.nx;
  const int m = std::max(6, (int)js_round(nx * f));
  const double mdx = m == nx ? h->d.dx : h->d.W / m;
  double t = std::isfinite(tension) ? tension : 0.5;
  t = t < 0 ? 0 : (t > 1 ? 1 : t);
  const double R = (1.6 + 2.2 * t) * h->S.spacing / mdx;
  const double iso = 1.5 * std::pow((1.6 + 2.2 * t) / 1.6, 1.5);
  const int rad = std::min(3, (int)std::ceil(R));
  const long long corners = (long long)(m + 1) * (m + 1) * (m + 1), cells = (long long)m * m * m;
  if (corners > h->mbCorners) {
    for (void* b : { (void*)h->mbAcc, (void*)h->mbField }) if (b) cudaFree(b);
    h->mbAcc = nullptr; h->mbField = nullptr; h->mbCorners = 0;
    WS_TRY(cudaMalloc(&h->mbAcc, sizeof(double) * (size_t)corners));
    WS_TRY(cudaMalloc(&h->mbField, sizeof(float) * (size_t)corners));
    h->mbCorners = corners;
  }
  if (cells > h->mbCells) {
    if (h->mbPartials) cudaFree(h->mbPartials);
    h->mbPartials = nullptr; h->mbCells = 0;
    WS_TRY(cudaMalloc(&h->mbPartials, sizeof(double2) * (size_t)(grid_for(cells, 128) + 1)));
    h->mbCells = cells;
  }
  h->mbM = m;
  launch_metaball_field(parts_of(h), m, mdx, R * R, rad, h->mbAcc, h->mbField, h->stream);
  if ((s = check_launch(h, h->S.nP ? 2 : 1))) return s;
  Dims dd = h->d;
  dd.nx = dd.ny = dd.nz = m; dd.dx = mdx; dd.nCells = cells;
  dims_fastdiv(dd);
  return mt_build(h, dd, h->mbField, iso, h->mbPartials, h->mball, vertices, volume);
}
extern "C" ws_status ws_metaball_download(ws_handle* h, float* pos, float* nrm, int64_t max_vertices) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  return mesh_download(h, h->mball, pos, nrm, max_vertices);
}
extern "C" ws_status ws_metaball_device(ws_handle* h, const float** pos, const float** nrm, int64_t* vertices) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !pos || !nrm || !vertices) return WS_ERR_INVALID;
  *pos = h->mball.pos; *nrm = h->mball.nrm; *vertices = h->mball.verts;
  return WS_OK;
}
extern "C" ws_status ws_metaball_field(ws_handle* h, float* field, int64_t capacity, int32_t* m) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  const long long corners = (long long)(h->mbM + 1) * (h->mbM + 1) * (h->mbM + 1);
  if (m) *m = h->mbM;
  if (!h->mbM || !field) return WS_OK;
  if (capacity < corners) return fail(h, WS_ERR_RANGE, "buffer holds fewer floats than the (m+1)^3 field");
  WS_TRY(cudaMemcpy(field, h->mbField, sizeof(float) * (size_t)corners, cudaMemcpyDeviceToHost));
  return WS_OK;
}

// ------------------------------------------------------------ render prep
// WaterScene.updateParticles (js/scene.js:1595-1922): scene flags and the
// per-class size/alpha/sprite resolved here (js/scene.js:1601-1602,
// 1783-1800), the per-particle work in ws_render.cu
extern "C" ws_status ws_render_particles(ws_handle* h, const ws_render_opts* o, int32_t counts[5], int64_t* points) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !o) return WS_ERR_INVALID;
  cudaSetDevice(h->device);
  ws_status s = sync_status(h); if (s) return s;
  RenderCfg c{};
  c.showBeads = o->show && o->beadsMode && o->waterOpa > 0.01 && !o->metaballMode;
  c.showSpray = o->show && o->pOpa > 0.01;
  c.planetLit = o->planetLit != 0; c.useLight = o->useLight != 0; c.useDepth = o->useDepth != 0;
  c.useTemp = o->useTemp != 0; c.spinCue = h->P.spinOn != 0; c.spinCol = o->spinColor != 0;
  c.sortOn = o->sortOn != 0;
  c.center[0] = h->d.W * 0.5; c.center[1] = h->d.H * 0.5; c.center[2] = h->d.D * 0.5;
  for (int i = 0; i < 3; i++) {
    c.sun[i] = o->sunDir[i]; c.water[i] = o->waterColor[i];
    c.cam[i] = c.sortOn ? o->cam[i] : c.center[i];            // unsorted: distance from the centre
  }
  double sp = h->S.spacing;
  if (!(std::isfinite(sp) && sp > 0.02)) sp = 0.06;
  const double wS = o->wScale ? o->wScale : 1;
  const double size[5] = { sp * 3.4, sp * 3.4 / 3, std::max(0.18 * wS, std::min(0.4 * wS, sp * 5)),
                           std::max(0.30 * wS, std::min(0.62 * wS, sp * 6.5)), sp * 3.4 };
  const double alpha[5] = { std::min(1.0, std::max(0.0, o->waterOpa)), std::min(1.0, 0.95 * o->pOpa),
                            0.23 * std::sqrt(o->pOpa), std::min(1.0, 0.88 * o->pOpa), 1 };
  const double sprite[5] = { 0, 1, 2, o->cloudSprite ? 5.0 : 3.0, 4 };
  for (int i = 0; i < 5; i++) { c.size[i] = (float)size[i]; c.alpha[i] = (float)alpha[i]; c.sprite[i] = (float)sprite[i]; }
  if (!h->rdrScratch) {
    size_t cap = (size_t)h->capacity;
    WS_TRY(cudaMalloc(&h->rdrScratch, render_scratch_bytes(h->capacity)));
    WS_TRY(cudaMalloc(&h->rdr.pos, sizeof(float) * 3 * cap));
    WS_TRY(cudaMalloc(&h->rdr.col, sizeof(float) * 3 * cap));
    WS_TRY(cudaMalloc(&h->rdr.alpha, sizeof(float) * cap));
    WS_TRY(cudaMalloc(&h->rdr.size, sizeof(float) * cap));
    WS_TRY(cudaMalloc(&h->rdr.sprite, sizeof(float) * cap));
  }
  h->rdrPoints = 0;
  int32_t cnt[5] = { 0, 0, 0, 0, 0 };
  if (c.showBeads || c.showSpray) {
    launch_render_particles(c, parts_of(h), h->rdrScratch, h->rdr, h->stream);
    if ((s = check_launch(h, h->S.nP ? 4 : 0))) return s;
    WS_TRY(cudaMemcpyAsync(cnt, h->rdrScratch, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
    WS_TRY(cudaStreamSynchronize(h->stream));
  }
  for (int i = 0; i < 5; i++) h->rdrPoints += cnt[i];
  if (counts) for (int i = 0; i < 5; i++) counts[i] = cnt[i];
  if (points) *points = h->rdrPoints;
  return WS_OK;
}
extern "C" ws_status ws_render_download(ws_handle* h, float* pos, float* col, float* alpha, float* size, float* sprite,
                                        int64_t max_points) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h) return WS_ERR_INVALID;
  if (max_points < h->rdrPoints) return fail(h, WS_ERR_RANGE, "buffers hold fewer points than the draw list");
  const size_t n = (size_t)h->rdrPoints;
  if (pos) WS_TRY(cudaMemcpy(pos, h->rdr.pos, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost));
  if (col) WS_TRY(cudaMemcpy(col, h->rdr.col, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost));
  if (alpha) WS_TRY(cudaMemcpy(alpha, h->rdr.alpha, sizeof(float) * n, cudaMemcpyDeviceToHost));
  if (size) WS_TRY(cudaMemcpy(size, h->rdr.size, sizeof(float) * n, cudaMemcpyDeviceToHost));
  if (sprite) WS_TRY(cudaMemcpy(sprite, h->rdr.sprite, sizeof(float) * n, cudaMemcpyDeviceToHost));
  return WS_OK;
}
extern "C" ws_status ws_render_device(ws_handle* h, const float** pos, const float** col, const float** alpha,
                                      const float** size, const float** sprite, int64_t* points) {
  if (h && h->asyncRunning.load(std::memory_order_acquire)) return WS_ERR_BUSY;
  join_copies(h);
  if (!h || !pos || !col || !alpha || !size || !sprite || !points) return WS_ERR_INVALID;
  *pos = h->rdr.pos; *col = h->rdr.col; *alpha = h->rdr.alpha; *size = h->rdr.size; *sprite = h->rdr.sprite;
  *points = h->rdrPoints;
  return WS_OK;
}
