// ws_terrain.h — world setup (terrain generator and water fill) of libwatersim.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include <algorithm>
#include "../../include/watersim.h"

namespace wsterrain {

struct Terrain {
  int n = 0;
  double dv = 0, Rsl = 0, Rlo = 0, Rhi = 0, landFrac = 0;
  std::vector<uint8_t> solid;
  std::vector<float> R;
};

struct GenInput {
  uint32_t seed;
  double coreR, seaLevel, bumpiness, dx, cx, cy, cz;
  int nx;
  cudaStream_t stream;
};

struct FillInput {
  uint32_t seed;
  int nx, ny, nz;
  double dx, cx, cy, cz, coreR, depth, targetParticles;
  long long capacity;
};

struct FillOutput {
  double spacing = 0;
  long long capUsed = 0;
  std::vector<float> px, py, pz;
};

int generate(const GenInput& in, Terrain& out, std::string& err);
double water_volume(const Terrain& t, const FillInput& in);
int fill(const Terrain& t, const FillInput& in, FillOutput& out);

}  // namespace wsterrain
