// ws_particles.cu — particle kernels of the substep: fused G2P + advection
// (js/solver.js:1646-2292), the serial-order vapour pass, order-preserving
// compaction, and the interaction impulses (:3852-3908).
#include "ws_kernels.cuh"

// ------------------------------------------------------------ fused G2P + advect
// One thread per particle. The G2P part (_g2pChunk :1646-1756) leaves the
// sampled new-grid velocity in registers, which is exactly what the
// reference hands to advection through _advU/_advV/_advW (:1725, :2178).
// Particles are independent in both loops of the reference, so fusing them
// changes no result. Vapour parcels (pflag 2/3) consume the serial LCG
// streams _cfS/_bfS and are advanced by k_vapor_advect instead.
// Float locals fvx/fvy/fvz hold the float32 array contents (every store of
// the reference rounds to float32); positions are JS doubles until stored.
__global__ void __launch_bounds__(256, 4) k_g2p_advect(Dims d, GridDev g, PartsDev P, TerrainDev t,
                                                    AdvectParams ap, DevStatus* st) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  int air = 0;
  if (p < P.nP) {
    int fl = P.pflag[p];
    const double dx = d.dx, dt = ap.dt, maxSpeed = ap.maxSpeed, oceanR = ap.oceanR;
    const double cx = d.cx, cy = d.cy, cz = d.cz;
    const float xf = P.px[p], yf = P.py[p], zf = P.pz[p];
    double x = xf, y = yf, z = zf;
    float fvx = P.pvx[p], fvy = P.pvy[p], fvz = P.pvz[p];
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;       // _advU/_advV/_advW (FP32 samples)
    int cool = 0, coolWrite = 0;
    // ---------------- G2P
    if (fl != 0) {
      air = 1;
    } else if ((cool = P.pcool[p]) > 0) {
      coolWrite = 1; cool--;
      double gdt = dt; if (gdt == 0) gdt = ap.dtLast; if (gdt == 0) gdt = 0.01;
      fvy = (float)((double)fvy - ap.gravity * gdt);
      sample_vel3_f(d, g.vel, xf, yf, zf, a0, a1, a2);
    } else {
      // FP32 sampling at the stored position (exact face indices and fractions)
      Stencil3 S;
      face_stencil3_f(d, xf, yf, zf, S);
      const float ou = stencil_sample(d, g.velO, S, 0), ov = stencil_sample(d, g.velO, S, 1);
      const float ow = stencil_sample(d, g.velO, S, 2);
      a0 = stencil_sample(d, g.vel, S, 0); a1 = stencil_sample(d, g.vel, S, 1); a2 = stencil_sample(d, g.vel, S, 2);
      const float pic = (float)ap.pic, flip = (float)(1 - ap.pic);
      fvx = fmaf(fvx + a0 - ou, flip, a0 * pic);
      fvy = fmaf(fvy + a1 - ov, flip, a1 * pic);
      fvz = fmaf(fvz + a2 - ow, flip, a2 * pic);
      const float pv2 = fvx * fvx + fvy * fvy + fvz * fvz, msf = (float)maxSpeed;
      if (pv2 > msf * msf) {
        const float psc = msf / sqrtf(pv2);
        fvx *= psc; fvy *= psc; fvz *= psc;
      }
      int ci = jfloor_clamp(over_dx(d, x), 0, d.nx - 1), cj = jfloor_clamp(over_dx(d, y), 0, d.ny - 1), ck = jfloor_clamp(over_dx(d, z), 0, d.nz - 1);
      long long c = ((long long)ck * d.ny + cj) * d.nx + ci; long long nxy = (long long)d.nx * d.ny;
      const uint8_t* type = g.type;
      if (type[c] == WS_AIR) {
        bool fluidNbr =
          (ci > 0 && type[c - 1] == WS_FLUID) || (ci < d.nx - 1 && type[c + 1] == WS_FLUID) ||
          (cj > 0 && type[c - d.nx] == WS_FLUID) || (cj < d.ny - 1 && type[c + d.nx] == WS_FLUID) ||
          (ck > 0 && type[c - nxy] == WS_FLUID) || (ck < d.nz - 1 && type[c + nxy] == WS_FLUID);
        bool onRock = false;
        if (!fluidNbr && t.has) {                       // _onRockBelow, :581-587
          double ex = x - cx, ey = y - cy, ez = z - cz;
          double el = sqrt(ex * ex + ey * ey + ez * ez); if (el == 0) el = 1e-9;
          double s9 = dx * 0.9 / el;
          onRock = rock_cell_at(d, g.staticTypes, x - ex * s9, y - ey * s9, z - ez * s9);
        }
        if (!fluidNbr && !onRock) { fl = 1; air = 1; P.pflag[p] = 1; }
      }
    }
    // ---------------- advection (:1793-2291)
    const double domHi = d.domainR - dx * 0.02;
    const double xLo = dx * 1.02, xHi = d.W - dx * 1.02, yLo = dx * 1.02, yHi = d.H - dx * 1.02;
    const double zLo = dx * 1.02, zHi = d.D - dx * 1.02;
    const bool hasTerr = t.has;
    bool writePos = true;
    if (fl == 5) {                                         // ice, :1797-1864
      if (P.pAir[p] == 1.f || !hasTerr) {
        fvx = 0.f; fvy = 0.f; fvz = 0.f; writePos = false;
      } else {
        double dragK = 12, gI = ap.gravity; if (gI == 0) gI = 9.81;
        double exI = x - cx, eyI = y - cy, ezI = z - cz;
        double elI = sqrt(exI * exI + eyI * eyI + ezI * ezI); if (elI == 0) elI = 1e-9;
        double axI = -gI * 0.6 * exI / elI, ayI = -gI * 0.6 * eyI / elI, azI = -gI * 0.6 * ezI / elI;
        fvx = (float)((double)fvx + (axI - dragK * fvx) * dt);
        fvy = (float)((double)fvy + (ayI - dragK * fvy) * dt);
        fvz = (float)((double)fvz + (azI - dragK * fvz) * dt);
        x += fvx * dt; y += fvy * dt; z += fvz * dt;
        double rrI = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
        double top = oceanR + ap.atmosphereH;
        if (rrI > top) {
          double scI = top / rrI;
          x = cx + (x - cx) * scI; y = cy + (y - cy) * scI; z = cz + (z - cz) * scI;
          fvx = (float)(fvx * 0.5); fvy = (float)(fvy * 0.5); fvz = (float)(fvz * 0.5);
        }
        if (rock_cell_at(d, g.staticTypes, x, y, z)) {
          P.pAir[p] = 1.f; fvx = fvy = fvz = 0.f;
        } else {
          double ciF = floor(over_dx(d, x)), cjF = floor(over_dx(d, y)), ckF = floor(over_dx(d, z));
          if (ciF >= 0 && cjF >= 0 && ckF >= 0 && ciF < d.nx && cjF < d.ny && ckF < d.nz &&
              g.type[((long long)ckF * d.ny + (long long)cjF) * d.nx + (long long)ciF] == WS_FLUID) {
            double exF = x - cx, eyF = y - cy, ezF = z - cz;
            double elF = sqrt(exF * exF + eyF * eyF + ezF * ezF); if (elF == 0) elF = 1e-9;
            double stepF = dx * 0.5;
            for (int mf = 0; mf < 12; mf++) {
              double qx = x + exF / elF * stepF, qy = y + eyF / elF * stepF, qz = z + ezF / elF * stepF;
              double qi = floor(over_dx(d, qx)), qj = floor(over_dx(d, qy)), qk = floor(over_dx(d, qz));
              if (qi < 0 || qj < 0 || qk < 0 || qi >= d.nx || qj >= d.ny || qk >= d.nz) break;
              if (g.type[((long long)qk * d.ny + (long long)qj) * d.nx + (long long)qi] != WS_FLUID) break;
              x = qx; y = qy; z = qz;
            }
            P.pAir[p] = 1.f; fvx = fvy = fvz = 0.f;
            P.pWx[p] = 0.f; P.pWy[p] = 0.f; P.pWz[p] = 0.f;
          }
        }
      }
    } else if (fl == 1 || fl == 4) {                       // ballistic, :1865-1976
      double vx = fvx, vy = fvy, vz = fvz;
      double gx = x - cx, gy = y - cy, gz = z - cz;
      double gr2 = gx * gx + gy * gy + gz * gz;
      double ga = ap.gravity * oceanR * oceanR * dt / (gr2 * sqrt(gr2));
      fvx = (float)(vx - gx * ga); fvy = (float)(vy - gy * ga); fvz = (float)(vz - gz * ga);
      double dr = 1 - 2.5 * dt; if (dr < 0) dr = 0;
      fvx = (float)(fvx * dr); fvy = (float)(fvy * dr); fvz = (float)(fvz * dr);
      double dsp = sqrt((double)fvx * fvx + (double)fvy * fvy + (double)fvz * fvz);
      if (dsp > maxSpeed) { double dsc = maxSpeed / dsp; fvx = (float)(fvx * dsc); fvy = (float)(fvy * dsc); fvz = (float)(fvz * dsc); }
      x += fvx * dt; y += fvy * dt; z += fvz * dt;
      double bx = x - cx, by = y - cy, bz = z - cz;
      double br = sqrt(bx * bx + by * by + bz * bz); if (br == 0) br = 1e-9;
      double skyHi = oceanR + ap.atmosphereH;
      if (br > skyHi) {
        double sc0 = skyHi / br;
        x = cx + bx * sc0; y = cy + by * sc0; z = cz + bz * sc0;
        double vr0 = ((double)fvx * bx + (double)fvy * by + (double)fvz * bz) / br;
        if (vr0 > 0) {
          fvx = (float)(fvx - bx / br * vr0 * 1.15); fvy = (float)(fvy - by / br * vr0 * 1.15); fvz = (float)(fvz - bz / br * vr0 * 1.15);
        }
      } else if (br <= domHi) {
        int tries0 = 0;
        while (hasTerr && rock_cell_at(d, g.staticTypes, x, y, z) && tries0 < 8) {
          double rW0 = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
          double stW0 = dmin(dx * 0.5, domHi - rW0);
          if (stW0 <= 1e-5) { tries0 = 8; break; }
          x += bx / br * stW0; y += by / br * stW0; z += bz / br * stW0;
          tries0++;
        }
        if (!hasTerr && br < ap.coreR + dx * 1.02) {
          double sc1 = (ap.coreR + dx * 1.02) / br;
          x = cx + bx * sc1; y = cy + by * sc1; z = cz + bz * sc1;
          tries0 = 1;
        }
        if (tries0 > 0) {
          if (hasTerr) {
            double exS = x - cx, eyS = y - cy, ezS = z - cz;
            double erS = sqrt(exS * exS + eyS * eyS + ezS * ezS); if (erS == 0) erS = 1e-9;
            double wantS = terrain_radius_at(t, ap.coreR, x, y, z) + dx * 0.06;
            if (erS > wantS) { x = cx + exS / erS * wantS; y = cy + eyS / erS * wantS; z = cz + ezS / erS * wantS; }
            int kS = 0;
            while (rock_cell_at(d, g.staticTypes, x, y, z) && kS < 4) {
              x += exS / erS * dx * 0.5; y += eyS / erS * dx * 0.5; z += ezS / erS * dx * 0.5;
              kS++;
            }
          }
          double vr1 = ((double)fvx * bx + (double)fvy * by + (double)fvz * bz) / br;
          fvx = (float)(fvx - bx / br * vr1); fvy = (float)(fvy - by / br * vr1); fvz = (float)(fvz - bz / br * vr1);
          fvx = (float)(fvx * 0.3); fvy = (float)(fvy * 0.3); fvz = (float)(fvz * 0.3);
          fl = 0;
        }
      }
      int ci = jfloor_clamp(over_dx(d, x), 0, d.nx - 1), cj = jfloor_clamp(over_dx(d, y), 0, d.ny - 1), ck = jfloor_clamp(over_dx(d, z), 0, d.nz - 1);
      if (g.type[((long long)ck * d.ny + cj) * d.nx + ci] == WS_FLUID) {
        fvx = (float)(fvx * 0.45); fvy = (float)(fvy * 0.45); fvz = (float)(fvz * 0.45);
        if (fvy > 0.5f) fvy = 0.5f;
        cool = 2; coolWrite = 1;
        fl = 0;
      }
      P.pflag[p] = (uint8_t)fl;
    } else if (fl == 2 || fl == 3) {
      writePos = false;                                    // k_vapor_advect owns these
    } else {                                               // grid-coupled fluid, :2176-2290
      // Velocities in FP32; the position update and every test of a position
      // (domain shell, rock cells) in double, as the reference computes them.
      float v2x = a0, v2y = a1, v2z = a2;
      float sp2 = a0 * a0 + a1 * a1 + a2 * a2;
      if (sp2 > 0.25f) {
        const float hdt = (float)(0.5 * dt);
        float mx = fmaf(hdt, a0, xf), my = fmaf(hdt, a1, yf), mz = fmaf(hdt, a2, zf);
        const float xLof = (float)xLo, xHif = (float)xHi, yLof = (float)yLo, yHif = (float)yHi;
        const float zLof = (float)zLo, zHif = (float)zHi;
        mx = mx < xLof ? xLof : (mx > xHif ? xHif : mx);
        my = my < yLof ? yLof : (my > yHif ? yHif : my);
        mz = mz < zLof ? zLof : (mz > zHif ? zHif : mz);
        sample_vel3_f(d, g.vel, mx, my, mz, v2x, v2y, v2z);
      }
      sp2 = v2x * v2x + v2y * v2y + v2z * v2z;
      const float msf = (float)maxSpeed;
      if (sp2 > msf * msf) {
        const float sc = msf / sqrtf(sp2);
        v2x *= sc; v2y *= sc; v2z *= sc;
        fvx *= sc; fvy *= sc; fvz *= sc;
      }
      x += (double)v2x * dt; y += (double)v2y * dt; z += (double)v2z * dt;
      double nx2 = x - cx, ny2 = y - cy, nz2 = z - cz;
      double nr = sqrt(nx2 * nx2 + ny2 * ny2 + nz2 * nz2); if (nr == 0) nr = 1e-9;
      const double inr = 1.0 / nr;
      if (nr > domHi) {
        double sc2 = domHi / nr;
        x = cx + nx2 * sc2; y = cy + ny2 * sc2; z = cz + nz2 * sc2;
        fvy = (float)(-fabs((double)fvy) * 0.1 - 0.3);
        fl = 1; P.pflag[p] = 1;
      }
      if (nr < domHi) {
        int tries = 0;
        while (hasTerr && rock_cell_at(d, g.staticTypes, x, y, z) && tries < 8) {
          double rW2 = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
          double stW2 = dmin(dx * 0.5, domHi - rW2);
          if (stW2 <= 1e-5) { tries = 8; break; }
          x += nx2 / nr * stW2; y += ny2 / nr * stW2; z += nz2 / nr * stW2;
          tries++;
        }
        if (tries > 0) {
          if (hasTerr) {
            double exS2 = x - cx, eyS2 = y - cy, ezS2 = z - cz;
            double erS2 = sqrt(exS2 * exS2 + eyS2 * eyS2 + ezS2 * ezS2); if (erS2 == 0) erS2 = 1e-9;
            double wantS2 = terrain_radius_at(t, ap.coreR, x, y, z) + dx * 0.06;
            if (erS2 > wantS2) { x = cx + exS2 / erS2 * wantS2; y = cy + eyS2 / erS2 * wantS2; z = cz + ezS2 / erS2 * wantS2; }
            int kS2 = 0;
            while (rock_cell_at(d, g.staticTypes, x, y, z) && kS2 < 4) {
              x += exS2 / erS2 * dx * 0.5; y += eyS2 / erS2 * dx * 0.5; z += ezS2 / erS2 * dx * 0.5;
              kS2++;
            }
          }
          double vr2 = ((double)fvx * nx2 + (double)fvy * ny2 + (double)fvz * nz2) / nr;
          if (vr2 < 0) { fvx = (float)(fvx - nx2 / nr * vr2); fvy = (float)(fvy - ny2 / nr * vr2); fvz = (float)(fvz - nz2 / nr * vr2); }
        }
        if (hasTerr && (tries > 0 || rock_cell_at(d, g.staticTypes, x - nx2 * inr * dx, y - ny2 * inr * dx, z - nz2 * inr * dx))) {
          double fr0 = 1 - 0.6 * dt; if (fr0 < 0) fr0 = 0;
          const float fr = (float)fr0;
          fvx *= fr; fvy *= fr; fvz *= fr;
        }
      }
      // radial damping and drag (velocities only): FP32
      const float sx = (float)(x - cx), sy = (float)(y - cy), sz = (float)(z - cz);
      float sr = sqrtf(sx * sx + sy * sy + sz * sz); if (sr == 0.f) sr = 1e-9f;
      const float isr = 1.f / sr;
      const float vrad = (fvx * sx + fvy * sy + fvz * sz) * isr;
      double da = 1.0 * dt; if (da > 0.5) da = 0.5;
      const float kr = vrad * (float)da * isr;
      fvx = fmaf(-sx, kr, fvx); fvy = fmaf(-sy, kr, fvy); fvz = fmaf(-sz, kr, fvz);
      double dg = 1 - 0.42 * dt; if (dg < 0) dg = 0;
      const float dgf = (float)dg;
      fvx *= dgf; fvy *= dgf; fvz *= dgf;
    }
    if (fl != 2 && fl != 3) { P.pvx[p] = fvx; P.pvy[p] = fvy; P.pvz[p] = fvz; }
    if (writePos) { P.px[p] = (float)x; P.py[p] = (float)y; P.pz[p] = (float)z; }
    if (coolWrite) P.pcool[p] = (uint8_t)cool;
    if (fl != 2 && fl != 3) particle_sound(d, x, y, z, fvx, fvy, fvz, &st->err, false);
  }
  // airborne count (G2P's airCount): exact integer sum
  int wsum = warp_sum(air);
  if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(&st->airborne, wsum);
}
void launch_g2p_advect(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t,
                       const AdvectParams& ap, DevStatus* st, cudaStream_t s) {
  if (P.nP <= 0) return;
  k_g2p_advect<<<grid_for(P.nP, 256), 256, 0, s>>>(d, g, P, t, ap, st);
}

// ------------------------------------------------------------ order-preserving compaction
// Indices p with pred(pflag[p]) in increasing order: per-block counts, one
// block scans the counts, then each block writes its ranks.
__device__ __forceinline__ bool pred_flag(int mode, uint8_t f) {
  if (mode == 0) return f == 2 || f == 3;       // vapour parcels
  if (mode == 1) return f == 0;                  // grid-coupled fluid
  return f != 0;                                 // a byte predicate array
}
__global__ void k_compact_count(const uint8_t* __restrict__ fl, int nP, int mode, int* __restrict__ blockCounts) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  int v = (p < nP && pred_flag(mode, fl[p])) ? 1 : 0;
  int c = __syncthreads_count(v);
  if (threadIdx.x == 0) blockCounts[blockIdx.x] = c;
}
__global__ void k_compact_scan(int* __restrict__ blockCounts, int nb, int* __restrict__ total) {
  __shared__ int warpTot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < nb ? blockCounts[i] : 0;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) warpTot[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int w = lane < (int)(blockDim.x >> 5) ? warpTot[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, w, o); if (lane >= o) w += y; }
      warpTot[lane] = w;
    }
    __syncthreads();
    int excl = x - v + (wid > 0 ? warpTot[wid - 1] : 0) + carry;
    if (i < nb) blockCounts[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}
__global__ void k_compact_scatter(const uint8_t* __restrict__ fl, int nP, int mode,
                                  const int* __restrict__ blockOffsets, int* __restrict__ out) {
  __shared__ int warpTot[32];
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  int v = (p < nP && pred_flag(mode, fl[p])) ? 1 : 0;
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned m = __ballot_sync(0xffffffffu, v);
  int rank = __popc(m & ((1u << lane) - 1u));
  if (lane == 0) warpTot[wid] = __popc(m);
  __syncthreads();
  int off = 0;
  for (int w = 0; w < wid; w++) off += warpTot[w];
  if (v) out[blockOffsets[blockIdx.x] + off + rank] = p;
}
void launch_compact(const uint8_t* fl, int nP, int mode, int* blockCounts, int* out, int* total, cudaStream_t s) {
  int nb = (int)grid_for(nP, 256);
  k_compact_count<<<nb, 256, 0, s>>>(fl, nP, mode, blockCounts);
  k_compact_scan<<<1, 1024, 0, s>>>(blockCounts, nb, total);
  k_compact_scatter<<<nb, 256, 0, s>>>(fl, nP, mode, blockCounts, out);
}

// ------------------------------------------------------------ vapour pass
// Atmospheric branch of _advectChunk (js/solver.js:1978-2174) with the
// reference's serial LCG draws reproduced exactly: one CTA walks the vapour
// list in index order, 1024 parcels at a time. Which parcels draw from _cfS
// (ceiling bounce) depends only on each parcel's own state, so a block scan
// gives each drawing parcel its position k in the stream and lcg_jump gives
// its value; the floor draws (_bfS) depend on the ceiling outcome and get a
// second scan. RNG states live in device memory between calls.
__device__ __forceinline__ int block_excl_scan(int v, int* warpTot, int& total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
  if (lane == 31) warpTot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < nw ? warpTot[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, w, o); if (lane >= o) w += y; }
    warpTot[lane] = w;
  }
  __syncthreads();
  int excl = x - v + (wid > 0 ? warpTot[wid - 1] : 0);
  total = warpTot[nw - 1];
  __syncthreads();
  return excl;
}
__global__ void __launch_bounds__(1024) k_vapor_advect(Dims d, GridDev g, PartsDev P, TerrainDev t, AdvectParams ap,
                                                       const int* __restrict__ vIdx, const int* __restrict__ nVp,
                                                       uint32_t* __restrict__ rng, DevStatus* st) {
  __shared__ int warpTot[32];
  const int nV = *nVp;
  uint32_t cfS = rng[0], bfS = rng[1];
  const double dx = d.dx, dt = ap.dt, maxSpeed = ap.maxSpeed, oceanR = ap.oceanR;
  const double cx = d.cx, cy = d.cy, cz = d.cz, domHi = d.domainR - dx * 0.02;
  int drawsA = 0, drawsB = 0;
  for (int base = 0; base < nV; base += blockDim.x) {
    int idx = base + threadIdx.x;
    bool act = idx < nV;
    int p = act ? vIdx[idx] : 0;
    double x = 0, y = 0, z = 0, Tv = 0, vCx = 0, vCy = 0, vCz = 0, vCr = 1, vrC2 = 0, prf = 0;
    float fvx = 0, fvy = 0, fvz = 0, fAir = 0;
    int fl = 0, wantA = 0;
    if (act) {
      fl = P.pflag[p];
      x = P.px[p]; y = P.py[p]; z = P.pz[p];
      double vx = P.pvx[p], vy = P.pvy[p], vz = P.pvz[p];
      Tv = P.pT[p];
      fAir = (float)((double)P.pAir[p] + dt);
      double vEx = x - cx, vEy = y - cy, vEz = z - cz;
      double vEr = sqrt(vEx * vEx + vEy * vEy + vEz * vEz); if (vEr == 0) vEr = 1e-9;
      double ux = vEx / vEr, uy = vEy / vEr, uz = vEz / vEr;
      double exposure = ux * ap.windS[0] + uy * ap.windS[1] + uz * ap.windS[2];
      double jet = dmin(oceanR * 0.58, maxSpeed * 0.45);
      double returnFlow = dmin(oceanR * 0.32, maxSpeed * 0.25);
      double vr = vx * ux + vy * uy + vz * uz;
      double radial = -ap.gravity * 0.06;
      double wx = -uz * jet - (ap.windS[0] - exposure * ux) * returnFlow;
      double wy = -(ap.windS[1] - exposure * uy) * returnFlow;
      double wz = ux * jet - (ap.windS[2] - exposure * uz) * returnFlow;
      double relax = dmin(1, dt * 1.3);
      fvx = (float)(vx + (wx - (vx - vr * ux)) * relax + ux * radial * dt);
      fvy = (float)(vy + (wy - (vy - vr * uy)) * relax + uy * radial * dt);
      fvz = (float)(vz + (wz - (vz - vr * uz)) * relax + uz * radial * dt);
      double svv = (double)fvx * fvx + (double)fvy * fvy + (double)fvz * fvz;
      if (svv > maxSpeed * maxSpeed) {
        double svs = maxSpeed / sqrt(svv);
        fvx = (float)(fvx * svs); fvy = (float)(fvy * svs); fvz = (float)(fvz * svs);
      }
      x += fvx * dt; y += fvy * dt; z += fvz * dt;
      vCx = x - cx; vCy = y - cy; vCz = z - cz;
      vCr = sqrt(vCx * vCx + vCy * vCy + vCz * vCz); if (vCr == 0) vCr = 1e-9;
      double ceilR = oceanR + ap.atmosphereH - 1e-3 * dx;
      if (t.has) { double RtE = terrain_radius_at(t, ap.coreR, x, y, z); if (RtE + 0.02 > ceilR) ceilR = RtE + 0.02; }
      if (vCr > ceilR) {
        double scE = ceilR / vCr;
        x = cx + vCx * scE; y = cy + vCy * scE; z = cz + vCz * scE;
        double vrE = ((double)fvx * vCx + (double)fvy * vCy + (double)fvz * vCz) / vCr;
        if (vrE > 0) {
          fvx = (float)(fvx - vCx / vCr * vrE * 2); fvy = (float)(fvy - vCy / vCr * vrE * 2); fvz = (float)(fvz - vCz / vCr * vrE * 2);
        }
      }
      vrC2 = ((double)fvx * vCx + (double)fvy * vCy + (double)fvz * vCz) / vCr;
      if (vrC2 > 0 && vCr > oceanR) {
        double hh = (vCr - oceanR) / (ap.atmosphereH > 1e-4 ? ap.atmosphereH : 1e-4);
        if (hh > 1) hh = 1;
        prf = ap.ceilReflect == 1 ? hh * hh : ap.ceilReflect == 2 ? (exp(3 * hh) - 1) * 0.0523957 : hh;
        wantA = prf > 0;
      }
    }
    int totA;
    int kA = block_excl_scan(wantA, warpTot, totA);
    int wantB = 0; double fCx = 0, fCy = 0, fCz = 0, fCr = 1, vrF = 0;
    if (act) {
      if (wantA) {
        uint32_t sA = lcg_jump(cfS, (uint32_t)kA + 1u);
        if (sA / 4294967296.0 < prf * dt * 4) {
          fvx = (float)(fvx - vCx / vCr * vrC2 * 2); fvy = (float)(fvy - vCy / vCr * vrC2 * 2); fvz = (float)(fvz - vCz / vCr * vrC2 * 2);
        }
      }
      fCx = x - cx; fCy = y - cy; fCz = z - cz;
      fCr = sqrt(fCx * fCx + fCy * fCy + fCz * fCz); if (fCr == 0) fCr = 1e-9;
      if (fCr < oceanR + 0.15 * dx) {
        vrF = ((double)fvx * fCx + (double)fvy * fCy + (double)fvz * fCz) / fCr;
        wantB = vrF < 0;
      }
    }
    cfS = lcg_jump(cfS, (uint32_t)totA); drawsA += totA;
    int totB;
    int kB = block_excl_scan(wantB, warpTot, totB);
    if (act) {
      if (wantB) {
        uint32_t sB = lcg_jump(bfS, (uint32_t)kB + 1u);
        double floorR = oceanR + 0.15 * dx;
        double sc = sB / 4294967296.0 < 0.07 ? floorR / fCr : (floorR + 0.02 * dx) / fCr;
        x = cx + fCx * sc; y = cy + fCy * sc; z = cz + fCz * sc;
        fvx = (float)(fvx - fCx / fCr * vrF * 2); fvy = (float)(fvy - fCy / fCr * vrF * 2); fvz = (float)(fvz - fCz / fCr * vrF * 2);
      }
      int triesE = 0;
      double rNow3 = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
      while (t.has && rNow3 < d.domainR && rock_cell_at(d, g.staticTypes, x, y, z) && triesE < 8) {
        double rW3 = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz));
        double stW3 = dmin(dx * 0.5, domHi - rW3);
        if (stW3 <= 1e-5) break;
        x += vCx / vCr * stW3; y += vCy / vCr * stW3; z += vCz / vCr * stW3;
        triesE++;
      }
      if (triesE > 0) {
        double vrT = ((double)fvx * vCx + (double)fvy * vCy + (double)fvz * vCz) / vCr;
        if (vrT < 0) {
          double bT = 1.5 * vrT / vCr;
          fvx = (float)(fvx - vCx * bT); fvy = (float)(fvy - vCy * bT); fvz = (float)(fvz - vCz * bT);
        }
        fvx = (float)(fvx * 0.92); fvy = (float)(fvy * 0.92); fvz = (float)(fvz * 0.92);
      }
      int ciV = jfloor_clamp(over_dx(d, x), 0, d.nx - 1), cjV = jfloor_clamp(over_dx(d, y), 0, d.ny - 1), ckV = jfloor_clamp(over_dx(d, z), 0, d.nz - 1);
      bool backToSea = g.type[((long long)ckV * d.ny + cjV) * d.nx + ciV] == WS_FLUID;
      if (backToSea) {
        double bx2 = x - cx, by2 = y - cy, bz2 = z - cz;
        double br2 = sqrt(bx2 * bx2 + by2 * by2 + bz2 * bz2); if (br2 == 0) br2 = 1e-9;
        if (br2 > oceanR + 0.15 * dx) backToSea = false;
        else if (((double)fvx * bx2 + (double)fvy * by2 + (double)fvz * bz2) / br2 > 0.02) backToSea = false;
      }
      P.px[p] = (float)x; P.py[p] = (float)y; P.pz[p] = (float)z;
      if (backToSea) {
        fvx = fvy = fvz = 0.f; fAir = 0.f; fl = 0;
      } else if (fl == 2 && ((Tv <= ap.rainTe && (double)fAir >= ap.rainLiftAge) || fAir > 40.f)) {
        fvx = fvy = fvz = 0.f; fAir = 0.f; fl = 4;
      }
      P.pvx[p] = fvx; P.pvy[p] = fvy; P.pvz[p] = fvz; P.pAir[p] = fAir; P.pflag[p] = (uint8_t)fl;
    }
    bfS = lcg_jump(bfS, (uint32_t)totB); drawsB += totB;
    __syncthreads();
  }
  if (threadIdx.x == 0) { rng[0] = cfS; rng[1] = bfS; st->cfA = drawsA; st->bfB = drawsB; }
}
void launch_vapor_advect(const Dims& d, const GridDev& g, const PartsDev& P, const TerrainDev& t, const AdvectParams& ap,
                         const int* vIdx, const int* nV, uint32_t* rng, DevStatus* st, cudaStream_t s) {
  k_vapor_advect<<<1, 1024, 0, s>>>(d, g, P, t, ap, vIdx, nV, rng, st);
}

// ------------------------------------------------------------ impulses
// applyImpulseSphere, js/solver.js:3852-3864
__global__ void k_impulse_sphere(PartsDev P, double cx, double cy, double cz, double R, double fx, double fy, double fz) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  double ex = P.px[p] - cx, ey = P.py[p] - cy, ez = P.pz[p] - cz;
  double d2 = ex * ex + ey * ey + ez * ez;
  if (d2 > R * R) return;
  double fall = 1 - sqrt(d2) / R;
  P.pvx[p] = (float)((double)P.pvx[p] + fx * fall);
  P.pvy[p] = (float)((double)P.pvy[p] + fy * fall);
  P.pvz[p] = (float)((double)P.pvz[p] + fz * fall);
  if (P.pflag[p] != 0) P.pflag[p] = 0;
  P.pcool[p] = 0;
}
void launch_impulse_sphere(const PartsDev& P, double cx, double cy, double cz, double R, double fx, double fy, double fz, cudaStream_t s) {
  if (P.nP <= 0) return;
  k_impulse_sphere<<<grid_for(P.nP, 256), 256, 0, s>>>(P, cx, cy, cz, R, fx, fy, fz);
}
// stirAt, js/solver.js:3895-3908
__global__ void k_stir_at(PartsDev P, double cx, double cy, double cz, double vx, double vy, double vz, double R, double dt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  double ex = P.px[p] - cx, ey = P.py[p] - cy, ez = P.pz[p] - cz;
  double d2 = ex * ex + ey * ey + ez * ez;
  if (d2 > R * R) return;
  double k = dmin(1, 14 * dt), fall = 1 - sqrt(d2) / R;
  P.pvx[p] = (float)((double)P.pvx[p] + (vx * 1.25 - (double)P.pvx[p]) * k * fall);
  P.pvy[p] = (float)((double)P.pvy[p] + (vy * 1.25 - (double)P.pvy[p]) * k * fall);
  P.pvz[p] = (float)((double)P.pvz[p] + (vz * 1.25 - (double)P.pvz[p]) * k * fall);
  P.pflag[p] = 0;
}
void launch_stir_at(const PartsDev& P, double cx, double cy, double cz, double vx, double vy, double vz, double R, double dt, cudaStream_t s) {
  if (P.nP <= 0) return;
  k_stir_at<<<grid_for(P.nP, 256), 256, 0, s>>>(P, cx, cy, cz, vx, vy, vz, R, dt);
}
// Seeded Gaussian stir kick (the 128^3 planet workload's forcing): the host
// draws the surface point and tangent from stirS; each grid-coupled particle
// within 3 sigma gains peak * exp(-|x - c|^2 / (2 sigma^2)) along the tangent.
__global__ void k_stir_gaussian(PartsDev P, double pcx, double pcy, double pcz, double tx, double ty, double tz,
                                double sigma, double peak) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nP) return;
  if (P.pflag[p] != 0) return;
  double ex = P.px[p] - pcx, ey = P.py[p] - pcy, ez = P.pz[p] - pcz;
  double d2 = ex * ex + ey * ey + ez * ez;
  if (d2 >= 9 * sigma * sigma) return;
  double a = peak * exp(-d2 * (1 / (2 * sigma * sigma)));
  P.pvx[p] = (float)((double)P.pvx[p] + a * tx);
  P.pvy[p] = (float)((double)P.pvy[p] + a * ty);
  P.pvz[p] = (float)((double)P.pvz[p] + a * tz);
}
void launch_stir_gaussian(const PartsDev& P, double pcx, double pcy, double pcz, double tx, double ty, double tz,
                          double sigma, double peak, cudaStream_t s) {
  if (P.nP <= 0) return;
  k_stir_gaussian<<<grid_for(P.nP, 256), 256, 0, s>>>(P, pcx, pcy, pcz, tx, ty, tz, sigma, peak);
}
