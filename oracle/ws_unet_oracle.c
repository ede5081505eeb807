/*
 * ws_unet_oracle.c — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the warm-start U-Net of libwatersim (the learned
 * initial guess of the pressure solve; the reference has no counterpart —
 * js/solver.js:1312-1410 starts SOR from the previous q). It is the checker
 * for the network's forward output and its loss gradients on the GPU; only
 * tests/ load it.
 *
 * Definition (identical on both sides):
 *  - levels n_0 = grid, n_{l+1} = ceil(n_l / 2); tiles of 8 x 16 x 8 voxels;
 *    a level-0 tile is active when it holds a fluid cell, a level-(l+1) tile
 *    when any of its 2x2x2 child tiles is; activations of inactive tiles are
 *    zero and are read as zero by every operator;
 *  - input channels (16, 4 used): r0 / sigma, fluid, solid, air;
 *  - conv3(x)[co] = relu(sum_t sum_ci x(v + off_t)[ci] W[co][ci][t] + b[co]),
 *    t = (dz * 3 + dy) * 3 + dx with offsets (dz-1, dy-1, dx-1);
 *  - pool = mean of the 8 children; up = nearest (the parent's value);
 *  - network: e0a, e0b | pool | e1a, e1b | pool | ba, bb | up, concat s1 |
 *    d1a, d1b | up, concat s0 | d0a, d0b | head out = wh . h + bh;
 *  - loss = sum over fluid cells (out - t)^2 / nFluid.
 * round = 1 applies the GPU's BF16 rounding (round to nearest even) at the
 * same points: weights, input, every stored activation and every stored
 * gradient tensor; accumulation is in double here (FP32 on the GPU).
 * round = 0 computes everything in double, for finite-difference checks.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define TX 8
#define TY 16
#define TZ 8
#define NLAYERS 10

typedef struct { const char* name; int level, c0, c1, cout; } layer_t;
static const layer_t LAYERS[NLAYERS] = {
  {"e0a", 0, 0, 16, 16}, {"e0b", 0, 0, 16, 16}, {"e1a", 1, 0, 16, 32}, {"e1b", 1, 0, 32, 32},
  {"ba", 2, 0, 32, 64},  {"bb", 2, 0, 64, 64},  {"d1a", 1, 64, 32, 32}, {"d1b", 1, 0, 32, 32},
  {"d0a", 0, 32, 16, 16}, {"d0b", 0, 0, 16, 16},
};

typedef struct { int nx, ny, nz, ntx, nty, ntz; long nv; uint8_t* act; } lev_t;

static int g_round = 1;
/* BF16 round to nearest even of a float value (IEEE binary32 -> upper 16 bits) */
static double rb(double x) {
  if (!g_round) return x;
  float f = (float)x;
  uint32_t u; memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  memcpy(&f, &u, 4);
  return (double)f;
}

static long woff_of[NLAYERS], boff_of[NLAYERS], head_off, nparams_total;
static void layout(void) {
  long n = 0;
  for (int l = 0; l < NLAYERS; l++) {
    woff_of[l] = n; n += 27L * (LAYERS[l].c0 + LAYERS[l].c1) * LAYERS[l].cout;
    boff_of[l] = n; n += LAYERS[l].cout;
  }
  head_off = n; n += 17;
  nparams_total = n;
}
int64_t un_num_params(void) { layout(); return nparams_total; }

static int active(const lev_t* L, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= L->nx || y >= L->ny || z >= L->nz) return 0;
  return L->act[((z / TZ) * L->nty + y / TY) * L->ntx + x / TX];
}
static long vidx(const lev_t* L, int x, int y, int z) { return ((long)z * L->ny + y) * L->nx + x; }

/* input value of a conv at voxel (x,y,z), channel c: concat(up(src0), src1) */
static double in_at(const lev_t* L, const lev_t* C, const double* src0, int c0, const double* src1, int c1,
                    int x, int y, int z, int c) {
  if (!active(L, x, y, z)) return 0.0;
  if (c < c0) return src0[vidx(C, x >> 1, y >> 1, z >> 1) * c0 + c];
  return src1[vidx(L, x, y, z) * c1 + (c - c0)];
}

static void conv_fwd(const lev_t* L, const lev_t* C, int l, const double* W, const double* b,
                     const double* src0, const double* src1, double* out) {
  const int c0 = LAYERS[l].c0, c1 = LAYERS[l].c1, cin = c0 + c1, cout = LAYERS[l].cout;
  memset(out, 0, sizeof(double) * L->nv * cout);
  double* acc = (double*)malloc(sizeof(double) * cout);
  for (int z = 0; z < L->nz; z++) for (int y = 0; y < L->ny; y++) for (int x = 0; x < L->nx; x++) {
    if (!active(L, x, y, z)) continue;
    for (int co = 0; co < cout; co++) acc[co] = 0;
    for (int t = 0; t < 27; t++) {
      int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
      int X = x + dx, Y = y + dy, Z = z + dz;
      if (!active(L, X, Y, Z)) continue;
      for (int ci = 0; ci < cin; ci++) {
        double v = in_at(L, C, src0, c0, src1, c1, X, Y, Z, ci);
        if (v == 0.0) continue;
        for (int co = 0; co < cout; co++) acc[co] += v * W[((long)co * cin + ci) * 27 + t];
      }
    }
    for (int co = 0; co < cout; co++) {
      double r = acc[co] + b[co];
      out[vidx(L, x, y, z) * cout + co] = rb(r > 0 ? r : 0.0);
    }
  }
  free(acc);
}
/* dW, db of layer l from its input and dZ; dX (masked by mask > 0 when
 * given, or split into the upsampled part dup and the skip part dskip) */
static void conv_bwd(const lev_t* L, const lev_t* C, int l, const double* W, const double* src0, const double* src1,
                     const double* dz, double* gW, double* gb, const double* mask, double* dx0, double* dx1) {
  const int c0 = LAYERS[l].c0, c1 = LAYERS[l].c1, cin = c0 + c1, cout = LAYERS[l].cout;
  for (int z = 0; z < L->nz; z++) for (int y = 0; y < L->ny; y++) for (int x = 0; x < L->nx; x++) {
    if (!active(L, x, y, z)) continue;
    const double* d = dz + vidx(L, x, y, z) * cout;
    for (int co = 0; co < cout; co++) gb[co] += d[co];
    for (int t = 0; t < 27; t++) {
      int X = x + t % 3 - 1, Y = y + (t / 3) % 3 - 1, Z = z + t / 9 - 1;
      if (!active(L, X, Y, Z)) continue;
      for (int ci = 0; ci < cin; ci++) {
        double v = in_at(L, C, src0, c0, src1, c1, X, Y, Z, ci);
        if (v == 0.0) continue;
        for (int co = 0; co < cout; co++) gW[((long)co * cin + ci) * 27 + t] += v * d[co];
      }
    }
  }
  if (!dx0 && !dx1) return;
  double* acc = (double*)malloc(sizeof(double) * cin);
  for (int z = 0; z < L->nz; z++) for (int y = 0; y < L->ny; y++) for (int x = 0; x < L->nx; x++) {
    if (!active(L, x, y, z)) continue;
    for (int ci = 0; ci < cin; ci++) acc[ci] = 0;
    for (int t = 0; t < 27; t++) {
      int X = x - (t % 3 - 1), Y = y - ((t / 3) % 3 - 1), Z = z - (t / 9 - 1);
      if (!active(L, X, Y, Z)) continue;
      const double* d = dz + vidx(L, X, Y, Z) * cout;
      for (int co = 0; co < cout; co++) {
        if (d[co] == 0.0) continue;
        for (int ci = 0; ci < cin; ci++) acc[ci] += d[co] * W[((long)co * cin + ci) * 27 + t];
      }
    }
    long v = vidx(L, x, y, z);
    if (c0 > 0) {
      for (int ci = 0; ci < c0; ci++) dx0[v * c0 + ci] = rb(acc[ci]);
      for (int ci = c0; ci < cin; ci++) dx1[v * c1 + ci - c0] = rb(acc[ci]);
    } else {
      for (int ci = 0; ci < cin; ci++) {
        double r = acc[ci];
        if (mask && !(mask[v * cin + ci] > 0)) r = 0;
        dx0[v * cin + ci] = rb(r);
      }
    }
  }
  free(acc);
}
static void pool_fwd(const lev_t* F, const lev_t* C, const double* fine, double* coarse, int ch) {
  memset(coarse, 0, sizeof(double) * C->nv * ch);
  for (int z = 0; z < C->nz; z++) for (int y = 0; y < C->ny; y++) for (int x = 0; x < C->nx; x++) {
    if (!active(C, x, y, z)) continue;
    for (int c = 0; c < ch; c++) {
      double s = 0;
      for (int k = 0; k < 8; k++) {
        int fx = 2 * x + (k & 1), fy = 2 * y + ((k >> 1) & 1), fz = 2 * z + (k >> 2);
        if (active(F, fx, fy, fz)) s += fine[vidx(F, fx, fy, fz) * ch + c];
      }
      coarse[vidx(C, x, y, z) * ch + c] = rb(s * 0.125);
    }
  }
}
static void up_bwd(const lev_t* C, const lev_t* F, const double* dup, const double* act, double* dc, int ch) {
  memset(dc, 0, sizeof(double) * C->nv * ch);
  for (int z = 0; z < C->nz; z++) for (int y = 0; y < C->ny; y++) for (int x = 0; x < C->nx; x++) {
    if (!active(C, x, y, z)) continue;
    long v = vidx(C, x, y, z);
    for (int c = 0; c < ch; c++) {
      double s = 0;
      for (int k = 0; k < 8; k++) {
        int fx = 2 * x + (k & 1), fy = 2 * y + ((k >> 1) & 1), fz = 2 * z + (k >> 2);
        if (active(F, fx, fy, fz)) s += dup[vidx(F, fx, fy, fz) * ch + c];
      }
      dc[v * ch + c] = rb(act[v * ch + c] > 0 ? s : 0.0);
    }
  }
}
static void pool_bwd_add(const lev_t* F, const lev_t* C, const double* dskip, const double* dpool,
                         const double* s, double* ds, int ch) {
  memset(ds, 0, sizeof(double) * F->nv * ch);
  for (int z = 0; z < F->nz; z++) for (int y = 0; y < F->ny; y++) for (int x = 0; x < F->nx; x++) {
    if (!active(F, x, y, z)) continue;
    long v = vidx(F, x, y, z), p = vidx(C, x >> 1, y >> 1, z >> 1);
    for (int c = 0; c < ch; c++)
      ds[v * ch + c] = rb(s[v * ch + c] > 0 ? dskip[v * ch + c] + 0.125 * dpool[p * ch + c] : 0.0);
  }
}

typedef struct {
  lev_t L[3];
  double *x, *e0a, *s0, *p1, *e1a, *s1, *p2, *ba, *bb, *d1a, *d1b, *d0a, *h;
  double* W;      /* rounded weights (biases and head unrounded) */
  double* out;
  int nFluid;
} net_t;

static void build_levels(net_t* N, int nx, int ny, int nz, const uint8_t* types) {
  for (int l = 0; l < 3; l++) {
    lev_t* L = &N->L[l];
    L->nx = nx; L->ny = ny; L->nz = nz;
    L->ntx = (nx + TX - 1) / TX; L->nty = (ny + TY - 1) / TY; L->ntz = (nz + TZ - 1) / TZ;
    L->nv = (long)nx * ny * nz;
    L->act = (uint8_t*)calloc((size_t)L->ntx * L->nty * L->ntz, 1);
    nx = (nx + 1) / 2; ny = (ny + 1) / 2; nz = (nz + 1) / 2;
  }
  lev_t* L0 = &N->L[0];
  N->nFluid = 0;
  for (int z = 0; z < L0->nz; z++) for (int y = 0; y < L0->ny; y++) for (int x = 0; x < L0->nx; x++)
    if (types[vidx(L0, x, y, z)] == 1) { L0->act[((z / TZ) * L0->nty + y / TY) * L0->ntx + x / TX] = 1; N->nFluid++; }
  for (int l = 1; l < 3; l++) {
    lev_t *L = &N->L[l], *F = &N->L[l - 1];
    for (int tz = 0; tz < L->ntz; tz++) for (int ty = 0; ty < L->nty; ty++) for (int tx = 0; tx < L->ntx; tx++) {
      int a = 0;
      for (int k = 0; k < 8; k++) {
        int fx = 2 * tx + (k & 1), fy = 2 * ty + ((k >> 1) & 1), fz = 2 * tz + (k >> 2);
        if (fx < F->ntx && fy < F->nty && fz < F->ntz) a |= F->act[(fz * F->nty + fy) * F->ntx + fx];
      }
      L->act[(tz * L->nty + ty) * L->ntx + tx] = (uint8_t)a;
    }
  }
}
static double* zalloc(long n) { return (double*)calloc((size_t)n, sizeof(double)); }

static void net_forward(net_t* N, const float* params, const float* r0n, const uint8_t* types) {
  lev_t *L0 = &N->L[0], *L1 = &N->L[1], *L2 = &N->L[2];
  layout();
  N->W = zalloc(nparams_total);
  for (long i = 0; i < nparams_total; i++) N->W[i] = params[i];
  for (int l = 0; l < NLAYERS; l++) {
    long n = 27L * (LAYERS[l].c0 + LAYERS[l].c1) * LAYERS[l].cout;
    for (long i = 0; i < n; i++) N->W[woff_of[l] + i] = rb(params[woff_of[l] + i]);
  }
  N->x = zalloc(L0->nv * 16);
  for (int z = 0; z < L0->nz; z++) for (int y = 0; y < L0->ny; y++) for (int x = 0; x < L0->nx; x++) {
    if (!active(L0, x, y, z)) continue;
    long v = vidx(L0, x, y, z);
    N->x[v * 16 + 0] = rb(r0n[v]);
    N->x[v * 16 + 1] = types[v] == 1; N->x[v * 16 + 2] = types[v] == 2; N->x[v * 16 + 3] = types[v] == 0;
  }
#define WL(l) (N->W + woff_of[l]), (N->W + boff_of[l])
  N->e0a = zalloc(L0->nv * 16); conv_fwd(L0, L1, 0, WL(0), NULL, N->x, N->e0a);
  N->s0 = zalloc(L0->nv * 16); conv_fwd(L0, L1, 1, WL(1), NULL, N->e0a, N->s0);
  N->p1 = zalloc(L1->nv * 16); pool_fwd(L0, L1, N->s0, N->p1, 16);
  N->e1a = zalloc(L1->nv * 32); conv_fwd(L1, L2, 2, WL(2), NULL, N->p1, N->e1a);
  N->s1 = zalloc(L1->nv * 32); conv_fwd(L1, L2, 3, WL(3), NULL, N->e1a, N->s1);
  N->p2 = zalloc(L2->nv * 32); pool_fwd(L1, L2, N->s1, N->p2, 32);
  N->ba = zalloc(L2->nv * 64); conv_fwd(L2, NULL, 4, WL(4), NULL, N->p2, N->ba);
  N->bb = zalloc(L2->nv * 64); conv_fwd(L2, NULL, 5, WL(5), NULL, N->ba, N->bb);
  N->d1a = zalloc(L1->nv * 32); conv_fwd(L1, L2, 6, WL(6), N->bb, N->s1, N->d1a);
  N->d1b = zalloc(L1->nv * 32); conv_fwd(L1, L2, 7, WL(7), NULL, N->d1a, N->d1b);
  N->d0a = zalloc(L0->nv * 16); conv_fwd(L0, L1, 8, WL(8), N->d1b, N->s0, N->d0a);
  N->h = zalloc(L0->nv * 16); conv_fwd(L0, L1, 9, WL(9), NULL, N->d0a, N->h);
  N->out = zalloc(L0->nv);
  const double* hw = N->W + head_off;
  for (int z = 0; z < L0->nz; z++) for (int y = 0; y < L0->ny; y++) for (int x = 0; x < L0->nx; x++) {
    if (!active(L0, x, y, z)) continue;
    long v = vidx(L0, x, y, z);
    double o = hw[16];
    for (int c = 0; c < 16; c++) o += hw[c] * N->h[v * 16 + c];
    N->out[v] = o;
  }
}
static void net_free(net_t* N) {
  double* b[] = { N->x, N->e0a, N->s0, N->p1, N->e1a, N->s1, N->p2, N->ba, N->bb, N->d1a, N->d1b, N->d0a, N->h,
                  N->W, N->out };
  for (unsigned i = 0; i < sizeof(b) / sizeof(b[0]); i++) free(b[i]);
  for (int l = 0; l < 3; l++) free(N->L[l].act);
}

/* network output (before the gain) at every cell, 0 outside active tiles */
void un_forward(int nx, int ny, int nz, const float* params, const float* r0n, const uint8_t* types, int round,
                float* out) {
  net_t N; memset(&N, 0, sizeof(N));
  g_round = round;
  build_levels(&N, nx, ny, nz, types);
  net_forward(&N, params, r0n, types);
  for (long v = 0; v < N.L[0].nv; v++) out[v] = (float)N.out[v];
  net_free(&N);
}

/* loss over fluid cells against target (already divided by the gain) and
 * its gradient with respect to every parameter (flat, like the weights) */
double un_loss_grad(int nx, int ny, int nz, const float* params, const float* r0n, const uint8_t* types,
                    const float* target, int round, double* grads) {
  net_t N; memset(&N, 0, sizeof(N));
  g_round = round;
  build_levels(&N, nx, ny, nz, types);
  net_forward(&N, params, r0n, types);
  lev_t *L0 = &N.L[0], *L1 = &N.L[1], *L2 = &N.L[2];
  memset(grads, 0, sizeof(double) * nparams_total);
  const double* hw = N.W + head_off;
  double loss = 0;
  int nf = N.nFluid > 0 ? N.nFluid : 1;
  double* gh = zalloc(L0->nv * 16);
  for (int z = 0; z < L0->nz; z++) for (int y = 0; y < L0->ny; y++) for (int x = 0; x < L0->nx; x++) {
    if (!active(L0, x, y, z)) continue;
    long v = vidx(L0, x, y, z);
    double dout = 0;
    if (types[v] == 1) { double diff = N.out[v] - target[v]; loss += diff * diff / nf; dout = 2 * diff / nf; }
    for (int c = 0; c < 16; c++) {
      grads[head_off + c] += dout * N.h[v * 16 + c];
      gh[v * 16 + c] = rb(N.h[v * 16 + c] > 0 ? dout * hw[c] : 0.0);
    }
    grads[head_off + 16] += dout;
  }
#define GL(l) (grads + woff_of[l]), (grads + boff_of[l])
  double* gd0a = zalloc(L0->nv * 16);
  conv_bwd(L0, L1, 9, N.W + woff_of[9], NULL, N.d0a, gh, GL(9), N.d0a, gd0a, NULL);
  double *gup1 = zalloc(L0->nv * 32), *gs0a = zalloc(L0->nv * 16);
  conv_bwd(L0, L1, 8, N.W + woff_of[8], N.d1b, N.s0, gd0a, GL(8), NULL, gup1, gs0a);
  double* gd1b = zalloc(L1->nv * 32); up_bwd(L1, L0, gup1, N.d1b, gd1b, 32);
  double* gd1a = zalloc(L1->nv * 32);
  conv_bwd(L1, L2, 7, N.W + woff_of[7], NULL, N.d1a, gd1b, GL(7), N.d1a, gd1a, NULL);
  double *gup2 = zalloc(L1->nv * 64), *gs1a = zalloc(L1->nv * 32);
  conv_bwd(L1, L2, 6, N.W + woff_of[6], N.bb, N.s1, gd1a, GL(6), NULL, gup2, gs1a);
  double* gbb = zalloc(L2->nv * 64); up_bwd(L2, L1, gup2, N.bb, gbb, 64);
  double* gba = zalloc(L2->nv * 64);
  conv_bwd(L2, NULL, 5, N.W + woff_of[5], NULL, N.ba, gbb, GL(5), N.ba, gba, NULL);
  double* gp2 = zalloc(L2->nv * 32);
  conv_bwd(L2, NULL, 4, N.W + woff_of[4], NULL, N.p2, gba, GL(4), NULL, gp2, NULL);
  double* gs1 = zalloc(L1->nv * 32); pool_bwd_add(L1, L2, gs1a, gp2, N.s1, gs1, 32);
  double* ge1a = zalloc(L1->nv * 32);
  conv_bwd(L1, L2, 3, N.W + woff_of[3], NULL, N.e1a, gs1, GL(3), N.e1a, ge1a, NULL);
  double* gp1 = zalloc(L1->nv * 16);
  conv_bwd(L1, L2, 2, N.W + woff_of[2], NULL, N.p1, ge1a, GL(2), NULL, gp1, NULL);
  double* gs0 = zalloc(L0->nv * 16); pool_bwd_add(L0, L1, gs0a, gp1, N.s0, gs0, 16);
  double* ge0a = zalloc(L0->nv * 16);
  conv_bwd(L0, L1, 1, N.W + woff_of[1], NULL, N.e0a, gs0, GL(1), N.e0a, ge0a, NULL);
  conv_bwd(L0, L1, 0, N.W + woff_of[0], NULL, N.x, ge0a, GL(0), NULL, NULL, NULL);
  double* fr[] = { gh, gd0a, gup1, gs0a, gd1b, gd1a, gup2, gs1a, gbb, gba, gp2, gs1, ge1a, gp1, gs0, ge0a };
  for (unsigned i = 0; i < sizeof(fr) / sizeof(fr[0]); i++) free(fr[i]);
  net_free(&N);
  return loss;
}
