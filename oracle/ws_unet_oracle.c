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
 *  - network (3 levels): e0a, e0b | pool | e1a, e1b | pool | ba, bb | up,
 *    concat s1 | d1a, d1b | up, concat s0 | d0a, d0b | head out = wh . h + bh;
 *    with 4 levels e2a, e2b | pool sit before the bottleneck (now 64 -> 128
 *    channels) and d2a, d2b (up, concat s2) after it; channels 16 << level;
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
#define MAXLEV 4
#define MAXLAYERS (4 * (MAXLEV - 1) + 2)

typedef struct { const char* name; int level, c0, c1, cout; } layer_t;
/* the layers of the network in use (forward order): per level l below the
 * bottleneck e<l>a, e<l>b; the bottleneck ba, bb; per level l from the
 * bottleneck down d<l>a (upsampled input | skip), d<l>b */
static layer_t LAYERS[MAXLAYERS];
static int g_levels = 0, NLAYERS = 0;
static void set_levels(int levels) {
  static const char* encA[] = { "e0a", "e1a", "e2a" };
  static const char* encB[] = { "e0b", "e1b", "e2b" };
  static const char* decA[] = { "d0a", "d1a", "d2a" };
  static const char* decB[] = { "d0b", "d1b", "d2b" };
  int n = 0;
  for (int l = 0; l + 1 < levels; l++) {
    int c = 16 << l, cin = l == 0 ? 16 : 16 << (l - 1);
    layer_t a = { encA[l], l, 0, cin, c }, b = { encB[l], l, 0, c, c };
    LAYERS[n++] = a; LAYERS[n++] = b;
  }
  int cb = 16 << (levels - 1);
  layer_t ba = { "ba", levels - 1, 0, cb / 2, cb }, bb = { "bb", levels - 1, 0, cb, cb };
  LAYERS[n++] = ba; LAYERS[n++] = bb;
  for (int l = levels - 2; l >= 0; l--) {
    int c = 16 << l;
    layer_t a = { decA[l], l, 2 * c, c, c }, b = { decB[l], l, 0, c, c };
    LAYERS[n++] = a; LAYERS[n++] = b;
  }
  g_levels = levels; NLAYERS = n;
}
static int enc_a(int l) { return 2 * l; }
static int enc_b(int l) { return 2 * l + 1; }
static int bot_a(void) { return 2 * (g_levels - 1); }
static int bot_b(void) { return 2 * (g_levels - 1) + 1; }
static int dec_a(int l) { return 2 * (g_levels - 1) + 2 + 2 * (g_levels - 2 - l); }
static int dec_b(int l) { return dec_a(l) + 1; }
static int chan(int l) { return 16 << l; }

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

static long woff_of[MAXLAYERS], boff_of[MAXLAYERS], head_off, nparams_total;
static void layout(void) {
  long n = 0;
  for (int l = 0; l < NLAYERS; l++) {
    woff_of[l] = n; n += 27L * (LAYERS[l].c0 + LAYERS[l].c1) * LAYERS[l].cout;
    boff_of[l] = n; n += LAYERS[l].cout;
  }
  head_off = n; n += 17;
  nparams_total = n;
}
int64_t un_num_params_levels(int levels) { set_levels(levels); layout(); return nparams_total; }
int64_t un_num_params(void) { return un_num_params_levels(3); }

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
  lev_t L[MAXLEV];
  double *x, *ea[MAXLEV], *sk[MAXLEV], *pl[MAXLEV], *bA, *bB, *da[MAXLEV], *db[MAXLEV];
  double* W;      /* rounded weights (biases and head unrounded) */
  double* out;
  int nFluid;
} net_t;

static void build_levels(net_t* N, int nx, int ny, int nz, const uint8_t* types) {
  for (int l = 0; l < g_levels; l++) {
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
  for (int l = 1; l < g_levels; l++) {
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
  lev_t* L0 = &N->L[0];
  const int LB = g_levels - 1;
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
  const double* cur = N->x;
  for (int l = 0; l < LB; l++) {
    lev_t *L = &N->L[l], *C = &N->L[l + 1];
    N->ea[l] = zalloc(L->nv * chan(l)); conv_fwd(L, C, enc_a(l), WL(enc_a(l)), NULL, cur, N->ea[l]);
    N->sk[l] = zalloc(L->nv * chan(l)); conv_fwd(L, C, enc_b(l), WL(enc_b(l)), NULL, N->ea[l], N->sk[l]);
    N->pl[l + 1] = zalloc(C->nv * chan(l)); pool_fwd(L, C, N->sk[l], N->pl[l + 1], chan(l));
    cur = N->pl[l + 1];
  }
  lev_t* LBt = &N->L[LB];
  N->bA = zalloc(LBt->nv * chan(LB)); conv_fwd(LBt, NULL, bot_a(), WL(bot_a()), NULL, cur, N->bA);
  N->bB = zalloc(LBt->nv * chan(LB)); conv_fwd(LBt, NULL, bot_b(), WL(bot_b()), NULL, N->bA, N->bB);
  const double* up = N->bB;
  for (int l = LB - 1; l >= 0; l--) {
    lev_t *L = &N->L[l], *C = &N->L[l + 1];
    N->da[l] = zalloc(L->nv * chan(l)); conv_fwd(L, C, dec_a(l), WL(dec_a(l)), up, N->sk[l], N->da[l]);
    N->db[l] = zalloc(L->nv * chan(l)); conv_fwd(L, C, dec_b(l), WL(dec_b(l)), NULL, N->da[l], N->db[l]);
    up = N->db[l];
  }
  N->out = zalloc(L0->nv);
  const double* hw = N->W + head_off;
  const double* h = N->db[0];
  for (int z = 0; z < L0->nz; z++) for (int y = 0; y < L0->ny; y++) for (int x = 0; x < L0->nx; x++) {
    if (!active(L0, x, y, z)) continue;
    long v = vidx(L0, x, y, z);
    double o = hw[16];
    for (int c = 0; c < 16; c++) o += hw[c] * h[v * 16 + c];
    N->out[v] = o;
  }
}
static void net_free(net_t* N) {
  free(N->x); free(N->bA); free(N->bB); free(N->W); free(N->out);
  for (int l = 0; l < MAXLEV; l++) { free(N->ea[l]); free(N->sk[l]); free(N->pl[l]); free(N->da[l]); free(N->db[l]); }
  for (int l = 0; l < g_levels; l++) free(N->L[l].act);
}

/* network output (before the gain) at every cell, 0 outside active tiles */
void un_forward_levels(int nx, int ny, int nz, int levels, const float* params, const float* r0n, const uint8_t* types,
                       int round, float* out) {
  net_t N; memset(&N, 0, sizeof(N));
  g_round = round;
  set_levels(levels);
  build_levels(&N, nx, ny, nz, types);
  net_forward(&N, params, r0n, types);
  for (long v = 0; v < N.L[0].nv; v++) out[v] = (float)N.out[v];
  net_free(&N);
}
void un_forward(int nx, int ny, int nz, const float* params, const float* r0n, const uint8_t* types, int round,
                float* out) {
  un_forward_levels(nx, ny, nz, 3, params, r0n, types, round, out);
}

/* loss over fluid cells against target (already divided by the gain) and
 * its gradient with respect to every parameter (flat, like the weights) */
double un_loss_grad_levels(int nx, int ny, int nz, int levels, const float* params, const float* r0n,
                           const uint8_t* types, const float* target, int round, double* grads) {
  net_t N; memset(&N, 0, sizeof(N));
  g_round = round;
  set_levels(levels);
  build_levels(&N, nx, ny, nz, types);
  net_forward(&N, params, r0n, types);
  const int LB = g_levels - 1;
  lev_t* L0 = &N.L[0];
  memset(grads, 0, sizeof(double) * nparams_total);
  const double* hw = N.W + head_off;
  const double* h = N.db[0];
  double loss = 0;
  int nf = N.nFluid > 0 ? N.nFluid : 1;
  double *gdb[MAXLEV] = { 0 }, *gda[MAXLEV] = { 0 }, *gup[MAXLEV] = { 0 }, *gsa[MAXLEV] = { 0 };
  double *gp[MAXLEV] = { 0 }, *gs[MAXLEV] = { 0 }, *gea[MAXLEV] = { 0 };
  gdb[0] = zalloc(L0->nv * 16);
  for (int z = 0; z < L0->nz; z++) for (int y = 0; y < L0->ny; y++) for (int x = 0; x < L0->nx; x++) {
    if (!active(L0, x, y, z)) continue;
    long v = vidx(L0, x, y, z);
    double dout = 0;
    if (types[v] == 1) { double diff = N.out[v] - target[v]; loss += diff * diff / nf; dout = 2 * diff / nf; }
    for (int c = 0; c < 16; c++) {
      grads[head_off + c] += dout * h[v * 16 + c];
      gdb[0][v * 16 + c] = rb(h[v * 16 + c] > 0 ? dout * hw[c] : 0.0);
    }
    grads[head_off + 16] += dout;
  }
#define GL(l) (grads + woff_of[l]), (grads + boff_of[l])
#define WOF(l) (N.W + woff_of[l])
  double *gbA = zalloc(N.L[LB].nv * chan(LB)), *gbB = zalloc(N.L[LB].nv * chan(LB));
  /* decoder, from level 0 up */
  for (int l = 0; l < LB; l++) {
    lev_t *L = &N.L[l], *C = &N.L[l + 1];
    gda[l] = zalloc(L->nv * chan(l));
    conv_bwd(L, C, dec_b(l), WOF(dec_b(l)), NULL, N.da[l], gdb[l], GL(dec_b(l)), N.da[l], gda[l], NULL);
    const double* upSrc = l + 1 < LB ? N.db[l + 1] : N.bB;
    gup[l] = zalloc(L->nv * chan(l + 1)); gsa[l] = zalloc(L->nv * chan(l));
    conv_bwd(L, C, dec_a(l), WOF(dec_a(l)), upSrc, N.sk[l], gda[l], GL(dec_a(l)), NULL, gup[l], gsa[l]);
    double* tgt = gbB;
    if (l + 1 < LB) { gdb[l + 1] = zalloc(C->nv * chan(l + 1)); tgt = gdb[l + 1]; }
    up_bwd(C, L, gup[l], upSrc, tgt, chan(l + 1));
  }
  /* bottleneck */
  lev_t* LBt = &N.L[LB];
  conv_bwd(LBt, NULL, bot_b(), WOF(bot_b()), NULL, N.bA, gbB, GL(bot_b()), N.bA, gbA, NULL);
  gp[LB] = zalloc(LBt->nv * chan(LB - 1));
  conv_bwd(LBt, NULL, bot_a(), WOF(bot_a()), NULL, N.pl[LB], gbA, GL(bot_a()), NULL, gp[LB], NULL);
  /* encoder, from the deepest level down */
  for (int l = LB - 1; l >= 0; l--) {
    lev_t *L = &N.L[l], *C = &N.L[l + 1];
    gs[l] = zalloc(L->nv * chan(l)); pool_bwd_add(L, C, gsa[l], gp[l + 1], N.sk[l], gs[l], chan(l));
    gea[l] = zalloc(L->nv * chan(l));
    conv_bwd(L, C, enc_b(l), WOF(enc_b(l)), NULL, N.ea[l], gs[l], GL(enc_b(l)), N.ea[l], gea[l], NULL);
    if (l > 0) {
      gp[l] = zalloc(L->nv * chan(l - 1));
      conv_bwd(L, C, enc_a(l), WOF(enc_a(l)), NULL, N.pl[l], gea[l], GL(enc_a(l)), NULL, gp[l], NULL);
    } else {
      conv_bwd(L, C, enc_a(0), WOF(enc_a(0)), NULL, N.x, gea[0], GL(enc_a(0)), NULL, NULL, NULL);
    }
  }
  for (int l = 0; l < MAXLEV; l++) { free(gdb[l]); free(gda[l]); free(gup[l]); free(gsa[l]); free(gp[l]); free(gs[l]); free(gea[l]); }
  free(gbA); free(gbB);
  net_free(&N);
  return loss;
}
double un_loss_grad(int nx, int ny, int nz, const float* params, const float* r0n, const uint8_t* types,
                    const float* target, int round, double* grads) {
  return un_loss_grad_levels(nx, ny, nz, 3, params, r0n, types, target, round, grads);
}
