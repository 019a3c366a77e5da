/*
 * sk_oracle_net.c -- CPU oracle of the learned FGMRES preconditioner.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference has no learned preconditioner
 * (its FGMRES, sparkit/data/fgmres.hpp:96-428, takes any callable as the
 * variable preconditioner); this file restates, in plain C and double
 * precision, the network, its input features, its training loss and the
 * analytic backward pass that the CUDA library implements, so that the
 * library's forward output and parameter gradients can be checked.
 *
 * With round_bf16 != 0 every tensor the library stores in BF16 is rounded
 * to BF16 (round to nearest even) at the same points; the arithmetic in
 * between is double, where the library accumulates in FP32, so the two
 * agree to accumulation-order rounding plus an occasional one-ulp BF16
 * difference.  With round_bf16 == 0 nothing is rounded, which is the form
 * the finite-difference check of the gradients uses.
 *
 * Network (all convolutions 3x3, zero padding, stride 1; NHWC tensors):
 *   level 0 (H x W): e0 = relu(conv0(x; 8->16))
 *   level 1 (H/2):   e1 = relu(conv1(pool(e0); 16->32))
 *   level 2 (H/4):   e2 = relu(conv2(pool(e1); 32->64))
 *   level 3 (H/8):   e3 = relu(conv3(pool(e2); 64->64)); b3 = relu(conv4(e3))
 *   level 2:         d2 = relu(conv5(up(b3) + e2; 64->32))
 *   level 1:         d1 = relu(conv6(up(d2) + e1; 32->16))
 *   level 0:         d0 = relu(conv7(up(d1) + e0; 16->16)); y = conv8(d0; 16->1)
 * pool = 2x2 average, up = nearest-neighbour 2x.
 *
 * Parameters, flat FP32 in layer order: W_l[cout][9][cin] (tap t = 3 ky +
 * kx reads input pixel (y + ky - 1, x + kx - 1)) then b_l[cout].
 *
 * Features of a residual r on a 5-point grid with coefficient planes
 * (diag d, west w, east e, south s, north n, inverse diagonal invd):
 *   rt = r * invd (double), s = sqrt(mean(rt^2)),
 *   x[.,0] = bf16(float(rt / s)), x[.,1..4] = bf16(float(w|e|s|n * invd)),
 *   x[.,5..7] = 0.
 * The preconditioner returns z = s * y.
 *
 * Loss of a batch of (r, e) pairs (e the error x* - x_k, so that A e = r):
 *   tgt = float(e / s), dif = y - tgt, rho = A dif (the 5-point stencil of
 *   the coefficient planes, zero outside the grid),
 *   L = mean_b [ |rho|^2 / |r / s|^2 + mu |dif|^2 / |tgt|^2 ].
 */
#include "sk_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NL 9
static const int CIN[NL] = {8, 16, 32, 64, 64, 64, 32, 16, 16};
static const int COUT[NL] = {16, 32, 64, 64, 64, 32, 16, 16, 1};

int64_t skon_param_count(void) {
  int64_t n = 0;
  for (int l = 0; l < NL; ++l) n += (int64_t)COUT[l] * 9 * CIN[l] + COUT[l];
  return n;
}

static int64_t woff(int l) {
  int64_t n = 0;
  for (int k = 0; k < l; ++k) n += (int64_t)COUT[k] * 9 * CIN[k] + COUT[k];
  return n;
}

/* round to nearest even BF16 of a float */
static float bf16f(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return f; /* inf / nan unchanged */
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  memcpy(&f, &u, 4);
  return f;
}

static double q(double v, int rb) { return rb ? (double)bf16f((float)v) : v; }

/* 3x3 convolution of in[B][H][W][ci] with W[co][9][ci] (+ bias when b is
 * non-null), no rounding, into out[B][H][W][co] (overwritten). */
static void conv(int B, int H, int W, int ci, int co, const double* in, const double* w,
                 const double* b, double* out) {
  for (int bb = 0; bb < B; ++bb)
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x)
        for (int o = 0; o < co; ++o) {
          double acc = 0.0;
          for (int t = 0; t < 9; ++t) {
            const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
            if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
            const double* px = in + (((int64_t)bb * H + yy) * W + xx) * ci;
            const double* wr = w + ((int64_t)o * 9 + t) * ci;
            for (int c = 0; c < ci; ++c) acc += px[c] * wr[c];
          }
          out[(((int64_t)bb * H + y) * W + x) * co + o] = acc + (b ? b[o] : 0.0);
        }
}

/* transposed convolution: dx[y][x][c] = sum_t sum_o g[y-ky+1][x-kx+1][o] W[o][t][c] */
static void conv_t(int B, int H, int W, int ci, int co, const double* g, const double* w, double* dx) {
  for (int bb = 0; bb < B; ++bb)
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x)
        for (int c = 0; c < ci; ++c) {
          double acc = 0.0;
          for (int t = 0; t < 9; ++t) {
            const int yy = y - (t / 3) + 1, xx = x - (t % 3) + 1;
            if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
            const double* gp = g + (((int64_t)bb * H + yy) * W + xx) * co;
            for (int o = 0; o < co; ++o) acc += gp[o] * w[((int64_t)o * 9 + t) * ci + c];
          }
          dx[(((int64_t)bb * H + y) * W + x) * ci + c] = acc;
        }
}

/* dW[o][t][c] += sum g[y][x][o] in[y+ky-1][x+kx-1][c]; db[o] += sum g */
static void conv_w(int B, int H, int W, int ci, int co, const double* g, const double* in, double* dw,
                   double* db) {
  for (int bb = 0; bb < B; ++bb)
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x) {
        const double* gp = g + (((int64_t)bb * H + y) * W + x) * co;
        for (int o = 0; o < co; ++o) {
          if (gp[o] == 0.0) continue;
          db[o] += gp[o];
          for (int t = 0; t < 9; ++t) {
            const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
            if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
            const double* px = in + (((int64_t)bb * H + yy) * W + xx) * ci;
            double* wr = dw + ((int64_t)o * 9 + t) * ci;
            for (int c = 0; c < ci; ++c) wr[c] += gp[o] * px[c];
          }
        }
      }
}

static void relu_q(int64_t n, double* a, int relu, int rb) {
  for (int64_t i = 0; i < n; ++i) {
    double v = a[i];
    if (relu && !(v > 0.0)) v = 0.0;
    a[i] = q(v, rb);
  }
}

/* 2x2 average pool, [B][H][W][c] -> [B][H/2][W/2][c] */
static void pool(int B, int H, int W, int c, const double* in, double* out, int rb) {
  const int h = H / 2, w = W / 2;
  for (int bb = 0; bb < B; ++bb)
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x)
        for (int k = 0; k < c; ++k) {
          const double* p = in + (((int64_t)bb * H + 2 * y) * W + 2 * x) * c + k;
          const double s = (p[0] + p[c]) + (p[(int64_t)W * c] + p[(int64_t)W * c + c]);
          out[(((int64_t)bb * h + y) * w + x) * c + k] = q(0.25 * s, rb);
        }
}

/* out = up(coarse) + skip at [B][H][W][c] */
static void upadd(int B, int H, int W, int c, const double* coarse, const double* skip, double* out, int rb) {
  const int h = H / 2, w = W / 2;
  for (int bb = 0; bb < B; ++bb)
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x)
        for (int k = 0; k < c; ++k) {
          const int64_t i = (((int64_t)bb * H + y) * W + x) * c + k;
          out[i] = q(coarse[(((int64_t)bb * h + y / 2) * w + x / 2) * c + k] + skip[i], rb);
        }
}

/* g_coarse = q(sum of the 4 fine gradients) * (act > 0) */
static void upadd_bwd(int B, int H, int W, int c, const double* dfine, const double* act, double* g, int rb) {
  const int h = H / 2, w = W / 2;
  for (int bb = 0; bb < B; ++bb)
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x)
        for (int k = 0; k < c; ++k) {
          const double* p = dfine + (((int64_t)bb * H + 2 * y) * W + 2 * x) * c + k;
          const double s = (p[0] + p[c]) + (p[(int64_t)W * c] + p[(int64_t)W * c + c]);
          const int64_t i = (((int64_t)bb * h + y) * w + x) * c + k;
          g[i] = act[i] > 0.0 ? q(s, rb) : 0.0;
        }
}

/* g = q(dskip + 0.25 up(dpool)) * (act > 0), all at the fine level */
static void pool_bwd(int B, int H, int W, int c, const double* dskip, const double* dpool, const double* act,
                     double* g, int rb) {
  const int h = H / 2, w = W / 2;
  for (int bb = 0; bb < B; ++bb)
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x)
        for (int k = 0; k < c; ++k) {
          const int64_t i = (((int64_t)bb * H + y) * W + x) * c + k;
          const double v = dskip[i] + 0.25 * dpool[(((int64_t)bb * h + y / 2) * w + x / 2) * c + k];
          g[i] = act[i] > 0.0 ? q(v, rb) : 0.0;
        }
}

/* Features of B residuals; coef holds per sample 6 planes of H*W floats:
 * d, w, e, s, n, invd.  Returns the scales s_b. */
void skon_features(int B, int H, int W, const double* r, const float* coef, int rb, double* xin, double* scale) {
  const int64_t P = (int64_t)H * W;
  for (int bb = 0; bb < B; ++bb) {
    const float* cf = coef + (int64_t)bb * 6 * P;
    const double* rr = r + bb * P;
    double ss = 0.0;
    for (int64_t p = 0; p < P; ++p) {
      const double rt = rr[p] * (double)cf[5 * P + p];
      ss += rt * rt;
    }
    const double s = sqrt(ss / (double)P);
    scale[bb] = s;
    for (int64_t p = 0; p < P; ++p) {
      double* xp = xin + (bb * P + p) * 8;
      const float inv = cf[5 * P + p];
      const double rt = rr[p] * (double)inv;
      xp[0] = s > 0.0 ? q((double)(float)(rt / s), rb) : 0.0;
      for (int k = 0; k < 4; ++k) xp[1 + k] = q((double)(cf[(1 + k) * P + p] * inv), rb);
      xp[5] = xp[6] = xp[7] = 0.0;
    }
  }
}

typedef struct {
  double *x0, *e0, *p0, *e1, *p1, *e2, *p2, *e3, *b3, *u2, *d2, *u1, *d1, *u0, *d0, *y;
} acts_t;

static void acts_alloc(acts_t* a, int B, int H, int W) {
  const int64_t P0 = (int64_t)B * H * W, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  a->x0 = calloc(P0 * 8, 8);
  a->e0 = calloc(P0 * 16, 8);
  a->p0 = calloc(P1 * 16, 8);
  a->e1 = calloc(P1 * 32, 8);
  a->p1 = calloc(P2 * 32, 8);
  a->e2 = calloc(P2 * 64, 8);
  a->p2 = calloc(P3 * 64, 8);
  a->e3 = calloc(P3 * 64, 8);
  a->b3 = calloc(P3 * 64, 8);
  a->u2 = calloc(P2 * 64, 8);
  a->d2 = calloc(P2 * 32, 8);
  a->u1 = calloc(P1 * 32, 8);
  a->d1 = calloc(P1 * 16, 8);
  a->u0 = calloc(P0 * 16, 8);
  a->d0 = calloc(P0 * 16, 8);
  a->y = calloc(P0, 8);
}

static void acts_free(acts_t* a) {
  double** p = (double**)a;
  for (size_t i = 0; i < sizeof(acts_t) / sizeof(double*); ++i) free(p[i]);
}

static void load_params(const float* params, double* wd) {
  const int64_t n = skon_param_count();
  for (int64_t i = 0; i < n; ++i) wd[i] = (double)params[i];
}

/* forward from a.x0; rb also rounds the weights to BF16 (the library keeps
 * FP32 master weights and convolves with their BF16 copy; biases stay FP32) */
static void forward(int B, int H, int W, const double* wd, acts_t* a, int rb) {
  const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  const int64_t P0 = (int64_t)B * H * W, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  const double* Wl[NL];
  const double* bl[NL];
  for (int l = 0; l < NL; ++l) {
    Wl[l] = wd + woff(l);
    bl[l] = Wl[l] + (int64_t)COUT[l] * 9 * CIN[l];
  }
  conv(B, H, W, 8, 16, a->x0, Wl[0], bl[0], a->e0);
  relu_q(P0 * 16, a->e0, 1, rb);
  pool(B, H, W, 16, a->e0, a->p0, rb);
  conv(B, H1, W1, 16, 32, a->p0, Wl[1], bl[1], a->e1);
  relu_q(P1 * 32, a->e1, 1, rb);
  pool(B, H1, W1, 32, a->e1, a->p1, rb);
  conv(B, H2, W2, 32, 64, a->p1, Wl[2], bl[2], a->e2);
  relu_q(P2 * 64, a->e2, 1, rb);
  pool(B, H2, W2, 64, a->e2, a->p2, rb);
  conv(B, H3, W3, 64, 64, a->p2, Wl[3], bl[3], a->e3);
  relu_q(P3 * 64, a->e3, 1, rb);
  conv(B, H3, W3, 64, 64, a->e3, Wl[4], bl[4], a->b3);
  relu_q(P3 * 64, a->b3, 1, rb);
  upadd(B, H2, W2, 64, a->b3, a->e2, a->u2, rb);
  conv(B, H2, W2, 64, 32, a->u2, Wl[5], bl[5], a->d2);
  relu_q(P2 * 32, a->d2, 1, rb);
  upadd(B, H1, W1, 32, a->d2, a->e1, a->u1, rb);
  conv(B, H1, W1, 32, 16, a->u1, Wl[6], bl[6], a->d1);
  relu_q(P1 * 16, a->d1, 1, rb);
  upadd(B, H, W, 16, a->d1, a->e0, a->u0, rb);
  conv(B, H, W, 16, 16, a->u0, Wl[7], bl[7], a->d0);
  relu_q(P0 * 16, a->d0, 1, rb);
  conv(B, H, W, 16, 1, a->d0, Wl[8], bl[8], a->y);
  if (rb)
    for (int64_t i = 0; i < P0; ++i) a->y[i] = (double)(float)a->y[i];
}

static void round_weights(double* wd, int rb) {
  if (!rb) return;
  for (int l = 0; l < NL; ++l) {
    double* w = wd + woff(l);
    const int64_t nw = (int64_t)COUT[l] * 9 * CIN[l];
    for (int64_t i = 0; i < nw; ++i) w[i] = q(w[i], 1);
  }
}

/* z = s * net(features(v)) for one grid; y_out (may be NULL) gets y. */
void skon_apply(int H, int W, const float* params, const double* v, const float* coef, int rb, double* z,
                double* y_out) {
  const int64_t P = (int64_t)H * W;
  double* wd = malloc(skon_param_count() * 8);
  load_params(params, wd);
  round_weights(wd, rb);
  acts_t a;
  acts_alloc(&a, 1, H, W);
  double s = 0.0;
  skon_features(1, H, W, v, coef, rb, a.x0, &s);
  forward(1, H, W, wd, &a, rb);
  for (int64_t p = 0; p < P; ++p) {
    z[p] = s * a.y[p];
    if (y_out) y_out[p] = a.y[p];
  }
  acts_free(&a);
  free(wd);
}

/* Loss of a batch and, when grad is non-null, its gradient with respect to
 * the flat parameters (double, skon_param_count() entries). */
double skon_loss_grad(int B, int H, int W, const float* params, const double* r, const double* e,
                      const float* coef, double mu, int rb, double* grad, double* y_out) {
  const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  const int64_t P = (int64_t)H * W, P0 = B * P, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  const int64_t np = skon_param_count();
  double* wd = malloc(np * 8);
  load_params(params, wd);
  round_weights(wd, rb);
  acts_t a;
  acts_alloc(&a, B, H, W);
  double* s = calloc(B, 8);
  skon_features(B, H, W, r, coef, rb, a.x0, s);
  forward(B, H, W, wd, &a, rb);
  if (y_out) memcpy(y_out, a.y, P0 * 8);
  double* dif = calloc(P0, 8);
  double* rho = calloc(P0, 8);
  double* gy = calloc(P0, 8);
  double loss = 0.0;
  for (int bb = 0; bb < B; ++bb) {
    const float* cf = coef + (int64_t)bb * 6 * P;
    const double sb = s[bb];
    double rn2 = 0.0, tn2 = 0.0, rho2 = 0.0, d2 = 0.0;
    for (int64_t p = 0; p < P; ++p) {
      const double rs = sb > 0.0 ? r[bb * P + p] / sb : 0.0;
      rn2 += rs * rs;
      double tg = sb > 0.0 ? e[bb * P + p] / sb : 0.0;
      if (rb) tg = (double)(float)tg;
      tn2 += tg * tg;
      dif[bb * P + p] = a.y[bb * P + p] - tg;
      d2 += dif[bb * P + p] * dif[bb * P + p];
    }
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x) {
        const int64_t p = (int64_t)y * W + x;
        const double* df = dif + bb * P;
        double v = (double)cf[p] * df[p];
        if (x > 0) v += (double)cf[P + p] * df[p - 1];
        if (x + 1 < W) v += (double)cf[2 * P + p] * df[p + 1];
        if (y > 0) v += (double)cf[3 * P + p] * df[p - W];
        if (y + 1 < H) v += (double)cf[4 * P + p] * df[p + W];
        rho[bb * P + p] = v;
        rho2 += v * v;
      }
    const double wr = rn2 > 0.0 ? 1.0 / rn2 : 0.0;
    const double wt = tn2 > 0.0 ? mu / tn2 : 0.0;
    loss += rho2 * wr + d2 * wt;
    /* dL/dy = (2 / B) (A^T rho / rn2 + mu dif / tn2) */
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x) {
        const int64_t p = (int64_t)y * W + x;
        const double* rh = rho + bb * P;
        double v = (double)cf[p] * rh[p];
        if (x > 0) v += (double)cf[2 * P + p - 1] * rh[p - 1];      /* east coefficient of the west cell */
        if (x + 1 < W) v += (double)cf[P + p + 1] * rh[p + 1];      /* west coefficient of the east cell */
        if (y > 0) v += (double)cf[4 * P + p - W] * rh[p - W];      /* north coefficient of the south cell */
        if (y + 1 < H) v += (double)cf[3 * P + p + W] * rh[p + W];  /* south coefficient of the north cell */
        gy[bb * P + p] = (2.0 / B) * (v * wr + dif[bb * P + p] * wt);
      }
  }
  loss /= B;
  if (grad) {
    memset(grad, 0, np * 8);
    double *gw[NL], *gb[NL];
    for (int l = 0; l < NL; ++l) {
      gw[l] = grad + woff(l);
      gb[l] = gw[l] + (int64_t)COUT[l] * 9 * CIN[l];
    }
    const double* Wl[NL];
    for (int l = 0; l < NL; ++l) Wl[l] = wd + woff(l);
    double* g8 = calloc(P0, 8);
    for (int64_t i = 0; i < P0; ++i) g8[i] = q((double)(float)gy[i], rb);
    double* g7 = calloc(P0 * 16, 8);
    double* du0 = calloc(P0 * 16, 8);
    double* g6 = calloc(P1 * 16, 8);
    double* du1 = calloc(P1 * 32, 8);
    double* g5 = calloc(P2 * 32, 8);
    double* du2 = calloc(P2 * 64, 8);
    double* g4 = calloc(P3 * 64, 8);
    double* g3 = calloc(P3 * 64, 8);
    double* dp2 = calloc(P3 * 64, 8);
    double* g2 = calloc(P2 * 64, 8);
    double* dp1 = calloc(P2 * 32, 8);
    double* g1 = calloc(P1 * 32, 8);
    double* dp0 = calloc(P1 * 16, 8);
    double* g0 = calloc(P0 * 16, 8);
    conv_w(B, H, W, 16, 1, g8, a.d0, gw[8], gb[8]);
    conv_t(B, H, W, 16, 1, g8, Wl[8], g7);
    for (int64_t i = 0; i < P0 * 16; ++i) g7[i] = a.d0[i] > 0.0 ? q(g7[i], rb) : 0.0;
    conv_w(B, H, W, 16, 16, g7, a.u0, gw[7], gb[7]);
    conv_t(B, H, W, 16, 16, g7, Wl[7], du0);
    relu_q(P0 * 16, du0, 0, rb);
    upadd_bwd(B, H, W, 16, du0, a.d1, g6, rb);
    conv_w(B, H1, W1, 32, 16, g6, a.u1, gw[6], gb[6]);
    conv_t(B, H1, W1, 32, 16, g6, Wl[6], du1);
    relu_q(P1 * 32, du1, 0, rb);
    upadd_bwd(B, H1, W1, 32, du1, a.d2, g5, rb);
    conv_w(B, H2, W2, 64, 32, g5, a.u2, gw[5], gb[5]);
    conv_t(B, H2, W2, 64, 32, g5, Wl[5], du2);
    relu_q(P2 * 64, du2, 0, rb);
    upadd_bwd(B, H2, W2, 64, du2, a.b3, g4, rb);
    conv_w(B, H3, W3, 64, 64, g4, a.e3, gw[4], gb[4]);
    conv_t(B, H3, W3, 64, 64, g4, Wl[4], g3);
    for (int64_t i = 0; i < P3 * 64; ++i) g3[i] = a.e3[i] > 0.0 ? q(g3[i], rb) : 0.0;
    conv_w(B, H3, W3, 64, 64, g3, a.p2, gw[3], gb[3]);
    conv_t(B, H3, W3, 64, 64, g3, Wl[3], dp2);
    relu_q(P3 * 64, dp2, 0, rb);
    pool_bwd(B, H2, W2, 64, du2, dp2, a.e2, g2, rb);
    conv_w(B, H2, W2, 32, 64, g2, a.p1, gw[2], gb[2]);
    conv_t(B, H2, W2, 32, 64, g2, Wl[2], dp1);
    relu_q(P2 * 32, dp1, 0, rb);
    pool_bwd(B, H1, W1, 32, du1, dp1, a.e1, g1, rb);
    conv_w(B, H1, W1, 16, 32, g1, a.p0, gw[1], gb[1]);
    conv_t(B, H1, W1, 16, 32, g1, Wl[1], dp0);
    relu_q(P1 * 16, dp0, 0, rb);
    pool_bwd(B, H, W, 16, du0, dp0, a.e0, g0, rb);
    conv_w(B, H, W, 8, 16, g0, a.x0, gw[0], gb[0]);
    free(g8); free(g7); free(du0); free(g6); free(du1); free(g5); free(du2); free(g4);
    free(g3); free(dp2); free(g2); free(dp1); free(g1); free(dp0); free(g0);
  }
  free(dif); free(rho); free(gy); free(s); free(wd);
  acts_free(&a);
  return loss;
}

/* One Adam step on FP32 parameters, as the library's kernel does it:
 * m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2;
 * p -= lr * (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps). */
void skon_adam(int64_t n, float* p, float* m, float* v, const float* g, float lr, float b1, float b2, float eps,
               int64_t t) {
  const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
  for (int64_t i = 0; i < n; ++i) {
    m[i] = b1 * m[i] + (1.0f - b1) * g[i];
    v[i] = b2 * v[i] + (1.0f - b2) * g[i] * g[i];
    const float mh = m[i] / c1, vh = v[i] / c2;
    p[i] -= lr * mh / (sqrtf(vh) + eps);
  }
}
