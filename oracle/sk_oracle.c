/*
 * sk_oracle.c -- instantiates the CPU oracle (sk_oracle_impl.h) for double
 * and float.  TEST INFRASTRUCTURE ONLY; built with -ffp-contract=off so that
 * every multiply and add rounds separately, as in the reference's plain
 * x86-64 build.  See sk_oracle.h for what the oracle is pinned against.
 */
#include "sk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SKO_PI 3.141592653589793238462643383279502884

/* 0: reference order (sequential); 1: chunked order; 2: reversed order
 * (1 and 2: sensitivity studies). */
static int sko_dot_order = 0;
void sko_set_dot_order(int mode) { sko_dot_order = mode; }

/* ------------------------------------------------------------------ */
/* The start vectors of the reference's Lanczos (lanczos.hpp:115-120,  */
/* :211-217): std::mt19937 (Matsumoto and Nishimura 1998) fed through  */
/* std::uniform_real_distribution<T>{-1, 1} as libstdc++ implements it */
/* (generate_canonical: ceil(digits / 32) draws d_k combined as        */
/* sum_k d_k 2^(32k) / 2^(32K) in T, clamped below 1; then a + (b-a)u).  */
/* ------------------------------------------------------------------ */
typedef struct {
  uint32_t mt[624];
  int idx;
} sko_mt19937;

static void sko_mt_seed(sko_mt19937* g, uint32_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 624; ++i)
    g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
  g->idx = 624;
}

static uint32_t sko_mt_next(sko_mt19937* g) {
  if (g->idx >= 624) {
    for (int i = 0; i < 624; ++i) {
      uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
      uint32_t v = g->mt[(i + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908b0dfu;
      g->mt[i] = v;
    }
    g->idx = 0;
  }
  uint32_t y = g->mt[g->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

static double sko_uniform_pm1_f64(sko_mt19937* g) {
  double sum = 0.0, tmp = 1.0;
  for (int k = 0; k < 2; ++k) {
    sum += (double)sko_mt_next(g) * tmp;
    tmp *= 4294967296.0;
  }
  double u = sum / tmp;
  if (u >= 1.0) u = nextafter(1.0, 0.0);
  return u * (1.0 - -1.0) + -1.0;
}

static float sko_uniform_pm1_f32(sko_mt19937* g) {
  float sum = (float)sko_mt_next(g);
  float u = sum / 4294967296.0f;
  if (u >= 1.0f) u = nextafterf(1.0f, 0.0f);
  return u * (1.0f - -1.0f) + -1.0f;
}

#define SKO_T double
#define SKO_SFX f64
#define SKO_SQRT sqrt
#define SKO_COS cos
#define SKO_FABS fabs
#define SKO_UNIFORM sko_uniform_pm1_f64
#include "sk_oracle_impl.h"
#include "sk_oracle_lanczos.h"
#undef SKO_UNIFORM
#undef SKO_T
#undef SKO_SFX
#undef SKO_SQRT
#undef SKO_COS
#undef SKO_FABS

#define SKO_T float
#define SKO_SFX f32
#define SKO_SQRT sqrtf
#define SKO_COS cosf
#define SKO_FABS fabsf
#define SKO_UNIFORM sko_uniform_pm1_f32
#include "sk_oracle_impl.h"
#include "sk_oracle_lanczos.h"
#undef SKO_UNIFORM
#undef SKO_T
#undef SKO_SFX
#undef SKO_SQRT
#undef SKO_COS
#undef SKO_FABS
