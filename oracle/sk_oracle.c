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

/* 0: reference order (sequential); 1: chunked order (sensitivity studies). */
static int sko_dot_order = 0;
void sko_set_dot_order(int mode) { sko_dot_order = mode; }

#define SKO_T double
#define SKO_SFX f64
#define SKO_SQRT sqrt
#define SKO_COS cos
#define SKO_FABS fabs
#include "sk_oracle_impl.h"
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
#include "sk_oracle_impl.h"
#undef SKO_T
#undef SKO_SFX
#undef SKO_SQRT
#undef SKO_COS
#undef SKO_FABS
