/*
 * TEST INFRASTRUCTURE ONLY.  CPU oracle for the 3-D Maxwell (Yee) path; only
 * tests/ loads it, as the checker.  The product path never calls into it.
 *
 * Exported symbols: tide_oracle_em3d_{forward,backward}_{float,double}
 * (arguments documented in em3d_oracle_impl.h).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Stencil order of every following call (2, 4, 6 or 8). */
static int g_em3d_stencil = 2;
void tide_oracle_em3d_set_stencil(int st) {
  g_em3d_stencil = (st == 4 || st == 6 || st == 8) ? st : 2;
}

#define REAL float
#define SFX float
#include "em3d_oracle_impl.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX double
#include "em3d_oracle_impl.h"
#undef REAL
#undef SFX
