/*
 * TEST INFRASTRUCTURE ONLY.  CPU oracle for the TM2D time-stepping path;
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * it, as the checker.  The product path never calls into this library.
 *
 * Exported symbols: tide_oracle_tm_{forward,forward_with_storage,backward,
 *   born_forward}_
 * {float,double}.  Their arguments mirror the reference native ABI
 * (src/tide/backend_utils.py:256-308) minus the storage-mode, stream, file
 * and Debye arguments, with the stencil order as the first argument.
 * Debye media: tide_oracle_tm_debye_{forward_with_storage,backward}_
 * {float,double}, taking the TideTMDebye argument struct of
 * include/tide_b200_debye.h with host pointers.
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "tide_b200_debye.h"

/* Gradient shot-reduction order of the backward, see tm2d_oracle_impl.h. */
static int g_oracle_grad_order = 0;
void tide_oracle_set_grad_order(int order) { g_oracle_grad_order = order; }

#define REAL float
#define SFX float
#include "tm2d_oracle_impl.h"
#include "tm2d_debye_oracle_impl.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX double
#include "tm2d_oracle_impl.h"
#include "tm2d_debye_oracle_impl.h"
#undef REAL
#undef SFX

const char *tide_oracle_version(void) { return "tm2d-oracle-1"; }
