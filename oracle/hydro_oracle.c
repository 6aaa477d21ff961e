/*
 * Oracle (test infrastructure only; nothing in the product links it).
 * CPU restatement of the reference's finite-volume path in plain C, compiled
 * with -ffp-contract=off, in both of the reference's precisions:
 *   *_f64  DATATYPE = double (hydro2d/kernel.hpp:24-37)
 *   *_f32  DATATYPE = float under USE_FLOAT (hydro2d/kernel.hpp:9-22)
 * The arithmetic lives in hydro_oracle_impl.h, which cites the reference line for
 * every function. Parity is pinned against the reference's own kernel.cxx compiled
 * unchanged (oracle/_ref/libref*.so, see oracle/Makefile) and against the numbers
 * printed in the reference's hardware run logs (tests/golden/).
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#define T double
#define SUF _f64
#define TSQRT sqrt
#define L(x) x
#include "hydro_oracle_impl.h"
#undef T
#undef SUF
#undef TSQRT
#undef L

#define T float
#define SUF _f32
#define TSQRT sqrtf
#define L(x) x##f
#include "hydro_oracle_impl.h"
#undef T
#undef SUF
#undef TSQRT
#undef L
