/*
 * ORACLE / TEST INFRASTRUCTURE - never part of the product.
 * CPU restatement of the reference P-SV scheme, built in float (_f, the
 * reference's own rounding) and double (_d, the FP64 oracle).
 */
#include "psv_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OR_CAT2(a, b) a##b
#define OR_CAT(a, b) OR_CAT2(a, b)

#define REAL float
#define SFX _f
#include "psv_oracle_impl.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX _d
#include "psv_oracle_impl.h"
#undef REAL
#undef SFX
