/* CPU oracle for the MPDATA transport step -- TEST INFRASTRUCTURE ONLY.
 * Instantiates mpdata_oracle_impl.h in single and double precision and in
 * the reference's INTEGER mode (real = long).  Built by oracle/Makefile with
 * strict IEEE flags; never linked by the library. */
#include "mpdata_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Floating point: ONE 1, HALF 0.5, QUAT 0.25 (core/include/smolar_int.h:12-25). */
#define R_IS_INTEGER 0
#define R_DIV(a, b) ((a) / (b))
#define R_DIV_RESET() ((void)0)
#define R_DIV_FAILED() 0

#define R float
#define SFX(name) name##_f32
#define TINY FLT_MIN
#define RMAX fmaxf
#define RMIN fminf
#define R_ONE ((R)1)
#define R_HALF ((R)0.5)
#define R_QUAT ((R)0.25)
#include "mpdata_oracle_impl.h"
#undef R
#undef SFX
#undef TINY
#undef RMAX
#undef RMIN

#define R double
#define SFX(name) name##_f64
#define TINY DBL_MIN
#define RMAX fmax
#define RMIN fmin
#include "mpdata_oracle_impl.h"
#undef R
#undef SFX
#undef TINY
#undef RMAX
#undef RMIN
#undef R_ONE
#undef R_HALF
#undef R_QUAT
#undef R_IS_INTEGER
#undef R_DIV
#undef R_DIV_RESET
#undef R_DIV_FAILED

/* INTEGER mode (smolar.h:14-16, smolar_int.h:27-31): real = long, ONE 4,
 * HALF 2, QUAT 1, MINVAL 1.  A zero divisor (where the reference's idiv
 * traps) gives 0 and is recorded; oracle_smolar_i64 then returns -2. */
static int g_int_div_zero;

static long oracle_idiv(long a, long b)
{
    if (b == 0) {
        g_int_div_zero = 1;
        return 0;
    }
    return a / b;
}

static long oracle_lmax(long a, long b) { return a > b ? a : b; }
static long oracle_lmin(long a, long b) { return a < b ? a : b; }

#define R_IS_INTEGER 1
#define R_DIV(a, b) oracle_idiv((a), (b))
#define R_DIV_RESET() (g_int_div_zero = 0)
#define R_DIV_FAILED() g_int_div_zero

#define R long
#define SFX(name) name##_i64
#define TINY 1L
#define RMAX oracle_lmax
#define RMIN oracle_lmin
#define R_ONE 4L
#define R_HALF 2L
#define R_QUAT 1L
#include "mpdata_oracle_impl.h"
