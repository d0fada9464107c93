/* CPU oracle for the MPDATA transport step -- TEST INFRASTRUCTURE ONLY.
 * Instantiates mpdata_oracle_impl.h in single and double precision.  Built
 * by oracle/Makefile with strict IEEE flags; never linked by the library. */
#include "mpdata_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define R float
#define SFX(name) name##_f32
#define TINY FLT_MIN
#define RMAX fmaxf
#define RMIN fminf
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
