/* Force-included (gcc -include) when compiling the reference's vv.c only.
 *
 * vv_pass (core/src/vv.c:81-82 of the reference) never writes the y-face
 * pseudo-velocity at column i=1 of interior rows, so that column keeps
 * whatever its malloc'd buffer held.  Routing that file's malloc through
 * calloc makes the column deterministic (0 on odd corrective passes, the
 * advective face value on even ones), which is what the default glibc
 * allocator gives for fresh pages.  Test infrastructure only. */
#include <malloc.h>
#include <stdlib.h>
#define malloc(nbytes) calloc(1, (nbytes))
