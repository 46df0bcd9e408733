/* CPU restatement of the reference deform-and-render chain -- TEST ORACLE.
 * See hc_oracle.h.  Each stage lives in an .inc file that is compiled once in
 * double (FP64 oracle) and once in float (host-core baseline). */
#include "hc_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define REAL double
#define SFX(x) x##_f64
#include "hc_oracle_render.inc"
#undef REAL
#undef SFX

#define REAL float
#define SFX(x) x##_f32
#include "hc_oracle_render.inc"
#undef REAL
#undef SFX
