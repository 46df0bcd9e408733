/* CPU restatement of the reference deform-and-render chain -- TEST ORACLE.
 * See hc_oracle.h.  Each stage lives in an .inc file that is compiled once in
 * double (FP64 oracle) and once in float (host-core baseline); the embedded
 * graph forward is also compiled with double outputs for finite differences. */
#include "hc_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define REAL double
#define SFX(x) x##_f64
#define OUTT float
#include "hc_oracle_vec.inc"
#include "hc_oracle_render.inc"
#include "hc_oracle_render_grad.inc"
#include "hc_oracle_eg.inc"
#undef REAL
#undef SFX
#undef OUTT

#define REAL float
#define SFX(x) x##_f32
#define OUTT float
#include "hc_oracle_vec.inc"
#include "hc_oracle_render.inc"
#include "hc_oracle_render_grad.inc"
#include "hc_oracle_eg.inc"
#undef REAL
#undef SFX
#undef OUTT

#define REAL double
#define SFX(x) x##_f64d
#define OUTT double
#define HCO_FORWARD_ONLY
#include "hc_oracle_vec.inc"
#include "hc_oracle_eg.inc"
#undef REAL
#undef SFX
#undef OUTT
#undef HCO_FORWARD_ONLY

/* host kinematics and Pose2EG, float only (the reference computes them in float) */
#include "hc_oracle_fk.inc"
