/* Test infrastructure (oracle): instantiates the substep restatement (oracle_sim.h) in
 * FP32 and FP64.  See oracle.h for what is restated and which reference files it follows. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "oracle_internal.h"

#define R float
#define SFX _f32
#define R_LOG logf
#define R_EXP expf
#define R_SQRT oracle_ref_sqrtf
#define R_STDSQRT sqrtf
#define R_FLOOR floorf
#define R_ABS fabsf
#define OR_SVD oracle_svd_f32
#include "oracle_sim.h"
#undef R
#undef SFX
#undef R_LOG
#undef R_EXP
#undef R_SQRT
#undef R_STDSQRT
#undef R_FLOOR
#undef R_ABS
#undef OR_SVD

#define R double
#define SFX _f64
#define R_LOG log
#define R_EXP exp
#define R_SQRT sqrt
#define R_STDSQRT sqrt
#define R_FLOOR floor
#define R_ABS fabs
#define OR_SVD oracle_svd_f64
#include "oracle_sim.h"
