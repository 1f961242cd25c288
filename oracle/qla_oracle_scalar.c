/*
 * Test infrastructure (the oracle) -- NOT product code.
 * QLA_F_ / QLA_D_ real, complex and integer fields; see
 * qla_oracle_scalar_body.h.  The F library calls the float libm functions,
 * the D library the double ones (lib/perl/build_qla.pl:186-355).
 */
#define _GNU_SOURCE
#include <math.h>

#include "qla_oracle.h"

#define R float
#define SFX f
#define MSIN sinf
#define MCOS cosf
#define MTAN tanf
#define MASIN asinf
#define MACOS acosf
#define MATAN atanf
#define MSQRT sqrtf
#define MFABS fabsf
#define MEXP expf
#define MLOG logf
#define MLOG10 log10f
#define MSINH sinhf
#define MCOSH coshf
#define MTANH tanhf
#define MCEIL ceilf
#define MFLOOR floorf
#define MROUND roundf
#define MATAN2 atan2f
#define MSINCOS sincosf
#define MCOPYSIGN copysignf
#include "qla_oracle_scalar_body.h"
#undef R
#undef SFX
#undef MSIN
#undef MCOS
#undef MTAN
#undef MASIN
#undef MACOS
#undef MATAN
#undef MSQRT
#undef MFABS
#undef MEXP
#undef MLOG
#undef MLOG10
#undef MSINH
#undef MCOSH
#undef MTANH
#undef MCEIL
#undef MFLOOR
#undef MROUND
#undef MATAN2
#undef MSINCOS
#undef MCOPYSIGN

#define R double
#define SFX d
#define MSIN sin
#define MCOS cos
#define MTAN tan
#define MASIN asin
#define MACOS acos
#define MATAN atan
#define MSQRT sqrt
#define MFABS fabs
#define MEXP exp
#define MLOG log
#define MLOG10 log10
#define MSINH sinh
#define MCOSH cosh
#define MTANH tanh
#define MCEIL ceil
#define MFLOOR floor
#define MROUND round
#define MATAN2 atan2
#define MSINCOS sincos
#define MCOPYSIGN copysign
#include "qla_oracle_scalar_body.h"
