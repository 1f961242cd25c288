/*
 * Test infrastructure (the oracle) -- NOT product code.
 * Matrix functions (exp, expA, expTA, log, sqrt, invsqrt, sqrtPH, invsqrtPH,
 * inverse, det, eigenvalues, M^-1 V and M^-1 M) restated from the reference's
 * code templates, in F and D precision, for any colour count up to 16 (the
 * reference's QLA_F3/D3 and QLA_FN/DN builds of the same templates).  The
 * libm calls of the F build are the float ones (sqrtf, acosf, cbrtf,
 * sincosf, atan2f, copysignf, sinhf, expf), as in the templates' QLA_Precision == 'F'
 * branch and lib/cmath.
 */
#define _GNU_SOURCE
#include <float.h>
#include <math.h>
#include <string.h>
#include "qla_oracle.h"

#define ORA_NCMAX 16

#define R float
#define SFX f
#define M_SQRT sqrtf
#define M_FABS fabsf
#define M_ACOS acosf
#define M_CBRT cbrtf
#define M_SINCOS sincosf
#define M_ATAN2 atan2f
#define M_COPYSIGN copysignf
#define M_SINH sinhf
#define M_EXP expf
#include "qla_oracle_mfunc_body.h"
#undef R
#undef SFX
#undef M_SQRT
#undef M_FABS
#undef M_ACOS
#undef M_CBRT
#undef M_SINCOS
#undef M_ATAN2
#undef M_COPYSIGN
#undef M_SINH
#undef M_EXP

#define R double
#define SFX d
#define M_SQRT sqrt
#define M_FABS fabs
#define M_ACOS acos
#define M_CBRT cbrt
#define M_SINCOS sincos
#define M_ATAN2 atan2
#define M_COPYSIGN copysign
#define M_SINH sinh
#define M_EXP exp
#include "qla_oracle_mfunc_body.h"
#undef R
#undef SFX
