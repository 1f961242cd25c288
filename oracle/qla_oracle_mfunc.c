/*
 * Test infrastructure (the oracle) -- NOT product code.
 * Matrix functions (exp, sqrt, inverse, det) restated from the reference's
 * code templates, in F and D precision, for any colour count up to 16 (the
 * reference's QLA_F3/D3 and QLA_FN/DN builds of the same templates).
 */
#include <float.h>
#include <math.h>
#include <string.h>
#include "qla_oracle.h"

#define ORA_NCMAX 16

#define R float
#define SFX f
#include "qla_oracle_mfunc_body.h"
#undef R
#undef SFX

#define R double
#define SFX d
#include "qla_oracle_mfunc_body.h"
#undef R
#undef SFX
