/*
 * Test infrastructure (the oracle) -- NOT product code.
 * Element-wise families, site-local dot products and the ColorVector outer
 * product in F and D precision; see qla_oracle_ewise_body.h.
 */
#include "qla_oracle.h"

#define R float
#define SFX f
#include "qla_oracle_ewise_body.h"
#undef R
#undef SFX

#define R double
#define SFX d
#include "qla_oracle_ewise_body.h"
#undef R
#undef SFX
