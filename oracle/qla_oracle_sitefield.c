/*
 * Test infrastructure (the oracle) -- NOT product code.
 * Fills, copymask, components, gamma multiplication, traces, global
 * reductions of DiracPropagators and global sums in F and D precision; see
 * qla_oracle_sitefield_body.h.
 */
#include "qla_oracle.h"

#define R float
#define SFX f
#include "qla_oracle_sitefield_body.h"
#undef R
#undef SFX

#define R double
#define SFX d
#include "qla_oracle_sitefield_body.h"
#undef R
#undef SFX
