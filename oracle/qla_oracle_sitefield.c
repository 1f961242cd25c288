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

void ora_convert_df(double *r, const float *a, long n, int nr, const int *idx_a, const int *gang)
{
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k;
    for (int c = 0; c < nr; c++) r[k * nr + c] = (double)a[ka * nr + c];
  }
}

void ora_convert_fd(float *r, const double *a, long n, int nr, const int *idx_a, const int *gang)
{
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k;
    for (int c = 0; c < nr; c++) r[k * nr + c] = (float)a[ka * nr + c];
  }
}
