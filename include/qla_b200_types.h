/*
 * qla_b200_types.h -- QLA site-record types, laid out exactly as QLA 1.9.0
 * defines them, so that arrays built for the reference library can be handed
 * to this one unchanged.
 *
 * The layouts are the ABI contract and must be identical to the reference's:
 *   complex:  include/qla_complex.h:27-40  ({real, imag}; float 8-B aligned,
 *                                           double 16-B aligned)
 *   records:  include/qla_types.h:29-33    (ColorVector V[nc],
 *             HalfFermion H[nc][2], DiracFermion D[nc][4], ColorMatrix M[nc][nc],
 *             DiracPropagator P[nc][4][nc][4]; colour-major, spin inner)
 *
 * When the reference's own qla_types.h / qla_complex.h were included first,
 * their (identical) definitions are used and this file adds nothing.
 */
#ifndef QLA_B200_TYPES_H
#define QLA_B200_TYPES_H

#ifndef _QLA_COMPLEX_H
#define _QLA_COMPLEX_H
typedef int QLA_Int;
typedef float QLA_F_Real;
typedef double QLA_D_Real;

typedef struct {
  QLA_F_Real real;
  QLA_F_Real imag;
} QLA_F_Complex __attribute__((aligned(8)));

typedef struct {
  QLA_D_Real real;
  QLA_D_Real imag;
} QLA_D_Complex __attribute__((aligned(16)));
#endif /* _QLA_COMPLEX_H */

#ifndef _QLA_TYPES_H
#define _QLA_TYPES_H
#define QLA_Ns 4

typedef QLA_F_Complex QLA_F3_ColorVector[3];
typedef QLA_F_Complex QLA_F3_HalfFermion[3][2];
typedef QLA_F_Complex QLA_F3_DiracFermion[3][4];
typedef QLA_F_Complex QLA_F3_ColorMatrix[3][3];
typedef QLA_F_Complex QLA_F3_DiracPropagator[3][4][3][4];

typedef QLA_F_Complex QLA_F2_ColorVector[2];
typedef QLA_F_Complex QLA_F2_HalfFermion[2][2];
typedef QLA_F_Complex QLA_F2_DiracFermion[2][4];
typedef QLA_F_Complex QLA_F2_ColorMatrix[2][2];
typedef QLA_F_Complex QLA_F2_DiracPropagator[2][4][2][4];

typedef QLA_D_Complex QLA_D2_ColorVector[2];
typedef QLA_D_Complex QLA_D2_HalfFermion[2][2];
typedef QLA_D_Complex QLA_D2_DiracFermion[2][4];
typedef QLA_D_Complex QLA_D2_ColorMatrix[2][2];
typedef QLA_D_Complex QLA_D2_DiracPropagator[2][4][2][4];

typedef QLA_D_Complex QLA_D3_ColorVector[3];
typedef QLA_D_Complex QLA_D3_HalfFermion[3][2];
typedef QLA_D_Complex QLA_D3_DiracFermion[3][4];
typedef QLA_D_Complex QLA_D3_ColorMatrix[3][3];
typedef QLA_D_Complex QLA_D3_DiracPropagator[3][4][3][4];
#endif /* _QLA_TYPES_H */

/* per-site random-number generator state (include/qla_random.h:8-14): seven
 * feedback-shift-register words, the congruential multiplier, addend and
 * state, and a float scale; QLA_gaussian's MILC variant keeps its spare
 * deviate in `addend` / `scale` */
#ifndef _QLA_RANDOM_H
#define _QLA_RANDOM_H
typedef struct {
  unsigned int r0, r1, r2, r3, r4, r5, r6;
  unsigned int multiplier, addend, ic_state;
  float scale;
} QLA_RandomState;

#ifdef __cplusplus
extern "C" {
#endif
/* host functions on one state in host memory (lib/random/QLA_random.c,
 * QLA_gaussian.c, QLA_seed_random.c), with the same results */
QLA_F_Real QLA_random(QLA_RandomState *prn_pt);
QLA_F_Real QLA_gaussian(QLA_RandomState *prn_pt);
void QLA_seed_random(QLA_RandomState *prn_pt, int seed, QLA_Int index);
/* non-zero: QLA_gaussian and the gaussian fills use MILC's polar method */
extern int QLA_use_milc_gaussian;
#ifdef __cplusplus
}
#endif
#endif /* _QLA_RANDOM_H */

/* QLA_FN / QLA_DN take the colour count at run time (include/qla_types.h:193-239,
 * C99 variable-length types); their arrays are passed as untyped pointers to
 * records of nc*nc (matrix) or nc (vector) complex numbers. */

#endif /* QLA_B200_TYPES_H */
