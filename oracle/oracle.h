/* oracle.h -- parameter block shared by the C oracle (qb200_oracle.c) and
 * the reference tile driver (ref_driver.cpp).  TEST INFRASTRUCTURE only. */
#ifndef QB200_ORACLE_H
#define QB200_ORACLE_H

#include "../include/qphix_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_WILSON = 0, ORACLE_CLOVER = 1, ORACLE_TM = 2, ORACLE_TMCLOV = 3 };

typedef struct oracle_params {
  double coeff_s, coeff_t_f, coeff_t_b;
  double alpha;
  double mu, muinv;
  double rho;
  unsigned tbc_mask;
  double tbc_phases[4][2];
  unsigned accumulate[8];
} oracle_params;

#ifdef __cplusplus
}
#endif

#endif
