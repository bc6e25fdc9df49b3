/* Dimensionless constant used by the reference's constants.h (CODATA value). */
#ifndef TV_ORACLE_GSL_CONST_NUM_H
#define TV_ORACLE_GSL_CONST_NUM_H
#define GSL_CONST_NUM_FINE_STRUCTURE (7.2973525698e-3)
#endif
