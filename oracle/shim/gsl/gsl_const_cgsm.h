/*
 * Physical constants in cgs units that the reference's constants.h names.
 * Values are the CODATA / IAU figures. None of them enters the gravity hot
 * path (the gravitational constant is defined by the reference itself).
 */
#ifndef TV_ORACLE_GSL_CONST_CGSM_H
#define TV_ORACLE_GSL_CONST_CGSM_H
#define GSL_CONST_CGSM_PLANCKS_CONSTANT_H (6.62606896e-27)
#define GSL_CONST_CGSM_BOLTZMANN (1.3806504e-16)
#define GSL_CONST_CGSM_ELECTRON_CHARGE (1.602176487e-20)
#define GSL_CONST_CGSM_ELECTRON_VOLT (1.602176487e-12)
#define GSL_CONST_CGSM_MASS_ELECTRON (9.10938188e-28)
#define GSL_CONST_CGSM_MASS_PROTON (1.67262158e-24)
#define GSL_CONST_CGSM_THOMSON_CROSS_SECTION (6.65245893699e-25)
#define GSL_CONST_CGSM_BARN (1e-24)
#define GSL_CONST_CGSM_SOLAR_MASS (1.98892e33)
#endif
