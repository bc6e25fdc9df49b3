/* Minimal stand-in for the GSL math header: the reference uses no symbol from it. */
#ifndef TV_ORACLE_GSL_MATH_H
#define TV_ORACLE_GSL_MATH_H
#include <math.h>
#endif
