/* Declaration of the one GSL sort the reference's sort self-test names. */
#ifndef TV_ORACLE_GSL_HEAPSORT_H
#define TV_ORACLE_GSL_HEAPSORT_H
#include <stddef.h>
int gsl_heapsort_index(size_t *perm, const void *data, size_t n, size_t size,
                       int (*cmp)(const void *, const void *));
#endif
