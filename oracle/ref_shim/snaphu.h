/* Minimal stand-in for the SNAPHU header that the reference cuPHU kernels
 * include.  Only the three items those kernels use are declared; their
 * layouts and values are the ones the reference states in its own source
 * (cuphu_cost.cu:65,189 for the two cost structs, cuphu_incrcost.cu:53,72
 * and cuphu_laplace.cu:62 for LARGESHORT = 32000).  This header is test
 * infrastructure for compiling the reference kernels as a parity oracle;
 * it is never part of the product library. */
#ifndef CUPHU_ORACLE_REF_SHIM_SNAPHU_H
#define CUPHU_ORACLE_REF_SHIM_SNAPHU_H
#include <limits.h>
typedef struct { short offset; short sigsq; } smoothcostT;
typedef struct { short offset; short sigsq; short dzmax; short laycost; } costT;
#define LARGESHORT 32000
#endif
