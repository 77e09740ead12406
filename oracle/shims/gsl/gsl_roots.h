/* GSL roots.h shim -- TEST INFRASTRUCTURE (oracle only).  cola.c includes this
 * header but calls no root finder (cola.c:49). */
#ifndef ORACLE_SHIM_GSL_ROOTS_H
#define ORACLE_SHIM_GSL_ROOTS_H
#endif
