/* GSL errno.h shim -- TEST INFRASTRUCTURE (oracle only). */
#ifndef ORACLE_SHIM_GSL_ERRNO_H
#define ORACLE_SHIM_GSL_ERRNO_H
#define GSL_SUCCESS 0
#define GSL_EMAXITER 11
#endif
