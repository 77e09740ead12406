/* GSL math.h shim -- TEST INFRASTRUCTURE (oracle only): constants only. */
#ifndef ORACLE_SHIM_GSL_MATH_H
#define ORACLE_SHIM_GSL_MATH_H
#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846264338328
#endif
#endif
