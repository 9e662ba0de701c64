/* Part of the GSL-subset shim used only to build the parity oracle. */
#ifndef PAWAN_SHIM_GSL_SPLINE_H
#define PAWAN_SHIM_GSL_SPLINE_H
#include "pawan_gsl_shim.h"
#endif
