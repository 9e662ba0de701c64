/* Part of the GSL-subset shim used only to build the parity oracle. */
#ifndef PAWAN_SHIM_GSL_INTERP_H
#define PAWAN_SHIM_GSL_INTERP_H
#include "pawan_gsl_shim.h"
#endif
