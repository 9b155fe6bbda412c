// setup.h -- host set-up routines of the B200 path (see setup.cpp).
#pragma once

#include "../../include/molsim_gpu.h"

namespace msg {

double erf_molsim(double x);
void spme_factors(int s, int order, double alpha, const double box[3], double *mfac, double *emf, double *vmf);

}  // namespace msg
