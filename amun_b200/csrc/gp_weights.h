// gp_weights.h -- host computation of the Gaussian-process reconstruction
// weights (gp_weights.cpp).
#pragma once

namespace amun {

// prepare_gp (src/interpolations.F90:4438-4557): the ngp weights cgp of the
// one-dimensional Gaussian-process face value for the kernel width sgp,
// computed in quadruple precision and rounded to double.  Returns 0, or 202
// when the covariance matrix cannot be inverted (the reference's iret).
int gp_weights(int ngp, double sgp, double* cgp);

}  // namespace amun
