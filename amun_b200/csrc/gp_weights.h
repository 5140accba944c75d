// gp_weights.h -- host computation of the Gaussian-process reconstruction
// weights (gp_weights.cpp).
#pragma once

namespace amun {

// prepare_gp (src/interpolations.F90:4438-4557): the ngp weights cgp of the
// one-dimensional Gaussian-process face value for the kernel width sgp,
// computed in quadruple precision and rounded to double.  Returns 0, or 202
// when the covariance matrix cannot be inverted (the reference's iret).
int gp_weights(int ngp, double sgp, double* cgp);

// prepare_mgp (src/interpolations.F90:558-715): the weights of the
// multidimensional Gaussian-process face values over the ngp^ndims stencil
// (Fortran order, i fastest), stored [dir][side][point] (side 0 the
// reference's qi(...,1,dir), the state left of the face i+1/2).  Returns 0,
// or 201 when the covariance matrix cannot be inverted.
int mgp_weights(int ngp, double sgp, int ndims, double* ugp);

}  // namespace amun
