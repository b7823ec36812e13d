/*
 * Project-written stand-in for <gsl/gsl_randist.h>: the one routine the
 * reference calls (include/random.h:14, rand_gaussian).  A normal deviate
 * with standard deviation sigma, drawn by the Marsaglia polar method (not
 * GSL's ziggurat, so the stream differs from a GSL build; see gsl_rng.h).
 *
 * Both builds use this same generator, so a CPU run and a GPU run from the same seed
 * draw the same momenta and pseudo-fermions.
 */
#ifndef YAHMC_GSL_COMPAT_RANDIST_H
#define YAHMC_GSL_COMPAT_RANDIST_H

#include <math.h>
#include "gsl_rng.h"

static inline double gsl_ran_gaussian_ziggurat(gsl_rng *r, double sigma)
{
	double u, v, s;
	do {
		u = 2.0 * gsl_rng_uniform_pos(r) - 1.0;
		v = 2.0 * gsl_rng_uniform_pos(r) - 1.0;
		s = u * u + v * v;
	} while(s >= 1.0 || s == 0.0);
	return sigma * u * sqrt(-2.0 * log(s) / s);
}

#endif
