/*
 * Project-written stand-in for <gsl/gsl_randist.h>: the one routine the
 * reference calls (include/random.h:14, rand_gaussian).  A normal deviate
 * with standard deviation sigma, drawn by the Marsaglia polar method (not
 * GSL's ziggurat, so the stream differs from a GSL build; see gsl_rng.h).
 *
 * Test infrastructure only: linked into oracle/_ref, never into the product.
 */
#ifndef YAHMC_ORACLE_GSL_RANDIST_H
#define YAHMC_ORACLE_GSL_RANDIST_H

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
