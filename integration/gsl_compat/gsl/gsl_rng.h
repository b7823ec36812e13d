/*
 * Project-written stand-in for the two GSL headers the reference includes
 * (include/random.h:4-5).  GSL is not installed on this machine; the builds of the
 * reference here (the oracle's CPU build and the host application built on the engine's
 * shim) compile against this header instead.  A YaHMC installation links the real GSL.  The reference uses GSL for its
 * random-number stream alone (library/random.cpp:20-47, include/random.h:13-16);
 * no test pins that stream, so this header supplies the same API on top of a
 * different generator (xoshiro256** seeded through splitmix64).  Random fields
 * drawn through it are therefore NOT the ones a GSL build would draw; every
 * parity test injects its fields explicitly instead.
 *
 * Both builds use this same generator, so a CPU run and a GPU run from the same seed
 * draw the same momenta and pseudo-fermions.
 */
#ifndef YAHMC_GSL_COMPAT_RNG_H
#define YAHMC_GSL_COMPAT_RNG_H

#include <stdint.h>
#include <stdlib.h>
#include <stddef.h>

typedef struct {
	const char *name;
} gsl_rng_type;

typedef struct {
	const gsl_rng_type *type;
	uint64_t s[4];
} gsl_rng;

static const gsl_rng_type yahmc_gsl_xoshiro_type = {"xoshiro256**"};
static const gsl_rng_type *const gsl_rng_ranlxd1 = &yahmc_gsl_xoshiro_type;

static inline uint64_t yahmc_gsl_splitmix64(uint64_t *x)
{
	uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
	return z ^ (z >> 31);
}

static inline uint64_t yahmc_gsl_rotl(uint64_t x, int k)
{
	return (x << k) | (x >> (64 - k));
}

static inline uint64_t yahmc_gsl_next(gsl_rng *r)
{
	uint64_t *s = r->s;
	uint64_t result = yahmc_gsl_rotl(s[1] * 5, 7) * 9;
	uint64_t t = s[1] << 17;
	s[2] ^= s[0];
	s[3] ^= s[1];
	s[1] ^= s[2];
	s[0] ^= s[3];
	s[2] ^= t;
	s[3] = yahmc_gsl_rotl(s[3], 45);
	return result;
}

static inline void gsl_rng_env_setup(void) {}

static inline void gsl_rng_set(gsl_rng *r, unsigned long seed)
{
	uint64_t x = (uint64_t)seed;
	for(int i = 0; i < 4; i++) r->s[i] = yahmc_gsl_splitmix64(&x);
}

static inline gsl_rng *gsl_rng_alloc(const gsl_rng_type *t)
{
	gsl_rng *r = (gsl_rng*)malloc(sizeof(gsl_rng));
	r->type = t;
	gsl_rng_set(r, 0);
	return r;
}

static inline void gsl_rng_free(gsl_rng *r)
{
	free(r);
}

/* Uniform on the open interval (0,1): 53 random mantissa bits, never 0. */
static inline double gsl_rng_uniform_pos(gsl_rng *r)
{
	double u;
	do {
		u = (double)(yahmc_gsl_next(r) >> 11) * (1.0 / 9007199254740992.0);
	} while(u == 0.0);
	return u;
}

static inline size_t gsl_rng_size(const gsl_rng *r)
{
	(void)r;
	return sizeof(uint64_t) * 4;
}

static inline void *gsl_rng_state(const gsl_rng *r)
{
	return (void*)r->s;
}

#endif
