/*
 * rng.h -- random number generator of the CJMultiSlice class interface.
 *
 * Replaces the reference's CRng (src/rng.h:30-65, src/rng.cpp:30-89), which
 * CJMultiSlice::SetRng / GetRng exchange and from which the frozen-phonon
 * variant draws and the plasmon Monte-Carlo take their numbers.  The draw
 * formulas are the reference's, so the same seed gives the same variant
 * sequences: a std::mt19937 engine, integers uniform on [0, RAND_MAXROLL]
 * (std::uniform_int_distribution), unirand = rmin + k / RAND_MAXROLL *
 * (rmax - rmin), normal numbers from std::normal_distribution<double> and
 * Poisson numbers from a std::poisson_distribution<int> made per call.
 * Seed 0 means a seed from the clock.  Implemented in libjms_b200.so.
 */
#ifndef JMS_B200_RNG_H
#define JMS_B200_RNG_H

#include <random>

#ifndef RAND_MAXROLL
#define RAND_MAXROLL 0x7FFFFFFF
#endif

class CRng {
public:
	CRng();                 /* seeded from the clock */
	explicit CRng(int seed);
	~CRng();

	/* re-seeds the engine (0: from the clock) */
	void seed(int seed = 0);
	/* the seed last used */
	int get_seed(void);
	/* uniform integer in [0, RAND_MAXROLL] */
	int rand();
	/* uniform number in the closed range [rmin, rmax] */
	double unirand(double rmin = 0.0, double rmax = 1.0);
	/* uniform number in the half-open range [rmin, rmax) */
	double unirand_oub(double rmin = 0.0, double rmax = 1.0);
	/* normal number of mean mu and standard deviation sdev */
	double normrand(double mu = 0.0, double sdev = 1.0);
	/* Poisson number of mean mu */
	int poisrand(double mu = 1.0);

private:
	std::mt19937 urng;
	std::uniform_int_distribution<int> uni_dist;
	std::normal_distribution<double> norm_dist;
	int m_seed;
};

#endif /* JMS_B200_RNG_H */
