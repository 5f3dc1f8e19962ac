/* Stand-in for GSL's Bessel header: only the kaiser_bessel inserters call it,
 * and those are never exercised by the oracle pin.  TEST INFRASTRUCTURE ONLY. */
#ifndef FR_REFSHIM_GSL_BESSEL_H
#define FR_REFSHIM_GSL_BESSEL_H
#include <cstdlib>
inline double gsl_sf_bessel_i0_scaled(double) { std::abort(); }
#endif
