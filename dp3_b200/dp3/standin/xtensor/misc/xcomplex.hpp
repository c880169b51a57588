// Stand-in for xtensor's complex helpers header: DP3's AntennaConstraint
// includes it, and the eager stand-in tensors already handle complex values.
#ifndef DP3B200_STANDIN_XTENSOR_MISC_XCOMPLEX_HPP
#define DP3B200_STANDIN_XTENSOR_MISC_XCOMPLEX_HPP
#include "../containers/xtensor.hpp"
#endif
