/* Drop-in include path for C++ code written against the reference's
 * STKFMM/STKFMM.hpp: the same namespace, enums and classes, on this library. */
#ifndef STKFMM_B200_DROPIN_HPP
#define STKFMM_B200_DROPIN_HPP
#include "../stkfmm_b200.hpp"
#endif
