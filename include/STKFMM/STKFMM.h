/* Drop-in include path for C code written against the reference's
 * STKFMM/STKFMM.h: the same Stk3DFMM_* and StkWallFMM_* calls, on this library. */
#ifndef STKFMM_B200_DROPIN_H
#define STKFMM_B200_DROPIN_H
#include "../stkfmm_b200.h"
#endif
