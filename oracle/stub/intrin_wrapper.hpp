// Stand-in for the SCTL / PVFMM intrinsics header that STKFMM_common.hpp
// includes; nothing of it is used by the code the oracle compiles.
#pragma once
