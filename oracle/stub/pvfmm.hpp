// Stand-in for PVFMM's umbrella header, for the CPU oracle only.  The
// reference's Lib/include/STKFMM/stkfmm_helpers.hpp includes <pvfmm.hpp> but
// uses only the standard library (its surface generator, stkfmm::surface);
// this stub supplies those headers so that oracle/_ref can compile it in place
// from the reference tree.  Nothing of PVFMM is restated here.
#pragma once
#include <cmath>
#include <vector>
