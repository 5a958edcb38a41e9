// stk_kernel_table.hpp -- STKFMM KERNEL enum -> dimensions, names and the
// micro-kernel that fills each PVFMM kernel slot.
//
// Compositions follow the reference's BuildKernel calls (slot order s2m, s2l,
// s2t, m2m, m2l, m2t, l2t; NULL means "the kernel itself"):
//   LapPGrad      LaplaceLayerKernel.hpp:314-326
//   Stokes        StokesLayerKernel.hpp:39-42   (all slots stokes_vel)
//   RPY           RPYKernel.hpp:137-154
//   StokesRegVel  StokesRegSingleLayerKernel.hpp:211-218
//   PVel          StokesLayerKernel.hpp:45-50   (all slots stokes_pvel / stokes_doublepvel)
// Dimensions follow getKernelDimension (Lib/src/STKFMM.cpp:33-40).  For kernels
// without a double layer the reference returns PVFMM's default surf_dim, which
// is the coordinate dimension plus ker_dim[0] (PVFMM's Kernel constructor, not
// vendored); the same rule is used here.
#pragma once
#include "stk_ukernels.cuh"

namespace stk {

enum Slot : int {
    SLOT_S2T_SL = 0,
    SLOT_S2T_DL = 1,
    SLOT_S2M_SL = 2,
    SLOT_S2M_DL = 3,
    SLOT_M2X = 4,  // m2m, m2l, l2l
    SLOT_M2T = 5,
    SLOT_L2T = 6,
    SLOT_S2L_SL = 7,
    SLOT_S2L_DL = 8,
    SLOT_COUNT = 9
};

struct KernelInfo {
    unsigned id;
    const char *name;  // PVFMM ker_name of the top-level kernel
    int kdim_sl, kdim_dl, kdim_trg;
    int slot[SLOT_COUNT];
    // exponent k of the target rescaling trg *= sF^k per target component
    // (FMMData::scaleTrg, Lib/src/FMMData.cpp:319-470)
    int trg_scale_pow[16];
    // number of trailing SL components that scale like a double layer: 1 for the
    // trace / radius / regularisation of PVel-type, RPY and StokesRegVel, 4 for the
    // torque and regularisation of StokesRegVelOmega (FMMData.cpp:300-316)
    int sl_last_scales;
};

static const KernelInfo kKernels[] = {
    {1, "laplace_PGrad", 1, 3, 4,
     {UK_LAPLACE_PGRAD, UK_LAPLACE_DIPOLEPGRAD, UK_LAPLACE_P, UK_LAPLACE_DIPOLEP, UK_LAPLACE_P, UK_LAPLACE_PGRAD,
      UK_LAPLACE_PGRAD, UK_LAPLACE_P, UK_LAPLACE_DIPOLEP},
     {1, 2, 2, 2}, 0},
    // LaplaceLayerKernel<T>::PGradGrad (Lib/include/STKFMM/LaplaceLayerKernel.hpp:328-341)
    {2, "laplace_PGradGrad", 1, 3, 10,
     {UK_LAPLACE_PGRADGRAD, UK_LAPLACE_DIPOLEPGRADGRAD, UK_LAPLACE_P, UK_LAPLACE_DIPOLEP, UK_LAPLACE_P,
      UK_LAPLACE_PGRADGRAD, UK_LAPLACE_PGRADGRAD, UK_LAPLACE_P, UK_LAPLACE_DIPOLEP},
     {1, 2, 2, 2, 3, 3, 3, 3, 3, 3}, 0},
    // LaplaceLayerKernel<T>::QPGradGrad (LaplaceLayerKernel.hpp:343-356): no double layer;
    // quadrupole sources for S2T / S2M / S2L, laplace_pgradgrad for M2T / L2T
    {4, "laplace_QPGradGrad", 9, 12, 10,
     {UK_LAPLACE_QUADPGRADGRAD, -1, UK_LAPLACE_QUADP, -1, UK_LAPLACE_P, UK_LAPLACE_PGRADGRAD, UK_LAPLACE_PGRADGRAD,
      UK_LAPLACE_QUADP, -1},
     {3, 4, 4, 4, 5, 5, 5, 5, 5, 5}, 0},
    {8, "stokes_vel", 3, 6, 3,
     {UK_STOKES_VEL, -1, UK_STOKES_VEL, -1, UK_STOKES_VEL, UK_STOKES_VEL, UK_STOKES_VEL, UK_STOKES_VEL, -1},
     {1, 1, 1}, 0},
    {16, "rpy_ulapu", 4, 7, 6,
     {UK_RPY_ULAPU, -1, UK_RPY_U, -1, UK_STOKES_VEL, UK_STK_ULAPU, UK_STK_ULAPU, UK_RPY_U, -1},
     {1, 1, 1, 3, 3, 3}, 1},
    {32, "stokes_regvel", 4, 7, 3,
     {UK_STOKES_REGVEL, -1, UK_STOKES_REGVEL, -1, UK_STOKES_VEL, UK_STOKES_VEL, UK_STOKES_VEL, UK_STOKES_REGVEL, -1},
     {1, 1, 1}, 1},
    // StokesRegKernel<T>::FTVelOmega (StokesRegSingleLayerKernel.hpp:220-232): regularized
    // force + torque at S2T / S2M / S2L, stokes_vel translations, stokes_velomega at M2T / L2T
    {64, "stokes_regftvelomega", 7, 10, 6,
     {UK_STOKES_REGFTVELOMEGA, -1, UK_STOKES_REGFTVEL, -1, UK_STOKES_VEL, UK_STOKES_VELOMEGA, UK_STOKES_VELOMEGA,
      UK_STOKES_REGFTVEL, -1},
     {1, 1, 1, 2, 2, 2}, 4},
    {128, "stokes_PVel", 4, 9, 4,
     {UK_STOKES_PVEL, UK_STOKES_DOUBLEPVEL, UK_STOKES_PVEL, UK_STOKES_DOUBLEPVEL, UK_STOKES_PVEL, UK_STOKES_PVEL,
      UK_STOKES_PVEL, UK_STOKES_PVEL, UK_STOKES_DOUBLEPVEL},
     {2, 1, 1, 1}, 1},
    // StokesLayerKernel<T>::PVelGrad / PVelLaplacian / Traction (StokesLayerKernel.hpp:52-94):
    // stokes_PVel translations and check potentials, the derivative kernel for S2T, M2T, L2T
    {256, "stokes_PVelGrad", 4, 9, 16,
     {UK_STOKES_PVELGRAD, UK_STOKES_DOUBLEPVELGRAD, UK_STOKES_PVEL, UK_STOKES_DOUBLEPVEL, UK_STOKES_PVEL,
      UK_STOKES_PVELGRAD, UK_STOKES_PVELGRAD, UK_STOKES_PVEL, UK_STOKES_DOUBLEPVEL},
     {2, 1, 1, 1, 3, 3, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2}, 1},
    {512, "stokes_PVelLaplacian", 4, 9, 7,
     {UK_STOKES_PVELLAPLACIAN, UK_STOKES_DOUBLELAPLACIAN, UK_STOKES_PVEL, UK_STOKES_DOUBLEPVEL, UK_STOKES_PVEL,
      UK_STOKES_PVELLAPLACIAN, UK_STOKES_PVELLAPLACIAN, UK_STOKES_PVEL, UK_STOKES_DOUBLEPVEL},
     {2, 1, 1, 1, 3, 3, 3}, 1},
    {1024, "stokes_Traction", 4, 9, 9,
     {UK_STOKES_TRACTION, UK_STOKES_DOUBLETRACTION, UK_STOKES_PVEL, UK_STOKES_DOUBLEPVEL, UK_STOKES_PVEL,
      UK_STOKES_TRACTION, UK_STOKES_TRACTION, UK_STOKES_PVEL, UK_STOKES_DOUBLEPVEL},
     {2, 2, 2, 2, 2, 2, 2, 2, 2}, 1},
};
constexpr int kNumKernels = sizeof(kKernels) / sizeof(kKernels[0]);

inline const KernelInfo *find_kernel(unsigned id) {
    for (int i = 0; i < kNumKernels; i++)
        if (kKernels[i].id == id) return &kKernels[i];
    return nullptr;
}

// A kernel is evaluated by this library when its S2T single-layer slot is filled.
inline bool kernel_supported(const KernelInfo *k) { return k && k->slot[SLOT_S2T_SL] >= 0; }

}  // namespace stk
