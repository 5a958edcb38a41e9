/* stkfmm_b200.hpp -- C++ interface of the B200 STKFMM library.
 *
 * Mirrors the reference's C++ API (Lib/include/STKFMM/STKFMM.hpp and
 * STKFMM_common.hpp): namespace stkfmm; the enums PAXIS, PPKERNEL and KERNEL
 * with their values; asInteger, getKernelDimension and getKernelName; and the
 * classes Stk3DFMM and StkWallFMM with the same constructors and defaults, the
 * same methods, argument order and accumulate semantics.  Code written against
 * the reference builds against this header (or against include/STKFMM/STKFMM.hpp,
 * which includes it) and links libstkfmm_b200.so.
 *
 * Header only: every call goes through the C ABI of stkfmm_b200.h, which this
 * header declares inside namespace stkfmm::capi (every C call, constant and
 * handle type is there, e.g. stkfmm::capi::Stk3DFMM_evaluate_fmm_device).  A
 * translation unit includes either this header or stkfmm_b200.h, not both: the
 * handle types of the two would differ.
 *
 * Error behaviour: where the reference prints a message and calls exit(1) (size,
 * kernel and state errors, FMMData.cpp:184-195, STKFMM.cpp:53-55, 91-94), this
 * interface throws stkfmm::Error, which carries the C ABI's status code.
 *
 * Additions with no reference counterpart: setPrecision (FP64 or mixed P2P), and
 * the status codes of Error.
 */
#ifndef STKFMM_B200_HPP
#define STKFMM_B200_HPP

#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <utility>

/* The C ABI, declared inside stkfmm::capi so that no global Stk3DFMM or
 * StkWallFMM type is introduced (reference code writes, for instance,
 * `using Stk3DFMM = stkfmm::Stk3DFMM;` at global scope). */
namespace stkfmm {
namespace capi {
#define STKFMM_B200_IN_NAMESPACE
#include "stkfmm_b200.h"
#undef STKFMM_B200_IN_NAMESPACE
}  // namespace capi
}  // namespace stkfmm

namespace stkfmm {

/* periodic boundary condition (STKFMM_common.hpp:29-34) */
enum class PAXIS : unsigned { NONE = 0, PX = 1, PXY = 2, PXYZ = 3 };

/* sub-kernel of evaluateKernel (STKFMM_common.hpp:40-44) */
enum class PPKERNEL : unsigned { SLS2T = 1, DLS2T = 2, L2T = 4 };

/* kernels (STKFMM_common.hpp:46-62); LapGrad is the reference's internal test
 * kernel, outside its kernel map, and is refused here as there */
enum class KERNEL : unsigned {
    LapPGrad = 1,
    LapPGradGrad = 2,
    LapQPGradGrad = 4,
    Stokes = 8,
    RPY = 16,
    StokesRegVel = 32,
    StokesRegVelOmega = 64,
    PVel = 128,
    PVelGrad = 256,
    PVelLaplacian = 512,
    Traction = 1024,
    LapGrad = 2048
};

/* enum to its integer value (STKFMM_common.hpp:100-104) */
template <typename Enumeration>
auto asInteger(Enumeration const value) -> typename std::underlying_type<Enumeration>::type {
    return static_cast<typename std::underlying_type<Enumeration>::type>(value);
}

/* A failed call: what() names the call and the status; status() is the C ABI code. */
class Error : public std::runtime_error {
  public:
    Error(int status, const std::string &call)
        : std::runtime_error(call + ": " + capi::stk_status_string(status)), status_(status) {}
    int status() const { return status_; }

  private:
    int status_;
};

namespace detail {
inline void check(int status, const char *call) {
    if (status != capi::STK_OK) throw Error(status, call);
}
}  // namespace detail

/* (kdimSL, kdimDL, kdimTrg) (STKFMM.cpp:33-40) */
inline std::tuple<int, int, int> getKernelDimension(KERNEL kernel) {
    int d[3] = {0, 0, 0};
    detail::check(capi::stk_get_kernel_dimension(asInteger(kernel), d), "getKernelDimension");
    return std::make_tuple(d[0], d[1], d[2]);
}

/* PVFMM ker_name of the kernel (STKFMM.cpp:42-46) */
inline std::string getKernelName(KERNEL kernel) {
    const char *name = capi::stk_get_kernel_name(asInteger(kernel));
    if (!name) throw Error(capi::STK_ERR_KERNEL, "getKernelName");
    return name;
}

/* What kernelMap maps to: the fields of pvfmm::Kernel<double> that callers
 * of the reference read (ker_name, ker_dim, surf_dim). */
struct KernelDescriptor {
    std::string ker_name;
    int ker_dim[2];
    int surf_dim;
};

namespace detail {
inline const std::unordered_map<KERNEL, const KernelDescriptor *> &kernel_map() {
    static const KERNEL all[11] = {KERNEL::LapPGrad,     KERNEL::LapPGradGrad,      KERNEL::LapQPGradGrad,
                                   KERNEL::Stokes,       KERNEL::RPY,               KERNEL::StokesRegVel,
                                   KERNEL::StokesRegVelOmega, KERNEL::PVel,         KERNEL::PVelGrad,
                                   KERNEL::PVelLaplacian, KERNEL::Traction};
    static KernelDescriptor desc[11];
    static const std::unordered_map<KERNEL, const KernelDescriptor *> map = [] {
        std::unordered_map<KERNEL, const KernelDescriptor *> m;
        for (int i = 0; i < 11; i++) {
            int d[3] = {0, 0, 0};
            check(capi::stk_get_kernel_dimension(asInteger(all[i]), d), "kernelMap");
            desc[i].ker_name = getKernelName(all[i]);
            desc[i].ker_dim[0] = d[0];
            desc[i].ker_dim[1] = d[2];
            desc[i].surf_dim = d[1];
            m[all[i]] = &desc[i];
        }
        return m;
    }();
    return map;
}
}  // namespace detail

/* every kernel of the reference's map (STKFMM.cpp:18-31), iterable as there */
static const std::unordered_map<KERNEL, const KernelDescriptor *> &kernelMap = detail::kernel_map();

/* The common part of both FMMs (STKFMM.hpp:30-177). */
class STKFMM {
  public:
    STKFMM(int multOrder_, int maxPts_, PAXIS pbc_, unsigned int kernelComb_, bool enableFF_ = true)
        : multOrder(multOrder_), maxPts(maxPts_), pbc(pbc_), kernelComb(kernelComb_), enableFF(enableFF_) {}
    virtual ~STKFMM() {}
    /* one owner per handle: movable (so that `auto fmm = Stk3DFMM(...)` builds
     * under C++14, as the reference's Demo/Demo.cpp:25 writes it), not copyable */
    STKFMM(const STKFMM &) = delete;
    STKFMM &operator=(const STKFMM &) = delete;
    STKFMM(STKFMM &&) = default;

    /* a cubic box [origin, origin + len)^3 (half-cubic for the wall) */
    void setBox(double origin_[3], double len_) {
        setBoxImpl(origin_, len_);
        origin[0] = origin_[0];
        origin[1] = origin_[1];
        origin[2] = origin_[2];
        len = len_;
    }

    virtual void setPoints(const int nSL, const double *srcSLCoordPtr, const int nTrg, const double *trgCoordPtr,
                           const int nDL = 0, const double *srcDLCoordPtr = nullptr) = 0;
    virtual void setupTree(KERNEL kernel) = 0;
    /* trgValuePtr += FMM(sources) */
    virtual void evaluateFMM(const KERNEL kernel, const int nSL, const double *srcSLValuePtr, const int nTrg,
                             double *trgValuePtr, const int nDL = 0, const double *srcDLValuePtr = nullptr) = 0;
    virtual void clearFMM(KERNEL kernel) = 0;

    /* trgValuePtr += direct sum of one sub-kernel over all pairs, raw coordinates
     * (STKFMM.cpp:88-99; FMMData.cpp:252-283).  The kernel must be one of this
     * FMM's; nThreads is accepted and unused (the sum runs on the GPU). */
    void evaluateKernel(const KERNEL kernel, const int nThreads, const PPKERNEL p2p, const int nSrc,
                        double *srcCoordPtr, double *srcValuePtr, const int nTrg, double *trgCoordPtr,
                        double *trgValuePtr) {
        (void)nThreads;
        if (!hasKernel(kernel)) throw Error(capi::STK_ERR_KERNEL, "evaluateKernel");
        detail::check(capi::stk_evaluate_kernel(asInteger(kernel), asInteger(p2p), nSrc, srcCoordPtr, srcValuePtr, nTrg,
                                          trgCoordPtr, trgValuePtr, precision),
                      "evaluateKernel");
    }

    /* [xlow, xhigh, ylow, yhigh, zlow, zhigh] */
    std::tuple<double, double, double, double, double, double> getBox() const {
        return std::make_tuple(origin[0], origin[0] + len, origin[1], origin[1] + len, origin[2], origin[2] + len);
    }

    virtual void showActiveKernels() const = 0;
    bool isKernelActive(KERNEL kernel_) const { return asInteger(kernel_) & kernelComb; }
    int getMultOrder() const { return multOrder; }

    /* STK_FP64 (default) or STK_MIXED for the P2P kernels */
    virtual void setPrecision(int precision_) = 0;

  protected:
    const int multOrder;
    const int maxPts;
    PAXIS pbc;
    const unsigned kernelComb;
    const bool enableFF;
    int precision = capi::STK_FP64;
    double origin[3] = {0.0, 0.0, 0.0};
    double len = 1.0;

    virtual void setBoxImpl(double origin_[3], double len_) = 0;
    /* the kernels evaluateKernel accepts: those with an FMM in this object */
    virtual bool hasKernel(KERNEL kernel) const = 0;
};

/* FMM in free space or a periodic box (STKFMM.hpp:183-215, Stk3DFMM.cpp). */
class Stk3DFMM : public STKFMM {
  public:
    Stk3DFMM(int multOrder = 10, int maxPts = 2000, PAXIS pbc_ = PAXIS::NONE,
             unsigned int kernelComb_ = asInteger(KERNEL::Stokes) | asInteger(KERNEL::RPY), bool enableFF_ = true)
        : STKFMM(multOrder, maxPts, pbc_, kernelComb_, enableFF_) {
        h = capi::Stk3DFMM_create(multOrder, maxPts, (int)asInteger(pbc_), kernelComb_);
        if (!h) throw Error(capi::stk_device_count() > 0 ? capi::STK_ERR_INVALID_ARG : capi::STK_ERR_NO_DEVICE, "Stk3DFMM");
        if (!enableFF_) {
            const int rc = capi::Stk3DFMM_set_far_field(h, 0);
            if (rc) {
                capi::Stk3DFMM_destroy(h);
                throw Error(rc, "Stk3DFMM");
            }
        }
    }
    Stk3DFMM(Stk3DFMM &&o) noexcept : STKFMM(std::move(o)), h(o.h) { o.h = nullptr; }
    ~Stk3DFMM() { capi::Stk3DFMM_destroy(h); }

    void setPoints(const int nSL, const double *srcSLCoordPtr, const int nTrg, const double *trgCoordPtr,
                   const int nDL = 0, const double *srcDLCoordPtr = nullptr) override {
        detail::check(capi::Stk3DFMM_set_points(h, nSL, const_cast<double *>(srcSLCoordPtr), nTrg,
                                          const_cast<double *>(trgCoordPtr), nDL, const_cast<double *>(srcDLCoordPtr)),
                      "setPoints");
    }
    void setupTree(KERNEL kernel) override { detail::check(capi::Stk3DFMM_setup_tree(h, asInteger(kernel)), "setupTree"); }
    void evaluateFMM(const KERNEL kernel, const int nSL, const double *srcSLValuePtr, const int nTrg,
                     double *trgValuePtr, const int nDL = 0, const double *srcDLValuePtr = nullptr) override {
        detail::check(capi::Stk3DFMM_evaluate_fmm(h, asInteger(kernel), nSL, const_cast<double *>(srcSLValuePtr), nTrg,
                                            trgValuePtr, nDL, const_cast<double *>(srcDLValuePtr)),
                      "evaluateFMM");
    }
    void clearFMM(KERNEL kernel) override { detail::check(capi::Stk3DFMM_clear_fmm(h, asInteger(kernel)), "clearFMM"); }
    void showActiveKernels() const override { detail::check(capi::Stk3DFMM_show_active_kernels(h), "showActiveKernels"); }
    void setPrecision(int precision_) override {
        detail::check(capi::Stk3DFMM_set_precision(h, precision_), "setPrecision");
        precision = precision_;
    }

    /* the C handle, for the C ABI's further calls (device buffers, phases, shards) */
    capi::Stk3DFMM *handle() const { return h; }

  protected:
    void setBoxImpl(double origin_[3], double len_) override {
        detail::check(capi::Stk3DFMM_set_box(h, origin_, len_), "setBox");
    }
    bool hasKernel(KERNEL kernel) const override { return isKernelActive(kernel); }

  private:
    capi::Stk3DFMM *h = nullptr;
};

/* FMM above a no-slip wall, Stokes and RPY (STKFMM.hpp:221-271, StkWallFMM.cpp). */
class StkWallFMM : public STKFMM {
  public:
    StkWallFMM(int multOrder = 10, int maxPts = 2000, PAXIS pbc_ = PAXIS::NONE,
               unsigned int kernelComb_ = asInteger(KERNEL::Stokes) | asInteger(KERNEL::RPY), bool enableFF_ = true)
        : STKFMM(multOrder, maxPts, pbc_, kernelComb_, enableFF_) {
        h = capi::StkWallFMM_create(multOrder, maxPts, (int)asInteger(pbc_), kernelComb_);
        if (!h) throw Error(capi::stk_device_count() > 0 ? capi::STK_ERR_INVALID_ARG : capi::STK_ERR_NO_DEVICE, "StkWallFMM");
        if (!enableFF_) {
            const int rc = capi::StkWallFMM_set_far_field(h, 0);
            if (rc) {
                capi::StkWallFMM_destroy(h);
                throw Error(rc, "StkWallFMM");
            }
        }
    }
    StkWallFMM(StkWallFMM &&o) noexcept : STKFMM(std::move(o)), h(o.h) { o.h = nullptr; }
    ~StkWallFMM() { capi::StkWallFMM_destroy(h); }

    void setPoints(const int nSL, const double *srcSLCoordPtr, const int nTrg, const double *trgCoordPtr,
                   const int nDL = 0, const double *srcDLCoordPtr = nullptr) override {
        detail::check(capi::StkWallFMM_set_points(h, nSL, const_cast<double *>(srcSLCoordPtr), nTrg,
                                            const_cast<double *>(trgCoordPtr), nDL,
                                            const_cast<double *>(srcDLCoordPtr)),
                      "setPoints");
    }
    void setupTree(KERNEL kernel) override { detail::check(capi::StkWallFMM_setup_tree(h, asInteger(kernel)), "setupTree"); }
    void evaluateFMM(const KERNEL kernel, const int nSL, const double *srcSLValuePtr, const int nTrg,
                     double *trgValuePtr, const int nDL = 0, const double *srcDLValuePtr = nullptr) override {
        detail::check(capi::StkWallFMM_evaluate_fmm(h, asInteger(kernel), nSL, const_cast<double *>(srcSLValuePtr), nTrg,
                                              trgValuePtr, nDL, const_cast<double *>(srcDLValuePtr)),
                      "evaluateFMM");
    }
    void clearFMM(KERNEL kernel) override { detail::check(capi::StkWallFMM_clear_fmm(h, asInteger(kernel)), "clearFMM"); }
    void showActiveKernels() const override {
        detail::check(capi::StkWallFMM_show_active_kernels(h), "showActiveKernels");
    }
    void setPrecision(int precision_) override {
        detail::check(capi::StkWallFMM_set_precision(h, precision_), "setPrecision");
        precision = precision_;
    }

    capi::StkWallFMM *handle() const { return h; }

  protected:
    void setBoxImpl(double origin_[3], double len_) override {
        detail::check(capi::StkWallFMM_set_box(h, origin_, len_), "setBox");
    }
    /* the wall's sub-FMMs (StkWallFMM.cpp:5-32): Stokes with LapPGrad and
     * LapPGradGrad; RPY with LapPGrad, LapPGradGrad and LapQPGradGrad */
    bool hasKernel(KERNEL kernel) const override {
        const bool stokes = isKernelActive(KERNEL::Stokes), rpy = isKernelActive(KERNEL::RPY);
        switch (kernel) {
        case KERNEL::Stokes: return stokes;
        case KERNEL::RPY: return rpy;
        case KERNEL::LapPGrad:
        case KERNEL::LapPGradGrad: return stokes || rpy;
        case KERNEL::LapQPGradGrad: return rpy;
        default: return false;
        }
    }

  private:
    capi::StkWallFMM *h = nullptr;
};

}  // namespace stkfmm

#endif
