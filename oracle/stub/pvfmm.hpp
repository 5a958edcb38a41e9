// Stand-in for PVFMM's umbrella header, for the CPU oracle only (test
// infrastructure, never shipped).
//
// The reference's kernel headers (Lib/include/STKFMM/*Kernel.hpp and
// stkfmm_helpers.hpp) include <pvfmm.hpp> and build on four things from PVFMM
// and SCTL, which are not in the reference tree: the vector type a micro-kernel
// body runs on, sctl::approx_rsqrt / sctl::const_pi, the GenericKernel base
// whose Eval drives a uKerEval body over (target, source) pairs, and Kernel<T>
// with BuildKernel, which composes the FMM's per-slot kernels.  This file gives
// minimal versions of its own so that oracle/_ref can compile those headers in
// place and run their uKerEval bodies and compositions:
//
//   * Vec: one double; the comparison yields a mask.
//   * approx_rsqrt<digits>(r2[, mask]): exact 1/sqrt(r2) (0 where a mask is
//     given and fails); SCTL's Newton-digit approximation is not restated.
//   * GenericKernel<K>::Eval<T>: out[t] += ScaleFactor * sum_s uKerEval(x_t - x_s,
//     v_s) for dof = 1, sources in order.
//   * BuildKernel records the kernel's name, dimensions, its single- and
//     double-layer Eval functions and its sub-kernel pointers; a null sub-kernel
//     stands for the kernel itself, as PVFMM uses it.
//   * stokes_vel / StokesKernel<T>::velocity(): PVFMM's Stokeslet, declared so
//     that compositions naming it compile and can be recorded; its body is not
//     the reference's (the Stokeslet formula, 1/8pi (f/r + r (f.r)/r^3)).
//   * PtFMM, PtFMM_Tree, PtFMM_Data, Vector, BoundaryType and PtFMM_Evaluate:
//     enough for Lib/src/FMMData.cpp and STKFMM.cpp to compile and for an
//     FMMData to run its own steps around the FMM.  PtFMM::Initialize does
//     what PVFMM's kernel initialisation does for the slots (a null sub-kernel
//     becomes the kernel itself).  PtFMM_Evaluate has two modes, chosen by
//     stub_fmm_direct (defined by the program that uses this file): 0 sets every
//     target value to 1 (and the root's upward-equivalent density to
//     stub_root_equiv), so that what FMMData applies after it (periodizeFMM,
//     scaleTrg) shows; 1 returns what the FMM approximates, the direct sum of the kernel's
//     S2T single and double layer over all sources, so that the reference's own
//     FMMData, Stk3DFMM and StkWallFMM code around it runs as an exact method.
#pragma once
#include <mpi.h>

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef PVFMM_MAX_DEPTH
#define PVFMM_MAX_DEPTH 30
#endif
// KIFMM surface radii (in box half-widths) of PVFMM, the scaleIn / scaleOut of
// the reference's M2C generators
#define PVFMM_RAD0 1.05
#define PVFMM_RAD1 2.95

namespace sctl {

struct Mask {
    bool v;
};

struct Vec {
    using ScalarType = double;
    double v;
    Vec() : v(0.0) {}
    Vec(double x) : v(x) {}
    static Vec Zero() { return Vec(0.0); }
    Vec &operator+=(const Vec &o) {
        v += o.v;
        return *this;
    }
    Vec &operator-=(const Vec &o) {
        v -= o.v;
        return *this;
    }
    Vec &operator*=(const Vec &o) {
        v *= o.v;
        return *this;
    }
};
inline Vec operator+(const Vec &a, const Vec &b) { return Vec(a.v + b.v); }
inline Vec operator-(const Vec &a, const Vec &b) { return Vec(a.v - b.v); }
inline Vec operator*(const Vec &a, const Vec &b) { return Vec(a.v * b.v); }
inline Vec operator/(const Vec &a, const Vec &b) { return Vec(a.v / b.v); }
inline Vec operator-(const Vec &a) { return Vec(-a.v); }
inline Mask operator>(const Vec &a, const Vec &b) { return Mask{a.v > b.v}; }

template <class Real>
inline Real const_pi() {
    return (Real)3.14159265358979323846264338327950288;
}

template <int digits>
inline Vec approx_rsqrt(const Vec &r2, const Mask &m) {
    return m.v ? Vec(1.0 / std::sqrt(r2.v)) : Vec(0.0);
}

template <int digits>
inline Vec approx_rsqrt(const Vec &r2) {
    return Vec(1.0 / std::sqrt(r2.v));
}

}  // namespace sctl

namespace pvfmm {

namespace mem {
struct MemoryManager;
}

template <class T>
struct Kernel {
    typedef void (*Ker_t)(T *r_src, int src_cnt, T *v_src, int dof, T *r_trg, int trg_cnt, T *k_out,
                          mem::MemoryManager *mem_mgr);
    const char *ker_name = nullptr;
    int dim = 3;
    int ker_dim[2] = {0, 0};
    int surf_dim = 0;
    Ker_t ker_poten = nullptr;
    Ker_t dbl_layer_poten = nullptr;
    const Kernel<T> *k_s2m = nullptr, *k_s2l = nullptr, *k_s2t = nullptr, *k_m2m = nullptr, *k_m2l = nullptr,
                    *k_m2t = nullptr, *k_l2l = nullptr, *k_l2t = nullptr;
    bool scale_invar = true;
};

template <class T, typename Kernel<T>::Ker_t A, typename Kernel<T>::Ker_t B = nullptr>
Kernel<T> BuildKernel(const char *name, int dim, std::pair<int, int> k_dim, const Kernel<T> *k_s2m = nullptr,
                      const Kernel<T> *k_s2l = nullptr, const Kernel<T> *k_s2t = nullptr,
                      const Kernel<T> *k_m2m = nullptr, const Kernel<T> *k_m2l = nullptr,
                      const Kernel<T> *k_m2t = nullptr, const Kernel<T> *k_l2l = nullptr,
                      const Kernel<T> *k_l2t = nullptr, const void *vol_poten = nullptr, bool scale_invar = true) {
    (void)vol_poten;
    Kernel<T> k;
    k.ker_name = name;
    k.dim = dim;
    k.ker_dim[0] = k_dim.first;
    k.ker_dim[1] = k_dim.second;
    k.ker_poten = A;
    k.dbl_layer_poten = B;
    k.k_s2m = k_s2m;
    k.k_s2l = k_s2l;
    k.k_s2t = k_s2t;
    k.k_m2m = k_m2m;
    k.k_m2l = k_m2l;
    k.k_m2t = k_m2t;
    k.k_l2l = k_l2l;
    k.k_l2t = k_l2t;
    k.scale_invar = scale_invar;
    return k;
}

template <class K>
struct GenericKernel {
    template <class T>
    static void Eval(T *r_src, int src_cnt, T *v_src, int dof, T *r_trg, int trg_cnt, T *k_out,
                     mem::MemoryManager *) {
        (void)dof;
        run<T>(&K::template uKerEval<sctl::Vec, 16>, r_src, src_cnt, v_src, r_trg, trg_cnt, k_out);
    }

  private:
    template <class T, int N, int M>
    static void run(void (*fn)(sctl::Vec (&)[N], const sctl::Vec (&)[3], const sctl::Vec (&)[M], const void *),
                    T *r_src, int src_cnt, T *v_src, T *r_trg, int trg_cnt, T *k_out) {
        const T scale = K::template ScaleFactor<T>();
        for (int t = 0; t < trg_cnt; t++) {
            sctl::Vec u[N];
            for (int s = 0; s < src_cnt; s++) {
                const sctl::Vec r[3] = {sctl::Vec(r_trg[3 * t] - r_src[3 * s]),
                                        sctl::Vec(r_trg[3 * t + 1] - r_src[3 * s + 1]),
                                        sctl::Vec(r_trg[3 * t + 2] - r_src[3 * s + 2])};
                sctl::Vec f[M];
                for (int k = 0; k < M; k++) f[k] = sctl::Vec(v_src[(size_t)M * s + k]);
                fn(u, r, f, nullptr);
            }
            for (int i = 0; i < N; i++) k_out[(size_t)N * t + i] += scale * u[i].v;
        }
    }
};

struct stokes_vel : public GenericKernel<stokes_vel> {
    template <class Real>
    static Real ScaleFactor() {
        return 1.0 / (8.0 * sctl::const_pi<Real>());
    }
    template <class VecType, int digits>
    static void uKerEval(VecType (&u)[3], const VecType (&r)[3], const VecType (&f)[3], const void *) {
        const VecType r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const VecType rinv = sctl::approx_rsqrt<digits>(r2, r2 > VecType::Zero());
        const VecType fr = (f[0] * r[0] + f[1] * r[1] + f[2] * r[2]) * rinv * rinv * rinv;
        for (int i = 0; i < 3; i++) u[i] += f[i] * rinv + r[i] * fr;
    }
};

template <class T>
struct Vector {
    std::vector<T> v;
    Vector &operator=(const std::vector<T> &o) {
        v = o;
        return *this;
    }
    size_t Dim() const { return v.size(); }
    void Resize(size_t n) { v.resize(n); }
    void ReInit(size_t n) { v.assign(n, T(0)); }
    T *Begin() { return v.data(); }
    T &operator[](size_t i) { return v[i]; }
    const T &operator[](size_t i) const { return v[i]; }
};

enum class BoundaryType { FreeSpace, PX, PXY, PXYZ };

extern int stub_fmm_direct;
// ones mode: the root's upward-equivalent density the stand-in FMM leaves behind
// (read by FMMData::periodizeFMM); empty leaves it as it is
extern std::vector<double> stub_root_equiv;

template <class T>
struct PtFMM {
    const Kernel<T> *ker = nullptr;
    void Initialize(int, MPI_Comm, const Kernel<T> *k) {
        ker = k;
        Kernel<T> *kk = const_cast<Kernel<T> *>(k);
        const Kernel<T> **slots[] = {&kk->k_s2m, &kk->k_s2l, &kk->k_s2t, &kk->k_m2m,
                                     &kk->k_m2l, &kk->k_m2t, &kk->k_l2l, &kk->k_l2t};
        for (auto s : slots)
            if (!*s) *s = k;
    }
    void SetM2C(const double *) {}
};

template <class T>
struct PtFMM_Data {
    int dim = 3, max_depth = 0, max_pts = 0;
    Vector<T> pt_coord, src_coord, src_value, surf_coord, surf_value, trg_coord, trg_value;
    void Clear() {}
};

template <class T>
struct PtFMM_Node_Data {
    Vector<T> upward_equiv;
};

template <class T>
struct PtFMM_Node {
    PtFMM_Node_Data<T> data;
    PtFMM_Node_Data<T> *FMMData() { return &data; }
};

template <class T>
struct PtFMM_Tree {
    PtFMM_Node<T> root;
    PtFMM_Data<T> *data = nullptr;
    PtFMM<T> *fmm = nullptr;
    explicit PtFMM_Tree(MPI_Comm) {}
    void Initialize(PtFMM_Data<T> *d) { data = d; }
    void InitFMM_Tree(bool, BoundaryType) {}
    void SetupFMM(PtFMM<T> *m) { fmm = m; }
    void ClearFMMData() {}
    PtFMM_Node<T> *RootNode() { return &root; }
};

template <class T>
inline void PtFMM_Evaluate(PtFMM_Tree<T> *tree, std::vector<T> &trg_val, size_t, std::vector<T> *src_val = nullptr,
                           std::vector<T> *surf_val = nullptr) {
    if (!stub_fmm_direct) {
        std::fill(trg_val.begin(), trg_val.end(), T(1));
        if (!stub_root_equiv.empty()) tree->root.data.upward_equiv = stub_root_equiv;
        return;
    }
    std::fill(trg_val.begin(), trg_val.end(), T(0));
    const Kernel<T> *s2t = tree->fmm->ker->k_s2t;
    PtFMM_Data<T> &d = *tree->data;
    const int ntrg = (int)(d.trg_coord.Dim() / 3), nsrc = (int)(d.src_coord.Dim() / 3),
              nsurf = (int)(d.surf_coord.Dim() / 3);
    if (src_val && nsrc && s2t->ker_poten)
        s2t->ker_poten(d.src_coord.Begin(), nsrc, src_val->data(), 1, d.trg_coord.Begin(), ntrg, trg_val.data(),
                       nullptr);
    if (surf_val && nsurf && s2t->dbl_layer_poten)
        s2t->dbl_layer_poten(d.surf_coord.Begin(), nsurf, surf_val->data(), 1, d.trg_coord.Begin(), ntrg,
                             trg_val.data(), nullptr);
}

template <class T>
struct StokesKernel {
    static const Kernel<T> &velocity() {
        static Kernel<T> k = BuildKernel<T, stokes_vel::Eval<T>>("stokes_vel", 3, std::pair<int, int>(3, 3));
        return k;
    }
};

}  // namespace pvfmm
