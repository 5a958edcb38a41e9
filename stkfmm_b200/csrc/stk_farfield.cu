// stk_farfield.cu -- KIFMM far field on the GPU (see stk_farfield.hpp).
//
// Operators.  The translation kernels handled here (laplace_p, stokes_vel) are
// homogeneous of degree -1: K(s x) = K(x) / s.  With check and equivalent
// surfaces scaled with the box, the pseudo-inverses scale as 2^-l at level l
// and the kernel matrices as 2^l, so M2M, L2L and M2L (which includes the
// downward check-to-equivalent solve) are the same at every level.  They are
// built once per (kernel, p) from a reference box of side 1:
//   UC2UE = pinv(K(UC, UE)),  DC2DE = pinv(K(DC, DE))           (FP64 SVD)
//   M2M_o = UC2UE K(UC, UE_child o)        8 child octants
//   L2L_o = DC2DE_child K(DC_child o, DE)  8 child octants
//   M2L_d = DC2DE K(DC, UE shifted by d)   316 well-separated offsets d
// S2M and S2L produce check potentials directly (P2P), solved with 2^-l UC2UE /
// 2^-l DC2DE.  M2M, L2L and M2L run as cuBLAS DGEMMs; S2M, S2L, M2T (W-list)
// and L2T run on the list P2P kernel with the surface points as sources or
// targets.
#include <algorithm>
#include <tuple>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>

#include "../../include/stkfmm_b200.h"
#include "stk_farfield.hpp"
#include "stk_ewald.cuh"
#include "stk_ukernels.cuh"
#include "stk_umma.cuh"
#include "stk_work.hpp"

namespace stk {

namespace {

#define FCUDA(call)                                    \
    do {                                               \
        if ((call) != cudaSuccess) return STK_ERR_CUDA; \
    } while (0)
#define FBLAS(call)                                               \
    do {                                                          \
        if ((call) != CUBLAS_STATUS_SUCCESS) return STK_ERR_CUDA; \
    } while (0)

constexpr int kNumOffsets = 343;  // (dx, dy, dz) in [-3, 3]^3

// kernels of this file launched by the current evaluation on this host thread
thread_local int t_launches = 0;

// Points of the KIFMM cube surface on [-1, 1]^3, in the order of stkfmm::surface
// (Lib/include/STKFMM/stkfmm_helpers.hpp:46-85) before its affine map.
std::vector<double> unit_surface(int p) {
    const int n = 6 * (p - 1) * (p - 1) + 2;
    std::vector<double> c(3 * (size_t)n);
    c[0] = c[1] = c[2] = -1.0;
    int cnt = 1;
    const double q = p - 1;
    for (int i = 0; i < p - 1; i++)
        for (int j = 0; j < p - 1; j++, cnt++) {
            c[3 * cnt + 0] = -1.0;
            c[3 * cnt + 1] = (2.0 * (i + 1) - p + 1) / q;
            c[3 * cnt + 2] = (2.0 * j - p + 1) / q;
        }
    for (int i = 0; i < p - 1; i++)
        for (int j = 0; j < p - 1; j++, cnt++) {
            c[3 * cnt + 0] = (2.0 * i - p + 1) / q;
            c[3 * cnt + 1] = -1.0;
            c[3 * cnt + 2] = (2.0 * (j + 1) - p + 1) / q;
        }
    for (int i = 0; i < p - 1; i++)
        for (int j = 0; j < p - 1; j++, cnt++) {
            c[3 * cnt + 0] = (2.0 * (i + 1) - p + 1) / q;
            c[3 * cnt + 1] = (2.0 * j - p + 1) / q;
            c[3 * cnt + 2] = -1.0;
        }
    for (int i = 0; i < (n / 2) * 3; i++) c[3 * (size_t)cnt + i] = -c[i];
    return c;
}

// out[(i n + k) 3 + d] = centre(node_i) + alpha r(node_i) unit[k]; node_i = nodes[i]
// (or i when nodes is null), r = 0.5 * 2^-level.
__global__ void surface_points_kernel(const int *__restrict__ nodes, int m, const double *__restrict__ centre,
                                      const int *__restrict__ level, double alpha, const double *__restrict__ unit,
                                      int n, double *__restrict__ out) {
    const long long total = (long long)m * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / n), k = (int)(idx - (long long)i * n);
        const int b = nodes ? nodes[i] : i;
        const double r = alpha * ldexp(0.5, -level[b]);
#pragma unroll
        for (int d = 0; d < 3; d++) out[3 * idx + d] = centre[3 * (size_t)b + d] + r * unit[3 * k + d];
    }
}

// M[(i TDIM + a) + ld (j SDIM + c)] = SCALE comp_scale(a) K_ac(X_i - Y_j): the
// kernel matrix from unit source densities.
template <int UK>
__global__ void kernel_matrix_kernel(const double *__restrict__ X, int ni, const double *__restrict__ Y, int nj,
                                     double *__restrict__ M, int ld) {
    using K = Uk<UK>;
    const long long total = (long long)ni * nj;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % ni), j = (int)(idx / ni);
        const double dx = X[3 * i] - Y[3 * j], dy = X[3 * i + 1] - Y[3 * j + 1], dz = X[3 * i + 2] - Y[3 * j + 2];
        for (int c = 0; c < K::SDIM; c++) {
            double f[K::SDIM], v[K::NV], u[K::TDIM];
            for (int q = 0; q < K::SDIM; q++) f[q] = q == c ? 1.0 : 0.0;
            for (int a = 0; a < K::TDIM; a++) u[a] = 0.0;
            K::stage(f, v);
            K::eval(u, dx, dy, dz, v);
            for (int a = 0; a < K::TDIM; a++)
                M[(size_t)(i * K::TDIM + a) + (size_t)ld * (j * K::SDIM + c)] = K::SCALE * K::comp_scale(a) * u[a];
        }
    }
}

// Singly periodic (PX) far images: the images t = 2 .. kPxImages - 1 on both
// sides along x, summed directly with the micro-kernel, as the reference's
// generators do: t < SUM1D = 500000 for laplace_p and stokes_vel
// (M2L/Laplace/Laplace1D3D.cpp:18-28, M2L/Stokeslet/Stokes1D3D.cpp:37,
// M2L/SVD_pvfmm.hpp:35), t < 1000000 for stokes_pvel
// (M2L/StokesPVel/StokesPVel1D3D.cpp:36-46).  Their sums start at t = 3
// because PVFMM's lists reach two cells; this library's reach one.  The sum
// runs from the farthest images inwards with compensation; for a neutral
// (and force-free) root density the images' tail decays like a dipole
// lattice, so the cut-off costs about 1 / kPxImages of a dipole's field.
template <int UK>
constexpr int kPxImages = UK == UK_STOKES_PVEL ? 1000000 : 500000;

template <int UK>
__global__ void m2c_px_kernel(const double *__restrict__ X, int ni, const double *__restrict__ Y, int nj,
                              double *__restrict__ M, int ld) {
    using K = Uk<UK>;
    const long long total = (long long)ni * nj;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % ni), j = (int)(idx / ni);
        const double r0[3] = {X[3 * i] - Y[3 * j], X[3 * i + 1] - Y[3 * j + 1], X[3 * i + 2] - Y[3 * j + 2]};
        for (int col = 0; col < K::SDIM; col++) {
            double f[K::SDIM], v[K::NV], sum[K::TDIM], cmp[K::TDIM];
            for (int q = 0; q < K::SDIM; q++) f[q] = q == col ? 1.0 : 0.0;
            for (int q = 0; q < K::TDIM; q++) sum[q] = cmp[q] = 0.0;
            K::stage(f, v);
            for (int t = kPxImages<UK> - 1; t >= 2; t--) {
                double u[K::TDIM];
                for (int q = 0; q < K::TDIM; q++) u[q] = 0.0;
                K::eval(u, r0[0] + t, r0[1], r0[2], v);
                K::eval(u, r0[0] - t, r0[1], r0[2], v);
                for (int q = 0; q < K::TDIM; q++) {
                    const double y = u[q] - cmp[q], s2 = sum[q] + y;
                    cmp[q] = (s2 - sum[q]) - y;
                    sum[q] = s2;
                }
            }
            for (int q = 0; q < K::TDIM; q++)
                M[(size_t)(K::TDIM * i + q) + (size_t)ld * (K::SDIM * j + col)] = K::SCALE * K::comp_scale(q) * sum[q];
        }
    }
}

// Far field off (the reference's enableFF = false: no periodic far-image
// operator, FMMData.cpp:83-89): the periodic sum stops at the images that
// PVFMM's periodic lists reach, |s_i| <= 2 on each periodic axis (the block
// the reference's M2C generators leave to the tree, DIRECTLAYER = 2,
// M2L/SVD_pvfmm.hpp:34).  This build's lists reach |s_i| <= 1, so the ring of
// images between the two blocks goes through the root's equivalent density:
// M = sum over that ring of the translation kernel, summed directly with the
// micro-kernel.  PBC = 1, 2, 3: periodic in x; x and y; x, y and z.
template <int UK, int PBC>
__global__ void m2c_ring_kernel(const double *__restrict__ X, int ni, const double *__restrict__ Y, int nj,
                                double *__restrict__ M, int ld) {
    using K = Uk<UK>;
    constexpr int LB = PBC >= 2 ? 2 : 0, LC = PBC == 3 ? 2 : 0;
    const long long total = (long long)ni * nj;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % ni), j = (int)(idx / ni);
        const double r0[3] = {X[3 * i] - Y[3 * j], X[3 * i + 1] - Y[3 * j + 1], X[3 * i + 2] - Y[3 * j + 2]};
        double out[K::TDIM][K::SDIM];
        for (int p = 0; p < K::TDIM; p++)
            for (int q = 0; q < K::SDIM; q++) out[p][q] = 0.0;
        for (int a = -2; a <= 2; a++)
            for (int b = -LB; b <= LB; b++)
                for (int c = -LC; c <= LC; c++) {
                    if (a >= -1 && a <= 1 && b >= -1 && b <= 1 && c >= -1 && c <= 1) continue;
                    for (int col = 0; col < K::SDIM; col++) {
                        double f[K::SDIM], v[K::NV], u[K::TDIM];
                        for (int q = 0; q < K::SDIM; q++) f[q] = q == col ? 1.0 : 0.0;
                        for (int q = 0; q < K::TDIM; q++) u[q] = 0.0;
                        K::stage(f, v);
                        K::eval(u, r0[0] + a, r0[1] + b, r0[2] + c, v);
                        for (int q = 0; q < K::TDIM; q++) out[q][col] += K::SCALE * K::comp_scale(q) * u[q];
                    }
                }
        for (int p = 0; p < K::TDIM; p++)
            for (int q = 0; q < K::SDIM; q++)
                M[(size_t)(K::TDIM * i + p) + (size_t)ld * (K::SDIM * j + q)] = out[p][q];
    }
}

// Far-image operator of the periodic unit cell: M[(i kc + a) + ld (j ke + c)] =
// K_far(X_i - Y_j)_ac, the sum of the translation kernel over every periodic image
// outside the block the tree's periodic lists cover (images with |s| <= 1 on each
// periodic axis).  K_far = (Ewald sum over all images) - (that block, summed
// directly with the micro-kernel itself).  PBC = 3: periodic in x, y, z; PBC = 2:
// in x and y.  The Ewald sums are those of stk_ewald.cuh; for stokes_pvel the
// pressure row is -grad(psi).f / 4 pi and the trD column grad(psi) / 8 pi.
// Triply periodic stokes_pvel carries the reference's two extra terms
// (M2L/StokesPVel/StokesPVel3D3D.cpp:203-218): a pressure (x_i - 1/2).f that
// balances a net force, and on the trD column a velocity of half the source
// point's position wrapped into the cell (the net flux of a trD dipole; the
// unwrapped rest is added after the evaluation, pvel_net_flux_kernel).
// row_shift (nullable): subtracted from every column of row i (the Laplace
// neutraliser of m2c_neutral_kernel).
template <int UK, int PBC>
__global__ void m2c_kernel(const double *__restrict__ X, int ni, const double *__restrict__ Y, int nj,
                           double *__restrict__ M, int ld, const double *__restrict__ row_shift) {
    using K = Uk<UK>;
    constexpr double pi = ewald::kPi;
    const long long total = (long long)ni * nj;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % ni), j = (int)(idx / ni);
        const double r0[3] = {X[3 * i] - Y[3 * j], X[3 * i + 1] - Y[3 * j + 1], X[3 * i + 2] - Y[3 * j + 2]};
        double out[K::TDIM][K::SDIM];
        if (UK == UK_LAPLACE_P || UK == UK_STOKES_PVEL) {
            double pot, g[3];
            if (PBC == 3)
                ewald::lap3(r0, pot, g);
            else
                ewald::lap2(r0, pot, g);
            if constexpr (UK == UK_LAPLACE_P) {
                out[0][0] = pot / (4 * pi);
            } else {
                for (int q = 0; q < 3; q++) out[0][q] = -g[q] / (4 * pi);
                out[0][3] = 0.0;
                for (int p = 0; p < 3; p++) out[1 + p][3] = g[p] / (8 * pi);
            }
        }
        if (UK == UK_STOKES_VEL || UK == UK_STOKES_PVEL) {
            double G[3][3];
            if (PBC == 3)
                ewald::stk3(r0, G);
            else
                ewald::stk2(r0, G);
            constexpr int o = UK == UK_STOKES_PVEL ? 1 : 0;
            for (int p = 0; p < 3; p++)
                for (int q = 0; q < 3; q++) out[o + p][q] = G[p][q] / (8 * pi);
        }
        // minus the directly summed block of images, with the micro-kernel's own normalisation
        for (int a = -1; a <= 1; a++)
            for (int b = -1; b <= 1; b++)
                for (int c = (PBC == 3 ? -1 : 0); c <= (PBC == 3 ? 1 : 0); c++) {
                    const double dx = r0[0] + a, dy = r0[1] + b, dz = r0[2] + c;
                    for (int col = 0; col < K::SDIM; col++) {
                        double f[K::SDIM], v[K::NV], u[K::TDIM];
                        for (int q = 0; q < K::SDIM; q++) f[q] = q == col ? 1.0 : 0.0;
                        for (int q = 0; q < K::TDIM; q++) u[q] = 0.0;
                        K::stage(f, v);
                        K::eval(u, dx, dy, dz, v);
                        for (int q = 0; q < K::TDIM; q++) out[q][col] -= K::SCALE * K::comp_scale(q) * u[q];
                    }
                }
        if constexpr (UK == UK_STOKES_PVEL && PBC == 3) {
            for (int q = 0; q < 3; q++) out[0][q] += X[3 * i + q] - 0.5;
            for (int p = 0; p < 3; p++) {
                const double y = Y[3 * j + p];
                out[1 + p][3] += 0.5 * (y - floor(y));
            }
        }
        if (row_shift)
            for (int p = 0; p < K::TDIM; p++)
                for (int q = 0; q < K::SDIM; q++) out[p][q] -= row_shift[K::TDIM * i + p];
        for (int p = 0; p < K::TDIM; p++)
            for (int q = 0; q < K::SDIM; q++)
                M[(size_t)(K::TDIM * i + p) + (size_t)ld * (K::SDIM * j + q)] = out[p][q];
    }
}

// The reference's triply periodic Laplace operator pairs every equivalent
// charge with an opposite one at the cell centre N = (1/2, 1/2, 1/2)
// (M2L/Laplace/Laplace3D3D.cpp:266-273): w_i = K_far(X_i - N), the Ewald sum
// minus the 5 x 5 x 5 block of images the reference's generator sums directly
// (DIRECTLAYER = 2, M2L/SVD_pvfmm.hpp:34), is taken off every column of row i.
// For a neutral density the columns' sum of charges is zero and so is the
// term; for a charged one it is the reference's convention.
__global__ void m2c_neutral_kernel(const double *__restrict__ X, int ni, double *__restrict__ w) {
    constexpr double pi = ewald::kPi;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ni; i += gridDim.x * blockDim.x) {
        const double r0[3] = {X[3 * i] - 0.5, X[3 * i + 1] - 0.5, X[3 * i + 2] - 0.5};
        double pot, g[3];
        ewald::lap3(r0, pot, g);
        double near = 0.0;
        for (int a = -2; a <= 2; a++)
            for (int b = -2; b <= 2; b++)
                for (int c = -2; c <= 2; c++) {
                    const double x = r0[0] + a, y = r0[1] + b, z = r0[2] + c;
                    near += 1.0 / sqrt(x * x + y * y + z * z);
                }
        w[i] = (pot - near) / (4 * pi);
    }
}

// Triply periodic PVel, PVelGrad and PVelLaplacian: the net-flux correction of
// FMMData::periodizeFMM (Lib/src/FMMData.cpp:203-247).  With y_i the root's
// upward-equivalent points and trD_i their trD densities, every target's
// velocity (components 1..3) gets (1/2) sum_i (y_i - wrap(y_i)) trD_i; with the
// wrapped half inside the M2C operator that makes (1/2) sum_i y_i trD_i, half
// the trD dipole moment.  Each block reduces the n root values itself (in the
// same order) and adds the result to its targets.
constexpr int kNetFluxThreads = 256;  // the block size pvel_net_flux_kernel is launched with (a power of two)

__global__ void __launch_bounds__(kNetFluxThreads)
    pvel_net_flux_kernel(const double *__restrict__ phi_root, const double *__restrict__ ue_root, int n,
                         double *__restrict__ trg, long long ntrg, int td) {
    __shared__ double red[3][kNetFluxThreads];
    double u[3] = {0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double trd = phi_root[4 * i + 3];
        for (int c = 0; c < 3; c++) u[c] += floor(ue_root[3 * i + c]) * trd;
    }
    for (int c = 0; c < 3; c++) red[c][threadIdx.x] = u[c];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int c = 0; c < 3; c++) red[c][threadIdx.x] += red[c][threadIdx.x + h];
        __syncthreads();
    }
    const double U[3] = {0.5 * red[0][0], 0.5 * red[1][0], 0.5 * red[2][0]};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntrg;
         t += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; c++) trg[t * td + 1 + c] += U[c];
}

int kernel_matrix(int uk, const double *X, int ni, const double *Y, int nj, double *M, int ld, cudaStream_t s) {
    const long long total = (long long)ni * nj;
    const int threads = 256;
    const int grid = (int)std::min<long long>((total + threads - 1) / threads, 148 * 32);
    if (uk == UK_LAPLACE_P)
        kernel_matrix_kernel<UK_LAPLACE_P><<<grid, threads, 0, s>>>(X, ni, Y, nj, M, ld);
    else if (uk == UK_STOKES_VEL)
        kernel_matrix_kernel<UK_STOKES_VEL><<<grid, threads, 0, s>>>(X, ni, Y, nj, M, ld);
    else if (uk == UK_STOKES_PVEL)
        kernel_matrix_kernel<UK_STOKES_PVEL><<<grid, threads, 0, s>>>(X, ni, Y, nj, M, ld);
    else
        return STK_ERR_NOT_SUPPORTED;
    return cudaGetLastError() == cudaSuccess ? STK_OK : STK_ERR_CUDA;
}

// Per-component factors (up to 4 components, repeated over surface points).
struct CompF {
    double v[4];
};

// M[i + ld j] *= fr.v[i % dim] * fc.v[j % dim]   (rows x cols)
__global__ void scale_rc_kernel(double *__restrict__ M, int rows, int cols, int ld, int dim, CompF fr, CompF fc) {
    const long long total = (long long)rows * cols;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % rows), j = (int)(idx / rows);
        M[(size_t)i + (size_t)ld * j] *= fr.v[i % dim] * fc.v[j % dim];
    }
}

// Column c of buf (rows_per_col values, components interleaved with period dim)
// is multiplied per row by 2^(-level * e[row % dim]); level = col_level[c], or
// level_all when col_level is null.
__global__ void level_scale_kernel(double *__restrict__ buf, long long ncols, int rows_per_col, int dim,
                                   const int *__restrict__ col_level, int level_all, CompF e) {
    const long long total = ncols * rows_per_col;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long c = idx / rows_per_col;
        const int r = (int)(idx - c * rows_per_col);
        const int l = col_level ? col_level[c] : level_all;
        buf[idx] *= exp2(-(double)l * e.v[r % dim]);
    }
}

// W[i + m j] = U[j + m i] / S_i for S_i above the cut, else 0  (W = S^+ U^T)
__global__ void pinv_scale_kernel(const double *__restrict__ U, const double *__restrict__ S, int m, double rtol,
                                  double *__restrict__ W) {
    const double cut = rtol * S[0];
    const long long total = (long long)m * m;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % m), j = (int)(idx / m);
        const double si = S[i];
        W[idx] = si > cut ? U[j + (size_t)m * i] / si : 0.0;
    }
}

// dst[:, j] = src[:, cols[j]] for N-row columns (converted to the type of dst)
template <class TS, class TD>
__global__ void gather_cols_kernel(const TS *__restrict__ src, const int *__restrict__ cols, int m, int N,
                                   TD *__restrict__ dst) {
    const long long total = (long long)m * N;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(idx / N), r = (int)(idx - (long long)j * N);
        dst[idx] = (TD)src[(size_t)cols[j] * N + r];
    }
}

// dst[:, cols[j]] (= or +=) alpha src[:, j]; no two j may share a column
template <class TS>
__global__ void scatter_cols_kernel(const TS *__restrict__ src, const int *__restrict__ cols, int m, int N,
                                    double alpha, int add, double *__restrict__ dst) {
    const long long total = (long long)m * N;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(idx / N), r = (int)(idx - (long long)j * N);
        double *d = dst + (size_t)cols[j] * N + r;
        *d = add ? *d + alpha * (double)src[idx] : alpha * (double)src[idx];
    }
}

inline int grid_for(long long total) { return (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148 * 32)); }

template <class TS, class TD>
int gather_cols(const TS *src, const int *cols, int m, int N, TD *dst, cudaStream_t s) {
    if (m <= 0) return STK_OK;
    t_launches++;
    gather_cols_kernel<TS, TD><<<grid_for((long long)m * N), 256, 0, s>>>(src, cols, m, N, dst);
    return cudaGetLastError() == cudaSuccess ? STK_OK : STK_ERR_CUDA;
}

template <class TS>
int scatter_cols(const TS *src, const int *cols, int m, int N, double alpha, int add, double *dst, cudaStream_t s) {
    if (m <= 0) return STK_OK;
    t_launches++;
    scatter_cols_kernel<TS><<<grid_for((long long)m * N), 256, 0, s>>>(src, cols, m, N, alpha, add, dst);
    return cudaGetLastError() == cudaSuccess ? STK_OK : STK_ERR_CUDA;
}

// R[i + N j] = A[i + m j] for i <= j (the R factor of a QR factorisation)
__global__ void upper_copy_kernel(const double *__restrict__ A, long long m, int N, double *__restrict__ R) {
    const long long total = (long long)N * N;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % N), j = (int)(idx / N);
        if (i <= j) R[idx] = A[(size_t)i + (size_t)m * j];
    }
}

__global__ void to_float_kernel(const double *__restrict__ a, long long n, float *__restrict__ b) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

constexpr int kM2LChunk = 256;  // pairs (columns) per batched-GEMM problem of the M2L

// X[r + k j] = phi_hat[r + k gsrc[j]], or 0 for a padding column (gsrc[j] < 0)
template <class T>
__global__ void m2l_gather_kernel(const double *__restrict__ phi_hat, const int *__restrict__ gsrc, int k,
                                  long long ncol, T *__restrict__ X) {
    const long long total = ncol * k;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long j = idx / k;
        const int r = (int)(idx - j * k);
        const int a = gsrc[j];
        X[idx] = a >= 0 ? (T)phi_hat[(size_t)a * k + r] : (T)0;
    }
}

// psi_hat[r + k t] += sum, in order, of Y[r + k (col[e] - c0)] over target t's
// entries e in [beg[t], end[t]) -- its columns inside the current group, which
// starts at column c0 (a target's columns ascend, so they form one run per group)
template <class T>
__global__ void m2l_reduce_kernel(const T *__restrict__ Y, const int *__restrict__ beg, const int *__restrict__ end,
                                  const int *__restrict__ col, int nn, int k, long long c0,
                                  double *__restrict__ psi_hat) {
    const long long total = (long long)nn * k;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(idx / k), r = (int)(idx - (long long)t * k);
        const int e0 = beg[t], e1 = end[t];
        if (e0 == e1) continue;
        double acc = 0.0;
        for (int e = e0; e < e1; e++) acc += (double)Y[(size_t)((long long)col[e] - c0) * k + r];
        psi_hat[idx] += acc;
    }
}

// Complete-level M2L: Zc[row + R j] = Z[srow[row] + ldz pos] for pos = tab[q + nq j],
// q = rowq[row] (0 where the target j has no source at that offset)
template <class T>
__global__ void m2l_zgather_kernel(const T *__restrict__ Z, int ldz, const int *__restrict__ tab, int nq,
                                   const int *__restrict__ rowq, const int *__restrict__ srow, int R, int n8,
                                   T *__restrict__ Zc) {
    const long long total = (long long)n8 * R;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(idx / R), row = (int)(idx - (long long)j * R);
        const int pos = tab[(size_t)j * nq + rowq[row]];
        Zc[idx] = pos >= 0 ? Z[(size_t)pos * ldz + srow[row]] : T(0);
    }
}

// ---- operands of the tensor-core (3xTF32) M2L ----------------------------------
// the value in FP32, split into TF32 hi / lo parts (tf32_split_value)
__device__ __forceinline__ void tf32_hilo(double v, float &hi, float &lo) { tf32_split_value((float)v, hi, lo); }

// rows of a column-major k x rows FP64 matrix (its columns) as K-major rows of ld floats
__global__ void tc_rows_kernel(const double *__restrict__ src, int k, long long rows, int ld, float *__restrict__ hi,
                               float *__restrict__ lo) {
    const long long total = rows * ld;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / ld;
        const int j = (int)(idx - r * ld);
        float h = 0.f, l = 0.f;
        if (j < k) tf32_hilo(src[r * k + j], h, l);
        hi[idx] = h;
        lo[idx] = l;
    }
}

// the transpose: a column-major k x R FP64 block (ld k) as k K-major rows of ld floats
__global__ void tc_trows_kernel(const double *__restrict__ src, int k, int R, int ld, float *__restrict__ hi,
                                float *__restrict__ lo) {
    const long long total = (long long)k * ld;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(idx / ld), j = (int)(idx - (long long)m * ld);
        float h = 0.f, l = 0.f;
        if (j < R) tf32_hilo(src[(size_t)j * k + m], h, l);
        hi[idx] = h;
        lo[idx] = l;
    }
}

// phi_hat columns cols[j] (k values each, FP64) as K-major rows of ld floats, split;
// cols[j] < 0 (chunk padding) gives a zero row
__global__ void tc_gather_cols_kernel(const double *__restrict__ src, const int *__restrict__ cols, long long n,
                                      int k, int ld, float *__restrict__ hi, float *__restrict__ lo) {
    const long long total = n * ld;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long j = idx / ld;
        const int r = (int)(idx - j * ld);
        const int c = cols[j];
        float h = 0.f, l = 0.f;
        if (r < k && c >= 0) tf32_hilo(src[(size_t)c * k + r], h, l);
        hi[idx] = h;
        lo[idx] = l;
    }
}

// m2l_zgather_kernel's rows of one block, split, as the first `width` floats of
// each target's K-major row (pitch ld; zero beyond R)
__global__ void tc_zgather_kernel(const float *__restrict__ Z, int ldz, const int *__restrict__ tab, int nq,
                                  const int *__restrict__ rowq, const int *__restrict__ srow, int R, int width, int ld,
                                  int n8, float *__restrict__ hi, float *__restrict__ lo) {
    const long long total = (long long)n8 * width;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(i / width), row = (int)(i - (long long)j * width);
        const long long idx = (long long)j * ld + row;
        float v = 0.f;
        if (row < R) {
            const int pos = tab[(size_t)j * nq + rowq[row]];
            v = pos >= 0 ? Z[(size_t)pos * ldz + srow[row]] : 0.f;
        }
        float h, l;
        tf32_split_value(v, h, l);
        hi[idx] = h;
        lo[idx] = l;
    }
}

// A_inv = pinv(A) for an m x m column-major matrix (cuSOLVER SVD, FP64), cut
// at rtol * sigma_max.  A is overwritten.
int pinv(FarField &F, double *A, int m, double *A_inv, double rtol, cudaStream_t s) {
    cusolverDnSetStream(F.solver, s);
    int lwork = 0;
    if (cusolverDnDgesvd_bufferSize(F.solver, m, m, &lwork) != CUSOLVER_STATUS_SUCCESS) return STK_ERR_CUDA;
    DevBuf work, S, U, VT, W, info, rwork;
    int rc = work.reserve(sizeof(double) * (size_t)std::max(lwork, 1));
    if (!rc) rc = S.reserve(sizeof(double) * m);
    if (!rc) rc = U.reserve(sizeof(double) * (size_t)m * m);
    if (!rc) rc = VT.reserve(sizeof(double) * (size_t)m * m);
    if (!rc) rc = W.reserve(sizeof(double) * (size_t)m * m);
    if (!rc) rc = info.reserve(sizeof(int));
    if (!rc) rc = rwork.reserve(sizeof(double) * m);
    if (rc) return rc;
    if (cusolverDnDgesvd(F.solver, 'A', 'A', m, m, A, m, (double *)S.ptr, (double *)U.ptr, m, (double *)VT.ptr, m,
                         (double *)work.ptr, lwork, (double *)rwork.ptr, (int *)info.ptr) != CUSOLVER_STATUS_SUCCESS)
        return STK_ERR_CUDA;
    pinv_scale_kernel<<<grid_for((long long)m * m), 256, 0, s>>>((const double *)U.ptr, (const double *)S.ptr, m, rtol,
                                                               (double *)W.ptr);
    FCUDA(cudaGetLastError());
    const double one = 1.0, zero = 0.0;
    cublasSetStream(F.blas, s);
    // A_inv = V W = VT^T W
    FBLAS(cublasDgemm(F.blas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, m, &one, (const double *)VT.ptr, m,
                      (const double *)W.ptr, m, &zero, A_inv, m));
    int h_info = 0;
    FCUDA(cudaMemcpyAsync(&h_info, info.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    FCUDA(cudaStreamSynchronize(s));
    return h_info == 0 ? STK_OK : STK_ERR_CUDA;
}

// zero the strictly lower triangle of the leading n x n block of A (column-major, lda)
__global__ void zero_lower_kernel(double *A, long long lda, int n) {
    const long long total = (long long)n * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % n), j = (int)(idx / n);
        if (i > j) A[(long long)j * lda + i] = 0.0;
    }
}

// Singular values and right singular vectors of a stack of nblocks N x N blocks
// [B_0; B_1; ...] without holding the stack: a blockwise R-only QR.  A work
// matrix of (g + 1) N rows holds the running triangular factor R on top of the
// next g blocks (fill(b, dst, ld) writes block b); each QR of it leaves the new
// R in its first N rows, whose strictly lower part is cleared before the next
// group.  R^T R equals the stack's Gram matrix, so the SVD of the final R gives
// the stack's singular values and right singular vectors.  The group size keeps
// the work matrix within budget_bytes.
int stack_svd(FarField &F, int nblocks, int N, const std::function<int(int, double *, long long)> &fill, double *S,
              double *VT, cudaStream_t s, size_t budget_bytes) {
    const size_t blk = sizeof(double) * (size_t)N * N;
    int g = (int)std::max<size_t>(1, std::min<size_t>(nblocks, budget_bytes / blk > 1 ? budget_bytes / blk - 1 : 1));
    const long long m = (long long)(g + 1) * N;
    if (m > 0x7fffffffLL) return STK_ERR_SIZE;
    cusolverDnSetStream(F.solver, s);
    DevBuf W, work, tau, R, info, rwork;
    int rc = W.reserve(blk * (size_t)(g + 1));
    if (rc) return rc;
    int lq = 0, ls = 0;
    if (cusolverDnDgeqrf_bufferSize(F.solver, (int)m, N, (double *)W.ptr, (int)m, &lq) != CUSOLVER_STATUS_SUCCESS)
        return STK_ERR_CUDA;
    if (cusolverDnDgesvd_bufferSize(F.solver, N, N, &ls) != CUSOLVER_STATUS_SUCCESS) return STK_ERR_CUDA;
    rc = work.reserve(sizeof(double) * (size_t)std::max(std::max(lq, ls), 1));
    if (!rc) rc = tau.reserve(sizeof(double) * N);
    if (!rc) rc = R.reserve(blk);
    if (!rc) rc = info.reserve(2 * sizeof(int));
    if (!rc) rc = rwork.reserve(sizeof(double) * N);
    if (rc) return rc;
    double *Wp = (double *)W.ptr;
    FCUDA(cudaMemsetAsync(W.ptr, 0, blk * (size_t)(g + 1), s));  // R = 0 before the first group
    for (int b0 = 0; b0 < nblocks; b0 += g) {
        const int nb = std::min(g, nblocks - b0);
        for (int b = 0; b < g; b++) {
            double *dst = Wp + (size_t)(b + 1) * N;  // rows (b + 1) N .. of the work matrix
            if (b < nb) {
                if ((rc = fill(b0 + b, dst, m))) return rc;
            } else {
                FCUDA(cudaMemset2DAsync(dst, sizeof(double) * m, 0, sizeof(double) * N, N, s));
            }
        }
        if (cusolverDnDgeqrf(F.solver, (int)m, N, Wp, (int)m, (double *)tau.ptr, (double *)work.ptr, lq,
                             (int *)info.ptr) != CUSOLVER_STATUS_SUCCESS)
            return STK_ERR_CUDA;
        zero_lower_kernel<<<grid_for((long long)N * N), 256, 0, s>>>(Wp, m, N);
        FCUDA(cudaGetLastError());
    }
    FCUDA(cudaMemsetAsync(R.ptr, 0, blk, s));
    upper_copy_kernel<<<grid_for((long long)N * N), 256, 0, s>>>(Wp, m, N, (double *)R.ptr);
    FCUDA(cudaGetLastError());
    if (cusolverDnDgesvd(F.solver, 'N', 'A', N, N, (double *)R.ptr, N, S, nullptr, N, VT, N, (double *)work.ptr, ls,
                         (double *)rwork.ptr, (int *)info.ptr + 1) != CUSOLVER_STATUS_SUCCESS)
        return STK_ERR_CUDA;
    int h_info[2] = {0, 0};
    FCUDA(cudaMemcpyAsync(h_info, info.ptr, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    FCUDA(cudaStreamSynchronize(s));
    return h_info[0] == 0 && h_info[1] == 0 ? STK_OK : STK_ERR_CUDA;
}

int upload_points(DevBuf &b, const std::vector<double> &v, cudaStream_t s) {
    return b.upload(v.data(), v.size() * sizeof(double), s);
}

std::vector<double> scaled_surface(const std::vector<double> &unit, double cx, double cy, double cz, double r) {
    std::vector<double> o(unit.size());
    for (size_t i = 0; i < unit.size(); i += 3) {
        o[i] = cx + r * unit[i];
        o[i + 1] = cy + r * unit[i + 1];
        o[i + 2] = cz + r * unit[i + 2];
    }
    return o;
}

// ---- two-level M2L: per-offset low-rank factors ----------------------------------
//
// In the shared bases, C_d = U^T A_d V (k x k) has a much lower numerical rank
// for each single offset d than k (e.g. stokes_vel at p = 8: k = 716, r_d ~ 100 -
// 280).  C_d ~ P_d Q_d^T (k x r_d each) turns a pair's 2 k^2 flops into 4 k r_d.
// The surface points and the kernels are symmetric under the 48 signed axis
// permutations G of the cube, A_{G d} = T_out(G) A_d T_in(G)^T (T: the point
// permutation with the components rotated), so only the 16 offsets with
// |dx| >= |dy| >= |dz| >= 0 need an SVD; the others get P, Q from the mapped
// N-space factors: P_{G d} = U^T T_out L_d, Q_{G d} = V^T T_in R_d.

struct SignedPerm {
    int perm[3], sign[3];  // (G x)_a = sign[a] x[perm[a]]
};

// y[pi(i)] = G_comp x[i] for each of r columns (point-major, dim components per point);
// vector components start at vec0 (3 of them) when vec0 >= 0, the others are scalars
__global__ void sym_apply_kernel(const double *__restrict__ x, double *__restrict__ y, int n, int dim, int r,
                                 const int *__restrict__ pi, SignedPerm g, int vec0) {
    const long long total = (long long)n * r;
    const long long N = (long long)n * dim;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % n);
        const long long c = idx / n;
        const double *xi = x + c * N + (long long)i * dim;
        double *yo = y + c * N + (long long)pi[i] * dim;
        for (int a = 0; a < dim; a++) {
            const bool vec = vec0 >= 0 && a >= vec0 && a < vec0 + 3;
            yo[a] = vec ? g.sign[a - vec0] * xi[vec0 + g.perm[a - vec0]] : xi[a];
        }
    }
}

int build_m2l_lowrank(FarField &F, const std::vector<double> &unit, const double *Ut, const double *Vt,
                      const std::function<int(int, double *, int)> &offset_matrix, DevBuf &K, DevBuf &T,
                      cudaStream_t s) {
    const int n = F.n, N = F.n * F.ke, k = F.m2l_rank;
    const double one = 1.0, zero = 0.0;
    cublasSetStream(F.blas, s);
    // component layout of the equivalent densities (in) and check potentials (out)
    const int vec_in = F.m2x == UK_LAPLACE_P ? -1 : 0;
    const int vec_out = F.m2x == UK_LAPLACE_P ? -1 : F.m2x == UK_STOKES_PVEL ? 1 : 0;
    // representative and symmetry of every well-separated offset
    struct Rep {
        int rep;  // index of the representative offset
        SignedPerm g;
    };
    std::vector<int> rep_code;            // representative offsets (codes)
    std::vector<Rep> of(kNumOffsets, {-1, {{0, 1, 2}, {1, 1, 1}}});
    for (int code = 0; code < kNumOffsets; code++) {
        if (F.m2l_slot[code] < 0) continue;
        const int d[3] = {code % 7 - 3, (code / 7) % 7 - 3, code / 49 - 3};
        int o[3] = {0, 1, 2};
        std::stable_sort(o, o + 3, [&](int a, int b) { return std::abs(d[a]) > std::abs(d[b]); });
        const int d0[3] = {std::abs(d[o[0]]), std::abs(d[o[1]]), std::abs(d[o[2]])};
        const int rcode = (d0[0] + 3) + 7 * (d0[1] + 3) + 49 * (d0[2] + 3);
        SignedPerm g;
        for (int t = 0; t < 3; t++) {
            g.perm[o[t]] = t;
            g.sign[o[t]] = d[o[t]] < 0 ? -1 : 1;
        }
        int ri = (int)(std::find(rep_code.begin(), rep_code.end(), rcode) - rep_code.begin());
        if (ri == (int)rep_code.size()) rep_code.push_back(rcode);
        of[code] = {ri, g};
    }
    const int nrep = (int)rep_code.size();
    // SVD of C_d0 = U^T A_d0 V for each representative
    int lw = 0;
    if (cusolverDnDgesvd_bufferSize(F.solver, k, k, &lw) != CUSOLVER_STATUS_SUCCESS) return STK_ERR_CUDA;
    DevBuf C, W, Zt, Sg, work, info, rwork;
    int rc = C.reserve(sizeof(double) * (size_t)k * k);
    if (!rc) rc = W.reserve(sizeof(double) * (size_t)nrep * k * k);
    if (!rc) rc = Zt.reserve(sizeof(double) * (size_t)nrep * k * k);
    if (!rc) rc = Sg.reserve(sizeof(double) * (size_t)nrep * k);
    if (!rc) rc = work.reserve(sizeof(double) * (size_t)std::max(lw, 1));
    if (!rc) rc = info.reserve(sizeof(int) * nrep);
    if (!rc) rc = rwork.reserve(sizeof(double) * k);
    if (rc) return rc;
    cusolverDnSetStream(F.solver, s);
    for (int ri = 0; ri < nrep; ri++) {
        if ((rc = offset_matrix(rep_code[ri], (double *)K.ptr, N))) return rc;
        // T = A V (N x k), C = U^T T (k x k)
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_T, N, k, N, &one, (const double *)K.ptr, N, Vt, N, &zero,
                          (double *)T.ptr, N));
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, k, k, N, &one, Ut, N, (const double *)T.ptr, N, &zero,
                          (double *)C.ptr, k));
        if (cusolverDnDgesvd(F.solver, 'A', 'A', k, k, (double *)C.ptr, k, (double *)Sg.ptr + (size_t)ri * k,
                             (double *)W.ptr + (size_t)ri * k * k, k, (double *)Zt.ptr + (size_t)ri * k * k, k,
                             (double *)work.ptr, lw, (double *)rwork.ptr, (int *)info.ptr + ri) !=
            CUSOLVER_STATUS_SUCCESS)
            return STK_ERR_CUDA;
    }
    std::vector<double> sg((size_t)nrep * k);
    std::vector<int> hinfo(nrep);
    FCUDA(cudaMemcpyAsync(sg.data(), Sg.ptr, sizeof(double) * sg.size(), cudaMemcpyDeviceToHost, s));
    FCUDA(cudaMemcpyAsync(hinfo.data(), info.ptr, sizeof(int) * nrep, cudaMemcpyDeviceToHost, s));
    FCUDA(cudaStreamSynchronize(s));
    for (int v : hinfo)
        if (v != 0) return STK_ERR_CUDA;
    double smax = 0.0;
    for (int ri = 0; ri < nrep; ri++) smax = std::max(smax, sg[(size_t)ri * k]);
    // ranks at the shared bases' cut, relative to the largest C_d (a tenth of it
    // measured the same FMM error to three digits at p = 6 - 10, 9% slower)
#ifndef STK_M2L_PAIR_CUT
#define STK_M2L_PAIR_CUT 1.0
#endif
    std::vector<int> rrank(nrep, 1);
    for (int ri = 0; ri < nrep; ri++)
        for (int i = 0; i < k; i++)
            if (sg[(size_t)ri * k + i] > STK_M2L_PAIR_CUT * F.m2l_rtol * smax) rrank[ri] = i + 1;
    int rmaxr = 1;
    for (int r : rrank) rmaxr = std::max(rmaxr, r);
    // N-space factors of the representatives: L = U W_r S_r, R = V Z_r (N x r each)
    DevBuf Lrep, Rrep, Ws;
    size_t nspace = 0;
    std::vector<size_t> roff(nrep);
    for (int ri = 0; ri < nrep; ri++) {
        roff[ri] = nspace;
        nspace += (size_t)N * rrank[ri];
    }
    rc = Lrep.reserve(sizeof(double) * nspace);
    if (!rc) rc = Rrep.reserve(sizeof(double) * nspace);
    if (!rc) rc = Ws.reserve(sizeof(double) * (size_t)k * rmaxr);
    if (rc) return rc;
    for (int ri = 0; ri < nrep; ri++) {
        const int r = rrank[ri];
        // Ws = W_r S_r (k x r)
        FCUDA(cudaMemcpyAsync(Ws.ptr, (const double *)W.ptr + (size_t)ri * k * k, sizeof(double) * (size_t)k * r,
                              cudaMemcpyDeviceToDevice, s));
        FBLAS(cublasDdgmm(F.blas, CUBLAS_SIDE_RIGHT, k, r, (const double *)Ws.ptr, k,
                          (const double *)Sg.ptr + (size_t)ri * k, 1, (double *)Ws.ptr, k));
        // L = U Ws: U = (rows 0..k-1 of Ut)^T
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_T, CUBLAS_OP_N, N, r, k, &one, Ut, N, (const double *)Ws.ptr, k, &zero,
                          (double *)Lrep.ptr + roff[ri], N));
        // R = V Z_r, Z_r = (rows 0..r-1 of Zt)^T
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_T, CUBLAS_OP_T, N, r, k, &one, Vt, N,
                          (const double *)Zt.ptr + (size_t)ri * k * k, k, &zero, (double *)Rrep.ptr + roff[ri], N));
    }
    // surface point permutations of the symmetries in use
    std::map<long long, int> where;
    auto key = [&](double x, double y, double z) {
        const long long a = std::llround(x * (F.p - 1)) + 64, b = std::llround(y * (F.p - 1)) + 64,
                        c = std::llround(z * (F.p - 1)) + 64;
        return (a * 256 + b) * 256 + c;
    };
    for (int i = 0; i < n; i++) where[key(unit[3 * i], unit[3 * i + 1], unit[3 * i + 2])] = i;
    // per offset: P = U^T T_out L_rep, Q = V^T T_in R_rep
    size_t total = 0;
    int nslot = 0;
    for (int code = 0; code < kNumOffsets; code++)
        if (F.m2l_slot[code] >= 0) nslot++;
    F.m2l_r.assign(nslot, 0);
    F.m2l_rt.assign(nslot, 0);
    F.m2l_pq_off.assign(nslot, 0);
    for (int code = 0; code < kNumOffsets; code++) {
        const int sl = F.m2l_slot[code];
        if (sl < 0) continue;
        // ranks padded to a multiple of 32 (zero columns), so that offsets of similar
        // rank share one uniformly sized batched GEMM
        F.m2l_r[sl] = std::min(k, (rrank[of[code].rep] + 31) / 32 * 32);
        F.m2l_rt[sl] = rrank[of[code].rep];
        F.m2l_pq_off[sl] = total;
        total += (size_t)k * F.m2l_r[sl];
    }
    F.m2l_rmax = 1;
    for (int r : F.m2l_r) F.m2l_rmax = std::max(F.m2l_rmax, r);
    rc = F.m2l_p.reserve(sizeof(double) * std::max<size_t>(total, 1));
    if (!rc) rc = F.m2l_q.reserve(sizeof(double) * std::max<size_t>(total, 1));
    if (!rc) rc = F.m2l_p32.reserve(sizeof(float) * std::max<size_t>(total, 1));
    if (!rc) rc = F.m2l_q32.reserve(sizeof(float) * std::max<size_t>(total, 1));
    DevBuf Tm, pi;
    if (!rc) rc = Tm.reserve(sizeof(double) * (size_t)N * rmaxr);
    if (rc) return rc;
    FCUDA(cudaMemsetAsync(F.m2l_p.ptr, 0, sizeof(double) * total, s));
    FCUDA(cudaMemsetAsync(F.m2l_q.ptr, 0, sizeof(double) * total, s));
    std::vector<int> hpi(n);
    for (int code = 0; code < kNumOffsets; code++) {
        const int sl = F.m2l_slot[code];
        if (sl < 0) continue;
        const int ri = of[code].rep, r = rrank[ri];
        const SignedPerm g = of[code].g;
        for (int i = 0; i < n; i++) {
            double x[3] = {unit[3 * i], unit[3 * i + 1], unit[3 * i + 2]}, gx[3];
            for (int a = 0; a < 3; a++) gx[a] = g.sign[a] * x[g.perm[a]];
            auto it = where.find(key(gx[0], gx[1], gx[2]));
            if (it == where.end()) return STK_ERR_STATE;  // the surface is symmetric by construction
            hpi[i] = it->second;
        }
        rc = pi.upload(hpi.data(), sizeof(int) * n, s);
        if (rc) return rc;
        const int gr = grid_for((long long)n * r);
        double *P = (double *)F.m2l_p.ptr + F.m2l_pq_off[sl], *Q = (double *)F.m2l_q.ptr + F.m2l_pq_off[sl];
        sym_apply_kernel<<<gr, 256, 0, s>>>((const double *)Lrep.ptr + roff[ri], (double *)Tm.ptr, n, F.kc, r,
                                            (const int *)pi.ptr, g, vec_out);
        FCUDA(cudaGetLastError());
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, k, r, N, &one, Ut, N, (const double *)Tm.ptr, N, &zero, P,
                          k));
        sym_apply_kernel<<<gr, 256, 0, s>>>((const double *)Rrep.ptr + roff[ri], (double *)Tm.ptr, n, F.ke, r,
                                            (const int *)pi.ptr, g, vec_in);
        FCUDA(cudaGetLastError());
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, k, r, N, &one, Vt, N, (const double *)Tm.ptr, N, &zero, Q,
                          k));
        // pi and Tm are reused by the next offset: keep the stream order (no host wait needed)
    }
    to_float_kernel<<<grid_for((long long)total), 256, 0, s>>>((const double *)F.m2l_p.ptr, (long long)total,
                                                              (float *)F.m2l_p32.ptr);
    to_float_kernel<<<grid_for((long long)total), 256, 0, s>>>((const double *)F.m2l_q.ptr, (long long)total,
                                                              (float *)F.m2l_q32.ptr);
    FCUDA(cudaGetLastError());
    FCUDA(cudaStreamSynchronize(s));
    return STK_OK;
}

// Build the level-independent operators for (m2x, p).
int build_operators(FarField &F, cudaStream_t s) {
    const int n = F.n, N = F.n * F.ke;
    if (F.kc != F.ke) return STK_ERR_NOT_SUPPORTED;
    std::vector<double> unit = unit_surface(F.p);
    const double r0 = 0.5;  // reference box: side 1, centred at 0
    DevBuf X, Y, K, T;
    int rc = K.reserve(sizeof(double) * (size_t)N * N);
    if (!rc) rc = T.reserve(sizeof(double) * (size_t)N * N);
    if (!rc) rc = F.uc2ue.reserve(sizeof(double) * (size_t)N * N);
    if (!rc) rc = F.dc2de.reserve(sizeof(double) * (size_t)N * N);
    if (!rc) rc = F.m2m.reserve(sizeof(double) * (size_t)N * N * 8);
    if (!rc) rc = F.l2l.reserve(sizeof(double) * (size_t)N * N * 8);
    if (rc) return rc;
    // relative SVD cut: sqrt of the unit roundoff 2^-53, as in the reference's
    // pinv (M2L/SVD_pvfmm.hpp:599-604)
    const double rtol = std::sqrt(std::ldexp(1.0, -53));
    auto kmat = [&](const std::vector<double> &trg, const std::vector<double> &src, double *M) {
        int r = upload_points(X, trg, s);
        if (!r) r = upload_points(Y, src, s);
        if (!r) r = kernel_matrix(F.m2x, (const double *)X.ptr, n, (const double *)Y.ptr, n, M, N, s);
        return r;
    };
    const double one = 1.0, zero = 0.0, half = 0.5;
    cublasSetStream(F.blas, s);
    // UC2UE and DC2DE
    rc = kmat(scaled_surface(unit, 0, 0, 0, kRad1 * r0), scaled_surface(unit, 0, 0, 0, kRad0 * r0), (double *)K.ptr);
    if (!rc) rc = pinv(F, (double *)K.ptr, N, (double *)F.uc2ue.ptr, rtol, s);
    if (!rc) rc = kmat(scaled_surface(unit, 0, 0, 0, kRad0 * r0), scaled_surface(unit, 0, 0, 0, kRad1 * r0), (double *)K.ptr);
    if (!rc) rc = pinv(F, (double *)K.ptr, N, (double *)F.dc2de.ptr, rtol, s);
    if (rc) return rc;
    // M2M and L2L per child octant (child centre at +-r0/2, half-width r0/2)
    for (int o = 0; o < 8; o++) {
        const double cx = (o & 1) ? r0 / 2 : -r0 / 2, cy = (o & 2) ? r0 / 2 : -r0 / 2, cz = (o & 4) ? r0 / 2 : -r0 / 2;
        rc = kmat(scaled_surface(unit, 0, 0, 0, kRad1 * r0), scaled_surface(unit, cx, cy, cz, kRad0 * r0 / 2),
                  (double *)K.ptr);
        if (rc) return rc;
        if (F.scaled) {
            // child densities are normalised one level deeper: component c carries 2^-den_exp[c] more
            CompF one4 = {{1, 1, 1, 1}}, fc;
            for (int c = 0; c < 4; c++) fc.v[c] = std::exp2(-F.den_exp[c]);
            scale_rc_kernel<<<grid_for((long long)N * N), 256, 0, s>>>((double *)K.ptr, N, N, N, F.ke, one4, fc);
            FCUDA(cudaGetLastError());
        }
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, N, N, N, &one, (const double *)F.uc2ue.ptr, N,
                          (const double *)K.ptr, N, &zero, (double *)F.m2m.ptr + (size_t)o * N * N, N));
        rc = kmat(scaled_surface(unit, cx, cy, cz, kRad0 * r0 / 2), scaled_surface(unit, 0, 0, 0, kRad1 * r0),
                  (double *)K.ptr);
        if (rc) return rc;
        if (F.scaled) {
            // child check potentials are normalised one level deeper: component a carries 2^-pot_exp[a] more
            CompF one4 = {{1, 1, 1, 1}}, fr;
            for (int a = 0; a < 4; a++) fr.v[a] = std::exp2(-F.pot_exp[a]);
            scale_rc_kernel<<<grid_for((long long)N * N), 256, 0, s>>>((double *)K.ptr, N, N, N, F.kc, fr, one4);
            FCUDA(cudaGetLastError());
        }
        // the child's DC2DE is half the parent's (degree -1 kernels); rows o N .. of the 8N x N stack
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, N, N, N, &half, (const double *)F.dc2de.ptr, N,
                          (const double *)K.ptr, N, &zero, (double *)F.l2l.ptr + (size_t)o * N, 8 * N));
    }
    // M2L for every well-separated offset d of a same-level source box, in the
    // compressed form  M2L_d = DC2DE U C_d V^T,  C_d = U^T A_d V,  A_d = K(DC, UE + d).
    // U spans the columns of [A_d ...] and V the rows of [A_d; ...], both cut at
    // the relative singular value m2l_rtol, so one M2L costs 2 k^2 flops per pair
    // instead of 2 N^2.
    F.m2l_slot.assign(kNumOffsets, -1);
    int nslot = 0;
    for (int code = 0; code < kNumOffsets; code++) {
        const int dx = code % 7 - 3, dy = (code / 7) % 7 - 3, dz = code / 49 - 3;
        if (std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz))) >= 2) F.m2l_slot[code] = nslot++;
    }
    auto offset_matrix = [&](int code, double *M, int ld) {
        const double dx = code % 7 - 3, dy = (code / 7) % 7 - 3, dz = code / 49 - 3;
        int r = upload_points(X, scaled_surface(unit, 0, 0, 0, kRad0 * r0), s);
        if (!r) r = upload_points(Y, scaled_surface(unit, dx, dy, dz, kRad0 * r0), s);
        if (!r) r = kernel_matrix(F.m2x, (const double *)X.ptr, n, (const double *)Y.ptr, n, M, ld, s);
        return r;
    };
    // the 316-offset stack is never formed: blockwise R-only QR (stack_svd), at most
    // STKFMM_M2L_QR_BUDGET_MB (default 2048) MB of work matrix
    DevBuf VTv, VTu, Sv, Su;
    rc = VTv.reserve(sizeof(double) * (size_t)N * N);
    if (!rc) rc = VTu.reserve(sizeof(double) * (size_t)N * N);
    if (!rc) rc = Sv.reserve(sizeof(double) * N);
    if (!rc) rc = Su.reserve(sizeof(double) * N);
    if (rc) return rc;
    const char *env_budget = getenv("STKFMM_M2L_QR_BUDGET_MB");
    const size_t budget = (size_t)(env_budget ? atof(env_budget) : 2048.0) << 20;
    std::vector<int> slot_code(nslot);
    for (int code = 0; code < kNumOffsets; code++)
        if (F.m2l_slot[code] >= 0) slot_code[F.m2l_slot[code]] = code;
    // rows of [A_d; ...] -> V
    rc = stack_svd(F, nslot, N, [&](int b, double *dst, long long ld) { return offset_matrix(slot_code[b], dst, (int)ld); },
                   (double *)Sv.ptr, (double *)VTv.ptr, s, budget);
    if (rc) return rc;
    // columns of [A_d ...] = rows of [A_d^T; ...] -> U
    rc = stack_svd(
        F, nslot, N,
        [&](int b, double *dst, long long ld) {
            int r = offset_matrix(slot_code[b], (double *)K.ptr, N);
            if (r) return r;
            if (cublasDgeam(F.blas, CUBLAS_OP_T, CUBLAS_OP_N, N, N, &one, (const double *)K.ptr, N, &zero,
                            (const double *)K.ptr, N, dst, (int)ld) != CUBLAS_STATUS_SUCCESS)
                return (int)STK_ERR_CUDA;
            return (int)STK_OK;
        },
        (double *)Su.ptr, (double *)VTu.ptr, s, budget);
    if (rc) return rc;
    std::vector<double> sv(N), su(N);
    FCUDA(cudaMemcpyAsync(sv.data(), Sv.ptr, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
    FCUDA(cudaMemcpyAsync(su.data(), Su.ptr, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
    FCUDA(cudaStreamSynchronize(s));
    int k = 1;
    for (int i = 0; i < N; i++)
        if (sv[i] > F.m2l_rtol * sv[0] || su[i] > F.m2l_rtol * su[0]) k = std::max(k, i + 1);
    F.m2l_rank = k;
    rc = F.m2l_vt.reserve(sizeof(double) * (size_t)k * N);
    if (!rc) rc = F.m2l_e.reserve(sizeof(double) * (size_t)N * k);
    if (rc) return rc;
    // V^T: the first k rows of VTv;  E = DC2DE U,  U^T = the first k rows of VTu
    FBLAS(cublasDgeam(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, k, N, &one, (const double *)VTv.ptr, N, &zero,
                      (const double *)VTv.ptr, N, (double *)F.m2l_vt.ptr, k));
    FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_T, N, k, N, &one, (const double *)F.dc2de.ptr, N,
                      (const double *)VTu.ptr, N, &zero, (double *)F.m2l_e.ptr, N));
    rc = build_m2l_lowrank(F, unit, (const double *)VTu.ptr, (const double *)VTv.ptr, offset_matrix, K, T, s);
    if (rc) return rc;
    FCUDA(cudaStreamSynchronize(s));
    return STK_OK;
}

// Periodic far-image operator of the root: m2c_op = DC2DE M2C (FP64), mapping
// the root's upward equivalent density to its downward one.  far_field = 0:
// only the ring of images up to two cells away (m2c_ring_kernel).
int build_periodic(FarField &F, int pbc, int far_field, cudaStream_t s) {
    const int n = F.n, N = F.n * F.ke;
    std::vector<double> unit = unit_surface(F.p);
    // the root: centre (0.5, 0.5, 0.5), half-width 0.5; its UE and DC surfaces coincide (RAD0)
    DevBuf X, M2C, W;
    int rc = upload_points(X, scaled_surface(unit, 0.5, 0.5, 0.5, kRad0 * 0.5), s);
    if (!rc) rc = M2C.reserve(sizeof(double) * (size_t)N * N);
    if (!rc) rc = F.m2c_op.reserve(sizeof(double) * (size_t)N * N);
    if (rc) return rc;
    const int grid = grid_for((long long)n * n);
    const double *Xp = (const double *)X.ptr;
    double *Mp = (double *)M2C.ptr;
    const double *shift = nullptr;
#define STK_M2C(UKV, P) m2c_kernel<UKV, P><<<grid, 128, 0, s>>>(Xp, n, Xp, n, Mp, N, shift)
#define STK_RING(UKV, P) m2c_ring_kernel<UKV, P><<<grid, 128, 0, s>>>(Xp, n, Xp, n, Mp, N)
    if (!far_field) {
        if (pbc < 1 || pbc > 3) return STK_ERR_NOT_SUPPORTED;
        if (F.m2x == UK_LAPLACE_P) {
            if (pbc == 1) STK_RING(UK_LAPLACE_P, 1);
            if (pbc == 2) STK_RING(UK_LAPLACE_P, 2);
            if (pbc == 3) STK_RING(UK_LAPLACE_P, 3);
        } else if (F.m2x == UK_STOKES_VEL) {
            if (pbc == 1) STK_RING(UK_STOKES_VEL, 1);
            if (pbc == 2) STK_RING(UK_STOKES_VEL, 2);
            if (pbc == 3) STK_RING(UK_STOKES_VEL, 3);
        } else if (F.m2x == UK_STOKES_PVEL) {
            if (pbc == 1) STK_RING(UK_STOKES_PVEL, 1);
            if (pbc == 2) STK_RING(UK_STOKES_PVEL, 2);
            if (pbc == 3) STK_RING(UK_STOKES_PVEL, 3);
        } else {
            return STK_ERR_NOT_SUPPORTED;
        }
    } else if (pbc == 3 && F.m2x == UK_LAPLACE_P) {
        rc = W.reserve(sizeof(double) * (size_t)n);
        if (rc) return rc;
        m2c_neutral_kernel<<<(n + 127) / 128, 128, 0, s>>>(Xp, n, (double *)W.ptr);
        shift = (const double *)W.ptr;
        STK_M2C(UK_LAPLACE_P, 3);
    } else if (pbc == 3 && F.m2x == UK_STOKES_VEL)
        STK_M2C(UK_STOKES_VEL, 3);
    else if (pbc == 3 && F.m2x == UK_STOKES_PVEL)
        STK_M2C(UK_STOKES_PVEL, 3);
    else if (pbc == 2 && F.m2x == UK_LAPLACE_P)
        STK_M2C(UK_LAPLACE_P, 2);
    else if (pbc == 2 && F.m2x == UK_STOKES_VEL)
        STK_M2C(UK_STOKES_VEL, 2);
    else if (pbc == 2 && F.m2x == UK_STOKES_PVEL)
        STK_M2C(UK_STOKES_PVEL, 2);
    else if (pbc == 1 && F.m2x == UK_LAPLACE_P)
        m2c_px_kernel<UK_LAPLACE_P><<<grid, 128, 0, s>>>(Xp, n, Xp, n, Mp, N);
    else if (pbc == 1 && F.m2x == UK_STOKES_VEL)
        m2c_px_kernel<UK_STOKES_VEL><<<grid, 128, 0, s>>>(Xp, n, Xp, n, Mp, N);
    else if (pbc == 1 && F.m2x == UK_STOKES_PVEL)
        m2c_px_kernel<UK_STOKES_PVEL><<<grid, 128, 0, s>>>(Xp, n, Xp, n, Mp, N);
    else
        return STK_ERR_NOT_SUPPORTED;
#undef STK_M2C
#undef STK_RING
    FCUDA(cudaGetLastError());
    const double one = 1.0, zero = 0.0;
    cublasSetStream(F.blas, s);
    FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, N, N, N, &one, (const double *)F.dc2de.ptr, N,
                      (const double *)M2C.ptr, N, &zero, (double *)F.m2c_op.ptr, N));
    FCUDA(cudaStreamSynchronize(s));
    F.m2c_p = F.p;
    F.m2c_m2x = F.m2x;
    F.m2c_pbc = pbc;
    F.m2c_ff = far_field;
    return STK_OK;
}

// Set up one list pass: target boxes with contiguous target ranges, list entries
// over source boxes.  src_beg / src_end are device arrays owned elsewhere when
// own_src is false.
int setup_pass(ListPass &P, int uk, const std::vector<int> &tb, const std::vector<int> &te,
               const std::vector<int> &off, const std::vector<int> &ent, const int *h_src_beg, const int *h_src_end,
               int n_src_box, bool own_src, const std::vector<double> &centres, int balance_warps, cudaStream_t s,
               int shard_rank = 0, int shard_n = 1) {
    P.uk = uk;
    std::vector<WorkItem> items;
    build_list_items((int)tb.size(), tb.data(), te.data(), off.data(), ent.data(), h_src_beg, h_src_end, items,
                     P.pairs, balance_warps, shard_rank, shard_n);
    P.n_items = (int)items.size();
    int rc = P.items.upload(items.data(), items.size() * sizeof(WorkItem), s);
    if (!rc) rc = P.ent.upload(ent.data(), ent.size() * sizeof(int), s);
    if (!rc && own_src) rc = P.src_beg.upload(h_src_beg, sizeof(int) * n_src_box, s);
    if (!rc && own_src) rc = P.src_end.upload(h_src_end, sizeof(int) * n_src_box, s);
    if (!rc) rc = P.trg_box_centre.upload(centres.data(), centres.size() * sizeof(double), s);
    return rc;
}

int run_pass(const ListPass &P, int prec, const double *rec, const int *src_beg, const int *src_end,
             const double *trg_xyz, double *out, unsigned int *counter, int sms, cudaStream_t s) {
    if (P.n_items == 0) return STK_OK;
    t_launches++;
    ListP2PArgs a{};
    a.src_rec = rec;
    a.src_box_begin = src_beg;
    a.src_box_end = src_end;
    a.list_ent = (const int *)P.ent.ptr;
    a.items = (const WorkItem *)P.items.ptr;
    a.n_items = P.n_items;
    a.counter = counter;
    a.trg_xyz = trg_xyz;
    a.trg_out = out;
    a.box_centre = (const double *)P.trg_box_centre.ptr;
    a.period = 1.0;
    a.atomic_out = 0;
    a.trg_aux = nullptr;
    return launch_list_p2p(P.uk, prec, a, sms, s) == cudaSuccess ? STK_OK : STK_ERR_CUDA;
}

}  // namespace

FarField::~FarField() {
    if (blas) cublasDestroy(blas);
    if (solver) cusolverDnDestroy(solver);
    if (built) cudaEventDestroy(built);
    for (int i = 0; i < 8; i++) {
        if (tc_stream[i]) cudaStreamDestroy(tc_stream[i]);
        if (tc_ev[i]) cudaEventDestroy(tc_ev[i]);
    }
    if (tc_fork) cudaEventDestroy(tc_fork);
}

// ---- process-wide operator cache -------------------------------------------
// The level-independent operators depend only on (translation kernel, p, M2L
// cut) and the periodic M2C in addition on (pbc, far field on/off); the
// reference loads both from precomputed files (Lib/src/FMMData.cpp:13-56) instead
// of rebuilding them per FMM object.  Here the first handle that needs an entry
// builds it on its device and every later handle on that device aliases its
// buffers (DevBuf::share): the wall's Laplace sub-FMMs, repeated handles of one
// configuration.  Entries live while a handle holds them.
namespace {

struct OpsKey {
    int dev, m2x, p, pbc, ff;
    double rtol;
    bool operator<(const OpsKey &o) const {
        return std::tie(dev, m2x, p, pbc, ff, rtol) < std::tie(o.dev, o.m2x, o.p, o.pbc, o.ff, o.rtol);
    }
};
std::mutex g_ops_mu;
std::map<OpsKey, std::weak_ptr<FarField>> g_ops, g_m2c;

std::shared_ptr<FarField> cache_find(std::map<OpsKey, std::weak_ptr<FarField>> &m, const OpsKey &k) {
    std::lock_guard<std::mutex> lock(g_ops_mu);
    auto it = m.find(k);
    if (it == m.end()) return nullptr;
    auto sp = it->second.lock();
    if (!sp) m.erase(it);
    return sp;
}

void cache_put(std::map<OpsKey, std::weak_ptr<FarField>> &m, const OpsKey &k, const std::shared_ptr<FarField> &e) {
    std::lock_guard<std::mutex> lock(g_ops_mu);
    m[k] = e;
}

// dst aliases src's level-independent operators
void share_operators(FarField &dst, const FarField &src) {
    dst.m2l_rank = src.m2l_rank;
    dst.m2l_r = src.m2l_r;
    dst.m2l_rt = src.m2l_rt;
    dst.m2l_pq_off = src.m2l_pq_off;
    dst.m2l_rmax = src.m2l_rmax;
    dst.m2l_slot = src.m2l_slot;
    dst.uc2ue.share(src.uc2ue);
    dst.dc2de.share(src.dc2de);
    dst.m2m.share(src.m2m);
    dst.l2l.share(src.l2l);
    dst.m2l_p.share(src.m2l_p);
    dst.m2l_q.share(src.m2l_q);
    dst.m2l_p32.share(src.m2l_p32);
    dst.m2l_q32.share(src.m2l_q32);
    dst.m2l_vt.share(src.m2l_vt);
    dst.m2l_e.share(src.m2l_e);
}

// an event recorded on s after the work queued so far (the entry's build)
int record_built(FarField &e, cudaStream_t s) {
    if (!e.built && cudaEventCreateWithFlags(&e.built, cudaEventDisableTiming) != cudaSuccess) return STK_ERR_CUDA;
    return cudaEventRecord(e.built, s) == cudaSuccess ? STK_OK : STK_ERR_CUDA;
}

}  // namespace

// Tensor-core operands and tile tables of the mixed path's chunked M2L (the levels the
// dense M2L does not take).  Per group of column chunks two grouped GEMM launches:
//   stage 1  Z_c = Q_d^T X_c (r_d x 256 per chunk c of offset d), written split into
//            TF32 hi / lo parts as the next stage's K-major operand (rows of rmax);
//   stage 2  Y_c = P_d Z_c (k x 256), FP32, reduced per target as on the SIMT path.
// Every tile is 128 x 128 (rows of the factor x columns of the chunk) over the whole K.
// The operands (~8 (sum_d r_d k + nslot k rmax) bytes) must fit in 4 GiB, else the
// SIMT path stays; STKFMM_M2L_TC=0 turns both tensor-core paths off.
static int setup_m2l_chunks_tc(FarField &F, const std::vector<int> &chunk_slot, int nslot, cudaStream_t s) {
    F.tcc = false;
    const char *env_tc = getenv("STKFMM_M2L_TC");
    if ((env_tc && env_tc[0] == '0') || !umma_available() || F.m2l_chunks == 0) return STK_OK;
    const int k = F.m2l_rank, k4 = (k + 3) / 4 * 4, rmax = F.m2l_rmax;
    if (rmax % 4) return STK_OK;  // ranks are padded to multiples of 32
    long long qrows = 0;
    for (int sl = 0; sl < nslot; sl++) qrows += F.m2l_r[sl];
    const size_t bytes = 8 * ((size_t)qrows * k4 + (size_t)nslot * k * rmax);
    if (bytes > (4ull << 30)) return STK_OK;
    int rc = F.tcc_q_hi.reserve(sizeof(float) * (size_t)qrows * k4);
    if (!rc) rc = F.tcc_q_lo.reserve(sizeof(float) * (size_t)qrows * k4);
    if (!rc) rc = F.tcc_pt_hi.reserve(sizeof(float) * (size_t)nslot * k * rmax);
    if (!rc) rc = F.tcc_pt_lo.reserve(sizeof(float) * (size_t)nslot * k * rmax);
    if (!rc && !F.tc_err.ptr) rc = F.tc_err.reserve(sizeof(int) * 4);
    if (rc) return rc;
    // Q_d (k x r_d column-major, offsets back to back) read as qrows K-major rows of k
    tc_rows_kernel<<<grid_for(qrows * k4), 256, 0, s>>>((const double *)F.m2l_q.ptr, k, qrows, k4,
                                                        (float *)F.tcc_q_hi.ptr, (float *)F.tcc_q_lo.ptr);
    FCUDA(cudaGetLastError());
    for (int sl = 0; sl < nslot; sl++) {
        tc_trows_kernel<<<grid_for((long long)k * rmax), 256, 0, s>>>(
            (const double *)F.m2l_p.ptr + F.m2l_pq_off[sl], k, F.m2l_r[sl], rmax,
            (float *)F.tcc_pt_hi.ptr + (size_t)sl * k * rmax, (float *)F.tcc_pt_lo.ptr + (size_t)sl * k * rmax);
        FCUDA(cudaGetLastError());
    }
    FCUDA(cudaMemsetAsync(F.tc_err.ptr, 0, sizeof(int) * 4, s));
    // tile tables, group by group
    const int nc = F.m2l_chunks, gc = F.m2l_group_chunks, ngroups = (nc + gc - 1) / gc;
    std::vector<GroupTile> t1, t2;
    F.tcc_t1_off.assign(ngroups + 1, 0);
    F.tcc_t2_off.assign(ngroups + 1, 0);
    for (int g = 0; g < ngroups; g++) {
        F.tcc_t1_off[g] = (int)t1.size();
        F.tcc_t2_off[g] = (int)t2.size();
        for (int c = g * gc; c < std::min(nc, (g + 1) * gc); c++) {
            const int sl = chunk_slot[c], r = F.m2l_r[sl];
            const long long col = (long long)(c - g * gc) * kM2LChunk;  // first column within the group
            const int qrow0 = (int)(F.m2l_pq_off[sl] / (size_t)k);
            for (int nt = 0; nt < kM2LChunk / 128; nt++) {
                const long long cn = col + 128LL * nt;
                for (int m0 = 0; m0 < r; m0 += 128) {
                    const int mv = std::min(128, r - m0);
                    t1.push_back(GroupTile{qrow0 + m0, (int)cn, k, mv, mv, 128, rmax, 0, cn * rmax + m0});
                }
                for (int m0 = 0; m0 < k; m0 += 128) {
                    const int mv = std::min(128, k - m0);
                    t2.push_back(GroupTile{sl * k + m0, (int)cn, r, mv, mv, 128, k, 0, cn * k + m0});
                }
            }
        }
    }
    F.tcc_t1_off[ngroups] = (int)t1.size();
    F.tcc_t2_off[ngroups] = (int)t2.size();
    rc = F.tcc_tiles1.upload(t1.data(), sizeof(GroupTile) * t1.size(), s);
    if (!rc) rc = F.tcc_tiles2.upload(t2.data(), sizeof(GroupTile) * t2.size(), s);
    if (rc) return rc;
    F.tcc_q_rows = qrows;
    F.tcc = true;
    return STK_OK;
}

// Dense M2L of the complete levels (M2LDenseLevel).  A level l >= 4 qualifies
// when all 8^l boxes are present and its V lists hold at least 70% of 189 pairs
// per box (periodic and deep uniform levels); the stacked factors and the work
// buffers must fit in budgets (4 GiB each).  Smaller levels (<= 512 boxes, under
// 1e5 pairs) stay on the chunked path, so small trees build no stacked factors.
// STKFMM_M2L_DENSE=0 turns it off.
static int setup_m2l_dense(FarField &F, const Octree &T, int nslot, cudaStream_t s) {
    F.dense.clear();
    const char *env = getenv("STKFMM_M2L_DENSE");
    if (env && env[0] == '0') return STK_OK;
    const int k = F.m2l_rank;
    auto type_of = [&](int b) { return (int)((T.ix[b] & 1) | (T.iy[b] & 1) << 1 | (T.iz[b] & 1) << 2); };
    auto slot_of = [&](int b, int ent) {
        const int a = ent >> 5, code = ent & 31;
        const int sx = code % 3 - 1, sy = (code / 3) % 3 - 1, sz = code / 9 - 1;
        const int64_t L = 1LL << T.level[b];
        const int dx = (int)((int64_t)T.ix[a] + sx * L - T.ix[b]);
        const int dy = (int)((int64_t)T.iy[a] + sy * L - T.iy[b]);
        const int dz = (int)((int64_t)T.iz[a] + sz * L - T.iz[b]);
        if (std::abs(dx) > 3 || std::abs(dy) > 3 || std::abs(dz) > 3) return -1;
        return F.m2l_slot[(dx + 3) + 7 * (dy + 3) + 49 * (dz + 3)];
    };
    // candidate levels
    std::vector<int> levels;
    for (int l = 4; l <= T.depth() && l < 10; l++) {
        const long long n = (long long)T.level_begin[l + 1] - T.level_begin[l];
        if (n != (1LL << (3 * l))) continue;
        long long pairs = 0;
        for (int b = T.level_begin[l]; b < T.level_begin[l + 1]; b++) pairs += T.V.off[b + 1] - T.V.off[b];
        if (pairs >= 0.7 * 189.0 * (double)n) levels.push_back(l);
    }
    if (levels.empty()) return STK_OK;
    // offsets per (target type, source type), one pair per (target, offset)
    std::vector<char> in((size_t)64 * nslot, 0);
    std::vector<int> stamp(nslot, -1);
    for (int l : levels)
        for (int b = T.level_begin[l]; b < T.level_begin[l + 1]; b++)
            for (int e = T.V.off[b]; e < T.V.off[b + 1]; e++) {
                const int sl = slot_of(b, T.V.ent[e]);
                if (sl < 0 || stamp[sl] == b) return STK_OK;  // not the expected structure: chunked path
                stamp[sl] = b;
                in[(size_t)(8 * type_of(b) + type_of(T.V.ent[e] >> 5)) * nslot + sl] = 1;
            }
    // rows: blocks (c, c') of Pv_c in c' order; Qs_c' rows in slot order
    std::vector<int> rows_s((size_t)8 * nslot, -1);
    for (int cs = 0; cs < 8; cs++) {
        int r = 0;
        for (int sl = 0; sl < nslot; sl++) {
            bool used = false;
            for (int c = 0; c < 8; c++) used = used || in[(size_t)(8 * c + cs) * nslot + sl];
            if (!used) continue;
            rows_s[(size_t)cs * nslot + sl] = r;
            r += F.m2l_rt[sl];
        }
        F.dn_rs[cs] = r;
    }
    size_t ops = 0, rows_total = 0;
    for (int c = 0; c < 8; c++) {
        int r = 0;
        for (int cs = 0; cs < 8; cs++) {
            const int b = 8 * c + cs;
            F.dn_slots[b].clear();
            F.dn_pstart[b] = r;
            int rb = 0;
            for (int sl = 0; sl < nslot; sl++)
                if (in[(size_t)b * nslot + sl]) {
                    F.dn_slots[b].push_back(sl);
                    rb += F.m2l_rt[sl];
                }
            F.dn_q[b] = (int)F.dn_slots[b].size();
            F.dn_rcc[b] = rb;
            r += rb;
        }
        F.dn_rv[c] = r;
        ops += (size_t)k * (F.dn_rv[c] + F.dn_rs[c]);
        rows_total += r;
    }
    // budgets: stacked factors (FP64 + FP32) and the largest level's buffers (FP64)
    int rs_max = 1, rcc_max = 1;
    for (int c = 0; c < 8; c++) rs_max = std::max(rs_max, F.dn_rs[c]);
    for (int b = 0; b < 64; b++) rcc_max = std::max(rcc_max, F.dn_rcc[b]);
    const long long nmax = 1LL << (3 * levels.back()), n8max = nmax / 8;
    const size_t buf = sizeof(double) * ((size_t)2 * k * nmax + (size_t)(rs_max + rcc_max) * n8max);
    if (ops * 12 > (4ull << 30) || buf > (4ull << 30)) return STK_OK;

    // stacked factors
    int rc = F.dn_pv.reserve(sizeof(double) * (size_t)k * rows_total);
    size_t qs_total = 0;
    for (int c = 0; c < 8; c++) qs_total += F.dn_rs[c];
    if (!rc) rc = F.dn_qs.reserve(sizeof(double) * (size_t)k * std::max<size_t>(qs_total, 1));
    if (!rc) rc = F.dn_pv32.reserve(sizeof(float) * (size_t)k * rows_total);
    if (!rc) rc = F.dn_qs32.reserve(sizeof(float) * (size_t)k * std::max<size_t>(qs_total, 1));
    if (rc) return rc;
    size_t off = 0;
    for (int c = 0; c < 8; c++) {
        F.dn_pv_off[c] = off;
        for (int cs = 0; cs < 8; cs++)
            for (int sl : F.dn_slots[8 * c + cs]) {
                const size_t bytes = sizeof(double) * (size_t)k * F.m2l_rt[sl];
                FCUDA(cudaMemcpyAsync((double *)F.dn_pv.ptr + off, (const double *)F.m2l_p.ptr + F.m2l_pq_off[sl],
                                      bytes, cudaMemcpyDeviceToDevice, s));
                off += (size_t)k * F.m2l_rt[sl];
            }
    }
    off = 0;
    for (int cs = 0; cs < 8; cs++) {
        F.dn_qs_off[cs] = off;
        for (int sl = 0; sl < nslot; sl++) {
            if (rows_s[(size_t)cs * nslot + sl] < 0) continue;
            FCUDA(cudaMemcpyAsync((double *)F.dn_qs.ptr + off, (const double *)F.m2l_q.ptr + F.m2l_pq_off[sl],
                                  sizeof(double) * (size_t)k * F.m2l_rt[sl], cudaMemcpyDeviceToDevice, s));
            off += (size_t)k * F.m2l_rt[sl];
        }
    }
    to_float_kernel<<<grid_for((long long)k * rows_total), 256, 0, s>>>((const double *)F.dn_pv.ptr,
                                                                         (long long)k * rows_total,
                                                                         (float *)F.dn_pv32.ptr);
    to_float_kernel<<<grid_for((long long)k * qs_total), 256, 0, s>>>((const double *)F.dn_qs.ptr,
                                                                       (long long)k * qs_total,
                                                                       (float *)F.dn_qs32.ptr);
    FCUDA(cudaGetLastError());
    // tensor-core operands of the mixed path (3xTF32 hi / lo, K-major rows of a multiple
    // of 4 floats): Qs_c'^T per source type and Pv_{c,c'}^T per block, within 4 GiB
    F.tc = false;
    const char *env_tc = getenv("STKFMM_M2L_TC");
    if (!(env_tc && env_tc[0] == '0') && umma_available()) {
        const int k4 = (k + 3) / 4 * 4;
        size_t qa = 0, pa = 0;
        for (int cs = 0; cs < 8; cs++) {
            F.tc_qa_off[cs] = qa;
            qa += (size_t)F.dn_rs[cs] * k4;
        }
        for (int c = 0; c < 8; c++) {
            F.tc_pa_off[c] = pa;
            pa += (size_t)k * ((F.dn_rv[c] + 3) / 4 * 4);
        }
        if ((qa + pa) * 8 <= (4ull << 30)) {
            rc = F.tc_qa_hi.reserve(sizeof(float) * std::max<size_t>(qa, 4));
            if (!rc) rc = F.tc_qa_lo.reserve(sizeof(float) * std::max<size_t>(qa, 4));
            if (!rc) rc = F.tc_pa_hi.reserve(sizeof(float) * std::max<size_t>(pa, 4));
            if (!rc) rc = F.tc_pa_lo.reserve(sizeof(float) * std::max<size_t>(pa, 4));
            if (!rc) rc = F.tc_err.reserve(sizeof(int) * 4);
            if (rc) return rc;
            for (int cs = 0; cs < 8; cs++)
                if (F.dn_rs[cs])
                    tc_rows_kernel<<<grid_for((long long)F.dn_rs[cs] * k4), 256, 0, s>>>(
                        (const double *)F.dn_qs.ptr + F.dn_qs_off[cs], k, F.dn_rs[cs], k4,
                        (float *)F.tc_qa_hi.ptr + F.tc_qa_off[cs], (float *)F.tc_qa_lo.ptr + F.tc_qa_off[cs]);
            for (int c = 0; c < 8; c++)
                if (F.dn_rv[c])
                    tc_trows_kernel<<<grid_for((long long)k * F.dn_rv[c]), 256, 0, s>>>(
                        (const double *)F.dn_pv.ptr + F.dn_pv_off[c], k, F.dn_rv[c], (F.dn_rv[c] + 3) / 4 * 4,
                        (float *)F.tc_pa_hi.ptr + F.tc_pa_off[c], (float *)F.tc_pa_lo.ptr + F.tc_pa_off[c]);
            FCUDA(cudaGetLastError());
            FCUDA(cudaMemsetAsync(F.tc_err.ptr, 0, sizeof(int) * 4, s));
            F.tc = true;
        }
    }
    // per block row: its slot index and its row in Z_c'
    std::vector<int> rowq, srow;
    for (int b = 0; b < 64; b++) {
        F.dn_row_off[b] = rowq.size();
        const int cs = b % 8;
        for (int q = 0; q < F.dn_q[b]; q++) {
            const int sl = F.dn_slots[b][q];
            for (int i = 0; i < F.m2l_rt[sl]; i++) {
                rowq.push_back(q);
                srow.push_back(rows_s[(size_t)cs * nslot + sl] + i);
            }
        }
    }
    rc = F.dn_rowq.upload(rowq.data(), sizeof(int) * rowq.size(), s);
    if (!rc) rc = F.dn_srow.upload(srow.data(), sizeof(int) * srow.size(), s);
    if (rc) return rc;
    // per level: nodes in type order and the (c, c') source tables
    std::vector<int> qidx((size_t)64 * nslot, -1);
    for (int b = 0; b < 64; b++)
        for (int q = 0; q < F.dn_q[b]; q++) qidx[(size_t)b * nslot + F.dn_slots[b][q]] = q;
    for (int l : levels) {
        std::unique_ptr<M2LDenseLevel> D(new M2LDenseLevel());
        D->level = l;
        const int b0 = T.level_begin[l], n = T.level_begin[l + 1] - b0, n8 = n / 8;
        D->n8 = n8;
        std::vector<int> nodes, pos(n, -1), cnt(8, 0);
        nodes.reserve(n);
        for (int c = 0; c < 8; c++)
            for (int b = b0; b < b0 + n; b++)
                if (type_of(b) == c) {
                    pos[b - b0] = cnt[c]++;
                    nodes.push_back(b);
                }
        for (int c = 0; c < 8; c++)
            if (cnt[c] != n8) return STK_ERR_STATE;
        D->tab_off.assign(64, 0);
        size_t tsize = 0;
        for (int b = 0; b < 64; b++) {
            D->tab_off[b] = tsize;
            tsize += (size_t)n8 * F.dn_q[b];
        }
        std::vector<int> tab(std::max<size_t>(tsize, 1), -1);
        for (int t = b0; t < b0 + n; t++)
            for (int e = T.V.off[t]; e < T.V.off[t + 1]; e++) {
                const int a = T.V.ent[e] >> 5, sl = slot_of(t, T.V.ent[e]);
                const int b = 8 * type_of(t) + type_of(a);
                const int q = qidx[(size_t)b * nslot + sl];
                if (q < 0 || a < b0 || a >= b0 + n) return STK_ERR_STATE;
                tab[D->tab_off[b] + (size_t)pos[t - b0] * F.dn_q[b] + q] = pos[a - b0];
                D->pairs++;
            }
        rc = D->d_nodes.upload(nodes.data(), sizeof(int) * nodes.size(), s);
        if (!rc) rc = D->d_tab.upload(tab.data(), sizeof(int) * tab.size(), s);
        if (rc) return rc;
        F.dense.push_back(std::move(D));
    }
    // work buffers (FP64 size, FP32 views)
    rc = F.dn_phi.reserve(sizeof(double) * (size_t)k * nmax);
    if (!rc) rc = F.dn_psi.reserve(sizeof(double) * (size_t)k * nmax);
    if (!rc) rc = F.dn_z.reserve(sizeof(double) * (size_t)rs_max * n8max);
    if (!rc) rc = F.dn_zc.reserve(sizeof(double) * (size_t)rcc_max * n8max);
    if (!rc && F.tc) {
        // tensor-core work per level: phi operands (nmax rows of k4), the Z of all source types
        // (sum_c' rs_c' x n8max), and one concatenated Zc operand (n8max rows of ceil4(rv_max))
        // per concurrent target-type stream, within 16 GiB (fewer streams, else the SIMT path)
        const size_t k4 = (size_t)(k + 3) / 4 * 4;
        int rv_max = 1;
        size_t rs_sum = 0;
        for (int c = 0; c < 8; c++) {
            rv_max = std::max(rv_max, F.dn_rv[c]);
            rs_sum += F.dn_rs[c];
        }
        const size_t r4 = (size_t)(rv_max + 3) / 4 * 4;
        const size_t fixed = sizeof(float) * (2 * k4 * nmax + rs_sum * n8max);
        const size_t per_stream = sizeof(float) * 2 * r4 * n8max;
        F.tc_streams = 0;
        for (int ns = 8; ns >= 1 && !F.tc_streams; ns /= 2)
            if (fixed + ns * per_stream <= (16ull << 30)) F.tc_streams = ns;
        if (!F.tc_streams) {
            F.tc = false;
        } else {
            F.tc_zc_ld = (int)r4;
            rc = F.tc_b_hi.reserve(sizeof(float) * k4 * nmax);
            if (!rc) rc = F.tc_b_lo.reserve(sizeof(float) * k4 * nmax);
            if (!rc) rc = F.tc_z.reserve(sizeof(float) * std::max<size_t>(rs_sum * n8max, 4));
            if (!rc) rc = F.tc_zc_hi.reserve(per_stream / 2 * F.tc_streams);
            if (!rc) rc = F.tc_zc_lo.reserve(per_stream / 2 * F.tc_streams);
            for (int i = 0; i < F.tc_streams && !rc; i++) {
                if (!F.tc_stream[i] && cudaStreamCreateWithFlags(&F.tc_stream[i], cudaStreamNonBlocking) != cudaSuccess)
                    rc = STK_ERR_CUDA;
                if (!F.tc_ev[i] && cudaEventCreateWithFlags(&F.tc_ev[i], cudaEventDisableTiming) != cudaSuccess)
                    rc = STK_ERR_CUDA;
            }
            if (!F.tc_fork && cudaEventCreateWithFlags(&F.tc_fork, cudaEventDisableTiming) != cudaSuccess) rc = STK_ERR_CUDA;
        }
    }
    if (rc) return rc;
    FCUDA(cudaStreamSynchronize(s));
    return STK_OK;
}

int farfield_setup(Stk3DFMM *f, KernelData *kd) {
    const KernelInfo *ki = kd->info;
    // free space, or periodic in x (PX), x and y (PXY) or all axes (PXYZ): the far
    // images through the root's M2C operator
    const int m2x = ki->slot[SLOT_M2X];
    if (m2x != UK_LAPLACE_P && m2x != UK_STOKES_VEL && m2x != UK_STOKES_PVEL) return STK_ERR_NOT_SUPPORTED;

    if (!kd->far) kd->far.reset(new FarField());
    FarField &F = *kd->far;
    cudaStream_t s = f->stream;
    F.ready = false;
    if (!F.blas && cublasCreate(&F.blas) != CUBLAS_STATUS_SUCCESS) return STK_ERR_CUDA;
    if (!F.solver && cusolverDnCreate(&F.solver) != CUSOLVER_STATUS_SUCCESS) return STK_ERR_CUDA;
    const int p = f->mult_order;
    const int ke = uk_sdim_host(m2x), kc = uk_tdim_host(m2x);
    int rc = STK_OK;
    // relative singular-value cut of the compressed M2L (environment override for studies)
    const char *env_rtol = getenv("STKFMM_M2L_RTOL");
    // The cut follows the order's own truncation error: at p <= 8 (FMM error
    // ~1e-6) 3e-8 changes the error by under 1% (RPY / Stokes, 32k-200k points)
    // and drops the rank 716 -> 636 for stokes_vel; at p = 9, 10 (error ~1e-8
    // for Laplace) 1e-8 keeps it within 15%; at p = 11, 12 (error ~1e-9 for
    // PVel and Laplace) 1e-9 changes it by under 1%; higher orders keep more rank.
    const double m2l_rtol = env_rtol ? atof(env_rtol) : (p <= 8 ? 3e-8 : p <= 10 ? 1e-8 : p <= 12 ? 1e-9 : 1e-10);
    if (F.p != p || F.m2x != m2x || F.m2l_rtol != m2l_rtol) {
        F.m2l_rtol = m2l_rtol;
        for (int c = 0; c < 4; c++) F.pot_exp[c] = F.den_exp[c] = 0.0;
        F.scaled = m2x == UK_STOKES_PVEL;
        if (F.scaled) {
            F.pot_exp[0] = 1.0;  // pressure
            F.den_exp[3] = 1.0;  // trD
        }
        F.p = p;
        F.n = 6 * (p - 1) * (p - 1) + 2;
        F.ke = ke;
        F.kc = kc;
        F.m2x = m2x;
        int dev = 0;
        cudaGetDevice(&dev);
        const OpsKey key{dev, m2x, p, 0, 0, m2l_rtol};
        std::shared_ptr<FarField> e = cache_find(g_ops, key);
        if (e) {
            share_operators(F, *e);
            if (e->built && cudaStreamWaitEvent(s, e->built, 0) != cudaSuccess) return STK_ERR_CUDA;
        } else {
            rc = build_operators(F, s);
            if (rc) {
                F.p = 0;
                return rc;
            }
            e = std::make_shared<FarField>();
            share_operators(*e, F);
            if ((rc = record_built(*e, s))) return rc;
            cache_put(g_ops, key, e);
        }
        F.ops_ref = e;
        F.m2c_p = 0;  // the periodic operator follows the (possibly new) operators
    }
    F.periodic = f->pbc >= 1;
    const int far_field = f->enable_ff ? 1 : 0;
    if (F.periodic && (F.m2c_p != F.p || F.m2c_m2x != F.m2x || F.m2c_pbc != f->pbc || F.m2c_ff != far_field)) {
        int dev = 0;
        cudaGetDevice(&dev);
        const OpsKey key{dev, F.m2x, F.p, f->pbc, far_field, F.m2l_rtol};
        std::shared_ptr<FarField> e = cache_find(g_m2c, key);
        if (e) {
            F.m2c_op.share(e->m2c_op);
            F.m2c_p = F.p;
            F.m2c_m2x = F.m2x;
            F.m2c_pbc = f->pbc;
            F.m2c_ff = far_field;
            if (e->built && cudaStreamWaitEvent(s, e->built, 0) != cudaSuccess) return STK_ERR_CUDA;
        } else {
            rc = build_periodic(F, f->pbc, far_field, s);
            if (rc) return rc;
            e = std::make_shared<FarField>();
            e->m2c_op.share(F.m2c_op);
            if ((rc = record_built(*e, s))) return rc;
            cache_put(g_m2c, key, e);
        }
        F.m2c_ref = e;
    }
    const Octree &T = kd->tree;
    const int nn = T.num_nodes(), n = F.n, N = n * ke;
    std::vector<double> unit = unit_surface(p);
    rc = upload_points(F.unit_surf, unit, s);
    // node levels and centres on the device
    std::vector<int> lev(T.level.begin(), T.level.end());
    DevBuf &d_level = F.d_level;
    if (!rc) rc = d_level.upload(lev.data(), lev.size() * sizeof(int), s);
    const double *centre = (const double *)kd->d_centre.ptr;
    // every node's upward-equivalent and downward-equivalent surface
    if (!rc) rc = F.ue_xyz.reserve(sizeof(double) * 3 * (size_t)nn * n);
    if (!rc) rc = F.de_xyz.reserve(sizeof(double) * 3 * (size_t)nn * n);
    if (rc) return rc;
    surface_points_kernel<<<grid_for((long long)nn * n), 256, 0, s>>>(nullptr, nn, centre, (const int *)d_level.ptr,
                                                                      kRad0, (const double *)F.unit_surf.ptr, n,
                                                                      (double *)F.ue_xyz.ptr);
    surface_points_kernel<<<grid_for((long long)nn * n), 256, 0, s>>>(nullptr, nn, centre, (const int *)d_level.ptr,
                                                                      kRad1, (const double *)F.unit_surf.ptr, n,
                                                                      (double *)F.de_xyz.ptr);
    FCUDA(cudaGetLastError());
    rc = F.phi.reserve(sizeof(double) * (size_t)nn * N);
    if (!rc) rc = F.psi.reserve(sizeof(double) * (size_t)nn * N);
    if (!rc) rc = F.phi_hat.reserve(sizeof(double) * (size_t)nn * F.m2l_rank);
    if (!rc) rc = F.psi_hat.reserve(sizeof(double) * (size_t)nn * F.m2l_rank);
    if (rc) return rc;

    auto by_level = [&](std::vector<int> &nodes, std::vector<int> &off) {
        std::stable_sort(nodes.begin(), nodes.end(), [&](int a, int b) { return T.level[a] < T.level[b]; });
        off.assign(T.depth() + 2, 0);
        for (int b : nodes) off[T.level[b] + 1]++;
        for (int l = 0; l <= T.depth(); l++) off[l + 1] += off[l];
    };
    std::vector<double> ctr(3 * (size_t)nn);
    for (int i = 0; i < nn; i++) T.centre(i, &ctr[3 * (size_t)i]);
    const int bw = f->sms * 12;  // resident warps of the list kernel, roughly

    // SL and DL at the same points (the near field's fused case): the check
    // potentials of S2M / S2L come from one pass over records carrying both
    F.fused_src = kd->fused && (ki->id == STK_LapPGrad || ki->id == STK_PVel);
    F.fused_check_uk = ki->id == STK_LapPGrad ? UK_LAPLACE_SLDL_P : UK_STOKES_SLDL_PVEL;

    // far field split over the shard group (Stk3DFMM_set_allreduce): M2L / S2L by target node
    F.split = f->shard_n > 1 && f->allreduce != nullptr;
    for (int c = 0; c < 8; c++) F.dn_own[c] = !F.split || c % f->shard_n == f->shard_rank;

    // ---- S2M: leaves with sources; targets = their upward check surfaces ----
    F.s2m_nodes.clear();
    for (int b : T.leaves)
        if (T.src_count(b) > 0) F.s2m_nodes.push_back(b);
    by_level(F.s2m_nodes, F.s2m_level_off);
    const int ms = (int)F.s2m_nodes.size();
    rc = F.d_s2m_nodes.upload(F.s2m_nodes.data(), sizeof(int) * ms, s);
    if (!rc) rc = F.uc_xyz.reserve(sizeof(double) * 3 * (size_t)std::max(ms, 1) * n);
    if (!rc) rc = F.check.reserve(sizeof(double) * (size_t)std::max(ms, 1) * n * kc);
    if (rc) return rc;
    if (ms)
        surface_points_kernel<<<grid_for((long long)ms * n), 256, 0, s>>>(
            (const int *)F.d_s2m_nodes.ptr, ms, centre, (const int *)d_level.ptr, kRad1,
            (const double *)F.unit_surf.ptr, n, (double *)F.uc_xyz.ptr);
    {
        std::vector<int> tb(ms), te(ms), off(ms + 1), ent(ms);
        std::vector<double> cc(3 * (size_t)std::max(ms, 1));
        for (int i = 0; i < ms; i++) {
            tb[i] = i * n;
            te[i] = (i + 1) * n;
            off[i] = i;
            ent[i] = (F.s2m_nodes[i] << 5) | kShiftNone;
            for (int d = 0; d < 3; d++) cc[3 * i + d] = ctr[3 * (size_t)F.s2m_nodes[i] + d];
        }
        off[ms] = ms;
        for (int k = 0; k < 2; k++) {
            // SL and DL at the same points: one fused pass (its records carry both)
            const int uk = F.fused_src ? (k == 0 ? F.fused_check_uk : -1) : ki->slot[k == 0 ? SLOT_S2M_SL : SLOT_S2M_DL];
            F.s2m[k].reset();
            if (uk < 0 || T.sets[k].n == 0) continue;
            rc = setup_pass(F.s2m[k], uk, tb, te, off, ent, T.sets[k].node_begin.data(), T.sets[k].node_end.data(),
                            nn, false, cc, bw, s);
            if (rc) return rc;
        }
    }

    // W- and X-list interactions whose point count is at most the surface size
    // are cheaper, and exact, as direct source-to-target pairs: a W-list source
    // node with few sources, an X-list target node with few targets.  They join
    // the U list in the near-field pass of the FMM.
    // (with SL and DL at the same points one fused pass covers both sets)
    auto w_direct = [&](int a) {
        const int c0 = T.sets[0].count(a), c1 = T.sets[1].count(a);
        return (kd->fused ? std::max(c0, c1) : c0 + c1) <= n;
    };
    auto x_direct = [&](int c) { return T.trg_count(c) <= n; };

    // ---- near field of the FMM: U list + direct W / X entries, per target leaf ----
    {
        const PointSet &tg = T.sets[2];
        std::vector<int> noff(nn + 1, 0), nent;
        for (int b = 0; b < nn; b++) {
            noff[b] = (int)nent.size();
            if (!T.is_leaf(b) || tg.count(b) == 0) continue;
            for (int e = T.U.off[b]; e < T.U.off[b + 1]; e++) nent.push_back(T.U.ent[e]);
            for (int e = T.W.off[b]; e < T.W.off[b + 1]; e++)
                if (w_direct(T.W.ent[e] >> 5)) nent.push_back(T.W.ent[e]);
            for (int c = b; c >= 0; c = T.parent[c])
                if (x_direct(c))
                    for (int e = T.X.off[c]; e < T.X.off[c + 1]; e++) nent.push_back(T.X.ent[e]);
        }
        noff[nn] = (int)nent.size();
        for (int k = 0; k < 2; k++) {
            F.near[k].reset();
            if (T.sets[k].n == 0 || ki->slot[k == 0 ? SLOT_S2T_SL : SLOT_S2T_DL] < 0) continue;
            rc = setup_pass(F.near[k], ki->slot[k == 0 ? SLOT_S2T_SL : SLOT_S2T_DL], tg.node_begin, tg.node_end, noff,
                            nent, T.sets[k].node_begin.data(), T.sets[k].node_end.data(), nn, false, ctr, bw, s,
                            f->shard_rank, f->shard_n);
            if (rc) return rc;
        }
    }

    // ---- S2L: nodes with X lists; targets = their downward check surfaces ----
    F.s2l_nodes.clear();
    for (int b = 0; b < nn; b++)
        if (T.X.off[b + 1] > T.X.off[b] && !x_direct(b)) F.s2l_nodes.push_back(b);
    by_level(F.s2l_nodes, F.s2l_level_off);
    const int mx = (int)F.s2l_nodes.size();
    rc = F.d_s2l_nodes.upload(F.s2l_nodes.data(), sizeof(int) * mx, s);
    if (!rc) rc = F.dc_xyz.reserve(sizeof(double) * 3 * (size_t)std::max(mx, 1) * n);
    if (!rc) rc = F.dcheck.reserve(sizeof(double) * (size_t)std::max(mx, 1) * n * kc);
    if (rc) return rc;
    if (mx)
        surface_points_kernel<<<grid_for((long long)mx * n), 256, 0, s>>>(
            (const int *)F.d_s2l_nodes.ptr, mx, centre, (const int *)d_level.ptr, kRad0,
            (const double *)F.unit_surf.ptr, n, (double *)F.dc_xyz.ptr);
    {
        std::vector<int> tb(mx), te(mx), off(mx + 1, 0), ent;
        std::vector<double> cc(3 * (size_t)std::max(mx, 1));
        const std::vector<int> owner = far_owners(T, f->shard_n);
        for (int i = 0; i < mx; i++) {
            const int b = F.s2l_nodes[i];
            tb[i] = i * n;
            te[i] = (!F.split || owner[b] == f->shard_rank) ? (i + 1) * n : i * n;
            off[i] = (int)ent.size();
            for (int e = T.X.off[b]; e < T.X.off[b + 1]; e++) ent.push_back(T.X.ent[e]);
            for (int d = 0; d < 3; d++) cc[3 * i + d] = ctr[3 * (size_t)b + d];
        }
        off[mx] = (int)ent.size();
        for (int k = 0; k < 2; k++) {
            const int uk = F.fused_src ? (k == 0 ? F.fused_check_uk : -1) : ki->slot[k == 0 ? SLOT_S2L_SL : SLOT_S2L_DL];
            F.s2l[k].reset();
            if (uk < 0 || T.sets[k].n == 0) continue;
            rc = setup_pass(F.s2l[k], uk, tb, te, off, ent, T.sets[k].node_begin.data(), T.sets[k].node_end.data(),
                            nn, false, cc, bw, s);
            if (rc) return rc;
        }
    }

    // ---- M2T (W list) and L2T: targets = leaf targets; sources = node surfaces ----
    {
        std::vector<int> sb(nn), se(nn);
        for (int b = 0; b < nn; b++) {
            sb[b] = b * n;
            se[b] = (b + 1) * n;
        }
        const PointSet &tg = T.sets[2];
        std::vector<int> loff(nn + 1, 0), lent;
        for (int b = 0; b < nn; b++) {
            loff[b] = (int)lent.size();
            if (T.is_leaf(b) && tg.count(b) > 0) lent.push_back((b << 5) | kShiftNone);
        }
        loff[nn] = (int)lent.size();
        std::vector<int> woff(nn + 1, 0), went;
        for (int b = 0; b < nn; b++) {
            woff[b] = (int)went.size();
            for (int e = T.W.off[b]; e < T.W.off[b + 1]; e++)
                if (!w_direct(T.W.ent[e] >> 5)) went.push_back(T.W.ent[e]);
        }
        woff[nn] = (int)went.size();
        F.m2t.reset();
        F.l2t.reset();
        // target-side passes follow the handle's shard (the upward pass, S2L and the
        // M2L are computed in full on every shard)
        rc = setup_pass(F.m2t, ki->slot[SLOT_M2T], tg.node_begin, tg.node_end, woff, went, sb.data(), se.data(), nn,
                        true, ctr, bw, s, f->shard_rank, f->shard_n);
        if (!rc)
            rc = setup_pass(F.l2t, ki->slot[SLOT_L2T], tg.node_begin, tg.node_end, loff, lent, sb.data(), se.data(),
                            nn, true, ctr, bw, s, f->shard_rank, f->shard_n);
        if (rc) return rc;
    }

    // ---- M2M / L2L: non-leaf nodes per level ----
    F.parents.clear();
    F.parent_off.assign(T.depth() + 2, 0);
    for (int l = 0; l <= T.depth(); l++) {
        F.parent_off[l] = (int)F.parents.size();
        int j = 0;
        for (int b = T.level_begin[l]; b < T.level_begin[l + 1]; b++) {
            if (T.is_leaf(b)) continue;
            // children of the level-l parents fill level l+1 in parent order
            if (T.first_child[b] != T.level_begin[l + 1] + 8 * j) return STK_ERR_STATE;
            F.parents.push_back(b);
            j++;
        }
    }
    F.parent_off[T.depth() + 1] = (int)F.parents.size();
    rc = F.d_parents.upload(F.parents.data(), sizeof(int) * F.parents.size(), s);
    if (rc) return rc;

    // ---- M2L: V-list pairs grouped by offset ----
    {
        const int nslot = (int)std::count_if(F.m2l_slot.begin(), F.m2l_slot.end(), [](int v) { return v >= 0; });
        // far field split over the shard group: owners of the M2L / S2L target nodes
        const std::vector<int> owner = far_owners(T, f->shard_n);
        auto own = [&](int b) { return !F.split || owner[b] == f->shard_rank; };
        // complete levels go to the dense M2L (all pairs of their targets)
        rc = setup_m2l_dense(F, T, nslot, s);
        if (rc) return rc;
        std::vector<char> dense_lvl(T.depth() + 1, 0);
        for (auto &dl : F.dense) dense_lvl[dl->level] = 1;
        std::vector<std::vector<int>> srcs(nslot), trgs(nslot);
        std::vector<long long> slot_pairs(nslot, 0);
        for (int b = 0; b < nn; b++)
            for (int e = T.V.off[b]; e < T.V.off[b + 1]; e++) {
                const int a = T.V.ent[e] >> 5, code = T.V.ent[e] & 31;
                const int sx = code % 3 - 1, sy = (code / 3) % 3 - 1, sz = code / 9 - 1;
                const int64_t L = 1LL << T.level[b];
                const int dx = (int)((int64_t)T.ix[a] + sx * L - T.ix[b]);
                const int dy = (int)((int64_t)T.iy[a] + sy * L - T.iy[b]);
                const int dz = (int)((int64_t)T.iz[a] + sz * L - T.iz[b]);
                if (std::abs(dx) > 3 || std::abs(dy) > 3 || std::abs(dz) > 3) return STK_ERR_STATE;
                const int sl = F.m2l_slot[(dx + 3) + 7 * (dy + 3) + 49 * (dz + 3)];
                if (sl < 0) return STK_ERR_STATE;
                slot_pairs[sl]++;
                if (dense_lvl[T.level[b]] || !own(b)) continue;
                srcs[sl].push_back(a);
                trgs[sl].push_back(b);
            }
        // column chunks of kM2LChunk pairs of one offset; padded columns gather zeros
        std::vector<int> gsrc, chunk_slot;
        std::vector<std::vector<int>> cols_of(nn);  // per target node: its columns, by offset
        long long pairs = 0;
        for (int sl = 0; sl < nslot; sl++) {
            const int m = (int)srcs[sl].size();
            for (int c0 = 0; c0 < m; c0 += kM2LChunk) {
                const int base = (int)gsrc.size();
                chunk_slot.push_back(sl);
                for (int i = 0; i < kM2LChunk; i++) {
                    const bool real = c0 + i < m;
                    gsrc.push_back(real ? srcs[sl][c0 + i] : -1);
                    if (real) cols_of[trgs[sl][c0 + i]].push_back(base + i);
                }
            }
            pairs += m;
        }
        for (auto &dl : F.dense) pairs += dl->pairs;
        F.m2l_pairs = pairs;
        F.m2l_chunks = (int)chunk_slot.size();
        F.m2l_cols = (long long)gsrc.size();
        std::vector<int> red_off(nn + 1, 0), red_col;
        red_col.reserve(pairs);
        for (int b = 0; b < nn; b++) {
            red_off[b] = (int)red_col.size();
            red_col.insert(red_col.end(), cols_of[b].begin(), cols_of[b].end());
        }
        red_off[nn] = (int)red_col.size();
        const int k = F.m2l_rank;
        rc = F.d_m2l_gsrc.upload(gsrc.data(), sizeof(int) * gsrc.size(), s);
        if (!rc) rc = F.d_m2l_red_off.upload(red_off.data(), sizeof(int) * red_off.size(), s);
        if (!rc) rc = F.d_m2l_red_col.upload(red_col.data(), sizeof(int) * red_col.size(), s);
        if (rc) return rc;
        // columns are processed in groups of whole chunks that keep the gathered sources and
        // the products within ~2 GiB each
        const int nc = F.m2l_chunks;
        const size_t per_chunk = (size_t)kM2LChunk * k * sizeof(double);
        F.m2l_group_chunks = (int)std::max<size_t>(1, std::min<size_t>(nc, (2ull << 30) / per_chunk));
        const int gc = F.m2l_group_chunks;
        const size_t gcols = (size_t)gc * kM2LChunk;
        // per group g and target t: the first of t's entries whose column is in group g or later
        const int ngroups = (nc + gc - 1) / gc;
        std::vector<int> gstart((size_t)(ngroups + 1) * nn);
        for (int b = 0; b < nn; b++) {
            int e = red_off[b];
            for (int g = 0; g <= ngroups; g++) {
                const long long gcol0 = (long long)g * gc * kM2LChunk;
                while (e < red_off[b + 1] && red_col[e] < gcol0) e++;
                gstart[(size_t)g * nn + b] = e;
            }
        }
        rc = F.d_m2l_gstart.upload(gstart.data(), sizeof(int) * gstart.size(), s);
        if (rc) return rc;
        const int rmax = F.m2l_rmax;
        // k4 (not k) per column: the tensor-core path keeps split FP32 rows of k4 floats here
        rc = F.m2l_x.reserve(sizeof(double) * (size_t)((k + 3) / 4 * 4) * gcols);
        if (!rc) rc = F.m2l_y.reserve(sizeof(double) * (size_t)k * gcols);
        if (!rc) rc = F.m2l_z.reserve(sizeof(double) * (size_t)rmax * gcols);
        if (rc) return rc;
        // Per group of columns and padded rank r: two batched GEMMs over that group's
        // chunks whose offset has rank r,
        //   Z_c = Q_d^T X_c (r x 256),  Y_c = P_d Z_c (k x 256).
        // Pointer arrays in (group, rank, chunk) order -- A: the offset's factor; B, C:
        // the chunk's slot in its group -- as FP64 and FP32 views of the same buffers.
        std::vector<int> order;
        F.m2l_seg.clear();
        for (int g = 0; g < ngroups; g++) {
            const int c0 = g * gc, c1e = std::min(nc, c0 + gc);
            std::map<int, std::vector<int>> by_rank;
            for (int c = c0; c < c1e; c++) by_rank[F.m2l_r[chunk_slot[c]]].push_back(c);
            for (auto &kv : by_rank) {
                F.m2l_seg.push_back({g, kv.first, (int)order.size(), (int)kv.second.size()});
                order.insert(order.end(), kv.second.begin(), kv.second.end());
            }
        }
        std::vector<const void *> a1(nc), b1(nc), a2(nc), a1f(nc), b1f(nc), a2f(nc);
        std::vector<void *> c1(nc), c2(nc), c1f(nc), c2f(nc);
        for (int i = 0; i < nc; i++) {
            const int c = order[i], sl = chunk_slot[c];
            const size_t j = (size_t)(c % gc);  // slot within its group
            a1[i] = (const double *)F.m2l_q.ptr + F.m2l_pq_off[sl];
            a2[i] = (const double *)F.m2l_p.ptr + F.m2l_pq_off[sl];
            a1f[i] = (const float *)F.m2l_q32.ptr + F.m2l_pq_off[sl];
            a2f[i] = (const float *)F.m2l_p32.ptr + F.m2l_pq_off[sl];
            b1[i] = (const double *)F.m2l_x.ptr + j * kM2LChunk * k;
            b1f[i] = (const float *)F.m2l_x.ptr + j * kM2LChunk * k;
            c1[i] = (double *)F.m2l_z.ptr + j * kM2LChunk * rmax;
            c1f[i] = (float *)F.m2l_z.ptr + j * kM2LChunk * rmax;
            c2[i] = (double *)F.m2l_y.ptr + j * kM2LChunk * k;
            c2f[i] = (float *)F.m2l_y.ptr + j * kM2LChunk * k;
        }
        rc = F.d_m2l_ptr[0].upload(a1.data(), sizeof(void *) * nc, s);
        if (!rc) rc = F.d_m2l_ptr[1].upload(b1.data(), sizeof(void *) * nc, s);
        if (!rc) rc = F.d_m2l_ptr[2].upload(c1.data(), sizeof(void *) * nc, s);
        if (!rc) rc = F.d_m2l_ptr[3].upload(a2.data(), sizeof(void *) * nc, s);
        if (!rc) rc = F.d_m2l_ptr[4].upload(c2.data(), sizeof(void *) * nc, s);
        if (!rc) rc = F.d_m2l_ptr32[0].upload(a1f.data(), sizeof(void *) * nc, s);
        if (!rc) rc = F.d_m2l_ptr32[1].upload(b1f.data(), sizeof(void *) * nc, s);
        if (!rc) rc = F.d_m2l_ptr32[2].upload(c1f.data(), sizeof(void *) * nc, s);
        if (!rc) rc = F.d_m2l_ptr32[3].upload(a2f.data(), sizeof(void *) * nc, s);
        if (!rc) rc = F.d_m2l_ptr32[4].upload(c2f.data(), sizeof(void *) * nc, s);
        if (rc) return rc;
        rc = setup_m2l_chunks_tc(F, chunk_slot, nslot, s);
        if (rc) return rc;
        F.m2l_flops = 0;
        for (int c = 0; c < nc; c++) F.m2l_flops += 4.0 * k * F.m2l_r[chunk_slot[c]] * kM2LChunk;
        F.m2l_flops_alg = 4.0 * (double)k * N * nn;
        for (int sl = 0; sl < nslot; sl++) F.m2l_flops_alg += 4.0 * k * F.m2l_rt[sl] * (double)slot_pairs[sl];
        F.m2l_flops += 4.0 * (double)k * N * nn;
        for (auto &dl : F.dense)
            for (int c = 0; c < 8; c++) F.m2l_flops += 2.0 * k * (F.dn_rs[c] + F.dn_rv[c]) * (double)dl->n8;
        // host vectors above are pageable: their copies complete before upload returns
        int maxm = 0;
        for (int l = 0; l <= T.depth(); l++) maxm = std::max(maxm, F.parent_off[l + 1] - F.parent_off[l]);
        maxm = std::max(maxm, std::max(ms, mx));
        rc = F.tmp0.reserve(sizeof(double) * (size_t)std::max(maxm, 1) * N);
        if (!rc) rc = F.tmp1.reserve(sizeof(double) * (size_t)std::max(maxm, 1) * N);
        if (rc) return rc;
    }
    FCUDA(cudaStreamSynchronize(s));
    F.ready = true;
    return STK_OK;
}

// The mixed path's dense M2L of one complete level on the tensor cores
// (3xTF32 tcgen05 GEMMs, stk_umma.cu; Z and Psi FP32 as on the SIMT path):
//   1. Z_c' = Qs_c'^T Phi_c' for the 8 source types, all kept (one GEMM each);
//   2. per target type c: the rows of every block (c, c') gathered into one
//      operand Zcat_c (dn_rv[c] rows per target, blocks in c' order), and
//      Psi_c = Pv_c Zcat_c as ONE GEMM over K = dn_rv[c] -- the sum over the
//      source types runs inside the GEMM's K loop, in a fixed order
//      (deterministic) -- the 8 target types on concurrent streams, so that the
//      narrow GEMMs (M = k, N = boxes per type) together fill the GPU.
static int m2l_dense_level_tc(FarField &F, const M2LDenseLevel &D, const double *phi_hat, double *psi_hat,
                              cudaStream_t s) {
    const int k = F.m2l_rank, n8 = D.n8, n = 8 * n8, k4 = (k + 3) / 4 * 4;
    const int *nodes = (const int *)D.d_nodes.ptr;
    float *psi = (float *)F.dn_psi.ptr, *Z = (float *)F.tc_z.ptr;
    float *bh = (float *)F.tc_b_hi.ptr, *bl = (float *)F.tc_b_lo.ptr;
    int *err = (int *)F.tc_err.ptr;
    t_launches++;
    tc_gather_cols_kernel<<<grid_for((long long)n * k4), 256, 0, s>>>(phi_hat, nodes, n, k, k4, bh, bl);
    FCUDA(cudaGetLastError());
    FCUDA(cudaMemsetAsync(psi, 0, sizeof(float) * (size_t)k * n, s));  // types this rank does not own stay 0
    size_t zoff[8];
    size_t zo = 0;
    for (int cs = 0; cs < 8; cs++) {
        zoff[cs] = zo;
        const int rs = F.dn_rs[cs];
        if (!rs) continue;
        t_launches++;
        FCUDA(umma_gemm_3xtf32(rs, n8, k,
                               Tf32Split{(const float *)F.tc_qa_hi.ptr + F.tc_qa_off[cs],
                                         (const float *)F.tc_qa_lo.ptr + F.tc_qa_off[cs], k4},
                               Tf32Split{bh + (size_t)cs * n8 * k4, bl + (size_t)cs * n8 * k4, k4}, Z + zo, rs, 0, err,
                               s));
        zo += (size_t)rs * n8;
    }
    // fork: target types round-robin over the streams, each with its own Zcat buffer
    FCUDA(cudaEventRecord(F.tc_fork, s));
    const int ns = F.tc_streams, ld = F.tc_zc_ld;
    bool used[8] = {};
    for (int c = 0; c < 8; c++) {
        const int rv = F.dn_rv[c];
        if (!rv || !F.dn_own[c]) continue;
        const int si = c % ns;
        cudaStream_t st = F.tc_stream[si];
        if (!used[si]) FCUDA(cudaStreamWaitEvent(st, F.tc_fork, 0));
        used[si] = true;
        float *zh = (float *)F.tc_zc_hi.ptr + (size_t)si * ld * n8, *zl = (float *)F.tc_zc_lo.ptr + (size_t)si * ld * n8;
        const int rv4 = (rv + 3) / 4 * 4;  // row pitch; the GEMM reads K = rv (TMA zero-fills beyond)
        for (int cs = 0; cs < 8; cs++) {
            const int b = 8 * c + cs, R = F.dn_rcc[b];
            if (!R) continue;
            t_launches++;
            // rows [pstart_b, pstart_b + R) of every target's Zcat_c row (pitch rv4)
            tc_zgather_kernel<<<grid_for((long long)n8 * R), 256, 0, st>>>(
                Z + zoff[cs], F.dn_rs[cs], (const int *)D.d_tab.ptr + D.tab_off[b], F.dn_q[b],
                (const int *)F.dn_rowq.ptr + F.dn_row_off[b], (const int *)F.dn_srow.ptr + F.dn_row_off[b], R, R, rv4,
                n8, zh + F.dn_pstart[b], zl + F.dn_pstart[b]);
            FCUDA(cudaGetLastError());
        }
        t_launches++;
        FCUDA(umma_gemm_3xtf32(k, n8, rv,
                               Tf32Split{(const float *)F.tc_pa_hi.ptr + F.tc_pa_off[c],
                                         (const float *)F.tc_pa_lo.ptr + F.tc_pa_off[c], rv4},
                               Tf32Split{zh, zl, rv4}, psi + (size_t)c * n8 * k, k, 0, err, st));
    }
    // join
    for (int si = 0; si < ns; si++)
        if (used[si]) {
            FCUDA(cudaEventRecord(F.tc_ev[si], F.tc_stream[si]));
            FCUDA(cudaStreamWaitEvent(s, F.tc_ev[si], 0));
        }
    return scatter_cols<float>(psi, nodes, n, k, 1.0, 1, psi_hat, s);
}

// Dense M2L of one complete level: psi_hat[:, t] += sum over the level's V-list
// pairs, by box parity type (M2LDenseLevel), in T = double (FP64) or float (mixed).
template <class T>
static int m2l_dense_level(FarField &F, const M2LDenseLevel &D, const double *phi_hat, double *psi_hat,
                           cudaStream_t s) {
    const bool f32 = std::is_same<T, float>::value;
    const int k = F.m2l_rank, n8 = D.n8, n = 8 * n8;
    const cudaDataType_t dt = f32 ? CUDA_R_32F : CUDA_R_64F;
    const cublasComputeType_t ct = f32 ? CUBLAS_COMPUTE_32F : CUBLAS_COMPUTE_64F;
    const T one = T(1), zero = T(0);
    T *phi = (T *)F.dn_phi.ptr, *psi = (T *)F.dn_psi.ptr, *Z = (T *)F.dn_z.ptr, *Zc = (T *)F.dn_zc.ptr;
    const T *pv = f32 ? (const T *)F.dn_pv32.ptr : (const T *)F.dn_pv.ptr;
    const T *qs = f32 ? (const T *)F.dn_qs32.ptr : (const T *)F.dn_qs.ptr;
    const int *nodes = (const int *)D.d_nodes.ptr;
    if constexpr (std::is_same<T, float>::value) {
        if (F.tc) return m2l_dense_level_tc(F, D, phi_hat, psi_hat, s);
    }
    int rc = gather_cols<double, T>(phi_hat, nodes, n, k, phi, s);
    if (rc) return rc;
    FCUDA(cudaMemsetAsync(psi, 0, sizeof(T) * (size_t)k * n, s));
    for (int cs = 0; cs < 8; cs++) {
        const int rs = F.dn_rs[cs];
        if (!rs) continue;
        // Z = Qs_c'^T Phi_c': every offset of the source type at once
        FBLAS(cublasGemmEx(F.blas, CUBLAS_OP_T, CUBLAS_OP_N, rs, n8, k, &one, qs + F.dn_qs_off[cs], dt, k,
                           phi + (size_t)cs * n8 * k, dt, k, &zero, Z, dt, rs, ct, CUBLAS_GEMM_DEFAULT));
        for (int c = 0; c < 8; c++) {
            const int b = 8 * c + cs, R = F.dn_rcc[b];
            if (!R || !F.dn_own[c]) continue;
            t_launches++;
            m2l_zgather_kernel<T><<<grid_for((long long)n8 * R), 256, 0, s>>>(
                Z, rs, (const int *)D.d_tab.ptr + D.tab_off[b], F.dn_q[b], (const int *)F.dn_rowq.ptr + F.dn_row_off[b],
                (const int *)F.dn_srow.ptr + F.dn_row_off[b], R, n8, Zc);
            FCUDA(cudaGetLastError());
            // Psi_c += Pv_{c,c'} Zc (source types in a fixed order: deterministic)
            FBLAS(cublasGemmEx(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, k, n8, R, &one,
                               pv + F.dn_pv_off[c] + (size_t)k * F.dn_pstart[b], dt, k, Zc, dt, R, &one,
                               psi + (size_t)c * n8 * k, dt, k, ct, CUBLAS_GEMM_DEFAULT));
        }
    }
    return scatter_cols<T>(psi, nodes, n, k, 1.0, 1, psi_hat, s);
}

int farfield_evaluate(Stk3DFMM *f, KernelData *kd, const double *d_sl, const double *d_dl, double *trg_sorted,
                      cudaStream_t s) {
    FarField &F = *kd->far;
    const KernelInfo *ki = kd->info;
    const Octree &T = kd->tree;
    const int nn = T.num_nodes(), n = F.n, ke = F.ke, kc = F.kc, N = n * ke;
    const int prec = f->precision;
    const int sms = f->sms;
    unsigned int *counter = (unsigned int *)kd->d_counter.ptr;
    const double one = 1.0, zero = 0.0;
    cublasSetStream(F.blas, s);
    double *phi = (double *)F.phi.ptr, *psi = (double *)F.psi.ptr;
    double *X = (double *)F.tmp0.ptr, *Y = (double *)F.tmp1.ptr;
    t_launches = 0;
    FCUDA(cudaMemsetAsync(phi, 0, sizeof(double) * (size_t)nn * N, s));
    FCUDA(cudaMemsetAsync(psi, 0, sizeof(double) * (size_t)nn * N, s));

    // source records of the point sets for the S2M / S2L kernels
    auto pack_points = [&](int k, int uk) -> int {
        const int rs = uk_record_stride(uk);
        const PointSet &ps = T.sets[k];
        int rc = F.rec_pts[k].reserve(sizeof(double) * (size_t)std::max(ps.n, 1) * rs);
        if (rc) return rc;
        t_launches++;
        // fused check pass: SL values then DL values in one record
        const bool both = F.fused_src && k == 0 && d_dl;
        if (launch_pack_records(ps.n, (const int *)kd->d_perm[k].ptr, (const double *)kd->d_xyz[k].ptr,
                                k == 0 ? d_sl : d_dl, k == 0 ? ki->kdim_sl : ki->kdim_dl, both ? d_dl : nullptr,
                                both ? ki->kdim_dl : 0, rs, (double *)F.rec_pts[k].ptr, s) != cudaSuccess)
            return STK_ERR_CUDA;
        return STK_OK;
    };

    // ---- upward pass: S2M, then check -> equivalent per level ----
    const int ms = (int)F.s2m_nodes.size();
    if (ms) {
        FCUDA(cudaMemsetAsync(F.check.ptr, 0, sizeof(double) * (size_t)ms * n * kc, s));
        for (int k = 0; k < 2; k++) {
            if (F.s2m[k].uk < 0 || (k == 1 && !d_dl)) continue;
            int rc = pack_points(k, F.s2m[k].uk);
            if (!rc)
                rc = run_pass(F.s2m[k], prec, (const double *)F.rec_pts[k].ptr, (const int *)kd->d_beg[k].ptr,
                              (const int *)kd->d_end[k].ptr, (const double *)F.uc_xyz.ptr, (double *)F.check.ptr,
                              counter, sms, s);
            if (rc) return rc;
        }
        for (int l = 0; l + 1 < (int)F.s2m_level_off.size(); l++) {
            const int a = F.s2m_level_off[l], m = F.s2m_level_off[l + 1] - a;
            if (m <= 0) continue;
            double alpha = std::ldexp(1.0, -l);
            if (F.scaled) {
                // normalised check potential: 2^-l (1 + pot_exp[a]) per component
                CompF e;
                for (int c = 0; c < 4; c++) e.v[c] = 1.0 + F.pot_exp[c];
                level_scale_kernel<<<grid_for((long long)m * n * kc), 256, 0, s>>>(
                    (double *)F.check.ptr + (size_t)a * n * kc, m, n * kc, kc, nullptr, l, e);
                FCUDA(cudaGetLastError());
                t_launches++;
                alpha = 1.0;
            }
            FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, N, m, n * kc, &alpha, (const double *)F.uc2ue.ptr, N,
                              (const double *)F.check.ptr + (size_t)a * n * kc, n * kc, &zero, Y, N));
            int rc = scatter_cols(Y, (const int *)F.d_s2m_nodes.ptr + a, m, N, 1.0, 0, phi, s);
            if (rc) return rc;
        }
    }
    FCUDA(cudaEventRecord(kd->ph[1], s));
    // M2M, bottom up: parents of level l from the contiguous children block at level l+1
    const int *d_parents = (const int *)F.d_parents.ptr;
    for (int l = T.depth() - 1; l >= 0; l--) {
        const int a = F.parent_off[l], m = F.parent_off[l + 1] - a;
        if (m == 0) continue;
        const double *Xc = phi + (size_t)T.level_begin[l + 1] * N;
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, N, m, 8 * N, &one, (const double *)F.m2m.ptr, N, Xc, 8 * N,
                          &zero, Y, N));
        int rc = scatter_cols(Y, d_parents + a, m, N, 1.0, 0, phi, s);
        if (rc) return rc;
    }

    FCUDA(cudaEventRecord(kd->ph[2], s));
    // ---- downward pass: compressed M2L per offset ----
    const int k = F.m2l_rank;
    double *phi_hat = (double *)F.phi_hat.ptr, *psi_hat = (double *)F.psi_hat.ptr;
    // The basis products phi_hat = V^T phi and psi += (DC2DE U) psi_hat stay FP64 in both
    // paths.  Their sums cancel strongly: the equivalent densities of the pseudo-inverse
    // solves are much larger than the fields they stand for.  FP32-accurate products
    // (3xTF32 on the tensor cores) raised the mixed Stokes FMM's error from 2.8e-7 to
    // 5.2e-7 (V^T phi alone) and 7.3e-7 (both); p = 8, 12000 clustered points.
    FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, k, nn, N, &one, (const double *)F.m2l_vt.ptr, k, phi, N,
                      &zero, phi_hat, k));
    // gather the sources of every (offset, chunk) column, one batched GEMM over the
    // chunks, then each target sums its columns in offset order (deterministic)
    FCUDA(cudaMemsetAsync(psi_hat, 0, sizeof(double) * (size_t)nn * k, s));
    const int nc = F.m2l_chunks, gc = F.m2l_group_chunks;
    for (int c0 = 0; c0 < nc; c0 += gc) {
        const int *gbeg = (const int *)F.d_m2l_gstart.ptr + (size_t)(c0 / gc) * nn, *gend = gbeg + nn;
        const int ncg = std::min(gc, nc - c0);
        const long long col0 = (long long)c0 * kM2LChunk, ncol = (long long)ncg * kM2LChunk;
        const int *gsrc = (const int *)F.d_m2l_gsrc.ptr + col0;
        const int gg = grid_for(ncol * k);
        t_launches += 2;
        const bool mixed = prec == PREC_MIXED;
        const int rmax = F.m2l_rmax;
        const double one64 = 1.0, zero64 = 0.0;
        const float one32 = 1.0f, zero32 = 0.0f;
        const void *alpha = mixed ? (const void *)&one32 : (const void *)&one64;
        const void *beta = mixed ? (const void *)&zero32 : (const void *)&zero64;
        const cudaDataType_t dt = mixed ? CUDA_R_32F : CUDA_R_64F;
        const cublasComputeType_t ct = mixed ? CUBLAS_COMPUTE_32F : CUBLAS_COMPUTE_64F;
        DevBuf *P = mixed ? F.d_m2l_ptr32 : F.d_m2l_ptr;
        if (mixed && F.tcc) {
            // tensor cores: split gather, Z = Q_d^T X (split), Y = P_d Z, in two grouped launches
            const int g = c0 / gc, k4 = (k + 3) / 4 * 4;
            float *xh = (float *)F.m2l_x.ptr, *xl = xh + (size_t)ncol * k4;
            float *zh = (float *)F.m2l_z.ptr, *zl = zh + (size_t)ncol * rmax;
            int *err = (int *)F.tc_err.ptr;
            t_launches += 3;
            tc_gather_cols_kernel<<<grid_for(ncol * k4), 256, 0, s>>>(phi_hat, gsrc, ncol, k, k4, xh, xl);
            FCUDA(cudaGetLastError());
            FCUDA(umma_grouped_3xtf32(Tf32Rows{(const float *)F.tcc_q_hi.ptr, (const float *)F.tcc_q_lo.ptr,
                                               (int)F.tcc_q_rows, k, k4},
                                      Tf32Rows{xh, xl, (int)ncol, k, k4},
                                      (const GroupTile *)F.tcc_tiles1.ptr + F.tcc_t1_off[g],
                                      F.tcc_t1_off[g + 1] - F.tcc_t1_off[g], zh, zl, err, s));
            FCUDA(umma_grouped_3xtf32(Tf32Rows{(const float *)F.tcc_pt_hi.ptr, (const float *)F.tcc_pt_lo.ptr,
                                               (int)F.m2l_r.size() * k, rmax, rmax},
                                      Tf32Rows{zh, zl, (int)ncol, rmax, rmax},
                                      (const GroupTile *)F.tcc_tiles2.ptr + F.tcc_t2_off[g],
                                      F.tcc_t2_off[g + 1] - F.tcc_t2_off[g], (float *)F.m2l_y.ptr, nullptr, err, s));
            m2l_reduce_kernel<float><<<grid_for((long long)nn * k), 256, 0, s>>>(
                (const float *)F.m2l_y.ptr, gbeg, gend, (const int *)F.d_m2l_red_col.ptr, nn, k, col0, psi_hat);
            FCUDA(cudaGetLastError());
            continue;
        }
        if (mixed)
            m2l_gather_kernel<float><<<gg, 256, 0, s>>>(phi_hat, gsrc, k, ncol, (float *)F.m2l_x.ptr);
        else
            m2l_gather_kernel<double><<<gg, 256, 0, s>>>(phi_hat, gsrc, k, ncol, (double *)F.m2l_x.ptr);
        FCUDA(cudaGetLastError());
        for (const M2LSeg &sg : F.m2l_seg) {
            if (sg.group != c0 / gc) continue;
            // Z = Q_d^T X (r x 256), then Y = P_d Z (k x 256), for the segment's chunks
            FBLAS(cublasGemmBatchedEx(F.blas, CUBLAS_OP_T, CUBLAS_OP_N, sg.rank, kM2LChunk, k, alpha,
                                      (const void *const *)P[0].ptr + sg.start, dt, k,
                                      (const void *const *)P[1].ptr + sg.start, dt, k, beta,
                                      (void *const *)P[2].ptr + sg.start, dt, rmax, sg.count, ct,
                                      CUBLAS_GEMM_DEFAULT));
            FBLAS(cublasGemmBatchedEx(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, k, kM2LChunk, sg.rank, alpha,
                                      (const void *const *)P[3].ptr + sg.start, dt, k,
                                      (const void *const *)P[2].ptr + sg.start, dt, rmax, beta,
                                      (void *const *)P[4].ptr + sg.start, dt, k, sg.count, ct, CUBLAS_GEMM_DEFAULT));
        }
        if (mixed)
            m2l_reduce_kernel<float><<<grid_for((long long)nn * k), 256, 0, s>>>(
                (const float *)F.m2l_y.ptr, gbeg, gend, (const int *)F.d_m2l_red_col.ptr, nn, k, col0, psi_hat);
        else
            m2l_reduce_kernel<double><<<grid_for((long long)nn * k), 256, 0, s>>>(
                (const double *)F.m2l_y.ptr, gbeg, gend, (const int *)F.d_m2l_red_col.ptr, nn, k, col0, psi_hat);
        FCUDA(cudaGetLastError());
    }
    // complete levels: dense M2L by box type
    for (auto &Dp : F.dense) {
        const int rcd = prec == PREC_MIXED ? m2l_dense_level<float>(F, *Dp, phi_hat, psi_hat, s)
                                           : m2l_dense_level<double>(F, *Dp, phi_hat, psi_hat, s);
        if (rcd) return rcd;
    }
    FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, N, nn, k, &one, (const double *)F.m2l_e.ptr, N, psi_hat, k,
                      &one, psi, N));
    // triply periodic: the root's far images (FP64)
    if (F.periodic && (!F.split || f->shard_rank == 0))
        FBLAS(cublasDgemv(F.blas, CUBLAS_OP_N, N, N, &one, (const double *)F.m2c_op.ptr, N, phi, 1, &one, psi, 1));
    FCUDA(cudaEventRecord(kd->ph[3], s));
    // S2L (X list): downward check potentials, solved per level
    const int mx = (int)F.s2l_nodes.size();
    if (mx) {
        FCUDA(cudaMemsetAsync(F.dcheck.ptr, 0, sizeof(double) * (size_t)mx * n * kc, s));
        bool any = false;
        for (int k = 0; k < 2; k++) {
            if (F.s2l[k].uk < 0 || F.s2l[k].n_items == 0 || (k == 1 && !d_dl)) continue;
            int rc = pack_points(k, F.s2l[k].uk);
            if (!rc)
                rc = run_pass(F.s2l[k], prec, (const double *)F.rec_pts[k].ptr, (const int *)kd->d_beg[k].ptr,
                              (const int *)kd->d_end[k].ptr, (const double *)F.dc_xyz.ptr, (double *)F.dcheck.ptr,
                              counter, sms, s);
            if (rc) return rc;
            any = true;
        }
        if (any)
            for (int l = 0; l + 1 < (int)F.s2l_level_off.size(); l++) {
                const int a = F.s2l_level_off[l], m = F.s2l_level_off[l + 1] - a;
                if (m <= 0) continue;
                double alpha = std::ldexp(1.0, -l);
                if (F.scaled) {
                    CompF e;
                    for (int c = 0; c < 4; c++) e.v[c] = 1.0 + F.pot_exp[c];
                    level_scale_kernel<<<grid_for((long long)m * n * kc), 256, 0, s>>>(
                        (double *)F.dcheck.ptr + (size_t)a * n * kc, m, n * kc, kc, nullptr, l, e);
                    FCUDA(cudaGetLastError());
                    t_launches++;
                    alpha = 1.0;
                }
                FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, N, m, n * kc, &alpha, (const double *)F.dc2de.ptr,
                                  N, (const double *)F.dcheck.ptr + (size_t)a * n * kc, n * kc, &zero, Y, N));
                int rc = scatter_cols(Y, (const int *)F.d_s2l_nodes.ptr + a, m, N, 1.0, 1, psi, s);
                if (rc) return rc;
            }
    }
    // split far field: every rank holds its target nodes' M2L / S2L contributions;
    // one sum over the shard group gives all ranks the whole downward densities
    if (F.split && f->allreduce(psi, (long long)nn * N, (void *)s, f->allreduce_user) != 0) return STK_ERR_CUDA;
    FCUDA(cudaEventRecord(kd->ph[4], s));
    // L2L, top down: the level-l children block of the level-(l-1) parents
    for (int l = 1; l <= T.depth(); l++) {
        const int a = F.parent_off[l - 1], m = F.parent_off[l] - a;
        if (m == 0) continue;
        int rc = gather_cols(psi, d_parents + a, m, N, X, s);
        if (rc) return rc;
        FBLAS(cublasDgemm(F.blas, CUBLAS_OP_N, CUBLAS_OP_N, 8 * N, m, N, &one, (const double *)F.l2l.ptr, 8 * N, X, N,
                          &one, psi + (size_t)T.level_begin[l] * N, 8 * N));
    }

    // ---- evaluation at the targets: L2T and M2T (W list) ----
    const long long npts = (long long)nn * n;
    auto pack_surface = [&](const DevBuf &xyz, const double *dens, int uk) -> int {
        const int rs = uk_record_stride(uk);
        int rc = F.rec_surf.reserve(sizeof(double) * (size_t)npts * rs);
        if (rc) return rc;
        t_launches++;
        if (launch_pack_records((int)npts, nullptr, (const double *)xyz.ptr, dens, ke, nullptr, 0, rs,
                                (double *)F.rec_surf.ptr, s) != cudaSuccess)
            return STK_ERR_CUDA;
        return STK_OK;
    };
    FCUDA(cudaEventRecord(kd->ph[5], s));
    const double *trg_xyz = (const double *)kd->d_xyz[2].ptr;
    if (F.scaled) {
        // back to physical densities at each node's level: component c times 2^-l den_exp[c]
        CompF e;
        for (int c = 0; c < 4; c++) e.v[c] = F.den_exp[c];
        level_scale_kernel<<<grid_for((long long)nn * N), 256, 0, s>>>(psi, nn, N, ke, (const int *)F.d_level.ptr, 0,
                                                                      e);
        level_scale_kernel<<<grid_for((long long)nn * N), 256, 0, s>>>(phi, nn, N, ke, (const int *)F.d_level.ptr, 0,
                                                                      e);
        FCUDA(cudaGetLastError());
        t_launches += 2;
    }
    int rc = pack_surface(F.de_xyz, psi, F.l2t.uk);
    if (!rc)
        rc = run_pass(F.l2t, prec, (const double *)F.rec_surf.ptr, (const int *)F.l2t.src_beg.ptr,
                      (const int *)F.l2t.src_end.ptr, trg_xyz, trg_sorted, counter, sms, s);
    if (rc) return rc;
    FCUDA(cudaEventRecord(kd->ph[6], s));
    if (F.m2t.n_items) {
        rc = pack_surface(F.ue_xyz, phi, F.m2t.uk);
        if (!rc)
            rc = run_pass(F.m2t, prec, (const double *)F.rec_surf.ptr, (const int *)F.m2t.src_beg.ptr,
                          (const int *)F.m2t.src_end.ptr, trg_xyz, trg_sorted, counter, sms, s);
        if (rc) return rc;
    }
    // periodizeFMM: PVel, PVelGrad and PVelLaplacian only (not Traction), with the
    // far field on, on the first shard alone so that the shards' outputs still
    // sum to the whole
    const unsigned kid = ki->id;
    if (f->pbc == STK_PAXIS_PXYZ && f->enable_ff &&
        (kid == STK_PVel || kid == STK_PVelGrad || kid == STK_PVelLaplacian) && f->shard_rank == 0 && f->ntrg > 0) {
        const int blocks = (int)std::min<long long>(((long long)f->ntrg + kNetFluxThreads - 1) / kNetFluxThreads, 148 * 4);
        pvel_net_flux_kernel<<<blocks, kNetFluxThreads, 0, s>>>(phi, (const double *)F.ue_xyz.ptr, n, trg_sorted,
                                                                f->ntrg, ki->kdim_trg);
        FCUDA(cudaGetLastError());
        t_launches++;
    }
    FCUDA(cudaEventRecord(kd->ph[7], s));
    F.launches = t_launches;
    return STK_OK;
}

int farfield_status(KernelData *kd) {
    if (!kd->far || !(kd->far->tc || kd->far->tcc) || !kd->far->tc_err.ptr) return STK_OK;
    int e = 0;
    if (cudaMemcpy(&e, kd->far->tc_err.ptr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return STK_ERR_CUDA;
    if (e == 0) return STK_OK;
    cudaMemset(kd->far->tc_err.ptr, 0, sizeof(int));
    fprintf(stderr, "stkfmm_b200: a tensor-core M2L GEMM stopped at a pipeline wait (code %d)\n", e);
    return STK_ERR_CUDA;
}

}  // namespace stk

// The reference's public surface helper stkfmm::surface(p, c, alpha, depth)
// (Lib/include/STKFMM/stkfmm_helpers.hpp:46-85): the same points in the same
// order, on the cube of side alpha 2^-depth with lower corner c.  Host only.
extern "C" int stk_surface(int p, const double *c, double alpha, int depth, double *out) {
    if (p < 2 || !c || !out || depth < 0) return STK_ERR_INVALID_ARG;
    const std::vector<double> u = stk::unit_surface(p);
    const double b = alpha * std::ldexp(0.5, -depth);
    for (size_t i = 0; i < u.size(); i++) out[i] = (u[i] + 1.0) * b + c[i % 3];
    return STK_OK;
}
