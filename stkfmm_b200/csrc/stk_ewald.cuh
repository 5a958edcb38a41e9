// stk_ewald.cuh -- periodic Green's functions of the unit cell by Ewald summation,
// for the far-image (M2C) operators of the periodic FMM.
//
// Restated from the reference's M2C generator (the formulas, in own code):
//   Laplace, triply periodic   M2L/Laplace/Laplace3D3D.cpp:14-84 (potential; gradient 86-200)
//   Laplace, doubly periodic   M2L/Laplace/Laplace2D3D.cpp:12-83 (potential),
//                              M2L/StokesPVel/StokesPVel2D3D.cpp:167-240 (gradient)
//   Stokeslet, triply periodic M2L/Stokeslet/Stokes3D3D.cpp:19-68
//   Stokeslet, doubly periodic M2L/Stokeslet/Stokes2D3D.cpp:19-168
// Doubly periodic cells repeat along x and y with period 1; z is free.  Every
// function returns the periodic sum without the kernel's 1/(4 pi) or 1/(8 pi),
// over all images including the one at r itself (for r = 0 that image is
// replaced by the Ewald self term).  Laplace: the zero-mean (3D) or the
// reference's (2D) normalisation; Stokeslet: the k = 0 mode dropped (3D) or
// the reference's k = 0 term (2D).
#pragma once
#include <cuda_runtime.h>

namespace stk {
namespace ewald {

constexpr double kPi = 3.14159265358979323846;
constexpr double kXi = 2.0;  // splitting parameter for a unit cell
constexpr int kReal = 5;     // real-space images |s_i| <= kReal
constexpr int kWave = 5;     // wave vectors 2 pi m, 0 < max |m_i| <= kWave
constexpr double kZero = 1e-13;

__device__ __forceinline__ double sq(double a) { return a * a; }

// d/dr [erfc(xi r) / r]
__device__ __forceinline__ double derfc_r(double xi, double r) {
    return -2.0 * xi * exp(-sq(xi * r)) / (sqrt(kPi) * r) - erfc(xi * r) / (r * r);
}

// ---- Laplace, triply periodic: potential (4 pi x zero-mean Green's function) and gradient ----
__device__ inline void lap3(const double r0[3], double &pot, double grad[3]) {
    const double xi = kXi, xi2 = xi * xi;
    pot = 0.0;
    grad[0] = grad[1] = grad[2] = 0.0;
    for (int a = -kReal; a <= kReal; a++)
        for (int b = -kReal; b <= kReal; b++)
            for (int c = -kReal; c <= kReal; c++) {
                const double r[3] = {r0[0] + a, r0[1] + b, r0[2] + c};
                const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                if (rr < kZero) {
                    pot += -2.0 * xi / sqrt(kPi);
                    continue;
                }
                pot += erfc(xi * rr) / rr;
                const double d = derfc_r(xi, rr) / rr;
                for (int k = 0; k < 3; k++) grad[k] += d * r[k];
            }
    for (int a = -kWave; a <= kWave; a++)
        for (int b = -kWave; b <= kWave; b++)
            for (int c = -kWave; c <= kWave; c++) {
                if (a == 0 && b == 0 && c == 0) continue;
                const double k[3] = {2 * kPi * a, 2 * kPi * b, 2 * kPi * c};
                const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                const double w = 4 * kPi * exp(-k2 / (4 * xi2)) / k2;
                const double ph = k[0] * r0[0] + k[1] * r0[1] + k[2] * r0[2];
                pot += w * cos(ph);
                const double sn = sin(ph);
                for (int q = 0; q < 3; q++) grad[q] -= w * k[q] * sn;
            }
    pot -= kPi / xi2;
}

// ---- Stokeslet, triply periodic (8 pi x G) ----
__device__ inline void stk3(const double r0[3], double G[3][3]) {
    const double xi = kXi, xi2 = xi * xi;
    for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) G[p][q] = 0.0;
    for (int a = -kReal; a <= kReal; a++)
        for (int b = -kReal; b <= kReal; b++)
            for (int c = -kReal; c <= kReal; c++) {
                const double r[3] = {r0[0] + a, r0[1] + b, r0[2] + c};
                const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                if (rr < kZero) {
                    for (int p = 0; p < 3; p++) G[p][p] += -4.0 * xi / sqrt(kPi);
                    continue;
                }
                const double ex = exp(-xi2 * rr * rr), ec = erfc(xi * rr);
                const double c1 = 2 * (xi * ex / (sqrt(kPi) * rr * rr) + ec / (2 * rr * rr * rr));
                const double c2 = 4 * xi / sqrt(kPi) * ex;
                for (int p = 0; p < 3; p++)
                    for (int q = 0; q < 3; q++)
                        G[p][q] += c1 * ((p == q ? rr * rr : 0.0) + r[p] * r[q]) - (p == q ? c2 : 0.0);
            }
    for (int a = -kWave; a <= kWave; a++)
        for (int b = -kWave; b <= kWave; b++)
            for (int c = -kWave; c <= kWave; c++) {
                if (a == 0 && b == 0 && c == 0) continue;
                const double k[3] = {2 * kPi * a, 2 * kPi * b, 2 * kPi * c};
                const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                const double w = 8 * kPi * (1 + k2 / (4 * xi2)) * exp(-k2 / (4 * xi2)) / (k2 * k2) *
                                 cos(k[0] * r0[0] + k[1] * r0[1] + k[2] * r0[2]);
                for (int p = 0; p < 3; p++)
                    for (int q = 0; q < 3; q++) G[p][q] += w * ((p == q ? k2 : 0.0) - k[p] * k[q]);
            }
}

// z-profiles of the doubly periodic wave terms (k = |k_xy| > 0)
__device__ __forceinline__ double th_plus(double k, double xi, double z) { return exp(k * z) * erfc(k / (2 * xi) + xi * z); }
__device__ __forceinline__ double th_minus(double k, double xi, double z) { return exp(-k * z) * erfc(k / (2 * xi) - xi * z); }

// ---- Laplace, doubly periodic: potential and gradient ----
__device__ inline void lap2(const double r0[3], double &pot, double grad[3]) {
    const double xi = kXi, z = r0[2];
    pot = 0.0;
    grad[0] = grad[1] = grad[2] = 0.0;
    for (int a = -kReal; a <= kReal; a++)
        for (int b = -kReal; b <= kReal; b++) {
            const double r[3] = {r0[0] + a, r0[1] + b, z};
            const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            if (rr < kZero) {
                pot += -2.0 * xi / sqrt(kPi);
                continue;
            }
            pot += erfc(xi * rr) / rr;
            const double d = derfc_r(xi, rr) / rr;
            for (int k = 0; k < 3; k++) grad[k] += d * r[k];
        }
    for (int a = -kWave; a <= kWave; a++)
        for (int b = -kWave; b <= kWave; b++) {
            if (a == 0 && b == 0) continue;
            const double kx = 2 * kPi * a, ky = 2 * kPi * b, k = sqrt(kx * kx + ky * ky);
            const double ph = kx * r0[0] + ky * r0[1];
            const double tp = th_plus(k, xi, z), tm = th_minus(k, xi, z);
            const double g = tp + tm;
            // d g / d z
            const double gz = k * (tp - tm) + 2 * xi / sqrt(kPi) *
                                                   (exp(-sq(-xi * z + k / (2 * xi)) - k * z) -
                                                    exp(-sq(xi * z + k / (2 * xi)) + k * z));
            pot += kPi * cos(ph) * g / k;
            grad[0] -= kPi * sin(ph) * g / k * kx;
            grad[1] -= kPi * sin(ph) * g / k * ky;
            grad[2] += kPi * cos(ph) * gz / k;
        }
    // k = 0 mode
    pot -= 2 * sqrt(kPi) * (exp(-sq(xi * z)) / xi + sqrt(kPi) * z * erf(xi * z));
    grad[2] -= 2 * kPi * erf(xi * z);
}

// ---- Stokeslet, doubly periodic (8 pi x G) ----
__device__ inline void stk2(const double r0[3], double G[3][3]) {
    const double xi = kXi, xi2 = xi * xi, z = r0[2], sp = sqrt(kPi);
    for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) G[p][q] = 0.0;
    for (int a = -kReal; a <= kReal; a++)
        for (int b = -kReal; b <= kReal; b++) {
            const double r[3] = {r0[0] + a, r0[1] + b, z};
            const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            if (rr < kZero) {
                for (int p = 0; p < 3; p++) G[p][p] += -4.0 * xi / sp;
                continue;
            }
            const double ex = exp(-xi2 * rr * rr), ec = erfc(xi * rr);
            const double c1 = 2 * (xi * ex / (sp * rr * rr) + ec / (2 * rr * rr * rr));
            const double c2 = 4 * xi / sp * ex;
            for (int p = 0; p < 3; p++)
                for (int q = 0; q < 3; q++) G[p][q] += c1 * ((p == q ? rr * rr : 0.0) + r[p] * r[q]) - (p == q ? c2 : 0.0);
        }
    for (int a = -kWave; a <= kWave; a++)
        for (int b = -kWave; b <= kWave; b++) {
            if (a == 0 && b == 0) continue;
            const double k1 = 2 * kPi * a, k2 = 2 * kPi * b, k = sqrt(k1 * k1 + k2 * k2);
            const double lb = exp(-k * k / (4 * xi2) - xi2 * z * z);
            const double tp = th_plus(k, xi, z), tm = th_minus(k, xi, z), ts = tp + tm, td = tp - tm;
            const double j00 = sp * lb * xi;
            const double j10 = kPi * ts / (4 * k);
            const double j20 = sp * lb / (4 * k * k * xi) +
                               kPi * (ts / (8 * k * k * k) - td * z / (8 * k * k) - ts / (16 * k * xi2));
            const double j12 = -kPi * ts * k / 4 + sp * lb * xi;
            const double j22 = kPi * (ts * k / (16 * xi2) + ts / (8 * k) + td * z / 8) - sp * lb / (4 * xi);
            const double k11 = -kPi * td / 4;
            const double k12 = kPi * (td / (16 * xi2) + ts * z / (8 * k));
            const double qi = 2 * (j00 / (4 * xi2) + j10);
            const double qxy = -2 * (j10 / (4 * xi2) + j20);
            const double qzz = -2 * (j12 / (4 * xi2) + j22);
            const double qim = -2 * (k11 / (4 * xi2) + k12);
            const double ph = k1 * r0[0] + k2 * r0[1], c = cos(ph), s = sin(ph);
            const double kv[2] = {k1, k2};
            for (int p = 0; p < 2; p++)
                for (int q = 0; q < 2; q++) G[p][q] += 4 * ((p == q ? qi : 0.0) + qxy * kv[p] * kv[q]) * c;
            G[2][2] += 4 * (qi + qzz) * c;
            for (int p = 0; p < 2; p++) {
                G[p][2] -= 4 * qim * kv[p] * s;
                G[2][p] -= 4 * qim * kv[p] * s;
            }
        }
    // k = 0 mode (x and y only)
    const double w0 = -4 * (kPi * z * erf(xi * z) + sp / (2 * xi) * exp(-xi2 * z * z));
    G[0][0] += w0;
    G[1][1] += w0;
}

}  // namespace ewald
}  // namespace stk
