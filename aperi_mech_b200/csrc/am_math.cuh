// am_math.cuh -- device-side 3x3 algebra and the material stress updates.
//
// Tensors are row-major a[i*3+j]. Every function is templated on the element
// arithmetic type T (double for the FP64 path, float for the mixed path). The
// neo-Hookean determinant and logarithm are always evaluated in FP64: near
// incompressibility log J is the most cancellation-prone quantity in the update.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace am {

enum MaterialKind : int32_t { kLinearElastic = 0, kNeoHookean = 1, kElasticSVK = 2 };

// 1/x: IEEE division in FP64; in the FP32 (mixed) path the fast single-precision
// division intrinsic (about 2 ulp), ample next to FP32 element arithmetic.
__device__ __forceinline__ double recip(double x) { return 1.0 / x; }
__device__ __forceinline__ float recip(float x) { return __fdividef(1.0f, x); }

template <typename T>
__device__ __forceinline__ T cof_inv3(const T* m, T* r, T det) {
    // r = adj(m) / det ; det supplied by the caller (see det3 / det_ap_im1).
    const T id = recip(det);
    r[0] = (m[4] * m[8] - m[5] * m[7]) * id;
    r[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    r[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    r[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    r[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    r[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    r[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
    return det;
}

// r = adj(m) (the transposed cofactor matrix): m r = det(m) I.
template <typename T>
__device__ __forceinline__ void adj3(const T* m, T* r) {
    r[0] = m[4] * m[8] - m[5] * m[7];
    r[1] = m[2] * m[7] - m[1] * m[8];
    r[2] = m[1] * m[5] - m[2] * m[4];
    r[3] = m[5] * m[6] - m[3] * m[8];
    r[4] = m[0] * m[8] - m[2] * m[6];
    r[5] = m[2] * m[3] - m[0] * m[5];
    r[6] = m[3] * m[7] - m[4] * m[6];
    r[7] = m[1] * m[6] - m[0] * m[7];
    r[8] = m[0] * m[4] - m[1] * m[3];
}

template <typename T>
__device__ __forceinline__ T det3(const T* m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) + m[1] * (m[5] * m[6] - m[3] * m[8]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// det(I + A) - 1 from the principal invariants of A (aperi-mech MathUtils.h:332-339).
template <typename T>
__device__ __forceinline__ double det_ap_im1(const T* A) {
    const double a00 = A[0], a01 = A[1], a02 = A[2], a10 = A[3], a11 = A[4], a12 = A[5], a20 = A[6], a21 = A[7],
                 a22 = A[8];
    return a00 + a11 + a22 - a01 * a10 * (1 + a22) + a00 * a11 * (1 + a22) - a02 * a20 * (1 + a11) -
           a12 * a21 * (1 + a00) + a00 * a22 + a11 * a22 + a01 * a12 * a20 + a02 * a10 * a21;
}

// log1p for the neo-Hookean log J. Near J = 1 (|x| <= 1/16, the usual range) the
// classical atanh form log1p(x) = 2 atanh(s) = 2 (s + s^3/3 + s^5/5 + ...), s = x/(2+x),
// truncated after s^11 (next term below 1e-19 relative), with 1/(2+x) from an FP32
// reciprocal refined by two Newton-Raphson steps; elsewhere CUDA's log1p.
__device__ __forceinline__ double log1p_nh(double x) {
    if (!(fabs(x) <= 0.0625)) return log1p(x);
    const double d = 2.0 + x;
    double r = static_cast<double>(__frcp_rn(static_cast<float>(d)));
    r = fma(r, fma(-d, r, 1.0), r);
    r = fma(r, fma(-d, r, 1.0), r);
    const double s = x * r, t = s * s;
    double p = 1.0 / 11.0;
    p = fma(p, t, 1.0 / 9.0);
    p = fma(p, t, 1.0 / 7.0);
    p = fma(p, t, 1.0 / 5.0);
    p = fma(p, t, 1.0 / 3.0);
    p = fma(p, t, 1.0);
    return 2.0 * s * p;
}

// First Piola-Kirchhoff stress P(H). Returns J (det F) for the neo-Hookean model
// (so callers can flag J <= 0) and 1 otherwise.
//   linear elastic  (LinearElastic.h:79-87): P = lambda tr(eps) I + 2 mu eps, eps = sym(H)
//   neo-Hookean     (NeoHooke.h:79-91):      tau = lambda log1p(J-1) I + mu (H H^T + H + H^T), P = tau F^-T
//   St-Venant-K.    (Elastic.h:70-78):       E = (H + H^T + H^T H)/2, S = lambda tr(E) I + 2 mu E, P = F S
// Neo-Hookean Kirchhoff stress tau = lambda log1p(J-1) I + mu (H H^T + H + H^T)
// (NeoHooke.h:79-91); returns J = det F (FP64).
// tau is symmetric: the upper triangle is formed and mirrored.
template <typename T>
__device__ __forceinline__ double nh_kirchhoff(T lambda, T mu, const T* H, T* tau) {
    const double Jm1 = det_ap_im1(H);
    const T lam_lnJ = T((double)lambda * log1p_nh(Jm1));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            const T hh = H[i * 3 + 0] * H[j * 3 + 0] + H[i * 3 + 1] * H[j * 3 + 1] + H[i * 3 + 2] * H[j * 3 + 2];
            tau[i * 3 + j] = mu * (hh + H[j * 3 + i] + H[i * 3 + j]) + (i == j ? lam_lnJ : T(0));
            if (j != i) tau[j * 3 + i] = tau[i * 3 + j];
        }
    return 1.0 + Jm1;
}

template <typename T>
__device__ __forceinline__ double stress(int32_t mat, T lambda, T mu, const T* H, T* P) {
    if (mat == kLinearElastic) {
        const T tr = H[0] + H[4] + H[8];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) P[i * 3 + j] = mu * (H[i * 3 + j] + H[j * 3 + i]) + (i == j ? lambda * tr : T(0));
        return 1.0;
    }
    T F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = H[k];
    F[0] += T(1);
    F[4] += T(1);
    F[8] += T(1);
    if (mat == kNeoHookean) {
        T tau[9];
        const double J = nh_kirchhoff(lambda, mu, H, tau);
        T Fi[9];
        cof_inv3(F, Fi, T(J));
        // P = tau F^-T : P_ij = sum_k tau_ik Fi_jk
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                P[i * 3 + j] = tau[i * 3 + 0] * Fi[j * 3 + 0] + tau[i * 3 + 1] * Fi[j * 3 + 1] + tau[i * 3 + 2] * Fi[j * 3 + 2];
        return J;
    }
    T E[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const T hth = H[0 * 3 + i] * H[0 * 3 + j] + H[1 * 3 + i] * H[1 * 3 + j] + H[2 * 3 + i] * H[2 * 3 + j];
            E[i * 3 + j] = T(0.5) * (H[i * 3 + j] + H[j * 3 + i] + hth);
        }
    const T trE = E[0] + E[4] + E[8];
    T S[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) S[k] = T(2) * mu * E[k];
    S[0] += lambda * trE;
    S[4] += lambda * trE;
    S[8] += lambda * trE;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            P[i * 3 + j] = F[i * 3 + 0] * S[0 * 3 + j] + F[i * 3 + 1] * S[1 * 3 + j] + F[i * 3 + 2] * S[2 * 3 + j];
    return 1.0;
}

// Directional derivative dP[L] at H (equal to the vector-Jacobian product since
// all three models are hyperelastic and dP/dH is major-symmetric), plus the
// contractions L : dP/dlambda and L : dP/dmu at fixed H. FP64 only.
__device__ __forceinline__ void stress_vjp(int32_t mat, double lambda, double mu, const double* H, const double* L,
                                           double* dP, double* l_dlam, double* l_dmu) {
    double F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = H[k];
    F[0] += 1.0;
    F[4] += 1.0;
    F[8] += 1.0;
    if (mat == kLinearElastic) {
        const double trL = L[0] + L[4] + L[8];
        const double trH = H[0] + H[4] + H[8];
        double sm = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int k = i * 3 + j;
                dP[k] = mu * (L[k] + L[j * 3 + i]) + (i == j ? lambda * trL : 0.0);
                sm += L[k] * (H[k] + H[j * 3 + i]);
            }
        *l_dlam = trL * trH;
        *l_dmu = sm;
        return;
    }
    if (mat == kNeoHookean) {
        // P = mu (F - F^-T) + lambda log J F^-T, so with d(F^-T) = -F^-T L^T F^-T:
        //   dP = mu L + (mu - lambda log J) F^-T L^T F^-T + lambda tr(F^-1 L) F^-T
        //   L : dP/dlambda = log J tr(F^-1 L),  L : dP/dmu = L : (F - F^-T)
        const double Jm1 = det_ap_im1(H);
        const double lnJ = log1p_nh(Jm1);
        double Fi[9];
        cof_inv3(F, Fi, 1.0 + Jm1);
        double trFiL = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int k = 0; k < 3; ++k) trFiL += Fi[i * 3 + k] * L[k * 3 + i];
        // T1 = L^T F^-T : T1_kj = sum_m L_mk Fi_jm ; then (F^-T T1)_ij = sum_k Fi_ki T1_kj
        double T1[9];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                T1[k * 3 + j] = L[0 * 3 + k] * Fi[j * 3 + 0] + L[1 * 3 + k] * Fi[j * 3 + 1] + L[2 * 3 + k] * Fi[j * 3 + 2];
        const double a = mu - lambda * lnJ, bt = lambda * trFiL;
        double sm = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int k = i * 3 + j;
                const double FiT = Fi[j * 3 + i];
                const double t = Fi[0 * 3 + i] * T1[0 * 3 + j] + Fi[1 * 3 + i] * T1[1 * 3 + j] + Fi[2 * 3 + i] * T1[2 * 3 + j];
                dP[k] = mu * L[k] + a * t + bt * FiT;
                sm += L[k] * (F[k] - FiT);
            }
        *l_dlam = lnJ * trFiL;
        *l_dmu = sm;
        return;
    }
    // St-Venant-Kirchhoff: P = F S ; dP = L S + F dS
    double E[9], dE[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double ftf = 0.0, d = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                ftf += F[k * 3 + i] * F[k * 3 + j];
                d += L[k * 3 + i] * F[k * 3 + j] + F[k * 3 + i] * L[k * 3 + j];
            }
            E[i * 3 + j] = 0.5 * ftf - (i == j ? 0.5 : 0.0);
            dE[i * 3 + j] = 0.5 * d;
        }
    const double trE = E[0] + E[4] + E[8];
    const double trdE = dE[0] + dE[4] + dE[8];
    double S[9], dS[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        S[k] = 2.0 * mu * E[k];
        dS[k] = 2.0 * mu * dE[k];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        S[i * 4] += lambda * trE;
        dS[i * 4] += lambda * trdE;
    }
    double sl = 0.0, sm = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double a = 0.0, fe = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                a += L[i * 3 + k] * S[k * 3 + j] + F[i * 3 + k] * dS[k * 3 + j];
                fe += F[i * 3 + k] * E[k * 3 + j];
            }
            dP[i * 3 + j] = a;
            sl += L[i * 3 + j] * trE * F[i * 3 + j];
            sm += L[i * 3 + j] * 2.0 * fe;
        }
    *l_dlam = sl;
    *l_dmu = sm;
}

}  // namespace am
