// am_oracle.cpp -- CPU FP64 restatement of aperi-mech's explicit-dynamics hot path.
//
// TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline). Nothing in
// the product links or calls this file. Every routine names the reference
// function it restates; the reference paths are relative to the aperi-mech
// source tree.
#include "am_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// 3x3 helpers, row-major a[i*3+j]
// ---------------------------------------------------------------------------
inline double det3(const double* m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// Adjugate inverse (the closed form Eigen uses for fixed 3x3 inverse()).
inline double inv3(const double* m, double* r) {
    const double c00 = m[4] * m[8] - m[5] * m[7];
    const double c01 = m[5] * m[6] - m[3] * m[8];
    const double c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    const double id = 1.0 / det;
    r[0] = c00 * id;
    r[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    r[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    r[3] = c01 * id;
    r[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    r[6] = c02 * id;
    r[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
    return det;
}

inline void matmul3(const double* a, const double* b, double* c) {  // c = a b
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c[i * 3 + j] = a[i * 3 + 0] * b[0 + j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
}
inline void matmul3_tN(const double* a, const double* b, double* c) {  // c = a^T b
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c[i * 3 + j] = a[0 + i] * b[0 + j] + a[3 + i] * b[3 + j] + a[6 + i] * b[6 + j];
}
inline void matmul3_Nt(const double* a, const double* b, double* c) {  // c = a b^T
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c[i * 3 + j] = a[i * 3 + 0] * b[j * 3 + 0] + a[i * 3 + 1] * b[j * 3 + 1] + a[i * 3 + 2] * b[j * 3 + 2];
}

// MathUtils.h:332-339 DetApIm1: det(I + A) - 1 from the principal invariants.
inline double det_ap_im1(const double* A) {
    const double a00 = A[0], a01 = A[1], a02 = A[2], a10 = A[3], a11 = A[4], a12 = A[5], a20 = A[6], a21 = A[7], a22 = A[8];
    return a00 + a11 + a22 - a01 * a10 * (1 + a22) + a00 * a11 * (1 + a22) - a02 * a20 * (1 + a11) -
           a12 * a21 * (1 + a00) + a00 * a22 + a11 * a22 + a01 * a12 * a20 + a02 * a10 * a21;
}

// Cofactor matrix det(F) F^-T: rows r1 x r2, r2 x r0, r0 x r1 of F's rows r0, r1, r2.
inline void cof3(const double* F, double* C) {
    for (int r = 0; r < 3; ++r) {
        const int a = (r + 1) % 3, c = (r + 2) % 3;
        for (int i = 0; i < 3; ++i) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
            C[r * 3 + i] = F[a * 3 + i1] * F[c * 3 + i2] - F[a * 3 + i2] * F[c * 3 + i1];
        }
    }
}

// ---------------------------------------------------------------------------
// Shape functions and Gauss quadrature
// ---------------------------------------------------------------------------
// ShapeFunctionsFunctorHex8.h:51-62 (node order :17-33).
void hex8_dN(const double xi[3], double* dN) {
    const double x = xi[0], y = xi[1], z = xi[2];
    const double t[24] = {
        -0.125 * (1.0 - y) * (1.0 - z), -0.125 * (1.0 - x) * (1.0 - z), -0.125 * (1.0 - x) * (1.0 - y),
        0.125 * (1.0 - y) * (1.0 - z),  -0.125 * (1.0 + x) * (1.0 - z), -0.125 * (1.0 + x) * (1.0 - y),
        0.125 * (1.0 + y) * (1.0 - z),  0.125 * (1.0 + x) * (1.0 - z),  -0.125 * (1.0 + x) * (1.0 + y),
        -0.125 * (1.0 + y) * (1.0 - z), 0.125 * (1.0 - x) * (1.0 - z),  -0.125 * (1.0 - x) * (1.0 + y),
        -0.125 * (1.0 - y) * (1.0 + z), -0.125 * (1.0 - x) * (1.0 + z), 0.125 * (1.0 - x) * (1.0 - y),
        0.125 * (1.0 - y) * (1.0 + z),  -0.125 * (1.0 + x) * (1.0 + z), 0.125 * (1.0 + x) * (1.0 - y),
        0.125 * (1.0 + y) * (1.0 + z),  0.125 * (1.0 + x) * (1.0 + z),  0.125 * (1.0 + x) * (1.0 + y),
        -0.125 * (1.0 + y) * (1.0 + z), 0.125 * (1.0 - x) * (1.0 + z),  0.125 * (1.0 - x) * (1.0 + y)};
    std::memcpy(dN, t, sizeof(t));
}

// ElementHexahedron8.h:105-117: 2x2x2 points at +-1/sqrt(3), weights 1, in node order.
void hex8_gauss_point(int gp, double xi[3]) {
    static const int s[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    const double loc = 1.0 / std::sqrt(3.0);
    for (int j = 0; j < 3; ++j) xi[j] = s[gp][j] * loc;
}

// ShapeFunctionsFunctorTet4.h:27-34.
const double kTet4dN[12] = {-1.0, -1.0, -1.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0};

// QuadratureGaussian.h:17-39 ComputeBMatrixAndWeight: J = X^T dN, B = dN J^-1, w = w_g det J.
template <int NN>
double gauss_bw(const double* X, const double* dN, double wg, double* B) {
    double J[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int a = 0; a < NN; ++a) s += X[a * 3 + i] * dN[a * 3 + j];
            J[i * 3 + j] = s;
        }
    double Ji[9];
    const double detJ = inv3(J, Ji);
    for (int a = 0; a < NN; ++a)
        for (int j = 0; j < 3; ++j)
            B[a * 3 + j] = dN[a * 3 + 0] * Ji[0 * 3 + j] + dN[a * 3 + 1] * Ji[1 * 3 + j] + dN[a * 3 + 2] * Ji[2 * 3 + j];
    return wg * detJ;
}

// ---------------------------------------------------------------------------
// Materials
// ---------------------------------------------------------------------------
// LinearElastic.h:79-87: eps = sym(H); P = lambda tr(eps) I + 2 mu eps.
// NeoHooke.h:79-91: tau = lambda log1p(J-1) I + mu (B - I); P = tau F^-T.
// Elastic.h:70-78 (St-Venant-Kirchhoff): E = 1/2(H + H^T + H^T H); S = 2 mu E + lambda trE I; P = (I+H) S.
void stress(int material, double lambda, double mu, const double* H, double* P) {
    if (material == OB_LINEAR_ELASTIC) {
        const double tr = H[0] + H[4] + H[8];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double eps = 0.5 * (H[i * 3 + j] + H[j * 3 + i]);
                P[i * 3 + j] = (i == j ? lambda * tr : 0.0) + 2.0 * mu * eps;
            }
    } else if (material == OB_NEO_HOOKEAN) {
        double HHt[9];
        matmul3_Nt(H, H, HHt);
        double BmI[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) BmI[i * 3 + j] = HHt[i * 3 + j] + H[j * 3 + i] + H[i * 3 + j];
        const double Jm1 = det_ap_im1(H);
        const double lnJ = std::log1p(Jm1);
        double tau[9];
        for (int k = 0; k < 9; ++k) tau[k] = mu * BmI[k];
        for (int i = 0; i < 3; ++i) tau[i * 4] += lambda * lnJ;
        double F[9], Fi[9];
        for (int k = 0; k < 9; ++k) F[k] = H[k];
        F[0] += 1.0; F[4] += 1.0; F[8] += 1.0;
        inv3(F, Fi);
        // P = tau * Fi^T
        matmul3_Nt(tau, Fi, P);
    } else {
        double HtH[9];
        matmul3_tN(H, H, HtH);
        double E[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) E[i * 3 + j] = 0.5 * (H[i * 3 + j] + H[j * 3 + i] + HtH[i * 3 + j]);
        const double trE = E[0] + E[4] + E[8];
        double S[9];
        for (int k = 0; k < 9; ++k) S[k] = 2.0 * mu * E[k];
        for (int i = 0; i < 3; ++i) S[i * 4] += lambda * trE;
        double F[9];
        for (int k = 0; k < 9; ++k) F[k] = H[k];
        F[0] += 1.0; F[4] += 1.0; F[8] += 1.0;
        matmul3(F, S, P);
    }
}

// Directional derivative dP[L] of the stress at H (equal to the VJP because all
// three models are hyperelastic, so dP/dH is major-symmetric), plus the partial
// derivatives of P with respect to lambda and mu (at fixed H).
void stress_tangent(int material, double lambda, double mu, const double* H, const double* L,
                    double* dP, double* dPdlam, double* dPdmu) {
    double F[9];
    for (int k = 0; k < 9; ++k) F[k] = H[k];
    F[0] += 1.0; F[4] += 1.0; F[8] += 1.0;
    if (material == OB_LINEAR_ELASTIC) {
        const double trL = L[0] + L[4] + L[8];
        const double trH = H[0] + H[4] + H[8];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const int k = i * 3 + j;
                dP[k] = (i == j ? lambda * trL : 0.0) + mu * (L[k] + L[j * 3 + i]);
                dPdlam[k] = (i == j ? trH : 0.0);
                dPdmu[k] = H[k] + H[j * 3 + i];
            }
    } else if (material == OB_NEO_HOOKEAN) {
        double Fi[9];
        inv3(F, Fi);
        const double lnJ = std::log1p(det_ap_im1(H));
        double FiL[9];
        matmul3(Fi, L, FiL);
        const double trFiL = FiL[0] + FiL[4] + FiL[8];
        double LFt[9], FLt[9];
        matmul3_Nt(L, F, LFt);
        matmul3_Nt(F, L, FLt);
        double dtau[9];
        for (int k = 0; k < 9; ++k) dtau[k] = mu * (LFt[k] + FLt[k]);
        for (int i = 0; i < 3; ++i) dtau[i * 4] += lambda * trFiL;
        double FiT[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) FiT[i * 3 + j] = Fi[j * 3 + i];
        double P[9];
        stress(material, lambda, mu, H, P);
        double t1[9], PLt[9], t2[9];
        matmul3(dtau, FiT, t1);
        matmul3_Nt(P, L, PLt);
        matmul3(PLt, FiT, t2);
        for (int k = 0; k < 9; ++k) dP[k] = t1[k] - t2[k];
        for (int k = 0; k < 9; ++k) {
            dPdlam[k] = lnJ * FiT[k];
            dPdmu[k] = F[k] - FiT[k];
        }
    } else {
        double E[9], FtF[9];
        matmul3_tN(F, F, FtF);
        for (int k = 0; k < 9; ++k) E[k] = 0.5 * FtF[k];
        E[0] -= 0.5; E[4] -= 0.5; E[8] -= 0.5;
        const double trE = E[0] + E[4] + E[8];
        double S[9];
        for (int k = 0; k < 9; ++k) S[k] = 2.0 * mu * E[k];
        for (int i = 0; i < 3; ++i) S[i * 4] += lambda * trE;
        double LtF[9], FtL[9];
        matmul3_tN(L, F, LtF);
        matmul3_tN(F, L, FtL);
        double dE[9];
        for (int k = 0; k < 9; ++k) dE[k] = 0.5 * (LtF[k] + FtL[k]);
        const double trdE = dE[0] + dE[4] + dE[8];
        double dS[9];
        for (int k = 0; k < 9; ++k) dS[k] = 2.0 * mu * dE[k];
        for (int i = 0; i < 3; ++i) dS[i * 4] += lambda * trdE;
        double a[9], b[9], FE[9];
        matmul3(L, S, a);
        matmul3(F, dS, b);
        matmul3(F, E, FE);
        for (int k = 0; k < 9; ++k) {
            dP[k] = a[k] + b[k];
            dPdlam[k] = trE * F[k];
            dPdmu[k] = 2.0 * FE[k];
        }
    }
}

inline void block_lame(const ob_block& b, int64_t e, double* lambda, double* mu) {
    if (b.mu_field != nullptr || b.kappa_field != nullptr) {
        const double mu0 = b.mu;
        const double kappa0 = b.lambda + 2.0 * b.mu / 3.0;
        const double m = b.mu_field ? b.mu_field[e] : mu0;
        const double k = b.kappa_field ? b.kappa_field[e] : kappa0;
        *mu = m;
        *lambda = k - 2.0 * m / 3.0;
    } else {
        *lambda = b.lambda;
        *mu = b.mu;
    }
}

int nodes_per_elem(int kind) { return kind == OB_HEX8_GAUSS ? 8 : 4; }

// Per element: the force contributions of its nodes (ComputeInternalForceGaussian.h:57-131;
// force.row(i) -= B.row(i) * P^T * w, accumulated over the Gauss points in order).
void gauss_element_force(const ob_block& b, int64_t e, const double* coords, const double* u, double* fe) {
    const int nn = nodes_per_elem(b.kind);
    double X[24], U[24];
    for (int a = 0; a < nn; ++a) {
        const int32_t n = b.conn[e * nn + a];
        for (int i = 0; i < 3; ++i) {
            X[a * 3 + i] = coords[n * 3 + i];
            U[a * 3 + i] = u[n * 3 + i];
        }
    }
    double lambda, mu;
    block_lame(b, e, &lambda, &mu);
    for (int k = 0; k < nn * 3; ++k) fe[k] = 0.0;
    const int ngp = (b.kind == OB_HEX8_GAUSS) ? 8 : 1;
    for (int gp = 0; gp < ngp; ++gp) {
        double B[24], w;
        if (b.kind == OB_HEX8_GAUSS) {
            double xi[3], dN[24];
            hex8_gauss_point(gp, xi);
            hex8_dN(xi, dN);
            w = gauss_bw<8>(X, dN, 1.0, B);
        } else {
            w = gauss_bw<4>(X, kTet4dN, 1.0 / 6.0, B);
        }
        // ComputeInternalForceBase.h:158-174 (Total Lagrangian): H = u^T B.
        double H[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
                for (int a = 0; a < nn; ++a) s += U[a * 3 + i] * B[a * 3 + j];
                H[i * 3 + j] = s;
            }
        double P[9];
        stress(b.material, lambda, mu, H, P);
        for (int a = 0; a < nn; ++a)
            for (int i = 0; i < 3; ++i) {
                const double t = B[a * 3 + 0] * P[i * 3 + 0] + B[a * 3 + 1] * P[i * 3 + 1] + B[a * 3 + 2] * P[i * 3 + 2];
                fe[a * 3 + i] -= t * w;
            }
    }
}

// Updated / semi-Lagrangian Gauss element (ComputeInternalForceGaussian.h:57-131 with
// ComputeInternalForceBase.h:158-174): B and w on the coordinates x (current or reference
// configuration), dH = inc^T B, H = dH + Href + dH Href stored per element (each Gauss
// point overwrites it, so the last one remains), P(H), then B F_ref and w / det F_ref with
// F_ref = I + Href (Href the element's, for every Gauss point).
void gauss_element_force_lagr(const ob_block& b, int64_t e, const double* coords, const double* inc,
                              const double* Href, double* Hout, double* fe) {
    const int nn = nodes_per_elem(b.kind);
    double X[24], U[24];
    for (int a = 0; a < nn; ++a) {
        const int32_t n = b.conn[e * nn + a];
        for (int i = 0; i < 3; ++i) {
            X[a * 3 + i] = coords[n * 3 + i];
            U[a * 3 + i] = inc[n * 3 + i];
        }
    }
    double lambda, mu;
    block_lame(b, e, &lambda, &mu);
    for (int k = 0; k < nn * 3; ++k) fe[k] = 0.0;
    double Fr[9];
    for (int k = 0; k < 9; ++k) Fr[k] = Href[k] + ((k % 4 == 0) ? 1.0 : 0.0);
    const double detFr = Fr[0] * (Fr[4] * Fr[8] - Fr[5] * Fr[7]) - Fr[1] * (Fr[3] * Fr[8] - Fr[5] * Fr[6]) +
                         Fr[2] * (Fr[3] * Fr[7] - Fr[4] * Fr[6]);
    const int ngp = (b.kind == OB_HEX8_GAUSS) ? 8 : 1;
    for (int gp = 0; gp < ngp; ++gp) {
        double B[24], w;
        if (b.kind == OB_HEX8_GAUSS) {
            double xi[3], dN[24];
            hex8_gauss_point(gp, xi);
            hex8_dN(xi, dN);
            w = gauss_bw<8>(X, dN, 1.0, B);
        } else {
            w = gauss_bw<4>(X, kTet4dN, 1.0 / 6.0, B);
        }
        double dH[9], H[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double t = 0.0;
                for (int a = 0; a < nn; ++a) t += U[a * 3 + i] * B[a * 3 + j];
                dH[i * 3 + j] = t;
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double t = 0.0;
                for (int k = 0; k < 3; ++k) t += dH[i * 3 + k] * Href[k * 3 + j];
                H[i * 3 + j] = dH[i * 3 + j] + Href[i * 3 + j] + t;
            }
        for (int k = 0; k < 9; ++k) Hout[k] = H[k];
        double P[9];
        stress(b.material, lambda, mu, H, P);
        const double wr = w / detFr;
        for (int a = 0; a < nn; ++a) {
            double Br[3];
            for (int j = 0; j < 3; ++j) Br[j] = B[a * 3 + 0] * Fr[0 * 3 + j] + B[a * 3 + 1] * Fr[1 * 3 + j] + B[a * 3 + 2] * Fr[2 * 3 + j];
            for (int i = 0; i < 3; ++i) {
                const double t = Br[0] * P[i * 3 + 0] + Br[1] * P[i * 3 + 1] + Br[2] * P[i * 3 + 2];
                fe[a * 3 + i] -= t * wr;
            }
        }
    }
}

// ComputeInternalForceSmoothedCell.h:86-117 (H gather), :186-224 (stress), :312-351 (force):
// H = sum_k u_k (x) b_k ; f_k += b_k (-V P^T).
void cell_force(const ob_block& b, int64_t c, const double* u, double* fk) {
    const int64_t s0 = b.cell_ptr[c], s1 = b.cell_ptr[c + 1];
    double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t s = s0; s < s1; ++s) {
        const int32_t n = b.cell_nodes[s];
        const double* g = b.cell_grads + 3 * s;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) H[i * 3 + j] += u[n * 3 + i] * g[j];
    }
    double lambda, mu;
    block_lame(b, c, &lambda, &mu);
    double P[9];
    stress(b.material, lambda, mu, H, P);
    const double V = b.cell_volumes[c];
    double st[9];  // stress_term = P^T * -V
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) st[i * 3 + j] = P[j * 3 + i] * -V;
    for (int64_t s = s0; s < s1; ++s) {
        const double* g = b.cell_grads + 3 * s;
        for (int i = 0; i < 3; ++i) fk[(s - s0) * 3 + i] = g[0] * st[0 * 3 + i] + g[1] * st[1 * 3 + i] + g[2] * st[2 * 3 + i];
    }
}

// F-bar smoothed cells (ForEachCellComputeForceFbar, ComputeInternalForceSmoothedCell.h:354-413),
// one cell g of subcells s in [group_ptr[g], group_ptr[g+1]):
//   H_s = sum_k u_k (x) b_k, J_s = DetApIm1(H_s) + 1                     (:86-117)
//   Jbar = sum_s J_s V_s / V_g, V_g = sum_s V_s                          (:120-148)
//   Hbar_s = js H_s + (js - 1) I, js = cbrt(Jbar / J_s), H itself when
//            |Jbar / J_s - 1| < 3 eps                                    (:150-183)
//   Pbar_s = P(Hbar_s)                                                   (:186-224)
//   p = sum_s js / (3 Jbar) V_s (Pbar_s : H_s + tr Pbar_s) / V_g          (:227-264)
//   P_s = js Pbar_s + (p - js / (3 J_s) Pbar_s : F_s) J_s F_s^-T          (:266-309)
//   f_k += b_k (-V_s P_s^T)                                              (:312-351)
void fbar_cell_forces(const ob_block& b, int64_t g, const double* u, double* slots) {
    const int64_t s0 = b.group_ptr[g], s1 = b.group_ptr[g + 1];
    if (s1 <= s0) return;
    const int64_t n = s1 - s0;
    std::vector<double> H(9 * n), J(n), js(n), Pb(9 * n);
    double Vg = 0.0, jv = 0.0;
    for (int64_t s = s0; s < s1; ++s) {
        double* h = &H[9 * (s - s0)];
        std::fill(h, h + 9, 0.0);
        for (int64_t e = b.cell_ptr[s]; e < b.cell_ptr[s + 1]; ++e) {
            const int32_t nd = b.cell_nodes[e];
            const double* gr = b.cell_grads + 3 * e;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) h[i * 3 + j] += u[nd * 3 + i] * gr[j];
        }
        J[s - s0] = det_ap_im1(h) + 1.0;
        jv += J[s - s0] * b.cell_volumes[s];
        Vg += b.cell_volumes[s];
    }
    const double Jbar = jv / Vg;
    double p = 0.0;
    for (int64_t s = s0; s < s1; ++s) {
        const int64_t q = s - s0;
        const double* h = &H[9 * q];
        const double ratio = Jbar / J[q];
        js[q] = std::cbrt(ratio);
        double hb[9];
        if (std::abs(ratio - 1.0) < 3.0 * 2.2204460492503131e-16) {
            std::copy(h, h + 9, hb);
        } else {
            for (int k = 0; k < 9; ++k) hb[k] = h[k] * js[q];
            for (int i = 0; i < 3; ++i) hb[i * 4] += js[q] - 1.0;
        }
        double lambda, mu;
        block_lame(b, s, &lambda, &mu);
        stress(b.material, lambda, mu, hb, &Pb[9 * q]);
        const double* P = &Pb[9 * q];
        double pf = P[0] + P[4] + P[8];
        for (int k = 0; k < 9; ++k) pf += P[k] * h[k];
        p += js[q] / (3.0 * Jbar) * b.cell_volumes[s] * pf;
    }
    p /= Vg;
    for (int64_t s = s0; s < s1; ++s) {
        const int64_t q = s - s0;
        const double* h = &H[9 * q];
        const double* Pbar = &Pb[9 * q];
        double F[9];
        std::copy(h, h + 9, F);
        F[0] += 1.0;
        F[4] += 1.0;
        F[8] += 1.0;
        double pf = 0.0;
        for (int k = 0; k < 9; ++k) pf += Pbar[k] * F[k];
        const double scal = (p - js[q] / (3.0 * J[q]) * pf) * J[q];
        // F^-T: (F^-T)_ij = cof(F)_ij / det F
        const double cof[9] = {F[4] * F[8] - F[5] * F[7], F[5] * F[6] - F[3] * F[8], F[3] * F[7] - F[4] * F[6],
                               F[2] * F[7] - F[1] * F[8], F[0] * F[8] - F[2] * F[6], F[1] * F[6] - F[0] * F[7],
                               F[1] * F[5] - F[2] * F[4], F[2] * F[3] - F[0] * F[5], F[0] * F[4] - F[1] * F[3]};
        double P[9];
        for (int k = 0; k < 9; ++k) P[k] = Pbar[k] * js[q] + scal * cof[k] / J[q];
        const double V = b.cell_volumes[s];
        for (int64_t e = b.cell_ptr[s]; e < b.cell_ptr[s + 1]; ++e) {
            const double* gr = b.cell_grads + 3 * e;
            for (int i = 0; i < 3; ++i)
                slots[e * 3 + i] = (gr[0] * P[i * 3 + 0] + gr[1] * P[i * 3 + 1] + gr[2] * P[i * 3 + 2]) * -V;
        }
    }
}

// VJP of the F-bar cell forces of one cell g (the adjoint extension; the reference has
// none). The forces above are f = -dW/du of W = sum_s V_s psi(Fbar_s), with
// Fbar_s = js F_s, js = cbrt(Jbar / J_s): P_s above is dW/dF_s / V_s. The Hessian of W
// is symmetric, so lam^T df/du is the derivative of f along L_s = sum_k lam_k (x) b_k:
//   dJ_s = cof(F_s) : L_s, dJbar = sum_s V_s dJ_s / V_g,
//   djs = js / 3 (dJbar / Jbar - dJ_s / J_s), dFbar = djs F + js L,
//   dPbar = dP/dF(Hbar)[dFbar], pf = Pbar : F, dpf = dPbar : F + Pbar : L,
//   dp = sum_s V_s (djs pf + js dpf - js pf dJbar / Jbar) / (3 Jbar) / V_g,
//   dscal = dp - (djs pf + js dpf) / (3 J) + js pf dJ / (3 J^2),
//   dP = djs Pbar + js dPbar + dscal cof(F) + scal dcof(F)[L]
// and slots get -V_s b_k dP^T. lam^T f = -dW[L] = -sum_s V_s Pbar_s : dFbar_s, so the
// moduli of subcell s enter only through Pbar_s: d(lam^T f)/dtheta_s = -V_s dPbar/dtheta : dFbar.
void fbar_cell_vjp(const ob_block& b, int64_t g, const double* u, const double* lam, double* slots, double* gmu,
                   double* gkappa) {
    const int64_t s0 = b.group_ptr[g], s1 = b.group_ptr[g + 1];
    if (s1 <= s0) return;
    const int64_t n = s1 - s0;
    std::vector<double> H(9 * n), L(9 * n), J(n), dJ(n), G(9 * n);
    double Vg = 0.0, jv = 0.0, djv = 0.0;
    for (int64_t s = s0; s < s1; ++s) {
        const int64_t q = s - s0;
        double* h = &H[9 * q];
        double* l = &L[9 * q];
        std::fill(h, h + 9, 0.0);
        std::fill(l, l + 9, 0.0);
        for (int64_t e = b.cell_ptr[s]; e < b.cell_ptr[s + 1]; ++e) {
            const int32_t nd = b.cell_nodes[e];
            const double* gr = b.cell_grads + 3 * e;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    h[i * 3 + j] += u[nd * 3 + i] * gr[j];
                    l[i * 3 + j] += lam[nd * 3 + i] * gr[j];
                }
        }
        double F[9];
        std::copy(h, h + 9, F);
        F[0] += 1.0;
        F[4] += 1.0;
        F[8] += 1.0;
        cof3(F, &G[9 * q]);
        J[q] = det_ap_im1(h) + 1.0;
        dJ[q] = 0.0;
        for (int k = 0; k < 9; ++k) dJ[q] += G[9 * q + k] * l[k];
        jv += J[q] * b.cell_volumes[s];
        djv += dJ[q] * b.cell_volumes[s];
        Vg += b.cell_volumes[s];
    }
    const double Jbar = jv / Vg, dJbar = djv / Vg;
    std::vector<double> js(n), djs(n), Pb(9 * n), dPb(9 * n), pf(n), dpf(n);
    double p = 0.0, dp = 0.0;
    for (int64_t s = s0; s < s1; ++s) {
        const int64_t q = s - s0;
        const double* h = &H[9 * q];
        const double* l = &L[9 * q];
        const double ratio = Jbar / J[q];
        js[q] = std::cbrt(ratio);
        djs[q] = js[q] / 3.0 * (dJbar / Jbar - dJ[q] / J[q]);
        double hb[9];
        if (std::abs(ratio - 1.0) < 3.0 * 2.2204460492503131e-16) {
            std::copy(h, h + 9, hb);
        } else {
            for (int k = 0; k < 9; ++k) hb[k] = h[k] * js[q];
            for (int i = 0; i < 3; ++i) hb[i * 4] += js[q] - 1.0;
        }
        double F[9], dFb[9];
        std::copy(h, h + 9, F);
        F[0] += 1.0;
        F[4] += 1.0;
        F[8] += 1.0;
        for (int k = 0; k < 9; ++k) dFb[k] = djs[q] * F[k] + js[q] * l[k];
        double lambda, mu;
        block_lame(b, s, &lambda, &mu);
        double dPl[9], dPm[9];
        stress(b.material, lambda, mu, hb, &Pb[9 * q]);
        stress_tangent(b.material, lambda, mu, hb, dFb, &dPb[9 * q], dPl, dPm);
        double sl = 0.0, sm = 0.0;
        pf[q] = dpf[q] = 0.0;
        for (int k = 0; k < 9; ++k) {
            sl += dFb[k] * dPl[k];
            sm += dFb[k] * dPm[k];
            pf[q] += Pb[9 * q + k] * F[k];
            dpf[q] += dPb[9 * q + k] * F[k] + Pb[9 * q + k] * l[k];
        }
        const double V = b.cell_volumes[s];
        // lambda = kappa - 2/3 mu, as in add_block_vjp
        if (gmu) gmu[s] = -V * (sm - 2.0 / 3.0 * sl);
        if (gkappa) gkappa[s] = -V * sl;
        p += V * js[q] * pf[q] / (3.0 * Jbar);
        dp += V * (djs[q] * pf[q] + js[q] * dpf[q] - js[q] * pf[q] * dJbar / Jbar) / (3.0 * Jbar);
    }
    p /= Vg;
    dp /= Vg;
    for (int64_t s = s0; s < s1; ++s) {
        const int64_t q = s - s0;
        const double* h = &H[9 * q];
        const double* l = &L[9 * q];
        double F[9];
        std::copy(h, h + 9, F);
        F[0] += 1.0;
        F[4] += 1.0;
        F[8] += 1.0;
        const double scal = p - js[q] * pf[q] / (3.0 * J[q]);
        const double dscal = dp - (djs[q] * pf[q] + js[q] * dpf[q]) / (3.0 * J[q]) +
                             js[q] * pf[q] * dJ[q] / (3.0 * J[q] * J[q]);
        // cof(F) rows are r1 x r2, r2 x r0, r0 x r1 of F's rows: its derivative along L
        double dG[9];
        for (int r = 0; r < 3; ++r) {
            const int a = (r + 1) % 3, c = (r + 2) % 3;
            for (int i = 0; i < 3; ++i) {
                const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
                dG[r * 3 + i] = l[a * 3 + i1] * F[c * 3 + i2] - l[a * 3 + i2] * F[c * 3 + i1] +
                                F[a * 3 + i1] * l[c * 3 + i2] - F[a * 3 + i2] * l[c * 3 + i1];
            }
        }
        double dP[9];
        for (int k = 0; k < 9; ++k)
            dP[k] = djs[q] * Pb[9 * q + k] + js[q] * dPb[9 * q + k] + dscal * G[9 * q + k] + scal * dG[k];
        const double V = b.cell_volumes[s];
        for (int64_t e = b.cell_ptr[s]; e < b.cell_ptr[s + 1]; ++e) {
            const double* gr = b.cell_grads + 3 * e;
            for (int i = 0; i < 3; ++i)
                slots[e * 3 + i] = (gr[0] * dP[i * 3 + 0] + gr[1] * dP[i * 3 + 1] + gr[2] * dP[i * 3 + 2]) * -V;
        }
    }
}

void add_block_forces(const ob_problem* p, const ob_block& b, const double* u, double* f) {
    if (b.kind == OB_CELLS) {
        const int64_t K = b.cell_ptr[b.num_elems];
        std::vector<double> slots(static_cast<size_t>(K) * 3);
        if (b.group_ptr) {
#pragma omp parallel for schedule(dynamic, 16)
            for (int64_t g = 0; g < b.num_groups; ++g) fbar_cell_forces(b, g, u, slots.data());
        } else {
#pragma omp parallel for schedule(static)
            for (int64_t c = 0; c < b.num_elems; ++c) cell_force(b, c, u, slots.data() + 3 * b.cell_ptr[c]);
        }
        // Scatter in entry order (Field::AtomicAdd in the reference; deterministic here).
        for (int64_t s = 0; s < K; ++s) {
            const int32_t n = b.cell_nodes[s];
            for (int i = 0; i < 3; ++i) f[n * 3 + i] += slots[s * 3 + i];
        }
        return;
    }
    const int nn = nodes_per_elem(b.kind);
    std::vector<double> slots(static_cast<size_t>(b.num_elems) * nn * 3);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < b.num_elems; ++e) gauss_element_force(b, e, p->coords, u, slots.data() + e * nn * 3);
    for (int64_t e = 0; e < b.num_elems; ++e)
        for (int a = 0; a < nn; ++a) {
            const int32_t n = b.conn[e * nn + a];
            for (int i = 0; i < 3; ++i) f[n * 3 + i] += slots[(e * nn + a) * 3 + i];
        }
}

// ---------------------------------------------------------------------------
// Boundary-condition time functions (MathUtils.h, BoundaryCondition.cpp:86-195)
// ---------------------------------------------------------------------------
double constant_interp(double x, const double* ab, const double* ord, int n) {
    if (n == 1) return ord[0];
    if (x < ab[0]) return 0.0;
    if (x > ab[n - 1]) return ord[n - 1];
    for (int i = 0; i < n - 1; ++i)
        if (x >= ab[i] && x <= ab[i + 1]) return ord[i];
    return 0.0;
}
double linear_interp(double x, const double* ab, const double* ord, int n) {
    if (n == 1) return ord[0];
    if (x < ab[0]) return ord[0];
    if (x > ab[n - 1]) return ord[n - 1];
    for (int i = 0; i < n - 1; ++i)
        if (x >= ab[i] && x <= ab[i + 1]) {
            const double slope = (ord[i + 1] - ord[i]) / (ab[i + 1] - ab[i]);
            return ord[i] + slope * (x - ab[i]);
        }
    return 0.0;
}
double smooth_step_d1(double x, const double* ab, const double* ord, int n) {
    if (n == 1 || x < ab[0] || x > ab[n - 1]) return 0.0;
    for (int i = 0; i < n - 1; ++i)
        if (x >= ab[i] && x <= ab[i + 1]) {
            const double t = (x - ab[i]) / (ab[i + 1] - ab[i]);
            return (ord[i + 1] - ord[i]) * (30.0 * t * t - 60.0 * t * t * t + 30.0 * t * t * t * t) / (ab[i + 1] - ab[i]);
        }
    return 0.0;
}
double smooth_step_d2(double x, const double* ab, const double* ord, int n) {
    if (n == 1 || x < ab[0] || x > ab[n - 1]) return 0.0;
    for (int i = 0; i < n - 1; ++i)
        if (x >= ab[i] && x <= ab[i + 1]) {
            const double t = (x - ab[i]) / (ab[i + 1] - ab[i]);
            return (ord[i + 1] - ord[i]) * (60.0 * t - 180.0 * t * t + 120.0 * t * t * t) / ((ab[i + 1] - ab[i]) * (ab[i + 1] - ab[i]));
        }
    return 0.0;
}

// velocity (which=0) or acceleration (which=1) scale of a BC at time t.
double bc_scale(const ob_bc& bc, int which, double t) {
    const int n = bc.num_points;
    if (bc.time_function == OB_TF_RAMP) {
        std::vector<double> d(n);
        for (int i = 0; i < n - 1; ++i) d[i] = (bc.ordinate[i + 1] - bc.ordinate[i]) / (bc.abscissa[i + 1] - bc.abscissa[i]);
        d[n - 1] = 0.0;
        if (bc.kind == OB_BC_DISPLACEMENT) return which == 0 ? constant_interp(t, bc.abscissa, d.data(), n) : 0.0;
        return which == 0 ? linear_interp(t, bc.abscissa, bc.ordinate, n) : constant_interp(t, bc.abscissa, d.data(), n);
    }
    if (bc.kind == OB_BC_DISPLACEMENT)
        return which == 0 ? smooth_step_d1(t, bc.abscissa, bc.ordinate, n) : smooth_step_d2(t, bc.abscissa, bc.ordinate, n);
    // velocity smooth step: v = SmoothStep, a = SmoothStep'
    if (which == 0) {
        // SmoothStepInterpolation (MathUtils.h:187-208)
        if (n == 1 || t < bc.abscissa[0]) return bc.ordinate[0];
        if (t > bc.abscissa[n - 1]) return bc.ordinate[n - 1];
        for (int i = 0; i < n - 1; ++i)
            if (t >= bc.abscissa[i] && t <= bc.abscissa[i + 1]) {
                const double s = (t - bc.abscissa[i]) / (bc.abscissa[i + 1] - bc.abscissa[i]);
                return bc.ordinate[i] + (bc.ordinate[i + 1] - bc.ordinate[i]) * s * s * s * (10.0 - 15.0 * s + 6.0 * s * s);
            }
        return 0.0;
    }
    return smooth_step_d1(t, bc.abscissa, bc.ordinate, n);
}

// BoundaryCondition::ApplyVelocity / ApplyAcceleration: overwrite prescribed components.
void apply_bcs(const ob_problem* p, int which, double t, double* x) {
    for (int k = 0; k < p->num_bcs; ++k) {
        const ob_bc& bc = p->bcs[k];
        if (t < bc.active_start || t > bc.active_end) continue;
        const double s = bc_scale(bc, which, t);
        for (int c = 0; c < 3; ++c) {
            if (!(bc.component_mask & (1 << c))) continue;
            const double val = bc.values[c] * s;
            for (int64_t i = 0; i < bc.num_nodes; ++i) x[bc.nodes[i] * 3 + c] = val;
        }
    }
}

// 1 where the dof is free at time t (for the adjoint), 0 where a BC overwrites it.
void free_mask(const ob_problem* p, double t, std::vector<double>& m) {
    m.assign(static_cast<size_t>(p->num_nodes) * 3, 1.0);
    for (int k = 0; k < p->num_bcs; ++k) {
        const ob_bc& bc = p->bcs[k];
        if (t < bc.active_start || t > bc.active_end) continue;
        for (int c = 0; c < 3; ++c) {
            if (!(bc.component_mask & (1 << c))) continue;
            for (int64_t i = 0; i < bc.num_nodes; ++i) m[bc.nodes[i] * 3 + c] = 0.0;
        }
    }
}

void compute_acceleration(const ob_problem* p, const double* m, const double* u, double* f, double* a) {
    const int64_t N = p->num_nodes;
    ob_internal_force(p, u, f);
    const double* g = p->body_accel;
    if (g[0] != 0.0 || g[1] != 0.0 || g[2] != 0.0)
        for (int64_t n = 0; n < N; ++n)
            for (int i = 0; i < 3; ++i) f[n * 3 + i] += g[i] * m[n];
    // ExplicitTimeIntegrator.h:247-283: a = f / m.
#pragma omp parallel for schedule(static)
    for (int64_t n = 0; n < N; ++n)
        for (int i = 0; i < 3; ++i) a[n * 3 + i] = f[n * 3 + i] / m[n];
}

// One central-difference step in the order of ExplicitSolver::Solve (src/Solvers/Explicit.cpp:383-483).
void cd_step(const ob_problem* p, const double* m, double dtn, double time, double* u, double* v, double* a, double* f) {
    const int64_t N = p->num_nodes;
    const double half = 0.5 * dtn;
    const double t_mid = time + 0.5 * dtn;
    const double t_next = time + dtn;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < N * 3; ++k) v[k] = v[k] + half * a[k];  // :286-326
    apply_bcs(p, 0, t_mid, v);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < N * 3; ++k) u[k] = u[k] + dtn * v[k];  // :97-134
    compute_acceleration(p, m, u, f, a);
    apply_bcs(p, 1, t_next, a);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < N * 3; ++k) v[k] += half * a[k];  // :329-364
}

std::vector<double> mass_of(const ob_problem* p) {
    std::vector<double> m(static_cast<size_t>(p->num_nodes));
    if (p->mass)
        std::copy(p->mass, p->mass + p->num_nodes, m.begin());
    else
        ob_lumped_mass(p, m.data());
    return m;
}

// VJP of the internal force of one block, accumulating gu (nodes) and writing gmu/gkappa (elements).
void add_block_vjp(const ob_problem* p, const ob_block& b, const double* u, const double* lam, double* gu,
                   double* gmu, double* gkappa) {
    const bool cells = b.kind == OB_CELLS;
    if (cells && b.group_ptr) {
        std::vector<double> slots(static_cast<size_t>(b.cell_ptr[b.num_elems]) * 3, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t g = 0; g < b.num_groups; ++g) fbar_cell_vjp(b, g, u, lam, slots.data(), gmu, gkappa);
        for (int64_t s = 0; s < b.num_elems; ++s)
            for (int64_t e = b.cell_ptr[s]; e < b.cell_ptr[s + 1]; ++e)
                for (int i = 0; i < 3; ++i) gu[b.cell_nodes[e] * 3 + i] += slots[e * 3 + i];
        return;
    }
    const int nn = cells ? 0 : nodes_per_elem(b.kind);
    std::vector<int64_t> start(b.num_elems + 1);
    for (int64_t e = 0; e <= b.num_elems; ++e) start[e] = cells ? b.cell_ptr[e] : e * nn;
    std::vector<double> slots(static_cast<size_t>(start[b.num_elems]) * 3, 0.0);
    std::vector<int32_t> dummy;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < b.num_elems; ++e) {
        double lambda, mu;
        block_lame(b, e, &lambda, &mu);
        double gl = 0.0, gm = 0.0;
        const int64_t s0 = start[e], s1 = start[e + 1];
        const int64_t ne = s1 - s0;
        std::vector<double> Bv(static_cast<size_t>(ne) * 3);
        std::vector<int32_t> nodes(ne);
        for (int64_t s = 0; s < ne; ++s) nodes[s] = cells ? b.cell_nodes[s0 + s] : b.conn[s0 + s];
        const int ngp = cells ? 1 : (b.kind == OB_HEX8_GAUSS ? 8 : 1);
        double X[24];
        if (!cells)
            for (int a = 0; a < nn; ++a)
                for (int i = 0; i < 3; ++i) X[a * 3 + i] = p->coords[nodes[a] * 3 + i];
        for (int gp = 0; gp < ngp; ++gp) {
            double w;
            if (cells) {
                for (int64_t s = 0; s < ne * 3; ++s) Bv[s] = b.cell_grads[s0 * 3 + s];
                w = b.cell_volumes[e];
            } else if (b.kind == OB_HEX8_GAUSS) {
                double xi[3], dN[24];
                hex8_gauss_point(gp, xi);
                hex8_dN(xi, dN);
                w = gauss_bw<8>(X, dN, 1.0, Bv.data());
            } else {
                w = gauss_bw<4>(X, kTet4dN, 1.0 / 6.0, Bv.data());
            }
            double H[9] = {0}, L[9] = {0};
            for (int64_t s = 0; s < ne; ++s)
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        H[i * 3 + j] += u[nodes[s] * 3 + i] * Bv[s * 3 + j];
                        L[i * 3 + j] += lam[nodes[s] * 3 + i] * Bv[s * 3 + j];
                    }
            double dP[9], dPl[9], dPm[9];
            stress_tangent(b.material, lambda, mu, H, L, dP, dPl, dPm);
            double sl = 0.0, sm = 0.0;
            for (int k = 0; k < 9; ++k) {
                sl += L[k] * dPl[k];
                sm += L[k] * dPm[k];
            }
            gl -= w * sl;
            gm -= w * sm;
            for (int64_t s = 0; s < ne; ++s)
                for (int i = 0; i < 3; ++i)
                    slots[(s0 + s) * 3 + i] -= w * (Bv[s * 3 + 0] * dP[i * 3 + 0] + Bv[s * 3 + 1] * dP[i * 3 + 1] + Bv[s * 3 + 2] * dP[i * 3 + 2]);
        }
        // lambda = kappa - 2/3 mu  =>  d/dmu|kappa = d/dmu|lambda - 2/3 d/dlambda ; d/dkappa = d/dlambda
        if (gmu) gmu[e] = gm - 2.0 / 3.0 * gl;
        if (gkappa) gkappa[e] = gl;
    }
    for (int64_t e = 0; e < b.num_elems; ++e)
        for (int64_t s = start[e]; s < start[e + 1]; ++s) {
            const int32_t n = cells ? b.cell_nodes[s] : b.conn[s];
            for (int i = 0; i < 3; ++i) gu[n * 3 + i] += slots[s * 3 + i];
        }
}

// 4x4 inverse by Gauss-Jordan elimination with partial pivoting (stands in for
// Eigen's fullPivLu().inverse() used by InvertMatrix<4>, MathUtils.h:307-319).
bool inv4(const double* M, double* R) {
    double A[4][8];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            A[i][j] = M[i * 4 + j];
            A[i][j + 4] = (i == j) ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
        if (A[piv][c] == 0.0) return false;
        if (piv != c)
            for (int j = 0; j < 8; ++j) std::swap(A[c][j], A[piv][j]);
        const double d = 1.0 / A[c][c];
        for (int j = 0; j < 8; ++j) A[c][j] *= d;
        for (int r = 0; r < 4; ++r) {
            if (r == c) continue;
            const double fct = A[r][c];
            if (fct == 0.0) continue;
            for (int j = 0; j < 8; ++j) A[r][j] -= fct * A[c][j];
        }
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) R[i * 4 + j] = A[i][j + 4];
    return true;
}

}  // namespace

extern "C" {

void ob_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ob_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void ob_tet4_gauss_bw(const double X[12], double B[12], double* w) { *w = gauss_bw<4>(X, kTet4dN, 1.0 / 6.0, B); }

void ob_hex8_gauss_bw(const double X[24], int gp, double B[24], double* w) {
    double xi[3], dN[24];
    hex8_gauss_point(gp, xi);
    hex8_dN(xi, dN);
    *w = gauss_bw<8>(X, dN, 1.0, B);
}

// QuadratureSmoothed.h:32-63 (Tet4, area-weighted face normals, Seacas face order).
void ob_tet4_smoothed_bw(const double X[12], double B[12], double* volume) {
    static const int faces[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 3, 2}, {0, 2, 1}};
    for (int k = 0; k < 12; ++k) B[k] = 0.0;
    double vol = 0.0;
    for (int j = 0; j < 4; ++j) {
        const double* p0 = X + 3 * faces[j][0];
        const double* p1 = X + 3 * faces[j][1];
        const double* p2 = X + 3 * faces[j][2];
        const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
        const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
        const double nrm[3] = {(e1[1] * e2[2] - e1[2] * e2[1]) / 2.0, (e1[2] * e2[0] - e1[0] * e2[2]) / 2.0,
                               (e1[0] * e2[1] - e1[1] * e2[0]) / 2.0};
        vol += p0[0] * nrm[0] + p0[1] * nrm[1] + p0[2] * nrm[2];
        for (int l = 0; l < 3; ++l)
            for (int i = 0; i < 3; ++i) B[faces[j][l] * 3 + i] += nrm[i] / 3.0;
    }
    vol /= 3.0;
    for (int k = 0; k < 12; ++k) B[k] /= vol;
    *volume = vol;
}

// QuadratureSmoothed.h:97-142 (Hex8, each quad face split into 4 triangles about its mid point).
void ob_hex8_smoothed_bw(const double X[24], double B[24], double* volume) {
    static const int faces[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
    for (int k = 0; k < 24; ++k) B[k] = 0.0;
    double vol = 0.0;
    for (int j = 0; j < 6; ++j) {
        double mid[3] = {0, 0, 0};
        for (int k = 0; k < 4; ++k)
            for (int i = 0; i < 3; ++i) mid[i] += X[faces[j][k] * 3 + i];
        for (int i = 0; i < 3; ++i) mid[i] /= 4.0;
        int km1 = 3;
        for (int k = 0; k < 4; ++k) {
            double e1[3], e2[3];
            for (int i = 0; i < 3; ++i) {
                e1[i] = X[faces[j][km1] * 3 + i] - mid[i];
                e2[i] = X[faces[j][k] * 3 + i] - mid[i];
            }
            const double nrm[3] = {(e1[1] * e2[2] - e1[2] * e2[1]) / 2.0, (e1[2] * e2[0] - e1[0] * e2[2]) / 2.0,
                                   (e1[0] * e2[1] - e1[1] * e2[0]) / 2.0};
            vol += mid[0] * nrm[0] + mid[1] * nrm[1] + mid[2] * nrm[2];
            for (int l = 0; l < 4; ++l) {
                const double wgt = (l == k || l == km1) ? 5.0 / 12.0 : 1.0 / 12.0;
                for (int i = 0; i < 3; ++i) B[faces[j][l] * 3 + i] += nrm[i] * wgt;
            }
            km1 = k;
        }
    }
    vol /= 3.0;
    for (int k = 0; k < 24; ++k) B[k] /= vol;
    *volume = vol;
}

// Materials/Base.h:47-158 LinearElasticProperties::CompleteProperties + CheckPhysicalBounds.
int ob_complete_properties(double props[5], char* msg, int msg_len) {
    double& E = props[0];
    double& nu = props[1];
    double& G = props[2];
    double& lam = props[3];
    double& K = props[4];
    auto def = [](double x) { return !std::isnan(x); };
    const int count = def(E) + def(nu) + def(G) + def(lam) + def(K);
    auto fail = [&](const char* m) {
        if (msg && msg_len > 0) std::snprintf(msg, msg_len, "%s", m);
        return -1;
    };
    if (count != 2) {
        char buf[96];
        std::snprintf(buf, sizeof(buf), "Exactly two properties must be defined. Defined: %d", count);
        return fail(buf);
    }
    if (def(K) && def(E)) {
        nu = (3 * K - E) / (6 * K);
        G = E / (2 * (1 + nu));
        lam = (E * nu) / ((1 + nu) * (1 - 2 * nu));
    } else if (def(K) && def(lam)) {
        G = (3 * (K - lam)) / 2;
        nu = lam / (2 * (lam + G));
        E = 2 * G * (1 + nu);
    } else if (def(K) && def(G)) {
        lam = K - (2.0 / 3.0) * G;
        nu = lam / (2 * (lam + G));
        E = 2 * G * (1 + nu);
    } else if (def(K) && def(nu)) {
        E = 3 * K * (1 - 2 * nu);
        G = E / (2 * (1 + nu));
        lam = (E * nu) / ((1 + nu) * (1 - 2 * nu));
    } else if (def(E) && def(lam)) {
        const double a = 2 * lam, b = lam + E, c = -lam;
        const double disc = b * b - 4 * a * c;
        nu = (-b + std::sqrt(disc)) / (2 * a);
        G = E / (2 * (1 + nu));
        K = lam + (2.0 / 3.0) * G;
    } else if (def(E) && def(G)) {
        nu = (E / (2 * G)) - 1;
        lam = (E * nu) / ((1 + nu) * (1 - 2 * nu));
        K = lam + (2.0 / 3.0) * G;
    } else if (def(E) && def(nu)) {
        G = E / (2 * (1 + nu));
        lam = (E * nu) / ((1 + nu) * (1 - 2 * nu));
        K = E / (3 * (1 - 2 * nu));
    } else if (def(lam) && def(G)) {
        K = lam + (2.0 / 3.0) * G;
        nu = lam / (2 * (lam + G));
        E = 2 * G * (1 + nu);
    } else if (def(lam) && def(nu)) {
        E = (lam * (1 + nu) * (1 - 2 * nu)) / nu;
        G = E / (2 * (1 + nu));
        K = lam + (2.0 / 3.0) * G;
    } else if (def(G) && def(nu)) {
        E = 2 * G * (1 + nu);
        lam = (2 * G * nu) / (1 - 2 * nu);
        K = (2 * G * (1 + nu)) / (3 * (1 - 2 * nu));
    } else {
        return fail("Unsupported property pair combination");
    }
    if (nu < -1.0 || nu >= 0.5) return fail("Poisson's ratio violation: must be in [-1, 0.5)");
    if (E <= 0.0) return fail("Young's modulus must be positive");
    if (G <= 0.0) return fail("Shear modulus must be positive");
    if (K <= 0.0) return fail("Bulk modulus must be positive");
    if (lam <= -(2.0 / 3.0) * G) return fail("Lame's parameter violation: lambda must be > -2G/3");
    return 0;
}

void ob_stress(int material, double lambda, double mu, int64_t n, const double* H, double* P) {
    for (int64_t k = 0; k < n; ++k) stress(material, lambda, mu, H + 9 * k, P + 9 * k);
}

// The two-pass functions applied to a nodal field x (N x 3) at the P points
// (FunctionEvaluationProcessor::ComputeValues, include/FunctionEvaluationProcessor.h:86-121):
// a row without neighbours copies its coefficient, others sum psi * coefficient over the
// neighbours in reverse order. With more points than nodes (two-pass nodal cells) a point
// without neighbours past the nodes has no coefficient to copy: it stays at zero.
static void rk_apply_rows(const ob_problem* p, const double* x, double* out) {
    const int64_t N = p->num_nodes, P = p->rk_rows > 0 ? p->rk_rows : N;
    for (int64_t i = 0; i < P; ++i) {
        const int64_t b = p->rk_ptr[i], e = p->rk_ptr[i + 1];
        for (int c = 0; c < 3; ++c) {
            if (b == e) {
                out[i * 3 + c] = i < N ? x[i * 3 + c] : 0.0;
                continue;
            }
            double s = 0.0;
            for (int64_t k = e; k-- > b;) s += x[p->rk_nbr[k] * 3 + c] * p->rk_values[k];
            out[i * 3 + c] = s;
        }
    }
}

// Point values scattered to the coefficients (ScatterValues, :130-174): psi_j(x_i) v_i added
// to node j of f; a row without neighbours passes its value through (a point past the nodes
// drops it). The reference adds with atomics in no fixed order; here the sum for each node
// runs over i ascending.
static void rk_scatter(const ob_problem* p, const double* v, double* f) {
    const int64_t N = p->num_nodes, P = p->rk_rows > 0 ? p->rk_rows : N;
    for (int64_t i = 0; i < P; ++i) {
        const int64_t b = p->rk_ptr[i], e = p->rk_ptr[i + 1];
        if (b == e) {
            if (i < N)
                for (int c = 0; c < 3; ++c) f[i * 3 + c] += v[i * 3 + c];
            continue;
        }
        for (int64_t k = b; k < e; ++k)
            for (int c = 0; c < 3; ++c) f[p->rk_nbr[k] * 3 + c] += p->rk_values[k] * v[i * 3 + c];
    }
}

// Internal force over all parts, overwriting f (the solver zeroes the force field
// before the contributions accumulate, src/Solvers/Explicit.cpp:157-163).
void ob_internal_force(const ob_problem* p, const double* u, double* f) {
    const int64_t N = p->num_nodes;
    std::fill(f, f + N * 3, 0.0);
    if (!p->rk_ptr) {
        for (int k = 0; k < p->num_blocks; ++k) add_block_forces(p, p->blocks[k], u, f);
        return;
    }
    // Two-pass method (ExplicitSolver::ComputeForce, src/Solvers/Explicit.cpp:146-186): the
    // blocks on the physical displacement at the points, their forces scattered back.
    const int64_t P = p->rk_rows > 0 ? p->rk_rows : N;
    std::vector<double> up(P * 3), fl(P * 3, 0.0);
    rk_apply_rows(p, u, up.data());
    for (int k = 0; k < p->num_blocks; ++k) add_block_forces(p, p->blocks[k], up.data(), fl.data());
    rk_scatter(p, fl.data(), f);
}

// ComputeElementVolumeFunctor.h:20-79: V_e = sum_gp w_gp.
void ob_element_volumes(const ob_problem* p, int32_t block, double* vol) {
    const ob_block& b = p->blocks[block];
    if (b.kind == OB_CELLS) {
        for (int64_t c = 0; c < b.num_elems; ++c) vol[c] = b.cell_volumes[c];
        return;
    }
    const int nn = nodes_per_elem(b.kind);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < b.num_elems; ++e) {
        double X[24];
        for (int a = 0; a < nn; ++a)
            for (int i = 0; i < 3; ++i) X[a * 3 + i] = p->coords[b.conn[e * nn + a] * 3 + i];
        double V = 0.0, B[24];
        if (b.kind == OB_HEX8_GAUSS) {
            for (int gp = 0; gp < 8; ++gp) {
                double xi[3], dN[24];
                hex8_gauss_point(gp, xi);
                hex8_dN(xi, dN);
                V += gauss_bw<8>(X, dN, 1.0, B);
            }
        } else {
            V = gauss_bw<4>(X, kTet4dN, 1.0 / 6.0, B);
        }
        vol[e] = V;
    }
}

// src/MassUtils.cpp:17-46: m_a += rho V_e / n_en over the Gauss blocks, in element order.
void ob_lumped_mass(const ob_problem* p, double* m) {
    std::fill(m, m + p->num_nodes, 0.0);
    for (int k = 0; k < p->num_blocks; ++k) {
        const ob_block& b = p->blocks[k];
        if (b.kind == OB_CELLS) continue;
        const int nn = nodes_per_elem(b.kind);
        std::vector<double> vol(b.num_elems);
        ob_element_volumes(p, k, vol.data());
        for (int64_t e = 0; e < b.num_elems; ++e) {
            const double me = vol[e] * b.density / nn;
            for (int a = 0; a < nn; ++a) m[b.conn[e * nn + a]] += me;
        }
    }
}

// DirectTimeStepper (include/TimeStepper.h:97-128) driven by ExplicitSolver::Solve's
// `while (!AtEnd(time))` loop with `time += time_increment`.
int64_t ob_direct_time_schedule(double dt, double t_end, int64_t max_steps, double* dts) {
    double time = 0.0;
    int64_t n = 0;
    while (!(time >= t_end) && n < max_steps) {
        double d;
        if (time + dt <= t_end)
            d = dt;
        else if (time > t_end)
            d = 0.0;
        else
            d = t_end - time;
        if (dts) dts[n] = d;
        time += d;
        ++n;
    }
    return n;
}

int ob_init_acceleration(const ob_problem* p, const double* u, double* a) {
    std::vector<double> m = mass_of(p);
    std::vector<double> f(static_cast<size_t>(p->num_nodes) * 3);
    compute_acceleration(p, m.data(), u, f.data(), a);
    return 0;
}

int ob_explicit_steps(const ob_problem* p, int64_t nsteps, const double* dts, double t0, double* u, double* v, double* a) {
    std::vector<double> m = mass_of(p);
    std::vector<double> f(static_cast<size_t>(p->num_nodes) * 3);
    double time = t0;
    for (int64_t n = 0; n < nsteps; ++n) {
        cd_step(p, m.data(), dts[n], time, u, v, a, f.data());
        time += dts[n];
    }
    return 0;
}

int ob_lagrangian_force(const ob_problem* p, ob_lagrangian* s, double* f) {
    const int64_t N = p->num_nodes;
    std::fill(f, f + N * 3, 0.0);
    int64_t base = 0;
    for (int k = 0; k < p->num_blocks; ++k) {
        const ob_block& b = p->blocks[k];
        if (b.kind == OB_CELLS) return -1;
        const int nn = nodes_per_elem(b.kind);
        std::vector<double> slots(static_cast<size_t>(b.num_elems) * nn * 3);
        const double* href = s->formulation == OB_SEMI ? s->Href : s->H;
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < b.num_elems; ++e) {
            double hr[9];
            std::copy(href + 9 * (base + e), href + 9 * (base + e) + 9, hr);
            gauss_element_force_lagr(b, e, s->x, s->inc, hr, s->H + 9 * (base + e), slots.data() + e * nn * 3);
        }
        for (int64_t e = 0; e < b.num_elems; ++e)
            for (int a = 0; a < nn; ++a) {
                const int32_t n = b.conn[e * nn + a];
                for (int i = 0; i < 3; ++i) f[n * 3 + i] += slots[(e * nn + a) * 3 + i];
            }
        base += b.num_elems;
    }
    return 0;
}

namespace {
void lagr_acceleration(const ob_problem* p, ob_lagrangian* s, const double* m, double* f, double* a) {
    const int64_t N = p->num_nodes;
    ob_lagrangian_force(p, s, f);
    const double* g = p->body_accel;
    if (g[0] != 0.0 || g[1] != 0.0 || g[2] != 0.0)
        for (int64_t n = 0; n < N; ++n)
            for (int i = 0; i < 3; ++i) f[n * 3 + i] += g[i] * m[n];
    for (int64_t n = 0; n < N; ++n)
        for (int i = 0; i < 3; ++i) a[n * 3 + i] = f[n * 3 + i] / m[n];
}
}  // namespace

int ob_lagrangian_init(const ob_problem* p, ob_lagrangian* s, double* a) {
    if (s->formulation != OB_UPDATED && s->formulation != OB_SEMI) return -1;
    std::vector<double> m = mass_of(p);
    std::vector<double> f(static_cast<size_t>(p->num_nodes) * 3);
    lagr_acceleration(p, s, m.data(), f.data(), a);
    return 0;
}

// One step of ExplicitSolver::Solve (src/Solvers/Explicit.cpp:383-483) with the updated or
// semi displacement update (UpdateDisplacementsUpdatedFunctor, ExplicitTimeIntegrator.h:
// 141-244) and the reference-configuration update at the end of the step (UpdateShapeFunctions
// :195-214; ExplicitTimeIntegratorSemi::UpdateReferenceConfiguration :511-541; the updated
// formulation's current coordinates advance every step, :470-478).
int ob_lagrangian_steps(const ob_problem* p, ob_lagrangian* s, int64_t nsteps, const double* dts, double t0, double* u,
                        double* v, double* a) {
    if (s->formulation != OB_UPDATED && s->formulation != OB_SEMI) return -1;
    if (s->formulation == OB_SEMI && s->update_interval < 1) return -1;
    const int64_t N = p->num_nodes;
    std::vector<double> m = mass_of(p);
    std::vector<double> f(static_cast<size_t>(N) * 3);
    int64_t E = 0;
    for (int k = 0; k < p->num_blocks; ++k) E += p->blocks[k].num_elems;
    double time = t0;
    for (int64_t k = 0; k < nsteps; ++k) {
        const double dtn = dts[k], half = 0.5 * dtn;
        for (int64_t q = 0; q < N * 3; ++q) v[q] = v[q] + half * a[q];
        apply_bcs(p, 0, time + 0.5 * dtn, v);
        for (int64_t q = 0; q < N * 3; ++q) {
            const double d = dtn * v[q];
            u[q] = u[q] + d;
            if (s->formulation == OB_SEMI)
                s->inc[q] += d;
            else
                s->inc[q] = d;
        }
        lagr_acceleration(p, s, m.data(), f.data(), a);
        apply_bcs(p, 1, time + dtn, a);
        for (int64_t q = 0; q < N * 3; ++q) v[q] += half * a[q];
        time += dtn;
        s->n += 1;
        if (s->formulation == OB_UPDATED) {
            for (int64_t q = 0; q < N * 3; ++q) s->x[q] = s->x[q] + s->inc[q];
        } else if (s->n % s->update_interval == 0) {
            for (int64_t q = 0; q < N * 3; ++q) {
                s->x[q] = s->x[q] + s->inc[q];
                s->inc[q] = 0.0;
            }
            std::copy(s->H, s->H + 9 * E, s->Href);
        }
    }
    return 0;
}

// ExplicitSolver::Solve (src/Solvers/Explicit.cpp:308-498): initial force and
// acceleration at t=0 (no BC on a^0), then the central-difference loop.
int ob_explicit_solve(const ob_problem* p, double dt, double t_end, int64_t max_steps, double* u, double* v, double* a,
                      int64_t* steps_done) {
    std::vector<double> m = mass_of(p);
    std::vector<double> f(static_cast<size_t>(p->num_nodes) * 3);
    compute_acceleration(p, m.data(), u, f.data(), a);
    const int64_t n = ob_direct_time_schedule(dt, t_end, max_steps, nullptr);
    std::vector<double> dts(n);
    ob_direct_time_schedule(dt, t_end, max_steps, dts.data());
    double time = 0.0;
    for (int64_t k = 0; k < n; ++k) {
        cd_step(p, m.data(), dts[k], time, u, v, a, f.data());
        time += dts[k];
    }
    if (steps_done) *steps_done = n;
    return 0;
}

// With the two-pass coupling the force is f = Psi^T F(Psi u): its VJP with cotangent lam is
// Psi^T VJP_F(Psi u, Psi lam), and the modulus gradients are F's at (Psi u, Psi lam).
void ob_vjp_force(const ob_problem* p, const double* u, const double* lam, double* gu, double* gmu, double* gkappa) {
    std::fill(gu, gu + p->num_nodes * 3, 0.0);
    const double* uu = u;
    const double* ll = lam;
    double* g = gu;
    std::vector<double> up, lp, gl;
    if (p->rk_ptr) {
        const int64_t P = p->rk_rows > 0 ? p->rk_rows : p->num_nodes;
        up.resize(P * 3);
        lp.resize(P * 3);
        gl.assign(P * 3, 0.0);
        rk_apply_rows(p, u, up.data());
        rk_apply_rows(p, lam, lp.data());
        uu = up.data();
        ll = lp.data();
        g = gl.data();
    }
    int64_t off = 0;
    for (int k = 0; k < p->num_blocks; ++k) {
        add_block_vjp(p, p->blocks[k], uu, ll, g, gmu ? gmu + off : nullptr, gkappa ? gkappa + off : nullptr);
        off += p->blocks[k].num_elems;
    }
    if (p->rk_ptr) rk_scatter(p, gl.data(), gu);
}

// Discrete adjoint of the central-difference trajectory (new capability): the
// forward pass stores every displacement; the reverse pass transposes each
// operation of cd_step in reverse order. L = sum_s |u_s^K|^2.
int ob_adjoint(const ob_problem* p, int64_t nsteps, double dt, const double* u0, const double* v0, int32_t num_sensors,
               const int32_t* sensors, double* loss, double* gmu, double* gkappa) {
    const int64_t N = p->num_nodes;
    const size_t N3 = static_cast<size_t>(N) * 3;
    std::vector<double> m = mass_of(p);
    std::vector<double> u(u0, u0 + N3), v(v0, v0 + N3), a(N3), f(N3);
    std::vector<std::vector<double>> us;
    us.reserve(nsteps + 1);
    us.push_back(u);
    compute_acceleration(p, m.data(), u.data(), f.data(), a.data());
    double time = 0.0;
    std::vector<double> times(nsteps);
    for (int64_t n = 0; n < nsteps; ++n) {
        times[n] = time;
        cd_step(p, m.data(), dt, time, u.data(), v.data(), a.data(), f.data());
        time += dt;
        us.push_back(u);
    }
    double L = 0.0;
    std::vector<double> ub(N3, 0.0), vb(N3, 0.0), ab(N3, 0.0), fb(N3), gu(N3), mk;
    for (int32_t s = 0; s < num_sensors; ++s)
        for (int i = 0; i < 3; ++i) {
            const double x = u[sensors[s] * 3 + i];
            L += x * x;
            ub[sensors[s] * 3 + i] += 2.0 * x;
        }
    int64_t ne = 0;
    for (int k = 0; k < p->num_blocks; ++k) ne += p->blocks[k].num_elems;
    std::vector<double> gm(ne, 0.0), gk(ne, 0.0), tm(ne), tk(ne);
    const double h = 0.5 * dt;
    for (int64_t n = nsteps - 1; n >= 0; --n) {
        const double t_mid = times[n] + 0.5 * dt, t_next = times[n] + dt;
        std::vector<double> vhb = vb;
        free_mask(p, t_next, mk);
        for (size_t k = 0; k < N3; ++k) fb[k] = mk[k] * (ab[k] + h * vb[k]) / m[k / 3];
        ob_vjp_force(p, us[n + 1].data(), fb.data(), gu.data(), tm.data(), tk.data());
        for (int64_t e = 0; e < ne; ++e) {
            gm[e] += tm[e];
            gk[e] += tk[e];
        }
        free_mask(p, t_mid, mk);
        for (size_t k = 0; k < N3; ++k) {
            ub[k] += gu[k];
            vhb[k] += dt * ub[k];
            const double wb = mk[k] * vhb[k];
            vb[k] = wb;
            ab[k] = h * wb;
        }
    }
    for (size_t k = 0; k < N3; ++k) fb[k] = ab[k] / m[k / 3];
    ob_vjp_force(p, us[0].data(), fb.data(), gu.data(), tm.data(), tk.data());
    for (int64_t e = 0; e < ne; ++e) {
        gm[e] += tm[e];
        gk[e] += tk[e];
    }
    if (loss) *loss = L;
    if (gmu) std::copy(gm.begin(), gm.end(), gmu);
    if (gkappa) std::copy(gk.begin(), gk.end(), gkappa);
    return 0;
}

// MathUtils.h:321-330 ComputeKernel: cubic B-spline of r/R.
double ob_rk_kernel(const double d[3], double R) {
    const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / R;
    if (r < 0.5) return 1.0 + 6.0 * r * r * (-1.0 + r);
    if (r < 1.0) return 2.0 * (1.0 + r * (-3.0 + 3.0 * r - 1.0 * r * r));
    return 0.0;
}

// FunctionCreationProcessor.h:85-130 + ShapeFunctionsFunctorReproducingKernel.h:189-257
// (linear basis, BasesLinear :54-63): kernel with the neighbour's radius, moment
// matrix M = sum phi H H^T, psi_i = (M^-1 row 0) H_i phi_i; Shepard fallback.
int ob_rk_function_values(int64_t num_points, const double* points, const double* coords, const double* kernel_radius,
                          const int64_t* nbr_ptr, const int32_t* nbr, double* values) {
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : bad)
    for (int64_t i = 0; i < num_points; ++i) {
        const int64_t s0 = nbr_ptr[i], s1 = nbr_ptr[i + 1];
        const int64_t nn = s1 - s0;
        if (nn == 0) continue;
        if (nn == 1) {
            values[s0] = 1.0;
            continue;
        }
        std::vector<double> sh(nn * 3), phi(nn);
        double M[16] = {0};
        double ksum = 0.0;
        for (int64_t k = 0; k < nn; ++k) {
            const int32_t j = nbr[s0 + k];
            for (int c = 0; c < 3; ++c) sh[k * 3 + c] = points[i * 3 + c] - coords[j * 3 + c];
            phi[k] = ob_rk_kernel(&sh[k * 3], kernel_radius[j]);
            if (phi[k] == 0.0) continue;
            const double Hv[4] = {1.0, sh[k * 3], sh[k * 3 + 1], sh[k * 3 + 2]};
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c) M[r * 4 + c] += phi[k] * Hv[r] * Hv[c];
            ksum += phi[k];
        }
        double Mi[16];
        const bool ok = inv4(M, Mi);
        double nrm = 0.0;
        for (int k = 0; k < 16; ++k) nrm += Mi[k] * Mi[k];
        if (!ok || std::sqrt(nrm) < 1e-15) {
            for (int64_t k = 0; k < nn; ++k) values[s0 + k] = phi[k] / ksum;
            ++bad;
            continue;
        }
        for (int64_t k = 0; k < nn; ++k) {
            if (phi[k] == 0.0) {
                values[s0 + k] = 0.0;
                continue;
            }
            const double Hv[4] = {1.0, sh[k * 3], sh[k * 3 + 1], sh[k * 3 + 2]};
            values[s0 + k] = (Mi[0] * Hv[0] + Mi[1] * Hv[1] + Mi[2] * Hv[2] + Mi[3] * Hv[3]) * phi[k];
        }
    }
    return bad;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// RKPM one-pass nodal smoothing cells on tet-corner hexes.
//   points: vertices, unique edge midpoints (sorted (a,b)), unique face centroids
//   (sorted (a,b,c)), tet centroids -- the thex refinement's nodes;
//   neighbours: ball search with the neighbour's kernel radius, sorted by the
//   tweaked squared distance then node index, truncated to max_neighbors
//   (NeighborSearchProcessor.h:224-263, src/NeighborSearchProcessor.cpp:186-245,
//   NeighborSelectorFunctor.h:60-101);
//   functions: FunctionCreationProcessor.h:85-130;
//   cell gradients: SmoothedCellDataProcessor.h:541-675 (one-pass), with the corner
//   hexes' smoothed quadrature (QuadratureSmoothed.h:97-142);
//   mass: src/MassUtils.cpp:17-46 on the hexes, then FunctionEvaluationProcessor::ScatterValues
//   (FunctionEvaluationProcessor.h:130-176).
// ---------------------------------------------------------------------------
namespace {

struct ThexPoints {
    std::vector<double> xyz;                        // P x 3
    std::vector<std::array<int32_t, 2>> edges;      // sorted
    std::vector<std::array<int32_t, 3>> faces;      // sorted
    int64_t n_vert = 0;
    int64_t edge_id(int32_t a, int32_t b) const {
        std::array<int32_t, 2> k = {std::min(a, b), std::max(a, b)};
        return n_vert + (std::lower_bound(edges.begin(), edges.end(), k) - edges.begin());
    }
    int64_t face_id(int32_t a, int32_t b, int32_t c) const {
        std::array<int32_t, 3> k = {a, b, c};
        std::sort(k.begin(), k.end());
        return n_vert + static_cast<int64_t>(edges.size()) + (std::lower_bound(faces.begin(), faces.end(), k) - faces.begin());
    }
};

ThexPoints thex_points(int64_t N, const double* X, int64_t T, const int32_t* tets) {
    ThexPoints tp;
    tp.n_vert = N;
    for (int64_t t = 0; t < T; ++t) {
        const int32_t* v = tets + 4 * t;
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j) tp.edges.push_back({std::min(v[i], v[j]), std::max(v[i], v[j])});
        for (int i = 0; i < 4; ++i) {
            std::array<int32_t, 3> f;
            int k = 0;
            for (int j = 0; j < 4; ++j)
                if (j != i) f[k++] = v[j];
            std::sort(f.begin(), f.end());
            tp.faces.push_back(f);
        }
    }
    std::sort(tp.edges.begin(), tp.edges.end());
    tp.edges.erase(std::unique(tp.edges.begin(), tp.edges.end()), tp.edges.end());
    std::sort(tp.faces.begin(), tp.faces.end());
    tp.faces.erase(std::unique(tp.faces.begin(), tp.faces.end()), tp.faces.end());
    const int64_t P = N + static_cast<int64_t>(tp.edges.size() + tp.faces.size()) + T;
    tp.xyz.resize(static_cast<size_t>(P) * 3);
    for (int64_t i = 0; i < N * 3; ++i) tp.xyz[i] = X[i];
    int64_t p = N;
    for (const auto& e : tp.edges) {
        for (int c = 0; c < 3; ++c) tp.xyz[p * 3 + c] = (X[e[0] * 3 + c] + X[e[1] * 3 + c]) * 0.5;
        ++p;
    }
    for (const auto& f : tp.faces) {
        for (int c = 0; c < 3; ++c) tp.xyz[p * 3 + c] = ((X[f[0] * 3 + c] + X[f[1] * 3 + c]) + X[f[2] * 3 + c]) / 3.0;
        ++p;
    }
    for (int64_t t = 0; t < T; ++t) {
        std::array<int32_t, 4> s = {tets[4 * t], tets[4 * t + 1], tets[4 * t + 2], tets[4 * t + 3]};
        std::sort(s.begin(), s.end());
        for (int c = 0; c < 3; ++c)
            tp.xyz[p * 3 + c] = (((X[s[0] * 3 + c] + X[s[1] * 3 + c]) + X[s[2] * 3 + c]) + X[s[3] * 3 + c]) * 0.25;
        ++p;
    }
    return tp;
}

// The 8 thex points of the hex at corner i of tet t, in Hex8 node order.
void corner_hex(const ThexPoints& tp, const double* X, const int32_t* v, int64_t t, int i, int64_t out[8]) {
    int32_t o[3];
    int k = 0;
    for (int j = 0; j < 4; ++j)
        if (j != i) o[k++] = v[j];
    const int32_t c0 = v[i];
    double d[3][3];
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) d[a][c] = X[o[a] * 3 + c] - X[c0 * 3 + c];
    const double det = d[0][0] * (d[1][1] * d[2][2] - d[1][2] * d[2][1]) - d[0][1] * (d[1][0] * d[2][2] - d[1][2] * d[2][0]) +
                       d[0][2] * (d[1][0] * d[2][1] - d[1][1] * d[2][0]);
    if (det < 0) std::swap(o[1], o[2]);
    const int32_t a = o[0], b = o[1], c = o[2];
    out[0] = c0;
    out[1] = tp.edge_id(c0, a);
    out[2] = tp.face_id(c0, a, b);
    out[3] = tp.edge_id(c0, b);
    out[4] = tp.edge_id(c0, c);
    out[5] = tp.face_id(c0, a, c);
    out[6] = tp.n_vert + static_cast<int64_t>(tp.edges.size() + tp.faces.size()) + t;
    out[7] = tp.face_id(c0, b, c);
}

}  // namespace

namespace {

// Neighbours of every thex point (brute force over the active nodes, sorted by the tweaked
// squared distance, truncated to max_neighbors) and the function values there.
void thex_functions(int64_t N, const double* X, const double* R, int32_t max_neighbors, const ThexPoints& tp,
                    std::vector<int64_t>& ptr, std::vector<int32_t>& flat, std::vector<double>& psi) {
    const int64_t P = static_cast<int64_t>(tp.xyz.size() / 3);
    // Neighbours (brute force over the active nodes).
    std::vector<std::vector<int32_t>> nb(P);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t p = 0; p < P; ++p) {
        std::vector<std::pair<double, int32_t>> cand;
        const double* x = &tp.xyz[p * 3];
        for (int32_t j = 0; j < N; ++j) {
            const double dx = x[0] - X[j * 3], dy = x[1] - X[j * 3 + 1], dz = x[2] - X[j * 3 + 2];
            if (dx * dx + dy * dy + dz * dz > R[j] * R[j]) continue;
            const double tx = X[j * 3] * (1 + 1.0e-6) - x[0], ty = X[j * 3 + 1] * (1 + 1.0e-7) - x[1],
                         tz = X[j * 3 + 2] * (1 + 1.0e-8) - x[2];
            cand.push_back({tx * tx + ty * ty + tz * tz, j});
        }
        std::sort(cand.begin(), cand.end());
        if (static_cast<int32_t>(cand.size()) > max_neighbors) cand.resize(max_neighbors);
        for (const auto& c : cand) nb[p].push_back(c.second);
    }
    ptr.assign(P + 1, 0);
    for (int64_t p = 0; p < P; ++p) ptr[p + 1] = ptr[p] + static_cast<int64_t>(nb[p].size());
    flat.resize(ptr[P]);
    for (int64_t p = 0; p < P; ++p) std::copy(nb[p].begin(), nb[p].end(), flat.begin() + ptr[p]);
    psi.resize(ptr[P]);
    ob_rk_function_values(P, tp.xyz.data(), X, R, ptr.data(), flat.data(), psi.data());
}

}  // namespace

namespace {

// Nodal cells of the thex refinement, one-pass or two-pass. One-pass: a vertex cell's
// entries are the union of its corner-hex points' neighbours, b_j = sum_hex sum_k B_hex,k
// V_hex psi_k(j) / V_cell. Two-pass (SmoothedCellDataProcessor.h:541-675 without the
// functions): the entries are the corner-hex points themselves, b_p = sum_hex B_hex,k(p)
// V_hex / V_cell, and the functions couple the points to the vertices at run time.
int nodal_cells(bool two_pass, int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                int32_t max_neighbors, double density, int64_t* num_points, int64_t* num_nbr_entries,
                int64_t* num_cell_entries, double* points, int64_t* nbr_ptr, int32_t* nbr, double* values,
                int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads, double* cell_volumes, double* mass) {
    const ThexPoints tp = thex_points(N, X, T, tets);
    const int64_t P = static_cast<int64_t>(tp.xyz.size() / 3);
    std::vector<int64_t> ptr;
    std::vector<int32_t> flat;
    std::vector<double> psi;
    thex_functions(N, X, R, max_neighbors, tp, ptr, flat, psi);
    // Corner hexes of each vertex, in tet order.
    std::vector<std::vector<std::pair<int64_t, int>>> corners(N);
    for (int64_t t = 0; t < T; ++t)
        for (int i = 0; i < 4; ++i) corners[tets[4 * t + i]].push_back({t, i});
    std::vector<std::vector<int32_t>> cn(N);
    std::vector<std::vector<double>> cg(N);
    std::vector<double> cv(N, 0.0), mfe(P, 0.0);
    for (int32_t v = 0; v < N; ++v) {
        std::vector<int32_t> where(two_pass ? P : N, -1);
        for (const auto& ti : corners[v]) {
            int64_t hp[8];
            corner_hex(tp, X, tets + 4 * ti.first, ti.first, ti.second, hp);
            double hx[24], B[24], V;
            for (int k = 0; k < 8; ++k)
                for (int c = 0; c < 3; ++c) hx[k * 3 + c] = tp.xyz[hp[k] * 3 + c];
            ob_hex8_smoothed_bw(hx, B, &V);
            cv[v] += V;
            for (int k = 0; k < 8; ++k) mfe[hp[k]] += V * density / 8;
            if (two_pass) {
                for (int k = 0; k < 8; ++k) {
                    const int32_t q = static_cast<int32_t>(hp[k]);
                    if (where[q] < 0) {
                        where[q] = static_cast<int32_t>(cn[v].size());
                        cn[v].push_back(q);
                        cg[v].insert(cg[v].end(), {0.0, 0.0, 0.0});
                    }
                    for (int c = 0; c < 3; ++c) cg[v][where[q] * 3 + c] += B[k * 3 + c] * V;
                }
                continue;
            }
            for (int k = 0; k < 8; ++k)
                for (int64_t s = ptr[hp[k]]; s < ptr[hp[k] + 1]; ++s) {
                    const int32_t j = flat[s];
                    if (where[j] < 0) {
                        where[j] = static_cast<int32_t>(cn[v].size());
                        cn[v].push_back(j);
                        cg[v].insert(cg[v].end(), {0.0, 0.0, 0.0});
                    }
                    for (int c = 0; c < 3; ++c) cg[v][where[j] * 3 + c] += B[k * 3 + c] * V * psi[s];
                }
        }
        for (double& g : cg[v]) g /= cv[v];
    }
    int64_t K = 0;
    for (int32_t v = 0; v < N; ++v) K += static_cast<int64_t>(cn[v].size());
    if (num_points) *num_points = P;
    if (num_nbr_entries) *num_nbr_entries = ptr[P];
    if (num_cell_entries) *num_cell_entries = K;
    if (points) std::copy(tp.xyz.begin(), tp.xyz.end(), points);
    if (nbr_ptr) std::copy(ptr.begin(), ptr.end(), nbr_ptr);
    if (nbr) std::copy(flat.begin(), flat.end(), nbr);
    if (values) std::copy(psi.begin(), psi.end(), values);
    if (cell_ptr) {
        cell_ptr[0] = 0;
        for (int32_t v = 0; v < N; ++v) cell_ptr[v + 1] = cell_ptr[v] + static_cast<int64_t>(cn[v].size());
    }
    int64_t off = 0;
    for (int32_t v = 0; v < N; ++v) {
        if (cell_nodes) std::copy(cn[v].begin(), cn[v].end(), cell_nodes + off);
        if (cell_grads) std::copy(cg[v].begin(), cg[v].end(), cell_grads + 3 * off);
        off += static_cast<int64_t>(cn[v].size());
    }
    if (cell_volumes) std::copy(cv.begin(), cv.end(), cell_volumes);
    if (mass) {
        std::fill(mass, mass + N, 0.0);
        for (int64_t p = 0; p < P; ++p)
            for (int64_t s = ptr[p]; s < ptr[p + 1]; ++s) mass[flat[s]] += mfe[p] * psi[s];
    }
    return 0;
}

}  // namespace

extern "C" int ob_rkpm_nodal_cells(int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                                   int32_t max_neighbors, double density, int64_t* num_points, int64_t* num_nbr_entries,
                                   int64_t* num_cell_entries, double* points, int64_t* nbr_ptr, int32_t* nbr,
                                   double* values, int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads,
                                   double* cell_volumes, double* mass) {
    return nodal_cells(false, N, X, T, tets, R, max_neighbors, density, num_points, num_nbr_entries, num_cell_entries,
                       points, nbr_ptr, nbr, values, cell_ptr, cell_nodes, cell_grads, cell_volumes, mass);
}

extern "C" int ob_rkpm_nodal_cells_two_pass(int64_t N, const double* X, int64_t T, const int32_t* tets,
                                            const double* R, int32_t max_neighbors, double density,
                                            int64_t* num_points, int64_t* num_nbr_entries, int64_t* num_cell_entries,
                                            double* points, int64_t* nbr_ptr, int32_t* nbr, double* values,
                                            int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads,
                                            double* cell_volumes, double* mass) {
    return nodal_cells(true, N, X, T, tets, R, max_neighbors, density, num_points, num_nbr_entries, num_cell_entries,
                       points, nbr_ptr, nbr, values, cell_ptr, cell_nodes, cell_grads, cell_volumes, mass);
}

// Nodal cells split into subcells (subdomains 0): each corner hex keeps its own entries
// (the union of its eight points' neighbours, first appearance order) and gradients
// b_j = sum_k B_hex,k psi_k(j) (SmoothedCellDataProcessor.h:541-675 one-pass, with the
// subcell volume equal to the hex volume); the hexes of a vertex, in tet order, form its
// cell.
extern "C" int ob_rkpm_nodal_subcells(int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                                      int32_t max_neighbors, double density, int64_t* num_cell_entries,
                                      int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads, double* cell_volumes,
                                      int64_t* group_ptr) {
    (void)density;
    const ThexPoints tp = thex_points(N, X, T, tets);
    std::vector<int64_t> ptr;
    std::vector<int32_t> flat;
    std::vector<double> psi;
    thex_functions(N, X, R, max_neighbors, tp, ptr, flat, psi);
    std::vector<std::vector<std::pair<int64_t, int>>> corners(N);
    for (int64_t t = 0; t < T; ++t)
        for (int i = 0; i < 4; ++i) corners[tets[4 * t + i]].push_back({t, i});
    std::vector<int32_t> where(N, -1);
    std::vector<int32_t> sn;
    std::vector<double> sg, sv;
    std::vector<int64_t> sptr(1, 0), gptr(1, 0);
    for (int32_t v = 0; v < N; ++v) {
        for (const auto& ti : corners[v]) {
            int64_t hp[8];
            corner_hex(tp, X, tets + 4 * ti.first, ti.first, ti.second, hp);
            double hx[24], B[24], V;
            for (int k = 0; k < 8; ++k)
                for (int c = 0; c < 3; ++c) hx[k * 3 + c] = tp.xyz[hp[k] * 3 + c];
            ob_hex8_smoothed_bw(hx, B, &V);
            const int64_t base = sptr.back();
            std::vector<int32_t> used;
            for (int k = 0; k < 8; ++k)
                for (int64_t s = ptr[hp[k]]; s < ptr[hp[k] + 1]; ++s) {
                    const int32_t j = flat[s];
                    if (where[j] < 0) {
                        where[j] = static_cast<int32_t>(sn.size() - base);
                        sn.push_back(j);
                        sg.insert(sg.end(), {0.0, 0.0, 0.0});
                        used.push_back(j);
                    }
                    for (int c = 0; c < 3; ++c) sg[(base + where[j]) * 3 + c] += B[k * 3 + c] * V * psi[s];
                }
            for (int64_t e = base; e < static_cast<int64_t>(sn.size()); ++e)
                for (int c = 0; c < 3; ++c) sg[e * 3 + c] /= V;
            for (int32_t j : used) where[j] = -1;
            sv.push_back(V);
            sptr.push_back(static_cast<int64_t>(sn.size()));
        }
        gptr.push_back(static_cast<int64_t>(sv.size()));
    }
    if (num_cell_entries) *num_cell_entries = static_cast<int64_t>(sn.size());
    if (cell_ptr) std::copy(sptr.begin(), sptr.end(), cell_ptr);
    if (cell_nodes) std::copy(sn.begin(), sn.end(), cell_nodes);
    if (cell_grads) std::copy(sg.begin(), sg.end(), cell_grads);
    if (cell_volumes) std::copy(sv.begin(), sv.end(), cell_volumes);
    if (group_ptr) std::copy(gptr.begin(), gptr.end(), group_ptr);
    return 0;
}

// ---------------------------------------------------------------------------
// RKPM one-pass element smoothing cells (element_smoothing_cell, subdomains 1, with
// approximation_space reproducing_kernel): every tet is a cell whose entries are the
// union of its four vertices' neighbours; b_{t,j} = sum_k B_{t,k} V_t psi_k(j) / V_t
// (SmoothedCellDataProcessor.h:541-675 one-pass, QuadratureSmoothed.h:32-63 for the tet's
// smoothed gradients); functions at the vertices only (FunctionCreationProcessor.h:85-130);
// mass rho V_t / 4 to the vertices, scattered through the functions
// (src/MassUtils.cpp:17-46, FunctionEvaluationProcessor.h:130-176).
// Two calls: sizes first (outputs NULL), then the arrays.
// ---------------------------------------------------------------------------
namespace {
int element_cells_impl(int nn, int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                       int32_t max_neighbors, double density, int64_t* num_nbr_entries, int64_t* num_cell_entries,
                       int64_t* nbr_ptr, int32_t* nbr, double* values, int64_t* cell_ptr, int32_t* cell_nodes,
                       double* cell_grads, double* cell_volumes, double* mass) {
    std::vector<std::vector<int32_t>> nb(N);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t p = 0; p < N; ++p) {
        std::vector<std::pair<double, int32_t>> cand;
        const double* x = &X[p * 3];
        for (int32_t j = 0; j < N; ++j) {
            const double dx = x[0] - X[j * 3], dy = x[1] - X[j * 3 + 1], dz = x[2] - X[j * 3 + 2];
            if (dx * dx + dy * dy + dz * dz > R[j] * R[j]) continue;
            const double tx = X[j * 3] * (1 + 1.0e-6) - x[0], ty = X[j * 3 + 1] * (1 + 1.0e-7) - x[1],
                         tz = X[j * 3 + 2] * (1 + 1.0e-8) - x[2];
            cand.push_back({tx * tx + ty * ty + tz * tz, j});
        }
        std::sort(cand.begin(), cand.end());
        if (static_cast<int32_t>(cand.size()) > max_neighbors) cand.resize(max_neighbors);
        for (const auto& c : cand) nb[p].push_back(c.second);
    }
    std::vector<int64_t> ptr(N + 1, 0);
    for (int64_t p = 0; p < N; ++p) ptr[p + 1] = ptr[p] + static_cast<int64_t>(nb[p].size());
    std::vector<int32_t> flat(ptr[N]);
    for (int64_t p = 0; p < N; ++p) std::copy(nb[p].begin(), nb[p].end(), flat.begin() + ptr[p]);
    std::vector<double> psi(ptr[N]);
    ob_rk_function_values(N, X, X, R, ptr.data(), flat.data(), psi.data());
    std::vector<std::vector<int32_t>> cn(T);
    std::vector<std::vector<double>> cg(T);
    std::vector<double> cv(T, 0.0), mfe(N, 0.0);
    for (int64_t t = 0; t < T; ++t) {
        const int32_t* v = tets + nn * t;
        double xt[24], B[24], V;
        for (int k = 0; k < nn; ++k)
            for (int c = 0; c < 3; ++c) xt[k * 3 + c] = X[v[k] * 3 + c];
        if (nn == 8)
            ob_hex8_smoothed_bw(xt, B, &V);
        else
            ob_tet4_smoothed_bw(xt, B, &V);
        cv[t] = V;
        for (int k = 0; k < nn; ++k) {
            mfe[v[k]] += density * V / nn;
            for (int64_t s = ptr[v[k]]; s < ptr[v[k] + 1]; ++s) {
                const int32_t j = flat[s];
                int64_t idx = std::find(cn[t].begin(), cn[t].end(), j) - cn[t].begin();
                if (idx == static_cast<int64_t>(cn[t].size())) {
                    cn[t].push_back(j);
                    cg[t].insert(cg[t].end(), {0.0, 0.0, 0.0});
                }
                for (int c = 0; c < 3; ++c) cg[t][idx * 3 + c] += B[k * 3 + c] * V * psi[s];
            }
        }
        for (double& g : cg[t]) g /= V;
    }
    int64_t K = 0;
    for (int64_t t = 0; t < T; ++t) K += static_cast<int64_t>(cn[t].size());
    if (num_nbr_entries) *num_nbr_entries = ptr[N];
    if (num_cell_entries) *num_cell_entries = K;
    if (nbr_ptr) std::copy(ptr.begin(), ptr.end(), nbr_ptr);
    if (nbr) std::copy(flat.begin(), flat.end(), nbr);
    if (values) std::copy(psi.begin(), psi.end(), values);
    if (cell_ptr) {
        cell_ptr[0] = 0;
        for (int64_t t = 0; t < T; ++t) cell_ptr[t + 1] = cell_ptr[t] + static_cast<int64_t>(cn[t].size());
    }
    int64_t off = 0;
    for (int64_t t = 0; t < T; ++t) {
        if (cell_nodes) std::copy(cn[t].begin(), cn[t].end(), cell_nodes + off);
        if (cell_grads) std::copy(cg[t].begin(), cg[t].end(), cell_grads + 3 * off);
        off += static_cast<int64_t>(cn[t].size());
    }
    if (cell_volumes) std::copy(cv.begin(), cv.end(), cell_volumes);
    if (mass) {
        std::fill(mass, mass + N, 0.0);
        for (int64_t p = 0; p < N; ++p)
            for (int64_t s = ptr[p]; s < ptr[p + 1]; ++s) mass[flat[s]] += mfe[p] * psi[s];
    }
    return 0;
}
}  // namespace

extern "C" int ob_rkpm_element_cells(int64_t N, const double* X, int64_t T, const int32_t* tets, const double* R,
                                     int32_t max_neighbors, double density, int64_t* num_nbr_entries,
                                     int64_t* num_cell_entries, int64_t* nbr_ptr, int32_t* nbr, double* values,
                                     int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads, double* cell_volumes,
                                     double* mass) {
    return element_cells_impl(4, N, X, T, tets, R, max_neighbors, density, num_nbr_entries, num_cell_entries, nbr_ptr,
                              nbr, values, cell_ptr, cell_nodes, cell_grads, cell_volumes, mass);
}

// The same for Hex8 elements (ElementReproducingKernelHex8 with element cells): the smoothed
// Hex8 gradients (QuadratureSmoothed.h:97-142), mass rho V / 8 to the vertices.
extern "C" int ob_rkpm_hex8_element_cells(int64_t N, const double* X, int64_t E, const int32_t* hexes, const double* R,
                                          int32_t max_neighbors, double density, int64_t* num_nbr_entries,
                                          int64_t* num_cell_entries, int64_t* nbr_ptr, int32_t* nbr, double* values,
                                          int64_t* cell_ptr, int32_t* cell_nodes, double* cell_grads,
                                          double* cell_volumes, double* mass) {
    return element_cells_impl(8, N, X, E, hexes, R, max_neighbors, density, num_nbr_entries, num_cell_entries, nbr_ptr,
                              nbr, values, cell_ptr, cell_nodes, cell_grads, cell_volumes, mass);
}

// ---------------------------------------------------------------------------
// Stable time increment by the power method: PowerMethodProcessor::ComputeStableTimeIncrement
// (include/PowerMethodProcessor.h:331-480) with PerturbDisplacementCoefficients (:222-270),
// ComputeNextEigenvector (:272-330) and NormalizeField (EntityProcessor.h:676-697).
// v is the current eigenvector estimate (already scaled by eps*l on the first call, as
// InitializeEigenvector :196-220 does) and is updated in place. A dof is prescribed when
// any boundary condition names its component (the essential_boundary field).
// ---------------------------------------------------------------------------
extern "C" double ob_stable_time_increment(const ob_problem* p, const double* u, double* v, const double* l,
                                           double previous, int32_t num_iterations, double eps, double tol,
                                           double vartol, int32_t* iterations, int32_t* converged_out) {
    const int64_t N = p->num_nodes;
    std::vector<char> fixed(3 * N, 0);
    for (int32_t b = 0; b < p->num_bcs; ++b)
        for (int64_t k = 0; k < p->bcs[b].num_nodes; ++k)
            for (int c = 0; c < 3; ++c)
                if (p->bcs[b].component_mask >> c & 1) fixed[3 * p->bcs[b].nodes[k] + c] = 1;
    const std::vector<double> m = mass_of(p);
    std::vector<double> fu(3 * N), fe(3 * N), ue(3 * N);
    ob_internal_force(p, u, fu.data());
    double stable_np1 = previous == 0.0 ? 1.0e-16 : previous;
    const int W = 5;
    double recent[5] = {0, 0, 0, 0, 0};
    bool converged = false, oscillating = false;
    int32_t used = num_iterations;
    for (int32_t k = 0; k < num_iterations; ++k) {
        const double stable_n = stable_np1;
        for (int64_t i = 0; i < 3 * N; ++i) ue[i] = fixed[i] ? u[i] : u[i] + v[i] * l[i / 3] * eps;
        ob_internal_force(p, ue.data(), fe.data());
        double sum = 0.0;
        for (int64_t i = 0; i < 3 * N; ++i) {
            v[i] = fixed[i] ? 0.0 : (fe[i] - fu[i]) / (l[i / 3] * eps * m[i / 3]);
            sum += v[i] * v[i];
        }
        const double lambda = std::sqrt(sum);
        for (int64_t i = 0; i < 3 * N; ++i) v[i] /= lambda;
        stable_np1 = 2.0 / std::sqrt(lambda);
        recent[k % W] = stable_np1;
        if (std::abs(stable_np1 - stable_n) < tol * stable_np1) {
            converged = true;
            used = k + 1;
            break;
        }
        if (k >= W) {
            double mean = 0.0, var = 0.0;
            for (double r : recent) mean += r;
            mean /= W;
            for (double r : recent) var += (r - mean) * (r - mean);
            var /= (W - 1);
            if (k > W + 1) {
                double alt = 0.0;
                for (int i = 0; i < W - 1; ++i) {
                    const double diff = recent[i + 1] - recent[i];
                    if (i > 0 && diff * alt < 0) {
                        oscillating = true;
                    } else {
                        oscillating = false;
                        break;
                    }
                    alt = diff;
                }
            }
            if (var < vartol * mean || (oscillating && var < vartol * mean * 2.0)) {
                converged = true;
                used = k + 1;
                break;
            }
        }
    }
    if (iterations) *iterations = used;
    if (converged_out) *converged_out = converged ? 1 : 0;
    if (!converged || oscillating) return *std::min_element(recent, recent + W);
    return stable_np1;
}
