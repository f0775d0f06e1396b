// Per-(vertex, element) energy terms of the FEM energies, in registers:
//   * Neo-Hookean tet: SkyePhyX src/physics/neohookeanfem.cpp:40-110 with
//     NeoHookeanMath (src/helpers/math.cpp:10-231);
//   * StVK triangle membrane: src/physics/stvkfem.cpp:38-86 with STVKMath
//     (src/helpers/math.cpp:234-357).
// The 3x3 SVD is one-sided (Hestenes) Jacobi and the symmetric eigenproblem
// cyclic Jacobi (Golub & Van Loan, "Matrix Computations", 8.4-8.6); both
// produce the decompositions the reference asks Eigen for (sorted singular
// values, rotation-signed U/V; ascending eigenvalues).  The projected Hessian
// is a spectral function, so it does not depend on the basis each solver picks.
#pragma once
#include "avbd_common.cuh"

namespace avbd {

AVBD_HD float det3(const M3& m) {
    // first-column cofactor expansion
    return m3(m, 0, 0) * (m3(m, 1, 1) * m3(m, 2, 2) - m3(m, 1, 2) * m3(m, 2, 1)) -
           m3(m, 1, 0) * (m3(m, 0, 1) * m3(m, 2, 2) - m3(m, 0, 2) * m3(m, 2, 1)) +
           m3(m, 2, 0) * (m3(m, 0, 1) * m3(m, 1, 2) - m3(m, 0, 2) * m3(m, 1, 1));
}

AVBD_HD void jacobi_cs(float app, float aqq, float apq, float& c, float& s) {
    const float tau = (aqq - app) * fast_rcp(2.f * apq);
    const float at = fabsf(tau);
    const float r = 1.f + tau * tau;
    const float root = r < 1e30f ? r * fast_rsqrt(r) : at;   // sqrt(1 + tau^2), no overflow
    const float t = (tau >= 0.f ? 1.f : -1.f) * fast_rcp(at + root);
    c = fast_rsqrt(1.f + t * t);
    s = t * c;
}

AVBD_HD void rot_cols(V3& a, V3& b, float c, float s) {
    V3 na = c * a - s * b;
    V3 nb = s * a + c * b;
    a = na;
    b = nb;
}

AVBD_HD void swap3(V3& a, V3& b) { V3 t = a; a = b; b = t; }
AVBD_HD void swapf(float& a, float& b) { float t = a; a = b; b = t; }

// F = U diag(S) V^T, S sorted decreasing, U and V rotations after the sign
// fix of NeoHookeanMath::svd (math.cpp:13-35).
AVBD_HD void svd3(const M3& F, M3& U, V3& S, M3& V) {
    V3 a0 = F.c[0], a1 = F.c[1], a2 = F.c[2];
    V3 v0 = v3(1, 0, 0), v1 = v3(0, 1, 0), v2 = v3(0, 0, 1);
    const float eps2 = 1.1920929e-07f * 1.1920929e-07f;   // |a_p . a_q| <= eps |a_p| |a_q|, squared
    for (int sweep = 0; sweep < 64; ++sweep) {
        bool rotated = false;
#define AVBD_SVD_PAIR(ap, aq, vp, vq)                                           \
        {                                                                       \
            float al = sqnorm(ap), be = sqnorm(aq), ga = dot(ap, aq);           \
            if (!(ga == 0.f || ga * ga <= eps2 * (al * be))) {                  \
                float c, s;                                                     \
                jacobi_cs(al, be, ga, c, s);                                    \
                rot_cols(ap, aq, c, s);                                         \
                rot_cols(vp, vq, c, s);                                         \
                rotated = true;                                                 \
            }                                                                   \
        }
        AVBD_SVD_PAIR(a0, a1, v0, v1)
        AVBD_SVD_PAIR(a0, a2, v0, v2)
        AVBD_SVD_PAIR(a1, a2, v1, v2)
#undef AVBD_SVD_PAIR
        if (!rotated) break;
    }
    float s0 = norm(a0), s1 = norm(a1), s2 = norm(a2);
    // stable sort by decreasing singular value (bubble network)
    if (s0 < s1) { swapf(s0, s1); swap3(a0, a1); swap3(v0, v1); }
    if (s1 < s2) { swapf(s1, s2); swap3(a1, a2); swap3(v1, v2); }
    if (s0 < s1) { swapf(s0, s1); swap3(a0, a1); swap3(v0, v1); }
    const float tiny = 1.17549435e-38f;
    V3 u0 = s0 > tiny ? a0 * fast_rcp(s0) : v3(1, 0, 0);
    V3 u1 = s1 > tiny ? a1 * fast_rcp(s1) : v3(0, 1, 0);
    V3 u2 = s2 > tiny ? a2 * fast_rcp(s2) : cross(u0, u1);
    U.c[0] = u0; U.c[1] = u1; U.c[2] = u2;
    V.c[0] = v0; V.c[1] = v1; V.c[2] = v2;
    S = v3(s0, s1, s2);
    if (det3(U) < 0.f) { U.c[2] = -U.c[2]; S.z = -S.z; }
    if (det3(V) < 0.f) { V.c[2] = -V.c[2]; S.z = -S.z; }
}

// Symmetric 3x3 eigen-decomposition, eigenvalues increasing (cyclic Jacobi).
// A given by its entries; eigenvectors returned as columns of Q.
AVBD_HD void eig3(float a00, float a11, float a22, float a01, float a02, float a12, V3& w, M3& Q) {
    float A[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};
    float Vm[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    const float eps = 1.1920929e-07f;
    for (int sweep = 0; sweep < 64; ++sweep) {
        bool rotated = false;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0;
            const int q = pq == 0 ? 1 : 2;
            float apq = A[p][q];
            if (apq == 0.f) continue;
            if (fabsf(apq) <= eps * 0.5f * sqrtf(fabsf(A[p][p] * A[q][q]))) {
                A[p][q] = A[q][p] = 0.f;
                continue;
            }
            float c, s;
            jacobi_cs(A[p][p], A[q][q], apq, c, s);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float akp = A[k][p], akq = A[k][q];
                A[k][p] = c * akp - s * akq;
                A[k][q] = s * akp + c * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float apk = A[p][k], aqk = A[q][k];
                A[p][k] = c * apk - s * aqk;
                A[q][k] = s * apk + c * aqk;
            }
            A[p][q] = A[q][p] = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float vkp = Vm[k][p], vkq = Vm[k][q];
                Vm[k][p] = c * vkp - s * vkq;
                Vm[k][q] = s * vkp + c * vkq;
            }
            rotated = true;
        }
        if (!rotated) break;
    }
    float e0 = A[0][0], e1 = A[1][1], e2 = A[2][2];
    V3 q0 = v3(Vm[0][0], Vm[1][0], Vm[2][0]);
    V3 q1 = v3(Vm[0][1], Vm[1][1], Vm[2][1]);
    V3 q2 = v3(Vm[0][2], Vm[1][2], Vm[2][2]);
    if (e1 < e0) { swapf(e0, e1); swap3(q0, q1); }
    if (e2 < e1) { swapf(e1, e2); swap3(q1, q2); }
    if (e1 < e0) { swapf(e0, e1); swap3(q0, q1); }
    w = v3(e0, e1, e2);
    Q.c[0] = q0; Q.c[1] = q1; Q.c[2] = q2;
}

// Symmetric 2x2 eigen-decomposition, eigenvalues increasing.
AVBD_HD void eig2(float a00, float a11, float a01, float& w0, float& w1, float& c00, float& c10, float& c01,
                  float& c11) {
    float p00 = a00, p11 = a11, p01 = a01;
    float x0 = 1.f, y0 = 0.f, x1 = 0.f, y1 = 1.f;   // columns (x0,y0), (x1,y1)
    const float eps = 1.1920929e-07f;
    if (p01 != 0.f && !(fabsf(p01) <= eps * 0.5f * sqrtf(fabsf(p00 * p11)))) {
        float c, s;
        jacobi_cs(p00, p11, p01, c, s);
        float n00 = c * (c * p00 - s * p01) - s * (c * p01 - s * p11);
        float n11 = s * (s * p00 + c * p01) + c * (s * p01 + c * p11);
        p00 = n00;
        p11 = n11;
        x0 = c; y0 = -s; x1 = s; y1 = c;
    }
    if (p11 < p00) {
        w0 = p11; w1 = p00;
        c00 = x1; c10 = y1; c01 = x0; c11 = y0;
    } else {
        w0 = p00; w1 = p11;
        c00 = x0; c10 = y0; c01 = x1; c11 = y1;
    }
}

// ProjectEigenvalues (math.cpp:137-171) of COUNT values; the count is a
// template argument so the loops unroll and ev stays in registers.
template <int COUNT>
AVBD_HD void project_eigenvalues(float* ev, int mode, float rho, float threshold = 0.01f, float epsilon = 1e-6f) {
    bool use_abs = false;
    if (mode == 0) {
        use_abs = false;
    } else if (mode == 1) {
        use_abs = true;
    } else {
        use_abs = fabsf(rho - 1.f) > threshold;
    }
    if (!use_abs) {
#pragma unroll
        for (int i = 0; i < COUNT; ++i) ev[i] = fmaxf(epsilon, ev[i]);
        return;
    }
#pragma unroll
    for (int i = 0; i < COUNT; ++i) {
        ev[i] = fabsf(ev[i]);
        if (ev[i] < epsilon) ev[i] = epsilon;
    }
}
// Symmetric 3x3 accumulator (upper part implied).
struct S3 { float xx, yy, zz, xy, xz, yz; };
AVBD_HD void s3_zero(S3& h) { h.xx = h.yy = h.zz = h.xy = h.xz = h.yz = 0.f; }
AVBD_HD void s3_add_outer(S3& h, float lam, V3 w) {
    h.xx += lam * (w.x * w.x); h.yy += lam * (w.y * w.y); h.zz += lam * (w.z * w.z);
    h.xy += lam * (w.y * w.x); h.xz += lam * (w.z * w.x); h.yz += lam * (w.z * w.y);
}

// Vertex block of the projected Hessian from a decomposition F = U S V^T
// (NeoHookeanMath::ReconstructVertexHessian, math.cpp:196-231): the scaling
// block a.. (3x3, symmetric) and the twist / flip eigenvalues ev[3..8]
// (ev[0..2] are filled here), each mode contracted with V^T gradN.
// Every mode vector lies in the span of U's columns, so the sum of the
// rank-one terms is assembled as a 3x3 K in U's basis and turned once into
// H = restVolume U K U^T (the same matrix, with a third of the multiplies of
// summing nine outer products in world coordinates).  With g = V^T gradN:
//   scaling modes: K = diag(g) proj(A) diag(g);
//   twist / flip (i, j), vectors (g_j e_i -+ g_i e_j) / sqrt 2:
//     K_ii += (l_t + l_f) g_j^2 / 2, K_jj += (l_t + l_f) g_i^2 / 2,
//     K_ij += (l_f - l_t) g_i g_j / 2.
AVBD_HD void vertex_hessian(const M3& U, const M3& V, V3 gradN, float a00, float a11, float a22, float a01, float a02,
                            float a12, float (&ev)[9], int mode, float rho, float restVolume, S3& H) {
    const float g0 = dot(V.c[0], gradN), g1 = dot(V.c[1], gradN), g2 = dot(V.c[2], gradN);
    float k00, k11, k22, k01, k02, k12;
    // Scaling modes: when A is positive definite (all Cholesky pivots > 0) both ABSOLUTE and CLAMP
    // projections leave it unchanged up to the 1e-6 floor, so proj(A) = A needs no eigensolve.
    // (reciprocal pivots: the test only chooses between two forms of the same matrix)
    const float piv0 = a00;
    const float r0 = fast_rcp(piv0);
    const float l10 = a01 * r0, l20 = a02 * r0;
    const float piv1 = a11 - l10 * a01;
    const float l21 = (a12 - l20 * a01) * fast_rcp(piv1);
    const float piv2 = a22 - l20 * a02 - l21 * l21 * piv1;
    if (piv0 > 0.f && piv1 > 0.f && piv2 > 0.f) {
        k00 = a00 * (g0 * g0); k11 = a11 * (g1 * g1); k22 = a22 * (g2 * g2);
        k01 = a01 * (g0 * g1); k02 = a02 * (g0 * g2); k12 = a12 * (g1 * g2);
        project_eigenvalues<6>(ev + 3, mode, rho);
    } else {
        V3 w;
        M3 Q;
        eig3(a00, a11, a22, a01, a02, a12, w, Q);
        ev[0] = w.x; ev[1] = w.y; ev[2] = w.z;
        project_eigenvalues<9>(ev, mode, rho);
        k00 = k11 = k22 = k01 = k02 = k12 = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float c0 = Q.c[k].x * g0, c1 = Q.c[k].y * g1, c2 = Q.c[k].z * g2;
            const float l = ev[k];
            k00 += l * (c0 * c0); k11 += l * (c1 * c1); k22 += l * (c2 * c2);
            k01 += l * (c0 * c1); k02 += l * (c0 * c2); k12 += l * (c1 * c2);
        }
    }
    // twist / flip pairs (0,1): ev[3], ev[6]; (0,2): ev[4], ev[7]; (1,2): ev[5], ev[8]
    {
        const float s01 = 0.5f * (ev[3] + ev[6]), d01 = 0.5f * (ev[6] - ev[3]);
        const float s02 = 0.5f * (ev[4] + ev[7]), d02 = 0.5f * (ev[7] - ev[4]);
        const float s12 = 0.5f * (ev[5] + ev[8]), d12 = 0.5f * (ev[8] - ev[5]);
        const float q0 = g0 * g0, q1 = g1 * g1, q2 = g2 * g2;
        k00 += s01 * q1 + s02 * q2;
        k11 += s01 * q0 + s12 * q2;
        k22 += s02 * q0 + s12 * q1;
        k01 += d01 * (g0 * g1);
        k02 += d02 * (g0 * g2);
        k12 += d12 * (g1 * g2);
    }
    // H = restVolume U K U^T; T = K U^T (row m of T = sum_n K_mn u_n)
    k00 *= restVolume; k11 *= restVolume; k22 *= restVolume;
    k01 *= restVolume; k02 *= restVolume; k12 *= restVolume;
    const V3 u0 = U.c[0], u1 = U.c[1], u2 = U.c[2];
    const V3 t0 = k00 * u0 + k01 * u1 + k02 * u2;
    const V3 t1 = k01 * u0 + k11 * u1 + k12 * u2;
    const V3 t2 = k02 * u0 + k12 * u1 + k22 * u2;
    // H_ab = sum_m u_m[a] t_m[b]
    H.xx = u0.x * t0.x + u1.x * t1.x + u2.x * t2.x;
    H.yy = u0.y * t0.y + u1.y * t1.y + u2.y * t2.y;
    H.zz = u0.z * t0.z + u1.z * t1.z + u2.z * t2.z;
    H.xy = u0.x * t0.y + u1.x * t1.y + u2.x * t2.y;
    H.xz = u0.x * t0.z + u1.x * t1.z + u2.x * t2.z;
    H.yz = u0.y * t0.z + u1.y * t1.z + u2.y * t2.z;
}

// NeoHookeanFEM::ComputeEnergyTerms for vertex `role` of the tet
// (neohookeanfem.cpp:40-83, HandleInvertedElement :86-110).
AVBD_HD void neohookean_terms(V3 p0, V3 p1, V3 p2, V3 p3, const float* DmInv, V3 gradN, float restVolume, float mu,
                              float lambda, int mode, float rho, V3& grad, S3& H) {
    M3 Ds;
    Ds.c[0] = p1 - p0; Ds.c[1] = p2 - p0; Ds.c[2] = p3 - p0;
    M3 F;
#pragma unroll
    for (int j = 0; j < 3; ++j)
        F.c[j] = Ds.c[0] * DmInv[3 * j + 0] + Ds.c[1] * DmInv[3 * j + 1] + Ds.c[2] * DmInv[3 * j + 2];
    const float J = det3(F);
    // cofactor matrix of F (math.cpp:67-78)
    const float f00 = m3(F, 0, 0), f01 = m3(F, 0, 1), f02 = m3(F, 0, 2);
    const float f10 = m3(F, 1, 0), f11 = m3(F, 1, 1), f12 = m3(F, 1, 2);
    const float f20 = m3(F, 2, 0), f21 = m3(F, 2, 1), f22 = m3(F, 2, 2);
    M3 cof;
    cof.c[0] = v3(f11 * f22 - f12 * f21, -(f01 * f22 - f02 * f21), f01 * f12 - f02 * f11);
    cof.c[1] = v3(-(f10 * f22 - f12 * f20), f00 * f22 - f02 * f20, -(f00 * f12 - f02 * f10));
    cof.c[2] = v3(f10 * f21 - f11 * f20, -(f00 * f21 - f01 * f20), f00 * f11 - f01 * f10);
    if (J <= 1e-6f) {
        const float stiff = mu + lambda;
        V3 dJ = matvec(cof, gradN);
        float pm = stiff * (1e-6f - J);
        grad = (-restVolume * pm) * dJ;
        float d = restVolume * stiff;
        H.xx = d; H.yy = d; H.zz = d; H.xy = 0.f; H.xz = 0.f; H.yz = 0.f;
        return;
    }
    const float logJ = logf(J);
    // one division by J; the other quotients multiply by its reciprocal
    const float invJ = 1.f / J;
    const float scalar = (lambda * logJ - mu) * invJ;
    M3 P;
#pragma unroll
    for (int j = 0; j < 3; ++j) P.c[j] = mu * F.c[j] + scalar * cof.c[j];
    grad = matvec(P, gradN) * restVolume;

    M3 U, V;
    V3 S;
    svd3(F, U, S, V);
    // ComputeEnergyHessian (math.cpp:86-134)
    const float s0 = S.x, s1 = S.y, s2 = S.z;
    float ev[9];
    ev[0] = ev[1] = ev[2] = 0.f;
    const float dPhi = scalar;
    ev[3] = mu + dPhi * s2; ev[4] = mu + dPhi * s1; ev[5] = mu + dPhi * s0;
    ev[6] = mu - dPhi * s2; ev[7] = mu - dPhi * s1; ev[8] = mu - dPhi * s0;
    const float diagExtra = mu + lambda * (1.0f - logJ);
    // scaling block A (math.cpp:112-119)
    const float a00 = mu + diagExtra * fast_rcp(s0 * s0), a11 = mu + diagExtra * fast_rcp(s1 * s1),
                a22 = mu + diagExtra * fast_rcp(s2 * s2);
    const float a01 = lambda * s2 * invJ, a02 = lambda * s1 * invJ, a12 = lambda * s0 * invJ;
    vertex_hessian(U, V, gradN, a00, a11, a22, a01, a02, a12, ev, mode, rho, restVolume, H);
}

// St. Venant-Kirchhoff tet, vertex `role` (no reference counterpart; restated
// from the StVK energy Psi = mu tr(E^2) + lambda/2 tr(E)^2, E = (F^T F - I)/2,
// in the style of NeoHookeanFEM / STVKFEM).  Principal-stretch form
// psi = mu/4 sum (s_i^2 - 1)^2 + lambda/8 (sum s_i^2 - 3)^2 gives the scaling
// block d2psi/ds_i ds_j and the twist / flip eigenvalues (psi_i +- psi_j) /
// (s_i +- s_j) in closed form; projection and reconstruction are the
// Neo-Hookean ones.  An element below 1% of its rest volume takes the
// isotropic penalty of STVKFEM::HandleInvertedElement (stvkfem.cpp:75-86).
AVBD_HD void stvk_tet_terms(V3 p0, V3 p1, V3 p2, V3 p3, const float* DmInv, V3 gradN, float restVolume, float mu,
                            float lambda, int mode, float rho, V3& grad, S3& H) {
    M3 Ds;
    Ds.c[0] = p1 - p0; Ds.c[1] = p2 - p0; Ds.c[2] = p3 - p0;
    M3 F;
#pragma unroll
    for (int j = 0; j < 3; ++j)
        F.c[j] = Ds.c[0] * DmInv[3 * j + 0] + Ds.c[1] * DmInv[3 * j + 1] + Ds.c[2] * DmInv[3 * j + 2];
    const float J = det3(F);
    if (J < 0.01f) {
        const float stiff = mu + lambda;
        grad = (restVolume * stiff) * matvec(F, gradN);
        const float d = restVolume * stiff;
        H.xx = d; H.yy = d; H.zz = d; H.xy = 0.f; H.xz = 0.f; H.yz = 0.f;
        return;
    }
    // E = (F^T F - I) / 2, P = F (2 mu E + lambda tr(E) I)
    float C[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[i][j] = dot(F.c[i], F.c[j]);
    const float trE = 0.5f * (C[0][0] + C[1][1] + C[2][2] - 3.f);
    M3 P;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        V3 col = v3(0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float Ekj = 0.5f * (C[k][j] - (k == j ? 1.f : 0.f));
            const float Skj = 2.f * mu * Ekj + (k == j ? lambda * trE : 0.f);
            col = col + F.c[k] * Skj;
        }
        P.c[j] = col;
    }
    grad = matvec(P, gradN) * restVolume;

    M3 U, V;
    V3 S;
    svd3(F, U, S, V);
    const float s0 = S.x, s1 = S.y, s2 = S.z;
    const float q0 = s0 * s0, q1 = s1 * s1, q2 = s2 * s2;
    const float c = 0.5f * lambda * (q0 + q1 + q2 - 3.f);
    float ev[9];
    ev[0] = ev[1] = ev[2] = 0.f;
    ev[3] = mu * (q0 - s0 * s1 + q1 - 1.f) + c;   // twist (0,1)
    ev[4] = mu * (q0 - s0 * s2 + q2 - 1.f) + c;   // twist (0,2)
    ev[5] = mu * (q1 - s1 * s2 + q2 - 1.f) + c;   // twist (1,2)
    ev[6] = mu * (q0 + s0 * s1 + q1 - 1.f) + c;   // flip (0,1)
    ev[7] = mu * (q0 + s0 * s2 + q2 - 1.f) + c;   // flip (0,2)
    ev[8] = mu * (q1 + s1 * s2 + q2 - 1.f) + c;   // flip (1,2)
    const float a00 = mu * (3.f * q0 - 1.f) + c + lambda * q0;
    const float a11 = mu * (3.f * q1 - 1.f) + c + lambda * q1;
    const float a22 = mu * (3.f * q2 - 1.f) + c + lambda * q2;
    const float a01 = lambda * s0 * s1, a02 = lambda * s0 * s2, a12 = lambda * s1 * s2;
    vertex_hessian(U, V, gradN, a00, a11, a22, a01, a02, a12, ev, mode, rho, restVolume, H);
}

// STVKFEM::ComputeEnergyTerms for vertex `role` of the triangle
// (stvkfem.cpp:38-86) with STVKMath (math.cpp:234-357).
// DmInv2D column-major (m00, m10, m01, m11); gradN is 2D.
AVBD_HD void stvk_terms(V3 p0, V3 p1, V3 p2, float4 DmInv, float gnx, float gny, float restArea, float mu,
                        float lambda, int mode, float rho, V3& grad, S3& H) {
    V3 e0 = p1 - p0, e1 = p2 - p0;
    // F (3x2) = Ds (3x2) * DmInv (2x2)
    V3 F0 = e0 * DmInv.x + e1 * DmInv.y;
    V3 F1 = e0 * DmInv.z + e1 * DmInv.w;
    const float stiff = mu + lambda;
    if (norm(cross(e0, e1)) < 2.f * restArea * 0.01f) {
        V3 P0 = stiff * F0, P1 = stiff * F1;
        grad = restArea * (P0 * gnx + P1 * gny);
        float d = restArea * stiff;
        H.xx = d; H.yy = d; H.zz = d; H.xy = 0.f; H.xz = 0.f; H.yz = 0.f;
        return;
    }
    // L = 0.5 (F^T F - I)
    const float c00 = dot(F0, F0), c01 = dot(F0, F1), c11 = dot(F1, F1);
    const float L00 = 0.5f * (c00 - 1.f), L01 = 0.5f * c01, L11 = 0.5f * (c11 - 1.f);
    const float trL = L00 + L11;
    // P = F (2 mu L + lambda trL I)
    const float S00 = 2.f * mu * L00 + lambda * trL, S01 = 2.f * mu * L01, S11 = 2.f * mu * L11 + lambda * trL;
    V3 P0 = F0 * S00 + F1 * S01;
    V3 P1 = F0 * S01 + F1 * S11;
    grad = restArea * (P0 * gnx + P1 * gny);

    // SVD of the 3x2 F: one Jacobi rotation on the two columns
    V3 a0 = F0, a1 = F1;
    float vx0 = 1.f, vy0 = 0.f, vx1 = 0.f, vy1 = 1.f;
    const float eps = 1.1920929e-07f;
    for (int sweep = 0; sweep < 64; ++sweep) {
        float al = sqnorm(a0), be = sqnorm(a1), ga = dot(a0, a1);
        if (ga == 0.f || fabsf(ga) <= eps * sqrtf(al * be)) break;
        float c, s;
        jacobi_cs(al, be, ga, c, s);
        rot_cols(a0, a1, c, s);
        float nx0 = c * vx0 - s * vx1, ny0 = c * vy0 - s * vy1;
        float nx1 = s * vx0 + c * vx1, ny1 = s * vy0 + c * vy1;
        vx0 = nx0; vy0 = ny0; vx1 = nx1; vy1 = ny1;
    }
    float s0 = norm(a0), s1 = norm(a1);
    if (s0 < s1) {
        swapf(s0, s1); swap3(a0, a1);
        swapf(vx0, vx1); swapf(vy0, vy1);
    }
    const float tiny = 1.17549435e-38f;
    V3 u0 = s0 > tiny ? a0 / s0 : v3(1, 0, 0);
    V3 u1 = s1 > tiny ? a1 / s1 : v3(0, 1, 0);
    if (vx0 * vy1 - vx1 * vy0 < 0.f) { vx1 = -vx1; vy1 = -vy1; s1 = -s1; }   // math.cpp:246-250

    // ComputeEnergyHessian (math.cpp:285-321)
    float ev[4];
    const float trS = s0 * s0 + s1 * s1;
    const float d0 = s0 * (mu * (s0 * s0 - 1.f) + 0.5f * lambda * (trS - 2.f));
    const float d1 = s1 * (mu * (s1 * s1 - 1.f) + 0.5f * lambda * (trS - 2.f));
    ev[2] = (s0 + s1 > 1e-8f) ? (d0 + d1) / (s0 + s1) : -(mu + lambda);
    ev[3] = (fabsf(s0 - s1) > 1e-8f) ? (d0 - d1) / (s0 - s1) : (3.f * mu + 2.f * lambda) * s0 * s0 - mu - lambda;
    const float A00 = 3.f * mu * s0 * s0 + 0.5f * lambda * (3.f * s0 * s0 + s1 * s1) - mu - lambda;
    const float A11 = 3.f * mu * s1 * s1 + 0.5f * lambda * (3.f * s1 * s1 + s0 * s0) - mu - lambda;
    const float A01 = lambda * s0 * s1;
    float q00, q10, q01, q11;
    eig2(A00, A11, A01, ev[0], ev[1], q00, q10, q01, q11);
    project_eigenvalues<4>(ev, mode, rho);
    // ReconstructVertexHessian (math.cpp:324-356)
    const float vg0 = vx0 * gnx + vy0 * gny;
    const float vg1 = vx1 * gnx + vy1 * gny;
    s3_zero(H);
    s3_add_outer(H, ev[0], (q00 * vg0) * u0 + (q10 * vg1) * u1);
    s3_add_outer(H, ev[1], (q01 * vg0) * u0 + (q11 * vg1) * u1);
    const float is2 = 0.70710678118f;
    s3_add_outer(H, ev[2], is2 * (vg1 * u0 - vg0 * u1));
    s3_add_outer(H, ev[3], is2 * (vg1 * u0 + vg0 * u1));
    H.xx *= restArea; H.yy *= restArea; H.zz *= restArea;
    H.xy *= restArea; H.xz *= restArea; H.yz *= restArea;
}

}  // namespace avbd
