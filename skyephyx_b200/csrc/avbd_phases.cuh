// Per-item phase functions of the AVBD step (SkyePhyX Solver::Step,
// src/physics/solver.cpp:199-627).  Each function processes ONE item (a body,
// a candidate pair, a force) and is called by both drivers: the grid-wide
// kernels of the single-scene path and the persistent per-scene kernel of the
// batched path.  A body is always processed by one thread in a fixed
// incidence order, so a scene's result does not depend on which driver, CTA
// or batch composition runs it.
#pragma once
#include "avbd_common.cuh"
#include "avbd_fem.cuh"
#include "avbd_narrow.cuh"

#if defined(__CUDA_ARCH__)
#define AVBD_ATOMIC_ADD(p, v) atomicAdd((p), (v))
#else
#define AVBD_ATOMIC_ADD(p, v) avbd_host_atomic_add((p), (v))
static inline int avbd_host_atomic_add(int* p, int v) { int o = *p; *p = o + v; return o; }
#endif

namespace avbd {

AVBD_HD bool is_inf(float x) { return isinf(x); }

// Transform::TransformPoint (geometry.hpp:70-73): R (S p) + x
AVBD_HD V3 transform_point(const World& W, int b, V3 p) {
    V3 s = v3(W.scale[b]);
    return qrotate(q4(W.rot[b]), v3(s.x * p.x, s.y * p.y, s.z * p.z)) + v3(W.pos[b]);
}

// ===========================================================================
// Phase 0 + 4: mass cache (solver.cpp:215-231) and prediction (:324-385)
// ===========================================================================
AVBD_HD void predict_body(const World& W, int b) {
    const int fl = W.flags[b];
    if (fl & kBodyRemoved) return;
    const float dt = W.P.dt;
    Q4 rot = q4(W.rot[b]);
    const bool is_static = (fl & kBodyStatic) != 0;
    const bool particle = (fl & kBodyParticle) != 0;
    if (!is_static) {
        float4 mI = W.massI[b];
        if (mI.x > 0.f) {
            M3 R = rotmat(rot);
            // (R I) R^T, lower triangle (i >= j)
            V3 RI0 = R.c[0] * mI.y, RI1 = R.c[1] * mI.z, RI2 = R.c[2] * mI.w;
            auto e = [&](int i, int j) {
                return comp(RI0, i) * m3(R, j, 0) + comp(RI1, i) * m3(R, j, 1) + comp(RI2, i) * m3(R, j, 2);
            };
            float4 a, c;
            a.x = mI.x; a.y = e(0, 0); a.z = e(1, 1); a.w = e(2, 2);
            c.x = e(1, 0); c.y = e(2, 0); c.z = e(2, 1); c.w = 0.f;
            W.Mw0[b] = a;
            W.Mw1[b] = c;
        }
    }
    // cwiseMin(+50).cwiseMax(-50): min first, then max
    const V3 omega = v3(fmaxf(fminf(W.omega[b].x, kMaxRotationVelocity), -kMaxRotationVelocity),
               fmaxf(fminf(W.omega[b].y, kMaxRotationVelocity), -kMaxRotationVelocity),
               fmaxf(fminf(W.omega[b].z, kMaxRotationVelocity), -kMaxRotationVelocity));
    W.omega[b] = f4(omega);
    const V3 pos = v3(W.pos[b]);
    const V3 vel = v3(W.vel[b]);
    const V3 g = v3(0.f, kGravityY, 0.f);
    V3 ipos = pos + vel * dt;
    if (!is_static) ipos = ipos + (g * dt) * dt;
    Q4 irot = rot;
    Q4 newrot = rot;
    if (!is_static && !particle) {
        // wq = w (x) q with w = (0, omega)
        Q4 q = rot;
        float wqw = -(omega.x * q.x + omega.y * q.y + omega.z * q.z);
        V3 wqv = q.w * omega + cross(omega, qvec(q));
        Q4 qi;
        qi.w = q.w + 0.5f * wqw * dt;
        qi.x = q.x + 0.5f * wqv.x * dt;
        qi.y = q.y + 0.5f * wqv.y * dt;
        qi.z = q.z + 0.5f * wqv.z * dt;
        irot = qnormalize(qi);
        newrot = irot;
    }
    // adaptive gravity warm start
    V3 acc = (vel - v3(W.pvel[b])) / dt;
    const float gmag = 9.81f;
    V3 gdir = g / gmag;
    float aw = dot(acc, gdir) / gmag;
    aw = clampf(aw, 0.f, 1.f);
    V3 npos = pos + vel * dt + ((g * dt) * dt) * aw;
    W.ipos[b] = f4(ipos);
    W.irot[b] = f4(irot);
    W.lpos[b] = f4(pos);
    W.lrot[b] = f4(rot);
    W.pos[b] = f4(npos);
    W.rot[b] = f4(newrot);
    W.dlin[b] = f4(npos - pos);
    W.dang[b] = f4(rotation_difference(newrot, rot));
}

// ===========================================================================
// Phase 1: broadphase (solver.cpp:233-256).  The owner of a pair is its lower
// body index i; it enumerates j > i of the same scene and keeps pairs whose
// circumscribed spheres overlap (exact predicate of the reference) and that
// no live joint/spring links (isConstrainedTo, force.hpp:81-89).
// ===========================================================================
// Static partner list of body i, (partner body, force) pairs; read once per
// broadphase row, so a body without joints or springs costs no lookup per pair.
struct Partners {
    int off, n;
};
AVBD_HD Partners partners_of(const World& W, int i) {
    Partners p;
    p.off = W.spartner_off[i];
    p.n = W.spartner_n[i];
    return p;
}

// isConstrainedTo: a live joint or spring of i (partners p) links it to j.
AVBD_HD bool pair_constrained(const World& W, Partners p, int j) {
    for (int k = p.off; k < p.off + p.n; ++k) {
        int2 pf = reinterpret_cast<const int2*>(W.spartner)[k];
        if (pf.x == j && !(W.ftype[pf.y] & kForceRemoved)) return true;
    }
    return false;
}

AVBD_HD bool sphere_overlap(float4 pi, float4 pj, float ri, float rj) {
    V3 d = xsub(v3(pi), v3(pj));
    float dist = xnorm(d);
    return dist < XADD(ri, rj);
}

// The same decision as sphere_overlap, settled by a squared-distance test
// wherever the two sides are further apart than any rounding of either form
// (relative band 1e-5, against errors of a few 1e-7); pairs inside the band
// take the exact test.
AVBD_HD bool sphere_overlap_fast(float4 pi, float4 pj, float ri, float rj) {
    const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const float d2 = dx * dx + dy * dy + dz * dz;
    const float r = ri + rj;
    if (!(r > 0.f)) return sphere_overlap(pi, pj, ri, rj);   // removed (-inf) or degenerate radii
    const float r2 = r * r;
    if (d2 > r2 * 1.00001f) return false;
    if (d2 < r2 * 0.99999f) return true;
    return sphere_overlap(pi, pj, ri, rj);
}

// Returns the number of candidates owned by body i; writes them when out != 0.
AVBD_HD int broadphase_body(const World& W, const SceneDesc& sc, int i, int2* out, int cap) {
    if (W.flags[i] & kBodyRemoved) return 0;
    const float4 pi = W.pos[i];
    const float ri = W.scale[i].w;
    const int end = sc.body0 + sc.nbody;
    const Partners pp = partners_of(W, i);
    int n = 0;
    for (int j = i + 1; j < end; ++j) {
        if (W.flags[j] & kBodyRemoved) continue;
        if (!sphere_overlap_fast(pi, W.pos[j], ri, W.scale[j].w)) continue;
        if (pair_constrained(W, pp, j)) continue;
        if (out && n < cap) out[n] = make_int2(i, j);
        ++n;
    }
    return n;
}

// Same as broadphase_body with the scene's (position, radius) staged in
// shared memory (radius = -inf marks a removed body).
AVBD_HD int broadphase_body_staged(const World& W, const SceneDesc& sc, int i, const float4* sp, int2* out, int cap) {
    const int li = i - sc.body0;
    const float4 pi = sp[li];
    if (isinf(pi.w)) return 0;
    const Partners pp = partners_of(W, i);
    int n = 0;
    for (int lj = li + 1; lj < sc.nbody; ++lj) {
        const float4 pj = sp[lj];
        if (!sphere_overlap_fast(pi, pj, pi.w, pj.w)) continue;
        const int j = sc.body0 + lj;
        if (pair_constrained(W, pp, j)) continue;
        if (out && n < cap) out[n] = make_int2(i, j);
        ++n;
    }
    return n;
}

// ===========================================================================
// Phase 2 (forces): Manifold::Initialize (manifold.cpp:32-194) on one
// candidate slot, followed by the warm-start penalty decay (solver.cpp:274-291).
// Old contacts come from the previous step's table (binary search by pair).
// ===========================================================================
AVBD_HD int find_old_slot(const int2* pairs, int lo, int hi, int a, int b) {
    // pairs[lo, hi) sorted by (x, y)
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        int2 p = pairs[mid];
        if (p.x < a || (p.x == a && p.y < b)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

AVBD_HD void narrowphase_slot(const World& W, const SceneDesc& sc, SceneState* st, int slot, int cur, int old_count) {
    const int prev = cur ^ 1;
    const int2 ab = W.cpair[cur][slot];
    const int A = ab.x, B = ab.y;
    Collision col;
    collide_box_box(v3(W.pos[A]), q4(W.rot[A]), v3(W.scale[A]), v3(W.pos[B]), q4(W.rot[B]), v3(W.scale[B]), col);
    if (col.n == 0) {
        W.cn[cur][slot] = 0;
        return;
    }
    // contact slots from the scene's pool (bump allocation; placement does not affect results)
    const int kofs = AVBD_ATOMIC_ADD(&st->kused[cur], col.n);
    if (kofs + col.n > sc.kcap) {
        W.cn[cur][slot] = 0;
        st->need_k = 1;
        return;
    }
    const int base = sc.k0 + kofs;
#ifdef __CUDA_ARCH__
    if (!AVBD_CHECK(W, kofs >= 0 && kofs + col.n <= sc.kcap, 6, kofs + col.n, sc.kcap)) {
        W.cn[cur][slot] = 0;
        return;
    }
#endif
    W.kbase[cur][slot] = base;
    W.cn[cur][slot] = col.n;
    const int li = AVBD_ATOMIC_ADD(&st->nlive[cur], 1);
    if (li < sc.candcap) W.live[cur][sc.cand0 + li] = slot;
    const float fr = XSQRT(XMUL(W.friction[A], W.friction[B]));
    W.cfric[cur][slot] = fr;
    // previous contacts of the same pair
    int os = -1, on = 0;
    int birth = st->step;   // a manifold that had contacts last step persists (keeps its place in Mesh::forces)
    if (old_count > 0) {
        int k = find_old_slot(W.cpair[prev], sc.cand0, sc.cand0 + old_count, A, B);
        if (k < sc.cand0 + old_count) {
            int2 p = W.cpair[prev][k];
            if (p.x == A && p.y == B) {
                on = W.cn[prev][k];
                if (on > 0) { os = W.kbase[prev][k]; birth = W.cbirth[prev][k]; }
            }
        }
    }
    W.cbirth[cur][slot] = birth;
    if (on > 0) AVBD_ATOMIC_ADD(&st->nmatched, 1);
    const Params& P = W.P;
    const Q4 qA = q4(W.rot[A]), qB = q4(W.rot[B]);
    const M3 RA = xrotmat(qA), RB = xrotmat(qB);
    const V3 posA = v3(W.pos[A]), posB = v3(W.pos[B]);
    for (int i = 0; i < col.n; ++i) {
        Contact c = col.c[i];
        float pen[3] = {0.f, 0.f, 0.f}, lam[3] = {0.f, 0.f, 0.f};
        float stick = 0.f;
        bool is_new = true;
        for (int j = 0; j < on; ++j) {
            const int oj = os + j;
            if (W.kid[prev][oj] == c.id) {
                float4 op = W.kpen[prev][oj], ol = W.klam[prev][oj];
                pen[0] = op.x; pen[1] = op.y; pen[2] = op.z;
                lam[0] = ol.x; lam[1] = ol.y; lam[2] = ol.z;
                stick = W.krAw[prev][oj].w;
                if (stick != 0.f) {
                    c.rA = v3(W.krA[prev][oj]);
                    c.rB = v3(W.krB[prev][oj]);
                }
                is_new = false;
                break;
            }
        }
        // Jacobian directions (manifold.cpp:111-157)
        V3 n = v3(-c.normal.x, -c.normal.y, -c.normal.z);
        V3 t1 = fabsf(n.x) > 0.9f ? xcross(n, v3(0.f, 1.f, 0.f)) : xcross(n, v3(1.f, 0.f, 0.f));
        {
            float n2 = xdot(t1, t1);
            if (n2 > 0.f) t1 = xdiv(t1, XSQRT(n2));
        }
        V3 t2 = xcross(n, t1);
        V3 rAw = xmatvec(RA, c.rA);
        V3 rBw = xmatvec(RB, c.rB);
        V3 rd = xsub(xadd(posA, rAw), xadd(posB, rBw));
        float C0x = XADD(xdot(n, rd), kCollisionMargin);
        float C0y = xdot(t1, rd);
        float C0z = xdot(t2, rd);
        if (is_new) {
            pen[0] = clampf(c.penetration * P.on_penetration_penalty, kPenaltyMin, kNewContactPenaltyMax);
            pen[1] = kPenaltyMin;
            pen[2] = kPenaltyMin;
        }
        // warm start of the force rows (solver.cpp:280-291); manifold rows have infinite stiffness
        for (int r = 0; r < 3; ++r) {
            if (!P.post_stabilization) lam[r] *= P.alpha * P.gamma;
            float np = pen[r] * P.gamma;
            if (np < kPenaltyMin) np = kPenaltyMin;
            if (np > kPenaltyMax) np = kPenaltyMax;
            pen[r] = np;
        }
        const int o = base + i;
        W.kid[cur][o] = c.id;
        W.krA[cur][o] = f4(c.rA, c.penetration);
        W.krB[cur][o] = f4(c.rB);
        W.kn[cur][o] = f4(n, C0x);
        W.kt1[cur][o] = f4(t1, C0y);
        W.kt2[cur][o] = f4(t2, C0z);
        W.krAw[cur][o] = f4(rAw, stick);
        W.krBw[cur][o] = f4(rBw);
        W.kpen[cur][o] = make_float4(pen[0], pen[1], pen[2], 0.f);
        W.klam[cur][o] = make_float4(lam[0], lam[1], lam[2], 0.f);
    }
}

// ===========================================================================
// Phase 2 (joints / springs): Joint::Initialize (joint.cpp:69-94),
// Spring::Initialize (force.hpp:106), then the penalty decay.
// ===========================================================================
AVBD_HD V3 angular_error(Q4 qA, Q4 qB, Q4 rest, float arm) {
    Q4 e = qmul(qmul(qconj(qA), qB), qconj(rest));
    return quaternion_to_rotvec(e) * arm;
}

AVBD_HD void joint_positions(const World& W, int f, V3& worldA, V3& worldB, Q4& qA, Q4& qB) {
    const int2 ab = W.fbody[f];
    const V3 rA = v3(W.frA[f]), rB = v3(W.frB[f]);
    worldA = ab.x >= 0 ? transform_point(W, ab.x, rA) : rA;
    worldB = transform_point(W, ab.y, rB);
    qA = ab.x >= 0 ? q4(W.rot[ab.x]) : q4(1.f, 0.f, 0.f, 0.f);
    qB = q4(W.rot[ab.y]);
}

// Returns true when the force is dropped this step (the contact graph changes).
AVBD_HD bool force_init(const World& W, int f) {
    int t = W.ftype[f];
    if (t & kForceRemoved) return false;
    if (t & kForceDisabled) {   // Initialize() returns false -> RemoveForce
        W.ftype[f] = t | kForceRemoved;
        return true;
    }
    const int nrows = (t & 15) == kForceJoint ? 6 : 1;
    if ((t & 15) == kForceJoint) {
        V3 wA, wB;
        Q4 qA, qB;
        joint_positions(W, f, wA, wB, qA, qB);
        W.fC0p[f] = f4(wA - wB);
        W.fC0a[f] = f4(angular_error(qA, qB, q4(W.fq[f]), W.fparam[f].x));
    }
    for (int r = 0; r < nrows; ++r) {
        const int i = f * 6 + r;
        if (!W.P.post_stabilization) W.flam[i] *= W.P.alpha * W.P.gamma;
        float np = W.fpen[i] * W.P.gamma;
        if (np < kPenaltyMin) np = kPenaltyMin;
        if (np > kPenaltyMax) np = kPenaltyMax;
        W.fpen[i] = fminf(np, W.fk[i]);
    }
    return false;
}

// Joint::ComputeConstraints (joint.cpp:97-124)
AVBD_HD void joint_C(const World& W, int f, float alpha, float C[6]) {
    V3 wA, wB;
    Q4 qA, qB;
    joint_positions(W, f, wA, wB, qA, qB);
    V3 cp = wA - wB;
    V3 ca = angular_error(qA, qB, q4(W.fq[f]), W.fparam[f].x);
    const float* k = W.fk + f * 6;
    const V3 c0p = v3(W.fC0p[f]), c0a = v3(W.fC0a[f]);
    for (int i = 0; i < 3; ++i) {
        C[i] = is_inf(k[i]) ? comp(cp, i) - comp(c0p, i) * alpha : comp(cp, i);
        C[3 + i] = is_inf(k[3 + i]) ? comp(ca, i) - comp(c0a, i) * alpha : comp(ca, i);
    }
}

// Spring::ComputeConstraints (spring.cpp:40-48)
AVBD_HD float spring_C(const World& W, int f) {
    const int2 ab = W.fbody[f];
    V3 pA = ab.x >= 0 ? transform_point(W, ab.x, v3(W.frA[f])) : v3(W.frA[f]);
    V3 pB = transform_point(W, ab.y, v3(W.frB[f]));
    return norm(pB - pA) - W.fparam[f].x;
}

// ===========================================================================
// 6x6 symmetric system, LDL^T with symmetric diagonal pivoting and the
// pseudo-inverse of D (the decomposition the reference asks Eigen::LDLT for,
// solver.cpp:437-438).
// ===========================================================================
struct Sys6 {
    float a[6][6];   // lower triangle accumulated; upper mirrored before factorising
    float r[6];
};

AVBD_HD void sys_add_row(Sys6& s, const float J[6], float pen, float f) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        s.r[i] += J[i] * f;
#pragma unroll
        for (int j = 0; j <= i; ++j) s.a[i][j] += (J[i] * J[j]) * pen;
    }
}

// The factorisation runs on the leading N x N block (N = 6, or 3 when rows
// and columns 3..5 and r[3..5] are exactly zero, as for a particle with only
// energy terms: the zero rows never win a pivot, every product they enter is
// an exact zero, and their unknowns come out 0 either way, so N = 3 performs
// the N = 6 arithmetic on the translational block minus those exact zeros).
template <int M, int N, int K, int Q>
AVBD_HD void sym_swap(float (&a)[M][M]) {
#pragma unroll
    for (int j = 0; j < N; ++j) swapf(a[K][j], a[Q][j]);
#pragma unroll
    for (int i = 0; i < N; ++i) swapf(a[i][K], a[i][Q]);
}

template <int M, int N, int K>
AVBD_HD void ldlt_pivot(float (&a)[M][M], int p) {
    if (K < 1 && 1 < N && p == 1) sym_swap<M, N, K, (1 < N ? 1 : 0)>(a);
    if (K < 2 && 2 < N && p == 2) sym_swap<M, N, K, (2 < N ? 2 : 0)>(a);
    if (K < 3 && 3 < N && p == 3) sym_swap<M, N, K, (3 < N ? 3 : 0)>(a);
    if (K < 4 && 4 < N && p == 4) sym_swap<M, N, K, (4 < N ? 4 : 0)>(a);
    if (K < 5 && 5 < N && p == 5) sym_swap<M, N, K, (5 < N ? 5 : 0)>(a);
}

template <int M, int N, int K>
AVBD_HD void ldlt_step(float (&a)[M][M], float (&d)[M], int (&t)[M]) {
    int p = K;
    float best = fabsf(a[K][K]);
#pragma unroll
    for (int i = K + 1; i < N; ++i)
        if (fabsf(a[i][i]) > best) { best = fabsf(a[i][i]); p = i; }
    t[K] = p;
    ldlt_pivot<M, N, K>(a, p);
    const float dk = a[K][K];
    d[K] = dk;
    if (dk != 0.f) {
#pragma unroll
        for (int i = K + 1; i < N; ++i) {
            const float lik = a[i][K] / dk;
#pragma unroll
            for (int j = K + 1; j <= i; ++j) a[i][j] = a[i][j] - lik * a[j][K];
        }
#pragma unroll
        for (int i = K + 1; i < N; ++i) a[i][K] = a[i][K] / dk;
#pragma unroll
        for (int i = K + 1; i < N; ++i)
#pragma unroll
            for (int j = i + 1; j < N; ++j) a[i][j] = a[j][i];
    } else {
#pragma unroll
        for (int i = K + 1; i < N; ++i) a[i][K] = 0.f;
    }
}

// Solves the leading N x N block of a (lower triangle given) for r; x[N..M) = 0.
template <int M, int N>
AVBD_HD void ldlt_solve(float (&a)[M][M], const float (&r)[M], float (&x)[M]) {
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = i + 1; j < N; ++j) a[i][j] = a[j][i];
    float d[M];
    int t[M];
#pragma unroll
    for (int i = 0; i < M; ++i) t[i] = i;
    ldlt_step<M, N, 0>(a, d, t);
    ldlt_step<M, N, 1>(a, d, t);
    ldlt_step<M, N, 2>(a, d, t);
    if constexpr (N > 3) {
        ldlt_step<M, N, 3>(a, d, t);
        ldlt_step<M, N, 4>(a, d, t);
        ldlt_step<M, N, 5>(a, d, t);
    }
#pragma unroll
    for (int i = 0; i < M; ++i) x[i] = i < N ? r[i] : 0.f;
#pragma unroll
    for (int k = 0; k + 1 < N; ++k) {
#pragma unroll
        for (int q = k + 1; q < N; ++q)
            if (t[k] == q) swapf(x[k], x[q]);
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        float v = x[i];
#pragma unroll
        for (int j = 0; j < i; ++j) v = v - a[i][j] * x[j];
        x[i] = v;
    }
    const float tiny = 1.17549435e-38f;
#pragma unroll
    for (int i = 0; i < N; ++i) x[i] = (fabsf(d[i]) > tiny) ? x[i] / d[i] : 0.f;
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
        float v = x[i];
#pragma unroll
        for (int j = i + 1; j < N; ++j) v = v - a[j][i] * x[j];
        x[i] = v;
    }
#pragma unroll
    for (int k = N - 2; k >= 0; --k) {
#pragma unroll
        for (int q = k + 1; q < N; ++q)
            if (t[k] == q) swapf(x[k], x[q]);
    }
}

// LDL^T of the leading N x N block without pivoting, one reciprocal per
// pivot.  The primal systems are symmetric positive definite whenever every
// diagonal block carries mass (inertial term plus positive semidefinite force
// and energy rows), and for those pivoting only changes rounding; the pivot
// search and the symmetric swaps are most of the pivoted solver's latency.
// Returns false, leaving x untouched, when a pivot is not clearly positive
// (e.g. a rotational block made of contact rows alone): the caller then uses
// the pivoted solver, which handles semidefinite systems.
template <int M, int N>
AVBD_HD bool ldlt_solve_spd(const float (&a)[M][M], const float (&r)[M], float (&x)[M]) {
    float l[N][N];
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) l[i][j] = a[i][j];
    float dinv[N];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const float dk = l[k][k];
        ok = ok && dk > 1e-6f * a[k][k];   // false for NaN too
        const float inv = fast_rcp(dk);
        dinv[k] = inv;
#pragma unroll
        for (int i = k + 1; i < N; ++i) {
            const float lik = l[i][k] * inv;
#pragma unroll
            for (int j = k + 1; j <= i; ++j) l[i][j] = l[i][j] - lik * l[j][k];
        }
#pragma unroll
        for (int i = k + 1; i < N; ++i) l[i][k] = l[i][k] * inv;
    }
    if (!ok) return false;
    float y[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        float v = r[i];
#pragma unroll
        for (int j = 0; j < i; ++j) v = v - l[i][j] * y[j];
        y[i] = v;
    }
#pragma unroll
    for (int i = 0; i < N; ++i) y[i] = y[i] * dinv[i];
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
        float v = y[i];
#pragma unroll
        for (int j = i + 1; j < N; ++j) v = v - l[j][i] * y[j];
        y[i] = v;
    }
#pragma unroll
    for (int i = 0; i < M; ++i) x[i] = i < N ? y[i] : 0.f;
    return true;
}

// True when rows 3..5 of the lower triangle and r[3..5] are all zero.
AVBD_HD bool sys_rotation_free(const Sys6& s) {
    bool z = s.r[3] == 0.f && s.r[4] == 0.f && s.r[5] == 0.f;
#pragma unroll
    for (int i = 3; i < 6; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) z = z && s.a[i][j] == 0.f;
    return z;
}

AVBD_HD void ldlt_solve6(Sys6& s, float (&x)[6]) {
    if (sys_rotation_free(s)) {
        if (!ldlt_solve_spd<6, 3>(s.a, s.r, x)) ldlt_solve<6, 3>(s.a, s.r, x);
    } else {
        if (!ldlt_solve_spd<6, 6>(s.a, s.r, x)) ldlt_solve<6, 6>(s.a, s.r, x);
    }
}

// ===========================================================================
// Phase 5.1 / 7: primal block update of one body (solver.cpp:392-448, :538-596)
// ===========================================================================
AVBD_HD void dot6(const float J[6], V3 dl, V3 da, float& acc) {
    acc += J[0] * dl.x + J[1] * dl.y + J[2] * dl.z + J[3] * da.x + J[4] * da.y + J[5] * da.z;
}

// Adds one manifold's rows for body b (role 0 = A, 1 = B).
AVBD_HD void primal_manifold(const World& W, int cur, int slot, int role, float alpha, bool write_stick, Sys6& s) {
    const int2 ab = W.cpair[cur][slot];
    if ((W.flags[ab.x] | W.flags[ab.y]) & kBodyRemoved) return;   // Mesh::~Mesh dropped it
    const int nc = W.cn[cur][slot];
    const float fr = W.cfric[cur][slot];
    const V3 dlA = v3(W.dlin[ab.x]), daA = v3(W.dang[ab.x]);
    const V3 dlB = v3(W.dlin[ab.y]), daB = v3(W.dang[ab.y]);
    const float oma = 1.f - alpha;
    const int kb = W.kbase[cur][slot];
    for (int k = 0; k < nc; ++k) {
        const int o = kb + k;
        const float4 n4 = W.kn[cur][o], t14 = W.kt1[cur][o], t24 = W.kt2[cur][o];
        const float4 rA4 = W.krAw[cur][o], rB4 = W.krBw[cur][o];
        const float4 pen = W.kpen[cur][o], lam = W.klam[cur][o];
        const V3 rAw = v3(rA4), rBw = v3(rB4);
        const V3 dirs[3] = {v3(n4), v3(t14), v3(t24)};
        const float C0[3] = {n4.w, t14.w, t24.w};
        const float pens[3] = {pen.x, pen.y, pen.z};
        const float lams[3] = {lam.x, lam.y, lam.z};
        const float bound = fabsf(lam.x) * fr;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const V3 d = dirs[r];
            const V3 ca = cross(rAw, d), cb = cross(rBw, d);
            const float JA[6] = {d.x, d.y, d.z, ca.x, ca.y, ca.z};
            const float JB[6] = {-d.x, -d.y, -d.z, -cb.x, -cb.y, -cb.z};
            float dA = 0.f, dB = 0.f;
            dot6(JA, dlA, daA, dA);
            dot6(JB, dlB, daB, dB);
            const float C = (oma * C0[r] + dA) + dB;
            const float fmin = r == 0 ? -INFINITY : -bound;
            const float fmax = r == 0 ? 0.f : bound;
            const float f = clampf(pens[r] * C + lams[r], fmin, fmax);
            sys_add_row(s, role == 0 ? JA : JB, pens[r], f);
        }
        if (write_stick) {
            // Manifold::ComputeConstraints stick test (manifold.cpp:229-234)
            const float tl = sqrtf(lam.y * lam.y + lam.z * lam.z);
            const float tc = sqrtf(t14.w * t14.w + t24.w * t24.w);
            float4 w = rA4;
            w.w = (tl < bound && tc < kStickThreshold) ? 1.f : 0.f;
            W.krAw[cur][o] = w;
        }
    }
}

// Adds one joint's rows (joint.cpp:97-173) for body b.
AVBD_HD void primal_joint(const World& W, int f, int b, float alpha, Sys6& s) {
    float C[6];
    joint_C(W, f, alpha, C);
    const int2 ab = W.fbody[f];
    const bool isA = (b == ab.x);
    const int bb = isA ? ab.x : ab.y;
    const V3 rl = v3(isA ? W.frA[f] : W.frB[f]);
    const V3 sc = v3(W.scale[bb]);
    const V3 r = qrotate(q4(W.rot[bb]), v3(sc.x * rl.x, sc.y * rl.y, sc.z * rl.z));
    const float arm = W.fparam[f].x;
    const float sg = isA ? 1.f : -1.f;
    for (int i = 0; i < 6; ++i) {
        const int row = f * 6 + i;
        const float k = W.fk[row];
        const float pen = W.fpen[row];
        const float lam = is_inf(k) ? W.flam[row] : 0.f;
        const float fv = clampf(pen * C[i] + lam, W.ffmin[row], W.ffmax[row]);
        float J[6];
        float h55 = 0.f;
        if (i < 3) {
            V3 e = v3(i == 0, i == 1, i == 2);
            V3 rc = cross(r, e);
            J[0] = sg * e.x; J[1] = sg * e.y; J[2] = sg * e.z;
            J[3] = sg * rc.x; J[4] = sg * rc.y; J[5] = sg * rc.z;
            h55 = -sg * comp(r, i);
        } else {
            J[0] = J[1] = J[2] = 0.f;
            J[3] = J[4] = J[5] = 0.f;
            J[i] = -sg * arm;    // rows 3+m: tail = -/+ torqueArm * e_m
        }
        sys_add_row(s, J, pen, fv);
        // includeHessian: G(j,j) = |H col j| |f|; only H(5,5) is non-zero
        s.a[5][5] += fabsf(h55) * fabsf(fv);
    }
}

// Adds one spring's row (spring.cpp:40-109) for body b.
AVBD_HD void primal_spring(const World& W, int f, int b, Sys6& s) {
    const int2 ab = W.fbody[f];
    const int row = f * 6;
    const V3 rAl = v3(W.frA[f]), rBl = v3(W.frB[f]);
    const V3 pA = ab.x >= 0 ? transform_point(W, ab.x, rAl) : rAl;
    const V3 pB = transform_point(W, ab.y, rBl);
    const V3 d = pB - pA;
    const float L = norm(d);
    const float L2 = sqnorm(d);
    const float C = L - W.fparam[f].x;
    const float k = W.fk[row];
    const float pen = W.fpen[row];
    const float lam = is_inf(k) ? W.flam[row] : 0.f;
    const float fv = clampf(pen * C + lam, W.ffmin[row], W.ffmax[row]);
    float J[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float G[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (!(L2 < 1e-6f)) {
        const V3 n = d / L;
        // dxx = (I - n n^T) / L
        float dxx[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) dxx[i][j] = ((i == j ? 1.f : 0.f) - comp(n, i) * comp(n, j)) / L;
        const bool isA = (b == ab.x && ab.x >= 0);
        const V3 r = isA ? qrotate(q4(W.rot[ab.x]), rAl) : qrotate(q4(W.rot[ab.y]), rBl);
        // S = -skew(r) for A, skew(r) for B; dxr = dxx S^T; drr = S dxx S^T -/+ skew(n) skew(r)
        float Sm[3][3] = {{0.f, -r.z, r.y}, {r.z, 0.f, -r.x}, {-r.y, r.x, 0.f}};
        const float sg = isA ? -1.f : 1.f;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Sm[i][j] *= sg;
        float dxr[3][3], drr[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                float v = 0.f;
                for (int m = 0; m < 3; ++m) v += dxx[i][m] * Sm[j][m];
                dxr[i][j] = v;
            }
        const float Kn[3][3] = {{0.f, -n.z, n.y}, {n.z, 0.f, -n.x}, {-n.y, n.x, 0.f}};
        const float Kr[3][3] = {{0.f, -r.z, r.y}, {r.z, 0.f, -r.x}, {-r.y, r.x, 0.f}};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                float v = 0.f;
                for (int m = 0; m < 3; ++m) v += Sm[i][m] * dxr[m][j];   // S (dxx S^T)
                float nr = 0.f;
                for (int m = 0; m < 3; ++m) nr += Kn[i][m] * Kr[m][j];
                drr[i][j] = v + (isA ? -nr : nr);
            }
        if (isA) {
            const V3 c = cross(n, r);
            J[0] = -n.x; J[1] = -n.y; J[2] = -n.z; J[3] = c.x; J[4] = c.y; J[5] = c.z;
        } else {
            const V3 c = cross(r, n);
            J[0] = n.x; J[1] = n.y; J[2] = n.z; J[3] = c.x; J[4] = c.y; J[5] = c.z;
        }
        // column norms of H = [dxx dxr; dxr^T drr]
        for (int j = 0; j < 3; ++j) {
            float c0 = 0.f, c1 = 0.f;
            for (int i = 0; i < 3; ++i) { c0 += dxx[i][j] * dxx[i][j]; c0 += dxr[j][i] * dxr[j][i]; }
            for (int i = 0; i < 3; ++i) { c1 += dxr[i][j] * dxr[i][j]; c1 += drr[i][j] * drr[i][j]; }
            G[j] = sqrtf(c0) * fabsf(fv);
            G[3 + j] = sqrtf(c1) * fabsf(fv);
        }
    }
    sys_add_row(s, J, pen, fv);
    for (int j = 0; j < 6; ++j) s.a[j][j] += G[j];
}

// Inertial term M/dt^2 and its right-hand side (solver.cpp:396-397).
AVBD_HD void primal_init_mass(const World& W, int b, Sys6& s) {
    const float dt = W.P.dt;
    const float dt2 = dt * dt;
    const float4 M0 = W.Mw0[b], M1 = W.Mw1[b];
    const float m = M0.x / dt2;
    s.a[0][0] = m; s.a[1][1] = m; s.a[2][2] = m;
    s.a[3][3] = M0.y / dt2; s.a[4][4] = M0.z / dt2; s.a[5][5] = M0.w / dt2;
    s.a[4][3] = M1.x / dt2; s.a[5][3] = M1.y / dt2; s.a[5][4] = M1.z / dt2;
    const V3 dl = v3(W.pos[b]) - v3(W.ipos[b]);
    const V3 da = rotation_difference(q4(W.rot[b]), q4(W.irot[b]));
    s.r[0] = m * dl.x; s.r[1] = m * dl.y; s.r[2] = m * dl.z;
    s.r[3] = s.a[3][3] * da.x + s.a[4][3] * da.y + s.a[5][3] * da.z;
    s.r[4] = s.a[4][3] * da.x + s.a[4][4] * da.y + s.a[5][4] * da.z;
    s.r[5] = s.a[5][3] * da.x + s.a[5][4] * da.y + s.a[5][5] * da.z;
}

AVBD_HD void sys_zero(Sys6& s) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        s.r[i] = 0.f;
#pragma unroll
        for (int j = 0; j < 6; ++j) s.a[i][j] = 0.f;
    }
}

// Shape gradient of a tet's vertex `role` from its Dm^-1 (column-major):
// gradN1..3 are the rows of Dm^-1 and gradN0 = -g1 - g2 - g3, with the
// reference's operations (neohookeanfem.cpp:31-36), so the values equal the
// ones the host computes bit for bit; nothing stores them.
AVBD_HD V3 tet_shape_grad(const float* D, uint32_t role) {
    if (role == 0) return v3(((-D[0]) - D[1]) - D[2], ((-D[3]) - D[4]) - D[5], ((-D[6]) - D[7]) - D[8]);
    if (role == 1) return v3(D[0], D[3], D[6]);
    if (role == 2) return v3(D[1], D[4], D[7]);
    return v3(D[2], D[5], D[8]);
}

// Gradient and projected Hessian of tet `idx` for its vertex `role`
// (NeoHookeanFEM::ComputeEnergyTerms, neohookeanfem.cpp:40-90, or the StVK
// tet); false for a removed tet.
AVBD_HD bool tet_term(const World& W, int idx, int role, V3& g, S3& H) {
    const int4 v = W.tidx[idx];
    const float4 tp = W.tparam[idx];
    if (tp.w != 0.f) return false;   // removed energy
    const float* D = W.tDmInv + (size_t)idx * 9;
    const V3 gn = tet_shape_grad(D, (uint32_t)role);
    if (W.tkind[idx] == kTetStvk)
        stvk_tet_terms(v3(W.pos[v.x]), v3(W.pos[v.y]), v3(W.pos[v.z]), v3(W.pos[v.w]), D, gn, tp.x, tp.y, tp.z,
                       W.P.projection_mode, W.P.trust_region_rho, g, H);
    else
        neohookean_terms(v3(W.pos[v.x]), v3(W.pos[v.y]), v3(W.pos[v.z]), v3(W.pos[v.w]), D, gn, tp.x, tp.y, tp.z,
                         W.P.projection_mode, W.P.trust_region_rho, g, H);
    return true;
}

// The record of a tet term for the flat sweep (slot q of the tet-term
// records), from the tet's data; made with the colouring.
__device__ __forceinline__ void write_term_record(const World& W, size_t q, uint32_t ent) {
    const int idx = (int)ent_index(ent);
    const int4 v = W.tidx[idx];
    const float4 tp = W.tparam[idx];
    const float* D = W.tDmInv + (size_t)idx * 9;
    uint32_t x = (uint32_t)v.x | (ent_role(ent) << kTermRoleShift);
    if (W.tkind[idx] == kTetStvk) x |= kTermStvk;
    if (tp.w != 0.f) x |= kTermRemoved;
    W.trv[q] = make_int4((int)x, v.y, v.z, v.w);
    W.trm0[q] = make_float4(D[0], D[1], D[2], D[3]);
    W.trm1[q] = make_float4(D[4], D[5], D[6], D[7]);
    W.trm2[q] = make_float4(D[8], tp.x, tp.y, tp.z);
}

// tet_term from the record in slot q: streamed loads (each record is read
// once per sweep) and the shape gradient of the term's vertex from Dm^-1.
__device__ __forceinline__ bool tet_term_record(const World& W, size_t q, V3& g, S3& H) {
    const int4 a = __ldcs(W.trv + q);
    const uint32_t x = (uint32_t)a.x;
    if (x & kTermRemoved) return false;
    const float4 m0 = __ldcs(W.trm0 + q), m1 = __ldcs(W.trm1 + q), m2 = __ldcs(W.trm2 + q);
    const float D[9] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w, m2.x};
    const uint32_t role = (x >> kTermRoleShift) & 3u;
    const V3 gn = tet_shape_grad(D, role);
    const V3 p0 = v3(W.pos[x & kTermIdMask]), p1 = v3(W.pos[a.y]), p2 = v3(W.pos[a.z]), p3 = v3(W.pos[a.w]);
    if (x & kTermStvk)
        stvk_tet_terms(p0, p1, p2, p3, D, gn, m2.y, m2.z, m2.w, W.P.projection_mode, W.P.trust_region_rho, g, H);
    else
        neohookean_terms(p0, p1, p2, p3, D, gn, m2.y, m2.z, m2.w, W.P.projection_mode, W.P.trust_region_rho, g, H);
    return true;
}

// Rounded adds: the term is rounded before it is accumulated, whether it was
// just computed (inlined) or read back from shared memory, so every sweep
// variant sums the same values.
AVBD_HD void sys_add_energy(Sys6& s, float gx, float gy, float gz, float hxx, float hyy, float hzz, float hxy,
                            float hxz, float hyz) {
    s.r[0] = XADD(s.r[0], gx); s.r[1] = XADD(s.r[1], gy); s.r[2] = XADD(s.r[2], gz);
    s.a[0][0] = XADD(s.a[0][0], hxx); s.a[1][1] = XADD(s.a[1][1], hyy); s.a[2][2] = XADD(s.a[2][2], hzz);
    s.a[1][0] = XADD(s.a[1][0], hxy); s.a[2][0] = XADD(s.a[2][0], hxz); s.a[2][1] = XADD(s.a[2][1], hyz);
}

AVBD_HD void sys_add_energy(Sys6& s, const V3& g, const S3& H) {
    sys_add_energy(s, g.x, g.y, g.z, H.xx, H.yy, H.zz, H.xy, H.xz, H.yz);
}

// Adds the rows of incidence entries e0 + first, e0 + first + stride, ... < e1
// of body b (solver.cpp:399-435): forces (manifolds, joints, springs) then
// energies.
AVBD_HD void primal_entry_range(const World& W, int cur, int b, float alpha, bool write_stick, int e0, int e1,
                                int first, int stride, Sys6& s) {
    for (int e = e0 + first; e < e1; e += stride) {
        const uint32_t ent = W.inc[e];
        const uint32_t kind = ent_kind(ent), idx = ent_index(ent);
        if (kind == kEntManifold) {
            primal_manifold(W, cur, (int)idx, (int)ent_role(ent), alpha, write_stick, s);
        } else if (kind == kEntForce) {
            const int t = W.ftype[idx];
            if (t & kForceRemoved) continue;
            if ((t & 15) == kForceJoint) primal_joint(W, (int)idx, b, alpha, s);
            else primal_spring(W, (int)idx, b, s);
        } else if (kind == kEntTet) {
            V3 g;
            S3 H;
            if (tet_term(W, (int)idx, (int)ent_role(ent), g, H)) sys_add_energy(s, g, H);
        } else {
            const int4 v = W.ridx[idx];
            const float4 rp = W.rparam[idx];
            if (rp.w != 0.f) continue;
            const int role = (int)ent_role(ent);
            const float* gn = W.rgradN + (size_t)idx * 6 + role * 2;
            V3 g;
            S3 H;
            stvk_terms(v3(W.pos[v.x]), v3(W.pos[v.y]), v3(W.pos[v.z]), W.rDmInv[idx], gn[0], gn[1], rp.x, rp.y,
                       rp.z, W.P.projection_mode, W.P.trust_region_rho, g, H);
            sys_add_energy(s, g, H);
        }
    }
}

AVBD_HD void primal_entries(const World& W, int cur, int b, float alpha, bool write_stick, int first, int stride,
                            Sys6& s) {
    const int e0 = W.inc_off[b];
    primal_entry_range(W, cur, b, alpha, write_stick, e0, e0 + W.inc_cnt[b], first, stride, s);
}

// LDLT solve and pose update (solver.cpp:437-448).
AVBD_HD void primal_apply(const World& W, int b, const float (&x)[6]) {
    const V3 pos = v3(W.pos[b]);
    const Q4 rot = q4(W.rot[b]);
    const V3 npos = pos - v3(x[0], x[1], x[2]);
    // a zero rotation step gives dq = (1, 0, 0, 0) and qmul(dq, rot) = rot
    // exactly (up to the sign of zero components), so it is skipped
    const bool turn = x[3] != 0.f || x[4] != 0.f || x[5] != 0.f;
    const Q4 nrot = qnormalize(turn ? qmul(quaternion_from_difference(v3(x[3], x[4], x[5]), -1.f), rot) : rot);
    W.pos[b] = f4(npos);
    W.rot[b] = f4(nrot);
    W.dlin[b] = f4(npos - v3(W.lpos[b]));
    W.dang[b] = f4(rotation_difference(nrot, q4(W.lrot[b])));
}

// A particle has no rotational inertia (solver.cpp:119-131): whenever force
// rows reach its rotational block, that block holds contact torques alone and
// is close to singular, so the solve follows the reference's factorisation
// step for step (symmetric pivoting on the largest diagonal, the pivot rule
// of the Eigen LDLT it calls at solver.cpp:437-438) instead of the unpivoted
// shortcut, whose different elimination order rounds differently.
AVBD_HD void primal_finish(const World& W, int b, Sys6& s) {
    float x[6];
    if ((W.flags[b] & kBodyParticle) && !sys_rotation_free(s)) ldlt_solve<6, 6>(s.a, s.r, x);
    else ldlt_solve6(s, x);
    primal_apply(W, b, x);
}

// A particle whose incidence holds only energy terms has exactly zero
// rotational rows (no inertia, no force rows): its translational 3x3 system
// alone performs the same arithmetic as primal_init_mass + ldlt_solve<6, 3>.
struct Sys3 {
    float a[3][3];
    float r[3];
};

AVBD_HD bool energy_only_particle(const World& W, int b) {
    if (!(W.flags[b] & kBodyParticle)) return false;
    const float4 M0 = W.Mw0[b], M1 = W.Mw1[b];
    return M0.y == 0.f && M0.z == 0.f && M0.w == 0.f && M1.x == 0.f && M1.y == 0.f && M1.z == 0.f;
}

AVBD_HD void particle_init_mass(const World& W, int b, Sys3& s) {
    const float dt = W.P.dt;
    const float dt2 = dt * dt;
    const float m = W.Mw0[b].x / dt2;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) s.a[i][j] = i == j ? m : 0.f;
    const V3 dl = v3(W.pos[b]) - v3(W.ipos[b]);
    s.r[0] = m * dl.x; s.r[1] = m * dl.y; s.r[2] = m * dl.z;
}


AVBD_HD void particle_finish(const World& W, int b, Sys3& s) {
    float x3[3];
    if (!ldlt_solve_spd<3, 3>(s.a, s.r, x3)) ldlt_solve<3, 3>(s.a, s.r, x3);
    const float x[6] = {x3[0], x3[1], x3[2], 0.f, 0.f, 0.f};
    primal_apply(W, b, x);
}

// One body by one thread, in the reference's summation order.
AVBD_HD void primal_body(const World& W, int cur, int b, float alpha, bool write_stick) {
    Sys6 s;
    sys_zero(s);
    primal_init_mass(W, b, s);
    primal_entries(W, cur, b, alpha, write_stick, 0, 1, s);
    primal_finish(W, b, s);
}

// ===========================================================================
// Phase 5.3: dual update (solver.cpp:457-489)
// ===========================================================================
// Dual of one row; returns true when the row fractures.
AVBD_HD bool dual_row(float C, float k, float fmin, float fmax, float frac, float beta, float& pen, float& lam) {
    const float l0 = is_inf(k) ? lam : 0.f;
    float l = l0 + pen * C;
    if (l < fmin) l = fmin;
    else if (l > fmax) l = fmax;
    lam = l;
    if (fabsf(l) >= frac) return true;
    if (l > fmin && l < fmax) pen = fminf(pen + beta * fabsf(C), fminf(k, kPenaltyMax));
    return false;
}

// write_stick: the last ComputeConstraints call of the step decides the stick
// flag, so only the final dual sweep needs to store it.
AVBD_HD void dual_manifold(const World& W, int cur, int slot, float alpha, bool write_stick = true) {
    const int nc = W.cn[cur][slot];
    if (nc == 0) return;
    const int2 ab = W.cpair[cur][slot];
    const float fr = W.cfric[cur][slot];
    const V3 dlA = v3(W.dlin[ab.x]), daA = v3(W.dang[ab.x]);
    const V3 dlB = v3(W.dlin[ab.y]), daB = v3(W.dang[ab.y]);
    const float oma = 1.f - alpha;
    const float beta = W.P.beta;
    const int kb = W.kbase[cur][slot];
    for (int k = 0; k < nc; ++k) {
        const int o = kb + k;
        const float4 n4 = W.kn[cur][o], t14 = W.kt1[cur][o], t24 = W.kt2[cur][o];
        float4 rA4 = W.krAw[cur][o];
        const V3 rAw = v3(rA4), rBw = v3(W.krBw[cur][o]);
        float4 pen = W.kpen[cur][o], lam = W.klam[cur][o];
        const V3 dirs[3] = {v3(n4), v3(t14), v3(t24)};
        const float C0[3] = {n4.w, t14.w, t24.w};
        float C[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const V3 d = dirs[r];
            const V3 ca = cross(rAw, d), cb = cross(rBw, d);
            const float JA[6] = {d.x, d.y, d.z, ca.x, ca.y, ca.z};
            const float JB[6] = {-d.x, -d.y, -d.z, -cb.x, -cb.y, -cb.z};
            float dA = 0.f, dB = 0.f;
            dot6(JA, dlA, daA, dA);
            dot6(JB, dlB, daB, dB);
            C[r] = (oma * C0[r] + dA) + dB;
        }
        const float bound = fabsf(lam.x) * fr;
        const float tl = sqrtf(lam.y * lam.y + lam.z * lam.z);
        const float tc = sqrtf(t14.w * t14.w + t24.w * t24.w);
        if (write_stick) {
            rA4.w = (tl < bound && tc < kStickThreshold) ? 1.f : 0.f;
            W.krAw[cur][o] = rA4;
        }
        dual_row(C[0], INFINITY, -INFINITY, 0.f, INFINITY, beta, pen.x, lam.x);
        dual_row(C[1], INFINITY, -bound, bound, INFINITY, beta, pen.y, lam.y);
        dual_row(C[2], INFINITY, -bound, bound, INFINITY, beta, pen.z, lam.z);
        W.kpen[cur][o] = pen;
        W.klam[cur][o] = lam;
    }
}

// Returns true when the force fractured (its linked bodies then reset their manifolds).
AVBD_HD bool dual_force(const World& W, int f, float alpha) {
    const int t = W.ftype[f];
    if (t & kForceRemoved) return false;
    const float beta = W.P.beta;
    bool broke = false;
    if ((t & 15) == kForceJoint) {
        float C[6];
        joint_C(W, f, alpha, C);
        for (int i = 0; i < 6; ++i) {
            const int row = f * 6 + i;
            if (dual_row(C[i], W.fk[row], W.ffmin[row], W.ffmax[row], W.ffrac[row], beta, W.fpen[row],
                         W.flam[row])) {
                broke = true;
                break;
            }
        }
        if (broke) {
            for (int i = 0; i < 6; ++i) { W.flam[f * 6 + i] = 0.f; W.fpen[f * 6 + i] = 0.f; }
        }
    } else {
        const int row = f * 6;
        const float C = spring_C(W, f);
        if (dual_row(C, W.fk[row], W.ffmin[row], W.ffmax[row], W.ffrac[row], beta, W.fpen[row], W.flam[row])) {
            broke = true;
            W.flam[row] = 0.f;
            W.fpen[row] = 0.f;
        }
    }
    if (broke) {
        W.ftype[f] = t | kForceDisabled;      // Force::Disable (force.hpp:57-66)
        const int2 ab = W.fbody[f];
        if (ab.x >= 0) W.reset_flag[ab.x] = 1;
        W.reset_flag[ab.y] = 1;
    }
    return broke;
}

// Force::ResetValues on every manifold of a body linked to a fractured force
// (solver.cpp:473-481).  Order independent: a reset manifold ends the sweep
// with lambda = penalty = 0 whether it was visited before or after the reset.
AVBD_HD void fracture_reset_slot(const World& W, int cur, int slot) {
    const int nc = W.cn[cur][slot];
    if (nc == 0) return;
    const int2 ab = W.cpair[cur][slot];
    if (!(W.reset_flag[ab.x] | W.reset_flag[ab.y])) return;
    const int kb = W.kbase[cur][slot];
    for (int k = 0; k < nc; ++k) {
        const int o = kb + k;
        W.kpen[cur][o] = make_float4(0.f, 0.f, 0.f, 0.f);
        W.klam[cur][o] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// ===========================================================================
// Phase 6: velocity update, explosion and out-of-bounds (solver.cpp:493-534)
// Returns bit 0 = exploded, bit 1 = NaN, bit 2 = out of bounds.
// ===========================================================================
AVBD_HD int velocity_body(const World& W, int b) {
    const int fl = W.flags[b];
    if (fl & kBodyRemoved) return 0;
    const float dt = W.P.dt;
    int res = 0;
    if (!(fl & kBodyStatic)) {
        W.pvel[b] = W.vel[b];
        const V3 pos = v3(W.pos[b]);
        const V3 v = (pos - v3(W.lpos[b])) / dt;
        W.vel[b] = f4(v);
        if (!(fl & kBodyParticle)) W.omega[b] = f4(rotation_difference(q4(W.rot[b]), q4(W.lrot[b])) / dt);
        if (pos.x < kBoundMin || pos.x > kBoundMax || pos.y < kBoundMin || pos.y > kBoundMax ||
            pos.z < kBoundMin || pos.z > kBoundMax)
            res |= 4;
        if (isnan(pos.x) || isnan(pos.y) || isnan(pos.z)) res |= 2;
    }
    const float4 v = W.vel[b];
    if (v.x > kMaxVelocity || v.y > kMaxVelocity || v.z > kMaxVelocity || v.x < -kMaxVelocity ||
        v.y < -kMaxVelocity || v.z < -kMaxVelocity)
        res |= 1;
    return res;
}

}  // namespace avbd
