// Shared definitions of the AVBD device library: constants, the device world
// layout (structure of arrays), and small vector / quaternion helpers.
//
// Arithmetic convention.  Functions marked "exact" use the X* macros, which
// round every operation to nearest-even without FMA contraction (the
// __f*_rn intrinsics on the device; host builds use -ffp-contract=off).  They
// follow the reference's expression order term by term, so the narrowphase
// (contact counts, feature ids, contact geometry) matches the CPU oracle bit
// for bit on equal inputs.  Everything else uses ordinary fused arithmetic.
#pragma once

#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define AVBD_HD __host__ __device__ __forceinline__
#define AVBD_D __device__ __forceinline__
#else
#define AVBD_HD inline
#define AVBD_D inline
#endif

#if defined(__CUDA_ARCH__)
#define XMUL(a, b) __fmul_rn((a), (b))
#define XADD(a, b) __fadd_rn((a), (b))
#define XSUB(a, b) __fsub_rn((a), (b))
#define XDIV(a, b) __fdiv_rn((a), (b))
#define XSQRT(a) __fsqrt_rn(a)
#else
#define XMUL(a, b) ((a) * (b))
#define XADD(a, b) ((a) + (b))
#define XSUB(a, b) ((a) - (b))
#define XDIV(a, b) ((a) / (b))
#define XSQRT(a) sqrtf(a)
#endif

namespace avbd {

// ---- constants of the reference (solver.cpp:7-15, force.hpp:149-150, constants.hpp:11-12) ----
constexpr float kGravityY = -9.81f;
constexpr float kPenaltyMin = 1.0f;
constexpr float kPenaltyMax = 1000000000.0f;
constexpr float kMaxRotationVelocity = 50.0f;
constexpr float kMaxVelocity = 500.0f;
constexpr float kCollisionMargin = 0.0005f;
constexpr float kStickThreshold = 0.01f;
constexpr float kBoundMin = -50.f;
constexpr float kBoundMax = 50.f;
constexpr float kNewContactPenaltyMax = 100000.0f;   // manifold.cpp:186

constexpr int kMaxContacts = 8;       // Manifold::contactPoints[8] (force.hpp:172)
constexpr int kMaxColours = 1024;     // colour slots per scene
constexpr int kSceneStamps = 9;         // AVBD_SCENE_STAMPS: start, 7 phase ends, end
constexpr int kColourWorkBuckets = 16; // work classes used to order bodies within a colour
constexpr int kGroupFlat = 64;         // SceneDesc::group of scenes swept term-per-lane (AVBD_GROUP_FLAT)
constexpr int kStagedBodies = 2560;    // batched kernel: shared-memory stage of a 256-thread CTA in float4 (40 KB);
                                       // smaller CTAs get proportionally less

// tet energy models
constexpr int kTetNeoHookean = 0;      // NeoHookeanFEM (neohookeanfem.cpp)
constexpr int kTetStvk = 1;            // St. Venant-Kirchhoff tet (no reference counterpart)
// Top bits of a tet-term record's first vertex id (ids stay below kMaxPoolBodies).
constexpr int kTermRoleShift = 28;     // 2 bits: the vertex the term is for
constexpr uint32_t kTermStvk = 1u << 30;
constexpr uint32_t kTermRemoved = 1u << 31;
constexpr uint32_t kTermIdMask = (1u << kTermRoleShift) - 1u;
constexpr long long kMaxPoolBodies = 1ll << kTermRoleShift;

// body flags
constexpr int kBodyStatic = 1;
constexpr int kBodyParticle = 2;
constexpr int kBodyHasMass = 4;       // !isStatic && mass > 0 at the mass cache
constexpr int kBodyRemoved = 8;
constexpr int kBodyModelShift = 8;    // flags bits 8..11: the body's ModelType (geometry.hpp:17-22)

// incidence entry kinds (top 3 bits) and roles (next 2 bits)
constexpr uint32_t kEntForce = 0u;
constexpr uint32_t kEntManifold = 1u;
constexpr uint32_t kEntTet = 2u;
constexpr uint32_t kEntTri = 3u;
AVBD_HD uint32_t ent_make(uint32_t kind, uint32_t role, uint32_t idx) { return (kind << 29) | (role << 27) | idx; }
AVBD_HD uint32_t ent_kind(uint32_t e) { return e >> 29; }
AVBD_HD uint32_t ent_role(uint32_t e) { return (e >> 27) & 3u; }
AVBD_HD uint32_t ent_index(uint32_t e) { return e & 0x07FFFFFFu; }

// force kinds
constexpr int kForceJoint = 0;
constexpr int kForceSpring = 1;
constexpr int kForceDisabled = 1 << 4;   // Force::disabled (force.hpp:42)
constexpr int kForceRemoved = 1 << 5;    // dropped by Initialize() == false
constexpr int kForceRope = 1 << 6;       // Spring::isRope (spring.cpp:20-24)

// scene status (avbd.h)
constexpr int kStatusOk = 0;
constexpr int kStatusExploded = 1;
constexpr int kStatusNan = 2;
constexpr int kStatusCapacity = 3;
constexpr int kStatusTimeout = 4;

struct Params {
    int num_iterations;
    float dt;
    float alpha;
    float beta;
    float gamma;
    float on_penetration_penalty;
    int post_stabilization;
    int projection_mode;
    float trust_region_rho;
};

// Per-scene description.  All indices are global into the world's pools.
struct SceneDesc {
    int body0, nbody;        // bodies
    int force0, nforce;      // joints + springs
    int tet0, ntet;          // Neo-Hookean tets
    int tri0, ntri;          // StVK triangles
    int cand0, candcap;      // candidate-pair / manifold slots
    int k0, kcap;            // contact slots (bump-allocated per step)
    int inc0, inccap;        // incidence (CSR) entries
    int ndynamic;
    int group;               // lanes per body in the primal sweep (1, 2, 4, 8, 16, 32) or kGroupFlat
};

// Per-scene mutable counters (device).
struct SceneState {
    int status;              // kStatus*
    int cur;                 // manifold table holding the live manifolds
    int ncand[2];            // candidate slots of each table
    int kused[2];            // contact slots used by each table
    int ncolours;
    int flags;               // bit 0 exploded, 1 NaN, 2 out of bounds, 3 fracture this sweep
    int ninc;                // incidence entries this step
    int need_cand;           // capacity requests (set when a table was too small)
    int need_k;
    int need_inc;
    int step;                // steps taken (stamps manifold creation)
    int nlive[2];            // live manifolds of each table
    int nmatched;            // live manifolds this step whose pair was live last step
    int topo;                // bumped when a force or body is removed
    int coloured_topo;       // topo value the current colouring was made for
    int colours_valid;       // the colour lists describe the current contact graph
    int npend;               // batched narrowphase: candidate pairs not separated by an axis this step
    int pad;
};

// Structure-of-arrays device world.  One instance is passed by value to kernels.
struct World {
    int nscenes;
    int stage_bodies;   // batched kernel: float4 slots of dynamic shared memory per CTA
    int team_work;      // batched kernel: bodies + tets per lane below which a team splits (0 = never)
    int fem_team_work;  // the same for scenes with tets (0 = never)
    int grid_min;       // batched kernel: scenes from this many bodies use the grid broadphase (0 = never)
    int* fail_count;    // batched kernel: scene steps stopped by a full table (host grows and catches up)
    int* check;         // debug builds: first failed index check (code, index, bound) and the failure count
    unsigned long long* scene_ns;   // batched kernel, optional: per scene slot kSceneStamps global-timer
                                    // readings (ns) through its last step
    const SceneDesc* scenes;
    SceneState* sstate;

    // ---- bodies (global index b) ----
    float4* pos;        // xyz
    float4* rot;        // quaternion x y z w
    float4* scale;      // sx sy sz, w = detectionRadius
    float4* lpos;       // lastPosition
    float4* lrot;       // lastRotation
    float4* ipos;       // inertialPosition
    float4* irot;       // inertialRotation
    float4* vel;        // velocity
    float4* omega;      // angularVelocity
    float4* pvel;       // prevVelocity
    float4* dlin;       // pos - lastPosition (cached per body update)
    float4* dang;       // RotationDifference(rot, lastRotation)
    float4* massI;      // mass, body-frame inertia diagonal (x, y, z)
    float4* Mw0;        // cachedGeneralizedMass: m, world I (xx, yy, zz)
    float4* Mw1;        // world I (xy, xz, yz), unused
    int* flags;
    float* friction;
    float4* color;      // Mesh::color (r g b 1): read only by the instance export
    int* colour;
    int* local;         // body index within its scene
    int* reset_flag;    // set by a fracturing force for the manifold reset pass

    // ---- static incidence (forces + energies), per body, built at upload ----
    const int* sinc_off;     // per body: first entry in sinc
    const int* sinc_n;       // per body: number of entries
    const int* sinc_nf;      // per body: leading force entries (energy entries follow)
    const uint32_t* sinc;    // entries
    const int* spartner_off; // per body: first joint/spring partner (broadphase filter)
    const int* spartner_n;   // per body: number of partners
    const int* spartner;     // (partner body, force) pairs, as int2

    // ---- per-step incidence (CSR) ----
    int* inc_off;       // per body start (global into inc), inc_off[b]..inc_off[b]+inc_cnt[b]
    int* inc_cnt;
    uint32_t* inc;      // entries
    int* cntB;          // per body count of manifolds where it is body B
    int* bcur;          // per body cursor for the B-side scatter

    // ---- broadphase candidates / manifolds (double-buffered tables) ----
    int* cand_cnt;      // per body number of candidates it owns (as body A)
    int* cand_off;      // per body start (scene-local slot)
    int2* cpair[2];     // (A, B) global body ids per slot
    int* cn[2];         // contact count per slot
    float* cfric[2];    // friction per slot
    int* kbase[2];      // first contact slot of each candidate slot
    int* cbirth[2];     // step at which the slot's manifold was created (Mesh::forces order)
    int* live[2];       // live manifold slots of each table, nlive[t] of them from the scene's cand0
    // contact slots: slot * kMaxContacts + k
    uint32_t* kid[2];
    float4* krA[2];     // local rA (xyz), w = penetration
    float4* krB[2];     // local rB
    float4* kn[2];      // n = -normal (xyz), w = C0[0]
    float4* kt1[2];     // t1, w = C0[1]
    float4* kt2[2];     // t2, w = C0[2]
    float4* krAw[2];    // rotA * rA, w = stick (0/1)
    float4* krBw[2];    // rotB * rB
    float4* kpen[2];    // penalty n, t1, t2
    float4* klam[2];    // lambda n, t1, t2

    // ---- joints and springs (global force index f) ----
    int* ftype;         // kForce* | flags
    int2* fbody;        // (A or -1, B) global body ids
    float4* frA;        // local rA (world point when A = -1)
    float4* frB;
    float4* fq;         // joint restRotation (x y z w)
    float4* fparam;     // joint: torqueArm; spring: restLength
    float4* fC0p;       // joint C0_pos
    float4* fC0a;       // joint C0_ang
    float* fk;          // stiffness [f*6 + row]
    float* ffrac;       // fracture
    float* ffmin;       // fminMagnitude
    float* ffmax;       // fmaxMagnitude
    float* fpen;        // penalty
    float* flam;        // lambda

    // ---- Neo-Hookean tets ----
    int4* tidx;
    float* tDmInv;      // 9 per tet, column-major
    float4* tparam;     // restVolume, mu, lambda
    int* tkind;         // energy model of each tet (kTetNeoHookean, kTetStvk)

    // ---- StVK triangles ----
    int4* ridx;
    float4* rDmInv;     // 2x2 column-major
    float* rgradN;      // 6 per tri: gradN0..2 (2D)
    float4* rparam;     // restArea, mu, lambda

    // ---- colouring ----
    int* col_list;      // per scene region [body0, body0+nbody): bodies grouped by colour
    int* col_tinc;      // flat-sweep scenes: inclusive prefix of tet terms over the scene's col_list
    // Flat-sweep scenes: one record per tet term in colour-list order (4 slots
    // per tet from 4 * tet0), written with the colouring so the sweep reads
    // them coalesced instead of gathering tet data.  trv: the tet's vertex ids,
    // .x carrying the term's role, model and removal in its top bits
    // (kTermRoleShift...); trm0..2: Dm^-1 (column-major), restVolume, mu, lambda.
    int4* trv;
    float4* trm0;       // Dm^-1[0..3]
    float4* trm1;       // Dm^-1[4..7]
    float4* trm2;       // Dm^-1[8], restVolume, mu, lambda
    int* col_start;     // per scene kMaxColours+1 offsets (scene * (kMaxColours+1))

    Params P;
};

// ---------------------------------------------------------------------------
// Vector helpers
// ---------------------------------------------------------------------------
struct V3 { float x, y, z; };
// Fast reciprocal and reciprocal square root (a couple of ulp on the device,
// where they replace IEEE divide / square-root sequences on latency-critical
// chains; plain on the host).
#if defined(__CUDA_ARCH__)
AVBD_HD float fast_rcp(float x) { return __fdividef(1.f, x); }
AVBD_HD float fast_rsqrt(float x) { return rsqrtf(x); }
#else
AVBD_HD float fast_rcp(float x) { return 1.f / x; }
AVBD_HD float fast_rsqrt(float x) { return 1.f / sqrtf(x); }
#endif

struct Q4 { float x, y, z, w; };   // quaternion, Eigen coefficient order

AVBD_HD V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
AVBD_HD V3 v3(float4 a) { return v3(a.x, a.y, a.z); }
AVBD_HD Q4 q4(float4 a) { Q4 q; q.x = a.x; q.y = a.y; q.z = a.z; q.w = a.w; return q; }
AVBD_HD Q4 q4(float w, float x, float y, float z) { Q4 q; q.x = x; q.y = y; q.z = z; q.w = w; return q; }
AVBD_HD float4 f4(V3 a, float w = 0.f) { float4 r; r.x = a.x; r.y = a.y; r.z = a.z; r.w = w; return r; }
AVBD_HD float4 f4(Q4 a) { float4 r; r.x = a.x; r.y = a.y; r.z = a.z; r.w = a.w; return r; }
AVBD_HD float comp(const V3& a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// ---- fused (ordinary) arithmetic ----
AVBD_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
AVBD_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
AVBD_HD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
AVBD_HD V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
AVBD_HD V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
AVBD_HD V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
AVBD_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
AVBD_HD V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
AVBD_HD float sqnorm(V3 a) { return dot(a, a); }
AVBD_HD float norm(V3 a) { return sqrtf(sqnorm(a)); }

// ---- exact (unfused, reference order) arithmetic ----
AVBD_HD V3 xadd(V3 a, V3 b) { return v3(XADD(a.x, b.x), XADD(a.y, b.y), XADD(a.z, b.z)); }
AVBD_HD V3 xsub(V3 a, V3 b) { return v3(XSUB(a.x, b.x), XSUB(a.y, b.y), XSUB(a.z, b.z)); }
AVBD_HD V3 xmul(V3 a, float s) { return v3(XMUL(a.x, s), XMUL(a.y, s), XMUL(a.z, s)); }
AVBD_HD V3 xdiv(V3 a, float s) { return v3(XDIV(a.x, s), XDIV(a.y, s), XDIV(a.z, s)); }
AVBD_HD float xdot(V3 a, V3 b) { return XADD(XADD(XMUL(a.x, b.x), XMUL(a.y, b.y)), XMUL(a.z, b.z)); }
AVBD_HD V3 xcross(V3 a, V3 b) {
    return v3(XSUB(XMUL(a.y, b.z), XMUL(a.z, b.y)), XSUB(XMUL(a.z, b.x), XMUL(a.x, b.z)),
              XSUB(XMUL(a.x, b.y), XMUL(a.y, b.x)));
}
AVBD_HD float xnorm(V3 a) { return XSQRT(xdot(a, a)); }

// 3x3 matrix, column-major columns c[0..2]
struct M3 { V3 c[3]; };
AVBD_HD float m3(const M3& m, int i, int j) { return comp(m.c[j], i); }

// Quaternion::toRotationMatrix (exact, coefficient order of the standard formula)
AVBD_HD M3 xrotmat(Q4 q) {
    const float tx = XMUL(2.f, q.x), ty = XMUL(2.f, q.y), tz = XMUL(2.f, q.z);
    const float twx = XMUL(tx, q.w), twy = XMUL(ty, q.w), twz = XMUL(tz, q.w);
    const float txx = XMUL(tx, q.x), txy = XMUL(ty, q.x), txz = XMUL(tz, q.x);
    const float tyy = XMUL(ty, q.y), tyz = XMUL(tz, q.y), tzz = XMUL(tz, q.z);
    M3 r;
    r.c[0] = v3(XSUB(1.f, XADD(tyy, tzz)), XADD(txy, twz), XSUB(txz, twy));
    r.c[1] = v3(XSUB(txy, twz), XSUB(1.f, XADD(txx, tzz)), XADD(tyz, twx));
    r.c[2] = v3(XADD(txz, twy), XSUB(tyz, twx), XSUB(1.f, XADD(txx, tyy)));
    return r;
}
// R * v, row i = (R(i,0) v0 + R(i,1) v1) + R(i,2) v2 (exact)
AVBD_HD V3 xmatvec(const M3& r, V3 v) {
    return v3(XADD(XADD(XMUL(r.c[0].x, v.x), XMUL(r.c[1].x, v.y)), XMUL(r.c[2].x, v.z)),
              XADD(XADD(XMUL(r.c[0].y, v.x), XMUL(r.c[1].y, v.y)), XMUL(r.c[2].y, v.z)),
              XADD(XADD(XMUL(r.c[0].z, v.x), XMUL(r.c[1].z, v.y)), XMUL(r.c[2].z, v.z)));
}
// R^T * v (exact): component k = dot(col_k, v)
AVBD_HD V3 xmattvec(const M3& r, V3 v) { return v3(xdot(r.c[0], v), xdot(r.c[1], v), xdot(r.c[2], v)); }

// ---- fused matrix helpers ----
AVBD_HD M3 rotmat(Q4 q) {
    const float tx = 2.f * q.x, ty = 2.f * q.y, tz = 2.f * q.z;
    const float twx = tx * q.w, twy = ty * q.w, twz = tz * q.w;
    const float txx = tx * q.x, txy = ty * q.x, txz = tz * q.x;
    const float tyy = ty * q.y, tyz = tz * q.y, tzz = tz * q.z;
    M3 r;
    r.c[0] = v3(1.f - (tyy + tzz), txy + twz, txz - twy);
    r.c[1] = v3(txy - twz, 1.f - (txx + tzz), tyz + twx);
    r.c[2] = v3(txz + twy, tyz - twx, 1.f - (txx + tyy));
    return r;
}
AVBD_HD V3 matvec(const M3& r, V3 v) { return r.c[0] * v.x + r.c[1] * v.y + r.c[2] * v.z; }

// ---- quaternions (fused) ----
AVBD_HD Q4 qmul(Q4 a, Q4 b) {
    return q4(a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
              a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z, a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x);
}
AVBD_HD Q4 qconj(Q4 a) { return q4(a.w, -a.x, -a.y, -a.z); }
AVBD_HD V3 qvec(Q4 a) { return v3(a.x, a.y, a.z); }
AVBD_HD Q4 qnormalize(Q4 q) {
    float n2 = ((q.x * q.x + q.y * q.y) + q.z * q.z) + q.w * q.w;
    if (n2 > 0.f) {
        const float inv = fast_rsqrt(n2);
        q.x *= inv; q.y *= inv; q.z *= inv; q.w *= inv;
    }
    return q;
}
// v + w*t + u x t with t = 2 (u x v)  (Quaternion * Vector3)
AVBD_HD V3 qrotate(Q4 q, V3 v) {
    V3 u = qvec(q);
    V3 uv = cross(u, v);
    uv = uv + uv;
    return v + q.w * uv + cross(u, uv);
}

// RotationDifference (math.hpp:10-28)
AVBD_HD V3 rotation_difference(Q4 q, Q4 p) {
    Q4 dq = qmul(q, qconj(p));
    if (dq.w < 0.f) { dq.x = -dq.x; dq.y = -dq.y; dq.z = -dq.z; dq.w = -dq.w; }
    V3 v = qvec(dq);
    float sin_half = norm(v);
    if (sin_half < 1e-6f) return 2.f * v;
    float half = atan2f(sin_half, dq.w);
    return (2.f * half * fast_rcp(sin_half)) * v;
}
// QuaternionFromDifference (math.hpp:31-48)
AVBD_HD Q4 quaternion_from_difference(V3 v, float sign) {
    float angle = norm(v);
    Q4 q;
    if (angle < 1e-6f) {
        q.w = 1.f;
        V3 h = (sign * 0.5f) * v;
        q.x = h.x; q.y = h.y; q.z = h.z;
    } else {
        float ha = 0.5f * angle;
        float s, c;
        sincosf(ha, &s, &c);
        q.w = c;
        V3 h = (sign * s * fast_rcp(angle)) * v;
        q.x = h.x; q.y = h.y; q.z = h.z;
    }
    return qnormalize(q);
}
// QuaternionToRotVec (math.hpp:51-63)
AVBD_HD V3 quaternion_to_rotvec(Q4 q) {
    Q4 qn = q.w >= 0.f ? q : q4(-q.w, -q.x, -q.y, -q.z);
    V3 v = qvec(qn);
    float sin_half = norm(v);
    if (sin_half < 1e-6f) return v3(0.f, 0.f, 0.f);
    float half = atan2f(sin_half, qn.w);
    return v * (2.f * half / sin_half);
}

AVBD_HD float clampf(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }


// Index checks of debug builds (-DAVBD_CHECKS, skyephyx_b200.build
// checks=True): a failed check records the first violation (code, index,
// bound) and counts it in the world's check word, and the caller skips the
// access; nothing traps.  Release builds compile the checks away.  Codes:
// 1 / 2 incidence entry (owned / B side) outside the scene's incidence
// region, 3 a broadphase row wrote another count than it counted, 4 a colour
// list slot outside the scene's bodies, 5 a tet-term record outside the
// scene's records, 6 a contact block outside the scene's contact region.
#if defined(AVBD_CHECKS) && defined(__CUDACC__)
__device__ __forceinline__ bool avbd_check(const World& W, bool ok, int code, long long index, long long bound) {
    if (ok) return true;
    if (W.check) {
        if (atomicCAS(W.check, 0, code) == 0) {
            W.check[1] = (int)index;
            W.check[2] = (int)bound;
        }
        atomicAdd(W.check + 3, 1);
    }
    return false;
}
#define AVBD_CHECK(W, ok, code, index, bound) avbd_check((W), (ok), (code), (long long)(index), (long long)(bound))
#else
#define AVBD_CHECK(W, ok, code, index, bound) true
#endif

AVBD_HD uint32_t colour_priority(uint32_t x) {
    // integer mixer (Wellons "lowbias32"); the CPU colouring twin uses the same function
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return x;
}

}  // namespace avbd
