// Box-box narrowphase: 15-axis SAT, Sutherland-Hodgman face clipping and
// edge-edge closest points, restated from SkyePhyX
// src/physics/collision.cpp:26-447 with exact (unfused) arithmetic in the
// reference's expression order, so feature ids, counts and contact geometry
// match the CPU oracle bit for bit on equal inputs.
#pragma once
#include "avbd_common.cuh"

namespace avbd {

struct Contact {
    V3 position;
    V3 normal;          // points A -> B
    float penetration;
    V3 rA, rB;          // body-local anchors
    uint32_t id;
};

struct Collision {
    Contact c[kMaxContacts];
    int n;
};

// createID (collision.cpp:26-32)
AVBD_HD uint32_t create_id(int type, int axis_a, int axis_b, int vertex) {
    return ((uint32_t)type & 0x3u) | (((uint32_t)axis_a & 0x7u) << 2) | (((uint32_t)axis_b & 0x7u) << 5) |
           (((uint32_t)vertex & 0xFu) << 8);
}

// Sutherland-Hodgman clip of a convex polygon against one plane
// (PolygonFaceClip, collision.cpp:81-105).
AVBD_HD int polygon_face_clip(const V3* in, int num_in, V3 pn, float po, V3* out) {
    if (num_in < 1) return 0;
    int k = 0;
    for (int i = 0; i < num_in; i++) {
        int j = (i + 1) % num_in;
        float di = XSUB(xdot(pn, in[i]), po);
        float dj = XSUB(xdot(pn, in[j]), po);
        if (di <= 0.f) out[k++] = in[i];
        if (k >= 8) return k;
        if ((di > 0.f) != (dj > 0.f)) {
            float t = XDIV(di, XSUB(di, dj));
            out[k++] = xadd(in[i], xmul(xsub(in[j], in[i]), t));
            if (k >= 8) return k;
        }
    }
    return k;
}

// FaceFaceContacts (collision.cpp:108-183). "A" is the reference box here.
AVBD_HD void face_face_contacts(V3 posA, const M3& rotA, V3 posB, const M3& rotB, V3 refHalfs, V3 incHalfs,
                                int refAxis, float refSign, V3 normal, int axisType, int axisA, int axisB,
                                Collision& out) {
    const V3 refC = posA, incC = posB;
    V3 refN = xmul(rotA.c[refAxis], refSign);
    float refOff = XADD(xdot(refN, refC), comp(refHalfs, refAxis));

    // FindIncidentFace (collision.cpp:65-77)
    float minDot = 3.402823466e+38f;
    int incAxis = 0;
    float incSign = 0.f;
    for (int a = 0; a < 3; a++) {
        float d = xdot(rotB.c[a], refN);
        if (d < minDot) { minDot = d; incAxis = a; incSign = 1.f; }
        if (-d < minDot) { minDot = -d; incAxis = a; incSign = -1.f; }
    }
    // GetBoxVerticesWorld (collision.cpp:36-59)
    V3 buf1[8], buf2[8];
    {
        int u = (incAxis + 1) % 3, v = (incAxis + 2) % 3;
        V3 fc = xadd(incC, xmul(rotB.c[incAxis], XMUL(incSign, comp(incHalfs, incAxis))));
        V3 uv = xmul(rotB.c[u], comp(incHalfs, u));
        V3 vv = xmul(rotB.c[v], comp(incHalfs, v));
        if (incSign > 0) {
            buf1[0] = xadd(xadd(fc, uv), vv);
            buf1[1] = xsub(xadd(fc, uv), vv);
            buf1[2] = xsub(xsub(fc, uv), vv);
            buf1[3] = xadd(xsub(fc, uv), vv);
        } else {
            buf1[0] = xsub(xsub(fc, uv), vv);
            buf1[1] = xadd(xsub(fc, uv), vv);
            buf1[2] = xadd(xadd(fc, uv), vv);
            buf1[3] = xsub(xadd(fc, uv), vv);
        }
    }
    int u = (refAxis + 1) % 3, v = (refAxis + 2) % 3;
    V3 pn[4];
    float po[4];
    pn[0] = rotA.c[u];
    po[0] = XADD(xdot(rotA.c[u], refC), comp(refHalfs, u));
    pn[1] = v3(-rotA.c[u].x, -rotA.c[u].y, -rotA.c[u].z);
    po[1] = XADD(-xdot(rotA.c[u], refC), comp(refHalfs, u));
    pn[2] = rotA.c[v];
    po[2] = XADD(xdot(rotA.c[v], refC), comp(refHalfs, v));
    pn[3] = v3(-rotA.c[v].x, -rotA.c[v].y, -rotA.c[v].z);
    po[3] = XADD(-xdot(rotA.c[v], refC), comp(refHalfs, v));

    int n = 4;
    n = polygon_face_clip(buf1, n, pn[0], po[0], buf2);
    if (n < 1) return;
    n = polygon_face_clip(buf2, n, pn[1], po[1], buf1);
    if (n < 1) return;
    n = polygon_face_clip(buf1, n, pn[2], po[2], buf2);
    if (n < 1) return;
    n = polygon_face_clip(buf2, n, pn[3], po[3], buf1);
    if (n < 1) return;

    for (int i = 0; i < n; i++) {
        float sep = XSUB(xdot(refN, buf1[i]), refOff);
        if (sep <= 0.f) {
            Contact& c = out.c[out.n];
            V3 proj = xsub(buf1[i], xmul(refN, sep));
            c.position = proj;
            c.normal = normal;
            c.penetration = -sep;
            c.rA = xmattvec(rotA, xsub(proj, posA));
            c.rB = xmattvec(rotB, xsub(buf1[i], posB));
            c.id = create_id(axisType, axisA, axisB, i);
            out.n++;
            if (out.n >= 8) return;
        }
    }
}

// ClosestPointTwoLineSegments (collision.cpp:186-213)
AVBD_HD void closest_point_segments(V3 p1, V3 d1, V3 p2, V3 d2, float& s, float& t) {
    V3 r = xsub(p1, p2);
    float a = xdot(d1, d1);
    float b = xdot(d1, d2);
    float c = xdot(d2, d2);
    float d = xdot(d1, r);
    float e = xdot(d2, r);
    float denom = XSUB(XMUL(a, c), XMUL(b, b));
    if (denom < 1e-6f) {
        s = 0.0f;
        t = (b > c ? XDIV(d, b) : XDIV(e, c));
    } else {
        s = XDIV(XSUB(XMUL(b, e), XMUL(c, d)), denom);
        t = XDIV(XSUB(XMUL(a, e), XMUL(b, d)), denom);
    }
    s = clampf(s, 0.0f, 1.0f);
    t = clampf(t, 0.0f, 1.0f);
}

// LineLineContacts (collision.cpp:216-267)
AVBD_HD void line_line_contacts(V3 posA, V3 scaleA, const M3& rotA, V3 posB, V3 scaleB, const M3& rotB, V3 normal,
                                int axisA, int axisB, Collision& out) {
    V3 d = xsub(posB, posA);
    int uA = (axisA + 1) % 3, vA = (axisA + 2) % 3;
    float sUA = (xdot(rotA.c[uA], d) > 0.f) ? 1.0f : -1.0f;
    float sVA = (xdot(rotA.c[vA], d) > 0.f) ? 1.0f : -1.0f;
    V3 midA = xadd(xadd(posA, xmul(rotA.c[uA], XMUL(XMUL(sUA, comp(scaleA, uA)), 0.5f))),
                   xmul(rotA.c[vA], XMUL(XMUL(sVA, comp(scaleA, vA)), 0.5f)));
    V3 dirA = rotA.c[axisA];
    float lenA = comp(scaleA, axisA);
    V3 startA = xsub(midA, xmul(dirA, XMUL(lenA, 0.5f)));

    int uB = (axisB + 1) % 3, vB = (axisB + 2) % 3;
    V3 nd = v3(-d.x, -d.y, -d.z);
    float sUB = (xdot(rotB.c[uB], nd) > 0.f) ? 1.0f : -1.0f;
    float sVB = (xdot(rotB.c[vB], nd) > 0.f) ? 1.0f : -1.0f;
    V3 midB = xadd(xadd(posB, xmul(rotB.c[uB], XMUL(XMUL(sUB, comp(scaleB, uB)), 0.5f))),
                   xmul(rotB.c[vB], XMUL(XMUL(sVB, comp(scaleB, vB)), 0.5f)));
    V3 dirB = rotB.c[axisB];
    float lenB = comp(scaleB, axisB);
    V3 startB = xsub(midB, xmul(dirB, XMUL(lenB, 0.5f)));

    float s, t;
    closest_point_segments(startA, xmul(dirA, lenA), startB, xmul(dirB, lenB), s, t);
    V3 cA = xadd(startA, xmul(dirA, XMUL(s, lenA)));
    V3 cB = xadd(startB, xmul(dirB, XMUL(t, lenB)));

    Contact& c = out.c[0];
    V3 sum = xadd(cA, cB);
    c.position = v3(XMUL(0.5f, sum.x), XMUL(0.5f, sum.y), XMUL(0.5f, sum.z));
    c.normal = normal;
    c.penetration = xdot(xsub(cB, cA), normal);
    if (c.penetration < 0.f) c.penetration = -c.penetration;
    c.rA = xmattvec(rotA, xsub(cA, posA));
    c.rB = xmattvec(rotB, xsub(cB, posB));
    c.id = create_id(2, axisA, axisB, 0);
    out.n = 1;
}

// The separating-axis part of CollisionSpace::CollisionBoxBox
// (collision.cpp:271-373): the axis of least penetration (0-2 faces of A, 3-5
// faces of B, 6-14 edge pairs) and its sign, or -1 if an axis separates the
// boxes (no contacts).  scale = full box edges.
AVBD_HD int box_box_sat(const M3& rotA, V3 scaleA, const M3& rotB, V3 scaleB, V3 d, float& bestSign) {
    float C[3][3], AR[3][3], T[3];
    for (int i = 0; i < 3; i++) {
        T[i] = xdot(rotA.c[i], d);
        for (int j = 0; j < 3; j++) {
            C[i][j] = xdot(rotA.c[i], rotB.c[j]);
            AR[i][j] = XADD(fabsf(C[i][j]), 1e-6f);
        }
    }
    const V3 hA = xmul(scaleA, 0.5f), hB = xmul(scaleB, 0.5f);
    float best = 3.402823466e+38f;
    int bestAxis = -1;
    bestSign = 1.f;
#define AVBD_TEST_AXIS(idx, pen, sgn)              \
    {                                              \
        if ((pen) < 0.f) return -1;                \
        if ((pen) < best) {                        \
            best = (pen); bestAxis = (idx); bestSign = (sgn); \
        }                                          \
    }
    for (int i = 0; i < 3; i++) {
        float rA = XMUL(comp(scaleA, i), 0.5f);
        float rB = XADD(XADD(XMUL(AR[i][0], hB.x), XMUL(AR[i][1], hB.y)), XMUL(AR[i][2], hB.z));
        float dist = fabsf(T[i]);
        float pen = XSUB(XADD(rA, rB), dist);
        float s = (T[i] > 0.f) ? 1.0f : -1.0f;
        AVBD_TEST_AXIS(i, pen, s);
    }
    for (int i = 0; i < 3; i++) {
        float rA = XADD(XADD(XMUL(AR[0][i], hA.x), XMUL(AR[1][i], hA.y)), XMUL(AR[2][i], hA.z));
        float rB = XMUL(comp(scaleB, i), 0.5f);
        float cT = XADD(XADD(XMUL(C[0][i], T[0]), XMUL(C[1][i], T[1])), XMUL(C[2][i], T[2]));
        float dist = fabsf(cT);
        float pen = XSUB(XADD(rA, rB), dist);
        float s = (cT > 0.f) ? 1.0f : -1.0f;
        AVBD_TEST_AXIS(3 + i, pen, s);
    }
    const float bestFace = best;
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            float cl = XSUB(1.f, XMUL(C[i][j], C[i][j]));
            if (cl < 1e-6f) continue;
            float invLen = XDIV(1.f, XSQRT(cl));
            int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
            int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            float rA = XADD(XMUL(XMUL(comp(scaleA, i1), 0.5f), AR[i2][j]), XMUL(XMUL(comp(scaleA, i2), 0.5f), AR[i1][j]));
            float rB = XADD(XMUL(XMUL(comp(scaleB, j1), 0.5f), AR[i][j2]), XMUL(XMUL(comp(scaleB, j2), 0.5f), AR[i][j1]));
            float raw = XSUB(XMUL(T[i2], C[i1][j]), XMUL(T[i1], C[i2][j]));
            float dist = fabsf(raw);
            float pen = XMUL(XSUB(XADD(rA, rB), dist), invLen);
            float s = (raw > 0.f) ? 1.0f : -1.0f;
            if (pen < XADD(XMUL(0.95f, bestFace), 0.005f)) AVBD_TEST_AXIS(6 + i * 3 + j, pen, s);
        }
    }
#undef AVBD_TEST_AXIS
    return bestAxis;
}

// CollisionSpace::CollisionBoxBox (collision.cpp:271-447).  scale = full box edges.
AVBD_HD void collide_box_box(V3 posA, Q4 qA, V3 scaleA, V3 posB, Q4 qB, V3 scaleB, Collision& out) {
    out.n = 0;
    const M3 rotA = xrotmat(qA);
    const M3 rotB = xrotmat(qB);
    const V3 d = xsub(posB, posA);
    float bestSign;
    const int bestAxis = box_box_sat(rotA, scaleA, rotB, scaleB, d, bestSign);
    if (bestAxis < 0) return;
    const V3 hA = xmul(scaleA, 0.5f), hB = xmul(scaleB, 0.5f);

    V3 normal;
    if (bestAxis < 3) {
        normal = xmul(rotA.c[bestAxis], bestSign);
    } else if (bestAxis < 6) {
        normal = xmul(rotB.c[bestAxis - 3], bestSign);
    } else {
        int i = (bestAxis - 6) / 3, j = (bestAxis - 6) % 3;
        normal = xcross(rotA.c[i], rotB.c[j]);
        float len = xnorm(normal);
        if (len < 1e-6f) return;
        normal = xdiv(normal, len);
        if (xdot(normal, d) < 0.f) normal = v3(-normal.x, -normal.y, -normal.z);
    }

    if (bestAxis < 3) {
        face_face_contacts(posA, rotA, posB, rotB, hA, hB, bestAxis, bestSign, normal, 0, bestAxis, 0, out);
    } else if (bestAxis < 6) {
        face_face_contacts(posB, rotB, posA, rotA, hB, hA, bestAxis - 3, -bestSign, normal, 1, 0, bestAxis - 3, out);
        for (int i = 0; i < out.n; i++) {
            V3 t = out.c[i].rA;
            out.c[i].rA = out.c[i].rB;
            out.c[i].rB = t;
        }
    } else {
        line_line_contacts(posA, scaleA, rotA, posB, scaleB, rotB, normal, (bestAxis - 6) / 3, (bestAxis - 6) % 3, out);
    }
}

}  // namespace avbd
