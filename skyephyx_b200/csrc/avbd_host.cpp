// Host staging of scenes (see avbd_host.h).  Compiled with -ffp-contract=off.
#include "avbd_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>

namespace avbd {

namespace {

float4 mk4(float x, float y, float z, float w = 0.f) {
    float4 r;
    r.x = x; r.y = y; r.z = z; r.w = w;
    return r;
}

// Quaternion (w, x, y, z) times vector, the shim/Eigen formula:
// t = 2 (u x v); v + w t + u x t
void qrot(const float* q, const float* v, float* out) {
    const float ux = q[1], uy = q[2], uz = q[3], w = q[0];
    float tx = uy * v[2] - uz * v[1];
    float ty = uz * v[0] - ux * v[2];
    float tz = ux * v[1] - uy * v[0];
    tx = tx + tx; ty = ty + ty; tz = tz + tz;
    const float cx = uy * tz - uz * ty;
    const float cy = uz * tx - ux * tz;
    const float cz = ux * ty - uy * tx;
    out[0] = (v[0] + w * tx) + cx;
    out[1] = (v[1] + w * ty) + cy;
    out[2] = (v[2] + w * tz) + cz;
}

// Transform::TransformPoint (geometry.hpp:70-73) on staged body state.
void transform_point_host(const HostScene& s, int b, const float* p, float* out) {
    const float4 sc = s.scale[b];
    const float sp[3] = {sc.x * p[0], sc.y * p[1], sc.z * p[2]};
    const float4 r = s.rot[b];
    const float q[4] = {r.w, r.x, r.y, r.z};
    float t[3];
    qrot(q, sp, t);
    out[0] = t[0] + s.pos[b].x;
    out[1] = t[1] + s.pos[b].y;
    out[2] = t[2] + s.pos[b].z;
}

// Hamilton product a * b, both (w, x, y, z).
void qmul_host(const float* a, const float* b, float* o) {
    o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
    o[2] = a[0] * b[2] + a[2] * b[0] + a[3] * b[1] - a[1] * b[3];
    o[3] = a[0] * b[3] + a[3] * b[0] + a[1] * b[2] - a[2] * b[1];
}

}  // namespace

int HostScene::add_body(int model, float density, float fr, const float* p, const float* s, const float* v,
                        const float* q, const float* w, bool is_static) {
    const float sx = s[0], sy = s[1], sz = s[2];
    // detectionRadius = scale.norm() * 0.5f (solver.cpp:65)
    const float radius = std::sqrt((sx * sx + sy * sy) + sz * sz) * 0.5f;
    float mass = 0.f, Ix = 0.f, Iy = 0.f, Iz = 0.f;
    if (!is_static) {
        const float sx2 = sx * sx, sy2 = sy * sy, sz2 = sz * sz;
        const float r = sx * 0.5f;
        if (model == 1) {   // ModelType_Sphere: double arithmetic from M_PI onwards
            mass = (float)((double)(density * (4.0f / 3.0f)) * M_PI * r * r * r);
            const float i = (2.0f / 5.0f) * mass * r * r;
            Ix = Iy = Iz = i;
        } else {
            mass = density * sx * sy * sz;
            if (model == 0) {
                const float m12 = mass / 12.0f;
                Ix = m12 * (sy2 + sz2);
                Iy = m12 * (sx2 + sz2);
                Iz = m12 * (sx2 + sy2);
            }
        }
    }
    pos.push_back(mk4(p[0], p[1], p[2]));
    rot.push_back(mk4(q[1], q[2], q[3], q[0]));
    scale.push_back(mk4(sx, sy, sz, radius));
    vel.push_back(mk4(v[0], v[1], v[2]));
    omega.push_back(mk4(w[0], w[1], w[2]));
    massI.push_back(mk4(mass, Ix, Iy, Iz));
    flags.push_back((is_static ? kBodyStatic : 0) | ((model & 15) << kBodyModelShift));
    friction.push_back(fr);
    color.push_back(mk4(1.f, 1.f, 1.f, 1.f));
    return (int)pos.size() - 1;
}

int HostScene::add_particle(float mass, float fr, const float* p, const float* v, bool is_static) {
    const float s[3] = {0.1f, 0.1f, 0.1f};
    const float q[4] = {1.f, 0.f, 0.f, 0.f};
    const float w[3] = {0.f, 0.f, 0.f};
    const float density = mass / (s[0] * s[1] * s[2]);
    const int b = add_body(0, density, fr, p, s, v, q, w, is_static);
    massI[b].y = massI[b].z = massI[b].w = 0.f;   // inertia zeroed (solver.cpp:124-126)
    omega[b] = mk4(0.f, 0.f, 0.f);
    flags[b] |= kBodyParticle;
    return b;
}

int HostScene::set_static(int body, bool st) {
    if (body < 0 || body >= nbody()) return -1;
    flags[body] = st ? (flags[body] | kBodyStatic) : (flags[body] & ~kBodyStatic);
    return 0;
}

int HostScene::add_spring(int a, const float* rA, int b, const float* rB, float k, float rest, bool rope,
                          float fracture) {
    if (b < 0 || b >= nbody() || a >= nbody() || a < -1 || a == b) return -1;
    float L = rest;
    if (L < 0.0f) {   // spring.cpp:30-35
        float wa[3], wb[3];
        if (a >= 0) transform_point_host(*this, a, rA, wa);
        else { wa[0] = rA[0]; wa[1] = rA[1]; wa[2] = rA[2]; }
        transform_point_host(*this, b, rB, wb);
        const float dx = wb[0] - wa[0], dy = wb[1] - wa[1], dz = wb[2] - wa[2];
        L = std::sqrt((dx * dx + dy * dy) + dz * dz);
    }
    ftype.push_back(kForceSpring | (rope ? kForceRope : 0));
    fbody.push_back(make_int2(a, b));
    frA.push_back(mk4(rA[0], rA[1], rA[2]));
    frB.push_back(mk4(rB[0], rB[1], rB[2]));
    fq.push_back(mk4(0.f, 0.f, 0.f, 1.f));
    fparam.push_back(mk4(L, 0.f, 0.f));
    for (int i = 0; i < 6; ++i) {
        fk.push_back(i == 0 ? k : INFINITY);
        ffrac.push_back(i == 0 ? fracture : INFINITY);
        ffmin.push_back(i == 0 ? (rope ? 0.0f : -INFINITY) : -INFINITY);
        ffmax.push_back(INFINITY);
    }
    return nforce() - 1;
}

int HostScene::add_joint(int a, const float* rA, int b, const float* rB, const float* k, const float* fracture) {
    if (b < 0 || b >= nbody() || a >= nbody() || a < -1 || a == b) return -1;
    float qa[4] = {1.f, 0.f, 0.f, 0.f};
    if (a >= 0) { qa[0] = rot[a].w; qa[1] = rot[a].x; qa[2] = rot[a].y; qa[3] = rot[a].z; }
    const float qb[4] = {rot[b].w, rot[b].x, rot[b].y, rot[b].z};
    const float qac[4] = {qa[0], -qa[1], -qa[2], -qa[3]};
    float rest[4];
    qmul_host(qac, qb, rest);   // restRotation = qA^* qB (joint.cpp:54-57)
    float sa[3] = {0.f, 0.f, 0.f};
    if (a >= 0) { sa[0] = scale[a].x; sa[1] = scale[a].y; sa[2] = scale[a].z; }
    const float t0 = sa[0] + scale[b].x, t1 = sa[1] + scale[b].y, t2 = sa[2] + scale[b].z;
    float arm = (t0 * t0 + t1 * t1) + t2 * t2;   // (scaleA + scaleB).squaredNorm() (joint.cpp:62)
    if (arm < 1e-6f) arm = 1.0f;
    ftype.push_back(kForceJoint);
    fbody.push_back(make_int2(a, b));
    frA.push_back(mk4(rA[0], rA[1], rA[2]));
    frB.push_back(mk4(rB[0], rB[1], rB[2]));
    fq.push_back(mk4(rest[1], rest[2], rest[3], rest[0]));
    fparam.push_back(mk4(arm, 0.f, 0.f));
    for (int i = 0; i < 6; ++i) {
        fk.push_back(k[i]);
        ffrac.push_back(fracture[i]);
        ffmin.push_back(-fracture[i]);
        ffmax.push_back(fracture[i]);
    }
    return nforce() - 1;
}

int HostScene::add_nh_tet(const int* v, float E, float nu) {
    for (int i = 0; i < 4; ++i) if (v[i] < 0 || v[i] >= nbody()) return -1;
    const float mu = E / (2.f * (1.f + nu));
    const float lam = E * nu / ((1.f + nu) * (1.f - 2.f * nu));
    const float4 p0 = pos[v[0]], p1 = pos[v[1]], p2 = pos[v[2]], p3 = pos[v[3]];
    // Dm columns (neohookeanfem.cpp:18-22), m(i, j) = column j component i
    const float m[3][3] = {{p1.x - p0.x, p2.x - p0.x, p3.x - p0.x},
                           {p1.y - p0.y, p2.y - p0.y, p3.y - p0.y},
                           {p1.z - p0.z, p2.z - p0.z, p3.z - p0.z}};
    // 3x3 inverse by the adjugate, as the oracle's Eigen shim computes it
    const float c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    const float c10 = m[0][2] * m[2][1] - m[0][1] * m[2][2];
    const float c20 = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    const float det = m[0][0] * c00 + m[1][0] * c10 + m[2][0] * c20;
    const float inv = 1.f / det;
    float r[3][3];
    r[0][0] = c00 * inv; r[0][1] = c10 * inv; r[0][2] = c20 * inv;
    r[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * inv;
    r[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * inv;
    r[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * inv;
    r[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * inv;
    r[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * inv;
    r[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * inv;
    // Dm.determinant() (first-column expansion, as the shim)
    const float dDm = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                      m[1][0] * (m[0][1] * m[2][2] - m[0][2] * m[2][1]) +
                      m[2][0] * (m[0][1] * m[1][2] - m[0][2] * m[1][1]);
    const float restVolume = std::fabs(dDm) / 6.f;
    int4 idx; idx.x = v[0]; idx.y = v[1]; idx.z = v[2]; idx.w = v[3];
    tidx.push_back(idx);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) tDmInv.push_back(r[i][j]);   // column-major
    // the shape gradients (neohookeanfem.cpp:31-36) are rebuilt from DmInv on the device
    tparam.push_back(mk4(restVolume, mu, lam, 0.f));
    tkind.push_back(kTetNeoHookean);
    return ntet() - 1;
}

// St. Venant-Kirchhoff tet: the same rest-shape data as the Neo-Hookean tet
// (Dm^-1, rest volume, shape gradients, Lame parameters); only the energy differs.
int HostScene::add_stvk_tet(const int* v, float E, float nu) {
    const int t = add_nh_tet(v, E, nu);
    if (t >= 0) tkind.back() = kTetStvk;
    return t;
}

int HostScene::add_stvk_tri(const int* v, float E, float nu) {
    for (int i = 0; i < 3; ++i) if (v[i] < 0 || v[i] >= nbody()) return -1;
    const float mu = E / (2.f * (1.f + nu));
    const float lam = E * nu / ((1.f + nu) * (1.f - 2.f * nu));
    const float4 p0 = pos[v[0]], p1 = pos[v[1]], p2 = pos[v[2]];
    const float e0[3] = {p1.x - p0.x, p1.y - p0.y, p1.z - p0.z};
    const float e1[3] = {p2.x - p0.x, p2.y - p0.y, p2.z - p0.z};
    const float x1 = std::sqrt((e0[0] * e0[0] + e0[1] * e0[1]) + e0[2] * e0[2]);
    const float x2 = ((e1[0] * e0[0] + e1[1] * e0[1]) + e1[2] * e0[2]) / x1;
    const float y2 = std::sqrt(std::max(0.f, ((e1[0] * e1[0] + e1[1] * e1[1]) + e1[2] * e1[2]) - x2 * x2));
    // Dm2D = [[x1, x2], [0, y2]]; 2x2 inverse as the shim computes it
    const float det = x1 * y2 - x2 * 0.f;
    const float inv = 1.f / det;
    const float i00 = y2 * inv, i01 = -x2 * inv, i10 = -0.f * inv, i11 = x1 * inv;
    const float restArea = 0.5f * x1 * y2;
    int4 idx; idx.x = v[0]; idx.y = v[1]; idx.z = v[2]; idx.w = -1;
    ridx.push_back(idx);
    rDmInv.push_back(mk4(i00, i10, i01, i11));   // column-major
    // gradN1 = row 0 of DmInv, gradN2 = row 1, gradN0 = -g1 - g2
    const float g1x = i00, g1y = i01, g2x = i10, g2y = i11;
    rgradN.push_back((-g1x) - g2x);
    rgradN.push_back((-g1y) - g2y);
    rgradN.push_back(g1x);
    rgradN.push_back(g1y);
    rgradN.push_back(g2x);
    rgradN.push_back(g2y);
    rparam.push_back(mk4(restArea, mu, lam, 0.f));
    return ntri() - 1;
}

int HostScene::make_tet_volume(float ox, float oy, float oz, int nx, int ny, int nz, float cell, float E, float nu,
                               float pm, float fr, bool pin_min_x, int model) {
    if (nx < 2 || ny < 2 || nz < 2) return -1;
    const int first = nbody();
    std::vector<int> parts((size_t)nx * ny * nz);
    auto idx = [&](int i, int j, int k) { return i + j * nx + k * nx * ny; };
    const float zero[3] = {0.f, 0.f, 0.f};
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                const float p[3] = {ox + i * cell, oy + j * cell, oz + k * cell};
                parts[idx(i, j, k)] = add_particle(pm, fr, p, zero, pin_min_x && (i == 0));
            }
    for (int ci = 0; ci < nx - 1; ci++)
        for (int cj = 0; cj < ny - 1; cj++)
            for (int ck = 0; ck < nz - 1; ck++) {
                const int v[8] = {parts[idx(ci, cj, ck)],         parts[idx(ci + 1, cj, ck)],
                                  parts[idx(ci, cj + 1, ck)],     parts[idx(ci + 1, cj + 1, ck)],
                                  parts[idx(ci, cj, ck + 1)],     parts[idx(ci + 1, cj, ck + 1)],
                                  parts[idx(ci, cj + 1, ck + 1)], parts[idx(ci + 1, cj + 1, ck + 1)]};
                const int t0[4] = {v[0], v[1], v[2], v[4]};
                const int t1[4] = {v[3], v[2], v[1], v[7]};
                const int t2[4] = {v[5], v[1], v[4], v[7]};
                const int t3[4] = {v[6], v[4], v[2], v[7]};
                const int t4[4] = {v[1], v[2], v[4], v[7]};
                for (const int* t : {t0, t1, t2, t3, t4}) {
                    if (model == kTetStvk) add_stvk_tet(t, E, nu);
                    else add_nh_tet(t, E, nu);
                }
            }
    return first;
}

int HostScene::make_tet_sphere(float cx, float cy, float cz, float radius, float res, float E, float nu,
                               float pm, float fr) {
    // GeometryHelpers::makeTetSphere (geometry.cpp:106-232): a centre
    // particle, N concentric shells of 6N x 3N ring particles plus two poles,
    // the innermost shell fanned to the centre, each outer shell joined to the
    // one inside by triangular prisms of 3 tets; every tet's last two
    // vertices swap when its rest volume would be negative.  Positions are
    // formed with the reference's float operations, in its order.
    const int N = std::max(1, (int)std::roundf(res));
    const int nLon = 6 * N, nLat = 3 * N, nShells = N;
    const int vps = 2 + nLat * nLon;
    std::vector<int> pts(1 + (size_t)nShells * vps, -1);
    auto sBase = [&](int sh) { return 1 + sh * vps; };
    auto sSouth = [&](int sh) { return sBase(sh); };
    auto sNorth = [&](int sh) { return sBase(sh) + 1; };
    auto sV = [&](int sh, int j, int i) { return sBase(sh) + 2 + j * nLon + ((i % nLon + nLon) % nLon); };
    const float zero[3] = {0.f, 0.f, 0.f};
    auto makeP = [&](float x, float y, float z) {
        const float p[3] = {x, y, z};
        return add_particle(pm, fr, p, zero, false);
    };
    const int first = nbody();
    pts[0] = makeP(cx, cy, cz);
    const float pi = (float)M_PI;
    for (int sh = 0; sh < nShells; sh++) {
        const float r = radius * (sh + 1) / (float)nShells;
        pts[sSouth(sh)] = makeP(cx, cy - r, cz);
        pts[sNorth(sh)] = makeP(cx, cy + r, cz);
        for (int j = 0; j < nLat; j++) {
            const float theta = pi * (j + 1) / (float)(nLat + 1);
            const float sinT = std::sin(theta), cosT = std::cos(theta);
            for (int i = 0; i < nLon; i++) {
                const float phi = 2.f * pi * i / (float)nLon;
                pts[sV(sh, j, i)] = makeP(cx + r * sinT * std::cos(phi), cy + r * cosT, cz + r * sinT * std::sin(phi));
            }
        }
    }
    auto addTet = [&](int a, int b, int c, int d) {
        const float4 pa = pos[a], pb = pos[b], pc = pos[c], pd = pos[d];
        // columns b - a, c - a, d - a; determinant by the first column's cofactors
        const float m00 = pb.x - pa.x, m10 = pb.y - pa.y, m20 = pb.z - pa.z;
        const float m01 = pc.x - pa.x, m11 = pc.y - pa.y, m21 = pc.z - pa.z;
        const float m02 = pd.x - pa.x, m12 = pd.y - pa.y, m22 = pd.z - pa.z;
        const float det = m00 * (m11 * m22 - m12 * m21) - m10 * (m01 * m22 - m02 * m21) +
                          m20 * (m01 * m12 - m02 * m11);
        if (det < 0.f) std::swap(c, d);
        const int v[4] = {a, b, c, d};
        add_nh_tet(v, E, nu);
    };
    auto addPrism = [&](int P0, int P1, int P2, int Q0, int Q1, int Q2) {
        addTet(P0, P1, P2, Q2);
        addTet(P0, Q1, P1, Q2);
        addTet(P0, Q0, Q1, Q2);
    };
    for (int sh = 0; sh < nShells; sh++) {
        const bool fan = sh == 0;
        const int sIn = sh - 1;
        for (int i = 0; i < nLon; i++) {
            const int i1 = (i + 1) % nLon;
            if (fan) addTet(pts[0], pts[sNorth(sh)], pts[sV(sh, 0, i)], pts[sV(sh, 0, i1)]);
            else addPrism(pts[sNorth(sIn)], pts[sV(sIn, 0, i)], pts[sV(sIn, 0, i1)], pts[sNorth(sh)],
                          pts[sV(sh, 0, i)], pts[sV(sh, 0, i1)]);
            const int jS = nLat - 1;
            if (fan) addTet(pts[0], pts[sSouth(sh)], pts[sV(sh, jS, i)], pts[sV(sh, jS, i1)]);
            else addPrism(pts[sSouth(sIn)], pts[sV(sIn, jS, i)], pts[sV(sIn, jS, i1)], pts[sSouth(sh)],
                          pts[sV(sh, jS, i)], pts[sV(sh, jS, i1)]);
        }
        for (int j = 0; j < nLat - 1; j++)
            for (int i = 0; i < nLon; i++) {
                const int i1 = (i + 1) % nLon;
                if (fan) {
                    addTet(pts[0], pts[sV(sh, j, i)], pts[sV(sh, j, i1)], pts[sV(sh, j + 1, i1)]);
                    addTet(pts[0], pts[sV(sh, j, i)], pts[sV(sh, j + 1, i1)], pts[sV(sh, j + 1, i)]);
                } else {
                    addPrism(pts[sV(sIn, j, i)], pts[sV(sIn, j, i1)], pts[sV(sIn, j + 1, i1)], pts[sV(sh, j, i)],
                             pts[sV(sh, j, i1)], pts[sV(sh, j + 1, i1)]);
                    addPrism(pts[sV(sIn, j, i)], pts[sV(sIn, j + 1, i1)], pts[sV(sIn, j + 1, i)], pts[sV(sh, j, i)],
                             pts[sV(sh, j + 1, i1)], pts[sV(sh, j + 1, i)]);
                }
            }
    }
    return first;
}

void HostScene::build_static_incidence(std::vector<int>& off, std::vector<int>& cnt, std::vector<int>& nf,
                                       std::vector<uint32_t>& ent, std::vector<int>& poff, std::vector<int>& pcnt,
                                       std::vector<int2>& partners, int body_base, int force_base, int tet_base,
                                       int tri_base) const {
    // counting sort by body: per body its forces in force order, then its
    // tets in tet order, then its triangles; partners in force order
    const int n = nbody();
    nf.assign(n, 0);
    pcnt.assign(n, 0);
    std::vector<int> ne(n, 0);
    for (int f = 0; f < nforce(); ++f) {
        const int2 ab = fbody[f];
        if (ab.x >= 0) {
            ++nf[ab.x];
            ++pcnt[ab.x];
            ++pcnt[ab.y];
        }
        ++nf[ab.y];
    }
    for (int t = 0; t < ntet(); ++t) {
        ++ne[tidx[t].x]; ++ne[tidx[t].y]; ++ne[tidx[t].z]; ++ne[tidx[t].w];
    }
    for (int t = 0; t < ntri(); ++t) {
        ++ne[ridx[t].x]; ++ne[ridx[t].y]; ++ne[ridx[t].z];
    }
    off.resize(n);
    cnt.resize(n);
    poff.resize(n);
    int acc = 0, pacc = 0;
    for (int b = 0; b < n; ++b) {
        off[b] = acc;
        cnt[b] = nf[b] + ne[b];
        acc += cnt[b];
        poff[b] = pacc;
        pacc += pcnt[b];
    }
    ent.resize(acc);
    partners.resize(pacc);
    std::vector<int> fcur(n, 0), ecur(n, 0), pcur(n, 0);
    for (int f = 0; f < nforce(); ++f) {
        const int2 ab = fbody[f];
        if (ab.x >= 0) {
            ent[off[ab.x] + fcur[ab.x]++] = ent_make(kEntForce, 0, (uint32_t)(force_base + f));
            partners[poff[ab.x] + pcur[ab.x]++] = make_int2(body_base + ab.y, force_base + f);
            partners[poff[ab.y] + pcur[ab.y]++] = make_int2(body_base + ab.x, force_base + f);
        }
        ent[off[ab.y] + fcur[ab.y]++] = ent_make(kEntForce, 1, (uint32_t)(force_base + f));
    }
    for (int t = 0; t < ntet(); ++t) {
        const int v[4] = {tidx[t].x, tidx[t].y, tidx[t].z, tidx[t].w};
        for (int r = 0; r < 4; ++r)
            ent[off[v[r]] + nf[v[r]] + ecur[v[r]]++] = ent_make(kEntTet, (uint32_t)r, (uint32_t)(tet_base + t));
    }
    for (int t = 0; t < ntri(); ++t) {
        const int v[3] = {ridx[t].x, ridx[t].y, ridx[t].z};
        for (int r = 0; r < 3; ++r)
            ent[off[v[r]] + nf[v[r]] + ecur[v[r]]++] = ent_make(kEntTri, (uint32_t)r, (uint32_t)(tri_base + t));
    }
}

}  // namespace avbd
