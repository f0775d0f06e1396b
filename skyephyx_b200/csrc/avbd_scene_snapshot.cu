// Snapshot and restore of one scene inside a batch (avbd_batch_scene_snapshot
// / avbd_batch_scene_restore in include/avbd.h).  No counterpart in the
// reference, whose state lives in Mesh/Force objects (solver.hpp:28-64).
//
// A snapshot holds every device value of the scene: its slices of the body,
// force, tet and triangle pools, both manifold tables and contact pools, its
// incidence and static-incidence ranges, its colour starts, descriptor and
// counters.  A restore places the scene anew (first fit, so usually at other
// offsets), copies the slices in and shifts every stored index (body, force,
// tet, triangle, manifold slot, contact slot and incidence positions) by the
// distance the scene moved.  The restored scene then takes the same steps,
// bit for bit, as it would have without the interruption: serving
// pre-emption (retire a scene, admit it again later) and deterministic replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <initializer_list>
#include <vector>

#include "avbd_pools.h"

using namespace avbd;
using namespace avbd::host;

namespace {

enum Unit { kUBody, kUForce, kUTet, kUTri, kUCand, kUK, kUInc, kUSinc, kUSp, kUnits };

// One device array of the pools: base pointer, bytes per element, elements
// per unit (6 rows per force, 9 Dm^-1 entries per tet, ...), the unit.
struct Slice {
    void* base;
    int elem;
    int per;
    Unit unit;
};

std::vector<Slice> scene_slices(const Pools& P) {
    const World& W = P.W;
    std::vector<Slice> s;
    auto add = [&](const void* p, int elem, int per, Unit u) { s.push_back({const_cast<void*>(p), elem, per, u}); };
    for (const float4* p : {W.pos, W.rot, W.scale, W.lpos, W.lrot, W.ipos, W.irot, W.vel, W.omega, W.pvel, W.dlin,
                            W.dang, W.massI, W.Mw0, W.Mw1, W.color})
        add(p, 16, 1, kUBody);
    for (const int* p : std::initializer_list<const int*>{W.flags, W.colour, W.local, W.reset_flag, W.sinc_off, W.sinc_n, W.sinc_nf, W.spartner_off,
                         W.spartner_n, W.inc_off, W.inc_cnt, W.cntB, W.bcur, W.cand_cnt, W.cand_off, W.col_list,
                         W.col_tinc})
        add(p, 4, 1, kUBody);
    add(W.friction, 4, 1, kUBody);
    add(W.ftype, 4, 1, kUForce);
    add(W.fbody, 8, 1, kUForce);
    for (const float4* p : {W.frA, W.frB, W.fq, W.fparam, W.fC0p, W.fC0a}) add(p, 16, 1, kUForce);
    for (const float* p : {W.fk, W.ffrac, W.ffmin, W.ffmax, W.fpen, W.flam}) add(p, 4, 6, kUForce);
    add(W.tidx, 16, 1, kUTet);
    add(W.tDmInv, 4, 9, kUTet);
    add(W.tparam, 16, 1, kUTet);
    add(W.tkind, 4, 1, kUTet);
    add(W.trv, 16, 4, kUTet);
    for (const float4* p : {W.trm0, W.trm1, W.trm2}) add(p, 16, 4, kUTet);
    add(W.ridx, 16, 1, kUTri);
    add(W.rDmInv, 16, 1, kUTri);
    add(W.rgradN, 4, 6, kUTri);
    add(W.rparam, 16, 1, kUTri);
    for (int t = 0; t < 2; ++t) {
        add(W.cpair[t], 8, 1, kUCand);
        for (const int* p : {W.cn[t], W.kbase[t], W.cbirth[t], W.live[t]}) add(p, 4, 1, kUCand);
        add(W.cfric[t], 4, 1, kUCand);
        add(W.kid[t], 4, 1, kUK);
        for (const float4* p : {W.krA[t], W.krB[t], W.kn[t], W.kt1[t], W.kt2[t], W.krAw[t], W.krBw[t], W.kpen[t],
                                W.klam[t]})
            add(p, 16, 1, kUK);
    }
    add(W.inc, 4, 1, kUInc);
    add(W.sinc, 4, 1, kUSinc);
    add(W.spartner, 8, 1, kUSp);
    return s;
}

void region_units(const Region& r, int start[kUnits], int count[kUnits]) {
    const int st[kUnits] = {r.body0, r.force0, r.tet0, r.tri0, r.cand0, r.k0, r.inc0, r.sinc0, r.sp0};
    const int ct[kUnits] = {r.nbody, r.nforce, r.ntet, r.ntri, r.ncand, r.nk, r.ninc, r.nsinc, r.nsp};
    for (int u = 0; u < kUnits; ++u) { start[u] = st[u]; count[u] = ct[u]; }
}

constexpr uint32_t kSceneSnapMagic = 0x53435641u;   // "AVCS"

struct SceneSnapHeader {
    uint32_t magic;
    uint32_t nslices;
    Region src;            // where the scene lay when it was taken
    SceneDesc desc;
    SceneState state;
    int64_t dynamic;
    int64_t bytes;         // total, header included
};

int64_t scene_snapshot_bytes(const AvbdBatch* b, int slot) {
    int start[kUnits], count[kUnits];
    region_units(b->regions[slot], start, count);
    int64_t bytes = sizeof(SceneSnapHeader) + (int64_t)(kMaxColours + 1) * sizeof(int);
    for (const Slice& s : scene_slices(b->P)) bytes += (int64_t)count[s.unit] * s.per * s.elem;
    return bytes;
}

// Shifts every stored index of a scene that moved by the given unit deltas.
__global__ void k_relocate_scene(const __grid_constant__ World W, Region r, int db, int df, int dt, int dr, int dc,
                                 int dk, int di, int ds, int dp) {
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    for (int i = t0; i < r.nbody; i += stride) {
        const int b = r.body0 + i;
        W.inc_off[b] += di;
        const_cast<int*>(W.sinc_off)[b] += ds;
        const_cast<int*>(W.spartner_off)[b] += dp;
        W.col_list[b] += db;
    }
    for (int i = t0; i < r.nforce; i += stride) {
        int2 ab = W.fbody[r.force0 + i];
        if (ab.x >= 0) ab.x += db;
        ab.y += db;
        W.fbody[r.force0 + i] = ab;
    }
    for (int i = t0; i < r.ntet; i += stride) {
        int4 v = W.tidx[r.tet0 + i];
        v.x += db; v.y += db; v.z += db; v.w += db;
        W.tidx[r.tet0 + i] = v;
        for (int q = 0; q < 4; ++q) {
            int4 a = W.trv[4 * (size_t)(r.tet0 + i) + q];
            const uint32_t x = (uint32_t)a.x;
            a.x = (int)((x & ~kTermIdMask) | (((x & kTermIdMask) + (uint32_t)db) & kTermIdMask));
            a.y += db; a.z += db; a.w += db;
            W.trv[4 * (size_t)(r.tet0 + i) + q] = a;
        }
    }
    for (int i = t0; i < r.ntri; i += stride) {
        int4 v = W.ridx[r.tri0 + i];
        v.x += db; v.y += db; v.z += db;
        W.ridx[r.tri0 + i] = v;
    }
    for (int i = t0; i < r.ncand; i += stride) {
        for (int t = 0; t < 2; ++t) {
            int2 ab = W.cpair[t][r.cand0 + i];
            ab.x += db; ab.y += db;
            W.cpair[t][r.cand0 + i] = ab;
            W.kbase[t][r.cand0 + i] += dk;
            W.live[t][r.cand0 + i] += dc;
        }
    }
    auto shift = [&](uint32_t e) {
        const uint32_t kind = ent_kind(e), idx = ent_index(e);
        const int d = kind == kEntForce ? df : kind == kEntManifold ? dc : kind == kEntTet ? dt : dr;
        return ent_make(kind, ent_role(e), (uint32_t)((int)idx + d));
    };
    for (int i = t0; i < r.ninc; i += stride) W.inc[r.inc0 + i] = shift(W.inc[r.inc0 + i]);
    for (int i = t0; i < r.nsinc; i += stride)
        const_cast<uint32_t*>(W.sinc)[r.sinc0 + i] = shift(W.sinc[r.sinc0 + i]);
    for (int i = t0; i < r.nsp; i += stride) {
        int2* sp = reinterpret_cast<int2*>(const_cast<int*>(W.spartner));
        int2 pf = sp[r.sp0 + i];
        pf.x += db; pf.y += df;
        sp[r.sp0 + i] = pf;
    }
}

bool live(const AvbdBatch* b, int scene) {
    return b && scene >= 0 && scene < (int)b->state.size() && b->state[scene] == 1;
}

}  // namespace

extern "C" {

int64_t avbd_batch_scene_snapshot_bytes(AvbdBatch* b, int32_t scene) {
    if (!live(b, scene)) return AVBD_ERR_INVALID;
    return scene_snapshot_bytes(b, scene);
}

int32_t avbd_batch_scene_snapshot(AvbdBatch* b, int32_t scene, void* dst, int64_t bytes) {
    if (!live(b, scene) || !dst) return AVBD_ERR_INVALID;
    if (int r = batch_settle(b)) return r;
    const int64_t need = scene_snapshot_bytes(b, scene);
    if (bytes < need) return AVBD_ERR_INVALID;
    if (cudaSetDevice(b->device) != cudaSuccess) return AVBD_ERR_CUDA;
    const std::vector<Slice> slices = scene_slices(b->P);
    SceneSnapHeader h{};
    h.magic = kSceneSnapMagic;
    h.nslices = (uint32_t)slices.size();
    h.src = b->regions[scene];
    h.desc = b->descs[scene];
    h.dynamic = b->dynamic[scene];
    h.bytes = need;
    char* out = static_cast<char*>(dst);
    if (cudaMemcpy(&h.state, b->P.d_sstate + scene, sizeof(SceneState), cudaMemcpyDeviceToHost) != cudaSuccess)
        return AVBD_ERR_CUDA;
    if (cudaMemcpy(out, &h, sizeof(h), cudaMemcpyDefault) != cudaSuccess) return AVBD_ERR_CUDA;
    size_t at = sizeof(h);
    const size_t cbytes = (size_t)(kMaxColours + 1) * sizeof(int);
    cudaMemcpyAsync(out + at, b->P.W.col_start + (size_t)scene * (kMaxColours + 1), cbytes, cudaMemcpyDefault,
                    b->stream);
    at += cbytes;
    int start[kUnits], count[kUnits];
    region_units(h.src, start, count);
    for (const Slice& s : slices) {
        const size_t n = (size_t)count[s.unit] * s.per * s.elem;
        if (n) cudaMemcpyAsync(out + at, static_cast<char*>(s.base) + (size_t)start[s.unit] * s.per * s.elem, n,
                               cudaMemcpyDefault, b->stream);
        at += n;
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    return 0;
}

int32_t avbd_batch_scene_restore(AvbdBatch* b, const void* src, int64_t bytes) {
    if (!b || !src || bytes < (int64_t)sizeof(SceneSnapHeader)) return AVBD_ERR_INVALID;
    if (!b->reserved) return AVBD_ERR_STATE;
    if (int r = batch_settle(b)) return r;
    if (cudaSetDevice(b->device) != cudaSuccess) return AVBD_ERR_CUDA;
    SceneSnapHeader h{};
    if (cudaMemcpy(&h, src, sizeof(h), cudaMemcpyDefault) != cudaSuccess) return AVBD_ERR_CUDA;
    const std::vector<Slice> slices = scene_slices(b->P);
    if (h.magic != kSceneSnapMagic || h.nslices != slices.size() || h.bytes != bytes) return AVBD_ERR_INVALID;
    // a slot and ranges of the snapshot's sizes
    int slot = -1;
    for (size_t i = 0; i < b->state.size(); ++i)
        if (b->state[i] == 0) { slot = (int)i; break; }
    if (slot < 0) {
        if ((int)b->state.size() >= b->P.ns) return AVBD_ERR_NOMEM;
        slot = (int)b->state.size();
        b->scenes.emplace_back();
        b->state.push_back(0);
        b->regions.emplace_back();
        b->descs.emplace_back();
        b->bodies.push_back(0);
        b->dynamic.push_back(0);
    }
    Allocs& A = b->A;
    Region r = h.src;
    int* at[kUnits] = {&r.body0, &r.force0, &r.tet0, &r.tri0, &r.cand0, &r.k0, &r.inc0, &r.sinc0, &r.sp0};
    Ranges* pool[kUnits] = {&A.bodies, &A.forces, &A.tets, &A.tris, &A.cand, &A.k, &A.inc, &A.sinc, &A.sp};
    int start[kUnits], count[kUnits];
    region_units(h.src, start, count);
    for (int u = 0; u < kUnits; ++u) {
        const int s0 = count[u] > 0 ? pool[u]->alloc(count[u]) : 0;
        if (s0 < 0) {
            for (int v = 0; v < u; ++v) pool[v]->release(*at[v], count[v]);
            return AVBD_ERR_NOMEM;
        }
        *at[u] = s0;
    }
    const char* in = static_cast<const char*>(src);
    size_t pos = sizeof(h);
    const size_t cbytes = (size_t)(kMaxColours + 1) * sizeof(int);
    cudaMemcpyAsync(b->P.W.col_start + (size_t)slot * (kMaxColours + 1), in + pos, cbytes, cudaMemcpyDefault,
                    b->stream);
    pos += cbytes;
    int dst0[kUnits], dcount[kUnits];
    region_units(r, dst0, dcount);
    for (const Slice& s : slices) {
        const size_t n = (size_t)count[s.unit] * s.per * s.elem;
        if (n) cudaMemcpyAsync(static_cast<char*>(s.base) + (size_t)dst0[s.unit] * s.per * s.elem, in + pos, n,
                               cudaMemcpyDefault, b->stream);
        pos += n;
    }
    const int d[kUnits] = {r.body0 - h.src.body0, r.force0 - h.src.force0, r.tet0 - h.src.tet0, r.tri0 - h.src.tri0,
                           r.cand0 - h.src.cand0, r.k0 - h.src.k0, r.inc0 - h.src.inc0, r.sinc0 - h.src.sinc0,
                           r.sp0 - h.src.sp0};
    const int n = std::max({r.nbody, r.nforce, r.ntet, r.ntri, r.ncand, r.ninc, r.nsinc, r.nsp, 1});
    k_relocate_scene<<<blocks_for(n), kThreads, 0, b->stream>>>(b->P.W, r, d[kUBody], d[kUForce], d[kUTet],
                                                                 d[kUTri], d[kUCand], d[kUK], d[kUInc], d[kUSinc],
                                                                 d[kUSp]);
    SceneDesc desc = h.desc;
    desc.body0 = r.body0; desc.force0 = r.force0; desc.tet0 = r.tet0; desc.tri0 = r.tri0;
    desc.cand0 = r.cand0; desc.k0 = r.k0; desc.inc0 = r.inc0;
    cudaMemcpyAsync(b->P.d_scenes + slot, &desc, sizeof(desc), cudaMemcpyHostToDevice, b->stream);
    cudaMemcpyAsync(b->P.d_sstate + slot, &h.state, sizeof(SceneState), cudaMemcpyHostToDevice, b->stream);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    b->regions[slot] = r;
    b->descs[slot] = desc;
    b->bodies[slot] = r.nbody;
    b->dynamic[slot] = (int)h.dynamic;
    b->state[slot] = 1;
    b->scenes[slot] = HostScene();
    if ((int)b->steps_due.size() <= slot) b->steps_due.resize(slot + 1, 0);
    b->steps_due[slot] = h.state.step;
    b->order_dirty = true;
    return cudaGetLastError() == cudaSuccess ? slot : AVBD_ERR_CUDA;
}

}  // extern "C"
