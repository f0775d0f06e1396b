// C-ABI of the AVBD library (include/avbd.h): device pools, the single-scene
// launch sequence, the batched persistent kernel, and readback.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/avbd.h"
#include "avbd_host.h"
#include "avbd_step.cuh"
#include "avbd_batch.h"

using namespace avbd;

// ===========================================================================
// Kernels of the single-scene path (grid-wide over the items of scene 0)
// ===========================================================================
namespace {

constexpr int kThreads = 128;

__global__ void k_bp_count(const __grid_constant__ World W) {
    const SceneDesc sc = W.scenes[0];
    for (int b = sc.body0 + blockIdx.x * blockDim.x + threadIdx.x; b < sc.body0 + sc.nbody;
         b += gridDim.x * blockDim.x)
        W.cand_cnt[b] = broadphase_body(W, sc, b, nullptr, 0);
}

__global__ void k_scan_cand(const __grid_constant__ World W) {
    __shared__ TeamShared s_team;
    const Team T = Team::cta(&s_team, nullptr, 0);
    const SceneDesc sc = W.scenes[0];
    const int total = block_exclusive_scan(T, W.cand_cnt + sc.body0, W.cand_off + sc.body0, sc.nbody);
    if (threadIdx.x == 0) W.sstate[0].need_cand = total;
}

__global__ void k_bp_write(const __grid_constant__ World W, int cur) {
    const SceneDesc sc = W.scenes[0];
    for (int b = sc.body0 + blockIdx.x * blockDim.x + threadIdx.x; b < sc.body0 + sc.nbody;
         b += gridDim.x * blockDim.x)
        broadphase_body(W, sc, b, W.cpair[cur] + sc.cand0 + W.cand_off[b], W.cand_cnt[b]);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        W.sstate[0].kused[cur] = 0;
        W.sstate[0].need_k = 0;
        W.sstate[0].nlive[cur] = 0;
        W.sstate[0].nmatched = 0;
    }
}

__global__ void k_narrow(const __grid_constant__ World W, int cur, int ncand, int old_count) {
    const SceneDesc sc = W.scenes[0];
    for (int c = sc.cand0 + blockIdx.x * blockDim.x + threadIdx.x; c < sc.cand0 + ncand;
         c += gridDim.x * blockDim.x)
        narrowphase_slot(W, sc, W.sstate, c, cur, old_count);
}

__global__ void k_force_init(const __grid_constant__ World W) {
    const SceneDesc sc = W.scenes[0];
    for (int f = sc.force0 + blockIdx.x * blockDim.x + threadIdx.x; f < sc.force0 + sc.nforce;
         f += gridDim.x * blockDim.x)
        if (force_init(W, f)) atomicAdd(&W.sstate[0].topo, 1);
}

__global__ void k_incidence_colour(const __grid_constant__ World W, int cur) {
    __shared__ TeamShared s_team;
    __shared__ float4 s_count[(kMaxColours + 1 + 3) / 4];   // colour counts
    const Team T = Team::cta(&s_team, s_count, (kMaxColours + 1 + 3) / 4);
    const SceneDesc sc = W.scenes[0];
    SceneState* st = W.sstate;
    if (!build_incidence(T, W, sc, st, cur)) {
        if (threadIdx.x == 0) st->status = kStatusCapacity;
        return;
    }
    colour_scene_cached(T, W, sc, st, 0, cur);
}

__global__ void k_predict(const __grid_constant__ World W) {
    const SceneDesc sc = W.scenes[0];
    for (int b = sc.body0 + blockIdx.x * blockDim.x + threadIdx.x; b < sc.body0 + sc.nbody;
         b += gridDim.x * blockDim.x)
        predict_body(W, b);
}

// One colour of the primal sweep, groups of G lanes per body across the grid.
template <int G>
__global__ void k_primal(const __grid_constant__ World W, int cur, int first, int count, float alpha,
                         int write_stick) {
    const SceneDesc sc = W.scenes[0];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x % G, gid = t / G, ngroups = gridDim.x * blockDim.x / G;
    for (int base = 0; base < count; base += ngroups) {
        const int i = base + gid;
        int b = i < count ? W.col_list[sc.body0 + first + i] : -1;
        if (b >= 0 && (W.flags[b] & kBodyRemoved)) b = -1;
        primal_group<G>(W, cur, b, alpha, write_stick != 0, lane);
    }
}

void launch_primal(int group, const World& W, int cur, int first, int count, float alpha, int stick, cudaStream_t s) {
    const int threads = kThreads;
    const int blocks = std::max(1, std::min((count * group + threads - 1) / threads, 148 * 32));
    switch (group) {
        case 32: k_primal<32><<<blocks, threads, 0, s>>>(W, cur, first, count, alpha, stick); break;
        case 16: k_primal<16><<<blocks, threads, 0, s>>>(W, cur, first, count, alpha, stick); break;
        case 8: k_primal<8><<<blocks, threads, 0, s>>>(W, cur, first, count, alpha, stick); break;
        case 4: k_primal<4><<<blocks, threads, 0, s>>>(W, cur, first, count, alpha, stick); break;
        case 2: k_primal<2><<<blocks, threads, 0, s>>>(W, cur, first, count, alpha, stick); break;
        default: k_primal<1><<<blocks, threads, 0, s>>>(W, cur, first, count, alpha, stick); break;
    }
}

__global__ void k_dual(const __grid_constant__ World W, int cur, int nlive, float alpha, int last) {
    const SceneDesc sc = W.scenes[0];
    const int n = sc.nforce + nlive;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i < sc.nforce) {
            if (dual_force(W, sc.force0 + i, alpha)) atomicOr(&W.sstate[0].flags, 8);
        } else {
            dual_manifold(W, cur, W.live[cur][sc.cand0 + i - sc.nforce], alpha, last != 0);
        }
    }
}

__global__ void k_fracture_reset(const __grid_constant__ World W, int cur, int nlive) {
    if (!(W.sstate[0].flags & 8)) return;
    const SceneDesc sc = W.scenes[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nlive; i += gridDim.x * blockDim.x)
        fracture_reset_slot(W, cur, W.live[cur][sc.cand0 + i]);
}

__global__ void k_fracture_clear(const __grid_constant__ World W) {
    if (!(W.sstate[0].flags & 8)) return;
    const SceneDesc sc = W.scenes[0];
    for (int b = sc.body0 + blockIdx.x * blockDim.x + threadIdx.x; b < sc.body0 + sc.nbody;
         b += gridDim.x * blockDim.x)
        W.reset_flag[b] = 0;
}

__global__ void k_flags_clear(const __grid_constant__ World W, int mask) {
    if (threadIdx.x == 0) W.sstate[0].flags &= ~mask;
}

__global__ void k_step_done(const __grid_constant__ World W) {
    if (threadIdx.x == 0) W.sstate[0].step += 1;
}

__global__ void k_velocity(const __grid_constant__ World W) {
    const SceneDesc sc = W.scenes[0];
    int acc = 0;
    for (int b = sc.body0 + blockIdx.x * blockDim.x + threadIdx.x; b < sc.body0 + sc.nbody;
         b += gridDim.x * blockDim.x)
        acc |= velocity_body(W, b);
    if (acc) atomicOr(&W.sstate[0].flags, acc);
}

__global__ void k_remove_oob(const __grid_constant__ World W) {
    const SceneDesc sc = W.scenes[0];
    for (int b = sc.body0 + blockIdx.x * blockDim.x + threadIdx.x; b < sc.body0 + sc.nbody;
         b += gridDim.x * blockDim.x) {
        const int fl = W.flags[b];
        if ((fl & (kBodyStatic | kBodyRemoved)) != 0) continue;
        const float4 p = W.pos[b];
        if (p.x < kBoundMin || p.x > kBoundMax || p.y < kBoundMin || p.y > kBoundMax || p.z < kBoundMin ||
            p.z > kBoundMax) {
            W.flags[b] = fl | kBodyRemoved;
            atomicAdd(&W.sstate[0].topo, 1);
            for (int e = W.sinc_off[b]; e < W.sinc_off[b] + W.sinc_n[b]; ++e) {
                const uint32_t ent = W.sinc[e];
                const uint32_t k = ent_kind(ent), idx = ent_index(ent);
                if (k == kEntForce) atomicOr(&W.ftype[idx], kForceRemoved);
                else if (k == kEntTet) W.tparam[idx].w = 1.f;
                else if (k == kEntTri) W.rparam[idx].w = 1.f;
            }
        }
    }
}

// RemoveBody / RemoveForce / RemoveEnergy on an uploaded world: the same marks
// as the out-of-bounds removal, plus a topology bump so the colouring is redone.
// kind 0 body, 1 force, 2 tet, 3 triangle; idx is the global index.
__global__ void k_remove_item(const __grid_constant__ World W, int kind, int idx) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    if (kind == 0) {
        W.flags[idx] |= kBodyRemoved;
        for (int e = W.sinc_off[idx]; e < W.sinc_off[idx] + W.sinc_n[idx]; ++e) {
            const uint32_t ent = W.sinc[e];
            const uint32_t k = ent_kind(ent), i = ent_index(ent);
            if (k == kEntForce) W.ftype[i] |= kForceRemoved;
            else if (k == kEntTet) W.tparam[i].w = 1.f;
            else if (k == kEntTri) W.rparam[i].w = 1.f;
        }
    } else if (kind == 1) {
        W.ftype[idx] |= kForceRemoved;
    } else if (kind == 2) {
        W.tparam[idx].w = 1.f;
    } else {
        W.rparam[idx].w = 1.f;
    }
    W.sstate[0].topo += 1;
}

__global__ void k_collide(const __grid_constant__ World W, int a, int b, uint32_t* ids, float* data, int* n) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    Collision col;
    collide_box_box(v3(W.pos[a]), q4(W.rot[a]), v3(W.scale[a]), v3(W.pos[b]), q4(W.rot[b]), v3(W.scale[b]), col);
    *n = col.n;
    for (int k = 0; k < col.n; ++k) {
        const Contact& c = col.c[k];
        ids[k] = c.id;
        float* d = data + 13 * k;
        d[0] = c.penetration;
        d[1] = c.normal.x; d[2] = c.normal.y; d[3] = c.normal.z;
        d[4] = c.rA.x; d[5] = c.rA.y; d[6] = c.rA.z;
        d[7] = c.rB.x; d[8] = c.rB.y; d[9] = c.rB.z;
        d[10] = c.position.x; d[11] = c.position.y; d[12] = c.position.z;
    }
}

// ===========================================================================
// Batched path: the persistent kernel builds live in their own translation
// units (avbd_batch_v.cu, compiled once per build); this table indexes them.
// ===========================================================================
struct BatchVariant {
    BatchKernel fn;
    int max_threads;
};
// Index = register variant of avbd_batch_set_kernel.
const BatchVariant kBatchVariants[] = {
    {nullptr, 0},
    {batch_kernel_v1(), 256}, {batch_kernel_v2(), 256}, {batch_kernel_v3(), 256},
    {batch_kernel_v4(), 256}, {batch_kernel_v5(), 512}, {batch_kernel_v6(), 512},
    {batch_kernel_v7(), 1024},
};
constexpr int kNumBatchVariants = 7;

int blocks_for(int n, int threads = kThreads) {
    int b = (n + threads - 1) / threads;
    return std::max(1, std::min(b, 148 * 32));
}

}  // namespace

// ===========================================================================
// Device pools
// ===========================================================================
namespace {

struct Pools {
    World W{};
    int device = 0;
    // capacities
    int nb = 0, nf = 0, nt = 0, nr = 0, ns = 0;
    int ncand = 0, nk = 0, ninc = 0, nsinc = 0, nsp = 0;
    std::vector<void*> owned;
    std::vector<size_t> owned_bytes;   // size of each owned allocation (snapshots)
    SceneDesc* d_scenes = nullptr;
    SceneState* d_sstate = nullptr;

    ~Pools() { release(); }
    void release() {
        for (void* p : owned) cudaFree(p);
        owned.clear();
        owned_bytes.clear();
        W = World{};
    }
    // zero = false for arrays every reader finds written first (contact points:
    // the narrowphase fills a slot before any phase reads it)
    template <typename T>
    cudaError_t alloc(T*& p, size_t n, bool zero = true) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) return e;
        if (zero) cudaMemset(q, 0, std::max<size_t>(n, 1) * sizeof(T));
        owned.push_back(q);
        owned_bytes.push_back(std::max<size_t>(n, 1) * sizeof(T));
        p = static_cast<T*>(q);
        return cudaSuccess;
    }
    template <typename T>
    cudaError_t alloc_c(const T*& p, size_t n) {
        T* q = nullptr;
        cudaError_t e = alloc(q, n);
        p = q;
        return e;
    }
    void forget(void* p) {
        auto it = std::find(owned.begin(), owned.end(), p);
        if (it != owned.end()) {
            cudaFree(p);
            owned_bytes.erase(owned_bytes.begin() + (it - owned.begin()));
            owned.erase(it);
        }
    }

    cudaError_t allocate_all() {
        cudaError_t e = cudaSuccess;
        if (nb >= kMaxPoolBodies) return cudaErrorInvalidValue;   // tet-term records keep ids in 28 bits
#define A(expr) if ((e = (expr)) != cudaSuccess) return e
        A(alloc(d_scenes, ns));
        A(alloc(d_sstate, ns));
        W.scenes = d_scenes;
        W.sstate = d_sstate;
        W.nscenes = ns;
        A(alloc(W.pos, nb)); A(alloc(W.rot, nb)); A(alloc(W.scale, nb)); A(alloc(W.lpos, nb));
        A(alloc(W.lrot, nb)); A(alloc(W.ipos, nb)); A(alloc(W.irot, nb)); A(alloc(W.vel, nb));
        A(alloc(W.omega, nb)); A(alloc(W.pvel, nb)); A(alloc(W.dlin, nb)); A(alloc(W.dang, nb));
        A(alloc(W.massI, nb)); A(alloc(W.Mw0, nb)); A(alloc(W.Mw1, nb));
        A(alloc(W.flags, nb)); A(alloc(W.friction, nb)); A(alloc(W.colour, nb)); A(alloc(W.local, nb));
        A(alloc(W.reset_flag, nb));
        A(alloc_c(W.sinc_off, nb)); A(alloc_c(W.sinc_n, nb)); A(alloc_c(W.sinc_nf, nb)); A(alloc_c(W.sinc, nsinc));
        A(alloc_c(W.spartner_off, nb)); A(alloc_c(W.spartner_n, nb)); A(alloc_c(W.spartner, 2 * (size_t)nsp));
        A(alloc(W.inc_off, nb)); A(alloc(W.inc_cnt, nb)); A(alloc(W.cntB, nb)); A(alloc(W.bcur, nb));
        A(alloc(W.cand_cnt, nb)); A(alloc(W.cand_off, nb));
        A(alloc(W.col_list, nb)); A(alloc(W.col_tinc, nb)); A(alloc(W.col_start, (size_t)ns * (kMaxColours + 1)));
        A(alloc(W.ftype, nf)); A(alloc(W.fbody, nf)); A(alloc(W.frA, nf)); A(alloc(W.frB, nf));
        A(alloc(W.fq, nf)); A(alloc(W.fparam, nf)); A(alloc(W.fC0p, nf)); A(alloc(W.fC0a, nf));
        A(alloc(W.fk, 6 * (size_t)nf)); A(alloc(W.ffrac, 6 * (size_t)nf)); A(alloc(W.ffmin, 6 * (size_t)nf));
        A(alloc(W.ffmax, 6 * (size_t)nf)); A(alloc(W.fpen, 6 * (size_t)nf)); A(alloc(W.flam, 6 * (size_t)nf));
        A(alloc(W.tidx, nt)); A(alloc(W.tDmInv, 9 * (size_t)nt)); A(alloc(W.tgradN, 12 * (size_t)nt));
        A(alloc(W.tparam, nt)); A(alloc(W.tkind, nt));
        A(alloc(W.trv, 4 * (size_t)nt)); A(alloc(W.trm0, 4 * (size_t)nt)); A(alloc(W.trm1, 4 * (size_t)nt));
        A(alloc(W.trm2, 4 * (size_t)nt));
        A(alloc(W.ridx, nr)); A(alloc(W.rDmInv, nr)); A(alloc(W.rgradN, 6 * (size_t)nr)); A(alloc(W.rparam, nr));
        A(alloc(W.inc, ninc));
        for (int t = 0; t < 2; ++t) A(alloc_tables(t, ncand, nk));
#undef A
        return e;
    }

    cudaError_t alloc_tables(int t, int nc, int k) {
        cudaError_t e = cudaSuccess;
#define A(expr) if ((e = (expr)) != cudaSuccess) return e
        A(alloc(W.cpair[t], nc)); A(alloc(W.cn[t], nc)); A(alloc(W.cfric[t], nc)); A(alloc(W.kbase[t], nc));
        A(alloc(W.cbirth[t], nc)); A(alloc(W.live[t], nc));
        A(alloc(W.kid[t], k, false)); A(alloc(W.krA[t], k, false)); A(alloc(W.krB[t], k, false));
        A(alloc(W.kn[t], k, false)); A(alloc(W.kt1[t], k, false)); A(alloc(W.kt2[t], k, false));
        A(alloc(W.krAw[t], k, false)); A(alloc(W.krBw[t], k, false)); A(alloc(W.kpen[t], k, false));
        A(alloc(W.klam[t], k, false));
#undef A
        return e;
    }

    template <typename T>
    cudaError_t grow(T*& p, size_t old_n, size_t new_n, size_t keep) {
        T* q = nullptr;
        cudaError_t e = alloc(q, new_n);
        if (e != cudaSuccess) return e;
        if (keep) cudaMemcpy(q, p, std::min(keep, old_n) * sizeof(T), cudaMemcpyDeviceToDevice);
        forget(p);
        p = q;
        return cudaSuccess;
    }

    // Grows the candidate tables of both buffers to nc slots (keeping the
    // first keep0/keep1 slots) and the contact pools to k slots.
    cudaError_t grow_tables(int nc, int k, int keep_c0, int keep_c1, int keep_k0, int keep_k1) {
        cudaError_t e = cudaSuccess;
        for (int t = 0; t < 2; ++t) {
            const int kc = t ? keep_c1 : keep_c0, kk = t ? keep_k1 : keep_k0;
            if (nc > ncand) {
                if ((e = grow(W.cpair[t], ncand, nc, kc)) != cudaSuccess) return e;
                if ((e = grow(W.cn[t], ncand, nc, kc)) != cudaSuccess) return e;
                if ((e = grow(W.cfric[t], ncand, nc, kc)) != cudaSuccess) return e;
                if ((e = grow(W.kbase[t], ncand, nc, kc)) != cudaSuccess) return e;
                if ((e = grow(W.cbirth[t], ncand, nc, kc)) != cudaSuccess) return e;
                if ((e = grow(W.live[t], ncand, nc, kc)) != cudaSuccess) return e;
            }
            if (k > nk) {
                if ((e = grow(W.kid[t], nk, k, kk)) != cudaSuccess) return e;
                if ((e = grow(W.krA[t], nk, k, kk)) != cudaSuccess) return e;
                if ((e = grow(W.krB[t], nk, k, kk)) != cudaSuccess) return e;
                if ((e = grow(W.kn[t], nk, k, kk)) != cudaSuccess) return e;
                if ((e = grow(W.kt1[t], nk, k, kk)) != cudaSuccess) return e;
                if ((e = grow(W.kt2[t], nk, k, kk)) != cudaSuccess) return e;
                if ((e = grow(W.krAw[t], nk, k, kk)) != cudaSuccess) return e;
                if ((e = grow(W.krBw[t], nk, k, kk)) != cudaSuccess) return e;
                if ((e = grow(W.kpen[t], nk, k, kk)) != cudaSuccess) return e;
                if ((e = grow(W.klam[t], nk, k, kk)) != cudaSuccess) return e;
            }
        }
        ncand = std::max(ncand, nc);
        nk = std::max(nk, k);
        return e;
    }
};

// Lanes per body in the primal sweep: FEM vertices gather about 20 tets each,
// rigid bodies a handful of manifolds.
int scene_group(const HostScene& h, int rigid_group, int fem_group) {
    if (h.ntet() == 0 && h.ntri() == 0) return rigid_group;
    if (fem_group == kGroupFlat && h.ntri() > 0) return 4;   // the flat sweep takes tet energies only
    return fem_group;
}

// Capacity policy of one scene.
void scene_caps(const HostScene& h, int& candcap, int& kcap) {
    const int n = h.nbody();
    candcap = 16 * n + 64;   // a body in a column stack overlaps ~18 circumscribed spheres (owns ~9)
    kcap = 8 * n + 128;      // live contact points average ~1.5 per body; a scene that needs more grows
}


// First-fit allocator of index ranges in one pool, with coalescing frees.
struct Ranges {
    int cap = 0;
    std::map<int, int> free_;   // start -> length
    void reset(int c) {
        cap = c;
        free_.clear();
        if (c > 0) free_[0] = c;
    }
    int alloc(int n) {
        if (n <= 0) return 0;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                const int s = it->first, len = it->second;
                free_.erase(it);
                if (len > n) free_[s + n] = len - n;
                return s;
            }
        }
        return -1;
    }
    void release(int s, int n) {
        if (n <= 0) return;
        auto it = free_.emplace(s, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

// Where one scene lives in the pools.
struct Region {
    int body0 = 0, nbody = 0, force0 = 0, nforce = 0, tet0 = 0, ntet = 0, tri0 = 0, ntri = 0;
    int cand0 = 0, ncand = 0, k0 = 0, nk = 0, inc0 = 0, ninc = 0, sinc0 = 0, nsinc = 0, sp0 = 0, nsp = 0;
};

struct Allocs {
    Ranges bodies, forces, tets, tris, cand, k, inc, sinc, sp;
    void reset(const Pools& P) {
        bodies.reset(P.nb); forces.reset(P.nf); tets.reset(P.nt); tris.reset(P.nr); cand.reset(P.ncand);
        k.reset(P.nk); inc.reset(P.ninc); sinc.reset(P.nsinc); sp.reset(P.nsp);
    }
    void release(const Region& r) {
        bodies.release(r.body0, r.nbody); forces.release(r.force0, r.nforce); tets.release(r.tet0, r.ntet);
        tris.release(r.tri0, r.ntri); cand.release(r.cand0, r.ncand); k.release(r.k0, r.nk);
        inc.release(r.inc0, r.ninc); sinc.release(r.sinc0, r.nsinc); sp.release(r.sp0, r.nsp);
    }
};

// Static incidence of a scene, built once per placement.
struct StaticInc {
    std::vector<int> off, cnt, nf, poff, pcnt;
    std::vector<uint32_t> ent;
    std::vector<int2> partners;
};

// Reserves pool ranges for a scene; false (and nothing held) if a pool is full.
bool place_scene(Allocs& A, const HostScene& h, int candcap, int kcap, int nsinc, int nsp, Region& r) {
    r = Region{};
    r.nbody = h.nbody(); r.nforce = h.nforce(); r.ntet = h.ntet(); r.ntri = h.ntri();
    r.ncand = candcap; r.nk = kcap; r.nsinc = nsinc; r.nsp = nsp; r.ninc = nsinc + 2 * candcap;
    bool ok = true;
    auto take = [&](Ranges& rg, int n, int& at) {
        if (!ok) return;
        at = rg.alloc(n);
        if (at < 0) { ok = false; at = 0; }
    };
    Region got;   // ranges taken so far, for the rollback
    take(A.bodies, r.nbody, r.body0); if (ok) { got.body0 = r.body0; got.nbody = r.nbody; }
    take(A.forces, r.nforce, r.force0); if (ok) { got.force0 = r.force0; got.nforce = r.nforce; }
    take(A.tets, r.ntet, r.tet0); if (ok) { got.tet0 = r.tet0; got.ntet = r.ntet; }
    take(A.tris, r.ntri, r.tri0); if (ok) { got.tri0 = r.tri0; got.ntri = r.ntri; }
    take(A.cand, r.ncand, r.cand0); if (ok) { got.cand0 = r.cand0; got.ncand = r.ncand; }
    take(A.k, r.nk, r.k0); if (ok) { got.k0 = r.k0; got.nk = r.nk; }
    take(A.inc, r.ninc, r.inc0); if (ok) { got.inc0 = r.inc0; got.ninc = r.ninc; }
    take(A.sinc, r.nsinc, r.sinc0); if (ok) { got.sinc0 = r.sinc0; got.nsinc = r.nsinc; }
    take(A.sp, r.nsp, r.sp0); if (ok) { got.sp0 = r.sp0; got.nsp = r.nsp; }
    if (!ok) A.release(got);
    return ok;
}

// Where upload_scene's data goes.  DirectSink: straight to the device, one
// copy per array of the scene.  StagedSink: into one host buffer per device
// array at the scene's offsets, flushed with one copy per array, for packing
// many scenes into fresh (zeroed) pools at once.
struct DirectSink {
    cudaStream_t st;
    template <typename T>
    void put(T* dst, const std::vector<T>& src, size_t at) {
        if (!src.empty()) cudaMemcpyAsync(dst + at, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st);
    }
    template <typename T>
    void zero(T* dst, size_t at, size_t n) {
        if (n) cudaMemsetAsync(dst + at, 0, n * sizeof(T), st);
    }
    void finish() { cudaStreamSynchronize(st); }   // the caller's host vectors are temporaries
};

struct StagedSink {
    struct Buf {
        char* host = nullptr;   // calloc'd: untouched pages read as zero and cost nothing
        size_t cap = 0, lo = SIZE_MAX, hi = 0;
        bool locked = false;    // [lo, hi) page-locked
    };
    std::map<char*, Buf> bufs;
    const Pools* P = nullptr;   // allocation sizes: each buffer is sized once to its pool array
    cudaStream_t st = nullptr;
    std::mutex m;               // scenes are staged from several host threads
    bool overflow = false;      // a write outside its pool array (never expected)
    ~StagedSink() { release(); }
    // The host buffer of pool array `dst` with [off, off + n) marked written;
    // null (and overflow set) if that range lies outside the array.
    char* span(void* dst, size_t off, size_t n) {
        std::lock_guard<std::mutex> lock(m);
        Buf& b = bufs[static_cast<char*>(dst)];
        if (!b.host) {
            size_t cap = off + n;
            if (P)
                for (size_t i = 0; i < P->owned.size(); ++i)
                    if (P->owned[i] == dst) cap = std::max(cap, P->owned_bytes[i]);
            b.host = static_cast<char*>(std::calloc(cap, 1));
            b.cap = b.host ? cap : 0;
        }
        if (b.cap < off + n) {
            overflow = true;
            return nullptr;
        }
        b.lo = std::min(b.lo, off);
        b.hi = std::max(b.hi, off + n);
        return b.host;
    }
    template <typename T>
    void put(T* dst, const std::vector<T>& src, size_t at) {
        if (src.empty()) return;
        if (char* h = span(dst, at * sizeof(T), src.size() * sizeof(T)))
            std::memcpy(h + at * sizeof(T), src.data(), src.size() * sizeof(T));
    }
    template <typename T>
    void zero(T* dst, size_t at, size_t n) {
        if (!n) return;
        if (char* h = span(dst, at * sizeof(T), n * sizeof(T))) std::memset(h + at * sizeof(T), 0, n * sizeof(T));
    }
    void finish() {}
    // Page-locks the written range of every buffer, so the copies run at the
    // link's rate instead of through the driver's pageable bounce buffers.
    void lock() {
        for (auto& kv : bufs)
            if (kv.second.hi > kv.second.lo && !kv.second.locked)
                kv.second.locked = cudaHostRegister(kv.second.host + kv.second.lo, kv.second.hi - kv.second.lo,
                                                    cudaHostRegisterDefault) == cudaSuccess;
        cudaGetLastError();   // a refused registration leaves a pageable (slower) copy
    }
    // One copy per written range, then the stream is synchronised; the host
    // buffers are kept until release() (page-locked memory is slow to free).
    bool flush() {
        copied = 0;
        for (auto& kv : bufs)
            if (kv.second.hi > kv.second.lo) {
                cudaMemcpyAsync(kv.first + kv.second.lo, kv.second.host + kv.second.lo, kv.second.hi - kv.second.lo,
                                cudaMemcpyHostToDevice, st);
                copied += (int64_t)(kv.second.hi - kv.second.lo);
            }
        cudaStreamSynchronize(st);
        return !overflow;
    }
    int64_t copied = 0;   // bytes the last flush copied
    void release() {
        for (auto& kv : bufs) {
            if (kv.second.locked) cudaHostUnregister(kv.second.host + kv.second.lo);
            std::free(kv.second.host);
        }
        bufs.clear();
    }
};

// Writes a placed scene (as staged) into the pools and its descriptor/state
// into scene slot `slot`.
template <typename Sink>
void upload_scene(Pools& P, const HostScene& h, const StaticInc& si, const Region& r, int group, int slot,
                  SceneDesc& d, Sink& sink) {
    d.body0 = r.body0; d.nbody = r.nbody;
    d.force0 = r.force0; d.nforce = r.nforce;
    d.tet0 = r.tet0; d.ntet = r.ntet;
    d.tri0 = r.tri0; d.ntri = r.ntri;
    d.cand0 = r.cand0; d.candcap = r.ncand;
    d.k0 = r.k0; d.kcap = r.nk;
    d.inc0 = r.inc0; d.inccap = r.ninc;
    d.ndynamic = h.ndynamic();
    d.group = group;
    World& W = P.W;
    sink.put(W.pos, h.pos, d.body0); sink.put(W.rot, h.rot, d.body0); sink.put(W.scale, h.scale, d.body0);
    sink.put(W.vel, h.vel, d.body0); sink.put(W.omega, h.omega, d.body0); sink.put(W.massI, h.massI, d.body0);
    sink.put(W.flags, h.flags, d.body0); sink.put(W.friction, h.friction, d.body0);
    sink.put(W.lpos, h.pos, d.body0); sink.put(W.lrot, h.rot, d.body0);
    sink.put(W.ipos, h.pos, d.body0); sink.put(W.irot, h.rot, d.body0);
    sink.zero(W.pvel, d.body0, d.nbody);
    sink.zero(W.reset_flag, d.body0, d.nbody);
    std::vector<int> tmp(d.nbody);
    for (int b = 0; b < d.nbody; ++b) tmp[b] = b;
    sink.put(W.local, tmp, d.body0);
    for (int b = 0; b < d.nbody; ++b) tmp[b] = si.off[b] + r.sinc0;
    sink.put(const_cast<int*>(W.sinc_off), tmp, d.body0);
    sink.put(const_cast<int*>(W.sinc_n), si.cnt, d.body0);
    sink.put(const_cast<int*>(W.sinc_nf), si.nf, d.body0);
    sink.put(const_cast<uint32_t*>(W.sinc), si.ent, r.sinc0);
    for (int b = 0; b < d.nbody; ++b) tmp[b] = si.poff[b] + r.sp0;
    sink.put(const_cast<int*>(W.spartner_off), tmp, d.body0);
    sink.put(const_cast<int*>(W.spartner_n), si.pcnt, d.body0);
    sink.put(reinterpret_cast<int2*>(const_cast<int*>(W.spartner)), si.partners, r.sp0);
    std::vector<int2> fb = h.fbody;
    for (auto& ab : fb) { if (ab.x >= 0) ab.x += d.body0; ab.y += d.body0; }
    sink.put(W.ftype, h.ftype, d.force0); sink.put(W.fbody, fb, d.force0); sink.put(W.frA, h.frA, d.force0);
    sink.put(W.frB, h.frB, d.force0); sink.put(W.fq, h.fq, d.force0); sink.put(W.fparam, h.fparam, d.force0);
    sink.put(W.fk, h.fk, 6 * (size_t)d.force0); sink.put(W.ffrac, h.ffrac, 6 * (size_t)d.force0);
    sink.put(W.ffmin, h.ffmin, 6 * (size_t)d.force0); sink.put(W.ffmax, h.ffmax, 6 * (size_t)d.force0);
    sink.zero(W.fpen, 6 * (size_t)d.force0, 6 * (size_t)d.nforce);
    sink.zero(W.flam, 6 * (size_t)d.force0, 6 * (size_t)d.nforce);
    std::vector<int4> ti = h.tidx;
    for (auto& t : ti) { t.x += d.body0; t.y += d.body0; t.z += d.body0; t.w += d.body0; }
    sink.put(W.tidx, ti, d.tet0); sink.put(W.tDmInv, h.tDmInv, 9 * (size_t)d.tet0);
    sink.put(W.tgradN, h.tgradN, 12 * (size_t)d.tet0); sink.put(W.tparam, h.tparam, d.tet0);
    sink.put(W.tkind, h.tkind, d.tet0);
    std::vector<int4> ri = h.ridx;
    for (auto& t : ri) { t.x += d.body0; t.y += d.body0; t.z += d.body0; }
    sink.put(W.ridx, ri, d.tri0); sink.put(W.rDmInv, h.rDmInv, d.tri0);
    sink.put(W.rgradN, h.rgradN, 6 * (size_t)d.tri0); sink.put(W.rparam, h.rparam, d.tri0);
    sink.put(P.d_scenes, std::vector<SceneDesc>(1, d), slot);
    sink.zero(P.d_sstate, slot, 1);
    sink.finish();
}

// Static incidence entries and joint/spring partner entries a scene needs.
void static_counts(const HostScene& h, int& nsinc, int& nsp) {
    nsinc = 4 * h.ntet() + 3 * h.ntri();
    nsp = 0;
    for (const int2& ab : h.fbody) {
        nsinc += ab.x >= 0 ? 2 : 1;
        nsp += ab.x >= 0 ? 2 : 0;
    }
}

StaticInc static_incidence(const HostScene& h, const Region& r) {
    StaticInc si;
    h.build_static_incidence(si.off, si.cnt, si.nf, si.ent, si.poff, si.pcnt, si.partners, r.body0, r.force0, r.tet0,
                             r.tri0);
    return si;
}

Params to_params(const AvbdParams& p) {
    Params q;
    q.num_iterations = p.num_iterations;
    q.dt = p.step_value;
    q.alpha = p.alpha;
    q.beta = p.beta;
    q.gamma = p.gamma;
    q.on_penetration_penalty = p.on_penetration_penalty;
    q.post_stabilization = p.post_stabilization;
    q.projection_mode = p.projection_mode;
    q.trust_region_rho = p.trust_region_rho;
    return q;
}

bool valid_params(const AvbdParams* p) {
    return p && p->num_iterations >= 0 && p->step_value > 0.f && p->projection_mode >= 0 && p->projection_mode <= 2;
}

int device_ready(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return AVBD_ERR_NODEVICE;
    if (device < 0 || device >= n) return AVBD_ERR_INVALID;
    return cudaSetDevice(device) == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

}  // namespace

// ===========================================================================
// Single-scene world
// ===========================================================================
struct AvbdWorld {
    AvbdParams params{};
    int device = 0;
    HostScene h;
    bool uploaded = false;
    bool stopped = false;
    int stop_status = AVBD_STATUS_OK;   // EXPLODED or NAN once stopped
    Pools P;
    std::vector<SceneDesc> descs;
    int group = 0;   // lanes per body in the primal (0 = by scene kind)
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8] = {};
    AvbdTimings timings{};
    int ncolours = 0;
    std::vector<int> col_start;
    SceneState st{};   // host mirror of the scene counters after the last step
};

namespace {

int sync_state(AvbdWorld* w) {
    if (cudaMemcpyAsync(&w->st, w->P.d_sstate, sizeof(SceneState), cudaMemcpyDeviceToHost, w->stream) != cudaSuccess)
        return AVBD_ERR_CUDA;
    if (cudaStreamSynchronize(w->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    return 0;
}

int upload(AvbdWorld* w) {
    int r = device_ready(w->device);
    if (r) return r;
    if (!w->stream) {
        if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess) return AVBD_ERR_CUDA;
        for (auto& e : w->ev) cudaEventCreate(&e);
    }
    int cc, kc, nsinc, nsp;
    scene_caps(w->h, cc, kc);
    static_counts(w->h, nsinc, nsp);
    const int g = w->group > 0 ? w->group : scene_group(w->h, 4, 8);
    Pools& P = w->P;
    P.release();
    P.ns = 1; P.nb = w->h.nbody(); P.nf = w->h.nforce(); P.nt = w->h.ntet(); P.nr = w->h.ntri();
    P.ncand = cc; P.nk = kc; P.nsinc = nsinc; P.nsp = nsp; P.ninc = nsinc + 2 * cc;
    if (P.allocate_all() != cudaSuccess) return AVBD_ERR_NOMEM;
    Allocs A;
    A.reset(P);
    Region reg;
    if (!place_scene(A, w->h, cc, kc, nsinc, nsp, reg)) return AVBD_ERR_NOMEM;
    w->descs.assign(1, SceneDesc{});
    DirectSink sink{w->stream};
    upload_scene(P, w->h, static_incidence(w->h, reg), reg, g, 0, w->descs[0], sink);
    if (cudaGetLastError() != cudaSuccess) return AVBD_ERR_CUDA;
    P.W.P = to_params(w->params);
    w->uploaded = true;
    return 0;
}

// Grows tables of scene 0 so the candidate slots / contacts / incidence fit.
int ensure_caps(AvbdWorld* w, int need_cand, int need_k) {
    SceneDesc& d = w->descs[0];
    bool changed = false;
    int nc = d.candcap, nk = d.kcap;
    if (need_cand > nc) { nc = std::max(need_cand + need_cand / 2, 2 * nc); changed = true; }
    if (need_k > nk) { nk = std::max(need_k + need_k / 2, 2 * nk); changed = true; }
    if (!changed) return 0;
    cudaStreamSynchronize(w->stream);
    SceneState st;
    cudaMemcpy(&st, w->P.d_sstate, sizeof(SceneState), cudaMemcpyDeviceToHost);
    if (w->P.grow_tables(nc, nk, st.ncand[0], st.ncand[1], st.kused[0], st.kused[1]) != cudaSuccess)
        return AVBD_ERR_NOMEM;
    const int ns = w->P.nsinc;
    const int inccap = ns + 2 * nc;
    if (inccap > w->P.ninc) {
        if (w->P.grow(w->P.W.inc, (size_t)w->P.ninc, (size_t)inccap, 0) != cudaSuccess) return AVBD_ERR_NOMEM;
        w->P.ninc = inccap;
    }
    d.candcap = nc;
    d.kcap = nk;
    d.inccap = inccap;
    cudaMemcpy(w->P.d_scenes, &d, sizeof(SceneDesc), cudaMemcpyHostToDevice);
    return 0;
}

float ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

int world_step(AvbdWorld* w) {
    if (w->stopped) return w->stop_status;
    if (!w->uploaded) {
        int r = upload(w);
        if (r) return r;
    }
    if (cudaSetDevice(w->device) != cudaSuccess) return AVBD_ERR_CUDA;
    Pools& P = w->P;
    P.W.P = to_params(w->params);
    const SceneDesc& d = w->descs[0];
    cudaStream_t s = w->stream;
    int r = sync_state(w);
    if (r) return r;
    const int old = w->st.cur, cur = old ^ 1;
    const int old_count = w->st.ncand[old];
    cudaEventRecord(w->ev[0], s);
    // ---- broadphase ----
    k_bp_count<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W);
    k_scan_cand<<<1, 1024, 0, s>>>(P.W);
    if ((r = sync_state(w))) return r;
    const int ncand = w->st.need_cand;
    if ((r = ensure_caps(w, ncand, 0))) return r;
    k_bp_write<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W, cur);
    cudaEventRecord(w->ev[1], s);
    // ---- narrowphase + manifold warm start (re-run after growing the contact pool) ----
    for (int attempt = 0; attempt < 4; ++attempt) {
        k_narrow<<<blocks_for(ncand), kThreads, 0, s>>>(P.W, cur, ncand, old_count);
        if ((r = sync_state(w))) return r;
        if (!w->st.need_k) break;
        if ((r = ensure_caps(w, 0, w->st.kused[cur]))) return r;
        SceneState fix = w->st;
        fix.kused[cur] = 0;
        fix.need_k = 0;
        fix.nlive[cur] = 0;
        fix.nmatched = 0;
        cudaMemcpy(P.d_sstate, &fix, sizeof(SceneState), cudaMemcpyHostToDevice);
    }
    if (w->st.need_k) return AVBD_STATUS_CAPACITY;
    {
        SceneState upd = w->st;
        upd.ncand[cur] = ncand;
        upd.cur = cur;
        upd.status = kStatusOk;
        upd.flags = 0;
        cudaMemcpyAsync(P.d_sstate, &upd, sizeof(SceneState), cudaMemcpyHostToDevice, s);
    }
    if (d.nforce) k_force_init<<<blocks_for(d.nforce), kThreads, 0, s>>>(P.W);
    // ---- incidence + colouring (one CTA) ----
    k_incidence_colour<<<1, 1024, 0, s>>>(P.W, cur);
    cudaEventRecord(w->ev[2], s);
    if ((r = sync_state(w))) return r;
    if (w->st.status != kStatusOk) return w->st.status == kStatusTimeout ? AVBD_STATUS_TIMEOUT : AVBD_STATUS_CAPACITY;
    const int ncol = w->st.ncolours;
    const int nlive = w->st.nlive[cur];
    w->ncolours = ncol;
    w->col_start.resize(ncol + 1);
    cudaMemcpyAsync(w->col_start.data(), P.W.col_start, (ncol + 1) * sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    cudaEventRecord(w->ev[3], s);
    // ---- prediction ----
    k_predict<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W);
    cudaEventRecord(w->ev[4], s);
    // ---- iterations ----
    const float alpha = w->params.alpha;
    const bool has_fracture = d.nforce > 0;
    for (int it = 0; it < w->params.num_iterations; ++it) {
        for (int c = 0; c < ncol; ++c) {
            const int n = w->col_start[c + 1] - w->col_start[c];
            if (n > 0) launch_primal(d.group, P.W, cur, w->col_start[c], n, alpha, 0, s);
        }
        const int last = it == w->params.num_iterations - 1;
        if (d.nforce + nlive > 0)
            k_dual<<<blocks_for(d.nforce + nlive), kThreads, 0, s>>>(P.W, cur, nlive, alpha, last);
        if (has_fracture) {
            k_fracture_reset<<<blocks_for(nlive), kThreads, 0, s>>>(P.W, cur, nlive);
            k_fracture_clear<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W);
            k_flags_clear<<<1, 32, 0, s>>>(P.W, 8);
        }
    }
    cudaEventRecord(w->ev[5], s);
    // ---- velocities ----
    k_velocity<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W);
    if ((r = sync_state(w))) return r;
    cudaEventRecord(w->ev[6], s);
    int status = AVBD_STATUS_OK;
    if (w->st.flags & 1) status = AVBD_STATUS_EXPLODED;
    else if (w->st.flags & 2) status = AVBD_STATUS_NAN;
    if (status != AVBD_STATUS_OK) {
        w->stopped = true;
        w->stop_status = status;
        cudaStreamSynchronize(s);
        return status;
    }
    if (w->st.flags & 4) k_remove_oob<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W);
    k_step_done<<<1, 32, 0, s>>>(P.W);
    // ---- post-stabilisation ----
    if (w->params.post_stabilization) {
        for (int c = 0; c < ncol; ++c) {
            const int n = w->col_start[c + 1] - w->col_start[c];
            if (n > 0) launch_primal(d.group, P.W, cur, w->col_start[c], n, 0.f, 1, s);
        }
    }
    cudaEventRecord(w->ev[7], s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return AVBD_ERR_CUDA;
    if (cudaGetLastError() != cudaSuccess) return AVBD_ERR_CUDA;
    AvbdTimings& t = w->timings;
    t.broad_phase_ms = ev_ms(w->ev[0], w->ev[1]);
    t.warmstart_ms = ev_ms(w->ev[1], w->ev[2]);
    t.colouring_ms = 0.f;
    t.prediction_ms = ev_ms(w->ev[3], w->ev[4]);
    t.primal_dual_ms = ev_ms(w->ev[4], w->ev[5]);
    t.velocity_update_ms = ev_ms(w->ev[5], w->ev[6]);
    t.post_stab_ms = ev_ms(w->ev[6], w->ev[7]);
    t.total_substep_ms = ev_ms(w->ev[0], w->ev[7]);
    return AVBD_STATUS_OK;
}

}  // namespace

// ===========================================================================
// Batch
// ===========================================================================
struct AvbdBatch {
    AvbdParams params{};
    int device = 0;
    // scene slots (scene id = slot); a retired slot is reused by a later scene
    std::vector<HostScene> scenes;   // staged copies (emptied when a scene retires)
    std::vector<int> state;          // 0 free, 1 live, 2 staged (not placed yet)
    std::vector<Region> regions;
    std::vector<SceneDesc> descs;
    std::vector<int> bodies;         // body count of each slot's scene
    std::vector<int> dynamic;        // dynamic bodies of each slot's scene
    bool reserved = false;           // pools allocated
    Pools P;
    Allocs A;
    int* d_order = nullptr;          // live slots, largest first
    int* d_nlive = nullptr;
    int* d_queue = nullptr;
    int nlive = 0;
    bool order_dirty = true;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int threads = 0, ctas_per_sm = 0;   // 0 = automatic
    int group_rigid = 4, group_fem = 8;  // lanes per body in the primal sweep
    int variant = 1;                     // build of the persistent kernel (1..7, see kBatchVariants)
    int grid = 0;
    int stage = 0;   // float4 slots of dynamic shared memory per CTA
    int team_work = 0;   // bodies + tets per lane below which a CTA team splits (0 = never)
    int fem_team_work = 0;   // the same for scenes with tets
    int grid_min = 128;  // scenes from this many bodies use the grid broadphase (0 = never)
    std::vector<long long> steps_due;   // steps each slot's scene should have taken
    int* d_fail = nullptr;               // scene steps stopped by a full table (device counter)
    int* d_fix_order = nullptr;          // catch-up queue
    int* d_fix_n = nullptr;
    float last_ms = 0.f;
    // Scenes placed and staged into page-locked host buffers by
    // avbd_batch_prepare, copied to the pools by the next step.
    std::unique_ptr<StagedSink> upload;
    bool upload_pending = false;
    bool upload_pinned = false;   // the staging buffers are page-locked
    int64_t uploaded_bytes = 0;   // host-to-device bytes of the last staged upload
};

namespace {

void batch_drop_graph(AvbdBatch* b) {
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
}

int batch_stream(AvbdBatch* b) {
    int r = device_ready(b->device);
    if (r) return r;
    if (!b->stream) {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return AVBD_ERR_CUDA;
        cudaEventCreate(&b->e0);
        cudaEventCreate(&b->e1);
    }
    return 0;
}

// Allocates the pools with the given capacities (empty of scenes).
int batch_reserve(AvbdBatch* b, int64_t bodies, int64_t forces, int64_t tets, int64_t tris, int64_t nscenes,
                  int64_t nsinc, int64_t nsp) {
    int r = batch_stream(b);
    if (r) return r;
    const int64_t ncand = 16 * bodies + 64 * nscenes, nk = 8 * bodies + 128 * nscenes;
    const int64_t ninc = nsinc + 2 * ncand;
    const int64_t lim = 0x07FFFFFF;   // incidence entries index 27 bits
    if (bodies > lim || forces > lim || tets > lim || tris > lim || ncand > lim || nk > INT32_MAX || ninc > INT32_MAX ||
        nsinc > INT32_MAX || nscenes > (1 << 20))
        return AVBD_ERR_INVALID;
    Pools& P = b->P;
    P.release();
    P.ns = (int)nscenes; P.nb = (int)bodies; P.nf = (int)forces; P.nt = (int)tets; P.nr = (int)tris;
    P.ncand = (int)ncand; P.nk = (int)nk; P.nsinc = (int)nsinc; P.nsp = (int)nsp; P.ninc = (int)ninc;
    if (P.allocate_all() != cudaSuccess) {
        P.release();
        return AVBD_ERR_NOMEM;
    }
    P.W.P = to_params(b->params);
    b->A.reset(P);
    if (b->d_order) cudaFree(b->d_order);
    if (b->d_nlive) cudaFree(b->d_nlive);
    if (b->d_queue) cudaFree(b->d_queue);
    if (b->d_fail) cudaFree(b->d_fail);
    if (b->d_fix_order) cudaFree(b->d_fix_order);
    if (b->d_fix_n) cudaFree(b->d_fix_n);
    if (cudaMalloc(&b->d_order, std::max<int64_t>(nscenes, 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_nlive, sizeof(int)) != cudaSuccess || cudaMalloc(&b->d_queue, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_fail, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_fix_order, std::max<int64_t>(nscenes, 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_fix_n, sizeof(int)) != cudaSuccess)
        return AVBD_ERR_NOMEM;
    cudaMemset(b->d_fail, 0, sizeof(int));
    cudaMemset(b->d_nlive, 0, sizeof(int));
    b->reserved = true;
    b->order_dirty = true;
    batch_drop_graph(b);
    return 0;
}

// Takes pool ranges for the staged scene of `slot`; AVBD_ERR_NOMEM if the pools are full.
int batch_place(AvbdBatch* b, int slot) {
    if (slot >= b->P.ns) return AVBD_ERR_NOMEM;
    const HostScene& h = b->scenes[slot];
    int cc, kc, nsinc, nsp;
    scene_caps(h, cc, kc);
    static_counts(h, nsinc, nsp);
    Region reg;
    if (!place_scene(b->A, h, cc, kc, nsinc, nsp, reg)) return AVBD_ERR_NOMEM;
    b->regions[slot] = reg;
    return 0;
}

// Writes a placed scene through `sink` and marks it live.
template <typename Sink>
void batch_upload(AvbdBatch* b, int slot, Sink& sink) {
    const HostScene& h = b->scenes[slot];
    const Region& reg = b->regions[slot];
    upload_scene(b->P, h, static_incidence(h, reg), reg, scene_group(h, b->group_rigid, b->group_fem), slot,
                 b->descs[slot], sink);
}

// Places and uploads the staged scene of `slot` (live admission).
int batch_admit(AvbdBatch* b, int slot) {
    int r = batch_place(b, slot);
    if (r) return r;
    DirectSink sink{b->stream};
    batch_upload(b, slot, sink);
    b->state[slot] = 1;
    if ((int)b->steps_due.size() <= slot) b->steps_due.resize(slot + 1, 0);
    b->steps_due[slot] = 0;
    b->order_dirty = true;
    return 0;
}

// Uploads the live queue (largest scenes first) when it changed.
void batch_sync_order(AvbdBatch* b) {
    if (!b->order_dirty) return;
    std::vector<int> order;
    for (size_t i = 0; i < b->state.size(); ++i)
        if (b->state[i] == 1) order.push_back((int)i);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const SceneDesc& a = b->descs[x];
        const SceneDesc& c = b->descs[y];
        return (a.nbody + a.ntet) > (c.nbody + c.ntet);
    });
    b->nlive = (int)order.size();
    if (!order.empty())
        cudaMemcpyAsync(b->d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
    cudaMemcpyAsync(b->d_nlive, &b->nlive, sizeof(int), cudaMemcpyHostToDevice, b->stream);
    cudaStreamSynchronize(b->stream);
    b->order_dirty = false;
}

// First step without an explicit reservation: pools sized to the staged scenes.
// Reserves fresh pools for every staged scene, places them, and stages them
// into page-locked host buffers from all host threads (their ranges are
// disjoint); the copy waits for batch_flush.
int batch_stage(AvbdBatch* b, bool pin) {
    int64_t nb = 0, nf = 0, nt = 0, nr = 0, nsinc = 0, nsp = 0;
    for (size_t i = 0; i < b->scenes.size(); ++i) {
        if (b->state[i] != 2) continue;
        const HostScene& h = b->scenes[i];
        int a, c;
        static_counts(h, a, c);
        nb += h.nbody(); nf += h.nforce(); nt += h.ntet(); nr += h.ntri(); nsinc += a; nsp += c;
    }
    int r = batch_reserve(b, nb, nf, nt, nr, (int64_t)b->scenes.size(), nsinc, nsp);
    if (r) return r;
    std::vector<int> slots;
    for (size_t i = 0; i < b->scenes.size(); ++i)
        if (b->state[i] == 2) {
            if ((r = batch_place(b, (int)i))) return r;
            slots.push_back((int)i);
        }
    if (b->upload) b->upload->release();
    b->upload.reset(new StagedSink());
    StagedSink& staged = *b->upload;
    staged.st = b->stream;
    staged.P = &b->P;
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t k = next++; k < slots.size(); k = next++) batch_upload(b, slots[k], staged);
    };
    const unsigned nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nthreads && slots.size() > 64; ++t) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    if (staged.overflow) return AVBD_ERR_STATE;
    if (pin) staged.lock();
    b->upload_pinned = pin;
    for (int i : slots) {
        b->state[i] = 1;
        if ((int)b->steps_due.size() <= i) b->steps_due.resize(i + 1, 0);
        b->steps_due[i] = 0;
        b->scenes[i] = HostScene();   // the staged copy is what is uploaded
    }
    b->upload_pending = true;
    b->order_dirty = true;
    return cudaGetLastError() == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

// Copies the staged scenes into the pools (one copy per device array).
int batch_flush(AvbdBatch* b) {
    if (!b->upload_pending) return 0;
    b->upload_pending = false;
    if (!b->upload->flush()) return AVBD_ERR_STATE;
    b->uploaded_bytes = b->upload->copied;
    // pageable staging is not kept; page-locked staging (avbd_batch_prepare)
    // is held until the batch is destroyed, since unpinning it costs about as
    // much as the copy
    if (!b->upload_pinned) b->upload.reset();
    return cudaGetLastError() == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

int batch_launch_shape(AvbdBatch* b) {
    const BatchVariant& kv = kBatchVariants[b->variant];
    int threads = b->threads > 0 ? std::min(b->threads, kv.max_threads) : kv.max_threads;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    int per_sm = 0;
    const int stage = std::max(256, kStagedBodies * threads / 256);
    const size_t smem = stage * sizeof(float4);
    cudaFuncSetAttribute(kv.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kv.fn, threads, smem);
    if (per_sm < 1) per_sm = 1;
    if (b->ctas_per_sm > 0) per_sm = std::min(per_sm, b->ctas_per_sm);
    b->threads = threads;
    b->stage = stage;
    b->ctas_per_sm = per_sm;
    b->grid = sms * per_sm;
    return 0;
}

int batch_build_graph(AvbdBatch* b);

// Shifts the contact bases and live-slot entries of a relocated manifold table.
__global__ void k_rebase_table(const __grid_constant__ World W, int t, int cand0, int nslot, int nlive, int dk, int dc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nslot; i += gridDim.x * blockDim.x) {
        W.kbase[t][cand0 + i] += dk;
        if (i < nlive) W.live[t][cand0 + i] += dc;
    }
}

// Extends a pool's free ranges after the pool grew from old_cap to new_cap.
void ranges_extend(Ranges& rg, int old_cap, int new_cap) {
    if (new_cap <= old_cap) return;
    rg.cap = new_cap;
    rg.release(old_cap, new_cap - old_cap);
}

template <typename T>
void copy_range(T* base, int to, int from, int n, cudaStream_t st) {
    if (n > 0) cudaMemcpyAsync(base + to, base + from, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, st);
}

// Gives a scene stopped by a full candidate, contact or incidence table larger
// ranges (growing a pool when it has no room), moves its last completed
// manifold table and that table's contacts there, and clears the status so
// its step can run again.  The moved table is the one the next step warm
// starts from; the other table only held the interrupted attempt.
int batch_grow_scene(AvbdBatch* b, int slot, const SceneState& st) {
    Pools& P = b->P;
    Allocs& A = b->A;
    Region& r = b->regions[slot];
    SceneDesc& d = b->descs[slot];
    const int t = st.cur;
    const int nc = std::max(2 * r.ncand, st.need_cand + st.need_cand / 2 + 64);
    const int nk = std::max(2 * r.nk, st.need_k + st.need_k / 2 + 128);
    const int ni = r.nsinc + 2 * nc;
    int c0 = A.cand.alloc(nc), k0 = A.k.alloc(nk), i0 = A.inc.alloc(ni);
    if (c0 < 0 || k0 < 0 || i0 < 0) {
        if (c0 >= 0) A.cand.release(c0, nc);
        if (k0 >= 0) A.k.release(k0, nk);
        if (i0 >= 0) A.inc.release(i0, ni);
        // grow the pools, keeping every scene's contents
        cudaStreamSynchronize(b->stream);
        const int oc = P.ncand, ok = P.nk, oi = P.ninc;
        const int gc = std::max(oc + nc, oc + oc / 2), gk = std::max(ok + nk, ok + ok / 2);
        const int gi = std::max(oi + ni, oi + oi / 2);
        if (P.grow_tables(gc, gk, oc, oc, ok, ok) != cudaSuccess) return AVBD_ERR_NOMEM;
        if (P.grow(P.W.inc, (size_t)oi, (size_t)gi, (size_t)oi) != cudaSuccess) return AVBD_ERR_NOMEM;
        P.ninc = gi;
        ranges_extend(A.cand, oc, gc);
        ranges_extend(A.k, ok, gk);
        ranges_extend(A.inc, oi, gi);
        batch_drop_graph(b);   // the graph holds the old pool pointers
        c0 = A.cand.alloc(nc); k0 = A.k.alloc(nk); i0 = A.inc.alloc(ni);
        if (c0 < 0 || k0 < 0 || i0 < 0) return AVBD_ERR_NOMEM;
    }
    World& W = P.W;
    cudaStream_t s = b->stream;
    const int nslot = st.ncand[t], ncont = st.kused[t];
    copy_range(W.cpair[t], c0, r.cand0, nslot, s);
    copy_range(W.cn[t], c0, r.cand0, nslot, s);
    copy_range(W.cfric[t], c0, r.cand0, nslot, s);
    copy_range(W.kbase[t], c0, r.cand0, nslot, s);
    copy_range(W.cbirth[t], c0, r.cand0, nslot, s);
    copy_range(W.live[t], c0, r.cand0, nslot, s);
    copy_range(W.kid[t], k0, r.k0, ncont, s);
    copy_range(W.krA[t], k0, r.k0, ncont, s);
    copy_range(W.krB[t], k0, r.k0, ncont, s);
    copy_range(W.kn[t], k0, r.k0, ncont, s);
    copy_range(W.kt1[t], k0, r.k0, ncont, s);
    copy_range(W.kt2[t], k0, r.k0, ncont, s);
    copy_range(W.krAw[t], k0, r.k0, ncont, s);
    copy_range(W.krBw[t], k0, r.k0, ncont, s);
    copy_range(W.kpen[t], k0, r.k0, ncont, s);
    copy_range(W.klam[t], k0, r.k0, ncont, s);
    if (nslot > 0)
        k_rebase_table<<<blocks_for(nslot), kThreads, 0, s>>>(W, t, c0, nslot, st.nlive[t], k0 - r.k0, c0 - r.cand0);
    A.cand.release(r.cand0, r.ncand);
    A.k.release(r.k0, r.nk);
    A.inc.release(r.inc0, r.ninc);
    r.cand0 = c0; r.ncand = nc; r.k0 = k0; r.nk = nk; r.inc0 = i0; r.ninc = ni;
    d.cand0 = c0; d.candcap = nc; d.k0 = k0; d.kcap = nk; d.inc0 = i0; d.inccap = ni;
    SceneState fixed = st;
    fixed.status = kStatusOk;
    fixed.need_cand = fixed.need_k = fixed.need_inc = 0;
    cudaMemcpyAsync(P.d_scenes + slot, &d, sizeof(SceneDesc), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(P.d_sstate + slot, &fixed, sizeof(SceneState), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    return 0;
}

// Runs one step of the listed scenes only (same kernel build and launch shape).
int batch_step_listed(AvbdBatch* b, const std::vector<int>& slots) {
    const int n = (int)slots.size();
    cudaStream_t s = b->stream;
    cudaMemcpyAsync(b->d_fix_order, slots.data(), n * sizeof(int), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(b->d_fix_n, &n, sizeof(int), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(b->d_queue, 0, sizeof(int), s);
    World W = b->P.W;
    W.stage_bodies = b->stage;
    W.team_work = b->team_work;
    W.fem_team_work = b->fem_team_work;
    W.grid_min = b->grid_min;
    W.fail_count = b->d_fail;
    const int* order = b->d_fix_order;
    const int* nlive = b->d_fix_n;
    int* queue = b->d_queue;
    void* args[] = {&W, &order, &nlive, &queue};
    if (cudaLaunchKernel((const void*)kBatchVariants[b->variant].fn, dim3(b->grid), dim3(b->threads), args,
                         (size_t)b->stage * sizeof(float4), s) != cudaSuccess)
        return AVBD_ERR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

// After a batched step: scenes a full table stopped get larger tables and
// take the steps they missed (a few rounds, in case one growth is not enough).
int batch_fix_capacity(AvbdBatch* b) {
    const int nslots = (int)b->state.size();
    std::vector<SceneState> hs(nslots);
    for (int round = 0; round < 4; ++round) {
        int fails = 0;
        cudaMemcpy(&fails, b->d_fail, sizeof(int), cudaMemcpyDeviceToHost);
        if (fails == 0) return 0;
        cudaMemset(b->d_fail, 0, sizeof(int));
        if (cudaMemcpy(hs.data(), b->P.d_sstate, nslots * sizeof(SceneState), cudaMemcpyDeviceToHost) != cudaSuccess)
            return AVBD_ERR_CUDA;
        std::vector<int> grown;
        for (int i = 0; i < nslots; ++i) {
            if (b->state[i] != 1 || hs[i].status != kStatusCapacity) continue;
            if (!(hs[i].need_cand || hs[i].need_k || hs[i].need_inc)) continue;   // colour slots: not growable
            if (batch_grow_scene(b, i, hs[i]) == 0) grown.push_back(i);
        }
        if (grown.empty()) return 0;
        if (!b->graph) batch_build_graph(b);
        // catch up: every grown scene takes the steps it missed
        for (;;) {
            std::vector<int> due;
            if (cudaMemcpy(hs.data(), b->P.d_sstate, nslots * sizeof(SceneState), cudaMemcpyDeviceToHost) !=
                cudaSuccess)
                return AVBD_ERR_CUDA;
            for (int i : grown)
                if (hs[i].status == kStatusOk && hs[i].step < b->steps_due[i]) due.push_back(i);
            if (due.empty()) break;
            int r = batch_step_listed(b, due);
            if (r) return r;
        }
    }
    return 0;
}

int batch_build_graph(AvbdBatch* b) {
    batch_drop_graph(b);
    cudaGraph_t g;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return AVBD_ERR_CUDA;
    cudaMemsetAsync(b->d_queue, 0, sizeof(int), b->stream);
    b->P.W.stage_bodies = b->stage;
    b->P.W.team_work = b->team_work;
    b->P.W.fem_team_work = b->fem_team_work;
    b->P.W.grid_min = b->grid_min;
    b->P.W.fail_count = b->d_fail;
    const size_t smem = (size_t)b->stage * sizeof(float4);
    {
        const int* order = b->d_order;
        const int* nlive = b->d_nlive;
        int* queue = b->d_queue;
        void* args[] = {&b->P.W, &order, &nlive, &queue};
        cudaLaunchKernel((const void*)kBatchVariants[b->variant].fn, dim3(b->grid), dim3(b->threads), args, smem,
                         b->stream);
    }
    if (cudaStreamEndCapture(b->stream, &g) != cudaSuccess) return AVBD_ERR_CUDA;
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    return e == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

}  // namespace

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

void avbd_default_params(AvbdParams* p) {
    if (!p) return;
    p->num_iterations = 10;
    p->step_value = 1.0f / 60.0f;
    p->alpha = 0.95f;
    p->beta = 100000.0f;
    p->gamma = 0.99f;
    p->on_penetration_penalty = 0.f;
    p->post_stabilization = 1;
    p->projection_mode = AVBD_PROJECT_ABSOLUTE;
    p->trust_region_rho = 0.f;
}

const char* avbd_status_string(int32_t code) {
    switch (code) {
        case AVBD_STATUS_OK: return "ok";
        case AVBD_STATUS_EXPLODED: return "exploded";
        case AVBD_STATUS_NAN: return "nan";
        case AVBD_STATUS_CAPACITY: return "capacity";
        case AVBD_STATUS_TIMEOUT: return "timeout";
        case AVBD_ERR_INVALID: return "invalid argument";
        case AVBD_ERR_CUDA: return "cuda error";
        case AVBD_ERR_NOMEM: return "out of memory";
        case AVBD_ERR_STATE: return "invalid state";
        case AVBD_ERR_NODEVICE: return "no cuda device";
        default: return "unknown";
    }
}

int32_t avbd_world_create(const AvbdParams* params, int32_t device, AvbdWorld** out) {
    if (!out) return AVBD_ERR_INVALID;
    AvbdParams p;
    avbd_default_params(&p);
    if (params) {
        if (!valid_params(params)) return AVBD_ERR_INVALID;
        p = *params;
    }
    int r = device_ready(device);
    if (r) return r;
    AvbdWorld* w = new (std::nothrow) AvbdWorld();
    if (!w) return AVBD_ERR_NOMEM;
    w->params = p;
    w->device = device;
    *out = w;
    return 0;
}

int32_t avbd_world_destroy(AvbdWorld* w) {
    if (!w) return AVBD_ERR_INVALID;
    cudaSetDevice(w->device);
    if (w->stream) {
        cudaStreamSynchronize(w->stream);
        for (auto& e : w->ev) cudaEventDestroy(e);
        cudaStreamDestroy(w->stream);
    }
    delete w;
    return 0;
}

int32_t avbd_world_clear(AvbdWorld* w) {
    if (!w) return AVBD_ERR_INVALID;
    w->h.clear();
    w->P.release();
    w->uploaded = false;
    w->stopped = false;
    return 0;
}

int32_t avbd_set_params(AvbdWorld* w, const AvbdParams* p) {
    if (!w || !valid_params(p)) return AVBD_ERR_INVALID;
    w->params = *p;
    return 0;
}

int32_t avbd_get_params(const AvbdWorld* w, AvbdParams* out) {
    if (!w || !out) return AVBD_ERR_INVALID;
    *out = w->params;
    return 0;
}

#define AVBD_STAGING_ONLY(w) \
    if (!(w)) return AVBD_ERR_INVALID; \
    if ((w)->uploaded) return AVBD_ERR_STATE;

int32_t avbd_add_body(AvbdWorld* w, int32_t model, float density, float friction, const float pos[3],
                      const float scale[3], const float vel[3], const float quat[4], const float omega[3],
                      int32_t is_static) {
    AVBD_STAGING_ONLY(w);
    if (!pos || !scale || !vel || !quat || !omega || model < 0 || model > 2) return AVBD_ERR_INVALID;
    return w->h.add_body(model, density, friction, pos, scale, vel, quat, omega, is_static != 0);
}

int32_t avbd_add_bodies(AvbdWorld* w, int32_t n, int32_t model, const float* density, const float* friction,
                        const float* pos, const float* scale, const float* vel, const float* quat, const float* omega,
                        const int32_t* is_static) {
    AVBD_STAGING_ONLY(w);
    if (n < 0 || !density || !friction || !pos || !scale || !quat || !is_static || model < 0 || model > 2)
        return AVBD_ERR_INVALID;
    const float zero[3] = {0.f, 0.f, 0.f};
    const int first = w->h.nbody();
    for (int i = 0; i < n; ++i)
        w->h.add_body(model, density[i], friction[i], pos + 3 * i, scale + 3 * i, vel ? vel + 3 * i : zero,
                      quat + 4 * i, omega ? omega + 3 * i : zero, is_static[i] != 0);
    return first;
}

int32_t avbd_add_particle(AvbdWorld* w, float mass, float friction, const float pos[3], const float vel[3],
                          int32_t is_static) {
    AVBD_STAGING_ONLY(w);
    if (!pos || !vel) return AVBD_ERR_INVALID;
    return w->h.add_particle(mass, friction, pos, vel, is_static != 0);
}

int32_t avbd_set_body_static(AvbdWorld* w, int32_t body, int32_t is_static) {
    AVBD_STAGING_ONLY(w);
    return w->h.set_static(body, is_static != 0) ? AVBD_ERR_INVALID : 0;
}

int32_t avbd_add_spring(AvbdWorld* w, int32_t a, const float rA[3], int32_t b, const float rB[3], float k,
                        float rest, int32_t is_rope, float fracture) {
    AVBD_STAGING_ONLY(w);
    if (!rA || !rB) return AVBD_ERR_INVALID;
    int r = w->h.add_spring(a, rA, b, rB, k, rest, is_rope != 0, fracture);
    return r < 0 ? AVBD_ERR_INVALID : r;
}

int32_t avbd_add_joint(AvbdWorld* w, int32_t a, const float rA[3], int32_t b, const float rB[3],
                       const float stiffness[6], const float fracture[6]) {
    AVBD_STAGING_ONLY(w);
    if (!rA || !rB || !stiffness || !fracture) return AVBD_ERR_INVALID;
    int r = w->h.add_joint(a, rA, b, rB, stiffness, fracture);
    return r < 0 ? AVBD_ERR_INVALID : r;
}

int32_t avbd_add_neohookean_tet(AvbdWorld* w, const int32_t v[4], float E, float nu) {
    AVBD_STAGING_ONLY(w);
    if (!v) return AVBD_ERR_INVALID;
    int r = w->h.add_nh_tet(v, E, nu);
    return r < 0 ? AVBD_ERR_INVALID : r;
}

int32_t avbd_add_stvk_tri(AvbdWorld* w, const int32_t v[3], float E, float nu) {
    AVBD_STAGING_ONLY(w);
    if (!v) return AVBD_ERR_INVALID;
    int r = w->h.add_stvk_tri(v, E, nu);
    return r < 0 ? AVBD_ERR_INVALID : r;
}

// ---- snapshot / restore of a stepped world: every device allocation of the
// world byte for byte (bodies, forces, energies, both manifold tables and
// their contacts, incidence, colour lists and counters) after a header. ----
struct SnapshotHeader {
    uint32_t magic;     // 'AVSN'
    uint32_t version;
    int32_t nalloc;
    int32_t stopped;
    int64_t total;
};
constexpr uint32_t kSnapshotMagic = 0x4e535641u;

static int64_t snapshot_bytes(const AvbdWorld* w) {
    int64_t n = sizeof(SnapshotHeader) + (int64_t)w->P.owned_bytes.size() * sizeof(int64_t);
    for (size_t b : w->P.owned_bytes) n += (int64_t)b;
    return n;
}

int64_t avbd_snapshot_bytes(const AvbdWorld* w) {
    if (!w) return AVBD_ERR_INVALID;
    if (!w->uploaded) return AVBD_ERR_STATE;
    return snapshot_bytes(w);
}

int32_t avbd_snapshot(AvbdWorld* w, void* dst, int64_t bytes) {
    if (!w || !dst) return AVBD_ERR_INVALID;
    if (!w->uploaded) return AVBD_ERR_STATE;
    if (bytes < snapshot_bytes(w)) return AVBD_ERR_INVALID;
    if (cudaSetDevice(w->device) != cudaSuccess) return AVBD_ERR_CUDA;
    const Pools& P = w->P;
    std::vector<char> head(sizeof(SnapshotHeader) + P.owned_bytes.size() * sizeof(int64_t));
    SnapshotHeader h{kSnapshotMagic, 1u, (int32_t)P.owned.size(), w->stopped ? 1 : 0, snapshot_bytes(w)};
    std::memcpy(head.data(), &h, sizeof(h));
    for (size_t i = 0; i < P.owned_bytes.size(); ++i) {
        const int64_t b = (int64_t)P.owned_bytes[i];
        std::memcpy(head.data() + sizeof(h) + i * sizeof(int64_t), &b, sizeof(b));
    }
    char* out = static_cast<char*>(dst);
    if (cudaMemcpyAsync(out, head.data(), head.size(), cudaMemcpyDefault, w->stream) != cudaSuccess)
        return AVBD_ERR_CUDA;
    size_t off = head.size();
    for (size_t i = 0; i < P.owned.size(); ++i) {
        if (cudaMemcpyAsync(out + off, P.owned[i], P.owned_bytes[i], cudaMemcpyDefault, w->stream) != cudaSuccess)
            return AVBD_ERR_CUDA;
        off += P.owned_bytes[i];
    }
    return cudaStreamSynchronize(w->stream) == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

int32_t avbd_restore(AvbdWorld* w, const void* src, int64_t bytes) {
    if (!w || !src) return AVBD_ERR_INVALID;
    if (!w->uploaded) return AVBD_ERR_STATE;
    if (cudaSetDevice(w->device) != cudaSuccess) return AVBD_ERR_CUDA;
    Pools& P = w->P;
    const char* in = static_cast<const char*>(src);
    SnapshotHeader h{};
    if (bytes < (int64_t)sizeof(h)) return AVBD_ERR_INVALID;
    if (cudaMemcpy(&h, in, sizeof(h), cudaMemcpyDefault) != cudaSuccess) return AVBD_ERR_CUDA;
    if (h.magic != kSnapshotMagic || h.version != 1u || bytes < h.total) return AVBD_ERR_INVALID;
    // the world's tables must have the sizes they had when the snapshot was taken
    if (h.nalloc != (int32_t)P.owned.size() || h.total != snapshot_bytes(w)) return AVBD_ERR_STATE;
    std::vector<int64_t> sizes(h.nalloc);
    if (cudaMemcpy(sizes.data(), in + sizeof(h), sizes.size() * sizeof(int64_t), cudaMemcpyDefault) != cudaSuccess)
        return AVBD_ERR_CUDA;
    for (size_t i = 0; i < sizes.size(); ++i)
        if (sizes[i] != (int64_t)P.owned_bytes[i]) return AVBD_ERR_STATE;
    size_t off = sizeof(h) + sizes.size() * sizeof(int64_t);
    for (size_t i = 0; i < P.owned.size(); ++i) {
        if (cudaMemcpyAsync(P.owned[i], in + off, P.owned_bytes[i], cudaMemcpyDefault, w->stream) != cudaSuccess)
            return AVBD_ERR_CUDA;
        off += P.owned_bytes[i];
    }
    if (cudaStreamSynchronize(w->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    w->stopped = h.stopped != 0;
    return sync_state(w);
}

// kind 0 body, 1 force, 2 tet, 3 triangle (see k_remove_item).
static int32_t world_remove(AvbdWorld* w, int kind, int32_t id) {
    if (!w) return AVBD_ERR_INVALID;
    HostScene& h = w->h;
    const int n = kind == 0 ? h.nbody() : kind == 1 ? h.nforce() : kind == 2 ? h.ntet() : h.ntri();
    if (id < 0 || id >= n) return AVBD_ERR_INVALID;
    if (!w->uploaded) {
        if (kind == 0) {
            h.flags[id] |= kBodyRemoved;
            for (int f = 0; f < h.nforce(); ++f)
                if (h.fbody[f].x == id || h.fbody[f].y == id) h.ftype[f] |= kForceRemoved;
            for (int t = 0; t < h.ntet(); ++t) {
                const int4 v = h.tidx[t];
                if (v.x == id || v.y == id || v.z == id || v.w == id) h.tparam[t].w = 1.f;
            }
            for (int t = 0; t < h.ntri(); ++t) {
                const int4 v = h.ridx[t];
                if (v.x == id || v.y == id || v.z == id) h.rparam[t].w = 1.f;
            }
        } else if (kind == 1) {
            h.ftype[id] |= kForceRemoved;
        } else if (kind == 2) {
            h.tparam[id].w = 1.f;
        } else {
            h.rparam[id].w = 1.f;
        }
        return 0;
    }
    if (cudaSetDevice(w->device) != cudaSuccess) return AVBD_ERR_CUDA;
    const SceneDesc& d = w->descs[0];
    const int base = kind == 0 ? d.body0 : kind == 1 ? d.force0 : kind == 2 ? d.tet0 : d.tri0;
    k_remove_item<<<1, 32, 0, w->stream>>>(w->P.W, kind, base + id);
    return cudaStreamSynchronize(w->stream) == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

int32_t avbd_remove_body(AvbdWorld* w, int32_t body) { return world_remove(w, 0, body); }
int32_t avbd_remove_force(AvbdWorld* w, int32_t force) { return world_remove(w, 1, force); }
int32_t avbd_remove_neohookean_tet(AvbdWorld* w, int32_t tet) { return world_remove(w, 2, tet); }
int32_t avbd_remove_stvk_tri(AvbdWorld* w, int32_t tri) { return world_remove(w, 3, tri); }

int32_t avbd_add_stvk_tet(AvbdWorld* w, const int32_t v[4], float E, float nu) {
    AVBD_STAGING_ONLY(w);
    if (!v) return AVBD_ERR_INVALID;
    int r = w->h.add_stvk_tet(v, E, nu);
    return r < 0 ? AVBD_ERR_INVALID : r;
}

int32_t avbd_make_stvk_tet_volume(AvbdWorld* w, float ox, float oy, float oz, int32_t nx, int32_t ny, int32_t nz,
                                  float cell, float E, float nu, float pm, float friction, int32_t pin) {
    AVBD_STAGING_ONLY(w);
    int r = w->h.make_tet_volume(ox, oy, oz, nx, ny, nz, cell, E, nu, pm, friction, pin != 0, kTetStvk);
    return r < 0 ? AVBD_ERR_INVALID : r;
}

int32_t avbd_make_tet_volume(AvbdWorld* w, float ox, float oy, float oz, int32_t nx, int32_t ny, int32_t nz,
                             float cell, float E, float nu, float pm, float friction, int32_t pin) {
    AVBD_STAGING_ONLY(w);
    int r = w->h.make_tet_volume(ox, oy, oz, nx, ny, nz, cell, E, nu, pm, friction, pin != 0);
    return r < 0 ? AVBD_ERR_INVALID : r;
}

int32_t avbd_step(AvbdWorld* w) {
    if (!w) return AVBD_ERR_INVALID;
    return world_step(w);
}

int32_t avbd_step_dt(AvbdWorld* w, float dt, int32_t iterations) {
    if (!w || !(dt > 0.f) || iterations < 0) return AVBD_ERR_INVALID;
    w->params.step_value = dt;
    w->params.num_iterations = iterations;
    return world_step(w);
}

int32_t avbd_num_bodies(const AvbdWorld* w) { return w ? w->h.nbody() : AVBD_ERR_INVALID; }
int32_t avbd_num_dynamic_bodies(const AvbdWorld* w) { return w ? w->h.ndynamic() : AVBD_ERR_INVALID; }
int32_t avbd_emergency_stop(const AvbdWorld* w) { return w ? (w->stopped ? 1 : 0) : AVBD_ERR_INVALID; }

int32_t avbd_get_state(AvbdWorld* w, float* pos, float* quat, float* vel, float* omega) {
    if (!w) return AVBD_ERR_INVALID;
    const int n = w->h.nbody();
    if (!w->uploaded) {
        for (int i = 0; i < n; ++i) {
            const float4 p = w->h.pos[i], q = w->h.rot[i], v = w->h.vel[i], o = w->h.omega[i];
            if (pos) { pos[3 * i] = p.x; pos[3 * i + 1] = p.y; pos[3 * i + 2] = p.z; }
            if (quat) { quat[4 * i] = q.w; quat[4 * i + 1] = q.x; quat[4 * i + 2] = q.y; quat[4 * i + 3] = q.z; }
            if (vel) { vel[3 * i] = v.x; vel[3 * i + 1] = v.y; vel[3 * i + 2] = v.z; }
            if (omega) { omega[3 * i] = o.x; omega[3 * i + 1] = o.y; omega[3 * i + 2] = o.z; }
        }
        return n;
    }
    cudaSetDevice(w->device);
    std::vector<float4> buf(n);
    const World& W = w->P.W;
    auto fetch = [&](const float4* src, float* dst, int comps, bool quat_order) -> int {
        if (!dst) return 0;
        if (cudaMemcpy(buf.data(), src, n * sizeof(float4), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
        for (int i = 0; i < n; ++i) {
            const float4 x = buf[i];
            if (quat_order) { dst[4 * i] = x.w; dst[4 * i + 1] = x.x; dst[4 * i + 2] = x.y; dst[4 * i + 3] = x.z; }
            else { dst[comps * i] = x.x; dst[comps * i + 1] = x.y; dst[comps * i + 2] = x.z; }
        }
        return 0;
    };
    if (fetch(W.pos, pos, 3, false) || fetch(W.rot, quat, 4, true) || fetch(W.vel, vel, 3, false) ||
        fetch(W.omega, omega, 3, false))
        return AVBD_ERR_CUDA;
    // a removed body (RemoveBody or out of bounds) has no state: it reads NaN
    std::vector<int> fl(n);
    if (n > 0 && cudaMemcpy(fl.data(), W.flags, n * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return AVBD_ERR_CUDA;
    const float nan = std::numeric_limits<float>::quiet_NaN();
    for (int i = 0; i < n; ++i) {
        if (!(fl[i] & kBodyRemoved)) continue;
        for (int k = 0; k < 3; ++k) {
            if (pos) pos[3 * i + k] = nan;
            if (vel) vel[3 * i + k] = nan;
            if (omega) omega[3 * i + k] = nan;
        }
        if (quat) for (int k = 0; k < 4; ++k) quat[4 * i + k] = nan;
    }
    return n;
}

int32_t avbd_force_live(AvbdWorld* w, int32_t force) {
    if (!w || force < 0 || force >= w->h.nforce()) return AVBD_ERR_INVALID;
    int t = w->h.ftype[force];
    if (w->uploaded) {
        cudaSetDevice(w->device);
        if (cudaMemcpy(&t, w->P.W.ftype + force, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
            return AVBD_ERR_CUDA;
    }
    return (t & (kForceDisabled | kForceRemoved)) ? 0 : 1;
}

int32_t avbd_set_state(AvbdWorld* w, const float* pos, const float* quat, const float* vel, const float* omega) {
    if (!w) return AVBD_ERR_INVALID;
    const int n = w->h.nbody();
    for (int i = 0; i < n; ++i) {
        if (pos) { w->h.pos[i].x = pos[3 * i]; w->h.pos[i].y = pos[3 * i + 1]; w->h.pos[i].z = pos[3 * i + 2]; }
        if (quat) {
            w->h.rot[i].w = quat[4 * i]; w->h.rot[i].x = quat[4 * i + 1];
            w->h.rot[i].y = quat[4 * i + 2]; w->h.rot[i].z = quat[4 * i + 3];
        }
        if (vel) { w->h.vel[i].x = vel[3 * i]; w->h.vel[i].y = vel[3 * i + 1]; w->h.vel[i].z = vel[3 * i + 2]; }
        if (omega) {
            w->h.omega[i].x = omega[3 * i]; w->h.omega[i].y = omega[3 * i + 1]; w->h.omega[i].z = omega[3 * i + 2];
        }
    }
    if (w->uploaded) {
        cudaSetDevice(w->device);
        const World& W = w->P.W;
        if (pos) cudaMemcpy(W.pos, w->h.pos.data(), n * sizeof(float4), cudaMemcpyHostToDevice);
        if (quat) cudaMemcpy(W.rot, w->h.rot.data(), n * sizeof(float4), cudaMemcpyHostToDevice);
        if (vel) cudaMemcpy(W.vel, w->h.vel.data(), n * sizeof(float4), cudaMemcpyHostToDevice);
        if (omega) cudaMemcpy(W.omega, w->h.omega.data(), n * sizeof(float4), cudaMemcpyHostToDevice);
    }
    return 0;
}

int32_t avbd_get_contacts(AvbdWorld* w, int32_t max, int32_t* pairs, int32_t* counts, uint32_t* ids, float* data) {
    if (!w) return AVBD_ERR_INVALID;
    if (!w->uploaded) return 0;
    cudaSetDevice(w->device);
    SceneState st;
    cudaMemcpy(&st, w->P.d_sstate, sizeof(SceneState), cudaMemcpyDeviceToHost);
    const int cur = st.cur, nc = st.ncand[cur];
    const World& W = w->P.W;
    std::vector<int2> cp(nc);
    std::vector<int> cn(nc), kb(nc);
    cudaMemcpy(cp.data(), W.cpair[cur], nc * sizeof(int2), cudaMemcpyDeviceToHost);
    cudaMemcpy(cn.data(), W.cn[cur], nc * sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(kb.data(), W.kbase[cur], nc * sizeof(int), cudaMemcpyDeviceToHost);
    const int nk = st.kused[cur];
    std::vector<uint32_t> kid(nk);
    std::vector<float4> rA(nk), rB(nk), kn(nk), pen(nk), lam(nk);
    if (nk > 0) {
        cudaMemcpy(kid.data(), W.kid[cur], nk * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(rA.data(), W.krA[cur], nk * sizeof(float4), cudaMemcpyDeviceToHost);
        cudaMemcpy(rB.data(), W.krB[cur], nk * sizeof(float4), cudaMemcpyDeviceToHost);
        cudaMemcpy(kn.data(), W.kn[cur], nk * sizeof(float4), cudaMemcpyDeviceToHost);
        cudaMemcpy(pen.data(), W.kpen[cur], nk * sizeof(float4), cudaMemcpyDeviceToHost);
        cudaMemcpy(lam.data(), W.klam[cur], nk * sizeof(float4), cudaMemcpyDeviceToHost);
    }
    int m = 0;
    for (int c = 0; c < nc; ++c) {
        if (cn[c] == 0) continue;
        if (m < max) {
            if (pairs) { pairs[2 * m] = cp[c].x; pairs[2 * m + 1] = cp[c].y; }
            if (counts) counts[m] = cn[c];
            for (int k = 0; k < 8; ++k) {
                if (ids) ids[8 * m + k] = k < cn[c] ? kid[kb[c] + k] : 0xFFFFFFFFu;
                if (data) {
                    float* d = data + (size_t)(8 * m + k) * 16;
                    std::memset(d, 0, 16 * sizeof(float));
                    if (k < cn[c]) {
                        const int o = kb[c] + k;
                        d[0] = rA[o].w;
                        d[1] = -kn[o].x; d[2] = -kn[o].y; d[3] = -kn[o].z;
                        d[4] = rA[o].x; d[5] = rA[o].y; d[6] = rA[o].z;
                        d[7] = rB[o].x; d[8] = rB[o].y; d[9] = rB[o].z;
                        d[10] = pen[o].x; d[11] = pen[o].y; d[12] = pen[o].z;
                        d[13] = lam[o].x; d[14] = lam[o].y; d[15] = lam[o].z;
                    }
                }
            }
        }
        ++m;
    }
    return m;
}

int32_t avbd_get_colours(AvbdWorld* w, int32_t* colours) {
    if (!w || !colours) return AVBD_ERR_INVALID;
    const int n = w->h.nbody();
    if (!w->uploaded) {
        for (int i = 0; i < n; ++i) colours[i] = -1;
        return 0;
    }
    cudaSetDevice(w->device);
    cudaMemcpy(colours, w->P.W.colour, n * sizeof(int), cudaMemcpyDeviceToHost);
    for (int i = 0; i < n; ++i) if (colours[i] < 0) colours[i] = -1;
    return w->ncolours;
}

int32_t avbd_get_timings(const AvbdWorld* w, AvbdTimings* out) {
    if (!w || !out) return AVBD_ERR_INVALID;
    *out = w->timings;
    return 0;
}

int32_t avbd_collide(AvbdWorld* w, int32_t a, int32_t b, uint32_t* ids, float* data) {
    if (!w || a < 0 || b < 0 || a >= w->h.nbody() || b >= w->h.nbody()) return AVBD_ERR_INVALID;
    if (!w->uploaded) {
        int r = upload(w);
        if (r) return r;
    }
    cudaSetDevice(w->device);
    uint32_t* d_ids = nullptr;
    float* d_data = nullptr;
    int* d_n = nullptr;
    cudaMalloc(&d_ids, 8 * sizeof(uint32_t));
    cudaMalloc(&d_data, 8 * 13 * sizeof(float));
    cudaMalloc(&d_n, sizeof(int));
    k_collide<<<1, 32, 0, w->stream>>>(w->P.W, a, b, d_ids, d_data, d_n);
    int n = 0;
    cudaStreamSynchronize(w->stream);
    cudaMemcpy(&n, d_n, sizeof(int), cudaMemcpyDeviceToHost);
    if (ids) cudaMemcpy(ids, d_ids, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (data) cudaMemcpy(data, d_data, 8 * 13 * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d_ids);
    cudaFree(d_data);
    cudaFree(d_n);
    return cudaGetLastError() == cudaSuccess ? n : AVBD_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Batch
// ---------------------------------------------------------------------------
int32_t avbd_batch_create(const AvbdParams* params, int32_t device, AvbdBatch** out) {
    if (!out) return AVBD_ERR_INVALID;
    AvbdParams p;
    avbd_default_params(&p);
    if (params) {
        if (!valid_params(params)) return AVBD_ERR_INVALID;
        p = *params;
    }
    int r = device_ready(device);
    if (r) return r;
    AvbdBatch* b = new (std::nothrow) AvbdBatch();
    if (!b) return AVBD_ERR_NOMEM;
    b->params = p;
    b->device = device;
    *out = b;
    return 0;
}

int32_t avbd_batch_destroy(AvbdBatch* b) {
    if (!b) return AVBD_ERR_INVALID;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    if (b->upload) b->upload->release();
    if (b->d_order) cudaFree(b->d_order);
    if (b->d_nlive) cudaFree(b->d_nlive);
    if (b->d_queue) cudaFree(b->d_queue);
    if (b->d_fail) cudaFree(b->d_fail);
    if (b->d_fix_order) cudaFree(b->d_fix_order);
    if (b->d_fix_n) cudaFree(b->d_fix_n);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return 0;
}

int32_t avbd_batch_reserve(AvbdBatch* b, int64_t bodies, int64_t forces, int64_t tets, int64_t tris, int32_t scenes) {
    if (!b || bodies < 0 || forces < 0 || tets < 0 || tris < 0 || scenes < 1) return AVBD_ERR_INVALID;
    if (b->reserved) return AVBD_ERR_STATE;
    int r = batch_reserve(b, bodies, forces, tets, tris, scenes, 2 * forces + 4 * tets + 3 * tris, 2 * forces);
    if (r) return r;
    for (size_t i = 0; i < b->scenes.size(); ++i)
        if (b->state[i] == 2 && (r = batch_admit(b, (int)i))) return r;
    return 0;
}

// Scenes staged by avbd_batch_prepare reach the device with the first step;
// every entry point that reads device state or hands out pool space first
// completes that copy, so it never acts on unwritten memory and a later copy
// never overwrites a range given to another scene.
static int batch_settle(AvbdBatch* b) {
    if (!b->upload_pending) return 0;
    if (cudaSetDevice(b->device) != cudaSuccess) return AVBD_ERR_CUDA;
    return batch_flush(b);
}

int32_t avbd_batch_add_scene(AvbdBatch* b, const AvbdWorld* w) {
    if (!b || !w) return AVBD_ERR_INVALID;
    if (int r = batch_settle(b)) return r;
    int slot = -1;
    for (size_t i = 0; i < b->state.size(); ++i)
        if (b->state[i] == 0) { slot = (int)i; break; }
    if (slot < 0) {
        if (b->reserved && (int)b->state.size() >= b->P.ns) return AVBD_ERR_NOMEM;
        slot = (int)b->state.size();
        b->scenes.emplace_back();
        b->state.push_back(0);
        b->regions.emplace_back();
        b->descs.emplace_back();
        b->bodies.push_back(0);
        b->dynamic.push_back(0);
    }
    b->scenes[slot] = w->h;
    b->bodies[slot] = w->h.nbody();
    b->dynamic[slot] = w->h.ndynamic();
    b->state[slot] = 2;
    if (b->reserved) {
        cudaSetDevice(b->device);
        int r = batch_admit(b, slot);
        if (r) {   // no room in the pools: nothing was placed
            b->scenes[slot] = HostScene();
            b->state[slot] = 0;
            return r;
        }
        b->scenes[slot] = HostScene();   // the device holds it now
    }
    return slot;
}

int32_t avbd_batch_remove_scene(AvbdBatch* b, int32_t scene) {
    if (!b || scene < 0 || scene >= (int)b->state.size() || b->state[scene] == 0) return AVBD_ERR_INVALID;
    if (int r = batch_settle(b)) return r;
    if (b->state[scene] == 1) {
        b->A.release(b->regions[scene]);
        b->order_dirty = true;
    }
    b->state[scene] = 0;
    b->scenes[scene] = HostScene();
    b->bodies[scene] = 0;
    b->dynamic[scene] = 0;
    return 0;
}

int32_t avbd_batch_prepare(AvbdBatch* b) {
    if (!b) return AVBD_ERR_INVALID;
    if (b->reserved) return 0;
    int r = batch_stage(b, true);
    if (r) return r;
    cudaSetDevice(b->device);
    if (!b->grid) batch_launch_shape(b);
    return cudaGetLastError() == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

int32_t avbd_batch_step(AvbdBatch* b, int32_t steps) {
    if (!b || steps < 0) return AVBD_ERR_INVALID;
    int r;
    if (!b->reserved && (r = batch_stage(b, false))) return r;
    cudaSetDevice(b->device);
    if ((r = batch_flush(b))) return r;
    batch_sync_order(b);
    if (!b->grid) batch_launch_shape(b);
    b->P.W.P = to_params(b->params);
    if (!b->graph && (r = batch_build_graph(b))) return r;
    cudaMemsetAsync(b->d_fail, 0, sizeof(int), b->stream);
    cudaEventRecord(b->e0, b->stream);
    for (int i = 0; i < steps; ++i)
        if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    cudaEventRecord(b->e1, b->stream);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    cudaEventElapsedTime(&b->last_ms, b->e0, b->e1);
    if (cudaGetLastError() != cudaSuccess) return AVBD_ERR_CUDA;
    for (size_t i = 0; i < b->state.size() && i < b->steps_due.size(); ++i)
        if (b->state[i] == 1) b->steps_due[i] += steps;
    if ((r = batch_fix_capacity(b))) return r;
    return AVBD_STATUS_OK;
}

int32_t avbd_batch_num_scenes(const AvbdBatch* b) {
    if (!b) return AVBD_ERR_INVALID;
    int n = 0;
    for (int s : b->state) n += s != 0;
    return n;
}

static bool live_slot(const AvbdBatch* b, int scene) {
    return b && scene >= 0 && scene < (int)b->state.size() && b->state[scene] == 1;
}

int32_t avbd_batch_scene_status(AvbdBatch* b, int32_t scene) {
    if (!b || scene < 0 || scene >= (int)b->state.size() || b->state[scene] == 0) return AVBD_ERR_INVALID;
    if (b->state[scene] == 2) return AVBD_STATUS_OK;
    if (int r = batch_settle(b)) return r;
    cudaSetDevice(b->device);
    SceneState st;
    if (cudaMemcpy(&st, b->P.d_sstate + scene, sizeof(SceneState), cudaMemcpyDeviceToHost) != cudaSuccess)
        return AVBD_ERR_CUDA;
    return st.status;
}

int32_t avbd_batch_scene_info(AvbdBatch* b, int32_t scene, int32_t out[6]) {
    if (!b || !out || scene < 0 || scene >= (int)b->state.size() || b->state[scene] == 0) return AVBD_ERR_INVALID;
    if (b->state[scene] == 2) { for (int i = 0; i < 6; ++i) out[i] = 0; return 0; }
    if (int r = batch_settle(b)) return r;
    cudaSetDevice(b->device);
    SceneState st;
    if (cudaMemcpy(&st, b->P.d_sstate + scene, sizeof(SceneState), cudaMemcpyDeviceToHost) != cudaSuccess)
        return AVBD_ERR_CUDA;
    out[0] = st.status; out[1] = st.ncolours; out[2] = st.ncand[st.cur]; out[3] = st.kused[st.cur];
    out[4] = st.ninc; out[5] = st.step;
    return 0;
}

int32_t avbd_batch_scene_bodies(const AvbdBatch* b, int32_t scene) {
    if (!b || scene < 0 || scene >= (int)b->state.size() || b->state[scene] == 0) return AVBD_ERR_INVALID;
    return b->bodies[scene];
}

int64_t avbd_batch_dynamic_bodies(const AvbdBatch* b) {
    if (!b) return AVBD_ERR_INVALID;
    int64_t n = 0;
    for (size_t i = 0; i < b->state.size(); ++i)
        if (b->state[i] != 0) n += b->dynamic[i];
    return n;
}

int32_t avbd_batch_get_state(AvbdBatch* b, int32_t scene, float* pos, float* quat, float* vel, float* omega) {
    if (!live_slot(b, scene)) return AVBD_ERR_INVALID;
    if (int r = batch_settle(b)) return r;
    const int n = b->bodies[scene];
    cudaSetDevice(b->device);
    const int b0 = b->descs[scene].body0;
    std::vector<float4> buf(n);
    const World& W = b->P.W;
    auto fetch = [&](const float4* src, float* dst, bool q) {
        if (!dst || n == 0) return;
        cudaMemcpy(buf.data(), src + b0, n * sizeof(float4), cudaMemcpyDeviceToHost);
        for (int i = 0; i < n; ++i) {
            const float4 x = buf[i];
            if (q) { dst[4 * i] = x.w; dst[4 * i + 1] = x.x; dst[4 * i + 2] = x.y; dst[4 * i + 3] = x.z; }
            else { dst[3 * i] = x.x; dst[3 * i + 1] = x.y; dst[3 * i + 2] = x.z; }
        }
    };
    fetch(W.pos, pos, false);
    fetch(W.rot, quat, true);
    fetch(W.vel, vel, false);
    fetch(W.omega, omega, false);
    return n;
}

int32_t avbd_batch_get_all_poses(AvbdBatch* b, float* pos, float* quat, int64_t max_bodies) {
    if (!b || !b->reserved) return AVBD_ERR_STATE;
    if (int r = batch_settle(b)) return r;
    cudaSetDevice(b->device);
    const int n = b->P.nb;
    if (n > max_bodies) return AVBD_ERR_INVALID;
    const World& W = b->P.W;
    if (pos && cudaMemcpyAsync(pos, W.pos, n * sizeof(float4), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess)
        return AVBD_ERR_CUDA;
    if (quat && cudaMemcpyAsync(quat, W.rot, n * sizeof(float4), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess)
        return AVBD_ERR_CUDA;
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    return n;
}

int32_t avbd_batch_scene_body_offset(const AvbdBatch* b, int32_t scene) {
    if (!live_slot(b, scene)) return AVBD_ERR_INVALID;
    return b->descs[scene].body0;
}

// Device bytes per unit of each pool (allocate_all / alloc_tables).
constexpr int64_t kBytesPerBody = 15 * 16 + 18 * 4;        // float4 state + per-body ints
constexpr int64_t kBytesPerCand = 2 * (8 + 4 + 4 + 4 + 4 + 4);  // two manifold tables
constexpr int64_t kBytesPerContact = 2 * (4 + 9 * 16);      // two contact pools
constexpr int64_t kBytesPerForce = 4 + 8 + 6 * 16 + 6 * 6 * 4;
constexpr int64_t kBytesPerTet = 16 + 36 + 48 + 16 + 16 + 4;
constexpr int64_t kBytesPerTri = 16 + 16 + 24 + 16;

int64_t avbd_scene_footprint_bytes(const AvbdWorld* w) {
    if (!w) return AVBD_ERR_INVALID;
    int cc, kc, nsinc, nsp;
    scene_caps(w->h, cc, kc);
    static_counts(w->h, nsinc, nsp);
    int64_t bytes = (int64_t)w->h.nbody() * kBytesPerBody + (int64_t)w->h.nforce() * kBytesPerForce +
                    (int64_t)w->h.ntet() * kBytesPerTet + (int64_t)w->h.ntri() * kBytesPerTri;
    bytes += (int64_t)cc * kBytesPerCand + (int64_t)kc * kBytesPerContact;
    bytes += 4 * ((int64_t)nsinc + 2 * cc) + 4 * (int64_t)nsinc + 8 * (int64_t)nsp;
    bytes += sizeof(SceneDesc) + sizeof(SceneState) + 4 * (kMaxColours + 1);
    return bytes;
}

int64_t avbd_batch_uploaded_bytes(const AvbdBatch* b) { return b ? b->uploaded_bytes : AVBD_ERR_INVALID; }

int32_t avbd_batch_set_launch(AvbdBatch* b, int32_t threads, int32_t ctas_per_sm) {
    if (!b || threads < 0 || ctas_per_sm < 0 || (threads && (threads % 32 || threads > 1024))) return AVBD_ERR_INVALID;
    b->threads = threads;
    b->ctas_per_sm = ctas_per_sm;
    b->grid = 0;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_set_kernel(AvbdBatch* b, int32_t register_variant) {
    if (!b || register_variant < 1 || register_variant > kNumBatchVariants) return AVBD_ERR_INVALID;
    b->variant = register_variant;
    b->grid = 0;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_set_team_work(AvbdBatch* b, int32_t units_per_lane) {
    if (!b || units_per_lane < 0) return AVBD_ERR_INVALID;
    b->team_work = units_per_lane;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_set_fem_team_work(AvbdBatch* b, int32_t units_per_lane) {
    if (!b || units_per_lane < 0) return AVBD_ERR_INVALID;
    b->fem_team_work = units_per_lane;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_set_grid_broadphase(AvbdBatch* b, int32_t min_bodies) {
    if (!b || min_bodies < 0) return AVBD_ERR_INVALID;
    b->grid_min = min_bodies;
    batch_drop_graph(b);
    return 0;
}

int32_t avbd_batch_get_launch(const AvbdBatch* b, int32_t* threads, int32_t* ctas_per_sm) {
    if (!b) return AVBD_ERR_INVALID;
    if (threads) *threads = b->threads;
    if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
    return 0;
}

float avbd_batch_last_ms(const AvbdBatch* b) { return b ? b->last_ms : -1.f; }

static_assert(kGroupFlat == AVBD_GROUP_FLAT, "flat sweep selector");
static bool valid_group(int g) { return g == 1 || g == 2 || g == 4 || g == 8 || g == 16 || g == 32; }

int32_t avbd_batch_set_groups(AvbdBatch* b, int32_t rigid_group, int32_t fem_group) {
    if (!b || !valid_group(rigid_group) || !(valid_group(fem_group) || fem_group == kGroupFlat))
        return AVBD_ERR_INVALID;
    if (b->reserved) return AVBD_ERR_STATE;
    b->group_rigid = rigid_group;
    b->group_fem = fem_group;
    return 0;
}

int32_t avbd_set_group(AvbdWorld* w, int32_t group) {
    if (!w || (group != 0 && !valid_group(group))) return AVBD_ERR_INVALID;
    if (w->uploaded) return AVBD_ERR_STATE;
    w->group = group;
    return 0;
}

}  // extern "C"

// ===========================================================================
// Allocation-free box-box collision queries.
//
// For callers that must not allocate device memory during a call: code
// running under a fixed memory budget or a custom pool, hosts that forbid
// cudaMalloc/cudaFree on their hot path (they synchronise the device and can
// fail), and libraries embedded in another runtime that owns all allocations.
// The scratch lives in one file-scope device array of fixed size instead.
// ===========================================================================
namespace {

constexpr int kNoAllocMaxPairs = AVBD_COLLIDE_NOALLOC_MAX_PAIRS;

struct NoAllocScratch {
    int32_t body_a[kNoAllocMaxPairs];
    int32_t body_b[kNoAllocMaxPairs];
    int counts[kNoAllocMaxPairs];
    uint32_t ids[kNoAllocMaxPairs * 8];
    float data[kNoAllocMaxPairs * 8 * 13];
};

// Shared by every call on a device; it keeps the last call's contents.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of g_noalloc_scratch per device, looked up on the first
// call on that device; the lookup is serialised so concurrent first calls
// from several host threads do not race on the cache.
constexpr int kNoAllocMaxDevices = 64;
std::atomic<NoAllocScratch*> g_noalloc_ptr[kNoAllocMaxDevices] = {};
std::mutex g_noalloc_lookup;

NoAllocScratch* noalloc_scratch(int device) {
    NoAllocScratch* s = g_noalloc_ptr[device].load(std::memory_order_acquire);
    if (s) return s;
    std::lock_guard<std::mutex> lock(g_noalloc_lookup);
    s = g_noalloc_ptr[device].load(std::memory_order_relaxed);
    if (!s) {
        // with `device` current: the host name g_noalloc_scratch is only a
        // stand-in, the kernel needs the address on that device
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return nullptr;
        s = static_cast<NoAllocScratch*>(p);
        g_noalloc_ptr[device].store(s, std::memory_order_release);
    }
    return s;
}

// Puts back the caller's current device when the call returns.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() { if (cudaGetDevice(&prev) != cudaSuccess) prev = -1; }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

__global__ void k_collide_pairs_noalloc(const __grid_constant__ World W, NoAllocScratch* s, int n, int nbody) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int2 ab = make_int2(s->body_a[i], s->body_b[i]);
        uint32_t* ids = s->ids + 8 * i;
        float* data = s->data + 8 * 13 * i;
        int cnt = 0;
        if (ab.x >= 0 && ab.y >= 0 && ab.x < nbody && ab.y < nbody) {
            Collision col;
            collide_box_box(v3(W.pos[ab.x]), q4(W.rot[ab.x]), v3(W.scale[ab.x]), v3(W.pos[ab.y]), q4(W.rot[ab.y]),
                            v3(W.scale[ab.y]), col);
            cnt = col.n;
            for (int k = 0; k < col.n; ++k) {
                const Contact& c = col.c[k];
                float* d = data + 13 * k;
                ids[k] = c.id;
                d[0] = c.penetration;
                d[1] = c.normal.x; d[2] = c.normal.y; d[3] = c.normal.z;
                d[4] = c.rA.x; d[5] = c.rA.y; d[6] = c.rA.z;
                d[7] = c.rB.x; d[8] = c.rB.y; d[9] = c.rB.z;
                d[10] = c.position.x; d[11] = c.position.y; d[12] = c.position.z;
            }
        }
        // slots past the contact count keep nothing from an earlier call
        for (int k = cnt; k < 8; ++k) {
            ids[k] = 0xFFFFFFFFu;
            for (int q = 0; q < 13; ++q) data[13 * k + q] = 0.f;
        }
        s->counts[i] = ab.x >= 0 && ab.y >= 0 && ab.x < nbody && ab.y < nbody ? cnt : -1;
    }
}

}  // namespace

extern "C" int32_t avbd_collide_noalloc(AvbdWorld* w, int32_t n, const int32_t* body_a, const int32_t* body_b,
                                        uint32_t* ids, float* data, int32_t* counts) {
    if (!w || n < 0 || (n > 0 && (!body_a || !body_b || !ids || !data || !counts))) return AVBD_ERR_INVALID;
    if (n > kNoAllocMaxPairs) {
        std::fprintf(stderr, "avbd_collide_noalloc: %d pairs exceed the maximum of %d per call\n", n,
                     kNoAllocMaxPairs);
        return AVBD_ERR_INVALID;
    }
    if (!w->uploaded) return AVBD_ERR_STATE;   // the world must already live on the device
    if (w->device < 0 || w->device >= kNoAllocMaxDevices) return AVBD_ERR_INVALID;
    DeviceGuard keep_device;
    if (cudaSetDevice(w->device) != cudaSuccess) return AVBD_ERR_CUDA;
    NoAllocScratch* s = noalloc_scratch(w->device);
    if (!s) return AVBD_ERR_CUDA;
    if (n == 0) return 0;
    cudaStream_t st = w->stream;
    if (cudaMemcpyAsync(s->body_a, body_a, n * sizeof(int32_t), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(s->body_b, body_b, n * sizeof(int32_t), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return AVBD_ERR_CUDA;
    k_collide_pairs_noalloc<<<(n + 127) / 128, 128, 0, st>>>(w->P.W, s, n, w->h.nbody());
    if (cudaGetLastError() != cudaSuccess) return AVBD_ERR_CUDA;
    if (cudaMemcpyAsync(counts, s->counts, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(ids, s->ids, (size_t)n * 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(data, s->data, (size_t)n * 8 * 13 * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return AVBD_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return AVBD_ERR_CUDA;
    for (int i = 0; i < n; ++i)
        if (counts[i] < 0) return AVBD_ERR_INVALID;
    return 0;
}
