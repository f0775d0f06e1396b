// Host-side state shared by the translation units of the library: device
// pools of a world or batch (structure of arrays, first-fit ranges), the
// scene upload, and the AvbdWorld / AvbdBatch handles of include/avbd.h.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/avbd.h"
#include "avbd_common.cuh"
#include "avbd_host.h"

namespace avbd {
namespace host {

constexpr int kThreads = 128;   // block size of the grid-wide kernels

inline int blocks_for(int n, int threads = kThreads) {
    int b = (n + threads - 1) / threads;
    return std::max(1, std::min(b, 148 * 32));
}

// A named NVTX range over a scope: phases of the host loops show up on the
// timeline of an attached profiler (nvtx3 is header-only; without a tool the
// calls return at once).
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

// Consecutive phases of one loop as NVTX ranges: next() closes the open one.
struct PhaseRanges {
    bool open = false;
    void next(const char* name) {
        if (open) nvtxRangePop();
        nvtxRangePushA(name);
        open = true;
    }
    void end() {
        if (open) nvtxRangePop();
        open = false;
    }
    ~PhaseRanges() { end(); }
};

inline bool valid_group(int g) { return g == 1 || g == 2 || g == 4 || g == 8 || g == 16 || g == 32; }

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
        A(alloc(W.color, nb));
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
        A(alloc(W.tidx, nt)); A(alloc(W.tDmInv, 9 * (size_t)nt));
        A(alloc(W.tparam, nt)); A(alloc(W.tkind, nt));
        A(alloc(W.trv, 4 * (size_t)nt)); A(alloc(W.trm0, 4 * (size_t)nt)); A(alloc(W.trm1, 4 * (size_t)nt));
        A(alloc(W.trm2, 4 * (size_t)nt));
        A(alloc(W.ridx, nr)); A(alloc(W.rDmInv, nr)); A(alloc(W.rgradN, 6 * (size_t)nr)); A(alloc(W.rparam, nr));
        A(alloc(W.inc, ninc));
        A(alloc(W.check, 4));
        for (int t = 0; t < 2; ++t) A(alloc_tables(t, ncand, nk));
#undef A
        // the zeroing memsets run on the legacy stream; the uploads that follow
        // run on non-blocking streams and must find the pools zeroed
        return cudaStreamSynchronize(cudaStreamLegacy);
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
inline int scene_group(const HostScene& h, int rigid_group, int fem_group) {
    if (h.ntet() == 0 && h.ntri() == 0) return rigid_group;
    if (fem_group == kGroupFlat && h.ntri() > 0) return 4;   // the flat sweep takes tet energies only
    return fem_group;
}

// Capacity policy of one scene.
inline void scene_caps(const HostScene& h, int& candcap, int& kcap) {
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
inline bool place_scene(Allocs& A, const HostScene& h, int candcap, int kcap, int nsinc, int nsp, Region& r) {
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
// many scenes into fresh (zeroed) pools at once; what is zero there already
// (cleared arrays, all-zero data such as scenes at rest) is not copied.
struct DirectSink {
    cudaStream_t st;
    template <typename T>
    void put(T* dst, const std::vector<T>& src, size_t at) {
        if (!src.empty()) cudaMemcpyAsync(dst + at, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st);
    }
    // `src` into arrays dst[0..n) at the same offset: one host copy, the
    // others device to device
    template <typename T>
    void put_all(T* const* dst, int n, const std::vector<T>& src, size_t at) {
        put(dst[0], src, at);
        for (int i = 1; i < n && !src.empty(); ++i)
            cudaMemcpyAsync(dst[i] + at, dst[0] + at, src.size() * sizeof(T), cudaMemcpyDeviceToDevice, st);
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
    // Arrays written as copies of another array's range (put_all): filled on
    // the device from their source after the host copies, [lo, hi) in bytes.
    struct Mirror {
        char* src = nullptr;
        size_t lo = SIZE_MAX, hi = 0;
    };
    std::map<char*, Mirror> mirrors;
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
        const size_t n = src.size() * sizeof(T);
        const unsigned char* p = reinterpret_cast<const unsigned char*>(src.data());
        size_t i = 0;
        while (i < n && p[i] == 0) ++i;
        if (i == n) { fits(dst, at * sizeof(T) + n); return; }   // the pool holds these zero bytes already
        if (char* h = span(dst, at * sizeof(T), n)) std::memcpy(h + at * sizeof(T), src.data(), n);
    }
    template <typename T>
    void put_all(T* const* dst, int n, const std::vector<T>& src, size_t at) {
        put(dst[0], src, at);
        if (src.empty()) return;
        std::lock_guard<std::mutex> lock(m);
        for (int i = 1; i < n; ++i) {
            Mirror& mi = mirrors[reinterpret_cast<char*>(dst[i])];
            mi.src = reinterpret_cast<char*>(dst[0]);
            mi.lo = std::min(mi.lo, at * sizeof(T));
            mi.hi = std::max(mi.hi, (at + src.size()) * sizeof(T));
        }
    }
    // fresh pools are zeroed when allocated
    template <typename T>
    void zero(T* dst, size_t at, size_t n) {
        if (n) fits(dst, (at + n) * sizeof(T));
    }
    // Sets overflow if pool array `dst` is shorter than `end` bytes.
    void fits(const void* dst, size_t end) {
        if (!P) return;
        for (size_t i = 0; i < P->owned.size(); ++i)
            if (P->owned[i] == dst) {
                if (P->owned_bytes[i] < end) {
                    std::lock_guard<std::mutex> lock(m);
                    overflow = true;
                }
                return;
            }
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
        for (auto& kv : mirrors)
            if (kv.second.hi > kv.second.lo)
                cudaMemcpyAsync(kv.first + kv.second.lo, kv.second.src + kv.second.lo, kv.second.hi - kv.second.lo,
                                cudaMemcpyDeviceToDevice, st);
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
        mirrors.clear();
    }
};

// Stages scene uploads in a page-locked arena and records one copy (or
// memset) per written range, so they can be issued later on a stream without
// the host waiting: the serving loop stages newcomers while a step runs.  The
// arena must not be reused or grown while the stream still reads it.
struct ArenaSink {
    struct Op {
        void* dst;
        size_t off;     // arena offset of the source bytes (copies)
        size_t bytes;
        bool memset;
    };
    char* arena = nullptr;
    size_t cap = 0, used = 0;
    std::vector<Op> ops;
    bool pinned = false;
    ArenaSink() = default;
    ArenaSink(const ArenaSink&) = delete;
    ArenaSink& operator=(const ArenaSink&) = delete;
    ~ArenaSink() { release(); }
    void release() {
        if (arena) { if (pinned) cudaFreeHost(arena); else std::free(arena); }
        arena = nullptr;
        cap = used = 0;
    }
    // Grows the arena to hold `bytes`, keeping what is staged.
    bool grow(size_t bytes) {
        if (bytes <= cap) return true;
        size_t ncap = std::max(bytes, 2 * cap);
        void* p = nullptr;
        bool pin = cudaHostAlloc(&p, ncap, cudaHostAllocDefault) == cudaSuccess;
        if (!pin) { cudaGetLastError(); p = std::malloc(ncap); }
        if (!p) return false;
        if (used) std::memcpy(p, arena, used);
        const size_t keep = used;
        release();
        arena = static_cast<char*>(p);
        cap = ncap;
        used = keep;
        pinned = pin;
        return true;
    }
    void clear() { used = 0; ops.clear(); }
    bool overflow = false;   // the arena could not grow (host memory)
    template <typename T>
    void put(T* dst, const std::vector<T>& src, size_t at) {
        if (src.empty()) return;
        const size_t n = src.size() * sizeof(T);
        const size_t off = (used + 15) & ~size_t(15);
        if (!grow(off + n)) { overflow = true; return; }
        std::memcpy(arena + off, src.data(), n);
        used = off + n;
        ops.push_back({static_cast<void*>(dst + at), off, n, false});
    }
    // one staged copy of `src`, scattered to every array dst[0..n)
    template <typename T>
    void put_all(T* const* dst, int n, const std::vector<T>& src, size_t at) {
        put(dst[0], src, at);
        if (src.empty() || overflow) return;
        const Op first = ops.back();
        for (int i = 1; i < n; ++i) ops.push_back({static_cast<void*>(dst[i] + at), first.off, first.bytes, false});
    }
    template <typename T>
    void zero(T* dst, size_t at, size_t n) {
        if (n) ops.push_back({static_cast<void*>(dst + at), 0, n * sizeof(T), true});
    }
    void finish() {}
    // Appends the op table to the arena as ScatterOps (16-byte aligned) and
    // returns its offset, for a single copy of data and table followed by a
    // device scatter; -1 if the arena cannot grow.
    struct ScatterOp {
        unsigned long long dst, src, bytes;   // src: arena offset; bytes | 1 << 63 for a memset
    };
    int64_t append_table() {
        const size_t off = (used + 15) & ~size_t(15);
        const size_t n = ops.size() * sizeof(ScatterOp);
        if (!grow(off + n)) { overflow = true; return -1; }
        ScatterOp* t = reinterpret_cast<ScatterOp*>(arena + off);
        for (size_t i = 0; i < ops.size(); ++i) {
            const Op& o = ops[i];
            t[i].dst = reinterpret_cast<unsigned long long>(o.dst);
            t[i].src = o.off;
            t[i].bytes = (unsigned long long)o.bytes | (o.memset ? (1ull << 63) : 0ull);
        }
        used = off + n;
        return (int64_t)off;
    }
    // Issues every recorded copy and memset on `st`; returns the bytes copied.
    int64_t issue(cudaStream_t st) const {
        int64_t bytes = 0;
        for (const Op& o : ops) {
            if (o.memset) {
                cudaMemsetAsync(o.dst, 0, o.bytes, st);
            } else {
                cudaMemcpyAsync(o.dst, arena + o.off, o.bytes, cudaMemcpyHostToDevice, st);
                bytes += (int64_t)o.bytes;
            }
        }
        return bytes;
    }
};

// Writes a placed scene (as staged) into the pools and its descriptor/state
// into scene slot `slot`.
template <typename Sink>
inline void upload_scene(Pools& P, const HostScene& h, const StaticInc& si, const Region& r, int group, int slot,
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
    sink.put(W.vel, h.vel, d.body0); sink.put(W.omega, h.omega, d.body0); sink.put(W.massI, h.massI, d.body0);
    sink.put(W.flags, h.flags, d.body0); sink.put(W.friction, h.friction, d.body0);
    sink.put(W.color, h.color, d.body0);
    // lastPosition and inertialPosition start equal to the pose: one upload of each
    float4* const pos_to[3] = {W.pos, W.lpos, W.ipos};
    float4* const rot_to[3] = {W.rot, W.lrot, W.irot};
    sink.put_all(pos_to, 3, h.pos, d.body0); sink.put_all(rot_to, 3, h.rot, d.body0);
    sink.put(W.scale, h.scale, d.body0);
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
    sink.put(W.tparam, h.tparam, d.tet0);
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
inline void static_counts(const HostScene& h, int& nsinc, int& nsp) {
    nsinc = 4 * h.ntet() + 3 * h.ntri();
    nsp = 0;
    for (const int2& ab : h.fbody) {
        nsinc += ab.x >= 0 ? 2 : 1;
        nsp += ab.x >= 0 ? 2 : 0;
    }
}

inline StaticInc static_incidence(const HostScene& h, const Region& r) {
    StaticInc si;
    h.build_static_incidence(si.off, si.cnt, si.nf, si.ent, si.poff, si.pcnt, si.partners, r.body0, r.force0, r.tet0,
                             r.tri0);
    return si;
}

inline Params to_params(const AvbdParams& p) {
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

inline bool valid_params(const AvbdParams* p) {
    return p && p->num_iterations >= 0 && p->step_value > 0.f && p->projection_mode >= 0 && p->projection_mode <= 2;
}

inline int device_ready(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return AVBD_ERR_NODEVICE;
    if (device < 0 || device >= n) return AVBD_ERR_INVALID;
    return cudaSetDevice(device) == cudaSuccess ? 0 : AVBD_ERR_CUDA;
}

}  // namespace host
}  // namespace avbd

// ===========================================================================
// Single-scene world (one Solver)
// ===========================================================================
struct AvbdWorld {
    AvbdParams params{};
    int device = 0;
    avbd::HostScene h;
    bool uploaded = false;
    bool stopped = false;
    int stop_status = AVBD_STATUS_OK;   // EXPLODED or NAN once stopped
    avbd::host::Pools P;
    std::vector<avbd::SceneDesc> descs;
    int group = 0;   // lanes per body in the primal (0 = by scene kind)
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8] = {};
    AvbdTimings timings{};
    int ncolours = 0;
    std::vector<int> col_start;
    avbd::SceneState st{};   // host mirror of the scene counters after the last step
    void* grid = nullptr;     // device scratch of the grid broadphase (avbd_api.cu)
    void* colour = nullptr;   // device scratch of the grid-wide colouring (avbd_api.cu)
    // colouring neighbour lists: up to 3 per incidence entry, at 3 x the entry's offset
    int* nbr = nullptr;
    int* nbr_cnt = nullptr;
    unsigned long long* nbr_key = nullptr;   // pass-0 priority of each body
    int* nbr_pos = nullptr;                  // per body: neighbours scanned this pass
    unsigned long long* nbr_used = nullptr;  // per body: colours seen so far
    size_t nbr_cap = 0;
};

// ===========================================================================
// Batch (many scenes, one persistent kernel per step)
// ===========================================================================
struct AvbdBatch {
    AvbdParams params{};
    int device = 0;
    // scene slots (scene id = slot); a retired slot is reused by a later scene
    std::vector<avbd::HostScene> scenes;   // staged copies (emptied when a scene retires)
    std::vector<int> state;          // 0 free, 1 live, 2 staged (not placed yet)
    std::vector<avbd::host::Region> regions;
    std::vector<avbd::SceneDesc> descs;
    std::vector<int> bodies;         // body count of each slot's scene
    std::vector<int> dynamic;        // dynamic bodies of each slot's scene
    bool reserved = false;           // pools allocated
    avbd::host::Pools P;
    avbd::host::Allocs A;
    int* d_order = nullptr;          // live slots, largest first (queue_key)
    int queue_body_weight = 1;       // queue key = weight x bodies + tets (avbd_batch_set_queue_weight)
    int* d_nlive = nullptr;
    int* d_queue = nullptr;
    int nlive = 0;
    bool order_dirty = true;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    // avbd_batch_read_poses: two device snapshots of (pos, rot), read back on a copy stream
    float4* d_pose_snap[2] = {nullptr, nullptr};
    int64_t pose_snap_n = 0;
    int pose_snap_cur = 0;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t snap_ev[2] = {nullptr, nullptr}, read_ev[2] = {nullptr, nullptr};
    cudaGraphExec_t graph = nullptr;
    int threads = 0, ctas_per_sm = 0;   // 0 = automatic
    int group_rigid = 4, group_fem = 8;  // lanes per body in the primal sweep
    int variant = 1;                     // build of the persistent kernel (1..7, see kBatchVariants)
    int grid = 0;
    int stage = 0;   // float4 slots of dynamic shared memory per CTA
    int team_work = 0;   // bodies + tets per lane below which a CTA team splits (0 = never)
    int fem_team_work = 0;   // the same for scenes with tets
    int grid_min = 128;  // scenes from this many bodies use the grid broadphase (0 = never)
    int cluster = 1;     // CTAs per thread-block cluster (1 = plain launch)
    int cluster_min = 0; // bodies + tets from which a scene is run by a whole cluster
    std::vector<long long> steps_due;   // steps each slot's scene should have taken
    int* d_fail = nullptr;               // scene steps stopped by a full table (device counter)
    unsigned long long* d_scene_ns = nullptr;   // per-slot step start/end (avbd_batch_set_scene_timing)
    int* d_fix_order = nullptr;          // catch-up queue
    int* d_fix_n = nullptr;
    float last_ms = 0.f;
    // Scenes placed and staged into page-locked host buffers by
    // avbd_batch_prepare, copied to the pools by the next step.
    std::unique_ptr<avbd::host::StagedSink> upload;
    bool upload_pending = false;
    bool upload_pinned = false;   // the staging buffers are page-locked
    int64_t uploaded_bytes = 0;   // host-to-device bytes of the last staged upload
};

// Queue order of a scene: estimated work, largest first.  With clusters the
// key stays bodies + tets, the unit of the cluster threshold.
inline int64_t queue_key(const AvbdBatch* b, const avbd::SceneDesc& d) {
    const int64_t w = b->cluster > 1 ? 1 : b->queue_body_weight;
    return w * d.nbody + d.ntet;
}

namespace avbd {
namespace host {

// Instance export of the bodies [body0, body0 + nbody) (avbd_api.cu).
int export_instances(const World& W, int body0, int nbody, AvbdInstance* dst, int32_t capacity,
                     int32_t first_per_model[3], int32_t count_per_model[3], cudaStream_t st);

// Batch internals (avbd_batch_host.cu) used by the serving loop.
int batch_stream(AvbdBatch* b);
int batch_reserve(AvbdBatch* b, int64_t bodies, int64_t forces, int64_t tets, int64_t tris, int64_t nscenes,
                  int64_t nsinc, int64_t nsp);
int batch_place(AvbdBatch* b, int slot);
int batch_flush(AvbdBatch* b);
int batch_launch_shape(AvbdBatch* b);
// Scenes at the head of the size-ordered list that a whole cluster runs.
int cluster_scenes(const AvbdBatch* b, const std::vector<int>& order);
// Launches the batch's persistent kernel build (in clusters when set) on its stream.
cudaError_t launch_batch_kernel(AvbdBatch* b, const World& W, const int* order, const int* nlive, int* queue);
int batch_build_graph(AvbdBatch* b);
void batch_sync_order(AvbdBatch* b);
// Grows the scenes a full table stopped and re-runs the steps they missed;
// `grown` (optional) counts the scenes grown.
int batch_fix_capacity(AvbdBatch* b, int64_t* grown = nullptr);
int batch_settle(AvbdBatch* b);
void batch_drop_graph(AvbdBatch* b);

}  // namespace host
}  // namespace avbd
