// Step drivers of the batched path.  Team-cooperative functions (scans,
// incidence build, Jones-Plassmann colouring, colour lists) run on the team
// (a CTA, part of one, or a thread-block cluster) that owns a scene; the
// persistent batched kernel strings every phase of a scene's step together
// on that team.  The single-scene path (avbd_api.cu) launches the same
// per-item functions as grid-wide kernels, with grid-wide counterparts of the
// team functions.
#pragma once
#include <cooperative_groups.h>

#include "avbd_phases.cuh"

namespace avbd {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxTeams = 8;          // teams a CTA may split into

// Scalars a team shares through shared memory.
constexpr int kGridMaxBig = 32;   // big bodies (kept out of the broadphase grid) a scene may have

struct TeamShared {
    int q, flags, remaining, progress, maxc, carry, nbig;
    int warp_tot[32];
    int red[8];
    int big[kGridMaxBig];
};

// Consecutive whole warps of a CTA that run one scene together: the whole CTA
// (barrier 0, i.e. __syncthreads) or a power-of-two part of it with its own
// named barrier (a single warp uses __syncwarp).  Teams only split, so the
// teams alive at one time partition the CTA's warps; a team's barrier id and
// shared slot follow from its first warp, which no other live team shares.
constexpr int kClusterBar = -2;   // Team::bar of a team that is a whole thread-block cluster

struct Team {
    int rank;          // thread index within the team
    int size;          // threads (a multiple of 32)
    int first_warp;    // first warp of the team within the CTA
    int bar;           // named barrier id (0 for the whole CTA, kClusterBar for a cluster)
    TeamShared* sh;    // the team's shared scalars
    float4* stage;     // the team's slice of the dynamic shared memory
    int stage_cap;     // float4 slots in that slice

    __device__ __forceinline__ void sync() const {
        if (bar == 0) __syncthreads();
        else if (bar == kClusterBar) cooperative_groups::this_cluster().sync();
        else if (size == 32) __syncwarp();
        else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(size) : "memory");
    }
    // Every thread of the thread-block cluster as one team: ranks run over
    // the cluster's CTAs, and the team's shared scalars and stage are those
    // of its first CTA, reached through distributed shared memory.  The
    // cluster barrier orders global and shared memory across its CTAs.
    __device__ __forceinline__ static Team cluster(TeamShared* shared, float4* stage, int stage_cap) {
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        Team t;
        t.rank = (int)(cl.block_rank() * blockDim.x + threadIdx.x);
        t.size = (int)(cl.num_blocks() * blockDim.x);
        t.first_warp = 0;
        t.bar = kClusterBar;
        t.sh = cl.map_shared_rank(shared, 0);
        t.stage = cl.map_shared_rank(stage, 0);
        t.stage_cap = stage_cap;
        return t;
    }
    // Smallest team a CTA splits into: a warp, or an eighth of a larger CTA.
    __device__ __forceinline__ static int min_size() { return max(32, (int)(blockDim.x / kMaxTeams)); }
    __device__ __forceinline__ static Team cta(TeamShared* shared, float4* stage, int stage_cap) {
        Team t;
        t.rank = threadIdx.x;
        t.size = blockDim.x;
        t.first_warp = 0;
        t.bar = 0;
        t.sh = shared;
        t.stage = stage;
        t.stage_cap = stage_cap;
        return t;
    }
    // The lower or upper half of this team, as a team of its own.
    __device__ __forceinline__ Team half(bool lower, TeamShared* shared) const {
        Team t;
        const int h = size / 2;
        t.size = h;
        t.rank = lower ? rank : rank - h;
        t.first_warp = first_warp + (lower ? 0 : h / 32);
        const int slot = t.first_warp / (min_size() / 32);
        t.bar = h == 32 ? -1 : 1 + slot;
        t.sh = shared + slot;
        t.stage_cap = stage_cap / 2;
        t.stage = stage + (lower ? 0 : t.stage_cap);
        return t;
    }
};

// Exclusive scan of in[0, n) into out[0, n) by one team; returns the total.
// in and out may alias.
static __device__ int block_exclusive_scan(const Team& T, const int* in, int* out, int n) {
    const int lane = T.rank & 31, warp = T.rank >> 5, nwarps = T.size >> 5;
    if (T.rank == 0) T.sh->carry = 0;
    T.sync();
    for (int base = 0; base < n; base += T.size) {
        const int i = base + T.rank;
        const int v = i < n ? in[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) T.sh->warp_tot[warp] = x;
        T.sync();
        if (warp == 0) {
            int w = lane < nwarps ? T.sh->warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(kFull, w, o);
                if (lane >= o) w += y;
            }
            T.sh->warp_tot[lane] = w;
        }
        T.sync();
        const int prefix = T.sh->carry + (warp > 0 ? T.sh->warp_tot[warp - 1] : 0);
        if (i < n) out[i] = prefix + x - v;
        T.sync();
        if (T.rank == T.size - 1) T.sh->carry = prefix + x;
        T.sync();
    }
    const int total = T.sh->carry;
    T.sync();
    return total;
}

// ---------------------------------------------------------------------------
// Incidence (CSR) of one scene: per body
//   [static forces][manifolds as body B, by slot][manifolds as body A][energies]
// which follows Mesh::forces then Mesh::energies (solver.cpp:395-435).
// Static and removed bodies get no entries: nothing solves or colours them,
// and a ground box touching thousands of boxes would otherwise be one
// thread's serial work.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool body_fixed(const World& W, int b) {
    return (W.flags[b] & (kBodyStatic | kBodyRemoved)) != 0;
}

static __device__ int owned_live(const World& W, int cur, int b, int base_slot) {
    const int c0 = W.cand_off[b] + base_slot, c1 = c0 + W.cand_cnt[b];
    int n = 0;
    for (int c = c0; c < c1; ++c) n += W.cn[cur][c] > 0 ? 1 : 0;
    return n;
}

// Insertion sort of manifold entries by (birth step, slot).
__device__ __forceinline__ void sort_manifold_entries(const World& W, int cur, uint32_t* seg, int n) {
    for (int i = 1; i < n; ++i) {
        const uint32_t v = seg[i];
        const int bv = W.cbirth[cur][ent_index(v)];
        int j = i - 1;
        while (j >= 0) {
            const uint32_t u = seg[j];
            const int bu = W.cbirth[cur][ent_index(u)];
            if (bu < bv || (bu == bv && ent_index(u) < ent_index(v))) break;
            seg[j + 1] = u;
            --j;
        }
        seg[j + 1] = v;
    }
}

// Returns false (and sets need_inc) when the scene's incidence region is too small.
static __device__ __noinline__ bool build_incidence(const Team& T, const World& W, const SceneDesc& sc, SceneState* st,
                                             int cur) {
    const int tid = T.rank, nt = T.size;
    const int b0 = sc.body0, b1 = sc.body0 + sc.nbody;
    const int ncand = st->ncand[cur];
    for (int b = b0 + tid; b < b1; b += nt) W.cntB[b] = 0;
    T.sync();
    for (int c = sc.cand0 + tid; c < sc.cand0 + ncand; c += nt)
        if (W.cn[cur][c] > 0) atomicAdd(&W.cntB[W.cpair[cur][c].y], 1);
    T.sync();
    for (int b = b0 + tid; b < b1; b += nt) {
        const int ns = W.sinc_n[b];
        W.inc_cnt[b] = body_fixed(W, b) ? 0 : ns + W.cntB[b] + owned_live(W, cur, b, sc.cand0);
    }
    T.sync();
    const int total = block_exclusive_scan(T, W.inc_cnt + b0, W.inc_off + b0, sc.nbody);
    if (total > sc.inccap) {
        if (tid == 0) { st->need_inc = total; }
        return false;
    }
    for (int b = b0 + tid; b < b1; b += nt) {
        const int off = sc.inc0 + W.inc_off[b];
        W.inc_off[b] = off;
        W.bcur[b] = 0;
        if (body_fixed(W, b)) continue;
        if (!AVBD_CHECK(W, off + W.inc_cnt[b] <= sc.inc0 + sc.inccap, 1, off + W.inc_cnt[b], sc.inc0 + sc.inccap)) {
            W.inc_cnt[b] = 0;   // readers then see no entries rather than unwritten ones
            continue;
        }
        const int s0 = W.sinc_off[b], nf = W.sinc_nf[b], ns = W.sinc_n[b];
        int k = off;
        for (int e = 0; e < nf; ++e) W.inc[k++] = W.sinc[s0 + e];
        k += W.cntB[b];
        const int c0 = W.cand_off[b] + sc.cand0, c1 = c0 + W.cand_cnt[b];
        for (int c = c0; c < c1; ++c)
            if (W.cn[cur][c] > 0) W.inc[k++] = ent_make(kEntManifold, 0, (uint32_t)c);
        for (int e = nf; e < ns; ++e) W.inc[k++] = W.sinc[s0 + e];
    }
    T.sync();
    for (int c = sc.cand0 + tid; c < sc.cand0 + ncand; c += nt) {
        if (W.cn[cur][c] == 0) continue;
        const int B = W.cpair[cur][c].y;
        if (body_fixed(W, B)) continue;
        const int p = atomicAdd(&W.bcur[B], 1);
        if (!AVBD_CHECK(W, p < W.cntB[B], 2, p, W.cntB[B])) continue;
        W.inc[W.inc_off[B] + W.sinc_nf[B] + p] = ent_make(kEntManifold, 1, (uint32_t)c);
    }
    T.sync();
    // order each body's manifolds as Mesh::forces holds them: by creation step,
    // then by pair (creation order within a broadphase pass)
    for (int b = b0 + tid; b < b1; b += nt) {
        if (body_fixed(W, b)) continue;
        uint32_t* seg = W.inc + W.inc_off[b] + W.sinc_nf[b];
        const int n = W.inc_cnt[b] - W.sinc_n[b];
        sort_manifold_entries(W, cur, seg, n);
    }
    if (tid == 0) st->ninc = total;
    T.sync();
    return true;
}

// ---------------------------------------------------------------------------
// Colouring of the dynamic bodies of one scene: Jones-Plassmann first-fit
// (equal to sequential greedy colouring in priority order), largest degree
// first, then one iterated-greedy pass that never adds colours and usually
// removes the thin last classes (see colour_before / jp_pass).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool prio_less(uint32_t ha, int la, uint32_t hb, int lb) {
    return ha != hb ? ha < hb : la < lb;
}

template <typename Fn>
__device__ __forceinline__ void for_each_neighbour(const World& W, int cur, int b, Fn fn) {
    const int e0 = W.inc_off[b], e1 = e0 + W.inc_cnt[b];
    for (int e = e0; e < e1; ++e) {
        const uint32_t ent = W.inc[e];
        const uint32_t kind = ent_kind(ent), idx = ent_index(ent);
        if (kind == kEntManifold) {
            const int2 ab = W.cpair[cur][idx];
            fn(ab.x == b ? ab.y : ab.x);
        } else if (kind == kEntForce) {
            if (W.ftype[idx] & kForceRemoved) continue;
            const int2 ab = W.fbody[idx];
            const int o = ab.x == b ? ab.y : ab.x;
            if (o >= 0) fn(o);
        } else if (kind == kEntTet) {
            if (W.tparam[idx].w != 0.f) continue;
            const int4 v = W.tidx[idx];
            if (v.x != b) fn(v.x);
            if (v.y != b) fn(v.y);
            if (v.z != b) fn(v.z);
            if (v.w != b) fn(v.w);
        } else {
            if (W.rparam[idx].w != 0.f) continue;
            const int4 v = W.ridx[idx];
            if (v.x != b) fn(v.x);
            if (v.y != b) fn(v.y);
            if (v.z != b) fn(v.z);
        }
    }
}

// ---------------------------------------------------------------------------
// Primal update of one body by a group of G lanes (G divides 32, groups are
// warp-aligned): lane l gathers incidence entries l, l+G, ...; the 27
// accumulators (lower triangle + right-hand side) are summed across the group
// by a butterfly; lane 0 adds nothing more and solves.  Every lane of a warp
// must call this the same number of times (b < 0 for an idle group).
// ---------------------------------------------------------------------------
template <int G>
__device__ __forceinline__ void primal_group(const World& W, int cur, int b, float alpha, bool write_stick, int lane) {
    Sys6 s;
    sys_zero(s);
    if (b >= 0) {
        if (lane == 0) primal_init_mass(W, b, s);
        primal_entries(W, cur, b, alpha, write_stick, lane, G, s);
    }
    if (G > 1) {
#pragma unroll
        for (int off = G / 2; off >= 1; off >>= 1) {
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                s.r[i] += __shfl_xor_sync(kFull, s.r[i], off);
#pragma unroll
                for (int j = 0; j <= i; ++j) s.a[i][j] += __shfl_xor_sync(kFull, s.a[i][j], off);
            }
        }
    }
    if (b >= 0 && lane == 0) primal_finish(W, b, s);
}

// Sweeps the bodies list[0, n) with groups of G lanes of the calling team.
template <int G>
static __device__ void primal_sweep_cta(const Team& T, const World& W, int cur, const int* list, int n, float alpha,
                                 bool write_stick) {
    const int lane = T.rank % G, gid = T.rank / G, ngroups = T.size / G;
    for (int base = 0; base < n; base += ngroups) {
        const int i = base + gid;
        int b = i < n ? list[i] : -1;
        if (b >= 0 && (W.flags[b] & kBodyRemoved)) b = -1;
        primal_group<G>(W, cur, b, alpha, write_stick, lane);
    }
}

static __device__ __noinline__ void primal_sweep_cta_dispatch(const Team& T, const World& W, int cur, const int* list, int n,
                                                          float alpha, bool write_stick, int group) {
    switch (group) {
        case 32: primal_sweep_cta<32>(T, W, cur, list, n, alpha, write_stick); break;
        case 16: primal_sweep_cta<16>(T, W, cur, list, n, alpha, write_stick); break;
        case 8: primal_sweep_cta<8>(T, W, cur, list, n, alpha, write_stick); break;
        case 4: primal_sweep_cta<4>(T, W, cur, list, n, alpha, write_stick); break;
        case 2: primal_sweep_cta<2>(T, W, cur, list, n, alpha, write_stick); break;
        default: primal_sweep_cta<1>(T, W, cur, list, n, alpha, write_stick); break;
    }
}

// ---------------------------------------------------------------------------
// Term-per-lane primal sweep of one colour, for scenes whose energies are all
// tetrahedra.  Up to nslots (particle, tet) terms of the colour are
// evaluated at once, one per lane, into shared memory; then each particle
// adds its inertia, its force and manifold rows and its tet terms in
// incidence order (the reference's order) and solves, its nine sums split
// over up to nine lanes when the chunk has few particles.  Lanes stay busy
// whatever the particles' degrees.  tinc (the scene's col_tinc) holds the
// inclusive prefix of tet terms over the colour list, and the tet-term
// records from rec0 on hold the terms in that order (both made with the
// colouring); the colour occupies list positions [c0, c1).  sm: 9 * nslots
// words of shared memory (the broadphase's stage, reused).
// ---------------------------------------------------------------------------

__device__ __forceinline__ int tet_terms(const World& W, int b) { return W.sinc_n[b] - W.sinc_nf[b]; }

// Any body of a flat-swept colour: inertia, force and manifold rows, then its
// tet terms from slot q0 on (q0 < 0: terms evaluated here, the slots did not
// hold them).  Out of line: the 6x6 system stays out of the sweep's registers.
static __device__ __noinline__ void flat_finish_body(const World& W, int cur, int b, int e0, int e1, int q0, float alpha,
                                              bool write_stick, const float* sm, int nslots) {
    Sys6 s;
    sys_zero(s);
    primal_init_mass(W, b, s);
    if (q0 < 0) {
        primal_entry_range(W, cur, b, alpha, write_stick, e0, e1, 0, 1, s);
    } else {
        const int nterm = tet_terms(W, b);
        primal_entry_range(W, cur, b, alpha, write_stick, e0, e1 - nterm, 0, 1, s);
        for (int q = q0; q < q0 + nterm; ++q) {
            // a removed tet left zeros: adding them changes no value
            sys_add_energy(s, sm[0 * nslots + q], sm[1 * nslots + q], sm[2 * nslots + q],
                           sm[3 * nslots + q], sm[4 * nslots + q], sm[5 * nslots + q],
                           sm[6 * nslots + q], sm[7 * nslots + q], sm[8 * nslots + q]);
        }
    }
    primal_finish(W, b, s);
}

// Value of component k (the slots' order: gradient x y z, Hessian xx yy zz,
// xy xz yz) of a particle system.
__device__ __forceinline__ float sys3_component(const Sys3& s, int k) {
    return k == 0 ? s.r[0] : k == 1 ? s.r[1] : k == 2 ? s.r[2] : k == 3 ? s.a[0][0] : k == 4 ? s.a[1][1]
         : k == 5 ? s.a[2][2] : k == 6 ? s.a[1][0] : k == 7 ? s.a[2][0] : s.a[2][1];
}

// Finish of the particles [v, vend) of a flat chunk whose terms sit in the
// slots, L lanes per particle (L in 1, 3, 9; 32 / L particles per warp): lane
// `sub` of a particle's group adds components [sub * 9/L, (sub + 1) * 9/L) of
// its terms, each in incidence order from the inertia's value, so every sum
// is the one a single lane makes; the group's first lane gathers the nine
// sums by shuffles and solves.  A particle with force or manifold rows, or a
// rigid body, is finished by its first lane alone.  The loop bound is
// uniform over each warp, so the shuffles run with the whole warp.
template <int L>
static __device__ __noinline__ void flat_finish_split(const Team& T, const World& W, int cur, const int* list,
                                                  const int* tinc, int base, int v, int vend, float alpha,
                                                  bool write_stick, const float* sm, int nslots) {
    constexpr int G = 32 / L, C = 9 / L;
    const int lane = T.rank & 31, grp = lane / L, sub = lane - grp * L;
    const int stride = (T.size >> 5) * G;
    for (int j0 = v + (T.rank >> 5) * G; j0 < vend; j0 += stride) {
        const int j = j0 + grp;
        int b = -1;
        if (grp < G && j < vend) {
            b = list[j];
            if (W.flags[b] & kBodyRemoved) b = -1;
        }
        bool lean = false;
        int e0 = 0, e1 = 0, q0 = 0;
        float acc[C];
#pragma unroll
        for (int k = 0; k < C; ++k) acc[k] = 0.f;
        if (b >= 0) {
            e0 = W.inc_off[b];
            e1 = e0 + W.inc_cnt[b];
            q0 = (j == 0 ? 0 : tinc[j - 1]) - base;
            const int nterm = tinc[j] - base - q0;
            lean = e1 - e0 == nterm && energy_only_particle(W, b);
            if (lean) {
                Sys3 s;
                particle_init_mass(W, b, s);
#pragma unroll
                for (int k = 0; k < C; ++k) acc[k] = sys3_component(s, sub * C + k);
                for (int q = q0; q < q0 + nterm; ++q)
#pragma unroll
                    for (int k = 0; k < C; ++k) acc[k] = XADD(acc[k], sm[(sub * C + k) * nslots + q]);
            }
        }
        float f[9];
        if constexpr (L == 1) {
#pragma unroll
            for (int k = 0; k < 9; ++k) f[k] = acc[k];
        } else {
#pragma unroll
            for (int s = 0; s < L; ++s)
#pragma unroll
                for (int k = 0; k < C; ++k) f[s * C + k] = __shfl_sync(0xffffffffu, acc[k], grp * L + s);
        }
        if (b >= 0 && sub == 0) {
            if (lean) {
                Sys3 s;
                s.r[0] = f[0]; s.r[1] = f[1]; s.r[2] = f[2];
                s.a[0][0] = f[3]; s.a[1][1] = f[4]; s.a[2][2] = f[5];
                s.a[1][0] = f[6]; s.a[2][0] = f[7]; s.a[2][1] = f[8];
                s.a[0][1] = 0.f; s.a[0][2] = 0.f; s.a[1][2] = 0.f;
                particle_finish(W, b, s);
            } else {
                flat_finish_body(W, cur, b, e0, e1, q0, alpha, write_stick, sm, nslots);
            }
        }
    }
}

static __device__ __noinline__ void primal_sweep_flat(const Team& T, const World& W, int cur, const int* list,
                                               const int* tinc, size_t rec0, int c0, int c1, float alpha,
                                               bool write_stick) {
    float* sm = reinterpret_cast<float*>(T.stage);
    const int nslots = T.stage_cap * 4 / 9;
    const int tid = T.rank, nt = T.size;
    for (int v = c0; v < c1;) {
        const int base = v == 0 ? 0 : tinc[v - 1];
        // the longest run of particles [v, vend) whose terms fit the slots (at least one)
        int vend = c1;
        if (tinc[c1 - 1] - base > nslots) {
            int lo = v + 1, hi = c1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (tinc[mid - 1] - base <= nslots) lo = mid;
                else hi = mid - 1;
            }
            vend = lo;
        }
        const int total = tinc[vend - 1] - base;
        const bool flat = total <= nslots;
        if (flat) {
            for (int q = tid; q < total; q += nt) {
                V3 g = v3(0.f, 0.f, 0.f);
                S3 H;
                s3_zero(H);
                tet_term_record(W, rec0 + base + q, g, H);   // removed tets stay zero
                sm[0 * nslots + q] = g.x; sm[1 * nslots + q] = g.y; sm[2 * nslots + q] = g.z;
                sm[3 * nslots + q] = H.xx; sm[4 * nslots + q] = H.yy; sm[5 * nslots + q] = H.zz;
                sm[6 * nslots + q] = H.xy; sm[7 * nslots + q] = H.xz; sm[8 * nslots + q] = H.yz;
            }
            T.sync();
        }
        if (!flat) {
            // one particle whose terms alone exceed the slots: evaluated in place
            for (int j = v + tid; j < vend; j += nt) {
                const int b = list[j];
                if (W.flags[b] & kBodyRemoved) continue;
                flat_finish_body(W, cur, b, W.inc_off[b], W.inc_off[b] + W.inc_cnt[b], -1, alpha, write_stick, sm,
                                 nslots);
            }
        } else {
            // as many lanes per particle as keep the team busy in one pass
            const int np = vend - v, nw = nt >> 5;
            if (np <= 3 * nw)
                flat_finish_split<9>(T, W, cur, list, tinc, base, v, vend, alpha, write_stick, sm, nslots);
            else if (np <= 10 * nw)
                flat_finish_split<3>(T, W, cur, list, tinc, base, v, vend, alpha, write_stick, sm, nslots);
            else
                flat_finish_split<1>(T, W, cur, list, tinc, base, v, vend, alpha, write_stick, sm, nslots);
        }
        T.sync();
        v = vend;
    }
}

// One colour of a scene's primal sweep, by the scene's lane grouping.
__device__ __forceinline__ void primal_colour(const Team& T, const World& W, const SceneDesc& sc, int cur,
                                              const int* cs, int c, float alpha, bool write_stick) {
    if (sc.group == kGroupFlat)
        primal_sweep_flat(T, W, cur, W.col_list + sc.body0, W.col_tinc + sc.body0, 4 * (size_t)sc.tet0,
                          cs[c], cs[c + 1], alpha, write_stick);
    else
        primal_sweep_cta_dispatch(T, W, cur, W.col_list + sc.body0 + cs[c], cs[c + 1] - cs[c], alpha, write_stick,
                                  sc.group);
}

static __device__ __noinline__ bool colour_scene(const Team& T, const World& W, const SceneDesc& sc, SceneState* st,
                                          int scene, int cur);

// Per-scene device timing (W.scene_ns set): the global timer when the team
// reaches stamp k of the scene's step (0 start, 1 broadphase done, 2
// narrowphase, 3 joint/spring warm start and incidence, 4 colouring, 5
// prediction, 6 iterations, 7 velocities and removals, 8 end).
__device__ __forceinline__ void scene_stamp(const World& W, const Team& T, int scene, int k) {
    if (W.scene_ns && T.rank == 0) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        W.scene_ns[(size_t)kSceneStamps * scene + k] = t;
    }
}

// Keeps the previous step's colouring when the contact graph is unchanged:
// the same number of live manifolds in both tables, every live one already
// live last step, and no force or body removed since the colouring was made.
// The colouring is a deterministic function of that graph, so reusing it is
// exact.
static __device__ bool colour_scene_cached(const Team& T, const World& W, const SceneDesc& sc, SceneState* st, int scene,
                                    int cur) {
    const int old = cur ^ 1;
    const bool reuse = st->colours_valid && st->nlive[cur] == st->nlive[old] && st->nmatched == st->nlive[cur] &&
                       st->topo == st->coloured_topo;
    T.sync();
    if (reuse) return true;
    const bool ok = colour_scene(T, W, sc, st, scene, cur);
    if (T.rank == 0) {
        st->colours_valid = ok ? 1 : 0;
        st->coloured_topo = st->topo;
    }
    T.sync();
    return ok;
}

// Live incidence entries of body b: the forces and energies it takes part in.
__device__ __forceinline__ int live_degree(const World& W, int b) {
    const int e0 = W.inc_off[b], e1 = e0 + W.inc_cnt[b];
    int n = 0;
    for (int e = e0; e < e1; ++e) {
        const uint32_t ent = W.inc[e];
        const uint32_t kind = ent_kind(ent), idx = ent_index(ent);
        if (kind == kEntManifold) ++n;
        else if (kind == kEntForce) n += (W.ftype[idx] & kForceRemoved) ? 0 : 1;
        else if (kind == kEntTet) n += W.tparam[idx].w != 0.f ? 0 : 1;
        else n += W.rparam[idx].w != 0.f ? 0 : 1;
    }
    return n;
}

// Colouring priority: body u precedes body v.  Pass 0: larger live degree
// (W.cntB) first, then (hash(local index), local index); pass 1 (iterated
// greedy): larger pass-0 colour (W.bcur) first, then as pass 0.
__device__ __forceinline__ bool colour_before(const World& W, int pass, int u, int v) {
    if (pass == 1) {
        const int pu = W.bcur[u], pv = W.bcur[v];
        if (pu != pv) return pu > pv;
    }
    const int du = W.cntB[u], dv = W.cntB[v];
    if (du != dv) return du > dv;
    const int lu = W.local[u], lv = W.local[v];
    return prio_less(colour_priority((uint32_t)lu), lu, colour_priority((uint32_t)lv), lv);
}

// Resumable scan state of a body in a Jones-Plassmann pass, in per-body
// scratch the colouring does not otherwise use (the broadphase refills it
// next step): W.cand_off the next incidence entry to scan (bit 30: a
// neighbour holds a colour >= 64), W.cand_cnt / W.col_tinc the low / high
// words of the mask of colours < 64 seen so far.
constexpr int kJpWide = 1 << 30;

__device__ __forceinline__ void jp_scan_reset(const World& W, int b) {
    W.cand_off[b] = W.inc_off[b];
    W.cand_cnt[b] = 0;
    W.col_tinc[b] = 0;
}

// Scans body b's incidence from its saved entry: colours of coloured
// neighbours go into the mask (they all precede b: a follower waits for
// b), and the scan stops at the first entry holding an uncoloured neighbour
// that precedes b.  True when every entry was scanned (b is ready).
__device__ __forceinline__ bool jp_scan(const World& W, int cur, int pass, int b, volatile const int* col,
                                        unsigned long long& used, bool& wide) {
    int pos = W.cand_off[b];
    wide = (pos & kJpWide) != 0;
    int e = pos & ~kJpWide;
    used = (unsigned long long)(uint32_t)W.cand_cnt[b] | ((unsigned long long)(uint32_t)W.col_tinc[b] << 32);
    const int e1 = W.inc_off[b] + W.inc_cnt[b];
    bool ready = true;
    auto visit = [&](int n) {
        if (!ready || n < 0 || n == b) return;
        const int cn = col[n];
        if (cn == -2) return;
        if (cn >= 0) {
            if (cn < 64) used |= 1ull << cn;
            else wide = true;
            return;
        }
        if (colour_before(W, pass, n, b)) ready = false;
    };
    for (; e < e1; ++e) {
        const uint32_t ent = W.inc[e];
        const uint32_t kind = ent_kind(ent), idx = ent_index(ent);
        if (kind == kEntManifold) {
            const int2 ab = W.cpair[cur][idx];
            visit(ab.x == b ? ab.y : ab.x);
        } else if (kind == kEntForce) {
            if (W.ftype[idx] & kForceRemoved) continue;
            const int2 ab = W.fbody[idx];
            visit(ab.x == b ? ab.y : ab.x);
        } else if (kind == kEntTet) {
            if (W.tparam[idx].w != 0.f) continue;
            const int4 v = W.tidx[idx];
            visit(v.x); visit(v.y); visit(v.z); visit(v.w);
        } else {
            if (W.rparam[idx].w != 0.f) continue;
            const int4 v = W.ridx[idx];
            visit(v.x); visit(v.y); visit(v.z);
        }
        if (!ready) break;   // resume at this entry (its colours, seen again, change nothing)
    }
    W.cand_off[b] = e | (wide ? kJpWide : 0);
    W.cand_cnt[b] = (int)(uint32_t)used;
    W.col_tinc[b] = (int)(uint32_t)(used >> 32);
    return ready;
}

// One Jones-Plassmann pass over the scene's uncoloured (-1) bodies: a body
// takes the smallest colour its preceding neighbours do not use once they
// are all coloured, which equals sequential greedy colouring in priority
// order whatever the thread schedule.  A body's scan resumes each round at
// the entry that held it up (jp_scan), so a pass reads each incidence entry
// about once.  False (status TIMEOUT) if it stalls.
static __device__ bool jp_pass(const Team& T, const World& W, const SceneDesc& sc, SceneState* st, int cur, int pass) {
    int& s_remaining = T.sh->remaining;
    int& s_progress = T.sh->progress;
    int& s_maxc = T.sh->maxc;
    const int tid = T.rank, nt = T.size;
    const int b0 = sc.body0, b1 = sc.body0 + sc.nbody;
    volatile int* col = W.colour;
    const int max_rounds = sc.nbody + 2;
    for (int b = b0 + tid; b < b1; b += nt) jp_scan_reset(W, b);
    T.sync();
    for (int round = 0;; ++round) {
        if (tid == 0) { s_remaining = 0; s_progress = 0; }
        T.sync();
        for (int b = b0 + tid; b < b1; b += nt) {
            if (col[b] != -1) continue;
            unsigned long long used;
            bool wide;
            if (!jp_scan(W, cur, pass, b, col, used, wide)) { s_remaining = 1; continue; }
            int chosen = ~used ? __ffsll((long long)~used) - 1 : -1;
            if (chosen < 0 || wide) {
                // some neighbour holds a colour >= 64: first fit over 64-colour windows
                chosen = -1;
                for (int base = 0; base < kMaxColours && chosen < 0; base += 64) {
                    unsigned long long w = 0ull;
                    for_each_neighbour(W, cur, b, [&](int n) {
                        const int cn = col[n];
                        if (cn < base || cn >= base + 64) return;
                        if (colour_before(W, pass, n, b)) w |= 1ull << (cn - base);
                    });
                    if (~w) chosen = base + __ffsll((long long)~w) - 1;
                }
            }
            if (chosen < 0 || chosen >= kMaxColours) {
                st->status = kStatusCapacity;
                chosen = kMaxColours - 1;
            }
            col[b] = chosen;
            atomicMax(&s_maxc, chosen + 1);
            s_progress = 1;
        }
        T.sync();
        const int remaining = s_remaining, progress = s_progress;
        T.sync();   // every thread has read the flags before thread 0 resets them
        if (!remaining) return true;
        if (!progress || round > max_rounds) {
            if (tid == 0) st->status = kStatusTimeout;
            T.sync();
            return false;
        }
    }
}

// Returns false (status TIMEOUT or CAPACITY set) if colouring could not finish.
// The colour counts live in the team's stage (at least kMaxColours + 1 ints).
// Priorities read W.cntB and W.bcur, free once the incidence is built.
static __device__ __noinline__ bool colour_scene(const Team& T, const World& W, const SceneDesc& sc, SceneState* st,
                                          int scene, int cur) {
    int& s_maxc = T.sh->maxc;
    int* s_count = reinterpret_cast<int*>(T.stage);
    const int tid = T.rank, nt = T.size;
    const int b0 = sc.body0, b1 = sc.body0 + sc.nbody;
    volatile int* col = W.colour;
    for (int b = b0 + tid; b < b1; b += nt) {
        col[b] = (W.flags[b] & (kBodyStatic | kBodyRemoved)) ? -2 : -1;
        W.cntB[b] = live_degree(W, b);
    }
    if (tid == 0) s_maxc = 0;
    T.sync();
    if (!jp_pass(T, W, sc, st, cur, 0)) return false;
    for (int b = b0 + tid; b < b1; b += nt) {
        const int c = col[b];
        W.bcur[b] = c;
        if (c >= 0) col[b] = -1;
    }
    if (tid == 0) s_maxc = 0;
    T.sync();
    if (!jp_pass(T, W, sc, st, cur, 1)) return false;
    const int ncol = s_maxc;
    T.sync();
    // colour lists: counting sort of the dynamic bodies by colour
    for (int c = tid; c <= ncol; c += nt) s_count[c] = 0;
    T.sync();
    for (int b = b0 + tid; b < b1; b += nt) {
        const int c = col[b];
        if (c >= 0) atomicAdd(&s_count[c], 1);
    }
    T.sync();
    int* cs = W.col_start + (size_t)scene * (kMaxColours + 1);
    if (tid == 0) {
        int acc = 0;
        for (int c = 0; c < ncol; ++c) { cs[c] = acc; acc += s_count[c]; s_count[c] = cs[c]; }
        cs[ncol] = acc;
        st->ncolours = ncol;
    }
    T.sync();
    // Within a colour, bodies are ordered by decreasing work (incidence entries
    // per lane of a body group), so the bodies sharing a warp take similar
    // time.  Bodies of one colour share no constraint, so their order within
    // the colour does not change any result.
    const int g = (sc.group > 0 && sc.group <= 32) ? sc.group : 1;
    for (int key = kColourWorkBuckets - 1; key >= 0; --key) {
        for (int b = b0 + tid; b < b1; b += nt) {
            const int c = col[b];
            if (c < 0) continue;
            const int k = min(kColourWorkBuckets - 1, (W.inc_cnt[b] + g - 1) / g);
            if (k != key) continue;
            const int at = atomicAdd(&s_count[c], 1);
            if (AVBD_CHECK(W, at >= 0 && at < sc.nbody, 4, at, sc.nbody)) W.col_list[b0 + at] = b;
        }
        T.sync();
    }
    if (sc.group == kGroupFlat) {
        // inclusive prefix of tet terms over the list
        const int n = cs[ncol];
        int* tinc = W.col_tinc + b0;
        for (int i = tid; i < n; i += nt) tinc[i] = tet_terms(W, W.col_list[b0 + i]);
        T.sync();
        block_exclusive_scan(T, tinc, tinc, n);
        // the tet-term records of every listed particle, in list order
        const size_t rec0 = 4 * (size_t)sc.tet0;
        for (int i = tid; i < n; i += nt) {
            const int b = W.col_list[b0 + i];
            const int k = tet_terms(W, b);
            const uint32_t* ent = W.inc + W.inc_off[b] + W.inc_cnt[b] - k;
            const int q0 = tinc[i];
            if (!AVBD_CHECK(W, q0 + k <= 4 * sc.ntet, 5, q0 + k, 4 * sc.ntet)) continue;
            for (int e = 0; e < k; ++e) write_term_record(W, rec0 + q0 + e, ent[e]);
            tinc[i] = q0 + k;
        }
        T.sync();
    }
    return st->status == kStatusOk;
}

// Phase loops of one scene kept out of line, so each gets its own register
// allocation instead of the union of every inlined phase.
//
// Narrowphase in two passes.  Most candidate pairs (bounding spheres that
// overlap) are separated by an axis, and a pair that touches costs several
// times more (clipping, contact matching and writes); with one pair per lane,
// a warp would wait on its few touching lanes at every turn.  So the first
// pass runs the separating-axis test on every pair and lists the pairs that
// touch, warp by warp, and the second pass makes their manifolds with every
// lane busy.  The list borrows the other table's live list, which nothing
// reads again before this step's narrowphase rewrites that table's slots.
static __device__ __noinline__ void narrowphase_cta(const Team& T, const World& W, const SceneDesc& sc, SceneState* st,
                                             int cur, int ncand, int old_count) {
    int* pend = W.live[cur ^ 1] + sc.cand0;
    const int lane = threadIdx.x & 31;
    for (int c0 = sc.cand0; c0 < sc.cand0 + ncand; c0 += T.size) {   // uniform over the team's warps
        const int c = c0 + T.rank;
        bool touch = false;
        if (c < sc.cand0 + ncand) {
            const int2 ab = W.cpair[cur][c];
            const float4 pa = W.pos[ab.x], pb = W.pos[ab.y];
            float sign;
            touch = box_box_sat(xrotmat(q4(W.rot[ab.x])), v3(W.scale[ab.x]), xrotmat(q4(W.rot[ab.y])),
                                v3(W.scale[ab.y]), xsub(v3(pb), v3(pa)), sign) >= 0;
            if (!touch) W.cn[cur][c] = 0;
        }
        const unsigned m = __ballot_sync(0xffffffffu, touch);
        if (m) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&st->npend, __popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            const int at = base + __popc(m & ((1u << lane) - 1u));
            if (touch && AVBD_CHECK(W, at < ncand, 7, at, ncand)) pend[at] = c;
        }
    }
    T.sync();
    const int npend = __ldcg(&st->npend);
    for (int i = T.rank; i < npend; i += T.size) narrowphase_slot(W, sc, st, __ldcg(pend + i), cur, old_count);
}

// Returns true if this thread saw a force fracture.  Manifolds come from the
// step's live list (each manifold's dual is independent of the others).
static __device__ __noinline__ bool dual_cta(const Team& T, const World& W, const SceneDesc& sc, int cur, int nlive,
                                      bool last) {
    bool broke = false;
    for (int f = sc.force0 + T.rank; f < sc.force0 + sc.nforce; f += T.size)
        if (dual_force(W, f, W.P.alpha)) broke = true;
    const int* live = W.live[cur] + sc.cand0;
    for (int i = T.rank; i < nlive; i += T.size) dual_manifold(W, cur, live[i], W.P.alpha, last);
    return broke;
}

// ---------------------------------------------------------------------------
// Uniform-grid broadphase of one scene (the same candidate set and order as
// the all-pairs loop of broadphase_body, found in about O(n) instead of
// O(n^2)).  Cells are 2R wide, R the largest detection radius, so two
// overlapping spheres (distance < r_i + r_j <= 2R) sit in the same or
// adjacent cells; each body tests the bodies of its 27 neighbouring cells
// with the exact sphere test and the joint/spring filter, and its candidate
// list is sorted by partner index, as the reference's nested loop emits it.
// Scratch: the team's stage after the staged poses (cell starts, 16-bit
// items) when it fits, else W.bcur and W.cntB; W.cand_off holds each body's
// rank in its cell before it takes the candidate offsets.  Returns the
// candidate count; writes the pairs when they fit candcap; returns -1 when
// the extents are not finite (the caller then uses the all-pairs loop).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ord_float(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float unord_float(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__device__ __forceinline__ float4 body_sphere(const World& W, const SceneDesc& sc, const float4* sp, int li) {
    if (sp) return sp[li];
    const int b = sc.body0 + li;
    float4 p = W.pos[b];
    p.w = (W.flags[b] & kBodyRemoved) ? -INFINITY : W.scale[b].w;
    return p;
}

struct GridDims {
    float minx, miny, minz, inv_h;
    int nx, ny, nz;
    __device__ __forceinline__ int cell_axis(float v, float mn, int n) const {
        const int c = (int)((v - mn) * inv_h);
        return c < 0 ? 0 : (c >= n ? n - 1 : c);
    }
    __device__ __forceinline__ int cell(const float4& p) const {
        return (cell_axis(p.z, minz, nz) * ny + cell_axis(p.y, miny, ny)) * nx + cell_axis(p.x, minx, nx);
    }
};

// Cell starts (ncell + 1) and cell items (body local indices) of the grid:
// in shared memory after the staged poses when they fit, else in per-body
// scratch (W.bcur, W.cntB); plus the scene's big bodies (radius above rbig),
// which stay out of the grid.
struct GridCells {
    const int* cstart;
    const unsigned short* items16;   // shared-memory items
    const int* items32;              // global items
    const int* big;                  // local indices of the big bodies
    int nbig;
    float rbig;
    __device__ __forceinline__ int item(int k) const { return items16 ? (int)items16[k] : items32[k]; }
};

// True when (li, lj), lj > li, is a broadphase candidate: the reference's
// sphere test and no live joint/spring between them (isConstrainedTo).
__device__ __forceinline__ bool grid_pair(const World& W, const SceneDesc& sc, const float4* sp, const float4& pi,
                                          const Partners& pp, int lj) {
    const float4 pj = body_sphere(W, sc, sp, lj);
    if (!sphere_overlap_fast(pi, pj, pi.w, pj.w)) return false;
    return !pair_constrained(W, pp, sc.body0 + lj);
}

// SORTED: the caller visits partners in increasing order, so a candidate is
// appended; otherwise it is inserted in partner order, as the all-pairs loop
// emits them.
template <bool WRITE, bool SORTED = false>
__device__ __forceinline__ void grid_test(const World& W, const SceneDesc& sc, const float4* sp, const float4& pi,
                                          const Partners& pp, int li, int lj, int2* out, int& n) {
    if (lj <= li) return;
    if (!grid_pair(W, sc, sp, pi, pp, lj)) return;
    if (WRITE) {
        const int bi = sc.body0 + li, bj = sc.body0 + lj;
        int j = n - 1;
        if (!SORTED)
            while (j >= 0 && out[j].y > bj) { out[j + 1] = out[j]; --j; }
        out[j + 1] = make_int2(bi, bj);
    }
    ++n;
}

// A big body's all-pairs row by the whole team: each chunk of partners is
// tested one per thread and its candidates placed by a team-wide count, so
// the row comes out in partner order (as the all-pairs loop emits it)
// without one thread walking it.  Returns the row's candidates.
template <bool WRITE>
__device__ int big_row(const Team& T, const World& W, const SceneDesc& sc, const float4* sp, int li, int2* out) {
    const int lane = T.rank & 31, warp = T.rank >> 5, nwarps = T.size >> 5;
    const float4 pi = body_sphere(W, sc, sp, li);
    const Partners pp = partners_of(W, sc.body0 + li);
    if (T.rank == 0) T.sh->carry = 0;
    T.sync();
    if (!isinf(pi.w)) {
        for (int c0 = li + 1; c0 < sc.nbody; c0 += T.size) {
            const int lj = c0 + T.rank;
            const bool hit = lj < sc.nbody && grid_pair(W, sc, sp, pi, pp, lj);
            const unsigned bal = __ballot_sync(kFull, hit);
            if (lane == 0) T.sh->warp_tot[warp] = __popc(bal);
            T.sync();
            int before = T.sh->carry, chunk = 0;
            for (int w = 0; w < nwarps; ++w) {
                const int c = T.sh->warp_tot[w];
                if (w < warp) before += c;
                chunk += c;
            }
            if (WRITE && hit)
                out[before + __popc(bal & ((1u << lane) - 1u))] = make_int2(sc.body0 + li, sc.body0 + lj);
            T.sync();
            if (T.rank == 0) T.sh->carry += chunk;
            T.sync();
        }
    }
    const int total = T.sh->carry;
    T.sync();
    return total;
}

// Candidates of a small body (big bodies' rows come from big_row).
template <bool WRITE>
__device__ __forceinline__ int grid_candidates(const World& W, const SceneDesc& sc, const float4* sp, const GridDims& g,
                                               const GridCells& gc, int li, int2* out) {
    const float4 pi = body_sphere(W, sc, sp, li);
    if (isinf(pi.w)) return 0;
    const Partners pp = partners_of(W, sc.body0 + li);
    int n = 0;
    if (pi.w > gc.rbig) {
        // a big body: its all-pairs row, in partner order
        for (int lj = li + 1; lj < sc.nbody; ++lj) grid_test<WRITE, true>(W, sc, sp, pi, pp, li, lj, out, n);
        return n;
    }
    const int cx = g.cell_axis(pi.x, g.minx, g.nx), cy = g.cell_axis(pi.y, g.miny, g.ny),
              cz = g.cell_axis(pi.z, g.minz, g.nz);
    for (int z = max(cz - 1, 0); z <= min(cz + 1, g.nz - 1); ++z)
        for (int y = max(cy - 1, 0); y <= min(cy + 1, g.ny - 1); ++y) {
            const int row = (z * g.ny + y) * g.nx;
            // the three cells of a row are contiguous in the item list
            const int k0 = gc.cstart[row + max(cx - 1, 0)], k1 = gc.cstart[row + min(cx + 1, g.nx - 1) + 1];
            for (int k = k0; k < k1; ++k) grid_test<WRITE>(W, sc, sp, pi, pp, li, gc.item(k), out, n);
        }
    for (int k = 0; k < gc.nbig; ++k) grid_test<WRITE>(W, sc, sp, pi, pp, li, gc.big[k], out, n);
    return n;
}

static __device__ __noinline__ int broadphase_grid(const Team& T, const World& W, const SceneDesc& sc, int cur,
                                            const float4* sp) {
    const int tid = T.rank, nt = T.size, n = sc.nbody, b0 = sc.body0;
    int* red = T.sh->red;
    // 1. smallest radius; bodies above 8x it are "big" and stay out of the grid
    if (tid == 0) red[7] = ord_float(INFINITY);
    T.sync();
    {
        float rmin = INFINITY;
        for (int li = tid; li < n; li += nt) {
            const float4 p = body_sphere(W, sc, sp, li);
            if (!isinf(p.w)) rmin = fminf(rmin, p.w);
        }
        atomicMin(&red[7], ord_float(rmin));
    }
    T.sync();
    const float rbig = 8.f * unord_float(red[7]);
    T.sync();
    // 2. extents and largest radius of the small bodies; the big ones listed
    int* big = T.sh->big;
    if (tid == 0) {
        red[0] = red[1] = red[2] = ord_float(INFINITY);
        red[3] = red[4] = red[5] = ord_float(-INFINITY);
        red[6] = ord_float(0.f);
        T.sh->nbig = 0;
    }
    T.sync();
    {
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY}, mr = 0.f;
        for (int li = tid; li < n; li += nt) {
            const float4 p = body_sphere(W, sc, sp, li);
            if (isinf(p.w)) continue;
            if (p.w > rbig) {
                const int k = atomicAdd(&T.sh->nbig, 1);
                if (k < kGridMaxBig) big[k] = li;
                continue;
            }
            mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
            mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
            mr = fmaxf(mr, p.w);
        }
        for (int a = 0; a < 3; ++a) {
            atomicMin(&red[a], ord_float(mn[a]));
            atomicMax(&red[3 + a], ord_float(mx[a]));
        }
        atomicMax(&red[6], ord_float(mr));
    }
    T.sync();
    GridDims g;
    g.minx = unord_float(red[0]); g.miny = unord_float(red[1]); g.minz = unord_float(red[2]);
    const float ex = unord_float(red[3]) - g.minx, ey = unord_float(red[4]) - g.miny,
                ez = unord_float(red[5]) - g.minz;
    const float R = unord_float(red[6]);
    const int nbig = T.sh->nbig;
    T.sync();   // red[] and the count are read by every thread before they are reused
    if (!(ex >= 0.f && ey >= 0.f && ez >= 0.f) || !(ex < 1e30f && ey < 1e30f && ez < 1e30f) || !(R < 1e30f) ||
        !(rbig < 1e30f) || nbig > kGridMaxBig)
        return -1;   // nothing small, non-finite extents or many big bodies: the all-pairs loop
    // at most n / 2 cells, so the cell table fits beside the items
    const int maxcell = max(1, n / 2);
    float h = fmaxf(2.f * R * 1.0001f, 1e-6f);
    for (int it = 0; it < 64; ++it) {
        g.nx = (int)(ex / h) + 1; g.ny = (int)(ey / h) + 1; g.nz = (int)(ez / h) + 1;
        if ((long long)g.nx * g.ny * g.nz <= maxcell) break;
        h *= 1.25f;
    }
    if ((long long)g.nx * g.ny * g.nz > maxcell) return -1;
    g.inv_h = 1.f / h;
    const int ncell = g.nx * g.ny * g.nz;
    // shared layout after the staged poses: int cstart[ncell + 1], ushort items[n]
    const size_t used = sp ? (size_t)n * sizeof(float4) : 0;
    const size_t need = (size_t)(ncell + 1) * sizeof(int) + (size_t)n * sizeof(unsigned short);
    const bool in_smem = used + need <= (size_t)T.stage_cap * sizeof(float4) && n < 65536;
    int* cstart = in_smem ? reinterpret_cast<int*>(reinterpret_cast<char*>(T.stage) + used) : W.bcur + b0;
    unsigned short* items16 = in_smem ? reinterpret_cast<unsigned short*>(cstart + ncell + 1) : nullptr;
    int* items32 = W.cntB + b0;
    int* rank = W.cand_off + b0;   // a body's rank within its cell
    for (int c = tid; c <= ncell; c += nt) cstart[c] = 0;
    T.sync();
    for (int li = tid; li < n; li += nt) {
        const float4 p = body_sphere(W, sc, sp, li);
        if (isinf(p.w) || p.w > rbig) continue;
        rank[li] = atomicAdd(&cstart[g.cell(p)], 1);
    }
    T.sync();
    const int placed = block_exclusive_scan(T, cstart, cstart, ncell);
    if (tid == 0) cstart[ncell] = placed;
    for (int li = tid; li < n; li += nt) {
        const float4 p = body_sphere(W, sc, sp, li);
        if (isinf(p.w) || p.w > rbig) continue;
        const int k = cstart[g.cell(p)] + rank[li];
        if (in_smem) items16[k] = (unsigned short)li;
        else items32[k] = li;
    }
    T.sync();
    GridCells gc;
    gc.cstart = cstart;
    gc.items16 = in_smem ? items16 : nullptr;
    gc.items32 = items32;
    gc.big = big;
    gc.nbig = nbig;
    gc.rbig = rbig;
    auto is_big = [&](int li) {
        const float4 p = body_sphere(W, sc, sp, li);
        return !isinf(p.w) && p.w > rbig;
    };
    for (int li = tid; li < n; li += nt)
        if (!is_big(li)) W.cand_cnt[b0 + li] = grid_candidates<false>(W, sc, sp, g, gc, li, nullptr);
    for (int k = 0; k < nbig; ++k) {
        const int cnt = big_row<false>(T, W, sc, sp, big[k], nullptr);
        if (tid == 0) W.cand_cnt[b0 + big[k]] = cnt;
    }
    T.sync();
    const int ncand = block_exclusive_scan(T, W.cand_cnt + b0, W.cand_off + b0, n);
    if (ncand > sc.candcap) return ncand;
    for (int li = tid; li < n; li += nt) {
        if (is_big(li)) continue;
        const int wrote = grid_candidates<true>(W, sc, sp, g, gc, li, W.cpair[cur] + sc.cand0 + W.cand_off[b0 + li]);
        AVBD_CHECK(W, wrote == W.cand_cnt[b0 + li], 3, wrote, W.cand_cnt[b0 + li]);
    }
    for (int k = 0; k < nbig; ++k)
        big_row<true>(T, W, sc, sp, big[k], W.cpair[cur] + sc.cand0 + W.cand_off[b0 + big[k]]);
    T.sync();
    return ncand;
}

// ---------------------------------------------------------------------------
// Whole step of one scene by one team (batched path).
// ---------------------------------------------------------------------------
static __device__ void scene_step(const World& W, int scene, const Team& T) {
    const SceneDesc sc = W.scenes[scene];
    SceneState* st = W.sstate + scene;
    const int tid = T.rank, nt = T.size;
    int& s_flags = T.sh->flags;
    if (st->status != kStatusOk && st->status != kStatusCapacity && st->status != kStatusTimeout) return;
    T.sync();
    if (tid == 0) { st->status = kStatusOk; st->need_cand = 0; st->need_k = 0; st->need_inc = 0; }
    const int old = st->cur, cur = old ^ 1;
    const int b0 = sc.body0, b1 = sc.body0 + sc.nbody;
    // 1. broadphase: count, scan, capacity check, write; positions and radii
    //    staged in shared memory when the scene fits
    float4* s_bodies = T.stage;
    const bool staged = sc.nbody <= T.stage_cap;
    if (staged) {
        for (int b = b0 + tid; b < b1; b += nt) {
            float4 p = W.pos[b];
            p.w = (W.flags[b] & kBodyRemoved) ? -INFINITY : W.scale[b].w;
            s_bodies[b - b0] = p;
        }
        T.sync();
    }
    int ncand = (W.grid_min > 0 && sc.nbody >= W.grid_min) ? broadphase_grid(T, W, sc, cur, staged ? s_bodies : nullptr)
                                                             : -1;
    if (ncand < 0) {
        for (int b = b0 + tid; b < b1; b += nt)
            W.cand_cnt[b] = staged ? broadphase_body_staged(W, sc, b, s_bodies, nullptr, 0)
                                   : broadphase_body(W, sc, b, nullptr, 0);
        T.sync();
        ncand = block_exclusive_scan(T, W.cand_cnt + b0, W.cand_off + b0, sc.nbody);
        if (ncand <= sc.candcap) {
            for (int b = b0 + tid; b < b1; b += nt) {
                int2* out = W.cpair[cur] + sc.cand0 + W.cand_off[b];
                if (staged) broadphase_body_staged(W, sc, b, s_bodies, out, W.cand_cnt[b]);
                else broadphase_body(W, sc, b, out, W.cand_cnt[b]);
            }
        }
    }
    if (ncand > sc.candcap) {
        if (tid == 0) {
            st->status = kStatusCapacity;
            st->need_cand = ncand;
            if (W.fail_count) atomicAdd(W.fail_count, 1);
        }
        return;
    }
    if (tid == 0) { st->kused[cur] = 0; st->nlive[cur] = 0; st->nmatched = 0; st->npend = 0; }
    T.sync();
    scene_stamp(W, T, scene, 1);
    // 2. narrowphase + manifold warm start into the other table
    const int old_count = st->ncand[old];
    narrowphase_cta(T, W, sc, st, cur, ncand, old_count);
    T.sync();
    if (st->need_k) {
        if (tid == 0) {
            st->status = kStatusCapacity;
            st->need_k = st->kused[cur];
            if (W.fail_count) atomicAdd(W.fail_count, 1);
        }
        return;
    }
    if (tid == 0) { st->ncand[cur] = ncand; st->cur = cur; }
    scene_stamp(W, T, scene, 2);
    // 2b. joints / springs warm start
    for (int f = sc.force0 + tid; f < sc.force0 + sc.nforce; f += nt)
        if (force_init(W, f)) atomicAdd(&st->topo, 1);
    T.sync();
    // incidence
    if (!build_incidence(T, W, sc, st, cur)) {
        if (tid == 0) {
            st->status = kStatusCapacity;
            if (W.fail_count) atomicAdd(W.fail_count, 1);
        }
        return;
    }
    scene_stamp(W, T, scene, 3);
    // colouring
    if (!colour_scene_cached(T, W, sc, st, scene, cur)) return;
    scene_stamp(W, T, scene, 4);
    // 4. prediction
    for (int b = b0 + tid; b < b1; b += nt) predict_body(W, b);
    T.sync();
    const int ncol = st->ncolours;
    const int nlive = st->nlive[cur];
    const int* cs = W.col_start + (size_t)scene * (kMaxColours + 1);
    scene_stamp(W, T, scene, 5);
    // 5. iterations
    for (int it = 0; it < W.P.num_iterations; ++it) {
        for (int c = 0; c < ncol; ++c) {
            primal_colour(T, W, sc, cur, cs, c, W.P.alpha, false);
            T.sync();
        }
        if (tid == 0) s_flags = 0;
        T.sync();
        if (dual_cta(T, W, sc, cur, nlive, it == W.P.num_iterations - 1)) s_flags = 1;
        T.sync();
        const int fractured = s_flags;
        T.sync();
        if (fractured) {
            for (int i = tid; i < nlive; i += nt) fracture_reset_slot(W, cur, W.live[cur][sc.cand0 + i]);
            T.sync();
            for (int b = b0 + tid; b < b1; b += nt) W.reset_flag[b] = 0;
            T.sync();
        }
    }
    scene_stamp(W, T, scene, 6);
    // 6. velocities, explosion, out of bounds
    if (tid == 0) s_flags = 0;
    T.sync();
    for (int b = b0 + tid; b < b1; b += nt) {
        const int r = velocity_body(W, b);
        if (r) atomicOr(&s_flags, r);
    }
    T.sync();
    const int vf = s_flags;
    T.sync();
    if (vf & 1) { if (tid == 0) st->status = kStatusExploded; return; }
    if (vf & 2) { if (tid == 0) st->status = kStatusNan; return; }
    if (vf & 4) {
        // RemoveBody of every out-of-bounds body (solver.cpp:530-534, geometry.cpp:11-25)
        for (int b = b0 + tid; b < b1; b += nt) {
            const int fl = W.flags[b];
            if ((fl & (kBodyStatic | kBodyRemoved)) != 0) continue;
            const float4 p = W.pos[b];
            if (p.x < kBoundMin || p.x > kBoundMax || p.y < kBoundMin || p.y > kBoundMax || p.z < kBoundMin ||
                p.z > kBoundMax) {
                W.flags[b] = fl | kBodyRemoved;
                atomicAdd(&st->topo, 1);
                for (int e = W.sinc_off[b]; e < W.sinc_off[b] + W.sinc_n[b]; ++e) {
                    const uint32_t ent = W.sinc[e];
                    const uint32_t k = ent_kind(ent), idx = ent_index(ent);
                    if (k == kEntForce) atomicOr(&W.ftype[idx], kForceRemoved);
                    else if (k == kEntTet) W.tparam[idx].w = 1.f;
                    else if (k == kEntTri) W.rparam[idx].w = 1.f;
                }
            }
        }
        T.sync();
    }
    if (tid == 0) st->step += 1;
    scene_stamp(W, T, scene, 7);
    // 7. post-stabilisation
    if (W.P.post_stabilization) {
        for (int c = 0; c < ncol; ++c) {
            primal_colour(T, W, sc, cur, cs, c, 0.f, true);
            T.sync();
        }
    }
}

}  // namespace avbd
