// Step drivers.  Block-cooperative functions (scans, incidence build,
// Jones-Plassmann colouring, colour lists) run on one CTA per scene; the
// persistent batched kernel strings every phase of a scene's step together on
// one CTA, and the single-scene path launches the same per-item functions as
// grid-wide kernels between them.
#pragma once
#include "avbd_phases.cuh"

// Optional per-phase cycle counters (development builds with -DAVBD_PHASE_TIMING
// only; the hooks compile to nothing otherwise).
#ifdef AVBD_PHASE_TIMING
__device__ unsigned long long g_phase_cycles[2 * 16];
__device__ unsigned long long g_scene_cycles[1 << 16];
#define AVBD_PHASE_BEGIN(kind) long long _avbd_t0 = clock64(), _avbd_s0 = _avbd_t0; const int _avbd_kind = (kind);
#define AVBD_PHASE(k)                                                                               \
    if (threadIdx.x == 0) {                                                                         \
        long long _t = clock64();                                                                   \
        atomicAdd(&g_phase_cycles[_avbd_kind * 16 + (k)], (unsigned long long)(_t - _avbd_t0));     \
        _avbd_t0 = _t;                                                                              \
    }
#define AVBD_PHASE_END(scene) \
    if (threadIdx.x == 0 && (scene) < (1 << 16)) g_scene_cycles[(scene)] = (unsigned long long)(clock64() - _avbd_s0);
#else
#define AVBD_PHASE_BEGIN(kind)
#define AVBD_PHASE(k)
#define AVBD_PHASE_END(scene)
#endif

namespace avbd {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kStagedBodies = 2560;   // bodies whose pose fits the broadphase's shared-memory stage (40 KB)

// Exclusive scan of in[0, n) into out[0, n) by one CTA; returns the total.
// in and out may alias.
__device__ int block_exclusive_scan(const int* in, int* out, int n) {
    __shared__ int warp_tot[32];
    __shared__ int carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < n ? in[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int w = lane < nwarps ? warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(kFull, w, o);
                if (lane >= o) w += y;
            }
            warp_tot[lane] = w;
        }
        __syncthreads();
        const int prefix = carry + (warp > 0 ? warp_tot[warp - 1] : 0);
        if (i < n) out[i] = prefix + x - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = prefix + x;
        __syncthreads();
    }
    const int total = carry;
    __syncthreads();
    return total;
}

// ---------------------------------------------------------------------------
// Incidence (CSR) of one scene: per body
//   [static forces][manifolds as body B, by slot][manifolds as body A][energies]
// which follows Mesh::forces then Mesh::energies (solver.cpp:395-435).
// ---------------------------------------------------------------------------
__device__ int owned_live(const World& W, int cur, int b, int base_slot) {
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
__device__ __noinline__ bool build_incidence(const World& W, const SceneDesc& sc, SceneState* st, int cur) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int b0 = sc.body0, b1 = sc.body0 + sc.nbody;
    const int ncand = st->ncand[cur];
    for (int b = b0 + tid; b < b1; b += nt) W.cntB[b] = 0;
    __syncthreads();
    for (int c = sc.cand0 + tid; c < sc.cand0 + ncand; c += nt)
        if (W.cn[cur][c] > 0) atomicAdd(&W.cntB[W.cpair[cur][c].y], 1);
    __syncthreads();
    for (int b = b0 + tid; b < b1; b += nt) {
        const int ns = W.sinc_n[b];
        W.inc_cnt[b] = ns + W.cntB[b] + owned_live(W, cur, b, sc.cand0);
    }
    __syncthreads();
    const int total = block_exclusive_scan(W.inc_cnt + b0, W.inc_off + b0, sc.nbody);
    if (total > sc.inccap) {
        if (tid == 0) { st->need_inc = total; }
        return false;
    }
    for (int b = b0 + tid; b < b1; b += nt) {
        const int off = sc.inc0 + W.inc_off[b];
        W.inc_off[b] = off;
        const int s0 = W.sinc_off[b], nf = W.sinc_nf[b], ns = W.sinc_n[b];
        int k = off;
        for (int e = 0; e < nf; ++e) W.inc[k++] = W.sinc[s0 + e];
        k += W.cntB[b];
        const int c0 = W.cand_off[b] + sc.cand0, c1 = c0 + W.cand_cnt[b];
        for (int c = c0; c < c1; ++c)
            if (W.cn[cur][c] > 0) W.inc[k++] = ent_make(kEntManifold, 0, (uint32_t)c);
        for (int e = nf; e < ns; ++e) W.inc[k++] = W.sinc[s0 + e];
        W.bcur[b] = 0;
    }
    __syncthreads();
    for (int c = sc.cand0 + tid; c < sc.cand0 + ncand; c += nt) {
        if (W.cn[cur][c] == 0) continue;
        const int B = W.cpair[cur][c].y;
        const int p = atomicAdd(&W.bcur[B], 1);
        W.inc[W.inc_off[B] + W.sinc_nf[B] + p] = ent_make(kEntManifold, 1, (uint32_t)c);
    }
    __syncthreads();
    // order each body's manifolds as Mesh::forces holds them: by creation step,
    // then by pair (creation order within a broadphase pass)
    for (int b = b0 + tid; b < b1; b += nt) {
        uint32_t* seg = W.inc + W.inc_off[b] + W.sinc_nf[b];
        const int n = W.inc_cnt[b] - W.sinc_n[b];
        sort_manifold_entries(W, cur, seg, n);
    }
    if (tid == 0) st->ninc = total;
    __syncthreads();
    return true;
}

// ---------------------------------------------------------------------------
// Jones-Plassmann first-fit colouring of the dynamic bodies of one scene.
// Priority = (hash(local index), local index), smaller first.  A body takes
// the smallest colour not used by its smaller-priority neighbours once all of
// them are coloured, which equals sequential greedy colouring in priority
// order whatever the thread schedule (each body's colour depends only on the
// final colours of its smaller-priority neighbours).
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

// Sweeps the bodies list[0, n) with groups of G lanes of the calling CTA.
template <int G>
__device__ void primal_sweep_cta(const World& W, int cur, const int* list, int n, float alpha, bool write_stick) {
    const int lane = threadIdx.x % G, gid = threadIdx.x / G, ngroups = blockDim.x / G;
    for (int base = 0; base < n; base += ngroups) {
        const int i = base + gid;
        int b = i < n ? list[i] : -1;
        if (b >= 0 && (W.flags[b] & kBodyRemoved)) b = -1;
        primal_group<G>(W, cur, b, alpha, write_stick, lane);
    }
}

__device__ __noinline__ void primal_sweep_cta_dispatch(const World& W, int cur, const int* list, int n, float alpha,
                                                          bool write_stick, int group) {
    switch (group) {
        case 32: primal_sweep_cta<32>(W, cur, list, n, alpha, write_stick); break;
        case 16: primal_sweep_cta<16>(W, cur, list, n, alpha, write_stick); break;
        case 8: primal_sweep_cta<8>(W, cur, list, n, alpha, write_stick); break;
        case 4: primal_sweep_cta<4>(W, cur, list, n, alpha, write_stick); break;
        case 2: primal_sweep_cta<2>(W, cur, list, n, alpha, write_stick); break;
        default: primal_sweep_cta<1>(W, cur, list, n, alpha, write_stick); break;
    }
}

// ---------------------------------------------------------------------------
// Term-per-lane primal sweep of one colour, for scenes whose energies are all
// tetrahedra.  Up to kFlatSlots (particle, tet) terms of the colour are
// evaluated at once, one per lane, into shared memory; then one lane per
// particle adds its inertia, its force and manifold rows and its tet terms in
// incidence order (the reference's order) and solves.  Lanes stay busy
// whatever the particles' degrees.  tinc (the scene's col_tinc) holds the
// inclusive prefix of tet terms over the colour list; the colour occupies
// list positions [c0, c1).  sm: 10 * kFlatSlots words of shared memory.
// ---------------------------------------------------------------------------
constexpr int kFlatSlots = 1024;
static_assert(10 * kFlatSlots * sizeof(float) <= kStagedBodies * sizeof(float4),
              "the flat sweep reuses the broadphase's dynamic shared memory");

__device__ __forceinline__ int tet_terms(const World& W, int b) { return W.sinc_n[b] - W.sinc_nf[b]; }

__device__ __noinline__ void primal_sweep_flat(const World& W, int cur, const int* list, const int* tinc, int c0,
                                               int c1, float alpha, bool write_stick, float* sm) {
    int* smap = reinterpret_cast<int*>(sm + 9 * kFlatSlots);
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int v = c0; v < c1;) {
        const int base = v == 0 ? 0 : tinc[v - 1];
        // the longest run of particles [v, vend) whose terms fit the slots (at least one)
        int lo = v + 1, hi = c1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tinc[mid - 1] - base <= kFlatSlots) lo = mid;
            else hi = mid - 1;
        }
        const int vend = lo;
        const int total = tinc[vend - 1] - base;
        const bool flat = total <= kFlatSlots;
        if (flat) {
            for (int j = v + tid; j < vend; j += nt)
                for (int q = (j == 0 ? 0 : tinc[j - 1]) - base; q < tinc[j] - base; ++q) smap[q] = j;
            __syncthreads();
            for (int q = tid; q < total; q += nt) {
                const int j = smap[q];
                const int b = list[j];
                const int k = q - ((j == 0 ? 0 : tinc[j - 1]) - base);
                const uint32_t ent = W.inc[W.inc_off[b] + W.inc_cnt[b] - tet_terms(W, b) + k];
                V3 g = v3(0.f, 0.f, 0.f);
                S3 H;
                s3_zero(H);
                if (!(W.flags[b] & kBodyRemoved)) tet_term(W, (int)ent_index(ent), (int)ent_role(ent), g, H);
                sm[0 * kFlatSlots + q] = g.x; sm[1 * kFlatSlots + q] = g.y; sm[2 * kFlatSlots + q] = g.z;
                sm[3 * kFlatSlots + q] = H.xx; sm[4 * kFlatSlots + q] = H.yy; sm[5 * kFlatSlots + q] = H.zz;
                sm[6 * kFlatSlots + q] = H.xy; sm[7 * kFlatSlots + q] = H.xz; sm[8 * kFlatSlots + q] = H.yz;
            }
            __syncthreads();
        }
        for (int j = v + tid; j < vend; j += nt) {
            const int b = list[j];
            if (W.flags[b] & kBodyRemoved) continue;
            Sys6 s;
            sys_zero(s);
            primal_init_mass(W, b, s);
            const int e0 = W.inc_off[b], e1 = e0 + W.inc_cnt[b];
            if (!flat) {
                primal_entry_range(W, cur, b, alpha, write_stick, e0, e1, 0, 1, s);
            } else {
                const int nterm = tet_terms(W, b);
                primal_entry_range(W, cur, b, alpha, write_stick, e0, e1 - nterm, 0, 1, s);
                const int q0 = (j == 0 ? 0 : tinc[j - 1]) - base;
                for (int q = q0; q < q0 + nterm; ++q) {
                    // a removed tet left zeros: adding them changes no value
                    sys_add_energy(s, sm[0 * kFlatSlots + q], sm[1 * kFlatSlots + q], sm[2 * kFlatSlots + q],
                                   sm[3 * kFlatSlots + q], sm[4 * kFlatSlots + q], sm[5 * kFlatSlots + q],
                                   sm[6 * kFlatSlots + q], sm[7 * kFlatSlots + q], sm[8 * kFlatSlots + q]);
                }
            }
            primal_finish(W, b, s);
        }
        __syncthreads();
        v = vend;
    }
}

// One colour of a scene's primal sweep, by the scene's lane grouping.
__device__ __forceinline__ void primal_colour(const World& W, const SceneDesc& sc, int cur, const int* cs, int c,
                                              float alpha, bool write_stick, float* sm) {
    if (sc.group == kGroupFlat)
        primal_sweep_flat(W, cur, W.col_list + sc.body0, W.col_tinc + sc.body0, cs[c], cs[c + 1], alpha, write_stick,
                          sm);
    else
        primal_sweep_cta_dispatch(W, cur, W.col_list + sc.body0 + cs[c], cs[c + 1] - cs[c], alpha, write_stick,
                                  sc.group);
}

__device__ __noinline__ bool colour_scene(const World& W, const SceneDesc& sc, SceneState* st, int scene, int cur);

// Keeps the previous step's colouring when the contact graph is unchanged:
// the same number of live manifolds in both tables, every live one already
// live last step, and no force or body removed since the colouring was made.
// The colouring is a deterministic function of that graph, so reusing it is
// exact.
__device__ bool colour_scene_cached(const World& W, const SceneDesc& sc, SceneState* st, int scene, int cur) {
    const int old = cur ^ 1;
    const bool reuse = st->colours_valid && st->nlive[cur] == st->nlive[old] && st->nmatched == st->nlive[cur] &&
                       st->topo == st->coloured_topo;
    __syncthreads();
    if (reuse) return true;
    const bool ok = colour_scene(W, sc, st, scene, cur);
    if (threadIdx.x == 0) {
        st->colours_valid = ok ? 1 : 0;
        st->coloured_topo = st->topo;
    }
    __syncthreads();
    return ok;
}

// Returns false (status TIMEOUT or CAPACITY set) if colouring could not finish.
__device__ __noinline__ bool colour_scene(const World& W, const SceneDesc& sc, SceneState* st, int scene, int cur) {
    __shared__ int s_remaining, s_progress, s_maxc;
    __shared__ int s_count[kMaxColours + 1];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int b0 = sc.body0, b1 = sc.body0 + sc.nbody;
    volatile int* col = W.colour;
    for (int b = b0 + tid; b < b1; b += nt) col[b] = (W.flags[b] & (kBodyStatic | kBodyRemoved)) ? -2 : -1;
    if (tid == 0) s_maxc = 0;
    __syncthreads();
    const int max_rounds = sc.nbody + 2;
    for (int round = 0;; ++round) {
        if (tid == 0) { s_remaining = 0; s_progress = 0; }
        __syncthreads();
        for (int b = b0 + tid; b < b1; b += nt) {
            if (col[b] != -1) continue;
            const int lb = W.local[b];
            const uint32_t hb = colour_priority((uint32_t)lb);
            bool ready = true;
            for_each_neighbour(W, cur, b, [&](int n) {
                if (!ready) return;
                const int cn = col[n];
                if (cn == -2) return;
                const int ln = W.local[n];
                if (prio_less(colour_priority((uint32_t)ln), ln, hb, lb) && cn < 0) ready = false;
            });
            if (!ready) { s_remaining = 1; continue; }
            int chosen = -1;
            for (int base = 0; base < kMaxColours && chosen < 0; base += 64) {
                unsigned long long used = 0ull;
                for_each_neighbour(W, cur, b, [&](int n) {
                    const int cn = col[n];
                    if (cn < base || cn >= base + 64) return;
                    const int ln = W.local[n];
                    if (prio_less(colour_priority((uint32_t)ln), ln, hb, lb)) used |= 1ull << (cn - base);
                });
                if (~used) chosen = base + __ffsll((long long)~used) - 1;
            }
            if (chosen < 0 || chosen >= kMaxColours) {
                st->status = kStatusCapacity;
                chosen = kMaxColours - 1;
            }
            col[b] = chosen;
            atomicMax(&s_maxc, chosen + 1);
            s_progress = 1;
        }
        __syncthreads();
        const int remaining = s_remaining, progress = s_progress;
        __syncthreads();   // every thread has read the flags before thread 0 resets them
        if (!remaining) break;
        if (!progress || round > max_rounds) {
            if (tid == 0) st->status = kStatusTimeout;
            __syncthreads();
            return false;
        }
    }
    const int ncol = s_maxc;
    __syncthreads();
    // colour lists: counting sort of the dynamic bodies by colour
    for (int c = tid; c <= ncol; c += nt) s_count[c] = 0;
    __syncthreads();
    for (int b = b0 + tid; b < b1; b += nt) {
        const int c = col[b];
        if (c >= 0) atomicAdd(&s_count[c], 1);
    }
    __syncthreads();
    int* cs = W.col_start + (size_t)scene * (kMaxColours + 1);
    if (tid == 0) {
        int acc = 0;
        for (int c = 0; c < ncol; ++c) { cs[c] = acc; acc += s_count[c]; s_count[c] = cs[c]; }
        cs[ncol] = acc;
        st->ncolours = ncol;
    }
    __syncthreads();
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
            if (k == key) W.col_list[b0 + atomicAdd(&s_count[c], 1)] = b;
        }
        __syncthreads();
    }
    if (sc.group == kGroupFlat) {
        // inclusive prefix of tet terms over the list
        const int n = cs[ncol];
        int* tinc = W.col_tinc + b0;
        for (int i = tid; i < n; i += nt) tinc[i] = tet_terms(W, W.col_list[b0 + i]);
        __syncthreads();
        block_exclusive_scan(tinc, tinc, n);
        for (int i = tid; i < n; i += nt) tinc[i] += tet_terms(W, W.col_list[b0 + i]);
        __syncthreads();
    }
    return st->status == kStatusOk;
}

// Phase loops of one scene kept out of line, so each gets its own register
// allocation instead of the union of every inlined phase.
__device__ __noinline__ void narrowphase_cta(const World& W, const SceneDesc& sc, SceneState* st, int cur, int ncand,
                                             int old_count) {
    for (int c = sc.cand0 + threadIdx.x; c < sc.cand0 + ncand; c += blockDim.x)
        narrowphase_slot(W, sc, st, c, cur, old_count);
}

// Returns true if this thread saw a force fracture.  Manifolds come from the
// step's live list (each manifold's dual is independent of the others).
__device__ __noinline__ bool dual_cta(const World& W, const SceneDesc& sc, int cur, int nlive, bool last) {
    bool broke = false;
    for (int f = sc.force0 + threadIdx.x; f < sc.force0 + sc.nforce; f += blockDim.x)
        if (dual_force(W, f, W.P.alpha)) broke = true;
    const int* live = W.live[cur] + sc.cand0;
    for (int i = threadIdx.x; i < nlive; i += blockDim.x) dual_manifold(W, cur, live[i], W.P.alpha, last);
    return broke;
}

// ---------------------------------------------------------------------------
// Whole step of one scene on one CTA (batched path).
// ---------------------------------------------------------------------------
__device__ void scene_step(const World& W, int scene) {
    const SceneDesc sc = W.scenes[scene];
    SceneState* st = W.sstate + scene;
    const int tid = threadIdx.x, nt = blockDim.x;
    __shared__ int s_flags;
    if (st->status != kStatusOk && st->status != kStatusCapacity && st->status != kStatusTimeout) return;
    __syncthreads();
    if (tid == 0) { st->status = kStatusOk; st->need_cand = 0; st->need_k = 0; st->need_inc = 0; }
    AVBD_PHASE_BEGIN(sc.ntet > 0 ? 1 : 0);
    const int old = st->cur, cur = old ^ 1;
    const int b0 = sc.body0, b1 = sc.body0 + sc.nbody;
    // 1. broadphase: count, scan, capacity check, write; positions and radii
    //    staged in shared memory when the scene fits
    extern __shared__ float4 s_bodies[];
    const bool staged = sc.nbody <= kStagedBodies;
    if (staged) {
        for (int b = b0 + tid; b < b1; b += nt) {
            float4 p = W.pos[b];
            p.w = (W.flags[b] & kBodyRemoved) ? -INFINITY : W.scale[b].w;
            s_bodies[b - b0] = p;
        }
        __syncthreads();
    }
    for (int b = b0 + tid; b < b1; b += nt)
        W.cand_cnt[b] = staged ? broadphase_body_staged(W, sc, b, s_bodies, nullptr, 0)
                               : broadphase_body(W, sc, b, nullptr, 0);
    __syncthreads();
    const int ncand = block_exclusive_scan(W.cand_cnt + b0, W.cand_off + b0, sc.nbody);
    if (ncand > sc.candcap) {
        if (tid == 0) { st->status = kStatusCapacity; st->need_cand = ncand; }
        return;
    }
    for (int b = b0 + tid; b < b1; b += nt) {
        int2* out = W.cpair[cur] + sc.cand0 + W.cand_off[b];
        if (staged) broadphase_body_staged(W, sc, b, s_bodies, out, W.cand_cnt[b]);
        else broadphase_body(W, sc, b, out, W.cand_cnt[b]);
    }
    if (tid == 0) { st->kused[cur] = 0; st->nlive[cur] = 0; st->nmatched = 0; }
    __syncthreads();
    AVBD_PHASE(0);
    // 2. narrowphase + manifold warm start into the other table
    const int old_count = st->ncand[old];
    narrowphase_cta(W, sc, st, cur, ncand, old_count);
    __syncthreads();
    if (st->need_k) {
        if (tid == 0) { st->status = kStatusCapacity; st->need_k = st->kused[cur]; }
        return;
    }
    if (tid == 0) { st->ncand[cur] = ncand; st->cur = cur; }
    AVBD_PHASE(1);
    // 2b. joints / springs warm start
    for (int f = sc.force0 + tid; f < sc.force0 + sc.nforce; f += nt)
        if (force_init(W, f)) atomicAdd(&st->topo, 1);
    __syncthreads();
    // incidence
    if (!build_incidence(W, sc, st, cur)) {
        if (tid == 0) st->status = kStatusCapacity;
        return;
    }
    AVBD_PHASE(2);
    // colouring
    if (!colour_scene_cached(W, sc, st, scene, cur)) return;
    AVBD_PHASE(3);
    // 4. prediction
    for (int b = b0 + tid; b < b1; b += nt) predict_body(W, b);
    __syncthreads();
    AVBD_PHASE(4);
    const int ncol = st->ncolours;
    const int nlive = st->nlive[cur];
    const int* cs = W.col_start + (size_t)scene * (kMaxColours + 1);
    // 5. iterations
    for (int it = 0; it < W.P.num_iterations; ++it) {
        for (int c = 0; c < ncol; ++c) {
            primal_colour(W, sc, cur, cs, c, W.P.alpha, false, reinterpret_cast<float*>(s_bodies));
            __syncthreads();
        }
        AVBD_PHASE(5);
        if (tid == 0) s_flags = 0;
        __syncthreads();
        if (dual_cta(W, sc, cur, nlive, it == W.P.num_iterations - 1)) s_flags = 1;
        __syncthreads();
        const int fractured = s_flags;
        __syncthreads();
        if (fractured) {
            for (int i = tid; i < nlive; i += nt) fracture_reset_slot(W, cur, W.live[cur][sc.cand0 + i]);
            __syncthreads();
            for (int b = b0 + tid; b < b1; b += nt) W.reset_flag[b] = 0;
            __syncthreads();
        }
        AVBD_PHASE(6);
    }
    // 6. velocities, explosion, out of bounds
    if (tid == 0) s_flags = 0;
    __syncthreads();
    for (int b = b0 + tid; b < b1; b += nt) {
        const int r = velocity_body(W, b);
        if (r) atomicOr(&s_flags, r);
    }
    __syncthreads();
    const int vf = s_flags;
    __syncthreads();
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
        __syncthreads();
    }
    if (tid == 0) st->step += 1;
    AVBD_PHASE(7);
    // 7. post-stabilisation
    if (W.P.post_stabilization) {
        for (int c = 0; c < ncol; ++c) {
            primal_colour(W, sc, cur, cs, c, 0.f, true, reinterpret_cast<float*>(s_bodies));
            __syncthreads();
        }
    }
    AVBD_PHASE(8);
    AVBD_PHASE_END(scene);
}

}  // namespace avbd
