// C-ABI of the single-scene path (include/avbd.h): the grid-wide kernels and
// launch sequence of one world, scene building, readback, snapshots and the
// allocation-free collision queries.  The batched path is in
// avbd_batch_host.cu, the pools and handles in avbd_pools.h.
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
#include "avbd_pools.h"
#include "avbd_step.cuh"

using namespace avbd;
using namespace avbd::host;

// ===========================================================================
// Kernels of the single-scene path (grid-wide over the items of scene 0)
// ===========================================================================
namespace {

constexpr int kGridMinBodies = 128;   // single-scene bodies from which the broadphase uses the grid


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

__global__ void k_bp_write(const __grid_constant__ World W, int cur, int all_pairs) {
    const SceneDesc sc = W.scenes[0];
    if (all_pairs)
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

// ---------------------------------------------------------------------------
// Uniform-grid broadphase of the single scene, grid-wide: the batched path's
// grid (broadphase_grid: cells 2R wide, R the largest radius of the small
// bodies, the big bodies' all-pairs rows beside it, candidate lists sorted by
// partner) built by a counting sort over the whole GPU instead of one CTA.
// Same candidate set and order as the reference's all-pairs loop
// (solver.cpp:233-256).  Scratch: W.bcur (cell starts), W.cntB (cell items),
// W.cand_off (each body's rank in its cell, before it takes the offsets).
// ---------------------------------------------------------------------------
struct GridState {
    int red[8];               // order-preserving float bits: min xyz, max xyz, max radius, min radius
    int nbig;
    int big[kGridMaxBig];
    GridDims g;
    int ncell;
    int valid;                // 0: use the all-pairs loop this step
    float rbig;
};

__global__ void k_grid_reset(GridState* gs) {
    if (threadIdx.x != 0) return;
    for (int a = 0; a < 3; ++a) { gs->red[a] = ord_float(INFINITY); gs->red[3 + a] = ord_float(-INFINITY); }
    gs->red[6] = ord_float(0.f);
    gs->red[7] = ord_float(INFINITY);
    gs->nbig = 0;
}

__global__ void k_grid_rmin(const __grid_constant__ World W, GridState* gs) {
    const SceneDesc sc = W.scenes[0];
    float rmin = INFINITY;
    for (int li = blockIdx.x * blockDim.x + threadIdx.x; li < sc.nbody; li += gridDim.x * blockDim.x) {
        const float4 p = body_sphere(W, sc, nullptr, li);
        if (!isinf(p.w)) rmin = fminf(rmin, p.w);
    }
    for (int o = 16; o > 0; o >>= 1) rmin = fminf(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
    if ((threadIdx.x & 31) == 0) atomicMin(&gs->red[7], ord_float(rmin));
}

__global__ void k_grid_extent(const __grid_constant__ World W, GridState* gs) {
    const SceneDesc sc = W.scenes[0];
    const float rbig = 8.f * unord_float(gs->red[7]);
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY}, mr = 0.f;
    for (int li = blockIdx.x * blockDim.x + threadIdx.x; li < sc.nbody; li += gridDim.x * blockDim.x) {
        const float4 p = body_sphere(W, sc, nullptr, li);
        if (isinf(p.w)) continue;
        if (p.w > rbig) {
            const int k = atomicAdd(&gs->nbig, 1);
            if (k < kGridMaxBig) gs->big[k] = li;
            continue;
        }
        mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
        mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
        mr = fmaxf(mr, p.w);
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
        mr = fmaxf(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(&gs->red[a], ord_float(mn[a]));
            atomicMax(&gs->red[3 + a], ord_float(mx[a]));
        }
        atomicMax(&gs->red[6], ord_float(mr));
    }
}

// Grid dimensions (as broadphase_grid chooses them: at most nbody / 2 cells).
__global__ void k_grid_setup(const __grid_constant__ World W, GridState* gs) {
    if (threadIdx.x != 0) return;
    const SceneDesc sc = W.scenes[0];
    GridDims g;
    g.minx = unord_float(gs->red[0]); g.miny = unord_float(gs->red[1]); g.minz = unord_float(gs->red[2]);
    const float ex = unord_float(gs->red[3]) - g.minx, ey = unord_float(gs->red[4]) - g.miny,
                ez = unord_float(gs->red[5]) - g.minz;
    const float R = unord_float(gs->red[6]);
    const float rbig = 8.f * unord_float(gs->red[7]);
    gs->rbig = rbig;
    gs->valid = 0;
    if (!(ex >= 0.f && ey >= 0.f && ez >= 0.f) || !(ex < 1e30f && ey < 1e30f && ez < 1e30f) || !(R < 1e30f) ||
        !(rbig < 1e30f) || gs->nbig > kGridMaxBig)
        return;
    const int maxcell = max(1, sc.nbody / 2);
    float h = fmaxf(2.f * R * 1.0001f, 1e-6f);
    for (int it = 0; it < 64; ++it) {
        g.nx = (int)(ex / h) + 1; g.ny = (int)(ey / h) + 1; g.nz = (int)(ez / h) + 1;
        if ((long long)g.nx * g.ny * g.nz <= maxcell) break;
        h *= 1.25f;
    }
    if ((long long)g.nx * g.ny * g.nz > maxcell) return;
    g.inv_h = 1.f / h;
    gs->g = g;
    gs->ncell = g.nx * g.ny * g.nz;
    gs->valid = 1;
}

__global__ void k_grid_clear(const __grid_constant__ World W, const GridState* gs) {
    if (!gs->valid) return;
    int* cstart = W.bcur + W.scenes[0].body0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= gs->ncell; c += gridDim.x * blockDim.x) cstart[c] = 0;
}

__global__ void k_grid_rank(const __grid_constant__ World W, const GridState* gs) {
    if (!gs->valid) return;
    const SceneDesc sc = W.scenes[0];
    int* cstart = W.bcur + sc.body0;
    for (int li = blockIdx.x * blockDim.x + threadIdx.x; li < sc.nbody; li += gridDim.x * blockDim.x) {
        const float4 p = body_sphere(W, sc, nullptr, li);
        if (isinf(p.w) || p.w > gs->rbig) continue;
        W.cand_off[sc.body0 + li] = atomicAdd(&cstart[gs->g.cell(p)], 1);
    }
}

__global__ void k_grid_scan(const __grid_constant__ World W, const GridState* gs) {
    __shared__ TeamShared s_team;
    if (!gs->valid) return;
    const Team T = Team::cta(&s_team, nullptr, 0);
    int* cstart = W.bcur + W.scenes[0].body0;
    const int total = block_exclusive_scan(T, cstart, cstart, gs->ncell);
    if (threadIdx.x == 0) cstart[gs->ncell] = total;
}

__global__ void k_grid_scatter(const __grid_constant__ World W, const GridState* gs) {
    if (!gs->valid) return;
    const SceneDesc sc = W.scenes[0];
    const int* cstart = W.bcur + sc.body0;
    for (int li = blockIdx.x * blockDim.x + threadIdx.x; li < sc.nbody; li += gridDim.x * blockDim.x) {
        const float4 p = body_sphere(W, sc, nullptr, li);
        if (isinf(p.w) || p.w > gs->rbig) continue;
        W.cntB[sc.body0 + cstart[gs->g.cell(p)] + W.cand_off[sc.body0 + li]] = li;
    }
}

__device__ __forceinline__ GridCells grid_cells(const World& W, const SceneDesc& sc, const GridState* gs) {
    GridCells gc;
    gc.cstart = W.bcur + sc.body0;
    gc.items16 = nullptr;
    gc.items32 = W.cntB + sc.body0;
    gc.big = gs->big;
    gc.nbig = gs->nbig;
    gc.rbig = gs->rbig;
    return gc;
}

// The big bodies' all-pairs rows (a floor or wall overlaps most of the
// scene): one block per big body, each chunk of partners tested by the
// block's threads and its candidates placed by a block-wide prefix count, so
// the row comes out in partner order without one thread walking it.
template <bool WRITE>
__global__ void __launch_bounds__(1024) k_bp_big(const __grid_constant__ World W, const GridState* gs, int cur) {
    __shared__ int s_warp[32];
    __shared__ int s_total;
    if (!gs->valid) return;
    const SceneDesc sc = W.scenes[0];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int k = blockIdx.x; k < gs->nbig; k += gridDim.x) {
        const int li = gs->big[k];
        const int b = sc.body0 + li;
        const float4 pi = body_sphere(W, sc, nullptr, li);
        const Partners pp = partners_of(W, b);
        int2* out = WRITE ? W.cpair[cur] + sc.cand0 + W.cand_off[b] : nullptr;
        const int cap = WRITE ? W.cand_cnt[b] : 0;
        if (threadIdx.x == 0) s_total = 0;
        __syncthreads();
        for (int c0 = li + 1; c0 < sc.nbody; c0 += blockDim.x) {
            const int lj = c0 + threadIdx.x;
            const bool hit = !isinf(pi.w) && lj < sc.nbody && grid_pair(W, sc, nullptr, pi, pp, lj);
            const unsigned bal = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) s_warp[warp] = __popc(bal);
            __syncthreads();
            int before = s_total, chunk = 0;
            for (int w = 0; w < nwarps; ++w) {
                if (w < warp) before += s_warp[w];
                chunk += s_warp[w];
            }
            const int at = before + __popc(bal & ((1u << lane) - 1u));
            if (WRITE && hit && at < cap) out[at] = make_int2(b, sc.body0 + lj);
            __syncthreads();
            if (threadIdx.x == 0) s_total += chunk;
            __syncthreads();
        }
        if (!WRITE && threadIdx.x == 0) W.cand_cnt[b] = s_total;
        __syncthreads();
    }
}

// Candidates per body (count pass) or their pairs (write pass), from the
// grid when it is valid this step, else from the all-pairs loop.  The big
// bodies' rows come from k_bp_big.
template <bool WRITE>
__global__ void k_bp_grid(const __grid_constant__ World W, const GridState* gs, int cur) {
    const SceneDesc sc = W.scenes[0];
    const bool grid = gs->valid != 0;
    const GridDims g = gs->g;
    const GridCells gc = grid_cells(W, sc, gs);
    for (int li = blockIdx.x * blockDim.x + threadIdx.x; li < sc.nbody; li += gridDim.x * blockDim.x) {
        const int b = sc.body0 + li;
        if (grid && !(W.flags[b] & kBodyRemoved) && W.scale[b].w > gc.rbig) continue;   // k_bp_big
        if (!WRITE) {
            W.cand_cnt[b] = grid ? grid_candidates<false>(W, sc, nullptr, g, gc, li, nullptr)
                                 : broadphase_body(W, sc, b, nullptr, 0);
        } else {
            int2* out = W.cpair[cur] + sc.cand0 + W.cand_off[b];
            if (grid) {
                const int wrote = grid_candidates<true>(W, sc, nullptr, g, gc, li, out);
                AVBD_CHECK(W, wrote == W.cand_cnt[b], 3, wrote, W.cand_cnt[b]);
            }
            else broadphase_body(W, sc, b, out, W.cand_cnt[b]);
        }
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


// ---------------------------------------------------------------------------
// Incidence and colouring of the single scene, grid-wide: the stages of
// build_incidence and colour_scene (one team per scene in the batched path)
// as kernels over all bodies.  Each Jones-Plassmann round is one launch; the
// host launches rounds in chunks and reads in between whether the pass has
// ended, so the colouring equals sequential greedy in priority order
// whatever the schedule, as in the batched path.
// ---------------------------------------------------------------------------
struct ColourState {
    int skip;                       // the previous colouring still holds (or the step already failed)
    int done;                       // the current pass ended (read by the host with skip)
    int rf[3][2];                   // per round (mod 3): bodies remaining, progress made
    int stalled;
    int maxc;                       // colours used
    int count[kMaxColours + 1];     // bodies per colour, then list cursors
};

#define AVBD_BODIES(b)                                                                                   \
    for (int b = sc.body0 + blockIdx.x * blockDim.x + threadIdx.x; b < sc.body0 + sc.nbody;            \
         b += gridDim.x * blockDim.x)
#define AVBD_SLOTS(c, n)                                                                                 \
    for (int c = sc.cand0 + blockIdx.x * blockDim.x + threadIdx.x; c < sc.cand0 + (n); c += gridDim.x * blockDim.x)

__global__ void k_inc_count_b(const __grid_constant__ World W, int cur) {
    const SceneDesc sc = W.scenes[0];
    AVBD_SLOTS(c, W.sstate->ncand[cur])
        if (W.cn[cur][c] > 0) atomicAdd(&W.cntB[W.cpair[cur][c].y], 1);
}

__global__ void k_inc_count(const __grid_constant__ World W, int cur) {
    const SceneDesc sc = W.scenes[0];
    AVBD_BODIES(b) W.inc_cnt[b] = body_fixed(W, b) ? 0 : W.sinc_n[b] + W.cntB[b] + owned_live(W, cur, b, sc.cand0);
}

__global__ void k_inc_scan(const __grid_constant__ World W) {
    __shared__ TeamShared s_team;
    const Team T = Team::cta(&s_team, nullptr, 0);
    const SceneDesc sc = W.scenes[0];
    SceneState* st = W.sstate;
    const int total = block_exclusive_scan(T, W.inc_cnt + sc.body0, W.inc_off + sc.body0, sc.nbody);
    if (threadIdx.x == 0) {
        st->ninc = total;
        if (total > sc.inccap) { st->need_inc = total; st->status = kStatusCapacity; }
    }
}

__global__ void k_inc_fill(const __grid_constant__ World W, int cur) {
    const SceneDesc sc = W.scenes[0];
    if (W.sstate->status != kStatusOk) return;
    AVBD_BODIES(b) {
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
}

__global__ void k_inc_fill_b(const __grid_constant__ World W, int cur) {
    const SceneDesc sc = W.scenes[0];
    if (W.sstate->status != kStatusOk) return;
    AVBD_SLOTS(c, W.sstate->ncand[cur]) {
        if (W.cn[cur][c] == 0) continue;
        const int B = W.cpair[cur][c].y;
        if (body_fixed(W, B)) continue;
        const int p = atomicAdd(&W.bcur[B], 1);
        if (!AVBD_CHECK(W, p < W.cntB[B], 2, p, W.cntB[B])) continue;
        W.inc[W.inc_off[B] + W.sinc_nf[B] + p] = ent_make(kEntManifold, 1, (uint32_t)c);
    }
}

// Each body's manifolds as Mesh::forces holds them: by creation step, then pair.
__global__ void k_inc_sort(const __grid_constant__ World W, int cur) {
    const SceneDesc sc = W.scenes[0];
    if (W.sstate->status != kStatusOk) return;
    AVBD_BODIES(b) {
        if (!body_fixed(W, b))
            sort_manifold_entries(W, cur, W.inc + W.inc_off[b] + W.sinc_nf[b], W.inc_cnt[b] - W.sinc_n[b]);
    }
}

// Whether the colouring is redone this step (colour_scene_cached's test):
// not when the contact graph is the one the colours were made for.
__global__ void k_col_prepare(const __grid_constant__ World W, ColourState* cs, int cur) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const SceneState* st = W.sstate;
    const int old = cur ^ 1;
    const bool reuse = st->colours_valid && st->nlive[cur] == st->nlive[old] && st->nmatched == st->nlive[cur] &&
                       st->topo == st->coloured_topo;
    cs->skip = (reuse || st->status != kStatusOk) ? 1 : 0;
    cs->done = cs->skip;
    cs->stalled = 0;
    cs->maxc = 0;
    for (int r = 0; r < 3; ++r) cs->rf[r][0] = cs->rf[r][1] = 0;
    for (int c = 0; c <= kMaxColours; ++c) cs->count[c] = 0;
}

// Neighbour lists and priorities of the colouring, once per colouring.
struct ColourLists {
    int* nbr;                  // body b's dynamic neighbours from 3 * (inc_off[b] - inc0), one per
                               // live neighbour visit of for_each_neighbour (repeats kept)
    int* cnt;
    unsigned long long* key;   // u precedes v in pass 0 iff key[u] > key[v]
    int* pos;                  // neighbours already scanned this pass (bit 30: one held a colour >= 64)
    unsigned long long* used;  // colours < 64 of the scanned neighbours
};
constexpr int kPosWide = 1 << 30;

// Pass-0 priority as one integer: larger live degree first, then smaller
// colour_priority(local index), which is a bijection, so ties cannot remain
// (colour_before's order exactly).
__device__ __forceinline__ unsigned long long colour_key(int degree, int local) {
    return ((unsigned long long)(unsigned)degree << 32) | (unsigned long long)(~colour_priority((uint32_t)local));
}

// Live degree and pass-0 priority of every dynamic body.
__global__ void k_col_init(const __grid_constant__ World W, const ColourState* cs, ColourLists L) {
    const SceneDesc sc = W.scenes[0];
    if (cs->skip) return;
    AVBD_BODIES(b) {
        if (body_fixed(W, b)) {
            W.colour[b] = -2;
            L.cnt[b] = 0;
            continue;
        }
        W.colour[b] = -1;
        L.key[b] = colour_key(live_degree(W, b), W.local[b]);
    }
}

// Body u precedes body v in the pass's order (colour_before with the
// pass-0 priority as one integer).
__device__ __forceinline__ bool precedes(const World& W, const ColourLists& L, int pass, int u, int v) {
    if (pass == 1) {
        const int pu = W.bcur[u], pv = W.bcur[v];
        if (pu != pv) return pu > pv;
    }
    return L.key[u] > L.key[v];
}

// Each dynamic body's list of the neighbours that precede it in this pass
// (one entry per neighbour visit of for_each_neighbour; repeats kept), the
// only ones a Jones-Plassmann body waits for or takes colours from.
__global__ void k_col_pred(const __grid_constant__ World W, const ColourState* cs, ColourLists L, int cur, int pass) {
    const SceneDesc sc = W.scenes[0];
    if (cs->skip) return;
    AVBD_BODIES(b) {
        L.pos[b] = 0;
        L.used[b] = 0ull;
        if (body_fixed(W, b)) continue;
        int* out = L.nbr + 3 * (size_t)(W.inc_off[b] - sc.inc0);
        int n = 0;
        for_each_neighbour(W, cur, b, [&](int o) {
            if (o != b && !body_fixed(W, o) && precedes(W, L, pass, o, b)) out[n++] = o;
        });
        L.cnt[b] = n;
    }
}

// Second pass (iterated greedy): the first pass's colours become priorities.
__global__ void k_col_repass(const __grid_constant__ World W, ColourState* cs) {
    const SceneDesc sc = W.scenes[0];
    if (cs->skip) return;
    AVBD_BODIES(b) {
        const int c = W.colour[b];
        W.bcur[b] = c;
        if (c >= 0) W.colour[b] = -1;
    }
}

__global__ void k_col_next_pass(ColourState* cs) {
    if (cs->skip || blockIdx.x != 0 || threadIdx.x != 0) return;
    cs->done = 0;
    cs->maxc = 0;
    for (int r = 0; r < 3; ++r) cs->rf[r][0] = cs->rf[r][1] = 0;
}

constexpr int kJpSweeps = 16;   // sweeps over a thread's bodies per round launch

// Colours are read and written with relaxed GPU-scope accesses: every sweep
// must see what other blocks wrote meanwhile (a plain or .cg load could be
// merged across sweeps), and nothing else is ordered by them.
__device__ __forceinline__ int ld_colour(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_colour(int* p, int v) {
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
constexpr int kJpChunk = 8;     // predecessors whose colours are fetched together

// One Jones-Plassmann round (jp_pass's loop body) over the predecessor
// lists: a body takes the smallest colour its predecessors do not use once
// they are all coloured, which is sequential greedy in priority order
// whatever the schedule.  Colours are final once written, so a body resumes
// its scan at the predecessor that held it up, with the colours seen so far
// (pos / used).  A thread sweeps its bodies up to kJpSweeps times, picking
// up predecessors that other blocks coloured meanwhile.  Round r records its
// flags in slot r % 3, reads round r - 1's from slot (r - 1) % 3 to see
// whether the pass ended, and clears slot (r + 1) % 3 for the next round.
__global__ void k_jp_round(const __grid_constant__ World W, ColourState* cs, ColourLists L, int pass, int round) {
    const SceneDesc sc = W.scenes[0];
    if (cs->done) return;
    if (round > 0) {
        const int* prev = cs->rf[(round + 2) % 3];
        if (!prev[0] || !prev[1]) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                cs->done = 1;
                if (prev[0]) { cs->stalled = 1; W.sstate->status = kStatusTimeout; }
            }
            return;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { cs->rf[(round + 1) % 3][0] = 0; cs->rf[(round + 1) % 3][1] = 0; }
    int* flags = cs->rf[round % 3];
    int* col = W.colour;
    bool remaining = false, progress = false;
    for (int sweep = 0; sweep < kJpSweeps; ++sweep) {
        bool left = false;
        AVBD_BODIES(b) {
            if (ld_colour(col + b) != -1) continue;
            const int* nb = L.nbr + 3 * (size_t)(W.inc_off[b] - sc.inc0);
            const int n = L.cnt[b];
            int pos = L.pos[b];
            bool wide = (pos & kPosWide) != 0;
            int i = pos & ~kPosWide;
            unsigned long long used = L.used[b];
            bool ready = true;
            while (i < n) {
                int cu[kJpChunk];
#pragma unroll
                for (int k = 0; k < kJpChunk; ++k) cu[k] = ld_colour(col + (i + k < n ? nb[i + k] : b));
                const int m = min(kJpChunk, n - i);
                int k = 0;
                for (; k < m; ++k) {
                    if (cu[k] < 0) { ready = false; break; }   // a predecessor is not coloured yet
                    if (cu[k] < 64) used |= 1ull << cu[k];
                    else wide = true;
                }
                i += k;
                if (!ready) break;
            }
            if (!ready) {
                L.pos[b] = i | (wide ? kPosWide : 0);
                L.used[b] = used;
                left = true;
                continue;
            }
            int chosen = ~used ? __ffsll((long long)~used) - 1 : -1;
            if (chosen < 0 || wide) {
                // some neighbour holds a colour >= 64: first fit over 64-colour windows
                chosen = -1;
                for (int base = 0; base < kMaxColours && chosen < 0; base += 64) {
                    unsigned long long w = 0ull;
                    for (int j = 0; j < n; ++j) {
                        const int c = ld_colour(col + nb[j]);
                        if (c >= base && c < base + 64) w |= 1ull << (c - base);
                    }
                    if (~w) chosen = base + __ffsll((long long)~w) - 1;
                }
            }
            if (chosen < 0 || chosen >= kMaxColours) {
                W.sstate->status = kStatusCapacity;
                chosen = kMaxColours - 1;
            }
            st_colour(col + b, chosen);
            atomicMax(&cs->maxc, chosen + 1);
            progress = true;
        }
        remaining = left;
        if (!left) break;
    }
    if (__any_sync(0xffffffffu, remaining) && (threadIdx.x & 31) == 0) atomicOr(&flags[0], 1);
    if (__any_sync(0xffffffffu, progress) && (threadIdx.x & 31) == 0) atomicOr(&flags[1], 1);
}

// A pass that took more rounds than bodies (cannot happen for a proper
// priority order) stops the step with TIMEOUT.
__global__ void k_col_timeout(const __grid_constant__ World W, ColourState* cs) {
    if (blockIdx.x != 0 || threadIdx.x != 0 || cs->done) return;
    cs->done = 1;
    cs->stalled = 1;
    W.sstate->status = kStatusTimeout;
}

__global__ void k_col_count(const __grid_constant__ World W, ColourState* cs) {
    const SceneDesc sc = W.scenes[0];
    if (cs->skip || cs->stalled) return;
    AVBD_BODIES(b) {
        const int c = W.colour[b];
        if (c >= 0) atomicAdd(&cs->count[c], 1);
    }
}

__global__ void k_col_starts(const __grid_constant__ World W, ColourState* cs) {
    if (cs->skip || cs->stalled || blockIdx.x != 0 || threadIdx.x != 0) return;
    int* out = W.col_start;   // scene slot 0
    const int ncol = cs->maxc;
    int acc = 0;
    for (int c = 0; c < ncol; ++c) { out[c] = acc; acc += cs->count[c]; cs->count[c] = out[c]; }
    out[ncol] = acc;
    W.sstate->ncolours = ncol;
}

// Lanes per body of a scene with energies when the caller fixed none: from
// the step's incidence entries per body (a 0.05 m tet block's particles
// carry about 90, and 32 lanes share them).
__host__ __device__ __forceinline__ int adaptive_group(int ninc, int nbody) {
    const int per_body = (ninc + nbody - 1) / max(nbody, 1);
    return per_body > 48 ? 32 : per_body > 24 ? 16 : 8;
}

// Colour lists, bodies of more work first within a colour (one launch per
// work class, so the classes stay in order).  Work is counted in entries per
// lane of the lanes-per-body the sweep will use (adaptive: from this step's
// incidence, as the host picks it after the colouring).
__global__ void k_col_list(const __grid_constant__ World W, ColourState* cs, int key, int adaptive) {
    const SceneDesc sc = W.scenes[0];
    if (cs->skip || cs->stalled) return;
    const int g = adaptive ? adaptive_group(W.sstate->ninc, sc.nbody)
                           : (sc.group > 0 && sc.group <= 32) ? sc.group : 1;
    AVBD_BODIES(b) {
        const int c = W.colour[b];
        if (c < 0) continue;
        if (min(kColourWorkBuckets - 1, (W.inc_cnt[b] + g - 1) / g) != key) continue;
        const int at = atomicAdd(&cs->count[c], 1);
        if (AVBD_CHECK(W, at >= 0 && at < sc.nbody, 4, at, sc.nbody)) W.col_list[sc.body0 + at] = b;
    }
}

__global__ void k_col_done(const __grid_constant__ World W, const ColourState* cs) {
    if (cs->skip || blockIdx.x != 0 || threadIdx.x != 0) return;
    SceneState* st = W.sstate;
    st->colours_valid = (!cs->stalled && st->status == kStatusOk) ? 1 : 0;
    st->coloured_topo = st->topo;
}

#undef AVBD_BODIES
#undef AVBD_SLOTS

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

// Headless instance export (RenderEngine::UpdateInstanceBuffer,
// RenderEngine.cpp:951-1000): one 128-byte record per live body, packed by
// model type in ModelType order and by body id within a type, the order the
// renderer's per-model batches take.  One CTA: per model, a chunked scan of
// "live body of this model" gives each body its place.
__global__ void __launch_bounds__(1024) k_export_instances(const __grid_constant__ World W, int body0, int nbody,
                                                           AvbdInstance* dst, int cap, int* counts) {
    __shared__ int s_warp[32];
    __shared__ int s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    if (tid == 0) s_base = 0;
    __syncthreads();
    for (int m = 0; m < 3; ++m) {
        if (tid == 0) counts[m] = s_base;   // first instance of this model (counts[3 + m]: how many)
        const int start = s_base;
        __syncthreads();
        for (int c0 = 0; c0 < nbody; c0 += blockDim.x) {
            const int i = c0 + tid;
            bool take = false;
            if (i < nbody) {
                const int fl = W.flags[body0 + i];
                take = !(fl & kBodyRemoved) && ((fl >> kBodyModelShift) & 15) == m;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, take);
            if (lane == 0) s_warp[warp] = __popc(bal);
            __syncthreads();
            int before = 0, total = 0;
            for (int w = 0; w < nwarps; ++w) {
                const int v = s_warp[w];
                if (w < warp) before += v;
                total += v;
            }
            const int k = s_base + before + __popc(bal & ((1u << lane) - 1u));
            if (take && k < cap) {
                const int b = body0 + i;
                const Q4 q = q4(W.rot[b]);
                const M3 R = rotmat(q);
                const float4 s = W.scale[b], p = W.pos[b], col = W.color[b];
                float4* out = reinterpret_cast<float4*>(dst + k);
                // modelMatrix (column-major 4x4): R diag(s) | position
                out[0] = make_float4(R.c[0].x * s.x, R.c[0].y * s.x, R.c[0].z * s.x, 0.f);
                out[1] = make_float4(R.c[1].x * s.y, R.c[1].y * s.y, R.c[1].z * s.y, 0.f);
                out[2] = make_float4(R.c[2].x * s.z, R.c[2].y * s.z, R.c[2].z * s.z, 0.f);
                out[3] = make_float4(p.x, p.y, p.z, 1.f);
                // normalMatrix: (R diag(s))^-T = R diag(1/s), columns padded to 4
                out[4] = make_float4(R.c[0].x / s.x, R.c[0].y / s.x, R.c[0].z / s.x, 0.f);
                out[5] = make_float4(R.c[1].x / s.y, R.c[1].y / s.y, R.c[1].z / s.y, 0.f);
                out[6] = make_float4(R.c[2].x / s.z, R.c[2].y / s.z, R.c[2].z / s.z, 0.f);
                out[7] = make_float4(col.x, col.y, col.z, 1.f);
            }
            __syncthreads();
            if (tid == 0) s_base += total;
            __syncthreads();
        }
        if (tid == 0) counts[3 + m] = s_base - start;
        __syncthreads();
    }
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

}  // namespace

namespace avbd {
namespace host {

int export_instances(const World& W, int body0, int nbody, AvbdInstance* dst, int32_t capacity,
                     int32_t first_per_model[3], int32_t count_per_model[3], cudaStream_t st) {
    if (!dst || capacity < 0) return AVBD_ERR_INVALID;
    cudaPointerAttributes attr{};
    const bool on_device = cudaPointerGetAttributes(&attr, dst) == cudaSuccess &&
                           (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    AvbdInstance* out = dst;
    int* d_counts = nullptr;
    if (cudaMalloc(&d_counts, 6 * sizeof(int)) != cudaSuccess) return AVBD_ERR_NOMEM;
    if (!on_device && capacity > 0 &&
        cudaMalloc(&out, (size_t)capacity * sizeof(AvbdInstance)) != cudaSuccess) {
        cudaFree(d_counts);
        return AVBD_ERR_NOMEM;
    }
    k_export_instances<<<1, 1024, 0, st>>>(W, body0, nbody, out, capacity, d_counts);
    int counts[6] = {};
    cudaMemcpyAsync(counts, d_counts, sizeof(counts), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    const int total = counts[3] + counts[4] + counts[5];
    if (e == cudaSuccess && !on_device && capacity > 0)
        e = cudaMemcpy(dst, out, (size_t)std::min(total, capacity) * sizeof(AvbdInstance), cudaMemcpyDeviceToHost);
    if (!on_device && capacity > 0) cudaFree(out);
    cudaFree(d_counts);
    if (e != cudaSuccess) return AVBD_ERR_CUDA;
    for (int m = 0; m < 3; ++m) {
        if (first_per_model) first_per_model[m] = counts[m];
        if (count_per_model) count_per_model[m] = counts[3 + m];
    }
    return total > capacity ? AVBD_ERR_INVALID : total;
}

}  // namespace host
}  // namespace avbd

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
    GridState* gs = nullptr;
    ColourState* cs = nullptr;
    if (P.alloc(gs, 1) != cudaSuccess || P.alloc(cs, 1) != cudaSuccess) return AVBD_ERR_NOMEM;
    w->grid = gs;
    w->colour = cs;
    w->nbr_cap = 3 * (size_t)P.ninc;
    if (P.alloc(w->nbr, w->nbr_cap, false) != cudaSuccess || P.alloc(w->nbr_cnt, (size_t)P.nb) != cudaSuccess ||
        P.alloc(w->nbr_key, (size_t)P.nb) != cudaSuccess || P.alloc(w->nbr_pos, (size_t)P.nb) != cudaSuccess ||
        P.alloc(w->nbr_used, (size_t)P.nb) != cudaSuccess)
        return AVBD_ERR_NOMEM;
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
    if (3 * (size_t)w->P.ninc > w->nbr_cap) {
        if (w->P.grow(w->nbr, w->nbr_cap, 3 * (size_t)w->P.ninc, 0) != cudaSuccess) return AVBD_ERR_NOMEM;
        w->nbr_cap = 3 * (size_t)w->P.ninc;
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
    const Range range("avbd_step");
    PhaseRanges phases;
    cudaEventRecord(w->ev[0], s);
    phases.next("broadphase");
    // ---- broadphase: uniform grid from kGridMinBodies bodies, else all pairs ----
    const bool use_grid = d.nbody >= kGridMinBodies;
    GridState* gs = static_cast<GridState*>(w->grid);
    if (use_grid) {
        const int nb = blocks_for(d.nbody);
        k_grid_reset<<<1, 32, 0, s>>>(gs);
        k_grid_rmin<<<nb, kThreads, 0, s>>>(P.W, gs);
        k_grid_extent<<<nb, kThreads, 0, s>>>(P.W, gs);
        k_grid_setup<<<1, 32, 0, s>>>(P.W, gs);
        k_grid_clear<<<nb, kThreads, 0, s>>>(P.W, gs);
        k_grid_rank<<<nb, kThreads, 0, s>>>(P.W, gs);
        k_grid_scan<<<1, 1024, 0, s>>>(P.W, gs);
        k_grid_scatter<<<nb, kThreads, 0, s>>>(P.W, gs);
        k_bp_grid<false><<<nb, kThreads, 0, s>>>(P.W, gs, cur);
        k_bp_big<false><<<kGridMaxBig, 1024, 0, s>>>(P.W, gs, cur);
    } else {
        k_bp_count<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W);
    }
    k_scan_cand<<<1, 1024, 0, s>>>(P.W);
    if ((r = sync_state(w))) return r;
    const int ncand = w->st.need_cand;
    if ((r = ensure_caps(w, ncand, 0))) return r;
    if (use_grid) {
        k_bp_grid<true><<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W, gs, cur);
        k_bp_big<true><<<kGridMaxBig, 1024, 0, s>>>(P.W, gs, cur);
    }
    k_bp_write<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W, cur, use_grid ? 0 : 1);
    cudaEventRecord(w->ev[1], s);
    phases.next("narrowphase, warm start, incidence");
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
    // ---- incidence, grid-wide ----
    const int nb = blocks_for(d.nbody), nc = blocks_for(std::max(ncand, 1));
    cudaMemsetAsync(P.W.cntB + d.body0, 0, (size_t)d.nbody * sizeof(int), s);
    k_inc_count_b<<<nc, kThreads, 0, s>>>(P.W, cur);
    k_inc_count<<<nb, kThreads, 0, s>>>(P.W, cur);
    k_inc_scan<<<1, 1024, 0, s>>>(P.W);
    k_inc_fill<<<nb, kThreads, 0, s>>>(P.W, cur);
    k_inc_fill_b<<<nc, kThreads, 0, s>>>(P.W, cur);
    k_inc_sort<<<nb, kThreads, 0, s>>>(P.W, cur);
    cudaEventRecord(w->ev[2], s);
    phases.next("colouring");
    // ---- colouring, grid-wide (skipped when the contact graph is unchanged) ----
    const int adaptive = w->group == 0 && (w->h.ntet() > 0 || w->h.ntri() > 0) && d.nbody > 0;
    {
        ColourState* cs = static_cast<ColourState*>(w->colour);
        const ColourLists L{w->nbr, w->nbr_cnt, w->nbr_key, w->nbr_pos, w->nbr_used};
        k_col_prepare<<<1, 32, 0, s>>>(P.W, cs, cur);
        k_col_init<<<nb, kThreads, 0, s>>>(P.W, cs, L);
        // Rounds in chunks of 8; between chunks the host reads whether the
        // pass has ended (and, after the first, whether colouring is skipped).
        int flags[2] = {0, 0};   // skip, done
        for (int pass = 0; pass < 2 && !flags[0]; ++pass) {
            if (pass == 1) {
                k_col_repass<<<nb, kThreads, 0, s>>>(P.W, cs);
                k_col_next_pass<<<1, 32, 0, s>>>(cs);
            }
            k_col_pred<<<nb, kThreads, 0, s>>>(P.W, cs, L, cur, pass);
            int round = 0;
            flags[1] = 0;
            while (!flags[1] && round <= d.nbody + 2) {
                for (int k = 0; k < 8; ++k, ++round) k_jp_round<<<nb, kThreads, 0, s>>>(P.W, cs, L, pass, round);
                cudaMemcpyAsync(flags, &cs->skip, 2 * sizeof(int), cudaMemcpyDeviceToHost, s);
                if (cudaStreamSynchronize(s) != cudaSuccess) return AVBD_ERR_CUDA;
            }
            if (!flags[1]) k_col_timeout<<<1, 32, 0, s>>>(P.W, cs);
        }
        k_col_count<<<nb, kThreads, 0, s>>>(P.W, cs);
        k_col_starts<<<1, 32, 0, s>>>(P.W, cs);
        for (int key = kColourWorkBuckets - 1; key >= 0; --key) k_col_list<<<nb, kThreads, 0, s>>>(P.W, cs, key, adaptive);
        k_col_done<<<1, 32, 0, s>>>(P.W, cs);
    }
    cudaEventRecord(w->ev[3], s);
    phases.next("prediction");
    if ((r = sync_state(w))) return r;
    if (w->st.status != kStatusOk) return w->st.status == kStatusTimeout ? AVBD_STATUS_TIMEOUT : AVBD_STATUS_CAPACITY;
    const int ncol = w->st.ncolours;
    const int nlive = w->st.nlive[cur];
    // Lanes per body: fixed by avbd_set_group, else by the scene kind and,
    // for scenes with energies, by this step's incidence entries per body
    // (a 0.05 m tet block's particles carry about 90: 32 lanes share them).
    const int group = adaptive ? adaptive_group(w->st.ninc, d.nbody) : d.group;
    w->ncolours = ncol;
    w->col_start.resize(ncol + 1);
    cudaMemcpyAsync(w->col_start.data(), P.W.col_start, (ncol + 1) * sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    // ---- prediction ----
    k_predict<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W);
    cudaEventRecord(w->ev[4], s);
    phases.next("iterations");
    // ---- iterations ----
    const float alpha = w->params.alpha;
    const bool has_fracture = d.nforce > 0;
    for (int it = 0; it < w->params.num_iterations; ++it) {
        for (int c = 0; c < ncol; ++c) {
            const int n = w->col_start[c + 1] - w->col_start[c];
            if (n > 0) launch_primal(group, P.W, cur, w->col_start[c], n, alpha, 0, s);
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
    phases.next("velocity");
    // ---- velocities ----
    k_velocity<<<blocks_for(d.nbody), kThreads, 0, s>>>(P.W);
    if ((r = sync_state(w))) return r;
    cudaEventRecord(w->ev[6], s);
    phases.next("post-stabilisation");
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
            if (n > 0) launch_primal(group, P.W, cur, w->col_start[c], n, 0.f, 1, s);
        }
    }
    cudaEventRecord(w->ev[7], s);
    phases.end();
    if (cudaStreamSynchronize(s) != cudaSuccess) return AVBD_ERR_CUDA;
    if (cudaGetLastError() != cudaSuccess) return AVBD_ERR_CUDA;
    AvbdTimings& t = w->timings;
    t.broad_phase_ms = ev_ms(w->ev[0], w->ev[1]);
    t.warmstart_ms = ev_ms(w->ev[1], w->ev[2]);
    t.colouring_ms = ev_ms(w->ev[2], w->ev[3]);
    t.prediction_ms = ev_ms(w->ev[3], w->ev[4]);
    t.primal_dual_ms = ev_ms(w->ev[4], w->ev[5]);
    t.velocity_update_ms = ev_ms(w->ev[5], w->ev[6]);
    t.post_stab_ms = ev_ms(w->ev[6], w->ev[7]);
    t.total_substep_ms = ev_ms(w->ev[0], w->ev[7]);
    return AVBD_STATUS_OK;
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

int32_t avbd_set_body_color(AvbdWorld* w, int32_t body, const float rgb[3]) {
    if (!w || !rgb || body < 0 || body >= w->h.nbody()) return AVBD_ERR_INVALID;
    w->h.color[body] = make_float4(rgb[0], rgb[1], rgb[2], 1.f);
    if (w->uploaded) {
        cudaSetDevice(w->device);
        if (cudaMemcpy(w->P.W.color + w->descs[0].body0 + body, &w->h.color[body], sizeof(float4),
                       cudaMemcpyHostToDevice) != cudaSuccess)
            return AVBD_ERR_CUDA;
    }
    return 0;
}

int32_t avbd_export_instances(AvbdWorld* w, AvbdInstance* dst, int32_t capacity, int32_t first_per_model[3],
                              int32_t count_per_model[3]) {
    if (!w) return AVBD_ERR_INVALID;
    if (!w->uploaded) {
        int r = upload(w);
        if (r) return r;
    }
    if (cudaSetDevice(w->device) != cudaSuccess) return AVBD_ERR_CUDA;
    return export_instances(w->P.W, w->descs[0].body0, w->h.nbody(), dst, capacity, first_per_model,
                            count_per_model, w->stream);
}

int32_t avbd_make_tet_sphere(AvbdWorld* w, float cx, float cy, float cz, float radius, float res, float E, float nu,
                             float pm, float friction) {
    AVBD_STAGING_ONLY(w);
    if (!(radius > 0.f) || !(res > 0.f) || res > 64.f) return AVBD_ERR_INVALID;
    return w->h.make_tet_sphere(cx, cy, cz, radius, res, E, nu, pm, friction);
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
        const float nan = std::numeric_limits<float>::quiet_NaN();
        for (int i = 0; i < n; ++i) {
            float4 p = w->h.pos[i], q = w->h.rot[i], v = w->h.vel[i], o = w->h.omega[i];
            if (w->h.flags[i] & kBodyRemoved) p = q = v = o = make_float4(nan, nan, nan, nan);
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

int32_t avbd_check_word(const AvbdWorld* w, int32_t out[4]) {
    if (!w || !out) return AVBD_ERR_INVALID;
#ifdef AVBD_CHECKS
    for (int i = 0; i < 4; ++i) out[i] = 0;
    if (!w->uploaded || !w->P.W.check) return 1;
    cudaSetDevice(w->device);
    if (w->stream) cudaStreamSynchronize(w->stream);
    return cudaMemcpy(out, w->P.W.check, 4 * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess ? 1 : AVBD_ERR_CUDA;
#else
    return 0;
#endif
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
