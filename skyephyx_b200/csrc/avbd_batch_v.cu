// One build of the batched persistent kernel: one step of many scenes per
// launch.  Compiled once per build with AVBD_BATCH_ID (1..7) selecting the
// CTA size and register budget (see avbd_batch.h).
#include "avbd_batch.h"
#include "avbd_step.cuh"

#ifndef AVBD_BATCH_ID
#error "compile with -DAVBD_BATCH_ID=<1..7>"
#endif
#if AVBD_BATCH_ID == 1
#define AVBD_MAXT 256
#define AVBD_MINB 1
#elif AVBD_BATCH_ID == 2
#define AVBD_MAXT 256
#define AVBD_MINB 2
#elif AVBD_BATCH_ID == 3
#define AVBD_MAXT 256
#define AVBD_MINB 3
#elif AVBD_BATCH_ID == 4
#define AVBD_MAXT 256
#define AVBD_MINB 4
#elif AVBD_BATCH_ID == 5
#define AVBD_MAXT 512
#define AVBD_MINB 1
#elif AVBD_BATCH_ID == 6
#define AVBD_MAXT 512
#define AVBD_MINB 2
#elif AVBD_BATCH_ID == 7
#define AVBD_MAXT 1024
#define AVBD_MINB 1
#else
#error "AVBD_BATCH_ID must be 1..7"
#endif

namespace avbd {
namespace {

// Runs one scene's step on team T, stamping its start and end when timing is on
// (scene_step stamps the phase ends in between).
__device__ __forceinline__ void timed_scene_step(const World& W, int scene, const Team& T) {
    scene_stamp(W, T, scene, 0);
    scene_step(W, scene, T);
    T.sync();
    scene_stamp(W, T, scene, kSceneStamps - 1);
}

// MAXT is the largest CTA the build serves and MINB sets its register budget
// (about 65536 / (MAXT * MINB) per thread).  The 256-thread builds keep a
// step in about 156 (MINB 1), 128, 80 or 64 registers; the 512- and
// 1024-thread builds give a large scene more lanes.  The autotuner picks one.
//
// A CTA starts as one team pulling scenes from the queue (largest first).  A
// scene whose work (bodies + tets) is at most team_work per lane of half the
// team is run by the lower half while the upper half, now a team of its own,
// pulls the next scene; teams keep splitting this way down to
// Team::min_size(), so small scenes run several to a CTA without waiting on
// each other's barriers.
__device__ __forceinline__ bool scene_fits_half(const World& W, int scene, int team_size) {
    const SceneDesc& d = W.scenes[scene];
    const int work = d.ntet > 0 ? W.fem_team_work : W.team_work;
    if (work <= 0 || team_size / 2 < Team::min_size()) return false;
    return (long long)(d.nbody + d.ntet) <= (long long)work * (team_size / 2);
}

// Launched plain or in thread-block clusters.  In clusters, the scenes at
// the head of the queue (the largest; nlive[1] of them) are each run by a
// whole cluster first; then every CTA pulls the remaining scenes as above.
// Cluster barriers need every thread of the cluster, so the cluster phase
// is left by all of its CTAs together, on the same queue ticket.
template <int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_batch_step(const __grid_constant__ World W, const int* order,
                                                             const int* nlive_ptr, int* queue) {
    __shared__ TeamShared s_team[kMaxTeams];
    extern __shared__ float4 s_stage[];
    const int nlive = nlive_ptr[0];   // live scenes, read from device memory so the graph stays replayable
    const int nlarge = min(nlive_ptr[1], nlive);
    const bool clustered = cooperative_groups::this_cluster().num_blocks() > 1;
    if (clustered && nlarge > 0) {
        const Team C = Team::cluster(s_team, s_stage, W.stage_bodies);
        for (;;) {
            if (C.rank == 0) C.sh->q = atomicAdd(queue + 1, 1);
            C.sync();
            const int q = C.sh->q;
            C.sync();   // every CTA read the ticket before the next one is drawn
            if (q >= nlarge) break;
            timed_scene_step(W, order[q], C);
        }
    }
    const int first = clustered ? nlarge : 0;
    Team T = Team::cta(s_team, s_stage, W.stage_bodies);
    int scene = -1;
    for (;;) {
        if (scene < 0) {
            if (T.rank == 0) T.sh->q = first + atomicAdd(queue, 1);
            T.sync();
            const int q = T.sh->q;
            T.sync();
            if (q >= nlive) break;
            scene = order[q];
        }
        if (scene_fits_half(W, scene, T.size)) {
            const bool lower = T.rank < T.size / 2;
            T = T.half(lower, s_team);
            if (!lower) scene = -1;
            continue;
        }
        timed_scene_step(W, scene, T);
        scene = -1;
    }
}

}  // namespace

#define AVBD_CAT2(a, b) a##b
#define AVBD_CAT(a, b) AVBD_CAT2(a, b)
BatchKernel AVBD_CAT(batch_kernel_v, AVBD_BATCH_ID)() { return k_batch_step<AVBD_MAXT, AVBD_MINB>; }

}  // namespace avbd
