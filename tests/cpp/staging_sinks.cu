// Host-only check of the scene staging sinks (no GPU needed: nothing here is
// copied to a device; the arena's page-locked allocation falls back to plain
// host memory when no device is present).  Prints OK or the failed checks.
#include <cstdio>
#include <vector>

#include "avbd_pools.h"

using avbd::host::ArenaSink;
using avbd::host::StagedSink;

static int g_failed = 0;
#define EXPECT(cond)                                                        \
    do {                                                                    \
        if (!(cond)) {                                                      \
            std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #cond);    \
            ++g_failed;                                                     \
        }                                                                   \
    } while (0)

int main() {
    // Stand-ins for device arrays: only their addresses are recorded.
    static float4 pos[16], lpos[16], ipos[16], vel[16];
    float4* const to[3] = {pos, lpos, ipos};
    std::vector<float4> pose = {make_float4(1, 2, 3, 0), make_float4(4, 5, 6, 0), make_float4(7, 8, 9, 0)};
    std::vector<float4> rest(3, make_float4(0, 0, 0, 0));
    std::vector<float4> negzero(3, make_float4(-0.f, 0, 0, 0));

    // the pools' arrays as the staging buffers size themselves to them
    avbd::host::Pools pools;
    for (float4* p : {pos, lpos, ipos, vel}) {
        pools.owned.push_back(p);
        pools.owned_bytes.push_back(sizeof(pos));
    }
    {   // staged: one host buffer for the pose, the two copies filled on the device
        StagedSink s;
        s.P = &pools;
        s.put_all(to, 3, pose, 2);
        EXPECT(s.bufs.size() == 1);
        EXPECT(s.bufs.count(reinterpret_cast<char*>(pos)) == 1);
        const StagedSink::Buf& b = s.bufs[reinterpret_cast<char*>(pos)];
        EXPECT(b.lo == 2 * sizeof(float4) && b.hi == 5 * sizeof(float4));
        EXPECT(s.mirrors.size() == 2);
        for (float4* m : {lpos, ipos}) {
            const StagedSink::Mirror& mi = s.mirrors[reinterpret_cast<char*>(m)];
            EXPECT(mi.src == reinterpret_cast<char*>(pos));
            EXPECT(mi.lo == 2 * sizeof(float4) && mi.hi == 5 * sizeof(float4));
        }
        // the mirrors' ranges follow every scene written
        s.put_all(to, 3, pose, 9);
        EXPECT(s.mirrors[reinterpret_cast<char*>(lpos)].hi == 12 * sizeof(float4));
        // all-zero data and cleared ranges are left to the zeroed pools
        s.put(vel, rest, 0);
        s.zero(vel, 0, 16);
        EXPECT(s.bufs.count(reinterpret_cast<char*>(vel)) == 0);
        // -0.0 is not zero bytes: it is copied
        s.put(vel, negzero, 4);
        EXPECT(s.bufs.count(reinterpret_cast<char*>(vel)) == 1);
        EXPECT(!s.overflow);
        // a write past its pool array is refused, written data or zeros
        s.put(vel, pose, 15);
        EXPECT(s.overflow);
        StagedSink t;
        t.P = &pools;
        t.put(vel, rest, 15);
        EXPECT(t.overflow);
    }
    {   // arena: one staged copy, scattered to all three arrays
        ArenaSink a;
        a.put_all(to, 3, pose, 1);
        EXPECT(!a.overflow);
        EXPECT(a.ops.size() == 3);
        EXPECT(a.used == 3 * sizeof(float4));
        if (a.ops.size() == 3) {
            for (int i = 0; i < 3; ++i) {
                EXPECT(a.ops[i].dst == static_cast<void*>(to[i] + 1));
                EXPECT(a.ops[i].off == a.ops[0].off && a.ops[i].bytes == 3 * sizeof(float4));
                EXPECT(!a.ops[i].memset);
            }
        }
        const int64_t table = a.append_table();
        EXPECT(table >= 0 && table % 16 == 0);
    }
    pools.owned.clear();   // stand-ins, not device allocations
    pools.owned_bytes.clear();
    if (g_failed) return 1;
    std::printf("OK\n");
    return 0;
}
