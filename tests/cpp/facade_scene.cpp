// Builds a small scene through the C++ facade (include/avbd.hpp), steps it and
// prints every body's pose as hexadecimal float bits, one body per line.
// tests/test_gpu_parity.py builds the same scene through the Python API and
// compares the bits.
#include <cstdio>
#include <cstring>
#include <vector>

#include "avbd.hpp"

static unsigned bits(float f) {
    unsigned u;
    std::memcpy(&u, &f, 4);
    return u;
}

int main() {
    avbd::Solver s;
    s.AddBody(avbd::ModelType_Cube, 1.f, 0.5f, {0.f, -0.5f, 0.f}, {20.f, 1.f, 20.f}, {}, {}, {}, true);
    int prev = -1;
    for (int i = 0; i < 4; ++i) {
        const int b = s.AddBody(avbd::ModelType_Cube, 1000.f, 0.5f, {0.125f * i, 0.5f + 1.0f * i, 0.f},
                                {1.f, 1.f, 1.f}, {0.f, 0.f, 0.25f * i});
        if (prev >= 0 && i == 3) s.AddJoint(prev, {0.f, 0.5f, 0.f}, b, {0.f, -0.5f, 0.f});
        prev = b;
    }
    const int spring = s.AddSpring(-1, {3.f, 5.f, 0.f}, prev, {0.f, 0.f, 0.f}, 1000.f);
    s.AddSpring(-1, {-3.f, 5.f, 0.f}, prev, {0.f, 0.f, 0.f}, 500.f);
    s.RemoveForce(spring);
    s.MakeTetVolume({4.f, 1.f, 0.f}, 3, 2, 2, 0.5f, 1e4f, 0.3f, 1.f, 0.5f, true);
    for (int k = 0; k < 5; ++k)
        if (s.Step() != AVBD_STATUS_OK) return 2;
    std::vector<avbd::Vec3> p;
    std::vector<avbd::Quat> q;
    s.GetPoses(p, q);
    for (size_t i = 0; i < p.size(); ++i)
        std::printf("%08x %08x %08x %08x %08x %08x %08x\n", bits(p[i].x), bits(p[i].y), bits(p[i].z), bits(q[i].w),
                    bits(q[i].x), bits(q[i].y), bits(q[i].z));
    return 0;
}
