// Host-side staging of one scene, mirroring the reference constructors:
// Solver::AddBody / AddParticle (solver.cpp:50-131), Joint (joint.cpp:24-66),
// Spring (spring.cpp:13-37), NeoHookeanFEM (neohookeanfem.cpp:5-37), STVKFEM
// (stvkfem.cpp:5-35), GeometryHelpers::makeTetVolume (geometry.cpp:30-94).
// Derived quantities (mass, inertia, detection radius, rest rotation, torque
// arm, rest length, Dm^-1, rest volume/area, shape gradients) are computed
// in float with the reference's expression order (this file is compiled with
// -ffp-contract=off), so the device receives the values the reference holds.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>

#include "avbd_common.cuh"

namespace avbd {

struct HostScene {
    // bodies
    std::vector<float4> pos, rot, scale, vel, omega, massI, color;
    std::vector<int> flags;
    std::vector<float> friction;
    // joints / springs
    std::vector<int> ftype;
    std::vector<int2> fbody;
    std::vector<float4> frA, frB, fq, fparam;
    std::vector<float> fk, ffrac, ffmin, ffmax;   // 6 per force
    // Neo-Hookean tets
    std::vector<int4> tidx;
    std::vector<float> tDmInv;
    std::vector<float4> tparam;
    std::vector<int> tkind;   // kTetNeoHookean or kTetStvk
    // StVK triangles
    std::vector<int4> ridx;
    std::vector<float4> rDmInv;
    std::vector<float> rgradN;
    std::vector<float4> rparam;

    int nbody() const { return (int)pos.size(); }
    int nforce() const { return (int)ftype.size(); }
    int ntet() const { return (int)tidx.size(); }
    int ntri() const { return (int)ridx.size(); }
    int ndynamic() const {
        int n = 0;
        for (int f : flags) n += (f & (kBodyStatic | kBodyRemoved)) ? 0 : 1;
        return n;
    }
    void clear() { *this = HostScene(); }

    int add_body(int model, float density, float friction_, const float* p, const float* s, const float* v,
                 const float* q_wxyz, const float* w, bool is_static);
    int add_particle(float mass, float friction_, const float* p, const float* v, bool is_static);
    int set_static(int body, bool is_static);
    int add_spring(int a, const float* rA, int b, const float* rB, float k, float rest, bool rope, float fracture);
    int add_joint(int a, const float* rA, int b, const float* rB, const float* k, const float* fracture);
    int add_nh_tet(const int* v, float E, float nu);
    int add_stvk_tet(const int* v, float E, float nu);
    int add_stvk_tri(const int* v, float E, float nu);
    int make_tet_volume(float ox, float oy, float oz, int nx, int ny, int nz, float cell, float E, float nu,
                        float particle_mass, float friction_, bool pin_min_x, int model = kTetNeoHookean);
    int make_tet_sphere(float cx, float cy, float cz, float radius, float res, float E, float nu,
                        float particle_mass, float friction_);

    // Static incidence (forces then energies per body) and joint/spring partner
    // lists.  Offsets are relative to the scene's own entry / partner arrays;
    // entry indices and partner bodies are global (shifted by the bases).
    void build_static_incidence(std::vector<int>& off, std::vector<int>& cnt, std::vector<int>& nf,
                                std::vector<uint32_t>& ent, std::vector<int>& poff, std::vector<int>& pcnt,
                                std::vector<int2>& partners, int body_base, int force_base, int tet_base,
                                int tri_base) const;
};

}  // namespace avbd
