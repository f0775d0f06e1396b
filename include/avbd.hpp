// C++ facade over the AVBD C-ABI with the method names of the reference's
// `class Solver` (src/physics/solver.hpp:22-94), for code that drives the
// reference directly.  Header only; link against libavbd.so.
//
// Differences from the reference surface, as in the C-ABI:
//   * bodies, forces and energies are handles (ids), not owning pointers, and
//     ids stay stable after a removal (the reference swap-removes, solver.cpp:104-115);
//   * Neo-Hookean tets and StVK triangles are added and removed by their own
//     calls (the reference's AddEnergy takes either through a base pointer);
//   * vectors and quaternions are plain structs (the reference uses Eigen);
//   * errors from the C-ABI raise avbd::Error (the reference asserts).
#pragma once

#include <cmath>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "avbd.h"

namespace avbd {

struct Vec3 {
    float x = 0.f, y = 0.f, z = 0.f;
};
// Quaternion in the reference's (w, x, y, z) constructor order.
struct Quat {
    float w = 1.f, x = 0.f, y = 0.f, z = 0.f;
};

enum ModelType { ModelType_Cube = 0 };   // geometry.hpp:17-22 (only boxes collide)

class Error : public std::runtime_error {
  public:
    Error(const std::string& what, int code) : std::runtime_error(what + ": " + avbd_status_string(code)), code_(code) {}
    int code() const { return code_; }

  private:
    int code_;
};

class Solver {
  public:
    // Solver::Solver / Solver::Start (solver.cpp:18-33) on CUDA device `device`.
    explicit Solver(int device = 0) {
        avbd_default_params(&params_);
        check(avbd_world_create(&params_, device, &w_), "avbd_world_create");
    }
    ~Solver() {
        if (w_) avbd_world_destroy(w_);
    }
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;
    Solver(Solver&& o) noexcept : w_(std::exchange(o.w_, nullptr)), params_(o.params_) {}
    Solver& operator=(Solver&& o) noexcept {
        if (this != &o) {
            if (w_) avbd_world_destroy(w_);
            w_ = std::exchange(o.w_, nullptr);
            params_ = o.params_;
        }
        return *this;
    }

    // The reference's public parameters (solver.hpp:64-80): edit, then ApplyParams().
    AvbdParams& params() { return params_; }
    void ApplyParams() { check(avbd_set_params(w_, &params_), "avbd_set_params"); }

    // Solver::AddBody (solver.cpp:50-101); returns the body id.
    int AddBody(ModelType model, float density, float friction, Vec3 pos, Vec3 scale, Vec3 vel = {},
                Quat rot = {}, Vec3 angularVelocity = {}, bool isStatic = false) {
        const float p[3] = {pos.x, pos.y, pos.z}, s[3] = {scale.x, scale.y, scale.z}, v[3] = {vel.x, vel.y, vel.z};
        const float q[4] = {rot.w, rot.x, rot.y, rot.z};
        const float w[3] = {angularVelocity.x, angularVelocity.y, angularVelocity.z};
        return check(avbd_add_body(w_, model, density, friction, p, s, v, q, w, isStatic ? 1 : 0), "avbd_add_body");
    }
    // Solver::AddParticle (solver.cpp:119-131).
    int AddParticle(float mass, float friction, Vec3 pos, Vec3 vel = {}, bool isStatic = false) {
        const float p[3] = {pos.x, pos.y, pos.z}, v[3] = {vel.x, vel.y, vel.z};
        return check(avbd_add_particle(w_, mass, friction, p, v, isStatic ? 1 : 0), "avbd_add_particle");
    }
    // AddForce(std::make_unique<Spring>(...)) (force.hpp:95); bodyA = -1 anchors rA in world space.
    int AddSpring(int bodyA, Vec3 rA, int bodyB, Vec3 rB, float stiffness, float restLength = -1.f,
                  bool isRope = false, float fracture = INFINITY) {
        const float a[3] = {rA.x, rA.y, rA.z}, b[3] = {rB.x, rB.y, rB.z};
        return check(avbd_add_spring(w_, bodyA, a, bodyB, b, stiffness, restLength, isRope ? 1 : 0, fracture),
                     "avbd_add_spring");
    }
    // AddForce(std::make_unique<Joint>(...)) (force.hpp:119-122); per-row stiffness and fracture.
    int AddJoint(int bodyA, Vec3 rA, int bodyB, Vec3 rB, const float stiffness[6], const float fracture[6]) {
        const float a[3] = {rA.x, rA.y, rA.z}, b[3] = {rB.x, rB.y, rB.z};
        return check(avbd_add_joint(w_, bodyA, a, bodyB, b, stiffness, fracture), "avbd_add_joint");
    }
    // A joint with every row hard and unbreakable (the Joint constructor's defaults).
    int AddJoint(int bodyA, Vec3 rA, int bodyB, Vec3 rB) {
        const float inf[6] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY};
        return AddJoint(bodyA, rA, bodyB, rB, inf, inf);
    }
    // AddEnergy(std::make_unique<NeoHookeanFEM>(...)) (energy.hpp:50-52).
    int AddNeoHookeanFEM(int v0, int v1, int v2, int v3, float youngsModulus, float poissonRatio) {
        const int32_t v[4] = {v0, v1, v2, v3};
        return check(avbd_add_neohookean_tet(w_, v, youngsModulus, poissonRatio), "avbd_add_neohookean_tet");
    }
    // AddEnergy(std::make_unique<STVKFEM>(...)) (energy.hpp:90-92).
    int AddSTVKFEM(int v0, int v1, int v2, float youngsModulus, float poissonRatio) {
        const int32_t v[3] = {v0, v1, v2};
        return check(avbd_add_stvk_tri(w_, v, youngsModulus, poissonRatio), "avbd_add_stvk_tri");
    }
    // GeometryHelpers::makeTetVolume (geometry.cpp:30-94); returns the first particle id.
    int MakeTetVolume(Vec3 origin, int nx, int ny, int nz, float cellSize, float youngsModulus, float poissonRatio,
                      float particleMass = 1.f, float friction = 0.5f, bool pinMinX = false) {
        return check(avbd_make_tet_volume(w_, origin.x, origin.y, origin.z, nx, ny, nz, cellSize, youngsModulus,
                                          poissonRatio, particleMass, friction, pinMinX ? 1 : 0),
                     "avbd_make_tet_volume");
    }

    void RemoveBody(int body) { check(avbd_remove_body(w_, body), "avbd_remove_body"); }
    void RemoveForce(int force) { check(avbd_remove_force(w_, force), "avbd_remove_force"); }
    void RemoveNeoHookeanFEM(int tet) { check(avbd_remove_neohookean_tet(w_, tet), "avbd_remove_neohookean_tet"); }
    void RemoveSTVKFEM(int tri) { check(avbd_remove_stvk_tri(w_, tri), "avbd_remove_stvk_tri"); }
    // Solver::Clear (solver.cpp:36-47).
    void Clear() { check(avbd_world_clear(w_), "avbd_world_clear"); }

    // Solver::Step() (solver.cpp:199-627).  Returns AVBD_STATUS_OK, or
    // EXPLODED / NAN (the scene is frozen, as emergencyStop) or CAPACITY /
    // TIMEOUT (the step was not applied).
    int Step() { return check(avbd_step(w_), "avbd_step"); }

    bool emergencyStop() const { return avbd_emergency_stop(w_) != 0; }
    int numBodies() const { return avbd_num_bodies(w_); }
    AvbdTimings timings() const {
        AvbdTimings t{};
        check(avbd_get_timings(w_, &t), "avbd_get_timings");
        return t;
    }
    // Poses of every body (bodyPtrs[i]->transform), by id.
    void GetPoses(std::vector<Vec3>& positions, std::vector<Quat>& rotations) {
        const int n = numBodies();
        std::vector<float> p(3 * (size_t)n), q(4 * (size_t)n);
        check(avbd_get_state(w_, p.data(), q.data(), nullptr, nullptr), "avbd_get_state");
        positions.resize(n);
        rotations.resize(n);
        for (int i = 0; i < n; ++i) {
            positions[i] = Vec3{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
            rotations[i] = Quat{q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
        }
    }
    AvbdWorld* handle() { return w_; }

  private:
    static int check(int r, const char* what) {
        if (r < 0) throw Error(what, r);
        return r;
    }
    AvbdWorld* w_ = nullptr;
    AvbdParams params_{};
};

}  // namespace avbd
