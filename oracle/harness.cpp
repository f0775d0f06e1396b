// CPU oracle for the AVBD step: TEST INFRASTRUCTURE ONLY.
//
// This translation unit is linked with the reference's own, unmodified physics
// sources (src/physics/*.cpp, src/helpers/geometry.cpp, src/helpers/math.cpp of
// SkyePhyX) compiled against the Eigen-API shim in oracle/eigen_shim.  It gives
// the tests and the CPU baseline a C-ABI to:
//   * build scenes through the reference's Solver API (solver.hpp:43-49,
//     force.hpp:95,119-122, energy.hpp:50-52,90-92, geometry.hpp:270);
//   * run the reference's Solver::Step() as written (solver.cpp:199-627);
//   * run orc_step_coloured(): a restatement of Solver::Step() that differs
//     only in the order the primal sweeps (solver.cpp:392-449 and :538-596)
//     visit bodies: colour by colour (ascending colour, ascending body index),
//     with the colouring computed by the CPU twin of the device colouring
//     right after the force warm-start (phase 2).  Every per-force and
//     per-energy computation is the reference's own routine.
//   * read back poses, contact manifolds and colours.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "physics/solver.hpp"
#include "physics/force.hpp"
#include "physics/energy.hpp"
#include "physics/collision.hpp"
#include "constants.hpp"

namespace {

const Eigen::Vector3f kGravity(0.0f, -9.81f, 0.0f);   // solver.cpp:7
const float kPenaltyMin = 1.0f;                       // solver.cpp:9
const float kPenaltyMax = 1000000000.0f;              // solver.cpp:10
const float kMaxRotationVelocity = 50.0f;             // solver.cpp:13
const float kMaxVelocity = 500.0f;                    // solver.cpp:15

struct Orc {
    Solver solver;
    std::vector<Mesh*> bodies;     // by creation id; null once the body is removed
    std::vector<Force*> forces;    // user forces by creation id
    std::vector<Energy*> energies; // by creation id
    std::vector<int> colour;       // by body creation id, -1 = static/uncoloured/removed
    int num_colours = 0;
    double phase_ms[8] = {0};
};

uint32_t colour_hash(uint32_t x) {
    // integer mixer (Wellons "lowbias32"); must equal avbd_colour_priority() on the device
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return x;
}

// CPU twin of the device colouring: greedy first-fit in priority order, where
// priority is (degree descending, hash(creation id), creation id), degree
// being the number of forces and energies a body takes part in; then one
// iterated-greedy pass (priority: first-pass colour descending, then as
// before).  Edges join dynamic bodies that share a force (manifold, joint,
// spring) or an energy.
void colour_bodies(Orc& o) {
    Solver& s = o.solver;
    const int n = (int)s.bodyPtrs.size();
    // creation id of each body by solver index (they differ once a body was
    // swap-removed, solver.cpp:104-115; the device keeps creation ids)
    std::vector<int> cid(n, -1);
    {
        std::unordered_map<const Mesh*, int> id;
        for (size_t i = 0; i < o.bodies.size(); ++i)
            if (o.bodies[i]) id[o.bodies[i]] = (int)i;
        for (int i = 0; i < n; ++i) cid[i] = id.count(s.bodyPtrs[i]) ? id[s.bodyPtrs[i]] : i;
    }
    std::vector<std::vector<int>> adj(n);
    auto link = [&](const std::vector<Mesh*>& lb) {
        for (size_t a = 0; a < lb.size(); ++a)
            for (size_t b = 0; b < lb.size(); ++b) {
                if (a == b) continue;
                Mesh* x = lb[a]; Mesh* y = lb[b];
                if (x->isStatic || y->isStatic || x == y) continue;
                adj[x->solverIndex].push_back(y->solverIndex);
            }
    };
    for (Force* f : s.forcePtrs) link(f->linkedBodies);
    for (Energy* e : s.energyPtrs) link(e->linkedBodies);
    // priority: more forces and energies first (largest degree first), then hash, then index
    std::vector<int> deg(n, 0);
    for (Force* f : s.forcePtrs)
        for (Mesh* m : f->linkedBodies) ++deg[m->solverIndex];
    for (Energy* e : s.energyPtrs)
        for (Mesh* m : e->linkedBodies) ++deg[m->solverIndex];
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        if (deg[a] != deg[b]) return deg[a] > deg[b];
        const int ca = cid[a], cb = cid[b];
        uint32_t ha = colour_hash((uint32_t)ca), hb = colour_hash((uint32_t)cb);
        return ha != hb ? ha < hb : ca < cb;
    });
    auto greedy = [&](const std::vector<int>& ord, std::vector<int>& col) {
        col.assign(n, -1);
        int ncol = 0;
        std::vector<char> used;
        for (int v : ord) {
            if (s.bodyPtrs[v]->isStatic) continue;
            used.assign(ncol + 1, 0);
            for (int u : adj[v]) if (col[u] >= 0) used[col[u]] = 1;
            int c = 0;
            while (used[c]) ++c;
            col[v] = c;
            if (c + 1 > ncol) ncol = c + 1;
        }
        return ncol;
    };
    std::vector<int> col;
    int ncol = greedy(order, col);
    {
        // one iterated-greedy pass (never more colours): the classes in reverse
        // order, each class in the first pass's priority order
        std::vector<int> prev = col;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return prev[a] > prev[b]; });
        ncol = greedy(order, col);
    }
    o.colour.assign(o.bodies.size(), -1);
    for (int i = 0; i < n; ++i)
        if (cid[i] >= 0 && cid[i] < (int)o.colour.size()) o.colour[cid[i]] = col[i];
    o.num_colours = ncol;
}

// Creation ids whose body or user force the solver no longer holds become
// null: bodies removed out of bounds (solver.cpp:530-534), forces dropped by
// Initialize() after a fracture disabled them (:293-294) or destroyed with
// their body (geometry.cpp:11-25).
void forget_removed(Orc& o) {
    std::unordered_set<const Mesh*> live(o.solver.bodyPtrs.begin(), o.solver.bodyPtrs.end());
    for (Mesh*& m : o.bodies)
        if (m && !live.count(m)) m = nullptr;
    std::unordered_set<const Force*> held;
    for (auto& f : o.solver.solverForces) held.insert(f.get());
    for (Force*& f : o.forces)
        if (f && !held.count(f)) f = nullptr;
}

// One primal block update of one body (solver.cpp:394-448; post-stab form
// :540-595 with alpha = 0).
void primal_body(Solver& s, Mesh* mesh, float alpha) {
    const float dt = s.stepValue;
    Matrix6f lhs = mesh->cachedGeneralizedMass / (dt * dt);
    Vector6f rhs = lhs * mesh->GetDisplacementFromInertial();
    for (Force* force : mesh->forces) {
        force->ComputeConstraints(alpha);
        force->ComputeDerivatives(mesh);
        const int nc = force->numConstraints();
        for (int i = 0; i < nc; ++i) {
            ConstraintPointProperties& cp = force->constraintPoints[i];
            float lambda = std::isinf(cp.stiffness) ? cp.lambda : 0.f;
            float f = std::clamp(cp.penalty * cp.C + lambda, cp.fminMagnitude, cp.fmaxMagnitude);
            Matrix6f H = cp.H;
            Matrix6f G = Matrix6f::Zero();
            for (int j = 0; j < 6; ++j) G(j, j) = H.col(j).norm() * std::abs(f);
            const Vector6f J = cp.J;
            rhs += J * f;
            lhs.noalias() += J * J.transpose() * cp.penalty;
            if (force->includeHessian) lhs.noalias() += G;
        }
    }
    for (Energy* energy : mesh->energies) {
        energy->ComputeEnergyTerms(mesh, s.projectionMode, s.trustRegionRho);
        rhs += energy->grad;
        lhs += energy->hess;
    }
    Eigen::LDLT<Matrix6f> ldlt;
    ldlt.compute(lhs);
    Vector6f dx = ldlt.solve(rhs);
    Eigen::Vector3f dx_lin = dx.head<3>();
    Eigen::Vector3f dx_ang = dx.tail<3>();
    Eigen::Vector3f pos = mesh->transform.GetPosition();
    mesh->transform.SetPosition(pos - dx_lin);
    Quaternionf dq = QuaternionFromDifference(dx_ang, -1.f);
    Quaternionf rot = mesh->transform.GetRotation();
    mesh->transform.SetRotation((dq * rot).normalized());
}

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Restatement of Solver::Step() (solver.cpp:199-627) with colour-ordered
// primal sweeps.  identity_order = 1 visits bodies in index order, which is
// exactly the reference's order (self-check: bitwise equal to Solver::Step()).
int step_coloured(Orc& o, int identity_order) {
    Solver& s = o.solver;
    if (s.emergencyStop) return 1;                                         // :201
    auto t0 = std::chrono::steady_clock::now();
    s.RebuildPtrCaches();
    for (Mesh* mesh : s.bodyPtrs) {                                         // :215-231
        if (mesh->isStatic) continue;
        Quaternionf q = mesh->transform.GetRotation();
        mesh->cachedRotationMatrix = q.toRotationMatrix();
        if (!mesh->isStatic && mesh->mass > 0.f) {
            Matrix6f& M = mesh->cachedGeneralizedMass;
            M.setZero();
            M.block<3, 3>(0, 0) = Eigen::Matrix3f::Identity() * mesh->mass;
            M.block<3, 3>(3, 3) = mesh->cachedRotationMatrix * mesh->inertiaTensorBody *
                                  mesh->cachedRotationMatrix.transpose();
        }
    }
    auto tp = std::chrono::steady_clock::now();
    const int N = (int)s.bodyPtrs.size();                                   // :233-256
    for (int i = 0; i < N; ++i)
        for (int j = i + 1; j < N; ++j) {
            Mesh* a = s.bodyPtrs[i];
            Mesh* b = s.bodyPtrs[j];
            float distance = (a->transform.GetPosition() - b->transform.GetPosition()).norm();
            if (distance < a->detectionRadius + b->detectionRadius)
                if (!isConstrainedTo(a, b)) s.AddForce(std::make_unique<Manifold>(&s, a, b));
        }
    o.phase_ms[0] = ms_since(tp);
    tp = std::chrono::steady_clock::now();
    s.forcePtrs.clear();                                                    // :259-297
    for (auto& f : s.solverForces) s.forcePtrs.push_back(f.get());
    std::vector<Force*> toRemove;
    for (Force* force : s.forcePtrs) {
        if (!force->Initialize()) { toRemove.push_back(force); continue; }
        const int nc = force->numConstraints();
        for (int i = 0; i < nc; ++i) {
            ConstraintPointProperties& cp = force->constraintPoints[i];
            if (!s.postStabilization) cp.lambda *= s.alpha * s.gamma;
            float p = cp.penalty * s.gamma;
            if (p < kPenaltyMin) p = kPenaltyMin;
            if (p > kPenaltyMax) p = kPenaltyMax;
            cp.penalty = p;
            cp.penalty = std::min(cp.penalty, cp.stiffness);
        }
    }
    for (Force* f : toRemove) s.RemoveForce(f);
    s.forcePtrs.clear();
    for (auto& f : s.solverForces) s.forcePtrs.push_back(f.get());
    s.energyPtrs.clear();                                                   // :299-322
    for (auto& e : s.solverEnergies) s.energyPtrs.push_back(e.get());
    std::vector<Energy*> eRemove;
    for (Energy* e : s.energyPtrs) {
        if (!e->Initialize()) { eRemove.push_back(e); continue; }
        e->ComputeEnergyTerms(nullptr, s.projectionMode, s.trustRegionRho);
    }
    for (Energy* e : eRemove) s.RemoveEnergy(e);
    s.energyPtrs.clear();
    for (auto& e : s.solverEnergies) s.energyPtrs.push_back(e.get());
    o.phase_ms[1] = ms_since(tp);

    // colouring (new; CPU twin of the device colouring)
    tp = std::chrono::steady_clock::now();
    std::vector<Mesh*> sweep;
    if (identity_order) {
        for (Mesh* m : s.bodyPtrs) sweep.push_back(m);
        o.colour.assign(o.bodies.size(), -1);
        o.num_colours = 0;
    } else {
        colour_bodies(o);
        // ascending colour, ascending creation id within a colour
        for (int c = 0; c < o.num_colours; ++c)
            for (size_t i = 0; i < o.bodies.size(); ++i)
                if (o.bodies[i] && o.colour[i] == c) sweep.push_back(o.bodies[i]);
    }
    o.phase_ms[2] = ms_since(tp);

    tp = std::chrono::steady_clock::now();
    const float dt = s.stepValue;                                           // :324-385
    for (Mesh* mesh : s.bodyPtrs) {
        mesh->angularVelocity = mesh->angularVelocity
            .cwiseMin(Eigen::Vector3f::Constant(kMaxRotationVelocity))
            .cwiseMax(Eigen::Vector3f::Constant(-kMaxRotationVelocity));
        Eigen::Vector3f pos = mesh->transform.GetPosition();
        mesh->inertialPosition = pos + mesh->velocity * dt;
        if (!mesh->isStatic) mesh->inertialPosition += kGravity * dt * dt;
        Quaternionf rot = mesh->transform.GetRotation();
        mesh->inertialRotation = rot;
        if (!mesh->isStatic && !mesh->isParticle) {
            Quaternionf q = mesh->inertialRotation;
            Quaternionf w(0.f, mesh->angularVelocity.x(), mesh->angularVelocity.y(), mesh->angularVelocity.z());
            Quaternionf wq;
            wq.w() = w.w() * q.w() - w.vec().dot(q.vec());
            wq.vec() = w.w() * q.vec() + q.w() * w.vec() + w.vec().cross(q.vec());
            q.w() += 0.5f * wq.w() * dt;
            q.vec() += 0.5f * wq.vec() * dt;
            mesh->inertialRotation = q.normalized();
        }
        Eigen::Vector3f linearAcceleration = (mesh->velocity - mesh->prevVelocity) / dt;
        float gravityMagnitude = kGravity.norm();
        float accelWeight = 0.0f;
        if (gravityMagnitude > 1e-6f) {
            Eigen::Vector3f gravityDir = kGravity / gravityMagnitude;
            float accelAlongGravity = linearAcceleration.dot(gravityDir);
            accelWeight = accelAlongGravity / gravityMagnitude;
            accelWeight = std::clamp(accelWeight, 0.f, 1.f);
        }
        mesh->lastPosition = pos;
        mesh->lastRotation = rot;
        Eigen::Vector3f newPos = pos + mesh->velocity * dt + kGravity * dt * dt * accelWeight;
        mesh->transform.SetPosition(newPos);
        if (!mesh->isStatic && !mesh->isParticle) {
            Quaternionf q = rot;
            Quaternionf w(0.f, mesh->angularVelocity.x(), mesh->angularVelocity.y(), mesh->angularVelocity.z());
            Quaternionf wq;
            wq.w() = w.w() * q.w() - w.vec().dot(q.vec());
            wq.vec() = w.w() * q.vec() + q.w() * w.vec() + w.vec().cross(q.vec());
            q.w() += 0.5f * wq.w() * dt;
            q.vec() += 0.5f * wq.vec() * dt;
            mesh->transform.SetRotation(q.normalized());
        }
    }
    o.phase_ms[3] = ms_since(tp);

    tp = std::chrono::steady_clock::now();
    for (int iter = 0; iter < s.numIterations; ++iter) {                   // :389-490
        for (Mesh* mesh : sweep) {
            if (mesh->isStatic) continue;
            primal_body(s, mesh, s.alpha);
        }
        for (Force* force : s.forcePtrs) {                                  // :457-489
            force->ComputeConstraints(s.alpha);
            const int nc = force->numConstraints();
            for (int i = 0; i < nc; ++i) {
                ConstraintPointProperties& cp = force->constraintPoints[i];
                float lambda = std::isinf(cp.stiffness) ? cp.lambda : 0.f;
                cp.lambda = lambda + cp.penalty * cp.C;
                if (cp.lambda < cp.fminMagnitude) cp.lambda = cp.fminMagnitude;
                else if (cp.lambda > cp.fmaxMagnitude) cp.lambda = cp.fmaxMagnitude;
                if (std::abs(cp.lambda) >= cp.fracture) {
                    for (Mesh* body : force->linkedBodies)
                        for (Force* other : body->forces)
                            if (other->isManifold) other->ResetValues();
                    force->Disable();
                    break;
                }
                if (cp.lambda > cp.fminMagnitude && cp.lambda < cp.fmaxMagnitude)
                    cp.penalty = std::min(cp.penalty + s.beta * std::abs(cp.C), std::min(cp.stiffness, kPenaltyMax));
            }
        }
    }
    o.phase_ms[4] = ms_since(tp);

    tp = std::chrono::steady_clock::now();
    std::vector<Mesh*> oob;                                                 // :493-534
    for (Mesh* mesh : s.bodyPtrs) {
        if (mesh->isStatic) continue;
        mesh->prevVelocity = mesh->velocity;
        mesh->prevAngularVelocity = mesh->angularVelocity;
        Eigen::Vector3f pos = mesh->transform.GetPosition();
        Eigen::Vector3f newVelocity = (pos - mesh->lastPosition) / dt;
        if (mesh->isDragged) { newVelocity += mesh->addedDragVelocity; mesh->addedDragVelocity.setZero(); }
        mesh->velocity = newVelocity;
        if (!mesh->isParticle)
            mesh->angularVelocity = RotationDifference(mesh->transform.GetRotation(), mesh->lastRotation) / dt;
        Eigen::Vector3f p = mesh->transform.GetPosition();
        if (p.x() < MINBOUNDS[0] || p.x() > MAXBOUNDS[0] || p.y() < MINBOUNDS[1] || p.y() > MAXBOUNDS[1] ||
            p.z() < MINBOUNDS[2] || p.z() > MAXBOUNDS[2])
            oob.push_back(mesh);
    }
    for (Mesh* mesh : s.bodyPtrs) {                                         // :182-196
        const Eigen::Vector3f& v = mesh->velocity;
        if (v.x() > kMaxVelocity || v.y() > kMaxVelocity || v.z() > kMaxVelocity ||
            v.x() < -kMaxVelocity || v.y() < -kMaxVelocity || v.z() < -kMaxVelocity) {
            s.emergencyStop = true;
            break;
        }
    }
    if (s.emergencyStop) { forget_removed(o); return 1; }
    o.phase_ms[5] = ms_since(tp);
    if (!oob.empty()) {
        // The post-stabilisation sweep visits the surviving bodies only: the
        // reference walks bodyPtrs as RemoveBody's swap leaves it (identity
        // order), the coloured harness keeps its colour order.
        std::unordered_set<const Mesh*> gone(oob.begin(), oob.end());
        std::vector<Mesh*> kept;
        for (Mesh* m : sweep)
            if (!gone.count(m)) kept.push_back(m);
        sweep.swap(kept);
        for (size_t i = 0; i < o.bodies.size(); ++i)
            if (gone.count(o.bodies[i])) { o.bodies[i] = nullptr; if (i < o.colour.size()) o.colour[i] = -1; }
        for (Mesh* m : oob) s.RemoveBody(m);
        if (identity_order) sweep.assign(s.bodyPtrs.begin(), s.bodyPtrs.end());
    }

    tp = std::chrono::steady_clock::now();
    if (s.postStabilization)                                                // :536-597
        for (Mesh* mesh : sweep) {
            if (mesh->isStatic) continue;
            primal_body(s, mesh, 0.0f);
        }
    o.phase_ms[6] = ms_since(tp);
    o.phase_ms[7] = ms_since(t0);
    forget_removed(o);
    return 0;
}

Mesh* body_or_null(Orc* o, int id) {
    if (id < 0 || id >= (int)o->bodies.size()) return nullptr;
    return o->bodies[id];
}

}  // namespace

extern "C" {

void* orc_create(void) { return new Orc(); }
void orc_destroy(void* h) { delete static_cast<Orc*>(h); }

// Solver public parameters (solver.hpp:69-84).
void orc_set_params(void* h, int iterations, float dt, float alpha, float beta, float gamma,
                    float on_penetration_penalty, int post_stabilization, int projection_mode) {
    Solver& s = static_cast<Orc*>(h)->solver;
    s.numIterations = iterations;
    s.stepValue = dt;
    s.alpha = alpha;
    s.beta = beta;
    s.gamma = gamma;
    s.onPenetrationPenalty = on_penetration_penalty;
    s.postStabilization = post_stabilization != 0;
    s.projectionMode = (EigenProjectionMode)projection_mode;
}

// Solver::AddBody (solver.cpp:50-101); quat is (w, x, y, z).
int orc_add_box(void* h, int model_type, float density, float friction, const float* pos, const float* scale,
                const float* vel, const float* quat, const float* omega, int is_static) {
    Orc* o = static_cast<Orc*>(h);
    Mesh* m = o->solver.AddBody((ModelType)model_type, density, friction,
                                Eigen::Vector3f(pos[0], pos[1], pos[2]),
                                Eigen::Vector3f(scale[0], scale[1], scale[2]),
                                Eigen::Vector3f(vel[0], vel[1], vel[2]),
                                Quaternionf(quat[0], quat[1], quat[2], quat[3]),
                                Eigen::Vector3f(omega[0], omega[1], omega[2]), is_static != 0);
    o->bodies.push_back(m);
    return (int)o->bodies.size() - 1;
}

// n x Solver::AddBody from arrays (vel / omega may be null = zero).
int orc_add_bodies(void* h, int n, int model_type, const float* density, const float* friction, const float* pos,
                   const float* scale, const float* vel, const float* quat, const float* omega, const int* is_static) {
    const float zero[3] = {0.f, 0.f, 0.f};
    int first = -1;
    for (int i = 0; i < n; ++i) {
        int id = orc_add_box(h, model_type, density[i], friction[i], pos + 3 * i, scale + 3 * i,
                             vel ? vel + 3 * i : zero, quat + 4 * i, omega ? omega + 3 * i : zero, is_static[i]);
        if (i == 0) first = id;
    }
    return first;
}

// Solver::AddParticle (solver.cpp:119-131).
int orc_add_particle(void* h, float mass, float friction, const float* pos, const float* vel, int is_static) {
    Orc* o = static_cast<Orc*>(h);
    Mesh* m = o->solver.AddParticle(mass, friction, Eigen::Vector3f(pos[0], pos[1], pos[2]),
                                    Eigen::Vector3f(vel[0], vel[1], vel[2]), is_static != 0);
    m->isParticle = true;
    o->bodies.push_back(m);
    return (int)o->bodies.size() - 1;
}

// Pinning after creation, as levels.h:472-473 does with isStatic.
int orc_set_static(void* h, int body, int is_static) {
    Mesh* m = body_or_null(static_cast<Orc*>(h), body);
    if (!m) return -1;
    m->isStatic = is_static != 0;
    return 0;
}

// Spring (force.hpp:95, spring.cpp:13-37); a = -1 anchors rA in world space.
int orc_add_spring(void* h, int a, const float* rA, int b, const float* rB, float stiffness, float rest_length,
                   int is_rope, float fracture) {
    Orc* o = static_cast<Orc*>(h);
    Mesh* B = body_or_null(o, b);
    if (!B) return -1;
    Spring* sp = new Spring(&o->solver, body_or_null(o, a), Eigen::Vector3f(rA[0], rA[1], rA[2]), B,
                            Eigen::Vector3f(rB[0], rB[1], rB[2]), stiffness, rest_length, is_rope != 0);
    sp->constraintPoints[0].fracture = fracture;
    o->solver.AddForce(std::unique_ptr<Force>(sp));
    o->forces.push_back(sp);
    return (int)o->forces.size() - 1;
}

// Joint (force.hpp:119-122, joint.cpp:24-66).
int orc_add_joint(void* h, int a, const float* rA, int b, const float* rB, const float* stiffness,
                  const float* fracture) {
    Orc* o = static_cast<Orc*>(h);
    Mesh* B = body_or_null(o, b);
    if (!B) return -1;
    Vector6f k, fr;
    for (int i = 0; i < 6; ++i) { k[i] = stiffness[i]; fr[i] = fracture[i]; }
    Joint* j = new Joint(&o->solver, body_or_null(o, a), Eigen::Vector3f(rA[0], rA[1], rA[2]), B,
                         Eigen::Vector3f(rB[0], rB[1], rB[2]), k, fr);
    o->solver.AddForce(std::unique_ptr<Force>(j));
    o->forces.push_back(j);
    return (int)o->forces.size() - 1;
}

// NeoHookeanFEM (energy.hpp:50-52, neohookeanfem.cpp:5-37).
int orc_add_nh_tet(void* h, const int* v, float E, float nu) {
    Orc* o = static_cast<Orc*>(h);
    Mesh* b[4];
    for (int i = 0; i < 4; ++i) if (!(b[i] = body_or_null(o, v[i]))) return -1;
    Energy* e = o->solver.AddEnergy(std::make_unique<NeoHookeanFEM>(&o->solver, b[0], b[1], b[2], b[3], E, nu));
    o->energies.push_back(e);
    return (int)o->energies.size() - 1;
}

// St. Venant-Kirchhoff tet: no counterpart in the reference (which has the StVK
// triangle only).  Restated here from the energy Psi = mu tr(E^2) +
// lambda/2 tr(E)^2, E = (F^T F - I)/2, on the reference's own machinery: the
// rest data exactly as the NeoHookeanFEM constructor (neohookeanfem.cpp:5-37),
// NeoHookeanMath::svd / ProjectEigenvalues / ReconstructVertexHessian
// (math.cpp), and the principal-stretch eigen-system of StVK: scaling block
// d2psi/ds_i ds_j of psi = mu/4 sum (s_i^2 - 1)^2 + lambda/8 (sum s_i^2 - 3)^2
// and twist / flip eigenvalues (psi_i +- psi_j)/(s_i +- s_j) in closed form,
// ordered as NeoHookeanMath::ComputeEnergyHessian orders its own.  An element
// below 1% of its rest volume takes STVKFEM's isotropic penalty
// (stvkfem.cpp:75-86).  Parity against a reference implementation is unpinned.
struct StvkTetEnergy : Energy {
    Mesh *body0, *body1, *body2, *body3;
    float restVolume, lameMu, lameLambda;
    Eigen::Matrix3f DmInv;
    Eigen::Vector3f gradN0, gradN1, gradN2, gradN3;
    float trustRegionThreshold = 0.01f;

    StvkTetEnergy(Solver* solver, Mesh* b0, Mesh* b1, Mesh* b2, Mesh* b3, float E, float nu)
        : Energy(solver, {b0, b1, b2, b3}), body0(b0), body1(b1), body2(b2), body3(b3) {
        lameMu = E / (2.f * (1.f + nu));
        lameLambda = E * nu / ((1.f + nu) * (1.f - 2.f * nu));
        const Eigen::Vector3f p0 = b0->transform.GetPosition(), p1 = b1->transform.GetPosition();
        const Eigen::Vector3f p2 = b2->transform.GetPosition(), p3 = b3->transform.GetPosition();
        Eigen::Matrix3f Dm;
        Dm.col(0) = p1 - p0;
        Dm.col(1) = p2 - p0;
        Dm.col(2) = p3 - p0;
        DmInv = Dm.inverse();
        restVolume = std::abs(Dm.determinant()) / 6.f;
        const Eigen::Matrix3f DmInvT = DmInv.transpose();
        gradN1 = DmInvT.col(0);
        gradN2 = DmInvT.col(1);
        gradN3 = DmInvT.col(2);
        gradN0 = -gradN1 - gradN2 - gradN3;
    }
    bool Initialize() override { return true; }
    int numBodies() const override { return 4; }
    void AddLineData(std::vector<GPULineData>&) const override {}
    void AddDebugPointData(std::vector<GPUDebugPointData>&) const override {}

    void ComputeEnergyTerms(Mesh* mesh, EigenProjectionMode projectionMode, float trustRegionRho) override {
        using namespace NeoHookeanMath;
        const Eigen::Vector3f p0 = body0->transform.GetPosition(), p1 = body1->transform.GetPosition();
        const Eigen::Vector3f p2 = body2->transform.GetPosition(), p3 = body3->transform.GetPosition();
        const Eigen::Matrix3f F = DeformationGradient(p0, p1, p2, p3, DmInv);
        const float J = F.determinant();
        Eigen::Vector3f gradN = gradN0;
        if (mesh == body1) gradN = gradN1;
        else if (mesh == body2) gradN = gradN2;
        else if (mesh == body3) gradN = gradN3;
        grad.setZero();
        hess.setZero();
        if (J < 0.01f) {
            const float stiff = lameMu + lameLambda;
            grad.head<3>() = restVolume * ((stiff * F) * gradN);
            hess.block<3, 3>(0, 0) = restVolume * stiff * Eigen::Matrix3f::Identity();
            return;
        }
        const Eigen::Matrix3f E = 0.5f * (F.transpose() * F - Eigen::Matrix3f::Identity());
        const Eigen::Matrix3f S = 2.f * lameMu * E + lameLambda * E.trace() * Eigen::Matrix3f::Identity();
        const Eigen::Matrix3f P = F * S;
        grad.head<3>() = P * gradN * restVolume;

        const SVDDecomposition d = svd(F);
        const float s0 = d.S(0), s1 = d.S(1), s2 = d.S(2);
        const float q0 = s0 * s0, q1 = s1 * s1, q2 = s2 * s2;
        const float mu = lameMu, lam = lameLambda;
        const float c = 0.5f * lam * (q0 + q1 + q2 - 3.f);
        HessianDecomposition h{};
        h.eigenValues[3] = mu * (q0 - s0 * s1 + q1 - 1.f) + c;   // twist (0,1)
        h.eigenValues[4] = mu * (q0 - s0 * s2 + q2 - 1.f) + c;   // twist (0,2)
        h.eigenValues[5] = mu * (q1 - s1 * s2 + q2 - 1.f) + c;   // twist (1,2)
        h.eigenValues[6] = mu * (q0 + s0 * s1 + q1 - 1.f) + c;   // flip (0,1)
        h.eigenValues[7] = mu * (q0 + s0 * s2 + q2 - 1.f) + c;   // flip (0,2)
        h.eigenValues[8] = mu * (q1 + s1 * s2 + q2 - 1.f) + c;   // flip (1,2)
        Eigen::Matrix3f a;
        a(0, 0) = mu * (3.f * q0 - 1.f) + c + lam * q0;
        a(1, 1) = mu * (3.f * q1 - 1.f) + c + lam * q1;
        a(2, 2) = mu * (3.f * q2 - 1.f) + c + lam * q2;
        a(0, 1) = a(1, 0) = lam * s0 * s1;
        a(0, 2) = a(2, 0) = lam * s0 * s2;
        a(1, 2) = a(2, 1) = lam * s1 * s2;
        Eigen::SelfAdjointEigenSolver<Eigen::Matrix3f> es(a);
        for (int k = 0; k < 3; ++k) {
            h.eigenValues[k] = es.eigenvalues()(k);
            h.scalingVectors[k] = es.eigenvectors().col(k);
        }
        float proj[9];
        for (int i = 0; i < 9; ++i) proj[i] = h.eigenValues[i];
        ProjectEigenvalues(proj, 9, projectionMode, trustRegionRho, trustRegionThreshold);
        hess.block<3, 3>(0, 0) = ReconstructVertexHessian(d, h, proj, gradN, restVolume);
    }
};

int orc_add_stvk_tet(void* h, const int* v, float E, float nu) {
    Orc* o = static_cast<Orc*>(h);
    Mesh* b[4];
    for (int i = 0; i < 4; ++i) if (!(b[i] = body_or_null(o, v[i]))) return -1;
    Energy* e = o->solver.AddEnergy(std::make_unique<StvkTetEnergy>(&o->solver, b[0], b[1], b[2], b[3], E, nu));
    o->energies.push_back(e);
    return (int)o->energies.size() - 1;
}

// STVKFEM triangle membrane (energy.hpp:90-92, stvkfem.cpp:5-35).
int orc_add_stvk_tri(void* h, const int* v, float E, float nu) {
    Orc* o = static_cast<Orc*>(h);
    Mesh* b[3];
    for (int i = 0; i < 3; ++i) if (!(b[i] = body_or_null(o, v[i]))) return -1;
    Energy* e = o->solver.AddEnergy(std::make_unique<STVKFEM>(&o->solver, b[0], b[1], b[2], E, nu));
    o->energies.push_back(e);
    return (int)o->energies.size() - 1;
}

// GeometryHelpers::makeTetVolume (geometry.cpp:30-94) through the reference
// itself; bodies and energies it creates are appended in creation order.
int orc_make_tet_volume(void* h, float ox, float oy, float oz, int nx, int ny, int nz, float cell, float E, float nu,
                        float particle_mass, float friction, int pin_min_x) {
    Orc* o = static_cast<Orc*>(h);
    const size_t b0 = o->solver.solverBodies.size();
    const size_t e0 = o->solver.solverEnergies.size();
    GeometryHelpers::makeTetVolume(&o->solver, ox, oy, oz, nx, ny, nz, cell, E, nu, Eigen::Vector3f(1, 1, 1),
                                   particle_mass, friction, pin_min_x != 0);
    const int first = (int)o->bodies.size();
    for (size_t i = b0; i < o->solver.solverBodies.size(); ++i) o->bodies.push_back(o->solver.solverBodies[i].get());
    for (size_t i = e0; i < o->solver.solverEnergies.size(); ++i)
        o->energies.push_back(o->solver.solverEnergies[i].get());
    return first;
}

// GeometryHelpers::makeTetSphere (geometry.cpp:106-232), the reference's own.
int orc_make_tet_sphere(void* h, float cx, float cy, float cz, float radius, float res, float E, float nu,
                        float particle_mass, float friction) {
    Orc* o = static_cast<Orc*>(h);
    const size_t b0 = o->solver.solverBodies.size();
    const size_t e0 = o->solver.solverEnergies.size();
    GeometryHelpers::makeTetSphere(&o->solver, cx, cy, cz, radius, res, E, nu, Eigen::Vector3f(1, 1, 1),
                                   particle_mass, friction);
    const int first = (int)o->bodies.size();
    for (size_t i = b0; i < o->solver.solverBodies.size(); ++i) o->bodies.push_back(o->solver.solverBodies[i].get());
    for (size_t i = e0; i < o->solver.solverEnergies.size(); ++i)
        o->energies.push_back(o->solver.solverEnergies[i].get());
    return first;
}

// makeTetVolume's particles and tets (geometry.cpp:30-94) with StVK tets: the
// reference builds the volume with Neo-Hookean tets, which are then replaced,
// in creation order, by StVK tets on the same bodies.
int orc_make_stvk_tet_volume(void* h, float ox, float oy, float oz, int nx, int ny, int nz, float cell, float E,
                             float nu, float particle_mass, float friction, int pin_min_x) {
    Orc* o = static_cast<Orc*>(h);
    const size_t e0 = o->solver.solverEnergies.size();
    const int first = orc_make_tet_volume(h, ox, oy, oz, nx, ny, nz, cell, E, nu, particle_mass, friction, pin_min_x);
    std::vector<NeoHookeanFEM*> made;
    for (size_t i = e0; i < o->solver.solverEnergies.size(); ++i)
        made.push_back(static_cast<NeoHookeanFEM*>(o->solver.solverEnergies[i].get()));
    const size_t k0 = o->energies.size() - made.size();
    o->energies.resize(k0);
    for (NeoHookeanFEM* nh : made) {
        Mesh* b[4] = {nh->body0, nh->body1, nh->body2, nh->body3};
        o->solver.RemoveEnergy(nh);
        o->energies.push_back(o->solver.AddEnergy(std::make_unique<StvkTetEnergy>(&o->solver, b[0], b[1], b[2], b[3],
                                                                                  E, nu)));
    }
    return first;
}

// The reference step, unmodified.
int orc_step(void* h) {
    Orc* o = static_cast<Orc*>(h);
    if (o->solver.emergencyStop) return 1;
    o->solver.Step();
    forget_removed(*o);
    return o->solver.emergencyStop ? 1 : 0;
}

int orc_step_coloured(void* h, int identity_order) { return step_coloured(*static_cast<Orc*>(h), identity_order); }

// Runs `steps` reference steps on each of n solvers spread over `threads`
// host threads (independent Solver instances share no mutable state).
double orc_step_many(void** hs, int n, int steps, int threads, int coloured) {
    auto t0 = std::chrono::steady_clock::now();
    if (threads < 1) threads = 1;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([=]() {
            for (int i = t; i < n; i += threads)
                for (int k = 0; k < steps; ++k) {
                    if (coloured) step_coloured(*static_cast<Orc*>(hs[i]), 0);
                    else orc_step(hs[i]);
                }
        });
    for (auto& th : pool) th.join();
    return ms_since(t0);
}

int orc_num_bodies(void* h) { return (int)static_cast<Orc*>(h)->bodies.size(); }
int orc_num_dynamic(void* h) {
    int n = 0;
    for (Mesh* m : static_cast<Orc*>(h)->solver.bodyPtrs) n += m->isStatic ? 0 : 1;
    return n;
}
int orc_emergency_stop(void* h) { return static_cast<Orc*>(h)->solver.emergencyStop ? 1 : 0; }

// Long-horizon measures of the current state, from the reference's own
// routines, so that a GPU run (its poses written in with orc_set_state) and
// the FP64 run are measured the same way:
//   out[0] max |C| over hard rows (infinite stiffness: the joints' locked
//          rows) at alpha = 0, i.e. the raw positional / torque-arm-scaled
//          angular violation (Joint::ComputeConstraints, joint.cpp:97-124);
//          soft rows (springs, a hinge's free rows) are not constraints;
//   out[1] deepest penetration over every overlapping body pair: the
//          broadphase sphere test (solver.cpp:233-256), then
//          CollisionSpace::CollisionBoxBox (collision.cpp:271-447);
//   out[2] kinetic energy, 1/2 m v.v + 1/2 w.(R I R^T) w of dynamic bodies;
//   out[3] gravitational potential energy, m 9.81 y of dynamic bodies;
//   out[4] elastic energy, the sum of Energy::cachedEnergy after
//          ComputeEnergyTerms(nullptr, ...) (the warm start, solver.cpp:299-322);
//   out[5] dynamic bodies whose position is not finite.
void orc_metrics(void* h, double* out) {
    Orc* o = static_cast<Orc*>(h);
    Solver& s = o->solver;
    s.RebuildPtrCaches();
    double maxC = 0.0, maxPen = 0.0, kin = 0.0, pot = 0.0, ela = 0.0, bad = 0.0;
    for (auto& fp : s.solverForces) {
        Force* f = fp.get();
        if (f->isManifold || f->disabled) continue;
        f->ComputeConstraints(0.0f);
        for (int i = 0; i < f->numConstraints(); ++i) {
            if (!std::isinf(f->constraintPoints[i].stiffness)) continue;
            const double c = std::abs((double)f->constraintPoints[i].C);
            if (c > maxC || c != c) maxC = c;
        }
    }
    const int N = (int)s.bodyPtrs.size();
    for (int i = 0; i < N; ++i)
        for (int j = i + 1; j < N; ++j) {
            Mesh* a = s.bodyPtrs[i];
            Mesh* b = s.bodyPtrs[j];
            if (a->isStatic && b->isStatic) continue;
            const double d = (a->transform.GetPosition() - b->transform.GetPosition()).norm();
            if (!(d < (double)(a->detectionRadius + b->detectionRadius))) continue;
            CollisionResult r = CollisionSpace::CollisionBoxBox(a, b);
            for (int k = 0; k < r.numContacts; ++k)
                maxPen = std::max(maxPen, (double)r.contactPoints[k].penetration);
        }
    for (Mesh* m : s.bodyPtrs) {
        if (m->isStatic) continue;
        const Eigen::Vector3f p = m->transform.GetPosition();
        if (!std::isfinite(p.x()) || !std::isfinite(p.y()) || !std::isfinite(p.z())) { bad += 1.0; continue; }
        kin += 0.5 * (double)m->mass * (double)m->velocity.squaredNorm();
        const Eigen::Matrix3f R = m->transform.GetRotation().toRotationMatrix();
        const Eigen::Vector3f Iw = R * (m->inertiaTensorBody * (R.transpose() * m->angularVelocity));
        kin += 0.5 * (double)m->angularVelocity.dot(Iw);
        pot += (double)m->mass * 9.81 * (double)p.y();
    }
    for (auto& ep : s.solverEnergies) {
        ep->ComputeEnergyTerms(nullptr, s.projectionMode, s.trustRegionRho);
        ela += (double)ep->GetCachedEnergy();
    }
    out[0] = maxC; out[1] = maxPen; out[2] = kin; out[3] = pot; out[4] = ela; out[5] = bad;
}

// 1 while user force `id` (a joint or spring) takes part in the step; 0 once
// a fracture disabled it (force.hpp:57-66) or the solver dropped it.
int orc_force_live(void* h, int id) {
    Orc* o = static_cast<Orc*>(h);
    if (id < 0 || id >= (int)o->forces.size()) return -1;
    const Force* f = o->forces[id];
    return f && !f->disabled ? 1 : 0;
}

// Poses by creation id: pos (n x 3), quat (n x 4, w x y z), vel/omega (n x 3);
// a removed body reads NaN.
void orc_get_state(void* h, float* pos, float* quat, float* vel, float* omega) {
    Orc* o = static_cast<Orc*>(h);
    const float nan = std::numeric_limits<float>::quiet_NaN();
    for (size_t i = 0; i < o->bodies.size(); ++i) {
        Mesh* m = o->bodies[i];
        if (!m) {
            if (pos) for (int k = 0; k < 3; ++k) pos[3 * i + k] = nan;
            if (quat) for (int k = 0; k < 4; ++k) quat[4 * i + k] = nan;
            if (vel) for (int k = 0; k < 3; ++k) vel[3 * i + k] = nan;
            if (omega) for (int k = 0; k < 3; ++k) omega[3 * i + k] = nan;
            continue;
        }
        Eigen::Vector3f p = m->transform.GetPosition();
        Quaternionf q = m->transform.GetRotation();
        if (pos) { pos[3 * i] = p.x(); pos[3 * i + 1] = p.y(); pos[3 * i + 2] = p.z(); }
        if (quat) { quat[4 * i] = q.w(); quat[4 * i + 1] = q.x(); quat[4 * i + 2] = q.y(); quat[4 * i + 3] = q.z(); }
        if (vel) for (int k = 0; k < 3; ++k) vel[3 * i + k] = m->velocity[k];
        if (omega) for (int k = 0; k < 3; ++k) omega[3 * i + k] = m->angularVelocity[k];
    }
}

// Overwrites the pose/velocity of every body (test setup for kernel-level checks).
void orc_set_state(void* h, const float* pos, const float* quat, const float* vel, const float* omega) {
    Orc* o = static_cast<Orc*>(h);
    for (size_t i = 0; i < o->bodies.size(); ++i) {
        Mesh* m = o->bodies[i];
        if (!m) continue;
        if (pos) m->transform.SetPosition(Eigen::Vector3f(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]));
        if (quat) m->transform.SetRotation(Quaternionf(quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3]));
        if (vel) m->velocity = Eigen::Vector3f(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        if (omega) m->angularVelocity = Eigen::Vector3f(omega[3 * i], omega[3 * i + 1], omega[3 * i + 2]);
    }
}

// Live contact manifolds after the last step, in forcePtrs order.
// pairs: (A, B) creation ids; counts; ids (8 per manifold); per contact
// floats: penetration, normal xyz, rA xyz, rB xyz, penalty x3, lambda x3 (16).
int orc_get_contacts(void* h, int max_manifolds, int* pairs, int* counts, uint32_t* ids, float* data) {
    Orc* o = static_cast<Orc*>(h);
    int n = 0;
    for (auto& fp : o->solver.solverForces) {
        Manifold* m = dynamic_cast<Manifold*>(fp.get());
        if (!m) continue;
        if (n < max_manifolds) {
            int ia = -1, ib = -1;
            for (size_t i = 0; i < o->bodies.size(); ++i) {
                if (!o->bodies[i]) continue;
                if (o->bodies[i] == m->bodyA) ia = (int)i;
                if (o->bodies[i] == m->bodyB) ib = (int)i;
            }
            if (pairs) { pairs[2 * n] = ia; pairs[2 * n + 1] = ib; }
            if (counts) counts[n] = m->numContactPoints;
            for (int k = 0; k < 8; ++k) {
                if (ids) ids[8 * n + k] = k < m->numContactPoints ? m->contactPoints[k].id : 0xFFFFFFFFu;
                if (data) {
                    float* d = data + (size_t)(8 * n + k) * 16;
                    std::memset(d, 0, 16 * sizeof(float));
                    if (k < m->numContactPoints) {
                        const ContactPoint& c = m->contactPoints[k];
                        d[0] = c.penetration;
                        for (int q = 0; q < 3; ++q) { d[1 + q] = c.normal[q]; d[4 + q] = c.rA[q]; d[7 + q] = c.rB[q]; }
                        for (int q = 0; q < 3; ++q) {
                            d[10 + q] = m->constraintPoints[3 * k + q].penalty;
                            d[13 + q] = m->constraintPoints[3 * k + q].lambda;
                        }
                    }
                }
            }
        }
        ++n;
    }
    return n;
}

// CollisionSpace::CollisionBoxBox on two bodies as they stand (collision.cpp:271-447).
int orc_collide(void* h, int a, int b, uint32_t* ids, float* data) {
    Orc* o = static_cast<Orc*>(h);
    Mesh* A = body_or_null(o, a);
    Mesh* B = body_or_null(o, b);
    if (!A || !B) return -1;
    CollisionResult r = CollisionSpace::CollisionBoxBox(A, B);
    for (int k = 0; k < r.numContacts; ++k) {
        const ContactPoint& c = r.contactPoints[k];
        if (ids) ids[k] = c.id;
        if (data) {
            float* d = data + 13 * k;
            d[0] = c.penetration;
            for (int q = 0; q < 3; ++q) {
                d[1 + q] = c.normal[q]; d[4 + q] = c.rA[q]; d[7 + q] = c.rB[q];
            }
            for (int q = 0; q < 3; ++q) d[10 + q] = c.position[q];
        }
    }
    return r.numContacts;
}

// Colours of the last orc_step_coloured(0) call, by creation id (-1 = static).
int orc_get_colours(void* h, int* colours) {
    Orc* o = static_cast<Orc*>(h);
    for (size_t i = 0; i < o->colour.size() && i < o->bodies.size(); ++i) colours[i] = o->colour[i];
    return o->num_colours;
}

// Per-phase wall times of the last orc_step_coloured() call (ms): broadphase,
// warm-start, colouring, prediction, primal+dual, velocity, post-stab, total.
void orc_get_phase_ms(void* h, double* out) {
    Orc* o = static_cast<Orc*>(h);
    for (int i = 0; i < 8; ++i) out[i] = o->phase_ms[i];
}

// The reference's own SolverTimings of its last Step() (solver.hpp:10-19).
void orc_get_solver_timings(void* h, float* out) {
    const SolverTimings& t = static_cast<Orc*>(h)->solver.timings;
    out[0] = t.broadPhaseMs; out[1] = t.warmstartMs; out[2] = t.predictionMs; out[3] = t.primalDualMs;
    out[4] = t.velocityUpdateMs; out[5] = t.postStabMs; out[6] = t.totalSubstepMs;
}

}  // extern "C"

// ---- Eigen-shim self-test entry points (checked against numpy in tests) ----
extern "C" {

// x = A^{-1} b through Eigen::LDLT<Matrix6f> (solver.cpp:437-438); A column-major.
void orc_shim_ldlt6(const float* A, const float* b, float* x) {
    Matrix6f M;
    Vector6f r;
    for (int j = 0; j < 6; ++j) { r[j] = b[j]; for (int i = 0; i < 6; ++i) M(i, j) = A[i + 6 * j]; }
    Eigen::LDLT<Matrix6f> l;
    l.compute(M);
    Vector6f s = l.solve(r);
    for (int i = 0; i < 6; ++i) x[i] = s[i];
}

// NeoHookeanMath::svd (math.cpp:13-35): F = U diag(S) V^T, column-major.
void orc_shim_svd3(const float* F, float* U, float* S, float* V) {
    Eigen::Matrix3f M;
    for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) M(i, j) = F[i + 3 * j];
    NeoHookeanMath::SVDDecomposition d = NeoHookeanMath::svd(M);
    for (int j = 0; j < 3; ++j) {
        S[j] = d.S[j];
        for (int i = 0; i < 3; ++i) { U[i + 3 * j] = d.U(i, j); V[i + 3 * j] = d.V(i, j); }
    }
}

// Eigen::SelfAdjointEigenSolver<Matrix3f> (math.cpp:121).
void orc_shim_eig3(const float* A, float* w, float* V) {
    Eigen::Matrix3f M;
    for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) M(i, j) = A[i + 3 * j];
    Eigen::SelfAdjointEigenSolver<Eigen::Matrix3f> es(M);
    for (int j = 0; j < 3; ++j) {
        w[j] = es.eigenvalues()[j];
        for (int i = 0; i < 3; ++i) V[i + 3 * j] = es.eigenvectors()(i, j);
    }
}

// STVKMath::svd (math.cpp:237-253) on a 3x2 F.
void orc_shim_svd32(const float* F, float* U, float* S, float* V) {
    STVKMath::F32 M;
    for (int j = 0; j < 2; ++j) for (int i = 0; i < 3; ++i) M(i, j) = F[i + 3 * j];
    STVKMath::SVDDecomposition d = STVKMath::svd(M);
    for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) U[i + 3 * j] = d.U(i, j);
    for (int j = 0; j < 2; ++j) { S[j] = d.S[j]; for (int i = 0; i < 2; ++i) V[i + 2 * j] = d.V(i, j); }
}

}  // extern "C"
