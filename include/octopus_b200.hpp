// octopus_b200.hpp — header-only C++ adapters with the reference's GPU solver class shapes,
// implemented on the C ABI of octopus_b200.h.  A caller written against OctopusEngine's
//
//     GPU_ParticleSystem* ps = new GPU_ParticleSystem(positions, masses);
//     GPU_Integrator* integ  = new GPU_VBD(ps, iterations, rho);
//     integ->add_dynamics(new GPU_VBD_FEM(elem, topo, geometry, material, E, nu, damping, version, target));
//     integ->add_constraint(new GPU_Fix_Constraint(geometry, new Plane(o, n)));
//     for (int i = 0; i < sub_it; ++i) integ->step(ps, dt / sub_it);
//     ps->get_position(geometry);
//
// (octopus/src/Script/Dynamic/Cuda_ParticleSystem_Dynamic.cpp:17-31,
//  octopus/src/Script/Dynamic/Cuda_VBD_FEM_Dynamic.cpp:13-28) compiles unchanged against
// namespace octb.  The objects collect their arguments; the first step() creates one
// oct_scene that holds the particle system, the solver, the FEM object and the fixation.
// Differences from the reference, all deliberate: errors throw octb::Error instead of
// being ignored; the colour order is ascending (reproducible) instead of clock-shuffled;
// no VTK side file is written on construction.
#pragma once
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "octopus_b200.h"

namespace octb {

using scalar = float;
struct Vector3 {
    float x = 0, y = 0, z = 0;
    Vector3() = default;
    Vector3(float a, float b, float c) : x(a), y(b), z(c) {}
};
namespace Mesh {
using Geometry = std::vector<Vector3>;
using Topology = std::vector<int>;
}  // namespace Mesh
enum Element { Line, Triangle, Quad, Tetra, Pyramid, Prism, Hexa, Tetra10, Tetra20, Hexa27 };
enum Material { Hooke, StVK, NeoHooke, Stable_NeoHooke, Corotated, FixedCorotated };
enum Mass_Distribution { Uniform, FemShape };
enum VBD_Version { Base, Threaded_Quadrature, Reduction_Symmetry, Better_Coloration };
enum XPBD_FEM_VERSION { XPBD, Quadrature, OptiShared, OptiGroup };

struct Error : std::runtime_error {
    oct_status status;
    Error(oct_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};
inline void check(oct_status s, const char* where, oct_ctx* ctx = nullptr) {
    if (s != OCT_OK) throw Error(s, std::string(where) + ": " + (ctx ? oct_last_error(ctx) : "status " + std::to_string((int)s)));
}

// One context per thread (device 0, default budget) shared by the adapters.
inline oct_ctx* default_context() {
    thread_local struct Holder {
        oct_ctx* c = nullptr;
        ~Holder() { if (c) oct_ctx_destroy(c); }
    } h;
    if (!h.c) check(oct_ctx_create(0, 0, &h.c), "oct_ctx_create");
    return h.c;
}

// Tools/Area.h Plane: dot(p - o, n) > 0.
struct Area { virtual ~Area() = default; };
struct Plane : Area {
    Plane(const Vector3& o_, const Vector3& n_) : o(o_), n(n_) {}
    Vector3 o, n;
};

struct GPU_ParticleSystem;

struct GPU_Dynamic {
    virtual ~GPU_Dynamic() = default;
    virtual void start(GPU_ParticleSystem*, scalar) {}
    virtual void step(GPU_ParticleSystem*, scalar) {}
    bool active = true;
};

// GPU_ParticleSystem (octopus/include/GPU/GPU_ParticleSystem.h:54-73)
struct GPU_ParticleSystem {
    GPU_ParticleSystem(const std::vector<Vector3>& positions, const std::vector<scalar>& masses)
        : init_positions(positions), masses(masses) {}
    int nb_particles() const { return (int)init_positions.size(); }
    void get_position(std::vector<Vector3>& out) const { read(out, true); }
    void get_velocity(std::vector<Vector3>& out) const { read(out, false); }
    std::vector<Vector3> init_positions;
    std::vector<scalar> masses;
    oct_scene* scene = nullptr;   // set when the integrator first steps

  private:
    void read(std::vector<Vector3>& out, bool pos) const {
        out.resize(init_positions.size());
        if (!scene) {
            for (size_t i = 0; i < out.size(); ++i) out[i] = pos ? init_positions[i] : Vector3();
            return;
        }
        std::vector<float> buf(out.size() * 3);
        check(pos ? oct_scene_get_positions(scene, buf.data()) : oct_scene_get_velocities(scene, buf.data()),
              "get_position/get_velocity");
        for (size_t i = 0; i < out.size(); ++i) out[i] = Vector3(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]);
    }
};

// FEM objects: GPU_VBD_FEM / GPU_PBD_FEM / GPU_FEM_Explicit collect the mesh and material.
struct GPU_FEM : GPU_Dynamic {
    GPU_FEM(Element e, const Mesh::Geometry& g, const Mesh::Topology& t, scalar young_, scalar poisson_, Material m)
        : element(e), geometry(g), topology(t), young(young_), poisson(poisson_), material(m) {}
    Element element;
    Mesh::Geometry geometry;
    Mesh::Topology topology;
    scalar young, poisson;
    Material material;
    scalar damping = 0;

    // Queries of GPU_FEM (octopus/include/GPU/GPU_FEM.h:66-70), available once the integrator
    // has stepped the particle system (the scene is created at the first step).
    std::vector<scalar> get_stress(const GPU_ParticleSystem* ps) const { return element_data(ps, OCT_DIAG_STRESS_ACCUMULATED); }
    std::vector<scalar> get_volume(const GPU_ParticleSystem* ps) const { return element_data(ps, OCT_DIAG_VOLUME); }
    std::vector<scalar> get_inverted(const GPU_ParticleSystem* ps) const { return element_data(ps, OCT_DIAG_INVERTED); }
    // the reference getter launches the inversion kernel (octopus/src/GPU/GPU_FEM.cu:237-245)
    std::vector<scalar> get_volume_diff(const GPU_ParticleSystem* ps) const { return element_data(ps, OCT_DIAG_INVERTED); }
    virtual std::vector<Vector3> get_forces(const GPU_ParticleSystem* ps, scalar dt) const {
        std::vector<Vector3> out(ps->nb_particles());
        if (!ps->scene) return out;
        std::vector<float> buf(out.size() * 3);
        check(oct_scene_vertex_residuals(ps->scene, dt, buf.data()), "get_forces");
        for (size_t i = 0; i < out.size(); ++i) out[i] = Vector3(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]);
        return out;
    }

  private:
    std::vector<scalar> element_data(const GPU_ParticleSystem* ps, int kind) const {
        if (!ps->scene) throw Error(OCT_EINVAL, "GPU_FEM query before the integrator's first step");
        int32_t nn = 0, ne = 0, nc = 0, nf = 0;
        check(oct_scene_info(ps->scene, &nn, &ne, &nc, &nf), "oct_scene_info");
        std::vector<scalar> out(ne);
        check(oct_scene_element_data(ps->scene, kind, out.data()), "GPU_FEM query");
        return out;
    }
};
struct GPU_VBD_FEM : GPU_FEM {
    GPU_VBD_FEM(const Element& e, const Mesh::Topology& t, const Mesh::Geometry& g, const Material& m, const scalar& young_,
                const scalar& poisson_, const scalar& damping_, const VBD_Version& v = Reduction_Symmetry,
                const int& target = -1)
        : GPU_FEM(e, g, t, young_, poisson_, m), version(v), target_color(target) { damping = damping_; }
    VBD_Version version;
    int target_color;
};
struct GPU_PBD_FEM : GPU_FEM {
    GPU_PBD_FEM(Element e, const Mesh::Geometry& g, const Mesh::Topology& t, scalar young_, scalar poisson_, Material m,
                XPBD_FEM_VERSION v = OptiShared)
        : GPU_FEM(e, g, t, young_, poisson_, m), version(v) {}
    XPBD_FEM_VERSION version;
};
struct GPU_FEM_Explicit : GPU_FEM {
    GPU_FEM_Explicit(Element e, const Mesh::Geometry& g, const Mesh::Topology& t, scalar young_, scalar poisson_, Material m,
                     scalar damping_)
        : GPU_FEM(e, g, t, young_, poisson_, m) { damping = damping_; }
};

// Axis (octopus/include/Tools/Axis.h): a position and a rotation (column-major 3x3).
struct Axis {
    Vector3 pos{0.f, 0.f, 0.f};
    float rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    void move(const Vector3& m) { pos = Vector3(pos.x + m.x, pos.y + m.y, pos.z + m.z); }
    void setPosition(const Vector3& p) { pos = p; }
    void setRotation(const float r[9]) { for (int k = 0; k < 9; ++k) rot[k] = r[k]; }
    const Vector3& position() const { return pos; }
    const float* rotation() const { return rot; }
};

// GPU_Fix_Constraint(positions, Area*) (octopus/src/GPU/GPU_Constraint.cu:94-107): the nodes
// inside the area follow com + axis.position + axis.rotation (X - com).  Each constraint of an
// integrator is one rigid group of the scene (at most four); moving its axis between steps
// moves the group.
struct GPU_Fix_Constraint : GPU_Dynamic {
    GPU_Fix_Constraint(const Mesh::Geometry& positions, Area* area) {
        if (auto* p = dynamic_cast<Plane*>(area)) {
            for (size_t i = 0; i < positions.size(); ++i) {
                const Vector3& q = positions[i];
                const float d = (q.x - p->o.x) * p->n.x + (q.y - p->o.y) * p->n.y + (q.z - p->o.z) * p->n.z;
                if (d > 0) ids.push_back((int)i);
            }
        }
        delete area;
    }
    std::vector<int> ids;
    Axis axis;
    float sent[12] = {0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1};   // axis last sent to the scene (the identity at set-up)
};

// GPU_Box_Limit(pmin, pmax) (octopus/include/GPU/GPU_Constraint.h:20-25): free nodes clamped
// to the box (one box per integrator).
struct GPU_Box_Limit : GPU_Dynamic {
    GPU_Box_Limit(const Vector3& pmin_, const Vector3& pmax_) : pmin(pmin_), pmax(pmax_) {}
    Vector3 pmin, pmax;
};

// Scripted effects (octopus/include/GPU/GPU_Constraint.h:28-80); `active` is read at every step.
struct GPU_Effect : GPU_Dynamic {
    int kind = OCT_EFFECT_CRUSH;
    float params[2] = {0.f, 0.f};
    int index = -1;         // slot in the scene, set at the first step
    bool applied = false;   // last active state sent to the scene
};
struct GPU_Crush : GPU_Effect {
    GPU_Crush() { kind = OCT_EFFECT_CRUSH; }
};
struct GPU_RandomSphere : GPU_Effect {
    GPU_RandomSphere(const Mesh::Geometry&, scalar radius) { kind = OCT_EFFECT_RANDOM_SPHERE; params[0] = radius; }
};
struct GPU_HighStretch : GPU_Effect {
    GPU_HighStretch(int nb_constraint, scalar max_dist) {
        kind = OCT_EFFECT_HIGH_STRETCH;
        params[0] = (float)nb_constraint;
        params[1] = max_dist;
    }
};

// GPU_Integrator and the three solvers (octopus/include/GPU/GPU_Integrator.h:11-36).
struct GPU_Integrator : GPU_Dynamic {
    virtual void add_dynamics(GPU_Dynamic* d) { dynamics.push_back(d); }
    virtual void add_constraint(GPU_Dynamic* c) { constraints.push_back(c); }
    void step(GPU_ParticleSystem* ps, scalar dt) override {
        if (!ps->scene) commit(ps);
        // constraint state read at every step: fixation axes and effect activity
        int g = 0;
        for (auto* c : constraints) {
            if (auto* f = dynamic_cast<GPU_Fix_Constraint*>(c)) {
                const float off[3] = {f->axis.pos.x, f->axis.pos.y, f->axis.pos.z};
                if (std::memcmp(off, f->sent, sizeof(off)) != 0 || std::memcmp(f->axis.rot, f->sent + 3, sizeof(f->axis.rot)) != 0) {
                    check(oct_scene_set_fixation_group(ps->scene, g, off, f->axis.rot), "fixation axis");
                    std::memcpy(f->sent, off, sizeof(off));
                    std::memcpy(f->sent + 3, f->axis.rot, sizeof(f->axis.rot));
                }
                ++g;
            } else if (auto* e = dynamic_cast<GPU_Effect*>(c)) {
                if (e->active != e->applied) {
                    check(oct_scene_set_effect_active(ps->scene, e->index, e->active ? 1 : 0), "effect");
                    e->applied = e->active;
                }
            }
        }
        check(oct_scene_step(ps->scene, dt, 1), "GPU_Integrator::step", default_context());
    }
    ~GPU_Integrator() override {
        for (auto* d : dynamics) delete d;
        for (auto* c : constraints) delete c;
        if (owned) oct_scene_destroy(owned);
    }
    std::vector<GPU_Dynamic*> dynamics, constraints;
    scalar gravity[3] = {0.f, -9.81f, 0.f};   // Dynamic::gravity() default of the reference scenes

  protected:
    virtual void fill(oct_scene_desc& d) = 0;
    void commit(GPU_ParticleSystem* ps) {
        GPU_FEM* fem = nullptr;
        for (auto* d : dynamics) if ((fem = dynamic_cast<GPU_FEM*>(d))) break;   // first FEM object
        if (!fem) throw Error(OCT_EINVAL, "integrator has no FEM dynamics");
        oct_scene_desc d;
        oct_desc_init(&d);
        std::vector<float> X(ps->init_positions.size() * 3);
        for (size_t i = 0; i < ps->init_positions.size(); ++i) {
            X[3 * i] = ps->init_positions[i].x; X[3 * i + 1] = ps->init_positions[i].y; X[3 * i + 2] = ps->init_positions[i].z;
        }
        std::vector<int> fixed, group;
        int n_groups = 0;
        for (auto* c : constraints)
            if (auto* f = dynamic_cast<GPU_Fix_Constraint*>(c)) {
                if (n_groups == 4) throw Error(OCT_ENOTSUP, "at most four GPU_Fix_Constraint per integrator");
                fixed.insert(fixed.end(), f->ids.begin(), f->ids.end());
                group.insert(group.end(), f->ids.size(), n_groups++);
            }
        const int ne = fem->element == Tetra ? 4 : fem->element == Hexa ? 8 : fem->element == Tetra10 ? 10 :
                       fem->element == Tetra20 ? 20 : 27;
        d.element = fem->element;
        d.n_nodes = ps->nb_particles();
        d.positions = X.data();
        d.n_elements = (int)fem->topology.size() / ne;
        d.topology = fem->topology.data();
        d.masses = ps->masses.data();
        d.material = fem->material;
        d.young = fem->young;
        d.poisson = fem->poisson;
        d.damping = fem->damping;
        for (int k = 0; k < 3; ++k) d.gravity[k] = gravity[k];
        d.n_fixed = (int)fixed.size();
        d.fixed_ids = fixed.empty() ? nullptr : fixed.data();
        d.fixed_group = fixed.empty() ? nullptr : group.data();
        for (auto* c : constraints)
            if (auto* b = dynamic_cast<GPU_Box_Limit*>(c)) {
                d.box_limit = 1;
                d.box_min[0] = b->pmin.x; d.box_min[1] = b->pmin.y; d.box_min[2] = b->pmin.z;
                d.box_max[0] = b->pmax.x; d.box_max[1] = b->pmax.y; d.box_max[2] = b->pmax.z;
            }
        fill(d);
        if (auto* v = dynamic_cast<GPU_VBD_FEM*>(fem)) { d.vbd_version = v->version; d.target_color = v->target_color; }
        if (auto* x = dynamic_cast<GPU_PBD_FEM*>(fem)) d.xpbd_version = x->version;
        oct_ctx* ctx = default_context();
        check(oct_scene_create(ctx, &d, &owned), "oct_scene_create", ctx);
        ps->scene = owned;
        for (auto* c : constraints)
            if (auto* e = dynamic_cast<GPU_Effect*>(c)) check(oct_scene_add_effect(owned, e->kind, e->params, &e->index), "effect", ctx);
    }
    oct_scene* owned = nullptr;
};

struct GPU_VBD : GPU_Integrator {
    GPU_VBD(GPU_ParticleSystem*, const int it, const scalar rho) : iteration(it), _rho(rho) {}
    int iteration;
    scalar _rho;

  protected:
    void fill(oct_scene_desc& d) override { d.solver = OCT_SOLVER_VBD; d.iterations = iteration; d.rho = _rho; }
};
struct GPU_PBD : GPU_Integrator {
    explicit GPU_PBD(const scalar global_damping = 0.f) : _global_damping(global_damping) {}
    scalar _global_damping;

  protected:
    void fill(oct_scene_desc& d) override { d.solver = OCT_SOLVER_XPBD; d.global_damping = _global_damping; }
};
struct GPU_SemiExplicit : GPU_Integrator {
  protected:
    void fill(oct_scene_desc& d) override { d.solver = OCT_SOLVER_EXPLICIT; }
};

// compute_fem_mass (octopus/src/Dynamic/FEM/FEM_Shape.cpp:86-121).
inline std::vector<scalar> compute_fem_mass(const Element& e, const Mesh::Geometry& g, const Mesh::Topology& t,
                                            scalar density, Mass_Distribution distrib = Uniform) {
    std::vector<float> X(g.size() * 3), m(g.size());
    for (size_t i = 0; i < g.size(); ++i) { X[3 * i] = g[i].x; X[3 * i + 1] = g[i].y; X[3 * i + 2] = g[i].z; }
    const int ne = e == Tetra ? 4 : e == Hexa ? 8 : e == Tetra10 ? 10 : e == Tetra20 ? 20 : 27;
    check(oct_lumped_masses(e, X.data(), (int)g.size(), t.data(), (int)t.size() / ne, density, distrib, m.data()),
          "compute_fem_mass");
    return m;
}

}  // namespace octb
