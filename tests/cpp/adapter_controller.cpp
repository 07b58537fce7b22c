// Drives the reference-shaped adapters the way Cuda_Constraint_Rigid_Controller does
// (octopus/src/Script/Dynamic/Cuda_Constraint_Rigid_Controller.cpp): a P1 beam held by two
// GPU_Fix_Constraint (x = 0 face and x = 1 face), the second one's axis moved down every frame,
// a GPU_HighStretch switched on for frames 3 and 4, and a GPU_Box_Limit; prints the final
// positions.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "octopus_b200.hpp"

int main(int argc, char** argv) {
    using namespace octb;
    const int frames = argc > 1 ? std::atoi(argv[1]) : 6;
    int32_t nn = 0, ne = 0;
    const float size[3] = {1.0f, 0.25f, 0.25f};
    check(oct_beam_mesh(OCT_TETRA, 8, 2, 2, size, nullptr, &nn, &ne, nullptr, nullptr), "beam sizes");
    std::vector<float> X(3 * nn);
    std::vector<int> T(4 * ne);
    check(oct_beam_mesh(OCT_TETRA, 8, 2, 2, size, nullptr, &nn, &ne, X.data(), T.data()), "beam");
    Mesh::Geometry geometry(nn);
    for (int i = 0; i < nn; ++i) geometry[i] = Vector3(X[3 * i], X[3 * i + 1], X[3 * i + 2]);

    auto* ps = new GPU_ParticleSystem(geometry, compute_fem_mass(Tetra, geometry, T, 1000.f, FemShape));
    auto* integrator = new GPU_VBD(ps, 10, 0.f);
    integrator->gravity[0] = 0.f; integrator->gravity[1] = 0.f; integrator->gravity[2] = -9.81f;
    integrator->add_dynamics(new GPU_VBD_FEM(Tetra, T, geometry, Stable_NeoHooke, 1e5f, 0.45f, 0.f, Reduction_Symmetry, -1));
    auto* left = new GPU_Fix_Constraint(geometry, new Plane(Vector3(0.01f, 0, 0), Vector3(-1, 0, 0)));
    auto* right = new GPU_Fix_Constraint(geometry, new Plane(Vector3(0.99f, 0, 0), Vector3(1, 0, 0)));
    auto* stretch = new GPU_HighStretch(6, 0.03f);
    stretch->active = false;
    integrator->add_constraint(left);
    integrator->add_constraint(right);
    integrator->add_constraint(stretch);
    integrator->add_constraint(new GPU_Box_Limit(Vector3(-10, -5, -10), Vector3(10, 5, 10)));
    for (int f = 0; f < frames; ++f) {
        right->axis.move(Vector3(0.f, 0.f, -0.01f));
        stretch->active = f == 3 || f == 4;
        integrator->step(ps, 1.f / 60.f);
    }
    ps->get_position(geometry);
    for (const Vector3& p : geometry) std::printf("%.9g %.9g %.9g\n", p.x, p.y, p.z);
    delete integrator;
    delete ps;
    return 0;
}
