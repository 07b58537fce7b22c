// Drives the reference-shaped C++ adapters (include/octopus_b200.hpp) the way
// Cuda_VBD_FEM_Dynamic + Cuda_ParticleSystem_Dynamics do, on config 1 (8x2x2 P1 beam,
// Stable Neo-Hookean E=1e5 nu=0.45, 20 iterations), and prints the final positions.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "octopus_b200.hpp"

int main(int argc, char** argv) {
    using namespace octb;
    const int frames = argc > 1 ? std::atoi(argv[1]) : 5;
    int32_t nn = 0, ne = 0;
    const float size[3] = {1.0f, 0.25f, 0.25f};
    check(oct_beam_mesh(OCT_TETRA, 8, 2, 2, size, nullptr, &nn, &ne, nullptr, nullptr), "beam sizes");
    std::vector<float> X(3 * nn);
    std::vector<int> T(4 * ne);
    check(oct_beam_mesh(OCT_TETRA, 8, 2, 2, size, nullptr, &nn, &ne, X.data(), T.data()), "beam");
    Mesh::Geometry geometry(nn);
    for (int i = 0; i < nn; ++i) geometry[i] = Vector3(X[3 * i], X[3 * i + 1], X[3 * i + 2]);

    std::vector<scalar> masses = compute_fem_mass(Tetra, geometry, T, 1000.f, FemShape);
    auto* ps = new GPU_ParticleSystem(geometry, masses);
    auto* integrator = new GPU_VBD(ps, 20, 0.f);
    integrator->gravity[0] = 0.f; integrator->gravity[1] = 0.f; integrator->gravity[2] = -9.81f;
    auto* fem = new GPU_VBD_FEM(Tetra, T, geometry, Stable_NeoHooke, 1e5f, 0.45f, 0.f, Reduction_Symmetry, -1);
    integrator->add_dynamics(fem);
    integrator->add_constraint(new GPU_Fix_Constraint(geometry, new Plane(Vector3(0.01f, 0, 0), Vector3(-1, 0, 0))));
    const int sub_it = 1;
    for (int f = 0; f < frames; ++f)
        for (int i = 0; i < sub_it; ++i) integrator->step(ps, 0.01f / sub_it);
    ps->get_position(geometry);
    for (const Vector3& p : geometry) std::printf("%.9g %.9g %.9g\n", p.x, p.y, p.z);
    // GPU_FEM queries: total volume, inverted elements, largest residual force
    double volume = 0, inverted = 0, rmax = 0;
    for (scalar v : fem->get_volume(ps)) volume += v;
    for (scalar v : fem->get_inverted(ps)) inverted += v;
    for (const Vector3& r : fem->get_forces(ps, 0.01f)) rmax = std::max(rmax, (double)std::fabs(r.z));
    std::fprintf(stderr, "volume %.9g inverted %g rmax %.9g\n", volume, inverted, rmax);
    delete integrator;
    delete ps;
    return 0;
}
