// Host-side building blocks of the scene set-up: element tables, shape functions and
// quadrature, beam meshes, lumped masses, graph colourings.  All of it runs once per scene
// on the host; the per-step work is on the GPU.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace octb {

enum Element { kTetra = 3, kPyramid = 4, kPrism = 5, kHexa = 6, kTetra10 = 7, kTetra20 = 8, kHexa27 = 9 };
enum Material { kHooke = 0, kStVK = 1, kNeoHooke = 2, kStableNeoHooke = 3 };

int element_nodes(int element);        // -1 if unsupported
int element_quadrature(int element);   // -1 if unsupported

// Shape-function derivatives at the quadrature points and the quadrature weights of the
// reference element (the reference's FEM_Shape tables, octopus/include/Dynamic/FEM/FEM_Shape.h).
struct ShapeTable {
    int ne = 0, nq = 0;
    std::vector<double> qp;   // nq * 3
    std::vector<double> w;    // nq
    std::vector<double> dN;   // (q * ne + i) * 3 + k
};
bool shape_table(int element, ShapeTable& out);
// Shape-function values at reference coordinates x[3] (N: nodes of the element) and the
// reference-element node coordinates (X: 3 per node).
bool shape_values(int element, const double* x, double* N);
bool reference_nodes(int element, double* X);

// Beam meshes as BeamMeshGenerator builds them (octopus/src/Mesh/Generator/BeamGenerator.cpp):
// hex grid of nx*ny*nz cells over size sx*sy*sz at an offset; tetra elements use the 6-tet
// cell split; P2/P3/Q2 promote the linear mesh.  FP32 geometry, as the reference.
bool beam_mesh(int element, int nx, int ny, int nz, float sx, float sy, float sz, float ox, float oy, float oz,
               std::vector<float>& X, std::vector<int32_t>& topo);

// compute_fem_mass (octopus/src/Dynamic/FEM/FEM_Shape.cpp:86-121).
// Boundary nodes of a mesh, ascending (MeshTools::Get_Surface_Geometry_Ids).
std::vector<int32_t> surface_nodes(int element, const int32_t* topo, int n_elements);
void lumped_masses(int element, const float* X, int n_nodes, const int32_t* topo, int n_elements, float density,
                   int distribution, std::vector<float>& mass);

// Graph colourings with the reference's tie-breaking (octopus/include/Tools/Graph.h).
struct Coloring {
    int n_colors = 0;
    std::vector<int32_t> colors;
};
// Primal vertex graph as CSR with edge multiplicities (the reference keeps a multiset).
struct PrimalGraph {
    int n = 0;
    std::vector<int64_t> off;      // n + 1
    std::vector<int32_t> nbr;      // unique neighbours, ascending
    std::vector<int32_t> mult;     // multiplicity of each neighbour entry
    std::vector<int64_t> degree;   // multiset size
};
void build_primal_graph(int ne, const int32_t* topo, int n_elements, int n_nodes, PrimalGraph& g);
void build_dual_vertex_graph(int ne, const int32_t* topo, int n_elements, int n_nodes, PrimalGraph& g);
Coloring color_dsat(const PrimalGraph& g);
Coloring color_greedy(const PrimalGraph& g);
Coloring color_greedy_slf(const PrimalGraph& g);
void color_reduction(const PrimalGraph& g, Coloring& c, int target);
int64_t count_conflicts(const PrimalGraph& g, const Coloring& c);

}  // namespace octb
