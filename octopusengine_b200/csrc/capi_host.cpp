// C ABI of the host-side building blocks (meshes, masses, shape tables, colourings).
#include <algorithm>

#include "../../include/octopus_b200.h"
#include "host.hpp"

using namespace octb;

extern "C" {

oct_status oct_beam_mesh(int element, int nx, int ny, int nz, const float size[3], const float offset[3], int32_t* n_nodes,
                         int32_t* n_elements, float* positions, int32_t* topology) {
    if (!size || !n_nodes || !n_elements) return OCT_EINVAL;
    const float o0 = offset ? offset[0] : 0.f, o1 = offset ? offset[1] : 0.f, o2 = offset ? offset[2] : 0.f;
    std::vector<float> X;
    std::vector<int32_t> T;
    if (!beam_mesh(element, nx, ny, nz, size[0], size[1], size[2], o0, o1, o2, X, T)) return OCT_EINVAL;
    const int ne = element_nodes(element);
    const int32_t nn = (int32_t)(X.size() / 3), nel = (int32_t)(T.size() / ne);
    if (positions || topology) {
        if (*n_nodes < nn || *n_elements < nel) return OCT_EINVAL;
        if (positions) std::copy(X.begin(), X.end(), positions);
        if (topology) std::copy(T.begin(), T.end(), topology);
    }
    *n_nodes = nn;
    *n_elements = nel;
    return OCT_OK;
}

oct_status oct_lumped_masses(int element, const float* positions, int n_nodes, const int32_t* topology, int n_elements,
                             float density, int distribution, float* out) {
    if (!positions || !topology || !out || n_nodes <= 0 || n_elements <= 0 || element_nodes(element) < 0) return OCT_EINVAL;
    std::vector<float> m;
    lumped_masses(element, positions, n_nodes, topology, n_elements, density, distribution, m);
    std::copy(m.begin(), m.end(), out);
    return OCT_OK;
}

oct_status oct_shape_table(int element, int32_t* nq, double* coords, double* weights, double* dN) {
    ShapeTable s;
    if (!shape_table(element, s)) return OCT_EINVAL;
    if (nq) *nq = s.nq;
    if (coords) std::copy(s.qp.begin(), s.qp.end(), coords);
    if (weights) std::copy(s.w.begin(), s.w.end(), weights);
    if (dN) std::copy(s.dN.begin(), s.dN.end(), dN);
    return OCT_OK;
}

oct_status oct_color(int element, const int32_t* topology, int n_elements, int n_nodes, int algo, int target,
                     int32_t* colors, int32_t* n_colors, int64_t* conflicts) {
    const int ne = element_nodes(element);
    if (ne < 0 || !topology || n_elements <= 0 || n_nodes <= 0 || !colors || !n_colors) return OCT_EINVAL;
    for (int64_t k = 0; k < (int64_t)n_elements * ne; ++k)
        if (topology[k] < 0 || topology[k] >= n_nodes) return OCT_EINVAL;
    PrimalGraph g;
    Coloring c;
    if (algo == 2) {
        build_dual_vertex_graph(ne, topology, n_elements, n_nodes, g);
        c = color_greedy_slf(g);
    } else {
        build_primal_graph(ne, topology, n_elements, n_nodes, g);
        c = algo == 1 ? color_greedy(g) : color_dsat(g);
        if (target > 0) color_reduction(g, c, target);
    }
    std::copy(c.colors.begin(), c.colors.end(), colors);
    *n_colors = c.n_colors;
    if (conflicts) *conflicts = count_conflicts(g, c);
    return OCT_OK;
}

}  // extern "C"
