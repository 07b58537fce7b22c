// VTK 5.1 ASCII unstructured-grid files: the writer of VTK_Formater
// (octopus/src/Mesh/Converter/VTK_Formater.cpp), the reader of VTK_Loader
// (octopus/src/Mesh/Converter/MeshLoader.cpp:97-330) and the per-frame FEM record of
// FEM_VTK_Recorder::save (octopus/src/Script/Record/Recorder.cpp:117-171), on one element type.
//
// The text layout follows the reference's byte for byte (default stream formatting of the
// values, one OFFSETS line per element type, one element per CONNECTIVITY line, trailing
// spaces), so files written here and by the reference are interchangeable.  Hexa27 nodes are
// written in VTK's order (VTK_QUADRATIC_HEXAHEDRON), which swaps the reference's edge and
// face-centre nodes 12-15 <-> 16-19, 20 <-> 24 and 21 <-> 22; the reader swaps them back.
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/octopus_b200.h"

namespace {

int nodes_of(int e) {
    switch (e) { case 3: return 4; case 6: return 8; case 7: return 10; case 8: return 20; case 9: return 27; default: return -1; }
}
// VTK cell type ids (VTK_Formater::get_cell_type)
int vtk_cell_type(int e) {
    switch (e) { case 3: return 10; case 6: return 12; case 7: return 24; case 8: return 71; case 9: return 29; default: return 0; }
}
int element_of_vtk(int t) {
    switch (t) { case 10: return 3; case 12: return 6; case 24: return 7; case 71: return 8; case 29: return 9; default: return -1; }
}
// Position in the element of the node written at VTK slot j (an involution).
int hexa27_vtk_swap(int j) {
    switch (j) {
        case 12: return 16; case 16: return 12; case 13: return 17; case 17: return 13;
        case 14: return 18; case 18: return 14; case 15: return 19; case 19: return 15;
        case 20: return 24; case 24: return 20; case 21: return 22; case 22: return 21;
        default: return j;
    }
}

void write_field(std::ofstream& f, const oct_vtk_field& fd, int n) {
    if (fd.components == 1) {
        f << "SCALARS " << fd.name << " float 1\n";
        f << "LOOKUP_TABLE default\n";
        for (int i = 0; i < n; ++i) f << fd.data[i] << " ";
        f << "\n";
    } else {
        f << "VECTORS " << fd.name << " float\n";
        for (int i = 0; i < n; ++i) f << fd.data[3 * i] << " " << fd.data[3 * i + 1] << " " << fd.data[3 * i + 2] << "  ";
        f << "\n";
    }
}

// Whitespace-separated tokens of the file with line starts marked, for keyword searches.
struct Tokens {
    std::vector<std::string> tok;
    std::vector<char> line_start;
    bool load(const char* path) {
        std::ifstream f(path);
        if (!f.good()) return false;
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream ss(line);
            std::string t;
            bool first = true;
            while (ss >> t) { tok.push_back(t); line_start.push_back(first); first = false; }
        }
        return true;
    }
    // index of the first token equal to key that starts a line, from position from
    long find(const std::string& key, long from = 0) const {
        for (long i = from; i < (long)tok.size(); ++i)
            if (line_start[i] && tok[i] == key) return i;
        return -1;
    }
};

}  // namespace

extern "C" {

oct_status oct_vtk_write(const char* path, const float* positions, int32_t n_nodes, int32_t element,
                         const int32_t* topology, int32_t n_elements, const oct_vtk_field* fields, int32_t n_fields) {
    const int ne = nodes_of(element);
    if (!path || !positions || n_nodes <= 0 || ne < 0 || n_elements < 0 || (n_elements > 0 && !topology) ||
        n_fields < 0 || (n_fields > 0 && !fields))
        return OCT_EINVAL;
    for (int k = 0; k < n_fields; ++k) {
        const oct_vtk_field& fd = fields[k];
        if (!fd.name || !fd.data || (fd.components != 1 && fd.components != 3) ||
            (fd.location != OCT_VTK_POINT && fd.location != OCT_VTK_CELL))
            return OCT_EINVAL;
    }
    std::ofstream f(path);
    if (!f.good()) return OCT_EINVAL;
    f << "# vtk DataFile Version 5.1\n";
    f << "vtk output\n";
    f << "ASCII\n\n";
    f << "DATASET UNSTRUCTURED_GRID\n";
    f << "POINTS " << n_nodes << " float\n";
    for (int i = 0; i < n_nodes; ++i) f << positions[3 * i] << " " << positions[3 * i + 1] << " " << positions[3 * i + 2] << "\n";
    f << "\n";
    f << "CELLS " << n_elements + 1 << " " << (long long)n_elements * ne << "\n";
    f << "OFFSETS vtktypeint64\n";
    if (n_elements > 0) {
        long long off = 0;
        for (int e = 0; e <= n_elements; ++e) { f << off << " "; off += ne; }
        f << "\n";
    }
    f << "CONNECTIVITY vtktypeint64\n";
    for (int e = 0; e < n_elements; ++e) {
        const int32_t* t = topology + (size_t)e * ne;
        for (int j = 0; j < ne; ++j) f << t[element == OCT_HEXA27 ? hexa27_vtk_swap(j) : j] << " ";
        f << "\n";
    }
    f << "CELL_TYPES " << n_elements << "\n";
    if (n_elements > 0) {
        const int ct = vtk_cell_type(element);
        for (int e = 0; e < n_elements; ++e) f << ct << " ";
        f << "\n";
    }
    f << "\n";
    bool point_open = false, cell_open = false;
    for (int k = 0; k < n_fields; ++k)
        if (fields[k].location == OCT_VTK_POINT) {
            if (!point_open) { f << "POINT_DATA " << n_nodes << "\n"; point_open = true; }
            write_field(f, fields[k], n_nodes);
        }
    for (int k = 0; k < n_fields; ++k)
        if (fields[k].location == OCT_VTK_CELL) {
            if (!cell_open) { f << "CELL_DATA " << n_elements << "\n"; cell_open = true; }
            write_field(f, fields[k], n_elements);
        }
    f.close();
    return f.good() ? OCT_OK : OCT_EINVAL;
}

oct_status oct_vtk_read_mesh(const char* path, int32_t* element, int32_t* n_nodes, int32_t* n_elements, float* positions,
                             int32_t* topology) {
    if (!path || !element || !n_nodes || !n_elements) return OCT_EINVAL;
    Tokens T;
    if (!T.load(path)) return OCT_EINVAL;
    if (T.find("ASCII") < 0) return OCT_ENOTSUP;   // binary files are not read (as VTK_Loader)
    const long ds = T.find("DATASET");
    if (ds < 0 || ds + 1 >= (long)T.tok.size() || T.tok[ds + 1] != "UNSTRUCTURED_GRID") return OCT_ENOTSUP;
    const long pp = T.find("POINTS", ds);
    const long cc = T.find("CELLS", ds);
    const long cn = T.find("CONNECTIVITY", ds);
    const long ct = T.find("CELL_TYPES", ds);
    if (pp < 0 || cc < 0 || cn < 0 || ct < 0) return OCT_EINVAL;
    const int np = std::atoi(T.tok[pp + 1].c_str());
    const long n_ids = std::atol(T.tok[cc + 2].c_str());
    const int nc = std::atoi(T.tok[ct + 1].c_str());
    if (np <= 0 || nc < 0 || pp + 3 + 3L * np > (long)T.tok.size() || cn + 2 + n_ids > (long)T.tok.size() ||
        ct + 2 + nc > (long)T.tok.size())
        return OCT_EINVAL;
    int elem = -1;
    for (int k = 0; k < nc; ++k) {
        const int e = element_of_vtk(std::atoi(T.tok[ct + 2 + k].c_str()));
        if (e < 0) return OCT_ENOTSUP;
        if (elem >= 0 && e != elem) return OCT_ENOTSUP;   // one element type per scene
        elem = e;
    }
    const int ne = elem < 0 ? 0 : nodes_of(elem);
    if ((long)nc * ne != n_ids) return OCT_EINVAL;
    *element = elem < 0 ? 0 : elem;
    *n_nodes = np;
    *n_elements = nc;
    if (positions)
        for (long i = 0; i < 3L * np; ++i) positions[i] = std::strtof(T.tok[pp + 3 + i].c_str(), nullptr);
    if (topology)
        for (int e = 0; e < nc; ++e)
            for (int j = 0; j < ne; ++j) {
                const int src = elem == OCT_HEXA27 ? hexa27_vtk_swap(j) : j;
                const int v = std::atoi(T.tok[cn + 2 + (long)e * ne + src].c_str());
                if (v < 0 || v >= np) return OCT_EINVAL;
                topology[(size_t)e * ne + j] = v;
            }
    return OCT_OK;
}

oct_status oct_vtk_read_field(const char* path, const char* name, int32_t components, int32_t n, float* out) {
    if (!path || !name || !out || n < 0 || (components != 1 && components != 3)) return OCT_EINVAL;
    Tokens T;
    if (!T.load(path)) return OCT_EINVAL;
    const std::string key = components == 1 ? "SCALARS" : "VECTORS";
    for (long i = T.find(key); i >= 0; i = T.find(key, i + 1)) {
        if (i + 1 >= (long)T.tok.size() || T.tok[i + 1] != name) continue;
        long v = i + (components == 1 ? 4 : 3);   // SCALARS name float 1 / VECTORS name float
        if (components == 1) {
            if (v + 1 < (long)T.tok.size() && T.tok[v] == "LOOKUP_TABLE") v += 2;
        }
        if (v + (long)n * components > (long)T.tok.size()) return OCT_EINVAL;
        for (long k = 0; k < (long)n * components; ++k) out[k] = std::strtof(T.tok[v + k].c_str(), nullptr);
        return OCT_OK;
    }
    return OCT_EINVAL;
}

oct_status oct_scene_write_vtk(oct_scene* s, const char* path) {
    if (!s || !path) return OCT_EINVAL;
    int32_t nn = 0, nel = 0, nc = 0, nf = 0;
    oct_status st = oct_scene_info(s, &nn, &nel, &nc, &nf);
    if (st) return st;
    int32_t element = 0;
    st = oct_scene_element_type(s, &element);
    if (st) return st;
    const int ne = nodes_of(element);
    std::vector<float> X(3 * (size_t)nn), p(3 * (size_t)nn), m(nn), u(3 * (size_t)nn), un(nn), smooth(nn, 0.f);
    std::vector<int32_t> topo((size_t)nel * ne);
    std::vector<float> stress(nel), vol(nel), dvol(nel), inv(nel);
    if ((st = oct_scene_get_rest_positions(s, X.data())) || (st = oct_scene_get_positions(s, p.data())) ||
        (st = oct_scene_get_masses(s, m.data())) || (st = oct_scene_get_topology(s, topo.data())) ||
        (st = oct_scene_element_data(s, OCT_DIAG_STRESS_ACCUMULATED, stress.data())) ||
        (st = oct_scene_element_data(s, OCT_DIAG_VOLUME, vol.data())) ||
        (st = oct_scene_element_data(s, OCT_DIAG_VOLUME_DIFF, dvol.data())) ||
        (st = oct_scene_element_data(s, OCT_DIAG_INVERTED, inv.data())))
        return st;
    for (int i = 0; i < nn; ++i) {
        for (int k = 0; k < 3; ++k) u[3 * i + k] = p[3 * i + k] - X[3 * i + k];
        un[i] = std::sqrt(u[3 * i] * u[3 * i] + u[3 * i + 1] * u[3 * i + 1] + u[3 * i + 2] * u[3 * i + 2]);
    }
    // get_stress_vertices (Cuda_FEM_Dynamic.h:89-110): element stress added to each of its
    // nodes, divided by the node's mass
    for (int e = 0; e < nel; ++e)
        for (int j = 0; j < ne; ++j) smooth[topo[(size_t)e * ne + j]] += stress[e];
    for (int i = 0; i < nn; ++i) smooth[i] /= m[i];
    const oct_vtk_field f[] = {
        {"weights", OCT_VTK_POINT, 1, m.data()},         {"u_norm", OCT_VTK_POINT, 1, un.data()},
        {"u", OCT_VTK_POINT, 3, u.data()},               {"smooth_stress", OCT_VTK_POINT, 1, smooth.data()},
        {"stress", OCT_VTK_CELL, 1, stress.data()},      {"volume", OCT_VTK_CELL, 1, vol.data()},
        {"volume_diff", OCT_VTK_CELL, 1, dvol.data()},   {"inverted", OCT_VTK_CELL, 1, inv.data()},
    };
    return oct_vtk_write(path, X.data(), nn, element, topo.data(), nel, f, (int32_t)(sizeof(f) / sizeof(f[0])));
}

}  // extern "C"
