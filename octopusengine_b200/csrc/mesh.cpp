// Beam meshes and lumped masses.
//
// The grid, the per-cell node order and the 6-tetrahedra split follow the reference's
// BeamMeshGenerator (octopus/src/Mesh/Generator/BeamGenerator.cpp:5-43, :86-92); the
// higher-order promotions follow tetra4_to_tetra10 (:172-214), tetra4_to_tetra20
// (:216-295) and hexa_to_hexa27 (:297-380).  New nodes are numbered in first-encounter
// order while walking the elements, which is what makes the numbering match the
// reference's; the lookup of already-created edge/face nodes uses hash maps keyed by the
// sorted corner ids instead of ordered maps (same result, O(1) lookups).
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <set>
#include <unordered_map>
#include <vector>

#include "host.hpp"

namespace octb {

namespace {

struct F3 { float x, y, z; };
inline F3 add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 mul(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }

inline uint64_t key2(int a, int b) {
    if (a > b) std::swap(a, b);
    return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
}
struct Key3Hash {
    size_t operator()(const std::array<int, 3>& k) const {
        uint64_t h = (uint64_t)k[0] * 0x9E3779B97F4A7C15ull ^ ((uint64_t)k[1] << 21) ^ ((uint64_t)k[2] << 42);
        return (size_t)(h ^ (h >> 29));
    }
};
struct Key4Hash {
    size_t operator()(const std::array<int, 4>& k) const {
        uint64_t h = 1469598103934665603ull;
        for (int v : k) { h ^= (uint64_t)(uint32_t)v; h *= 1099511628211ull; }
        return (size_t)h;
    }
};

void grid(bool tetra, int nx, int ny, int nz, float sx, float sy, float sz, F3 off, std::vector<F3>& X,
          std::vector<int32_t>& T) {
    const int Nx = nx + 1, Ny = ny + 1, Nz = nz + 1;
    const float xs = sx / float(Nx - 1), ys = sy / float(Ny - 1), zs = sz / float(Nz - 1);
    X.reserve((size_t)Nx * Ny * Nz);
    for (int z = 0; z < Nz; ++z)
        for (int y = 0; y < Ny; ++y)
            for (int x = 0; x < Nx; ++x) X.push_back({float(x) * xs + off.x, float(y) * ys + off.y, float(z) * zs + off.z});
    // per cell: bottom quad at y, top quad at y+1, each ordered (x,z) (x+1,z) (x+1,z+1) (x,z+1)
    static const int kSixTets[24] = {0, 4, 6, 5, 3, 6, 2, 0, 0, 4, 7, 6, 3, 6, 0, 7, 2, 0, 6, 1, 6, 0, 5, 1};
    T.reserve((size_t)nx * ny * nz * (tetra ? 24 : 8));
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                auto id = [&](int a, int b, int c) { return a + b * Nx + c * Nx * Ny; };
                const int c[8] = {id(x, y, z), id(x + 1, y, z), id(x + 1, y, z + 1), id(x, y, z + 1),
                                  id(x, y + 1, z), id(x + 1, y + 1, z), id(x + 1, y + 1, z + 1), id(x, y + 1, z + 1)};
                if (tetra) for (int k : kSixTets) T.push_back(c[k]);
                else for (int k = 0; k < 8; ++k) T.push_back(c[k]);
            }
}

void promote_p2(std::vector<F3>& X, std::vector<int32_t>& T) {
    static const int E[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
    std::unordered_map<uint64_t, int> edges;
    edges.reserve(T.size() * 2);
    std::vector<int32_t> out;
    out.reserve(T.size() / 4 * 10);
    for (size_t i = 0; i < T.size(); i += 4) {
        int ids[10];
        for (int j = 0; j < 4; ++j) ids[j] = T[i + j];
        for (int k = 0; k < 6; ++k) {
            const int a = ids[E[k][0]], b = ids[E[k][1]];
            auto ins = edges.emplace(key2(a, b), (int)X.size());
            if (ins.second) {
                const F3 pa = X[std::min(a, b)], pb = X[std::max(a, b)];
                X.push_back(mul(add(pa, pb), 0.5f));
            }
            ids[4 + k] = ins.first->second;
        }
        out.insert(out.end(), ids, ids + 10);
    }
    T.swap(out);
}

void promote_p3(std::vector<F3>& X, std::vector<int32_t>& T) {
    static const int E[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
    static const int F[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 3, 2}, {0, 2, 1}};
    struct EdgeNodes { int first_vertex, n0; };
    std::unordered_map<uint64_t, EdgeNodes> edges;
    std::unordered_map<std::array<int, 3>, int, Key3Hash> faces;
    edges.reserve(T.size() * 2);
    faces.reserve(T.size() * 2);
    std::vector<int32_t> out;
    out.reserve(T.size() / 4 * 20);
    for (size_t i = 0; i < T.size(); i += 4) {
        int ids[20];
        for (int j = 0; j < 4; ++j) ids[j] = T[i + j];
        int j = 4;
        for (int k = 0; k < 6; ++k) {
            const int a = ids[E[k][0]], b = ids[E[k][1]];
            auto it = edges.find(key2(a, b));
            if (it == edges.end()) {
                const int n0 = (int)X.size();
                for (int w = 0; w < 2; ++w) {
                    const float t = float(w + 1) / 3.f;
                    X.push_back(add(mul(X[a], 1.f - t), mul(X[b], t)));
                }
                edges.emplace(key2(a, b), EdgeNodes{a, n0});
                ids[j++] = n0; ids[j++] = n0 + 1;
            } else if (it->second.first_vertex == a) {
                ids[j++] = it->second.n0; ids[j++] = it->second.n0 + 1;
            } else {   // the edge was created walking b -> a: its nodes run the other way
                ids[j++] = it->second.n0 + 1; ids[j++] = it->second.n0;
            }
        }
        for (int k = 0; k < 4; ++k) {
            const int a = ids[F[k][0]], b = ids[F[k][1]], c = ids[F[k][2]];
            std::array<int, 3> key = {a, b, c};
            std::sort(key.begin(), key.end());
            auto ins = faces.emplace(key, (int)X.size());
            if (ins.second) {
                const float w = 1.f / 3.f;
                X.push_back(add(add(mul(X[a], w), mul(X[b], w)), mul(X[c], w)));
            }
            ids[j++] = ins.first->second;
        }
        out.insert(out.end(), ids, ids + 20);
    }
    T.swap(out);
}

void promote_q2(std::vector<F3>& X, std::vector<int32_t>& T) {
    static const int E[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5}, {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 4}};
    static const int F[6][4] = {{0, 1, 2, 3}, {4, 5, 1, 0}, {5, 6, 2, 1}, {3, 2, 6, 7}, {7, 4, 0, 3}, {7, 6, 5, 4}};
    std::unordered_map<uint64_t, int> edges;
    std::unordered_map<std::array<int, 4>, int, Key4Hash> faces;
    edges.reserve(T.size());
    faces.reserve(T.size());
    std::vector<int32_t> out;
    out.reserve(T.size() / 8 * 27);
    for (size_t i = 0; i < T.size(); i += 8) {
        int ids[27];
        for (int j = 0; j < 8; ++j) ids[j] = T[i + j];
        int j = 8;
        for (int k = 0; k < 12; ++k) {
            const int a = ids[E[k][0]], b = ids[E[k][1]];
            auto ins = edges.emplace(key2(a, b), (int)X.size());
            if (ins.second) X.push_back(mul(add(X[a], X[b]), 0.5f));
            ids[j++] = ins.first->second;
        }
        for (int k = 0; k < 6; ++k) {
            int v[4];
            for (int q = 0; q < 4; ++q) v[q] = ids[F[k][q]];
            std::array<int, 4> key = {v[0], v[1], v[2], v[3]};
            std::sort(key.begin(), key.end());
            auto ins = faces.emplace(key, (int)X.size());
            if (ins.second) {
                const float w = 0.25f;
                X.push_back(add(add(add(mul(X[v[0]], w), mul(X[v[1]], w)), mul(X[v[2]], w)), mul(X[v[3]], w)));
            }
            ids[j++] = ins.first->second;
        }
        F3 c = {0, 0, 0};
        for (int k = 0; k < 8; ++k) c = add(c, X[ids[k]]);
        c = {c.x / 8.f, c.y / 8.f, c.z / 8.f};
        ids[j] = (int)X.size();
        X.push_back(c);
        out.insert(out.end(), ids, ids + 27);
    }
    T.swap(out);
}

}  // namespace

bool beam_mesh(int e, int nx, int ny, int nz, float sx, float sy, float sz, float ox, float oy, float oz,
               std::vector<float>& Xout, std::vector<int32_t>& T) {
    if (element_nodes(e) < 0 || nx < 1 || ny < 1 || nz < 1) return false;
    const bool tetra = e == kTetra || e == kTetra10 || e == kTetra20;
    std::vector<F3> X;
    T.clear();
    grid(tetra, nx, ny, nz, sx, sy, sz, {ox, oy, oz}, X, T);
    if (e == kTetra10) promote_p2(X, T);
    if (e == kTetra20) promote_p3(X, T);
    if (e == kHexa27) promote_q2(X, T);
    Xout.resize(X.size() * 3);
    for (size_t i = 0; i < X.size(); ++i) { Xout[3 * i] = X[i].x; Xout[3 * i + 1] = X[i].y; Xout[3 * i + 2] = X[i].z; }
    return true;
}

void lumped_masses(int e, const float* X, int n, const int32_t* T, int n_elem, float density, int distribution,
                   std::vector<float>& mass) {
    ShapeTable s;
    shape_table(e, s);
    const int ne = s.ne;
    std::vector<float> dN(s.dN.begin(), s.dN.end());
    // element volume as FEM_Generic::compute_volume: sum_q |det J_q| w_q in FP32
    auto volume = [&](int el) {
        float vol = 0.f;
        for (int q = 0; q < s.nq; ++q) {
            float J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // J[col][row]
            for (int k = 0; k < ne; ++k) {
                const float* x = X + 3 * T[(size_t)el * ne + k];
                const float* d = &dN[((size_t)q * ne + k) * 3];
                for (int c = 0; c < 3; ++c)
                    for (int r = 0; r < 3; ++r) J[c][r] += x[r] * d[c];
            }
            const float det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) -
                              J[1][0] * (J[0][1] * J[2][2] - J[2][1] * J[0][2]) +
                              J[2][0] * (J[0][1] * J[1][2] - J[1][1] * J[0][2]);
            vol += std::fabs(det) * (float)s.w[q];
        }
        return vol;
    };
    mass.assign(n, 0.f);
    if (distribution == 1) {
        const float vd = density / (float)ne;
        for (int el = 0; el < n_elem; ++el) {
            const float V = volume(el);
            for (int j = 0; j < ne; ++j) mass[T[(size_t)el * ne + j]] += vd * V;
        }
    } else {
        float total = 0.f;
        for (int el = 0; el < n_elem; ++el) total += volume(el);
        total *= density;
        total /= (float)n;
        for (int i = 0; i < n; ++i) mass[i] = total;
    }
}

// Nodes on the mesh boundary, ascending (MeshTools::Get_Surface_Geometry_Ids,
// octopus/include/Mesh/MeshTools.h:64-89: the nodes of the element faces that no other element
// shares).  A face is keyed by its sorted corner ids; its nodes are every node of the element
// whose reference coordinates lie on that face (corners, edge and face nodes).
std::vector<int32_t> surface_nodes(int e, const int32_t* T, int n_elem) {
    const int ne = element_nodes(e);
    std::vector<double> rn(3 * ne);
    reference_nodes(e, rn.data());
    const bool tet = e == kTetra || e == kTetra10 || e == kTetra20;
    const int nc = tet ? 4 : 8, nf = tet ? 4 : 6;
    // on_face[f] = local nodes on face f
    std::vector<std::vector<int>> on_face(nf);
    for (int j = 0; j < ne; ++j) {
        const double* x = &rn[3 * j];
        for (int f = 0; f < nf; ++f) {
            bool on;
            if (tet) on = std::fabs(f == 0 ? 1.0 - x[0] - x[1] - x[2] : x[f - 1]) < 1e-9;   // L_f = 0
            else on = std::fabs(x[f / 2] - (f % 2 ? 1.0 : -1.0)) < 1e-9;
            if (on) on_face[f].push_back(j);
        }
    }
    std::map<std::vector<int32_t>, std::pair<int, std::pair<int, int>>> faces;   // corners -> (count, (element, face))
    for (int el = 0; el < n_elem; ++el)
        for (int f = 0; f < nf; ++f) {
            std::vector<int32_t> key;
            for (int j : on_face[f]) if (j < nc) key.push_back(T[(size_t)el * ne + j]);
            std::sort(key.begin(), key.end());
            auto it = faces.find(key);
            if (it == faces.end()) faces.emplace(key, std::make_pair(1, std::make_pair(el, f)));
            else it->second.first++;
        }
    std::set<int32_t> ids;
    for (const auto& [key, v] : faces) {
        if (v.first != 1) continue;
        const int el = v.second.first, f = v.second.second;
        for (int j : on_face[f]) ids.insert(T[(size_t)el * ne + j]);
    }
    return std::vector<int32_t>(ids.begin(), ids.end());
}

}  // namespace octb
