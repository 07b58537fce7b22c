// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle.h).  Restates the reference's
// hot-path algorithms; every function names the reference file:line it follows.
// Paths are relative to the OctopusEngine project root.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <queue>
#include <random>
#include <set>
#include <thread>
#include <tuple>
#include <vector>

namespace orc {

// ----------------------------------------------------------------------------- math
// Column-major 3x3 like glm: m.c[j] is column j, m(i,j) = c[j][i].
template <class T> struct V3 {
    T x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class T> V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V3<T> operator*(T s, V3<T> a) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}

template <class T> struct M3 {
    V3<T> c[3];
    M3() {}
    explicit M3(T d) { c[0] = {d, 0, 0}; c[1] = {0, d, 0}; c[2] = {0, 0, d}; }
    V3<T>& operator[](int j) { return c[j]; }
    const V3<T>& operator[](int j) const { return c[j]; }
};
template <class T> M3<T> operator+(const M3<T>& a, const M3<T>& b) { M3<T> r; for (int j = 0; j < 3; ++j) r[j] = a[j] + b[j]; return r; }
template <class T> M3<T> operator-(const M3<T>& a, const M3<T>& b) { M3<T> r; for (int j = 0; j < 3; ++j) r[j] = a[j] - b[j]; return r; }
template <class T> M3<T> operator-(const M3<T>& a) { M3<T> r; for (int j = 0; j < 3; ++j) r[j] = -a[j]; return r; }
template <class T> M3<T> operator*(const M3<T>& a, T s) { M3<T> r; for (int j = 0; j < 3; ++j) r[j] = a[j] * s; return r; }
template <class T> M3<T> operator*(T s, const M3<T>& a) { return a * s; }
template <class T> V3<T> operator*(const M3<T>& m, V3<T> v) { return m[0] * v.x + m[1] * v.y + m[2] * v.z; }
template <class T> M3<T> operator*(const M3<T>& a, const M3<T>& b) { M3<T> r; for (int j = 0; j < 3; ++j) r[j] = a * b[j]; return r; }
template <class T> M3<T> transpose(const M3<T>& m) {
    M3<T> r;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r[i][j] = m[j][i];
    return r;
}
template <class T> M3<T> outer(V3<T> a, V3<T> b) {  // a b^T
    M3<T> r;
    for (int j = 0; j < 3; ++j) r[j] = a * b[j];
    return r;
}
template <class T> T det(const M3<T>& m) {
    return m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2])
         - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2])
         + m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
}
// Inverse through the adjugate (transposed cofactors) divided by the determinant.
template <class T> M3<T> inverse(const M3<T>& m) {
    const T inv = T(1) / det(m);
    M3<T> r;
    r[0][0] = (m[1][1] * m[2][2] - m[2][1] * m[1][2]) * inv;
    r[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * inv;
    r[2][0] = (m[1][0] * m[2][1] - m[2][0] * m[1][1]) * inv;
    r[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * inv;
    r[1][1] = (m[0][0] * m[2][2] - m[2][0] * m[0][2]) * inv;
    r[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * inv;
    r[0][2] = (m[0][1] * m[1][2] - m[1][1] * m[0][2]) * inv;
    r[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * inv;
    r[2][2] = (m[0][0] * m[1][1] - m[1][0] * m[0][1]) * inv;
    return r;
}
// Cofactor matrix by column cross products (CUMatrix.cu:28-30).
template <class T> M3<T> com(const M3<T>& m) {
    M3<T> r;
    r[0] = cross(m[1], m[2]); r[1] = cross(m[2], m[0]); r[2] = cross(m[0], m[1]);
    return r;
}
template <class T> M3<T> hat(V3<T> v) {  // CUMatrix.cu:20-26, column-major construction
    M3<T> r;
    r[0] = {T(0), v.z, -v.y}; r[1] = {-v.z, T(0), v.x}; r[2] = {v.y, -v.x, T(0)};
    return r;
}
template <class T> T trace(const M3<T>& m) { return m[0][0] + m[1][1] + m[2][2]; }
template <class T> T squared_trace(const M3<T>& m) {  // CUMatrix.cu:38-41
    return m[0][0] * m[0][0] + m[1][1] * m[1][1] + m[2][2] * m[2][2]
         + (m[0][1] * m[1][0] + m[1][2] * m[2][1] + m[2][0] * m[0][2]) * T(2);
}
template <class T> T squared_norm(const M3<T>& m) {
    T s = 0;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) s += m[i][j] * m[i][j];
    return s;
}
template <class T> T length(V3<T> v) { return std::sqrt(dot(v, v)); }

// ----------------------------------------------------------------------------- elements
enum Element { Line, Triangle, Quad, Tetra, Pyramid, Prism, Hexa, Tetra10, Tetra20, Hexa27 };
int nodes_of(int e) {
    switch (e) {
        case Tetra: return 4; case Pyramid: return 5; case Prism: return 6; case Hexa: return 8;
        case Tetra10: return 10; case Tetra20: return 20; case Hexa27: return 27;
        default: return -1;
    }
}

// ----------------------------------------------------------------------------- shapes
// Shape functions restated from FEM_Shape.h build_shape (Tetra_4 :47-49, Hexa_8 :207-221,
// Tetra_10 :257-271, Tetra_20 :452-478, Hexa_27 :657-689), written over barycentric /
// 1-D Lagrange factors; derivatives by forward-mode dual numbers.  Quadrature points and
// weights: Tetra_4 :40-46, Hexa_8 :178-189, Tetra_10 :230-237, Tetra_20 :277-333 (the
// 11-point polyfem rule), Hexa_27 :486-520.
struct Dual {
    double v, d[3];
    Dual(double a = 0) : v(a) { d[0] = d[1] = d[2] = 0; }
};
static Dual operator+(Dual a, Dual b) { Dual r(a.v + b.v); for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] + b.d[k]; return r; }
static Dual operator-(Dual a, Dual b) { Dual r(a.v - b.v); for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] - b.d[k]; return r; }
static Dual operator*(Dual a, Dual b) { Dual r(a.v * b.v); for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k]; return r; }
static Dual operator*(double s, Dual a) { Dual r(a.v * s); for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * s; return r; }

static const double T20_QP[11][3] = {
    {0.040490506727590428, 0.013560701879802881, 0.77125473269537614},
    {0.75250850700965499, 0.068099370938206658, 0.097987203649279112},
    {0.067223294893383398, 0.035183929773598716, 0.15636389323939529},
    {0.41926631387951302, 0.047781435559086663, 0.47961101102565507},
    {0.45076587609127683, 0.059456616299433829, 0.056824017127933668},
    {0.12941137378891041, 0.33019041483746447, 0.0023910074574393647},
    {0.12154199133392780, 0.30649398842969028, 0.56297276014304609},
    {0.097204644587583267, 0.68439041545304002, 0.11180076739738309},
    {0.029569495206479612, 0.31790356021339461, 0.32329398483747895},
    {0.43271023904776856, 0.35382323920929709, 0.10962240533194123},
    {0.24027666492807262, 0.12680172591539202, 0.32847320672203845}};
static const double T20_W[11] = {
    0.039251090924839957, 0.055273369155936898, 0.055393798871576368, 0.059933185146559528,
    0.069469965937635367, 0.076162715245558357, 0.079426680068025307, 0.10646803415549010,
    0.11023423242849766, 0.15497611601624608, 0.19341081204963445};

// Tetra_20 node layout: corners 0-3, edge nodes (a -> b, one third from a) 4-15, faces 16-19.
static const int T20_EDGE[12][2] = {{0, 1}, {1, 0}, {1, 2}, {2, 1}, {2, 0}, {0, 2},
                                    {0, 3}, {3, 0}, {1, 3}, {3, 1}, {2, 3}, {3, 2}};
static const int T20_FACE[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 2, 3}, {0, 1, 2}};
// Tetra_10 edge nodes 4-9.
static const int T10_EDGE[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
// Hexa_8 / Hexa_27 reference coordinates (FEM_Shape.h:192-197, :535-577).
static const int H27_NODE[27][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
    {0, -1, -1}, {1, 0, -1}, {0, 1, -1}, {-1, 0, -1}, {-1, -1, 0}, {1, -1, 0}, {1, 1, 0}, {-1, 1, 0},
    {0, -1, 1}, {1, 0, 1}, {0, 1, 1}, {-1, 0, 1}, {0, 0, -1}, {0, -1, 0}, {1, 0, 0}, {0, 1, 0},
    {-1, 0, 0}, {0, 0, 1}, {0, 0, 0}};

static Dual lag1d(int node, Dual s) {  // quadratic Lagrange on {-1,0,1}
    if (node == -1) return 0.5 * (s * (s - Dual(1)));
    if (node == 1) return 0.5 * (s * (s + Dual(1)));
    return (Dual(1) - s) * (Dual(1) + s);
}

static void shape_values(int e, Dual x, Dual y, Dual z, Dual* N) {
    Dual L[4] = {Dual(1) - x - y - z, x, y, z};
    switch (e) {
        case Tetra:
            for (int i = 0; i < 4; ++i) N[i] = L[i];
            break;
        case Tetra10:
            for (int i = 0; i < 4; ++i) N[i] = L[i] * (2.0 * L[i] - Dual(1));
            for (int k = 0; k < 6; ++k) N[4 + k] = 4.0 * (L[T10_EDGE[k][0]] * L[T10_EDGE[k][1]]);
            break;
        case Tetra20:
            for (int i = 0; i < 4; ++i) N[i] = 0.5 * ((3.0 * L[i] - Dual(1)) * (3.0 * L[i] - Dual(2)) * L[i]);
            for (int k = 0; k < 12; ++k) {
                const Dual& a = L[T20_EDGE[k][0]];
                const Dual& b = L[T20_EDGE[k][1]];
                N[4 + k] = 4.5 * (a * b * (3.0 * a - Dual(1)));
            }
            for (int k = 0; k < 4; ++k) N[16 + k] = 27.0 * (L[T20_FACE[k][0]] * L[T20_FACE[k][1]] * L[T20_FACE[k][2]]);
            break;
        case Hexa:
            for (int i = 0; i < 8; ++i)
                N[i] = 0.125 * ((Dual(1) + H27_NODE[i][0] * x) * (Dual(1) + H27_NODE[i][1] * y) * (Dual(1) + H27_NODE[i][2] * z));
            break;
        case Hexa27:
            for (int i = 0; i < 27; ++i) N[i] = lag1d(H27_NODE[i][0], x) * lag1d(H27_NODE[i][1], y) * lag1d(H27_NODE[i][2], z);
            break;
    }
}

struct Shape {
    int nb = 0, nq = 0;
    std::vector<double> qp, w;  // nq*3, nq
    std::vector<double> dN;     // nq*nb*3
};

static bool build_shape(int e, Shape& s) {
    s.nb = nodes_of(e);
    std::vector<double> qp, w;
    if (e == Tetra) { qp = {0.25, 0.25, 0.25}; w = {1.0 / 6.0}; }
    else if (e == Hexa) {
        const double c = 1.0 / std::sqrt(3.0);
        const int sg[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1}};
        for (auto& g : sg) for (int k = 0; k < 3; ++k) qp.push_back(c * g[k]);
        w.assign(8, 1.0);
    } else if (e == Tetra10) {
        const double a = (5.0 - std::sqrt(5.0)) / 20.0, b = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0;
        qp = {b, a, a, a, b, a, a, a, b, a, a, a};
        w.assign(4, 1.0 / 24.0);
    } else if (e == Tetra20) {
        for (int q = 0; q < 11; ++q) { for (int k = 0; k < 3; ++k) qp.push_back(T20_QP[q][k]); w.push_back(T20_W[q] / 6.0); }
    } else if (e == Hexa27) {
        const double v = std::sqrt(3.0 / 5.0);
        const double z8 = 8.0 / 9.0, f5 = 5.0 / 9.0;
        // the 27 quadrature points follow the node layout of H27_NODE scaled by v
        for (int q = 0; q < 27; ++q) {
            double wq = 1;
            for (int k = 0; k < 3; ++k) { qp.push_back(v * H27_NODE[q][k]); wq *= H27_NODE[q][k] == 0 ? z8 : f5; }
            w.push_back(wq);
        }
    } else return false;
    s.nq = (int)w.size();
    s.qp = qp; s.w = w;
    s.dN.assign(s.nq * s.nb * 3, 0.0);
    for (int q = 0; q < s.nq; ++q) {
        Dual x(qp[3 * q]), y(qp[3 * q + 1]), z(qp[3 * q + 2]);
        x.d[0] = 1; y.d[1] = 1; z.d[2] = 1;
        Dual N[27];
        shape_values(e, x, y, z, N);
        for (int i = 0; i < s.nb; ++i) for (int k = 0; k < 3; ++k) s.dN[(q * s.nb + i) * 3 + k] = N[i].d[k];
    }
    return true;
}

// ----------------------------------------------------------------------------- meshes
// BeamMeshGenerator::build / build_geometry_grid / get_cell_vertices_ids
// (BeamGenerator.cpp:5-43), HexaBeamGenerator (:45-49), TetraBeamGenerator 6-tet split
// (:86-92), tetra4_to_tetra10 (:172-214), tetra4_to_tetra20 (:216-295), hexa_to_hexa27
// (:297-380) with the converter edge/face tables of MeshConverter.h:92-100,137-150.
struct Mesh {
    std::vector<V3<float>> X;
    std::vector<int> topo;
};

static void beam_linear(bool tetra, int nx, int ny, int nz, float sx, float sy, float sz, V3<float> off, Mesh& m) {
    const int Nx = nx + 1, Ny = ny + 1, Nz = nz + 1;
    const float xs = sx / float(Nx - 1), ys = sy / float(Ny - 1), zs = sz / float(Nz - 1);
    for (int z = 0; z < Nz; ++z)
        for (int y = 0; y < Ny; ++y)
            for (int x = 0; x < Nx; ++x)
                m.X.push_back({float(x) * xs + off.x, float(y) * ys + off.y, float(z) * zs + off.z});
    auto id = [&](int x, int y, int z) { return x + y * Nx + z * Ny * Nx; };
    static const int six[24] = {0, 4, 6, 5, 3, 6, 2, 0, 0, 4, 7, 6, 3, 6, 0, 7, 2, 0, 6, 1, 6, 0, 5, 1};
    for (int z = 0; z < Nz - 1; ++z)
        for (int y = 0; y < Ny - 1; ++y)
            for (int x = 0; x < Nx - 1; ++x) {
                int c[8] = {id(x, y, z), id(x + 1, y, z), id(x + 1, y, z + 1), id(x, y, z + 1),
                            id(x, y + 1, z), id(x + 1, y + 1, z), id(x + 1, y + 1, z + 1), id(x, y + 1, z + 1)};
                if (tetra) for (int k : six) m.topo.push_back(c[k]);
                else for (int k = 0; k < 8; ++k) m.topo.push_back(c[k]);
            }
}

static void to_tetra10(Mesh& m) {
    std::map<std::pair<int, int>, int> edges;
    std::vector<int> out;
    static const int E[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
    for (size_t i = 0; i < m.topo.size(); i += 4) {
        int ids[10];
        for (int j = 0; j < 4; ++j) ids[j] = m.topo[i + j];
        for (int k = 0; k < 6; ++k) {
            int a = ids[E[k][0]], b = ids[E[k][1]];
            if (a > b) std::swap(a, b);
            auto it = edges.find({a, b});
            int nid;
            if (it != edges.end()) nid = it->second;
            else {
                nid = (int)m.X.size();
                V3<float> pa = m.X[a], pb = m.X[b];
                m.X.push_back(0.5f * (pa + pb));
                edges[{a, b}] = nid;
            }
            ids[4 + k] = nid;
        }
        out.insert(out.end(), ids, ids + 10);
    }
    m.topo = out;
}

static void to_tetra20(Mesh& m) {
    static const int E[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
    static const int F[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 3, 2}, {0, 2, 1}};
    // edge key: sorted pair -> (first vertex as first met, the two node ids)
    std::map<std::pair<int, int>, std::pair<int, std::pair<int, int>>> edges;
    std::map<std::array<int, 3>, int> faces;
    std::vector<int> out;
    for (size_t i = 0; i < m.topo.size(); i += 4) {
        int ids[20];
        for (int j = 0; j < 4; ++j) ids[j] = m.topo[i + j];
        int j = 4;
        for (int k = 0; k < 6; ++k) {
            const int a = ids[E[k][0]], b = ids[E[k][1]];
            std::pair<int, int> key(std::min(a, b), std::max(a, b));
            auto it = edges.find(key);
            int n0, n1;
            if (it != edges.end()) {
                n0 = it->second.second.first; n1 = it->second.second.second;
                if (a != it->second.first) std::swap(n0, n1);
            } else {
                n0 = (int)m.X.size();
                for (int w = 0; w < 2; ++w) {
                    const float wt = float(w + 1) / 3.f;
                    m.X.push_back(m.X[a] * (1.f - wt) + m.X[b] * wt);
                }
                n1 = n0 + 1;
                edges[key] = {a, {n0, n1}};
            }
            ids[j++] = n0; ids[j++] = n1;
        }
        for (int k = 0; k < 4; ++k) {
            const int a = ids[F[k][0]], b = ids[F[k][1]], c = ids[F[k][2]];
            std::array<int, 3> key = {a, b, c};
            std::sort(key.begin(), key.end());
            auto it = faces.find(key);
            int nid;
            if (it != faces.end()) nid = it->second;
            else {
                const float w = 1.f / 3.f;
                nid = (int)m.X.size();
                m.X.push_back(m.X[a] * w + m.X[b] * w + m.X[c] * w);
                faces[key] = nid;
            }
            ids[j++] = nid;
        }
        out.insert(out.end(), ids, ids + 20);
    }
    m.topo = out;
}

static void to_hexa27(Mesh& m) {
    static const int E[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5}, {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 4}};
    static const int F[6][4] = {{0, 1, 2, 3}, {4, 5, 1, 0}, {5, 6, 2, 1}, {3, 2, 6, 7}, {7, 4, 0, 3}, {7, 6, 5, 4}};
    std::map<std::pair<int, int>, int> edges;
    std::map<std::array<int, 4>, int> faces;
    std::vector<int> out;
    for (size_t i = 0; i < m.topo.size(); i += 8) {
        int ids[27];
        for (int j = 0; j < 8; ++j) ids[j] = m.topo[i + j];
        int j = 8;
        for (int k = 0; k < 12; ++k) {
            const int a = ids[E[k][0]], b = ids[E[k][1]];
            std::pair<int, int> key(std::min(a, b), std::max(a, b));
            auto it = edges.find(key);
            int nid;
            if (it != edges.end()) nid = it->second;
            else {
                nid = (int)m.X.size();
                m.X.push_back(0.5f * (m.X[a] + m.X[b]));
                edges[key] = nid;
            }
            ids[j++] = nid;
        }
        for (int k = 0; k < 6; ++k) {
            int v[4];
            for (int q = 0; q < 4; ++q) v[q] = ids[F[k][q]];
            std::array<int, 4> key = {v[0], v[1], v[2], v[3]};
            std::sort(key.begin(), key.end());
            auto it = faces.find(key);
            int nid;
            if (it != faces.end()) nid = it->second;
            else {
                const float w = 0.25f;
                nid = (int)m.X.size();
                m.X.push_back(m.X[v[0]] * w + m.X[v[1]] * w + m.X[v[2]] * w + m.X[v[3]] * w);
                faces[key] = nid;
            }
            ids[j++] = nid;
        }
        V3<float> c;
        for (int k = 0; k < 8; ++k) c = c + m.X[ids[k]];
        c = c / 8.f;
        ids[j] = (int)m.X.size();
        m.X.push_back(c);
        out.insert(out.end(), ids, ids + 27);
    }
    m.topo = out;
}

// ----------------------------------------------------------------------------- graphs
// Graph::build_primal (Graph.h:36-54): multiset adjacency, degree counts duplicates.
struct Graph {
    int n = 0;
    std::vector<int> degree;
    std::vector<std::multiset<int>> adj;
};
static Graph build_primal(int ne, const int* topo, int n_elem) {
    Graph g;
    g.n = *std::max_element(topo, topo + ne * n_elem) + 1;
    g.adj.resize(g.n);
    g.degree.resize(g.n);
    for (int i = 0; i < ne * n_elem; i += ne)
        for (int j = 0; j < ne; ++j)
            for (int k = 0; k < ne; ++k)
                if (k != j) g.adj[topo[i + j]].insert(topo[i + k]);
    for (int i = 0; i < g.n; ++i) g.degree[i] = (int)g.adj[i].size();
    return g;
}
// Graph::build_dual_vertex (Graph.h:56-85).
static Graph build_dual_vertex(int ne, const int* topo, int n_elem) {
    Graph g;
    g.n = n_elem;
    g.adj.resize(g.n);
    g.degree.assign(g.n, 0);
    const int nv = *std::max_element(topo, topo + ne * n_elem) + 1;
    std::vector<std::vector<int>> owners(nv);
    for (int e = 0; e < n_elem; ++e) for (int i = 0; i < ne; ++i) owners[topo[e * ne + i]].push_back(e);
    for (int v = 0; v < nv; ++v)
        for (size_t j = 0; j < owners[v].size(); ++j)
            for (size_t k = j + 1; k < owners[v].size(); ++k) {
                const int a = owners[v][j], b = owners[v][k];
                g.adj[a].insert(b); g.adj[b].insert(a);
                g.degree[a]++; g.degree[b]++;
            }
    return g;
}

// GraphColoration::find_color_greedy (Graph.h:906-926)
static void greedy_pick(const Graph& g, int i, int& nb_color, std::vector<int>& colors) {
    std::set<int> used;
    for (int id : g.adj[i]) if (colors[id] != -1) used.insert(colors[id]);
    for (int c = 0; c < nb_color; ++c)
        if (!used.count(c)) { colors[i] = c; return; }
    colors[i] = nb_color++;
}

// GraphColoration::DSAT (Graph.h:321-371) with Node/maxSat ordering (:884-904): the queue
// is a set ordered by (saturation, degree, vertex) descending; degrees drop once per
// multiset occurrence.
static int dsat(const Graph& g, std::vector<int>& colors) {
    typedef std::tuple<int, int, int> Node;
    std::set<Node, std::greater<Node>> q;
    std::vector<bool> used(g.n, false);
    colors.assign(g.n, -1);
    std::vector<int> degree(g.degree);
    std::vector<std::set<int>> adjc(g.n);
    for (int v = 0; v < g.n; ++v) q.emplace(0, degree[v], v);
    while (!q.empty()) {
        const int vid = std::get<2>(*q.begin());
        q.erase(q.begin());
        for (int v : g.adj[vid]) if (colors[v] != -1) used[colors[v]] = true;
        int i;
        for (i = 0; i < (int)used.size(); ++i) if (!used[i]) break;
        for (int v : g.adj[vid]) if (colors[v] != -1) used[colors[v]] = false;
        colors[vid] = i;
        for (int v : g.adj[vid]) {
            if (colors[v] == -1) {
                q.erase(Node((int)adjc[v].size(), degree[v], v));
                adjc[v].insert(i);
                degree[v]--;
                q.emplace((int)adjc[v].size(), degree[v], v);
            }
        }
    }
    return *std::max_element(colors.begin(), colors.end()) + 1;
}

// GraphColoration::Greedy_SLF (Graph.h:237-277): smallest-last ordering with a min-heap of
// (degree, id), then greedy colouring in that order.
static int greedy_slf(const Graph& g, std::vector<int>& colors) {
    int nb_color = 0;
    const int n = g.n;
    typedef std::pair<int, int> PV;
    std::priority_queue<PV, std::vector<PV>, std::greater<PV>> h;
    for (int i = 0; i < n; ++i) h.push({g.degree[i], i});
    std::vector<int> ids(n, 0);
    std::vector<bool> removed(n, false);
    std::vector<int> degree = g.degree;
    for (int i = n - 1; i >= 0; i--) {
        while (!h.empty() && removed[h.top().second]) h.pop();
        const int v = h.top().second;
        h.pop();
        removed[v] = true;
        ids[i] = v;
        for (int nb : g.adj[v])
            if (!removed[nb]) { degree[nb]--; h.push({degree[nb], nb}); }
    }
    colors.assign(n, -1);
    for (int i : ids) greedy_pick(g, i, nb_color, colors);
    return nb_color;
}

// GraphReduction::ColorReduction (Graph.h:941-969)
static void color_reduction(const Graph& g, std::vector<int>& colors, int target) {
    std::set<int> to_color;
    for (int i = 0; i < g.n; ++i) if (colors[i] >= target) to_color.insert(i);
    for (int vid : to_color) {
        std::vector<int> occ(target, 0);
        for (int a : g.adj[vid]) { if (colors[a] >= target) continue; occ[colors[a]]++; }
        colors[vid] = (int)(std::min_element(occ.begin(), occ.end()) - occ.begin());
    }
}

// ----------------------------------------------------------------------------- materials
enum Material { Hooke = 0, StVK = 1, NeoHooke = 2, StableNeoHooke = 3, Corotated = 4, FixedCorotated = 5 };

// PK1 stresses, GPU_FEM_Material.cu:5-36
template <class T> M3<T> pk1(int mat, T lambda, T mu, const M3<T>& F) {
    const M3<T> I(T(1));
    if (mat == Hooke) {
        M3<T> E = T(0.5) * (transpose(F) + F) - I;
        return M3<T>(lambda * trace(E)) + mu * E;
    }
    if (mat == StVK) {
        M3<T> E = T(0.5) * (transpose(F) * F - I);
        return lambda * trace(E) * F + T(2) * mu * F * E;
    }
    const T alpha = mat == NeoHooke ? T(1) : T(1) + mu / lambda;
    return lambda * (det(F) - alpha) * com(F) + mu * F;
}

// Energies, FEM_ContinuousMaterial.cpp:10-15,31-36,70-74,83-87
template <class T> T energy(int mat, T lambda, T mu, const M3<T>& F) {
    const M3<T> I(T(1));
    if (mat == Hooke || mat == StVK) {
        M3<T> E = mat == Hooke ? T(0.5) * (transpose(F) + F) - I : T(0.5) * (transpose(F) * F - I);
        const T tr = trace(E);
        return T(0.5) * lambda * tr * tr + mu * squared_norm(E);
    }
    const T alpha = mat == NeoHooke ? T(1) : T(1) + mu / lambda;
    const T d = det(F) - alpha;
    return T(0.5) * mu * (squared_norm(F) - T(3)) + T(0.5) * lambda * d * d;
}

// Upper-triangle Hessian blocks d2W/dF_i dF_j, GPU_FEM_Material.cu:133-207
// (k = 0:(0,0) 1:(0,1) 2:(0,2) 3:(1,1) 4:(1,2) 5:(2,2)).
template <class T> void hessian_sym(int mat, T lambda, T mu, const M3<T>& F, M3<T> B[6]) {
    if (mat == Hooke) {
        for (int k = 0; k < 6; ++k) B[k] = M3<T>(T(0));
        B[0] = B[3] = B[5] = M3<T>(mu + lambda);
        return;
    }
    if (mat == StVK) {
        const M3<T> FFt = F * transpose(F), FtF = transpose(F) * F;
        const M3<T> diag = M3<T>(T(0.5) * lambda * trace(FFt) - mu) + mu * FFt;
        B[1] = B[2] = B[4] = M3<T>(T(0));
        B[0] = B[3] = B[5] = diag;
        for (int i = 0, k = 0; i <= 2; ++i)
            for (int j = i; j <= 2; ++j, ++k) {
                B[k] = B[k] + T(0.5) * lambda * outer(F[i], F[j]);
                B[k] = B[k] + mu * outer(F[j], F[i]);
                B[k] = B[k] + M3<T>(FtF[i][j]);
            }
        return;
    }
    const M3<T> cF = com(F);
    const T alpha = mat == NeoHooke ? T(1) : T(1) + mu / lambda;
    const T s = lambda * (det(F) - alpha);
    B[1] = hat(F[2]) * s;
    B[2] = -hat(F[1]) * s;
    B[4] = hat(F[0]) * s;
    B[0] = B[3] = B[5] = M3<T>(mu);
    for (int i = 0, k = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j, ++k) B[k] = B[k] + outer(cF[j], cF[i]) * lambda;
}

// assemble_sub_hessian_sym, GPU_FEM_Material.cu:250-261
template <class T> M3<T> assemble_sym(V3<T> g, T V, M3<T> B[6]) {
    M3<T> H(T(0));
    H = H + g[1] * g[0] * (B[1] + transpose(B[1]));
    H = H + g[2] * g[0] * (B[2] + transpose(B[2]));
    H = H + g[2] * g[1] * (B[4] + transpose(B[4]));
    H = H + g[0] * g[0] * B[0];
    H = H + g[1] * g[1] * B[3];
    H = H + g[2] * g[2] * B[5];
    return H * V;
}

// ----------------------------------------------------------------------------- FEM data
template <class T> struct Fem {
    int elem = 0, ne = 0, nq = 0, n_elem = 0;
    std::vector<int> topo;
    std::vector<M3<T>> JX_inv;  // E*Q
    std::vector<T> V;           // E*Q
    std::vector<V3<T>> dN;      // Q*ne
    std::vector<T> weights;
    std::vector<T> lambda, mu;  // per element
    int material = StableNeoHooke;
};

// GPU_FEM::GPU_FEM + build_fem_const (GPU_FEM.cu:155-215): J = sum X_k (x) dN_qk,
// V = |det J| w_q, JX_inv = J^-1.  Lame parameters from (E, nu) (GPU_FEM.cu:162-163).
template <class T> bool build_fem(const orc_desc* d, Fem<T>& f) {
    Shape s;
    if (!build_shape(d->element, s) || d->material < Hooke || d->material > FixedCorotated) return false;
    f.elem = d->element; f.ne = s.nb; f.nq = s.nq; f.n_elem = d->n_elements; f.material = d->material;
    f.topo.assign(d->topology, d->topology + (size_t)f.ne * f.n_elem);
    for (int q = 0; q < f.nq; ++q) {
        f.weights.push_back((T)s.w[q]);
        for (int i = 0; i < f.ne; ++i) {
            const double* p = &s.dN[(q * f.ne + i) * 3];
            f.dN.push_back({(T)p[0], (T)p[1], (T)p[2]});
        }
    }
    f.JX_inv.resize((size_t)f.n_elem * f.nq);
    f.V.resize((size_t)f.n_elem * f.nq);
    for (int e = 0; e < f.n_elem; ++e)
        for (int q = 0; q < f.nq; ++q) {
            M3<T> J(T(0));
            for (int k = 0; k < f.ne; ++k) {
                const float* x = d->positions + 3 * f.topo[e * f.ne + k];
                J = J + outer(V3<T>((T)x[0], (T)x[1], (T)x[2]), f.dN[q * f.ne + k]);
            }
            f.V[e * f.nq + q] = std::abs(det(J)) * f.weights[q];
            f.JX_inv[e * f.nq + q] = inverse(J);
        }
    f.lambda.resize(f.n_elem); f.mu.resize(f.n_elem);
    for (int e = 0; e < f.n_elem; ++e) {
        const T E = (T)(d->young_per_element ? d->young_per_element[e] : d->young), nu = (T)d->poisson;
        f.lambda[e] = E * nu / ((T(1) + nu) * (T(1) - T(2) * nu));
        f.mu[e] = E / (T(2) * (T(1) + nu));
    }
    return true;
}

template <class T> M3<T> deformation(const Fem<T>& f, const std::vector<V3<T>>& p, int e, int q) {
    M3<T> Jx(T(0));
    for (int i = 0; i < f.ne; ++i) Jx = Jx + outer(p[f.topo[e * f.ne + i]], f.dN[q * f.ne + i]);
    return Jx * f.JX_inv[e * f.nq + q];
}

// ----------------------------------------------------------------------------- particle state
template <class T> struct State {
    int n = 0;
    std::vector<V3<T>> p, last_p, init_p, v, f, y, prev_it_p, prev_it2_p, p_new;
    std::vector<T> m, w;
    std::vector<int> mask;
    V3<T> g;
    std::vector<int> fixed, fgroup;
    V3<T> com[4], off[4];
    M3<T> R[4];
    bool box = false;
    V3<T> bmin, bmax;
    // scripted effects (GPU_Crush / GPU_RandomSphere / GPU_HighStretch)
    struct Effect { int kind; bool active; std::vector<int> ids; V3<T> c; T radius, max_dist, t; };
    std::vector<Effect> effects;
};

// GPU_ParticleSystem ctor (GPU_ParticleSystem.cu:6-22) and GPU_Fix_Constraint ctor
// (GPU_Constraint.cu:94-107).  An initial velocity is encoded as last_p = p - v0*dt at the
// first step (GPU VBD reads the implicit velocity, GPU_VBD.cu:14).
template <class T> void init_state(const orc_desc* d, State<T>& s) {
    s.n = d->n_nodes;
    s.p.resize(s.n); s.m.resize(s.n); s.w.resize(s.n);
    for (int i = 0; i < s.n; ++i) {
        s.p[i] = {(T)d->positions[3 * i], (T)d->positions[3 * i + 1], (T)d->positions[3 * i + 2]};
        s.m[i] = (T)d->masses[i];
        s.w[i] = T(1) / s.m[i];
    }
    s.last_p = s.init_p = s.y = s.prev_it_p = s.prev_it2_p = s.p_new = s.p;
    s.v.assign(s.n, V3<T>());
    s.f.assign(s.n, V3<T>());
    if (d->initial_velocity)
        for (int i = 0; i < s.n; ++i)
            s.v[i] = {(T)d->initial_velocity[3 * i], (T)d->initial_velocity[3 * i + 1], (T)d->initial_velocity[3 * i + 2]};
    s.mask.assign(s.n, 1);
    s.g = {(T)d->gravity[0], (T)d->gravity[1], (T)d->gravity[2]};
    s.fixed.assign(d->fixed_ids, d->fixed_ids + d->n_fixed);
    s.fgroup.assign(s.fixed.size(), 0);
    if (d->fixed_group) for (size_t k = 0; k < s.fixed.size(); ++k) s.fgroup[k] = d->fixed_group[k];
    for (int g = 0; g < 4; ++g) {   // float centre of mass per group (GPU_Constraint.cu:94-107)
        V3<float> c;
        int cnt = 0;
        for (size_t k = 0; k < s.fixed.size(); ++k) {
            if (s.fgroup[k] != g) continue;
            const int id = s.fixed[k];
            c = c + V3<float>(d->positions[3 * id], d->positions[3 * id + 1], d->positions[3 * id + 2]);
            ++cnt;
        }
        if (cnt) c = c / float(cnt);
        s.com[g] = {(T)c.x, (T)c.y, (T)c.z};
        s.off[g] = V3<T>();
        s.R[g] = M3<T>(T(1));
    }
    s.box = d->box_limit != 0;
    s.bmin = {(T)d->box_min[0], (T)d->box_min[1], (T)d->box_min[2]};
    s.bmax = {(T)d->box_max[0], (T)d->box_max[1], (T)d->box_max[2]};
}

// kernel_constraint_fix (GPU_Constraint.cu:8-20) with identity rotation and zero offset,
// then kernel_constraint_box_limit (:80-92) when enabled.
// The sine hash of kernel_constraint_random_sphere (GPU_Constraint.cu:36-51), in T.
template <class T> T fract(T x) { return x - std::floor(x); }
template <class T> T hash1(T v) { return fract(std::sin(v * T(91.3458f)) * T(47453.5453f)); }
template <class T> T hash2(T a, T b) { return fract(std::sin(a * T(12.9898f) + b * T(78.233f)) * T(43758.5453f)); }

template <class T> void apply_constraints(State<T>& s, T dt) {
    for (size_t k = 0; k < s.fixed.size(); ++k) {
        const int id = s.fixed[k], g = s.fgroup[k];
        s.p[id] = s.off[g] + s.com[g] + s.R[g] * (s.init_p[id] - s.com[g]);
        s.v[id] = V3<T>();
        s.f[id] = V3<T>();
        s.mask[id] = 0;
    }
    // effects after the fixation, in creation order (kernel_constraint_crush / random_sphere /
    // high_stretch, GPU_Constraint.cu:22-92)
    for (auto& e : s.effects) {
        if (!e.active) continue;
        if (e.kind == 2) {
            e.t = std::min(e.t + dt, e.max_dist);
            for (int id : e.ids) {
                if (s.mask[id] == 0) continue;
                const V3<T> d = s.init_p[id] - e.c;
                s.p[id] = s.init_p[id] + d / length(d) * e.t;
            }
            continue;
        }
        for (int i = 0; i < s.n; ++i) {
            if (s.mask[i] == 0) continue;
            if (e.kind == 0) {
                s.p[i].y = T(0);
            } else {
                const V3<T>& x = s.init_p[i];
                const T h = hash1(x.z);
                const T rx = hash2(x.x + h, x.y + h) * T(2) - T(1);
                const T ry = hash1(rx * T(i)) * T(2) - T(1);
                const T rz = hash1(rx * ry) * T(2) - T(1);
                const T r = hash1(rz * rx * ry);
                const V3<T> d(rx, ry, rz);
                s.p[i] = e.c + d / length(d) * (e.radius * r);
            }
            s.last_p[i] = s.p[i];
            s.v[i] = V3<T>();
            s.f[i] = V3<T>();
        }
    }
    if (s.box)
        for (int i = 0; i < s.n; ++i) {
            if (s.mask[i] == 0) continue;
            for (int k = 0; k < 3; ++k) s.p[i][k] = std::min(std::max(s.p[i][k], s.bmin[k]), s.bmax[k]);
        }
}

template <class T> void apply_initial_velocity(State<T>& s, T dt) {
    for (int i = 0; i < s.n; ++i) s.last_p[i] = s.p[i] - s.v[i] * dt;
}

template <class T> void scene_energy(const Fem<T>& f, const State<T>& s, double* parts) {
    double kin = 0, ela = 0, grav = 0;
    for (int i = 0; i < s.n; ++i) {
        kin += 0.5 * (double)s.m[i] * (double)dot(s.v[i], s.v[i]);
        grav -= (double)s.m[i] * (double)dot(s.g, s.p[i]);
    }
    for (int e = 0; e < f.n_elem; ++e)
        for (int q = 0; q < f.nq; ++q)
            ela += (double)energy(f.material, f.lambda[e], f.mu[e], deformation(f, s.p, e, q)) * (double)f.V[e * f.nq + q];
    parts[0] = kin; parts[1] = ela; parts[2] = grav; parts[3] = kin + ela + grav;
}

// ----------------------------------------------------------------------------- GPU-semantics VBD
// Owner lists: per node, (element, local index) in element order.
using Owners = std::vector<std::vector<std::pair<int, int>>>;

template <class T> struct VBD {
    Fem<T> fem;
    State<T> s;
    // multigrid (MG_VBD_FEM, MG_VertexBlockDescent.cpp:134-239): level 1 is the linear mesh of
    // the corners, solved with its own colouring and masses; mid nodes follow by prolongation
    bool mg = false;
    int max_it[2] = {0, 0}, it_count = 0, current = 1;
    Fem<T> fem_lin;
    std::vector<std::vector<int>> by_color_lin;
    Owners owners_lin;
    std::vector<T> m_lin;
    std::vector<int> pro_edge, pro_face, pro_vol;   // (id, 2 / 4 / 8 corner ids) per entry
    int iterations = 1;
    T rho = 0, damping = 0;
    bool in_place = false;
    int n_colors = 0;
    std::vector<std::vector<int>> by_color;                 // ascending vertex ids per colour
    std::vector<std::vector<std::pair<int, int>>> owners;   // (eid, local id), element order
    int order_mode = 0;
    std::mt19937 rng;
    bool first = true;
    bool has_v0 = false;
};

template <class T> void vbd_vertex(const Fem<T>& f, const Owners& owners, const State<T>& s, int vid, T dt, V3<T>& fi,
                                   M3<T>& H);
template <class T> void vbd_vertex(VBD<T>& b, int vid, T dt, V3<T>& fi, M3<T>& H) {
    vbd_vertex(b.fem, b.owners, b.s, vid, dt, fi, H);
}
template <class T> void vbd_vertex(const Fem<T>& f, const Owners& owners, const State<T>& s, int vid, T dt, V3<T>& fi,
                                   M3<T>& H) {
    // kernel_vbd_solve_v3/v4 body: per (owner, qp) compute_f_H_sym (GPU_VBD_FEM.cu:42-63),
    // summed over the vertex's owners in element order and its quadrature points.
    (void)dt;
    fi = V3<T>();
    H = M3<T>(T(0));
    for (auto [eid, r] : owners[vid])
        for (int q = 0; q < f.nq; ++q) {
            const M3<T>& Ji = f.JX_inv[eid * f.nq + q];
            const T V = f.V[eid * f.nq + q];
            M3<T> Jx(T(0));
            for (int i = 0; i < f.ne; ++i) Jx = Jx + outer(s.p[f.topo[eid * f.ne + i]], f.dN[q * f.ne + i]);
            const M3<T> F = Jx * Ji;
            const V3<T> g = transpose(Ji) * f.dN[q * f.ne + r];
            const M3<T> P = pk1(f.material, f.lambda[eid], f.mu[eid], F);
            fi = fi - (P * g) * V;
            M3<T> B[6];
            hessian_sym(f.material, f.lambda[eid], f.mu[eid], F, B);
            H = H + assemble_sym(g, V, B);
        }
}

// compute_correction (GPU_VBD_FEM.cu:107-122)
template <class T> V3<T> vbd_correction(const State<T>& s, int vid, T damping, T dt, V3<T> fi, M3<T> H, T mass = T(-1)) {
    fi = fi - (damping / dt) * H * (s.p[vid] - s.last_p[vid]);
    H = H + (damping / dt) * H;
    const T mh2 = (mass >= T(0) ? mass : s.m[vid]) / (dt * dt);
    fi = fi - mh2 * (s.p[vid] - s.y[vid]);
    H[0][0] += mh2; H[1][1] += mh2; H[2][2] += mh2;
    const T dH = std::abs(det(H));
    return dH > T(1e-6f) ? inverse(H) * fi : V3<T>();
}

// P1_to_P2 / Q1_to_Q2::prolongation (MG_VertexBlockDescent.cpp:37-96): each mid node moves by
// the mean displacement since the sub-step start of its edge / face / element corners.
template <class T> void mg_prolong(VBD<T>& b) {
    State<T>& s = b.s;
    auto apply = [&](const std::vector<int>& list, int k, T w) {
        for (size_t i = 0; i < list.size(); i += k + 1) {
            V3<T> d;
            for (int j = 1; j <= k; ++j) d = d + (s.p[list[i + j]] - s.last_p[list[i + j]]);
            s.p[list[i]] = s.last_p[list[i]] + d * w;
        }
    };
    apply(b.pro_edge, 2, T(0.5f));
    apply(b.pro_face, 4, T(0.25f));
    apply(b.pro_vol, 8, T(0.125f));
}

// Host threads for the vertices of one colour (orc_set_threads).  The vertices of a colour of
// a conflict-free colouring share no element, so each one reads only other colours' positions
// and solving them in any order, or at once, gives the same result bit for bit; with conflicts
// (ColorReduction) the Jacobi path writes p_new and is order-free too.
static int g_threads = 1;
template <class F> static void parallel_for(size_t n, F&& body) {
    const int t = (int)std::min<size_t>((size_t)g_threads, n / 256 + 1);
    if (t <= 1) { for (size_t i = 0; i < n; ++i) body(i); return; }
    std::vector<std::thread> pool;
    const size_t chunk = (n + t - 1) / t;
    for (int k = 0; k < t; ++k)
        pool.emplace_back([&, k]() { for (size_t i = k * chunk; i < std::min(n, (k + 1) * chunk); ++i) body(i); });
    for (auto& th : pool) th.join();
}

// GPU_VBD::step (GPU_VBD.cu:38-61) + GPU_VBD_FEM::step (GPU_VBD_FEM.cu:712-755) for one
// sub-step of length dt.
template <class T> void vbd_substep(VBD<T>& b, T dt) {
    State<T>& s = b.s;
    if (b.first && b.has_v0) apply_initial_velocity(s, dt);
    b.first = false;
    // kernel_integration (GPU_VBD.cu:6-18)
    for (int i = 0; i < s.n; ++i) {
        s.prev_it_p[i] = s.p[i];
        const V3<T> a = s.g + s.f[i] * s.w[i];
        s.y[i] = s.p[i] + ((s.p[i] - s.last_p[i]) * (T(1) / dt) + a * dt) * dt;
        s.last_p[i] = s.p[i];
        s.p[i] = s.y[i];
        s.f[i] = V3<T>();
    }
    T omega = 1;
    std::vector<int> order(b.n_colors);
    for (int j = 0; j < b.iterations; ++j) {
        // multigrid schedule (MG_VBD_FEM::solve): max_it[1] iterations on the linear level,
        // then max_it[0] on the full one, counted across sub-steps; entering the linear level
        // prolongs the mid nodes first
        int level = 0;
        if (b.mg) {
            const int last = b.current;
            b.it_count++;
            while (b.it_count > b.max_it[b.current]) { b.it_count = 1; b.current = (b.current + 1) % 2; }
            level = b.current;
            if (last != level && level == 1) mg_prolong(b);
        }
        const Fem<T>& fl = level ? b.fem_lin : b.fem;
        const Owners& ol = level ? b.owners_lin : b.owners;
        const auto& colours = level ? b.by_color_lin : b.by_color;
        const bool in_place = level ? true : b.in_place;
        order.resize(colours.size());
        std::iota(order.begin(), order.end(), 0);
        if (b.order_mode == 1) std::shuffle(order.begin(), order.end(), b.rng);
        for (int c : order) {
            const std::vector<int>& vs = colours[c];
            if (in_place) {
                parallel_for(vs.size(), [&](size_t k) {
                    const int vid = vs[k];
                    if (s.mask[vid] == 0) return;
                    V3<T> fi; M3<T> H;
                    vbd_vertex(fl, ol, s, vid, dt, fi, H);
                    s.p[vid] = s.p[vid] + vbd_correction(s, vid, b.damping, dt, fi, H, level ? b.m_lin[vid] : T(-1));
                });
            } else {
                parallel_for(vs.size(), [&](size_t k) {
                    const int vid = vs[k];
                    if (s.mask[vid] == 0) return;
                    V3<T> fi; M3<T> H;
                    vbd_vertex(fl, ol, s, vid, dt, fi, H);
                    s.p_new[vid] = s.p[vid] + vbd_correction(s, vid, b.damping, dt, fi, H);
                });
                for (int vid : vs) if (s.mask[vid] != 0) s.p[vid] = s.p_new[vid];   // kernel_copy_in_position
            }
        }
        apply_constraints(s, dt);
        if (b.mg && b.current == 1) mg_prolong(b);   // MG_VertexBlockDescent::step: interpolate after each iteration
        if (b.rho > T(0) && b.rho > T(1.17549435e-38f * 1e6f)) {   // GPU_VBD.cu:50-56
            if (j == 1) omega = T(2) / (T(2) - b.rho * b.rho);
            else if (j > 1) omega = T(4) / (T(4) - b.rho * b.rho * omega);
            for (int i = 0; i < s.n; ++i) {
                if (j >= 2) s.p[i] = s.prev_it2_p[i] + omega * (s.p[i] - s.prev_it2_p[i]);
                s.prev_it2_p[i] = s.prev_it_p[i];
                s.prev_it_p[i] = s.p[i];
            }
        }
    }
    for (int i = 0; i < s.n; ++i) s.v[i] = (s.p[i] - s.last_p[i]) / dt;   // kernel_velocity_update
}

template <class T> VBD<T>* vbd_create(const orc_desc* d) {
    auto* b = new VBD<T>();
    if (!build_fem(d, b->fem)) { delete b; return nullptr; }
    init_state(d, b->s);
    b->iterations = d->iterations;
    b->rho = (T)d->rho;
    b->damping = (T)d->damping;
    b->in_place = d->in_place != 0;
    b->n_colors = d->n_colors;
    b->by_color.assign(d->n_colors, {});
    for (int i = 0; i < d->n_nodes; ++i)
        if (d->colors[i] >= 0 && d->colors[i] < d->n_colors) b->by_color[d->colors[i]].push_back(i);
    // build_owner_data (GPU_VBD_FEM.cu:677-690)
    b->owners.assign(d->n_nodes, {});
    for (int e = 0; e < d->n_elements; ++e)
        for (int j = 0; j < b->fem.ne; ++j) b->owners[d->topology[e * b->fem.ne + j]].push_back({e, j});
    b->order_mode = d->order_mode;
    b->rng.seed((unsigned)d->seed);
    b->has_v0 = d->initial_velocity != nullptr;
    if (d->mg_linear > 0.f) {
        if ((d->element != Tetra10 && d->element != Hexa27) || !d->mg_masses) { delete b; return nullptr; }
        const int nl = d->element == Tetra10 ? 4 : 8, ne = b->fem.ne, E = d->n_elements;
        const int it_lin = (int)((float)d->iterations * d->mg_linear);
        b->mg = true;
        b->max_it[0] = d->iterations - it_lin;
        b->max_it[1] = it_lin;
        std::vector<int32_t> lin((size_t)E * nl);
        for (int e = 0; e < E; ++e) for (int j = 0; j < nl; ++j) lin[(size_t)e * nl + j] = d->topology[(size_t)e * ne + j];
        orc_desc dl = *d;
        dl.element = d->element == Tetra10 ? Tetra : Hexa;
        dl.topology = lin.data();
        if (!build_fem(&dl, b->fem_lin)) { delete b; return nullptr; }
        // colouring of the corner graph: DSAT on the corners numbered in ascending order
        std::vector<int> compact(d->n_nodes, -1), back;
        for (int32_t v : lin) compact[v] = 0;
        for (int i = 0; i < d->n_nodes; ++i) if (compact[i] == 0) { compact[i] = (int)back.size(); back.push_back(i); }
        std::vector<int32_t> lc(lin.size());
        for (size_t k = 0; k < lin.size(); ++k) lc[k] = compact[lin[k]];
        Graph g = build_primal(nl, lc.data(), E);
        std::vector<int> col;
        const int nc = dsat(g, col);
        b->by_color_lin.assign(nc, {});
        for (size_t k = 0; k < back.size(); ++k) b->by_color_lin[col[k]].push_back(back[k]);
        b->owners_lin.assign(d->n_nodes, {});
        for (int e = 0; e < E; ++e) for (int j = 0; j < nl; ++j) b->owners_lin[lin[(size_t)e * nl + j]].push_back({e, j});
        b->m_lin.assign(d->n_nodes, T(0));
        for (int i = 0; i < d->n_nodes; ++i) b->m_lin[i] = (T)d->mg_masses[i];
        // prolongation lists, first visit in element order (P1_to_P2 / Q1_to_Q2 constructors)
        std::vector<char> seen(d->n_nodes, 0);
        const int* t = d->topology;
        if (d->element == Tetra10) {
            static const int ed[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
            for (int e = 0; e < E; ++e)
                for (int j = 4; j < 10; ++j) {
                    const int v = t[e * 10 + j];
                    if (seen[v]) continue;
                    seen[v] = 1;
                    b->pro_edge.insert(b->pro_edge.end(), {v, t[e * 10 + ed[j - 4][0]], t[e * 10 + ed[j - 4][1]]});
                }
        } else {
            // the reference's edge list ends with {7, 0} for node 19 (the edge is 7-4)
            static const int ed[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5}, {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 0}};
            static const int fc[6][4] = {{0, 1, 2, 3}, {0, 1, 4, 5}, {1, 2, 5, 6}, {2, 3, 6, 7}, {3, 0, 7, 4}, {4, 5, 6, 7}};
            for (int e = 0; e < E; ++e) {
                const int* c = t + (size_t)e * 27;
                for (int k = 0; k < 12; ++k) {
                    const int v = c[8 + k];
                    if (seen[v]) continue;
                    seen[v] = 1;
                    b->pro_edge.insert(b->pro_edge.end(), {v, c[ed[k][0]], c[ed[k][1]]});
                }
                for (int k = 0; k < 6; ++k) {
                    const int v = c[20 + k];
                    if (seen[v]) continue;
                    seen[v] = 1;
                    b->pro_face.insert(b->pro_face.end(), {v, c[fc[k][0]], c[fc[k][1]], c[fc[k][2]], c[fc[k][3]]});
                }
                b->pro_vol.push_back(c[26]);
                for (int j = 0; j < 8; ++j) b->pro_vol.push_back(c[j]);
            }
        }
    }
    return b;
}

template <class T> void residual_norms(VBD<T>& b, T dt, double* out) {
    double sum = 0, mx = 0;
    for (int v = 0; v < b.s.n; ++v) {
        if (b.s.mask[v] == 0) continue;
        V3<T> fi; M3<T> H;
        vbd_vertex(b, v, dt, fi, H);
        // kernel_vbd_compute_residual (GPU_VBD_FEM.cu:482-546)
        fi = fi - (b.damping / dt) * H * (b.s.p[v] - b.s.last_p[v]);
        fi = fi - (b.s.m[v] / (dt * dt)) * (b.s.p[v] - b.s.y[v]);
        const double r = std::sqrt((double)dot(fi, fi));
        sum += r;
        mx = std::max(mx, r);
    }
    out[0] = sum; out[1] = mx;
}

template <class T> void residual_vectors(VBD<T>& b, T dt, double* out) {
    for (int v = 0; v < b.s.n; ++v) {
        V3<T> fi;
        if (b.s.mask[v] != 0) {   // kernel_vbd_compute_residual writes r only for unmasked vertices
            M3<T> H;
            vbd_vertex(b, v, dt, fi, H);
            fi = fi - (b.damping / dt) * H * (b.s.p[v] - b.s.last_p[v]);
            fi = fi - (b.s.m[v] / (dt * dt)) * (b.s.p[v] - b.s.y[v]);
        }
        out[3 * v] = fi.x; out[3 * v + 1] = fi.y; out[3 * v + 2] = fi.z;
    }
}

// Per-element diagnostics of GPU_FEM (GPU_FEM.cu:20-107) on absolute positions.
//   kind 0 stress   sum_q von_mises(P F^T / det F) V_q with F_q = Jx_q JX_inv_q
//   kind 4 stress   the same with Jx accumulated over the quadrature points, as
//                   kernel_compute_stress (:20-43) does (it never resets Jx)
//                   (materials without a VBD stress, Corotated and FixedCorotated, give P = 0)
//   kind 1 volume   kernel_compute_volume (:45-64): sum_q |det Jx_q| w_q
//   kind 2 diff     kernel_compute_volume_diff (:66-85): sum_q (|det Jx_q| w_q - V_q)
//   kind 5 volume   kind 1 with Jx accumulated over the quadrature points as in kind 4, the form
//                   of the "volume" field of the reference's result files
//                   (assets/result/vtk/References/*.vtk)
//   kind 6 diff     kind 2 with the same accumulation (their "volume_diff" field)
//   kind 3 inverted kernel_compute_inverted (:87-107): 1 when sum_q det(Jx_q JX_inv_q) w_q < -1e-6
//                   (the kernel indexes JX_inv[eid + qid], outside the element's records and,
//                   for eid >= E Q / (Q + 1), outside the buffer; the record of q is used here)
template <class T> void element_data(const Fem<T>& f, const State<T>& s, int kind, double* out) {
    for (int e = 0; e < f.n_elem; ++e) {
        const int* topo = &f.topo[(size_t)e * f.ne];
        T acc = 0;
        M3<T> Jacc(T(0));
        for (int q = 0; q < f.nq; ++q) {
            M3<T> Jx(T(0));
            for (int i = 0; i < f.ne; ++i) Jx = Jx + outer(s.p[topo[i]], f.dN[q * f.ne + i]);
            const M3<T>& Ji = f.JX_inv[(size_t)e * f.nq + q];
            const T Vq = f.V[(size_t)e * f.nq + q];
            if (kind == 0 || kind == 4) {
                Jacc = Jacc + Jx;
                const M3<T> F = (kind == 4 ? Jacc : Jx) * Ji;
                const M3<T> P = f.material > StableNeoHooke ? M3<T>(T(0)) : pk1(f.material, f.lambda[e], f.mu[e], F);
                const M3<T> C = P * transpose(F) * (T(1) / det(F));   // pk1_to_cauchy_stress
                const T s01 = C[0][0] - C[1][1], s12 = C[1][1] - C[2][2], s02 = C[0][0] - C[2][2];
                T vm = T(0.5) * (s01 * s01 + s12 * s12 + s02 * s02);   // von_mises_stress (GPU_FEM_Material.cu:223-230)
                vm += T(3) * (C[0][1] * C[0][1] + C[1][2] * C[1][2] + C[0][2] * C[0][2]);
                acc += std::sqrt(vm) * Vq;
            } else if (kind == 1) {
                acc += std::fabs(det(Jx)) * f.weights[q];
            } else if (kind == 2) {
                acc += std::fabs(det(Jx)) * f.weights[q] - Vq;
            } else if (kind == 5 || kind == 6) {
                Jacc = Jacc + Jx;
                acc += std::fabs(det(Jacc)) * f.weights[q] - (kind == 6 ? Vq : T(0));
            } else {
                acc += det(Jx * Ji) * f.weights[q];
            }
        }
        out[e] = kind == 3 ? (acc > T(-1e-6) ? 0.0 : 1.0) : (double)acc;
    }
}

// ----------------------------------------------------------------------------- reference CPU VBD
// VertexBlockDescent::step (VertexBlockDescent.cpp:28-44), VBD_FEM::compute_inertia
// (VBD_FEM.cpp:13-18), solve (:47-57), solve_vertex (:61-85), solve_element (:87-110),
// assemble_hessian (:240-254), plot_residual/compute_forces (:113-158), chebyshev
// (VertexBlockDescent.cpp:12-26), RB_Fixation (Constraint.cpp:20-37), EulerSemiExplicit
// (Solver.cpp:12-18).  FP32 throughout, single thread, Stable Neo-Hookean sub-Hessian as
// M_Stable_NeoHooke::get_sub_hessian (FEM_ContinuousMaterial.cpp:89-116).
struct CpuVBD {
    Fem<float> fem;
    int n = 0;
    std::vector<V3<float>> p, last_p, init_p, v, y, prev_x, prev_prev_x;
    std::vector<float> m;
    std::vector<char> active;
    std::vector<int> fixed;
    V3<float> com, g;
    std::vector<std::vector<std::pair<int, int>>> owners;
    int iterations = 1;
    float rho = 0, damping = 0;
};

static void cpu_sub_hessian(int mat, float lambda, float mu, const M3<float>& F, M3<float> B[9]) {
    // full 9-block form; the 6 distinct blocks equal hessian_sym's, mirrored
    M3<float> S[6];
    hessian_sym<float>(mat, lambda, mu, F, S);
    B[0] = S[0]; B[1] = S[1]; B[2] = S[2]; B[4] = S[3]; B[5] = S[4]; B[8] = S[5];
    if (mat == StVK || mat == Hooke) { B[3] = S[1]; B[6] = S[2]; B[7] = S[4]; }
    else {
        // hat blocks are antisymmetric in the 9-block layout (FEM_ContinuousMaterial.cpp:95-103)
        const M3<float> cF = com(F);
        const float alpha = mat == NeoHooke ? 1.f : 1.f + mu / lambda;
        const float s = lambda * (det(F) - alpha);
        B[3] = -(hat(F[2]) * s); B[6] = hat(F[1]) * s; B[7] = -(hat(F[0]) * s);
        B[3] = B[3] + outer(cF[0], cF[1]) * lambda;
        B[6] = B[6] + outer(cF[0], cF[2]) * lambda;
        B[7] = B[7] + outer(cF[1], cF[2]) * lambda;
    }
}

static M3<float> cpu_assemble(const M3<float> B[9], V3<float> g) {
    M3<float> H(0.f);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            M3<float> Hkl;
            for (int l = 0; l < 3; ++l) for (int k = 0; k < 3; ++k) Hkl[k][l] = B[k + l * 3][i][j];
            H[i][j] = dot(g, Hkl * g);
        }
    return H;
}

static void cpu_vbd_substep(CpuVBD& c, float dt, bool residual_pass) {
    const Fem<float>& f = c.fem;
    for (int i = 0; i < c.n; ++i) c.y[i] = c.p[i] + c.v[i] * dt + c.g * dt * dt;   // compute_inertia
    for (int i = 0; i < c.n; ++i) {                                               // step_solver
        c.last_p[i] = c.p[i];
        if (!c.active[i]) continue;
        c.v[i] = c.v[i] + c.g * dt;
        c.p[i] = c.p[i] + c.v[i] * dt;
    }
    float omega = 0;
    for (int j = 0; j < c.iterations; ++j) {
        for (int vid = 0; vid < c.n; ++vid) {
            if (!c.active[vid]) continue;
            V3<float> fi; M3<float> H(0.f);
            for (auto [eid, r] : c.owners[vid])
                for (int q = 0; q < f.nq; ++q) {
                    M3<float> Jx(0.f);
                    for (int i = 0; i < f.ne; ++i) Jx = Jx + outer(c.p[f.topo[eid * f.ne + i]], f.dN[q * f.ne + i]);
                    const M3<float> F = Jx * f.JX_inv[eid * f.nq + q];
                    const V3<float> g = transpose(f.JX_inv[eid * f.nq + q]) * f.dN[q * f.ne + r];
                    const M3<float> P = pk1<float>(f.material, f.lambda[eid], f.mu[eid], F);
                    fi = fi - (P * g) * f.V[eid * f.nq + q];
                    M3<float> B[9];
                    cpu_sub_hessian(f.material, f.lambda[eid], f.mu[eid], F, B);
                    H = H + cpu_assemble(B, g) * f.V[eid * f.nq + q];
                }
            fi = fi - (c.damping / dt) * H * (c.p[vid] - c.last_p[vid]);
            H = H + (c.damping / dt) * H;
            fi = fi - (c.m[vid] / (dt * dt)) * (c.p[vid] - c.y[vid]);
            H = H + M3<float>(c.m[vid] / (dt * dt));
            const float dH = std::abs(det(H));
            if (dH > 1.17549435e-38f * 1e6f) c.p[vid] = c.p[vid] + inverse(H) * fi;
        }
        if (residual_pass) {   // plot_residual -> compute_forces, a full force pass
            std::vector<V3<float>> forces(c.n);
            for (int e = 0; e < f.n_elem; ++e)
                for (int q = 0; q < f.nq; ++q) {
                    M3<float> Jx(0.f);
                    for (int i = 0; i < f.ne; ++i) Jx = Jx + outer(c.p[f.topo[e * f.ne + i]], f.dN[q * f.ne + i]);
                    const M3<float>& Ji = f.JX_inv[e * f.nq + q];
                    const M3<float> P = pk1<float>(f.material, f.lambda[e], f.mu[e], Jx * Ji) * transpose(Ji) * f.V[e * f.nq + q];
                    for (int i = 0; i < f.ne; ++i) forces[f.topo[e * f.ne + i]] = forces[f.topo[e * f.ne + i]] - P * f.dN[q * f.ne + i];
                }
            float sum = 0;
            for (int i = 0; i < c.n; ++i) {
                forces[i] = forces[i] - (c.m[i] / (dt * dt)) * (c.p[i] - c.y[i]);
                if (c.active[i]) sum += length(forces[i]);
            }
            volatile float sink = sum; (void)sink;
        }
        for (int id : c.fixed) {   // RB_Fixation::apply, stiffness 1
            const V3<float> target = V3<float>() + c.com + M3<float>(1.f) * (c.init_p[id] - c.com);
            c.p[id] = c.p[id] + (target - c.p[id]) * 1.f;
            c.v[id] = V3<float>();
        }
        // chebyshev_acceleration with compute_omega (VertexBlockDescent.h:14-18)
        omega = j == 0 ? 1.f : (j == 1 ? 2.f / (2.f - c.rho * c.rho) : 4.f / (4.f - c.rho * c.rho * omega));
        for (int i = 0; i < c.n; ++i) {
            if (!c.active[i]) continue;
            if (j >= 2) c.p[i] = omega * (c.p[i] - c.prev_prev_x[i]) + c.prev_prev_x[i];
            c.prev_prev_x[i] = c.prev_x[i];
            c.prev_x[i] = c.p[i];
        }
    }
    for (int i = 0; i < c.n; ++i) if (c.active[i]) c.v[i] = (c.p[i] - c.last_p[i]) / dt;
}

// ----------------------------------------------------------------------------- XPBD
// GPU_PBD::step (GPU_PBD.cu:20-26): semi-implicit predictor (GPU_Integrator.cu:27-34), one
// pass over the element colours (Greedy_SLF on the vertex-dual graph) with kernel_XPBD_V0
// (GPU_PBD_FEM.cu:60-93), the constraints, then kernel_velocity_update with global damping
// (GPU_PBD.cu:8-18).  Constraint pairs per material: eval_material (GPU_PBD_FEM_Materials.cu:97-117).
// Rotation part of F by the quaternion iteration of Mueller et al., "A Robust Method to
// Extract the Rotational Part of Deformations" (MIG 2016), as mat3x3_polardecomposition
// (CUMatrix.cu:75-96) runs it: R starts at the identity, at most 10 iterations, stop when
// |omega| < 1e-8, omega = sum_i R_i x F_i * (1/|sum_i R_i . F_i| + 1e-9); S = R^T F.
template <class T> void polar(const M3<T>& F, M3<T>& R, M3<T>& S) {
    T qw = 1, qx = 0, qy = 0, qz = 0;
    R = M3<T>(T(1));
    for (int it = 0; it < 10; ++it) {
        const T den = T(1) / std::fabs(dot(R[0], F[0]) + dot(R[1], F[1]) + dot(R[2], F[2])) + T(1e-9);
        const V3<T> om = (cross(R[0], F[0]) + cross(R[1], F[1]) + cross(R[2], F[2])) * den;
        const T w = length(om);
        if (w < T(1e-8)) break;
        const V3<T> a = om / w;   // dq = (cos(w/2), a sin(w/2)); q = dq q; q /= |q|
        const T c = std::cos(w * T(0.5)), sn = std::sin(w * T(0.5));
        const T dw = c, dx = a.x * sn, dy = a.y * sn, dz = a.z * sn;
        const T nw = dw * qw - dx * qx - dy * qy - dz * qz;
        const T nx = dw * qx + dx * qw + dy * qz - dz * qy;
        const T ny = dw * qy - dx * qz + dy * qw + dz * qx;
        const T nz = dw * qz + dx * qy - dy * qx + dz * qw;
        const T inv = T(1) / std::sqrt(nw * nw + nx * nx + ny * ny + nz * nz);
        qw = nw * inv; qx = nx * inv; qy = ny * inv; qz = nz * inv;
        // rotation matrix of the unit quaternion, column-major
        R[0] = {T(1) - T(2) * (qy * qy + qz * qz), T(2) * (qx * qy + qw * qz), T(2) * (qx * qz - qw * qy)};
        R[1] = {T(2) * (qx * qy - qw * qz), T(1) - T(2) * (qx * qx + qz * qz), T(2) * (qy * qz + qw * qx)};
        R[2] = {T(2) * (qx * qz + qw * qy), T(2) * (qy * qz - qw * qx), T(1) - T(2) * (qx * qx + qy * qy)};
    }
    S = transpose(R) * F;
}

template <class T> void xpbd_pair(int mat, int m, T lambda, T mu, const M3<T>& F, M3<T>& P, T& C) {
    const M3<T> I(T(1));
    if (mat == Corotated || mat == FixedCorotated) {   // GPU_PBD_FEM_Materials.cu:67-95
        M3<T> R, S;
        polar(F, R, S);
        if (mat == Corotated) {
            if (m == 0) { C = squared_trace(S - I); P = R * (T(2) * trace(S - I) * I); }
            else { C = squared_norm(S); P = R * (T(2) * S - I); }
        } else {
            if (m == 0) { const T d = det(S) - T(1); C = d * d; P = R * (T(2) * d * com(S)); }
            else { C = T(2) * squared_norm(S); P = R * (T(4) * (S - I)); }
        }
    } else if (mat == Hooke) {
        if (m == 0) { const T tr = trace(T(0.5) * (transpose(F) + F) - I); C = tr * tr; P = T(2) * tr * I; }
        else { const M3<T> E = T(0.5) * (transpose(F) + F) - I; C = T(2) * squared_trace(E); P = T(4) * E; }
    } else if (mat == StVK) {
        if (m == 0) { const T tr = trace(T(0.5) * (transpose(F) * F - I)); C = tr * tr; P = T(2) * tr * F; }
        else { const M3<T> E = T(0.5) * (transpose(F) * F - I); P = T(4) * F * E; C = T(2) * squared_trace(E); }
    } else {
        const bool nh = mat == NeoHooke;   // NeoHooke -> snh pair, Stable_NeoHooke -> dsnh pair
        if (m == 0) {
            const T alpha = nh ? T(1) + mu / lambda : T(1);
            const T d = det(F) - alpha;
            C = d * d;
            P = T(2) * d * com(F);
        } else if (nh) { C = squared_norm(F) - T(3); P = T(2) * F; }
        else { C = squared_norm(F) - T(3) - T(2) * (det(F) - T(1)); P = T(2) * F - T(2) * com(F); }
    }
}

template <class T> struct XPBD {
    Fem<T> fem;
    State<T> s;
    T global_damping = 0;
    int version = 2;   // XPBD_FEM_VERSION: 0 XPBD, 1 Quadrature, 2 OptiShared, 3 OptiGroup
    std::vector<std::vector<int>> by_color;   // element ids per colour, ascending
    bool first = true, has_v0 = false;
};

template <class T> void xpbd_substep(XPBD<T>& x, T dt) {
    State<T>& s = x.s;
    const Fem<T>& f = x.fem;
    for (int i = 0; i < s.n; ++i) {   // kenerl_semi_exicit_integration
        s.last_p[i] = s.p[i];
        s.v[i] = s.v[i] + (s.g + s.f[i] * s.w[i]) * dt;
        s.p[i] = s.p[i] + s.v[i] * dt;
        s.f[i] = V3<T>();
    }
    std::vector<V3<T>> grad(f.ne);
    // GPU_PBD_FEM::step (:661-689): Tetra4 and version XPBD run kernel_XPBD_V0 (normalised
    // constraint sqrt|C|, masked update); Quadrature and OptiShared run kernel_XPBD_V1/V2
    // (:141-263: raw C, alpha = 4C/(k dt^2), beta = -2C/(S + alpha), no mask); OptiGroup
    // launches nothing for other elements.
    const bool v0 = f.ne == 4 || x.version == 0;
    if (!v0 && x.version != 1 && x.version != 2) x.by_color.clear();
    for (const auto& els : x.by_color)
        for (int eid : els) {
            const int* topo = &f.topo[eid * f.ne];
            for (int m = 0; m < 2; ++m) {
                T C = 0;
                for (int i = 0; i < f.ne; ++i) grad[i] = V3<T>();
                for (int q = 0; q < f.nq; ++q) {   // xpbd_constraint_fem_eval (:30-47)
                    const M3<T>& Ji = f.JX_inv[eid * f.nq + q];
                    const T V = f.V[eid * f.nq + q];
                    M3<T> Jx(T(0));
                    for (int i = 0; i < f.ne; ++i) Jx = Jx + outer(s.p[topo[i]], f.dN[q * f.ne + i]);
                    M3<T> P; T en;
                    xpbd_pair(f.material, m, f.lambda[eid], f.mu[eid], Jx * Ji, P, en);
                    P = P * transpose(Ji) * V;
                    C += en * V;
                    for (int i = 0; i < f.ne; ++i) grad[i] = grad[i] + P * f.dN[q * f.ne + i];
                }
                if (!v0) {
                    T S = 0;
                    for (int i = 0; i < f.ne; ++i) S += dot(grad[i], grad[i]) * s.w[topo[i]];
                    const T k = m == 0 ? f.lambda[eid] : f.mu[eid];
                    const T alpha = T(4) * C / (k * dt * dt);
                    const T beta = C < T(1e-12) ? T(0) : -T(2) * C / (S + alpha);
                    for (int i = 0; i < f.ne; ++i) {
                        const int vid = topo[i];
                        s.p[vid] = s.p[vid] + beta * s.w[vid] * grad[i];
                    }
                    continue;
                }
                C = C < T(0) ? -C : C;   // xpbd_convert_to_constraint (:49-58)
                C = std::sqrt(C);
                const T Ci = C < T(1e-12) ? T(0) : T(1) / (T(2) * C);
                for (int i = 0; i < f.ne; ++i) grad[i] = grad[i] * Ci;
                T sum = 0;   // xpbd_solve (:13-28)
                for (int i = 0; i < f.ne; ++i) sum += dot(grad[i], grad[i]) * s.w[topo[i]];
                const T k = m == 0 ? f.lambda[eid] : f.mu[eid];
                const T alpha = T(1) / (k * dt * dt);
                const T dl = -C / (sum + alpha);
                for (int i = 0; i < f.ne; ++i) {
                    const int vid = topo[i];
                    if (s.mask[vid] == 0) continue;
                    s.p[vid] = s.p[vid] + dl * s.w[vid] * grad[i];
                }
            }
        }
    apply_constraints(s, dt);
    for (int i = 0; i < s.n; ++i) {
        s.v[i] = (s.p[i] - s.last_p[i]) / dt;
        const T nv = length(s.v[i]);
        if (nv > T(1e-7)) {
            const T coef = x.global_damping * dt * s.w[i];
            const T dmp = -nv * (coef > T(1) ? T(1) : coef);
            s.v[i] = s.v[i] + (s.v[i] / nv) * dmp;
        }
    }
}

// ----------------------------------------------------------------------------- explicit
// GPU_SemiExplicit::step (GPU_Integrator.cu:36-42): kernel_fem_eval_force
// (GPU_FEM_Explicit.cu:5-64) writes f[v] = sum_(e,q) (-P dF/dx V - k_d H v[v]), then the
// semi-implicit update and the constraints.
template <class T> struct Explicit {
    Fem<T> fem;
    State<T> s;
    T damping = 0;
    std::vector<std::vector<std::pair<int, int>>> owners;
};

template <class T> void explicit_substep(Explicit<T>& x, T dt) {
    State<T>& s = x.s;
    const Fem<T>& f = x.fem;
    for (int vid = 0; vid < s.n; ++vid) {
        V3<T> acc;
        for (auto [eid, r] : x.owners[vid])
            for (int q = 0; q < f.nq; ++q) {
                const M3<T>& Ji = f.JX_inv[eid * f.nq + q];
                const T V = f.V[eid * f.nq + q];
                M3<T> Jx(T(0));
                for (int i = 0; i < f.ne; ++i) Jx = Jx + outer(s.p[f.topo[eid * f.ne + i]], f.dN[q * f.ne + i]);
                const M3<T> F = Jx * Ji;
                const M3<T> P = pk1(f.material, f.lambda[eid], f.mu[eid], F);
                const V3<T> g = transpose(Ji) * f.dN[q * f.ne + r];
                V3<T> fi = -(P * g) * V;
                M3<T> B[6];
                hessian_sym(f.material, f.lambda[eid], f.mu[eid], F, B);
                const M3<T> H = assemble_sym(g, V, B);
                fi = fi - x.damping * H * s.v[vid];
                acc = acc + fi;
            }
        s.f[vid] = acc;
    }
    for (int i = 0; i < s.n; ++i) {
        s.last_p[i] = s.p[i];
        s.v[i] = s.v[i] + (s.g + s.f[i] * s.w[i]) * dt;
        s.p[i] = s.p[i] + s.v[i] * dt;
        s.f[i] = V3<T>();
    }
    apply_constraints(s, dt);
}

template <class T> int get_state(const State<T>& s, int what, double* out) {
    const std::vector<V3<T>>* src = nullptr;
    switch (what) {
        case 0: src = &s.p; break; case 1: src = &s.v; break; case 2: src = &s.last_p; break; case 3: src = &s.y; break;
        case 4: for (int i = 0; i < s.n; ++i) out[i] = s.mask[i]; return 0;
        default: return -1;
    }
    for (int i = 0; i < s.n; ++i) for (int k = 0; k < 3; ++k) out[3 * i + k] = (double)(*src)[i][k];
    return 0;
}

template <class T> int set_state(State<T>& s, int what, const double* in) {
    std::vector<V3<T>>* dst = nullptr;
    switch (what) { case 0: dst = &s.p; break; case 1: dst = &s.v; break; case 2: dst = &s.last_p; break;
                 case 3: dst = &s.y; break; default: return -1; }
    for (int i = 0; i < s.n; ++i) for (int k = 0; k < 3; ++k) (*dst)[i][k] = (T)in[3 * i + k];
    return 0;
}

struct Handle {
    int kind;   // 0 vbd f32, 1 vbd f64, 2 xpbd f32, 3 xpbd f64, 4 explicit f32, 5 explicit f64
    void* ptr;
};

template <class T> XPBD<T>* xpbd_create_t(const orc_desc* d) {
    auto* x = new XPBD<T>();
    if (!build_fem(d, x->fem)) { delete x; return nullptr; }
    init_state(d, x->s);
    x->global_damping = (T)d->global_damping;
    x->version = d->xpbd_version;
    std::vector<int> c;
    Graph g = build_dual_vertex(x->fem.ne, d->topology, d->n_elements);
    const int nc = greedy_slf(g, c);
    x->by_color.assign(nc, {});
    for (int e = 0; e < d->n_elements; ++e) x->by_color[c[e]].push_back(e);   // build_thread_by_color
    return x;
}

template <class T> Explicit<T>* explicit_create_t(const orc_desc* d) {
    auto* x = new Explicit<T>();
    if (!build_fem(d, x->fem)) { delete x; return nullptr; }
    init_state(d, x->s);
    x->damping = (T)d->damping;
    x->owners.assign(d->n_nodes, {});
    for (int e = 0; e < d->n_elements; ++e)
        for (int j = 0; j < x->fem.ne; ++j) x->owners[d->topology[e * x->fem.ne + j]].push_back({e, j});
    return x;
}

template <class T> void set_fix(State<T>& s, int g, const float* off, const float* rot) {
    if (off) s.off[g] = {(T)off[0], (T)off[1], (T)off[2]};
    if (rot) for (int j = 0; j < 3; ++j) s.R[g][j] = {(T)rot[3 * j], (T)rot[3 * j + 1], (T)rot[3 * j + 2]};
}

template <class T> int add_effect(State<T>& s, int kind, const float* params, const int32_t* ids, int n_ids) {
    typename State<T>::Effect e{};
    e.kind = kind;
    e.active = false;
    // centre: (sum of the positions after the first) / count, in FP32 as the constructors
    float cx = 0.f, cy = 0.f, cz = 0.f;
    for (int i = 1; i < s.n; ++i) { cx += (float)s.init_p[i].x; cy += (float)s.init_p[i].y; cz += (float)s.init_p[i].z; }
    const float inv = 1.f / (float)s.n;
    e.c = {(T)(cx * inv), (T)(cy * inv), (T)(cz * inv)};
    e.radius = kind == 1 ? (T)params[0] : T(0);
    e.max_dist = kind == 2 ? (T)params[1] : T(0);
    e.t = T(0);
    if (kind == 2) e.ids.assign(ids, ids + n_ids);
    s.effects.push_back(e);
    return (int)s.effects.size() - 1;
}
template <class T> State<T>* state_of(Handle* h) {
    switch (h->kind) {
        case 0: case 1: return &((VBD<T>*)h->ptr)->s;
        case 2: case 3: return &((XPBD<T>*)h->ptr)->s;
        default: return &((Explicit<T>*)h->ptr)->s;
    }
}

}  // namespace orc

using namespace orc;

extern "C" {

int orc_elem_nodes(int e) { return nodes_of(e); }

int orc_polar(const double* F9, int fp64, double* R9, double* S9) {
    if (!F9) return -1;
    auto run = [&](auto zero) {
        using T = decltype(zero);
        M3<T> F, R, S;
        for (int j = 0; j < 3; ++j) F[j] = {(T)F9[3 * j], (T)F9[3 * j + 1], (T)F9[3 * j + 2]};
        polar(F, R, S);
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                if (R9) R9[3 * j + i] = R[j][i];
                if (S9) S9[3 * j + i] = S[j][i];
            }
    };
    if (fp64) run(0.0); else run(0.0f);
    return 0;
}

int orc_xpbd_pair(int material, int m, double lambda, double mu, const double* F9, double* P9, double* C) {
    if (!F9 || material < Hooke || material > FixedCorotated || m < 0 || m > 1) return -1;
    M3<double> F, P;
    for (int j = 0; j < 3; ++j) F[j] = {F9[3 * j], F9[3 * j + 1], F9[3 * j + 2]};
    double c = 0;
    xpbd_pair(material, m, lambda, mu, F, P, c);
    for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) if (P9) P9[3 * j + i] = P[j][i];
    if (C) *C = c;
    return 0;
}

int orc_beam_counts(int e, int nx, int ny, int nz, int* n_nodes, int* n_elements) {
    Mesh m;
    float d[3] = {1, 1, 1};
    if (orc_beam_mesh(e, nx, ny, nz, d[0], d[1], d[2], 0, 0, 0, nullptr, nullptr) < 0) return -1;
    // sizes computed by building the mesh: cheap for the sizes tests use
    const bool tetra = (e == Tetra || e == Tetra10 || e == Tetra20);
    beam_linear(tetra, nx, ny, nz, 1, 1, 1, {0, 0, 0}, m);
    if (e == Tetra10) to_tetra10(m);
    if (e == Tetra20) to_tetra20(m);
    if (e == Hexa27) to_hexa27(m);
    *n_nodes = (int)m.X.size();
    *n_elements = (int)(m.topo.size() / nodes_of(e));
    return 0;
}

int orc_beam_mesh(int e, int nx, int ny, int nz, float sx, float sy, float sz, float ox, float oy, float oz,
                  float* positions, int32_t* topology) {
    if (nodes_of(e) < 0 || e == Pyramid || e == Prism || nx < 1 || ny < 1 || nz < 1) return -1;
    if (!positions) return 0;
    Mesh m;
    const bool tetra = (e == Tetra || e == Tetra10 || e == Tetra20);
    beam_linear(tetra, nx, ny, nz, sx, sy, sz, {ox, oy, oz}, m);
    if (e == Tetra10) to_tetra10(m);
    if (e == Tetra20) to_tetra20(m);
    if (e == Hexa27) to_hexa27(m);
    for (size_t i = 0; i < m.X.size(); ++i) { positions[3 * i] = m.X[i].x; positions[3 * i + 1] = m.X[i].y; positions[3 * i + 2] = m.X[i].z; }
    std::copy(m.topo.begin(), m.topo.end(), topology);
    return 0;
}

int orc_shape(int e, int* nq, double* coords, double* weights, double* dN) {
    Shape s;
    if (!build_shape(e, s)) return -1;
    *nq = s.nq;
    if (coords) std::copy(s.qp.begin(), s.qp.end(), coords);
    if (weights) std::copy(s.w.begin(), s.w.end(), weights);
    if (dN) std::copy(s.dN.begin(), s.dN.end(), dN);
    return 0;
}

// compute_fem_mass (FEM_Shape.cpp:86-121) with FEM_Generic::compute_volume (FEM_Generic.cpp:25-36)
int orc_masses(int e, const float* X, int n, const int32_t* topo, int n_elem, float density, int distrib, float* mass) {
    Shape s;
    if (!build_shape(e, s)) return -1;
    const int ne = s.nb;
    std::vector<V3<float>> dN(s.nq * ne);
    for (int q = 0; q < s.nq; ++q) for (int i = 0; i < ne; ++i)
        dN[q * ne + i] = {(float)s.dN[(q * ne + i) * 3], (float)s.dN[(q * ne + i) * 3 + 1], (float)s.dN[(q * ne + i) * 3 + 2]};
    auto volume = [&](int el) {
        float vol = 0;
        for (int q = 0; q < s.nq; ++q) {
            M3<float> J(0.f);
            for (int k = 0; k < ne; ++k) {
                const float* x = X + 3 * topo[el * ne + k];
                J = J + outer(V3<float>(x[0], x[1], x[2]), dN[q * ne + k]);
            }
            vol += std::abs(det(J)) * (float)s.w[q];
        }
        return vol;
    };
    for (int i = 0; i < n; ++i) mass[i] = 0.f;
    if (distrib == 1) {
        const float vd = density / (float)ne;
        for (int el = 0; el < n_elem; ++el) {
            const float V = volume(el);
            for (int j = 0; j < ne; ++j) mass[topo[el * ne + j]] += vd * V;
        }
    } else {
        float pm = 0;
        for (int el = 0; el < n_elem; ++el) pm += volume(el);
        pm *= density;
        pm /= (float)n;
        for (int i = 0; i < n; ++i) mass[i] = pm;
    }
    return 0;
}

int orc_precompute(int e, const float* X, const int32_t* topo, int n_elem, int fp64, double* JX, double* Vout) {
    orc_desc d;
    std::memset(&d, 0, sizeof(d));
    d.element = e; d.positions = X; d.topology = topo; d.n_elements = n_elem; d.young = 1; d.poisson = 0.3f;
    auto dump = [&](auto& f) {
        for (size_t k = 0; k < f.JX_inv.size(); ++k) {
            for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) JX[9 * k + 3 * j + i] = (double)f.JX_inv[k][j][i];
            Vout[k] = (double)f.V[k];
        }
    };
    if (fp64) { Fem<double> f; if (!build_fem(&d, f)) return -1; dump(f); }
    else { Fem<float> f; if (!build_fem(&d, f)) return -1; dump(f); }
    return 0;
}

int orc_colour(int e, const int32_t* topo, int n_elem, int n_nodes, int algo, int target, int32_t* colors, int32_t* nb) {
    const int ne = nodes_of(e);
    if (ne < 0 || n_elem <= 0) return -1;
    std::vector<int> c;
    int nc;
    if (algo == 2) {
        Graph g = build_dual_vertex(ne, topo, n_elem);
        nc = greedy_slf(g, c);
    } else {
        Graph g = build_primal(ne, topo, n_elem);
        if (g.n != n_nodes) return -2;
        if (algo == 0) nc = dsat(g, c);
        else { nc = 0; c.assign(g.n, -1); for (int i = 0; i < g.n; ++i) greedy_pick(g, i, nc, c); }
        if (target >= 0) { color_reduction(g, c, target); nc = target; }
    }
    std::copy(c.begin(), c.end(), colors);
    *nb = nc;
    return 0;
}

// GraphColoration::Get_Conflict summed (Graph.h:863-881): each same-colour adjacency counts
// for both ends, per multiset occurrence.
int orc_conflicts(int e, const int32_t* topo, int n_elem, int n_nodes, const int32_t* colors) {
    Graph g = build_primal(nodes_of(e), topo, n_elem);
    (void)n_nodes;
    long long total = 0;
    for (int i = 0; i < g.n; ++i)
        for (int nbh : g.adj[i]) if (colors[nbh] == colors[i]) total += 2;
    return (int)total;
}

void* orc_vbd_create(const orc_desc* d, int fp64) {
    if (!d || !d->colors || !d->masses || d->material > StableNeoHooke) return nullptr;
    Handle* h = new Handle();
    h->kind = fp64 ? 1 : 0;
    h->ptr = fp64 ? (void*)vbd_create<double>(d) : (void*)vbd_create<float>(d);
    if (!h->ptr) { delete h; return nullptr; }
    return h;
}

int orc_vbd_step(void* hv, float frame_dt, int substeps) {
    Handle* h = (Handle*)hv;
    if (!h || substeps <= 0) return -1;
    const float sub = frame_dt / (float)substeps;
    for (int k = 0; k < substeps; ++k) {
        if (h->kind == 1) vbd_substep(*(VBD<double>*)h->ptr, (double)sub);
        else vbd_substep(*(VBD<float>*)h->ptr, sub);
    }
    return 0;
}

int orc_add_effect(void* hv, int kind, const float* params, const int32_t* ids, int n_ids) {
    Handle* h = (Handle*)hv;
    if (!h || kind < 0 || kind > 2 || (kind > 0 && !params) || (kind == 2 && n_ids > 0 && !ids)) return -1;
    const bool fp64 = h->kind % 2 == 1;
    return fp64 ? add_effect(*state_of<double>(h), kind, params, ids, n_ids) : add_effect(*state_of<float>(h), kind, params, ids, n_ids);
}

int orc_set_effect_active(void* hv, int index, int active) {
    Handle* h = (Handle*)hv;
    if (!h) return -1;
    if (h->kind % 2 == 1) {
        auto& v = state_of<double>(h)->effects;
        if (index < 0 || index >= (int)v.size()) return -1;
        v[index].active = active != 0;
    } else {
        auto& v = state_of<float>(h)->effects;
        if (index < 0 || index >= (int)v.size()) return -1;
        v[index].active = active != 0;
    }
    return 0;
}

int orc_set_fixation(void* hv, int g, const float* off, const float* rot) {
    Handle* h = (Handle*)hv;
    if (!h || g < 0 || g > 3) return -1;
    switch (h->kind) {
        case 0: set_fix(((VBD<float>*)h->ptr)->s, g, off, rot); break;
        case 1: set_fix(((VBD<double>*)h->ptr)->s, g, off, rot); break;
        case 2: set_fix(((XPBD<float>*)h->ptr)->s, g, off, rot); break;
        case 3: set_fix(((XPBD<double>*)h->ptr)->s, g, off, rot); break;
        case 4: set_fix(((Explicit<float>*)h->ptr)->s, g, off, rot); break;
        case 5: set_fix(((Explicit<double>*)h->ptr)->s, g, off, rot); break;
        default: return -1;
    }
    return 0;
}

int orc_vbd_get(void* hv, int what, double* out) {
    Handle* h = (Handle*)hv;
    return h->kind == 1 ? get_state(((VBD<double>*)h->ptr)->s, what, out) : get_state(((VBD<float>*)h->ptr)->s, what, out);
}
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

int orc_vbd_set(void* hv, int what, const double* in) {
    Handle* h = (Handle*)hv;
    return h->kind == 1 ? set_state(((VBD<double>*)h->ptr)->s, what, in) : set_state(((VBD<float>*)h->ptr)->s, what, in);
}
int orc_vbd_energy(void* hv, double* parts) {
    Handle* h = (Handle*)hv;
    if (h->kind == 1) { auto* b = (VBD<double>*)h->ptr; scene_energy(b->fem, b->s, parts); }
    else { auto* b = (VBD<float>*)h->ptr; scene_energy(b->fem, b->s, parts); }
    return 0;
}
int orc_vbd_residual(void* hv, float dt, double* out) {
    Handle* h = (Handle*)hv;
    if (h->kind == 1) residual_norms(*(VBD<double>*)h->ptr, (double)dt, out);
    else residual_norms(*(VBD<float>*)h->ptr, dt, out);
    return 0;
}
int orc_vbd_forces(void* hv, float dt, double* out) {
    Handle* h = (Handle*)hv;
    if (!h || !out || h->kind > 1) return -1;
    if (h->kind == 1) residual_vectors(*(VBD<double>*)h->ptr, (double)dt, out);
    else residual_vectors(*(VBD<float>*)h->ptr, dt, out);
    return 0;
}
int orc_element_data(void* hv, int kind, double* out) {
    Handle* h = (Handle*)hv;
    if (!h || !out || kind < 0 || kind > 6) return -1;
    switch (h->kind) {
        case 0: element_data(((VBD<float>*)h->ptr)->fem, ((VBD<float>*)h->ptr)->s, kind, out); break;
        case 1: element_data(((VBD<double>*)h->ptr)->fem, ((VBD<double>*)h->ptr)->s, kind, out); break;
        case 2: element_data(((XPBD<float>*)h->ptr)->fem, ((XPBD<float>*)h->ptr)->s, kind, out); break;
        case 3: element_data(((XPBD<double>*)h->ptr)->fem, ((XPBD<double>*)h->ptr)->s, kind, out); break;
        case 4: element_data(((Explicit<float>*)h->ptr)->fem, ((Explicit<float>*)h->ptr)->s, kind, out); break;
        case 5: element_data(((Explicit<double>*)h->ptr)->fem, ((Explicit<double>*)h->ptr)->s, kind, out); break;
        default: return -1;
    }
    return 0;
}
void orc_vbd_destroy(void* hv) {
    Handle* h = (Handle*)hv;
    if (!h) return;
    if (h->kind == 1) delete (VBD<double>*)h->ptr; else delete (VBD<float>*)h->ptr;
    delete h;
}

void* orc_cpuvbd_create(const orc_desc* d) {
    if (!d || !d->masses || d->material > StableNeoHooke) return nullptr;
    auto* c = new CpuVBD();
    if (!build_fem(d, c->fem)) { delete c; return nullptr; }
    c->n = d->n_nodes;
    c->p.resize(c->n);
    for (int i = 0; i < c->n; ++i) c->p[i] = {d->positions[3 * i], d->positions[3 * i + 1], d->positions[3 * i + 2]};
    c->last_p = c->init_p = c->y = c->prev_x = c->prev_prev_x = c->p;
    c->v.assign(c->n, V3<float>());
    if (d->initial_velocity)
        for (int i = 0; i < c->n; ++i) c->v[i] = {d->initial_velocity[3 * i], d->initial_velocity[3 * i + 1], d->initial_velocity[3 * i + 2]};
    c->m.assign(d->masses, d->masses + c->n);
    c->active.assign(c->n, 1);
    c->fixed.assign(d->fixed_ids, d->fixed_ids + d->n_fixed);
    V3<float> s;
    for (int id : c->fixed) { c->active[id] = 0; s = s + c->p[id]; }   // RB_Fixation::init
    c->com = c->fixed.empty() ? V3<float>() : s / (float)c->fixed.size();
    c->g = {d->gravity[0], d->gravity[1], d->gravity[2]};
    c->owners.assign(c->n, {});
    for (int e = 0; e < d->n_elements; ++e)
        for (int j = 0; j < c->fem.ne; ++j) c->owners[d->topology[e * c->fem.ne + j]].push_back({e, j});
    c->iterations = d->iterations;
    c->rho = d->rho;
    c->damping = d->damping;
    return c;
}

int orc_cpuvbd_step(void* h, float frame_dt, int substeps, int with_residual) {
    CpuVBD* c = (CpuVBD*)h;
    if (!c || substeps <= 0) return -1;
    const float sub = frame_dt / (float)substeps;
    for (int k = 0; k < substeps; ++k) cpu_vbd_substep(*c, sub, with_residual != 0);
    return 0;
}

int orc_cpuvbd_get(void* h, int what, double* out) {
    CpuVBD* c = (CpuVBD*)h;
    const std::vector<V3<float>>* src = what == 0 ? &c->p : (what == 1 ? &c->v : nullptr);
    if (!src) return -1;
    for (int i = 0; i < c->n; ++i) for (int k = 0; k < 3; ++k) out[3 * i + k] = (*src)[i][k];
    return 0;
}

void orc_cpuvbd_destroy(void* h) { delete (CpuVBD*)h; }

double orc_cpuvbd_run_many(void** hs, int n, float frame_dt, int substeps, int with_residual, int n_threads) {
    if (n_threads < 1) n_threads = 1;
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    std::atomic<int> next{0};
    for (int t = 0; t < n_threads; ++t)
        pool.emplace_back([&]() {
            for (int k = next++; k < n; k = next++) orc_cpuvbd_step(hs[k], frame_dt, substeps, with_residual);
        });
    for (auto& th : pool) th.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}


void* orc_xpbd_create(const orc_desc* d, int fp64) {
    if (!d || !d->masses) return nullptr;
    Handle* h = new Handle();
    h->kind = fp64 ? 3 : 2;
    h->ptr = fp64 ? (void*)xpbd_create_t<double>(d) : (void*)xpbd_create_t<float>(d);
    if (!h->ptr) { delete h; return nullptr; }
    return h;
}
int orc_xpbd_step(void* hv, float frame_dt, int substeps) {
    Handle* h = (Handle*)hv;
    const float sub = frame_dt / (float)substeps;
    for (int k = 0; k < substeps; ++k) {
        if (h->kind == 3) xpbd_substep(*(XPBD<double>*)h->ptr, (double)sub);
        else xpbd_substep(*(XPBD<float>*)h->ptr, sub);
    }
    return 0;
}
int orc_xpbd_get(void* hv, int what, double* out) {
    Handle* h = (Handle*)hv;
    return h->kind == 3 ? get_state(((XPBD<double>*)h->ptr)->s, what, out) : get_state(((XPBD<float>*)h->ptr)->s, what, out);
}
void orc_xpbd_destroy(void* hv) {
    Handle* h = (Handle*)hv;
    if (h->kind == 3) delete (XPBD<double>*)h->ptr; else delete (XPBD<float>*)h->ptr;
    delete h;
}

void* orc_explicit_create(const orc_desc* d, int fp64) {
    if (!d || !d->masses || d->material > StableNeoHooke) return nullptr;
    Handle* h = new Handle();
    h->kind = fp64 ? 5 : 4;
    h->ptr = fp64 ? (void*)explicit_create_t<double>(d) : (void*)explicit_create_t<float>(d);
    if (!h->ptr) { delete h; return nullptr; }
    return h;
}
int orc_explicit_step(void* hv, float frame_dt, int substeps) {
    Handle* h = (Handle*)hv;
    const float sub = frame_dt / (float)substeps;
    for (int k = 0; k < substeps; ++k) {
        if (h->kind == 5) explicit_substep(*(Explicit<double>*)h->ptr, (double)sub);
        else explicit_substep(*(Explicit<float>*)h->ptr, sub);
    }
    return 0;
}
int orc_explicit_get(void* hv, int what, double* out) {
    Handle* h = (Handle*)hv;
    return h->kind == 5 ? get_state(((Explicit<double>*)h->ptr)->s, what, out) : get_state(((Explicit<float>*)h->ptr)->s, what, out);
}
void orc_explicit_destroy(void* hv) {
    Handle* h = (Handle*)hv;
    if (h->kind == 5) delete (Explicit<double>*)h->ptr; else delete (Explicit<float>*)h->ptr;
    delete h;
}

}  // extern "C"
