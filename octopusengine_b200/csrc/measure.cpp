// Accuracy measures of the reference's experiments, on host arrays:
//   Error / MeshDiff_MSE          octopus/include/Script/Measure/MeshDiff.h:9-83
//   Beam_MSE_Sampling             octopus/include/Script/Measure/MeshDiff.h:85-258
//   FEM_Flexion_error_recorder    octopus/src/Script/Record/Recorder.cpp:190-220
//   FEM_Torsion_error_recorder    octopus/src/Script/Record/Recorder.cpp:222-330
// Geometry tests (boxes, barycentric coordinates) run in FP32 as the reference's do; the error
// sums are accumulated in FP64.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/octopus_b200.h"
#include "host.hpp"

using namespace octb;

namespace {

struct F3 { float x, y, z; };
inline F3 at(const float* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
inline F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
inline float len(F3 a) { return std::sqrt(dot(a, a)); }

// Error::update, with the sums in FP64: out = {MSE, RMSE, MAE, max, L1, L2}
struct Err {
    double l1 = 0, l2 = 0, mx = 0;
    long n = 0;
    void update(double ex, double ey, double ez) {
        const double l = std::sqrt(ex * ex + ey * ey + ez * ez);
        ++n;
        mx = std::max(mx, l);
        l2 += l * l;
        l1 += l;
    }
    void write(double* out) const {
        const double mse = n ? l2 / n : 0.0;
        out[0] = mse; out[1] = std::sqrt(mse); out[2] = n ? l1 / n : 0.0; out[3] = mx; out[4] = l1; out[5] = l2;
    }
};

int linear_of(int e) { return (e == kHexa || e == kHexa27) ? kHexa : kTetra; }

struct Box { F3 lo, hi; };
Box box_of(const float* X, const int32_t* ids, int n) {
    Box b{at(X, ids[0]), at(X, ids[0])};
    for (int i = 1; i < n; ++i) {
        const F3 p = at(X, ids[i]);
        b.lo = {std::min(b.lo.x, p.x), std::min(b.lo.y, p.y), std::min(b.lo.z, p.z)};
        b.hi = {std::max(b.hi.x, p.x), std::max(b.hi.y, p.y), std::max(b.hi.z, p.z)};
    }
    return b;
}
bool inside(const Box& b, F3 p) {
    return p.x >= b.lo.x && p.y >= b.lo.y && p.z >= b.lo.z && p.x <= b.hi.x && p.y <= b.hi.y && p.z <= b.hi.z;
}
float signed_volume(F3 a, F3 b, F3 c, F3 d) { return dot(d - a, cross(b - a, c - a)) / 6.f; }   // Tetraedron

struct Mesh {
    int element = 0, ne = 0, n_nodes = 0, n_elements = 0;
    std::vector<float> X;
    std::vector<int32_t> topo;
    F3 offset{};                      // rest bounding-box minimum
    std::vector<F3> sample;           // reference-element coordinates of each kept sample
    std::vector<int> sample_element;
};

}  // namespace

struct oct_sampler {
    std::vector<Mesh> meshes;
    int ref = 0;
};

extern "C" {

oct_status oct_shape_values(int32_t element, const double x[3], double* N) {
    if (!x || !N || element_nodes(element) < 0) return OCT_EINVAL;
    return shape_values(element, x, N) ? OCT_OK : OCT_EINVAL;
}

oct_status oct_reference_nodes(int32_t element, double* X) {
    if (!X || element_nodes(element) < 0) return OCT_EINVAL;
    return reference_nodes(element, X) ? OCT_OK : OCT_EINVAL;
}

oct_status oct_mesh_error(const float* a, const float* b, int32_t n, const float offset[3], double out[6]) {
    if (!a || !b || n < 0 || !out) return OCT_EINVAL;
    const double ox = offset ? offset[0] : 0.0, oy = offset ? offset[1] : 0.0, oz = offset ? offset[2] : 0.0;
    Err e;
    for (int i = 0; i < n; ++i)
        e.update((double)a[3 * i] - b[3 * i] - ox, (double)a[3 * i + 1] - b[3 * i + 1] - oy, (double)a[3 * i + 2] - b[3 * i + 2] - oz);
    e.write(out);
    return OCT_OK;
}

oct_status oct_beam_sampler_create(int32_t n_meshes, const int32_t* elements, const int32_t* n_nodes,
                                   const float* const* rest_positions, const int32_t* n_elements,
                                   const int32_t* const* topologies, int32_t ref, int32_t nb_sample, oct_sampler** out) {
    if (!out || n_meshes <= 0 || !elements || !n_nodes || !rest_positions || !n_elements || !topologies || ref < 0 ||
        ref >= n_meshes || nb_sample <= 0)
        return OCT_EINVAL;
    *out = nullptr;
    auto* S = new oct_sampler();
    S->ref = ref;
    S->meshes.resize(n_meshes);
    for (int m = 0; m < n_meshes; ++m) {
        Mesh& M = S->meshes[m];
        M.element = elements[m];
        M.ne = element_nodes(M.element);
        M.n_nodes = n_nodes[m];
        M.n_elements = n_elements[m];
        if (M.ne < 0 || M.n_nodes <= 0 || M.n_elements <= 0 || !rest_positions[m] || !topologies[m]) { delete S; return OCT_EINVAL; }
        M.X.assign(rest_positions[m], rest_positions[m] + 3 * (size_t)M.n_nodes);
        M.topo.assign(topologies[m], topologies[m] + (size_t)M.n_elements * M.ne);
        for (int32_t v : M.topo)
            if (v < 0 || v >= M.n_nodes) { delete S; return OCT_EINVAL; }
    }
    // global samples: a regular grid inside the reference mesh's box, 100 large_eps (1e-4) in
    // from its faces, nb_sample points per unit length
    const Mesh& R = S->meshes[ref];
    std::vector<int32_t> all(R.n_nodes);
    for (int i = 0; i < R.n_nodes; ++i) all[i] = i;
    const Box rb = box_of(R.X.data(), all.data(), R.n_nodes);
    const F3 size = rb.hi - rb.lo;
    const float e100 = 100.f * 1e-6f;
    const F3 maxs = size - F3{e100, e100, e100}, mins{e100, e100, e100};
    const F3 step = {(maxs.x - mins.x) / size.x * (1.f / nb_sample), (maxs.y - mins.y) / size.y * (1.f / nb_sample),
                     (maxs.z - mins.z) / size.z * (1.f / nb_sample)};
    std::vector<F3> global;
    for (int x = 0; x <= nb_sample * size.x; ++x)
        for (int y = 0; y <= nb_sample * size.y; ++y)
            for (int z = 0; z <= nb_sample * size.z; ++z) global.push_back(mins + F3{step.x * x, step.y * y, step.z * z});
    // locate every sample in an element of every mesh (rest state), through a uniform grid
    const int gx = (int)std::ceil(size.x * 2.f), gy = (int)std::ceil(size.y * 2.f), gz = (int)std::ceil(size.z * 2.f);
    std::vector<std::vector<int>> found(n_meshes, std::vector<int>(global.size(), -1));
    std::vector<std::vector<F3>> coord(n_meshes, std::vector<F3>(global.size()));
    for (int m = 0; m < n_meshes; ++m) {
        Mesh& M = S->meshes[m];
        std::vector<int32_t> ids(M.n_nodes);
        for (int i = 0; i < M.n_nodes; ++i) ids[i] = i;
        M.offset = box_of(M.X.data(), ids.data(), M.n_nodes).lo;
        const int lin = linear_of(M.element), nl = element_nodes(lin);
        std::vector<double> rn(3 * M.ne);
        reference_nodes(M.element, rn.data());
        std::vector<std::vector<int>> grid((size_t)gx * gy * gz);
        auto cell = [&](float v, int g) { return std::min(std::max((int)std::floor(v * g), 0), g - 1); };
        for (int e = 0; e < M.n_elements; ++e) {
            Box b = box_of(M.X.data(), M.topo.data() + (size_t)e * M.ne, nl);
            const F3 lo = b.lo - M.offset, hi = b.hi - M.offset;
            const int x0 = cell(lo.x / size.x - e100, gx), x1 = cell(hi.x / size.x + e100, gx);
            const int y0 = cell(lo.y / size.y - e100, gy), y1 = cell(hi.y / size.y + e100, gy);
            const int z0 = cell(lo.z / size.z - e100, gz), z1 = cell(hi.z / size.z + e100, gz);
            for (int x = x0; x <= x1; ++x)
                for (int y = y0; y <= y1; ++y)
                    for (int z = z0; z <= z1; ++z) grid[x + (size_t)y * gx + (size_t)z * gx * gy].push_back(e);
        }
        for (size_t k = 0; k < global.size(); ++k) {
            const F3 s = global[k], q = s + M.offset;
            const int cx = cell(s.x / size.x, gx), cy = cell(s.y / size.y, gy), cz = cell(s.z / size.z, gz);
            for (int e : grid[cx + (size_t)cy * gx + (size_t)cz * gx * gy]) {
                const int32_t* t = M.topo.data() + (size_t)e * M.ne;
                if (lin == kHexa) {
                    if (!inside(box_of(M.X.data(), t, nl), q)) continue;
                    const F3 o = at(M.X.data(), t[0]);
                    const F3 ax = at(M.X.data(), t[1]) - o, ay = at(M.X.data(), t[3]) - o, az = at(M.X.data(), t[4]) - o;
                    const F3 r = q - o;
                    const float lx = len(ax), ly = len(ay), lz = len(az);
                    F3 c = {dot(r, ax * (1.f / lx)) / lx, dot(r, ay * (1.f / ly)) / ly, dot(r, az * (1.f / lz)) / lz};
                    c = c * 2.f + F3{(float)rn[0], (float)rn[1], (float)rn[2]};   // unit cube -> [-1, 1]^3
                    found[m][k] = e;
                    coord[m][k] = c;
                    break;
                }
                const F3 p0 = at(M.X.data(), t[0]), p1 = at(M.X.data(), t[1]), p2 = at(M.X.data(), t[2]), p3 = at(M.X.data(), t[3]);
                const float V0 = signed_volume(p0, p1, p2, p3);
                const float eps = 1.17549435e-38f * 1e6f;
                if (!(V0 * signed_volume(q, p1, p2, p3) > -eps && V0 * signed_volume(p0, q, p2, p3) > -eps &&
                      V0 * signed_volume(p0, p1, q, p3) > -eps && V0 * signed_volume(p0, p1, p2, q) > -eps))
                    continue;
                const float iv = 1.f / V0;
                const float l0 = signed_volume(q, p1, p2, p3) * iv, l1 = signed_volume(p0, q, p2, p3) * iv,
                            l2 = signed_volume(p0, p1, q, p3) * iv;
                const float l3 = 1.f - l0 - l1 - l2;
                F3 c{0, 0, 0};
                const float L[4] = {l0, l1, l2, l3};
                for (int i = 0; i < 4; ++i) c = c + F3{(float)rn[3 * i], (float)rn[3 * i + 1], (float)rn[3 * i + 2]} * L[i];
                found[m][k] = e;
                coord[m][k] = c;
                break;
            }
        }
    }
    // keep the samples every mesh contains (the reference assumes all are found)
    for (size_t k = 0; k < global.size(); ++k) {
        bool all_found = true;
        for (int m = 0; m < n_meshes; ++m) all_found = all_found && found[m][k] >= 0;
        if (!all_found) continue;
        for (int m = 0; m < n_meshes; ++m) {
            S->meshes[m].sample.push_back(coord[m][k]);
            S->meshes[m].sample_element.push_back(found[m][k]);
        }
    }
    *out = S;
    return OCT_OK;
}

oct_status oct_beam_sampler_info(oct_sampler* S, int32_t* n_samples) {
    if (!S || !n_samples) return OCT_EINVAL;
    *n_samples = (int32_t)S->meshes[S->ref].sample.size();
    return OCT_OK;
}

// Beam_MSE_Sampling::get_error: each sample interpolated in mesh m's current positions and in
// the reference mesh's, both relative to their rest box minimum.
oct_status oct_beam_sampler_error(oct_sampler* S, int32_t m, const float* positions, const float* ref_positions,
                                  double out[6]) {
    if (!S || m < 0 || m >= (int)S->meshes.size() || !positions || !ref_positions || !out) return OCT_EINVAL;
    const Mesh& M = S->meshes[m];
    const Mesh& R = S->meshes[S->ref];
    std::vector<double> N(27), NR(27);
    Err e;
    for (size_t k = 0; k < M.sample.size(); ++k) {
        auto interp = [&](const Mesh& A, const float* P, std::vector<double>& w, double* p) {
            const double x[3] = {A.sample[k].x, A.sample[k].y, A.sample[k].z};
            shape_values(A.element, x, w.data());
            p[0] = p[1] = p[2] = 0.0;
            const int32_t* t = A.topo.data() + (size_t)A.sample_element[k] * A.ne;
            for (int j = 0; j < A.ne; ++j)
                for (int d = 0; d < 3; ++d) p[d] += P[3 * t[j] + d] * w[j];
        };
        double p[3], r[3];
        interp(M, positions, N, p);
        interp(R, ref_positions, NR, r);
        e.update((p[0] - M.offset.x) - (r[0] - R.offset.x), (p[1] - M.offset.y) - (r[1] - R.offset.y),
                 (p[2] - M.offset.z) - (r[2] - R.offset.z));
    }
    e.write(out);
    return OCT_OK;
}

oct_status oct_beam_sampler_destroy(oct_sampler* S) {
    if (!S) return OCT_EINVAL;
    delete S;
    return OCT_OK;
}

oct_status oct_flexion_error(const float* rest, const float* current, int32_t n, const float follow[3], const float target[3],
                             double* error, int32_t* particle) {
    if (!rest || !current || n <= 0 || !follow || !target || !error) return OCT_EINVAL;
    const F3 f{follow[0], follow[1], follow[2]};
    int id = -1;
    for (int i = 0; i < n && id < 0; ++i) {   // first particle within 1e-3 of the followed point
        const F3 d = at(rest, i) - f;
        if (dot(d, d) < 1e-6f) id = i;
    }
    if (id < 0) return OCT_EINVAL;
    const double dx = (double)target[0] - current[3 * id], dy = (double)target[1] - current[3 * id + 1],
                 dz = (double)target[2] - current[3 * id + 2];
    *error = dx * dx + dy * dy + dz * dz;
    if (particle) *particle = id;
    return OCT_OK;
}

oct_status oct_torsion_profile(int32_t element, const float* rest, const float* current, int32_t n_nodes,
                               const int32_t* topology, int32_t n_elements, int32_t samples_per_edge, float beam_length,
                               float* distance, float* angles, int32_t capacity, int32_t* count) {
    const int ne = element_nodes(element);
    if (ne < 0 || !rest || !current || n_nodes <= 0 || !topology || n_elements <= 0 || samples_per_edge < 2 ||
        !(beam_length > 0.f) || !count)
        return OCT_EINVAL;
    const int nl = element_nodes(linear_of(element));
    std::vector<double> rn(3 * ne), w(ne);
    reference_nodes(element, rn.data());
    std::vector<std::pair<float, float>> da;   // (distance, angle)
    for (int e = 0; e < n_elements; ++e) {
        const int32_t* t = topology + (size_t)e * ne;
        int edge[8], k = 0;
        for (int j = 0; j < nl; ++j) {   // corners on the beam's x axis edge (y = z = 0)
            const F3 p = at(rest, t[j]);
            if (p.y < 1e-6f && p.z < 1e-6f) edge[k++] = j;
        }
        if (k < 2) continue;
        const F3 a{(float)rn[3 * edge[0]], (float)rn[3 * edge[0] + 1], (float)rn[3 * edge[0] + 2]};
        const F3 b{(float)rn[3 * edge[1]], (float)rn[3 * edge[1] + 1], (float)rn[3 * edge[1] + 2]};
        for (int j = 0; j < samples_per_edge; ++j) {
            const float tt = (float)j / (float)(samples_per_edge - 1);
            const F3 r = (b - a) * tt + a;
            const double x[3] = {r.x, r.y, r.z};
            shape_values(element, x, w.data());
            F3 p0{0, 0, 0}, p{0, 0, 0};
            for (int l = 0; l < ne; ++l) {
                p = p + at(rest, t[l]) * (float)w[l];
                p0 = p0 + at(current, t[l]) * (float)w[l];
            }
            // angle of the edge point around the cross-section centre (0.5, 0.5) between the rest
            // and the current state, in degrees; distance along the beam of the current point
            float ix = p0.y - 0.5f, iy = p0.z - 0.5f, cx = p.y - 0.5f, cy = p.z - 0.5f;
            const float li = std::sqrt(ix * ix + iy * iy), lc = std::sqrt(cx * cx + cy * cy);
            ix /= li; iy /= li; cx /= lc; cy /= lc;
            const float ang = std::fabs(std::atan2(cx * iy - cy * ix, cx * ix + cy * iy)) * (180.f / 3.14159265358979f);
            da.push_back({p0.x / beam_length, ang});
        }
    }
    std::stable_sort(da.begin(), da.end(), [](const auto& u, const auto& v) { return u.first < v.first; });
    int n = 0;
    for (size_t i = 0; i < da.size();) {   // merge points closer than 1e-4 along the beam
        size_t j = 1;
        float sum = da[i].second;
        while (i + j < da.size() && std::fabs(da[i].first - da[i + j].first) < 1e-4f) sum += da[i + j++].second;
        if (n < capacity && distance && angles) { distance[n] = da[i].first; angles[n] = sum / (float)j; }
        ++n;
        i += j;
    }
    *count = n;
    return OCT_OK;
}

}  // extern "C"
