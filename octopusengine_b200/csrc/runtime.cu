// Host runtime behind the C ABI: contexts (device, stream, HBM budget), scenes (set-up on
// the host, state resident on the device), the per-scene step drivers that follow the
// reference's launch structure, and batches that step many scenes through one launch per
// (element type, colour) captured in a CUDA graph.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/octopus_b200.h"
#include "device.cuh"
#include "host.hpp"
#include "kernels.cuh"

using namespace octb;

namespace {
constexpr int kBlockThreads = 128;

// NVTX ranges around frames, sub-steps and colour sweeps (host side; a profiler shows them on
// the timeline, and without one they cost a pointer test).
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
};
constexpr int kNodeChunk = 256;
}  // namespace

struct oct_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    size_t budget = 0, used = 0;
    std::string err;
    int* d_error = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    uint64_t launches = 0;
    bool tables[10] = {false};
    std::mutex mu;       // guards the budget accounting and the shape-table upload
    std::mutex err_mu;   // guards err (scenes may be created from several host threads)
    // device blocks released by destroyed scenes and batches, kept for reuse (size -> pointer):
    // a request loop creates and destroys scenes every few frames, and cudaMalloc / cudaFree
    // synchronise the device
    std::multimap<size_t, void*> cache;
    size_t cached = 0;
};

namespace {

oct_status fail(oct_ctx* c, oct_status s, const std::string& msg) {
    if (c) {
        std::lock_guard<std::mutex> lock(c->err_mu);
        c->err = msg;
    }
    return s;
}

#define OCT_CUDA(ctx, call)                                                                        \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(ctx, OCT_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Device allocation accounted against the context budget.
// Frees every cached block (caller holds ctx->mu).
void trim_cache(oct_ctx* c) {
    for (auto& kv : c->cache) cudaFree(kv.second);
    c->cache.clear();
    c->cached = 0;
}

// Device allocation accounted against the context budget.  Released blocks go to the
// context's cache and are handed out again for requests of at most their size and more than
// half of it; the budget counts blocks in use plus cached ones, and the cache is trimmed
// before a request would exceed it.  A scene or batch is released only after the context's
// stream has drained, so no kernel still reads a block when it is reused.
struct DevMem {
    oct_ctx* ctx = nullptr;
    std::vector<std::pair<void*, size_t>> blocks;
    template <class T> oct_status alloc(T*& p, size_t n) {
        const size_t bytes = ((std::max<size_t>(n, 1) * sizeof(T) + 255) / 256) * 256;
        std::lock_guard<std::mutex> lock(ctx->mu);
        auto it = ctx->cache.lower_bound(bytes);
        if (it != ctx->cache.end() && it->first <= 2 * bytes) {
            p = (T*)it->second;
            blocks.push_back({it->second, it->first});
            ctx->used += it->first;
            ctx->cached -= it->first;
            ctx->cache.erase(it);
            return OCT_OK;
        }
        while (ctx->used + ctx->cached + bytes > ctx->budget && !ctx->cache.empty()) {
            auto big = std::prev(ctx->cache.end());
            cudaFree(big->second);
            ctx->cached -= big->first;
            ctx->cache.erase(big);
        }
        if (ctx->used + bytes > ctx->budget)
            return fail(ctx, OCT_ENOMEM_BUDGET, "HBM budget exceeded: need " + std::to_string(ctx->used + bytes) +
                                                    " bytes, budget " + std::to_string(ctx->budget));
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, bytes);
        if (e == cudaErrorMemoryAllocation && !ctx->cache.empty()) {   // device full of cached blocks
            cudaGetLastError();
            trim_cache(ctx);
            e = cudaMalloc(&q, bytes);
        }
        if (e != cudaSuccess) return fail(ctx, OCT_ECUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        blocks.push_back({q, bytes});
        ctx->used += bytes;
        p = (T*)q;
        return OCT_OK;
    }
    void release() {
        std::lock_guard<std::mutex> lock(ctx->mu);
        for (auto& b : blocks) {
            ctx->used -= b.second;
            ctx->cache.emplace(b.second, b.first);
            ctx->cached += b.second;
        }
        blocks.clear();
    }
};

}  // namespace

struct oct_scene {
    oct_ctx* ctx = nullptr;
    DevMem mem;
    int solver = 0, element = 0, material = 0, ne = 0, nq = 0;
    int64_t n_records = 0;          // distinct quadrature records the owner entries index
    int n_nodes = 0, n_elements = 0, n_fixed = 0, n_colors = 0;
    int iterations = 1, order_mode = 0, tpv = 8, precision = 0, max_valence = 0;
    float rho = 0.f, global_damping = 0.f;
    float young = 0.f, poisson = 0.f, density = 0.f;   // as described (run metadata)
    int last_substeps = 0;
    bool in_place = true, box = false, has_v0 = false;
    bool xpbd_raw = true, xpbd_project = true;   // XPBD update form; false: no projection (OptiGroup)
    // frame graph (oct_scene_set_capture): the sub-steps of one frame, replayed while the
    // frame's (dt, substeps) stay the same
    bool capture = false;
    cudaGraphExec_t frame_exec = nullptr;
    float frame_dt = -1.f;
    int frame_substeps = 0;
    uint64_t frame_launches = 0;
    std::mt19937 rng;
    std::vector<int32_t> colors, vids, color_off;   // colour-sorted slots
    std::vector<int32_t> own_off;                    // owner CSR offsets in slot order (host copy)
    std::vector<float> masses, X;
    std::vector<int32_t> fixed, fixed_group;
    float fix_host[kFixGroups * 16] = {0};
    float* d_fix = nullptr;
    // device
    SceneDev h{};
    SceneDev* d_scene = nullptr;
    int* d_pending = nullptr;
    int pending_host = 0;
    int* d_status = nullptr;        // SceneDev::status of the scene's own steps
    VWork* d_vwork = nullptr;
    std::vector<int> vwork_off;     // per colour: [vwork_off[c], vwork_off[c+1])
    NWork* d_nwork = nullptr;
    int n_nwork = 0;
    NWork* d_fwork = nullptr;
    int n_fwork = 0;
    int* d_elems = nullptr;         // XPBD: colour-sorted element ids
    int* d_etopo = nullptr;         // XPBD: their topology in colour order
    std::vector<int> elem_off;
    XWork* d_xwork = nullptr;       // XPBD: block work items of the scene's own steps
    std::vector<int> xwork_off;     // per colour: [xwork_off[c], xwork_off[c+1])
    double* d_red = nullptr;        // 4 doubles of reduction scratch
    float* d_io = nullptr;          // n_nodes x 3 floats: node state in and out (allocated on first use)
    float* d_diag = nullptr;        // per-element diagnostics output (allocated on first use)
    float4* d_contrib = nullptr;    // explicit: per-(element, local node) force contributions
    // scripted effects (oct_scene_add_effect): host copy of the device slots
    EffectDev effects[kMaxEffects];
    EffectDev* d_effects = nullptr;
    int n_effects = 0;
    std::vector<int32_t> topo_host;   // kept for the effects' surface extraction
    // multigrid VBD: the linear level as a scene of the corners, the corner map, the
    // prolongation lists and the iteration schedule (MG_VBD_FEM)
    oct_scene* mg_sub = nullptr;
    int* d_mg_map = nullptr;
    int n_mg_map = 0;
    int* d_pro[3] = {nullptr, nullptr, nullptr};   // edges (k 2), faces (k 4), volumes (k 8)
    int n_pro[3] = {0, 0, 0};
    int mg_max[2] = {0, 0}, mg_count = 0, mg_current = 1;
};

struct oct_batch {
    oct_ctx* ctx = nullptr;
    DevMem mem;
    std::vector<oct_scene*> scenes;
    SceneDev* d_scenes = nullptr;
    int* d_pending = nullptr;
    std::vector<int> pending_host;
    int* d_status = nullptr;        // SceneDev::status of each scene during the batch's frames
    int solver = OCT_SOLVER_VBD;    // VBD or XPBD: a batch holds scenes of one solver
    XWork* d_xwork = nullptr;       // XPBD: block items, per group and colour
    struct Group {
        int element, material, tpv;     // XPBD: tpv holds the raw (V1/V2) update flag
        bool in_place;
        std::vector<int> off;   // per colour, into the group's part of d_vwork (XPBD: d_xwork)
        int base = 0;
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
    };
    std::vector<Group> groups;
    VWork* d_vwork = nullptr;
    NWork* d_nwork = nullptr;
    int n_nwork = 0;
    NWork* d_fwork = nullptr;
    int n_fwork = 0;
    NWork* d_bwork = nullptr;
    int n_bwork = 0;
    int iterations = 1;
    float rho = 0.f;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    float graph_dt = -1.f;
    int graph_pending = -1;
    std::vector<size_t> state_off;
    long long* d_soff = nullptr;    // per-scene offsets into the staging buffer
    float* d_state = nullptr;       // staging buffer, allocated on first host-state transfer
};

namespace {

oct_status ensure_tables(oct_ctx* c, int element) {
    std::lock_guard<std::mutex> lock(c->mu);
    if (c->tables[element]) return OCT_OK;
    ShapeTable s;
    if (!shape_table(element, s)) return fail(c, OCT_EINVAL, "unsupported element");
    std::vector<float> f(s.dN.begin(), s.dN.end());
    f.resize(((f.size() + 3) / 4) * 4, 0.f);
    OCT_CUDA(c, upload_shape_tables(element, f.data(), (int)s.dN.size()));
    OCT_CUDA(c, upload_shape_tables_fp64(element, s.dN.data(), (int)s.dN.size(), s.w.data(), (int)s.w.size()));
    c->tables[element] = true;
    return OCT_OK;
}

// Lane-group items: a colour's vertices get at least the scene's lanes per vertex, and enough
// lanes that each averages at most kOwnersPerLane owners.  Lanes of one vertex gather
// overlapping nodes (its owners share most of theirs), so high-valence colours gain from wider
// groups, up to a point: the P2 corner colours (20 owners per vertex) of the 256-beam batch
// with 4 lanes instead of 2, P2 sweep 1.795 -> 1.728 ms; 8 lanes 1.827 ms, 16 lanes 2.100 ms;
// P1 (20-24 owners) with 8 lanes instead of 4, 0.221 -> 0.298 ms.
constexpr int kOwnersPerLane = 8;

// Split [begin, end) slots into work items for one scene: block-sized items of 128 / t slots
// (t lanes per vertex, the colour's count from tpv and kOwnersPerLane), or (tpv == 0) warp
// items packing whole vertices up to 32 (vertex, owner) pairs and at most 31 slots.
void append_vwork(std::vector<VWork>& out, int scene, int begin, int end, int tpv, const std::vector<int32_t>& own_off) {
    if (tpv > 0) {
        int t = tpv;
        if (end > begin) {
            const int64_t pairs = (int64_t)own_off[end] - own_off[begin];
            while (t < 32 && pairs > (int64_t)kOwnersPerLane * t * (end - begin)) t <<= 1;
        }
        const int vpb = kBlockThreads / t;
        for (int s = begin; s < end; s += vpb) out.push_back({scene, s, std::min(vpb, end - s), 0, 0u, 0, t, 0});
        return;
    }
    int s = begin;
    while (s < end) {
        int pairs = 0, n = 0;
        unsigned heads = 0;
        while (s + n < end && n < 31 && pairs + (own_off[s + n + 1] - own_off[s + n]) <= 32) {
            heads |= 1u << pairs;
            pairs += own_off[s + n + 1] - own_off[s + n];
            ++n;
        }
        out.push_back({scene, s, n, own_off[s], heads, pairs, 0, 0});
        s += n;
    }
}
void append_nwork(std::vector<NWork>& out, int scene, int n) {
    for (int s = 0; s < n; s += kNodeChunk) out.push_back({scene, s, std::min(kNodeChunk, n - s), 0});
}

// XPBD block items over [begin, end) of a scene's colour-sorted element list.
void append_xwork(std::vector<XWork>& out, int scene, int begin, int end, int per_block) {
    for (int e = begin; e < end; e += per_block) out.push_back({scene, e, std::min(per_block, end - e), 0});
}

// lanes per vertex chosen when the description leaves it at 0 (0 = packed pairs)
int measured_tpv(int element) {
    switch (element) {
        case kTetra: return 4;
        case kHexa: return 4;
        case kTetra10: return 1;   // corner colours widen to 4 lanes (kOwnersPerLane)
        default: return 0;
    }
}

int default_tpv(int element) {
    switch (element) {
        case kTetra: return 8;
        case kHexa: return 8;
        case kTetra10: return 8;
        case kTetra20: return 8;
        default: return 4;
    }
}

template <class T> oct_status upload(oct_ctx* c, DevMem& m, T*& d, const std::vector<T>& h) {
    oct_status st = m.alloc(d, h.size());
    if (st) return st;
    if (!h.empty()) OCT_CUDA(c, cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return OCT_OK;
}

oct_status check_error_word(oct_ctx* c) {
    int e = 0;
    OCT_CUDA(c, cudaMemcpy(&e, c->d_error, sizeof(int), cudaMemcpyDeviceToHost));
    if (e & 2) { int z = 0; cudaMemcpy(c->d_error, &z, sizeof(int), cudaMemcpyHostToDevice); return fail(c, OCT_ENUMERIC, "non-finite value in the scene state"); }
    if (e & 1) { int z = 0; cudaMemcpy(c->d_error, &z, sizeof(int), cudaMemcpyHostToDevice); return fail(c, OCT_ETIMEDOUT, "a bounded device wait timed out"); }
    return OCT_OK;
}

// Vertex work items of every colour for the scene's lane mapping (tpv), uploaded to the device.
oct_status build_vertex_work(oct_scene* s) {
    std::vector<VWork> vw;
    s->vwork_off.assign(1, 0);
    for (int k = 0; k + 1 < (int)s->color_off.size(); ++k) {
        append_vwork(vw, 0, s->color_off[k], s->color_off[k + 1], s->tpv, s->own_off);
        s->vwork_off.push_back((int)vw.size());
    }
    return upload(s->ctx, s->mem, s->d_vwork, vw);
}

oct_status build_scene(oct_ctx* c, const oct_scene_desc* d, oct_scene* s);


// Multigrid VBD (MG_VBD_FEM ctor, octopus/src/Dynamic/VBD/MG_VertexBlockDescent.cpp:134-176):
// the linear level is built as a scene of the corner nodes (numbered in ascending order)
// with the corner topology, its own DSAT colouring and lumped masses from the description's
// density and distribution; max_it = {iterations - lin, lin}, lin = iterations x mg_linear.
oct_status build_multigrid(oct_ctx* c, const oct_scene_desc* d, oct_scene* s) {
    if (d->solver != OCT_SOLVER_VBD || (d->element != kTetra10 && d->element != kHexa27))
        return fail(c, OCT_ENOTSUP, "multigrid VBD needs a P2 or Q2 VBD scene");
    if (d->rho > 0.f || d->order_mode != OCT_ORDER_ASCENDING)
        return fail(c, OCT_ENOTSUP, "multigrid VBD runs without Chebyshev and in the ascending colour order");
    if (!(d->mg_linear <= 1.f)) return fail(c, OCT_EINVAL, "mg_linear must be in (0, 1]");
    const int N = d->n_nodes, E = d->n_elements, NE = s->ne, NL = d->element == kTetra10 ? 4 : 8;
    std::vector<int32_t> compact(N, -1), back;
    for (int e = 0; e < E; ++e) for (int j = 0; j < NL; ++j) compact[d->topology[(size_t)e * NE + j]] = 0;
    for (int i = 0; i < N; ++i) if (compact[i] == 0) { compact[i] = (int32_t)back.size(); back.push_back(i); }
    std::vector<int32_t> lt((size_t)E * NL);
    for (int e = 0; e < E; ++e) for (int j = 0; j < NL; ++j) lt[(size_t)e * NL + j] = compact[d->topology[(size_t)e * NE + j]];
    std::vector<float> lx(3 * back.size());
    for (size_t k = 0; k < back.size(); ++k) for (int r = 0; r < 3; ++r) lx[3 * k + r] = d->positions[3 * back[k] + r];
    oct_scene_desc dl = *d;
    dl.element = d->element == kTetra10 ? kTetra : kHexa;
    dl.n_nodes = (int32_t)back.size();
    dl.positions = lx.data();
    dl.topology = lt.data();
    dl.masses = nullptr;
    dl.n_fixed = 0; dl.fixed_ids = nullptr; dl.fixed_group = nullptr; dl.fix_by_plane = 0;
    dl.initial_velocity = nullptr;
    dl.box_limit = 0;
    dl.threads_per_vertex = 0;
    dl.mg_linear = 0.f;
    auto* sub = new oct_scene();
    oct_status st = build_scene(c, &dl, sub);
    if (st) { sub->mem.release(); delete sub; return st; }
    s->mg_sub = sub;
    const int lin = (int)((float)s->iterations * d->mg_linear);
    s->mg_max[0] = s->iterations - lin;
    s->mg_max[1] = lin;
    s->mg_count = 0;
    s->mg_current = 1;
    // prolongation lists, first visit in element order (P1_to_P2 / Q1_to_Q2 ctors, :13-34,
    // :97-132); the reference's Q2 edge list ends with {7, 0} for node 19 (the edge is 7-4)
    std::vector<int32_t> pro[3];
    std::vector<char> seen(N, 0);
    const int32_t* t = d->topology;
    if (d->element == kTetra10) {
        static const int ed[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
        for (int e = 0; e < E; ++e)
            for (int j = 4; j < 10; ++j) {
                const int v = t[(size_t)e * 10 + j];
                if (seen[v]) continue;
                seen[v] = 1;
                pro[0].insert(pro[0].end(), {v, t[(size_t)e * 10 + ed[j - 4][0]], t[(size_t)e * 10 + ed[j - 4][1]]});
            }
    } else {
        static const int ed[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5}, {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 0}};
        static const int fc[6][4] = {{0, 1, 2, 3}, {0, 1, 4, 5}, {1, 2, 5, 6}, {2, 3, 6, 7}, {3, 0, 7, 4}, {4, 5, 6, 7}};
        for (int e = 0; e < E; ++e) {
            const int32_t* q = t + (size_t)e * 27;
            for (int k = 0; k < 12; ++k)
                if (!seen[q[8 + k]]) { seen[q[8 + k]] = 1; pro[0].insert(pro[0].end(), {q[8 + k], q[ed[k][0]], q[ed[k][1]]}); }
            for (int k = 0; k < 6; ++k)
                if (!seen[q[20 + k]]) {
                    seen[q[20 + k]] = 1;
                    pro[1].insert(pro[1].end(), {q[20 + k], q[fc[k][0]], q[fc[k][1]], q[fc[k][2]], q[fc[k][3]]});
                }
            pro[2].push_back(q[26]);
            for (int j = 0; j < 8; ++j) pro[2].push_back(q[j]);
        }
    }
    const int per[3] = {3, 5, 9};
    for (int k = 0; k < 3; ++k) {
        s->n_pro[k] = (int)pro[k].size() / per[k];
        if (s->n_pro[k] && (st = upload(c, s->mem, s->d_pro[k], pro[k]))) return st;
    }
    s->n_mg_map = (int)back.size();
    return upload(c, s->mem, s->d_mg_map, back);
}

oct_status build_scene(oct_ctx* c, const oct_scene_desc* d, oct_scene* s) {
    s->ctx = c;
    s->mem.ctx = c;
    s->solver = d->solver;
    s->element = d->element;
    s->material = d->material;
    s->young = d->young;
    s->poisson = d->poisson;
    s->density = d->density;
    s->ne = element_nodes(d->element);
    s->nq = element_quadrature(d->element);
    if (s->ne < 0) return fail(c, OCT_EINVAL, "unsupported element type");
    if (d->solver < 0 || d->solver > 2) return fail(c, OCT_EINVAL, "unknown solver");
    if (d->material < 0 || d->material > 5) return fail(c, OCT_EINVAL, "unsupported material");
    if (d->material > 3 && d->solver != OCT_SOLVER_XPBD)
        return fail(c, OCT_ENOTSUP, "Corotated and FixedCorotated are XPBD-only materials");
    if (d->xpbd_version < 0 || d->xpbd_version > 3) return fail(c, OCT_EINVAL, "unknown XPBD version");
    s->xpbd_raw = d->element != kTetra && (d->xpbd_version == OCT_XPBD_QUADRATURE || d->xpbd_version == OCT_XPBD_OPTISHARED);
    s->xpbd_project = d->element == kTetra || d->xpbd_version != OCT_XPBD_OPTIGROUP;
    if (d->n_nodes <= 0 || d->n_elements <= 0 || !d->positions || !d->topology) return fail(c, OCT_EINVAL, "empty mesh");
    s->n_nodes = d->n_nodes;
    s->n_elements = d->n_elements;
    const int N = s->n_nodes, E = s->n_elements, NE = s->ne, NQ = s->nq;
    for (int64_t k = 0; k < (int64_t)E * NE; ++k)
        if (d->topology[k] < 0 || d->topology[k] >= N) return fail(c, OCT_EINVAL, "topology index out of range");
    if ((int64_t)E >= (1ll << (31 - kOwnerShift))) return fail(c, OCT_EINVAL, "too many elements for one scene");
    oct_status st = ensure_tables(c, d->element);
    if (st) return st;
    if (d->solver != OCT_SOLVER_XPBD) {
        std::lock_guard<std::mutex> lock(c->mu);
        prepare_vertex(d->element, d->material);
    }
    s->iterations = std::max(1, d->iterations);
    s->rho = d->rho;
    s->order_mode = d->order_mode;
    s->rng.seed((unsigned)d->seed);
    s->precision = d->precision;
    s->global_damping = d->global_damping;
    s->box = d->box_limit != 0;
    s->has_v0 = d->initial_velocity != nullptr;
    s->tpv = d->threads_per_vertex < 0 ? 0 : d->threads_per_vertex;
    if (d->threads_per_vertex < -1 || (s->tpv != 0 && s->tpv != 1 && s->tpv != 2 && s->tpv != 4 && s->tpv != 8 &&
                                       s->tpv != 16 && s->tpv != 32))
        return fail(c, OCT_EINVAL, "threads_per_vertex must be -1 (packed), 0 (default) or a power of two <= 32");
    s->X.assign(d->positions, d->positions + 3 * (size_t)N);

    // masses (Cuda_FEM_Dynamic::get_fem_masses)
    if (d->masses) s->masses.assign(d->masses, d->masses + N);
    else lumped_masses(d->element, d->positions, N, d->topology, E, d->density, d->mass_distribution, s->masses);
    for (int i = 0; i < N; ++i)
        if (!(s->masses[i] > 0.f)) return fail(c, OCT_EINVAL, "non-positive node mass (node not in any element?)");

    // fixed nodes: explicit ids or Area::Plane test, ascending (GPU_Fix_Constraint ctor)
    if (d->fix_by_plane) {
        for (int i = 0; i < N; ++i) {
            const float* p = d->positions + 3 * i;
            const float v = (p[0] - d->plane_origin[0]) * d->plane_normal[0] + (p[1] - d->plane_origin[1]) * d->plane_normal[1] +
                            (p[2] - d->plane_origin[2]) * d->plane_normal[2];
            if (v > 0.f) s->fixed.push_back(i);
        }
    } else if (d->n_fixed > 0 && d->fixed_ids) {
        s->fixed.assign(d->fixed_ids, d->fixed_ids + d->n_fixed);
        for (int id : s->fixed) if (id < 0 || id >= N) return fail(c, OCT_EINVAL, "fixed id out of range");
    }
    s->n_fixed = (int)s->fixed.size();
    s->fixed_group.assign(s->n_fixed, 0);
    if (d->fixed_group && !d->fix_by_plane)
        for (int k = 0; k < s->n_fixed; ++k) {
            s->fixed_group[k] = d->fixed_group[k];
            if (d->fixed_group[k] < 0 || d->fixed_group[k] >= kFixGroups) return fail(c, OCT_EINVAL, "fixed group out of range");
        }
    // per group: centre of mass in float as GPU_Fix_Constraint (GPU_Constraint.cu:94-107),
    // zero offset, identity rotation
    for (int g = 0; g < kFixGroups; ++g) {
        float cx = 0, cy = 0, cz = 0;
        int cnt = 0;
        for (int k = 0; k < s->n_fixed; ++k) {
            if (s->fixed_group[k] != g) continue;
            const int id = s->fixed[k];
            cx += d->positions[3 * id]; cy += d->positions[3 * id + 1]; cz += d->positions[3 * id + 2];
            ++cnt;
        }
        if (cnt) { cx /= (float)cnt; cy /= (float)cnt; cz /= (float)cnt; }
        float* G = s->fix_host + 16 * g;
        G[0] = cx; G[1] = cy; G[2] = cz;
        for (int k = 0; k < 9; ++k) G[6 + k] = (k % 4 == 0) ? 1.f : 0.f;
    }

    // precompute per (element, quadrature point) in FP64 (GPU_FEM::build_fem_const,
    // octopus/src/GPU/GPU_FEM.cu:176-215) with the Lame parameters of GPU_FEM.cu:162-163
    ShapeTable sh;
    shape_table(d->element, sh);
    std::vector<float4> eq((size_t)E * NQ * 3);
    for (int e = 0; e < E; ++e) {
        const double Y = d->young_per_element ? d->young_per_element[e] : d->young, nu = d->poisson;
        const float lam = (float)(Y * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))), mu = (float)(Y / (2.0 * (1.0 + nu)));
        for (int q = 0; q < NQ; ++q) {
            double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // J[col][row] = sum_k X_k[row] dN_qk[col]
            for (int k = 0; k < NE; ++k) {
                const float* x = d->positions + 3 * d->topology[(size_t)e * NE + k];
                const double* dn = &sh.dN[((size_t)q * NE + k) * 3];
                for (int cc = 0; cc < 3; ++cc) for (int r = 0; r < 3; ++r) J[cc][r] += (double)x[r] * dn[cc];
            }
            const double det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) - J[1][0] * (J[0][1] * J[2][2] - J[2][1] * J[0][2]) +
                               J[2][0] * (J[0][1] * J[1][2] - J[1][1] * J[0][2]);
            if (!(std::fabs(det) > 0.0)) return fail(c, OCT_EINVAL, "degenerate element " + std::to_string(e));
            const double id = 1.0 / det;
            double I[3][3];   // inverse, I[col][row]
            I[0][0] = (J[1][1] * J[2][2] - J[2][1] * J[1][2]) * id;
            I[1][0] = -(J[1][0] * J[2][2] - J[2][0] * J[1][2]) * id;
            I[2][0] = (J[1][0] * J[2][1] - J[2][0] * J[1][1]) * id;
            I[0][1] = -(J[0][1] * J[2][2] - J[2][1] * J[0][2]) * id;
            I[1][1] = (J[0][0] * J[2][2] - J[2][0] * J[0][2]) * id;
            I[2][1] = -(J[0][0] * J[2][1] - J[2][0] * J[0][1]) * id;
            I[0][2] = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * id;
            I[1][2] = -(J[0][0] * J[1][2] - J[1][0] * J[0][2]) * id;
            I[2][2] = (J[0][0] * J[1][1] - J[1][0] * J[0][1]) * id;
            float4* r = &eq[((size_t)e * NQ + q) * 3];
            r[0] = make_float4((float)I[0][0], (float)I[0][1], (float)I[0][2], (float)I[1][0]);
            r[1] = make_float4((float)I[1][1], (float)I[1][2], (float)I[2][0], (float)I[2][1]);
            r[2] = make_float4((float)I[2][2], (float)std::fabs(det), lam, mu);
        }
    }
    // affine element maps (J the same at every quadrature point up to rounding, 1e-6
    // relative): one record per element
    bool affine = NQ > 1;
    for (size_t e = 0; e < (size_t)E && affine; ++e) {
        const float* r0 = reinterpret_cast<const float*>(&eq[e * NQ * 3]);
        float scale = 0.f;
        for (int k = 0; k < 9; ++k) scale = std::max(scale, std::fabs(r0[k]));
        for (int q = 1; q < NQ && affine; ++q) {
            const float* rq = reinterpret_cast<const float*>(&eq[(e * NQ + q) * 3]);
            for (int k = 0; k < 9; ++k) affine = affine && std::fabs(rq[k] - r0[k]) <= 1e-6f * scale;
            affine = affine && std::fabs(rq[9] - r0[9]) <= 1e-6f * std::fabs(r0[9]);
        }
    }
    if (affine) {
        for (size_t e = 1; e < (size_t)E; ++e) std::memmove(&eq[e * 3], &eq[e * NQ * 3], 3 * sizeof(float4));
        eq.resize((size_t)E * 3);
    }
    s->h.eq_stride = affine || NQ == 1 ? 1 : NQ;

    // colouring and slot order
    std::vector<int32_t> slot_vids;
    std::vector<std::vector<int32_t>> elems_by_color;
    if (d->solver == OCT_SOLVER_VBD) {
        PrimalGraph g;
        build_primal_graph(NE, d->topology, E, N, g);
        Coloring col = d->color_algo == OCT_COLOR_GREEDY ? color_greedy(g) : color_dsat(g);
        if (d->vbd_version == OCT_VBD_BETTER_COLORATION && d->target_color > 0 && d->target_color < col.n_colors)
            color_reduction(g, col, d->target_color);
        s->in_place = count_conflicts(g, col) == 0;
        s->colors = col.colors;
        s->n_colors = col.n_colors;
    } else if (d->solver == OCT_SOLVER_XPBD) {
        PrimalGraph g;
        build_dual_vertex_graph(NE, d->topology, E, N, g);
        Coloring col = color_greedy_slf(g);
        s->n_colors = col.n_colors;
        s->colors.assign(N, 0);
        elems_by_color.assign(col.n_colors, {});
        for (int e = 0; e < E; ++e) elems_by_color[col.colors[e]].push_back(e);   // build_thread_by_color
    } else {
        s->n_colors = 1;
        s->colors.assign(N, 0);
    }
    if (d->solver == OCT_SOLVER_XPBD) {
        s->n_colors = (int)elems_by_color.size();
        s->elem_off.assign(1, 0);
        std::vector<int32_t> flat;
        for (auto& v : elems_by_color) { flat.insert(flat.end(), v.begin(), v.end()); s->elem_off.push_back((int)flat.size()); }
        if ((st = upload(c, s->mem, s->d_elems, flat))) return st;
        // the topology in colour order: a block's node ids follow from its work item directly,
        // one dependent load fewer before the gathers (element ids only index the records)
        std::vector<int32_t> etopo(flat.size() * (size_t)NE);
        for (size_t k = 0; k < flat.size(); ++k)
            std::copy(d->topology + (size_t)flat[k] * NE, d->topology + (size_t)(flat[k] + 1) * NE, etopo.begin() + k * NE);
        if ((st = upload(c, s->mem, s->d_etopo, etopo))) return st;
        std::vector<XWork> xw;
        s->xwork_off.assign(1, 0);
        for (int k = 0; k + 1 < (int)s->elem_off.size(); ++k) {
            append_xwork(xw, 0, s->elem_off[k], s->elem_off[k + 1], xpbd_elements_per_block(d->element));
            s->xwork_off.push_back((int)xw.size());
        }
        if ((st = upload(c, s->mem, s->d_xwork, xw))) return st;
        // VBD-style slots are unused; keep the identity order for the getters
        for (int i = 0; i < N; ++i) slot_vids.push_back(i);
        s->color_off = {0, N};
    } else {
        const int C = s->n_colors;
        s->color_off.assign(C + 1, 0);
        for (int i = 0; i < N; ++i) s->color_off[s->colors[i] + 1]++;
        for (int k = 0; k < C; ++k) s->color_off[k + 1] += s->color_off[k];
        slot_vids.resize(N);
        std::vector<int> fillp(s->color_off.begin(), s->color_off.end() - 1);
        for (int i = 0; i < N; ++i) slot_vids[fillp[s->colors[i]]++] = i;   // ascending id within colour
    }
    s->vids = slot_vids;   // the reference order (GPU_VBD_FEM::create_buffers), reported by the getters
    // processing order: within each colour, vertices by decreasing owner count (ascending id
    // among equals), so the lanes of a warp get similar loads; results do not depend on the
    // order inside a colour.  (A Morton order of the rest positions among equals, tried so
    // that a warp's vertices share element nodes in L1, was not faster.)
    if (d->solver != OCT_SOLVER_XPBD) {
        std::vector<int32_t> val(N, 0);
        for (int64_t k = 0; k < (int64_t)E * NE; ++k) val[d->topology[k]]++;
        for (int k = 0; k + 1 < (int)s->color_off.size(); ++k)
            std::stable_sort(slot_vids.begin() + s->color_off[k], slot_vids.begin() + s->color_off[k + 1],
                             [&](int a, int b) { return val[a] > val[b]; });
    }

    // owner CSR in slot order (build_owner_data, GPU_VBD_FEM.cu:677-690: element order)
    std::vector<int32_t> cnt(N, 0);
    for (int64_t k = 0; k < (int64_t)E * NE; ++k) cnt[d->topology[k]]++;
    std::vector<int64_t> voff(N + 1, 0);
    for (int i = 0; i < N; ++i) voff[i + 1] = voff[i] + cnt[i];
    std::vector<int32_t> vown(voff[N]);
    std::vector<int64_t> vf(voff.begin(), voff.end() - 1);
    for (int e = 0; e < E; ++e)
        for (int j = 0; j < NE; ++j) vown[vf[d->topology[(size_t)e * NE + j]]++] = (e << kOwnerShift) | j;
    std::vector<int32_t> own_off(N + 1, 0), owners;
    owners.reserve(vown.size());
    int max_valence = 0;
    for (int sl = 0; sl < N; ++sl) {
        const int v = slot_vids[sl];
        owners.insert(owners.end(), vown.begin() + voff[v], vown.begin() + voff[v + 1]);
        own_off[sl + 1] = (int32_t)owners.size();
        max_valence = std::max(max_valence, own_off[sl + 1] - own_off[sl]);
    }
    // default mapping (per-colour sweep times measured on the batched workload): P1 tetrahedra
    // and Q1 hexahedra use 4 lanes per vertex, P2 tetrahedra 1 (4 on the corner colours, by
    // kOwnersPerLane; P2 sweep 1.672 ms against 1.730 ms with 2), each lane looping over a
    // share of the vertex's owners; the other elements one lane per (vertex, owner) pair packed into
    // warps; vertices with more than 32 owners fall back to a lane group per vertex
    if (d->threads_per_vertex == 0) s->tpv = measured_tpv(d->element);
    if (s->tpv == 0 && max_valence > 32) s->tpv = max_valence > 64 ? 32 : default_tpv(d->element);
    s->max_valence = max_valence;
    s->own_off = own_off;

    // device state
    std::vector<float4> X4(N), y4(N), zero4(N, make_float4(0, 0, 0, 0)), v4(N, make_float4(0, 0, 0, 0));
    for (int i = 0; i < N; ++i) {
        X4[i] = make_float4(d->positions[3 * i], d->positions[3 * i + 1], d->positions[3 * i + 2], 0.f);
        y4[i] = make_float4(0.f, 0.f, 0.f, s->masses[i]);
        if (d->initial_velocity)
            v4[i] = make_float4(d->initial_velocity[3 * i], d->initial_velocity[3 * i + 1], d->initial_velocity[3 * i + 2], 0.f);
    }
    std::vector<int32_t> mask(N, 1);
    std::vector<int32_t> topo(d->topology, d->topology + (size_t)E * NE);
    SceneDev& h = s->h;
    float4 *u, *ul, *y, *v, *un, *p1 = nullptr, *p2 = nullptr, *Xd;
    if ((st = upload(c, s->mem, u, zero4)) || (st = upload(c, s->mem, ul, zero4)) || (st = upload(c, s->mem, y, y4)) ||
        (st = upload(c, s->mem, v, v4)) || (st = upload(c, s->mem, Xd, X4)))
        return st;
    if ((st = s->mem.alloc(un, N))) return st;
    OCT_CUDA(c, cudaMemset(un, 0, sizeof(float4) * N));
    if (s->rho > 0.f) {
        if ((st = upload(c, s->mem, p1, zero4)) || (st = upload(c, s->mem, p2, zero4))) return st;
    }
    int *maskd, *topod, *vidsd, *offd, *ownd, *fixd = nullptr;
    float4* eqd;
    if ((st = upload(c, s->mem, maskd, mask)) || (st = upload(c, s->mem, topod, topo)) || (st = upload(c, s->mem, eqd, eq)) ||
        (st = upload(c, s->mem, vidsd, slot_vids)) || (st = upload(c, s->mem, offd, own_off)) || (st = upload(c, s->mem, ownd, owners)))
        return st;
    int* fgd = nullptr;
    if (s->n_fixed && ((st = upload(c, s->mem, fixd, s->fixed)) || (st = upload(c, s->mem, fgd, s->fixed_group)))) return st;
    if ((st = upload(c, s->mem, s->d_fix, std::vector<float>(s->fix_host, s->fix_host + kFixGroups * 16)))) return st;
    h.u = u; h.u_last = ul; h.y = y; h.v = v; h.u_new = un; h.prev1 = p1; h.prev2 = p2; h.mask = maskd; h.X = Xd;
    h.topo = topod; h.eq = eqd; h.vids = vidsd; h.own_off = offd; h.owners = ownd; h.fixed = fixd;
    h.fixed_group = fgd; h.fix = s->d_fix;
    if (d->solver == OCT_SOLVER_EXPLICIT && s->n_fixed) {   // the explicit update applies the fixation itself
        std::vector<int32_t> fix_of(N, -1);
        for (int k = 0; k < s->n_fixed; ++k) fix_of[s->fixed[k]] = s->fixed_group[k];
        int* fod;
        if ((st = upload(c, s->mem, fod, fix_of))) return st;
        h.fix_of = fod;
    }
    h.n_nodes = N; h.n_elements = E; h.n_fixed = s->n_fixed; h.element = d->element;
    h.damping = d->damping;
    h.gx = d->gravity[0]; h.gy = d->gravity[1]; h.gz = d->gravity[2];
    h.bminx = d->box_min[0]; h.bminy = d->box_min[1]; h.bminz = d->box_min[2];
    h.bmaxx = d->box_max[0]; h.bmaxy = d->box_max[1]; h.bmaxz = d->box_max[2];
    h.box_limit = s->box;
    h.precision = s->precision;
    // owner entries in slot order (EntryLayout in device.cuh) and the table of distinct
    // records they index; without entries (node ids past kIdBits, or more distinct P1 corner
    // records than the P1 entry can index) the colour kernels read owners, topology and records
    h.ent = nullptr;
    h.rtab = nullptr;
    if ((int64_t)N <= (int64_t)kIdMask + 1) {
        const int EW = entry_words(NE);
        const bool affine = h.eq_stride == 1;
        // distinct records, compared bit for bit (identical records give identical results)
        struct KeyHash {
            size_t operator()(const std::array<uint32_t, 12>& k) const {
                uint64_t h = 1469598103934665603ull;
                for (uint32_t v : k) { h ^= v; h *= 1099511628211ull; }
                return (size_t)h;
            }
        };
        std::unordered_map<std::array<uint32_t, 12>, int32_t, KeyHash> index;
        std::vector<float4> rtab;
        auto intern = [&](const float* rec12) {
            std::array<uint32_t, 12> k;
            std::memcpy(k.data(), rec12, sizeof(k));
            auto it = index.find(k);
            if (it != index.end()) return it->second;
            const int32_t id = (int32_t)(rtab.size() / 3);
            index.emplace(k, id);
            rtab.push_back(make_float4(rec12[0], rec12[1], rec12[2], rec12[3]));
            rtab.push_back(make_float4(rec12[4], rec12[5], rec12[6], rec12[7]));
            rtab.push_back(make_float4(rec12[8], rec12[9], rec12[10], rec12[11]));
            return id;
        };
        std::vector<int32_t> erec;   // per element (affine, not P1): its record index
        if (affine && NE != 4) {
            erec.resize(E);
            for (int e = 0; e < E; ++e) erec[e] = intern(reinterpret_cast<const float*>(&eq[(size_t)e * 3]));
        }
        std::vector<float4> ent((size_t)owners.size() * EW / 4, make_float4(0, 0, 0, 0));
        bool ok = true;
        for (size_t o = 0; o < owners.size() && ok; ++o) {
            int32_t* ei = reinterpret_cast<int32_t*>(&ent[o * EW / 4]);
            const int eid = owners[o] >> kOwnerShift, r = owners[o] & ((1 << kOwnerShift) - 1);
            const int32_t* te = &topo[(size_t)eid * NE];
            if (NE == 4) {
                // own node first, then the others in element order with G_j = JX_inv^T dN_j
                // (FP64 from the stored JX_inv columns m_b; dN_j from the shape table)
                const float* m = reinterpret_cast<const float*>(&eq[(size_t)eid * 3]);
                float rec[12];
                ei[0] = te[r];
                for (int i = 0, j = 1; i < NE; ++i) {
                    if (i == r) continue;
                    ei[j] = te[i];
                    const double* dn = &sh.dN[(size_t)i * 3];
                    for (int b = 0; b < 3; ++b)
                        rec[3 * (j - 1) + b] = (float)((double)m[3 * b] * dn[0] + (double)m[3 * b + 1] * dn[1] +
                                                       (double)m[3 * b + 2] * dn[2]);
                    ++j;
                }
                rec[9] = m[9];     // V
                rec[10] = m[10];   // lambda
                rec[11] = m[11];   // mu
                const int32_t id = intern(rec);
                if ((long long)id >= (1ll << (4 * kSpareBits))) { ok = false; break; }
                for (int j = 0; j < 4; ++j) ei[j] |= (int32_t)(((uint32_t)id >> (kSpareBits * j)) & ((1u << kSpareBits) - 1)) << kIdBits;
                continue;
            }
            const int32_t rec = affine ? erec[eid] : eid;
            for (int i = 0; i < NE; ++i) ei[i] = te[i];
            if (NE == 8) {
                ei[0] |= r << kIdBits;
                for (int j = 1; j < 8; ++j)
                    ei[j] |= (int32_t)((((uint64_t)(uint32_t)rec) >> (kSpareBits * (j - 1))) & ((1u << kSpareBits) - 1)) << kIdBits;
            } else {
                ei[NE] = r;
                ei[NE + 1] = rec;
            }
        }
        if (ok) {
            float4* entd;
            if ((st = upload(c, s->mem, entd, ent))) return st;
            h.ent = entd;
            if (!rtab.empty()) {
                float4* rtd;
                if ((st = upload(c, s->mem, rtd, rtab))) return st;
                h.rtab = rtd;
            }
            s->n_records = (int64_t)rtab.size() / 3;
        }
    }
    if (!h.ent && s->tpv == 0) s->tpv = default_tpv(d->element);   // the packed mapping streams entries
    for (int k = 0; k < kMaxEffects; ++k) { s->effects[k] = EffectDev{}; s->effects[k].kind = -1; }
    if ((st = upload(c, s->mem, s->d_effects, std::vector<EffectDev>(s->effects, s->effects + kMaxEffects)))) return st;
    h.effects = s->d_effects;
    h.elems = s->d_elems;
    h.etopo = s->d_etopo;
    h.global_damping = s->global_damping;
    if ((st = upload(c, s->mem, s->d_status, std::vector<int>{0}))) return st;
    h.status = s->d_status;
    s->topo_host.assign(d->topology, d->topology + (size_t)E * NE);
    if ((st = s->mem.alloc(s->d_scene, 1))) return st;
    OCT_CUDA(c, cudaMemcpy(s->d_scene, &h, sizeof(SceneDev), cudaMemcpyHostToDevice));
    // VBD moves by its implicit velocity, so an initial velocity waits for the first sub-step's
    // predictor; XPBD and explicit step the velocity array itself, which already holds it
    s->pending_host = s->has_v0 && d->solver == OCT_SOLVER_VBD ? 1 : 0;
    if ((st = upload(c, s->mem, s->d_pending, std::vector<int>{s->pending_host}))) return st;
    if ((st = s->mem.alloc(s->d_red, 4))) return st;
    if (d->solver == OCT_SOLVER_EXPLICIT && (st = s->mem.alloc(s->d_contrib, (size_t)E * NE))) return st;

    // work tables
    if ((st = build_vertex_work(s))) return st;
    std::vector<NWork> nw, fw;
    append_nwork(nw, 0, N);
    append_nwork(fw, 0, s->n_fixed);
    s->n_nwork = (int)nw.size();
    s->n_fwork = (int)fw.size();
    if ((st = upload(c, s->mem, s->d_nwork, nw)) || (st = upload(c, s->mem, s->d_fwork, fw))) return st;
    if (d->mg_linear > 0.f) return build_multigrid(c, d, s);
    return OCT_OK;
}

StepParams base_params(oct_ctx* c, float dt) {
    StepParams P{};
    P.dt = dt;
    P.inv_dt = 1.f / dt;
    P.omega = 1.f;
    P.error = c->d_error;
    return P;
}

void mg_prolong(oct_scene* s, cudaStream_t st) {
    const int k[3] = {2, 4, 8};
    const float w[3] = {0.5f, 0.25f, 0.125f};
    for (int i = 0; i < 3; ++i) {
        launch_mg_prolong(s->d_scene, s->d_pro[i], s->n_pro[i], k[i], w[i], st);
        if (s->n_pro[i]) s->ctx->launches++;
    }
}

// Scripted effects of one scene, in creation order (each a no-op while inactive).
void enqueue_effects(oct_scene* s, float dt, cudaStream_t st) {
    for (int k = 0; k < s->n_effects; ++k) {
        launch_effect(s->d_scene, s->d_nwork, s->n_nwork, k, s->effects[k].kind, dt, st);
        s->ctx->launches++;
    }
}

// One GPU_VBD::step (octopus/src/GPU/VBD/GPU_VBD.cu:38-61) of one scene with the reference's
// launch structure: predictor, iterations x (one launch per colour [+ commit] + constraints
// [+ Chebyshev]), velocity update.
void vbd_substep(oct_scene* s, float dt) {
    Range range("vbd_substep");
    oct_ctx* c = s->ctx;
    cudaStream_t st = c->stream;
    StepParams P = base_params(c, dt);
    P.pending_v0 = s->d_pending;
    P.in_place = s->in_place ? 1 : 0;
    const bool cheb = s->rho > 0.f && s->rho > 1.17549435e-38f * 1e6f;
    launch_predict(s->d_scene, s->d_nwork, s->n_nwork, 0, 0, cheb ? 1 : 0, P, st);
    c->launches++;
    if (s->pending_host) {
        cudaMemsetAsync(s->d_pending, 0, sizeof(int), st);
        s->pending_host = 0;
    }
    std::vector<int> order(s->n_colors);
    float omega = 1.f;
    for (int j = 0; j < s->iterations; ++j) {
        if (s->mg_sub) {
            // MG_VBD_FEM::solve schedule: mg_max[1] iterations on the linear level, then
            // mg_max[0] on the full one, counted across sub-steps; entering the linear level
            // prolongs the mid nodes first
            const int last = s->mg_current;
            s->mg_count++;
            while (s->mg_count > s->mg_max[s->mg_current]) { s->mg_count = 1; s->mg_current = (s->mg_current + 1) % 2; }
            if (s->mg_current == 1) {
                if (last != 1) mg_prolong(s, st);
                oct_scene* L = s->mg_sub;
                launch_mg_copy(s->d_scene, L->d_scene, s->d_mg_map, s->n_mg_map, 0, st);
                StepParams PL = P;
                PL.in_place = L->in_place ? 1 : 0;
                PL.pending_v0 = nullptr;
                for (int k = 0; k < L->n_colors; ++k) {
                    const int b = L->vwork_off[k], n = L->vwork_off[k + 1] - b;
                    launch_vertex(L->element, L->material, L->d_scene, L->d_vwork + b, n, L->tpv, 0, PL, nullptr, st);
                    if (!L->in_place) launch_commit(L->d_scene, L->d_vwork + b, n, st);
                    c->launches += L->in_place ? 1 : 2;
                }
                launch_mg_copy(s->d_scene, L->d_scene, s->d_mg_map, s->n_mg_map, 1, st);
                c->launches += 2;
                if (s->n_fixed) { launch_constraints(s->d_scene, s->d_fwork, s->n_fwork, 0, st); c->launches++; }
                enqueue_effects(s, dt, st);
                if (s->box) { launch_constraints(s->d_scene, s->d_nwork, s->n_nwork, 1, st); c->launches++; }
                mg_prolong(s, st);   // MG_VertexBlockDescent::step interpolates after every iteration
                continue;
            }
        }
        std::iota(order.begin(), order.end(), 0);
        if (s->order_mode == OCT_ORDER_SHUFFLED) std::shuffle(order.begin(), order.end(), s->rng);
        Range sweep("colour_sweep");
        for (int k : order) {
            const int b = s->vwork_off[k], n = s->vwork_off[k + 1] - b;
            launch_vertex(s->element, s->material, s->d_scene, s->d_vwork + b, n, s->tpv, 0, P, nullptr, st);
            c->launches++;
            if (!s->in_place) { launch_commit(s->d_scene, s->d_vwork + b, n, st); c->launches++; }
        }
        if (s->n_fixed) { launch_constraints(s->d_scene, s->d_fwork, s->n_fwork, 0, st); c->launches++; }
        enqueue_effects(s, dt, st);
        if (s->box) { launch_constraints(s->d_scene, s->d_nwork, s->n_nwork, 1, st); c->launches++; }
        if (cheb) {
            if (j == 1) omega = 2.f / (2.f - s->rho * s->rho);
            else if (j > 1) omega = 4.f / (4.f - s->rho * s->rho * omega);
            P.omega = omega;
            P.iteration = j;
            launch_chebyshev(s->d_scene, s->d_nwork, s->n_nwork, P, st);
            c->launches++;
        }
    }
    launch_velocity(s->d_scene, s->d_nwork, s->n_nwork, 0, P, st);
    c->launches++;
}

// GPU_PBD::step (octopus/src/GPU/PBD/GPU_PBD.cu:20-26).
void xpbd_substep(oct_scene* s, float dt) {
    Range range("xpbd_substep");
    oct_ctx* c = s->ctx;
    cudaStream_t st = c->stream;
    StepParams P = base_params(c, dt);
    launch_predict(s->d_scene, s->d_nwork, s->n_nwork, 1, 0, 0, P, st);
    c->launches++;
    for (int k = 0; k < s->n_colors && s->xpbd_project; ++k) {
        launch_xpbd(s->element, s->material, s->xpbd_raw, s->d_scene, s->d_xwork + s->xwork_off[k],
                    s->xwork_off[k + 1] - s->xwork_off[k], P, st);
        c->launches++;
    }
    if (s->n_fixed) { launch_constraints(s->d_scene, s->d_fwork, s->n_fwork, 0, st); c->launches++; }
    enqueue_effects(s, dt, st);
    if (s->box) { launch_constraints(s->d_scene, s->d_nwork, s->n_nwork, 1, st); c->launches++; }
    launch_velocity(s->d_scene, s->d_nwork, s->n_nwork, 1, P, st);
    c->launches++;
}

// GPU_SemiExplicit::step (octopus/src/GPU/GPU_Integrator.cu:36-42).
void explicit_substep(oct_scene* s, float dt) {
    Range range("explicit_substep");
    oct_ctx* c = s->ctx;
    cudaStream_t st = c->stream;
    StepParams P = base_params(c, dt);
    // element-centric force pass, then per node the sum over its owners and the semi-implicit
    // Euler update (GPU_FEM_Explicit::step then GPU_SemiExplicit's integration)
    launch_explicit_force(s->element, s->material, s->d_scene, s->n_elements, s->d_contrib, s->d_nwork, s->n_nwork, P, st);
    c->launches += 2;   // the fixation runs inside the update kernel (SceneDev::fix_of)
    enqueue_effects(s, dt, st);
    if (s->box) { launch_constraints(s->d_scene, s->d_nwork, s->n_nwork, 1, st); c->launches++; }
}

// Node state out: converted to n x 3 floats on the device and read back in one copy (the
// caller's buffer may be pinned or pageable); returns when `out` holds the values.
oct_status read_nodes(oct_scene* s, const float4* d, float* out, bool add_rest) {
    oct_ctx* c = s->ctx;
    oct_status st;
    if (!s->d_io && (st = s->mem.alloc(s->d_io, (size_t)s->n_nodes * 3))) return st;
    launch_nodes_out(d, add_rest ? s->h.X : nullptr, s->d_io, s->n_nodes, c->stream);
    OCT_CUDA(c, cudaMemcpyAsync(out, s->d_io, sizeof(float) * 3 * s->n_nodes, cudaMemcpyDeviceToHost, c->stream));
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    return OCT_OK;
}

// Node state in: one copy of the caller's n x 3 floats, converted on the device; returns when
// the caller may reuse `in`.
oct_status write_nodes(oct_scene* s, const float* in, float4* d, bool sub_rest) {
    oct_ctx* c = s->ctx;
    oct_status st;
    if (!s->d_io && (st = s->mem.alloc(s->d_io, (size_t)s->n_nodes * 3))) return st;
    OCT_CUDA(c, cudaMemcpyAsync(s->d_io, in, sizeof(float) * 3 * s->n_nodes, cudaMemcpyHostToDevice, c->stream));
    launch_nodes_in(s->d_io, sub_rest ? s->h.X : nullptr, d, s->n_nodes, c->stream);
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    return OCT_OK;
}

void run_frame(oct_scene* s, float sub, int substeps) {
    for (int k = 0; k < substeps; ++k) {
        if (s->solver == OCT_SOLVER_VBD) vbd_substep(s, sub);
        else if (s->solver == OCT_SOLVER_XPBD) xpbd_substep(s, sub);
        else explicit_substep(s, sub);
    }
}
void drop_frame_graph(oct_scene* s) {
    if (s->frame_exec) cudaGraphExecDestroy(s->frame_exec);
    s->frame_exec = nullptr;
    s->frame_dt = -1.f;
    s->frame_substeps = 0;
}
}  // namespace

// ============================================================================ C ABI
extern "C" {

void oct_desc_init(oct_scene_desc* d) {
    std::memset(d, 0, sizeof(*d));
    d->solver = OCT_SOLVER_VBD;
    d->element = OCT_TETRA;
    d->density = 1000.f;
    d->mass_distribution = OCT_MASS_FEMSHAPE;
    d->material = OCT_STABLE_NEOHOOKE;
    d->young = 1e6f;
    d->poisson = 0.45f;
    d->gravity[1] = -9.81f;
    d->iterations = 1;
    d->vbd_version = OCT_VBD_REDUCTION_SYMMETRY;
    d->target_color = -1;
    d->color_algo = OCT_COLOR_DSAT;
    d->precision = OCT_PREC_PLAIN;
    d->xpbd_version = OCT_XPBD_OPTISHARED;
    d->mg_linear = 0.f;
    for (int k = 0; k < 3; ++k) { d->box_min[k] = -1e30f; d->box_max[k] = 1e30f; }
}

oct_status oct_ctx_create(int device, size_t budget, oct_ctx** out) {
    if (!out) return OCT_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return OCT_ECUDA;
    if (device < 0 || device >= n) return OCT_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return OCT_ECUDA;
    auto* c = new oct_ctx();
    c->device = device;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    c->budget = budget ? budget : (size_t)(0.9 * (double)fr);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess || cudaMalloc(&c->d_error, sizeof(int)) != cudaSuccess ||
        cudaMemset(c->d_error, 0, sizeof(int)) != cudaSuccess || cudaEventCreate(&c->ev0) != cudaSuccess ||
        cudaEventCreate(&c->ev1) != cudaSuccess) {
        delete c;
        return OCT_ECUDA;
    }
    *out = c;
    return OCT_OK;
}

oct_status oct_ctx_destroy(oct_ctx* c) {
    if (!c) return OCT_EINVAL;
    cudaStreamSynchronize(c->stream);
    {
        std::lock_guard<std::mutex> lock(c->mu);
        trim_cache(c);
    }
    cudaFree(c->d_error);
    cudaEventDestroy(c->ev0);
    cudaEventDestroy(c->ev1);
    cudaStreamDestroy(c->stream);
    delete c;
    return OCT_OK;
}

const char* oct_last_error(oct_ctx* c) { return c ? c->err.c_str() : "null context"; }

oct_status oct_ctx_memory(oct_ctx* c, size_t* used, size_t* budget) {
    if (!c) return OCT_EINVAL;
    if (used) *used = c->used;
    if (budget) *budget = c->budget;
    return OCT_OK;
}

oct_status oct_scene_footprint(const oct_scene_desc* d, size_t* bytes) {
    if (!d || !bytes) return OCT_EINVAL;
    const int ne = element_nodes(d->element), nq = element_quadrature(d->element);
    if (ne < 0 || d->n_nodes <= 0 || d->n_elements <= 0) return OCT_EINVAL;
    const size_t N = d->n_nodes, E = d->n_elements;
    size_t b = N * (6 * sizeof(float4) + 3 * sizeof(int)) + (d->rho > 0.f ? 2 * N * sizeof(float4) : 0);
    b += E * ne * sizeof(int) * 2 + E * nq * 3 * sizeof(float4);   // topology, owners, quadrature records
    b += E * ne * (size_t)entry_words(ne) * sizeof(float);                  // owner entries
    b += (ne == 4 ? 4 : 1) * E * 3 * sizeof(float4);                        // distinct records, at most
    if (d->solver == OCT_SOLVER_EXPLICIT) b += E * ne * sizeof(float4) + N * sizeof(int);   // contributions, fixation map
    b += (N / 16 + 64) * sizeof(VWork) + (N / 256 + 8) * 2 * sizeof(NWork) + (size_t)std::max(d->n_fixed, 0) * sizeof(int);
    if (d->solver == OCT_SOLVER_XPBD) b += E * (ne + 1) * sizeof(int);   // colour-sorted element ids and topology
    b += 4096;   // descriptors and reduction scratch
    *bytes = b;
    return OCT_OK;
}

oct_status oct_scene_create(oct_ctx* c, const oct_scene_desc* d, oct_scene** out) {
    if (!c || !d || !out) return OCT_EINVAL;
    *out = nullptr;
    cudaSetDevice(c->device);
    auto* s = new oct_scene();
    oct_status st = build_scene(c, d, s);
    if (st) { s->mem.release(); delete s; return st; }
    *out = s;
    return OCT_OK;
}

oct_status oct_scene_destroy(oct_scene* s) {
    if (!s) return OCT_EINVAL;
    cudaStreamSynchronize(s->ctx->stream);
    if (s->mg_sub) oct_scene_destroy(s->mg_sub);
    drop_frame_graph(s);
    s->mem.release();
    delete s;
    return OCT_OK;
}

oct_status oct_scene_step(oct_scene* s, float frame_dt, int substeps) {
    if (!s || substeps <= 0 || !(frame_dt > 0.f)) return OCT_EINVAL;
    Range range("oct_scene_step");
    oct_ctx* c = s->ctx;
    const float sub = frame_dt / (float)substeps;
    s->last_substeps = substeps;
    // the first frame after set-up (pending initial velocity) and shuffled colour orders run
    // launch by launch; otherwise a captured frame is replayed
    const bool graph = s->capture && s->order_mode != OCT_ORDER_SHUFFLED && !s->pending_host && !s->mg_sub;
    if (graph && (!s->frame_exec || s->frame_dt != frame_dt || s->frame_substeps != substeps)) {
        drop_frame_graph(s);
        const uint64_t l0 = c->launches;
        OCT_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        run_frame(s, sub, substeps);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        s->frame_launches = c->launches - l0;
        c->launches = l0;
        if (e != cudaSuccess) return fail(c, OCT_ECUDA, std::string("frame capture: ") + cudaGetErrorString(e));
        const cudaError_t ei = cudaGraphInstantiate(&s->frame_exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            s->frame_exec = nullptr;
            return fail(c, OCT_ECUDA, std::string("frame graph: ") + cudaGetErrorString(ei));
        }
        s->frame_dt = frame_dt;
        s->frame_substeps = substeps;
    }
    cudaEventRecord(c->ev0, c->stream);
    if (graph) {
        OCT_CUDA(c, cudaGraphLaunch(s->frame_exec, c->stream));
        c->launches += s->frame_launches;
    } else {
        run_frame(s, sub, substeps);
    }
    cudaEventRecord(c->ev1, c->stream);
    OCT_CUDA(c, cudaGetLastError());
    return OCT_OK;
}

oct_status oct_scene_set_capture(oct_scene* s, int on) {
    if (!s) return OCT_EINVAL;
    OCT_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    s->capture = on != 0;
    drop_frame_graph(s);
    return OCT_OK;
}

oct_status oct_scene_sync(oct_scene* s) {
    if (!s) return OCT_EINVAL;
    oct_ctx* c = s->ctx;
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1);
    return check_error_word(c);
}

oct_status oct_scene_get_positions(oct_scene* s, float* out) {
    if (!s || !out) return OCT_EINVAL;
    return read_nodes(s, s->h.u, out, true);
}
oct_status oct_scene_get_velocities(oct_scene* s, float* out) {
    if (!s || !out) return OCT_EINVAL;
    return read_nodes(s, s->h.v, out, false);
}
oct_status oct_scene_set_positions(oct_scene* s, const float* in) {
    if (!s || !in) return OCT_EINVAL;
    return write_nodes(s, in, s->h.u, true);
}
oct_status oct_scene_set_velocities(oct_scene* s, const float* in) {
    if (!s || !in) return OCT_EINVAL;
    oct_status st = write_nodes(s, in, s->h.v, false);
    if (st || s->solver != OCT_SOLVER_VBD) return st;
    // VBD moves by the implicit velocity (p - last_p) / dt; like an initial velocity, the set
    // velocities become it at the scene's next sub-step (u_last = u - v dt in the predictor)
    s->pending_host = 1;
    OCT_CUDA(s->ctx, cudaMemcpy(s->d_pending, &s->pending_host, sizeof(int), cudaMemcpyHostToDevice));
    return OCT_OK;
}

oct_status oct_scene_info(oct_scene* s, int32_t* nn, int32_t* ne, int32_t* nc, int32_t* nf) {
    if (!s) return OCT_EINVAL;
    if (nn) *nn = s->n_nodes;
    if (ne) *ne = s->n_elements;
    if (nc) *nc = s->n_colors;
    if (nf) *nf = s->n_fixed;
    return OCT_OK;
}

oct_status oct_scene_get_coloring(oct_scene* s, int32_t* colors, int32_t* order) {
    if (!s) return OCT_EINVAL;
    if (colors) std::copy(s->colors.begin(), s->colors.end(), colors);
    if (order) std::copy(s->vids.begin(), s->vids.end(), order);
    return OCT_OK;
}

oct_status oct_scene_element_type(oct_scene* s, int32_t* element) {
    if (!s || !element) return OCT_EINVAL;
    *element = s->element;
    return OCT_OK;
}

oct_status oct_scene_get_rest_positions(oct_scene* s, float* out) {
    if (!s || !out) return OCT_EINVAL;
    std::copy(s->X.begin(), s->X.end(), out);
    return OCT_OK;
}

oct_status oct_scene_get_topology(oct_scene* s, int32_t* out) {
    if (!s || !out) return OCT_EINVAL;
    OCT_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    OCT_CUDA(s->ctx, cudaMemcpy(out, s->h.topo, sizeof(int32_t) * (size_t)s->n_elements * s->ne, cudaMemcpyDeviceToHost));
    return OCT_OK;
}

// Run metadata as the reference's recorders write it into their JSON (MeshRecorder and
// FEM_Dynamic_Recorder::add_data_json, octopus/src/Script/Record/Recorder.cpp:12-36), the two
// objects under "mesh" and "fem"; numbers in the same default stream formatting.
oct_status oct_scene_metadata_json(oct_scene* s, char* out, size_t capacity, size_t* length) {
    if (!s) return OCT_EINVAL;
    static const char* elem_names[10] = {"Line", "Triangle", "Quad", "Tetra", "Pyramid", "Prism", "Hexa", "Tetra10",
                                         "Tetra20", "Hexa27"};
    static const char* mat_names[6] = {"Hooke", "SaintVenant", "Neo-Hooke", "Stable Neo-Hooke", "", ""};
    std::ostringstream j;
    j << "{\"mesh\" : {\"" << elem_names[s->element] << "\" : " << s->n_elements << ",\"vertices\" : " << s->n_nodes << "},"
      << "\"fem\" : {\"material\" : \"" << mat_names[s->material] << "\",\"poisson\" : " << s->poisson
      << ",\"young\" : " << s->young << ",\"sub_step\" : " << s->last_substeps << ",\"density\" : " << s->density << "}}";
    const std::string str = j.str();
    if (length) *length = str.size();
    if (!out) return OCT_OK;
    if (capacity < str.size() + 1) return fail(s->ctx, OCT_EINVAL, "metadata buffer too small");
    std::memcpy(out, str.c_str(), str.size() + 1);
    return OCT_OK;
}

oct_status oct_scene_get_masses(oct_scene* s, float* out) {
    if (!s || !out) return OCT_EINVAL;
    std::copy(s->masses.begin(), s->masses.end(), out);
    return OCT_OK;
}

oct_status oct_scene_set_fixation_group(oct_scene* s, int group, const float offset[3], const float rotation[9]) {
    if (!s || group < 0 || group >= kFixGroups) return OCT_EINVAL;
    float* G = s->fix_host + 16 * group;
    if (offset) { G[3] = offset[0]; G[4] = offset[1]; G[5] = offset[2]; }
    if (rotation) std::copy(rotation, rotation + 9, G + 6);
    OCT_CUDA(s->ctx, cudaMemcpyAsync(s->d_fix + 16 * group, G, 16 * sizeof(float), cudaMemcpyHostToDevice, s->ctx->stream));
    OCT_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    return OCT_OK;
}

oct_status oct_scene_set_fixation(oct_scene* s, const float offset[3], const float rotation[9]) {
    return oct_scene_set_fixation_group(s, 0, offset, rotation);
}

oct_status oct_scene_add_effect(oct_scene* s, int kind, const float* params, int32_t* index) {
    if (!s || kind < OCT_EFFECT_CRUSH || kind > OCT_EFFECT_HIGH_STRETCH) return OCT_EINVAL;
    if (s->n_effects >= kMaxEffects) return fail(s->ctx, OCT_ENOTSUP, "at most 4 effects per scene");
    oct_ctx* c = s->ctx;
    EffectDev e{};
    e.kind = kind;
    e.active = 0;   // created inactive, as the reference controller creates them
    // centre: sum of the rest positions after the first, divided by their count (the
    // GPU_RandomSphere / GPU_HighStretch constructors, GPU_Constraint.h:29-31,44-45)
    float cx = 0.f, cy = 0.f, cz = 0.f;
    for (int i = 1; i < s->n_nodes; ++i) { cx += s->X[3 * i]; cy += s->X[3 * i + 1]; cz += s->X[3 * i + 2]; }
    const float inv = 1.f / (float)s->n_nodes;
    e.cx = cx * inv; e.cy = cy * inv; e.cz = cz * inv;
    if (kind == OCT_EFFECT_RANDOM_SPHERE) {
        if (!params || !(params[0] > 0.f)) return OCT_EINVAL;
        e.radius = params[0];
    } else if (kind == OCT_EFFECT_HIGH_STRETCH) {
        if (!params || params[0] < 1.f || params[0] > 1024.f || !(params[1] >= 0.f)) return OCT_EINVAL;
        const int nb = (int)params[0];
        e.max_dist = params[1];
        // farthest-point choice among the boundary nodes (GPU_HighStretch ctor, :41-66): start
        // at the lowest surface id, then repeatedly the node farthest from the chosen ones
        const std::vector<int32_t> ids = surface_nodes(s->element, s->topo_host.data(), s->n_elements);
        std::vector<int32_t> chosen;
        std::vector<char> taken(s->n_nodes, 0);
        for (int i = 0; i < nb && !ids.empty(); ++i) {
            float best = 0.f;
            int cur = ids[0];
            for (int32_t a : ids) {
                if (taken[a]) continue;
                float d = 3.402823466e38f;
                for (int32_t b : chosen) {
                    const float dx = s->X[3 * a] - s->X[3 * b], dy = s->X[3 * a + 1] - s->X[3 * b + 1],
                                dz = s->X[3 * a + 2] - s->X[3 * b + 2];
                    d = std::min(d, dx * dx + dy * dy + dz * dz);
                }
                if (d > best) { cur = a; best = d; }
            }
            chosen.push_back(cur);
            taken[cur] = 1;
        }
        oct_status st;
        int32_t* d_ids = nullptr;
        float* d_t = nullptr;
        if ((st = upload(c, s->mem, d_ids, chosen)) || (st = upload(c, s->mem, d_t, std::vector<float>{0.f}))) return st;
        e.ids = d_ids;
        e.n = (int)chosen.size();
        e.t = d_t;
    }
    const int k = s->n_effects;
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    OCT_CUDA(c, cudaMemcpy(s->d_effects + k, &e, sizeof(EffectDev), cudaMemcpyHostToDevice));
    s->effects[k] = e;
    s->n_effects++;
    drop_frame_graph(s);
    if (index) *index = k;
    return OCT_OK;
}

oct_status oct_scene_set_effect_active(oct_scene* s, int32_t index, int active) {
    if (!s || index < 0 || index >= s->n_effects) return OCT_EINVAL;
    s->effects[index].active = active ? 1 : 0;
    OCT_CUDA(s->ctx, cudaMemcpyAsync(&s->d_effects[index].active, &s->effects[index].active, sizeof(int),
                                     cudaMemcpyHostToDevice, s->ctx->stream));
    if (!active && s->effects[index].kind == OCT_EFFECT_HIGH_STRETCH)   // the controller restarts the stretch
        OCT_CUDA(s->ctx, cudaMemsetAsync(s->effects[index].t, 0, sizeof(float), s->ctx->stream));
    OCT_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    return OCT_OK;
}

oct_status oct_scene_effect_ids(oct_scene* s, int32_t index, int32_t* ids, int32_t* n) {
    if (!s || !n || index < 0 || index >= s->n_effects) return OCT_EINVAL;
    const EffectDev& e = s->effects[index];
    *n = e.kind == OCT_EFFECT_HIGH_STRETCH ? e.n : 0;
    if (ids && *n) OCT_CUDA(s->ctx, cudaMemcpy(ids, e.ids, sizeof(int32_t) * e.n, cudaMemcpyDeviceToHost));
    return OCT_OK;
}

oct_status oct_surface_nodes(int32_t element, const int32_t* topology, int32_t n_elements, int32_t* ids, int32_t* n) {
    if (!topology || n_elements <= 0 || !n || element_nodes(element) < 0) return OCT_EINVAL;
    const std::vector<int32_t> v = surface_nodes(element, topology, n_elements);
    *n = (int32_t)v.size();
    if (ids) std::copy(v.begin(), v.end(), ids);
    return OCT_OK;
}

oct_status oct_ctx_wait_probe(oct_ctx* c, int32_t limit) {
    if (!c || limit <= 0 || limit > 1000000) return OCT_EINVAL;
    launch_wait_probe(c->d_error, limit, c->stream);
    OCT_CUDA(c, cudaGetLastError());
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_error_word(c);
}

// Checkpoint: per node u, u_last, v (9 floats) and the mask, then the fixation table
// (kFixGroups x 16), the effects' stretch distances (kMaxEffects), the multigrid schedule (3)
// and the pending initial-velocity flag.
// Checkpoint header: a format tag and the scene's shape, checked by restore before it reads
// anything else, so a checkpoint of another scene is refused instead of read past its end.
constexpr int32_t kCheckpointTag = 0x3154434F;   // "OCT1", stored as the bits of a float
constexpr int kCheckpointHeader = 4;              // tag, n_nodes, n_elements, element

oct_status oct_scene_state_size(oct_scene* s, size_t* n_floats) {
    if (!s || !n_floats) return OCT_EINVAL;
    *n_floats = kCheckpointHeader + (size_t)s->n_nodes * 10 + kFixGroups * 16 + kMaxEffects + 4;
    return OCT_OK;
}

oct_status oct_scene_save(oct_scene* s, float* out) {
    if (!s || !out) return OCT_EINVAL;
    oct_ctx* c = s->ctx;
    const int N = s->n_nodes;
    std::vector<float4> u(N), ul(N), v(N);
    std::vector<int> mask(N);
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    OCT_CUDA(c, cudaMemcpy(u.data(), s->h.u, sizeof(float4) * N, cudaMemcpyDeviceToHost));
    OCT_CUDA(c, cudaMemcpy(ul.data(), s->h.u_last, sizeof(float4) * N, cudaMemcpyDeviceToHost));
    OCT_CUDA(c, cudaMemcpy(v.data(), s->h.v, sizeof(float4) * N, cudaMemcpyDeviceToHost));
    OCT_CUDA(c, cudaMemcpy(mask.data(), s->h.mask, sizeof(int) * N, cudaMemcpyDeviceToHost));
    float* o = out;
    std::memcpy(o++, &kCheckpointTag, sizeof(float));
    *o++ = (float)N; *o++ = (float)s->n_elements; *o++ = (float)s->element;
    for (int i = 0; i < N; ++i) {
        *o++ = u[i].x; *o++ = u[i].y; *o++ = u[i].z;
        *o++ = ul[i].x; *o++ = ul[i].y; *o++ = ul[i].z;
        *o++ = v[i].x; *o++ = v[i].y; *o++ = v[i].z;
        *o++ = (float)mask[i];
    }
    std::copy(s->fix_host, s->fix_host + kFixGroups * 16, o);
    o += kFixGroups * 16;
    for (int k = 0; k < kMaxEffects; ++k) {
        float t = 0.f;
        if (k < s->n_effects && s->effects[k].kind == OCT_EFFECT_HIGH_STRETCH)
            OCT_CUDA(c, cudaMemcpy(&t, s->effects[k].t, sizeof(float), cudaMemcpyDeviceToHost));
        *o++ = t;
    }
    *o++ = (float)s->mg_count; *o++ = (float)s->mg_current; *o++ = (float)s->pending_host; *o++ = 0.f;
    return OCT_OK;
}

oct_status oct_scene_restore(oct_scene* s, const float* in) {
    if (!s || !in) return OCT_EINVAL;
    oct_ctx* c = s->ctx;
    const int N = s->n_nodes;
    int32_t tag = 0;
    std::memcpy(&tag, in, sizeof(float));
    if (tag != kCheckpointTag || in[1] != (float)N || in[2] != (float)s->n_elements || in[3] != (float)s->element)
        return fail(c, OCT_EINVAL, "checkpoint of another scene (or not a checkpoint)");
    std::vector<float4> u(N), ul(N), v(N);
    std::vector<int> mask(N);
    const float* p = in + kCheckpointHeader;
    for (int i = 0; i < N; ++i, p += 10) {
        u[i] = make_float4(p[0], p[1], p[2], 0.f);
        ul[i] = make_float4(p[3], p[4], p[5], 0.f);
        v[i] = make_float4(p[6], p[7], p[8], 0.f);
        mask[i] = p[9] != 0.f ? 1 : 0;
    }
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    OCT_CUDA(c, cudaMemcpy(s->h.u, u.data(), sizeof(float4) * N, cudaMemcpyHostToDevice));
    OCT_CUDA(c, cudaMemcpy(s->h.u_last, ul.data(), sizeof(float4) * N, cudaMemcpyHostToDevice));
    OCT_CUDA(c, cudaMemcpy(s->h.v, v.data(), sizeof(float4) * N, cudaMemcpyHostToDevice));
    OCT_CUDA(c, cudaMemcpy(s->h.mask, mask.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    std::copy(p, p + kFixGroups * 16, s->fix_host);
    OCT_CUDA(c, cudaMemcpy(s->d_fix, s->fix_host, sizeof(float) * kFixGroups * 16, cudaMemcpyHostToDevice));
    p += kFixGroups * 16;
    for (int k = 0; k < kMaxEffects; ++k, ++p)
        if (k < s->n_effects && s->effects[k].kind == OCT_EFFECT_HIGH_STRETCH)
            OCT_CUDA(c, cudaMemcpy(s->effects[k].t, p, sizeof(float), cudaMemcpyHostToDevice));
    s->mg_count = (int)p[0];
    s->mg_current = (int)p[1];
    s->pending_host = (int)p[2];
    OCT_CUDA(c, cudaMemcpy(s->d_pending, &s->pending_host, sizeof(int), cudaMemcpyHostToDevice));
    return OCT_OK;
}

oct_status oct_scene_set_precision(oct_scene* s, int precision) {
    if (!s || precision < 0 || precision > 1) return OCT_EINVAL;
    s->precision = precision;
    s->h.precision = precision;
    OCT_CUDA(s->ctx, cudaMemcpyAsync(s->d_scene, &s->h, sizeof(SceneDev), cudaMemcpyHostToDevice, s->ctx->stream));
    OCT_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    return OCT_OK;
}

oct_status oct_scene_energy(oct_scene* s, double out[4]) {
    if (!s || !out) return OCT_EINVAL;
    if (s->material > OCT_STABLE_NEOHOOKE) return fail(s->ctx, OCT_ENOTSUP, "no energy density for this material");
    oct_ctx* c = s->ctx;
    OCT_CUDA(c, cudaMemsetAsync(s->d_red, 0, 4 * sizeof(double), c->stream));
    launch_energy(s->element, s->material, s->d_scene, 0, s->n_nodes, s->n_elements, s->d_red, c->d_error, c->stream);
    OCT_CUDA(c, cudaMemcpyAsync(out, s->d_red, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    out[3] = out[0] + out[1] + out[2];
    return check_error_word(c);
}

oct_status oct_scene_element_data(oct_scene* s, int kind, float* out) {
    if (!s || !out || kind < OCT_DIAG_STRESS || kind > OCT_DIAG_VOLUME_DIFF_ACCUMULATED) return OCT_EINVAL;
    oct_ctx* c = s->ctx;
    oct_status st;
    if (!s->d_diag && (st = s->mem.alloc(s->d_diag, (size_t)s->n_elements))) return st;
    launch_element_diag(s->element, s->material, s->d_scene, 0, s->n_elements, kind, s->d_diag, c->stream);
    OCT_CUDA(c, cudaGetLastError());
    OCT_CUDA(c, cudaMemcpyAsync(out, s->d_diag, sizeof(float) * s->n_elements, cudaMemcpyDeviceToHost, c->stream));
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    return OCT_OK;
}

oct_status oct_scene_vertex_residuals(oct_scene* s, float dt, float* out) {
    if (!s || !out || !(dt > 0.f)) return OCT_EINVAL;
    if (s->solver != OCT_SOLVER_VBD) {   // GPU_FEM::get_forces: zeros for the other solvers
        std::fill(out, out + 3 * (size_t)s->n_nodes, 0.f);
        return OCT_OK;
    }
    oct_ctx* c = s->ctx;
    StepParams P = base_params(c, dt);
    OCT_CUDA(c, cudaMemsetAsync(s->d_red, 0, 4 * sizeof(double), c->stream));
    OCT_CUDA(c, cudaMemsetAsync(s->h.u_new, 0, sizeof(float4) * s->n_nodes, c->stream));
    for (int k = 0; k < s->n_colors; ++k) {
        const int b = s->vwork_off[k], n = s->vwork_off[k + 1] - b;
        launch_vertex(s->element, s->material, s->d_scene, s->d_vwork + b, n, s->tpv, 1, P, s->d_red, c->stream);
    }
    OCT_CUDA(c, cudaGetLastError());
    oct_status st = read_nodes(s, s->h.u_new, out, false);
    if (st) return st;
    return check_error_word(c);
}

oct_status oct_scene_residual(oct_scene* s, float dt, double out[2]) {
    if (!s || !out || !(dt > 0.f)) return OCT_EINVAL;
    if (s->solver != OCT_SOLVER_VBD) return OCT_ENOTSUP;
    oct_ctx* c = s->ctx;
    StepParams P = base_params(c, dt);
    OCT_CUDA(c, cudaMemsetAsync(s->d_red, 0, 4 * sizeof(double), c->stream));
    for (int k = 0; k < s->n_colors; ++k) {
        const int b = s->vwork_off[k], n = s->vwork_off[k + 1] - b;
        launch_vertex(s->element, s->material, s->d_scene, s->d_vwork + b, n, s->tpv, 1, P, s->d_red, c->stream);
    }
    OCT_CUDA(c, cudaMemcpyAsync(out, s->d_red, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_error_word(c);
}

oct_status oct_scene_status(oct_scene* s) {
    if (!s) return OCT_EINVAL;
    oct_ctx* c = s->ctx;
    int f = 0;
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    OCT_CUDA(c, cudaMemcpy(&f, s->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (f) OCT_CUDA(c, cudaMemset(s->d_status, 0, sizeof(int)));
    if (f & kStatusNonFinite) return fail(c, OCT_ENUMERIC, "non-finite position or velocity in the scene");
    if (f & kStatusTimeout) return fail(c, OCT_ETIMEDOUT, "a bounded device wait gave up on the scene's work");
    return check_error_word(c);
}

oct_status oct_batch_status(oct_batch* b, int32_t* out) {
    if (!b || !out) return OCT_EINVAL;
    oct_ctx* c = b->ctx;
    const size_t n = b->scenes.size();
    std::vector<int> f(n, 0);
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    OCT_CUDA(c, cudaMemcpy(f.data(), b->d_status, sizeof(int) * n, cudaMemcpyDeviceToHost));
    OCT_CUDA(c, cudaMemset(b->d_status, 0, sizeof(int) * n));
    int e = 0;   // context word: a time-out outside any one scene's work (constant-table staging)
    OCT_CUDA(c, cudaMemcpy(&e, c->d_error, sizeof(int), cudaMemcpyDeviceToHost));
    if (e & 1) {   // taken over by the per-scene statuses; the other bits stay for their own checks
        const int rest = e & ~1;
        OCT_CUDA(c, cudaMemcpy(c->d_error, &rest, sizeof(int), cudaMemcpyHostToDevice));
    }
    for (size_t i = 0; i < n; ++i)
        out[i] = (f[i] & kStatusNonFinite) ? OCT_ENUMERIC : ((f[i] & kStatusTimeout) || (e & 1)) ? OCT_ETIMEDOUT : OCT_OK;
    return OCT_OK;
}

oct_status oct_ctx_stream(oct_ctx* c, void** stream) {
    if (!c || !stream) return OCT_EINVAL;
    *stream = (void*)c->stream;
    return OCT_OK;
}

oct_status oct_fp32_peak(oct_ctx* c, double* tflops) {
    if (!c || !tflops) return OCT_EINVAL;
    launch_fma_peak(c->stream);   // warm-up
    OCT_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    double fmas = 0;
    for (int k = 0; k < 5; ++k) fmas += launch_fma_peak(c->stream);
    OCT_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    OCT_CUDA(c, cudaEventSynchronize(c->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    *tflops = 2.0 * fmas / (ms * 1e-3) / 1e12;
    return OCT_OK;
}

oct_status oct_last_step_ms(oct_ctx* c, float* ms) {
    if (!c || !ms) return OCT_EINVAL;
    *ms = c->last_ms;
    return OCT_OK;
}

oct_status oct_launch_count(oct_ctx* c, uint64_t* n) {
    if (!c || !n) return OCT_EINVAL;
    *n = c->launches;
    return OCT_OK;
}

// ---------------------------------------------------------------------------- batches
oct_status oct_batch_create(oct_ctx* c, oct_scene* const* scenes, int n, oct_batch** out) {
    if (!c || !scenes || n <= 0 || !out) return OCT_EINVAL;
    *out = nullptr;
    auto b = std::make_unique<oct_batch>();
    b->ctx = c;
    b->mem.ctx = c;
    if (!scenes[0]) return OCT_EINVAL;
    b->solver = scenes[0]->solver;
    if (b->solver == OCT_SOLVER_EXPLICIT) return fail(c, OCT_ENOTSUP, "batches hold VBD or XPBD scenes");
    const bool xpbd = b->solver == OCT_SOLVER_XPBD;
    b->iterations = scenes[0]->iterations;
    b->rho = scenes[0]->rho;
    std::vector<SceneDev> hs;
    std::vector<NWork> nw, fw, bw;
    std::map<std::pair<std::pair<int, int>, std::pair<int, int>>, int> gid;
    std::vector<std::vector<std::vector<VWork>>> gwork;   // group -> colour -> items
    std::vector<std::vector<std::vector<XWork>>> gxwork;  // XPBD: group -> colour -> items
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        oct_scene* s = scenes[i];
        if (!s || s->ctx != c) return fail(c, OCT_EINVAL, "scene from another context");
        if (s->solver != b->solver) return fail(c, OCT_ENOTSUP, "a batch holds scenes of one solver");
        if (!xpbd && (s->iterations != b->iterations || s->rho != b->rho))
            return fail(c, OCT_ENOTSUP, "batch scenes need equal iterations and rho");
        if (!xpbd && s->order_mode != OCT_ORDER_ASCENDING) return fail(c, OCT_ENOTSUP, "batches use the ascending colour order");
        if (s->mg_sub) return fail(c, OCT_ENOTSUP, "multigrid scenes are stepped alone");
        b->scenes.push_back(s);
        hs.push_back(s->h);
        b->pending_host.push_back(s->pending_host);
        b->state_off.push_back(off);
        off += (size_t)s->n_nodes * 6;
        append_nwork(nw, i, s->n_nodes);
        std::vector<NWork> f1;
        append_nwork(f1, i, s->n_fixed);
        fw.insert(fw.end(), f1.begin(), f1.end());
        if (s->box) append_nwork(bw, i, s->n_nodes);
        if (xpbd) {   // groups by (element, material, update form); scenes that project nothing add no work
            if (!s->xpbd_project) continue;
            auto key = std::make_pair(std::make_pair(s->element, s->material), std::make_pair(s->xpbd_raw ? 1 : 0, 0));
            auto it = gid.find(key);
            if (it == gid.end()) {
                it = gid.emplace(key, (int)b->groups.size()).first;
                oct_batch::Group g;
                g.element = s->element; g.material = s->material; g.tpv = s->xpbd_raw ? 1 : 0; g.in_place = true;
                b->groups.push_back(g);
                gxwork.emplace_back();
            }
            auto& cw = gxwork[it->second];
            const int nc = (int)s->elem_off.size() - 1;
            if ((int)cw.size() < nc) cw.resize(nc);
            for (int k = 0; k < nc; ++k)
                append_xwork(cw[k], i, s->elem_off[k], s->elem_off[k + 1], xpbd_elements_per_block(s->element));
            continue;
        }
        auto key = std::make_pair(std::make_pair(s->element, s->material), std::make_pair(s->tpv, s->in_place ? 1 : 0));
        auto it = gid.find(key);
        if (it == gid.end()) {
            it = gid.emplace(key, (int)b->groups.size()).first;
            oct_batch::Group g;
            g.element = s->element; g.material = s->material; g.tpv = s->tpv; g.in_place = s->in_place;
            b->groups.push_back(g);
            gwork.emplace_back();
        }
        auto& cw = gwork[it->second];
        if ((int)cw.size() < s->n_colors) cw.resize(s->n_colors);
        for (int k = 0; k < s->n_colors; ++k) append_vwork(cw[k], i, s->color_off[k], s->color_off[k + 1], s->tpv, s->own_off);
    }
    b->state_off.push_back(off);
    std::vector<VWork> all;
    std::vector<XWork> xall;
    for (size_t g = 0; g < b->groups.size(); ++g) {
        b->groups[g].off.assign(1, 0);
        if (xpbd) {
            b->groups[g].base = (int)xall.size();
            for (auto& items : gxwork[g]) {
                xall.insert(xall.end(), items.begin(), items.end());
                b->groups[g].off.push_back((int)(xall.size() - b->groups[g].base));
            }
        } else {
            b->groups[g].base = (int)all.size();
            for (auto& items : gwork[g]) {
                all.insert(all.end(), items.begin(), items.end());
                b->groups[g].off.push_back((int)(all.size() - b->groups[g].base));
            }
        }
        OCT_CUDA(c, cudaStreamCreateWithFlags(&b->groups[g].stream, cudaStreamNonBlocking));
        OCT_CUDA(c, cudaEventCreateWithFlags(&b->groups[g].done, cudaEventDisableTiming));
    }
    OCT_CUDA(c, cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    oct_status st;
    // the batch's scene copies report failures into the batch's own status array
    if ((st = upload(c, b->mem, b->d_status, std::vector<int>(b->scenes.size(), 0)))) { b->mem.release(); return st; }
    for (size_t i = 0; i < hs.size(); ++i) hs[i].status = b->d_status + i;
    if ((st = upload(c, b->mem, b->d_scenes, hs)) || (st = upload(c, b->mem, b->d_vwork, all)) ||
        (st = upload(c, b->mem, b->d_xwork, xall)) ||
        (st = upload(c, b->mem, b->d_nwork, nw)) || (st = upload(c, b->mem, b->d_fwork, fw)) ||
        (st = upload(c, b->mem, b->d_bwork, bw)) || (st = upload(c, b->mem, b->d_pending, b->pending_host))) {
        b->mem.release();
        return st;
    }
    std::vector<long long> soff(b->state_off.begin(), b->state_off.end());
    if ((st = upload(c, b->mem, b->d_soff, soff))) { b->mem.release(); return st; }
    b->n_nwork = (int)nw.size();
    b->n_fwork = (int)fw.size();
    b->n_bwork = (int)bw.size();
    *out = b.release();
    return OCT_OK;
}

namespace {
// Enqueue one sub-step of the whole batch on the context stream (captured into a graph).
// One GPU_PBD::step (octopus/src/GPU/PBD/GPU_PBD.cu:20-26) over all scenes of an XPBD batch:
// predictor, per colour one launch per (element type, material, update form) group with the
// groups on parallel branches, constraints, velocity update with each scene's damping.
void batch_substep_xpbd(oct_batch* b, float dt) {
    oct_ctx* c = b->ctx;
    cudaStream_t st = c->stream;
    StepParams P = base_params(c, dt);
    launch_predict(b->d_scenes, b->d_nwork, b->n_nwork, 1, 0, 0, P, st);
    cudaEventRecord(b->fork, st);
    for (auto& g : b->groups) {
        cudaStreamWaitEvent(g.stream, b->fork, 0);
        for (size_t k = 0; k + 1 < g.off.size(); ++k)
            launch_xpbd(g.element, g.material, g.tpv != 0, b->d_scenes, b->d_xwork + g.base + g.off[k],
                        g.off[k + 1] - g.off[k], P, g.stream);
        cudaEventRecord(g.done, g.stream);
        cudaStreamWaitEvent(st, g.done, 0);
    }
    if (b->n_fwork) launch_constraints(b->d_scenes, b->d_fwork, b->n_fwork, 0, st);
    for (auto* s : b->scenes)
        for (int k = 0; k < s->n_effects; ++k) launch_effect(s->d_scene, s->d_nwork, s->n_nwork, k, s->effects[k].kind, dt, st);
    if (b->n_bwork) launch_constraints(b->d_scenes, b->d_bwork, b->n_bwork, 1, st);
    launch_velocity(b->d_scenes, b->d_nwork, b->n_nwork, 1, P, st);
}

void batch_substep(oct_batch* b, float dt) {
    if (b->solver == OCT_SOLVER_XPBD) { batch_substep_xpbd(b, dt); return; }
    oct_ctx* c = b->ctx;
    cudaStream_t st = c->stream;
    StepParams P = base_params(c, dt);
    P.pending_v0 = b->d_pending;
    const bool cheb = b->rho > 0.f && b->rho > 1.17549435e-38f * 1e6f;
    launch_predict(b->d_scenes, b->d_nwork, b->n_nwork, 0, 0, cheb ? 1 : 0, P, st);
    cudaMemsetAsync(b->d_pending, 0, sizeof(int) * b->scenes.size(), st);
    float omega = 1.f;
    for (int j = 0; j < b->iterations; ++j) {
        cudaEventRecord(b->fork, st);
        for (auto& g : b->groups) {
            cudaStreamWaitEvent(g.stream, b->fork, 0);
            StepParams Pg = P;
            Pg.in_place = g.in_place ? 1 : 0;
            for (size_t k = 0; k + 1 < g.off.size(); ++k) {
                const VWork* w = b->d_vwork + g.base + g.off[k];
                const int n = g.off[k + 1] - g.off[k];
                launch_vertex(g.element, g.material, b->d_scenes, w, n, g.tpv, 0, Pg, nullptr, g.stream);
                if (!g.in_place) launch_commit(b->d_scenes, w, n, g.stream);
            }
            cudaEventRecord(g.done, g.stream);
            cudaStreamWaitEvent(st, g.done, 0);
        }
        if (b->n_fwork) launch_constraints(b->d_scenes, b->d_fwork, b->n_fwork, 0, st);
        for (auto* s : b->scenes)
            for (int k = 0; k < s->n_effects; ++k) launch_effect(s->d_scene, s->d_nwork, s->n_nwork, k, s->effects[k].kind, dt, st);
        if (b->n_bwork) launch_constraints(b->d_scenes, b->d_bwork, b->n_bwork, 1, st);
        if (cheb) {
            if (j == 1) omega = 2.f / (2.f - b->rho * b->rho);
            else if (j > 1) omega = 4.f / (4.f - b->rho * b->rho * omega);
            P.omega = omega;
            P.iteration = j;
            launch_chebyshev(b->d_scenes, b->d_nwork, b->n_nwork, P, st);
        }
    }
    launch_velocity(b->d_scenes, b->d_nwork, b->n_nwork, 0, P, st);
}

uint64_t batch_launches_per_substep(const oct_batch* b) {
    uint64_t n = 2;
    if (b->solver == OCT_SOLVER_XPBD) {
        for (auto& g : b->groups)
            for (size_t k = 0; k + 1 < g.off.size(); ++k) n += g.off[k + 1] > g.off[k] ? 1 : 0;
        if (b->n_fwork) ++n;
        if (b->n_bwork) ++n;
        for (auto* s : b->scenes) n += (uint64_t)s->n_effects;
        return n;
    }
    for (auto& g : b->groups) n += (uint64_t)(g.off.size() - 1) * (g.in_place ? 1 : 2) * b->iterations;
    if (b->n_fwork) n += b->iterations;
    if (b->n_bwork) n += b->iterations;
    if (b->rho > 0.f) n += b->iterations;
    return n;
}
}  // namespace

oct_status oct_batch_prepare(oct_batch* b, float frame_dt, int substeps) {
    if (!b || substeps <= 0 || !(frame_dt > 0.f)) return OCT_EINVAL;
    oct_ctx* c = b->ctx;
    const float sub = frame_dt / (float)substeps;
    if (b->exec && b->graph_dt == sub) return OCT_OK;
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    OCT_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    batch_substep(b, sub);
    OCT_CUDA(c, cudaStreamEndCapture(c->stream, &b->graph));
    OCT_CUDA(c, cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->graph_dt = sub;
    return OCT_OK;
}

oct_status oct_batch_step(oct_batch* b, float frame_dt, int substeps) {
    if (!b || substeps <= 0 || !(frame_dt > 0.f)) return OCT_EINVAL;
    Range range("oct_batch_step");
    oct_ctx* c = b->ctx;
    oct_status st = oct_batch_prepare(b, frame_dt, substeps);
    if (st) return st;
    cudaEventRecord(c->ev0, c->stream);
    for (int k = 0; k < substeps; ++k) {
        OCT_CUDA(c, cudaGraphLaunch(b->exec, c->stream));
        c->launches += batch_launches_per_substep(b);
    }
    cudaEventRecord(c->ev1, c->stream);
    for (size_t i = 0; i < b->scenes.size(); ++i) {
        // the batch applied the flags it took at creation; those scenes' own flags go too (a
        // flag set on a scene after the batch was created stays for the scene's own next step)
        if (!b->pending_host[i]) continue;
        oct_scene* s = b->scenes[i];
        cudaMemsetAsync(s->d_pending, 0, sizeof(int), c->stream);
        s->pending_host = 0;
        b->pending_host[i] = 0;
    }
    return OCT_OK;
}

oct_status oct_batch_destroy(oct_batch* b) {
    if (!b) return OCT_EINVAL;
    cudaStreamSynchronize(b->ctx->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto& g : b->groups) { cudaStreamDestroy(g.stream); cudaEventDestroy(g.done); }
    if (b->fork) cudaEventDestroy(b->fork);
    b->mem.release();
    delete b;
    return OCT_OK;
}

oct_status oct_batch_group_info(oct_batch* b, int g, int32_t* element, int32_t* material, double* flops, double* bytes,
                                int32_t* launches, int64_t* vertices) {
    if (!b || g < 0 || g >= (int)b->groups.size()) return OCT_EINVAL;
    if (b->solver != OCT_SOLVER_VBD) return OCT_ENOTSUP;
    const auto& G = b->groups[g];
    // Algorithmic work of one sweep: every free vertex of every scene of the group once.
    // flops: per (owner, quadrature point) term vbd_term_flops; bytes: per vertex u, u_last,
    // y read + u written (16 B each) + mask/slot/owner-offset ints, per owner entry 4 B,
    // per element its topology (4 NE) and quadrature records (48 NQ) once.
    double fl = 0, by = 0;
    int64_t nv = 0;
    const double tf = vbd_term_flops(G.element, G.material);
    for (auto* s : b->scenes) {
        if (s->element != G.element || s->material != G.material || s->tpv != G.tpv || s->in_place != G.in_place) continue;
        const int64_t free_nodes = s->n_nodes - s->n_fixed;
        const int64_t terms = (int64_t)s->n_elements * s->ne * s->nq;   // sum over vertices of owners x Q
        fl += tf * (double)terms * (double)free_nodes / (double)s->n_nodes;
        by += (double)s->n_nodes * (4 * 16 + 12) + (double)s->n_elements * s->ne * 4.0 +
              (double)s->n_elements * (4.0 * s->ne + 48.0 * s->nq);
        nv += free_nodes;
    }
    if (element) *element = G.element;
    if (material) *material = G.material;
    if (flops) *flops = fl;
    if (bytes) *bytes = by;
    if (launches) *launches = (int32_t)(G.off.size() - 1) * (G.in_place ? 1 : 2);
    if (vertices) *vertices = nv;
    return OCT_OK;
}

oct_status oct_batch_time_group(oct_batch* b, int g, int sweeps, float dt, float* ms) {
    if (!b || g < 0 || g >= (int)b->groups.size() || sweeps <= 0 || !ms || !(dt > 0.f)) return OCT_EINVAL;
    if (b->solver != OCT_SOLVER_VBD) return OCT_ENOTSUP;
    oct_ctx* c = b->ctx;
    const auto& G = b->groups[g];
    StepParams P = base_params(c, dt);
    P.in_place = G.in_place ? 1 : 0;
    OCT_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    for (int r = 0; r < sweeps; ++r)
        for (size_t k = 0; k + 1 < G.off.size(); ++k) {
            const VWork* w = b->d_vwork + G.base + G.off[k];
            const int n = G.off[k + 1] - G.off[k];
            launch_vertex(G.element, G.material, b->d_scenes, w, n, G.tpv, 0, P, nullptr, c->stream);
            if (!G.in_place) launch_commit(b->d_scenes, w, n, c->stream);
            c->launches += G.in_place ? 1 : 2;
        }
    OCT_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    OCT_CUDA(c, cudaEventSynchronize(c->ev1));
    OCT_CUDA(c, cudaGetLastError());
    cudaEventElapsedTime(ms, c->ev0, c->ev1);
    return OCT_OK;
}

oct_status oct_scene_set_mapping(oct_scene* s, int tpv) {
    if (!s) return OCT_EINVAL;
    if (s->solver == OCT_SOLVER_XPBD) return OCT_OK;   // element-centric: no vertex mapping
    int t = tpv < 0 ? 0 : (tpv == 0 ? measured_tpv(s->element) : tpv);
    if (tpv < -1 || (t != 0 && t != 1 && t != 2 && t != 4 && t != 8 && t != 16 && t != 32))
        return fail(s->ctx, OCT_EINVAL, "threads_per_vertex must be -1 (packed), 0 (default) or a power of two <= 32");
    if (t == 0 && s->max_valence > 32) {
        if (tpv < 0) return fail(s->ctx, OCT_ENOTSUP, "packed mapping needs at most 32 owners per vertex");
        t = s->max_valence > 64 ? 32 : default_tpv(s->element);
    }
    if (t == 0 && !s->h.ent) {
        if (tpv < 0) return fail(s->ctx, OCT_ENOTSUP, "packed mapping needs owner entries (scene past their index range)");
        t = default_tpv(s->element);
    }
    OCT_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    s->tpv = t;
    drop_frame_graph(s);
    return build_vertex_work(s);
}

oct_status oct_scene_get_mapping(oct_scene* s, int32_t* threads_per_vertex) {
    if (!s || !threads_per_vertex) return OCT_EINVAL;
    *threads_per_vertex = s->solver == OCT_SOLVER_XPBD ? 0 : (s->tpv == 0 ? -1 : s->tpv);
    return OCT_OK;
}

// Times one colour sweep of every group of a batch with the solve results written to the
// Jacobi buffer (u_new) and not committed, so the scenes' state is left as it was.
static oct_status time_batch_sweeps(oct_batch* b, int sweeps, float dt, float* ms) {
    oct_ctx* c = b->ctx;
    StepParams P = base_params(c, dt);
    P.in_place = 0;
    OCT_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    for (int r = 0; r < sweeps; ++r)
        for (const auto& G : b->groups)
            for (size_t k = 0; k + 1 < G.off.size(); ++k) {
                const int n = G.off[k + 1] - G.off[k];
                launch_vertex(G.element, G.material, b->d_scenes, b->d_vwork + G.base + G.off[k], n, G.tpv, 0, P, nullptr,
                              c->stream);
            }
    OCT_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    OCT_CUDA(c, cudaEventSynchronize(c->ev1));
    OCT_CUDA(c, cudaGetLastError());
    cudaEventElapsedTime(ms, c->ev0, c->ev1);
    return OCT_OK;
}

oct_status oct_autotune_mapping(oct_ctx* c, oct_scene* const* scenes, int n, float dt, int sweeps, int32_t chosen[10]) {
    if (!c || !scenes || n <= 0 || !(dt > 0.f) || sweeps <= 0) return OCT_EINVAL;
    if (chosen) std::fill(chosen, chosen + 10, 0);
    std::map<int, std::vector<oct_scene*>> by_element;
    for (int i = 0; i < n; ++i) {
        if (!scenes[i] || scenes[i]->ctx != c) return fail(c, OCT_EINVAL, "scene from another context");
        if (scenes[i]->solver == OCT_SOLVER_XPBD) continue;
        by_element[scenes[i]->element].push_back(scenes[i]);
    }
    for (auto& [element, list] : by_element) {
        int max_val = 0;
        bool entries = true;
        for (auto* s : list) { max_val = std::max(max_val, s->max_valence); entries = entries && s->h.ent; }
        std::vector<int> cands = {1, 2, 4, 8, 16, 32};
        if (max_val <= 32 && entries) cands.insert(cands.begin(), -1);
        const std::vector<int> old = [&] { std::vector<int> v; for (auto* s : list) v.push_back(s->tpv); return v; }();
        // the measured default is timed first and kept unless a candidate is clearly faster:
        // candidates that differ little (the per-colour lane rule makes neighbours build
        // nearly the same items) must not switch on timing noise
        int dflt = measured_tpv(element);
        if (dflt == 0) dflt = std::find(cands.begin(), cands.end(), -1) != cands.end() ? -1 : default_tpv(element);
        cands.erase(std::remove(cands.begin(), cands.end(), dflt), cands.end());
        cands.insert(cands.begin(), dflt);
        float best_ms = 1e30f, dflt_ms = 1e30f;
        int best = dflt;
        for (int cand : cands) {
            for (auto* s : list) s->tpv = cand < 0 ? 0 : cand;   // host field only: the batch builds its own tables
            oct_batch* b = nullptr;
            oct_status st = oct_batch_create(c, list.data(), (int)list.size(), &b);
            if (st) {
                for (size_t i = 0; i < list.size(); ++i) list[i]->tpv = old[i];
                return st;
            }
            float ms = 1e30f, t = 0.f;
            st = time_batch_sweeps(b, 1, dt, &t);   // warm-up
            for (int r = 0; r < 3 && !st; ++r) {     // best of three
                st = time_batch_sweeps(b, sweeps, dt, &t);
                ms = std::min(ms, t);
            }
            oct_batch_destroy(b);
            if (st) {
                for (size_t i = 0; i < list.size(); ++i) list[i]->tpv = old[i];
                return st;
            }
            if (cand == dflt) dflt_ms = ms;
            if (ms < best_ms && (cand == dflt || ms < 0.97f * dflt_ms)) { best_ms = ms; best = cand; }
        }
        for (size_t i = 0; i < list.size(); ++i) list[i]->tpv = old[i];
        for (auto* s : list) {
            oct_status st = oct_scene_set_mapping(s, best);
            if (st) return st;
        }
        if (chosen && element >= 0 && element < 10) chosen[element] = best;
    }
    return OCT_OK;
}

oct_status oct_batch_state_size(oct_batch* b, size_t* n) {
    if (!b || !n) return OCT_EINVAL;
    *n = b->state_off.back();
    return OCT_OK;
}

// Host <-> device state transfer of a batch: per scene n*3 displacements (p - X) then n*3
// velocities.  One contiguous copy to/from a device staging buffer and one kernel that
// scatters/gathers the float4 node arrays.
oct_status oct_batch_set_state(oct_batch* b, const float* host) {
    if (!b || !host) return OCT_EINVAL;
    oct_ctx* c = b->ctx;
    const size_t n = b->state_off.back();
    if (!b->d_state) { oct_status st = b->mem.alloc(b->d_state, n); if (st) return st; }
    OCT_CUDA(c, cudaMemcpyAsync(b->d_state, host, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    launch_state(b->d_scenes, b->d_nwork, b->n_nwork, b->d_soff, b->d_state, 0, c->stream);
    c->launches++;
    return OCT_OK;
}

oct_status oct_batch_get_state(oct_batch* b, float* host) {
    if (!b || !host) return OCT_EINVAL;
    oct_ctx* c = b->ctx;
    const size_t n = b->state_off.back();
    if (!b->d_state) { oct_status st = b->mem.alloc(b->d_state, n); if (st) return st; }
    launch_state(b->d_scenes, b->d_nwork, b->n_nwork, b->d_soff, b->d_state, 1, c->stream);
    c->launches++;
    OCT_CUDA(c, cudaMemcpyAsync(host, b->d_state, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    OCT_CUDA(c, cudaStreamSynchronize(c->stream));
    return OCT_OK;
}

}  // extern "C"
