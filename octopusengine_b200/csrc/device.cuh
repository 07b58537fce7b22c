// Device-side data layout shared by the kernels and the host runtime.
//
// Node state is stored per scene as separate float4 arrays (structure of arrays, one
// 16-byte vector per node so every gather is a single aligned load): the displacement
// u = p - X (positions are X + u), the previous step's displacement, the inertial target
// y with the lumped mass in .w, and the velocity.  Keeping u instead of p makes the
// deformation gradient F = I + sum_i u_i (x) dNx_i free of the cancellation that absolute
// positions cause in FP32 (F of the rest state is exactly I).
//
// Element data: topology E*NE ints, and per (element, quadrature point) a 48-byte record
// of three float4: JX_inv (column-major 9 floats), |det J|, lambda, mu (the quadrature
// volume is |det J| w_q with the compile-time weight w_q).  When every element's map is
// affine (straight-sided tetrahedra, parallelepiped hexahedra: all beam meshes) J does not
// vary over the quadrature points and one record per element is stored (eq_stride = 1
// instead of NQ), which divides the per-visit element bytes by NQ.  The inverse reference
// Jacobians are computed in FP64 on the host and rounded once.
//
// Colour-sorted vertex slots: vids[slot] is the node solved in that slot; slots of colour
// c are [color_off[c], color_off[c+1]) in ascending node id (GPU_VBD_FEM::create_buffers,
// octopus/src/GPU/VBD/GPU_VBD_FEM.cu:594-675); own_off/owners is the owner CSR in slot
// order with owners packed as (element id << 5) | local node index.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace octb {

constexpr int kMaxNE = 27;
constexpr int kMaxNQ = 27;
constexpr int kOwnerShift = 5;
constexpr int kFixGroups = 4;
constexpr int kMaxEffects = 4;

// Scripted constraint effects of the reference's rigid controller (GPU_Crush, GPU_RandomSphere,
// GPU_HighStretch; octopus/include/GPU/GPU_Constraint.h:20-80).  kind < 0: unused slot.  The
// active flag and the stretch distance t live on the device so that toggling an effect does
// not invalidate captured graphs.
struct EffectDev {
    int kind;           // 0 crush, 1 random sphere, 2 high stretch
    int active;
    int n;              // high stretch: number of ids
    int pad;
    const int* ids;     // high stretch: the stretched node ids
    float* t;           // high stretch: current distance (device)
    float cx, cy, cz;   // centre
    float radius;       // random sphere
    float max_dist;     // high stretch
    float pad2[3];
};

struct SceneDev {
    float4* u;          // displacement, per node
    float4* u_last;     // displacement at the start of the sub-step
    float4* y;          // inertial target (xyz) and mass (w)
    float4* v;          // velocity
    float4* u_new;      // Jacobi scratch (colourings with conflicts)
    float4* prev1;      // Chebyshev history (rho > 0)
    float4* prev2;
    int* mask;          // 1 = solved, 0 = fixed (GPU_ParticleSystem mask)
    const float4* X;    // rest positions
    const int* topo;    // n_elements * NE
    const float4* eq;   // n_elements * NQ * 3
    const int* vids;    // n_nodes, colour-sorted
    const int* own_off; // n_nodes + 1, slot order
    const int* owners;  // packed (eid << 5) | r
    const int* fixed;   // n_fixed node ids
    const int* fixed_group;            // n_fixed rigid-group indices
    const int* fix_of;                 // explicit: per node its rigid group if fixed, else -1 (or null)
    const float* fix;                  // kFixGroups x 16: com (3), offset (3), rotation (9, column-major), pad
    int n_nodes, n_elements, n_fixed, element;
    int eq_stride;                     // records per element: NQ, or 1 for affine elements
    const float4* ent;                 // owner entries in slot order (EntryLayout), or null
    const float4* rtab;                // distinct quadrature records of affine elements (3 float4 each)
    float damping;      // k_d
    float gx, gy, gz;
    float bminx, bminy, bminz, bmaxx, bmaxy, bmaxz;
    int box_limit;
    int precision;                     // 0 plain, 1 mixed
    EffectDev* effects;                // kMaxEffects slots (scene memory)
    int* status;                       // per-scene failure flags: kStatusTimeout, kStatusNonFinite
    const int* elems;                  // XPBD: element ids sorted by colour
    const int* etopo;                  // XPBD: their topology in the same order (NE ids per slot)
    float global_damping;              // XPBD velocity damping (GPU_PBD global_damping)
};

// One block of XPBD element work: `count` consecutive entries of one scene's colour-sorted
// element list from `begin` (at most the kernel's elements per block).
struct XWork {
    int scene;
    int begin;
    int count;
    int pad;
};

// Per-scene failure flags (SceneDev::status), read and cleared by the host after a frame.
constexpr int kStatusTimeout = 1;      // a bounded wait gave up on this scene's work
constexpr int kStatusNonFinite = 2;    // a node's position or velocity became NaN / Inf

// One unit of colour work: `count` consecutive colour slots of one scene.  With a fixed
// number of lanes per vertex an item fills one block (128 / lanes slots); in the packed
// mapping an item fills one warp (one lane per (vertex, owner) pair, at most 32 pairs) and
// pair_base is the owner-CSR offset of its first slot.
struct VWork {
    int scene;
    int slot_begin;
    int count;
    int pair_base;
    unsigned heads;   // packed items: bit p set when pair p starts a new vertex
    int n_pairs;      // packed items: number of (vertex, owner) pairs
    int tpv;          // lane-group items: lanes per vertex of this item; 0 = the launch's
    int pad1;
};

// Owner entries: one per (vertex, owner) pair in slot order, contiguous per vertex (and per
// warp item of the packed mapping, so one bulk copy stages a whole item in shared memory).
// An entry holds the owner element's node ids and an index into the scene's record table
// instead of the record itself: the quadrature record (JX_inv, V, lambda, mu; for P1 the
// G_j vectors, V, lambda, mu of the vertex's corner) of every affine element is stored once
// per distinct value (SceneDev::rtab), so a mesh whose elements repeat a few shapes (the
// generated beams and cubes: 6 tetrahedron shapes, 1 hexahedron) streams only node ids.  For
// non-affine elements the index is the element id into the per-point records (SceneDev::eq).
// Node ids take the low kIdBits bits of a word; the spare high bits carry the local index and
// the record index in the entries that have no room for separate words (P1, Q1).
constexpr int kIdBits = 27;
constexpr int kIdMask = (1 << kIdBits) - 1;
constexpr int kSpareBits = 32 - kIdBits;
template <int NE> struct EntryLayout {
    // node ids, then r, then the record index; padded to a multiple of 4 words
    static constexpr int kIds = 0, kR = NE, kRec = NE + 1;
    static constexpr int kWords = ((NE + 2) + 3) / 4 * 4;
    static constexpr long long kMaxRecords = 1ll << 31;
};
// P1: the four node ids with the vertex's own node first; the record index (of the
// element's record for that corner: G_j = JX_inv^T dN_j of the three other nodes in order,
// V, lambda, mu; since sum_i dN_i = 0, F = I + sum_j (u_j - u_own) (x) G_j and the vertex's
// own g = -(G_1 + G_2 + G_3)) is split over the ids' spare bits: 16 B per entry.
template <> struct EntryLayout<4> {
    static constexpr int kIds = 0;
    static constexpr int kWords = 4;
    static constexpr long long kMaxRecords = 1ll << (4 * kSpareBits);
};
// Q1: eight node ids; r in the spare bits of the first, the record index in those of the
// other seven: 32 B per entry.
template <> struct EntryLayout<8> {
    static constexpr int kIds = 0;
    static constexpr int kWords = 8;
    static constexpr long long kMaxRecords = 1ll << 31;
};
inline constexpr int entry_words(int ne) {
    return ne == 4 ? EntryLayout<4>::kWords : ne == 8 ? EntryLayout<8>::kWords : ((ne + 2) + 3) / 4 * 4;
}

// One unit of node-parallel work (predictor, velocity update, Chebyshev).
struct NWork {
    int scene;
    int begin;
    int count;
    int pad;
};

struct StepParams {
    float dt;
    float inv_dt;
    float omega;         // Chebyshev weight of this iteration
    int iteration;       // iteration index within the sub-step
    const int* pending_v0;   // per scene: 1 until its first sub-step has consumed the initial velocity
    int in_place;        // 1: write u directly, 0: write u_new (Jacobi within a colour)
    int* error;          // device error word (bounded waits, non-finite results)
};

}  // namespace octb
