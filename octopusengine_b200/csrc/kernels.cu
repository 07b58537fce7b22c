// sm_100a kernels of the soft-body FEM time step.
//
// VBD colour sweep (replaces kernel_vbd_solve_v1..v4 + kernel_copy_in_position,
// octopus/src/GPU/VBD/GPU_VBD_FEM.cu:124-413).  Work is vertex-centric like the reference,
// but a vertex is owned by a group of TPV lanes of one warp: lane k of the group takes the
// vertex's owners k, k+TPV, ..., gathers that element's node displacements once into
// registers and loops over all quadrature points, accumulating the vertex's force and
// 3x3 Hessian.  The group then reduces with warp shuffles (no shared-memory tree, no
// barrier inside divergent code) and lane 0 applies the damping/inertia terms and the
// 3x3 Newton step.  Many vertices (and scenes) run per block via a work table.
//
// Per-vertex Hessian block in closed form.  The reference assembles
//   H_r = sum_{i<=j} g_i g_j (B_ij + B_ij^T)   (GPU_FEM_Material.cu:250-261)
// from six 3x3 blocks B_ij = d2W/dF_i dF_j (:133-207), g = JX_inv^T dN_r.  Contracting the
// blocks with g once on paper gives, with a = F g, h = cof(F) g, |g|^2:
//   (Stable) Neo-Hookean: H = V (mu |g|^2 I + lambda h h^T)   (the hat(F_k) terms cancel
//                          in B + B^T)
//   Hooke:                H = V (mu + lambda) |g|^2 I
//   StVK (as written):    H = V (|g|^2 [(lambda/2 |F|^2 - mu) I + mu F F^T]
//                               + (lambda/2 + mu) a a^T + |a|^2 I)
// and the force -V P g with P from GPU_FEM_Material.cu:14-36.  This is the same
// arithmetic the reference performs, regrouped: ~100 FP32 instructions per (owner,
// quadrature point) instead of ~400.
//
// Node gathers read the displacement u (see device.cuh), F = I + Jx JX_inv with
// Jx = sum_i u_i (x) dN_qi.  The reference-element derivatives dN live in __constant__
// memory for the warp-uniform Jx loops and are staged into shared memory with a TMA bulk
// copy for the lane-varying dN_r lookups.
#include <cstdio>

#include "device.cuh"
#include "kernels.cuh"
#include "shape_tables.inc"

namespace octb {

template <int E> struct ElemT;
template <> struct ElemT<3> { static constexpr int NE = 4, NQ = 1; };
template <> struct ElemT<6> { static constexpr int NE = 8, NQ = 8; };
template <> struct ElemT<7> { static constexpr int NE = 10, NQ = 4; };
template <> struct ElemT<8> { static constexpr int NE = 20, NQ = 11; };
template <> struct ElemT<9> { static constexpr int NE = 27, NQ = 27; };

__constant__ float c_dN3[1 * 4 * 3];
__constant__ float c_dN6[8 * 8 * 3];
__constant__ float c_dN7[4 * 10 * 3];
__constant__ float c_dN8[11 * 20 * 3];
__constant__ float c_dN9[27 * 27 * 3];

template <int E> __device__ __forceinline__ const float* cdN();
template <> __device__ __forceinline__ const float* cdN<3>() { return c_dN3; }
template <> __device__ __forceinline__ const float* cdN<6>() { return c_dN6; }
template <> __device__ __forceinline__ const float* cdN<7>() { return c_dN7; }
template <> __device__ __forceinline__ const float* cdN<8>() { return c_dN8; }
template <> __device__ __forceinline__ const float* cdN<9>() { return c_dN9; }

// Global copies (16-byte padded) used as the TMA bulk-copy source.
__device__ __align__(16) float g_dN3[16];
__device__ __align__(16) float g_dN6[192];
__device__ __align__(16) float g_dN7[120];
__device__ __align__(16) float g_dN8[660];
__device__ __align__(16) float g_dN9[2188];
// FP64 copies of the tables for the diagnostics kernel.
__device__ double g_dNd3[12], g_dNd6[192], g_dNd7[120], g_dNd8[660], g_dNd9[2187];
__device__ double g_wd3[1], g_wd6[8], g_wd7[4], g_wd8[11], g_wd9[27];
template <int E> __device__ __forceinline__ const double* gdNd() {
    if constexpr (E == 3) return g_dNd3; else if constexpr (E == 6) return g_dNd6; else if constexpr (E == 7) return g_dNd7;
    else if constexpr (E == 8) return g_dNd8; else return g_dNd9;
}
template <int E> __device__ __forceinline__ const double* gwd() {
    if constexpr (E == 3) return g_wd3; else if constexpr (E == 6) return g_wd6; else if constexpr (E == 7) return g_wd7;
    else if constexpr (E == 8) return g_wd8; else return g_wd9;
}
template <int E> __device__ __forceinline__ const float* gdN();
template <> __device__ __forceinline__ const float* gdN<3>() { return g_dN3; }
template <> __device__ __forceinline__ const float* gdN<6>() { return g_dN6; }
template <> __device__ __forceinline__ const float* gdN<7>() { return g_dN7; }
template <> __device__ __forceinline__ const float* gdN<8>() { return g_dN8; }
template <> __device__ __forceinline__ const float* gdN<9>() { return g_dN9; }

// Reference-element derivative dN_qi[k] and quadrature weight w_q.  For every element but
// Hexa_27 the loops that read them are fully unrolled, so they are compile-time constants
// (exact zeros drop out of the FMAs); Hexa_27's 27 x 27 table is read from constant memory.
template <int E> __device__ __forceinline__ float dn(int q, int i, int k) {
    if constexpr (E == 9) return c_dN9[(q * 27 + i) * 3 + k];
    else return ShapeConst<E>::dN((q * ElemT<E>::NE + i) * 3 + k);
}
__constant__ float c_w9[27];
template <int E> __device__ __forceinline__ float wq(int q) {
    if constexpr (E == 9) return c_w9[q];
    else return ShapeConst<E>::w(q);
}

constexpr int kBlock = 128;
constexpr long kSpinLimit = 1L << 22;

// Programmatic dependent launch.  The kernels of a sub-step (predictor, colour sweeps,
// constraints, Chebyshev, velocity, XPBD colours) are launched with programmatic stream
// serialisation: each lets the next one launch once all its blocks have started
// (pdl_trigger), so that launch and the next kernel's data-independent prologue (the TMA
// staging of the constant dN table) overlap this kernel's tail; pdl_wait() then blocks until
// the preceding kernel has completed and its writes are visible.  Both are no-ops for a
// normal launch.  Every kernel launched by launch_pdl calls pdl_wait() before it reads
// anything a preceding kernel may write.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ------------------------------------------------------------------------ TMA staging
// One elected thread issues a cp.async.bulk global->shared copy tracked by an mbarrier;
// every thread waits on the barrier with an iteration limit.  The phase completes once for
// the whole block, so one thread seeing it complete means the copy has landed; the block
// decides together (__syncthreads_or) whether any thread saw it.  If none did, the kernel
// records a time-out, gives the copy in flight a second bounded wait (so it does not land
// after the fallback or after the block has left), then loads the table with plain loads:
// a wait can never hang the GPU and every thread reaches the same barriers.
__device__ __forceinline__ bool mbar_wait(unsigned mb, unsigned phase, long limit);
__device__ __forceinline__ void stage_table(float* s_dst, const float* g_src, int n_floats, unsigned long long* mbar,
                                            int* error) {
    const int bytes = ((n_floats * 4 + 15) / 16) * 16;
    const unsigned mb = (unsigned)__cvta_generic_to_shared(mbar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(s_dst);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(dst), "l"(g_src), "r"(bytes), "r"(mb) : "memory");
    }
    const bool done = mbar_wait(mb, 0, kSpinLimit);
    if (!__syncthreads_or(done)) {   // block-uniform: nobody saw the copy land
        if (threadIdx.x == 0 && error) atomicOr(error, 1);
        mbar_wait(mb, 0, kSpinLimit);
        __syncthreads();
        for (int i = threadIdx.x; i < n_floats; i += blockDim.x) s_dst[i] = g_src[i];
    }
    __syncthreads();
}

// ------------------------------------------------------------------------ L2 policies
// Node displacements are gathered many times per sweep (every element around a node) and,
// for a whole batch, fit in L2; the per-visit element stream (owners, topology, quadrature
// records) is read once per visit.  Loads carry L2 eviction priorities accordingly:
// gathers evict_last, streams evict_first (createpolicy + ld.global.nc.L2::cache_hint).
__device__ __forceinline__ unsigned long long policy_keep() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ unsigned long long policy_stream() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ float4 ld_hint(const float4* a, unsigned long long pol) {
    float4 v;
    asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_hint(const int* a, unsigned long long pol) {
    int v;
    asm("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
    return v;
}

// ------------------------------------------------------------------------ helpers
struct V3 { float x, y, z; };
__device__ __forceinline__ V3 mk(float a, float b, float c) { return {a, b, c}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
__device__ __forceinline__ V3 xyz(float4 a) { return {a.x, a.y, a.z}; }

// Compensated accumulation (Kahan): s + c carries the running sum to ~2^-48 relative.
__device__ __forceinline__ void kadd(float& s, float& c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// Element types whose mixed-precision force is compensated once per owner element, after a
// plain sum over its quadrature points, instead of once per point: the many-point elements
// (P3 11 points, Q2 27), where the per-point compensation is a long dependent chain (sweep
// rate measured +5 % P3, +32 % Q2; per point stays faster for P1, Q1 and P2).
#ifndef OCTB_COMPENSATE_PER_ELEMENT_EXTRA
#define OCTB_COMPENSATE_PER_ELEMENT_EXTRA 0   // bit E: also compensate per element for element type E
#endif
template <int E> struct CompensatePerElement {
    static constexpr bool value = E == 8 || E == 9 || ((OCTB_COMPENSATE_PER_ELEMENT_EXTRA >> E) & 1);
};

// Contribution of one quadrature point: f (3) and the symmetric H (6: 00 01 02 11 12 22).
template <int MAT>
__device__ __forceinline__ void material_terms(V3 F0, V3 F1, V3 F2, V3 g, float lam, float mu, float V, float out[9]) {
    const float gg = dot(g, g);
    const V3 a = F0 * g.x + F1 * g.y + F2 * g.z;   // F g
    if (MAT == 2 || MAT == 3) {
        const V3 C0 = cross(F1, F2), C1 = cross(F2, F0), C2 = cross(F0, F1);
        const float J = dot(F0, C0);
        const V3 h = C0 * g.x + C1 * g.y + C2 * g.z;   // cof(F) g
        // lambda (J - alpha) with alpha = 1 + mu/lambda (Stable NH) or 1 (NH)
        const float s = MAT == 3 ? lam * (J - 1.f) - mu : lam * (J - 1.f);
        const V3 Pg = a * mu + h * s;
        const float lv = lam * V, dv = mu * gg * V;
        out[0] = -V * Pg.x; out[1] = -V * Pg.y; out[2] = -V * Pg.z;
        out[3] = dv + lv * h.x * h.x; out[4] = lv * h.x * h.y; out[5] = lv * h.x * h.z;
        out[6] = dv + lv * h.y * h.y; out[7] = lv * h.y * h.z; out[8] = dv + lv * h.z * h.z;
    } else if (MAT == 0) {
        // E = (F + F^T)/2 - I ; P = lambda tr(E) I + mu E
        const float trE = F0.x + F1.y + F2.z - 3.f;
        // (E g)_r = sum_c E_rc g_c, E_rc = (F_rc + F_cr)/2 - d_rc, F_rc = column c row r
        const V3 Ftg = mk(dot(F0, g), dot(F1, g), dot(F2, g));   // F^T g
        const V3 Eg = (a + Ftg) * 0.5f - g;
        const V3 Pg = g * (lam * trE) + Eg * mu;
        const float d = (mu + lam) * gg * V;
        out[0] = -V * Pg.x; out[1] = -V * Pg.y; out[2] = -V * Pg.z;
        out[3] = d; out[4] = 0.f; out[5] = 0.f; out[6] = d; out[7] = 0.f; out[8] = d;
    } else {
        // StVK: E = (F^T F - I)/2, P = lambda tr(E) F + 2 mu F E
        const float f00 = dot(F0, F0), f01 = dot(F0, F1), f02 = dot(F0, F2);
        const float f11 = dot(F1, F1), f12 = dot(F1, F2), f22 = dot(F2, F2);
        const float nF = f00 + f11 + f22;
        const float trE = 0.5f * (nF - 3.f);
        const V3 Eg = mk(0.5f * ((f00 - 1.f) * g.x + f01 * g.y + f02 * g.z),
                         0.5f * (f01 * g.x + (f11 - 1.f) * g.y + f12 * g.z),
                         0.5f * (f02 * g.x + f12 * g.y + (f22 - 1.f) * g.z));
        const V3 FEg = F0 * Eg.x + F1 * Eg.y + F2 * Eg.z;
        const V3 Pg = a * (lam * trE) + FEg * (2.f * mu);
        const float dg = gg * (0.5f * lam * nF - mu) + dot(a, a);
        const float mg = mu * gg, ca = 0.5f * lam + mu;
        // F F^T = sum_c F_c F_c^T
        const float m00 = F0.x * F0.x + F1.x * F1.x + F2.x * F2.x, m01 = F0.x * F0.y + F1.x * F1.y + F2.x * F2.y;
        const float m02 = F0.x * F0.z + F1.x * F1.z + F2.x * F2.z, m11 = F0.y * F0.y + F1.y * F1.y + F2.y * F2.y;
        const float m12 = F0.y * F0.z + F1.y * F1.z + F2.y * F2.z, m22 = F0.z * F0.z + F1.z * F1.z + F2.z * F2.z;
        out[0] = -V * Pg.x; out[1] = -V * Pg.y; out[2] = -V * Pg.z;
        out[3] = V * (dg + mg * m00 + ca * a.x * a.x); out[4] = V * (mg * m01 + ca * a.x * a.y);
        out[5] = V * (mg * m02 + ca * a.x * a.z); out[6] = V * (dg + mg * m11 + ca * a.y * a.y);
        out[7] = V * (mg * m12 + ca * a.y * a.z); out[8] = V * (dg + mg * m22 + ca * a.z * a.z);
    }
}

// Hexa8 node signs (Element numbering of the reference: bottom face counter-clockwise, then the
// top face); its 2x2x2 Gauss points are the same signs over sqrt(3), in the same order.
__device__ constexpr int kHexSign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                           {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
struct HexCoef { V3 x, y, z, xy, xz, yz, xyz; };

// Monomial coefficients (times 1/8) of a trilinear field from its 8 nodal values:
// u = a0 + a_x xi + a_y eta + a_z zeta + a_xy xi eta + a_xz xi zeta + a_yz eta zeta + a_xyz xi eta zeta.
// Nodes i and i + 4 differ only in z; on each face, (0, 3) and (1, 2) differ only in y.
__device__ __forceinline__ void hex_q1_coefficients(const float* ux, const float* uy, const float* uz, HexCoef& h) {
    V3 p[4], m[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const V3 lo = mk(ux[i], uy[i], uz[i]), hi = mk(ux[i + 4], uy[i + 4], uz[i + 4]);
        p[i] = hi + lo;   // z-even
        m[i] = hi - lo;   // z-odd
    }
    // y stage on each half: x- pair (0, 3), x+ pair (1, 2)
    const V3 pe0 = p[0] + p[3], po0 = p[3] - p[0], pe1 = p[1] + p[2], po1 = p[2] - p[1];
    const V3 me0 = m[0] + m[3], mo0 = m[3] - m[0], me1 = m[1] + m[2], mo1 = m[2] - m[1];
    constexpr float s = 0.125f;
    h.x = (pe1 - pe0) * s;   h.y = (po1 + po0) * s;   h.xy = (po1 - po0) * s;
    h.z = (me1 + me0) * s;   h.xz = (me1 - me0) * s;  h.yz = (mo1 + mo0) * s;   h.xyz = (mo1 - mo0) * s;
}

// P2 (Tetra_10) Jx from its barycentric structure.  With L = (1 - xi - eta - zeta, xi, eta,
// zeta), du/dxi_k = D_k - D_0 where D_i = du/dL_i = (4 L_i - 1) u_i + 4 sum_j L_j u_ij (u_ij the
// edge node between corners i and j) is linear in L.  The 4-point rule puts L = b at one corner
// p(q) = (q + 1) mod 4 and L = a at the other three, so with S_i the sum of the three edge nodes
// at corner i and Pa_i = (4a - 1) u_i + 4a S_i:
//   D_i(q) = Pa_i + c w_i(q),  c = 4 (b - a),  w_i = u_i if i == p(q), else u_{i p(q)},
//   J_k(q) = R_k + c (w_k - w_0),  R_k = Pa_k - Pa_0,
// 18 operations per point after a 57-operation setup per element, instead of a dense 10-node
// contraction (63 FMAs per point).  p2_layout_matches() checks this layout against the dN
// table at compile time.
constexpr double kP2a = 0.1381966011250105152, kP2b = 0.5854101966249684544;   // (5 - sqrt 5)/20, (5 + 3 sqrt 5)/20
__host__ __device__ constexpr int p2_edge_node(int i, int j) {
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    return lo == 0 ? (hi == 1 ? 4 : hi == 2 ? 6 : 7) : lo == 1 ? (hi == 2 ? 5 : 8) : 9;
}
__host__ __device__ constexpr bool p2_layout_matches() {
    constexpr double dL[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int q = 0; q < 4; ++q) {
        double L[4] = {0, 0, 0, 0};
        for (int i = 0; i < 4; ++i) L[i] = i == (q + 1) % 4 ? kP2b : kP2a;
        for (int n = 0; n < 10; ++n)
            for (int k = 0; k < 3; ++k) {
                double v = 0;
                if (n < 4) {
                    v = (4 * L[n] - 1) * dL[n][k];
                } else {
                    for (int i = 0; i < 4; ++i)
                        for (int j = i + 1; j < 4; ++j)
                            if (p2_edge_node(i, j) == n) v = 4 * (L[j] * dL[i][k] + L[i] * dL[j][k]);
                }
                const double d = v - (double)ShapeConst<7>::dN((q * 10 + n) * 3 + k);
                if (d > 1e-6 || d < -1e-6) return false;
            }
    }
    return true;
}
static_assert(p2_layout_matches(), "P2 barycentric Jx: point or node layout differs from the dN table");

struct P2Base { V3 R1, R2, R3; };
__device__ __forceinline__ void p2_base(const float* ux, const float* uy, const float* uz, P2Base& b) {
    auto U = [&](int n) { return mk(ux[n], uy[n], uz[n]); };
    constexpr float ca = (float)(4 * kP2a - 1), cs = (float)(4 * kP2a);
    V3 Pa[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int j0 = i == 0 ? 1 : 0, j1 = i <= 1 ? 2 : 1, j2 = i <= 2 ? 3 : 2;
        const V3 S = U(p2_edge_node(i, j0)) + U(p2_edge_node(i, j1)) + U(p2_edge_node(i, j2));
        Pa[i] = U(i) * ca + S * cs;
    }
    b.R1 = Pa[1] - Pa[0]; b.R2 = Pa[2] - Pa[0]; b.R3 = Pa[3] - Pa[0];
}
// q is a constant once the point loop is unrolled, so the node choices below fold away.
__device__ __forceinline__ void p2_jacobian(const float* ux, const float* uy, const float* uz, const P2Base& b, int q,
                                            V3& J0, V3& J1, V3& J2) {
    auto U = [&](int n) { return mk(ux[n], uy[n], uz[n]); };
    const int p = (q + 1) & 3;
    constexpr float c = (float)(4 * (kP2b - kP2a));
    auto W = [&](int i) { return i == p ? U(i) : U(p2_edge_node(i, p)); };
    const V3 w0 = W(0);
    J0 = b.R1 + (W(1) - w0) * c;
    J1 = b.R2 + (W(2) - w0) * c;
    J2 = b.R3 + (W(3) - w0) * c;
}

// f and H contributions of one owner element (all its quadrature points) to its node r,
// given the element's node displacements and its first quadrature record (A, B, C); for
// non-affine elements the later records are read from rec.
template <int E, int MAT>
__device__ __forceinline__ void element_terms(const float* ux, const float* uy, const float* uz, int r, float4 A, float4 B,
                                              float4 C, const float4* __restrict__ rec, bool affine,
                                              const float* __restrict__ s_dN, bool mixed, float acc[9], float cmp[9],
                                              unsigned long long stream) {
    constexpr int NE = ElemT<E>::NE, NQ = ElemT<E>::NQ;
    float fs[3] = {0.f, 0.f, 0.f};   // CompensatePerElement: the element's force over its points
    // Q1: u(xi) is trilinear, so Jx at every point follows from the seven non-constant monomial
    // coefficients a_m = 1/8 sum_i s_m(i) u_i (three butterfly stages over the node signs)
    // instead of a dense 8-node contraction per point (hex_q1_coefficients).
    [[maybe_unused]] HexCoef hc;
    if constexpr (E == 6) hex_q1_coefficients(ux, uy, uz, hc);
    [[maybe_unused]] P2Base p2;
    if constexpr (E == 7) p2_base(ux, uy, uz, p2);
#pragma unroll (NQ <= 11 ? NQ : 1)
    for (int q = 0; q < NQ; ++q) {
        if (!affine && q > 0) { A = ld_hint(rec + 3 * q, stream); B = ld_hint(rec + 3 * q + 1, stream); C = ld_hint(rec + 3 * q + 2, stream); }
        // Jx columns: Jk = sum_i u_i dN_qi[k]
        V3 J0 = mk(0, 0, 0), J1 = mk(0, 0, 0), J2 = mk(0, 0, 0);
        if constexpr (E == 6) {
            // Gauss point q sits at (s_q0, s_q1, s_q2) / sqrt(3), s_q the signs of node q
            constexpr float c = 0.57735026918962576f;
            const float xi = c * kHexSign[q][0], et = c * kHexSign[q][1], ze = c * kHexSign[q][2];
            J0 = hc.x + hc.xy * et + hc.xz * ze + hc.xyz * (et * ze);
            J1 = hc.y + hc.xy * xi + hc.yz * ze + hc.xyz * (xi * ze);
            J2 = hc.z + hc.xz * xi + hc.yz * et + hc.xyz * (xi * et);
        } else if constexpr (E == 7) {
            p2_jacobian(ux, uy, uz, p2, q, J0, J1, J2);
        } else {
#pragma unroll
            for (int i = 0; i < NE; ++i) {
                const float d0 = dn<E>(q, i, 0), d1 = dn<E>(q, i, 1), d2 = dn<E>(q, i, 2);
                J0.x = fmaf(ux[i], d0, J0.x); J0.y = fmaf(uy[i], d0, J0.y); J0.z = fmaf(uz[i], d0, J0.z);
                J1.x = fmaf(ux[i], d1, J1.x); J1.y = fmaf(uy[i], d1, J1.y); J1.z = fmaf(uz[i], d1, J1.z);
                J2.x = fmaf(ux[i], d2, J2.x); J2.y = fmaf(uy[i], d2, J2.y); J2.z = fmaf(uz[i], d2, J2.z);
            }
        }
        // JX_inv columns m_b (m_b[k] = row k, column b)
        const V3 m0 = mk(A.x, A.y, A.z), m1 = mk(A.w, B.x, B.y), m2 = mk(B.z, B.w, C.x);
        const float V = C.y * wq<E>(q), lam = C.z, mu = C.w;
        // F_b = e_b + sum_k J_k m_b[k]
        V3 F0 = J0 * m0.x + J1 * m0.y + J2 * m0.z;
        V3 F1 = J0 * m1.x + J1 * m1.y + J2 * m1.z;
        V3 F2 = J0 * m2.x + J1 * m2.y + J2 * m2.z;
        F0.x += 1.f; F1.y += 1.f; F2.z += 1.f;
        const float* dr = s_dN + (q * NE + r) * 3;
        const V3 dnr = mk(dr[0], dr[1], dr[2]);
        const V3 g = mk(dot(m0, dnr), dot(m1, dnr), dot(m2, dnr));
        float t[9];
        material_terms<MAT>(F0, F1, F2, g, lam, mu, V, t);
        // mixed precision: compensated accumulation of the force, whose sum of nearly
        // cancelling element terms sets the converged solution; the Hessian only scales
        // the Newton step and is summed directly
        if (mixed) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (CompensatePerElement<E>::value) fs[k] += t[k];
                else kadd(acc[k], cmp[k], t[k]);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) acc[k] += t[k];
        }
#pragma unroll
        for (int k = 3; k < 9; ++k) acc[k] += t[k];
    }
    if (CompensatePerElement<E>::value && mixed) {
#pragma unroll
        for (int k = 0; k < 3; ++k) kadd(acc[k], cmp[k], fs[k]);
    }
}

// Owner given as a packed (element, local node) id: topology and records from global memory.
template <int E, int MAT>
__device__ __forceinline__ void owner_terms(const SceneDev& S, int packed, const float* __restrict__ s_dN, bool mixed,
                                            float acc[9], float cmp[9]) {
    constexpr int NE = ElemT<E>::NE;
    const int eid = packed >> kOwnerShift, r = packed & ((1 << kOwnerShift) - 1);
    const int* __restrict__ tp = S.topo + (size_t)eid * NE;
    const unsigned long long keep = policy_keep(), stream = policy_stream();
    float ux[NE], uy[NE], uz[NE];
#pragma unroll
    for (int i = 0; i < NE; ++i) {
        const float4 t = ld_hint(&S.u[ld_hint(tp + i, stream)], keep);
        ux[i] = t.x; uy[i] = t.y; uz[i] = t.z;
    }
    const float4* __restrict__ rec = S.eq + (size_t)eid * S.eq_stride * 3;
    const float4 A = ld_hint(rec, stream), B = ld_hint(rec + 1, stream), C = ld_hint(rec + 2, stream);
    element_terms<E, MAT>(ux, uy, uz, r, A, B, C, rec, S.eq_stride == 1, s_dN, mixed, acc, cmp, stream);
}

// Owner entry fields (EntryLayout): node ids in the low kIdBits bits; r and the record index
// in separate words, or (P1, Q1) in the ids' spare bits.
__device__ __forceinline__ int entry_node(const float* en, int i) { return __float_as_int(en[i]) & kIdMask; }
__device__ __forceinline__ unsigned entry_spare(const float* en, int i) { return (unsigned)__float_as_int(en[i]) >> kIdBits; }
template <int NE> __device__ __forceinline__ int entry_r(const float* en) {
    if constexpr (NE == 4) return 0;   // own node first
    else if constexpr (NE == 8) return (int)entry_spare(en, 0);
    else return __float_as_int(en[EntryLayout<NE>::kR]);
}
template <int NE> __device__ __forceinline__ int entry_rec(const float* en) {
    if constexpr (NE == 4) {
        return (int)(entry_spare(en, 0) | entry_spare(en, 1) << kSpareBits | entry_spare(en, 2) << (2 * kSpareBits) |
                     entry_spare(en, 3) << (3 * kSpareBits));
    } else if constexpr (NE == 8) {
        unsigned v = 0;
#pragma unroll
        for (int j = 1; j < 8; ++j) v |= entry_spare(en, j) << (kSpareBits * (j - 1));
        return (int)(v & 0x7fffffffu);
    } else {
        return __float_as_int(en[EntryLayout<NE>::kRec]);
    }
}

// Owner given as an entry (EntryLayout), staged in shared memory or held in registers.
template <int E, int MAT>
__device__ __forceinline__ void entry_terms(const SceneDev& S, const float* __restrict__ en, const float* __restrict__ s_dN,
                                            bool mixed, float acc[9], float cmp[9]) {
    constexpr int NE = ElemT<E>::NE, NQ = ElemT<E>::NQ;
    const unsigned long long keep = policy_keep(), stream = policy_stream();
    if constexpr (NE == 4) {   // P1: own node first, the corner's record holds G_j of the other three
        const float4 u0 = ld_hint(&S.u[entry_node(en, 0)], keep);
        const float4 u1 = ld_hint(&S.u[entry_node(en, 1)], keep);
        const float4 u2 = ld_hint(&S.u[entry_node(en, 2)], keep);
        const float4 u3 = ld_hint(&S.u[entry_node(en, 3)], keep);
        const float4* R = S.rtab + 3 * (size_t)entry_rec<NE>(en);
        const float4 R0 = ld_hint(R, keep), R1 = ld_hint(R + 1, keep), R2 = ld_hint(R + 2, keep);
        const V3 d1 = xyz(u1) - xyz(u0), d2 = xyz(u2) - xyz(u0), d3 = xyz(u3) - xyz(u0);
        const V3 g1 = mk(R0.x, R0.y, R0.z), g2 = mk(R0.w, R1.x, R1.y), g3 = mk(R1.z, R1.w, R2.x);
        // F_b = e_b + sum_j d_j G_j[b]
        V3 F0 = d1 * g1.x + d2 * g2.x + d3 * g3.x;
        V3 F1 = d1 * g1.y + d2 * g2.y + d3 * g3.y;
        V3 F2 = d1 * g1.z + d2 * g2.z + d3 * g3.z;
        F0.x += 1.f; F1.y += 1.f; F2.z += 1.f;
        const V3 g = mk(-(g1.x + g2.x + g3.x), -(g1.y + g2.y + g3.y), -(g1.z + g2.z + g3.z));
        float t[9];
        material_terms<MAT>(F0, F1, F2, g, R2.z, R2.w, R2.y * wq<E>(0), t);
        if (mixed) {
#pragma unroll
            for (int k = 0; k < 3; ++k) kadd(acc[k], cmp[k], t[k]);
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) acc[k] += t[k];
        }
#pragma unroll
        for (int k = 3; k < 9; ++k) acc[k] += t[k];
        return;
    } else {
    float ux[NE], uy[NE], uz[NE];
#pragma unroll
    for (int i = 0; i < NE; ++i) {
        const float4 t = ld_hint(&S.u[entry_node(en, i)], keep);
        ux[i] = t.x; uy[i] = t.y; uz[i] = t.z;
    }
    const int r = entry_r<NE>(en), rec = entry_rec<NE>(en);
    const bool affine = S.eq_stride == 1;
    // affine: the element's record in the table of distinct records (small, cached);
    // otherwise rec is the element id into its per-point records
    const float4* R = affine ? S.rtab + 3 * (size_t)rec : S.eq + (size_t)rec * NQ * 3;
    const float4 A = ld_hint(R, affine ? keep : stream), B = ld_hint(R + 1, affine ? keep : stream),
                 C = ld_hint(R + 2, affine ? keep : stream);
    element_terms<E, MAT>(ux, uy, uz, r, A, B, C, R, affine, s_dN, mixed, acc, cmp, stream);
    }
}

// Solve of one vertex: damping and inertia terms (compute_correction,
// octopus/src/GPU/VBD/GPU_VBD_FEM.cu:107-122), then the 3x3 Newton step.
__device__ __forceinline__ V3 newton_step(const float acc[9], float4 uu, float4 ul, float4 yy, float damping, float inv_dt,
                                          int precision) {
    float f0 = acc[0], f1 = acc[1], f2 = acc[2];
    float h00 = acc[3], h01 = acc[4], h02 = acc[5], h11 = acc[6], h12 = acc[7], h22 = acc[8];
    const float kd = damping * inv_dt;
    const float dx = uu.x - ul.x, dy = uu.y - ul.y, dz = uu.z - ul.z;
    f0 -= kd * (h00 * dx + h01 * dy + h02 * dz);
    f1 -= kd * (h01 * dx + h11 * dy + h12 * dz);
    f2 -= kd * (h02 * dx + h12 * dy + h22 * dz);
    const float s = 1.f + kd;
    h00 *= s; h01 *= s; h02 *= s; h11 *= s; h12 *= s; h22 *= s;
    const float mh2 = yy.w * inv_dt * inv_dt;
    f0 -= mh2 * (uu.x - yy.x); f1 -= mh2 * (uu.y - yy.y); f2 -= mh2 * (uu.z - yy.z);
    h00 += mh2; h11 += mh2; h22 += mh2;
    const float c00 = h11 * h22 - h12 * h12, c01 = h02 * h12 - h01 * h22, c02 = h01 * h12 - h02 * h11;
    const float c11 = h00 * h22 - h02 * h02, c12 = h01 * h02 - h00 * h12, c22 = h00 * h11 - h01 * h01;
    const float det = h00 * c00 + h01 * c01 + h02 * c02;
    const float ad = fabsf(det);
    if (precision == 0) {
        if (!(ad > 1e-6f)) return mk(0.f, 0.f, 0.f);
        const float id = 1.f / det;
        return mk((c00 * f0 + c01 * f1 + c02 * f2) * id, (c01 * f0 + c11 * f1 + c12 * f2) * id,
                  (c02 * f0 + c12 * f1 + c22 * f2) * id);
    }
    // Mixed precision: FP32 solve when the block is well conditioned, FP64 otherwise.
    const float hm = fmaxf(fmaxf(fabsf(h00), fabsf(h11)), fabsf(h22));
    if (ad > 1e-6f && ad > 1e-4f * hm * hm * hm) {
        const float id = 1.f / det;
        return mk((c00 * f0 + c01 * f1 + c02 * f2) * id, (c01 * f0 + c11 * f1 + c12 * f2) * id,
                  (c02 * f0 + c12 * f1 + c22 * f2) * id);
    }
    const double H00 = h00, H01 = h01, H02 = h02, H11 = h11, H12 = h12, H22 = h22;
    const double C00 = H11 * H22 - H12 * H12, C01 = H02 * H12 - H01 * H22, C02 = H01 * H12 - H02 * H11;
    const double C11 = H00 * H22 - H02 * H02, C12 = H01 * H02 - H00 * H12, C22 = H00 * H11 - H01 * H01;
    const double D = H00 * C00 + H01 * C01 + H02 * C02;
    const double hmd = (double)hm;
    if (!(fabs(D) > 1e-14 * hmd * hmd * hmd) || !(fabs(D) > 0.0)) return mk(0.f, 0.f, 0.f);
    const double iD = 1.0 / D;
    return mk((float)((C00 * f0 + C01 * f1 + C02 * f2) * iD), (float)((C01 * f0 + C11 * f1 + C12 * f2) * iD),
              (float)((C02 * f0 + C12 * f1 + C22 * f2) * iD));
}

// ------------------------------------------------------------------------ colour kernels
// Per-vertex epilogue. mode 0: VBD solve; mode 1: VBD residual (writes |r| reductions);
// mode 2: explicit force (kernel_fem_eval_force, GPU_FEM_Explicit.cu:5-64).
__device__ __forceinline__ void vertex_epilogue(const SceneDev& S, int vid, const float acc[9], int mode, const StepParams& P,
                                                double* red) {
    const float4 uu = S.u[vid], ul = S.u_last[vid], yy = S.y[vid];
    if (mode == 0) {
        const V3 d = newton_step(acc, uu, ul, yy, S.damping, P.inv_dt, S.precision);
        const float4 un = make_float4(uu.x + d.x, uu.y + d.y, uu.z + d.z, uu.w);
        if (P.in_place) S.u[vid] = un; else S.u_new[vid] = un;
    } else if (mode == 1) {
        // kernel_vbd_compute_residual (GPU_VBD_FEM.cu:482-546)
        const float kd = S.damping * P.inv_dt, mh2 = yy.w * P.inv_dt * P.inv_dt;
        const float dx = uu.x - ul.x, dy = uu.y - ul.y, dz = uu.z - ul.z;
        const double r0 = acc[0] - kd * (acc[3] * dx + acc[4] * dy + acc[5] * dz) - mh2 * (uu.x - yy.x);
        const double r1 = acc[1] - kd * (acc[4] * dx + acc[6] * dy + acc[7] * dz) - mh2 * (uu.y - yy.y);
        const double r2 = acc[2] - kd * (acc[5] * dx + acc[7] * dy + acc[8] * dz) - mh2 * (uu.z - yy.z);
        const double nr = sqrt(r0 * r0 + r1 * r1 + r2 * r2);
        S.u_new[vid] = make_float4((float)r0, (float)r1, (float)r2, 0.f);   // per-vertex residual (get_forces)
        if (!isfinite(nr)) atomicOr(P.error, 2);
        else {
            atomicAdd(red, nr);
            unsigned long long* mx = reinterpret_cast<unsigned long long*>(red + 1);
            atomicMax(mx, (unsigned long long)__double_as_longlong(nr));
        }
    } else {
        // f = sum(-P g V) - k_d H v, written to u_new (the force buffer of the explicit solver)
        const float4 vv = S.v[vid];
        const float kd = S.damping;
        float4 f;
        f.x = acc[0] - kd * (acc[3] * vv.x + acc[4] * vv.y + acc[5] * vv.z);
        f.y = acc[1] - kd * (acc[4] * vv.x + acc[6] * vv.y + acc[7] * vv.z);
        f.z = acc[2] - kd * (acc[5] * vv.x + acc[7] * vv.y + acc[8] * vv.z);
        f.w = 0.f;
        S.u_new[vid] = f;
    }
}

// Bounded wait on an mbarrier phase; false when the iteration limit ran out.
__device__ __forceinline__ bool mbar_wait(unsigned mb, unsigned phase, long limit) {
    unsigned done = 0;
    for (long it = 0; it < limit && !done; ++it)
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done) : "r"(mb), "r"(phase) : "memory");
    return done != 0;
}

// Packed mapping: one lane per (vertex, owner) pair.  The host packs whole vertices of one
// colour into warp items (at most 32 pairs each, heads = bit mask of each vertex's first
// pair), so lanes are busy whatever the valences; each vertex's terms are summed with a
// segmented shuffle reduction into its first lane, which runs the epilogue.  Each warp
// stages its items' owner entries (node ids, local index, quadrature record; contiguous in
// slot order) into shared memory with cp.async.bulk, double-buffered on two mbarriers:
// the next item's entries arrive while the current item computes, leaving the node-
// displacement gathers as the only dependent global loads.
// Resident blocks per SM each element type is compiled for (register cap without spills).
template <int E> struct MinBlocks { static constexpr int value = E == 3 ? 8 : (E == 7 ? 5 : (E == 6 ? 4 : (E == 8 ? 4 : 2))); };

template <int E, int MAT>
__global__ void __launch_bounds__(kBlock, MinBlocks<E>::value) k_vertex_packed(const SceneDev* __restrict__ scenes,
                                                          const VWork* __restrict__ work, int n_work, int mode,
                                                          StepParams P, double* red) {
    constexpr int NE = ElemT<E>::NE, NQ = ElemT<E>::NQ;
    constexpr int EW = EntryLayout<NE>::kWords;
    constexpr int WPB = kBlock / 32;
    __shared__ __align__(128) float s_dN[((NQ * NE * 3 + 3) / 4) * 4];
    __shared__ __align__(8) unsigned long long s_mbar;
    __shared__ __align__(8) unsigned long long s_bar[WPB][2];
    extern __shared__ __align__(128) float s_ent[];   // [WPB][2][32 * EW]
    stage_table(s_dN, gdN<E>(), NQ * NE * 3, &s_mbar, P.error);
    const unsigned full = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned bar0 = (unsigned)__cvta_generic_to_shared(&s_bar[warp][0]);
    const unsigned bar1 = (unsigned)__cvta_generic_to_shared(&s_bar[warp][1]);
    float* buf0 = s_ent + (size_t)warp * 2 * 32 * EW;
    float* buf1 = buf0 + 32 * EW;
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    auto issue = [&](int item, int b) {   // lane 0: bulk-copy the item's entries into buffer b
        const VWork wk = work[item];
        const float4* src = scenes[wk.scene].ent + (size_t)wk.pair_base * (EW / 4);
        const unsigned bytes = (unsigned)wk.n_pairs * EW * 4;
        const unsigned dst = (unsigned)__cvta_generic_to_shared(b ? buf1 : buf0);
        const unsigned bar = b ? bar1 : bar0;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
    };
    const int stride = gridDim.x * WPB;
    int w = blockIdx.x * WPB + warp;
    if (lane == 0 && w < n_work) issue(w, 0);   // work items and entries are static: before the wait
    pdl_wait();
    unsigned phase0 = 0, phase1 = 0;
    int drain = 0;   // after a time-out: 1 + the buffer whose copy timed out (+2 if the other is in flight)
    for (int k = 0; w < n_work; ++k, w += stride) {
        const int b = k & 1;
        if (lane == 0 && w + stride < n_work) issue(w + stride, b ^ 1);
        const VWork wk = work[w];
        const SceneDev& S = scenes[wk.scene];
        float* buf = b ? buf1 : buf0;
        const bool ok = mbar_wait(b ? bar1 : bar0, b ? phase1 : phase0, kSpinLimit);
        if (!__all_sync(full, ok)) {   // time-out (warp-uniform): leave the loop, handled below
            drain = 1 + b + (w + stride < n_work ? 2 : 0);
            break;
        }
        if (b) phase1 ^= 1; else phase0 ^= 1;
        const float* en = buf + lane * EW;
        const unsigned upto = wk.heads & ((2u << lane) - 1u);
        const int head = 31 - __clz(upto);
        const unsigned above = wk.heads & ~((2u << lane) - 1u);
        const int seg_end = above ? __ffs(above) - 1 : wk.n_pairs;
        int vid = 0;
        bool active = false;
        if (lane < wk.n_pairs) {
            vid = entry_node(en, entry_r<NE>(en));
            active = mode == 2 || S.mask[vid] != 0;
        }
        float acc[9], cmp[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) { acc[q] = 0.f; cmp[q] = 0.f; }
        const bool mixed = S.precision != 0;
        if (active) {
            entry_terms<E, MAT>(S, en, s_dN, mixed, acc, cmp);
            if (mixed) {
#pragma unroll
                for (int q = 0; q < 3; ++q) acc[q] -= cmp[q];
            }
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const float o = __shfl_down_sync(full, acc[q], off);
                if (lane + off < seg_end) acc[q] += o;
            }
        }
        if (active && lane == head) vertex_epilogue(S, vid, acc, mode, P, red);
        __syncwarp();   // buffer b is refilled by the next-but-one issue
    }
    if (drain) {
        // record the time-out (the warp's remaining items are not solved; the host reports
        // OCT_ETIMEDOUT), then give the timed-out copy, and the one issued into the other
        // buffer, a second bounded wait, so neither lands in shared memory after this warp
        // has stopped tracking it
        if (lane == 0) { atomicOr(P.error, 1); atomicOr(scenes[work[w].scene].status, kStatusTimeout); }
        const int b = (drain - 1) & 1;
        mbar_wait(b ? bar1 : bar0, b ? phase1 : phase0, kSpinLimit);
        if (drain > 2) mbar_wait(b ? bar0 : bar1, b ? phase0 : phase1, kSpinLimit);
        __syncwarp();
    }
    pdl_trigger();   // after the sweep: the next launch overlaps this kernel's tail only
}

template <int E> constexpr int packed_smem_bytes() { return (kBlock / 32) * 2 * 32 * EntryLayout<ElemT<E>::NE>::kWords * 4; }

// ------------------------------------------------------------------------ colour kernel
// mode 0: VBD solve; mode 1: VBD residual (r into u_new, |r| reductions); mode 2: explicit force.
// Resident blocks per SM the lane-group kernel is compiled for: P2 and Q1 are held to 128
// registers (4 blocks, 16 warps per SM; ptxas spills a few bytes), P1 to 80.
#ifndef OCTB_P2_MIN_BLOCKS
#define OCTB_P2_MIN_BLOCKS 4
#endif
#ifndef OCTB_Q1_MIN_BLOCKS
#define OCTB_Q1_MIN_BLOCKS 4
#endif
#ifndef OCTB_P1_MIN_BLOCKS
#define OCTB_P1_MIN_BLOCKS 6
#endif
template <int E> struct LaneMinBlocks {
    static constexpr int value = E == 3 ? OCTB_P1_MIN_BLOCKS : (E == 6 ? OCTB_Q1_MIN_BLOCKS : (E == 7 ? OCTB_P2_MIN_BLOCKS : 1));
};

template <int E, int MAT>
__global__ void __launch_bounds__(kBlock, LaneMinBlocks<E>::value) k_vertex(const SceneDev* __restrict__ scenes, const VWork* __restrict__ work,
                                                   int n_work, int tpv, int mode, StepParams P, double* red) {
    constexpr int NE = ElemT<E>::NE, NQ = ElemT<E>::NQ;
    __shared__ __align__(128) float s_dN[((NQ * NE * 3 + 3) / 4) * 4];
    __shared__ __align__(8) unsigned long long s_mbar;
    stage_table(s_dN, gdN<E>(), NQ * NE * 3, &s_mbar, P.error);
    pdl_wait();

    const int lane = threadIdx.x & 31;
    for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
        const VWork wk = work[w];
        const int t = wk.tpv ? wk.tpv : tpv;    // lanes per vertex of this item (block-uniform)
        const int glane = lane & (t - 1);        // lane within the vertex group
        const int group = threadIdx.x / t;       // vertex index within the block
        const SceneDev& S = scenes[wk.scene];
        const bool valid = group < wk.count;
        const int slot = wk.slot_begin + group;
        int vid = 0;
        bool active = false;
        if (valid) {
            vid = __ldg(S.vids + slot);
            active = mode == 2 || S.mask[vid] != 0;
        }
        float acc[9], cmp[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) { acc[k] = 0.f; cmp[k] = 0.f; }
        const bool mixed = S.precision != 0;
        if (active) {
            const int ob = __ldg(S.own_off + slot), oe = __ldg(S.own_off + slot + 1);
            if (S.ent) {
                // owner entries (contiguous per vertex): load the next one while this one computes
                constexpr int EW = EntryLayout<NE>::kWords;
                const float4* base = S.ent;
                const unsigned long long stream = policy_stream();
                int o = ob + glane;
                float4 nxt[EW / 4];
                if (o < oe) {
#pragma unroll
                    for (int j = 0; j < EW / 4; ++j) nxt[j] = ld_hint(base + (size_t)o * (EW / 4) + j, stream);
                }
                while (o < oe) {
                    float4 cur[EW / 4];
#pragma unroll
                    for (int j = 0; j < EW / 4; ++j) cur[j] = nxt[j];
                    const int on = o + t;
                    if (on < oe) {
#pragma unroll
                        for (int j = 0; j < EW / 4; ++j) nxt[j] = ld_hint(base + (size_t)on * (EW / 4) + j, stream);
                    }
                    entry_terms<E, MAT>(S, reinterpret_cast<const float*>(cur), s_dN, mixed, acc, cmp);
                    o = on;
                }
            } else {
                for (int o = ob + glane; o < oe; o += t) owner_terms<E, MAT>(S, __ldg(S.owners + o), s_dN, mixed, acc, cmp);
            }
            if (mixed) {
#pragma unroll
                for (int k = 0; k < 3; ++k) acc[k] -= cmp[k];
            }
        }
        for (int off = t >> 1; off > 0; off >>= 1) {
#pragma unroll
            for (int k = 0; k < 9; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], off);
        }
        if (active && glane == 0) vertex_epilogue(S, vid, acc, mode, P, red);
    }
    pdl_trigger();   // after the sweep: the next launch overlaps this kernel's tail only
}

// ------------------------------------------------------------------------ node kernels
constexpr int kNodeChunk = 256;

// Sub-step predictor.  kind 0: VBD (kernel_integration, GPU_VBD.cu:6-18) with the
// Chebyshev history seed; kind 1: semi-implicit Euler (kenerl_semi_exicit_integration,
// GPU_Integrator.cu:27-34), force taken from u_new for the explicit solver when use_force.
__global__ void k_predict(const SceneDev* __restrict__ scenes, const NWork* __restrict__ work, int n_work, int kind,
                          int use_force, int chebyshev, StepParams P) {
    (void)n_work;
    pdl_trigger();
    pdl_wait();
    const NWork wk = work[blockIdx.x];
    if (threadIdx.x >= wk.count) return;
    const SceneDev& S = scenes[wk.scene];
    const int i = wk.begin + threadIdx.x;
    const float dt = P.dt;
    float4 u = S.u[i], ul = S.u_last[i];
    if (kind == 0) {
        if (P.pending_v0 && P.pending_v0[wk.scene]) {   // initial velocity as the implicit velocity (u - u_last)/dt
            const float4 v = S.v[i];
            ul = make_float4(u.x - v.x * dt, u.y - v.y * dt, u.z - v.z * dt, ul.w);
        }
        if (chebyshev) S.prev1[i] = u;
        float4 y = S.y[i];
        y.x = u.x + ((u.x - ul.x) * P.inv_dt + S.gx * dt) * dt;
        y.y = u.y + ((u.y - ul.y) * P.inv_dt + S.gy * dt) * dt;
        y.z = u.z + ((u.z - ul.z) * P.inv_dt + S.gz * dt) * dt;
        S.y[i] = y;
        S.u_last[i] = u;
        S.u[i] = make_float4(y.x, y.y, y.z, u.w);
    } else {
        float4 v = S.v[i];
        const float w = 1.f / S.y[i].w;
        float fx = 0.f, fy = 0.f, fz = 0.f;
        if (use_force) { const float4 f = S.u_new[i]; fx = f.x; fy = f.y; fz = f.z; }
        S.u_last[i] = u;
        v.x += (S.gx + fx * w) * dt; v.y += (S.gy + fy * w) * dt; v.z += (S.gz + fz * w) * dt;
        u.x += v.x * dt; u.y += v.y * dt; u.z += v.z * dt;
        S.v[i] = v;
        S.u[i] = u;
        if (!isfinite(u.x + u.y + u.z + v.x + v.y + v.z)) atomicOr(S.status, kStatusNonFinite);
    }
}

// kernel_velocity_update (GPU_VBD.cu:20-25); with global damping for XPBD (GPU_PBD.cu:8-18).
__global__ void k_velocity(const SceneDev* __restrict__ scenes, const NWork* __restrict__ work, int n_work, int pbd,
                           StepParams P) {
    pdl_trigger();
    pdl_wait();
    const NWork wk = work[blockIdx.x];
    if (threadIdx.x >= wk.count) return;
    const SceneDev& S = scenes[wk.scene];
    const int i = wk.begin + threadIdx.x;
    const float4 u = S.u[i], ul = S.u_last[i];
    float4 v = make_float4((u.x - ul.x) / P.dt, (u.y - ul.y) / P.dt, (u.z - ul.z) / P.dt, 0.f);
    if (pbd) {
        const float nv = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
        if (nv > 1e-7f) {
            const float coef = S.global_damping * P.dt / S.y[i].w;
            const float d = -nv * (coef > 1.f ? 1.f : coef);
            v.x += v.x / nv * d; v.y += v.y / nv * d; v.z += v.z / nv * d;
        }
    }
    S.v[i] = v;
    // end of the sub-step: one check per node flags a scene whose state blew up
    if (!isfinite(u.x + u.y + u.z + v.x + v.y + v.z)) atomicOr(S.status, kStatusNonFinite);
}

// Chebyshev semi-iterative acceleration (kernel_chebychev_acceleration, GPU_VBD.cu:27-36).
__global__ void k_chebyshev(const SceneDev* __restrict__ scenes, const NWork* __restrict__ work, int n_work, StepParams P) {
    pdl_trigger();
    pdl_wait();
    const NWork wk = work[blockIdx.x];
    if (threadIdx.x >= wk.count) return;
    const SceneDev& S = scenes[wk.scene];
    const int i = wk.begin + threadIdx.x;
    float4 u = S.u[i];
    const float4 p2 = S.prev2[i];
    if (P.iteration >= 2) {
        u.x = p2.x + P.omega * (u.x - p2.x); u.y = p2.y + P.omega * (u.y - p2.y); u.z = p2.z + P.omega * (u.z - p2.z);
        S.u[i] = u;
    }
    S.prev2[i] = S.prev1[i];
    S.prev1[i] = u;
}

// Fixed nodes (kernel_constraint_fix, GPU_Constraint.cu:8-20) then, if enabled, the box
// clamp of free nodes (kernel_constraint_box_limit, :80-92).  One block per scene chunk.
// Fixation of node id to rigid group g (kernel_fix_constraint, GPU_Constraint.cu:8-20):
// position com + offset + R (X - com), velocity 0, mask 0.
__device__ __forceinline__ void fix_node(const SceneDev& S, int id, int g) {
    const float* G = S.fix + 16 * g;   // com, offset, rotation
    const float4 X = S.X[id];
    const float dx = X.x - G[0], dy = X.y - G[1], dz = X.z - G[2];
    const float* R = G + 6;
    const float rx = R[0] * dx + R[3] * dy + R[6] * dz;
    const float ry = R[1] * dx + R[4] * dy + R[7] * dz;
    const float rz = R[2] * dx + R[5] * dy + R[8] * dz;
    const float tx = (G[3] + G[0]) + rx, ty = (G[4] + G[1]) + ry, tz = (G[5] + G[2]) + rz;
    S.u[id] = make_float4(tx - X.x, ty - X.y, tz - X.z, 0.f);
    S.v[id] = make_float4(0.f, 0.f, 0.f, 0.f);
    S.mask[id] = 0;
}

__global__ void k_constraints(const SceneDev* __restrict__ scenes, const NWork* __restrict__ work, int n_work, int box_pass) {
    pdl_trigger();
    pdl_wait();
    const NWork wk = work[blockIdx.x];
    if (threadIdx.x >= wk.count) return;
    const SceneDev& S = scenes[wk.scene];
    const int k = wk.begin + threadIdx.x;
    if (!box_pass) {
        fix_node(S, S.fixed[k], S.fixed_group[k]);
    } else {
        if (S.mask[k] == 0) return;
        const float4 X = S.X[k];
        float4 u = S.u[k];
        const float px = fminf(fmaxf(X.x + u.x, S.bminx), S.bmaxx);
        const float py = fminf(fmaxf(X.y + u.y, S.bminy), S.bmaxy);
        const float pz = fminf(fmaxf(X.z + u.z, S.bminz), S.bmaxz);
        u.x = px - X.x; u.y = py - X.y; u.z = pz - X.z;
        S.u[k] = u;
    }
}

// Scripted effects (GPU_Constraint.cu:22-92), run after the fixation in creation order.
//   crush (kernel_constraint_crush): free nodes flattened to y = 0, last position = position,
//     velocity 0
//   random sphere (kernel_constraint_random_sphere): free nodes scattered inside a sphere by
//     the sine hash fract(sin(v) * k) of the reference, last position = position, velocity 0
//   high stretch (kernel_constraint_high_stretch): t = min(t + dt, max_dist), then each chosen
//     free node is pushed to X + normalize(X - c) t
__device__ __forceinline__ float hash1(float v) { const float x = sinf(v * 91.3458f) * 47453.5453f; return x - floorf(x); }
__device__ __forceinline__ float hash2(float a, float b) {
    const float x = sinf(a * 12.9898f + b * 78.233f) * 43758.5453f;
    return x - floorf(x);
}

__global__ void k_effect_nodes(const SceneDev* __restrict__ scene, const NWork* __restrict__ work, int slot) {
    const NWork wk = work[blockIdx.x];
    if (threadIdx.x >= wk.count) return;
    const SceneDev& S = *scene;
    const EffectDev& E = S.effects[slot];
    if (!E.active) return;
    const int i = wk.begin + threadIdx.x;
    if (S.mask[i] == 0) return;
    const float4 X = S.X[i];
    float px, py, pz;
    if (E.kind == 0) {
        const float4 u = S.u[i];
        px = X.x + u.x; py = 0.f; pz = X.z + u.z;
    } else {
        const float h = hash1(X.z);   // vec3_to_scalar_random(init_p)
        const float rx = hash2(X.x + h, X.y + h) * 2.f - 1.f;
        const float ry = hash1(rx * (float)i) * 2.f - 1.f;
        const float rz = hash1(rx * ry) * 2.f - 1.f;
        const float r = hash1(rz * rx * ry);
        const float inv = 1.f / sqrtf(rx * rx + ry * ry + rz * rz);
        px = E.cx + rx * inv * E.radius * r; py = E.cy + ry * inv * E.radius * r; pz = E.cz + rz * inv * E.radius * r;
    }
    const float4 u = make_float4(px - X.x, py - X.y, pz - X.z, 0.f);
    S.u[i] = u;
    S.u_last[i] = u;
    S.v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void k_effect_stretch(const SceneDev* __restrict__ scene, int slot, float dt) {
    const SceneDev& S = *scene;
    const EffectDev& E = S.effects[slot];
    if (!E.active) return;
    __shared__ float t;
    if (threadIdx.x == 0) {
        t = fminf(*E.t + dt, E.max_dist);
        *E.t = t;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < E.n; k += blockDim.x) {
        const int id = E.ids[k];
        if (S.mask[id] == 0) continue;
        const float4 X = S.X[id];
        const float dx = X.x - E.cx, dy = X.y - E.cy, dz = X.z - E.cz;
        const float inv = 1.f / sqrtf(dx * dx + dy * dy + dz * dz);
        const float4 u = S.u[id];
        S.u[id] = make_float4(dx * inv * t, dy * inv * t, dz * inv * t, u.w);
    }
}

// Multigrid VBD (MG_VBD_FEM, MG_VertexBlockDescent.cpp): the linear level is a scene of the
// corner nodes.  gather copies the corners' displacement, start-of-sub-step displacement,
// inertial target (its own masses kept) and mask into it; scatter copies the solved corners
// back; prolong moves each mid node by the mean displacement since the sub-step start of its
// k corners (P1_to_P2 / Q1_to_Q2::prolongation, :37-96).  list: per entry the mid node then
// its k corners.
__global__ void k_mg_copy(const SceneDev* __restrict__ main, const SceneDev* __restrict__ sub, const int* __restrict__ map,
                          int n, int dir) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int m = map[k];
    if (dir == 0) {
        sub->u[k] = main->u[m];
        sub->u_last[k] = main->u_last[m];
        const float4 y = main->y[m];
        const float w = sub->y[k].w;
        sub->y[k] = make_float4(y.x, y.y, y.z, w);
        sub->mask[k] = main->mask[m];
    } else {
        main->u[m] = sub->u[k];
    }
}

__global__ void k_mg_prolong(const SceneDev* __restrict__ main, const int* __restrict__ list, int count, int k, float w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int* e = list + (size_t)i * (k + 1);
    float dx = 0.f, dy = 0.f, dz = 0.f;
    for (int j = 1; j <= k; ++j) {
        const float4 u = main->u[e[j]], ul = main->u_last[e[j]];
        dx += u.x - ul.x; dy += u.y - ul.y; dz += u.z - ul.z;
    }
    const float4 ul = main->u_last[e[0]];
    main->u[e[0]] = make_float4(ul.x + dx * w, ul.y + dy * w, ul.z + dz * w, ul.w);
}

// Failure-detection probe: one thread waits, through the same bounded mbarrier wait as the
// colour kernels, on a phase that no copy and no thread will ever complete; when the limit
// runs out it records the time-out in the context's error word (bit 0) and returns.
__global__ void k_nodes_out(const float4* __restrict__ src, const float4* __restrict__ X, float* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = src[i];
    if (X) {
        const float4 x = X[i];
        a.x = x.x + a.x; a.y = x.y + a.y; a.z = x.z + a.z;
    }
    out[3 * i] = a.x; out[3 * i + 1] = a.y; out[3 * i + 2] = a.z;
}

__global__ void k_nodes_in(const float* __restrict__ in, const float4* __restrict__ X, float4* __restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a = in[3 * i], b = in[3 * i + 1], c = in[3 * i + 2];
    if (X) {
        const float4 x = X[i];
        a = a - x.x; b = b - x.y; c = c - x.z;
    }
    dst[i] = make_float4(a, b, c, 0.f);
}

__global__ void k_wait_probe(int* error, long limit) {
    __shared__ __align__(8) unsigned long long bar;
    const unsigned mb = (unsigned)__cvta_generic_to_shared(&bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (!mbar_wait(mb, 0, limit)) atomicOr(error, 1);
}

// Host-state staging of a batch: state[off_s + 3 i ...] = u_i then v_i (n*3 floats each).
// dir 0: staging -> node arrays, dir 1: node arrays -> staging.
__global__ void k_state(const SceneDev* __restrict__ scenes, const NWork* __restrict__ work, const long long* __restrict__ soff,
                        float* __restrict__ state, int dir) {
    const NWork wk = work[blockIdx.x];
    if (threadIdx.x >= wk.count) return;
    const SceneDev& S = scenes[wk.scene];
    const int i = wk.begin + threadIdx.x;
    float* p = state + soff[wk.scene] + 3ll * i;
    float* v = state + soff[wk.scene] + 3ll * S.n_nodes + 3ll * i;
    if (dir == 0) {
        float4 u = S.u[i];
        u.x = p[0]; u.y = p[1]; u.z = p[2];
        S.u[i] = u;
        S.v[i] = make_float4(v[0], v[1], v[2], 0.f);
    } else {
        const float4 u = S.u[i], w = S.v[i];
        p[0] = u.x; p[1] = u.y; p[2] = u.z;
        v[0] = w.x; v[1] = w.y; v[2] = w.z;
    }
}

void launch_state(const SceneDev* scenes, const NWork* work, int n_work, const long long* soff, float* state, int dir,
                  cudaStream_t st) {
    if (n_work <= 0) return;
    k_state<<<n_work, kNodeChunk, 0, st>>>(scenes, work, soff, state, dir);
}

// Jacobi commit of a colour (kernel_copy_in_position, GPU_VBD_FEM.cu:402-413).
__global__ void k_commit(const SceneDev* __restrict__ scenes, const VWork* __restrict__ work, int n_work) {
    pdl_trigger();
    pdl_wait();
    for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
        const VWork wk = work[w];
        const SceneDev& S = scenes[wk.scene];
        for (int k = threadIdx.x; k < wk.count; k += blockDim.x) {
            const int vid = S.vids[wk.slot_begin + k];
            if (S.mask[vid] != 0) S.u[vid] = S.u_new[vid];
        }
    }
}

// ------------------------------------------------------------------------ XPBD
// Coloured element projection of GPU_PBD_FEM::step (GPU_PBD_FEM.cu:640-717).  Elements of one
// colour share no node, so each is projected in place.  Per element two constraints run in
// sequence (m = 0 volumetric with stiffness lambda, m = 1 deviatoric with mu), from the
// eval_material pairs (GPU_PBD_FEM_Materials.cu:97-117).  Two update forms:
//   normalised (kernel_XPBD_V0, :13-93; every Tetra4 and XPBD_FEM_VERSION::XPBD):
//     C' = sqrt|C|, grad' = grad / 2C', dl = -C' / (sum w |grad'|^2 + 1/(k dt^2)),
//     fixed (mask 0) nodes are not moved;
//   raw (kernel_XPBD_V1/V2, :141-263; Quadrature and OptiShared on other elements):
//     alpha = 4C/(k dt^2), beta = C < 1e-12 ? 0 : -2C / (sum w |grad|^2 + alpha), every node
//     moves (the fixation resets fixed nodes after the sweep).
// Mapping: a group of G lanes of one warp per element.  Lane i gathers node i (registers and
// shared memory); lane q evaluates quadrature point q (F, the material pair, P~ = P JX_inv^T V
// into shared memory); lane i then forms grad_i = sum_q P~_q dN_qi.  The sums over q (C) and
// over nodes (sum w |grad|^2) are butterfly shuffles inside the group.  The reference-element
// table dN is staged into shared memory by one TMA bulk copy per block.

// Rotation R of F = R S by the quaternion iteration of Mueller et al., "A Robust Method to
// Extract the Rotational Part of Deformations" (MIG 2016), run as mat3x3_polardecomposition
// (CUMatrix.cu:75-96) runs it: R from the identity, at most 10 iterations, stop when
// |omega| < 1e-8, omega = sum_i R_i x F_i * (1/|sum_i R_i . F_i| + 1e-9).  Columns in and out.
__device__ __forceinline__ void polar_rotation(V3 F0, V3 F1, V3 F2, V3& R0, V3& R1, V3& R2) {
    float qw = 1.f, qx = 0.f, qy = 0.f, qz = 0.f;
    R0 = mk(1.f, 0.f, 0.f); R1 = mk(0.f, 1.f, 0.f); R2 = mk(0.f, 0.f, 1.f);
    for (int it = 0; it < 10; ++it) {
        const float den = 1.f / fabsf(dot(R0, F0) + dot(R1, F1) + dot(R2, F2)) + 1e-9f;
        const V3 cs = cross(R0, F0) + cross(R1, F1) + cross(R2, F2);
        const V3 om = cs * den;
        const float w = sqrtf(dot(om, om));
        if (w < 1e-8f) break;
        const V3 a = mk(om.x / w, om.y / w, om.z / w);
        float sn, c;
        sincosf(0.5f * w, &sn, &c);
        const float dx = a.x * sn, dy = a.y * sn, dz = a.z * sn;
        const float nw = c * qw - dx * qx - dy * qy - dz * qz;
        const float nx = c * qx + dx * qw + dy * qz - dz * qy;
        const float ny = c * qy - dx * qz + dy * qw + dz * qx;
        const float nz = c * qz + dx * qy - dy * qx + dz * qw;
        const float inv = 1.f / sqrtf(nw * nw + nx * nx + ny * ny + nz * nz);
        qw = nw * inv; qx = nx * inv; qy = ny * inv; qz = nz * inv;
        R0 = mk(1.f - 2.f * (qy * qy + qz * qz), 2.f * (qx * qy + qw * qz), 2.f * (qx * qz - qw * qy));
        R1 = mk(2.f * (qx * qy - qw * qz), 1.f - 2.f * (qx * qx + qz * qz), 2.f * (qy * qz + qw * qx));
        R2 = mk(2.f * (qx * qz + qw * qy), 2.f * (qy * qz - qw * qx), 1.f - 2.f * (qx * qx + qy * qy));
    }
}

template <int MAT>
__device__ __forceinline__ void xpbd_pair(int m, V3 F0, V3 F1, V3 F2, float lam, float mu, V3& P0, V3& P1, V3& P2, float& C) {
    if (MAT == 4 || MAT == 5) {
        // GPU_PBD_FEM_Materials.cu:67-95, with F = R S from the polar iteration
        V3 R0, R1, R2;
        polar_rotation(F0, F1, F2, R0, R1, R2);
        const V3 S0 = mk(dot(R0, F0), dot(R1, F0), dot(R2, F0)), S1 = mk(dot(R0, F1), dot(R1, F1), dot(R2, F1)),
                 S2 = mk(dot(R0, F2), dot(R1, F2), dot(R2, F2));
        const V3 RS0 = R0 * S0.x + R1 * S0.y + R2 * S0.z, RS1 = R0 * S1.x + R1 * S1.y + R2 * S1.z,
                 RS2 = R0 * S2.x + R1 * S2.y + R2 * S2.z;   // R S = columns of R S
        if (MAT == 4 && m == 0) {   // C = tr((S - I)^2), P = 2 tr(S - I) R
            const float a = S0.x - 1.f, b = S1.y - 1.f, c = S2.z - 1.f;
            C = a * a + b * b + c * c + (S0.y * S1.x + S1.z * S2.y + S2.x * S0.z) * 2.f;
            const float t = 2.f * (a + b + c);
            P0 = R0 * t; P1 = R1 * t; P2 = R2 * t;
        } else if (MAT == 4) {      // C = |S|^2, P = R (2 S - I)
            C = dot(S0, S0) + dot(S1, S1) + dot(S2, S2);
            P0 = RS0 * 2.f - R0; P1 = RS1 * 2.f - R1; P2 = RS2 * 2.f - R2;
        } else if (m == 0) {        // C = (det S - 1)^2, P = 2 (det S - 1) R cof(S)
            const V3 K0 = cross(S1, S2), K1 = cross(S2, S0), K2 = cross(S0, S1);
            const float d = dot(S0, K0) - 1.f;
            C = d * d;
            P0 = (R0 * K0.x + R1 * K0.y + R2 * K0.z) * (2.f * d);
            P1 = (R0 * K1.x + R1 * K1.y + R2 * K1.z) * (2.f * d);
            P2 = (R0 * K2.x + R1 * K2.y + R2 * K2.z) * (2.f * d);
        } else {                    // C = 2 |S|^2, P = 4 R (S - I)
            C = 2.f * (dot(S0, S0) + dot(S1, S1) + dot(S2, S2));
            P0 = (RS0 - R0) * 4.f; P1 = (RS1 - R1) * 4.f; P2 = (RS2 - R2) * 4.f;
        }
    } else if (MAT == 2 || MAT == 3) {
        const V3 C0 = cross(F1, F2), C1 = cross(F2, F0), C2 = cross(F0, F1);
        const float J = dot(F0, C0);
        if (m == 0) {
            const float alpha = MAT == 2 ? 1.f + mu / lam : 1.f;
            const float d = J - alpha;
            C = d * d;
            P0 = C0 * (2.f * d); P1 = C1 * (2.f * d); P2 = C2 * (2.f * d);
        } else if (MAT == 2) {
            C = dot(F0, F0) + dot(F1, F1) + dot(F2, F2) - 3.f;
            P0 = F0 * 2.f; P1 = F1 * 2.f; P2 = F2 * 2.f;
        } else {
            C = dot(F0, F0) + dot(F1, F1) + dot(F2, F2) - 3.f - 2.f * (J - 1.f);
            P0 = F0 * 2.f - C0 * 2.f; P1 = F1 * 2.f - C1 * 2.f; P2 = F2 * 2.f - C2 * 2.f;
        }
    } else if (MAT == 0) {
        // E = (F + F^T)/2 - I
        const float e00 = F0.x - 1.f, e11 = F1.y - 1.f, e22 = F2.z - 1.f;
        const float e01 = 0.5f * (F1.x + F0.y), e02 = 0.5f * (F2.x + F0.z), e12 = 0.5f * (F2.y + F1.z);
        if (m == 0) {
            const float tr = e00 + e11 + e22;
            C = tr * tr;
            P0 = mk(2.f * tr, 0, 0); P1 = mk(0, 2.f * tr, 0); P2 = mk(0, 0, 2.f * tr);
        } else {
            C = 2.f * (e00 * e00 + e11 * e11 + e22 * e22 + 2.f * (e01 * e01 + e02 * e02 + e12 * e12));
            P0 = mk(4.f * e00, 4.f * e01, 4.f * e02); P1 = mk(4.f * e01, 4.f * e11, 4.f * e12); P2 = mk(4.f * e02, 4.f * e12, 4.f * e22);
        }
    } else {
        const float f00 = dot(F0, F0), f01 = dot(F0, F1), f02 = dot(F0, F2), f11 = dot(F1, F1), f12 = dot(F1, F2), f22 = dot(F2, F2);
        const float e00 = 0.5f * (f00 - 1.f), e11 = 0.5f * (f11 - 1.f), e22 = 0.5f * (f22 - 1.f);
        const float e01 = 0.5f * f01, e02 = 0.5f * f02, e12 = 0.5f * f12;
        if (m == 0) {
            const float tr = e00 + e11 + e22;
            C = tr * tr;
            P0 = F0 * (2.f * tr); P1 = F1 * (2.f * tr); P2 = F2 * (2.f * tr);
        } else {
            C = 2.f * (e00 * e00 + e11 * e11 + e22 * e22 + 2.f * (e01 * e01 + e02 * e02 + e12 * e12));
            // P = 4 F E : column b = 4 sum_k F_k E_kb
            P0 = (F0 * e00 + F1 * e01 + F2 * e02) * 4.f;
            P1 = (F0 * e01 + F1 * e11 + F2 * e12) * 4.f;
            P2 = (F0 * e02 + F1 * e12 + F2 * e22) * 4.f;
        }
    }
}

// lanes per element: at least one per quadrature point
template <int E> struct XpbdLanes { static constexpr int G = E == 3 ? 4 : (E == 6 || E == 7 ? 8 : (E == 8 ? 16 : 32)); };

template <int G> __device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// MINB: resident blocks per SM the kernel is compiled for.  1 (96 registers for P2, 5 blocks)
// serves launches of under a wave (one scene's colour: per-element latency decides); 8 (64
// registers) serves batched launches of several waves, whose time is set by how many elements
// are in flight: the 256-scene XPBD frame 17.05 -> 15.65 ms, against a single P2 scene's frame
// 0.889 -> 0.989 ms with 6 blocks.
template <int E, int MAT, bool RAW, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_xpbd(const SceneDev* __restrict__ scenes, const XWork* __restrict__ work,
                                                 StepParams P) {
    constexpr int NE = ElemT<E>::NE, NQ = ElemT<E>::NQ, G = XpbdLanes<E>::G, GPB = kBlock / G;
    constexpr int NI = (NE + G - 1) / G;   // nodes per lane
    static_assert(NQ <= G, "one quadrature point per lane");
    __shared__ __align__(16) float s_dN[((NQ * NE * 3 + 3) / 4) * 4];
    __shared__ __align__(16) float4 s_pos[GPB][NE];
    __shared__ __align__(16) float4 s_P[GPB][NQ][3];
    __shared__ unsigned long long s_mbar;
    pdl_trigger();
    stage_table(s_dN, gdN<E>(), NQ * NE * 3, &s_mbar, P.error);
    pdl_wait();

    const int lane = threadIdx.x % G, grp = threadIdx.x / G;
    const XWork wk = work[blockIdx.x];   // GPB elements of one scene's colour
    const bool active = grp < wk.count;   // no early exit: every lane takes part in the shuffles
    const SceneDev& S = scenes[wk.scene];
    const int eid = active ? S.elems[wk.begin + grp] : 0;   // for the quadrature records only
    const int* tp = S.etopo + (size_t)(active ? wk.begin + grp : 0) * NE;
    int vid[NI];
    float4 u[NI];
    float w[NI];
    bool mv[NI];
#pragma unroll
    for (int k = 0; k < NI; ++k) {
        const int i = lane + k * G;
        vid[k] = -1; u[k] = make_float4(0.f, 0.f, 0.f, 0.f); w[k] = 0.f; mv[k] = false;
        if (active && i < NE) {
            vid[k] = tp[i];
            u[k] = S.u[vid[k]];
            w[k] = 1.f / S.y[vid[k]].w;
            mv[k] = RAW || S.mask[vid[k]] != 0;
        }
    }
    // quadrature record of lane q: JX_inv (columns m0 m1 m2), V, lambda, mu
    const int q = lane;
    const bool hasq = active && q < NQ;
    const float4* rec = S.eq + (size_t)eid * S.eq_stride * 3;
    const int qs = S.eq_stride == 1 ? 0 : 1;
    V3 m0 = mk(0, 0, 0), m1 = m0, m2 = m0;
    float V = 0.f;
    if (hasq) {
        const float4 A = rec[3 * q * qs], B = rec[3 * q * qs + 1], Cr = rec[3 * q * qs + 2];
        m0 = mk(A.x, A.y, A.z); m1 = mk(A.w, B.x, B.y); m2 = mk(B.z, B.w, Cr.x);
        V = Cr.y * wq<E>(q);
    }
    const float4 L = active ? rec[2] : make_float4(0.f, 0.f, 1.f, 1.f);
    const float lam = L.z, mu = L.w;
    const float dt2 = P.dt * P.dt;

    for (int m = 0; m < 2; ++m) {
#pragma unroll
        for (int k = 0; k < NI; ++k)
            if (lane + k * G < NE) s_pos[grp][lane + k * G] = u[k];
        __syncwarp();
        float Cq = 0.f;
        if (hasq) {
            V3 J0 = mk(0, 0, 0), J1 = J0, J2 = J0;
#pragma unroll
            for (int i = 0; i < NE; ++i) {
                const float4 p = s_pos[grp][i];
                const float* d = &s_dN[(q * NE + i) * 3];
                const V3 pu = mk(p.x, p.y, p.z);
                J0 = J0 + pu * d[0]; J1 = J1 + pu * d[1]; J2 = J2 + pu * d[2];
            }
            V3 F0 = J0 * m0.x + J1 * m0.y + J2 * m0.z, F1 = J0 * m1.x + J1 * m1.y + J2 * m1.z,
               F2 = J0 * m2.x + J1 * m2.y + J2 * m2.z;
            F0.x += 1.f; F1.y += 1.f; F2.z += 1.f;
            V3 P0, P1, P2;
            float en;
            xpbd_pair<MAT>(m, F0, F1, F2, lam, mu, P0, P1, P2, en);
            Cq = en * V;
            // P~ = P JX_inv^T V: column j = sum_k P_k (m_k)_j
            const V3 T0 = (P0 * m0.x + P1 * m1.x + P2 * m2.x) * V, T1 = (P0 * m0.y + P1 * m1.y + P2 * m2.y) * V,
                     T2 = (P0 * m0.z + P1 * m1.z + P2 * m2.z) * V;
            s_P[grp][q][0] = make_float4(T0.x, T0.y, T0.z, 0.f);
            s_P[grp][q][1] = make_float4(T1.x, T1.y, T1.z, 0.f);
            s_P[grp][q][2] = make_float4(T2.x, T2.y, T2.z, 0.f);
        }
        float C = group_sum<G>(Cq);
        __syncwarp();
        V3 g[NI];
        float ss = 0.f;
#pragma unroll
        for (int k = 0; k < NI; ++k) {
            const int i = lane + k * G;
            g[k] = mk(0, 0, 0);
            if (i < NE) {
#pragma unroll
                for (int qq = 0; qq < NQ; ++qq) {
                    const float* d = &s_dN[(qq * NE + i) * 3];
                    const float4 a = s_P[grp][qq][0], b = s_P[grp][qq][1], c = s_P[grp][qq][2];
                    g[k] = g[k] + mk(a.x, a.y, a.z) * d[0] + mk(b.x, b.y, b.z) * d[1] + mk(c.x, c.y, c.z) * d[2];
                }
            }
        }
        const float k_st = m == 0 ? lam : mu;
        float step;
        if (RAW) {
#pragma unroll
            for (int k = 0; k < NI; ++k) ss += dot(g[k], g[k]) * w[k];
            const float S2 = group_sum<G>(ss);
            const float alpha = 4.f * C / (k_st * dt2);
            step = C < 1e-12f ? 0.f : -2.f * C / (S2 + alpha);
        } else {
            C = sqrtf(C < 0.f ? -C : C);
            const float ci = C < 1e-12f ? 0.f : 1.f / (2.f * C);
#pragma unroll
            for (int k = 0; k < NI; ++k) { g[k] = g[k] * ci; ss += dot(g[k], g[k]) * w[k]; }
            const float S2 = group_sum<G>(ss);
            step = -C / (S2 + 1.f / (k_st * dt2));
        }
#pragma unroll
        for (int k = 0; k < NI; ++k)
            if (mv[k]) {
                const float f = step * w[k];
                u[k].x += f * g[k].x; u[k].y += f * g[k].y; u[k].z += f * g[k].z;
            }
        __syncwarp();   // every lane has read s_pos / s_P before the next constraint rewrites them
    }
#pragma unroll
    for (int k = 0; k < NI; ++k)
        if (vid[k] >= 0 && mv[k]) S.u[vid[k]] = u[k];
}

// ------------------------------------------------------------------------ diagnostics
// Per-element diagnostics of GPU_FEM (GPU_FEM.cu:20-107), one thread per element, in FP64 on
// the current absolute positions p = X + u (rounded to FP32 as the getters return them), with
// the rest Jacobian of each quadrature point recomputed from X: the exact value of the
// reference's formulas at those positions.
//   kind 0: sum_q von_mises(P F^T / det F) V_q, F = Jx_q JX_inv_q
//   kind 4: the same with Jx summed over the quadrature points, as kernel_compute_stress
//           (:20-43) accumulates it (equal to kind 0 for one-point elements)
//   kind 1: sum_q |det Jx_q| w_q                 (kernel_compute_volume)
//   kind 2: sum_q (|det Jx_q| w_q - V_q)         (kernel_compute_volume_diff)
//   kind 3: 1 if sum_q det(Jx_q JX_inv_q) w_q < -1e-6, else 0   (kernel_compute_inverted, with
//           the rest Jacobian of point q)
struct D3 { double x, y, z; };
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 dcross(D3 a, D3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
__device__ __forceinline__ double ddet(D3 a, D3 b, D3 c) { return ddot(a, dcross(b, c)); }
__device__ __forceinline__ double dget(D3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// PK1 of GPU_FEM_Material.cu:14-36 (columns); zero for the XPBD-only materials.
__device__ void pk1_d(int mat, D3 F0, D3 F1, D3 F2, double lam, double mu, D3& P0, D3& P1, D3& P2) {
    if (mat == 0) {   // hooke_stress: lambda tr(E) I + mu E, E = (F + F^T)/2 - I
        const double e00 = F0.x - 1.0, e11 = F1.y - 1.0, e22 = F2.z - 1.0;
        const double e01 = 0.5 * (F1.x + F0.y), e02 = 0.5 * (F2.x + F0.z), e12 = 0.5 * (F2.y + F1.z);
        const double t = lam * (e00 + e11 + e22);
        P0 = {t + mu * e00, mu * e01, mu * e02}; P1 = {mu * e01, t + mu * e11, mu * e12};
        P2 = {mu * e02, mu * e12, t + mu * e22};
    } else if (mat == 1) {   // stvk_stress: lambda tr(E) F + 2 mu F E, E = (F^T F - I)/2
        const double e00 = 0.5 * (ddot(F0, F0) - 1.0), e11 = 0.5 * (ddot(F1, F1) - 1.0), e22 = 0.5 * (ddot(F2, F2) - 1.0);
        const double e01 = 0.5 * ddot(F0, F1), e02 = 0.5 * ddot(F0, F2), e12 = 0.5 * ddot(F1, F2);
        const double t = lam * (e00 + e11 + e22);
        P0 = F0 * t + (F0 * e00 + F1 * e01 + F2 * e02) * (2.0 * mu);
        P1 = F1 * t + (F0 * e01 + F1 * e11 + F2 * e12) * (2.0 * mu);
        P2 = F2 * t + (F0 * e02 + F1 * e12 + F2 * e22) * (2.0 * mu);
    } else if (mat == 2 || mat == 3) {   // nh_stress / snh_stress: lambda (J - alpha) cof F + mu F
        const D3 C0 = dcross(F1, F2), C1 = dcross(F2, F0), C2 = dcross(F0, F1);
        const double sc = lam * (ddot(F0, C0) - (mat == 3 ? 1.0 + mu / lam : 1.0));
        P0 = C0 * sc + F0 * mu; P1 = C1 * sc + F1 * mu; P2 = C2 * sc + F2 * mu;
    } else {
        P0 = P1 = P2 = D3{0.0, 0.0, 0.0};
    }
}

// Inverse of the matrix with columns c0 c1 c2, as columns (adjugate / determinant).
__device__ __forceinline__ void dinv(D3 c0, D3 c1, D3 c2, D3& i0, D3& i1, D3& i2) {
    const D3 r0 = dcross(c1, c2), r1 = dcross(c2, c0), r2 = dcross(c0, c1);   // rows of the inverse x det
    const double id = 1.0 / ddot(c0, r0);
    i0 = D3{r0.x, r1.x, r2.x} * id; i1 = D3{r0.y, r1.y, r2.y} * id; i2 = D3{r0.z, r1.z, r2.z} * id;
}

// ------------------------------------------------------------------------ explicit force
// Element-centric force pass of the explicit integrator (the terms of kernel_fem_eval_force,
// octopus/src/GPU/Explicit/GPU_FEM_Explicit.cu:5-64: f_i = sum_q -V P g_iq, minus k_d (sum_q
// H_iq) v_i).  The explicit step has no colour order, so each element's deformation gradient
// is formed once per quadrature point instead of once per (node, point) as in the vertex
// kernel, and its nodes are gathered once instead of once per owner.  G lanes per element (as
// k_xpbd): lane i gathers node i, lane q forms F at point q into shared memory, then lane i
// evaluates its nodes' terms (material_terms, the arithmetic of the vertex kernel) at every
// point and writes its per-(element, local node) force to `contrib`; k_explicit_gather sums
// each node's owners in owner order.  Deterministic (no atomics).
// P~ = V P JX_inv^T (columns T0 T1 T2) of the first Piola-Kirchhoff stress of material_terms'
// materials, so that -V P g = -(T0 dN_0 + T1 dN_1 + T2 dN_2) for g = JX_inv^T dN.
template <int MAT>
__device__ __forceinline__ void pk1_tilde(V3 F0, V3 F1, V3 F2, float lam, float mu, float V, V3 m0, V3 m1, V3 m2,
                                          V3& T0, V3& T1, V3& T2) {
    V3 P0, P1, P2;   // columns of P
    if (MAT == 2 || MAT == 3) {   // P = mu F + s cof(F)
        const V3 C0 = cross(F1, F2), C1 = cross(F2, F0), C2 = cross(F0, F1);
        const float J = dot(F0, C0);
        const float sc = MAT == 3 ? lam * (J - 1.f) - mu : lam * (J - 1.f);
        P0 = F0 * mu + C0 * sc; P1 = F1 * mu + C1 * sc; P2 = F2 * mu + C2 * sc;
    } else if (MAT == 0) {        // P = lambda tr(E) I + mu E, E = (F + F^T)/2 - I
        const float trE = F0.x + F1.y + F2.z - 3.f;
        // E column c, row r: (F_rc + F_cr)/2 - d_rc, F_rc = row r of column c
        const V3 E0 = mk(F0.x - 1.f, 0.5f * (F0.y + F1.x), 0.5f * (F0.z + F2.x));
        const V3 E1 = mk(0.5f * (F1.x + F0.y), F1.y - 1.f, 0.5f * (F1.z + F2.y));
        const V3 E2 = mk(0.5f * (F2.x + F0.z), 0.5f * (F2.y + F1.z), F2.z - 1.f);
        const float lt = lam * trE;
        P0 = E0 * mu + mk(lt, 0.f, 0.f); P1 = E1 * mu + mk(0.f, lt, 0.f); P2 = E2 * mu + mk(0.f, 0.f, lt);
    } else {                      // StVK: P = lambda tr(E) F + 2 mu F E, E = (F^T F - I)/2
        const float f00 = dot(F0, F0), f01 = dot(F0, F1), f02 = dot(F0, F2);
        const float f11 = dot(F1, F1), f12 = dot(F1, F2), f22 = dot(F2, F2);
        const float trE = 0.5f * (f00 + f11 + f22 - 3.f);
        // column c of F E = sum_k F_k E_kc
        const V3 FE0 = F0 * (0.5f * (f00 - 1.f)) + F1 * (0.5f * f01) + F2 * (0.5f * f02);
        const V3 FE1 = F0 * (0.5f * f01) + F1 * (0.5f * (f11 - 1.f)) + F2 * (0.5f * f12);
        const V3 FE2 = F0 * (0.5f * f02) + F1 * (0.5f * f12) + F2 * (0.5f * (f22 - 1.f));
        const float lt = lam * trE, tm = 2.f * mu;
        P0 = F0 * lt + FE0 * tm; P1 = F1 * lt + FE1 * tm; P2 = F2 * lt + FE2 * tm;
    }
    // column j of P JX_inv^T = sum_k P_k (m_k)_j
    T0 = (P0 * m0.x + P1 * m1.x + P2 * m2.x) * V;
    T1 = (P0 * m0.y + P1 * m1.y + P2 * m2.y) * V;
    T2 = (P0 * m0.z + P1 * m1.z + P2 * m2.z) * V;
}

template <int E, int MAT>
__global__ void __launch_bounds__(kBlock) k_explicit_elem(const SceneDev* __restrict__ scenes, int n_elements,
                                                          float4* __restrict__ contrib, StepParams P) {
    constexpr int NE = ElemT<E>::NE, NQ = ElemT<E>::NQ, G = XpbdLanes<E>::G, GPB = kBlock / G;
    constexpr int NI = (NE + G - 1) / G;   // nodes per lane
    static_assert(NQ <= G, "one quadrature point per lane");
    __shared__ __align__(16) float s_dN[((NQ * NE * 3 + 3) / 4) * 4];
    __shared__ __align__(16) float4 s_u[GPB][NE];
    __shared__ __align__(16) float4 s_F[GPB][NQ][3];   // F columns at each point
    __shared__ __align__(16) float4 s_R[GPB][NQ][3];   // JX_inv columns, then (., V w_q, lambda, mu)
    __shared__ unsigned long long s_mbar;
    pdl_trigger();
    stage_table(s_dN, gdN<E>(), NQ * NE * 3, &s_mbar, P.error);
    pdl_wait();
    const SceneDev& S = scenes[0];
    const int lane = threadIdx.x % G, grp = threadIdx.x / G;
    const int eid = blockIdx.x * GPB + grp;
    const bool active = eid < n_elements;   // no early exit: the group synchronises with __syncwarp
    const int* tp = S.topo + (size_t)(active ? eid : 0) * NE;
#pragma unroll
    for (int k = 0; k < NI; ++k) {
        const int i = lane + k * G;
        if (active && i < NE) s_u[grp][i] = S.u[tp[i]];
    }
    __syncwarp();
    if (active && lane < NQ) {
        const int q = lane;
        const float4* rec = S.eq + ((size_t)eid * S.eq_stride + (S.eq_stride == 1 ? 0 : q)) * 3;
        const float4 A = rec[0], B = rec[1], C = rec[2];
        const V3 m0 = mk(A.x, A.y, A.z), m1 = mk(A.w, B.x, B.y), m2 = mk(B.z, B.w, C.x);
        V3 J0 = mk(0, 0, 0), J1 = J0, J2 = J0;
#pragma unroll
        for (int i = 0; i < NE; ++i) {
            const float4 uu = s_u[grp][i];
            const float* d = &s_dN[(q * NE + i) * 3];
            J0.x = fmaf(uu.x, d[0], J0.x); J0.y = fmaf(uu.y, d[0], J0.y); J0.z = fmaf(uu.z, d[0], J0.z);
            J1.x = fmaf(uu.x, d[1], J1.x); J1.y = fmaf(uu.y, d[1], J1.y); J1.z = fmaf(uu.z, d[1], J1.z);
            J2.x = fmaf(uu.x, d[2], J2.x); J2.y = fmaf(uu.y, d[2], J2.y); J2.z = fmaf(uu.z, d[2], J2.z);
        }
        V3 F0 = J0 * m0.x + J1 * m0.y + J2 * m0.z;
        V3 F1 = J0 * m1.x + J1 * m1.y + J2 * m1.z;
        V3 F2 = J0 * m2.x + J1 * m2.y + J2 * m2.z;
        F0.x += 1.f; F1.y += 1.f; F2.z += 1.f;
        if (S.damping == 0.f) {   // without damping only -V P g is needed: P~ once per point
            pk1_tilde<MAT>(F0, F1, F2, C.z, C.w, C.y * wq<E>(q), m0, m1, m2, F0, F1, F2);
        }
        s_F[grp][q][0] = make_float4(F0.x, F0.y, F0.z, 0.f);
        s_F[grp][q][1] = make_float4(F1.x, F1.y, F1.z, 0.f);
        s_F[grp][q][2] = make_float4(F2.x, F2.y, F2.z, 0.f);
        s_R[grp][q][0] = A;
        s_R[grp][q][1] = B;
        s_R[grp][q][2] = make_float4(C.x, C.y * wq<E>(q), C.z, C.w);
    }
    __syncwarp();
    const float kd = S.damping;
    if (kd == 0.f) {   // f_i = -sum_q P~_q dN_qi
#pragma unroll
        for (int k = 0; k < NI; ++k) {
            const int i = lane + k * G;
            if (!active || i >= NE) continue;
            float fx = 0.f, fy = 0.f, fz = 0.f;
#pragma unroll (NQ <= 11 ? NQ : 1)
            for (int q = 0; q < NQ; ++q) {
                const float4 t0 = s_F[grp][q][0], t1 = s_F[grp][q][1], t2 = s_F[grp][q][2];
                const float* dr = &s_dN[(q * NE + i) * 3];
                fx -= t0.x * dr[0] + t1.x * dr[1] + t2.x * dr[2];
                fy -= t0.y * dr[0] + t1.y * dr[1] + t2.y * dr[2];
                fz -= t0.z * dr[0] + t1.z * dr[1] + t2.z * dr[2];
            }
            contrib[(size_t)eid * NE + i] = make_float4(fx, fy, fz, 0.f);
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < NI; ++k) {
        const int i = lane + k * G;
        if (!active || i >= NE) continue;
        float acc[9];
#pragma unroll
        for (int t = 0; t < 9; ++t) acc[t] = 0.f;
#pragma unroll (NQ <= 11 ? NQ : 1)
        for (int q = 0; q < NQ; ++q) {
            const float4 f0 = s_F[grp][q][0], f1 = s_F[grp][q][1], f2 = s_F[grp][q][2];
            const float4 A = s_R[grp][q][0], B = s_R[grp][q][1], C = s_R[grp][q][2];
            const V3 m0 = mk(A.x, A.y, A.z), m1 = mk(A.w, B.x, B.y), m2 = mk(B.z, B.w, C.x);
            const float* dr = &s_dN[(q * NE + i) * 3];
            const V3 dnr = mk(dr[0], dr[1], dr[2]);
            const V3 g = mk(dot(m0, dnr), dot(m1, dnr), dot(m2, dnr));
            float t[9];
            material_terms<MAT>(mk(f0.x, f0.y, f0.z), mk(f1.x, f1.y, f1.z), mk(f2.x, f2.y, f2.z), g, C.z, C.w, C.y, t);
#pragma unroll
            for (int j = 0; j < 9; ++j) acc[j] += t[j];
        }
        const float4 vv = S.v[tp[i]];
        float4 f;
        f.x = acc[0] - kd * (acc[3] * vv.x + acc[4] * vv.y + acc[5] * vv.z);
        f.y = acc[1] - kd * (acc[4] * vv.x + acc[6] * vv.y + acc[7] * vv.z);
        f.z = acc[2] - kd * (acc[5] * vv.x + acc[7] * vv.y + acc[8] * vv.z);
        f.w = 0.f;
        contrib[(size_t)eid * NE + i] = f;
    }
}

// Per node: the sum of its owners' element contributions in owner order (compensated in
// mixed precision), kept in u_new (the force buffer of the explicit solver), then the
// semi-implicit Euler update of that node (kenerl_semi_exicit_integration,
// octopus/src/GPU/GPU_Integrator.cu:27-34; the arithmetic of k_predict kind 1) and, for a
// fixed node, its fixation (fix_node, as k_constraints).  work indexes
// the scene's slots (one colour: every node).
__global__ void k_explicit_gather(const SceneDev* __restrict__ scenes, const NWork* __restrict__ work,
                                  const float4* __restrict__ contrib, int ne, StepParams P) {
    pdl_trigger();
    pdl_wait();
    const NWork wk = work[blockIdx.x];
    if ((int)threadIdx.x >= wk.count) return;
    const SceneDev& S = scenes[wk.scene];
    const int slot = wk.begin + threadIdx.x;
    const int vid = S.vids[slot];
    const int ob = S.own_off[slot], oe = S.own_off[slot + 1];
    const bool mixed = S.precision != 0;
    float fx = 0.f, fy = 0.f, fz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    for (int o = ob; o < oe; ++o) {
        const int packed = __ldg(S.owners + o);
        const float4 c = contrib[(size_t)(packed >> kOwnerShift) * ne + (packed & ((1 << kOwnerShift) - 1))];
        if (mixed) { kadd(fx, cx, c.x); kadd(fy, cy, c.y); kadd(fz, cz, c.z); }
        else { fx += c.x; fy += c.y; fz += c.z; }
    }
    if (mixed) { fx -= cx; fy -= cy; fz -= cz; }
    S.u_new[vid] = make_float4(fx, fy, fz, 0.f);
    const float dt = P.dt;
    float4 u = S.u[vid], v = S.v[vid];
    const float w = 1.f / S.y[vid].w;
    S.u_last[vid] = u;
    v.x += (S.gx + fx * w) * dt; v.y += (S.gy + fy * w) * dt; v.z += (S.gz + fz * w) * dt;
    u.x += v.x * dt; u.y += v.y * dt; u.z += v.z * dt;
    S.v[vid] = v;
    S.u[vid] = u;
    if (!isfinite(u.x + u.y + u.z + v.x + v.y + v.z)) atomicOr(S.status, kStatusNonFinite);
    // then the fixation of the sub-step (GPU_SemiExplicit::step applies the constraints after
    // the integration): fixed nodes are set to their group's target
    if (S.fix_of) {
        const int g = S.fix_of[vid];
        if (g >= 0) fix_node(S, vid, g);
    }
}

template <int E>
__global__ void __launch_bounds__(kBlock) k_element_diag(const SceneDev* __restrict__ scenes, int scene, int kind,
                                                         int material, float* __restrict__ out) {
    constexpr int NE = ElemT<E>::NE, NQ = ElemT<E>::NQ;
    const SceneDev& S = scenes[scene];
    const int eid = blockIdx.x * blockDim.x + threadIdx.x;
    if (eid >= S.n_elements) return;
    const int* tp = S.topo + (size_t)eid * NE;
    const double* dN = gdNd<E>();
    const double* wt = gwd<E>();
    const float4 c0 = S.eq[(size_t)eid * S.eq_stride * 3 + 2];   // lambda, mu of the element
    const double lam = c0.z, mu = c0.w;
    D3 A0 = {0, 0, 0}, A1 = A0, A2 = A0;   // accumulated Jx (kinds 4, 5, 6)
    double acc = 0.0;
    for (int q = 0; q < NQ; ++q) {
        D3 J0 = {0, 0, 0}, J1 = J0, J2 = J0, R0 = J0, R1 = J0, R2 = J0;
        for (int i = 0; i < NE; ++i) {
            const int v = tp[i];
            const float4 u = S.u[v], X = S.X[v];
            const D3 p = {(double)(X.x + u.x), (double)(X.y + u.y), (double)(X.z + u.z)};
            const D3 x = {(double)X.x, (double)X.y, (double)X.z};
            const double* d = dN + (q * NE + i) * 3;
            J0 = J0 + p * d[0]; J1 = J1 + p * d[1]; J2 = J2 + p * d[2];
            R0 = R0 + x * d[0]; R1 = R1 + x * d[1]; R2 = R2 + x * d[2];
        }
        const double w = wt[q];
        const double Vq = fabs(ddet(R0, R1, R2)) * w;
        if (kind == 1) { acc += fabs(ddet(J0, J1, J2)) * w; continue; }
        if (kind == 2) { acc += fabs(ddet(J0, J1, J2)) * w - Vq; continue; }
        if (kind == 5 || kind == 6) {
            A0 = A0 + J0; A1 = A1 + J1; A2 = A2 + J2;
            acc += fabs(ddet(A0, A1, A2)) * w - (kind == 6 ? Vq : 0.0);
            continue;
        }
        D3 m0, m1, m2;   // JX_inv columns
        dinv(R0, R1, R2, m0, m1, m2);
        if (kind == 4) { A0 = A0 + J0; A1 = A1 + J1; A2 = A2 + J2; J0 = A0; J1 = A1; J2 = A2; }
        const D3 F0 = J0 * m0.x + J1 * m0.y + J2 * m0.z, F1 = J0 * m1.x + J1 * m1.y + J2 * m1.z,
                 F2 = J0 * m2.x + J1 * m2.y + J2 * m2.z;
        if (kind == 3) { acc += ddet(F0, F1, F2) * w; continue; }
        D3 P0, P1, P2;
        pk1_d(material, F0, F1, F2, lam, mu, P0, P1, P2);
        // Cauchy C = P F^T / det F: C(r, k) = sum_j P_j[r] F_j[k]
        const double id = 1.0 / ddet(F0, F1, F2);
        double Cm[3][3];
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k)
                Cm[r][k] = (dget(P0, r) * dget(F0, k) + dget(P1, r) * dget(F1, k) + dget(P2, r) * dget(F2, k)) * id;
        // von_mises_stress (GPU_FEM_Material.cu:223-230) with m[col][row] = Cm[row][col]
        const double s01 = Cm[0][0] - Cm[1][1], s12 = Cm[1][1] - Cm[2][2], s02 = Cm[0][0] - Cm[2][2];
        double vm = 0.5 * (s01 * s01 + s12 * s12 + s02 * s02);
        vm += 3.0 * (Cm[1][0] * Cm[1][0] + Cm[2][1] * Cm[2][1] + Cm[2][0] * Cm[2][0]);
        acc += sqrt(vm) * Vq;
    }
    out[eid] = kind == 3 ? (acc > -1e-6 ? 0.f : 1.f) : (float)acc;
}

template <int E>
void diag_launch(int mat, const SceneDev* scenes, int scene, int n_elements, int kind, float* out, cudaStream_t st) {
    k_element_diag<E><<<(n_elements + kBlock - 1) / kBlock, kBlock, 0, st>>>(scenes, scene, kind, mat, out);
}

// ------------------------------------------------------------------------ FP64 energy
// Kinetic + elastic + gravity energy of one scene in FP64 (new: the reference has no
// energy evaluator; material energies of FEM_ContinuousMaterial.cpp:10-87).
template <int E>
__global__ void k_energy_elements(const SceneDev* __restrict__ scenes, int scene, int material, double* out, int* error) {
    constexpr int NE = ElemT<E>::NE, NQ = ElemT<E>::NQ;
    const SceneDev& S = scenes[scene];
    double local = 0.0;
    for (int eid = blockIdx.x * blockDim.x + threadIdx.x; eid < S.n_elements; eid += gridDim.x * blockDim.x) {
        const int* tp = S.topo + (size_t)eid * NE;
        const float* cd = cdN<E>();
        for (int q = 0; q < NQ; ++q) {
            const size_t ri = ((size_t)eid * S.eq_stride + (S.eq_stride == 1 ? 0 : q)) * 3;
            const float4 A = S.eq[ri], B = S.eq[ri + 1], C = S.eq[ri + 2];
            double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // J[col][row]
            for (int i = 0; i < NE; ++i) {
                const float4 u = S.u[tp[i]];
                for (int c = 0; c < 3; ++c) {
                    const double d = cd[(q * NE + i) * 3 + c];
                    J[c][0] += (double)u.x * d; J[c][1] += (double)u.y * d; J[c][2] += (double)u.z * d;
                }
            }
            const double m[3][3] = {{A.x, A.y, A.z}, {A.w, B.x, B.y}, {B.z, B.w, C.x}};   // m[col][row]
            double F[3][3];   // F[col][row]
            for (int b = 0; b < 3; ++b)
                for (int r = 0; r < 3; ++r) F[b][r] = (b == r ? 1.0 : 0.0) + J[0][r] * m[b][0] + J[1][r] * m[b][1] + J[2][r] * m[b][2];
            const double lam = C.z, mu = C.w, V = (double)C.y * (double)wq<E>(q);
            double psi;
            if (material == 2 || material == 3) {
                const double det = F[0][0] * (F[1][1] * F[2][2] - F[2][1] * F[1][2]) - F[1][0] * (F[0][1] * F[2][2] - F[2][1] * F[0][2]) +
                                   F[2][0] * (F[0][1] * F[1][2] - F[1][1] * F[0][2]);
                double n2 = 0;
                for (int b = 0; b < 3; ++b) for (int r = 0; r < 3; ++r) n2 += F[b][r] * F[b][r];
                const double alpha = material == 3 ? 1.0 + mu / lam : 1.0;
                psi = 0.5 * mu * (n2 - 3.0) + 0.5 * lam * (det - alpha) * (det - alpha);
            } else {
                double Em[3][3];
                for (int b = 0; b < 3; ++b)
                    for (int r = 0; r < 3; ++r) {
                        if (material == 0) Em[b][r] = 0.5 * (F[b][r] + F[r][b]) - (b == r ? 1.0 : 0.0);
                        else {
                            double s = 0;
                            for (int k = 0; k < 3; ++k) s += F[b][k] * F[r][k];
                            Em[b][r] = 0.5 * (s - (b == r ? 1.0 : 0.0));
                        }
                    }
                const double tr = Em[0][0] + Em[1][1] + Em[2][2];
                double n2 = 0;
                for (int b = 0; b < 3; ++b) for (int r = 0; r < 3; ++r) n2 += Em[b][r] * Em[b][r];
                psi = 0.5 * lam * tr * tr + mu * n2;
            }
            local += psi * V;
        }
    }
    if (!isfinite(local)) atomicOr(error, 2);
    for (int off = 16; off > 0; off >>= 1) local += __shfl_xor_sync(0xffffffffu, local, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(out + 1, local);
}

__global__ void k_energy_nodes(const SceneDev* __restrict__ scenes, int scene, double* out, int* error) {
    const SceneDev& S = scenes[scene];
    double kin = 0.0, grav = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n_nodes; i += gridDim.x * blockDim.x) {
        const float4 v = S.v[i], u = S.u[i], X = S.X[i];
        const double m = S.y[i].w;
        kin += 0.5 * m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
        const double px = (double)X.x + u.x, py = (double)X.y + u.y, pz = (double)X.z + u.z;
        grav -= m * (S.gx * px + S.gy * py + S.gz * pz);
    }
    if (!isfinite(kin) || !isfinite(grav)) atomicOr(error, 2);
    for (int off = 16; off > 0; off >>= 1) {
        kin += __shfl_xor_sync(0xffffffffu, kin, off);
        grav += __shfl_xor_sync(0xffffffffu, grav, off);
    }
    if ((threadIdx.x & 31) == 0) { atomicAdd(out + 0, kin); atomicAdd(out + 2, grav); }
}

// ------------------------------------------------------------------------ launchers
namespace {
// Launch with programmatic stream serialisation (pdl_trigger / pdl_wait in the kernel).
template <class... P, class... A>
void launch_pdl(void (*kernel)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t st, A... args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <class K> int persistent_grid(K kernel, int n_work, size_t smem = 0) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, smem);
    if (per_sm < 1) per_sm = 1;
    const int g = sms * per_sm;
    return n_work < g ? n_work : g;
}

// Persistent grid size (SMs x resident blocks) of each vertex-kernel instantiation,
// computed once outside any stream capture by prepare_vertex.
template <int E, int MAT, bool PACKED> int& grid_cap() {
    static int cap = 0;
    return cap;
}

template <int E, int MAT>
void vertex_dispatch(const SceneDev* scenes, const VWork* work, int n_work, int tpv, int mode, const StepParams& P,
                     double* red, cudaStream_t st) {
    if (mode < 0) {   // preparation call: fill the caches only
        if (grid_cap<E, MAT, false>() <= 0) grid_cap<E, MAT, false>() = persistent_grid(k_vertex<E, MAT>, 1 << 30);
        if (grid_cap<E, MAT, true>() <= 0) {
            cudaFuncSetAttribute(k_vertex_packed<E, MAT>, cudaFuncAttributeMaxDynamicSharedMemorySize, packed_smem_bytes<E>());
            grid_cap<E, MAT, true>() = persistent_grid(k_vertex_packed<E, MAT>, 1 << 30, packed_smem_bytes<E>());
        }
        return;
    }
    if (tpv == 0) {
        int cap = grid_cap<E, MAT, true>();
        if (cap <= 0) cap = 148 * 4;
        const int blocks = (n_work + kBlock / 32 - 1) / (kBlock / 32);
        launch_pdl(k_vertex_packed<E, MAT>, blocks < cap ? blocks : cap, kBlock, packed_smem_bytes<E>(), st, scenes, work, n_work, mode, P, red);
        return;
    }
    int cap = grid_cap<E, MAT, false>();
    if (cap <= 0) cap = 148 * 4;
    const int grid = n_work < cap ? n_work : cap;
    launch_pdl(k_vertex<E, MAT>, grid, kBlock, 0, st, scenes, work, n_work, tpv, mode, P, red);
}

template <int E>
void vertex_mat(int mat, const SceneDev* scenes, const VWork* work, int n_work, int tpv, int mode, const StepParams& P,
                double* red, cudaStream_t st) {
    switch (mat) {
        case 0: vertex_dispatch<E, 0>(scenes, work, n_work, tpv, mode, P, red, st); break;
        case 1: vertex_dispatch<E, 1>(scenes, work, n_work, tpv, mode, P, red, st); break;
        case 2: vertex_dispatch<E, 2>(scenes, work, n_work, tpv, mode, P, red, st); break;
        default: vertex_dispatch<E, 3>(scenes, work, n_work, tpv, mode, P, red, st); break;
    }
}

template <int E, bool RAW, int MINB>
void xpbd_launch(int mat, const SceneDev* scenes, const XWork* work, int n_work, const StepParams& P, cudaStream_t st) {
    switch (mat) {
        case 0: launch_pdl(k_xpbd<E, 0, RAW, MINB>, n_work, kBlock, 0, st, scenes, work, P); break;
        case 1: launch_pdl(k_xpbd<E, 1, RAW, MINB>, n_work, kBlock, 0, st, scenes, work, P); break;
        case 2: launch_pdl(k_xpbd<E, 2, RAW, MINB>, n_work, kBlock, 0, st, scenes, work, P); break;
        case 3: launch_pdl(k_xpbd<E, 3, RAW, MINB>, n_work, kBlock, 0, st, scenes, work, P); break;
        case 4: launch_pdl(k_xpbd<E, 4, RAW, MINB>, n_work, kBlock, 0, st, scenes, work, P); break;
        default: launch_pdl(k_xpbd<E, 5, RAW, MINB>, n_work, kBlock, 0, st, scenes, work, P); break;
    }
}
template <int E, bool RAW>
void xpbd_mat(int mat, const SceneDev* scenes, const XWork* work, int n_work, const StepParams& P, cudaStream_t st) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    if (n_work > 5 * sms) xpbd_launch<E, RAW, 8>(mat, scenes, work, n_work, P, st);   // more than a wave at 5 blocks/SM
    else xpbd_launch<E, RAW, 1>(mat, scenes, work, n_work, P, st);
}
template <int E>
void xpbd_form(int mat, bool raw, const SceneDev* scenes, const XWork* work, int n_work, const StepParams& P,
               cudaStream_t st) {
    if (raw) xpbd_mat<E, true>(mat, scenes, work, n_work, P, st);
    else xpbd_mat<E, false>(mat, scenes, work, n_work, P, st);
}
}  // namespace

// FP32 issue-rate microbenchmark: 8 independent FMA chains per thread held in registers.
__global__ void k_fma_peak(float* out, int iters, float a, float b) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-7f + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == 12345.f) out[0] = s;   // keeps the chains live
}

double launch_fma_peak(cudaStream_t st) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    static float* sink = nullptr;
    if (!sink) cudaMalloc(&sink, sizeof(float));
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    k_fma_peak<<<blocks, threads, 0, st>>>(sink, iters, 0.9999f, 1e-4f);
    return (double)blocks * threads * iters * 8;
}

// Flops the colour kernel executes per (owner, quadrature point), FMA = 2: Jx, F = I + Jx JX_inv
// (48), g = JX_inv^T dN_r (15), the material terms, 9 accumulations.  Jx: P1 forms F from three
// node differences (9, and g from 6 adds); Q1 from its monomial coefficients (90 per element
// over 8 points, then 54); P2 from its barycentric form (69 per element over 4 points, then 27);
// P3 and Q2 by the dense contraction (18 NE).
double vbd_term_flops(int element, int material) {
    double jx = 0, gf = 15.0;
    switch (element) {
        case 3: jx = 9.0; gf = 6.0; break;
        case 6: jx = 90.0 / 8.0 + 54.0; break;
        case 7: jx = 69.0 / 4.0 + 27.0; break;
        case 8: jx = 18.0 * 20; break;
        default: jx = 18.0 * 27; break;
    }
    const double mat = material == 0 ? 60.0 : (material == 1 ? 190.0 : 100.0);
    return jx + 48.0 + gf + mat + 9.0;
}

cudaError_t upload_shape_tables_fp64(int element, const double* dN, int n, const double* w, int nq) {
    cudaError_t e1, e2;
    switch (element) {
        case 3: e1 = cudaMemcpyToSymbol(g_dNd3, dN, n * 8); e2 = cudaMemcpyToSymbol(g_wd3, w, nq * 8); break;
        case 6: e1 = cudaMemcpyToSymbol(g_dNd6, dN, n * 8); e2 = cudaMemcpyToSymbol(g_wd6, w, nq * 8); break;
        case 7: e1 = cudaMemcpyToSymbol(g_dNd7, dN, n * 8); e2 = cudaMemcpyToSymbol(g_wd7, w, nq * 8); break;
        case 8: e1 = cudaMemcpyToSymbol(g_dNd8, dN, n * 8); e2 = cudaMemcpyToSymbol(g_wd8, w, nq * 8); break;
        case 9: e1 = cudaMemcpyToSymbol(g_dNd9, dN, n * 8); e2 = cudaMemcpyToSymbol(g_wd9, w, nq * 8); break;
        default: return cudaErrorInvalidValue;
    }
    return e1 != cudaSuccess ? e1 : e2;
}

cudaError_t upload_shape_tables(int element, const float* dN, int n_floats) {
    cudaError_t e1, e2;
    switch (element) {
        case 3: e1 = cudaMemcpyToSymbol(c_dN3, dN, n_floats * 4); e2 = cudaMemcpyToSymbol(g_dN3, dN, n_floats * 4); break;
        case 6: e1 = cudaMemcpyToSymbol(c_dN6, dN, n_floats * 4); e2 = cudaMemcpyToSymbol(g_dN6, dN, n_floats * 4); break;
        case 7: e1 = cudaMemcpyToSymbol(c_dN7, dN, n_floats * 4); e2 = cudaMemcpyToSymbol(g_dN7, dN, n_floats * 4); break;
        case 8: e1 = cudaMemcpyToSymbol(c_dN8, dN, n_floats * 4); e2 = cudaMemcpyToSymbol(g_dN8, dN, n_floats * 4); break;
        case 9:
            e1 = cudaMemcpyToSymbol(c_dN9, dN, n_floats * 4);
            e2 = cudaMemcpyToSymbol(g_dN9, dN, n_floats * 4);
            if (e1 == cudaSuccess) {
                float w9[27];
                for (int q = 0; q < 27; ++q) w9[q] = ShapeConst<9>::w(q);
                e1 = cudaMemcpyToSymbol(c_w9, w9, sizeof(w9));
            }
            break;
        default: return cudaErrorInvalidValue;
    }
    return e1 != cudaSuccess ? e1 : e2;
}

void prepare_vertex(int element, int material) {
    StepParams P{};
    launch_vertex(element, material, nullptr, nullptr, 1, 1, -1, P, nullptr, nullptr);
}

void launch_vertex(int element, int material, const SceneDev* scenes, const VWork* work, int n_work, int tpv, int mode,
                   const StepParams& P, double* red, cudaStream_t st) {
    if (n_work <= 0) return;
    switch (element) {
        case 3: vertex_mat<3>(material, scenes, work, n_work, tpv, mode, P, red, st); break;
        case 6: vertex_mat<6>(material, scenes, work, n_work, tpv, mode, P, red, st); break;
        case 7: vertex_mat<7>(material, scenes, work, n_work, tpv, mode, P, red, st); break;
        case 8: vertex_mat<8>(material, scenes, work, n_work, tpv, mode, P, red, st); break;
        case 9: vertex_mat<9>(material, scenes, work, n_work, tpv, mode, P, red, st); break;
    }
}

void launch_commit(const SceneDev* scenes, const VWork* work, int n_work, cudaStream_t st) {
    if (n_work <= 0) return;
    launch_pdl(k_commit, n_work, kBlock, 0, st, scenes, work, n_work);
}

void launch_predict(const SceneDev* scenes, const NWork* work, int n_work, int kind, int use_force, int chebyshev,
                    const StepParams& P, cudaStream_t st) {
    if (n_work <= 0) return;
    launch_pdl(k_predict, n_work, kNodeChunk, 0, st, scenes, work, n_work, kind, use_force, chebyshev, P);
}

void launch_velocity(const SceneDev* scenes, const NWork* work, int n_work, int pbd, const StepParams& P,
                     cudaStream_t st) {
    if (n_work <= 0) return;
    launch_pdl(k_velocity, n_work, kNodeChunk, 0, st, scenes, work, n_work, pbd, P);
}

void launch_chebyshev(const SceneDev* scenes, const NWork* work, int n_work, const StepParams& P, cudaStream_t st) {
    if (n_work <= 0) return;
    launch_pdl(k_chebyshev, n_work, kNodeChunk, 0, st, scenes, work, n_work, P);
}

void launch_effect(const SceneDev* scene, const NWork* work, int n_work, int slot, int kind, float dt, cudaStream_t st) {
    if (kind == 2) k_effect_stretch<<<1, 256, 0, st>>>(scene, slot, dt);
    else if (n_work > 0) k_effect_nodes<<<n_work, kNodeChunk, 0, st>>>(scene, work, slot);
}

void launch_mg_copy(const SceneDev* main, const SceneDev* sub, const int* map, int n, int dir, cudaStream_t st) {
    if (n > 0) k_mg_copy<<<(n + 255) / 256, 256, 0, st>>>(main, sub, map, n, dir);
}
void launch_mg_prolong(const SceneDev* main, const int* list, int count, int k, float w, cudaStream_t st) {
    if (count > 0) k_mg_prolong<<<(count + 255) / 256, 256, 0, st>>>(main, list, count, k, w);
}

void launch_wait_probe(int* error, long limit, cudaStream_t st) { k_wait_probe<<<1, 1, 0, st>>>(error, limit); }
void launch_nodes_out(const float4* src, const float4* X, float* out, int n, cudaStream_t st) {
    if (n > 0) k_nodes_out<<<(n + 255) / 256, 256, 0, st>>>(src, X, out, n);
}
void launch_nodes_in(const float* in, const float4* X, float4* dst, int n, cudaStream_t st) {
    if (n > 0) k_nodes_in<<<(n + 255) / 256, 256, 0, st>>>(in, X, dst, n);
}

void launch_constraints(const SceneDev* scenes, const NWork* work, int n_work, int box_pass, cudaStream_t st) {
    if (n_work <= 0) return;
    launch_pdl(k_constraints, n_work, kNodeChunk, 0, st, scenes, work, n_work, box_pass);
}

void launch_xpbd(int element, int material, bool raw, const SceneDev* scenes, const XWork* work, int n_work,
                 const StepParams& P, cudaStream_t st) {
    if (n_work <= 0) return;
    switch (element) {
        case 3: xpbd_form<3>(material, false, scenes, work, n_work, P, st); break;   // always V0
        case 6: xpbd_form<6>(material, raw, scenes, work, n_work, P, st); break;
        case 7: xpbd_form<7>(material, raw, scenes, work, n_work, P, st); break;
        case 8: xpbd_form<8>(material, raw, scenes, work, n_work, P, st); break;
        case 9: xpbd_form<9>(material, raw, scenes, work, n_work, P, st); break;
    }
}

namespace {
template <int E>
void explicit_mat(int mat, const SceneDev* scenes, int n_elements, float4* contrib, const StepParams& P, cudaStream_t st) {
    const int grid = (n_elements + kBlock / XpbdLanes<E>::G - 1) / (kBlock / XpbdLanes<E>::G);
    switch (mat) {
        case 0: launch_pdl(k_explicit_elem<E, 0>, grid, kBlock, 0, st, scenes, n_elements, contrib, P); break;
        case 1: launch_pdl(k_explicit_elem<E, 1>, grid, kBlock, 0, st, scenes, n_elements, contrib, P); break;
        case 2: launch_pdl(k_explicit_elem<E, 2>, grid, kBlock, 0, st, scenes, n_elements, contrib, P); break;
        default: launch_pdl(k_explicit_elem<E, 3>, grid, kBlock, 0, st, scenes, n_elements, contrib, P); break;
    }
}
}  // namespace

void launch_explicit_force(int element, int material, const SceneDev* scene, int n_elements, float4* contrib,
                           const NWork* slots, int n_slots, const StepParams& P, cudaStream_t st) {
    if (n_elements <= 0) return;
    switch (element) {
        case 3: explicit_mat<3>(material, scene, n_elements, contrib, P, st); break;
        case 6: explicit_mat<6>(material, scene, n_elements, contrib, P, st); break;
        case 7: explicit_mat<7>(material, scene, n_elements, contrib, P, st); break;
        case 8: explicit_mat<8>(material, scene, n_elements, contrib, P, st); break;
        case 9: explicit_mat<9>(material, scene, n_elements, contrib, P, st); break;
        default: return;
    }
    if (n_slots > 0)
        launch_pdl(k_explicit_gather, n_slots, kNodeChunk, 0, st, scene, slots, (const float4*)contrib,
                   element == 3 ? 4 : element == 6 ? 8 : element == 7 ? 10 : element == 8 ? 20 : 27, P);
}

int xpbd_elements_per_block(int element) {
    switch (element) {
        case 3: return kBlock / XpbdLanes<3>::G;
        case 6: return kBlock / XpbdLanes<6>::G;
        case 7: return kBlock / XpbdLanes<7>::G;
        case 8: return kBlock / XpbdLanes<8>::G;
        case 9: return kBlock / XpbdLanes<9>::G;
        default: return 1;
    }
}

void launch_element_diag(int element, int material, const SceneDev* scenes, int scene, int n_elements, int kind, float* out,
                         cudaStream_t st) {
    if (n_elements <= 0) return;
    switch (element) {
        case 3: diag_launch<3>(material, scenes, scene, n_elements, kind, out, st); break;
        case 6: diag_launch<6>(material, scenes, scene, n_elements, kind, out, st); break;
        case 7: diag_launch<7>(material, scenes, scene, n_elements, kind, out, st); break;
        case 8: diag_launch<8>(material, scenes, scene, n_elements, kind, out, st); break;
        case 9: diag_launch<9>(material, scenes, scene, n_elements, kind, out, st); break;
    }
}

void launch_energy(int element, int material, const SceneDev* scenes, int scene, int n_nodes, int n_elements, double* out,
                   int* error, cudaStream_t st) {
    const int gn = (n_nodes + 255) / 256 < 1184 ? (n_nodes + 255) / 256 : 1184;
    const int ge = (n_elements + 255) / 256 < 1184 ? (n_elements + 255) / 256 : 1184;
    k_energy_nodes<<<gn > 0 ? gn : 1, 256, 0, st>>>(scenes, scene, out, error);
    switch (element) {
        case 3: k_energy_elements<3><<<ge > 0 ? ge : 1, 256, 0, st>>>(scenes, scene, material, out, error); break;
        case 6: k_energy_elements<6><<<ge > 0 ? ge : 1, 256, 0, st>>>(scenes, scene, material, out, error); break;
        case 7: k_energy_elements<7><<<ge > 0 ? ge : 1, 256, 0, st>>>(scenes, scene, material, out, error); break;
        case 8: k_energy_elements<8><<<ge > 0 ? ge : 1, 256, 0, st>>>(scenes, scene, material, out, error); break;
        case 9: k_energy_elements<9><<<ge > 0 ? ge : 1, 256, 0, st>>>(scenes, scene, material, out, error); break;
    }
}

}  // namespace octb
