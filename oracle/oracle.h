/* CPU oracle for the OctopusEngine soft-body FEM time step — TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C++, the reference algorithms on the hot path so
 * that tests can check the CUDA product against them.  Only tests/, the smoke()
 * check and bench.py's CPU-baseline leg may load it; the product never links it.
 *
 * Pinning: the shape tables are checked against golden vectors extracted from the
 * reference's FEM_Shape.h, the beam meshes and lumped masses against the meshes the
 * reference itself wrote (assets/result/vtk/References).  The dynamics
 * (VBD / XPBD / explicit) follow the cited reference functions; the reference
 * cannot be compiled here (glm and the other submodules are absent), so the
 * dynamics are pinned at the level of the restated formulas, not of reference runs.
 *
 * Every function takes plain pointers and returns 0 on success, a negative value
 * on bad input.
 */
#ifndef OCT_ORACLE_H
#define OCT_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Scene description shared by every oracle solver (all arrays are host memory). */
typedef struct orc_desc {
    int32_t element;          /* reference Element enum value (Tetra=3 ... Hexa27=9) */
    int32_t n_nodes;
    const float* positions;   /* n_nodes*3 */
    int32_t n_elements;
    const int32_t* topology;  /* n_elements*nodes_per_element */
    const float* masses;      /* n_nodes */
    int32_t material;         /* Hooke=0, StVK=1, NeoHooke=2, Stable_NeoHooke=3, Corotated=4,
                                 FixedCorotated=5 (XPBD only) */
    float young, poisson;
    const float* young_per_element; /* NULL or n_elements (per-element Young modulus) */
    float damping;
    float gravity[3];
    int32_t n_fixed;
    const int32_t* fixed_ids;
    const int32_t* fixed_group;     /* NULL or per fixed id its rigid group 0..3 */
    const float* initial_velocity;  /* NULL or n_nodes*3 */
    /* VBD */
    int32_t iterations;
    float rho;                /* Chebyshev spectral radius, 0 = off */
    int32_t in_place;         /* 1: v3 in-place within colour, 0: v4 Jacobi within colour */
    int32_t n_colors;
    const int32_t* colors;    /* n_nodes colour ids (from orc_colour) */
    int32_t order_mode;       /* 0 ascending colours, 1 shuffled per iteration with seed */
    uint64_t seed;
    int32_t box_limit;        /* 1: clamp free nodes to [box_min, box_max] after each iteration */
    float box_min[3], box_max[3];
    /* XPBD */
    float global_damping;
    int32_t xpbd_version;     /* XPBD_FEM_VERSION: 0 XPBD, 1 Quadrature, 2 OptiShared, 3 OptiGroup */
    /* multigrid VBD (P2 / Q2 only): fraction of the iterations on the linear corner mesh, and
     * the node masses of that linear mesh (n_nodes; corner entries used); 0 = off */
    float mg_linear;
    const float* mg_masses;
} orc_desc;

int orc_elem_nodes(int element);
int orc_beam_counts(int element, int nx, int ny, int nz, int* n_nodes, int* n_elements);
int orc_beam_mesh(int element, int nx, int ny, int nz, float sx, float sy, float sz,
                  float ox, float oy, float oz, float* positions, int32_t* topology);
int orc_shape(int element, int* n_quadrature, double* coords, double* weights, double* dN);
int orc_masses(int element, const float* positions, int n_nodes, const int32_t* topology,
               int n_elements, float density, int distribution, float* masses);
int orc_precompute(int element, const float* positions, const int32_t* topology, int n_elements,
                   int fp64, double* JX_inv, double* V);
/* algo 0 = DSAT (Graph.h:321-371), 1 = Greedy (:200-207), 2 = Greedy_SLF on the vertex-dual
 * element graph (:237-277, :56-85).  target >= 0 applies ColorReduction (:941-969). */
int orc_colour(int element, const int32_t* topology, int n_elements, int n_nodes, int algo,
               int target, int32_t* colors, int32_t* n_colors);
int orc_conflicts(int element, const int32_t* topology, int n_elements, int n_nodes,
                  const int32_t* colors);

/* GPU-semantics VBD (GPU_VBD.cu / GPU_VBD_FEM.cu), T = float or double. */
void* orc_vbd_create(const orc_desc* d, int fp64);
int orc_vbd_step(void* h, float frame_dt, int substeps);
int orc_vbd_get(void* h, int what, double* out);   /* what: 0 p, 1 v, 2 last_p, 3 y, 4 mask */
/* Host threads the GPU-semantics VBD sweep may use for the vertices of one colour (default 1;
 * results are the same bit for bit for any count). */
void orc_set_threads(int n);
int orc_vbd_set(void* h, int what, const double* in);  /* what: 0 p, 1 v, 2 last_p, 3 y */
int orc_vbd_energy(void* h, double* parts);         /* kinetic, elastic, gravity, total */
int orc_vbd_residual(void* h, float dt, double* out_norms); /* [sum |r|, max |r|] of free nodes */
/* Per-vertex residual force of kernel_vbd_compute_residual (GPU_VBD_FEM.cu:482-559), n*3;
 * fixed (masked) vertices 0. */
int orc_vbd_forces(void* h, float dt, double* out);
void orc_vbd_destroy(void* h);

/* Per-element diagnostics of GPU_FEM (GPU_FEM.cu:20-107) on any solver handle: kind 0 von Mises
 * stress, 1 volume, 2 volume change, 3 inverted flag, 4 von Mises stress with Jx accumulated
 * over the quadrature points (kernel_compute_stress as written), 5 volume and 6 volume change
 * with the same accumulation (the fields of the reference's result files); out: n_elements. */
int orc_element_data(void* h, int kind, double* out);

/* Rigid motion of fixation group g (GPU_Fix_Constraint axis): p = offset + com + R (X - com),
 * R column-major; works on VBD, XPBD and explicit handles. */
int orc_set_fixation(void* h, int group, const float* offset, const float* rotation);

/* Scripted effect on any handle (GPU_Crush kind 0, GPU_RandomSphere kind 1 with params[0] the
 * radius, GPU_HighStretch kind 2 with params[1] the maximum distance and the moved ids), created
 * inactive; returns its index.  Effects run after the fixation, in creation order. */
int orc_add_effect(void* h, int kind, const float* params, const int32_t* ids, int n_ids);
int orc_set_effect_active(void* h, int index, int active);

/* Polar decomposition F = R S of mat3x3_polardecomposition (CUMatrix.cu:75-96), column-major,
 * in float (fp64 = 0) or double; and one XPBD constraint pair (eval_material,
 * GPU_PBD_FEM_Materials.cu:97-117) in double. */
int orc_polar(const double* F9, int fp64, double* R9, double* S9);
int orc_xpbd_pair(int material, int m, double lambda, double mu, const double* F9, double* P9, double* C);

/* Reference CPU VBD (VertexBlockDescent.cpp + VBD_FEM.cpp): single-thread Gauss-Seidel in
 * vertex order with the per-iteration full force pass (plot_residual). */
void* orc_cpuvbd_create(const orc_desc* d);
int orc_cpuvbd_step(void* h, float frame_dt, int substeps, int with_residual_pass);
int orc_cpuvbd_get(void* h, int what, double* out);
void orc_cpuvbd_destroy(void* h);
/* Run several independent CPU VBD scenes on n_threads host threads; returns seconds. */
double orc_cpuvbd_run_many(void** hs, int n, float frame_dt, int substeps, int with_residual_pass,
                           int n_threads);

/* GPU-semantics XPBD (GPU_PBD.cu + GPU_PBD_FEM.cu V0 kernel) and explicit
 * (GPU_Integrator.cu + GPU_FEM_Explicit.cu). */
void* orc_xpbd_create(const orc_desc* d, int fp64);
int orc_xpbd_step(void* h, float frame_dt, int substeps);
int orc_xpbd_get(void* h, int what, double* out);
void orc_xpbd_destroy(void* h);
void* orc_explicit_create(const orc_desc* d, int fp64);
int orc_explicit_step(void* h, float frame_dt, int substeps);
int orc_explicit_get(void* h, int what, double* out);
void orc_explicit_destroy(void* h);

#ifdef __cplusplus
}
#endif
#endif
