/* octopus_b200 — Blackwell (sm_100a) soft-body FEM time step, C ABI.
 *
 * Drop-in boundary for OctopusEngine's GPU solver objects.  One opaque scene bundles what
 * the reference splits over several classes:
 *   GPU_ParticleSystem(positions, masses)         octopus/include/GPU/GPU_ParticleSystem.h:54-73
 *   GPU_VBD(ps, iteration, rho)                    octopus/include/GPU/VBD/GPU_VBD.h:15-26
 *   GPU_VBD_FEM(element, topology, geometry, material, young, poisson, damping,
 *               version, target_color)             octopus/include/GPU/VBD/GPU_VBD_FEM.h:62-65
 *   GPU_PBD(global_damping) + GPU_PBD_FEM(...)     octopus/include/GPU/PBD/GPU_PBD.h:12-16,
 *                                                  octopus/include/GPU/PBD/GPU_PBD_FEM.h:19-20
 *   GPU_SemiExplicit + GPU_FEM_Explicit(...)       octopus/include/GPU/GPU_Integrator.h:34-36,
 *                                                  octopus/include/GPU/Explicit/GPU_FEM_Explicit.h:14-15
 *   GPU_Fix_Constraint(positions, Area*)           octopus/include/GPU/GPU_Constraint.h:11-18
 *   Cuda_ParticleSystem_Dynamics::update (sub-step loop)
 *                                                  octopus/src/Script/Dynamic/Cuda_ParticleSystem_Dynamic.cpp:17-31
 * The C++ adapters in octopus_b200.hpp restore the reference class shapes on top of this.
 *
 * Conventions: every call returns an oct_status; arrays are plain host pointers unless a
 * name says "device"; handles are owned by their context; one context per host thread.
 */
#ifndef OCTOPUS_B200_H
#define OCTOPUS_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef enum oct_status {
    OCT_OK = 0,
    OCT_EINVAL = 1,          /* bad argument */
    OCT_ENOMEM_BUDGET = 2,   /* request exceeds the context's HBM budget (nothing allocated) */
    OCT_ETIMEDOUT = 3,       /* a bounded device-side wait ran out */
    OCT_ENUMERIC = 4,        /* NaN/Inf found in a scene's state */
    OCT_ECUDA = 5,           /* a CUDA call failed; see oct_last_error */
    OCT_ENOTSUP = 6          /* combination not supported */
} oct_status;

/* Element ids are the reference's Element enum values (octopus/include/Mesh/Elements.h:4-15). */
enum { OCT_TETRA = 3, OCT_HEXA = 6, OCT_TETRA10 = 7, OCT_TETRA20 = 8, OCT_HEXA27 = 9 };
/* Material enum (octopus/include/Dynamic/FEM/ContinuousMaterial.h:8-10).  Corotated and
 * FixedCorotated exist only as XPBD constraint pairs in the reference (the GPU VBD and explicit
 * paths evaluate no stress for them); other solvers reject them with OCT_ENOTSUP. */
enum { OCT_HOOKE = 0, OCT_STVK = 1, OCT_NEOHOOKE = 2, OCT_STABLE_NEOHOOKE = 3, OCT_COROTATED = 4,
       OCT_FIXED_COROTATED = 5 };
/* Mass_Distribution (octopus/include/Dynamic/FEM/FEM_Shape.h:693-696). */
enum { OCT_MASS_UNIFORM = 0, OCT_MASS_FEMSHAPE = 1 };
/* Solvers. */
enum { OCT_SOLVER_VBD = 0, OCT_SOLVER_XPBD = 1, OCT_SOLVER_EXPLICIT = 2 };
/* VBD_Version (octopus/include/GPU/VBD/GPU_VBD_FEM.h:13-15): Base, Threaded_Quadrature and
 * Reduction_Symmetry update in place within a colour; Better_Coloration applies
 * ColorReduction to target_color and updates all vertices of a colour from the same state. */
enum { OCT_VBD_BASE = 0, OCT_VBD_THREADED_QUADRATURE = 1, OCT_VBD_REDUCTION_SYMMETRY = 2, OCT_VBD_BETTER_COLORATION = 3 };
/* XPBD_FEM_VERSION (octopus/include/GPU/PBD/GPU_PBD_FEM.h:11-13; GPU_PBD_FEM::step,
 * octopus/src/GPU/PBD/GPU_PBD_FEM.cu:661-689).  Tetra4 always uses the normalised V0 update;
 * for other elements XPBD selects V0, Quadrature and OptiShared (the reference default) the raw
 * V1/V2 update, and OptiGroup projects nothing, as in the reference. */
enum { OCT_XPBD_XPBD = 0, OCT_XPBD_QUADRATURE = 1, OCT_XPBD_OPTISHARED = 2, OCT_XPBD_OPTIGROUP = 3 };
/* Colouring algorithms (octopus/include/Tools/Graph.h). */
enum { OCT_COLOR_DSAT = 0, OCT_COLOR_GREEDY = 1 };
/* Colour order per iteration: ascending (fixed, reproducible), or a std::shuffle with an
 * std::mt19937 seeded once per scene (the reference reseeds from the clock each call). */
enum { OCT_ORDER_ASCENDING = 0, OCT_ORDER_SHUFFLED = 1 };
/* Precision: PLAIN = FP32 with the reference's Newton-skip rule (|det H| <= 1e-6);
 * MIXED = FP32 bulk with compensated accumulation, FP64 Newton solve for ill-conditioned
 * blocks, FP64 energy/residual reductions. */
enum { OCT_PREC_PLAIN = 0, OCT_PREC_MIXED = 1 };

typedef struct oct_ctx oct_ctx;
typedef struct oct_scene oct_scene;
typedef struct oct_batch oct_batch;
typedef struct oct_server oct_server;

typedef struct oct_scene_desc {
    int32_t solver;                 /* OCT_SOLVER_* */
    int32_t element;                /* OCT_TETRA ... OCT_HEXA27 */
    int32_t n_nodes;
    const float* positions;         /* n_nodes*3 rest positions (Mesh::Geometry) */
    int32_t n_elements;
    const int32_t* topology;        /* n_elements*nodes_per_element (Mesh::Topology) */
    const float* masses;            /* n_nodes, or NULL: computed from density/mass_distribution */
    float density;
    int32_t mass_distribution;      /* OCT_MASS_* */
    int32_t material;               /* OCT_HOOKE ... OCT_STABLE_NEOHOOKE */
    float young, poisson;
    const float* young_per_element; /* NULL or n_elements: per-element Young modulus */
    float damping;                  /* VBD / explicit Rayleigh-like damping k_d */
    float gravity[3];
    int32_t n_fixed;                /* fixed-node list (GPU_Fix_Constraint ids)... */
    const int32_t* fixed_ids;
    const int32_t* fixed_group;     /* NULL, or per fixed id its rigid group 0..3 (one
                                       GPU_Fix_Constraint each; the reference scenes attach two) */
    int32_t fix_by_plane;           /* ...or nodes with dot(p - origin, normal) > 0 (Area::Plane) */
    float plane_origin[3], plane_normal[3];
    const float* initial_velocity;  /* NULL or n_nodes*3 */
    /* VBD */
    int32_t iterations;
    float rho;                      /* Chebyshev spectral radius; 0 disables */
    int32_t vbd_version;            /* OCT_VBD_* */
    int32_t target_color;           /* for OCT_VBD_BETTER_COLORATION; < 0 means no reduction */
    int32_t color_algo;             /* OCT_COLOR_* */
    int32_t order_mode;             /* OCT_ORDER_* */
    uint64_t seed;
    /* XPBD */
    float global_damping;
    int32_t precision;              /* OCT_PREC_* */
    int32_t box_limit;              /* 1: clamp free nodes to [box_min, box_max] each iteration */
    float box_min[3], box_max[3];
    int32_t threads_per_vertex;     /* 0 = measured default per element, -1 = one lane per
                                       (vertex, owner) pair packed into warps, 1..32 = lanes per
                                       vertex (power of two; a colour whose vertices average
                                       more than 8 owners per lane gets wider groups) */
    int32_t xpbd_version;           /* OCT_XPBD_* (default OCT_XPBD_OPTISHARED) */
    float mg_linear;                /* multigrid VBD for P2 / Q2 (MG_VBD_FEM,
                                       octopus/include/Dynamic/VBD/MG_VertexBlockDescent.h:52-74):
                                       fraction of the iterations solved on the linear mesh of
                                       the corners, with its own colouring and masses (from
                                       density and mass_distribution); mid nodes follow by
                                       prolongation.  0 = off.  Such scenes are stepped alone
                                       (no batch, no frame graph), without Chebyshev. */
} oct_scene_desc;

/* Context: device, stream, HBM budget (bytes; 0 = 90% of free device memory). */
oct_status oct_ctx_create(int device, size_t hbm_budget, oct_ctx** out);
oct_status oct_ctx_destroy(oct_ctx* ctx);
const char* oct_last_error(oct_ctx* ctx);
oct_status oct_ctx_memory(oct_ctx* ctx, size_t* used, size_t* budget);
void oct_desc_init(oct_scene_desc* d);   /* fills defaults (VBD, Stable NH, g = (0,-9.81,0)) */

/* Scene = particle system + solver + FEM object + fix constraint.  Replaces
 * Cuda_FEM_Dynamic::init (octopus/include/Script/Dynamic/Cuda_FEM_Dynamic.h:18-25). */
oct_status oct_scene_create(oct_ctx* ctx, const oct_scene_desc* desc, oct_scene** out);
oct_status oct_scene_destroy(oct_scene* s);
/* Cuda_ParticleSystem_Dynamics::update: `substeps` integrator steps of frame_dt/substeps,
 * asynchronous on the context stream (the reference's GPU_Integrator::step calls). */
oct_status oct_scene_step(oct_scene* s, float frame_dt, int substeps);
oct_status oct_scene_sync(oct_scene* s);
/* Frame graphs (new; the reference launches every kernel from the host): with capture on, a
 * frame's sub-steps are captured once into a CUDA graph and replayed while frame_dt and
 * substeps stay the same.  Off by default.  Frames with the shuffled colour order, and the
 * first frame after a pending initial velocity, still run launch by launch. */
oct_status oct_scene_set_capture(oct_scene* s, int on);
/* GPU_ParticleSystem::get_position / get_velocity (synchronous D2H into host arrays). */
oct_status oct_scene_get_positions(oct_scene* s, float* out_n3);
oct_status oct_scene_get_velocities(oct_scene* s, float* out_n3);
/* Node state in (new: the reference has getters only).  VBD moves by the implicit velocity
 * (p - last_p) / dt (GPU_VBD.cu:6-18), so on a VBD scene the velocities set here become that
 * implicit velocity at the scene's next own sub-step, as oct_scene_desc.initial_velocity does
 * (a batch takes the flag when it is created); positions set alone keep the previous
 * last_p.  Setting positions and then zero velocities restarts a VBD scene at rest in the
 * given configuration. */
oct_status oct_scene_set_positions(oct_scene* s, const float* in_n3);
oct_status oct_scene_set_velocities(oct_scene* s, const float* in_n3);
oct_status oct_scene_info(oct_scene* s, int32_t* n_nodes, int32_t* n_elements, int32_t* n_colors, int32_t* n_fixed);
/* Colouring and colour-sorted vertex order (GPU_VBD_FEM::create_buffers). */
oct_status oct_scene_get_coloring(oct_scene* s, int32_t* colors, int32_t* vertex_order);
/* Lumped masses used by the scene (compute_fem_mass). */
oct_status oct_scene_get_masses(oct_scene* s, float* out_n);
/* Element type, rest positions (n_nodes*3) and topology (n_elements*nodes_per_element) of a
 * scene, as given at creation (GPU_FEM's mesh; the VTK recorder writes them). */
oct_status oct_scene_element_type(oct_scene* s, int32_t* element);
oct_status oct_scene_get_rest_positions(oct_scene* s, float* out_n3);
oct_status oct_scene_get_topology(oct_scene* s, int32_t* out);
/* Run metadata in the JSON of MeshRecorder and FEM_Dynamic_Recorder::add_data_json
 * (octopus/src/Script/Record/Recorder.cpp:12-36): {"mesh" : {...}, "fem" : {...}}.  With out
 * NULL only *length is set; otherwise capacity must hold length + 1 bytes. */
oct_status oct_scene_metadata_json(oct_scene* s, char* out, size_t capacity, size_t* length);
/* Move the fixed nodes rigidly: p = offset + com + R (init_p - com), R column-major 3x3
 * (GPU_Fix_Constraint axis, octopus/src/GPU/GPU_Constraint.cu:108-112).  _group addresses
 * one of the four rigid groups (oct_scene_set_fixation is group 0); batches holding the
 * scene see the change. */
oct_status oct_scene_set_fixation(oct_scene* s, const float offset[3], const float rotation[9]);
oct_status oct_scene_set_fixation_group(oct_scene* s, int group, const float offset[3], const float rotation[9]);
/* Switches the scene between OCT_PREC_PLAIN and OCT_PREC_MIXED for its own steps (a batch
 * keeps the precision its scenes had when the batch was created). */
oct_status oct_scene_set_precision(oct_scene* s, int precision);
/* Scripted effects of the reference's rigid controller (Cuda_Constraint_Rigid_Controller,
 * octopus/src/Script/Dynamic/Cuda_Constraint_Rigid_Controller.cpp:9-23; GPU_Crush,
 * GPU_RandomSphere, GPU_HighStretch, octopus/include/GPU/GPU_Constraint.h:20-80, kernels
 * octopus/src/GPU/GPU_Constraint.cu:22-92):
 *   OCT_EFFECT_CRUSH          free nodes flattened to y = 0 (velocity 0)
 *   OCT_EFFECT_RANDOM_SPHERE  free nodes scattered in a sphere of radius params[0] about the
 *                             node centroid by the reference's sine hash
 *   OCT_EFFECT_HIGH_STRETCH   params[0] boundary nodes chosen farthest-first are pushed away
 *                             from the centroid by t, t growing by dt per call up to params[1]
 * Deactivating a high stretch resets its distance to 0, as the controller does when it turns the
 * effect off (Cuda_Constraint_Rigid_Controller.cpp:72-76,150-153).
 * Effects are created inactive (as the controller creates them) and run, while active, after
 * the fixation and before the box limit, in creation order, wherever the constraints run (every
 * VBD iteration; every XPBD or explicit sub-step).  At most 4 per scene; add them before the
 * scene joins a batch (the batch's graph is captured with the effects it finds); toggling works
 * at any time. */
enum { OCT_EFFECT_CRUSH = 0, OCT_EFFECT_RANDOM_SPHERE = 1, OCT_EFFECT_HIGH_STRETCH = 2 };
oct_status oct_scene_add_effect(oct_scene* s, int kind, const float* params, int32_t* index);
oct_status oct_scene_set_effect_active(oct_scene* s, int32_t index, int active);
/* The node ids a high-stretch effect moves (n = 0 for the other kinds). */
oct_status oct_scene_effect_ids(oct_scene* s, int32_t index, int32_t* ids, int32_t* n);
/* Boundary nodes of a mesh, ascending (MeshTools::Get_Surface_Geometry_Ids,
 * octopus/include/Mesh/MeshTools.h:64-89); ids may be NULL to get the count. */
oct_status oct_surface_nodes(int32_t element, const int32_t* topology, int32_t n_elements, int32_t* ids, int32_t* n);
/* FP64 diagnostics: kinetic, elastic, gravity potential, total energy; and the VBD
 * residual r = f - M/dt^2 (p - y) - damping term (kernel_vbd_compute_residual) as
 * [sum |r|, max |r|] over free nodes.  Both return OCT_ENUMERIC on NaN/Inf state. */
oct_status oct_scene_energy(oct_scene* s, double out4[4]);
oct_status oct_scene_residual(oct_scene* s, float dt, double out2[2]);
/* Per-element diagnostics of GPU_FEM::get_stress / get_volume / get_volume_diff / get_inverted
 * (octopus/include/GPU/GPU_FEM.h:66-69; kernels octopus/src/GPU/GPU_FEM.cu:20-107), evaluated in
 * FP64 on the current positions (the exact value of the reference's formulas there),
 * out: n_elements floats.
 *   OCT_DIAG_STRESS      sum_q von Mises(Cauchy(F_q)) V_q, F_q = Jx_q JX_inv_q
 *   OCT_DIAG_STRESS_ACCUMULATED  the same with Jx summed over the quadrature points, as
 *                        kernel_compute_stress accumulates it (equal for one-point elements;
 *                        octb::GPU_FEM::get_stress returns this one)
 *   OCT_DIAG_VOLUME      sum_q |det Jx_q| w_q
 *   OCT_DIAG_VOLUME_DIFF sum_q (|det Jx_q| w_q - V_q)   (the reference getter launches the
 *                        inversion kernel instead; octb::GPU_FEM::get_volume_diff does the same)
 *   OCT_DIAG_INVERTED    1 where sum_q det(F_q) w_q < -1e-6, else 0
 *   OCT_DIAG_VOLUME_ACCUMULATED       sum_q |det(sum_{q' <= q} Jx_q')| w_q: the volume with the
 *                        stress kernel's accumulation, the form of the "volume" field in the
 *                        reference's result files (assets/result/vtk/References/*.vtk)
 *   OCT_DIAG_VOLUME_DIFF_ACCUMULATED  the same minus sum_q V_q (their "volume_diff" field)
 * Corotated and FixedCorotated have no stress (0), as in the reference. */
enum { OCT_DIAG_STRESS = 0, OCT_DIAG_VOLUME = 1, OCT_DIAG_VOLUME_DIFF = 2, OCT_DIAG_INVERTED = 3,
       OCT_DIAG_STRESS_ACCUMULATED = 4, OCT_DIAG_VOLUME_ACCUMULATED = 5, OCT_DIAG_VOLUME_DIFF_ACCUMULATED = 6 };
oct_status oct_scene_element_data(oct_scene* s, int kind, float* out_n_elements);
/* Per-vertex residual force of GPU_VBD_FEM::get_forces (octopus/src/GPU/VBD/GPU_VBD_FEM.cu:
 * 482-559) for sub-step dt: elastic + damping + inertia terms, 0 on fixed vertices; zeros for
 * XPBD and explicit scenes (GPU_FEM::get_forces).  out: n_nodes*3. */
oct_status oct_scene_vertex_residuals(oct_scene* s, float dt, float* out_n3);
/* Failure state of a scene's own steps (new: the reference checks nothing).  Waits for the
 * context stream, then reads and clears the flags the scene's kernels raised since the last
 * query: OCT_ENUMERIC when a node's position or velocity became NaN / Inf in a sub-step,
 * OCT_ETIMEDOUT when a bounded device wait gave up (the rest of that colour sweep was left
 * unsolved), else the context's own error word (OCT_OK when clear). */
oct_status oct_scene_status(oct_scene* s);

/* Batch: many scenes stepped together, one launch per (element type, colour) across all
 * scenes, driven by a per-scene work table, the sub-step captured as a CUDA graph.  The
 * scenes are all VBD scenes of this context with equal iteration counts, or all XPBD scenes
 * (GPU_PBD::step over every scene: one launch per (element type, material, update form,
 * colour) with the element colours of all scenes, each scene with its own global damping);
 * explicit scenes are stepped alone (OCT_ENOTSUP). */
/* Lane mapping of a VBD or explicit scene's vertex kernel (same values as
 * oct_scene_desc.threads_per_vertex: -1 packed pairs, 0 measured default, 1..32 lanes per
 * vertex).  OCT_ENOTSUP for the packed mapping when a vertex has more than 32 owners. */
oct_status oct_scene_set_mapping(oct_scene* s, int threads_per_vertex);
/* The mapping in effect: -1 packed pairs, else lanes per vertex (the measured default and the
 * fallback for vertices with more than 32 owners resolved); 0 for XPBD scenes. */
oct_status oct_scene_get_mapping(oct_scene* s, int32_t* threads_per_vertex);
/* Mapping autotuner (new): for each element type among the VBD and explicit scenes (XPBD
 * scenes are skipped), times one colour sweep of all its scenes under every candidate mapping
 * (packed pairs when every scene has owner entries and at most 32 owners per vertex, 1, 2, 4,
 * 8, 16, 32 lanes per vertex; best of three timings each) and sets the fastest on those
 * scenes, keeping the measured default unless another mapping is at least 3 % faster.  The timed sweeps write only the Jacobi
 * scratch buffer, so positions and velocities are unchanged.  chosen (may be NULL): per
 * element id the mapping picked (-1 packed), 0 for element types absent.  Run it before
 * oct_batch_create; it leaves no batch behind. */
oct_status oct_autotune_mapping(oct_ctx* ctx, oct_scene* const* scenes, int n, float dt, int sweeps, int32_t chosen[10]);
oct_status oct_batch_create(oct_ctx* ctx, oct_scene* const* scenes, int n, oct_batch** out);
oct_status oct_batch_step(oct_batch* b, float frame_dt, int substeps);
/* Failure state of every scene during the batch's frames, in one read: out[i] (n scenes, in
 * the order given to oct_batch_create) is OCT_OK, OCT_ENUMERIC or OCT_ETIMEDOUT as for
 * oct_scene_status; a time-out that belongs to no single scene (a kernel's constant-table
 * staging) is reported for all.  Waits for the context stream; reading clears the flags.
 * Scenes are independent, so one scene's failure leaves the others' results intact. */
oct_status oct_batch_status(oct_batch* b, int32_t* out_n_scenes);
/* Captures the sub-step graph for (frame_dt, substeps) without launching it, so that a later
 * oct_batch_step starts at once (the serving loop prepares the next batch this way while the
 * current frame runs). */
oct_status oct_batch_prepare(oct_batch* b, float frame_dt, int substeps);
oct_status oct_batch_destroy(oct_batch* b);
/* End-to-end helpers: upload all scenes' positions+velocities from one host array (scene
 * order, n_i*6 floats each: p then v) and read them back. */
oct_status oct_batch_set_state(oct_batch* b, const float* host_state);
oct_status oct_batch_get_state(oct_batch* b, float* host_state);
oct_status oct_batch_state_size(oct_batch* b, size_t* n_floats);

/* Host-side scene building blocks (no GPU needed).
 * Beam mesh as BeamMeshGenerator + promotions build it (octopus/src/Mesh/Generator/BeamGenerator.cpp:5-380):
 * call with positions == NULL to get the sizes, then with arrays of those sizes. */
oct_status oct_beam_mesh(int element, int nx, int ny, int nz, const float size[3], const float offset[3],
                         int32_t* n_nodes, int32_t* n_elements, float* positions, int32_t* topology);
/* compute_fem_mass (octopus/src/Dynamic/FEM/FEM_Shape.cpp:86-121). */
oct_status oct_lumped_masses(int element, const float* positions, int n_nodes, const int32_t* topology, int n_elements,
                             float density, int distribution, float* out_masses);
/* Shape-function derivatives at the quadrature points (FEM_Shape::build): coords nq*3,
 * weights nq, dN nq*nodes*3; any output may be NULL. */
oct_status oct_shape_table(int element, int32_t* n_quadrature, double* coords, double* weights, double* dN);
/* Vertex colouring as GPU_VBD_FEM::build_graph_color (DSAT or Greedy on the primal graph,
 * optional ColorReduction to target when target > 0), or, with algo = 2, the element
 * colouring of GPU_PBD_FEM::build_graph_color (Greedy_SLF on the vertex-dual graph; colors
 * then has n_elements entries).  conflicts = same-colour adjacencies counted per multiset
 * occurrence at both ends (GraphColoration::Get_Conflict summed). */
oct_status oct_color(int element, const int32_t* topology, int n_elements, int n_nodes, int algo, int target,
                     int32_t* colors, int32_t* n_colors, int64_t* conflicts);

/* Device bytes a scene built from desc will hold (estimate used for HBM admission). */
oct_status oct_scene_footprint(const oct_scene_desc* desc, size_t* bytes);

/* Serving loop: continuous batching of (scene, steps) requests on one device.  Requests are
 * admitted while HBM budget and slots allow; the host set-up of newly admitted scenes runs
 * on worker threads while the GPU advances the active batch, and admitted scenes join the
 * batch at the next frame boundary; finished scenes leave it and free their memory.  Every
 * frame advances all active scenes by frame_dt (substeps x iterations VBD). */
typedef struct oct_server_config {
    size_t hbm_budget;        /* bytes of scene state the server may hold (0 = context budget) */
    int32_t max_scenes;       /* active slots */
    float frame_dt;
    int32_t substeps;
    int32_t iterations;       /* overrides desc->iterations of submitted scenes */
    int32_t precision;        /* OCT_PREC_* for submitted scenes */
    int32_t setup_threads;    /* host threads for scene set-up (0 = hardware concurrency) */
} oct_server_config;

typedef struct oct_server_stats {
    int64_t submitted, admitted, finished, rejected, queued, active;
    int64_t frames;
    double p50_step_ms, p99_step_ms, mean_step_ms;   /* device time of a batched frame */
    double vertex_iterations;                         /* total free-vertex updates done */
    double busy_ms;                                   /* summed device time of the frames */
    size_t bytes_in_use;
    double gap_ms;      /* device idle time between consecutive frames of a busy period */
    int64_t failed;     /* requests ended by OCT_ENUMERIC / OCT_ETIMEDOUT (oct_server_poll says which) */
} oct_server_stats;

oct_status oct_server_create(oct_ctx* ctx, const oct_server_config* cfg, oct_server** out);
/* Queues a request; the desc and its arrays are copied.  OCT_ENOMEM_BUDGET if the scene can
 * never fit the server budget (the request is rejected, nothing is queued). */
oct_status oct_server_submit(oct_server* srv, const oct_scene_desc* desc, int32_t steps, int64_t* request_id);
/* One scheduling round: start admissions that fit, run one batched frame of the active
 * scenes, retire finished requests.  Returns the number of active scenes after the frame. */
oct_status oct_server_tick(oct_server* srv, int32_t* n_active);
/* done = 1 when the request has finished; then positions (n_nodes*3, may be NULL) are copied out.
 * After every frame the server reads the per-scene failure state (oct_batch_status): a request
 * whose state went NaN / Inf or whose work timed out leaves at once, done = 1, and poll returns
 * OCT_ENUMERIC or OCT_ETIMEDOUT for it (no positions); the other requests go on unchanged. */
oct_status oct_server_poll(oct_server* srv, int64_t request_id, int32_t* done, float* positions);
oct_status oct_server_get_stats(oct_server* srv, oct_server_stats* out);
oct_status oct_server_destroy(oct_server* srv);

/* VTK 5.1 ASCII unstructured grids, one element type (VTK_Formater::save_mesh and
 * add_scalar_data / add_vector_data, octopus/src/Mesh/Converter/VTK_Formater.cpp; VTK_Loader::load
 * and get_point_data_v3, octopus/src/Mesh/Converter/MeshLoader.cpp:97-330).  The text matches the
 * reference writer's byte for byte; Hexa27 nodes go to and come from VTK's node order. */
enum { OCT_VTK_POINT = 0, OCT_VTK_CELL = 1 };
typedef struct oct_vtk_field {
    const char* name;
    int32_t location;      /* OCT_VTK_POINT (n_nodes values) or OCT_VTK_CELL (n_elements values) */
    int32_t components;    /* 1: SCALARS, 3: VECTORS */
    const float* data;
} oct_vtk_field;
oct_status oct_vtk_write(const char* path, const float* positions, int32_t n_nodes, int32_t element,
                         const int32_t* topology, int32_t n_elements, const oct_vtk_field* fields, int32_t n_fields);
/* Reads a mesh; with positions and topology NULL only the sizes and element type are set.
 * OCT_ENOTSUP for binary files, other datasets or mixed element types. */
oct_status oct_vtk_read_mesh(const char* path, int32_t* element, int32_t* n_nodes, int32_t* n_elements, float* positions,
                             int32_t* topology);
/* Reads n values of the named SCALARS (components 1) or VECTORS (components 3) field. */
oct_status oct_vtk_read_field(const char* path, const char* name, int32_t components, int32_t n, float* out);
/* One frame of FEM_VTK_Recorder::save (octopus/src/Script/Record/Recorder.cpp:117-171): rest mesh,
 * point data weights (masses), u_norm, u (displacement), smooth_stress; cell data stress
 * (OCT_DIAG_STRESS_ACCUMULATED), volume, volume_diff, inverted.  The reference's recorder writes
 * the inversion flags under volume_diff and zeros under inverted; here both hold their values. */
oct_status oct_scene_write_vtk(oct_scene* s, const char* path);

/* Shape-function values N (nodes of the element) at reference coordinates x
 * (FEM_Shape::build_shape, octopus/include/Dynamic/FEM/FEM_Shape.h) and the reference-element
 * node coordinates (3 per node; FEM_Shape::get_vertices for the corners). */
oct_status oct_shape_values(int32_t element, const double x[3], double* N);
oct_status oct_reference_nodes(int32_t element, double* X);

/* Accuracy measures of the reference's experiments (octopus/include/Script/Measure/MeshDiff.h,
 * octopus/src/Script/Record/Recorder.cpp:190-330); errors accumulated in FP64.
 * out6 = {MSE, RMSE, MAE, max, L1, L2} of the per-point error vectors (Error::update). */
/* MeshDiff_MSE: e_i = a_i - b_i - offset (offset may be NULL). */
oct_status oct_mesh_error(const float* a, const float* b, int32_t n, const float offset[3], double out6[6]);
/* Beam_MSE_Sampling: a regular grid of samples (nb_sample per unit length) inside the
 * reference mesh's box is located, at rest, in an element of every mesh; the error of mesh m
 * compares the samples interpolated in its current positions and in the reference mesh's,
 * each relative to its rest box minimum.  Samples some mesh does not contain are dropped. */
typedef struct oct_sampler oct_sampler;
oct_status oct_beam_sampler_create(int32_t n_meshes, const int32_t* elements, const int32_t* n_nodes,
                                   const float* const* rest_positions, const int32_t* n_elements,
                                   const int32_t* const* topologies, int32_t reference, int32_t nb_sample, oct_sampler** out);
oct_status oct_beam_sampler_info(oct_sampler* s, int32_t* n_samples);
oct_status oct_beam_sampler_error(oct_sampler* s, int32_t mesh, const float* positions, const float* reference_positions,
                                  double out6[6]);
oct_status oct_beam_sampler_destroy(oct_sampler* s);
/* FEM_Flexion_error_recorder: |target - p|^2 of the first particle whose rest position is
 * within 1e-3 of follow; its index in *particle (may be NULL). */
oct_status oct_flexion_error(const float* rest, const float* current, int32_t n, const float follow[3], const float target[3],
                             double* error, int32_t* particle);
/* FEM_Torsion_error_recorder: samples_per_edge points on every element edge lying on the beam's
 * y = z = 0 edge; for each, the rotation angle (degrees) about the section centre (0.5, 0.5)
 * between rest and current state, against its current x / beam_length; sorted by distance,
 * points closer than 1e-4 merged (angles averaged).  *count = number of points (the arrays
 * receive at most capacity). */
oct_status oct_torsion_profile(int32_t element, const float* rest, const float* current, int32_t n_nodes,
                               const int32_t* topology, int32_t n_elements, int32_t samples_per_edge, float beam_length,
                               float* distance, float* angles, int32_t capacity, int32_t* count);

/* Checkpoint / restore of one scene (new; the reference's DataRecorder writes no restorable
 * state): a 4-float header (format tag, node count, element count, element type), then per
 * node the displacement, the start-of-sub-step displacement, the velocity and the fixed mask,
 * then the fixation groups, the effects' stretch distances, the multigrid schedule and the
 * pending initial velocity.  A restored scene continues exactly as the saved one; restore
 * checks the header first and refuses (OCT_EINVAL) a checkpoint of a scene of another shape. */
oct_status oct_scene_state_size(oct_scene* s, size_t* n_floats);
oct_status oct_scene_save(oct_scene* s, float* out);
oct_status oct_scene_restore(oct_scene* s, const float* in);

/* Failure-detection probe (new): runs the colour kernels' bounded mbarrier wait on a phase
 * that never completes, with at most limit (<= 1e6) polls, and returns OCT_ETIMEDOUT through
 * the context's error word; the context stays usable. */
oct_status oct_ctx_wait_probe(oct_ctx* ctx, int32_t limit);

/* Measurement helpers.  The context's CUDA stream (cudaStream_t), to record events on it. */
oct_status oct_ctx_stream(oct_ctx* ctx, void** stream);
/* Measured FP32 FMA throughput of the device (TFLOP/s) from a register-resident FMA loop. */
oct_status oct_fp32_peak(oct_ctx* ctx, double* tflops);
/* Per element group g of a VBD batch (scenes sharing element type, material and thread
 * mapping): the FP32 flops the colour kernel executes and the minimal DRAM bytes of one VBD
 * colour sweep (all colours once), its launch count and vertex updates.  Returns OCT_EINVAL
 * past the last group, OCT_ENOTSUP for an XPBD batch. */
oct_status oct_batch_group_info(oct_batch* b, int g, int32_t* element, int32_t* material, double* flops_per_sweep,
                                double* bytes_per_sweep, int32_t* launches_per_sweep, int64_t* vertices_per_sweep);
/* Runs `sweeps` colour sweeps of group g of a VBD batch alone on the context stream (outside
 * the graph, state advances as in an iteration) and returns their total device time (CUDA
 * events); OCT_ENOTSUP for an XPBD batch. */
oct_status oct_batch_time_group(oct_batch* b, int g, int sweeps, float dt, float* ms);

/* Allocation-free FP64 elastic energy (no counterpart entry point in the reference; its CPU
 * materials' get_energy, FEM_ContinuousMaterial.cpp:10-87, give the densities).  For callers that must not allocate device memory when they call
 * it: a host application whose device memory belongs to its own pool and which forbids
 * driver allocations inside its frame loop, or a real-time loop that cannot take the
 * latency and implicit synchronisation of cudaMalloc/cudaFree.  Computes
 * sum_e sum_q Psi(F) |det J| w_q in FP64 from device positions and rest positions
 * (n_nodes*3 floats each) and the device topology, writing one double to d_out, in a fixed
 * summation order (the same bits on every call).  Intermediate storage is a static
 * per-device array of one double per element, at most 1 << 20 elements (8 MiB); larger
 * meshes are rejected with OCT_EINVAL.  Calls that overlap on the GPU race on that array.
 * The first call on a device sets it up (takes the array's device address, uploads the
 * Hexa_27 tables) and should come before any stream capture.  stream: a cudaStream_t, or
 * NULL for the default stream.  Nothing is allocated. */
oct_status oct_elastic_energy_noalloc(int element, int material, const float* d_positions, const float* d_rest_positions,
                                      const int32_t* d_topology, int n_elements, float young, float poisson,
                                      double* d_out, void* stream);

/* Device timing of the last oct_scene_step / oct_batch_step (ms, CUDA events). */
oct_status oct_last_step_ms(oct_ctx* ctx, float* ms);
/* Number of kernel launches issued by this context since creation. */
oct_status oct_launch_count(oct_ctx* ctx, uint64_t* n);

#ifdef __cplusplus
}
#endif
#endif
