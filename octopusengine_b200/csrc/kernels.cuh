// Host-callable launchers of the kernels in kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include "device.cuh"

namespace octb {

cudaError_t upload_shape_tables(int element, const float* dN, int n_floats);
cudaError_t upload_shape_tables_fp64(int element, const double* dN, int n, const double* w, int nq);
// Caches the persistent grid size of the vertex kernel for (element, material); call
// outside stream capture.
void prepare_vertex(int element, int material);
// mode 0: VBD solve, 1: VBD residual (red[0] += |r|, red[1] = max |r|), 2: explicit force
void launch_vertex(int element, int material, const SceneDev* scenes, const VWork* work, int n_work, int tpv, int mode,
                   const StepParams& P, double* red, cudaStream_t st);
void launch_commit(const SceneDev* scenes, const VWork* work, int n_work, cudaStream_t st);
// Explicit sub-step without the constraints: the element-centric force pass (per-(element,
// local node) contributions into contrib, n_elements x NE float4), then per node the sum over
// its owners into u_new and the semi-implicit Euler update (slots: node chunks over the
// scene's slots).
void launch_explicit_force(int element, int material, const SceneDev* scene, int n_elements, float4* contrib,
                           const NWork* slots, int n_slots, const StepParams& P, cudaStream_t st);
// kind 0: VBD predictor, kind 1: semi-implicit Euler (use_force: add the force in u_new)
void launch_predict(const SceneDev* scenes, const NWork* work, int n_work, int kind, int use_force, int chebyshev,
                    const StepParams& P, cudaStream_t st);
// pbd: the GPU_PBD velocity update with each scene's global damping
void launch_velocity(const SceneDev* scenes, const NWork* work, int n_work, int pbd, const StepParams& P,
                     cudaStream_t st);
void launch_chebyshev(const SceneDev* scenes, const NWork* work, int n_work, const StepParams& P, cudaStream_t st);
// box_pass 0: work indexes fixed-id chunks; 1: work indexes node chunks (box clamp)
void launch_constraints(const SceneDev* scenes, const NWork* work, int n_work, int box_pass, cudaStream_t st);
// Multigrid VBD: corner copy between a scene and its linear level (dir 0 gather, 1 scatter)
// and the prolongation of mid nodes from k corners with weight w.
void launch_mg_copy(const SceneDev* main, const SceneDev* sub, const int* map, int n, int dir, cudaStream_t st);
void launch_mg_prolong(const SceneDev* main, const int* list, int count, int k, float w, cudaStream_t st);
// Node state as the reference's n x 3 float arrays: out = src (+ X when X is given) and
// dst = in (- X when X is given), w = 0.
void launch_nodes_out(const float4* src, const float4* X, float* out, int n, cudaStream_t st);
void launch_nodes_in(const float* in, const float4* X, float4* dst, int n, cudaStream_t st);
// Failure-detection probe: a bounded wait on a phase nothing completes (error bit 0 on time-out).
void launch_wait_probe(int* error, long limit, cudaStream_t st);
// One scripted effect of one scene (kind 0 crush / 1 random sphere over the node chunks in
// work, kind 2 high stretch over its ids); a no-op while the effect is inactive.
void launch_effect(const SceneDev* scene, const NWork* work, int n_work, int slot, int kind, float dt, cudaStream_t st);
// raw: the kernel_XPBD_V1/V2 update form (ignored for Tetra4, which always uses V0); one block
// per work item (xpbd_elements_per_block elements of one scene's colour)
void launch_xpbd(int element, int material, bool raw, const SceneDev* scenes, const XWork* work, int n_work,
                 const StepParams& P, cudaStream_t st);
int xpbd_elements_per_block(int element);
// Per-element diagnostics of GPU_FEM (kind 0 stress, 1 volume, 2 volume change, 3 inverted,
// 4 stress with the reference kernel's accumulated Jx).
void launch_element_diag(int element, int material, const SceneDev* scenes, int scene, int n_elements, int kind, float* out,
                         cudaStream_t st);
void launch_energy(int element, int material, const SceneDev* scenes, int scene, int n_nodes, int n_elements, double* out,
                   int* error, cudaStream_t st);

// Batch host-state staging: dir 0 scatters state into u/v, dir 1 gathers u/v into state.
void launch_state(const SceneDev* scenes, const NWork* work, int n_work, const long long* soff, float* state, int dir,
                  cudaStream_t st);
// FP32 FMA microbenchmark: returns the number of FMAs issued by the launch.
double launch_fma_peak(cudaStream_t st);
// Algorithmic FP32 flops of one (owner, quadrature point) term of the VBD kernel.
double vbd_term_flops(int element, int material);

}  // namespace octb
