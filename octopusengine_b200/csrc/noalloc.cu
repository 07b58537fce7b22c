// Allocation-free FP64 elastic energy of a mesh state.
//
// Some callers cannot allocate device memory at the moment they need a diagnostic: a host
// application whose device memory is owned by its own pool allocator and which forbids
// driver allocations inside its frame loop, or a real-time loop that cannot take the
// latency and implicit synchronisation of cudaMalloc/cudaFree.  oct_elastic_energy_noalloc
// serves them: the caller passes device inputs and a device output, and the only
// intermediate storage is the file-scope array below.
//
// The computation is the elastic part of oct_scene_energy (sum over elements and
// quadrature points of Psi(F) V, FP64), made deterministic: each element's energy goes to
// its own scratch slot and one block sums the slots in a fixed order, so repeated calls on
// the same state return the same bits.
//
// Scratch: g_energy_scratch holds one double per element, kNoAllocMaxElements of them
// (8 MiB); every device that loads this library keeps it until the process exits.  Calls
// with more elements are rejected with OCT_EINVAL.  All calls share the array and every
// call overwrites the slots it reads, so nothing needs clearing between calls, but two
// calls that overlap on the GPU (different streams, or different host threads on one
// device) race on it: order them on one stream or serialise them.
//
// Set-up: the first call on a device, with that device current, takes the array's device
// address with cudaGetSymbolAddress (the host-side symbol is only a stand-in, not a device
// address) and uploads the Hexa_27 derivative table to constant memory.  That first call
// should therefore come before any stream capture.
#include <mutex>

#include "../../include/octopus_b200.h"
#include "shape_tables.inc"

namespace {

constexpr int kNoAllocMaxElements = 1 << 20;
__device__ __align__(256) double g_energy_scratch[kNoAllocMaxElements];
__constant__ float c_noalloc_dN9[27 * 27 * 3];
__constant__ float c_noalloc_w9[27];

template <int E> struct Nodes;
template <> struct Nodes<3> { static constexpr int NE = 4, NQ = 1; };
template <> struct Nodes<6> { static constexpr int NE = 8, NQ = 8; };
template <> struct Nodes<7> { static constexpr int NE = 10, NQ = 4; };
template <> struct Nodes<8> { static constexpr int NE = 20, NQ = 11; };
template <> struct Nodes<9> { static constexpr int NE = 27, NQ = 27; };

template <int E> __device__ __forceinline__ double dnq(int q, int i, int k) {
    if constexpr (E == 9) return c_noalloc_dN9[(q * 27 + i) * 3 + k];
    else return octb::ShapeConst<E>::dN((q * Nodes<E>::NE + i) * 3 + k);
}
template <int E> __device__ __forceinline__ double wqq(int q) {
    if constexpr (E == 9) return c_noalloc_w9[q];
    else return octb::ShapeConst<E>::w(q);
}

__device__ __forceinline__ double det3(const double m[3][3]) {   // m[col][row]
    return m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
           m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
}

// Energy density of the reference materials (FEM_ContinuousMaterial.cpp:10-15,31-36,70-74,83-87).
__device__ double psi(int material, double lam, double mu, const double F[3][3]) {
    if (material == 2 || material == 3) {
        double n2 = 0;
        for (int b = 0; b < 3; ++b) for (int r = 0; r < 3; ++r) n2 += F[b][r] * F[b][r];
        const double d = det3(F) - (material == 3 ? 1.0 + mu / lam : 1.0);
        return 0.5 * mu * (n2 - 3.0) + 0.5 * lam * d * d;
    }
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
    return 0.5 * lam * tr * tr + mu * n2;
}

template <int E>
__global__ void k_element_energy(const float* __restrict__ p, const float* __restrict__ X, const int* __restrict__ topo,
                                 int n_elements, int material, double lam, double mu, double* __restrict__ scratch) {
    constexpr int NE = Nodes<E>::NE, NQ = Nodes<E>::NQ;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_elements; e += gridDim.x * blockDim.x) {
        const int* t = topo + (size_t)e * NE;
        double sum = 0.0;
#pragma unroll (E == 9 ? 1 : NQ)
        for (int q = 0; q < NQ; ++q) {
            double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Jx[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll (E == 9 ? 1 : NE)
            for (int i = 0; i < NE; ++i) {
                const float* x = X + 3 * (size_t)t[i];
                const float* y = p + 3 * (size_t)t[i];
                for (int c = 0; c < 3; ++c) {
                    const double d = dnq<E>(q, i, c);
                    for (int r = 0; r < 3; ++r) { J[c][r] += (double)x[r] * d; Jx[c][r] += (double)y[r] * d; }
                }
            }
            const double dj = det3(J), id = 1.0 / dj;
            double I[3][3];   // J^-1, I[col][row]
            I[0][0] = (J[1][1] * J[2][2] - J[2][1] * J[1][2]) * id;
            I[1][0] = -(J[1][0] * J[2][2] - J[2][0] * J[1][2]) * id;
            I[2][0] = (J[1][0] * J[2][1] - J[2][0] * J[1][1]) * id;
            I[0][1] = -(J[0][1] * J[2][2] - J[2][1] * J[0][2]) * id;
            I[1][1] = (J[0][0] * J[2][2] - J[2][0] * J[0][2]) * id;
            I[2][1] = -(J[0][0] * J[2][1] - J[2][0] * J[0][1]) * id;
            I[0][2] = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * id;
            I[1][2] = -(J[0][0] * J[1][2] - J[1][0] * J[0][2]) * id;
            I[2][2] = (J[0][0] * J[1][1] - J[1][0] * J[0][1]) * id;
            double F[3][3];   // F = Jx J^-1, F[col][row]
            for (int b = 0; b < 3; ++b)
                for (int r = 0; r < 3; ++r) F[b][r] = Jx[0][r] * I[b][0] + Jx[1][r] * I[b][1] + Jx[2][r] * I[b][2];
            sum += psi(material, lam, mu, F) * fabs(dj) * wqq<E>(q);
        }
        scratch[e] = sum;
    }
}

// Fixed-order sum of scratch[0, n): thread k adds slots k, k + 1024, ... then a shared-memory
// tree over the 1024 partial sums.
__global__ void k_fixed_order_sum(const double* __restrict__ scratch, int n, double* __restrict__ out) {
    __shared__ double s[1024];
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += 1024) v += scratch[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

std::mutex g_setup_mu;
double* g_scratch_addr[64] = {nullptr};

// Once per device, with that device current: the scratch array's device address and the
// Hexa_27 tables.
cudaError_t setup_device(int dev, double** addr) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!g_scratch_addr[dev]) {
        void* a = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&a, g_energy_scratch);
        if (e != cudaSuccess) return e;
        float dN9[27 * 27 * 3], w9[27];
        for (int k = 0; k < 27 * 27 * 3; ++k) dN9[k] = octb::ShapeConst<9>::dN(k);
        for (int q = 0; q < 27; ++q) w9[q] = octb::ShapeConst<9>::w(q);
        if ((e = cudaMemcpyToSymbol(c_noalloc_dN9, dN9, sizeof(dN9))) != cudaSuccess) return e;
        if ((e = cudaMemcpyToSymbol(c_noalloc_w9, w9, sizeof(w9))) != cudaSuccess) return e;
        g_scratch_addr[dev] = (double*)a;
    }
    *addr = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" oct_status oct_elastic_energy_noalloc(int element, int material, const float* d_positions,
                                                 const float* d_rest_positions, const int32_t* d_topology, int n_elements,
                                                 float young, float poisson, double* d_out, void* stream) {
    if (!d_positions || !d_rest_positions || !d_topology || !d_out || n_elements <= 0) return OCT_EINVAL;
    if (n_elements > kNoAllocMaxElements) return OCT_EINVAL;   // beyond the static scratch
    if (material < 0 || material > 3) return OCT_EINVAL;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return OCT_ECUDA;
    double* scratch = nullptr;
    if (setup_device(dev, &scratch) != cudaSuccess) return OCT_ECUDA;
    const double Y = young, nu = poisson;
    const double lam = Y * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = Y / (2.0 * (1.0 + nu));
    cudaStream_t st = (cudaStream_t)stream;
    const int threads = 128, blocks = (n_elements + threads - 1) / threads < 4096 ? (n_elements + threads - 1) / threads : 4096;
    // a launch error left on this thread by an earlier call is not this call's failure: clear
    // it so the checks after the launches see only their own
    (void)cudaGetLastError();
    switch (element) {
        case 3: k_element_energy<3><<<blocks, threads, 0, st>>>(d_positions, d_rest_positions, d_topology, n_elements, material, lam, mu, scratch); break;
        case 6: k_element_energy<6><<<blocks, threads, 0, st>>>(d_positions, d_rest_positions, d_topology, n_elements, material, lam, mu, scratch); break;
        case 7: k_element_energy<7><<<blocks, threads, 0, st>>>(d_positions, d_rest_positions, d_topology, n_elements, material, lam, mu, scratch); break;
        case 8: k_element_energy<8><<<blocks, threads, 0, st>>>(d_positions, d_rest_positions, d_topology, n_elements, material, lam, mu, scratch); break;
        case 9: k_element_energy<9><<<blocks, threads, 0, st>>>(d_positions, d_rest_positions, d_topology, n_elements, material, lam, mu, scratch); break;
        default: return OCT_EINVAL;
    }
    if (cudaGetLastError() != cudaSuccess) return OCT_ECUDA;
    k_fixed_order_sum<<<1, 1024, 0, st>>>(scratch, n_elements, d_out);
    return cudaGetLastError() == cudaSuccess ? OCT_OK : OCT_ECUDA;
}
