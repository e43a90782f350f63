// dsmc_trace_noalloc: the tracing check of dsmc_trace for callers that must
// not allocate device memory.
//
// Some hosts cannot call cudaMalloc at the point where they want to run a
// check: a solver that reserved the whole device up front for its own memory
// pool, or a coupling loop that forbids allocation after start-up so its
// memory footprint stays fixed. dsmc_trace stages its host arrays in device
// buffers it allocates for each call; this variant stages them in one
// file-scope device array instead, so the call makes no device allocation.
// Its messages are formatted into a fixed buffer; no C++ exception leaves it.
#include "dsmc_gpu.h"
#include "dsmc_kernels.cuh"

#include <cstdio>
#include <cstring>
#include <mutex>

namespace dsmc {
DevMesh engine_mesh(const DsmcHandle* h);
DevConsts engine_consts(const DsmcHandle* h);
int engine_precision(const DsmcHandle* h);
int engine_device(const DsmcHandle* h);
cudaStream_t engine_stream(const DsmcHandle* h);
unsigned long long* engine_counters(const DsmcHandle* h);
void engine_set_error(DsmcHandle* h, const char* msg) noexcept;
}  // namespace dsmc

namespace {

// Per particle: px,py,pz,vx,vy,vz,dt in (7 doubles), cell in, 6 int outputs
// (cell, ifout, face, tri, ncross, last cell), 6 working reals in and out
// (as doubles at most), 7 doubles out (px..vz, dt).
constexpr size_t kPerParticle = 7 * 8 + 4 + 6 * 4 + 6 * 8 + 6 * 8 + 7 * 8;
constexpr size_t kScratchBytes = (size_t)DSMC_NOALLOC_MAX_TRACE * kPerParticle + 4096;

// Shared by every call on a device; each GPU that loads the library keeps
// it until the process exits.
static __device__ __align__(256) unsigned char g_trace_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
unsigned char* g_scratchPtr[kMaxDevices] = {};

void set_cuda_error(DsmcHandle* h, const char* what, cudaError_t e) noexcept
{
    char msg[256];
    std::snprintf(msg, sizeof msg, "dsmc_trace_noalloc: %s: %s", what, cudaGetErrorString(e));
    dsmc::engine_set_error(h, msg);
}

// The address of g_trace_scratch as a device pointer, found once per device
// with that device current (the host-side name of the array is only a
// stand-in and must not be passed to a kernel).
cudaError_t scratch_for_device(int dev, unsigned char** out) noexcept
{
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::unique_lock<std::mutex> lock(g_setupMutex, std::defer_lock);
    try {
        lock.lock();
    } catch (...) {
        return cudaErrorUnknown;
    }
    if (!g_scratchPtr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_trace_scratch);
        if (e != cudaSuccess) return e;
        g_scratchPtr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratchPtr[dev];
    return cudaSuccess;
}

// absolute FP64 input -> the precision's particle representation
__global__ void to_working(int n, const double* in, const int* cell, const double* center, int mixed, void* work)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int k = 0; k < 6; ++k) {
            double v = in[(size_t)k * n + i];
            if (mixed) {
                if (k < 3) v -= center[(size_t)cell[i] * 3 + k];
                static_cast<float*>(work)[(size_t)k * n + i] = (float)v;
            } else {
                static_cast<double*>(work)[(size_t)k * n + i] = v;
            }
        }
    }
}

// the precision's output -> absolute FP64
__global__ void from_working(int n, const void* work, const int* last, const double* center, int mixed, double* out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int k = 0; k < 6; ++k) {
            double v = mixed ? (double)static_cast<const float*>(work)[(size_t)k * n + i]
                             : static_cast<const double*>(work)[(size_t)k * n + i];
            if (mixed && k < 3) v = center[(size_t)last[i] * 3 + k] + v;
            out[(size_t)k * n + i] = v;
        }
    }
}

}  // namespace

extern "C" int dsmc_trace_noalloc(DsmcHandle* h, int64_t n, const double* px, const double* py, const double* pz,
                                  const double* vx, const double* vy, const double* vz, const double* dt,
                                  const int32_t* cell, int32_t stop_at_wall, int32_t* out_cell, int32_t* out_ifout,
                                  int32_t* out_face, int32_t* out_tri, int32_t* out_ncross, double* out_px,
                                  double* out_py, double* out_pz, double* out_vx, double* out_vy, double* out_vz,
                                  double* out_dt)
{
    if (!h) return DSMC_E_INVALID;
    if (n < 0 || n > DSMC_NOALLOC_MAX_TRACE) {
        dsmc::engine_set_error(h, "dsmc_trace_noalloc: n must be between 0 and DSMC_NOALLOC_MAX_TRACE (32768)");
        return DSMC_E_INVALID;
    }
    if (n == 0) return DSMC_OK;
    if (!px || !py || !pz || !vx || !vy || !vz || !dt || !cell) {
        dsmc::engine_set_error(h, "dsmc_trace_noalloc: null input array");
        return DSMC_E_INVALID;
    }
    const dsmc::DevMesh M = dsmc::engine_mesh(h);
    for (int64_t i = 0; i < n; ++i)
        if (cell[i] < 0 || cell[i] >= M.ncell) {
            dsmc::engine_set_error(h, "dsmc_trace_noalloc: cell id out of range");
            return DSMC_E_INVALID;
        }
    const int dev = dsmc::engine_device(h);
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) {
        set_cuda_error(h, "cudaSetDevice", e);
        return DSMC_E_CUDA;
    }
    unsigned char* base = nullptr;
    e = scratch_for_device(dev, &base);
    if (e != cudaSuccess) {
        set_cuda_error(h, "cudaGetSymbolAddress", e);
        return DSMC_E_CUDA;
    }
    const int ni = (int)n;
    const size_t N = (size_t)ni;
    // carve the scratch (every region 256-byte aligned)
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += (bytes + 255) & ~(size_t)255;
        return p;
    };
    double* dIn = reinterpret_cast<double*>(take(7 * N * 8));      // px..vz, dt
    int* dCell = reinterpret_cast<int*>(take(N * 4));
    int* dOutI = reinterpret_cast<int*>(take(6 * N * 4));          // cell, ifout, face, tri, ncross, last
    void* dWorkIn = take(6 * N * 8);
    void* dWorkOut = take(6 * N * 8);
    double* dOut = reinterpret_cast<double*>(take(7 * N * 8));     // px..vz, dt
    if (off > kScratchBytes) {
        dsmc::engine_set_error(h, "dsmc_trace_noalloc: scratch layout exceeds its size");
        return DSMC_E_INVALID;
    }
    const int mixed = dsmc::engine_precision(h) == DSMC_PRECISION_MIXED;
    const dsmc::DevConsts Cst = dsmc::engine_consts(h);
    cudaStream_t s = dsmc::engine_stream(h);
    const double* src[7] = {px, py, pz, vx, vy, vz, dt};
    for (int k = 0; k < 7 && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(dIn + (size_t)k * N, src[k], N * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dCell, cell, N * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        const int g = (ni + 255) / 256 < 1024 ? (ni + 255) / 256 : 1024;
        to_working<<<g, 256, 0, s>>>(ni, dIn, dCell, M.cellCenter, mixed, dWorkIn);
        int* oi[6];
        for (int k = 0; k < 6; ++k) oi[k] = dOutI + (size_t)k * N;
        if (mixed) {
            const float* wi = static_cast<const float*>(dWorkIn);
            float* wo = static_cast<float*>(dWorkOut);
            dsmc::launch_trace_check<float>(M, Cst, ni, wi, wi + N, wi + 2 * N, wi + 3 * N, wi + 4 * N, wi + 5 * N,
                                            dIn + 6 * N, dCell, stop_at_wall, oi[0], oi[1], oi[2], oi[3], oi[4], oi[5],
                                            wo, wo + N, wo + 2 * N, wo + 3 * N, wo + 4 * N, wo + 5 * N, dOut + 6 * N,
                                            dsmc::engine_counters(h), s);
        } else {
            const double* wi = static_cast<const double*>(dWorkIn);
            double* wo = static_cast<double*>(dWorkOut);
            dsmc::launch_trace_check<double>(M, Cst, ni, wi, wi + N, wi + 2 * N, wi + 3 * N, wi + 4 * N, wi + 5 * N,
                                             dIn + 6 * N, dCell, stop_at_wall, oi[0], oi[1], oi[2], oi[3], oi[4], oi[5],
                                             wo, wo + N, wo + 2 * N, wo + 3 * N, wo + 4 * N, wo + 5 * N, dOut + 6 * N,
                                             dsmc::engine_counters(h), s);
        }
        from_working<<<g, 256, 0, s>>>(ni, dWorkOut, oi[5], M.cellCenter, mixed, dOut);
        e = cudaGetLastError();
    }
    int32_t* hi[5] = {out_cell, out_ifout, out_face, out_tri, out_ncross};
    for (int k = 0; k < 5 && e == cudaSuccess; ++k)
        if (hi[k]) e = cudaMemcpyAsync(hi[k], dOutI + (size_t)k * N, N * 4, cudaMemcpyDeviceToHost, s);
    double* hd[7] = {out_px, out_py, out_pz, out_vx, out_vy, out_vz, out_dt};
    for (int k = 0; k < 7 && e == cudaSuccess; ++k)
        if (hd[k]) e = cudaMemcpyAsync(hd[k], dOut + (size_t)k * N, N * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_cuda_error(h, "copy or launch", e);
        return DSMC_E_CUDA;
    }
    return DSMC_OK;
}
