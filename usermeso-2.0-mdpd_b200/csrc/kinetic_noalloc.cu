// Kinetic sums over caller-owned device arrays without any allocation.
//
// Who needs this: a host code that already owns every byte it wants on the device and calls
// into this library from inside its own timestep -- e.g. a LAMMPS fix or compute whose atoms
// live in USER-MESO-style device arrays, or an application whose caching allocator or fixed
// HBM arena has reserved the device memory. Such callers cannot let the library call
// cudaMalloc/cudaFree: those calls synchronise the whole device (stalling the caller's own
// streams in the middle of its step) and fail outright when the caller's pool holds the
// memory. The thermo entry points of a handle (mdpd_thermo, mdpd_batch_thermo) reduce into
// buffers allocated with the handle; this entry point instead keeps its per-block partial
// sums in one fixed device array, g_kin_scratch below, that the library holds for the life
// of the process on every GPU it is loaded on.
//
// The reduction is the same two-stage, fixed-order FP64 sum as the handle's thermo
// (per-block partials, then one block summing them in block order), so results do not depend
// on scheduling and are identical from call to call.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "mdpd.h"

namespace {

constexpr int kThreads = 256;                                   // threads per block
constexpr int kPerThread = 4;                                   // particles per thread
constexpr int kChunk = kThreads * kPerThread;                   // particles per block
constexpr int64_t kMaxParticles = int64_t(1) << 24;             // 16,777,216 per call
constexpr int kMaxChunks = (int)(kMaxParticles / kChunk);       // 16,384 partial rows
constexpr int kSums = 11;                                       // doubles per row
constexpr int kMaxDevices = 64;

// Per-block partial rows [kMaxChunks][kSums] followed by one row of totals:
// (16,384 + 1) x 11 doubles = 1.44 MB of device memory per GPU, held until the process exits.
// Nothing here has to start at zero: every call writes each partial row it later reads and
// then writes the totals row, so what a previous call left behind is never read.
static __device__ __align__(256) double g_kin_scratch[(kMaxChunks + 1) * kSums];

__global__ void __launch_bounds__(kThreads)
k_kinetic_chunks(const double *__restrict__ vx, const double *__restrict__ vy,
                 const double *__restrict__ vz, const double *__restrict__ mass,
                 const int32_t *__restrict__ mask, int32_t groupbit, int n, double *__restrict__ rows)
{
    __shared__ double s_red[kThreads / 32][kSums];
    double a[kSums];
#pragma unroll
    for (int q = 0; q < kSums; ++q) a[q] = 0.0;
    const int base = blockIdx.x * kChunk + threadIdx.x;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int i = base + k * kThreads;
        if (i < n && (!mask || (mask[i] & groupbit))) {
            const double m = mass[i], x = vx[i], y = vy[i], z = vz[i];
            a[0] += m * (x * x + y * y + z * z);
            a[1] += m * x, a[2] += m * y, a[3] += m * z;
            a[4] += m * x * x, a[5] += m * y * y, a[6] += m * z * z;
            a[7] += m * x * y, a[8] += m * x * z, a[9] += m * y * z;
            a[10] += 1.0;
        }
    }
#pragma unroll
    for (int q = 0; q < kSums; ++q)
        for (int o = 16; o > 0; o >>= 1) a[q] += __shfl_down_sync(0xffffffffu, a[q], o);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int q = 0; q < kSums; ++q) s_red[threadIdx.x / 32][q] = a[q];
    __syncthreads();
    if (threadIdx.x < kSums) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += s_red[w][threadIdx.x];
        rows[(size_t)blockIdx.x * kSums + threadIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kThreads) k_kinetic_total(int nchunk, double *__restrict__ rows)
{
    // one block: strided sums over the partial rows, then a fixed tree
    __shared__ double s[kThreads];
    for (int q = 0; q < kSums; ++q) {
        double t = 0.0;
        for (int c = threadIdx.x; c < nchunk; c += kThreads) t += rows[(size_t)c * kSums + q];
        s[threadIdx.x] = t;
        __syncthreads();
        for (int w = kThreads / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) rows[(size_t)kMaxChunks * kSums + q] = s[0];
        __syncthreads();
    }
}

std::mutex g_setup_mu;
double *g_scratch_ptr[kMaxDevices] = {};

int fail(char *err, int64_t err_len, int code, const char *msg)
{
    if (err && err_len > 0) {
        std::strncpy(err, msg, (size_t)err_len - 1);
        err[err_len - 1] = '\0';
    }
    return code;
}

int fail_cuda(char *err, int64_t err_len, const char *what, cudaError_t e)
{
    char buf[256];
    std::snprintf(buf, sizeof buf, "mdpd_kinetic_sums_noalloc: %s: %s", what, cudaGetErrorString(e));
    return fail(err, err_len, MDPD_ERR_CUDA, buf);
}

// The device address of g_kin_scratch on the current device. Host code must not pass
// g_kin_scratch itself to a kernel: on the host that name is only a stand-in for the device
// symbol, so a kernel given it would fault or, where the GPU can reach host memory, silently
// read and write the wrong memory. The address is looked up once per device, with that
// device current, and cached for the life of the process (a cudaDeviceReset by the host
// application invalidates it: the symbol may then live elsewhere).
cudaError_t scratch_for_current_device(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_kin_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

bool on_device(const void *p, int dev)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // do not leave this query's error for the next caller to find
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" int mdpd_kinetic_sums_noalloc(const double *vx, const double *vy, const double *vz,
                                         const double *mass, const int32_t *mask, int32_t groupbit,
                                         int64_t n, void *stream, double *sums, char *err,
                                         int64_t err_len)
{
    if (err && err_len > 0) err[0] = '\0';
    if (!sums) return fail(err, err_len, MDPD_ERR_ARG, "mdpd_kinetic_sums_noalloc: sums is NULL");
    if (n < 0) return fail(err, err_len, MDPD_ERR_ARG, "mdpd_kinetic_sums_noalloc: n < 0");
    if (n > kMaxParticles) {
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "mdpd_kinetic_sums_noalloc: n = %lld exceeds the %lld particles its fixed "
                      "device scratch holds; split the arrays or use mdpd_thermo",
                      (long long)n, (long long)kMaxParticles);
        return fail(err, err_len, MDPD_ERR_ARG, buf);
    }
    for (int q = 0; q < kSums; ++q) sums[q] = 0.0;
    if (n == 0) return MDPD_OK;
    if (!vx || !vy || !vz || !mass)
        return fail(err, err_len, MDPD_ERR_ARG, "mdpd_kinetic_sums_noalloc: NULL input array");

    double *rows = nullptr;
    cudaError_t e = scratch_for_current_device(&rows);
    if (e != cudaSuccess) return fail_cuda(err, err_len, "cudaGetSymbolAddress", e);
    int dev = 0;
    cudaGetDevice(&dev);
    const void *ins[5] = {vx, vy, vz, mass, mask};
    for (int k = 0; k < 5; ++k)
        if (ins[k] && !on_device(ins[k], dev))
            return fail(err, err_len, MDPD_ERR_ARG,
                        "mdpd_kinetic_sums_noalloc: input arrays must be device memory of the "
                        "current device");

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the call ends by copying to pageable host memory and synchronising its stream, which a
    // stream under capture cannot do: refuse rather than invalidate the caller's capture
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(s, &cap)) != cudaSuccess) return fail_cuda(err, err_len, "stream query", e);
    if (cap != cudaStreamCaptureStatusNone)
        return fail(err, err_len, MDPD_ERR_ARG,
                    "mdpd_kinetic_sums_noalloc: the stream is being captured; call it outside any capture");
    const int nchunk = (int)((n + kChunk - 1) / kChunk);
    k_kinetic_chunks<<<nchunk, kThreads, 0, s>>>(vx, vy, vz, mass, mask, groupbit, (int)n, rows);
    k_kinetic_total<<<1, kThreads, 0, s>>>(nchunk, rows);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail_cuda(err, err_len, "launch", e);
    e = cudaMemcpyAsync(sums, rows + (size_t)kMaxChunks * kSums, sizeof(double) * kSums,
                        cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return fail_cuda(err, err_len, "copy of the sums", e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail_cuda(err, err_len, "stream", e);
    return MDPD_OK;
}
