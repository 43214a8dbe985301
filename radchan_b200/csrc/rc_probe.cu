// rc_probe.cu -- the gather-throughput probe that the march kernel's
// roofline is stated against (rc_probe_gather, radchan.h).
//
// Each step of the march reads one 4-byte temperature coordinate from a
// cell that neighbouring lanes do not share, so the memory system serves it
// as one 32-byte sector; at the benchmark's sizes the temperature pyramid
// and the tables (about 1.4 MB at 64^3) stay resident in L2 (126 MB), and
// HBM is idle.  The ceiling for that access pattern is therefore the rate
// at which L2 (or L1 + L2) serves random 32-byte sectors, not the HBM copy
// bandwidth.  The probe measures it: every lane reads 4 bytes from a
// pseudo-random sector of an array of the given size, eight independent
// reads in flight per lane, at full occupancy on every SM.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "radchan.h"

namespace {

constexpr int kProbeBlock = 256;
constexpr int kProbeUnroll = 8;

// mode 0: ld.global.cg (L2 only); mode 1: ld.global.nc (read-only path
// through L1, as the march reads its pyramid and tables).
template <int MODE>
__global__ void __launch_bounds__(kProbeBlock) k_gather_probe(const float *__restrict__ a, uint32_t nsect,
                                                              int iters, float *sink) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t x = tid * 2654435761u + 12345u;
    float acc = 0.f;
    for (int it = 0; it < iters; ++it) {
        uint32_t idx[kProbeUnroll];
#pragma unroll
        for (int u = 0; u < kProbeUnroll; ++u) {
            x = x * 1664525u + 1013904223u;
            // sector by multiply-high (uniform over [0, nsect)), word in it
            idx[u] = __umulhi(x, nsect) * 8u + ((x >> 7) & 7u);
        }
        float v[kProbeUnroll];
#pragma unroll
        for (int u = 0; u < kProbeUnroll; ++u) v[u] = MODE == 0 ? __ldcg(a + idx[u]) : __ldg(a + idx[u]);
#pragma unroll
        for (int u = 0; u < kProbeUnroll; ++u) acc += v[u];
    }
    sink[tid] = acc;
}

int g_probe_err(std::string *msg, const char *what, cudaError_t e) {
    if (msg) *msg = std::string(what) + ": " + cudaGetErrorString(e);
    return RC_E_CUDA;
}

}  // namespace

extern "C" int rc_probe_gather(int device, size_t bytes, int mode, int iters, double *sectors_per_s,
                               float *ms_best) {
    if (bytes < 4096 || bytes > ((size_t)1 << 33) || (mode != 0 && mode != 1) || iters < 1 || !sectors_per_s)
        return RC_E_INVALID;
    std::string msg;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return g_probe_err(&msg, "cudaSetDevice", e);
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    const int blocks = nsm * (2048 / kProbeBlock);
    const uint32_t nsect = (uint32_t)(bytes / 32);
    float *a = nullptr, *sink = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = RC_OK;
    float best = 0.f;
    auto fail = [&](const char *what, cudaError_t err) {
        rc = g_probe_err(&msg, what, err);
    };
    if ((e = cudaMalloc((void **)&a, (size_t)nsect * 32)) != cudaSuccess) fail("cudaMalloc", e);
    if (!rc && (e = cudaMalloc((void **)&sink, (size_t)blocks * kProbeBlock * sizeof(float))) != cudaSuccess)
        fail("cudaMalloc", e);
    if (!rc && (e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) fail("stream", e);
    if (!rc && (e = cudaEventCreate(&e0)) != cudaSuccess) fail("event", e);
    if (!rc && (e = cudaEventCreate(&e1)) != cudaSuccess) fail("event", e);
    if (!rc && (e = cudaMemsetAsync(a, 0x3c, (size_t)nsect * 32, st)) != cudaSuccess) fail("memset", e);
    for (int rep = 0; !rc && rep < 4; ++rep) {
        // the first launch warms the array into the caches; the best of
        // the following three is reported
        cudaEventRecord(e0, st);
        if (mode == 0) k_gather_probe<0><<<blocks, kProbeBlock, 0, st>>>(a, nsect, iters, sink);
        else k_gather_probe<1><<<blocks, kProbeBlock, 0, st>>>(a, nsect, iters, sink);
        cudaEventRecord(e1, st);
        if ((e = cudaGetLastError()) != cudaSuccess) {
            fail("k_gather_probe", e);
            break;
        }
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) {
            fail("k_gather_probe", e);
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    if (!rc) {
        const double loads = (double)blocks * kProbeBlock * iters * kProbeUnroll;
        *sectors_per_s = loads / (best / 1000.0);
        if (ms_best) *ms_best = best;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (a) cudaFree(a);
    if (sink) cudaFree(sink);
    return rc;
}
