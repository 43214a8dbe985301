// ref_driver.cu -- calls the reference's own entry points (mc_gpu_ then
// get_results_, src/montecarlo/mc_gpu_noint.cu:660, :876) from a C ABI that
// ctypes can load.  Compiled together with the reference's sources by
// oracle/ref_build.py; used only to produce the statistical parity fixtures
// under tests/golden/ (the reference resets the device in get_results_, so it
// always runs in a process of its own).
#include <cuda_runtime.h>

#include <chrono>

extern "C" void mc_gpu_(float *Tfort, int *zstart, int *rank);
extern "C" void get_results_(float *resfort, float *varfort, int *rank);

extern "C" int ref_solve(float *T, int zstart, float *Q, float *sigma, double *ms) {
    int z = zstart, rank = 0;
    auto t0 = std::chrono::steady_clock::now();
    mc_gpu_(T, &z, &rank);
    get_results_(Q, sigma, &rank);
    auto t1 = std::chrono::steady_clock::now();
    if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return (int)cudaGetLastError();
}
