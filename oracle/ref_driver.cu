// ref_driver.cu -- calls the reference's own entry points (mc_gpu_ then
// get_results_, src/montecarlo/mc_gpu_noint.cu:660, :876) from a C ABI that
// ctypes can load.  Compiled together with the reference's sources by
// oracle/ref_build.py; used to produce the statistical parity fixtures under
// tests/golden/ and to time the reference's CUDA build next to this solver
// (bench.py's reference arm).  The reference resets the device in
// get_results_, so it always runs in a process of its own.
#include <cuda_runtime.h>

#include <chrono>

extern "C" void mc_gpu_(float *Tfort, int *zstart, int *rank);
extern "C" void get_results_(float *resfort, float *varfort, int *rank);

// ms[0]: mc_gpu_ + get_results_ wall time; ms[1]: mc_gpu_ alone (table
// files read, uploads, launches; it returns with the kernels in flight);
// ms[2]: from mc_gpu_'s return until the device is idle (the kernels that
// were still running); ms[3]: get_results_ (copies, scatter, device reset).
extern "C" int ref_solve_timed(float *T, int zstart, float *Q, float *sigma, double *ms) {
    int z = zstart, rank = 0;
    using clk = std::chrono::steady_clock;
    auto d = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    auto t0 = clk::now();
    mc_gpu_(T, &z, &rank);
    auto t1 = clk::now();
    cudaError_t e = cudaDeviceSynchronize();
    auto t2 = clk::now();
    get_results_(Q, sigma, &rank);
    auto t3 = clk::now();
    if (ms) {
        ms[0] = d(t0, t3);
        ms[1] = d(t0, t1);
        ms[2] = d(t1, t2);
        ms[3] = d(t2, t3);
    }
    return e != cudaSuccess ? (int)e : (int)cudaGetLastError();
}

extern "C" int ref_solve(float *T, int zstart, float *Q, float *sigma, double *ms) {
    double m[4];
    int rc = ref_solve_timed(T, zstart, Q, sigma, m);
    if (ms) *ms = m[0];
    return rc;
}
