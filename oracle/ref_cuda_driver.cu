// Driver for the reference's own CUDA propagator — TEST INFRASTRUCTURE.
//
// Linked by oracle/build.py with the reference sources compiled from the
// reference tree (src/initialize.cu, src/liouville.cu, src/matrix_storage.cu,
// src/matrix_util.cu, src/cuda_sparse_backend_plan.cu, src/psd/*.cu,
// src/library/backend_profiling.cpp) in FP64 (oracle/ref_cuda_prelude.h) with
// the shape taken from the environment (oracle/ref_cuda_params.cu).  It calls
// the reference's own set-up and step functions, as its session does
// (src/library/legacy_runtime_session.cu:53-100): `initialize()`
// (src/initialize.cu:342-353), then `develop()` once per step
// (src/liouville.cu:502-590), and reads the state `dRho` the way its result
// extractor does (src/library/result_extractor.cu:35-90: slab 0, row-major).
// This file holds no reference code: it only calls it.
//
// Usage:
//   ref_cuda_propagator [--steps S] [--trace FILE] [--diag FILE] [--state FILE]
//                       [--time K] [--warmup W]
//   --trace FILE  write rho_0 at t = 0, dt, ..., S*dt (N*N complex128 each,
//                 re/im interleaved, row-major) to FILE
//   --diag FILE   write Re diag(rho_0) at t = 0, dt, ..., S*dt (N float64 each)
//   --state FILE  write the whole hierarchy (H*N*N complex128) after S steps
//   --time K      after the S steps and W warm-up steps, time K steps with CUDA
//                 events on the legacy default stream (which orders against
//                 every blocking stream the reference creates)
// One JSON line on stdout reports the shape, the timing and any CUDA error.

#include "initialize.h"
#include "liouville.h"
#include "matrix_storage.h"
#include "parameters.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

std::string g_error;

bool check(cudaError_t err, const char* what)
{
    if (err != cudaSuccess && g_error.empty()) {
        g_error = std::string(what) + ": " + cudaGetErrorString(err);
    }
    return err == cudaSuccess;
}

bool write_slabs(FILE* f, std::size_t first, std::size_t count)
{
    std::vector<Complex> host(count);
    thrust::copy_n(dRho.begin() + first, count, host.begin());
    std::vector<double> out(2 * count);
    for (std::size_t i = 0; i < count; ++i) {
        out[2 * i] = static_cast<double>(host[i].x);
        out[2 * i + 1] = static_cast<double>(host[i].y);
    }
    return std::fwrite(out.data(), sizeof(double), out.size(), f) == out.size();
}

bool write_diagonal(FILE* f)
{
    const int n = Param::N;
    std::vector<Complex> host(static_cast<std::size_t>(Param::N2));
    thrust::copy_n(dRho.begin(), host.size(), host.begin());
    std::vector<double> out(n);
    for (int i = 0; i < n; ++i) out[i] = static_cast<double>(host[static_cast<std::size_t>(i) * (n + 1)].x);
    return std::fwrite(out.data(), sizeof(double), out.size(), f) == out.size();
}

}  // namespace

int main(int argc, char** argv)
{
    long steps = 0, timed = 0, warmup = 0;
    const char* trace_path = nullptr;
    const char* state_path = nullptr;
    const char* diag_path = nullptr;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&](void) -> const char* {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value after %s\n", a.c_str());
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--steps") steps = std::atol(next());
        else if (a == "--trace") trace_path = next();
        else if (a == "--state") state_path = next();
        else if (a == "--diag") diag_path = next();
        else if (a == "--time") timed = std::atol(next());
        else if (a == "--warmup") warmup = std::atol(next());
        else {
            std::fprintf(stderr, "unknown argument %s\n", a.c_str());
            return 2;
        }
    }

    const auto t_init0 = std::chrono::steady_clock::now();
    initialize();
    check(cudaDeviceSynchronize(), "initialize");
    const double init_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_init0).count();
    const std::size_t n2 = static_cast<std::size_t>(Param::N2);

    FILE* trace = nullptr;
    if (trace_path) {
        trace = std::fopen(trace_path, "wb");
        if (!trace) {
            std::fprintf(stderr, "cannot open %s\n", trace_path);
            return 2;
        }
        write_slabs(trace, 0, n2);
    }
    FILE* diag = nullptr;
    if (diag_path) {
        diag = std::fopen(diag_path, "wb");
        if (!diag) {
            std::fprintf(stderr, "cannot open %s\n", diag_path);
            return 2;
        }
        write_diagonal(diag);
    }
    double first_step_ms = 0.0;
    for (long s = 0; s < steps && g_error.empty(); ++s) {
        const auto t0 = std::chrono::steady_clock::now();
        develop();
        check(cudaDeviceSynchronize(), "develop");
        if (s == 0) {
            first_step_ms =
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        if (trace) write_slabs(trace, 0, n2);
        if (diag) write_diagonal(diag);
    }
    if (trace) std::fclose(trace);
    if (diag) std::fclose(diag);
    if (state_path && g_error.empty()) {
        FILE* f = std::fopen(state_path, "wb");
        if (!f) {
            std::fprintf(stderr, "cannot open %s\n", state_path);
            return 2;
        }
        write_slabs(f, 0, static_cast<std::size_t>(hierarchySize) * n2);
        std::fclose(f);
    }

    double ms_per_step = 0.0, wall_ms_per_step = 0.0;
    if (timed > 0 && g_error.empty()) {
        for (long s = 0; s < warmup; ++s) develop();
        check(cudaDeviceSynchronize(), "warm-up");
        cudaEvent_t e0, e1;
        check(cudaEventCreate(&e0), "event");
        check(cudaEventCreate(&e1), "event");
        const auto w0 = std::chrono::steady_clock::now();
        check(cudaEventRecord(e0, 0), "event record");
        for (long s = 0; s < timed; ++s) develop();
        check(cudaEventRecord(e1, 0), "event record");
        check(cudaEventSynchronize(e1), "timed steps");
        check(cudaDeviceSynchronize(), "timed steps");
        const auto w1 = std::chrono::steady_clock::now();
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        ms_per_step = ms / timed;
        wall_ms_per_step = std::chrono::duration<double, std::milli>(w1 - w0).count() / timed;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    check(cudaGetLastError(), "last error");
    std::size_t mem_free = 0, mem_total = 0;
    cudaMemGetInfo(&mem_free, &mem_total);

    std::printf("{\"dim\": %d, \"modes\": %d, \"max_depth\": %d, \"hierarchy_size\": %d, \"dt\": %.17g, "
                "\"precision\": \"%s\", \"init_ms\": %.3f, \"steps\": %ld, \"first_step_ms\": %.3f, "
                "\"timed_steps\": %ld, \"warmup\": %ld, \"ms_per_step\": %.6f, \"wall_ms_per_step\": %.6f, "
                "\"ado_steps_per_s\": %.3f, \"device_bytes_in_use\": %zu, \"cuda_error\": \"%s\"}\n",
                Param::N, Param::KMax + 1, Param::JMax, hierarchySize, Param::Step,
                sizeof(real) == 8 ? "double" : "single", init_ms, steps, first_step_ms, timed, warmup,
                ms_per_step, wall_ms_per_step,
                ms_per_step > 0 ? hierarchySize * 1000.0 / ms_per_step : 0.0, mem_total - mem_free,
                g_error.c_str());
    std::fflush(stdout);

    clearLiouvilleStorage();
    clearMatrixStorage();
    return g_error.empty() ? 0 : 1;
}
