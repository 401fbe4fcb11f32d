// Test-only host build of the exploration score's per-trace code
// (neurogpu_b200/csrc/explore.cuh), so CPU tests can compare it with the
// restatement of scipy's find_peaks.  Compiled by tests/test_explore.py with
// nvcc into a host shared library.
#include <stdint.h>

#include <vector>

#include "../../neurogpu_b200/csrc/explore.cuh"

// v: [n_traces][n_samples] float32 (host); out: [n_traces] counts
extern "C" void probe_dvdt_peaks(const float* v, int n_traces, int n_samples, double dt, double height,
                                 int distance, int32_t* out) {
    ngpu::PeakArgs a;
    a.v = v;
    a.stride_trace = n_samples;
    a.stride_sample = 1;
    a.n_traces = n_traces;
    a.n_samples = n_samples;
    a.dt = dt;
    a.height = height;
    a.distance = distance;
    a.cap = ngpu::peak_scratch_cap(n_samples);
    std::vector<int32_t> pos((size_t)a.cap * (n_traces > 0 ? n_traces : 1));
    a.pos = pos.data();
    a.out = out;
    for (int t = 0; t < n_traces; ++t) out[t] = ngpu::dvdt_peaks_trace(a, t);
}
