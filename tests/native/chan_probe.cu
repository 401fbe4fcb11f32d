// Test-only host build of the product's channel code (neurogpu_b200/csrc),
// so CPU tests can compare its equations with the oracle's node functions.
// Compiled by tests/test_channels_host.py with nvcc into a host shared library.
#include <stdint.h>

#include "../../neurogpu_b200/csrc/channels_mainen.cuh"
#include "../../neurogpu_b200/csrc/channels_ttpc.cuh"

template <typename R>
static void node(int mechset, int init, uint32_t mask, R v, R dt, R* st, const float* pr, R* I, R* G) {
    R i = 0, g = 0;
    if (mechset == 0) {
        if (init) ngpu::ttpc_node<R, true>(mask, v, dt, st, pr, i, g);
        else ngpu::ttpc_node<R, false>(mask, v, dt, st, pr, i, g);
    } else {
        if (init) ngpu::mainen_node<R, true>(mask, v, dt, st, pr, i, g);
        else ngpu::mainen_node<R, false>(mask, v, dt, st, pr, i, g);
    }
    *I = i;
    *G = g;
}

// st: [rows][32] (lane 0 used), pr: [rows][32] floats (lane 0 used)
extern "C" void probe_node_f64(int mechset, int init, uint32_t mask, double v, double dt, double* st,
                               const float* pr, double* I, double* G) {
    node<double>(mechset, init, mask, v, dt, st, pr, I, G);
}
extern "C" void probe_node_f32(int mechset, int init, uint32_t mask, float v, float dt, float* st,
                               const float* pr, float* I, float* G) {
    node<float>(mechset, init, mask, v, dt, st, pr, I, G);
}
