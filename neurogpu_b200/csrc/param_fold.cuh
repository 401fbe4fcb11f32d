// Parameters compiled into the runtime-specialised kernel as constants.
//
// A parameter that holds one value for every parameter set and every
// section whose nodes use its mechanism (the kinetic constants of a model,
// as opposed to the conductances a fit varies) need not be read per node and
// step.  The runtime-specialised translation unit declares such parameters
// as specialisations ParamFold<P> (P: the parameter's index in its mechanism
// set) before it includes the kernels; everywhere else the primary template
// applies and the parameter is read from its row.  The value is the exact
// float the row would hold, written as a hexadecimal literal.
#pragma once
#include "ngpu_math.cuh"

namespace ngpu {

template <int P>
struct ParamFold {
    static constexpr bool on = false;
    static constexpr float v = 0.f;
};

// parameter P of the node, at row q of its parameter rows
template <typename R, int P>
NGPU_HD R pload(const float* __restrict__ pr, int q) {
    if constexpr (ParamFold<P>::on) return (R)ParamFold<P>::v;
    else return (R)pr[q * 32];
}

// parameters B .. B+N-1 at rows q .. q+N-1 into out[0..N)
template <typename R, int B, int N, int K = 0>
NGPU_HD void pload_n(const float* __restrict__ pr, int q, R* out) {
    if constexpr (K < N) {
        out[K] = pload<R, B + K>(pr, q + K);
        pload_n<R, B, N, K + 1>(pr, q, out);
    }
}

}  // namespace ngpu
