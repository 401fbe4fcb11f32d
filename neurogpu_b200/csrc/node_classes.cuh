// Mechanism-set classes: channel code compiled for fixed masks.
//
// A node's channel update branches on each mechanism of its mask; over a
// runtime mask the compiler turns the short load / store blocks of absent
// mechanisms into predicated instructions that every node issues.  A kernel
// instantiated with a MaskList also carries a copy of the channel code per
// listed mask, with the mask a compile-time constant (MaskC): every
// mechanism test folds away and the compiler schedules all of the node's
// gates together.  A node whose mask is listed gets the list index as its
// class; any other node runs the generic code.  The ahead-of-time kernels
// use the empty list; the host generates, compiles (NVRTC) and caches a
// kernel per model with the model's own masks (ngpu.cu, jit_module).
#pragma once
#include "ngpu_math.cuh"

namespace ngpu {

// a mechanism mask known at compile time; converts to its value
template <uint32_t M>
struct MaskC {
    static constexpr uint32_t value = M;
    __host__ __device__ constexpr operator uint32_t() const { return M; }
};

template <uint32_t... Ms>
struct MaskList {
    static constexpr int size = (int)sizeof...(Ms);
};

using NoClasses = MaskList<>;

constexpr int kGenericClass = 255;
constexpr int kMaxClasses = 16;  // masks compiled per kernel; further masks stay generic

}  // namespace ngpu
