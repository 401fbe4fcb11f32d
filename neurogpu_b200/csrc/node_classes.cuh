// Mechanism sets compiled as straight-line channel code.
//
// A node's channel update branches on each mechanism of its mask.  For the
// masks listed here the kernel also carries a copy of the channel code with
// the mask fixed at compile time; there every mechanism test folds away and
// the compiler schedules all of the node's gates together.  A node whose
// mask is listed is given the list index as its class (node_class); any
// other node runs the generic code.
#pragma once
#include <stdint.h>
#include <type_traits>

namespace ngpu {

template <uint32_t... Ms>
struct MaskList {
    static constexpr int size = (int)sizeof...(Ms);
};

// TTPC: basal (Ih, pas); apical (Ih, Im, NaTs2_t, pas, SKv3_1); axon; apical
// hot zone; soma.  Mainen: soma+dendrite, axon, soma with kv.
using TTPCClasses = MaskList<0x408u, 0x1618u, 0x1de7u, 0x1e1fu, 0x1e6fu>;
using MainenClasses = MaskList<0x6fu, 0x70u, 0x7fu>;

constexpr int kGenericClass = 255;

template <uint32_t... Ms>
inline int class_in(MaskList<Ms...>, uint32_t mask) {
    const uint32_t v[] = {Ms...};
    for (int k = 0; k < (int)sizeof...(Ms); ++k)
        if (v[k] == mask) return k;
    return kGenericClass;
}

// mechset: 0 TTPC, 1 Mainen
inline int node_class(int mechset, uint32_t mask) {
    return mechset == 0 ? class_in(TTPCClasses{}, mask) : class_in(MainenClasses{}, mask);
}

}  // namespace ngpu
