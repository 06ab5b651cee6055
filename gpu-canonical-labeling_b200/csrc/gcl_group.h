// gcl_group.h -- automorphism group order from stored automorphisms (host).
#pragma once
#include <cstdint>
#include <string>

namespace gcl {

// Order of the group generated by `count` permutations of {0..n-1}
// (auts + a*stride, u16 images).  Returns false when the Schreier-Sims
// completion exceeds `work_cap` elementary operations (0 = no cap).
// digits receives the order in decimal, base_len the length of the base.
bool group_order(uint32_t n, const uint16_t* auts, uint64_t count, uint64_t stride,
                 uint64_t work_cap, double* log10_order, std::string* digits,
                 uint64_t* base_len);

enum { kOrderOk = 0, kOrderWorkCap = 1, kOrderNotABase = 2 };

// Same, given a base: nbase distinct points that only the identity fixes all
// of (for a graph, the individualized vertices of the search's first path:
// an automorphism fixing them fixes the first leaf's discrete partition).
// Schreier generators are then sifted on their base images alone and only
// those that become strong generators are multiplied out in full.  The
// caller vouches for the base: the completion does not search for an element
// that fixes it, and returns kOrderNotABase only when it meets one (an input
// or a residue other than the identity fixing every base point); otherwise
// kOrderOk or kOrderWorkCap.
int group_order_with_base(uint32_t n, const uint16_t* auts, uint64_t count, uint64_t stride,
                          const uint32_t* base, uint32_t nbase, uint64_t work_cap,
                          double* log10_order, std::string* digits, uint64_t* base_len);

}  // namespace gcl
