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

}  // namespace gcl
