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

// The order as the product over the first path's levels of the orbit of its
// vertex b_i under the stored automorphisms that fix b_0..b_{i-1} -- the
// search's group order (nauty's grpsize).  Valid for automorphisms a complete
// search stored, all of them: every first-path sibling in the orbit of b_i is
// either searched, and a leaf equivalent to the first leaf under it gives an
// automorphism fixing b_0..b_{i-1} that moves b_i there, or skipped as
// equivalent to one that is; so these automorphisms form a strong generating
// set for that base.  O(stored x n).  false: a base point is not below n.
bool group_order_base_orbits(uint32_t n, const uint16_t* auts, uint64_t count, uint64_t stride,
                             const uint32_t* base, uint32_t nbase, double* log10_order,
                             std::string* digits);

// The order of Aut(G) from a complete search: the `count` automorphisms it
// stored (every one it found) and its first path's nbase individualized
// vertices.  The order is the product of the basic orbits
// (group_order_base_orbits); the Schreier-Sims completion checks it, general
// and then on the known base, within check_cap operations each (0: no
// check).  kOrderOk with *checked = 1 when a completion finished and agreed,
// 0 when both ran out of work, and -1 when a completion finished with
// another order, which is then the one returned (the order of the group the
// automorphisms generate, which needs less of them than the product does);
// kOrderNotABase for a base that is none.
int group_order_of_search(uint32_t n, const uint16_t* auts, uint64_t count, uint64_t stride,
                          const uint32_t* base, uint32_t nbase, uint64_t check_cap,
                          double* log10_order, std::string* digits, int* checked);

}  // namespace gcl
