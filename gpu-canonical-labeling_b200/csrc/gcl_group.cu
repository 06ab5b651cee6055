// gcl_group.cu -- order of the automorphism group from the automorphisms the
// search stores (host code).
//
// The reference prints only how many automorphisms it stored
// (sequential.cpp:83), a number that depends on the traversal and on
// max_aut.  The automorphisms a complete search finds generate the whole
// group: every leaf equivalent to the first leaf is either visited or pruned
// through a stored automorphism (orbit pruning, the jump after an
// automorphism), and the group acts regularly on those leaves.  The order
// follows from a base and strong generating set built by the deterministic
// Schreier-Sims algorithm: |G| = product over the base of the basic orbit
// lengths.
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "gcl_group.h"

namespace gcl {
namespace {

using Perm = std::vector<uint32_t>;

// Coset representatives are kept as explicit permutations (u and u^-1, u16
// images) while the chain holds at most this many entries (128 MiB); beyond
// it a level falls back to walking its Schreier vector.
constexpr uint64_t kTransversalEntries = 1ull << 26;

struct Level {
  uint32_t base = 0;
  std::vector<int> S;              // strong generators fixing the base points before this one
  std::vector<int32_t> sv;         // per point: generator that reached it, -1 base, -2 outside
  std::vector<int32_t> slot;       // per point: its index in orbit, -1 outside
  std::vector<uint32_t> orbit;     // the basic orbit in the order its points were reached
  std::vector<uint32_t> applied;   // per orbit point: generators of S applied to it so far
  std::vector<uint32_t> tested;    // per orbit point: generators whose Schreier generator sifted
  std::vector<uint16_t> u, uinv;   // explicit representatives, orbit-major, n images each
  bool explicit_u = false;
};

struct Chain {
  uint32_t n = 0;
  std::vector<Perm> gens, inv;  // strong generators and their inverses
  std::vector<Level> lv;
  uint64_t work = 0, work_cap = 0;  // multiplication budget (0 = none)
  uint64_t entries = 0;             // explicit representative entries held
  // the levels' base points are a base of the group (only the identity fixes
  // them all): Schreier generators are sifted on their base images alone
  bool known_base = false;
  bool not_a_base = false;  // an element other than the identity fixed every base point
  std::vector<int> path;    // scratch: a representative's generator word
  std::vector<uint32_t> bi; // scratch: base images

  bool is_id(const Perm& p) const {
    for (uint32_t x = 0; x < n; ++x)
      if (p[x] != x) return false;
    return true;
  }

  int add_gen(const Perm& p) {
    gens.push_back(p);
    Perm q(n);
    for (uint32_t x = 0; x < n; ++x) q[p[x]] = x;
    inv.push_back(std::move(q));
    return (int)gens.size() - 1;
  }

  void drop_explicit(Level& L) {
    entries -= L.u.size() + L.uinv.size();
    std::vector<uint16_t>().swap(L.u);
    std::vector<uint16_t>().swap(L.uinv);
    L.explicit_u = false;
  }

  // y = g(x) joins the orbit; its representative is g u_x
  void add_point(Level& L, size_t k, int g, uint32_t y) {
    L.sv[y] = g;
    L.slot[y] = (int32_t)L.orbit.size();
    L.orbit.push_back(y);
    L.applied.push_back(0);
    L.tested.push_back(0);
    if (!L.explicit_u) return;
    if (entries + 2ull * n > kTransversalEntries) {
      drop_explicit(L);
      return;
    }
    const Perm& gp = gens[g];
    const Perm& gi = inv[g];
    const size_t base_off = k * n, off = L.u.size();
    L.u.resize(off + n);
    L.uinv.resize(off + n);
    for (uint32_t z = 0; z < n; ++z) {
      L.u[off + z] = (uint16_t)gp[L.u[base_off + z]];
      L.uinv[off + z] = L.uinv[base_off + gi[z]];
    }
    entries += 2ull * n;
    work += 2ull * n;
  }

  void new_level(uint32_t b) {
    lv.emplace_back();
    Level& L = lv.back();
    L.base = b;
    L.sv.assign(n, -2);
    L.slot.assign(n, -1);
    L.sv[b] = -1;
    L.slot[b] = 0;
    L.orbit.push_back(b);
    L.applied.push_back(0);
    L.tested.push_back(0);
    if (entries + 2ull * n <= kTransversalEntries) {
      L.explicit_u = true;
      L.u.resize(n);
      L.uinv.resize(n);
      for (uint32_t z = 0; z < n; ++z) L.u[z] = L.uinv[z] = (uint16_t)z;
      entries += 2ull * n;
    }
  }

  // grow the basic orbit of level i under the generators added since the
  // last call (the points already reached keep their representatives)
  void extend(size_t i) {
    Level& L = lv[i];
    for (size_t k = 0; k < L.orbit.size(); ++k) {
      const uint32_t x = L.orbit[k];
      for (size_t gi = L.applied[k]; gi < L.S.size(); ++gi) {
        const int g = L.S[gi];
        const uint32_t y = gens[g][x];
        if (L.sv[y] == -2) add_point(L, k, g, y);
      }
      work += L.S.size() - L.applied[k];
      L.applied[k] = (uint32_t)L.S.size();
    }
  }

  // h <- u_x^{-1} h, where u_x maps the level's base point to x
  void strip(const Level& L, uint32_t x, Perm& h) {
    if (L.explicit_u) {
      const uint16_t* ui = L.uinv.data() + (size_t)L.slot[x] * n;
      for (uint32_t p = 0; p < n; ++p) h[p] = ui[h[p]];
      work += n;
      return;
    }
    while (L.sv[x] >= 0) {
      const Perm& gi = inv[L.sv[x]];
      for (uint32_t p = 0; p < n; ++p) h[p] = gi[h[p]];
      x = gi[x];
      work += n;
    }
  }

  // t <- u_p as a permutation
  void rep(const Level& L, uint32_t p, Perm& t) {
    if (L.explicit_u) {
      const uint16_t* up = L.u.data() + (size_t)L.slot[p] * n;
      for (uint32_t z = 0; z < n; ++z) t[z] = up[z];
      work += n;
      return;
    }
    for (uint32_t z = 0; z < n; ++z) t[z] = z;
    std::vector<int> path;
    while (L.sv[p] >= 0) {
      path.push_back(L.sv[p]);
      p = inv[L.sv[p]][p];
    }
    for (size_t q = path.size(); q-- > 0;) {
      const Perm& g = gens[path[q]];
      for (uint32_t z = 0; z < n; ++z) t[z] = g[t[z]];
      work += n;
    }
  }

  // the generators along the Schreier vector from x back to the base point
  // (last applied first): u_x = path[0] path[1] ... path[k-1]
  void word(const Level& L, uint32_t x) {
    path.clear();
    while (L.sv[x] >= 0) {
      path.push_back(L.sv[x]);
      x = inv[L.sv[x]][x];
    }
  }

  // bi[m] <- u_p(bi[m]) for m in [lo, hi)
  void apply_rep(const Level& L, uint32_t p, size_t lo, size_t hi) {
    if (L.explicit_u) {
      const uint16_t* up = L.u.data() + (size_t)L.slot[p] * n;
      for (size_t m = lo; m < hi; ++m) bi[m] = up[bi[m]];
      work += hi - lo;
      return;
    }
    word(L, p);
    for (size_t m = lo; m < hi; ++m) {
      uint32_t z = bi[m];
      for (size_t q = path.size(); q-- > 0;) z = gens[path[q]][z];
      bi[m] = z;
    }
    work += (hi - lo) * path.size();
  }

  // bi[m] <- u_x^{-1}(bi[m]) for m in [lo, hi)
  void apply_rep_inv(const Level& L, uint32_t x, size_t lo, size_t hi) {
    if (L.explicit_u) {
      const uint16_t* ui = L.uinv.data() + (size_t)L.slot[x] * n;
      for (size_t m = lo; m < hi; ++m) bi[m] = ui[bi[m]];
      work += hi - lo;
      return;
    }
    word(L, x);
    for (size_t m = lo; m < hi; ++m) {
      uint32_t z = bi[m];
      for (size_t q = 0; q < path.size(); ++q) z = inv[path[q]][z];
      bi[m] = z;
    }
    work += (hi - lo) * path.size();
  }

  // sift the element whose base images are bi[from..] from level `from`;
  // returns the level where it left the chain, lv.size() if it fixes every
  // base point after the strips (with a known base: the identity)
  size_t sift_images(size_t from) {
    for (size_t i = from; i < lv.size(); ++i) {
      const uint32_t x = bi[i];
      if (x == lv[i].base) continue;  // u of the base point is the identity
      if (lv[i].sv[x] == -2) return i;
      apply_rep_inv(lv[i], x, i, lv.size());
    }
    return lv.size();
  }

  // sift h from level `from`; returns the level where it left the chain
  // (lv.size() if it passed every level) and leaves the residue in h
  size_t sift(Perm& h, size_t from) {
    for (size_t i = from; i < lv.size(); ++i) {
      const uint32_t x = h[lv[i].base];
      if (x == lv[i].base) continue;  // u of the base point is the identity
      if (lv[i].sv[x] == -2) return i;
      strip(lv[i], x, h);
    }
    return lv.size();
  }

  // a residue that left the chain at level j joins S[from..j] (it fixes the
  // base points before j); one that passed every level moves a new base point
  void insert(const Perm& h, size_t from, size_t j) {
    if (j == lv.size()) {
      uint32_t b = 0;
      while (b < n && h[b] == b) ++b;
      new_level(b);
    }
    const int id = add_gen(h);
    for (size_t l = from; l <= j; ++l) lv[l].S.push_back(id);
  }

  // Deterministic Schreier-Sims from level i up to level 0: at every level
  // each Schreier generator u_{s(p)}^-1 s u_p (p in the basic orbit, s in S)
  // sifts through the deeper levels to the identity, else its residue
  // becomes a strong generator and the deeper levels it joined are completed
  // first.  Orbits only grow and keep their representatives, so each
  // (point, generator) pair is tested once; pairs that are edges of the
  // orbit's search tree give the identity and are skipped.
  bool complete(size_t i) {
    Perm t(n), h(n);
    while (true) {
      extend(i);
      size_t next = i;
      bool inserted = false;
      for (size_t k = 0; k < lv[i].orbit.size() && !inserted; ++k) {
        const uint32_t p = lv[i].orbit[k];
        for (size_t gi = lv[i].tested[k]; gi < lv[i].S.size(); ++gi) {
          const int sid = lv[i].S[gi];
          const Perm& s = gens[sid];
          const uint32_t y = s[p];
          lv[i].tested[k] = (uint32_t)gi + 1;
          if (lv[i].sv[y] == sid) continue;  // a tree edge: u_y = s u_p
          if (known_base) {
            // t = u_y^-1 s u_p fixes the base points up to i; its images of
            // the deeper ones decide whether it is the identity
            const size_t L = lv.size();
            for (size_t m = i + 1; m < L; ++m) bi[m] = lv[m].base;
            apply_rep(lv[i], p, i + 1, L);
            for (size_t m = i + 1; m < L; ++m) bi[m] = s[bi[m]];
            apply_rep_inv(lv[i], y, i + 1, L);
            if (sift_images(i + 1) == L) {
              if (work_cap && work > work_cap) return false;
              continue;
            }
          }
          rep(lv[i], p, h);
          for (uint32_t z = 0; z < n; ++z) t[z] = s[h[z]];
          work += n;
          strip(lv[i], y, t);
          const size_t j = sift(t, i + 1);
          if (known_base && j == lv.size()) {
            // the base images said otherwise, or the points are no base
            not_a_base = true;
            return false;
          }
          if (j < lv.size() || !is_id(t)) {
            insert(t, i + 1, j);
            next = j;
            inserted = true;
            break;
          }
          if (work_cap && work > work_cap) return false;
        }
      }
      if (work_cap && work > work_cap) return false;
      if (inserted) {
        i = next;
        continue;
      }
      if (i == 0) return true;
      --i;
    }
  }
};

// decimal product of the basic orbit lengths
std::string big_product(const std::vector<uint64_t>& f) {
  std::vector<uint32_t> d{1};  // base 1e9, little endian
  for (uint64_t x : f) {
    uint64_t carry = 0;
    for (uint32_t& w : d) {
      const unsigned __int128 v = (unsigned __int128)w * x + carry;
      w = (uint32_t)(v % 1000000000u);
      carry = (uint64_t)(v / 1000000000u);
    }
    while (carry) {
      d.push_back((uint32_t)(carry % 1000000000u));
      carry /= 1000000000u;
    }
  }
  std::string s = std::to_string(d.back());
  char buf[16];
  for (size_t k = d.size() - 1; k-- > 0;) {
    std::snprintf(buf, sizeof buf, "%09u", d[k]);
    s += buf;
  }
  return s;
}

}  // namespace

namespace {

int run(Chain& C, const uint16_t* auts, uint64_t count, uint64_t stride, double* log10_order,
        std::string* digits, uint64_t* base_len) {
  const uint32_t n = C.n;
  Perm p(n);
  for (uint64_t a = 0; a < count; ++a) {
    for (uint32_t x = 0; x < n; ++x) p[x] = auts[a * stride + x];
    if (C.is_id(p)) continue;
    // a generator the chain already contains sifts to the identity
    const size_t j = C.sift(p, 0);
    if (j == C.lv.size()) {
      if (C.is_id(p)) continue;
      if (C.known_base) return kOrderNotABase;
    }
    C.insert(p, 0, j);
    if (!C.complete(j)) return C.not_a_base ? kOrderNotABase : kOrderWorkCap;
  }
  std::vector<uint64_t> f;
  double lg = 0;
  for (size_t i = 0; i < C.lv.size(); ++i) {
    C.extend(i);
    f.push_back(C.lv[i].orbit.size());
    lg += std::log10((double)C.lv[i].orbit.size());
  }
  *log10_order = lg;
  *digits = big_product(f);
  *base_len = C.lv.size();
  return kOrderOk;
}

}  // namespace

bool group_order(uint32_t n, const uint16_t* auts, uint64_t count, uint64_t stride,
                 uint64_t work_cap, double* log10_order, std::string* digits,
                 uint64_t* base_len) {
  Chain C;
  C.n = n;
  C.work_cap = work_cap;
  return run(C, auts, count, stride, log10_order, digits, base_len) == kOrderOk;
}

bool group_order_base_orbits(uint32_t n, const uint16_t* auts, uint64_t count, uint64_t stride,
                             const uint32_t* base, uint32_t nbase, double* log10_order,
                             std::string* digits) {
  for (uint32_t m = 0; m < nbase; ++m)
    if (base[m] >= n) return false;
  // automorphisms by level: the first base point each moves (none: dropped)
  std::vector<std::vector<uint64_t>> at(nbase);
  for (uint64_t a = 0; a < count; ++a) {
    const uint16_t* pm = auts + a * stride;
    uint32_t j = 0;
    while (j < nbase && pm[base[j]] == base[j]) ++j;
    if (j < nbase) at[j].push_back(a);
  }
  // deepest level first: the generators fixing b_0..b_{i-1} are those of
  // levels >= i, so each level adds its own to one running union-find
  std::vector<uint32_t> par(n), size(n, 1);
  for (uint32_t x = 0; x < n; ++x) par[x] = x;
  auto find = [&](uint32_t x) {
    while (par[x] != x) {
      par[x] = par[par[x]];
      x = par[x];
    }
    return x;
  };
  std::vector<uint64_t> f(nbase, 1);
  for (uint32_t i = nbase; i-- > 0;) {
    for (uint64_t a : at[i]) {
      const uint16_t* pm = auts + a * stride;
      for (uint32_t x = 0; x < n; ++x) {
        uint32_t rx = find(x), ry = find(pm[x]);
        if (rx == ry) continue;
        if (size[rx] < size[ry]) std::swap(rx, ry);
        par[ry] = rx;
        size[rx] += size[ry];
      }
    }
    f[i] = size[find(base[i])];
  }
  double lg = 0;
  for (uint64_t x : f) lg += std::log10((double)x);
  *log10_order = lg;
  *digits = big_product(f);
  return true;
}

int group_order_with_base(uint32_t n, const uint16_t* auts, uint64_t count, uint64_t stride,
                          const uint32_t* base, uint32_t nbase, uint64_t work_cap,
                          double* log10_order, std::string* digits, uint64_t* base_len) {
  Chain C;
  C.n = n;
  C.work_cap = work_cap;
  C.known_base = true;
  std::vector<char> seen(n, 0);
  for (uint32_t m = 0; m < nbase; ++m) {
    if (base[m] >= n || seen[base[m]]) return kOrderNotABase;
    seen[base[m]] = 1;
    C.new_level(base[m]);
  }
  C.bi.resize(nbase);
  return run(C, auts, count, stride, log10_order, digits, base_len);
}

int group_order_of_search(uint32_t n, const uint16_t* auts, uint64_t count, uint64_t stride,
                          const uint32_t* base, uint32_t nbase, uint64_t check_cap,
                          double* log10_order, std::string* digits, int* checked) {
  *checked = 0;
  if (!group_order_base_orbits(n, auts, count, stride, base, nbase, log10_order, digits))
    return kOrderNotABase;
  if (check_cap == 0) return kOrderOk;
  double lg = 0;
  std::string d;
  uint64_t bl = 0;
  // the general completion first (cheapest where the orbits are short),
  // then the completion on the search's base (long orbits)
  int rc = group_order(n, auts, count, stride, check_cap, &lg, &d, &bl) ? kOrderOk : kOrderWorkCap;
  if (rc == kOrderWorkCap)
    rc = group_order_with_base(n, auts, count, stride, base, nbase, check_cap, &lg, &d, &bl);
  if (rc == kOrderNotABase) return kOrderNotABase;
  if (rc == kOrderWorkCap) return kOrderOk;  // unchecked: the orbit product stands
  if (d != *digits) {
    // the stored automorphisms are no strong generating set for the base:
    // the completion's order (of the group they generate) is the one to trust
    *log10_order = lg;
    *digits = d;
    *checked = -1;
    return kOrderOk;
  }
  *checked = 1;
  return kOrderOk;
}

}  // namespace gcl
