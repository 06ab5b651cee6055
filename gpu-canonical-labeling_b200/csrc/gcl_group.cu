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

struct Chain {
  uint32_t n = 0;
  std::vector<Perm> gens, inv;           // strong generators and their inverses
  std::vector<uint32_t> base;
  std::vector<std::vector<int>> S;       // S[i]: generators fixing base[0..i-1]
  std::vector<std::vector<int32_t>> sv;  // Schreier vectors: generator reaching the point,
                                         // -1 at the base point, -2 outside the orbit
  std::vector<std::vector<uint32_t>> orbit;
  uint64_t work = 0, work_cap = 0;       // multiplication budget (0 = none)

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

  // orbit of base[i] under S[i], with its Schreier vector
  void build_orbit(size_t i) {
    std::vector<int32_t>& v = sv[i];
    v.assign(n, -2);
    std::vector<uint32_t>& o = orbit[i];
    o.clear();
    v[base[i]] = -1;
    o.push_back(base[i]);
    for (size_t k = 0; k < o.size(); ++k) {
      const uint32_t x = o[k];
      for (int g : S[i]) {
        const uint32_t y = gens[g][x];
        if (v[y] == -2) {
          v[y] = g;
          o.push_back(y);
        }
      }
    }
    work += (uint64_t)o.size() * S[i].size();
  }

  // h <- u_x^{-1} h, where u_x maps base[i] to x (walks the Schreier vector)
  void strip_rep(size_t i, uint32_t x, Perm& h) {
    while (sv[i][x] >= 0) {
      const Perm& gi = inv[sv[i][x]];
      for (uint32_t p = 0; p < n; ++p) h[p] = gi[h[p]];
      x = gi[x];
      work += n;
    }
  }

  // sift h from level `from`; returns the level where it left the chain
  // (base.size() if it passed every level) and leaves the residue in h
  size_t sift(Perm& h, size_t from) {
    for (size_t i = from; i < base.size(); ++i) {
      const uint32_t x = h[base[i]];
      if (sv[i][x] == -2) return i;
      strip_rep(i, x, h);
    }
    return base.size();
  }

  void new_level(uint32_t b) {
    base.push_back(b);
    S.emplace_back();
    sv.emplace_back();
    orbit.emplace_back();
  }

  // a residue that left the chain at level j joins S[from..j] (it fixes the
  // base points before j); a residue that passed every level moves a new
  // base point
  size_t insert(const Perm& h, size_t from, size_t j) {
    if (j == base.size()) {
      uint32_t b = 0;
      while (b < n && h[b] == b) ++b;
      new_level(b);
    }
    const int id = add_gen(h);
    for (size_t l = from; l <= j; ++l) S[l].push_back(id);
    return j;
  }

  // complete the chain: every Schreier generator of every level sifts to the
  // identity (Schreier-Sims, deterministic form)
  bool complete() {
    if (base.empty()) return true;
    size_t i = base.size() - 1;
    for (size_t l = 0; l < base.size(); ++l) build_orbit(l);
    while (true) {
      bool changed = false;
      build_orbit(i);
      Perm h(n), t(n);
      for (size_t k = 0; k < orbit[i].size() && !changed; ++k) {
        const uint32_t p = orbit[i][k];
        for (size_t si = 0; si < S[i].size() && !changed; ++si) {
          const Perm& s = gens[S[i][si]];
          // h = u_{s(p)}^{-1} s u_p
          for (uint32_t x = 0; x < n; ++x) h[x] = x;
          // u_p: base[i] -> p, built as a product along the Schreier vector
          {
            uint32_t y = p;
            std::vector<int> path;
            while (sv[i][y] >= 0) {
              path.push_back(sv[i][y]);
              y = inv[sv[i][y]][y];
            }
            for (size_t q = path.size(); q-- > 0;) {
              const Perm& g = gens[path[q]];
              for (uint32_t x = 0; x < n; ++x) h[x] = g[h[x]];
              work += n;
            }
          }
          for (uint32_t x = 0; x < n; ++x) t[x] = s[h[x]];
          strip_rep(i, s[p], t);
          work += n;
          const size_t j = sift(t, i + 1);
          if (j < base.size() || !is_id(t)) {
            insert(t, i + 1, j);
            for (size_t l = i + 1; l < base.size(); ++l) build_orbit(l);
            i = base.size() - 1;
            changed = true;
          }
          if (work_cap && work > work_cap) return false;
        }
      }
      if (changed) continue;
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

bool group_order(uint32_t n, const uint16_t* auts, uint64_t count, uint64_t stride,
                 uint64_t work_cap, double* log10_order, std::string* digits,
                 uint64_t* base_len) {
  Chain C;
  C.n = n;
  C.work_cap = work_cap;
  Perm p(n);
  for (uint64_t a = 0; a < count; ++a) {
    for (uint32_t x = 0; x < n; ++x) p[x] = auts[a * stride + x];
    if (C.is_id(p)) continue;
    // skip generators the chain already contains
    if (!C.base.empty()) {
      Perm h = p;
      const size_t j = C.sift(h, 0);
      if (j == C.base.size() && C.is_id(h)) continue;
      C.insert(h, 0, j);
    } else {
      C.insert(p, 0, 0);
    }
    if (!C.complete()) return false;
  }
  std::vector<uint64_t> f;
  double lg = 0;
  for (size_t i = 0; i < C.base.size(); ++i) {
    f.push_back(C.orbit[i].size());
    lg += std::log10((double)C.orbit[i].size());
  }
  *log10_order = lg;
  *digits = big_product(f);
  *base_len = C.base.size();
  return true;
}

}  // namespace gcl
