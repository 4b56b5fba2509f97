// Binomial checkpointing for the reversal of a fixed-step trajectory, in the
// manner of Griewank's revolve (A. Griewank, A. Walther, "Algorithm 799:
// revolve", ACM TOMS 26 (2000) 19-45).  Host code only: the schedule is
// the same whether the executor runs the steps on the device or counts them.
//
// A budget of S snapshots holds S states at once, the initial one among them
// (slot 0).  To reverse steps [l, r) from the state of step l held in a slot
// with c slots still free: advance m steps into a new slot, reverse [l + m, r)
// with c - 1 free slots, then [l, l + m) with c (the new slot is free again);
// one step is reversed by recording its stage states and running the adjoint
// stages; with no free slot every step is reached from l again.  The split m
// minimises the forward steps of the whole reversal,
//   F(1, c) = 1,  F(n, 0) = n (n + 1) / 2,
//   F(n, c) = min_m  m + F(n - m, c - 1) + F(m, c),
// by dynamic programming over n and c while n^2 S / 2 stays under
// kRevolveDpWork; longer trajectories split by the binomial rule (beta(c, t) = C(c + t, c) steps
// need t passes with c free slots, and the right part takes beta(c - 1, t)).
// The forward trajectory stores the states of the first descent (the spine)
// as it passes them, so the reversal starts at the last of them; its splits
// minimise G(n, c) = min_m G(n - m, c - 1) + F(m, c) (the spine's own advances
// are the forward pass's), with G(1, c) = 1 and G(n, 0) = F(n, 0).
#pragma once

#include <algorithm>
#include <vector>

namespace apollo {

inline double revolve_beta(int c, int t) {
  double b = 1.0;
  for (int i = 1; i <= c; ++i) b = b * (t + i) / i;
  return b;
}

constexpr double kRevolveDpWork = 1.5e8;  // split candidates the dynamic program may examine

struct RevolvePlan {
  int n = 0;      // trajectory steps
  int S = 0;      // snapshot slots, the initial state's included
  std::vector<int> arg;  // [n + 1][S] best split for (length, free slots); empty: binomial rule
  std::vector<int> sarg;  // the same for the spine

  int split(int len, int c) const {
    if (!arg.empty()) return arg[(size_t)len * S + c];
    int t = 1;
    while (revolve_beta(c, t) < len) ++t;
    const double right = std::min<double>(revolve_beta(c - 1, t), (double)(len - 1));
    return std::max(1, len - (int)right);
  }

  void build(int nsteps, int snapshots) {
    n = nsteps;
    S = snapshots;
    arg.clear();
    sarg.clear();
    if (S < 2 || 0.5 * (double)n * n * S > kRevolveDpWork) return;
    std::vector<long long> F((size_t)(n + 1) * S, 0), G((size_t)(n + 1) * S, 0);
    arg.assign((size_t)(n + 1) * S, 1);
    sarg.assign((size_t)(n + 1) * S, 1);
    auto idx = [&](int len, int c) { return (size_t)len * S + c; };
    for (int len = 1; len <= n; ++len) {
      F[idx(len, 0)] = G[idx(len, 0)] = (long long)len * (len + 1) / 2;
      for (int c = 1; c < S; ++c) {
        if (len == 1) {
          F[idx(len, c)] = G[idx(len, c)] = 1;
          continue;
        }
        long long bf = -1, bg = -1;
        int mf = 1, mg = 1;
        for (int m = 1; m < len; ++m) {
          const long long f = m + F[idx(len - m, c - 1)] + F[idx(m, c)];
          const long long g = G[idx(len - m, c - 1)] + F[idx(m, c)];
          if (bf < 0 || f < bf) {
            bf = f;
            mf = m;
          }
          if (bg < 0 || g < bg) {
            bg = g;
            mg = m;
          }
        }
        F[idx(len, c)] = bf;
        G[idx(len, c)] = bg;
        arg[idx(len, c)] = mf;
        sarg[idx(len, c)] = mg;
      }
    }
  }

  // The first descent: p[k] is the step whose state slot k holds, with
  // S - 1 - k slots free after it.
  std::vector<int> spine() const {
    std::vector<int> p{0};
    int l = 0, c = S - 1;
    while (n - l > 1 && c > 0) {
      l += sarg.empty() ? split(n - l, c) : sarg[(size_t)(n - l) * S + c];
      --c;
      p.push_back(l);
    }
    return p;
  }
};

// The reversal of steps [0, n) after a forward pass that stored the spine.
// Exec supplies (each returning 0 or an error status):
//   copy(dst, src)             a slot's state into another (dst -1: the work buffer)
//   advance(slot, from, count) count steps from step `from` on a slot (-1: the work buffer)
//   leaf(j, slot)              record step j from the state in slot (-1: the work
//                              buffer) and run its adjoint
template <class Exec>
struct RevolveRun {
  const RevolvePlan& plan;
  Exec& x;

  // The left part [l, l + m) is reversed by the same loop (a tail call), so
  // the recursion is only as deep as the free slots.
  int rev(int l, int r, int c, int slot) {
    for (;;) {
      const int len = r - l;
      if (len == 1) return x.leaf(l, slot);
      if (c == 0) {
        for (int j = r - 1; j >= l; --j) {
          int st = x.copy(-1, slot);
          if (!st) st = x.advance(-1, l, j - l);
          if (!st) st = x.leaf(j, -1);
          if (st) return st;
        }
        return 0;
      }
      const int m = plan.split(len, c);
      const int ns = plan.S - c;  // slots fill and free last in, first out
      int st = x.copy(ns, slot);
      if (!st) st = x.advance(ns, l, m);
      if (!st) st = rev(l + m, r, c - 1, ns);
      if (st) return st;
      r = l + m;
    }
  }

  int run() {
    const std::vector<int> p = plan.spine();
    const int K = (int)p.size() - 1;
    int st = rev(p[K], plan.n, plan.S - 1 - K, K);
    for (int k = K - 1; k >= 0 && !st; --k) st = rev(p[k], p[k + 1], plan.S - 1 - k, k);
    return st;
  }
};

}  // namespace apollo
