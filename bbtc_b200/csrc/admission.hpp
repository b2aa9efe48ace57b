// Admission policy of the request server (server.cu), kept free of CUDA so
// that it can be compiled and tested on its own.
//
// A loader takes, among the pending requests that the HBM budget admits (or
// that can never fit, so that they fail at once), the oldest one that has
// waited its class's aging time or more (`small_aging_ns` for small requests,
// `aging_ns` for large ones), else the one with the fewest edges: small
// requests overtake large loads, large ones are not starved, and a small
// request is not passed over by smaller ones for longer than its aging time.
// A loader reserved for small requests sees only those.  No counterpart in the
// reference, which counts one graph per process.
#pragma once
#include <cstddef>
#include <cstdint>

namespace bbtc {

struct AdmitLimits {
  uint64_t budget;       // device bytes admitted requests may hold
  uint64_t in_use;       // bytes held now
  uint64_t small_edges;  // a request of at most this many edges is small
  uint64_t aging_ns;     // waited this long: taken before smaller ones
  uint64_t now_ns;
  bool small_only;       // the loader takes small requests only
  size_t scan_limit;     // pending requests looked at
  bool large_ok = true;  // false: as many large requests are loading as the server allows at once
  uint64_t small_aging_ns = 0;  // a small request waiting this long is taken before smaller ones (0: aging_ns)
};

// Index in `pending` (a random-access sequence of pointers to objects with
// fields m, reserved and t_submit, oldest first) of the request to load, or
// SIZE_MAX when none may be loaded now.
template <class Seq>
size_t admit_pick(const Seq& pending, const AdmitLimits& lim) {
  size_t best = SIZE_MAX;
  const size_t n = pending.size() < lim.scan_limit ? pending.size() : lim.scan_limit;
  for (size_t i = 0; i < n; i++) {
    const auto* r = pending[i];
    if ((lim.small_only || !lim.large_ok) && r->m > lim.small_edges) continue;
    const bool never = r->reserved > lim.budget;
    if (!never && lim.in_use + r->reserved > lim.budget && lim.in_use != 0) continue;
    const uint64_t aging = r->m <= lim.small_edges && lim.small_aging_ns ? lim.small_aging_ns : lim.aging_ns;
    if (lim.now_ns - r->t_submit >= aging) return i;
    if (best == SIZE_MAX || r->m < pending[best]->m) best = i;
  }
  return best;
}

}  // namespace bbtc
