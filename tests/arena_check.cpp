// CPU check of the serving loop's device-memory arena (csrc/arena.h): random
// allocations and releases against a shadow list of live blocks.  Prints "ok"
// or the first violated invariant and exits non-zero.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "arena.h"

struct Blk { size_t off, size; };

int main() {
  wrt::Arena a;
  const size_t cap = (size_t)64 << 20;
  a.reset(cap);
  std::mt19937_64 rng(12345);
  std::vector<Blk> live;
  size_t used = 0;
  for (int step = 0; step < 200000; ++step) {
    const bool do_alloc = live.empty() || (rng() % 100) < 55;
    if (do_alloc) {
      const size_t want = 1 + rng() % ((rng() % 10 == 0) ? (8u << 20) : (64u << 10));
      std::vector<size_t> probe = {want};
      const bool predicted = a.fits(probe.begin(), probe.end());
      size_t off = 0;
      const bool ok = a.alloc(want, &off);
      if (ok != predicted) { printf("fits() disagrees with alloc() at step %d\n", step); return 1; }
      if (!ok) continue;
      const size_t sz = wrt::Arena::round_up(want);
      if (off % wrt::Arena::kAlign || off + sz > cap) { printf("bad block %zu+%zu\n", off, sz); return 1; }
      for (const Blk &b : live)
        if (off < b.off + b.size && b.off < off + sz) { printf("overlap at step %d\n", step); return 1; }
      live.push_back({off, sz});
      used += sz;
    } else {
      const size_t k = rng() % live.size();
      if (!a.release(live[k].off)) { printf("release refused a live block\n"); return 1; }
      used -= live[k].size;
      live[k] = live.back();
      live.pop_back();
    }
    if (a.used() != used || a.live_blocks() != live.size()) { printf("accounting off at step %d\n", step); return 1; }
  }
  if (a.release(1)) { printf("released a non-block\n"); return 1; }
  for (const Blk &b : live) a.release(b.off);
  if (a.used() != 0 || a.free_blocks() != 1 || a.largest_free() != cap) {
    printf("did not coalesce back to one block: %zu free blocks\n", a.free_blocks());
    return 1;
  }
  printf("ok peak=%zu\n", a.peak());
  return 0;
}
