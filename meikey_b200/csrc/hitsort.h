// Candidate hits in (index, needle) order.  A launch's hits lie in a bounded index range and
// arrive nearly in order, so large sets are first distributed into buckets of about 32 by
// the top bits of (index - lowest index), in one counting pass and one scatter, and each
// bucket is then sorted on its own.
#pragma once
#include <stdint.h>

#include <string.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "../../include/meikey_b200.h"

namespace mkhits {

inline bool less(const mk_hit& a, const mk_hit& b) {
    return a.index != b.index ? a.index < b.index : a.needle < b.needle;
}

inline void sort_hits(mk_hit* v, size_t n) {
    if (n < 4096) {
        std::sort(v, v + n, less);
        return;
    }
    uint64_t lo = ~0ull, hi = 0;
    for (size_t i = 0; i < n; i++) {
        const mk_hit& h = v[i];
        lo = std::min(lo, h.index);
        hi = std::max(hi, h.index);
    }
    // one bucket per ~32 records, on the top bits of (index - lo)
    int bb = 0;
    while (bb < 20 && (size_t(1) << bb) < n / 32) bb++;
    int shift = 0;
    while (shift < 64 && ((hi - lo) >> shift) >= (uint64_t(1) << bb)) shift++;
    const size_t nb = size_t(1) << bb;
    std::vector<uint32_t> start(nb + 1, 0);
    for (size_t i = 0; i < n; i++) start[((v[i].index - lo) >> shift) + 1]++;
    for (size_t b = 0; b < nb; b++) start[b + 1] += start[b];
    std::vector<mk_hit> out(n);
    {
        std::vector<uint32_t> next(start.begin(), start.end() - 1);
        for (size_t i = 0; i < n; i++) out[next[(v[i].index - lo) >> shift]++] = v[i];
    }
    for (size_t b = 0; b < nb; b++)
        if (start[b + 1] - start[b] > 1) std::sort(out.begin() + start[b], out.begin() + start[b + 1], less);
    memcpy(v, out.data(), n * sizeof(mk_hit));
}

inline void sort_hits(std::vector<mk_hit>& v) { sort_hits(v.data(), v.size()); }

// The hits of a job's last launch: records are copied straight into it from the device, and
// growing it does not zero-fill.  `scratch` serves per-needle selections.  A released job's
// buffer goes back to its context for the next job, so its pages are already mapped.
struct HitBuf {
    std::unique_ptr<mk_hit[]> p;
    size_t n = 0, cap = 0;
    std::vector<uint64_t> scratch;
    void clear() { n = 0; }
    // room for m records; the old contents are dropped when it grows
    void resize_uninit(size_t m) {
        if (m > cap) {
            p.reset(new mk_hit[m]);
            cap = m;
        }
        n = m;
    }
    mk_hit* data() { return p.get(); }
    const mk_hit* data() const { return p.get(); }
};

}  // namespace mkhits
