// Host-side order of candidate hits (csrc/hitsort.h) against std::sort on the same records:
// random sets around the radix path's size threshold, duplicates of one index with several
// needles, one-index sets (every digit constant), and index ranges wide enough for the
// comparison-sort fallback.  Prints "ok <case>" per case; exit status 1 on a difference.
#include <stdio.h>

#include <algorithm>
#include <random>
#include <vector>

#include "../../meikey_b200/csrc/hitsort.h"

static int check(const char* name, std::vector<mk_hit> v) {
    std::vector<mk_hit> want = v;
    std::stable_sort(want.begin(), want.end(), mkhits::less);
    mkhits::sort_hits(v);
    for (size_t i = 0; i < v.size(); i++)
        if (v[i].index != want[i].index || v[i].needle != want[i].needle) {
            printf("FAIL %s at %zu\n", name, i);
            return 1;
        }
    printf("ok %s\n", name);
    return 0;
}

int main() {
    std::mt19937_64 rng(7);
    int bad = 0;
    const size_t sizes[] = {0, 1, 4095, 4096, 100000, 3000000};
    for (size_t n : sizes) {
        std::vector<mk_hit> v(n);
        const uint64_t base = rng();
        for (auto& h : v) h = mk_hit{base / 2 + rng() % (1ull << 31), (uint32_t)(rng() % 137), 0};
        char name[64];
        snprintf(name, sizeof name, "random n=%zu", n);
        bad += check(name, v);
    }
    {
        std::vector<mk_hit> v(50000);
        for (auto& h : v) h = mk_hit{1ull << 40, (uint32_t)(rng() % 9), 0};  // one index, many needles
        bad += check("one index", v);
        for (auto& h : v) h = mk_hit{12345, 3, 0};  // every key equal
        bad += check("all equal", v);
    }
    {
        std::vector<mk_hit> v(20000);
        for (auto& h : v) h = mk_hit{rng(), (uint32_t)(rng() % 200), 0};  // full 64-bit range: fallback
        bad += check("wide range", v);
        for (size_t i = 0; i < v.size(); i++) v[i] = mk_hit{~0ull - i % 5000, (uint32_t)(i % 7), 0};
        bad += check("top of the index space", v);
    }
    {
        // nearly sorted, as a ring written iteration by iteration is
        std::vector<mk_hit> v(200000);
        for (size_t i = 0; i < v.size(); i++) v[i] = mk_hit{(uint64_t)i * 37 + rng() % 4000, (uint32_t)(rng() % 72), 0};
        bad += check("nearly sorted", v);
    }
    return bad ? 1 : 0;
}
