// Staged autotuner over kernel options (the reference's measure / fastest / fastest_staged,
// src/service/gpu.rs:302-393 and 1016-1113), written against the library's own C ABI.
//
// Stage 1 creates a context for every candidate with the self-check on, so a variant whose
// keys differ from the host derivation is dropped (MK_ERR_SELF_CHECK), and times one launch
// of about `trial_keys` candidates after a warm-up launch: of a fixed secure-path job
// (mk_autotune) or of the caller's own job (mk_autotune_job: seed source, key and needles,
// since the best options depend on the matching work, e.g. inverter_rotates for many needles).  Stage 2 keeps the
// `finalists` fastest, holds their contexts together and times them in rounds of
// alternating order (forward, backward, forward), keeping each one's best rate, so that a
// drift of the clock over the sweep does not favour whichever ran first.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/meikey_b200.h"
#include "abi_guard.h"

namespace {

// a fixed secure-path job: ChaCha20 seeds and one 7-character case-sensitive needle
const uint8_t TUNE_KEY[32] = {0x74, 0x75, 0x6e, 0x65, 0x2d, 0x6b, 0x65, 0x79, 0x01, 0x23, 0x45, 0x67, 0x89, 0xab, 0xcd, 0xef,
                              0x10, 0x32, 0x54, 0x76, 0x98, 0xba, 0xdc, 0xfe, 0x0f, 0x1e, 0x2d, 0x3c, 0x4b, 0x5a, 0x69, 0x78};
const char TUNE_NEEDLE[] = "8or5lx1";

struct Live {
    mk_ctx* ctx = nullptr;
    mk_job* job = nullptr;
};

// the job every candidate is timed on
struct TrialJob {
    const uint8_t* key;
    int source;
    const mk_needle* needles;
    uint32_t n_needles;
};

int open_entry(int device, const mk_options& o, const TrialJob& tj, Live& lv) {
    mk_options opt = o;
    opt.self_check = 1;
    int st = mk_ctx_create(device, &opt, &lv.ctx);
    if (st != MK_OK) {
        mk_ctx_destroy(lv.ctx);
        lv.ctx = nullptr;
        return st;
    }
    st = mk_job_prepare(lv.ctx, tj.key, tj.source, tj.needles, tj.n_needles, 0, &lv.job);
    if (st != MK_OK) {
        mk_ctx_destroy(lv.ctx);
        lv.ctx = nullptr;
    }
    return st;
}

void close_entry(Live& lv) {
    mk_job_destroy(lv.job);
    mk_ctx_destroy(lv.ctx);
    lv = Live{};
}

// keys/s of one launch of about `keys` candidates starting at `base`
int time_launch(Live& lv, uint64_t keys, uint64_t base, double* rate) {
    const uint64_t kpi = mk_keys_per_iter(lv.ctx);
    const uint32_t iters = (uint32_t)std::max<uint64_t>(1, (keys + kpi - 1) / kpi);
    int st = mk_ctx_record(lv.ctx, 14);
    if (!st) st = mk_job_enqueue(lv.job, base, iters);
    if (!st) st = mk_ctx_record(lv.ctx, 15);
    float ms = 0;
    if (!st) st = mk_ctx_elapsed(lv.ctx, 14, 15, &ms);
    if (st) return st;
    *rate = ms > 0 ? (double)(kpi * iters) / (ms * 1e-3) : 0.0;
    return MK_OK;
}

}  // namespace

static int autotune(int device, mk_tune_entry* entries, uint32_t n, uint32_t finalists, uint64_t trial_keys,
                    const TrialJob& tj, uint32_t* best) {
    if (!entries || !best || n == 0 || trial_keys == 0) return MK_ERR_BAD_ARG;
    uint64_t base = 1ull << 50;
    // stage 1
    for (uint32_t i = 0; i < n; i++) {
        mk_tune_entry& e = entries[i];
        e.stage = 1;
        e.keys_per_s = 0;
        Live lv;
        e.status = open_entry(device, e.options, tj, lv);
        if (e.status != MK_OK) continue;
        double warm = 0, rate = 0;
        e.status = time_launch(lv, trial_keys / 4, base, &warm);
        base += trial_keys;
        if (e.status == MK_OK) e.status = time_launch(lv, trial_keys, base, &rate);
        base += 2 * trial_keys;
        e.keys_per_s = rate;
        close_entry(lv);
    }
    std::vector<uint32_t> order;
    for (uint32_t i = 0; i < n; i++)
        if (entries[i].status == MK_OK) order.push_back(i);
    if (order.empty()) return MK_ERR_NO_SETTINGS;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return entries[a].keys_per_s > entries[b].keys_per_s; });
    if (finalists > 1 && order.size() > 1) {
        order.resize(std::min<size_t>(order.size(), finalists));
        std::vector<Live> live(order.size());
        int st = MK_OK;
        for (size_t k = 0; k < order.size() && st == MK_OK; k++) {
            st = open_entry(device, entries[order[k]].options, tj, live[k]);
            entries[order[k]].stage = 2;
            entries[order[k]].keys_per_s = 0;
        }
        for (int round = 0; round < 3 && st == MK_OK; round++) {
            for (size_t q = 0; q < order.size() && st == MK_OK; q++) {
                const size_t k = (round & 1) ? order.size() - 1 - q : q;
                double rate = 0;
                st = time_launch(live[k], 2 * trial_keys, base, &rate);
                base += 2 * trial_keys;
                entries[order[k]].keys_per_s = std::max(entries[order[k]].keys_per_s, rate);
            }
        }
        for (auto& lv : live) close_entry(lv);
        if (st != MK_OK) return st;
        std::sort(order.begin(), order.end(),
                  [&](uint32_t a, uint32_t b) { return entries[a].keys_per_s > entries[b].keys_per_s; });
    }
    *best = order[0];
    return MK_OK;
}

extern "C" int mk_autotune(int device, mk_tune_entry* entries, uint32_t n, uint32_t finalists, uint64_t trial_keys,
                           uint32_t* best) try {
    const mk_needle nd{(const uint8_t*)TUNE_NEEDLE, (uint32_t)strlen(TUNE_NEEDLE), 0, MK_MODE_CONTAINS};
    return autotune(device, entries, n, finalists, trial_keys, TrialJob{TUNE_KEY, MK_SEED_CHACHA20, &nd, 1}, best);
} MK_ABI_CATCH(nullptr)

extern "C" int mk_autotune_job(int device, mk_tune_entry* entries, uint32_t n, uint32_t finalists, uint64_t trial_keys,
                               const uint8_t key[32], int seed_source, const mk_needle* needles, uint32_t n_needles,
                               uint32_t* best) try {
    if (!key || (n_needles && !needles)) return MK_ERR_BAD_ARG;
    return autotune(device, entries, n, finalists, trial_keys, TrialJob{key, seed_source, needles, n_needles}, best);
} MK_ABI_CATCH(nullptr)
