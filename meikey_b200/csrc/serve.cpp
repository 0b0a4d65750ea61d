// Host loops above the launch engine:
//
//   mk_search       the searcher of one job (Searcher::run over Engine, src/service/search.rs:33-40,
//                   src/service/gpu.rs:917-996): launches over consecutive ranges, confirms
//                   candidates on the host in index order, honours a tries budget, a time
//                   limit and a cancel request from the progress callback, returns only a
//                   host-verified key.
//   mk_server_*     continuous batching of many jobs (no counterpart in the reference): one
//                   candidate stream, every tick one launch that tests the needles of all
//                   admitted jobs; jobs are admitted at tick boundaries as needle slots and
//                   device memory free up, shortest expected search first.  A job admitted
//                   at stream index a searches [a, a + budget): its result is the lowest
//                   index there whose key matches (confirmed on the host) and that no other
//                   job has received, which is what mk_search of the same job from index a
//                   finds alone once the indices delivered before it are skipped.  One
//                   index (one secret) goes to one job only, as two runs of the reference
//                   never share a random key (src/service/gpu.rs:924-925).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/meikey_b200.h"
#include "abi_guard.h"
#include "hitsort.h"
#include "jobs.h"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Probability that a uniformly random key matches a DFA table over the 43 searched
// characters (the first of them takes 16 values, the others 64): the state distribution
// propagated character by character.
double dfa_match_probability(const uint8_t* table, uint32_t states) {
    std::vector<double> d(states, 0.0), nd(states);
    d[1 % states] = 1.0;
    auto next = [&](uint32_t s, uint32_t v) {
        size_t at = ((size_t)s * 65 + v) * 2;
        return (uint32_t)table[at] | (uint32_t)table[at + 1] << 8;
    };
    for (int pos = 0; pos < 43; pos++) {
        std::fill(nd.begin(), nd.end(), 0.0);
        const uint32_t values = pos == 0 ? 16 : 64;
        for (uint32_t s = 0; s < states; s++) {
            if (d[s] == 0.0) continue;
            const double w = d[s] / values;
            for (uint32_t v = 0; v < values; v++) nd[next(s, v)] += w;
        }
        d.swap(nd);
    }
    double p = d[0];
    for (uint32_t s = 1; s < states; s++)
        if (next(s, 64)) p += d[s];
    return p;
}

// All hits of the job's last launch (sorted by index).
int fetch_hits(mk_job* job, std::vector<mk_hit>& hits) {
    uint32_t written = 0;
    uint64_t total = 0;
    int st = mk_job_hits(job, nullptr, 0, &written, &total);
    if (st != MK_OK) return st;
    hits.resize(total);
    st = mk_job_hits(job, hits.data(), (uint32_t)total, &written, &total);
    if (st != MK_OK) return st;
    hits.resize(written);
    return MK_OK;
}

}  // namespace

extern "C" double mk_expected_tries(const mk_needle* nd) try {
    if (!nd || !nd->bytes || nd->len == 0) return 0.0;
    if (nd->mode == MK_MODE_REGEX) {
        double p = dfa_match_probability(nd->bytes, nd->len);
        return p > 0 ? 1.0 / p : INFINITY;
    }
    // text needles: the DFA of the escaped needle (suffix: anchored at the end)
    std::string rx;
    for (uint32_t i = 0; i < nd->len; i++) {
        char ch = (char)nd->bytes[i];
        if (ch == '+' || ch == '/') rx += '\\';
        rx += ch;
    }
    if (nd->mode == MK_MODE_SUFFIX) rx += '$';
    std::vector<uint8_t> table(4096 * 130);
    uint32_t states = 0;
    // a needle that no key can match (e.g. a 43-character one whose first character is not
    // among the 16 values of that position) is refused by the compiler
    if (mk_regex_compile(rx.c_str(), nd->fold ? 0 : 1, 4096, table.data(), &states, nullptr, 0) != MK_OK)
        return INFINITY;
    double p = dfa_match_probability(table.data(), states);
    return p > 0 ? 1.0 / p : INFINITY;
} catch (...) {
    return 0.0;
}

namespace {

// What stops a search loop from outside: the combinators' shared flag (a key was found by
// another searcher, or the caller cancelled), and the searched indices reported as they grow.
struct Shared {
    std::atomic<int>* cancel = nullptr;
    std::atomic<uint64_t>* tries = nullptr;
};

// The loop of Searcher::run over one job (src/service/gpu.rs:917-996): launches of cfg->iters
// iterations over cfg->first, first + keys_per_iter·iters, ...; after each launch its
// candidates are confirmed on the host in index order and the first that matches with its
// real x sign ends the search.  A set `cancel` ends it before the next launch, and a launch
// it cut short (the job's stop word) is not confirmed and not counted.
int search_loop(mk_job* job, const mk_search_config* cfg, mk_progress_fn progress, void* user, mk_outcome* out,
                const Shared& sh) {
    memset(out, 0, sizeof *out);
    const double t0 = now_s();
    const uint64_t kpi = mk_job_keys_per_iter(job);
    if (kpi == 0) return MK_ERR_BAD_ARG;
    // [first, end): at most max_tries indices, and never past the end of the 64-bit index space
    const uint64_t end = (cfg->max_tries && cfg->max_tries <= ~0ull - cfg->first) ? cfg->first + cfg->max_tries : ~0ull;
    uint64_t base = cfg->first;
    std::vector<mk_hit> hits;
    auto cancelled = [&] { return sh.cancel && sh.cancel->load() != 0; };
    for (;;) {
        if (cancelled()) {
            out->status = MK_ERR_STOPPED;
            return MK_OK;
        }
        const uint64_t left = end - base;  // > 0 here
        const uint64_t want = left / kpi + (left % kpi != 0);
        uint32_t iters = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(cfg->iters, want));
        int found = 0;
        uint64_t lowest = 0;
        int st = mk_job_launch(job, base, iters, &found, &lowest);
        // more candidates than the hit ring holds: the kept ones need not be the lowest, so
        // the same range is searched again in shorter launches (down to one iteration)
        while (st == MK_ERR_HIT_RING_FULL && iters > 1) {
            iters /= 2;
            st = mk_job_launch(job, base, iters, &found, &lowest);
        }
        if (st != MK_OK && st != MK_ERR_STOPPED) return st;
        if (cancelled()) {
            out->status = MK_ERR_STOPPED;
            out->elapsed_s = now_s() - t0;
            return MK_OK;
        }
        const uint64_t span = kpi * iters;
        if (found) {
            if (int e = fetch_hits(job, hits)) return e;
            const uint32_t written = (uint32_t)hits.size();
            for (uint32_t k = 0; k < written; k++) {
                const mk_hit& h = hits[k];
                if (h.index < base || h.index >= end) continue;
                int ok = 0;
                st = mk_job_confirm(job, h.index, h.needle, out->pk, out->secret, &ok);
                if (st != MK_OK) return st;
                if (ok) {
                    out->status = MK_OK;
                    out->index = h.index;
                    out->needle = h.needle;
                    out->tries = h.index - cfg->first + 1;
                    out->elapsed_s = now_s() - t0;
                    if (sh.tries) sh.tries->fetch_add(h.index - base + 1);
                    return MK_OK;
                }
            }
        }
        const bool wrapped = base + span < base;
        const uint64_t next = wrapped ? end : std::min(base + span, end);
        if (sh.tries) sh.tries->fetch_add(next - base);
        base = next;
        out->tries = base - cfg->first;
        out->elapsed_s = now_s() - t0;
        if (base >= end) {
            out->status = MK_ERR_STOPPED;  // budget spent without a confirmed key
            return MK_OK;
        }
        if (cfg->time_limit_s > 0 && out->elapsed_s >= cfg->time_limit_s) {
            out->status = MK_ERR_STOPPED;
            return MK_OK;
        }
        if (progress && progress(user, out->tries, out->elapsed_s)) {
            out->status = MK_ERR_STOPPED;  // cancelled
            return MK_OK;
        }
    }
}

// Runs `workers` (each returns a status and reports its tries into `tries`) on host threads
// of their own while the calling thread reports progress about every 100 ms (summed tries);
// a nonzero progress return, or the time limit, sets `cancel` and calls `stop_all`.  Returns
// the first worker error, MK_ERR_OUT_OF_MEMORY when a host thread could not start.
int run_workers(std::vector<std::function<int()>>& workers, std::atomic<int>& cancel, std::atomic<uint64_t>& tries,
                const std::function<void()>& stop_all, mk_progress_fn progress, void* user, double time_limit_s,
                double t0) {
    const size_t n = workers.size();
    std::vector<int> status(n, MK_OK);
    std::atomic<size_t> running{n};
    std::mutex mu;
    std::condition_variable cv;
    std::vector<std::thread> threads;
    bool started_all = true;
    try {
        threads.reserve(n);
        for (size_t k = 0; k < n; k++)
            threads.emplace_back([&, k] {
                int st = MK_OK;
                try {
                    st = workers[k]();
                } catch (...) {
                    st = mkabi::host_failure(nullptr);
                }
                status[k] = st;
                if (st != MK_OK && cancel.exchange(1) == 0) stop_all();
                std::lock_guard<std::mutex> lock(mu);
                running--;
                cv.notify_all();
            });
    } catch (...) {
        started_all = false;  // the host would not start another thread
        running -= n - threads.size();
        if (cancel.exchange(1) == 0) stop_all();
    }
    {
        std::unique_lock<std::mutex> lock(mu);
        while (running.load() > 0) {
            cv.wait_for(lock, std::chrono::milliseconds(100));
            if (running.load() == 0 || cancel.load()) continue;
            const double el = now_s() - t0;
            lock.unlock();
            const bool stop = (progress && progress(user, tries.load(), el)) || (time_limit_s > 0 && el >= time_limit_s);
            if (stop && cancel.exchange(1) == 0) stop_all();
            lock.lock();
        }
    }
    for (auto& t : threads) t.join();
    if (!started_all) return MK_ERR_OUT_OF_MEMORY;
    for (int st : status)
        if (st != MK_OK) return st;
    return MK_OK;
}

}  // namespace

extern "C" int mk_search(mk_job* job, const mk_search_config* cfg, mk_progress_fn progress, void* user,
                         mk_outcome* out) try {
    if (!job || !cfg || !out || cfg->iters == 0) return MK_ERR_BAD_ARG;
    return search_loop(job, cfg, progress, user, out, Shared{});
} MK_ABI_CATCH(nullptr)

extern "C" int mk_search_many(mk_job* const* jobs, uint32_t n, const mk_search_config* cfgs, mk_progress_fn progress,
                              void* user, mk_outcome* out, uint32_t* winner) try {
    if (!jobs || !cfgs || !out || !winner || n == 0 || n > 64) return MK_ERR_BAD_ARG;
    for (uint32_t k = 0; k < n; k++) {
        if (!jobs[k] || cfgs[k].iters == 0) return MK_ERR_BAD_ARG;
        for (uint32_t q = 0; q < k; q++)  // one host thread per context
            if (mkjobs::context_of(jobs[q]) == mkjobs::context_of(jobs[k])) return MK_ERR_BAD_ARG;
    }
    memset(out, 0, sizeof *out);
    *winner = n;
    const double t0 = now_s();
    std::atomic<int> cancel{0};
    std::atomic<uint64_t> tries{0};
    std::atomic<uint32_t> first_found{n};
    std::vector<mk_outcome> outs(n);
    auto stop_all = [&] {
        for (uint32_t q = 0; q < n; q++) mk_job_stop(jobs[q], 1);
    };
    std::vector<std::function<int()>> workers;
    for (uint32_t k = 0; k < n; k++)
        workers.push_back([&, k] {
            // the calling thread reports progress; the time limit is checked there too
            mk_search_config cfg = cfgs[k];
            cfg.time_limit_s = 0;
            int st = search_loop(jobs[k], &cfg, nullptr, nullptr, &outs[k], Shared{&cancel, &tries});
            if (st == MK_OK && outs[k].status == MK_OK) {
                uint32_t none = n;
                if (first_found.compare_exchange_strong(none, k)) {
                    cancel.store(1);
                    for (uint32_t q = 0; q < n; q++)
                        if (q != k) mk_job_stop(jobs[q], 1);
                }
            }
            return st;
        });
    int st = run_workers(workers, cancel, tries, stop_all, progress, user, cfgs[0].time_limit_s, t0);
    for (uint32_t q = 0; q < n; q++) mk_job_stop(jobs[q], 0);  // withdraw the stop requests
    const uint32_t w = first_found.load();
    if (w < n) {
        *out = outs[w];
        *winner = w;
    } else {
        out->status = MK_ERR_STOPPED;
    }
    out->tries = tries.load();
    out->elapsed_s = now_s() - t0;
    return st;
} MK_ABI_CATCH(nullptr)

extern "C" int mk_search_both(mk_job* job, const mk_search_config* cfg, uint32_t cpu_threads, uint64_t cpu_first,
                              mk_progress_fn progress, void* user, mk_outcome* out, uint32_t* winner) try {
    if (!job || !cfg || !out || !winner || cfg->iters == 0 || cpu_threads > 256) return MK_ERR_BAD_ARG;
    memset(out, 0, sizeof *out);
    *winner = 2;
    const double t0 = now_s();
    std::atomic<int> cancel{0};
    std::atomic<uint64_t> tries{0}, next_cpu{cpu_first};
    std::atomic<uint32_t> first_found{2};
    mk_outcome gpu_out{}, cpu_out{};
    cpu_out.status = MK_ERR_STOPPED;  // no host key yet (a zeroed outcome would read as MK_OK)
    std::mutex cpu_mu;
    auto stop_all = [&] { mk_job_stop(job, 1); };
    auto claim = [&](uint32_t who) {
        uint32_t none = 2;
        if (!first_found.compare_exchange_strong(none, who)) return false;
        cancel.store(1);
        if (who == 1) mk_job_stop(job, 1);
        return true;
    };
    std::vector<std::function<int()>> workers;
    workers.push_back([&] {
        mk_search_config c = *cfg;
        c.time_limit_s = 0;
        int st = search_loop(job, &c, nullptr, nullptr, &gpu_out, Shared{&cancel, &tries});
        if (st == MK_OK && gpu_out.status == MK_OK) claim(0);
        return st;
    });
    // CPU searchers: chunks of consecutive indices from cpu_first, the host derivation and a
    // full match (x sign known), the reference's Parallel worker (src/service/search.rs:195-317)
    const uint64_t CHUNK = 64;
    for (uint32_t t = 0; t < cpu_threads; t++)
        workers.push_back([&] {
            uint8_t pk[32], secret[32];
            while (!cancel.load()) {
                const uint64_t a = next_cpu.fetch_add(CHUNK);
                for (uint64_t i = a; i < a + CHUNK; i++) {
                    uint32_t needle = 0;
                    const int m = mkjobs::host_match(job, i, pk, secret, &needle);
                    if (m < 0) return (int)MK_ERR_BAD_ARG;
                    if (m == 1) {
                        tries.fetch_add(i - a + 1);
                        std::lock_guard<std::mutex> lock(cpu_mu);
                        if (first_found.load() == 2 && (cpu_out.status != MK_OK || i < cpu_out.index)) {
                            cpu_out.status = MK_OK;
                            cpu_out.index = i;
                            cpu_out.needle = needle;
                            memcpy(cpu_out.pk, pk, 32);
                            memcpy(cpu_out.secret, secret, 32);
                        }
                        claim(1);
                        return (int)MK_OK;
                    }
                }
                tries.fetch_add(CHUNK);
            }
            return (int)MK_OK;
        });
    int st = run_workers(workers, cancel, tries, stop_all, progress, user, cfg->time_limit_s, t0);
    mk_job_stop(job, 0);
    const uint32_t w = first_found.load();
    if (w == 0) *out = gpu_out;
    else if (w == 1) *out = cpu_out;
    else out->status = MK_ERR_STOPPED;
    *winner = w;
    out->tries = tries.load();
    out->elapsed_s = now_s() - t0;
    return st;
} MK_ABI_CATCH(nullptr)

// ---------------------------------------------------------------------------
// continuous batching
// ---------------------------------------------------------------------------

namespace {

struct ServedJob {
    uint64_t id = 0;
    uint32_t mode = 0, fold = 0;
    std::vector<uint8_t> bytes;
    uint32_t len = 0;
    double expected = 0;     // expected tries
    uint64_t admit = 0;      // stream index at admission
    uint64_t submitted_seq = 0;
    double device_bytes = 0; // device memory it holds while admitted (estimate at admission)
};

}  // namespace

struct mk_server {
    mk_ctx* ctx = nullptr;
    mk_job* job = nullptr;
    mk_server_options opt{};
    uint64_t pos = 0;         // next stream index
    uint64_t kpi = 0;
    uint64_t seq = 0;
    std::deque<ServedJob> queued;
    std::vector<ServedJob> active;  // slot order = needle order of the launch
    std::vector<mk_job_result> done;
    std::vector<mk_hit> hits;
    bool needles_dirty = true;
    // stream indices whose key went to a job: each goes to one job only (indices below every
    // admitted job's start and the stream position can never be hit again and are dropped)
    std::set<uint64_t> delivered;
};

static void to_needle(const ServedJob& j, mk_needle& nd) {
    nd.bytes = j.bytes.data();
    nd.len = j.len;
    nd.fold = j.fold;
    nd.mode = j.mode;
}

extern "C" int mk_server_create(mk_ctx* ctx, const uint8_t key[32], int seed_source, const mk_server_options* options,
                                uint64_t first, mk_server** out) try {
    if (!ctx || !key || !options || !out) return MK_ERR_BAD_ARG;
    const mk_server_options& o = *options;
    if (o.max_jobs == 0 || o.max_jobs > 128 || o.iters_per_tick == 0 || o.budget == 0) return MK_ERR_OUT_OF_RANGE;
    *out = nullptr;
    std::unique_ptr<mk_server> s(new (std::nothrow) mk_server);
    if (!s) return MK_ERR_OUT_OF_MEMORY;
    s->ctx = ctx;
    s->opt = o;
    s->pos = first;
    s->kpi = mk_keys_per_iter(ctx);
    int st = mk_job_prepare(ctx, key, seed_source, nullptr, 0, 0, &s->job);
    if (st != MK_OK) return st;
    *out = s.release();
    return MK_OK;
} MK_ABI_CATCH(nullptr)

extern "C" void mk_server_destroy(mk_server* s) try {
    if (!s) return;
    mk_job_destroy(s->job);
    delete s;
} MK_ABI_CATCH_VOID

extern "C" int mk_server_submit(mk_server* s, const mk_needle* nd, uint64_t id) try {
    if (!s || !nd || !nd->bytes || nd->len == 0) return MK_ERR_BAD_ARG;
    ServedJob j;
    j.id = id;
    j.mode = nd->mode;
    j.fold = nd->fold;
    j.len = nd->len;
    const size_t bytes = nd->mode == MK_MODE_REGEX ? (size_t)nd->len * 130 : nd->len;
    j.bytes.assign(nd->bytes, nd->bytes + bytes);
    // the needle must be valid on its own (checked now, so a bad one never blocks a tick)
    if (int st = mk_needles_check(nd, 1)) return st;
    j.expected = mk_expected_tries(nd);
    j.submitted_seq = s->seq++;
    s->queued.push_back(std::move(j));
    return MK_OK;
} MK_ABI_CATCH(nullptr)

// candidates expected per tick for a job (x sign unknown doubles the rate at worst)
static double hits_per_tick(const mk_server* s, const ServedJob& j) {
    const double span = (double)s->kpi * s->opt.iters_per_tick;
    return j.expected > 0 ? 2.0 * span / j.expected : span;
}

// hit-ring entries a job reserves: four times its expected candidates per tick, plus 64
static double ring_entries(const mk_server* s, const ServedJob& j) { return 4.0 * hits_per_tick(s, j) + 64.0; }

// Device memory a job holds while admitted: its reserved hit-ring records (16 bytes each),
// its DFA table (states x 130 bytes, 16-byte aligned) and its slot of the job state (64 bytes).
static double job_device_bytes(const mk_server* s, const ServedJob& j) {
    const double dfa = j.mode == MK_MODE_REGEX ? (double)(((size_t)j.len * 130 + 15) & ~(size_t)15) : 0.0;
    return 16.0 * ring_entries(s, j) + dfa + 64.0;
}

static int admit(mk_server* s) {
    if (s->queued.empty()) return MK_OK;
    // shortest expected search first; ties in submission order
    std::stable_sort(s->queued.begin(), s->queued.end(),
                     [](const ServedJob& a, const ServedJob& b) { return a.expected < b.expected; });
    double ring = 0, mem = 0;
    for (auto& a : s->active) {
        ring += ring_entries(s, a);
        mem += a.device_bytes;
    }
    std::vector<mk_needle> nds;
    for (auto it = s->queued.begin(); it != s->queued.end();) {
        if (s->active.size() >= s->opt.max_jobs) break;
        const double need = ring_entries(s, *it), bytes = job_device_bytes(s, *it);
        // a job waits until hit-ring entries and device memory free up (a job is always
        // admitted when none is active)
        const bool ring_full = s->opt.hit_capacity && ring + need > (double)s->opt.hit_capacity;
        const bool mem_full = s->opt.device_bytes && mem + bytes > (double)s->opt.device_bytes;
        if ((ring_full || mem_full) && !s->active.empty()) {
            ++it;
            continue;
        }
        // does it still fit the matcher's shift-and state / regex slots?
        nds.clear();
        for (auto& a : s->active) {
            mk_needle nd;
            to_needle(a, nd);
            nds.push_back(nd);
        }
        mk_needle nd;
        to_needle(*it, nd);
        nds.push_back(nd);
        if (mk_needles_check(nds.data(), (uint32_t)nds.size()) != MK_OK) {
            ++it;
            continue;
        }
        ServedJob j = std::move(*it);
        it = s->queued.erase(it);
        j.admit = s->pos;
        j.device_bytes = bytes;
        ring += need;
        mem += bytes;
        s->active.push_back(std::move(j));
        s->needles_dirty = true;
    }
    return MK_OK;
}

static void finish(mk_server* s, size_t slot, int status, uint64_t index, uint64_t tries, const uint8_t* pk,
                  const uint8_t* secret) {
    const ServedJob& j = s->active[slot];
    mk_job_result r{};
    r.id = j.id;
    r.status = status;
    r.admit_index = j.admit;
    r.index = index;
    r.tries = tries;
    r.expected_tries = j.expected;
    if (pk) memcpy(r.pk, pk, 32);
    if (secret) memcpy(r.secret, secret, 32);
    s->done.push_back(r);
}

extern "C" int mk_server_tick(mk_server* s, uint32_t* active, uint32_t* queued) try {
    if (!s) return MK_ERR_BAD_ARG;
    int st = admit(s);
    if (st) return st;
    if (s->active.empty()) {
        if (active) *active = 0;
        if (queued) *queued = (uint32_t)s->queued.size();
        return MK_OK;
    }
    std::vector<mk_needle> nds(s->active.size());
    for (size_t k = 0; k < s->active.size(); k++) to_needle(s->active[k], nds[k]);
    if (s->needles_dirty) {
        st = mk_job_update(s->job, nds.data(), (uint32_t)nds.size());
        if (st) return st;
        s->needles_dirty = false;
    }
    // one tick over [pos, pos + span); a hit-ring overflow re-runs the range in halves
    const uint64_t span = s->kpi * s->opt.iters_per_tick;
    std::vector<mk_hit> hits;
    std::vector<std::pair<uint64_t, uint32_t>> todo{{s->pos, s->opt.iters_per_tick}};
    while (!todo.empty()) {
        auto [b, it] = todo.back();
        todo.pop_back();
        int found = 0;
        uint64_t lowest = 0;
        st = mk_job_launch(s->job, b, it, &found, &lowest);
        if (st == MK_ERR_HIT_RING_FULL && it > 1) {
            todo.push_back({b + s->kpi * (it / 2), it - it / 2});
            todo.push_back({b, it / 2});
            continue;
        }
        if (st != MK_OK) return st;
        if (!found) continue;
        std::vector<mk_hit> part;
        if (int e = fetch_hits(s->job, part)) return e;
        hits.insert(hits.end(), part.begin(), part.end());
    }
    mkhits::sort_hits(hits);
    // per job, in index order: the first candidate that matches with its real x sign
    std::vector<char> closed(s->active.size(), 0);
    uint8_t pk[32], secret[32];
    for (const mk_hit& h : hits) {
        const size_t k = h.needle;
        if (k >= s->active.size() || closed[k]) continue;
        const ServedJob& j = s->active[k];
        if (h.index < j.admit || h.index >= j.admit + s->opt.budget) continue;
        // hits are in (index, slot) order: of two jobs matching one key, the one admitted
        // earlier receives it and the other goes on to its next candidate
        if (s->delivered.count(h.index)) continue;
        int ok = 0;
        st = mk_job_confirm(s->job, h.index, h.needle, pk, secret, &ok);
        if (st != MK_OK) return st;
        if (ok) {
            finish(s, k, MK_OK, h.index, h.index - j.admit + 1, pk, secret);
            closed[k] = 1;
            s->delivered.insert(h.index);
        }
    }
    s->pos += span;
    for (size_t k = 0; k < s->active.size(); k++) {
        const ServedJob& j = s->active[k];
        if (!closed[k] && s->pos >= j.admit + s->opt.budget) {
            finish(s, k, MK_ERR_STOPPED, 0, s->opt.budget, nullptr, nullptr);  // censored at the budget
            closed[k] = 1;
        }
    }
    size_t w = 0;  // keep the open jobs in slot order (no self-move: it would empty the needle bytes)
    for (size_t k = 0; k < s->active.size(); k++) {
        if (closed[k]) continue;
        if (w != k) s->active[w] = std::move(s->active[k]);
        w++;
    }
    if (w != s->active.size()) s->needles_dirty = true;
    s->active.resize(w);
    uint64_t low = s->pos;  // no job will search below this
    for (const ServedJob& j : s->active) low = std::min(low, j.admit);
    s->delivered.erase(s->delivered.begin(), s->delivered.lower_bound(low));
    if (active) *active = (uint32_t)s->active.size();
    if (queued) *queued = (uint32_t)s->queued.size();
    return MK_OK;
} MK_ABI_CATCH(nullptr)

extern "C" int mk_server_results(mk_server* s, mk_job_result* out, uint32_t cap, uint32_t* n) try {
    if (!s || !n || (cap && !out)) return MK_ERR_BAD_ARG;
    const uint32_t k = (uint32_t)std::min<size_t>(cap, s->done.size());
    for (uint32_t i = 0; i < k; i++) out[i] = s->done[i];
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return MK_OK;
} MK_ABI_CATCH(nullptr)

extern "C" uint64_t mk_server_position(const mk_server* s) { return s ? s->pos : 0; }
