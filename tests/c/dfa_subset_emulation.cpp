// CPU restatement of the device DFA builder's algorithm (k_dfa_build in dfa_build.cu) over the
// NFA tables the host exports for it (mkre::nfa_tables), checked against the host compiler
// (mk_regex_compile).  The device kernel resolves the successors of DFA_CHUNK (state, value)
// pairs of a frontier against the states found so far, then numbers the new sets in (state,
// value) order; this program runs the same steps one pair at a time and compares status, error
// text, state count and table bytes for every pattern read from stdin, one per line:
// "<case_sensitive 0|1> <max_states> <pattern>".  Prints the count of differences.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <string>
#include <vector>

#include "meikey_b200.h"
#include "../../meikey_b200/csrc/regex.h"

namespace {

const uint32_t CHUNK = 4096;

typedef std::vector<uint32_t> Set;  // words of the NFA set, then the flags word

// successor of state k on value v: 0 for the accept state, else -1 with the set in `out`
int step(const mkre::NfaTables& t, const std::vector<Set>& keys, uint32_t k, uint32_t v, Set& out) {
    const uint32_t W = t.words;
    const Set& S = keys[k];
    const bool first = k == 0, prev_word = (S[W] & 1u) != 0, word = v < 62;
    Set C(W, 0), nx(W, 0);
    if (t.track_word) {
        const uint32_t c = (first ? 4u : 0u) | (prev_word ? 2u : 0u) | (word ? 1u : 0u);
        for (uint32_t i = 0; i < W; i++)
            if (S[i] & t.decm[c * W + i]) return 0;
        for (uint32_t i = 0; i < W; i++)
            for (uint32_t b = S[i]; b; b &= b - 1) {
                const size_t s = i * 32 + __builtin_ctz(b);
                for (uint32_t j = 0; j < W; j++) C[j] |= t.dec[(c * (size_t)t.n + s) * W + j];
            }
    } else {
        for (uint32_t i = 0; i < W; i++) C[i] = S[i];
        if ((C[t.match >> 5] >> (t.match & 31)) & 1u) return 0;
    }
    nx[t.start >> 5] |= 1u << (t.start & 31);
    for (uint32_t i = 0; i < W; i++)
        for (uint32_t b = C[i]; b; b &= b - 1) {
            const uint32_t s = i * 32 + __builtin_ctz(b);
            const int32_t to = t.sym_to[s];
            if (to >= 0 && ((t.sym[s] >> v) & 1ull)) nx[to >> 5] |= 1u << (to & 31);
        }
    for (uint32_t i = 0; i < W; i++)
        if (nx[i] & t.plainm[i]) return 0;
    out.assign(W + 1, 0);
    for (uint32_t i = 0; i < W; i++)
        for (uint32_t b = nx[i]; b; b &= b - 1) {
            const size_t s = i * 32 + __builtin_ctz(b);
            for (uint32_t j = 0; j < W; j++) out[j] |= t.plain[s * W + j];
        }
    out[W] = t.track_word && word ? 1u : 0u;
    return -1;
}

// MK_OK with the table, or MK_ERR_PATTERN with the text in *err
int build(const mkre::NfaTables& t, uint32_t max_states, std::vector<uint8_t>& table, uint32_t& states,
          std::string* err) {
    const uint32_t W = t.words;
    std::vector<Set> keys;
    std::map<Set, int> ids;
    Set k0(t.k0);
    k0.push_back(t.track_start ? 2u : 0u);
    keys.push_back(k0);
    ids[k0] = 1;
    std::vector<uint16_t> rows((size_t)max_states * 65, 0);
    for (uint32_t lo = 0; lo < keys.size();) {
        const uint32_t hi = (uint32_t)keys.size();
        for (uint32_t k = lo; k < hi; k++) {
            const uint32_t c = (k == 0 ? 2u : 0u) | (keys[k][W] & 1u);
            bool eoi = false;
            for (uint32_t i = 0; i < W; i++) eoi |= (keys[k][i] & t.endm[c * W + i]) != 0;
            rows[(size_t)(k + 1) * 65 + 64] = eoi;
        }
        for (uint64_t base = (uint64_t)lo * 64; base < (uint64_t)hi * 64; base += CHUNK) {
            const uint32_t cnt = (uint32_t)std::min<uint64_t>(CHUNK, (uint64_t)hi * 64 - base);
            std::vector<Set> cand(cnt);
            std::vector<int> id(cnt);
            for (uint32_t i = 0; i < cnt; i++) {  // the parallel part: lookups of known states
                id[i] = step(t, keys, (uint32_t)((base + i) >> 6), (uint32_t)((base + i) & 63), cand[i]);
                if (id[i] < 0) {
                    auto it = ids.find(cand[i]);
                    if (it != ids.end()) id[i] = it->second;
                }
            }
            for (uint32_t i = 0; i < cnt; i++) {  // the numbering part, in (state, value) order
                if (id[i] >= 0) continue;
                auto it = ids.find(cand[i]);
                if (it != ids.end()) {
                    id[i] = it->second;
                    continue;
                }
                if (keys.size() + 2 > max_states) {
                    *err = mkre::too_complex(max_states);
                    return MK_ERR_PATTERN;
                }
                keys.push_back(cand[i]);
                id[i] = (int)keys.size();
                ids[cand[i]] = id[i];
            }
            for (uint32_t i = 0; i < cnt; i++) rows[(size_t)(((base + i) >> 6) + 1) * 65 + ((base + i) & 63)] = id[i];
        }
        lo = hi;
    }
    states = (uint32_t)keys.size() + 1;
    rows[64] = 1;  // the accept state accepts at the end of the input
    table.assign((size_t)states * 130, 0);
    for (size_t i = 0; i < (size_t)states * 65; i++) {
        table[2 * i] = (uint8_t)rows[i];
        table[2 * i + 1] = (uint8_t)(rows[i] >> 8);
    }
    return mkre::check_table(table.data(), states, err);
}

}  // namespace

int main() {
    int differ = 0, n = 0, built = 0;
    char line[4096];
    while (fgets(line, sizeof line, stdin)) {
        size_t len = strlen(line);
        if (len && line[len - 1] == '\n') line[--len] = 0;
        const char* sp = strchr(line + 2, ' ');
        if (len < 4 || !sp) continue;
        const int cs = line[0] == '1';
        const uint32_t max_states = (uint32_t)atoi(line + 2);
        const char* pattern = sp + 1;
        std::vector<uint8_t> host((size_t)max_states * 130);
        uint32_t host_states = 0;
        char host_err[256];
        const int hs = mk_regex_compile(pattern, cs, max_states, host.data(), &host_states, host_err, sizeof host_err);
        mkre::NfaTables t;
        std::string err;
        std::vector<uint8_t> dev;
        uint32_t dev_states = 0;
        int ds = mkre::nfa_tables(pattern, cs, 64, &t, &err);
        if (ds == MK_OK) ds = build(t, max_states, dev, dev_states, &err);
        n++;
        built += ds == MK_OK;
        const bool same = hs == ds && (hs != MK_OK ? err == host_err
                                                   : host_states == dev_states &&
                                                         memcmp(host.data(), dev.data(), (size_t)host_states * 130) == 0);
        if (!same) {
            differ++;
            printf("differs: cs=%d max=%u '%s' host %d/%u '%s' emulated %d/%u '%s'\n", cs, max_states, pattern, hs,
                   host_states, host_err, ds, dev_states, err.c_str());
        }
    }
    printf("%d patterns, %d built, %d differ\n", n, built, differ);
    return differ != 0;
}
