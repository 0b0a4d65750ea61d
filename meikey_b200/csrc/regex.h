// Host side of the device DFA builder (mk_regex_compile_device): a pattern's Thompson NFA
// flattened into the tables the subset construction on the GPU reads (dfa_build.cu), and the
// checks on a finished table.  The construction is the one mk_regex_compile runs on the
// host, so both give the same table.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace mkre {

// NFA of a pattern for the subset construction: n states, sets of states as bitsets of
// `words` 32-bit words.  A DFA state is a set S (closed over plain epsilon edges) with two
// flags: bit 0 the previous character was a word character (kept only when the pattern has
// word assertions), bit 1 nothing has been read yet (kept only when start assertions can be
// reached through word assertions).
struct NfaTables {
    uint32_t n = 0, words = 0;
    int start = 0, match = 0;
    bool track_word = false, track_start = false;
    std::vector<uint32_t> k0;      // [words] the start state's set; its flags are 2·track_start
    std::vector<int32_t> sym_to;   // [n] target of the state's symbol edge, -1 for none
    std::vector<uint64_t> sym;     // [n] base64 values on that edge
    std::vector<uint32_t> plain;   // [n][words] closure of each state over plain edges
    std::vector<uint32_t> plainm;  // [words] states whose plain closure holds the match state
    // track_word only: closure of each state with the assertions decided for context
    // c = 4·first + 2·previous-is-word + next-is-word (the next character known)
    std::vector<uint32_t> dec;     // [8][n][words]
    std::vector<uint32_t> decm;    // [8][words] states whose decided closure holds the match state
    // states whose closure at the end of the input, context 2·first + previous-is-word, holds
    // the match state
    std::vector<uint32_t> endm;    // [4][words]
};

// Parses `pattern` (the dialect of mk_regex_compile) and builds its tables.  MK_OK, or
// MK_ERR_PATTERN with the message in *err (the same messages as mk_regex_compile, plus one
// for an NFA of more than 32·max_words states).
int nfa_tables(const char* pattern, int case_sensitive, uint32_t max_words, NfaTables* out, std::string* err);

// MK_ERR_PATTERN (message in *err) when no public key can match the table of `states` rows.
int check_table(const uint8_t* table, uint32_t states, std::string* err);

// The error text of a DFA with more than max_states states.
std::string too_complex(uint32_t max_states);

}  // namespace mkre
