// Structures shared by the host runtime and the device kernels.
#pragma once
#include <stdint.h>

namespace mkb {

// Comb geometry for the fixed-base multiply.
//
// A clamped scalar is s = 2^254 + 8·m with m = bits 3..253 (251 bits), so
// s·B = 2^254·B + Σ_i d_i · (2^(off_i) · 8B) where d_i are the digits of m.
// Rows 0..rows-2 use signed digits in [-2^(w-1), 2^(w-1)) with a carry into the next
// row; the top row's digit is unsigned in [0, 2^w_top] and its entries include the
// 2^254·B term.  Row i holds entries k·2^(off_i)·8B for k = 0..cols_i-1.
constexpr int MAX_ROWS = 64;  // 63 rows of 4-bit digits at most

struct CombGeom {
    uint32_t rows;
    uint32_t width[MAX_ROWS];
    uint32_t offset[MAX_ROWS];   // bit offset of digit i inside m
    uint64_t row_base[MAX_ROWS]; // first entry of row i
    uint64_t cols[MAX_ROWS];
    uint64_t entries;
};

// Words per table entry: (y+x, y-x, 2dxy) canonical, 8 little-endian u32 each.
constexpr int ENTRY_WORDS = 24;
// Comb-table entries sit 128 bytes apart (the last 32 bytes unused), so that every gather
// reads exactly one aligned 128-byte line instead of straddling two half of the time.
constexpr int COMB_STRIDE_WORDS = 32;

// Matcher: up to MAX_NEEDLES needles tested in one pass.
//   text needles (contains / suffix, fold): bit-parallel shift-and over the 43 searched
//   base64 characters; needle n occupies bits [bit0, bit0+len) of a multi-word state.
//   regex needles: DFA walk over a states×65×u16 table in device memory.
constexpr int MAX_NEEDLES = 128;
constexpr int SA_WORDS = 8;  // shift-and state words (512 bits of concatenated needles)

struct MatchSet {
    uint32_t n_text;              // text needles packed into the shift-and state
    uint32_t n_regex;             // regex needles
    uint32_t sa_words;            // words of shift-and state in use
    uint32_t short_words;         // with gram4: the leading words, holding the needles shorter than 4
                                  // characters, that every key scans; the rest only when gram4 fires
    uint32_t narrow;              // 1: the text needles fit in 32 bits of state (word 0, low half)
    // shift-and: per word and value v (0..63) the bits of needle positions accepting v.  Word
    // major, so that the 32 lanes' reads of one word at different values spread over the
    // shared-memory banks (value major, a row of 64 bytes put every lane on bank 0 or 16)
    uint64_t mask[SA_WORDS][64];
    uint64_t first_bit[SA_WORDS]; // bit 0 of every text needle (set on each step)
    uint64_t last_bit[SA_WORDS];  // last bit of every contains-needle
    uint64_t suffix_bit[SA_WORDS];// last bit of every suffix-needle (tested at the end only)
    uint16_t text_id[MAX_NEEDLES];// caller's needle index per text needle
    uint16_t text_last[MAX_NEEDLES]; // global bit index of each text needle's last bit
    // regex needles
    const uint8_t* dfa[16];
    uint32_t dfa_states[16];
    uint16_t regex_id[16];
    // prefilter of the text needles of 4 or more characters (null: none): bit g of 2^24 is set
    // when some such needle starts with the 4 base64 values g = v0<<18 | v1<<12 | v2<<6 | v3
    // (all case variants of a folded needle)
    const uint32_t* gram4;
};

constexpr uint32_t GRAM4_WORDS = 1u << 19;  // 2^24 bits
constexpr uint32_t GRAM4_MIN_NEEDLES = 8;   // long text needles from which a job uses the prefilter

struct HitRecord {
    uint64_t index;
    uint32_t needle;
    uint32_t reserved;
};

// Device-side job state for one launch.
struct JobDevice {
    uint32_t hit_count;     // total hits found (may exceed capacity)
    uint32_t status;        // 0 ok, bit 0: stopped on the stop word
    uint32_t stop;          // host-writable stop word (nonzero stops at the next iteration)
    uint32_t pad;
};

}  // namespace mkb
