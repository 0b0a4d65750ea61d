// Library-internal access to a job for the host loops (serve.cpp); not part of the C ABI.
#pragma once
#include <stdint.h>

#include "../../include/meikey_b200.h"

namespace mkjobs {

// the context a job was prepared on
mk_ctx* context_of(const mk_job* job);
// The host derivation of index `index` of the job's key stream tested against every needle
// of the job with the real x sign: writes the public key and the secret, sets *needle to the
// first needle that matches and returns 1, or returns 0 when none matches (-1 for an
// incremental start scalar at or above 2^255).  Touches no shared state.
int host_match(const mk_job* job, uint64_t index, uint8_t pk[32], uint8_t secret[32], uint32_t* needle);

}  // namespace mkjobs
