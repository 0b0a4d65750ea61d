// C++ exceptions never cross the C ABI.  Every entry point that can allocate host memory or
// start a host thread runs its body in a function-try-block whose handler turns the
// exception into a status: a host allocation or thread that could not be had is
// MK_ERR_OUT_OF_MEMORY (a Rust or ctypes caller would otherwise see the process abort).
#pragma once
#include <new>
#include <string>
#include <system_error>

#include "../../include/meikey_b200.h"

namespace mkabi {

// Status of the exception being handled; its text goes to *msg when msg is not null.
inline int host_failure(std::string* msg) noexcept {
    const char* what = "host resources exhausted";
    try {
        throw;
    } catch (const std::bad_alloc&) {
        what = "host allocation failed";
    } catch (const std::system_error&) {
        what = "a host thread or resource could not be had";
    } catch (...) {
    }
    if (msg) {
        try {
            *msg = what;
        } catch (...) {
        }
    }
    return MK_ERR_OUT_OF_MEMORY;
}

}  // namespace mkabi

// handler of an entry point returning a status (errp: the context's error text, or null)
#define MK_ABI_CATCH(errp) \
    catch (...) {          \
        return mkabi::host_failure(errp); \
    }
// handler of an entry point without a status (a release: nothing is left to report)
#define MK_ABI_CATCH_VOID \
    catch (...) {         \
    }
