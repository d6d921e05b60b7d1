// The C ABI's exception barrier: run a body, map any exception to a status.
#pragma once

#include <exception>
#include <new>
#include <string>

#include "common.cuh"

namespace aphi_b200 {

// The calling thread's last error message. A plain character array, so that
// it stays usable while the process tears down: a caller may release handles
// from its own static destructors, after the thread's C++ thread_local
// objects have been destroyed.
constexpr int kLastErrorBytes = 1024;
extern thread_local char g_last_error[kLastErrorBytes];
void set_last_error(const char* msg);
inline void set_last_error(const std::string& msg) { set_last_error(msg.c_str()); }

template <class F>
int guard(F&& body) {
    try {
        body();
        g_last_error[0] = 0;
        return APHI_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc& e) {
        set_last_error(std::string("host allocation failed: ") + e.what());
        return APHI_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return APHI_ERR_INVALID;
    } catch (...) {
        set_last_error("unknown exception");
        return APHI_ERR_INVALID;
    }
}

}  // namespace aphi_b200
