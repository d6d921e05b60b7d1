// The C ABI's exception barrier: run a body, map any exception to a status.
#pragma once

#include <exception>
#include <new>
#include <string>

#include "common.cuh"

namespace aphi_b200 {

extern thread_local std::string g_last_error;

template <class F>
int guard(F&& body) {
    try {
        body();
        g_last_error.clear();
        return APHI_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.status;
    } catch (const std::bad_alloc& e) {
        g_last_error = std::string("host allocation failed: ") + e.what();
        return APHI_ERR_OOM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return APHI_ERR_INVALID;
    } catch (...) {
        g_last_error = "unknown exception";
        return APHI_ERR_INVALID;
    }
}

}  // namespace aphi_b200
