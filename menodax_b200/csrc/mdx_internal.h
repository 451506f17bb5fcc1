// Internal entry points shared by the translation units of the native library.
// Not part of the C ABI.
#pragma once
#include "../../include/menodax.h"

namespace mdx_internal {

// mdx_solve with `counter` (when not NULL) as the persistent kernel's queue head
// in place of the caller's workspace.
int solve_with_counter(mdx_plan* plan, const mdx_solve_desc* desc, void* stream, int* counter);

// The device of the calling thread's current CUDA context, whether that
// context is the device's primary context, and (when ctx_id is not NULL) the
// context's process-unique ID.  Fails when no context is current.
int current_device(int* device, bool* is_primary, unsigned long long* ctx_id = nullptr);

// Record `message` as the calling thread's last error and return `code`.
int fail_message(int code, const char* message);

}  // namespace mdx_internal
