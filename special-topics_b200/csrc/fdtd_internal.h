// fdtd_internal.h -- what the library's translation units share and do not
// export: the thread-local error message behind fdtd_last_error() and the
// device port traces of a handle.
#pragma once

struct fdtd_ctx;

// Records `msg` as this thread's last error and returns `code`.
__attribute__((visibility("hidden"))) int fdtd_internal_fail(int code, const char* msg);

// Device port traces of a handle: V and I are [probes][nsteps] FP64 arrays;
// *steps = completed steps.  Returns 0, or a status code (and message) when
// the handle has no voltage or no current probe.
__attribute__((visibility("hidden"))) int fdtd_internal_traces(const fdtd_ctx* c, const double** V,
                                                               const double** I, int* nsteps, int* steps,
                                                               int* device);
