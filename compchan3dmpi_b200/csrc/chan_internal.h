// chan_internal.h -- calls between the solver (chanrhs.cu) and the closure
// MLP (closure.cu) translation units of libchanrhs.so.  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

struct chan_ctx;
struct chan_closure;

// Closure inputs and targets: 13 features (the 9 velocity gradients du_a/dx_b
// with a, b over (x, spanwise, wall-normal), the 3 temperature gradients and
// y+) and 9 subgrid fluxes (tau_uu, tau_vv, tau_ww, tau_uv, tau_uw, tau_vw,
// q_u, q_v, q_w).
constexpr int kClIn = 13, kClOut = 9;

// Append samples of the filtered state of context c to X [n][13] / T [n][9]
// (device arrays, room for `capacity` rows); *added receives the count.
// Sample points every (sx, sy, sz) grid points; box filter of width fw in
// x and spanwise.  Queued on the context's stream, which is synchronised.
int chan_internal_sample(chan_ctx *c, float *X, float *T, long long capacity, int sx, int sy, int sz, int fw,
                         long long *added);

// MLP inference on device arrays: Y [n][9] in physical units from X [n][13]
// (soa: X [13][n] and Y [9][n]); sets *flag (device) when a normalised output
// exceeds the closure's limit.  Queued on `stream`, not synchronised.
int chan_internal_infer(chan_closure *m, const float *X, float *Y, long long n, bool soa, cudaStream_t stream,
                        int *flag);
int chan_internal_closure_device(chan_closure *m);
