// Device side of the serving loop (serve3d.cu): the request slot table and
// the kernel that keeps every admitted solve's windows, convergence test and
// gradual start on the device, so that the loop over sampling periods runs
// on the GPU without the host.
//
// One launch of the serving graph is a conditional while-loop (a CUDA graph
// conditional node) whose body is one sampling period of the batch: the
// steps of every member (sample_every steps), the fixed-order force sums of
// that period's sample, and serve_period_kernel.  The kernel folds each
// running slot's sample into its window, applies the slot's rule (windows
// until |delta Cd| < tolerance - and, when asked, force ranges within the
// reference's steady bound - or the cap, or a fixed run length), writes the
// slot's inlet velocity for the next period while its gradual start lasts,
// and ends the loop after the period in which a slot finished, after a bound
// on periods per launch, or when the host raised its flag (new solves wait
// to join).  The host then reads the table back once, retires the finished
// solves, joins the new ones and launches the graph again.
//
// Every sum and quotient is an unfused binary64 operation, so a slot's
// results are the same for any mix and any split of the run into launches.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "orrery_lbm.h"

namespace orr {

// One admitted solve (in the batch's member order).
struct ServeSlot {
    // Set at admission.
    double qa;              // 1/2 rho U^2 A: Cd = Fx / qa
    double length;          // reference length: Cm = Mz / (qa L)
    double centre[2];       // moment centre (x, y) of the pitching moment about z
    double tolerance;       // on |delta Cd| between consecutive windows
    double steady_range;    // > 0: window force ranges within steady_range |mean Fx| to settle
    uint64_t window;        // steps per window
    uint64_t max_steps;     // step cap, or the run's length (fixed steps)
    uint32_t mode;          // ORR_RUN_*
    uint32_t ramp_count;    // sampling intervals of the gradual start (0: none)
    const void* ramp;       // inlet velocity of intervals 0 .. ramp_count (3 arithmetic values each;
                            // entry ramp_count is the full inlet velocity)
    void* inlet;            // the solver's device inlet velocity (3 arithmetic values)
    // Evolving.
    uint64_t steps;
    uint64_t window_steps;
    uint64_t window_samples;
    double window_sum[6];
    double window_lo[3];    // force sample extremes of the window (x, y, z)
    double window_hi[3];
    double previous_cd;
    uint32_t have_previous;
    int32_t state;          // ORR_SOLVE_RUNNING until the slot is done
    // Result (when done).
    double cd, cl, cm, delta;
    double mean[6];
};

// Launch counters: [0] periods run by the current launch, [1] set when the
// host's flag ended it.
constexpr uint32_t kServeCounters = 2;

// One sampling period of `period` steps is over for every running slot;
// `sums` holds its force sample (6 values per slot).  One block.
template <class A>
__global__ void serve_period_kernel(ServeSlot* __restrict__ slots, uint32_t n, const double* __restrict__ sums,
                                    uint32_t period, uint32_t max_periods, const volatile uint32_t* host_flag,
                                    uint32_t* __restrict__ counters, cudaGraphConditionalHandle handle) {
    bool finished = false;
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        ServeSlot& s = slots[k];
        if (s.state != ORR_SOLVE_RUNNING) {
            continue;
        }
        const double* f = sums + 6ull * k;
        const uint64_t first = s.steps;
        s.steps += period;
        // A fixed-length solve sums only its last window.
        const bool counted = s.mode != ORR_RUN_FIXED_STEPS || first >= s.max_steps - s.window;
        if (counted) {
            s.window_steps += period;
            for (int v = 0; v < 6; ++v) s.window_sum[v] = __dadd_rn(s.window_sum[v], f[v]);
            for (int v = 0; v < 3; ++v) {
                const bool first_sample = s.window_samples == 0;
                s.window_lo[v] = first_sample ? f[v] : fmin(s.window_lo[v], f[v]);
                s.window_hi[v] = first_sample ? f[v] : fmax(s.window_hi[v], f[v]);
            }
            s.window_samples += 1;
        }
        bool finite = true;
        for (int v = 0; v < 6; ++v) finite = finite && isfinite(f[v]);
        if (!finite) {
            s.state = ORR_SOLVE_FAILED;
            finished = true;
            continue;
        }
        if (!(s.mode == ORR_RUN_FIXED_STEPS && s.steps < s.max_steps) && s.window_steps >= s.window) {
            double mean[6];
            const double samples = static_cast<double>(s.window_samples);
            for (int v = 0; v < 6; ++v) mean[v] = __ddiv_rn(s.window_sum[v], samples);
            // Coefficients (set_coefficients, aero_result.h:92; moment about
            // the centre, lbm_aero_solver3d.cpp:428-431).
            const double mz = __dsub_rn(mean[5], __dsub_rn(__dmul_rn(s.centre[0], mean[1]),
                                                          __dmul_rn(s.centre[1], mean[0])));
            const double cd = __ddiv_rn(mean[0], s.qa), cl = __ddiv_rn(mean[1], s.qa);
            const double cm = __ddiv_rn(mz, __dmul_rn(s.qa, s.length));
            bool done = false;
            if (s.mode == ORR_RUN_FIXED_STEPS) {
                s.state = ORR_SOLVE_COMPLETED;
                s.delta = 0.0;
                done = true;
            } else {
                const double delta = s.have_previous ? fabs(__dsub_rn(cd, s.previous_cd)) : INFINITY;
                s.have_previous = 1u;
                s.previous_cd = cd;
                s.delta = delta;
                // The reference adapter's steady test: every force range of
                // the window within steady_range |mean drag force|.
                bool steady = true;
                if (s.steady_range > 0.0) {
                    const double bound = __dmul_rn(s.steady_range, fabs(mean[0]));
                    for (int v = 0; v < 3; ++v) {
                        steady = steady && __dsub_rn(s.window_hi[v], s.window_lo[v]) <= bound;
                    }
                }
                if (delta < s.tolerance && steady) {
                    s.state = ORR_SOLVE_CONVERGED;
                    done = true;
                } else if (s.steps >= s.max_steps) {
                    s.state = ORR_SOLVE_CAPPED;
                    done = true;
                }
            }
            s.cd = cd;
            s.cl = cl;
            s.cm = cm;
            for (int v = 0; v < 6; ++v) s.mean[v] = mean[v];
            if (!done) {
                s.window_steps = 0;
                s.window_samples = 0;
                for (int v = 0; v < 6; ++v) s.window_sum[v] = 0.0;
            }
            finished = finished || done;
        }
        // The inlet velocity of the next interval (whose first step is
        // s.steps) while the gradual start lasts; the last entry of the
        // table is the full velocity.
        if (s.state == ORR_SOLVE_RUNNING && s.ramp_count > 0) {
            const uint64_t j = s.steps / period;
            if (j <= s.ramp_count) {
                const A* from = static_cast<const A*>(s.ramp) + 3 * j;
                A* to = static_cast<A*>(s.inlet);
                to[0] = from[0];
                to[1] = from[1];
                to[2] = from[2];
            }
        }
    }
    const bool any = __syncthreads_or(finished ? 1 : 0) != 0;
    if (threadIdx.x == 0) {
        const uint32_t periods = counters[0] + 1u;
        counters[0] = periods;
        const bool asked = *host_flag != 0u;
        if (asked) {
            counters[1] = 1u;
        }
        if (any || asked || periods >= max_periods) {
            cudaGraphSetConditional(handle, 0u);
        }
    }
}

} // namespace orr
