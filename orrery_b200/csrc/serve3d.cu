// Serving loop for D3Q19 drag solves (orr_serve_*): continuous batching of
// solve requests on one device.  The reference has no server: a drag table
// (atmo::sample_cd_table, src/atmo/cd_sampling.cpp:98-120) runs its solves
// one after another through LbmAeroSolver3D, each until its coefficients
// settle.  Here requests of any lattice size arrive at any time and share
// the device:
//
//   submit     copies the request (configuration, solid mask, optional
//              distances and initial fields) into a FIFO queue; returns at
//              once with an id.
//   device     a device-resident loop (serve_loop.cuh): one launch of the
//   loop       serving graph is a conditional while-loop over sampling
//              periods of all admitted lattices as one batch (batch3d.cu:
//              `sample_every` steps of every member, then the fixed-order
//              batched force sample), and a kernel that keeps each solve's
//              slot on the device: window means, the convergence rule, the
//              gradual start.  The loop ends by itself after the period in
//              which a solve finished, when the host asks (new solves wait
//              to join), or after kMaxPeriods periods.
//   worker     one thread per server.  It launches the loop and, while the
//              device runs it, admits queued requests in arrival order as
//              long as a slot is free and the admitted lattices' device
//              memory stays within the budget: planning, allocation, upload
//              and initialisation of the new solvers overlap the loop.  When
//              the loop ends it reads the slot table back once, retires the
//              solves that are done (freeing their memory), adds the
//              admitted ones to the batch and launches the loop again.
//   done       a solve is done when the mean drag coefficient of its last
//              window of `window` steps differs from the previous window's
//              by less than `tolerance` and, with a steady range, the
//              window's force ranges are within it (converged), when it reaches
//              `max_steps` (capped), or when its force stops being finite
//              (failed); a fixed-steps solve when it has run `max_steps`
//              steps (completed, the means over its last window).
//   ramp       a solve with ramp_steps > 0 starts at rest and its inlet
//              velocity follows the reference adapter's gradual start, set
//              on the device before every sampling interval (batch3d).
//
// Each solve's populations and force sums are exactly those it would have
// alone (batch members do not interact, and the force sums have a fixed
// order), so its result does not depend on the mix it was served in.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numbers>
#include <string>
#include <thread>
#include <vector>

#include "batch3d_state.cuh"
#include "common.h"
#include "plan.h"
#include "serve_loop.cuh"
#include "solver3d_state.cuh"
#include "trace.h"

namespace {

using namespace orr;
using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    orr_lbm3d_config config{};
    std::vector<uint8_t> solid;
    std::vector<double> distance;
    std::vector<double> fields;   // rho, ux, uy, uz (4 cells) or empty
    int32_t allow_high_mach = 0;
    uint32_t window = 500;
    uint32_t mode = ORR_RUN_UNTIL_SETTLED;
    double tolerance = 1e-4;
    uint64_t max_steps = 0;
    double ramp_steps = 0.0;      // gradual start (0: none)
    double steady_range = 0.0;    // steady test of the settle rule (0: off)
    double area = 1.0, length = 1.0;
    double centre[3] = {0.0, 0.0, 0.0};
    uint64_t estimate = 0;        // device bytes before planning
};

struct Record {
    orr_solve_result result{};
};

// A solve on the device.
struct Active {
    std::shared_ptr<Request> req;
    orr_lbm3d* solver = nullptr;
    uint64_t bytes = 0;
    ServeSlot slot{};        // host copy of its slot, as of the last read-back
    void* ramp = nullptr;    // device table of its gradual start (owned), or null
};

// Sampling periods a launch of the serving loop runs at most before the host
// looks again (when no solve finishes and none waits to join).
constexpr uint32_t kMaxPeriods = 1000;

double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

template <std::size_t N> void copy_text(char (&out)[N], const std::string& text) {
    const std::size_t n = std::min(text.size(), N - 1);
    std::memcpy(out, text.data(), n);
    out[n] = '\0';
}

} // namespace

struct orr_server {
    orr_serve_options opt{};
    Clock::time_point t0 = Clock::now();
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;       // new work or stop
    std::condition_variable changed;  // a result changed state
    bool stop = false;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<uint64_t, Record> records;
    uint64_t next_id = 1;
    std::string error;
    std::string worker_error;

    // Statistics (under mu).
    uint64_t completed = 0, failed = 0, chunks = 0;
    double lattice_updates = 0.0, busy_seconds = 0.0, active_sum = 0.0;
    uint64_t peak_bytes = 0;
    double first_arrival = -1.0, last_finish = 0.0;
    std::vector<double> latencies;

    // Worker-owned.
    orr_batch3d* batch = nullptr;
    std::vector<Active> active;
    std::vector<Active> joining;
    uint64_t used_bytes = 0;

    ~orr_server() { shutdown(); }

    void shutdown() noexcept {
        {
            std::lock_guard<std::mutex> lock(mu);
            stop = true;
        }
        cv.notify_all();
        if (worker.joinable()) {
            worker.join();
        }
        // The worker has stopped and its last launch has completed; the loop
        // graph goes before the memory its nodes name, then the solvers,
        // then the batch.
        cudaSetDevice(opt.device);
        if (batch && batch->stream) {
            cudaStreamSynchronize(batch->stream);
        }
        release_loop();
        for (auto* list : {&active, &joining}) {
            for (Active& a : *list) {
                if (a.solver) orr_lbm3d_destroy(a.solver);
                if (a.ramp) cudaFree(a.ramp);
            }
            list->clear();
        }
        if (batch) {
            orr_batch3d_destroy(batch);
            batch = nullptr;
        }
    }

    void finish(const Active& a, int32_t state, double cd, double cl, double cm, double delta,
                const double* mean, const std::string& message) {
        std::lock_guard<std::mutex> lock(mu);
        orr_solve_result& r = records[a.req->id].result;
        r.state = state;
        r.steps = a.slot.steps;
        r.cd = cd;
        r.cl = cl;
        r.cm = cm;
        r.delta_cd = delta;
        if (mean != nullptr) {
            std::memcpy(r.force, mean, 3 * sizeof(double));
            std::memcpy(r.moment, mean + 3, 3 * sizeof(double));
        }
        r.finished_s = seconds_since(t0);
        copy_text(r.message, message);
        if (state == ORR_SOLVE_FAILED) {
            ++failed;
        } else {
            ++completed;
            latencies.push_back(r.finished_s - r.arrival_s);
        }
        last_finish = std::max(last_finish, r.finished_s);
        changed.notify_all();
    }

    // Creates the solver of a request (host planning, device allocation and
    // upload, initial state).  Returns false (and records the failure) if the
    // request is refused.
    bool start(const std::shared_ptr<Request>& q, Active& a) {
        orr_solver_options o{};
        o.storage = opt.storage;
        o.allow_high_mach = q->allow_high_mach;
        o.device = opt.device;
        o.block_x = 0;
        o.kernel = ORR_KERNEL_AUTO;
        o.stages = 0;
        orr_lbm3d* s = nullptr;
        orr_status st = orr_lbm3d_create(&q->config, q->solid.data(),
                                         q->distance.empty() ? nullptr : q->distance.data(), &o, &s);
        std::string why;
        if (st != ORR_OK) {
            why = orr_last_error();
        } else if (!q->fields.empty()) {
            const std::size_t n = q->solid.size();
            st = orr_lbm3d_initialize(s, q->fields.data(), q->fields.data() + n, q->fields.data() + 2 * n,
                                      q->fields.data() + 3 * n);
            if (st != ORR_OK) why = orr_lbm3d_last_error(s);
        }
        void* ramp = nullptr;
        uint32_t ramp_count = 0;
        if (st == ORR_OK && q->ramp_steps > 0.0) {
            // Gradual start: at rest, then the inlet velocity of each
            // sampling interval from a table planned here with the reference
            // adapter's rule (LbmAeroSolver3D::step, lbm_aero_solver3d.cpp:
            // 398-412: the fraction (1 - cos(pi s / T)) / 2 of the interval's
            // first step s, in binary64, rounded as an inlet upload rounds);
            // its last entry is the full velocity.
            try {
                initialize_at_rest(s);
                const double every = static_cast<double>(opt.sample_every);
                ramp_count = static_cast<uint32_t>(std::ceil(q->ramp_steps / every));
                const std::size_t ab = s->abytes;
                std::vector<unsigned char> table((ramp_count + 1u) * 3u * ab);
                for (uint32_t j = 0; j <= ramp_count; ++j) {
                    const double start = static_cast<double>(j) * every;
                    const double fraction =
                        start >= q->ramp_steps ? 1.0 : 0.5 * (1.0 - std::cos(std::numbers::pi * start / q->ramp_steps));
                    const double u[3] = {q->config.inlet_ux, q->config.inlet_uy, q->config.inlet_uz};
                    for (int d = 0; d < 3; ++d) {
                        const double v = fraction * u[d];
                        unsigned char* at = table.data() + (3u * j + static_cast<uint32_t>(d)) * ab;
                        if (ab == sizeof(double)) {
                            std::memcpy(at, &v, sizeof v);
                        } else {
                            const float f = to_f32(v);
                            std::memcpy(at, &f, sizeof f);
                        }
                    }
                }
                check(cudaMalloc(&ramp, table.size()), "serve: ramp table");
                // On the solver's stream, which the batch's stream waits for
                // before the loop reads the table.
                check(cudaMemcpyAsync(ramp, table.data(), table.size(), cudaMemcpyHostToDevice, s->stream),
                      "serve: ramp table");
                check(cudaStreamSynchronize(s->stream), "serve: ramp table");
            } catch (const Refusal& r) {
                st = r.status;
                why = r.text;
            } catch (const CudaError& e) {
                st = ORR_ERR_CUDA;
                why = describe(e);
            }
        }
        if (st != ORR_OK) {
            if (ramp) cudaFree(ramp);
            if (s) orr_lbm3d_destroy(s);
            Active none;
            none.req = q;
            finish(none, ORR_SOLVE_FAILED, 0, 0, 0, 0, nullptr, why);
            return false;
        }
        a.req = q;
        a.solver = s;
        a.ramp = ramp;
        // The slot (set_coefficients, aero_result.h:92: Cd = Fx / (1/2 rho U^2 A)).
        ServeSlot& slot = a.slot;
        slot = ServeSlot{};
        const double u = q->config.inlet_ux;
        slot.qa = 0.5 * u * u * q->area;
        slot.length = q->length;
        slot.centre[0] = q->centre[0];
        slot.centre[1] = q->centre[1];
        slot.tolerance = q->tolerance;
        slot.steady_range = q->steady_range;
        slot.window = q->window;
        slot.max_steps = q->max_steps;
        slot.mode = q->mode;
        slot.ramp_count = ramp_count;
        slot.ramp = ramp;
        slot.inlet = s->inlet_dev();
        slot.state = ORR_SOLVE_RUNNING;
        const std::size_t slots = s->plan.wall_q.size() / d3::Q;
        a.bytes = memory3d(q->config, s->plan.link_cell.size(), slots, opt.storage).value_or(q->estimate);
        {
            std::lock_guard<std::mutex> lock(mu);
            orr_solve_result& r = records[q->id].result;
            r.state = ORR_SOLVE_RUNNING;
            r.admitted_s = seconds_since(t0);
            r.device_bytes = a.bytes;
        }
        return true;
    }

    // Admits queued requests in arrival order while a slot is free and the
    // budget holds.  A request that cannot fit even on an empty device is
    // refused.
    void admit() {
        for (;;) {
            std::shared_ptr<Request> q;
            bool refuse = false;
            {
                std::lock_guard<std::mutex> lock(mu);
                if (queue.empty() || stop) {
                    return;
                }
                if (active.size() + joining.size() >= opt.max_active) {
                    return;
                }
                q = queue.front();
                if (used_bytes + q->estimate > opt.memory_budget) {
                    if (!active.empty() || !joining.empty()) {
                        return;   // wait for memory to free up
                    }
                    refuse = true;
                }
                queue.pop_front();
            }
            if (refuse) {
                Active none;
                none.req = q;
                finish(none, ORR_SOLVE_FAILED, 0, 0, 0, 0, nullptr,
                       "serve: the lattice needs more device memory than the budget");
                continue;
            }
            Active a;
            if (start(q, a)) {
                used_bytes += a.bytes;
                joining.push_back(a);
            }
            std::lock_guard<std::mutex> lock(mu);
            peak_bytes = std::max(peak_bytes, used_bytes);
        }
    }

    // Records the result of a slot that is done and releases its solve.
    void retire(Active& a) {
        const ServeSlot& sl = a.slot;
        if (sl.state == ORR_SOLVE_FAILED) {
            // The reference adapter's warning for the same event
            // (lbm_aero_solver3d.cpp:585-588).
            finish(a, ORR_SOLVE_FAILED, 0, 0, 0, 0, nullptr,
                   "lbm.diverged: the lattice state is no longer finite (numerical instability)");
        } else {
            finish(a, sl.state, sl.cd, sl.cl, sl.cm, sl.delta, sl.mean,
                   sl.state == ORR_SOLVE_CAPPED ? "serve: step cap reached before convergence" : "");
        }
        orr_batch3d_remove(batch, a.solver);
        orr_lbm3d_destroy(a.solver);
        a.solver = nullptr;
        if (a.ramp) {
            cudaFree(a.ramp);
            a.ramp = nullptr;
        }
        used_bytes -= a.bytes;
    }

    // ---- the serving graph: a conditional while-loop over sampling periods

    cudaGraphExec_t loop_exec = nullptr;
    ServeSlot* slots_dev = nullptr;
    std::size_t slots_cap = 0;
    uint32_t* counters_dev = nullptr;
    uint32_t* flag_host = nullptr;   // mapped, pinned: the host asks the loop to end
    uint32_t* flag_dev = nullptr;
    cudaEvent_t loop_done = nullptr;
    bool loop_stale = true;
    std::vector<ServeSlot> slots_host;

    void release_loop() noexcept {
        if (loop_exec) cudaGraphExecDestroy(loop_exec);
        loop_exec = nullptr;
        if (slots_dev) cudaFree(slots_dev);
        slots_dev = nullptr;
        slots_cap = 0;
        if (counters_dev) cudaFree(counters_dev);
        counters_dev = nullptr;
        if (flag_host) cudaFreeHost(flag_host);
        flag_host = flag_dev = nullptr;
        if (loop_done) cudaEventDestroy(loop_done);
        loop_done = nullptr;
    }

    // Captures the loop for the current members: its body is one sampling
    // period of the batch (the members' steps, the force sample) and
    // serve_period_kernel, which ends the loop.
    void build_loop() {
        if (counters_dev == nullptr) {
            check(cudaMalloc(reinterpret_cast<void**>(&counters_dev), kServeCounters * sizeof(uint32_t)),
                  "serve: counters");
            check(cudaHostAlloc(reinterpret_cast<void**>(&flag_host), sizeof(uint32_t), cudaHostAllocMapped),
                  "serve: flag");
            check(cudaHostGetDevicePointer(reinterpret_cast<void**>(&flag_dev), flag_host, 0), "serve: flag");
            check(cudaEventCreateWithFlags(&loop_done, cudaEventDisableTiming), "serve: event");
        }
        const std::size_t n = active.size();
        if (n > slots_cap) {
            if (slots_dev) cudaFree(slots_dev);
            slots_dev = nullptr;
            check(cudaMalloc(reinterpret_cast<void**>(&slots_dev), n * sizeof(ServeSlot)), "serve: slot table");
            slots_cap = n;
        }
        batch->prepare_loop(opt.sample_every);
        if (loop_exec) {
            cudaGraphExecDestroy(loop_exec);
            loop_exec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        check(cudaGraphCreate(&graph, 0), "serve: loop graph");
        try {
            cudaGraphConditionalHandle handle{};
            check(cudaGraphConditionalHandleCreate(&handle, graph, 1u, cudaGraphCondAssignDefault),
                  "serve: loop condition");
            cudaGraphNodeParams params{};
            params.type = cudaGraphNodeTypeConditional;
            params.conditional.handle = handle;
            params.conditional.type = cudaGraphCondTypeWhile;
            params.conditional.size = 1;
            cudaGraphNode_t node = nullptr;
            check(cudaGraphAddNode(&node, graph, nullptr, 0, &params), "serve: loop node");
            cudaGraph_t body = params.conditional.phGraph_out[0];
            check(cudaStreamBeginCaptureToGraph(batch->stream, body, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal),
                  "serve: loop capture");
            const uint64_t before = batch->launches;
            try {
                batch->launch_steps(opt.sample_every);
                batch->launch_sample(false);
                check(launch_period(handle, static_cast<uint32_t>(n)), "serve: period kernel");
            } catch (...) {
                cudaGraph_t dropped = nullptr;
                cudaStreamEndCapture(batch->stream, &dropped);
                batch->launches = before;
                throw;
            }
            batch->launches = before;
            cudaGraph_t captured = nullptr;
            check(cudaStreamEndCapture(batch->stream, &captured), "serve: loop capture");
            check(cudaGraphInstantiate(&loop_exec, graph, 0), "serve: loop instantiate");
        } catch (...) {
            cudaGraphDestroy(graph);
            throw;
        }
        cudaGraphDestroy(graph);
        loop_stale = false;
    }

    cudaError_t launch_period(cudaGraphConditionalHandle handle, uint32_t n) {
        if (opt.storage == ORR_STORAGE_F64) {
            serve_period_kernel<double><<<1, 256, 0, batch->stream>>>(slots_dev, n, batch->sums, opt.sample_every,
                                                                      kMaxPeriods, flag_dev, counters_dev, handle);
        } else {
            serve_period_kernel<float><<<1, 256, 0, batch->stream>>>(slots_dev, n, batch->sums, opt.sample_every,
                                                                     kMaxPeriods, flag_dev, counters_dev, handle);
        }
        return cudaGetLastError();
    }

    static void check_status(orr_status st, const char* what) {
        if (st != ORR_OK) {
            throw Refusal{st, std::string(what) + ": " + orr_last_error()};
        }
    }

    void loop() {
        try {
            require_device(opt.device);
            check(cudaSetDevice(opt.device), "cudaSetDevice");
            check_status(orr_batch3d_create(opt.device, &batch), "serve: batch");
            orr_batch_schedule sched{};
            // Automatic: the row kernel with every lattice on its own graph
            // branch (up to 64), the fastest schedule measured on the served
            // sphere-cone stream and on the batch of wings.
            sched.kernel = opt.kernel == ORR_KERNEL_STAGED ? ORR_KERNEL_STAGED : ORR_KERNEL_ROWS;
            sched.block = opt.block ? opt.block : (sched.kernel == ORR_KERNEL_ROWS ? 128 : 256);
            sched.stages = opt.stages;
            sched.branches = opt.kernel == ORR_KERNEL_AUTO && opt.branches == 0 ? 64u : opt.branches;
            if (orr_batch3d_set_schedule(batch, &sched) != ORR_OK) {
                throw Refusal{ORR_ERR_INVALID, orr_batch3d_last_error(batch)};
            }
            uint32_t counters[kServeCounters] = {0, 0};
            for (;;) {
                {
                    std::unique_lock<std::mutex> lock(mu);
                    cv.wait(lock, [&] { return stop || !queue.empty() || !active.empty() || !joining.empty(); });
                    if (stop) {
                        return;
                    }
                }
                // New solvers join between launches, in admission order.
                for (Active& a : joining) {
                    if (orr_batch3d_add(batch, a.solver) != ORR_OK) {
                        throw Refusal{ORR_ERR_STATE, orr_batch3d_last_error(batch)};
                    }
                    active.push_back(a);
                    loop_stale = true;
                }
                joining.clear();
                if (active.empty()) {
                    orr::Zone zone("serve_admit");
                    admit();
                    continue;
                }
                if (loop_stale) {
                    build_loop();
                }
                // The slot table in member order, then the loop.
                const std::size_t n = active.size();
                slots_host.resize(n);
                for (std::size_t k = 0; k < n; ++k) slots_host[k] = active[k].slot;
                check(cudaMemcpyAsync(slots_dev, slots_host.data(), n * sizeof(ServeSlot), cudaMemcpyHostToDevice,
                                      batch->stream),
                      "serve: slot table");
                check(cudaMemsetAsync(counters_dev, 0, kServeCounters * sizeof(uint32_t), batch->stream),
                      "serve: counters");
                *reinterpret_cast<volatile uint32_t*>(flag_host) = 0u;
                const auto launch_start = Clock::now();
                {
                    orr::Zone zone("serve_loop");
                    batch->wait_members();
                    check(cudaGraphLaunch(loop_exec, batch->stream), "serve: loop launch");
                    check(cudaEventRecord(loop_done, batch->stream), "serve: loop event");
                }
                // While the loop runs on the device, admit queued requests;
                // once one is ready to join, ask the loop to end after its
                // current period.  Every period ends (bounded waits inside
                // the step kernels), and the loop after at most kMaxPeriods.
                for (;;) {
                    {
                        orr::Zone zone("serve_admit");
                        admit();
                    }
                    bool ask = !joining.empty();
                    {
                        std::lock_guard<std::mutex> lock(mu);
                        ask = ask || stop;
                    }
                    if (ask) {
                        *reinterpret_cast<volatile uint32_t*>(flag_host) = 1u;
                    }
                    const cudaError_t q = cudaEventQuery(loop_done);
                    if (q == cudaSuccess) {
                        break;
                    }
                    if (q != cudaErrorNotReady) {
                        check(q, "serve: loop");
                    }
                    std::unique_lock<std::mutex> lock(mu);
                    cv.wait_for(lock, std::chrono::microseconds(200), [&] { return stop; });
                }
                check(cudaMemcpyAsync(slots_host.data(), slots_dev, n * sizeof(ServeSlot), cudaMemcpyDeviceToHost,
                                      batch->stream),
                      "serve: slot table");
                check(cudaMemcpyAsync(counters, counters_dev, sizeof counters, cudaMemcpyDeviceToHost,
                                      batch->stream),
                      "serve: counters");
                check(cudaStreamSynchronize(batch->stream), "serve: loop");
                batch->finish_loop(static_cast<uint64_t>(counters[0]) * opt.sample_every);
                batch->check_status();
                const double busy = std::chrono::duration<double>(Clock::now() - launch_start).count();
                double updates = 0.0;
                for (const Active& a : active) {
                    updates += static_cast<double>(a.solver->g.cells) * opt.sample_every * counters[0];
                }
                {
                    std::lock_guard<std::mutex> lock(mu);
                    chunks += counters[0];
                    busy_seconds += busy;
                    lattice_updates += updates;
                    active_sum += static_cast<double>(n) * counters[0];
                }
                // Retire the slots that are done; members sit in the batch in
                // the order of `active`.
                std::vector<Active> keep;
                keep.reserve(n);
                for (std::size_t k = 0; k < n; ++k) {
                    Active& a = active[k];
                    a.slot = slots_host[k];
                    if (a.slot.state != ORR_SOLVE_RUNNING) {
                        retire(a);
                        loop_stale = true;
                    } else {
                        keep.push_back(a);
                    }
                }
                active.swap(keep);
            }
        } catch (const Refusal& r) {
            std::lock_guard<std::mutex> lock(mu);
            worker_error = r.text;
        } catch (const CudaError& e) {
            std::lock_guard<std::mutex> lock(mu);
            worker_error = describe(e);
        } catch (const std::exception& e) {
            std::lock_guard<std::mutex> lock(mu);
            worker_error = e.what();
        }
        // Fail whatever is left.
        std::lock_guard<std::mutex> lock(mu);
        for (auto& [id, rec] : records) {
            if (rec.result.state == ORR_SOLVE_QUEUED || rec.result.state == ORR_SOLVE_RUNNING) {
                rec.result.state = ORR_SOLVE_FAILED;
                copy_text(rec.result.message, "serve: the worker stopped: " + worker_error);
                ++failed;
            }
        }
        queue.clear();
        changed.notify_all();
    }
};

namespace {

orr_server* server_of(orr_server* s) {
    if (s == nullptr) {
        throw Refusal{ORR_ERR_INVALID, "null server handle"};
    }
    return s;
}

// Nearest-rank percentile.
double percentile(std::vector<double> v, double p) {
    if (v.empty()) {
        return 0.0;
    }
    std::sort(v.begin(), v.end());
    const double rank = std::ceil(p / 100.0 * static_cast<double>(v.size()));
    const std::size_t k = static_cast<std::size_t>(std::max(1.0, rank)) - 1;
    return v[std::min(k, v.size() - 1)];
}

bool done_state(int32_t st) {
    return st != ORR_SOLVE_QUEUED && st != ORR_SOLVE_RUNNING;
}

} // namespace

extern "C" {

orr_status orr_serve_create(const orr_serve_options* options, orr_server** out) {
    if (out == nullptr || options == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *out = nullptr;
    return orr::guarded(nullptr, [&]() -> orr_status {
        const orr_serve_options& o = *options;
        if (o.storage < ORR_STORAGE_F32 || o.storage > ORR_STORAGE_F64) {
            throw Refusal{ORR_ERR_INVALID, "serve: unknown population storage"};
        }
        if (o.storage == ORR_STORAGE_BF16) {
            // Served solves promise a drag coefficient within 0.5% of binary64;
            // bfloat16 keeps 8 significant bits of f - w and measured 7.1e-3 on
            // the 512 x 256 x 256 ellipsoid at Re 1000.
            throw Refusal{ORR_ERR_INVALID,
                          "serve: bfloat16 storage is not served: its drag coefficient misses the 0.5% bound "
                          "against binary64; use binary16 or binary32"};
        }
        if (o.max_active == 0 || o.memory_budget == 0) {
            throw Refusal{ORR_ERR_INVALID, "serve: max_active and memory_budget must be positive"};
        }
        if (o.sample_every == 0 || o.sample_every % 2 != 0 || o.chunk_steps == 0 ||
            o.chunk_steps % o.sample_every != 0) {
            throw Refusal{ORR_ERR_INVALID, "serve: sample_every must be even and divide chunk_steps"};
        }
        require_device(o.device);
        auto s = std::make_unique<orr_server>();
        s->opt = o;
        s->worker = std::thread([p = s.get()] { p->loop(); });
        *out = s.release();
        return ORR_OK;
    });
}

void orr_serve_destroy(orr_server* server) {
    delete server;
}

const char* orr_serve_last_error(const orr_server* server) {
    return server ? server->error.c_str() : orr_last_error();
}

orr_status orr_serve_submit(orr_server* server, const orr_solve_request* request, uint64_t* id) {
    return orr::guarded(server ? &server->error : nullptr, [&]() -> orr_status {
        orr_server* s = server_of(server);
        if (request == nullptr || request->config == nullptr || request->solid == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "serve: null request, configuration or mask"};
        }
        const orr_solve_request& r = *request;
        const orr_lbm3d_config& c = *r.config;
        if (r.window == 0 || r.window % s->opt.chunk_steps != 0) {
            throw Refusal{ORR_ERR_INVALID, "serve: the window must be a positive multiple of chunk_steps"};
        }
        if (r.sample_every != 0 && r.sample_every != s->opt.sample_every) {
            throw Refusal{ORR_ERR_INVALID, "serve: the request's sampling differs from the server's"};
        }
        if (r.mode != ORR_RUN_UNTIL_SETTLED && r.mode != ORR_RUN_FIXED_STEPS) {
            throw Refusal{ORR_ERR_INVALID, "serve: unknown run mode"};
        }
        const bool fixed = r.mode == ORR_RUN_FIXED_STEPS;
        if ((!fixed && !(r.tolerance > 0.0)) || !(r.reference_area > 0.0) || !(r.reference_length > 0.0)) {
            throw Refusal{ORR_ERR_INVALID, "serve: tolerance, area and length must be positive"};
        }
        if (fixed && (r.max_steps < r.window || r.max_steps % s->opt.chunk_steps != 0)) {
            throw Refusal{ORR_ERR_INVALID, "serve: a fixed-steps solve needs max_steps a multiple of chunk_steps "
                                           "and at least one window"};
        }
        if (!(r.ramp_steps >= 0.0) || !std::isfinite(r.ramp_steps)) {
            throw Refusal{ORR_ERR_INVALID, "serve: ramp_steps must be finite and not negative"};
        }
        if (!(r.steady_range >= 0.0) || !std::isfinite(r.steady_range)) {
            throw Refusal{ORR_ERR_INVALID, "serve: steady_range must be finite and not negative"};
        }
        if (c.x_boundary != ORR_X_INFLOW_OUTFLOW || !(c.inlet_ux != 0.0)) {
            throw Refusal{ORR_ERR_INVALID, "serve: drag solves need an inflow with a non-zero inlet speed"};
        }
        if (std::string problem = problem3d(c, r.solid, r.distance, s->opt.storage, r.allow_high_mach != 0);
            !problem.empty()) {
            throw Refusal{ORR_ERR_INVALID, problem};
        }
        const bool any = r.rho || r.ux || r.uy || r.uz;
        const bool all = r.rho && r.ux && r.uy && r.uz;
        if (any && !all) {
            throw Refusal{ORR_ERR_INVALID, "serve: initial fields need all four arrays or none"};
        }
        if (any && r.ramp_steps > 0.0) {
            throw Refusal{ORR_ERR_INVALID, "serve: a ramped solve starts at rest (no initial fields)"};
        }
        auto q = std::make_shared<Request>();
        q->config = c;
        const std::size_t cells = static_cast<std::size_t>(c.nx) * c.ny * c.nz;
        q->solid.assign(r.solid, r.solid + cells);
        if (r.distance) q->distance.assign(r.distance, r.distance + cells);
        if (all) {
            q->fields.resize(4 * cells);
            std::memcpy(q->fields.data(), r.rho, cells * 8);
            std::memcpy(q->fields.data() + cells, r.ux, cells * 8);
            std::memcpy(q->fields.data() + 2 * cells, r.uy, cells * 8);
            std::memcpy(q->fields.data() + 3 * cells, r.uz, cells * 8);
        }
        q->allow_high_mach = r.allow_high_mach;
        q->window = r.window;
        q->mode = r.mode;
        q->tolerance = r.tolerance;
        q->max_steps = r.max_steps ? r.max_steps : UINT64_MAX;
        q->ramp_steps = r.ramp_steps;
        q->steady_range = r.steady_range;
        q->area = r.reference_area;
        q->length = r.reference_length;
        std::memcpy(q->centre, r.moment_centre, sizeof(q->centre));
        // Device bytes before planning: the links (16 bytes each) are not
        // known yet; 19 per solid node bounds them.
        const uint64_t solid_nodes = static_cast<uint64_t>(std::count(q->solid.begin(), q->solid.end(), 1));
        q->estimate = memory3d(c, 19 * solid_nodes, 0, s->opt.storage).value_or(UINT64_MAX);
        {
            std::lock_guard<std::mutex> lock(s->mu);
            if (!s->worker_error.empty()) {
                throw Refusal{ORR_ERR_STATE, "serve: the worker stopped: " + s->worker_error};
            }
            q->id = s->next_id++;
            orr_solve_result& res = s->records[q->id].result;
            res = orr_solve_result{};
            res.state = ORR_SOLVE_QUEUED;
            res.arrival_s = seconds_since(s->t0);
            if (s->first_arrival < 0.0) s->first_arrival = res.arrival_s;
            s->queue.push_back(q);
        }
        s->cv.notify_all();
        if (id) *id = q->id;
        return ORR_OK;
    });
}

orr_status orr_serve_poll(orr_server* server, uint64_t id, orr_solve_result* result) {
    return orr::guarded(server ? &server->error : nullptr, [&]() -> orr_status {
        orr_server* s = server_of(server);
        if (result == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "serve: null result"};
        }
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->records.find(id);
        if (it == s->records.end()) {
            throw Refusal{ORR_ERR_INVALID, "serve: unknown request id"};
        }
        *result = it->second.result;
        return ORR_OK;
    });
}

orr_status orr_serve_wait(orr_server* server, uint64_t id, double timeout_s, orr_solve_result* result) {
    return orr::guarded(server ? &server->error : nullptr, [&]() -> orr_status {
        orr_server* s = server_of(server);
        std::unique_lock<std::mutex> lock(s->mu);
        if (s->records.find(id) == s->records.end()) {
            throw Refusal{ORR_ERR_INVALID, "serve: unknown request id"};
        }
        const bool ok = s->changed.wait_for(lock, std::chrono::duration<double>(timeout_s),
                                            [&] { return done_state(s->records[id].result.state); });
        if (result) *result = s->records[id].result;
        if (!ok) {
            throw Refusal{ORR_ERR_TIMEOUT, "serve: the solve is not done yet"};
        }
        return ORR_OK;
    });
}

orr_status orr_serve_drain(orr_server* server, double timeout_s) {
    return orr::guarded(server ? &server->error : nullptr, [&]() -> orr_status {
        orr_server* s = server_of(server);
        std::unique_lock<std::mutex> lock(s->mu);
        const auto all_done = [&] {
            for (const auto& [id, rec] : s->records) {
                if (!done_state(rec.result.state)) {
                    return false;
                }
            }
            return true;
        };
        if (!s->changed.wait_for(lock, std::chrono::duration<double>(timeout_s), all_done)) {
            throw Refusal{ORR_ERR_TIMEOUT, "serve: solves still running"};
        }
        return ORR_OK;
    });
}

orr_status orr_serve_stats(orr_server* server, orr_serve_statistics* stats) {
    return orr::guarded(server ? &server->error : nullptr, [&]() -> orr_status {
        orr_server* s = server_of(server);
        if (stats == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "serve: null statistics"};
        }
        std::lock_guard<std::mutex> lock(s->mu);
        orr_serve_statistics t{};
        t.submitted = s->next_id - 1;
        t.completed = s->completed;
        t.failed = s->failed;
        for (const auto& [id, rec] : s->records) {
            if (rec.result.state == ORR_SOLVE_QUEUED) ++t.queued;
            if (rec.result.state == ORR_SOLVE_RUNNING) ++t.active;
        }
        t.latency_p50_s = percentile(s->latencies, 50.0);
        t.latency_p99_s = percentile(s->latencies, 99.0);
        double sum = 0.0;
        for (double v : s->latencies) sum += v;
        t.latency_mean_s = s->latencies.empty() ? 0.0 : sum / static_cast<double>(s->latencies.size());
        const double span = s->last_finish - std::max(s->first_arrival, 0.0);
        t.solves_per_second = span > 0.0 ? static_cast<double>(s->completed) / span : 0.0;
        t.lattice_updates = s->lattice_updates;
        t.busy_seconds = s->busy_seconds;
        t.peak_device_bytes = s->peak_bytes;
        t.mean_active = s->chunks ? s->active_sum / static_cast<double>(s->chunks) : 0.0;
        t.chunks = s->chunks;
        t.worker_failed = s->worker_error.empty() ? 0 : 1;
        copy_text(t.message, s->worker_error);
        *stats = t;
        return ORR_OK;
    });
}

} // extern "C"
