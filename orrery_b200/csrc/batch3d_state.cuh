// State of a batch of D3Q19 solvers (the handle behind orr_batch3d_*),
// shared by the batch entry points and the serving loop.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "solver3d_state.cuh"

namespace orr {

// Candidate schedules of the autotuner (kernel, block, stages, nodes per
// thread of a staged span or of the row-tile step, graph branches: 64
// branches means one per member up to 64).
struct Candidate {
    int32_t kernel;
    uint32_t block;
    uint32_t stages;
    uint32_t npt;
    uint32_t branches;
};
inline constexpr Candidate kCandidates[] = {
    {ORR_KERNEL_STAGED, 256, 3, 2, 0},  {ORR_KERNEL_STAGED, 256, 2, 1, 0},
    {ORR_KERNEL_STAGED, 256, 2, 2, 64}, {ORR_KERNEL_STAGED, 256, 3, 2, 64},
    {ORR_KERNEL_STAGED, 256, 4, 1, 64}, {ORR_KERNEL_STAGED, 128, 3, 2, 64},
    {ORR_KERNEL_ROWS, 128, 0, 0, 0},    {ORR_KERNEL_ROWS, 128, 0, 0, 64},
    {ORR_KERNEL_ROWS, 128, 0, 2, 0},    {ORR_KERNEL_ROWS, 128, 0, 2, 64},
    {ORR_KERNEL_ROWS, 64, 0, 0, 0},     {ORR_KERNEL_ROWS, 64, 0, 0, 64},
};

} // namespace orr

struct orr_batch3d {
    int device = 0;
    int32_t storage = -1;
    bool smag = false;
    const Ops3D* ops = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::vector<orr_lbm3d*> members;
    std::vector<cudaEvent_t> member_events;

    // Schedule.
    int32_t kernel = ORR_KERNEL_STAGED;
    uint32_t block = 256;
    uint32_t stages = 0;      // 0: the shape's default
    uint32_t npt = 0;         // nodes per thread of a staged span (0: the storage's default),
                              // or of the row-tile step (2: the pair step where it serves a member)
    uint32_t branches = 0;    // 0: one stream; else members spread over this many graph branches
    StagedShape shape{};

    // Branched schedule: member k runs its own single-lattice launches (its
    // entry solo[k], items solo_items[k], grid solo_grid[k]) on branch
    // stream lane_of[k]; a fork event starts the branches, join events end
    // them.
    std::vector<cudaStream_t> branch_streams;
    std::vector<cudaEvent_t> join_events;
    cudaEvent_t fork_event = nullptr;
    std::vector<unsigned char> solo;
    std::size_t solo_stride = 0;
    std::vector<ItemCounts> solo_items;
    std::vector<uint32_t> solo_grid;
    std::vector<uint32_t> lane_of;

    // State of the current table: parities and epochs of the members when it
    // was built, and the steps taken since (mod 2).
    bool dirty = true;
    std::vector<int> parity;
    std::vector<uint64_t> epochs;
    uint32_t flip = 0;
    ItemCounts items{};
    void* table = nullptr;
    std::size_t table_bytes = 0;
    std::vector<unsigned char> host_table; // host copy of the entries
    uint32_t* status = nullptr;
    cudaGraphExec_t graph = nullptr;
    uint32_t graph_sample = 0;    // sampling interval the graph was captured with (0: none)

    // Batched forces.
    void* jobs = nullptr;
    std::size_t jobs_bytes = 0;
    double* partial = nullptr;
    std::size_t partial_count = 0;
    double* sums = nullptr;       // 6 per member
    std::size_t sums_count = 0;
    uint64_t chunks = 0;
    std::vector<ForceJob> host_jobs;

    uint64_t launches = 0;
    std::string error;

    ~orr_batch3d() { release(); }

    void release() noexcept {
        cudaSetDevice(device);
        for (orr_lbm3d* m : members) {
            m->batch = nullptr;
        }
        members.clear();
        if (graph) cudaGraphExecDestroy(graph);
        for (cudaEvent_t e : member_events) cudaEventDestroy(e);
        member_events.clear();
        for (cudaEvent_t e : join_events) cudaEventDestroy(e);
        join_events.clear();
        for (cudaStream_t s : branch_streams) cudaStreamDestroy(s);
        branch_streams.clear();
        if (fork_event) cudaEventDestroy(fork_event);
        fork_event = nullptr;
        for (void* p : {table, static_cast<void*>(status), jobs, static_cast<void*>(partial),
                        static_cast<void*>(sums)}) {
            if (p) cudaFree(p);
        }
        if (done) cudaEventDestroy(done);
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        if (stream) cudaStreamDestroy(stream);
        graph = nullptr;
        table = jobs = nullptr;
        status = nullptr;
        partial = sums = nullptr;
        done = t0 = t1 = nullptr;
        stream = nullptr;
    }

    void drop_graph() {
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
    }

    template <class T> static void grow(T*& p, std::size_t& have, std::size_t need, const char* what) {
        if (need <= have && p != nullptr) {
            return;
        }
        if (p) cudaFree(p);
        p = nullptr;
        have = 0;
        check(cudaMalloc(reinterpret_cast<void**>(&p), std::max<std::size_t>(need, 1) * sizeof(T)), what);
        have = need;
    }
    static void grow_bytes(void*& p, std::size_t& have, std::size_t need, const char* what) {
        if (need <= have && p != nullptr) {
            return;
        }
        if (p) cudaFree(p);
        p = nullptr;
        have = 0;
        check(cudaMalloc(&p, std::max<std::size_t>(need, 1)), what);
        have = need;
    }

    bool stale() const {
        if (dirty) {
            return true;
        }
        for (std::size_t k = 0; k < members.size(); ++k) {
            if (members[k]->epoch != epochs[k] || members[k]->cur != (parity[k] ^ static_cast<int>(flip))) {
                return true;
            }
        }
        return false;
    }

    template <class A> void fill_table(std::vector<Lattice3D<A>>& lats) {
        lats.resize(members.size());
        for (std::size_t k = 0; k < members.size(); ++k) {
            orr_lbm3d* m = members[k];
            Lattice3D<A>& L = lats[k];
            L = Lattice3D<A>{};
            L.g = m->g;
            if constexpr (sizeof(A) == 8) {
                L.p = m->phys64;
            } else {
                L.p = m->phys32;
            }
            L.b = m->buffers();
            L.f[0] = m->f[0];
            L.f[1] = m->f[1];
            L.parity = static_cast<uint32_t>(m->cur);
            L.staged = stageable(m->g) ? 1u : 0u;
        }
        items = number_items(lats.data(), lats.size(), block, shape.npt);
        host_table.resize(lats.size() * sizeof(Lattice3D<A>));
        std::memcpy(host_table.data(), lats.data(), host_table.size());
        grow_bytes(table, table_bytes, lats.size() * sizeof(Lattice3D<A>), "batch table");
        check(cudaMemcpyAsync(table, lats.data(), lats.size() * sizeof(Lattice3D<A>), cudaMemcpyHostToDevice,
                              stream),
              "batch table upload");
        check(cudaStreamSynchronize(stream), "batch table upload");
    }

    // Rebuilds the tables from the members' current state (flip restarts at 0).
    void rebuild() {
        drop_graph();
        parity.resize(members.size());
        epochs.resize(members.size());
        for (std::size_t k = 0; k < members.size(); ++k) {
            parity[k] = members[k]->cur;
            epochs[k] = members[k]->epoch;
        }
        flip = 0;
        if (members.empty()) {
            dirty = false;
            return;
        }
        if (kernel == ORR_KERNEL_STAGED) {
            if (!all_flat()) {
                throw Refusal{ORR_ERR_INVALID, "batch3d: the staged step needs members with periodic or "
                                               "free-slip sides and halfway walls"};
            }
            shape = staged_shape(*ops, smag, block, npt ? npt : default_npt(storage), stages, device);
            if (shape.per_sm <= 0) {
                throw Refusal{ORR_ERR_INVALID, "batch3d: the staged step cannot launch with this shape"};
            }
            if (storage == ORR_STORAGE_F64) {
                std::vector<Lattice3D<double>> lats;
                fill_table(lats);
            } else {
                std::vector<Lattice3D<float>> lats;
                fill_table(lats);
            }
            const uint64_t most = std::max<uint64_t>({items.staged, items.direct, 1});
            if (branches > 0) {
                if (storage == ORR_STORAGE_F64) {
                    fill_solo<double>();
                } else {
                    fill_solo<float>();
                }
            }
            shape.grid = static_cast<uint32_t>(std::min<uint64_t>(shape.grid, most));
        }
        if (branches > 0) {
            assign_lanes();
        }
        // Force jobs read the buffer that is current at flip 0 (sampling at
        // even step counts only).
        host_jobs.resize(members.size());
        chunks = 0;
        for (std::size_t k = 0; k < members.size(); ++k) {
            orr_lbm3d* m = members[k];
            ForceJob& J = host_jobs[k];
            J.f = m->f[parity[k]];
            J.lcell = m->lcell;
            J.ldir = m->ldir;
            J.lq = m->lq;
            J.links = m->plan.link_cell.size();
            J.chunk_begin = chunks;
            J.nx = m->g.nx;
            J.plane = m->g.plane;
            J.cells = m->g.cells;
            chunks += (J.links + kForceChunk - 1) / kForceChunk;
        }
        grow_bytes(jobs, jobs_bytes, host_jobs.size() * sizeof(ForceJob), "batch force table");
        check(cudaMemcpyAsync(jobs, host_jobs.data(), host_jobs.size() * sizeof(ForceJob),
                              cudaMemcpyHostToDevice, stream),
              "batch force table upload");
        grow(partial, partial_count, std::max<uint64_t>(chunks, 1) * 6, "batch force partials");
        grow(sums, sums_count, members.size() * 6, "batch force sums");
        check(cudaStreamSynchronize(stream), "batch force table upload");
        dirty = false;
    }

    bool branched() const { return branches > 0; }

    bool all_flat() const {
        for (const orr_lbm3d* m : members) {
            if (!m->g.flat) return false;
        }
        return true;
    }

    // One row-tile step of member m from buffer `from` on stream s.
    void member_step(orr_lbm3d* m, uint32_t from, cudaStream_t s) {
        check(ops->step(m->g, m->phys(), m->f[from], m->f[1 - from], m->buffers(), smag, block,
                        npt == 2 ? 2u : 1u, s),
              "batch step kernel");
    }

    // Per-member single-lattice entries of the branched staged schedule; each
    // member's grid is its share of the whole launch's CTAs by node count.
    template <class A> void fill_solo() {
        const std::size_t n = members.size();
        solo_stride = sizeof(Lattice3D<A>);
        solo.assign(n * solo_stride, 0);
        solo_items.assign(n, ItemCounts{});
        solo_grid.assign(n, 1);
        const auto* all = reinterpret_cast<const Lattice3D<A>*>(host_table.data());
        double total = 0.0;
        for (const orr_lbm3d* m : members) total += static_cast<double>(m->g.cells);
        for (std::size_t k = 0; k < n; ++k) {
            Lattice3D<A> L = all[k];
            solo_items[k] = number_items(&L, 1, shape.block, shape.npt);
            std::memcpy(solo.data() + k * solo_stride, &L, sizeof(L));
            const double share = static_cast<double>(members[k]->g.cells) / total;
            const uint64_t g = static_cast<uint64_t>(std::lround(share * shape.grid));
            const uint64_t most = std::max<uint64_t>({solo_items[k].staged, solo_items[k].direct, 1});
            solo_grid[k] = static_cast<uint32_t>(std::clamp<uint64_t>(g, 1, most));
        }
    }

    // Members to branches: largest first, each to the least-loaded branch.
    void assign_lanes() {
        const std::size_t n = members.size();
        const std::size_t lanes = std::min<std::size_t>(branches, n);
        while (branch_streams.size() < lanes) {
            cudaStream_t s = nullptr;
            check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "batch branch stream");
            branch_streams.push_back(s);
            cudaEvent_t e = nullptr;
            check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch branch event");
            join_events.push_back(e);
        }
        if (fork_event == nullptr) {
            check(cudaEventCreateWithFlags(&fork_event, cudaEventDisableTiming), "batch branch event");
        }
        std::vector<std::size_t> order(n);
        for (std::size_t k = 0; k < n; ++k) order[k] = k;
        std::sort(order.begin(), order.end(),
                  [&](std::size_t a, std::size_t b) { return members[a]->g.cells > members[b]->g.cells; });
        std::vector<double> load(lanes, 0.0);
        lane_of.assign(n, 0);
        for (std::size_t k : order) {
            const std::size_t lane =
                static_cast<std::size_t>(std::min_element(load.begin(), load.end()) - load.begin());
            lane_of[k] = static_cast<uint32_t>(lane);
            load[lane] += static_cast<double>(members[k]->g.cells);
        }
    }

    // `count` steps of every member on the branches: fork from the batch
    // stream, each member's steps in order on its branch, join back.
    void launch_branched(uint32_t count) {
        const std::size_t lanes = std::min<std::size_t>(branches, members.size());
        check(cudaEventRecord(fork_event, stream), "batch fork");
        for (std::size_t b = 0; b < lanes; ++b) {
            check(cudaStreamWaitEvent(branch_streams[b], fork_event, 0), "batch fork");
        }
        for (uint32_t step = 0; step < count; ++step) {
            for (std::size_t k = 0; k < members.size(); ++k) {
                orr_lbm3d* m = members[k];
                cudaStream_t s = branch_streams[lane_of[k]];
                const uint32_t from = static_cast<uint32_t>(parity[k]) ^ flip;
                if (kernel == ORR_KERNEL_STAGED) {
                    // The entry's parity is the member's at the rebuild:
                    // its source is f[parity ^ flip].
                    check(ops->staged(solo.data() + k * solo_stride, nullptr, 1, solo_items[k].staged,
                                      solo_items[k].direct, flip, shape.stages, smag, shape.block, shape.npt,
                                      solo_grid[k], status, s),
                          "batch step kernel");
                } else {
                    member_step(m, from, s);
                }
                ++launches;
            }
            flip ^= 1u;
        }
        for (std::size_t b = 0; b < lanes; ++b) {
            check(cudaEventRecord(join_events[b], branch_streams[b]), "batch join");
            check(cudaStreamWaitEvent(stream, join_events[b], 0), "batch join");
        }
    }

    // `count` steps of every member with the current schedule.
    void launch_steps(uint32_t count) {
        if (branched()) {
            launch_branched(count);
        } else {
            for (uint32_t k = 0; k < count; ++k) launch_step();
        }
    }

    // One step of every member (flip = steps since the table, mod 2).
    void launch_step() {
        if (kernel == ORR_KERNEL_STAGED) {
            check(ops->staged(members.size() == 1 ? host_table.data() : nullptr, table,
                              static_cast<uint32_t>(members.size()), items.staged, items.direct, flip,
                              shape.stages, smag, shape.block, shape.npt, shape.grid, status, stream),
                  "batch step kernel");
            ++launches;
        } else {
            for (std::size_t k = 0; k < members.size(); ++k) {
                member_step(members[k], static_cast<uint32_t>(parity[k]) ^ flip, stream);
                ++launches;
            }
        }
        flip ^= 1u;
    }

    // Sum of the members' force and moment into sums[6 k ..] (flip must be 0).
    void launch_sample(bool accumulate) {
        check(ops->force_batch(jobs, static_cast<uint32_t>(members.size()), chunks, partial, sums, accumulate,
                               stream),
              "batch force kernels");
        launches += chunks > 0 ? 2 : 1;
    }

    // kGraphSteps steps, with a force sample after every `sample` steps
    // when sample > 0 (kGraphSteps is then a multiple of it).
    void build_graph(uint32_t sample, uint32_t steps) {
        drop_graph();
        cudaGraph_t captured = nullptr;
        const uint64_t before = launches;
        const uint32_t flip_before = flip;
        check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "batch graph capture");
        try {
            if (sample > 0) {
                for (uint32_t k = 0; k < steps; k += sample) {
                    launch_steps(sample);
                    launch_sample(true);
                }
            } else {
                launch_steps(steps);
            }
        } catch (...) {
            cudaStreamEndCapture(stream, &captured);
            if (captured) cudaGraphDestroy(captured);
            launches = before;
            flip = flip_before;
            throw;
        }
        launches = before;
        flip = flip_before;
        check(cudaStreamEndCapture(stream, &captured), "batch graph capture");
        const cudaError_t e = cudaGraphInstantiate(&graph, captured, 0);
        cudaGraphDestroy(captured);
        check(e, "batch graph instantiate");
        graph_sample = sample;
        graph_steps = steps;
        graph_launches = launches_per_step() * steps + (sample > 0 ? (steps / sample) * (chunks > 0 ? 2 : 1) : 0);
    }
    uint32_t graph_steps = 0;
    uint64_t graph_launches = 0;

    uint64_t launches_per_step() const {
        return kernel == ORR_KERNEL_STAGED && !branched() ? 1 : members.size();
    }

    void wait_members() {
        for (std::size_t k = 0; k < members.size(); ++k) {
            check(cudaEventRecord(member_events[k], members[k]->stream), "batch event");
            check(cudaStreamWaitEvent(stream, member_events[k], 0), "batch event");
        }
    }

    void release_members(uint64_t count) {
        check(cudaEventRecord(done, stream), "batch event");
        for (std::size_t k = 0; k < members.size(); ++k) {
            orr_lbm3d* m = members[k];
            check(cudaStreamWaitEvent(m->stream, done, 0), "batch event");
            m->cur = parity[k] ^ static_cast<int>(flip);
            m->steps += count;
        }
    }

    // `count` steps of every member; with sample > 0 the force is summed into
    // the device sums after every `sample` steps (count a multiple of it,
    // sample even).
    void run(uint64_t count, uint32_t sample) {
        if (members.empty() || count == 0) {
            return;
        }
        if (stale() || (sample > 0 && flip != 0)) {
            rebuild();
        }
        wait_members();
        if (sample > 0) {
            check(cudaMemsetAsync(sums, 0, members.size() * 6 * sizeof(double), stream), "batch sums");
        }
        // Graphs cover whole sampling periods: the largest multiple of
        // `sample` up to kGraphSteps (at least one period).
        const uint32_t period = sample > 0 ? std::max<uint32_t>(1u, kGraphSteps / sample) * sample
                                           : kGraphSteps;
        uint64_t done_steps = 0;
        const auto single = [&]() {
            launch_steps(1);
            ++done_steps;
            if (sample > 0 && done_steps % sample == 0) {
                launch_sample(true);
            }
        };
        if (flip != 0) {
            single();
        }
        if (count - done_steps >= period) {
            if (!graph || graph_sample != sample || graph_steps != period) {
                build_graph(sample, period);
            }
            while (count - done_steps >= period) {
                check(cudaGraphLaunch(graph, stream), "batch graph launch");
                launches += graph_launches;
                done_steps += period;
            }
        }
        while (done_steps < count) {
            single();
        }
        release_members(count);
    }

    // The serving loop's use of the batch (serve3d.cu): before capturing one
    // sampling period of `sample` (even) steps as the body of its device
    // loop, the tables of the current members; after a launch that ran
    // `count` steps, the members' step counts and stream order.
    void prepare_loop(uint32_t sample) {
        (void)sample;
        if (stale() || flip != 0) {
            rebuild();
        }
    }
    void finish_loop(uint64_t count) { release_members(count); }

    void check_status() {
        uint32_t word = 0;
        check(cudaMemcpyAsync(&word, status, sizeof(word), cudaMemcpyDeviceToHost, stream), "batch status");
        check(cudaStreamSynchronize(stream), "batch status");
        if (word != 0u) {
            throw Refusal{ORR_ERR_TIMEOUT, "batch3d: a staged step gave up waiting for its row copies; the "
                                        "members' populations are invalid until they are initialised"};
        }
    }

    // Milliseconds per step of the current schedule over `graphs` graphs of
    // kGraphSteps steps (after one untimed graph).
    double time_schedule(uint32_t graphs) {
        run(kGraphSteps, 0);
        wait_members();
        check(cudaEventRecord(t0, stream), "tune event");
        for (uint32_t k = 0; k < graphs; ++k) {
            run_graph_only();
        }
        check(cudaEventRecord(t1, stream), "tune event");
        release_members(static_cast<uint64_t>(graphs) * kGraphSteps);
        check(cudaEventSynchronize(t1), "tune event");
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, t0, t1), "tune event");
        return static_cast<double>(ms) / (static_cast<double>(graphs) * kGraphSteps);
    }

    void run_graph_only() {
        if (!graph || graph_sample != 0 || graph_steps != kGraphSteps) {
            build_graph(0, kGraphSteps);
        }
        check(cudaGraphLaunch(graph, stream), "batch graph launch");
        launches += graph_launches;
    }
};

