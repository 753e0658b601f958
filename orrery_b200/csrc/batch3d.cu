// A batch of D3Q19 solvers advanced together (no counterpart in the
// reference, which steps one lattice per solver through its backend).
//
// Members are ordinary solver handles (orr_lbm3d): their tables, buffers and
// read-back entry points are untouched; while a solver belongs to a batch its
// own step() is refused and the batch steps it.  A step of the batch is
//   staged schedule   one launch of the persistent staged kernel over a
//                     device table with one Lattice3D entry per member (all
//                     members' row tiles in one global work list), or
//   rows schedule     one row-tile kernel launch per member,
// captured as CUDA graphs of kGraphSteps steps.  Every schedule runs the same
// per-node code, so a member's populations after n steps do not depend on
// the schedule or on the other members (bit for bit).  The autotuner times
// the candidate schedules on the batch itself: its trial steps are real
// steps of every member.
//
// Forces are summed by the batched fixed-order reduction (force_batch):
// the same values for a lattice alone or in any mix.
//
// Streams: the batch has its own stream.  Before it steps, it waits for the
// work already queued on each member's stream; afterwards each member's
// stream waits for the batch, so member read-backs see the new state.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "batch3d_state.cuh"
#include "common.h"
#include "trace.h"
#include "solver3d_state.cuh"

using namespace orr;

namespace {

orr_batch3d* batch_of(orr_batch3d* b) {
    if (b == nullptr) {
        throw Refusal{ORR_ERR_INVALID, "null batch handle"};
    }
    check(cudaSetDevice(b->device), "cudaSetDevice");
    return b;
}

} // namespace

// Called by orr_lbm3d_destroy for a member that is still in a batch.
void orr_batch3d_forget(orr_batch3d* b, orr_lbm3d* m) noexcept {
    auto it = std::find(b->members.begin(), b->members.end(), m);
    if (it == b->members.end()) {
        return;
    }
    const std::size_t k = static_cast<std::size_t>(it - b->members.begin());
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    cudaEventDestroy(b->member_events[k]);
    b->member_events.erase(b->member_events.begin() + static_cast<std::ptrdiff_t>(k));
    b->members.erase(it);
    m->batch = nullptr;
    b->dirty = true;
    if (b->members.empty()) {
        b->storage = -1;
    }
}

extern "C" {

orr_status orr_batch3d_create(int32_t device, orr_batch3d** out) {
    if (out == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null output handle");
    }
    *out = nullptr;
    return orr::guarded(nullptr, [&]() -> orr_status {
        require_device(device);
        auto b = std::make_unique<orr_batch3d>();
        b->device = device;
        check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "batch stream");
        check(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "batch event");
        check(cudaEventCreate(&b->t0), "batch event");
        check(cudaEventCreate(&b->t1), "batch event");
        // The status word and the staged step's stall-request word.
        check(cudaMalloc(&b->status, 2 * sizeof(uint32_t)), "batch status");
        check(cudaMemsetAsync(b->status, 0, 2 * sizeof(uint32_t), b->stream), "batch status");
        check(cudaStreamSynchronize(b->stream), "batch create");
        *out = b.release();
        return ORR_OK;
    });
}

void orr_batch3d_destroy(orr_batch3d* batch) {
    if (batch != nullptr) {
        cudaSetDevice(batch->device);
        cudaStreamSynchronize(batch->stream);
    }
    delete batch;
}

const char* orr_batch3d_last_error(const orr_batch3d* batch) {
    return batch ? batch->error.c_str() : orr_last_error();
}

orr_status orr_batch3d_add(orr_batch3d* batch, orr_lbm3d* solver) {
    return orr::guarded(batch ? &batch->error : nullptr, [&]() -> orr_status {
        orr_batch3d* b = batch_of(batch);
        if (solver == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "batch3d: null solver handle"};
        }
        if (solver->batch != nullptr) {
            throw Refusal{ORR_ERR_INVALID, "batch3d: the solver already belongs to a batch"};
        }
        if (solver->device != b->device) {
            throw Refusal{ORR_ERR_INVALID, "batch3d: the solver lives on another device"};
        }
        if (!b->members.empty()) {
            if (solver->storage != b->storage) {
                throw Refusal{ORR_ERR_INVALID, "batch3d: all members store their populations in one form"};
            }
            if (solver->smag != b->smag) {
                throw Refusal{ORR_ERR_INVALID,
                              "batch3d: all members use the Smagorinsky closure, or none does"};
            }
        } else {
            b->storage = solver->storage;
            b->smag = solver->smag;
            b->ops = solver->ops;
        }
        cudaEvent_t e = nullptr;
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch event");
        b->member_events.push_back(e);
        b->members.push_back(solver);
        solver->batch = b;
        b->dirty = true;
        return ORR_OK;
    });
}

orr_status orr_batch3d_remove(orr_batch3d* batch, orr_lbm3d* solver) {
    return orr::guarded(batch ? &batch->error : nullptr, [&]() -> orr_status {
        orr_batch3d* b = batch_of(batch);
        if (solver == nullptr || solver->batch != b) {
            throw Refusal{ORR_ERR_INVALID, "batch3d: the solver is not a member of this batch"};
        }
        orr_batch3d_forget(b, solver);
        return ORR_OK;
    });
}

orr_status orr_batch3d_size(const orr_batch3d* batch, uint32_t* members, uint64_t* cells) {
    if (batch == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null batch handle");
    }
    uint64_t n = 0;
    for (const orr_lbm3d* m : batch->members) {
        n += m->g.cells;
    }
    if (members) *members = static_cast<uint32_t>(batch->members.size());
    if (cells) *cells = n;
    return ORR_OK;
}

orr_status orr_batch3d_set_schedule(orr_batch3d* batch, const orr_batch_schedule* schedule) {
    return orr::guarded(batch ? &batch->error : nullptr, [&]() -> orr_status {
        orr_batch3d* b = batch_of(batch);
        if (schedule == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "batch3d: null schedule"};
        }
        const orr_batch_schedule& s = *schedule;
        if (s.kernel == ORR_KERNEL_STAGED) {
            if (s.block != 128 && s.block != 256) {
                throw Refusal{ORR_ERR_INVALID, "batch3d: the staged step takes block 128 or 256"};
            }
            if (s.stages > kMaxStages) {
                throw Refusal{ORR_ERR_INVALID, "batch3d: stages must be 0 (tuned) or 1 to 8"};
            }
            if (s.nodes_per_thread > 2) {
                throw Refusal{ORR_ERR_INVALID, "batch3d: nodes_per_thread must be 0 (default), 1 or 2"};
            }
        } else if (s.kernel == ORR_KERNEL_ROWS) {
            if (s.block == 0 || s.block > 256 || s.block % 32 != 0) {
                throw Refusal{ORR_ERR_INVALID, "batch3d: the row step takes a block of 32 to 256 threads"};
            }
            if (s.nodes_per_thread > 2) {
                throw Refusal{ORR_ERR_INVALID, "batch3d: nodes_per_thread must be 0 (default), 1 or 2"};
            }
        } else {
            throw Refusal{ORR_ERR_INVALID, "batch3d: unknown step kernel"};
        }
        b->kernel = s.kernel;
        b->block = s.block;
        b->stages = s.kernel == ORR_KERNEL_STAGED ? s.stages : 0;
        b->npt = s.nodes_per_thread;
        b->branches = s.branches;
        b->dirty = true;
        return ORR_OK;
    });
}

orr_status orr_batch3d_schedule(const orr_batch3d* batch, orr_batch_schedule* schedule) {
    if (batch == nullptr || schedule == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    orr_batch_schedule s{};
    s.kernel = batch->kernel;
    s.block = batch->block;
    s.stages = batch->kernel == ORR_KERNEL_STAGED ? (batch->shape.stages ? batch->shape.stages : batch->stages) : 0;
    s.grid = batch->kernel == ORR_KERNEL_STAGED ? batch->shape.grid : 0;
    s.nodes_per_thread = batch->kernel == ORR_KERNEL_STAGED
                             ? (batch->shape.npt && !batch->dirty ? batch->shape.npt : batch->npt)
                             : (batch->npt == 2 ? 2u : 1u);
    s.branches = batch->branches;
    s.ms_per_step = 0.0;
    *schedule = s;
    return ORR_OK;
}

orr_status orr_batch3d_step(orr_batch3d* batch, uint64_t count) {
    orr::Zone zone("batch_step");
    return orr::guarded(batch ? &batch->error : nullptr, [&]() -> orr_status {
        orr_batch3d* b = batch_of(batch);
        b->run(count, 0);
        return ORR_OK;
    });
}

orr_status orr_batch3d_step_sampled(orr_batch3d* batch, uint64_t count, uint32_t sample_every,
                                    double* sums) {
    orr::Zone zone("batch_step");
    return orr::guarded(batch ? &batch->error : nullptr, [&]() -> orr_status {
        orr_batch3d* b = batch_of(batch);
        if (sample_every == 0 || sample_every % 2 != 0 || count % sample_every != 0) {
            throw Refusal{ORR_ERR_INVALID,
                          "batch3d: the sampling interval must be even and divide the step count"};
        }
        if (b->members.empty()) {
            return ORR_OK;
        }
        b->run(count, sample_every);
        if (b->kernel == ORR_KERNEL_STAGED) {
            b->check_status();
        }
        if (sums != nullptr) {
            check(cudaMemcpyAsync(sums, b->sums, b->members.size() * 6 * sizeof(double), cudaMemcpyDeviceToHost,
                                  b->stream),
                  "batch sums read-back");
        }
        check(cudaStreamSynchronize(b->stream), "batch sums read-back");
        return ORR_OK;
    });
}

orr_status orr_batch3d_forces(orr_batch3d* batch, double* force_moment) {
    return orr::guarded(batch ? &batch->error : nullptr, [&]() -> orr_status {
        orr_batch3d* b = batch_of(batch);
        if (force_moment == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "batch3d: null output"};
        }
        if (b->members.empty()) {
            return ORR_OK;
        }
        if (b->stale()) {
            b->rebuild();
        }
        if (b->flip != 0) {
            throw Refusal{ORR_ERR_INVALID, "batch3d: forces are sampled after an even number of batch steps"};
        }
        b->wait_members();
        b->launch_sample(false);
        if (b->kernel == ORR_KERNEL_STAGED) {
            b->check_status();
        }
        check(cudaMemcpyAsync(force_moment, b->sums, b->members.size() * 6 * sizeof(double),
                              cudaMemcpyDeviceToHost, b->stream),
              "batch force read-back");
        check(cudaStreamSynchronize(b->stream), "batch force read-back");
        return ORR_OK;
    });
}

orr_status orr_batch3d_tune(orr_batch3d* batch, uint32_t graphs_per_trial, orr_batch_schedule* trials,
                            uint32_t capacity, uint32_t* count) {
    return orr::guarded(batch ? &batch->error : nullptr, [&]() -> orr_status {
        orr_batch3d* b = batch_of(batch);
        if (b->members.empty()) {
            throw Refusal{ORR_ERR_INVALID, "batch3d: nothing to tune in an empty batch"};
        }
        const uint32_t graphs = std::max<uint32_t>(graphs_per_trial, 1);
        double best = 0.0;
        Candidate pick = kCandidates[0];
        uint32_t n = 0;
        for (const Candidate& c : kCandidates) {
            if (c.kernel == ORR_KERNEL_STAGED &&
                (!b->all_flat() || b->ops->staged_occupancy(b->smag, c.block, c.npt, c.stages) <= 0)) {
                continue;
            }
            b->kernel = c.kernel;
            b->block = c.block;
            b->stages = c.stages;
            b->npt = c.npt;
            b->branches = c.branches;
            b->dirty = true;
            const double ms = b->time_schedule(graphs);
            if (trials != nullptr && n < capacity) {
                orr_batch_schedule& t = trials[n];
                t.kernel = c.kernel;
                t.block = c.block;
                t.stages = c.stages;
                t.nodes_per_thread = c.npt;
                t.branches = c.branches;
                t.grid = c.kernel == ORR_KERNEL_STAGED ? b->shape.grid : 0;
                t.ms_per_step = ms;
            }
            ++n;
            if (best == 0.0 || ms < best) {
                best = ms;
                pick = c;
            }
        }
        b->kernel = pick.kernel;
        b->block = pick.block;
        b->stages = pick.stages;
        b->npt = pick.npt;
        b->branches = pick.branches;
        b->dirty = true;
        if (count) *count = n;
        return ORR_OK;
    });
}

orr_status orr_batch3d_synchronize(orr_batch3d* batch) {
    return orr::guarded(batch ? &batch->error : nullptr, [&]() -> orr_status {
        orr_batch3d* b = batch_of(batch);
        check(cudaStreamSynchronize(b->stream), "batch synchronize");
        if (b->kernel == ORR_KERNEL_STAGED && !b->members.empty()) {
            b->check_status();
        }
        return ORR_OK;
    });
}

orr_status orr_batch3d_stream(const orr_batch3d* batch, void** stream) {
    if (batch == nullptr || stream == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *stream = batch->stream;
    return ORR_OK;
}

orr_status orr_batch3d_launch_count(const orr_batch3d* batch, uint64_t* launches) {
    if (batch == nullptr || launches == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *launches = batch->launches;
    return ORR_OK;
}

} // extern "C"
