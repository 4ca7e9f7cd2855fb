// profile.cpp -- launch counting and optional per-kernel CUDA-event timing.
//
// Every kernel launch of the library increments a process-wide counter
// (raft_launch_count).  When timing is enabled (raft_profile_enable(1)),
// the filter and backprojector launches are bracketed by CUDA events on the
// stream they are issued on; raft_profile_read() synchronises those events
// and returns the summed device time per kernel class.
#include "profile.hpp"

#include <atomic>
#include <mutex>
#include <vector>

namespace raft {

static std::atomic<long long> g_launches{0};
static std::atomic<int> g_profile{0};
static std::mutex g_prof_mtx;
struct Rec {
    int kind;
    cudaEvent_t a, b;
};
static std::vector<Rec> g_recs;

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

ProfScope::ProfScope(int kind, cudaStream_t st) : kind_(kind), st_(st)
{
    count_launch();
    if (!g_profile.load()) return;
    cudaEventCreate(&a_);
    cudaEventCreate(&b_);
    cudaEventRecord(a_, st_);
    active_ = true;
}

ProfScope::~ProfScope()
{
    if (!active_) return;
    cudaEventRecord(b_, st_);
    std::lock_guard<std::mutex> lk(g_prof_mtx);
    g_recs.push_back({kind_, a_, b_});
}

}  // namespace raft

extern "C" {

long long raft_launch_count(void) { return raft::g_launches.load(); }

void raft_profile_enable(int on)
{
    raft::g_profile.store(on ? 1 : 0);
}

// Sums device time (ms) and launch counts per kernel class since the last
// read: classes 0 filter, 1 backprojector, 2 projector.  Returns records read.
int raft_profile_read(double *ms, long long *counts, int nclasses)
{
    std::vector<raft::Rec> recs;
    {
        std::lock_guard<std::mutex> lk(raft::g_prof_mtx);
        recs.swap(raft::g_recs);
    }
    for (int c = 0; c < nclasses; c++) {
        if (ms) ms[c] = 0.0;
        if (counts) counts[c] = 0;
    }
    for (auto &r : recs) {
        float t = 0.f;
        cudaEventSynchronize(r.b);
        cudaEventElapsedTime(&t, r.a, r.b);
        if (r.kind >= 0 && r.kind < nclasses) {
            if (ms) ms[r.kind] += t;
            if (counts) counts[r.kind] += 1;
        }
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    return (int)recs.size();
}

}  // extern "C"
