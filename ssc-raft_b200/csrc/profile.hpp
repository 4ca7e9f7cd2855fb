// profile.hpp -- launch accounting shared by the kernel launchers.
#pragma once
#include <cuda_runtime.h>

namespace raft {

enum ProfKind : int { PROF_FILTER = 0, PROF_BACKPROJECT = 1, PROF_PROJECT = 2, PROF_OTHER = 3 };

void count_launch();

// RAII: counts one launch; with profiling on, records events around it.
class ProfScope {
  public:
    ProfScope(int kind, cudaStream_t st);
    ~ProfScope();

  private:
    int kind_;
    cudaStream_t st_;
    cudaEvent_t a_ = nullptr, b_ = nullptr;
    bool active_ = false;
};

}  // namespace raft
