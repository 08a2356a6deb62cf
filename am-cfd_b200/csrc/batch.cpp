// Parameter-sweep runner: many independent solver contexts on one GPU.
//
// The reference solves one melt-pool instance per process (main.cpp:25-233);
// a process-parameter sweep is many such runs.  Here every instance is a
// context with its own CUDA stream, and a pool of host threads drives them:
// a thread takes the next context in array order and runs all of its steps, so
// the GPU always has several instances' kernels queued from different streams.
// Contexts are never shared between threads; per-context state (the stream, the
// device status block, the error string) is all the step path touches.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "amcfd.h"

namespace amcfd {
int ctx_kind(const amcfd_ctx *ctx);
}

extern "C" int amcfd_run_batch(amcfd_ctx *const *ctxs, int n, int nsteps, int nthreads,
                               amcfd_step_report *reports, int *status)
{
    if (!ctxs || n < 0 || nsteps < 0 || nthreads < 0 || nthreads > 64) return AMCFD_E_ARG;
    if (n == 0) return 0;
    for (int q = 0; q < n; ++q)
        if (!ctxs[q]) return AMCFD_E_ARG;
    const int nt = std::min(n, nthreads == 0 ? 64 : nthreads);
    std::vector<int> st(n, 0), done(n, 0);
    std::vector<amcfd_step_report> rep(n);
    // The first step of the first context of each kind runs here, alone: it loads
    // every kernel that kind launches (a kernel's first launch loads its module,
    // which must not happen while another thread captures a graph).
    std::vector<int> kinds;
    for (int q = 0; q < n && nsteps > 0; ++q) {
        const int k = amcfd::ctx_kind(ctxs[q]);
        if (std::find(kinds.begin(), kinds.end(), k) != kinds.end()) continue;
        kinds.push_back(k);
        st[q] = amcfd_step(ctxs[q], &rep[q]);
        done[q] = 1;
    }
    std::atomic<int> next{0};
    auto work = [&]() {
        for (;;) {
            const int q = next.fetch_add(1);
            if (q >= n) return;
            int rc = st[q];
            for (int s = done[q]; s < nsteps && rc == 0; ++s) rc = amcfd_step(ctxs[q], &rep[q]);
            st[q] = rc;
            if (reports) reports[q] = rep[q];
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(nt);
    for (int t = 0; t < nt; ++t) pool.emplace_back(work);
    for (auto &th : pool) th.join();
    int first = 0;
    for (int q = 0; q < n; ++q) {
        if (status) status[q] = st[q];
        if (first == 0 && st[q] != 0) first = st[q];
    }
    return first;
}
