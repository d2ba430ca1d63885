// host_pool.h -- one process-wide pool of host worker threads for the
// parallel loops of the tile parser and of tdp_tile_attach.
//
// Starting a thread costs tens of microseconds and an attach runs several
// parallel loops per tile (record placement, voxel counts, object records,
// prefix sums), so the loops borrow long-lived workers instead of starting
// their own.  The pool is sized by the CPUs the process may run on (its
// affinity mask), started on first use, and started again in a child
// process after fork (the parent's workers do not exist there).
#pragma once

#include <functional>

namespace tdp {

// threads the process may run on (at least 1)
int host_threads();

// fn(k) for every k in [0, n), on the pool's workers and the calling thread;
// returns when every call has returned.  A call made from inside fn runs its
// tasks serially on the calling thread.  One loop runs at a time; concurrent
// callers queue.  If a call throws, the loop still waits for the calls in
// flight and then rethrows the first exception (tasks not yet started when
// the throwing thread stopped may be skipped).
void host_for(long n, const std::function<void(long)>& fn);

// fn(b, e) over [0, n) in at most host_threads() contiguous ranges of at
// least `grain` items each (one range, on the calling thread, for small n)
template <typename Fn>
void host_ranges(long n, long grain, Fn&& fn) {
    if (n <= 0) return;
    long nt = grain > 0 ? n / grain : n;
    if (nt > host_threads()) nt = host_threads();
    if (nt <= 1) {
        fn(0L, n);
        return;
    }
    host_for(nt, [&](long k) { fn(n * k / nt, n * (k + 1) / nt); });
}

}  // namespace tdp
