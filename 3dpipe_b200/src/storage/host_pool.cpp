// host_pool.cpp -- see host_pool.h.
#include "host_pool.h"

#include <sched.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>

namespace tdp {
namespace {

// One loop: tasks are claimed through `next`; `refs` counts the workers
// inside it, so the caller can tell when none of them still touches it.
struct Job {
    const std::function<void(long)>* fn = nullptr;
    long n = 0;
    std::atomic<long> next{0};
    int refs = 0;                // guarded by Pool::m
    std::exception_ptr error;    // the first task that threw (guarded by Pool::m)
};

struct Pool {
    std::mutex loop;  // one loop at a time
    std::mutex m;
    std::condition_variable work, idle;
    Job* cur = nullptr;
    unsigned long long gen = 0;
    std::vector<std::thread> workers;
};

thread_local bool t_in_task = false;

// Runs tasks until none is left; a task that throws ends this thread's share
// (the exception is returned; threads still in the loop take the rest).
std::exception_ptr run_tasks(Job& J) {
    const bool outer = t_in_task;
    t_in_task = true;
    std::exception_ptr err;
    try {
        for (long k = J.next++; k < J.n; k = J.next++) (*J.fn)(k);
    } catch (...) {
        err = std::current_exception();
    }
    t_in_task = outer;
    return err;
}

void worker_main(Pool* P) {
    unsigned long long seen = 0;
    std::unique_lock<std::mutex> lk(P->m);
    for (;;) {
        P->work.wait(lk, [&] { return P->gen != seen; });
        seen = P->gen;
        Job* J = P->cur;
        if (!J) continue;
        ++J->refs;
        lk.unlock();
        std::exception_ptr err = run_tasks(*J);
        lk.lock();
        if (err && !J->error) J->error = err;
        if (--J->refs == 0) P->idle.notify_all();
    }
}

int affinity_threads() {
    cpu_set_t s;
    CPU_ZERO(&s);
    if (sched_getaffinity(0, sizeof(s), &s) == 0) {
        const int c = CPU_COUNT(&s);
        if (c > 0) return c;
    }
    return (int)std::max(1u, std::thread::hardware_concurrency());
}

std::mutex g_make;
Pool* g_pool = nullptr;
pid_t g_owner = 0;

// The pool of this process: made on first use, and made again in a child
// after fork (the old object is abandoned: its workers and the state of
// its mutexes belong to the parent).
Pool* pool() {
    std::lock_guard<std::mutex> g(g_make);
    const pid_t me = getpid();
    if (!g_pool || g_owner != me) {
        Pool* P = new Pool();
        const int nw = std::min(host_threads(), 64) - 1;
        for (int i = 0; i < nw; ++i) {
            P->workers.emplace_back(worker_main, P);
            P->workers.back().detach();
        }
        g_pool = P;
        g_owner = me;
    }
    return g_pool;
}

}  // namespace

int host_threads() {
    static const int n = affinity_threads();
    return n;
}

void host_for(long n, const std::function<void(long)>& fn) {
    if (n <= 0) return;
    if (n == 1 || t_in_task || host_threads() <= 1) {
        for (long k = 0; k < n; ++k) fn(k);
        return;
    }
    Pool* P = pool();
    std::lock_guard<std::mutex> one(P->loop);
    Job J;
    J.fn = &fn;
    J.n = n;
    {
        std::lock_guard<std::mutex> lk(P->m);
        P->cur = &J;
        ++P->gen;
    }
    P->work.notify_all();
    std::exception_ptr err = run_tasks(J);
    // every task is claimed once the caller's own loop ends (or has thrown);
    // wait for the workers still running one, after which none can enter
    // this job, then pass on the first exception a task threw
    {
        std::unique_lock<std::mutex> lk(P->m);
        P->cur = nullptr;
        P->idle.wait(lk, [&] { return J.refs == 0; });
        if (!err) err = J.error;
    }
    if (err) std::rethrow_exception(err);
}

}  // namespace tdp
