// serve.hpp -- a serving runtime for trees: requests to build new trees and
// to update or release resident ones, run concurrently under a device-memory
// budget.
//
// The reference has no serving layer; its callers build and update one tree
// at a time.  Here a request queue feeds `slots` worker threads.  Every
// resident tree keeps its buffers (and its own copy of its coordinates) on
// the device between requests and runs on its own CUDA stream, so requests
// on different trees overlap on the GPU.  Admission:
//   * a build is admitted when the memory it needs fits the budget next to
//     the resident trees and the builds in flight; builds are admitted in
//     arrival order (a large build is not starved by smaller ones behind it);
//   * updates and releases need no new memory and pass waiting builds;
//   * requests on one tree run in arrival order, one at a time.
// An update that exceeds the tree's capacity is completed by the
// resizeBuffers()/update() retry of the reference's callers.  Results are
// those of the same requests run one at a time (tested).
#pragma once

#include <condition_variable>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"

namespace aot
{
struct ServeRequest
{
    enum Op { Build = 0, Update = 1, Release = 2 };
    int op = Build;
    long long tree = 0;     // caller-chosen id (unique among resident trees)
    EngineConfig cfg;       // build: tree config (the stream is the server's)
    size_t n = 0;           // build: particles; update: must match the tree
    const void *x = nullptr, *y = nullptr, *z = nullptr;  // build/update: coordinates (device or pinned host)
    bool digest = false;    // hash the tree's outputs when the request completes
};

struct ServeResult
{
    int status = 0;          // ao_status
    std::string message;
    double queuedMs = 0;     // submit -> start
    double latencyMs = 0;    // submit -> result ready
    size_t leaves = 0;
    int resizes = 0;
    unsigned long long digest = 0;
};

struct ServeStats
{
    size_t submitted = 0, completed = 0, failed = 0, residentTrees = 0;
    size_t residentBytes = 0, peakBytes = 0;
    double p50Ms = 0, p99Ms = 0, meanMs = 0, maxMs = 0, particlesPerS = 0, spanS = 0;
    unsigned long long particles = 0;
};

class Server
{
public:
    Server(int slots, size_t budgetBytes);
    ~Server();
    Server(const Server &) = delete;
    Server &operator=(const Server &) = delete;

    long long submit(const ServeRequest &r);  // returns a ticket; never blocks on the GPU
    ServeResult wait(long long ticket);       // blocks until that request is done
    void drain();                             // blocks until every submitted request is done
    ServeStats stats();
    void resetStats();

private:
    struct Tree;
    struct Job
    {
        long long ticket;
        ServeRequest req;
        std::chrono::steady_clock::time_point submitted;
        size_t reserve = 0;  // bytes reserved at admission (builds)
    };
    void worker();
    bool admit(Job &out);  // with mu held
    void run(Job &job, ServeResult &res);

    int device_ = 0;
    size_t budget_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    std::deque<Job> queue_;
    std::map<long long, std::unique_ptr<Tree>> trees_;
    std::map<long long, ServeResult> results_;
    std::map<long long, int> pendingOps_;  // queued or running requests per tree id
    size_t resident_ = 0, reserved_ = 0, peak_ = 0, running_ = 0;
    long long nextTicket_ = 1;
    bool stop_ = false;
    std::vector<std::thread> workers_;
    // statistics
    std::vector<double> latencies_;
    size_t submitted_ = 0, failed_ = 0;
    unsigned long long particles_ = 0;
    std::chrono::steady_clock::time_point first_, last_;
    bool any_ = false;
};
}  // namespace aot
