// serve.cpp -- the serving runtime (serve.hpp).
#include "serve.hpp"

#include <algorithm>
#include <set>
#include <stdexcept>

namespace aot
{
struct Server::Tree
{
    std::unique_ptr<TreeEngine> engine;
    DevMem coords[3];  // the tree's own copy of its coordinates
    cudaStream_t stream = nullptr;
    size_t n = 0, realBytes = 4, bytes = 0;
    bool busy = true;
};

namespace
{
using Clock = std::chrono::steady_clock;

double ms(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); }

// device bytes a build of n particles may need before it is measured: its
// coordinates, keys and permutation (both halves), the key sample, the sort's
// look-back status (room for every sort configuration the tuner may time:
// 10 passes of 2048-key tiles, 256 digits of 8 B, 10 B per particle), the
// leaf arrays and (NFCount) the node table
size_t buildEstimate(const ServeRequest &r)
{
    const size_t n = r.n, rb = r.cfg.real ? 8 : 4;
    const size_t leaves = r.cfg.nf ? n + 4096 : n / std::max(1u, r.cfg.bucket) * 8 + 4096;
    // NFCount trees add the node table: a quarter slot of 48 B per leaf of capacity
    return n * (3 * rb + 24 + 8 + 11) + leaves * (r.cfg.nf ? 64 + 12 : 64) + (size_t(1) << 20);
}

// exception -> ao_status (as the C ABI maps them)
int statusOf(const std::exception_ptr &e, std::string &msg)
{
    try
    {
        std::rethrow_exception(e);
    }
    catch (const std::invalid_argument &x)
    {
        msg = x.what();
        return 1;
    }
    catch (const std::length_error &x)
    {
        msg = x.what();
        return 3;
    }
    catch (const std::logic_error &x)
    {
        msg = x.what();
        return 2;
    }
    catch (const CudaError &x)
    {
        msg = x.what();
        return x.code == cudaErrorMemoryAllocation ? 5 : 4;
    }
    catch (const std::bad_alloc &x)
    {
        msg = x.what();
        return 5;
    }
    catch (const std::exception &x)
    {
        msg = x.what();
        return 6;
    }
    catch (...)
    {
        msg = "unknown error";
        return 6;
    }
}

// FNV-1a over the tree's output buffers (keys, permutation, cornerstone, counts, near-field counts)
unsigned long long digestOf(const TreeEngine &e)
{
    unsigned long long h = 1469598103934665603ull;
    std::vector<unsigned char> host;
    for (int which : {int(TreeEngine::ParticleKeys), int(TreeEngine::Perm), int(TreeEngine::Cornerstone),
                      int(TreeEngine::LeafCounts), int(TreeEngine::NearFieldCounts)})
    {
        if (which == TreeEngine::NearFieldCounts && e.config().kind != 0) continue;
        const void *p = nullptr;
        size_t len = 0, cap = 0, elem = 0;
        e.buffer(which, &p, &len, &cap, &elem);
        host.resize(len * elem);
        if (!host.empty()) AOT_CHECK(cudaMemcpy(host.data(), p, host.size(), cudaMemcpyDeviceToHost));
        for (unsigned char c : host) h = (h ^ c) * 1099511628211ull;
        h = (h ^ 0xff) * 1099511628211ull;  // buffer separator
    }
    return h;
}
}  // namespace

Server::Server(int slots, size_t budgetBytes) : budget_(budgetBytes)
{
    if (slots <= 0) throw std::invalid_argument("server: need at least one slot");
    if (budgetBytes == 0) throw std::invalid_argument("server: the memory budget must be positive");
    AOT_CHECK(cudaGetDevice(&device_));
    // the streams and events of `slots` requests in flight (a tree's stream,
    // its engine's read-back and side streams, three events), created now
    // rather than by the first requests
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    for (int i = 0; i < 3 * slots; ++i) streams.push_back(blockcache::takeStream());
    for (int i = 0; i < 3 * slots; ++i) events.push_back(blockcache::takeEvent());
    for (cudaStream_t st : streams) blockcache::giveStream(st, device_);
    for (cudaEvent_t e : events) blockcache::giveEvent(e, device_);
    for (int i = 0; i < slots; ++i) workers_.emplace_back([this] { worker(); });
}

Server::~Server()
{
    {
        std::lock_guard<std::mutex> lock(mu_);
        for (Job &j : queue_)
        {
            ServeResult r;
            r.status = 6;
            r.message = "server: destroyed before the request ran";
            results_[j.ticket] = r;
        }
        queue_.clear();
        stop_ = true;
    }
    cv_.notify_all();
    for (std::thread &t : workers_) t.join();
    for (auto &kv : trees_)
    {
        kv.second->engine.reset();
        if (kv.second->stream) blockcache::giveStream(kv.second->stream, device_);
    }
}

long long Server::submit(const ServeRequest &r)
{
    if (r.op < ServeRequest::Build || r.op > ServeRequest::Release)
        throw std::invalid_argument("server: unknown request");
    if (r.op != ServeRequest::Release && r.n > 0 && (!r.x || !r.y || !r.z))
        throw std::invalid_argument("server: null coordinates");
    long long t;
    {
        std::lock_guard<std::mutex> lock(mu_);
        if (stop_) throw std::logic_error("server: stopping");
        t = nextTicket_++;
        Job j{t, r, Clock::now(), 0};
        if (!any_)
        {
            first_ = j.submitted;
            any_ = true;
        }
        queue_.push_back(j);
        ++submitted_;
        ++pendingOps_[r.tree];
    }
    cv_.notify_all();
    return t;
}

// The first queued request that may run now: not behind an earlier request
// on its tree, and (builds) fitting the budget, builds in arrival order.
bool Server::admit(Job &out)
{
    std::set<long long> blocked;
    bool buildWaits = false;
    for (auto it = queue_.begin(); it != queue_.end(); ++it)
    {
        Job &j = *it;
        const long long id = j.req.tree;
        if (blocked.count(id)) continue;
        auto tr = trees_.find(id);
        if (j.req.op == ServeRequest::Build)
        {
            if (tr != trees_.end())
            {
                if (tr->second->busy) { blocked.insert(id); continue; }
                // duplicate id: run() reports it
            }
            else
            {
                if (buildWaits) { blocked.insert(id); continue; }
                const size_t est = buildEstimate(j.req);
                if (est <= budget_ && resident_ + reserved_ + est > budget_)
                {
                    buildWaits = true;
                    blocked.insert(id);
                    continue;
                }
                j.reserve = est <= budget_ ? est : 0;  // above the budget: run() reports it
                reserved_ += j.reserve;
                if (est <= budget_)
                {
                    auto t = std::make_unique<Tree>();
                    t->busy = true;
                    trees_[id] = std::move(t);
                }
            }
        }
        else if (tr != trees_.end())
        {
            if (tr->second->busy) { blocked.insert(id); continue; }
            tr->second->busy = true;
        }
        out = j;
        queue_.erase(it);
        peak_ = std::max(peak_, resident_ + reserved_);
        return true;
    }
    return false;
}

void Server::worker()
{
    (void)cudaSetDevice(device_);
    sleepingWaits(true);  // many workers wait at once: do not spin
    std::unique_lock<std::mutex> lk(mu_);
    for (;;)
    {
        Job job;
        bool got = false;
        cv_.wait(lk, [&] {
            got = admit(job);
            return got || (stop_ && queue_.empty());
        });
        if (!got) return;
        ++running_;
        lk.unlock();
        ServeResult res;
        run(job, res);
        const Clock::time_point end = Clock::now();
        lk.lock();
        --running_;
        res.latencyMs = ms(job.submitted, end);
        last_ = std::max(last_, end);
        if (res.status == 0)
        {
            latencies_.push_back(res.latencyMs);
            if (job.req.op != ServeRequest::Release) particles_ += job.req.n;
        }
        else
        {
            ++failed_;
        }
        results_[job.ticket] = res;
        auto p = pendingOps_.find(job.req.tree);
        if (p != pendingOps_.end() && --p->second == 0) pendingOps_.erase(p);
        lk.unlock();
        cv_.notify_all();
        done_.notify_all();
        lk.lock();
    }
}

void Server::run(Job &job, ServeResult &res)
{
    const ServeRequest &r = job.req;
    const Clock::time_point start = Clock::now();
    res.queuedMs = ms(job.submitted, start);
    Tree *t = nullptr;
    {
        std::lock_guard<std::mutex> lock(mu_);
        auto it = trees_.find(r.tree);
        if (it != trees_.end()) t = it->second.get();
    }
    try
    {
        if (r.op == ServeRequest::Build)
        {
            if (job.reserve == 0)
            {
                if (t) throw std::invalid_argument("server: a resident tree already has this id");
                throw std::length_error("server: the build needs more device memory than the whole budget");
            }
            t->stream = blockcache::takeStream();
            EngineConfig cfg = r.cfg;
            cfg.tuneSort = false;  // no timing runs inside a request
            cfg.stream = t->stream;
            t->n = r.n;
            t->realBytes = cfg.real ? 8 : 4;
            const void *src[3] = {r.x, r.y, r.z};
            for (int k = 0; k < 3; ++k)
            {
                t->coords[k].reserve(std::max<size_t>(r.n * t->realBytes, 16));
                if (r.n)
                    AOT_CHECK(cudaMemcpyAsync(t->coords[k].p, src[k], r.n * t->realBytes, cudaMemcpyDefault,
                                              t->stream));
            }
            t->engine = std::make_unique<TreeEngine>(t->coords[0].p, t->coords[1].p, t->coords[2].p, r.n, cfg);
            t->engine->build();
        }
        else if (r.op == ServeRequest::Update)
        {
            if (!t || !t->engine) throw std::invalid_argument("server: no resident tree with this id");
            if (r.n != t->n) throw std::invalid_argument("server: an update must keep the tree's particle count");
            const void *src[3] = {r.x, r.y, r.z};
            for (int k = 0; k < 3; ++k)
                if (r.n)
                    AOT_CHECK(cudaMemcpyAsync(t->coords[k].p, src[k], r.n * t->realBytes, cudaMemcpyDefault,
                                              t->stream));
            t->engine->update();
            while (t->engine->doBuffersNeedResize())
            {
                if (++res.resizes > 64) throw std::runtime_error("server: update did not fit after 64 resizes");
                t->engine->resizeBuffers();
                t->engine->update();
            }
        }
        else
        {
            if (!t || !t->engine) throw std::invalid_argument("server: no resident tree with this id");
            t->engine.reset();  // synchronises the tree's stream
            for (DevMem &c : t->coords) c.release();
            blockcache::giveStream(t->stream, device_);
            t->stream = nullptr;
        }
        if (t && t->engine)
        {
            res.leaves = t->engine->numLeaves();
            if (r.digest) res.digest = digestOf(*t->engine);
        }
    }
    catch (...)
    {
        res.status = statusOf(std::current_exception(), res.message);
    }
    // bookkeeping
    std::lock_guard<std::mutex> lock(mu_);
    reserved_ -= job.reserve;
    if (!t) return;
    if (r.op == ServeRequest::Build)
    {
        // rejected at admission (duplicate id, above the budget): nothing was created
        if (job.reserve == 0) return;
        if (res.status != 0)
        {
            // a failed build leaves no tree behind
            t->engine.reset();
            if (t->stream) blockcache::giveStream(t->stream, device_);
            trees_.erase(r.tree);
            return;
        }
    }
    if (r.op == ServeRequest::Release && res.status == 0)
    {
        resident_ -= t->bytes;
        trees_.erase(r.tree);
        return;
    }
    if (t->engine)
    {
        const size_t now = t->engine->deviceBytes() + t->coords[0].bytes + t->coords[1].bytes + t->coords[2].bytes;
        resident_ = resident_ - t->bytes + now;
        t->bytes = now;
    }
    peak_ = std::max(peak_, resident_ + reserved_);
    t->busy = false;
}

ServeResult Server::wait(long long ticket)
{
    std::unique_lock<std::mutex> lk(mu_);
    if (ticket <= 0 || ticket >= nextTicket_) throw std::invalid_argument("server: unknown ticket");
    done_.wait(lk, [&] { return results_.count(ticket) != 0; });
    ServeResult r = results_[ticket];
    results_.erase(ticket);
    return r;
}

void Server::drain()
{
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return queue_.empty() && running_ == 0; });
}

ServeStats Server::stats()
{
    std::lock_guard<std::mutex> lock(mu_);
    ServeStats s;
    s.submitted = submitted_;
    s.completed = latencies_.size() + failed_;
    s.failed = failed_;
    s.residentTrees = trees_.size();
    s.residentBytes = resident_;
    s.peakBytes = peak_;
    s.particles = particles_;
    if (!latencies_.empty())
    {
        std::vector<double> v = latencies_;
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) { return v[std::min(v.size() - 1, size_t(q * double(v.size() - 1) + 0.5))]; };
        s.p50Ms = pct(0.50);
        s.p99Ms = pct(0.99);
        s.maxMs = v.back();
        double sum = 0;
        for (double x : v) sum += x;
        s.meanMs = sum / double(v.size());
    }
    if (any_ && last_ > first_)
    {
        s.spanS = std::chrono::duration<double>(last_ - first_).count();
        s.particlesPerS = double(particles_) / s.spanS;
    }
    return s;
}

void Server::resetStats()
{
    std::lock_guard<std::mutex> lock(mu_);
    latencies_.clear();
    submitted_ = failed_ = 0;
    particles_ = 0;
    any_ = false;
    peak_ = resident_ + reserved_;
    last_ = Clock::time_point{};
}
}  // namespace aot
