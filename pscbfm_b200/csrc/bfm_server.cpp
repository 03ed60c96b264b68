// Server: continuous batching of "run this system for M MCS, sample observables every k" jobs.
//
// Jobs are submitted from any host thread (the system is described by a handle configured with
// the setter API; the server copies that description). A worker thread admits pending jobs in
// arrival order while their estimated device bytes fit the budget and initialises them
// (colouring, upload) while the GPU runs the others. Running jobs are grouped into lanes by how
// they run: one lane for the systems on the grid-phase kernels and one per size class of the
// systems that fit one CTA (resident kernel). Each lane is a Batch advanced in chunks on its own
// streams; the lanes run concurrently and the worker services whichever lane finishes a chunk
// first, so small jobs never wait for the chunks of large ones. A chunk ends at the nearest sample
// point of the lane's jobs (capped at kMaxChunkMcs), so every job samples exactly at its
// multiples of k; a job whose end falls inside a chunk runs only its remaining MCS. Finished and
// cancelled jobs leave between chunks and their memory is freed in stream order. Each job keeps
// its own draw stream, so its result equals running it alone.
//
// Failure handling stays on the host: a malformed job fails at submit, a job larger than the
// budget is refused, a job whose set-up throws is marked failed, and a worker that dies marks
// every job failed and makes later calls return an error instead of hanging. No wait is unbounded.

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "bfm_engine.hpp"
#include "bfm_server.hpp"

namespace bfm {

using Clock = std::chrono::steady_clock;

// longest stretch of MCS a lane advances between two admission points
constexpr int32_t kMaxChunkMcs = 256;
// lanes of the systems on the grid-phase kernels (kGridLane .. kGridLane + kGridLanes - 1);
// resident lanes are 0..4 (log2 monomers per thread)
constexpr int kGridLane = 100;
constexpr int kGridLanes = 4;

struct Server::Job {
    uint64_t id = 0;
    int state = kJobPending;
    std::unique_ptr<Updater> u;
    int32_t nMcs = 0, every = 0, done = 0;
    size_t bytes = 0;
    Clock::time_point arrival, start, finish;
    std::vector<long long> samples;
    std::vector<int32_t> xyz;
    std::string error;
    bool cancel = false;
};

size_t Server::estimateBytes(Updater const& setup)
{
    // An upper bound of what the job holds on the device, before it is coloured: the arena of
    // Updater::initialize with the largest values colouring can give (greedy colouring uses at
    // most maxc + 1 colours; each colour group is padded to 32 slots; one group may hold every
    // monomer; 64-bit bond codes), the observables arena, and the job's share of its lane's step
    // entries (a chunk of at most kMaxChunkMcs MCS, buffers grown to twice the need).
    uint32_t const n = setup.nMonomers();
    uint32_t const maxc = std::max(setup.maxNeighbours(), 1u);
    uint32_t const nC = maxc + 1;
    uint32_t const npad = std::max(n + 32u * nC, 32u);
    uint32_t const nwords = (uint32_t)(setup.latticeVolume() / 64);
    uint32_t const ntab = (setup.latticeSide(0) + setup.latticeSide(1) + setup.latticeSide(2)) / 4;
    size_t const arena = arena_layout(n, npad, maxc, nwords, ntab, nC, std::max(n, 1u), kCode64).bytes;
    size_t const obs = observables_bytes(npad, setup.countMolecules());
    size_t const steps = 2ull * sizeof(StepEntry) * kMaxChunkMcs * nC;
    return arena + obs + steps;
}

Server::Server(int gpu, size_t budgetBytes, uint32_t maxJobs) : gpu_(gpu), budget_(budgetBytes), maxJobs_(maxJobs)
{
    if (budgetBytes == 0) throw std::invalid_argument("[Server] zero memory budget");
    if (maxJobs == 0) throw std::invalid_argument("[Server] zero job slots");
    cuda_check(cudaSetDevice(gpu), "cudaSetDevice");
    // jobs allocate from the device's stream-ordered pool; keep up to the budget in the pool
    // between jobs instead of returning it to the CUDA driver at every synchronisation (this
    // process only)
    cudaMemPool_t pool;
    cuda_check(cudaDeviceGetDefaultMemPool(&pool, gpu), "cudaDeviceGetDefaultMemPool");
    uint64_t keep = budgetBytes;
    cuda_check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    t0_ = Clock::now();
    worker_ = std::thread([this] { workerMain(); });
}

Server::~Server()
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    if (worker_.joinable()) worker_.join();
}

uint64_t Server::submit(Updater const& setup, int32_t nMcs, int32_t every)
{
    if (nMcs <= 0) throw std::invalid_argument("[Server::submit] the job needs at least one MCS");
    if (every <= 0) throw std::invalid_argument("[Server::submit] the sample interval must be positive");
    setup.checkSetup();   // malformed systems fail here, on the caller's thread
    auto job = std::make_shared<Job>();
    job->nMcs = nMcs;
    job->every = every;
    job->bytes = estimateBytes(setup);
    if (job->bytes > budget_)
        throw BudgetError("[Server::submit] the job needs about " + std::to_string(job->bytes) +
                          " device bytes, more than the whole budget of " + std::to_string(budget_));
    job->u.reset(new Updater(gpu_));
    job->u->copySetup(setup);
    job->u->setBatchOnly(true);
    std::lock_guard<std::mutex> lk(mu_);
    if (dead_) throw std::runtime_error("[Server::submit] the server worker has stopped: " + deathReason_);
    if (stop_) throw std::runtime_error("[Server::submit] the server is shutting down");
    job->id = nextId_++;
    job->arrival = Clock::now();
    jobs_[job->id] = job;
    pending_.push_back(job);
    cv_.notify_all();
    return job->id;
}

int Server::status(uint64_t id)
{
    std::lock_guard<std::mutex> lk(mu_);
    return find(id)->state;
}

void Server::cancel(uint64_t id)
{
    std::lock_guard<std::mutex> lk(mu_);
    auto j = find(id);
    if (j->state == kJobPending) {
        pending_.erase(std::remove(pending_.begin(), pending_.end(), j), pending_.end());
        j->state = kJobCancelled;
        j->u.reset();
        j->finish = Clock::now();
        doneCv_.notify_all();
    } else if (j->state == kJobRunning) {
        j->cancel = true;   // the worker removes it between chunks
    }
}

bool Server::wait(uint64_t id, double timeoutS)
{
    std::unique_lock<std::mutex> lk(mu_);
    auto j = find(id);
    auto const deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeoutS));
    return doneCv_.wait_until(lk, deadline, [&] { return j->state >= kJobDone; });
}

void Server::result(uint64_t id, int32_t* xyz, uint32_t n, long long* samples, uint64_t capWords, uint32_t* nSamples,
                    double* latencyS)
{
    std::lock_guard<std::mutex> lk(mu_);
    auto j = find(id);
    if (j->state == kJobFailed) throw std::runtime_error("[Server::result] job failed: " + j->error);
    if (j->state == kJobCancelled) throw std::runtime_error("[Server::result] job was cancelled");
    if (j->state != kJobDone) throw BusyError("[Server::result] job not finished");
    if (xyz) {
        if (n != j->xyz.size() / 3) throw std::invalid_argument("[Server::result] wrong monomer count");
        std::memcpy(xyz, j->xyz.data(), j->xyz.size() * sizeof(int32_t));
    }
    if (samples) {
        if (capWords < j->samples.size()) throw std::invalid_argument("[Server::result] sample buffer too small");
        std::memcpy(samples, j->samples.data(), j->samples.size() * sizeof(long long));
    }
    if (nSamples) *nSamples = (uint32_t)(j->nMcs / j->every + (j->nMcs % j->every ? 1 : 0));
    if (latencyS) *latencyS = std::chrono::duration<double>(j->finish - j->arrival).count();
}

void Server::stats(double out[8])
{
    std::lock_guard<std::mutex> lk(mu_);
    std::vector<double> lat;
    double failed = 0, moves = 0;
    for (auto const& kv : jobs_) {
        auto const& j = kv.second;
        if (j->state == kJobDone) {
            lat.push_back(std::chrono::duration<double>(j->finish - j->arrival).count());
            moves += (double)j->nMcs * (double)(j->xyz.size() / 3);
        }
        if (j->state == kJobFailed) failed += 1;
    }
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double p) {
        if (lat.empty()) return 0.0;
        size_t const i = std::min(lat.size() - 1, (size_t)(p * (double)lat.size()));
        return lat[i];
    };
    double mean = 0;
    for (double v : lat) mean += v;
    out[0] = (double)lat.size();
    out[1] = failed;
    out[2] = moves;
    out[3] = pct(0.50);
    out[4] = pct(0.99);
    out[5] = lat.empty() ? 0.0 : mean / (double)lat.size();
    out[6] = (double)residentBytes_;
    out[7] = std::chrono::duration<double>(Clock::now() - t0_).count();
}

void Server::jobTimes(uint64_t id, double out[3])
{
    std::lock_guard<std::mutex> lk(mu_);
    auto j = find(id);
    auto since = [&](Clock::time_point t) { return std::chrono::duration<double>(t - t0_).count(); };
    out[0] = since(j->arrival);
    out[1] = j->state == kJobPending || j->start == Clock::time_point{} ? -1.0 : since(j->start);
    out[2] = j->state >= kJobDone ? since(j->finish) : -1.0;
}

uint64_t Server::sampleWords(uint64_t id)
{
    std::lock_guard<std::mutex> lk(mu_);
    auto j = find(id);
    if (j->state == kJobFailed) throw std::runtime_error("[Server::sampleWords] job failed: " + j->error);
    if (j->state == kJobCancelled) throw std::runtime_error("[Server::sampleWords] job was cancelled");
    if (j->state != kJobDone) throw BusyError("[Server::sampleWords] job not finished");
    return j->samples.size();
}

void Server::injectFault(int kind)
{
    std::lock_guard<std::mutex> lk(mu_);
    fault_ = kind;
    cv_.notify_all();
}

bool Server::dead()
{
    std::lock_guard<std::mutex> lk(mu_);
    return dead_;
}

std::shared_ptr<Server::Job> Server::find(uint64_t id)
{
    auto it = jobs_.find(id);
    if (it == jobs_.end()) throw std::out_of_range("[Server] unknown job id");
    return it->second;
}

// ------------------------------------------------------------------------------------ worker

namespace {

// the resident lane of a freshly initialised system that fits one CTA, or -1
int resident_lane_of(Updater const& u)
{
    if (!u.residentEligible()) return -1;
    int c = 0;
    while ((kResidentBlock << c) < u.maxGroup()) ++c;
    return c;
}

}  // namespace

struct Server::Lane {
    std::vector<std::shared_ptr<Job>> jobs;       // members of the batch, in batch order
    std::vector<std::shared_ptr<Job>> incoming;   // initialised, join at the next chunk
    std::unique_ptr<Batch> batch;
    std::vector<int32_t> mcs;                     // MCS of each member in the chunk in flight
    bool changed = false, inFlight = false;
    cudaEvent_t done = nullptr;
    ~Lane()
    {
        batch.reset();   // waits for its own streams
        if (done) cudaEventDestroy(done);
    }
};

void Server::workerMain()
{
    try {
        cuda_check(cudaSetDevice(gpu_), "cudaSetDevice");
        std::map<int, Lane> lanes;
        long long* stage = nullptr;   // pinned staging of one chunk's observable samples
        size_t stageWords = 0;
        struct StageFree {
            long long*& p;
            ~StageFree() { cudaFreeHost(p); }
        } stageFree{stage};

        auto running = [&]() {
            size_t n = 0;
            for (auto const& kv : lanes) n += kv.second.jobs.size() + kv.second.incoming.size();
            return n;
        };
        auto checkFault = [&]() {
            std::lock_guard<std::mutex> lk(mu_);
            if (fault_ == 1) throw std::runtime_error("injected worker fault");
            return stop_;
        };

        // Systems that fit one CTA go to the resident lane of their size class. The others go to
        // the grid lane with the least work left (monomers x remaining MCS): each grid lane is
        // bound by the latency of its launches, so spreading long jobs over several lanes that run
        // concurrently keeps each near its own speed.
        auto lane_for = [&](Job const& j) {
            int const r = resident_lane_of(*j.u);
            if (r >= 0) return r;
            int best = kGridLane;
            double bestLoad = -1.0;
            for (int k = 0; k < kGridLanes; ++k) {
                double load = 0.0;
                auto it = lanes.find(kGridLane + k);
                if (it != lanes.end()) {
                    for (auto const& q : it->second.jobs) load += (double)q->u->nMonomers() * (q->nMcs - q->done);
                    for (auto const& q : it->second.incoming) load += (double)q->u->nMonomers() * (q->nMcs - q->done);
                }
                if (bestLoad < 0.0 || load < bestLoad) {
                    bestLoad = load;
                    best = kGridLane + k;
                }
            }
            return best;
        };

        // take pending jobs in arrival order while they fit; set them up outside the lock
        auto admit = [&]() {
            bool any = false;
            for (;;) {
                std::shared_ptr<Job> j;
                {
                    std::lock_guard<std::mutex> lk(mu_);
                    if (pending_.empty() || running() >= maxJobs_) return any;
                    auto const& head = pending_.front();
                    if (residentBytes_ + head->bytes > budget_) return any;
                    j = head;
                    pending_.pop_front();
                    residentBytes_ += j->bytes;
                    j->state = kJobRunning;
                    j->start = Clock::now();
                }
                try {
                    j->u->initialize();
                    lanes[lane_for(*j)].incoming.push_back(j);
                    any = true;
                } catch (std::exception const& e) {
                    std::lock_guard<std::mutex> lk(mu_);
                    j->state = kJobFailed;
                    j->error = e.what();
                    j->finish = Clock::now();
                    residentBytes_ -= j->bytes;
                    j->u.reset();
                    doneCv_.notify_all();
                }
            }
        };

        auto launch = [&](Lane& L) {
            if (!L.incoming.empty()) {
                L.jobs.insert(L.jobs.end(), L.incoming.begin(), L.incoming.end());
                L.incoming.clear();
                L.changed = true;
            }
            if (L.jobs.empty()) return;
            if (L.changed || !L.batch) {
                std::vector<Updater*> members;
                for (auto const& j : L.jobs) members.push_back(j->u.get());
                if (L.batch) L.batch->setMembers(members.data(), (uint32_t)members.size());
                else L.batch.reset(new Batch(gpu_, members.data(), (uint32_t)members.size()));
                L.changed = false;
            }
            if (!L.done) cuda_check(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming), "cudaEventCreate");
            int32_t chunk = kMaxChunkMcs;
            for (auto const& j : L.jobs) chunk = std::min(chunk, j->every - j->done % j->every);
            L.mcs.resize(L.jobs.size());
            for (size_t i = 0; i < L.jobs.size(); ++i) L.mcs[i] = std::min(chunk, L.jobs[i]->nMcs - L.jobs[i]->done);
            L.batch->run(L.mcs.data());
            cuda_check(cudaEventRecord(L.done, L.batch->stream()), "event");
            L.inFlight = true;
        };

        auto complete = [&](Lane& L) {
            L.inFlight = false;
            // observable samples: all computed and copied back before one wait per sampling job
            std::vector<size_t> at(L.jobs.size(), SIZE_MAX);
            size_t words = 0;
            for (size_t i = 0; i < L.jobs.size(); ++i) {
                auto const& j = L.jobs[i];
                j->done += L.mcs[i];
                if (L.mcs[i] > 0 && (j->done % j->every == 0 || j->done == j->nMcs)) {
                    at[i] = words;
                    words += obs_words(j->u->nMolecules());
                }
            }
            if (words > stageWords) {
                cudaFreeHost(stage);
                stage = nullptr;
                stageWords = 0;
                cuda_check(cudaMallocHost(&stage, sizeof(long long) * words * 2), "cudaMallocHost(samples)");
                stageWords = words * 2;
            }
            for (size_t i = 0; i < L.jobs.size(); ++i)
                if (at[i] != SIZE_MAX) L.jobs[i]->u->observablesAsync(stage + at[i]);
            for (size_t i = 0; i < L.jobs.size(); ++i)
                if (at[i] != SIZE_MAX) {
                    auto const& j = L.jobs[i];
                    j->u->synchronize();
                    size_t const w = obs_words(j->u->nMolecules());
                    j->samples.insert(j->samples.end(), stage + at[i], stage + at[i] + w);
                }
            std::vector<std::shared_ptr<Job>> keep;
            for (auto const& j : L.jobs) {
                bool cancelled;
                {
                    std::lock_guard<std::mutex> lk(mu_);
                    cancelled = j->cancel;
                }
                if (j->done == j->nMcs || cancelled) {
                    std::vector<int32_t> xyz;
                    if (!cancelled) {
                        xyz.resize(3ull * j->u->nMonomers());
                        j->u->getCoordinates(xyz.data(), j->u->nMonomers());
                    }
                    L.changed = true;   // the batch gets its new member list before its next run
                    std::unique_ptr<Updater> gone;
                    {
                        std::lock_guard<std::mutex> lk(mu_);
                        j->xyz.swap(xyz);
                        j->state = cancelled ? kJobCancelled : kJobDone;
                        j->finish = Clock::now();
                        residentBytes_ -= j->bytes;
                        gone.swap(j->u);
                        doneCv_.notify_all();
                    }
                    gone.reset();   // frees the job's device memory in stream order, outside the lock
                } else {
                    keep.push_back(j);
                }
            }
            L.jobs.swap(keep);
        };

        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                if (fault_ == 1) throw std::runtime_error("injected worker fault");
                if (stop_) break;
                if (running() == 0 && pending_.empty()) cv_.wait_for(lk, std::chrono::milliseconds(5));
                if (stop_) break;
            }
            admit();
            for (auto& kv : lanes)
                if (!kv.second.inFlight) launch(kv.second);
            // service the first lane that finishes; set arrivals up meanwhile
            for (;;) {
                bool progressed = false, busy = false;
                for (auto& kv : lanes) {
                    Lane& L = kv.second;
                    if (!L.inFlight) continue;
                    cudaError_t const q = cudaEventQuery(L.done);
                    if (q == cudaSuccess) {
                        complete(L);
                        progressed = true;
                    } else if (q == cudaErrorNotReady) {
                        busy = true;
                    } else {
                        cuda_check(q, "lane");
                    }
                }
                if (progressed || !busy) break;
                if (checkFault()) break;
                if (admit()) break;   // an idle lane may take the new job now
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
        }
        for (auto& kv : lanes) {
            kv.second.batch.reset();
            for (auto const& j : kv.second.jobs) j->u.reset();
            for (auto const& j : kv.second.incoming) j->u.reset();
        }
    } catch (std::exception const& e) {
        std::lock_guard<std::mutex> lk(mu_);
        dead_ = true;
        deathReason_ = e.what();
        for (auto& kv : jobs_)
            if (kv.second->state < kJobDone) {
                kv.second->state = kJobFailed;
                kv.second->error = std::string("server worker stopped: ") + e.what();
                kv.second->finish = Clock::now();
            }
        pending_.clear();
        doneCv_.notify_all();
    }
}

}  // namespace bfm
