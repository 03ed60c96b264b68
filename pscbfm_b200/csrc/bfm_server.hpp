// Server for "run this system for M MCS, sample observables every k" jobs (bfm_server.cpp).
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>

namespace bfm {

class Updater;

struct BudgetError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct BusyError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

enum JobState : int { kJobPending = 0, kJobRunning = 1, kJobDone = 2, kJobCancelled = 3, kJobFailed = 4 };

class Server {
public:
    Server(int gpu, size_t budgetBytes, uint32_t maxJobs);
    ~Server();
    Server(Server const&) = delete;
    Server& operator=(Server const&) = delete;

    uint64_t submit(Updater const& setup, int32_t nMcs, int32_t every);
    int status(uint64_t id);
    void cancel(uint64_t id);
    bool wait(uint64_t id, double timeoutS);   // true when the job reached a final state
    void result(uint64_t id, int32_t* xyz, uint32_t n, long long* samples, uint64_t capWords, uint32_t* nSamples,
                double* latencyS);
    // completed, failed, attempted moves of completed jobs, p50 s, p99 s, mean s, resident bytes, elapsed s
    void stats(double out[8]);
    void jobTimes(uint64_t id, double out[3]);
    uint64_t sampleWords(uint64_t id);            // int64 words of a finished job's samples   // arrival, admission, completion (s since create; -1: not yet)
    void injectFault(int kind);                // 1: the worker thread throws at its next loop
    bool dead();
    static size_t estimateBytes(Updater const& setup);

private:
    struct Job;
    struct Lane;
    std::shared_ptr<Job> find(uint64_t id);
    void workerMain();

    int gpu_;
    size_t budget_;
    uint32_t maxJobs_;
    std::mutex mu_;
    std::condition_variable cv_, doneCv_;
    std::map<uint64_t, std::shared_ptr<Job>> jobs_;
    std::deque<std::shared_ptr<Job>> pending_;
    size_t residentBytes_ = 0;
    uint64_t nextId_ = 1;
    bool stop_ = false, dead_ = false;
    int fault_ = 0;
    std::string deathReason_;
    std::chrono::steady_clock::time_point t0_;
    std::thread worker_;
};

}  // namespace bfm
