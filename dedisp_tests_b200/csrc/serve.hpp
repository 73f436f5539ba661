// Streaming dedispersion server (no counterpart in the reference, whose
// plans process one complete series per call).
//
// Beams deliver their samples in gulps of any length. For each beam the
// server keeps, in device memory, the last max_delay input rows (the overlap
// tail), so a gulp of n rows yields exactly n output samples per DM: the
// dedispersion of tail + gulp (the tail starts as max_delay zero rows, as if
// the beam had been silent before). Gulps of one beam are processed in
// submission order; gulps of different beams run concurrently on a pool of
// workers. Each worker is one host thread with its own CUDA stream and its
// own plan (a TDD plan, or an FDD plan with segmented time-series output), so
// every beam of a kind shares the workers of that kind. All device memory
// (tails, worker plans at the largest gulp, worker output buffers) is
// allocated by start(), which fails if it exceeds the HBM budget; submit()
// then never allocates, and a gulp waits in the queue until a worker of its
// kind is free (admission by budget: the in-flight gulps are bounded by the
// workers whose memory fits). Each gulp's submit-to-completion latency
// (host clock) and device time (CUDA events) are recorded.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace dedisp {
namespace detail {

struct ServeConfig {
    size_t nchans = 0;
    float dt = 0.f, f0 = 0.f, df = 0.f;
    int in_nbits = 8;
    int device = 0;
    size_t hbm_budget = 0;     // bytes of device memory the server may hold
    size_t max_gulp = 0;       // largest gulp (samples)
    size_t fdd_max_gulp = 0;   // largest gulp of an FDD beam (0: max_gulp)
    int tdd_workers = 1;
    int fdd_workers = 0;
    int fdd_precision = 1;     // 0 FP32 CUDA-core MAC, 1 3xBF16 tensor-core MAC
    size_t fdd_segment = 0;    // FDD segment FFT length (0: the plan's rule)
};

struct GulpRecord {
    int beam = -1;
    size_t nsamps = 0;
    double t_submit = 0, t_start = 0, t_done = 0;  // seconds (steady clock)
    float device_ms = 0.f;
    int worker = -1;
};

class StreamServer {
public:
    explicit StreamServer(const ServeConfig& cfg);
    ~StreamServer();

    // kind 0: TDD, 1: FDD. Before start().
    int add_beam(const float* dms, size_t ndm, int kind);
    size_t max_delay(int beam) const;
    size_t dm_count(int beam) const;

    // Allocates everything (runs one warm-up gulp per worker); returns the
    // device bytes held. Throws DEDISP_MEM_ALLOC_FAILED above the budget.
    size_t start();

    // Queues the next n rows (host, time-major packed) of `beam`. `d_out`:
    // device buffer for dm_count x n floats (row stride n), or nullptr to use
    // the worker's own buffer (overwritten by that worker's next gulp). The
    // host rows must stay valid until the gulp completes.
    long submit(int beam, const uint8_t* rows, size_t n, float* d_out);
    bool done(long ticket);
    void wait(long ticket);
    void drain();

    std::vector<GulpRecord> records() const;
    size_t bytes_held() const { return m_bytes; }

private:
    struct Beam;
    struct Worker;
    struct Job {
        long ticket;
        int beam;
        const uint8_t* rows;
        size_t n;
        float* d_out;
        double t_submit;
    };
    void worker_loop(Worker* w);
    void run_job(Worker* w, const Job& j, GulpRecord& rec);

    ServeConfig m_cfg;
    size_t m_row_bytes = 0;
    std::vector<float> m_delays;
    std::vector<std::unique_ptr<Beam>> m_beams;
    std::vector<std::unique_ptr<Worker>> m_workers;
    bool m_started = false;
    bool m_stop = false;
    size_t m_bytes = 0;

    mutable std::mutex m_mu;
    std::condition_variable m_cv_work, m_cv_done;
    std::deque<Job> m_queue;
    std::vector<GulpRecord> m_records;  // by ticket
    std::vector<char> m_done;
    std::string m_error;
};

}  // namespace detail
}  // namespace dedisp
