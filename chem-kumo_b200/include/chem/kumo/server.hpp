#pragma once
// Serving loop of the B200 grid evaluator (new; chem-kumo has no serving
// counterpart).  Requests of different molecules and sizes are queued,
// admitted in arrival order while their device-memory footprint fits an HBM
// budget and an active slot is free, and run concurrently, each on its own
// CUDA stream, so that their kernels overlap on the device while later
// requests arrive (continuous batching); one host thread per active slot
// issues its request's launches.  Small requests (up to
// ServerOptions::graph_points points, grids converted to explicit points) whose
// shape (molecule, options, properties, point bucket) has been met before are
// replayed from a CUDA graph captured at the second meeting; the others run
// the regular device path.  Results land in
// the caller's host arrays; latency is measured from submit to the moment the
// results are in those arrays.
#include <chrono>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <string>
#include <thread>
#include <vector>

#include "chem/kumo/evaluator.hpp"

namespace chem::kumo {

struct ServerOptions {
    int device = 0;
    /// Device memory the active requests may hold together (molecule copies,
    /// scratch, inputs and outputs); 0 = 150 GB capped at 90% of free memory.
    std::size_t hbm_budget = 0;
    int max_active = 8;                      ///< requests in flight (one launcher thread and stream pair each)
    std::size_t graph_points = 65536;        ///< largest request replayed from a CUDA graph
    std::size_t request_scratch = 1ull << 30;  ///< AO scratch per request (sets its wave size)
    /// Page-locked host arena for staging results and points, allocated once
    /// at start (0: none, every staging buffer page-locked on demand).
    std::size_t staging_bytes = 2ull << 30;
};

struct ServeRequest {
    const Molecule* molecule = nullptr;  ///< must outlive the request
    EvaluationOptions options;
    Request request;
    std::optional<Grid> grid;            ///< a grid, or
    std::vector<double> points;          ///< 3 x N host points (x, y, z per point)
    std::vector<double*> outputs;        ///< per property: channels x N host doubles, caller-owned
};

struct ServeStats {
    std::size_t submitted = 0, completed = 0, failed = 0;
    std::size_t points = 0;               ///< points of the completed requests
    double p50_ms = 0, p99_ms = 0, mean_ms = 0, max_ms = 0;
    double busy_s = 0;                    ///< first submit to last completion
    double points_per_s = 0;
    std::size_t graph_captures = 0, graph_replays = 0, direct_runs = 0;
    std::size_t peak_bytes = 0;           ///< largest admitted footprint sum
    std::size_t budget_bytes = 0;
    double launch_s = 0;                  ///< host time spent issuing requests, summed over the launcher threads
    double copy_s = 0;                    ///< completion-thread time copying results
    double queue_ms = 0;                  ///< mean time from submit to admission
};

class Server {
public:
    explicit Server(ServerOptions options = {});
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    /// Queues a request (validated first, with the evaluator's exceptions);
    /// returns its ticket.  Thread-safe.
    std::uint64_t submit(ServeRequest request);
    /// Waits up to timeout_s for a ticket; true once its results are in the
    /// caller's arrays.  Rethrows the request's error as runtime_error.
    bool wait(std::uint64_t ticket, double timeout_s);
    /// Waits for every submitted request.
    void drain();
    ServeStats stats() const;
    /// Clears the latency record and counters (not the graph cache).
    void reset_stats();

    struct Impl;

private:
    std::unique_ptr<Impl> impl_;
};

}  // namespace chem::kumo
