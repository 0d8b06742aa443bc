// Serving loop (see chem/kumo/server.hpp).
//
// Threads: the caller's (submit / wait); one scheduler thread that admits
// requests; one launcher thread per active slot (ServerOptions::max_active),
// each with its own streams and event, which issues an admitted request's
// device work, waits for it and hands it on; and one completion thread that
// copies results from page-locked staging into the caller's arrays, so that
// large copies never hold up admission or launches.  Several host threads
// issue launches at once, so the host time of one request's launches (tens of
// kernels, allocations and copies for a large cube) does not hold up the
// others.
//
// Admission: FIFO; the head request starts when a slot (stream) is free and
// the footprint sum of the active requests plus the resident molecule copies
// stays within the HBM budget.  Footprint of a request: its outputs, its
// points and its AO scratch (ServerOptions::request_scratch, which also sets
// its wave size), plus the molecule's device copy when it is not resident yet
// (molecule copies then stay resident).
//
// Creating a server loads every kernel of the library on its device
// (kumo_dev::preload_kernels), so that no launcher waits while CUDA loads a
// kernel at its first launch.
//
// Graph path (requests of at most graph_points points): the points are padded
// to a power-of-two bucket (>= 128) by repeating the last point, which leaves
// the last block's bounding box and screening unchanged; one CUDA graph per
// (molecule, options, properties, bucket) holds the whole device evaluation
// between fixed device buffers, with page-locked staging on both sides; a
// replay is one H2D copy, one graph launch and one D2H copy.  Concurrent
// requests of the same key use separate graph instances.
#include "chem/kumo/server.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

#include "device_state.hpp"
#include "grid_geometry.hpp"

namespace chem::kumo {

namespace detail {
void prepare_device_for_capture();
void set_tile_probing(bool on);
}

namespace {

using clock_type = std::chrono::steady_clock;
using detail::check_cuda;

std::size_t round_bucket(std::size_t n) {
    std::size_t b = 128;
    while (b < n) b <<= 1;
    return b;
}

// Device bytes a molecule's resident copy will take (DeviceMolecule).
std::size_t molecule_bytes_estimate(const Molecule& m) {
    const std::size_t n = m.basis_size();
    const std::size_t nmo = m.orbital_count(SpinChannel::Alpha) + (m.unrestricted() ? m.orbital_count(SpinChannel::Beta) : 0);
    const std::size_t occ = m.occupied_count(SpinChannel::Alpha) + m.occupied_count(SpinChannel::Beta) + 32;
    // P_total and P_spin in FP64 and as 8-byte BF16 piece elements, all MO
    // coefficients, the occupied MOs in FP64 and as pieces, and the tables.
    return 2 * n * n * (8 + 8) + n * nmo * 8 + n * occ * (8 + 6) + (std::size_t(4) << 20);
}

// Grid points in the device's arithmetic (point_at: origin + ((s_a i + s_b j) + s_c k)).
void grid_to_points(const Grid& g, std::vector<double>& pts) {
    const std::size_t n = detail::validated_point_count(g);
    pts.resize(3 * n);
    std::size_t q = 0;
    for (std::size_t i = 0; i < g.counts[0]; ++i)
        for (std::size_t j = 0; j < g.counts[1]; ++j)
            for (std::size_t k = 0; k < g.counts[2]; ++k, ++q)
                for (int a = 0; a < 3; ++a) {
                    const double di = static_cast<double>(i), dj = static_cast<double>(j), dk = static_cast<double>(k);
                    const double t = (g.steps.m[0 + a] * di + g.steps.m[3 + a] * dj) + g.steps.m[6 + a] * dk;
                    pts[3 * q + a] = g.origin[a] + t;
                }
}

struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    double* d_points = nullptr;
    double* d_out = nullptr;
    double* h_points = nullptr;  // page-locked
    double* h_out = nullptr;     // page-locked
    bool own_host = true;        // false when both come from the server's staging arena
    std::size_t bucket = 0;
    std::size_t channels = 0;
    std::atomic<bool> busy{false};  // set by the scheduler, cleared by the completion thread
    ~GraphEntry() {
        if (exec) cudaGraphExecDestroy(exec);
        cudaFree(d_points);
        cudaFree(d_out);
        if (own_host) {
            cudaFreeHost(h_points);
            cudaFreeHost(h_out);
        }
    }
};

struct Ticket {
    bool done = false;
    std::string error;
    double latency_ms = 0;
};

}  // namespace

struct Server::Impl {
    ServerOptions opt;
    std::size_t budget = 0;

    mutable std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;

    struct Pending {
        std::uint64_t ticket;
        ServeRequest req;
        clock_type::time_point t_submit;
        std::size_t n = 0;
        std::size_t channels = 0;
        std::size_t footprint = 0;
        bool graph = false;
        // Mixed-form grid on the graph path: the grid's points in tile order
        // (detail::tile_order; n_eval of them, padding slots repeating their
        // tile's first point), so that the replay evaluates the same blocks
        // as the grid evaluated alone; tile_index maps them back.
        std::size_t n_eval = 0;
        std::vector<long long> tile_index;
    };
    struct Active {
        Pending p;
        cudaStream_t stream = nullptr;
        cudaEvent_t event = nullptr;
        GraphEntry* entry = nullptr;      // graph path
        double* stage = nullptr;          // direct path: page-locked results
        std::size_t stage_bytes = 0;
        double* pstage = nullptr;         // direct path: page-locked points
        std::size_t pstage_bytes = 0;
        std::size_t row = 0;              // row length of the staged results (bucket or n)
        bool high_priority = false;       // on the launcher's high-priority stream
    };
    std::deque<Pending> queue;    // submitted, not admitted
    std::deque<Pending> ready;    // admitted, waiting for a launcher
    std::deque<Active> finished;  // handed to the completion thread
    bool stop_launchers = false, stop_completer = false;
    std::condition_variable cv_ready;
    int inflight = 0;  // admitted and not yet handed to the completion thread
    std::unordered_map<std::uint64_t, Ticket> tickets;
    std::uint64_t next_ticket = 1;

    // Streams of small requests (at most graph_points points) take the
    // device's highest priority, those of larger requests its lowest: a
    // small request's blocks are scheduled as soon as SMs free up, instead of
    // after every queued block of a large cube.  Each launcher owns one of each.
    int prio_low = 0, prio_high = 0;
    std::mutex gmu;  // graphs, seen
    std::map<std::string, std::vector<std::unique_ptr<GraphEntry>>> graphs;
    std::map<std::string, int> seen;  // small-request keys met so far (a graph is captured on the second)
    std::mutex smu;  // free_stage, arena_used
    std::multimap<std::size_t, double*> free_stage;  // page-locked staging by size
    // Page-locked arena, allocated once at start: staging buffers are carved
    // from it (page-locking on demand synchronises the device and stalls the
    // scheduler while the GPU is busy); beyond it, cudaHostAlloc.
    char* arena = nullptr;
    std::size_t arena_size = 0, arena_used = 0;
    double* pinned(std::size_t cls, bool& from_arena) {
        if (arena && arena_used + cls <= arena_size) {
            double* p = reinterpret_cast<double*>(arena + arena_used);
            arena_used += cls;
            from_arena = true;
            return p;
        }
        void* p = nullptr;
        check_cuda(cudaHostAlloc(&p, cls, cudaHostAllocDefault), "cudaHostAlloc (staging)");
        from_arena = false;
        return static_cast<double*>(p);
    }
    bool in_arena(const void* p) const {
        const char* c = static_cast<const char*>(p);
        return arena && c >= arena && c < arena + arena_size;
    }
    std::vector<const Molecule*> resident;  // guarded by mu
    std::size_t resident_bytes = 0, active_bytes = 0;

    // Statistics (guarded by mu).
    std::vector<double> latencies;
    ServeStats st;
    double queue_sum_ms = 0;
    std::size_t admitted = 0;
    std::optional<clock_type::time_point> t_first, t_last;

    std::thread scheduler, completer;
    std::vector<std::thread> launchers;

    struct Lanes {  // one launcher's streams and completion event
        cudaStream_t lo = nullptr, hi = nullptr;
        cudaEvent_t event = nullptr;
    };
    void run_scheduler();
    void run_launcher();
    void run_completer();
    // Issues p's device work on one of the lanes' streams and records the
    // lanes' event after it; false (the ticket failed) if issuing threw.
    bool launch(Pending& p, const Lanes& lanes, Active& a);
    GraphEntry* graph_for(const Pending& p, cudaStream_t stream);
    double* get_stage(std::size_t bytes);
    void put_stage(std::size_t bytes, double* p);
    std::string key_of(const Pending& p) const;
    void fail(std::uint64_t ticket, const std::string& what, clock_type::time_point t0);
};

std::string Server::Impl::key_of(const Pending& p) const {
    std::ostringstream k;
    const auto& o = p.req.options;
    k << static_cast<const void*>(p.req.molecule) << '|' << static_cast<int>(o.precision) << '|'
      << static_cast<int>(o.backend) << '|' << o.screening_threshold << '|' << o.block_size << '|'
      << o.potential_tolerance << '|' << round_bucket(p.n_eval);
    for (const auto& q : p.req.request.properties())
        k << '|' << static_cast<int>(q.kind) << ',' << static_cast<int>(q.component) << ','
          << static_cast<int>(q.channel) << ',' << q.orbital_index;
    return k.str();
}

// Page-locked staging in power-of-two size classes (page-locking is slow and
// synchronises the device, so buffers are kept and reused).
std::size_t stage_class(std::size_t bytes) {
    std::size_t c = 4096;
    while (c < bytes) c <<= 1;
    return c;
}

void Server::Impl::put_stage(std::size_t bytes, double* p) {
    std::lock_guard<std::mutex> lock(smu);
    free_stage.emplace(stage_class(bytes), p);
}

double* Server::Impl::get_stage(std::size_t bytes) {
    const std::size_t cls = stage_class(bytes);
    std::lock_guard<std::mutex> lock(smu);
    auto it = free_stage.find(cls);
    if (it != free_stage.end()) {
        double* p = it->second;
        free_stage.erase(it);
        return p;
    }
    bool from_arena = false;
    return pinned(cls, from_arena);
}

GraphEntry* Server::Impl::graph_for(const Pending& p, cudaStream_t stream) {
    const std::string key = key_of(p);
    {
        std::lock_guard<std::mutex> glock(gmu);
        for (auto& e : graphs[key]) {
            bool idle = false;
            if (e->busy.compare_exchange_strong(idle, true)) {
                std::lock_guard<std::mutex> lock(mu);
                ++st.graph_replays;
                return e.get();
            }
        }
    }
    auto e = std::make_unique<GraphEntry>();
    e->bucket = round_bucket(p.n_eval);
    e->channels = p.channels;
    check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&e->d_points), sizeof(double) * 3 * e->bucket, stream),
               "cudaMallocAsync (serving points)");
    check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&e->d_out),
                               sizeof(double) * std::max<std::size_t>(e->channels * e->bucket, 1), stream),
               "cudaMallocAsync (serving outputs)");
    {
        const std::size_t pb = stage_class(sizeof(double) * 3 * e->bucket);
        const std::size_t ob = stage_class(sizeof(double) * std::max<std::size_t>(e->channels * e->bucket, 1));
        std::unique_lock<std::mutex> slock(smu);
        if (arena && arena_used + pb + ob <= arena_size) {
            bool unused = false;
            e->h_points = pinned(pb, unused);
            e->h_out = pinned(ob, unused);
            e->own_host = false;
        } else {
            slock.unlock();
            check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&e->h_points), pb, cudaHostAllocDefault),
                       "cudaHostAlloc (serving points)");
            check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&e->h_out), ob, cudaHostAllocDefault),
                       "cudaHostAlloc (serving outputs)");
        }
    }
    std::vector<double*> outs;
    std::size_t off = 0;
    for (const auto& q : p.req.request.properties()) {
        outs.push_back(e->d_out + off * e->bucket);
        off += property_channels(q.kind);
    }
    EvaluationOptions o = p.req.options;
    o.scratch_bytes = opt.request_scratch;
    o.progress = {};
    const Evaluator ev(*p.req.molecule, o);
    cudaGraph_t graph = nullptr;
    check_cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
    try {
        ev.evaluate_device(Points{e->d_points, e->bucket}, p.req.request, outs.data(), stream);
    } catch (...) {
        cudaStreamEndCapture(stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    check_cuda(cudaStreamEndCapture(stream, &graph), "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&e->exec, graph, 0);
    cudaGraphDestroy(graph);
    check_cuda(ie, "cudaGraphInstantiate");
    e->busy = true;
    {
        std::lock_guard<std::mutex> lock(mu);
        ++st.graph_captures;
    }
    GraphEntry* got = e.get();
    std::lock_guard<std::mutex> glock(gmu);
    graphs[key].push_back(std::move(e));
    return got;
}

void Server::Impl::fail(std::uint64_t ticket, const std::string& what, clock_type::time_point t0) {
    std::lock_guard<std::mutex> lock(mu);
    auto& t = tickets[ticket];
    t.done = true;
    t.error = what;
    t.latency_ms = std::chrono::duration<double, std::milli>(clock_type::now() - t0).count();
    ++st.failed;
    cv_done.notify_all();
}

bool Server::Impl::launch(Pending& p, const Lanes& lanes, Active& a) {
    const bool small = p.n_eval <= opt.graph_points;
    a.stream = small ? lanes.hi : lanes.lo;
    a.high_priority = small;
    a.event = lanes.event;
    const Molecule& mol = *p.req.molecule;
    const auto& props = p.req.request.properties();
    try {
        if (!mol.device_if_resident()) {
            (void)mol.device();
            std::lock_guard<std::mutex> lock(mu);
            if (std::find(resident.begin(), resident.end(), &mol) == resident.end()) {
                resident.push_back(&mol);
                resident_bytes += mol.device_bytes();
            }
        }
        if (p.graph) {
            // A request shape met for the first time runs the regular path;
            // its graph is captured when the shape comes again.
            const std::string key = key_of(p);
            std::lock_guard<std::mutex> glock(gmu);
            if (seen[key]++ == 0 && graphs.find(key) == graphs.end()) p.graph = false;
        }
        if (p.graph) {
            if (p.req.grid) {
                grid_to_points(*p.req.grid, p.req.points);
                if (!p.tile_index.empty()) {
                    // Tile order; a padding slot repeats its tile's first point.
                    std::vector<double> tiled(3 * p.n_eval);
                    for (std::size_t q = 0; q < p.n_eval; ++q) {
                        const long long g = p.tile_index[q] >= 0 ? p.tile_index[q] : p.tile_index[q & ~std::size_t(127)];
                        std::memcpy(&tiled[3 * q], &p.req.points[3 * static_cast<std::size_t>(g)], 3 * sizeof(double));
                    }
                    p.req.points.swap(tiled);
                }
            }
            GraphEntry* e = graph_for(p, a.stream);
            a.entry = e;
            const std::size_t n = p.n_eval, b = e->bucket;
            std::memcpy(e->h_points, p.req.points.data(), sizeof(double) * 3 * n);
            for (std::size_t q = n; q < b; ++q) std::memcpy(e->h_points + 3 * q, e->h_points + 3 * (n - 1), 3 * sizeof(double));
            check_cuda(cudaMemcpyAsync(e->d_points, e->h_points, sizeof(double) * 3 * b, cudaMemcpyHostToDevice, a.stream),
                       "cudaMemcpyAsync (serving points)");
            check_cuda(cudaGraphLaunch(e->exec, a.stream), "cudaGraphLaunch");
            check_cuda(cudaMemcpyAsync(e->h_out, e->d_out, sizeof(double) * e->channels * b, cudaMemcpyDeviceToHost,
                                       a.stream),
                       "cudaMemcpyAsync (serving results)");
            a.row = b;
        } else {
            EvaluationOptions o = p.req.options;
            o.scratch_bytes = opt.request_scratch;
            o.progress = {};
            const Evaluator ev(mol, o);
            const std::size_t n = p.n;
            a.stage_bytes = sizeof(double) * std::max<std::size_t>(p.channels * n, 1);
            a.stage = get_stage(a.stage_bytes);
            double* d_out = nullptr;
            check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&d_out), a.stage_bytes, a.stream), "cudaMallocAsync (outputs)");
            std::vector<double*> outs;
            std::size_t off = 0;
            for (const auto& q : props) {
                outs.push_back(d_out + off * n);
                off += property_channels(q.kind);
            }
            double* d_pts = nullptr;
            if (p.req.grid) {
                ev.evaluate_device(*p.req.grid, p.req.request, outs.data(), a.stream);
            } else {
                check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&d_pts), sizeof(double) * 3 * n, a.stream),
                           "cudaMallocAsync (points)");
                // Points go up from page-locked staging, held until the request completes.
                a.pstage_bytes = sizeof(double) * 3 * n;
                a.pstage = get_stage(a.pstage_bytes);
                std::memcpy(a.pstage, p.req.points.data(), a.pstage_bytes);
                check_cuda(cudaMemcpyAsync(d_pts, a.pstage, a.pstage_bytes, cudaMemcpyHostToDevice, a.stream),
                           "cudaMemcpyAsync (points)");
                ev.evaluate_device(Points{d_pts, n}, p.req.request, outs.data(), a.stream);
            }
            check_cuda(cudaMemcpyAsync(a.stage, d_out, a.stage_bytes, cudaMemcpyDeviceToHost, a.stream),
                       "cudaMemcpyAsync (results)");
            cudaFreeAsync(d_out, a.stream);
            if (d_pts) cudaFreeAsync(d_pts, a.stream);
            a.row = n;
            std::lock_guard<std::mutex> lock(mu);
            ++st.direct_runs;
        }
        check_cuda(cudaEventRecord(a.event, a.stream), "cudaEventRecord");
    } catch (const std::exception& ex) {
        // Work already queued on the stream may still read the staging: let it finish.
        cudaStreamSynchronize(a.stream);
        cudaGetLastError();
        if (a.entry) a.entry->busy = false;
        if (a.stage) put_stage(a.stage_bytes, a.stage);
        if (a.pstage) put_stage(a.pstage_bytes, a.pstage);
        a.entry = nullptr;
        a.stage = a.pstage = nullptr;
        fail(p.ticket, ex.what(), p.t_submit);
        return false;
    }
    return true;
}

void Server::Impl::run_scheduler() {
    check_cuda(cudaSetDevice(opt.device), "cudaSetDevice");  // device_if_resident compares devices
    std::unique_lock<std::mutex> lock(mu);
    for (;;) {
        // Admission, in arrival order: the head request starts when a slot is
        // free and its footprint fits the budget beside the active requests.
        while (!queue.empty() && inflight < opt.max_active) {
            Pending& head = queue.front();
            const bool resident_now = head.req.molecule->device_if_resident() != nullptr;
            const std::size_t need = head.footprint + (resident_now ? 0 : molecule_bytes_estimate(*head.req.molecule));
            if (inflight > 0 && resident_bytes + active_bytes + need > budget) break;
            Pending p = std::move(head);
            queue.pop_front();
            active_bytes += p.footprint;
            ++inflight;
            queue_sum_ms += std::chrono::duration<double, std::milli>(clock_type::now() - p.t_submit).count();
            ++admitted;
            st.peak_bytes = std::max(st.peak_bytes, resident_bytes + active_bytes);
            ready.push_back(std::move(p));
            cv_ready.notify_one();
        }
        if (stop && queue.empty() && inflight == 0) break;
        // Woken by submit and by every completion.
        cv_work.wait(lock);
    }
}

void Server::Impl::run_launcher() {
    check_cuda(cudaSetDevice(opt.device), "cudaSetDevice");
    // No synchronous tile-shape probes on the serving threads (they would
    // hold up launches); grids take a shape already measured, or the default.
    detail::set_tile_probing(false);
    Lanes lanes;
    check_cuda(cudaStreamCreateWithPriority(&lanes.lo, cudaStreamNonBlocking, prio_low), "cudaStreamCreateWithPriority");
    check_cuda(cudaStreamCreateWithPriority(&lanes.hi, cudaStreamNonBlocking, prio_high), "cudaStreamCreateWithPriority");
    // Blocking synchronisation: a launcher waiting for its request sleeps.
    check_cuda(cudaEventCreateWithFlags(&lanes.event, cudaEventDisableTiming | cudaEventBlockingSync), "cudaEventCreate");
    for (;;) {
        Pending p;
        {
            std::unique_lock<std::mutex> lock(mu);
            cv_ready.wait(lock, [&] { return stop_launchers || !ready.empty(); });
            if (ready.empty()) break;
            p = std::move(ready.front());
            ready.pop_front();
        }
        const auto tl = clock_type::now();
        Active a;
        const bool ok = launch(p, lanes, a);
        const double dt = std::chrono::duration<double>(clock_type::now() - tl).count();
        cudaError_t q = cudaSuccess;
        if (ok) {
            q = cudaEventSynchronize(a.event);
            if (a.pstage) {
                put_stage(a.pstage_bytes, a.pstage);
                a.pstage = nullptr;
            }
            if (q != cudaSuccess) {
                cudaGetLastError();
                if (a.entry) a.entry->busy = false;
                if (a.stage) put_stage(a.stage_bytes, a.stage);
                fail(p.ticket, std::string("CUDA error: ") + cudaGetErrorString(q), p.t_submit);
            }
        }
        std::lock_guard<std::mutex> lock(mu);
        st.launch_s += dt;
        active_bytes -= p.footprint;
        --inflight;
        if (ok && q == cudaSuccess) {
            a.p = std::move(p);
            finished.push_back(std::move(a));
        }
        cv_work.notify_all();
    }
    cudaStreamSynchronize(lanes.lo);
    cudaStreamSynchronize(lanes.hi);
    cudaStreamDestroy(lanes.lo);
    cudaStreamDestroy(lanes.hi);
    cudaEventDestroy(lanes.event);
}

void Server::Impl::run_completer() {
    check_cuda(cudaSetDevice(opt.device), "cudaSetDevice");
    for (;;) {
        Active a;
        {
            std::unique_lock<std::mutex> lock(mu);
            cv_work.wait(lock, [&] { return stop_completer || !finished.empty(); });
            if (finished.empty()) return;
            a = std::move(finished.front());
            finished.pop_front();
        }
        const auto tc = clock_type::now();
        const double* src = a.entry ? a.entry->h_out : a.stage;
        const auto& props = a.p.req.request.properties();
        const bool tiled = a.entry && !a.p.tile_index.empty();
        std::size_t off = 0;
        for (std::size_t i = 0; i < props.size(); ++i) {
            const std::size_t ch = property_channels(props[i].kind);
            for (std::size_t c = 0; c < ch; ++c) {
                double* dst = a.p.req.outputs[i] + c * a.p.n;
                const double* row = src + (off + c) * a.row;
                if (tiled) {
                    for (std::size_t q = 0; q < a.p.n_eval; ++q)
                        if (a.p.tile_index[q] >= 0) dst[a.p.tile_index[q]] = row[q];
                } else {
                    std::memcpy(dst, row, sizeof(double) * a.p.n);
                }
            }
            off += ch;
        }
        const auto now = clock_type::now();
        if (a.entry) a.entry->busy = false;
        if (a.stage) put_stage(a.stage_bytes, a.stage);
        std::lock_guard<std::mutex> lock(mu);
        st.copy_s += std::chrono::duration<double>(now - tc).count();
        auto& t = tickets[a.p.ticket];
        t.done = true;
        t.latency_ms = std::chrono::duration<double, std::milli>(now - a.p.t_submit).count();
        latencies.push_back(t.latency_ms);
        ++st.completed;
        st.points += a.p.n;
        t_last = now;
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

}  // namespace chem::kumo

namespace chem::kumo {

Server::Server(ServerOptions options) : impl_(std::make_unique<Impl>()) {
    Impl& m = *impl_;
    m.opt = options;
    if (m.opt.max_active < 1) throw std::invalid_argument("max_active must be at least 1");
    check_cuda(cudaSetDevice(m.opt.device), "cudaSetDevice");
    std::size_t free_b = 0, total_b = 0;
    check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const std::size_t cap = static_cast<std::size_t>(0.9 * static_cast<double>(free_b));
    m.budget = m.opt.hbm_budget ? std::min(m.opt.hbm_budget, cap) : std::min<std::size_t>(150ull * 1000 * 1000 * 1000, cap);
    m.st.budget_bytes = m.budget;
    if (m.opt.staging_bytes) {
        check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&m.arena), m.opt.staging_bytes, cudaHostAllocDefault),
                   "cudaHostAlloc (staging arena)");
        m.arena_size = m.opt.staging_bytes;
    }
    check_cuda(cudaDeviceGetStreamPriorityRange(&m.prio_low, &m.prio_high), "cudaDeviceGetStreamPriorityRange");
    detail::prepare_device_for_capture();
    for (int i = 0; i < m.opt.max_active; ++i)
        m.launchers.emplace_back([&m] {
            try {
                m.run_launcher();
            } catch (const std::exception& e) {
                // This launcher cannot issue work: fail what it would take.
                std::unique_lock<std::mutex> lock(m.mu);
                for (;;) {
                    m.cv_ready.wait(lock, [&] { return m.stop_launchers || !m.ready.empty(); });
                    if (m.ready.empty()) return;
                    Impl::Pending p = std::move(m.ready.front());
                    m.ready.pop_front();
                    auto& t = m.tickets[p.ticket];
                    t.done = true;
                    t.error = std::string("serving launcher stopped: ") + e.what();
                    ++m.st.failed;
                    m.active_bytes -= p.footprint;
                    --m.inflight;
                    m.cv_done.notify_all();
                    m.cv_work.notify_all();
                }
            }
        });
    m.scheduler = std::thread([&m] {
        try {
            m.run_scheduler();
        } catch (const std::exception& e) {
            std::lock_guard<std::mutex> lock(m.mu);
            for (auto& p : m.queue) {
                auto& t = m.tickets[p.ticket];
                t.done = true;
                t.error = std::string("serving loop stopped: ") + e.what();
            }
            m.queue.clear();
            m.cv_done.notify_all();
        }
    });
    m.completer = std::thread([&m] { m.run_completer(); });
}

Server::~Server() {
    Impl& m = *impl_;
    {
        std::lock_guard<std::mutex> lock(m.mu);
        m.stop = true;
        m.cv_work.notify_all();
    }
    if (m.scheduler.joinable()) m.scheduler.join();
    {
        std::lock_guard<std::mutex> lock(m.mu);
        m.stop_launchers = true;
        m.cv_ready.notify_all();
    }
    for (auto& t : m.launchers)
        if (t.joinable()) t.join();
    {
        std::lock_guard<std::mutex> lock(m.mu);
        m.stop_completer = true;
        m.cv_work.notify_all();
    }
    if (m.completer.joinable()) m.completer.join();
    cudaSetDevice(m.opt.device);
    cudaDeviceSynchronize();
    m.graphs.clear();
    for (auto& [b, p] : m.free_stage)
        if (!m.in_arena(p)) cudaFreeHost(p);
    if (m.arena) cudaFreeHost(m.arena);
}

std::uint64_t Server::submit(ServeRequest r) {
    Impl& m = *impl_;
    if (!r.molecule) throw std::invalid_argument("serving request without a molecule");
    const Evaluator ev(*r.molecule, r.options);  // option checks
    ev.validate(r.request);
    Impl::Pending p;
    if (r.grid) {
        p.n = detail::validated_point_count(*r.grid);
    } else {
        if (r.points.size() % 3) throw std::invalid_argument("points must hold 3 coordinates per point");
        p.n = r.points.size() / 3;
        for (double x : r.points)
            if (!std::isfinite(x)) throw std::invalid_argument("evaluation points must be finite");
    }
    const auto& props = r.request.properties();
    if (r.outputs.size() != props.size()) throw std::invalid_argument("one output array per property");
    for (double* o : r.outputs)
        if (!o && p.n) throw std::invalid_argument("null output array");
    for (const auto& q : props) p.channels += property_channels(q.kind);
    bool esp = false;
    for (const auto& q : props) esp |= q.kind == PropertyKind::ElectrostaticPotential;
    p.n_eval = p.n;
    const bool tiles = r.grid && r.options.precision == Precision::Mixed && detail::mixed_grid_tiles(r.options.block_size);
    detail::TileShape ts;
    if (tiles) {
        ts = detail::choose_tiles(*r.grid);
        p.n_eval = static_cast<std::size_t>(ts.padded());
    }
    p.graph = p.n > 0 && p.n_eval <= m.opt.graph_points && !esp;
    if (p.graph && tiles) detail::tile_order(*r.grid, ts, p.tile_index);
    const std::size_t rows = p.graph ? round_bucket(p.n_eval) : p.n;
    const std::size_t nblocks = (rows + 127) / 128;
    const std::size_t per_block = 10 * r.molecule->basis_size() * 128 * 8 + 8 * r.molecule->basis_size();
    p.footprint = p.channels * rows * 8 + 3 * rows * 8 + std::min(m.opt.request_scratch, nblocks * per_block) +
                  (std::size_t(8) << 20);
    if (p.footprint > m.budget) throw std::invalid_argument("request exceeds the serving HBM budget");
    p.req = std::move(r);
    p.t_submit = clock_type::now();
    std::lock_guard<std::mutex> lock(m.mu);
    p.ticket = m.next_ticket++;
    m.tickets[p.ticket] = {};
    ++m.st.submitted;
    if (!m.t_first) m.t_first = p.t_submit;
    const std::uint64_t t = p.ticket;
    m.queue.push_back(std::move(p));
    m.cv_work.notify_all();
    return t;
}

bool Server::wait(std::uint64_t ticket, double timeout_s) {
    Impl& m = *impl_;
    std::unique_lock<std::mutex> lock(m.mu);
    auto it = m.tickets.find(ticket);
    if (it == m.tickets.end()) throw std::invalid_argument("unknown serving ticket");
    const auto deadline = clock_type::now() + std::chrono::duration_cast<clock_type::duration>(
                                                  std::chrono::duration<double>(std::max(0.0, timeout_s)));
    m.cv_done.wait_until(lock, deadline, [&] { return m.tickets[ticket].done; });
    const Ticket& t = m.tickets[ticket];
    if (!t.done) return false;
    if (!t.error.empty()) throw std::runtime_error(t.error);
    return true;
}

void Server::drain() {
    Impl& m = *impl_;
    std::unique_lock<std::mutex> lock(m.mu);
    m.cv_done.wait(lock, [&] {
        for (const auto& [k, t] : m.tickets)
            if (!t.done) return false;
        return true;
    });
}

ServeStats Server::stats() const {
    const Impl& m = *impl_;
    std::lock_guard<std::mutex> lock(m.mu);
    ServeStats s = m.st;
    std::vector<double> l = m.latencies;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {
            const double pos = q * static_cast<double>(l.size() - 1);
            const std::size_t i = static_cast<std::size_t>(pos);
            const double f = pos - static_cast<double>(i);
            return i + 1 < l.size() ? l[i] * (1 - f) + l[i + 1] * f : l[i];
        };
        s.p50_ms = pct(0.5);
        s.p99_ms = pct(0.99);
        double sum = 0;
        for (double x : l) sum += x;
        s.mean_ms = sum / static_cast<double>(l.size());
        s.max_ms = l.back();
    }
    if (m.admitted) s.queue_ms = m.queue_sum_ms / static_cast<double>(m.admitted);
    if (m.t_first && m.t_last) {
        s.busy_s = std::chrono::duration<double>(*m.t_last - *m.t_first).count();
        if (s.busy_s > 0) s.points_per_s = static_cast<double>(s.points) / s.busy_s;
    }
    return s;
}

void Server::reset_stats() {
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lock(m.mu);
    m.latencies.clear();
    m.queue_sum_ms = 0;
    m.admitted = 0;
    const std::size_t budget = m.st.budget_bytes;
    m.st = ServeStats{};
    m.st.budget_bytes = budget;
    m.t_first.reset();
    m.t_last.reset();
}

}  // namespace chem::kumo
