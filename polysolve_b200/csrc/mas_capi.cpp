// Host side of the B200 MAS-PCG solver behind the C ABI (include/polysolve_mas.h).
//
// MasSolver mirrors MASSolver::MASSolverImpl (src/polysolve/linear/MASSolver.cu:134-595):
// parameters and info, ordering + permutation, the permuted block matrix, the MAS
// preconditioner and the PCG loop. Differences by design:
//   * the ordering is Morton (positions given) or graph bisection instead of KaMinPar;
//   * all scalars live on the device; the iteration is launched in chunks and the host only
//     looks at the device state between chunks (one chunk ahead), instead of a blocking read
//     every 10 iterations (MASSolver.cu:533-560);
//   * extension parameters (precision, true_residual_period, check_period, initial_guess, beta,
//     ordering) default to the reference's behaviour.

#include "polysolve_mas.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <limits>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>
#include <omp.h>

#include "mas_internal.h"
#include "mas_json.h"
#include "mas_ordering.h"
#include "mas_trainer.h"

using namespace pmas;

namespace
{
    struct Params
    {
        // Reference keys (MASSolver.cu:137-143, impl defaults).
        int block_dim = 1;
        int max_iter = 5000;
        double rel_tol = 1e-5;
        double abs_tol = 1e-8;
        bool lazy = false;
        bool use_prec_norm = false;
        // Extensions; defaults reproduce the reference's algorithm.
        int storage = STORE_F64; // precision of the stored MAS inverses
        int true_residual_period = 4;
        int check_period = 10;
        bool initial_guess_input = false;
        bool initial_guess_learned = false; // x0 from the solver's own kept solutions
        bool polak_ribiere = false;
        std::string ordering = "auto";
        int poll_period = 10;
        // Values-only refactorizations rebuild the MAS inverses every this many calls (1: every
        // call, as the reference); in between PCG runs with the current A and the last inverses,
        // a valid preconditioner all the same (the tolerance is met as usual).
        int preconditioner_refresh = 1;
        bool profile = false; // time every kernel launch with CUDA events
        bool graphs = true;   // replay chunks of iterations as a CUDA graph
        // Launch the PCG iteration kernels with programmatic dependent launch (each may become
        // resident while its predecessor drains); false: plain stream order.
        bool chained = true;
        // Iterations of each bounded device-side wait before the solve stops with MAS_ERR_TIMEOUT
        // (0: every wait gives up at once -- the test of the timeout path).
        long long wait_limit = MBAR_SPIN_LIMIT_DEFAULT;
        // Right-hand sides per group of several-right-hand-side solves: 0 = 16 for more than four
        // right-hand sides with block_dim 3, else 4; or 4 / 16 explicitly.
        int rhs_group = 0;
        // Sixteen-right-hand-side MAS apply: warp tensor cores (mma.sync, binary16 upper-triangle
        // storage) or the fifth-generation tensor cores (tcgen05.mma into tensor memory, from a full
        // binary16 copy of the inverses built on first use after each factorization).
        bool wide_tc = false;
        // Slots per loop trip of the SpMV (1, 2, 4): a launch-shape choice for the autotuner.
        int spmv_unroll = 2;
        // mas_solve_batch: one launch per PCG phase for each group of systems (fused), or one
        // CUDA stream per system driven by host threads (streams, measured faster on the
        // 64-system workload: 37.7-37.9 against 38.2-38.4 ms per batch).
        bool batch_fused = false;
        // Minimum items per warp of the MAS apply (a launch shape for the autotuner: 1 suits a
        // lone solve, more suits batches of small systems).
        int apply_ipw = 1;
        // Fused groups of a batch, each on its own stream (systems split by size into groups of
        // about equal work); 0 = automatic (1, measured best).
        int batch_groups = 0;
    };

    const char *status_string(int s)
    {
        switch (s)
        {
        case MAS_STATUS_RUNNING:
            return "Running";
        case MAS_STATUS_REACH_RELATIVE_TOLERANCE:
            return "Reach relative tolerance";
        case MAS_STATUS_REACH_ABSOLUTE_TOLERANCE:
            return "Reach absolute tolerance";
        case MAS_STATUS_REACH_MAX_ITERATIONS:
            return "Reach max iterations";
        default:
            return "Unknown";
        }
    }

    int get_int(const Json &v, const char *key)
    {
        if (v.type != Json::Number || !v.is_integer)
            throw Error(ERR_INVALID, std::string("[MAS] parameter ") + key + " must be an integer");
        return (int)v.num;
    }
    double get_num(const Json &v, const char *key)
    {
        if (v.type != Json::Number)
            throw Error(ERR_INVALID, std::string("[MAS] parameter ") + key + " must be a number");
        return v.num;
    }
    bool get_bool(const Json &v, const char *key)
    {
        if (v.type != Json::Bool)
            throw Error(ERR_INVALID, std::string("[MAS] parameter ") + key + " must be a boolean");
        return v.b;
    }
    std::string get_str(const Json &v, const char *key)
    {
        if (v.type != Json::String)
            throw Error(ERR_INVALID, std::string("[MAS] parameter ") + key + " must be a string");
        return v.str;
    }

    const char *KNOWN_KEYS[] = {"block_dim", "max_iter", "relative_tolerance", "absolute_tolerance",
                                "lazy_partitioning", "use_preconditioned_residual_norm", "precision",
                                "true_residual_period", "check_period", "initial_guess", "beta", "ordering",
                                "poll_period", "profile_kernels", "cuda_graphs", "preconditioner_refresh",
                                "device_wait_limit", "rhs_group", "chained_launch", "wide_apply", "spmv_unroll",
                                "batch_launch", "batch_groups", "apply_items_per_warp"};

    // MASSolverImpl::set_parameters (MASSolver.cu:198-212) plus the extension keys.
    void apply_mas_params(Params &p, const Json &m, bool strict)
    {
        if (m.type != Json::Object)
            throw Error(ERR_INVALID, "[MAS] \"MAS\" parameters must be an object");
        if (strict)
            for (const auto &kv : m.obj)
            {
                bool ok = false;
                for (const char *k : KNOWN_KEYS)
                    ok = ok || kv.first == k;
                if (!ok)
                    throw Error(ERR_INVALID, "[MAS] invalid input json: unknown key /MAS/" + kv.first);
            }
        Params q = p;
        if (auto *v = m.find("block_dim"))
        {
            q.block_dim = get_int(*v, "block_dim");
            if (q.block_dim < 1 || q.block_dim > 3)
                throw Error(ERR_INVALID, "[MAS] block_dim must be 1, 2 or 3");
        }
        if (auto *v = m.find("max_iter"))
            q.max_iter = get_int(*v, "max_iter");
        if (auto *v = m.find("relative_tolerance"))
            q.rel_tol = get_num(*v, "relative_tolerance");
        if (auto *v = m.find("absolute_tolerance"))
            q.abs_tol = get_num(*v, "absolute_tolerance");
        if (auto *v = m.find("lazy_partitioning"))
            q.lazy = get_bool(*v, "lazy_partitioning");
        if (auto *v = m.find("use_preconditioned_residual_norm"))
            q.use_prec_norm = get_bool(*v, "use_preconditioned_residual_norm");
        if (auto *v = m.find("precision"))
        {
            const std::string s = get_str(*v, "precision");
            if (s != "fp64" && s != "fp32" && s != "fp16")
                throw Error(ERR_INVALID, "[MAS] precision must be \"fp64\", \"fp32\" or \"fp16\"");
            q.storage = s == "fp64" ? STORE_F64 : (s == "fp32" ? STORE_F32 : STORE_F16);
        }
        if (auto *v = m.find("true_residual_period"))
        {
            q.true_residual_period = get_int(*v, "true_residual_period");
            if (q.true_residual_period < 1)
                throw Error(ERR_INVALID, "[MAS] true_residual_period must be >= 1");
        }
        if (auto *v = m.find("check_period"))
        {
            q.check_period = get_int(*v, "check_period");
            if (q.check_period < 1)
                throw Error(ERR_INVALID, "[MAS] check_period must be >= 1");
        }
        if (auto *v = m.find("initial_guess"))
        {
            const std::string s = get_str(*v, "initial_guess");
            if (s != "zero" && s != "input" && s != "learned")
                throw Error(ERR_INVALID, "[MAS] initial_guess must be \"zero\", \"input\" or \"learned\"");
            q.initial_guess_input = (s == "input");
            q.initial_guess_learned = (s == "learned");
        }
        if (auto *v = m.find("beta"))
        {
            const std::string s = get_str(*v, "beta");
            if (s != "fletcher_reeves" && s != "polak_ribiere")
                throw Error(ERR_INVALID, "[MAS] beta must be \"fletcher_reeves\" or \"polak_ribiere\"");
            q.polak_ribiere = (s == "polak_ribiere");
        }
        if (auto *v = m.find("ordering"))
        {
            const std::string s = get_str(*v, "ordering");
            if (s != "auto" && s != "morton" && s != "graph" && s != "natural")
                throw Error(ERR_INVALID, "[MAS] ordering must be \"auto\", \"morton\", \"graph\" or \"natural\"");
            q.ordering = s;
        }
        if (auto *v = m.find("profile_kernels"))
            q.profile = get_bool(*v, "profile_kernels");
        if (auto *v = m.find("cuda_graphs"))
            q.graphs = get_bool(*v, "cuda_graphs");
        if (auto *v = m.find("chained_launch"))
            q.chained = get_bool(*v, "chained_launch");
        if (auto *v = m.find("spmv_unroll"))
        {
            q.spmv_unroll = get_int(*v, "spmv_unroll");
            if (q.spmv_unroll != 1 && q.spmv_unroll != 2 && q.spmv_unroll != 4)
                throw Error(ERR_INVALID, "[MAS] spmv_unroll must be 1, 2 or 4");
        }
        if (auto *v = m.find("wide_apply"))
        {
            const std::string w = get_str(*v, "wide_apply");
            if (w != "mma_sync" && w != "tcgen05")
                throw Error(ERR_INVALID, "[MAS] wide_apply must be \"mma_sync\" or \"tcgen05\"");
            q.wide_tc = (w == "tcgen05");
        }
        if (auto *v = m.find("batch_launch"))
        {
            const std::string w = get_str(*v, "batch_launch");
            if (w != "fused" && w != "streams")
                throw Error(ERR_INVALID, "[MAS] batch_launch must be \"fused\" or \"streams\"");
            q.batch_fused = (w == "fused");
        }
        if (auto *v = m.find("apply_items_per_warp"))
        {
            q.apply_ipw = get_int(*v, "apply_items_per_warp");
            if (q.apply_ipw < 1 || q.apply_ipw > 64)
                throw Error(ERR_INVALID, "[MAS] apply_items_per_warp must be 1 to 64");
        }
        if (auto *v = m.find("batch_groups"))
        {
            q.batch_groups = get_int(*v, "batch_groups");
            if (q.batch_groups < 0 || q.batch_groups > 64)
                throw Error(ERR_INVALID, "[MAS] batch_groups must be 0 (automatic) to 64");
        }
        if (auto *v = m.find("poll_period"))
        {
            q.poll_period = get_int(*v, "poll_period");
            if (q.poll_period < 1)
                throw Error(ERR_INVALID, "[MAS] poll_period must be >= 1");
        }
        if (auto *v = m.find("preconditioner_refresh"))
        {
            q.preconditioner_refresh = get_int(*v, "preconditioner_refresh");
            if (q.preconditioner_refresh < 1)
                throw Error(ERR_INVALID, "[MAS] preconditioner_refresh must be >= 1");
        }
        if (auto *v = m.find("rhs_group"))
        {
            q.rhs_group = get_int(*v, "rhs_group");
            if (q.rhs_group != 0 && q.rhs_group != RHS_GROUP && q.rhs_group != RHS_WIDE)
                throw Error(ERR_INVALID, "[MAS] rhs_group must be 0, 4 or 16");
        }
        if (auto *v = m.find("device_wait_limit"))
        {
            q.wait_limit = get_int(*v, "device_wait_limit");
            if (q.wait_limit < 0)
                throw Error(ERR_INVALID, "[MAS] device_wait_limit must be >= 0");
        }
        p = q;
    }

    std::string g_create_error;
} // namespace

struct mas_solver
{
    Params p;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr; // own_stream or the caller's (mas_set_stream)
    std::string last_error;

    // Kernel accounting: launches per kind, and CUDA-event time per kind when profiling.
    struct KStat
    {
        long long launches = 0;
        double ms = 0.0;
    };
    std::vector<std::pair<std::string, KStat>> kstats;
    long long total_launches = 0;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
    size_t ev_used = 0;
    cudaEvent_t ev_origin = nullptr; // solve start, for the profiled launch timeline
    std::vector<std::pair<int, std::pair<float, float>>> timeline; // kind, start ms, end ms (profiled)

    // CUDA graphs of `chunk` PCG iterations, replayed until the device flags done. When the
    // true-residual period is a multiple of the chunk, graph[0] has no true-residual SpMV and
    // graph[1] recomputes it in its last iteration; otherwise graph[0] launches the (device-gated)
    // true-residual SpMV in every iteration.
    cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
    uint64_t graph_key = 0;
    bool graph_aligned = false;
    bool capturing = false;
    std::vector<std::pair<int, long long>> graph_counts[2]; // kernels per kind in one replay
    int capture_slot = 0;

    // Info of the last solve (MASSolver.cu:145-149).
    int iterations = 0;
    double residual_norm = 0.0;
    int status = MAS_STATUS_RUNNING;
    double rr0 = 0.0, rz0 = 0.0;
    double solve_ms = 0.0, factorize_ms = 0.0;
    std::vector<std::pair<std::string, double>> factorize_phases; // host-clock ms per phase
    DevBuf<double> refresh_vals; // CSC values on the device (kept: nnz doubles)
    // Pinned double buffer for large uploads from pageable host memory (the CSC values).
    static constexpr size_t STAGE_BYTES = (size_t)16 << 20;
    char *h_stage = nullptr;
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    int launched_iterations = 0;

    std::vector<double> positions;
    long long positions_version = 0;  // bumped by set_positions
    long long ordered_version = -1;   // positions_version the current ordering was built from
    std::string ordered_mode;         // the ordering parameter it was built with
    int first_iso_bank_cached = 0;
    int refreshes_skipped = 0;      // values-only refactorizations since the inverses were rebuilt
    bool preconditioner_current = true;

    // Ordering / pattern state.
    int n = 0, V = 0, banks = 0, bd = 0;
    long long nnz = 0;
    uint64_t pattern = 0;
    std::string ordering_used;
    std::vector<int> padded;
    DevBuf<int> d_padded, d_node_real;
    BankedMatrix A;
    MasDevice mas;
    bool factorized = false;

    DevBuf<double> x, b, r, pv, z, Ap, io;
    DevBuf<PcgState> st;
    DevBuf<double> partials;
    int red_capacity = 0;

    // Several right-hand sides at once: groups of RHS_GROUP interleaved vectors, one PcgState
    // per right-hand side plus the group record, their own graphs.
    DevBuf<double> gx, gb, gr, gp, gz, gAp, grc, gzc, gio, gpartials;
    DevBuf<PcgState> gst;
    cudaGraphExec_t ggraph[2] = {nullptr, nullptr};
    std::vector<std::pair<int, long long>> ggraph_counts[2];

    // Learned warm start: the last four solutions (padded order), the network's weights and
    // scratch, and the record of the last prediction.
    DevBuf<double> hist[WS_HISTORY]; // ring: hist[hist_newest] is the last solution
    int hist_newest = 0, hist_count = 0;
    DevBuf<float> ws_params;
    DevBuf<uint16_t> ws_wl; // bf16 bits of the layer weights
    bool ws_loaded = false;
    DevBuf<int> ws_diag;
    DevBuf<float> ws_wslot, ws_feat;
    DevBuf<uint16_t> ws_h0, ws_h1;
    DevBuf<double> ws_c, ws_yc, ws_rg, ws_y[WS_HISTORY], ws_partials;
    DevBuf<WsState> ws_state;
    WsState *h_ws = nullptr; // pinned copy of the last prediction's record
    bool ws_graph_valid = false;
    bool ws_predicted = false; // the last solve's x0 came from the network pipeline
    std::string x0_source = "zero";
    cudaEvent_t ws_ev[2] = {nullptr, nullptr};
    double warm_start_ms = 0.0;
    bool keep_stats = false; // the warm start's launches belong to the next solve's statistics
    bool in_multi = false;
    uint64_t ggraph_key = 0;
    bool ggraph_aligned = false;
    std::vector<int> rhs_iterations, rhs_status;
    std::vector<double> rhs_error;
    bool last_multi = false; // the last solve was a several-right-hand-side solve
    PcgState *h_st = nullptr; // pinned, 2 slots

    ~mas_solver()
    {
        if (stream)
        {
            cudaSetDevice(device);
            cudaStreamSynchronize(stream);
        }
        for (cudaEvent_t e : ev_pool)
            cudaEventDestroy(e);
        for (auto &g : graph_exec)
            if (g)
                cudaGraphExecDestroy(g);
        for (auto &g : ggraph)
            if (g)
                cudaGraphExecDestroy(g);
        if (h_st)
            cudaFreeHost(h_st);
        if (h_ws)
            cudaFreeHost(h_ws);
        if (h_stage)
            cudaFreeHost(h_stage);
        for (cudaEvent_t e : stage_ev)
            if (e)
                cudaEventDestroy(e);
        for (cudaEvent_t e : ws_ev)
            if (e)
                cudaEventDestroy(e);
        if (own_stream)
            cudaStreamDestroy(own_stream);
    }

    int stat_index(const char *kind)
    {
        for (size_t i = 0; i < kstats.size(); ++i)
            if (kstats[i].first == kind)
                return (int)i;
        kstats.emplace_back(kind, KStat{});
        return (int)kstats.size() - 1;
    }

    cudaEvent_t pool_event()
    {
        if (ev_used == ev_pool.size())
        {
            cudaEvent_t e;
            cuda_check(cudaEventCreate(&e), "event");
            ev_pool.push_back(e);
        }
        return ev_pool[ev_used++];
    }

    // Launch through here: counts kernels (`kernels` per call) and, when profiling, brackets the
    // launch with events on the launching stream.
    // f returns the number of kernels it launched (or void: `kernels`).
    template <class F>
    void run(const char *kind, int kernels, F &&f)
    {
        run_on(stream, kind, kernels, std::forward<F>(f));
    }

    template <class F>
    void run_on(cudaStream_t on, const char *kind, int kernels, F &&f)
    {
        const int idx = stat_index(kind);
        cudaEvent_t a = nullptr, b = nullptr;
        if (p.profile)
        {
            a = pool_event();
            b = pool_event();
            cuda_check(cudaEventRecord(a, on), "event");
        }
        if constexpr (std::is_same_v<decltype(f()), int>)
            kernels = f();
        else
            f();
        if (capturing)
        {
            bool found = false;
            for (auto &gc : graph_counts[capture_slot])
                if (gc.first == idx)
                {
                    gc.second += kernels;
                    found = true;
                }
            if (!found)
                graph_counts[capture_slot].push_back({idx, kernels});
        }
        else
        {
            kstats[idx].second.launches += kernels;
            total_launches += kernels;
        }
        if (p.profile)
        {
            cuda_check(cudaEventRecord(b, on), "event");
            ev_pending.push_back({idx, {a, b}});
        }
    }

    // The MAS apply of the current r, whose level-0 restriction is already in rc: the coarse
    // levels above the first, then every inverse (last CTA: PCG scalars). mode 1 = initial,
    // 2 = iteration.
    void apply_levels(const MasView &mv, const PcgConfig &cfg, int mode)
    {
        PcgState *S = st.get();
        run("coarse_levels", 0, [&] { return launch_coarse_levels(mv, S, stream); });
        run("mas_apply", 1, [&] { launch_mas_apply(mv, r.get(), z.get(), S, red(), cfg, mode, stream); });
    }

    void collect_profile()
    {
        timeline.clear();
        for (auto &e : ev_pending)
        {
            float ms = 0.f;
            cuda_check(cudaEventElapsedTime(&ms, e.second.first, e.second.second), "event time");
            kstats[e.first].second.ms += ms;
            if (ev_origin && timeline.size() < 400)
            {
                float t0 = 0.f, t1 = 0.f;
                cudaEventElapsedTime(&t0, ev_origin, e.second.first);
                cudaEventElapsedTime(&t1, ev_origin, e.second.second);
                timeline.push_back({e.first, {t0, t1}});
            }
        }
        ev_pending.clear();
        ev_used = 0;
    }

    void init_device()
    {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        {
            cudaGetLastError();
            throw Error(ERR_NO_DEVICE, "No Nvidia GPU!!");
        }
        cuda_check(cudaGetDevice(&device), "get device");
        cuda_check(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking), "stream create");
        stream = own_stream;
        cuda_check(cudaMallocHost(&h_st, 2 * sizeof(PcgState)), "pinned state");
    }

    // Host -> device copy of a large pageable array: host threads copy 16 MB chunks into a pinned
    // double buffer while the previous chunk's DMA runs (a plain pageable copy goes through one
    // staging thread of the driver). Small arrays take the plain path.
    void upload_pageable(void *dst, const void *src, size_t bytes)
    {
        if (bytes < 2 * STAGE_BYTES)
        {
            cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream), "upload");
            return;
        }
        if (!h_stage)
        {
            cuda_check(cudaMallocHost(&h_stage, 2 * STAGE_BYTES), "pinned staging");
            for (cudaEvent_t &e : stage_ev)
                cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        }
        const int threads = std::max(1, std::min(8, omp_get_max_threads()));
        bool used[2] = {false, false};
        for (size_t off = 0, i = 0; off < bytes; off += STAGE_BYTES, ++i)
        {
            const int slot = (int)(i & 1);
            const size_t len = std::min(STAGE_BYTES, bytes - off);
            if (used[slot])
                cuda_check(cudaEventSynchronize(stage_ev[slot]), "staging");
            char *buf = h_stage + slot * STAGE_BYTES;
            const char *from = static_cast<const char *>(src) + off;
#pragma omp parallel for num_threads(threads) schedule(static)
            for (int t = 0; t < threads; ++t)
            {
                const size_t a = len * t / threads, z = len * (t + 1) / threads;
                std::memcpy(buf + a, from + a, z - a);
            }
            cuda_check(cudaMemcpyAsync(static_cast<char *>(dst) + off, buf, len, cudaMemcpyHostToDevice, stream),
                       "upload");
            cuda_check(cudaEventRecord(stage_ev[slot], stream), "event");
            used[slot] = true;
        }
    }

    // Device -> host copy into pageable memory, the reverse of upload_pageable: 16 MB chunks DMA'd
    // into the pinned double buffer while host threads copy the previous chunk out.
    void download_pageable(void *dst, const void *src, size_t bytes)
    {
        if (bytes < 2 * STAGE_BYTES)
        {
            cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream), "download");
            cuda_check(cudaStreamSynchronize(stream), "download");
            return;
        }
        if (!h_stage)
        {
            cuda_check(cudaMallocHost(&h_stage, 2 * STAGE_BYTES), "pinned staging");
            for (cudaEvent_t &e : stage_ev)
                cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        }
        const int threads = std::max(1, std::min(8, omp_get_max_threads()));
        const size_t chunks = (bytes + STAGE_BYTES - 1) / STAGE_BYTES;
        auto start = [&](size_t i) {
            const size_t off = i * STAGE_BYTES, len = std::min(STAGE_BYTES, bytes - off);
            cuda_check(cudaMemcpyAsync(h_stage + (i & 1) * STAGE_BYTES, static_cast<const char *>(src) + off, len,
                                       cudaMemcpyDeviceToHost, stream),
                       "download");
            cuda_check(cudaEventRecord(stage_ev[i & 1], stream), "event");
        };
        start(0);
        for (size_t i = 0; i < chunks; ++i)
        {
            if (i + 1 < chunks)
                start(i + 1); // stream order: chunk i + 1 goes into the other buffer
            cuda_check(cudaEventSynchronize(stage_ev[i & 1]), "staging");
            const size_t off = i * STAGE_BYTES, len = std::min(STAGE_BYTES, bytes - off);
            const char *buf = h_stage + (i & 1) * STAGE_BYTES;
            char *to = static_cast<char *>(dst) + off;
#pragma omp parallel for num_threads(threads) schedule(static)
            for (int t = 0; t < threads; ++t)
            {
                const size_t a = len * t / threads, z = len * (t + 1) / threads;
                std::memcpy(to + a, buf + a, z - a);
            }
        }
    }

    // MASSolverImpl::factorize (MASSolver.cu:292-374).
    // declared: a values-only refactorization the caller declares (mas_factorize_values): the
    // pattern is the last factorization's, so the row indices are neither read nor hashed.
    void factorize(int n_, const int *outer, const int *inner, const double *vals, long long nnz_,
                   bool declared = false)
    {
        auto t0 = std::chrono::steady_clock::now();
        auto tp = t0;
        factorize_phases.clear();
        ws_graph_valid = false; // the neighbour weights follow the values
        inv_tc_valid = false;   // so does the tcgen05 copy of the inverses
        auto phase = [&](const char *name) {
            const auto now = std::chrono::steady_clock::now();
            factorize_phases.emplace_back(name, std::chrono::duration<double, std::milli>(now - tp).count());
            tp = now;
        };
        cuda_check(cudaSetDevice(device), "set device");
        if (declared)
        {
            if (!factorized)
                throw Error(ERR_NOT_FACTORIZED, "[MAS] factorize_values: no earlier factorization to reuse.");
            if (!vals || n_ != n || nnz_ != nnz)
                throw Error(ERR_INVALID, "[MAS] factorize_values: the values do not match the factorized pattern.");
        }
        else if (n_ <= 0 || !outer || !inner || !vals)
            throw Error(ERR_INVALID, "[MAS] factorize: invalid matrix arguments.");
        if (!declared && (outer[0] != 0 || (long long)outer[n_] != nnz_ || nnz_ < 0))
            throw Error(ERR_INVALID, "[MAS] factorize: outer index array is inconsistent with nnz.");
        if (nnz_ > 2147483647LL)
            throw Error(ERR_INVALID, "[MAS] A is too large. Non-zero number exceeding int32 max.");
        const int bd_ = p.block_dim;
        const int V_ = (n_ + bd_ - 1) / bd_;
        // The pattern hash (host threads) runs while the values go to the device: both paths
        // below need them there.
        uint64_t h = 0;
        bool pattern_ok = false;
        // Host threads split between the two (measured on a 16-core host: 8 + 8 beats sharing all
        // cores between both, which oversubscribes them).
        const int upload_threads = std::max(1, std::min(8, omp_get_max_threads()));
        const int hash_threads = std::max(1, omp_get_max_threads() - upload_threads);
        if (declared)
        {
            h = pattern;
            pattern_ok = true;
            refresh_vals.alloc(nnz_ > 0 ? nnz_ : 1, "MAS permuted_bsr input_csc");
            upload_pageable(refresh_vals.get(), vals, sizeof(double) * (size_t)nnz_);
        }
        else
        {
            std::thread hasher([&] { h = pattern_hash(n_, outer, inner, nnz_, &pattern_ok, hash_threads); });
            try
            {
                refresh_vals.alloc(nnz_ > 0 ? nnz_ : 1, "MAS permuted_bsr input_csc");
                upload_pageable(refresh_vals.get(), vals, sizeof(double) * (size_t)nnz_);
            }
            catch (...)
            {
                hasher.join();
                throw;
            }
            hasher.join();
        }
        if (!pattern_ok)
            throw Error(ERR_INVALID, "[MAS] Invalid CSC: row index out of range or decreasing column pointers.");
        // The ordering is a pure function of the pattern, the positions and the ordering
        // parameter: it is rebuilt only when one of them changed (lazy_partitioning keeps it even
        // then, as the reference does, MASSolver.cu:304-320).
        const bool shape_same = factorized && padded.size() == (size_t)V_ && bd_ == bd && n_ == n;
        const bool inputs_same = shape_same && h == pattern && nnz_ == nnz && positions_version == ordered_version &&
                                 p.ordering == ordered_mode;
        const bool rebuild_order = !(shape_same && (p.lazy || inputs_same));
        const bool same_pattern = factorized && !rebuild_order && h == pattern && nnz_ == nnz && bd_ == A.bd &&
                                  mas.storage == p.storage;
        if (declared && !same_pattern)
            throw Error(ERR_INVALID, "[MAS] factorize_values: positions, ordering, block_dim or precision changed "
                                     "since the last factorization; call factorize.");
        phase(declared ? "upload" : "pattern_check_and_upload");

        if (rebuild_order)
        {
            std::vector<uint8_t> iso = isolated_blocks(n_, outer, inner, bd_);
            std::string mode = p.ordering;
            if (mode == "auto")
                mode = (positions.size() == (size_t)V_ * 3) ? "morton" : "graph";
            int nb = 0;
            if (mode == "morton")
            {
                if (positions.size() != (size_t)V_ * 3)
                    throw Error(ERR_INVALID, "[MAS] ordering \"morton\" needs positions for every block row.");
                padded = morton_padded(positions.data(), V_, iso, &nb);
            }
            else if (mode == "graph")
                padded = graph_padded(n_, outer, inner, bd_, iso, &nb);
            else
                padded = natural_padded(V_, &nb);
            ordering_used = mode;
            ordered_version = positions_version;
            ordered_mode = p.ordering;
            banks = nb;
            V = V_;
            n = n_;
            bd = bd_;
            d_padded.alloc(V_, "MAS ordering");
            cuda_check(cudaMemcpyAsync(d_padded.get(), padded.data(), sizeof(int) * V_, cudaMemcpyHostToDevice, stream),
                       "upload ordering");
            std::vector<int> real(banks * 32, 0);
            for (int v = 0; v < V_; ++v)
                real[padded[v]] = 1;
            d_node_real.alloc(real.size(), "MAS ordering");
            cuda_check(cudaMemcpyAsync(d_node_real.get(), real.data(), sizeof(int) * real.size(),
                                       cudaMemcpyHostToDevice, stream),
                       "upload ordering");
            cuda_check(cudaStreamSynchronize(stream), "ordering");
            phase("ordering");
        }
        factorized = false;
        {
            DevBuf<double> &d_vals = refresh_vals; // uploaded above
            if (same_pattern)
            {
                rescatter_values(A, nnz_, d_vals.get(), stream);
            }
            else
            {
                DevBuf<int> d_outer, d_inner;
                d_outer.alloc(n_ + 1, "MAS permuted_bsr input_csc");
                d_inner.alloc(nnz_ > 0 ? nnz_ : 1, "MAS permuted_bsr input_csc");
                cuda_check(cudaMemcpyAsync(d_outer.get(), outer, sizeof(int) * (n_ + 1), cudaMemcpyHostToDevice, stream),
                           "upload outer");
                cuda_check(cudaMemcpyAsync(d_inner.get(), inner, sizeof(int) * nnz_, cudaMemcpyHostToDevice, stream),
                           "upload inner");
                A.slice.reset();
                A.cols.reset();
                A.vals.reset();
                A.scatter.reset();
                build_banked(A, n_, nnz_, d_outer.get(), d_inner.get(), d_vals.get(), bd_, V_, banks, d_padded.get(),
                             stream);
            }
            cuda_check(cudaStreamSynchronize(stream), "matrix upload");
            phase("matrix_upload");
        }
        nnz = nnz_;
        pattern = h;

        if (same_pattern)
        {
            // Values only: the coarse space, buffers and captured graphs stay valid.
            if (refreshes_skipped + 1 >= p.preconditioner_refresh)
            {
                refresh_mas_values(mas, A, d_node_real.get(), p.storage, stream); // syncs, checks pivots
                phase("mas_inverses");
                factorize_phases.emplace_back("gpu_level0_inverses", mas.inverse_ms[0]);
                factorize_phases.emplace_back("gpu_coarse_sums", mas.inverse_ms[1]);
                factorize_phases.emplace_back("gpu_coarse_inverses", mas.inverse_ms[2]);
                refreshes_skipped = 0;
                preconditioner_current = true;
            }
            else
            {
                ++refreshes_skipped; // PCG uses the new A with the previous inverses
                preconditioner_current = false;
            }
            factorized = true;
            factorize_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            return;
        }
        // Trailing banks of isolated rows (no off-diagonal block): the coarse levels skip them.
        int first_iso_bank = banks;
        {
            const std::vector<uint8_t> iso = isolated_blocks(n_, outer, inner, bd_);
            for (int v = 0; v < V_; ++v)
                if (iso[v])
                    first_iso_bank = std::min(first_iso_bank, padded[v] / 32);
            for (int v = 0; v < V_ && first_iso_bank < banks; ++v)
                if (!iso[v] && padded[v] / 32 >= first_iso_bank)
                    first_iso_bank = banks;
        }
        build_mas(mas, A, d_node_real.get(), p.storage, first_iso_bank, stream);
        phase("mas_build");
        hist_count = 0; // a new pattern or ordering: the kept solutions no longer apply
        refreshes_skipped = 0;
        preconditioner_current = true;
        prepare_kernels(bd_, p.storage);
        if (p.storage == STORE_F16)
        {
            prepare_kernels_g(bd_);
            if (bd_ == 3)
                prepare_kernels_w();
        }
        drop_graph();

        const size_t len = (size_t)banks * 32 * bd_;
        x.alloc(len, "device_buffers x");
        b.alloc(len, "device_buffers b");
        r.alloc(len, "device_buffers r");
        pv.alloc(len, "device_buffers p");
        z.alloc(len, "device_buffers z");
        Ap.alloc(len, "device_buffers Ap");
        io.alloc((size_t)n_ > len ? (size_t)n_ : len, "device_buffers io");
        st.alloc(1, "device_buffers scalars");
        red_capacity = std::max({(banks + 7) / 8, mas.total_coarse, device_sm_count() * 8}) + 160;
        partials.alloc((size_t)red_capacity * 9, "device_buffers reduction");
        cuda_check(cudaMemsetAsync(x.get(), 0, x.bytes(), stream), "memset");
        cuda_check(cudaMemsetAsync(pv.get(), 0, pv.bytes(), stream), "memset");
        cuda_check(cudaMemsetAsync(z.get(), 0, z.bytes(), stream), "memset");
        cuda_check(cudaMemsetAsync(Ap.get(), 0, Ap.bytes(), stream), "memset");
        cuda_check(cudaStreamSynchronize(stream), "factorize");
        phase("buffers");
        factorized = true;
        factorize_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }

    void require_factorized(int len)
    {
        if (!factorized || len != n || len <= 0)
            throw Error(ERR_NOT_FACTORIZED, "[MAS] Size mismatch. Did you forget to call factorize?");
    }

    ReduceBuf red()
    {
        double *base = partials.get();
        const size_t c = (size_t)red_capacity;
        return ReduceBuf{base, red_capacity, base + 2 * c, base + 3 * c};
    }

    PcgConfig config() const
    {
        PcgConfig c;
        c.max_iter = p.max_iter;
        c.rel_tol = p.rel_tol;
        c.abs_tol = p.abs_tol;
        c.use_prec_norm = p.use_prec_norm ? 1 : 0;
        c.check_period = p.check_period;
        c.polak_ribiere = p.polak_ribiere ? 1 : 0;
        c.level_num = mas.level_num;
        c.wait_limit = p.wait_limit;
        return c;
    }

    // One PCG iteration's kernels (MASSolver.cu:498-583). residual: launch the true-residual SpMV
    // and its restriction (both check (st->iter + 1) % P == 0 on the device and return at once
    // otherwise; update_xr restricts r on the other iterations).
    void launch_iteration(const BankedView &Av, const MasView &mv, const PcgConfig &cfg, int P, bool residual)
    {
        PcgState *S = st.get();
        run("spmv_pap", 1, [&] { launch_spmv(SPMV_PAP, Av, pv.get(), Ap.get(), nullptr, S, red(), 1, 0, stream); });
        run("update_xr", 1, [&] { launch_update_xr(mv, x.get(), r.get(), pv.get(), Ap.get(), S, red(), P, stream); });
        if (residual)
        {
            run("spmv_residual", 1,
                [&] { launch_spmv(SPMV_RESIDUAL, Av, x.get(), r.get(), b.get(), S, red(), 1, P, stream); });
            run("restrict", 0, [&] { return launch_restrict(mv, r.get(), S, P, stream); });
        }
        apply_levels(mv, cfg, 2);
        run("update_p", 1, [&] { launch_update_p(mv, x.get(), pv.get(), z.get(), S, 0, stream); });
    }

    void drop_graph()
    {
        for (int i = 0; i < 2; ++i)
        {
            if (graph_exec[i])
                cudaGraphExecDestroy(graph_exec[i]);
            graph_exec[i] = nullptr;
            graph_counts[i].clear();
            if (ggraph[i])
                cudaGraphExecDestroy(ggraph[i]);
            ggraph[i] = nullptr;
            ggraph_counts[i].clear();
        }
        graph_key = 0;
        ggraph_key = 0;
    }

    void capture(int slot, const BankedView &Av, const MasView &mv, const PcgConfig &cfg, int P, int chunk,
                 bool aligned)
    {
        cudaGraph_t graph = nullptr;
        capture_slot = slot;
        cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        capturing = true;
        try
        {
            for (int i = 0; i < chunk; ++i)
                launch_iteration(Av, mv, cfg, P, aligned ? (slot == 1 && i == chunk - 1) : true);
        }
        catch (...)
        {
            capturing = false;
            cudaStreamEndCapture(stream, &graph);
            if (graph)
                cudaGraphDestroy(graph);
            cudaGetLastError();
            graph_counts[slot].clear();
            throw;
        }
        capturing = false;
        cuda_check(cudaStreamEndCapture(stream, &graph), "end capture");
        cudaError_t e = cudaGraphInstantiate(&graph_exec[slot], graph, 0);
        cudaGraphDestroy(graph);
        cuda_check(e, "graph instantiate");
    }

    void ensure_graph(const BankedView &Av, const MasView &mv, const PcgConfig &cfg, int P, int chunk)
    {
        uint64_t key = 1469598103934665603ull;
        auto mix = [&key](uint64_t v) {
            key ^= v;
            key *= 1099511628211ull;
        };
        for (const void *ptr : {(const void *)x.get(), (const void *)b.get(), (const void *)r.get(),
                                (const void *)pv.get(), (const void *)z.get(), (const void *)Ap.get(),
                                (const void *)st.get(), (const void *)partials.get(), (const void *)Av.vals, mv.inv,
                                (const void *)stream})
            mix((uint64_t)(uintptr_t)ptr);
        mix((uint64_t)cfg.max_iter);
        mix((uint64_t)cfg.check_period);
        mix((uint64_t)cfg.use_prec_norm);
        mix((uint64_t)cfg.polak_ribiere);
        mix((uint64_t)cfg.wait_limit);
        mix((uint64_t)chained_launch());
        mix((uint64_t)spmv_unroll());
        mix((uint64_t)apply_items_per_warp());
        uint64_t bits;
        std::memcpy(&bits, &cfg.rel_tol, 8);
        mix(bits);
        std::memcpy(&bits, &cfg.abs_tol, 8);
        mix(bits);
        mix((uint64_t)P);
        mix((uint64_t)chunk);
        if (graph_exec[0] && key == graph_key)
            return;
        drop_graph();
        graph_aligned = (P % chunk == 0);
        capture(0, Av, mv, cfg, P, chunk, graph_aligned);
        if (graph_aligned)
            capture(1, Av, mv, cfg, P, chunk, true);
        graph_key = key;
    }

    // pcg_solve (MASSolver.cu:469-595) on device-resident b_ / x_ (padded order).
    void pcg()
    {
        const BankedView Av = A.view();
        const MasView mv = mas.view();
        const PcgConfig cfg = config();
        PcgState *S = st.get();
        cudaEvent_t e0, e1;
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        cuda_check(cudaEventRecord(e0, stream), "event");
        ev_origin = e0;
        if (!keep_stats) // per-solve kernel statistics
            for (auto &ks : kstats)
                ks.second = KStat{};
        keep_stats = false;
        set_chained_launch(p.chained);
        set_spmv_unroll(p.spmv_unroll);
        set_apply_items_per_warp(p.apply_ipw);
        launch_pcg_init_state(S, stream);
        // r = b - A x, rr0, the level-0 restriction of r, then z = M^-1 r
        run("spmv_residual", 1, [&] { launch_spmv(SPMV_RESIDUAL, Av, x.get(), r.get(), b.get(), S, red(), 0, 0, stream); });
        run("restrict", 0, [&] { return launch_restrict(mv, r.get(), S, 0, stream); });
        apply_levels(mv, cfg, 1);
        run("update_p", 1, [&] { launch_update_p(mv, x.get(), pv.get(), z.get(), S, 1, stream); });
        cuda_check(cudaMemcpyAsync(&h_st[0], S, sizeof(PcgState), cudaMemcpyDeviceToHost, stream), "state");
        cuda_check(cudaStreamSynchronize(stream), "pcg init");
        rz0 = h_st[0].rz0;
        rr0 = h_st[0].rr0;
        if (h_st[0].error == ERR_TIMEOUT)
        {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw Error(ERR_TIMEOUT, "[MAS] a device-side wait timed out.");
        }
        if (h_st[0].error == ERR_NONFINITE || std::isnan(rz0) || !std::isfinite(rz0))
        {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw Error(ERR_NONFINITE, "[MAS] Invalid initial residual.");
        }
        status = MAS_STATUS_RUNNING;
        const int P = p.true_residual_period;
        const int chunk = p.poll_period;
        const bool graphs = p.graphs && !p.profile;
        if (graphs)
            ensure_graph(Av, mv, cfg, P, chunk);
        int launched = 0;
        bool stop = false;
        int pending = -1; // slot holding the previous chunk's state copy
        cudaEvent_t chunk_ev[2];
        cuda_check(cudaEventCreateWithFlags(&chunk_ev[0], cudaEventDisableTiming), "event");
        cuda_check(cudaEventCreateWithFlags(&chunk_ev[1], cudaEventDisableTiming), "event");
        int slot_flip = 0;
        for (int k0 = 1; k0 <= p.max_iter && !stop; k0 += chunk)
        {
            const int k1 = std::min(p.max_iter, k0 + chunk - 1);
            if (graphs)
            {
                const int g = (graph_aligned && (k0 + chunk - 1) % P == 0) ? 1 : 0;
                cuda_check(cudaGraphLaunch(graph_exec[g], stream), "graph launch");
                for (auto &gc : graph_counts[g])
                {
                    kstats[gc.first].second.launches += gc.second;
                    total_launches += gc.second;
                }
            }
            else
                for (int k = k0; k <= k1; ++k)
                    launch_iteration(Av, mv, cfg, P, k % P == 0);
            launched = k1;
            const int slot = (slot_flip++) & 1;
            cuda_check(cudaMemcpyAsync(&h_st[slot], S, sizeof(PcgState), cudaMemcpyDeviceToHost, stream), "state");
            cuda_check(cudaEventRecord(chunk_ev[slot], stream), "event");
            // Look at the previous chunk's state while this chunk runs.
            if (pending >= 0)
            {
                cuda_check(cudaEventSynchronize(chunk_ev[pending]), "chunk");
                if (h_st[pending].done)
                    stop = true;
            }
            pending = slot;
        }
        cuda_check(cudaEventRecord(e1, stream), "event");
        cuda_check(cudaMemcpyAsync(&h_st[0], S, sizeof(PcgState), cudaMemcpyDeviceToHost, stream), "state");
        cuda_check(cudaStreamSynchronize(stream), "pcg");
        collect_profile();
        ev_origin = nullptr;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        solve_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(chunk_ev[0]);
        cudaEventDestroy(chunk_ev[1]);
        launched_iterations = launched;
        const PcgState &f = h_st[0];
        if (f.error == ERR_TIMEOUT)
            throw Error(ERR_TIMEOUT, "[MAS] a device-side wait timed out.");
        if (p.max_iter >= 1)
            iterations = f.iter;
        residual_norm = f.res_norm;
        status = f.status;
        if (p.max_iter < 1 && iterations == p.max_iter)
            status = MAS_STATUS_REACH_MAX_ITERATIONS;
    }

    void load_rhs_device(const double *d_src_b, const double *d_src_x)
    {
        const size_t len = (size_t)banks * 32 * bd;
        run("permute_in", 2, [&] { launch_permute_in(n, bd, V, d_padded.get(), d_src_b, b.get(), len, stream); });
        if (p.initial_guess_input && d_src_x)
            run("permute_in", 2, [&] { launch_permute_in(n, bd, V, d_padded.get(), d_src_x, x.get(), len, stream); });
        else
            cuda_check(cudaMemsetAsync(x.get(), 0, x.bytes(), stream), "memset");
    }

    // ---- Learned warm start ----------------------------------------------------------------
    void set_warm_start_model(const float *prm, long long count)
    {
        cuda_check(cudaSetDevice(device), "set device");
        if (!prm || count != WS_PARAMS)
            throw Error(ERR_INVALID, "[MAS] warm start model: expected " + std::to_string(WS_PARAMS) +
                                         " float32 parameters");
        for (long long i = 0; i < count; ++i)
            if (!std::isfinite(prm[i]))
                throw Error(ERR_INVALID, "[MAS] warm start model: non-finite parameter");
        // Layer weights to bf16 (round to nearest even) for the tensor-core products.
        std::vector<uint16_t> wl((size_t)WS_LAYERS * WS_LAYER_WEIGHTS);
        const int per_layer = WS_HIDDEN * 2 * WS_HIDDEN + WS_HIDDEN;
        for (int l = 0; l < WS_LAYERS; ++l)
        {
            const float *src = prm + WS_HIDDEN * WS_FEATURES + WS_HIDDEN + (size_t)l * per_layer;
            for (int i = 0; i < WS_LAYER_WEIGHTS; ++i)
            {
                uint32_t u;
                std::memcpy(&u, src + i, 4);
                u += 0x7FFFu + ((u >> 16) & 1u);
                wl[(size_t)l * WS_LAYER_WEIGHTS + i] = (uint16_t)(u >> 16);
            }
        }
        ws_params.alloc(WS_PARAMS, "warm start model");
        ws_wl.alloc(wl.size(), "warm start model");
        cuda_check(cudaMemcpyAsync(ws_params.get(), prm, sizeof(float) * WS_PARAMS, cudaMemcpyHostToDevice, stream),
                   "upload model");
        cuda_check(cudaMemcpyAsync(ws_wl.get(), wl.data(), sizeof(uint16_t) * wl.size(), cudaMemcpyHostToDevice,
                                   stream),
                   "upload model");
        cuda_check(cudaStreamSynchronize(stream), "upload model");
        ws_loaded = true;
    }

    WsBuffers ws_buffers()
    {
        const size_t nodes = (size_t)banks * 32;
        const size_t len = nodes * 3;
        ws_diag.alloc(nodes, "warm start scratch");
        ws_wslot.alloc((size_t)std::max<long long>(A.slots, 1) * 32, "warm start scratch");
        ws_feat.alloc(nodes * WS_FEATURES, "warm start scratch");
        ws_h0.alloc(nodes * WS_HIDDEN, "warm start scratch");
        ws_h1.alloc(nodes * WS_HIDDEN, "warm start scratch");
        ws_c.alloc(len, "warm start scratch");
        ws_yc.alloc(len, "warm start scratch");
        ws_rg.alloc(len, "warm start scratch");
        for (DevBuf<double> &v : ws_y)
            v.alloc(len, "warm start scratch");
        const int capacity = std::max((int)((nodes + 255) / 256), ws_reduce_ctas());
        if (ws_partials.n < (size_t)capacity * WS_GRAM)
            ws_partials.alloc((size_t)capacity * WS_GRAM, "warm start scratch");
        if (!ws_state.get())
        {
            ws_state.alloc(1, "warm start scratch");
            cuda_check(cudaMemsetAsync(ws_state.get(), 0, sizeof(WsState), stream), "memset");
        }
        if (!h_ws)
            cuda_check(cudaMallocHost(&h_ws, sizeof(WsState)), "pinned warm start record");
        if (!ws_ev[0])
        {
            cuda_check(cudaEventCreate(&ws_ev[0]), "event");
            cuda_check(cudaEventCreate(&ws_ev[1]), "event");
        }
        WsBuffers w;
        w.params = ws_params.get();
        w.wl = ws_wl.get();
        w.diag_slot = ws_diag.get();
        w.wslot = ws_wslot.get();
        w.feat = ws_feat.get();
        w.h[0] = ws_h0.get();
        w.h[1] = ws_h1.get();
        w.c = ws_c.get();
        w.yc = ws_yc.get();
        w.rg = ws_rg.get();
        w.st = ws_state.get();
        w.partials = ws_partials.get();
        w.capacity = (int)(ws_partials.n / WS_GRAM);
        return w;
    }

    bool learned_active() const { return p.initial_guess_learned && !in_multi; }

    // x (padded order) for the next solve of a sequence: zero, the last solution, or the
    // network's prediction combined with the kept solutions (b already loaded).
    void warm_start_guess()
    {
        ws_predicted = false;
        warm_start_ms = 0.0;
        if (hist_count == 0)
        {
            cuda_check(cudaMemsetAsync(x.get(), 0, x.bytes(), stream), "memset");
            x0_source = "zero";
            return;
        }
        const double *x1 = hist[hist_newest].get();
        if (hist_count < 2 || !ws_loaded || bd != 3)
        {
            cuda_check(cudaMemcpyAsync(x.get(), x1, x.bytes(), cudaMemcpyDeviceToDevice, stream), "copy x0");
            x0_source = "previous";
            return;
        }
        const double *xs[WS_HISTORY];
        for (int j = 0; j < hist_count; ++j)
            xs[j] = hist[(hist_newest - j + WS_HISTORY) % WS_HISTORY].get();
        for (auto &ks : kstats)
            ks.second = KStat{};
        keep_stats = true;
        WsBuffers w = ws_buffers();
        cuda_check(cudaEventRecord(ws_ev[0], stream), "event");
        ws_pipeline(w, xs, hist_count);
        cuda_check(cudaEventRecord(ws_ev[1], stream), "event");
        cuda_check(cudaMemcpyAsync(h_ws, ws_state.get(), sizeof(WsState), cudaMemcpyDeviceToHost, stream),
                   "warm start record");
        ws_predicted = true;
        x0_source = "learned";
    }

    // The prediction from the kept solutions xs[0] (newest) .. xs[count - 1], count >= 2: their
    // products with A, the network, A c, the Galerkin combination into x.
    void ws_pipeline(const WsBuffers &w, const double *const *xs, int count)
    {
        const size_t len = (size_t)banks * 32 * bd;
        const BankedView Av = A.view();
        if (!ws_graph_valid)
        {
            run("ws_graph", 1, [&] { launch_ws_graph(Av, w, stream); });
            ws_graph_valid = true;
        }
        WsHistory h;
        const int have = std::min(count, WS_HISTORY);
        for (int j = 0; j < WS_HISTORY; ++j)
        {
            const int src = std::min(j, have - 1); // missing: repeat the oldest (zero difference)
            h.x[j] = xs[src];
            h.y[j] = ws_y[src].get();
        }
        run("spmv_vectors", 1, [&] {
            double *ys[WS_HISTORY];
            for (int j = 0; j < have; ++j)
                ys[j] = ws_y[j].get();
            launch_spmv_vectors(Av, xs, ys, have, stream); // one pass over A for all kept solutions
        });
        run("ws_network", 0, [&] { return launch_ws_network(Av, w, b.get(), h, len, stream); });
        run("spmv_plain", 1, [&] { launch_spmv(SPMV_PLAIN, Av, w.c, w.yc, nullptr, nullptr, red(), 0, 0, stream); });
        run("ws_combine", 0, [&] { return launch_ws_combine(w, b.get(), h, x.get(), len, stream); });
    }

    // After a solve: keep x as the newest solution; read the prediction's record and time.
    void finish_warm_start()
    {
        if (ws_predicted)
        {
            cuda_check(cudaStreamSynchronize(stream), "warm start");
            float ms = 0.f;
            cuda_check(cudaEventElapsedTime(&ms, ws_ev[0], ws_ev[1]), "event time");
            warm_start_ms = ms;
            if (h_ws->fallback)
                x0_source = "previous (fallback)";
        }
        const size_t len = (size_t)banks * 32 * bd;
        for (DevBuf<double> &hb : hist)
            hb.alloc(len, "warm start history");
        if (hist_count > 0)
            hist_newest = (hist_newest + 1) % WS_HISTORY;
        cuda_check(cudaMemcpyAsync(hist[hist_newest].get(), x.get(), x.bytes(), cudaMemcpyDeviceToDevice, stream),
                   "keep solution");
        hist_count = std::min(hist_count + 1, WS_HISTORY);
    }

    // Tests: the prediction for caller-order b and kept solutions hhist[j * n ..] (newest first,
    // 2 <= nhist <= 4) without a solve; outputs in caller order (c, x0: n values; features:
    // V * 16; state: sums 5, Galerkin matrix and right-hand side WS_GRAM, coefficients WS_BASIS,
    // energy, energy of x1, fallback, rank).
    void debug_warm_start(const double *hb, const double *hhist, int nhist, double *hc, double *hx0,
                          float *hfeat, double *hstate)
    {
        cuda_check(cudaSetDevice(device), "set device");
        require_factorized(n);
        if (!ws_loaded || bd != 3)
            throw Error(ERR_INVALID, "[MAS] warm start: no model loaded or block_dim is not 3");
        if (!hb || !hhist || nhist < 2 || nhist > WS_HISTORY)
            throw Error(ERR_INVALID, "[MAS] warm start: b and 2 to 4 kept solutions are needed");
        const size_t len = (size_t)banks * 32 * bd;
        DevBuf<double> dh[WS_HISTORY];
        const double *xs[WS_HISTORY];
        cuda_check(cudaMemcpyAsync(io.get(), hb, sizeof(double) * n, cudaMemcpyHostToDevice, stream), "upload");
        launch_permute_in(n, bd, V, d_padded.get(), io.get(), b.get(), len, stream);
        for (int j = 0; j < nhist; ++j)
        {
            dh[j].alloc(len, "debug");
            cuda_check(cudaMemcpyAsync(io.get(), hhist + (size_t)j * n, sizeof(double) * n, cudaMemcpyHostToDevice,
                                       stream),
                       "upload");
            launch_permute_in(n, bd, V, d_padded.get(), io.get(), dh[j].get(), len, stream);
            xs[j] = dh[j].get();
        }
        WsBuffers w = ws_buffers();
        ws_pipeline(w, xs, nhist);
        if (hc)
        {
            launch_permute_out(n, bd, V, d_padded.get(), w.c, io.get(), stream);
            cuda_check(cudaMemcpyAsync(hc, io.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, stream), "download");
            cuda_check(cudaStreamSynchronize(stream), "debug warm start");
        }
        if (hx0)
        {
            launch_permute_out(n, bd, V, d_padded.get(), x.get(), io.get(), stream);
            cuda_check(cudaMemcpyAsync(hx0, io.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, stream), "download");
            cuda_check(cudaStreamSynchronize(stream), "debug warm start");
        }
        if (hfeat)
        {
            DevBuf<float> f;
            f.alloc((size_t)V * WS_FEATURES, "debug");
            launch_ws_features_out(V, d_padded.get(), w.feat, f.get(), stream);
            cuda_check(cudaMemcpyAsync(hfeat, f.get(), f.bytes(), cudaMemcpyDeviceToHost, stream), "download");
            cuda_check(cudaStreamSynchronize(stream), "debug warm start");
        }
        WsState hs;
        cuda_check(cudaMemcpyAsync(&hs, ws_state.get(), sizeof(WsState), cudaMemcpyDeviceToHost, stream), "download");
        cuda_check(cudaStreamSynchronize(stream), "debug warm start");
        if (hstate)
        {
            int k = 0;
            for (double v : hs.sums)
                hstate[k++] = v;
            for (double v : hs.gram)
                hstate[k++] = v;
            for (double v : hs.coef)
                hstate[k++] = v;
            hstate[k++] = hs.energy;
            hstate[k++] = hs.energy_prev;
            hstate[k++] = hs.fallback;
            hstate[k++] = hs.rank;
            for (double v : hs.coef_hist)
                hstate[k++] = v;
        }
    }

    // One training sample for the warm-start network: the prediction pipeline up to the features
    // (x_g over the kept solutions, r_g, raw features and their sums) for caller-order b and nhist
    // (2 to 4) kept solutions history[j * n ..] (x_{k-1} first), and the exact solution x_k.
    void collect_training_sample(mas_ws_trainer &t, const double *hb, const double *hhist, int nhist,
                                 const double *hx, int len_in)
    {
        cuda_check(cudaSetDevice(device), "set device");
        require_factorized(len_in);
        if (t.device != device)
            throw Error(ERR_INVALID, "[MAS] warm start trainer: the solver and the trainer are on different devices");
        if (bd != 3)
            throw Error(ERR_INVALID, "[MAS] the learned warm start needs block_dim 3");
        if (!hb || !hhist || !hx || nhist < 2 || nhist > WS_HISTORY)
            throw Error(ERR_INVALID, "[MAS] warm start trainer: b, x and 2 to 4 kept solutions are needed");
        const size_t len = (size_t)banks * 32 * bd;
        DevBuf<double> dh[WS_HISTORY], dxe;
        const double *xs[WS_HISTORY];
        cuda_check(cudaMemcpyAsync(io.get(), hb, sizeof(double) * n, cudaMemcpyHostToDevice, stream), "upload");
        launch_permute_in(n, bd, V, d_padded.get(), io.get(), b.get(), len, stream);
        for (int j = 0; j < nhist; ++j)
        {
            dh[j].alloc(len, "warm start trainer collection");
            cuda_check(cudaMemcpyAsync(io.get(), hhist + (size_t)j * n, sizeof(double) * n, cudaMemcpyHostToDevice,
                                       stream),
                       "upload");
            launch_permute_in(n, bd, V, d_padded.get(), io.get(), dh[j].get(), len, stream);
            xs[j] = dh[j].get();
        }
        dxe.alloc(len, "warm start trainer collection");
        cuda_check(cudaMemcpyAsync(io.get(), hx, sizeof(double) * n, cudaMemcpyHostToDevice, stream), "upload");
        launch_permute_in(n, bd, V, d_padded.get(), io.get(), dxe.get(), len, stream);
        WsBuffers w = ws_buffers();
        const BankedView Av = A.view();
        if (!ws_graph_valid)
        {
            launch_ws_graph(Av, w, stream);
            ws_graph_valid = true;
        }
        WsHistory h;
        for (int j = 0; j < WS_HISTORY; ++j)
        {
            const int src = std::min(j, nhist - 1);
            h.x[j] = xs[src];
            h.y[j] = ws_y[src].get();
        }
        {
            double *ys[WS_HISTORY];
            for (int j = 0; j < nhist; ++j)
                ys[j] = ws_y[j].get();
            launch_spmv_vectors(Av, xs, ys, nhist, stream);
        }
        launch_ws_features(Av, w, b.get(), h, len, stream);
        const uint64_t key = pattern ^ ((uint64_t)ordered_version * 0x9E3779B97F4A7C15ull) ^ (uint64_t)nnz;
        const int pat = t.pattern_for(this, key, A, w.diag_slot, stream);
        t.add_sample(pat, A, w.wslot, w.feat, w.st, w.rg, h, dxe.get(), len, stream);
        cuda_check(cudaStreamSynchronize(stream), "warm start trainer collection");
    }

    // ---- Several right-hand sides at once (RHS_GROUP per group, binary16 inverses). ----------
    bool multi_supported() const
    {
        return factorized && mas.storage == STORE_F16 && !p.polak_ribiere && !p.initial_guess_input;
    }

    // Group width w (RHS_GROUP or RHS_WIDE) of the several-right-hand-side buffers and kernels.
    int gwidth = RHS_GROUP;
    bool wide() const { return gwidth == RHS_WIDE; }
    // The tcgen05 apply's copy of the inverses (valid until the next factorization).
    DevBuf<unsigned char> inv_tc;
    bool inv_tc_valid = false;

    void ensure_tc_storage(const MasView &mv)
    {
        if (inv_tc_valid)
            return;
        inv_tc.alloc(tc_storage_bytes(mv), "MAS tc inverse storage");
        launch_inv_to_tc(mv, inv_tc.get(), stream);
        inv_tc_valid = true;
    }

    void launch_wide_apply(const MasView &mv, const PcgConfig &cfg, int mode)
    {
        if (p.wide_tc)
            launch_mas_apply_tc(mv, inv_tc.get(), gr.get(), gz.get(), gst.get(), red_g(), cfg, mode, stream);
        else
            launch_mas_apply_w(mv, gr.get(), gz.get(), gst.get(), red_g(), cfg, mode, stream);
    }
    int red_capacity_g() const { return wide() ? wide_reduce_ctas() : red_capacity; }

    void alloc_multi(int width = RHS_GROUP)
    {
        if (width != gwidth)
            for (DevBuf<double> *v : {&gx, &gb, &gr, &gp, &gz, &gAp, &grc, &gzc, &gio, &gpartials})
                v->reset(); // other sizes; the captured graphs go with them (their key has the pointers)
        gwidth = width;
        const size_t len = (size_t)banks * 32 * bd * width;
        for (DevBuf<double> *v : {&gx, &gb, &gr, &gp, &gz, &gAp})
            v->alloc(len, "device_buffers several right-hand sides");
        const size_t clen = (size_t)std::max(mas.coarse_nodes, 1) * bd * width;
        grc.alloc(clen, "MAS coarse_vectors several right-hand sides");
        gzc.alloc(clen, "MAS coarse_vectors several right-hand sides");
        gio.alloc((size_t)n * width, "device_buffers several right-hand sides");
        gpartials.alloc((size_t)red_capacity_g() * 6 * width, "device_buffers reduction");
        gst.alloc(RHS_WIDE + 1, "device_buffers state");
        // Coarse slots past the component counts are read by the coarse products and must be zero.
        cuda_check(cudaMemsetAsync(grc.get(), 0, grc.bytes(), stream), "memset");
        cuda_check(cudaMemsetAsync(gzc.get(), 0, gzc.bytes(), stream), "memset");
    }

    ReduceBuf red_g()
    {
        double *base = gpartials.get();
        const size_t c = (size_t)red_capacity_g();
        return ReduceBuf{base, red_capacity_g(), base + 2 * gwidth * c, base + 3 * gwidth * c};
    }

    MasView view_g() const { return mas.view(grc.get(), gzc.get()); }

    void launch_iteration_g(const BankedView &Av, const MasView &mv, const PcgConfig &cfg, int P, bool residual)
    {
        PcgState *S = gst.get();
        PcgState *grp = S + gwidth;
        if (wide())
        {
            run("spmv_pap", 1,
                [&] { launch_spmv_w(SPMV_PAP, Av, gp.get(), gAp.get(), nullptr, S, red_g(), 1, 0, stream); });
            run("update_xr", 1,
                [&] { launch_update_xr_w(mv, gx.get(), gr.get(), gp.get(), gAp.get(), S, red_g(), P, stream); });
            if (residual)
            {
                run("spmv_residual", 1, [&] {
                    launch_spmv_w(SPMV_RESIDUAL, Av, gx.get(), gr.get(), gb.get(), S, red_g(), 1, P, stream);
                });
                run("restrict", 0, [&] { return launch_restrict_w(mv, gr.get(), grp, P, stream); });
            }
            run("coarse_levels", 0, [&] { return launch_coarse_levels_w(mv, grp, stream); });
            run("mas_apply", 1, [&] { launch_wide_apply(mv, cfg, 2); });
            run("update_p", 1, [&] { launch_update_p_w(mv, gx.get(), gp.get(), gz.get(), S, 0, stream); });
            return;
        }
        run("spmv_pap", 1, [&] { launch_spmv_g(SPMV_PAP, Av, gp.get(), gAp.get(), nullptr, S, red_g(), 1, 0, stream); });
        run("update_xr", 1,
            [&] { launch_update_xr_g(mv, gx.get(), gr.get(), gp.get(), gAp.get(), S, red_g(), P, stream); });
        if (residual)
        {
            run("spmv_residual", 1,
                [&] { launch_spmv_g(SPMV_RESIDUAL, Av, gx.get(), gr.get(), gb.get(), S, red_g(), 1, P, stream); });
            run("restrict", 0, [&] { return launch_restrict_g(mv, gr.get(), grp, P, stream); });
        }
        run("coarse_levels", 0, [&] { return launch_coarse_levels_g(mv, stream); });
        run("mas_apply", 1, [&] { launch_mas_apply_g(mv, gr.get(), gz.get(), S, red_g(), cfg, 2, stream); });
        run("update_p", 1, [&] { launch_update_p_g(mv, gx.get(), gp.get(), gz.get(), S, 0, stream); });
    }

    void capture_g(int slot, const BankedView &Av, const MasView &mv, const PcgConfig &cfg, int P, int chunk,
                   bool aligned)
    {
        cudaGraph_t graph = nullptr;
        capture_slot = slot;
        cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        capturing = true;
        auto saved = std::move(graph_counts[slot]);
        graph_counts[slot].clear();
        try
        {
            for (int i = 0; i < chunk; ++i)
                launch_iteration_g(Av, mv, cfg, P, aligned ? (slot == 1 && i == chunk - 1) : true);
        }
        catch (...)
        {
            capturing = false;
            cudaStreamEndCapture(stream, &graph);
            if (graph)
                cudaGraphDestroy(graph);
            cudaGetLastError();
            graph_counts[slot] = std::move(saved);
            throw;
        }
        capturing = false;
        ggraph_counts[slot] = std::move(graph_counts[slot]);
        graph_counts[slot] = std::move(saved);
        cuda_check(cudaStreamEndCapture(stream, &graph), "end capture");
        cudaError_t e = cudaGraphInstantiate(&ggraph[slot], graph, 0);
        cudaGraphDestroy(graph);
        cuda_check(e, "graph instantiate");
    }

    void ensure_graph_g(const BankedView &Av, const MasView &mv, const PcgConfig &cfg, int P, int chunk)
    {
        uint64_t key = 1469598103934665603ull;
        auto mix = [&key](uint64_t v) {
            key ^= v;
            key *= 1099511628211ull;
        };
        for (const void *ptr : {(const void *)gx.get(), (const void *)gb.get(), (const void *)gr.get(),
                                (const void *)gp.get(), (const void *)gz.get(), (const void *)gAp.get(),
                                (const void *)gst.get(), (const void *)gpartials.get(), (const void *)grc.get(),
                                (const void *)Av.vals, mv.inv, (const void *)stream})
            mix((uint64_t)(uintptr_t)ptr);
        mix((uint64_t)cfg.max_iter);
        mix((uint64_t)cfg.check_period);
        mix((uint64_t)cfg.use_prec_norm);
        mix((uint64_t)cfg.wait_limit);
        mix((uint64_t)gwidth);
        mix((uint64_t)p.wide_tc);
        mix((uint64_t)(uintptr_t)inv_tc.get());
        uint64_t bits;
        std::memcpy(&bits, &cfg.rel_tol, 8);
        mix(bits);
        std::memcpy(&bits, &cfg.abs_tol, 8);
        mix(bits);
        mix((uint64_t)P);
        mix((uint64_t)chunk);
        if (ggraph[0] && key == ggraph_key)
            return;
        for (int i = 0; i < 2; ++i)
        {
            if (ggraph[i])
                cudaGraphExecDestroy(ggraph[i]);
            ggraph[i] = nullptr;
            ggraph_counts[i].clear();
        }
        ggraph_aligned = (P % chunk == 0);
        capture_g(0, Av, mv, cfg, P, chunk, ggraph_aligned);
        if (ggraph_aligned)
            capture_g(1, Av, mv, cfg, P, chunk, true);
        ggraph_key = key;
    }

    // The PCG loop of one group: `cols` live right-hand sides (the others start finished).
    void pcg_multi(int cols)
    {
        const BankedView Av = A.view();
        const MasView mv = view_g();
        const PcgConfig cfg = config();
        const int W = gwidth;
        PcgState *S = gst.get();
        std::vector<PcgState> hinit((size_t)W + 1), hs((size_t)W + 1);
        std::memset(hinit.data(), 0, sizeof(PcgState) * hinit.size());
        for (int g = cols; g < W; ++g)
            hinit[g].done = 1;
        cuda_check(cudaMemcpyAsync(S, hinit.data(), sizeof(PcgState) * (W + 1), cudaMemcpyHostToDevice, stream),
                   "state");
        if (wide() && p.wide_tc)
            ensure_tc_storage(mv);
        if (wide())
        {
            run("spmv_residual", 1,
                [&] { launch_spmv_w(SPMV_RESIDUAL, Av, gx.get(), gr.get(), gb.get(), S, red_g(), 0, 0, stream); });
            run("restrict", 0, [&] { return launch_restrict_w(mv, gr.get(), S + W, 0, stream); });
            run("coarse_levels", 0, [&] { return launch_coarse_levels_w(mv, S + W, stream); });
            run("mas_apply", 1, [&] { launch_wide_apply(mv, cfg, 1); });
            run("update_p", 1, [&] { launch_update_p_w(mv, gx.get(), gp.get(), gz.get(), S, 1, stream); });
        }
        else
        {
            run("spmv_residual", 1,
                [&] { launch_spmv_g(SPMV_RESIDUAL, Av, gx.get(), gr.get(), gb.get(), S, red_g(), 0, 0, stream); });
            run("restrict", 0, [&] { return launch_restrict_g(mv, gr.get(), S + W, 0, stream); });
            run("coarse_levels", 0, [&] { return launch_coarse_levels_g(mv, stream); });
            run("mas_apply", 1, [&] { launch_mas_apply_g(mv, gr.get(), gz.get(), S, red_g(), cfg, 1, stream); });
            run("update_p", 1, [&] { launch_update_p_g(mv, gx.get(), gp.get(), gz.get(), S, 1, stream); });
        }
        cuda_check(cudaMemcpyAsync(hs.data(), S, sizeof(PcgState) * (W + 1), cudaMemcpyDeviceToHost, stream), "state");
        cuda_check(cudaStreamSynchronize(stream), "pcg init");
        if (hs[W].error == ERR_TIMEOUT)
            throw Error(ERR_TIMEOUT, "[MAS] a device-side wait timed out.");
        if (hs[W].error == ERR_CUDA)
            throw Error(ERR_CUDA, "[MAS] a kernel's self-check rejected a memory access.");
        for (int g = 0; g < cols; ++g)
            if (hs[g].error == ERR_NONFINITE || std::isnan(hs[g].rz0) || !std::isfinite(hs[g].rz0))
                throw Error(ERR_NONFINITE, "[MAS] Invalid initial residual.");
        const int P = p.true_residual_period;
        const int chunk = p.poll_period;
        const bool graphs = p.graphs && !p.profile;
        if (graphs)
            ensure_graph_g(Av, mv, cfg, P, chunk);
        for (int k0 = 1; k0 <= p.max_iter; k0 += chunk)
        {
            const int k1 = std::min(p.max_iter, k0 + chunk - 1);
            if (graphs)
            {
                const int g = (ggraph_aligned && (k0 + chunk - 1) % P == 0) ? 1 : 0;
                cuda_check(cudaGraphLaunch(ggraph[g], stream), "graph launch");
                for (auto &gc : ggraph_counts[g])
                {
                    kstats[gc.first].second.launches += gc.second;
                    total_launches += gc.second;
                }
            }
            else
                for (int k = k0; k <= k1; ++k)
                    launch_iteration_g(Av, mv, cfg, P, k % P == 0);
            cuda_check(cudaMemcpyAsync(&hs[W], S + W, sizeof(PcgState), cudaMemcpyDeviceToHost, stream), "state");
            cuda_check(cudaStreamSynchronize(stream), "chunk");
            if (hs[W].done)
                break;
        }
        cuda_check(cudaMemcpyAsync(hs.data(), S, sizeof(PcgState) * (W + 1), cudaMemcpyDeviceToHost, stream), "state");
        cuda_check(cudaStreamSynchronize(stream), "pcg");
        if (hs[W].error == ERR_TIMEOUT)
            throw Error(ERR_TIMEOUT, "[MAS] a device-side wait timed out.");
        if (hs[W].error == ERR_CUDA)
            throw Error(ERR_CUDA, "[MAS] a kernel's self-check rejected a memory access.");
        for (int g = 0; g < cols; ++g)
        {
            rhs_iterations.push_back(hs[g].iter);
            rhs_status.push_back(hs[g].status == 0 ? MAS_STATUS_REACH_MAX_ITERATIONS : hs[g].status);
            rhs_error.push_back(hs[g].res_norm);
        }
    }

    // Group width of a several-right-hand-side solve (the rhs_group parameter; automatic: sixteen
    // for more than four right-hand sides with block_dim 3).
    int group_width(int nrhs) const
    {
        if (p.rhs_group == RHS_WIDE && bd == 3)
            return RHS_WIDE;
        if (p.rhs_group == 0 && bd == 3 && nrhs > RHS_GROUP)
            return RHS_WIDE;
        return RHS_GROUP;
    }

    // Column-major B (n x nrhs) -> X; each group of right-hand sides shares every matrix and inverse read.
    void solve_multi(const double *hB, double *hX, int len, int nrhs)
    {
        cuda_check(cudaSetDevice(device), "set device");
        require_factorized(len);
        if (!multi_supported())
        {
            // Each column from x0 = 0 (or the caller's x); the warm-start history is untouched.
            in_multi = true;
            try
            {
                for (int c = 0; c < nrhs; ++c)
                    solve(hB + (size_t)c * n, hX + (size_t)c * n, n);
            }
            catch (...)
            {
                in_multi = false;
                throw;
            }
            in_multi = false;
            return;
        }
        const int W = group_width(nrhs);
        alloc_multi(W);
        for (auto &ks : kstats)
            ks.second = KStat{};
        rhs_iterations.clear();
        rhs_status.clear();
        rhs_error.clear();
        const size_t glen = (size_t)banks * 32 * bd * W;
        auto t0 = std::chrono::steady_clock::now();
        for (int c0 = 0; c0 < nrhs; c0 += W)
        {
            const int cols = std::min(W, nrhs - c0);
            upload_pageable(gio.get(), hB + (size_t)c0 * n, sizeof(double) * (size_t)n * cols);
            run("permute_in", 2, [&] {
                if (wide())
                    launch_permute_in_w(n, V, cols, d_padded.get(), gio.get(), gb.get(), glen, stream);
                else
                    launch_permute_in_g(n, bd, V, cols, d_padded.get(), gio.get(), gb.get(), glen, stream);
            });
            cuda_check(cudaMemsetAsync(gx.get(), 0, gx.bytes(), stream), "memset");
            pcg_multi(cols);
            run("permute_out", 1, [&] {
                if (wide())
                    launch_permute_out_w(n, cols, d_padded.get(), gx.get(), gio.get(), stream);
                else
                    launch_permute_out_g(n, bd, cols, d_padded.get(), gx.get(), gio.get(), stream);
            });
            download_pageable(hX + (size_t)c0 * n, gio.get(), sizeof(double) * (size_t)n * cols);
            collect_profile();
        }
        solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        iterations = rhs_iterations.empty() ? 0 : *std::max_element(rhs_iterations.begin(), rhs_iterations.end());
        residual_norm = rhs_error.empty() ? 0.0 : *std::max_element(rhs_error.begin(), rhs_error.end());
        status = MAS_STATUS_REACH_RELATIVE_TOLERANCE;
        for (int st_ : rhs_status)
            if (st_ == MAS_STATUS_REACH_MAX_ITERATIONS)
                status = MAS_STATUS_REACH_MAX_ITERATIONS;
        last_multi = true;
    }

    // MASSolverImpl::solve (MASSolver.cu:376-409).
    void solve(const double *hb, double *hx, int len)
    {
        cuda_check(cudaSetDevice(device), "set device");
        require_factorized(len);
        last_multi = false;
        if (!hb || !hx)
            throw Error(ERR_INVALID, "[MAS] solve: null vector.");
        cuda_check(cudaMemcpyAsync(io.get(), hb, sizeof(double) * n, cudaMemcpyHostToDevice, stream), "upload b");
        const size_t blen = (size_t)banks * 32 * bd;
        run("permute_in", 2, [&] { launch_permute_in(n, bd, V, d_padded.get(), io.get(), b.get(), blen, stream); });
        if (learned_active())
            warm_start_guess();
        else
        {
            if (p.initial_guess_input)
            {
                cuda_check(cudaMemcpyAsync(io.get(), hx, sizeof(double) * n, cudaMemcpyHostToDevice, stream),
                           "upload x");
                run("permute_in", 2,
                    [&] { launch_permute_in(n, bd, V, d_padded.get(), io.get(), x.get(), blen, stream); });
            }
            else
                cuda_check(cudaMemsetAsync(x.get(), 0, x.bytes(), stream), "memset");
            x0_source = p.initial_guess_input ? "input" : "zero";
        }
        pcg();
        run("permute_out", 1, [&] { launch_permute_out(n, bd, V, d_padded.get(), x.get(), io.get(), stream); });
        cuda_check(cudaMemcpyAsync(hx, io.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, stream), "download x");
        if (learned_active())
            finish_warm_start();
        cuda_check(cudaStreamSynchronize(stream), "solve");
    }

    // ---- Fused batch (mas_solve_batch): this handle's share --------------------------------
    // Solves that can join a fused batch: graphs on, no per-launch profiling, no learned warm
    // start (its prediction pipeline is per handle), at least one iteration.
    bool batch_fusable() const
    {
        return factorized && p.batch_fused && p.graphs && !p.profile && !learned_active() && p.max_iter >= 1;
    }

    // Byte-comparable (a fused batch's kept tables are matched by memcmp): every padding byte zero.
    BatchSystem batch_system()
    {
        BatchSystem s;
        std::memset(&s, 0, sizeof(s));
        const BankedView av = A.view();
        s.A.bd = av.bd;
        s.A.banks = av.banks;
        s.A.slice = av.slice;
        s.A.rowlen = av.rowlen;
        s.A.cols = av.cols;
        s.A.vals = av.vals;
        const MasView mv = mas.view();
        static_assert(sizeof(MasView) == 248, "a MasView member was added: copy it below as well");
        MasView &m = s.mas; // member by member into the zeroed record
        m.bd = mv.bd;
        m.banks = mv.banks;
        m.level_num = mv.level_num;
        m.total_coarse = mv.total_coarse;
        std::copy(mv.coff, mv.coff + MAX_COARSE, m.coff);
        std::copy(mv.mat_offsets, mv.mat_offsets + LEVELS, m.mat_offsets);
        std::copy(mv.mat_counts, mv.mat_counts + LEVELS, m.mat_counts);
        std::copy(mv.cco_nums, mv.cco_nums + MAX_COARSE, m.cco_nums);
        m.storage = mv.storage;
        m.first_iso_bank = mv.first_iso_bank;
        std::copy(mv.real_count, mv.real_count + MAX_COARSE, m.real_count);
        m.n_coarse_active = mv.n_coarse_active;
        m.coarse_active = mv.coarse_active;
        m.inv = mv.inv;
        m.inv_scale = mv.inv_scale;
        m.lcco0 = mv.lcco0;
        m.cco0_base = mv.cco0_base;
        m.cslot = mv.cslot;
        m.parent = mv.parent;
        m.ticket = mv.ticket;
        std::copy(mv.kid_ptr, mv.kid_ptr + MAX_COARSE, m.kid_ptr);
        m.kids = mv.kids;
        m.identity = mv.identity;
        m.rc = mv.rc;
        m.zc = mv.zc;
        const PcgConfig cf = config();
        s.cfg.max_iter = cf.max_iter;
        s.cfg.rel_tol = cf.rel_tol;
        s.cfg.abs_tol = cf.abs_tol;
        s.cfg.use_prec_norm = cf.use_prec_norm;
        s.cfg.check_period = cf.check_period;
        s.cfg.polak_ribiere = cf.polak_ribiere;
        s.cfg.level_num = cf.level_num;
        s.cfg.wait_limit = cf.wait_limit;
        const ReduceBuf rb = red();
        s.red.partials = rb.partials;
        s.red.capacity = rb.capacity;
        s.red.rr_parts = rb.rr_parts;
        s.red.rz_parts = rb.rz_parts;
        s.st = st.get();
        s.x = x.get();
        s.r = r.get();
        s.p = pv.get();
        s.z = z.get();
        s.Ap = Ap.get();
        s.b = b.get();
        return s;
    }

    // Input step of a fused batch solve on this handle's stream: b (and x0) into the padded
    // vectors, as solve / solve_device do.
    void batch_load(const double *src_b, const double *src_x, bool device_pointers, int len)
    {
        cuda_check(cudaSetDevice(device), "set device");
        require_factorized(len);
        if (!src_b || !src_x)
            throw Error(ERR_INVALID, "[MAS] solve: null vector.");
        last_multi = false;
        for (auto &ks : kstats) // per-solve kernel statistics
            ks.second = KStat{};
        keep_stats = false;
        if (device_pointers)
            load_rhs_device(src_b, src_x);
        else
        {
            cuda_check(cudaMemcpyAsync(io.get(), src_b, sizeof(double) * n, cudaMemcpyHostToDevice, stream),
                       "upload b");
            const size_t blen = (size_t)banks * 32 * bd;
            run("permute_in", 2,
                [&] { launch_permute_in(n, bd, V, d_padded.get(), io.get(), b.get(), blen, stream); });
            if (p.initial_guess_input)
            {
                cuda_check(cudaMemcpyAsync(io.get(), src_x, sizeof(double) * n, cudaMemcpyHostToDevice, stream),
                           "upload x");
                run("permute_in", 2,
                    [&] { launch_permute_in(n, bd, V, d_padded.get(), io.get(), x.get(), blen, stream); });
            }
            else
                cuda_check(cudaMemsetAsync(x.get(), 0, x.bytes(), stream), "memset");
        }
        x0_source = p.initial_guess_input ? "input" : "zero";
    }

    // Result step: the final state (as pcg() reads it), then x back to the caller.
    void batch_finish(const PcgState &f, int launched, double ms, double *dst_x, bool device_pointers)
    {
        cuda_check(cudaSetDevice(device), "set device");
        rz0 = f.rz0;
        rr0 = f.rr0;
        solve_ms = ms;
        launched_iterations = launched;
        if (f.error == ERR_TIMEOUT)
            throw Error(ERR_TIMEOUT, "[MAS] a device-side wait timed out.");
        if ((f.error == ERR_NONFINITE && f.iter == 0) || std::isnan(f.rz0) || !std::isfinite(f.rz0))
            throw Error(ERR_NONFINITE, "[MAS] Invalid initial residual.");
        iterations = f.iter;
        residual_norm = f.res_norm;
        status = f.status;
        if (device_pointers)
            run("permute_out", 1, [&] { launch_permute_out(n, bd, V, d_padded.get(), x.get(), dst_x, stream); });
        else
        {
            run("permute_out", 1, [&] { launch_permute_out(n, bd, V, d_padded.get(), x.get(), io.get(), stream); });
            cuda_check(cudaMemcpyAsync(dst_x, io.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, stream),
                       "download x");
        }
        cuda_check(cudaStreamSynchronize(stream), "solve");
    }

    // Launches of a fused batch, counted on one handle of the batch (kernel_launches_total).
    void add_launches(const char *kind, long long k)
    {
        kstats[stat_index(kind)].second.launches += k;
        total_launches += k;
    }

    void solve_device(const double *d_b, double *d_x, int len)
    {
        cuda_check(cudaSetDevice(device), "set device");
        require_factorized(len);
        last_multi = false;
        load_rhs_device(d_b, learned_active() ? nullptr : d_x);
        if (learned_active())
            warm_start_guess();
        else
            x0_source = p.initial_guess_input ? "input" : "zero";
        pcg();
        run("permute_out", 1, [&] { launch_permute_out(n, bd, V, d_padded.get(), x.get(), d_x, stream); });
        if (learned_active())
            finish_warm_start();
        cuda_check(cudaStreamSynchronize(stream), "solve");
    }

    std::string info_json() const
    {
        Json o;
        o.type = Json::Object;
        auto num = [](double v, bool integer) {
            Json j;
            j.type = Json::Number;
            j.num = v;
            j.is_integer = integer;
            return j;
        };
        auto str = [](const std::string &s) {
            Json j;
            j.type = Json::String;
            j.str = s;
            return j;
        };
        auto boolean = [](bool v) {
            Json j;
            j.type = Json::Bool;
            j.b = v;
            return j;
        };
        if (last_multi)
        {
            Json it, stv, er;
            it.type = stv.type = er.type = Json::Array;
            for (size_t i = 0; i < rhs_iterations.size(); ++i)
            {
                it.arr.push_back(num(rhs_iterations[i], true));
                stv.arr.push_back(str(status_string(rhs_status[i])));
                er.arr.push_back(num(rhs_error[i], false));
            }
            o.obj.emplace_back("rhs_iterations", it);
            o.obj.emplace_back("rhs_status", stv);
            o.obj.emplace_back("rhs_error", er);
        }
        o.obj.emplace_back("solver_iter", num(iterations, true));
        o.obj.emplace_back("solver_error", num(residual_norm, false));
        o.obj.emplace_back("solver_status", str(status_string(status)));
        const double ref = p.use_prec_norm ? std::sqrt(std::fabs(rz0)) : std::sqrt(std::fabs(rr0));
        o.obj.emplace_back("relative_residual", num(ref > 0 ? residual_norm / ref : 0.0, false));
        o.obj.emplace_back("precision",
                           str(p.storage == STORE_F64 ? "fp64" : (p.storage == STORE_F32 ? "fp32" : "fp16")));
        o.obj.emplace_back("x0_source", str(x0_source));
        if (p.initial_guess_learned)
        {
            Json ws, cf;
            ws.type = Json::Object;
            cf.type = Json::Array;
            const bool have = ws_predicted && h_ws;
            for (int i = 0; i < WS_BASIS; ++i)
                cf.arr.push_back(num(have ? h_ws->coef[i] : 0.0, false));
            ws.obj.emplace_back("model_loaded", boolean(ws_loaded));
            ws.obj.emplace_back("history", num(hist_count, true));
            ws.obj.emplace_back("predicted", boolean(have));
            ws.obj.emplace_back("coefficients", cf);
            ws.obj.emplace_back("energy", num(have ? h_ws->energy : 0.0, false));
            ws.obj.emplace_back("energy_previous", num(have ? h_ws->energy_prev : 0.0, false));
            ws.obj.emplace_back("fallback", boolean(have && h_ws->fallback));
            ws.obj.emplace_back("rank", num(have ? h_ws->rank : 0, true));
            ws.obj.emplace_back("ms", num(warm_start_ms, false));
            o.obj.emplace_back("warm_start", ws);
        }
        o.obj.emplace_back("ordering", str(ordering_used));
        o.obj.emplace_back("solve_ms", num(solve_ms, false));
        o.obj.emplace_back("factorize_ms", num(factorize_ms, false));
        o.obj.emplace_back("preconditioner_current", boolean(preconditioner_current));
        {
            Json fp;
            fp.type = Json::Object;
            for (const auto &ph : factorize_phases)
                fp.obj.emplace_back(ph.first, num(ph.second, false));
            o.obj.emplace_back("factorize_phases_ms", fp);
        }
        o.obj.emplace_back("launched_iterations", num(launched_iterations, true));
        o.obj.emplace_back("banks", num(banks, true));
        o.obj.emplace_back("coarse_levels", num(mas.level_num, true));
        o.obj.emplace_back("kernel_launches_total", num((double)total_launches, true));
        Json kl, km;
        kl.type = km.type = Json::Object;
        for (const auto &ks : kstats)
        {
            kl.obj.emplace_back(ks.first, num((double)ks.second.launches, true));
            km.obj.emplace_back(ks.first, num(ks.second.ms, false));
        }
        o.obj.emplace_back("kernel_launches", kl);
        if (p.profile)
        {
            o.obj.emplace_back("kernel_ms", km);
            Json tl;
            tl.type = Json::Array;
            for (const auto &t : timeline)
            {
                Json row;
                row.type = Json::Array;
                row.arr.push_back(str(kstats[t.first].first));
                row.arr.push_back(num(t.second.first, false));
                row.arr.push_back(num(t.second.second, false));
                tl.arr.push_back(row);
            }
            o.obj.emplace_back("kernel_timeline", tl);
        }
        o.obj.emplace_back("subdomain_matrices", num(mas.total_mats, true));
        o.obj.emplace_back("coarse_matrices_active", num(mas.n_coarse_active, true));
        o.obj.emplace_back("isolated_banks", num(banks - mas.first_iso_bank, true));
        return o.dump();
    }
};

// ------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------

namespace
{
    template <class F>
    int guarded(mas_solver *h, F &&f)
    {
        try
        {
            f();
            if (h)
                h->last_error.clear();
            return MAS_OK;
        }
        catch (const Error &e)
        {
            if (h)
                h->last_error = e.what();
            else
                g_create_error = e.what();
            return e.code;
        }
        catch (const std::bad_alloc &)
        {
            if (h)
                h->last_error = "[MAS] host allocation failed";
            return ERR_OOM;
        }
        catch (const std::exception &e)
        {
            if (h)
                h->last_error = std::string("[MAS] ") + e.what();
            else
                g_create_error = std::string("[MAS] ") + e.what();
            return ERR_INVALID;
        }
    }

    int create_common(Params p, mas_solver **out)
    {
        *out = nullptr;
        auto *h = new mas_solver();
        h->p = p;
        int rc = guarded(nullptr, [&] { h->init_device(); });
        if (rc != MAS_OK)
        {
            delete h;
            return rc;
        }
        *out = h;
        return MAS_OK;
    }

    // Runs fn(i) for i in [0, count) on up to `workers` host threads.
    template <class F>
    void parallel_for(int count, int workers, F &&fn)
    {
        workers = std::max(1, std::min(workers, count));
        std::atomic<int> next{0};
        auto work = [&] {
            for (int i = next.fetch_add(1); i < count; i = next.fetch_add(1))
                fn(i);
        };
        if (workers <= 1)
        {
            work();
            return;
        }
        std::vector<std::thread> pool;
        pool.reserve((size_t)workers);
        for (int w = 0; w < workers; ++w)
            pool.emplace_back(work);
        for (auto &t : pool)
            t.join();
    }

    // A fused batch: the device copy of the batch's systems, the CTA tables of its unfinished
    // systems, and the stream its launches run on. Kept for reuse while the systems (every
    // pointer, size and PCG setting) stay the same.
    struct FusedBatch
    {
        int device = -1;
        cudaStream_t stream = nullptr;
        std::vector<BatchSystem> host_sys;
        int bd = 0, storage = 0;
        std::vector<int> grids;         // BPH_COUNT CTAs per system (its own launches' grids)
        DevBuf<BatchSystem> sys;
        DevBuf<int4> table;              // the CTA entries of every phase (BatchView::map)
        int4 *h_table = nullptr;         // pinned, 2 slots of the same size
        DevBuf<PcgState> states;         // 2 slots of count gathered states
        PcgState *h_states = nullptr;    // pinned, 2 slots
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr}; // start, end, two chunk slots

        int count() const { return (int)host_sys.size(); }
        size_t table_len() const
        {
            size_t t = 0;
            for (int g : grids)
                t += (size_t)g;
            return t > 0 ? t : 1;
        }

        ~FusedBatch()
        {
            if (device >= 0)
                cudaSetDevice(device);
            if (stream)
                cudaStreamSynchronize(stream);
            for (auto &e : ev)
                if (e)
                    cudaEventDestroy(e);
            if (h_states)
                cudaFreeHost(h_states);
            if (h_table)
                cudaFreeHost(h_table);
            sys.reset();
            table.reset();
            states.reset();
            if (stream)
                cudaStreamDestroy(stream);
        }

        bool same(int dev, const std::vector<BatchSystem> &s, const std::vector<int> &g) const
        {
            return dev == device && s.size() == host_sys.size() && g == grids &&
                   std::memcmp(s.data(), host_sys.data(), s.size() * sizeof(BatchSystem)) == 0;
        }

        void build(int dev, std::vector<BatchSystem> s, std::vector<int> g, int bd_, int storage_)
        {
            device = dev;
            host_sys = std::move(s);
            grids = std::move(g);
            bd = bd_;
            storage = storage_;
            const int c = count();
            cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "batch stream");
            for (auto &e : ev)
                cuda_check(cudaEventCreate(&e), "event");
            cuda_check(cudaMallocHost(&h_states, sizeof(PcgState) * 2 * (size_t)c), "pinned states");
            cuda_check(cudaMallocHost(&h_table, sizeof(int4) * 2 * table_len()), "pinned tables");
            sys.alloc((size_t)c, "batch systems");
            table.alloc(table_len(), "batch tables");
            states.alloc((size_t)2 * c, "batch states");
            cuda_check(cudaMemcpyAsync(sys.get(), host_sys.data(), sizeof(BatchSystem) * (size_t)c,
                                       cudaMemcpyHostToDevice, stream),
                       "upload batch");
            cuda_check(cudaStreamSynchronize(stream), "upload batch");
        }

        // Launch entries of the systems with active[k] set (each system's CTAs in order, the
        // systems in batch order), written into pinned slot `slot` and copied (in stream order,
        // after every earlier launch) to the device table; returns the view and the CTA totals
        // per phase.
        BatchView upload_active(const std::vector<char> &active, int slot, int (&totals)[BPH_COUNT])
        {
            const int c = count();
            int4 *h = h_table + (size_t)slot * table_len();
            BatchView v{sys.get(), table.get(), {}, c};
            size_t e = 0;
            for (int ph = 0; ph < BPH_COUNT; ++ph)
            {
                v.off[ph] = (int)e;
                for (int k = 0; k < c; ++k)
                {
                    if (!active[(size_t)k])
                        continue;
                    const int g = grids[(size_t)k * BPH_COUNT + ph];
                    for (int b = 0; b < g; ++b)
                        h[e++] = make_int4(k, b, g, 0);
                }
                totals[ph] = (int)e - v.off[ph];
            }
            if (e > 0)
                cuda_check(cudaMemcpyAsync(table.get(), h, sizeof(int4) * e, cudaMemcpyHostToDevice, stream),
                           "upload tables");
            return v;
        }

        // Every system (state reset and gather launches).
        BatchView all() const { return BatchView{sys.get(), nullptr, {}, count()}; }

        // One batched PCG iteration (the launch order of mas_solver::launch_iteration); returns
        // the kernels launched.
        long long iteration(const BatchView &v, const int (&totals)[BPH_COUNT], int P, bool residual)
        {
            long long k = 0;
            auto counted = [&k](int total) { k += total > 0 ? 1 : 0; };
            launch_spmv_batch(SPMV_PAP, v, bd, totals[BPH_SPMV], 1, 0, stream);
            counted(totals[BPH_SPMV]);
            launch_update_xr_batch(v, bd, totals[BPH_UPDATE_XR], P, stream);
            counted(totals[BPH_UPDATE_XR]);
            if (residual)
            {
                launch_spmv_batch(SPMV_RESIDUAL, v, bd, totals[BPH_SPMV], 1, P, stream);
                counted(totals[BPH_SPMV]);
                launch_restrict_batch(v, bd, totals[BPH_RESTRICT], P, stream);
                counted(totals[BPH_RESTRICT]);
            }
            launch_coarse_levels_batch(v, bd, totals[BPH_COARSE], stream);
            counted(totals[BPH_COARSE]);
            launch_mas_apply_batch(v, bd, storage, totals[BPH_APPLY], 2, stream);
            counted(totals[BPH_APPLY]);
            launch_update_p_batch(v, bd, totals[BPH_UPDATE_P], 0, stream);
            counted(totals[BPH_UPDATE_P]);
            return k;
        }
    };

    std::mutex g_fused_mu;
    std::vector<std::unique_ptr<FusedBatch>> g_fused; // most recently used last
    constexpr size_t FUSED_CACHE = 16;

    // One fused group on its own stream: systems sys[k] (handles hs[k]), their ready events;
    // writes each system's final state into out[k], the group's elapsed ms and launched
    // iterations. The loop is pcg()'s: initial residual and apply, then chunks of poll_period
    // iterations with the host reading all states one chunk behind and dropping finished
    // systems from the next chunk's launch tables.
    void run_fused_group(int dev, const std::vector<mas_solver *> &hs, std::vector<BatchSystem> sys,
                         std::vector<int> grids, const std::vector<cudaEvent_t> &ready, std::vector<PcgState> &out,
                         double &ms_out, int &launched_out)
    {
        cuda_check(cudaSetDevice(dev), "set device");
        const Params &p0 = hs[0]->p;
        const int P = p0.true_residual_period, chunk = p0.poll_period;
        const int c = (int)hs.size();
        int max_iter = 1;
        for (const mas_solver *h : hs)
            max_iter = std::max(max_iter, h->p.max_iter);
        set_spmv_unroll(p0.spmv_unroll);
        set_chained_launch(p0.chained);
        set_apply_items_per_warp(p0.apply_ipw);
        std::unique_ptr<FusedBatch> fb;
        {
            std::lock_guard<std::mutex> lock(g_fused_mu);
            for (size_t i = 0; i < g_fused.size(); ++i)
                if (g_fused[i]->same(dev, sys, grids))
                {
                    fb = std::move(g_fused[i]);
                    g_fused.erase(g_fused.begin() + (long)i);
                    break;
                }
        }
        if (!fb)
        {
            fb = std::make_unique<FusedBatch>();
            fb->build(dev, std::move(sys), std::move(grids), hs[0]->bd, hs[0]->mas.storage);
        }
        FusedBatch &F = *fb;
        cudaStream_t s = F.stream;
        for (cudaEvent_t e : ready)
            cuda_check(cudaStreamWaitEvent(s, e, 0), "batch wait");
        cuda_check(cudaEventRecord(F.ev[0], s), "event");
        long long launches = 0;
        // pcg(): r = b - A x, rr0, the level-0 restriction, z = M^-1 r (rz0), p = z.
        std::vector<char> active((size_t)c, 1);
        int totals[BPH_COUNT];
        int tslot = 0;
        BatchView v = F.upload_active(active, tslot, totals);
        launch_init_states_batch(F.all(), s);
        launch_spmv_batch(SPMV_RESIDUAL, v, F.bd, totals[BPH_SPMV], 0, 0, s);
        launch_restrict_batch(v, F.bd, totals[BPH_RESTRICT], 0, s);
        launch_coarse_levels_batch(v, F.bd, totals[BPH_COARSE], s);
        launch_mas_apply_batch(v, F.bd, F.storage, totals[BPH_APPLY], 1, s);
        launch_update_p_batch(v, F.bd, totals[BPH_UPDATE_P], 1, s);
        launches += 1;
        for (int ph : {BPH_SPMV, BPH_RESTRICT, BPH_COARSE, BPH_APPLY, BPH_UPDATE_P})
            launches += totals[ph] > 0 ? 1 : 0;
        int launched = 0, pending = -1, flip = 0;
        bool stop = false;
        for (int k0 = 1; k0 <= max_iter && !stop; k0 += chunk)
        {
            for (int k = k0; k < k0 + chunk; ++k)
                launches += F.iteration(v, totals, P, k % P == 0);
            launched = std::min(max_iter, k0 + chunk - 1);
            const int slot = (flip++) & 1;
            launch_gather_states_batch(F.all(), F.states.get() + (size_t)slot * c, s);
            launches += 1;
            cuda_check(cudaMemcpyAsync(F.h_states + (size_t)slot * c, F.states.get() + (size_t)slot * c,
                                       sizeof(PcgState) * (size_t)c, cudaMemcpyDeviceToHost, s),
                       "states");
            cuda_check(cudaEventRecord(F.ev[2 + slot], s), "event");
            // The previous chunk's states (read while this chunk runs): stop when every system
            // is done, else drop the finished ones from the next chunk's tables.
            if (pending >= 0)
            {
                cuda_check(cudaEventSynchronize(F.ev[2 + pending]), "chunk");
                bool changed = false, any = false;
                for (int k = 0; k < c; ++k)
                {
                    const bool on = F.h_states[(size_t)pending * c + k].done == 0;
                    changed = changed || (on != (active[(size_t)k] != 0));
                    active[(size_t)k] = on ? 1 : 0;
                    any = any || on;
                }
                stop = !any;
                if (changed && !stop)
                {
                    // The pinned slot written two updates ago was copied before launches whose
                    // chunk event has been waited on since.
                    tslot ^= 1;
                    v = F.upload_active(active, tslot, totals);
                }
            }
            pending = slot;
        }
        cuda_check(cudaEventRecord(F.ev[1], s), "event");
        launch_gather_states_batch(F.all(), F.states.get(), s);
        launches += 1;
        cuda_check(cudaMemcpyAsync(F.h_states, F.states.get(), sizeof(PcgState) * (size_t)c, cudaMemcpyDeviceToHost, s),
                   "states");
        cuda_check(cudaStreamSynchronize(s), "batch");
        hs[0]->add_launches("batch", launches);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, F.ev[0], F.ev[1]);
        out.assign(F.h_states, F.h_states + c);
        ms_out = ms;
        launched_out = launched;
        std::lock_guard<std::mutex> lock(g_fused_mu);
        g_fused.push_back(std::move(fb));
        if (g_fused.size() > FUSED_CACHE)
            g_fused.erase(g_fused.begin());
    }

    // mas_solve_batch with one launch per PCG phase for each group of unfinished systems:
    // per-handle input steps on the handles' own streams (host threads), the groups' batched PCG
    // on their own streams (one host thread each), then the per-handle result steps. The systems
    // are sorted by size and cut into batch_groups runs of about equal work (dof^(4/3) each), so
    // a group's systems finish after similar iteration counts and the groups' phase boundaries
    // overlap on the GPU. Each system's kernels run the same bodies over the same CTA
    // coordinates as in its own solve, so its iterates, iteration count and status are those of
    // mas_solve bit for bit. Returns false (nothing done) when the handles cannot be fused.
    bool solve_fused(mas_solver *const *handles, int count, const double *const *b, double *const *x, const int *n,
                     bool device_pointers, int workers, std::vector<int> &rc)
    {
        const Params &p0 = handles[0]->p;
        for (int i = 0; i < count; ++i)
        {
            const mas_solver *h = handles[i];
            if (!h->batch_fusable() || h->device != handles[0]->device || h->bd != handles[0]->bd ||
                h->mas.storage != handles[0]->mas.storage || h->p.true_residual_period != p0.true_residual_period ||
                h->p.poll_period != p0.poll_period || h->p.spmv_unroll != p0.spmv_unroll ||
                h->p.batch_groups != p0.batch_groups || h->p.chained != p0.chained ||
                h->p.apply_ipw != p0.apply_ipw)
                return false;
        }
        const int dev = handles[0]->device;
        cuda_check(cudaSetDevice(dev), "set device");
        set_apply_items_per_warp(p0.apply_ipw); // the apply grids below are the handles' own
        // Input steps; systems whose input is rejected keep their error and leave the batch.
        std::vector<cudaEvent_t> ready((size_t)count, nullptr);
        parallel_for(count, workers, [&](int i) {
            mas_solver *h = handles[i];
            rc[(size_t)i] = guarded(h, [&] {
                h->batch_load(b[i], x[i], device_pointers, n[i]);
                ready[(size_t)i] = h->pool_event();
                cuda_check(cudaEventRecord(ready[(size_t)i], h->stream), "event");
            });
        });
        std::vector<int> live;
        for (int i = 0; i < count; ++i)
            if (rc[(size_t)i] == MAS_OK)
                live.push_back(i);
        // The ready events are pool events: free them once the groups have waited on them.
        struct FreeEvents
        {
            mas_solver *const *h;
            int count;
            ~FreeEvents()
            {
                for (int i = 0; i < count; ++i)
                    h[i]->ev_used = 0;
            }
        } free_events{handles, count};
        if (live.empty())
            return true;
        // Groups: live systems by size, cut into runs of about equal work.
        std::sort(live.begin(), live.end(), [&](int a, int c2) {
            return handles[a]->n != handles[c2]->n ? handles[a]->n > handles[c2]->n : a < c2;
        });
        const int G = std::max(1, std::min((int)live.size(), p0.batch_groups > 0 ? p0.batch_groups : 1));
        std::vector<double> cost(live.size());
        double total = 0.0;
        for (size_t k = 0; k < live.size(); ++k)
            total += (cost[k] = std::pow((double)handles[live[k]]->n, 4.0 / 3.0));
        std::vector<std::vector<int>> groups;
        double acc = 0.0;
        for (size_t k = 0; k < live.size(); ++k)
        {
            const int g = std::min(G - 1, (int)(acc / total * G));
            while ((int)groups.size() <= g)
                groups.emplace_back();
            groups[(size_t)g].push_back(live[k]);
            acc += cost[k];
        }
        groups.erase(std::remove_if(groups.begin(), groups.end(), [](const std::vector<int> &g) { return g.empty(); }),
                     groups.end());
        struct GroupRun
        {
            std::vector<mas_solver *> hs;
            std::vector<BatchSystem> sys;
            std::vector<int> grids;
            std::vector<cudaEvent_t> ready;
            std::vector<PcgState> out;
            double ms = 0.0;
            int launched = 0;
            int rc = MAS_OK;
            std::string err;
        };
        std::vector<GroupRun> runs(groups.size());
        for (size_t gi = 0; gi < groups.size(); ++gi)
        {
            GroupRun &R = runs[gi];
            for (int i : groups[gi])
            {
                mas_solver *h = handles[i];
                R.hs.push_back(h);
                R.ready.push_back(ready[(size_t)i]);
                R.sys.push_back(h->batch_system());
                const BatchSystem &s = R.sys.back();
                const int g[BPH_COUNT] = {spmv_grid(s.A),         update_xr_grid(s.mas), restrict_grid(s.mas),
                                          coarse_levels_grid(s.mas), mas_apply_grid(s.mas), update_p_grid(s.mas)};
                if (g[BPH_SPMV] > s.red.capacity || g[BPH_UPDATE_XR] > s.red.capacity ||
                    g[BPH_APPLY] > s.red.capacity)
                    throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
                R.grids.insert(R.grids.end(), g, g + BPH_COUNT);
            }
        }
        parallel_for((int)runs.size(), (int)runs.size(), [&](int gi) {
            GroupRun &R = runs[(size_t)gi];
            try
            {
                run_fused_group(dev, R.hs, R.sys, R.grids, R.ready, R.out, R.ms, R.launched);
            }
            catch (const Error &e)
            {
                R.rc = e.code;
                R.err = e.what();
            }
            catch (const std::exception &e)
            {
                R.rc = ERR_INVALID;
                R.err = std::string("[MAS] ") + e.what();
            }
        });
        // Result steps.
        std::vector<std::pair<int, int>> work; // (group, position)
        for (size_t gi = 0; gi < runs.size(); ++gi)
            for (size_t k = 0; k < runs[gi].hs.size(); ++k)
                work.push_back({(int)gi, (int)k});
        parallel_for((int)work.size(), workers, [&](int w) {
            const GroupRun &R = runs[(size_t)work[(size_t)w].first];
            const int k = work[(size_t)w].second;
            const int i = groups[(size_t)work[(size_t)w].first][(size_t)k];
            mas_solver *h = handles[i];
            if (R.rc != MAS_OK)
            {
                h->last_error = R.err;
                rc[(size_t)i] = R.rc;
                return;
            }
            rc[(size_t)i] = guarded(h, [&] { h->batch_finish(R.out[(size_t)k], R.launched, R.ms, x[i], device_pointers); });
        });
        return true;
    }
} // namespace

extern "C" int mas_create(const char *solver, const char *precond, mas_solver **out)
{
    (void)precond;
    if (!out)
        return MAS_ERR_INVALID;
    *out = nullptr;
    if (!solver || std::strcmp(solver, "MAS") != 0)
    {
        g_create_error = std::string("[MAS] Unknown solver ") + (solver ? solver : "(null)") + "; this library provides \"MAS\".";
        return MAS_ERR_INVALID;
    }
    g_create_error.clear();
    return create_common(Params{}, out);
}

extern "C" int mas_create_json(const char *params_json, int strict_validation, mas_solver **out)
{
    if (!out)
        return MAS_ERR_INVALID;
    *out = nullptr;
    Params p;
    // Spec defaults injected by Solver::create(json) (linear-solver-spec.json:481-509).
    p.max_iter = 10000;
    p.rel_tol = 1e-4;
    p.abs_tol = 1e-8;
    p.lazy = true;
    p.block_dim = 1;
    p.use_prec_norm = false;
    int rc = guarded(nullptr, [&] {
        Json j = Json::parse(params_json ? params_json : "{}");
        if (j.type != Json::Object)
            throw Error(ERR_INVALID, "[MAS] invalid input json: parameters must be an object");
        if (auto *s = j.find("solver"))
        {
            if (s->type != Json::String || s->str != "MAS")
                throw Error(ERR_INVALID, "[MAS] invalid input json: this library provides only solver \"MAS\"");
        }
        if (strict_validation)
            for (const auto &kv : j.obj)
                if (kv.first != "solver" && kv.first != "precond" && kv.first != "MAS")
                    throw Error(ERR_INVALID, "[MAS] invalid input json: unknown key /" + kv.first);
        if (auto *m = j.find("MAS"))
            if (m->type != Json::Null)
                apply_mas_params(p, *m, strict_validation != 0);
    });
    if (rc != MAS_OK)
        return rc;
    g_create_error.clear();
    return create_common(p, out);
}

extern "C" void mas_destroy(mas_solver *h)
{
    delete h;
}

extern "C" int mas_set_parameters(mas_solver *h, const char *params_json)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        Json j = Json::parse(params_json ? params_json : "{}");
        const Json *m = j.find("MAS");
        if (!m)
            return; // MASSolver::set_parameters returns silently (MASSolver.cu:607-611)
        apply_mas_params(h->p, *m, false);
    });
}

extern "C" int mas_get_info(const mas_solver *h, char *buf, size_t cap, size_t *needed)
{
    if (!h)
        return MAS_ERR_INVALID;
    const std::string s = h->info_json();
    if (needed)
        *needed = s.size() + 1;
    if (buf && cap > 0)
    {
        const size_t k = std::min(cap - 1, s.size());
        std::memcpy(buf, s.data(), k);
        buf[k] = '\0';
    }
    return MAS_OK;
}

extern "C" const char *mas_name(void)
{
    return "MAS";
}

extern "C" int mas_analyze_pattern(mas_solver *h, int n, const int *outer, const int *inner, int nnz, int precond_num)
{
    (void)precond_num;
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        if (n < 0 || (n > 0 && (!outer || !inner)) || nnz < 0)
            throw Error(ERR_INVALID, "[MAS] analyze_pattern: invalid matrix arguments.");
    });
}

extern "C" int mas_set_positions(mas_solver *h, const double *xyz, int nverts)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        if (nverts < 0 || (nverts > 0 && !xyz))
            throw Error(ERR_INVALID, "[MAS] set_positions: invalid arguments.");
        h->positions.assign(xyz, xyz + (size_t)nverts * 3);
        ++h->positions_version;
        h->padded.clear(); // a new geometry invalidates a lazily kept ordering
    });
}

extern "C" int mas_set_warm_start_model(mas_solver *h, const float *params, long long count)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] { h->set_warm_start_model(params, count); });
}

extern "C" int mas_reset_warm_start(mas_solver *h)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] { h->hist_count = 0; });
}

extern "C" int mas_debug_warm_start(mas_solver *h, const double *b, const double *history, int nhist, double *c_out,
                                    double *x0_out, float *features_out, double *state_out)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] { h->debug_warm_start(b, history, nhist, c_out, x0_out, features_out, state_out); });
}

extern "C" int mas_factorize_csc(mas_solver *h, int n, const int *outer, const int *inner, const double *vals, int nnz)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] { h->factorize(n, outer, inner, vals, nnz); });
}

extern "C" int mas_factorize_values(mas_solver *h, const double *vals, int nnz)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] { h->factorize(h->n, nullptr, nullptr, vals, nnz, true); });
}

extern "C" int mas_solve(mas_solver *h, const double *b, double *x, int n)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] { h->solve(b, x, n); });
}

extern "C" int mas_solve_multi(mas_solver *h, const double *B, double *X, int n, int nrhs)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        if (nrhs < 0)
            throw Error(ERR_INVALID, "[MAS] solve_multi: nrhs must be >= 0");
        if (nrhs > 0)
            h->solve_multi(B, X, n, nrhs);
    });
}

extern "C" int mas_solve_batch(mas_solver *const *handles, int count, const double *const *b, double *const *x,
                               const int *n, int device_pointers, int threads, int *statuses)
{
    if (count < 0 || (count > 0 && (!handles || !b || !x || !n)))
        return MAS_ERR_INVALID;
    for (int i = 0; i < count; ++i)
        if (!handles[i])
            return MAS_ERR_INVALID;
    for (int i = 0; i < count; ++i)
        for (int j = i + 1; j < count; ++j)
            if (handles[i] == handles[j])
            {
                handles[i]->last_error = "[MAS] solve_batch: the same handle appears twice.";
                return MAS_ERR_INVALID;
            }
    int workers = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    workers = std::max(1, std::min({workers, count, 64}));
    std::vector<int> rc((size_t)count, MAS_OK);
    bool fused = false;
    if (count > 0)
    {
        auto fail_all = [&](int code, const std::string &msg) {
            fused = true;
            for (int i = 0; i < count; ++i)
                if (rc[(size_t)i] == MAS_OK)
                {
                    rc[(size_t)i] = code;
                    handles[i]->last_error = msg;
                }
        };
        try
        {
            fused = solve_fused(handles, count, b, x, n, device_pointers != 0, workers, rc);
        }
        catch (const Error &e)
        {
            fail_all(e.code, e.what());
        }
        catch (const std::exception &e)
        {
            fail_all(ERR_INVALID, std::string("[MAS] ") + e.what());
        }
    }
    // Otherwise one CUDA stream per system, driven by a pool of host threads.
    if (!fused)
        parallel_for(count, workers, [&](int i) {
            mas_solver *h = handles[i];
            rc[(size_t)i] = guarded(h, [&] {
                if (device_pointers)
                    h->solve_device(b[i], x[i], n[i]);
                else
                    h->solve(b[i], x[i], n[i]);
            });
        });
    int first = MAS_OK;
    for (int i = 0; i < count; ++i)
    {
        if (statuses)
            statuses[i] = rc[(size_t)i];
        if (first == MAS_OK && rc[(size_t)i] != MAS_OK)
            first = rc[(size_t)i];
    }
    return first;
}

extern "C" int mas_solve_device(mas_solver *h, const double *d_b, double *d_x, int n)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] { h->solve_device(d_b, d_x, n); });
}

extern "C" int mas_set_stream(mas_solver *h, void *stream)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        cuda_check(cudaStreamSynchronize(h->stream), "stream switch");
        h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
    });
}

extern "C" int mas_spmv_dot_noalloc(mas_solver *h, const double *d_x, double *d_y, double *d_dot, int len,
                                    void *stream)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        if (!h->factorized)
            throw Error(ERR_NOT_FACTORIZED, "[MAS] spmv_dot_noalloc: call factorize first.");
        if (len != h->banks * 32 * h->bd)
            throw Error(ERR_INVALID, "[MAS] spmv_dot_noalloc: len must be nodes * block_dim = " +
                                         std::to_string(h->banks * 32 * h->bd) + ".");
        if (!d_x || !d_y || !d_dot)
            throw Error(ERR_INVALID, "[MAS] spmv_dot_noalloc: null device pointer.");
        // The kernel reads x while other warps write y (and x . y into *d_dot): the three buffers
        // must not overlap, or y and the dot come out wrong without any error.
        const uintptr_t x0 = reinterpret_cast<uintptr_t>(d_x), y0 = reinterpret_cast<uintptr_t>(d_y);
        const uintptr_t bytes = sizeof(double) * (uintptr_t)len, dot = reinterpret_cast<uintptr_t>(d_dot);
        auto inside = [](uintptr_t p, uintptr_t lo, uintptr_t nbytes) { return p + sizeof(double) > lo && p < lo + nbytes; };
        if ((x0 < y0 + bytes && y0 < x0 + bytes) || inside(dot, x0, bytes) || inside(dot, y0, bytes))
            throw Error(ERR_INVALID, "[MAS] spmv_dot_noalloc: d_x, d_y and d_dot must not overlap.");
        cuda_check(cudaSetDevice(h->device), "set device");
        launch_spmv_dot_noalloc(h->A.view(), d_x, d_y, d_dot, stream ? static_cast<cudaStream_t>(stream) : h->stream);
    });
}

extern "C" int mas_ws_trainer_add_sample(mas_ws_trainer *t, mas_solver *h, const double *b, const double *history,
                                         int nhist, const double *x_exact, int n)
{
    if (!h || !t)
        return MAS_ERR_INVALID;
    const int rc = guarded(h, [&] { h->collect_training_sample(*t, b, history, nhist, x_exact, n); });
    t->last_error = h->last_error;
    return rc;
}

extern "C" int mas_debug_fail_allocation(long long after)
{
    set_alloc_failure(after);
    return MAS_OK;
}

extern "C" const char *mas_last_error(const mas_solver *h)
{
    if (!h)
        return g_create_error.c_str();
    return h->last_error.c_str();
}

extern "C" int mas_get_sizes(const mas_solver *h, int *sizes)
{
    if (!h || !sizes)
        return MAS_ERR_INVALID;
    sizes[0] = h->n;
    sizes[1] = h->bd;
    sizes[2] = h->V;
    sizes[3] = h->banks;
    sizes[4] = h->banks * 32;
    sizes[5] = h->A.nnzb;
    sizes[6] = h->mas.level_num;
    sizes[7] = h->mas.total_mats;
    for (int i = 0; i < 4; ++i)
        sizes[8 + i] = h->mas.cco_nums[i];
    return MAS_OK;
}

extern "C" int mas_get_ordering(const mas_solver *h, int *padded, int V)
{
    if (!h || !padded || V != (int)h->padded.size())
        return MAS_ERR_INVALID;
    std::memcpy(padded, h->padded.data(), sizeof(int) * V);
    return MAS_OK;
}

extern "C" int mas_order_blocks(int n, const int *outer, const int *inner, int block_dim, const double *xyz,
                                const char *mode, int *padded, int *banks)
{
    if (n <= 0 || !outer || !inner || !padded || !banks || block_dim < 1 || block_dim > 3 || !mode)
        return MAS_ERR_INVALID;
    try
    {
        const int V = (n + block_dim - 1) / block_dim;
        bool pattern_ok = false;
        pattern_hash(n, outer, inner, outer[n], &pattern_ok);
        if (!pattern_ok)
            return MAS_ERR_INVALID;
        std::vector<uint8_t> iso = isolated_blocks(n, outer, inner, block_dim);
        std::vector<int> p;
        const std::string m = mode;
        if (m == "morton")
        {
            if (!xyz)
                return MAS_ERR_INVALID;
            p = morton_padded(xyz, V, iso, banks);
        }
        else if (m == "graph")
            p = graph_padded(n, outer, inner, block_dim, iso, banks);
        else if (m == "natural")
            p = natural_padded(V, banks);
        else
            return MAS_ERR_INVALID;
        std::memcpy(padded, p.data(), sizeof(int) * V);
        return MAS_OK;
    }
    catch (...)
    {
        return MAS_ERR_INVALID;
    }
}

extern "C" int mas_get_coarse_map(const mas_solver *h, int *map, int nodes)
{
    if (!h || !map || !h->factorized || nodes != h->banks * 32)
        return MAS_ERR_INVALID;
    auto *hh = const_cast<mas_solver *>(h);
    return guarded(hh, [&] {
        cuda_check(cudaSetDevice(h->device), "set device");
        cuda_check(cudaMemcpy(map, h->mas.map.get(), sizeof(int) * (size_t)nodes * 4, cudaMemcpyDeviceToHost), "map");
    });
}

namespace
{
    // IEEE binary16 bit pattern -> value.
    double half_bits_to_double(uint16_t h)
    {
        const int sign = h >> 15, e = (h >> 10) & 31, m = h & 1023;
        double v;
        if (e == 0)
            v = std::ldexp((double)m, -24);
        else if (e == 31)
            v = m ? std::numeric_limits<double>::quiet_NaN() : std::numeric_limits<double>::infinity();
        else
            v = std::ldexp((double)(m + 1024), e - 25);
        return sign ? -v : v;
    }
} // namespace

extern "C" int mas_get_inverses(const mas_solver *h, double *out, size_t count)
{
    if (!h || !out || !h->factorized)
        return MAS_ERR_INVALID;
    const int bd = h->bd;
    const int N = 32 * bd;
    const size_t S = (size_t)N * (N + 1) / 2;
    if (count != S * h->mas.total_mats)
        return MAS_ERR_INVALID;
    auto *hh = const_cast<mas_solver *>(h);
    return guarded(hh, [&] {
        cuda_check(cudaSetDevice(h->device), "set device");
        const int storage = h->mas.storage;
        const size_t Ss = (size_t)inv_stride(bd, storage); // stored values per matrix
        const size_t stored = Ss * h->mas.total_mats;
        std::vector<double> tp(stored);
        if (storage == STORE_F32)
        {
            std::vector<float> f(stored);
            cuda_check(cudaMemcpy(f.data(), h->mas.inv32.get(), sizeof(float) * stored, cudaMemcpyDeviceToHost), "inv");
            for (size_t i = 0; i < stored; ++i)
                tp[i] = f[i];
        }
        else if (storage == STORE_F16)
        {
            std::vector<uint16_t> f(stored);
            std::vector<double> sc((size_t)h->mas.total_mats);
            cuda_check(cudaMemcpy(f.data(), h->mas.inv16.get(), sizeof(uint16_t) * stored, cudaMemcpyDeviceToHost),
                       "inv");
            cuda_check(cudaMemcpy(sc.data(), h->mas.inv_scale.get(), sizeof(double) * sc.size(),
                                  cudaMemcpyDeviceToHost),
                       "inv scale");
            for (size_t i = 0; i < stored; ++i)
                tp[i] = half_bits_to_double(f[i]) * sc[i / Ss];
        }
        else
            cuda_check(cudaMemcpy(tp.data(), h->mas.inv64.get(), sizeof(double) * stored, cudaMemcpyDeviceToHost),
                       "inv");
        for (int m = 0; m < h->mas.total_mats; ++m)
            for (int i = 0; i < N; ++i)
                for (int j = i; j < N; ++j)
                    out[(size_t)m * S + (size_t)i * N - (size_t)i * (i + 1) / 2 + j] =
                        tp[(size_t)m * Ss +
                           (storage == STORE_F16 ? mma16_index(bd, i, j) : tile_packed_index(bd, i, j))];
    });
}

extern "C" int mas_debug_spmv(mas_solver *h, const double *xin, double *y, int len)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        cuda_check(cudaSetDevice(h->device), "set device");
        if (!h->factorized || len != h->banks * 32 * h->bd)
            throw Error(ERR_NOT_FACTORIZED, "[MAS] debug_spmv: size mismatch.");
        cuda_check(cudaMemcpyAsync(h->x.get(), xin, sizeof(double) * len, cudaMemcpyHostToDevice, h->stream), "x");
        launch_spmv(SPMV_PLAIN, h->A.view(), h->x.get(), h->Ap.get(), nullptr, nullptr, h->red(), 0, 0, h->stream);
        cuda_check(cudaMemcpyAsync(y, h->Ap.get(), sizeof(double) * len, cudaMemcpyDeviceToHost, h->stream), "y");
        cuda_check(cudaStreamSynchronize(h->stream), "spmv");
    });
}

extern "C" int mas_debug_apply(mas_solver *h, const double *rin, double *zout, int len)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        cuda_check(cudaSetDevice(h->device), "set device");
        if (!h->factorized || len != h->banks * 32 * h->bd)
            throw Error(ERR_NOT_FACTORIZED, "[MAS] debug_apply: size mismatch.");
        cuda_check(cudaMemcpyAsync(h->r.get(), rin, sizeof(double) * len, cudaMemcpyHostToDevice, h->stream), "r");
        const MasView mv = h->mas.view();
        launch_restrict(mv, h->r.get(), nullptr, 0, h->stream);
        launch_coarse_levels(mv, nullptr, h->stream);
        launch_mas_apply(mv, h->r.get(), h->z.get(), nullptr, h->red(), h->config(), 0, h->stream);
        launch_prolong(mv, h->z.get(), h->Ap.get(), h->stream);
        cuda_check(cudaMemcpyAsync(zout, h->Ap.get(), sizeof(double) * len, cudaMemcpyDeviceToHost, h->stream), "z");
        cuda_check(cudaStreamSynchronize(h->stream), "apply");
    });
}

// Test hooks of the several-right-hand-side kernels (padded, interleaved vectors of
// RHS_GROUP columns): z = M^-1 r, and y = A x.
extern "C" int mas_debug_apply_multi(mas_solver *h, const double *rin, double *zout, int len)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        cuda_check(cudaSetDevice(h->device), "set device");
        if (!h->multi_supported() || len != h->banks * 32 * h->bd * RHS_GROUP)
            throw Error(ERR_NOT_FACTORIZED, "[MAS] debug_apply_multi: size mismatch or not fp16.");
        h->alloc_multi();
        PcgState hinit[RHS_GROUP + 1];
        std::memset(hinit, 0, sizeof(hinit));
        cuda_check(cudaMemcpyAsync(h->gst.get(), hinit, sizeof(hinit), cudaMemcpyHostToDevice, h->stream), "state");
        cuda_check(cudaMemcpyAsync(h->gr.get(), rin, sizeof(double) * len, cudaMemcpyHostToDevice, h->stream), "r");
        const MasView mv = h->view_g();
        launch_restrict_g(mv, h->gr.get(), h->gst.get() + RHS_GROUP, 0, h->stream);
        launch_coarse_levels_g(mv, h->stream);
        launch_mas_apply_g(mv, h->gr.get(), h->gz.get(), h->gst.get(), h->red_g(), h->config(), 1, h->stream);
        launch_update_p_g(mv, h->gx.get(), h->gp.get(), h->gz.get(), h->gst.get(), 1, h->stream);
        cuda_check(cudaMemcpyAsync(zout, h->gp.get(), sizeof(double) * len, cudaMemcpyDeviceToHost, h->stream), "z");
        cuda_check(cudaStreamSynchronize(h->stream), "apply");
    });
}

extern "C" int mas_debug_spmv_multi(mas_solver *h, const double *xin, double *yout, int len)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        cuda_check(cudaSetDevice(h->device), "set device");
        if (!h->multi_supported() || len != h->banks * 32 * h->bd * RHS_GROUP)
            throw Error(ERR_NOT_FACTORIZED, "[MAS] debug_spmv_multi: size mismatch or not fp16.");
        h->alloc_multi();
        PcgState hinit[RHS_GROUP + 1];
        std::memset(hinit, 0, sizeof(hinit));
        cuda_check(cudaMemcpyAsync(h->gst.get(), hinit, sizeof(hinit), cudaMemcpyHostToDevice, h->stream), "state");
        cuda_check(cudaMemcpyAsync(h->gp.get(), xin, sizeof(double) * len, cudaMemcpyHostToDevice, h->stream), "x");
        launch_spmv_g(SPMV_PAP, h->A.view(), h->gp.get(), h->gAp.get(), nullptr, h->gst.get(), h->red_g(), 1, 0,
                      h->stream);
        cuda_check(cudaMemcpyAsync(yout, h->gAp.get(), sizeof(double) * len, cudaMemcpyDeviceToHost, h->stream), "y");
        cuda_check(cudaStreamSynchronize(h->stream), "spmv");
    });
}

// Test hook: the device vectors after `iters` iterations of the several-right-hand-side loop
// (iters = 0: after the initial residual and apply), for the columns of a padded interleaved B.
// out: x, r, p, z (each len values) and the RHS_GROUP + 1 states (raw bytes appended).
extern "C" int mas_debug_multi_state(mas_solver *h, const double *Bpad, int len, int iters, double *out,
                                     void *states)
{
    if (!h)
        return MAS_ERR_INVALID;
    return guarded(h, [&] {
        cuda_check(cudaSetDevice(h->device), "set device");
        if (!h->multi_supported() || len != h->banks * 32 * h->bd * RHS_GROUP)
            throw Error(ERR_NOT_FACTORIZED, "[MAS] debug_multi_state: size mismatch or not fp16.");
        h->alloc_multi();
        cuda_check(cudaMemcpyAsync(h->gb.get(), Bpad, sizeof(double) * len, cudaMemcpyHostToDevice, h->stream), "b");
        cuda_check(cudaMemsetAsync(h->gx.get(), 0, h->gx.bytes(), h->stream), "memset");
        const int saved_max = h->p.max_iter;
        const bool saved_graphs = h->p.graphs;
        h->p.max_iter = iters;
        h->p.graphs = false;
        try
        {
            h->rhs_iterations.clear();
            h->rhs_status.clear();
            h->rhs_error.clear();
            h->pcg_multi(RHS_GROUP);
        }
        catch (...)
        {
            h->p.max_iter = saved_max;
            h->p.graphs = saved_graphs;
            throw;
        }
        h->p.max_iter = saved_max;
        h->p.graphs = saved_graphs;
        const double *src[4] = {h->gx.get(), h->gr.get(), h->gp.get(), h->gz.get()};
        for (int k = 0; k < 4; ++k)
            cuda_check(cudaMemcpyAsync(out + (size_t)k * len, src[k], sizeof(double) * len, cudaMemcpyDeviceToHost,
                                       h->stream),
                       "state vectors");
        cuda_check(cudaMemcpyAsync(states, h->gst.get(), sizeof(PcgState) * (RHS_GROUP + 1), cudaMemcpyDeviceToHost,
                                   h->stream),
                   "states");
        cuda_check(cudaStreamSynchronize(h->stream), "debug");
    });
}
