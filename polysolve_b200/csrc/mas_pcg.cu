// PCG vector kernels (sm_100a) and device-memory plumbing.
//
// The reference runs each vector step as its own launch (axpby / inner_product / scalar_division,
// MASSolver.cu:46-81, InnerProduct.cu:16-45) with a memset and an FP64 atomicAdd per dot. Here:
//   update_xr: r -= alpha Ap ; rr = r . r ; level-0 restriction of r  (one pass; on true-residual
//              iterations only x += alpha p, then r = b - A x follows in the SpMV)
//   update_p:  x += alpha p (the iteration's x update, moved here: this pass reads p anyway);
//              p = z0 + P zc + beta p    (the MAS prolongation fused in; beta from the device
//                                         state, set by the MAS apply)
// alpha / beta are read from the device-resident PcgState, and every dot is a deterministic
// two-stage reduction, so no host round trip is needed inside the iteration.

#include <atomic>
#include <cstdio>
#include <mutex>
#include <string>
#include <unordered_map>

#include "mas_common.cuh"

namespace pmas
{
    void cuda_check(cudaError_t e, const char *what)
    {
        if (e != cudaSuccess)
            throw Error(ERR_CUDA, std::string("[MAS] CUDA error in ") + what + ": " + cudaGetErrorString(e));
    }

    // Test hook (mas_debug_fail_allocation): the number of device allocations still to succeed
    // before one fails as if the device were out of memory; -1 = off.
    static std::atomic<long long> g_alloc_fail_after{-1};

    void set_alloc_failure(long long after) { g_alloc_fail_after.store(after < 0 ? -1 : after); }

    // Allocation with the reference's out-of-memory message (mas_utils/CudaUtils.cuh:68-79).
    void *device_alloc(size_t bytes, const char *ctx)
    {
        void *p = nullptr;
        cudaError_t e = cudaErrorMemoryAllocation;
        long long left = g_alloc_fail_after.load();
        bool injected = false;
        while (left >= 0)
        {
            // left == 0: this allocation fails (once); otherwise count it down.
            if (g_alloc_fail_after.compare_exchange_weak(left, left - 1))
            {
                injected = (left == 0);
                break;
            }
        }
        if (!injected)
            e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess)
            return p;
        if (e != cudaErrorMemoryAllocation)
            cuda_check(e, ctx);
        cudaGetLastError();
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t mb = 1024ull * 1024ull;
        throw Error(ERR_OOM, std::string("[MAS] Failed to allocate ") + std::to_string((bytes + mb - 1) / mb) +
                                 " MB for " + (ctx ? ctx : "cuda allocation") + "; only " +
                                 std::to_string(free_b / mb) + " MB free.");
    }

    void device_free(void *p)
    {
        if (p)
            cudaFree(p);
    }

    static thread_local bool t_chained_launch = true;
    void set_chained_launch(bool on) { t_chained_launch = on; }
    bool chained_launch() { return t_chained_launch; }
    static thread_local int t_spmv_unroll = 2;
    void set_spmv_unroll(int u) { t_spmv_unroll = u; }
    int spmv_unroll() { return t_spmv_unroll; }
    static thread_local int t_apply_ipw = 1;
    void set_apply_items_per_warp(int k) { t_apply_ipw = k < 1 ? 1 : k; }
    int apply_items_per_warp() { return t_apply_ipw; }

    namespace
    {
        constexpr int UPD_THREADS = 256;

        // r -= alpha Ap ; rr = r . r (ticket: the last CTA sums the partials) ; and the level-0
        // restriction of the new r (per-bank component sums, the MAS apply's first step); x +=
        // alpha p is left to update_p (st->x_defer). One warp per bank, its 32 * BD values read
        // coalesced (value t * 32 + lane). On a true-residual iteration only x is updated here:
        // r, rr and the restriction follow the SpMV.
        template <int BD>
        __device__ __forceinline__ void update_xr_body(const MasView &mas, double *__restrict__ x,
                                                       double *__restrict__ r, const double *__restrict__ p,
                                                       const double *__restrict__ Ap, PcgState *st,
                                                       const ReduceBuf &red, int period, Cta cta)
        {
            pdl_wait();
            if (st->done)
                return;
            const double alpha = st->alpha;
            const bool due = period > 0 && (st->iter + 1) % period == 0;
            if (cta.x == 0 && threadIdx.x == 0)
                st->x_defer = due ? -1 : st->iter + 1;
            const int lane = threadIdx.x & 31;
            const int total_warps = cta.n * (UPD_THREADS / 32);
            const bool restrict_r = !due && mas.level_num > 0;
            double part = 0.0;
            // Two-stage pipeline over the warp's banks (one or two in the resident grid): the next
            // bank's loads (x and p, or Ap and r, and its restriction keys) are issued before this
            // bank's update and restriction. Same arithmetic in the same order as one bank at a time.
            double na[BD], nb[BD];
            int nkey = -1, nbase = 0;
            auto load = [&](int bank) {
                const long long b0 = (long long)bank * 32 * BD + lane;
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    if (due)
                    {
                        na[t] = x[b0 + t * 32];
                        nb[t] = p[b0 + t * 32];
                    }
                    else
                    {
                        na[t] = Ap[b0 + t * 32];
                        nb[t] = r[b0 + t * 32];
                    }
                }
                if (restrict_r && bank < mas.first_iso_bank)
                {
                    nkey = mas.lcco0[(long long)bank * 32 + lane];
                    nbase = mas.cco0_base[bank];
                }
            };
            const int first = cta.x * (UPD_THREADS / 32) + (threadIdx.x >> 5);
            if (first < mas.banks)
                load(first);
            for (int bank = first; bank < mas.banks; bank += total_warps)
            {
                double av[BD], bv[BD];
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    av[t] = na[t];
                    bv[t] = nb[t];
                }
                const int key = nkey, base = nbase;
                if (bank + total_warps < mas.banks)
                    load(bank + total_warps);
                const long long b0 = (long long)bank * 32 * BD + lane;
                double rv[BD];
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    rv[t] = 0.0;
                    if (due)
                        x[b0 + t * 32] = fma(alpha, bv[t], av[t]);
                    else
                    {
                        rv[t] = fma(-alpha, av[t], bv[t]);
                        r[b0 + t * 32] = rv[t];
                        part = fma(rv[t], rv[t], part);
                    }
                }
                if (restrict_r && bank < mas.first_iso_bank)
                    bank_restrict_keyed<BD>(rv, key, base, mas.rc);
            }
            pdl_release();
            if (due)
                return;
            double v1[1] = {part}, tot[1];
            if (grid_reduce<1, UPD_THREADS>(v1, red.rr_parts, &st->counter[1], tot, cta) && threadIdx.x == 0)
                st->rr = tot[0];
        }

        template <int BD>
        __global__ void __launch_bounds__(UPD_THREADS) k_update_xr(MasView mas, double *__restrict__ x,
                                                                   double *__restrict__ r, const double *__restrict__ p,
                                                                   const double *__restrict__ Ap, PcgState *st,
                                                                   ReduceBuf red, int period)
        {
            update_xr_body<BD>(mas, x, r, p, Ap, st, red, period, native_cta());
        }

        template <int BD>
        __global__ void __launch_bounds__(UPD_THREADS) k_update_xr_batch(BatchView v, int period)
        {
            const int4 e = batch_entry(v, BPH_UPDATE_XR);
            const BatchSystem &sy = v.sys[e.x];
            const Cta cta{e.y, e.z};
            const MasView mas = sy.mas;
            const ReduceBuf red = sy.red;
            update_xr_body<BD>(mas, sy.x, sy.r, sy.p, sy.Ap, sy.st, red, period,
                               cta);
        }

        // x += alpha p when update_xr left it (see PcgState::x_defer), also on the iteration that
        // stops the solve; p = z0 + sum_l zc[cslot_l(node)] + beta p; warps stride over banks,
        // coalesced.
        template <int BD>
        __device__ __forceinline__ void update_p_body(const MasView &mas, double *__restrict__ x,
                                                      double *__restrict__ p, const double *__restrict__ z0,
                                                      const PcgState *st, int first, Cta cta)
        {
            pdl_wait();
            const int it = st->iter;
            const bool xdo = !first && st->x_defer == it && st->x_applied != it;
            const bool pdo = !st->done;
            if (!xdo && !pdo)
                return;
            const double alpha = st->alpha;
            const double beta = first ? 0.0 : st->beta;
            const int lane = threadIdx.x & 31;
            const int total_warps = cta.n * (UPD_THREADS / 32);
            const double *__restrict__ zc = mas.zc;
            const double iso_scale = 1.0 + mas.level_num;
            for (int bank = cta.x * (UPD_THREADS / 32) + (threadIdx.x >> 5); bank < mas.banks; bank += total_warps)
            {
                const long long b0 = (long long)bank * 32 * BD;
                if (bank >= mas.first_iso_bank)
                {
                    // Isolated rows: every coarse level adds z0 again (coarse block A_uu).
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                    {
                        const long long idx = b0 + t * 32 + lane;
                        const double po = first ? 0.0 : p[idx];
                        if (xdo)
                            x[idx] = fma(alpha, po, x[idx]);
                        if (pdo)
                        {
                            const double v = iso_scale * z0[idx];
                            p[idx] = first ? v : fma(beta, po, v);
                        }
                    }
                    continue;
                }
                // Loads first (z0, p, x and the coarse slots), then the coarse-value gathers.
                double zv[BD], pold[BD], xv[BD];
                int4 cs[BD];
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    const int e = t * 32 + lane;
                    const int node = e / BD;
                    zv[t] = pdo ? z0[b0 + e] : 0.0;
                    pold[t] = first ? 0.0 : p[b0 + e];
                    xv[t] = xdo ? x[b0 + e] : 0.0;
                    cs[t] = pdo ? mas.cslot[(long long)bank * 32 + node] : make_int4(-1, -1, -1, -1);
                }
                if (xdo)
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                        x[b0 + t * 32 + lane] = fma(alpha, pold[t], xv[t]);
                if (!pdo)
                    continue;
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    const int e = t * 32 + lane;
                    const int comp = e - (e / BD) * BD;
                    // Unconditional loads (slot -1 reads zc[comp], then drops it): all in flight.
                    const double g0 = zc[(size_t)max(cs[t].x, 0) * BD + comp];
                    const double g1 = zc[(size_t)max(cs[t].y, 0) * BD + comp];
                    const double g2 = zc[(size_t)max(cs[t].z, 0) * BD + comp];
                    const double g3 = zc[(size_t)max(cs[t].w, 0) * BD + comp];
                    double v = zv[t];
                    v += cs[t].x >= 0 ? g0 : 0.0;
                    v += cs[t].y >= 0 ? g1 : 0.0;
                    v += cs[t].z >= 0 ? g2 : 0.0;
                    v += cs[t].w >= 0 ? g3 : 0.0;
                    p[b0 + e] = first ? v : fma(beta, pold[t], v);
                }
            }
        }

        template <int BD>
        __global__ void __launch_bounds__(UPD_THREADS) k_update_p(MasView mas, double *__restrict__ x,
                                                                  double *__restrict__ p,
                                                                  const double *__restrict__ z0, const PcgState *st,
                                                                  int first)
        {
            update_p_body<BD>(mas, x, p, z0, st, first, native_cta());
        }

        template <int BD>
        __global__ void __launch_bounds__(UPD_THREADS) k_update_p_batch(BatchView v, int first)
        {
            const int4 e = batch_entry(v, BPH_UPDATE_P);
            const BatchSystem &sy = v.sys[e.x];
            const Cta cta{e.y, e.z};
            const MasView mas = sy.mas;
            update_p_body<BD>(mas, sy.x, sy.p, sy.z, sy.st, first, cta);
        }

        // Every system's PcgState copied into out[s] (one host read of the whole batch's states).
        __global__ void k_gather_states_batch(BatchView v, PcgState *out)
        {
            const unsigned *src = reinterpret_cast<const unsigned *>(v.sys[blockIdx.x].st);
            unsigned *dst = reinterpret_cast<unsigned *>(out + blockIdx.x);
            for (int i = threadIdx.x; i < (int)(sizeof(PcgState) / sizeof(unsigned)); i += blockDim.x)
                dst[i] = __ldcg(src + i);
        }

        // Every system's PcgState set to zero (the batched form of launch_pcg_init_state).
        __global__ void k_init_states_batch(BatchView v)
        {
            unsigned *w = reinterpret_cast<unsigned *>(v.sys[blockIdx.x].st);
            for (int i = threadIdx.x; i < (int)(sizeof(PcgState) / sizeof(unsigned)); i += blockDim.x)
                w[i] = 0u;
        }

        // dst (padded, node-major, zero elsewhere) <- src (caller's order, length n)
        __global__ void k_permute_in(int n, int bd, int V, const int *__restrict__ padded_of_block,
                                     const double *__restrict__ src, double *__restrict__ dst)
        {
            const long long total = (long long)V * bd;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
                 i += (long long)gridDim.x * blockDim.x)
            {
                const int blk = (int)(i / bd), c = (int)(i % bd);
                dst[(long long)padded_of_block[blk] * bd + c] = (i < n) ? src[i] : 0.0;
            }
        }

        __global__ void k_permute_out(int n, int bd, const int *__restrict__ padded_of_block,
                                      const double *__restrict__ src, double *__restrict__ dst)
        {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
                 i += (long long)gridDim.x * blockDim.x)
            {
                const int blk = (int)(i / bd), c = (int)(i % bd);
                dst[i] = src[(long long)padded_of_block[blk] * bd + c];
            }
        }

        __global__ void k_zero(double *p, long long n)
        {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
                 i += (long long)gridDim.x * blockDim.x)
                p[i] = 0.0;
        }

        int grid_for(long long n, int threads = 256)
        {
            long long g = (n + threads - 1) / threads;
            if (g > 148LL * 16)
                g = 148LL * 16;
            return (int)(g < 1 ? 1 : g);
        }
    } // namespace

    namespace
    {
        // CTAs of UPD_THREADS threads of `kernel` resident on the whole device at once.
        template <class K>
        int resident_ctas(K kernel)
        {
            static std::mutex mu;
            static std::unordered_map<const void *, int> cache; // kernel -> CTAs per SM
            int per_sm = 0;
            {
                std::lock_guard<std::mutex> lock(mu);
                auto it = cache.find((const void *)kernel);
                if (it != cache.end())
                    per_sm = it->second;
            }
            if (per_sm == 0)
            {
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, UPD_THREADS, 0) != cudaSuccess ||
                    per_sm < 1)
                {
                    cudaGetLastError();
                    per_sm = 1;
                }
                std::lock_guard<std::mutex> lock(mu);
                cache[(const void *)kernel] = per_sm;
            }
            return per_sm * device_sm_count();
        }

        // Resident grid (one wave, warps loop over banks): update_xr, whose rr ticket then has
        // few arrivals.
        template <class K>
        int bank_grid(int banks, K kernel)
        {
            const int need = (banks + UPD_THREADS / 32 - 1) / (UPD_THREADS / 32);
            const int cap = resident_ctas(kernel);
            return need < cap ? need : cap;
        }

        // One warp per bank: the hardware hands CTAs to SMs as others finish, which balances the
        // end of a short streaming kernel without a reduction (update_p).
        int bank_grid_all(int banks) { return (banks + UPD_THREADS / 32 - 1) / (UPD_THREADS / 32); }
    } // namespace

    int update_xr_grid(const MasView &mas)
    {
        // One resident wave: as many CTAs as fit on the device at once.
        int grid = mas.bd == 1 ? bank_grid(mas.banks, k_update_xr<1>)
                               : (mas.bd == 2 ? bank_grid(mas.banks, k_update_xr<2>) : bank_grid(mas.banks, k_update_xr<3>));
        return grid < 1 ? 1 : grid;
    }

    int update_p_grid(const MasView &mas) { return bank_grid_all(mas.banks); }

    void launch_update_xr_batch(const BatchView &v, int bd, int total, int period, cudaStream_t s)
    {
        if (total <= 0)
            return;
        if (bd == 1)
            launch_chained(chained_launch(), k_update_xr_batch<1>, total, UPD_THREADS, 0, s, v, period);
        else if (bd == 2)
            launch_chained(chained_launch(), k_update_xr_batch<2>, total, UPD_THREADS, 0, s, v, period);
        else
            launch_chained(chained_launch(), k_update_xr_batch<3>, total, UPD_THREADS, 0, s, v, period);
        cuda_check(cudaGetLastError(), "batched update_xr launch");
    }

    void launch_update_p_batch(const BatchView &v, int bd, int total, int first, cudaStream_t s)
    {
        if (total <= 0)
            return;
        if (bd == 1)
            launch_chained(chained_launch(), k_update_p_batch<1>, total, UPD_THREADS, 0, s, v, first);
        else if (bd == 2)
            launch_chained(chained_launch(), k_update_p_batch<2>, total, UPD_THREADS, 0, s, v, first);
        else
            launch_chained(chained_launch(), k_update_p_batch<3>, total, UPD_THREADS, 0, s, v, first);
        cuda_check(cudaGetLastError(), "batched update_p launch");
    }

    void launch_gather_states_batch(const BatchView &v, PcgState *out, cudaStream_t s)
    {
        if (v.count <= 0)
            return;
        k_gather_states_batch<<<v.count, 64, 0, s>>>(v, out);
        cuda_check(cudaGetLastError(), "batched state gather launch");
    }

    void launch_init_states_batch(const BatchView &v, cudaStream_t s)
    {
        if (v.count <= 0)
            return;
        k_init_states_batch<<<v.count, 64, 0, s>>>(v);
        cuda_check(cudaGetLastError(), "batched state reset launch");
    }

    void launch_update_xr(const MasView &mas, double *x, double *r, const double *p, const double *Ap, PcgState *st,
                          ReduceBuf red, int period, cudaStream_t s)
    {
        auto go = [&](auto kernel) {
            const int grid = update_xr_grid(mas);
            if (grid > red.capacity)
                throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
            launch_chained(chained_launch(), kernel, grid, UPD_THREADS, 0, s, mas, x, r, p, Ap, st, red, period);
        };
        if (mas.bd == 1)
            go(k_update_xr<1>);
        else if (mas.bd == 2)
            go(k_update_xr<2>);
        else
            go(k_update_xr<3>);
        cuda_check(cudaGetLastError(), "update_xr launch");
    }

    void launch_update_p(const MasView &mas, double *x, double *p, const double *z0, PcgState *st, int first,
                         cudaStream_t s)
    {
        auto go = [&](auto kernel) {
            const int grid = update_p_grid(mas);
            if (grid > 0)
                launch_chained(chained_launch(), kernel, grid, UPD_THREADS, 0, s, mas, x, p, z0, st, first);
        };
        if (mas.bd == 1)
            go(k_update_p<1>);
        else if (mas.bd == 2)
            go(k_update_p<2>);
        else
            go(k_update_p<3>);
        cuda_check(cudaGetLastError(), "update_p launch");
    }

    void launch_permute_in(int n, int bd, int V, const int *padded_of_block, const double *src, double *dst,
                           size_t dst_len, cudaStream_t s)
    {
        k_zero<<<grid_for((long long)dst_len), 256, 0, s>>>(dst, (long long)dst_len);
        k_permute_in<<<grid_for((long long)V * bd), 256, 0, s>>>(n, bd, V, padded_of_block, src, dst);
        cuda_check(cudaGetLastError(), "permute_in launch");
    }

    void launch_permute_out(int n, int bd, int V, const int *padded_of_block, const double *src, double *dst,
                            cudaStream_t s)
    {
        (void)V;
        k_permute_out<<<grid_for(n), 256, 0, s>>>(n, bd, padded_of_block, src, dst);
        cuda_check(cudaGetLastError(), "permute_out launch");
    }

    void launch_zero(double *p, size_t n, cudaStream_t s)
    {
        if (n == 0)
            return;
        k_zero<<<grid_for((long long)n), 256, 0, s>>>(p, (long long)n);
        cuda_check(cudaGetLastError(), "zero launch");
    }

    void launch_pcg_init_state(PcgState *st, cudaStream_t s)
    {
        cuda_check(cudaMemsetAsync(st, 0, sizeof(PcgState), s), "state reset");
    }
} // namespace pmas
