// Block SpMV on the bank-sliced matrix (sm_100a), FP64.
//
// Replaces the reference's cusparseSpMV on a row-major BSR (MASSolver.cu:271-290,
// CuSparseWrapper.hpp:141-154). One warp per bank: lane l owns block row bank * 32 + l and walks
// the bank's slots; a slot is one block per lane, read with coalesced 128-bit loads (512 B per
// value pair per warp), so every byte of A is read once, fully coalesced, with no reduction
// across lanes. x is gathered by column (it stays L2-resident: 12.8 MB at 1.6 M DOF).
//
// Fused epilogues (one pass over A per PCG step):
//   SPMV_PAP:      y = A p, pAp = p . y, alpha = rz / pAp (0 if |pAp| < 1e-20, MASSolver.cu:46-56)
//   SPMV_RESIDUAL: y = b - A x, rr = y . y (and ||b||^2 on the initial residual).
// The dot products are deterministic two-stage reductions (per-CTA partials, last CTA sums).

#include "mas_common.cuh"

namespace pmas
{
    namespace
    {
        constexpr int SPMV_THREADS = 256;
        constexpr int BANKS_PER_CTA = SPMV_THREADS / 32;

        // UNROLL slots per loop trip, their loads in flight together (the spmv_unroll parameter:
        // 1, 2 or 4; 2 measured best at 1.6 M DOF). Minimum one CTA per SM: the compiler then keeps
        // the unrolled slots' loads in flight (80 registers at 2, 3 CTAs per SM), measured faster
        // than the occupancy-first 44-register build at 1.6 M DOF.
        template <int BD, int MODE, int UNROLL>
        __device__ __forceinline__ void spmv_body(const BankedView &A, const double *__restrict__ x,
                                                  double *__restrict__ y, const double *__restrict__ b, PcgState *st,
                                                  const ReduceBuf &red, int iter, int period, Cta cta)
        {
            constexpr int BS = BD * BD;
            constexpr int PAIRS = BS / 2;
            pdl_wait();
            // The previous iteration's update_p has run: its deferred x update is applied.
            if (MODE == SPMV_PAP && cta.x == 0 && threadIdx.x == 0)
                st->x_applied = st->x_defer;
            if (MODE != SPMV_PLAIN && st->done)
                return;
            // In-loop true residual: only every `period`-th iteration (iteration = st->iter + 1).
            if (MODE == SPMV_RESIDUAL && period > 0 && (st->iter + 1) % period != 0)
                return;
            const int lane = threadIdx.x & 31;
            const int bank = cta.x * BANKS_PER_CTA + (threadIdx.x >> 5);
            double part = 0.0, bb = 0.0;
            if (bank < A.banks)
            {
                const int u = bank * 32 + lane;
                const long long s0 = A.slice[bank];
                const int len = A.rowlen[u];
                const int *cp = A.cols + s0 * 32 + lane;
                const double *vp = A.vals + s0 * 32 * BS;
                double acc[BD];
#pragma unroll
                for (int i = 0; i < BD; ++i)
                    acc[i] = 0.0;
                // The matrix streams through L2 with evict-first priority (x, the gathered vector,
                // and the other PCG vectors stay resident); two slots' loads in flight per lane.
                const uint64_t pol = l2_evict_first_policy();
#pragma unroll UNROLL
                for (int k = 0; k < len; ++k)
                {
                    const int col = ld_stream_s32(cp + (long long)k * 32, pol);
                    const double *blk = vp + (long long)k * 32 * BS;
                    double v[BS];
#pragma unroll
                    for (int p = 0; p < PAIRS; ++p)
                    {
                        const double2 t = ld_stream_f64x2(blk + p * 64 + lane * 2, pol);
                        v[2 * p] = t.x;
                        v[2 * p + 1] = t.y;
                    }
                    if (BS & 1)
                        v[BS - 1] = ld_stream_f64(blk + PAIRS * 64 + lane, pol);
                    double xc[BD];
#pragma unroll
                    for (int j = 0; j < BD; ++j)
                        xc[j] = __ldg(x + (long long)col * BD + j);
#pragma unroll
                    for (int i = 0; i < BD; ++i)
#pragma unroll
                        for (int j = 0; j < BD; ++j)
                            acc[i] = fma(v[i * BD + j], xc[j], acc[i]);
                }
                if (MODE == SPMV_PLAIN)
                {
#pragma unroll
                    for (int i = 0; i < BD; ++i)
                        y[(long long)u * BD + i] = acc[i];
                }
                else if (MODE == SPMV_PAP)
                {
#pragma unroll
                    for (int i = 0; i < BD; ++i)
                    {
                        y[(long long)u * BD + i] = acc[i];
                        part = fma(acc[i], x[(long long)u * BD + i], part);
                    }
                }
                else
                {
                    double rv[BD];
#pragma unroll
                    for (int i = 0; i < BD; ++i)
                    {
                        const double bv = b[(long long)u * BD + i];
                        rv[i] = bv - acc[i];
                        y[(long long)u * BD + i] = rv[i];
                        part = fma(rv[i], rv[i], part);
                        bb = fma(bv, bv, bb);
                    }
                }
            }
            pdl_release(); // the successor may start launching; the reduction below is the tail
            if (MODE == SPMV_PLAIN)
                return;
            if (MODE == SPMV_RESIDUAL && period > 0)
            {
                // In-loop true residual: rr = r . r (ticket on its own counter).
                double v1[1] = {part}, t1[1];
                if (grid_reduce<1, SPMV_THREADS>(v1, red.rr_parts, &st->counter[2], t1, cta) && threadIdx.x == 0)
                    st->rr = t1[0];
                return;
            }
            // rr0 = ||b||^2: equal to the reference's r.r at x = 0 (MASSolver.cu:488-494), and keeps
            // "relative" relative to ||b|| when an initial guess is used.
            double v2[2] = {part, bb}, tot[2];
            if (grid_reduce<2, SPMV_THREADS>(v2, red.partials, &st->counter[0], tot, cta) && threadIdx.x == 0)
            {
                if (MODE == SPMV_PAP)
                {
                    st->pAp = tot[0];
                    st->alpha = (fabs(tot[0]) < 1e-20) ? 0.0 : st->rz / tot[0];
                }
                else
                {
                    st->rr = tot[0];
                    if (iter == 0)
                        st->rr0 = tot[1];
                }
            }
        }

        template <int BD, int MODE, int UNROLL = 2>
        __global__ void __launch_bounds__(SPMV_THREADS, 1) k_spmv(BankedView A, const double *__restrict__ x,
                                                               double *__restrict__ y, const double *__restrict__ b,
                                                               PcgState *st, ReduceBuf red, int iter, int period)
        {
            spmv_body<BD, MODE, UNROLL>(A, x, y, b, st, red, iter, period, native_cta());
        }

        // The same SpMV for every system of a batch in one launch: p.Ap (MODE SPMV_PAP: x = p,
        // y = Ap) or the true residual (x, y = r, b).
        template <int BD, int MODE, int UNROLL = 2>
        __global__ void __launch_bounds__(SPMV_THREADS, 1) k_spmv_batch(BatchView v, int iter, int period)
        {
            const int4 e = batch_entry(v, BPH_SPMV);
            const BatchSystem &sy = v.sys[e.x];
            const Cta cta{e.y, e.z};
            const BankedView A = sy.A;
            const ReduceBuf red = sy.red;
            if (MODE == SPMV_PAP)
                spmv_body<BD, MODE, UNROLL>(A, sy.p, sy.Ap, nullptr, sy.st, red, iter, period, cta);
            else
                spmv_body<BD, MODE, UNROLL>(A, sy.x, sy.r, sy.b, sy.st, red, iter, period, cta);
        }

        template <int BD>
        void launch_bd(int mode, const BankedView &A, const double *x, double *y, const double *b, PcgState *st,
                       ReduceBuf red, int iter, int period, cudaStream_t s)
        {
            const int grid = spmv_grid(A);
            if (grid == 0)
                return;
            if (mode != SPMV_PLAIN && grid > red.capacity)
                throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
            const bool ch = chained_launch();
            auto go = [&]<int U>() {
                switch (mode)
                {
                case SPMV_PLAIN:
                    k_spmv<BD, SPMV_PLAIN, U><<<grid, SPMV_THREADS, 0, s>>>(A, x, y, b, st, red, iter, period);
                    break;
                case SPMV_PAP:
                    launch_chained(ch, k_spmv<BD, SPMV_PAP, U>, grid, SPMV_THREADS, 0, s, A, x, y, b, st, red, iter,
                                   period);
                    break;
                default:
                    launch_chained(ch, k_spmv<BD, SPMV_RESIDUAL, U>, grid, SPMV_THREADS, 0, s, A, x, y, b, st, red,
                                   iter, period);
                    break;
                }
            };
            const int u = spmv_unroll();
            if (u == 1)
                go.template operator()<1>();
            else if (u == 4)
                go.template operator()<4>();
            else
                go.template operator()<2>();
            cuda_check(cudaGetLastError(), "spmv launch");
        }
        template <int BD>
        void launch_batch_bd(int mode, const BatchView &v, int total, int iter, int period, cudaStream_t s)
        {
            auto go = [&]<int U>() {
                if (mode == SPMV_PAP)
                    launch_chained(chained_launch(), k_spmv_batch<BD, SPMV_PAP, U>, total, SPMV_THREADS, 0, s, v, iter, period);
                else
                    launch_chained(chained_launch(), k_spmv_batch<BD, SPMV_RESIDUAL, U>, total, SPMV_THREADS, 0, s, v, iter,
                                   period);
            };
            const int u = spmv_unroll();
            if (u == 1)
                go.template operator()<1>();
            else if (u == 4)
                go.template operator()<4>();
            else
                go.template operator()<2>();
            cuda_check(cudaGetLastError(), "batched spmv launch");
        }

        struct VecPtrs
        {
            const double *x[SPMV_MAX_VECTORS];
            double *y[SPMV_MAX_VECTORS];
        };

        // y_v = A x_v for NV separate vectors: each block of A is read once and applied to all of
        // them (the learned warm start's products with the kept solutions).
        template <int BD, int NV>
        __global__ void __launch_bounds__(SPMV_THREADS, 1) k_spmv_vectors(BankedView A, VecPtrs v)
        {
            constexpr int BS = BD * BD;
            constexpr int PAIRS = BS / 2;
            const int lane = threadIdx.x & 31;
            const int bank = blockIdx.x * BANKS_PER_CTA + (threadIdx.x >> 5);
            if (bank >= A.banks)
                return;
            const int u = bank * 32 + lane;
            const long long s0 = A.slice[bank];
            const int len = A.rowlen[u];
            const int *cp = A.cols + s0 * 32 + lane;
            const double *vp = A.vals + s0 * 32 * BS;
            double acc[NV][BD];
#pragma unroll
            for (int q = 0; q < NV; ++q)
#pragma unroll
                for (int i = 0; i < BD; ++i)
                    acc[q][i] = 0.0;
            const uint64_t pol = l2_evict_first_policy();
            for (int k = 0; k < len; ++k)
            {
                const int col = ld_stream_s32(cp + (long long)k * 32, pol);
                const double *blk = vp + (long long)k * 32 * BS;
                double m[BS];
#pragma unroll
                for (int p = 0; p < PAIRS; ++p)
                {
                    const double2 t = ld_stream_f64x2(blk + p * 64 + lane * 2, pol);
                    m[2 * p] = t.x;
                    m[2 * p + 1] = t.y;
                }
                if (BS & 1)
                    m[BS - 1] = ld_stream_f64(blk + PAIRS * 64 + lane, pol);
#pragma unroll
                for (int q = 0; q < NV; ++q)
                {
                    double xc[BD];
#pragma unroll
                    for (int j = 0; j < BD; ++j)
                        xc[j] = __ldg(v.x[q] + (long long)col * BD + j);
#pragma unroll
                    for (int i = 0; i < BD; ++i)
#pragma unroll
                        for (int j = 0; j < BD; ++j)
                            acc[q][i] = fma(m[i * BD + j], xc[j], acc[q][i]);
                }
            }
#pragma unroll
            for (int q = 0; q < NV; ++q)
#pragma unroll
                for (int i = 0; i < BD; ++i)
                    v.y[q][(long long)u * BD + i] = acc[q][i];
        }

        template <int BD>
        void launch_vectors_bd(const BankedView &A, const VecPtrs &v, int count, cudaStream_t s)
        {
            const int grid = (A.banks + BANKS_PER_CTA - 1) / BANKS_PER_CTA;
            if (grid == 0)
                return;
            switch (count)
            {
            case 1:
                k_spmv_vectors<BD, 1><<<grid, SPMV_THREADS, 0, s>>>(A, v);
                break;
            case 2:
                k_spmv_vectors<BD, 2><<<grid, SPMV_THREADS, 0, s>>>(A, v);
                break;
            case 3:
                k_spmv_vectors<BD, 3><<<grid, SPMV_THREADS, 0, s>>>(A, v);
                break;
            default:
                k_spmv_vectors<BD, 4><<<grid, SPMV_THREADS, 0, s>>>(A, v);
                break;
            }
            cuda_check(cudaGetLastError(), "spmv vectors launch");
        }
    } // namespace

    int spmv_grid(const BankedView &A) { return (A.banks + BANKS_PER_CTA - 1) / BANKS_PER_CTA; }

    void launch_spmv_batch(int mode, const BatchView &v, int bd, int total, int iter, int period, cudaStream_t s)
    {
        if (mode != SPMV_PAP && mode != SPMV_RESIDUAL)
            throw Error(ERR_INVALID, "[MAS] internal: batched SpMV modes are p.Ap and the true residual");
        if (total <= 0)
            return;
        if (bd == 1)
            launch_batch_bd<1>(mode, v, total, iter, period, s);
        else if (bd == 2)
            launch_batch_bd<2>(mode, v, total, iter, period, s);
        else
            launch_batch_bd<3>(mode, v, total, iter, period, s);
    }

    void launch_spmv_vectors(const BankedView &A, const double *const *x, double *const *y, int count, cudaStream_t s)
    {
        if (count < 1 || count > SPMV_MAX_VECTORS)
            throw Error(ERR_INVALID, "[MAS] internal: 1 to 4 vectors per SpMV pass");
        VecPtrs v{};
        for (int q = 0; q < count; ++q)
        {
            v.x[q] = x[q];
            v.y[q] = y[q];
        }
        switch (A.bd)
        {
        case 1:
            launch_vectors_bd<1>(A, v, count, s);
            break;
        case 2:
            launch_vectors_bd<2>(A, v, count, s);
            break;
        case 3:
            launch_vectors_bd<3>(A, v, count, s);
            break;
        default:
            throw Error(ERR_INVALID, "[MAS] block_dim must be 1, 2 or 3");
        }
    }

    void launch_spmv(int mode, const BankedView &A, const double *x, double *y, const double *b, PcgState *st,
                     ReduceBuf red, int iter, int period, cudaStream_t s)
    {
        switch (A.bd)
        {
        case 1:
            launch_bd<1>(mode, A, x, y, b, st, red, iter, period, s);
            break;
        case 2:
            launch_bd<2>(mode, A, x, y, b, st, red, iter, period, s);
            break;
        case 3:
            launch_bd<3>(mode, A, x, y, b, st, red, iter, period, s);
            break;
        default:
            throw Error(ERR_INVALID, "[MAS] block_dim must be 1, 2 or 3");
        }
    }
} // namespace pmas
