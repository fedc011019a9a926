// Several right-hand sides at once (sm_100a): G = RHS_GROUP independent PCG solves that share
// every read of the matrix and of the MAS inverses.
//
// The reference solves one right-hand side per call (MASSolver.cu:376-409); a caller with 16
// right-hand sides pays 16 passes over A (615 MB at 1.6 M DOF) and the inverses per iteration.
// Here the G vectors of a group are interleaved (value index = (node * bd + component) * G + g),
// so one warp-per-bank pass over A serves all G (the x gathers read G contiguous values), the
// vector kernels stream G times the data with per-right-hand-side scalars, and the restriction and
// the coarse levels treat the G right-hand sides as bd * G components of one node. The tensor-core
// MAS apply for a group lives in mas_apply.cu (the B operand's 8 columns hold the G hi / lo
// splits). Each right-hand side has its own PcgState (alpha, beta, convergence, status); entry G
// of the state array is the group record (iteration counter, all-done flag).

#include "mas_common.cuh"

namespace pmas
{
    namespace
    {
        constexpr int G = RHS_GROUP;
        constexpr int MT = 256; // threads per CTA of the multi kernels

        // Two slots per loop trip with at most 128 registers (two CTAs per SM): both slots' loads
        // and gathers in flight.
        template <int BD, int MODE>
        __global__ void __launch_bounds__(MT, 2) k_spmv_g(BankedView A, const double *__restrict__ x,
                                                      double *__restrict__ y, const double *__restrict__ b,
                                                      PcgState *st, ReduceBuf red, int iter, int period)
        {
            constexpr int BS = BD * BD;
            constexpr int PAIRS = BS / 2;
            PcgState *grp = st + G;
            // The previous iteration's update_p has run: its deferred x update is applied.
            if (MODE == SPMV_PAP && blockIdx.x == 0 && threadIdx.x == 0)
                grp->x_applied = grp->x_defer;
            if (grp->done)
                return;
            if (MODE == SPMV_RESIDUAL && period > 0 && (grp->iter + 1) % period != 0)
                return;
            const int lane = threadIdx.x & 31;
            const int bank = blockIdx.x * (MT / 32) + (threadIdx.x >> 5);
            double part[G], bb[G];
#pragma unroll
            for (int g = 0; g < G; ++g)
                part[g] = bb[g] = 0.0;
            if (bank < A.banks)
            {
                const int u = bank * 32 + lane;
                const long long s0 = A.slice[bank];
                const int len = A.rowlen[u];
                const int *cp = A.cols + s0 * 32 + lane;
                const double *vp = A.vals + s0 * 32 * BS;
                double acc[BD][G];
#pragma unroll
                for (int i = 0; i < BD; ++i)
#pragma unroll
                    for (int g = 0; g < G; ++g)
                        acc[i][g] = 0.0;
                const uint64_t pol = l2_evict_first_policy();
#pragma unroll 2
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
#pragma unroll
                    for (int j = 0; j < BD; ++j)
                    {
                        const double2 *xp = reinterpret_cast<const double2 *>(x + ((long long)col * BD + j) * G);
                        double xc[G];
#pragma unroll
                        for (int h = 0; h < G / 2; ++h)
                        {
                            const double2 t = __ldg(xp + h);
                            xc[2 * h] = t.x;
                            xc[2 * h + 1] = t.y;
                        }
#pragma unroll
                        for (int i = 0; i < BD; ++i)
#pragma unroll
                            for (int g = 0; g < G; ++g)
                                acc[i][g] = fma(v[i * BD + j], xc[g], acc[i][g]);
                    }
                }
#pragma unroll
                for (int i = 0; i < BD; ++i)
#pragma unroll
                    for (int g = 0; g < G; ++g)
                    {
                        const long long idx = ((long long)u * BD + i) * G + g;
                        if (MODE == SPMV_PAP)
                        {
                            y[idx] = acc[i][g];
                            part[g] = fma(acc[i][g], x[idx], part[g]);
                        }
                        else
                        {
                            const double bv = b[idx];
                            const double rv = bv - acc[i][g];
                            y[idx] = rv;
                            part[g] = fma(rv, rv, part[g]);
                            bb[g] = fma(bv, bv, bb[g]);
                        }
                    }
            }
            if (MODE == SPMV_RESIDUAL && period > 0)
            {
                double tot[G];
                if (grid_reduce<G, MT>(part, red.rr_parts, &grp->counter[2], tot) && threadIdx.x == 0)
#pragma unroll
                    for (int g = 0; g < G; ++g)
                        if (!st[g].done)
                            st[g].rr = tot[g];
                return;
            }
            double v2[2 * G], tot[2 * G];
#pragma unroll
            for (int g = 0; g < G; ++g)
            {
                v2[g] = part[g];
                v2[G + g] = bb[g];
            }
            if (grid_reduce<2 * G, MT>(v2, red.partials, &grp->counter[0], tot) && threadIdx.x == 0)
            {
#pragma unroll
                for (int g = 0; g < G; ++g)
                {
                    if (st[g].done)
                    {
                        st[g].alpha = 0.0; // a finished right-hand side keeps its x and r
                        continue;
                    }
                    if (MODE == SPMV_PAP)
                    {
                        st[g].pAp = tot[g];
                        st[g].alpha = (fabs(tot[g]) < 1e-20) ? 0.0 : st[g].rz / tot[g];
                    }
                    else
                    {
                        st[g].rr = tot[g];
                        if (iter == 0)
                            st[g].rr0 = tot[G + g];
                    }
                }
            }
        }

        // x += alpha_g p ; r -= alpha_g Ap ; rr_g ; restriction of every r_g (as bd * G components).
        template <int BD>
        __global__ void __launch_bounds__(MT) k_update_xr_g(MasView mas, double *__restrict__ x, double *__restrict__ r,
                                                           const double *__restrict__ p,
                                                           const double *__restrict__ Ap, PcgState *st,
                                                           ReduceBuf red, int period)
        {
            constexpr int BDG = BD * G;
            PcgState *grp = st + G;
            if (grp->done)
                return;
            double alpha[G];
#pragma unroll
            for (int g = 0; g < G; ++g)
                alpha[g] = st[g].alpha;
            const bool due = period > 0 && (grp->iter + 1) % period == 0;
            if (blockIdx.x == 0 && threadIdx.x == 0)
                grp->x_defer = due ? -1 : grp->iter + 1; // x += alpha p otherwise runs in update_p
            const int lane = threadIdx.x & 31;
            const int total_warps = gridDim.x * (MT / 32);
            const bool restrict_r = !due && mas.level_num > 0;
            double part[G];
#pragma unroll
            for (int g = 0; g < G; ++g)
                part[g] = 0.0;
            for (int bank = blockIdx.x * (MT / 32) + (threadIdx.x >> 5); bank < mas.banks; bank += total_warps)
            {
                const long long b0 = (long long)bank * 32 * BDG + lane;
                double xv[BDG], pv[BDG], av[BDG], rv[BDG];
#pragma unroll
                for (int t = 0; t < BDG; ++t)
                {
                    xv[t] = pv[t] = av[t] = rv[t] = 0.0;
                    if (due)
                    {
                        xv[t] = x[b0 + t * 32];
                        pv[t] = p[b0 + t * 32];
                    }
                    else
                    {
                        av[t] = Ap[b0 + t * 32];
                        rv[t] = r[b0 + t * 32];
                    }
                }
#pragma unroll
                for (int t = 0; t < BDG; ++t)
                {
                    const int g = (t * 32 + lane) % G; // G divides 32: g = lane % G
                    const double a = alpha[g];
                    if (due)
                        x[b0 + t * 32] = fma(a, pv[t], xv[t]);
                    if (!due)
                    {
                        rv[t] = fma(-a, av[t], rv[t]);
                        r[b0 + t * 32] = rv[t];
#pragma unroll
                        for (int h = 0; h < G; ++h)
                            if (h == g)
                                part[h] = fma(rv[t], rv[t], part[h]);
                    }
                }
                if (restrict_r && bank < mas.first_iso_bank)
                    bank_restrict<BDG>(rv, bank, mas.lcco0, mas.cco0_base, mas.rc);
            }
            if (due)
                return;
            double tot[G];
            if (grid_reduce<G, MT>(part, red.rr_parts, &grp->counter[1], tot) && threadIdx.x == 0)
#pragma unroll
                for (int g = 0; g < G; ++g)
                    if (!st[g].done)
                        st[g].rr = tot[g];
        }

        // x_g += alpha_g p_g when update_xr left it (PcgState::x_defer);
        // p_g = z0_g + prolongation(zc_g) + beta_g p_g (first: p = z).
        template <int BD>
        __global__ void __launch_bounds__(MT) k_update_p_g(MasView mas, double *__restrict__ x, double *__restrict__ p,
                                                          const double *__restrict__ z0, const PcgState *st,
                                                          int first)
        {
            constexpr int BDG = BD * G;
            const PcgState *grp = st + G;
            const int it = grp->iter;
            const bool xdo = !first && grp->x_defer == it && grp->x_applied != it;
            if (grp->done && !xdo)
                return;
            double beta[G], alpha[G];
            bool skip[G];
#pragma unroll
            for (int g = 0; g < G; ++g)
            {
                beta[g] = first ? 0.0 : st[g].beta;
                alpha[g] = st[g].alpha;
                skip[g] = st[g].done != 0 || grp->done != 0;
            }
            const int lane = threadIdx.x & 31;
            const double *__restrict__ zc = mas.zc;
            const double iso_scale = 1.0 + mas.level_num;
            const int bank = blockIdx.x * (MT / 32) + (threadIdx.x >> 5);
            if (bank >= mas.banks)
                return;
            const long long b0 = (long long)bank * 32 * BDG;
            const bool iso = bank >= mas.first_iso_bank;
            double zv[BDG], pold[BDG], xv[BDG];
            int4 cs[BDG];
#pragma unroll
            for (int t = 0; t < BDG; ++t)
            {
                const int e = t * 32 + lane; // node-local value: node * BDG + component * G + g
                zv[t] = z0[b0 + e];
                pold[t] = first ? 0.0 : p[b0 + e];
                xv[t] = xdo ? x[b0 + e] : 0.0;
                cs[t] = iso ? make_int4(-1, -1, -1, -1) : mas.cslot[(long long)bank * 32 + e / BDG];
            }
            if (xdo)
#pragma unroll
                for (int t = 0; t < BDG; ++t)
                {
                    const int g = (t * 32 + lane) % G;
                    double a = 0.0;
#pragma unroll
                    for (int h = 0; h < G; ++h)
                        if (h == g)
                            a = alpha[h];
                    x[b0 + t * 32 + lane] = fma(a, pold[t], xv[t]);
                }
#pragma unroll
            for (int t = 0; t < BDG; ++t)
            {
                const int e = t * 32 + lane;
                const int comp = e % BDG; // component * G + g
                const int g = comp % G;
                double v;
                if (iso)
                    v = iso_scale * zv[t];
                else
                {
                    const double g0 = zc[(size_t)max(cs[t].x, 0) * BDG + comp];
                    const double g1 = zc[(size_t)max(cs[t].y, 0) * BDG + comp];
                    const double g2 = zc[(size_t)max(cs[t].z, 0) * BDG + comp];
                    const double g3 = zc[(size_t)max(cs[t].w, 0) * BDG + comp];
                    v = zv[t];
                    v += cs[t].x >= 0 ? g0 : 0.0;
                    v += cs[t].y >= 0 ? g1 : 0.0;
                    v += cs[t].z >= 0 ? g2 : 0.0;
                    v += cs[t].w >= 0 ? g3 : 0.0;
                }
                bool sk = false;
                double bt = 0.0;
#pragma unroll
                for (int h = 0; h < G; ++h)
                    if (h == g)
                    {
                        sk = skip[h];
                        bt = beta[h];
                    }
                if (!sk)
                    p[b0 + e] = first ? v : fma(bt, pold[t], v);
            }
        }

        // Restriction of r (initial residual, true-residual iterations): bd * G components per node.
        template <int BDG>
        __global__ void __launch_bounds__(256) k_restrict_g(int banks, const double *__restrict__ r,
                                                            const int *__restrict__ lcco0,
                                                            const int *__restrict__ cco0_base, double *rc,
                                                            const PcgState *grp, int period)
        {
            if (grp->done)
                return;
            if (period > 0 && (grp->iter + 1) % period != 0)
                return;
            const int lane = threadIdx.x & 31;
            const int bank = blockIdx.x * 8 + (threadIdx.x >> 5);
            if (bank >= banks)
                return;
            const long long b0 = (long long)bank * 32 * BDG;
            double reg[BDG];
#pragma unroll
            for (int t = 0; t < BDG; ++t)
                reg[t] = r[b0 + t * 32 + lane];
            bank_restrict<BDG>(reg, bank, lcco0, cco0_base, rc);
        }

        // Caller columns c0 .. c0 + cols - 1 of the column-major B (n x nrhs) into the interleaved
        // padded layout; missing columns (cols < G) and padding are zero.
        __global__ void k_permute_in_g(int n, int bd, int V, int cols, const int *__restrict__ padded_of_block,
                                       const double *__restrict__ B, double *__restrict__ dst)
        {
            const long long total = (long long)V * bd * G;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
                 i += (long long)gridDim.x * blockDim.x)
            {
                const long long row = i / G;
                const int g = (int)(i % G);
                const int blk = (int)(row / bd), c = (int)(row % bd);
                const double v = (g < cols && row < n) ? B[(long long)g * n + row] : 0.0;
                dst[((long long)padded_of_block[blk] * bd + c) * G + g] = v;
            }
        }

        __global__ void k_permute_out_g(int n, int bd, int cols, const int *__restrict__ padded_of_block,
                                        const double *__restrict__ src, double *__restrict__ X)
        {
            const long long total = (long long)n * cols;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
                 i += (long long)gridDim.x * blockDim.x)
            {
                const int g = (int)(i / n);
                const long long row = i % n;
                const int blk = (int)(row / bd), c = (int)(row % bd);
                X[i] = src[((long long)padded_of_block[blk] * bd + c) * G + g];
            }
        }

        int grid_cap(long long n)
        {
            long long g = (n + 255) / 256;
            const long long cap = (long long)device_sm_count() * 16;
            if (g > cap)
                g = cap;
            return (int)(g < 1 ? 1 : g);
        }

        template <class F>
        auto by_bd(int bd, F &&f)
        {
            return bd == 1 ? f.template operator()<1>() : (bd == 2 ? f.template operator()<2>() : f.template operator()<3>());
        }
    } // namespace

    void launch_spmv_g(int mode, const BankedView &A, const double *x, double *y, const double *b, PcgState *st,
                       ReduceBuf red, int iter, int period, cudaStream_t s)
    {
        const int grid = (A.banks + MT / 32 - 1) / (MT / 32);
        if (grid == 0)
            return;
        if (grid > red.capacity)
            throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
        by_bd(A.bd, [&]<int BD>() {
            if (mode == SPMV_PAP)
                k_spmv_g<BD, SPMV_PAP><<<grid, MT, 0, s>>>(A, x, y, b, st, red, iter, period);
            else
                k_spmv_g<BD, SPMV_RESIDUAL><<<grid, MT, 0, s>>>(A, x, y, b, st, red, iter, period);
        });
        cuda_check(cudaGetLastError(), "multi spmv launch");
    }

    void launch_update_xr_g(const MasView &mas, double *x, double *r, const double *p, const double *Ap,
                            PcgState *st, ReduceBuf red, int period, cudaStream_t s)
    {
        int grid = (mas.banks + MT / 32 - 1) / (MT / 32);
        const int cap = device_sm_count() * 4;
        grid = grid < cap ? grid : cap;
        if (grid < 1)
            grid = 1;
        if (grid > red.capacity)
            throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
        by_bd(mas.bd, [&]<int BD>() { k_update_xr_g<BD><<<grid, MT, 0, s>>>(mas, x, r, p, Ap, st, red, period); });
        cuda_check(cudaGetLastError(), "multi update_xr launch");
    }

    void launch_update_p_g(const MasView &mas, double *x, double *p, const double *z0, PcgState *st, int first,
                           cudaStream_t s)
    {
        const int grid = (mas.banks + MT / 32 - 1) / (MT / 32);
        if (grid == 0)
            return;
        by_bd(mas.bd, [&]<int BD>() { k_update_p_g<BD><<<grid, MT, 0, s>>>(mas, x, p, z0, st, first); });
        cuda_check(cudaGetLastError(), "multi update_p launch");
    }

    int launch_restrict_g(const MasView &mas, const double *r, const PcgState *grp, int period, cudaStream_t s)
    {
        if (mas.first_iso_bank <= 0 || mas.level_num <= 0)
            return 0;
        const int grid = (mas.first_iso_bank + 7) / 8;
        by_bd(mas.bd, [&]<int BD>() {
            k_restrict_g<BD * G><<<grid, 256, 0, s>>>(mas.first_iso_bank, r, mas.lcco0, mas.cco0_base, mas.rc, grp,
                                                      period);
        });
        cuda_check(cudaGetLastError(), "multi restrict launch");
        return 1;
    }

    void launch_permute_in_g(int n, int bd, int V, int cols, const int *padded_of_block, const double *B, double *dst,
                             size_t dst_len, cudaStream_t s)
    {
        launch_zero(dst, dst_len, s);
        k_permute_in_g<<<grid_cap((long long)V * bd * G), 256, 0, s>>>(n, bd, V, cols, padded_of_block, B, dst);
        cuda_check(cudaGetLastError(), "multi permute_in launch");
    }

    void launch_permute_out_g(int n, int bd, int cols, const int *padded_of_block, const double *src, double *X,
                              cudaStream_t s)
    {
        k_permute_out_g<<<grid_cap((long long)n * cols), 256, 0, s>>>(n, bd, cols, padded_of_block, src, X);
        cuda_check(cudaGetLastError(), "multi permute_out launch");
    }
} // namespace pmas
