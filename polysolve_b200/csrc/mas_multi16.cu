// Sixteen right-hand sides at once (sm_100a, block size 3): the wide group kernels.
//
// The group kernels of mas_multi.cu give every lane all G values of its rows (G = 4); at G = 16 that
// would need some 200 registers per lane. Here the mapping follows the interleaved layout (value
// index (node * 3 + component) * 16 + g): a lane keeps one right-hand side g = lane % 16 (or a pair
// of them) and the warp walks a bank's 1,536 values in steps of 32, so loads stay coalesced (128 B
// per 16 lanes) and the registers per lane do not grow with G.
//
//   k_spmv_w       a CTA per bank (grid-stride over banks), a warp per 4 rows: 8 lanes per row, each
//                  with a pair of right-hand sides; the block values are loaded once per row (the
//                  8 lanes read the same address) and the x gathers read 16 contiguous doubles per
//                  column and component. Per-right-hand-side p.Ap / r.r (and b.b) by a deterministic
//                  grid sum; alpha of every right-hand side in the last CTA.
//   k_update_xr_w  r -= alpha_g Ap ; r.r per g ; the level-0 restriction of r (x += alpha_g p only on
//                  true-residual iterations; otherwise in k_update_p_w, see PcgState::x_defer),
//                  summed per bank component in shared memory in node order (48 values per node and
//                  component: 3 components x 16 right-hand sides; within a step of 32 values no two
//                  lanes touch the same sum).
//   k_update_p_w   x_g += alpha_g p_g (deferred) ; p_g = z0_g + prolongation(zc_g) + beta_g p_g.
//   k_restrict_w   the restriction alone (initial residual, true-residual iterations).
//
// One matrix pass serves all sixteen right-hand sides; the MAS apply of the group (every inverse
// read once for sixteen right-hand sides) and the coarse levels are in mas_apply.cu.

#include <algorithm>
#include <mutex>
#include <string>
#include <unordered_map>

#include "mas_common.cuh"

namespace pmas
{
    namespace
    {
        constexpr int G = RHS_WIDE;
        constexpr int VN = 3 * G;   // values per node (3 components x 16 right-hand sides)
        constexpr int WT_ = 256;    // threads per CTA
        constexpr int WW = WT_ / 32;
        static_assert(G == 16, "the lane mappings below assume 16 right-hand sides");

        // ---- SpMV: y = A x (PAP: p.Ap, alpha) or y = b - A x (RESIDUAL: r.r, b.b) ------------
        // Slots (stored blocks) of the warp's four rows go through a ring of SP_STAGES shared-memory
        // stages filled by cp.async SP_STAGES - 1 slots ahead: each lane copies the three 16-byte x
        // pieces it multiplies (x[col][j][2 gq .. 2 gq + 1]) and lanes 0-4 of each row the block's
        // values (four 16-byte pairs, one 8-byte value). The copies need no registers, so a warp keeps
        // five slots of gathers in flight; the columns come from registers loaded at the bank's start
        // (slots gq + 8 i of the row in lane gq's register i, up to SP_MAXLEN slots; longer rows take
        // the plain loop).
        constexpr int SP_STAGES = 4;
        constexpr int SP_XB = 32 * 3 * 16;       // x pieces of the 32 lanes
        constexpr int SP_MB = 4 * 5 * 16;        // block values of the four rows
        constexpr int SP_SB = SP_XB + SP_MB;     // one stage
        constexpr int SP_WARP = SP_STAGES * SP_SB;
        constexpr int SP_SMEM = WW * SP_WARP;
        constexpr int SP_REGS = 8;
        constexpr int SP_MAXLEN = 8 * SP_REGS;
        static_assert(SP_SB % 16 == 0, "16-byte aligned stages");

        // The copies of slot sl (warp-uniform; every lane calls) of the lane's row into its stage: the
        // column from register sl / 8 of lane (row base) + sl % 8, selected without indexing (the
        // registers stay registers), then the lane's three x pieces and, in lanes 0-4 of the row,
        // the block values. Sources are checked (column range, 16-byte alignment): a bad one is
        // recorded in the group's error word and skipped.
        struct ColRegs
        {
            int c0, c1, c2, c3, c4, c5, c6, c7;
        };

        __device__ __forceinline__ void sp_issue(unsigned char *wbase, ColRegs colr, int sl, int len,
                                                 long long u, long long nodes, int lane, int rs, int gq, int rb,
                                                 const double *x, const double *vals, long long s0, PcgState *grp)
        {
            const int r8 = sl >> 3;
            const int reg = r8 < 4 ? (r8 < 2 ? (r8 == 0 ? colr.c0 : colr.c1) : (r8 == 2 ? colr.c2 : colr.c3))
                                   : (r8 < 6 ? (r8 == 4 ? colr.c4 : colr.c5) : (r8 == 6 ? colr.c6 : colr.c7));
            const long long col = __shfl_sync(FULL, reg, (lane & ~7) | (sl & 7));
            if (sl >= len)
                return;
            unsigned char *sp = wbase + (sl % SP_STAGES) * SP_SB;
            const double *blk = vals + (s0 + sl) * 32 * 9;
            const double *xs = x + (col * 3) * G + 2 * gq;
            const bool bad = col < 0 || col >= nodes ||
                             ((reinterpret_cast<uintptr_t>(xs) | reinterpret_cast<uintptr_t>(blk) |
                               reinterpret_cast<uintptr_t>(sp)) &
                              15) != 0;
            if (bad)
            {
                atomicExch(&grp->error, ERR_CUDA);
                return;
            }
#pragma unroll
            for (int j = 0; j < 3; ++j)
                cp_async16_ca(sp + (lane * 3 + j) * 16, xs + j * G);
            if (gq < 4)
                cp_async16_cg(sp + SP_XB + (rs * 5 + gq) * 16, blk + gq * 64 + rb * 2);
            else if (gq == 4)
                cp_async8_ca(sp + SP_XB + (rs * 5 + 4) * 16, blk + 256 + rb);
        }

        template <int MODE>
        __global__ void __launch_bounds__(WT_) k_spmv_w(BankedView A, const double *__restrict__ x,
                                                        double *__restrict__ y, const double *__restrict__ b,
                                                        PcgState *st, ReduceBuf red, int iter, int period)
        {
            extern __shared__ __align__(16) unsigned char sp_smem[];
            PcgState *grp = st + G;
            // The previous iteration's update_p has run: its deferred x update is applied.
            if (MODE == SPMV_PAP && blockIdx.x == 0 && threadIdx.x == 0)
                grp->x_applied = grp->x_defer;
            if (grp->done)
                return;
            if (MODE == SPMV_RESIDUAL && period > 0 && (grp->iter + 1) % period != 0)
                return;
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            const int rs = lane >> 3, gq = lane & 7; // row of the warp's four, pair of right-hand sides
            const int rb = w * 4 + rs;               // row within the bank
            const uint64_t pol = l2_evict_first_policy();
            unsigned char *wbase = sp_smem + (size_t)w * SP_WARP;
            const long long nodes = (long long)A.banks * 32;
            double part[2] = {0.0, 0.0}, bb[2] = {0.0, 0.0};
            for (int bank = blockIdx.x; bank < A.banks; bank += gridDim.x)
            {
                const long long u = (long long)bank * 32 + rb;
                const long long s0 = A.slice[bank];
                const int len = A.rowlen[u];
                int maxlen = max(len, __shfl_xor_sync(FULL, len, 8));
                maxlen = max(maxlen, __shfl_xor_sync(FULL, maxlen, 16));
                double acc[3][2];
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    acc[i][0] = acc[i][1] = 0.0;
                if (maxlen <= SP_MAXLEN)
                {
                    // Columns of slots gq + 8 i of the lane's row (i < 8).
                    auto colat = [&](int i) -> int {
                        const int sl = gq + 8 * i;
                        return sl < len ? ld_stream_s32(A.cols + (s0 + sl) * 32 + rb, pol) : (int)u;
                    };
                    const ColRegs colr{colat(0), colat(1), colat(2), colat(3), colat(4), colat(5), colat(6), colat(7)};
#pragma unroll
                    for (int d = 0; d < SP_STAGES - 1; ++d)
                    {
                        if (d < maxlen)
                            sp_issue(wbase, colr, d, len, u, nodes, lane, rs, gq, rb, x, A.vals, s0, grp);
                        cp_async_commit();
                    }
                    for (int k = 0; k < maxlen; ++k)
                    {
                        if (k + SP_STAGES - 1 < maxlen)
                            sp_issue(wbase, colr, k + SP_STAGES - 1, len, u, nodes, lane, rs, gq, rb, x, A.vals, s0,
                                     grp);
                        cp_async_commit();
                        cp_async_wait<SP_STAGES - 1>();
                        __syncwarp();
                        if (k < len)
                        {
                            const unsigned char *sp = wbase + (k % SP_STAGES) * SP_SB;
                            const double *mv = reinterpret_cast<const double *>(sp + SP_XB + rs * 80);
                            double v[9];
#pragma unroll
                            for (int q = 0; q < 4; ++q)
                            {
                                const double2 t = *reinterpret_cast<const double2 *>(mv + 2 * q);
                                v[2 * q] = t.x;
                                v[2 * q + 1] = t.y;
                            }
                            v[8] = mv[8];
#pragma unroll
                            for (int j = 0; j < 3; ++j)
                            {
                                const double2 xv = *reinterpret_cast<const double2 *>(sp + (lane * 3 + j) * 16);
#pragma unroll
                                for (int i = 0; i < 3; ++i)
                                {
                                    acc[i][0] = fma(v[i * 3 + j], xv.x, acc[i][0]);
                                    acc[i][1] = fma(v[i * 3 + j], xv.y, acc[i][1]);
                                }
                            }
                        }
                        __syncwarp();
                    }
                    cp_async_wait<0>();
                }
                else
                    for (int k = 0; k < maxlen; ++k)
                    {
                        double v[9];
                        long long col = u;
                        if (k < len)
                        {
                            const long long slot = s0 + k;
                            col = ld_stream_s32(A.cols + slot * 32 + rb, pol);
                            const double *blk = A.vals + slot * 32 * 9;
#pragma unroll
                            for (int q = 0; q < 4; ++q)
                            {
                                const double2 t = ld_stream_f64x2(blk + q * 64 + rb * 2, pol);
                                v[2 * q] = t.x;
                                v[2 * q + 1] = t.y;
                            }
                            v[8] = ld_stream_f64(blk + 256 + rb, pol);
                        }
                        else
                        {
#pragma unroll
                            for (int q = 0; q < 9; ++q)
                                v[q] = 0.0;
                        }
#pragma unroll
                        for (int j = 0; j < 3; ++j)
                        {
                            const double2 xv =
                                __ldg(reinterpret_cast<const double2 *>(x + (col * 3 + j) * G + 2 * gq));
#pragma unroll
                            for (int i = 0; i < 3; ++i)
                            {
                                acc[i][0] = fma(v[i * 3 + j], xv.x, acc[i][0]);
                                acc[i][1] = fma(v[i * 3 + j], xv.y, acc[i][1]);
                            }
                        }
                    }
#pragma unroll
                for (int i = 0; i < 3; ++i)
                {
                    const long long idx = (u * 3 + i) * G + 2 * gq;
                    if (MODE == SPMV_PAP)
                    {
                        *reinterpret_cast<double2 *>(y + idx) = make_double2(acc[i][0], acc[i][1]);
                        const double2 xv = *reinterpret_cast<const double2 *>(x + idx);
                        part[0] = fma(acc[i][0], xv.x, part[0]);
                        part[1] = fma(acc[i][1], xv.y, part[1]);
                    }
                    else
                    {
                        const double2 bv = *reinterpret_cast<const double2 *>(b + idx);
                        const double r0 = bv.x - acc[i][0], r1 = bv.y - acc[i][1];
                        *reinterpret_cast<double2 *>(y + idx) = make_double2(r0, r1);
                        part[0] = fma(r0, r0, part[0]);
                        part[1] = fma(r1, r1, part[1]);
                        bb[0] = fma(bv.x, bv.x, bb[0]);
                        bb[1] = fma(bv.y, bv.y, bb[1]);
                    }
                }
            }
            // Per right-hand side: sum the warp's four rows (lanes gq, gq + 8, gq + 16, gq + 24).
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int o = 8; o < 32; o <<= 1)
                {
                    part[h] += __shfl_xor_sync(FULL, part[h], o);
                    bb[h] += __shfl_xor_sync(FULL, bb[h], o);
                }
            __shared__ double wsum[WW][2 * G];
            __shared__ double cta[2 * G], tot[2 * G];
            if (lane < 8)
            {
                wsum[w][2 * lane] = part[0];
                wsum[w][2 * lane + 1] = part[1];
                wsum[w][G + 2 * lane] = bb[0];
                wsum[w][G + 2 * lane + 1] = bb[1];
            }
            __syncthreads();
            if (threadIdx.x < 2 * G)
            {
                double s = 0.0;
                for (int ww = 0; ww < WW; ++ww)
                    s += wsum[ww][threadIdx.x];
                cta[threadIdx.x] = s;
            }
            unsigned *counter = (MODE == SPMV_RESIDUAL && period > 0) ? &grp->counter[2] : &grp->counter[0];
            if (!grid_reduce_cta<2 * G, WT_>(cta, red.partials, counter, tot) || threadIdx.x >= G)
                return;
            const int g = threadIdx.x;
            PcgState &sg = st[g];
            if (MODE == SPMV_RESIDUAL && period > 0)
            {
                if (!sg.done)
                    sg.rr = tot[g];
                return;
            }
            if (sg.done)
            {
                sg.alpha = 0.0; // a finished right-hand side keeps its x and r
                return;
            }
            if (MODE == SPMV_PAP)
            {
                sg.pAp = tot[g];
                sg.alpha = (fabs(tot[g]) < 1e-20) ? 0.0 : sg.rz / tot[g];
            }
            else
            {
                sg.rr = tot[g];
                if (iter == 0)
                    sg.rr0 = tot[G + g];
            }
        }

        // Level-0 restriction of one bank's r values, accumulated in the warp's shared-memory sums
        // (acc: up to 32 components x VN values). Call restrict_begin once per bank, restrict_add for
        // each step of 32 values in increasing order, restrict_end to store the component sums.
        __device__ __forceinline__ int restrict_begin(const MasView &mas, int bank, double *acc, int &lc)
        {
            const int lane = threadIdx.x & 31;
            lc = mas.lcco0[(long long)bank * 32 + lane];
            int m = lc;
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1)
                m = max(m, __shfl_xor_sync(FULL, m, o));
            const int ncco = m + 1;
            for (int i = lane; i < ncco * VN; i += 32)
                acc[i] = 0.0;
            __syncwarp();
            return ncco;
        }

        // Value e (bank-local index) with value v: node e / VN, component-and-g c = e % VN. The 32
        // values of a step are consecutive, so their c differ and no two lanes add to one sum.
        __device__ __forceinline__ void restrict_add(double *acc, int lc, int e, double v)
        {
            const int node = e / VN, c = e - node * VN;
            const int cco = __shfl_sync(FULL, lc, node);
            if (cco >= 0)
                acc[cco * VN + c] += v;
        }

        __device__ __forceinline__ void restrict_end(const MasView &mas, int bank, const double *acc, int ncco)
        {
            const int lane = threadIdx.x & 31;
            __syncwarp();
            double *dst = mas.rc + (size_t)mas.cco0_base[bank] * VN;
            for (int i = lane; i < ncco * VN; i += 32)
                dst[i] = acc[i];
            __syncwarp();
        }

        constexpr int XR_SMEM = WW * 32 * VN * 8; // per-warp component sums (96 KB per CTA)

        __global__ void __launch_bounds__(WT_) k_update_xr_w(MasView mas, double *__restrict__ x,
                                                             double *__restrict__ r, const double *__restrict__ p,
                                                             const double *__restrict__ Ap, PcgState *st,
                                                             ReduceBuf red, int period)
        {
            extern __shared__ double xr_acc[];
            PcgState *grp = st + G;
            if (grp->done)
                return;
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            const double a = st[lane & (G - 1)].alpha;
            const bool due = period > 0 && (grp->iter + 1) % period == 0;
            if (blockIdx.x == 0 && threadIdx.x == 0)
                grp->x_defer = due ? -1 : grp->iter + 1;
            const bool restrict_r = !due && mas.level_num > 0;
            double *acc = xr_acc + (size_t)w * 32 * VN;
            double part = 0.0;
            for (int bank = blockIdx.x * WW + w; bank < mas.banks; bank += gridDim.x * WW)
            {
                const long long b0 = (long long)bank * 32 * VN;
                const bool rs = restrict_r && bank < mas.first_iso_bank;
                int lc = -1, ncco = 0;
                if (rs)
                    ncco = restrict_begin(mas, bank, acc, lc);
                for (int t0 = 0; t0 < VN; t0 += 4)
                {
                    double xv[4], pv[4], av[4], rv[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                    {
                        const long long e = b0 + (t0 + j) * 32 + lane;
                        xv[j] = due ? x[e] : 0.0;
                        pv[j] = due ? p[e] : 0.0;
                        av[j] = due ? 0.0 : Ap[e];
                        rv[j] = due ? 0.0 : r[e];
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                    {
                        const int el = (t0 + j) * 32 + lane;
                        if (due)
                            x[b0 + el] = fma(a, pv[j], xv[j]);
                        if (!due)
                        {
                            rv[j] = fma(-a, av[j], rv[j]);
                            r[b0 + el] = rv[j];
                            part = fma(rv[j], rv[j], part);
                        }
                        if (rs)
                            restrict_add(acc, lc, el, rv[j]);
                    }
                }
                if (rs)
                    restrict_end(mas, bank, acc, ncco);
            }
            if (due)
                return;
            part += __shfl_xor_sync(FULL, part, 16); // lanes g and g + 16 hold right-hand side g
            __shared__ double wsum[WW][G];
            __shared__ double cta[G], tot[G];
            if (lane < G)
                wsum[w][lane] = part;
            __syncthreads();
            if (threadIdx.x < G)
            {
                double s = 0.0;
                for (int ww = 0; ww < WW; ++ww)
                    s += wsum[ww][threadIdx.x];
                cta[threadIdx.x] = s;
            }
            if (grid_reduce_cta<G, WT_>(cta, red.rr_parts, &grp->counter[1], tot) && threadIdx.x < G)
                if (!st[threadIdx.x].done)
                    st[threadIdx.x].rr = tot[threadIdx.x];
        }

        __global__ void __launch_bounds__(WT_) k_restrict_w(MasView mas, const double *__restrict__ r,
                                                            const PcgState *grp, int period)
        {
            extern __shared__ double xr_acc[];
            if (grp->done)
                return;
            if (period > 0 && (grp->iter + 1) % period != 0)
                return;
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            double *acc = xr_acc + (size_t)w * 32 * VN;
            for (int bank = blockIdx.x * WW + w; bank < mas.first_iso_bank; bank += gridDim.x * WW)
            {
                const long long b0 = (long long)bank * 32 * VN;
                int lc = -1;
                const int ncco = restrict_begin(mas, bank, acc, lc);
                for (int t0 = 0; t0 < VN; t0 += 4)
                {
                    double rv[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        rv[j] = r[b0 + (t0 + j) * 32 + lane];
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        restrict_add(acc, lc, (t0 + j) * 32 + lane, rv[j]);
                }
                restrict_end(mas, bank, acc, ncco);
            }
        }

        // p_g = z0_g + sum_l zc_g[cslot_l(node)] + beta_g p_g (first: p = z); a warp per bank.
        __global__ void __launch_bounds__(WT_) k_update_p_w(MasView mas, double *__restrict__ x,
                                                            double *__restrict__ p,
                                                            const double *__restrict__ z0, const PcgState *st,
                                                            int first)
        {
            const PcgState *grp = st + G;
            const int it = grp->iter;
            const bool xdo = !first && grp->x_defer == it && grp->x_applied != it;
            if (grp->done && !xdo)
                return;
            const int lane = threadIdx.x & 31;
            const int bank = blockIdx.x * WW + (threadIdx.x >> 5);
            if (bank >= mas.banks)
                return;
            const int g = lane & (G - 1);
            const double beta = first ? 0.0 : st[g].beta;
            const double a = st[g].alpha;
            const bool skip = st[g].done != 0 || grp->done != 0;
            const double *__restrict__ zc = mas.zc;
            const double iso_scale = 1.0 + mas.level_num;
            const bool iso = bank >= mas.first_iso_bank;
            const long long b0 = (long long)bank * 32 * VN;
            for (int t0 = 0; t0 < VN; t0 += 4)
            {
                double zv[4], po[4], xv[4];
                int4 cs[4];
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    const int el = (t0 + j) * 32 + lane;
                    zv[j] = z0[b0 + el];
                    po[j] = first ? 0.0 : p[b0 + el];
                    xv[j] = xdo ? x[b0 + el] : 0.0;
                    cs[j] = iso ? make_int4(-1, -1, -1, -1) : mas.cslot[(long long)bank * 32 + el / VN];
                }
                if (xdo)
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        x[b0 + (t0 + j) * 32 + lane] = fma(a, po[j], xv[j]);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    const int el = (t0 + j) * 32 + lane;
                    const int c = el % VN;
                    double v;
                    if (iso)
                        v = iso_scale * zv[j];
                    else
                    {
                        const double g0 = zc[(size_t)max(cs[j].x, 0) * VN + c];
                        const double g1 = zc[(size_t)max(cs[j].y, 0) * VN + c];
                        const double g2 = zc[(size_t)max(cs[j].z, 0) * VN + c];
                        const double g3 = zc[(size_t)max(cs[j].w, 0) * VN + c];
                        v = zv[j];
                        v += cs[j].x >= 0 ? g0 : 0.0;
                        v += cs[j].y >= 0 ? g1 : 0.0;
                        v += cs[j].z >= 0 ? g2 : 0.0;
                        v += cs[j].w >= 0 ? g3 : 0.0;
                    }
                    if (!skip)
                        p[b0 + el] = first ? v : fma(beta, po[j], v);
                }
            }
        }

        // Caller columns 0 .. cols - 1 of the column-major B (n x cols) into the interleaved padded
        // layout (missing columns and padding zero), and back.
        __global__ void k_permute_in_w(int n, int V, int cols, const int *__restrict__ padded_of_block,
                                       const double *__restrict__ B, double *__restrict__ dst)
        {
            const long long total = (long long)V * 3 * G;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
                 i += (long long)gridDim.x * blockDim.x)
            {
                const long long row = i / G;
                const int g = (int)(i % G);
                const int blk = (int)(row / 3), c = (int)(row % 3);
                const double v = (g < cols && row < n) ? B[(long long)g * n + row] : 0.0;
                dst[((long long)padded_of_block[blk] * 3 + c) * G + g] = v;
            }
        }

        __global__ void k_permute_out_w(int n, int cols, const int *__restrict__ padded_of_block,
                                        const double *__restrict__ src, double *__restrict__ X)
        {
            const long long total = (long long)n * cols;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
                 i += (long long)gridDim.x * blockDim.x)
            {
                const int g = (int)(i / n);
                const long long row = i % n;
                const int blk = (int)(row / 3), c = (int)(row % 3);
                X[i] = src[((long long)padded_of_block[blk] * 3 + c) * G + g];
            }
        }

        int cap_grid(long long n)
        {
            long long g = (n + 255) / 256;
            const long long cap = (long long)device_sm_count() * 16;
            if (g > cap)
                g = cap;
            return (int)(g < 1 ? 1 : g);
        }

        template <class K>
        int resident_per_sm(K kernel, int smem)
        {
            static std::mutex mu;
            static std::unordered_map<const void *, int> cache;
            std::lock_guard<std::mutex> lock(mu);
            auto it = cache.find((const void *)kernel);
            if (it != cache.end())
                return it->second;
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, WT_, smem) != cudaSuccess || per_sm < 1)
            {
                cudaGetLastError();
                per_sm = 1;
            }
            cache[(const void *)kernel] = per_sm;
            return per_sm;
        }
    } // namespace

    int wide_reduce_ctas() { return device_sm_count() * 16; }

    void prepare_kernels_w()
    {
        cuda_check(cudaFuncSetAttribute(k_spmv_w<SPMV_PAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, SP_SMEM),
                   "wide spmv smem attribute");
        cuda_check(cudaFuncSetAttribute(k_spmv_w<SPMV_RESIDUAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, SP_SMEM),
                   "wide spmv smem attribute");
        cuda_check(cudaFuncSetAttribute(k_update_xr_w, cudaFuncAttributeMaxDynamicSharedMemorySize, XR_SMEM),
                   "wide update smem attribute");
        cuda_check(cudaFuncSetAttribute(k_restrict_w, cudaFuncAttributeMaxDynamicSharedMemorySize, XR_SMEM),
                   "wide restrict smem attribute");
    }

    void launch_spmv_w(int mode, const BankedView &A, const double *x, double *y, const double *b, PcgState *st,
                       ReduceBuf red, int iter, int period, cudaStream_t s)
    {
        if (A.bd != 3)
            throw Error(ERR_INVALID, "[MAS] sixteen right-hand sides need block_dim 3");
        if (A.banks == 0)
            return;
        auto go = [&](auto kernel) {
            int grid = resident_per_sm(kernel, SP_SMEM) * device_sm_count();
            grid = std::min({grid, A.banks, red.capacity});
            kernel<<<grid, WT_, SP_SMEM, s>>>(A, x, y, b, st, red, iter, period);
        };
        if (mode == SPMV_PAP)
            go(k_spmv_w<SPMV_PAP>);
        else
            go(k_spmv_w<SPMV_RESIDUAL>);
        cuda_check(cudaGetLastError(), "wide spmv launch");
    }

    void launch_update_xr_w(const MasView &mas, double *x, double *r, const double *p, const double *Ap,
                            PcgState *st, ReduceBuf red, int period, cudaStream_t s)
    {
        int grid = resident_per_sm(k_update_xr_w, XR_SMEM) * device_sm_count();
        grid = std::min({grid, (mas.banks + WW - 1) / WW, red.capacity});
        grid = std::max(grid, 1);
        k_update_xr_w<<<grid, WT_, XR_SMEM, s>>>(mas, x, r, p, Ap, st, red, period);
        cuda_check(cudaGetLastError(), "wide update_xr launch");
    }

    void launch_update_p_w(const MasView &mas, double *x, double *p, const double *z0, PcgState *st, int first,
                           cudaStream_t s)
    {
        const int grid = (mas.banks + WW - 1) / WW;
        if (grid > 0)
            k_update_p_w<<<grid, WT_, 0, s>>>(mas, x, p, z0, st, first);
        cuda_check(cudaGetLastError(), "wide update_p launch");
    }

    int launch_restrict_w(const MasView &mas, const double *r, const PcgState *grp, int period, cudaStream_t s)
    {
        if (mas.first_iso_bank <= 0 || mas.level_num <= 0)
            return 0;
        int grid = resident_per_sm(k_restrict_w, XR_SMEM) * device_sm_count();
        grid = std::min(grid, (mas.first_iso_bank + WW - 1) / WW);
        k_restrict_w<<<grid, WT_, XR_SMEM, s>>>(mas, r, grp, period);
        cuda_check(cudaGetLastError(), "wide restrict launch");
        return 1;
    }

    void launch_permute_in_w(int n, int V, int cols, const int *padded_of_block, const double *B, double *dst,
                             size_t dst_len, cudaStream_t s)
    {
        launch_zero(dst, dst_len, s);
        k_permute_in_w<<<cap_grid((long long)V * 3 * G), 256, 0, s>>>(n, V, cols, padded_of_block, B, dst);
        cuda_check(cudaGetLastError(), "wide permute_in launch");
    }

    void launch_permute_out_w(int n, int cols, const int *padded_of_block, const double *src, double *X,
                              cudaStream_t s)
    {
        k_permute_out_w<<<cap_grid((long long)n * cols), 256, 0, s>>>(n, cols, padded_of_block, src, X);
        cuda_check(cudaGetLastError(), "wide permute_out launch");
    }
} // namespace pmas
