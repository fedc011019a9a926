// MAS preconditioner apply (sm_100a): z = sum_l P_l A_l^-1 P_l^T r.
//
// The reference (MASPreconditioner.cu:1099-1164) zeroes two multi-level vectors, restricts with
// warp segmented sums plus FP64 atomics, multiplies every level's packed 96 x 96 inverse with one
// 96-thread CTA each (symv_upper_packed, :665-705), and prolongs in a third kernel. Here:
//
//  * k_restrict: the level-0 restriction (per-bank sums of each connected component),
//    deterministic, first kernel of the coarse chain;
//  * k_coarse_sum: coarse level l sums from level l-1 (every level-l component merges at most 32
//    level-(l-1) components of one bank), one warp per component, one launch per level;
//  * k_coarse_symv: one CTA per coarse matrix (one warp per column tile, matrix read from global
//    memory), zc = A_l^-1 rc, and rc . zc for the PCG dot (identity inverses -- banks of isolated
//    rows -- skip the multiply);
//  * k_symv0: persistent warps stream the level-0 inverses through shared memory with
//    cp.async.bulk (two stages per warp, mbarrier completion) and write z0 = A_0^-1 r with per-CTA
//    r . z0. The coarse levels do not feed it, so the host runs them concurrently on a second
//    stream; k_finalize (one CTA, after the join) sums the partials and runs the reference's PCG
//    bookkeeping (rz = r . z0 + rc . zc, convergence, beta). The prolongation z = z0 + P zc is fused
//    into the p update (update_p): PCG uses z only there and in r . z = r . z0 + (P^T r) . zc.
//
// Inverses are stored tile-packed (mas_internal.h): the same N (N + 1) / 2 values as packed upper
// storage, laid out so a warp reads every 32 x 32 tile conflict-free and uses each value for both
// y_I += T x_J and y_J += T^T x_I; the transposed sums are combined across lanes with a
// 31-shuffle reduce-transpose per column tile.

#include "mas_common.cuh"

namespace pmas
{
    namespace
    {
        template <class Real>
        struct Vec4;
        template <>
        struct Vec4<float>
        {
            using type = float4;
        };
        template <>
        struct Vec4<double>
        {
            using type = double4;
        };

        // Lane l receives sum over lanes of c[l]; c is destroyed. 31 shuffles.
        template <class Real>
        __device__ __forceinline__ Real transpose_sum32(Real (&c)[32], int lane)
        {
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1)
            {
                const bool upper = (lane & s) != 0;
#pragma unroll
                for (int i = 0; i < s; ++i)
                {
                    const Real send = upper ? c[i] : c[i + s];
                    const Real keep = upper ? c[i + s] : c[i];
                    c[i] = keep + __shfl_xor_sync(FULL, send, s);
                }
            }
            return c[0];
        }

        // Column tile J of y = M x for one tile-packed symmetric matrix (shared memory): adds the
        // row contributions of tiles (I, J), I <= J, to yr[I] and the transposed contributions
        // (rows of tile J) to yr[J]. Lane l owns rows 32 t + l.
        template <int T, class Real>
        __device__ __forceinline__ void symv_column(const Real *__restrict__ M, const Real *__restrict__ xs, int lane,
                                                    int J, Real (&yr)[T])
        {
            using V4 = typename Vec4<Real>::type;
            int off = 0;
#pragma unroll
            for (int jj = 0; jj < T; ++jj)
                if (jj < J)
                    off += jj * 1024 + 528;
            Real cy[32];
#pragma unroll
            for (int j = 0; j < 32; ++j)
                cy[j] = Real(0);
#pragma unroll
            for (int I = 0; I < T; ++I)
            {
                if (I >= J)
                    break;
                const Real *tile = M + off + I * 1024;
                const Real xI = xs[32 * I + lane];
                Real a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
                for (int j4 = 0; j4 < 8; ++j4)
                {
                    const V4 v = *reinterpret_cast<const V4 *>(tile + j4 * 128 + lane * 4);
                    const V4 xv = *reinterpret_cast<const V4 *>(xs + 32 * J + 4 * j4);
                    a0 = fma(v.x, xv.x, a0);
                    a1 = fma(v.y, xv.y, a1);
                    a2 = fma(v.z, xv.z, a2);
                    a3 = fma(v.w, xv.w, a3);
                    cy[4 * j4 + 0] = fma(v.x, xI, cy[4 * j4 + 0]);
                    cy[4 * j4 + 1] = fma(v.y, xI, cy[4 * j4 + 1]);
                    cy[4 * j4 + 2] = fma(v.z, xI, cy[4 * j4 + 2]);
                    cy[4 * j4 + 3] = fma(v.w, xI, cy[4 * j4 + 3]);
                }
                yr[I] += (a0 + a1) + (a2 + a3);
            }
            // Diagonal tile, upper triangle by columns.
            const Real *dt = M + off + J * 1024;
            const Real xJ = xs[32 * J + lane];
            Real a0 = 0, a1 = 0;
#pragma unroll
            for (int j = 0; j < 32; ++j)
            {
                const Real v = (lane <= j) ? dt[j * (j + 1) / 2 + lane] : Real(0);
                const Real xj = xs[32 * J + j];
                if (j & 1)
                    a1 = fma(v, xj, a1);
                else
                    a0 = fma(v, xj, a0);
                cy[j] = fma((lane < j) ? v : Real(0), xJ, cy[j]);
            }
            yr[J] += (a0 + a1) + transpose_sum32<Real>(cy, lane);
        }

        // y = M x by one warp (all column tiles).
        template <int T, class Real>
        __device__ __forceinline__ void symv_tiles(const Real *__restrict__ M, const Real *__restrict__ xs, int lane,
                                                   Real (&yr)[T])
        {
#pragma unroll
            for (int t = 0; t < T; ++t)
                yr[t] = Real(0);
#pragma unroll
            for (int J = 0; J < T; ++J)
                symv_column<T, Real>(M, xs, lane, J, yr);
        }

        // Finish of an iteration (last CTA of k_symv0): the reference's per-iteration scalar work
        // and convergence test (MASSolver.cu:505, 526-583), on the device.
        __device__ void pcg_finalize(PcgState *st, const PcgConfig &cfg, int mode, double rz_fine, double rzx_fine)
        {
            int iter;
            const double rz = rz_fine + st->rz_coarse;
            const double rzcross = rzx_fine + st->rzx_coarse;
            if (mode == 1)
            {
                st->rz = rz;
                st->rz0 = rz;
                st->iter = 0;
                if (isnan(rz) || !isfinite(rz))
                {
                    st->error = ERR_NONFINITE;
                    st->done = 1;
                }
                return;
            }
            // Iteration number from the device state, so a captured chunk of iterations replays.
            iter = st->iter + 1;
            const double rz_old = st->rz;
            st->rz_old = rz_old;
            st->rz = rz;
            st->rzold_cross = rzcross;
            st->iter = iter;
            bool conv = false;
            if (iter % cfg.check_period == 0)
            {
                const double rel2 = cfg.rel_tol * cfg.rel_tol, abs2 = cfg.abs_tol * cfg.abs_tol;
                if (cfg.use_prec_norm)
                {
                    st->res_norm = sqrt(rz);
                    if (rz <= rel2 * st->rz0 || rz <= abs2)
                    {
                        st->status = (rz <= abs2) ? 2 : 1;
                        conv = true;
                    }
                }
                else
                {
                    const double rr = st->rr;
                    st->res_norm = sqrt(rr);
                    if (rr <= rel2 * st->rr0 || rr <= abs2)
                    {
                        st->status = (rr <= abs2) ? 2 : 1;
                        conv = true;
                    }
                }
            }
            if (conv)
                st->done = 1;
            else if (cfg.polak_ribiere)
            {
                const double beta = (fabs(rz_old) < 1e-20) ? 0.0 : (rz - rzcross) / rz_old;
                st->beta = beta > 0.0 ? beta : 0.0;
            }
            else
                st->beta = (fabs(rz_old) < 1e-20) ? 0.0 : rz / rz_old;
            if (iter == cfg.max_iter)
            {
                st->status = 3;
                st->done = 1;
            }
        }

        template <int BD, class Real>
        struct Symv0Layout
        {
            static constexpr int N = 32 * BD;
            static constexpr int S = N * (N + 1) / 2;
            static constexpr int STAGE_BYTES = S * (int)sizeof(Real);
            static constexpr int XS_BYTES = ((N * (int)sizeof(Real)) + 15) / 16 * 16;
            static constexpr int WARP_BYTES = 2 * STAGE_BYTES + XS_BYTES + 16;
            static constexpr int SMEM_LIMIT = 232448 - 1024; // leave room for static shared memory
            static constexpr int W0 = SMEM_LIMIT / WARP_BYTES;
            static constexpr int WARPS = W0 > 16 ? 16 : W0;
            static_assert(STAGE_BYTES % 16 == 0, "bulk copies need 16-byte multiples");
        };

        // mode 0: plain apply; 1: initial PCG apply (rz0); 2: PCG iteration.
        template <int BD, class Real, int MODE>
        __global__ void __launch_bounds__(Symv0Layout<BD, Real>::WARPS * 32)
            k_symv0(MasView mas, const double *__restrict__ r, double *__restrict__ z0, PcgState *st, ReduceBuf red,
                    PcgConfig cfg, int iter)
        {
            using L = Symv0Layout<BD, Real>;
            constexpr int N = L::N, S = L::S, WARPS = L::WARPS;
            constexpr int THREADS = WARPS * 32;
            if (MODE != 0 && st->done)
                return;
            extern __shared__ __align__(128) unsigned char smem[];
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            unsigned char *base = smem + (size_t)w * L::WARP_BYTES;
            Real *stage0 = reinterpret_cast<Real *>(base);
            Real *stage1 = reinterpret_cast<Real *>(base + L::STAGE_BYTES);
            Real *xs = reinterpret_cast<Real *>(base + 2 * L::STAGE_BYTES);
            uint64_t *bar = reinterpret_cast<uint64_t *>(base + 2 * L::STAGE_BYTES + L::XS_BYTES);
            const Real *__restrict__ inv = static_cast<const Real *>(mas.inv);
            const int banks = mas.banks;
            const int total_warps = gridDim.x * WARPS;
            const int gw = blockIdx.x * WARPS + w;
            int *errp = st ? &st->error : nullptr;
            const bool pr = (MODE == 2) && cfg.polak_ribiere;

            if (lane == 0)
            {
                mbar_init(&bar[0], 1);
                mbar_init(&bar[1], 1);
                fence_mbar_init();
            }
            __syncwarp();
            if (lane == 0)
            {
                if (gw < banks)
                    bulk_load(stage0, inv + (size_t)gw * S, L::STAGE_BYTES, &bar[0]);
                if (gw + total_warps < banks)
                    bulk_load(stage1, inv + (size_t)(gw + total_warps) * S, L::STAGE_BYTES, &bar[1]);
            }
            double part[4] = {0.0, 0.0, 0.0, 0.0}; // r.z0, r.z0_old; the same over isolated banks
            uint32_t phase0 = 0, phase1 = 0;
            bool ok = true;
            // r of the current bank, prefetched one bank ahead.
            double r_next[BD];
            if (gw < banks)
#pragma unroll
                for (int t = 0; t < BD; ++t)
                    r_next[t] = r[(size_t)gw * N + t * 32 + lane];
            int k = 0;
            for (int m = gw; m < banks; m += total_warps, ++k)
            {
                const bool s1 = (k & 1) != 0;
                Real *stage = s1 ? stage1 : stage0;
                uint64_t *b = s1 ? &bar[1] : &bar[0];
                double r64[BD];
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    r64[t] = r_next[t];
                    xs[t * 32 + lane] = (Real)r64[t];
                }
                const int mnext = m + total_warps;
                if (mnext < banks)
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                        r_next[t] = r[(size_t)mnext * N + t * 32 + lane];
                double zold[BD];
                if (pr)
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                        zold[t] = z0[(size_t)m * N + t * 32 + lane];
                __syncwarp();
                if (!mbar_wait_bounded(b, s1 ? phase1 : phase0, errp))
                {
                    ok = false;
                    break;
                }
                if (s1)
                    phase1 ^= 1u;
                else
                    phase0 ^= 1u;
                Real yr[BD];
                symv_tiles<BD, Real>(stage, xs, lane, yr);
                __syncwarp();
                const int mn = m + 2 * total_warps;
                if (lane == 0 && mn < banks)
                {
                    fence_proxy_async_smem();
                    bulk_load(stage, inv + (size_t)mn * S, L::STAGE_BYTES, b);
                }
                const int off = (m >= mas.first_iso_bank) ? 2 : 0;
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    const double zv = (double)yr[t];
                    z0[(size_t)m * N + t * 32 + lane] = zv;
                    part[off] = fma(zv, r64[t], part[off]);
                    if (pr)
                        part[off + 1] = fma(zold[t], r64[t], part[off + 1]);
                }
            }
            if (!ok)
            {
                // Drain this warp's other outstanding copy (bounded) before leaving.
                if (lane == 0)
                {
                    for (long long i = 0; i < MBAR_SPIN_LIMIT; ++i)
                        if (mbar_try_wait(&bar[0], phase0) && mbar_try_wait(&bar[1], phase1))
                            break;
                }
                __syncwarp();
            }
            if (MODE == 0)
                return;
            double t[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
                t[i] = block_sum<THREADS>(part[i]);
            if (threadIdx.x == 0)
            {
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    red.rz_parts[4 * blockIdx.x + i] = t[i];
                if (blockIdx.x == 0)
                    st->n_rz = gridDim.x;
            }
        }

        // The iteration's bookkeeping in one CTA: sum the per-CTA partials in a fixed order (1024
        // threads, loads unrolled so each thread has its few loads in flight at once).
        constexpr int FIN_THREADS = 1024;
        __global__ void __launch_bounds__(FIN_THREADS) k_finalize(PcgState *st, ReduceBuf red, PcgConfig cfg, int mode)
        {
            if (st->done)
                return;
            const int n_rz = st->n_rz, n_co = st->n_co, n_rr = (mode == 2) ? st->n_rr : 0;
            double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
            for (int i = threadIdx.x; i < n_rz; i += FIN_THREADS)
            {
                v[0] += __ldcg(red.rz_parts + 4 * i);
                v[1] += __ldcg(red.rz_parts + 4 * i + 1);
                v[5] += __ldcg(red.rz_parts + 4 * i + 2);
                v[6] += __ldcg(red.rz_parts + 4 * i + 3);
            }
#pragma unroll 4
            for (int i = threadIdx.x; i < n_co; i += FIN_THREADS)
            {
                v[2] += __ldcg(red.co_parts + 2 * i);
                v[3] += __ldcg(red.co_parts + 2 * i + 1);
            }
#pragma unroll 4
            for (int i = threadIdx.x; i < n_rr; i += FIN_THREADS)
                v[4] += __ldcg(red.rr_parts + i);
            double t[7];
#pragma unroll
            for (int i = 0; i < 7; ++i)
                t[i] = block_sum<FIN_THREADS>(v[i]);
            if (threadIdx.x == 0)
            {
                // Isolated rows: z = (1 + L) z0, so their r.z is (1 + L) r.z0 -- r.z0 is already in
                // the level-0 sums, the coarse levels add L r.z0.
                const double L = (double)cfg.level_num;
                st->rz_coarse = t[2] + L * t[5];
                st->rzx_coarse = t[3] + L * t[6];
                if (mode == 2)
                    st->rr = t[4];
                pcg_finalize(st, cfg, mode, t[0] + t[5], t[1] + t[6]);
            }
        }

        // Coarse level l sums: rc[node] = sum of rc over its <= 32 children (previous level).
        template <int BD>
        __global__ void k_coarse_sum(MasView mas, int first_node, int count, const PcgState *st)
        {
            if (st && st->done)
                return;
            const int lane = threadIdx.x & 31;
            const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            if (i >= count)
                return;
            const int cn = first_node + i;
            const int b = mas.child_ptr[cn], e = mas.child_ptr[cn + 1];
            double s[BD];
#pragma unroll
            for (int c = 0; c < BD; ++c)
                s[c] = 0.0;
            if (b + lane < e)
            {
                const int ch = mas.children[b + lane];
#pragma unroll
                for (int c = 0; c < BD; ++c)
                    s[c] = mas.rc[(size_t)ch * BD + c];
            }
#pragma unroll
            for (int c = 0; c < BD; ++c)
            {
                const double v = warp_sum(s[c]);
                if (lane == 0)
                    mas.rc[(size_t)cn * BD + c] = v;
            }
        }

        // One CTA (BD warps, one per column tile) per coarse matrix: zc = A^-1 rc on its 32 coarse
        // nodes; in PCG modes per-CTA rc . zc (and rc . zc_old). The matrix is read straight from
        // global memory (each warp's tile reads are coalesced), so a CTA needs only ~2 KB of shared
        // memory and can run beside the level-0 kernel, which holds most of every SM's.
        template <int BD, class Real, int PCG>
        __global__ void __launch_bounds__(BD * 32) k_coarse_symv(MasView mas, PcgState *st, ReduceBuf red, int pr)
        {
            constexpr int N = 32 * BD, S = N * (N + 1) / 2;
            if (PCG && st->done)
                return;
            __shared__ __align__(16) Real xs[N];
            __shared__ Real ypart[BD][N];
            const int g = mas.coarse_active[blockIdx.x];
            const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
            const size_t v0 = (size_t)g * N; // first coarse value of this matrix
            double part[2] = {0.0, 0.0};
            double rcv[BD], zold[BD];
#pragma unroll
            for (int t = 0; t < BD; ++t)
                zold[t] = 0.0;
            if (w == 0)
            {
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    rcv[t] = mas.rc[v0 + t * 32 + lane];
                    if (PCG && pr)
                        zold[t] = mas.zc[v0 + t * 32 + lane];
                }
            }
            if (mas.identity[g])
            {
                if (w == 0)
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                    {
                        mas.zc[v0 + t * 32 + lane] = rcv[t];
                        part[0] = fma(rcv[t], rcv[t], part[0]);
                        part[1] = fma(rcv[t], zold[t], part[1]);
                    }
            }
            else
            {
                const Real *M = static_cast<const Real *>(mas.inv) + (size_t)(mas.banks + g) * S;
                for (int i = tid; i < N; i += BD * 32)
                    xs[i] = (Real)mas.rc[v0 + i];
                __syncthreads();
                Real yr[BD];
#pragma unroll
                for (int t = 0; t < BD; ++t)
                    yr[t] = Real(0);
                symv_column<BD, Real>(M, xs, lane, w, yr);
#pragma unroll
                for (int t = 0; t < BD; ++t)
                    ypart[w][t * 32 + lane] = (t <= w) ? yr[t] : Real(0);
                __syncthreads();
                if (w == 0)
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                    {
                        Real y = Real(0);
#pragma unroll
                        for (int J = 0; J < BD; ++J)
                            y += ypart[J][t * 32 + lane];
                        const double zv = (double)y;
                        mas.zc[v0 + t * 32 + lane] = zv;
                        part[0] = fma(rcv[t], zv, part[0]);
                        part[1] = fma(rcv[t], zold[t], part[1]);
                    }
            }
            if (!PCG)
                return;
            const double t0 = block_sum<BD * 32>(part[0]);
            const double t1 = block_sum<BD * 32>(part[1]);
            if (threadIdx.x == 0)
            {
                red.co_parts[2 * blockIdx.x] = t0;
                red.co_parts[2 * blockIdx.x + 1] = t1;
                if (blockIdx.x == 0)
                    st->n_co = gridDim.x;
            }
        }

        // Level-0 restriction: per bank, the sum of r over each connected component (first coarse
        // level). One warp per bank; the bank's 32 * BD values are read coalesced (value e = t * 32
        // + lane) and regrouped by node with shuffles -- no shared memory, so these CTAs fit beside
        // the level-0 MAS kernel. Sums in a fixed order (deterministic).
        template <int BD>
        __global__ void __launch_bounds__(256) k_restrict(int banks, const double *__restrict__ r,
                                                          const int *__restrict__ lcco0,
                                                          const int *__restrict__ cco0_base, double *rc,
                                                          const PcgState *st)
        {
            if (st && st->done)
                return;
            const int lane = threadIdx.x & 31;
            const int bank = blockIdx.x * 8 + (threadIdx.x >> 5);
            if (bank >= banks)
                return;
            const long long b0 = (long long)bank * 32 * BD;
            double reg[BD];
#pragma unroll
            for (int t = 0; t < BD; ++t)
                reg[t] = r[b0 + t * 32 + lane];
            double rv[BD];
#pragma unroll
            for (int i = 0; i < BD; ++i)
            {
                const int e = lane * BD + i; // this lane's node component i
                const int src = e & 31, tsel = e >> 5;
                double v = 0.0;
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    const double got = __shfl_sync(FULL, reg[t], src);
                    if (t == tsel)
                        v = got;
                }
                rv[i] = v;
            }
            warp_segment_store<BD>(rv, lcco0[(long long)bank * 32 + lane], cco0_base[bank], rc);
        }

        template <int BD>
        __global__ void k_prolong(MasView mas, const double *__restrict__ z0, double *__restrict__ z)
        {
            const long long len = (long long)mas.banks * 32 * BD;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
                 i += (long long)gridDim.x * blockDim.x)
            {
                const long long node = i / BD;
                const int comp = (int)(i % BD);
                if ((node >> 5) >= mas.first_iso_bank)
                {
                    z[i] = (1.0 + mas.level_num) * z0[i];
                    continue;
                }
                const int4 cs = mas.cslot[node];
                double v = z0[i];
                if (cs.x >= 0)
                    v += mas.zc[(size_t)cs.x * BD + comp];
                if (cs.y >= 0)
                    v += mas.zc[(size_t)cs.y * BD + comp];
                if (cs.z >= 0)
                    v += mas.zc[(size_t)cs.z * BD + comp];
                if (cs.w >= 0)
                    v += mas.zc[(size_t)cs.w * BD + comp];
                z[i] = v;
            }
        }

        template <int BD, class Real>
        void prepare_variant()
        {
            using L = Symv0Layout<BD, Real>;
            const int smem = L::WARPS * L::WARP_BYTES;
            cuda_check(cudaFuncSetAttribute(k_symv0<BD, Real, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "symv0 smem attribute");
            cuda_check(cudaFuncSetAttribute(k_symv0<BD, Real, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "symv0 smem attribute");
            cuda_check(cudaFuncSetAttribute(k_symv0<BD, Real, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "symv0 smem attribute");
        }

        template <int BD, class Real>
        int coarse_launch(const MasView &mas, const double *r, PcgState *st, ReduceBuf red, int mode, int pr,
                          cudaStream_t s)
        {
            int launches = 0;
            if (mas.first_iso_bank > 0)
            {
                k_restrict<BD><<<(mas.first_iso_bank + 7) / 8, 256, 0, s>>>(mas.first_iso_bank, r, mas.lcco0,
                                                                           mas.cco0_base, mas.rc, mode ? st : nullptr);
                ++launches;
            }
            if (mas.total_coarse == 0)
            {
                if (mode != 0)
                    cuda_check(cudaMemsetAsync(&st->n_co, 0, sizeof(int), s), "memset");
                return launches;
            }
            for (int l = 1; l < mas.level_num; ++l)
            {
                const int count = mas.real_count[l];
                if (count <= 0)
                    continue;
                k_coarse_sum<BD><<<(count + 7) / 8, 256, 0, s>>>(mas, mas.coff[l], count, mode ? st : nullptr);
                ++launches;
            }
            const int pcg = mode != 0 ? 1 : 0;
            if (pcg)
            {
                if (mas.n_coarse_active > red.capacity)
                    throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
                if (mas.n_coarse_active > 0)
                    k_coarse_symv<BD, Real, 1><<<mas.n_coarse_active, BD * 32, 0, s>>>(mas, st, red, pr);
                else
                    cuda_check(cudaMemsetAsync(&st->n_co, 0, sizeof(int), s), "memset");
            }
            else if (mas.n_coarse_active > 0)
                k_coarse_symv<BD, Real, 0><<<mas.n_coarse_active, BD * 32, 0, s>>>(mas, st, red, 0);
            ++launches;
            cuda_check(cudaGetLastError(), "coarse launch");
            return launches;
        }

        template <int BD, class Real, int MODE>
        void symv0_launch_mode(const MasView &mas, const double *r, double *z, PcgState *st, ReduceBuf red,
                               PcgConfig cfg, int iter, cudaStream_t s)
        {
            using L = Symv0Layout<BD, Real>;
            const int sms = device_sm_count();
            const size_t smem = (size_t)L::WARPS * L::WARP_BYTES;
            int grid = (mas.banks + L::WARPS - 1) / L::WARPS;
            if (grid > sms)
                grid = sms;
            if (grid < 1)
                grid = 1;
            if (MODE != 0 && grid > red.capacity)
                throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
            k_symv0<BD, Real, MODE><<<grid, L::WARPS * 32, smem, s>>>(mas, r, z, st, red, cfg, iter);
            cuda_check(cudaGetLastError(), "symv0 launch");
        }

        template <int BD, class Real>
        void symv0_launch(const MasView &mas, const double *r, double *z, PcgState *st, ReduceBuf red, PcgConfig cfg,
                          int iter, int mode, cudaStream_t s)
        {
            if (mode == 0)
                symv0_launch_mode<BD, Real, 0>(mas, r, z, st, red, cfg, iter, s);
            else if (mode == 1)
                symv0_launch_mode<BD, Real, 1>(mas, r, z, st, red, cfg, iter, s);
            else
                symv0_launch_mode<BD, Real, 2>(mas, r, z, st, red, cfg, iter, s);
        }
    } // namespace

    int device_sm_count()
    {
        static int cached_dev = -1, cached = 148;
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev != cached_dev)
        {
            int v = 0;
            if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
                cached = v;
            cached_dev = dev;
        }
        return cached;
    }

    void prepare_kernels(int bd, int fp32)
    {
        device_sm_count();
        if (fp32)
        {
            if (bd == 1)
                prepare_variant<1, float>();
            else if (bd == 2)
                prepare_variant<2, float>();
            else
                prepare_variant<3, float>();
        }
        else
        {
            if (bd == 1)
                prepare_variant<1, double>();
            else if (bd == 2)
                prepare_variant<2, double>();
            else
                prepare_variant<3, double>();
        }
    }

    int launch_coarse(const MasView &mas, const double *r, PcgState *st, ReduceBuf red, int mode, int pr,
                      cudaStream_t s)
    {
        if (mas.fp32)
        {
            if (mas.bd == 1)
                return coarse_launch<1, float>(mas, r, st, red, mode, pr, s);
            if (mas.bd == 2)
                return coarse_launch<2, float>(mas, r, st, red, mode, pr, s);
            return coarse_launch<3, float>(mas, r, st, red, mode, pr, s);
        }
        if (mas.bd == 1)
            return coarse_launch<1, double>(mas, r, st, red, mode, pr, s);
        if (mas.bd == 2)
            return coarse_launch<2, double>(mas, r, st, red, mode, pr, s);
        return coarse_launch<3, double>(mas, r, st, red, mode, pr, s);
    }

    void launch_symv0(const MasView &mas, const double *r, double *z, PcgState *st, ReduceBuf red, PcgConfig cfg,
                      int iter, int mode, cudaStream_t s)
    {
        if (mas.fp32)
        {
            if (mas.bd == 1)
                symv0_launch<1, float>(mas, r, z, st, red, cfg, iter, mode, s);
            else if (mas.bd == 2)
                symv0_launch<2, float>(mas, r, z, st, red, cfg, iter, mode, s);
            else
                symv0_launch<3, float>(mas, r, z, st, red, cfg, iter, mode, s);
        }
        else
        {
            if (mas.bd == 1)
                symv0_launch<1, double>(mas, r, z, st, red, cfg, iter, mode, s);
            else if (mas.bd == 2)
                symv0_launch<2, double>(mas, r, z, st, red, cfg, iter, mode, s);
            else
                symv0_launch<3, double>(mas, r, z, st, red, cfg, iter, mode, s);
        }
    }

    void launch_finalize(PcgState *st, ReduceBuf red, PcgConfig cfg, int mode, cudaStream_t s)
    {
        k_finalize<<<1, FIN_THREADS, 0, s>>>(st, red, cfg, mode);
        cuda_check(cudaGetLastError(), "finalize launch");
    }

    void launch_prolong(const MasView &mas, const double *z0, double *z, cudaStream_t s)
    {
        const long long len = (long long)mas.banks * 32 * mas.bd;
        long long g = (len + 255) / 256;
        if (g > 148 * 16)
            g = 148 * 16;
        if (g < 1)
            g = 1;
        if (mas.bd == 1)
            k_prolong<1><<<(int)g, 256, 0, s>>>(mas, z0, z);
        else if (mas.bd == 2)
            k_prolong<2><<<(int)g, 256, 0, s>>>(mas, z0, z);
        else
            k_prolong<3><<<(int)g, 256, 0, s>>>(mas, z0, z);
        cuda_check(cudaGetLastError(), "prolong launch");
    }
} // namespace pmas
