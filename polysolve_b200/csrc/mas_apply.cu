// MAS preconditioner apply (sm_100a): z = sum_l P_l A_l^-1 P_l^T r.
//
// The reference (MASPreconditioner.cu:1099-1164) zeroes two multi-level vectors, restricts with
// warp segmented sums plus FP64 atomics, multiplies every level's packed 96 x 96 inverse with one
// 96-thread CTA each (symv_upper_packed, :665-705), and prolongs in a third kernel. Here a PCG
// iteration's apply is two launches:
//
//  * the level-0 restriction (per-bank sums of each connected component) is fused into the kernel
//    that produces r (update_xr; k_restrict after a true-residual SpMV);
//  * k_coarse_levels: every coarse level above the first in one launch -- one CTA per third-level
//    node sums its second-level children (a warp each, lane per child) and then itself, so both
//    levels take one round; the last CTA to finish (atomic ticket) sums a fourth level;
//  * k_mas_apply: persistent warps stream every inverse -- the level-0 subdomain matrices, then
//    the active coarse matrices -- through shared memory with cp.async.bulk (two stages per warp,
//    mbarrier completion) and write z0 = A_0^-1 r and zc = A_l^-1 rc with per-CTA partial dots;
//    the last CTA (atomic ticket) sums them in a fixed order and runs the reference's per-iteration
//    scalar work and convergence test. The prolongation z = z0 + P zc is fused into the p update
//    (update_p): PCG uses z only there and in r . z = r . z0 + (P^T r) . zc.
//
// Inverses are stored tile-packed (mas_internal.h): the same N (N + 1) / 2 values as packed upper
// storage, laid out so a warp reads every 32 x 32 tile conflict-free and uses each value for both
// y_I += T x_J and y_J += T^T x_I; the transposed sums are combined across lanes with a
// 31-shuffle reduce-transpose per column tile. Storage is FP64, FP32 or binary16 with one
// power-of-two scale per matrix (FP32 arithmetic for both reduced formats).

#include "mas_common.cuh"

namespace pmas
{
    namespace
    {
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
        template <int T, class Store, class Real = typename StoreTraits<Store>::Real>
        __device__ __forceinline__ void symv_column(const Store *__restrict__ M, const Real *__restrict__ xs, int lane,
                                                    int J, Real (&yr)[T])
        {
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
                const Store *tile = M + off + I * 1024;
                const Real xI = xs[32 * I + lane];
                Real a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
                for (int j4 = 0; j4 < 8; ++j4)
                {
                    const auto v = load4(tile + j4 * 128 + lane * 4);
                    const auto xv = load4(xs + 32 * J + 4 * j4);
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
            const Store *dt = M + off + J * 1024;
            const Real xJ = xs[32 * J + lane];
            Real a0 = 0, a1 = 0;
#pragma unroll
            for (int j = 0; j < 32; ++j)
            {
                const Real v = (lane <= j) ? (Real)load1(dt + j * (j + 1) / 2 + lane) : Real(0);
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
        template <int T, class Store, class Real = typename StoreTraits<Store>::Real>
        __device__ __forceinline__ void symv_tiles(const Store *__restrict__ M, const Real *__restrict__ xs, int lane,
                                                   Real (&yr)[T])
        {
#pragma unroll
            for (int t = 0; t < T; ++t)
                yr[t] = Real(0);
#pragma unroll
            for (int J = 0; J < T; ++J)
                symv_column<T, Store>(M, xs, lane, J, yr);
        }

        // ---- Binary16 (mma16 layout): warp tensor-core products, m16n8k16, FP32 accumulation. ----
        __device__ __forceinline__ void ldsm_x4(uint32_t (&a)[4], uint32_t addr)
        {
            asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                         : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                         : "r"(addr));
        }
        __device__ __forceinline__ void ldsm_x4_trans(uint32_t (&a)[4], uint32_t addr)
        {
            asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                         : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                         : "r"(addr));
        }
        __device__ __forceinline__ uint32_t ldsm_x1(uint32_t addr)
        {
            uint32_t a;
            asm volatile("ldmatrix.sync.aligned.m8n8.x1.shared.b16 {%0}, [%1];" : "=r"(a) : "r"(addr));
            return a;
        }
        __device__ __forceinline__ void mma_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
        {
            asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                         "{%8, %9}, {%0, %1, %2, %3};"
                         : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                         : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
        }

        // y = M x for one mma16 matrix in shared memory, by one warp. x enters as two binary16
        // columns (xh + xl = x scaled, ~22 significant bits), the B operand's columns 0 and 1; the
        // FP32 products of column 0 and 1 are added back. Each 16 x 16 block above the diagonal
        // is used twice: as stored for its block row and, loaded transposed, for its block
        // column. The result goes through ys (shared, N floats): lane l gets rows 32 t + l.
        template <int BD>
        __device__ __forceinline__ void symv_mma16(const __half *M, const __half *xh, const __half *xl, float *ys,
                                                   int lane, float (&yr)[BD])
        {
            constexpr int NS = 2 * BD, NB = NS * (NS - 1) / 2;
            const int g = lane >> 2, q = lane & 3;
            const int c = lane >> 3, rr = lane & 7; // ldmatrix: lanes 8c..8c+7 give the rows of core c
            uint32_t bf[NS][2];
            const __half *xsrc = (g == 0) ? xh : xl;
#pragma unroll
            for (int S = 0; S < NS; ++S)
            {
                bf[S][0] = g < 2 ? *reinterpret_cast<const uint32_t *>(xsrc + 16 * S + 2 * q) : 0u;
                bf[S][1] = g < 2 ? *reinterpret_cast<const uint32_t *>(xsrc + 16 * S + 2 * q + 8) : 0u;
            }
            float d[NS][4];
#pragma unroll
            for (int R = 0; R < NS; ++R)
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    d[R][i] = 0.f;
            const uint32_t mbase = smem_addr(M);
            const int ct = (c == 1) ? 2 : (c == 2 ? 1 : c); // fragment c of a transposed block
            const uint32_t row_off = (uint32_t)(rr * 16);
#pragma unroll
            for (int R = 0; R < NS; ++R)
#pragma unroll
                for (int S = R + 1; S < NS; ++S)
                {
                    const uint32_t blk = mbase + (uint32_t)((R * (2 * NS - R - 1) / 2 + (S - R - 1)) * 512);
                    uint32_t a[4];
                    ldsm_x4(a, blk + c * 128 + row_off);
                    mma_16816(d[R], a, bf[S][0], bf[S][1]);
                    ldsm_x4_trans(a, blk + ct * 128 + row_off);
                    mma_16816(d[S], a, bf[R][0], bf[R][1]);
                }
            // Diagonal blocks [[D0, C], [C^T, D1]]: transposed loads of (D0, C, -, D1) give
            // fragments 0, 1, 3 (D0, D1 are symmetric); fragment 2 (C) is a plain load.
            const int cd = (c == 1) ? 1 : (c == 3 ? 2 : 0);
#pragma unroll
            for (int R = 0; R < NS; ++R)
            {
                const uint32_t blk = mbase + (uint32_t)((NB * 256 + R * 192) * 2);
                uint32_t a[4];
                ldsm_x4_trans(a, blk + cd * 128 + row_off);
                a[2] = ldsm_x1(blk + 128 + row_off);
                mma_16816(d[R], a, bf[R][0], bf[R][1]);
            }
            if (q == 0)
#pragma unroll
                for (int R = 0; R < NS; ++R)
                {
                    ys[16 * R + g] = d[R][0] + d[R][1];
                    ys[16 * R + g + 8] = d[R][2] + d[R][3];
                }
            __syncwarp();
#pragma unroll
            for (int t = 0; t < BD; ++t)
                yr[t] = ys[t * 32 + lane];
        }

        // The reference's per-iteration scalar work and convergence test (MASSolver.cu:505,
        // 526-583), run by the last CTA of the apply. rz = r . z, rzcross = r . z_old (Polak-Ribiere).
        __device__ void pcg_finalize(PcgState *st, const PcgConfig &cfg, int mode, double rz, double rzcross)
        {
            if (st->error == ERR_TIMEOUT)
            {
                // A bounded wait gave up in this apply: z is incomplete, stop the solve here.
                st->done = 1;
                return;
            }
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
            const int iter = st->iter + 1;
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

        template <int BD, class Store>
        struct ApplyLayout
        {
            using Real = typename StoreTraits<Store>::Real;
            static constexpr int N = 32 * BD;
            static constexpr bool MMA = StoreTraits<Store>::SCALED; // binary16: mma16 layout
            static constexpr int S = MMA ? (2 * BD) * (2 * BD - 1) / 2 * 256 + 2 * BD * 192 : N * (N + 1) / 2;
            static constexpr int STAGE_BYTES = S * (int)sizeof(Store);
            // x: Real values, or binary16 hi / lo columns plus the FP32 result rows.
            static constexpr int XS_BYTES = MMA ? 8 * N : ((N * (int)sizeof(Real)) + 15) / 16 * 16;
            static constexpr int WARP_BYTES = 2 * STAGE_BYTES + XS_BYTES + 16;
            static constexpr int SMEM_LIMIT = 232448 - 1024; // leave room for static shared memory
            static constexpr int W0 = SMEM_LIMIT / WARP_BYTES;
            static constexpr int WARPS = W0 > 16 ? 16 : W0;
            static_assert(STAGE_BYTES % 16 == 0, "bulk copies need 16-byte multiples");
        };

        // Partial dots of the apply, per CTA: r.z0 and r.z0_old over banks with coupled rows, the
        // same over banks of isolated rows, rc.zc and rc.zc_old over the coarse matrices.
        constexpr int APPLY_PARTS = 6;

        // Work item m: m < banks -> level-0 matrix m (input r, output z0); otherwise coarse matrix
        // g = coarse_active[m - banks] (matrix banks + g, input rc, output zc, 32 coarse nodes
        // from g * 32). mode 0: plain apply; 1: initial PCG apply (rz0); 2: PCG iteration.
        // prefetch_first: issue the first two inverse copies before waiting for the predecessor
        // (a chained launch of one system); otherwise a finished solve returns before any copy
        // (the batched launch, where most CTAs may belong to finished systems).
        template <int BD, class Store, int MODE>
        __device__ __forceinline__ void mas_apply_body(const MasView &mas, const double *__restrict__ r,
                                                       double *__restrict__ z0, PcgState *st, const ReduceBuf &red,
                                                       const PcgConfig &cfg, Cta cta, bool prefetch_first)
        {
            if (!prefetch_first && MODE != 0 && st->done)
                return;
            using L = ApplyLayout<BD, Store>;
            using Real = typename L::Real;
            constexpr int N = L::N, S = L::S, WARPS = L::WARPS;
            constexpr int THREADS = WARPS * 32;
            extern __shared__ __align__(128) unsigned char smem[];
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            unsigned char *base = smem + (size_t)w * L::WARP_BYTES;
            Store *stage0 = reinterpret_cast<Store *>(base);
            Store *stage1 = reinterpret_cast<Store *>(base + L::STAGE_BYTES);
            Real *xs = reinterpret_cast<Real *>(base + 2 * L::STAGE_BYTES);
            __half *xh = reinterpret_cast<__half *>(base + 2 * L::STAGE_BYTES);
            __half *xl = xh + N;
            float *ys = reinterpret_cast<float *>(base + 2 * L::STAGE_BYTES + 4 * N);
            uint64_t *bar = reinterpret_cast<uint64_t *>(base + 2 * L::STAGE_BYTES + L::XS_BYTES);
            const Store *__restrict__ inv = static_cast<const Store *>(mas.inv);
            const int banks = mas.banks;
            const int items = banks + mas.n_coarse_active;
            const int total_warps = cta.n * WARPS;
            const int gw = cta.x * WARPS + w;
            int *errp = st ? &st->error : nullptr;
            const bool pr = (MODE == 2) && cfg.polak_ribiere;
            // Matrix index and input vector of an item (coarse vectors: g * N).
            auto mat_of = [&](int m) { return m < banks ? m : banks + mas.coarse_active[m - banks]; };
            auto in_of = [&](int m) -> const double * {
                return m < banks ? r + (size_t)m * N : mas.rc + (size_t)(mat_of(m) - banks) * N;
            };

            const uint64_t pol = l2_evict_first_policy(); // the inverses stream, the vectors stay
            if (lane == 0)
            {
                mbar_init(&bar[0], 1);
                mbar_init(&bar[1], 1);
                fence_mbar_init();
            }
            __syncwarp();
            if (lane == 0)
            {
                if (gw < items)
                    bulk_load_stream(stage0, inv + (size_t)mat_of(gw) * S, L::STAGE_BYTES, &bar[0], pol);
                if (gw + total_warps < items)
                    bulk_load_stream(stage1, inv + (size_t)mat_of(gw + total_warps) * S, L::STAGE_BYTES, &bar[1], pol);
            }
            // Copies issued and not yet consumed, per stage (drained if a wait gives up).
            bool pending[2] = {gw < items, gw + total_warps < items};
            // The first two inverses are on their way (no kernel of a solve writes them); now wait
            // for the predecessor (launched chained in a PCG iteration).
            pdl_wait();
            if (MODE != 0 && st->done)
            {
                if (lane == 0)
                    mbar_drain(bar, pending, {0u, 0u});
                __syncwarp();
                return;
            }
            double part[APPLY_PARTS];
#pragma unroll
            for (int i = 0; i < APPLY_PARTS; ++i)
                part[i] = 0.0;
            uint32_t phase0 = 0, phase1 = 0;
            bool ok = true;
            // Input (and binary16 scale) of the current item, prefetched one item ahead.
            double r_next[BD], scale_next = 1.0;
            if (gw < items)
            {
                const double *in = in_of(gw);
#pragma unroll
                for (int t = 0; t < BD; ++t)
                    r_next[t] = in[t * 32 + lane];
                if (StoreTraits<Store>::SCALED)
                    scale_next = mas.inv_scale[mat_of(gw)];
            }
            int k = 0;
            for (int m = gw; m < items; m += total_warps, ++k)
            {
                const bool s1 = (k & 1) != 0;
                Store *stage = s1 ? stage1 : stage0;
                uint64_t *b = s1 ? &bar[1] : &bar[0];
                const bool coarse = m >= banks;
                const int mat = mat_of(m);
                double *out = coarse ? mas.zc + (size_t)(mat - banks) * N : z0 + (size_t)m * N;
                double r64[BD];
#pragma unroll
                for (int t = 0; t < BD; ++t)
                    r64[t] = r_next[t];
                const double mscale = scale_next;
                double xscale = 1.0; // binary16 input: x * xscale split into hi + lo
                if constexpr (L::MMA)
                {
                    double amax = 0.0;
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                        amax = fmax(amax, fabs(r64[t]));
#pragma unroll
                    for (int o = 16; o >= 1; o >>= 1)
                        amax = fmax(amax, __shfl_xor_sync(FULL, amax, o));
                    xscale = (amax > 0.0 && isfinite(amax)) ? ldexp(1.0, 14 - ilogb(amax)) : 1.0;
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                    {
                        const float v = (float)(r64[t] * xscale);
                        const __half h = __float2half_rn(v);
                        xh[t * 32 + lane] = h;
                        xl[t * 32 + lane] = __float2half_rn(v - __half2float(h));
                    }
                }
                else
                {
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                        xs[t * 32 + lane] = (Real)r64[t];
                }
                const int mnext = m + total_warps;
                if (mnext < items)
                {
                    const double *in = in_of(mnext);
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                        r_next[t] = in[t * 32 + lane];
                    if (StoreTraits<Store>::SCALED)
                        scale_next = mas.inv_scale[mat_of(mnext)];
                }
                double zold[BD];
                if (pr)
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                        zold[t] = out[t * 32 + lane];
                __syncwarp();
                if (!mbar_wait_bounded(b, s1 ? phase1 : phase0, errp, cfg.wait_limit))
                {
                    ok = false;
                    break;
                }
                pending[s1 ? 1 : 0] = false;
                if (s1)
                    phase1 ^= 1u;
                else
                    phase0 ^= 1u;
                // Coarse matrices of isolated rows are exactly the identity: z = r, unrounded.
                const bool ident = coarse && mas.identity[mat - banks];
                Real yr[BD];
                if (!ident)
                {
                    if constexpr (L::MMA)
                        symv_mma16<BD>(reinterpret_cast<const __half *>(stage), xh, xl, ys, lane, yr);
                    else
                        symv_tiles<BD, Store>(stage, xs, lane, yr);
                }
                __syncwarp();
                const int mn = m + 2 * total_warps;
                if (mn < items)
                {
                    if (lane == 0)
                    {
                        fence_proxy_async_smem();
                        bulk_load_stream(stage, inv + (size_t)mat_of(mn) * S, L::STAGE_BYTES, b, pol);
                    }
                    pending[s1 ? 1 : 0] = true;
                }
                const double scale = StoreTraits<Store>::SCALED ? mscale / xscale : 1.0;
                double d0 = 0.0, d1 = 0.0;
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    double zv;
                    if (ident)
                        zv = r64[t];
                    else
                        zv = StoreTraits<Store>::SCALED ? (double)yr[t] * scale : (double)yr[t];
                    out[t * 32 + lane] = zv;
                    d0 = fma(zv, r64[t], d0);
                    if (pr)
                        d1 = fma(zold[t], r64[t], d1);
                }
                // Fixed slots (no dynamic indexing, so part[] stays in registers).
                if (coarse)
                {
                    part[4] += d0;
                    part[5] += d1;
                }
                else if (m >= mas.first_iso_bank)
                {
                    part[2] += d0;
                    part[3] += d1;
                }
                else
                {
                    part[0] += d0;
                    part[1] += d1;
                }
            }
            if (!ok)
            {
                // Drain this warp's outstanding copies (bounded) before leaving.
                if (lane == 0)
                    mbar_drain(bar, pending, {phase0, phase1});
                __syncwarp();
            }
            pdl_release(); // this warp's items are done: the successor may start launching
            if (MODE == 0)
                return;
            double tot[APPLY_PARTS];
            if (grid_reduce<APPLY_PARTS, THREADS>(part, red.rz_parts, &st->counter[4], tot, cta) && threadIdx.x == 0)
            {
                // Isolated rows: z = (1 + L) z0, so their r.z is (1 + L) r.z0 -- r.z0 is in the
                // level-0 sums, the coarse levels add L r.z0.
                const double Lc = (double)cfg.level_num;
                st->rz_coarse = tot[4] + Lc * tot[2];
                st->rzx_coarse = tot[5] + Lc * tot[3];
                pcg_finalize(st, cfg, MODE, tot[0] + tot[2] + st->rz_coarse, tot[1] + tot[3] + st->rzx_coarse);
            }
        }

        template <int BD, class Store, int MODE>
        __global__ void __launch_bounds__(ApplyLayout<BD, Store>::WARPS * 32)
            k_mas_apply(MasView mas, const double *__restrict__ r, double *__restrict__ z0, PcgState *st,
                        ReduceBuf red, PcgConfig cfg)
        {
            mas_apply_body<BD, Store, MODE>(mas, r, z0, st, red, cfg, native_cta(), true);
        }

        // The apply of every system of a batch (MODE 1: initial, 2: iteration) in one launch.
        template <int BD, class Store, int MODE>
        __global__ void __launch_bounds__(ApplyLayout<BD, Store>::WARPS * 32) k_mas_apply_batch(BatchView v)
        {
            const int4 e = batch_entry(v, BPH_APPLY);
            const BatchSystem &sy = v.sys[e.x];
            const Cta cta{e.y, e.z};
            const MasView mas = sy.mas;
            const ReduceBuf red = sy.red;
            const PcgConfig cfg = sy.cfg;
            mas_apply_body<BD, Store, MODE>(mas, sy.r, sy.z, sy.st, red, cfg, cta,
                                            false);
        }

        // ---- G right-hand sides at once (binary16 inverses only): the B operand's eight columns
        // hold the hi / lo splits of the G = RHS_GROUP vectors, so one pass over an inverse and the
        // same 36 MMAs serve all of them; every lane of a fragment quad holds a different
        // right-hand side of the result. Vectors are interleaved (value e of right-hand side g at
        // e * G + g). Per-right-hand-side dots and PCG steps; st[G] is the group record.
        template <int BD>
        struct ApplyLayoutG
        {
            static constexpr int N = 32 * BD;
            static constexpr int G = RHS_GROUP;
            static constexpr int S = (2 * BD) * (2 * BD - 1) / 2 * 256 + 2 * BD * 192;
            static constexpr int STAGE_BYTES = S * 2;
            static constexpr int XS_BYTES = 8 * G * N; // hi, lo (binary16) and the FP32 result rows
            static constexpr int WARP_BYTES = 2 * STAGE_BYTES + XS_BYTES + 16;
            static constexpr int SMEM_LIMIT = 232448 - 1024;
            static constexpr int W0 = SMEM_LIMIT / WARP_BYTES;
            static constexpr int WARPS = W0 > 16 ? 16 : W0;
            static_assert(STAGE_BYTES % 16 == 0, "bulk copies need 16-byte multiples");
            static_assert(2 * G == 8, "the B operand has eight columns: G hi / lo pairs");
        };

        // XS, YS: strides (values) between consecutive right-hand sides in xh / xl and in ys.
        template <int BD, int XS = 32 * BD, int YS = 32 * BD>
        __device__ __forceinline__ void symv_mma16_g(const __half *M, const __half *xh, const __half *xl, float *ys,
                                                     int lane)
        {
            constexpr int NS = 2 * BD, NB = NS * (NS - 1) / 2;
            const int g = lane >> 2, q = lane & 3;
            const int c = lane >> 3, rr = lane & 7;
            // B column n = g: right-hand side g / 2, hi (even) or lo (odd).
            const __half *xsrc = ((g & 1) ? xl : xh) + (g >> 1) * XS;
            uint32_t bf[NS][2];
#pragma unroll
            for (int S = 0; S < NS; ++S)
            {
                bf[S][0] = *reinterpret_cast<const uint32_t *>(xsrc + 16 * S + 2 * q);
                bf[S][1] = *reinterpret_cast<const uint32_t *>(xsrc + 16 * S + 2 * q + 8);
            }
            float d[NS][4];
#pragma unroll
            for (int R = 0; R < NS; ++R)
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    d[R][i] = 0.f;
            const uint32_t mbase = smem_addr(M);
            const int ct = (c == 1) ? 2 : (c == 2 ? 1 : c);
            const uint32_t row_off = (uint32_t)(rr * 16);
#pragma unroll
            for (int R = 0; R < NS; ++R)
#pragma unroll
                for (int S = R + 1; S < NS; ++S)
                {
                    const uint32_t blk = mbase + (uint32_t)((R * (2 * NS - R - 1) / 2 + (S - R - 1)) * 512);
                    uint32_t a[4];
                    ldsm_x4(a, blk + c * 128 + row_off);
                    mma_16816(d[R], a, bf[S][0], bf[S][1]);
                    ldsm_x4_trans(a, blk + ct * 128 + row_off);
                    mma_16816(d[S], a, bf[R][0], bf[R][1]);
                }
            const int cd = (c == 1) ? 1 : (c == 3 ? 2 : 0);
#pragma unroll
            for (int R = 0; R < NS; ++R)
            {
                const uint32_t blk = mbase + (uint32_t)((NB * 256 + R * 192) * 2);
                uint32_t a[4];
                ldsm_x4_trans(a, blk + cd * 128 + row_off);
                a[2] = ldsm_x1(blk + 128 + row_off);
                mma_16816(d[R], a, bf[R][0], bf[R][1]);
            }
            // Columns 2q, 2q + 1 of rows g, g + 8 of each block row: right-hand side q.
#pragma unroll
            for (int R = 0; R < NS; ++R)
            {
                ys[q * YS + 16 * R + g] = d[R][0] + d[R][1];
                ys[q * YS + 16 * R + g + 8] = d[R][2] + d[R][3];
            }
            __syncwarp();
        }

        template <int BD, int MODE>
        __global__ void __launch_bounds__(ApplyLayoutG<BD>::WARPS * 32)
            k_mas_apply_g(MasView mas, const double *__restrict__ r, double *__restrict__ z0, PcgState *st,
                          ReduceBuf red, PcgConfig cfg)
        {
            using L = ApplyLayoutG<BD>;
            constexpr int N = L::N, S = L::S, WARPS = L::WARPS, G = L::G;
            constexpr int THREADS = WARPS * 32;
            PcgState *grp = st + G;
            if (grp->done)
                return;
            extern __shared__ __align__(128) unsigned char smem[];
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            unsigned char *base = smem + (size_t)w * L::WARP_BYTES;
            __half *stage0 = reinterpret_cast<__half *>(base);
            __half *stage1 = reinterpret_cast<__half *>(base + L::STAGE_BYTES);
            __half *xh = reinterpret_cast<__half *>(base + 2 * L::STAGE_BYTES);
            __half *xl = xh + G * N;
            float *ys = reinterpret_cast<float *>(base + 2 * L::STAGE_BYTES + 4 * G * N);
            uint64_t *bar = reinterpret_cast<uint64_t *>(base + 2 * L::STAGE_BYTES + L::XS_BYTES);
            const __half *__restrict__ inv = static_cast<const __half *>(mas.inv);
            const int banks = mas.banks;
            const int items = banks + mas.n_coarse_active;
            const int total_warps = gridDim.x * WARPS;
            const int gw = blockIdx.x * WARPS + w;
            auto mat_of = [&](int m) { return m < banks ? m : banks + mas.coarse_active[m - banks]; };
            auto in_of = [&](int m) -> const double * {
                return m < banks ? r + (size_t)m * N * G : mas.rc + (size_t)(mat_of(m) - banks) * N * G;
            };
            const uint64_t pol = l2_evict_first_policy();
            if (lane == 0)
            {
                mbar_init(&bar[0], 1);
                mbar_init(&bar[1], 1);
                fence_mbar_init();
            }
            __syncwarp();
            if (lane == 0)
            {
                if (gw < items)
                    bulk_load_stream(stage0, inv + (size_t)mat_of(gw) * S, L::STAGE_BYTES, &bar[0], pol);
                if (gw + total_warps < items)
                    bulk_load_stream(stage1, inv + (size_t)mat_of(gw + total_warps) * S, L::STAGE_BYTES, &bar[1],
                                     pol);
            }
            bool pending[2] = {gw < items, gw + total_warps < items};
            double part[3 * G]; // per right-hand side: coupled banks, isolated banks, coarse
#pragma unroll
            for (int i = 0; i < 3 * G; ++i)
                part[i] = 0.0;
            uint32_t phase0 = 0, phase1 = 0;
            bool ok = true;
            int k = 0;
            for (int m = gw; m < items; m += total_warps, ++k)
            {
                const bool s1 = (k & 1) != 0;
                __half *stage = s1 ? stage1 : stage0;
                uint64_t *b = s1 ? &bar[1] : &bar[0];
                const bool coarse = m >= banks;
                const int mat = mat_of(m);
                const double *in = in_of(m);
                double *out = coarse ? mas.zc + (size_t)(mat - banks) * N * G : z0 + (size_t)m * N * G;
                double r64[BD][G];
#pragma unroll
                for (int t = 0; t < BD; ++t)
#pragma unroll
                    for (int h = 0; h < G / 2; ++h)
                    {
                        const double2 v = *reinterpret_cast<const double2 *>(in + (t * 32 + lane) * G + 2 * h);
                        r64[t][2 * h] = v.x;
                        r64[t][2 * h + 1] = v.y;
                    }
                double xscale[G];
#pragma unroll
                for (int gg = 0; gg < G; ++gg)
                {
                    double amax = 0.0;
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                        amax = fmax(amax, fabs(r64[t][gg]));
#pragma unroll
                    for (int o = 16; o >= 1; o >>= 1)
                        amax = fmax(amax, __shfl_xor_sync(FULL, amax, o));
                    xscale[gg] = (amax > 0.0 && isfinite(amax)) ? ldexp(1.0, 14 - ilogb(amax)) : 1.0;
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                    {
                        const float v = (float)(r64[t][gg] * xscale[gg]);
                        const __half h = __float2half_rn(v);
                        xh[gg * N + t * 32 + lane] = h;
                        xl[gg * N + t * 32 + lane] = __float2half_rn(v - __half2float(h));
                    }
                }
                __syncwarp();
                if (!mbar_wait_bounded(b, s1 ? phase1 : phase0, &grp->error, cfg.wait_limit))
                {
                    ok = false;
                    break;
                }
                pending[s1 ? 1 : 0] = false;
                if (s1)
                    phase1 ^= 1u;
                else
                    phase0 ^= 1u;
                const bool ident = coarse && mas.identity[mat - banks];
                if (!ident)
                    symv_mma16_g<BD>(stage, xh, xl, ys, lane);
                __syncwarp();
                const int mn = m + 2 * total_warps;
                if (mn < items)
                {
                    if (lane == 0)
                    {
                        fence_proxy_async_smem();
                        bulk_load_stream(stage, inv + (size_t)mat_of(mn) * S, L::STAGE_BYTES, b, pol);
                    }
                    pending[s1 ? 1 : 0] = true;
                }
                const double mscale = mas.inv_scale[mat];
                const int slot = coarse ? 2 : ((m >= mas.first_iso_bank) ? 1 : 0);
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    double zv[G];
#pragma unroll
                    for (int gg = 0; gg < G; ++gg)
                    {
                        zv[gg] = ident ? r64[t][gg] : (double)ys[gg * N + t * 32 + lane] * (mscale / xscale[gg]);
                        const double d = zv[gg] * r64[t][gg];
                        if (slot == 0)
                            part[gg] += d;
                        else if (slot == 1)
                            part[G + gg] += d;
                        else
                            part[2 * G + gg] += d;
                    }
#pragma unroll
                    for (int h = 0; h < G / 2; ++h)
                        *reinterpret_cast<double2 *>(out + (t * 32 + lane) * G + 2 * h) =
                            make_double2(zv[2 * h], zv[2 * h + 1]);
                }
                __syncwarp();
            }
            if (!ok)
            {
                if (lane == 0)
                    mbar_drain(bar, pending, {phase0, phase1});
                __syncwarp();
            }
            double tot[3 * G];
            if (grid_reduce<3 * G, THREADS>(part, red.rz_parts, &grp->counter[4], tot) && threadIdx.x == 0)
            {
                const double Lc = (double)cfg.level_num;
                int all_done = 1;
#pragma unroll
                for (int gg = 0; gg < G; ++gg)
                {
                    PcgState *sg = st + gg;
                    if (!sg->done)
                    {
                        sg->rz_coarse = tot[2 * G + gg] + Lc * tot[G + gg];
                        pcg_finalize(sg, cfg, MODE, tot[gg] + tot[G + gg] + sg->rz_coarse, 0.0);
                        if (sg->error)
                            grp->error = sg->error;
                    }
                    all_done &= sg->done ? 1 : 0;
                }
                grp->iter = MODE == 1 ? 0 : grp->iter + 1;
                if (all_done || grp->error)
                    grp->done = 1;
            }
        }

        // ---- RHS_WIDE (16) right-hand sides at once (block size 3, binary16 inverses): the B operand
        // of each m16n8k16 holds four right-hand sides' hi / lo splits, so each inverse is multiplied in
        // four n-tiles (symv_mma16_g per tile) and read from memory once for all sixteen. Lane l loads,
        // splits and stores right-hand side g = l % 16 (values e = 2 t + l / 16 of the matrix's 96), so
        // every load and store of the interleaved vectors is 128 B per 16 lanes. xh / xl and ys use
        // padded strides per right-hand side (100 halves, 97 floats) that spread the 16 lanes' words
        // over the shared-memory banks.
        struct ApplyLayoutW
        {
            static constexpr int BD = 3, N = 96, G = RHS_WIDE;
            static constexpr int XS = N + 4, YS = N + 1;
            static constexpr int S = (2 * BD) * (2 * BD - 1) / 2 * 256 + 2 * BD * 192;
            static constexpr int STAGE_BYTES = S * 2;
            static constexpr int XS_BYTES = 2 * 2 * G * XS + 4 * G * YS; // hi, lo, FP32 result
            static constexpr int WARP_BYTES = 2 * STAGE_BYTES + XS_BYTES + 16;
            static constexpr int SMEM_LIMIT = 232448 - 2048; // static shared memory: the grid sum's groups
            static constexpr int W0 = SMEM_LIMIT / WARP_BYTES;
            static constexpr int WARPS = W0 > 16 ? 16 : W0;
            static_assert(STAGE_BYTES % 16 == 0 && WARP_BYTES % 16 == 0 && XS_BYTES % 8 == 0, "alignment");
            static_assert((WARPS + 2) * 3 * G * 8 <= WARP_BYTES, "the final sums reuse the first warp's area");
        };

        template <int MODE>
        __global__ void __launch_bounds__(ApplyLayoutW::WARPS * 32)
            k_mas_apply_w(MasView mas, const double *__restrict__ r, double *__restrict__ z0, PcgState *st,
                          ReduceBuf red, PcgConfig cfg)
        {
            using L = ApplyLayoutW;
            constexpr int N = L::N, S = L::S, WARPS = L::WARPS, G = L::G, XS = L::XS, YS = L::YS;
            constexpr int THREADS = WARPS * 32;
            constexpr int VW = N / 2; // values of a matrix per lane (two lanes per right-hand side)
            PcgState *grp = st + G;
            if (grp->done)
                return;
            extern __shared__ __align__(128) unsigned char smem[];
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            unsigned char *base = smem + (size_t)w * L::WARP_BYTES;
            __half *stage0 = reinterpret_cast<__half *>(base);
            __half *stage1 = reinterpret_cast<__half *>(base + L::STAGE_BYTES);
            __half *xh = reinterpret_cast<__half *>(base + 2 * L::STAGE_BYTES);
            __half *xl = xh + G * XS;
            float *ys = reinterpret_cast<float *>(base + 2 * L::STAGE_BYTES + 4 * G * XS);
            uint64_t *bar = reinterpret_cast<uint64_t *>(base + 2 * L::STAGE_BYTES + L::XS_BYTES);
            const __half *__restrict__ inv = static_cast<const __half *>(mas.inv);
            const int banks = mas.banks;
            const int items = banks + mas.n_coarse_active;
            const int total_warps = gridDim.x * WARPS;
            const int gw = blockIdx.x * WARPS + w;
            auto mat_of = [&](int m) { return m < banks ? m : banks + mas.coarse_active[m - banks]; };
            auto in_of = [&](int m) -> const double * {
                return m < banks ? r + (size_t)m * N * G : mas.rc + (size_t)(mat_of(m) - banks) * N * G;
            };
            const uint64_t pol = l2_evict_first_policy();
            if (lane == 0)
            {
                mbar_init(&bar[0], 1);
                mbar_init(&bar[1], 1);
                fence_mbar_init();
            }
            __syncwarp();
            if (lane == 0)
            {
                if (gw < items)
                    bulk_load_stream(stage0, inv + (size_t)mat_of(gw) * S, L::STAGE_BYTES, &bar[0], pol);
                if (gw + total_warps < items)
                    bulk_load_stream(stage1, inv + (size_t)mat_of(gw + total_warps) * S, L::STAGE_BYTES, &bar[1],
                                     pol);
            }
            bool pending[2] = {gw < items, gw + total_warps < items};
            const int g = lane & (G - 1), half = lane >> 4;
            double part[3] = {0.0, 0.0, 0.0}; // this lane's right-hand side: coupled, isolated, coarse
            uint32_t phase0 = 0, phase1 = 0;
            bool ok = true;
            int k = 0;
            for (int m = gw; m < items; m += total_warps, ++k)
            {
                const bool s1 = (k & 1) != 0;
                __half *stage = s1 ? stage1 : stage0;
                uint64_t *b = s1 ? &bar[1] : &bar[0];
                const bool coarse = m >= banks;
                const int mat = mat_of(m);
                const double *in = in_of(m);
                double *out = coarse ? mas.zc + (size_t)(mat - banks) * N * G : z0 + (size_t)m * N * G;
                double r64[VW];
#pragma unroll
                for (int t = 0; t < VW; ++t)
                    r64[t] = in[(2 * t + half) * G + g];
                double amax = 0.0;
#pragma unroll
                for (int t = 0; t < VW; ++t)
                    amax = fmax(amax, fabs(r64[t]));
                amax = fmax(amax, __shfl_xor_sync(FULL, amax, 16));
                const double xscale = (amax > 0.0 && isfinite(amax)) ? ldexp(1.0, 14 - ilogb(amax)) : 1.0;
#pragma unroll
                for (int t = 0; t < VW; ++t)
                {
                    const float v = (float)(r64[t] * xscale);
                    const __half h = __float2half_rn(v);
                    xh[g * XS + 2 * t + half] = h;
                    xl[g * XS + 2 * t + half] = __float2half_rn(v - __half2float(h));
                }
                __syncwarp();
                if (!mbar_wait_bounded(b, s1 ? phase1 : phase0, &grp->error, cfg.wait_limit))
                {
                    ok = false;
                    break;
                }
                pending[s1 ? 1 : 0] = false;
                if (s1)
                    phase1 ^= 1u;
                else
                    phase0 ^= 1u;
                const bool ident = coarse && mas.identity[mat - banks];
                if (!ident)
#pragma unroll
                    for (int nt = 0; nt < G / 4; ++nt)
                        symv_mma16_g<3, XS, YS>(stage, xh + 4 * nt * XS, xl + 4 * nt * XS, ys + 4 * nt * YS, lane);
                __syncwarp();
                const int mn = m + 2 * total_warps;
                if (mn < items)
                {
                    if (lane == 0)
                    {
                        fence_proxy_async_smem();
                        bulk_load_stream(stage, inv + (size_t)mat_of(mn) * S, L::STAGE_BYTES, b, pol);
                    }
                    pending[s1 ? 1 : 0] = true;
                }
                const double sc = mas.inv_scale[mat] / xscale;
                double d = 0.0;
#pragma unroll
                for (int t = 0; t < VW; ++t)
                {
                    const int e = 2 * t + half;
                    const double zv = ident ? r64[t] : (double)ys[g * YS + e] * sc;
                    out[e * G + g] = zv;
                    d = fma(zv, r64[t], d);
                }
                if (coarse)
                    part[2] += d;
                else if (m >= mas.first_iso_bank)
                    part[1] += d;
                else
                    part[0] += d;
                __syncwarp();
            }
            if (!ok)
            {
                if (lane == 0)
                    mbar_drain(bar, pending, {phase0, phase1});
                __syncwarp();
            }
            // Every warp is past its last stage (no copy in flight): the first warp's area holds the
            // per-warp sums, the CTA's sums and the totals.
            __syncthreads();
            double *wsum = reinterpret_cast<double *>(smem);
            double *cta = wsum + WARPS * 3 * G, *tot = cta + 3 * G;
#pragma unroll
            for (int i = 0; i < 3; ++i)
                part[i] += __shfl_xor_sync(FULL, part[i], 16);
            if (lane < G)
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    wsum[w * 3 * G + i * G + lane] = part[i];
            __syncthreads();
            if (threadIdx.x < 3 * G)
            {
                double s = 0.0;
                for (int ww = 0; ww < WARPS; ++ww)
                    s += wsum[ww * 3 * G + threadIdx.x];
                cta[threadIdx.x] = s;
            }
            if (grid_reduce_cta<3 * G, THREADS>(cta, red.rz_parts, &grp->counter[4], tot) && threadIdx.x == 0)
            {
                const double Lc = (double)cfg.level_num;
                int all_done = 1;
                for (int gg = 0; gg < G; ++gg)
                {
                    PcgState *sg = st + gg;
                    if (!sg->done)
                    {
                        sg->rz_coarse = tot[2 * G + gg] + Lc * tot[G + gg];
                        pcg_finalize(sg, cfg, MODE, tot[gg] + tot[G + gg] + sg->rz_coarse, 0.0);
                        if (sg->error)
                            grp->error = sg->error;
                    }
                    all_done &= sg->done ? 1 : 0;
                }
                grp->iter = MODE == 1 ? 0 : grp->iter + 1;
                if (all_done || grp->error)
                    grp->done = 1;
            }
        }

        // ---- Sixteen right-hand sides on the fifth-generation tensor cores (tcgen05) ------------
        // Inverse storage "tc" (built from the mma16 storage, the same binary16 values): the full
        // 96 x 96 matrix in 16 x 16 tiles, tile (i, s) (rows 16 i .., columns 16 s ..) at byte
        // s * TC_SLAB_G + i * 512, each tile the four 8 x 8 core matrices [rows 0-7 | cols 0-7],
        // [rows 0-7 | cols 8-15], [rows 8-15 | cols 0-7], [rows 8-15 | cols 8-15] of 16-byte rows:
        // the canonical no-swizzle K-major operand layout with 128 bytes between the two K halves of
        // a core pair and 256 bytes between 8-row groups. Column slab s is the A operand of one K = 16
        // step; in shared memory the slabs are TC_SLAB_S apart with rows 96-127 zero (M = 128).
        // The B operand is the item's 16 right-hand sides split into binary16 hi and lo parts
        // (N = 32: columns g and 16 + g), D = A B^T accumulates in FP32 in tensor memory.
        constexpr int TC_N = 96, TC_G = RHS_WIDE, TC_THREADS = 128;
        constexpr int TC_SLAB_G = 6 * 512;          // bytes of a column slab in global memory
        constexpr int TC_SLAB_S = 8 * 512;          // in shared memory (M = 128 rows)
        constexpr int TC_MAT_BYTES = 6 * TC_SLAB_G; // 18432 bytes per matrix

        __host__ __device__ constexpr int tc_offset(int row, int col)
        {
            return (col >> 4) * TC_SLAB_G + (row >> 4) * 512 + ((row >> 3) & 1) * 256 + ((col >> 3) & 1) * 128 +
                   (row & 7) * 16 + (col & 7) * 2;
        }

        // B operand element (n, k): K steps 1 KB apart, 8-column groups 256 bytes apart.
        __device__ __forceinline__ int tc_b_offset(int n, int k)
        {
            return (k >> 4) * 1024 + (n >> 3) * 256 + ((k >> 3) & 1) * 128 + (n & 7) * 16 + (k & 7) * 2;
        }

        struct TcLayout
        {
            static constexpr int A_BYTES = 6 * TC_SLAB_S;     // one stage of A
            static constexpr int X_BYTES = TC_N * TC_G * 8;   // one stage of the FP64 input block
            static constexpr int B_BYTES = 6 * 1024;
            static constexpr int OFF_X = 2 * A_BYTES;
            static constexpr int OFF_B = OFF_X + 2 * X_BYTES;
            static constexpr int OFF_AMAX = OFF_B + B_BYTES;  // [8][16] doubles
            static constexpr int OFF_XSC = OFF_AMAX + 8 * TC_G * 8;
            static constexpr int OFF_WSUM = OFF_XSC + TC_G * 8; // [4 warps][3][16] doubles
            static constexpr int OFF_BAR = OFF_WSUM + 4 * 3 * TC_G * 8;
            static constexpr int BYTES = OFF_BAR + 64;
            static_assert(OFF_X % 1024 == 0 && OFF_B % 128 == 0 && OFF_BAR % 16 == 0, "alignment");
        };

        // mma16 -> tc storage, one CTA per matrix.
        __global__ void __launch_bounds__(256) k_inv_to_tc(const __half *__restrict__ inv, __half *__restrict__ out)
        {
            constexpr int S16 = 6 * 5 / 2 * 256 + 6 * 192;
            const __half *src = inv + (size_t)blockIdx.x * S16;
            unsigned char *dst = reinterpret_cast<unsigned char *>(out) + (size_t)blockIdx.x * TC_MAT_BYTES;
            for (int e = threadIdx.x; e < TC_N * TC_N; e += blockDim.x)
            {
                const int row = e / TC_N, col = e - row * TC_N;
                *reinterpret_cast<__half *>(dst + tc_offset(row, col)) = src[mma16_index(3, row, col)];
            }
        }

        // The sixteen-right-hand-side MAS apply on tcgen05 (same work items, scales, outputs, dots
        // and PCG steps as k_mas_apply_w). One CTA of four warps per item at a time, items strided
        // over the grid; per item the inverse (six slab copies) and the 96 x 16 FP64 input block
        // arrive by bulk copies on one mbarrier, two items ahead. The four warps split the input into
        // binary16 hi / lo (per-column power-of-two scale), thread 0 issues six MMAs and commits them
        // to an mbarrier, and warps 0-2 read rows 0-95 of the accumulator (tcgen05.ld), combine hi +
        // lo, scale to FP64, store z and add the dots. Every wait is bounded (MAS_ERR_TIMEOUT).
        template <int MODE>
        __global__ void __launch_bounds__(TC_THREADS) k_mas_apply_tc(MasView mas, const __half *__restrict__ inv_tc,
                                                                     const double *__restrict__ r,
                                                                     double *__restrict__ z0, PcgState *st,
                                                                     ReduceBuf red, PcgConfig cfg)
        {
            using L = TcLayout;
            constexpr int N = TC_N, G = TC_G;
            PcgState *grp = st + G;
            if (grp->done)
                return;
            extern __shared__ __align__(1024) unsigned char smem[];
            const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
            unsigned char *sA = smem, *sX = smem + L::OFF_X, *sB = smem + L::OFF_B;
            double *amax_s = reinterpret_cast<double *>(smem + L::OFF_AMAX);
            double *xsc_s = reinterpret_cast<double *>(smem + L::OFF_XSC);
            double *wsum = reinterpret_cast<double *>(smem + L::OFF_WSUM);
            uint64_t *tma_bar = reinterpret_cast<uint64_t *>(smem + L::OFF_BAR); // [2]
            uint64_t *mma_bar = tma_bar + 2;
            uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tma_bar + 3);
            const int banks = mas.banks, items = banks + mas.n_coarse_active;
            auto mat_of = [&](int m) { return m < banks ? m : banks + mas.coarse_active[m - banks]; };
            auto in_of = [&](int m) -> const double * {
                return m < banks ? r + (size_t)m * N * G : mas.rc + (size_t)(mat_of(m) - banks) * N * G;
            };
            const uint64_t pol = l2_evict_first_policy();
            if (tid == 0)
            {
                mbar_init(&tma_bar[0], 1);
                mbar_init(&tma_bar[1], 1);
                mbar_init(mma_bar, 1);
                fence_mbar_init();
            }
            if (w == 0)
                tmem_alloc(tmem_slot, 32);
            // Rows 96-127 of every slab of both A stages: zero (the bulk copies fill rows 0-95).
            for (int i = tid; i < 2 * 6 * 64; i += TC_THREADS)
            {
                const int stg = i / 384, rem = i - stg * 384, slab = rem >> 6, q = rem & 63;
                reinterpret_cast<uint4 *>(sA + stg * L::A_BYTES + slab * TC_SLAB_S + 6 * 512)[q] = make_uint4(0, 0, 0, 0);
            }
            for (int i = tid; i < 4 * 3 * G; i += TC_THREADS)
                wsum[i] = 0.0;
            fence_proxy_async_smem();
            tc_fence_before_sync();
            __syncthreads();
            tc_fence_after_sync();
            const uint32_t taddr = *tmem_slot;
            const int m0 = blockIdx.x, stride = gridDim.x;
            // Thread 0: the inverse and the input block of item m into stage stg.
            auto issue = [&](int m, int stg) {
                const unsigned char *src = reinterpret_cast<const unsigned char *>(inv_tc) + (size_t)mat_of(m) * TC_MAT_BYTES;
                mbar_arrive_expect_tx(&tma_bar[stg], TC_MAT_BYTES + L::X_BYTES);
#pragma unroll 1
                for (int s = 0; s < 6; ++s)
                    bulk_copy_g2s_hint(sA + stg * L::A_BYTES + s * TC_SLAB_S, src + s * TC_SLAB_G, TC_SLAB_G,
                                       &tma_bar[stg], pol);
                bulk_copy_g2s(sX + stg * L::X_BYTES, in_of(m), L::X_BYTES, &tma_bar[stg]);
            };
            bool pending[2] = {m0 < items, m0 + stride < items};
            if (tid == 0)
            {
                if (pending[0])
                    issue(m0, 0);
                if (pending[1])
                    issue(m0 + stride, 1);
            }
            uint32_t tphase[2] = {0u, 0u}, mphase = 0u;
            bool mma_pending = false, ok = true;
            const uint32_t idesc = tc_idesc_f16_f32(128, 32);
            double dsum[G];
#pragma unroll
            for (int gg = 0; gg < G; ++gg)
                dsum[gg] = 0.0;
            int cat = 0; // dots of coupled banks, isolated banks, coarse matrices
            // This warp's running dots into its slots of category c (each category once per CTA:
            // items increase, and the categories with them).
            auto flush = [&](int c) {
#pragma unroll
                for (int gg = 0; gg < G; ++gg)
                {
                    const double v = warp_sum(dsum[gg]);
                    if (lane == 0)
                        wsum[(w * 3 + c) * G + gg] = v;
                    dsum[gg] = 0.0;
                }
            };
            const int g = tid & (G - 1), rg = tid >> 4; // input split: column g, rows 12 rg .. 12 rg + 11
            int k = 0;
            for (int m = m0; m < items; m += stride, ++k)
            {
                const int stg = k & 1;
                const bool wok = mbar_wait_bounded(&tma_bar[stg], tphase[stg], &grp->error, cfg.wait_limit);
                if (!__syncthreads_and(wok))
                {
                    ok = false;
                    break;
                }
                pending[stg] = false;
                tphase[stg] ^= 1u;
                const bool coarse = m >= banks;
                const int mat = mat_of(m);
                const int mcat = coarse ? 2 : (m >= mas.first_iso_bank ? 1 : 0);
                if (mcat != cat)
                {
                    flush(cat);
                    cat = mcat;
                }
                const double *x = reinterpret_cast<const double *>(sX + stg * L::X_BYTES);
                const bool ident = coarse && mas.identity[mat - banks];
                double xv[12], am = 0.0;
#pragma unroll
                for (int i = 0; i < 12; ++i)
                {
                    xv[i] = x[(rg * 12 + i) * G + g];
                    am = fmax(am, fabs(xv[i]));
                }
                amax_s[rg * G + g] = am;
                __syncthreads();
                double amx = 0.0;
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    amx = fmax(amx, amax_s[q * G + g]);
                const double xscale = (amx > 0.0 && isfinite(amx)) ? ldexp(1.0, 14 - ilogb(amx)) : 1.0;
                if (rg == 0)
                    xsc_s[g] = mas.inv_scale[mat] / xscale; // column g's factor back to matrix values
                if (!ident)
                {
                    // Row pairs (kk, kk + 1) are adjacent in the operand layout: one 32-bit store
                    // per pair and part.
#pragma unroll
                    for (int i = 0; i < 12; i += 2)
                    {
                        const int kk = rg * 12 + i;
                        const float v0 = (float)(xv[i] * xscale), v1 = (float)(xv[i + 1] * xscale);
                        const __half h0 = __float2half_rn(v0), h1 = __float2half_rn(v1);
                        *reinterpret_cast<__half2 *>(sB + tc_b_offset(g, kk)) = __halves2half2(h0, h1);
                        *reinterpret_cast<__half2 *>(sB + tc_b_offset(G + g, kk)) =
                            __halves2half2(__float2half_rn(v0 - __half2float(h0)), __float2half_rn(v1 - __half2float(h1)));
                    }
                    fence_proxy_async_smem();
                }
                tc_fence_before_sync();
                __syncthreads();
                if (!ident)
                {
                    if (tid == 0)
                    {
                        tc_fence_after_sync();
                        const unsigned char *a = sA + stg * L::A_BYTES;
#pragma unroll
                        for (int s = 0; s < 6; ++s)
                            tc_mma_f16(taddr, tc_smem_desc(a + s * TC_SLAB_S, 128, 256), tc_smem_desc(sB + s * 1024, 128, 256),
                                       idesc, s > 0);
                        tc_commit(mma_bar);
                    }
                    mma_pending = true;
                    const bool mok = mbar_wait_bounded(mma_bar, mphase, &grp->error, cfg.wait_limit);
                    if (!__syncthreads_and(mok))
                    {
                        ok = false;
                        break;
                    }
                    mma_pending = false;
                    mphase ^= 1u;
                    tc_fence_after_sync();
                }
                if (w < 3)
                {
                    const int row = 32 * w + lane;
                    double *out = (coarse ? mas.zc + (size_t)(mat - banks) * N * G : z0 + (size_t)m * N * G) + (size_t)row * G;
                    const double *xr = x + row * G;
                    float hi[16], lo[16];
                    if (!ident)
                    {
                        const uint32_t ta = taddr + ((uint32_t)(32 * w) << 16);
                        tc_ld16(ta, hi);
                        tc_ld16(ta + 16, lo);
                        tc_wait_ld();
                    }
#pragma unroll
                    for (int gg = 0; gg < G; gg += 2)
                    {
                        double zv[2];
#pragma unroll
                        for (int h = 0; h < 2; ++h)
                        {
                            const double xin = xr[gg + h];
                            zv[h] = ident ? xin : (double)(hi[gg + h] + lo[gg + h]) * xsc_s[gg + h];
                            dsum[gg + h] = fma(zv[h], xin, dsum[gg + h]);
                        }
                        *reinterpret_cast<double2 *>(out + gg) = make_double2(zv[0], zv[1]);
                    }
                }
                tc_fence_before_sync();
                __syncthreads(); // accumulator read, the stage's A and X free
                const int mn = m + 2 * stride;
                pending[stg] = mn < items;
                if (tid == 0 && mn < items)
                    issue(mn, stg);
            }
            if (!ok && tid == 0)
            {
                // Leave nothing in flight: the MMAs and the bulk copies (bounded, default limit).
                if (mma_pending)
                    for (long long i = 0; i < MBAR_SPIN_LIMIT; ++i)
                        if (mbar_try_wait(mma_bar, mphase))
                            break;
                mbar_drain(tma_bar, pending, {tphase[0], tphase[1]});
            }
            flush(cat);
            tc_fence_before_sync();
            __syncthreads();
            if (w == 0)
            {
                tc_fence_after_sync();
                tmem_dealloc(taddr, 32);
            }
            // CTA sums (warps in order) into the first warp's slots, then the grid sum.
            double *cta = amax_s; // free now: 3 G doubles
            if (tid < 3 * G)
            {
                double s = 0.0;
                for (int ww = 0; ww < 4; ++ww)
                    s += wsum[ww * 3 * G + tid];
                cta[tid] = s;
            }
            __shared__ double totals[3 * G];
            if (grid_reduce_cta<3 * G, TC_THREADS>(cta, red.rz_parts, &grp->counter[4], totals) && tid == 0)
            {
                const double Lc = (double)cfg.level_num;
                int all_done = 1;
                for (int gg = 0; gg < G; ++gg)
                {
                    PcgState *sg = st + gg;
                    if (!sg->done)
                    {
                        sg->rz_coarse = totals[2 * G + gg] + Lc * totals[G + gg];
                        pcg_finalize(sg, cfg, MODE, totals[gg] + totals[G + gg] + sg->rz_coarse, 0.0);
                        if (sg->error)
                            grp->error = sg->error;
                    }
                    all_done &= sg->done ? 1 : 0;
                }
                grp->iter = MODE == 1 ? 0 : grp->iter + 1;
                if (all_done || grp->error)
                    grp->done = 1;
            }
        }

        // Coarse levels above the first from its components rc (level 0 of the coarse vector).
        // Each real node of level l sums its (at most 32) children of level l - 1 in a warp
        // (lane = child, in increasing order; deterministic). With three or more levels one CTA
        // (32 warps) per level-2 node computes its level-1 children (a warp each) and then itself
        // from them, so both levels take one round; a fourth level is summed by the last CTA to
        // finish (atomic ticket).
        constexpr int LEVEL_THREADS = 1024;

        template <int BD>
        __device__ __forceinline__ void kid_sum(const MasView &mas, int l, int i, bool cg, double (&v)[BD])
        {
            const int lane = threadIdx.x & 31;
            const int b = mas.kid_ptr[l][i], e = mas.kid_ptr[l][i + 1];
#pragma unroll
            for (int c = 0; c < BD; ++c)
                v[c] = 0.0;
            if (b + lane < e)
            {
                const size_t node = (size_t)mas.coff[l - 1] + mas.kids[b + lane];
#pragma unroll
                for (int c = 0; c < BD; ++c)
                    v[c] = cg ? __ldcg(mas.rc + node * BD + c) : mas.rc[node * BD + c];
            }
#pragma unroll
            for (int c = 0; c < BD; ++c)
                v[c] = warp_sum(v[c]);
        }

        template <int BD>
        __device__ __forceinline__ void coarse_levels_body(const MasView &mas, const PcgState *st, Cta cta)
        {
            pdl_wait();
            if (st && st->done)
                return;
            constexpr int W = LEVEL_THREADS / 32;
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            __shared__ double part[W][BD];
            __shared__ int is_last;
            if (mas.level_num == 2)
            {
                const int i = cta.x * W + w;
                if (i >= mas.real_count[1])
                    return;
                double v[BD];
                kid_sum<BD>(mas, 1, i, false, v);
                if (lane == 0)
#pragma unroll
                    for (int c = 0; c < BD; ++c)
                        mas.rc[((size_t)mas.coff[1] + i) * BD + c] = v[c];
                return;
            }
            // Level-2 node j = cta.x; warp w: its w-th level-1 child.
            const int j = cta.x;
            const int kb = mas.kid_ptr[2][j], ke = mas.kid_ptr[2][j + 1];
            if (kb + w < ke)
            {
                const int i = mas.kids[kb + w];
                double v[BD];
                kid_sum<BD>(mas, 1, i, false, v);
                if (lane == 0)
#pragma unroll
                    for (int c = 0; c < BD; ++c)
                    {
                        mas.rc[((size_t)mas.coff[1] + i) * BD + c] = v[c];
                        part[w][c] = v[c];
                    }
            }
            __syncthreads();
            if (w == 0)
            {
#pragma unroll
                for (int c = 0; c < BD; ++c)
                {
                    const double t = warp_sum(kb + lane < ke ? part[lane][c] : 0.0);
                    if (lane == 0)
                        mas.rc[((size_t)mas.coff[2] + j) * BD + c] = t;
                }
            }
            if (mas.level_num <= 3)
                return;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                __threadfence(); // cumulative: orders this CTA's stores (seen at the barrier) first
                is_last = atomicAdd(mas.ticket, 1u) == (unsigned)cta.n - 1;
            }
            __syncthreads();
            if (!is_last)
                return;
            __threadfence();
            for (int k = w; k < mas.real_count[3]; k += W)
            {
                double v[BD];
                kid_sum<BD>(mas, 3, k, true, v);
                if (lane == 0)
#pragma unroll
                    for (int c = 0; c < BD; ++c)
                        mas.rc[((size_t)mas.coff[3] + k) * BD + c] = v[c];
            }
            if (threadIdx.x == 0)
                *mas.ticket = 0u;
        }

        template <int BD>
        __global__ void __launch_bounds__(LEVEL_THREADS) k_coarse_levels(MasView mas, const PcgState *st)
        {
            coarse_levels_body<BD>(mas, st, native_cta());
        }

        template <int BD>
        __global__ void __launch_bounds__(LEVEL_THREADS) k_coarse_levels_batch(BatchView v)
        {
            const int4 e = batch_entry(v, BPH_COARSE);
            const BatchSystem &sy = v.sys[e.x];
            const Cta cta{e.y, e.z};
            const MasView mas = sy.mas;
            coarse_levels_body<BD>(mas, sy.st, cta);
        }

        // The coarse levels for nodes of NC components (the wide groups: 3 components x 16 right-hand
        // sides), the same sums as k_coarse_levels in chunks of CH components, so the registers do not
        // grow with NC.
        template <int NC, int CH>
        __device__ __forceinline__ void kid_sum_chunk(const MasView &mas, int l, int i, bool cg, int c0,
                                                      double (&v)[CH])
        {
            const int lane = threadIdx.x & 31;
            const int b = mas.kid_ptr[l][i], e = mas.kid_ptr[l][i + 1];
#pragma unroll
            for (int c = 0; c < CH; ++c)
                v[c] = 0.0;
            if (b + lane < e)
            {
                const size_t node = (size_t)mas.coff[l - 1] + mas.kids[b + lane];
#pragma unroll
                for (int c = 0; c < CH; ++c)
                    v[c] = cg ? __ldcg(mas.rc + node * NC + c0 + c) : mas.rc[node * NC + c0 + c];
            }
#pragma unroll
            for (int c = 0; c < CH; ++c)
                v[c] = warp_sum(v[c]);
        }

        template <int NC, int CH>
        __global__ void __launch_bounds__(LEVEL_THREADS) k_coarse_levels_c(MasView mas, const PcgState *grp)
        {
            static_assert(NC % CH == 0, "whole chunks");
            if (grp && grp->done)
                return;
            constexpr int W = LEVEL_THREADS / 32;
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            __shared__ double part[W][NC];
            __shared__ int is_last;
            if (mas.level_num == 2)
            {
                const int i = blockIdx.x * W + w;
                if (i >= mas.real_count[1])
                    return;
                for (int c0 = 0; c0 < NC; c0 += CH)
                {
                    double v[CH];
                    kid_sum_chunk<NC, CH>(mas, 1, i, false, c0, v);
                    if (lane == 0)
#pragma unroll
                        for (int c = 0; c < CH; ++c)
                            mas.rc[((size_t)mas.coff[1] + i) * NC + c0 + c] = v[c];
                }
                return;
            }
            const int j = blockIdx.x;
            const int kb = mas.kid_ptr[2][j], ke = mas.kid_ptr[2][j + 1];
            if (kb + w < ke)
            {
                const int i = mas.kids[kb + w];
                for (int c0 = 0; c0 < NC; c0 += CH)
                {
                    double v[CH];
                    kid_sum_chunk<NC, CH>(mas, 1, i, false, c0, v);
                    if (lane == 0)
#pragma unroll
                        for (int c = 0; c < CH; ++c)
                        {
                            mas.rc[((size_t)mas.coff[1] + i) * NC + c0 + c] = v[c];
                            part[w][c0 + c] = v[c];
                        }
                }
            }
            __syncthreads();
            // The level-2 node's components, one per warp (in the same order as one warp would sum them).
            for (int c = w; c < NC; c += W)
            {
                const double t = warp_sum(kb + lane < ke ? part[lane][c] : 0.0);
                if (lane == 0)
                    mas.rc[((size_t)mas.coff[2] + j) * NC + c] = t;
            }
            if (mas.level_num <= 3)
                return;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                __threadfence();
                is_last = atomicAdd(mas.ticket, 1u) == gridDim.x - 1;
            }
            __syncthreads();
            if (!is_last)
                return;
            __threadfence();
            for (int k = w; k < mas.real_count[3]; k += W)
                for (int c0 = 0; c0 < NC; c0 += CH)
                {
                    double v[CH];
                    kid_sum_chunk<NC, CH>(mas, 3, k, true, c0, v);
                    if (lane == 0)
#pragma unroll
                        for (int c = 0; c < CH; ++c)
                            mas.rc[((size_t)mas.coff[3] + k) * NC + c0 + c] = v[c];
                }
            if (threadIdx.x == 0)
                *mas.ticket = 0u;
        }

        // Level-0 restriction of r (initial residual, true-residual iterations, plain applies).
        // With period > 0 it runs only on iterations st->iter + 1 that are multiples of period.
        template <int BD>
        __device__ __forceinline__ void restrict_body(int banks, const double *__restrict__ r,
                                                      const int *__restrict__ lcco0, const int *__restrict__ cco0_base,
                                                      double *rc, const PcgState *st, int period, Cta cta)
        {
            pdl_wait();
            if (st && st->done)
                return;
            if (st && period > 0 && (st->iter + 1) % period != 0)
                return;
            const int lane = threadIdx.x & 31;
            const int bank = cta.x * 8 + (threadIdx.x >> 5);
            if (bank >= banks)
                return;
            const long long b0 = (long long)bank * 32 * BD;
            double reg[BD];
#pragma unroll
            for (int t = 0; t < BD; ++t)
                reg[t] = r[b0 + t * 32 + lane];
            bank_restrict<BD>(reg, bank, lcco0, cco0_base, rc);
        }

        template <int BD>
        __global__ void __launch_bounds__(256) k_restrict(int banks, const double *__restrict__ r,
                                                          const int *__restrict__ lcco0,
                                                          const int *__restrict__ cco0_base, double *rc,
                                                          const PcgState *st, int period)
        {
            restrict_body<BD>(banks, r, lcco0, cco0_base, rc, st, period, native_cta());
        }

        template <int BD>
        __global__ void __launch_bounds__(256) k_restrict_batch(BatchView v, int period)
        {
            const int4 e = batch_entry(v, BPH_RESTRICT);
            const BatchSystem &sy = v.sys[e.x];
            const Cta cta{e.y, e.z};
            restrict_body<BD>(sy.mas.first_iso_bank, sy.r, sy.mas.lcco0, sy.mas.cco0_base, sy.mas.rc, sy.st, period,
                              cta);
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

        template <int BD, class Store>
        void prepare_variant()
        {
            using L = ApplyLayout<BD, Store>;
            const int smem = L::WARPS * L::WARP_BYTES;
            cuda_check(cudaFuncSetAttribute(k_mas_apply<BD, Store, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            smem),
                       "apply smem attribute");
            cuda_check(cudaFuncSetAttribute(k_mas_apply<BD, Store, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            smem),
                       "apply smem attribute");
            cuda_check(cudaFuncSetAttribute(k_mas_apply<BD, Store, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            smem),
                       "apply smem attribute");
            cuda_check(cudaFuncSetAttribute(k_mas_apply_batch<BD, Store, 1>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "apply smem attribute");
            cuda_check(cudaFuncSetAttribute(k_mas_apply_batch<BD, Store, 2>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "apply smem attribute");
        }

        template <int BD, class Store, int MODE>
        void apply_launch_mode(const MasView &mas, const double *r, double *z, PcgState *st, ReduceBuf red,
                               PcgConfig cfg, cudaStream_t s)
        {
            using L = ApplyLayout<BD, Store>;
            const size_t smem = (size_t)L::WARPS * L::WARP_BYTES;
            const int grid = mas_apply_grid(mas);
            if (MODE != 0 && grid > red.capacity)
                throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
            // Chained in the PCG loop only: the kernel reads inverses before pdl_wait(), and a plain
            // apply may follow the kernels that write them.
            launch_chained(MODE != 0 && chained_launch(), k_mas_apply<BD, Store, MODE>, grid, L::WARPS * 32, smem, s,
                           mas, r, z, st, red, cfg);
        }

        template <int BD, class Store>
        void apply_launch(const MasView &mas, const double *r, double *z, PcgState *st, ReduceBuf red, PcgConfig cfg,
                          int mode, cudaStream_t s)
        {
            if (mode == 0)
                apply_launch_mode<BD, Store, 0>(mas, r, z, st, red, cfg, s);
            else if (mode == 1)
                apply_launch_mode<BD, Store, 1>(mas, r, z, st, red, cfg, s);
            else
                apply_launch_mode<BD, Store, 2>(mas, r, z, st, red, cfg, s);
        }

        // Calls f.template operator()<BD, Store>() for the block size and storage type.
        template <class F>
        auto dispatch(int bd, int storage, F &&f)
        {
            switch (storage)
            {
            case STORE_F64:
                return bd == 1 ? f.template operator()<1, double>()
                               : (bd == 2 ? f.template operator()<2, double>() : f.template operator()<3, double>());
            case STORE_F16:
                return bd == 1 ? f.template operator()<1, __half>()
                               : (bd == 2 ? f.template operator()<2, __half>() : f.template operator()<3, __half>());
            default:
                return bd == 1 ? f.template operator()<1, float>()
                               : (bd == 2 ? f.template operator()<2, float>() : f.template operator()<3, float>());
            }
        }

        template <class F>
        auto dispatch_bd(int bd, F &&f)
        {
            return bd == 1 ? f.template operator()<1>() : (bd == 2 ? f.template operator()<2>() : f.template operator()<3>());
        }
    } // namespace

    int device_sm_count()
    {
        // Per host thread: batched solves run handles on several threads at once.
        static thread_local int cached_dev = -1, cached = 148;
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

    void prepare_kernels(int bd, int storage)
    {
        device_sm_count();
        dispatch(bd, storage, [&]<int BD, class Store>() { prepare_variant<BD, Store>(); });
    }

    int restrict_grid(const MasView &mas)
    {
        if (mas.first_iso_bank <= 0 || mas.level_num <= 0)
            return 0;
        return (mas.first_iso_bank + 7) / 8;
    }

    int coarse_levels_grid(const MasView &mas)
    {
        if (mas.level_num <= 1 || mas.real_count[1] <= 0)
            return 0;
        const int grid = mas.level_num == 2 ? (mas.real_count[1] + LEVEL_THREADS / 32 - 1) / (LEVEL_THREADS / 32)
                                            : mas.real_count[2];
        return grid > 0 ? grid : 0;
    }

    // At least apply_items_per_warp() items per warp (1 by default: the most CTAs, the lowest
    // latency for a lone solve). In batches of small systems more items per warp measured
    // faster: a warp's two-stage copy pipeline runs past its start-up latency, and fewer SMs are
    // held by one system's apply while other systems' kernels run.
    int mas_apply_grid(const MasView &mas)
    {
        return dispatch(mas.bd, mas.storage, [&]<int BD, class Store>() {
            using L = ApplyLayout<BD, Store>;
            const int sms = device_sm_count();
            const int items = mas.banks + mas.n_coarse_active;
            const int per_cta = L::WARPS * apply_items_per_warp();
            int grid = (items + per_cta - 1) / per_cta;
            if (grid > sms)
                grid = sms;
            return grid < 1 ? 1 : grid;
        });
    }

    void launch_restrict_batch(const BatchView &v, int bd, int total, int period, cudaStream_t s)
    {
        if (total <= 0)
            return;
        dispatch_bd(bd, [&]<int BD>() {
            launch_chained(chained_launch(), k_restrict_batch<BD>, total, 256, 0, s, v, period);
        });
        cuda_check(cudaGetLastError(), "batched restrict launch");
    }

    void launch_coarse_levels_batch(const BatchView &v, int bd, int total, cudaStream_t s)
    {
        if (total <= 0)
            return;
        dispatch_bd(bd, [&]<int BD>() {
            launch_chained(chained_launch(), k_coarse_levels_batch<BD>, total, LEVEL_THREADS, 0, s, v);
        });
        cuda_check(cudaGetLastError(), "batched coarse levels launch");
    }

    void launch_mas_apply_batch(const BatchView &v, int bd, int storage, int total, int mode, cudaStream_t s)
    {
        if (mode != 1 && mode != 2)
            throw Error(ERR_INVALID, "[MAS] internal: batched applies are the initial and the iteration apply");
        if (total <= 0)
            return;
        dispatch(bd, storage, [&]<int BD, class Store>() {
            using L = ApplyLayout<BD, Store>;
            const size_t smem = (size_t)L::WARPS * L::WARP_BYTES;
            if (mode == 1)
                launch_chained(chained_launch(), k_mas_apply_batch<BD, Store, 1>, total, L::WARPS * 32, smem, s, v);
            else
                launch_chained(chained_launch(), k_mas_apply_batch<BD, Store, 2>, total, L::WARPS * 32, smem, s, v);
        });
        cuda_check(cudaGetLastError(), "batched apply launch");
    }

    int launch_restrict(const MasView &mas, const double *r, const PcgState *st, int period, cudaStream_t s)
    {
        const int grid = restrict_grid(mas);
        if (grid <= 0)
            return 0;
        dispatch_bd(mas.bd, [&]<int BD>() {
            launch_chained(chained_launch(), k_restrict<BD>, grid, 256, 0, s, mas.first_iso_bank, r, mas.lcco0,
                           mas.cco0_base, mas.rc, st, period);
        });
        return 1;
    }

    int launch_coarse_levels(const MasView &mas, const PcgState *st, cudaStream_t s)
    {
        const int grid = coarse_levels_grid(mas);
        if (grid <= 0)
            return 0;
        dispatch_bd(mas.bd,
                    [&]<int BD>() { launch_chained(chained_launch(), k_coarse_levels<BD>, grid, LEVEL_THREADS, 0, s, mas, st); });
        return 1;
    }

    void prepare_kernels_g(int bd)
    {
        dispatch_bd(bd, [&]<int BD>() {
            using L = ApplyLayoutG<BD>;
            const int smem = L::WARPS * L::WARP_BYTES;
            cuda_check(cudaFuncSetAttribute(k_mas_apply_g<BD, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "apply smem attribute");
            cuda_check(cudaFuncSetAttribute(k_mas_apply_g<BD, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "apply smem attribute");
        });
        if (bd == 3)
        {
            const int smem = ApplyLayoutW::WARPS * ApplyLayoutW::WARP_BYTES;
            cuda_check(cudaFuncSetAttribute(k_mas_apply_w<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "wide apply smem attribute");
            cuda_check(cudaFuncSetAttribute(k_mas_apply_w<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "wide apply smem attribute");
            cuda_check(cudaFuncSetAttribute(k_mas_apply_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            TcLayout::BYTES),
                       "tcgen05 apply smem attribute");
            cuda_check(cudaFuncSetAttribute(k_mas_apply_tc<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            TcLayout::BYTES),
                       "tcgen05 apply smem attribute");
        }
    }

    void launch_mas_apply_g(const MasView &mas, const double *r, double *z, PcgState *st, ReduceBuf red, PcgConfig cfg,
                            int mode, cudaStream_t s)
    {
        if (mas.storage != STORE_F16)
            throw Error(ERR_INVALID, "[MAS] several right-hand sides at once need precision fp16");
        dispatch_bd(mas.bd, [&]<int BD>() {
            using L = ApplyLayoutG<BD>;
            const int items = mas.banks + mas.n_coarse_active;
            int grid = (items + L::WARPS - 1) / L::WARPS;
            const int sms = device_sm_count();
            grid = grid > sms ? sms : (grid < 1 ? 1 : grid);
            if (grid * 3 * RHS_GROUP > red.capacity * 6)
                throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
            const size_t smem = (size_t)L::WARPS * L::WARP_BYTES;
            if (mode == 1)
                k_mas_apply_g<BD, 1><<<grid, L::WARPS * 32, smem, s>>>(mas, r, z, st, red, cfg);
            else
                k_mas_apply_g<BD, 2><<<grid, L::WARPS * 32, smem, s>>>(mas, r, z, st, red, cfg);
        });
        cuda_check(cudaGetLastError(), "multi apply launch");
    }

    int launch_coarse_levels_g(const MasView &mas, cudaStream_t s)
    {
        if (mas.level_num <= 1 || mas.real_count[1] <= 0)
            return 0;
        const int grid = mas.level_num == 2 ? (mas.real_count[1] + LEVEL_THREADS / 32 - 1) / (LEVEL_THREADS / 32)
                                            : mas.real_count[2];
        if (grid <= 0)
            return 0;
        dispatch_bd(mas.bd, [&]<int BD>() {
            k_coarse_levels<BD * RHS_GROUP><<<grid, LEVEL_THREADS, 0, s>>>(mas, nullptr);
        });
        cuda_check(cudaGetLastError(), "multi coarse levels launch");
        return 1;
    }

    int launch_coarse_levels_w(const MasView &mas, const PcgState *grp, cudaStream_t s)
    {
        if (mas.level_num <= 1 || mas.real_count[1] <= 0)
            return 0;
        const int grid = mas.level_num == 2 ? (mas.real_count[1] + LEVEL_THREADS / 32 - 1) / (LEVEL_THREADS / 32)
                                            : mas.real_count[2];
        if (grid <= 0)
            return 0;
        k_coarse_levels_c<3 * RHS_WIDE, 8><<<grid, LEVEL_THREADS, 0, s>>>(mas, grp);
        cuda_check(cudaGetLastError(), "wide coarse levels launch");
        return 1;
    }

    void launch_mas_apply_w(const MasView &mas, const double *r, double *z, PcgState *st, ReduceBuf red,
                            PcgConfig cfg, int mode, cudaStream_t s)
    {
        using L = ApplyLayoutW;
        if (mas.bd != 3 || mas.storage != STORE_F16)
            throw Error(ERR_INVALID, "[MAS] sixteen right-hand sides need block_dim 3 and fp16 inverses");
        const int items = mas.banks + mas.n_coarse_active;
        int grid = (items + L::WARPS - 1) / L::WARPS;
        const int sms = device_sm_count();
        grid = grid > sms ? sms : (grid < 1 ? 1 : grid);
        if (grid > red.capacity)
            throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
        const size_t smem = (size_t)L::WARPS * L::WARP_BYTES;
        if (mode == 1)
            k_mas_apply_w<1><<<grid, L::WARPS * 32, smem, s>>>(mas, r, z, st, red, cfg);
        else
            k_mas_apply_w<2><<<grid, L::WARPS * 32, smem, s>>>(mas, r, z, st, red, cfg);
        cuda_check(cudaGetLastError(), "wide apply launch");
    }

    size_t tc_storage_bytes(const MasView &mas) { return (size_t)(mas.banks + mas.total_coarse) * TC_MAT_BYTES; }

    void launch_inv_to_tc(const MasView &mas, void *out, cudaStream_t s)
    {
        if (mas.bd != 3 || mas.storage != STORE_F16)
            throw Error(ERR_INVALID, "[MAS] the tcgen05 apply needs block_dim 3 and fp16 inverses");
        const int mats = mas.banks + mas.total_coarse;
        if (mats > 0)
            k_inv_to_tc<<<mats, 256, 0, s>>>(static_cast<const __half *>(mas.inv), static_cast<__half *>(out));
        cuda_check(cudaGetLastError(), "tc storage launch");
    }

    void launch_mas_apply_tc(const MasView &mas, const void *inv_tc_v, const double *r, double *z, PcgState *st,
                             ReduceBuf red, PcgConfig cfg, int mode, cudaStream_t s)
    {
        const __half *inv_tc = static_cast<const __half *>(inv_tc_v);
        if (mas.bd != 3 || mas.storage != STORE_F16 || !inv_tc)
            throw Error(ERR_INVALID, "[MAS] the tcgen05 apply needs block_dim 3, fp16 inverses and the tc storage");
        const int items = mas.banks + mas.n_coarse_active;
        int grid = 2 * device_sm_count(); // two CTAs per SM (83 KB of shared memory each)
        grid = grid > items ? items : grid;
        grid = grid > red.capacity ? red.capacity : grid;
        grid = grid < 1 ? 1 : grid;
        const size_t smem = TcLayout::BYTES;
        if (mode == 1)
            k_mas_apply_tc<1><<<grid, TC_THREADS, smem, s>>>(mas, inv_tc, r, z, st, red, cfg);
        else
            k_mas_apply_tc<2><<<grid, TC_THREADS, smem, s>>>(mas, inv_tc, r, z, st, red, cfg);
        cuda_check(cudaGetLastError(), "tcgen05 apply launch");
    }

    void launch_mas_apply(const MasView &mas, const double *r, double *z, PcgState *st, ReduceBuf red, PcgConfig cfg,
                          int mode, cudaStream_t s)
    {
        dispatch(mas.bd, mas.storage,
                 [&]<int BD, class Store>() { apply_launch<BD, Store>(mas, r, z, st, red, cfg, mode, s); });
    }

    void launch_prolong(const MasView &mas, const double *z0, double *z, cudaStream_t s)
    {
        const long long len = (long long)mas.banks * 32 * mas.bd;
        long long g = (len + 255) / 256;
        if (g > 148 * 16)
            g = 148 * 16;
        if (g < 1)
            g = 1;
        dispatch_bd(mas.bd, [&]<int BD>() { k_prolong<BD><<<(int)g, 256, 0, s>>>(mas, z0, z); });
        cuda_check(cudaGetLastError(), "prolong launch");
    }
} // namespace pmas
