// Training of the learned warm start's network on the GPU (sm_100a): the project's own forward and
// backward kernels and an Adam step. No reference counterpart: the reference starts every solve from
// x0 = 0 (MASSolver.cu:395-398).
//
// A training sample is one step k of a sequence of systems with one pattern: the solver's own
// prediction pipeline, run with the kept solutions x_{k-1} .. x_{k-4}, gives the history guess x_g,
// its residual r_g = b - A x_g and the normalised features; the exact solution x_k gives the error
// e = x_k - x_g. The network's correction c should point along e in the energy norm; the loss is
//
//     1 - rho,   rho = (c . r_g)^2 / ((c . A c) (e . r_g))      (A e = r_g),
//
// the fraction of the history guess's squared energy error that remains after the optimal step
// along c (the solver's second Galerkin pass does at least as well). It is invariant to the scale of
// c. Samples live in HBM in the solver's padded (subdomain) block order: the banked pattern of the
// sequence (shared by its samples), the block values in FP32 (for A c), the neighbour weights and
// their transposes, the features, r_g, s_q and e . r_g.
//
// One step over a sample (128 vertices per CTA in every per-vertex kernel, so every kernel that
// contributes to the gradient writes one partial row per CTA; a fixed-order sum over the CTAs makes
// the gradient deterministic):
//
//   k_tr_in_fwd      z0 = W_in f + b_in (FP32), h0 = bf16(relu(z0))            (as k_ws_input)
//   k_ws_layer<true> x3: m = sum_j w_ij h_j, z = [h ; m] W_l^T + b_l on BF16 mma.sync with FP32
//                    accumulation, h' = bf16(h + relu(z)); m and z kept for the reverse pass
//   k_tr_out_fwd     c = s_q (W_out h3 + b_out)                                  (as k_ws_output)
//   k_tr_spmv_loss   A c (FP32 values, FP64 sums), c . r_g and c . A c (deterministic grid sum);
//                    the last CTA forms rho, the loss and dL/dc = k_r r_g + k_a A c
//   k_tr_out_bwd     g = s_q dL/dc, dL/dh3 = W_out^T g; partial dL/dW_out, dL/db_out
//   k_tr_layer_bwd   x3 (reverse): gz = dL/dh' * [z > 0] (bf16); on the tensor cores
//                    dL/d[h ; m] = gz W_l and the partial dL/dW_l = gz^T [h ; m]; partial dL/db_l
//   k_tr_gather_T    dL/dh = dL/dh' + dL/dh-part + sum_i w_ij dL/dm_i (the gather's transpose:
//                    a gather over the same symmetric pattern with the mirrored weights, no atomics)
//   k_tr_in_bwd      gz0 = dL/dh0 * [z0 > 0]; partial dL/dW_in, dL/db_in
//   k_tr_reduce      the gradient = the fixed-order sum of the per-CTA partials
//   k_tr_adam        Adam (FP32 state), and the BF16 copy of the layer weights for the next forward
//
// Rounding points (what the float64 oracle's emulation of this pass rounds): the forward rounds as
// inference does (h, m, W_l in bf16); the reverse pass rounds gz and W_l to bf16 for the two tensor-
// core products and keeps everything else in FP32 (the bias gradient sums the unrounded gz).

#include <algorithm>
#include <cmath>

#include "mas_ws_common.cuh"

namespace pmas
{
    namespace
    {
        constexpr int TT = TILE; // threads (= vertices) per CTA of the per-vertex training kernels
        static_assert(TILE == 128, "the training kernels assume 128-vertex tiles");
        constexpr int P = WS_PARAMS;
        constexpr int GS = H + 8; // shared row stride of the gz tile (bf16): 144 B, conflict-free
        constexpr int LB_THREADS = 256;
        constexpr int LB_SMEM = TILE * GS * 2 + TILE * TS * 2 + H * TS * 2 + 4 * H * 4;
        constexpr int GT_ROWS = 16; // rows per CTA of the transposed gather (two per warp)

        __device__ __forceinline__ void ldsm_x4_t(uint32_t (&a)[4], uint32_t addr)
        {
            asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                         : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                         : "r"(addr));
        }

        // ---- collection of a sample ------------------------------------------------------------

        // Block values to FP32, layout [slot][q][lane] (coalesced per q).
        __global__ void k_tr_vals32(BankedView A, long long slots, float *__restrict__ out)
        {
            const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            if (i >= slots * 32)
                return;
            const long long slot = i >> 5;
            const int lane = (int)(i & 31);
#pragma unroll
            for (int q = 0; q < 9; ++q)
                out[slot * 288 + q * 32 + lane] = (float)A.vals[banked_value_index(slot, lane, q, 3)];
        }

        // mirror[(s0 + k) * 32 + lane(u)] = the slot entry of row j = cols[...] that holds u (-1:
        // none); real[u] = the node has a row with a diagonal block (the network's vertices).
        __global__ void k_tr_mirror(BankedView A, const int *__restrict__ diag_slot, int *__restrict__ mirror,
                                    uint8_t *__restrict__ real)
        {
            const int u = blockIdx.x * blockDim.x + threadIdx.x;
            if (u >= A.banks * 32)
                return;
            const int lane = u & 31;
            const long long s0 = A.slice[u >> 5];
            const int len = A.rowlen[u];
            real[u] = node_real(A.rowlen, diag_slot, u) ? 1 : 0;
            for (int k = 0; k < len; ++k)
            {
                const int j = A.cols[(s0 + k) * 32 + lane];
                const long long sj = A.slice[j >> 5];
                const int lj = A.rowlen[j];
                long long found = -1;
                for (int k2 = 0; k2 < lj; ++k2)
                    if (A.cols[(sj + k2) * 32 + (j & 31)] == u)
                    {
                        found = (sj + k2) * 32 + (j & 31);
                        break;
                    }
                mirror[(s0 + k) * 32 + lane] = (int)found;
            }
        }

        __global__ void k_tr_weights_t(long long entries, const int *__restrict__ mirror,
                                       const float *__restrict__ wslot, float *__restrict__ wT)
        {
            const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            if (i >= entries)
                return;
            const int m = mirror[i];
            wT[i] = m >= 0 ? wslot[m] : 0.f;
        }

        // Normalised features (exactly as k_ws_input normalises them), 0 for other nodes.
        __global__ void k_tr_features(int nodes, const uint8_t *__restrict__ real, const float *__restrict__ raw,
                                      const WsState *ws, float *__restrict__ out)
        {
            const int u = blockIdx.x * blockDim.x + threadIdx.x;
            if (u >= nodes)
                return;
            float f[F];
#pragma unroll
            for (int i = 0; i < F; ++i)
                f[i] = 0.f;
            if (real[u])
            {
                const Norms nm = norms(ws);
#pragma unroll
                for (int i = 0; i < F; ++i)
                    f[i] = raw[(long long)u * F + i];
#pragma unroll
                for (int i = 0; i < 3; ++i)
                {
                    f[i] *= nm.iq;
                    f[3 + i] *= nm.iv;
                    f[6 + i] *= nm.ip;
                }
                f[15] -= nm.mlog;
            }
            float4 *dst = reinterpret_cast<float4 *>(out + (long long)u * F);
#pragma unroll
            for (int i = 0; i < F / 4; ++i)
                dst[i] = make_float4(f[4 * i], f[4 * i + 1], f[4 * i + 2], f[4 * i + 3]);
        }

        // sc[1] = e . r_g with e = x_exact - x_g, x_g = sum_i coef_hist_i v_i over the kept solutions;
        // the last CTA also stores sc[0] = s_q = rms of q = D^-1 r_g (the output scale).
        __global__ void __launch_bounds__(256) k_tr_error_dot(WsHistory h, const WsState *ws,
                                                              const double *__restrict__ xe,
                                                              const double *__restrict__ rg, size_t len,
                                                              double *partials, unsigned *counter, double *sc)
        {
            double cf[WS_HISTORY];
#pragma unroll
            for (int i = 0; i < WS_HISTORY; ++i)
                cf[i] = ws->coef_hist[i];
            double acc[1] = {0.0};
            for (size_t k = (size_t)blockIdx.x * 256 + threadIdx.x; k < len; k += (size_t)gridDim.x * 256)
            {
                double xg = cf[0] * h.x[0][k];
#pragma unroll
                for (int i = 1; i < WS_HISTORY; ++i)
                    xg += cf[i] * (h.x[i - 1][k] - h.x[i][k]);
                acc[0] = fma(xe[k] - xg, rg[k], acc[0]);
            }
            double tot[1];
            if (grid_reduce<1, 256>(acc, partials, counter, tot) && threadIdx.x == 0)
            {
                const double cnt = ws->sums[4];
                sc[0] = cnt > 0.0 ? sqrt(ws->sums[0] / (3.0 * cnt)) : 0.0;
                sc[1] = tot[0];
            }
        }

        // ---- forward ---------------------------------------------------------------------------

        __global__ void __launch_bounds__(TT) k_tr_in_fwd(int nodes, const uint8_t *__restrict__ real,
                                                          const float *__restrict__ feat, const float *__restrict__ prm,
                                                          float *__restrict__ z0, __nv_bfloat162 *__restrict__ h)
        {
            __shared__ __align__(16) float wsm[H * F + H];
            for (int i = threadIdx.x; i < H * F + H; i += TT)
                wsm[i] = prm[OFF_WIN + i];
            __syncthreads();
            const int u = blockIdx.x * TT + threadIdx.x;
            if (u >= nodes)
                return;
            uint4 *dst = reinterpret_cast<uint4 *>(h + (long long)u * (H / 2));
            float4 *zd = reinterpret_cast<float4 *>(z0 + (long long)u * H);
            if (!real[u])
            {
#pragma unroll
                for (int i = 0; i < H / 8; ++i)
                    dst[i] = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
                for (int i = 0; i < H / 4; ++i)
                    zd[i] = make_float4(0.f, 0.f, 0.f, 0.f);
                return;
            }
            float f[F];
            const float4 *fp = reinterpret_cast<const float4 *>(feat + (long long)u * F);
#pragma unroll
            for (int i = 0; i < F / 4; ++i)
            {
                const float4 t = fp[i];
                f[4 * i] = t.x;
                f[4 * i + 1] = t.y;
                f[4 * i + 2] = t.z;
                f[4 * i + 3] = t.w;
            }
#pragma unroll
            for (int c = 0; c < H / 8; ++c)
            {
                uint4 out;
                __nv_bfloat162 *ob = reinterpret_cast<__nv_bfloat162 *>(&out);
                float zz[8];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    const int o0 = c * 8 + 2 * k, o1 = o0 + 1;
                    float a0 = wsm[H * F + o0], a1 = wsm[H * F + o1];
#pragma unroll
                    for (int i = 0; i < F; ++i)
                    {
                        a0 = fmaf(wsm[o0 * F + i], f[i], a0);
                        a1 = fmaf(wsm[o1 * F + i], f[i], a1);
                    }
                    ob[k] = __float22bfloat162_rn(make_float2(fmaxf(a0, 0.f), fmaxf(a1, 0.f)));
                    zz[2 * k] = a0;
                    zz[2 * k + 1] = a1;
                }
                dst[c] = out;
                zd[2 * c] = make_float4(zz[0], zz[1], zz[2], zz[3]);
                zd[2 * c + 1] = make_float4(zz[4], zz[5], zz[6], zz[7]);
            }
        }

        __global__ void __launch_bounds__(TT) k_tr_out_fwd(int nodes, const uint8_t *__restrict__ real,
                                                           const __nv_bfloat162 *__restrict__ h,
                                                           const float *__restrict__ prm, const double *__restrict__ sc,
                                                           double *__restrict__ c)
        {
            __shared__ float wo[3 * H + 3];
            for (int i = threadIdx.x; i < 3 * H + 3; i += TT)
                wo[i] = prm[OFF_WOUT + i];
            __syncthreads();
            const int u = blockIdx.x * TT + threadIdx.x;
            if (u >= nodes)
                return;
            if (!real[u])
            {
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    c[(long long)u * 3 + i] = 0.0;
                return;
            }
            const double sq = sc[0];
            const uint4 *src = reinterpret_cast<const uint4 *>(h + (long long)u * (H / 2));
            float s3[3] = {wo[3 * H], wo[3 * H + 1], wo[3 * H + 2]};
#pragma unroll
            for (int ch = 0; ch < H / 8; ++ch)
            {
                const uint4 q = src[ch];
                const __nv_bfloat162 *qb = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    const float2 hv = __bfloat1622float2(qb[k]);
                    const int o = ch * 8 + 2 * k;
#pragma unroll
                    for (int i = 0; i < 3; ++i)
                        s3[i] = fmaf(wo[i * H + o + 1], hv.y, fmaf(wo[i * H + o], hv.x, s3[i]));
                }
            }
#pragma unroll
            for (int i = 0; i < 3; ++i)
                c[(long long)u * 3 + i] = sq * (double)s3[i];
        }

        // A c over the sample's FP32 block values (warp per bank, lane per row), c . r_g, c . A c;
        // the last CTA forms rho, the loss and the coefficients of dL/dc = k_r r_g + k_a A c.
        __global__ void __launch_bounds__(256) k_tr_spmv_loss(WsTrainView S, const double *__restrict__ c,
                                                              double *__restrict__ Ac, WsTrainState *st,
                                                              double *partials)
        {
            const int lane = threadIdx.x & 31;
            const int bank = blockIdx.x * 8 + (threadIdx.x >> 5);
            double part[2] = {0.0, 0.0};
            if (bank < S.banks)
            {
                const int u = bank * 32 + lane;
                const long long s0 = S.slice[bank];
                const int len = S.rowlen[u];
                double acc[3] = {0.0, 0.0, 0.0};
                for (int k = 0; k < len; ++k)
                {
                    const long long slot = s0 + k;
                    const int col = S.cols[slot * 32 + lane];
                    const float *v = S.vals32 + slot * 288 + lane;
                    const double x0 = c[(long long)col * 3], x1 = c[(long long)col * 3 + 1],
                                 x2 = c[(long long)col * 3 + 2];
#pragma unroll
                    for (int i = 0; i < 3; ++i)
                    {
                        acc[i] = fma((double)v[(3 * i) * 32], x0, acc[i]);
                        acc[i] = fma((double)v[(3 * i + 1) * 32], x1, acc[i]);
                        acc[i] = fma((double)v[(3 * i + 2) * 32], x2, acc[i]);
                    }
                }
#pragma unroll
                for (int i = 0; i < 3; ++i)
                {
                    const long long k = (long long)u * 3 + i;
                    Ac[k] = acc[i];
                    part[0] = fma(c[k], S.re[k], part[0]);
                    part[1] = fma(c[k], acc[i], part[1]);
                }
            }
            double tot[2];
            if (grid_reduce<2, 256>(part, partials, &st->counter[0], tot) && threadIdx.x == 0)
            {
                const double a = tot[0], q = tot[1], ere = S.sc[1];
                const bool ok = q > 0.0 && ere > 0.0 && isfinite(a) && isfinite(q);
                st->a = a;
                st->q = q;
                st->rho = ok ? a * a / (q * ere) : 0.0;
                st->loss = 1.0 - st->rho;
                // d(1 - rho)/dc = -2a/(q ere) r_g + 2a^2/(q^2 ere) A c
                st->kr = ok ? -2.0 * a / (q * ere) : 0.0;
                st->ka = ok ? 2.0 * a * a / (q * q * ere) : 0.0;
            }
        }

        // ---- reverse pass ----------------------------------------------------------------------

        __global__ void __launch_bounds__(TT) k_tr_out_bwd(WsTrainView S, const __nv_bfloat16 *__restrict__ h3,
                                                           const double *__restrict__ Ac, const WsTrainState *st,
                                                           const float *__restrict__ prm, float *__restrict__ gh,
                                                           float *__restrict__ partials)
        {
            __shared__ float wo[3 * H];
            __shared__ float gs[TT][3];
            __shared__ float hs[TT][H + 1];
            const int nodes = S.banks * 32;
            for (int i = threadIdx.x; i < 3 * H; i += TT)
                wo[i] = prm[OFF_WOUT + i];
            const int base = blockIdx.x * TT;
            for (int i = threadIdx.x; i < TT * H; i += TT)
            {
                const int v = i / H, k = i % H, u = base + v;
                hs[v][k] = (u < nodes && S.real[u]) ? __bfloat162float(h3[(long long)u * H + k]) : 0.f;
            }
            const int u = base + threadIdx.x;
            float g[3] = {0.f, 0.f, 0.f};
            if (u < nodes && S.real[u])
            {
                const double sq = S.sc[0], kr = st->kr, ka = st->ka;
#pragma unroll
                for (int i = 0; i < 3; ++i)
                {
                    const long long k = (long long)u * 3 + i;
                    g[i] = (float)(sq * (kr * S.re[k] + ka * Ac[k]));
                }
            }
#pragma unroll
            for (int i = 0; i < 3; ++i)
                gs[threadIdx.x][i] = g[i];
            __syncthreads();
            if (u < nodes)
            {
                float4 *gd = reinterpret_cast<float4 *>(gh + (long long)u * H);
#pragma unroll
                for (int k4 = 0; k4 < H / 4; ++k4)
                {
                    float o[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                    {
                        const int k = 4 * k4 + j;
                        o[j] = fmaf(g[2], wo[2 * H + k], fmaf(g[1], wo[H + k], g[0] * wo[k]));
                    }
                    gd[k4] = make_float4(o[0], o[1], o[2], o[3]);
                }
            }
            float *prow = partials + (size_t)blockIdx.x * P;
            for (int p = threadIdx.x; p < 3 * H + 3; p += TT)
            {
                float s = 0.f;
                if (p < 3 * H)
                {
                    const int i = p / H, k = p % H;
                    for (int v = 0; v < TT; ++v)
                        s = fmaf(gs[v][i], hs[v][k], s);
                }
                else
                    for (int v = 0; v < TT; ++v)
                        s += gs[v][p - 3 * H];
                prow[OFF_WOUT + p] = s;
            }
        }

        // Reverse pass of one layer for a tile of 128 vertices (8 warps): gz = dL/dh' * [z > 0];
        // dL/d[h ; m] = gz W_l (each warp: its 16 vertices x 128) and the partial dL/dW_l = gz^T [h ; m]
        // (each warp: 16 outputs x 64 inputs, K = the 128 vertices) on BF16 mma.sync.
        __global__ void __launch_bounds__(LB_THREADS) k_tr_layer_bwd(WsTrainView S, const float *__restrict__ ghn,
                                                                     const float *__restrict__ z,
                                                                     const __nv_bfloat16 *__restrict__ hl,
                                                                     const __nv_bfloat16 *__restrict__ ml,
                                                                     const uint16_t *__restrict__ wl, int layer,
                                                                     float *__restrict__ g1, float *__restrict__ gm,
                                                                     float *__restrict__ partials)
        {
            extern __shared__ __align__(16) unsigned char lb_smem[];
            __nv_bfloat16 *GZ = reinterpret_cast<__nv_bfloat16 *>(lb_smem);
            __nv_bfloat16 *T = GZ + TILE * GS;
            __nv_bfloat16 *Wsm = T + TILE * TS;
            float *bsum = reinterpret_cast<float *>(Wsm + H * TS);
            const int nodes = S.banks * 32;
            const int base = blockIdx.x * TILE;
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            {
                // gz (bf16) and the bias partial: thread = (hidden unit, group of 32 vertices).
                const int k = threadIdx.x & (H - 1), grp = threadIdx.x >> 6;
                float bs = 0.f;
                for (int vv = 0; vv < 32; ++vv)
                {
                    const int v = grp * 32 + vv, u = base + v;
                    float gz = 0.f;
                    if (u < nodes && S.real[u])
                    {
                        const long long i = (long long)u * H + k;
                        gz = z[i] > 0.f ? ghn[i] : 0.f;
                    }
                    GZ[v * GS + k] = __float2bfloat16_rn(gz);
                    bs += gz;
                }
                bsum[grp * H + k] = bs;
            }
            // [h ; m] rows: 16 chunks of 8 bf16 (eight of h, eight of m) per vertex.
            for (int i = threadIdx.x; i < TILE * 16; i += LB_THREADS)
            {
                const int row = i >> 4, ch = i & 15, u = base + row;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (u < nodes)
                    v = ch < 8 ? *reinterpret_cast<const uint4 *>(hl + (long long)u * H + ch * 8)
                               : *reinterpret_cast<const uint4 *>(ml + (long long)u * H + (ch - 8) * 8);
                *reinterpret_cast<uint4 *>(&T[row * TS + ch * 8]) = v;
            }
            for (int i = threadIdx.x; i < H * 16; i += LB_THREADS)
            {
                const int row = i >> 4, ch = i & 15;
                *reinterpret_cast<uint4 *>(&Wsm[row * TS + ch * 8]) =
                    __ldg(reinterpret_cast<const uint4 *>(wl + row * 2 * H) + ch);
            }
            __syncthreads();
            const uint32_t gzb = smem_addr(GZ), tb = smem_addr(T), wb = smem_addr(Wsm);
            const int r8 = lane & 7, mat = lane >> 3;
            const int g = lane >> 2, c2 = (lane & 3) * 2;
            {
                // dL/d[h ; m] = gz (16 x 64 per warp) x W_l (64 x 128).
                float d[16][4];
#pragma unroll
                for (int nt = 0; nt < 16; ++nt)
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        d[nt][i] = 0.f;
                const int arow = warp * 16 + (lane & 15), acol = (lane >> 4) * 8;
#pragma unroll
                for (int ks = 0; ks < H / 16; ++ks)
                {
                    uint32_t a[4];
                    ldsm_x4(a, gzb + (uint32_t)((arow * GS + ks * 16 + acol) * 2));
#pragma unroll
                    for (int np = 0; np < 8; ++np)
                    {
                        uint32_t b[4];
                        const int krow = ks * 16 + r8 + (mat & 1) * 8, ncol = np * 16 + (mat >> 1) * 8;
                        ldsm_x4_t(b, wb + (uint32_t)((krow * TS + ncol) * 2));
                        mma_bf16(d[2 * np], a, b[0], b[1]);
                        mma_bf16(d[2 * np + 1], a, b[2], b[3]);
                    }
                }
#pragma unroll
                for (int half = 0; half < 2; ++half)
                {
                    const int u = base + warp * 16 + g + half * 8;
                    if (u >= nodes)
                        continue;
#pragma unroll
                    for (int nt = 0; nt < 16; ++nt)
                    {
                        const int col = nt * 8 + c2;
                        const float2 v = make_float2(d[nt][2 * half], d[nt][2 * half + 1]);
                        if (col < H)
                        {
                            const float2 gn = *reinterpret_cast<const float2 *>(ghn + (long long)u * H + col);
                            const bool rl = S.real[u] != 0;
                            *reinterpret_cast<float2 *>(g1 + (long long)u * H + col) =
                                rl ? make_float2(gn.x + v.x, gn.y + v.y) : make_float2(0.f, 0.f);
                        }
                        else
                            *reinterpret_cast<float2 *>(gm + (long long)u * H + (col - H)) = v;
                    }
                }
            }
            {
                // Partial dL/dW_l = gz^T (64 x 128 vertices) x [h ; m] (128 vertices x 128): warp w
                // takes outputs 16 (w & 3) .. + 15 and inputs 64 (w >> 2) .. + 63.
                const int m0 = (warp & 3) * 16, n0 = (warp >> 2) * 64;
                float e[8][4];
#pragma unroll
                for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        e[nt][i] = 0.f;
#pragma unroll
                for (int ks = 0; ks < TILE / 16; ++ks)
                {
                    uint32_t a[4];
                    {
                        const int vrt = ks * 16 + r8 + (mat >> 1) * 8, unit = m0 + (mat & 1) * 8;
                        ldsm_x4_t(a, gzb + (uint32_t)((vrt * GS + unit) * 2));
                    }
#pragma unroll
                    for (int np = 0; np < 4; ++np)
                    {
                        uint32_t b[4];
                        const int vrt = ks * 16 + r8 + (mat & 1) * 8, feat = n0 + np * 16 + (mat >> 1) * 8;
                        ldsm_x4_t(b, tb + (uint32_t)((vrt * TS + feat) * 2));
                        mma_bf16(e[2 * np], a, b[0], b[1]);
                        mma_bf16(e[2 * np + 1], a, b[2], b[3]);
                    }
                }
                float *prow = partials + (size_t)blockIdx.x * P + off_layer(layer);
#pragma unroll
                for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                    for (int half = 0; half < 2; ++half)
                    {
                        const int unit = m0 + g + half * 8, feat = n0 + nt * 8 + c2;
                        prow[unit * 2 * H + feat] = e[nt][2 * half];
                        prow[unit * 2 * H + feat + 1] = e[nt][2 * half + 1];
                    }
                if (threadIdx.x < H)
                    prow[H * 2 * H + threadIdx.x] = bsum[threadIdx.x] + bsum[H + threadIdx.x] +
                                                    bsum[2 * H + threadIdx.x] + bsum[3 * H + threadIdx.x];
            }
        }

        // dL/dh_j = g1_j + sum over the row's slots of wT * gm[col] (wT: the weight w_ij of the
        // mirrored entry, i.e. how much h_j fed m_i); half a warp per row, 4 values per lane.
        __global__ void __launch_bounds__(256) k_tr_gather_t(WsTrainView S, const float *__restrict__ g1,
                                                             const float *__restrict__ gm, float *__restrict__ gh)
        {
            const int nodes = S.banks * 32;
            const int lane = threadIdx.x & 31, hl = lane & 15;
            const int j = blockIdx.x * GT_ROWS + (threadIdx.x >> 4);
            const bool valid = j < nodes;
            const int len = valid ? S.rowlen[j] : 0;
            const long long s0 = valid ? S.slice[j >> 5] : 0;
            int maxlen = max(len, __shfl_xor_sync(FULL, len, 16));
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
            if (valid)
                acc = reinterpret_cast<const float4 *>(g1)[(long long)j * (H / 4) + hl];
            const float4 *gm4 = reinterpret_cast<const float4 *>(gm);
            for (int k0 = 0; k0 < maxlen; k0 += 16)
            {
                const int kk = k0 + hl;
                int col = valid ? j : 0;
                float w = 0.f;
                if (kk < len)
                {
                    const long long e = (s0 + kk) * 32 + (j & 31);
                    col = S.cols[e];
                    w = S.wT[e];
                }
                const int cnt = min(16, maxlen - k0);
                for (int q = 0; q < cnt; ++q)
                {
                    const int cq = __shfl_sync(FULL, col, q, 16);
                    const float wq = __shfl_sync(FULL, w, q, 16);
                    const float4 v = gm4[(long long)cq * (H / 4) + hl];
                    acc.x = fmaf(wq, v.x, acc.x);
                    acc.y = fmaf(wq, v.y, acc.y);
                    acc.z = fmaf(wq, v.z, acc.z);
                    acc.w = fmaf(wq, v.w, acc.w);
                }
            }
            if (valid)
                reinterpret_cast<float4 *>(gh)[(long long)j * (H / 4) + hl] =
                    S.real[j] ? acc : make_float4(0.f, 0.f, 0.f, 0.f);
        }

        __global__ void __launch_bounds__(TT) k_tr_in_bwd(WsTrainView S, const float *__restrict__ gh0,
                                                          const float *__restrict__ z0, float *__restrict__ partials)
        {
            __shared__ float G[TT][H + 1];
            __shared__ float Fm[TT][F + 1];
            const int nodes = S.banks * 32;
            const int base = blockIdx.x * TT;
            for (int i = threadIdx.x; i < TT * H; i += TT)
            {
                const int v = i / H, k = i % H, u = base + v;
                float gz = 0.f;
                if (u < nodes && S.real[u])
                {
                    const long long e = (long long)u * H + k;
                    gz = z0[e] > 0.f ? gh0[e] : 0.f;
                }
                G[v][k] = gz;
            }
            for (int i = threadIdx.x; i < TT * F; i += TT)
            {
                const int v = i / F, f = i % F, u = base + v;
                Fm[v][f] = (u < nodes && S.real[u]) ? S.feat[(long long)u * F + f] : 0.f;
            }
            __syncthreads();
            float *prow = partials + (size_t)blockIdx.x * P;
            for (int p = threadIdx.x; p < H * F + H; p += TT)
            {
                float s = 0.f;
                if (p < H * F)
                {
                    const int k = p / F, f = p % F;
                    for (int v = 0; v < TT; ++v)
                        s = fmaf(G[v][k], Fm[v][f], s);
                }
                else
                    for (int v = 0; v < TT; ++v)
                        s += G[v][p - H * F];
                prow[OFF_WIN + p] = s;
            }
        }

        __global__ void k_tr_reduce(int ctas, const float *__restrict__ partials, float *__restrict__ grad)
        {
            const int p = blockIdx.x * blockDim.x + threadIdx.x;
            if (p >= P)
                return;
            float s = 0.f;
            for (int c = 0; c < ctas; ++c)
                s += partials[(size_t)c * P + p];
            grad[p] = s;
        }

        // Adam (torch's formulation: p -= lr / (1 - b1^t) * m / (sqrt(v) / sqrt(1 - b2^t) + eps)) and
        // the BF16 copy of the layer weights (round to nearest even, as the host conversion).
        __global__ void k_tr_adam(float *__restrict__ prm, float *__restrict__ m, float *__restrict__ v,
                                  const float *__restrict__ grad, uint16_t *__restrict__ wl, float lr, float b1,
                                  float b2, float eps, float bc1, float bc2_sqrt)
        {
            const int p = blockIdx.x * blockDim.x + threadIdx.x;
            if (p >= P)
                return;
            const float gp = grad[p];
            const float mp = b1 * m[p] + (1.f - b1) * gp;
            const float vp = b2 * v[p] + (1.f - b2) * gp * gp;
            m[p] = mp;
            v[p] = vp;
            const float np = prm[p] - (lr / bc1) * mp / (sqrtf(vp) / bc2_sqrt + eps);
            prm[p] = np;
            for (int l = 0; l < WS_LAYERS; ++l)
            {
                const int o = p - off_layer(l);
                if (o >= 0 && o < WS_LAYER_WEIGHTS)
                    wl[(size_t)l * WS_LAYER_WEIGHTS + o] = __bfloat16_as_ushort(__float2bfloat16_rn(np));
            }
        }

        __global__ void k_tr_weights_bf16(const float *__restrict__ prm, uint16_t *__restrict__ wl)
        {
            const int i = blockIdx.x * blockDim.x + threadIdx.x;
            if (i >= WS_LAYERS * WS_LAYER_WEIGHTS)
                return;
            const int l = i / WS_LAYER_WEIGHTS, o = i % WS_LAYER_WEIGHTS;
            wl[i] = __bfloat16_as_ushort(__float2bfloat16_rn(prm[off_layer(l) + o]));
        }

        int ctas_of(int nodes) { return (nodes + TILE - 1) / TILE; }
    } // namespace

    int ws_train_ctas(int nodes) { return ctas_of(nodes); }

    void launch_tr_pattern(const BankedView &A, const int *diag_slot, long long slots, int *mirror, uint8_t *real,
                           cudaStream_t s)
    {
        const int nodes = A.banks * 32;
        cuda_check(cudaMemsetAsync(mirror, 0xFF, sizeof(int) * (size_t)slots * 32, s), "mirror reset");
        if (nodes == 0)
            return;
        k_tr_mirror<<<(nodes + 255) / 256, 256, 0, s>>>(A, diag_slot, mirror, real);
        cuda_check(cudaGetLastError(), "training mirror launch");
    }

    void launch_tr_sample(const BankedView &A, long long slots, const int *mirror, const uint8_t *real,
                          const float *wslot, const float *feat_raw, const WsState *ws, const double *rg,
                          const WsHistory &hist, const double *x_exact, size_t len, float *vals32, float *wslot_out,
                          float *wT, float *feat, double *re, double *sc, double *partials, unsigned *counter,
                          int capacity, cudaStream_t s)
    {
        const int nodes = A.banks * 32;
        const long long entries = slots * 32;
        if (entries > 0)
        {
            const unsigned g = (unsigned)((entries + 255) / 256);
            k_tr_vals32<<<g, 256, 0, s>>>(A, slots, vals32);
            cuda_check(cudaGetLastError(), "training values launch");
            k_tr_weights_t<<<g, 256, 0, s>>>(entries, mirror, wslot, wT);
            cuda_check(cudaGetLastError(), "training weights launch");
            cuda_check(cudaMemcpyAsync(wslot_out, wslot, sizeof(float) * entries, cudaMemcpyDeviceToDevice, s),
                       "training weights copy");
        }
        if (nodes > 0)
        {
            k_tr_features<<<(nodes + 255) / 256, 256, 0, s>>>(nodes, real, feat_raw, ws, feat);
            cuda_check(cudaGetLastError(), "training features launch");
        }
        cuda_check(cudaMemcpyAsync(re, rg, sizeof(double) * len, cudaMemcpyDeviceToDevice, s), "training residual copy");
        const int grid = std::min(capacity, std::max(1, (int)((len + 255) / 256)));
        cuda_check(cudaMemsetAsync(counter, 0, sizeof(unsigned), s), "ticket reset");
        k_tr_error_dot<<<grid, 256, 0, s>>>(hist, ws, x_exact, rg, len, partials, counter, sc);
        cuda_check(cudaGetLastError(), "training error dot launch");
    }

    int launch_tr_forward(const WsTrainView &S, const float *prm, const uint16_t *wl, const WsTrainScratch &w,
                          cudaStream_t s)
    {
        const int nodes = S.banks * 32;
        const int ctas = ctas_of(nodes);
        if (nodes == 0)
            return 0;
        k_tr_in_fwd<<<ctas, TT, 0, s>>>(nodes, S.real, S.feat, prm, w.z0, reinterpret_cast<__nv_bfloat162 *>(w.h[0]));
        cuda_check(cudaGetLastError(), "training input launch");
        constexpr int LAYER_SMEM = (TILE + H) * TS * 2 + H * 4;
        cuda_check(cudaFuncSetAttribute(k_ws_layer<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, LAYER_SMEM),
                   "layer smem attribute");
        const BankedView A{3, S.banks, S.slice, S.rowlen, S.cols, nullptr};
        for (int l = 0; l < WS_LAYERS; ++l)
        {
            k_ws_layer<true><<<ctas, LT, LAYER_SMEM, s>>>(
                A, S.wslot, reinterpret_cast<const __nv_bfloat16 *>(w.h[l]), wl + (size_t)l * WS_LAYER_WEIGHTS,
                prm + off_layer(l) + H * 2 * H, S.diag_slot, reinterpret_cast<__nv_bfloat16 *>(w.h[l + 1]),
                reinterpret_cast<__nv_bfloat16 *>(w.m[l]), w.z[l]);
            cuda_check(cudaGetLastError(), "training layer launch");
        }
        k_tr_out_fwd<<<ctas, TT, 0, s>>>(nodes, S.real, reinterpret_cast<const __nv_bfloat162 *>(w.h[WS_LAYERS]),
                                         prm, S.sc, w.c);
        cuda_check(cudaGetLastError(), "training output launch");
        k_tr_spmv_loss<<<(S.banks + 7) / 8, 256, 0, s>>>(S, w.c, w.Ac, w.st, w.red);
        cuda_check(cudaGetLastError(), "training loss launch");
        return 3 + WS_LAYERS;
    }

    int launch_tr_backward(const WsTrainView &S, const float *prm, const uint16_t *wl, const WsTrainScratch &w,
                           float *grad, cudaStream_t s)
    {
        const int nodes = S.banks * 32;
        const int ctas = ctas_of(nodes);
        if (nodes == 0)
        {
            cuda_check(cudaMemsetAsync(grad, 0, sizeof(float) * P, s), "gradient reset");
            return 0;
        }
        k_tr_out_bwd<<<ctas, TT, 0, s>>>(S, reinterpret_cast<const __nv_bfloat16 *>(w.h[WS_LAYERS]), w.Ac, w.st, prm,
                                         w.gh, w.partials);
        cuda_check(cudaGetLastError(), "training output reverse launch");
        cuda_check(cudaFuncSetAttribute(k_tr_layer_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, LB_SMEM),
                   "layer reverse smem attribute");
        for (int l = WS_LAYERS - 1; l >= 0; --l)
        {
            k_tr_layer_bwd<<<ctas, LB_THREADS, LB_SMEM, s>>>(
                S, w.gh, w.z[l], reinterpret_cast<const __nv_bfloat16 *>(w.h[l]),
                reinterpret_cast<const __nv_bfloat16 *>(w.m[l]), wl + (size_t)l * WS_LAYER_WEIGHTS, l, w.g1, w.gm,
                w.partials);
            cuda_check(cudaGetLastError(), "training layer reverse launch");
            k_tr_gather_t<<<(nodes + GT_ROWS - 1) / GT_ROWS, 256, 0, s>>>(S, w.g1, w.gm, w.gh);
            cuda_check(cudaGetLastError(), "training gather reverse launch");
        }
        k_tr_in_bwd<<<ctas, TT, 0, s>>>(S, w.gh, w.z0, w.partials);
        cuda_check(cudaGetLastError(), "training input reverse launch");
        k_tr_reduce<<<(P + 255) / 256, 256, 0, s>>>(ctas, w.partials, grad);
        cuda_check(cudaGetLastError(), "training reduce launch");
        return 3 + 2 * WS_LAYERS;
    }

    void launch_tr_adam(float *prm, float *m, float *v, const float *grad, uint16_t *wl, float lr, long long step,
                        cudaStream_t s)
    {
        const double b1 = 0.9, b2 = 0.999;
        const float bc1 = (float)(1.0 - std::pow(b1, (double)step));
        const float bc2s = (float)std::sqrt(1.0 - std::pow(b2, (double)step));
        k_tr_adam<<<(P + 255) / 256, 256, 0, s>>>(prm, m, v, grad, wl, lr, (float)b1, (float)b2, 1e-8f, bc1, bc2s);
        cuda_check(cudaGetLastError(), "training adam launch");
    }

    void launch_tr_weights_bf16(const float *prm, uint16_t *wl, cudaStream_t s)
    {
        const int n = WS_LAYERS * WS_LAYER_WEIGHTS;
        k_tr_weights_bf16<<<(n + 255) / 256, 256, 0, s>>>(prm, wl);
        cuda_check(cudaGetLastError(), "training weight conversion launch");
    }
} // namespace pmas
