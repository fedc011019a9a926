// Learned starting guess for a sequence of systems with one pattern (sm_100a).
//
// The reference starts every PCG solve from x0 = 0 (MASSolver.cu:395-398) while its caller
// (nonlinear::Newton, Newton.cpp:173-214) solves a matrix of the same pattern with new values at
// every step. Here the solver keeps the last four solutions x1 (newest) .. x4 on the device and
// predicts x0:
//
//   k_ws_graph      once per factorization: each stored block's neighbour weight
//                   ||A_ij||_F / sum_{j' != i} ||A_ij'||_F and the slot of the diagonal block.
//   (SpMV x4)       y_i = A x_i for the kept solutions (the plain SpMV kernel).
//   k_ws_gram       (first pass, without c) the Galerkin combination x_g of the kept solutions;
//   k_ws_residual   r_g = b - A x_g from the products already at hand (no SpMV).
//   k_ws_features   per vertex: q = D^-1 r_g, v = x1 - x2, p = D^-1 b, the diagonal block scaled
//                   by trace / 3, log trace; the sums the normalisation needs (deterministic
//                   grid reduction).
//   k_ws_input      h = relu(W_in f + b_in) with the normalised features (FP32, BF16 out).
//   k_ws_layer x3   m = sum_j w_ij h_j (gathered from L2 into shared memory), then
//                   h += relu(W_l [h ; m] + b_l) on the tensor cores: BF16 mma.sync m16n8k16
//                   with FP32 accumulation, 64 vertices x 64 outputs x K = 128 per CTA.
//   k_ws_output     c = s_q (W_out h + b_out) (FP32 weights, FP64 out).
//   (SpMV)          y3 = A c.
//   k_ws_gram       (second pass) the 5 x 5 Galerkin system of the basis {x1, x1 - x2, x2 - x3, x3 - x4, c}
//                   and its right-hand side (20 dots, deterministic); the last CTA solves it
//                   with a pivoted Cholesky that drops dependent (or missing) vectors and falls
//                   back to x1 unless the energy 1/2 x.Ax - x.b drops below that of x1. The
//                   differences of past solutions carry their trend in k: the combination is a
//                   polynomial extrapolation in the step index, fitted in the energy norm;
//   k_ws_combine    x0 = sum_i coef_i v_i.
//
// All vectors are in the solver's padded (subdomain) order; nodes without a row (padding) get
// zero features, zero hidden states and c = 0. The work is small next to a solve: at 680 K DOF
// the three layers move about 30 MB of hidden states each (the gathers hit L2) and do
// 3 x 2 x 227 K x 64 x 128 = 11 GFLOP on the tensor pipe.

#include "mas_ws_common.cuh"

namespace pmas
{
    namespace
    {
        __device__ __forceinline__ double block_entry(const BankedView &A, long long slot, int lane, int q)
        {
            return A.vals[banked_value_index(slot, lane, q, 3)];
        }

        __device__ __forceinline__ double block_fro(const BankedView &A, long long slot, int lane)
        {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < 9; ++q)
            {
                const double v = block_entry(A, slot, lane, q);
                s = fma(v, v, s);
            }
            return sqrt(s);
        }

        // One thread per node (lanes of a warp = the 32 nodes of a bank: coalesced slot reads).
        __global__ void __launch_bounds__(WT) k_ws_graph(BankedView A, int *__restrict__ diag_slot,
                                                         float *__restrict__ wslot)
        {
            const int u = blockIdx.x * WT + threadIdx.x;
            if (u >= A.banks * 32)
                return;
            const int bank = u >> 5, lane = u & 31;
            const long long s0 = A.slice[bank];
            const int len = A.rowlen[u];
            // One pass over the row's blocks (norms kept in wslot), then the normalisation.
            double tot = 0.0;
            int dslot = -1;
            for (int k = 0; k < len; ++k)
            {
                const int col = A.cols[(s0 + k) * 32 + lane];
                float nrm = 0.f;
                if (col == u)
                    dslot = k;
                else
                {
                    const double f = block_fro(A, s0 + k, lane);
                    tot += f;
                    nrm = (float)f;
                }
                wslot[(s0 + k) * 32 + lane] = nrm;
            }
            const float inv = (tot > 0.0) ? (float)(1.0 / tot) : 0.f;
            for (int k = 0; k < len; ++k)
                wslot[(s0 + k) * 32 + lane] *= inv;
            diag_slot[u] = dslot;
        }

        // 3 x 3 inverse by cofactors; false if singular or not finite.
        __device__ __forceinline__ bool inv3(const double (&d)[9], double (&o)[9])
        {
            const double c00 = d[4] * d[8] - d[5] * d[7];
            const double c01 = d[5] * d[6] - d[3] * d[8];
            const double c02 = d[3] * d[7] - d[4] * d[6];
            const double det = d[0] * c00 + d[1] * c01 + d[2] * c02;
            if (!(fabs(det) > 0.0) || !isfinite(det))
                return false;
            const double r = 1.0 / det;
            o[0] = c00 * r;
            o[1] = (d[2] * d[7] - d[1] * d[8]) * r;
            o[2] = (d[1] * d[5] - d[2] * d[4]) * r;
            o[3] = c01 * r;
            o[4] = (d[0] * d[8] - d[2] * d[6]) * r;
            o[5] = (d[2] * d[3] - d[0] * d[5]) * r;
            o[6] = c02 * r;
            o[7] = (d[1] * d[6] - d[0] * d[7]) * r;
            o[8] = (d[0] * d[4] - d[1] * d[3]) * r;
            return true;
        }

        __global__ void __launch_bounds__(WT)
            k_ws_features(BankedView A, const int *__restrict__ diag_slot, const double *__restrict__ b,
                          const double *__restrict__ rg, const double *__restrict__ x1,
                          const double *__restrict__ x2, float *__restrict__ feat, WsState *ws, double *partials)
        {
            const int u = blockIdx.x * WT + threadIdx.x;
            double sums[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            if (u < A.banks * 32)
            {
                float f[F];
#pragma unroll
                for (int i = 0; i < F; ++i)
                    f[i] = 0.f;
                const int dslot = diag_slot[u];
                if (A.rowlen[u] > 0 && dslot >= 0)
                {
                    const int bank = u >> 5, lane = u & 31;
                    const long long slot = A.slice[bank] + dslot;
                    double d[9], di[9];
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        d[q] = block_entry(A, slot, lane, q);
                    const double tr = d[0] + d[4] + d[8];
                    if (tr > 0.0 && isfinite(tr) && inv3(d, di))
                    {
                        double re[3], bv[3], v[3];
#pragma unroll
                        for (int i = 0; i < 3; ++i)
                        {
                            const long long k = (long long)u * 3 + i;
                            bv[i] = b[k];
                            re[i] = rg[k];
                            v[i] = x1[k] - x2[k];
                        }
#pragma unroll
                        for (int i = 0; i < 3; ++i)
                        {
                            const double q = di[3 * i] * re[0] + di[3 * i + 1] * re[1] + di[3 * i + 2] * re[2];
                            const double p = di[3 * i] * bv[0] + di[3 * i + 1] * bv[1] + di[3 * i + 2] * bv[2];
                            f[i] = (float)q;
                            f[3 + i] = (float)v[i];
                            f[6 + i] = (float)p;
                            sums[0] = fma(q, q, sums[0]);
                            sums[1] = fma(v[i], v[i], sums[1]);
                            sums[2] = fma(p, p, sums[2]);
                        }
                        const double t = tr / 3.0;
                        f[9] = (float)(d[0] / t);
                        f[10] = (float)(d[4] / t);
                        f[11] = (float)(d[8] / t);
                        f[12] = (float)(d[1] / t);
                        f[13] = (float)(d[2] / t);
                        f[14] = (float)(d[5] / t);
                        const double lt = log(tr);
                        f[15] = (float)lt;
                        sums[3] = lt;
                        sums[4] = 1.0;
                    }
                }
                float4 *dst = reinterpret_cast<float4 *>(feat + (long long)u * F);
#pragma unroll
                for (int i = 0; i < F / 4; ++i)
                    dst[i] = make_float4(f[4 * i], f[4 * i + 1], f[4 * i + 2], f[4 * i + 3]);
            }
            double tot[5];
            if (grid_reduce<5, WT>(sums, partials, &ws->counter[0], tot) && threadIdx.x == 0)
                for (int i = 0; i < 5; ++i)
                    ws->sums[i] = tot[i];
        }

        // One thread per vertex: its 16 normalised features against W_in (shared memory, every
        // lane reading the same weight: broadcast), 64 hidden units written as eight 16-byte
        // stores.
        __global__ void __launch_bounds__(WT) k_ws_input(int nodes, const int *__restrict__ rowlen,
                                                         const int *__restrict__ diag_slot,
                                                         const float *__restrict__ feat, const float *__restrict__ prm,
                                                         const WsState *ws, __nv_bfloat162 *__restrict__ h)
        {
            __shared__ __align__(16) float wsm[H * F + H];
            for (int i = threadIdx.x; i < H * F + H; i += WT)
                wsm[i] = prm[OFF_WIN + i];
            __syncthreads();
            const int u = blockIdx.x * WT + threadIdx.x;
            if (u >= nodes)
                return;
            uint4 *dst = reinterpret_cast<uint4 *>(h + (long long)u * (H / 2));
            if (!node_real(rowlen, diag_slot, u))
            {
#pragma unroll
                for (int i = 0; i < H / 8; ++i)
                    dst[i] = make_uint4(0u, 0u, 0u, 0u);
                return;
            }
            const Norms nm = norms(ws);
            const float4 *fp = reinterpret_cast<const float4 *>(feat + (long long)u * F);
            float f[F];
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
            for (int i = 0; i < 3; ++i)
            {
                f[i] *= nm.iq;
                f[3 + i] *= nm.iv;
                f[6 + i] *= nm.ip;
            }
            f[15] -= nm.mlog;
#pragma unroll
            for (int c = 0; c < H / 8; ++c)
            {
                uint4 out;
                __nv_bfloat162 *ob = reinterpret_cast<__nv_bfloat162 *>(&out);
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
                }
                dst[c] = out;
            }
        }

        // c = s_q (W_out h + b_out): one thread per vertex (eight 16-byte loads of its hidden row,
        // W_out broadcast from shared memory).
        __global__ void __launch_bounds__(WT) k_ws_output(int nodes, const int *__restrict__ rowlen,
                                                          const int *__restrict__ diag_slot,
                                                          const __nv_bfloat162 *__restrict__ h,
                                                          const float *__restrict__ prm, const WsState *ws,
                                                          double *__restrict__ c)
        {
            __shared__ float wo[3 * H + 3];
            for (int i = threadIdx.x; i < 3 * H + 3; i += WT)
                wo[i] = prm[OFF_WOUT + i];
            __syncthreads();
            const int u = blockIdx.x * WT + threadIdx.x;
            if (u >= nodes)
                return;
            if (!node_real(rowlen, diag_slot, u))
            {
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    c[(long long)u * 3 + i] = 0.0;
                return;
            }
            const double cnt = ws->sums[4];
            const double sq = cnt > 0.0 ? sqrt(ws->sums[0] / (3.0 * cnt)) : 0.0;
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

        constexpr int GRAM_CTAS_PER_SM = 4;
        constexpr int NB = WS_BASIS;

        // Basis vector i and its product with A at element k.
        __device__ __forceinline__ void basis_at(const WsHistory &h, const double *__restrict__ c,
                                                 const double *__restrict__ yc, size_t k, double (&v)[NB],
                                                 double (&av)[NB])
        {
            v[0] = h.x[0][k];
            av[0] = h.y[0][k];
#pragma unroll
            for (int i = 1; i < WS_HISTORY; ++i)
            {
                v[i] = h.x[i - 1][k] - h.x[i][k];
                av[i] = h.y[i - 1][k] - h.y[i][k];
            }
            v[NB - 1] = c ? c[k] : 0.0; // first pass: no c yet
            av[NB - 1] = c ? yc[k] : 0.0;
        }

        // The Galerkin system of the basis; the last CTA solves it.
        __global__ void __launch_bounds__(WT)
            k_ws_gram(const double *__restrict__ b, WsHistory h, const double *__restrict__ c,
                      const double *__restrict__ yc, size_t len, WsState *ws, double *partials)
        {
            double s[WS_GRAM];
#pragma unroll
            for (int i = 0; i < WS_GRAM; ++i)
                s[i] = 0.0;
            for (size_t k = (size_t)blockIdx.x * WT + threadIdx.x; k < len; k += (size_t)gridDim.x * WT)
            {
                double v[NB], av[NB];
                basis_at(h, c, yc, k, v, av);
                const double bk = b[k];
                int e = 0;
#pragma unroll
                for (int i = 0; i < NB; ++i)
#pragma unroll
                    for (int j = i; j < NB; ++j)
                    {
                        s[e] = fma(v[i], av[j], s[e]);
                        ++e;
                    }
#pragma unroll
                for (int i = 0; i < NB; ++i)
                    s[e + i] = fma(v[i], bk, s[e + i]);
            }
            double t[WS_GRAM];
            if (!grid_reduce<WS_GRAM, WT>(s, partials, &ws->counter[1], t) || threadIdx.x != 0)
                return;
            for (int i = 0; i < WS_GRAM; ++i)
                ws->gram[i] = t[i];
            double G[NB][NB], g[NB];
            {
                int e = 0;
                for (int i = 0; i < NB; ++i)
                    for (int j = i; j < NB; ++j)
                    {
                        G[i][j] = t[e];
                        G[j][i] = t[e];
                        ++e;
                    }
                for (int i = 0; i < NB; ++i)
                    g[i] = t[e + i];
            }
            // Cholesky of the kept vectors, in order; a vector whose pivot is below 1e-10 of its
            // diagonal (dependent on the kept ones) or not positive is dropped.
            double L[NB][NB];
            bool keep[NB];
            int rank = 0;
            for (int i = 0; i < NB; ++i)
            {
                keep[i] = false;
                for (int j = 0; j < NB; ++j)
                    L[i][j] = 0.0;
            }
            for (int i = 0; i < NB; ++i)
            {
                if (!(G[i][i] > 0.0) || !isfinite(G[i][i]))
                    continue;
                double dsum = G[i][i];
                for (int j = 0; j < i; ++j)
                {
                    if (!keep[j])
                        continue;
                    double v = G[i][j];
                    for (int k = 0; k < j; ++k)
                        if (keep[k])
                            v -= L[i][k] * L[j][k];
                    L[i][j] = v / L[j][j];
                    dsum -= L[i][j] * L[i][j];
                }
                if (dsum > 1e-10 * G[i][i] && isfinite(dsum))
                {
                    L[i][i] = sqrt(dsum);
                    keep[i] = true;
                    ++rank;
                }
                else
                    for (int j = 0; j < i; ++j)
                        L[i][j] = 0.0;
            }
            double y[NB], z[NB];
            for (int i = 0; i < NB; ++i)
                y[i] = z[i] = 0.0;
            for (int i = 0; i < NB; ++i) // L z = g
                if (keep[i])
                {
                    double v = g[i];
                    for (int j = 0; j < i; ++j)
                        if (keep[j])
                            v -= L[i][j] * z[j];
                    z[i] = v / L[i][i];
                }
            for (int i = NB - 1; i >= 0; --i) // L^T y = z
                if (keep[i])
                {
                    double v = z[i];
                    for (int j = i + 1; j < NB; ++j)
                        if (keep[j])
                            v -= L[j][i] * y[j];
                    y[i] = v / L[i][i];
                }
            double e = 0.0; // 1/2 y.Gy - y.g
            bool finite = true;
            for (int i = 0; i < NB; ++i)
            {
                double gy = 0.0;
                for (int j = 0; j < NB; ++j)
                    gy += G[i][j] * y[j];
                e += y[i] * (0.5 * gy - g[i]);
                finite = finite && isfinite(y[i]);
            }
            const double e1 = 0.5 * G[0][0] - g[0];
            const bool ok = rank > 0 && finite && isfinite(e) && e < e1;
            ws->fallback = ok ? 0 : 1;
            ws->rank = rank;
            for (int i = 0; i < NB; ++i)
                ws->coef[i] = ok ? y[i] : (i == 0 ? 1.0 : 0.0);
            ws->energy = ok ? e : e1;
            ws->energy_prev = e1;
        }

        __global__ void __launch_bounds__(WT) k_ws_combine(WsHistory h, const double *__restrict__ c,
                                                           const WsState *ws, double *__restrict__ x, size_t len)
        {
            double cf[NB];
#pragma unroll
            for (int i = 0; i < NB; ++i)
                cf[i] = ws->coef[i];
            for (size_t k = (size_t)blockIdx.x * WT + threadIdx.x; k < len; k += (size_t)gridDim.x * WT)
            {
                double v = cf[0] * h.x[0][k];
#pragma unroll
                for (int i = 1; i < WS_HISTORY; ++i)
                    v += cf[i] * (h.x[i - 1][k] - h.x[i][k]);
                x[k] = v + cf[NB - 1] * c[k];
            }
        }

        // r_g = b - A x_g with x_g the first pass's combination (A x_g from the y_i); also keeps
        // the first pass's coefficients.
        __global__ void __launch_bounds__(WT) k_ws_residual(const double *__restrict__ b, WsHistory h,
                                                            WsState *ws, double *__restrict__ rg, size_t len)
        {
            double cf[NB];
#pragma unroll
            for (int i = 0; i < NB; ++i)
                cf[i] = ws->coef[i];
            for (size_t k = (size_t)blockIdx.x * WT + threadIdx.x; k < len; k += (size_t)gridDim.x * WT)
            {
                double ax = cf[0] * h.y[0][k];
#pragma unroll
                for (int i = 1; i < WS_HISTORY; ++i)
                    ax += cf[i] * (h.y[i - 1][k] - h.y[i][k]);
                rg[k] = b[k] - ax;
            }
            if (blockIdx.x == 0 && threadIdx.x < NB)
                ws->coef_hist[threadIdx.x] = cf[threadIdx.x];
        }

        __global__ void k_ws_features_out(int V, const int *__restrict__ padded, const float *__restrict__ feat,
                                          float *__restrict__ out)
        {
            const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            if (i >= (long long)V * F)
                return;
            const int v = (int)(i / F), f = (int)(i % F);
            out[i] = feat[(long long)padded[v] * F + f];
        }
    } // namespace

    int ws_reduce_ctas() { return device_sm_count() * GRAM_CTAS_PER_SM; }

    void launch_ws_graph(const BankedView &A, const WsBuffers &w, cudaStream_t s)
    {
        if (A.bd != 3)
            throw Error(ERR_INVALID, "[MAS] the learned warm start needs block_dim 3");
        const int nodes = A.banks * 32;
        if (nodes == 0)
            return;
        k_ws_graph<<<(nodes + WT - 1) / WT, WT, 0, s>>>(A, w.diag_slot, w.wslot);
        cuda_check(cudaGetLastError(), "warm start graph launch");
    }

    int launch_ws_features(const BankedView &A, const WsBuffers &w, const double *b, const WsHistory &hist,
                           size_t len, cudaStream_t s)
    {
        const int nodes = A.banks * 32;
        if (nodes == 0)
            return 0;
        const int grid_v = (nodes + WT - 1) / WT;
        const int grid_r = ws_reduce_ctas();
        if (grid_v > w.capacity || grid_r > w.capacity)
            throw Error(ERR_INVALID, "[MAS] warm start reduction scratch too small");
        k_ws_gram<<<grid_r, WT, 0, s>>>(b, hist, nullptr, nullptr, len, w.st, w.partials);
        cuda_check(cudaGetLastError(), "warm start gram launch");
        k_ws_residual<<<grid_r, WT, 0, s>>>(b, hist, w.st, w.rg, len);
        cuda_check(cudaGetLastError(), "warm start residual launch");
        k_ws_features<<<grid_v, WT, 0, s>>>(A, w.diag_slot, b, w.rg, hist.x[0], hist.x[1], w.feat, w.st, w.partials);
        cuda_check(cudaGetLastError(), "warm start features launch");
        return 3;
    }

    int launch_ws_network(const BankedView &A, const WsBuffers &w, const double *b, const WsHistory &hist,
                          size_t len, cudaStream_t s)
    {
        const double *x1 = hist.x[0], *x2 = hist.x[1];
        const int nodes = A.banks * 32;
        if (nodes == 0)
            return 0;
        const int grid_v = (nodes + WT - 1) / WT;
        const int grid_r = ws_reduce_ctas();
        if (grid_v > w.capacity || grid_r > w.capacity)
            throw Error(ERR_INVALID, "[MAS] warm start reduction scratch too small");
        // First pass: x_g over the kept solutions alone, and its residual.
        k_ws_gram<<<grid_r, WT, 0, s>>>(b, hist, nullptr, nullptr, len, w.st, w.partials);
        cuda_check(cudaGetLastError(), "warm start gram launch");
        k_ws_residual<<<grid_r, WT, 0, s>>>(b, hist, w.st, w.rg, len);
        cuda_check(cudaGetLastError(), "warm start residual launch");
        k_ws_features<<<grid_v, WT, 0, s>>>(A, w.diag_slot, b, w.rg, x1, x2, w.feat, w.st, w.partials);
        cuda_check(cudaGetLastError(), "warm start features launch");
        k_ws_input<<<(nodes + WT - 1) / WT, WT, 0, s>>>(nodes, A.rowlen, w.diag_slot, w.feat, w.params, w.st,
                                                        reinterpret_cast<__nv_bfloat162 *>(w.h[0]));
        cuda_check(cudaGetLastError(), "warm start input launch");
        const int grid_t = (nodes + TILE - 1) / TILE;
        constexpr int LAYER_SMEM = (TILE + H) * TS * 2 + H * 4;
        static_assert((TILE * TS * 2) % 16 == 0 && ((TILE + H) * TS * 2) % 16 == 0, "shared layout");
        cuda_check(cudaFuncSetAttribute(k_ws_layer<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, LAYER_SMEM),
                   "layer smem attribute");
        for (int l = 0; l < WS_LAYERS; ++l)
        {
            k_ws_layer<false><<<grid_t, LT, LAYER_SMEM, s>>>(
                A, w.wslot, reinterpret_cast<const __nv_bfloat16 *>(w.h[l & 1]), w.wl + (size_t)l * WS_LAYER_WEIGHTS,
                w.params + off_layer(l) + H * 2 * H, w.diag_slot, reinterpret_cast<__nv_bfloat16 *>(w.h[(l + 1) & 1]),
                nullptr, nullptr);
            cuda_check(cudaGetLastError(), "warm start layer launch");
        }
        k_ws_output<<<(nodes + WT - 1) / WT, WT, 0, s>>>(nodes, A.rowlen, w.diag_slot,
                                          reinterpret_cast<const __nv_bfloat162 *>(w.h[WS_LAYERS & 1]), w.params, w.st,
                                          w.c);
        cuda_check(cudaGetLastError(), "warm start output launch");
        return 5 + WS_LAYERS;
    }

    int launch_ws_combine(const WsBuffers &w, const double *b, const WsHistory &hist, double *x, size_t len,
                          cudaStream_t s)
    {
        const int grid = ws_reduce_ctas();
        if (grid > w.capacity)
            throw Error(ERR_INVALID, "[MAS] warm start reduction scratch too small");
        k_ws_gram<<<grid, WT, 0, s>>>(b, hist, w.c, w.yc, len, w.st, w.partials);
        cuda_check(cudaGetLastError(), "warm start gram launch");
        k_ws_combine<<<grid, WT, 0, s>>>(hist, w.c, w.st, x, len);
        cuda_check(cudaGetLastError(), "warm start combine launch");
        return 2;
    }

    void launch_ws_features_out(int V, const int *padded_of_block, const float *feat, float *out, cudaStream_t s)
    {
        const long long total = (long long)V * F;
        if (total == 0)
            return;
        k_ws_features_out<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(V, padded_of_block, feat, out);
        cuda_check(cudaGetLastError(), "warm start features out launch");
    }
} // namespace pmas
