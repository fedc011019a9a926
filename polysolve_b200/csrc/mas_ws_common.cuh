// Device definitions shared by the learned warm start's inference kernels (mas_warmstart.cu) and
// its training kernels (mas_ws_train.cu): the parameter layout, the per-vertex normalisation, the
// BF16 tensor-core fragment helpers and the message-passing layer (gather of the neighbours'
// hidden states + [h ; m] x W_l^T on mma.sync m16n8k16 with FP32 accumulation).
//
// Included by .cu files only; everything is in an anonymous namespace (one copy per file).
#pragma once

#include <cuda_bf16.h>

#include "mas_common.cuh"

namespace pmas
{
    namespace
    {
        constexpr int F = WS_FEATURES;
        constexpr int H = WS_HIDDEN;
        constexpr int WT = 256;         // threads of the per-vertex kernels
        constexpr int TILE = 128;       // vertices per CTA of a layer
        constexpr int LT = 256;         // threads of a layer CTA (8 warps x 16 vertices)
        constexpr int TS = 2 * H + 8;   // shared row stride (bf16): 272 B, conflict-free ldmatrix

        // Parameter offsets in the flat float32 vector (the .psws layout).
        constexpr int OFF_WIN = 0;
        constexpr int OFF_BIN = OFF_WIN + H * F;
        __host__ __device__ constexpr int off_layer(int l) { return OFF_BIN + H + l * (H * 2 * H + H); }
        constexpr int OFF_WOUT = off_layer(WS_LAYERS);
        constexpr int OFF_BOUT = OFF_WOUT + 3 * H;
        static_assert(OFF_BOUT + 3 == WS_PARAMS, "parameter layout");
        struct Norms
        {
            float iq, iv, ip, mlog; // 1 / rms (0 if the rms is 0) and the mean log trace
        };

        __device__ __forceinline__ Norms norms(const WsState *ws)
        {
            const double cnt = ws->sums[4];
            Norms n{0.f, 0.f, 0.f, 0.f};
            if (cnt > 0.0)
            {
                const double dofs = 3.0 * cnt;
                const double sq = sqrt(ws->sums[0] / dofs), sv = sqrt(ws->sums[1] / dofs),
                             sp = sqrt(ws->sums[2] / dofs);
                n.iq = sq > 0.0 ? (float)(1.0 / sq) : 0.f;
                n.iv = sv > 0.0 ? (float)(1.0 / sv) : 0.f;
                n.ip = sp > 0.0 ? (float)(1.0 / sp) : 0.f;
                n.mlog = (float)(ws->sums[3] / cnt);
            }
            return n;
        }

        __device__ __forceinline__ bool node_real(const int *rowlen, const int *diag_slot, int u)
        {
            return rowlen[u] > 0 && diag_slot[u] >= 0;
        }

        __device__ __forceinline__ void ldsm_x4(uint32_t (&a)[4], uint32_t addr)
        {
            asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                         : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                         : "r"(addr));
        }

        __device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
        {
            asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                         "{%8, %9}, {%0, %1, %2, %3};"
                         : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                         : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
        }

        // One message-passing layer for a tile of TILE vertices. Shared tile T[v] = [h_v ; m_v]
        // (bf16, K = 128), W_l as rows of K (the mma's column-major B), then each warp multiplies
        // its 16 vertices by W_l^T: 8 k-steps x 8 n-tiles of m16n8k16. SAVE (training): also
        // write m (bf16, as multiplied) and the pre-activation z = acc + b (FP32) of every vertex.
        template <bool SAVE>
        __global__ void __launch_bounds__(LT, 4) k_ws_layer(BankedView A, const float *__restrict__ wslot,
                                                         const __nv_bfloat16 *__restrict__ hin,
                                                         const uint16_t *__restrict__ wl, const float *__restrict__ bl,
                                                         const int *__restrict__ diag_slot,
                                                         __nv_bfloat16 *__restrict__ hout,
                                                         __nv_bfloat16 *__restrict__ m_out, float *__restrict__ z_out)
        {
            // Dynamic shared memory (52 KB: four CTAs, 32 warps per SM): the tile, W_l, the bias.
            extern __shared__ __align__(16) unsigned char layer_smem[];
            __nv_bfloat16 *T = reinterpret_cast<__nv_bfloat16 *>(layer_smem);
            __nv_bfloat16 *Wsm = T + TILE * TS;
            float *bias = reinterpret_cast<float *>(Wsm + H * TS);
            const int nodes = A.banks * 32;
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            // W_l: 64 rows x 128 bf16 = 16 chunks of 16 B per row.
            for (int i = threadIdx.x; i < H * 16; i += LT)
            {
                const int row = i >> 4, ch = i & 15;
                *reinterpret_cast<uint4 *>(&Wsm[row * TS + ch * 8]) =
                    __ldg(reinterpret_cast<const uint4 *>(wl + row * 2 * H) + ch);
            }
            if (threadIdx.x < H)
                bias[threadIdx.x] = bl[threadIdx.x];
            // Gather: warp w fills rows 16 w .. 16 w + 15, four at a time: lane group q = lane / 8
            // takes one row, lane gl = lane % 8 its hidden units 8 gl .. 8 gl + 7 (16-byte loads),
            // so four rows' neighbour loads are in flight together. Every lane runs the warp's
            // longest row; slots past a row's end carry w = 0 and the row's own (valid) index.
            const uint4 *h8 = reinterpret_cast<const uint4 *>(hin);
            const int gq = lane >> 3, gl = lane & 7;
            int my_len = 0;
            long long my_s0 = 0;
            {
                const int u = blockIdx.x * TILE + warp * 16 + (lane & 15);
                if (u < nodes && node_real(A.rowlen, diag_slot, u))
                {
                    my_len = A.rowlen[u];
                    my_s0 = A.slice[u >> 5];
                }
            }
            for (int rb = 0; rb < 16; rb += 4)
            {
                const int rl = rb + gq;
                const int r = warp * 16 + rl;
                const int u = blockIdx.x * TILE + r;
                const int len = __shfl_sync(FULL, my_len, rl);
                const long long s0 = __shfl_sync(FULL, my_s0, rl);
                int maxlen = len;
#pragma unroll
                for (int o = 8; o < 32; o <<= 1)
                    maxlen = max(maxlen, __shfl_xor_sync(FULL, maxlen, o));
                float acc[8];
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    acc[i] = 0.f;
                uint4 self = make_uint4(0u, 0u, 0u, 0u);
                if (len > 0)
                    self = h8[(long long)u * (H / 8) + gl];
                const int uu = (u < nodes) ? u : 0;
                for (int k0 = 0; k0 < maxlen; k0 += 8)
                {
                    const int kk = k0 + gl;
                    int col = uu;
                    float w = 0.f;
                    if (kk < len)
                    {
                        col = A.cols[(s0 + kk) * 32 + (u & 31)];
                        w = wslot[(s0 + kk) * 32 + (u & 31)];
                    }
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                    {
                        const int cj = __shfl_sync(FULL, col, j, 8);
                        const float wj = __shfl_sync(FULL, w, j, 8);
                        const uint4 hv = h8[(long long)cj * (H / 8) + gl];
                        const __nv_bfloat162 *hb = reinterpret_cast<const __nv_bfloat162 *>(&hv);
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                        {
                            const float2 f2 = __bfloat1622float2(hb[i]);
                            acc[2 * i] = fmaf(wj, f2.x, acc[2 * i]);
                            acc[2 * i + 1] = fmaf(wj, f2.y, acc[2 * i + 1]);
                        }
                    }
                }
                uint4 m8;
                __nv_bfloat162 *mb = reinterpret_cast<__nv_bfloat162 *>(&m8);
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    mb[i] = __float22bfloat162_rn(make_float2(acc[2 * i], acc[2 * i + 1]));
                *reinterpret_cast<uint4 *>(&T[r * TS + 8 * gl]) = self;
                *reinterpret_cast<uint4 *>(&T[r * TS + H + 8 * gl]) = m8;
                if (SAVE && u < nodes)
                    *reinterpret_cast<uint4 *>(m_out + (long long)u * H + 8 * gl) = m8;
            }
            __syncthreads();

            // Tensor-core product of the warp's 16 rows with W_l^T.
            float d[8][4];
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    d[nt][i] = 0.f;
            const uint32_t tbase = smem_addr(T), wbase = smem_addr(Wsm);
            const int arow = warp * 16 + (lane & 15), acol = (lane >> 4) * 8;
            const int brow = (lane & 7) + ((lane >> 4) << 3), bcol = ((lane >> 3) & 1) * 8;
#pragma unroll
            for (int ks = 0; ks < (2 * H) / 16; ++ks)
            {
                uint32_t a[4];
                ldsm_x4(a, tbase + (uint32_t)((arow * TS + ks * 16 + acol) * 2));
#pragma unroll
                for (int np = 0; np < 4; ++np)
                {
                    uint32_t bfr[4];
                    ldsm_x4(bfr, wbase + (uint32_t)(((np * 16 + brow) * TS + ks * 16 + bcol) * 2));
                    mma_bf16(d[2 * np], a, bfr[0], bfr[1]);
                    mma_bf16(d[2 * np + 1], a, bfr[2], bfr[3]);
                }
            }
            __syncwarp();
            // Epilogue: h_out = h + relu(acc + b), written over the warp's own rows of T.
            const int g = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int half = 0; half < 2; ++half)
                {
                    const int r = warp * 16 + g + half * 8;
                    const int col = nt * 8 + c2;
                    __nv_bfloat162 *tp = reinterpret_cast<__nv_bfloat162 *>(&T[r * TS + col]);
                    const float2 hs = __bfloat1622float2(*tp);
                    const float z0 = d[nt][2 * half] + bias[col], z1 = d[nt][2 * half + 1] + bias[col + 1];
                    const float v0 = hs.x + fmaxf(z0, 0.f);
                    const float v1 = hs.y + fmaxf(z1, 0.f);
                    *tp = __float22bfloat162_rn(make_float2(v0, v1));
                    if (SAVE)
                    {
                        const int u = blockIdx.x * TILE + r;
                        if (u < nodes)
                            *reinterpret_cast<float2 *>(z_out + (long long)u * H + col) = make_float2(z0, z1);
                    }
                }
            __syncwarp();
            __nv_bfloat162 *o2 = reinterpret_cast<__nv_bfloat162 *>(hout);
            for (int rr = 0; rr < 16; ++rr)
            {
                const int r = warp * 16 + rr;
                const int u = blockIdx.x * TILE + r;
                if (u >= nodes)
                    break;
                __nv_bfloat162 v = __float2bfloat162_rn(0.f);
                if (node_real(A.rowlen, diag_slot, u))
                    v = *reinterpret_cast<const __nv_bfloat162 *>(&T[r * TS + 2 * lane]);
                o2[(long long)u * (H / 2) + lane] = v;
            }
        }
    } // namespace
} // namespace pmas
