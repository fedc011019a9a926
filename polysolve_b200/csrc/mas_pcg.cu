// PCG vector kernels (sm_100a) and device-memory plumbing.
//
// The reference runs each vector step as its own launch (axpby / inner_product / scalar_division,
// MASSolver.cu:46-81, InnerProduct.cu:16-45) with a memset and an FP64 atomicAdd per dot. Here:
//   update_xr: x += alpha p ; r -= alpha Ap ; rr = r . r            (one pass; on true-residual
//              iterations only x, then r = b - A x follows in the SpMV)
//   update_p:  p = z0 + P zc + beta p             (the MAS prolongation fused in; beta from the
//                                                  device state, set by the MAS apply)
// alpha / beta are read from the device-resident PcgState, and every dot is a deterministic
// two-stage reduction, so no host round trip is needed inside the iteration.

#include <cstdio>
#include <string>

#include "mas_common.cuh"

namespace pmas
{
    void cuda_check(cudaError_t e, const char *what)
    {
        if (e != cudaSuccess)
            throw Error(ERR_CUDA, std::string("[MAS] CUDA error in ") + what + ": " + cudaGetErrorString(e));
    }

    // Allocation with the reference's out-of-memory message (mas_utils/CudaUtils.cuh:68-79).
    void *device_alloc(size_t bytes, const char *ctx)
    {
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
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

    namespace
    {
        constexpr int UPD_THREADS = 256;

        // x += alpha p ; r -= alpha Ap ; per-CTA r . r (summed by the finalize kernel). Grid-stride
        // over the vectors with coalesced accesses. On a true-residual iteration only x is updated.
        __global__ void __launch_bounds__(UPD_THREADS) k_update_xr(long long len, double *__restrict__ x,
                                                                   double *__restrict__ r, const double *__restrict__ p,
                                                                   const double *__restrict__ Ap, PcgState *st,
                                                                   ReduceBuf red, int period)
        {
            if (st->done)
                return;
            const double alpha = st->alpha;
            const bool due = period > 0 && (st->iter + 1) % period == 0;
            const long long stride = (long long)gridDim.x * UPD_THREADS;
            double part = 0.0;
            if (due)
            {
                for (long long i = blockIdx.x * (long long)UPD_THREADS + threadIdx.x; i < len; i += stride)
                    x[i] = fma(alpha, p[i], x[i]);
                return;
            }
            for (long long i = blockIdx.x * (long long)UPD_THREADS + threadIdx.x; i < len; i += stride)
            {
                x[i] = fma(alpha, p[i], x[i]);
                const double rv = fma(-alpha, Ap[i], r[i]);
                r[i] = rv;
                part = fma(rv, rv, part);
            }
            const double rr = block_sum<UPD_THREADS>(part);
            if (threadIdx.x == 0)
            {
                red.rr_parts[blockIdx.x] = rr;
                if (blockIdx.x == 0)
                    st->n_rr = gridDim.x;
            }
        }

        // p = z0 + sum_l zc[cslot_l(node)] + beta p; warps stride over banks, coalesced.
        template <int BD>
        __global__ void __launch_bounds__(UPD_THREADS) k_update_p(MasView mas, double *__restrict__ p,
                                                                  const double *__restrict__ z0, const PcgState *st,
                                                                  int first)
        {
            if (st->done)
                return;
            const double beta = first ? 0.0 : st->beta;
            const int lane = threadIdx.x & 31;
            const int total_warps = gridDim.x * (UPD_THREADS / 32);
            const double *__restrict__ zc = mas.zc;
            const double iso_scale = 1.0 + mas.level_num;
            for (int bank = blockIdx.x * (UPD_THREADS / 32) + (threadIdx.x >> 5); bank < mas.banks; bank += total_warps)
            {
                const long long b0 = (long long)bank * 32 * BD;
                if (bank >= mas.first_iso_bank)
                {
                    // Isolated rows: every coarse level adds z0 again (coarse block A_uu).
#pragma unroll
                    for (int t = 0; t < BD; ++t)
                    {
                        const long long idx = b0 + t * 32 + lane;
                        const double v = iso_scale * z0[idx];
                        p[idx] = first ? v : fma(beta, p[idx], v);
                    }
                    continue;
                }
#pragma unroll
                for (int t = 0; t < BD; ++t)
                {
                    const int e = t * 32 + lane;
                    const int node = e / BD, comp = e - node * BD;
                    const int4 cs = mas.cslot[(long long)bank * 32 + node];
                    const long long idx = b0 + e;
                    double v = z0[idx];
                    if (cs.x >= 0)
                        v += zc[(size_t)cs.x * BD + comp];
                    if (cs.y >= 0)
                        v += zc[(size_t)cs.y * BD + comp];
                    if (cs.z >= 0)
                        v += zc[(size_t)cs.z * BD + comp];
                    if (cs.w >= 0)
                        v += zc[(size_t)cs.w * BD + comp];
                    p[idx] = first ? v : fma(beta, p[idx], v);
                }
            }
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
        int bank_grid(int banks)
        {
            const int need = (banks + UPD_THREADS / 32 - 1) / (UPD_THREADS / 32);
            const int cap = device_sm_count() * 8;
            return need < cap ? need : cap;
        }
    } // namespace

    void launch_update_xr(int banks, int bd, double *x, double *r, const double *p, const double *Ap, PcgState *st,
                          ReduceBuf red, int period, cudaStream_t s)
    {
        const long long len = (long long)banks * 32 * bd;
        long long g = (len + UPD_THREADS - 1) / UPD_THREADS;
        const long long cap = (long long)device_sm_count() * 8;
        if (g > cap)
            g = cap;
        if (g < 1)
            g = 1;
        if (g > red.capacity)
            throw Error(ERR_INVALID, "[MAS] reduction scratch too small");
        k_update_xr<<<(int)g, UPD_THREADS, 0, s>>>(len, x, r, p, Ap, st, red, period);
        cuda_check(cudaGetLastError(), "update_xr launch");
    }

    void launch_update_p(const MasView &mas, double *p, const double *z0, PcgState *st, int first, cudaStream_t s)
    {
        const int grid = bank_grid(mas.banks);
        if (grid == 0)
            return;
        switch (mas.bd)
        {
        case 1:
            k_update_p<1><<<grid, UPD_THREADS, 0, s>>>(mas, p, z0, st, first);
            break;
        case 2:
            k_update_p<2><<<grid, UPD_THREADS, 0, s>>>(mas, p, z0, st, first);
            break;
        default:
            k_update_p<3><<<grid, UPD_THREADS, 0, s>>>(mas, p, z0, st, first);
            break;
        }
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
