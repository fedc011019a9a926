// CSC -> permuted bank-sliced block matrix, on the device (sm_100a).
//
// Reference: BSRMatrix.cu:195-430 builds a permuted row-major BSR (64-bit key radix sort, RLE,
// histogram, scans) and pads the trailing block's missing diagonal with 1.0 (:123-134, :189-190).
// The same steps are needed here (sort entries by (block row, block col), find unique blocks,
// count per row), but the output is the bank-sliced layout the SpMV streams, block rows are
// already in the padded subdomain order, and the position of every CSC entry is kept
// (`scatter`) so a refactorization with an unchanged pattern is a single scatter kernel.

#include <cub/cub.cuh>

#include "mas_common.cuh"

namespace pmas
{
    namespace
    {
        constexpr unsigned PAD_MARK = 0xFFFFFFFFu;

        // One warp per CSC column: key = (row node << 32) | col node; payload = (offset << 32) | k.
        __global__ void k_keys(int n, const int *__restrict__ outer, const int *__restrict__ inner, int bd, int V,
                               int npad, const int *__restrict__ padded, unsigned long long *keys,
                               unsigned long long *payloads, int *bad)
        {
            const int lane = threadIdx.x & 31;
            const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
            const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
            for (long long j = warp; j < n; j += nwarps)
            {
                const int b = outer[j], e = outer[j + 1];
                const int bco = (int)(j / bd);
                const unsigned w = (unsigned)padded[bco];
                const int cj = (int)(j - (long long)bco * bd);
                for (int k = b + lane; k < e; k += 32)
                {
                    const int i = inner[k];
                    if (i < 0 || i >= n)
                    {
                        atomicExch(bad, 1);
                        keys[k] = 0ull;
                        payloads[k] = ((unsigned long long)0 << 32) | (unsigned)k;
                        continue;
                    }
                    const int bro = i / bd;
                    const unsigned u = (unsigned)padded[bro];
                    const int off = (i - bro * bd) * bd + cj;
                    keys[k] = ((unsigned long long)u << 32) | w;
                    payloads[k] = ((unsigned long long)off << 32) | (unsigned)k;
                }
            }
            // Trailing padding entries.
            const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
            if (tid < npad)
            {
                const unsigned tail = (unsigned)padded[V - 1];
                const int local = (bd - npad) + (int)tid;
                const int off = local * bd + local;
                const long long at = (long long)outer[n] + tid;
                keys[at] = ((unsigned long long)tail << 32) | tail;
                payloads[at] = ((unsigned long long)off << 32) | PAD_MARK;
            }
        }

        __global__ void k_heads(long long E, const unsigned long long *__restrict__ keys, int *head)
        {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < E;
                 i += (long long)gridDim.x * blockDim.x)
                head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
        }

        __global__ void k_rowlen(long long E, const unsigned long long *__restrict__ keys, const int *__restrict__ head,
                                 int *rowlen)
        {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < E;
                 i += (long long)gridDim.x * blockDim.x)
                if (head[i])
                    atomicAdd(&rowlen[keys[i] >> 32], 1);
        }

        __global__ void k_width(int banks, const int *__restrict__ rowlen, long long *width)
        {
            const int lane = threadIdx.x & 31;
            const int bank = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            if (bank >= banks)
                return;
            int v = rowlen[bank * 32 + lane];
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1)
                v = max(v, __shfl_xor_sync(FULL, v, o));
            if (lane == 0)
                width[bank] = v;
        }

        __global__ void k_fill(long long E, int bd, const unsigned long long *__restrict__ keys,
                               const unsigned long long *__restrict__ payloads, const int *__restrict__ bid_incl,
                               const int *__restrict__ row_start, const long long *__restrict__ slice,
                               const double *__restrict__ csc_vals, int *cols, double *vals, long long *scatter,
                               long long *pad_pos)
        {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < E;
                 i += (long long)gridDim.x * blockDim.x)
            {
                const unsigned long long key = keys[i];
                const int u = (int)(key >> 32);
                const int w = (int)(key & 0xFFFFFFFFull);
                const int bidx = bid_incl[i] - 1;
                const int rank = bidx - row_start[u];
                const long long slot = slice[u >> 5] + rank;
                const int lane = u & 31;
                const bool head = (i == 0) || (keys[i - 1] != key);
                if (head)
                    cols[slot * 32 + lane] = w;
                const unsigned long long pl = payloads[i];
                const int off = (int)(pl >> 32);
                const unsigned k = (unsigned)(pl & 0xFFFFFFFFull);
                const long long pos = banked_value_index(slot, lane, off, bd);
                if (k == PAD_MARK)
                {
                    vals[pos] = 1.0;
                    pad_pos[off / (bd + 1)] = pos;
                }
                else
                {
                    vals[pos] = csc_vals[k];
                    scatter[k] = pos;
                }
            }
        }

        __global__ void k_rescatter(long long nnz, const long long *__restrict__ scatter,
                                    const double *__restrict__ csc_vals, double *vals)
        {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nnz;
                 i += (long long)gridDim.x * blockDim.x)
                vals[scatter[i]] = csc_vals[i];
        }

        int grid_for(long long n, int threads = 256)
        {
            long long g = (n + threads - 1) / threads;
            if (g > 148LL * 32)
                g = 148LL * 32;
            return (int)(g < 1 ? 1 : g);
        }

        int bits_for(long long v)
        {
            int b = 1;
            while (b < 31 && (1LL << b) <= v)
                ++b;
            return b;
        }
    } // namespace

    void build_banked(BankedMatrix &M, int n, long long nnz, const int *d_outer, const int *d_inner,
                      const double *d_vals, int bd, int V, int banks, const int *d_padded_of_block, cudaStream_t s)
    {
        const int npad = bd * V - n;
        const long long E = nnz + npad;
        const int nodes = banks * 32;
        M.bd = bd;
        M.banks = banks;
        M.nodes = nodes;

        DevBuf<unsigned long long> keys, keys_alt, pay, pay_alt;
        keys.alloc(E, "MAS banked_matrix staging");
        keys_alt.alloc(E, "MAS banked_matrix staging");
        pay.alloc(E, "MAS banked_matrix staging");
        pay_alt.alloc(E, "MAS banked_matrix staging");
        DevBuf<int> bad;
        bad.alloc(1, "MAS banked_matrix flag");
        cuda_check(cudaMemsetAsync(bad.get(), 0, sizeof(int), s), "memset");

        {
            long long threads_needed = (long long)n * 32;
            if (threads_needed < npad)
                threads_needed = npad;
            int grid = grid_for(threads_needed);
            k_keys<<<grid, 256, 0, s>>>(n, d_outer, d_inner, bd, V, npad, d_padded_of_block, keys.get(),
                                        pay.get(), bad.get());
            cuda_check(cudaGetLastError(), "keys launch");
        }
        int h_bad = 0;
        cuda_check(cudaMemcpyAsync(&h_bad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s), "copy flag");
        cuda_check(cudaStreamSynchronize(s), "keys");
        if (h_bad)
            throw Error(ERR_INVALID, "[MAS] Invalid CSC: row index out of range.");

        cub::DoubleBuffer<unsigned long long> dk(keys.get(), keys_alt.get());
        cub::DoubleBuffer<unsigned long long> dp(pay.get(), pay_alt.get());
        const int end_bit = 32 + bits_for(nodes);
        size_t tmp_bytes = 0;
        cuda_check(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, dk, dp, E, 0, end_bit, s), "sort size");
        DevBuf<unsigned char> tmp;
        tmp.alloc(tmp_bytes, "MAS banked_matrix sort");
        cuda_check(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, dk, dp, E, 0, end_bit, s), "sort");
        const unsigned long long *sk = dk.Current();
        const unsigned long long *sp = dp.Current();

        DevBuf<int> head, bid;
        head.alloc(E, "MAS banked_matrix heads");
        bid.alloc(E, "MAS banked_matrix heads");
        k_heads<<<grid_for(E), 256, 0, s>>>(E, sk, head.get());
        cuda_check(cudaGetLastError(), "heads launch");
        size_t scan_bytes = 0;
        cuda_check(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, head.get(), bid.get(), E, s), "scan size");
        DevBuf<unsigned char> tmp2;
        tmp2.alloc(scan_bytes, "MAS banked_matrix scan");
        cuda_check(cub::DeviceScan::InclusiveSum(tmp2.get(), scan_bytes, head.get(), bid.get(), E, s), "scan");
        int nnzb = 0;
        cuda_check(cudaMemcpyAsync(&nnzb, bid.get() + (E - 1), sizeof(int), cudaMemcpyDeviceToHost, s), "nnzb");

        M.rowlen.alloc(nodes, "MAS banked_matrix rowlen");
        cuda_check(cudaMemsetAsync(M.rowlen.get(), 0, sizeof(int) * nodes, s), "memset");
        k_rowlen<<<grid_for(E), 256, 0, s>>>(E, sk, head.get(), M.rowlen.get());
        cuda_check(cudaGetLastError(), "rowlen launch");

        DevBuf<long long> width;
        width.alloc(banks + 1, "MAS banked_matrix width");
        cuda_check(cudaMemsetAsync(width.get(), 0, sizeof(long long) * (banks + 1), s), "memset");
        k_width<<<(banks * 32 + 255) / 256, 256, 0, s>>>(banks, M.rowlen.get(), width.get());
        cuda_check(cudaGetLastError(), "width launch");
        M.slice.alloc(banks + 1, "MAS banked_matrix slices");
        size_t b1 = 0;
        cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, b1, width.get(), M.slice.get(), banks + 1, s), "scan size");
        DevBuf<int> row_start;
        row_start.alloc(nodes, "MAS banked_matrix row_start");
        size_t b2 = 0;
        cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, b2, M.rowlen.get(), row_start.get(), nodes, s), "scan size");
        DevBuf<unsigned char> tmp3;
        tmp3.alloc(b1 > b2 ? b1 : b2, "MAS banked_matrix scan");
        cuda_check(cub::DeviceScan::ExclusiveSum(tmp3.get(), b1, width.get(), M.slice.get(), banks + 1, s), "scan");
        cuda_check(cub::DeviceScan::ExclusiveSum(tmp3.get(), b2, M.rowlen.get(), row_start.get(), nodes, s), "scan");
        long long slots = 0;
        cuda_check(cudaMemcpyAsync(&slots, M.slice.get() + banks, sizeof(long long), cudaMemcpyDeviceToHost, s),
                   "slots");
        cuda_check(cudaStreamSynchronize(s), "banked sizes");
        M.nnzb = nnzb;
        M.slots = slots;

        M.cols.alloc((size_t)slots * 32, "MAS banked_matrix cols");
        M.vals.alloc((size_t)slots * 32 * bd * bd, "MAS banked_matrix vals");
        M.scatter.alloc((size_t)nnz, "MAS banked_matrix scatter");
        cuda_check(cudaMemsetAsync(M.cols.get(), 0, M.cols.bytes(), s), "memset");
        cuda_check(cudaMemsetAsync(M.vals.get(), 0, M.vals.bytes(), s), "memset");
        DevBuf<long long> pad_pos;
        pad_pos.alloc(3, "MAS banked_matrix pads");
        cuda_check(cudaMemsetAsync(pad_pos.get(), 0xFF, 3 * sizeof(long long), s), "memset");
        k_fill<<<grid_for(E), 256, 0, s>>>(E, bd, sk, sp, bid.get(), row_start.get(), M.slice.get(), d_vals,
                                           M.cols.get(), M.vals.get(), M.scatter.get(), pad_pos.get());
        cuda_check(cudaGetLastError(), "fill launch");
        cuda_check(cudaMemcpyAsync(M.pad_index, pad_pos.get(), 3 * sizeof(long long), cudaMemcpyDeviceToHost, s),
                   "pads");
        cuda_check(cudaStreamSynchronize(s), "banked fill");
        M.npad = npad;
    }

    void rescatter_values(BankedMatrix &M, long long nnz, const double *d_vals, cudaStream_t s)
    {
        k_rescatter<<<grid_for(nnz), 256, 0, s>>>(nnz, M.scatter.get(), d_vals, M.vals.get());
        cuda_check(cudaGetLastError(), "rescatter launch");
    }
} // namespace pmas
