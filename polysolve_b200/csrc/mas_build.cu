// MAS preconditioner factorization on the device (sm_100a).
//
// Restates MASPreconditioner::factorize (MASPreconditioner.cu:982-1097) on the padded numbering:
//  1. level-0 coarse space: connected components of each bank (32 nodes) from bitmask closure of
//     the in-bank neighbour masks (:128-213), numbered by lowest lane, offset by an exclusive scan
//     over banks (:323-340);
//  2. levels 1..3: masks of neighbouring components inside banks of 32 consecutive component ids
//     (:222-275), components again (:281-318), global ids (:345-363); stop when nothing merges
//     (:464-469);
//  3. subdomain matrices: level 0 straight from each bank's rows (upper triangle, no atomics);
//     coarse levels hold the reference's sums (same bank, row <= col, diagonal block upper only,
//     A_ij + A_ij^T when two nodes collapse, :494-591) but build them hierarchically and without
//     atomics: the Galerkin blocks S_0(a, b) = sum of the fine blocks A_uw with map(u) = a,
//     map(w) = b, then S_(l+1)(A, B) = sum of S_l(a, b) over the children pairs, each a
//     fixed-order sum over a record list sorted once per coarse space (deterministic: the same
//     values give the same bits; the reference's FP64 atomics do not);
//  4. zero diagonals -> 1 (:779-796) and an in-place symmetric sweep inverse in FP64 (the
//     Beaton / Goodnight sweep operator, as in batched_invert_upper :799-900), with a device error
//     flag instead of an exception; the result is stored tile-packed in FP64 or FP32.

#include <algorithm>
#include <mutex>
#include <cub/cub.cuh>
#include <type_traits>
#include <vector>

#include "mas_common.cuh"

namespace pmas
{
    MasView MasDevice::view(double *rc_override, double *zc_override) const
    {
        MasView v{};
        v.bd = bd;
        v.banks = banks;
        v.level_num = level_num;
        v.total_coarse = total_coarse;
        for (int i = 0; i < LEVELS; ++i)
        {
            v.mat_offsets[i] = mat_offsets[i];
            v.mat_counts[i] = mat_counts[i];
        }
        for (int i = 0; i < MAX_COARSE; ++i)
        {
            v.cco_nums[i] = cco_nums[i];
            v.coff[i] = coff[i];
        }
        v.storage = storage;
        v.first_iso_bank = first_iso_bank;
        for (int i = 0; i < MAX_COARSE; ++i)
            v.real_count[i] = real_count[i];
        v.n_coarse_active = n_coarse_active;
        v.coarse_active = coarse_active.get();
        v.inv = storage == STORE_F64 ? (const void *)inv64.get()
                : (storage == STORE_F16 ? (const void *)inv16.get() : (const void *)inv32.get());
        v.inv_scale = inv_scale.get();
        v.lcco0 = lcco0.get();
        v.cco0_base = cco0_base.get();
        v.cslot = cslot.get();
        v.parent = parent.get();
        v.ticket = ticket.get();
        for (int l = 0; l < MAX_COARSE; ++l)
            v.kid_ptr[l] = kid_ptr_all.get() ? kid_ptr_all.get() + kid_ptr_off[l] : nullptr;
        v.kids = kids.get();
        v.identity = identity.get();
        v.rc = rc_override ? rc_override : rc.get();
        v.zc = zc_override ? zc_override : zc.get();
        return v;
    }

    namespace
    {
        __device__ __forceinline__ int ctz32(unsigned x) { return __ffs(x) - 1; }

        // Bitmask closure inside a warp; masks in shared memory (32 per warp). Returns the local
        // component id of this lane (-1 if invalid) and writes the component count to *count.
        __device__ __forceinline__ int warp_components(unsigned mask, bool valid, unsigned *sm, int *count)
        {
            const int lane = threadIdx.x & 31;
            sm[lane] = valid ? mask : 0u;
            __syncwarp();
            unsigned conn = valid ? mask : 0u;
            if (valid)
            {
                unsigned visited = 1u << lane;
                unsigned todo = conn & ~visited;
                while (todo)
                {
                    const int v = ctz32(todo);
                    conn |= sm[v];
                    visited |= 1u << v;
                    todo = conn & ~visited;
                }
            }
            const int lead = valid ? ctz32(conn) : -1;
            const unsigned leads = __ballot_sync(FULL, valid && lead == lane);
            __syncwarp();
            *count = __popc(leads);
            if (!valid)
                return -1;
            return __popc(leads & ((1u << lead) - 1u));
        }

        __global__ void k_cco_lv0(BankedView A, const int *__restrict__ node_real, int *lcco0, int *cnt)
        {
            __shared__ unsigned sm[8][32];
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            const int bank = blockIdx.x * 8 + w;
            if (bank >= A.banks)
                return;
            const int u = bank * 32 + lane;
            const bool real = node_real[u] != 0;
            unsigned m = 1u << lane;
            if (real)
            {
                const long long s0 = A.slice[bank];
                const int len = A.rowlen[u];
                for (int k = 0; k < len; ++k)
                {
                    const int c = A.cols[(s0 + k) * 32 + lane];
                    if ((c >> 5) == bank && node_real[c])
                        m |= 1u << (c & 31);
                }
            }
            int count;
            const int id = warp_components(m, real, sm[w], &count);
            lcco0[u] = id;
            if (lane == 0)
                cnt[bank] = count;
        }

        __global__ void k_map_lv0(int nodes, const int *__restrict__ lcco0, const int *__restrict__ base, int *map)
        {
            const int u = blockIdx.x * blockDim.x + threadIdx.x;
            if (u >= nodes)
                return;
            const int l = lcco0[u];
            map[(long long)u * 4 + 0] = l >= 0 ? base[u >> 5] + l : -1;
            map[(long long)u * 4 + 1] = -1;
            map[(long long)u * 4 + 2] = -1;
            map[(long long)u * 4 + 3] = -1;
        }

        __global__ void k_masks_lvx(BankedView A, const int *__restrict__ node_real, const int *__restrict__ map,
                                    int lv, unsigned *masks)
        {
            const int u = blockIdx.x * blockDim.x + threadIdx.x;
            if (u >= A.banks * 32 || !node_real[u])
                return;
            const int c = map[(long long)u * 4 + lv - 1];
            unsigned m = 1u << (c & 31);
            const long long s0 = A.slice[u >> 5];
            const int lane = u & 31;
            const int len = A.rowlen[u];
            for (int k = 0; k < len; ++k)
            {
                const int wn = A.cols[(s0 + k) * 32 + lane];
                if (!node_real[wn])
                    continue;
                const int cw = map[(long long)wn * 4 + lv - 1];
                if ((c >> 5) == (cw >> 5))
                    m |= 1u << (cw & 31);
            }
            atomicOr(&masks[c], m);
        }

        __global__ void k_cco_lvx(int C, const unsigned *__restrict__ masks, int *lid, int *cnt)
        {
            __shared__ unsigned sm[8][32];
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            const int bank = blockIdx.x * 8 + w;
            const int c = bank * 32 + lane;
            if (bank * 32 >= C)
                return;
            const bool valid = c < C;
            int count;
            const int id = warp_components(valid ? masks[c] : 0u, valid, sm[w], &count);
            if (valid)
                lid[c] = id;
            if (lane == 0)
                cnt[bank] = count;
        }

        __global__ void k_map_lvx(int nodes, int lv, const int *__restrict__ lid, const int *__restrict__ base, int *map)
        {
            const int u = blockIdx.x * blockDim.x + threadIdx.x;
            if (u >= nodes)
                return;
            const int prev = map[(long long)u * 4 + lv - 1];
            map[(long long)u * 4 + lv] = prev >= 0 ? base[prev >> 5] + lid[prev] : -1;
        }

        // ----------------------------------------------------------------------------------
        // Dense symmetric work matrix in shared memory (N x N, FP64), sweep inverse, store.
        // ----------------------------------------------------------------------------------
        __device__ __forceinline__ void store_value(double *o, double v, double) { *o = v; }
        __device__ __forceinline__ void store_value(float *o, double v, double) { *o = (float)v; }
        // Binary16: scaled by the matrix's power of two, rounded to FP32 and then to nearest-even.
        __device__ __forceinline__ void store_value(__half *o, double v, double sc)
        {
            *o = __float2half_rn((float)(v * sc));
        }

        // Work matrix in shared memory: N x N FP64 with a row stride of N + 2 doubles, so eight
        // consecutive rows at one column fall in eight different 16-byte bank groups (the tiled
        // update below reads and writes 4-row x 4-column tiles and their transposes), followed
        // by the pivot records of one block of INV_KB pivots.
        constexpr int INV_KB = 8;
        constexpr int INV_NCOEF = INV_KB * (2 * INV_KB + 1);
        __host__ __device__ constexpr int inv_ld(int n) { return n + 2; }
        __host__ __device__ constexpr size_t inv_smem_bytes(int n)
        {
            return ((size_t)n * inv_ld(n) + INV_NCOEF) * sizeof(double);
        }

        // Inverts the symmetric N x N matrix A (shared memory, stride inv_ld(N), both triangles
        // kept) and stores the inverse in `out` (tile-packed; binary16: mma16); *scale_out
        // receives the factor that turns stored values back into matrix values (1 unless
        // binary16); *ident_out (if given) 1 when the inverse is exactly the identity.
        template <int BD, class Out>
        __device__ void invert_and_store(double *A, double *coef, Out *out, double *scale_out, int *ident_out,
                                         int *flag)
        {
            constexpr int N = 32 * BD;
            constexpr int LD = inv_ld(N);
            const int tid = threadIdx.x, nt = blockDim.x;
            __shared__ int bad;
            if (tid == 0)
                bad = 0;
            for (int i = tid; i < N; i += nt)
                if (A[i * LD + i] == 0.0)
                    A[i * LD + i] = 1.0;
            __syncthreads();
            // Blocked sweep (KB pivots per block; both triangles kept exactly symmetric):
            //  1. warp 0 sweeps the KB x KB pivot block pivot by pivot and records, per pivot q, its
            //     value d_q, pivot-row entries r_t = A[q][t] and scaled entries s_t = r_t / d_q;
            //  2. every column c outside the block replays those pivots on its KB panel entries
            //     (one thread per column, registers) with the single-pivot rule;
            //  3. the block's rank-KB update A[t][c] -= sum_q A[t][q] W[q][c] of the upper triangle
            //     outside the block (A[t][q]: the block's columns, untouched so far; W: the swept
            //     panel), in 4 x 4 register tiles, one tile per thread, each mirrored;
            //  4. the panel is mirrored into the block's columns. The same operator as N single
            //     pivots (upper-triangle products for both triangles, each element's KB products
            //     subtracted in pivot order), with N / KB rounds of block-wide barriers.
            // Look-ahead: during step 3 warp 0 updates the next block's own tiles first and then
            // runs step 1 for it, while the other warps update the remaining tiles; step 1 and
            // step 3 touch disjoint elements (and the pivot records are free once step 2 is done).
            constexpr int KB = INV_KB;
            static_assert(N % KB == 0 && KB % 4 == 0, "pivot blocks of whole tiles");
            const int lane = tid & 31, warp = tid >> 5;
            double *cd = coef;                // [KB] pivots
            double *cr = coef + KB;           // [KB][KB] pivot-row entries (0 at the pivot)
            double *cs = coef + KB + KB * KB; // [KB][KB] scaled entries
            constexpr int TR = N / 4;               // tile rows
            constexpr int TK = TR - KB / 4;         // tile rows outside a pivot block
            constexpr int TILES = TK * (TK + 1) / 2; // upper-triangle tiles outside it

            // Step 1 for the block at bs (warp 0, all lanes).
            auto sweep_block = [&](int bs) {
                for (int qq = 0; qq < KB; ++qq)
                {
                    const int q = bs + qq;
                    const double d = A[q * LD + q];
                    if (lane == 0 && (!isfinite(d) || d == 0.0))
                        bad = 1;
                    if (lane < KB)
                    {
                        const double rq = (lane == qq) ? 0.0 : A[q * LD + bs + lane];
                        cr[qq * KB + lane] = rq;
                        cs[qq * KB + lane] = rq / d; // the row scale, one division per row
                    }
                    if (lane == 0)
                        cd[qq] = d;
                    __syncwarp();
                    for (int e = lane; e < KB * KB; e += 32)
                    {
                        const int ti = e / KB, ci = e % KB;
                        double u;
                        if (ti == qq)
                            u = (ci == qq) ? -1.0 / d : cs[qq * KB + ci];
                        else if (ci == qq)
                            u = cs[qq * KB + ti];
                        else
                            u = A[(bs + ti) * LD + bs + ci] -
                                (ti <= ci ? cs[qq * KB + ti] * cr[qq * KB + ci] : cs[qq * KB + ci] * cr[qq * KB + ti]);
                        if (!isfinite(u))
                            bad = 1;
                        A[(bs + ti) * LD + bs + ci] = u;
                    }
                    __syncwarp();
                }
            };

            // Step 3 for tile (i, j), i <= j, of the TK x TK grid of tiles outside the block at b0
            // (tile rows at or after the block's skip its KB / 4 tile rows). Threads with
            // consecutive tile columns J of one tile row share a warp quarter, and the row stride
            // is 49 16-byte units (1 mod 8): a thread reads and writes the two halves of a 4-wide
            // row segment in the order set by bit 2 of J, and stores the transposed tile's rows in
            // an order rotated by J, so the 16-byte accesses of a quarter warp fall in different
            // bank groups.
            auto update_tile = [&](int b0, int i, int j) {
                const int pb = b0 / 4;
                const int I = i < pb ? i : i + KB / 4;
                const int J = j < pb ? j : j + KB / 4;
                const int t0 = 4 * I, c0 = 4 * J;
                const int h0 = (J >> 2) & 1; // half of a row segment accessed first
                auto load_seg = [&](int row, double (&v)[4]) {
                    const double2 f = *reinterpret_cast<const double2 *>(A + row * LD + c0 + 2 * h0);
                    const double2 g = *reinterpret_cast<const double2 *>(A + row * LD + c0 + 2 - 2 * h0);
                    v[0] = h0 ? g.x : f.x;
                    v[1] = h0 ? g.y : f.y;
                    v[2] = h0 ? f.x : g.x;
                    v[3] = h0 ? f.y : g.y;
                };
                double u[4][4];
#pragma unroll
                for (int r = 0; r < 4; ++r)
                    load_seg(t0 + r, u[r]);
#pragma unroll
                for (int q2 = 0; q2 < KB; q2 += 2)
                {
                    double pc[4][2], wr[2][4];
#pragma unroll
                    for (int r = 0; r < 4; ++r)
                    {
                        const double2 pv = *reinterpret_cast<const double2 *>(A + (t0 + r) * LD + b0 + q2);
                        pc[r][0] = pv.x;
                        pc[r][1] = pv.y;
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        load_seg(b0 + q2 + h, wr[h]);
#pragma unroll
                    for (int h = 0; h < 2; ++h)
#pragma unroll
                        for (int r = 0; r < 4; ++r)
#pragma unroll
                            for (int c = 0; c < 4; ++c)
                                u[r][c] -= pc[r][h] * wr[h][c];
                }
                int badt = 0;
#pragma unroll
                for (int r = 0; r < 4; ++r)
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (t0 != c0 || r <= c)
                            badt |= !isfinite(u[r][c]);
                if (badt)
                    bad = 1;
                if (t0 != c0)
                {
#pragma unroll
                    for (int r = 0; r < 4; ++r)
                    {
                        double2 *row = reinterpret_cast<double2 *>(A + (t0 + r) * LD + c0);
                        row[h0] = h0 ? make_double2(u[r][2], u[r][3]) : make_double2(u[r][0], u[r][1]);
                        row[1 - h0] = h0 ? make_double2(u[r][0], u[r][1]) : make_double2(u[r][2], u[r][3]);
                    }
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                    {
                        const int cc = (c + J) & 3; // rotated transposed-row order
                        double col[4];
#pragma unroll
                        for (int r = 0; r < 4; ++r)
                            col[r] = cc == 0 ? u[r][0] : (cc == 1 ? u[r][1] : (cc == 2 ? u[r][2] : u[r][3]));
                        *reinterpret_cast<double2 *>(A + (c0 + cc) * LD + t0) = make_double2(col[0], col[1]);
                        *reinterpret_cast<double2 *>(A + (c0 + cc) * LD + t0 + 2) = make_double2(col[2], col[3]);
                    }
                }
                else
                {
                    // Diagonal tile: its upper triangle, mirrored (the lower products are not used,
                    // as in the single-pivot sweep).
#pragma unroll
                    for (int r = 0; r < 4; ++r)
#pragma unroll
                        for (int c = r; c < 4; ++c)
                        {
                            A[(t0 + r) * LD + t0 + c] = u[r][c];
                            A[(t0 + c) * LD + t0 + r] = u[r][c];
                        }
                }
            };

            if (warp == 0)
                sweep_block(0);
            __syncthreads();
            for (int b0 = 0; b0 < N; b0 += KB)
            {
                // Step 2 with the records of block b0 (written by its step 1).
                for (int c = tid; c < N; c += nt)
                {
                    if ((unsigned)(c - b0) < (unsigned)KB)
                        continue;
                    double v[KB];
#pragma unroll
                    for (int i = 0; i < KB; ++i)
                        v[i] = A[(b0 + i) * LD + c];
                    int badc = 0;
#pragma unroll
                    for (int qq = 0; qq < KB; ++qq)
                    {
                        const double d = cd[qq];
                        const double a = v[qq];      // A[q][c] before pivot q
                        const double as = a / d;     // its row scale
#pragma unroll
                        for (int i = 0; i < KB; ++i)
                        {
                            const int t = b0 + i;
                            if (i == qq)
                                v[i] = as;
                            else
                                v[i] = v[i] - (t <= c ? cs[qq * KB + i] * a : as * cr[qq * KB + i]);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < KB; ++i)
                    {
                        badc |= !isfinite(v[i]);
                        A[(b0 + i) * LD + c] = v[i];
                    }
                    if (badc)
                        bad = 1;
                }
                __syncthreads();
                const int pb = b0 / 4;
                const bool ahead = b0 + KB < N;
                if (ahead && warp == 0)
                {
                    // The next block's tiles (compressed (pb, pb), (pb, pb + 1), (pb + 1, pb + 1)),
                    // then its step 1.
                    if (lane < 3)
                        update_tile(b0, pb + (lane == 2 ? 1 : 0), pb + (lane >= 1 ? 1 : 0));
                    __syncwarp();
                    sweep_block(b0 + KB);
                }
                else
                {
                    const int first = ahead ? 32 : 0;
                    for (int k = tid - first; k < TILES; k += nt - first)
                    {
                        int i = 0, rem = k;
                        while (rem >= TK - i)
                        {
                            rem -= TK - i;
                            ++i;
                        }
                        const int j = i + rem;
                        if (ahead && (unsigned)(i - pb) < 2u && j <= pb + 1)
                            continue; // the next block's own tiles: warp 0
                        update_tile(b0, i, j);
                    }
                }
                __syncthreads();
                // The panel into the block's columns: one row t per thread, its KB entries written
                // as contiguous pairs (consecutive rows: different bank groups).
                for (int t = tid; t < N; t += nt)
                {
                    if ((unsigned)(t - b0) < (unsigned)KB)
                        continue;
#pragma unroll
                    for (int q2 = 0; q2 < KB; q2 += 2)
                        *reinterpret_cast<double2 *>(A + t * LD + b0 + q2) =
                            make_double2(A[(b0 + q2) * LD + t], A[(b0 + q2 + 1) * LD + t]);
                }
                __syncthreads();
            }
            // Binary16 storage: one power-of-two scale per matrix maps the largest magnitude into
            // [2^14, 2^15), well inside the format's range (max 65504) and clear of its subnormals.
            double sc = 1.0;
            if constexpr (StoreTraits<Out>::SCALED)
            {
                __shared__ unsigned long long amax_bits;
                if (tid == 0)
                    amax_bits = 0ull;
                __syncthreads();
                unsigned long long m = 0ull;
                for (int e = tid; e < N * N; e += nt)
                {
                    const int t = e / N, c = e - t * N;
                    if (t > c)
                        continue;
                    // Non-negative doubles order like their bit patterns.
                    const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(A[t * LD + c]));
                    m = b > m ? b : m;
                }
                atomicMax(&amax_bits, m);
                __syncthreads();
                const double amax = __longlong_as_double((long long)amax_bits);
                sc = (amax > 0.0 && isfinite(amax)) ? ldexp(1.0, 14 - ilogb(amax)) : 1.0;
            }
            if (tid == 0)
                *scale_out = 1.0 / sc;
            // Exactly the identity (a coarse matrix of isolated rows): the apply copies instead.
            if (ident_out)
            {
                __shared__ int is_id;
                if (tid == 0)
                    is_id = 1;
                __syncthreads();
                for (int e = tid; e < N * N; e += nt)
                {
                    const int t = e / N, c = e - t * N;
                    if (t <= c && -A[t * LD + c] != (t == c ? 1.0 : 0.0))
                        is_id = 0;
                }
                __syncthreads();
                if (tid == 0)
                    *ident_out = is_id;
            }
            if constexpr (StoreTraits<Out>::SCALED)
            {
                // Binary16: mma16 layout (tensor-core fragments).
                constexpr int S16 = (2 * BD) * (2 * BD - 1) / 2 * 256 + 2 * BD * 192;
                for (int idx = tid; idx < S16; idx += nt)
                {
                    int row, cl;
                    mma16_rowcol(BD, idx, row, cl);
                    const double v = -A[row * LD + cl];
                    if (!isfinite(v))
                        bad = 1;
                    store_value(out + idx, v, sc);
                }
                __syncthreads();
                if (tid == 0 && bad)
                    atomicExch(flag, ERR_INVERSE);
                return;
            }
            // Store -A (the inverse) tile-packed.
            constexpr int S = N * (N + 1) / 2;
            for (int idx = tid; idx < S; idx += nt)
            {
                // Decode the tile-packed index.
                int rem = idx, J = 0;
                while (rem >= J * 1024 + 528)
                {
                    rem -= J * 1024 + 528;
                    ++J;
                }
                int row, cl;
                if (rem < J * 1024)
                {
                    const int I = rem >> 10, e = rem & 1023;
                    const int j4 = e >> 7, l = (e & 127) >> 2, jj = e & 3;
                    row = 32 * I + l;
                    cl = 32 * J + 4 * j4 + jj;
                }
                else
                {
                    const int e = rem - J * 1024;
                    int j = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
                    while (j * (j + 1) / 2 > e)
                        --j;
                    while ((j + 1) * (j + 2) / 2 <= e)
                        ++j;
                    row = 32 * J + (e - j * (j + 1) / 2);
                    cl = 32 * J + j;
                }
                const double v = -A[row * LD + cl];
                if (!isfinite(v))
                    bad = 1;
                store_value(out + idx, v, sc);
            }
            __syncthreads();
            if (tid == 0 && bad)
                atomicExch(flag, ERR_INVERSE);
        }

        // Three CTAs per SM (shared memory: 76 KB each at block_dim 3; registers capped to fit).
        template <int BD, class Out>
        __global__ void __launch_bounds__(256, 3) k_assemble_invert_lv0(BankedView A, const int *__restrict__ node_real,
                                                                        Out *out, double *scale, int *flag)
        {
            constexpr int N = 32 * BD, LD = inv_ld(N);
            constexpr int S = StoreTraits<Out>::SCALED ? (2 * BD) * (2 * BD - 1) / 2 * 256 + 2 * BD * 192
                                                       : N * (N + 1) / 2;
            extern __shared__ __align__(16) double dsm[];
            double *M = dsm;
            double *coef = dsm + N * LD;
            const int bank = blockIdx.x;
            for (int i = threadIdx.x; i < N * LD; i += blockDim.x)
                M[i] = 0.0;
            __syncthreads();
            // 8 threads per node, each walking a subset of the node's slots.
            const int lane = threadIdx.x >> 3, sub = threadIdx.x & 7;
            const int u = bank * 32 + lane;
            if (node_real[u])
            {
                const long long s0 = A.slice[bank];
                const int len = A.rowlen[u];
                for (int k = sub; k < len; k += 8)
                {
                    const long long slot = s0 + k;
                    const int w = A.cols[slot * 32 + lane];
                    if ((w >> 5) != bank || !node_real[w])
                        continue;
                    const int lw = w & 31;
                    if (lw < lane)
                        continue; // upper triangle in node order (reference skips tid > j)
#pragma unroll
                    for (int bi = 0; bi < BD; ++bi)
#pragma unroll
                        for (int bj = 0; bj < BD; ++bj)
                        {
                            if (lw == lane && bi > bj)
                                continue;
                            const double v = A.vals[banked_value_index(slot, lane, bi * BD + bj, BD)];
                            const int row = lane * BD + bi, cl = lw * BD + bj;
                            M[row * LD + cl] = v;
                            M[cl * LD + row] = v;
                        }
                }
            }
            __syncthreads();
            invert_and_store<BD, Out>(M, coef, out + (size_t)bank * S, scale + bank, nullptr, flag);
        }

        template <int BD, class Out>
        __global__ void __launch_bounds__(256, 3) k_invert_coarse(const double *__restrict__ staging, Out *out,
                                                                  double *scale, int *identity, int *flag)
        {
            constexpr int N = 32 * BD, LD = inv_ld(N);
            constexpr int S = StoreTraits<Out>::SCALED ? (2 * BD) * (2 * BD - 1) / 2 * 256 + 2 * BD * 192
                                                       : N * (N + 1) / 2;
            extern __shared__ __align__(16) double dsm[];
            double *M = dsm;
            double *coef = dsm + N * LD;
            const double *src = staging + (size_t)blockIdx.x * N * N;
            for (int e = threadIdx.x; e < N * N; e += blockDim.x)
            {
                const int r = e / N, c = e - r * N;
                M[r * LD + c] = (r <= c) ? src[r * N + c] : src[c * N + r];
            }
            __syncthreads();
            invert_and_store<BD, Out>(M, coef, out + (size_t)blockIdx.x * S, scale + blockIdx.x, identity + blockIdx.x,
                                      flag);
        }

        __global__ void k_cslot(int nodes, int level_num, const int *__restrict__ map, int coff0, int coff1, int coff2,
                                int coff3, int4 *cslot)
        {
            const int u = blockIdx.x * blockDim.x + threadIdx.x;
            if (u >= nodes)
                return;
            const int coff[4] = {coff0, coff1, coff2, coff3};
            int v[4];
#pragma unroll
            for (int l = 0; l < 4; ++l)
            {
                const int c = map[(long long)u * 4 + l];
                v[l] = (l < level_num && c >= 0) ? coff[l] + c : -1;
            }
            cslot[u] = make_int4(v[0], v[1], v[2], v[3]);
        }

        int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

        template <class T>
        void exclusive_scan(const T *in, T *out, int n, cudaStream_t s)
        {
            size_t bytes = 0;
            cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s), "scan size");
            DevBuf<unsigned char> tmp;
            tmp.alloc(bytes, "MAS coarse_space scan");
            cuda_check(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, in, out, n, s), "scan");
            cuda_check(cudaStreamSynchronize(s), "scan sync");
        }


        // ---- Deterministic hierarchical coarse assembly -------------------------------------
        // Record rules: the source block X enters its target as X, X^T, or X + X^T (two distinct
        // nodes collapsing into one coarse node).
        constexpr int RULE_PLAIN = 0, RULE_TRANS = 1, RULE_SYM = 2;

        __device__ __forceinline__ void pair_rule(long long a, long long b, bool same_source_node, long long cn,
                                                  long long &key, int &rule)
        {
            if (a < b)
            {
                key = a * cn + b;
                rule = RULE_PLAIN;
            }
            else if (a > b)
            {
                key = b * cn + a;
                rule = RULE_TRANS;
            }
            else
            {
                key = a * cn + a;
                rule = same_source_node ? RULE_PLAIN : RULE_SYM;
            }
        }

        // Level 0 records: one per coupled fine pair (u <= w), both real.
        __global__ void k_fine_pair_count(BankedView A, const int *__restrict__ node_real, long long *cnt)
        {
            const int u = blockIdx.x * blockDim.x + threadIdx.x;
            if (u >= A.banks * 32)
                return;
            long long c = 0;
            if (node_real[u])
            {
                const long long s0 = A.slice[u >> 5];
                const int lane = u & 31, len = A.rowlen[u];
                for (int k = 0; k < len; ++k)
                {
                    const int w = A.cols[(s0 + k) * 32 + lane];
                    if (w >= u && node_real[w])
                        ++c;
                }
            }
            cnt[u] = c;
        }

        __global__ void k_fine_pair_emit(BankedView A, const int *__restrict__ node_real, const int *__restrict__ map,
                                         const long long *__restrict__ off, long long cn, long long *keys,
                                         long long *payload)
        {
            const int u = blockIdx.x * blockDim.x + threadIdx.x;
            if (u >= A.banks * 32 || !node_real[u])
                return;
            const long long s0 = A.slice[u >> 5];
            const int lane = u & 31, len = A.rowlen[u];
            long long pos = off[u];
            const long long a = map[(long long)u * 4];
            for (int k = 0; k < len; ++k)
            {
                const long long slot = s0 + k;
                const int w = A.cols[slot * 32 + lane];
                if (w < u || !node_real[w])
                    continue;
                const long long b = map[(long long)w * 4];
                long long key;
                int rule;
                pair_rule(a, b, w == u, cn, key, rule);
                keys[pos] = key;
                payload[pos] = ((slot * 32 + lane) << 2) | rule;
                ++pos;
            }
        }

        // Level l + 1 records: one per level-l target, through the parents.
        __global__ void k_coarse_pair_emit(const int2 *__restrict__ pair, int targets, const int *__restrict__ parent,
                                           long long cn, long long *keys, long long *payload)
        {
            const int t = blockIdx.x * blockDim.x + threadIdx.x;
            if (t >= targets)
                return;
            const int2 p = pair[t];
            long long key;
            int rule;
            pair_rule(parent[p.x], parent[p.y], p.x == p.y, cn, key, rule);
            keys[t] = key;
            payload[t] = ((long long)t << 2) | rule;
        }

        __global__ void k_key_heads(const long long *__restrict__ keys, long long n, int *head)
        {
            const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            if (i < n)
                head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
            else if (i == n)
                head[i] = 0;
        }

        __global__ void k_key_targets(const long long *__restrict__ keys, const int *__restrict__ head,
                                      const int *__restrict__ hidx, long long n, long long cn, int *ptr, int2 *pair)
        {
            const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
            if (i < n && head[i])
            {
                const int t = hidx[i];
                ptr[t] = (int)i;
                pair[t] = make_int2((int)(keys[i] / cn), (int)(keys[i] % cn));
            }
            if (i == n)
                ptr[hidx[n]] = (int)n;
        }

        // One thread per target: the fixed-order sum of its records; same-bank pairs also go to
        // the upper triangle of their coarse matrix in the staging buffer.
        template <int BD>
        __global__ void __launch_bounds__(256)
            k_coarse_sum(bool fine, const long long *__restrict__ src, const int *__restrict__ ptr,
                         const int2 *__restrict__ pair, int targets, BankedView A, const double *__restrict__ prev,
                         double *__restrict__ vals, double *__restrict__ staging)
        {
            constexpr int BS = BD * BD, N = 32 * BD;
            const int t = blockIdx.x * blockDim.x + threadIdx.x;
            if (t >= targets)
                return;
            double acc[BS];
#pragma unroll
            for (int q = 0; q < BS; ++q)
                acc[q] = 0.0;
            const int r1 = ptr[t + 1];
            for (int r = ptr[t]; r < r1; ++r)
            {
                const long long rec = src[r];
                const int rule = (int)(rec & 3);
                const long long idx = rec >> 2;
                double x[BS];
                if (fine)
                {
#pragma unroll
                    for (int q = 0; q < BS; ++q)
                        x[q] = A.vals[banked_value_index(idx >> 5, (int)(idx & 31), q, BD)];
                }
                else
                {
#pragma unroll
                    for (int q = 0; q < BS; ++q)
                        x[q] = prev[idx * BS + q];
                }
#pragma unroll
                for (int i = 0; i < BD; ++i)
#pragma unroll
                    for (int j = 0; j < BD; ++j)
                    {
                        const double xt = x[j * BD + i];
                        const double v = rule == RULE_PLAIN ? x[i * BD + j]
                                                            : (rule == RULE_TRANS ? xt : x[i * BD + j] + xt);
                        acc[i * BD + j] += v;
                    }
            }
#pragma unroll
            for (int q = 0; q < BS; ++q)
                vals[(long long)t * BS + q] = acc[q];
            const int2 p = pair[t];
            if ((p.x >> 5) != (p.y >> 5))
                return;
            double *mat = staging + (size_t)(p.x >> 5) * N * N;
#pragma unroll
            for (int i = 0; i < BD; ++i)
#pragma unroll
                for (int j = 0; j < BD; ++j)
                {
                    const int row = (p.x & 31) * BD + i, col = (p.y & 31) * BD + j;
                    if (row <= col)
                        mat[row * N + col] = acc[i * BD + j];
                }
        }

        int key_bits(long long cn)
        {
            const unsigned long long top = (unsigned long long)cn * (unsigned long long)cn;
            int bits = 1;
            while (bits < 64 && (top >> bits) != 0)
                ++bits;
            return bits;
        }

        // The record lists of every coarse level (once per coarse space).
        void build_coarse_sums(MasDevice &M, const BankedMatrix &A, const int *d_node_real, cudaStream_t s)
        {
            const long long cn = std::max(M.coarse_nodes, 1);
            const int nodes = A.banks * 32;
            for (int l = 0; l < MAX_COARSE; ++l)
            {
                MasDevice::CoarseSum &cs = M.csum[l];
                cs.src.reset();
                cs.ptr.reset();
                cs.pair.reset();
                cs.vals.reset();
                cs.targets = 0;
                cs.records = 0;
                if (l >= M.level_num)
                    continue;
                long long R = 0;
                DevBuf<long long> keys, pay;
                if (l == 0)
                {
                    DevBuf<long long> cnt, off;
                    cnt.alloc((size_t)nodes + 1, "MAS coarse_sums");
                    off.alloc((size_t)nodes + 1, "MAS coarse_sums");
                    cuda_check(cudaMemsetAsync(cnt.get(), 0, cnt.bytes(), s), "memset");
                    if (nodes > 0)
                        k_fine_pair_count<<<div_up(nodes, 256), 256, 0, s>>>(A.view(), d_node_real, cnt.get());
                    cuda_check(cudaGetLastError(), "pair count launch");
                    exclusive_scan(cnt.get(), off.get(), nodes + 1, s);
                    cuda_check(cudaMemcpy(&R, off.get() + nodes, sizeof(long long), cudaMemcpyDeviceToHost), "count");
                    keys.alloc((size_t)std::max(R, 1LL), "MAS coarse_sums");
                    pay.alloc((size_t)std::max(R, 1LL), "MAS coarse_sums");
                    if (nodes > 0)
                        k_fine_pair_emit<<<div_up(nodes, 256), 256, 0, s>>>(A.view(), d_node_real, M.map.get(), off.get(),
                                                                            cn, keys.get(), pay.get());
                    cuda_check(cudaGetLastError(), "pair emit launch");
                }
                else
                {
                    const MasDevice::CoarseSum &pv = M.csum[l - 1];
                    R = pv.targets;
                    keys.alloc((size_t)std::max(R, 1LL), "MAS coarse_sums");
                    pay.alloc((size_t)std::max(R, 1LL), "MAS coarse_sums");
                    if (R > 0)
                        k_coarse_pair_emit<<<div_up((int)R, 256), 256, 0, s>>>(pv.pair.get(), pv.targets, M.parent.get(),
                                                                               cn, keys.get(), pay.get());
                    cuda_check(cudaGetLastError(), "coarse pair emit launch");
                }
                if (R == 0)
                    continue;
                if (R > 2147483000LL)
                    throw Error(ERR_INVALID, "[MAS] coarse assembly: too many block pairs");
                // Stable radix sort by target: records keep their emission order within a target.
                DevBuf<long long> keys_s;
                keys_s.alloc((size_t)R, "MAS coarse_sums");
                cs.src.alloc((size_t)R, "MAS coarse_sums");
                const int bits = key_bits(cn);
                size_t tb = 0;
                cuda_check(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.get(), keys_s.get(), pay.get(), cs.src.get(),
                                                           (int)R, 0, bits, s),
                           "sort size");
                DevBuf<unsigned char> tmp;
                tmp.alloc(std::max<size_t>(tb, 1), "MAS coarse_sums sort");
                cuda_check(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, keys.get(), keys_s.get(), pay.get(), cs.src.get(),
                                                           (int)R, 0, bits, s),
                           "sort");
                DevBuf<int> head, hidx;
                head.alloc((size_t)R + 1, "MAS coarse_sums");
                hidx.alloc((size_t)R + 1, "MAS coarse_sums");
                const int g1 = (int)((R + 1 + 255) / 256);
                k_key_heads<<<g1, 256, 0, s>>>(keys_s.get(), R, head.get());
                cuda_check(cudaGetLastError(), "heads launch");
                exclusive_scan(head.get(), hidx.get(), (int)R + 1, s);
                int T = 0;
                cuda_check(cudaMemcpy(&T, hidx.get() + R, sizeof(int), cudaMemcpyDeviceToHost), "targets");
                cs.ptr.alloc((size_t)T + 1, "MAS coarse_sums");
                cs.pair.alloc((size_t)std::max(T, 1), "MAS coarse_sums");
                k_key_targets<<<g1, 256, 0, s>>>(keys_s.get(), head.get(), hidx.get(), R, cn, cs.ptr.get(), cs.pair.get());
                cuda_check(cudaGetLastError(), "targets launch");
                cs.vals.alloc((size_t)std::max(T, 1) * A.bd * A.bd, "MAS coarse_sums");
                cs.targets = T;
                cs.records = R;
                cuda_check(cudaStreamSynchronize(s), "coarse sums");
            }
        }

        template <int BD, class Out>
        void assemble_and_invert(MasDevice &M, const BankedMatrix &A, const int *d_node_real, Out *out, const int *coff,
                                 cudaStream_t s)
        {
            double *scale = M.inv_scale.get();
            constexpr int N = 32 * BD;
            const size_t smem = inv_smem_bytes(N);
            cuda_check(cudaFuncSetAttribute(k_assemble_invert_lv0<BD, Out>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem),
                       "assemble smem attribute");
            cuda_check(cudaFuncSetAttribute(k_invert_coarse<BD, Out>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem),
                       "invert smem attribute");
            if (!M.inv_ev[0])
                for (cudaEvent_t &e : M.inv_ev)
                    cuda_check(cudaEventCreate(&e), "event");
            cuda_check(cudaEventRecord(M.inv_ev[0], s), "event");
            if (M.banks > 0)
            {
                k_assemble_invert_lv0<BD, Out><<<M.banks, 256, smem, s>>>(A.view(), d_node_real, out, scale, M.flag.get());
                cuda_check(cudaGetLastError(), "assemble lv0 launch");
            }
            cuda_check(cudaEventRecord(M.inv_ev[1], s), "event");
            if (M.total_coarse > 0)
            {
                DevBuf<double> &staging = M.staging;
                staging.alloc((size_t)M.total_coarse * N * N, "MAS coarse_matrices staging");
                cuda_check(cudaMemsetAsync(staging.get(), 0, staging.bytes(), s), "memset");
                for (int l = 0; l < M.level_num; ++l)
                {
                    const MasDevice::CoarseSum &cs = M.csum[l];
                    if (cs.targets == 0)
                        continue;
                    k_coarse_sum<BD><<<div_up(cs.targets, 256), 256, 0, s>>>(
                        l == 0, cs.src.get(), cs.ptr.get(), cs.pair.get(), cs.targets, A.view(),
                        l > 0 ? M.csum[l - 1].vals.get() : nullptr, cs.vals.get(), staging.get());
                    cuda_check(cudaGetLastError(), "coarse sum launch");
                }
                cuda_check(cudaEventRecord(M.inv_ev[2], s), "event");
                const size_t S = (size_t)inv_stride(BD, M.storage);
                k_invert_coarse<BD, Out><<<M.total_coarse, 256, smem, s>>>(staging.get(), out + (size_t)M.banks * S,
                                                                          scale + M.banks, M.identity.get(),
                                                                          M.flag.get());
                cuda_check(cudaGetLastError(), "invert coarse launch");
            }
            else
                cuda_check(cudaEventRecord(M.inv_ev[2], s), "event");
            cuda_check(cudaEventRecord(M.inv_ev[3], s), "event");
        }
    } // namespace

    namespace
    {
        // Level-0 and coarse matrices assembled from the current values of A and inverted in the
        // storage precision (the coarse space in M must match A's pattern).
        void build_inverses(MasDevice &M, const BankedMatrix &A, const int *d_node_real, int storage, const int *coff,
                            cudaStream_t s)
        {
            const int bd = A.bd, banks = A.banks;
            const size_t S = (size_t)inv_stride(bd, storage);
            if (storage != STORE_F64)
                M.inv64.reset();
            if (storage != STORE_F32)
                M.inv32.reset();
            if (storage != STORE_F16)
                M.inv16.reset();
            M.storage = storage;
            cuda_check(cudaMemsetAsync(M.flag.get(), 0, sizeof(int), s), "memset");
            if (storage == STORE_F64)
                M.inv64.alloc(S * M.total_mats, "MAS coarse_matrices");
            else if (storage == STORE_F16)
                M.inv16.alloc(S * M.total_mats, "MAS coarse_matrices");
            else
                M.inv32.alloc(S * M.total_mats, "MAS coarse_matrices");
            M.inv_scale.alloc(M.total_mats > 0 ? M.total_mats : 1, "MAS coarse_matrices scales");
            M.identity.alloc(M.total_coarse > 0 ? M.total_coarse : 1, "MAS coarse_matrices identity");
            cuda_check(cudaMemsetAsync(M.identity.get(), 0, M.identity.bytes(), s), "memset");
            auto run = [&](auto *out) {
                using Out = std::remove_pointer_t<decltype(out)>;
                auto per_bd = [&](auto bdc) {
                    constexpr int BD = decltype(bdc)::value;
                    assemble_and_invert<BD, Out>(M, A, d_node_real, out, coff, s);
                };
                if (bd == 1)
                    per_bd(std::integral_constant<int, 1>{});
                else if (bd == 2)
                    per_bd(std::integral_constant<int, 2>{});
                else
                    per_bd(std::integral_constant<int, 3>{});
            };
            if (storage == STORE_F64)
                run(M.inv64.get());
            else if (storage == STORE_F16)
                run(reinterpret_cast<__half *>(M.inv16.get()));
            else
                run(M.inv32.get());
            int h_flag = 0;
            cuda_check(cudaMemcpyAsync(&h_flag, M.flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s), "flag");
            cuda_check(cudaStreamSynchronize(s), "mas build");
            for (int i = 0; i < 3; ++i)
                cuda_check(cudaEventElapsedTime(&M.inverse_ms[i], M.inv_ev[i], M.inv_ev[i + 1]), "event time");
            if (h_flag)
                throw Error(ERR_INVERSE, "[MAS] MAS packed inverse failed.");
        }
    } // namespace

    namespace
    {
    } // namespace

    void build_mas(MasDevice &M, const BankedMatrix &A, const int *d_node_real, int storage, int first_iso_bank,
                   cudaStream_t s)
    {
        const int bd = A.bd, banks = A.banks, nodes = A.nodes;
        M.bd = bd;
        M.banks = banks;
        M.nodes = nodes;
        M.storage = storage;
        M.flag.alloc(1, "MAS flag");
        cuda_check(cudaMemsetAsync(M.flag.get(), 0, sizeof(int), s), "memset");

        // --- level 0 components
        M.lcco0.alloc(nodes, "MAS coarse_space lcco0");
        M.cco0_base.alloc(banks + 1, "MAS coarse_space base");
        M.map.alloc((size_t)nodes * 4, "MAS coarse_space map");
        DevBuf<int> cnt;
        cnt.alloc(banks + 1, "MAS coarse_space counts");
        cuda_check(cudaMemsetAsync(cnt.get(), 0, sizeof(int) * (banks + 1), s), "memset");
        k_cco_lv0<<<div_up(banks, 8), 256, 0, s>>>(A.view(), d_node_real, M.lcco0.get(), cnt.get());
        cuda_check(cudaGetLastError(), "cco lv0 launch");
        exclusive_scan(cnt.get(), M.cco0_base.get(), banks + 1, s);
        int C = 0;
        cuda_check(cudaMemcpy(&C, M.cco0_base.get() + banks, sizeof(int), cudaMemcpyDeviceToHost), "count");
        k_map_lv0<<<div_up(nodes, 256), 256, 0, s>>>(nodes, M.lcco0.get(), M.cco0_base.get(), M.map.get());
        cuda_check(cudaGetLastError(), "map lv0 launch");
        for (int i = 0; i < MAX_COARSE; ++i)
            M.cco_nums[i] = 0;
        M.cco_nums[0] = C;
        M.level_num = 1;

        // --- levels 1..3
        DevBuf<unsigned> masks;
        DevBuf<int> lid, lbase, lcnt;
        masks.alloc(C > 0 ? C : 1, "MAS coarse_space masks");
        lid.alloc(C > 0 ? C : 1, "MAS coarse_space lid");
        for (int lv = 1; lv < MAX_COARSE && C > 0; ++lv)
        {
            const int cb = div_up(C, 32);
            lcnt.alloc(cb + 1, "MAS coarse_space counts");
            lbase.alloc(cb + 1, "MAS coarse_space base");
            cuda_check(cudaMemsetAsync(masks.get(), 0, sizeof(unsigned) * C, s), "memset");
            cuda_check(cudaMemsetAsync(lcnt.get(), 0, sizeof(int) * (cb + 1), s), "memset");
            k_masks_lvx<<<div_up(nodes, 256), 256, 0, s>>>(A.view(), d_node_real, M.map.get(), lv, masks.get());
            cuda_check(cudaGetLastError(), "masks launch");
            k_cco_lvx<<<div_up(cb, 8), 256, 0, s>>>(C, masks.get(), lid.get(), lcnt.get());
            cuda_check(cudaGetLastError(), "cco lvx launch");
            exclusive_scan(lcnt.get(), lbase.get(), cb + 1, s);
            int next = 0;
            cuda_check(cudaMemcpy(&next, lbase.get() + cb, sizeof(int), cudaMemcpyDeviceToHost), "count");
            k_map_lvx<<<div_up(nodes, 256), 256, 0, s>>>(nodes, lv, lid.get(), lbase.get(), M.map.get());
            cuda_check(cudaGetLastError(), "map lvx launch");
            if (next == C)
                break;
            C = next;
            M.cco_nums[lv] = C;
            M.level_num = lv + 1;
        }
        // Unused levels back to -1 (the early-stop level was written but is not used).
        if (M.level_num < MAX_COARSE)
        {
            std::vector<int> hmap((size_t)nodes * 4);
            cuda_check(cudaMemcpy(hmap.data(), M.map.get(), hmap.size() * sizeof(int), cudaMemcpyDeviceToHost), "map");
            for (int u = 0; u < nodes; ++u)
                for (int l = M.level_num; l < MAX_COARSE; ++l)
                    hmap[(size_t)u * 4 + l] = -1;
            cuda_check(cudaMemcpy(M.map.get(), hmap.data(), hmap.size() * sizeof(int), cudaMemcpyHostToDevice), "map");
        }

        // --- matrix counts and coarse vector layout
        for (int i = 0; i < LEVELS; ++i)
            M.mat_counts[i] = M.mat_offsets[i] = 0;
        M.mat_counts[0] = banks;
        M.total_mats = banks;
        int coff[4] = {0, 0, 0, 0};
        int cn = 0;
        for (int l = 0; l < M.level_num; ++l)
        {
            M.mat_offsets[l + 1] = M.total_mats;
            M.mat_counts[l + 1] = div_up(M.cco_nums[l], 32);
            M.total_mats += M.mat_counts[l + 1];
            coff[l] = cn;
            cn += M.mat_counts[l + 1] * 32;
        }
        M.total_coarse = M.total_mats - banks;
        M.coarse_nodes = cn;

        M.cslot.alloc(nodes, "MAS coarse_space slots");
        k_cslot<<<div_up(nodes, 256), 256, 0, s>>>(nodes, M.level_num, M.map.get(), coff[0], coff[1], coff[2], coff[3],
                                                  M.cslot.get());
        cuda_check(cudaGetLastError(), "cslot launch");

        // Parents: for each coarse node of level l - 1, the level-l coarse node it merges into
        // (every level-l node has at most 32 children, all in one group of 32 consecutive ids).
        for (int l = 0; l < MAX_COARSE; ++l)
            M.coff[l] = coff[l];
        {
            std::vector<int> hmap((size_t)nodes * 4);
            cuda_check(cudaMemcpy(hmap.data(), M.map.get(), hmap.size() * sizeof(int), cudaMemcpyDeviceToHost), "map");
            std::vector<int> parent((size_t)cn, -1); // coarse node -> next-level coarse node
            for (int u = 0; u < nodes; ++u)
                for (int l = 1; l < M.level_num; ++l)
                {
                    const int c = hmap[(size_t)u * 4 + l - 1], up = hmap[(size_t)u * 4 + l];
                    if (c >= 0 && up >= 0)
                        parent[(size_t)coff[l - 1] + c] = coff[l] + up;
                }
            // The coarse-level sums rely on it: the children of every node share one 32-id group
            // (so at most 32 children).
            {
                std::vector<int> group((size_t)cn, -1);
                for (int c = 0; c < cn; ++c)
                {
                    const int pa = parent[c];
                    if (pa < 0)
                        continue;
                    const int g = c >> 5; // coff[] are multiples of 32
                    if (group[pa] < 0)
                        group[pa] = g;
                    else if (group[pa] != g)
                        throw Error(ERR_INVALID, "[MAS] internal: coarse component spans two groups of 32");
                }
            }
            // Isolated-row suffix: the components of the trailing isolated banks must be the
            // largest ids at every level; otherwise the shortcut is off (first_iso_bank = banks).
            int fib = first_iso_bank < banks ? first_iso_bank : banks;
            for (int l = 0; l < MAX_COARSE; ++l)
                M.real_count[l] = (l < M.level_num) ? M.cco_nums[l] : 0;
            if (fib < banks)
            {
                std::vector<int> hreal((size_t)nodes);
                cuda_check(cudaMemcpy(hreal.data(), d_node_real, sizeof(int) * nodes, cudaMemcpyDeviceToHost), "real");
                int rc_l[MAX_COARSE];
                bool ok = true;
                for (int l = 0; l < M.level_num && ok; ++l)
                {
                    int first_iso = 1 << 30, last_real = -1;
                    for (int u = 0; u < nodes; ++u)
                    {
                        if (!hreal[u])
                            continue;
                        const int c = hmap[(size_t)u * 4 + l];
                        if ((u >> 5) >= fib)
                            first_iso = std::min(first_iso, c);
                        else
                            last_real = std::max(last_real, c);
                    }
                    ok = last_real < first_iso;
                    rc_l[l] = first_iso;
                }
                if (ok)
                    for (int l = 0; l < M.level_num; ++l)
                        M.real_count[l] = rc_l[l];
                else
                    fib = banks;
            }
            M.first_iso_bank = fib;
            std::vector<int> active;
            for (int l = 0; l < M.level_num; ++l)
            {
                const int need = div_up(M.real_count[l], 32);
                for (int g = 0; g < need; ++g)
                    active.push_back(M.mat_offsets[l + 1] - banks + g);
            }
            M.n_coarse_active = (int)active.size();
            M.coarse_active.alloc(active.empty() ? 1 : active.size(), "MAS coarse_space active");
            if (!active.empty())
                cuda_check(cudaMemcpy(M.coarse_active.get(), active.data(), active.size() * sizeof(int),
                                      cudaMemcpyHostToDevice),
                           "active");
            M.parent.alloc(cn > 0 ? cn : 1, "MAS coarse_space parents");
            if (cn > 0)
                cuda_check(cudaMemcpy(M.parent.get(), parent.data(), (size_t)cn * sizeof(int), cudaMemcpyHostToDevice),
                           "parents");
            M.ticket.alloc(1, "MAS coarse_space ticket");
            cuda_check(cudaMemsetAsync(M.ticket.get(), 0, sizeof(unsigned), s), "memset");
            // Children lists (local ids) of the real nodes of levels 1..level_num-1.
            {
                std::vector<int> ptr_all, kid;
                for (int l = 0; l < MAX_COARSE; ++l)
                    M.kid_ptr_off[l] = 0;
                for (int l = 1; l < M.level_num; ++l)
                {
                    std::vector<std::vector<int>> ch((size_t)M.real_count[l]);
                    for (int i = 0; i < M.real_count[l - 1]; ++i)
                    {
                        const int pa = parent[(size_t)coff[l - 1] + i];
                        if (pa >= 0 && pa - coff[l] < M.real_count[l])
                            ch[(size_t)(pa - coff[l])].push_back(i);
                    }
                    M.kid_ptr_off[l] = (int)ptr_all.size();
                    ptr_all.push_back((int)kid.size());
                    for (auto &c : ch)
                    {
                        if (c.size() > 32)
                            throw Error(ERR_INVALID, "[MAS] internal: coarse node with more than 32 children");
                        kid.insert(kid.end(), c.begin(), c.end());
                        ptr_all.push_back((int)kid.size());
                    }
                }
                M.kid_ptr_all.alloc(ptr_all.empty() ? 1 : ptr_all.size(), "MAS coarse_space children");
                M.kids.alloc(kid.empty() ? 1 : kid.size(), "MAS coarse_space children");
                if (!ptr_all.empty())
                    cuda_check(cudaMemcpy(M.kid_ptr_all.get(), ptr_all.data(), ptr_all.size() * sizeof(int),
                                          cudaMemcpyHostToDevice),
                               "children");
                if (!kid.empty())
                    cuda_check(cudaMemcpy(M.kids.get(), kid.data(), kid.size() * sizeof(int), cudaMemcpyHostToDevice),
                               "children");
            }
        }

        // Coarse vectors (zero once: slots past the component counts stay zero).
        M.rc.alloc((size_t)(cn > 0 ? cn : 1) * bd, "MAS coarse_vectors r");
        M.zc.alloc((size_t)(cn > 0 ? cn : 1) * bd, "MAS coarse_vectors z");
        cuda_check(cudaMemsetAsync(M.rc.get(), 0, M.rc.bytes(), s), "memset");
        cuda_check(cudaMemsetAsync(M.zc.get(), 0, M.zc.bytes(), s), "memset");

        build_coarse_sums(M, A, d_node_real, s);
        build_inverses(M, A, d_node_real, storage, coff, s);
    }

    void refresh_mas_values(MasDevice &M, const BankedMatrix &A, const int *d_node_real, int storage, cudaStream_t s)
    {
        if (M.bd != A.bd || M.banks != A.banks || M.nodes != A.nodes)
            throw Error(ERR_INVALID, "[MAS] internal: refresh with a different pattern");
        build_inverses(M, A, d_node_real, storage, M.coff, s);
    }
} // namespace pmas
