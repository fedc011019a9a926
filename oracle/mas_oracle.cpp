// ORACLE — test infrastructure only. Not part of the product, never linked into it.
//
// A CPU restatement, in plain C++ with OpenMP, of polysolve's MAS-preconditioned CG
// (src/polysolve/linear/MASSolver.cu and src/polysolve/linear/mas_utils/*). It is used by
// tests/ (as the checker), by __graft_entry__.smoke() and by bench.py's CPU baseline legs.
//
// Parity status: parity unpinned. The reference's CUDA path cannot be compiled in this image
// (it needs CCCL 3.3 headers, Eigen, KaMinPar, spdlog, jse), and the reference's tests hold no
// golden vectors for MAS (only residual thresholds on data that is not shipped). This file
// follows the reference's semantics step by step; each function cites what it restates.
//
// Given the same block permutation and partition offsets, the integer structures (BSR pattern,
// padded maps, coarse-space maps, level counts) are exact, and the floating-point results agree
// up to summation order (the reference sums with FP64 atomics in nondeterministic order).
//
// Conventions (as in the reference):
//   perm[old_block] = new_block (partition-sorted), block rows of one partition contiguous;
//   part_offsets[P+1] CSR-style; vectors inside the solver are in new (permuted) block order.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <string>
#include <vector>
#include <omp.h>

namespace
{
    constexpr int BANK = 32;            // MASPreconditioner.cu:33
    constexpr int MAX_COARSE = 4;       // MASPreconditioner.hpp:11
    constexpr int LEVELS = MAX_COARSE + 1;

    inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

    inline int popc(uint32_t x) { return __builtin_popcount(x); }
    inline int ctz(uint32_t x) { return __builtin_ctz(x); }

    // Packed upper row-major index (MASPreconditioner.cu:484-491).
    inline long long upper_index(int dim, int i, int j)
    {
        if (i > j)
            std::swap(i, j);
        return (long long)i * dim - (long long)i * (i + 1) / 2 + j;
    }

    struct Oracle
    {
        // BSR in permuted block order (BSRMatrix.cu:195-430).
        int n = 0;      // scalar rows of A
        int bd = 1;     // block dim
        int V = 0;      // block rows
        int nnzb = 0;
        std::vector<int> rows, cols;
        std::vector<double> vals;
        std::vector<int> perm, inv_perm;
        std::vector<int> part_offsets;

        // Padded topology (MASPreconditioner.cu:58-110, 1003-1049).
        int P = 0, padded = 0;
        std::vector<int> r2p, p2r;

        // Coarse space (MASPreconditioner.cu:376-481).
        std::vector<int> map; // V * MAX_COARSE
        int cco_nums[MAX_COARSE] = {0, 0, 0, 0};
        int level_num = 0;

        // Coarse matrices (MASPreconditioner.cu:939-979).
        int mat_dim = 0;
        long long storage = 0;
        int mat_offsets[LEVELS] = {0}, mat_counts[LEVELS] = {0};
        int total_mats = 0;
        std::vector<double> mats; // inverses, packed upper
        int level_offsets[LEVELS] = {0}, level_sizes[LEVELS] = {0};
        int total_level_nodes = 0;
        bool inverse_ok = true;

        std::string error;
    };

    // ------------------------------------------------------------------------------------
    // CSC -> permuted BSR (BSRMatrix.cu:91-135 keys, 165-193 fill, trailing pad = 1.0).
    // ------------------------------------------------------------------------------------
    bool build_bsr(Oracle &o, int n, const int *outer, const int *inner, const double *vals, int bd,
                   const int *perm)
    {
        o.n = n;
        o.bd = bd;
        o.V = div_up(n, bd);
        const int padded_scalars = bd * o.V - n;
        o.perm.assign(perm, perm + o.V);
        o.inv_perm.assign(o.V, -1);
        for (int i = 0; i < o.V; ++i)
        {
            if (perm[i] < 0 || perm[i] >= o.V || o.inv_perm[perm[i]] != -1)
            {
                o.error = "invalid permutation";
                return false;
            }
            o.inv_perm[perm[i]] = i;
        }
        // Collect (new block row, new block col, offset, value) per entry; the trailing block's
        // missing diagonal entries are padded with 1.0.
        struct E
        {
            uint64_t key;
            int off;
            double v;
        };
        std::vector<std::vector<E>> per_row(o.V);
        for (int col = 0; col < n; ++col)
            for (int k = outer[col]; k < outer[col + 1]; ++k)
            {
                int row = inner[k];
                int bro = row / bd, bco = col / bd;
                int br = perm[bro], bc = perm[bco];
                int off = (row - bro * bd) * bd + (col - bco * bd);
                per_row[br].push_back(E{(uint64_t)(uint32_t)bc, off, vals[k]});
            }
        if (padded_scalars > 0)
        {
            int tail = perm[o.V - 1];
            for (int t = 0; t < padded_scalars; ++t)
            {
                int local = (bd - padded_scalars) + t;
                per_row[tail].push_back(E{(uint64_t)(uint32_t)tail, local * bd + local, 1.0});
            }
        }
        o.rows.assign(o.V + 1, 0);
        for (int r = 0; r < o.V; ++r)
        {
            auto &lst = per_row[r];
            std::stable_sort(lst.begin(), lst.end(), [](const E &a, const E &b) { return a.key < b.key; });
            int uniq = 0;
            for (size_t i = 0; i < lst.size(); ++i)
                if (i == 0 || lst[i].key != lst[i - 1].key)
                    ++uniq;
            o.rows[r + 1] = o.rows[r] + uniq;
        }
        o.nnzb = o.rows[o.V];
        o.cols.assign(o.nnzb, 0);
        o.vals.assign((size_t)o.nnzb * bd * bd, 0.0);
        for (int r = 0; r < o.V; ++r)
        {
            auto &lst = per_row[r];
            int b = o.rows[r] - 1;
            for (size_t i = 0; i < lst.size(); ++i)
            {
                if (i == 0 || lst[i].key != lst[i - 1].key)
                {
                    ++b;
                    o.cols[b] = (int)lst[i].key;
                }
                o.vals[(size_t)b * bd * bd + lst[i].off] = lst[i].v;
            }
            std::vector<E>().swap(lst);
        }
        return true;
    }

    // ------------------------------------------------------------------------------------
    // Padded maps (MASPreconditioner.cu:58-88).
    // ------------------------------------------------------------------------------------
    void build_padded(Oracle &o)
    {
        o.P = (int)o.part_offsets.size() - 1;
        o.padded = o.P * BANK;
        o.r2p.assign(o.V, -1);
        o.p2r.assign(o.padded, -1);
        for (int p = 0; p < o.P; ++p)
        {
            int b = o.part_offsets[p], e = o.part_offsets[p + 1];
            for (int l = 0; l < e - b; ++l)
            {
                o.r2p[b + l] = p * BANK + l;
                o.p2r[p * BANK + l] = b + l;
            }
        }
    }

    // Bank-local connected components of 32 nodes given neighbour masks (self bit included):
    // closure of each mask, lead = lowest lane of the component, local id = rank of the lead.
    // MASPreconditioner.cu:189-212 (lv0) and :294-317 (lvx). valid marks lanes that exist.
    void bank_components(const uint32_t *nbr, uint32_t valid, int *local_id, int &count)
    {
        uint32_t conn[BANK];
        uint32_t leads = 0;
        for (int l = 0; l < BANK; ++l)
        {
            if (!((valid >> l) & 1u))
                continue;
            uint32_t c = nbr[l];
            uint32_t visited = 1u << l;
            uint32_t todo = c ^ visited;
            while (todo)
            {
                int v = ctz(todo);
                c |= nbr[v];
                visited |= 1u << v;
                todo = c ^ visited;
            }
            conn[l] = c;
            if (ctz(c) == l)
                leads |= 1u << l;
        }
        for (int l = 0; l < BANK; ++l)
        {
            if (!((valid >> l) & 1u))
            {
                local_id[l] = -1;
                continue;
            }
            int lead = ctz(conn[l]);
            uint32_t before = (uint32_t)((1ull << lead) - 1ull);
            local_id[l] = popc(leads & before);
        }
        count = popc(leads);
    }

    // ------------------------------------------------------------------------------------
    // Coarse space hierarchy (MASPreconditioner.cu:128-481). Neighbour lists are not compacted
    // here; compaction in the reference only removes neighbours that already share the CCO.
    // ------------------------------------------------------------------------------------
    void build_coarse_space(Oracle &o)
    {
        o.map.assign((size_t)o.V * MAX_COARSE, 0);
        for (int &c : o.cco_nums)
            c = 0;
        // Level 0: components inside each partition bank.
        std::vector<int> cnt(o.P, 0), local(o.padded, -1);
        for (int b = 0; b < o.P; ++b)
        {
            uint32_t nbr[BANK] = {0};
            uint32_t valid = 0;
            for (int l = 0; l < BANK; ++l)
            {
                int rid = o.p2r[b * BANK + l];
                if (rid < 0)
                    continue;
                valid |= 1u << l;
                uint32_t m = 1u << l;
                for (int k = o.rows[rid]; k < o.rows[rid + 1]; ++k)
                {
                    int pj = o.r2p[o.cols[k]];
                    if (pj / BANK == b)
                        m |= 1u << (pj % BANK);
                }
                nbr[l] = m;
            }
            bank_components(nbr, valid, &local[b * BANK], cnt[b]);
        }
        std::vector<int> excl(o.P + 1, 0);
        for (int b = 0; b < o.P; ++b)
            excl[b + 1] = excl[b] + cnt[b];
        for (int r = 0; r < o.V; ++r)
        {
            int p = o.r2p[r];
            o.map[(size_t)r * MAX_COARSE] = local[p] + excl[p / BANK];
        }
        int cco_num = excl[o.P];
        o.cco_nums[0] = cco_num;
        o.level_num = 1;

        for (int lv = 1; lv < MAX_COARSE; ++lv)
        {
            std::vector<uint32_t> nbr(cco_num, 0);
            for (int r = 0; r < o.V; ++r)
            {
                int c = o.map[(size_t)r * MAX_COARSE + lv - 1];
                uint32_t m = 1u << (c % BANK);
                for (int k = o.rows[r]; k < o.rows[r + 1]; ++k)
                {
                    int cj = o.map[(size_t)o.cols[k] * MAX_COARSE + lv - 1];
                    if (c / BANK == cj / BANK)
                        m |= 1u << (cj % BANK);
                }
                nbr[c] |= m;
            }
            int banks = div_up(cco_num, BANK);
            std::vector<int> bcnt(banks, 0), blocal((size_t)banks * BANK, -1);
            for (int b = 0; b < banks; ++b)
            {
                uint32_t valid = 0;
                uint32_t m[BANK] = {0};
                for (int l = 0; l < BANK; ++l)
                {
                    int c = b * BANK + l;
                    if (c < cco_num)
                    {
                        valid |= 1u << l;
                        m[l] = nbr[c];
                    }
                }
                bank_components(m, valid, &blocal[(size_t)b * BANK], bcnt[b]);
            }
            std::vector<int> bex(banks + 1, 0);
            for (int b = 0; b < banks; ++b)
                bex[b + 1] = bex[b] + bcnt[b];
            for (int r = 0; r < o.V; ++r)
            {
                int prev = o.map[(size_t)r * MAX_COARSE + lv - 1];
                o.map[(size_t)r * MAX_COARSE + lv] = blocal[prev] + bex[prev / BANK];
            }
            int next = bex[banks];
            if (next == cco_num)
                break; // MASPreconditioner.cu:464-469
            cco_num = next;
            o.cco_nums[lv] = cco_num;
            o.level_num = lv + 1;
        }
    }

    // ------------------------------------------------------------------------------------
    // Coarse matrices: accumulate upper triangles, pad zero diagonals, sweep inverse
    // (MASPreconditioner.cu:494-591, 779-900, 939-979).
    // ------------------------------------------------------------------------------------
    void add_block(Oracle &o, double *mat, int ri, int rj, bool diag_block, bool collapsed, const double *blk)
    {
        const int bd = o.bd;
        for (int bi = 0; bi < bd; ++bi)
            for (int bj = 0; bj < bd; ++bj)
            {
                int row = ri * bd + bi, col = rj * bd + bj;
                if (row > col)
                    continue;
                if (diag_block && bi > bj)
                    continue;
                double v = blk[bi * bd + bj];
                if (collapsed)
                    v += blk[bj * bd + bi];
                mat[upper_index(o.mat_dim, row, col)] += v;
            }
    }

    // Symmetric Gauss-Jordan sweep on one packed matrix; returns false on a zero or non-finite
    // pivot or a non-finite update (MASPreconditioner.cu:799-900).
    bool sweep_invert(double *A, int N)
    {
        bool ok = true;
        std::vector<double> col(N);
        for (int pv = 0; pv < N; ++pv)
        {
            double piv = A[upper_index(N, pv, pv)];
            if (!std::isfinite(piv) || piv == 0.0)
                ok = false;
            for (int t = 0; t < N; ++t)
                col[t] = (t == pv) ? 0.0 : A[upper_index(N, t, pv)];
            for (int t = 0; t < N; ++t)
            {
                if (t == pv)
                    continue;
                double scale = col[t] / piv;
                for (int c = t; c < N; ++c)
                {
                    if (c == pv)
                        continue;
                    double u = A[upper_index(N, t, c)] - scale * col[c];
                    if (!std::isfinite(u))
                        ok = false;
                    A[upper_index(N, t, c)] = u;
                }
            }
            for (int t = 0; t < N; ++t)
            {
                double u = (t == pv) ? -1.0 / piv : col[t] / piv;
                if (!std::isfinite(u))
                    ok = false;
                else
                    A[upper_index(N, t, pv)] = u;
            }
        }
        const long long S = (long long)N * (N + 1) / 2;
        for (long long i = 0; i < S; ++i)
        {
            A[i] = -A[i];
            if (!std::isfinite(A[i]))
                ok = false;
        }
        return ok;
    }

    void build_matrices(Oracle &o)
    {
        o.mat_dim = BANK * o.bd;
        o.storage = (long long)o.mat_dim * (o.mat_dim + 1) / 2;
        for (int i = 0; i < LEVELS; ++i)
            o.mat_offsets[i] = o.mat_counts[i] = 0;
        o.mat_counts[0] = o.P;
        o.total_mats = o.P;
        for (int i = 0; i < o.level_num; ++i)
        {
            o.mat_offsets[i + 1] = o.total_mats;
            o.mat_counts[i + 1] = div_up(o.cco_nums[i], BANK);
            o.total_mats += o.mat_counts[i + 1];
        }
        o.mats.assign((size_t)o.total_mats * o.storage, 0.0);
        const int bs = o.bd * o.bd;
        // Level 0 (padded banks) in parallel over banks: a bank's rows are contiguous.
#pragma omp parallel for schedule(dynamic, 16)
        for (int p = 0; p < o.P; ++p)
        {
            double *mat = o.mats.data() + (size_t)p * o.storage;
            for (int tid = o.part_offsets[p]; tid < o.part_offsets[p + 1]; ++tid)
            {
                int pi = o.r2p[tid];
                for (int k = o.rows[tid]; k < o.rows[tid + 1]; ++k)
                {
                    int j = o.cols[k];
                    if (tid > j)
                        continue;
                    int pj = o.r2p[j];
                    if (pi / BANK != pj / BANK)
                        continue;
                    add_block(o, mat, pi % BANK, pj % BANK, tid == j, false, &o.vals[(size_t)k * bs]);
                }
            }
        }
        // Coarse levels, serially in row order.
        for (int tid = 0; tid < o.V; ++tid)
            for (int k = o.rows[tid]; k < o.rows[tid + 1]; ++k)
            {
                int j = o.cols[k];
                if (tid > j)
                    continue;
                for (int lv = 0; lv < o.level_num; ++lv)
                {
                    int ci = o.map[(size_t)tid * MAX_COARSE + lv];
                    int cj = o.map[(size_t)j * MAX_COARSE + lv];
                    if (ci / BANK != cj / BANK)
                        continue;
                    double *mat = o.mats.data() + (size_t)(o.mat_offsets[lv + 1] + ci / BANK) * o.storage;
                    add_block(o, mat, ci % BANK, cj % BANK, tid == j, tid != j && ci == cj,
                              &o.vals[(size_t)k * bs]);
                }
            }
        // Pad zero diagonals, then invert every matrix.
        int fails = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : fails)
        for (int m = 0; m < o.total_mats; ++m)
        {
            double *mat = o.mats.data() + (size_t)m * o.storage;
            for (int r = 0; r < o.mat_dim; ++r)
            {
                double &d = mat[upper_index(o.mat_dim, r, r)];
                if (d == 0.0)
                    d = 1.0;
            }
            if (!sweep_invert(mat, o.mat_dim))
                ++fails;
        }
        o.inverse_ok = (fails == 0);
        // Multi-level vector layout (MASPreconditioner.cu:1078-1086).
        for (int i = 0; i < LEVELS; ++i)
            o.level_offsets[i] = o.level_sizes[i] = 0;
        o.level_sizes[0] = o.padded;
        o.total_level_nodes = o.padded;
        for (int i = 0; i < o.level_num; ++i)
        {
            o.level_offsets[i + 1] = o.total_level_nodes;
            o.level_sizes[i + 1] = o.mat_counts[i + 1] * BANK;
            o.total_level_nodes += o.level_sizes[i + 1];
        }
    }

    // ------------------------------------------------------------------------------------
    // Apply z = sum_l P_l A_l^-1 P_l^T r (MASPreconditioner.cu:593-777, 1099-1164).
    // ------------------------------------------------------------------------------------
    void mas_apply(const Oracle &o, const double *r, double *z)
    {
        const int bd = o.bd;
        const size_t total = (size_t)o.total_level_nodes * bd;
        std::vector<double> mlr(total, 0.0), mlz(total, 0.0);
        for (int p = 0; p < o.padded; ++p)
        {
            int rid = o.p2r[p];
            if (rid < 0)
                continue;
            for (int i = 0; i < bd; ++i)
                mlr[(size_t)p * bd + i] = r[(size_t)rid * bd + i];
        }
        for (int rid = 0; rid < o.V; ++rid)
            for (int lv = 0; lv < o.level_num; ++lv)
            {
                int c = o.map[(size_t)rid * MAX_COARSE + lv];
                for (int i = 0; i < bd; ++i)
                    mlr[(size_t)(o.level_offsets[lv + 1] + c) * bd + i] += r[(size_t)rid * bd + i];
            }
        const int N = o.mat_dim;
#pragma omp parallel for schedule(static)
        for (int m = 0; m < o.total_mats; ++m)
        {
            const double *A = o.mats.data() + (size_t)m * o.storage;
            const double *x = mlr.data() + (size_t)m * N;
            double *y = mlz.data() + (size_t)m * N;
            for (int row = 0; row < N; ++row)
            {
                double s = 0.0;
                for (int c = 0; c < N; ++c)
                    s += A[upper_index(N, row, c)] * x[c];
                y[row] = s;
            }
        }
#pragma omp parallel for schedule(static)
        for (int rid = 0; rid < o.V; ++rid)
        {
            int p = o.r2p[rid];
            for (int i = 0; i < bd; ++i)
                z[(size_t)rid * bd + i] = mlz[(size_t)p * bd + i];
            for (int lv = 0; lv < o.level_num; ++lv)
            {
                int c = o.map[(size_t)rid * MAX_COARSE + lv];
                for (int i = 0; i < bd; ++i)
                    z[(size_t)rid * bd + i] += mlz[(size_t)(o.level_offsets[lv + 1] + c) * bd + i];
            }
        }
    }

    void spmv(const Oracle &o, const double *x, double *y)
    {
        const int bd = o.bd, bs = bd * bd;
#pragma omp parallel for schedule(static)
        for (int r = 0; r < o.V; ++r)
        {
            double acc[3] = {0, 0, 0};
            for (int k = o.rows[r]; k < o.rows[r + 1]; ++k)
            {
                const double *b = &o.vals[(size_t)k * bs];
                const double *xc = x + (size_t)o.cols[k] * bd;
                for (int i = 0; i < bd; ++i)
                    for (int j = 0; j < bd; ++j)
                        acc[i] += b[i * bd + j] * xc[j];
            }
            for (int i = 0; i < bd; ++i)
                y[(size_t)r * bd + i] = acc[i];
        }
    }

    // Round a float to the nearest IEEE binary16 value (round to nearest even), returned as float.
    // Normal results keep 11 significant bits; below 2^-14 the step is the subnormal 2^-24.
    float half_round(float f)
    {
        if (!std::isfinite(f) || f == 0.0f)
            return f;
        int e;
        std::frexp(f, &e); // f = m 2^e, 0.5 <= |m| < 1
        const float q = std::ldexp(1.0f, std::max(e - 11, -24));
        const float r = std::nearbyint(f / q) * q;
        return std::fabs(r) > 65504.0f ? std::copysign(INFINITY, f) : r; // past the largest finite value
    }

    // Emulates storing the inverses in reduced precision (values rounded in place, arithmetic
    // stays FP64): mode 1 = FP32; mode 16 = binary16 with one power-of-two scale per matrix that
    // maps its largest magnitude into [2^14, 2^15).
    void round_storage(Oracle &o, int mode)
    {
        if (mode == 16)
        {
            for (int m = 0; m < o.total_mats; ++m)
            {
                double *mat = o.mats.data() + (size_t)m * o.storage;
                double amax = 0.0;
                for (long long i = 0; i < o.storage; ++i)
                    amax = std::max(amax, std::fabs(mat[i]));
                const double sc = (amax > 0.0 && std::isfinite(amax)) ? std::ldexp(1.0, 14 - std::ilogb(amax)) : 1.0;
                for (long long i = 0; i < o.storage; ++i)
                    mat[i] = (double)half_round((float)(mat[i] * sc)) / sc;
            }
        }
        else if (mode)
            for (double &v : o.mats)
                v = (double)(float)v;
    }

    // Deterministic dot: fixed chunks, summed in chunk order.
    double dot(const double *a, const double *b, size_t n)
    {
        const int chunks = 64;
        double part[chunks];
#pragma omp parallel for schedule(static)
        for (int c = 0; c < chunks; ++c)
        {
            size_t lo = n * c / chunks, hi = n * (c + 1) / chunks;
            double s = 0.0;
            for (size_t i = lo; i < hi; ++i)
                s += a[i] * b[i];
            part[c] = s;
        }
        double s = 0.0;
        for (int c = 0; c < chunks; ++c)
            s += part[c];
        return s;
    }
} // namespace

extern "C"
{
    struct orc_pcg_params
    {
        int max_iter;
        double rel_tol;
        double abs_tol;
        int use_preconditioned_residual_norm;
        int true_residual_period; // reference: 4 (MASSolver.cu:139)
        int check_period;         // reference: 10 (MASSolver.cu:533)
        int use_initial_guess;    // reference: 0, x forced to zero (MASSolver.cu:395-398)
        int mas_fp32;             // emulate inverse storage: 1 = FP32, 16 = FP16 with a per-matrix scale
        int polak_ribiere;        // beta = r.(z - z_old) / rz_old instead of rz / rz_old
    };

    struct orc_pcg_result
    {
        int iterations;
        int status; // 0 running, 1 rel tol, 2 abs tol, 3 max iterations, -1 invalid initial residual
        double residual_norm;
        double rz0, rr0;
    };

    void *orc_create(int n, const int *outer, const int *inner, const double *vals, int bd, const int *perm,
                     int nparts, const int *part_offsets)
    {
        if (n <= 0 || bd < 1 || bd > 3 || nparts < 1)
            return nullptr;
        auto *o = new Oracle();
        if (!build_bsr(*o, n, outer, inner, vals, bd, perm))
        {
            delete o;
            return nullptr;
        }
        o->part_offsets.assign(part_offsets, part_offsets + nparts + 1);
        if (o->part_offsets.back() != o->V)
        {
            delete o;
            return nullptr;
        }
        for (int p = 0; p < nparts; ++p)
            if (o->part_offsets[p + 1] - o->part_offsets[p] > BANK || o->part_offsets[p + 1] < o->part_offsets[p])
            {
                delete o;
                return nullptr;
            }
        build_padded(*o);
        build_coarse_space(*o);
        build_matrices(*o);
        return o;
    }

    void orc_free(void *h) { delete static_cast<Oracle *>(h); }

    int orc_inverse_ok(void *h) { return static_cast<Oracle *>(h)->inverse_ok ? 1 : 0; }

    int orc_sizes(void *h, int *out /* V, nnzb, P, padded, level_num, total_mats, mat_dim, total_level_nodes */)
    {
        auto *o = static_cast<Oracle *>(h);
        out[0] = o->V;
        out[1] = o->nnzb;
        out[2] = o->P;
        out[3] = o->padded;
        out[4] = o->level_num;
        out[5] = o->total_mats;
        out[6] = o->mat_dim;
        out[7] = o->total_level_nodes;
        return 0;
    }

    int orc_levels(void *h, int *cco_nums /*4*/, int *mat_counts /*5*/, int *mat_offsets /*5*/, int *level_offsets /*5*/)
    {
        auto *o = static_cast<Oracle *>(h);
        for (int i = 0; i < MAX_COARSE; ++i)
            cco_nums[i] = o->cco_nums[i];
        for (int i = 0; i < LEVELS; ++i)
        {
            mat_counts[i] = o->mat_counts[i];
            mat_offsets[i] = o->mat_offsets[i];
            level_offsets[i] = o->level_offsets[i];
        }
        return 0;
    }

    int orc_export_bsr(void *h, int *rows, int *cols, double *vals)
    {
        auto *o = static_cast<Oracle *>(h);
        std::memcpy(rows, o->rows.data(), o->rows.size() * sizeof(int));
        std::memcpy(cols, o->cols.data(), o->cols.size() * sizeof(int));
        std::memcpy(vals, o->vals.data(), o->vals.size() * sizeof(double));
        return 0;
    }

    int orc_export_maps(void *h, int *r2p, int *map)
    {
        auto *o = static_cast<Oracle *>(h);
        std::memcpy(r2p, o->r2p.data(), o->r2p.size() * sizeof(int));
        std::memcpy(map, o->map.data(), o->map.size() * sizeof(int));
        return 0;
    }

    int orc_export_inverses(void *h, double *out)
    {
        auto *o = static_cast<Oracle *>(h);
        std::memcpy(out, o->mats.data(), o->mats.size() * sizeof(double));
        return 0;
    }

    // Vectors in permuted block order (V * bd).
    int orc_apply(void *h, const double *r, double *z)
    {
        mas_apply(*static_cast<Oracle *>(h), r, z);
        return 0;
    }

    // out[i] = half_round(in[i]) (checks the binary16 rounding against IEEE conversions).
    int orc_half_round(const float *in, float *out, long long n)
    {
        for (long long i = 0; i < n; ++i)
            out[i] = half_round(in[i]);
        return 0;
    }

    // z = M^-1 r with the inverses stored as in round_storage(mode) (0 = FP64).
    int orc_apply_storage(void *h, const double *r, double *z, int mode)
    {
        auto *o = static_cast<Oracle *>(h);
        if (mode == 0)
        {
            mas_apply(*o, r, z);
            return 0;
        }
        const std::vector<double> saved = o->mats;
        round_storage(*o, mode);
        mas_apply(*o, r, z);
        o->mats = saved;
        return 0;
    }

    int orc_spmv(void *h, const double *x, double *y)
    {
        spmv(*static_cast<Oracle *>(h), x, y);
        return 0;
    }

    // MAS-PCG, restating MASSolverImpl::solve + pcg_solve (MASSolver.cu:376-409, 469-595).
    // b and x are in the caller's (original) order, length n.
    int orc_pcg(void *h, const double *b_in, double *x_io, const orc_pcg_params *pp, orc_pcg_result *res)
    {
        auto *o = static_cast<Oracle *>(h);
        const orc_pcg_params p = *pp;
        const int bd = o->bd;
        const size_t N = (size_t)o->V * bd;
        std::vector<double> b(N, 0.0), x(N, 0.0), r(N), z(N), pv(N), Ap(N), zold;
        std::vector<double> saved;
        if (p.mas_fp32)
        {
            saved = o->mats;
            round_storage(*o, p.mas_fp32);
        }
        // Permute b (and x) into block order; pad with zeros (MASSolver.cu:387-393).
        for (size_t nb = 0; nb < (size_t)o->V; ++nb)
            for (int c = 0; c < bd; ++c)
            {
                size_t src = (size_t)o->inv_perm[nb] * bd + c;
                b[nb * bd + c] = src < (size_t)o->n ? b_in[src] : 0.0;
                if (p.use_initial_guess)
                    x[nb * bd + c] = src < (size_t)o->n ? x_io[src] : 0.0;
            }
        res->iterations = 0;
        res->status = 0;
        res->residual_norm = 0.0;
        // r = b - A x
        spmv(*o, x.data(), r.data());
        for (size_t i = 0; i < N; ++i)
            r[i] = b[i] - r[i];
        mas_apply(*o, r.data(), z.data());
        pv = z;
        double rz = dot(r.data(), z.data(), N);
        const double rz0 = rz;
        res->rz0 = rz0;
        if (std::isnan(rz0) || !std::isfinite(rz0))
        {
            res->status = -1;
            if (p.mas_fp32)
                o->mats = saved;
            return 1;
        }
        // rr0 = ||b||^2: the reference computes r.r with x = 0 (MASSolver.cu:488-494), which is
        // ||b||^2; with an initial guess "relative" stays relative to ||b||.
        double rr0 = 0.0;
        if (!p.use_preconditioned_residual_norm)
            rr0 = dot(b.data(), b.data(), N);
        res->rr0 = rr0;
        if (p.polak_ribiere)
            zold = z;
        int iters = 0;
        for (int k = 1; k <= p.max_iter; ++k)
        {
            spmv(*o, pv.data(), Ap.data());
            double pAp = dot(pv.data(), Ap.data(), N);
            double alpha = (std::fabs(pAp) < 1e-20) ? 0.0 : rz / pAp;
            for (size_t i = 0; i < N; ++i)
                x[i] += alpha * pv[i];
            if (k % p.true_residual_period == 0)
            {
                spmv(*o, x.data(), r.data());
                for (size_t i = 0; i < N; ++i)
                    r[i] = b[i] - r[i];
            }
            else
            {
                for (size_t i = 0; i < N; ++i)
                    r[i] -= alpha * Ap[i];
            }
            mas_apply(*o, r.data(), z.data());
            double rz_old = rz;
            rz = dot(r.data(), z.data(), N);
            iters = k;
            bool conv = false;
            if (k % p.check_period == 0)
            {
                if (p.use_preconditioned_residual_norm)
                {
                    res->residual_norm = std::sqrt(rz);
                    if (rz <= p.rel_tol * p.rel_tol * rz0 || rz <= p.abs_tol * p.abs_tol)
                    {
                        res->status = (rz <= p.abs_tol * p.abs_tol) ? 2 : 1;
                        conv = true;
                    }
                }
                else
                {
                    double rr = dot(r.data(), r.data(), N);
                    res->residual_norm = std::sqrt(rr);
                    if (rr <= p.rel_tol * p.rel_tol * rr0 || rr <= p.abs_tol * p.abs_tol)
                    {
                        res->status = (rr <= p.abs_tol * p.abs_tol) ? 2 : 1;
                        conv = true;
                    }
                }
            }
            if (conv)
                break;
            double beta;
            if (p.polak_ribiere)
            {
                double rzo = 0.0;
                rzo = dot(r.data(), zold.data(), N);
                double num = rz - rzo;
                beta = (std::fabs(rz_old) < 1e-20) ? 0.0 : num / rz_old;
                if (beta < 0.0)
                    beta = 0.0;
                zold = z;
            }
            else
                beta = (std::fabs(rz_old) < 1e-20) ? 0.0 : rz / rz_old;
            for (size_t i = 0; i < N; ++i)
                pv[i] = z[i] + beta * pv[i];
        }
        if (p.max_iter >= 1)
            res->iterations = iters;
        if (res->iterations == p.max_iter)
            res->status = 3;
        for (size_t ob = 0; ob < (size_t)o->V; ++ob)
            for (int c = 0; c < bd; ++c)
            {
                size_t dst = ob * bd + c;
                if (dst < (size_t)o->n)
                    x_io[dst] = x[(size_t)o->perm[ob] * bd + c];
            }
        if (p.mas_fp32)
            o->mats = saved;
        return 0;
    }

    // Jacobi-preconditioned CG, restating the algorithm of Eigen::ConjugateGradient with its
    // default DiagonalPreconditioner (the reference's CPU CG path, Solver.cpp:294-303,
    // 436-438): stop when ||r||^2 < tol^2 ||b||^2. CSC of a symmetric matrix = its CSR.
    int orc_jacobi_pcg(int n, const int *outer, const int *inner, const double *vals, const double *b,
                       double *x, double tol, int max_iter, int *iters_out, double *relres_out)
    {
        std::vector<double> invd(n, 1.0), r(n), z(n), p(n), Ap(n);
        for (int c = 0; c < n; ++c)
            for (int k = outer[c]; k < outer[c + 1]; ++k)
                if (inner[k] == c && vals[k] != 0.0)
                    invd[c] = 1.0 / vals[k];
        auto matvec = [&](const double *in, double *out) {
#pragma omp parallel for schedule(static)
            for (int rr = 0; rr < n; ++rr)
            {
                double s = 0.0;
                for (int k = outer[rr]; k < outer[rr + 1]; ++k)
                    s += vals[k] * in[inner[k]];
                out[rr] = s;
            }
        };
        matvec(x, Ap.data());
        for (int i = 0; i < n; ++i)
            r[i] = b[i] - Ap[i];
        double bn2 = dot(b, b, n);
        if (bn2 == 0.0)
        {
            std::fill(x, x + n, 0.0);
            *iters_out = 0;
            *relres_out = 0.0;
            return 0;
        }
        double thr = std::max(tol * tol * bn2, std::numeric_limits<double>::min());
        double rn2 = dot(r.data(), r.data(), n);
        if (rn2 < thr)
        {
            *iters_out = 0;
            *relres_out = std::sqrt(rn2 / bn2);
            return 0;
        }
        for (int i = 0; i < n; ++i)
            p[i] = invd[i] * r[i];
        double absNew = dot(r.data(), p.data(), n);
        int i = 0;
        while (i < max_iter)
        {
            matvec(p.data(), Ap.data());
            double alpha = absNew / dot(p.data(), Ap.data(), n);
#pragma omp parallel for schedule(static)
            for (int q = 0; q < n; ++q)
            {
                x[q] += alpha * p[q];
                r[q] -= alpha * Ap[q];
            }
            rn2 = dot(r.data(), r.data(), n);
            if (rn2 < thr)
                break;
#pragma omp parallel for schedule(static)
            for (int q = 0; q < n; ++q)
                z[q] = invd[q] * r[q];
            double absOld = absNew;
            absNew = dot(r.data(), z.data(), n);
            double beta = absNew / absOld;
#pragma omp parallel for schedule(static)
            for (int q = 0; q < n; ++q)
                p[q] = z[q] + beta * p[q];
            ++i;
        }
        *iters_out = i;
        *relres_out = std::sqrt(rn2 / bn2);
        return 0;
    }
}
