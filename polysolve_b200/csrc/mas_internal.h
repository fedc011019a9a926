// Internal interfaces of the B200 MAS-PCG solver: device data layouts and the host-side launch
// functions that the .cu files define. Plain host C++ can include this file (no CUDA syntax).
//
// Numbering. The solver works in a "padded" block order: node = bank * 32 + lane. A bank is one
// 32-node subdomain of the MAS preconditioner (BANK_SIZE, mas_utils/MASPreconditioner.cu:33);
// lanes of a bank not covered by a real block row are virtual (padding) nodes with empty rows.
// Every vector inside the solver is node-major: value index = node * block_dim + component.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <cuda_runtime_api.h>

namespace pmas
{
    constexpr int BANK = 32;
    constexpr int MAX_COARSE = 4; // coarse levels (MASPreconditioner.hpp:11)
    constexpr int LEVELS = MAX_COARSE + 1;
    constexpr int RHS_GROUP = 4; // right-hand sides solved together (several-RHS solves)

    // Storage precision of the subdomain inverses. FP16 keeps one power-of-two scale per matrix
    // (largest magnitude -> [2^14, 2^15)); products are formed in FP32 and scaled back in FP64.
    enum : int
    {
        STORE_F64 = 0,
        STORE_F32 = 1,
        STORE_F16 = 2,
    };

    // Status codes (mirror include/polysolve_mas.h).
    enum : int
    {
        OK = 0,
        ERR_INVALID = 1,
        ERR_OOM = 2,
        ERR_NOT_FACTORIZED = 3,
        ERR_CUDA = 4,
        ERR_NONFINITE = 5,
        ERR_INVERSE = 6,
        ERR_TIMEOUT = 7,
        ERR_NO_DEVICE = 8,
    };

    struct Error : std::runtime_error
    {
        int code;
        Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
    };

    void cuda_check(cudaError_t e, const char *what);
    void *device_alloc(size_t bytes, const char *ctx); // throws Error(ERR_OOM) with MB figures
    void device_free(void *p);
    // Test hook: after `after` more successful device allocations the next one fails as if the
    // device were out of memory (once); negative: off.
    void set_alloc_failure(long long after);

    // Owning device buffer.
    template <class T>
    struct DevBuf
    {
        T *p = nullptr;
        size_t n = 0;
        DevBuf() = default;
        DevBuf(const DevBuf &) = delete;
        DevBuf &operator=(const DevBuf &) = delete;
        ~DevBuf() { reset(); }
        void reset()
        {
            if (p)
                device_free(p);
            p = nullptr;
            n = 0;
        }
        void alloc(size_t count, const char *ctx)
        {
            if (count == n && p)
                return;
            reset();
            if (count)
                p = static_cast<T *>(device_alloc(count * sizeof(T), ctx));
            n = count;
        }
        T *get() const { return p; }
        size_t bytes() const { return n * sizeof(T); }
    };

    // ---------------------------------------------------------------------------------------
    // Bank-sliced block matrix ("banked BSR"): every bank (32 block rows) is a slice of width
    // w_b = max row length in the bank; slot s of the slice holds the s-th block of each of the
    // 32 rows. Within a slot the bd*bd values of the 32 lanes are stored as value pairs
    // (q = 2p, 2p+1) interleaved per lane (16 B per lane, 512 B per pair plane), then the odd
    // last value (if bd*bd is odd) as a plane of 32 doubles: one warp reads a slot with
    // coalesced 128-bit loads.
    // ---------------------------------------------------------------------------------------
    struct BankedView
    {
        int bd;
        int banks;
        const long long *slice; // banks + 1, in slots
        const int *rowlen;      // nodes
        const int *cols;        // slots * 32, padded node ids
        const double *vals;     // slots * 32 * bd * bd
    };

    __host__ __device__ inline long long banked_value_index(long long slot, int lane, int q, int bd)
    {
        const int bs = bd * bd;
        const int pairs = bs / 2;
        const long long base = slot * 32LL * bs;
        if (q < 2 * pairs)
            return base + (long long)(q >> 1) * 64 + lane * 2 + (q & 1);
        return base + (long long)pairs * 64 + lane;
    }

    // ---------------------------------------------------------------------------------------
    // Subdomain matrix storage ("tile-packed"): an N x N symmetric matrix, N = 32 * bd, split
    // into bd x bd tiles of 32 x 32. For each column tile J: the off-diagonal tiles (I, J), I < J,
    // each 1024 values with element (l, j) of the tile at (j / 4) * 128 + l * 4 + j % 4; then the
    // diagonal tile's upper triangle, column j holding rows 0..j at offset j (j + 1) / 2 + l.
    // Total N (N + 1) / 2 values, the same count as the reference's packed upper storage.
    // ---------------------------------------------------------------------------------------
    __host__ __device__ inline int tile_packed_size(int bd) { return 32 * bd * (32 * bd + 1) / 2; }

    // Position of element (row, col) of the symmetric matrix in tile-packed storage.
    __host__ __device__ inline int tile_packed_index(int /*bd*/, int row, int col)
    {
        if (row > col)
        {
            int t = row;
            row = col;
            col = t;
        }
        const int I = row >> 5, J = col >> 5, l = row & 31, j = col & 31;
        int off = 0;
        for (int jj = 0; jj < J; ++jj)
            off += jj * 1024 + 528;
        if (I < J)
            return off + I * 1024 + (j >> 2) * 128 + l * 4 + (j & 3);
        return off + J * 1024 + j * (j + 1) / 2 + l;
    }

    // ---------------------------------------------------------------------------------------
    // Binary16 subdomain matrix storage ("mma16"): the N x N symmetric matrix (N = 32 * bd) in
    // 16 x 16 blocks, NS = N / 16 block rows, laid out for warp tensor-core fragments. First the
    // NS (NS - 1) / 2 blocks above the diagonal (block row R, block column S > R, row-major over
    // (R, S)), 256 values each as four 8 x 8 cores [rows 0-7 | cols 0-7], [rows 8-15 | cols 0-7],
    // [rows 0-7 | cols 8-15], [rows 8-15 | cols 8-15], each core row-major; then the NS diagonal
    // blocks, 192 values each: the two diagonal cores stored full (symmetric) and the core
    // [rows 0-7 | cols 8-15], as [D0 | C | D1]. The same blocks serve the rows below the diagonal
    // through transposed fragment loads.
    // ---------------------------------------------------------------------------------------
    __host__ __device__ inline int mma16_size(int bd)
    {
        const int ns = 2 * bd;
        return ns * (ns - 1) / 2 * 256 + ns * 192;
    }

    // Element of mma16 position idx (the row <= col one for symmetric pairs of a diagonal core).
    __host__ __device__ inline void mma16_rowcol(int bd, int idx, int &row, int &col)
    {
        const int ns = 2 * bd, nb = ns * (ns - 1) / 2;
        if (idx < nb * 256)
        {
            int blk = idx >> 8, R = 0;
            while (blk >= ns - 1 - R)
            {
                blk -= ns - 1 - R;
                ++R;
            }
            const int S = R + 1 + blk;
            const int core = (idx & 255) >> 6, e = idx & 63;
            row = 16 * R + (core & 1) * 8 + (e >> 3);
            col = 16 * S + (core >> 1) * 8 + (e & 7);
            return;
        }
        const int d = idx - nb * 256, R = d / 192, e = d % 192;
        int i, j;
        if (e < 64)
            i = e >> 3, j = e & 7;
        else if (e < 128)
            i = (e - 64) >> 3, j = 8 + ((e - 64) & 7);
        else
            i = 8 + ((e - 128) >> 3), j = 8 + ((e - 128) & 7);
        row = 16 * R + (i < j ? i : j);
        col = 16 * R + (i < j ? j : i);
    }

    // Values stored per subdomain matrix for a storage precision.
    __host__ __device__ inline int inv_stride(int bd, int storage)
    {
        return storage == STORE_F16 ? mma16_size(bd) : tile_packed_size(bd);
    }

    // Position of element (row, col) in mma16 storage (either triangle).
    __host__ __device__ inline int mma16_index(int bd, int row, int col)
    {
        const int ns = 2 * bd;
        int R = row >> 4, S = col >> 4, i = row & 15, j = col & 15;
        if (R > S)
        {
            int t = R;
            R = S;
            S = t;
            t = i;
            i = j;
            j = t;
        }
        if (R < S)
        {
            const int blk = R * (2 * ns - R - 1) / 2 + (S - R - 1);
            const int core = (i >> 3) + 2 * (j >> 3);
            return blk * 256 + core * 64 + (i & 7) * 8 + (j & 7);
        }
        const int base = ns * (ns - 1) / 2 * 256 + R * 192;
        if (i < 8 && j < 8)
            return base + i * 8 + j;
        if (i >= 8 && j >= 8)
            return base + 128 + (i - 8) * 8 + (j - 8);
        const int a = i < j ? i : j, b = i < j ? j : i; // a < 8 <= b
        return base + 64 + a * 8 + (b - 8);
    }

    // ---------------------------------------------------------------------------------------
    // MAS preconditioner on the device.
    // ---------------------------------------------------------------------------------------
    struct MasView
    {
        int bd;
        int banks;              // level-0 matrices
        int level_num;          // coarse levels in use (0..4)
        int total_coarse;       // coarse matrices (all levels >= 1)
        int coff[MAX_COARSE];   // first coarse node of each coarse level
        int mat_offsets[LEVELS];      // first matrix of each matrix level (0 = banks)
        int mat_counts[LEVELS];
        int cco_nums[MAX_COARSE];
        int storage;            // STORE_F64 / STORE_F32 / STORE_F16
        // Banks >= first_iso_bank hold only isolated rows (no off-diagonal block). Such a row is its
        // own component at every level with coarse block A_uu, so z_u = (1 + level_num) z0_u and the
        // coarse levels can skip it: only components < real_count[l] and the coarse matrices in
        // coarse_active are processed.
        int first_iso_bank;
        int real_count[MAX_COARSE];
        int n_coarse_active;
        const int *coarse_active;
        const void *inv;        // total_mats * tile_packed_size(bd): double, float or binary16
        const double *inv_scale; // total_mats: value = stored value * inv_scale (1 unless FP16)
        const int *lcco0;       // nodes: bank-local level-0 component id, -1 virtual
        const int *cco0_base;   // banks: first global level-0 component id of the bank
        const int4 *cslot;      // nodes: coarse-vector node of each coarse level (-1 unused)
        const int *parent;      // coarse nodes: the next level's coarse node it merges into (-1: none)
        unsigned *ticket;       // arrival counter of the coarse-level kernel (zero between launches)
        // Children of each real coarse node of levels 1..3 (local ids of the level below, in
        // increasing order, at most 32): node i of level l has kids[kid_ptr[l][i] .. [i + 1]).
        const int *kid_ptr[MAX_COARSE]; // [1..3] used
        const int *kids;
        const int *identity;    // coarse matrices: 1 if the inverse is exactly the identity
        double *rc;             // coarse residual, coarse nodes * bd (level-0 components first)
        double *zc;             // coarse correction, coarse nodes * bd
    };

    // Device-resident PCG state; all scalars of the reference (MASSolver.cu:178-183) plus control.
    struct PcgState
    {
        double rz, rz_old, pAp, alpha, beta, rr, rr0, rz0, res_norm, rzold_cross;
        double rz_coarse, rzx_coarse; // rc . zc and rc . zc_old of the coarse levels
        int iter;      // last finished iteration
        int done;      // 1: converged / stopped; kernels return immediately
        int status;    // MAS_STATUS_*
        int error;     // device-detected error code (ERR_NONFINITE, ERR_TIMEOUT)
        // x += alpha p runs in update_p (which reads p anyway) except on true-residual iterations:
        // update_xr records the iteration it left the update for (x_defer; -1: none), update_p does
        // it when x_defer is the finished iteration and x_applied is not, and the next SpMV p.Ap
        // records x_applied = x_defer, so a replayed chunk after the stop never adds it twice.
        int x_defer, x_applied;
        // Arrival tickets of the grid reductions: [0] SpMV p.Ap / initial residual, [1] update_xr,
        // [2] in-loop true residual, [4] MAS apply. The last CTA resets its ticket to zero.
        unsigned int counter[8];
    };

    // Default iteration limit of a bounded device-side wait (an mbarrier wait of a bulk copy).
    constexpr long long MBAR_SPIN_LIMIT_DEFAULT = 1LL << 20;

    struct PcgConfig
    {
        int max_iter;
        double rel_tol, abs_tol;
        int use_prec_norm;
        int check_period;
        int polak_ribiere;
        int level_num; // coarse levels in use (isolated rows: z = (1 + level_num) z0)
        long long wait_limit; // iterations of each bounded device-side wait before ERR_TIMEOUT
    };

    // Scratch of the deterministic two-stage reductions: every CTA writes its partial sums, the
    // last CTA to arrive (atomic ticket) adds them in a fixed order.
    struct ReduceBuf
    {
        double *partials; // 2 * capacity: SpMV p.Ap (and b.b on the initial residual)
        int capacity;     // max CTAs of any reduced launch
        double *rr_parts; // capacity: r.r from the kernel that produced r this iteration
        double *rz_parts; // 6 * capacity: the MAS apply's dots (r.z0, r.z0_old, the same over
                          // isolated banks, rc.zc, rc.zc_old)
    };

    // ---------------------------------------------------------------------------------------
    // Fused batch (mas_solve_batch): one launch per PCG phase serves every system of a batch.
    // System s owns the CTAs [start[s], start[s + 1]) of a phase's launch and runs them as CTAs
    // 0 .. start[s + 1] - start[s] - 1 of the launch it would get alone, through the same kernel
    // body, so each system's iterates are those of its own solve bit for bit.
    // ---------------------------------------------------------------------------------------
    struct BatchSystem
    {
        BankedView A;
        MasView mas;
        PcgConfig cfg;
        ReduceBuf red;
        PcgState *st;
        double *x, *r, *p, *z, *Ap;
        const double *b;
    };

    enum BatchPhase : int
    {
        BPH_SPMV = 0,
        BPH_UPDATE_XR,
        BPH_RESTRICT,
        BPH_COARSE,
        BPH_APPLY,
        BPH_UPDATE_P,
        BPH_COUNT
    };

    // The systems of a batched launch: CTA b of phase ph serves system e.x of sys as CTA e.y of
    // the e.z CTAs of that system's own launch, e = map[off[ph] + b] (one load per CTA). Only
    // unfinished systems get entries; the state reset and gather launches take every system
    // (map unused, count = all).
    struct BatchView
    {
        const BatchSystem *sys; // every system of the batch (device memory)
        const int4 *map;        // the phases' CTA entries (device memory)
        int off[BPH_COUNT];     // first entry of each phase
        int count;              // systems (state reset and gather)
    };

    // ---------------------------------------------------------------------------------------
    // Launchers (defined in the .cu files). All take the solver's stream.
    // ---------------------------------------------------------------------------------------

    // mas_bsr.cu: CSC (device) -> banked matrix. padded_of_block[V] maps old block rows to
    // padded nodes. Allocates the outputs. scatter[k] = value index of CSC entry k.
    struct BankedMatrix
    {
        int bd = 0, banks = 0, nodes = 0;
        long long slots = 0;
        int nnzb = 0;
        DevBuf<long long> slice;
        DevBuf<int> rowlen;
        DevBuf<int> cols;
        DevBuf<double> vals;
        DevBuf<long long> scatter; // per CSC entry
        long long pad_index[3] = {-1, -1, -1}; // value slots padded with 1.0 (trailing block)
        int npad = 0;
        BankedView view() const
        {
            return BankedView{bd, banks, slice.get(), rowlen.get(), cols.get(), vals.get()};
        }
    };

    void build_banked(BankedMatrix &M, int n, long long nnz, const int *d_outer, const int *d_inner,
                      const double *d_vals, int bd, int V, int banks, const int *d_padded_of_block,
                      cudaStream_t s);
    void rescatter_values(BankedMatrix &M, long long nnz, const double *d_vals, cudaStream_t s);

    // Programmatic dependent launch of the single-right-hand-side PCG kernels (SpMV, update_xr,
    // restrict, coarse levels, MAS apply, update_p): each may become resident while its
    // predecessor drains. On by default; per calling thread (mas_pcg.cu).
    void set_chained_launch(bool on);
    bool chained_launch();
    // Slots per loop trip of the single-right-hand-side SpMV (1, 2 or 4); per calling thread.
    void set_spmv_unroll(int u);
    int spmv_unroll();
    // Minimum items per warp of the single-right-hand-side MAS apply of the calling thread (its
    // grid: min(SMs, items / (warps per CTA * this))); the apply_items_per_warp parameter.
    void set_apply_items_per_warp(int k);
    int apply_items_per_warp();

    // mas_spmv.cu
    enum SpmvMode : int
    {
        SPMV_PLAIN = 0,    // y = A x
        SPMV_PAP = 1,      // y = A p ; pAp = p . y ; alpha = rz / pAp
        SPMV_RESIDUAL = 2, // y = b - A x ; rr = y . y (iter 0: also rr0 = b . b)
    };
    // period > 0 (SPMV_RESIDUAL in the PCG loop): runs only when (st->iter + 1) % period == 0.
    void launch_spmv(int mode, const BankedView &A, const double *x, double *y, const double *b, PcgState *st,
                     ReduceBuf red, int iter, int period, cudaStream_t s);
    // CTAs of one system's SpMV launch; the batched SpMV (mode SPMV_PAP or SPMV_RESIDUAL) over
    // `total` CTAs with the spmv_unroll variant of the calling thread.
    int spmv_grid(const BankedView &A);
    void launch_spmv_batch(int mode, const BatchView &v, int bd, int total, int iter, int period, cudaStream_t s);
    // y_v = A x_v for count (1..4) separate vectors in one pass over A.
    constexpr int SPMV_MAX_VECTORS = 4;
    void launch_spmv_vectors(const BankedView &A, const double *const *x, double *const *y, int count, cudaStream_t s);

    // mas_pcg.cu
    // x += alpha p; unless this iteration recomputes the true residual ((st->iter + 1) % period == 0):
    // r -= alpha Ap, rr = r . r and the level-0 restriction of r into rc.
    void launch_update_xr(const MasView &mas, double *x, double *r, const double *p, const double *Ap, PcgState *st,
                          ReduceBuf red, int period, cudaStream_t s);
    // x += alpha p (deferred from update_xr, see PcgState::x_defer); p = z0 + prolongation(zc) + beta p
    // (z0: level-0 part of z = M^-1 r)
    void launch_update_p(const MasView &mas, double *x, double *p, const double *z0, PcgState *st, int first,
                         cudaStream_t s);
    void launch_permute_in(int n, int bd, int V, const int *padded_of_block, const double *src, double *dst,
                           size_t dst_len, cudaStream_t s);
    void launch_permute_out(int n, int bd, int V, const int *padded_of_block, const double *src, double *dst,
                            cudaStream_t s);
    void launch_pcg_init_state(PcgState *st, cudaStream_t s);
    // Grids of one system's update launches, and the batched launches (every system's state
    // reset to zero by launch_init_states_batch, one CTA per system).
    int update_xr_grid(const MasView &mas);
    int update_p_grid(const MasView &mas);
    void launch_update_xr_batch(const BatchView &v, int bd, int total, int period, cudaStream_t s);
    void launch_update_p_batch(const BatchView &v, int bd, int total, int first, cudaStream_t s);
    void launch_init_states_batch(const BatchView &v, cudaStream_t s);
    void launch_gather_states_batch(const BatchView &v, PcgState *out, cudaStream_t s);

    // mas_apply.cu: the MAS apply. The coarse residual rc is built by the level-0 restriction
    // (fused into update_xr, or launch_restrict) and launch_coarse_levels; launch_mas_apply then
    // multiplies every inverse.
    // Level-0 restriction of r into rc (with period > 0: only on true-residual iterations);
    // returns the number of kernels launched.
    int launch_restrict(const MasView &mas, const double *r, const PcgState *st, int period, cudaStream_t s);
    // Coarse levels >= 2 summed from the first coarse level; returns the number of kernels launched.
    int launch_coarse_levels(const MasView &mas, const PcgState *st, cudaStream_t s);
    // z0 = A_0^-1 r and zc = A_l^-1 rc for all coarse levels (rc must be complete); mode 1 / 2 also
    // run the PCG scalar step in the last CTA (1: initial apply, 2: iteration).
    void launch_mas_apply(const MasView &mas, const double *r, double *z0, PcgState *st, ReduceBuf red,
                          PcgConfig cfg, int mode, cudaStream_t s);
    void launch_prolong(const MasView &mas, const double *z0, double *z, cudaStream_t s);
    // Grids of one system's restrict, coarse-level and apply launches (0: none), and the
    // batched launches (mode 1 / 2 applies only).
    int restrict_grid(const MasView &mas);
    int coarse_levels_grid(const MasView &mas);
    int mas_apply_grid(const MasView &mas);
    void launch_restrict_batch(const BatchView &v, int bd, int total, int period, cudaStream_t s);
    void launch_coarse_levels_batch(const BatchView &v, int bd, int total, cudaStream_t s);
    void launch_mas_apply_batch(const BatchView &v, int bd, int storage, int total, int mode, cudaStream_t s);

    // Several right-hand sides (groups of RHS_GROUP, interleaved vectors, state array of
    // RHS_GROUP + 1 entries: one per right-hand side, then the group record). mas_multi.cu and
    // mas_apply.cu; the MAS apply needs binary16 inverses.
    void launch_spmv_g(int mode, const BankedView &A, const double *x, double *y, const double *b, PcgState *st,
                       ReduceBuf red, int iter, int period, cudaStream_t s);
    void launch_update_xr_g(const MasView &mas, double *x, double *r, const double *p, const double *Ap,
                            PcgState *st, ReduceBuf red, int period, cudaStream_t s);
    void launch_update_p_g(const MasView &mas, double *x, double *p, const double *z0, PcgState *st, int first,
                           cudaStream_t s);
    int launch_restrict_g(const MasView &mas, const double *r, const PcgState *grp, int period, cudaStream_t s);
    int launch_coarse_levels_g(const MasView &mas, cudaStream_t s);
    void launch_mas_apply_g(const MasView &mas, const double *r, double *z0, PcgState *st, ReduceBuf red,
                            PcgConfig cfg, int mode, cudaStream_t s);
    void prepare_kernels_g(int bd);
    void launch_permute_in_g(int n, int bd, int V, int cols, const int *padded_of_block, const double *B, double *dst,
                             size_t dst_len, cudaStream_t s);
    void launch_permute_out_g(int n, int bd, int cols, const int *padded_of_block, const double *src, double *X,
                              cudaStream_t s);
    // The same group kernels for RHS_WIDE right-hand sides (block size 3, binary16 inverses only):
    // mas_multi16.cu (SpMV, vector updates, restriction, permutations) and mas_apply.cu (coarse levels,
    // MAS apply). Vectors interleaved as above with G = RHS_WIDE; state array of RHS_WIDE + 1 entries.
    // Reductions: red.partials holds 2 RHS_WIDE, red.rr_parts RHS_WIDE and red.rz_parts 3 RHS_WIDE
    // values per CTA of wide_reduce_ctas() CTAs at most.
    constexpr int RHS_WIDE = 16;
    int wide_reduce_ctas();
    void launch_spmv_w(int mode, const BankedView &A, const double *x, double *y, const double *b, PcgState *st,
                       ReduceBuf red, int iter, int period, cudaStream_t s);
    void launch_update_xr_w(const MasView &mas, double *x, double *r, const double *p, const double *Ap,
                            PcgState *st, ReduceBuf red, int period, cudaStream_t s);
    void launch_update_p_w(const MasView &mas, double *x, double *p, const double *z0, PcgState *st, int first,
                           cudaStream_t s);
    int launch_restrict_w(const MasView &mas, const double *r, const PcgState *grp, int period, cudaStream_t s);
    int launch_coarse_levels_w(const MasView &mas, const PcgState *grp, cudaStream_t s);
    void launch_mas_apply_w(const MasView &mas, const double *r, double *z0, PcgState *st, ReduceBuf red,
                            PcgConfig cfg, int mode, cudaStream_t s);
    // The same on the fifth-generation tensor cores (tcgen05.mma, accumulator in tensor memory) from
    // the "tc" storage of the inverses (full binary16 matrices in the canonical operand layout),
    // built from the mma16 storage by launch_inv_to_tc into tc_storage_bytes(mas) bytes.
    size_t tc_storage_bytes(const MasView &mas);
    void launch_inv_to_tc(const MasView &mas, void *out, cudaStream_t s);
    void launch_mas_apply_tc(const MasView &mas, const void *inv_tc, const double *r, double *z, PcgState *st,
                             ReduceBuf red, PcgConfig cfg, int mode, cudaStream_t s);
    void launch_permute_in_w(int n, int V, int cols, const int *padded_of_block, const double *B, double *dst,
                             size_t dst_len, cudaStream_t s);
    void launch_permute_out_w(int n, int cols, const int *padded_of_block, const double *src, double *X,
                              cudaStream_t s);
    void prepare_kernels_w();
    // Set kernel attributes (large shared memory) for every variant used with this block size and
    // precision, so launches inside a CUDA graph capture never touch function attributes.
    void prepare_kernels(int bd, int storage);
    int device_sm_count();

    // mas_build.cu: the MAS hierarchy and inverses.
    struct MasDevice
    {
        int bd = 0, banks = 0, nodes = 0;
        int level_num = 0;
        int cco_nums[MAX_COARSE] = {0, 0, 0, 0};
        int mat_counts[LEVELS] = {0, 0, 0, 0, 0};
        int mat_offsets[LEVELS] = {0, 0, 0, 0, 0};
        int total_mats = 0, total_coarse = 0;
        int coarse_nodes = 0;
        int storage = STORE_F32;
        DevBuf<int> node_real;   // nodes: 1 if the node is a real block row
        DevBuf<int> map;         // nodes * 4
        DevBuf<int> lcco0;
        DevBuf<int> cco0_base;
        DevBuf<int4> cslot;
        DevBuf<int> parent, identity;
        DevBuf<unsigned> ticket;
        DevBuf<int> kid_ptr_all, kids; // kid_ptr of levels 1..3 back to back
        int kid_ptr_off[MAX_COARSE] = {0, 0, 0, 0};
        int first_iso_bank = 0;
        int real_count[MAX_COARSE] = {0, 0, 0, 0};
        DevBuf<int> coarse_active;
        int n_coarse_active = 0;
        int coff[MAX_COARSE] = {0, 0, 0, 0};
        DevBuf<float> inv32;
        DevBuf<double> inv64;
        DevBuf<uint16_t> inv16;  // IEEE binary16 bits
        DevBuf<double> inv_scale;
        DevBuf<double> rc, zc;
        DevBuf<int> flag;        // device error flag for the inverses
        // Deterministic coarse assembly (pattern-dependent, built once per coarse space): at
        // coarse level l, the blocks of the Galerkin operator S_l over coupled pairs (a <= b) of
        // level-l nodes (global coarse ids), each the fixed-order sum of its sources (records):
        // level 0 from the fine blocks of A, level l + 1 from the level-l pairs via the parents.
        struct CoarseSum
        {
            DevBuf<long long> src; // records sorted by target: source index << 2 | rule
            DevBuf<int> ptr;       // targets + 1 record offsets
            DevBuf<int2> pair;     // (a, b) of each target
            DevBuf<double> vals;   // targets * bd * bd block values (refreshed with the values)
            int targets = 0;
            long long records = 0;
        };
        CoarseSum csum[MAX_COARSE];
        DevBuf<double> staging;  // coarse matrices before inversion (kept across refreshes)
        // GPU time of the last assembly + inversion: level 0, coarse sums, coarse inverses (ms).
        float inverse_ms[3] = {0.f, 0.f, 0.f};
        cudaEvent_t inv_ev[4] = {nullptr, nullptr, nullptr, nullptr};
        ~MasDevice()
        {
            for (cudaEvent_t &e : inv_ev)
                if (e)
                    cudaEventDestroy(e);
        }
        MasView view(double *rc_override = nullptr, double *zc_override = nullptr) const;
    };

    // first_iso_bank: first bank of the trailing isolated rows (banks if none / not trailing).
    void build_mas(MasDevice &M, const BankedMatrix &A, const int *d_node_real, int storage, int first_iso_bank,
                   cudaStream_t s);
    // Same pattern, new values: re-assemble and re-invert only (the coarse space is kept).
    void refresh_mas_values(MasDevice &M, const BankedMatrix &A, const int *d_node_real, int storage, cudaStream_t s);

    // mas_pcg.cu: misc
    void launch_zero(double *p, size_t n, cudaStream_t s);

    // ---------------------------------------------------------------------------------------
    // mas_warmstart.cu: the learned starting guess for a sequence of systems (same pattern):
    // x_g, the energy-minimising combination of the kept solutions x1 .. x4 (as x1 and the
    // differences x_i - x_(i+1)); a message-passing network over the vertex graph predicts a
    // correction c of x_g from its residual, the diagonal blocks and the last step; x0 is the
    // energy-minimising combination of the same basis and c, x1 if that is not lower. Block size
    // 3 only.
    // ---------------------------------------------------------------------------------------
    constexpr int WS_FEATURES = 16, WS_HIDDEN = 64, WS_LAYERS = 3;
    constexpr int WS_PARAMS = WS_HIDDEN * WS_FEATURES + WS_HIDDEN +
                              WS_LAYERS * (WS_HIDDEN * 2 * WS_HIDDEN + WS_HIDDEN) + 3 * WS_HIDDEN + 3;
    constexpr int WS_LAYER_WEIGHTS = WS_HIDDEN * 2 * WS_HIDDEN; // bf16 values of one W_l
    constexpr int WS_HISTORY = 4;              // kept solutions x1 (newest) .. x4
    constexpr int WS_BASIS = WS_HISTORY + 1;   // x1, x1 - x2, x2 - x3, x3 - x4, c
    constexpr int WS_GRAM = WS_BASIS * (WS_BASIS + 1) / 2 + WS_BASIS;

    struct WsState
    {
        double sums[5];       // sum over real vertices of |q|^2, |v|^2, |p|^2, log trace, count
        double gram[WS_GRAM]; // v_i . A v_j (i <= j, row by row), then v_i . b
        double coef[WS_BASIS]; // x0 = sum_i coef_i v_i
        double energy, energy_prev; // 1/2 x.Ax - x.b of x0 and of x1
        int fallback;    // 1: x0 = x1 (the combination was degenerate or not lower)
        int rank;        // basis vectors kept by the Galerkin solve
        unsigned counter[2];
        double coef_hist[WS_BASIS]; // x_g = sum_i coef_hist_i v_i (the basis without c)
    };

    // The kept solutions (newest first) and their products with the current A; a missing one
    // repeats the oldest present, so its difference is zero and the Galerkin solve drops it.
    struct WsHistory
    {
        const double *x[WS_HISTORY];
        const double *y[WS_HISTORY];
    };

    struct WsBuffers
    {
        const float *params;   // WS_PARAMS float32 (the .psws layout)
        const uint16_t *wl;    // WS_LAYERS * WS_LAYER_WEIGHTS bf16 bits of the W_l
        int *diag_slot;        // nodes: slot of the diagonal block in the node's row (-1: none)
        float *wslot;          // slots * 32: neighbour weight of each stored block
        float *feat;           // nodes * WS_FEATURES raw features
        uint16_t *h[2];        // nodes * WS_HIDDEN bf16 hidden states (ping-pong)
        double *c, *yc;        // correction and A c (padded order, nodes * 3)
        double *rg;            // b - A x_g, the residual the network's features start from
        WsState *st;
        double *partials;      // WS_GRAM * capacity
        int capacity;          // CTAs of the reduced launches
    };

    // Neighbour weights and diagonal slots of the current values (once per factorization).
    void launch_ws_graph(const BankedView &A, const WsBuffers &w, cudaStream_t s);
    // x_g's residual (Galerkin over the kept solutions only) into w.rg, then features ..
    // correction c (needs hist.y = A x_i). Returns kernels.
    int launch_ws_network(const BankedView &A, const WsBuffers &w, const double *b, const WsHistory &hist,
                          size_t len, cudaStream_t s);
    // Galerkin combination into x (needs w.yc = A c). Returns kernels.
    int launch_ws_combine(const WsBuffers &w, const double *b, const WsHistory &hist, double *x, size_t len,
                          cudaStream_t s);
    int ws_reduce_ctas();
    // Features of the vertices in caller order (tests): out[v * 16 + f] = feat[padded[v] * 16 + f].
    void launch_ws_features_out(int V, const int *padded_of_block, const float *feat, float *out, cudaStream_t s);

    // ---------------------------------------------------------------------------------------
    // mas_ws_train.cu: training of the warm start's network on the GPU (forward, reverse pass,
    // Adam). A sample is stored in the solver's padded block order: the banked pattern of its
    // sequence plus its own values, weights, features, r_g and scalars (s_q, e . r_g).
    // ---------------------------------------------------------------------------------------
    struct WsTrainState
    {
        double a, q;        // c . r_g and c . A c
        double rho, loss;   // rho = a^2 / (q e.r_g), loss = 1 - rho
        double kr, ka;      // dL/dc = kr r_g + ka A c
        unsigned counter[2];
    };

    struct WsTrainView
    {
        int banks;
        const long long *slice;
        const int *rowlen;
        const int *cols;
        const int *diag_slot;
        const uint8_t *real;   // nodes: 1 for the network's vertices (a row with a diagonal block)
        const float *vals32;   // slots * 288: block values [slot][q][lane]
        const float *wslot;    // slots * 32: neighbour weight w_ij of row i's entry for j
        const float *wT;       // slots * 32: the mirrored weight w_ji of the same entry
        const float *feat;     // nodes * 16 normalised features
        const double *re;      // nodes * 3: r_g
        const double *sc;      // [0] s_q, [1] e . r_g
    };

    struct WsTrainScratch
    {
        float *z0;                      // nodes * 64 input-layer pre-activation
        float *z[WS_LAYERS];            // layer pre-activations
        uint16_t *h[WS_LAYERS + 1];     // bf16 hidden states h0 .. h3
        uint16_t *m[WS_LAYERS];         // bf16 messages
        double *c, *Ac;                 // nodes * 3
        float *gh, *g1, *gm;            // nodes * 64 gradients
        float *partials;                // ctas * WS_PARAMS
        double *red;                    // reduction scratch of the loss
        WsTrainState *st;
    };

    int ws_train_ctas(int nodes);
    // Mirror map and real-vertex mask of a pattern (mirror: slots * 32 ints).
    void launch_tr_pattern(const BankedView &A, const int *diag_slot, long long slots, int *mirror, uint8_t *real,
                           cudaStream_t s);
    // One sample from the solver's prediction buffers (features, r_g, WsState after the first
    // Galerkin pass) and the exact solution; writes the sample's arrays and sc = {s_q, e . r_g}.
    void launch_tr_sample(const BankedView &A, long long slots, const int *mirror, const uint8_t *real,
                          const float *wslot, const float *feat_raw, const WsState *ws, const double *rg,
                          const WsHistory &hist, const double *x_exact, size_t len, float *vals32, float *wslot_out,
                          float *wT, float *feat, double *re, double *sc, double *partials, unsigned *counter,
                          int capacity, cudaStream_t s);
    // Forward pass and loss (into scratch.st); returns the kernels launched.
    int launch_tr_forward(const WsTrainView &S, const float *prm, const uint16_t *wl, const WsTrainScratch &w,
                          cudaStream_t s);
    // Reverse pass after launch_tr_forward: the gradient of the loss (WS_PARAMS floats).
    int launch_tr_backward(const WsTrainView &S, const float *prm, const uint16_t *wl, const WsTrainScratch &w,
                           float *grad, cudaStream_t s);
    void launch_tr_adam(float *prm, float *m, float *v, const float *grad, uint16_t *wl, float lr, long long step,
                        cudaStream_t s);
    void launch_tr_weights_bf16(const float *prm, uint16_t *wl, cudaStream_t s);
    // First pass of the prediction only (x_g, r_g, raw features and their sums; no network).
    int launch_ws_features(const BankedView &A, const WsBuffers &w, const double *b, const WsHistory &hist,
                           size_t len, cudaStream_t s);

    // mas_noalloc.cu: y = A x and *dot = x . y with the reduction scratch in a static device array
    // (no allocation). Throws Error(ERR_INVALID) beyond noalloc_max_banks() banks.
    void launch_spmv_dot_noalloc(const BankedView &A, const double *x, double *y, double *dot, cudaStream_t s);
    int noalloc_max_banks();
} // namespace pmas
