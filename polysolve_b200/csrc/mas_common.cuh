// Device helpers shared by the MAS-PCG kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "mas_internal.h"

namespace pmas
{
    constexpr unsigned FULL = 0xFFFFFFFFu;

    // ---------------------------------------------------------------------------------------
    // Programmatic dependent launch. The PCG iteration kernels are launched with programmatic
    // stream serialization (launch_chained): such a kernel may become resident while its
    // predecessor in the stream drains, so it calls pdl_wait() before it reads or writes anything
    // that the predecessor (or any earlier kernel) touches. pdl_wait() returns once the
    // predecessor grid has completed and its writes are visible, and at once for a kernel
    // launched without the attribute. pdl_release() lets the successor start launching once every
    // CTA of this grid has called it or exited; it does not make any write visible early.
    // ---------------------------------------------------------------------------------------
    __device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
    __device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

    // Launch `kernel` in stream order; with chained = true it may overlap the predecessor's tail
    // (the kernel must start with pdl_wait()). Works under stream capture (programmatic edges).
    template <class... P, class... A>
    void launch_chained(bool chained, void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                        A &&...args)
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = chained ? 1 : 0;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cuda_check(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...), "kernel launch");
    }

    // Inverse storage types: the arithmetic type of each and loads of one / four consecutive
    // stored values converted to it. Binary16 values are read as IEEE bits (the buffers are
    // uint16_t on the host) and multiplied in FP32.
    template <class Store>
    struct StoreTraits;
    template <>
    struct StoreTraits<double>
    {
        using Real = double;
        static constexpr bool SCALED = false;
    };
    template <>
    struct StoreTraits<float>
    {
        using Real = float;
        static constexpr bool SCALED = false;
    };
    template <>
    struct StoreTraits<__half>
    {
        using Real = float;
        static constexpr bool SCALED = true;
    };

    __device__ __forceinline__ double4 load4(const double *p) { return *reinterpret_cast<const double4 *>(p); }
    __device__ __forceinline__ float4 load4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
    __device__ __forceinline__ float4 load4(const __half *p)
    {
        const uint2 u = *reinterpret_cast<const uint2 *>(p);
        const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    __device__ __forceinline__ double load1(const double *p) { return *p; }
    __device__ __forceinline__ float load1(const float *p) { return *p; }
    __device__ __forceinline__ float load1(const __half *p) { return __half2float(*p); }

    __device__ __forceinline__ double warp_sum(double v)
    {
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1)
            v += __shfl_xor_sync(FULL, v, o);
        return v;
    }

    __device__ __forceinline__ float warp_sum(float v)
    {
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1)
            v += __shfl_xor_sync(FULL, v, o);
        return v;
    }

    // Deterministic CTA-wide sum; the result is valid in thread 0. Every thread must call it.
    template <int THREADS>
    __device__ __forceinline__ double block_sum(double v)
    {
        __shared__ double sh[THREADS / 32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        v = warp_sum(v);
        __syncthreads();
        if (lane == 0)
            sh[w] = v;
        __syncthreads();
        double t = 0.0;
        if (threadIdx.x == 0)
            for (int i = 0; i < THREADS / 32; ++i)
                t += sh[i];
        return t;
    }

    // A CTA's place in the grid that serves one system: the hardware grid of a launch for one
    // system, or the range of a batched launch's grid that serves one system of the batch. The
    // kernel bodies index work and reduction partials by it, so both launches give the same bits.
    struct Cta
    {
        int x; // index within the system's grid
        int n; // CTAs serving the system
    };

    __device__ __forceinline__ Cta native_cta() { return Cta{(int)blockIdx.x, (int)gridDim.x}; }

    // The system (x) and CTA coordinates (y of z) that this CTA of a batched launch serves in
    // phase ph.
    __device__ __forceinline__ int4 batch_entry(const BatchView &v, int ph)
    {
        return __ldg(v.map + v.off[ph] + blockIdx.x);
    }

    // Deterministic grid-wide sum of NV values per CTA: every CTA writes its block sum to
    // partials[cta.x * NV + i]; the last CTA to arrive (atomic ticket) adds the partials in a
    // fixed order. Returns true in the last CTA, with tot[] the totals (valid in all its
    // threads). Every thread of every CTA must call it.
    template <int NV, int THREADS>
    __device__ __forceinline__ bool grid_reduce(double (&v)[NV], double *partials, unsigned *counter, double (&tot)[NV],
                                                Cta cta)
    {
        constexpr int W = THREADS / 32;
        __shared__ double sh[W][NV];
        __shared__ int is_last;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
        for (int i = 0; i < NV; ++i)
            v[i] = warp_sum(v[i]);
        if (lane == 0)
#pragma unroll
            for (int i = 0; i < NV; ++i)
                sh[w][i] = v[i];
        __syncthreads();
        if (threadIdx.x == 0)
        {
#pragma unroll
            for (int i = 0; i < NV; ++i)
            {
                double s = 0.0;
                for (int ww = 0; ww < W; ++ww)
                    s += sh[ww][i];
                partials[(size_t)cta.x * NV + i] = s;
            }
            __threadfence();
            unsigned t = atomicAdd(counter, 1u);
            is_last = (t == (unsigned)cta.n - 1);
        }
        __syncthreads();
        if (!is_last)
            return false;
        __threadfence();
        double s[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i)
        {
            s[i] = 0.0;
            for (int b = threadIdx.x; b < cta.n; b += THREADS)
                s[i] += __ldcg(partials + (size_t)b * NV + i);
            s[i] = warp_sum(s[i]);
        }
        __syncthreads();
        if (lane == 0)
#pragma unroll
            for (int i = 0; i < NV; ++i)
                sh[w][i] = s[i];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < NV; ++i)
        {
            double t = 0.0;
            for (int ww = 0; ww < W; ++ww)
                t += sh[ww][i];
            tot[i] = t;
        }
        if (threadIdx.x == 0)
            *counter = 0u;
        return true;
    }

    template <int NV, int THREADS>
    __device__ __forceinline__ bool grid_reduce(double (&v)[NV], double *partials, unsigned *counter, double (&tot)[NV])
    {
        return grid_reduce<NV, THREADS>(v, partials, counter, tot, native_cta());
    }

    // Deterministic grid-wide sum of NV values per CTA already summed into shared memory (vals, NV
    // doubles, written before the call by the CTA; every thread must call it). Each CTA writes its
    // row of partials; the last CTA to arrive (atomic ticket) sums the rows in a fixed order: THREADS /
    // NV thread groups take strided subsets of the CTAs, then thread i adds the groups' sums of value i
    // in group order. Returns true in the last CTA, with tot (shared memory, NV doubles) filled.
    template <int NV, int THREADS>
    __device__ __forceinline__ bool grid_reduce_cta(const double *vals, double *partials, unsigned *counter,
                                                    double *tot)
    {
        static_assert(NV <= THREADS, "one thread per value at least");
        constexpr int GROUPS = THREADS / NV;
        __shared__ double gsum[GROUPS][NV];
        __shared__ int is_last;
        __syncthreads();
        for (int i = threadIdx.x; i < NV; i += THREADS)
            partials[(size_t)blockIdx.x * NV + i] = vals[i];
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0)
            is_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
        __syncthreads();
        if (!is_last)
            return false;
        __threadfence();
        const int i = threadIdx.x % NV, grp = threadIdx.x / NV;
        if (grp < GROUPS)
        {
            double s = 0.0;
            for (int c = grp; c < (int)gridDim.x; c += GROUPS)
                s += __ldcg(partials + (size_t)c * NV + i);
            gsum[grp][i] = s;
        }
        __syncthreads();
        if (threadIdx.x < NV)
        {
            double t = 0.0;
            for (int g = 0; g < GROUPS; ++g)
                t += gsum[g][threadIdx.x];
            tot[threadIdx.x] = t;
        }
        __syncthreads();
        if (threadIdx.x == 0)
            *counter = 0u;
        return true;
    }

    // Sum of a per-lane value over the lanes whose key equals each distinct key of the warp,
    // written by lane 0 of each group to out[(base + key) * BD + i]. Keys < 0 are skipped.
    // Order of additions is fixed (xor butterfly), so results are deterministic.
    // Keys held by a single lane (e.g. isolated rows, one component each) are stored directly.
    template <int BD>
    __device__ __forceinline__ void warp_segment_store(const double (&val)[BD], int key, int base, double *out)
    {
        const int lane = threadIdx.x & 31;
        const unsigned group = __match_any_sync(FULL, key);
        const bool single = (group == (1u << lane));
        if (single && key >= 0)
#pragma unroll
            for (int i = 0; i < BD; ++i)
                out[(size_t)(base + key) * BD + i] = val[i];
        unsigned pending = __ballot_sync(FULL, key >= 0 && !single);
        while (pending)
        {
            const int leader = __ffs(pending) - 1;
            const int k = __shfl_sync(FULL, key, leader);
            const bool in = (key == k);
#pragma unroll
            for (int i = 0; i < BD; ++i)
            {
                double s = warp_sum(in ? val[i] : 0.0);
                if (lane == 0)
                    out[(size_t)(base + k) * BD + i] = s;
            }
            pending &= ~__ballot_sync(FULL, in);
        }
    }

    // Level-0 restriction of one bank: reg[t] holds the bank's values t * 32 + lane (coalesced
    // layout); the values are regrouped by node with shuffles and summed per connected component
    // of the bank into rc (first coarse level). Every lane of the warp must call it.
    // key = lcco0[bank * 32 + lane], base = cco0_base[bank], loaded by the caller (ahead of time).
    template <int BD>
    __device__ __forceinline__ void bank_restrict_keyed(const double (&reg)[BD], int key, int base, double *rc)
    {
        const int lane = threadIdx.x & 31;
        double rv[BD];
#pragma unroll
        for (int i = 0; i < BD; ++i)
        {
            const int e = lane * BD + i; // this lane's node, component i
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
        warp_segment_store<BD>(rv, key, base, rc);
    }

    template <int BD>
    __device__ __forceinline__ void bank_restrict(const double (&reg)[BD], int bank, const int *__restrict__ lcco0,
                                                  const int *__restrict__ cco0_base, double *rc)
    {
        const int lane = threadIdx.x & 31;
        bank_restrict_keyed<BD>(reg, lcco0[(long long)bank * 32 + lane], cco0_base[bank], rc);
    }

    // ---------------------------------------------------------------------------------------
    // mbarrier + bulk copy (cp.async.bulk, the 1D TMA path) with bounded waits.
    // ---------------------------------------------------------------------------------------
    __device__ __forceinline__ uint32_t smem_addr(const void *p)
    {
        return static_cast<uint32_t>(__cvta_generic_to_shared(p));
    }

    __device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    }

    __device__ __forceinline__ void fence_mbar_init()
    {
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }

    __device__ __forceinline__ void fence_proxy_async_smem()
    {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }

    // Arm the barrier for `bytes` and start a global -> shared bulk copy completing on it.
    // dst, src and bytes must be 16-byte aligned / multiples of 16.
    __device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
    {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_addr(dst)),
            "l"(src), "r"(bytes), "r"(smem_addr(bar))
            : "memory");
    }

    // ---------------------------------------------------------------------------------------
    // L2 residency: the matrices stream through once per iteration (hundreds of MB), the PCG
    // vectors (13 MB each at 1.6 M DOF) are re-read by every kernel. Streams are loaded with
    // evict-first priority so the vectors stay in the 126 MB L2.
    // ---------------------------------------------------------------------------------------
    __device__ __forceinline__ uint64_t l2_evict_first_policy()
    {
        uint64_t pol;
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
        return pol;
    }

    __device__ __forceinline__ void bulk_load_stream(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                                     uint64_t policy)
    {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], "
                     "%2, [%3], %4;" ::"r"(smem_addr(dst)),
                     "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
                     : "memory");
    }

    // Arm a barrier for `bytes` of transactions (one arrival), then issue copies completing on it.
    __device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
    {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                     : "memory");
    }

    // Global -> shared bulk copy completing on `bar` (armed separately); 16-byte aligned, multiple of 16.
    __device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
    {
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(dst)),
                     "l"(src), "r"(bytes), "r"(smem_addr(bar))
                     : "memory");
    }

    __device__ __forceinline__ void bulk_copy_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                                       uint64_t policy)
    {
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], "
                     "%2, [%3], %4;" ::"r"(smem_addr(dst)),
                     "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
                     : "memory");
    }

    // ---------------------------------------------------------------------------------------
    // Fifth-generation tensor cores (tcgen05): tensor-memory allocation, MMA with both operands in
    // shared memory, completion through an mbarrier, and loads of the accumulator.
    // ---------------------------------------------------------------------------------------
    // Allocate `cols` (power of two >= 32) tensor-memory columns; warp-wide. The address lands in
    // *slot (shared memory).
    __device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t cols)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                     "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }

    __device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols)
    {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
    }

    __device__ __forceinline__ void tc_fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
    __device__ __forceinline__ void tc_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

    // Shared-memory matrix descriptor, no swizzle: core matrices of 8 rows x 16 bytes (rows 16 bytes
    // apart); lbo = bytes between the two 8-element halves of a 16-element K step, sbo = bytes
    // between consecutive 8-row groups along M (or N). Version field 1 (bit 46).
    __device__ __forceinline__ uint64_t tc_smem_desc(const void *p, uint32_t lbo, uint32_t sbo)
    {
        const uint32_t a = smem_addr(p);
        return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
               ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
    }

    // Instruction descriptor of kind::f16: binary16 A and B (both K-major), FP32 accumulator, M x N.
    __host__ __device__ constexpr uint32_t tc_idesc_f16_f32(int m, int n)
    {
        return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
    }

    // D (tensor memory) = A B^T (+ D when accumulate); issued by one thread.
    __device__ __forceinline__ void tc_mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                               bool accumulate)
    {
        const uint32_t acc = accumulate ? 1u : 0u, zero = 0u;
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d_tmem),
                     "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(zero)
                     : "memory");
    }

    // Arrive on `bar` once every MMA issued so far by this thread has completed.
    __device__ __forceinline__ void tc_commit(uint64_t *bar)
    {
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(bar))
                     : "memory");
    }

    // 16 consecutive FP32 columns of this thread's tensor-memory lane (warp w reads lanes
    // 32 (w % 4) ..); completes at tc_wait_ld().
    __device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16])
    {
        uint32_t r[16];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                     "%12, %13, %14, %15}, [%16];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                       "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                       "=r"(r[14]), "=r"(r[15])
                     : "r"(taddr)
                     : "memory");
#pragma unroll
        for (int i = 0; i < 16; ++i)
            v[i] = __uint_as_float(r[i]);
    }

    __device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

    __device__ __forceinline__ double2 ld_stream_f64x2(const double *p, uint64_t pol)
    {
        double2 v;
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                     : "=d"(v.x), "=d"(v.y)
                     : "l"(p), "l"(pol));
        return v;
    }

    __device__ __forceinline__ double ld_stream_f64(const double *p, uint64_t pol)
    {
        double v;
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
        return v;
    }

    __device__ __forceinline__ int ld_stream_s32(const int *p, uint64_t pol)
    {
        int v;
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
        return v;
    }

    // Asynchronous global -> shared copies (cp.async, completion tracked per thread by commit / wait
    // groups): 16 bytes cached in L1 and L2 (.ca) or in L2 only (.cg), and 8 bytes (.ca).
    __device__ __forceinline__ void cp_async16_ca(void *dst, const void *src)
    {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
    }

    __device__ __forceinline__ void cp_async16_cg(void *dst, const void *src)
    {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
    }

    __device__ __forceinline__ void cp_async8_ca(void *dst, const void *src)
    {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
    }

    __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

    template <int N>
    __device__ __forceinline__ void cp_async_wait()
    {
        asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
    }

    __device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
    {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        return ok != 0;
    }

    // Default iteration limit of a bounded device-side wait (PcgConfig::wait_limit; the solver
    // parameter device_wait_limit lowers it, down to 0 = give up at once, to test the timeout path).
    constexpr long long MBAR_SPIN_LIMIT = MBAR_SPIN_LIMIT_DEFAULT;

    // Wait for phase `parity` of the barrier with an iteration limit; warp-collective (all 32 lanes
    // call it and get the same answer: the phase counts as complete only when every lane saw it,
    // so every lane has acquired the copied data). On timeout records ERR_TIMEOUT in *err and
    // returns false.
    __device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *err,
                                                      long long limit = MBAR_SPIN_LIMIT)
    {
        for (long long i = 0; i < limit; ++i)
            if (__all_sync(FULL, mbar_try_wait(bar, parity)))
                return true;
        if (err && (threadIdx.x & 31) == 0)
            atomicExch(err, ERR_TIMEOUT);
        return false;
    }

    // After a wait gave up: wait (bounded by the default limit, whatever the caller's limit was)
    // for the copies this warp still has in flight, so none lands in shared memory after the CTA
    // has left. pending[s]: a copy was issued to stage s and not consumed; phase[s]: its parity.
    // Called by lane 0.
    __device__ __forceinline__ void mbar_drain(uint64_t *bar, const bool (&pending)[2], const uint32_t (&phase)[2])
    {
#pragma unroll
        for (int s = 0; s < 2; ++s)
            if (pending[s])
                for (long long i = 0; i < MBAR_SPIN_LIMIT; ++i)
                    if (mbar_try_wait(&bar[s], phase[s]))
                        break;
    }
} // namespace pmas
