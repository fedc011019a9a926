// y = A x and x . y on the factorized block matrix without any device allocation.
//
// Callers that cannot allocate device memory at call time -- code inside a CUDA stream capture
// (where cudaMalloc is not allowed), solvers embedded in applications that reserve all device
// memory up front and treat any later allocation as an error, or real-time loops that cannot afford
// cudaMalloc's implicit synchronization -- still need the fused SpMV + dot of the PCG loop. This
// variant of the banked SpMV keeps its reduction scratch (per-CTA partial sums and the ticket of
// the last CTA) in a file-scope static __device__ array instead of memory the solver allocates.
//
// Limits and rules:
//   * the array holds NOALLOC_MAX_CTAS partials plus one double for the ticket (256 KB + 8 B on
//     every GPU where this module is loaded, held until the process exits): at most
//     NOALLOC_MAX_CTAS * 8 banks, i.e. 262,144
//     banks = 8,388,608 block rows; larger matrices are rejected with an error;
//   * every call shares the array: calls that overlap on the GPU (on different streams, or from
//     different handles on one device) race and must be serialized by the caller;
//   * the ticket is cleared before each launch; the partials need no clearing;
//   * x, y and the dot must be distinct, non-overlapping device buffers (the kernel reads x while
//     other warps write y); overlapping pointers are rejected by the entry point;
//   * the first call on a device looks the array's device address up (cudaGetSymbolAddress with
//     that device current). Under CUDA's lazy module loading (the default) that lookup is also what
//     loads this module onto the device and gives the array its 256 KB of device memory, so the
//     first call must come before any stream capture and before the application reserves the rest
//     of the device's memory;
//   * the address is cached per device together with the id of the CUDA context it was looked up
//     in; after a cudaDeviceReset (a new primary context) the next call looks it up again, which
//     loads the module into the new context -- the same "first call" rule applies then.

#include <cuda.h>

#include <mutex>
#include <string>

#include "mas_common.cuh"

namespace pmas
{
    namespace
    {
        constexpr int NOALLOC_THREADS = 256;
        constexpr int NOALLOC_BANKS_PER_CTA = NOALLOC_THREADS / 32;
        constexpr int NOALLOC_MAX_CTAS = 32768;

        // [0, NOALLOC_MAX_CTAS): per-CTA partial sums; the last slot holds the ticket counter.
        static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_CTAS + 1];

        template <int BD>
        __global__ void __launch_bounds__(NOALLOC_THREADS)
            k_spmv_dot_noalloc(BankedView A, const double *__restrict__ x, double *__restrict__ y, double *dot,
                               double *scratch)
        {
            constexpr int BS = BD * BD;
            constexpr int PAIRS = BS / 2;
            const int lane = threadIdx.x & 31;
            const int bank = blockIdx.x * NOALLOC_BANKS_PER_CTA + (threadIdx.x >> 5);
            double part = 0.0;
            if (bank < A.banks)
            {
                const int u = bank * 32 + lane;
                const long long s0 = A.slice[bank];
                const int len = A.rowlen[u];
                const int *cp = A.cols + s0 * 32 + lane;
                const double *vp = A.vals + s0 * 32 * BS;
                double acc[BD];
#pragma unroll
                for (int i = 0; i < BD; ++i)
                    acc[i] = 0.0;
                for (int k = 0; k < len; ++k)
                {
                    const int col = __ldg(cp + (long long)k * 32);
                    const double *blk = vp + (long long)k * 32 * BS;
                    double v[BS];
#pragma unroll
                    for (int p = 0; p < PAIRS; ++p)
                    {
                        const double2 t = __ldg(reinterpret_cast<const double2 *>(blk + p * 64 + lane * 2));
                        v[2 * p] = t.x;
                        v[2 * p + 1] = t.y;
                    }
                    if (BS & 1)
                        v[BS - 1] = __ldg(blk + PAIRS * 64 + lane);
#pragma unroll
                    for (int i = 0; i < BD; ++i)
#pragma unroll
                        for (int j = 0; j < BD; ++j)
                            acc[i] = fma(v[i * BD + j], __ldg(x + (long long)col * BD + j), acc[i]);
                }
#pragma unroll
                for (int i = 0; i < BD; ++i)
                {
                    y[(long long)u * BD + i] = acc[i];
                    part = fma(acc[i], x[(long long)u * BD + i], part);
                }
            }
            double v1[1] = {part}, tot[1];
            unsigned *ticket = reinterpret_cast<unsigned *>(scratch + NOALLOC_MAX_CTAS);
            if (grid_reduce<1, NOALLOC_THREADS>(v1, scratch, ticket, tot) && threadIdx.x == 0)
                *dot = tot[0];
        }

        // Device address of the scratch array per device, with the id of the context it belongs to.
        constexpr int MAX_DEVICES = 64;
        std::mutex g_lookup_mutex;
        double *g_scratch_addr[MAX_DEVICES] = {nullptr};
        unsigned long long g_scratch_ctx[MAX_DEVICES] = {0};

        // Unique id of the current CUDA context (driver entry points cuCtxGetCurrent / cuCtxGetId,
        // looked up through the runtime); 0 when they are unavailable.
        unsigned long long current_context_id()
        {
            using GetCurrent = CUresult (*)(CUcontext *);
            using GetId = CUresult (*)(CUcontext, unsigned long long *);
            static GetCurrent get_current = nullptr;
            static GetId get_id = nullptr;
            static std::once_flag once;
            std::call_once(once, [] {
                void *f = nullptr;
                cudaDriverEntryPointQueryResult q;
                if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
                    q == cudaDriverEntryPointSuccess)
                    get_current = reinterpret_cast<GetCurrent>(f);
                f = nullptr;
                if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
                    q == cudaDriverEntryPointSuccess)
                    get_id = reinterpret_cast<GetId>(f);
                cudaGetLastError();
            });
            CUcontext ctx = nullptr;
            unsigned long long id = 0;
            if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS)
                return id;
            return 0;
        }
    } // namespace

    int noalloc_max_banks() { return NOALLOC_MAX_CTAS * NOALLOC_BANKS_PER_CTA; }

    void launch_spmv_dot_noalloc(const BankedView &A, const double *x, double *y, double *dot, cudaStream_t s)
    {
        if (A.banks > noalloc_max_banks())
            throw Error(ERR_INVALID, "[MAS] spmv_dot_noalloc: the matrix has " + std::to_string(A.banks) +
                                         " banks; the static scratch supports at most " +
                                         std::to_string(noalloc_max_banks()) + " banks (" +
                                         std::to_string(noalloc_max_banks() * 32) + " block rows).");
        int dev = 0;
        cuda_check(cudaGetDevice(&dev), "get device");
        if (dev < 0 || dev >= MAX_DEVICES)
            throw Error(ERR_INVALID, "[MAS] spmv_dot_noalloc: device index out of range");
        double *scratch = nullptr;
        {
            const unsigned long long ctx = current_context_id();
            std::lock_guard<std::mutex> lock(g_lookup_mutex);
            if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx)
            {
                void *p = nullptr;
                cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "scratch symbol address");
                g_scratch_addr[dev] = static_cast<double *>(p);
                g_scratch_ctx[dev] = ctx;
            }
            scratch = g_scratch_addr[dev];
        }
        const int grid = (A.banks + NOALLOC_BANKS_PER_CTA - 1) / NOALLOC_BANKS_PER_CTA;
        cuda_check(cudaMemsetAsync(scratch + NOALLOC_MAX_CTAS, 0, sizeof(double), s), "clear ticket");
        if (grid == 0)
        {
            cuda_check(cudaMemsetAsync(dot, 0, sizeof(double), s), "clear dot");
            return;
        }
        switch (A.bd)
        {
        case 1:
            k_spmv_dot_noalloc<1><<<grid, NOALLOC_THREADS, 0, s>>>(A, x, y, dot, scratch);
            break;
        case 2:
            k_spmv_dot_noalloc<2><<<grid, NOALLOC_THREADS, 0, s>>>(A, x, y, dot, scratch);
            break;
        default:
            k_spmv_dot_noalloc<3><<<grid, NOALLOC_THREADS, 0, s>>>(A, x, y, dot, scratch);
            break;
        }
        cuda_check(cudaGetLastError(), "spmv_dot_noalloc launch");
    }
} // namespace pmas
