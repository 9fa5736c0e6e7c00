// noalloc.cu -- an eo scalar product that allocates no device memory.
//
// Who needs it: callers that must not allocate device memory themselves or
// let a library do it behind their back -- an application whose memory pool
// owns all of the GPU's free memory (a cudaMalloc would fail or fragment it),
// a time-critical loop that cannot afford the implicit device-wide
// synchronisation cudaMalloc/cudaFree can cause, or a host program that bans
// allocation by plugins.  Such a caller owns its input and output buffers and
// passes raw device pointers.
//
// The reduction needs scratch (one partial sum per block and the last-block
// ticket).  Here that scratch is a file-scope device array of fixed size,
// loaded with the library: every GPU that loads the library holds these
// 256 KiB (plus 256 bytes) until the process exits.  Host code cannot use the array's name as a
// device address, so on the first call on each device the entry point looks
// up the array's device address with cudaGetSymbolAddress (with that device
// current) and passes it to the kernel.  That first call therefore does extra
// set-up work and should be made before any stream capture starts.
//
// All calls share the one array and it keeps the last call's contents: the
// ticket is cleared on the caller's stream before each launch, and calls
// whose work overlaps on the GPU (different streams, or several host threads
// on one device) race on the array and give wrong results.
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/cl2qcd_b200.h"
#include "blas.cuh"

namespace {

constexpr int NOALLOC_MAX_BLOCKS = C2Q_NOALLOC_MAX_SITES / c2q::BLAS_THREADS;

// [0, 256): the last-block ticket (first 4 bytes); then 2 doubles per block.
constexpr size_t SCRATCH_TICKET_BYTES = 256;
constexpr size_t SCRATCH_BYTES        = SCRATCH_TICKET_BYTES + (size_t)NOALLOC_MAX_BLOCKS * 2 * sizeof(double);

static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[MAX_DEVICES] = {};

// Device address of the scratch array on the current device (looked up once per device).
int scratch_address(void** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return C2Q_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p        = nullptr;
        cudaError_t e  = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "c2q_scalar_product_eo_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                    cudaGetErrorString(e));
            return C2Q_CUDA_ERROR;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return C2Q_OK;
}

}  // namespace

extern "C" {

C2Q_EXPORT int c2q_scalar_product_eo_noalloc(const void* x_soa, const void* y_soa, int n_sites, int stride,
                                             double* result_dev, void* cuda_stream)
{
    if (!x_soa || !y_soa || !result_dev || n_sites <= 0 || stride < n_sites) return C2Q_BAD_ARG;
    // the kernel reads the fields as double2 and writes two doubles: refuse
    // pointers it could not use (a misaligned view) before anything launches
    if ((((uintptr_t)x_soa | (uintptr_t)y_soa) & 15u) || ((uintptr_t)result_dev & 7u)) {
        fprintf(stderr, "c2q_scalar_product_eo_noalloc: x and y must be 16-byte aligned, result 8-byte aligned\n");
        return C2Q_BAD_ARG;
    }
    if (n_sites > C2Q_NOALLOC_MAX_SITES) {
        fprintf(stderr,
                "c2q_scalar_product_eo_noalloc: %d sites exceed the fixed scratch of this entry point "
                "(at most %d eo sites); use c2q_scalar_product for larger fields\n",
                n_sites, C2Q_NOALLOC_MAX_SITES);
        return C2Q_BAD_ARG;
    }
    void* scratch = nullptr;
    int rc        = scratch_address(&scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    // the ticket must start at zero for every launch
    if (cudaMemsetAsync(scratch, 0, sizeof(unsigned), s) != cudaSuccess) return C2Q_CUDA_ERROR;

    c2q::BlasArgs<64> A{};
    A.x            = c2q::SpinorPtr<64>{const_cast<void*>(x_soa), nullptr};
    A.y            = c2q::SpinorPtr<64>{const_cast<void*>(y_soa), nullptr};
    A.n            = n_sites;
    A.stride       = stride;
    A.dot          = 1;  // sum conj(x) y, no field written
    A.red.ticket   = static_cast<unsigned*>(scratch);
    A.red.partials = reinterpret_cast<double*>(static_cast<unsigned char*>(scratch) + SCRATCH_TICKET_BYTES);
    A.red.result   = result_dev;
    A.red.sc       = nullptr;
    A.red.fin      = c2q::FIN_STORE_RESULT;
    const int blocks = (n_sites + c2q::BLAS_THREADS - 1) / c2q::BLAS_THREADS;
    c2q::blas_kernel<64><<<blocks, c2q::BLAS_THREADS, 0, s>>>(A);
    return cudaGetLastError() == cudaSuccess ? C2Q_OK : C2Q_CUDA_ERROR;
}

}  // extern "C"
