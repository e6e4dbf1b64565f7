// sigma without any device allocation in the call.
//
// risqgpu_sigma stages the caller's vector through cudaMalloc'd buffers: the
// caller-order x is permuted into the library's internal (sorted) order, H is
// applied, and the result is permuted back.  Some callers cannot have a library
// allocate device memory on their behalf: a host code whose own pool allocator
// owns the device memory budget, or a solver loop that overlaps work on several
// streams and cannot afford the device-wide synchronisation that cudaFree
// implies on every Davidson iteration.  risqgpu_sigma_noalloc does the same work
// with both permuted vectors held in one file-scope device array of fixed size,
// so the call itself allocates nothing: the caller passes device pointers for x
// and y, and the matrix was allocated earlier, by risqgpu_build_h.
#include <mutex>

#include "internal.cuh"

namespace risq {

// Largest determinant set the call accepts: both internal-order vectors
// (2 x 2^20 doubles, 16 MiB) fit the array.  Every GPU that loads the library
// holds this array until the process exits.
constexpr int64_t kNoAllocMaxDets = (int64_t)1 << 20;

}  // namespace risq

static __device__ __align__(256) double g_sigma_scratch[2 * risq::kNoAllocMaxDets];

namespace risq {

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// The array's device address, looked up once per device with that device
// current.  In host code the symbol name is only a host-side stand-in, so the
// address must come from cudaGetSymbolAddress before any kernel receives it.
int scratch_address(risqgpu* h, double** out) {
    if (h->device < 0 || h->device >= kMaxDevices) {
        h->err = "device index out of range for the no-alloc scratch table";
        return RISQGPU_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[h->device]) {
        double* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**)&p, g_sigma_scratch);
        if (e != cudaSuccess) {
            h->err = std::string("cudaGetSymbolAddress(g_sigma_scratch): ") + cudaGetErrorString(e);
            return RISQGPU_ERR_CUDA;
        }
        g_scratch_ptr[h->device] = p;
    }
    *out = g_scratch_ptr[h->device];
    return RISQGPU_OK;
}

}  // namespace

}  // namespace risq

using namespace risq;

extern "C" int risqgpu_sigma_noalloc(risqgpu_t* h, const double* x_dev, double* y_dev) {
    if (!h || !x_dev || !y_dev) return RISQGPU_ERR_INVALID;
    if (!h->built) {
        h->err = "sigma before build";
        return RISQGPU_ERR_INVALID;
    }
    const int64_t n = (int64_t)h->N;
    if (n > kNoAllocMaxDets) {
        h->err = "risqgpu_sigma_noalloc accepts at most " + std::to_string(kNoAllocMaxDets) +
                 " determinants (fixed scratch array); this set has " + std::to_string(n);
        return RISQGPU_ERR_CAPACITY;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != h->device) {
        const cudaError_t e = cudaSetDevice(h->device);
        if (e != cudaSuccess) {
            h->err = std::string("cudaSetDevice(") + std::to_string(h->device) + "): " + cudaGetErrorString(e);
            return RISQGPU_ERR_CUDA;
        }
    }
    double* scratch = nullptr;
    int rc = scratch_address(h, &scratch);
    if (rc == RISQGPU_OK) {
        // both halves are written in full before they are read, so nothing is cleared;
        // x is copied into the first half before y is written, so x_dev may equal y_dev
        double* xi = scratch;
        double* yi = scratch + kNoAllocMaxDets;
        rc = permute_in(h, x_dev, xi);
        if (rc == RISQGPU_OK) rc = sigma_device(h, xi, yi, 0);
        if (rc == RISQGPU_OK) rc = permute_out(h, yi, y_dev);
        if (rc == RISQGPU_OK) rc = sync(h, "sigma_noalloc");
    }
    if (prev >= 0 && prev != h->device) cudaSetDevice(prev);
    return rc;
}
