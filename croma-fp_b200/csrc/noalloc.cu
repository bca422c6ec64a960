// noalloc.cu -- the batched implicit Chang-Cooper step without any device
// allocation.
//
// solve_cc_cuda_batch (ref_abi.cu) copies host arrays into device buffers it
// allocates for each call.  Some callers cannot allow that: a host code that
// has already handed the device's memory to its own pool allocator (a second
// allocator would fail or fragment it), a time step that must not call
// cudaMalloc/cudaFree because those can synchronise the whole device and stall
// the caller's other streams, or a caller whose memory budget is fixed before
// the run starts.  solve_cc_cuda_batch_noalloc serves them: the caller passes
// device pointers for every input and output, and the only scratch the solve
// needs -- the Thomas c' coefficients, one double per row -- lives in
// g_noalloc_scratch below, a fixed array that is part of this library's
// device image.
//
// Limits and sharing:
//   * nsys * nrow must not exceed kNoallocMaxRows (524,288 rows, 4 MiB of
//     scratch); larger batches are rejected with -1 and a message.
//   * Every GPU that loads this library holds the array until the process
//     exits.
//   * All calls on a device share the one array and it keeps whatever the
//     last call left there.  The c' values are written before they are read,
//     and the error word at its head is cleared at the start of every call.
//     Two calls whose kernels overlap on the GPU (different streams, or
//     different host threads) race on the array and corrupt each other's
//     results: serialise them, e.g. on one stream.
//   * The first call on each device looks the array's device address up with
//     cudaGetSymbolAddress (with that device current) and caches it.  The
//     stream must belong to the current device (checked: -1 otherwise); a
//     cudaDeviceReset on a device ends the cached address's validity, so the
//     library is not used on that device after one.
//   * The call waits for its stream to finish the solve so that it can report
//     a singular pivot (-2); a stream that is being captured is refused (-1)
//     before anything is launched, since the wait would break the capture.
#include <mutex>

#include "croma_ctx.cuh"

namespace croma {
namespace {

constexpr size_t kNoallocMaxRows = (size_t)1 << 19;
constexpr size_t kNoallocHead = 32;   // doubles reserved at the front: error word

// The library's only allocation-free scratch: [head | c' of nsys * nrow rows].
static __device__ __align__(256) double g_noalloc_scratch[kNoallocHead + kNoallocMaxRows];

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_lock;

// Device address of the scratch array for the current device (looked up
// once per device).
cudaError_t scratch_address(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_scratch_lock);
    if (!g_scratch_addr[dev]) {
        double *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

// One implicit step per system: x_out = M^{-1} (x_in + dt * src), M the CC
// matrix b_i x_i - a_i x_{i-1} - c_i x_{i+1}; fp_thomas_solve_ws with the RHS
// of solve_cc_batch_cpu_timed (src/fp_shared_core.c:226-257, 564-615).
// Layout [nsys][nrow]; scratch = error word at [0], c' from [kNoallocHead].
__global__ void cc_thomas_scratch_kernel(int nsys, int nrow, double dt, const double *a, const double *b,
                                         const double *c, const double *src, const double *x_in,
                                         double *x_out, double *scratch)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    unsigned *err = reinterpret_cast<unsigned *>(scratch);
    const size_t o = (size_t)s * nrow;
    double *cp = scratch + kNoallocHead + o;
    double *x = x_out + o;
    if (fabs(b[o]) <= 1.0e-300) { atomicOr(err, kErrSingular); return; }
    cp[0] = -c[o] / b[o];
    x[0] = (dt * src[o] + x_in[o]) / b[o];
    for (int i = 1; i < nrow; i++) {
        const double den = b[o + i] + a[o + i] * cp[i - 1];
        if (fabs(den) <= 1.0e-300) { atomicOr(err, kErrSingular); return; }
        cp[i] = (i == nrow - 1) ? 0.0 : -c[o + i] / den;
        x[i] = ((dt * src[o + i] + x_in[o + i]) + a[o + i] * x[i - 1]) / den;
    }
    for (int i = nrow - 2; i >= 0; i--) x[i] -= cp[i] * x[i + 1];
}

}  // namespace
}  // namespace croma

using namespace croma;

extern "C" int solve_cc_cuda_batch_noalloc(int nsys, int nrow, double dt, const double *a, const double *b,
                                           const double *c, const double *source, const double *state_in,
                                           double *state_out, void *stream)
{
    if (nsys <= 0 || nrow <= 1 || !a || !b || !c || !source || !state_in || !state_out) {
        set_error("solve_cc_cuda_batch_noalloc: invalid arguments");
        return -1;
    }
    if ((size_t)nsys * (size_t)nrow > kNoallocMaxRows) {
        set_error("solve_cc_cuda_batch_noalloc: nsys * nrow exceeds the fixed scratch of 524288 rows; "
                  "split the batch or use solve_cc_cuda_batch");
        return -1;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CROMA_CUDA(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        set_error("solve_cc_cuda_batch_noalloc: the stream is being captured; the call waits for its stream "
                  "and cannot run inside a capture");
        return -1;
    }
    int cur = 0, sdev = 0;
    CROMA_CUDA(cudaGetDevice(&cur));
    CROMA_CUDA(cudaStreamGetDevice(st, &sdev));
    if (sdev != cur) {
        set_error("solve_cc_cuda_batch_noalloc: the stream belongs to another device than the current one");
        return -1;
    }
    double *scratch = nullptr;
    CROMA_CUDA(scratch_address(&scratch));
    CROMA_CUDA(cudaMemsetAsync(scratch, 0, sizeof(double), st));
    cc_thomas_scratch_kernel<<<(nsys + 127) / 128, 128, 0, st>>>(nsys, nrow, dt, a, b, c, source, state_in,
                                                                  state_out, scratch);
    CROMA_CUDA(cudaGetLastError());
    unsigned err = 0;
    CROMA_CUDA(cudaMemcpyAsync(&err, scratch, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CROMA_CUDA(cudaStreamSynchronize(st));
    if (err) {
        set_error("solve_cc_cuda_batch_noalloc: singular tridiagonal pivot");
        return -2;
    }
    return 0;
}
