// noalloc.cu -- sphere fill fractions without any device allocation.
//
// fdtd_b200_sphere_fractions_noalloc computes exactly what the sphere
// rasteriser's kernel computes for one box of cells, but its device-side
// output staging is a file-scope __device__ array instead of memory obtained
// from cudaMalloc.  It exists for callers that cannot allocate device memory
// at the moment they need the fractions: a host thread that builds scenes
// while another thread of the same process is capturing a CUDA graph (an
// allocation there would invalidate the capture), a real-time loop that must
// never enter the allocator, or a process whose device memory is owned by a
// pool allocator of another framework.
//
// Work is issued on a stream of this file's own, created non-blocking, so it
// never synchronises with the legacy default stream (and through it with a
// stream another thread is capturing), and the results come back with
// asynchronous copies on that stream followed by a wait on that stream only.
#include <cuda_runtime.h>

#include <mutex>

#include "engine.h"

// The fill-fraction kernel of the sphere rasteriser (defined in engine.cu).
__global__ void k_sphere_fractions(double cx, double cy, double cz, double r, int i0, int j0, int k0, int ni, int nj,
                                   int nk, double *f, double *n2);

// Staging for one call: fractions in [0, MAX), squared normals in [MAX, 2 MAX).
// 2^20 samples per array, 16 MiB in all, resident on every GPU that loads
// the library until the process exits.
#define RFB_NOALLOC_MAX_SAMPLES (1u << 20)
static __device__ __align__(256) double g_sphere_scratch[2 * (size_t)RFB_NOALLOC_MAX_SAMPLES];

// Per device, looked up once with that device current: the staging array's
// device address (the host-side name is only a stand-in, not an address) and
// the non-blocking stream the calls run on.
#define RFB_NOALLOC_MAX_DEVICES 64
namespace {
struct NoallocDevice {
    double *scratch = nullptr;
    cudaStream_t stream = nullptr;
};
std::mutex g_setup_mu;
NoallocDevice g_dev[RFB_NOALLOC_MAX_DEVICES];
}  // namespace

static const NoallocDevice *setup_current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= RFB_NOALLOC_MAX_DEVICES) {
        rfb_set_error("fdtd_b200_sphere_fractions_noalloc: no usable current CUDA device");
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    NoallocDevice &d = g_dev[dev];
    if (!d.scratch) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sphere_scratch);
        if (e != cudaSuccess || !p) {
            rfb_set_error("fdtd_b200_sphere_fractions_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return nullptr;
        }
        d.scratch = (double *)p;
    }
    if (!d.stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            d.stream = nullptr;
            rfb_set_error("fdtd_b200_sphere_fractions_noalloc: stream creation failed: %s", cudaGetErrorString(e));
            return nullptr;
        }
    }
    return &d;
}

extern "C" int fdtd_b200_sphere_fractions_noalloc(const double centre[3], double radius, int i0, int j0, int k0,
                                                  int ni, int nj, int nk, double *f, double *n2) {
    if (!centre || !f || !n2 || ni <= 0 || nj <= 0 || nk <= 0) {
        rfb_set_error("fdtd_b200_sphere_fractions_noalloc: NULL pointer or empty box");
        return -1;
    }
    const unsigned long long n = 3ull * (unsigned long long)ni * (unsigned long long)nj * (unsigned long long)nk;
    if (n > RFB_NOALLOC_MAX_SAMPLES) {
        rfb_set_error("fdtd_b200_sphere_fractions_noalloc: box of %llu samples exceeds the maximum of %u",
                      n, (unsigned)RFB_NOALLOC_MAX_SAMPLES);
        return -1;
    }
    const NoallocDevice *d = setup_current_device();
    if (!d) return -1;
    double *sf = d->scratch, *sn = d->scratch + RFB_NOALLOC_MAX_SAMPLES;
    // This thread's capture mode becomes thread-local for the call: a graph
    // capture another thread runs in the global mode then ignores the call's
    // copies (to pageable host memory) and its wait, which touch only this
    // file's own stream; the caller's mode is restored before returning.
    cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    cudaError_t e = cudaThreadExchangeStreamCaptureMode(&mode);
    if (e != cudaSuccess) {
        rfb_set_error("fdtd_b200_sphere_fractions_noalloc: %s", cudaGetErrorString(e));
        return -1;
    }
    // every one of the n samples of both arrays is written by the kernel, so
    // nothing left by an earlier call needs clearing
    k_sphere_fractions<<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>(centre[0], centre[1], centre[2], radius,
                                                                           i0, j0, k0, ni, nj, nk, sf, sn);
    e = cudaGetLastError();
    if (e == cudaSuccess) rfb_count_launch();
    if (e == cudaSuccess) e = cudaMemcpyAsync(f, sf, n * sizeof(double), cudaMemcpyDeviceToHost, d->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(n2, sn, n * sizeof(double), cudaMemcpyDeviceToHost, d->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    cudaThreadExchangeStreamCaptureMode(&mode);
    if (e != cudaSuccess) {
        rfb_set_error("fdtd_b200_sphere_fractions_noalloc: %s", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}
