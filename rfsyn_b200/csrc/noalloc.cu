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

// Device address of the staging array, looked up once per device with that
// device current (the host-side name is only a stand-in, not an address).
#define RFB_NOALLOC_MAX_DEVICES 64
static std::mutex g_setup_mu;
static double *g_scratch_addr[RFB_NOALLOC_MAX_DEVICES];

static double *scratch_for_current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= RFB_NOALLOC_MAX_DEVICES) {
        rfb_set_error("fdtd_b200_sphere_fractions_noalloc: no usable current CUDA device");
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sphere_scratch);
        if (e != cudaSuccess || !p) {
            rfb_set_error("fdtd_b200_sphere_fractions_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return nullptr;
        }
        g_scratch_addr[dev] = (double *)p;
    }
    return g_scratch_addr[dev];
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
    double *scratch = scratch_for_current_device();
    if (!scratch) return -1;
    double *sf = scratch, *sn = scratch + RFB_NOALLOC_MAX_SAMPLES;
    // every one of the n samples of both arrays is written by the kernel, so
    // nothing left by an earlier call needs clearing
    k_sphere_fractions<<<(unsigned)((n + 255) / 256), 256>>>(centre[0], centre[1], centre[2], radius, i0, j0, k0, ni,
                                                             nj, nk, sf, sn);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(f, sf, n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(n2, sn, n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        rfb_set_error("fdtd_b200_sphere_fractions_noalloc: %s", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}
